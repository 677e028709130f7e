// Oracle geometry core: vectors, frames, rational Bezier patches and curves in f64.
//
// TEST INFRASTRUCTURE ONLY. This directory is the CPU restatement of the reference's
// exact evaluator that the CUDA library is checked against; nothing in the product
// links it. Every routine names the reference function it restates.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <utility>
#include <vector>

namespace oracle {

constexpr double INF = std::numeric_limits<double>::infinity();
constexpr double PI = 3.14159265358979323846;

struct V3 {
  double x = 0, y = 0, z = 0;
  V3() = default;
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  V3 operator+(V3 o) const { return {x + o.x, y + o.y, z + o.z}; }
  V3 operator-(V3 o) const { return {x - o.x, y - o.y, z - o.z}; }
  V3 operator*(double s) const { return {x * s, y * s, z * s}; }
  V3 operator-() const { return {-x, -y, -z}; }
  double dot(V3 o) const { return x * o.x + y * o.y + z * o.z; }
  V3 cross(V3 o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
  double len() const { return std::sqrt(dot(*this)); }
  V3 unit() const {
    double l = len();
    return l > 0 ? *this * (1.0 / l) : *this;
  }
  double operator[](int k) const { return k == 0 ? x : (k == 1 ? y : z); }
};

using Box = std::pair<V3, V3>;

inline V3 vmin(V3 a, V3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
inline Box empty_box() { return {V3(1e300, 1e300, 1e300), V3(-1e300, -1e300, -1e300)}; }
inline void grow(Box& b, V3 q) {
  b.first = vmin(b.first, q);
  b.second = vmax(b.second, q);
}

// surface3.rs:978 box_dist
inline double box_dist(V3 p, const Box& b) {
  V3 d(std::max(std::max(b.first.x - p.x, p.x - b.second.x), 0.0),
       std::max(std::max(b.first.y - p.y, p.y - b.second.y), 0.0),
       std::max(std::max(b.first.z - p.z, p.z - b.second.z), 0.0));
  return d.len();
}

// curve3.rs:1042 box_gap
inline double box_gap(const Box& a, const Box& b) {
  auto g = [](double l1, double h1, double l2, double h2) { return std::max(std::max(l1 - h2, l2 - h1), 0.0); };
  return V3(g(a.first.x, a.second.x, b.first.x, b.second.x), g(a.first.y, a.second.y, b.first.y, b.second.y),
            g(a.first.z, a.second.z, b.first.z, b.second.z))
      .len();
}

// curve3.rs:40-52 Frame::{local, world, dir}
struct Frame {
  V3 o, z, x;
  V3 y() const { return z.cross(x); }
  V3 local(V3 p) const {
    V3 d = p - o;
    return {d.dot(x), d.dot(y()), d.dot(z)};
  }
  V3 world(V3 l) const { return o + x * l.x + y() * l.y + z * l.z; }
  V3 dir(V3 l) const { return x * l.x + y() * l.y + z * l.z; }
};

using H4 = std::array<double, 4>;

inline V3 hp(const H4& h) { return {h[0] / h[3], h[1] / h[3], h[2] / h[3]}; }

// ---------------------------------------------------------------- Bernstein basis

constexpr int BMAX = 16;

// surface3.rs:207-243 bernstein_small: basis of degree n at t with first and second
// derivatives, from the de Casteljau triangle.
inline void bernstein(int n, double t, double* b, double* d1, double* d2) {
  double cur[BMAX] = {0}, l1[BMAX] = {0}, l2[BMAX] = {0};
  cur[0] = 1.0;
  if (n >= 1 && n - 1 == 0) std::copy(cur, cur + BMAX, l1);
  if (n >= 2 && n - 2 == 0) std::copy(cur, cur + BMAX, l2);
  for (int k = 1; k <= n; k++) {
    for (int i = k; i >= 0; i--) {
      double left = i > 0 ? cur[i - 1] : 0.0;
      double right = i < k ? cur[i] : 0.0;
      cur[i] = (1.0 - t) * right + t * left;
    }
    if (n >= 1 && k == n - 1) std::copy(cur, cur + BMAX, l1);
    if (n >= 2 && k == n - 2) std::copy(cur, cur + BMAX, l2);
  }
  auto get = [](const double* lv, int len, int i) { return (i < 0 || i >= len) ? 0.0 : lv[i]; };
  for (int i = 0; i <= n; i++) {
    d1[i] = n >= 1 ? n * (get(l1, n, i - 1) - get(l1, n, i)) : 0.0;
    d2[i] = n >= 2 ? double(n * (n - 1)) * (get(l2, n - 1, i - 2) - 2.0 * get(l2, n - 1, i - 1) + get(l2, n - 1, i)) : 0.0;
    b[i] = cur[i];
  }
}

// ---------------------------------------------------------------- patches

// surface3.rs:248-256 SEval
struct SEval {
  V3 p, ps, pt, pss, pst, ptt;
};

// surface3.rs:259-266 Patch: a rational Bezier patch, pw[i][j] with i along u.
struct Patch {
  int du = 0, dv = 0;
  std::vector<H4> pw;  // (du+1)*(dv+1), (i, j) at i*(dv+1)+j
  double u0 = 0, u1 = 1, v0 = 0, v1 = 1;
  const H4& at(int i, int j) const { return pw[i * (dv + 1) + j]; }
  H4& at(int i, int j) { return pw[i * (dv + 1) + j]; }

  Box bbox() const {
    Box b = empty_box();
    for (auto& h : pw) grow(b, hp(h));
    return b;
  }

  // surface3.rs:299-325 Patch::eval (eval_small)
  SEval eval(double s, double t) const {
    double bu[BMAX], bu1[BMAX], bu2[BMAX], bv[BMAX], bv1[BMAX], bv2[BMAX];
    bernstein(du, s, bu, bu1, bu2);
    bernstein(dv, t, bv, bv1, bv2);
    double a[6][4] = {{0}};
    for (int i = 0; i <= du; i++)
      for (int j = 0; j <= dv; j++) {
        const H4& h = at(i, j);
        double w[6] = {bu[i] * bv[j], bu1[i] * bv[j], bu[i] * bv1[j], bu2[i] * bv[j], bu1[i] * bv1[j], bu[i] * bv2[j]};
        for (int k = 0; k < 6; k++)
          for (int c = 0; c < 4; c++) a[k][c] += w[k] * h[c];
      }
    auto v3 = [](const double* x) { return V3(x[0], x[1], x[2]); };
    double w = a[0][3];
    SEval e;
    e.p = v3(a[0]) * (1.0 / w);
    e.ps = (v3(a[1]) - e.p * a[1][3]) * (1.0 / w);
    e.pt = (v3(a[2]) - e.p * a[2][3]) * (1.0 / w);
    e.pss = (v3(a[3]) - e.ps * (2.0 * a[1][3]) - e.p * a[3][3]) * (1.0 / w);
    e.pst = (v3(a[4]) - e.ps * a[2][3] - e.pt * a[1][3] - e.p * a[4][3]) * (1.0 / w);
    e.ptt = (v3(a[5]) - e.pt * (2.0 * a[2][3]) - e.p * a[5][3]) * (1.0 / w);
    return e;
  }

  // surface3.rs:351-383 split_u / split_v by de Casteljau
  std::pair<Patch, Patch> split_u(double s) const;
  std::pair<Patch, Patch> split_v(double t) const;
  // surface3.rs:979-985 quarters
  void quarters(Patch out[4]) const {
    auto ab = split_u(0.5);
    auto a = ab.first.split_v(0.5);
    auto b = ab.second.split_v(0.5);
    out[0] = a.first;
    out[1] = a.second;
    out[2] = b.first;
    out[3] = b.second;
  }
  // surface3.rs:401-447 newton_iters
  std::pair<double, double> newton_iters(V3 p, double s, double t, double s0, double s1, double t0, double t1,
                                         int iters) const;
  std::pair<double, double> newton_capped(V3 p, double s, double t, int iters) const {
    return newton_iters(p, s, t, 0.0, 1.0, 0.0, 1.0, iters);
  }
  // surface3.rs:694-730 no_critical_point
  bool no_critical_point(V3 p) const;
};

// surface3.rs:565-572 critical
inline bool critical(V3 p, const SEval& e) {
  V3 r = e.p - p;
  auto big = [](V3 x) { return std::max(std::max(std::fabs(x.x), std::fabs(x.y)), std::fabs(x.z)); };
  double round = 1024.0 * 2.220446049250313e-16 * (big(e.p) + big(p) + r.len());
  auto ok = [&](V3 d) { return std::fabs(r.dot(d)) <= (round + 1e-12 * d.len()) * d.len(); };
  return ok(e.ps) && ok(e.pt);
}

// surface3.rs:973-975 slab_bound
inline double slab_bound(const Patch& pa, V3 p, V3 n) {
  double m = INF;
  for (auto& h : pa.pw) m = std::min(m, (p - hp(h)).dot(n));
  return m;
}

// ---------------------------------------------------------------- curves

// curve3.rs:75-80 Eval3
struct Eval3 {
  V3 p, d1, d2;
};

// curve3.rs:66-72 Bez3: a rational Bezier piece, homogeneous, local s in [0, 1],
// with its parameter range on the source curve.
struct Bez3 {
  std::vector<H4> pw;
  double t0 = 0, t1 = 1;
  int degree() const { return int(pw.size()) - 1; }
  V3 start() const { return hp(pw.front()); }
  V3 end() const { return hp(pw.back()); }
  Eval3 eval(double s) const;
  std::pair<Bez3, Bez3> split(double s) const;
  Bez3 reversed() const {
    Bez3 r = *this;
    std::reverse(r.pw.begin(), r.pw.end());
    r.t0 = t1;
    r.t1 = t0;
    return r;
  }
  double turning() const;
  double thickness() const;
  double newton(V3 p, double s) const;
  Box box() const {
    Box b = empty_box();
    for (auto& h : pw) grow(b, hp(h));
    return b;
  }
};

double seg_dist3(V3 p, V3 a, V3 b);

}  // namespace oracle

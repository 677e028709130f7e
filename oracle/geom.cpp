// Oracle geometry core (f64): patch splitting and Newton, the no-critical-point
// certificate, rational Bezier curves. TEST INFRASTRUCTURE ONLY.
#include "geom.hpp"

namespace oracle {

// surface3.rs:268-285 casteljau_split
static void casteljau_split(std::vector<H4> pts, double s, std::vector<H4>& left, std::vector<H4>& right) {
  int n = int(pts.size()) - 1;
  left.assign(1, pts[0]);
  right.assign(1, pts[n]);
  for (int level = 1; level <= n; level++) {
    for (int i = 0; i <= n - level; i++)
      for (int c = 0; c < 4; c++) pts[i][c] = (1.0 - s) * pts[i][c] + s * pts[i + 1][c];
    left.push_back(pts[0]);
    right.push_back(pts[n - level]);
  }
  std::reverse(right.begin(), right.end());
}

// surface3.rs:351-371 split_u
std::pair<Patch, Patch> Patch::split_u(double s) const {
  Patch l = *this, r = *this;
  std::vector<H4> col(du + 1), a, b;
  for (int j = 0; j <= dv; j++) {
    for (int i = 0; i <= du; i++) col[i] = at(i, j);
    casteljau_split(col, s, a, b);
    for (int i = 0; i <= du; i++) {
      l.at(i, j) = a[i];
      r.at(i, j) = b[i];
    }
  }
  double um = u0 + s * (u1 - u0);
  l.u1 = um;
  r.u0 = um;
  return {l, r};
}

// surface3.rs:372-383 split_v
std::pair<Patch, Patch> Patch::split_v(double t) const {
  Patch l = *this, r = *this;
  std::vector<H4> row(dv + 1), a, b;
  for (int i = 0; i <= du; i++) {
    for (int j = 0; j <= dv; j++) row[j] = at(i, j);
    casteljau_split(row, t, a, b);
    for (int j = 0; j <= dv; j++) {
      l.at(i, j) = a[j];
      r.at(i, j) = b[j];
    }
  }
  double vm = v0 + t * (v1 - v0);
  l.v1 = vm;
  r.v0 = vm;
  return {l, r};
}

// surface3.rs:401-447 newton_iters: Newton on |S - p|^2 with the active-set hold rule.
std::pair<double, double> Patch::newton_iters(V3 p, double s, double t, double s0, double s1, double t0, double t1,
                                              int iters) const {
  bool hold_s = false, hold_t = false;
  for (int it = 0; it < iters; it++) {
    SEval e = eval(s, t);
    V3 r = e.p - p;
    double g0 = e.ps.dot(r), g1 = e.pt.dot(r);
    double jss = e.ps.dot(e.ps), jst = e.ps.dot(e.pt), jtt = e.pt.dot(e.pt);
    double h0 = jss + e.pss.dot(r), h1 = jst + e.pst.dot(r), h2 = jtt + e.ptt.dot(r);
    double ds, dt;
    if (hold_s && hold_t) break;
    if (hold_s) {
      ds = 0.0;
      dt = -g1 / (h2 > 0.0 ? h2 : std::max(jtt, 1e-300));
    } else if (hold_t) {
      ds = -g0 / (h0 > 0.0 ? h0 : std::max(jss, 1e-300));
      dt = 0.0;
    } else {
      if (!(h0 > 0.0 && h0 * h2 - h1 * h1 > 0.0)) {
        h0 = jss;
        h1 = jst;
        h2 = jtt;
      }
      double det = h0 * h2 - h1 * h1;
      if (std::fabs(det) < 1e-300) break;
      ds = -(h2 * g0 - h1 * g1) / det;
      dt = -(h0 * g1 - h1 * g0) / det;
    }
    auto at_bound = [](double x, double d, double lo, double hi) { return (x <= lo && d < 0.0) || (x >= hi && d > 0.0); };
    if (!hold_s && at_bound(s, ds, s0, s1)) {
      hold_s = true;
      continue;
    }
    if (!hold_t && at_bound(t, dt, t0, t1)) {
      hold_t = true;
      continue;
    }
    double ns = std::min(std::max(s + ds, s0), s1), nt = std::min(std::max(t + dt, t0), t1);
    double moved = std::fabs(ns - s) + std::fabs(nt - t);
    s = ns;
    t = nt;
    if (moved < 1e-13) break;
  }
  return {s, t};
}

// ---------------------------------------------------------------- Bern2 (surface3.rs:583-682)

namespace {
struct Bern2 {
  int m, n;
  std::vector<double> c;
  double at(int i, int j) const { return c[i * (n + 1) + j]; }
};

std::vector<double> binomials(int n) {
  std::vector<double> b(n + 1, 1.0);
  for (int k = 1; k <= n; k++) b[k] = b[k - 1] * double(n + 1 - k) / double(k);
  return b;
}

Bern2 bmul(const Bern2& a, const Bern2& o) {
  int m = a.m + o.m, n = a.n + o.n;
  auto ba = binomials(a.m), bb = binomials(a.n), bo = binomials(o.m), bp = binomials(o.n);
  auto bm = binomials(m), bn = binomials(n);
  Bern2 r{m, n, std::vector<double>((m + 1) * (n + 1), 0.0)};
  for (int i = 0; i <= a.m; i++)
    for (int j = 0; j <= a.n; j++) {
      double x = a.c[i * (a.n + 1) + j] * ba[i] * bb[j];
      if (x == 0.0) continue;
      for (int k = 0; k <= o.m; k++)
        for (int l = 0; l <= o.n; l++) r.c[(i + k) * (n + 1) + j + l] += x * o.c[k * (o.n + 1) + l] * bo[k] * bp[l];
    }
  for (int k = 0; k <= m; k++)
    for (int l = 0; l <= n; l++) r.c[k * (n + 1) + l] /= bm[k] * bn[l];
  return r;
}

Bern2 d_u(const Bern2& a) {
  if (a.m == 0) return {0, a.n, std::vector<double>(a.n + 1, 0.0)};
  int n1 = a.n + 1;
  Bern2 r{a.m - 1, a.n, {}};
  for (int i = 0; i < a.m; i++)
    for (int j = 0; j < n1; j++) r.c.push_back(a.m * (a.c[(i + 1) * n1 + j] - a.c[i * n1 + j]));
  return r;
}

Bern2 d_v(const Bern2& a) {
  if (a.n == 0) return {a.m, 0, std::vector<double>(a.m + 1, 0.0)};
  int n1 = a.n + 1;
  Bern2 r{a.m, a.n - 1, {}};
  for (int i = 0; i <= a.m; i++)
    for (int j = 0; j < a.n; j++) r.c.push_back(a.n * (a.c[i * n1 + j + 1] - a.c[i * n1 + j]));
  return r;
}

Bern2 elevate_u(const Bern2& a) {
  int m = a.m + 1, n1 = a.n + 1;
  Bern2 r{m, a.n, std::vector<double>((m + 1) * n1, 0.0)};
  for (int i = 0; i <= m; i++) {
    double x = double(i) / m;
    for (int j = 0; j < n1; j++) {
      double lo = i > 0 ? a.c[(i - 1) * n1 + j] : 0.0;
      double hi = i < m ? a.c[i * n1 + j] : 0.0;
      r.c[i * n1 + j] = x * lo + (1.0 - x) * hi;
    }
  }
  return r;
}

Bern2 elevate_v(const Bern2& a) {
  int n = a.n + 1, n0 = a.n + 1;
  Bern2 r{a.m, n, std::vector<double>((a.m + 1) * (n + 1), 0.0)};
  for (int i = 0; i <= a.m; i++)
    for (int j = 0; j <= n; j++) {
      double x = double(j) / n;
      double lo = j > 0 ? a.c[i * n0 + j - 1] : 0.0;
      double hi = j < n ? a.c[i * n0 + j] : 0.0;
      r.c[i * (n + 1) + j] = x * lo + (1.0 - x) * hi;
    }
  return r;
}

Bern2 axpy(const Bern2& a, double x, const Bern2& o, double y) {
  Bern2 r{a.m, a.n, a.c};
  for (size_t k = 0; k < r.c.size(); k++) r.c[k] = x * a.c[k] + y * o.c[k];
  return r;
}

double max_abs(const Bern2& a) {
  double m = 0.0;
  for (double x : a.c) m = std::max(m, std::fabs(x));
  return m;
}
}  // namespace

// surface3.rs:694-730 Patch::no_critical_point
bool Patch::no_critical_point(V3 p) const {
  int m = du, n = dv;
  auto mk = [&](int comp, bool minus_p) {
    Bern2 b{m, n, {}};
    for (auto& h : pw) {
      double v = h[comp];
      if (minus_p) v = h[comp] - p[comp] * h[3];
      b.c.push_back(v);
    }
    return b;
  };
  Bern2 w = mk(3, false);
  for (double x : w.c)
    if (!(x > 0.0)) return false;
  SEval e = eval(0.5, 0.5);
  V3 r = e.p - p;
  double a = e.ps.dot(r), b = e.pt.dot(r);
  double l = std::hypot(a, b);
  if (!(l > 0.0)) return false;
  a /= l;
  b /= l;
  Bern2 q[3] = {mk(0, true), mk(1, true), mk(2, true)};
  Bern2 qu[3] = {d_u(q[0]), d_u(q[1]), d_u(q[2])};
  Bern2 qv[3] = {d_v(q[0]), d_v(q[1]), d_v(q[2])};
  auto dot = [](const Bern2* x, const Bern2* y) {
    Bern2 s = bmul(x[0], y[0]);
    for (int k = 1; k < 3; k++) s = axpy(s, 1.0, bmul(x[k], y[k]), 1.0);
    return s;
  };
  Bern2 qq = dot(q, q);
  Bern2 wu = d_u(w), wv = d_v(w);
  Bern2 gs = axpy(bmul(w, dot(q, qu)), 1.0, bmul(wu, qq), -1.0);
  Bern2 gt = axpy(bmul(w, dot(q, qv)), 1.0, bmul(wv, qq), -1.0);
  Bern2 f = axpy(elevate_u(gs), a, elevate_v(gt), b);
  auto qmax = [](const Bern2* x) { return std::max(std::max(max_abs(x[0]), max_abs(x[1])), max_abs(x[2])); };
  double q0 = qmax(q), q1 = qmax(qu), q2 = qmax(qv);
  double size = max_abs(w) * 3.0 * q0 * (std::fabs(a) * q1 + std::fabs(b) * q2) +
                (std::fabs(a) * max_abs(wu) + std::fabs(b) * max_abs(wv)) * 3.0 * q0 * q0;
  for (double x : f.c)
    if (!(x > 1e-11 * size)) return false;
  return true;
}

// ---------------------------------------------------------------- curves

// curve3.rs:129-156 Bez3::eval by de Casteljau, derivatives from its levels
Eval3 Bez3::eval(double s) const {
  int n = degree();
  std::vector<H4> b = pw;
  H4 d1h = {0, 0, 0, 0}, d2h = {0, 0, 0, 0};
  for (int level = 1; level <= n; level++) {
    if (n >= 2 && level == n - 1)
      for (int c = 0; c < 4; c++) d2h[c] = double(n * (n - 1)) * (b[2][c] - 2.0 * b[1][c] + b[0][c]);
    if (level == n)
      for (int c = 0; c < 4; c++) d1h[c] = n * (b[1][c] - b[0][c]);
    for (int i = 0; i <= n - level; i++)
      for (int c = 0; c < 4; c++) b[i][c] = (1.0 - s) * b[i][c] + s * b[i + 1][c];
  }
  double w = b[0][3];
  Eval3 e;
  e.p = hp(b[0]);
  e.d1 = (V3(d1h[0], d1h[1], d1h[2]) - e.p * d1h[3]) * (1.0 / w);
  e.d2 = (V3(d2h[0], d2h[1], d2h[2]) - e.d1 * (2.0 * d1h[3]) - e.p * d2h[3]) * (1.0 / w);
  return e;
}

// curve3.rs:157-173 Bez3::split
std::pair<Bez3, Bez3> Bez3::split(double s) const {
  std::vector<H4> l, r;
  casteljau_split(pw, s, l, r);
  double tm = t0 + s * (t1 - t0);
  Bez3 a{l, t0, tm}, b{r, tm, t1};
  return {a, b};
}

// curve3.rs:181-185 turning
double Bez3::turning() const {
  std::vector<V3> legs;
  for (size_t i = 1; i < pw.size(); i++) {
    V3 d = hp(pw[i]) - hp(pw[i - 1]);
    if (d.len() > 1e-14) legs.push_back(d);
  }
  double t = 0.0;
  for (size_t i = 1; i < legs.size(); i++) t += std::atan2(legs[i - 1].cross(legs[i]).len(), legs[i - 1].dot(legs[i]));
  return t;
}

// curve3.rs:205-212 seg_dist3
double seg_dist3(V3 p, V3 a, V3 b) {
  V3 ab = b - a;
  double l2 = ab.dot(ab);
  double t = l2 > 0.0 ? std::min(std::max((p - a).dot(ab) / l2, 0.0), 1.0) : 0.0;
  return (p - (a + ab * t)).len();
}

// curve3.rs:186-190 thickness
double Bez3::thickness() const {
  V3 a = start(), b = end();
  double m = 0.0;
  for (auto& h : pw) m = std::max(m, seg_dist3(hp(h), a, b));
  return m;
}

// curve3.rs:191-213 Bez3::newton
double Bez3::newton(V3 p, double s) const {
  for (int it = 0; it < 40; it++) {
    Eval3 e = eval(s);
    V3 r = e.p - p;
    double f = e.d1.dot(r);
    double fp = e.d2.dot(r) + e.d1.dot(e.d1);
    if (fp <= 0.0) fp = e.d1.dot(e.d1);
    if (std::fabs(fp) < 1e-300) break;
    double ns = std::min(std::max(s - f / fp, 0.0), 1.0);
    if (std::fabs(ns - s) < 1e-15) return ns;
    s = ns;
  }
  return s;
}

}  // namespace oracle

// Host-side geometry for packing: Bezier evaluation and splitting, interval
// derivative bounds (convexity certificates), and the trim-tree builder.
#include "host_geom.h"

#include <algorithm>
#include <limits>

namespace icam {

static void bern3(double t, double b[4], double d[4], double dd[4]) {
  double s = 1.0 - t;
  b[0] = s * s * s;
  b[1] = 3 * s * s * t;
  b[2] = 3 * s * t * t;
  b[3] = t * t * t;
  d[0] = -3 * s * s;
  d[1] = 3 * s * s - 6 * s * t;
  d[2] = 6 * s * t - 3 * t * t;
  d[3] = 3 * t * t;
  dd[0] = 6 * s;
  dd[1] = -12 * s + 6 * t;
  dd[2] = 6 * s - 12 * t;
  dd[3] = 6 * t;
}

void Bicubic::eval(double s, double t, V* P, V* Ps, V* Pt, V* Pss, V* Pst, V* Ptt) const {
  double bu[4], du[4], ddu[4], bv[4], dv[4], ddv[4];
  bern3(s, bu, du, ddu);
  bern3(t, bv, dv, ddv);
  double a[6][4] = {{0}};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double w[6] = {bu[i] * bv[j], du[i] * bv[j], bu[i] * dv[j], ddu[i] * bv[j], du[i] * dv[j], bu[i] * ddv[j]};
      for (int k = 0; k < 6; k++)
        for (int c = 0; c < 4; c++) a[k][c] += w[k] * p[i][j][c];
    }
  auto v = [](const double* x) { return V(x[0], x[1], x[2]); };
  double w = a[0][3];
  V p0 = v(a[0]) * (1 / w);
  V ps = (v(a[1]) - p0 * a[1][3]) * (1 / w);
  V pt = (v(a[2]) - p0 * a[2][3]) * (1 / w);
  if (P) *P = p0;
  if (Ps) *Ps = ps;
  if (Pt) *Pt = pt;
  if (Pss) *Pss = (v(a[3]) - ps * (2 * a[1][3]) - p0 * a[3][3]) * (1 / w);
  if (Pst) *Pst = (v(a[4]) - ps * a[2][3] - pt * a[1][3] - p0 * a[4][3]) * (1 / w);
  if (Ptt) *Ptt = (v(a[5]) - pt * (2 * a[2][3]) - p0 * a[5][3]) * (1 / w);
}

static void split4(const H in[4], double s, H l[4], H r[4]) {
  H b[4] = {in[0], in[1], in[2], in[3]};
  l[0] = b[0];
  r[3] = b[3];
  for (int level = 1; level <= 3; level++) {
    for (int i = 0; i <= 3 - level; i++)
      for (int c = 0; c < 4; c++) b[i][c] = (1 - s) * b[i][c] + s * b[i + 1][c];
    l[level] = b[0];
    r[3 - level] = b[3 - level];
  }
}

void Bicubic::split_u(double s, Bicubic* l, Bicubic* r) const {
  for (int j = 0; j < 4; j++) {
    H col[4] = {p[0][j], p[1][j], p[2][j], p[3][j]}, a[4], b[4];
    split4(col, s, a, b);
    for (int i = 0; i < 4; i++) {
      l->p[i][j] = a[i];
      r->p[i][j] = b[i];
    }
  }
  double um = u0 + s * (u1 - u0);
  l->u0 = u0, l->u1 = um, r->u0 = um, r->u1 = u1;
  l->v0 = r->v0 = v0;
  l->v1 = r->v1 = v1;
}

void Bicubic::split_v(double t, Bicubic* l, Bicubic* r) const {
  for (int i = 0; i < 4; i++) split4(p[i], t, l->p[i], r->p[i]);
  double vm = v0 + t * (v1 - v0);
  l->v0 = v0, l->v1 = vm, r->v0 = vm, r->v1 = v1;
  l->u0 = r->u0 = u0;
  l->u1 = r->u1 = u1;
}

std::vector<H> elevate(const std::vector<H>& q) {
  int n = int(q.size()) - 1;
  std::vector<H> r;
  r.push_back(q[0]);
  for (int i = 1; i <= n; i++) {
    double a = double(i) / (n + 1);
    H h;
    for (int c = 0; c < 4; c++) h[c] = a * q[i - 1][c] + (1 - a) * q[i][c];
    r.push_back(h);
  }
  r.push_back(q[n]);
  return r;
}

// ---------------------------------------------------------------- interval bounds

namespace {
struct Iv {
  double lo, hi;
};
Iv iv_of(const std::vector<double>& xs) {
  Iv r{std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity()};
  for (double x : xs) r = {std::min(r.lo, x), std::max(r.hi, x)};
  return r;
}
Iv add(Iv a, Iv b) { return {a.lo + b.lo, a.hi + b.hi}; }
Iv sub(Iv a, Iv b) { return {a.lo - b.hi, a.hi - b.lo}; }
Iv mul(Iv a, Iv b) {
  double p[4] = {a.lo * b.lo, a.lo * b.hi, a.hi * b.lo, a.hi * b.hi};
  return {*std::min_element(p, p + 4), *std::max_element(p, p + 4)};
}
Iv scale(Iv a, double k) { return k >= 0 ? Iv{a.lo * k, a.hi * k} : Iv{a.hi * k, a.lo * k}; }
Iv divpos(Iv a, Iv w) { return mul(a, Iv{1.0 / w.hi, 1.0 / w.lo}); }
double mig(Iv a) { return (a.lo <= 0 && a.hi >= 0) ? 0.0 : std::min(std::fabs(a.lo), std::fabs(a.hi)); }
double mag(Iv a) { return std::max(std::fabs(a.lo), std::fabs(a.hi)); }
}  // namespace

// surface3.rs:862-925 patch_bounds: hulls of the Bernstein coefficients of the
// homogeneous derivatives relative to the control points' mean, the rational quotient
// rule in interval arithmetic, parameters scaled to unit tangents at the middle, and
// lambda_min(G) from the entries' intervals or by Weyl's inequality from the middle.
bool patch_bounds(const Bicubic& pa, double* sa_out, double* sb_out, double* lam_out, double d2[3][3][2],
                  double* rho) {
  const int du = 3, dv = 3;
  V c;
  for (auto& r : pa.p)
    for (auto& h : r) c = c + hv(h);
  c = c * (1.0 / 16.0);
  auto q = [&](int i, int j) {
    const H& h = pa.p[i][j];
    return H{h[0] - c.x * h[3], h[1] - c.y * h[3], h[2] - c.z * h[3], h[3]};
  };
  auto hull = [&](auto f) {
    std::array<Iv, 4> out;
    for (int k = 0; k < 4; k++) {
      std::vector<double> v;
      for (int i = 0; i <= du; i++)
        for (int j = 0; j <= dv; j++) {
          double x;
          if (f(i, j, k, &x)) v.push_back(x);
        }
      out[k] = v.empty() ? Iv{0, 0} : iv_of(v);
    }
    return out;
  };
  double fu = du, fv = dv;
  auto A = hull([&](int i, int j, int k, double* x) { *x = q(i, j)[k]; return true; });
  auto As = hull([&](int i, int j, int k, double* x) {
    if (i >= du) return false;
    *x = fu * (q(i + 1, j)[k] - q(i, j)[k]);
    return true;
  });
  auto At = hull([&](int i, int j, int k, double* x) {
    if (j >= dv) return false;
    *x = fv * (q(i, j + 1)[k] - q(i, j)[k]);
    return true;
  });
  auto Ass = hull([&](int i, int j, int k, double* x) {
    if (i + 1 >= du) return false;
    *x = fu * (fu - 1) * (q(i + 2, j)[k] - 2 * q(i + 1, j)[k] + q(i, j)[k]);
    return true;
  });
  auto Ast = hull([&](int i, int j, int k, double* x) {
    if (i >= du || j >= dv) return false;
    *x = fu * fv * (q(i + 1, j + 1)[k] - q(i + 1, j)[k] - q(i, j + 1)[k] + q(i, j)[k]);
    return true;
  });
  auto Att = hull([&](int i, int j, int k, double* x) {
    if (j + 1 >= dv) return false;
    *x = fv * (fv - 1) * (q(i, j + 2)[k] - 2 * q(i, j + 1)[k] + q(i, j)[k]);
    return true;
  });
  Iv w = A[3];
  if (!(w.lo > 0)) return false;
  Iv s[3], ss[3], st[3], sss[3], sst[3], stt[3];
  for (int k = 0; k < 3; k++) {
    std::vector<double> xs;
    for (auto& r : pa.p)
      for (auto& h : r) xs.push_back(hv(h)[k] - c[k]);
    s[k] = iv_of(xs);
  }
  for (int k = 0; k < 3; k++) {
    ss[k] = divpos(sub(As[k], mul(s[k], As[3])), w);
    st[k] = divpos(sub(At[k], mul(s[k], At[3])), w);
  }
  for (int k = 0; k < 3; k++) {
    sss[k] = divpos(sub(sub(Ass[k], scale(mul(ss[k], As[3]), 2.0)), mul(s[k], Ass[3])), w);
    sst[k] = divpos(sub(sub(sub(Ast[k], mul(ss[k], At[3])), mul(st[k], As[3])), mul(s[k], Ast[3])), w);
    stt[k] = divpos(sub(sub(Att[k], scale(mul(st[k], At[3]), 2.0)), mul(s[k], Att[3])), w);
  }
  V p0, ps0, pt0;
  pa.eval(0.5, 0.5, &p0, &ps0, &pt0, nullptr, nullptr, nullptr);
  double sa = ps0.len() > 0 ? ps0.len() : 1.0, sb = pt0.len() > 0 ? pt0.len() : 1.0;
  for (int k = 0; k < 3; k++) {
    ss[k] = scale(ss[k], 1 / sa);
    st[k] = scale(st[k], 1 / sb);
    sss[k] = scale(sss[k], 1 / (sa * sa));
    sst[k] = scale(sst[k], 1 / (sa * sb));
    stt[k] = scale(stt[k], 1 / (sb * sb));
  }
  ps0 = ps0 * (1 / sa);
  pt0 = pt0 * (1 / sb);
  double ga = 0, gc = 0;
  for (int k = 0; k < 3; k++) {
    ga += mig(ss[k]) * mig(ss[k]);
    gc += mig(st[k]) * mig(st[k]);
  }
  Iv gbi = add(add(mul(ss[0], st[0]), mul(ss[1], st[1])), mul(ss[2], st[2]));
  double gb = mag(gbi);
  double by_entries = 0.5 * ((ga + gc) - std::sqrt((ga - gc) * (ga - gc) + 4 * gb * gb));
  double a0 = ps0.dot(ps0), b0 = ps0.dot(pt0), c0 = pt0.dot(pt0);
  double sigma0 = std::sqrt(std::max(0.5 * ((a0 + c0) - std::sqrt((a0 - c0) * (a0 - c0) + 4 * b0 * b0)), 0.0));
  double dev = 0;
  for (int k = 0; k < 3; k++) {
    dev += std::pow(std::max(std::fabs(ss[k].lo - ps0[k]), std::fabs(ss[k].hi - ps0[k])), 2);
    dev += std::pow(std::max(std::fabs(st[k].lo - pt0[k]), std::fabs(st[k].hi - pt0[k])), 2);
  }
  double by_middle = std::pow(std::max(sigma0 - std::sqrt(dev), 0.0), 2);
  double lam = std::max(by_entries, by_middle);
  *sa_out = sa;
  *sb_out = sb;
  *lam_out = lam;
  Iv* d[3] = {sss, sst, stt};
  double h2 = 0;
  for (int m = 0; m < 3; m++)
    for (int k = 0; k < 3; k++) {
      d2[m][k][0] = d[m][k].lo;
      d2[m][k][1] = d[m][k].hi;
      h2 += (m == 1 ? 2.0 : 1.0) * mag(d[m][k]) * mag(d[m][k]);
    }
  *rho = lam > 0 ? (h2 > 0 ? 0.99 * lam / std::sqrt(h2) : 1e300) : 0.0;
  return true;
}

// surface3.rs:933-965 bez_bounds for a rational cubic
bool piece_bounds(const H cp[4], double* lam_out, double d2[3][2]) {
  const int n = 3;
  V c;
  for (int i = 0; i < 4; i++) c = c + hv(cp[i]);
  c = c * 0.25;
  auto q = [&](int i) {
    const H& h = cp[i];
    return H{h[0] - c.x * h[3], h[1] - c.y * h[3], h[2] - c.z * h[3], h[3]};
  };
  Iv A[4], A1[4], A2[4];
  for (int k = 0; k < 4; k++) {
    std::vector<double> a, a1, a2;
    for (int i = 0; i <= n; i++) {
      a.push_back(q(i)[k]);
      if (i < n) a1.push_back(n * (q(i + 1)[k] - q(i)[k]));
      if (i + 1 < n) a2.push_back(n * (n - 1) * (q(i + 2)[k] - 2 * q(i + 1)[k] + q(i)[k]));
    }
    A[k] = iv_of(a);
    A1[k] = iv_of(a1);
    A2[k] = iv_of(a2);
  }
  Iv w = A[3];
  if (!(w.lo > 0)) return false;
  Iv s[3], d1[3], dd[3];
  for (int k = 0; k < 3; k++) {
    std::vector<double> xs;
    for (int i = 0; i < 4; i++) xs.push_back(hv(cp[i])[k] - c[k]);
    s[k] = iv_of(xs);
    d1[k] = divpos(sub(A1[k], mul(s[k], A1[3])), w);
  }
  for (int k = 0; k < 3; k++) dd[k] = divpos(sub(sub(A2[k], scale(mul(d1[k], A1[3]), 2.0)), mul(s[k], A2[3])), w);
  Cubic3 z;
  for (int i = 0; i < 4; i++) z.c[i] = cp[i];
  V p0, e1;
  z.eval(0.5, &p0, &e1);
  double spread = 0, m2 = 0;
  for (int k = 0; k < 3; k++) {
    spread += std::pow(std::max(std::fabs(d1[k].lo - e1[k]), std::fabs(d1[k].hi - e1[k])), 2);
    m2 += mig(d1[k]) * mig(d1[k]);
  }
  double l = std::max(m2, std::pow(std::max(e1.len() - std::sqrt(spread), 0.0), 2));
  *lam_out = l;
  for (int k = 0; k < 3; k++) {
    d2[k][0] = dd[k].lo;
    d2[k][1] = dd[k].hi;
  }
  return true;
}

// lam + sum_k min((C - p)_k C''_k) > 1e-6 lam with C - p over the box grown by `need`:
// each component of C - p within [-(w_k + need), w_k + need].
bool piece_certifies(const Cubic3& z, double need) {
  double lam, d2[3][2];
  if (!piece_bounds(z.c, &lam, d2)) return false;
  Bx b = z.box();
  double e = 0.0;
  for (int k = 0; k < 3; k++) {
    double w = b.hi[k] - b.lo[k] + need;
    e -= w * std::max(std::fabs(d2[k][0]), std::fabs(d2[k][1]));
  }
  return lam + e > 1e-6 * lam;
}

void Cubic3::eval(double s, V* P, V* D1) const {
  double b[4], d[4], dd[4];
  bern3(s, b, d, dd);
  double a[2][4] = {{0}};
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 4; k++) {
      a[0][k] += b[i] * c[i][k];
      a[1][k] += d[i] * c[i][k];
    }
  V p(a[0][0] / a[0][3], a[0][1] / a[0][3], a[0][2] / a[0][3]);
  if (P) *P = p;
  if (D1) *D1 = (V(a[1][0], a[1][1], a[1][2]) - p * a[1][3]) * (1.0 / a[0][3]);
}

void Cubic3::split(double s, Cubic3* l, Cubic3* r) const { split4(c, s, l->c, r->c); }

double Cubic3::turning() const {
  std::vector<V> legs;
  for (int i = 1; i < 4; i++) {
    V d = hv(c[i]) - hv(c[i - 1]);
    if (d.len() > 1e-14) legs.push_back(d);
  }
  double t = 0;
  for (size_t i = 1; i < legs.size(); i++) t += std::atan2(legs[i - 1].cross(legs[i]).len(), legs[i - 1].dot(legs[i]));
  return t;
}

double Cubic3::thickness() const {
  V a = hv(c[0]), b = hv(c[3]), ab = b - a;
  double m = 0, l2 = ab.dot(ab);
  for (int i = 0; i < 4; i++) {
    V p = hv(c[i]);
    double t = l2 > 0 ? std::min(std::max((p - a).dot(ab) / l2, 0.0), 1.0) : 0.0;
    m = std::max(m, (p - (a + ab * t)).len());
  }
  return m;
}

// ---------------------------------------------------------------- trim trees

static const double REF_U = 0.5137, REF_V = 0.4871;  // trim2.rs:102
static const int MAX_TREE_DEPTH = 10;                // trim2.rs:99
// A cell with loop pieces in it is split down to this depth even when few pieces touch
// it (the reference stops at four): a point's parity walk is then needed only within a
// cell of the loops, 1/128 of the domain across, and the answer is the same.
static const int MIN_MIXED_DEPTH = 7;

double tp_coord(const TP& p, int k, double t) {
  // a constant coordinate is that constant exactly (trim2.rs:135-139)
  double e0 = p.c[0][k] / p.c[0][2];
  if (e0 == p.c[1][k] / p.c[1][2] && e0 == p.c[2][k] / p.c[2][2] && e0 == p.c[3][k] / p.c[3][2]) return e0;
  double s = 1 - t, b[4] = {s * s * s, 3 * s * s * t, 3 * s * t * t, t * t * t};
  double n = 0, w = 0;
  for (int i = 0; i < 4; i++) {
    n += b[i] * p.c[i][k];
    w += b[i] * p.c[i][2];
  }
  return n / w;
}

// The sign-carrying numerator of d(coordinate k)/dt.
double tp_dnum(const TP& p, int k, double t) {
  double s = 1 - t, b[4] = {s * s * s, 3 * s * s * t, 3 * s * t * t, t * t * t};
  double d[3] = {3 * s * s, 6 * s * t, 3 * t * t};
  double n = 0, w = 0, n1 = 0, w1 = 0;
  for (int i = 0; i < 4; i++) {
    n += b[i] * p.c[i][k];
    w += b[i] * p.c[i][2];
  }
  for (int i = 0; i < 3; i++) {
    n1 += d[i] * (p.c[i + 1][k] - p.c[i][k]);
    w1 += d[i] * (p.c[i + 1][2] - p.c[i][2]);
  }
  return n1 * w - n * w1;
}

static double endv(const TP& p, int i, int k) { return p.c[i][k] / p.c[i][2]; }

// Half-open crossing of a monotone coordinate (trim2.rs:1155-1190), safeguarded Newton
// on the cubic sum_i B_i (c_i - x w_i).
bool tp_cross(const TP& p, int k, double x, double* tout) {
  double p0 = endv(p, 0, k), p1 = endv(p, 3, k);
  if (!(std::min(p0, p1) <= x && x < std::max(p0, p1))) return false;
  double a[4];
  for (int i = 0; i < 4; i++) a[i] = p.c[i][k] - x * p.c[i][2];
  auto f = [&](double t) {
    double s = 1 - t;
    return s * s * s * a[0] + 3 * s * s * t * a[1] + 3 * s * t * t * a[2] + t * t * t * a[3];
  };
  auto df = [&](double t) {
    double s = 1 - t;
    return 3 * (s * s * (a[1] - a[0]) + 2 * s * t * (a[2] - a[1]) + t * t * (a[3] - a[2]));
  };
  double lo = 0, hi = 1, flo = f(0);
  if (flo == 0) {
    *tout = 0;
    return true;
  }
  double t = std::min(std::max((x - p0) / (p1 - p0), 0.0), 1.0);
  for (int it = 0; it < 60; it++) {
    double ft = f(t);
    if (ft == 0) break;
    if ((ft < 0) == (flo < 0)) {
      lo = t;
      flo = ft;
    } else {
      hi = t;
    }
    double d = df(t);
    double nt = d != 0 ? t - ft / d : 0.5 * (lo + hi);
    if (!(nt > lo && nt < hi)) nt = 0.5 * (lo + hi);
    if (std::fabs(nt - t) <= 1e-16) {
      t = nt;
      break;
    }
    t = nt;
  }
  *tout = t;
  return true;
}

static void tp_split(const TP& p, double s, TP* l, TP* r) {
  double b[4][3];
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 3; k++) b[i][k] = p.c[i][k];
  for (int k = 0; k < 3; k++) {
    l->c[0][k] = b[0][k];
    r->c[3][k] = b[3][k];
  }
  for (int level = 1; level <= 3; level++) {
    for (int i = 0; i <= 3 - level; i++)
      for (int k = 0; k < 3; k++) b[i][k] = (1 - s) * b[i][k] + s * b[i + 1][k];
    for (int k = 0; k < 3; k++) {
      l->c[level][k] = b[0][k];
      r->c[3 - level][k] = b[3 - level][k];
    }
  }
}

// Splits a piece where either coordinate's derivative changes sign, so each part is
// monotone in both.
static void monotone_parts(const TP& p, std::vector<TP>& out) {
  std::vector<double> cuts;
  const int N = 256;
  for (int k = 0; k < 2; k++) {
    double scale = 0;
    for (int i = 0; i <= N; i++) scale = std::max(scale, std::fabs(tp_dnum(p, k, double(i) / N)));
    if (!(scale > 0)) continue;
    double prev = tp_dnum(p, k, 0);
    for (int i = 1; i <= N; i++) {
      double t = double(i) / N, cur = tp_dnum(p, k, t);
      if ((prev < 0 && cur > 0) || (prev > 0 && cur < 0)) {
        double a = double(i - 1) / N, b = t, fa = prev;
        for (int it = 0; it < 100; it++) {
          double m = 0.5 * (a + b), fm = tp_dnum(p, k, m);
          if ((fm < 0) == (fa < 0)) {
            a = m;
            fa = fm;
          } else {
            b = m;
          }
        }
        double tt = 0.5 * (a + b);
        if (tt > 1e-9 && tt < 1 - 1e-9) cuts.push_back(tt);
      }
      if (std::fabs(cur) > 1e-13 * scale) prev = cur;
    }
  }
  std::sort(cuts.begin(), cuts.end());
  TP rest = p;
  double done = 0;
  for (double t : cuts) {
    if (t - done < 1e-9) continue;
    TP l, r;
    tp_split(rest, (t - done) / (1 - done), &l, &r);
    out.push_back(l);
    rest = r;
    done = t;
  }
  out.push_back(rest);
}

static std::array<double, 4> tp_box(const TP& p) {
  std::array<double, 4> b = {1e300, 1e300, -1e300, -1e300};
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 2; k++) {
      double v = endv(p, i, k);
      b[k] = std::min(b[k], v);
      b[2 + k] = std::max(b[2 + k], v);
    }
  return b;
}

static bool boxes_meet(const double alo[2], const double ahi[2], const double blo[2], const double bhi[2]) {
  return alo[0] <= bhi[0] && blo[0] <= ahi[0] && alo[1] <= bhi[1] && blo[1] <= ahi[1];
}

TP TrimTree::shifted(int i) const {
  TP c = pieces[inst[i].first];
  for (int j = 0; j < 4; j++)
    for (int k = 0; k < 2; k++) c.c[j][k] += inst[i].second[k] * c.c[j][2];
  return c;
}

// trim2.rs:1192-1259: parity of the path a -> (a.u, b.v) -> b, moved up by e and right
// by e^2, against the given pieces.
bool TrimTree::parity(const double a[2], const double b[2], const std::vector<int>& among) const {
  int n = 0;
  bool up = a[1] < b[1], right = a[0] < b[0];
  for (int i : among) {
    TP c = shifted(i);
    double t;
    if (a[1] != b[1] && tp_cross(c, 0, a[0], &t)) {
      double y = tp_coord(c, 1, t);
      if (up ? (y > a[1] && y <= b[1]) : (y > b[1] && y <= a[1])) n++;
    }
    if (a[0] != b[0] && tp_cross(c, 1, b[1], &t)) {
      double x = tp_coord(c, 0, t);
      auto slope_pos = [&]() {
        double du = tp_dnum(c, 0, t), dv = tp_dnum(c, 1, t);
        if (dv == 0) dv = endv(c, 3, 1) - endv(c, 0, 1);
        return du * dv > 0;
      };
      bool counted;
      if (x == b[0])
        counted = (!slope_pos()) == right;
      else if (x == a[0])
        counted = slope_pos() == right;
      else
        counted = right ? (x > a[0] && x < b[0]) : (x > b[0] && x < a[0]);
      if (counted) n++;
    }
  }
  return n & 1;
}

double TrimTree::dist2(int i, const double q[2]) const {
  TP c = shifted(i);
  auto d2 = [&](double t) {
    double u = tp_coord(c, 0, t) - q[0], v = tp_coord(c, 1, t) - q[1];
    return u * u + v * v;
  };
  double best = 1e300, bt = 0;
  for (int k = 0; k <= 16; k++) {
    double d = d2(k / 16.0);
    if (d < best) best = d, bt = k / 16.0;
  }
  double a = std::max(bt - 1 / 16.0, 0.0), b = std::min(bt + 1 / 16.0, 1.0);
  for (int it = 0; it < 40; it++) {
    double x = a + 0.381966 * (b - a), y = b - 0.381966 * (b - a);
    if (d2(x) < d2(y))
      b = y;
    else
      a = x;
  }
  return std::min(best, d2(0.5 * (a + b)));
}

// trim2.rs:1352-1392: a point off piece p's middle (left or right) whose nearest loop
// point is that middle, inside the domain.
bool TrimTree::offset_point(const TP& p, const std::vector<int>& all, bool left, double out[2]) const {
  double small = std::min(hi[0] - lo[0], hi[1] - lo[1]);
  double m[2] = {tp_coord(p, 0, 0.5), tp_coord(p, 1, 0.5)};
  for (int k = 0; k < 2; k++)
    if (period[k] > 0) {
      double x = std::fmod(m[k] - lo[k], period[k]);
      m[k] = lo[k] + (x < 0 ? x + period[k] : x);
    }
  double du = tp_coord(p, 0, 0.51) - tp_coord(p, 0, 0.49), dv = tp_coord(p, 1, 0.51) - tp_coord(p, 1, 0.49);
  double l = std::sqrt(du * du + dv * dv);
  if (!(l > 0)) return false;
  double sd = left ? 1 : -1, n0 = -dv / l * sd, n1 = du / l * sd;
  for (double delta = 1e-3 * small; delta >= 1e-6 * small; delta *= 0.5) {
    double r[2] = {m[0] + n0 * delta, m[1] + n1 * delta};
    bool ok = true;
    for (int k = 0; k < 2; k++)
      if (!(period[k] > 0 || (r[k] > lo[k] + 0.5 * delta && r[k] < hi[k] - 0.5 * delta))) ok = false;
    if (!ok) continue;
    double nearest = 1e300;
    for (int i : all) nearest = std::min(nearest, dist2(i, r));
    if (nearest >= delta * delta * (1 - 1e-9)) {
      out[0] = r[0];
      out[1] = r[1];
      return true;
    }
  }
  return false;
}

bool TrimTree::build(const std::vector<TP>& raw, const double lo_[2], const double hi_[2], const double per[2],
                     bool left, std::string* err) {
  pieces.clear();
  for (auto& p : raw) monotone_parts(p, pieces);
  for (int k = 0; k < 2; k++) {
    lo[k] = lo_[k];
    hi[k] = hi_[k];
    period[k] = per[k];
  }
  inside_left = left;
  double rlo[2] = {lo[0], lo[1]}, rhi[2] = {hi[0], hi[1]};
  for (int k = 0; k < 2; k++)
    if (period[k] > 0) rlo[k] -= period[k], rhi[k] += period[k];
  inst.clear();
  for (int i = 0; i < int(pieces.size()); i++) {
    auto b = tp_box(pieces[i]);
    long r0[2] = {0, 0}, r1[2] = {0, 0};
    for (int k = 0; k < 2; k++)
      if (period[k] > 0) {
        r0[k] = long(std::ceil((rlo[k] - b[2 + k]) / period[k]));
        r1[k] = long(std::floor((rhi[k] - b[k]) / period[k]));
      }
    for (long a = r0[0]; a <= r1[0]; a++)
      for (long c = r0[1]; c <= r1[1]; c++) inst.push_back({i, {a * period[0], c * period[1]}});
  }
  std::vector<std::array<double, 4>> boxes;
  std::vector<int> all;
  for (int i = 0; i < int(inst.size()); i++) {
    boxes.push_back(tp_box(shifted(i)));
    all.push_back(i);
  }
  TCell root;
  root.lo[0] = lo[0], root.lo[1] = lo[1], root.hi[0] = hi[0], root.hi[1] = hi[1];
  root.r[0] = lo[0] + (hi[0] - lo[0]) * REF_U;
  root.r[1] = lo[1] + (hi[1] - lo[1]) * REF_V;
  root.inside = 1;
  root.kind = 0;
  if (!pieces.empty()) {
    std::vector<int> order(pieces.size());
    for (int i = 0; i < int(order.size()); i++) order[i] = i;
    auto chord = [&](int i) { return std::hypot(endv(pieces[i], 3, 0) - endv(pieces[i], 0, 0), endv(pieces[i], 3, 1) - endv(pieces[i], 0, 1)); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return chord(a) > chord(b); });
    bool found = false, side = true;
    double r[2];
    for (int i = 0; i < int(order.size()) && i < 64 && !found; i++)
      for (int l = 1; l >= 0 && !found; l--)
        if (offset_point(pieces[order[i]], all, l == 1, r)) found = true, side = l == 1;
    if (!found) {
      if (err) *err = "no loop piece gives a settled reference point inside the domain";
      return false;
    }
    root.inside = ((side == inside_left) ^ parity(r, root.r, all)) ? 1 : 0;
  }
  cells.clear();
  cells.push_back(root);
  build_cell(0, all, boxes, 0);
  return true;
}

void TrimTree::build_cell(int id, const std::vector<int>& cand, const std::vector<std::array<double, 4>>& boxes,
                          int depth) {
  double clo[2] = {cells[id].lo[0], cells[id].lo[1]}, chi[2] = {cells[id].hi[0], cells[id].hi[1]};
  double r[2] = {cells[id].r[0], cells[id].r[1]};
  int inside = cells[id].inside;
  std::vector<int> touching;
  for (int i : cand) {
    double blo[2] = {boxes[i][0], boxes[i][1]}, bhi[2] = {boxes[i][2], boxes[i][3]};
    if (boxes_meet(clo, chi, blo, bhi)) touching.push_back(i);
  }
  if (touching.empty()) {
    cells[id].kind = 0;
    return;
  }
  if (depth >= MAX_TREE_DEPTH || (touching.size() <= 4 && depth >= MIN_MIXED_DEPTH)) {
    cells[id].kind = 1;
    cells[id].among = touching;
    return;
  }
  double m[2] = {0.5 * (clo[0] + chi[0]), 0.5 * (clo[1] + chi[1])};
  double q[4][4] = {{clo[0], clo[1], m[0], m[1]}, {m[0], clo[1], chi[0], m[1]}, {clo[0], m[1], m[0], chi[1]}, {m[0], m[1], chi[0], chi[1]}};
  int kids[4];
  for (int k = 0; k < 4; k++) {
    TCell c;
    c.lo[0] = q[k][0], c.lo[1] = q[k][1], c.hi[0] = q[k][2], c.hi[1] = q[k][3];
    c.r[0] = c.lo[0] + (c.hi[0] - c.lo[0]) * REF_U;
    c.r[1] = c.lo[1] + (c.hi[1] - c.lo[1]) * REF_V;
    c.inside = inside ^ (parity(r, c.r, touching) ? 1 : 0);
    c.kind = 0;
    int kid = int(cells.size());
    cells.push_back(c);
    build_cell(kid, touching, boxes, depth + 1);
    kids[k] = kid;
  }
  cells[id].kind = 2;
  for (int k = 0; k < 4; k++) cells[id].kids[k] = kids[k];
}

bool TrimTree::inside(double u, double v) const {
  double q[2] = {u, v};
  for (int k = 0; k < 2; k++) {
    if (period[k] > 0) {
      double x = std::fmod(q[k] - lo[k], period[k]);
      q[k] = lo[k] + (x < 0 ? x + period[k] : x);
    } else {
      q[k] = std::min(std::max(q[k], lo[k]), hi[k]);
    }
  }
  if (pieces.empty()) return true;
  int id = 0;
  for (;;) {
    const TCell& c = cells[id];
    if (c.kind == 0) return c.inside;
    if (c.kind == 1) return c.inside ^ parity(c.r, q, c.among);
    double m0 = 0.5 * (c.lo[0] + c.hi[0]), m1 = 0.5 * (c.lo[1] + c.hi[1]);
    id = c.kids[int(q[0] >= m0) + 2 * int(q[1] >= m1)];
  }
}

// trim2.rs:1119-1135 meets_box for a monotone piece
static bool piece_meets(const TP& c, const double lo[2], const double hi[2]) {
  auto b = tp_box(c);
  double blo[2] = {b[0], b[1]}, bhi[2] = {b[2], b[3]};
  if (!boxes_meet(blo, bhi, lo, hi)) return false;
  double u0 = endv(c, 0, 0), u3 = endv(c, 3, 0);
  auto param_at = [&](double x) {
    if (x == u0) return 0.0;
    if (x == u3) return 1.0;
    double t;
    if (tp_cross(c, 0, x, &t)) return t;
    return std::fabs(x - u0) < std::fabs(x - u3) ? 0.0 : 1.0;
  };
  double ta = 0, tb = 1;
  if (u0 != u3) {
    ta = param_at(std::max(lo[0], std::min(u0, u3)));
    tb = param_at(std::min(hi[0], std::max(u0, u3)));
  }
  double va = tp_coord(c, 1, ta), vb = tp_coord(c, 1, tb);
  return std::min(va, vb) <= hi[1] && std::max(va, vb) >= lo[1];
}

int TrimTree::class_in(int id, const double blo[2], const double bhi[2]) const {
  const TCell& c = cells[id];
  double ilo[2] = {std::max(blo[0], c.lo[0]), std::max(blo[1], c.lo[1])};
  double ihi[2] = {std::min(bhi[0], c.hi[0]), std::min(bhi[1], c.hi[1])};
  if (c.kind == 0) return c.inside;
  if (c.kind == 1) {
    double g = 1e-12 * (std::fabs(hi[0] - lo[0]) + std::fabs(hi[1] - lo[1]));
    double glo[2] = {ilo[0] - g, ilo[1] - g}, ghi[2] = {ihi[0] + g, ihi[1] + g};
    for (int i : c.among)
      if (piece_meets(shifted(i), glo, ghi)) return -1;
    double m[2] = {0.5 * (ilo[0] + ihi[0]), 0.5 * (ilo[1] + ihi[1])};
    return c.inside ^ (parity(c.r, m, c.among) ? 1 : 0);
  }
  int answer = -2;
  for (int k : c.kids) {
    const TCell& kc = cells[k];
    if (!boxes_meet(kc.lo, kc.hi, blo, bhi)) continue;
    int a = class_in(k, blo, bhi);
    if (a == -1) return -1;
    if (answer == -2)
      answer = a;
    else if (answer != a)
      return -1;
  }
  return answer == -2 ? -1 : answer;
}

int TrimTree::box_class(const double blo[2], const double bhi[2]) const {
  if (pieces.empty()) return 1;
  return class_in(0, blo, bhi);
}

}  // namespace icam

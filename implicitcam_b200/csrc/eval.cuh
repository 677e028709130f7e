// Device evaluators of the exact part field, one feature at a time, in double
// precision: each answers "does this feature hold a point nearer than `cutoff`, and if
// so its distance and sign" by the reference evaluator's rules
// (crates/icam-core/src/solid3.rs:1758-1816 sdf_within):
//  - an analytic face contributes its closed-form foot when the foot lies in the face
//    by its loops (solid3.rs:1911-1925);
//  - a B-spline face contributes the critical points of the squared distance inside
//    it (surface3.rs:1214-1297); here each certified sub-patch holds at most one, the
//    unique minimum of a strictly convex function over its rectangle, found by the
//    projected Newton of surface3.rs:401-447;
//  - an edge contributes an interior foot, signed by its two faces' normals summed
//    (solid3.rs:1775-1782);
//  - a vertex its distance, signed by its angle-weighted pseudo-normal.
// Sign rule: x < 0 ? -1 : +1 (solid3.rs:1764).
#pragma once

#include <cuda_runtime.h>

#include "pack.h"

namespace icam {

#define HD __host__ __device__ __forceinline__
#define HDI __host__ __device__ inline
// out of line: paths the hot loops seldom take, kept out of their instruction stream
#define HDC __host__ __device__ inline __noinline__

HD double3 mk(double x, double y, double z) { return make_double3(x, y, z); }
HD double3 operator+(double3 a, double3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
HD double3 operator-(double3 a, double3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
HD double3 operator*(double3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
HD double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HD double3 cross(double3 a, double3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
HD double len(double3 a) { return sqrt(dot(a, a)); }
HD double3 unit(double3 a) {
  double l = len(a);
  return l > 0 ? a * (1.0 / l) : a;
}
HD double3 ld3(const double* p) { return mk(p[0], p[1], p[2]); }
HD double sgn(double x) { return x < 0.0 ? -1.0 : 1.0; }

// surface3.rs:978 box_dist
HD double box_dist(double3 p, const double* b) {
  double dx = fmax(fmax(b[0] - p.x, p.x - b[3]), 0.0);
  double dy = fmax(fmax(b[1] - p.y, p.y - b[4]), 0.0);
  double dz = fmax(fmax(b[2] - p.z, p.z - b[5]), 0.0);
  return sqrt(dx * dx + dy * dy + dz * dz);
}
HD double box_dist_f(double3 p, const float* lo, const float* hi) {
  double dx = fmax(fmax(double(lo[0]) - p.x, p.x - double(hi[0])), 0.0);
  double dy = fmax(fmax(double(lo[1]) - p.y, p.y - double(hi[1])), 0.0);
  double dz = fmax(fmax(double(lo[2]) - p.z, p.z - double(hi[2])), 0.0);
  return sqrt(dx * dx + dy * dy + dz * dz);
}

constexpr double DIST_EPS = 1e-9;  // surface3.rs:975

// ---------------------------------------------------------------- analytic faces

struct AxialD {
  double theta, rho, h;
  double3 er;
};
HD AxialD axial(const DFace& f, double3 p) {
  double3 d = p - ld3(f.o);
  double lx = dot(d, ld3(f.x)), ly = dot(d, ld3(f.y)), lz = dot(d, ld3(f.z));
  double rho = sqrt(lx * lx + ly * ly);
  double th = rho > 0.0 ? atan2(ly, lx) : 0.0;
  double s, c;
  sincos(th, &s, &c);
  return {th, rho, lz, ld3(f.x) * c + ld3(f.y) * s};
}

// surface3.rs:85-129 foot; surface3.rs:132-148 normal (times the sense); the loops'
// parameters of the foot (trim2.rs:1904-1933 with the angle itself). Returns false for
// a singular foot (a cone's apex), where edges and vertices answer.
HDC bool analytic_foot_curved(const DFace& f, double3 p, double3* q, double3* n, double* u, double* v);

// Planes inline; the curved kinds (with their trigonometry) out of line.
HDI bool analytic_foot(const DFace& f, double3 p, double3* q, double3* n, double* u, double* v) {
  if (f.kind == S_PLANE) {
    double3 z = ld3(f.z);
    double3 d = p - ld3(f.o);
    double h = dot(d, z);
    *q = p - z * h;
    *n = z * f.sense;
    double3 e = *q - ld3(f.o);
    *u = dot(e, ld3(f.x));
    *v = dot(e, ld3(f.y));
    return true;
  }
  return analytic_foot_curved(f, p, q, n, u, v);
}

HDC bool analytic_foot_curved(const DFace& f, double3 p, double3* q, double3* n, double* u, double* v) {
  switch (f.kind) {
    case S_CYLINDER: {
      AxialD ax = axial(f, p);
      *q = ld3(f.o) + ax.er * f.a + ld3(f.z) * ax.h;
      *n = ax.er * f.sense;
      *u = ax.theta;
      *v = ax.h;
      return true;
    }
    case S_CONE: {
      AxialD ax = axial(f, p);
      double sa, ca;
      sincos(f.b, &sa, &ca);
      double ha = -f.a / tan(f.b);
      double s = ax.rho * sa + (ax.h - ha) * ca;
      if (s <= 0.0) return false;
      *q = ld3(f.o) + ax.er * (s * sa) + ld3(f.z) * (ha + s * ca);
      *n = (ax.er * ca - ld3(f.z) * sa) * f.sense;
      *u = ax.theta;
      *v = ha + s * ca;
      return true;
    }
    case S_SPHERE: {
      double3 d = p - ld3(f.o);
      double l = len(d);
      *q = l > 0.0 ? ld3(f.o) + d * (f.a / l) : ld3(f.o) + ld3(f.x) * f.a;
      *n = unit(*q - ld3(f.o)) * f.sense;
      AxialD ax = axial(f, *q);
      *u = ax.theta;
      *v = atan2(ax.h, ax.rho);
      return true;
    }
    default: {  // torus
      double major = f.a, minor = f.b;
      AxialD ax = axial(f, p);
      double3 c = ld3(f.o) + ax.er * major;
      double3 d = p - c;
      double l = len(d);
      double3 qq = l > 0.0 ? c + d * (minor / l) : c + ax.er * minor;
      if (!(dot(qq - ld3(f.o), ax.er) >= 0.0 || fabs(major) > minor)) return false;  // a tip
      *q = qq;
      *n = unit(qq - c) * f.sense;
      AxialD aq = axial(f, qq);
      *u = aq.theta;
      *v = atan2(aq.h, aq.rho - major);
      return true;
    }
  }
}

// ---------------------------------------------------------------- trim parity

// The coordinate k of a rational cubic loop piece (u w, v w, w) shifted by `sh`. A
// coordinate constant along the piece is that constant exactly (trim2.rs:135-139
// b_eval: the weighted sums need not round back to it, and grid points lie on such
// lines).
HD double tp_coord(const double* c, const double* sh, int k, double t) {
  double e0 = c[k] / c[2];
  if (e0 == c[3 + k] / c[5] && e0 == c[6 + k] / c[8] && e0 == c[9 + k] / c[11]) return e0 + sh[k];
  double s = 1.0 - t;
  double b0 = s * s * s, b1 = 3.0 * s * s * t, b2 = 3.0 * s * t * t, b3 = t * t * t;
  double w = b0 * c[2] + b1 * c[5] + b2 * c[8] + b3 * c[11];
  double n = b0 * c[k] + b1 * c[3 + k] + b2 * c[6 + k] + b3 * c[9 + k];
  return n / w + sh[k];
}

// The sign-carrying numerator of the derivative of coordinate k.
HD double tp_dnum(const double* c, int k, double t) {
  double s = 1.0 - t;
  double b0 = s * s * s, b1 = 3.0 * s * s * t, b2 = 3.0 * s * t * t, b3 = t * t * t;
  double d0 = 3.0 * s * s, d1 = 6.0 * s * t, d2 = 3.0 * t * t;
  double n = b0 * c[k] + b1 * c[3 + k] + b2 * c[6 + k] + b3 * c[9 + k];
  double w = b0 * c[2] + b1 * c[5] + b2 * c[8] + b3 * c[11];
  double n1 = d0 * (c[3 + k] - c[k]) + d1 * (c[6 + k] - c[3 + k]) + d2 * (c[9 + k] - c[6 + k]);
  double w1 = d0 * (c[5] - c[2]) + d1 * (c[8] - c[5]) + d2 * (c[11] - c[8]);
  return n1 * w - n * w1;
}

// trim2.rs:1155-1190 crossing on a rational piece: where coordinate k equals x, for x in
// the half-open range of its end values; safeguarded Newton on sum_i B_i (c_i - x w_i).
HDI bool tp_cross(const double* c, const double* sh, int k, double x, double* tout) {
  double xs = x - sh[k];
  double p0 = c[k] / c[2], p1 = c[9 + k] / c[11];
  if (!(fmin(p0, p1) <= xs && xs < fmax(p0, p1))) return false;
  double a0 = c[k] - xs * c[2], a1 = c[3 + k] - xs * c[5], a2 = c[6 + k] - xs * c[8], a3 = c[9 + k] - xs * c[11];
  double lo = 0.0, hi = 1.0, flo = a0;
  if (flo == 0.0) {
    *tout = 0.0;
    return true;
  }
  double t = fmin(fmax((xs - p0) / (p1 - p0), 0.0), 1.0);
  for (int it = 0; it < 60; it++) {
    double s = 1.0 - t;
    double ft = s * s * s * a0 + 3.0 * s * s * t * a1 + 3.0 * s * t * t * a2 + t * t * t * a3;
    if (ft == 0.0) break;
    if ((ft < 0.0) == (flo < 0.0)) {
      lo = t;
      flo = ft;
    } else {
      hi = t;
    }
    double d = 3.0 * (s * s * (a1 - a0) + 2.0 * s * t * (a2 - a1) + t * t * (a3 - a2));
    double nt = d != 0.0 ? t - ft / d : 0.5 * (lo + hi);
    if (!(nt > lo && nt < hi)) nt = 0.5 * (lo + hi);
    if (fabs(nt - t) <= 1e-16) {
      t = nt;
      break;
    }
    t = nt;
  }
  *tout = t;
  return true;
}

// trim2.rs:1192-1259 parity of the path a -> (a.u, b.v) -> b, symbolically raised by e
// and moved right by e^2, against the instances in `among`.
HDC bool trim_parity(const DPack& P, const double* a, const double* b, const int32_t* among, int count) {
  int n = 0;
  bool up = a[1] < b[1], right = a[0] < b[0];
  for (int i = 0; i < count; i++) {
    const DInst& in = P.insts[among[i]];
    const double* c = P.tpieces + 12 * size_t(in.piece);
    const double* sh = in.shift;
    double t;
    if (a[1] != b[1] && tp_cross(c, sh, 0, a[0], &t)) {
      double y = tp_coord(c, sh, 1, t);
      if (up ? (y > a[1] && y <= b[1]) : (y > b[1] && y <= a[1])) n++;
    }
    if (a[0] != b[0] && tp_cross(c, sh, 1, b[1], &t)) {
      double x = tp_coord(c, sh, 0, t);
      bool counted;
      if (x == b[0] || x == a[0]) {
        double du = tp_dnum(c, 0, t), dv = tp_dnum(c, 1, t);
        if (dv == 0.0) dv = c[10] / c[11] - c[1] / c[2];
        bool slope_pos = du * dv > 0.0;
        counted = x == b[0] ? ((!slope_pos) == right) : (slope_pos == right);
      } else {
        counted = right ? (x > a[0] && x < b[0]) : (x > b[0] && x < a[0]);
      }
      if (counted) n++;
    }
  }
  return n & 1;
}

// trim2.rs:1433-1457 inside: reduce (u, v) into the domain, descend to its cell, and
// flip the cell's answer by the parity of the path from its reference point.
HDI bool trim_inside(const DPack& P, const DFace& f, double u, double v) {
  if (f.trim < 0) return true;
  double q[2] = {u, v};
  for (int k = 0; k < 2; k++) {
    if (f.period[k] > 0.0) {
      double x = fmod(q[k] - f.lo[k], f.period[k]);
      q[k] = f.lo[k] + (x < 0.0 ? x + f.period[k] : x);
    } else {
      q[k] = fmin(fmax(q[k], f.lo[k]), f.hi[k]);
    }
  }
  int id = f.trim;
  for (int guard = 0; guard < 64; guard++) {
    const DCell& c = P.cells[id];
    if (c.kind == 0) return c.inside;
    if (c.kind == 1) return c.inside ^ trim_parity(P, c.r, q, P.among + c.first, c.count);
    double m0 = 0.5 * (c.lo[0] + c.hi[0]), m1 = 0.5 * (c.lo[1] + c.hi[1]);
    id = c.kids[int(q[0] >= m0) + 2 * int(q[1] >= m1)];
  }
  return false;
}

// What trim_inside answers over a whole parameter box [blo, bhi] of a face without
// periodic directions: 1 inside or 0 outside when every cell the box meets (closed
// boxes, so a point on a split line counts for both sides) is a leaf without loop
// pieces and they agree, -1 otherwise (the point test decides). Points reduced into the
// domain as trim_inside reduces them.
HDI int trim_box_class(const DPack& P, const DFace& f, const double blo[2], const double bhi[2]) {
  if (f.trim < 0) return 1;
  if (f.period[0] > 0.0 || f.period[1] > 0.0) return -1;
  double lo[2], hi[2];
  for (int k = 0; k < 2; k++) {
    lo[k] = fmin(fmax(blo[k], f.lo[k]), f.hi[k]);
    hi[k] = fmin(fmax(bhi[k], f.lo[k]), f.hi[k]);
  }
  int stack[48];
  int sp = 0, answer = -2, visited = 0;
  stack[sp++] = f.trim;
  while (sp > 0) {
    const DCell& c = P.cells[stack[--sp]];
    if (++visited > 256 || c.kind == 1) return -1;
    if (c.kind == 0) {
      if (answer == -2)
        answer = c.inside;
      else if (answer != c.inside)
        return -1;
      continue;
    }
    for (int q = 0; q < 4; q++) {
      const DCell& kc = P.cells[c.kids[q]];
      if (kc.lo[0] > hi[0] || kc.hi[0] < lo[0] || kc.lo[1] > hi[1] || kc.hi[1] < lo[1]) continue;
      if (sp >= 48) return -1;
      stack[sp++] = c.kids[q];
    }
  }
  return answer == -2 ? -1 : answer;
}

// ---------------------------------------------------------------- bicubic patches

struct SE {
  double3 p, ps, pt, pss, pst, ptt;
};

HD void bern3(double t, double* b, double* d, double* dd) {
  double s = 1.0 - t;
  b[0] = s * s * s;
  b[1] = 3.0 * s * s * t;
  b[2] = 3.0 * s * t * t;
  b[3] = t * t * t;
  d[0] = -3.0 * s * s;
  d[1] = 3.0 * s * s - 6.0 * s * t;
  d[2] = 6.0 * s * t - 3.0 * t * t;
  d[3] = 3.0 * t * t;
  dd[0] = 6.0 * s;
  dd[1] = 6.0 * t - 12.0 * s;
  dd[2] = 6.0 * s - 12.0 * t;
  dd[3] = 6.0 * t;
}

// surface3.rs:299-325 eval for a bicubic: point and derivatives by the quotient rule on
// the homogeneous sums.
HD SE eval_bicubic(const double4* cp, double s, double t) {
  double bu[4], du[4], ddu[4], bv[4], dv[4], ddv[4];
  bern3(s, bu, du, ddu);
  bern3(t, bv, dv, ddv);
  double4 a0 = {0, 0, 0, 0}, a1 = a0, a2 = a0, a3 = a0, a4 = a0, a5 = a0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    // rows first: sums along v with each v-basis
    double4 r0 = {0, 0, 0, 0}, r1 = r0, r2 = r0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      double4 c = cp[4 * i + j];
      r0.x += bv[j] * c.x, r0.y += bv[j] * c.y, r0.z += bv[j] * c.z, r0.w += bv[j] * c.w;
      r1.x += dv[j] * c.x, r1.y += dv[j] * c.y, r1.z += dv[j] * c.z, r1.w += dv[j] * c.w;
      r2.x += ddv[j] * c.x, r2.y += ddv[j] * c.y, r2.z += ddv[j] * c.z, r2.w += ddv[j] * c.w;
    }
    a0.x += bu[i] * r0.x, a0.y += bu[i] * r0.y, a0.z += bu[i] * r0.z, a0.w += bu[i] * r0.w;
    a1.x += du[i] * r0.x, a1.y += du[i] * r0.y, a1.z += du[i] * r0.z, a1.w += du[i] * r0.w;
    a2.x += bu[i] * r1.x, a2.y += bu[i] * r1.y, a2.z += bu[i] * r1.z, a2.w += bu[i] * r1.w;
    a3.x += ddu[i] * r0.x, a3.y += ddu[i] * r0.y, a3.z += ddu[i] * r0.z, a3.w += ddu[i] * r0.w;
    a4.x += du[i] * r1.x, a4.y += du[i] * r1.y, a4.z += du[i] * r1.z, a4.w += du[i] * r1.w;
    a5.x += bu[i] * r2.x, a5.y += bu[i] * r2.y, a5.z += bu[i] * r2.z, a5.w += bu[i] * r2.w;
  }
  double iw = 1.0 / a0.w;
  SE e;
  e.p = mk(a0.x, a0.y, a0.z) * iw;
  e.ps = (mk(a1.x, a1.y, a1.z) - e.p * a1.w) * iw;
  e.pt = (mk(a2.x, a2.y, a2.z) - e.p * a2.w) * iw;
  e.pss = (mk(a3.x, a3.y, a3.z) - e.ps * (2.0 * a1.w) - e.p * a3.w) * iw;
  e.pst = (mk(a4.x, a4.y, a4.z) - e.ps * a2.w - e.pt * a1.w - e.p * a4.w) * iw;
  e.ptt = (mk(a5.x, a5.y, a5.z) - e.pt * (2.0 * a2.w) - e.p * a5.w) * iw;
  return e;
}

// Projected Newton on |S - p|^2 over [0, 1]^2 (surface3.rs:401-447 newton_iters, with
// Gauss-Newton where the Hessian is not positive definite). A parameter on its bound
// is held there while the gradient points out of the square (the active set of the
// bound-constrained problem), so on a strictly convex part the iteration ends at its
// unique minimum, inside or on its border. *conv: it stopped on a step under 1e-13,
// or with both parameters held.
HDI void newton_bicubic(const double4* cp, double3 p, double* ps_, double* pt_, int iters, bool* conv) {
  double s = *ps_, t = *pt_;
  *conv = false;
  for (int it = 0; it < iters; it++) {
    SE e = eval_bicubic(cp, s, t);
    double3 r = e.p - p;
    double g0 = dot(e.ps, r), g1 = dot(e.pt, r);
    double jss = dot(e.ps, e.ps), jst = dot(e.ps, e.pt), jtt = dot(e.pt, e.pt);
    double h0 = jss + dot(e.pss, r), h1 = jst + dot(e.pst, r), h2 = jtt + dot(e.ptt, r);
    bool hold_s = (s <= 0.0 && g0 > 0.0) || (s >= 1.0 && g0 < 0.0);
    bool hold_t = (t <= 0.0 && g1 > 0.0) || (t >= 1.0 && g1 < 0.0);
    double ds, dt;
    if (hold_s && hold_t) {
      *conv = true;
      break;
    }
    if (hold_s) {
      ds = 0.0;
      dt = -g1 / (h2 > 0.0 ? h2 : fmax(jtt, 1e-300));
    } else if (hold_t) {
      ds = -g0 / (h0 > 0.0 ? h0 : fmax(jss, 1e-300));
      dt = 0.0;
    } else {
      if (!(h0 > 0.0 && h0 * h2 - h1 * h1 > 0.0)) {
        h0 = jss;
        h1 = jst;
        h2 = jtt;
      }
      double det = h0 * h2 - h1 * h1;
      if (fabs(det) < 1e-300) break;
      ds = -(h2 * g0 - h1 * g1) / det;
      dt = -(h0 * g1 - h1 * g0) / det;
    }
    double ns = fmin(fmax(s + ds, 0.0), 1.0), nt = fmin(fmax(t + dt, 0.0), 1.0);
    double moved = fabs(ns - s) + fabs(nt - t);
    s = ns;
    t = nt;
    if (moved < 1e-13) {
      *conv = true;
      break;
    }
  }
  *ps_ = s;
  *pt_ = t;
}

// newton_bicubic that also hands back the patch at the point it returns, so that the
// caller needs no evaluation of its own: on a step under 1e-13 it returns the point the
// step starts from (within that step of the other end; its gradient is within rounding
// of zero, so the critical-point test reads the same), with both parameters held the
// point itself. *e is meaningful when *conv.
HDI void newton_bicubic_e(const double4* cp, double3 p, double* ps_, double* pt_, int iters, bool* conv, SE* e_out) {
  double s = *ps_, t = *pt_;
  *conv = false;
  for (int it = 0; it < iters; it++) {
    SE e = eval_bicubic(cp, s, t);
    *e_out = e;
    double3 r = e.p - p;
    double g0 = dot(e.ps, r), g1 = dot(e.pt, r);
    double jss = dot(e.ps, e.ps), jst = dot(e.ps, e.pt), jtt = dot(e.pt, e.pt);
    double h0 = jss + dot(e.pss, r), h1 = jst + dot(e.pst, r), h2 = jtt + dot(e.ptt, r);
    bool hold_s = (s <= 0.0 && g0 > 0.0) || (s >= 1.0 && g0 < 0.0);
    bool hold_t = (t <= 0.0 && g1 > 0.0) || (t >= 1.0 && g1 < 0.0);
    double ds, dt;
    if (hold_s && hold_t) {
      *conv = true;
      break;
    }
    if (hold_s) {
      ds = 0.0;
      dt = -g1 / (h2 > 0.0 ? h2 : fmax(jtt, 1e-300));
    } else if (hold_t) {
      ds = -g0 / (h0 > 0.0 ? h0 : fmax(jss, 1e-300));
      dt = 0.0;
    } else {
      if (!(h0 > 0.0 && h0 * h2 - h1 * h1 > 0.0)) {
        h0 = jss;
        h1 = jst;
        h2 = jtt;
      }
      double det = h0 * h2 - h1 * h1;
      if (fabs(det) < 1e-300) break;
      ds = -(h2 * g0 - h1 * g1) / det;
      dt = -(h0 * g1 - h1 * g0) / det;
    }
    double ns = fmin(fmax(s + ds, 0.0), 1.0), nt = fmin(fmax(t + dt, 0.0), 1.0);
    if (fabs(ns - s) + fabs(nt - t) < 1e-13) {
      *conv = true;
      break;
    }
    s = ns;
    t = nt;
  }
  *ps_ = s;
  *pt_ = t;
}

// ---------------------------------------------------------------- single precision (mixed path)

// The bicubic in floats over control points rebased to the sub-patch's centre: the
// point and first and second derivatives, as eval_bicubic.
struct SEf {
  float3 p, ps, pt, pss, pst, ptt;
};

HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
HD float dotf(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

HD SEf eval_bicubic_f(const float4* cp, float s, float t) {
  float su = 1.f - s, sv = 1.f - t;
  float bv[4] = {sv * sv * sv, 3.f * sv * sv * t, 3.f * sv * t * t, t * t * t};
  float dv[4] = {-3.f * sv * sv, 3.f * sv * sv - 6.f * sv * t, 6.f * sv * t - 3.f * t * t, 3.f * t * t};
  float ddv[4] = {6.f * sv, 6.f * t - 12.f * sv, 6.f * sv - 12.f * t, 6.f * t};
  float4 a0 = {0, 0, 0, 0}, a1 = a0, a2 = a0, a3 = a0, a4 = a0, a5 = a0;
  // the rows one at a time (not unrolled): a quarter of the code, which the instruction
  // cache holds beside the rest of the walk (measured: node phase 5% faster); row i's
  // Bernstein value and derivatives in u made in the loop, so that no array is indexed
  // by the loop's counter
#pragma unroll 1
  for (int i = 0; i < 4; i++) {
    float bui, dui, ddui;
    if (i == 0) {
      bui = su * su * su, dui = -3.f * su * su, ddui = 6.f * su;
    } else if (i == 1) {
      bui = 3.f * su * su * s, dui = 3.f * su * su - 6.f * su * s, ddui = 6.f * s - 12.f * su;
    } else if (i == 2) {
      bui = 3.f * su * s * s, dui = 6.f * su * s - 3.f * s * s, ddui = 6.f * su - 12.f * s;
    } else {
      bui = s * s * s, dui = 3.f * s * s, ddui = 6.f * s;
    }
    float4 r0 = {0, 0, 0, 0}, r1 = r0, r2 = r0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float4 c = cp[4 * i + j];
      r0.x += bv[j] * c.x, r0.y += bv[j] * c.y, r0.z += bv[j] * c.z, r0.w += bv[j] * c.w;
      r1.x += dv[j] * c.x, r1.y += dv[j] * c.y, r1.z += dv[j] * c.z, r1.w += dv[j] * c.w;
      r2.x += ddv[j] * c.x, r2.y += ddv[j] * c.y, r2.z += ddv[j] * c.z, r2.w += ddv[j] * c.w;
    }
    a0.x += bui * r0.x, a0.y += bui * r0.y, a0.z += bui * r0.z, a0.w += bui * r0.w;
    a1.x += dui * r0.x, a1.y += dui * r0.y, a1.z += dui * r0.z, a1.w += dui * r0.w;
    a2.x += bui * r1.x, a2.y += bui * r1.y, a2.z += bui * r1.z, a2.w += bui * r1.w;
    a3.x += ddui * r0.x, a3.y += ddui * r0.y, a3.z += ddui * r0.z, a3.w += ddui * r0.w;
    a4.x += dui * r1.x, a4.y += dui * r1.y, a4.z += dui * r1.z, a4.w += dui * r1.w;
    a5.x += bui * r2.x, a5.y += bui * r2.y, a5.z += bui * r2.z, a5.w += bui * r2.w;
  }
  float iw = 1.f / a0.w;
  SEf e;
  e.p = f3(a0.x * iw, a0.y * iw, a0.z * iw);
  e.ps = f3((a1.x - e.p.x * a1.w) * iw, (a1.y - e.p.y * a1.w) * iw, (a1.z - e.p.z * a1.w) * iw);
  e.pt = f3((a2.x - e.p.x * a2.w) * iw, (a2.y - e.p.y * a2.w) * iw, (a2.z - e.p.z * a2.w) * iw);
  e.pss = f3((a3.x - 2.f * e.ps.x * a1.w - e.p.x * a3.w) * iw, (a3.y - 2.f * e.ps.y * a1.w - e.p.y * a3.w) * iw,
             (a3.z - 2.f * e.ps.z * a1.w - e.p.z * a3.w) * iw);
  e.pst = f3((a4.x - e.ps.x * a2.w - e.pt.x * a1.w - e.p.x * a4.w) * iw,
             (a4.y - e.ps.y * a2.w - e.pt.y * a1.w - e.p.y * a4.w) * iw,
             (a4.z - e.ps.z * a2.w - e.pt.z * a1.w - e.p.z * a4.w) * iw);
  e.ptt = f3((a5.x - 2.f * e.pt.x * a2.w - e.p.x * a5.w) * iw, (a5.y - 2.f * e.pt.y * a2.w - e.p.y * a5.w) * iw,
             (a5.z - 2.f * e.pt.z * a2.w - e.p.z * a5.w) * iw);
  return e;
}

// The projected Newton of newton_bicubic in floats (rebased point p), to a step under
// 1e-6 of the square; the double polish takes it from there.
// *last: the patch at the point of the last step's start (within that step of the end).
// Returns whether it converged (a step under 1e-6, or both parameters held).
HDI bool newton_bicubic_f(const float4* cp, float3 p, float* ps_, float* pt_, int iters, SEf* last,
                          int* evals = nullptr) {
  float s = *ps_, t = *pt_;
  bool conv = false;
  for (int it = 0; it < iters; it++) {
    if (evals) ++*evals;
    SEf e = eval_bicubic_f(cp, s, t);
    *last = e;
    float3 r = f3(e.p.x - p.x, e.p.y - p.y, e.p.z - p.z);
    float g0 = dotf(e.ps, r), g1 = dotf(e.pt, r);
    float jss = dotf(e.ps, e.ps), jst = dotf(e.ps, e.pt), jtt = dotf(e.pt, e.pt);
    float h0 = jss + dotf(e.pss, r), h1 = jst + dotf(e.pst, r), h2 = jtt + dotf(e.ptt, r);
    bool hold_s = (s <= 0.f && g0 > 0.f) || (s >= 1.f && g0 < 0.f);
    bool hold_t = (t <= 0.f && g1 > 0.f) || (t >= 1.f && g1 < 0.f);
    float ds, dt;
    if (hold_s && hold_t) {
      conv = true;
      break;
    }
    if (hold_s) {
      ds = 0.f;
      dt = -g1 / (h2 > 0.f ? h2 : fmaxf(jtt, 1e-30f));
    } else if (hold_t) {
      ds = -g0 / (h0 > 0.f ? h0 : fmaxf(jss, 1e-30f));
      dt = 0.f;
    } else {
      if (!(h0 > 0.f && h0 * h2 - h1 * h1 > 0.f)) {
        h0 = jss;
        h1 = jst;
        h2 = jtt;
      }
      float det = h0 * h2 - h1 * h1;
      if (fabsf(det) < 1e-30f) break;
      float id = 1.f / det;
      ds = -(h2 * g0 - h1 * g1) * id;
      dt = -(h0 * g1 - h1 * g0) * id;
    }
    float ns = fminf(fmaxf(s + ds, 0.f), 1.f), nt = fminf(fmaxf(t + dt, 0.f), 1.f);
    float moved = fabsf(ns - s) + fabsf(nt - t);
    s = ns;
    t = nt;
    if (moved < 1e-6f) {
      conv = true;
      break;
    }
  }
  *ps_ = s;
  *pt_ = t;
  return conv;
}

// is_critical at float rounding (1024 units of the last place) for the rebased point p.
HD bool is_critical_f(float3 p, const SEf& e) {
  float3 r = f3(e.p.x - p.x, e.p.y - p.y, e.p.z - p.z);
  float big = fmaxf(fmaxf(fabsf(e.p.x), fabsf(e.p.y)), fabsf(e.p.z)) + fmaxf(fmaxf(fabsf(p.x), fabsf(p.y)), fabsf(p.z));
  float round = 1024.f * 1.1920929e-7f * (big + sqrtf(dotf(r, r)));
  float ls = sqrtf(dotf(e.ps, e.ps)), lt = sqrtf(dotf(e.pt, e.pt));
  return fabsf(dotf(r, e.ps)) <= round * ls && fabsf(dotf(r, e.pt)) <= round * lt;
}

// surface3.rs:565-572 critical
HD bool is_critical(double3 p, const SE& e) {
  double3 r = e.p - p;
  double big = fmax(fmax(fabs(e.p.x), fabs(e.p.y)), fabs(e.p.z)) + fmax(fmax(fabs(p.x), fabs(p.y)), fabs(p.z));
  double round = 1024.0 * 2.220446049250313e-16 * (big + len(r));
  double ls = len(e.ps), lt = len(e.pt);
  return fabs(dot(r, e.ps)) <= (round + 1e-12 * ls) * ls && fabs(dot(r, e.pt)) <= (round + 1e-12 * lt) * lt;
}

// The same with each tangent's rounding allowance raised by how much shorter than
// `scale` (the part's size) the tangent is. Beside a pole the tangent along the
// collapsing side is the difference of nearly equal control points, its direction
// known only to about eps * scale / |S_s|, and the reference's allowance rejects the
// nearest point there (its residual is that rounding); used for sub-patches with a
// side on a pole's.
HD bool is_critical_scaled(double3 p, const SE& e, double scale) {
  double3 r = e.p - p;
  double big = fmax(fmax(fabs(e.p.x), fabs(e.p.y)), fabs(e.p.z)) + fmax(fmax(fabs(p.x), fabs(p.y)), fabs(p.z));
  double round = 1024.0 * 2.220446049250313e-16 * (big + len(r));
  double ls = len(e.ps), lt = len(e.pt);
  double rs = round * fmax(1.0, scale / ls), rt = round * fmax(1.0, scale / lt);
  return fabs(dot(r, e.ps)) <= (rs + 1e-12 * ls) * ls && fabs(dot(r, e.pt)) <= (rt + 1e-12 * lt) * lt;
}

// Interval product.
HD void imul(double alo, double ahi, double blo, double bhi, double* lo, double* hi) {
  double p0 = alo * blo, p1 = alo * bhi, p2 = ahi * blo, p3 = ahi * bhi;
  *lo = fmin(fmin(p0, p1), fmin(p2, p3));
  *hi = fmax(fmax(p0, p1), fmax(p2, p3));
}

// Whether |S - p|^2 is strictly convex over the sub-patch for every p in [plo, phi]:
// in the sub-patch's scaled parameters its Hessian is G + (S - p).S_ij, whose least
// eigenvalue is at least lam + min_i(E_ii - |E_12|) (Gershgorin) with E_ij the interval
// of (S - p).S_ij over S in the control box and S_ij in their bounds
// (surface3.rs:814-845 convex_radius, tightened by the offset box as gpu.wgsl:1547-1604).
// Never for a sub-patch with a side on a pole's: the metric degenerates there, the
// bound is at best semi-definite, and projected Newton can rest on the pole with the
// nearest point a little inside; such a sub-patch is always searched by subdivision.
HD bool sub_convex(const DSub& s, double3 plo, double3 phi) {
  if (s.pole_sides != 0) return false;
  double dlo[3] = {s.box[0] - phi.x, s.box[1] - phi.y, s.box[2] - phi.z};
  double dhi[3] = {s.box[3] - plo.x, s.box[4] - plo.y, s.box[5] - plo.z};
  double elo[3], ehi[3];
  for (int m = 0; m < 3; m++) {
    elo[m] = ehi[m] = 0.0;
    for (int k = 0; k < 3; k++) {
      double lo, hi;
      imul(dlo[k], dhi[k], s.d2[m][k][0], s.d2[m][k][1], &lo, &hi);
      elo[m] += lo;
      ehi[m] += hi;
    }
  }
  double off = fmax(fabs(elo[1]), fabs(ehi[1]));
  double lmin = s.lam + fmin(elo[0] - off, elo[2] - off);
  return lmin > 1e-6 * s.lam;
}

// The same for a spline edge piece: |C'|^2 + (C - p).C'' > 0 over it.
HD bool piece_convex(const DPiece& c, double3 plo, double3 phi) {
  double dlo[3] = {c.box[0] - phi.x, c.box[1] - phi.y, c.box[2] - phi.z};
  double dhi[3] = {c.box[3] - plo.x, c.box[4] - plo.y, c.box[5] - plo.z};
  double e = 0.0;
  for (int k = 0; k < 3; k++) {
    double lo, hi;
    imul(dlo[k], dhi[k], c.d2[k][0], c.d2[k][1], &lo, &hi);
    e += lo;
  }
  return c.lam + e > 1e-6 * c.lam;
}

// ---------------------------------------------------------------- subdivision fallback

// The control points of the part [s0, s1] x [t0, t1] of a bicubic (de Casteljau: the
// curve's part past s0, then the first (s1 - s0) / (1 - s0) of that).
HD void part4(double4 c[4], double a, double b) {
  // keep [a, 1]: the triangle's last points, c[i] = P_i^(3-i) (in place, i rising)
  if (a > 0.0) {
#pragma unroll
    for (int level = 1; level <= 3; level++)
#pragma unroll
      for (int i = 0; i <= 3 - level; i++) {
        c[i].x = (1 - a) * c[i].x + a * c[i + 1].x, c[i].y = (1 - a) * c[i].y + a * c[i + 1].y;
        c[i].z = (1 - a) * c[i].z + a * c[i + 1].z, c[i].w = (1 - a) * c[i].w + a * c[i + 1].w;
      }
  }
  // keep [0, (b - a) / (1 - a)] of that: the triangle's first points (in place, i falling)
  double t = a < 1.0 ? (b - a) / (1.0 - a) : 1.0;
  if (t < 1.0) {
#pragma unroll
    for (int level = 1; level <= 3; level++)
#pragma unroll
      for (int i = 3; i >= level; i--) {
        c[i].x = (1 - t) * c[i - 1].x + t * c[i].x, c[i].y = (1 - t) * c[i - 1].y + t * c[i].y;
        c[i].z = (1 - t) * c[i - 1].z + t * c[i].z, c[i].w = (1 - t) * c[i - 1].w + t * c[i].w;
      }
  }
}

HDI void extract_rect(const double4* cp, double s0, double s1, double t0, double t1, double4* q) {
#pragma unroll
  for (int j = 0; j < 4; j++) {
    double4 c[4] = {cp[j], cp[4 + j], cp[8 + j], cp[12 + j]};
    part4(c, s0, s1);
#pragma unroll
    for (int i = 0; i < 4; i++) q[4 * i + j] = c[i];
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double4 c[4] = {q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
    part4(c, t0, t1);
#pragma unroll
    for (int j = 0; j < 4; j++) q[4 * i + j] = c[j];
  }
}

// The convexity certificate of a bicubic computed on the device (surface3.rs:862-925
// patch_bounds, as the pack builder computes it): writes a DSub-like bound set.
HDI bool rect_bounds(const double4* q, double* box, double& lam, double d2[3][3][2], double d1[2][3][2]) {
  double cx = 0, cy = 0, cz = 0;
  for (int k = 0; k < 16; k++) {
    double iw = 1.0 / q[k].w;
    double x = q[k].x * iw, y = q[k].y * iw, z = q[k].z * iw;
    cx += x, cy += y, cz += z;
    box[0] = k ? fmin(box[0], x) : x, box[1] = k ? fmin(box[1], y) : y, box[2] = k ? fmin(box[2], z) : z;
    box[3] = k ? fmax(box[3], x) : x, box[4] = k ? fmax(box[4], y) : y, box[5] = k ? fmax(box[5], z) : z;
  }
  cx *= 1.0 / 16, cy *= 1.0 / 16, cz *= 1.0 / 16;
  auto Q = [&](int i, int j, int c) {
    const double4& h = q[4 * i + j];
    return c == 0 ? h.x - cx * h.w : c == 1 ? h.y - cy * h.w : c == 2 ? h.z - cz * h.w : h.w;
  };
  // hulls of the homogeneous derivatives' Bernstein coefficients
  double As[4][2], At[4][2], Ass[4][2], Ast[4][2], Att[4][2], A[4][2];
  for (int c = 0; c < 4; c++) {
    A[c][0] = As[c][0] = At[c][0] = Ass[c][0] = Ast[c][0] = Att[c][0] = INFINITY;
    A[c][1] = As[c][1] = At[c][1] = Ass[c][1] = Ast[c][1] = Att[c][1] = -INFINITY;
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        double x = Q(i, j, c);
        A[c][0] = fmin(A[c][0], x), A[c][1] = fmax(A[c][1], x);
        if (i < 3) {
          double y = 3.0 * (Q(i + 1, j, c) - x);
          As[c][0] = fmin(As[c][0], y), As[c][1] = fmax(As[c][1], y);
        }
        if (j < 3) {
          double y = 3.0 * (Q(i, j + 1, c) - x);
          At[c][0] = fmin(At[c][0], y), At[c][1] = fmax(At[c][1], y);
        }
        if (i < 2) {
          double y = 6.0 * (Q(i + 2, j, c) - 2.0 * Q(i + 1, j, c) + x);
          Ass[c][0] = fmin(Ass[c][0], y), Ass[c][1] = fmax(Ass[c][1], y);
        }
        if (i < 3 && j < 3) {
          double y = 9.0 * (Q(i + 1, j + 1, c) - Q(i + 1, j, c) - Q(i, j + 1, c) + x);
          Ast[c][0] = fmin(Ast[c][0], y), Ast[c][1] = fmax(Ast[c][1], y);
        }
        if (j < 2) {
          double y = 6.0 * (Q(i, j + 2, c) - 2.0 * Q(i, j + 1, c) + x);
          Att[c][0] = fmin(Att[c][0], y), Att[c][1] = fmax(Att[c][1], y);
        }
      }
  }
  if (!(A[3][0] > 0.0)) return false;
  double wl = 1.0 / A[3][1], wh = 1.0 / A[3][0];
  auto sub = [](const double* a, const double* b, double* r) { r[0] = a[0] - b[1], r[1] = a[1] - b[0]; };
  auto mul = [](const double* a, const double* b, double* r) { imul(a[0], a[1], b[0], b[1], &r[0], &r[1]); };
  double S[3][2] = {{box[0] - cx, box[3] - cx}, {box[1] - cy, box[4] - cy}, {box[2] - cz, box[5] - cz}};
  double ss[3][2], st[3][2], tmp[2], tmp2[2], winv[2] = {wl, wh};
  for (int k = 0; k < 3; k++) {
    mul(S[k], As[3], tmp), sub(As[k], tmp, tmp2), mul(tmp2, winv, ss[k]);
    mul(S[k], At[3], tmp), sub(At[k], tmp, tmp2), mul(tmp2, winv, st[k]);
  }
  double sss[3][2], sst[3][2], stt[3][2], t3[2];
  for (int k = 0; k < 3; k++) {
    mul(ss[k], As[3], tmp), tmp[0] *= 2, tmp[1] *= 2, sub(Ass[k], tmp, tmp2), mul(S[k], Ass[3], tmp), sub(tmp2, tmp, t3),
        mul(t3, winv, sss[k]);
    mul(ss[k], At[3], tmp), sub(Ast[k], tmp, tmp2), mul(st[k], As[3], tmp), sub(tmp2, tmp, t3), mul(S[k], Ast[3], tmp),
        sub(t3, tmp, tmp2), mul(tmp2, winv, sst[k]);
    mul(st[k], At[3], tmp), tmp[0] *= 2, tmp[1] *= 2, sub(Att[k], tmp, tmp2), mul(S[k], Att[3], tmp), sub(tmp2, tmp, t3),
        mul(t3, winv, stt[k]);
  }
  SE e0 = eval_bicubic(q, 0.5, 0.5);
  double sa = len(e0.ps), sb = len(e0.pt);
  sa = sa > 0 ? sa : 1.0, sb = sb > 0 ? sb : 1.0;
  double p0[3] = {e0.ps.x / sa, e0.ps.y / sa, e0.ps.z / sa}, t0[3] = {e0.pt.x / sb, e0.pt.y / sb, e0.pt.z / sb};
  double ga = 0, gc = 0, gbl = 0, gbh = 0, dev = 0;
  for (int k = 0; k < 3; k++) {
    double a0 = ss[k][0] / sa, a1 = ss[k][1] / sa, b0 = st[k][0] / sb, b1 = st[k][1] / sb;
    double ma = (a0 <= 0 && a1 >= 0) ? 0.0 : fmin(fabs(a0), fabs(a1));
    double mb = (b0 <= 0 && b1 >= 0) ? 0.0 : fmin(fabs(b0), fabs(b1));
    ga += ma * ma, gc += mb * mb;
    double lo, hi;
    imul(a0, a1, b0, b1, &lo, &hi);
    gbl += lo, gbh += hi;
    dev += pow(fmax(fabs(a0 - p0[k]), fabs(a1 - p0[k])), 2) + pow(fmax(fabs(b0 - t0[k]), fabs(b1 - t0[k])), 2);
    d1[0][k][0] = a0, d1[0][k][1] = a1, d1[1][k][0] = b0, d1[1][k][1] = b1;
    d2[0][k][0] = sss[k][0] / (sa * sa), d2[0][k][1] = sss[k][1] / (sa * sa);
    d2[1][k][0] = sst[k][0] / (sa * sb), d2[1][k][1] = sst[k][1] / (sa * sb);
    d2[2][k][0] = stt[k][0] / (sb * sb), d2[2][k][1] = stt[k][1] / (sb * sb);
  }
  double gb = fmax(fabs(gbl), fabs(gbh));
  double by_entries = 0.5 * ((ga + gc) - sqrt((ga - gc) * (ga - gc) + 4.0 * gb * gb));
  double a0 = p0[0] * p0[0] + p0[1] * p0[1] + p0[2] * p0[2], c0 = t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2];
  double b0 = p0[0] * t0[0] + p0[1] * t0[1] + p0[2] * t0[2];
  double sigma0 = sqrt(fmax(0.5 * ((a0 + c0) - sqrt((a0 - c0) * (a0 - c0) + 4.0 * b0 * b0)), 0.0));
  double by_middle = pow(fmax(sigma0 - sqrt(dev), 0.0), 2);
  lam = fmax(by_entries, by_middle);
  return true;
}

// Whether |S - p|^2 is strictly convex over a part whose bounds are given (sub_convex
// for a part computed on the device).
HDI bool rect_convex(const double* box, double lam, const double d2[3][3][2], double3 p) {
  double dlo[3] = {box[0] - p.x, box[1] - p.y, box[2] - p.z}, dhi[3] = {box[3] - p.x, box[4] - p.y, box[5] - p.z};
  double elo[3], ehi[3];
  for (int m = 0; m < 3; m++) {
    elo[m] = ehi[m] = 0.0;
    for (int k = 0; k < 3; k++) {
      double lo, hi;
      imul(dlo[k], dhi[k], d2[m][k][0], d2[m][k][1], &lo, &hi);
      elo[m] += lo, ehi[m] += hi;
    }
  }
  double off = fmax(fabs(elo[1]), fabs(ehi[1]));
  return lam + fmin(elo[0] - off, elo[2] - off) > 1e-6 * lam;
}

// Whether |S - p|^2 has no critical point on the part: along the unit direction (a, b)
// of the gradient at the part's Newton point, a g_s + b g_t = (S - p).(a S_s + b S_t)
// (scaled parameters) keeps one strict sign over the part, by interval arithmetic on
// the control box and the tangents' bounds (the reference's no_critical_point,
// surface3.rs:694-730, tests the same combination on its Bernstein form).
HDI bool rect_no_critical(const double* box, const double d1[2][3][2], double3 p, double a, double b) {
  double lo = 0.0, hi = 0.0;
  double pp[3] = {p.x, p.y, p.z};
  for (int k = 0; k < 3; k++) {
    double ulo = a >= 0 ? a * d1[0][k][0] : a * d1[0][k][1], uhi = a >= 0 ? a * d1[0][k][1] : a * d1[0][k][0];
    double vlo = b >= 0 ? b * d1[1][k][0] : b * d1[1][k][1], vhi = b >= 0 ? b * d1[1][k][1] : b * d1[1][k][0];
    double l, h;
    imul(box[k] - pp[k], box[3 + k] - pp[k], ulo + vlo, uhi + vhi, &l, &h);
    lo += l, hi += h;
  }
  double scale = fmax(fabs(lo), fabs(hi));
  return lo > 1e-12 * scale || hi < -1e-12 * scale;
}

// ---------------------------------------------------------------- rational cubic pieces

struct CE {
  double3 p, d1, d2;
};

HD CE eval_cubic(const double (*c)[4], double s) {
  double b[4], d[4], dd[4];
  bern3(s, b, d, dd);
  double a[3][4] = {{0}};
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      a[0][k] += b[i] * c[i][k];
      a[1][k] += d[i] * c[i][k];
      a[2][k] += dd[i] * c[i][k];
    }
  double iw = 1.0 / a[0][3];
  CE e;
  e.p = mk(a[0][0], a[0][1], a[0][2]) * iw;
  e.d1 = (mk(a[1][0], a[1][1], a[1][2]) - e.p * a[1][3]) * iw;
  e.d2 = (mk(a[2][0], a[2][1], a[2][2]) - e.d1 * (2.0 * a[1][3]) - e.p * a[2][3]) * iw;
  return e;
}

// curve3.rs:191-213 Bez3::newton
HDI double newton_cubic(const double (*c)[4], double3 p, double s, bool* conv) {
  *conv = false;
  for (int it = 0; it < 40; it++) {
    CE e = eval_cubic(c, s);
    double3 r = e.p - p;
    double f = dot(e.d1, r);
    double fp = dot(e.d2, r) + dot(e.d1, e.d1);
    if (fp <= 0.0) fp = dot(e.d1, e.d1);
    if (fabs(fp) < 1e-300) break;
    double ns = fmin(fmax(s - f / fp, 0.0), 1.0);
    // a step under 1e-13: the reference's Bez3::newton (curve3.rs:191-213) steps on to
    // 1e-15 or 40 steps, but on a short piece (|C'| of a fraction of a mm) the rounding
    // of f / fp alone moves s by more than 1e-15, so that test fails where the solve has
    // long converged; the point found is the same to within that rounding
    if (fabs(ns - s) < 1e-13) {
      *conv = true;
      return ns;
    }
    s = ns;
  }
  return s;
}

}  // namespace icam

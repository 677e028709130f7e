// The exact field at one point over a list of candidate features (double precision):
// the per-feature evaluators of eval.cuh combined by the reference's rules, and the
// lower bounds the culling uses.
#pragma once

#include "eval.cuh"

namespace icam {

constexpr double SQRT3 = 1.7320508075688772;

// A read brick (cell side h) whose centre distance dc puts every node on one side of the
// surface by more than an i16 step of the clamp (the field is 1-Lipschitz and a node is
// at most 4h sqrt(3) from the centre): the brick packs to AIR (dc > 0) or SOLID whatever
// its nodes read, every exactly read value quantising to at least one step of dc's sign.
// `extra` widens the test (the decision leaves room for the brick kernel's own rounding).
__host__ __device__ inline bool settles_by_sign(double dc, double h, double clamp, double extra = 0.0) {
  return fabs(dc) - 4.0 * h * SQRT3 > clamp * (1.0 / 32767.0) + 1e-9 * (1.0 + fabs(dc)) + extra;
}

// What a point's evaluation keeps: the least distance found, its signed value, and
// the least lower bound among features it could not decide.
struct Acc {
  double best;   // |d| of the nearest answer so far (the cutoff for the next feature)
  double sd;     // its signed distance (NaN while nothing nearer than the cap is known)
  double und;    // least lower bound of an undecided feature
  int why;       // why-code of that undecided feature (gpu.wgsl:1623-1628: 6 stack, 8 budget)
  double ub;     // least distance of any face point seen: the answer is no farther
  // Features whose certificate fails here, left for subdivision until every cheaper
  // feature has tightened the bound (codes and their lower bounds).
  int nd;
  uint32_t dcode[8];
  double dlb[8];
  bool record;  // only record a failing certificate's bound in und (the caller walks the tree later)
};

constexpr int MAX_DEFER = 8;

HD void acc_init(Acc& A, double cap) {
  A.best = cap;
  A.sd = NAN;
  A.und = INFINITY;
  A.why = 0;
  A.ub = INFINITY;
  A.nd = 0;
  A.record = false;
}

// Lower bound on the distance from c to a feature, by kind (solid3.rs:1661-1690
// candidates): an analytic face's untrimmed surface, a line or arc edge's exact
// distance, a vertex's, the box of anything else.
HDI double item_lb(const DPack& P, uint32_t code, double3 c) {
  uint32_t k = code >> IK_SHIFT, i = code & IK_MASK;
  switch (k) {
    case IK_FACE: {
      const DFace& f = P.faces[i];
      double b = box_dist(c, f.box);
      double3 q, n;
      double u, v;
      double d = b;
      if (analytic_foot(f, c, &q, &n, &u, &v)) d = fmax(d, len(c - q));
      else if (f.kind == S_CONE) {
        double3 apex = ld3(f.o) + ld3(f.z) * (-f.a / tan(f.b));
        d = fmax(d, len(c - apex));
      }
      return d;
    }
    case IK_SUB:
      return box_dist(c, P.subs[i].box);
    case IK_EDGE: {
      const DEdge& e = P.edges[i];
      if (e.kind == 0) {
        double3 a = ld3(e.a), ab = ld3(e.b) - a;
        double l2 = dot(ab, ab);
        double t = l2 > 0.0 ? fmin(fmax(dot(c - a, ab) / l2, 0.0), 1.0) : 0.0;
        return len(c - (a + ab * t));
      } else {
        double3 d = c - ld3(e.o);
        double lx = dot(d, ld3(e.x)), ly = dot(d, ld3(e.y)), lz = dot(d, ld3(e.z));
        double rho = sqrt(lx * lx + ly * ly);
        // distance to the whole circle: a lower bound on the arc's
        return sqrt((rho - e.r) * (rho - e.r) + lz * lz);
      }
    }
    case IK_PIECE:
      return box_dist(c, P.pieces[i].box);
    default: {
      const DVert& v = P.verts[i];
      return len(c - ld3(v.p));
    }
  }
}

// The outward normal of face fi at a point q of one of its edges (solid3.rs:1891-1897
// normal_at): analytic faces in closed form; a B-spline face by Newton on the span
// holding the seed (u, v), which the pack stores per edge-piece end.
HDI double3 face_normal_at(const DPack& P, int fi, double3 q, double u, double v) {
  const DFace& f = P.faces[fi];
  if (f.kind != S_NURBS) {
    double3 qq, n;
    double uu, vv;
    if (analytic_foot(f, q, &qq, &n, &uu, &vv)) return n;
    return mk(0, 0, 0);
  }
  const DNurbs& nb = P.nurbs[f.nurbs];
  const double* ub = P.breaks + nb.first_break;
  const double* vb = ub + nb.nsu + 1;
  int a = 0, b = 0;
  for (int i = nb.nsu - 1; i >= 0; i--)
    if (ub[i] <= u) {
      a = i;
      break;
    }
  for (int j = nb.nsv - 1; j >= 0; j--)
    if (vb[j] <= v) {
      b = j;
      break;
    }
  const double4* cp = P.span_cp + 16 * size_t(nb.first_span + a * nb.nsv + b);
  double s = fmin(fmax((u - ub[a]) / (ub[a + 1] - ub[a]), 0.0), 1.0);
  double t = fmin(fmax((v - vb[b]) / (vb[b + 1] - vb[b]), 0.0), 1.0);
  bool conv;
  newton_bicubic(cp, q, &s, &t, 8, &conv);
  SE e = eval_bicubic(cp, s, t);
  return unit(cross(e.ps, e.pt)) * f.sense;
}

HD void take(Acc& A, double d, double signed_d) {
  A.best = d;
  A.sd = signed_d;
}

HD void undecided(Acc& A, double lb, int why) {
  if (lb < A.und) {
    A.und = lb;
    A.why = why;
  }
}

// A sub-patch the certificate does not cover at p: branch and bound over its parts
// (surface3.rs:1214-1297 closest_trimmed, restricted to one sub-patch). Each part gets
// its own interval bounds; a part they certify convex at p is answered by Newton alone,
// any other gives a bound (its Newton point when that lies in the face), a slab bound
// along the direction to it (surface3.rs:973) and splits in four. Budget and stack
// give up with why-codes 8 and 6 (gpu.wgsl:1623-1628).
HDI void bb_sub(const DPack& P, int si, double3 p, Acc& A) {
  const DSub& s = P.subs[si];
  const double4* cp = P.sub_cp + 16 * size_t(si);
  const DFace& f = P.faces[s.face];
  struct R {
    double s0, s1, t0, t1, lb;
    int depth;
  };
  R st[64];
  int sp = 0;
  st[sp++] = {0.0, 1.0, 0.0, 1.0, box_dist(p, s.box), 0};
  // the least distance of a point of this face found by this search (best_d); the
  // nearest boundary point seen anywhere (ub) only prunes what lies past it
  double bound = A.best;
  const double far = A.ub + DIST_EPS;
  int pops = 0;
  double4 q[16];
  while (sp > 0) {
    R r = st[--sp];
    if (r.lb >= bound - DIST_EPS || r.lb > far) continue;
    if (++pops > 4096) {
      undecided(A, r.lb, 8);
      return;
    }
    extract_rect(cp, r.s0, r.s1, r.t0, r.t1, q);
    double box[6], lam, d2[3][3][2], d1[2][3][2];
    if (!rect_bounds(q, box, lam, d2, d1)) {
      undecided(A, r.lb, 1);
      continue;
    }
    double lb = fmax(box_dist(p, box), r.lb);
    if (lb >= bound - DIST_EPS || lb > far) continue;
    // a part touching a pole's side: never certified convex, never cleared by the
    // critical-point test (the distance's minimum at the pole need not be critical)
    const bool pole = ((s.pole_sides & 1) && r.s0 == 0.0) || ((s.pole_sides & 2) && r.s1 == 1.0) ||
                      ((s.pole_sides & 4) && r.t0 == 0.0) || ((s.pole_sides & 8) && r.t1 == 1.0);
    bool cert = !pole && rect_convex(box, lam, d2, p);
    double ss = 0.5, tt = 0.5;
    bool conv;
    newton_bicubic(q, p, &ss, &tt, cert ? 16 : 12, &conv);
    SE e = eval_bicubic(q, ss, tt);
    double d = len(e.p - p);
    double3 n = cross(e.ps, e.pt);
    if (d < bound) {
      double u = s.u0 + (r.s0 + ss * (r.s1 - r.s0)) * (s.u1 - s.u0);
      double v = s.v0 + (r.t0 + tt * (r.t1 - r.t0)) * (s.v1 - s.v0);
      if (s.klass == 1 || trim_inside(P, f, u, v)) {
        bound = d;
        A.ub = fmin(A.ub, d);
        // beside a pole the tangent along the collapsing side is known only to the
        // rounding of nearly equal control points: its allowance scales with the part
        const bool crit = s.pole_sides ? is_critical_scaled(p, e, len(mk(box[3], box[4], box[5]) - mk(box[0], box[1], box[2])))
                                       : is_critical(p, e);
        if (d < A.best && crit && len(n) > 0.0) {
          double3 nn = unit(n) * f.sense;
          take(A, d, d * sgn(dot(p - e.p, nn)));
        }
      }
    }
    if (cert && conv) continue;  // its one minimum is known
    // no critical point in the part: nothing of the face's is here (surface3.rs:1280-1282)
    if (!pole) {
      double3 r = e.p - p;
      double gs = dot(r, e.ps), gt = dot(r, e.pt), gl = sqrt(gs * gs + gt * gt);
      if (gl > 0.0 && rect_no_critical(box, d1, p, gs / gl, gt / gl)) continue;
    }
    double3 dir = d > 1e-12 ? (p - e.p) * (1.0 / d) : unit(n);
    double slab = INFINITY;
    for (int k = 0; k < 16; k++) {
      double iw = 1.0 / q[k].w;
      slab = fmin(slab, dot(p - mk(q[k].x * iw, q[k].y * iw, q[k].z * iw), dir));
    }
    if (slab >= bound - DIST_EPS || slab > far || r.depth >= 40) continue;
    if (sp + 4 > 64) {
      undecided(A, fmax(lb, slab), 6);
      continue;
    }
    double sm = 0.5 * (r.s0 + r.s1), tm = 0.5 * (r.t0 + r.t1), cl = fmax(lb, slab);
    st[sp++] = {r.s0, sm, r.t0, tm, cl, r.depth + 1};
    st[sp++] = {r.s0, sm, tm, r.t1, cl, r.depth + 1};
    st[sp++] = {sm, r.s1, r.t0, tm, cl, r.depth + 1};
    st[sp++] = {sm, r.s1, tm, r.t1, cl, r.depth + 1};
  }
}

// A spline edge piece the certificate does not cover at p: the nearest point of the
// piece by branch and bound over its halves (curve3.rs:408-471 Spline3::closest), taken
// when it is not one of the edge's ends.
HDI void bb_piece(const DPack& P, int pi, double3 p, Acc& A) {
  const DPiece& c = P.pieces[pi];
  struct R {
    double a, b, lb;
    int depth;
  };
  R st[64];
  int sp = 0;
  st[sp++] = {0.0, 1.0, 0.0, 0};
  double bound = A.best, best_s = -1.0;
  const double far = A.ub + 1e-12;  // parts past the nearest boundary point seen cannot answer
  double3 best_q = mk(0, 0, 0);
  int pops = 0;
  while (sp > 0) {
    R r = st[--sp];
    if (r.lb >= bound - 1e-12 || r.lb > far) continue;
    if (++pops > 4096) {
      undecided(A, r.lb, 8);
      return;
    }
    double4 z[4] = {make_double4(c.cp[0][0], c.cp[0][1], c.cp[0][2], c.cp[0][3]),
                    make_double4(c.cp[1][0], c.cp[1][1], c.cp[1][2], c.cp[1][3]),
                    make_double4(c.cp[2][0], c.cp[2][1], c.cp[2][2], c.cp[2][3]),
                    make_double4(c.cp[3][0], c.cp[3][1], c.cp[3][2], c.cp[3][3])};
    part4(z, r.a, r.b);
    double zc[4][4];
    for (int k = 0; k < 4; k++) zc[k][0] = z[k].x, zc[k][1] = z[k].y, zc[k][2] = z[k].z, zc[k][3] = z[k].w;
    double3 a = mk(z[0].x / z[0].w, z[0].y / z[0].w, z[0].z / z[0].w);
    double3 b = mk(z[3].x / z[3].w, z[3].y / z[3].w, z[3].z / z[3].w);
    double3 ab = b - a;
    double l2 = dot(ab, ab);
    double f0 = l2 > 0.0 ? fmin(fmax(dot(p - a, ab) / l2, 0.0), 1.0) : 0.5;
    double thick = 0.0;
    for (int k = 0; k < 4; k++) {
      double3 x = mk(z[k].x / z[k].w, z[k].y / z[k].w, z[k].z / z[k].w);
      double t = l2 > 0.0 ? fmin(fmax(dot(x - a, ab) / l2, 0.0), 1.0) : 0.0;
      thick = fmax(thick, len(x - (a + ab * t)));
    }
    // the part lies within `thick` of its chord (curve3.rs:452-459)
    double own = fmax(r.lb, len(p - (a + ab * f0)) - thick);
    if (own >= bound - 1e-12 || own > far) continue;
    double seeds[3] = {f0, 0.0, 1.0};
    for (int k = 0; k < 5; k++) {
      bool conv;
      double sl = k < 3 ? newton_cubic(zc, p, seeds[k], &conv) : (k == 3 ? 0.0 : 1.0);
      double3 x = eval_cubic(zc, sl).p;
      double d = len(x - p);
      if (d < bound) {
        bound = d;
        best_s = r.a + sl * (r.b - r.a);
        best_q = x;
      }
    }
    if (r.depth < 40 && thick > 1e-12) {
      if (sp + 2 > 64) {
        undecided(A, r.lb, 6);
        continue;
      }
      double m = 0.5 * (r.a + r.b);
      double lbc = own;
      st[sp++] = {m, r.b, lbc, r.depth + 1};
      st[sp++] = {r.a, m, lbc, r.depth + 1};
    }
  }
  if (best_s < 0.0 || !(bound < A.best)) return;
  A.ub = fmin(A.ub, bound);
  if ((c.first && best_s <= 0.0) || (c.last && best_s >= 1.0)) return;
  const DEdge& ed = P.edges[c.edge];
  double3 pn = mk(0, 0, 0);
  for (int side = 0; side < 2; side++) {
    int fi = side == 0 ? ed.f0 : ed.f1;
    double u = c.uv[side][0][0] + best_s * (c.uv[side][1][0] - c.uv[side][0][0]);
    double v = c.uv[side][0][1] + best_s * (c.uv[side][1][1] - c.uv[side][0][1]);
    pn = pn + face_normal_at(P, fi, best_q, u, v);
  }
  take(A, bound, bound * sgn(dot(p - best_q, pn)));
}

HDI void subdivide(const DPack& P, uint32_t code, double3 p, Acc& A) {
  if ((code >> IK_SHIFT) == IK_SUB)
    bb_sub(P, int(code & IK_MASK), p, A);
  else
    bb_piece(P, int(code & IK_MASK), p, A);
}

// Leaves a feature whose certificate fails at p for later (subdivided now when the
// list is full).
HDI void defer(const DPack& P, uint32_t code, double lb, double3 p, Acc& A) {
  if (A.record) {
    A.und = fmin(A.und, lb);
    return;
  }
  if (A.nd < MAX_DEFER) {
    A.dcode[A.nd] = code;
    A.dlb[A.nd] = lb;
    A.nd++;
    return;
  }
  subdivide(P, code, p, A);
}

// The features left for later, nearest bound first, while they can still hold a
// nearer point.
HDI void resolve(const DPack& P, double3 p, Acc& A) {
  while (A.nd > 0) {
    int k = 0;
    for (int j = 1; j < A.nd; j++)
      if (A.dlb[j] < A.dlb[k]) k = j;
    uint32_t code = A.dcode[k];
    double lb = A.dlb[k];
    A.nd--;
    A.dcode[k] = A.dcode[A.nd];
    A.dlb[k] = A.dlb[A.nd];
    if (lb >= A.best - DIST_EPS || lb > A.ub + DIST_EPS) continue;
    subdivide(P, code, p, A);
  }
}

// One candidate for point p. `cert` is a precomputed convexity verdict (1 certified
// for every node of the brick, 0 unknown); seeds hold a Newton start for sub-patches.
HDI void eval_item(const DPack& P, uint32_t code, double3 p, Acc& A, int cert, double s0, double t0) {
  uint32_t k = code >> IK_SHIFT, i = code & IK_MASK;
  switch (k) {
    case IK_FACE: {
      const DFace& f = P.faces[i];
      if (box_dist(p, f.box) >= A.best) return;
      double3 q, n;
      double u, v;
      if (!analytic_foot(f, p, &q, &n, &u, &v)) return;
      double d = len(p - q);
      if (!(d < A.best)) return;
      if (!trim_inside(P, f, u, v)) return;
      take(A, d, d * sgn(dot(p - q, n)));
      return;
    }
    case IK_SUB: {
      const DSub& s = P.subs[i];
      double lb = box_dist(p, s.box);
      if (lb >= A.best) return;
      if (!cert && !sub_convex(s, p, p)) {
        defer(P, code, lb, p, A);
        return;
      }
      const double4* cp = P.sub_cp + 16 * size_t(i);
      double ss = s0, tt = t0;
      bool conv;
      newton_bicubic(cp, p, &ss, &tt, 16, &conv);
      if (!conv) {
        defer(P, code, lb, p, A);
        return;
      }
      SE e = eval_bicubic(cp, ss, tt);
      double d = len(e.p - p);
      if (!(d < A.best) || !is_critical(p, e)) return;
      double3 n = cross(e.ps, e.pt);
      if (!(len(n) > 0.0)) return;
      if (s.klass != 1) {
        const DFace& f = P.faces[s.face];
        if (!trim_inside(P, f, s.u0 + ss * (s.u1 - s.u0), s.v0 + tt * (s.v1 - s.v0))) return;
      }
      n = unit(n) * P.faces[s.face].sense;
      take(A, d, d * sgn(dot(p - e.p, n)));
      return;
    }
    case IK_EDGE: {
      const DEdge& e = P.edges[i];
      double3 q;
      double d;
      if (e.kind == 0) {  // curve3.rs:527-540
        double3 a = ld3(e.a), ab = ld3(e.b) - a;
        double l2 = dot(ab, ab);
        double t = l2 > 0.0 ? fmin(fmax(dot(p - a, ab) / l2, 0.0), 1.0) : 0.0;
        if (t <= 0.0 || t >= 1.0) return;
        q = a + ab * t;
        d = len(p - q);
      } else {  // curve3.rs:541-556
        double3 dd = p - ld3(e.o);
        double lx = dot(dd, ld3(e.x)), ly = dot(dd, ld3(e.y));
        if (lx == 0.0 && ly == 0.0) return;
        double t = atan2(ly, lx);
        bool full = fabs(fabs(e.sweep) - 6.283185307179586) < 1e-12;
        if (!full) {
          double dt = e.sweep >= 0.0 ? t - e.t0 : e.t0 - t;
          double m = fmod(dt, 6.283185307179586);
          if (m < 0) m += 6.283185307179586;
          if (!(m <= fabs(e.sweep))) return;
        }
        double sn, cs;
        sincos(t, &sn, &cs);
        q = ld3(e.o) + ld3(e.x) * (e.r * cs) + ld3(e.y) * (e.r * sn);
        d = len(p - q);
      }
      if (!(d < A.best)) return;
      double3 pn = face_normal_at(P, e.f0, q, 0, 0) + face_normal_at(P, e.f1, q, 0, 0);
      take(A, d, d * sgn(dot(p - q, pn)));
      return;
    }
    case IK_PIECE: {
      const DPiece& c = P.pieces[i];
      double lb = box_dist(p, c.box);
      if (lb >= A.best) return;
      double3 a = mk(c.cp[0][0] / c.cp[0][3], c.cp[0][1] / c.cp[0][3], c.cp[0][2] / c.cp[0][3]);
      double3 b = mk(c.cp[3][0] / c.cp[3][3], c.cp[3][1] / c.cp[3][3], c.cp[3][2] / c.cp[3][3]);
      double3 ab = b - a;
      double l2 = dot(ab, ab);
      double f0 = l2 > 0.0 ? fmin(fmax(dot(p - a, ab) / l2, 0.0), 1.0) : 0.5;
      double chord = len(p - (a + ab * f0));
      if (chord - c.thick >= A.best) return;
      if (!piece_convex(c, p, p)) {
        defer(P, code, fmax(lb, chord - c.thick), p, A);
        return;
      }
      bool conv;
      double s = newton_cubic(c.cp, p, f0, &conv);
      CE e = eval_cubic(c.cp, s);
      double d = len(e.p - p);
      // the raw ends, as Spline3::closest tries them (curve3.rs:428-433)
      double da = len(a - p), db = len(b - p);
      if (da < d) {
        d = da;
        s = 0.0;
        e.p = a;
      }
      if (db < d) {
        d = db;
        s = 1.0;
        e.p = b;
      }
      if (!conv && s > 0.0 && s < 1.0) {
        defer(P, code, fmax(lb, chord - c.thick), p, A);
        return;
      }
      if (!(d < A.best)) return;
      if ((c.first && s <= 0.0) || (c.last && s >= 1.0)) return;  // an end of the edge: its vertex answers
      const DEdge& ed = P.edges[c.edge];
      double3 pn = mk(0, 0, 0);
      for (int side = 0; side < 2; side++) {
        int fi = side == 0 ? ed.f0 : ed.f1;
        double u = c.uv[side][0][0] + s * (c.uv[side][1][0] - c.uv[side][0][0]);
        double v = c.uv[side][0][1] + s * (c.uv[side][1][1] - c.uv[side][0][1]);
        pn = pn + face_normal_at(P, fi, e.p, u, v);
      }
      take(A, d, d * sgn(dot(p - e.p, pn)));
      return;
    }
    default: {
      const DVert& v = P.verts[i];
      double3 x = ld3(v.p);
      double d = len(p - x);
      if (d < A.best) take(A, d, d * sgn(dot(p - x, ld3(v.pn))));
      return;
    }
  }
}

// Nearest-first descent of the feature tree for one point (the reference's
// BoxTree::nearest_first, solid3.rs:167-198, as a depth-first walk that visits the
// nearer child first and prunes on the best so far).
HDI void point_query(const DPack& P, double3 p, double cap, Acc& A) {
  acc_init(A, cap);
  int stack[64];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const DBvh& nd = P.bvh[stack[--sp]];
    if (box_dist_f(p, nd.lo, nd.hi) >= A.best) continue;
    if (nd.count > 0) {
      for (int k = 0; k < nd.count; k++) eval_item(P, P.items[nd.first + k], p, A, 0, 0.5, 0.5);
      continue;
    }
    const DBvh& l = P.bvh[nd.first];
    const DBvh& r = P.bvh[nd.first + 1];
    double dl = box_dist_f(p, l.lo, l.hi), dr = box_dist_f(p, r.lo, r.hi);
    if (sp + 2 > 64) continue;  // cannot happen for trees of depth < 64
    if (dl <= dr) {
      if (dr < A.best) stack[sp++] = nd.first + 1;
      if (dl < A.best) stack[sp++] = nd.first;
    } else {
      if (dl < A.best) stack[sp++] = nd.first;
      if (dr < A.best) stack[sp++] = nd.first + 1;
    }
  }
  resolve(P, p, A);
}

// A point's value by the reference kernel's contract (gpu.wgsl:1909-1921): the signed
// distance (flag 0), a lower bound past the cap (flag 1), or undecided (flag 2, value the
// why-code).
HD void finish(const Acc& A, double cap, double* value, int* flag) {
  if (A.und < A.best && A.und <= cap) {
    *value = A.why;
    *flag = 2;
  } else if (!isnan(A.sd) && A.best <= cap) {
    *value = A.sd;
    *flag = 0;
  } else {
    *value = cap;
    *flag = 1;
  }
}

}  // namespace icam

// What a warp shares when its lanes query points near one centre: the candidate list of
// the features near that centre (the reference's per-brick list, GpuPack::list, gpu.rs:709,
// restated for a warp), ranked by their bound, and Newton seeds of its sub-patches taken
// at the centre. Used by the brick kernel (bricks.cu) and the box decision (decide.cu).
#pragma once

#include "field.cuh"

namespace icam {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MAXC = 128;   // candidates a list may hold
constexpr int FR = 64;      // tree nodes one level of the list's walk may hold
constexpr int MAXSUB = 32;  // sub-patches seeded from the centre

// The features with a lower bound <= reach from c, unranked into tcode / tlb (at most
// CAP kept; the count returned may exceed it). The tree is walked a level at a time,
// a lane a node; a level wider than the frontier gives way to every leaf in turn, or,
// with WIDE_GIVES_UP on a tree of more than WIDE_LEAVES leaves (a scan of them all would
// cost more than the points' own tree walks), ends the walk with a count of
// LIST_TOO_WIDE (more than any room: the caller reads its points by the tree walk).
// *count is a shared counter of the warp; fr two frontier buffers of FR nodes.
constexpr int LIST_TOO_WIDE = 1 << 28;
constexpr int WIDE_LEAVES = 4096;
template <int CAP = MAXC, bool WIDE_GIVES_UP = false>
__device__ __forceinline__ int warp_list(const DPack& P, const int32_t* leaves, int n_leaves, double3 c, double reach,
                                         uint32_t* tcode, double* tlb, int32_t (*fr)[FR], int* count, int lane) {
  auto take_leaf = [&](const DBvh& nd) {
    for (int k = 0; k < nd.count; k++) {
      uint32_t code = P.items[nd.first + k];
      double lb = item_lb(P, code, c);
      if (lb <= reach) {
        int slot = atomicAdd(count, 1);
        if (slot < CAP) {
          tcode[slot] = code;
          tlb[slot] = lb;
        }
      }
    }
  };
  if (lane == 0) {
    *count = 0;
    fr[0][0] = 0;
  }
  __syncwarp();
  bool walked = true;
  int cur = 0, ncur = 1;
  while (ncur > 0) {
    int nnext = 0;
    for (int base = 0; base < ncur; base += 32) {
      const int i = base + lane;
      bool inner = false;
      int32_t kid = 0;
      if (i < ncur) {
        const DBvh& nd = P.bvh[fr[cur][i]];
        if (box_dist_f(c, nd.lo, nd.hi) <= reach) {
          if (nd.count > 0) {
            take_leaf(nd);
          } else {
            inner = true;
            kid = nd.first;
          }
        }
      }
      const unsigned m = __ballot_sync(FULL, inner);
      const int off = nnext + 2 * __popc(m & ((1u << lane) - 1u));
      if (inner && off + 1 < FR) {
        fr[cur ^ 1][off] = kid;
        fr[cur ^ 1][off + 1] = kid + 1;
      }
      nnext += 2 * __popc(m);
    }
    __syncwarp();
    if (nnext > FR) {
      walked = false;
      break;
    }
    cur ^= 1;
    ncur = nnext;
  }
  if (!walked && WIDE_GIVES_UP && n_leaves > WIDE_LEAVES) {
    __syncwarp();
    return LIST_TOO_WIDE;
  }
  if (!walked) {
    if (lane == 0) *count = 0;
    __syncwarp();
    for (int leaf = lane; leaf < n_leaves; leaf += 32) {
      const DBvh& nd = P.bvh[leaves[leaf]];
      if (box_dist_f(c, nd.lo, nd.hi) <= reach) take_leaf(nd);
    }
  }
  __syncwarp();
  // every lane reads the count before any lane may go on to reset it (a next list)
  const int n = *count;
  __syncwarp();
  return n;
}

// The first n of tcode / tlb ranked by bound into code / lb, ties by code so the order
// does not depend on the order the list was found in.
__device__ __forceinline__ void warp_rank(const uint32_t* tcode, const double* tlb, int n, uint32_t* code, double* lb,
                                          int lane) {
  for (int k = lane; k < n; k += 32) {
    double l = tlb[k];
    uint32_t cd = tcode[k];
    int rank = 0;
    for (int j = 0; j < n; j++) {
      double l2 = tlb[j];
      rank += (l2 < l) || (l2 == l && tcode[j] < cd);
    }
    code[rank] = cd;
    lb[rank] = l;
  }
  __syncwarp();
}

// A sub-patch's Newton solution nearest a centre c, for first-order seeds at points
// nearby: (s, t) there, the inverse Hessian of |S - c|^2 and the tangents, so that
// (s, t)(p) ~ (s, t) + H^-1 [S_s.(p - c), S_t.(p - c)].
struct Seed {
  double s, t, i00, i01, i11;
  double ss[3], st[3];
};

// Newton starts at (s0, t0): the sub-patch's centre, or a learned start.
__device__ __forceinline__ Seed seed_at(const double4* cp, double3 c, double s0 = 0.5, double t0 = 0.5) {
  double ss = s0, tt = t0;
  bool conv;
  newton_bicubic(cp, c, &ss, &tt, 12, &conv);
  SE e = eval_bicubic(cp, ss, tt);
  double3 r = e.p - c;
  double h0 = dot(e.ps, e.ps) + dot(e.pss, r), h1 = dot(e.ps, e.pt) + dot(e.pst, r), h2 = dot(e.pt, e.pt) + dot(e.ptt, r);
  if (!(h0 > 0.0 && h0 * h2 - h1 * h1 > 0.0)) h0 = dot(e.ps, e.ps), h1 = dot(e.ps, e.pt), h2 = dot(e.pt, e.pt);
  double det = h0 * h2 - h1 * h1;
  Seed sd;
  sd.s = ss, sd.t = tt;
  if (fabs(det) > 1e-300) {
    sd.i00 = h2 / det, sd.i01 = -h1 / det, sd.i11 = h0 / det;
  } else {
    sd.i00 = sd.i01 = sd.i11 = 0.0;
  }
  sd.ss[0] = e.ps.x, sd.ss[1] = e.ps.y, sd.ss[2] = e.ps.z;
  sd.st[0] = e.pt.x, sd.st[1] = e.pt.y, sd.st[2] = e.pt.z;
  return sd;
}

// The seed for a point c + dp, held in the square.
__device__ __forceinline__ void seed_params(const Seed& sd, double3 dp, double* ss, double* tt) {
  double gs = sd.ss[0] * dp.x + sd.ss[1] * dp.y + sd.ss[2] * dp.z;
  double gt = sd.st[0] * dp.x + sd.st[1] * dp.y + sd.st[2] * dp.z;
  *ss = fmin(fmax(sd.s + sd.i00 * gs + sd.i01 * gt, 0.0), 1.0);
  *tt = fmin(fmax(sd.t + sd.i01 * gs + sd.i11 * gt, 0.0), 1.0);
}

// A point the list could not settle (more candidates than the list holds, or a feature
// the subdivision below gave up on): the whole tree walk with every fallback, out of line
// so the common path keeps its registers.
static __device__ __noinline__ void point_fallback(const DPack& P, double3 p, double cap, double* value, int* flag) {
  Acc A;
  point_query(P, p, cap, A);
  finish(A, cap, value, flag);
}

// Edges, pieces and vertices: eval_item out of line (faces and sub-patches, the common
// candidates, are evaluated in the walk's own loop).
static __device__ __noinline__ void eval_item_cold(const DPack& P, uint32_t code, double3 p, Acc& A) {
  eval_item(P, code, p, A, 0, 0.5, 0.5);
}

// A point's features whose certificate failed there (at most two), searched by
// subdivision after every other candidate has tightened the bound, nearest bound first
// (the deferral of the tree walk, restated for the list). Out of line too.
static __device__ __noinline__ void point_resolve(const DPack& P, double3 p, uint32_t c0, double l0, uint32_t c1,
                                                  double l1, int nd, double* best, double* sd, double* und) {
  Acc B;
  B.best = *best;
  B.sd = *sd;
  B.und = INFINITY;
  B.why = 0;
  B.ub = INFINITY;
  B.nd = 0;
  B.record = false;
  if (nd == 2 && l1 < l0) {
    uint32_t tc = c0;
    c0 = c1, c1 = tc;
    double tl = l0;
    l0 = l1, l1 = tl;
  }
  if (l0 < B.best) subdivide(P, c0, p, B);
  if (nd == 2 && l1 < B.best) subdivide(P, c1, p, B);
  *best = B.best;
  *sd = B.sd;
  *und = B.und;
}

// A sub-patch's answer at p in double precision: projected Newton from (ss, tt), the
// critical-point test, a defined normal and (for a sub-patch across its face's loops)
// the loops' parity; taken into best / sd when nearer. 1 taken, 0 not, 2 the solve did
// not converge (the caller defers the sub-patch).
__device__ __forceinline__ int sub_exact(const DPack& P, const double4* cp, const DSub& s, double3 p, double ss,
                                         double tt, int iters, double* best, double* sd) {
  SE e;
  bool conv;
  newton_bicubic_e(cp, p, &ss, &tt, iters, &conv, &e);
  if (!conv) return 2;
  double d = len(e.p - p);
  if (!(d < *best) || !is_critical(p, e)) return 0;
  double3 nrm = cross(e.ps, e.pt);
  if (!(len(nrm) > 0.0)) return 0;
  if (s.klass != 1 && !trim_inside(P, P.faces[s.face], s.u0 + ss * (s.u1 - s.u0), s.v0 + tt * (s.v1 - s.v0)))
    return 0;
  *best = d;
  *sd = d * sgn(dot(p - e.p, unit(nrm) * P.faces[s.face].sense));
  return 1;
}
static __device__ __noinline__ int sub_exact_cold(const DPack& P, const double4* cp, const DSub& s, double3 p,
                                                  double ss, double tt, int iters, double* best, double* sd) {
  return sub_exact(P, cp, s, p, ss, tt, iters, best, sd);
}

// sub_convex for one point, out of line: most sub-patches are certified for a whole
// brick at once.
static __device__ __noinline__ bool sub_convex_at(const DSub& s, double3 p) { return sub_convex(s, p, p); }

// A warp's ranked candidates, in shared memory: code and bound at the centre c, a
// verdict per candidate (sub-patch: 1 convex over every point the warp asks about;
// plane: 1 its trim holds at every foot, 2 at none; else 0), the seed slot of each
// sub-patch (-1 none; slot null: no seeds, every solve starts at the centre), and room
// for the control net the warp is on.
struct WarpCands {
  const uint32_t* code;
  const double* lb;
  const float* lbs;  // the least bound from each candidate on, rounded down (null: lb, ranked by it)
  const int8_t* cert;
  const int8_t* slot;
  const Seed* seed;
  double4* net;
  float4* net32;
  int n;
  bool overflow;  // more candidates than the list holds: every point walks the tree
  // The list holds every feature whose bound from the centre is at most this (a list
  // taken again with a shorter reach when the whole one overflowed; infinite when whole):
  // a point whose answer is farther than reach_ok less its distance from the centre is
  // handed back for the tree walk.
  double reach_ok = INFINITY;
};

// The value of point p (lane's own; `live` false for a lane without one) over the ranked
// candidates, capped at `cap`, by the reference kernel's contract (gpu.wgsl:1909-1921:
// value and flag 0 exact / 1 bound / 2 undecided). Every lane of the warp calls it
// together: the lanes walk the same candidates in rank order and leave when no lane's
// point is nearer than the next bound. MIXED: sub-patches run Newton in floats on the
// rebased nets and are polished in doubles, with the critical-point test and the trim,
// only when their float distance can beat the answer so far.
template <bool MIXED, bool TAIL = true>
__device__ __forceinline__ void warp_point(const DPack& P, const WarpCands& W, double3 p, double3 c, bool live,
                                           double cap, int lane, double* value, int* flag) {
  const double rr = len(p - c);
  double best = live ? cap : -1.0;  // a lane without a point is done
  double sdv = NAN, und = INFINITY;
  // features left for subdivision: the first two, and how many
  uint32_t dc0 = 0, dc1 = 0;
  double dl0 = 0.0, dl1 = 0.0;
  int nd = 0;
  auto defer_item = [&](uint32_t code, double lb) {
    und = fmin(und, lb);
    if (nd == 0)
      dc0 = code, dl0 = lb;
    else if (nd == 1)
      dc1 = code, dl1 = lb;
    nd++;
  };
  for (int k = 0; k < W.n && !W.overflow; k++) {
    const double lbc = W.lb[k];
    const double lbk = W.lbs ? double(W.lbs[k]) : lbc;
    if (__all_sync(FULL, lbk - rr >= best)) break;  // nothing from here on is nearer
    const uint32_t code = W.code[k];
    const uint32_t kind = code >> IK_SHIFT, idx = code & IK_MASK;
    if (kind == IK_SUB) {  // the control net to shared memory, by the whole warp
      __syncwarp();
      if (lane < 16)
        W.net[lane] = P.sub_cp[16 * size_t(idx) + lane];
      else if (MIXED)
        W.net32[lane - 16] = P.sub_cp32[16 * size_t(idx) + lane - 16];
      __syncwarp();
    }
    if (lbc - rr >= best) continue;
    if (kind == IK_FACE) {  // eval_item's analytic face, inline
      if (W.cert[k] == 2) continue;  // no foot is within the trim
      const DFace& f = P.faces[idx];
      if (box_dist(p, f.box) >= best) continue;
      double3 q, fn;
      double u, v;
      if (!analytic_foot(f, p, &q, &fn, &u, &v)) continue;
      double d = len(p - q);
      if (!(d < best) || (W.cert[k] != 1 && !trim_inside(P, f, u, v))) continue;
      best = d;
      sdv = d * sgn(dot(p - q, fn));
      continue;
    }
    if (kind != IK_SUB) {
      Acc A;
      A.best = best;
      A.sd = sdv;
      A.und = INFINITY;
      A.why = 0;
      A.ub = INFINITY;
      A.nd = 0;
      A.record = true;  // an uncertified piece records its bound in und
      eval_item_cold(P, code, p, A);
      best = A.best;
      sdv = A.sd;
      if (A.und < INFINITY) defer_item(code, A.und);
      continue;
    }
    const DSub& s = P.subs[idx];
    double lb = box_dist(p, s.box);
    if (lb >= best) continue;
    if (!W.cert[k] && !sub_convex_at(s, p)) {
      defer_item(code, lb);
      continue;
    }
    const int slot = W.slot ? W.slot[k] : -1;
    double ss = 0.5, tt = 0.5;
    if (slot >= 0) seed_params(W.seed[slot], p - c, &ss, &tt);
    const double4* cp64 = W.net;
    if (MIXED) {
      const float4* cp32 = W.net32;
      float3 p32 = f3(float(p.x - s.c[0]), float(p.y - s.c[1]), float(p.z - s.c[2]));
      float sf = float(ss), tf = float(tt);
      SEf ef;
      const bool fconv = newton_bicubic_f(cp32, p32, &sf, &tf, 8, &ef);
      float3 rf = f3(ef.p.x - p32.x, ef.p.y - p32.y, ef.p.z - p32.z);
      double d32 = sqrt(double(dotf(rf, rf)));
      // a float distance past the answer by more than its error cannot win
      if (d32 > best + 1e-4 * (1.0 + best)) continue;
      // The float answer stands where it is well conditioned: converged and away from
      // the surface (so its sign is sure; about 2e-6 mm of error on the rebased net,
      // within the mixed form's 1e-7 of the diagonal). On a sub-patch across its face's
      // loops the foot's side of the loops is the double parity test at the float foot:
      // a foot within the float error of a loop moves the answer by the square of that
      // error. Everything else (the sign near zero, a stalled float solve) goes to the
      // double polish below.
      if (fconv && d32 > 1e-3) {
        if (!is_critical_f(p32, ef)) continue;
        float3 nf = f3(ef.ps.y * ef.pt.z - ef.ps.z * ef.pt.y, ef.ps.z * ef.pt.x - ef.ps.x * ef.pt.z,
                       ef.ps.x * ef.pt.y - ef.ps.y * ef.pt.x);
        if (!(dotf(nf, nf) > 0.f) || !(d32 < best)) continue;
        if (s.klass != 1 &&
            !trim_inside(P, P.faces[s.face], s.u0 + double(sf) * (s.u1 - s.u0), s.v0 + double(tf) * (s.v1 - s.v0)))
          continue;
        best = d32;
        sdv = d32 * sgn(-double(dotf(rf, nf)) * P.faces[s.face].sense);
        continue;
      }
      ss = sf, tt = tf;
    }
    // the double solve: the plain form's every solve, inline; the mixed form's few, out
    // of line so that its float loop stays small in the instruction cache
    const int got = MIXED ? sub_exact_cold(P, cp64, s, p, ss, tt, 19, &best, &sdv)
                          : sub_exact(P, cp64, s, p, ss, tt, 16, &best, &sdv);
    if (got == 2) defer_item(code, lb);
  }
  if (!live) return;
  // !TAIL: a point the list leaves undecided is handed back (flag 3) for the caller to
  // read by the whole tree walk later, out of the loop that calls this one
  if (!TAIL && (W.overflow || (und < best && und <= cap) || best > W.reach_ok - rr)) {
    *value = NAN, *flag = 3;
    return;
  }
  if (nd > 0 && nd <= 2 && und < best && und <= cap) point_resolve(P, p, dc0, dl0, dc1, dl1, nd, &best, &sdv, &und);
  if (W.overflow || (und < best && und <= cap) || best > W.reach_ok - rr) {
    point_fallback(P, p, cap, value, flag);
  } else if (!isnan(sdv) && best <= cap) {
    *value = sdv, *flag = 0;
  } else {
    *value = cap, *flag = 1;
  }
}

}  // namespace icam

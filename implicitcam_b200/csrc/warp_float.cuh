// The mixed form's node walk: a warp's lanes query nodes of one brick over the brick's
// ranked candidate list in single precision, every coordinate relative to the brick's
// centre (and a sub-patch's net to its own centre), the mixed precision's bulk step:
// planes and B-spline sub-patches in floats; the rare features (edges, pieces, vertices,
// curved faces) and the trim tests near loops in double precision out of line; and a
// node whose float answer cannot be trusted (near zero, where the sign is decided; a
// stalled or uncertified solve) handed back for the double walk of the plain form.
#pragma once

#include "warp_list.cuh"

namespace icam {

// Blocks of four warps a SM for the mixed form's kernels: the register budget their
// launch bounds give (65536 / (ICAM_MIXED_BLOCKS x 128) a thread). Measured on the
// freeform level at h = 0.1 mm: two blocks (255 registers) 36.8 ms a bake, three (168
// registers, the out-of-line double paths spilling past L1) 40.9 ms.
#ifndef ICAM_MIXED_BLOCKS
#define ICAM_MIXED_BLOCKS 2
#endif

// A float distance below this (mm) leaves its sign to the double walk: the float
// answers' error is ~1e-6 mm on the rebased nets, so above it the sign is sure.
constexpr float NEAR_ZERO = 1e-4f;

// seed_at in floats: the Newton solution nearest the centre on the rebased net (q the
// centre relative to the sub-patch's origin), the inverse Hessian and the tangents there.
struct SeedF {
  float s, t, i00, i01, i11;
  float ss[3], st[3];
};

__device__ __forceinline__ SeedF seed_at_f(const float4* cp32, float3 q, float s0, float t0) {
  float ss = s0, tt = t0;
  SEf e;
  newton_bicubic_f(cp32, q, &ss, &tt, 12, &e);
  float3 r = f3(e.p.x - q.x, e.p.y - q.y, e.p.z - q.z);
  float h0 = dotf(e.ps, e.ps) + dotf(e.pss, r), h1 = dotf(e.ps, e.pt) + dotf(e.pst, r),
        h2 = dotf(e.pt, e.pt) + dotf(e.ptt, r);
  if (!(h0 > 0.f && h0 * h2 - h1 * h1 > 0.f)) h0 = dotf(e.ps, e.ps), h1 = dotf(e.ps, e.pt), h2 = dotf(e.pt, e.pt);
  const float det = h0 * h2 - h1 * h1;
  SeedF sd;
  sd.s = ss, sd.t = tt;
  if (fabsf(det) > 1e-30f) {
    const float id = 1.f / det;
    sd.i00 = h2 * id, sd.i01 = -h1 * id, sd.i11 = h0 * id;
  } else {
    sd.i00 = sd.i01 = sd.i11 = 0.f;
  }
  sd.ss[0] = e.ps.x, sd.ss[1] = e.ps.y, sd.ss[2] = e.ps.z;
  sd.st[0] = e.pt.x, sd.st[1] = e.pt.y, sd.st[2] = e.pt.z;
  return sd;
}

// The first-order seed for a point dp from the centre, held in the square.
__device__ __forceinline__ void seed_params_f(const SeedF& sd, float3 dp, float* ss, float* tt) {
  const float gs = sd.ss[0] * dp.x + sd.ss[1] * dp.y + sd.ss[2] * dp.z;
  const float gt = sd.st[0] * dp.x + sd.st[1] * dp.y + sd.st[2] * dp.z;
  *ss = fminf(fmaxf(sd.s + sd.i00 * gs + sd.i01 * gt, 0.f), 1.f);
  *tt = fminf(fmaxf(sd.t + sd.i01 * gs + sd.i11 * gt, 0.f), 1.f);
}

// The trim test of face fi at the foot of point p on it, in double precision, out of
// line (planes straddling a loop, sub-patches across their loops).
static __device__ __noinline__ bool trim_at_cold(const DPack& P, int fi, double u, double v) {
  return trim_inside(P, P.faces[fi], u, v);
}
static __device__ __noinline__ bool plane_trim_cold(const DPack& P, int fi, double3 p) {
  const DFace& f = P.faces[fi];
  double3 q, n;
  double u, v;
  analytic_foot(f, p, &q, &n, &u, &v);
  return trim_inside(P, f, u, v);
}

// A rare feature in double precision (edge, piece, vertex, curved face), out of line:
// best / sd updated; false when the feature could not be decided here (its certificate
// failed: the node goes to the double walk).
static __device__ __noinline__ bool rare_item_cold(const DPack& P, uint32_t code, double3 p, float* best, float* sd) {
  Acc A;
  A.best = *best;
  A.sd = *sd;
  A.und = INFINITY;
  A.why = 0;
  A.ub = INFINITY;
  A.nd = 0;
  A.record = true;
  eval_item(P, code, p, A, 0, 0.5, 0.5);
  if (A.und < INFINITY) return false;
  if (A.best < double(*best)) *best = float(A.best), *sd = float(A.sd);
  return true;
}

// Control nets a warp keeps in shared memory for a whole brick (or box group): the
// first NRES sub-patches of its ranked list, staged by the tensor memory accelerator's
// bulk copies (cp.async.bulk, global to shared, completion on an mbarrier).
constexpr int NRES = 12;  // brick kernel; the box decision keeps NRES_D
constexpr int NRES_D = 8;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return uint32_t(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Lane 0: the bulk copies of n float nets (sub-patches idx[k], 256 bytes each, from
// cp32) into dst + 16 k, completing on the warp's barrier. Source and destination are
// 16-byte aligned (nets of 16 float4), as the bulk copy requires.
__device__ __forceinline__ void stage_nets(float4* dst, const float4* cp32, const uint32_t* idx, int n,
                                           uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // after the generic reads of the room
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(uint32_t(n) * 256u) : "memory");
  for (int k = 0; k < n; k++)
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 256, [%2];" ::"r"(
                     smem_u32(dst + 16 * k)),
                 "l"(cp32 + 16 * size_t(idx[k])), "r"(smem_u32(bar))
                 : "memory");
}
// Every lane: waits for the barrier's phase `parity` to complete, at most `limit` tries;
// false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = 1 << 22) {
  for (int i = 0; i < limit; i++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// A warp's ranked candidates for the float walk, in shared memory: code, bound at the
// centre rounded down, verdict (as WarpCands), seed slot, resident net slot (-1: load
// it), and two float4 of geometry relative to the centre c: a plane (z * sense,
// (o - c).(z * sense)), (NaN: a curved face); a sub-patch (its rebasing origin - c, the
// face's sense), (its control box's half extents, 1 if wholly inside its face's loops).
struct WarpCandsF {
  const uint32_t* code;
  const float* lb;
  const float* lbs;    // the least bound from each candidate on (the walk's exit): lb when ranked by it
  const int8_t* cert;
  const int8_t* slot;
  const SeedF* seed;
  const float4* geo;
  float4* net32;       // the room for a net not resident
  const float4* res;   // the resident nets, 16 float4 each
  const int8_t* rslot;
  int n;
  int iters;           // float Newton iterations a solve
  // every feature whose bound from the centre is at most this is in the list (a list
  // taken again with a shorter reach; infinite when whole), less the float error
  float reach_ok = INFINITY;
};

// The float walk of the lane's node (pc: its offset from the centre; p: the node in
// double, for the out-of-line double steps), capped at `cap`, all lanes together (a lane
// without a node passes live = false). Returns 0 with *value the signed distance, 1
// nothing within the cap, 3 the node is left for the double walk. (lastk, ls, lt): the
// candidate this lane's previous node took its answer from and that answer's (s, t), the
// start for the same candidate here (a neighbouring node's foot is close). qzero: a
// distance below it is kept whatever its sign (a caller that stores only i16 values,
// where such a distance and its opposite both round to zero); 0 otherwise.
__device__ __forceinline__ int warp_point_f(const DPack& P, const WarpCandsF& W, float3 pc, double3 p, bool live,
                                            float cap, int lane, float* value, int* lastk, float* ls, float* lt,
                                            float qzero = 0.f, int* n_evals = nullptr, int* n_solves = nullptr) {
  const float rr = sqrtf(dotf(pc, pc));
  // the cap widened by the float error: a node the walk finds nothing for is past the
  // cap in exact arithmetic too (flag 1); one found just past it keeps its value (flag 0)
  const float capw = cap * (1.f + 4e-6f) + 1e-6f;
  float best = live ? capw : -1.f;  // -1: done (no node, or left for the double walk)
  float sdv = NAN;
  bool pend = false;
  int wk = -1;
  float ws = 0.f, wt = 0.f;
  // sub-patches whose certificate fails here: left for the double subdivision once
  // everything else has tightened the bound (the first two; more: the double walk)
  uint32_t dc0 = 0, dc1 = 0;
  float dl0 = 0.f, dl1 = 0.f, und = INFINITY;
  int nd = 0;
  for (int k = 0; k < W.n; k++) {
    const float lbc = W.lb[k];
    if (__all_sync(FULL, W.lbs[k] - rr >= best)) break;  // nothing from here on is nearer
    const uint32_t code = W.code[k];
    const uint32_t kind = code >> IK_SHIFT, idx = code & IK_MASK;
    const float4* net = W.net32;
    const bool want = lbc - rr < best;
    if (kind == IK_SUB) {
      const int rs = W.rslot[k];
      if (rs >= 0) {
        net = W.res + 16 * rs;
      } else if (__any_sync(FULL, want)) {  // not resident: to shared memory by the whole warp
        __syncwarp();
        if (lane < 16) W.net32[lane] = P.sub_cp32[16 * size_t(idx) + lane];
        __syncwarp();
      }
    }
    if (!want) continue;
    const float4 g0 = W.geo[2 * k];
    if (kind == IK_FACE && !isnan(g0.w)) {  // a plane
      const int8_t ct = W.cert[k];
      if (ct == 2) continue;  // no foot within the trim
      const float sd = g0.x * pc.x + g0.y * pc.y + g0.z * pc.z - g0.w;
      const float d = fabsf(sd);
      if (!(d < best)) continue;
      if (ct != 1 && !plane_trim_cold(P, int(idx), p)) continue;
      best = d;
      sdv = sd;
      wk = -1;
      continue;
    }
    if (kind == IK_SUB) {
      const float4 g1 = W.geo[2 * k + 1];
      const float3 q = f3(pc.x - g0.x, pc.y - g0.y, pc.z - g0.z);
      const float bx = fmaxf(fabsf(q.x) - g1.x, 0.f), by = fmaxf(fabsf(q.y) - g1.y, 0.f),
                  bz = fmaxf(fabsf(q.z) - g1.z, 0.f);
      const float blb = sqrtf(bx * bx + by * by + bz * bz);
      if (!(blb < best)) continue;
      if (!W.cert[k] && !sub_convex_at(P.subs[idx], p)) {  // subdivision, after the rest
        und = fminf(und, blb);
        if (nd == 0)
          dc0 = code, dl0 = blb;
        else if (nd == 1)
          dc1 = code, dl1 = blb;
        nd++;
        continue;
      }
      float sf = 0.5f, tf = 0.5f;
      if (*lastk == k) {
        sf = *ls, tf = *lt;
      } else if (W.slot[k] >= 0) {
        seed_params_f(W.seed[W.slot[k]], pc, &sf, &tf);
      }
      SEf ef;
      if (n_solves) ++*n_solves;
      if (!newton_bicubic_f(net, q, &sf, &tf, W.iters, &ef, n_evals)) {  // stalled: the double walk
        pend = true;
        best = -1.f;
        continue;
      }
      const float3 rf = f3(ef.p.x - q.x, ef.p.y - q.y, ef.p.z - q.z);
      const float d32 = sqrtf(dotf(rf, rf));
      if (!(d32 < best) || !is_critical_f(q, ef)) continue;
      const float3 nf = f3(ef.ps.y * ef.pt.z - ef.ps.z * ef.pt.y, ef.ps.z * ef.pt.x - ef.ps.x * ef.pt.z,
                           ef.ps.x * ef.pt.y - ef.ps.y * ef.pt.x);
      if (!(dotf(nf, nf) > 0.f)) continue;
      if (g1.w != 1.f) {  // across its face's loops: the trim test in double
        const DSub& s = P.subs[idx];
        if (!trim_at_cold(P, s.face, s.u0 + double(sf) * (s.u1 - s.u0), s.v0 + double(tf) * (s.v1 - s.v0)))
          continue;
      }
      best = d32;
      sdv = -dotf(rf, nf) * g0.w < 0.f ? -d32 : d32;
      wk = k, ws = sf, wt = tf;
      continue;
    }
    // edges, pieces, vertices, curved faces
    if (!rare_item_cold(P, code, p, &best, &sdv)) {
      pend = true;
      best = -1.f;
    }
  }
  if (!live) return 1;
  if (best > W.reach_ok - rr) pend = true;  // a feature the shortened list left out may be nearer
  if (wk >= 0) *lastk = wk, *ls = ws, *lt = wt;
  if (!pend && nd > 0 && und < best) {  // the deferred sub-patches, by the double subdivision
    if (nd > 2) {
      pend = true;
    } else {
      double b64 = best, s64 = sdv, u64 = INFINITY;
      point_resolve(P, p, dc0, dl0, dc1, dl1, nd, &b64, &s64, &u64);
      if (u64 < b64) {
        pend = true;
      } else if (b64 < double(best)) {
        best = float(b64), sdv = float(s64);
        wk = -1;
      }
    }
  }
  if (pend) return 3;
  if (!isnan(sdv) && best <= capw) {
    if (best < NEAR_ZERO && !(best < qzero)) return 3;  // the sign near zero: double precision decides it
    *value = sdv;
    return 0;
  }
  *value = cap;
  return 1;
}

}  // namespace icam

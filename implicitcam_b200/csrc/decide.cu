// The box decision of a level (partcache.rs:226-331) on sm_100a: 32 boxes a warp, their
// centres read through one shared candidate list, each box then decided air or material,
// split, or (size 1) read.
#include "kernels.h"
#include "warp_float.cuh"
#include "warp_list.cuh"

namespace icam {

constexpr int DWARPS = 4;  // box groups a block works on at once, one a warp
// first_sign of a first box: +1 / -1 its exact value's sign, 0 none (not exact, or on the
// surface), pending (past its cut, sign not known), then air or material once known
constexpr int8_t FS_PENDING = 2, FS_AIR = 3, FS_SOLID = -3;

// A box group's list holds twice a brick's candidates: a box's cut reaches farther, and
// a list that overflows sends every lane to walk the tree alone.
constexpr int DMAXC = 2 * MAXC;
// A group whose list overflows is halved (each half lists again) while the list holds
// fewer than HALVE_BELOW times the room; past that (a part of many small faces, where
// even one box's cut holds far more than the room) halving would end in boxes walking
// the tree one lane at a time, so the group's lanes walk it each for its own box at once.
constexpr int HALVE_BELOW = 16;

struct DecideSmem {
  uint32_t tcode[DMAXC];  // the list before its ranking, and the walk's frontier
  double tlb[DMAXC];
  int32_t fr[2][FR];
  double lb[DMAXC];  // ranked candidates
  uint32_t code[DMAXC];
  Seed seed[MAXSUB];
  double4 net[16];
  float4 net32[16];
  int8_t cert[DMAXC];
  int8_t slot[DMAXC];
  int n;
};
static_assert(sizeof(DecideSmem) * DWARPS <= 48 * 1024, "static shared memory of a block");

// A box's radius from its corners grown by the clamp (lo, hi): the reference's, half
// their diagonal; under the tight rule (a level bake), the box's own half-diagonal,
// rounded up.
__device__ __forceinline__ double box_radius(const DecideArgs& a, double3 lo, double3 hi) {
  if (!a.tight) return 0.5 * len(hi - lo);
  const double g = 2.0 * a.clamp;
  return 0.5 * len(hi - lo - mk(g, g, g)) * (1.0 + 1e-12);
}

// One box's verdict from its centre's value (v, f) read within `cut` (partcache.rs:370-383:
// decided once the centre is known past the box grown by the clamp), the map entries it
// settles, and its children (up to 8: into kids, *nk of them, for the caller to append;
// appended here together when kids is null) or its read. verr: v's error bound (0 for a
// double reading; the float reading's caller has made sure the verdict does not lie
// within it), which the sign and bounds handed to the children and the read bricks
// allow for, so that the map is the exact reading's.
__device__ void decide_box(const DecideArgs& a, long long size, const Box4& b, double3 c, double r, double cut,
                           double v, int f, Box4* kids_out = nullptr, int* nk_out = nullptr, double verr = 0.0) {
  const DPack& P = a.P;
  const double side = 8.0 * a.h;
  double sd = NAN;  // the signed distance at the centre when known (its sign sure)
  int verdict;      // 0 split or read, 1 air, 2 material
  if (f == 0) {
    sd = fabs(v) > verr ? v : NAN;
    verdict = (v - r > a.clamp) ? 1 : ((v + r < -a.clamp) ? 2 : 0);
  } else if (f == 1) {
    // past the box: air or material as the parent's centre when the parent's centre lies
    // in this one's empty ball (partcache.rs:401-406); else read without the cut
    if (isfinite(b.parent_sd) && b.parent_sd != 0.0 && b.reach < cut * (1.0 - 1e-6)) {
      verdict = b.parent_sd > 0 ? 1 : 2;
    } else {
      point_fallback(P, c, INFINITY, &v, &f);
      if (f == 0) {
        sd = v;
        verdict = (v - r > a.clamp) ? 1 : ((v + r < -a.clamp) ? 2 : 0);
      } else {
        verdict = 0;
      }
    }
  } else {
    verdict = 0;
  }
  const long long nb0 = a.nb[0], nb1 = a.nb[1], nb2 = a.nb[2];
  if (verdict != 0) {
    uint32_t val = verdict == 1 ? 0xffffffffu : 0xfffffffeu;
    for (long long z = max(b.z, 0LL); z < min(b.z + size, nb2); z++)
      for (long long y = max(b.y, 0LL); y < min(b.y + size, nb1); y++)
        for (long long x = max(b.x, 0LL); x < min(b.x + size, nb0); x++) a.map[x + nb0 * (y + nb1 * z)] = val;
  } else if (size == 1) {
    long long idx = b.x + nb0 * (b.y + nb1 * b.z);
    a.map[idx] = 0xfffffff0u;  // read
    unsigned long long slot = atomicAdd(a.n_read, 1ull);
    if (slot < (unsigned long long)a.read_cap) {
      a.read_idx[slot] = idx;
      // a float reading hands on a lower bound of |sd| with its sign: the brick kernel's
      // shortcuts and its centre ball read the centre distance as a bound
      a.read_dc[slot] = isfinite(sd) ? copysign(fabs(sd) - verr, sd) : sd;
    }
  } else {
    const long long half = size / 2;
    Box4 kids[8];
    int nk = 0;
    // Bricks (children of size 1) settled by this box's exact centre distance sd: a child
    // whose centre lies within sd's empty ball has |v| <= |sd| + reach < r + clamp, so its
    // own reading would find it neither air nor material and read it; and when
    // |sd| - reach (a bound on |v| with sd's sign) already settles the brick by sign, the
    // brick kernel needs nothing more of it. Such a child is read with that bound as its
    // centre distance instead of being queried.
    const bool by_bound = half == 1 && isfinite(sd) && sd != 0.0 && fabs(sd) > verr;
    for (int q = 0; q < 8; q++) {
      Box4 k;
      k.x = b.x + half * (q & 1);
      k.y = b.y + half * ((q >> 1) & 1);
      k.z = b.z + half * ((q >> 2) & 1);
      if (!(k.x < nb0 && k.x + half > 0 && k.y < nb1 && k.y + half > 0 && k.z < nb2 && k.z + half > 0)) continue;
      double3 klo = mk(a.lo[0] + side * k.x - a.clamp, a.lo[1] + side * k.y - a.clamp, a.lo[2] + side * k.z - a.clamp);
      double3 khi = mk(a.lo[0] + side * (k.x + half) + a.clamp, a.lo[1] + side * (k.y + half) + a.clamp,
                       a.lo[2] + side * (k.z + half) + a.clamp);
      k.reach = len((klo + khi) * 0.5 - c);
      k.parent_sd = sd;
      if (by_bound) {
        const double rk = box_radius(a, klo, khi);
        const double bound = fabs(sd) - verr - k.reach;
        const double dcb = copysign(bound, sd);
        if (fabs(sd) + verr + k.reach < (rk + a.clamp) * (1.0 - 1e-12) && bound > 0.0 &&
            settles_by_sign(dcb, a.h, a.clamp, 1e-9 * (1.0 + a.clamp))) {
          const long long idx = k.x + nb0 * (k.y + nb1 * k.z);
          a.map[idx] = 0xfffffff0u;  // read
          unsigned long long slot = atomicAdd(a.n_read, 1ull);
          if (slot < (unsigned long long)a.read_cap) {
            a.read_idx[slot] = idx;
            a.read_dc[slot] = dcb;
          }
          continue;
        }
      }
      kids[nk++] = k;
    }
    if (kids_out) {
      for (int q = 0; q < nk; q++) kids_out[q] = kids[q];
      *nk_out = nk;
      return;
    }
    // together, so that the next level's warps take neighbouring boxes
    unsigned long long slot = atomicAdd(a.n_next, (unsigned long long)nk);
    for (int q = 0; q < nk; q++)
      if (slot + q < (unsigned long long)a.next_cap) a.next[slot + q] = kids[q];
  }
}

// The ball of the centres of lanes [l0, l0 + s) that hold a box (in: their live flags):
// the middle of their centres' box (gc), the farthest centre from it (R), and that box
// (bl, bh). Every lane calls it; the others take lane l0's centre, which lies inside.
__device__ __forceinline__ void centres_ball(double3 c, bool in, int l0, int lane, double3* gc, double* R,
                                             double bl[3], double bh[3]) {
  const double3 c0 = mk(__shfl_sync(FULL, c.x, l0), __shfl_sync(FULL, c.y, l0), __shfl_sync(FULL, c.z, l0));
  const double3 cc = in ? c : c0;
  bl[0] = bh[0] = cc.x, bl[1] = bh[1] = cc.y, bl[2] = bh[2] = cc.z;
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; k++) {
      bl[k] = fmin(bl[k], __shfl_xor_sync(FULL, bl[k], o));
      bh[k] = fmax(bh[k], __shfl_xor_sync(FULL, bh[k], o));
    }
  *gc = mk(0.5 * (bl[0] + bh[0]), 0.5 * (bl[1] + bh[1]), 0.5 * (bl[2] + bh[2]));
  double r = len(cc - *gc);
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(FULL, r, o));
  *R = r;
}

// gs (1 to 32) boxes of one size from boxes[g0 ..] (n in all), a lane each: their
// centres' bounding ball, the features within its radius plus the cut of its centre
// (listed and ranked once, sub-patches seeded there), every centre's value capped at the
// cut by the shared walk, then each box decided. A list that holds more features than
// its room splits the group in halves (down to one box), each half taking its own list:
// the boxes' readings are the same, and none walks the whole tree alone while a smaller
// list would do.
__device__ __forceinline__ void decide_group(const DecideArgs& a, const Box4* boxes, int64_t n, long long size,
                                             int64_t g0, int gs, DecideSmem& S, int lane, bool first) {
  const DPack& P = a.P;
  const double side = 8.0 * a.h;
  const int64_t i = g0 + lane;
  const bool live = lane < gs && i < n;
  const Box4 b = boxes[live ? i : g0];
  double3 lo = mk(a.lo[0] + side * b.x - a.clamp, a.lo[1] + side * b.y - a.clamp, a.lo[2] + side * b.z - a.clamp);
  double3 hi = mk(a.lo[0] + side * (b.x + size) + a.clamp, a.lo[1] + side * (b.y + size) + a.clamp,
                  a.lo[2] + side * (b.z + size) + a.clamp);
  const double3 c = (lo + hi) * 0.5;
  const double r = box_radius(a, lo, hi);
  const double cut = (r + a.clamp) * (1.0 + 1e-4);
  const int glanes = int(min(int64_t(gs), n - g0));  // lanes of the group holding a box
  double v = 0.0;
  int f = 1;
  for (int l0 = 0, sg = glanes; l0 < glanes;) {
    sg = min(sg, glanes - l0);
    const bool mine = lane >= l0 && lane < l0 + sg;
    double3 gc;
    double R, bl[3], bh[3];
    centres_ball(c, mine, l0, lane, &gc, &R, bl, bh);
    // every feature nearer than the cut to a centre has a bound <= R + cut from gc
    int nc = warp_list<DMAXC, true>(P, a.leaves, a.n_leaves, gc, R + cut, S.tcode, S.tlb, S.fr, &S.n, lane);
    const bool overflow = nc > DMAXC;
    if (overflow && sg > 1 && nc < HALVE_BELOW * DMAXC) {
      sg = (sg + 1) / 2;
      continue;
    }
    if (overflow) nc = 0;  // the points walk the tree: the list is not read (nor complete)
    warp_rank(S.tcode, S.tlb, nc, S.code, S.lb, lane);
    int subs_before = 0;
    for (int base = 0; base < nc; base += 32) {
      const int k = base + lane;
      const bool is_sub = k < nc && (S.code[k] >> IK_SHIFT) == IK_SUB;
      const unsigned m = __ballot_sync(FULL, is_sub);
      const int before = subs_before + __popc(m & ((1u << lane) - 1u));
      subs_before += __popc(m);
      if (k >= nc) continue;
      int slot = -1;
      if (is_sub && before < MAXSUB) {
        slot = before;
        S.seed[slot] = seed_at(P.sub_cp + 16 * size_t(S.code[k] & IK_MASK), gc);
      }
      S.cert[k] = 0;
      S.slot[k] = int8_t(slot);
    }
    __syncwarp();
    const WarpCands W{S.code, S.lb, nullptr, S.cert, S.slot, S.seed, S.net, S.net32, nc, overflow};
    double vv;
    int ff;
    warp_point<false>(P, W, c, gc, live && mine, cut, lane, &vv, &ff);
    if (mine) v = vv, f = ff;
    l0 += sg;
  }
  Box4 kids[8];
  int nk = 0;
  if (live) {
    if (first) {
      // a first box past its cut (air or material, its sign not known: it has no parent)
      // waits for k_first_signs; an exact value is a sign its neighbours may take
      a.first_sd[i] = f == 0 ? v : NAN;
      a.first_sign[i] = f == 1 ? FS_PENDING : ((f == 0 && v != 0.0) ? (v > 0 ? 1 : -1) : 0);
    }
    if (!(first && f == 1)) decide_box(a, size, b, c, r, cut, v, f, kids, &nk);
  }
  // the group's children appended together, in lane order, so that the next round's
  // groups take neighbouring boxes (a group's boxes are neighbours, their children too)
  int incl = nk;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += t;
  }
  const int total = __shfl_sync(FULL, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && total > 0) base = atomicAdd(a.n_next, (unsigned long long)total);
  base = __shfl_sync(FULL, base, 31);
  const unsigned long long off = base + (unsigned long long)(incl - nk);
  for (int q = 0; q < nk; q++)
    if (off + q < (unsigned long long)a.next_cap) a.next[off + q] = kids[q];
  __syncwarp();
}

// decide_group in the mixed form: the group's list ranked in double as there, then every
// centre read by the float walk (warp_float.cuh) over candidates certified for the whole
// group (sub-patches convex over the box of the group's centres, planes' trims over their
// feet), seeded in floats at the group's centre. A centre the float walk cannot settle,
// or whose verdict lies within the float error of its threshold (|v| = r + clamp), is
// read again by the double walk; the rest are decided on the float value, whose error
// bound decide_box allows for. The map is the double reading's.
struct DecideSmemF {
  union {
    struct {
      uint32_t tcode[DMAXC];  // the list before its ranking, and the walk's frontier
      double tlb[DMAXC];
      int32_t fr[2][FR];
    } list;
    float4 geo[2 * DMAXC];  // after the ranking: the candidates' float geometry
  } u;
  double lb[DMAXC];  // ranked candidates
  float lbf[DMAXC];
  uint32_t code[DMAXC];
  SeedF seed[MAXSUB];
  double4 net[16];
  float4 net32[16];
  float4 res[16 * NRES_D];  // the first NRES_D sub-patches' nets, staged by bulk copies
  int8_t cert[DMAXC];
  int8_t slot[DMAXC];
  int8_t rslot[DMAXC];
  uint32_t residx[NRES_D];
  uint64_t bar;
  uint32_t phase;  // the barrier's phase (lane 0 keeps it for the warp)
  int n;
  int err;         // a bulk copy that did not complete in time
};

__device__ __forceinline__ void decide_group_f(const DecideArgs& a, const Box4* boxes, int64_t n, long long size,
                                               int64_t g0, int gs, DecideSmemF& S, int lane, bool first) {
  const DPack& P = a.P;
  const double side = 8.0 * a.h;
  const int64_t i = g0 + lane;
  const bool live = lane < gs && i < n;
  const Box4 b = boxes[live ? i : g0];
  double3 lo = mk(a.lo[0] + side * b.x - a.clamp, a.lo[1] + side * b.y - a.clamp, a.lo[2] + side * b.z - a.clamp);
  double3 hi = mk(a.lo[0] + side * (b.x + size) + a.clamp, a.lo[1] + side * (b.y + size) + a.clamp,
                  a.lo[2] + side * (b.z + size) + a.clamp);
  const double3 c = (lo + hi) * 0.5;
  const double r = box_radius(a, lo, hi);
  const double cut = (r + a.clamp) * (1.0 + 1e-4);
  const int glanes = int(min(int64_t(gs), n - g0));  // lanes of the group holding a box
  double v = 0.0, verr = 0.0;
  int f = 1;
  for (int l0 = 0, sg = glanes; l0 < glanes;) {
    sg = min(sg, glanes - l0);
    const bool mine = lane >= l0 && lane < l0 + sg;
    const bool mlive = live && mine;
    double3 gc;
    double R, bl[3], bh[3];
    centres_ball(c, mine, l0, lane, &gc, &R, bl, bh);
    int nc = warp_list<DMAXC, true>(P, a.leaves, a.n_leaves, gc, R + cut, S.u.list.tcode, S.u.list.tlb, S.u.list.fr, &S.n,
                              lane);
    const bool overflow = nc > DMAXC;
    if (overflow && sg > 1 && nc < HALVE_BELOW * DMAXC) {
      sg = (sg + 1) / 2;
      continue;
    }
    if (overflow) nc = 0;  // the points walk the tree: the list is not read (nor complete)
    warp_rank(S.u.list.tcode, S.u.list.tlb, nc, S.code, S.lb, lane);
    const double3 blo = mk(bl[0], bl[1], bl[2]), bhi = mk(bh[0], bh[1], bh[2]);
    int subs_before = 0;
    for (int base = 0; base < nc; base += 32) {
      const int k = base + lane;
      const bool is_sub = k < nc && (S.code[k] >> IK_SHIFT) == IK_SUB;
      const unsigned m = __ballot_sync(FULL, is_sub);
      const int before = subs_before + __popc(m & ((1u << lane) - 1u));
      subs_before += __popc(m);
      if (k >= nc) continue;
      const uint32_t code = S.code[k], idx = code & IK_MASK;
      int slot = -1, rslot = -1;
      int8_t cert = 0;
      float4 g0v = make_float4(0.f, 0.f, 0.f, 0.f), g1v = g0v;
      S.lbf[k] = __double2float_rd(S.lb[k]);
      if (is_sub) {
        const DSub& s = P.subs[idx];
        cert = sub_convex(s, blo, bhi) ? 1 : 0;
        g0v = make_float4(float(s.c[0] - gc.x), float(s.c[1] - gc.y), float(s.c[2] - gc.z), float(P.faces[s.face].sense));
        g1v = make_float4(__double2float_ru(0.5 * (s.box[3] - s.box[0])), __double2float_ru(0.5 * (s.box[4] - s.box[1])),
                          __double2float_ru(0.5 * (s.box[5] - s.box[2])), s.klass == 1 ? 1.f : 0.f);
        if (before < NRES_D) {
          rslot = before;
          S.residx[before] = idx;
        }
        if (before < MAXSUB) {
          slot = before;
          const float3 qc = f3(float(gc.x - s.c[0]), float(gc.y - s.c[1]), float(gc.z - s.c[2]));
          S.seed[slot] = seed_at_f(P.sub_cp32 + 16 * size_t(idx), qc, 0.5f, 0.5f);
        }
      } else if ((code >> IK_SHIFT) == IK_FACE) {
        const DFace& f = P.faces[idx];
        if (f.kind == S_PLANE) {
          const double3 z = ld3(f.z) * f.sense, o = ld3(f.o);
          g0v = make_float4(float(z.x), float(z.y), float(z.z), float(dot(o - gc, z)));
          double tlo[2] = {INFINITY, INFINITY}, thi[2] = {-INFINITY, -INFINITY};
          const double3 zz = ld3(f.z), fx = ld3(f.x), fy = ld3(f.y);
          for (int q = 0; q < 8; q++) {
            double3 x = mk(q & 1 ? bh[0] : bl[0], q & 2 ? bh[1] : bl[1], q & 4 ? bh[2] : bl[2]);
            double3 e = (x - zz * dot(x - o, zz)) - o;
            double u = dot(e, fx), v = dot(e, fy);
            tlo[0] = fmin(tlo[0], u), thi[0] = fmax(thi[0], u);
            tlo[1] = fmin(tlo[1], v), thi[1] = fmax(thi[1], v);
          }
          double mg = 1e-9 * (1.0 + fmax(fmax(fabs(tlo[0]), fabs(thi[0])), fmax(fabs(tlo[1]), fabs(thi[1]))));
          tlo[0] -= mg, tlo[1] -= mg, thi[0] += mg, thi[1] += mg;
          const int cls = trim_box_class(P, f, tlo, thi);
          cert = cls == 1 ? 1 : (cls == 0 ? 2 : 0);
        } else {
          g0v.w = NAN;
        }
      }
      S.u.geo[2 * k] = g0v;
      S.u.geo[2 * k + 1] = g1v;
      S.cert[k] = cert;
      S.slot[k] = int8_t(slot);
      S.rslot[k] = int8_t(rslot);
    }
    // the first NRES_D sub-patches' nets into shared memory for the group
    const int nres = min(subs_before, NRES_D);
    __syncwarp();
    if (nres > 0) {
      uint32_t ph = S.phase;
      if (lane == 0) stage_nets(S.res, P.sub_cp32, S.residx, nres, &S.bar);
      if (!mbar_wait(&S.bar, ph)) {  // never expected: let the copies land, then read from global
        mbar_wait(&S.bar, ph);
        if (lane == 0) S.err = 1;
      }
      __syncwarp();
      if (lane == 0) S.phase = ph ^ 1u;
    }
    __syncwarp();
    float vf = 0.f;
    int ff = 3;
    if (!overflow) {
      int8_t* rs = S.rslot;
      if (S.err) {  // no resident nets: every net from global memory
        for (int k = lane; k < nc; k += 32) rs[k] = -1;
        __syncwarp();
      }
      const WarpCandsF W{S.code, S.lbf, S.lbf, S.cert, S.slot, S.seed, S.u.geo, S.net32, S.res, rs, nc, 16};
      int lastk = -1;
      float ls = 0.f, lt = 0.f;
      ff = warp_point_f(P, W, f3(float(c.x - gc.x), float(c.y - gc.y), float(c.z - gc.z)), c, mlive, float(cut),
                        lane, &vf, &lastk, &ls, &lt);
    }
    if (mine) {
      v = vf, f = ff, verr = 0.0;
      if (f == 0) {
        verr = 1e-4 + 4e-6 * (fabs(v) + R);
        if (fabs(fabs(v) - (r + a.clamp)) <= verr) f = 3;  // the verdict is within the float error
      }
    }
    const bool pd = mlive && f == 3;
    if (__any_sync(FULL, pd)) {  // the double walk over the same candidates, centre starts
      const WarpCands W64{S.code, S.lb, nullptr, S.cert, nullptr, nullptr, S.net, S.net32, nc, overflow};
      double v64;
      int f64;
      warp_point<false>(P, W64, c, gc, pd, cut, lane, &v64, &f64);
      if (pd) v = v64, f = f64, verr = 0.0;
      if (a.n_double && pd) atomicAdd(a.n_double, 1ull);
    }
    l0 += sg;
  }
  Box4 kids[8];
  int nk = 0;
  if (live) {
    if (first) {
      a.first_sd[i] = f == 0 ? v : NAN;
      a.first_sign[i] = f == 1 ? FS_PENDING : ((f == 0 && fabs(v) > verr && v != 0.0) ? (v > 0 ? 1 : -1) : 0);
    }
    if (!(first && f == 1)) decide_box(a, size, b, c, r, cut, v, f, kids, &nk, verr);
  }
  int incl = nk;
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += t;
  }
  const int total = __shfl_sync(FULL, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && total > 0) base = atomicAdd(a.n_next, (unsigned long long)total);
  base = __shfl_sync(FULL, base, 31);
  const unsigned long long off = base + (unsigned long long)(incl - nk);
  for (int q = 0; q < nk; q++)
    if (off + q < (unsigned long long)a.next_cap) a.next[off + q] = kids[q];
  __syncwarp();
}

// The centre, radius and cut of a box of `size` bricks (as decide_group computes them).
__device__ __forceinline__ void box_geometry(const DecideArgs& a, const Box4& b, long long size, double3* c, double* r,
                                             double* cut) {
  const double side = 8.0 * a.h;
  double3 lo = mk(a.lo[0] + side * b.x - a.clamp, a.lo[1] + side * b.y - a.clamp, a.lo[2] + side * b.z - a.clamp);
  double3 hi = mk(a.lo[0] + side * (b.x + size) + a.clamp, a.lo[1] + side * (b.y + size) + a.clamp,
                  a.lo[2] + side * (b.z + size) + a.clamp);
  *c = (lo + hi) * 0.5;
  *r = box_radius(a, lo, hi);
  *cut = (*r + a.clamp) * (1.0 + 1e-4);
}

// The first boxes past their cut (no feature within it, so air or material; with no
// parent, their sign is not known), one block a level. A box's sign is that of any box
// whose centre lies within its cut and whose sign is known: the cut's ball holds no
// surface. Known signs spread from the boxes read exactly through the grid's face
// neighbours until none changes (at most n sweeps); a box then known fills its map
// entries; one no neighbour reached (no box of the level read exactly within its chain)
// is read without a bound and decided as any other.
__device__ void first_signs(const DecideArgs& a, int64_t n, bool fill = true) {
  const long long fx = a.first_dims[0], fy = a.first_dims[1], fz = a.first_dims[2];
  volatile int8_t* sg = a.first_sign;
  __shared__ int changed;
  for (int64_t sweep = 0; sweep <= n; sweep++) {
    __syncthreads();
    if (threadIdx.x == 0) changed = 0;
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
      if (sg[i] != FS_PENDING) continue;
      const long long ix = i % fx, iy = (i / fx) % fy, iz = i / (fx * fy);
      double3 ci, cj;
      double ri, cuti, rj, cutj;
      box_geometry(a, a.boxes[i], a.size, &ci, &ri, &cuti);
      int8_t got = 0;
      for (int d = 0; d < 6 && !got; d++) {
        const long long jx = ix + (d == 0) - (d == 1), jy = iy + (d == 2) - (d == 3), jz = iz + (d == 4) - (d == 5);
        if (jx < 0 || jy < 0 || jz < 0 || jx >= fx || jy >= fy || jz >= fz) continue;
        const int64_t j = jx + fx * (jy + fy * jz);
        const int8_t sj = sg[j];
        if (sj == 0 || sj == FS_PENDING) continue;
        box_geometry(a, a.boxes[j], a.size, &cj, &rj, &cutj);
        if (len(cj - ci) < cuti * (1.0 - 1e-6)) got = sj > 0 ? FS_AIR : FS_SOLID;
      }
      if (got) {
        sg[i] = got;
        changed = 1;
      }
    }
    __syncthreads();
    if (!changed) break;
  }
  __syncthreads();
  const long long nb0 = a.nb[0], nb1 = a.nb[1], nb2 = a.nb[2];
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int8_t si = sg[i];
    const Box4 b = a.boxes[i];
    if (si == FS_AIR || si == FS_SOLID) {
      if (!fill) continue;  // k_first_fill writes them over the whole grid
      const uint32_t val = si == FS_AIR ? 0xffffffffu : 0xfffffffeu;
      for (long long z = max(b.z, 0LL); z < min(b.z + a.size, nb2); z++)
        for (long long y = max(b.y, 0LL); y < min(b.y + a.size, nb1); y++)
          for (long long x = max(b.x, 0LL); x < min(b.x + a.size, nb0); x++) a.map[x + nb0 * (y + nb1 * z)] = val;
    } else if (si == FS_PENDING) {
      double3 c;
      double r, cut, v;
      int f;
      box_geometry(a, b, a.size, &c, &r, &cut);
      point_fallback(a.P, c, INFINITY, &v, &f);
      decide_box(a, a.size, b, c, r, cut, v, f);
    }
  }
}

__global__ void __launch_bounds__(256) k_first_signs(DecideArgs a, int64_t n) { first_signs(a, n, false); }

// The map entries of the first boxes whose sign k_first_signs found (most of a level's
// volume, far from the part): one thread a brick over the whole grid instead of the
// sweep's single block.
__global__ void __launch_bounds__(256) k_first_fill(DecideArgs a, int64_t n) {
  const long long s = a.size, per = s * s * s;
  const long long nb0 = a.nb[0], nb1 = a.nb[1], nb2 = a.nb[2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * per;
       t += (long long)gridDim.x * blockDim.x) {
    const int64_t i = t / per;
    const int8_t si = a.first_sign[i];
    if (si != FS_AIR && si != FS_SOLID) continue;
    const long long k = t - i * per;
    const Box4 b = a.boxes[i];
    const long long x = b.x + k % s, y = b.y + (k / s) % s, z = b.z + k / (s * s);
    if (x < 0 || y < 0 || z < 0 || x >= nb0 || y >= nb1 || z >= nb2) continue;
    a.map[x + nb0 * (y + nb1 * z)] = si == FS_AIR ? 0xffffffffu : 0xfffffffeu;
  }
}

// The boxes a warp takes together: 32 when there are enough groups of 32 to fill the
// GPU's warp slots (two 4-warp blocks an SM), else fewer (down to 4), so that a round of
// few boxes (the first, of large boxes with long lists) spreads over more warps.
__host__ __device__ inline int group_size(int64_t n, int sms) {
  int gs = 32;
  while (gs > 4 && n / gs < int64_t(sms) * 2 * DWARPS) gs /= 2;
  return gs;
}

// This size's box count and group size: the launch's, or read from the device.
__device__ __forceinline__ void round_count(const DecideArgs& a, int gs_launch, int64_t* n, int* gs) {
  *n = a.n;
  *gs = gs_launch;
  if (a.n_in) {
    *n = min(int64_t(*a.n_in), a.n);
    *gs = group_size(*n, a.sms);
  }
}

__global__ void __launch_bounds__(DWARPS * 32, 2) k_decide_w(DecideArgs a, int gs_launch) {
  __shared__ DecideSmem smem[DWARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t n;
  int gs;
  round_count(a, gs_launch, &n, &gs);
  for (int64_t g0 = (int64_t(blockIdx.x) * DWARPS + warp) * gs; g0 < n; g0 += int64_t(gridDim.x) * DWARPS * gs)
    decide_group(a, a.boxes, n, a.size, g0, gs, smem[warp], lane, a.first_sd != nullptr);
}

// The mixed form's decision of one box size: three blocks a SM (the float walk's
// registers), the groups' room in dynamic shared memory.
// A warp's bulk-copy barrier, once at the start of a float decision kernel.
__device__ __forceinline__ void decide_f_init(DecideSmemF& S, int lane) {
  if (lane == 0) {
    mbar_init(&S.bar);
    S.phase = 0;
    S.err = 0;
  }
  __syncwarp();
}

__global__ void __launch_bounds__(DWARPS * 32, ICAM_MIXED_BLOCKS) k_decide_wf(DecideArgs a, int gs_launch) {
  extern __shared__ __align__(16) unsigned char dsm[];
  DecideSmemF* smem = reinterpret_cast<DecideSmemF*>(dsm);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  decide_f_init(smem[warp], lane);
  int64_t n;
  int gs;
  round_count(a, gs_launch, &n, &gs);
  for (int64_t g0 = (int64_t(blockIdx.x) * DWARPS + warp) * gs; g0 < n; g0 += int64_t(gridDim.x) * DWARPS * gs)
    decide_group_f(a, a.boxes, n, a.size, g0, gs, smem[warp], lane, a.first_sd != nullptr);
}

// A batch's round (one box size a part): the counts the last round appended become this
// round's, the next counts start at zero, and the parts' groups of 32 are numbered.
// One thread: a batch holds tens to thousands of parts.
__global__ void k_decide_prep(DecideBatchArgs b, int round) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int64_t total = 0;
  for (int p = 0; p < b.n_parts; p++) {
    unsigned long long* cur = b.cnt + 2 * p + (round & 1);
    unsigned long long* next = b.cnt + 2 * p + ((round + 1) & 1);
    const DecideArgs& a = b.args[2 * p + (round & 1)];
    if (*cur > (unsigned long long)a.next_cap) {
      *b.err = 1;
      *cur = (unsigned long long)a.next_cap;
    }
    *next = 0;
    total += int64_t(*cur);
  }
  const int gs = group_size(total, b.sms);
  int64_t g = 0;
  for (int p = 0; p < b.n_parts; p++) {
    const unsigned long long cur = b.cnt[2 * p + (round & 1)];
    b.boxes_read[0] += cur;
    b.groups[p] = g;
    g += int64_t((cur + gs - 1) / gs);
  }
  b.groups[b.n_parts] = g;
  b.groups[b.n_parts + 1] = gs;
}

// A batch's round: every part's boxes of this round's size, 32 of one part a warp, the
// warps taking groups across all parts from the numbering k_decide_prep made.
template <bool F32>
__global__ void __launch_bounds__(DWARPS * 32, F32 ? ICAM_MIXED_BLOCKS : 2) k_decide_batch(DecideBatchArgs b, int round) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (F32) decide_f_init(reinterpret_cast<DecideSmemF*>(dsm)[warp], lane);
  const int64_t total = b.groups[b.n_parts];
  const int gs = int(b.groups[b.n_parts + 1]);
  for (int64_t g = int64_t(blockIdx.x) * DWARPS + warp; g < total; g += int64_t(gridDim.x) * DWARPS) {
    int lo = 0, hi = b.n_parts;  // the part: groups[p] <= g < groups[p + 1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (b.groups[mid] <= g) lo = mid;
      else hi = mid;
    }
    const DecideArgs& a = b.args[2 * lo + (round & 1)];
    const int64_t n = int64_t(b.cnt[2 * lo + (round & 1)]);
    if (F32)
      decide_group_f(a, a.boxes, n, a.size >> round, (g - b.groups[lo]) * gs, gs,
                     reinterpret_cast<DecideSmemF*>(dsm)[warp], lane, round == 0);
    else
      decide_group(a, a.boxes, n, a.size >> round, (g - b.groups[lo]) * gs, gs,
                   reinterpret_cast<DecideSmem*>(dsm)[warp], lane, round == 0);
  }
}

// A batch's first boxes past their cut, one block a part (first_signs).
__global__ void __launch_bounds__(256) k_first_signs_batch(DecideBatchArgs b) {
  const int p = blockIdx.x;
  first_signs(b.args[2 * p], int64_t(b.cnt[2 * p]));
}

void launch_decide(const DecideArgs& a, cudaStream_t s, bool first, bool mixed) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = mixed ? ICAM_MIXED_BLOCKS : 2;
  const int gs = group_size(a.n, sms);
  const int64_t want = a.n_in ? int64_t(sms) * per_sm : (a.n + DWARPS * gs - 1) / (DWARPS * gs);
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sms) * per_sm)));
  if (mixed) {
    const size_t smem = sizeof(DecideSmemF) * DWARPS;
    cudaFuncSetAttribute(k_decide_wf, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    k_decide_wf<<<grid, DWARPS * 32, smem, s>>>(a, gs);
  } else {
    k_decide_w<<<grid, DWARPS * 32, 0, s>>>(a, gs);
  }
  if (first) {  // the first size's count is the host's (n_in unset)
    k_first_signs<<<1, 256, 0, s>>>(a, a.n);
    const long long work = a.n * a.size * a.size * a.size;
    const int fg = int(std::max<long long>(1, std::min<long long>((work + 255) / 256, (long long)sms * 8)));
    k_first_fill<<<fg, 256, 0, s>>>(a, a.n);
  }
}

void launch_decide_batch(const DecideBatchArgs& b, int rounds, cudaStream_t s) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  DecideBatchArgs bb = b;
  bb.sms = sms;
  const size_t smem = b.mixed ? sizeof(DecideSmemF) * DWARPS : sizeof(DecideSmem) * DWARPS;
  if (b.mixed) cudaFuncSetAttribute(k_decide_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  for (int r = 0; r < rounds; r++) {
    k_decide_prep<<<1, 32, 0, s>>>(bb, r);
    if (b.mixed)
      k_decide_batch<true><<<sms * ICAM_MIXED_BLOCKS, DWARPS * 32, smem, s>>>(bb, r);
    else
      k_decide_batch<false><<<sms * 2, DWARPS * 32, smem, s>>>(bb, r);
    if (r == 0) k_first_signs_batch<<<b.n_parts, 256, 0, s>>>(bb);
  }
}

}  // namespace icam

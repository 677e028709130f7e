// The brick kernel of the exact part field on sm_100a: one warp a brick, from the
// brick's candidate list to its packed words (the reference's per-brick list, read and
// post-processing, partcache.rs:759-970).
#include <type_traits>

#include "kernels.h"
#include "seednet.cuh"
#include "brick_post.cuh"
#include "warp_list.cuh"

namespace icam {

constexpr int MAX_WARPS = 4;  // bricks a block works on at once, one a warp (1, 2 or 4)

// A warp's shared memory for its brick. The list before its ranking and the walk's
// frontier share room with the node values, which come later.
struct BrickSmem {
  union {
    double f[729];  // node values: exact, signed far, bridged; NaN while unknown
    struct {
      uint32_t code[MAXC];
      double lb[MAXC];
      int32_t fr[2][FR];
    } list;
  } u;
  double lb[MAXC];  // ranked candidates: lower bound at the centre, code
  uint32_t code[MAXC];
  double4 net[16];  // the control net of the sub-patch the warp is on
  float4 net32[16];
  union {
    Seed seed[MAXSUB];
    RowMasks mk;  // after the nodes: node masks by row
  } v;
  int8_t flag[729];
  int8_t cert[MAXC];
  int8_t slot[MAXC];
  int n;
};
static_assert(sizeof(BrickSmem) * MAX_WARPS <= 48 * 1024, "shared memory of a block");

// One brick a warp:
//  0. a brick whose centre distance puts every node past the clamp is written at once;
//  1. list: the tree walked a level at a time by the warp, every leaf within half
//     sqrt(3) + clamp of the brick's centre giving its features within that bound
//     (GpuPack::list with r = 0, partcache.rs:767), ranked by the bound;
//  2. each of the first MAXSUB sub-patches: its convexity certified for the whole brick
//     and its Newton solution at the centre kept for seeds, a lane each (started where
//     the seed network puts it when one is given); each plane's trim classified over
//     the feet of the whole brick;
//  3. 23 passes of 32 nodes, each node's value by the warp's shared candidate walk
//     (warp_point, warp_list.cuh), capped at the clamp;
//  4. far nodes signed, undecided ones bridged, quantised and packed.
// Two blocks a SM: the evaluators' register need (255 a thread) left unspilled beats
// more warps with spills (measured: 8 warps a SM 240 ms, 16 warps 280 ms a bake).
// BATCH: bricks of many parts in one launch, each brick's part in a.part_of and that
// part's pack, level and seed network in a.parts.
template <bool MIXED, bool BATCH>
__global__ void __launch_bounds__(MAX_WARPS * 32, 2) k_bricks_t(BrickArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BrickSmem* smem = reinterpret_cast<BrickSmem*>(smem_raw);
  const int warps = int(blockDim.x >> 5);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BrickSmem& S = smem[warp];
  unsigned long long* work = a.stats ? a.stats + 15 : nullptr;
  auto next_brick = [&](int64_t cur) -> int64_t {
    if (work) {
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(work, 1ull);
      return int64_t(__shfl_sync(FULL, b, 0));
    }
    return cur < 0 ? int64_t(blockIdx.x) * warps + warp : cur + int64_t(gridDim.x) * warps;
  };
  for (int64_t bi = next_brick(-1); bi < a.n; bi = next_brick(bi)) {
    const PartParams* Q = BATCH ? a.parts + a.part_of[bi] : nullptr;
    const DPack& P = BATCH ? Q->P : a.P;
    const double h = BATCH ? Q->h : a.h, clamp = BATCH ? Q->clamp : a.clamp;
    const int32_t* leaves = BATCH ? Q->leaves : a.leaves;
    const int32_t n_leaves = BATCH ? Q->n_leaves : a.n_leaves;
    double3 first = mk(a.firsts[3 * bi], a.firsts[3 * bi + 1], a.firsts[3 * bi + 2]);
    const double half = 4.0 * h;
    const double3 c = first + mk(half, half, half);
    const double reach = half * SQRT3 + clamp;
    const double dc = a.dcs ? a.dcs[bi] : NAN;
    // ---- 0. every node past the clamp, known from the centre alone: the field is
    // 1-Lipschitz, so |d(node)| >= |dc| - half sqrt(3), and with a margin far above the
    // rounding of both every node would come out a bound (flag 1) and the whole brick
    // the centre's sign (partcache.rs:876-892). Same outputs as reading it.
    if (isfinite(dc) && fabs(dc) - half * SQRT3 > clamp + 1e-6 * (1.0 + clamp)) {
      for (int nn = lane; nn < 729; nn += 32) {
        if (a.d_out) a.d_out[bi * 729 + nn] = clamp;
        if (a.flag_out) a.flag_out[bi * 729 + nn] = 1;
      }
      const uint32_t q = dc > 0 ? 32767u : uint32_t(uint16_t(int16_t(-32767)));
      if (a.words_out)
        for (int w = lane; w < WORD_STRIDE / 4; w += 32)
          reinterpret_cast<uint4*>(a.words_out + bi * WORD_STRIDE)[w] =
              w < 91 ? make_uint4(q | (q << 16), q | (q << 16), q | (q << 16), q | (q << 16))
                     : make_uint4(q, 0u, 0u, 0u);  // word 364 (node 728 alone), then padding
      if (lane == 0) {
        if (a.kind_out) a.kind_out[bi] = dc > 0 ? 1 : 2;
        if (a.stats) atomicAdd(&a.stats[1], 729ull);
      }
      continue;
    }
    // ---- 0b. every node on one side of the surface by more than an i16 step, known from
    // the centre alone (|d(node) - dc| <= half sqrt(3)): the brick's kind is the centre's
    // sign. The packing (partcache.rs:962-970) makes a brick AIR when every stored value
    // is > 0 and SOLID when every one is <= 0; a node read exactly stores
    // round(d / clamp * 32767), at least 1 for d > clamp / 32767 and at most -1 for
    // d < -clamp / 32767, and a node settled from another stores the clamp with that
    // node's sign, the same. A level bake keeps no words of such a brick, so none are
    // written. Same map as reading it.
    if (a.kind_only && isfinite(dc) && settles_by_sign(dc, h, clamp)) {
      if (lane == 0) {
        if (a.kind_out) a.kind_out[bi] = dc > 0 ? 1 : 2;
        if (a.stats) atomicAdd(&a.stats[11], 1ull);
      }
      continue;
    }
    // ---- 1. list
    int n = warp_list(P, leaves, n_leaves, c, reach, S.u.list.code, S.u.list.lb, S.u.list.fr, &S.n, lane);
    // a list past its room taken again with a shorter reach (bricks_mixed.cu, step 1)
    double reach_ok = INFINITY;
    for (int tries = 0; n > MAXC && tries < 4; tries++) {
      reach_ok = (tries == 0 ? reach : reach_ok) * 0.8;
      n = warp_list(P, leaves, n_leaves, c, reach_ok, S.u.list.code, S.u.list.lb, S.u.list.fr, &S.n, lane);
    }
    const bool overflow = n > MAXC;
    if (overflow) n = MAXC;
    warp_rank(S.u.list.code, S.u.list.lb, n, S.code, S.lb, lane);
    // ---- 2. certify and seed the first MAXSUB sub-patches, a lane each
    {
      int subs_before = 0;
      for (int base = 0; base < n; base += 32) {
        const int k = base + lane;
        const bool is_sub = k < n && (S.code[k] >> IK_SHIFT) == IK_SUB;
        const unsigned m = __ballot_sync(FULL, is_sub);
        const int before = subs_before + __popc(m & ((1u << lane) - 1u));
        subs_before += __popc(m);
        const double s0 = 0.5, t0 = 0.5;  // the plain form starts at the sub-patch's centre
        if (k >= n) continue;
        int slot = -1;
        int8_t cert = 0;
        if (is_sub) {
          const uint32_t idx = S.code[k] & IK_MASK;
          const DSub& s = P.subs[idx];
          cert = sub_convex(s, first, first + mk(8 * h, 8 * h, 8 * h)) ? 1 : 0;
          if (before < MAXSUB) {
            slot = before;
            S.v.seed[slot] = seed_at(P.sub_cp + 16 * size_t(idx), c, s0, t0);
          }
        } else if ((S.code[k] >> IK_SHIFT) == IK_FACE) {
          // a plane's trim over the feet of the whole brick (the box's corners projected,
          // with a margin over their rounding): 1 all inside, 2 all outside, 0 ask a node
          const DFace& f = P.faces[S.code[k] & IK_MASK];
          if (f.kind == S_PLANE) {
            double blo[2] = {INFINITY, INFINITY}, bhi[2] = {-INFINITY, -INFINITY};
            const double3 z = ld3(f.z), o = ld3(f.o), fx = ld3(f.x), fy = ld3(f.y);
            for (int q = 0; q < 8; q++) {
              double3 x = first + mk(q & 1 ? 8 * h : 0.0, q & 2 ? 8 * h : 0.0, q & 4 ? 8 * h : 0.0);
              double3 e = (x - z * dot(x - o, z)) - o;
              double u = dot(e, fx), v = dot(e, fy);
              blo[0] = fmin(blo[0], u), bhi[0] = fmax(bhi[0], u);
              blo[1] = fmin(blo[1], v), bhi[1] = fmax(bhi[1], v);
            }
            double m = 1e-9 * (1.0 + fmax(fmax(fabs(blo[0]), fabs(bhi[0])), fmax(fabs(blo[1]), fabs(bhi[1]))));
            blo[0] -= m, blo[1] -= m, bhi[0] += m, bhi[1] += m;
            int cls = trim_box_class(P, f, blo, bhi);
            cert = cls == 1 ? 1 : (cls == 0 ? 2 : 0);
          }
        }
        S.cert[k] = cert;
        S.slot[k] = int8_t(slot);
      }
    }
    __syncwarp();
    // ---- 3. every node: the warp's lanes walk the same ranked candidates together
    int cnt[3] = {0, 0, 0};
    int pending = 0;
    const WarpCands W{S.code, S.lb, nullptr, S.cert, S.slot, S.v.seed, S.net, S.net32, n, overflow, reach_ok};
    for (int nn0 = 0; nn0 < 729; nn0 += 32) {
      const int nn = nn0 + lane;
      const bool live = nn < 729;
      double3 p = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
      double v;
      int f;
      warp_point<MIXED, false>(P, W, p, c, live, clamp, lane, &v, &f);
      if (!live) continue;
      S.flag[nn] = int8_t(f);
      if (f == 3) {
        pending++;
        continue;
      }
      if (a.d_out) a.d_out[bi * 729 + nn] = v;
      if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
      S.u.f[nn] = f == 0 ? v : NAN;
      cnt[f]++;
    }
    __syncwarp();
    // the nodes the list left undecided (rare: a feature whose certificate failed there,
    // or more candidates than the list holds): the whole tree walk, a lane a node, kept
    // out of the loop above so that its code stays small
    if (__any_sync(FULL, pending > 0)) {
      for (int nn = lane; nn < 729; nn += 32) {
        if (S.flag[nn] != 3) continue;
        double3 p = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
        double v;
        int f;
        point_fallback(P, p, clamp, &v, &f);
        if (a.d_out) a.d_out[bi * 729 + nn] = v;
        if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
        S.flag[nn] = int8_t(f);
        S.u.f[nn] = f == 0 ? v : NAN;
        cnt[f]++;
      }
      __syncwarp();
    }
    const int n_exact = __reduce_add_sync(FULL, cnt[0]), n_far = __reduce_add_sync(FULL, cnt[1]),
              n_und = __reduce_add_sync(FULL, cnt[2]);
    int provisional = 0;
    if (a.words_out || a.kind_out)
      provisional = brick_post<double>(S.u.f, S.flag, S.v.mk, first, h, clamp, dc, 0.0, n_far,
                                       a.words_out ? a.words_out + bi * WORD_STRIDE : nullptr,
                                       a.kind_out ? a.kind_out + bi : nullptr, lane);
    if (a.stats) brick_census(P, S.code, n, overflow, n_exact, n_far, n_und, provisional, a.stats, lane);
    __syncwarp();
  }
}

void launch_bricks(const BrickArgs& a, cudaStream_t s, int warps) {
  warps = warps == 1 || warps == 2 ? warps : MAX_WARPS;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // eight warps a SM whatever the block (the register budget), a block per brick at most
  const int64_t want = (a.n + warps - 1) / warps;
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sms) * (8 / warps))));
  const size_t smem = sizeof(BrickSmem) * warps;
  const bool batch = a.parts != nullptr;
  if (a.mixed) return launch_bricks_mixed(a, s, warps);
  if (batch)
    k_bricks_t<false, true><<<grid, warps * 32, smem, s>>>(a);
  else
    k_bricks_t<false, false><<<grid, warps * 32, smem, s>>>(a);
}

}  // namespace icam

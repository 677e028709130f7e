// The mixed form's brick kernel on sm_100a (ICAM_MIXED, ICAM_MIXED_LEARNED): one warp a
// brick, as the plain kernel (bricks.cu), with the node work split by precision. The
// bulk runs in single precision (warp_float.cuh), every lane sweeping a run of 23
// neighbouring nodes so that each Newton solve starts from the previous node's foot;
// the few nodes the float walk cannot settle (a distance near zero, where the sign is
// decided; a stalled or uncertified solve; a deferred feature) are gathered and read by
// the plain form's double walk afterwards, 32 at a time, so the hot loop carries no
// double evaluator and the kernel runs at three blocks a SM instead of two.
#include "brick_post.cuh"
#include "kernels.h"
#include "seednet.cuh"
#include "warp_float.cuh"

namespace icam {

namespace {

constexpr int MW = 4;  // bricks a block works on at once, one a warp (1, 2 or 4)
constexpr int SN_ROOM = 32 * SN_KS * 2 + 32 * 8 * 4;  // the seed network's activations

struct BrickSmemF {
  union {
    struct {
      union {
        float f[729];  // node values: exact, signed far, bridged; NaN while unknown
        struct {
          uint32_t code[MAXC];
          double lb[MAXC];
          int32_t fr[2][FR];
        } list;
      } u;
      float4 res[16 * NRES];  // the resident nets (staged after the seed network has run)
    } w;
    unsigned char net[SN_ROOM];  // the seed network's activations, before the nets come
  } x;
  double lb64[MAXC];  // ranked candidates: lower bound at the centre (double, then float
  float lbf[MAXC];    //   rounded down), the least bound from each on, code, float geometry
  float lbs[MAXC];    //   (WarpCandsF); lbs holds the ranking keys until the walk
  uint32_t code[MAXC];
  float4 geo[2 * MAXC];
  double4 net[16];  // the control net the double walk is on
  float4 net32[16];
  union {
    SeedF seed[MAXSUB];
    RowMasks mk;        // after the nodes: node masks by row
    int16_t pend[736];  // between: the nodes left for the double walk
  } v;
  int8_t flag[729];
  int8_t cert[MAXC];
  int8_t slot[MAXC];
  int8_t rslot[MAXC];
  uint32_t residx[NRES];
  uint64_t bar;  // the bulk copies' barrier
  int n;
};
static_assert(sizeof(((BrickSmemF*)0)->x) >= SN_ROOM, "the seed network's room");

// The i16 step's half: a distance below it (less the float error) rounds to zero on
// either side of the surface, so a bake that keeps only i16 values needs no sign for it.
__device__ __forceinline__ float quantised_zero(double clamp) {
  return float(fmax(0.5 * clamp / 32767.0 - 5e-6, 0.0));
}

// One brick a warp:
//  0. the centre-distance shortcuts of the plain kernel, with the centre distance known
//     within a.dc_err;
//  1. the list and its ranking (double, as the plain kernel);
//  2. per candidate (a lane each): its bound rounded down to a float, its geometry
//     relative to the centre, its certificate (sub-patch convex over the brick; plane
//     trim over the brick's feet) and, for the first MAXSUB sub-patches, a float Newton
//     solution at the centre for seeds (started where the seed network puts it);
//  3. the nodes by the float walk in three groups of 32 columns (x fastest, then y),
//     each column swept in z: the warp's 32 nodes lie close together at every step (so
//     they walk few candidates beyond their own), and a lane's next node is its last
//     one's neighbour (so its solve starts at that node's foot);
//  4. the nodes left over, 32 at a time, by the plain form's double walk;
//  5. far nodes signed, undecided ones bridged, quantised and packed.
template <bool BATCH>
__global__ void __launch_bounds__(MW * 32, ICAM_MIXED_BLOCKS) k_bricks_m(BrickArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BrickSmemF* smem = reinterpret_cast<BrickSmemF*>(smem_raw);
  const int warps = int(blockDim.x >> 5);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BrickSmemF& S = smem[warp];
  unsigned long long* work = a.stats ? a.stats + 15 : nullptr;
  if (lane == 0) mbar_init(&S.bar);
  __syncwarp();
  uint32_t phase = 0;
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
    const float* net_feat = BATCH ? Q->net_feat : a.net_feat;
    // the seed network's weights are read through L1 from global memory: staged in shared
    // memory they took 25 KB a block of the L1 the kernel's spills live in (measured:
    // learned node phase 28.7 ms staged, 27.4 ms read)
    const void* net_w = BATCH ? Q->net_w : a.net_w;
    const double3 first = mk(a.firsts[3 * bi], a.firsts[3 * bi + 1], a.firsts[3 * bi + 2]);
    const double half = 4.0 * h;
    const double3 c = first + mk(half, half, half);
    const double reach = half * SQRT3 + clamp;
    const double dc = a.dcs ? a.dcs[bi] : NAN;
    const double dce = a.dc_err;
    // ---- 0. every node past the clamp (bricks.cu, step 0), with dc known within dce
    if (isfinite(dc) && fabs(dc) - dce - half * SQRT3 > clamp + 1e-6 * (1.0 + clamp)) {
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
    // ---- 0b. every node on one side by more than an i16 step (bricks.cu, step 0b)
    if (a.kind_only && isfinite(dc) && fabs(dc) > dce && settles_by_sign(fabs(dc) - dce, h, clamp)) {
      if (lane == 0) {
        if (a.kind_out) a.kind_out[bi] = dc > 0 ? 1 : 2;
        if (a.stats) atomicAdd(&a.stats[11], 1ull);
      }
      continue;
    }
    // ---- 1. list
    int n = warp_list(P, leaves, n_leaves, c, reach, S.x.w.u.list.code, S.x.w.u.list.lb, S.x.w.u.list.fr, &S.n, lane);
    // a list past its room is taken again with a shorter reach (down to 0.8^4 of it) until
    // it fits: its nodes whose answer lies within the shorter reach (less their distance
    // from the centre) need nothing more, the rest go to the tree walk
    double reach_ok = INFINITY;
    for (int tries = 0; n > MAXC && tries < 4; tries++) {
      reach_ok = (tries == 0 ? reach : reach_ok) * 0.8;
      n = warp_list(P, leaves, n_leaves, c, reach_ok, S.x.w.u.list.code, S.x.w.u.list.lb, S.x.w.u.list.fr, &S.n, lane);
    }
    const bool overflow = n > MAXC;
    if (overflow) n = MAXC;
    warp_rank(S.x.w.u.list.code, S.x.w.u.list.lb, n, S.code, S.lb64, lane);
    // ---- 2. per candidate
    {
      int subs_before = 0;
      for (int base = 0; base < n; base += 32) {
        const int k = base + lane;
        const bool is_sub = k < n && (S.code[k] >> IK_SHIFT) == IK_SUB;
        const unsigned m = __ballot_sync(FULL, is_sub);
        const int before = subs_before + __popc(m & ((1u << lane) - 1u));
        subs_before += __popc(m);
        float s0 = 0.5f, t0 = 0.5f;
        // the seed network's starts, this group of candidates on the tensor cores (groups
        // holding sub-patches that take seeds only)
        if (net_w && __any_sync(FULL, is_sub && before < MAXSUB)) {
          float x[SN_IN], y[3];
          const int fi = is_sub ? int(S.code[k] & IK_MASK) : 0;
          sn_input(net_feat + size_t(fi) * SN_FEAT, c, x);
          __nv_bfloat16* act = reinterpret_cast<__nv_bfloat16*>(S.x.net);
          sn_forward_warp(net_w, act, reinterpret_cast<float*>(act + 32 * SN_KS), x, y, lane);
          s0 = fminf(fmaxf(y[0], 0.f), 1.f), t0 = fminf(fmaxf(y[1], 0.f), 1.f);
          // the net's distance from the centre (its third output is d / L), the ranking key
          if (is_sub) S.lbs[k] = fmaxf(y[2] / net_feat[size_t(S.code[k] & IK_MASK) * SN_FEAT + 12], 0.f);
        }
        if (k >= n) continue;
        const uint32_t code = S.code[k], idx = code & IK_MASK;
        int slot = -1, rslot = -1;
        int8_t cert = 0;
        float4 g0 = make_float4(0.f, 0.f, 0.f, 0.f), g1 = g0;
        S.lbf[k] = __double2float_rd(S.lb64[k]);
        // the key: the net's distance for a sub-patch it saw (no nearer than the bound), else the bound
        S.lbs[k] = (net_w && is_sub && before < MAXSUB && !__isnanf(S.lbs[k])) ? fmaxf(S.lbs[k], S.lbf[k]) : S.lbf[k];
        if (is_sub) {
          const DSub& s = P.subs[idx];
          cert = sub_convex(s, first, first + mk(8 * h, 8 * h, 8 * h)) ? 1 : 0;
          g0 = make_float4(float(s.c[0] - c.x), float(s.c[1] - c.y), float(s.c[2] - c.z), float(P.faces[s.face].sense));
          // half extents rounded up: a lower bound stays a lower bound
          g1 = make_float4(__double2float_ru(0.5 * (s.box[3] - s.box[0])), __double2float_ru(0.5 * (s.box[4] - s.box[1])),
                           __double2float_ru(0.5 * (s.box[5] - s.box[2])), s.klass == 1 ? 1.f : 0.f);
          if (before < NRES) {
            rslot = before;
            S.residx[before] = idx;
          }
          if (before < MAXSUB) {
            slot = before;
            const float3 qc = f3(float(c.x - s.c[0]), float(c.y - s.c[1]), float(c.z - s.c[2]));
            S.v.seed[slot] = seed_at_f(P.sub_cp32 + 16 * size_t(idx), qc, s0, t0);
          }
        } else if ((code >> IK_SHIFT) == IK_FACE) {
          const DFace& f = P.faces[idx];
          if (f.kind == S_PLANE) {
            const double3 z = ld3(f.z) * f.sense, o = ld3(f.o);
            g0 = make_float4(float(z.x), float(z.y), float(z.z), float(dot(o - c, z)));
            // the trim over the feet of the whole brick: 1 all inside, 2 all outside, 0 ask
            double blo[2] = {INFINITY, INFINITY}, bhi[2] = {-INFINITY, -INFINITY};
            const double3 zz = ld3(f.z), fx = ld3(f.x), fy = ld3(f.y);
            for (int q = 0; q < 8; q++) {
              double3 x = first + mk(q & 1 ? 8 * h : 0.0, q & 2 ? 8 * h : 0.0, q & 4 ? 8 * h : 0.0);
              double3 e = (x - zz * dot(x - o, zz)) - o;
              double u = dot(e, fx), v = dot(e, fy);
              blo[0] = fmin(blo[0], u), bhi[0] = fmax(bhi[0], u);
              blo[1] = fmin(blo[1], v), bhi[1] = fmax(bhi[1], v);
            }
            double mg = 1e-9 * (1.0 + fmax(fmax(fabs(blo[0]), fabs(bhi[0])), fmax(fabs(blo[1]), fabs(bhi[1]))));
            blo[0] -= mg, blo[1] -= mg, bhi[0] += mg, bhi[1] += mg;
            const int cls = trim_box_class(P, f, blo, bhi);
            cert = cls == 1 ? 1 : (cls == 0 ? 2 : 0);
          } else {
            g0.w = NAN;  // a curved face: the double evaluator
          }
        }
        S.geo[2 * k] = g0;
        S.geo[2 * k + 1] = g1;
        S.cert[k] = cert;
        S.slot[k] = int8_t(slot);
        S.rslot[k] = int8_t(rslot);
      }
      __syncwarp();
      // ICAM_MIXED_LEARNED: the candidates ranked by the seed network's distance instead of
      // their bound, so that the walk meets the nearest sub-patch first and the bound it
      // sets rules the others out; the walk leaves once the least bound of what is left
      // (lbs, the suffix minimum) is past every lane's answer, so the answers are the same
      if (net_w) {
        int pos[MAXC / 32];
#pragma unroll
        for (int q = 0; q < MAXC / 32; q++) {
          const int k = lane + 32 * q;
          pos[q] = k;
          if (k < n) {
            const float key = S.lbs[k];
            int p = 0;
            for (int j = 0; j < n; j++) {
              const float kj = S.lbs[j];
              p += (kj < key) || (kj == key && j < k);
            }
            pos[q] = p;
          }
        }
        auto move = [&](auto* arr) {
          decltype(+arr[0]) val[MAXC / 32];
#pragma unroll
          for (int q = 0; q < MAXC / 32; q++)
            if (lane + 32 * q < n) val[q] = arr[lane + 32 * q];
          __syncwarp();
#pragma unroll
          for (int q = 0; q < MAXC / 32; q++)
            if (lane + 32 * q < n) arr[pos[q]] = val[q];
          __syncwarp();
        };
        move(S.code);
        move(S.lb64);
        move(S.lbf);
        move(S.cert);
        move(S.slot);
        move(S.rslot);
        {
          float4 va[MAXC / 32], vb[MAXC / 32];
#pragma unroll
          for (int q = 0; q < MAXC / 32; q++)
            if (lane + 32 * q < n) va[q] = S.geo[2 * (lane + 32 * q)], vb[q] = S.geo[2 * (lane + 32 * q) + 1];
          __syncwarp();
#pragma unroll
          for (int q = 0; q < MAXC / 32; q++)
            if (lane + 32 * q < n) S.geo[2 * pos[q]] = va[q], S.geo[2 * pos[q] + 1] = vb[q];
          __syncwarp();
        }
        if (lane == 0) {
          float m = INFINITY;
          for (int k = n - 1; k >= 0; k--) {
            m = fminf(m, S.lbf[k]);
            S.lbs[k] = m;
          }
        }
        __syncwarp();
      }
      // the first NRES sub-patches' nets staged into shared memory for the whole brick
      const int nres = min(subs_before, NRES);
      if (nres > 0) {
        if (lane == 0) stage_nets(S.x.w.res, P.sub_cp32, S.residx, nres, &S.bar);
        if (!mbar_wait(&S.bar, phase)) {  // never expected: record it, let the copies land, leave
          if (a.stats && lane == 0) atomicAdd(&a.stats[13], 1ull);
          mbar_wait(&S.bar, phase);
          return;
        }
        phase ^= 1u;
      }
    }
    __syncwarp();
    // ---- 3. the float walk: column 32 g + lane of the 81, swept in z
    int cnt[3] = {0, 0, 0};
    int pending = 0, n_evals = 0, n_solves = 0;
    {
      const WarpCandsF W{S.code, S.lbf, S.lbs, S.cert, S.slot, S.v.seed, S.geo, S.net32, S.x.w.res, S.rslot, n, 8,
                         float(reach_ok * (1.0 - 1e-6)) - 1e-5f};
      int lastk = -1;
      float ls = 0.f, lt = 0.f;
      const float hf = float(h);
      const float qz = (a.d_out || a.flag_out) ? 0.f : quantised_zero(clamp);
      for (int q = 0; q < 27; q++) {
        const int col = 32 * (q / 9) + lane, kk = q % 9;
        const bool live = col < 81;
        const int nn = live ? col + 81 * kk : 0;
        const int i = nn % 9, j = (nn / 9) % 9;
        const float3 pc = f3(hf * float(i - 4), hf * float(j - 4), hf * float(kk - 4));
        const double3 p = first + mk(h * i, h * j, h * kk);
        float v = 0.f;
        int f = 3;
        if (!overflow)
          f = warp_point_f(P, W, pc, p, live, float(clamp), lane, &v, &lastk, &ls, &lt, qz, &n_evals, &n_solves);
        if (!live) continue;
        S.flag[nn] = int8_t(f);
        if (f == 3) {
          pending++;
          continue;
        }
        if (a.d_out) a.d_out[bi * 729 + nn] = double(v);
        if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
        S.x.w.u.f[nn] = f == 0 ? v : NAN;
        cnt[f]++;
      }
    }
    __syncwarp();
    // ---- 4. the nodes left over, gathered and read by the double walk
    const int npend = __reduce_add_sync(FULL, pending);
    if (npend > 0) {
      int base = 0;
      for (int nn0 = 0; nn0 < 729; nn0 += 32) {
        const int nn = nn0 + lane;
        const bool pd = nn < 729 && S.flag[nn] == 3;
        const unsigned m = __ballot_sync(FULL, pd);
        if (pd) S.v.pend[base + __popc(m & ((1u << lane) - 1u))] = int16_t(nn);
        base += __popc(m);
      }
      __syncwarp();
      // the double walk's list: the same candidates, centre starts (no seeds)
      const WarpCands W64{S.code, S.lb64, net_w ? S.lbs : nullptr, S.cert, nullptr, nullptr, S.net, S.net32, n, overflow,
                          reach_ok};
      int tail = 0;
      for (int b0 = 0; b0 < npend; b0 += 32) {
        const bool live = b0 + lane < npend;
        const int nn = live ? S.v.pend[b0 + lane] : 0;
        const double3 p = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
        double v;
        int f;
        warp_point<false, false>(P, W64, p, c, live, clamp, lane, &v, &f);
        if (!live) continue;
        S.flag[nn] = int8_t(f);
        if (f == 3) {
          tail++;
          continue;
        }
        if (a.d_out) a.d_out[bi * 729 + nn] = v;
        if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
        S.x.w.u.f[nn] = f == 0 ? float(v) : NAN;
        cnt[f]++;
      }
      __syncwarp();
      // what the list cannot settle: the whole tree walk
      if (__any_sync(FULL, tail > 0)) {
        for (int q = lane; q < npend; q += 32) {
          const int nn = S.v.pend[q];
          if (S.flag[nn] != 3) continue;
          const double3 p = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
          double v;
          int f;
          point_fallback(P, p, clamp, &v, &f);
          if (a.d_out) a.d_out[bi * 729 + nn] = v;
          if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
          S.flag[nn] = int8_t(f);
          S.x.w.u.f[nn] = f == 0 ? float(v) : NAN;
          cnt[f]++;
        }
      }
      __syncwarp();
      if (a.stats && lane == 0) atomicAdd(&a.stats[12], (unsigned long long)npend);
    }
    const int n_exact = __reduce_add_sync(FULL, cnt[0]), n_far = __reduce_add_sync(FULL, cnt[1]),
              n_und = __reduce_add_sync(FULL, cnt[2]);
    int provisional = 0;
    if (a.words_out || a.kind_out)
      provisional = brick_post<float>(S.x.w.u.f, S.flag, S.v.mk, first, h, clamp, dc, dce, n_far,
                                      a.words_out ? a.words_out + bi * WORD_STRIDE : nullptr,
                                      a.kind_out ? a.kind_out + bi : nullptr, lane);
    if (a.stats) {
      brick_census(P, S.code, n, overflow, n_exact, n_far, n_und, provisional, a.stats, lane);
      n_evals = __reduce_add_sync(FULL, n_evals);
      n_solves = __reduce_add_sync(FULL, n_solves);
      if (lane == 0 && n_solves) {
        atomicAdd(&a.stats[16], (unsigned long long)n_evals);
        atomicAdd(&a.stats[17], (unsigned long long)n_solves);
      }
    }
    __syncwarp();
  }
}

}  // namespace

void launch_bricks_mixed(const BrickArgs& a, cudaStream_t s, int warps) {
  warps = warps == 1 || warps == 2 ? warps : MW;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool batch = a.parts != nullptr;
  const size_t smem = sizeof(BrickSmemF) * warps;
  auto kern = batch ? k_bricks_m<true> : k_bricks_m<false>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(BrickSmemF) * MW));
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem);
  const int64_t want = (a.n + warps - 1) / warps;
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sms) * std::max(per_sm, 1))));
  kern<<<grid, warps * 32, smem, s>>>(a);
}

}  // namespace icam

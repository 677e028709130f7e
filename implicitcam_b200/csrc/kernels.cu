// Kernels of the exact part field on sm_100a: point queries through the feature tree,
// the fused brick kernel (culling, every node's exact value, the far-node fill and
// bridging of partcache.rs:790-917, quantisation and packing), and the box decision of
// a level (partcache.rs:226-331).
#include <cub/cub.cuh>

#include <type_traits>

#include "field.cuh"
#include "kernels.h"

namespace icam {

// ---------------------------------------------------------------- point queries

__global__ void k_points(DPack P, const double* __restrict__ xyz, int64_t n, double cap, double* __restrict__ value,
                         int8_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double3 p = mk(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    Acc A;
    point_query(P, p, cap, A);
    double v;
    int f;
    finish(A, cap, &v, &f);
    value[i] = v;
    flag[i] = int8_t(f);
  }
}

// ---------------------------------------------------------------- bricks

constexpr int BRICK_THREADS = 256;
constexpr int MAXC = 128;   // candidates a brick may list
constexpr int MAXSUB = 32;  // sub-patch control nets staged in shared memory a brick

// The 26 neighbours of node n inside the brick, in the reference's order (dk, dj, di
// from -1 to 1, partcache.rs:829-839).
__device__ __forceinline__ int nb_of(int n, int k, double* dist) {
  int i = n % 9, j = (n / 9) % 9, kk = n / 81;
  int o = k < 13 ? k : k + 1;  // skip (0,0,0)
  int di = o % 3 - 1, dj = (o / 3) % 3 - 1, dk = o / 9 - 1;
  int a = i + di, b = j + dj, c = kk + dk;
  if (a < 0 || a > 8 || b < 0 || b > 8 || c < 0 || c > 8) return -1;
  *dist = sqrt(double(di * di + dj * dj + dk * dk));
  return a + 9 * b + 81 * c;
}

// A node the candidate list could not settle (more candidates than the list holds, or a
// feature whose certificate fails there): the whole tree walk with every fallback, out
// of line so the common path keeps its registers.
__device__ __noinline__ void node_fallback(const DPack& P, double3 p, double clamp, double* value, int* flag) {
  Acc A;
  point_query(P, p, clamp, A);
  finish(A, clamp, value, flag);
}

// A staged sub-patch's solution at the brick's centre, for first-order seeds at the
// nodes: (s, t) there, the inverse Hessian of |S - c|^2 and the tangents, so that
// (s, t)(p) ~ (s, t) + H^-1 [S_s.(p - c), S_t.(p - c)].
struct Seed {
  double s, t, i00, i01, i11;
  double ss[3], st[3];
};

// One brick a block (the reference's per-brick list and read, partcache.rs:759-917):
//  1. list: the tree's leaves and their features within half sqrt(3) + clamp of the
//     brick's centre (GpuPack::list with r = 0, partcache.rs:767), ranked by that bound;
//  2. each sub-patch among the first MAXSUB: its control net staged in shared memory,
//     its convexity certified for the whole brick, and its Newton solution at the
//     centre kept for seeds;
//  3. candidate by candidate, every lane on its nodes at once (the warp leaves when all
//     its nodes are nearer than the next bound), each node capped at the clamp; a
//     feature uncertified at a node sends that node to the tree walk afterwards;
//  4. far nodes signed, undecided ones bridged, quantised and packed.
// MIXED: sub-patches run Newton in floats on the rebased nets and are polished in
// doubles (with the critical-point test and the trim) only when their float distance
// can beat the node's answer.
template <bool MIXED>
__global__ void __launch_bounds__(BRICK_THREADS, 2) k_bricks_t(BrickArgs a) {
  const DPack& P = a.P;
  __shared__ uint32_t s_tcode[MAXC];
  __shared__ double s_tlb[MAXC];
  __shared__ uint32_t s_code[MAXC];
  __shared__ double s_lb[MAXC];
  __shared__ int8_t s_cert[MAXC];
  __shared__ int8_t s_slot[MAXC];
  __shared__ Seed s_seed[MAXSUB];
  __shared__ typename std::conditional<MIXED, float4, double4>::type s_cp[MAXSUB * 16];
  __shared__ int s_n;
  __shared__ double s_f[729];
  __shared__ double s_exact[729];
  __shared__ int8_t s_flag[729];
  __shared__ int s_changed;
  __shared__ int s_cnt[4];
  const int tid = threadIdx.x;
  for (int64_t bi = blockIdx.x; bi < a.n; bi += gridDim.x) {
    const double h = a.h, clamp = a.clamp;
    double3 first = mk(a.firsts[3 * bi], a.firsts[3 * bi + 1], a.firsts[3 * bi + 2]);
    double half = 4.0 * h;
    double3 c = first + mk(half, half, half);
    double reach = half * SQRT3 + clamp;
    if (tid == 0) s_n = 0;
    if (tid < 4) s_cnt[tid] = 0;
    __syncthreads();
    // ---- 1. list
    for (int leaf = tid; leaf < a.n_leaves; leaf += BRICK_THREADS) {
      const DBvh& nd = P.bvh[a.leaves[leaf]];
      if (box_dist_f(c, nd.lo, nd.hi) > reach) continue;
      for (int k = 0; k < nd.count; k++) {
        uint32_t code = P.items[nd.first + k];
        double lb = item_lb(P, code, c);
        if (lb <= reach) {
          int slot = atomicAdd(&s_n, 1);
          if (slot < MAXC) {
            s_tcode[slot] = code;
            s_tlb[slot] = lb;
          }
        }
      }
    }
    __syncthreads();
    int n = s_n;
    bool overflow = n > MAXC;
    if (overflow) n = MAXC;
    // rank sort: ties by code so the order does not depend on the list's arrival order
    for (int k = tid; k < n; k += BRICK_THREADS) {
      double lb = s_tlb[k];
      uint32_t code = s_tcode[k];
      int rank = 0;
      for (int j = 0; j < n; j++) {
        double l2 = s_tlb[j];
        rank += (l2 < lb) || (l2 == lb && s_tcode[j] < code);
      }
      s_code[rank] = code;
      s_lb[rank] = lb;
    }
    __syncthreads();
    // ---- 2. stage, certify and seed the first MAXSUB sub-patches
    for (int k = tid; k < n; k += BRICK_THREADS) {
      uint32_t code = s_code[k];
      int slot = -1;
      s_cert[k] = 0;
      if ((code >> IK_SHIFT) == IK_SUB) {
        int before = 0;
        for (int j = 0; j < k; j++) before += (s_code[j] >> IK_SHIFT) == IK_SUB;
        const DSub& s = P.subs[code & IK_MASK];
        s_cert[k] = sub_convex(s, first, first + mk(8 * h, 8 * h, 8 * h)) ? 1 : 0;
        if (before < MAXSUB) {
          slot = before;
          const double4* cp = P.sub_cp + 16 * size_t(code & IK_MASK);
          double ss = 0.5, tt = 0.5;
          bool conv;
          newton_bicubic(cp, c, &ss, &tt, 12, &conv);
          SE e = eval_bicubic(cp, ss, tt);
          double3 r = e.p - c;
          double h0 = dot(e.ps, e.ps) + dot(e.pss, r), h1 = dot(e.ps, e.pt) + dot(e.pst, r),
                 h2 = dot(e.pt, e.pt) + dot(e.ptt, r);
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
          s_seed[slot] = sd;
        }
      }
      s_slot[k] = int8_t(slot);
    }
    __syncthreads();
    for (int e = tid; e < n * 16; e += BRICK_THREADS) {  // control nets of the staged sub-patches
      int k = e >> 4, j = e & 15;
      int slot = s_slot[k];
      if (slot < 0) continue;
      uint32_t i = s_code[k] & IK_MASK;
      if (MIXED)
        reinterpret_cast<float4*>(s_cp)[16 * slot + j] = P.sub_cp32[16 * size_t(i) + j];
      else
        reinterpret_cast<double4*>(s_cp)[16 * slot + j] = P.sub_cp[16 * size_t(i) + j];
    }
    __syncthreads();
    // ---- 3. every node: the warp's lanes walk the same ranked candidates together
    for (int nn0 = 0; nn0 < 729; nn0 += BRICK_THREADS) {
      const int nn = nn0 + tid;
      const bool live = nn < 729;
      double3 p = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
      double rr = len(p - c);
      double best = live ? clamp : -1.0;  // a lane past the last node is done
      double sdv = NAN, und = INFINITY;
      if (!overflow) {
        for (int k = 0; k < n; k++) {
          double lbc = s_lb[k];
          if (__all_sync(0xffffffffu, lbc - rr >= best)) break;  // ranked: nothing later is nearer
          if (lbc - rr >= best) continue;
          uint32_t code = s_code[k];
          uint32_t kind = code >> IK_SHIFT, idx = code & IK_MASK;
          if (kind != IK_SUB) {
            Acc A;
            A.best = best;
            A.sd = sdv;
            A.und = und;
            A.why = 0;
            A.ub = INFINITY;
            A.nd = 0;
            A.record = true;  // an uncertified piece records its bound in und
            eval_item(P, code, p, A, 0, 0.5, 0.5);
            best = A.best;
            sdv = A.sd;
            und = A.und;
            continue;
          }
          const DSub& s = P.subs[idx];
          double lb = box_dist(p, s.box);
          if (lb >= best) continue;
          if (!s_cert[k] && !sub_convex(s, p, p)) {
            und = fmin(und, lb);
            continue;
          }
          int slot = s_slot[k];
          double ss = 0.5, tt = 0.5;
          if (slot >= 0) {
            const Seed& sd = s_seed[slot];
            double3 dp = p - c;
            double gs = sd.ss[0] * dp.x + sd.ss[1] * dp.y + sd.ss[2] * dp.z;
            double gt = sd.st[0] * dp.x + sd.st[1] * dp.y + sd.st[2] * dp.z;
            ss = fmin(fmax(sd.s + sd.i00 * gs + sd.i01 * gt, 0.0), 1.0);
            tt = fmin(fmax(sd.t + sd.i01 * gs + sd.i11 * gt, 0.0), 1.0);
          }
          const double4* cp64 = (!MIXED && slot >= 0) ? reinterpret_cast<const double4*>(s_cp) + 16 * slot
                                                      : P.sub_cp + 16 * size_t(idx);
          bool conv;
          if (MIXED) {
            const float4* cp32 = slot >= 0 ? reinterpret_cast<const float4*>(s_cp) + 16 * slot
                                           : P.sub_cp32 + 16 * size_t(idx);
            float3 p32 = f3(float(p.x - s.c[0]), float(p.y - s.c[1]), float(p.z - s.c[2]));
            float sf = float(ss), tf = float(tt);
            newton_bicubic_f(cp32, p32, &sf, &tf, 8);
            SEf ef = eval_bicubic_f(cp32, sf, tf);
            float3 rf = f3(ef.p.x - p32.x, ef.p.y - p32.y, ef.p.z - p32.z);
            double d32 = sqrt(double(dotf(rf, rf)));
            // a float distance past the answer by more than its error cannot win
            if (d32 > best + 1e-4 * (1.0 + best)) continue;
            ss = sf, tt = tf;
            newton_bicubic(cp64, p, &ss, &tt, 3, &conv);
            if (!conv) newton_bicubic(cp64, p, &ss, &tt, 16, &conv);
          } else {
            newton_bicubic(cp64, p, &ss, &tt, 16, &conv);
          }
          if (!conv) {
            und = fmin(und, lb);
            continue;
          }
          SE e = eval_bicubic(cp64, ss, tt);
          double d = len(e.p - p);
          if (!(d < best) || !is_critical(p, e)) continue;
          double3 nrm = cross(e.ps, e.pt);
          if (!(len(nrm) > 0.0)) continue;
          if (s.klass != 1 &&
              !trim_inside(P, P.faces[s.face], s.u0 + ss * (s.u1 - s.u0), s.v0 + tt * (s.v1 - s.v0)))
            continue;
          best = d;
          sdv = d * sgn(dot(p - e.p, unit(nrm) * P.faces[s.face].sense));
        }
      }
      if (!live) continue;
      double v;
      int f;
      if (overflow || (und < best && und <= clamp)) {
        node_fallback(P, p, clamp, &v, &f);
      } else if (!isnan(sdv) && best <= clamp) {
        v = sdv, f = 0;
      } else {
        v = clamp, f = 1;
      }
      if (a.d_out) a.d_out[bi * 729 + nn] = v;
      if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
      s_flag[nn] = int8_t(f);
      s_f[nn] = f == 0 ? v : NAN;
      s_exact[nn] = s_f[nn];
      atomicAdd(&s_cnt[f], 1);
    }
    __syncthreads();
    if (a.words_out || a.kind_out) {
      // ---- far nodes signed by a neighbour within a cell diagonal (partcache.rs:845-858)
      auto fill = [&]() {
        for (;;) {
          if (tid == 0) s_changed = 0;
          __syncthreads();
          for (int nn = tid; nn < 729; nn += BRICK_THREADS) {
            if (s_flag[nn] != 1 || !isnan(s_f[nn])) continue;
            for (int k = 0; k < 26; k++) {
              double dd;
              int m = nb_of(nn, k, &dd);
              if (m < 0) continue;
              double fm = s_f[m];
              if (fm != 0.0 && !isnan(fm)) {
                s_f[nn] = copysign(clamp, fm);
                s_changed = 1;
                break;
              }
            }
          }
          __syncthreads();
          if (!s_changed) break;
          __syncthreads();
        }
      };
      fill();
      double dc = a.dcs ? a.dcs[bi] : NAN;
      // ---- far nodes in the centre's empty ball, or the centre in theirs (partcache.rs:860-875)
      if (isfinite(dc) && dc != 0.0) {
        double rch = 0.999 * fmax(clamp, fabs(dc));
        for (int nn = tid; nn < 729; nn += BRICK_THREADS) {
          if (s_flag[nn] != 1 || !isnan(s_f[nn])) continue;
          double3 x = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
          if (len(x - c) < rch) s_f[nn] = copysign(clamp, dc);
        }
        __syncthreads();
        fill();
      }
      // ---- every node far: the centre's sign (partcache.rs:876-892)
      if (s_cnt[1] == 729 && isfinite(dc) && dc != 0.0) {
        for (int nn = tid; nn < 729; nn += BRICK_THREADS) s_f[nn] = copysign(clamp, dc);
        __syncthreads();
      }
      // ---- bridging: the mean of the known neighbours, held in the brackets the exact
      // ones give (partcache.rs:893-916), pass after pass
      int provisional = 0;
      for (int pass = 0; pass < 729; pass++) {
        if (tid == 0) s_changed = 0;
        __syncthreads();
        double nv[3];
        int todo[3];
        int nt = 0;
        for (int nn = tid; nn < 729; nn += BRICK_THREADS) {
          if (!isnan(s_f[nn])) continue;
          double sum = 0.0, lo = -clamp, hi = clamp;
          int cnt = 0;
          for (int k = 0; k < 26; k++) {
            double dd;
            int m = nb_of(nn, k, &dd);
            if (m < 0) continue;
            if (!isnan(s_f[m])) {
              sum += s_f[m];
              cnt++;
            }
            if (!isnan(s_exact[m])) {
              lo = fmax(lo, s_exact[m] - dd * h);
              hi = fmin(hi, s_exact[m] + dd * h);
            }
          }
          if (cnt == 0) continue;
          double vm = sum / cnt;
          nv[nt] = lo <= hi ? fmin(fmax(vm, lo), hi) : 0.5 * (lo + hi);
          todo[nt++] = nn;
        }
        __syncthreads();
        for (int q = 0; q < nt; q++) {
          s_f[todo[q]] = nv[q];
          s_changed = 1;
          provisional++;
        }
        __syncthreads();
        if (!s_changed) break;
      }
      // nothing around them known: the brick's far side, taken as air
      for (int nn = tid; nn < 729; nn += BRICK_THREADS)
        if (isnan(s_f[nn])) {
          s_f[nn] = clamp;
          provisional++;
        }
      if (provisional) atomicAdd(&s_cnt[3], provisional);
      __syncthreads();
      // ---- quantise and pack
      int pos = 1, nonpos = 1;
      for (int nn = tid; nn < 729; nn += BRICK_THREADS) {
        double x = fmin(fmax(s_f[nn] / clamp, -1.0), 1.0) * 32767.0;
        double q = round(x);
        s_f[nn] = q;
        if (!(q > 0)) pos = 0;
        if (!(q <= 0)) nonpos = 0;
      }
      int all_pos = __syncthreads_and(pos), all_nonpos = __syncthreads_and(nonpos);
      int kind = all_pos ? 1 : (all_nonpos ? 2 : 0);
      if (a.kind_out && tid == 0) a.kind_out[bi] = kind;
      if (a.words_out)
        for (int w = tid; w < 365; w += BRICK_THREADS) {
          uint32_t lo = uint32_t(uint16_t(int16_t(s_f[2 * w])));
          uint32_t hi = 2 * w + 1 < 729 ? uint32_t(uint16_t(int16_t(s_f[2 * w + 1]))) << 16 : 0u;
          a.words_out[bi * 365 + w] = lo | hi;
        }
    }
    if (tid == 0 && a.stats) {
      atomicAdd((unsigned long long*)&a.stats[0], (unsigned long long)s_cnt[0]);
      atomicAdd((unsigned long long*)&a.stats[1], (unsigned long long)s_cnt[1]);
      atomicAdd((unsigned long long*)&a.stats[2], (unsigned long long)s_cnt[2]);
      atomicAdd((unsigned long long*)&a.stats[3], (unsigned long long)s_cnt[3]);
      atomicAdd((unsigned long long*)&a.stats[4], (unsigned long long)n);
      // the census by kind, B-spline sub-patches counted by their distinct spans
      unsigned long long kinds[5] = {0, 0, 0, 0, 0};
      for (int k = 0; k < n; k++) {
        uint32_t kind = s_code[k] >> IK_SHIFT;
        if (kind == IK_SUB) {
          const DSub& s = P.subs[s_code[k] & IK_MASK];
          bool seen = false;
          for (int j = 0; j < k && !seen; j++)
            if ((s_code[j] >> IK_SHIFT) == IK_SUB) {
              const DSub& o = P.subs[s_code[j] & IK_MASK];
              seen = o.nurbs == s.nurbs && o.span_a == s.span_a && o.span_b == s.span_b;
            }
          if (!seen) kinds[1]++;
        } else {
          kinds[kind == IK_FACE ? 0 : kind == IK_EDGE ? 2 : kind == IK_PIECE ? 3 : 4]++;
        }
      }
      for (int k = 0; k < 5; k++) atomicAdd((unsigned long long*)&a.stats[6 + k], kinds[k]);
      if (overflow) atomicAdd((unsigned long long*)&a.stats[5], 1ull);
    }
    __syncthreads();
  }
}

template __global__ void k_bricks_t<false>(BrickArgs);
template __global__ void k_bricks_t<true>(BrickArgs);

// ---------------------------------------------------------------- the decision of a level

// One box of bricks [first, first + size) a thread: its centre read within `cut`
// (partcache.rs:370-383: a box is decided once its centre is known past the box grown by
// the clamp), decided air or material, split, or (size 1) read.
__global__ void k_decide(DecideArgs a) {
  const DPack& P = a.P;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.n; i += int64_t(gridDim.x) * blockDim.x) {
    Box4 b = a.boxes[i];
    double side = 8.0 * a.h;
    double3 lo = mk(a.lo[0] + side * b.x - a.clamp, a.lo[1] + side * b.y - a.clamp, a.lo[2] + side * b.z - a.clamp);
    double3 hi = mk(a.lo[0] + side * (b.x + a.size) + a.clamp, a.lo[1] + side * (b.y + a.size) + a.clamp,
                    a.lo[2] + side * (b.z + a.size) + a.clamp);
    double3 c = (lo + hi) * 0.5;
    double r = 0.5 * len(hi - lo);
    double cut = (r + a.clamp) * (1.0 + 1e-4);
    Acc A;
    point_query(P, c, cut, A);
    double v;
    int f;
    finish(A, cut, &v, &f);
    double sd = NAN;  // the signed distance at the centre when known
    int verdict;      // 0 split or read, 1 air, 2 material
    if (f == 0) {
      sd = v;
      verdict = (v - r > a.clamp) ? 1 : ((v + r < -a.clamp) ? 2 : 0);
    } else if (f == 1) {
      // past the box: air or material as the parent's centre when the parent's centre
      // lies in this one's empty ball (partcache.rs:401-406); else read without the cut
      double reach = b.reach;
      if (isfinite(b.parent_sd) && b.parent_sd != 0.0 && reach < cut * (1.0 - 1e-6)) {
        verdict = b.parent_sd > 0 ? 1 : 2;
      } else {
        point_query(P, c, INFINITY, A);
        finish(A, INFINITY, &v, &f);
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
    long long nb0 = a.nb[0], nb1 = a.nb[1], nb2 = a.nb[2];
    if (verdict != 0) {
      uint32_t val = verdict == 1 ? 0xffffffffu : 0xfffffffeu;
      for (long long z = max(b.z, 0LL); z < min(b.z + a.size, nb2); z++)
        for (long long y = max(b.y, 0LL); y < min(b.y + a.size, nb1); y++)
          for (long long x = max(b.x, 0LL); x < min(b.x + a.size, nb0); x++) a.map[x + nb0 * (y + nb1 * z)] = val;
    } else if (a.size == 1) {
      long long idx = b.x + nb0 * (b.y + nb1 * b.z);
      a.map[idx] = 0xfffffff0u;  // read
      unsigned long long slot = atomicAdd((unsigned long long*)a.n_read, 1ull);
      if (slot < (unsigned long long)a.read_cap) {
        a.read_idx[slot] = idx;
        a.read_dc[slot] = sd;
      }
    } else {
      long long half = a.size / 2;
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
        unsigned long long slot = atomicAdd((unsigned long long*)a.n_next, 1ull);
        if (slot < (unsigned long long)a.next_cap) a.next[slot] = k;
      }
    }
  }
}

// The read bricks' first nodes and centre distances, in brick order.
__global__ void k_gather_firsts(const int64_t* idx, int64_t n, int64_t nb0, int64_t nb1, double h, double lo0,
                                double lo1, double lo2, double* firsts) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t b = idx[i];
    int64_t x = b % nb0, y = (b / nb0) % nb1, z = b / (nb0 * nb1);
    double side = 8.0 * h;
    firsts[3 * i] = lo0 + side * x;
    firsts[3 * i + 1] = lo1 + side * y;
    firsts[3 * i + 2] = lo2 + side * z;
  }
}

// Map entries of the read bricks, and each stored brick's words moved to its slot.
__global__ void k_assemble(const int64_t* idx, const int32_t* kind, const int64_t* slot, int64_t n,
                           const uint32_t* words, uint32_t* map, uint32_t* atlas) {
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    int k = kind[i];
    if (threadIdx.x == 0) map[idx[i]] = k == 1 ? 0xffffffffu : (k == 2 ? 0xfffffffeu : uint32_t(slot[i]));
    if (k == 0 && atlas)
      for (int w = threadIdx.x; w < 365; w += blockDim.x) atlas[slot[i] * 365 + w] = words[i * 365 + w];
  }
}

__global__ void k_is_words(const int32_t* kind, int64_t n, int64_t* flag) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    flag[i] = kind[i] == 0 ? 1 : 0;
}

// Independent FMA chains, eight a thread, for the throughput probe.
template <class T>
__global__ void k_fma(T* out, int iters) {
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = T(threadIdx.x + k);
  const T m = T(0.999999), c = T(1e-7);
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = a[k] * m + c;
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == T(-1)) out[0] = s;
}
template __global__ void k_fma<double>(double*, int);
template __global__ void k_fma<float>(float*, int);

__global__ void k_warm(float* out, int iters) {
  float x = float(threadIdx.x);
  for (int i = 0; i < iters; i++) x = fmaf(x, 1.0000001f, 0.5f);
  if (x == 0.0f) out[0] = x;
}

}  // namespace icam

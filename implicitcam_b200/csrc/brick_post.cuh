// The end of a brick read, shared by the brick kernels (bricks.cu, bricks_mixed.cu): a
// brick's node values (exact ones, NaN for the rest) become its packed words and its
// kind (partcache.rs:790-970), and its census is counted.
#pragma once

#include "warp_list.cuh"

namespace icam {

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

__device__ __forceinline__ uint32_t spread(uint32_t m) { return m | (m << 1) | (m >> 1); }

// Row masks grown by one node in every direction (the 26-neighbourhood and the node):
// rows r of this lane, up to three.
__device__ __forceinline__ uint32_t dilate_row(const uint32_t* m, int r) {
  int j = r % 9, k = r / 9;
  uint32_t d = 0;
#pragma unroll
  for (int dk = -1; dk <= 1; dk++) {
    int kk = k + dk;
    if (kk < 0 || kk > 8) continue;
#pragma unroll
    for (int dj = -1; dj <= 1; dj++) {
      int jj = j + dj;
      if (jj < 0 || jj > 8) continue;
      d |= spread(m[jj + 9 * kk]);
    }
  }
  return d & 0x1ffu;
}

// Node masks by row (row j + 9 k, bit i of node i + 9 j + 81 k).
struct RowMasks {
  uint32_t m0[81], m1[81], m2[81];
};

// Far nodes signed by a signed neighbour, until nothing changes (partcache.rs:845-858):
// m0 / m1 the nodes of positive / negative value, m2 the far nodes not yet signed. A
// far node lies farther than the clamp from the surface, so its neighbours within a
// cell diagonal all share its sign when the clamp is at least that diagonal; a node
// offered both signs takes the positive one.
__device__ __forceinline__ void flood(RowMasks& M, int lane) {
  for (;;) {
    uint32_t np[3], nq[3];
    bool any = false;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      int r = lane + 32 * q;
      np[q] = nq[q] = 0;
      if (r < 81) {
        uint32_t o = M.m2[r];
        if (o) {
          np[q] = dilate_row(M.m0, r) & o;
          nq[q] = dilate_row(M.m1, r) & o & ~np[q];
          any |= (np[q] | nq[q]) != 0;
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 3; q++) {
      int r = lane + 32 * q;
      if (r < 81 && (np[q] | nq[q])) {
        M.m0[r] |= np[q];
        M.m1[r] |= nq[q];
        M.m2[r] &= ~(np[q] | nq[q]);
      }
    }
    __syncwarp();
    if (!__any_sync(FULL, any)) break;
  }
}

// The brick's words and kind from its node values f (T: double, or float in the mixed
// kernel; exact values, NaN where not known) and flags (1 far): far nodes signed by a
// neighbour, by the centre's empty ball (radius 0.999 max(clamp, |dc| - dc_err): dc is
// the centre's distance within dc_err), bridged, quantised and packed. words (365) and
// kind (0 words, 1 air, 2 solid) are written when given. Returns this lane's count of
// bridged nodes.
template <class T>
__device__ int brick_post(T* f, const int8_t* flag, RowMasks& M, double3 first, double h, double clamp, double dc,
                          double dc_err, int n_far, uint32_t* words, int32_t* kind, int lane) {
  int provisional = 0;
  const double3 c = first + mk(4.0 * h, 4.0 * h, 4.0 * h);
  const bool dc_signed = isfinite(dc) && fabs(dc) > dc_err;
  // every node far with the centre's sign known: the last rule decides them all
  // (partcache.rs:876-892), whatever the fill and the ball would have given
  const bool all_far = n_far == 729 && dc_signed && dc != 0.0;
  if (all_far) {
    for (int nn = lane; nn < 729; nn += 32) f[nn] = T(copysign(clamp, dc));
  } else {
    // ---- far nodes signed by a neighbour within a cell diagonal (partcache.rs:845-858)
    for (int r = lane; r < 81; r += 32) {
      uint32_t pm = 0, qm = 0, om = 0;
      for (int i = 0; i < 9; i++) {
        T v = f[9 * r + i];
        if (v > T(0))
          pm |= 1u << i;
        else if (v < T(0))
          qm |= 1u << i;
        else if (isnan(v) && flag[9 * r + i] == 1)
          om |= 1u << i;
      }
      M.m0[r] = pm, M.m1[r] = qm, M.m2[r] = om;
    }
    __syncwarp();
    flood(M, lane);
    // ---- far nodes in the centre's empty ball, or the centre in theirs (partcache.rs:860-875)
    if (dc_signed && dc != 0.0) {
      double rch = 0.999 * fmax(clamp, fabs(dc) - dc_err);
      for (int r = lane; r < 81; r += 32) {
        uint32_t om = M.m2[r], hit = 0;
        for (int i = 0; i < 9; i++) {
          if (!((om >> i) & 1u)) continue;
          int nn = 9 * r + i;
          double3 x = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
          if (len(x - c) < rch) hit |= 1u << i;
        }
        if (hit) {
          M.m2[r] = om & ~hit;
          if (dc > 0)
            M.m0[r] |= hit;
          else
            M.m1[r] |= hit;
        }
      }
      __syncwarp();
      flood(M, lane);
    }
    for (int r = lane; r < 81; r += 32) {
      uint32_t pm = M.m0[r], qm = M.m1[r];
      for (int i = 0; i < 9; i++) {
        int nn = 9 * r + i;
        if (!isnan(f[nn])) continue;
        if ((pm >> i) & 1u)
          f[nn] = T(clamp);
        else if ((qm >> i) & 1u)
          f[nn] = T(-clamp);
      }
    }
  }
  __syncwarp();
  // ---- bridging: the mean of the known neighbours, held in the brackets the exact
  // ones give (partcache.rs:893-916), pass after pass; m0 the nodes known when the
  // pass began, m1 the nodes it sets
  for (int r = lane; r < 81; r += 32) {
    uint32_t km = 0;
    for (int i = 0; i < 9; i++)
      if (!isnan(f[9 * r + i])) km |= 1u << i;
    M.m0[r] = km;
  }
  __syncwarp();
  for (int pass = 0; pass < 729; pass++) {
    bool any = false;
    for (int r = lane; r < 81; r += 32) {
      uint32_t sm = dilate_row(M.m0, r) & ~M.m0[r] & 0x1ffu;
      M.m1[r] = sm;
      any |= sm != 0;
    }
    if (!__any_sync(FULL, any)) break;
    __syncwarp();
    for (int nn = lane; nn < 729; nn += 32) {
      if (!((M.m1[nn / 9] >> (nn % 9)) & 1u)) continue;
      double sum = 0.0, lo = -clamp, hi = clamp;
      int cn = 0;
      for (int k = 0; k < 26; k++) {
        double dd;
        int m = nb_of(nn, k, &dd);
        if (m < 0) continue;
        if ((M.m0[m / 9] >> (m % 9)) & 1u) {
          sum += double(f[m]);
          cn++;
          if (flag[m] == 0) {
            lo = fmax(lo, double(f[m]) - dd * h);
            hi = fmin(hi, double(f[m]) + dd * h);
          }
        }
      }
      double vm = sum / cn;
      f[nn] = T(lo <= hi ? fmin(fmax(vm, lo), hi) : 0.5 * (lo + hi));
      provisional++;
    }
    __syncwarp();
    for (int r = lane; r < 81; r += 32) M.m0[r] |= M.m1[r];
    __syncwarp();
  }
  // nothing around them known: the brick's far side, taken as air
  for (int nn = lane; nn < 729; nn += 32)
    if (isnan(f[nn])) {
      f[nn] = T(clamp);
      provisional++;
    }
  __syncwarp();
  // ---- quantise and pack: a lane eight nodes, four words stored at once (words is
  // 16-byte aligned, WORD_STRIDE words a brick; the three past the 365th are zero)
  bool pos = true, nonpos = true;
  for (int w4 = lane; w4 < 92; w4 += 32) {
    uint32_t word[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int w = 4 * w4 + e;
      word[e] = 0u;
      if (w >= 365) continue;
      double q0 = round(fmin(fmax(double(f[2 * w]) / clamp, -1.0), 1.0) * 32767.0);
      pos = pos && q0 > 0;
      nonpos = nonpos && q0 <= 0;
      word[e] = uint32_t(uint16_t(int16_t(q0)));
      if (2 * w + 1 < 729) {
        double q1 = round(fmin(fmax(double(f[2 * w + 1]) / clamp, -1.0), 1.0) * 32767.0);
        pos = pos && q1 > 0;
        nonpos = nonpos && q1 <= 0;
        word[e] |= uint32_t(uint16_t(int16_t(q1))) << 16;
      }
    }
    if (words) reinterpret_cast<uint4*>(words)[w4] = make_uint4(word[0], word[1], word[2], word[3]);
  }
  const bool all_pos = __all_sync(FULL, pos), all_nonpos = __all_sync(FULL, nonpos);
  if (kind && lane == 0) *kind = all_pos ? 1 : (all_nonpos ? 2 : 0);
  return provisional;
}

// The census of a brick's list by kind (B-spline sub-patches counted by their distinct
// spans) and the brick's counts, added to the kernel's counters (BrickArgs::stats).
__device__ __forceinline__ void brick_census(const DPack& P, const uint32_t* code, int n, bool overflow, int n_exact,
                                             int n_far, int n_und, int provisional, unsigned long long* stats,
                                             int lane) {
  provisional = __reduce_add_sync(FULL, provisional);
  unsigned kinds[5] = {0, 0, 0, 0, 0};
  for (int k = lane; k < n; k += 32) {
    uint32_t kd = code[k] >> IK_SHIFT;
    if (kd == IK_SUB) {
      const DSub& s = P.subs[code[k] & IK_MASK];
      bool seen = false;
      for (int j = 0; j < k && !seen; j++)
        if ((code[j] >> IK_SHIFT) == IK_SUB) {
          const DSub& o = P.subs[code[j] & IK_MASK];
          seen = o.nurbs == s.nurbs && o.span_a == s.span_a && o.span_b == s.span_b;
        }
      if (!seen) kinds[1]++;
    } else {
      kinds[kd == IK_FACE ? 0 : kd == IK_EDGE ? 2 : kd == IK_PIECE ? 3 : 4]++;
    }
  }
  for (int k = 0; k < 5; k++) kinds[k] = __reduce_add_sync(FULL, kinds[k]);
  if (lane == 0) {
    atomicAdd(&stats[0], (unsigned long long)n_exact);
    atomicAdd(&stats[1], (unsigned long long)n_far);
    atomicAdd(&stats[2], (unsigned long long)n_und);
    if (provisional) atomicAdd(&stats[3], (unsigned long long)provisional);
    atomicAdd(&stats[4], (unsigned long long)n);
    for (int k = 0; k < 5; k++)
      if (kinds[k]) atomicAdd(&stats[6 + k], (unsigned long long)kinds[k]);
    if (overflow) atomicAdd(&stats[5], 1ull);
  }
}

}  // namespace icam

// Kernels of the exact part field on sm_100a besides the brick kernel (bricks.cu): point
// queries through the feature tree, the box decision of a level (partcache.rs:226-331),
// the gather of the read bricks and the assembly of the map and the atlas.
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

void launch_fma(bool fp64, void* out, int blocks, int threads, int iters, cudaStream_t s) {
  if (fp64)
    k_fma<double><<<blocks, threads, 0, s>>>(static_cast<double*>(out), iters);
  else
    k_fma<float><<<blocks, threads, 0, s>>>(static_cast<float*>(out), iters);
}

__global__ void k_warm(float* out, int iters) {
  float x = float(threadIdx.x);
  for (int i = 0; i < iters; i++) x = fmaf(x, 1.0000001f, 0.5f);
  if (x == 0.0f) out[0] = x;
}

}  // namespace icam

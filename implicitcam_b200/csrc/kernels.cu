// Kernels of the exact part field on sm_100a besides the brick kernel (bricks.cu) and the
// box decision (decide.cu): point queries through the feature tree, the gather of the
// read bricks and the assembly of the map and the atlas.
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
      for (int w = threadIdx.x; w < 365; w += blockDim.x) atlas[slot[i] * 365 + w] = words[i * WORD_STRIDE + w];
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

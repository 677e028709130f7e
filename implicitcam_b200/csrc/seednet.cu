// The seed network (seednet.cuh) on the device: its per sub-patch features, training
// pairs made by the exact FP64 evaluator, the training step (hand-written forward and
// backward passes in FP32, Adam), the A/B check of its seeds against the sub-patch-centre
// start, and the C entry points of include/icam_cuda.h for all of it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/icam_cuda.h"
#include "pack_state.h"
#include "seednet.cuh"

using namespace icam;

namespace icam {

// ---------------------------------------------------------------- features and pairs

__device__ __forceinline__ uint64_t sn_mix(uint64_t z) {  // splitmix64
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double sn_unif(uint64_t& st) {
  st = sn_mix(st);
  return double(st >> 11) * (1.0 / 9007199254740992.0);
}

// Each sub-patch's frame at its centre (S(0.5, 0.5); S_s; the normal), 1 / L with L its
// diagonal, and its descriptor: the four corners in that frame over L (12), |S_s| / L,
// |S_t| / L, the cosine between them, and the normal curvature along S_s times L.
__global__ void k_sn_feat(DPack P, float* feat) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_subs; i += gridDim.x * blockDim.x) {
    const double4* cp = P.sub_cp + 16 * size_t(i);
    SE e = eval_bicubic(cp, 0.5, 0.5);
    double L = fmax(P.subs[i].diag, 1e-12);
    double3 e1 = unit(e.ps), e3 = unit(cross(e.ps, e.pt)), e2 = cross(e3, e1);
    float* F = feat + size_t(i) * SN_FEAT;
    F[0] = float(e.p.x), F[1] = float(e.p.y), F[2] = float(e.p.z);
    F[3] = float(e1.x), F[4] = float(e1.y), F[5] = float(e1.z);
    F[6] = float(e2.x), F[7] = float(e2.y), F[8] = float(e2.z);
    F[9] = float(e3.x), F[10] = float(e3.y), F[11] = float(e3.z);
    F[12] = float(1.0 / L), F[13] = F[14] = F[15] = 0.f;
    const double cs[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
    for (int q = 0; q < 4; q++) {
      double3 d = eval_bicubic(cp, cs[q][0], cs[q][1]).p - e.p;
      F[16 + 3 * q] = float(dot(d, e1) / L);
      F[17 + 3 * q] = float(dot(d, e2) / L);
      F[18 + 3 * q] = float(dot(d, e3) / L);
    }
    double ls = len(e.ps), lt = len(e.pt);
    F[28] = float(ls / L);
    F[29] = float(lt / L);
    F[30] = float(dot(e.ps, e.pt) / fmax(ls * lt, 1e-300));
    F[31] = float(dot(e.pss, e3) / fmax(ls * ls, 1e-300) * L);
  }
}

// The nearest point of sub-patch `si` to p by the exact evaluator: projected Newton from
// `s0, t0` and from the centre, the nearer converged answer (the nearer of both if
// neither converged). Iterations spent in *used.
__device__ void sn_exact(const DPack& P, int si, double3 p, double s0, double t0, double* s, double* t, double* d) {
  const double4* cp = P.sub_cp + 16 * size_t(si);
  double bs = 0.5, bt = 0.5, bd = INFINITY;
  bool bc = false;
  const double starts[2][2] = {{s0, t0}, {0.5, 0.5}};
  for (int q = 0; q < 2; q++) {
    double ss = starts[q][0], tt = starts[q][1];
    bool conv;
    newton_bicubic(cp, p, &ss, &tt, 24, &conv);
    double dd = len(eval_bicubic(cp, ss, tt).p - p);
    if ((conv && !bc) || (conv == bc && dd < bd)) bs = ss, bt = tt, bd = dd, bc = conv;
  }
  *s = bs, *t = bt, *d = bd;
}

// One query for sub-patch si from stream st: a point of the sub-patch moved along its
// normal by up to `need` (denser near the surface), and half the time across it by up
// to half its size, so that some feet lie on its border.
__device__ double3 sn_query(const DPack& P, const float* feat, uint64_t& st, double need, int* si, double* s0,
                            double* t0) {
  int i = int(sn_unif(st) * P.n_subs);
  i = min(i, P.n_subs - 1);
  const double4* cp = P.sub_cp + 16 * size_t(i);
  double u = sn_unif(st), v = sn_unif(st);
  SE e = eval_bicubic(cp, u, v);
  double3 n = unit(cross(e.ps, e.pt));
  double r = 2.0 * sn_unif(st) - 1.0;
  double3 p = e.p + n * (need * r * fabs(r));
  if (sn_unif(st) < 0.5) {
    const float* F = feat + size_t(i) * SN_FEAT;
    double L = 1.0 / double(F[12]);
    double a = (sn_unif(st) - 0.5) * L, b = (sn_unif(st) - 0.5) * L;
    p = p + mk(F[3], F[4], F[5]) * a + mk(F[6], F[7], F[8]) * b;
  }
  *si = i, *s0 = u, *t0 = v;
  return p;
}

// n training pairs: inputs (SN_INP a pair, zero padded) and targets (s, t, d / L, 1).
// The stream of pair k is seed, *step (when given), k.
__global__ void k_sn_data(DPack P, const float* feat, int64_t n, uint64_t seed, const unsigned long long* step,
                          double need, float* x, float* y) {
  const uint64_t base = sn_mix(seed ^ (step ? sn_mix(*step + 1) : 0ull));
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x) {
    uint64_t st = base ^ sn_mix(uint64_t(k) * 0x9e3779b97f4a7c15ull);
    int si;
    double s0, t0;
    double3 p = sn_query(P, feat, st, need, &si, &s0, &t0);
    double s, t, d;
    sn_exact(P, si, p, s0, t0, &s, &t, &d);
    const float* F = feat + size_t(si) * SN_FEAT;
    float in[SN_IN];
    sn_input(F, p, in);
    for (int j = 0; j < SN_INP; j++) x[k * SN_INP + j] = j < SN_IN ? in[j] : 0.f;
    y[k * 4] = float(s), y[k * 4 + 1] = float(t), y[k * 4 + 2] = float(d * double(F[12])), y[k * 4 + 3] = 1.f;
  }
}

// ---------------------------------------------------------------- training

constexpr int SN_ROWS = 64;  // samples a block of the training step

// Loss per sample: (s - s*)^2 + (t - t*)^2 + 0.1 (d - d*)^2, averaged over the batch of
// n. Forward pass, backward pass, gradients added into grads and the loss into *loss,
// 64 samples a block of 256 threads, activations in shared memory.
__global__ void __launch_bounds__(256) k_sn_grad(const float* __restrict__ W, const float* __restrict__ x,
                                                 const float* __restrict__ y, int64_t n, float* grads, float* loss,
                                                 const unsigned long long* step) {
  extern __shared__ float sm[];
  float* X = sm;                              // 64 x 32
  float* H1 = X + SN_ROWS * SN_INP;           // 64 x 64
  float* H2 = H1 + SN_ROWS * SN_H;            // 64 x 64
  float* H3 = H2 + SN_ROWS * SN_H;            // 64 x 64
  float* O = H3 + SN_ROWS * SN_H;             // 64 x 8
  float* red = O + SN_ROWS * SN_OUTP;         // 256
  const int tid = threadIdx.x;
  const int64_t r0 = int64_t(blockIdx.x) * SN_ROWS;
  const int rows = int(n - r0 < SN_ROWS ? n - r0 : SN_ROWS);
  const float inv_n = 1.f / float(n);
  for (int e = tid; e < SN_ROWS * SN_INP; e += 256) X[e] = (e / SN_INP) < rows ? x[r0 * SN_INP + e] : 0.f;
  __syncthreads();
  auto dense = [&](const float* in, int K, const float* w, const float* b, int N, float* out, bool relu) {
    for (int e = tid; e < SN_ROWS * N; e += 256) {
      int s = e / N, j = e % N;
      float a = b[j];
      for (int k = 0; k < K; k++) a = fmaf(in[s * K + k], w[k * N + j], a);
      out[e] = relu ? fmaxf(a, 0.f) : a;
    }
    __syncthreads();
  };
  dense(X, SN_INP, W + SN_W1, W + SN_B1, SN_H, H1, true);
  dense(H1, SN_H, W + SN_W2, W + SN_B2, SN_H, H2, true);
  dense(H2, SN_H, W + SN_W3, W + SN_B3, SN_H, H3, true);
  dense(H3, SN_H, W + SN_W4, W + SN_B4, SN_OUTP, O, false);
  // output deltas (in place of the outputs) and the loss
  float l = 0.f;
  for (int e = tid; e < SN_ROWS * SN_OUTP; e += 256) {
    int s = e / SN_OUTP, j = e % SN_OUTP;
    float d = 0.f;
    if (s < rows && j < SN_OUT) {
      float wgt = j == 2 ? 0.1f : 1.f;
      float diff = O[e] - y[(r0 + s) * 4 + j];
      l += wgt * diff * diff;
      d = 2.f * wgt * diff * inv_n;
    }
    O[e] = d;
  }
  red[tid] = l;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (tid < o) red[tid] += red[tid + o];
    __syncthreads();
  }
  if (tid == 0) atomicAdd(loss + (step ? *step : 0ull), red[0] * inv_n);
  // a layer's weight and bias gradients from its input and output deltas, then the
  // deltas of its input (through the ReLU) in place of the input
  auto back = [&](float* in, int K, const float* w, int wo, int bo, const float* dout, int N, bool prop) {
    for (int e = tid; e < K * N; e += 256) {
      int k = e / N, j = e % N;
      float a = 0.f;
      for (int s = 0; s < SN_ROWS; s++) a = fmaf(in[s * K + k], dout[s * N + j], a);
      if (a != 0.f) atomicAdd(grads + wo + e, a);
    }
    for (int j = tid; j < N; j += 256) {
      float a = 0.f;
      for (int s = 0; s < SN_ROWS; s++) a += dout[s * N + j];
      if (a != 0.f) atomicAdd(grads + bo + j, a);
    }
    __syncthreads();
    if (!prop) return;
    for (int e = tid; e < SN_ROWS * K; e += 256) {
      int s = e / K, k = e % K;
      float a = 0.f;
      if (in[e] > 0.f)
        for (int j = 0; j < N; j++) a = fmaf(dout[s * N + j], w[k * N + j], a);
      in[e] = a;
    }
    __syncthreads();
  };
  back(H3, SN_H, W + SN_W4, SN_W4, SN_B4, O, SN_OUTP, true);
  back(H2, SN_H, W + SN_W3, SN_W3, SN_B3, H3, SN_H, true);
  back(H1, SN_H, W + SN_W2, SN_W2, SN_B2, H2, SN_H, true);
  back(X, SN_INP, W + SN_W1, SN_W1, SN_B1, H1, SN_H, false);
}

// Adam on every parameter; the step count from *step, then advanced. One block, so that
// every thread has read the step before it moves.
__global__ void k_sn_adam(float* W, const float* g, float* m, float* v, int n, float lr, unsigned long long* step) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float t = float(*step + 1);
  const float c1 = 1.f - powf(b1, t), c2 = 1.f - powf(b2, t);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi, v[i] = vi;
    W[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
  __syncthreads();
  if (threadIdx.x == 0) *step += 1;
}

// The BF16 transposed copy the kernels read (seednet.cuh), and the FP32 biases after it.
__global__ void k_sn_pack(const float* W, void* wbf) {
  __nv_bfloat16* T = static_cast<__nv_bfloat16*>(wbf);
  float* B = reinterpret_cast<float*>(T + SN_TBF);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < SN_TBF + SN_NBIAS; e += gridDim.x * blockDim.x) {
    if (e >= SN_TBF) {
      int b = e - SN_TBF;
      B[b] = b < SN_H ? W[SN_B1 + b] : b < 2 * SN_H ? W[SN_B2 + b - SN_H] : b < 3 * SN_H ? W[SN_B3 + b - 2 * SN_H]
                                                                                       : W[SN_B4 + b - 3 * SN_H];
      continue;
    }
    float val = 0.f;
    if (e < SN_T2) {
      int j = e / SN_KS1, k = e % SN_KS1;
      if (k < SN_INP) val = W[SN_W1 + k * SN_H + j];
    } else if (e < SN_T3) {
      int j = (e - SN_T2) / SN_KS, k = (e - SN_T2) % SN_KS;
      if (k < SN_H) val = W[SN_W2 + k * SN_H + j];
    } else if (e < SN_T4) {
      int j = (e - SN_T3) / SN_KS, k = (e - SN_T3) % SN_KS;
      if (k < SN_H) val = W[SN_W3 + k * SN_H + j];
    } else {
      int j = (e - SN_T4) / SN_KS, k = (e - SN_T4) % SN_KS;
      if (k < SN_H) val = W[SN_W4 + k * SN_OUTP + j];
    }
    T[e] = __float2bfloat16_rn(val);
  }
}

// ---------------------------------------------------------------- the A/B check

constexpr int SN_ITMAX = 24;
// stats: [0] pairs, [1] Newton iterations from the net's seeds, [2] from the centre,
// [3] fallbacks (the net's start failed its checks), [4] pairs whose answers differ by
// more than 1e-9 L, [5..5+SN_ITMAX] iteration histogram from the net's seeds,
// [6+SN_ITMAX..] from the centre; maxdiff: the largest |d_net - d_centre| / L (bits).
__global__ void k_sn_ab(DPack P, const float* feat, const void* wbf, int64_t n, uint64_t seed, double need,
                        unsigned long long* stats, unsigned long long* maxdiff) {
  __shared__ __align__(16) __nv_bfloat16 act[4][32 * SN_KS];
  __shared__ float out[4][32 * 8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t base = sn_mix(seed);
  for (int64_t g0 = (int64_t(blockIdx.x) * 4 + warp) * 32; g0 < n; g0 += int64_t(gridDim.x) * 4 * 32) {
    const int64_t k = g0 + lane;
    const bool live = k < n;
    uint64_t st = base ^ sn_mix(uint64_t(live ? k : g0) * 0x9e3779b97f4a7c15ull);
    int si;
    double s0, t0;
    double3 p = sn_query(P, feat, st, need, &si, &s0, &t0);
    const float* F = feat + size_t(si) * SN_FEAT;
    float in[SN_IN], o[3];
    sn_input(F, p, in);
    sn_forward_warp(wbf, act[warp], out[warp], in, o, lane);
    if (!live) continue;
    const double4* cp = P.sub_cp + 16 * size_t(si);
    auto solve = [&](double s, double t, int* used, bool* conv, double* ds, double* dt) {
      int it = 0;
      *conv = false;
      while (it < SN_ITMAX && !*conv) {
        newton_bicubic(cp, p, &s, &t, 1, conv);
        it++;
      }
      *used = it, *ds = s, *dt = t;
    };
    // the net's seed, checked: converged, and a critical point or a held border point
    int it_n, it_c;
    bool cn, cc;
    double sn, tn, sc, tc;
    solve(fmin(fmax(double(o[0]), 0.0), 1.0), fmin(fmax(double(o[1]), 0.0), 1.0), &it_n, &cn, &sn, &tn);
    SE en = eval_bicubic(cp, sn, tn);
    bool ok = cn && (is_critical(p, en) || sn <= 0.0 || sn >= 1.0 || tn <= 0.0 || tn >= 1.0);
    solve(0.5, 0.5, &it_c, &cc, &sc, &tc);
    double dcen = len(eval_bicubic(cp, sc, tc).p - p);
    double dnet = len(en.p - p);
    if (!ok) {  // multi-start fallback: the centre's answer stands
      atomicAdd(&stats[3], 1ull);
      dnet = dcen;
    }
    double L = 1.0 / double(F[12]);
    double diff = fabs(dnet - dcen) / L;
    atomicAdd(&stats[0], 1ull);
    atomicAdd(&stats[1], (unsigned long long)it_n);
    atomicAdd(&stats[2], (unsigned long long)it_c);
    if (diff > 1e-9) atomicAdd(&stats[4], 1ull);
    atomicAdd(&stats[5 + min(it_n, SN_ITMAX)], 1ull);
    atomicAdd(&stats[6 + SN_ITMAX + min(it_c, SN_ITMAX)], 1ull);
    atomicMax(maxdiff, (unsigned long long)__double_as_longlong(diff));
  }
}

}  // namespace icam

// ---------------------------------------------------------------- C entry points

namespace {

int sn_fail(IcamPack* pk, int code, const std::string& msg) {
  if (pk) pk->err = msg;
  return code;
}

#define SNCK(call)                                                                                \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return sn_fail(pk, ICAM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int sn_alloc(IcamPack* pk, size_t bytes, void** out) {
  SNCK(cudaMalloc(out, bytes));
  pk->owned.push_back(*out);
  return ICAM_OK;
}

// Features, weights and moments allocated and the features computed, once a pack.
int sn_setup(IcamPack* pk) {
  SeedNetState& N = pk->net;
  if (N.params) return ICAM_OK;
  if (pk->dev.n_subs == 0) return sn_fail(pk, ICAM_ERR_ARG, "the solid has no B-spline sub-patches to seed");
  void* p;
  int r;
  if ((r = sn_alloc(pk, size_t(pk->dev.n_subs) * SN_FEAT * sizeof(float), &p))) return r;
  N.feat = static_cast<float*>(p);
  if ((r = sn_alloc(pk, 4 * SN_PARAMS * sizeof(float), &p))) return r;
  N.params = static_cast<float*>(p);
  N.grads = N.params + SN_PARAMS;
  N.adam_m = N.grads + SN_PARAMS;
  N.adam_v = N.adam_m + SN_PARAMS;
  if ((r = sn_alloc(pk, SN_WBYTES, &N.wbf))) return r;
  if ((r = sn_alloc(pk, sizeof(unsigned long long), &p))) return r;
  N.step = static_cast<unsigned long long*>(p);
  k_sn_feat<<<std::max(1, std::min(1184, (pk->dev.n_subs + 127) / 128)), 128, 0, pk->stream>>>(pk->dev, N.feat);
  SNCK(cudaGetLastError());
  // He-uniform initial weights (a fixed stream), zero biases, zero moments
  std::vector<float> w(SN_PARAMS, 0.f);
  uint64_t s = 0x5eed5eedull;
  auto unif = [&]() {
    s += 0x9e3779b97f4a7c15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return double(z >> 11) / 9007199254740992.0;
  };
  auto fill = [&](int off, int K, int N_, int kin) {
    double a = std::sqrt(6.0 / kin);
    for (int k = 0; k < K; k++)
      for (int j = 0; j < N_; j++) w[off + k * N_ + j] = k < kin ? float((2 * unif() - 1) * a) : 0.f;
  };
  fill(SN_W1, SN_INP, SN_H, SN_IN);
  fill(SN_W2, SN_H, SN_H, SN_H);
  fill(SN_W3, SN_H, SN_H, SN_H);
  fill(SN_W4, SN_H, SN_OUTP, SN_H);
  for (int k = 0; k < SN_H; k++)
    for (int j = SN_OUT; j < SN_OUTP; j++) w[SN_W4 + k * SN_OUTP + j] = 0.f;
  SNCK(cudaMemcpyAsync(N.params, w.data(), SN_PARAMS * sizeof(float), cudaMemcpyHostToDevice, pk->stream));
  SNCK(cudaMemsetAsync(N.adam_m, 0, 2 * SN_PARAMS * sizeof(float), pk->stream));
  SNCK(cudaMemsetAsync(N.step, 0, sizeof(unsigned long long), pk->stream));
  return ICAM_OK;
}

int sn_batch(IcamPack* pk, int64_t batch) {
  SeedNetState& N = pk->net;
  if (N.batch_cap >= batch) return ICAM_OK;
  void* p;
  int r;
  if ((r = sn_alloc(pk, size_t(batch) * (SN_INP + 4) * sizeof(float), &p))) return r;
  N.x = static_cast<float*>(p);
  N.y = N.x + size_t(batch) * SN_INP;
  N.batch_cap = batch;
  return ICAM_OK;
}

int sn_pack(IcamPack* pk) {
  k_sn_pack<<<64, 256, 0, pk->stream>>>(pk->net.params, pk->net.wbf);
  SNCK(cudaGetLastError());
  pk->net.ready = true;
  return ICAM_OK;
}

size_t sn_grad_smem() { return size_t(SN_ROWS) * (SN_INP + 3 * SN_H + SN_OUTP) * sizeof(float) + 256 * sizeof(float); }

}  // namespace

extern "C" {

int icam_seednet_samples(IcamPack* pk, size_t n, uint64_t seed, double need, float* x_out, float* y_out) {
  if (!pk || (n && (!x_out || !y_out))) return sn_fail(pk, ICAM_ERR_ARG, "null argument");
  if (!(need > 0)) return sn_fail(pk, ICAM_ERR_ARG, "need must be positive");
  if (n == 0) return ICAM_OK;
  SNCK(cudaSetDevice(pk->device));
  int r;
  if ((r = sn_setup(pk)) || (r = sn_batch(pk, int64_t(n)))) return r;
  k_sn_data<<<int(std::min<int64_t>(1184, (int64_t(n) + 127) / 128)), 128, 0, pk->stream>>>(
      pk->dev, pk->net.feat, int64_t(n), seed, nullptr, need, pk->net.x, pk->net.y);
  SNCK(cudaGetLastError());
  SNCK(cudaMemcpyAsync(x_out, pk->net.x, n * SN_INP * sizeof(float), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaMemcpyAsync(y_out, pk->net.y, n * 4 * sizeof(float), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

int icam_seednet_params(IcamPack* pk, float* get, const float* set, size_t* n_params) {
  if (!pk) return sn_fail(pk, ICAM_ERR_ARG, "null argument");
  if (n_params) *n_params = SN_PARAMS;
  if (!get && !set) return ICAM_OK;
  SNCK(cudaSetDevice(pk->device));
  int r;
  if ((r = sn_setup(pk))) return r;
  if (set) {
    SNCK(cudaMemcpyAsync(pk->net.params, set, SN_PARAMS * sizeof(float), cudaMemcpyHostToDevice, pk->stream));
    if ((r = sn_pack(pk))) return r;
  }
  if (get) SNCK(cudaMemcpyAsync(get, pk->net.params, SN_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

int icam_seednet_grad(IcamPack* pk, const float* x, const float* y, size_t n, float* grad_out, double* loss_out) {
  if (!pk || !x || !y || !grad_out || !loss_out || n == 0) return sn_fail(pk, ICAM_ERR_ARG, "null argument");
  SNCK(cudaSetDevice(pk->device));
  int r;
  if ((r = sn_setup(pk)) || (r = sn_batch(pk, int64_t(n)))) return r;
  SeedNetState& N = pk->net;
  void* lp;
  if ((r = sn_alloc(pk, sizeof(float), &lp))) return r;
  SNCK(cudaMemcpyAsync(N.x, x, n * SN_INP * sizeof(float), cudaMemcpyHostToDevice, pk->stream));
  SNCK(cudaMemcpyAsync(N.y, y, n * 4 * sizeof(float), cudaMemcpyHostToDevice, pk->stream));
  SNCK(cudaMemsetAsync(N.grads, 0, SN_PARAMS * sizeof(float), pk->stream));
  SNCK(cudaMemsetAsync(lp, 0, sizeof(float), pk->stream));
  SNCK(cudaFuncSetAttribute(k_sn_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sn_grad_smem())));
  k_sn_grad<<<int((n + SN_ROWS - 1) / SN_ROWS), 256, sn_grad_smem(), pk->stream>>>(N.params, N.x, N.y, int64_t(n),
                                                                                   N.grads, (float*)lp, nullptr);
  SNCK(cudaGetLastError());
  float l = 0.f;
  SNCK(cudaMemcpyAsync(grad_out, N.grads, SN_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaMemcpyAsync(&l, lp, sizeof(float), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaStreamSynchronize(pk->stream));
  *loss_out = l;
  return ICAM_OK;
}

int icam_seednet_train(IcamPack* pk, int64_t steps, int64_t batch, uint64_t seed, double need, double lr,
                       float* loss_out) {
  if (!pk || steps < 0 || batch <= 0) return sn_fail(pk, ICAM_ERR_ARG, "bad argument");
  if (!(need > 0) || !(lr > 0)) return sn_fail(pk, ICAM_ERR_ARG, "need and lr must be positive");
  SNCK(cudaSetDevice(pk->device));
  int r;
  if ((r = sn_setup(pk)) || (r = sn_batch(pk, batch))) return r;
  SeedNetState& N = pk->net;
  if (N.loss_cap < steps) {
    void* p;
    if ((r = sn_alloc(pk, size_t(std::max<int64_t>(steps, 1)) * sizeof(float), &p))) return r;
    N.loss = static_cast<float*>(p);
    N.loss_cap = steps;
  }
  SNCK(cudaMemsetAsync(N.loss, 0, size_t(std::max<int64_t>(steps, 1)) * sizeof(float), pk->stream));
  SNCK(cudaMemsetAsync(N.step, 0, sizeof(unsigned long long), pk->stream));
  SNCK(cudaMemsetAsync(N.adam_m, 0, 2 * SN_PARAMS * sizeof(float), pk->stream));
  SNCK(cudaFuncSetAttribute(k_sn_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sn_grad_smem())));
  // one step: fresh pairs from the exact evaluator, gradients, Adam; captured once as a
  // CUDA graph and replayed (the step number lives on the device)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const int data_grid = int(std::min<int64_t>(1184, (batch + 127) / 128));
  const int grad_grid = int((batch + SN_ROWS - 1) / SN_ROWS);
  SNCK(cudaStreamBeginCapture(pk->stream, cudaStreamCaptureModeThreadLocal));
  k_sn_data<<<data_grid, 128, 0, pk->stream>>>(pk->dev, N.feat, batch, seed, N.step, need, N.x, N.y);
  cudaMemsetAsync(N.grads, 0, SN_PARAMS * sizeof(float), pk->stream);
  k_sn_grad<<<grad_grid, 256, sn_grad_smem(), pk->stream>>>(N.params, N.x, N.y, batch, N.grads, N.loss, N.step);
  k_sn_adam<<<1, 1024, 0, pk->stream>>>(N.params, N.grads, N.adam_m, N.adam_v, SN_PARAMS, float(lr), N.step);
  cudaError_t ce = cudaStreamEndCapture(pk->stream, &graph);
  if (ce != cudaSuccess) return sn_fail(pk, ICAM_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&exec, graph, 0);
  if (ce != cudaSuccess) {
    cudaGraphDestroy(graph);
    return sn_fail(pk, ICAM_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce));
  }
  for (int64_t s = 0; s < steps && ce == cudaSuccess; s++) ce = cudaGraphLaunch(exec, pk->stream);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return sn_fail(pk, ICAM_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(ce));
  if ((r = sn_pack(pk))) return r;
  if (loss_out && steps > 0)
    SNCK(cudaMemcpyAsync(loss_out, N.loss, size_t(steps) * sizeof(float), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaStreamSynchronize(pk->stream));
  return ICAM_OK;
}

int icam_seednet_ab(IcamPack* pk, size_t n, uint64_t seed, double need, double stats[8]) {
  if (!pk || !stats) return sn_fail(pk, ICAM_ERR_ARG, "null argument");
  if (!pk->net.ready) return sn_fail(pk, ICAM_ERR_ARG, "the seed network is not trained or loaded");
  SNCK(cudaSetDevice(pk->device));
  void* p;
  int r;
  const int nst = 6 + 2 * (SN_ITMAX + 1) + 1;
  if ((r = sn_alloc(pk, nst * sizeof(unsigned long long), &p))) return r;
  unsigned long long* st = static_cast<unsigned long long*>(p);
  SNCK(cudaMemsetAsync(st, 0, nst * sizeof(unsigned long long), pk->stream));
  k_sn_ab<<<int(std::min<size_t>(296, (n + 127) / 128 + 1)), 128, 0, pk->stream>>>(
      pk->dev, pk->net.feat, pk->net.wbf, int64_t(n), seed, need, st, st + nst - 1);
  SNCK(cudaGetLastError());
  std::vector<unsigned long long> h(nst);
  SNCK(cudaMemcpyAsync(h.data(), st, nst * sizeof(unsigned long long), cudaMemcpyDeviceToHost, pk->stream));
  SNCK(cudaStreamSynchronize(pk->stream));
  double pairs = double(std::max<unsigned long long>(h[0], 1));
  auto p99 = [&](int off) {
    unsigned long long acc = 0, want = (unsigned long long)std::ceil(0.99 * double(h[0]));
    for (int k = 0; k <= SN_ITMAX; k++) {
      acc += h[off + k];
      if (acc >= want) return double(k);
    }
    return double(SN_ITMAX);
  };
  unsigned long long md = h[nst - 1];
  double maxdiff;
  std::memcpy(&maxdiff, &md, sizeof(double));
  stats[0] = double(h[0]);
  stats[1] = double(h[1]) / pairs;  // mean iterations from the net's seeds
  stats[2] = double(h[2]) / pairs;  // from the centre
  stats[3] = p99(5);
  stats[4] = p99(6 + SN_ITMAX);
  stats[5] = double(h[3]) / pairs;  // fallback rate
  stats[6] = double(h[4]);          // pairs whose answers differ
  stats[7] = maxdiff;               // largest answer difference over L
  return ICAM_OK;
}

}  // extern "C"

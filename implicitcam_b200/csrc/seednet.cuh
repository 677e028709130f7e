// The seed network: a small MLP that, given a query point and a sub-patch, predicts the
// (s, t) of the sub-patch's point nearest the query (a Newton seed) and that distance (a
// ranking score). Input: the query in the sub-patch's local frame (3) and a 16-number
// descriptor of the sub-patch; hidden layers 64-64-64 with ReLU; output (s, t, d / L).
// It has no counterpart in the reference, which starts every Newton solve at the
// sub-patch's centre (gpu.wgsl node_hit; surface3.rs newton_iters); a seed from the net
// is only a start, and the solve it starts is checked as any other.
//
// Weights: an FP32 master copy for training (layout SN_*), and for inference a BF16 copy
// with each layer transposed (row = output unit), read by the tensor cores through
// warp-level mma.sync (m16n8k16, BF16 in, FP32 accumulate), 32 queries a warp.
#pragma once

#include <cuda_bf16.h>

#include "eval.cuh"

namespace icam {

constexpr int SN_IN = 19, SN_INP = 32, SN_H = 64, SN_OUT = 3, SN_OUTP = 8;
// FP32 master layout, W[k][n] row k (input) column n (output)
constexpr int SN_W1 = 0, SN_B1 = SN_W1 + SN_INP * SN_H, SN_W2 = SN_B1 + SN_H, SN_B2 = SN_W2 + SN_H * SN_H,
              SN_W3 = SN_B2 + SN_H, SN_B3 = SN_W3 + SN_H * SN_H, SN_W4 = SN_B3 + SN_H, SN_B4 = SN_W4 + SN_H * SN_OUTP,
              SN_PARAMS = SN_B4 + SN_OUTP;
// BF16 inference copy: W^T[n][k], rows padded by 8 against shared-memory bank conflicts,
// then the biases in FP32 (b1, b2, b3: 64 each, b4: 8)
constexpr int SN_KS1 = SN_INP + 8, SN_KS = SN_H + 8;
constexpr int SN_T1 = 0, SN_T2 = SN_T1 + SN_H * SN_KS1, SN_T3 = SN_T2 + SN_H * SN_KS, SN_T4 = SN_T3 + SN_H * SN_KS,
              SN_TBF = SN_T4 + SN_OUTP * SN_KS;  // BF16 elements
constexpr int SN_NBIAS = 3 * SN_H + SN_OUTP;
constexpr size_t SN_WBYTES = size_t(SN_TBF) * 2 + size_t(SN_NBIAS) * 4;
// Per sub-patch features: the local frame at its centre (origin, three unit axes), 1 / L
// (L its diagonal), then the 16-number descriptor.
constexpr int SN_FEAT = 32, SN_DESC = 16;

// The net's 19 inputs for query p and sub-patch features F.
__device__ __forceinline__ void sn_input(const float* F, double3 p, float* x) {
  float d0 = float(p.x - double(F[0])), d1 = float(p.y - double(F[1])), d2 = float(p.z - double(F[2]));
  float il = F[12];
  x[0] = (d0 * F[3] + d1 * F[4] + d2 * F[5]) * il;
  x[1] = (d0 * F[6] + d1 * F[7] + d2 * F[8]) * il;
  x[2] = (d0 * F[9] + d1 * F[10] + d2 * F[11]) * il;
#pragma unroll
  for (int k = 0; k < SN_DESC; k++) x[3 + k] = F[16 + k];
}

__device__ __forceinline__ void sn_mma(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t sn_ld2(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// One layer for the warp's 32 rows: act (32 x K, stride SN_KS, BF16) times W^T (N x K,
// stride ws) plus bias; ReLU and back into act in place, or (last layer) FP32 into out
// (32 x 8). Fragment layout of m16n8k16: lane = 4 g + t holds A rows g, g+8 at columns
// 2t, 2t+1 (+8), B column g at rows 2t, 2t+1 (+8), C rows g, g+8 at columns 2t, 2t+1.
template <int K, int N, bool LAST>
__device__ __forceinline__ void sn_layer(__nv_bfloat16* act, const __nv_bfloat16* wt, int ws, const float* bias,
                                         float* out, int lane) {
  const int g = lane >> 2, t = lane & 3;
  float acc[2][N / 8][4];
#pragma unroll
  for (int nt = 0; nt < N / 8; nt++) {
    const float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) acc[mt][nt][0] = b0, acc[mt][nt][1] = b1, acc[mt][nt][2] = b0, acc[mt][nt][3] = b1;
  }
  // the k-steps one at a time (not unrolled): a quarter of the code beside the brick
  // kernel's walk in the instruction cache (measured: learned node phase 27.2 -> 26.9 ms)
#pragma unroll 1
  for (int ks = 0; ks < K / 16; ks++) {
    uint32_t a[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      const __nv_bfloat16* r0 = act + (mt * 16 + g) * SN_KS + ks * 16 + 2 * t;
      const __nv_bfloat16* r1 = r0 + 8 * SN_KS;
      a[mt][0] = sn_ld2(r0), a[mt][1] = sn_ld2(r1), a[mt][2] = sn_ld2(r0 + 8), a[mt][3] = sn_ld2(r1 + 8);
    }
#pragma unroll
    for (int nt = 0; nt < N / 8; nt++) {
      const __nv_bfloat16* w = wt + (nt * 8 + g) * ws + ks * 16 + 2 * t;
      const uint32_t b[2] = {sn_ld2(w), sn_ld2(w + 8)};
#pragma unroll
      for (int mt = 0; mt < 2; mt++) sn_mma(acc[mt][nt], a[mt], b);
    }
  }
  __syncwarp();
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int nt = 0; nt < N / 8; nt++) {
      const int row = mt * 16 + g, col = nt * 8 + 2 * t;
      if (LAST) {
        out[row * 8 + col] = acc[mt][nt][0], out[row * 8 + col + 1] = acc[mt][nt][1];
        out[(row + 8) * 8 + col] = acc[mt][nt][2], out[(row + 8) * 8 + col + 1] = acc[mt][nt][3];
      } else {
        *reinterpret_cast<__nv_bfloat162*>(act + row * SN_KS + col) =
            __floats2bfloat162_rn(fmaxf(acc[mt][nt][0], 0.f), fmaxf(acc[mt][nt][1], 0.f));
        *reinterpret_cast<__nv_bfloat162*>(act + (row + 8) * SN_KS + col) =
            __floats2bfloat162_rn(fmaxf(acc[mt][nt][2], 0.f), fmaxf(acc[mt][nt][3], 0.f));
      }
    }
  __syncwarp();
}

// The net for the warp's 32 queries, every lane calling: x the lane's 19 inputs, y its
// 3 outputs. wbf: the BF16 weights then FP32 biases; act: the warp's 32 x SN_KS BF16
// buffer; out: its 32 x 8 floats.
__device__ __forceinline__ void sn_forward_warp(const void* wbf, __nv_bfloat16* act, float* out, const float* x,
                                                float* y, int lane) {
  const __nv_bfloat16* W = static_cast<const __nv_bfloat16*>(wbf);
  const float* B = reinterpret_cast<const float*>(W + SN_TBF);
#pragma unroll
  for (int k = 0; k < SN_INP; k += 2)
    *reinterpret_cast<__nv_bfloat162*>(act + lane * SN_KS + k) =
        __floats2bfloat162_rn(k < SN_IN ? x[k] : 0.f, k + 1 < SN_IN ? x[k + 1] : 0.f);
  __syncwarp();
  sn_layer<SN_INP, SN_H, false>(act, W + SN_T1, SN_KS1, B, out, lane);
  sn_layer<SN_H, SN_H, false>(act, W + SN_T2, SN_KS, B + SN_H, out, lane);
  sn_layer<SN_H, SN_H, false>(act, W + SN_T3, SN_KS, B + 2 * SN_H, out, lane);
  sn_layer<SN_H, SN_OUTP, true>(act, W + SN_T4, SN_KS, B + 3 * SN_H, out, lane);
  y[0] = out[lane * 8], y[1] = out[lane * 8 + 1], y[2] = out[lane * 8 + 2];
  __syncwarp();
}

}  // namespace icam

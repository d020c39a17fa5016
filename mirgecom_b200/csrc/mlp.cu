// Learned initial guess for the mixture-temperature Newton solve.
//
// A small MLP maps the mixture's internal energy and species mass fractions
// (8 inputs for the 7-species mechanism) to a temperature:
//     z1 = W1 x + b1 (64),  h1 = tanh(z1)
//     z2 = W2 h1 + b2 (64), h2 = tanh(z2)
//     y  = w3 . h2 + b3,     T = out_shift + out_scale * y
// with x the normalised inputs.  The matrix products run on the bf16 tensor
// cores (mma m16n8k16, float32 accumulate); biases, activations, the output
// layer and all gradients are float32; the optimiser keeps float32 master
// weights and refreshes the bf16 copies.
//
// One warp handles a tile of 16 samples.  The layer-1 accumulator fragments
// are re-packed in registers as the layer-2 A operand (the m16n8 accumulator
// layout of two adjacent n-tiles is exactly the m16k16 A layout), so the
// hidden activations never leave registers in inference.
//
// Training is three launches per step: forward + backward to the pre-
// activation gradients (k_mlp_fwd_bwd, which also reduces the bias and
// output-layer gradients), the weight gradients as split-K products over
// the samples (k_mlp_wgrad), and Adam (k_mlp_adam).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "physics.cuh"
#include "../../include/mgc_b200.h"

namespace {

using namespace mgc;

constexpr int H = 64;       // hidden width
constexpr int KIN = 16;     // input features padded to one k-step
constexpr int W2S = 72;     // padded bf16 row stride of W2 / W2^T in shared memory

// parameter offsets inside the float32 master vector
constexpr int P_W1 = 0;                  // [H][KIN]
constexpr int P_B1 = P_W1 + H * KIN;     // [H]
constexpr int P_W2 = P_B1 + H;           // [H][H]  (out, in)
constexpr int P_B2 = P_W2 + H * H;       // [H]
constexpr int P_W3 = P_B2 + H;           // [H]
constexpr int P_B3 = P_W3 + H;           // [1]
constexpr int NPARAM = P_B3 + 1;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// tanh x = 1 - 2 / (exp(2x) + 1), with exp(2x) = 2^(2x / ln 2) from the
// ex2.approx instruction and the reciprocal from rcp.approx: about 2e-7
// absolute error (far below the bf16 spacing of the activations), two
// special-function operations, no cancellation issue at large |x| (the
// quotient tends to 0 or 2).
__device__ __forceinline__ float tanh_fast(float x) {
  float e, r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(x * 2.8853900817779268f));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e + 1.0f));
  return fmaf(-2.0f, r, 1.0f);
}

// Inference activations: two tanh per special-function operation
// (tanh.approx.f16x2: f16 arguments and results, maximum relative error about
// 2^-11).  The guess only seeds the Newton solve, whose accepted temperature
// does not depend on where it started; training keeps tanh_fast.
__device__ __forceinline__ void tanh2_infer(float x0, float x1, float& y0, float& y1) {
  const __half2 h = __floats2half2_rn(x0, x1);
  uint32_t in = *reinterpret_cast<const uint32_t*>(&h), out;
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(out) : "r"(in));
  const __half2 r = *reinterpret_cast<const __half2*>(&out);
  y0 = __low2float(r);
  y1 = __high2float(r);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct Net {
  const __nv_bfloat16* w1;    // [H][KIN]
  const __nv_bfloat16* w2;    // [H][H]   (out, in)
  const __nv_bfloat16* w2t;   // [H][H]   (in, out)
  const float* p;             // float32 master vector (biases, w3, b3)
  float in_shift[8], in_scale[8];
  float out_shift, out_scale;
};

// Stage the bf16 weights in shared memory with padded rows.
__device__ __forceinline__ void stage_weights(const Net& net, __nv_bfloat16* w1s,
                                              __nv_bfloat16* w2s, __nv_bfloat16* w2ts,
                                              float* /*bias*/) {
  for (int i = threadIdx.x; i < H * KIN; i += blockDim.x) w1s[(i / KIN) * (KIN + 8) + i % KIN] = net.w1[i];
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
    w2s[(i / H) * W2S + i % H] = net.w2[i];
    if (w2ts) w2ts[(i / H) * W2S + i % H] = net.w2t[i];
  }
}

// bias layout in shared memory: [0,H) b1, [H,2H) b2, [2H,3H) w3, [3H] b3
__device__ __forceinline__ void stage_bias(const Net& net, float* bias) {
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    bias[i] = net.p[P_B1 + i];
    bias[H + i] = net.p[P_B2 + i];
    bias[2 * H + i] = net.p[P_W3 + i];
  }
  if (threadIdx.x == 0) bias[3 * H] = net.p[P_B3];
}

// Forward pass of one 16-sample tile held as bf16 features xs[16][KIN+8].
// Returns the per-lane accumulator fragments of z1/z2 (pre-activation) and
// h1/h2 (activations) plus the outputs y[g], y[g+8].
struct Tile {
  float h1[8][4];
  float h2[8][4];
  float y0, y1;
};

__device__ __forceinline__ void forward_tile(const __nv_bfloat16* xs, const __nv_bfloat16* w1s,
                                             const __nv_bfloat16* w2s, const float* bias,
                                             Tile& tl) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr int XS = KIN + 8;
  // layer 1: A = X (16 x 16), B = W1^T (16 x 64)
  const uint32_t a0 = *reinterpret_cast<const uint32_t*>(xs + g * XS + 2 * t);
  const uint32_t a1 = *reinterpret_cast<const uint32_t*>(xs + (g + 8) * XS + 2 * t);
  const uint32_t a2 = *reinterpret_cast<const uint32_t*>(xs + g * XS + 2 * t + 8);
  const uint32_t a3 = *reinterpret_cast<const uint32_t*>(xs + (g + 8) * XS + 2 * t + 8);
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    // B[k][n] = W1[n][k]: pairs along k are contiguous in a W1 row
    const __nv_bfloat16* wr = w1s + (nt * 8 + g) * (KIN + 8);
    const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr + 2 * t);
    const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + 2 * t + 8);
    mma_bf16(d, a0, a1, a2, a3, b0, b1);
    const float bb0 = bias[nt * 8 + 2 * t], bb1 = bias[nt * 8 + 2 * t + 1];
    tl.h1[nt][0] = tanh_fast(d[0] + bb0);
    tl.h1[nt][1] = tanh_fast(d[1] + bb1);
    tl.h1[nt][2] = tanh_fast(d[2] + bb0);
    tl.h1[nt][3] = tanh_fast(d[3] + bb1);
  }
  // layer 2: A = H1 (16 x 64) re-packed from the accumulators, B = W2^T
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    const __nv_bfloat16* wr = w2s + (nt * 8 + g) * W2S;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint32_t x0 = pack_bf16(tl.h1[2 * kk][0], tl.h1[2 * kk][1]);
      const uint32_t x1 = pack_bf16(tl.h1[2 * kk][2], tl.h1[2 * kk][3]);
      const uint32_t x2 = pack_bf16(tl.h1[2 * kk + 1][0], tl.h1[2 * kk + 1][1]);
      const uint32_t x3 = pack_bf16(tl.h1[2 * kk + 1][2], tl.h1[2 * kk + 1][3]);
      const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr + kk * 16 + 2 * t);
      const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + kk * 16 + 2 * t + 8);
      mma_bf16(d, x0, x1, x2, x3, b0, b1);
    }
    const float bb0 = bias[H + nt * 8 + 2 * t], bb1 = bias[H + nt * 8 + 2 * t + 1];
    tl.h2[nt][0] = tanh_fast(d[0] + bb0);
    tl.h2[nt][1] = tanh_fast(d[1] + bb1);
    tl.h2[nt][2] = tanh_fast(d[2] + bb0);
    tl.h2[nt][3] = tanh_fast(d[3] + bb1);
  }
  // layer 3 (float32): partial dot products, reduced over the 4 lanes of a row
  float s0 = 0.f, s1 = 0.f;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float w0 = bias[2 * H + nt * 8 + 2 * t], w1v = bias[2 * H + nt * 8 + 2 * t + 1];
    s0 += w0 * tl.h2[nt][0] + w1v * tl.h2[nt][1];
    s1 += w0 * tl.h2[nt][2] + w1v * tl.h2[nt][3];
  }
  s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
  s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
  tl.y0 = s0 + bias[3 * H];
  tl.y1 = s1 + bias[3 * H];
}

// Inference-only forward pass of one 16-sample tile: the same arithmetic as
// forward_tile, with the layer-1 activations kept only as the packed bf16
// pairs that form the layer-2 A fragments and the output layer accumulated
// per layer-2 n-tile, so no activation array stays live.  Lanes with
// lane % 4 == 0 hold y[g], y[g+8] in y0, y1.
__device__ __forceinline__ void forward_tile_y(const __nv_bfloat16* xs,
                                               const __nv_bfloat16* w1s,
                                               const __nv_bfloat16* w2s, const float* bias,
                                               float& y0, float& y1) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr int XS = KIN + 8;
  const uint32_t a0 = *reinterpret_cast<const uint32_t*>(xs + g * XS + 2 * t);
  const uint32_t a1 = *reinterpret_cast<const uint32_t*>(xs + (g + 8) * XS + 2 * t);
  const uint32_t a2 = *reinterpret_cast<const uint32_t*>(xs + g * XS + 2 * t + 8);
  const uint32_t a3 = *reinterpret_cast<const uint32_t*>(xs + (g + 8) * XS + 2 * t + 8);
  uint32_t hp[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    const __nv_bfloat16* wr = w1s + (nt * 8 + g) * (KIN + 8);
    mma_bf16(d, a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(wr + 2 * t),
             *reinterpret_cast<const uint32_t*>(wr + 2 * t + 8));
    const float bb0 = bias[nt * 8 + 2 * t], bb1 = bias[nt * 8 + 2 * t + 1];
    float h0, h1, h2, h3;
    tanh2_infer(d[0] + bb0, d[1] + bb1, h0, h1);
    tanh2_infer(d[2] + bb0, d[3] + bb1, h2, h3);
    hp[nt][0] = pack_bf16(h0, h1);
    hp[nt][1] = pack_bf16(h2, h3);
  }
  float s0 = 0.f, s1 = 0.f;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    const __nv_bfloat16* wr = w2s + (nt * 8 + g) * W2S;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma_bf16(d, hp[2 * kk][0], hp[2 * kk][1], hp[2 * kk + 1][0], hp[2 * kk + 1][1],
               *reinterpret_cast<const uint32_t*>(wr + kk * 16 + 2 * t),
               *reinterpret_cast<const uint32_t*>(wr + kk * 16 + 2 * t + 8));
    const float bb0 = bias[H + nt * 8 + 2 * t], bb1 = bias[H + nt * 8 + 2 * t + 1];
    const float w0 = bias[2 * H + nt * 8 + 2 * t], w1v = bias[2 * H + nt * 8 + 2 * t + 1];
    float h0, h1, h2, h3;
    tanh2_infer(d[0] + bb0, d[1] + bb1, h0, h1);
    tanh2_infer(d[2] + bb0, d[3] + bb1, h2, h3);
    s0 += w0 * h0 + w1v * h1;
    s1 += w0 * h2 + w1v * h3;
  }
  s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
  s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
  y0 = s0 + bias[3 * H];
  y1 = s1 + bias[3 * H];
}

constexpr int WARPS = 4;

// {{{ inference on a conserved state

template <int DIM, int NS>
__global__ void __launch_bounds__(WARPS * 32) k_mlp_infer(int64_t n, const float* __restrict__ q,
                                                          Net net, float* __restrict__ tout) {
  __shared__ __align__(16) __nv_bfloat16 w1s[H * (KIN + 8)];
  __shared__ __align__(16) __nv_bfloat16 w2s[H * W2S];
  __shared__ float bias[3 * H + 1];
  __shared__ __align__(16) __nv_bfloat16 xs_all[WARPS][16 * (KIN + 8)];
  stage_weights(net, w1s, w2s, nullptr, bias);
  stage_bias(net, bias);
  __syncthreads();
  constexpr int NC = DIM + 2 + NS;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __nv_bfloat16* xs = xs_all[warp];
  const int64_t ntiles = (n + 15) / 16;
  for (int64_t tile = (int64_t)blockIdx.x * WARPS + warp; tile < ntiles;
       tile += (int64_t)gridDim.x * WARPS) {
    if (lane < 16) {
      const int64_t s = tile * 16 + lane;
      float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (s < n) {
        const float rho = q[s];
        float ke = 0.f;
#pragma unroll
        for (int i = 0; i < DIM; ++i) {
          const float m = q[(int64_t)(2 + i) * n + s];
          ke += m * m;
        }
        f[0] = (q[n + s] - 0.5f * ke / rho) / rho;
#pragma unroll
        for (int k = 0; k < NS && k < 7; ++k) f[1 + k] = q[(int64_t)(2 + DIM + k) * n + s] / rho;
      }
#pragma unroll
      for (int j = 0; j < KIN; j += 2) {
        const float v0 = j < 8 ? (f[j] - net.in_shift[j]) * net.in_scale[j] : 0.f;
        const float v1 = j + 1 < 8 ? (f[j + 1] - net.in_shift[j + 1]) * net.in_scale[j + 1] : 0.f;
        *reinterpret_cast<uint32_t*>(xs + lane * (KIN + 8) + j) = pack_bf16(v0, v1);
      }
    }
    __syncwarp();
    float y0, y1;
    forward_tile_y(xs, w1s, w2s, bias, y0, y1);
    if ((lane & 3) == 0) {
      const int g = lane >> 2;
      const int64_t s0 = tile * 16 + g, s1 = s0 + 8;
      if (s0 < n) tout[s0] = net.out_shift + net.out_scale * y0;
      if (s1 < n) tout[s1] = net.out_shift + net.out_scale * y1;
    }
    __syncwarp();
  }
}

// }}}

// {{{ training: forward + backward to pre-activation gradients

// x: [n][8] normalised inputs, tgt: [n] normalised targets.
// Writes xb [n][KIN] (bf16 inputs), h1b [n][H] (bf16), dz1 / dz2 [n][H]
// (bf16) and accumulates the gradients of b1, b2, w3, b3 and the loss sum.
__global__ void __launch_bounds__(WARPS * 32) k_mlp_fwd_bwd(
    int64_t n, const float* __restrict__ x, const float* __restrict__ tgt, Net net,
    __nv_bfloat16* __restrict__ xb, __nv_bfloat16* __restrict__ h1b,
    __nv_bfloat16* __restrict__ dz1b, __nv_bfloat16* __restrict__ dz2b,
    float* __restrict__ grad, float* __restrict__ loss, float inv_n) {
  __shared__ __align__(16) __nv_bfloat16 w1s[H * (KIN + 8)];
  __shared__ __align__(16) __nv_bfloat16 w2s[H * W2S];
  __shared__ __align__(16) __nv_bfloat16 w2ts[H * W2S];
  __shared__ float bias[3 * H + 1];
  __shared__ float gacc[3 * H + 2];      // db1, db2, dw3, db3, loss
  __shared__ __align__(16) __nv_bfloat16 xs_all[WARPS][16 * (KIN + 8)];
  stage_weights(net, w1s, w2s, w2ts, bias);
  stage_bias(net, bias);
  for (int i = threadIdx.x; i < 3 * H + 2; i += blockDim.x) gacc[i] = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  __nv_bfloat16* xs = xs_all[warp];
  const int64_t ntiles = (n + 15) / 16;
  float db1[8][2], db2[8][2], dw3[8][2], db3 = 0.f, lsum = 0.f;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
    db1[nt][0] = db1[nt][1] = db2[nt][0] = db2[nt][1] = dw3[nt][0] = dw3[nt][1] = 0.f;
  for (int64_t tile = (int64_t)blockIdx.x * WARPS + warp; tile < ntiles;
       tile += (int64_t)gridDim.x * WARPS) {
    if (lane < 16) {
      const int64_t s = tile * 16 + lane;
#pragma unroll
      for (int j = 0; j < KIN; j += 2) {
        const float v0 = (s < n && j < 8) ? x[s * 8 + j] : 0.f;
        const float v1 = (s < n && j + 1 < 8) ? x[s * 8 + j + 1] : 0.f;
        const uint32_t pk = pack_bf16(v0, v1);
        *reinterpret_cast<uint32_t*>(xs + lane * (KIN + 8) + j) = pk;
        if (s < n) *reinterpret_cast<uint32_t*>(xb + s * KIN + j) = pk;
      }
    }
    __syncwarp();
    Tile tl;
    forward_tile(xs, w1s, w2s, bias, tl);
    const int64_t s0 = tile * 16 + g, s1 = s0 + 8;
    const bool v0 = s0 < n, v1 = s1 < n;
    // dL/dy for L = (1/n) sum (y - t)^2
    const float r0 = v0 ? tl.y0 - tgt[s0] : 0.f;
    const float r1 = v1 ? tl.y1 - tgt[s1] : 0.f;
    if (t == 0) lsum += r0 * r0 + r1 * r1;
    const float dy0 = 2.f * r0 * inv_n, dy1 = 2.f * r1 * inv_n;
    if (t == 0) db3 += dy0 + dy1;
    // dz2 = dy w3 (1 - h2^2); dw3 += dy h2
    float dz2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c0 = nt * 8 + 2 * t;
      const float w0 = bias[2 * H + c0], w1v = bias[2 * H + c0 + 1];
      dw3[nt][0] += dy0 * tl.h2[nt][0] + dy1 * tl.h2[nt][2];
      dw3[nt][1] += dy0 * tl.h2[nt][1] + dy1 * tl.h2[nt][3];
      dz2[nt][0] = dy0 * w0 * (1.f - tl.h2[nt][0] * tl.h2[nt][0]);
      dz2[nt][1] = dy0 * w1v * (1.f - tl.h2[nt][1] * tl.h2[nt][1]);
      dz2[nt][2] = dy1 * w0 * (1.f - tl.h2[nt][2] * tl.h2[nt][2]);
      dz2[nt][3] = dy1 * w1v * (1.f - tl.h2[nt][3] * tl.h2[nt][3]);
      db2[nt][0] += dz2[nt][0] + dz2[nt][2];
      db2[nt][1] += dz2[nt][1] + dz2[nt][3];
    }
    // dh1 = dz2 W2 on the tensor cores: A = dZ2 (16 x 64), B[k][n] = W2[k][n]
    // (pairs along k contiguous in a row of W2^T)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      const __nv_bfloat16* wr = w2ts + (nt * 8 + g) * W2S;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint32_t x0 = pack_bf16(dz2[2 * kk][0], dz2[2 * kk][1]);
        const uint32_t x1 = pack_bf16(dz2[2 * kk][2], dz2[2 * kk][3]);
        const uint32_t x2 = pack_bf16(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
        const uint32_t x3 = pack_bf16(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
        const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr + kk * 16 + 2 * t);
        const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + kk * 16 + 2 * t + 8);
        mma_bf16(d, x0, x1, x2, x3, b0, b1);
      }
      const int c0 = nt * 8 + 2 * t;
      const float dz1_00 = d[0] * (1.f - tl.h1[nt][0] * tl.h1[nt][0]);
      const float dz1_01 = d[1] * (1.f - tl.h1[nt][1] * tl.h1[nt][1]);
      const float dz1_10 = d[2] * (1.f - tl.h1[nt][2] * tl.h1[nt][2]);
      const float dz1_11 = d[3] * (1.f - tl.h1[nt][3] * tl.h1[nt][3]);
      db1[nt][0] += dz1_00 + dz1_10;
      db1[nt][1] += dz1_01 + dz1_11;
      if (v0) {
        *reinterpret_cast<uint32_t*>(dz1b + s0 * H + c0) = pack_bf16(dz1_00, dz1_01);
        *reinterpret_cast<uint32_t*>(dz2b + s0 * H + c0) = pack_bf16(dz2[nt][0], dz2[nt][1]);
        *reinterpret_cast<uint32_t*>(h1b + s0 * H + c0) = pack_bf16(tl.h1[nt][0], tl.h1[nt][1]);
      }
      if (v1) {
        *reinterpret_cast<uint32_t*>(dz1b + s1 * H + c0) = pack_bf16(dz1_10, dz1_11);
        *reinterpret_cast<uint32_t*>(dz2b + s1 * H + c0) = pack_bf16(dz2[nt][2], dz2[nt][3]);
        *reinterpret_cast<uint32_t*>(h1b + s1 * H + c0) = pack_bf16(tl.h1[nt][2], tl.h1[nt][3]);
      }
    }
    __syncwarp();
  }
  // reduce the per-lane vector gradients over the 8 row groups (lanes with
  // equal t), then over warps in shared memory, then across CTAs in HBM
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float a = db1[nt][h], b = db2[nt][h], c = dw3[nt][h];
#pragma unroll
      for (int off = 4; off < 32; off <<= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
        c += __shfl_xor_sync(0xffffffffu, c, off);
      }
      if (g == 0) {
        atomicAdd(&gacc[nt * 8 + 2 * t + h], a);
        atomicAdd(&gacc[H + nt * 8 + 2 * t + h], b);
        atomicAdd(&gacc[2 * H + nt * 8 + 2 * t + h], c);
      }
    }
#pragma unroll
  for (int off = 4; off < 32; off <<= 1) {
    db3 += __shfl_xor_sync(0xffffffffu, db3, off);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
  }
  if (lane == 0) {
    atomicAdd(&gacc[3 * H], db3);
    atomicAdd(&gacc[3 * H + 1], lsum);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    atomicAdd(&grad[P_B1 + i], gacc[i]);
    atomicAdd(&grad[P_B2 + i], gacc[H + i]);
    atomicAdd(&grad[P_W3 + i], gacc[2 * H + i]);
  }
  if (threadIdx.x == 0) {
    atomicAdd(&grad[P_B3], gacc[3 * H]);
    atomicAdd(loss, gacc[3 * H + 1] * inv_n);
  }
}

// dW[o][i] += sum_s dz[s][o] a[s][i]  (o < H, i < KA), split over samples.
// Each warp owns one 16-row m-tile of o; a chunk of 16 samples is one k-step.
template <int KA>
__global__ void __launch_bounds__(WARPS * 32) k_mlp_wgrad(int64_t n,
                                                          const __nv_bfloat16* __restrict__ dz,
                                                          const __nv_bfloat16* __restrict__ a,
                                                          float* __restrict__ dw) {
  __shared__ __align__(16) __nv_bfloat16 dzt[H][16 + 8];   // [o][s]
  __shared__ __align__(16) __nv_bfloat16 at[KA][16 + 8];   // [i][s]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr int NT = KA / 8;
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const int64_t nchunks = (n + 15) / 16;
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < 16 * H; i += blockDim.x) {
      const int s = i / H, o = i % H;
      const int64_t gs = ch * 16 + s;
      dzt[o][s] = gs < n ? dz[gs * H + o] : __float2bfloat16(0.f);
    }
    for (int i = threadIdx.x; i < 16 * KA; i += blockDim.x) {
      const int s = i / KA, c = i % KA;
      const int64_t gs = ch * 16 + s;
      at[c][s] = gs < n ? a[gs * KA + c] : __float2bfloat16(0.f);
    }
    __syncthreads();
    // A[m=o][k=s] = dz^T, B[k=s][n=i] = a
    const int o0 = warp * 16;
    const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&dzt[o0 + g][2 * t]);
    const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&dzt[o0 + g + 8][2 * t]);
    const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&dzt[o0 + g][2 * t + 8]);
    const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&dzt[o0 + g + 8][2 * t + 8]);
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&at[j * 8 + g][2 * t]);
      const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&at[j * 8 + g][2 * t + 8]);
      mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
    }
  }
  const int o0 = warp * 16;
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const int c0 = j * 8 + 2 * t;
    atomicAdd(&dw[(o0 + g) * KA + c0], acc[j][0]);
    atomicAdd(&dw[(o0 + g) * KA + c0 + 1], acc[j][1]);
    atomicAdd(&dw[(o0 + g + 8) * KA + c0], acc[j][2]);
    atomicAdd(&dw[(o0 + g + 8) * KA + c0 + 1], acc[j][3]);
  }
}

// Adam on the float32 master vector; refreshes the bf16 copies of W1, W2, W2^T.
__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ gr,
                           float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                           float b2, float eps, float bc1, float bc2,
                           __nv_bfloat16* __restrict__ w1, __nv_bfloat16* __restrict__ w2,
                           __nv_bfloat16* __restrict__ w2t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    if (i < P_B1 && (i % KIN) >= 8) pi = 0.f;       // padded input columns stay zero
    p[i] = pi;
    if (i < P_B1) w1[i] = __float2bfloat16(pi);
    if (i >= P_W2 && i < P_B2) {
      const int o = (i - P_W2) / H, k = (i - P_W2) % H;
      w2[o * H + k] = __float2bfloat16(pi);
      w2t[k * H + o] = __float2bfloat16(pi);
    }
  }
}

// bf16 copies from the master vector (initialisation / after a host update)
__global__ void k_mlp_refresh(const float* __restrict__ p, __nv_bfloat16* __restrict__ w1,
                              __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w2t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    if (i < P_B1) w1[i] = __float2bfloat16(p[i]);
    if (i >= P_W2 && i < P_B2) {
      const int o = (i - P_W2) / H, k = (i - P_W2) % H;
      w2[o * H + k] = __float2bfloat16(p[i]);
      w2t[k * H + o] = __float2bfloat16(p[i]);
    }
  }
}

Net make_net(const mgc_mlp_t* w) {
  Net net;
  net.w1 = reinterpret_cast<const __nv_bfloat16*>(w->w1_bf16);
  net.w2 = reinterpret_cast<const __nv_bfloat16*>(w->w2_bf16);
  net.w2t = reinterpret_cast<const __nv_bfloat16*>(w->w2t_bf16);
  net.p = w->params;
  for (int i = 0; i < 8; ++i) {
    net.in_shift[i] = w->in_shift[i];
    net.in_scale[i] = w->in_scale[i];
  }
  net.out_shift = w->out_shift;
  net.out_scale = w->out_scale;
  return net;
}

bool mlp_ok(const mgc_mlp_t* w) {
  return w && w->params && w->w1_bf16 && w->w2_bf16 && w->w2t_bf16;
}

int grid_for(int64_t tiles) {
  int64_t nb = (tiles + WARPS - 1) / WARPS;
  if (nb > 148 * 8) nb = 148 * 8;
  return nb < 1 ? 1 : (int)nb;
}

// {{{ mixture temperature with the learned guess (fused)

// A seed whose first Newton step is at most this large already needs no more
// float32 steps than a network guess would (the step after it is below
// k dT^2 = 0.05 K, and the trained network's validation error is larger than
// this), so a warp whose seeds all pass skips the network.
constexpr float kWarmSeedK = 4.0f;

// One warp per 32 nodes.  First every lane takes one float32 Newton step
// from its seed; when all the warp's steps are within kWarmSeedK the solve
// simply continues from there (iteration count + 100 marks these nodes).
// Otherwise the network runs on the warp's two 16-sample tiles (features
// from the node's float64 energy and mass fractions), the guesses go through
// shared memory, and each lane solves its node's temperature with
// mixed_newton from the guess, falling back to the seed when the float64
// residual check fails (iteration count + 1000 marks it).
template <int DIM, int NS>
__global__ void __launch_bounds__(WARPS * 32, 6) k_mixture_state_learned(
    int64_t n, const float* __restrict__ q, const float* __restrict__ tseed, Net net,
    float* __restrict__ tout, int32_t* __restrict__ iters, int maxit, double rtol,
    int32_t* __restrict__ status) {
  __shared__ __align__(16) __nv_bfloat16 w1s[H * (KIN + 8)];
  __shared__ __align__(16) __nv_bfloat16 w2s[H * W2S];
  __shared__ float bias[3 * H + 1];
  __shared__ __align__(16) __nv_bfloat16 xs_all[WARPS][32 * (KIN + 8)];
  __shared__ float tg_all[WARPS][32];
  stage_weights(net, w1s, w2s, nullptr, bias);
  stage_bias(net, bias);
  __syncthreads();
  constexpr int NC = DIM + 2 + NS;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __nv_bfloat16* xs = xs_all[warp];
  float* tg = tg_all[warp];
  bool miss = false;
  const int64_t nchunks = (n + 31) / 32;
  for (int64_t ch = (int64_t)blockIdx.x * WARPS + warp; ch < nchunks;
       ch += (int64_t)gridDim.x * WARPS) {
    const int64_t s = ch * 32 + lane;
    const bool valid = s < n;
    float qq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) qq[c] = valid ? q[(int64_t)c * n + s] : (c == 0 ? 1.f : 0.f);
    float y[NS], e32;
    double yd[NS], e64;
    mixed_newton_inputs<DIM, NS>(qq, y, yd, e32, e64);
    // one float32 step from the seed; a warm warp continues from there
    const float ts = valid ? tseed[s] : 1000.f;
    float t, em, cv;
    mixture_e_cv<float, NS>(y, ts, em, cv);
    const float dt0 = (e32 - em) / cv;
    int used, mx;
    if (__all_sync(0xffffffffu, !valid || (ts > 0.f && fabsf(dt0) <= kWarmSeedK))) {
      const float k = mech<float>().newton_k, rt = (float)rtol;
      t = ts + dt0;
      used = 101;        // one step, + 100: the network was skipped
      mx = (k * dt0 * dt0 <= 0.25f * sqrtf(rt * fabsf(t) / k)) ? 0 : maxit - 1;
    } else {
      // network guess for the warp's 32 nodes (features from the inputs)
      float f[8];
      f[0] = e32;
#pragma unroll
      for (int k = 0; k < 7; ++k) f[1 + k] = k < NS ? y[k] : 0.f;
#pragma unroll
      for (int j = 0; j < KIN; j += 2) {
        const float v0 = j < 8 ? (f[j] - net.in_shift[j]) * net.in_scale[j] : 0.f;
        const float v1 = j + 1 < 8 ? (f[j + 1] - net.in_shift[j + 1]) * net.in_scale[j + 1] : 0.f;
        *reinterpret_cast<uint32_t*>(xs + lane * (KIN + 8) + j) = pack_bf16(v0, v1);
      }
      __syncwarp();
#pragma unroll 1
      for (int half = 0; half < 2; ++half) {
        float y0, y1;
        forward_tile_y(xs + half * 16 * (KIN + 8), w1s, w2s, bias, y0, y1);
        if ((lane & 3) == 0) {
          const int g = lane >> 2;
          tg[half * 16 + g] = net.out_shift + net.out_scale * y0;
          tg[half * 16 + g + 8] = net.out_shift + net.out_scale * y1;
        }
      }
      __syncwarp();
      t = tg[lane];
      used = 0;
      mx = maxit;
      __syncwarp();
      // the Newton inputs are derived again (the second read of q hits L1),
      // so that none of them stays live across the network
#pragma unroll
      for (int c = 0; c < NC; ++c) qq[c] = valid ? q[(int64_t)c * n + s] : (c == 0 ? 1.f : 0.f);
      mixed_newton_inputs<DIM, NS>(qq, y, yd, e32, e64);
    }
    if (valid) {
      bool ok = mixed_newton<NS>(y, yd, e32, e64, t, mx, rtol, used);
      if (!ok) {
        used += 1000;
        t = ts;
        ok = mixed_newton<NS>(y, yd, e32, e64, t, maxit, rtol, used);
      }
      if (!ok) miss = true;
      tout[s] = t;
      if (iters) iters[s] = used;
    }
  }
  if (miss) atomicOr(status, ST_NEWTON_MISS);
}

// }}}

bool g_mech_ready_mlp[64] = {};

}  // namespace

namespace mgc {

// this unit's copy of the mechanism tables (mgc_set_mechanism)
int mlp_upload_mechanism(const Mechanism* m) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MGC_E_CUDA;
  if (cudaMemcpyToSymbol(c_mech, m, sizeof(Mechanism)) != cudaSuccess) return MGC_E_CUDA;
  const MechanismT<float> f = narrow_mechanism(*m);
  if (cudaMemcpyToSymbol(c_mech32, &f, sizeof(f)) != cudaSuccess) return MGC_E_CUDA;
  g_mech_ready_mlp[dev] = true;
  return MGC_OK;
}

}  // namespace mgc

extern "C" {

int mgc_mlp_nparams(void) { return NPARAM; }

int mgc_mlp_refresh(const mgc_mlp_t* w, void* stream) {
  if (!mlp_ok(w)) return MGC_E_INVALID;
  k_mlp_refresh<<<8, 256, 0, (cudaStream_t)stream>>>(
      w->params, reinterpret_cast<__nv_bfloat16*>(w->w1_bf16),
      reinterpret_cast<__nv_bfloat16*>(w->w2_bf16), reinterpret_cast<__nv_bfloat16*>(w->w2t_bf16));
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

int mgc_mlp_infer(int dim, int nspecies, int64_t n, const float* q, const mgc_mlp_t* w,
                  float* t_out, void* stream) {
  if (!mlp_ok(w) || !q || !t_out || n < 0 || nspecies != 7 || (dim != 2 && dim != 3))
    return MGC_E_INVALID;
  if (n == 0) return MGC_OK;
  const Net net = make_net(w);
  const int nb = grid_for((n + 15) / 16);
  if (dim == 3)
    k_mlp_infer<3, 7><<<nb, WARPS * 32, 0, (cudaStream_t)stream>>>(n, q, net, t_out);
  else
    k_mlp_infer<2, 7><<<nb, WARPS * 32, 0, (cudaStream_t)stream>>>(n, q, net, t_out);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

size_t mgc_mlp_train_workspace_bytes(int64_t n) {
  return (size_t)n * (KIN + 3 * H) * sizeof(__nv_bfloat16) + 256;
}

int mgc_mlp_train_grad(int64_t n, const float* x, const float* target, const mgc_mlp_t* w,
                       void* workspace, size_t workspace_bytes, float* grad, float* loss,
                       void* stream) {
  if (!mlp_ok(w) || !x || !target || !grad || !loss || n <= 0 || !workspace)
    return MGC_E_INVALID;
  if (workspace_bytes < mgc_mlp_train_workspace_bytes(n)) return MGC_E_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  __nv_bfloat16* xb = static_cast<__nv_bfloat16*>(workspace);
  __nv_bfloat16* h1b = xb + (size_t)n * KIN;
  __nv_bfloat16* dz1b = h1b + (size_t)n * H;
  __nv_bfloat16* dz2b = dz1b + (size_t)n * H;
  if (cudaMemsetAsync(grad, 0, NPARAM * sizeof(float), s) != cudaSuccess) return MGC_E_CUDA;
  if (cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) return MGC_E_CUDA;
  const Net net = make_net(w);
  const int nb = grid_for((n + 15) / 16);
  k_mlp_fwd_bwd<<<nb, WARPS * 32, 0, s>>>(n, x, target, net, xb, h1b, dz1b, dz2b, grad, loss,
                                         1.0f / (float)n);
  const int nbw = (int)((n + 15) / 16 < 148 * 4 ? (n + 15) / 16 : 148 * 4);
  k_mlp_wgrad<H><<<nbw, WARPS * 32, 0, s>>>(n, dz2b, h1b, grad + P_W2);
  k_mlp_wgrad<KIN><<<nbw, WARPS * 32, 0, s>>>(n, dz1b, xb, grad + P_W1);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

int mgc_mlp_adam(const mgc_mlp_t* w, const float* grad, float* m, float* v, float lr,
                 float beta1, float beta2, float eps, int step, void* stream) {
  if (!mlp_ok(w) || !grad || !m || !v || step < 1) return MGC_E_INVALID;
  const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
  k_mlp_adam<<<8, 256, 0, (cudaStream_t)stream>>>(
      w->params, grad, m, v, lr, beta1, beta2, eps, bc1, bc2,
      reinterpret_cast<__nv_bfloat16*>(w->w1_bf16), reinterpret_cast<__nv_bfloat16*>(w->w2_bf16),
      reinterpret_cast<__nv_bfloat16*>(w->w2t_bf16));
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

int mgc_mixture_temperature_learned_f32(int dim, const mgc_gas_t* gas, int64_t nnodes,
                                        const float* q, const float* t_seed,
                                        const mgc_mlp_t* mlp, float* t_out,
                                        int32_t* iterations, int maxit, float rtol,
                                        int32_t* status, void* stream) {
  if (!gas || gas->eos_kind != MGC_EOS_MIXTURE || gas->nspecies != 7 || !mlp_ok(mlp) ||
      nnodes < 0 || !q || !t_seed || !t_out || !status || maxit < 1 || !(rtol > 0.f) ||
      (dim != 2 && dim != 3))
    return MGC_E_INVALID;
  if (nnodes == 0) return MGC_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MGC_E_CUDA;
  if (!g_mech_ready_mlp[dev]) return MGC_E_NOT_READY;
  const Net net = make_net(mlp);
  cudaStream_t s = (cudaStream_t)stream;
  auto kern = dim == 3 ? k_mixture_state_learned<3, 7> : k_mixture_state_learned<2, 7>;
  // grid-stride over 32-node chunks: one wave of resident blocks
  int sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, 0) != cudaSuccess)
    return MGC_E_CUDA;
  const int64_t want = ((nnodes + 31) / 32 + WARPS - 1) / WARPS;
  int64_t nb = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  if (nb > want) nb = want;
  kern<<<(unsigned)(nb > 0 ? nb : 1), WARPS * 32, 0, s>>>(nnodes, q, t_seed, net, t_out,
                                                          iterations, maxit, (double)rtol, status);
  return cudaGetLastError() == cudaSuccess ? MGC_OK : MGC_E_CUDA;
}

}  // extern "C"

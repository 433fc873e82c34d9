// Learned drop tolerances for the approximate inverse: per-row features and
// a small MLP (32 -> 64 -> 64 -> 2) trained and run on the GPU.
//
// The reference picks one global drop tolerance for fastainv_sym by a
// golden-section search that costs a full build and solve per probe
// (fastainv/droptol-tuning.h:4-103).  Here a per-row network predicts, from
// local matrix features, the drop tolerance of each row of the factor and a
// diagonal rescale of that row (applied through fastainv_sym_ex); the
// caller keeps the plain build as the fallback and the yardstick.
//
// Network: y = W3 relu(W2 relu(W1 x + b1) + b2) + b3 with BF16 weights and
// inputs and FP32 accumulation.  Layers 1 and 2 (and the weight gradients of
// both) run on the tensor cores with mma.sync m16n8k16 (BF16 in, FP32
// accumulate): at 12.5 kflop per 64-byte feature row the network is
// bandwidth-bound, far below the point where tcgen05's larger tiles would
// pay.  Layer 3 (two outputs) runs on the FP32 cores.  Rounding points, which
// the CPU oracle reproduces: x, W1, W2, W3 and the layer-1 activations are
// BF16; the layer-2 activations stay FP32 for layer 3; in the backward pass
// the layer-2 and layer-1 activation gradients are rounded to BF16 where they
// feed a tensor-core product (dH1 = dH2 W2, dW2 = dH2^T H1, dW1 = dH1^T X)
// and kept FP32 for the bias gradients and dW3.
//
// Training is deterministic: each CTA accumulates its rows' gradients in a
// fixed order and writes one partial per CTA; a second kernel adds the
// partials in CTA order; Adam runs on FP32 master weights.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "cuda_util.cuh"

namespace ispm {
namespace {

constexpr int kIn = 32, kH = 64, kOut = 2;
constexpr int kW1 = 0, kB1 = kW1 + kH * kIn, kW2 = kB1 + kH, kB2 = kW2 + kH * kH,
              kW3 = kB2 + kH, kB3 = kW3 + kOut * kH, kParams = kB3 + kOut;
constexpr int kPart = kParams + 1;  // + loss
constexpr int kWarps = 4, kThreads = 32 * kWarps;
constexpr int kBlockRows = 128;     // rows per CTA step: 32 per warp, two 16-row tiles
constexpr int kLd1 = kIn + 8;       // padded smem row lengths (bank-conflict-free
constexpr int kLd2 = kH + 8;        // fragment loads)
constexpr int kLdT = kBlockRows + 8;
constexpr int kRed = 2 * kH + kOut * kH + kOut + 1;  // db1, db2, dW3, db3, loss

using bf16 = __nv_bfloat16;

struct Smem {
  bf16 w1[kH * kLd1];
  bf16 w2[kH * kLd2];
  bf16 w2t[kH * kLd2];
  float b1[kH], b2[kH], w3[kOut * kH], b3[kOut];
  float red[kWarps][kRed];
  // training staging, transposed: [feature][row of the CTA step]
  bf16 xt[kIn * kLdT];
  bf16 h1t[kH * kLdT];
  bf16 d2t[kH * kLdT];
  bf16 d1t[kH * kLdT];
};

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ float lo_f(uint32_t v)
{
  return __uint_as_float(v << 16);
}

__device__ __forceinline__ float hi_f(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

__device__ __forceinline__ uint32_t ld32(const bf16 *p)
{
  return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ void st2(bf16 *p0, bf16 *p1, uint32_t v)
{
  *reinterpret_cast<uint16_t *>(p0) = (uint16_t)(v & 0xffffu);
  *reinterpret_cast<uint16_t *>(p1) = (uint16_t)(v >> 16);
}

// D += A B, m16n8k16, BF16 inputs, FP32 accumulators.
__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                    uint32_t b1)
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Weights into shared memory (BF16-rounded), W2 also transposed.
__device__ void load_weights(Smem &s, const float *__restrict__ prm, bool train)
{
  for (int i = threadIdx.x; i < kH * kIn; i += blockDim.x)
    s.w1[(i / kIn) * kLd1 + i % kIn] = __float2bfloat16_rn(prm[kW1 + i]);
  for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
    const bf16 v = __float2bfloat16_rn(prm[kW2 + i]);
    s.w2[(i / kH) * kLd2 + i % kH] = v;
    if (train)
      s.w2t[(i % kH) * kLd2 + i / kH] = v;
  }
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    s.b1[i] = prm[kB1 + i];
    s.b2[i] = prm[kB2 + i];
  }
  for (int i = threadIdx.x; i < kOut * kH; i += blockDim.x)
    s.w3[i] = __bfloat162float(__float2bfloat16_rn(prm[kW3 + i]));
  if (threadIdx.x < kOut)
    s.b3[threadIdx.x] = prm[kB3 + threadIdx.x];
  if (train)
    for (int i = threadIdx.x; i < kWarps * kRed; i += blockDim.x)
      (&s.red[0][0])[i] = 0.f;
}

// Sum over the 8 lanes sharing threadID_in_group (lane bits 2..4).
__device__ __forceinline__ float sum_g(float v)
{
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  return v;
}

// One 16-row tile: forward pass (and, when training, the backward pass up
// to the staged activation gradients).  Rows >= M contribute nothing.
template <bool TRAIN>
__device__ __forceinline__ void tile(Smem &s, const bf16 *__restrict__ X,
                                     const float2 *__restrict__ T, const float2 *__restrict__ Wt,
                                     float2 *__restrict__ Y, long long r0, long long M,
                                     float scale, int lr0)
{
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, w = threadIdx.x >> 5;
  const long long ra = r0 + g, rb = r0 + g + 8;
  const bool va = ra < M, vb = rb < M;
  // X fragments (K = 32: two k-steps)
  uint32_t xa[2][4];
#pragma unroll
  for (int kk = 0; kk < 2; kk++) {
    const int c = kk * 16 + 2 * t;
    xa[kk][0] = va ? __ldg(reinterpret_cast<const unsigned *>(X + ra * kIn + c)) : 0u;
    xa[kk][1] = vb ? __ldg(reinterpret_cast<const unsigned *>(X + rb * kIn + c)) : 0u;
    xa[kk][2] = va ? __ldg(reinterpret_cast<const unsigned *>(X + ra * kIn + c + 8)) : 0u;
    xa[kk][3] = vb ? __ldg(reinterpret_cast<const unsigned *>(X + rb * kIn + c + 8)) : 0u;
  }
  // layer 1 -> relu -> BF16 A fragments of layer 2
  uint32_t ha[4][4];
#pragma unroll
  for (int jp = 0; jp < 4; jp++) {
    float h[2][4];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int j = 2 * jp + q, c = 8 * j + 2 * t;
      h[q][0] = s.b1[c], h[q][1] = s.b1[c + 1], h[q][2] = s.b1[c], h[q][3] = s.b1[c + 1];
#pragma unroll
      for (int kk = 0; kk < 2; kk++) {
        const bf16 *wr = s.w1 + (8 * j + g) * kLd1 + kk * 16 + 2 * t;
        mma(h[q], xa[kk], ld32(wr), ld32(wr + 8));
      }
#pragma unroll
      for (int e = 0; e < 4; e++)
        h[q][e] = fmaxf(h[q][e], 0.f);
    }
    ha[jp][0] = pack2(h[0][0], h[0][1]);
    ha[jp][1] = pack2(h[0][2], h[0][3]);
    ha[jp][2] = pack2(h[1][0], h[1][1]);
    ha[jp][3] = pack2(h[1][2], h[1][3]);
  }
  // layer 2 (pre-activations), then layer 3 on the FP32 cores
  float h2[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int c = 8 * j + 2 * t;
    h2[j][0] = s.b2[c], h2[j][1] = s.b2[c + 1], h2[j][2] = s.b2[c], h2[j][3] = s.b2[c + 1];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const bf16 *wr = s.w2 + (8 * j + g) * kLd2 + kk * 16 + 2 * t;
      mma(h2[j], ha[kk], ld32(wr), ld32(wr + 8));
    }
  }
  float ya[kOut], yb[kOut];
#pragma unroll
  for (int o = 0; o < kOut; o++) {
    float pa = 0.f, pb = 0.f;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = 8 * j + 2 * t;
      pa = fmaf(fmaxf(h2[j][0], 0.f), s.w3[o * kH + c], pa);
      pa = fmaf(fmaxf(h2[j][1], 0.f), s.w3[o * kH + c + 1], pa);
      pb = fmaf(fmaxf(h2[j][2], 0.f), s.w3[o * kH + c], pb);
      pb = fmaf(fmaxf(h2[j][3], 0.f), s.w3[o * kH + c + 1], pb);
    }
    pa += __shfl_xor_sync(0xffffffffu, pa, 1);
    pa += __shfl_xor_sync(0xffffffffu, pa, 2);
    pb += __shfl_xor_sync(0xffffffffu, pb, 1);
    pb += __shfl_xor_sync(0xffffffffu, pb, 2);
    ya[o] = pa + s.b3[o];
    yb[o] = pb + s.b3[o];
  }
  if constexpr (!TRAIN) {
    if (t == 0) {
      if (va)
        Y[ra] = make_float2(ya[0], ya[1]);
      if (vb)
        Y[rb] = make_float2(yb[0], yb[1]);
    }
    return;
  } else {
    // dL/dy for L = sum_rows sum_o w_o (y_o - t_o)^2 * scale
    float dya[kOut] = {0.f, 0.f}, dyb[kOut] = {0.f, 0.f}, loss = 0.f;
    if (va) {
      const float2 tt = T[ra], ww = Wt ? Wt[ra] : make_float2(1.f, 1.f);
      const float e0 = ya[0] - tt.x, e1 = ya[1] - tt.y;
      dya[0] = 2.f * scale * ww.x * e0;
      dya[1] = 2.f * scale * ww.y * e1;
      loss += scale * (ww.x * e0 * e0 + ww.y * e1 * e1);
    }
    if (vb) {
      const float2 tt = T[rb], ww = Wt ? Wt[rb] : make_float2(1.f, 1.f);
      const float e0 = yb[0] - tt.x, e1 = yb[1] - tt.y;
      dyb[0] = 2.f * scale * ww.x * e0;
      dyb[1] = 2.f * scale * ww.y * e1;
      loss += scale * (ww.x * e0 * e0 + ww.y * e1 * e1);
    }
    float *red = s.red[w];
    // db3, loss: every t-lane holds the same values; reduce over rows (g)
    {
      const float l = sum_g(t == 0 ? loss : 0.f);
      const float d0 = sum_g(t == 0 ? dya[0] + dyb[0] : 0.f);
      const float d1 = sum_g(t == 0 ? dya[1] + dyb[1] : 0.f);
      if (lane == 0) {
        red[2 * kH + kOut * kH + 0] += d0;
        red[2 * kH + kOut * kH + 1] += d1;
        red[2 * kH + kOut * kH + kOut] += l;
      }
    }
    // dW3 = dy^T relu(h2); dH2 = (dy W3) * [h2 > 0]; db2
    uint32_t da[4][4];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = 8 * j + 2 * t;
      float d[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int cc = c + (e & 1);
        const float dy0 = e < 2 ? dya[0] : dyb[0], dy1 = e < 2 ? dya[1] : dyb[1];
        d[e] = h2[j][e] > 0.f ? fmaf(dy0, s.w3[cc], dy1 * s.w3[kH + cc]) : 0.f;
      }
#pragma unroll
      for (int e2 = 0; e2 < 2; e2++) {
        const int cc = c + e2;
        const float r0v = fmaxf(h2[j][e2], 0.f), r1v = fmaxf(h2[j][e2 + 2], 0.f);
        const float w30 = sum_g(fmaf(dya[0], r0v, dyb[0] * r1v));
        const float w31 = sum_g(fmaf(dya[1], r0v, dyb[1] * r1v));
        const float b2s = sum_g(d[e2] + d[e2 + 2]);
        if (g == 0) {
          red[kH + cc] += b2s;
          red[2 * kH + cc] += w30;
          red[2 * kH + kH + cc] += w31;
        }
      }
      const uint32_t p01 = pack2(d[0], d[1]), p23 = pack2(d[2], d[3]);
      da[j >> 1][(j & 1) * 2 + 0] = p01;
      da[j >> 1][(j & 1) * 2 + 1] = p23;
      // stage dH2^T (BF16)
      const int la = lr0 + g, lb = lr0 + g + 8;
      st2(s.d2t + c * kLdT + la, s.d2t + (c + 1) * kLdT + la, p01);
      st2(s.d2t + c * kLdT + lb, s.d2t + (c + 1) * kLdT + lb, p23);
    }
    // dH1 = (dH2 W2) * [h1 > 0]; db1; stage dH1^T and H1^T, X^T
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = 8 * j + 2 * t;
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const bf16 *wr = s.w2t + (8 * j + g) * kLd2 + kk * 16 + 2 * t;
        mma(d, da[kk], ld32(wr), ld32(wr + 8));
      }
      // h1 of these positions: A fragment of layer-2 k-step j/2, half j&1
      const uint32_t hv01 = ha[j >> 1][(j & 1) * 2 + 0], hv23 = ha[j >> 1][(j & 1) * 2 + 1];
      if (!(lo_f(hv01) > 0.f)) d[0] = 0.f;
      if (!(hi_f(hv01) > 0.f)) d[1] = 0.f;
      if (!(lo_f(hv23) > 0.f)) d[2] = 0.f;
      if (!(hi_f(hv23) > 0.f)) d[3] = 0.f;
#pragma unroll
      for (int e2 = 0; e2 < 2; e2++) {
        const float b1s = sum_g(d[e2] + d[e2 + 2]);
        if (g == 0)
          red[c + e2] += b1s;
      }
      const int la = lr0 + g, lb = lr0 + g + 8;
      const uint32_t p01 = pack2(d[0], d[1]), p23 = pack2(d[2], d[3]);
      st2(s.d1t + c * kLdT + la, s.d1t + (c + 1) * kLdT + la, p01);
      st2(s.d1t + c * kLdT + lb, s.d1t + (c + 1) * kLdT + lb, p23);
      st2(s.h1t + c * kLdT + la, s.h1t + (c + 1) * kLdT + la, hv01);
      st2(s.h1t + c * kLdT + lb, s.h1t + (c + 1) * kLdT + lb, hv23);
    }
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const int c = kk * 16 + 2 * t;
      const int la = lr0 + g, lb = lr0 + g + 8;
      st2(s.xt + c * kLdT + la, s.xt + (c + 1) * kLdT + la, xa[kk][0]);
      st2(s.xt + c * kLdT + lb, s.xt + (c + 1) * kLdT + lb, xa[kk][1]);
      st2(s.xt + (c + 8) * kLdT + la, s.xt + (c + 9) * kLdT + la, xa[kk][2]);
      st2(s.xt + (c + 8) * kLdT + lb, s.xt + (c + 9) * kLdT + lb, xa[kk][3]);
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    mlp_forward_kernel(const float *__restrict__ prm, const bf16 *__restrict__ X,
                       float2 *__restrict__ Y, long long M)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &s = *reinterpret_cast<Smem *>(smem_raw);
  load_weights(s, prm, false);
  __syncthreads();
  const int w = threadIdx.x >> 5;
  for (long long r0 = (long long)blockIdx.x * kBlockRows; r0 < M;
       r0 += (long long)gridDim.x * kBlockRows)
    for (int mt = 0; mt < 2; mt++)
      tile<false>(s, X, nullptr, nullptr, Y, r0 + 32 * w + 16 * mt, M, 0.f, 0);
}

// Loss and gradient partials of one CTA (part[blockIdx.x][kPart]).
__global__ void __launch_bounds__(kThreads)
    mlp_train_kernel(const float *__restrict__ prm, const bf16 *__restrict__ X,
                     const float2 *__restrict__ T, const float2 *__restrict__ Wt, long long M,
                     float scale, float *__restrict__ part)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &s = *reinterpret_cast<Smem *>(smem_raw);
  load_weights(s, prm, true);
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, w = threadIdx.x >> 5;
  float acc2[8][4], acc1[4][4];
#pragma unroll
  for (int j = 0; j < 8; j++)
#pragma unroll
    for (int e = 0; e < 4; e++)
      acc2[j][e] = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int e = 0; e < 4; e++)
      acc1[j][e] = 0.f;
  for (long long r0 = (long long)blockIdx.x * kBlockRows; r0 < M;
       r0 += (long long)gridDim.x * kBlockRows) {
    for (int mt = 0; mt < 2; mt++)
      tile<true>(s, X, T, Wt, nullptr, r0 + 32 * w + 16 * mt, M, scale, 32 * w + 16 * mt);
    __syncthreads();
    // dW2 += dH2^T H1 (warp w: output rows 16w..16w+15), dW1 += dH1^T X
#pragma unroll
    for (int kk = 0; kk < kBlockRows / 16; kk++) {
      uint32_t a2[4], a1[4];
      const bf16 *p2 = s.d2t + (16 * w + g) * kLdT + kk * 16 + 2 * t;
      a2[0] = ld32(p2), a2[1] = ld32(p2 + 8 * kLdT), a2[2] = ld32(p2 + 8),
      a2[3] = ld32(p2 + 8 * kLdT + 8);
      const bf16 *p1 = s.d1t + (16 * w + g) * kLdT + kk * 16 + 2 * t;
      a1[0] = ld32(p1), a1[1] = ld32(p1 + 8 * kLdT), a1[2] = ld32(p1 + 8),
      a1[3] = ld32(p1 + 8 * kLdT + 8);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const bf16 *b = s.h1t + (8 * j + g) * kLdT + kk * 16 + 2 * t;
        mma(acc2[j], a2, ld32(b), ld32(b + 8));
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const bf16 *b = s.xt + (8 * j + g) * kLdT + kk * 16 + 2 * t;
        mma(acc1[j], a1, ld32(b), ld32(b + 8));
      }
    }
    __syncthreads();
  }
  float *out = part + (size_t)blockIdx.x * kPart;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int c = 8 * j + 2 * t, ra = 16 * w + g;
    out[kW2 + ra * kH + c] = acc2[j][0];
    out[kW2 + ra * kH + c + 1] = acc2[j][1];
    out[kW2 + (ra + 8) * kH + c] = acc2[j][2];
    out[kW2 + (ra + 8) * kH + c + 1] = acc2[j][3];
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int c = 8 * j + 2 * t, ra = 16 * w + g;
    out[kW1 + ra * kIn + c] = acc1[j][0];
    out[kW1 + ra * kIn + c + 1] = acc1[j][1];
    out[kW1 + (ra + 8) * kIn + c] = acc1[j][2];
    out[kW1 + (ra + 8) * kIn + c + 1] = acc1[j][3];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRed; i += blockDim.x) {
    float v = 0.f;
    for (int ww = 0; ww < kWarps; ww++)
      v += s.red[ww][i];
    int dst;
    if (i < kH)
      dst = kB1 + i;
    else if (i < 2 * kH)
      dst = kB2 + (i - kH);
    else if (i < 2 * kH + kOut * kH)
      dst = kW3 + (i - 2 * kH);
    else if (i < 2 * kH + kOut * kH + kOut)
      dst = kB3 + (i - 2 * kH - kOut * kH);
    else
      dst = kParams;  // loss
    out[dst] = v;
  }
}

// grad[p] = sum over CTAs of part[cta][p], in CTA order.
__global__ void mlp_reduce_kernel(const float *__restrict__ part, int n_cta,
                                  float *__restrict__ grad)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kPart)
    return;
  float v = 0.f;
  for (int c = 0; c < n_cta; c++)
    v += part[(size_t)c * kPart + p];
  grad[p] = v;
}

__global__ void mlp_adam_kernel(float *__restrict__ prm, float *__restrict__ m,
                                float *__restrict__ v, const float *__restrict__ grad, float lr,
                                float b1, float b2, float eps, float c1, float c2, float wd)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams)
    return;
  const float gr = grad[p] + wd * prm[p];
  const float mm = b1 * m[p] + (1.f - b1) * gr;
  const float vv = b2 * v[p] + (1.f - b2) * gr * gr;
  m[p] = mm;
  v[p] = vv;
  prm[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

// ---- per-row features ------------------------------------------------------

constexpr int kFeat = 32;

// Feature row of matrix row i (CSR, FP64 values):
//  0: log(a_ii) / 8             1: sum_{j != i} |a_ij| / a_ii
//  2..27: |a_ij| / a_ii of the 26 neighbours (dz, dy, dx) in {-1,0,1}^3 \ 0,
//         lexicographic, located through the grid dimensions (nx, ny); with
//         nx = 0 the off-diagonal entries in column order
//  28: 1 for a row with more than 7 entries (27-point stencil), else 0
//  29: log(max |a_ij| / min |a_ij|) / 8 over the off-diagonal entries
//  30: row length / 27          31: 1
__global__ void row_features_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                    const double *__restrict__ v, int nx, int ny,
                                    bf16 *__restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int e0 = rp[i], e1 = rp[i + 1];
  double aii = 0.0, off = 0.0, mx = 0.0, mn = 0.0;
  int n_off = 0;
  for (int e = e0; e < e1; e++) {
    const double a = fabs(v[e]);
    if (ci[e] == i) {
      aii = v[e];
    } else if (a > 0.0) {
      off += a;
      mx = n_off ? fmax(mx, a) : a;
      mn = n_off ? fmin(mn, a) : a;
      n_off++;
    }
  }
  const double d = aii > 0.0 ? aii : 1.0;
  float f[kFeat];
  for (int k = 0; k < kFeat; k++)
    f[k] = 0.f;
  f[0] = (float)(log(d) / 8.0);
  f[1] = (float)(off / d);
  const long long plane = (long long)nx * ny;
  int pos = 0;
  for (int e = e0; e < e1; e++) {
    if (ci[e] == i)
      continue;
    int k = -1;
    if (nx > 0) {
      const long long dd = (long long)ci[e] - i;
      const long long dz = (dd + plane + nx + 1) >= 0 ? (dd + plane + nx + 1) / plane - 1 : -2;
      const long long rem = dd - dz * plane;
      const long long dy = (rem + nx + 1) >= 0 ? (rem + nx + 1) / nx - 1 : -2;
      const long long dx = rem - dy * nx;
      if (dz >= -1 && dz <= 1 && dy >= -1 && dy <= 1 && dx >= -1 && dx <= 1) {
        const int q = (int)((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
        k = q < 13 ? q : q - 1;
      }
    } else if (pos < 26) {
      k = pos;
    }
    pos++;
    if (k >= 0)
      f[2 + k] = (float)(fabs(v[e]) / d);
  }
  f[28] = (e1 - e0) > 7 ? 1.f : 0.f;
  f[29] = n_off >= 2 ? (float)(log(mx / mn) / 8.0) : 0.f;
  f[30] = (float)(e1 - e0) / 27.f;
  f[31] = 1.f;
  uint32_t *o = reinterpret_cast<uint32_t *>(out + (size_t)i * kFeat);
  for (int k = 0; k < kFeat; k += 2)
    o[k / 2] = pack2(f[k], f[k + 1]);
}

int train_grid(long long M)
{
  const long long blocks = (M + kBlockRows - 1) / kBlockRows;
  return (int)std::max(1LL, std::min(blocks, (long long)device_sm_count() * 2));
}

int fwd_grid(long long M)
{
  const long long blocks = (M + kBlockRows - 1) / kBlockRows;
  return (int)std::max(1LL, std::min(blocks, (long long)device_sm_count() * 4));
}

int set_smem_attrs()
{
  static bool done = false;
  if (done)
    return ISPM_OK;
  ISPM_CUDA_TRY(cudaFuncSetAttribute(mlp_forward_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(Smem)));
  ISPM_CUDA_TRY(cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(Smem)));
  done = true;
  return ISPM_OK;
}

}  // namespace
}  // namespace ispm

struct ispm_mlp {
  float *prm = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *part = nullptr;
  int part_cta = 0;
  int step = 0;
  ~ispm_mlp()
  {
    for (float *p : {prm, m, v, grad, part})
      if (p)
        cudaFree(p);
  }
};

using namespace ispm;

extern "C" {

int ispm_mlp_n_params(void) { return kParams; }

int ispm_mlp_create(const float *init_params, ispm_mlp **out)
{
  clear_error();
  if (!out || !init_params)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  *out = nullptr;
  std::unique_ptr<ispm_mlp> h(new (std::nothrow) ispm_mlp);
  if (!h)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  for (float **pp : {&h->prm, &h->m, &h->v, &h->grad}) {
    if (cudaMalloc(pp, sizeof(float) * kPart) != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "cudaMalloc");
    }
    ISPM_CUDA_TRY(cudaMemset(*pp, 0, sizeof(float) * kPart));
  }
  ISPM_CUDA_TRY(cudaMemcpy(h->prm, init_params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  if (int e = set_smem_attrs())
    return e;
  *out = h.release();
  return ISPM_OK;
}

int ispm_mlp_get_params(const ispm_mlp *m, float *host_out)
{
  clear_error();
  if (!m || !host_out)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  ISPM_CUDA_TRY(cudaMemcpy(host_out, m->prm, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  return ISPM_OK;
}

int ispm_mlp_set_params(ispm_mlp *m, const float *host_in)
{
  clear_error();
  if (!m || !host_in)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  ISPM_CUDA_TRY(cudaMemcpy(m->prm, host_in, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  ISPM_CUDA_TRY(cudaMemset(m->m, 0, sizeof(float) * kPart));
  ISPM_CUDA_TRY(cudaMemset(m->v, 0, sizeof(float) * kPart));
  m->step = 0;
  return ISPM_OK;
}

int ispm_mlp_forward(const ispm_mlp *m, long long n_rows, const void *feat_bf16, float *out,
                     void *stream)
{
  clear_error();
  if (!m || n_rows < 0 || (n_rows && (!feat_bf16 || !out)))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (!aligned(feat_bf16, 4) || !aligned(out, 8))
    return fail(ISPM_ERR_INVALID, "features must be 4-byte, outputs 8-byte aligned");
  if (n_rows == 0)
    return ISPM_OK;
  if (int e = set_smem_attrs())
    return e;
  // the forward pass uses only the weight part of the shared-memory layout
  mlp_forward_kernel<<<fwd_grid(n_rows), kThreads, offsetof(Smem, red), (cudaStream_t)stream>>>(
      m->prm, (const bf16 *)feat_bf16, (float2 *)out, n_rows);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  return ISPM_OK;
}

int ispm_mlp_loss_grad(ispm_mlp *m, long long n_rows, const void *feat_bf16,
                       const float *target, const float *weight, float *grad_out,
                       double *loss_out, void *stream)
{
  clear_error();
  if (!m || n_rows <= 0 || !feat_bf16 || !target)
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (!aligned(feat_bf16, 4) || !aligned(target, 8) || (weight && !aligned(weight, 8)))
    return fail(ISPM_ERR_INVALID, "misaligned features / targets / weights");
  if (int e = set_smem_attrs())
    return e;
  const int grid = train_grid(n_rows);
  if (grid > m->part_cta) {
    if (m->part)
      cudaFree(m->part);
    m->part = nullptr;
    if (cudaMalloc(&m->part, sizeof(float) * kPart * grid) != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "cudaMalloc");
    }
    m->part_cta = grid;
  }
  cudaStream_t s = (cudaStream_t)stream;
  mlp_train_kernel<<<grid, kThreads, sizeof(Smem), s>>>(
      m->prm, (const bf16 *)feat_bf16, (const float2 *)target, (const float2 *)weight, n_rows,
      1.0f / (float)n_rows, m->part);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  mlp_reduce_kernel<<<(kPart + 255) / 256, 256, 0, s>>>(m->part, grid, m->grad);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  if (grad_out)
    ISPM_CUDA_TRY(cudaMemcpyAsync(grad_out, m->grad, sizeof(float) * kParams,
                                  cudaMemcpyDeviceToHost, s));
  if (loss_out) {
    float l = 0.f;
    ISPM_CUDA_TRY(cudaMemcpyAsync(&l, m->grad + kParams, sizeof(float), cudaMemcpyDeviceToHost, s));
    ISPM_CUDA_TRY(cudaStreamSynchronize(s));
    *loss_out = l;
  } else if (grad_out) {
    ISPM_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return ISPM_OK;
}

int ispm_mlp_adam_step(ispm_mlp *m, float lr, float beta1, float beta2, float eps,
                       float weight_decay, void *stream)
{
  clear_error();
  if (!m || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1))
    return fail(ISPM_ERR_INVALID, "bad Adam parameters");
  m->step++;
  const float c1 = 1.f - std::pow(beta1, (float)m->step);
  const float c2 = 1.f - std::pow(beta2, (float)m->step);
  mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      m->prm, m->m, m->v, m->grad, lr, beta1, beta2, eps, c1, c2, weight_decay);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  return ISPM_OK;
}

void ispm_mlp_free(ispm_mlp *m) { delete m; }

int ispm_row_features(int n, const int *row_ptr, const int *cols, const double *vals, int nx,
                      int ny, void *out_bf16, void *stream)
{
  clear_error();
  if (n < 0 || (n && (!row_ptr || !cols || !vals || !out_bf16)) || nx < 0 || ny < 0 ||
      (nx > 0) != (ny > 0))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (!aligned(out_bf16, 4))
    return fail(ISPM_ERR_INVALID, "features must be 4-byte aligned");
  if (n == 0)
    return ISPM_OK;
  row_features_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      n, row_ptr, cols, vals, nx, ny, (bf16 *)out_bf16);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  return ISPM_OK;
}

}  // extern "C"

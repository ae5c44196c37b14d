// fno.cu -- forward and backward kernels of the Fourier neural operator used
// as the coarse propagator of the parareal driver, plus the grid transfers
// between the solver grid and the FNO grid.  BF16 weights, FP32 activations
// and FP32 accumulation; every reduction runs in a fixed order, so training
// is run-to-run reproducible.
//
// A Fourier layer is  v' = act(W v + b + K v),  K v = F^-1 (R . F v)|modes,
// where F keeps mx x my x mz modes (kx in [0, mx), ky, kz in the lowest
// |k|).  The truncated transforms are dense contractions with small DFT
// matrices (he4_fno_contract), applied axis by axis; their adjoints are the
// same contractions with the conjugate-transposed matrices and the real /
// complex flags swapped, which is how the backward pass runs them.
#include <cuda_bf16.h>

#include <stdlib.h>

#include <algorithm>

#include "../../include/he4_fno.h"
#include "common.cuh"
#include "reduce.cuh"

namespace he4 {
namespace fno {

constexpr int kThreads = 256;

static inline unsigned blocks_for(int64_t n, int t = kThreads) {
  return (unsigned)std::min<int64_t>((n + t - 1) / t, (int64_t)148 * 32);
}

__device__ __forceinline__ float bf(uint16_t u) { return __uint_as_float((uint32_t)u << 16); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// ---------------------------------------------------------------------------
// axis contraction  y[o][k][r] = sum_j A[k][j] x[o][j][r]
// ---------------------------------------------------------------------------
template <bool IN_REAL, bool OUT_REAL>
__global__ void k_contract(const void *__restrict__ xv, void *__restrict__ yv, const float2 *__restrict__ A,
                           int64_t outer, int J, int K, int64_t inner, int accumulate) {
  extern __shared__ float2 sA[];
  for (int t = threadIdx.x; t < J * K; t += blockDim.x) sA[t] = A[t];
  __syncthreads();
  const int64_t total = outer * K * inner;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx % inner;
    const int64_t q = idx / inner;
    const int k = (int)(q % K);
    const int64_t o = q / K;
    float re = 0.f, im = 0.f;
    const int64_t base = o * J * inner + r;
    for (int j = 0; j < J; j++) {
      const float2 a = sA[k * J + j];
      if (IN_REAL) {
        const float x = reinterpret_cast<const float *>(xv)[base + (int64_t)j * inner];
        re += a.x * x;
        im += a.y * x;
      } else {
        const float2 x = reinterpret_cast<const float2 *>(xv)[base + (int64_t)j * inner];
        re += a.x * x.x - a.y * x.y;
        im += a.x * x.y + a.y * x.x;
      }
    }
    const int64_t oi = (o * K + k) * inner + r;
    if (OUT_REAL) {
      float *y = reinterpret_cast<float *>(yv);
      y[oi] = accumulate ? y[oi] + re : re;
    } else {
      float2 *y = reinterpret_cast<float2 *>(yv);
      if (accumulate) {
        const float2 p = y[oi];
        y[oi] = make_float2(p.x + re, p.y + im);
      } else {
        y[oi] = make_float2(re, im);
      }
    }
  }
}

// The same contraction with each thread holding KC consecutive output modes
// k0 .. k0+KC-1 of one (o, r): every input x[o][j][r] is loaded once per KC
// outputs instead of once per output, and the KC rows of A it multiplies are
// read from shared memory by the whole warp at once.  Each output sums over
// j in the same order as k_contract.
template <bool IN_REAL, bool OUT_REAL, int KC>
__global__ void __launch_bounds__(256) k_contract_kc(const void *__restrict__ xv, void *__restrict__ yv,
                                                     const float2 *__restrict__ A, int64_t outer, int J, int K,
                                                     int64_t inner, int accumulate) {
  extern __shared__ float2 sA[];
  for (int t = threadIdx.x; t < J * K; t += blockDim.x) sA[t] = A[t];
  __syncthreads();
  const int nkc = (K + KC - 1) / KC;
  const int64_t total = outer * nkc * inner;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx % inner;
    const int64_t q = idx / inner;
    const int k0 = (int)(q % nkc) * KC;
    const int64_t o = q / nkc;
    float re[KC], im[KC];
#pragma unroll
    for (int kk = 0; kk < KC; kk++) re[kk] = im[kk] = 0.f;
    const int64_t base = o * J * inner + r;
#pragma unroll 4
    for (int j = 0; j < J; j++) {
      float xr, xi = 0.f;
      if (IN_REAL) {
        xr = reinterpret_cast<const float *>(xv)[base + (int64_t)j * inner];
      } else {
        const float2 x = reinterpret_cast<const float2 *>(xv)[base + (int64_t)j * inner];
        xr = x.x;
        xi = x.y;
      }
#pragma unroll
      for (int kk = 0; kk < KC; kk++) {
        const float2 a = sA[min(k0 + kk, K - 1) * J + j];
        if (IN_REAL) {
          re[kk] += a.x * xr;
          im[kk] += a.y * xr;
        } else {
          re[kk] += a.x * xr - a.y * xi;
          im[kk] += a.x * xi + a.y * xr;
        }
      }
    }
#pragma unroll
    for (int kk = 0; kk < KC; kk++) {
      const int k = k0 + kk;
      if (k >= K) break;
      const int64_t oi = (o * K + k) * inner + r;
      if (OUT_REAL) {
        float *y = reinterpret_cast<float *>(yv);
        y[oi] = accumulate ? y[oi] + re[kk] : re[kk];
      } else {
        float2 *y = reinterpret_cast<float2 *>(yv);
        if (accumulate) {
          const float2 p = y[oi];
          y[oi] = make_float2(p.x + re[kk], p.y + im[kk]);
        } else {
          y[oi] = make_float2(re[kk], im[kk]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// spectral channel mixing
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 load_bf2(const uint16_t *R, int64_t e) {
  const uint32_t u = reinterpret_cast<const uint32_t *>(R)[e];
  return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}

__global__ void k_mix(const float2 *__restrict__ x, const uint16_t *__restrict__ R, float2 *__restrict__ y, int B,
                      int ci, int co, int M) {
  const int64_t total = (int64_t)B * co * M;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M);
    const int o = (int)((idx / M) % co);
    const int b = (int)(idx / ((int64_t)M * co));
    float re = 0.f, im = 0.f;
    for (int i = 0; i < ci; i++) {
      const float2 v = x[((int64_t)b * ci + i) * M + m];
      const float2 w = load_bf2(R, ((int64_t)i * co + o) * M + m);
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
    }
    y[idx] = make_float2(re, im);
  }
}

__global__ void k_mix_gx(const float2 *gy, const uint16_t *__restrict__ R, float2 *gx,
                         int B, int ci, int co, int M) {
  const int64_t total = (int64_t)B * ci * M;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M);
    const int i = (int)((idx / M) % ci);
    const int b = (int)(idx / ((int64_t)M * ci));
    float re = 0.f, im = 0.f;
    for (int o = 0; o < co; o++) {
      const float2 g = gy[((int64_t)b * co + o) * M + m];
      const float2 w = load_bf2(R, ((int64_t)i * co + o) * M + m);
      // g * conj(w)
      re += g.x * w.x + g.y * w.y;
      im += g.y * w.x - g.x * w.y;
    }
    gx[idx] = make_float2(re, im);
  }
}

__global__ void k_mix_gR(const float2 *__restrict__ gy, const float2 *__restrict__ x, float2 *__restrict__ gR,
                         int B, int ci, int co, int M) {
  const int64_t total = (int64_t)ci * co * M;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M);
    const int o = (int)((idx / M) % co);
    const int i = (int)(idx / ((int64_t)M * co));
    float re = 0.f, im = 0.f;
    for (int b = 0; b < B; b++) {
      const float2 v = x[((int64_t)b * ci + i) * M + m];
      const float2 g = gy[((int64_t)b * co + o) * M + m];
      // conj(v) * g
      re += v.x * g.x + v.y * g.y;
      im += v.x * g.y - v.y * g.x;
    }
    gR[idx] = make_float2(re, im);
  }
}

// ---------------------------------------------------------------------------
// pointwise layers
// ---------------------------------------------------------------------------
constexpr int kMaxCh = 64;

template <int CI>
__global__ void k_pointwise(const float *__restrict__ x, const uint16_t *__restrict__ W,
                            const float *__restrict__ bias, const float *__restrict__ add, float *__restrict__ pre,
                            float *__restrict__ y, int B, int co, int64_t P, int act) {
  __shared__ float sW[kMaxCh * kMaxCh];
  __shared__ float sb[kMaxCh];
  for (int t = threadIdx.x; t < co * CI; t += blockDim.x) sW[t] = bf(W[t]);
  for (int t = threadIdx.x; t < co; t += blockDim.x) sb[t] = bias ? bias[t] : 0.f;
  __syncthreads();
  const int64_t total = (int64_t)B * P;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = idx / P, p = idx - b * P;
    float xv[CI];
#pragma unroll
    for (int i = 0; i < CI; i++) xv[i] = x[(b * CI + i) * P + p];
    for (int o = 0; o < co; o++) {
      float s = sb[o];
#pragma unroll
      for (int i = 0; i < CI; i++) s += sW[o * CI + i] * xv[i];
      const int64_t oi = (b * co + o) * P + p;
      if (add) s += add[oi];
      if (pre) pre[oi] = s;
      y[oi] = act ? gelu(s) : s;
    }
  }
}

// ---------------------------------------------------------------------------
// pointwise layers on the tensor cores: y = W x (+ bias, + add, act) for
// channel counts that are multiples of 16, as BF16 mma.sync (m16n8k16, FP32
// accumulate).  The weights are BF16 already; each FP32 activation is split
// into three BF16 pieces x = x0 + x1 + x2 (x0 = bf16(x), x1 = bf16(x - x0),
// x2 = bf16(x - x0 - x1): 24 significant bits), and W x0 + W x1 + W x2
// accumulate in FP32, so the layer keeps FP32 accuracy while every product
// runs on the tensor cores.  TRANS: A = W^T (the input gradient W^T g).
// A CTA of 4 warps takes tiles of 64 points; warp w owns points 16w..16w+15
// of the tile (two n8 tiles) and every output channel (MC/16 m16 tiles).
// ---------------------------------------------------------------------------
constexpr int kTcPts = 64;

__device__ __forceinline__ uint32_t pack_bf2(float lo, float hi) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// x = x0 + x1 + x2 in BF16: 24 significant bits of an FP32 value
__device__ __forceinline__ void split3_bf16(float v, uint16_t &p0, uint16_t &p1, uint16_t &p2) {
  const __nv_bfloat16 v0 = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(v0);
  const __nv_bfloat16 v1 = __float2bfloat16_rn(r1);
  const __nv_bfloat16 v2 = __float2bfloat16_rn(r1 - __bfloat162float(v1));
  p0 = __bfloat16_as_ushort(v0);
  p1 = __bfloat16_as_ushort(v1);
  p2 = __bfloat16_as_ushort(v2);
}

template <int KC, int MC, bool TRANS>
__global__ void __launch_bounds__(128) k_pointwise_tc(const float *__restrict__ x, const uint16_t *__restrict__ W,
                                                      const float *__restrict__ bias, const float *__restrict__ add,
                                                      float *__restrict__ pre, float *__restrict__ y, int64_t P,
                                                      int64_t ntiles, int act) {
  constexpr int KS = KC + 8;  // padded row of the B pieces (bank-conflict free fragment loads)
  __shared__ __align__(16) uint16_t xs[3][kTcPts][KS];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  // A fragments of the whole weight matrix (MC/16 x KC/16 tiles), in registers
  uint32_t afr[MC / 16][KC / 16][4];
#pragma unroll
  for (int mt = 0; mt < MC / 16; mt++)
#pragma unroll
    for (int kt = 0; kt < KC / 16; kt++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int m = mt * 16 + g + ((q & 1) ? 8 : 0), k = kt * 16 + 2 * t + ((q & 2) ? 8 : 0);
        // A[m][k] = W[m][k] (W is [MC][KC]) or W^T: W[k][m] (W is [KC][MC])
        const uint16_t lo = TRANS ? W[(size_t)k * MC + m] : W[(size_t)m * KC + k];
        const uint16_t hi = TRANS ? W[(size_t)(k + 1) * MC + m] : W[(size_t)m * KC + k + 1];
        afr[mt][kt][q] = (uint32_t)lo | ((uint32_t)hi << 16);
      }
  const int64_t tiles_per_b = P / kTcPts;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t b = tile / tiles_per_b, p0 = (tile - b * tiles_per_b) * kTcPts;
    __syncthreads();
    // the tile's inputs as three BF16 pieces, point-major
    for (int e = tid; e < KC * kTcPts; e += 128) {
      const int k = e / kTcPts, p = e - k * kTcPts;
      const float v = x[(b * KC + k) * P + p0 + p];
      const __nv_bfloat16 v0 = __float2bfloat16_rn(v);
      const float r1 = v - __bfloat162float(v0);
      const __nv_bfloat16 v1 = __float2bfloat16_rn(r1);
      const __nv_bfloat16 v2 = __float2bfloat16_rn(r1 - __bfloat162float(v1));
      xs[0][p][k] = __bfloat16_as_ushort(v0);
      xs[1][p][k] = __bfloat16_as_ushort(v1);
      xs[2][p][k] = __bfloat16_as_ushort(v2);
    }
    __syncthreads();
    float acc[MC / 16][2][4];
#pragma unroll
    for (int mt = 0; mt < MC / 16; mt++)
#pragma unroll
      for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[mt][nt][q] = 0.f;
#pragma unroll
    for (int pc = 2; pc >= 0; pc--)  // smallest pieces first
#pragma unroll
      for (int kt = 0; kt < KC / 16; kt++)
#pragma unroll
        for (int nt = 0; nt < 2; nt++) {
          const uint16_t *row = &xs[pc][warp * 16 + nt * 8 + g][kt * 16 + 2 * t];
          const uint32_t b0 = *reinterpret_cast<const uint32_t *>(row);
          const uint32_t b1 = *reinterpret_cast<const uint32_t *>(row + 8);
#pragma unroll
          for (int mt = 0; mt < MC / 16; mt++) mma_bf16_16816(acc[mt][nt], afr[mt][kt], b0, b1);
        }
    // epilogue: bias, skip term, pre-activation, activation
#pragma unroll
    for (int mt = 0; mt < MC / 16; mt++)
#pragma unroll
      for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
          const int o = mt * 16 + g + hf * 8;
          const int64_t pp = p0 + warp * 16 + nt * 8 + 2 * t;
          const int64_t oi = (b * MC + o) * P + pp;
          float s0 = acc[mt][nt][2 * hf], s1 = acc[mt][nt][2 * hf + 1];
          if (bias) {
            const float bb = bias[o];
            s0 += bb;
            s1 += bb;
          }
          if (add) {
            const float2 ad = *reinterpret_cast<const float2 *>(add + oi);
            s0 += ad.x;
            s1 += ad.y;
          }
          if (pre) *reinterpret_cast<float2 *>(pre + oi) = make_float2(s0, s1);
          *reinterpret_cast<float2 *>(y + oi) = act ? make_float2(gelu(s0), gelu(s1)) : make_float2(s0, s1);
        }
  }
}

// Weight and bias gradients on the tensor cores: gW = g x^T summed over the
// points (M = CO output channels, N = CI input channels, K = points), both
// operands FP32 split into three BF16 pieces and the six products of piece
// orders a + b <= 2 accumulated in FP32 (the dropped terms are below 2^-24
// of each product).  Each of kWgBlocks CTAs sums a fixed chunk of whole
// 64-point tiles and writes its partials in k_pointwise_wgrad's layout
// (pair o * (CI + 1) + i, the bias at i = CI), so the same fixed-order
// k_wgrad_finish completes both kernels.
template <int CI, int CO>
__global__ void __launch_bounds__(128) k_pointwise_wgrad_tc(const float *__restrict__ g, const float *__restrict__ x,
                                                            float *__restrict__ part, int64_t P, int64_t ntiles) {
  constexpr int TS = kTcPts + 8;  // padded point rows
  __shared__ __align__(16) uint16_t gs[3][CO][TS];
  __shared__ __align__(16) uint16_t xs[3][CI][TS];
  __shared__ float bpart_s[CO][kTcPts];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, t = lane & 3;
  constexpr int MT = CO / 16, NT = CI / 8, TILES = MT * NT, PER_WARP = (TILES + 3) / 4;
  float acc[PER_WARP][4];
#pragma unroll
  for (int q = 0; q < PER_WARP; q++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc[q][c] = 0.f;
  // bias gradient partials: thread tid stages point tid % 64 of channels
  // tid / 64 + 2i of g, and sums them over its tiles
  constexpr int GI = CO * kTcPts / 128, XI = CI * kTcPts / 128;
  float bpart[GI];
#pragma unroll
  for (int i = 0; i < GI; i++) bpart[i] = 0.f;
  const int64_t per = (ntiles + gridDim.x - 1) / gridDim.x;
  const int64_t t0 = blockIdx.x * per, t1 = (t0 + per < ntiles) ? t0 + per : ntiles;
  const int64_t tiles_per_b = P / kTcPts;
  const int pp = tid % kTcPts, c0 = tid / kTcPts;
  for (int64_t tile = t0; tile < t1; tile++) {
    const int64_t b = tile / tiles_per_b, p0 = (tile - b * tiles_per_b) * kTcPts;
    // this tile's values in registers before the barrier, so their loads
    // overlap the previous tile's products in other warps
    float gv[GI], xv[XI];
#pragma unroll
    for (int i = 0; i < GI; i++) gv[i] = g[(b * CO + c0 + 2 * i) * P + p0 + pp];
#pragma unroll
    for (int i = 0; i < XI; i++) xv[i] = x[(b * CI + c0 + 2 * i) * P + p0 + pp];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < GI; i++) {
      bpart[i] += gv[i];
      split3_bf16(gv[i], gs[0][c0 + 2 * i][pp], gs[1][c0 + 2 * i][pp], gs[2][c0 + 2 * i][pp]);
    }
#pragma unroll
    for (int i = 0; i < XI; i++) split3_bf16(xv[i], xs[0][c0 + 2 * i][pp], xs[1][c0 + 2 * i][pp], xs[2][c0 + 2 * i][pp]);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER_WARP; q++) {
      const int tl = warp * PER_WARP + q;
      if (tl >= TILES) break;
      const int mt = tl / NT, nt = tl % NT;
#pragma unroll
      for (int kt = 0; kt < kTcPts / 16; kt++)
#pragma unroll
        for (int pa = 2; pa >= 0; pa--)
#pragma unroll
          for (int pb = 2 - pa; pb >= 0; pb--) {
            const uint16_t *ar0 = &gs[pa][mt * 16 + gq][kt * 16 + 2 * t];
            const uint16_t *ar1 = &gs[pa][mt * 16 + gq + 8][kt * 16 + 2 * t];
            const uint32_t a[4] = {*reinterpret_cast<const uint32_t *>(ar0), *reinterpret_cast<const uint32_t *>(ar1),
                                   *reinterpret_cast<const uint32_t *>(ar0 + 8),
                                   *reinterpret_cast<const uint32_t *>(ar1 + 8)};
            const uint16_t *br = &xs[pb][nt * 8 + gq][kt * 16 + 2 * t];
            mma_bf16_16816(acc[q], a, *reinterpret_cast<const uint32_t *>(br),
                           *reinterpret_cast<const uint32_t *>(br + 8));
          }
    }
  }
  constexpr int npair = CO * (CI + 1);
  float *out = part + (int64_t)blockIdx.x * npair;
#pragma unroll
  for (int q = 0; q < PER_WARP; q++) {
    const int tl = warp * PER_WARP + q;
    if (tl >= TILES) break;
    const int mt = tl / NT, nt = tl % NT;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int o = mt * 16 + gq + ((c & 2) ? 8 : 0), i = nt * 8 + 2 * t + (c & 1);
      out[o * (CI + 1) + i] = acc[q][c];
    }
  }
  // bias: the 64 partials of each channel summed in point order
#pragma unroll
  for (int i = 0; i < GI; i++) bpart_s[c0 + 2 * i][pp] = bpart[i];
  __syncthreads();
  if (tid < CO) {
    float s = 0.f;
    for (int q = 0; q < kTcPts; q++) s += bpart_s[tid][q];
    out[tid * (CI + 1) + CI] = s;
  }
}

// The truncated transforms along x (the contiguous axis, inner = 1) as
// real GEMMs on the tensor cores: C[m][n] (+)= sum_k A[m][k] B[k][n] over
// the rows m of the activations.
//  - real in, complex out (Fx and the adjoint GxH): A = x [outer][J],
//    B[j][2k + c] = (Re, Im) of the DFT matrix entry (k, j); C is the
//    complex result [outer][K] as 2K interleaved floats;
//  - complex in, real out (Gx and FxH): A = x [outer][J] complex as 2J
//    floats, B[2j + c][k] = (Re, -Im) of entry (k, j); C = Re(sum) [outer][K].
// Both operands are FP32 split into three BF16 pieces and the six piece
// pairs of order <= 2 accumulate in FP32, so the results keep FP32
// accuracy.  A CTA of four warps takes 64 rows per tile (warp w: rows
// 16w..16w+15) and every output column.

template <int KG, int NN>
__global__ void __launch_bounds__(128) k_contract_x_tc(const float *__restrict__ x, float *__restrict__ y,
                                                       const float2 *__restrict__ Am, int64_t rows, int J, int K,
                                                       int in_real, int acc) {
  constexpr int KS = KG + 8;
  __shared__ __align__(16) uint16_t as[3][64][KS];
  __shared__ __align__(16) uint16_t bs[3][NN][KS];  // B transposed: [n][k]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, gq = lane >> 2, t = lane & 3;
  const int kreal = in_real ? J : 2 * J, nreal = in_real ? 2 * K : K;
  for (int e = tid; e < NN * KG; e += 128) {
    const int n = e / KG, k = e % KG;
    float v = 0.f;
    if (n < nreal && k < kreal) {
      if (in_real) {  // B[j = k][2kk + c]
        const float2 a = Am[(n >> 1) * J + k];
        v = (n & 1) ? a.y : a.x;
      } else {  // B[2j + c][kk = n]
        const float2 a = Am[n * J + (k >> 1)];
        v = (k & 1) ? -a.y : a.x;
      }
    }
    split3_bf16(v, bs[0][n][k], bs[1][n][k], bs[2][n][k]);
  }
  const int64_t ntiles = (rows + 63) / 64;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t r0 = tile * 64;
    __syncthreads();
    for (int e = tid; e < 64 * KG; e += 128) {
      const int r = e / KG, k = e % KG;
      const float v = (r0 + r < rows && k < kreal) ? x[(r0 + r) * kreal + k] : 0.f;
      split3_bf16(v, as[0][r][k], as[1][r][k], as[2][r][k]);
    }
    __syncthreads();
    float c[NN / 8][4];
#pragma unroll
    for (int nt = 0; nt < NN / 8; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) c[nt][q] = 0.f;
#pragma unroll
    for (int kt = 0; kt < KG / 16; kt++)
#pragma unroll
      for (int pa = 2; pa >= 0; pa--) {
        const uint16_t *ar0 = &as[pa][warp * 16 + gq][kt * 16 + 2 * t];
        const uint16_t *ar1 = &as[pa][warp * 16 + gq + 8][kt * 16 + 2 * t];
        const uint32_t a[4] = {*reinterpret_cast<const uint32_t *>(ar0), *reinterpret_cast<const uint32_t *>(ar1),
                               *reinterpret_cast<const uint32_t *>(ar0 + 8),
                               *reinterpret_cast<const uint32_t *>(ar1 + 8)};
#pragma unroll
        for (int pb = 2 - pa; pb >= 0; pb--)
#pragma unroll
          for (int nt = 0; nt < NN / 8; nt++) {
            const uint16_t *br = &bs[pb][nt * 8 + gq][kt * 16 + 2 * t];
            mma_bf16_16816(c[nt], a, *reinterpret_cast<const uint32_t *>(br),
                           *reinterpret_cast<const uint32_t *>(br + 8));
          }
      }
#pragma unroll
    for (int nt = 0; nt < NN / 8; nt++)
#pragma unroll
      for (int hf = 0; hf < 2; hf++) {
        const int64_t r = r0 + warp * 16 + gq + hf * 8;
        const int n = nt * 8 + 2 * t;
        if (r >= rows || n >= nreal) continue;
        float2 *dst = reinterpret_cast<float2 *>(y + r * nreal + n);  // nreal even: 8-byte aligned
        float2 v = make_float2(c[nt][2 * hf], c[nt][2 * hf + 1]);
        if (acc) {
          const float2 o = *dst;
          v.x += o.x;
          v.y += o.y;
        }
        *dst = v;
      }
  }
}

static int launched();

// the tensor-core form applies: channel counts of 16 or 32 (register-held
// weight fragments) and whole 64-point tiles
// HE4_FNO_TENSOR_CORES=0 keeps every layer on the CUDA-core kernels (for
// comparisons; the results agree to FP32 rounding)
static bool pointwise_tc_ok(int kc, int mc, int64_t P) {
  static const bool off = [] {
    const char *s = getenv("HE4_FNO_TENSOR_CORES");
    return s && s[0] == '0';
  }();
  return !off && (kc == 16 || kc == 32) && (mc == 16 || mc == 32) && P % kTcPts == 0;
}

static int launch_pointwise_tc(const float *x, const uint16_t *W, const float *bias, const float *add, float *pre,
                               float *y, int batch, int kc, int mc, int64_t P, int act, bool trans, cudaStream_t s) {
  const int64_t ntiles = (int64_t)batch * (P / kTcPts);
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)148 * 8);
#define HE4_PW_TC(KC_, MC_)                                                                                  \
  if (kc == KC_ && mc == MC_) {                                                                           \
    if (trans)                                                                                            \
      k_pointwise_tc<KC_, MC_, true><<<grid, 128, 0, s>>>(x, W, bias, add, pre, y, P, ntiles, act);      \
    else                                                                                                  \
      k_pointwise_tc<KC_, MC_, false><<<grid, 128, 0, s>>>(x, W, bias, add, pre, y, P, ntiles, act);     \
    return launched();                                                                                    \
  }
  HE4_PW_TC(16, 16)
  HE4_PW_TC(16, 32)
  HE4_PW_TC(32, 16)
  HE4_PW_TC(32, 32)
#undef HE4_PW_TC
  set_error("pointwise tensor-core kernel: channels %d -> %d", kc, mc);
  return HE4_E_ARG;
}

__global__ void k_act_bwd(float *__restrict__ g, const float *__restrict__ pre, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    g[i] *= gelu_grad(pre[i]);
}

template <int CO>
__global__ void k_pointwise_gx(const float *__restrict__ g, const uint16_t *__restrict__ W, float *__restrict__ gx,
                               int B, int ci, int64_t P) {
  __shared__ float sW[kMaxCh * kMaxCh];
  for (int t = threadIdx.x; t < CO * ci; t += blockDim.x) sW[t] = bf(W[t]);
  __syncthreads();
  const int64_t total = (int64_t)B * P;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = idx / P, p = idx - b * P;
    float gv[CO];
#pragma unroll
    for (int o = 0; o < CO; o++) gv[o] = g[(b * CO + o) * P + p];
    for (int i = 0; i < ci; i++) {
      float s = 0.f;
#pragma unroll
      for (int o = 0; o < CO; o++) s += sW[o * ci + i] * gv[o];
      gx[(b * ci + i) * P + p] = s;
    }
  }
}

// weight and bias gradients: block partials over fixed point ranges, then a
// fixed-order sum over the blocks
constexpr int kWgBlocks = 592;  // four 128-thread CTAs per SM for the tensor-core form
constexpr int kWgTile = 64;

__global__ void k_pointwise_wgrad(const float *__restrict__ g, const float *__restrict__ x, float *__restrict__ part,
                                  int B, int ci, int co, int64_t P) {
  // rows padded by one: the threads of a warp read different channels at
  // the same point, which an unpadded 64-float pitch maps to one bank
  __shared__ float sx[kMaxCh][kWgTile + 1];
  __shared__ float sg[kMaxCh][kWgTile + 1];
  const int npair = co * (ci + 1);
  const int64_t total = (int64_t)B * P;
  const int64_t chunk = (total + gridDim.x - 1) / gridDim.x;
  const int64_t t0 = blockIdx.x * chunk, t1 = (t0 + chunk < total) ? t0 + chunk : total;
  // each thread owns pairs threadIdx.x, threadIdx.x + blockDim.x, ...
  constexpr int kMaxPairs = (kMaxCh * (kMaxCh + 1) + kThreads - 1) / kThreads;
  float acc[kMaxPairs];
#pragma unroll
  for (int q = 0; q < kMaxPairs; q++) acc[q] = 0.f;
  for (int64_t tt = t0; tt < t1; tt += kWgTile) {
    const int nt = (t1 - tt < kWgTile) ? (int)(t1 - tt) : kWgTile;
    __syncthreads();
    for (int e = threadIdx.x; e < (ci + co) * kWgTile; e += blockDim.x) {
      const int c = e / kWgTile, u = e % kWgTile;
      float v = 0.f;
      if (u < nt) {
        const int64_t t = tt + u, b = t / P, p = t - b * P;
        v = (c < ci) ? x[(b * ci + c) * P + p] : g[(b * co + (c - ci)) * P + p];
      }
      if (c < ci)
        sx[c][u] = v;
      else
        sg[c - ci][u] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kMaxPairs; q++) {
      const int pr = threadIdx.x + q * kThreads;
      if (pr >= npair) break;
      const int o = pr / (ci + 1), i = pr % (ci + 1);
      float s = 0.f;
      if (i < ci)
        for (int u = 0; u < nt; u++) s += sg[o][u] * sx[i][u];
      else
        for (int u = 0; u < nt; u++) s += sg[o][u];
      acc[q] += s;
    }
  }
#pragma unroll
  for (int q = 0; q < kMaxPairs; q++) {
    const int pr = threadIdx.x + q * kThreads;
    if (pr < npair) part[(int64_t)blockIdx.x * npair + pr] = acc[q];
  }
}

// one warp per (output, input or bias) pair: lane l sums the partials of
// blocks l, l + 32, ... in FP64, then a fixed shuffle tree adds the lanes,
// so the order (and the result) is the same on every run
__global__ void k_wgrad_finish(const float *__restrict__ part, float *__restrict__ gW, float *__restrict__ gb,
                               int nblk, int ci, int co) {
  const int npair = co * (ci + 1);
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (int pr = blockIdx.x * wpb + (threadIdx.x >> 5); pr < npair; pr += gridDim.x * wpb) {
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += (double)part[(int64_t)b * npair + pr];
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if (lane != 0) continue;
    const int o = pr / (ci + 1), i = pr % (ci + 1);
    if (i < ci) {
      if (gW) gW[o * ci + i] = (float)s;
    } else if (gb) {
      gb[o] = (float)s;
    }
  }
}

// ---------------------------------------------------------------------------
// loss, optimizer
// ---------------------------------------------------------------------------
constexpr int kLossBlocks = 296;

__global__ void k_loss_part(const float *__restrict__ pred, const float *__restrict__ tgt, double *part, int64_t n) {
  __shared__ double sh[32];
  double e = 0.0, t2 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double d = (double)pred[i] - (double)tgt[i];
    e += d * d;
    t2 += (double)tgt[i] * tgt[i];
  }
  e = block_sum(e, sh);
  t2 = block_sum(t2, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = e;
    part[gridDim.x + blockIdx.x] = t2;
  }
}

__global__ void k_loss_finish(const double *part, int nb, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double e = 0.0, t2 = 0.0;
    for (int b = 0; b < nb; b++) {
      e += part[b];
      t2 += part[nb + b];
    }
    out[0] = e / (t2 > 0 ? t2 : 1.0);
    out[1] = t2;
  }
}

__global__ void k_loss_grad(const float *__restrict__ pred, const float *__restrict__ tgt, float *grad,
                            const double *out, int64_t n) {
  const double t2 = out[1] > 0 ? out[1] : 1.0;
  const float c = (float)(2.0 / t2);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    grad[i] = c * (pred[i] - tgt[i]);
}

__device__ __forceinline__ uint16_t to_bf16(float f) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

__global__ void k_adam(float *p, const float *__restrict__ g, float *m, float *v, uint16_t *pb, int64_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (pb) pb[i] = to_bf16(pi);
  }
}

__global__ void k_to_bf16(const float *__restrict__ x, uint16_t *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = to_bf16(x[i]);
}

// ---------------------------------------------------------------------------
// grid transfer
// ---------------------------------------------------------------------------
__global__ void k_restrict(const double *__restrict__ src, float *__restrict__ dst, int nf, int f, int cplx,
                           float scale) {
  const int nc = nf / f;
  const int64_t nc3 = (int64_t)nc * nc * nc;
  const float inv = scale / (float)(f * f * f);
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc3; c += (int64_t)gridDim.x * blockDim.x) {
    const int cx = (int)(c % nc), cy = (int)((c / nc) % nc), cz = (int)(c / ((int64_t)nc * nc));
    double re = 0.0, im = 0.0;
    for (int dz = 0; dz < f; dz++)
      for (int dy = 0; dy < f; dy++)
        for (int dx = 0; dx < f; dx++) {
          const int64_t fi = ((int64_t)(cz * f + dz) * nf + (cy * f + dy)) * nf + (cx * f + dx);
          if (cplx) {
            re += src[2 * fi];
            im += src[2 * fi + 1];
          } else {
            re += src[fi];
          }
        }
    dst[c] = (float)re * inv;
    if (cplx) dst[nc3 + c] = (float)im * inv;
  }
}

__global__ void k_prolong_add(const float *__restrict__ src, double2 *dst, int nf, int f, float scale) {
  const int nc = nf / f;
  const int64_t nc3 = (int64_t)nc * nc * nc;
  const int64_t nf3 = (int64_t)nf * nf * nf;
  const float off = 0.5f * (float)(f - 1);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nf3; q += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % nf), y = (int)((q / nf) % nf), z = (int)(q / ((int64_t)nf * nf));
    const float ux = (x - off) / f, uy = (y - off) / f, uz = (z - off) / f;
    const int x0 = (int)floorf(ux), y0 = (int)floorf(uy), z0 = (int)floorf(uz);
    const float wx = ux - x0, wy = uy - y0, wz = uz - z0;
    float re = 0.f, im = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int ix = ((x0 + (c & 1)) % nc + nc) % nc;
      const int iy = ((y0 + ((c >> 1) & 1)) % nc + nc) % nc;
      const int iz = ((z0 + (c >> 2)) % nc + nc) % nc;
      const float w = ((c & 1) ? wx : 1.f - wx) * (((c >> 1) & 1) ? wy : 1.f - wy) * ((c >> 2) ? wz : 1.f - wz);
      const int64_t ci = ((int64_t)iz * nc + iy) * nc + ix;
      re += w * src[ci];
      im += w * src[nc3 + ci];
    }
    double2 d = dst[q];
    d.x += (double)(scale * re);
    d.y += (double)(scale * im);
    dst[q] = d;
  }
}

__global__ void k_deposit_coarse(const double *__restrict__ r, int npar, float *dst, int nc, double xmax) {
  const double hc = 2.0 * xmax / nc;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npar; p += gridDim.x * blockDim.x) {
    const double a = (r[p] + xmax) / hc, b = (r[npar + p] + xmax) / hc, c = (r[2 * npar + p] + xmax) / hc;
    if (!(a >= 0 && a < nc && b >= 0 && b < nc && c >= 0 && c < nc)) continue;
    const int ix = (int)a, iy = (int)b, iz = (int)c;
    // counts stay below 2^24, so FP32 additions of 1 are exact and order-free
    atomicAdd(&dst[((int64_t)iz * nc + iy) * nc + ix], 1.0f);
  }
}

__global__ void k_scale(float *x, int64_t n, float s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= s;
}

// parareal correction: u_new = s (g_new + fine - g_old), written over u
// (the previous iterate).  Pass 1 sums |g_new + fine - g_old|^2 and
// |fine|^2 per block; s = sqrt(sum |fine|^2 / sum |u_new|^2) when the norm
// projection is on (the fine propagator conserves the norm), else 1.  Pass 2
// writes u and sums |u_new - u|^2 and |u|^2 per block.
__global__ void k_parareal_norms(const double *__restrict__ gnew, const double *__restrict__ fine,
                                 const double *__restrict__ gold, int64_t n, double *part) {
  __shared__ double sh[32];
  double nn = 0.0, ff = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = (gnew[i] + fine[i]) - gold[i];
    nn += v * v;
    ff += fine[i] * fine[i];
  }
  nn = block_sum(nn, sh);
  ff = block_sum(ff, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = nn;
    part[gridDim.x + blockIdx.x] = ff;
  }
}

__global__ void k_parareal(const double *__restrict__ gnew, const double *__restrict__ fine,
                           const double *__restrict__ gold, double *u, int64_t n, const double *scale,
                           double *part) {
  __shared__ double sh[32];
  double sc = 1.0;
  if (scale) sc = (scale[0] > 0.0) ? sqrt(scale[1] / scale[0]) : 1.0;
  double dd = 0.0, uu = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double old = u[i];
    const double v = sc * ((gnew[i] + fine[i]) - gold[i]);
    u[i] = v;
    dd += (v - old) * (v - old);
    uu += old * old;
  }
  dd = block_sum(dd, sh);
  uu = block_sum(uu, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = dd;
    part[gridDim.x + blockIdx.x] = uu;
  }
}

__global__ void k_sum2(const double *part, int nb, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < nb; i++) {
      a += part[i];
      b += part[nb + i];
    }
    out[0] = a;
    out[1] = b;
  }
}

static int launched() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("FNO kernel launch: %s", cudaGetErrorString(e));
    return HE4_E_CUDA;
  }
  return HE4_OK;
}

#define FNO_CI_SWITCH(ci, KER, ...)                            \
  switch (ci) {                                                 \
    case 1: KER<1><<<__VA_ARGS__; break;                        \
    case 2: KER<2><<<__VA_ARGS__; break;                        \
    case 3: KER<3><<<__VA_ARGS__; break;                        \
    case 4: KER<4><<<__VA_ARGS__; break;                        \
    case 8: KER<8><<<__VA_ARGS__; break;                        \
    case 16: KER<16><<<__VA_ARGS__; break;                      \
    case 32: KER<32><<<__VA_ARGS__; break;                      \
    case 64: KER<64><<<__VA_ARGS__; break;                      \
    default:                                                    \
      set_error("FNO: %d channels are not supported", (int)ci); \
      return HE4_E_UNSUPPORTED;                                 \
  }

}  // namespace fno
}  // namespace he4

using namespace he4;
using namespace he4::fno;

namespace {
// HE4_FNO_CONTRACT_KC=0 selects the one-output-per-thread contraction (for
// comparisons; same sums)
bool contract_kc_on() {
  static const bool on = [] {
    const char *e = getenv("HE4_FNO_CONTRACT_KC");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <int KC>
int launch_contract_kc(const void *x, void *y, const float2 *A2, int64_t outer, int J, int K, int64_t inner,
                       int in_real, int out_real, int accumulate, size_t sm, cudaStream_t s) {
  const unsigned g = blocks_for(outer * ((K + KC - 1) / KC) * inner);
  if (in_real && out_real)
    k_contract_kc<true, true, KC><<<g, kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  else if (in_real)
    k_contract_kc<true, false, KC><<<g, kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  else if (out_real)
    k_contract_kc<false, true, KC><<<g, kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  else
    k_contract_kc<false, false, KC><<<g, kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  return launched();
}
}  // namespace

extern "C" {

int he4_fno_contract(const void *x, void *y, const float *A, int32_t outer, int32_t J, int32_t K, int32_t inner,
                     int32_t in_real, int32_t out_real, int32_t accumulate, void *stream) {
  if (!x || !y || !A || outer < 1 || J < 1 || K < 1 || inner < 1 || (int64_t)J * K * 8 > 48 * 1024) {
    set_error("he4_fno_contract: invalid arguments");
    return HE4_E_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t total = (int64_t)outer * K * inner;
  const size_t sm = sizeof(float2) * J * K;
  const float2 *A2 = reinterpret_cast<const float2 *>(A);
  // along the contiguous axis, real <-> complex: tensor-core GEMMs
  if (inner == 1 && in_real != out_real && pointwise_tc_ok(16, 16, 64)) {
    const int kreal = in_real ? J : 2 * J, nreal = in_real ? 2 * K : K;
    const unsigned grid = (unsigned)std::min<int64_t>(((int64_t)outer + 63) / 64, (int64_t)148 * 8);
    const float *xf = reinterpret_cast<const float *>(x);
    float *yf = reinterpret_cast<float *>(y);
    if (kreal <= 32 && nreal <= 64 && nreal % 2 == 0) {
      k_contract_x_tc<32, 64><<<grid, 128, 0, s>>>(xf, yf, A2, outer, J, K, in_real, accumulate);
      return launched();
    }
    if (kreal <= 64 && nreal <= 24 && nreal % 2 == 0) {
      k_contract_x_tc<64, 24><<<grid, 128, 0, s>>>(xf, yf, A2, outer, J, K, in_real, accumulate);
      return launched();
    }
  }
  // back to a full axis (K a multiple of 16: the adjoint directions), 16
  // output modes per thread: 22 us against 27 us at 64^3, width 32.  Onto the
  // 12 retained modes one output per thread keeps 12x the threads in flight
  // and is faster (27 us against 40 us with 12 modes per thread).
  if (contract_kc_on() && K % 16 == 0)
    return launch_contract_kc<16>(x, y, A2, outer, J, K, inner, in_real, out_real, accumulate, sm, s);
  if (in_real && out_real)
    k_contract<true, true><<<blocks_for(total), kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  else if (in_real)
    k_contract<true, false><<<blocks_for(total), kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  else if (out_real)
    k_contract<false, true><<<blocks_for(total), kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  else
    k_contract<false, false><<<blocks_for(total), kThreads, sm, s>>>(x, y, A2, outer, J, K, inner, accumulate);
  return launched();
}

int he4_fno_mix(const float *x, const uint16_t *R, float *y, int32_t batch, int32_t cin, int32_t cout,
                int32_t modes, void *stream) {
  if (!x || !R || !y || batch < 1 || cin < 1 || cout < 1 || modes < 1) {
    set_error("he4_fno_mix: invalid arguments");
    return HE4_E_ARG;
  }
  const int64_t total = (int64_t)batch * cout * modes;
  k_mix<<<blocks_for(total), kThreads, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float2 *>(x), R,
                                                                  reinterpret_cast<float2 *>(y), batch, cin, cout,
                                                                  modes);
  return launched();
}

int he4_fno_mix_bwd(const float *gy, const float *x, const uint16_t *R, float *gx, float *gR, int32_t batch,
                    int32_t cin, int32_t cout, int32_t modes, void *stream) {
  if (!gy || !x || !R || batch < 1 || cin < 1 || cout < 1 || modes < 1) {
    set_error("he4_fno_mix_bwd: invalid arguments");
    return HE4_E_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const float2 *g2 = reinterpret_cast<const float2 *>(gy), *x2 = reinterpret_cast<const float2 *>(x);
  // gR first: gx may overwrite x
  if (gR) {
    k_mix_gR<<<blocks_for((int64_t)cin * cout * modes), kThreads, 0, s>>>(g2, x2, reinterpret_cast<float2 *>(gR),
                                                                         batch, cin, cout, modes);
    HE4_TRY(launched());
  }
  if (gx) {
    k_mix_gx<<<blocks_for((int64_t)batch * cin * modes), kThreads, 0, s>>>(g2, R, reinterpret_cast<float2 *>(gx),
                                                                          batch, cin, cout, modes);
    HE4_TRY(launched());
  }
  return HE4_OK;
}

int he4_fno_pointwise(const float *x, const uint16_t *W, const float *bias, const float *add, float *pre, float *y,
                      int32_t batch, int32_t cin, int32_t cout, int64_t npts, int32_t act, void *stream) {
  if (!x || !W || !y || batch < 1 || cin < 1 || cout < 1 || cout > kMaxCh || npts < 1) {
    set_error("he4_fno_pointwise: invalid arguments");
    return HE4_E_ARG;
  }
  if (pointwise_tc_ok(cin, cout, npts))
    return launch_pointwise_tc(x, W, bias, add, pre, y, batch, cin, cout, npts, act, false, (cudaStream_t)stream);
  const int64_t total = (int64_t)batch * npts;
  FNO_CI_SWITCH(cin, k_pointwise, blocks_for(total), kThreads, 0, (cudaStream_t)stream >>>(x, W, bias, add, pre, y,
                                                                                         batch, cout, npts, act));
  return launched();
}

int64_t he4_fno_pointwise_work(int32_t batch, int32_t cin, int32_t cout, int64_t npts) {
  (void)batch;
  (void)npts;
  return (int64_t)kWgBlocks * cout * (cin + 1);
}

int he4_fno_pointwise_bwd(float *gy, const float *pre, const float *x, const uint16_t *W, float *gx, float *gW,
                          float *gbias, float *work, int32_t batch, int32_t cin, int32_t cout, int64_t npts,
                          int32_t act, void *stream) {
  if (!gy || !x || !W || batch < 1 || cin < 1 || cout < 1 || cin > kMaxCh || cout > kMaxCh || npts < 1 ||
      (act && !pre) || ((gW || gbias) && !work)) {
    set_error("he4_fno_pointwise_bwd: invalid arguments");
    return HE4_E_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t total = (int64_t)batch * npts;
  if (act) {
    k_act_bwd<<<blocks_for(total * cout), kThreads, 0, s>>>(gy, pre, total * cout);
    HE4_TRY(launched());
  }
  if (gx) {
    if (pointwise_tc_ok(cout, cin, npts)) {
      HE4_TRY(launch_pointwise_tc(gy, W, nullptr, nullptr, nullptr, gx, batch, cout, cin, npts, 0, true, s));
    } else {
      FNO_CI_SWITCH(cout, k_pointwise_gx, blocks_for(total), kThreads, 0, s >>>(gy, W, gx, batch, cin, npts));
      HE4_TRY(launched());
    }
  }
  if (gW || gbias) {
    const int64_t ntiles = (int64_t)batch * (npts / kTcPts);
    if (pointwise_tc_ok(cin, cout, npts) && cin == 32 && cout == 32)
      k_pointwise_wgrad_tc<32, 32><<<kWgBlocks, 128, 0, s>>>(gy, x, work, npts, ntiles);
    else if (pointwise_tc_ok(cin, cout, npts) && cin == 16 && cout == 16)
      k_pointwise_wgrad_tc<16, 16><<<kWgBlocks, 128, 0, s>>>(gy, x, work, npts, ntiles);
    else
      k_pointwise_wgrad<<<kWgBlocks, kThreads, 0, s>>>(gy, x, work, batch, cin, cout, npts);
    HE4_TRY(launched());
    const int wpb = kThreads / 32;  // one warp per pair
    k_wgrad_finish<<<(cout * (cin + 1) + wpb - 1) / wpb, kThreads, 0, s>>>(work, gW, gbias, kWgBlocks, cin, cout);
    HE4_TRY(launched());
  }
  return HE4_OK;
}

int he4_fno_loss(const float *pred, const float *target, float *grad, double *out, int64_t n, double *work,
                 void *stream) {
  if (!pred || !target || !out || !work || n < 1) {
    set_error("he4_fno_loss: invalid arguments");
    return HE4_E_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  k_loss_part<<<kLossBlocks, kThreads, 0, s>>>(pred, target, work, n);
  HE4_TRY(launched());
  k_loss_finish<<<1, 32, 0, s>>>(work, kLossBlocks, out);
  HE4_TRY(launched());
  if (grad) {
    k_loss_grad<<<blocks_for(n), kThreads, 0, s>>>(pred, target, grad, out, n);
    HE4_TRY(launched());
  }
  return HE4_OK;
}

int he4_fno_adam(float *p, const float *g, float *m, float *v, uint16_t *pb, int64_t n, float lr, float beta1,
                 float beta2, float eps, int32_t step, void *stream) {
  if (!p || !g || !m || !v || n < 1 || step < 1) {
    set_error("he4_fno_adam: invalid arguments");
    return HE4_E_ARG;
  }
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_adam<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(p, g, m, v, pb, n, lr, beta1, beta2, eps, c1, c2);
  return launched();
}

int he4_fno_to_bf16(const float *x, uint16_t *y, int64_t n, void *stream) {
  if (!x || !y || n < 1) {
    set_error("he4_fno_to_bf16: invalid arguments");
    return HE4_E_ARG;
  }
  k_to_bf16<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(x, y, n);
  return launched();
}

int he4_fno_restrict(const double *src, float *dst, int32_t nf, int32_t f, int32_t complex_src, float scale,
                     void *stream) {
  if (!src || !dst || f < 1 || nf < f || nf % f != 0) {
    set_error("he4_fno_restrict: invalid arguments");
    return HE4_E_ARG;
  }
  const int64_t nc = nf / f;
  k_restrict<<<blocks_for(nc * nc * nc), kThreads, 0, (cudaStream_t)stream>>>(src, dst, nf, f, complex_src, scale);
  return launched();
}

int he4_fno_prolong_add(const float *src, double *dst, int32_t nf, int32_t f, float scale, void *stream) {
  if (!src || !dst || f < 1 || nf < f || nf % f != 0) {
    set_error("he4_fno_prolong_add: invalid arguments");
    return HE4_E_ARG;
  }
  k_prolong_add<<<blocks_for((int64_t)nf * nf * nf), kThreads, 0, (cudaStream_t)stream>>>(
      src, reinterpret_cast<double2 *>(dst), nf, f, scale);
  return launched();
}

int he4_fno_deposit(const double *r, int32_t npar, float *dst, int32_t nc, double xmax, float scale, void *stream) {
  if (!r || !dst || npar < 1 || nc < 1 || !(xmax > 0)) {
    set_error("he4_fno_deposit: invalid arguments");
    return HE4_E_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n3 = (int64_t)nc * nc * nc;
  if (cudaMemsetAsync(dst, 0, sizeof(float) * n3, s) != cudaSuccess) {
    set_error("he4_fno_deposit: memset failed");
    return HE4_E_CUDA;
  }
  k_deposit_coarse<<<blocks_for(npar), kThreads, 0, s>>>(r, npar, dst, nc, xmax);
  HE4_TRY(launched());
  const double hc = 2.0 * xmax / nc;
  k_scale<<<blocks_for(n3), kThreads, 0, s>>>(dst, n3, (float)(scale / (npar * hc * hc * hc)));
  return launched();
}

int he4_parareal_correct(const double *gnew, const double *fine, const double *gold, double *u, int64_t n,
                         int32_t renorm, double *out, double *work, void *stream) {
  if (!gnew || !fine || !gold || !u || !out || !work || n < 1) {
    set_error("he4_parareal_correct: invalid arguments");
    return HE4_E_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (renorm) {
    k_parareal_norms<<<kLossBlocks, kThreads, 0, s>>>(gnew, fine, gold, n, work);
    HE4_TRY(launched());
    k_sum2<<<1, 32, 0, s>>>(work, kLossBlocks, out + 2);
    HE4_TRY(launched());
  }
  k_parareal<<<kLossBlocks, kThreads, 0, s>>>(gnew, fine, gold, u, n, renorm ? out + 2 : nullptr, work);
  HE4_TRY(launched());
  k_sum2<<<1, 32, 0, s>>>(work, kLossBlocks, out);
  return launched();
}

}  // extern "C"

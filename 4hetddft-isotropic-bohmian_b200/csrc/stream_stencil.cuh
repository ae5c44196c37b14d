// stream_stencil.cuh -- z-marching stencils fed by bulk asynchronous copies.
//
// A CTA owns TY full x rows (j0 .. j0+TY-1) of the grid and marches through
// a chunk of z planes.  Every plane's input rows travel from global to
// shared memory as 1D bulk copies (cp.async.bulk, one row per copy,
// completing on the stage's mbarrier with a transaction count), S planes
// ahead of the one being computed, so each SM keeps tens of KB in flight
// without holding them in registers.  The x taps wrap inside the full row,
// the y taps read TY + 2M rows of the plane, the z taps a ring of the last
// 2M + S planes' centre rows.  Periodic grids only (icon = 8); the row
// length NX is a template parameter (128, 256 or 512) and TY must
// divide ny.
//
// Every wait on an mbarrier is bounded (one second of %globaltimer); a CTA
// whose copies do not arrive sets bit 0 of *err, waits (bounded again) for
// the copies it issued, and leaves without writing further output, so the
// host sees HE4_E_CUDA instead of a hung GPU.
#pragma once
#include "bulk.cuh"
#include "common.cuh"

namespace he4 {

__device__ __forceinline__ int wrapn(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Elements of padding on each side of a row whose x taps wrap: at least M,
// a whole number of 16-byte units (the pads are filled by bulk copies of
// the row's last / first PAD elements, which start 16-byte aligned).
template <typename T, int M>
struct RowPad {
  static constexpr int value = (int)(((M * sizeof(T) + 15) / 16) * 16 / sizeof(T));
};

// Shared-memory layout of one CTA (bytes), for S stages of TY rows of NX
// points.  h0 rows (x taps) carry RowPad elements on both sides.
// CD (centre values direct): den, lin and dencg, which each thread reads at
// its own points only, come straight from global memory instead of through
// shared memory, which leaves room for a third CTA per SM.
template <typename TI, bool OTC, int M, int TY, int S, int NX, bool CD = false>
struct Pot4StreamLayout {
  static constexpr int RH = S + 2 * M;  // h2 ring: planes k-M .. k+M plus the S-1 in flight
  static constexpr int PX = RowPad<TI, M>::value, RS0 = NX + 2 * PX;
  static constexpr size_t rt = (size_t)NX * sizeof(TI), rd = (size_t)NX * sizeof(double);
  static constexpr size_t bars = 0, den = 128, lin = den + (CD ? 0 : (size_t)S * TY * rd),
                          dcg = lin + (CD ? 0 : (size_t)S * TY * rt), h0 = dcg + (CD ? 0 : (size_t)S * TY * rt),
                          h1 = h0 + (OTC ? (size_t)S * TY * RS0 * sizeof(TI) : 0),
                          h2 = h1 + (OTC ? (size_t)S * (TY + 2 * M) * rt : 0),
                          total = h2 + (OTC ? (size_t)RH * TY * rt : 0);
};

// Central first-derivative weights w_u (u = 1..M, w_-u = -w_u, w_0 = 0)
// split into float pieces w_u = hi_u + lo_u (|lo_u| <= 2^-24 |w_u|): the
// float-math pot4 forms sum_u (hi_u + lo_u) (h(+u) - h(-u)) in FP32, so the
// weights enter with ~48 significant bits and the differences of
// neighbouring values round far less than the taps themselves.
struct SplitTaps {
  float hi[3][6], lo[3][6];
};

// pot4 of the merged evaluation (poten.f90:80-92,122-124 with term_alfa's
// divergence term, term_alfa.f90:110-113): the same arithmetic as
// k_pot4_merged_z, rows streamed.  Grid: (ny / TY, z chunks of zc planes).
// FM (float grids of the FP32-convolution form, antisymmetric first-
// derivative rows): the pointwise assembly in FP32 -- the divergence with
// split weights (SplitTaps), the correlation term from the float dencg, the
// solid penalty from tanh written through e = exp(-2|x|) (1 + tanh x =
// 2/(1+e) for x >= 0, 2e/(1+e) below; 1 - tanh^2 x = 4e/(1+e)^2), which
// also avoids the cancellation of 1 + tanh x for x << 0 -- and only the
// final three-term sum in FP64.  Five float/double conversions per point
// instead of 23.
template <typename TI, bool OTC, int M, int TY, int S, int NX, bool FM = false>
__global__ void __launch_bounds__(256) k_pot4_stream(const TI *__restrict__ lin, const double *__restrict__ den,
                                                     const TI *__restrict__ dencg, const TI *__restrict__ h0,
                                                     const TI *__restrict__ h1, const TI *__restrict__ h2,
                                                     double *__restrict__ pot4, Stencil st, Geo g, OtArgs a, int zc,
                                                     unsigned *err, SplitTaps tp) {
  extern __shared__ __align__(128) unsigned char smem[];
  using L = Pot4StreamLayout<TI, OTC, M, TY, S, NX, FM>;
  constexpr int RH = L::RH, PX = L::PX, RS0 = L::RS0;
  constexpr unsigned rt = (unsigned)L::rt, rd = (unsigned)L::rd, pb = (unsigned)(PX * sizeof(TI));
  const int ny = g.ny, nz = g.nz;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::bars);
  double *sden = reinterpret_cast<double *>(smem + L::den);
  TI *slin = reinterpret_cast<TI *>(smem + L::lin);
  TI *sdcg = reinterpret_cast<TI *>(smem + L::dcg);
  TI *sh0 = reinterpret_cast<TI *>(smem + L::h0);
  TI *sh1 = reinterpret_cast<TI *>(smem + L::h1);
  TI *sh2 = reinterpret_cast<TI *>(smem + L::h2);
  const int j0 = blockIdx.x * TY;
  const int k0 = blockIdx.y * zc;
  const int k1 = min(k0 + zc, nz);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t ps = (size_t)ny * NX;
  if (k0 >= nz) return;
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // h2 ring slot of plane p (p >= k0 - M)
  auto slot = [&](int p) { return (p - (k0 - M)) % RH; };
  // the copies of plane k into stage s (warp 0), plus, with `pro`, the h2
  // planes k0-M .. k0+M-1 that precede the first stage's
  auto issue = [&](int k, int s, bool pro) {
    const unsigned bytes = (FM ? 0 : TY * rd + 2 * TY * rt) +
                           (OTC ? (TY * (2 * rt + 2 * pb) + (TY + 2 * M) * rt + (pro ? 2 * M * TY * rt : 0)) : 0);
    if (lane == 0) mbar_expect_tx(&bar[s], bytes);
    __syncwarp();
    const size_t pk = (size_t)k * ps;
    for (int r = lane; r < TY; r += 32) {
      const size_t o = pk + (size_t)(j0 + r) * NX;
      if (!FM) {
        bulk_row(sden + ((size_t)s * TY + r) * NX, den + o, rd, &bar[s]);
        bulk_row(slin + ((size_t)s * TY + r) * NX, lin + o, rt, &bar[s]);
        bulk_row(sdcg + ((size_t)s * TY + r) * NX, dencg + o, rt, &bar[s]);
      }
      if (OTC) {
        TI *row = sh0 + ((size_t)s * TY + r) * RS0;
        bulk_row(row + PX, h0 + o, rt, &bar[s]);
        bulk_row(row, h0 + o + NX - PX, pb, &bar[s]);     // left pad: the row's last PX points
        bulk_row(row + PX + NX, h0 + o, pb, &bar[s]);     // right pad: its first PX points
        const size_t o2 = (size_t)wrapn(k + M, nz) * ps + (size_t)(j0 + r) * NX;
        bulk_row(sh2 + ((size_t)slot(k + M) * TY + r) * NX, h2 + o2, rt, &bar[s]);
      }
    }
    if (OTC) {
      for (int r = lane; r < TY + 2 * M; r += 32) {
        const size_t o = pk + (size_t)wrapn(j0 - M + r, ny) * NX;
        bulk_row(sh1 + ((size_t)s * (TY + 2 * M) + r) * NX, h1 + o, rt, &bar[s]);
      }
      if (pro)
        for (int q = lane; q < 2 * M * TY; q += 32) {
          const int p = k0 - M + q / TY, r = q % TY;
          const size_t o2 = (size_t)wrapn(p, nz) * ps + (size_t)(j0 + r) * NX;
          bulk_row(sh2 + ((size_t)slot(p) * TY + r) * NX, h2 + o2, rt, &bar[s]);
        }
    }
  };
  if (warp == 0)
    for (int q = 0; q < S && k0 + q < k1; q++) issue(k0 + q, q, q == 0);
  const double a0 = a.cp4 / 2.0, a1 = a.cpp4 / 3.0, adiv = a.h2o2m4 * a.alphas;
  const float fa0 = (float)a0, fa1 = (float)a1, fcs = (float)a.c_solid, fbeta = (float)a.beta;
  constexpr int NPT = TY * NX, NQ = NPT / 256;
  static_assert(NPT % 256 == 0, "a plane's points are whole multiples of the CTA");
  for (int k = k0; k < k1; k++) {
    const int it = k - k0, s = it % S;
    // FM: this plane's den, lin and dencg at the thread's own points, from
    // global memory, issued before the wait so their latency overlaps it
    double dq[FM ? NQ : 1];
    TI lq[FM ? NQ : 1], cq[FM ? NQ : 1];
    if constexpr (FM) {
      const size_t b0 = (size_t)k * ps + (size_t)j0 * NX;
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        dq[q] = __ldg(den + b0 + tid + 256 * q);
        lq[q] = __ldg(lin + b0 + tid + 256 * q);
        cq[q] = __ldg(dencg + b0 + tid + 256 * q);
      }
    }
    const bool ok = mbar_wait_bounded(&bar[s], (unsigned)((it / S) & 1));
    if (__syncthreads_or(!ok)) {
      // copies that did not arrive: flag, drain (bounded) what this CTA
      // issued, leave
      if (tid == 0) {
        atomicOr(err, 1u);
        for (int q = it; q < k1 - k0 && q < it + S; q++) mbar_wait_bounded(&bar[q % S], (unsigned)((q / S) & 1));
      }
      return;
    }
    const double *dd = sden + (size_t)s * TY * NX;
    const TI *ll = slin + (size_t)s * TY * NX;
    const TI *cc = sdcg + (size_t)s * TY * NX;
    const TI *x0 = sh0 + (size_t)s * TY * RS0 + PX;
    const TI *y1 = sh1 + (size_t)s * (TY + 2 * M) * NX;
    const TI *zr[2 * M + 1];
#pragma unroll
    for (int u = 0; u <= 2 * M; u++) zr[u] = sh2 + (size_t)slot(k - M + u) * TY * NX;
    double *out = pot4 + (size_t)k * ps + (size_t)j0 * NX;
#pragma unroll
    for (int p = tid; p < NPT; p += 256) {
      const int r = p / NX, x = p % NX;
      if constexpr (FM) {
        const int qi = (p - tid) / 256;
        const double d = dq[qi];
        const float xs = (float)(a.beta * (d - a.den_m)), df = (float)d;
        const float e = expf(-2.0f * fabsf(xs)), q = 1.0f / (1.0f + e);
        const float opt = (xs >= 0.0f ? 2.0f : 2.0f * e) * q, omt = 4.0f * e * q * q;
        const float dc = cq[qi];
        const float cp = dc * dc * (fa0 + fa1 * dc) + fcs * (opt + fbeta * df * omt);
        double v = (double)lq[qi] + (double)cp;
        if (OTC) {
          const TI *xr = x0 + r * RS0 + x;
          const TI *yc = y1 + r * NX + x;
          float sh = 0.0f, sl = 0.0f;
#pragma unroll
          for (int u = M; u >= 1; u--) {
            const float ex = xr[u] - xr[-u], ey = yc[(M + u) * NX] - yc[(M - u) * NX],
                        ez = zr[M + u][p] - zr[M - u][p];
            sh = fmaf(tp.hi[0][u - 1], ex, sh);
            sl = fmaf(tp.lo[0][u - 1], ex, sl);
            sh = fmaf(tp.hi[1][u - 1], ey, sh);
            sl = fmaf(tp.lo[1][u - 1], ey, sl);
            sh = fmaf(tp.hi[2][u - 1], ez, sh);
            sl = fmaf(tp.lo[2][u - 1], ez, sl);
          }
          v += (double)(sh + sl) * adiv;
        }
        out[p] = v;
        continue;
      }
      const double d = dd[p];
      const double th = tanh(a.beta * (d - a.den_m));
      const double pen = a.c_solid * (1.0 + th + a.beta * d * (1.0 - th * th));
      const double dc = (double)cc[p];
      double v = (double)ll[p] + dc * dc * (a0 + a1 * dc) + pen;
      if (OTC) {
        double d0 = 0.0, d1 = 0.0, d2 = 0.0;
        const TI *xr = x0 + r * RS0 + x;
        const TI *yc = y1 + r * NX + x;
#pragma unroll
        for (int u = -M; u <= M; u++) d0 += st.w1[0][u + M] * (double)xr[u];
#pragma unroll
        for (int u = -M; u <= M; u++) d1 += st.w1[1][u + M] * (double)yc[(M + u) * NX];
#pragma unroll
        for (int u = -M; u <= M; u++) d2 += st.w1[2][u + M] * (double)zr[u + M][p];
        v += (d0 + d1 + d2) * adiv;
      }
      out[p] = v;
    }
    __syncthreads();  // stage s and the ring slot of plane k-M are free
    if (warp == 0 && k + S < k1) issue(k + S, s, false);
  }
}

// Density gradient (derden.f90:26-28) streamed: plane k's TY + 2M rows
// (x and y taps; rows padded for the x wrap) per stage, the centre rows of
// planes k-M .. k+M in a ring.
template <typename TO, int M, int TY, int S, int NX>
struct GradStreamLayout {
  static constexpr int RH = S + 2 * M;
  static constexpr int PX = RowPad<double, M>::value, RS = NX + 2 * PX;
  static constexpr size_t rd = (size_t)NX * sizeof(double);
  static constexpr size_t bars = 0, yb = 128, zr = yb + (size_t)S * (TY + 2 * M) * RS * sizeof(double),
                          total = zr + (size_t)RH * TY * rd;
};

template <typename TO, int M, int TY, int S, int NX>
__global__ void __launch_bounds__(256) k_grad_stream(const double *__restrict__ f, TO *__restrict__ dx,
                                                     TO *__restrict__ dy, TO *__restrict__ dz, Stencil st, Geo g,
                                                     int zc, unsigned *err) {
  extern __shared__ __align__(128) unsigned char smem[];
  using L = GradStreamLayout<TO, M, TY, S, NX>;
  constexpr int RH = L::RH, PX = L::PX, RS = L::RS;
  constexpr unsigned rd = (unsigned)L::rd, pb = (unsigned)(PX * sizeof(double));
  const int ny = g.ny, nz = g.nz;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::bars);
  double *syb = reinterpret_cast<double *>(smem + L::yb);
  double *szr = reinterpret_cast<double *>(smem + L::zr);
  const int j0 = blockIdx.x * TY;
  const int k0 = blockIdx.y * zc;
  const int k1 = min(k0 + zc, nz);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t ps = (size_t)ny * NX;
  if (k0 >= nz) return;
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto slot = [&](int p) { return (p - (k0 - M)) % RH; };
  auto issue = [&](int k, int s, bool pro) {
    const unsigned bytes = (TY + 2 * M) * (rd + 2 * pb) + TY * rd + (pro ? 2 * M * TY * rd : 0);
    if (lane == 0) mbar_expect_tx(&bar[s], bytes);
    __syncwarp();
    const size_t pk = (size_t)k * ps;
    for (int r = lane; r < TY + 2 * M; r += 32) {
      const double *src = f + pk + (size_t)wrapn(j0 - M + r, ny) * NX;
      double *row = syb + ((size_t)s * (TY + 2 * M) + r) * RS;
      bulk_row(row + PX, src, rd, &bar[s]);
      bulk_row(row, src + NX - PX, pb, &bar[s]);
      bulk_row(row + PX + NX, src, pb, &bar[s]);
    }
    for (int r = lane; r < TY; r += 32) {
      const size_t o2 = (size_t)wrapn(k + M, nz) * ps + (size_t)(j0 + r) * NX;
      bulk_row(szr + ((size_t)slot(k + M) * TY + r) * NX, f + o2, rd, &bar[s]);
    }
    if (pro)
      for (int q = lane; q < 2 * M * TY; q += 32) {
        const int p = k0 - M + q / TY, r = q % TY;
        const size_t o2 = (size_t)wrapn(p, nz) * ps + (size_t)(j0 + r) * NX;
        bulk_row(szr + ((size_t)slot(p) * TY + r) * NX, f + o2, rd, &bar[s]);
      }
  };
  if (warp == 0)
    for (int q = 0; q < S && k0 + q < k1; q++) issue(k0 + q, q, q == 0);
  constexpr int NPT = TY * NX;
  for (int k = k0; k < k1; k++) {
    const int it = k - k0, s = it % S;
    const bool ok = mbar_wait_bounded(&bar[s], (unsigned)((it / S) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(err, 1u);
        for (int q = it; q < k1 - k0 && q < it + S; q++) mbar_wait_bounded(&bar[q % S], (unsigned)((q / S) & 1));
      }
      return;
    }
    const double *yb = syb + (size_t)s * (TY + 2 * M) * RS + PX;
    const double *zr[2 * M + 1];
#pragma unroll
    for (int u = 0; u <= 2 * M; u++) zr[u] = szr + (size_t)slot(k - M + u) * TY * NX;
    const size_t base = (size_t)k * ps + (size_t)j0 * NX;
#pragma unroll
    for (int p = tid; p < NPT; p += 256) {
      const int r = p / NX, x = p % NX;
      const double *c = yb + (r + M) * RS + x;
      double ax = 0.0, ay = 0.0, az = 0.0;
#pragma unroll
      for (int t = -M; t <= M; t++) ax += st.w1[0][t + M] * c[t];
#pragma unroll
      for (int t = -M; t <= M; t++) ay += st.w1[1][t + M] * c[t * RS];
#pragma unroll
      for (int u = -M; u <= M; u++) az += st.w1[2][u + M] * zr[u + M][p];
      dx[base + p] = (TO)ax;
      dy[base + p] = (TO)ay;
      dz[base + p] = (TO)az;
    }
    __syncthreads();
    if (warp == 0 && k + S < k1) issue(k + S, s, false);
  }
}

}  // namespace he4

// fft_passes.cuh -- the register-resident x, y and z pass kernels (lengths
// 16..256, powers of two), templated on the complex type of the spectra:
// double2 (plain FP64 form) or float2 (FP32-convolution form).  Real grids
// are FP64 in both forms; the x passes convert on load and store.
#pragma once
#include <cuda_pipeline.h>

#include <type_traits>

#include "common.cuh"
#include "fft_reg.cuh"

namespace he4 {

constexpr int kRegThreads = 256;
constexpr int kRegBatch = 8;

// Four-step split N = N1 * N2 of the register path: N2 must be a multiple
// of N1 and both must have a codelet (2, 4, 8, 16).  The first choice is the
// default; the tile autotuner may pick the other.
inline int reg_default_n1(int n) { return n == 64 ? 8 : n == 128 ? 8 : n == 256 ? 16 : 4; }
inline bool reg_n1_ok(int n, int n1) {
  switch (n) {
    case 16: return n1 == 4 || n1 == 2;
    case 32: return n1 == 4 || n1 == 2;
    case 64: return n1 == 8 || n1 == 4;
    case 128: return n1 == 8;
    case 256: return n1 == 16;
    default: return false;
  }
}
inline bool reg_ok(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256; }

// pencil enumeration for the y and z passes over a half spectrum
// [nz][ny][nxh].  Pencils are (kx, o) pairs, o = z for the y pass and o = y
// for the z pass.  Tiles of W pencils with consecutive kx come first; the
// nxh mod W leftover columns are grouped across o in the last tiles.
struct PencilMap {
  int nxh, nother, W;
  long so;  // stride between consecutive o
};

__device__ __forceinline__ long pencil_offset(const PencilMap &m, long pid, int *kx_out, int *o_out) {
  const int nfull = m.nxh / m.W;
  const long main = (long)nfull * m.W * m.nother;
  const long total = (long)m.nxh * m.nother;
  if (pid >= total) return -1;
  int kx, o;
  if (pid < main) {
    const long per = (long)nfull * m.W;
    o = (int)(pid / per);
    kx = (int)(pid - (long)o * per);
  } else {
    const int tw = m.nxh - nfull * m.W;
    const long r = pid - main;
    o = (int)(r / tw);
    kx = nfull * m.W + (int)(r - (long)o * tw);
  }
  *kx_out = kx;
  *o_out = o;
  return (long)o * m.so + kx;
}

constexpr int kMaxOut = 6;
template <typename C2>
struct ZOutT {
  C2 *out;
  const typename regfft::Re<C2>::type *kern;
  double coef;
  int dsym_axis;
  int boxz;  // store only the z planes of the force box
};
template <typename C2>
struct ZGroupT {
  const C2 *in;
  int nout;
  // xy_shared: three outputs with one kernel and coefficient and the
  // derivative symbols of axes z, x, y in that order.  D_x(kx) and D_y(ky)
  // are constant along a z pencil, so the x and y outputs are
  // i D IFFT_z(coef K X): the x output's inverse transform also writes the
  // y output, and the kernels run two transforms instead of three
  int xy_shared;
  ZOutT<C2> o[kMaxOut];
};

template <typename C2>
struct YRegArgs {
  PencilMap map;
  long sf;
  const C2 *tw;
  const BoxPair *box;  // non-null: only pencils whose z lies in the force box
  int nz;
  C2 *buf[kRegBatch];
};

template <typename C2>
struct ZRegArgs {
  PencilMap map;
  long sf;
  int nx, ny, nz;
  const typename regfft::Re<C2>::type *dsym;
  const C2 *tw;
  const BoxPair *box;  // for outputs with boxz
  ZGroupT<C2> g[kRegBatch];
};

template <typename C2>
struct XRegArgs {
  int nxh;
  long nrow;
  double scale;
  const C2 *tw;
  const BoxPair *box;  // non-null (C2R): only rows (y, z) inside the force box
  int ny, nz;
  const void *rin[kRegBatch];  // double, or float (TI) for the R2C of real32 grids
  C2 *cout[kRegBatch];
  const C2 *cin[kRegBatch];
  void *rout[kRegBatch];  // double, or float (TO) for the C2R into real32 grids
  XLoad ld;               // R2C: how input rows are formed
};

// one input element of the R2C pass (XLoad; OP is the compile-time op, TI
// the type of the real32-able grids)
template <int OP, typename TI>
__device__ __forceinline__ double xload(const XLoad &ld, const TI *__restrict__ in, long i) {
  if (OP == XLOAD_ALFA) return (1.0 - (double)static_cast<const TI *>(ld.aux0)[i] * ld.c0) * (double)in[i];
  if (OP == XLOAD_CORR) {
    const double d = static_cast<const double *>(ld.aux0)[i], c = (double)static_cast<const TI *>(ld.aux1)[i];
    return d * c * (ld.c0 + ld.c1 * c);
  }
  return (double)in[i];
}

// the same element as the spectrum's scalar T; with float spectra and float
// grids the source is formed in FP32 (float <-> double conversions run at a
// quarter of the FP64 rate on this GPU, and the spectrum keeps 24 bits
// anyway); c0f / c1f are ld.c0 / ld.c1 rounded to float once per thread
template <int OP, typename TI, typename T>
__device__ __forceinline__ T xload_t(const XLoad &ld, const TI *__restrict__ in, long i, float c0f, float c1f) {
  if constexpr (std::is_same<T, float>::value && std::is_same<TI, float>::value) {
    if (OP == XLOAD_ALFA) return fmaf(-static_cast<const float *>(ld.aux0)[i], c0f, 1.0f) * in[i];
    if (OP == XLOAD_CORR) {
      const float d = (float)static_cast<const double *>(ld.aux0)[i], c = static_cast<const float *>(ld.aux1)[i];
      return d * c * fmaf(c1f, c, c0f);
    }
    return in[i];
  } else {
    return (T)xload<OP, TI>(ld, in, i);
  }
}

template <int N, typename C2>
__device__ __forceinline__ void load_tw_n(C2 *s_tw, const C2 *__restrict__ g_tw) {
  for (int t = threadIdx.x; t < N; t += blockDim.x) s_tw[t] = g_tw[t];
}

template <int N, int N1, typename C2>
inline size_t smem_yz_reg() {
  constexpr int W = kRegThreads / N1;
  return sizeof(C2) * ((size_t)N * W + N) + (sizeof(long) + 2 * sizeof(int)) * W;
}
template <int N, int N1, typename C2>
inline size_t smem_x_reg() {
  constexpr int N2 = N / N1, P = kRegThreads / N1;
  return sizeof(C2) * ((size_t)P * N2 * (N1 + 1) + N);
}
template <int N, int N1, bool SINGLE, typename C2>
inline size_t smem_zconv() {
  using T = typename regfft::Re<C2>::type;
  constexpr int W = kRegThreads / N1;
  return sizeof(C2) * ((size_t)N * W + N) + sizeof(T) * (SINGLE ? 1 : 2) * (size_t)N * W +
         (sizeof(long) + 2 * sizeof(int)) * W;
}

// In-place transform of strided pencils (y pass, or z without multiply),
// persistent and software-pipelined: each CTA walks the
// pencil tiles blockIdx.x, blockIdx.x + gridDim.x, ... and loads the next
// tile's values into registers before transforming the current one, so the
// next tile's loads are in flight during the current tile's FFT and stores.
template <int N, int N1, bool INV, typename C2>
__global__ void __launch_bounds__(kRegThreads, sizeof(C2) == 8 ? 2 : 1) k_yz_pipe(YRegArgs<C2> a) {
  constexpr int N2 = N / N1, W = kRegThreads / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *S = reinterpret_cast<C2 *>(smem_raw), *tw = S + N * W;
  load_tw_n<N>(tw, a.tw);
  __syncthreads();
  const int w = threadIdx.x % W, j1 = threadIdx.x / W;
  C2 *data = a.buf[blockIdx.y];
  const long ntiles = (a.map.nxh * (long)a.map.nother + W - 1) / W;
  auto pencil = [&](long tile) -> long {
    if (tile >= ntiles) return -1;
    int kx, o;
    long of = pencil_offset(a.map, tile * W + w, &kx, &o);
    if (a.box && of >= 0) {
      int lo, hi;
      force_range(a.box, 2, a.nz, &lo, &hi);
      if (o < lo || o > hi) of = -1;
    }
    return of;
  };
  long t = blockIdx.x;
  long off = pencil(t);
  C2 v[N2];
#pragma unroll
  for (int j2 = 0; j2 < N2; j2++) v[j2] = (off >= 0) ? data[off + (j1 + N1 * j2) * a.sf] : regfft::mk<C2>(0, 0);
  regfft::LayoutYZ lay{W, w};
  for (; t < ntiles; t += gridDim.x) {
    const long offn = pencil(t + gridDim.x);
    C2 vn[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++)
      vn[j2] = (offn >= 0) ? data[offn + (j1 + N1 * j2) * a.sf] : regfft::mk<C2>(0, 0);
    regfft::fwd2<N, N1, INV>(v, S, lay, j1, tw);
    if (off >= 0) {
#pragma unroll
      for (int c = 0; c < N2 / N1; c++)
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) data[off + ((j1 + N1 * c) + N2 * k1) * a.sf] = v[c * N1 + k1];
    }
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = vn[j2];
    off = offn;
  }
}

// z pass: one input per group, FFT_z once, then for each output
// IFFT_z(coef * K(k) [* i D(k)] * X).  The kernel values K of an output are
// copied to shared memory with cp.async one output ahead (the first ones
// before the input is even loaded), so their latency hides behind the FFT
// work.  SINGLE: one output, multiplied in place (fewer registers).
template <int N, int N1, bool SINGLE, typename C2>
__global__ void __launch_bounds__(kRegThreads) k_zconv_reg(ZRegArgs<C2> a) {
  using T = typename regfft::Re<C2>::type;
  constexpr int N2 = N / N1, W = kRegThreads / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *S = reinterpret_cast<C2 *>(smem_raw), *tw = S + N * W;
  T *Ks = reinterpret_cast<T *>(tw + N);  // [SINGLE ? 1 : 2][N][W]
  long *offs = reinterpret_cast<long *>(Ks + (SINGLE ? 1 : 2) * N * W);
  int *kxs = reinterpret_cast<int *>(offs + W);
  int *kys = kxs + W;
  load_tw_n<N>(tw, a.tw);
  if (threadIdx.x < W) {
    int kx = 0, o = 0;
    offs[threadIdx.x] = pencil_offset(a.map, (long)blockIdx.y * W + threadIdx.x, &kx, &o);
    kxs[threadIdx.x] = kx;
    kys[threadIdx.x] = o;
  }
  __syncthreads();
  const ZGroupT<C2> &G = a.g[blockIdx.x];
  const bool xys = !SINGLE && G.xy_shared;
  const int nout = SINGLE ? 1 : (xys ? 2 : G.nout);
  auto prefetch = [&](int o) {
    const T *kern = G.o[o].kern;
    if (!kern) return;
    T *dst = Ks + (SINGLE ? 0 : (o & 1)) * N * W;
    for (int e = threadIdx.x; e < N * W; e += kRegThreads) {
      const int ww = e % W, k = e / W;
      const long of = offs[ww];
      if (of >= 0) __pipeline_memcpy_async(dst + e, kern + of + (long)k * a.sf, sizeof(T));
    }
  };
  prefetch(0);
  __pipeline_commit();
  const int w = threadIdx.x % W, j1 = threadIdx.x / W;
  const long off = offs[w];
  C2 v[N2];
#pragma unroll
  for (int j2 = 0; j2 < N2; j2++) v[j2] = (off >= 0) ? G.in[off + (j1 + N1 * j2) * a.sf] : regfft::mk<C2>(0, 0);
  regfft::LayoutYZ lay{W, w};
  regfft::fwd2<N, N1, false>(v, S, lay, j1, tw);
  const T dx = (off >= 0) ? a.dsym[kxs[w]] : T(0);
  const T dy = (off >= 0) ? a.dsym[a.nx + kys[w]] : T(0);
  for (int o = 0; o < nout; o++) {
    if (!SINGLE && o + 1 < nout) prefetch(o + 1);
    __pipeline_commit();
    __pipeline_wait_prior(1);
    __syncthreads();
    const ZOutT<C2> Z = G.o[o];
    const T *K = Ks + (SINGLE ? 0 : (o & 1)) * N * W;
    C2 u[SINGLE ? 1 : N2];
    C2 *x = SINGLE ? v : u;
    const T coef = (T)Z.coef;
#pragma unroll
    for (int c = 0; c < N2 / N1; c++)
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) {
        const int k = (j1 + N1 * c) + N2 * k1;
        T cf = coef;
        if (Z.kern && off >= 0) cf *= K[k * W + w];
        C2 y = regfft::scale(v[c * N1 + k1], cf);
        if (Z.dsym_axis >= 0 && !(xys && o == 1)) {
          const T ds = (Z.dsym_axis == 0) ? dx : (Z.dsym_axis == 1) ? dy : a.dsym[a.nx + a.ny + k];
          y = regfft::mk<C2>(-y.y * ds, y.x * ds);
        }
        x[c * N1 + k1] = y;
      }
    regfft::bwd2<N, N1, true>(*reinterpret_cast<C2(*)[N2]>(x), S, lay, j1, tw);
    if (off >= 0) {
      int zlo = 0, zhi = N - 1;
      if (Z.boxz) force_range(a.box, 2, a.nz, &zlo, &zhi);
      if (xys && o == 1) {  // x and y outputs: i D_x and i D_y times the transform
        C2 *oy = G.o[2].out;
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) {
          const int z = j1 + N1 * n2;
          if (z >= zlo && z <= zhi) {
            Z.out[off + z * a.sf] = regfft::mk<C2>(-x[n2].y * dx, x[n2].x * dx);
            oy[off + z * a.sf] = regfft::mk<C2>(-x[n2].y * dy, x[n2].x * dy);
          }
        }
      } else {
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) {
          const int z = j1 + N1 * n2;
          if (z >= zlo && z <= zhi) Z.out[off + z * a.sf] = x[n2];
        }
      }
    }
  }
}

// Persistent, software-pipelined z pass: each CTA walks the pencil tiles of
// one group; the next tile's input and the current output's kernel values
// are loaded into registers ahead of the transforms that need them.
template <int N, int N1, bool SINGLE, typename C2>
// FP32: two CTAs per SM (128 registers) beat one CTA with no spills; FP64
// spills heavily at that bound, so it keeps one CTA per SM
__global__ void __launch_bounds__(kRegThreads, sizeof(C2) == 8 ? 2 : 1) k_zconv_pipe(ZRegArgs<C2> a) {
  using T = typename regfft::Re<C2>::type;
  constexpr int N2 = N / N1, W = kRegThreads / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *S = reinterpret_cast<C2 *>(smem_raw), *tw = S + N * W;
  load_tw_n<N>(tw, a.tw);
  __syncthreads();
  const ZGroupT<C2> &G = a.g[blockIdx.x];
  const bool xys = !SINGLE && G.xy_shared;
  const int nout = SINGLE ? 1 : (xys ? 2 : G.nout);
  const int w = threadIdx.x % W, j1 = threadIdx.x / W;
  const long ntiles = (a.map.nxh * (long)a.map.nother + W - 1) / W;
  auto pencil = [&](long tile, int *kx, int *ky) -> long {
    *kx = 0;
    *ky = 0;
    if (tile >= ntiles) return -1;
    return pencil_offset(a.map, tile * W + w, kx, ky);
  };
  auto load_k = [&](const T *kern, long off, T (&K)[N2]) {
#pragma unroll
    for (int c = 0; c < N2 / N1; c++)
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) {
        const int k = (j1 + N1 * c) + N2 * k1;
        K[c * N1 + k1] = (kern && off >= 0) ? __ldg(kern + off + (long)k * a.sf) : T(0);
      }
  };
  regfft::LayoutYZ lay{W, w};
  long t = blockIdx.y;
  int kx, ky;
  long off = pencil(t, &kx, &ky);
  C2 v[N2];
#pragma unroll
  for (int j2 = 0; j2 < N2; j2++) v[j2] = (off >= 0) ? G.in[off + (j1 + N1 * j2) * a.sf] : regfft::mk<C2>(0, 0);
  for (; t < ntiles; t += gridDim.y) {
    int kxn, kyn;
    const long offn = pencil(t + gridDim.y, &kxn, &kyn);
    C2 vn[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++)
      vn[j2] = (offn >= 0) ? G.in[offn + (j1 + N1 * j2) * a.sf] : regfft::mk<C2>(0, 0);
    T K[N2];
    load_k(G.o[0].kern, off, K);
    regfft::fwd2<N, N1, false>(v, S, lay, j1, tw);
    const T dx = (off >= 0) ? a.dsym[kx] : T(0);
    const T dy = (off >= 0) ? a.dsym[a.nx + ky] : T(0);
    for (int o = 0; o < nout; o++) {
      T Kn[SINGLE ? 1 : N2];
      if (!SINGLE && o + 1 < nout) load_k(G.o[o + 1].kern, off, *reinterpret_cast<T(*)[N2]>(Kn));
      const ZOutT<C2> Z = G.o[o];
      C2 u[SINGLE ? 1 : N2];
      C2 *x = SINGLE ? v : u;
      const T coef = (T)Z.coef;
#pragma unroll
      for (int c = 0; c < N2 / N1; c++)
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) {
          const int k = (j1 + N1 * c) + N2 * k1;
          T cf = coef;
          if (Z.kern && off >= 0) cf *= K[c * N1 + k1];
          C2 y = regfft::scale(v[c * N1 + k1], cf);
          if (Z.dsym_axis >= 0 && !(xys && o == 1)) {
            const T ds = (Z.dsym_axis == 0) ? dx : (Z.dsym_axis == 1) ? dy : a.dsym[a.nx + a.ny + k];
            y = regfft::mk<C2>(-y.y * ds, y.x * ds);
          }
          x[c * N1 + k1] = y;
        }
      regfft::bwd2<N, N1, true>(*reinterpret_cast<C2(*)[N2]>(x), S, lay, j1, tw);
      if (off >= 0) {
        int zlo = 0, zhi = N - 1;
        if (Z.boxz) force_range(a.box, 2, a.nz, &zlo, &zhi);
        if (xys && o == 1) {  // x and y outputs: i D_x and i D_y times the transform
          C2 *oy = G.o[2].out;
#pragma unroll
          for (int n2 = 0; n2 < N2; n2++) {
            const int z = j1 + N1 * n2;
            if (z >= zlo && z <= zhi) {
              Z.out[off + z * a.sf] = regfft::mk<C2>(-x[n2].y * dx, x[n2].x * dx);
              oy[off + z * a.sf] = regfft::mk<C2>(-x[n2].y * dy, x[n2].x * dy);
            }
          }
        } else {
#pragma unroll
          for (int n2 = 0; n2 < N2; n2++) {
            const int z = j1 + N1 * n2;
            if (z >= zlo && z <= zhi) Z.out[off + z * a.sf] = x[n2];
          }
        }
      }
      if (!SINGLE) {
#pragma unroll
        for (int e = 0; e < N2; e++) K[e] = Kn[SINGLE ? 0 : e];
      }
    }
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = vn[j2];
    off = offn;
    kx = kxn;
    ky = kyn;
  }
}

template <int N, int N1, typename C2>
inline size_t smem_zpipe() {
  constexpr int W = kRegThreads / N1;
  return sizeof(C2) * ((size_t)N * W + N);
}

// x pass R2C: two real rows per complex pencil, Hermitian split
template <int N, int N1, typename C2, int OP = XLOAD_PLAIN, typename TI = double>
__global__ void __launch_bounds__(kRegThreads) k_xr2c_reg(XRegArgs<C2> a) {
  using T = typename regfft::Re<C2>::type;
  constexpr int N2 = N / N1, P = kRegThreads / N1, SP = N2 * (N1 + 1);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *S = reinterpret_cast<C2 *>(smem_raw), *tw = S + P * SP;
  load_tw_n<N>(tw, a.tw);
  __syncthreads();
  const int j1 = threadIdx.x % N1, p = threadIdx.x / N1;
  const long ra = (long)blockIdx.x * 2 * P + 2 * p, rb = ra + 1;
  const TI *in = static_cast<const TI *>(a.rin[blockIdx.y]);
  C2 *out = a.cout[blockIdx.y];
  // loads from clamped rows (unconditional, so they issue together), rows
  // past the end zeroed afterwards
  const long rac = ra < a.nrow ? ra : a.nrow - 1, rbc = rb < a.nrow ? rb : a.nrow - 1;
  const float c0f = (float)a.ld.c0, c1f = (float)a.ld.c1;
  T xa[N2], xb[N2];
#pragma unroll
  for (int j2 = 0; j2 < N2; j2++) {
    const int x = j1 + N1 * j2;
    xa[j2] = xload_t<OP, TI, T>(a.ld, in, rac * N + x, c0f, c1f);
    xb[j2] = xload_t<OP, TI, T>(a.ld, in, rbc * N + x, c0f, c1f);
  }
  C2 v[N2];
#pragma unroll
  for (int j2 = 0; j2 < N2; j2++)
    v[j2] = regfft::mk<C2>((ra < a.nrow) ? xa[j2] : T(0), (rb < a.nrow) ? xb[j2] : T(0));
  regfft::LayoutX lay{p * SP};
  regfft::fwd2<N, N1, false>(v, S, lay, j1, tw);
  C2 *Sp = S + p * SP;
#pragma unroll
  for (int c = 0; c < N2 / N1; c++)
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) Sp[(j1 + N1 * c) + N2 * k1] = v[c * N1 + k1];
  __syncthreads();
  for (int k = j1; k <= N / 2; k += N1) {
    const C2 zk = Sp[k];
    const C2 zmc = Sp[(N - k) & (N - 1)];
    const C2 zm = regfft::mk<C2>(zmc.x, -zmc.y);
    const C2 A = regfft::scale(regfft::add(zk, zm), T(0.5));
    const C2 d = regfft::scale(regfft::sub(zk, zm), T(0.5));
    if (ra < a.nrow) out[ra * a.nxh + k] = A;
    if (rb < a.nrow) out[rb * a.nxh + k] = regfft::mk<C2>(d.y, -d.x);
  }
}

// x pass C2R: Hermitian extension of two half spectra, inverse, two rows
template <int N, int N1, typename C2, typename TO = double>
__global__ void __launch_bounds__(kRegThreads) k_xc2r_reg(XRegArgs<C2> a) {
  constexpr int N2 = N / N1, P = kRegThreads / N1, SP = N2 * (N1 + 1);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *S = reinterpret_cast<C2 *>(smem_raw), *tw = S + P * SP;
  load_tw_n<N>(tw, a.tw);
  const int j1 = threadIdx.x % N1, p = threadIdx.x / N1;
  const long ra = (long)blockIdx.x * 2 * P + 2 * p, rb = ra + 1;
  // rows outside the force box (when restricted) are neither read nor written
  bool ina = ra < a.nrow, inb = rb < a.nrow;
  if (a.box) {
    int ylo, yhi, zlo, zhi;
    force_range(a.box, 1, a.ny, &ylo, &yhi);
    force_range(a.box, 2, a.nz, &zlo, &zhi);
    const int ya = (int)(ra % a.ny), za = (int)(ra / a.ny), yb = (int)(rb % a.ny), zb = (int)(rb / a.ny);
    ina = ina && ya >= ylo && ya <= yhi && za >= zlo && za <= zhi;
    inb = inb && yb >= ylo && yb <= yhi && zb >= zlo && zb <= zhi;
    if (!__syncthreads_or(ina || inb)) return;
  }
  const C2 *in = a.cin[blockIdx.y];
  TO *out = static_cast<TO *>(a.rout[blockIdx.y]);
  C2 *Sp = S + p * SP;
  // the Hermitian extension of one row pair into S: X = row a, Y = row b
  auto put = [&](int k, C2 X, C2 Y) {
    if (k == 0 || 2 * k == N) {  // DC / Nyquist of a real transform: drop Im
      X.y = 0;
      Y.y = 0;
    }
    Sp[k] = regfft::mk<C2>(X.x - Y.y, X.y + Y.x);
    if (k > 0 && N - k >= a.nxh) Sp[N - k] = regfft::mk<C2>(X.x + Y.y, Y.x - X.y);
  };
  for (int k = j1; k < a.nxh; k += N1)
    put(k, ina ? in[ra * a.nxh + k] : regfft::mk<C2>(0, 0), inb ? in[rb * a.nxh + k] : regfft::mk<C2>(0, 0));
  __syncthreads();
  C2 v[N2];
#pragma unroll
  for (int c = 0; c < N2 / N1; c++)
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) v[c * N1 + k1] = Sp[(j1 + N1 * c) + N2 * k1];
  __syncthreads();
  regfft::LayoutX lay{p * SP};
  regfft::bwd2<N, N1, true>(v, S, lay, j1, tw);
  const double sc = a.scale;
  if constexpr (std::is_same<TO, float>::value && std::is_same<C2, float2>::value) {
    // float spectra into float grids: no double round trip (the same
    // result whenever the scale is a power of two, as the callers' 1.0 is)
    const float scf = (float)sc;
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) {
      const int x = j1 + N1 * n2;
      if (ina) out[ra * N + x] = v[n2].x * scf;
      if (inb) out[rb * N + x] = v[n2].y * scf;
    }
  } else {
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) {
      const int x = j1 + N1 * n2;
      if (ina) out[ra * N + x] = (TO)((double)v[n2].x * sc);
      if (inb) out[rb * N + x] = (TO)((double)v[n2].y * sc);
    }
  }
}

// z pass summing several convolutions into one output:
//   out = IFFT_z( sum_j coef_j K_j(k) FFT_z(in_j) )
// Each term's kernel values are copied to shared memory with cp.async while
// the term's input is loaded and transformed.
constexpr int kMaxTerms = 4;
template <typename C2>
struct ZTermT {
  const C2 *in;
  const typename regfft::Re<C2>::type *kern;
  double coef;
};
template <typename C2>
struct ZSumArgs {
  PencilMap map;
  long sf;
  const C2 *tw;
  int nterm;
  ZTermT<C2> t[kMaxTerms];
  C2 *out;
};

template <int N, int N1, typename C2>
inline size_t smem_zsum() {
  using T = typename regfft::Re<C2>::type;
  constexpr int W = kRegThreads / N1;
  return sizeof(C2) * ((size_t)N * W + N) + sizeof(T) * (size_t)N * W + sizeof(long) * W;
}

template <int N, int N1, typename C2>
__global__ void __launch_bounds__(kRegThreads) k_zsum_reg(ZSumArgs<C2> a) {
  using T = typename regfft::Re<C2>::type;
  constexpr int N2 = N / N1, W = kRegThreads / N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *S = reinterpret_cast<C2 *>(smem_raw), *tw = S + N * W;
  T *Ks = reinterpret_cast<T *>(tw + N);  // [N][W]
  long *offs = reinterpret_cast<long *>(Ks + N * W);
  load_tw_n<N>(tw, a.tw);
  if (threadIdx.x < W) {
    int kx, o;
    offs[threadIdx.x] = pencil_offset(a.map, (long)blockIdx.x * W + threadIdx.x, &kx, &o);
  }
  __syncthreads();
  auto prefetch = [&](int j) {
    const T *kern = a.t[j].kern;
    for (int e = threadIdx.x; e < N * W; e += kRegThreads) {
      const int ww = e % W, k = e / W;
      const long of = offs[ww];
      if (of >= 0) __pipeline_memcpy_async(Ks + e, kern + of + (long)k * a.sf, sizeof(T));
    }
  };
  prefetch(0);
  __pipeline_commit();
  const int w = threadIdx.x % W, j1 = threadIdx.x / W;
  const long off = offs[w];
  regfft::LayoutYZ lay{W, w};
  C2 acc[N2];
#pragma unroll
  for (int e = 0; e < N2; e++) acc[e] = regfft::mk<C2>(0, 0);
  for (int j = 0; j < a.nterm; j++) {
    const C2 *in = a.t[j].in;
    C2 v[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; j2++) v[j2] = (off >= 0) ? in[off + (j1 + N1 * j2) * a.sf] : regfft::mk<C2>(0, 0);
    regfft::fwd2<N, N1, false>(v, S, lay, j1, tw);
    __pipeline_wait_prior(0);
    __syncthreads();  // term j's kernel values are in Ks
    const T coef = (T)a.t[j].coef;
#pragma unroll
    for (int c = 0; c < N2 / N1; c++)
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) {
        const int k = (j1 + N1 * c) + N2 * k1;
        const T cf = (off >= 0) ? coef * Ks[k * W + w] : T(0);
        const C2 x = v[c * N1 + k1];
        acc[c * N1 + k1] = regfft::mk<C2>(acc[c * N1 + k1].x + cf * x.x, acc[c * N1 + k1].y + cf * x.y);
      }
    if (j + 1 < a.nterm) {
      __syncthreads();  // everyone is done with Ks
      prefetch(j + 1);
    }
    __pipeline_commit();
  }
  regfft::bwd2<N, N1, true>(acc, S, lay, j1, tw);
  if (off >= 0) {
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) a.out[off + (j1 + N1 * n2) * a.sf] = acc[n2];
  }
}

template <int N, int N1, typename C2>
inline int reg_attrs() {
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_zsum_reg<N, N1, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_zsum<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_yz_pipe<N, N1, true, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_yz_reg<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_yz_pipe<N, N1, false, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_yz_reg<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_zconv_pipe<N, N1, true, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_zpipe<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_zconv_pipe<N, N1, false, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_zpipe<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_zconv_reg<N, N1, false, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_zconv<N, N1, false, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_xr2c_reg<N, N1, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_x_reg<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_xr2c_reg<N, N1, C2, XLOAD_ALFA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_x_reg<N, N1, C2>()));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_xr2c_reg<N, N1, C2, XLOAD_CORR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_x_reg<N, N1, C2>()));
  if constexpr (sizeof(C2) == 8) {  // real32 grids exist in the FP32-convolution form only
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_xr2c_reg<N, N1, C2, XLOAD_PLAIN, float>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x_reg<N, N1, C2>()));
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_xr2c_reg<N, N1, C2, XLOAD_ALFA, float>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x_reg<N, N1, C2>()));
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_xr2c_reg<N, N1, C2, XLOAD_CORR, float>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x_reg<N, N1, C2>()));
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_xc2r_reg<N, N1, C2, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_x_reg<N, N1, C2>()));
  }
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_xc2r_reg<N, N1, C2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_x_reg<N, N1, C2>()));
  return HE4_OK;
}

// run the statement with NN = n and N1_ = n1 (a pair reg_n1_ok accepts)
#define HE4_REG_CASE(a, b, ...)                   \
  if (n_ == a && n1_ == b) {                      \
    constexpr int NN = a, N1_ = b;                \
    __VA_ARGS__;                                  \
  } else
#define HE4_REG_SWITCH(n, n1, ...)                \
  do {                                            \
    const int n_ = (n), n1_ = (n1);               \
    HE4_REG_CASE(16, 4, __VA_ARGS__)              \
    HE4_REG_CASE(16, 2, __VA_ARGS__)              \
    HE4_REG_CASE(32, 4, __VA_ARGS__)              \
    HE4_REG_CASE(32, 2, __VA_ARGS__)              \
    HE4_REG_CASE(64, 8, __VA_ARGS__)              \
    HE4_REG_CASE(64, 4, __VA_ARGS__)              \
    HE4_REG_CASE(128, 8, __VA_ARGS__)             \
    HE4_REG_CASE(256, 16, __VA_ARGS__) {          \
      set_error("no register FFT for %d = %d x %d", n_, n1_, n_ / (n1_ ? n1_ : 1)); \
      return HE4_E_UNSUPPORTED;                   \
    }                                             \
  } while (0)

}  // namespace he4

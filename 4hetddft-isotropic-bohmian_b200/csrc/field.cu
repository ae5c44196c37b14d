// field.cu -- the mean-field evaluation: potenimp, poten (with term_alfa)
// and forceimp (potenimp.f90:1-73, poten.f90:5-129, term_alfa.f90:5-117,
// derden.f90:5-31, denpart/ironing potenimp.f90:294-371).
//
// Spectra: spec[0] holds the x/y-transformed density (fden before its z
// transform) for the whole evaluation; forceimp reuses it, since for the
// periodic stencils (icon=8) FFT(d_i rho) = i D_i(k) FFT(rho) exactly, D_i
// being the symbol of the npd-point first-derivative stencil.
#include <string.h>

#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "common.cuh"
#include "stencil.cuh"

namespace he4 {

static Geo geo(const Handle *h) { return Geo{h->nx, h->ny, h->nz, zpad_of(h->p.icon)}; }

// derden (derden.f90:26-28)
__global__ void k_grad(const double *__restrict__ f, double *dx, double *dy, double *dz, Stencil st, Geo g) {
  HE4_IJK(g);
  dx[t] = stencil_axis(f, st, 1, g, i, j, k, 0);
  dy[t] = stencil_axis(f, st, 1, g, i, j, k, 1);
  dz[t] = stencil_axis(f, st, 1, g, i, j, k, 2);
}

// The same stencils for a compile-time half width M, one CTA of 32 x 8
// threads marching over ZB consecutive z planes of its (x, y) tile: the z
// taps come from a register queue of each thread's column (ZB + 2M loads
// instead of ZB (2M + 1)), the x and y taps from a shared-memory copy of the
// plane's tile with its periodic halo (about 2 loads per point instead of
// 4M).  Every tap is summed in the order of stencil_axis, so the results are
// those of the one-plane kernels.
constexpr int kZB = 8;   // z extent the tile indices are checked for
constexpr int kZBg = 4;  // planes per CTA of the gradient stencil

struct OtArgs {
  double cp4, cpp4, den0s, h2o2m4, alphas, c_solid, beta, den_m;
};
}  // namespace he4
#include "stream_stencil.cuh"
namespace he4 {

// periodic index for i in [-n, 2n)
__device__ __forceinline__ int wrap2(int i, int n) { return i < 0 ? i + n : (i >= n ? (i >= 2 * n ? i - 2 * n : i - n) : i); }

// column values k0-M .. k0+ZB-1+M of f at (i, j); f double or float
template <int M, int ZB, typename T>
__device__ __forceinline__ void load_column(const T *__restrict__ f, const Geo &g, int i, int j, int k0,
                                            double (&q)[ZB + 2 * M]) {
  const T *col = f + (size_t)j * g.nx + i;
  const size_t ps = (size_t)g.ny * g.nx;
#pragma unroll
  for (int u = 0; u < ZB + 2 * M; u++) q[u] = (double)__ldg(col + (size_t)wrap2(k0 - M + u, g.nz) * ps);
}

// Plane k of f into the tile s[8 + 2 HY][32 + 2 HX] around (i0, j0): the
// centre cell of each thread (`centre` when it holds it, from global memory
// otherwise), an x halo of HX cells on both sides of each row and a y halo
// of HY rows above and below each column, all periodic.  Corners are not
// filled (the stencils are one-dimensional).
template <int HX, int HY, typename T>
__device__ __forceinline__ void fill_tile(const T *__restrict__ f, const Geo &g, int i0, int j0, int k,
                                          bool have, double centre, double (*s)[32 + 2 * HX]) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const T *plane = f + (size_t)k * g.ny * g.nx;
  const int gi = wrap2(i0 + tx, g.nx), gj = wrap2(j0 + ty, g.ny);
  s[ty + HY][tx + HX] = have ? centre : (double)__ldg(plane + (size_t)gj * g.nx + gi);
  if (HX > 0 && tx < HX) {
    s[ty + HY][tx] = (double)__ldg(plane + (size_t)gj * g.nx + wrap2(i0 - HX + tx, g.nx));
    s[ty + HY][tx + 32 + HX] = (double)__ldg(plane + (size_t)gj * g.nx + wrap2(i0 + 32 + tx, g.nx));
  }
  if (HY > 0 && ty < HY) {
    s[ty][tx + HX] = (double)__ldg(plane + (size_t)wrap2(j0 - HY + ty, g.ny) * g.nx + gi);
    s[ty + 8 + HY][tx + HX] = (double)__ldg(plane + (size_t)wrap2(j0 + 8 + ty, g.ny) * g.nx + gi);
  }
}

template <int M, int ZB, typename TO = double>
__global__ void __launch_bounds__(256) k_grad_z(const double *__restrict__ f, TO *dx, TO *dy, TO *dz, Stencil st,
                                                Geo g) {
  __shared__ double s[8 + 2 * M][32 + 2 * M];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 8, k0 = blockIdx.z * ZB;
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i < g.nx && j < g.ny;
  const size_t ps = (size_t)g.ny * g.nx;
  const int gi = wrap2(i, g.nx), gj = wrap2(j, g.ny);
  // every global load of the ZB planes up front: the z column (queue), the
  // x halo (threads tx < M) and the y halo (threads ty < M) of each plane;
  // the planes then only wait for shared memory
  double q[ZB + 2 * M], xl[ZB], xr[ZB], yl[ZB], yr[ZB];
  load_column<M, ZB>(f, g, gi, gj, k0, q);
#pragma unroll
  for (int zz = 0; zz < ZB; zz++) {
    const double *plane = f + (size_t)wrap2(k0 + zz, g.nz) * ps;
    xl[zz] = xr[zz] = yl[zz] = yr[zz] = 0.0;
    if (tx < M) {
      xl[zz] = __ldg(plane + (size_t)gj * g.nx + wrap2(i0 - M + tx, g.nx));
      xr[zz] = __ldg(plane + (size_t)gj * g.nx + wrap2(i0 + 32 + tx, g.nx));
    }
    if (ty < M) {
      yl[zz] = __ldg(plane + (size_t)wrap2(j0 - M + ty, g.ny) * g.nx + gi);
      yr[zz] = __ldg(plane + (size_t)wrap2(j0 + 8 + ty, g.ny) * g.nx + gi);
    }
  }
#pragma unroll
  for (int zz = 0; zz < ZB; zz++) {
    const int k = k0 + zz;
    if (k >= g.nz) break;
    __syncthreads();
    s[ty + M][tx + M] = q[zz + M];
    if (tx < M) {
      s[ty + M][tx] = xl[zz];
      s[ty + M][tx + 32 + M] = xr[zz];
    }
    if (ty < M) {
      s[ty][tx + M] = yl[zz];
      s[ty + 8 + M][tx + M] = yr[zz];
    }
    __syncthreads();
    if (!in) continue;
    double ax = 0.0, ay = 0.0, az = 0.0;
#pragma unroll
    for (int t = -M; t <= M; t++) ax += st.w1[0][t + M] * s[ty + M][tx + M + t];
#pragma unroll
    for (int t = -M; t <= M; t++) ay += st.w1[1][t + M] * s[ty + M + t][tx + M];
#pragma unroll
    for (int u = -M; u <= M; u++) az += st.w1[2][u + M] * q[zz + M + u];
    const size_t t = ((size_t)k * g.ny + j) * g.nx + i;
    dx[t] = (TO)ax;
    dy[t] = (TO)ay;
    dz[t] = (TO)az;
  }
}

// The same with each plane's tile halo loaded inside the plane loop (the
// float-output variant of the FP32-convolution form measured faster so).
template <int M, int ZB, typename TO = double>
__global__ void __launch_bounds__(256) k_grad_z_tile(const double *__restrict__ f, TO *dx, TO *dy, TO *dz, Stencil st,
                                                Geo g) {
  __shared__ double s[8 + 2 * M][32 + 2 * M];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 8, k0 = blockIdx.z * ZB;
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i < g.nx && j < g.ny;
  double q[ZB + 2 * M];
  if (in) load_column<M, ZB>(f, g, i, j, k0, q);
#pragma unroll
  for (int zz = 0; zz < ZB; zz++) {
    const int k = k0 + zz;
    if (k >= g.nz) break;
    __syncthreads();
    fill_tile<M, M>(f, g, i0, j0, k, in, in ? q[zz + M] : 0.0, s);
    __syncthreads();
    if (!in) continue;
    double ax = 0.0, ay = 0.0, az = 0.0;
#pragma unroll
    for (int t = -M; t <= M; t++) ax += st.w1[0][t + M] * s[ty + M][tx + M + t];
#pragma unroll
    for (int t = -M; t <= M; t++) ay += st.w1[1][t + M] * s[ty + M + t][tx + M];
#pragma unroll
    for (int u = -M; u <= M; u++) az += st.w1[2][u + M] * q[zz + M + u];
    const size_t t = ((size_t)k * g.ny + j) * g.nx + i;
    dx[t] = (TO)ax;
    dy[t] = (TO)ay;
    dz[t] = (TO)az;
  }
}

// Every input of the ZB planes of a thread (the z column of h2 with its
// halo, the centres of h0 and h1, lin, den and dencg) is loaded up front:
// the kernel is bound by memory latency, not by its (algorithmic) DRAM
// traffic, so each thread keeps ~30 independent loads in flight and the
// planes then only wait for the L2-resident tile halos.
constexpr int kZBp = 4;

template <bool OTC, int M, int ZB, typename TI = double, bool UP = true>
__global__ void __launch_bounds__(256) k_pot4_merged_z(const TI *__restrict__ lin, const double *__restrict__ den,
                                                       const TI *__restrict__ dencg, const TI *__restrict__ h0,
                                                       const TI *__restrict__ h1, const TI *__restrict__ h2,
                                                       double *pot4, Stencil st, Geo g, OtArgs a) {
  __shared__ double s0[8][32 + 2 * M];   // h0 with its x halo
  __shared__ double s1[8 + 2 * M][32];   // h1 with its y halo
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 8, k0 = blockIdx.z * ZB;
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i < g.nx && j < g.ny;
  const size_t ps = (size_t)g.ny * g.nx;
  double q[ZB + 2 * M], c0[ZB], c1[ZB], ld[ZB], dd[ZB], dcg[ZB];
  // tile halos of every plane, loaded with the rest (threads tx < M: the x
  // halo of h0; threads ty < M: the y halo of h1)
  TI xl[ZB], xr[ZB], yl[ZB], yr[ZB];
  const int gi = wrap2(i, g.nx), gj = wrap2(j, g.ny);
  if (OTC && UP) {
#pragma unroll
    for (int zz = 0; zz < ZB; zz++) {
      const size_t pl = (size_t)wrap2(k0 + zz, g.nz) * ps;
      xl[zz] = xr[zz] = yl[zz] = yr[zz] = TI(0);
      if (tx < M) {
        xl[zz] = __ldg(h0 + pl + (size_t)gj * g.nx + wrap2(i0 - M + tx, g.nx));
        xr[zz] = __ldg(h0 + pl + (size_t)gj * g.nx + wrap2(i0 + 32 + tx, g.nx));
      }
      if (ty < M) {
        yl[zz] = __ldg(h1 + pl + (size_t)wrap2(j0 - M + ty, g.ny) * g.nx + gi);
        yr[zz] = __ldg(h1 + pl + (size_t)wrap2(j0 + 8 + ty, g.ny) * g.nx + gi);
      }
    }
  }
  if (in) {
    if (OTC) load_column<M, ZB>(h2, g, i, j, k0, q);
#pragma unroll
    for (int zz = 0; zz < ZB; zz++) {
      const size_t t = (size_t)wrap2(k0 + zz, g.nz) * ps + (size_t)j * g.nx + i;
      if (OTC) {
        c0[zz] = (double)__ldg(h0 + t);
        c1[zz] = (double)__ldg(h1 + t);
      }
      ld[zz] = (double)__ldg(lin + t);
      dd[zz] = __ldg(den + t);
      dcg[zz] = (double)__ldg(dencg + t);
    }
  }
  const double a0 = a.cp4 / 2.0, a1 = a.cpp4 / 3.0;
#pragma unroll
  for (int zz = 0; zz < ZB; zz++) {
    const int k = k0 + zz;
    if (k >= g.nz) break;
    if (OTC && !UP) {
      __syncthreads();
      fill_tile<M, 0>(h0, g, i0, j0, k, in, in ? c0[zz] : 0.0, s0);
      fill_tile<0, M>(h1, g, i0, j0, k, in, in ? c1[zz] : 0.0, s1);
      __syncthreads();
    } else if (OTC) {
      __syncthreads();
      const size_t pl = (size_t)k * ps + (size_t)gj * g.nx + gi;
      s0[ty][tx + M] = in ? c0[zz] : (double)__ldg(h0 + pl);
      s1[ty + M][tx] = in ? c1[zz] : (double)__ldg(h1 + pl);
      if (tx < M) {
        s0[ty][tx] = (double)xl[zz];
        s0[ty][tx + 32 + M] = (double)xr[zz];
      }
      if (ty < M) {
        s1[ty][tx] = (double)yl[zz];
        s1[ty + 8 + M][tx] = (double)yr[zz];
      }
      __syncthreads();
    }
    if (!in) continue;
    const double d = dd[zz];
    const double th = tanh(a.beta * (d - a.den_m));
    const double pen = a.c_solid * (1.0 + th + a.beta * d * (1.0 - th * th));
    const double dc = dcg[zz];
    double v = ld[zz] + dc * dc * (a0 + a1 * dc) + pen;
    if (OTC) {
      double d0 = 0.0, d1 = 0.0, d2 = 0.0;
#pragma unroll
      for (int u = -M; u <= M; u++) d0 += st.w1[0][u + M] * s0[ty][tx + M + u];
#pragma unroll
      for (int u = -M; u <= M; u++) d1 += st.w1[1][u + M] * s1[ty + M + u][tx];
#pragma unroll
      for (int u = -M; u <= M; u++) d2 += st.w1[2][u + M] * q[zz + M + u];
      v += (d0 + d1 + d2) * a.h2o2m4 * a.alphas;
    }
    pot4[((size_t)k * g.ny + j) * g.nx + i] = v;
  }
}

// ---------------------------------------------------------------------------
// poten pointwise pieces
// ---------------------------------------------------------------------------

// sto1 = den*dencg*(cp4+cpp4*dencg) (poten.f90:62-64)
__global__ void k_corr_src(const double *__restrict__ den, const double *__restrict__ dencg, double *out, size_t n,
                           OtArgs a) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = den[t] * dencg[t] * (a.cp4 + a.cpp4 * dencg[t]);
}

// penalty (poten.f90:80-81) and pot4 = delj4 + dencg^2 (a0 + a1 dencg) + sto1 (poten.f90:88-92)
__global__ void k_pot4_base(const double *__restrict__ den, const double *__restrict__ dencg,
                            const double *__restrict__ delj4, const double *__restrict__ corr, double *penalty,
                            double *pot4, size_t n, OtArgs a) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double d = den[t];
  const double th = tanh(a.beta * (d - a.den_m));
  penalty[t] = a.c_solid * (1.0 + th + a.beta * d * (1.0 - th * th));
  const double dc = dencg[t];
  const double a0 = a.cp4 / 2.0, a1 = a.cpp4 / 3.0;
  pot4[t] = delj4[t] + dc * dc * (a0 + a1 * dc) + corr[t];
}

// falfs = 1 - denalf/den0s; g_i = falfs * d_i rho (term_alfa.f90:28-36)
__global__ void k_alfa1(const double *__restrict__ denalf, const double *__restrict__ dx,
                        const double *__restrict__ dy, const double *__restrict__ dz, double *falfs, double *g0,
                        double *g1, double *g2, size_t n, OtArgs a) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double f = 1.0 - denalf[t] / a.den0s;
  falfs[t] = f;
  g0[t] = f * dx[t];
  g1[t] = f * dy[t];
  g2[t] = f * dz[t];
}

// s = sum_i d_i rho * int_i ; h_i = falfs * int_i (term_alfa.f90:65-69, 87-92)
__global__ void k_alfa2(const double *__restrict__ dx, const double *__restrict__ dy, const double *__restrict__ dz,
                        const double *__restrict__ ix, const double *__restrict__ iy, const double *__restrict__ iz,
                        const double *__restrict__ falfs, double *s, double *h0, double *h1, double *h2, size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  s[t] = (dx[t] * ix[t]) + (dy[t] * iy[t]) + (dz[t] * iz[t]);
  const double f = falfs[t];
  h0[t] = f * ix[t];
  h1[t] = f * iy[t];
  h2[t] = f * iz[t];
}

// k_alfa2 with falfs formed from denalf (merged evaluation, which does not
// store falfs): f = 1 - denalf * (1/den0s)
// (T = float: the real32 grids of the FP32-convolution form; h_i may
// overwrite int_i in place, each thread reading its point before writing it)
template <typename T>
__global__ void k_alfa2m(const T *dx, const T *dy, const T *dz, const T *ix, const T *iy, const T *iz,
                         const T *denalf, double inv_den0s, T *s, T *h0, T *h1, T *h2, size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double a = ix[t], b = iy[t], c = iz[t];
  const double sx = (double)dx[t] * a, sy = (double)dy[t] * b, sz = (double)dz[t] * c;
  const double f = 1.0 - (double)denalf[t] * inv_den0s;
  s[t] = (T)((sx + sy) + sz);
  h0[t] = (T)(f * a);
  h1[t] = (T)(f * b);
  h2[t] = (T)(f * c);
}

// ualphas = (u1/den0s + sum_i d_i h_i) * h2o2m4 * alphas ; pot4 += ualphas
// (term_alfa.f90:110-113, poten.f90:101-104)
__global__ void k_alfa3(double *ualphas, const double *__restrict__ h0, const double *__restrict__ h1,
                        const double *__restrict__ h2, double *pot4, Stencil st, Geo g, OtArgs a) {
  HE4_IJK(g);
  const double d0 = stencil_axis(h0, st, 1, g, i, j, k, 0);
  const double d1 = stencil_axis(h1, st, 1, g, i, j, k, 1);
  const double d2 = stencil_axis(h2, st, 1, g, i, j, k, 2);
  const double u = ualphas[t] / a.den0s;
  const double ua = (u + d0 + d1 + d2) * a.h2o2m4 * a.alphas;
  ualphas[t] = ua;
  pot4[t] = pot4[t] + ua;
}

// pot4 = pot4 + uimp + penalty (poten.f90:122-124)
__global__ void k_pot4_final(double *pot4, const double *__restrict__ uimp, const double *__restrict__ penalty,
                             size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) pot4[t] = pot4[t] + uimp[t] + penalty[t];
}

// Merged assembly: lin = delj4 + uimp + sto1 + h2o2m4*alphas/den0s * u1,
// produced by one summed inverse transform, then
// pot4 = lin + dencg^2 (a0 + a1 dencg) + penalty + h2o2m4*alphas*sum_i d_i h_i
// (poten.f90:80-92,101-104,122-124 and term_alfa.f90:110-113 regrouped: every
// convolution that enters pot4 linearly shares one inverse FFT).
template <bool OTC>
__global__ void k_pot4_merged(const double *__restrict__ lin, const double *__restrict__ den,
                              const double *__restrict__ dencg, const double *__restrict__ h0,
                              const double *__restrict__ h1, const double *__restrict__ h2, double *pot4, Stencil st,
                              Geo g, OtArgs a) {
  HE4_IJK(g);
  const double d = den[t];
  const double th = tanh(a.beta * (d - a.den_m));
  const double pen = a.c_solid * (1.0 + th + a.beta * d * (1.0 - th * th));
  const double dc = dencg[t];
  const double a0 = a.cp4 / 2.0, a1 = a.cpp4 / 3.0;
  double v = lin[t] + dc * dc * (a0 + a1 * dc) + pen;
  if (OTC) {
    const double d0 = stencil_axis(h0, st, 1, g, i, j, k, 0);
    const double d1 = stencil_axis(h1, st, 1, g, i, j, k, 1);
    const double d2 = stencil_axis(h2, st, 1, g, i, j, k, 2);
    v += (d0 + d1 + d2) * a.h2o2m4 * a.alphas;
  }
  pot4[t] = v;
}

// ---------------------------------------------------------------------------
// gather of the force field at the particles
// ---------------------------------------------------------------------------
struct GatherArgs {
  int nx, ny, nz, npar;
  double x0, y0, z0, hx, hy, hz;
};

// trilinear blend of the 8 cell corners (blend_103, potenimp.f90:278-286)
__device__ __forceinline__ double blend103(double r, double s, double t, double x000, double x001, double x010,
                                           double x011, double x100, double x101, double x110, double x111) {
  return 1.0 * (+x000) + r * (-x000 + x100) + s * (-x000 + x010) + t * (-x000 + x001) +
         r * s * (+x000 - x100 - x010 + x110) + r * t * (+x000 - x100 - x001 + x101) +
         s * t * (+x000 - x010 - x001 + x011) + r * s * t * (-x000 + x100 + x010 + x001 - x011 - x101 - x110 + x111);
}

// interpola3 (potenimp.f90:91-114): one thread per (particle, component)
__global__ void k_gather(const double *__restrict__ rimp, const double *__restrict__ fx,
                         const double *__restrict__ fy, const double *__restrict__ fz, double *aimp, GatherArgs a) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 3 * a.npar) return;
  const int c = gid / a.npar, p = gid - c * a.npar;
  const double ax = (rimp[p] - a.x0) / a.hx + 1;
  const double ay = (rimp[a.npar + p] - a.y0) / a.hy + 1;
  const double az = (rimp[2 * a.npar + p] - a.z0) / a.hz + 1;
  const bool ok = ax > -1e9 && ax < 1e9 && ay > -1e9 && ay < 1e9 && az > -1e9 && az < 1e9;
  const int ix = ok ? (int)ax : 0, iy = ok ? (int)ay : 0, iz = ok ? (int)az : 0;
  if (!ok || ix >= a.nx || iy >= a.ny || iz >= a.nz || ix <= 0 || iy <= 0 || iz <= 0) {
    aimp[gid] = 0.0;
    return;
  }
  const double r = ax - ix, s = ay - iy, tt = az - iz;
  const double *f = (c == 0) ? fx : (c == 1) ? fy : fz;
  auto G = [&](int ii, int jj, int kk) { return f[((size_t)(kk - 1) * a.ny + (jj - 1)) * a.nx + (ii - 1)]; };
  aimp[gid] = blend103(r, s, tt, G(ix, iy, iz), G(ix, iy, iz + 1), G(ix, iy + 1, iz), G(ix, iy + 1, iz + 1),
                       G(ix + 1, iy, iz), G(ix + 1, iy, iz + 1), G(ix + 1, iy + 1, iz),
                       G(ix + 1, iy + 1, iz + 1));
}

// ---------------------------------------------------------------------------
// stencil launches: the z-marching kernels for npd = 7 and 13 when the grid
// is deep enough, the one-plane kernels otherwise
// ---------------------------------------------------------------------------
// The tiles' periodic indices stay in [-n, 2n) (what wrap2 folds) when
// nx >= 40, ny >= 16 and nz >= kZB + 2m: the farthest halo cell lies at most
// 36 cells beyond the last x index and 12 beyond the last y and z index.
static bool zmarch_ok(const Handle *h) {
  return h->p.icon == 8 && (h->st.m == 3 || h->st.m == 6) && h->nx >= 40 && h->ny >= 16 &&
         h->nz >= kZB + 2 * h->st.m;
}

static dim3 grid_z(const Geo &g, int zb = kZB) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + zb - 1) / zb); }

// ---------------------------------------------------------------------------
// streamed stencils (stream_stencil.cuh): launch shapes and per-device
// launch attributes
// ---------------------------------------------------------------------------
#ifndef HE4_STREAM_TY
#define HE4_STREAM_TY 4
#endif
#ifndef HE4_STREAM_S
#define HE4_STREAM_S 2
#endif
// Rows per CTA and planes in flight.  Measured at 256^3 (float grids,
// CUDA events, 20 launches): TY 4 / S 2 gives pot4 206 us and the gradient
// 143 us against 274 / 153 us for the register z-marching kernels; TY 2 /
// S 3, TY 2 / S 4 and TY 4 / S 3 were slower.  On FP64 grids the register
// kernels stay faster (pot4 247 vs 316 us, gradient 130 vs 139 us), so the
// streamed kernels serve the float grids of the FP32-convolution form.
constexpr int kStreamTY = HE4_STREAM_TY;
constexpr int kStreamS = HE4_STREAM_S;

// z planes per CTA: the chunk length whose grid fills the resident CTA
// slots best (fewest waves on a tie), at least 4 planes per chunk (small
// grids: 64^3 has 16 row tiles, so its chunks must be short to give the
// GPU enough CTAs; the longer z halo they re-read comes from L2)
static int stream_chunk(int nz, int ytiles, int resident) {
  int zcs[8];
  double effs[8], best = 0.0;
  for (int w = 1; w <= 8; w++) {
    int nch = std::min(nz, std::max(1, (w * resident) / ytiles));
    const int zc = std::max(4, (nz + nch - 1) / nch);
    const long ctas = (long)ytiles * ((nz + zc - 1) / zc);
    const long waves = (ctas + resident - 1) / resident;
    zcs[w - 1] = zc;
    effs[w - 1] = (double)ctas / (double)(waves * resident);
    best = std::max(best, effs[w - 1]);
  }
  // the longest chunk (least z halo, longest pipeline) within 2 % of the best fill
  int pick = nz;
  for (int w = 0; w < 8; w++)
    if (effs[w] >= best - 0.02 && (pick == nz || zcs[w] > pick)) pick = zcs[w];
  return pick;
}

// resident CTAs of a streamed kernel on the handle's device, with its
// dynamic shared memory limit raised there once (0: does not fit)
template <typename K>
static int stream_resident(const Handle *h, K kern, size_t smem) {
  // per (kernel, device): the dynamic shared memory limit set so far, and
  // the resident CTAs per shared memory size
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> limit;
  static std::map<std::pair<std::pair<const void *, int>, size_t>, int> res;
  if (smem > 227 * 1024) return 0;
  const std::pair<const void *, int> key((const void *)kern, h->dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = res.find({key, smem});
  if (it != res.end()) return it->second;
  if (limit[key] < smem) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    limit[key] = smem;
  }
  int nsm = 0, occ = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    return 0;
  }
  res[{key, smem}] = occ * nsm;
  return occ * nsm;
}

// the row-streamed kernels take periodic grids with 128, 256 or 512 points
// along x (a template parameter of the kernels) and a y extent the CTA rows
// divide; the shared memory fit is checked per launch.  At 64^3 the
// register z-marching kernels measured faster (FP32 step 0.39 against
// 0.42 ms), so that size keeps them.
static bool stream_ok(const Handle *h) {
  return h->p.icon == 8 && (h->st.m == 3 || h->st.m == 6) &&
         (h->nx == 128 || h->nx == 256 || h->nx == 512) && h->ny % kStreamTY == 0 &&
         h->ny >= 2 * h->st.m && h->nz >= 2 * h->st.m + 1;
}

// the first-derivative rows of `st` as SplitTaps; false unless every axis's
// row is antisymmetric with a zero centre (central periodic stencils)
static bool split_taps(const Stencil &st, SplitTaps *tp) {
  const int m = st.m;
  if (m > 6) return false;
  memset(tp, 0, sizeof(*tp));
  for (int ax = 0; ax < 3; ax++) {
    if (st.w1[ax][m] != 0.0) return false;
    for (int u = 1; u <= m; u++) {
      const double w = st.w1[ax][m + u];
      if (st.w1[ax][m - u] != -w) return false;
      tp->hi[ax][u - 1] = (float)w;
      tp->lo[ax][u - 1] = (float)(w - (double)tp->hi[ax][u - 1]);
    }
  }
  return true;
}

template <typename TI, bool OTC, int M, int NX>
static bool launch_pot4_stream(Handle *h, const TI *lin, const TI *dcg, const TI *h0, const TI *h1, const TI *h2,
                               const OtArgs &ot) {
  constexpr bool F = std::is_same<TI, float>::value;
  using L = Pot4StreamLayout<TI, OTC, M, kStreamTY, kStreamS, NX>;
  using LF = Pot4StreamLayout<TI, OTC, M, kStreamTY, kStreamS, NX, F>;  // centre values direct
  SplitTaps tp;
  const bool fm = F && h->pot4_split && split_taps(h->st, &tp);
  auto kern = fm ? k_pot4_stream<TI, OTC, M, kStreamTY, kStreamS, NX, F>
                 : k_pot4_stream<TI, OTC, M, kStreamTY, kStreamS, NX, false>;
  const size_t smem = fm ? LF::total : L::total;
  const int res = stream_resident(h, kern, smem);
  if (res == 0) return false;
  const Geo g = geo(h);
  const int yt = h->ny / kStreamTY, zc = stream_chunk(h->nz, yt, res);
  kern<<<dim3(yt, (h->nz + zc - 1) / zc), 256, smem, h->stream>>>(lin, h->den, dcg, h0, h1, h2, h->pot4, h->st, g, ot,
                                                                 zc, &h->gred->err, tp);
  HE4_LAUNCHED(h);
  return true;
}

template <typename TO, int M, int NX>
static bool launch_grad_stream(Handle *h, TO *dx, TO *dy, TO *dz) {
  using L = GradStreamLayout<TO, M, kStreamTY, kStreamS, NX>;
  auto kern = k_grad_stream<TO, M, kStreamTY, kStreamS, NX>;
  const int res = stream_resident(h, kern, L::total);
  if (res == 0) return false;
  const Geo g = geo(h);
  const int yt = h->ny / kStreamTY, zc = stream_chunk(h->nz, yt, res);
  kern<<<dim3(yt, (h->nz + zc - 1) / zc), 256, L::total, h->stream>>>(h->den, dx, dy, dz, h->st, g, zc,
                                                                     &h->gred->err);
  HE4_LAUNCHED(h);
  return true;
}

#define HE4_NX_SWITCH(nx, ...)                 \
  switch (nx) {                                \
    case 128: {                                \
      constexpr int NX_ = 128;                 \
      __VA_ARGS__;                             \
    }                                          \
    case 256: {                                \
      constexpr int NX_ = 256;                 \
      __VA_ARGS__;                             \
    }                                          \
    case 512: {                                \
      constexpr int NX_ = 512;                 \
      __VA_ARGS__;                             \
    }                                          \
    default: return false;                     \
  }

template <typename TO>
static bool grad_stream(Handle *h, TO *dx, TO *dy, TO *dz) {
  if (!stream_ok(h)) return false;
  if (h->st.m == 3) {
    HE4_NX_SWITCH(h->nx, return (launch_grad_stream<TO, 3, NX_>(h, dx, dy, dz)))
  }
  HE4_NX_SWITCH(h->nx, return (launch_grad_stream<TO, 6, NX_>(h, dx, dy, dz)))
}

template <typename TI, int M>
static bool pot4_stream_m(Handle *h, const TI *lin, const TI *dcg, const TI *h0, const TI *h1, const TI *h2,
                          const OtArgs &ot) {
  if (h->p.core4 == HE4_CORE_OTC) {
    HE4_NX_SWITCH(h->nx, return (launch_pot4_stream<TI, true, M, NX_>(h, lin, dcg, h0, h1, h2, ot)))
  }
  HE4_NX_SWITCH(h->nx, return (launch_pot4_stream<TI, false, M, NX_>(h, lin, dcg, h0, h1, h2, ot)))
}

template <typename TI>
static bool pot4_stream(Handle *h, const TI *lin, const TI *dcg, const TI *h0, const TI *h1, const TI *h2,
                        const OtArgs &ot) {
  if (!stream_ok(h)) return false;
  return h->st.m == 3 ? pot4_stream_m<TI, 3>(h, lin, dcg, h0, h1, h2, ot)
                      : pot4_stream_m<TI, 6>(h, lin, dcg, h0, h1, h2, ot);
}

bool real32_ok(const Handle *h) { return h->fp32 && zmarch_ok(h); }

// density gradient into the float grids g32[2..4] (FP32-convolution form)
int launch_grad_f32(Handle *h) {
  if (!h->real32) {
    set_error("the float-grid gradient needs the FP32-convolution form's float grids");
    return HE4_E_STATE;
  }
  const Geo g = geo(h);
  float *gx = h->g32[2], *gy = h->g32[3], *gz = h->g32[4];
  if (h->use_stream && grad_stream<float>(h, gx, gy, gz)) return HE4_OK;
  if (h->st.m == 3)
    k_grad_z_tile<3, kZB, float><<<grid_z(g), block3(), 0, h->stream>>>(h->den, gx, gy, gz, h->st, g);
  else
    k_grad_z_tile<6, kZB, float><<<grid_z(g), block3(), 0, h->stream>>>(h->den, gx, gy, gz, h->st, g);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int launch_grad(Handle *h) {
  const Geo g = geo(h);
  if (!zmarch_ok(h))
    k_grad<<<grid3(g), block3(), 0, h->stream>>>(h->den, h->dxden, h->dyden, h->dzden, h->st, g);
  else if (h->st.m == 3)
    k_grad_z<3, kZBg><<<grid_z(g, kZBg), block3(), 0, h->stream>>>(h->den, h->dxden, h->dyden, h->dzden, h->st, g);
  else
    k_grad_z<6, kZBg><<<grid_z(g, kZBg), block3(), 0, h->stream>>>(h->den, h->dxden, h->dyden, h->dzden, h->st, g);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

static OtArgs ot_args(const Handle *h);

// pot4 from lin = rtmp[0] and h_i = rtmp[1..3] (merged evaluation)
int launch_pot4_merged(Handle *h) {
  const Geo g = geo(h);
  const OtArgs ot = ot_args(h);
  const bool otc = (h->p.core4 == HE4_CORE_OTC);
  const double *h0 = otc ? h->rtmp[1] : nullptr, *h1 = otc ? h->rtmp[2] : nullptr, *h2 = otc ? h->rtmp[3] : nullptr;
  if (!zmarch_ok(h)) {
    if (otc)
      k_pot4_merged<true><<<grid3(g), block3(), 0, h->stream>>>(h->rtmp[0], h->den, h->dencg, h0, h1, h2, h->pot4,
                                                                h->st, g, ot);
    else
      k_pot4_merged<false><<<grid3(g), block3(), 0, h->stream>>>(h->rtmp[0], h->den, h->dencg, h0, h1, h2, h->pot4,
                                                                 h->st, g, ot);
  } else if (h->st.m == 3) {
    if (otc)
      k_pot4_merged_z<true, 3, kZBp><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(h->rtmp[0], h->den, h->dencg, h0, h1, h2,
                                                                          h->pot4, h->st, g, ot);
    else
      k_pot4_merged_z<false, 3, kZBp><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(h->rtmp[0], h->den, h->dencg, h0, h1,
                                                                           h2, h->pot4, h->st, g, ot);
  } else {
    if (otc)
      k_pot4_merged_z<true, 6, kZBp><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(h->rtmp[0], h->den, h->dencg, h0, h1, h2,
                                                                          h->pot4, h->st, g, ot);
    else
      k_pot4_merged_z<false, 6, kZBp><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(h->rtmp[0], h->den, h->dencg, h0, h1,
                                                                           h2, h->pot4, h->st, g, ot);
  }
  HE4_LAUNCHED(h);
  return HE4_OK;
}

// ---------------------------------------------------------------------------
// orchestration
// ---------------------------------------------------------------------------
static OtArgs ot_args(const Handle *h) {
  OtArgs a;
  a.cp4 = h->p.cp4;
  a.cpp4 = h->p.cpp4;
  a.den0s = h->p.den0s;
  a.h2o2m4 = h->p.h2o2m4;
  a.alphas = h->p.alphas;
  a.c_solid = h->p.c_solid;
  a.beta = h->p.beta_solid;
  a.den_m = h->p.den_m;
  return a;
}

static inline unsigned nblk(size_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

int field_potenimp(Handle *h, bool split) {
  // denpart: denx, psix, hpsix on the particle box (impurity.cu)
  HE4_TRY(impurity_density(h));
  // x/y transform of denx, kept in spec[4] for the merged assembly
  const double *in[1] = {h->denx};
  double2 *sp[1] = {h->spec[4]};
  HE4_TRY(fft_r2c(h, 1, in, sp));
  if (!split) return HE4_OK;
  // uimp = IFFT(FFT(denx) * Vq) * renor (potenimp.f90:17-19)
  ZOp op{h->spec[4], h->spec[1], h->vq, h->renor, -1};
  HE4_TRY(fft_z_conv(h, 1, &op));
  double2 *so[1] = {h->spec[1]};
  double *out[1] = {h->uimp};
  HE4_TRY(fft_c2r(h, 1, so, out));
  return HE4_OK;
}

// Merged form of poten (the time-step path): the linear convolutions that
// enter pot4 (delj4, uimp, the correlation term and the alpha_s u1 term) are
// summed in k space and inverted once; the correlation source and the
// falfs*grad(rho) sources of term_alfa are formed inside the x pass that
// transforms them; the named intermediate fields delj4, uimp, corr, ualphas,
// penalty and falfs are not written.
static int field_poten_merged(Handle *h) {
  const Geo g = geo(h);
  const size_t N = h->N;
  const OtArgs ot = ot_args(h);
  const bool otc = (h->p.core4 == HE4_CORE_OTC);
  {
    const double *in[1] = {h->den};
    double2 *sp[1] = {h->spec[0]};
    HE4_TRY(fft_r2c(h, 1, in, sp));
  }
  // dencg and denalf (poten.f90:34-38, 95-99)
  {
    ZOp ops[2] = {{h->spec[0], h->spec[1], h->wcgk, h->renor, -1}, {h->spec[0], h->spec[3], h->kalfs, h->renor, -1}};
    HE4_TRY(fft_z_conv(h, otc ? 2 : 1, ops));
    double2 *sp[2] = {h->spec[1], h->spec[3]};
    double *out[2] = {h->dencg, h->denalf};
    HE4_TRY(fft_c2r(h, otc ? 2 : 1, sp, out));
  }
  HE4_TRY(launch_grad(h));
  // correlation source den*dencg*(cp4+cpp4*dencg) formed in the x pass,
  // x/y transform kept in spec[5]
  {
    const void *in[1] = {h->den};
    double2 *sp[1] = {h->spec[5]};
    XLoad ld;
    ld.op = XLOAD_CORR;
    ld.aux0 = h->den;
    ld.aux1 = h->dencg;
    ld.c0 = ot.cp4;
    ld.c1 = ot.cpp4;
    HE4_TRY(fft_r2c_load(h, 1, in, sp, ld));
  }
  ZTerm terms[4] = {{h->spec[0], h->fvlj4, h->renor}, {h->spec[4], h->vq, h->renor}, {h->spec[5], h->wcgk, h->renor},
                    {h->spec[1], h->kalfs, h->renor * h->p.h2o2m4 * h->p.alphas / h->p.den0s}};
  if (otc) {
    const double inv_den0s = 1.0 / h->p.den0s;
    {
      // g_i = falfs * d_i rho formed in the x pass (falfs is not stored)
      const void *in[3] = {h->dxden, h->dyden, h->dzden};
      double2 *sp[3] = {h->spec[1], h->spec[2], h->spec[3]};
      XLoad ld;
      ld.op = XLOAD_ALFA;
      ld.aux0 = h->denalf;
      ld.c0 = inv_den0s;
      HE4_TRY(fft_r2c_load(h, 3, in, sp, ld));
      ZOp ops[3] = {{h->spec[1], h->spec[1], h->kalfs, h->renor, -1},
                    {h->spec[2], h->spec[2], h->kalfs, h->renor, -1},
                    {h->spec[3], h->spec[3], h->kalfs, h->renor, -1}};
      HE4_TRY(fft_z_conv(h, 3, ops));
      double *out[3] = {h->intx, h->inty, h->intz};
      HE4_TRY(fft_c2r(h, 3, sp, out));
    }
    k_alfa2m<double><<<nblk(N), 256, 0, h->stream>>>(h->dxden, h->dyden, h->dzden, h->intx, h->inty, h->intz, h->denalf,
                                            inv_den0s, h->rtmp[0], h->rtmp[1], h->rtmp[2], h->rtmp[3], N);
    HE4_LAUNCHED(h);
    const double *in[1] = {h->rtmp[0]};
    double2 *sp[1] = {h->spec[1]};
    HE4_TRY(fft_r2c(h, 1, in, sp));
  }
  HE4_TRY(fft_z_sum(h, otc ? 4 : 3, terms, h->spec[2]));
  {
    double2 *sp[1] = {h->spec[2]};
    double *out[1] = {h->rtmp[0]};
    HE4_TRY(fft_c2r(h, 1, sp, out));
  }
  HE4_TRY(launch_pot4_merged(h));
  return HE4_OK;
}

// field_poten_merged of the FP32-convolution form with float intermediate
// grids (Handle::real32): the same sequence; dencg, denalf, the gradients,
// the alpha_s integrals (overwritten by the h_i), s and lin are float, den
// and pot4 stay double; the gradient and the alpha_s products sum in FP64,
// the streamed pot4 assembly in FP32 with split weights (k_pot4_stream, FM).
static int field_poten_merged_f32(Handle *h) {
  const Geo g = geo(h);
  const size_t N = h->N;
  const OtArgs ot = ot_args(h);
  const bool otc = (h->p.core4 == HE4_CORE_OTC);
  float *dencg = h->g32[0], *denalf = h->g32[1], *gx = h->g32[2], *gy = h->g32[3], *gz = h->g32[4];
  float *hv[3] = {h->g32[5], h->g32[6], h->g32[7]}, *sl = h->g32[8];
  {
    const double *in[1] = {h->den};
    double2 *sp[1] = {h->spec[0]};
    HE4_TRY(fft_r2c(h, 1, in, sp));
  }
  {
    ZOp ops[2] = {{h->spec[0], h->spec[1], h->wcgk, h->renor, -1}, {h->spec[0], h->spec[3], h->kalfs, h->renor, -1}};
    HE4_TRY(fft_z_conv(h, otc ? 2 : 1, ops));
    double2 *sp[2] = {h->spec[1], h->spec[3]};
    float *out[2] = {dencg, denalf};
    HE4_TRY(fft_c2r_f32(h, otc ? 2 : 1, sp, out));
  }
  HE4_TRY(launch_grad_f32(h));
  {
    const void *in[1] = {h->den};
    double2 *sp[1] = {h->spec[5]};
    XLoad ld;
    ld.op = XLOAD_CORR;
    ld.real32 = 1;
    ld.aux0 = h->den;
    ld.aux1 = dencg;
    ld.c0 = ot.cp4;
    ld.c1 = ot.cpp4;
    HE4_TRY(fft_r2c_load(h, 1, in, sp, ld));
  }
  ZTerm terms[4] = {{h->spec[0], h->fvlj4, h->renor}, {h->spec[4], h->vq, h->renor}, {h->spec[5], h->wcgk, h->renor},
                    {h->spec[1], h->kalfs, h->renor * h->p.h2o2m4 * h->p.alphas / h->p.den0s}};
  if (otc) {
    const double inv_den0s = 1.0 / h->p.den0s;
    {
      const void *in[3] = {gx, gy, gz};
      double2 *sp[3] = {h->spec[1], h->spec[2], h->spec[3]};
      XLoad ld;
      ld.op = XLOAD_ALFA;
      ld.real32 = 1;
      ld.aux0 = denalf;
      ld.c0 = inv_den0s;
      HE4_TRY(fft_r2c_load(h, 3, in, sp, ld));
      ZOp ops[3] = {{h->spec[1], h->spec[1], h->kalfs, h->renor, -1},
                    {h->spec[2], h->spec[2], h->kalfs, h->renor, -1},
                    {h->spec[3], h->spec[3], h->kalfs, h->renor, -1}};
      HE4_TRY(fft_z_conv(h, 3, ops));
      HE4_TRY(fft_c2r_f32(h, 3, sp, hv));
    }
    // h_i over int_i in place; s into sl
    k_alfa2m<float><<<nblk(N), 256, 0, h->stream>>>(gx, gy, gz, hv[0], hv[1], hv[2], denalf, inv_den0s, sl, hv[0],
                                                   hv[1], hv[2], N);
    HE4_LAUNCHED(h);
    const void *in[1] = {sl};
    double2 *sp[1] = {h->spec[1]};
    XLoad ld;
    ld.real32 = 1;
    HE4_TRY(fft_r2c_load(h, 1, in, sp, ld));
  }
  HE4_TRY(fft_z_sum(h, otc ? 4 : 3, terms, h->spec[2]));
  {
    double2 *sp[1] = {h->spec[2]};
    float *out[1] = {sl};  // lin (s is consumed)
    HE4_TRY(fft_c2r_f32(h, 1, sp, out));
  }
  return launch_pot4_merged_f32(h);
}

// pot4 of the FP32-convolution form's merged evaluation: lin (in g32[8]),
// dencg (g32[0]) and h_i (g32[5..7]) are float grids, den and pot4 double
int launch_pot4_merged_f32(Handle *h) {
  if (!h->real32) {
    set_error("the float-grid pot4 stencil needs the FP32-convolution form's float grids");
    return HE4_E_STATE;
  }
  const Geo g = geo(h);
  const OtArgs ot = ot_args(h);
  const bool otc = (h->p.core4 == HE4_CORE_OTC);
  const float *sl = h->g32[8], *dencg = h->g32[0];
  const float *h0 = otc ? h->g32[5] : nullptr, *h1 = otc ? h->g32[6] : nullptr, *h2 = otc ? h->g32[7] : nullptr;
  if (h->use_stream && pot4_stream<float>(h, sl, dencg, h0, h1, h2, ot)) return HE4_OK;
  if (h->st.m == 3) {
    if (otc)
      k_pot4_merged_z<true, 3, kZBp, float, false><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(sl, h->den, dencg, h0, h1,
                                                                                       h2, h->pot4, h->st, g, ot);
    else
      k_pot4_merged_z<false, 3, kZBp, float, false><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(sl, h->den, dencg, h0, h1,
                                                                                        h2, h->pot4, h->st, g, ot);
  } else {
    if (otc)
      k_pot4_merged_z<true, 6, kZBp, float, false><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(sl, h->den, dencg, h0, h1,
                                                                                       h2, h->pot4, h->st, g, ot);
    else
      k_pot4_merged_z<false, 6, kZBp, float, false><<<grid_z(g, kZBp), block3(), 0, h->stream>>>(sl, h->den, dencg, h0, h1,
                                                                                        h2, h->pot4, h->st, g, ot);
  }
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int field_poten(Handle *h, bool split, double *pot4) {
  if (!split) return h->real32 ? field_poten_merged_f32(h) : field_poten_merged(h);
  const Geo g = geo(h);
  const size_t N = h->N;
  const OtArgs ot = ot_args(h);
  const bool otc = (h->p.core4 == HE4_CORE_OTC);
  // fden: x/y transform of den kept in spec[0] (poten.f90:27)
  {
    const double *in[1] = {h->den};
    double2 *sp[1] = {h->spec[0]};
    HE4_TRY(fft_r2c(h, 1, in, sp));
  }
  // dencg, delj4, (denalf): poten.f90:34-38, 46-50, 95-99
  {
    ZOp ops[3] = {{h->spec[0], h->spec[1], h->wcgk, h->renor, -1},
                  {h->spec[0], h->spec[2], h->fvlj4, h->renor, -1},
                  {h->spec[0], h->spec[3], h->kalfs, h->renor, -1}};
    const int nop = otc ? 3 : 2;
    HE4_TRY(fft_z_conv(h, nop, ops));
    double2 *sp[3] = {h->spec[1], h->spec[2], h->spec[3]};
    double *out[3] = {h->dencg, h->delj4, h->denalf};
    HE4_TRY(fft_c2r(h, nop, sp, out));
  }
  // derden
  HE4_TRY(launch_grad(h));
  // correlation convolution (poten.f90:62-74)
  k_corr_src<<<nblk(N), 256, 0, h->stream>>>(h->den, h->dencg, h->rtmp[0], N, ot);
  HE4_LAUNCHED(h);
  {
    const double *in[1] = {h->rtmp[0]};
    double2 *sp[1] = {h->spec[1]};
    HE4_TRY(fft_r2c(h, 1, in, sp));
    ZOp op{h->spec[1], h->spec[1], h->wcgk, h->renor, -1};
    HE4_TRY(fft_z_conv(h, 1, &op));
    double *out[1] = {h->corr};
    HE4_TRY(fft_c2r(h, 1, sp, out));
  }
  k_pot4_base<<<nblk(N), 256, 0, h->stream>>>(h->den, h->dencg, h->delj4, h->corr, h->penalty, pot4, N, ot);
  HE4_LAUNCHED(h);
  // term_alfa (term_alfa.f90:28-113), called for core4='OTC' only
  // (poten.f90:94-105).
  if (otc) {
    k_alfa1<<<nblk(N), 256, 0, h->stream>>>(h->denalf, h->dxden, h->dyden, h->dzden, h->falfs, h->rtmp[0],
                                           h->rtmp[1], h->rtmp[2], N, ot);
    HE4_LAUNCHED(h);
    {
      const double *in[3] = {h->rtmp[0], h->rtmp[1], h->rtmp[2]};
      double2 *sp[3] = {h->spec[1], h->spec[2], h->spec[3]};
      HE4_TRY(fft_r2c(h, 3, in, sp));
      ZOp ops[3] = {{h->spec[1], h->spec[1], h->kalfs, h->renor, -1},
                    {h->spec[2], h->spec[2], h->kalfs, h->renor, -1},
                    {h->spec[3], h->spec[3], h->kalfs, h->renor, -1}};
      HE4_TRY(fft_z_conv(h, 3, ops));
      double *out[3] = {h->intx, h->inty, h->intz};
      HE4_TRY(fft_c2r(h, 3, sp, out));
    }
    k_alfa2<<<nblk(N), 256, 0, h->stream>>>(h->dxden, h->dyden, h->dzden, h->intx, h->inty, h->intz, h->falfs,
                                           h->rtmp[0], h->rtmp[1], h->rtmp[2], h->rtmp[3], N);
    HE4_LAUNCHED(h);
    {
      const double *in[1] = {h->rtmp[0]};
      double2 *sp[1] = {h->spec[1]};
      HE4_TRY(fft_r2c(h, 1, in, sp));
      ZOp op{h->spec[1], h->spec[1], h->kalfs, h->renor, -1};
      HE4_TRY(fft_z_conv(h, 1, &op));
      double *out[1] = {h->ualphas};
      HE4_TRY(fft_c2r(h, 1, sp, out));
    }
    k_alfa3<<<grid3(g), block3(), 0, h->stream>>>(h->ualphas, h->rtmp[1], h->rtmp[2], h->rtmp[3], pot4, h->st,
                                                  g, ot);
    HE4_LAUNCHED(h);
  }
  k_pot4_final<<<nblk(N), 256, 0, h->stream>>>(pot4, h->uimp, h->penalty, N);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

// The force field f_i on the grid: the whole grid (full) or only the cells
// the trilinear gather reads (the impurity box widened by one cell), which
// is what a time step needs.
int field_forces(Handle *h, bool full) {
  // f_i = -IFFT(FFT(d_i rho) Vq) * renor / m_X = IFFT(-renor/m_X Vq i D_i fden)
  // (potenimp.f90:42-50, with the 1/m_X of :67-69 folded in)
  const double c = -h->renor / h->mAg_u;
  const int bz = full ? 0 : 1;
  if (h->p.icon == 8) {
    ZOp ops[3] = {{h->spec[0], h->spec[1], h->vq, c, 0, 0, bz},
                  {h->spec[0], h->spec[2], h->vq, c, 1, 0, bz},
                  {h->spec[0], h->spec[3], h->vq, c, 2, 0, bz}};
    HE4_TRY(fft_z_conv(h, 3, ops));
  } else {
    // non-periodic stencils: FFT(d_i rho) is no multiple of FFT(rho), so the
    // gradients of this evaluation are transformed as the reference does
    const double *in[3] = {h->dxden, h->dyden, h->dzden};
    double2 *sp[3] = {h->spec[1], h->spec[2], h->spec[3]};
    HE4_TRY(fft_r2c(h, 3, in, sp));
    ZOp ops[3] = {{h->spec[1], h->spec[1], h->vq, c, -1, 0, bz},
                  {h->spec[2], h->spec[2], h->vq, c, -1, 0, bz},
                  {h->spec[3], h->spec[3], h->vq, c, -1, 0, bz}};
    HE4_TRY(fft_z_conv(h, 3, ops));
  }
  double2 *sp[3] = {h->spec[1], h->spec[2], h->spec[3]};
  double *out[3] = {h->fx, h->fy, h->fz};
  if (full)
    HE4_TRY(fft_c2r(h, 3, sp, out));
  else
    HE4_TRY(fft_c2r_box(h, 3, sp, out));
  // quantum-potential term, nonzero only where denx > 0 (impurity.cu)
  HE4_TRY(impurity_force_q(h));
  h->forces_full = full ? 1 : 0;
  return HE4_OK;
}

int field_forceimp(Handle *h, bool full) {
  HE4_TRY(field_forces(h, full));
  GatherArgs a;
  a.nx = h->nx;
  a.ny = h->ny;
  a.nz = h->nz;
  a.npar = h->npar;
  a.x0 = -h->p.xmax;
  a.y0 = -h->p.ymax;
  a.z0 = -h->p.zmax;
  a.hx = h->hx;
  a.hy = h->hy;
  a.hz = h->hz;
  k_gather<<<nblk(3 * (size_t)h->npar), 256, 0, h->stream>>>(h->rimp, h->fx, h->fy, h->fz, h->aimp, a);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

}  // namespace he4

// impurity.cu -- the impurity density and its quantum force on the region
// the test particles occupy.
//
// denpart (potenimp.f90:294-338) histograms the particles (NGP), smooths the
// histogram ironx times (ironing.f90:19-28), takes psix = sqrt(denx) and
// hpsix = -h2o2mx lap(psix); forceimp adds (1/denx)(d psix hpsix - psix
// d hpsix)/m_X where denx > 0 (potenimp.f90:52-69).  All of these are zero
// away from the particle cloud, so they are computed on a box:
//   D    = NGP cells of the particles, widened by ironx (the support of denx,
//          psix and of the force term),
//   D+m  = D widened by the stencil half width (the support of hpsix).
// The box is found on the device every evaluation; the previous box is
// cleared first, so denx, psix and hpsix stay zero outside the current one
// and the full-grid FFT of denx sees exact zeros there.  When D+2m would
// reach a face of the grid (periodic wrap of the stencils, boundary rows the
// ironing leaves untouched) every box kernel covers the whole grid instead,
// which is the reference's computation as it stands.
#include <limits.h>

#include "common.cuh"
#include "stencil.cuh"

namespace he4 {

struct DepArgs {
  int nx, ny, nz, npar;
  double xmin, ymin, zmin, hx, hy, hz;
};

// NGP cell as the reference computes it: int(1.5 + (r - r0)/h), 1-based
__device__ __forceinline__ bool ngp_cell3(const DepArgs &a, double rx, double ry, double rz, int c[3]) {
  const double fx = 1.5 + (rx - a.xmin) / a.hx;
  const double fy = 1.5 + (ry - a.ymin) / a.hy;
  const double fz = 1.5 + (rz - a.zmin) / a.hz;
  if (!(fx > -1e9 && fx < 1e9 && fy > -1e9 && fy < 1e9 && fz > -1e9 && fz < 1e9)) return false;
  const int ix = (int)fx, iy = (int)fy, iz = (int)fz;  // truncation toward zero
  if (iz >= 1 && iz <= a.nz && iy >= 1 && iy <= a.ny && ix >= 1 && ix <= a.nx) {
    c[0] = ix - 1;
    c[1] = iy - 1;
    c[2] = iz - 1;
    return true;
  }
  return false;
}

__global__ void k_deposit(const double *__restrict__ rimp, unsigned int *counts, DepArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.npar) return;
  int c[3];
  if (ngp_cell3(a, rimp[p], rimp[a.npar + p], rimp[2 * a.npar + p], c))
    atomicAdd(counts + ((size_t)c[2] * a.ny + c[1]) * a.nx + c[0], 1u);
}

// prev = cur; cur = NGP cells of all particles widened by `iron`, or the
// whole grid when the widened box plus 2m reaches a face.  Every CTA folds
// the cells of its particles into the GridRed min/max scratch with integer
// atomics (exact, so the order does not matter); the CTA that finishes
// last forms the box and resets the scratch for the next launch.
__global__ void __launch_bounds__(kPartThreads) k_box_find(const double *__restrict__ rimp, DepArgs a, int iron, int m,
                                                           GridRed *gr, BoxPair *bp) {
  __shared__ int sh[6][kPartThreads / 32];
  __shared__ int last;
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.npar; p += gridDim.x * blockDim.x) {
    int c[3];
    if (ngp_cell3(a, rimp[p], rimp[a.npar + p], rimp[2 * a.npar + p], c)) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        mn[d] = min(mn[d], c[d]);
        mx[d] = max(mx[d], c[d]);
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_down_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_down_sync(0xffffffffu, mx[d], o));
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0)
    for (int d = 0; d < 3; d++) {
      sh[d][warp] = mn[d];
      sh[3 + d][warp] = mx[d];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < 3; d++) {
      for (int w = 1; w < nw; w++) {
        sh[d][0] = min(sh[d][0], sh[d][w]);
        sh[3 + d][0] = max(sh[3 + d][0], sh[3 + d][w]);
      }
      if (sh[d][0] != INT_MAX) {
        atomicMin(&gr->box[d], sh[d][0]);
        atomicMax(&gr->box[3 + d], sh[3 + d][0]);
      }
    }
    __threadfence();
    last = (atomicAdd(&gr->count[0], 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  int lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = atomicAdd(&gr->box[d], 0);
    hi[d] = atomicAdd(&gr->box[3 + d], 0);
    gr->box[d] = INT_MAX;
    gr->box[3 + d] = INT_MIN;
  }
  gr->count[0] = 0u;
  Box b;
  b.full = 0;
  b.empty = (lo[0] == INT_MAX);
  const int n[3] = {a.nx, a.ny, a.nz};
  for (int d = 0; d < 3; d++) {
    b.lo[d] = b.empty ? 0 : lo[d] - iron;
    b.hi[d] = b.empty ? -1 : hi[d] + iron;
    if (!b.empty && (b.lo[d] - 2 * m < 0 || b.hi[d] + 2 * m > n[d] - 1)) b.full = 1;
  }
  bp->prev = bp->cur;
  bp->cur = b;
}

// region of a box widened by e cells, or the whole grid; false if empty
__device__ __forceinline__ bool box_region(const Box &b, int e, const Geo &g, int lo[3], int len[3]) {
  if (b.full) {
    lo[0] = lo[1] = lo[2] = 0;
    len[0] = g.nx;
    len[1] = g.ny;
    len[2] = g.nz;
    return true;
  }
  if (b.empty) return false;
  for (int d = 0; d < 3; d++) {
    lo[d] = b.lo[d] - e;
    len[d] = b.hi[d] - b.lo[d] + 1 + 2 * e;
  }
  return true;
}

// grid-stride loop over the points of a box region
#define HE4_BOX_LOOP(box, e, g)                                                                     \
  int lo_[3], len_[3];                                                                               \
  if (!box_region((box), (e), (g), lo_, len_)) return;                                             \
  const size_t vol_ = (size_t)len_[0] * len_[1] * len_[2];                                          \
  for (size_t q_ = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q_ < vol_;                        \
       q_ += (size_t)gridDim.x * blockDim.x) {                                                       \
    const int i = lo_[0] + (int)(q_ % len_[0]);                                                     \
    const int j = lo_[1] + (int)((q_ / len_[0]) % len_[1]);                                         \
    const int k = lo_[2] + (int)(q_ / ((size_t)len_[0] * len_[1]));                                \
    const size_t t = ((size_t)k * (g).ny + j) * (g).nx + i;

#define HE4_BOX_END }

// zero the previous support (box widened by m) of denx, psix, hpsix, counts
__global__ void k_box_clear(const BoxPair *__restrict__ bp, double *denx, double *psix, double *hpsix,
                            unsigned int *counts, Geo g, int m) {
  const Box b = bp->prev;
  HE4_BOX_LOOP(b, m, g)
  denx[t] = 0.0;
  psix[t] = 0.0;
  hpsix[t] = 0.0;
  counts[t] = 0u;
  HE4_BOX_END
}

// denx = count / N_par / hxyz (potenimp.f90:322)
__global__ void k_denx_box(const BoxPair *__restrict__ bp, const unsigned int *__restrict__ counts, double *denx,
                           Geo g, double npar, double hxyz) {
  const Box b = bp->cur;
  HE4_BOX_LOOP(b, 0, g)
  denx[t] = (double)counts[t] / npar / hxyz;
  HE4_BOX_END
}

// one ironing pass src -> dst on the box: interior points get
// 1/12 (six neighbours) + 1/2 centre, points on a face are copied
// (ironing.f90:19-28); separately rounded products, no FMA, so the result
// is bit-identical to the reference's arithmetic
__global__ void k_iron_box(const BoxPair *__restrict__ bp, const double *__restrict__ src, double *dst, Geo g) {
  const Box b = bp->cur;
  HE4_BOX_LOOP(b, 0, g)
  double v;
  if (i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1 && k > 0 && k < g.nz - 1) {
    const size_t sy = g.nx, sz = (size_t)g.nx * g.ny;
    const double s6 = ((((src[t - 1] + src[t + 1]) + src[t - sy]) + src[t + sy]) + src[t - sz]) + src[t + sz];
    v = __dadd_rn(__dmul_rn(1.0 / 12.0, s6), __dmul_rn(0.5, src[t]));
  } else {
    v = src[t];
  }
  dst[t] = v;
  HE4_BOX_END
}

// denx <- src (if src != denx) and psix = sqrt(denx) on the box
__global__ void k_sqrt_box(const BoxPair *__restrict__ bp, const double *__restrict__ src, double *denx,
                           double *psix, Geo g) {
  const Box b = bp->cur;
  HE4_BOX_LOOP(b, 0, g)
  const double v = src[t];
  denx[t] = v;
  psix[t] = sqrt(v);
  HE4_BOX_END
}

// hpsix = -h2o2mx (d2x + d2y + d2z) psix on the box widened by m
// (potenimp.f90:332-335)
__global__ void k_lap_box(const BoxPair *__restrict__ bp, const double *__restrict__ psix, double *hpsix,
                          double scale, Stencil st, Geo g) {
  const Box b = bp->cur;
  HE4_BOX_LOOP(b, st.m, g)
  const double a = stencil_axis(psix, st, 2, g, i, j, k, 0);
  const double bb = stencil_axis(psix, st, 2, g, i, j, k, 1);
  const double c = stencil_axis(psix, st, 2, g, i, j, k, 2);
  hpsix[t] = scale * ((a + bb) + c);
  HE4_BOX_END
}

// f_i += (1/denx)(d_i psix hpsix - psix d_i hpsix) / m_X where denx > 0; the
// convolution part of f_i already carries its 1/m_X (potenimp.f90:63-69)
__global__ void k_force_q_box(const BoxPair *__restrict__ bp, double *fx, double *fy, double *fz,
                              const double *__restrict__ psix, const double *__restrict__ hpsix,
                              const double *__restrict__ denx, double mass, Stencil st, Geo g) {
  const Box b = bp->cur;
  HE4_BOX_LOOP(b, 0, g)
  const double dn = denx[t];
  if (dn > 0.0) {
    const double inv = 1.0 / dn;
    const double ps = psix[t], hp = hpsix[t];
    double *F[3] = {fx, fy, fz};
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      const double dps = stencil_axis(psix, st, 1, g, i, j, k, ax);
      const double dhp = stencil_axis(hpsix, st, 1, g, i, j, k, ax);
      F[ax][t] = F[ax][t] + inv * (dps * hp - ps * dhp) / mass;
    }
  }
  HE4_BOX_END
}

static DepArgs dep_args(const Handle *h) {
  DepArgs d;
  d.nx = h->nx;
  d.ny = h->ny;
  d.nz = h->nz;
  d.npar = h->npar;
  d.xmin = -h->p.xmax;
  d.ymin = -h->p.ymax;
  d.zmin = -h->p.zmax;
  d.hx = h->hx;
  d.hy = h->hy;
  d.hz = h->hz;
  return d;
}

static unsigned box_grid(const Handle *h) {
  // enough CTAs for a full-grid sweep, few enough that a small box costs
  // little more than the launch
  const size_t want = (h->N + 255) / 256;
  return (unsigned)(want < 148 * 8 ? want : 148 * 8);
}

int impurity_density(Handle *h) {
  const Geo g{h->nx, h->ny, h->nz, zpad_of(h->p.icon)};
  const DepArgs d = dep_args(h);
  const unsigned gb = box_grid(h);
  const unsigned pg = (unsigned)std::max(1, std::min(kPartMaxCta, (h->npar + kPartThreads - 1) / kPartThreads));
  k_box_find<<<pg, kPartThreads, 0, h->stream>>>(h->rimp, d, h->p.ironx, h->st.m, h->gred, h->box);
  HE4_LAUNCHED(h);
  k_box_clear<<<gb, 256, 0, h->stream>>>(h->box, h->denx, h->psix, h->hpsix, h->counts, g, h->st.m);
  HE4_LAUNCHED(h);
  k_deposit<<<(h->npar + 255) / 256, 256, 0, h->stream>>>(h->rimp, h->counts, d);
  HE4_LAUNCHED(h);
  k_denx_box<<<gb, 256, 0, h->stream>>>(h->box, h->counts, h->denx, g, (double)h->npar, h->hx * h->hy * h->hz);
  HE4_LAUNCHED(h);
  // ironing ping-pongs between denx and psix, both zero outside the box
  double *src = h->denx, *dst = h->psix;
  for (int it = 0; it < h->p.ironx; it++) {
    k_iron_box<<<gb, 256, 0, h->stream>>>(h->box, src, dst, g);
    HE4_LAUNCHED(h);
    std::swap(src, dst);
  }
  k_sqrt_box<<<gb, 256, 0, h->stream>>>(h->box, src, h->denx, h->psix, g);
  HE4_LAUNCHED(h);
  k_lap_box<<<gb, 256, 0, h->stream>>>(h->box, h->psix, h->hpsix, -h->h2o2mx, h->st, g);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int impurity_force_q(Handle *h) {
  const Geo g{h->nx, h->ny, h->nz, zpad_of(h->p.icon)};
  k_force_q_box<<<box_grid(h), 256, 0, h->stream>>>(h->box, h->fx, h->fy, h->fz, h->psix, h->hpsix, h->denx,
                                                   h->mAg_u, h->st, g);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int impurity_reset_box(Handle *h) {
  BoxPair bp{};
  bp.cur.full = 1;
  bp.prev.full = 1;
  HE4_CUDA_TRY(cudaMemcpyAsync(h->box, &bp, sizeof(BoxPair), cudaMemcpyHostToDevice, h->stream));
  return HE4_OK;
}

}  // namespace he4

// diag.cu -- device-side diagnostics of the pener blocks: the He atom number
// sum(den)*dxyz (DFT4He3d.f90:885-886) and the centre of mass of the density
// (r_cm.f90:23-58), reduced on the GPU so no field has to be copied out.
//
// Two entry points share the kernels: he4_diagnostics works on a handle and
// takes its per-plane partial sums from the handle's reduction workspace;
// he4_diagnostics_noalloc works on caller-owned device arrays and takes them
// from the fixed array below, so it allocates nothing.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "reduce.cuh"

// Scratch of he4_diagnostics_noalloc: four partial sums per z plane.  It is
// part of the library image, so every GPU that loads the library holds these
// 128 KiB until the process exits.
#define HE4_DIAG_NOALLOC_MAX_NZ 4096
static __device__ __align__(256) double g_diag_noalloc_part[4 * HE4_DIAG_NOALLOC_MAX_NZ];

namespace he4 {

struct DiagArgs {
  int nx, ny, nz;
  double x0, y0, z0, hx, hy, hz;
};

// one CTA per z plane: partial sums of den, den*x, den*y, den*z into
// part[q * nz + plane], q = 0..3
__global__ void k_diag_planes(const double *__restrict__ den, DiagArgs a, double *part) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  const double zz = a.z0 + a.hz * k;
  double s0 = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  const double *plane = den + (size_t)k * a.ny * a.nx;
  for (int t = threadIdx.x; t < a.nx * a.ny; t += blockDim.x) {
    const int i = t % a.nx, j = t / a.nx;
    const double v = plane[t];
    s0 += v;
    sx += v * (a.x0 + a.hx * i);
    sy += v * (a.y0 + a.hy * j);
    sz += v * zz;
  }
  const double r0 = block_sum(s0, sh);
  const double rx = block_sum(sx, sh);
  const double ry = block_sum(sy, sh);
  const double rz = block_sum(sz, sh);
  if (threadIdx.x == 0) {
    part[k] = r0;
    part[a.nz + k] = rx;
    part[2 * a.nz + k] = ry;
    part[3 * a.nz + k] = rz;
  }
}

// out = {sum*dxyz, xcm, ycm, zcm} with xcm = (sum den*x)*dxyz/n4 (r_cm.f90:54-56)
__global__ void k_diag_final(const double *__restrict__ part, int nz, double dxyz, double n4, double *out) {
  __shared__ double sh[32];
  for (int q = 0; q < 4; q++) {
    double acc = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) acc += part[q * nz + k];
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[q] = (q == 0) ? s * dxyz : s * dxyz / n4;
  }
}

static DiagArgs diag_args(int nx, int ny, int nz, double xmax, double ymax, double zmax) {
  DiagArgs a;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.hx = 2.0 * fabs(xmax) / nx;
  a.hy = 2.0 * fabs(ymax) / ny;
  a.hz = 2.0 * fabs(zmax) / nz;
  a.x0 = -xmax;
  a.y0 = -ymax;
  a.z0 = -zmax;
  return a;
}

// launches the two reduction kernels; part needs 4*nz doubles of scratch
static int launch_diag(const double *den, const DiagArgs &a, double dxyz, double n4, double *part, double *out,
                       cudaStream_t s, int64_t *launches) {
  k_diag_planes<<<a.nz, 256, 0, s>>>(den, a, part);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_diag_final<<<1, 1024, 0, s>>>(part, a.nz, dxyz, n4, out);
    e = cudaGetLastError();
  }
  if (launches) *launches += 2;
  if (e != cudaSuccess) {
    set_error("diagnostics launch: %s", cudaGetErrorString(e));
    return HE4_E_CUDA;
  }
  return HE4_OK;
}

// Device address of g_diag_noalloc_part, looked up once per device (with that
// device current) the first time he4_diagnostics_noalloc runs on it.  In host
// code the symbol is only a stand-in; kernels must be given this address.
// The cached address belongs to the device's primary context as it was at
// that first call: after cudaDeviceReset (which tears the context down, and
// the module with it) the address is stale, so a host that resets a device
// must not call he4_diagnostics_noalloc on it again in the same process.
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[kMaxDevices] = {nullptr};

static int noalloc_scratch(double **out) {
  int dev = -1;
  HE4_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal %d out of range", dev);
    return HE4_E_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_diag_noalloc_part);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress of the diagnostics scratch: %s", cudaGetErrorString(e));
      return HE4_E_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return HE4_OK;
}

int compute_diagnostics(Handle *h, int n4, double *host_out) {
  const DiagArgs a = diag_args(h->nx, h->ny, h->nz, h->p.xmax, h->p.ymax, h->p.zmax);
  // scratch: the reduction workspace (8 * nblocks >= 4 * nz doubles)
  HE4_TRY(launch_diag(h->den, a, h->dxyz, (double)n4, h->red, h->scal + 32, h->stream, &h->launches));
  HE4_CUDA_TRY(cudaMemcpyAsync(h->hscal + 32, h->scal + 32, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (int q = 0; q < 4; q++) host_out[q] = h->hscal[32 + q];
  return HE4_OK;
}

// ---------------------------------------------------------------------------
// Spherical bubble radius (bubble_radius_esferic.f90:1-134, called from
// DFT4He3d.f90:929-986)
// ---------------------------------------------------------------------------

// grid coordinate x(i+1) = -xmax + hx*i (DFT4He3d.f90:303) without FMA
// contraction, so host and device place every point identically
__host__ __device__ __forceinline__ double grid_coord(double x0, double h, int i) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(x0, __dmul_rn(h, (double)i));
#else
  return x0 + h * (double)i;
#endif
}

// one CTA per z plane: sum(den), max|den| and the three sums
// denx*x^2, denx*y^2, denx*z^2 of the impurity mean-square radii
// (DFT4He3d.f90:933-945), into part[q * nz + plane], q = 0..4
__global__ void k_bubble_planes(const double *__restrict__ den, const double *__restrict__ denx, DiagArgs a,
                                double *part) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  const double zk = grid_coord(a.z0, a.hz, k);
  const double z2 = zk * zk;
  double s0 = 0.0, mx = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
  const size_t off = (size_t)k * a.ny * a.nx;
  for (int j = threadIdx.y; j < a.ny; j += blockDim.y) {
    const double yj = grid_coord(a.y0, a.hy, j);
    const double y2 = yj * yj;
    for (int i = threadIdx.x; i < a.nx; i += blockDim.x) {
      const size_t t = off + (size_t)j * a.nx + i;
      const double v = den[t], w = denx[t];
      const double xi = grid_coord(a.x0, a.hx, i);
      s0 += v;
      mx = fmax(mx, fabs(v));
      sx += w * (xi * xi);
      sy += w * y2;
      sz += w * z2;
    }
  }
  // max first: block_sum leaves sh reusable after its trailing barrier
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) sh[tid >> 5] = mx;
  __syncthreads();
  if (tid == 0) {
    double m = sh[0];
    for (int w = 1; w < (blockDim.x * blockDim.y + 31) / 32; w++) m = fmax(m, sh[w]);
    part[a.nz + k] = m;
  }
  __syncthreads();
  const double r0 = block_sum(s0, sh);
  const double rx = block_sum(sx, sh);
  const double ry = block_sum(sy, sh);
  const double rz = block_sum(sz, sh);
  if (tid == 0) {
    part[k] = r0;
    part[2 * a.nz + k] = rx;
    part[3 * a.nz + k] = ry;
    part[4 * a.nz + k] = rz;
  }
}

// out[0..4] = sum over planes of part (max for q = 1)
__global__ void k_bubble_final(const double *__restrict__ part, int nz, double *out) {
  __shared__ double sh[32];
  for (int q = 0; q < 5; q++) {
    if (q == 1) {
      if (threadIdx.x == 0) {
        double m = 0.0;
        for (int k = 0; k < nz; k++) m = fmax(m, part[nz + k]);
        out[1] = m;
      }
      continue;
    }
    double acc = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) acc += part[q * nz + k];
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[q] = s;
  }
}

struct HistArgs {
  int nx, ny, nz, nr;
  double x0, y0, z0, hx, hy, hz;
  double xp, yp, zp;  // x(ipx), y(ipy), z(ipz)
  double dr;
  double scale;  // 2^S: fixed-point scale of the bin sums
};

// Radial histogram of den around (x(ipx), y(ipy), z(ipz))
// (bubble_radius_esferic.f90:45-62): bin ir = int(r/dr + 1.5), 1-based.
// Sums are accumulated as integers of den*2^S, first per CTA in shared
// memory, then into the global bins; integer addition is associative, so
// the result does not depend on the order of the atomics.  The host picks S
// so that no bin can overflow.  Points past the last bin (where the
// reference stops with '0001') are counted in bins[2*nr].
// Dynamic shared memory: nr long longs + nr unsigned ints.
__global__ void __launch_bounds__(256) k_bubble_hist(const double *__restrict__ den, HistArgs a,
                                                     unsigned long long *bins) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long *ssum = reinterpret_cast<unsigned long long *>(smem);
  unsigned int *scnt = reinterpret_cast<unsigned int *>(ssum + a.nr);
  for (int b = threadIdx.x; b < a.nr; b += blockDim.x) {
    ssum[b] = 0ull;
    scnt[b] = 0u;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int nrows = a.ny * a.nz;
  unsigned int outside = 0;
  for (int row = blockIdx.x * nwarps + warp; row < nrows; row += gridDim.x * nwarps) {
    const int j = row % a.ny, k = row / a.ny;
    const double dy = __dsub_rn(grid_coord(a.y0, a.hy, j), a.yp);
    const double dz = __dsub_rn(grid_coord(a.z0, a.hz, k), a.zp);
    const double y2 = __dmul_rn(dy, dy), z2 = __dmul_rn(dz, dz);
    const double *line = den + (size_t)row * a.nx;
    for (int i = lane; i < a.nx; i += 32) {
      const double dx = __dsub_rn(grid_coord(a.x0, a.hx, i), a.xp);
      const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), y2), z2));
      const double t = __dadd_rn(r / a.dr, 1.5);
      if (!(t < (double)(a.nr + 1))) {
        outside++;
        continue;
      }
      const int b = (int)t - 1;
      const long long q = __double2ll_rn(__dmul_rn(line[i], a.scale));
      atomicAdd(&ssum[b], (unsigned long long)q);
      atomicAdd(&scnt[b], 1u);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < a.nr; b += blockDim.x) {
    const unsigned int c = scnt[b];
    if (c) {
      atomicAdd(&bins[b], ssum[b]);
      atomicAdd(&bins[a.nr + b], (unsigned long long)c);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) outside += __shfl_down_sync(0xffffffffu, outside, o);
  if (lane == 0 && outside) atomicAdd(&bins[2 * a.nr], (unsigned long long)outside);
}

constexpr int kBubbleMaxNr = 8192;  // 96 KiB of shared bins per CTA

// Maxima / half-maximum search and Newton refinement on the spline of the
// normalised radial density (bubble_radius_esferic.f90:63-132).  Arrays
// are 1-based views as in the reference; denr is normalised in place.
static void bubble_search(int nr, double dr, double xnorm, const double xms[3], double *rr0, double *denr0,
                          BubbleResult *res, std::vector<double> &work) {
  const double pi = 3.141592653589793238462643;
  double *rr = rr0 - 1, *denr = denr0 - 1;
  work.assign(4 * (size_t)nr, 0.0);
  double *A = work.data() - 1, *B = A + nr, *C = B + nr, *D = C + nr;
  double dmax = denr[1];
  for (int i = 2; i <= nr; i++) dmax = fmax(dmax, denr[i]);
  // denmin is taken before the normalisation below (:66), as the reference does
  const double denmin = dmax * 0.75;
  double aux1 = 0.0;
  for (int i = 1; i <= nr; i++) {
    const double r = (double)(i - 1) * dr;
    rr[i] = r;
    aux1 += (r * r) * denr[i];
  }
  aux1 = aux1 * dr * 4.0 * pi;
  const double fac = xnorm / aux1;
  for (int i = 1; i <= nr; i++) denr[i] = denr[i] * fac;
  res->found[0] = res->found[1] = 0;
  res->ir = 0;
  res->rb = 0.0;
  if (spline_global(rr + 1, denr + 1, A + 1, B + 1, C + 1, D + 1, 0.0, 0.0, nr) != HE4_OK) return;
  const double rmin = 2.0;
  const double ams = fmax(fmax(xms[0], xms[1]), xms[2]);
  const int i0 = (int)(ams / dr + 1.5);
  // first local maximum beyond the impurity's extent (:79-86); the reference
  // starts at i0 >= 1 and reads denr(i0-1), so the scan starts at 2
  int j = i0 < 2 ? 2 : i0, ir = 0;
  for (; j <= nr - 1; j++) {
    if (denr[j] > denr[j - 1] && denr[j] > denr[j + 1]) {
      if (rr[j] < rmin || denr[j] < denmin) continue;
      ir = j;
      break;
    }
  }
  // a maximum at nr-1 counts as not found, as in :87
  if (j >= nr - 1) return;
  res->found[0] = 1;
  res->ir = ir;
  const double aux2 = denr[ir] * 0.5;
  const int it0 = i0;
  int i = 0;
  for (j = ir - 1; j >= it0 + 1; j--) {
    if ((denr[j - 1] - aux2) * (denr[j + 1] - aux2) < 0.0) {
      i = j;
      break;
    }
  }
  if (j == it0 || j == it0 - 1) return;  // :111
  double rb = rr[i];
  int it;
  const int niter = 100;
  const double eps = 1e-6;
  for (it = 1; it <= niter; it++) {
    const double f = ((D[i] * rb + C[i]) * rb + B[i]) * rb + A[i];
    const double df = (3.0 * D[i] * rb + 2.0 * C[i]) * rb + B[i];
    const double step = -(f - aux2) / df;
    rb = rb + step;
    if (fabs(step) < eps) break;
  }
  res->rb = rb;
  if (it >= niter) return;  // :127: converging on the last iteration also fails
  res->found[1] = 1;
}

int compute_bubble_radius(Handle *h, int nr, BubbleResult *res, double *rr_out, double *denr_out) {
  if (nr < 4 || nr > kBubbleMaxNr) {
    set_error("he4_bubble_radius: nr=%d outside [4, %d]", nr, kBubbleMaxNr);
    return HE4_E_ARG;
  }
  if (!h->field_valid) HE4_TRY(field_all(h, true));  // den and denx of the current state
  const DiagArgs a = diag_args(h->nx, h->ny, h->nz, h->p.xmax, h->p.ymax, h->p.zmax);
  // trajectory means (DFT4He3d.f90:893-895), the plane sums, one copy back
  HE4_TRY(particle_means(h, h->scal + 40));
  k_bubble_planes<<<a.nz, dim3(32, 8), 0, h->stream>>>(h->den, h->denx, a, h->red);
  HE4_LAUNCHED(h);
  k_bubble_final<<<1, 1024, 0, h->stream>>>(h->red, a.nz, h->scal + 49);
  HE4_LAUNCHED(h);
  HE4_CUDA_TRY(cudaMemcpyAsync(h->hscal + 40, h->scal + 40, 14 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const double *m = h->hscal + 40, *q = h->hscal + 49;
  if (!isfinite(q[0]) || !isfinite(q[1]) || !isfinite(q[2]) || !isfinite(q[3]) || !isfinite(q[4])) {
    set_error("he4_bubble_radius: non-finite density");
    return HE4_E_NONFINITE;
  }
  // xmsx = sqrt(sum denx x^2 * dxyz) with the program's dxyz (DFT4He3d.f90:945-947)
  for (int c = 0; c < 3; c++) res->xms[c] = sqrt(q[2 + c] * h->dxyz);
  // NGP cell of the mean position, ipx = 1.5 + (aux1 + xmax)/hx truncated (:896-898)
  const double lo[3] = {a.x0, a.y0, a.z0}, hh[3] = {a.hx, a.hy, a.hz};
  const int n[3] = {a.nx, a.ny, a.nz};
  double pc[3];
  for (int c = 0; c < 3; c++) {
    const double t = 1.5 + (m[c] - lo[c]) / hh[c];
    if (!(t >= 1.0 && t < n[c] + 1.0)) {
      set_error("he4_bubble_radius: mean impurity position %g outside the grid along axis %d", m[c], c);
      return HE4_E_ARG;
    }
    pc[c] = grid_coord(lo[c], hh[c], (int)t - 1);
  }
  // rmax from the grid's upper ends -x(1) = xmax (:22), dr = rmax/(nr-1)
  const double ex = -lo[0] - pc[0], ey = -lo[1] - pc[1], ez = -lo[2] - pc[2];
  const double rmax = sqrt(ex * ex + ey * ey + ez * ez);
  const double dr = rmax / (nr - 1);
  // xnorm with the bubble routine's own step x(2)-x(1) (:19-31)
  const double dx2 = grid_coord(a.x0, a.hx, 1) - a.x0, dy2 = grid_coord(a.y0, a.hy, 1) - a.y0,
               dz2 = grid_coord(a.z0, a.hz, 1) - a.z0;
  const double xnorm = q[0] * (dx2 * dy2 * dz2);
  // fixed-point scale: N * max|den| * 2^S < 2^61 bounds every bin sum
  const double N = (double)h->nx * h->ny * h->nz;
  int S = 60;
  if (q[1] > 0.0) S = (int)floor(61.0 - log2(N * q[1]));
  if (S > 200) S = 200;
  HistArgs ha;
  ha.nx = a.nx;
  ha.ny = a.ny;
  ha.nz = a.nz;
  ha.nr = nr;
  ha.x0 = a.x0;
  ha.y0 = a.y0;
  ha.z0 = a.z0;
  ha.hx = a.hx;
  ha.hy = a.hy;
  ha.hz = a.hz;
  ha.xp = pc[0];
  ha.yp = pc[1];
  ha.zp = pc[2];
  ha.dr = dr;
  ha.scale = ldexp(1.0, S);
  const size_t need = 2 * (size_t)nr + 1;
  if (h->bub_len < need) {
    cudaFree(h->bub);
    h->bub = nullptr;
    h->bub_len = 0;
    HE4_CUDA_TRY(cudaMalloc(&h->bub, need * sizeof(unsigned long long)));
    h->bub_len = need;
  }
  HE4_CUDA_TRY(cudaMemsetAsync(h->bub, 0, need * sizeof(unsigned long long), h->stream));
  const size_t shm = (size_t)nr * (sizeof(unsigned long long) + sizeof(unsigned int));
  HE4_CUDA_TRY(cudaFuncSetAttribute(k_bubble_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
  int per_sm = 0, nsm = 0, dev = 0;
  HE4_CUDA_TRY(cudaGetDevice(&dev));
  HE4_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  HE4_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bubble_hist, 256, shm));
  const int rows = a.ny * a.nz;
  int grid = nsm * (per_sm > 0 ? per_sm : 1);
  if (grid > (rows + 7) / 8) grid = (rows + 7) / 8;
  k_bubble_hist<<<grid, 256, shm, h->stream>>>(h->den, ha, h->bub);
  HE4_LAUNCHED(h);
  std::vector<unsigned long long> hb(need);
  HE4_CUDA_TRY(cudaMemcpyAsync(hb.data(), h->bub, need * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (hb[2 * nr]) {
    set_error("he4_bubble_radius: %llu points lie beyond r = rmax (the reference stops with '0001')",
              (unsigned long long)hb[2 * nr]);
    return HE4_E_ARG;
  }
  // bin means (:63-65)
  std::vector<double> rr(nr), denr(nr), work;
  const double inv = ldexp(1.0, -S);
  for (int b = 0; b < nr; b++) {
    const double sum = (double)(long long)hb[b] * inv;
    denr[b] = hb[nr + b] ? sum / (double)hb[nr + b] : 0.0;
  }
  bubble_search(nr, dr, xnorm, res->xms, rr.data(), denr.data(), res, work);
  if (rr_out) memcpy(rr_out, rr.data(), sizeof(double) * nr);
  if (denr_out) memcpy(denr_out, denr.data(), sizeof(double) * nr);
  return HE4_OK;
}

}  // namespace he4

extern "C" int he4_diagnostics_noalloc(const double *den, int32_t nx, int32_t ny, int32_t nz, double xmax,
                                       double ymax, double zmax, int32_t n4, double *out, void *stream) {
  using namespace he4;
  if (!den || !out || nx <= 0 || ny <= 0 || nz <= 0 || n4 <= 0 || !(xmax > 0) || !(ymax > 0) || !(zmax > 0)) {
    set_error("he4_diagnostics_noalloc: null array or non-positive size");
    return HE4_E_ARG;
  }
  if (nz > HE4_DIAG_NOALLOC_MAX_NZ) {
    set_error("he4_diagnostics_noalloc: nz=%d exceeds the fixed scratch of %d planes", nz, HE4_DIAG_NOALLOC_MAX_NZ);
    return HE4_E_ARG;
  }
  if ((int64_t)nx * ny > (int64_t)1 << 30) {
    set_error("he4_diagnostics_noalloc: nx*ny=%lld too large", (long long)nx * ny);
    return HE4_E_ARG;
  }
  double *part = nullptr;
  HE4_TRY(noalloc_scratch(&part));
  const DiagArgs a = diag_args(nx, ny, nz, xmax, ymax, zmax);
  const double dxyz = a.hx * a.hy * a.hz;
  return launch_diag(den, a, dxyz, (double)n4, part, out, static_cast<cudaStream_t>(stream), nullptr);
}

// diag.cu -- device-side diagnostics of the pener blocks: the He atom number
// sum(den)*dxyz (DFT4He3d.f90:885-886) and the centre of mass of the density
// (r_cm.f90:23-58), reduced on the GPU so no field has to be copied out.
//
// Two entry points share the kernels: he4_diagnostics works on a handle and
// takes its per-plane partial sums from the handle's reduction workspace;
// he4_diagnostics_noalloc works on caller-owned device arrays and takes them
// from the fixed array below, so it allocates nothing.
#include <mutex>

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
constexpr int kMaxDevices = 64;
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

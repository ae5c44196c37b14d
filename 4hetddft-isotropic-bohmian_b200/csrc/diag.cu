// diag.cu -- device-side diagnostics of the pener blocks: the He atom number
// sum(den)*dxyz (DFT4He3d.f90:885-886) and the centre of mass of the density
// (r_cm.f90:23-58), reduced on the GPU so no field has to be copied out.
#include "common.cuh"
#include "reduce.cuh"

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

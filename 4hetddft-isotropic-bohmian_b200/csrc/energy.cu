// energy.cu -- energy() (energy.f90:12-129) as one fused reduction pass.
//
// One kernel evaluates the first derivatives of psi (complex, npd-point
// periodic) and the seven grid sums of energy.f90 per CTA; a single CTA then
// adds the per-CTA partials in index order.  The host combines the sums with
// the same formulas as energy.f90:374-407.
#include "common.cuh"
#include "reduce.cuh"
#include "stencil.cuh"

namespace he4 {

struct EArgs {
  double aux1, aux2, beta, den_m;
  int otc;
};

constexpr int kESums = 7;  // ekin4, elj4, ecor4, ealphas, esolid, ekinqx, eHeX

__global__ void k_energy(const double2 *__restrict__ psi, const double *__restrict__ den,
                         const double *__restrict__ dencg, const double *__restrict__ delj4,
                         const double *__restrict__ falfs, const double *__restrict__ dx,
                         const double *__restrict__ dy, const double *__restrict__ dz,
                         const double *__restrict__ ix, const double *__restrict__ iy,
                         const double *__restrict__ iz, const double *__restrict__ psix,
                         const double *__restrict__ hpsix, const double *__restrict__ uimp, double *part,
                         size_t stride, Stencil st, Geo g, EArgs a) {
  __shared__ double sh[32];
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 8 + threadIdx.y;
  const int k = blockIdx.z;
  double v[kESums] = {0, 0, 0, 0, 0, 0, 0};
  if (i < g.nx && j < g.ny) {
    const size_t t = ((size_t)k * g.ny + j) * g.nx + i;
    const double2 d1 = stencil_axis_c(psi, st, 1, g, i, j, k, 0);
    const double2 d2 = stencil_axis_c(psi, st, 1, g, i, j, k, 1);
    const double2 d3 = stencil_axis_c(psi, st, 1, g, i, j, k, 2);
    v[0] = (d1.x * d1.x + d1.y * d1.y) + (d2.x * d2.x + d2.y * d2.y) + (d3.x * d3.x + d3.y * d3.y);
    const double dn = den[t], dc = dencg[t];
    v[1] = delj4[t] * dn;
    v[2] = dn * dc * dc * (a.aux1 + a.aux2 * dc);
    if (a.otc) v[3] = falfs[t] * (dx[t] * ix[t] + dy[t] * iy[t] + dz[t] * iz[t]);
    v[4] = dn * (1.0 + tanh(a.beta * (dn - a.den_m)));
    v[5] = psix[t] * hpsix[t];
    v[6] = uimp[t] * dn;
  }
  const size_t b = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
  for (int q = 0; q < kESums; q++) {
    const double s = block_sum(v[q], sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) part[q * stride + b] = s;
  }
}

__global__ void k_sumsq(const double *__restrict__ x, int n, double *out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int t = threadIdx.x; t < n; t += blockDim.x) acc += x[t] * x[t];
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) *out = s;
}

int compute_energy(Handle *h, he4_energies *E) {
  const Geo g{h->nx, h->ny, h->nz, zpad_of(h->p.icon)};
  const he4_params &p = h->p;
  EArgs a;
  a.aux1 = 0.5 * p.cp4;
  a.aux2 = (1.0 / 3.0) * p.cpp4;
  a.beta = p.beta_solid;
  a.den_m = p.den_m;
  a.otc = (p.core4 == HE4_CORE_OTC);
  dim3 gr = grid3(g);
  const size_t nb = (size_t)gr.x * gr.y * gr.z;
  if (kESums * nb > h->red_len) {
    set_error("reduction workspace too small");
    return HE4_E_STATE;
  }
  k_energy<<<gr, block3(), 0, h->stream>>>(h->psi, h->den, h->dencg, h->delj4, h->falfs, h->dxden, h->dyden,
                                           h->dzden, h->intx, h->inty, h->intz, h->psix, h->hpsix, h->uimp, h->red,
                                           nb, h->st, g, a);
  HE4_LAUNCHED(h);
  k_finalize_sums<<<1, 1024, 0, h->stream>>>(h->red, nb, (int)nb, kESums, 1.0, 1.0, h->scal + 16);
  HE4_LAUNCHED(h);
  k_sumsq<<<1, 1024, 0, h->stream>>>(h->vimp, 3 * h->npar, h->scal + 16 + kESums);
  HE4_LAUNCHED(h);
  HE4_CUDA_TRY(cudaMemcpyAsync(h->hscal + 16, h->scal + 16, sizeof(double) * (kESums + 1), cudaMemcpyDeviceToHost,
                               h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const double *s = h->hscal + 16;
  const double dxyz = h->dxyz;
  double ekin4 = p.h2o2m4 * s[0] * dxyz;
  double elj4 = 0.5 * s[1] * dxyz;
  double ecor4 = s[2] * dxyz;
  double ealphas = 0.0;
  if (a.otc) ealphas = -p.h2o2m4 * 0.5 * p.alphas * s[3] * dxyz;
  double esolid = p.c_solid * s[4] * dxyz;
  double etot4 = ekin4 + elj4 + ecor4 + esolid;
  if (a.otc) etot4 += ealphas;
  double ekinx = 0.5 * h->mAg_u * s[7] / h->npar;
  double ekinqx = s[5] * dxyz;
  double eHeX = s[6] * dxyz;
  double eimpu = ekinx + eHeX + ekinqx;
  E->etot = etot4 + eimpu;
  E->etot4 = etot4;
  E->ekin4 = ekin4;
  E->elj4 = elj4;
  E->ecor4 = ecor4;
  E->ealphas = ealphas;
  E->esolid = esolid;
  E->ekinx = ekinx;
  E->ekinqx = ekinqx;
  E->eHeX = eHeX;
  E->eimpu = eimpu;
  return HE4_OK;
}

}  // namespace he4

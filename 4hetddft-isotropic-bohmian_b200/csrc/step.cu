// step.cu -- RK-Gill starter and Hamming predictor-modifier-corrector for
// psi (complex, FP64) and for the Bohmian test particles.
//
// steprk.f90:1-128 and steppc.f90:1-155.  The reference moves history
// arrays with copies and ring indices; here the history buffers are pointers
// in the handle and the kernels write each new value straight into the slot
// it belongs to, so no array is copied:
//  * predictor: m is written into the psiold(ioldp(3)) buffer (read as
//    psi_{n-3} by the same thread first) and that buffer is swapped with psi,
//    which therefore lands in psiold(ioldp(3)) as steppc.f90:52 requires;
//  * corrector: psi_{n+1} goes to a scratch buffer that is swapped with psi.
// Each kernel evaluates the complex Laplacian of its input (npd-point
// periodic stencils) and H psi = timec*(h2o2m4*lap - pot4*psi) in registers.
#include <string.h>

#include <utility>

#include "common.cuh"
#include "reduce.cuh"
#include "stencil.cuh"

namespace he4 {

static Geo geo(const Handle *h) { return Geo{h->nx, h->ny, h->nz, zpad_of(h->p.icon)}; }

__global__ void k_finalize_sums(const double *__restrict__ part, size_t stride, int nb, int nvals, double mult,
                                double div, double *out) {
  __shared__ double sh[32];
  for (int v = 0; v < nvals; v++) {
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += part[v * stride + b];
    double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[v] = (s * mult) / div;
  }
}

struct PsiArgs {
  double h2o2m4, dt;
  const double *timec_re;  // [nz]
};

// H psi (the Sto4c of steppc.f90:46 / steprk.f90:218); ZPAD: icon=13
template <bool ZPAD>
__device__ __forceinline__ double2 hpsi_at(const double2 *__restrict__ psi, const double *__restrict__ pot4,
                                           const Stencil &st, const Geo &g, const PsiArgs &a, int i, int j, int k,
                                           size_t t) {
  const double2 lap = lap_c_t<ZPAD>(psi, st, g, i, j, k);
  const double2 ps = psi[t];
  const double v = pot4[t];
  const double2 w = make_double2(lap.x * a.h2o2m4 - v * ps.x, lap.y * a.h2o2m4 - v * ps.y);
  const double tr = a.timec_re[k];
  return make_double2(tr * w.x - w.y, tr * w.y + w.x);  // (tr + i) * w
}

// one RK-Gill stage (steprk.f90:211-229)
template <bool ZPAD>
__global__ void k_rk_stage(const double2 *__restrict__ psi, const double *__restrict__ pot4, double2 *q,
                           double2 *psi_out, double *den, double2 *h_first, double2 *p_first, double ar, double br,
                           double cr, Stencil st, Geo g, PsiArgs a) {
  HE4_IJK(g);
  const double2 s4 = hpsi_at<ZPAD>(psi, pot4, st, g, a, i, j, k, t);
  const double2 qv = q[t];
  const double2 s1 = make_double2(ar * (s4.x - br * qv.x), ar * (s4.y - br * qv.y));
  q[t] = make_double2(qv.x + 3.0 * s1.x - cr * s4.x, qv.y + 3.0 * s1.y - cr * s4.y);
  const double2 ps = psi[t];
  if (h_first) {
    h_first[t] = s4;
    p_first[t] = ps;
  }
  const double2 np = make_double2(ps.x + a.dt * s1.x, ps.y + a.dt * s1.y);
  psi_out[t] = np;
  den[t] = np.x * np.x + np.y * np.y;
}

// predictor + modifier (steppc.f90:36-56)
template <bool ZPAD>
__global__ void k_pc_predict(const double2 *__restrict__ psi, const double *__restrict__ pot4, double2 *p3,
                             const double2 *__restrict__ h1, double2 *h2, double2 *pc, double *den, Stencil st, Geo g,
                             PsiArgs a) {
  HE4_IJK(g);
  const double c112 = 112.0 / 121.0, c4o3 = 4.0 / 3.0;
  const double2 s4 = hpsi_at<ZPAD>(psi, pot4, st, g, a, i, j, k, t);
  const double2 o3 = p3[t], f1 = h1[t], f2 = h2[t];
  const double f = c4o3 * a.dt;
  const double2 pr = make_double2(o3.x + f * (2.0 * s4.x - f1.x + 2.0 * f2.x),
                                  o3.y + f * (2.0 * s4.y - f1.y + 2.0 * f2.y));
  const double2 pcv = pc[t];
  const double2 m = make_double2(pr.x - c112 * pcv.x, pr.y - c112 * pcv.y);
  p3[t] = m;
  pc[t] = pr;
  h2[t] = s4;
  den[t] = m.x * m.x + m.y * m.y;
}

// corrector + final value (steppc.f90:97-112); per-block partial sums of
// |pc| for errHe
template <bool ZPAD>
__global__ void k_pc_correct(const double2 *__restrict__ psi, const double *__restrict__ pot4,
                             const double2 *__restrict__ p3, const double2 *__restrict__ p2,
                             const double2 *__restrict__ h1, const double2 *__restrict__ h2, double2 *pc,
                             double2 *psi_out, double *den, double *part, Stencil st, Geo g, PsiArgs a) {
  __shared__ double sh[32];
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 8 + threadIdx.y;
  const int k = blockIdx.z;
  double e = 0.0;
  if (i < g.nx && j < g.ny) {
    const size_t t = ((size_t)k * g.ny + j) * g.nx + i;
    const double c9 = 9.0 / 121.0;
    const double2 s4 = hpsi_at<ZPAD>(psi, pot4, st, g, a, i, j, k, t);
    const double2 o3 = p3[t], o2 = p2[t], f1 = h1[t], f2 = h2[t];
    const double d3 = 3.0 * a.dt;
    const double2 s5 = make_double2(0.125 * (9.0 * o3.x - o2.x + d3 * (s4.x + 2.0 * f1.x - f2.x)),
                                    0.125 * (9.0 * o3.y - o2.y + d3 * (s4.y + 2.0 * f1.y - f2.y)));
    const double2 pco = pc[t];
    const double2 pcn = make_double2(pco.x - s5.x, pco.y - s5.y);
    pc[t] = pcn;
    const double2 np = make_double2(s5.x + c9 * pcn.x, s5.y + c9 * pcn.y);
    psi_out[t] = np;
    den[t] = np.x * np.x + np.y * np.y;
    e = sqrt(pcn.x * pcn.x + pcn.y * pcn.y);
  }
  const double s = block_sum(e, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    part[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
}

__global__ void k_den(const double2 *__restrict__ psi, double *den, size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    const double2 v = psi[t];
    den[t] = v.x * v.x + v.y * v.y;
  }
}

// ---------------------------------------------------------------------------
// particles: elementwise over n3 = 3 N_par values on part_grid() CTAs; the
// corrector errors and the means are grid-wide sums that stay deterministic
// (grid_sums_last: fixed-order per-CTA partials, summed in index order by
// the CTA that finishes last)
// ---------------------------------------------------------------------------
struct PartPtrs {
  double *rimp, *vimp, *aimp, *qr, *qv, *pcr, *pcv;
  double *r1, *r2, *r3, *v1, *v2, *v3, *a1, *a2;
  int n3;
};

static unsigned part_grid(int n) {
  return (unsigned)std::max(1, std::min(kPartMaxCta, (n + kPartThreads - 1) / kPartThreads));
}

// RK-Gill stage for positions and velocities (steprk.f90:236-260)
__global__ void __launch_bounds__(kPartThreads) k_part_rk(PartPtrs P, double ar, double br, double cr, double dt,
                                                          int first) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P.n3; t += gridDim.x * blockDim.x) {
    const double v = P.vimp[t];
    const double sr = ar * (v - br * P.qr[t]);
    P.qr[t] = P.qr[t] + 3.0 * sr - cr * v;
    if (first) P.r1[t] = P.rimp[t];
    P.rimp[t] = P.rimp[t] + dt * sr;
    const double acc = P.aimp[t];
    const double sv = ar * (acc - br * P.qv[t]);
    P.qv[t] = P.qv[t] + 3.0 * sv - cr * acc;
    if (first) {
      P.a1[t] = acc;
      P.v1[t] = v;
    }
    P.vimp[t] = v + dt * sv;
  }
}

// predictor + modifier for positions and velocities (steppc.f90:68-85).
// r1..r3 = rimpold(ioldr(1..3)) etc.
__global__ void __launch_bounds__(kPartThreads) k_part_predict(PartPtrs P, double dt) {
  const double c112 = 112.0 / 121.0, c4o3 = 4.0 / 3.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P.n3; t += gridDim.x * blockDim.x) {
    const double sr = P.r3[t] + c4o3 * dt * (2.0 * P.vimp[t] - P.v1[t] + 2.0 * P.v2[t]);
    P.r3[t] = P.rimp[t];
    P.rimp[t] = sr - c112 * P.pcr[t];
    P.pcr[t] = sr;
    const double sv = P.v3[t] + c4o3 * dt * (2.0 * P.aimp[t] - P.a1[t] + 2.0 * P.a2[t]);
    P.v3[t] = sv - c112 * P.pcv[t];
    P.pcv[t] = sv;
    P.a2[t] = P.aimp[t];
  }
}

// corrector for positions and velocities (steppc.f90:126-147); out[0..1] =
// errimp, errvimp (steppc.f90:136,147)
__global__ void __launch_bounds__(kPartThreads) k_part_correct(PartPtrs P, double dt, double npar, GridRed *gr,
                                                               double *out) {
  __shared__ double sh[kPartThreads / 32 + 1];
  const double c9 = 9.0 / 121.0;
  double e[2] = {0.0, 0.0};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P.n3; t += gridDim.x * blockDim.x) {
    const double sr = 0.125 * (9.0 * P.r3[t] - P.r2[t] + 3.0 * dt * (P.v3[t] + 2.0 * P.vimp[t] - P.v1[t]));
    const double pr = P.pcr[t] - sr;
    P.pcr[t] = pr;
    P.rimp[t] = sr + c9 * pr;
    e[0] += fabs(c9 * pr);
    // velocities use the pre-rotation ioldv slots (v2 = vimpold(ioldv(2)))
    const double sv = 0.125 * (9.0 * P.vimp[t] - P.v2[t] + 3.0 * dt * (P.aimp[t] + 2.0 * P.a1[t] - P.a2[t]));
    const double pv = P.pcv[t] - sv;
    P.pcv[t] = pv;
    P.v3[t] = P.vimp[t];
    P.vimp[t] = sv + c9 * pv;
    e[1] += fabs(c9 * pv);
  }
  double tot[2];
  if (grid_sums_last<2>(e, gr->part, &gr->count[1], sh, tot) && threadIdx.x == 0) {
    out[0] = tot[0] * 0.3333333333 / npar;
    out[1] = tot[1] * 0.3333333333 / npar;
  }
}

// means of rimp, vimp, aimp per axis (DFT4He3d.f90:864-878): out[a*3+c]
__global__ void __launch_bounds__(kPartThreads) k_part_means(const double *__restrict__ rimp,
                                                             const double *__restrict__ vimp,
                                                             const double *__restrict__ aimp, int npar, GridRed *gr,
                                                             double *out) {
  __shared__ double sh[kPartThreads / 32 + 1];
  double acc[9];
#pragma unroll
  for (int i = 0; i < 9; i++) acc[i] = 0.0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npar; p += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      acc[c] += rimp[c * npar + p];
      acc[3 + c] += vimp[c * npar + p];
      acc[6 + c] += aimp[c * npar + p];
    }
  }
  double tot[9];
  if (grid_sums_last<9>(acc, gr->part, &gr->count[2], sh, tot) && threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 9; i++) out[i] = tot[i] / npar;
}

// ---------------------------------------------------------------------------
// orchestration
// ---------------------------------------------------------------------------
static PsiArgs psi_args(const Handle *h, double dt) {
  PsiArgs a;
  a.h2o2m4 = h->p.h2o2m4;
  a.dt = dt;
  a.timec_re = h->timec_re;
  return a;
}

static PartPtrs part_ptrs(Handle *h) {
  PartPtrs P;
  P.rimp = h->rimp;
  P.vimp = h->vimp;
  P.aimp = h->aimp;
  P.qr = h->qr;
  P.qv = h->qv;
  P.pcr = h->pcr;
  P.pcv = h->pcv;
  P.r1 = h->rimpold[h->ioldr[0]];
  P.r2 = h->rimpold[h->ioldr[1]];
  P.r3 = h->rimpold[h->ioldr[2]];
  P.v1 = h->vimpold[h->ioldv[0]];
  P.v2 = h->vimpold[h->ioldv[1]];
  P.v3 = h->vimpold[h->ioldv[2]];
  P.a1 = h->aimpold[h->iolda[0]];
  P.a2 = h->aimpold[h->iolda[1]];
  P.n3 = 3 * h->npar;
  return P;
}

int compute_den(Handle *h) {
  k_den<<<(unsigned)((h->N + 255) / 256), 256, 0, h->stream>>>(h->psi, h->den, h->N);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int field_all(Handle *h, bool split) {
  split = split || !fft_z_sum_ok(h);
  h->field_valid = 0;
  h->split_valid = 0;
  HE4_TRY(field_potenimp(h, split));
  HE4_TRY(field_poten(h, split, h->pot4));
  HE4_TRY(field_forceimp(h, false));
  h->field_valid = 1;
  h->split_valid = split ? 1 : 0;
  return HE4_OK;
}

int field_split_fields(Handle *h) {
  // the split poten writes its pot4 into spec[5], free outside an evaluation
  // (2 (nx/2+1) >= nx reals per row)
  HE4_TRY(field_potenimp(h, true));
  HE4_TRY(field_poten(h, true, reinterpret_cast<double *>(h->spec[5])));
  h->split_valid = 1;
  return HE4_OK;
}

int particle_means(Handle *h, double *dmeans) {
  k_part_means<<<part_grid(h->npar), kPartThreads, 0, h->stream>>>(h->rimp, h->vimp, h->aimp, h->npar, h->gred,
                                                                   dmeans);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

template <typename T>
static void rot3(T *a) {  // (a0,a1,a2) <- (a2,a0,a1): physical shift of steprk.f90:224-226
  T t = a[2];
  a[2] = a[1];
  a[1] = a[0];
  a[0] = t;
}

// dres: device array, [0..2] errors (zero for RK) and [3..11] means
int step_rk(Handle *h, double dt, double *dres) {
  const Geo g = geo(h);
  if (!h->field_valid) HE4_TRY(field_all(h));  // DFT4He3d.f90:630-634
  const double s2 = sqrt(2.0);
  const double arun[4] = {0.5, 1.0 - 1.0 / s2, 1.0 + 1.0 / s2, 1.0 / 6.0};
  const double brun[4] = {2.0, 1.0, 1.0, 2.0};
  const double crun[4] = {0.5, 1.0 - 1.0 / s2, 1.0 + 1.0 / s2, 0.5};
  const PsiArgs pa = psi_args(h, dt);
  for (int jr = 0; jr < 4; jr++) {
    double2 *hf = nullptr, *pf = nullptr;
    if (jr == 0) {
      std::swap(h->hpsiold[0], h->hpsiold[1]);
      rot3(h->psiold);
      hf = h->hpsiold[0];
      pf = h->psiold[0];
    }
    if (g.zpad)
      k_rk_stage<true><<<grid3(g), block3(), 0, h->stream>>>(h->psi, h->pot4, h->q, h->ctmp, h->den, hf, pf,
                                                             arun[jr], brun[jr], crun[jr], h->st, g, pa);
    else
      k_rk_stage<false><<<grid3(g), block3(), 0, h->stream>>>(h->psi, h->pot4, h->q, h->ctmp, h->den, hf, pf,
                                                              arun[jr], brun[jr], crun[jr], h->st, g, pa);
    HE4_LAUNCHED(h);
    std::swap(h->psi, h->ctmp);
    if (jr == 0) {
      rot3(h->rimpold);
      rot3(h->vimpold);
      std::swap(h->aimpold[0], h->aimpold[1]);
    }
    // ring indices are the identity during the starter
    for (int i = 0; i < 3; i++) h->ioldr[i] = h->ioldv[i] = h->ioldp[i] = i;
    for (int i = 0; i < 2; i++) h->iolda[i] = h->ioldh[i] = i;
    k_part_rk<<<part_grid(3 * h->npar), kPartThreads, 0, h->stream>>>(part_ptrs(h), arun[jr], brun[jr], crun[jr],
                                                                       dt, jr == 0);
    HE4_LAUNCHED(h);
    if (jr <= 2) HE4_TRY(field_all(h));
  }
  HE4_TRY(field_all(h));
  HE4_CUDA_TRY(cudaMemsetAsync(dres, 0, 3 * sizeof(double), h->stream));
  HE4_TRY(particle_means(h, dres + 3));
  h->nsteps_done++;
  return HE4_OK;
}

int step_pc(Handle *h, double dt, double *dres) {
  const Geo g = geo(h);
  const PsiArgs pa = psi_args(h, dt);
  if (!h->field_valid) HE4_TRY(field_all(h));
  // predictor + modifier for psi
  {
    double2 *p3 = h->psiold[h->ioldp[2]];
    if (g.zpad)
      k_pc_predict<true><<<grid3(g), block3(), 0, h->stream>>>(h->psi, h->pot4, p3, h->hpsiold[h->ioldh[0]],
                                                               h->hpsiold[h->ioldh[1]], h->pc, h->den, h->st, g, pa);
    else
      k_pc_predict<false><<<grid3(g), block3(), 0, h->stream>>>(h->psi, h->pot4, p3, h->hpsiold[h->ioldh[0]],
                                                                h->hpsiold[h->ioldh[1]], h->pc, h->den, h->st, g, pa);
    HE4_LAUNCHED(h);
    std::swap(h->psi, h->psiold[h->ioldp[2]]);
    std::swap(h->ioldh[0], h->ioldh[1]);
  }
  // particles
  k_part_predict<<<part_grid(3 * h->npar), kPartThreads, 0, h->stream>>>(part_ptrs(h), dt);
  HE4_LAUNCHED(h);
  std::swap(h->iolda[0], h->iolda[1]);
  HE4_TRY(field_all(h));
  // corrector for psi
  {
    dim3 gr = grid3(g);
    const int nb = (int)(gr.x * gr.y * gr.z);
    if (g.zpad)
      k_pc_correct<true><<<gr, block3(), 0, h->stream>>>(h->psi, h->pot4, h->psiold[h->ioldp[2]],
                                                         h->psiold[h->ioldp[1]], h->hpsiold[h->ioldh[0]],
                                                         h->hpsiold[h->ioldh[1]], h->pc, h->ctmp, h->den, h->red,
                                                         h->st, g, pa);
    else
      k_pc_correct<false><<<gr, block3(), 0, h->stream>>>(h->psi, h->pot4, h->psiold[h->ioldp[2]],
                                                          h->psiold[h->ioldp[1]], h->hpsiold[h->ioldh[0]],
                                                          h->hpsiold[h->ioldh[1]], h->pc, h->ctmp, h->den, h->red,
                                                          h->st, g, pa);
    HE4_LAUNCHED(h);
    std::swap(h->psi, h->ctmp);
    rot3(h->ioldp);
    // errHe = 9/121 * sum|pc| / nxyz
    k_finalize_sums<<<1, 1024, 0, h->stream>>>(h->red, 0, nb, 1, 9.0 / 121.0, (double)h->N, dres);
    HE4_LAUNCHED(h);
  }
  // particles corrector (uses the pre-rotation ring indices), then rotations
  k_part_correct<<<part_grid(3 * h->npar), kPartThreads, 0, h->stream>>>(part_ptrs(h), dt, (double)h->npar,
                                                                           h->gred, dres + 1);
  HE4_LAUNCHED(h);
  rot3(h->ioldr);
  rot3(h->ioldv);
  HE4_TRY(field_all(h));
  HE4_TRY(particle_means(h, dres + 3));
  h->nsteps_done++;
  return HE4_OK;
}

// ---------------------------------------------------------------------------
// CUDA graphs of the PC step
// ---------------------------------------------------------------------------
StepState get_step_state(const Handle *h, double dt) {
  StepState s;
  memset(&s, 0, sizeof(s));
  s.psi = h->psi;
  s.ctmp = h->ctmp;
  for (int i = 0; i < 3; i++) {
    s.psiold[i] = h->psiold[i];
    s.rimpold[i] = h->rimpold[i];
    s.vimpold[i] = h->vimpold[i];
    s.ioldp[i] = h->ioldp[i];
    s.ioldr[i] = h->ioldr[i];
    s.ioldv[i] = h->ioldv[i];
  }
  for (int i = 0; i < 2; i++) {
    s.hpsiold[i] = h->hpsiold[i];
    s.aimpold[i] = h->aimpold[i];
    s.ioldh[i] = h->ioldh[i];
    s.iolda[i] = h->iolda[i];
  }
  s.dt = dt;
  return s;
}

void set_step_state(Handle *h, const StepState &s) {
  h->psi = s.psi;
  h->ctmp = s.ctmp;
  for (int i = 0; i < 3; i++) {
    h->psiold[i] = s.psiold[i];
    h->rimpold[i] = s.rimpold[i];
    h->vimpold[i] = s.vimpold[i];
    h->ioldp[i] = s.ioldp[i];
    h->ioldr[i] = s.ioldr[i];
    h->ioldv[i] = s.ioldv[i];
  }
  for (int i = 0; i < 2; i++) {
    h->hpsiold[i] = s.hpsiold[i];
    h->aimpold[i] = s.aimpold[i];
    h->ioldh[i] = s.ioldh[i];
    h->iolda[i] = s.iolda[i];
  }
}

void free_graphs(Handle *h) {
  for (StepGraph &g : h->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  h->graphs.clear();
}

// The PC step's buffer states repeat with period 30: the two swaps per step
// (psi with the history slot ioldp(3), then psi with ctmp) permute the five
// psi buffers with order 5, and the ring indices have period 6.  One graph
// per state; he4_set_state restores the allocation order, so every run
// walks the same 30 states.
constexpr size_t kMaxGraphs = 30;

// Capture one PC step from the current state (results into h->scal).  The
// host state advances exactly as an eager step would; the graph has not run.
static int capture_pc(Handle *h, double dt, StepGraph *out) {
  StepGraph g;
  g.before = get_step_state(h, dt);
  const int64_t l0 = h->launches;
  const int done0 = h->nsteps_done;
  HE4_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = step_pc(h, dt, h->scal);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
  h->nsteps_done = done0;
  g.kernels = h->launches - l0;
  h->launches = l0;
  if (rc != HE4_OK || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    set_step_state(h, g.before);
    if (rc == HE4_OK) set_error("stream capture of the PC step: %s", cudaGetErrorString(ce));
    cudaGetLastError();
    return rc != HE4_OK ? rc : HE4_E_CUDA;
  }
  g.graph = graph;
  const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
  if (ie != cudaSuccess) {
    cudaGraphDestroy(graph);
    set_step_state(h, g.before);
    set_error("graph instantiation: %s", cudaGetErrorString(ie));
    return HE4_E_CUDA;
  }
  g.after = get_step_state(h, dt);
  *out = g;
  return HE4_OK;
}

int run_pc_graphs(Handle *h, int n, double dt, double *dres) {
  if (!h->field_valid) HE4_TRY(field_all(h));
  for (int s = 0; s < n; s++) {
    const StepState now = get_step_state(h, dt);
    StepGraph *hit = nullptr;
    for (StepGraph &g : h->graphs)
      if (same_step_state(g.before, now)) {
        hit = &g;
        break;
      }
    if (!hit && h->graphs.size() < kMaxGraphs) {
      StepGraph g;
      HE4_TRY(capture_pc(h, dt, &g));
      h->graph_captures++;
      set_step_state(h, g.before);
      h->graphs.push_back(g);
      hit = &h->graphs.back();
    }
    if (hit) {
      HE4_CUDA_TRY(cudaGraphLaunch(hit->exec, h->stream));
      h->launches += hit->kernels;
      set_step_state(h, hit->after);
      h->nsteps_done++;
      // what the captured step's merged evaluation leaves, as step_pc does:
      // pot4 and the forces of the new state, not the split fields (delj4,
      // uimp, ...) nor the forces outside the particle box
      h->field_valid = 1;
      h->split_valid = 0;
      h->forces_full = 0;
      if (dres + 12 * (size_t)s != h->scal)
        HE4_CUDA_TRY(cudaMemcpyAsync(dres + 12 * (size_t)s, h->scal, 12 * sizeof(double), cudaMemcpyDeviceToDevice,
                                     h->stream));
    } else {
      h->steps_uncaptured++;
      HE4_TRY(step_pc(h, dt, dres + 12 * (size_t)s));
    }
  }
  return HE4_OK;
}

}  // namespace he4

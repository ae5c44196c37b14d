// abi.cu -- the extern "C" entry points of include/he4_tddft.h.
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include "common.cuh"

namespace he4 {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

static bool valid_n(int n) {
  // grid sizes accepted by the reference (tstgrid.f90:8-12)
  static const int nv[52] = {1,   2,   3,   4,   5,   6,   8,   9,   10,  12,  15,  16,  18,
                             20,  24,  25,  27,  30,  32,  36,  40,  45,  48,  50,  54,  60,
                             64,  72,  75,  80,  81,  90,  96,  100, 108, 120, 125, 128, 135,
                             144, 150, 160, 162, 180, 192, 200, 216, 225, 240, 243, 250, 256};
  for (int i = 0; i < 52; i++)
    if (nv[i] == n) return true;
  return false;
}

static int check_params(const he4_params *p) {
  if (!valid_n(p->nx) || !valid_n(p->ny) || !valid_n(p->nz)) {
    set_error("grid %dx%dx%d: every size must be a valid FFT size <= 256 (tstgrid)", p->nx, p->ny, p->nz);
    return HE4_E_ARG;
  }
  if (p->nx < 8 || p->ny < 8 || p->nz < 8) {
    set_error("grid sizes below 8 are not supported");
    return HE4_E_UNSUPPORTED;
  }
  if (p->npd < 3 || p->npd > 25 || p->npd % 2 == 0) {
    set_error("npd=%d must be odd in [3,25]", p->npd);
    return HE4_E_ARG;
  }
  if (p->npd > p->nx || p->npd > p->ny || p->npd > p->nz) {
    set_error("npd=%d exceeds a grid dimension", p->npd);
    return HE4_E_ARG;
  }
  if (p->icon != 8 && p->icon != 12 && p->icon != 13) {
    set_error("icon=%d: periodic (icon=8) and Redef's icon=12 and icon=13 boundaries are implemented", p->icon);
    return HE4_E_UNSUPPORTED;
  }
  if (p->icon == 12 && p->npd > 15) {
    set_error("icon=12 needs npd <= 15 (one-sided boundary rows of the Bickley matrix)");
    return HE4_E_UNSUPPORTED;
  }
  if (p->core4 != HE4_CORE_OT && p->core4 != HE4_CORE_OTC) {
    set_error("core4=%d is not supported", p->core4);
    return HE4_E_UNSUPPORTED;
  }
  if (p->n_par < 1 || p->n_par > (1 << 24)) {
    set_error("n_par=%d out of range", p->n_par);
    return HE4_E_ARG;
  }
  if (p->ironx < 0 || p->mimpur <= 0.0 || !(p->xmax > 0) || !(p->ymax > 0) || !(p->zmax > 0)) {
    set_error("invalid ironx, mimpur or box size");
    return HE4_E_ARG;
  }
  if (p->pot_kind != HE4_POT_TABLE && p->pot_kind != HE4_POT_MORSE && p->pot_kind != HE4_POT_NULL &&
      p->pot_kind != HE4_POT_RTABLE && p->pot_kind != HE4_POT_HE2S_FCI) {
    set_error("unknown pot_kind %d", p->pot_kind);
    return HE4_E_ARG;
  }
  if (p->precision != HE4_PREC_FP64 && p->precision != HE4_PREC_FP32CONV) {
    set_error("precision mode %d is not implemented", p->precision);
    return HE4_E_UNSUPPORTED;
  }
  if (p->precision == HE4_PREC_FP32CONV) {
    auto reg = [](int n) { return n >= 16 && n <= 256 && (n & (n - 1)) == 0; };
    if (!reg(p->nx) || !reg(p->ny) || !reg(p->nz)) {
      set_error("the FP32-convolution form needs power-of-two axes in [16, 256] (got %d x %d x %d)", p->nx, p->ny,
                p->nz);
      return HE4_E_UNSUPPORTED;
    }
  }
  return HE4_OK;
}

template <typename T>
static int dalloc(T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (n ? n : 1));
  if (e != cudaSuccess) {
    set_error("cudaMalloc of %zu bytes: %s", sizeof(T) * n, cudaGetErrorString(e));
    *p = nullptr;
    return HE4_E_NOMEM;
  }
  return HE4_OK;
}

static void free_all(Handle *h) {
  free_graphs(h);
  fft_plan_free(h->fft);
  void *ptrs[] = {h->wcgk, h->fvlj4, h->kalfs, h->vq, h->pmod, h->dsym, h->timec_re, h->psi, h->psiold[0],
                  h->psiold[1], h->psiold[2], h->hpsiold[0], h->hpsiold[1], h->pc, h->q, h->ctmp, h->den, h->pot4,
                  h->dencg, h->delj4, h->denalf, h->ualphas, h->falfs, h->intx, h->inty, h->intz, h->dxden,
                  h->dyden, h->dzden, h->penalty, h->corr, h->denx, h->psix, h->hpsix, h->uimp, h->fx, h->fy,
                  h->fz, h->rtmp[0], h->rtmp[1], h->rtmp[2], h->rtmp[3], h->counts, h->rimp, h->vimp, h->aimp,
                  h->rimpold[0], h->rimpold[1], h->rimpold[2], h->vimpold[0], h->vimpold[1], h->vimpold[2],
                  h->aimpold[0], h->aimpold[1], h->qr, h->qv, h->pcr, h->pcv, h->red, h->scal, h->bub, h->box, h->gred, h->st_lo,
                  h->k32[0], h->k32[1], h->k32[2], h->k32[3], h->dsym32};
  for (void *p : ptrs) cudaFree(p);
  for (int i = 0; i < 9; i++) cudaFree(h->g32[i]);
  if (h->snap_stream) cudaStreamSynchronize(h->snap_stream);
  cudaFree(h->snap_dev);
  if (h->snap_host) cudaFreeHost(h->snap_host);
  if (h->snap_taken) cudaEventDestroy(h->snap_taken);
  if (h->snap_done) cudaEventDestroy(h->snap_done);
  if (h->snap_stream) cudaStreamDestroy(h->snap_stream);
  for (int i = 0; i < 8; i++) cudaFree(h->spec[i]);
  if (h->hscal) cudaFreeHost(h->hscal);
  if (h->stream) cudaStreamDestroy(h->stream);
}

static int create(const he4_params *pin, Handle *h) {
  HE4_TRY(check_params(pin));
  h->p = *pin;
  h->p.vq_table = nullptr;
  h->p.vr_table = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return HE4_E_NODEVICE;
  }
  if (pin->device < 0 || pin->device >= ndev || pin->device >= kMaxDevices) {
    set_error("device %d out of range (%d devices)", pin->device, ndev);
    return HE4_E_ARG;
  }
  h->dev = pin->device;
  // HE4_STREAM_STENCILS=0 selects the register z-marching stencils instead of
  // the bulk-copy streamed ones (same results to rounding; for comparisons)
  {
    const char *s = getenv("HE4_STREAM_STENCILS");
    h->use_stream = (s && s[0] == '0') ? 0 : 1;
    // HE4_POT4_SPLIT=0: the FP32 form's pot4 stencil sums in FP64 instead
    const char *q = getenv("HE4_POT4_SPLIT");
    h->pot4_split = (q && q[0] == '0') ? 0 : 1;
    // HE4_ZCONV_SHARE_XY=0: the x and y force outputs transformed separately
    const char *z = getenv("HE4_ZCONV_SHARE_XY");
    h->zconv_share_xy = (z && z[0] == '0') ? 0 : 1;
  }
  HE4_CUDA_TRY(cudaSetDevice(h->dev));
  cudaDeviceProp prop;
  HE4_CUDA_TRY(cudaGetDeviceProperties(&prop, h->dev));
  if (prop.major < 10) {
    set_error("device %d (%s, sm_%d%d) is not an sm_100 GPU", h->dev, prop.name, prop.major, prop.minor);
    return HE4_E_NODEVICE;
  }
  HE4_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  const he4_params &p = h->p;
  h->nx = p.nx;
  h->ny = p.ny;
  h->nz = p.nz;
  h->nxh = p.nx / 2 + 1;
  h->npar = p.n_par;
  h->N = (size_t)p.nx * p.ny * p.nz;
  h->H = (size_t)h->nxh * p.ny * p.nz;
  h->hx = 2.0 * fabs(p.xmax) / p.nx;
  h->hy = 2.0 * fabs(p.ymax) / p.ny;
  h->hz = 2.0 * fabs(p.zmax) / p.nz;
  h->dxyz = h->hx * h->hy * h->hz;
  h->renor = 1.0 / ((double)p.nx * p.ny * p.nz);
  h->mAg_u = p.mimpur * 0.0206149591055;  // mp_u (modules.f90:314)
  h->h2o2mx = p.h2o2m4 * (4.002602 / p.mimpur);
  const size_t N = h->N, H = h->H, P3 = 3 * (size_t)h->npar;
  HE4_TRY(fft_plan_init(h->fft, p.nx, p.ny, p.nz));
  HE4_TRY(dalloc(&h->wcgk, H));
  HE4_TRY(dalloc(&h->fvlj4, H));
  HE4_TRY(dalloc(&h->kalfs, H));
  HE4_TRY(dalloc(&h->vq, H));
  HE4_TRY(dalloc(&h->pmod, H));
  HE4_TRY(dalloc(&h->dsym, (size_t)p.nx + p.ny + p.nz));
  HE4_TRY(dalloc(&h->timec_re, (size_t)p.nz));
  h->fp32 = (p.precision == HE4_PREC_FP32CONV);
  if (h->fp32) {
    for (int i = 0; i < 4; i++) HE4_TRY(dalloc(&h->k32[i], H));
    HE4_TRY(dalloc(&h->dsym32, (size_t)p.nx + p.ny + p.nz));
  }
  double2 **cfields[] = {&h->psi, &h->psiold[0], &h->psiold[1], &h->psiold[2], &h->hpsiold[0],
                         &h->hpsiold[1], &h->pc, &h->q, &h->ctmp};
  for (double2 **f : cfields) HE4_TRY(dalloc(f, N));
  double **rfields[] = {&h->den, &h->pot4, &h->dencg, &h->delj4, &h->denalf, &h->ualphas, &h->falfs,
                        &h->intx, &h->inty, &h->intz, &h->dxden, &h->dyden, &h->dzden, &h->penalty,
                        &h->corr, &h->denx, &h->psix, &h->hpsix, &h->uimp, &h->fx, &h->fy, &h->fz,
                        &h->rtmp[0], &h->rtmp[1], &h->rtmp[2], &h->rtmp[3]};
  for (double **f : rfields) HE4_TRY(dalloc(f, N));
  HE4_TRY(dalloc(&h->counts, N));
  HE4_TRY(dalloc(&h->box, 1));
  HE4_TRY(dalloc(&h->gred, 1));
  {
    GridRed g0;
    memset(&g0, 0, sizeof(g0));
    for (int d = 0; d < 3; d++) {
      g0.box[d] = INT_MAX;
      g0.box[3 + d] = INT_MIN;
    }
    HE4_CUDA_TRY(cudaMemcpy(h->gred, &g0, sizeof(GridRed), cudaMemcpyHostToDevice));
  }
  for (int i = 0; i < 6; i++) HE4_TRY(dalloc(&h->spec[i], H));
  double **pfields[] = {&h->rimp, &h->vimp, &h->aimp, &h->rimpold[0], &h->rimpold[1], &h->rimpold[2],
                        &h->vimpold[0], &h->vimpold[1], &h->vimpold[2], &h->aimpold[0], &h->aimpold[1],
                        &h->qr, &h->qv, &h->pcr, &h->pcv};
  for (double **f : pfields) HE4_TRY(dalloc(f, P3));
  {
    double2 *hc[7] = {h->psi, h->ctmp, h->psiold[0], h->psiold[1], h->psiold[2], h->hpsiold[0], h->hpsiold[1]};
    double *hp[8] = {h->rimpold[0], h->rimpold[1], h->rimpold[2], h->vimpold[0],
                     h->vimpold[1], h->vimpold[2], h->aimpold[0], h->aimpold[1]};
    memcpy(h->home_c, hc, sizeof(hc));
    memcpy(h->home_p, hp, sizeof(hp));
  }
  // per-CTA partial sums of the grid reductions (7 energy sums max)
  const size_t nblocks = (size_t)((p.nx + 31) / 32) * ((p.ny + 7) / 8) * p.nz;
  h->red_len = 8 * nblocks;
  HE4_TRY(dalloc(&h->red, h->red_len));
  HE4_TRY(dalloc(&h->scal, 64));
  HE4_CUDA_TRY(cudaMallocHost((void **)&h->hscal, 64 * sizeof(double)));
  // the histories start at zero (dimen.f90:75-79,133-134; DFT4He3d.f90:841-845)
  for (double2 **f : cfields) HE4_CUDA_TRY(cudaMemsetAsync(*f, 0, sizeof(double2) * N, h->stream));
  for (double **f : rfields) HE4_CUDA_TRY(cudaMemsetAsync(*f, 0, sizeof(double) * N, h->stream));
  for (double **f : pfields) HE4_CUDA_TRY(cudaMemsetAsync(*f, 0, sizeof(double) * P3, h->stream));
  HE4_CUDA_TRY(cudaMemsetAsync(h->counts, 0, sizeof(unsigned int) * N, h->stream));
  HE4_TRY(impurity_reset_box(h));
  he4_params with_table = p;
  with_table.vq_table = pin->vq_table;
  with_table.vr_table = pin->vr_table;
  h->p = with_table;
  int e = setup_kernels(h);
  h->p.vq_table = nullptr;
  h->p.vr_table = nullptr;
  HE4_TRY(e);
  // (after setup_kernels, which sets the stencil width real32_ok reads)
  h->real32 = real32_ok(h) ? 1 : 0;
  if (h->real32)
    for (int i = 0; i < 9; i++) {
      HE4_TRY(dalloc(&h->g32[i], N));
      HE4_CUDA_TRY(cudaMemsetAsync(h->g32[i], 0, sizeof(float) * N, h->stream));
    }
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

}  // namespace he4

using namespace he4;

extern "C" {

void he4_params_default(he4_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->nx = p->ny = p->nz = 64;
  p->xmax = p->ymax = p->zmax = 64.0;
  p->npd = 7;
  p->icon = 8;
  p->core4 = HE4_CORE_OT;
  p->cp4 = -2.41186e4;
  p->cpp4 = 1.85850e6;
  p->den4c = 0.062;
  p->alphas = 54.31;
  p->l_alfs = 1.0;
  p->den0s = 0.04;
  p->h2o2m4 = 6.05969638298;
  p->c_solid = 3.1577504e4;
  p->beta_solid = 40.0;
  p->den_m = 0.37;
  p->eps4 = 10.22;
  p->sigma4 = 2.556;
  p->b4 = -718.99;
  p->h4 = 2.190323;
  p->n_par = 100000;
  p->ironx = 1;
  p->mimpur = 4.002602;
  p->pot_kind = HE4_POT_NULL;
  p->r_cutoff = 3.0;
  p->umax = 400.0;
  p->nq = 1000;
  p->lambdah = 0.0;
  p->tzmean = 0.0;
  p->tzsurf = 1.0;
  p->precision = HE4_PREC_FP64;
  p->device = 0;
}

int he4_create(const he4_params *p, he4_handle **out) {
  if (!p || !out) {
    set_error("null argument");
    return HE4_E_ARG;
  }
  *out = nullptr;
  he4_handle *hh = new (std::nothrow) he4_handle();
  if (!hh) {
    set_error("host allocation failed");
    return HE4_E_NOMEM;
  }
  int e = create(p, &hh->h);
  if (e != HE4_OK) {
    free_all(&hh->h);
    delete hh;
    return e;
  }
  *out = hh;
  return HE4_OK;
}

void he4_destroy(he4_handle *hh) {
  if (!hh) return;
  cudaSetDevice(hh->h.dev);
  if (hh->h.stream) cudaStreamSynchronize(hh->h.stream);
  free_all(&hh->h);
  delete hh;
}

#define HANDLE_OR_FAIL(hh)                 \
  if (!(hh)) {                             \
    set_error("null handle");              \
    return HE4_E_ARG;                      \
  }                                        \
  Handle *h = &(hh)->h;                    \
  if (cudaSetDevice(h->dev) != cudaSuccess) { \
    set_error("cudaSetDevice failed");     \
    return HE4_E_CUDA;                     \
  }

#define NEED_STATE(h)                                   \
  if (!(h)->have_state) {                               \
    set_error("no state: call he4_set_state first");    \
    return HE4_E_STATE;                                 \
  }

int he4_set_state(he4_handle *hh, const double *psi, const double *rimp, const double *vimp) {
  HANDLE_OR_FAIL(hh);
  if (!psi || !rimp || !vimp) {
    set_error("null state array");
    return HE4_E_ARG;
  }
  const size_t N = h->N, P3 = 3 * (size_t)h->npar;
  // the rotating buffers back in their allocation order: the steps from
  // here walk the same cycle of buffer states as every earlier run, so the
  // graphs captured then are replayed (the contents are all rewritten below)
  h->psi = h->home_c[0];
  h->ctmp = h->home_c[1];
  for (int i = 0; i < 3; i++) {
    h->psiold[i] = h->home_c[2 + i];
    h->rimpold[i] = h->home_p[i];
    h->vimpold[i] = h->home_p[3 + i];
  }
  for (int i = 0; i < 2; i++) {
    h->hpsiold[i] = h->home_c[5 + i];
    h->aimpold[i] = h->home_p[6 + i];
  }
  HE4_CUDA_TRY(cudaMemcpyAsync(h->psi, psi, sizeof(double2) * N, cudaMemcpyDefault, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(h->rimp, rimp, sizeof(double) * P3, cudaMemcpyDefault, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(h->vimp, vimp, sizeof(double) * P3, cudaMemcpyDefault, h->stream));
  HE4_CUDA_TRY(cudaMemsetAsync(h->aimp, 0, sizeof(double) * P3, h->stream));
  double2 *cz[] = {h->psiold[0], h->psiold[1], h->psiold[2], h->hpsiold[0], h->hpsiold[1], h->pc, h->q};
  for (double2 *f : cz) HE4_CUDA_TRY(cudaMemsetAsync(f, 0, sizeof(double2) * N, h->stream));
  double *pz[] = {h->rimpold[0], h->rimpold[1], h->rimpold[2], h->vimpold[0], h->vimpold[1], h->vimpold[2],
                  h->aimpold[0], h->aimpold[1], h->qr, h->qv, h->pcr, h->pcv};
  for (double *f : pz) HE4_CUDA_TRY(cudaMemsetAsync(f, 0, sizeof(double) * P3, h->stream));
  for (int i = 0; i < 3; i++) h->ioldp[i] = h->ioldr[i] = h->ioldv[i] = i;
  for (int i = 0; i < 2; i++) h->ioldh[i] = h->iolda[i] = i;
  HE4_TRY(compute_den(h));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->have_state = 1;
  h->nsteps_done = 0;
  h->field_valid = 0;
  return HE4_OK;
}

int he4_get_state(he4_handle *hh, double *psi, double *rimp, double *vimp, double *aimp) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  const size_t P3 = 3 * (size_t)h->npar;
  if (psi) HE4_CUDA_TRY(cudaMemcpyAsync(psi, h->psi, sizeof(double2) * h->N, cudaMemcpyDefault, h->stream));
  if (rimp) HE4_CUDA_TRY(cudaMemcpyAsync(rimp, h->rimp, sizeof(double) * P3, cudaMemcpyDefault, h->stream));
  if (vimp) HE4_CUDA_TRY(cudaMemcpyAsync(vimp, h->vimp, sizeof(double) * P3, cudaMemcpyDefault, h->stream));
  if (aimp) HE4_CUDA_TRY(cudaMemcpyAsync(aimp, h->aimp, sizeof(double) * P3, cudaMemcpyDefault, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

// Checkpoint snapshot: a device-to-device copy of the state on the
// handle's stream, then a device-to-host copy on a copy stream that
// overlaps the time steps enqueued after it.
int he4_snapshot_begin(he4_handle *hh) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  const size_t P3 = 3 * (size_t)h->npar, n = 2 * h->N + 3 * P3;
  if (h->snap_pending) {  // one snapshot in flight at a time
    HE4_CUDA_TRY(cudaEventSynchronize(h->snap_done));
    h->snap_pending = 0;
  }
  if (!h->snap_dev) {
    // all five resources or none: a partial set is released and the
    // handle keeps none, so the next call starts over
    double *dev = nullptr, *host = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t taken = nullptr, done = nullptr;
    cudaError_t ce = cudaMalloc((void **)&dev, sizeof(double) * n);
    if (ce == cudaSuccess) ce = cudaMallocHost((void **)&host, sizeof(double) * n);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&taken, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
    if (ce != cudaSuccess) {
      if (done) cudaEventDestroy(done);
      if (taken) cudaEventDestroy(taken);
      if (st) cudaStreamDestroy(st);
      if (host) cudaFreeHost(host);
      if (dev) cudaFree(dev);
      set_error("he4_snapshot_begin allocation: %s", cudaGetErrorString(ce));
      return HE4_E_CUDA;
    }
    h->snap_dev = dev;
    h->snap_host = host;
    h->snap_stream = st;
    h->snap_taken = taken;
    h->snap_done = done;
  }
  double *d = h->snap_dev;
  HE4_CUDA_TRY(cudaMemcpyAsync(d, h->psi, sizeof(double2) * h->N, cudaMemcpyDeviceToDevice, h->stream));
  d += 2 * h->N;
  const double *parts[3] = {h->rimp, h->vimp, h->aimp};
  for (int a = 0; a < 3; a++)
    HE4_CUDA_TRY(cudaMemcpyAsync(d + a * P3, parts[a], sizeof(double) * P3, cudaMemcpyDeviceToDevice, h->stream));
  HE4_CUDA_TRY(cudaEventRecord(h->snap_taken, h->stream));
  HE4_CUDA_TRY(cudaStreamWaitEvent(h->snap_stream, h->snap_taken, 0));
  HE4_CUDA_TRY(cudaMemcpyAsync(h->snap_host, h->snap_dev, sizeof(double) * n, cudaMemcpyDeviceToHost, h->snap_stream));
  HE4_CUDA_TRY(cudaEventRecord(h->snap_done, h->snap_stream));
  h->snap_pending = 1;
  return HE4_OK;
}

int he4_snapshot_wait(he4_handle *hh, const double **psi, const double **rimp, const double **vimp,
                      const double **aimp) {
  HANDLE_OR_FAIL(hh);
  if (!h->snap_pending) {
    set_error("he4_snapshot_wait without a snapshot in flight");
    return HE4_E_STATE;
  }
  HE4_CUDA_TRY(cudaEventSynchronize(h->snap_done));
  h->snap_pending = 0;
  const size_t P3 = 3 * (size_t)h->npar;
  const double *b = h->snap_host;
  if (psi) *psi = b;
  b += 2 * h->N;
  if (rimp) *rimp = b;
  if (vimp) *vimp = b + P3;
  if (aimp) *aimp = b + 2 * P3;
  return HE4_OK;
}

}  // extern "C"

namespace he4 {
int check_kernel_errors(Handle *h) {
  unsigned *herr = reinterpret_cast<unsigned *>(h->hscal + 60);
  HE4_CUDA_TRY(cudaMemcpyAsync(herr, &h->gred->err, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (*herr) {
    const unsigned e = *herr;
    *herr = 0;
    HE4_CUDA_TRY(cudaMemsetAsync(&h->gred->err, 0, sizeof(unsigned), h->stream));
    HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
    set_error("a streamed stencil's bulk copies did not arrive within one second (device error word 0x%x)", e);
    return HE4_E_CUDA;
  }
  return HE4_OK;
}
}  // namespace he4

extern "C" {

static int sync_and_check(Handle *h) {
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return check_kernel_errors(h);
}

int he4_potenimp(he4_handle *hh) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  h->field_valid = 0;
  HE4_TRY(field_potenimp(h, true));
  h->split_valid = 0;
  return sync_and_check(h);
}

int he4_poten(he4_handle *hh) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  h->field_valid = 0;
  HE4_TRY(field_poten(h, true, h->pot4));
  h->split_valid = 1;
  return sync_and_check(h);
}

int he4_forceimp(he4_handle *hh) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  HE4_TRY(field_forceimp(h, true));
  h->field_valid = 1;  // potenimp, poten, forceimp: the reference's sequence
  return sync_and_check(h);
}

int he4_field(he4_handle *hh) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  HE4_TRY(field_all(h, true));
  return sync_and_check(h);
}

static int finite_all(const double *v, int n) {
  for (int i = 0; i < n; i++)
    if (!isfinite(v[i])) return 0;
  return 1;
}

int he4_step_rk(he4_handle *hh, double deltat, double means[9]) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  if (!isfinite(deltat)) {
    set_error("deltat is not finite");
    return HE4_E_ARG;
  }
  HE4_TRY(step_rk(h, deltat, h->scal));
  HE4_CUDA_TRY(cudaMemcpyAsync(h->hscal, h->scal, 12 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  HE4_TRY(check_kernel_errors(h));
  if (means) memcpy(means, h->hscal + 3, 9 * sizeof(double));
  if (!finite_all(h->hscal, 12)) {
    set_error("non-finite trajectory means after steprk");
    return HE4_E_NONFINITE;
  }
  return HE4_OK;
}

int he4_step_pc(he4_handle *hh, double deltat, double err[3], double means[9]) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  if (!isfinite(deltat)) {
    set_error("deltat is not finite");
    return HE4_E_ARG;
  }
  // the step's captured graph (replayed, or captured on first use) where
  // graphs are on, as he4_run does
  if (h->use_graphs && h->nsteps_done >= 3)
    HE4_TRY(run_pc_graphs(h, 1, deltat, h->scal));
  else
    HE4_TRY(step_pc(h, deltat, h->scal));
  HE4_CUDA_TRY(cudaMemcpyAsync(h->hscal, h->scal, 12 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  HE4_TRY(check_kernel_errors(h));
  if (err) memcpy(err, h->hscal, 3 * sizeof(double));
  if (means) memcpy(means, h->hscal + 3, 9 * sizeof(double));
  if (!finite_all(h->hscal, 12)) {
    set_error("non-finite errHe/errimp/errvimp or means after steppc");
    return HE4_E_NONFINITE;
  }
  return HE4_OK;
}

int he4_run(he4_handle *hh, int32_t nsteps, double deltat, double *err, double *means) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  if (nsteps < 0 || !isfinite(deltat)) {
    set_error("invalid nsteps or deltat");
    return HE4_E_ARG;
  }
  if (nsteps == 0) return HE4_OK;
  double *dres = nullptr;
  HE4_CUDA_TRY(cudaMallocAsync((void **)&dres, sizeof(double) * 12 * nsteps, h->stream));
  int e = HE4_OK;
  int s = 0;
  for (; s < nsteps && e == HE4_OK && h->nsteps_done < 3; s++) e = step_rk(h, deltat, dres + 12 * s);
  if (e == HE4_OK && s < nsteps) {
    if (h->use_graphs) {
      e = run_pc_graphs(h, nsteps - s, deltat, dres + 12 * s);
    } else {
      for (; s < nsteps && e == HE4_OK; s++) e = step_pc(h, deltat, dres + 12 * s);
    }
  }
  double *hres = nullptr;
  if (e == HE4_OK) {
    hres = (double *)malloc(sizeof(double) * 12 * nsteps);
    cudaError_t ce = cudaMemcpyAsync(hres, dres, sizeof(double) * 12 * nsteps, cudaMemcpyDeviceToHost, h->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) {
      set_error("he4_run copy-out: %s", cudaGetErrorString(ce));
      e = HE4_E_CUDA;
    }
  }
  cudaFreeAsync(dres, h->stream);
  if (e == HE4_OK) e = check_kernel_errors(h);
  if (e == HE4_OK) {
    for (int s = 0; s < nsteps; s++) {
      if (err) memcpy(err + 3 * s, hres + 12 * s, 3 * sizeof(double));
      if (means) memcpy(means + 9 * s, hres + 12 * s + 3, 9 * sizeof(double));
    }
    if (!finite_all(hres, 12 * nsteps)) {
      set_error("non-finite errors or means during he4_run");
      e = HE4_E_NONFINITE;
    }
  }
  free(hres);
  return e;
}

int he4_energy(he4_handle *hh, he4_energies *e) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  if (!e) {
    set_error("null energies");
    return HE4_E_ARG;
  }
  if (!h->field_valid) HE4_TRY(field_all(h, true));  // energy() follows a field evaluation
  if (!h->split_valid) HE4_TRY(field_split_fields(h));  // delj4, uimp of this state
  HE4_TRY(compute_energy(h, e));
  const double *v = &e->etot;
  if (!finite_all(v, 11)) {
    set_error("non-finite energy");
    return HE4_E_NONFINITE;
  }
  return HE4_OK;
}

int he4_diagnostics(he4_handle *hh, int32_t n4, double out[4]) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  if (!out || n4 <= 0) {
    set_error("he4_diagnostics needs an output array and n4 > 0");
    return HE4_E_ARG;
  }
  return compute_diagnostics(h, n4, out);
}

int he4_bubble_radius(he4_handle *hh, int32_t nr, double *rb, int32_t found[2], int32_t *ir, double xms[3],
                      double *rr, double *denr) {
  HANDLE_OR_FAIL(hh);
  NEED_STATE(h);
  if (!rb || !found) {
    set_error("he4_bubble_radius needs rb and found");
    return HE4_E_ARG;
  }
  BubbleResult res;
  HE4_TRY(compute_bubble_radius(h, nr, &res, rr, denr));
  *rb = res.rb;
  found[0] = res.found[0];
  found[1] = res.found[1];
  if (ir) *ir = res.ir;
  if (xms)
    for (int c = 0; c < 3; c++) xms[c] = res.xms[c];
  return HE4_OK;
}

int he4_get_field(he4_handle *hh, int32_t which, double *out) {
  HANDLE_OR_FAIL(hh);
  if (!out) {
    set_error("null output");
    return HE4_E_ARG;
  }
  const double *src = nullptr;
  // fields a merged (time-step) evaluation leaves unwritten
  if (h->field_valid && !h->split_valid &&
      (which == HE4_F_UIMP || which == HE4_F_DELJ4 || which == HE4_F_UALPHAS || which == HE4_F_PENALTY ||
       which == HE4_F_CORR || which == HE4_F_FALFS ||
       (h->real32 && (which == HE4_F_DENCG || which == HE4_F_DENALF || which == HE4_F_DXDEN ||
                      which == HE4_F_DYDEN || which == HE4_F_DZDEN || which == HE4_F_INTXALF ||
                      which == HE4_F_INTYALF || which == HE4_F_INTZALF))))
    HE4_TRY(field_split_fields(h));
  switch (which) {
    case HE4_F_DEN: src = h->den; break;
    case HE4_F_POT4: src = h->pot4; break;
    case HE4_F_DENX: src = h->denx; break;
    case HE4_F_PSIX: src = h->psix; break;
    case HE4_F_HPSIX: src = h->hpsix; break;
    case HE4_F_UIMP: src = h->uimp; break;
    case HE4_F_DENCG: src = h->dencg; break;
    case HE4_F_DELJ4: src = h->delj4; break;
    case HE4_F_DENALF: src = h->denalf; break;
    case HE4_F_UALPHAS: src = h->ualphas; break;
    case HE4_F_FALFS: src = h->falfs; break;
    case HE4_F_INTXALF: src = h->intx; break;
    case HE4_F_INTYALF: src = h->inty; break;
    case HE4_F_INTZALF: src = h->intz; break;
    case HE4_F_DXDEN: src = h->dxden; break;
    case HE4_F_DYDEN: src = h->dyden; break;
    case HE4_F_DZDEN: src = h->dzden; break;
    case HE4_F_FX:
    case HE4_F_FY:
    case HE4_F_FZ:
      // a time step computes the force field only where the particles read
      // it; complete it from the density spectrum of the same evaluation
      if (h->field_valid && !h->forces_full) HE4_TRY(field_forces(h, true));
      src = (which == HE4_F_FX) ? h->fx : (which == HE4_F_FY) ? h->fy : h->fz;
      break;
    case HE4_F_PENALTY: src = h->penalty; break;
    case HE4_F_CORR: src = h->corr; break;
    default:
      set_error("unknown field id %d", which);
      return HE4_E_ARG;
  }
  HE4_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * h->N, cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

int he4_get_kernel(he4_handle *hh, int32_t which, double *out) {
  HANDLE_OR_FAIL(hh);
  if (!out) {
    set_error("null output");
    return HE4_E_ARG;
  }
  const double *src = nullptr;
  switch (which) {
    case HE4_K_WCGK: src = h->wcgk; break;
    case HE4_K_FVLJ4: src = h->fvlj4; break;
    case HE4_K_KALFS: src = h->kalfs; break;
    case HE4_K_VQ: src = h->vq; break;
    case HE4_K_PMOD: src = h->pmod; break;
    default:
      set_error("unknown kernel id %d", which);
      return HE4_E_ARG;
  }
  HE4_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * h->H, cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

int he4_fft_r2c(he4_handle *hh, const double *in, double *out) {
  HANDLE_OR_FAIL(hh);
  if (!in || !out) {
    set_error("null buffer");
    return HE4_E_ARG;
  }
  HE4_CUDA_TRY(cudaMemcpyAsync(h->rtmp[0], in, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->stream));
  const double *src[1] = {h->rtmp[0]};
  double2 *dst[1] = {h->spec[1]};
  HE4_TRY(fft_r2c(h, 1, src, dst));
  HE4_TRY(fft_z_only(h, dst[0], false));
  if (h->fp32) {  // FP32 half spectrum -> FP64 for the caller
    HE4_TRY(widen(h, reinterpret_cast<const float *>(h->spec[1]), reinterpret_cast<double *>(h->spec[2]), 2 * h->H));
    dst[0] = h->spec[2];
  }
  HE4_CUDA_TRY(cudaMemcpyAsync(out, dst[0], sizeof(double2) * h->H, cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

int he4_fft_c2r(he4_handle *hh, const double *in, double *out) {
  HANDLE_OR_FAIL(hh);
  if (!in || !out) {
    set_error("null buffer");
    return HE4_E_ARG;
  }
  double2 *buf = h->spec[1];
  if (h->fp32) {  // the caller's FP64 half spectrum, rounded to FP32
    HE4_CUDA_TRY(cudaMemcpyAsync(h->spec[2], in, sizeof(double2) * h->H, cudaMemcpyHostToDevice, h->stream));
    HE4_TRY(narrow(h, reinterpret_cast<const double *>(h->spec[2]), reinterpret_cast<float *>(buf), 2 * h->H));
  } else {
    HE4_CUDA_TRY(cudaMemcpyAsync(buf, in, sizeof(double2) * h->H, cudaMemcpyHostToDevice, h->stream));
  }
  HE4_TRY(fft_z_only(h, buf, true));
  double2 *src[1] = {buf};
  double *dst[1] = {h->rtmp[0]};
  HE4_TRY(fft_c2r(h, 1, src, dst));
  HE4_CUDA_TRY(cudaMemcpyAsync(out, h->rtmp[0], sizeof(double) * h->N, cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

constexpr int kBenchKernels = 13;

static int launch_bench(Handle *h, int which) {
  switch (which) {
    case 0: {
      ZOp op{h->spec[0], h->spec[1], h->wcgk, h->renor, -1};
      return fft_z_conv(h, 1, &op);
    }
    case 1: {
      double2 *b[1] = {h->spec[1]};
      return fft_y(h, 1, b, false);
    }
    case 2: return fft_x_only(h, h->rtmp[0], h->spec[1], nullptr, nullptr, false);
    case 3: return fft_x_only(h, nullptr, nullptr, h->spec[1], h->rtmp[0], true);
    case 4: return fft_z_only(h, h->spec[1], false);
    case 5: {
      ZOp op{h->spec[0], h->spec[1], nullptr, h->renor, -1};
      return fft_z_conv(h, 1, &op);
    }
    case 6: {
      ZOp ops[3] = {{h->spec[0], h->spec[1], h->wcgk, h->renor, -1},
                    {h->spec[0], h->spec[2], h->fvlj4, h->renor, -1},
                    {h->spec[0], h->spec[3], h->kalfs, h->renor, -1}};
      return fft_z_conv(h, 3, ops);
    }
    case 7: return launch_grad(h);
    case 8: return launch_pot4_merged(h);
    case 9: return launch_pot4_merged_f32(h);
    case 10: return fft_x_c2r_f32_only(h, h->spec[1], h->g32[8]);
    case 11: return launch_grad_f32(h);
    case 12: {
      double2 *b[1] = {h->spec[1]};
      return fft_y(h, 1, b, true);
    }
    default: set_error("unknown kernel id %d", which); return HE4_E_ARG;
  }
}

int he4_bench_kernel(he4_handle *hh, int32_t which, int32_t reps, double *ms_per_launch, double *bytes_per_launch,
                     char *name, int32_t name_len) {
  HANDLE_OR_FAIL(hh);
  if (reps < 1 || !ms_per_launch || !bytes_per_launch) {
    set_error("invalid arguments");
    return HE4_E_ARG;
  }
  // kernel families the ids launch (the template arguments follow the grid
  // and the form; ncu's launch lists name them in full)
  static const char *names[kBenchKernels] = {
      "k_zconv (z conv, 1 output)", "k_yz_pipe (y pass)",           "k_xr2c_reg (x R2C)",
      "k_xc2r_reg (x C2R)",         "k_zconv (z pass, no multiply)", "k_zconv (z conv, no kernel)",
      "k_zconv (z conv, 3 outputs)", "k_grad_z (density gradient)",  "k_pot4_merged_z (pot4, FP64 grids)",
      "k_pot4_merged_z (pot4, float grids)", "k_xc2r_reg (x C2R, float rows)",
      "k_grad_z (density gradient, float grids)", "k_yz_pipe (y pass, inverse)"};
  const double H = (double)h->H, N = (double)h->N;
  // algorithmic bytes: read input once, write output once (+ the real
  // kernel); c and k are the sizes of a spectrum and a kernel element
  const double c = h->fp32 ? 8 : 16, k = h->fp32 ? 4 : 8;
  const double bytes[kBenchKernels] = {
      c * H + k * H + c * H, 2 * c * H, 8 * N + c * H, c * H + 8 * N, 2 * c * H, 2 * c * H,
      c * H + 3 * (k * H + c * H),
      // stencils: den in, three gradients out; lin, den, dencg, h0..h2 in, pot4 out
      4 * 8 * N, 7 * 8 * N,
      // float grids: lin, dencg, h0..h2 (4 B), den in and pot4 out (8 B)
      5 * 4 * N + 2 * 8 * N,
      // half spectrum in, float rows out
      c * H + 4 * N,
      // den in, three float gradients out
      8 * N + 3 * 4 * N,
      // inverse y pass, in place
      2 * c * H};
  if (which < 0 || which >= kBenchKernels) {
    set_error("unknown kernel id %d", which);
    return HE4_E_ARG;
  }
  if ((which == 9 || which == 10 || which == 11) && !h->real32) {
    set_error("kernel id %d needs the FP32-convolution form with float grids", which);
    return HE4_E_STATE;
  }
  HE4_TRY(launch_bench(h, which));  // warm-up
  cudaEvent_t e0, e1;
  HE4_CUDA_TRY(cudaEventCreate(&e0));
  HE4_CUDA_TRY(cudaEventCreate(&e1));
  HE4_CUDA_TRY(cudaEventRecord(e0, h->stream));
  int rc = HE4_OK;
  for (int i = 0; i < reps && rc == HE4_OK; i++) rc = launch_bench(h, which);
  HE4_CUDA_TRY(cudaEventRecord(e1, h->stream));
  HE4_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  HE4_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HE4_TRY(rc);
  // the timed launches overwrite evaluation buffers: the next step
  // evaluates the field of its state again
  h->field_valid = 0;
  h->split_valid = 0;
  *ms_per_launch = ms / reps;
  *bytes_per_launch = bytes[which];
  if (name && name_len > 0) {
    strncpy(name, names[which], name_len - 1);
    name[name_len - 1] = 0;
  }
  return HE4_OK;
}

int he4_device_ptr(he4_handle *hh, int32_t which, void **ptr) {
  HANDLE_OR_FAIL(hh);
  if (!ptr) {
    set_error("null output");
    return HE4_E_ARG;
  }
  switch (which) {
    case HE4_D_PSI: *ptr = h->psi; break;
    case HE4_D_RIMP: *ptr = h->rimp; break;
    case HE4_D_VIMP: *ptr = h->vimp; break;
    case HE4_D_DEN: *ptr = h->den; break;
    case HE4_D_DENX: *ptr = h->denx; break;
    default:
      set_error("unknown device array id %d", which);
      return HE4_E_ARG;
  }
  return HE4_OK;
}

int he4_get_stream(he4_handle *hh, void **stream) {
  HANDLE_OR_FAIL(hh);
  if (!stream) return HE4_E_ARG;
  *stream = (void *)h->stream;
  return HE4_OK;
}

int64_t he4_launch_count(he4_handle *hh) { return hh ? hh->h.launches : -1; }

int he4_graph_stats(he4_handle *hh, int64_t *captured, int64_t *uncaptured) {
  HANDLE_OR_FAIL(hh);
  if (captured) *captured = h->graph_captures;
  if (uncaptured) *uncaptured = h->steps_uncaptured;
  return HE4_OK;
}

const char *he4_strerror(int code) {
  switch (code) {
    case HE4_OK: return "ok";
    case HE4_E_ARG: return "invalid argument";
    case HE4_E_UNSUPPORTED: return "unsupported configuration";
    case HE4_E_NOMEM: return "out of memory";
    case HE4_E_CUDA: return "CUDA error";
    case HE4_E_STATE: return "invalid call order";
    case HE4_E_NONFINITE: return "non-finite result";
    case HE4_E_NODEVICE: return "no sm_100 device";
    default: return "unknown error";
  }
}

const char *he4_last_error(void) { return g_err; }

}  // extern "C"

// common.cuh -- shared declarations of the B200 time-step library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../../include/he4_tddft.h"

namespace he4 {

// ---------------------------------------------------------------------------
// error handling: every failing call records a message and returns a code.
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);

#define HE4_CUDA_TRY(expr)                                                      \
  do {                                                                          \
    cudaError_t e_ = (expr);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ::he4::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,               \
                       cudaGetErrorString(e_));                                 \
      return HE4_E_CUDA;                                                        \
    }                                                                           \
  } while (0)

#define HE4_TRY(expr)            \
  do {                           \
    int r_ = (expr);             \
    if (r_ != HE4_OK) return r_; \
  } while (0)

// after a kernel launch: record launch and check the launch error
#define HE4_LAUNCHED(h)                                                          \
  do {                                                                           \
    (h)->launches++;                                                             \
    cudaError_t e_ = cudaGetLastError();                                         \
    if (e_ != cudaSuccess) {                                                     \
      ::he4::set_error("%s:%d kernel launch: %s", __FILE__, __LINE__,            \
                       cudaGetErrorString(e_));                                  \
      return HE4_E_CUDA;                                                         \
    }                                                                            \
  } while (0)

// ---------------------------------------------------------------------------
// complex FP64 helpers
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__host__ __device__ __forceinline__ double2 cmuli(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// Per-device host caches (launch attributes, occupancy, scratch addresses)
// are arrays over the device ordinal; he4_create refuses ordinals past it.
constexpr int kMaxDevices = 64;

// ---------------------------------------------------------------------------
// FFT plan
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 12;
struct AxisPlan {
  int n = 0;
  int nst = 0;
  int radix[kMaxStages] = {0};
  double2 *tw = nullptr;   // device: exp(-2 pi i t / n), t in [0, n)
  float2 *tw32 = nullptr;  // the same, rounded to FP32 (FP32-convolution form)
};

struct FftPlan {
  int nx = 0, ny = 0, nz = 0, nxh = 0;
  AxisPlan ax, ay, az;
  int wy = 8, wz = 8;   // pencils per CTA in the y and z passes (generic path)
  int px = 8;           // complex pencils (= row pairs) per CTA in the x pass (generic path)
  int n1[3] = {0, 0, 0};  // four-step split N = N1 * N2 per axis (register path)
};

int fft_plan_init(FftPlan &P, int nx, int ny, int nz);
void fft_plan_free(FftPlan &P);
// tile shapes t = {n1x, n1y, n1z, px, wy, wz} (fft.cu)
int fft_set_tiles(FftPlan &P, const int *t);
void fft_get_tiles(const FftPlan &P, int *t);

// ---------------------------------------------------------------------------
// stencil weights (centre row of the Bickley matrix, times 1/h^order)
// ---------------------------------------------------------------------------
struct Stencil {
  int m = 3;                 // half width, npd = 2m+1
  double w1[3][25];          // first derivative, per axis
  double w2[3][25];          // second derivative, per axis
  // icon=12: device table [order-1][axis][c < m][2m+1] of the one-sided
  // Bickley rows of the first m points, times 1/h^order (null otherwise)
  const double *lo = nullptr;
};
int fd_weights(int npd, int order, double *w);
int fd_rows(int npd, int order, double *rows);

struct ZOp;  // z-pass operation (fft.cu)

// support box of the impurity fields (impurity.cu): inclusive cell ranges
struct Box {
  int lo[3], hi[3];
  int full;   // the whole grid (the box would wrap or reach a face)
  int empty;  // no particle inside the grid
};
struct BoxPair {
  Box cur, prev;
};

// Particle kernels run on up to kPartMaxCta CTAs of kPartThreads threads
// (a fixed cap, not the SM count, so their reductions give the same bits
// on every device).  Their grid-wide reductions keep per-CTA partials and
// a last-CTA counter here; box holds the running NGP min/max of k_box_find.
constexpr int kPartThreads = 256;
constexpr int kPartMaxCta = 296;
struct GridRed {
  double part[9 * kPartMaxCta];
  unsigned count[4];  // 0: box, 1: corrector errors, 2: means
  int box[6];         // min x, y, z, max x, y, z; reset by the last CTA
  unsigned err;       // bit 0: a streamed stencil's copies did not arrive
};

// ---------------------------------------------------------------------------
// host-side step state: which buffer holds which history level, the ring
// indices of steppc and the time step.  A captured PC step is valid for the
// state it started from and leaves the state it was captured to.
// ---------------------------------------------------------------------------
struct StepState {
  double2 *psi, *psiold[3], *hpsiold[2], *ctmp;
  double *rimpold[3], *vimpold[3], *aimpold[2];
  int ioldp[3], ioldh[2], ioldr[3], ioldv[3], iolda[2];
  double dt;
};
// member by member (a byte comparison would also compare the padding after
// iolda, which struct copies need not preserve: a state would then miss its
// captured graph and be captured again, or run uncaptured)
inline bool same_step_state(const StepState &a, const StepState &b) {
  if (a.psi != b.psi || a.ctmp != b.ctmp || a.dt != b.dt) return false;
  for (int i = 0; i < 3; i++)
    if (a.psiold[i] != b.psiold[i] || a.rimpold[i] != b.rimpold[i] || a.vimpold[i] != b.vimpold[i] ||
        a.ioldp[i] != b.ioldp[i] || a.ioldr[i] != b.ioldr[i] || a.ioldv[i] != b.ioldv[i])
      return false;
  for (int i = 0; i < 2; i++)
    if (a.hpsiold[i] != b.hpsiold[i] || a.aimpold[i] != b.aimpold[i] || a.ioldh[i] != b.ioldh[i] ||
        a.iolda[i] != b.iolda[i])
      return false;
  return true;
}

struct StepGraph {
  StepState before, after;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;
};

// ---------------------------------------------------------------------------
// the handle
// ---------------------------------------------------------------------------
struct Handle {
  he4_params p{};
  int nx = 0, ny = 0, nz = 0, nxh = 0, npar = 0;
  size_t N = 0, H = 0;
  double hx = 0, hy = 0, hz = 0, dxyz = 0, renor = 0, mAg_u = 0, h2o2mx = 0;
  int dev = 0;
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
  FftPlan fft;
  Stencil st;

  // FP32-convolution form: spectra hold float2, the k-space multiply uses
  // FP32 copies of the kernels and of the derivative symbol
  int fp32 = 0;
  float *k32[4] = {nullptr, nullptr, nullptr, nullptr};  // wcgk, fvlj4, kalfs, vq
  // FP32-convolution form with z-marching stencils: the merged evaluation
  // keeps its intermediate real grids in float (dencg, denalf, the three
  // density gradients, the three alpha_s integrals / products, s and lin)
  int real32 = 0;
  float *g32[9] = {nullptr};
  float *dsym32 = nullptr;
  // FP32 twin of one of the FP64 kernel arrays (nullptr for nullptr)
  const float *kern32(const double *k) const {
    if (!k) return nullptr;
    if (k == wcgk) return k32[0];
    if (k == fvlj4) return k32[1];
    if (k == kalfs) return k32[2];
    if (k == vq) return k32[3];
    return nullptr;
  }

  // k-space kernels [H] and derivative symbols
  double *wcgk = nullptr, *fvlj4 = nullptr, *kalfs = nullptr, *vq = nullptr, *pmod = nullptr;
  double *dsym = nullptr;     // [nx+ny+nz]: imaginary part of the periodic first-derivative symbol
  double *timec_re = nullptr; // [nz]

  // He fields
  double2 *psi = nullptr, *psiold[3] = {nullptr, nullptr, nullptr}, *hpsiold[2] = {nullptr, nullptr};
  double2 *pc = nullptr, *q = nullptr, *ctmp = nullptr;
  double *den = nullptr, *pot4 = nullptr, *dencg = nullptr, *delj4 = nullptr, *denalf = nullptr;
  double *ualphas = nullptr, *falfs = nullptr, *intx = nullptr, *inty = nullptr, *intz = nullptr;
  double *dxden = nullptr, *dyden = nullptr, *dzden = nullptr, *penalty = nullptr, *corr = nullptr;
  double *denx = nullptr, *psix = nullptr, *hpsix = nullptr, *uimp = nullptr;
  double *fx = nullptr, *fy = nullptr, *fz = nullptr;
  double *rtmp[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned int *counts = nullptr;
  BoxPair *box = nullptr;  // device: support of denx/psix/hpsix
  // spectra work buffers [H] complex
  double2 *spec[8] = {nullptr};

  // particles [3][npar]
  double *rimp = nullptr, *vimp = nullptr, *aimp = nullptr;
  double *rimpold[3] = {nullptr}, *vimpold[3] = {nullptr}, *aimpold[2] = {nullptr};
  double *qr = nullptr, *qv = nullptr, *pcr = nullptr, *pcv = nullptr;
  int ioldp[3] = {0, 1, 2}, ioldh[2] = {0, 1}, ioldr[3] = {0, 1, 2}, ioldv[3] = {0, 1, 2}, iolda[2] = {0, 1};
  // the buffers as allocated: he4_set_state puts every rotating pointer
  // back here, so each run from a new state walks the same 30 step states
  // (and reuses their captured graphs)
  double2 *home_c[7] = {nullptr};   // psi, ctmp, psiold[0..2], hpsiold[0..1]
  double *home_p[8] = {nullptr};    // rimpold[0..2], vimpold[0..2], aimpold[0..1]

  // reductions
  GridRed *gred = nullptr;    // particle-kernel partials, counters, box scratch
  double *st_lo = nullptr;    // icon=12 boundary rows (Stencil::lo)
  double *red = nullptr;      // partial sums workspace
  double *scal = nullptr;     // device scalars (errors, energies, means)
  double *hscal = nullptr;    // pinned host mirror of scal
  // checkpoint snapshot (he4_snapshot_begin / he4_snapshot_wait): device
  // copy of psi, rimp, vimp, aimp, its pinned host mirror, the copy stream
  double *snap_dev = nullptr;
  double *snap_host = nullptr;
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
  int snap_pending = 0;
  // radial histogram of the spherical bubble radius (grown on demand)
  unsigned long long *bub = nullptr;
  size_t bub_len = 0;

  int have_state = 0;
  int nsteps_done = 0;
  // pot4, aimp and the other fields belong to the current psi and rimp
  // (the field evaluation that DFT4He3d.f90:630-634 does before the loop)
  int field_valid = 0;
  // fx, fy, fz hold the whole grid (otherwise only the force box)
  int forces_full = 0;
  // uimp, delj4, corr, ualphas and penalty belong to the current evaluation
  // (a merged evaluation does not write them)
  int split_valid = 0;
  size_t red_len = 0;
  // captured PC steps (one per distinct StepState; the states repeat)
  std::vector<StepGraph> graphs;
  int use_graphs = 1;
  int64_t graph_captures = 0, steps_uncaptured = 0;  // he4_graph_stats
  // row-streamed (bulk-copy pipelined) stencils where the grid allows them
  int use_stream = 1;
  // FP32-form pot4 stencil: pointwise assembly in FP32 with split weights
  int pot4_split = 1;
  // force z convolution: one inverse transform for the x and y outputs
  int zconv_share_xy = 1;
};

// kernel-level entry points used by the ABI layer
int fft_r2c(Handle *h, int n, const double *const *in, double2 *const *out);
// x pass R2C whose input rows are formed on load from other grids:
//   XLOAD_ALFA: in_f * (1 - aux0 * c0)     (falfs * d_f rho, term_alfa.f90:28-36)
//   XLOAD_CORR: aux0 * aux1 * (c0 + c1 * aux1)  (poten.f90:62-64; `in` unused)
// With real32 the rows `in` and the grids formed from (aux0 of ALFA, aux1 of
// CORR) are float; aux0 of CORR (den) is always double.
enum { XLOAD_PLAIN = 0, XLOAD_ALFA = 1, XLOAD_CORR = 2 };
struct XLoad {
  int op = XLOAD_PLAIN;
  int real32 = 0;
  const void *aux0 = nullptr, *aux1 = nullptr;
  double c0 = 0.0, c1 = 0.0;
};
int fft_r2c_load(Handle *h, int n, const void *const *in, double2 *const *out, const XLoad &ld);
// inverse transform into float real grids (FP32-convolution form)
int fft_c2r_f32(Handle *h, int n, double2 *const *in, float *const *out);
int fft_c2r(Handle *h, int n, double2 *const *in, double *const *out);
int fft_y(Handle *h, int n, double2 *const *buf, bool inverse);
// z pass: for each op, out = IFFT_z(coef * K * FFT_z(in)); K may be null (=1)
// or the derivative symbol of an axis (kind 1..3).
struct ZOp {
  const double2 *in;
  double2 *out;
  const double *kern;
  double coef;
  int dsym_axis;  // -1 none, 0/1/2: multiply by i*dsym[axis](k)
  int mode = 0;   // 0: FFT_z, multiply, IFFT_z; 1: FFT_z only; 2: IFFT_z only
  int boxz = 0;   // store only the z planes of the force box (see force_range)
};
int fft_z_conv(Handle *h, int n, const ZOp *ops);
// z pass of a sum of convolutions: out = IFFT_z(sum_j coef_j K_j FFT_z(in_j))
// (register-path z lengths only; at most 4 terms)
struct ZTerm {
  const double2 *in;
  const double *kern;
  double coef;
};
int fft_z_sum(Handle *h, int nterm, const ZTerm *terms, double2 *out);
bool fft_z_sum_ok(const Handle *h);
// inverse y and x passes restricted to the pencils and rows of the force box
int fft_c2r_box(Handle *h, int n, double2 *const *in, double *const *out);

// The cells where the force field is needed: the impurity box widened by one
// cell (the trilinear gather reads cells floor(a) and floor(a)+1 around the
// NGP cell).  Whole axis when the box is full; lo > hi when it is empty.
__device__ __forceinline__ void force_range(const BoxPair *bp, int axis, int n, int *lo, int *hi) {
  const Box b = bp->cur;
  if (b.full) {
    *lo = 0;
    *hi = n - 1;
  } else if (b.empty) {
    *lo = 1;
    *hi = 0;
  } else {
    *lo = max(0, b.lo[axis] - 1);
    *hi = min(n - 1, b.hi[axis] + 1);
  }
}
// plain transform along z of one half spectrum, in place
int fft_z_only(Handle *h, double2 *buf, bool inverse);
// x pass alone (R2C: rin -> cout; C2R: cin -> rout)
int fft_x_only(Handle *h, const double *rin, double2 *cout, const double2 *cin, double *rout, bool inverse);
int fft_x_c2r_f32_only(Handle *h, const double2 *cin, float *rout);

int setup_kernels(Handle *h);
// element-wise FP64 <-> FP32 conversion of n reals on the handle's stream
int narrow(Handle *h, const double *in, float *out, size_t n);
int widen(Handle *h, const float *in, double *out, size_t n);

// split: also write the named intermediate fields (uimp; delj4, corr,
// ualphas, penalty) the way the reference's routines do; otherwise (the time
// step path) the linear convolutions entering pot4 share one inverse FFT.
// pot4: where the split poten writes its pot4.
int field_potenimp(Handle *h, bool split);
int field_poten(Handle *h, bool split, double *pot4);
// full: the force field on the whole grid; otherwise only where the gather
// reads it (a time step's need).  field_forces recomputes just the field.
int field_forceimp(Handle *h, bool full);
int field_forces(Handle *h, bool full);
// the stencil passes of an evaluation (also timed by he4_bench_kernel)
int launch_grad(Handle *h);
// the merged evaluation may keep float intermediate grids (Handle::real32)
bool real32_ok(const Handle *h);
int launch_pot4_merged(Handle *h);
int launch_pot4_merged_f32(Handle *h);
int launch_grad_f32(Handle *h);
// device error word of the step's kernels (GridRed::err): HE4_E_CUDA with a
// message when set, after which it is cleared; synchronises the stream
int check_kernel_errors(Handle *h);
// potenimp + poten + forceimp; marks the fields valid.  split = false takes
// the merged form when the z length allows it.
int field_all(Handle *h, bool split = false);
// after a merged evaluation: compute the named intermediate fields of the
// same state without touching pot4
int field_split_fields(Handle *h);
// impurity.cu: denx, psix, hpsix on the particle box; quantum force term;
// reset of the box to the whole grid
int impurity_density(Handle *h);
int impurity_force_q(Handle *h);
int impurity_reset_box(Handle *h);

// dres: device array of 12 doubles: errHe, errimp, errvimp, then the 9 means
int step_rk(Handle *h, double dt, double *dres);
int step_pc(Handle *h, double dt, double *dres);
// n PC steps from captured graphs (capturing the states not seen yet);
// results of step s land in dres[12 s .. 12 s + 11]
int run_pc_graphs(Handle *h, int n, double dt, double *dres);
void free_graphs(Handle *h);
StepState get_step_state(const Handle *h, double dt);
void set_step_state(Handle *h, const StepState &s);
int compute_energy(Handle *h, he4_energies *e);
int compute_diagnostics(Handle *h, int n4, double *host_out);
// spherical bubble radius around the mean impurity position; rr / denr may
// be null, otherwise they receive nr values
struct BubbleResult {
  double rb = 0.0;
  double xms[3] = {0.0, 0.0, 0.0};
  int found[2] = {0, 0};
  int ir = 0;
};
int compute_bubble_radius(Handle *h, int nr, BubbleResult *res, double *rr, double *denr);
int spline_global(const double *x, const double *y, double *A, double *B, double *C, double *D, double s1,
                  double sn, int n);
int compute_den(Handle *h);
int particle_means(Handle *h, double *means);

}  // namespace he4

struct he4_handle {
  he4::Handle h;
};

/* he4_fno.h -- C ABI of the Fourier-neural-operator coarse propagator used
 * by the parareal driver of the B200 time-step library.
 *
 * The reference has no learned component; this is an addition to it: a
 * small FNO (lifting, L Fourier layers, two-layer projection) on a cubic
 * grid of n^3 points, trained on trajectories produced by the solver itself
 * and used as the coarse step of a parareal scheme whose fine propagator is
 * the plain predictor-corrector integrator (he4_run).
 *
 * Every function launches on the given CUDA stream (NULL = legacy default
 * stream) and takes DEVICE pointers.  Activations, spectra and gradients are
 * FP32; the weights the forward and backward kernels read are BF16 (stored
 * as uint16_t bit patterns), every sum is accumulated in FP32.
 *
 * Layouts
 *   activations  [batch][channels][n^3]  (point index x fastest, then y, z)
 *   spectra      [batch][channels][mz][my][mx] complex (float2 pairs)
 *   contraction  y[o][k][r] = sum_j A[k][j] x[o][j][r]   (A complex, [K][J])
 *   spectral weights R[cin][cout][modes] complex BF16 pairs
 *   pointwise weights W[cout][cin] BF16, bias[cout] FP32
 * Return values: 0 or a negative HE4_E_* code (he4_tddft.h); the message is
 * in he4_last_error().
 */
#ifndef HE4_FNO_H
#define HE4_FNO_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = A x along one axis.  x is [outer][J][inner] (real if in_real, else
 * complex), y is [outer][K][inner] (the real part if out_real, else
 * complex); A is complex FP32 [K][J].  accumulate: y += instead of y =. */
int he4_fno_contract(const void *x, void *y, const float *A, int32_t outer, int32_t J, int32_t K, int32_t inner,
                     int32_t in_real, int32_t out_real, int32_t accumulate, void *stream);

/* spectral channel mixing: y[b][o][m] = sum_i x[b][i][m] R[i][o][m] */
int he4_fno_mix(const float *x, const uint16_t *R, float *y, int32_t batch, int32_t cin, int32_t cout,
                int32_t modes, void *stream);
/* its adjoints: gx[b][i][m] = sum_o gy[b][o][m] conj(R[i][o][m]);
 * gR[i][o][m] = sum_b conj(x[b][i][m]) gy[b][o][m] (FP32, overwritten).
 * gx may be the x buffer (gR is computed first); either output may be NULL. */
int he4_fno_mix_bwd(const float *gy, const float *x, const uint16_t *R, float *gx, float *gR, int32_t batch,
                    int32_t cin, int32_t cout, int32_t modes, void *stream);

/* pointwise layer: pre = W x + bias (+ add); y = act(pre), act 0 = identity,
 * 1 = GELU (erf form).  pre may be NULL (not stored), add may be NULL. */
int he4_fno_pointwise(const float *x, const uint16_t *W, const float *bias, const float *add, float *pre, float *y,
                      int32_t batch, int32_t cin, int32_t cout, int64_t npts, int32_t act, void *stream);
/* backward of he4_fno_pointwise.  gy is overwritten by gpre = gy act'(pre)
 * (the gradient of `add` as well); gx = W^T gpre (skipped when gx is NULL);
 * gW[cout][cin] and gbias[cout] are overwritten with sums over batch and
 * points (fixed-order reduction, run to run identical).  work: FP32 scratch
 * of he4_fno_pointwise_work() floats. */
int he4_fno_pointwise_bwd(float *gy, const float *pre, const float *x, const uint16_t *W, float *gx, float *gW,
                          float *gbias, float *work, int32_t batch, int32_t cin, int32_t cout, int64_t npts,
                          int32_t act, void *stream);
int64_t he4_fno_pointwise_work(int32_t batch, int32_t cin, int32_t cout, int64_t npts);

/* loss = sum (pred - target)^2 / sum target^2 over n values; grad (may be
 * NULL) = d loss / d pred.  out[0] = loss, out[1] = sum target^2 (device).
 * work: device scratch of HE4_FNO_LOSS_WORK doubles. */
#define HE4_FNO_LOSS_WORK 1024
int he4_fno_loss(const float *pred, const float *target, float *grad, double *out, int64_t n, double *work,
                 void *stream);

/* Adam step on FP32 master weights p with gradient g, moments m and v, and
 * the BF16 copy pb the kernels read (pb may be NULL). */
int he4_fno_adam(float *p, const float *g, float *m, float *v, uint16_t *pb, int64_t n, float lr, float beta1,
                 float beta2, float eps, int32_t step, void *stream);
/* FP32 -> BF16 (round to nearest even) */
int he4_fno_to_bf16(const float *x, uint16_t *y, int64_t n, void *stream);

/* grid transfer between the solver grid (nf^3, FP64, complex when
 * complex_src) and the FNO grid (nc^3 = (nf/f)^3, FP32):
 * restriction = average over f^3 blocks, times scale, into dst channel(s)
 * (two channels Re, Im for complex input). */
int he4_fno_restrict(const double *src, float *dst, int32_t nf, int32_t f, int32_t complex_src, float scale,
                     void *stream);
/* prolongation: dst (complex FP64, nf^3) += scale * trilinear interpolation
 * (periodic) of the two-channel coarse field src (Re, Im) */
int he4_fno_prolong_add(const float *src, double *dst, int32_t nf, int32_t f, float scale, void *stream);
/* nearest-grid-point particle density on the coarse grid: dst[nc^3] =
 * counts / (npar h_c^3) * scale for particles r[3][npar] in the box
 * [-xmax, xmax)^3 (FP64 positions) */
int he4_fno_deposit(const double *r, int32_t npar, float *dst, int32_t nc, double xmax, float scale, void *stream);

/* parareal correction of one state array (n FP64 values):
 * u <- s (g_new + fine - g_old), where u holds the previous iterate on
 * entry.  renorm: s rescales the result to the norm of `fine` (a projection
 * on the norm the fine propagator conserves; the fixed point, u = fine, is
 * unchanged), else s = 1.  out (device, 4 doubles): out[0] = sum (u_new -
 * u_old)^2, out[1] = sum u_old^2, out[2..3] = sum |g_new + fine - g_old|^2
 * and sum |fine|^2 (renorm only); fixed-order sums.  work:
 * HE4_FNO_LOSS_WORK doubles of device scratch. */
int he4_parareal_correct(const double *gnew, const double *fine, const double *gold, double *u, int64_t n,
                         int32_t renorm, double *out, double *work, void *stream);

#ifdef __cplusplus
}
#endif
#endif

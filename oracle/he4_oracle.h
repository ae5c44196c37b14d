/*
 * he4_oracle.h -- CPU FP64 oracle of the reference time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker or as the timed CPU baseline; the product path never
 * calls it.
 *
 * The functions mirror include/he4_tddft.h one to one with an ora_ prefix so
 * that parity tests drive both through the same call sequence.
 */
#ifndef HE4_ORACLE_H
#define HE4_ORACLE_H
#include <stdint.h>
#include "../include/he4_tddft.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_state ora_state;

int ora_create(const he4_params *p, ora_state **out);
void ora_destroy(ora_state *s);
int ora_set_state(ora_state *s, const double *psi, const double *rimp,
                  const double *vimp);
int ora_get_state(ora_state *s, double *psi, double *rimp, double *vimp,
                  double *aimp);
int ora_potenimp(ora_state *s);
int ora_poten(ora_state *s);
int ora_forceimp(ora_state *s);
int ora_field(ora_state *s);
int ora_step_rk(ora_state *s, double deltat, double means[9]);
int ora_step_pc(ora_state *s, double deltat, double err[3], double means[9]);
int ora_run(ora_state *s, int32_t nsteps, double deltat, double *err,
            double *means);
int ora_energy(ora_state *s, he4_energies *e);
int ora_diagnostics(ora_state *s, int32_t n4, double out[4]);
int ora_bubble_radius(ora_state *s, int32_t nr, double *rb, int32_t found[2],
                      int32_t *ir, double xms[3], double *rr, double *denr);
int ora_get_field(ora_state *s, int32_t which, double *out);
int ora_get_kernel(ora_state *s, int32_t which, double *out);
void ora_set_threads(int n);

/* Building blocks exposed for pinning tests. */
int ora_fd_weights(int npd, int id, double *w); /* centre row, no 1/h^id */
int ora_fd_rows(int npd, int id, double *rows); /* whole matrix, npd<=15 */
double ora_si(double x);                        /* sine integral Si(x)   */
double ora_v_he2s_fci(double x);                /* V_He2s_fci in K       */
int ora_fft3_r2c(int nx, int ny, int nz, const double *in, double *out);
int ora_fft3_c2r(int nx, int ny, int nz, const double *in, double *out);
int ora_spline(const double *x, const double *y, double *a, double *b,
               double *c, double *d, double s1, double sn, int n);
int ora_deriv(ora_state *s, int id, int axis, const double *f, double *df);
/* The search half of Bubble_Radius_esferic on a binned radial density
 * (denr is normalised in place; rr receives the bin radii). */
int ora_bubble_search(int32_t nr, double dr, double xnorm, const double xms[3],
                      double *rr, double *denr, double *rb, int32_t found[2],
                      int32_t *ir);

#ifdef __cplusplus
}
#endif
#endif

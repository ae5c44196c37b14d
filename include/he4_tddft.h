/*
 * he4_tddft.h -- C ABI of the B200 time-step library for the Orsay-Trento
 * time-dependent 4He density functional with a Bohmian test-particle impurity.
 *
 * The reference program (Fortran 90, DFT4He3d.f90) keeps all state in module
 * variables and calls argument-less subroutines.  This header replaces the
 * per-time-step calls of its main loop with explicit entry points on a handle
 * that owns every device array.  The Fortran host keeps the namelist parsing
 * (DFT4He3d.f90:147-187), readenc/printoutc file I/O and diagnostics and binds
 * these functions through an ISO_C_BINDING interface block, one bind(C)
 * interface per entry point below.
 *
 * Conventions
 *  - Grid arrays are x-fastest: C [nz][ny][nx] == Fortran a(nx,ny,nz).
 *  - Complex arrays are interleaved (re,im) doubles == Fortran complex(8).
 *  - Particle arrays are [3][n_par] == Fortran rimp(N_par,3).
 *  - Every function returns HE4_OK (0) or a negative HE4_E_* code; nothing
 *    aborts the host process.  he4_strerror() turns a code into text, and
 *    he4_last_error() returns the detail message of the last failing call on
 *    this thread.
 *  - One host thread per handle; handles are independent.
 */
#ifndef HE4_TDDFT_H
#define HE4_TDDFT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HE4_OK 0
#define HE4_E_ARG (-1)         /* invalid argument or parameter            */
#define HE4_E_UNSUPPORTED (-2) /* valid in the reference, not implemented   */
#define HE4_E_NOMEM (-3)       /* device or host allocation failed          */
#define HE4_E_CUDA (-4)        /* a CUDA runtime call failed                */
#define HE4_E_STATE (-5)       /* call order violated (e.g. no state set)   */
#define HE4_E_NONFINITE (-6)   /* a returned scalar is NaN or inf           */
#define HE4_E_NODEVICE (-7)    /* no usable sm_100 device                   */

/* core4 of the namelist (modules.f90:210): 'OT ' or 'OTC'. */
enum { HE4_CORE_OT = 0, HE4_CORE_OTC = 1 };

/* Source of the impurity pair-potential kernel Vq (DFT4He3d.f90:527-536). */
enum {
  HE4_POT_TABLE = 0, /* caller supplies Vq on the half-spectrum grid        */
  HE4_POT_MORSE = 1, /* V(r)=D[(1-exp(-a(r-re)))^2-1], r<r_cutoff -> umax,  */
                     /* transformed by the FT_V_spline procedure           */
  HE4_POT_NULL = 2,  /* V = 0 ('null' entry of Select_Pot)                  */
  HE4_POT_RTABLE = 3, /* caller samples V(r) (any Select_Pot entry) on a    */
                      /* uniform r grid; splined, r<r_cutoff -> umax, 0 past*/
                      /* the last point, transformed by FT_V_spline         */
  HE4_POT_HE2S_FCI = 4 /* Select_Pot 'He2S_fci' (V_impur.f90:179-183,       */
                       /* 2962-3008): He(2S)-He, sum of Pg(k) r^-(5+k),     */
                       /* k=1..11, evaluated on the device in double-double */
                       /* arithmetic (the reference uses real*16), 580.0065 K*/
                       /* inside 3.17502 A; r<r_cutoff -> umax as Select_Pot*/
};

/* Arithmetic of the convolution FFTs and the pointwise potential assembly.
 * HE4_PREC_FP64: everything in FP64 (the reference's arithmetic).
 * HE4_PREC_FP32CONV: the half spectra of the convolution FFTs, their
 *   twiddles, the k-space kernels (wcgk, fvlj4, kalfs, Vq) and the derivative
 *   symbol are FP32; real grids, the wavefunction update, the reductions and
 *   the particle integration stay FP64.  Needs every axis length to be a
 *   power of two in [16, 256]; otherwise he4_create returns
 *   HE4_E_UNSUPPORTED. */
enum { HE4_PREC_FP64 = 0, HE4_PREC_FP32CONV = 1 };

typedef struct he4_params {
  /* grid (namelist nx,ny,nz,xmax,ymax,zmax; DFT4He3d.f90:271-354) */
  int32_t nx, ny, nz;
  double xmax, ymax, zmax;
  /* derivatives (module deriva): npd odd in [3,25]; icon 8 = periodic,
   * icon 13 = centred stencils with f = 0 outside the grid (redef.f:133-170),
   * icon 12 = the same at the upper end and the Bickley matrix's one-sided
   * rows for the first npd/2 points (redef.f:133-150; npd <= 15) */
  int32_t npd, icon;
  /* functional */
  int32_t core4;
  double cp4, cpp4, den4c, alphas, l_alfs, den0s, h2o2m4;
  double c_solid, beta_solid, den_m; /* penalty C, beta, den_m (he4 module) */
  double eps4, sigma4, b4, h4;       /* screened LJ (lenard4), h4 = core   */
  /* impurity */
  int32_t n_par;  /* number of Bohmian test particles                     */
  int32_t ironx;  /* number of 7-point smoothings of denx (field module)  */
  double mimpur;  /* impurity mass in amu                                  */
  int32_t pot_kind;
  double morse_d, morse_alpha, morse_re, r_cutoff, umax;
  int32_t nq;              /* q-points of the FT_V_spline table            */
  const double *vq_table;  /* HE4_POT_TABLE: [nz][ny][nx/2+1] real values  */
  /* absorbing layer timec = (Lambdah(1+tanh((z-tzmean)/tzsurf)), 1) */
  double lambdah, tzmean, tzsurf;
  int32_t precision;
  int32_t device; /* CUDA device ordinal                                   */
  /* HE4_POT_RTABLE: V(r) in K at r_i = vr_r0 + i vr_dr, i < n_vr; needs
   * n_vr >= 4, vr_dr > 0 and vr_r0 <= r_cutoff (the table covers the
   * potential from the cutoff on).  Borrowed for he4_create only. */
  const double *vr_table;
  int32_t n_vr;
  double vr_r0, vr_dr;
} he4_params;

/* Energies of energy.f90:51-124, same names as module energies. */
typedef struct he4_energies {
  double etot, etot4, ekin4, elj4, ecor4, ealphas, esolid;
  double ekinx, ekinqx, eHeX, eimpu;
} he4_energies;

/* Real grid fields readable with he4_get_field (module arrays). */
enum {
  HE4_F_DEN = 0, HE4_F_POT4, HE4_F_DENX, HE4_F_PSIX, HE4_F_HPSIX, HE4_F_UIMP,
  HE4_F_DENCG, HE4_F_DELJ4, HE4_F_DENALF, HE4_F_UALPHAS, HE4_F_FALFS,
  HE4_F_INTXALF, HE4_F_INTYALF, HE4_F_INTZALF, HE4_F_DXDEN, HE4_F_DYDEN,
  HE4_F_DZDEN, HE4_F_FX, HE4_F_FY, HE4_F_FZ, HE4_F_PENALTY, HE4_F_CORR,
  HE4_F_COUNT
};

/* Half-spectrum kernels [nz][ny][nx/2+1] readable with he4_get_kernel. */
enum { HE4_K_WCGK = 0, HE4_K_FVLJ4, HE4_K_KALFS, HE4_K_VQ, HE4_K_PMOD,
       HE4_K_COUNT };

typedef struct he4_handle he4_handle;

/* Fill p with the reference defaults (modules.f90:15-19,81-90,124-139,
 * 144,205-210; DFT4He3d.f90:184-186). */
void he4_params_default(he4_params *p);

/* Replaces dimen (dimen.f90:29-143), fftini (fft.f90:5-76), Init_deriv_p
 * (init_deriv_parallel.f90:51-85) and the kernel construction of
 * DFT4He3d.f90:509-570 (fforma, FT_V_spline, initcg, kalfs). */
int he4_create(const he4_params *p, he4_handle **out);
void he4_destroy(he4_handle *h);

/* readenc mode 2 (readenc.f90:96-114): psi [nz][ny][nx] complex, rimp and
 * vimp [3][n_par].  Also sets den=|psi|^2 (readenc.f90:102), zeroes the
 * RK/PC histories (dimen.f90:75-79,133-134; DFT4He3d.f90:841-845) and makes
 * the next he4_run/he4_step call start with the RK-Gill starter.
 * The arrays of he4_set_state and he4_get_state may be host or device
 * memory (unified addressing); device arrays written on another stream must
 * be complete before the call. */
int he4_set_state(he4_handle *h, const double *psi, const double *rimp,
                  const double *vimp);
/* printoutc inputs (printoutc.f90:139-142) plus aimp. Any pointer may be NULL. */
int he4_get_state(he4_handle *h, double *psi, double *rimp, double *vimp,
                  double *aimp);

/* Field evaluation pieces: potenimp (potenimp.f90:1-20), poten
 * (poten.f90:5-129), forceimp (potenimp.f90:24-73), and all three in that
 * order (DFT4He3d.f90:630-634, 861-863). */
int he4_potenimp(he4_handle *h);
int he4_poten(he4_handle *h);
int he4_forceimp(he4_handle *h);
int he4_field(he4_handle *h);

/* One time step followed by the field evaluation of DFT4He3d.f90:861-863.
 * he4_step_rk = steprk (steprk.f90:1-128); he4_step_pc = steppc
 * (steppc.f90:1-155) and returns errHe, errimp, errvimp in err[3].
 * means[9] (nullable) = <rimp>,<vimp>,<aimp> per axis after the field
 * evaluation, internal units (DFT4He3d.f90:864-878). */
int he4_step_rk(he4_handle *h, double deltat, double means[9]);
int he4_step_pc(he4_handle *h, double deltat, double err[3], double means[9]);

/* The iteration loop of DFT4He3d.f90:848-863 for nsteps steps: the first
 * three steps after he4_set_state use steprk, the rest steppc (lrk=false).
 * err [nsteps][3] (zeros for RK steps) and means [nsteps][9] are nullable.
 * Runs from a captured CUDA graph after the first PC step. */
int he4_run(he4_handle *h, int32_t nsteps, double deltat, double *err,
            double *means);

/* energy() (energy.f90:12-129) evaluated on the current fields. */
int he4_energy(he4_handle *h, he4_energies *e);

/* Diagnostics of the pener block reduced on the device: out[0] = He atom
 * number sum(den)*dxyz (DFT4He3d.f90:885-886), out[1..3] = centre of mass
 * of den (r_cm.f90:23-58, divided by n4 as r_cm does). */
int he4_diagnostics(he4_handle *h, int32_t n4, double out[4]);

/* Spherical bubble radius around the impurity, the Lspherical_bubble
 * diagnostic of the pener block (DFT4He3d.f90:929-986 with
 * bubble_radius_esferic.f90:1-134), reduced on the device.  The centre is
 * the grid point (ipx,ipy,ipz) of the mean trajectory position
 * (DFT4He3d.f90:893-898); xms[3] receives the impurity mean-square radii
 * sqrt(sum denx x^2 dxyz) (DFT4He3d.f90:933-947).  den is averaged over nr
 * radial bins of width dr = rmax/(nr-1) (the reference uses nr = 501),
 * normalised to the atom number and splined; found[0] reports the first
 * density maximum past max(xms) (Lcontrol(1)), found[1] the half-maximum
 * crossing refined by Newton iterations (Lcontrol(2)); rb is the radius
 * when both are set; ir the 1-based bin of the maximum (0 if none).  rr and
 * denr (nr values each, may be NULL) receive the radii and the normalised
 * radial density.  The reference stops when a grid point lies past rmax
 * (the mean position has a positive grid coordinate); this returns
 * HE4_E_ARG instead.  nr must lie in [4, 8192]. */
int he4_bubble_radius(he4_handle *h, int32_t nr, double *rb, int32_t found[2],
                      int32_t *ir, double xms[3], double *rr, double *denr);

/* he4_diagnostics without a handle and without any allocation.  It has no
 * counterpart in the reference; it exists for callers that cannot call
 * cudaMalloc: hosts whose device memory belongs to another allocator (a
 * framework's memory pool, a Fortran runtime's device arrays) and that may
 * not add raw cudaMalloc/cudaFree calls, cudaFree being a device-wide
 * synchronisation.  den is a device array [nz][ny][nx]; out is a device
 * array of 4 doubles receiving what he4_diagnostics returns; stream is a
 * cudaStream_t (NULL: the legacy default stream); the call is asynchronous
 * on that stream.  Its scratch is a fixed 128 KiB array inside the library
 * (four partial sums per z plane), so nz may not exceed 4096: larger grids
 * return HE4_E_ARG.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress, with the device current); make
 * that first call before any stream capture.  The address stays cached for
 * the life of the process; after cudaDeviceReset on that device it is stale,
 * so do not call this function on a device the host has reset.  All calls
 * share the array: calls that may overlap on the GPU (other streams, other
 * threads) race and must be serialised by the caller. */
int he4_diagnostics_noalloc(const double *den, int32_t nx, int32_t ny, int32_t nz,
                            double xmax, double ymax, double zmax, int32_t n4,
                            double *out, void *stream);

/* Checkpoint without stopping the time loop (printoutc every pcurr steps,
 * DFT4He3d.f90:992-1009, printoutc.f90:67-76).  he4_snapshot_begin copies
 * psi, rimp, vimp and aimp into a device snapshot on the handle's stream and
 * returns at once; the snapshot then travels to pinned host memory owned by
 * the handle on a separate copy stream, overlapping the steps called next.
 * he4_snapshot_wait waits for that copy and returns pointers into the
 * pinned memory (psi [nz][ny][nx] complex as 2N doubles, the particle
 * arrays [3][n_par]), valid until the next he4_snapshot_begin or
 * he4_destroy.  One snapshot is in flight at a time: a second begin waits
 * for the first copy.  The first call allocates the snapshot (16N + 72 n_par
 * bytes on the device and as much pinned host memory). */
int he4_snapshot_begin(he4_handle *h);
int he4_snapshot_wait(he4_handle *h, const double **psi, const double **rimp,
                      const double **vimp, const double **aimp);

/* Copy-out of a real grid field ([nz][ny][nx]) or a half-spectrum kernel. */
int he4_get_field(he4_handle *h, int32_t which, double *out);
int he4_get_kernel(he4_handle *h, int32_t which, double *out);

/* The handle's 3D real FFT on host buffers (same transform as the
 * convolutions use; FFTW r2c/c2r conventions of fft.f90:43-65):
 * in [nz][ny][nx] real -> out [nz][ny][nx/2+1] complex, unnormalised, and
 * back (unnormalised: c2r(r2c(f)) = N f). */
int he4_fft_r2c(he4_handle *h, const double *in, double *out);
int he4_fft_c2r(he4_handle *h, const double *in, double *out);

/* Measurement hook: launches one kernel of the step `reps` times on the
 * handle's current buffers between two CUDA events on the handle's stream.
 * which: 0 z-pass convolution (FFT_z, kernel multiply, IFFT_z), 1 y pass,
 * 2 x pass R2C, 3 x pass C2R, 4 plain z pass, 5 z convolution without a
 * kernel, 6 z convolution with three outputs (these only touch FFT scratch
 * buffers), 7 the density gradient stencil, 8 the merged pot4 assembly on
 * FP64 grids, 9 the merged pot4 assembly on the float grids of the
 * FP32-convolution form, 10 the x pass C2R into a float grid, 11 the
 * density gradient into float grids, 12 the inverse y pass (9-11 need that
 * form; 7-11 rewrite fields of the current evaluation, so call them after a
 * field evaluation; the next step evaluates its field again).
 * Returns the mean time per launch, the algorithmic bytes one launch moves
 * (each input read once, each output written once) and the kernel's name. */
int he4_bench_kernel(he4_handle *h, int32_t which, int32_t reps, double *ms_per_launch,
                     double *bytes_per_launch, char *name, int32_t name_len);

/* Stream the handle launches on (cudaStream_t), for event timing. */
int he4_get_stream(he4_handle *h, void **stream);
/* Device address of one of the handle's state arrays, for device-side
 * coupling (the parareal driver, the FNO data pipeline): psi complex
 * [nz][ny][nx], rimp / vimp [3][n_par], den and denx [nz][ny][nx].  Valid
 * until he4_destroy; work on them must be ordered with the handle's stream. */
enum { HE4_D_PSI = 0, HE4_D_RIMP = 1, HE4_D_VIMP = 2, HE4_D_DEN = 3, HE4_D_DENX = 4 };
int he4_device_ptr(he4_handle *h, int32_t which, void **ptr);
/* Number of kernels this handle has launched (graph launches count the
 * kernels inside the graph). */
int64_t he4_launch_count(he4_handle *h);
/* CUDA-graph use of he4_run: how many PC-step graphs the handle captured
 * (one per distinct buffer rotation of the step; the rotations repeat every
 * 30 steps) and how many PC steps ran uncaptured (launched one kernel at a
 * time) because no captured graph matched.  Has no counterpart in the
 * reference. */
int he4_graph_stats(he4_handle *h, int64_t *captured, int64_t *uncaptured);

/* Tile shapes of the FFT passes: tiles = {n1 x, n1 y, n1 z, px, wy, wz}.
 * For axis lengths 16..256 (powers of two) n1 is the four-step split
 * N = n1 * (N / n1) of the register path (0 = default); for the other
 * lengths px / wy / wz are the pencils per CTA (multiples of 8 in [8, 32])
 * of the x, y and z passes.  Setting drops the handle's captured graphs. */
int he4_set_tiles(he4_handle *h, const int32_t tiles[6]);
int he4_get_tiles(he4_handle *h, int32_t tiles[6]);
/* Autotuner: coordinate search over the tile shapes of the three axes,
 * each candidate timed (CUDA events) as `reps` mean-field evaluations of
 * the current state; the fastest shapes are applied and returned. */
int he4_tune(he4_handle *h, int32_t reps, double *best_ms, int32_t tiles[6]);

/* Batched ensemble: n independent systems (grids may differ; one device)
 * advanced together by CUDA graphs that each hold K consecutive ensemble
 * PC steps (K = 30, 10, 5 or 1, the largest the remaining steps allow;
 * every member's K steps are one parallel branch of the graph), so 30
 * steps are one graph launch.  The graphs are captured on first use and
 * replayed; the members' buffer states repeat every 30 steps.  Members are ordinary
 * handles: he4_set_state / he4_get_state / he4_energy on
 * he4_batch_member(b, i) work as for any handle and are ordered after the
 * ensemble's work.  he4_batch_tune tunes one member per distinct grid and
 * applies its shapes to the others (tiles [n][6], ms [n], either may be
 * NULL).  he4_batch_run advances every member by nsteps (RK-Gill starter
 * first where a member needs it) and returns per member the largest
 * errHe/errimp/errvimp of the run (err_max [n][3]) and the last step's
 * means ([n][9]); HE4_E_NONFINITE names the first member that went
 * non-finite. */
typedef struct he4_batch he4_batch;
int he4_batch_create(int32_t n, const he4_params *params, he4_batch **out);
void he4_batch_destroy(he4_batch *b);
int32_t he4_batch_size(const he4_batch *b);
he4_handle *he4_batch_member(he4_batch *b, int32_t i);
int he4_batch_tune(he4_batch *b, int32_t reps, int32_t *tiles, double *ms);
int he4_batch_run(he4_batch *b, int32_t nsteps, double deltat, double *err_max, double *means);
int64_t he4_batch_launch_count(const he4_batch *b);

const char *he4_strerror(int code);
const char *he4_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HE4_TDDFT_H */

// setup.cu -- construction of the k-space kernels and stencil weights,
// done once in he4_create (DFT4He3d.f90:256,302-354,509-570).
//
//  * pmod, wcgk (initcg.f90:32-49), kalfs (DFT4He3d.f90:566-570) and the
//    screened Lennard-Jones kernel fvlj4 (fforma.f90:36-60, OT core) are
//    evaluated per half-spectrum point on the GPU.  The sine integral needed
//    by fforma (NAG S13ADF in the reference) is computed here by its power
//    series below 4 and by the continued fraction of E1(ix) (modified Lentz)
//    above, Si(x) = pi/2 + Im E1(ix).
//  * Vq follows FT_V_spline (FT_V_spline.f90:14-276): a cubic spline of V(r)
//    on 100001 points, its radial Fourier transform integrated analytically
//    segment by segment at Nq values of q (the 1e8-term sums run on the GPU,
//    one CTA per q), the small-q refit, a spline in q and its evaluation at
//    |p|, rounded to single precision as cmplx() does (DFT4He3d.f90:533).
//    The two tridiagonal spline solves are sequential and run on the host.
//  * Stencil weights: the centre row of the Bickley matrix (newder.f with
//    ICON=1, table mates.f:172-14043) from its closed form, rounded exactly.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cmath>

#include "common.cuh"
#include "reduce.cuh"

namespace he4 {

static constexpr double kPi = 3.14159265358979323846264338327950288;

// ---------------------------------------------------------------------------
// stencil weights
// ---------------------------------------------------------------------------
typedef unsigned __int128 u128;

static u128 gcd_u128(u128 a, u128 b) {
  while (b) {
    u128 t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// num/den (> 0) rounded to the nearest double, ties to even
static double div_round_nearest(u128 num, u128 den) {
  u128 q = num / den, r = num % den;
  int e = 0;
  const u128 lo = (u128)1 << 63, hi = (u128)1 << 64;
  while (q < lo) {
    r <<= 1;
    q <<= 1;
    if (r >= den) {
      q |= 1;
      r -= den;
    }
    e--;
  }
  bool sticky = (r != 0);
  while (q >= hi) {
    sticky = sticky || (q & 1);
    q >>= 1;
    e++;
  }
  uint64_t m = (uint64_t)q;
  uint64_t keep = m >> 11, rem = m & 0x7FFu;
  if (rem > 0x400u || (rem == 0x400u && (sticky || (keep & 1u)))) keep++;
  return ldexp((double)keep, e + 11);
}

static u128 factorial(int n) {
  u128 f = 1;
  for (int i = 2; i <= n; i++) f *= (u128)i;
  return f;
}

int fd_weights(int npd, int order, double *w) {
  if (npd < 3 || npd > 25 || npd % 2 == 0 || (order != 1 && order != 2)) return HE4_E_ARG;
  const int m = npd / 2;
  const u128 mm = factorial(m) * factorial(m);
  for (int j = 0; j < npd; j++) w[j] = 0.0;
  for (int j = 1; j <= m; j++) {
    // order 1: (-1)^(j+1) (m!)^2 / (j (m-j)! (m+j)!), antisymmetric
    // order 2: 2 (-1)^(j+1) (m!)^2 / (j^2 (m-j)! (m+j)!), symmetric
    u128 num = (order == 1) ? mm : 2 * mm;
    u128 den = (u128)j * factorial(m - j) * factorial(m + j);
    if (order == 2) den *= (u128)j;
    const u128 g = gcd_u128(num, den);
    double v = div_round_nearest(num / g, den / g);
    if (j % 2 == 0) v = -v;
    w[m + j] = v;
    w[m - j] = (order == 1) ? -v : v;
  }
  if (order == 2) {  // centre: -2 sum_{j<=m} 1/j^2
    u128 L = 1;
    for (int j = 1; j <= m; j++) L = L / gcd_u128(L, (u128)j) * (u128)j;
    const u128 L2 = L * L;
    u128 num = 0;
    for (int j = 1; j <= m; j++) num += L2 / ((u128)j * (u128)j);
    num *= 2;
    const u128 g = gcd_u128(num, L2);
    w[m] = -div_round_nearest(num / g, L2 / g);
  }
  return HE4_OK;
}

// The whole npd x npd Bickley matrix of order `order` (newder.f:99-125 with
// ICON=1; BLOCK DATA BLKDS, mates.f:172-14043): rows[c * npd + j] is the
// order-th derivative at node c of the Lagrange basis polynomial of node j
// over the nodes 0..npd-1 (unit spacing).  Exact integers (the basis
// numerator's coefficients, its denominator prod (j - q)), rounded once to
// nearest; the table's entries are these rationals.  npd <= 15 keeps every
// intermediate inside 128 bits.
int fd_rows(int npd, int order, double *rows) {
  typedef __int128 i128;
  if (npd < 3 || npd > 15 || npd % 2 == 0 || (order != 1 && order != 2)) return HE4_E_ARG;
  for (int j = 0; j < npd; j++) {
    i128 coef[16] = {0};  // prod_{q != j} (x - q), ascending powers
    coef[0] = 1;
    int deg = 0;
    i128 den = 1;
    for (int q = 0; q < npd; q++) {
      if (q == j) continue;
      for (int d = deg + 1; d >= 1; d--) coef[d] = coef[d - 1] - (i128)q * coef[d];
      coef[0] = -(i128)q * coef[0];
      deg++;
      den *= (i128)(j - q);
    }
    for (int c = 0; c < npd; c++) {
      i128 v = 0;
      for (int d = order; d <= deg; d++) {
        i128 f = 1, pw = 1;
        for (int u = 0; u < order; u++) f *= (i128)(d - u);
        for (int u = 0; u < d - order; u++) pw *= (i128)c;
        v += coef[d] * f * pw;
      }
      const bool neg = (v < 0) != (den < 0);
      const u128 num = (u128)(v < 0 ? -v : v), dd = (u128)(den < 0 ? -den : den);
      double r = 0.0;
      if (num != 0) {
        const u128 g = gcd_u128(num, dd);
        r = div_round_nearest(num / g, dd / g);
      }
      rows[c * npd + j] = neg ? -r : r;
    }
  }
  return HE4_OK;
}

// ---------------------------------------------------------------------------
// device special functions
// ---------------------------------------------------------------------------
__device__ double si_dev(double x) {
  const double ax = fabs(x);
  double r;
  if (ax == 0.0) return 0.0;
  if (ax < 4.0) {
    const double x2 = ax * ax;
    double term = ax, sum = ax;
    for (int n = 1; n < 60; n++) {
      term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
      const double t = term / (2.0 * n + 1.0);
      sum += t;
      if (fabs(t) < 1e-18 * fabs(sum)) break;
    }
    r = sum;
  } else {
    // continued fraction of E1(z), z = i ax, by the modified Lentz method
    double br = 1.0, bi = ax;                     // b = 1 + i ax
    double cr = 1e300, ci = 0.0;                  // c = 1/tiny
    double den = br * br + bi * bi;
    double dr = br / den, di = -bi / den;         // d = 1/b
    double hr = dr, hi = di;                      // h = d
    for (int i = 1; i < 1000; i++) {
      const double a = -(double)i * (double)i;
      br += 2.0;
      // d = 1/(a d + b)
      double tr = a * dr + br, ti = a * di + bi;
      den = tr * tr + ti * ti;
      dr = tr / den;
      di = -ti / den;
      // c = b + a/c
      den = cr * cr + ci * ci;
      const double acr = a * cr / den, aci = -a * ci / den;
      cr = br + acr;
      ci = bi + aci;
      // del = c d ; h *= del
      const double er = cr * dr - ci * di, ei = cr * di + ci * dr;
      const double nhr = hr * er - hi * ei, nhi = hr * ei + hi * er;
      hr = nhr;
      hi = nhi;
      if (fabs(er - 1.0) + fabs(ei) < 1e-17) break;
    }
    double s, c;
    sincos(ax, &s, &c);
    // h *= exp(-i ax)
    const double fr = hr * c + hi * s, fi = hi * c - hr * s;
    (void)fr;
    r = 0.5 * kPi + fi;
  }
  return x < 0 ? -r : r;
}

// sinint(a,x) of fforma.f90:143-196 for a > 0: pi/2 - Si(ax)
__device__ double sinint_dev(double a, double x) {
  const double r = si_dev(a * x);
  return (a > 0.0) ? 0.5 * kPi - r : 0.5 * kPi + r;
}

// int_x^inf sin(a t)/t^11 dt (sinx11, fforma.f90:73-102)
__device__ double sinx11_dev(double a, double x) {
  const double y = a * x, y2 = y * y;
  const double d[5] = {1.0, y2, y2 * y2, y2 * y2 * y2, (y2 * y2) * (y2 * y2)};
  const double b[5] = {40320.0, -720.0, 24.0, -2.0, 1.0};
  const double c[5] = {362880.0, -5040.0, 120.0, -6.0, 1.0};
  double bd = 0.0, cd = 0.0;
  for (int i = 0; i < 5; i++) {
    bd += b[i] * d[i];
    cd += c[i] * d[i];
  }
  const double x9 = x * x * x * x * x * x * x * x * x;
  double s, co;
  sincos(y, &s, &co);
  const double res1 = (a * bd * co + cd * s / x) / (3628800.0 * x9);
  const double res2 = -(pow(a, 10.0) * sinint_dev(a, x)) / 3628800.0;
  return res1 + res2;
}

// int_x^inf sin(a t)/t^5 dt (sinx5, fforma.f90:108-137)
__device__ double sinx5_dev(double a, double x) {
  const double y = a * x, y2 = y * y;
  const double bd = -2.0 + y2, cd = -6.0 + y2;
  double s, co;
  sincos(y, &s, &co);
  const double res1 = -(a * bd * co + cd * s / x) / (24.0 * x * x * x);
  const double res2 = (pow(a, 4.0) * sinint_dev(a, x)) / 24.0;
  return res1 + res2;
}

struct KArgs {
  int nxh, ny, nz;
  const double *px, *py, *pz;
  double eps, sigma, hc, l_alfs, bforce;
};

__global__ void k_kspace(KArgs a, double *pmod, double *wcgk, double *fvlj4, double *kalfs) {
  const size_t H = (size_t)a.nxh * a.ny * a.nz;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < H; t += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(t % a.nxh);
    const int iy = (int)((t / a.nxh) % a.ny);
    const int iz = (int)(t / ((size_t)a.nxh * a.ny));
    // same rounding as the reference: sqrt(px^2 + py^2 + pz^2), no fusing
    const double px2 = __dmul_rn(a.px[ix], a.px[ix]);
    const double py2 = __dmul_rn(a.py[iy], a.py[iy]);
    const double pz2 = __dmul_rn(a.pz[iz], a.pz[iz]);
    const double p = sqrt(__dadd_rn(__dadd_rn(px2, py2), pz2));
    pmod[t] = p;
    const double twopi = 2.0 * kPi;
    // fforma: OT core
    if (fabs(p) < 1e-10) {
      fvlj4[t] = a.bforce;
    } else {
      const double sigma6 = pow(a.sigma, 6.0), aux1 = 8.0 * a.eps;
      const double a2 = twopi * p;
      const double t1 = sinx11_dev(a2, a.hc), t2 = sinx5_dev(a2, a.hc);
      fvlj4[t] = (aux1 * sigma6 * (sigma6 * t1 - t2)) / p;
    }
    // initcg
    if (p > 0.0) {
      const double arg = twopi * p * a.hc;
      double s, c;
      sincos(arg, &s, &c);
      const double aux = s - arg * c;
      wcgk[t] = (fabs(aux) < 1e-10) ? 1.0 : 3.0 * aux / (arg * arg * arg);
    } else {
      wcgk[t] = 1.0;
    }
    const double e = kPi * a.l_alfs * p;
    kalfs[t] = exp(-(e * e));
  }
}

// ---------------------------------------------------------------------------
// FT_V_spline
// ---------------------------------------------------------------------------
// spline of a caller-sampled V(r) (HE4_POT_RTABLE): uniform nodes
// r_i = r0 + i dr, natural end conditions, global-form coefficients
struct RTable {
  int n = 0;
  double r0 = 0.0, dr = 0.0, rend = 0.0;
  std::vector<double> A, B, C, D;
};

static int rtable_build(const he4_params &p, RTable *t) {
  if (!p.vr_table || p.n_vr < 4 || !(p.vr_dr > 0.0) || !(p.vr_r0 <= p.r_cutoff + 1e-8)) {
    set_error("HE4_POT_RTABLE needs vr_table, n_vr >= 4, vr_dr > 0 and vr_r0 <= r_cutoff");
    return HE4_E_ARG;
  }
  const int n = p.n_vr;
  std::vector<double> x(n), y(n);
  for (int i = 0; i < n; i++) {
    x[i] = p.vr_r0 + (double)i * p.vr_dr;
    y[i] = p.vr_table[i];
    if (!std::isfinite(y[i])) {
      set_error("vr_table[%d] is not finite", i);
      return HE4_E_ARG;
    }
  }
  t->n = n;
  t->r0 = p.vr_r0;
  t->dr = p.vr_dr;
  t->rend = x[n - 1];
  t->A.resize(n);
  t->B.resize(n);
  t->C.resize(n);
  t->D.resize(n);
  return spline_global(x.data(), y.data(), t->A.data(), t->B.data(), t->C.data(), t->D.data(), 0.0, 0.0, n);
}

static double rtable_eval(const RTable &t, double r) {
  if (r > t.rend) return 0.0;
  int k = (int)((r - t.r0) / t.dr);
  if (k < 0) k = 0;
  if (k > t.n - 2) k = t.n - 2;
  return t.A[k] + r * (t.B[k] + r * (t.C[k] + r * t.D[k]));
}

// Select_Pot conventions (V_impur.f90:84-935): r < r_cutoff -> umax.  The
// caller-sampled table is evaluated here; the analytic entries run on the
// device (k_pair_pot).
static double pair_pot(const he4_params &p, const RTable *t, double r) {
  if (p.pot_kind == HE4_POT_NULL) return 0.0;
  if (r < p.r_cutoff) return p.umax;
  return rtable_eval(*t, r);
}

// ---------------------------------------------------------------------------
// analytic Select_Pot entries on the device
// ---------------------------------------------------------------------------
// double-double numbers (hi + lo, |lo| <= ulp(hi)/2): Knuth's two-sum and
// the FMA two-product give the exact rounding errors of + and *; a
// quotient takes one correction step on the residual
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD dd_two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return DD{s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ DD dd_fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = a + b;
  return DD{s, b - (s - a)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = dd_two_sum(a.hi, b.hi);
  const DD t = dd_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return dd_fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
  const double p = a.hi * b.hi;
  const double e = fma(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
  return dd_fast_two_sum(p, e);
}
__device__ __forceinline__ DD dd_recip(double x) {  // 1/x
  const double q = 1.0 / x;
  const double r = fma(-q, x, 1.0);  // exact residual 1 - q x
  return dd_fast_two_sum(q, r / x);
}

// Pg(1..11) of Block Data Inicio_LJ_V_He2s_fci (V_impur.f90:2965-2980),
// the real*16 decimal constants split into hi + lo doubles
__constant__ double kHe2sPg[11][2] = {
    {-0x1.42e15606a60a7p+26, 0x1.dd3a6436341a8p-28},  {0x1.47ef02a3e655bp+32, -0x1.eb16493dff276p-23},
    {-0x1.27401c07c6057p+37, -0x1.a220013722c39p-18}, {0x1.35469e31e7656p+41, -0x1.358c7b5bdc35ep-14},
    {-0x1.a0860d440150fp+44, -0x1.01b219d398bf1p-10}, {0x1.776e6d55a7e11p+47, 0x1.c4445ee71dc20p-7},
    {-0x1.c92e2141b13a0p+49, 0x1.990ffee5e8bcap-5},   {0x1.72ca490c9d9abp+51, -0x1.7f2e612330a62p-3},
    {-0x1.7f6ee42e976d9p+52, 0x1.9b19fd2a249b5p-11}, {0x1.c912072946918p+52, -0x1.491e80ea3b0f9p-2},
    {-0x1.ddbc07afa638dp+51, -0x1.cf3f1e0d13c9ep-4}};

// V_He2s_fci (V_impur.f90:2983-3008): fcutoff = 580.0065 K for
// x <= 3.17502 A, else sum_k Pg(k) (1/x)^(5+k); the reference sums in
// real*16, here in double-double, and rounds once to double
__device__ double v_he2s_fci_dev(double x) {
  if (x <= 3.17502) return 5.8000649999999996e+02;
  const DD xq = dd_recip(x);
  DD aux = dd_mul(xq, xq);        // xq^2
  aux = dd_mul(aux, dd_mul(aux, aux));  // xq^6 = xq^(k0+1), k0 = 5
  DD sto{0.0, 0.0};
  for (int k = 0; k < 11; k++) {
    sto = dd_add(sto, dd_mul(DD{kHe2sPg[k][0], kHe2sPg[k][1]}, aux));
    aux = dd_mul(aux, xq);
  }
  return sto.hi + sto.lo;
}

struct PotArgs {
  int kind;
  double r_cutoff, umax, d, alpha, re;
};

__device__ double pair_pot_dev(const PotArgs &p, double r) {
  if (p.kind == HE4_POT_NULL) return 0.0;
  if (r < p.r_cutoff) return p.umax;
  if (p.kind == HE4_POT_HE2S_FCI) return v_he2s_fci_dev(r);
  const double e = 1.0 - exp(-p.alpha * (r - p.re));
  return p.d * (e * e - 1.0);
}

__global__ void k_pair_pot(const double *__restrict__ r, int n, PotArgs p, double *__restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = pair_pot_dev(p, r[i]);
}

// cubic spline with end second derivatives s1, sn; global-form coefficients
// a + x(b + x(c + x d)) per interval (Maron's algorithm, mates.f:36-117)
int spline_global(const double *x, const double *y, double *A, double *B, double *C, double *D, double s1,
                  double sn, int n) {
  if (n < 4) return HE4_E_ARG;
  const int n1 = n - 1, n2 = n - 2;
  // 0-based: a[i] = h_i, d[i] = divided difference
  for (int i = 0; i < n1; i++) {
    if (x[i + 1] - x[i] < 1e-10) return HE4_E_ARG;
    A[i] = x[i + 1] - x[i];
    D[i] = (y[i + 1] - y[i]) / A[i];
  }
  for (int i = 0; i < n2; i++) {
    B[i] = 2.0 * (A[i] + A[i + 1]);
    const int k = n1 - 1 - i;  // 1-based n1-i
    D[k] = 6.0 * (D[k] - D[k - 1]);
  }
  D[1] = D[1] - A[0] * s1;
  D[n1 - 1] = D[n1 - 1] - A[n1 - 1] * sn;
  for (int i = 1; i < n2; i++) {
    const double r = A[i] / B[i - 1];
    B[i] = B[i] - r * A[i];
    D[i + 1] = D[i + 1] - r * D[i];
  }
  D[n1 - 1] = D[n1 - 1] / B[n2 - 1];
  for (int i = 1; i < n2; i++) {
    const int k = n1 - 1 - i;
    D[k] = (D[k] - A[k] * D[k + 1]) / B[k - 1];
  }
  D[n - 1] = sn;
  double si1 = s1;
  for (int i = 0; i < n1; i++) {
    const double si = si1;
    si1 = D[i + 1];
    const double h = A[i], hi = 1.0 / h;
    const double x0 = x[i], x1 = x[i + 1];
    A[i] = (hi / 6.0) * (si * x1 * x1 * x1 - si1 * x0 * x0 * x0) + hi * (y[i] * x1 - y[i + 1] * x0) +
           (h / 6.0) * (si1 * x0 - si * x1);
    B[i] = (hi / 2.0) * (si1 * x0 * x0 - si * x1 * x1) + hi * (y[i + 1] - y[i]) + (h / 6.0) * (si - si1);
    C[i] = (hi / 2.0) * (si * x1 - si1 * x0);
    D[i] = (hi / 6.0) * (si1 - si);
  }
  return HE4_OK;
}

struct FtArgs {
  const double *x, *A, *B, *C, *D;
  int nseg;
  double hp, rc, f0;
};

// Vpp(i) = 4 pi / q * [f0 (sin(q rc)/q - rc cos(q rc))/q + sum_j segment_j]
// (FT_V_spline.f90:151-225); one CTA per q point, deterministic block sum
__global__ void k_ft_radial(FtArgs a, double *vpp) {
  __shared__ double sh[32];
  const int i = blockIdx.x;
  const double p = (double)i * a.hp;
  const double qpi = 4.0 * kPi;
  double acc = 0.0;
  if (p == 0.0) {
    for (int j = threadIdx.x; j < a.nseg; j += blockDim.x) {
      const double xa = a.x[j], xb = a.x[j + 1];
      acc += a.A[j] / 3.0 * (xb * xb * xb - xa * xa * xa) + a.B[j] / 4.0 * (pow(xb, 4.0) - pow(xa, 4.0)) +
             a.C[j] / 5.0 * (pow(xb, 5.0) - pow(xa, 5.0)) + a.D[j] / 6.0 * (pow(xb, 6.0) - pow(xa, 6.0));
    }
    const double fi = block_sum(acc, sh);
    if (threadIdx.x == 0) vpp[i] = (a.rc * a.rc * a.rc * a.f0 / 3.0 + fi) * qpi;
    return;
  }
  const double q = 2.0 * kPi * p;
  const double c1 = 1.0 / q, c2 = c1 * c1, c3 = c2 * c1, c4 = c2 * c2, c5 = c4 * c1;
  for (int j = threadIdx.x; j < a.nseg; j += blockDim.x) {
    const double rj = a.x[j], rj1 = a.x[j + 1];
    double sj, cj, sj1, cj1;
    sincos(q * rj, &sj, &cj);
    sincos(q * rj1, &sj1, &cj1);
    const double A = a.A[j], B = a.B[j], C = a.C[j], D = a.D[j];
    acc += (A + (B + (C + D * rj) * rj) * rj) * rj * c1 * cj - (A + (B + (C + D * rj1) * rj1) * rj1) * rj1 * c1 * cj1 +
           (A + (2.0 * B + (3.0 * C + 4.0 * D * rj1) * rj1) * rj1) * c2 * sj1 -
           (A + (2.0 * B + (3.0 * C + 4.0 * D * rj) * rj) * rj) * c2 * sj +
           (2.0 * B + (6.0 * C + 12.0 * D * rj1) * rj1) * c3 * cj1 - (2.0 * B + (6.0 * C + 12.0 * D * rj) * rj) * c3 * cj +
           (6.0 * C + 24.0 * D * rj) * c4 * sj - (6.0 * C + 24.0 * D * rj1) * c4 * sj1 + 24.0 * D * c5 * (cj - cj1);
  }
  const double fi = block_sum(acc, sh);
  if (threadIdx.x == 0) {
    double s, c;
    sincos(q * a.rc, &s, &c);
    const double vp = a.f0 * c1 * (s * c1 - a.rc * c);
    vpp[i] = (vp + fi) * c1 * qpi;
  }
}

struct QArgs {
  const double *pp, *a, *b, *c, *d;
  int np;
  size_t H;
};

// Vq = real(cmplx(spline(|p|))) (findi + cubic, DFT4He3d.f90:527-536)
__global__ void k_vq_eval(QArgs q, const double *__restrict__ pmod, double *vq) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < q.H; t += (size_t)gridDim.x * blockDim.x) {
    const double x = pmod[t];
    int k;  // 0-based interval
    if (x > q.pp[q.np - 1]) {
      k = q.np - 2;
    } else if (x < q.pp[0]) {
      k = 0;
    } else {
      int lo = 0, hi = q.np - 1;
      do {
        const int it = (lo + hi) / 2;
        if (x > q.pp[it]) lo = it;
        if (x <= q.pp[it]) hi = it;
      } while (hi - lo > 1);
      k = lo;
    }
    const double v = q.a[k] + x * (q.b[k] + x * (q.c[k] + x * q.d[k]));
    vq[t] = (double)(float)v;
  }
}

template <typename T>
struct DevBuf {
  T *p = nullptr;
  ~DevBuf() { cudaFree(p); }
};

static int build_vq(Handle *h, double qmax, double hq) {
  const he4_params &P = h->p;
  const int N = 100001;
  const double r_max = 2000.0, eps = 1e-8, small_q = 1e-2, dr = 0.5;
  const int np = (int)(qmax / hq + 1.5);
  if (np < 4) {
    set_error("Vq table needs at least 4 q points (nq=%d)", P.nq);
    return HE4_E_ARG;
  }
  const double X1 = P.r_cutoff + eps, XN = r_max;
  const double hr = (XN - X1) / (N - 1);
  // V at the spline nodes, then at the six points of the end curvatures
  std::vector<double> x(N + 6), y(N + 6), A(N), B(N), C(N), D(N);
  for (int i = 0; i < N; i++) x[i] = (double)i * hr + X1;
  const double ends[6] = {X1, X1 + dr, X1 + dr + dr, XN - dr, XN, XN + dr};
  for (int i = 0; i < 6; i++) x[N + i] = ends[i];
  DevBuf<double> dx, dA, dB, dC, dD, dv;
  const size_t bytes = sizeof(double) * N;
  HE4_CUDA_TRY(cudaMalloc(&dx.p, sizeof(double) * (N + 6)));
  if (P.pot_kind == HE4_POT_RTABLE) {
    RTable tab;
    HE4_TRY(rtable_build(P, &tab));
    for (int i = 0; i < N + 6; i++) y[i] = pair_pot(P, &tab, x[i]);
  } else {
    // Select_Pot on the device
    DevBuf<double> dy;
    HE4_CUDA_TRY(cudaMalloc(&dy.p, sizeof(double) * (N + 6)));
    HE4_CUDA_TRY(cudaMemcpyAsync(dx.p, x.data(), sizeof(double) * (N + 6), cudaMemcpyHostToDevice, h->stream));
    const PotArgs pa{P.pot_kind, P.r_cutoff, P.umax, P.morse_d, P.morse_alpha, P.morse_re};
    k_pair_pot<<<(N + 6 + 255) / 256, 256, 0, h->stream>>>(dx.p, N + 6, pa, dy.p);
    HE4_LAUNCHED(h);
    HE4_CUDA_TRY(cudaMemcpyAsync(y.data(), dy.p, sizeof(double) * (N + 6), cudaMemcpyDeviceToHost, h->stream));
    HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  const double *ye = y.data() + N;
  const double S1 = (ye[0] - 2.0 * ye[1] + ye[2]) / (dr * dr);
  const double Sn = (ye[3] - 2.0 * ye[4] + ye[5]) / (dr * dr);
  HE4_TRY(spline_global(x.data(), y.data(), A.data(), B.data(), C.data(), D.data(), S1, Sn, N));
  HE4_CUDA_TRY(cudaMalloc(&dA.p, bytes));
  HE4_CUDA_TRY(cudaMalloc(&dB.p, bytes));
  HE4_CUDA_TRY(cudaMalloc(&dC.p, bytes));
  HE4_CUDA_TRY(cudaMalloc(&dD.p, bytes));
  HE4_CUDA_TRY(cudaMalloc(&dv.p, sizeof(double) * np));
  HE4_CUDA_TRY(cudaMemcpyAsync(dx.p, x.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dA.p, A.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dB.p, B.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dC.p, C.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dD.p, D.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  FtArgs fa{dx.p, dA.p, dB.p, dC.p, dD.p, N - 1, hq, P.r_cutoff, (P.pot_kind == HE4_POT_NULL) ? 0.0 : P.umax};
  k_ft_radial<<<np, 256, 0, h->stream>>>(fa, dv.p);
  HE4_LAUNCHED(h);
  std::vector<double> vpp(np), pp(np);
  HE4_CUDA_TRY(cudaMemcpyAsync(vpp.data(), dv.p, sizeof(double) * np, cudaMemcpyDeviceToHost, h->stream));
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (int i = 0; i < np; i++) pp[i] = (double)i * hq;
  // small-q refit (FT_V_spline.f90:230-264)
  {
    double xs[4], ys[4], as[4], bs[4], cs[4], ds[4];
    int iaux = 0;
    xs[0] = 0.0;
    ys[0] = vpp[0];
    for (int i = 1; i < np && iaux < 3; i++)
      if (pp[i] > small_q) {
        iaux++;
        xs[iaux] = pp[i];
        ys[iaux] = vpp[i];
      }
    if (iaux == 3 && spline_global(xs, ys, as, bs, cs, ds, 0.0, 0.0, 4) == HE4_OK) {
      for (int i = 1; i < np; i++) {
        if (pp[i] <= small_q)
          vpp[i] = as[0] + pp[i] * (bs[0] + pp[i] * (cs[0] + pp[i] * ds[0]));
        else
          break;
      }
    }
  }
  std::vector<double> qa(np), qb(np), qc(np), qd(np);
  HE4_TRY(spline_global(pp.data(), vpp.data(), qa.data(), qb.data(), qc.data(), qd.data(), 0.0, 0.0, np));
  DevBuf<double> dq;
  HE4_CUDA_TRY(cudaMalloc(&dq.p, sizeof(double) * 5 * np));
  HE4_CUDA_TRY(cudaMemcpyAsync(dq.p, pp.data(), sizeof(double) * np, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dq.p + np, qa.data(), sizeof(double) * np, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dq.p + 2 * np, qb.data(), sizeof(double) * np, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dq.p + 3 * np, qc.data(), sizeof(double) * np, cudaMemcpyHostToDevice, h->stream));
  HE4_CUDA_TRY(cudaMemcpyAsync(dq.p + 4 * np, qd.data(), sizeof(double) * np, cudaMemcpyHostToDevice, h->stream));
  QArgs qa_{dq.p, dq.p + np, dq.p + 2 * np, dq.p + 3 * np, dq.p + 4 * np, np, h->H};
  k_vq_eval<<<1024, 256, 0, h->stream>>>(qa_, h->pmod, h->vq);
  HE4_LAUNCHED(h);
  HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HE4_OK;
}

static double bforce_ot(double eps, double sigma, double hc) {
  const double pi4 = 4.0 * kPi, eps4 = 4.0 * eps;
  const double s6 = pow(sigma, 6), s12 = s6 * s6;
  return pi4 * eps4 * s12 / (9.0 * pow(hc, 9)) - pi4 * eps4 * s6 / (3.0 * pow(hc, 3));
}

__global__ void k_narrow(const double *__restrict__ in, float *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void k_widen(const float *__restrict__ in, double *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

static unsigned cast_grid(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

int narrow(Handle *h, const double *in, float *out, size_t n) {
  k_narrow<<<cast_grid(n), 256, 0, h->stream>>>(in, out, n);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int widen(Handle *h, const float *in, double *out, size_t n) {
  k_widen<<<cast_grid(n), 256, 0, h->stream>>>(in, out, n);
  HE4_LAUNCHED(h);
  return HE4_OK;
}

int setup_kernels(Handle *h) {
  const he4_params &P = h->p;
  const int nx = h->nx, ny = h->ny, nz = h->nz;
  // p grids (DFT4He3d.f90:321-342)
  const double hpx = 1.0 / (nx * h->hx), hpy = 1.0 / (ny * h->hy), hpz = 1.0 / (nz * h->hz);
  const double pmx = 1.0 / (2.0 * h->hx), pmy = 1.0 / (2.0 * h->hy), pmz = 1.0 / (2.0 * h->hz);
  std::vector<double> pall(nx + ny + nz);
  for (int i = 1; i <= nx; i++) pall[i - 1] = (i <= nx / 2 + 1) ? hpx * (i - 1) : -pmx + hpx * (i - (nx / 2 + 1));
  for (int i = 1; i <= ny; i++) pall[nx + i - 1] = (i <= ny / 2 + 1) ? hpy * (i - 1) : -pmy + hpy * (i - (ny / 2 + 1));
  for (int i = 1; i <= nz; i++)
    pall[nx + ny + i - 1] = (i <= nz / 2 + 1) ? hpz * (i - 1) : -pmz + hpz * (i - (nz / 2 + 1));
  DevBuf<double> dp;
  HE4_CUDA_TRY(cudaMalloc(&dp.p, sizeof(double) * pall.size()));
  HE4_CUDA_TRY(cudaMemcpyAsync(dp.p, pall.data(), sizeof(double) * pall.size(), cudaMemcpyHostToDevice, h->stream));
  KArgs ka{h->nxh, ny, nz, dp.p, dp.p + nx, dp.p + nx + ny, P.eps4, P.sigma4, P.h4, P.l_alfs,
           bforce_ot(P.eps4, P.sigma4, P.h4)};
  k_kspace<<<1024, 256, 0, h->stream>>>(ka, h->pmod, h->wcgk, h->fvlj4, h->kalfs);
  HE4_LAUNCHED(h);
  // Vq
  if (P.pot_kind == HE4_POT_TABLE) {
    if (!P.vq_table) {
      set_error("pot_kind=HE4_POT_TABLE needs vq_table");
      return HE4_E_ARG;
    }
    HE4_CUDA_TRY(cudaMemcpyAsync(h->vq, P.vq_table, sizeof(double) * h->H, cudaMemcpyHostToDevice, h->stream));
  } else {
    const double qmax = sqrt(pmx * pmx + pmy * pmy + pmz * pmz);
    const int nq = P.nq > 1 ? P.nq : 1000;
    HE4_TRY(build_vq(h, qmax, qmax / (nq - 1)));
  }
  // stencils (Init_deriv_p, Sto = 1/h**id)
  h->st.m = P.npd / 2;
  const double hh[3] = {h->hx, h->hy, h->hz};
  double w[25];
  for (int ax = 0; ax < 3; ax++) {
    HE4_TRY(fd_weights(P.npd, 1, w));
    double sto = 1.0 / hh[ax];
    for (int j = 0; j < 25; j++) h->st.w1[ax][j] = (j < P.npd) ? w[j] * sto : 0.0;
    HE4_TRY(fd_weights(P.npd, 2, w));
    sto = 1.0 / (hh[ax] * hh[ax]);
    for (int j = 0; j < 25; j++) h->st.w2[ax][j] = (j < P.npd) ? w[j] * sto : 0.0;
  }
  // icon=12: the one-sided rows of the first m points (rows 1..ko2 that
  // Redef leaves untouched, redef.f:133-150), scaled as the centre rows
  if (P.icon == 12) {
    const int m = h->st.m, K = P.npd;
    std::vector<double> r1((size_t)K * K), r2((size_t)K * K), lo((size_t)2 * 3 * m * K);
    HE4_TRY(fd_rows(K, 1, r1.data()));
    HE4_TRY(fd_rows(K, 2, r2.data()));
    for (int ax = 0; ax < 3; ax++) {
      const double s1 = 1.0 / hh[ax], s2 = 1.0 / (hh[ax] * hh[ax]);
      for (int c = 0; c < m; c++)
        for (int t = 0; t < K; t++) {
          lo[((size_t)(0 * 3 + ax) * m + c) * K + t] = r1[(size_t)c * K + t] * s1;
          lo[((size_t)(1 * 3 + ax) * m + c) * K + t] = r2[(size_t)c * K + t] * s2;
        }
    }
    HE4_CUDA_TRY(cudaMalloc((void **)&h->st_lo, sizeof(double) * lo.size()));
    HE4_CUDA_TRY(cudaMemcpy(h->st_lo, lo.data(), sizeof(double) * lo.size(), cudaMemcpyHostToDevice));
    h->st.lo = h->st_lo;
  }
  // imaginary part of the first-derivative symbol per axis:
  // D(k) = i * 2 sum_{t=1..m} w_t sin(2 pi t k / n)
  {
    std::vector<double> ds(nx + ny + nz);
    const int n3[3] = {nx, ny, nz};
    int off = 0;
    for (int ax = 0; ax < 3; ax++) {
      for (int k = 0; k < n3[ax]; k++) {
        long double acc = 0.0L;
        for (int t = 1; t <= h->st.m; t++)
          acc += (long double)h->st.w1[ax][h->st.m + t] *
                 sinl(2.0L * 3.14159265358979323846264338327950288L * (long double)t * k / n3[ax]);
        ds[off + k] = (double)(2.0L * acc);
      }
      off += n3[ax];
    }
    HE4_CUDA_TRY(cudaMemcpyAsync(h->dsym, ds.data(), sizeof(double) * ds.size(), cudaMemcpyHostToDevice, h->stream));
    if (h->fp32) {
      std::vector<float> ds32(ds.size());
      for (size_t i = 0; i < ds.size(); i++) ds32[i] = (float)ds[i];
      HE4_CUDA_TRY(cudaMemcpyAsync(h->dsym32, ds32.data(), sizeof(float) * ds32.size(), cudaMemcpyHostToDevice,
                                   h->stream));
      HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
  }
  // FP32 copies of the k-space kernels for the FP32-convolution form
  if (h->fp32) {
    const double *src[4] = {h->wcgk, h->fvlj4, h->kalfs, h->vq};
    for (int i = 0; i < 4; i++) HE4_TRY(narrow(h, src[i], h->k32[i], h->H));
  }
  // timec (DFT4He3d.f90:773-782), real part rounded to single precision
  {
    std::vector<double> tc(nz);
    for (int k = 0; k < nz; k++) {
      const double z = -P.zmax + h->hz * k;
      tc[k] = (double)(float)(P.lambdah * (1.0 + tanh((z - P.tzmean) / P.tzsurf)));
    }
    HE4_CUDA_TRY(cudaMemcpyAsync(h->timec_re, tc.data(), sizeof(double) * nz, cudaMemcpyHostToDevice, h->stream));
    HE4_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  return HE4_OK;
}

}  // namespace he4

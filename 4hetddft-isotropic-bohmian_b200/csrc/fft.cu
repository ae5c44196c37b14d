// fft.cu -- batched 3D real FFTs for the convolutions of the mean field.
//
// Replaces the FFTW plans and their executions (fft.f90:43-65, 79-207).
// Layout: real grids [nz][ny][nx]; half spectra [nz][ny][nx/2+1] (the FFTW
// r2c layout of the reference).  Forward transforms are unnormalised; the
// reference's backward scaling by renor = 1/N (fft.f90:130,138,...) is folded
// into the coefficient of the k-space multiply of the z pass.
//
// A 3D transform is three passes over HBM:
//   x pass  (R2C / C2R): two real rows packed into one complex pencil,
//   y pass  (complex), and
//   z pass  (complex) fused with the k-space kernel multiply and the inverse
//           z transform: FFT_z -> coef*K(k) (*i*D(k)) -> IFFT_z in one launch.
// Each CTA stages a tile of pencils in shared memory and runs a mixed-radix
// (2/3/4/5) Stockham transform between two shared buffers; pencils of one
// tile are contiguous in x so every global access is a coalesced segment.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include <cuda_pipeline.h>

#include "common.cuh"
#include "fft_passes.cuh"

namespace he4 {

static constexpr double kC3S = 0.86602540378443864676372317075293618;   // sin(2pi/3)
static constexpr double kC5C1 = 0.30901699437494742410229341718281906;  // cos(2pi/5)
static constexpr double kC5C2 = -0.80901699437494742410229341718281906; // cos(4pi/5)
static constexpr double kC5S1 = 0.95105651629515357211643933337938214;  // sin(2pi/5)
static constexpr double kC5S2 = 0.58778525229247312916870595463907277;  // sin(4pi/5)

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// small DFTs (forward: exp(-2 pi i jk/R); inverse: conjugate roots)
// ---------------------------------------------------------------------------
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  static __device__ __forceinline__ void run(double2 *u) {
    double2 t = u[0];
    u[0] = cadd(t, u[1]);
    u[1] = csub(t, u[1]);
  }
};

template <bool INV>
struct Dft<4, INV> {
  static __device__ __forceinline__ void run(double2 *u) {
    double2 a = cadd(u[0], u[2]), b = csub(u[0], u[2]);
    double2 c = cadd(u[1], u[3]), d = cmuli<INV>(csub(u[1], u[3]));
    u[0] = cadd(a, c);
    u[2] = csub(a, c);
    u[1] = cadd(b, d);
    u[3] = csub(b, d);
  }
};

template <bool INV>
struct Dft<3, INV> {
  static __device__ __forceinline__ void run(double2 *u) {
    double2 t1 = cadd(u[1], u[2]);
    double2 t2 = csub(u[0], cscale(t1, 0.5));
    double2 t3 = cscale(cmuli<INV>(csub(u[1], u[2])), kC3S);
    u[0] = cadd(u[0], t1);
    u[1] = cadd(t2, t3);
    u[2] = csub(t2, t3);
  }
};

template <bool INV>
struct Dft<5, INV> {
  static __device__ __forceinline__ void run(double2 *u) {
    double2 a1 = cadd(u[1], u[4]), b1 = csub(u[1], u[4]);
    double2 a2 = cadd(u[2], u[3]), b2 = csub(u[2], u[3]);
    double2 r1 = cadd(u[0], cadd(cscale(a1, kC5C1), cscale(a2, kC5C2)));
    double2 r2 = cadd(u[0], cadd(cscale(a1, kC5C2), cscale(a2, kC5C1)));
    double2 s1 = cmuli<INV>(cadd(cscale(b1, kC5S1), cscale(b2, kC5S2)));
    double2 s2 = cmuli<INV>(csub(cscale(b1, kC5S2), cscale(b2, kC5S1)));
    u[0] = cadd(u[0], cadd(a1, a2));
    u[1] = cadd(r1, s1);
    u[4] = csub(r1, s1);
    u[2] = cadd(r2, s2);
    u[3] = csub(r2, s2);
  }
};

// One Stockham stage on W pencils stored [n][ld] (pencil w at column w):
// butterfly i of pencil w reads x[i + j n/R], applies w_{pR}^{jk}
// (k = i mod p), runs the R-point DFT and writes y[(i/p) p R + k + j p].
template <int R, bool INV>
__device__ __forceinline__ void stage(const double2 *__restrict__ src, double2 *__restrict__ dst, int n,
                                      int p, int W, int ld, const double2 *__restrict__ tw) {
  const int m = n / R, tstep = n / (p * R);
  const int nb = m * W;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int w = b % W, i = b / W, k = i % p;
    double2 u[R];
#pragma unroll
    for (int j = 0; j < R; j++) u[j] = src[(i + j * m) * ld + w];
    if (k) {
#pragma unroll
      for (int j = 1; j < R; j++) {
        double2 t = tw[j * k * tstep];
        if (INV) t.y = -t.y;
        u[j] = cmul(u[j], t);
      }
    }
    Dft<R, INV>::run(u);
    const int j0 = (i / p) * p * R + k;
#pragma unroll
    for (int j = 0; j < R; j++) dst[(j0 + j * p) * ld + w] = u[j];
  }
}

// Full transform of W pencils; a holds the input, b is scratch.  Returns the
// buffer holding the natural-order result.
template <bool INV>
__device__ double2 *fft_smem(double2 *a, double2 *b, const AxisPlan &P, int W, int ld,
                             const double2 *__restrict__ tw) {
  int p = 1;
  for (int s = 0; s < P.nst; s++) {
    const int R = P.radix[s];
    switch (R) {
      case 4: stage<4, INV>(a, b, P.n, p, W, ld, tw); break;
      case 2: stage<2, INV>(a, b, P.n, p, W, ld, tw); break;
      case 3: stage<3, INV>(a, b, P.n, p, W, ld, tw); break;
      default: stage<5, INV>(a, b, P.n, p, W, ld, tw); break;
    }
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
    p *= R;
  }
  return a;
}

__device__ __forceinline__ void load_tw(double2 *s_tw, const AxisPlan &P) {
  for (int t = threadIdx.x; t < P.n; t += blockDim.x) s_tw[t] = P.tw[t];
}

// ---------------------------------------------------------------------------
// x pass
// ---------------------------------------------------------------------------
constexpr int kMaxBatch = 8;

struct XArgs {
  AxisPlan ax;
  int nxh, P;
  long nrow;
  double scale;
  const double *rin[kMaxBatch];
  double2 *cout[kMaxBatch];
  const double2 *cin[kMaxBatch];
  double *rout[kMaxBatch];
};

__global__ void __launch_bounds__(kThreads) k_fft_x_r2c(XArgs a) {
  extern __shared__ double2 smem[];
  const int n = a.ax.n, P = a.P, ld = P + 1, nxh = a.nxh;
  double2 *b0 = smem, *b1 = smem + n * ld, *tw = smem + 2 * n * ld;
  load_tw(tw, a.ax);
  const double *in = a.rin[blockIdx.y];
  double2 *out = a.cout[blockIdx.y];
  const long row0 = (long)blockIdx.x * 2 * P;
  for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
    const int q = e / n, x = e - q * n;
    const long ra = row0 + 2 * q, rb = ra + 1;
    double va = (ra < a.nrow) ? in[ra * n + x] : 0.0;
    double vb = (rb < a.nrow) ? in[rb * n + x] : 0.0;
    b0[x * ld + q] = make_double2(va, vb);
  }
  __syncthreads();
  double2 *res = fft_smem<false>(b0, b1, a.ax, P, ld, tw);
  for (int e = threadIdx.x; e < nxh * P; e += blockDim.x) {
    const int q = e / nxh, k = e - q * nxh;
    const long ra = row0 + 2 * q, rb = ra + 1;
    const double2 zk = res[k * ld + q];
    const double2 zm = cconj(res[((n - k) % n) * ld + q]);
    const double2 A = cscale(cadd(zk, zm), 0.5);
    const double2 d = cscale(csub(zk, zm), 0.5);
    if (ra < a.nrow) out[ra * nxh + k] = A;
    if (rb < a.nrow) out[rb * nxh + k] = make_double2(d.y, -d.x);
  }
}

__global__ void __launch_bounds__(kThreads) k_fft_x_c2r(XArgs a) {
  extern __shared__ double2 smem[];
  const int n = a.ax.n, P = a.P, ld = P + 1, nxh = a.nxh;
  double2 *b0 = smem, *b1 = smem + n * ld, *tw = smem + 2 * n * ld;
  load_tw(tw, a.ax);
  const double2 *in = a.cin[blockIdx.y];
  double *out = a.rout[blockIdx.y];
  const long row0 = (long)blockIdx.x * 2 * P;
  for (int e = threadIdx.x; e < nxh * P; e += blockDim.x) {
    const int q = e / nxh, k = e - q * nxh;
    const long ra = row0 + 2 * q, rb = ra + 1;
    double2 X = (ra < a.nrow) ? in[ra * nxh + k] : make_double2(0.0, 0.0);
    double2 Y = (rb < a.nrow) ? in[rb * nxh + k] : make_double2(0.0, 0.0);
    if (k == 0 || 2 * k == n) {  // DC / Nyquist of a real transform: drop Im
      X.y = 0.0;
      Y.y = 0.0;
    }
    b0[k * ld + q] = make_double2(X.x - Y.y, X.y + Y.x);  // X + iY
    if (k > 0 && n - k >= nxh) b0[(n - k) * ld + q] = make_double2(X.x + Y.y, Y.x - X.y);  // conj(X) + i conj(Y)
  }
  __syncthreads();
  double2 *res = fft_smem<true>(b0, b1, a.ax, P, ld, tw);
  const double sc = a.scale;
  for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
    const int q = e / n, x = e - q * n;
    const long ra = row0 + 2 * q, rb = ra + 1;
    const double2 v = res[x * ld + q];
    if (ra < a.nrow) out[ra * n + x] = v.x * sc;
    if (rb < a.nrow) out[rb * n + x] = v.y * sc;
  }
}

struct YArgs {
  AxisPlan ay;
  PencilMap map;
  long sf;  // element stride along the transformed axis
  double2 *buf[kMaxBatch];
};

template <bool INV>
__global__ void __launch_bounds__(kThreads) k_fft_y(YArgs a) {
  extern __shared__ double2 smem[];
  const int n = a.ay.n, W = a.map.W;
  double2 *b0 = smem, *b1 = smem + n * W, *tw = smem + 2 * n * W;
  long *offs = reinterpret_cast<long *>(tw + n);
  load_tw(tw, a.ay);
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    int kx, o;
    offs[w] = pencil_offset(a.map, (long)blockIdx.x * W + w, &kx, &o);
  }
  __syncthreads();
  double2 *data = a.buf[blockIdx.y];
  for (int e = threadIdx.x; e < n * W; e += blockDim.x) {
    const int w = e % W, j = e / W;
    const long off = offs[w];
    b0[j * W + w] = (off >= 0) ? data[off + j * a.sf] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2 *res = fft_smem<INV>(b0, b1, a.ay, W, W, tw);
  for (int e = threadIdx.x; e < n * W; e += blockDim.x) {
    const int w = e % W, j = e / W;
    const long off = offs[w];
    if (off >= 0) data[off + j * a.sf] = res[j * W + w];
  }
}

struct ZArgs {
  AxisPlan az;
  PencilMap map;
  long sf;
  int nx, ny, nz;
  const double *dsym;  // [nx | ny | nz]
  ZOp ops[kMaxBatch];
};

__global__ void __launch_bounds__(kThreads) k_fft_z_conv(ZArgs a) {
  extern __shared__ double2 smem[];
  const int n = a.az.n, W = a.map.W;
  double2 *b0 = smem, *b1 = smem + n * W, *tw = smem + 2 * n * W;
  long *offs = reinterpret_cast<long *>(tw + n);
  int *kxs = reinterpret_cast<int *>(offs + W);
  int *kys = kxs + W;
  load_tw(tw, a.az);
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    int kx = 0, o = 0;
    offs[w] = pencil_offset(a.map, (long)blockIdx.y * W + w, &kx, &o);
    kxs[w] = kx;
    kys[w] = o;
  }
  __syncthreads();
  const ZOp op = a.ops[blockIdx.x];
  for (int e = threadIdx.x; e < n * W; e += blockDim.x) {
    const int w = e % W, j = e / W;
    const long off = offs[w];
    b0[j * W + w] = (off >= 0) ? op.in[off + j * a.sf] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (op.mode != 0) {  // plain forward or inverse transform along z
    double2 *r = (op.mode == 1) ? fft_smem<false>(b0, b1, a.az, W, W, tw) : fft_smem<true>(b0, b1, a.az, W, W, tw);
    for (int e = threadIdx.x; e < n * W; e += blockDim.x) {
      const int w = e % W, j = e / W;
      const long off = offs[w];
      if (off >= 0) op.out[off + j * a.sf] = r[j * W + w];
    }
    return;
  }
  double2 *res = fft_smem<false>(b0, b1, a.az, W, W, tw);
  double2 *wk = (res == b0) ? b1 : b0;
  for (int e = threadIdx.x; e < n * W; e += blockDim.x) {
    const int w = e % W, j = e / W;
    const long off = offs[w];
    double c = op.coef;
    if (off >= 0 && op.kern) c *= op.kern[off + j * a.sf];
    double2 v = cscale(res[j * W + w], c);
    if (op.dsym_axis >= 0) {
      double ds;
      if (op.dsym_axis == 0) ds = a.dsym[kxs[w]];
      else if (op.dsym_axis == 1) ds = a.dsym[a.nx + kys[w]];
      else ds = a.dsym[a.nx + a.ny + j];
      v = make_double2(-v.y * ds, v.x * ds);  // times i*ds
    }
    wk[j * W + w] = v;
  }
  __syncthreads();
  double2 *out = (wk == b0) ? fft_smem<true>(b0, b1, a.az, W, W, tw) : fft_smem<true>(b1, b0, a.az, W, W, tw);
  for (int e = threadIdx.x; e < n * W; e += blockDim.x) {
    const int w = e % W, j = e / W;
    const long off = offs[w];
    if (off >= 0) op.out[off + j * a.sf] = out[j * W + w];
  }
}


// ---------------------------------------------------------------------------
// twiddle tables
// ---------------------------------------------------------------------------
static int axis_init(AxisPlan &A, int n) {
  A.n = n;
  A.nst = 0;
  int r = n;
  while (r % 4 == 0) { A.radix[A.nst++] = 4; r /= 4; }
  while (r % 2 == 0) { A.radix[A.nst++] = 2; r /= 2; }
  while (r % 3 == 0) { A.radix[A.nst++] = 3; r /= 3; }
  while (r % 5 == 0) { A.radix[A.nst++] = 5; r /= 5; }
  if (r != 1 || A.nst > kMaxStages) {
    set_error("FFT length %d is not of the form 2^a 3^b 5^c", n);
    return HE4_E_UNSUPPORTED;
  }
  double2 *tw = (double2 *)malloc(sizeof(double2) * n);
  float2 *tw32 = (float2 *)malloc(sizeof(float2) * n);
  for (int t = 0; t < n; t++) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
    const long double c = cosl(ang), s = sinl(ang);
    tw[t] = make_double2((double)c, (double)s);
    tw32[t] = make_float2((float)c, (float)s);
  }
  cudaError_t e = cudaMalloc(&A.tw, sizeof(double2) * n);
  if (e == cudaSuccess) e = cudaMemcpy(A.tw, tw, sizeof(double2) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&A.tw32, sizeof(float2) * n);
  if (e == cudaSuccess) e = cudaMemcpy(A.tw32, tw32, sizeof(float2) * n, cudaMemcpyHostToDevice);
  free(tw);
  free(tw32);
  if (e != cudaSuccess) {
    set_error("twiddle upload: %s", cudaGetErrorString(e));
    return HE4_E_CUDA;
  }
  return HE4_OK;
}

template <typename C2>
static const C2 *twid(const AxisPlan &A);
template <>
const double2 *twid<double2>(const AxisPlan &A) { return A.tw; }
template <>
const float2 *twid<float2>(const AxisPlan &A) { return A.tw32; }

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int tile_width(int n) {
  int w = 2048 / n;
  w = (w / 8) * 8;
  return std::max(8, std::min(32, w));
}

static size_t smem_x(const FftPlan &P) { return sizeof(double2) * (2 * (size_t)P.nx * (P.px + 1) + P.nx); }
static size_t smem_yz(int n, int W) {
  return sizeof(double2) * (2 * (size_t)n * W + n) + sizeof(long) * W + 2 * sizeof(int) * W;
}

// The dynamic shared memory limits of the generic-path kernels are set per
// device (a cudaFuncSetAttribute call applies to the current device only);
// per device they only ever grow, to the widest tiles any plan there uses.
// A maximum is recorded only after the attribute call succeeded, so a failed
// call is retried by the next plan.
static int generic_attrs(const FftPlan &P) {
  static std::mutex mu;
  static size_t max_x[kMaxDevices] = {0}, max_y[kMaxDevices] = {0}, max_z[kMaxDevices] = {0};
  int dev = 0;
  HE4_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal %d beyond the %d this library supports", dev, kMaxDevices);
    return HE4_E_ARG;
  }
  std::lock_guard<std::mutex> lock(mu);
  const size_t sx = smem_x(P), sy = smem_yz(P.ny, P.wy), sz = smem_yz(P.nz, P.wz);
  if (sx > max_x[dev]) {
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_fft_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx));
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx));
    max_x[dev] = sx;
  }
  if (sy > max_y[dev]) {
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_fft_y<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sy));
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_fft_y<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sy));
    max_y[dev] = sy;
  }
  if (sz > max_z[dev]) {
    HE4_CUDA_TRY(cudaFuncSetAttribute(k_fft_z_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz));
    max_z[dev] = sz;
  }
  return HE4_OK;
}

int fft_plan_init(FftPlan &P, int nx, int ny, int nz) {
  P.nx = nx;
  P.ny = ny;
  P.nz = nz;
  P.nxh = nx / 2 + 1;
  HE4_TRY(axis_init(P.ax, nx));
  HE4_TRY(axis_init(P.ay, ny));
  HE4_TRY(axis_init(P.az, nz));
  P.px = tile_width(nx);
  P.wy = tile_width(ny);
  P.wz = tile_width(nz);
  HE4_TRY(generic_attrs(P));
  const int ns[3] = {nx, ny, nz};
  for (int a = 0; a < 3; a++) {
    const int n = ns[a];
    P.n1[a] = reg_ok(n) ? reg_default_n1(n) : 0;
    if (!reg_ok(n)) continue;
    for (int n1 = 2; n1 <= 16; n1 *= 2) {
      if (!reg_n1_ok(n, n1)) continue;
      HE4_REG_SWITCH(n, n1, HE4_TRY((reg_attrs<NN, N1_, double2>())));
      HE4_REG_SWITCH(n, n1, HE4_TRY((reg_attrs<NN, N1_, float2>())));
    }
  }
  return HE4_OK;
}

// Tile shapes: t = {n1 x, n1 y, n1 z, px, wy, wz}.  n1 applies to register
// path axes (0 = default split), px / wy / wz (pencils per CTA, multiples of
// 8 in [8, 32]) to generic-path axes; entries for the other path are ignored.
int fft_set_tiles(FftPlan &P, const int *t) {
  const int ns[3] = {P.nx, P.ny, P.nz};
  int n1[3];
  for (int a = 0; a < 3; a++) {
    n1[a] = 0;
    if (!reg_ok(ns[a])) continue;
    n1[a] = t[a] ? t[a] : reg_default_n1(ns[a]);
    if (!reg_n1_ok(ns[a], n1[a])) {
      set_error("axis %d: no register FFT split %d x %d", a, n1[a], ns[a] / n1[a]);
      return HE4_E_ARG;
    }
  }
  FftPlan Q = P;
  Q.px = reg_ok(P.nx) ? P.px : t[3];
  Q.wy = reg_ok(P.ny) ? P.wy : t[4];
  Q.wz = reg_ok(P.nz) ? P.wz : t[5];
  const int ws[3] = {Q.px, Q.wy, Q.wz};
  for (int a = 0; a < 3; a++)
    if (ws[a] < 8 || ws[a] > 32 || ws[a] % 8) {
      set_error("tile width %d is not a multiple of 8 in [8, 32]", ws[a]);
      return HE4_E_ARG;
    }
  const size_t lim = 200 * 1024;
  if (smem_x(Q) > lim || smem_yz(Q.ny, Q.wy) > lim || smem_yz(Q.nz, Q.wz) > lim) {
    set_error("tile widths need more than %zu bytes of shared memory", lim);
    return HE4_E_ARG;
  }
  HE4_TRY(generic_attrs(Q));
  for (int a = 0; a < 3; a++) Q.n1[a] = n1[a];
  P = Q;
  return HE4_OK;
}

void fft_get_tiles(const FftPlan &P, int *t) {
  for (int a = 0; a < 3; a++) t[a] = P.n1[a];
  t[3] = P.px;
  t[4] = P.wy;
  t[5] = P.wz;
}

void fft_plan_free(FftPlan &P) {
  AxisPlan *axes[3] = {&P.ax, &P.ay, &P.az};
  for (AxisPlan *A : axes) {
    cudaFree(A->tw);
    cudaFree(A->tw32);
    A->tw = nullptr;
    A->tw32 = nullptr;
  }
}

// register-path x pass in the spectrum type C2; real grids FP64, or float
// (ld.real32 / out32) in the merged evaluation of the FP32-convolution form
template <typename C2>
static int x_pass_reg(Handle *h, int nb, const void *const *rin, double2 *const *cout, double2 *const *cin,
                      void *const *rout, bool inverse, const BoxPair *box, const XLoad &ld, bool out32) {
  const FftPlan &P = h->fft;
  const long nrow = (long)P.ny * P.nz;
  XRegArgs<C2> a{};
  a.nxh = P.nxh;
  a.nrow = nrow;
  a.scale = 1.0;
  a.tw = twid<C2>(P.ax);
  a.box = inverse ? box : nullptr;
  a.ny = P.ny;
  a.nz = P.nz;
  a.ld = ld;
  for (int i = 0; i < nb; i++) {
    if (inverse) {
      a.cin[i] = reinterpret_cast<const C2 *>(cin[i]);
      a.rout[i] = rout[i];
    } else {
      a.rin[i] = rin[i];
      a.cout[i] = reinterpret_cast<C2 *>(cout[i]);
    }
  }
  HE4_REG_SWITCH(P.nx, P.n1[0], {
    constexpr int Pp = kRegThreads / N1_;
    dim3 grid((unsigned)((nrow + 2 * Pp - 1) / (2 * Pp)), nb);
    const size_t sm = smem_x_reg<NN, N1_, C2>();
    if constexpr (sizeof(C2) == 8) {
      if (inverse && out32)
        k_xc2r_reg<NN, N1_, C2, float><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (inverse)
        k_xc2r_reg<NN, N1_, C2><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.real32 && ld.op == XLOAD_ALFA)
        k_xr2c_reg<NN, N1_, C2, XLOAD_ALFA, float><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.real32 && ld.op == XLOAD_CORR)
        k_xr2c_reg<NN, N1_, C2, XLOAD_CORR, float><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.real32)
        k_xr2c_reg<NN, N1_, C2, XLOAD_PLAIN, float><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.op == XLOAD_ALFA)
        k_xr2c_reg<NN, N1_, C2, XLOAD_ALFA><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.op == XLOAD_CORR)
        k_xr2c_reg<NN, N1_, C2, XLOAD_CORR><<<grid, kRegThreads, sm, h->stream>>>(a);
      else
        k_xr2c_reg<NN, N1_, C2><<<grid, kRegThreads, sm, h->stream>>>(a);
    } else {
      if (out32 || ld.real32) {
        set_error("float real grids need the FP32-convolution form");
        return HE4_E_ARG;
      }
      if (inverse)
        k_xc2r_reg<NN, N1_, C2><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.op == XLOAD_ALFA)
        k_xr2c_reg<NN, N1_, C2, XLOAD_ALFA><<<grid, kRegThreads, sm, h->stream>>>(a);
      else if (ld.op == XLOAD_CORR)
        k_xr2c_reg<NN, N1_, C2, XLOAD_CORR><<<grid, kRegThreads, sm, h->stream>>>(a);
      else
        k_xr2c_reg<NN, N1_, C2><<<grid, kRegThreads, sm, h->stream>>>(a);
    }
  });
  HE4_LAUNCHED(h);
  return HE4_OK;
}

// box (C2R only, register path): restrict to the rows of the force box
// rin / rout: double grids, or float grids when ld.real32 (R2C) / out32 (C2R)
static int x_pass_v(Handle *h, int n, const void *const *rin, double2 *const *cout, double2 *const *cin,
                    void *const *rout, bool inverse, const BoxPair *box, const XLoad &ld, bool out32) {
  const FftPlan &P = h->fft;
  const long nrow = (long)P.ny * P.nz;
  for (int b0 = 0; b0 < n; b0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, n - b0);
    if (reg_ok(P.nx)) {
      const void *const *ri = rin ? rin + b0 : nullptr;
      double2 *const *co = cout ? cout + b0 : nullptr;
      double2 *const *ci = cin ? cin + b0 : nullptr;
      void *const *ro = rout ? rout + b0 : nullptr;
      if (h->fp32)
        HE4_TRY(x_pass_reg<float2>(h, nb, ri, co, ci, ro, inverse, box, ld, out32));
      else
        HE4_TRY(x_pass_reg<double2>(h, nb, ri, co, ci, ro, inverse, box, ld, out32));
      continue;
    }
    if (ld.op != XLOAD_PLAIN || ld.real32 || out32) {
      set_error("formed-on-load x pass needs a register-path axis length");
      return HE4_E_UNSUPPORTED;
    }
    if (h->fp32) {
      set_error("FP32 spectra need register-path axis lengths");
      return HE4_E_UNSUPPORTED;
    }
    XArgs a{};
    a.ax = P.ax;
    a.nxh = P.nxh;
    a.P = P.px;
    a.nrow = nrow;
    a.scale = 1.0;
    for (int i = 0; i < nb; i++) {
      if (inverse) {
        a.cin[i] = cin[b0 + i];
        a.rout[i] = static_cast<double *>(rout[b0 + i]);
      } else {
        a.rin[i] = static_cast<const double *>(rin[b0 + i]);
        a.cout[i] = cout[b0 + i];
      }
    }
    dim3 grid((unsigned)((nrow + 2 * P.px - 1) / (2 * P.px)), nb);
    if (inverse)
      k_fft_x_c2r<<<grid, kThreads, smem_x(P), h->stream>>>(a);
    else
      k_fft_x_r2c<<<grid, kThreads, smem_x(P), h->stream>>>(a);
    HE4_LAUNCHED(h);
  }
  return HE4_OK;
}

static int x_pass(Handle *h, int n, const double *const *rin, double2 *const *cout, double2 *const *cin,
                  double *const *rout, bool inverse, const BoxPair *box = nullptr) {
  const void *ri[64];
  void *ro[64];
  if (n > 64) {
    set_error("x pass of more than 64 fields");
    return HE4_E_ARG;
  }
  for (int i = 0; i < n; i++) {
    ri[i] = rin ? rin[i] : nullptr;
    ro[i] = rout ? rout[i] : nullptr;
  }
  return x_pass_v(h, n, rin ? ri : nullptr, cout, cin, rout ? ro : nullptr, inverse, box, XLoad(), false);
}

// register-path transform of strided pencils in the spectrum type C2
template <typename C2>
static int yz_reg(Handle *h, int nb, double2 *const *buf, int axis, bool inverse, const BoxPair *box) {
  const FftPlan &P = h->fft;
  const int len = (axis == 1) ? P.ny : P.nz;
  PencilMap map;
  map.nxh = P.nxh;
  map.nother = (axis == 1) ? P.nz : P.ny;
  map.so = (axis == 1) ? (long)P.ny * P.nxh : P.nxh;
  const long total = (long)P.nxh * map.nother;
  YRegArgs<C2> a{};
  a.sf = (axis == 1) ? (long)P.nxh : (long)P.ny * P.nxh;
  a.tw = twid<C2>((axis == 1) ? P.ay : P.az);
  a.box = (axis == 1) ? box : nullptr;
  a.nz = P.nz;
  for (int i = 0; i < nb; i++) a.buf[i] = reinterpret_cast<C2 *>(buf[i]);
  HE4_REG_SWITCH(len, P.n1[axis], {
    constexpr int W = kRegThreads / N1_;
    map.W = W;
    a.map = map;
    const long ntiles = (total + W - 1) / W;
    // one wave of persistent CTAs: as many as fit on the SMs at once, per
    // instantiation and device; handles on other host threads may read it
    static std::atomic<int> per_sm[kMaxDevices][2];
    const int dev = h->dev;
    int ps = per_sm[dev][inverse ? 1 : 0].load(std::memory_order_relaxed);
    if (ps == 0) {
      int nsm = 0, occ = 0;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (inverse)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_yz_pipe<NN, N1_, true, C2>, kRegThreads,
                                                      smem_yz_reg<NN, N1_, C2>());
      else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_yz_pipe<NN, N1_, false, C2>, kRegThreads,
                                                      smem_yz_reg<NN, N1_, C2>());
      ps = std::max(1, occ) * std::max(1, nsm);
      per_sm[dev][inverse ? 1 : 0].store(ps, std::memory_order_relaxed);
    }
    dim3 grid((unsigned)std::min<long>(ntiles, std::max(1, ps / nb)), nb);
    if (inverse)
      k_yz_pipe<NN, N1_, true, C2><<<grid, kRegThreads, smem_yz_reg<NN, N1_, C2>(), h->stream>>>(a);
    else
      k_yz_pipe<NN, N1_, false, C2><<<grid, kRegThreads, smem_yz_reg<NN, N1_, C2>(), h->stream>>>(a);
  });
  HE4_LAUNCHED(h);
  return HE4_OK;
}

// in-place complex transform of every pencil along y (axis 1) or z (axis 2);
// box (y pass, register path): only pencils whose z lies in the force box
static int strided_pass(Handle *h, int n, double2 *const *buf, int axis, bool inverse,
                        const BoxPair *box = nullptr) {
  const FftPlan &P = h->fft;
  const int len = (axis == 1) ? P.ny : P.nz;
  for (int b0 = 0; b0 < n; b0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, n - b0);
    if (reg_ok(len)) {
      if (h->fp32)
        HE4_TRY(yz_reg<float2>(h, nb, buf + b0, axis, inverse, box));
      else
        HE4_TRY(yz_reg<double2>(h, nb, buf + b0, axis, inverse, box));
      continue;
    }
    if (h->fp32) {
      set_error("FP32 spectra need register-path axis lengths");
      return HE4_E_UNSUPPORTED;
    }
    PencilMap map;
    map.nxh = P.nxh;
    map.nother = (axis == 1) ? P.nz : P.ny;
    map.so = (axis == 1) ? (long)P.ny * P.nxh : P.nxh;
    const long sf = (axis == 1) ? (long)P.nxh : (long)P.ny * P.nxh;
    const long total = (long)P.nxh * map.nother;
    if (axis == 1) {
      YArgs a{};
      a.ay = P.ay;
      map.W = P.wy;
      a.map = map;
      a.sf = sf;
      for (int i = 0; i < nb; i++) a.buf[i] = buf[b0 + i];
      dim3 grid((unsigned)((total + P.wy - 1) / P.wy), nb);
      if (inverse)
        k_fft_y<true><<<grid, kThreads, smem_yz(P.ny, P.wy), h->stream>>>(a);
      else
        k_fft_y<false><<<grid, kThreads, smem_yz(P.ny, P.wy), h->stream>>>(a);
      HE4_LAUNCHED(h);
    } else {
      for (int i = 0; i < nb; i++) {
        ZOp op{buf[b0 + i], buf[b0 + i], nullptr, 1.0, -1, inverse ? 2 : 1};
        HE4_TRY(fft_z_conv(h, 1, &op));
      }
    }
  }
  return HE4_OK;
}

int fft_y(Handle *h, int n, double2 *const *buf, bool inverse) { return strided_pass(h, n, buf, 1, inverse); }

int fft_r2c(Handle *h, int n, const double *const *in, double2 *const *out) {
  HE4_TRY(x_pass(h, n, in, out, nullptr, nullptr, false));
  HE4_TRY(fft_y(h, n, out, false));
  return HE4_OK;
}

int fft_r2c_load(Handle *h, int n, const void *const *in, double2 *const *out, const XLoad &ld) {
  HE4_TRY(x_pass_v(h, n, in, out, nullptr, nullptr, false, nullptr, ld, false));
  HE4_TRY(fft_y(h, n, out, false));
  return HE4_OK;
}

int fft_c2r_f32(Handle *h, int n, double2 *const *in, float *const *out) {
  void *ro[64];
  if (n > 64) {
    set_error("x pass of more than 64 fields");
    return HE4_E_ARG;
  }
  for (int i = 0; i < n; i++) ro[i] = out[i];
  HE4_TRY(fft_y(h, n, in, true));
  HE4_TRY(x_pass_v(h, n, nullptr, nullptr, in, ro, true, nullptr, XLoad(), true));
  return HE4_OK;
}

int fft_c2r(Handle *h, int n, double2 *const *in, double *const *out) {
  HE4_TRY(fft_y(h, n, in, true));
  HE4_TRY(x_pass(h, n, nullptr, nullptr, in, out, true));
  return HE4_OK;
}

int fft_c2r_box(Handle *h, int n, double2 *const *in, double *const *out) {
  HE4_TRY(strided_pass(h, n, in, 1, true, h->box));
  HE4_TRY(x_pass(h, n, nullptr, nullptr, in, out, true, h->box));
  return HE4_OK;
}

// kernel array of an operation in the spectrum type's real type
template <typename C2>
static const typename regfft::Re<C2>::type *kern_of(const Handle *h, const double *k);
template <>
const double *kern_of<double2>(const Handle *, const double *k) { return k; }
template <>
const float *kern_of<float2>(const Handle *h, const double *k) { return h->kern32(k); }

template <typename C2>
static const typename regfft::Re<C2>::type *dsym_of(const Handle *h);
template <>
const double *dsym_of<double2>(const Handle *h) { return h->dsym; }
template <>
const float *dsym_of<float2>(const Handle *h) { return h->dsym32; }

// register-path fused z pass: consecutive operations on the same input share
// one forward transform
template <typename C2>
static int zconv_reg(Handle *h, int n, const ZOp *ops) {
  const FftPlan &P = h->fft;
  ZGroupT<C2> groups[64];
  int ng = 0;
  for (int i = 0; i < n; i++) {
    const C2 *in = reinterpret_cast<const C2 *>(ops[i].in);
    if (ng == 0 || groups[ng - 1].in != in || groups[ng - 1].nout == kMaxOut) {
      if (ng == 64) {
        set_error("too many z-pass groups");
        return HE4_E_ARG;
      }
      groups[ng].in = in;
      groups[ng].nout = 0;
      ng++;
    }
    if (ops[i].kern && !kern_of<C2>(h, ops[i].kern)) {
      set_error("no FP32 copy of a z-pass kernel");
      return HE4_E_ARG;
    }
    ZGroupT<C2> &g = groups[ng - 1];
    g.xy_shared = 0;
    g.o[g.nout++] = ZOutT<C2>{reinterpret_cast<C2 *>(ops[i].out), kern_of<C2>(h, ops[i].kern), ops[i].coef,
                              ops[i].dsym_axis, ops[i].boxz};
  }
  // the three derivative outputs of one kernel (the force field): ordered
  // z, x, y so that the x and y outputs share one inverse transform
  for (int i = 0; i < ng; i++) {
    ZGroupT<C2> &g = groups[i];
    if (g.nout != 3 || !h->zconv_share_xy) continue;
    int at[3] = {-1, -1, -1};
    bool same = true;
    for (int o = 0; o < 3; o++) {
      const ZOutT<C2> &z = g.o[o];
      same = same && z.kern == g.o[0].kern && z.coef == g.o[0].coef && z.boxz == g.o[0].boxz;
      if (z.dsym_axis >= 0 && z.dsym_axis < 3) at[z.dsym_axis] = o;
    }
    if (!same || at[0] < 0 || at[1] < 0 || at[2] < 0) continue;
    const ZOutT<C2> oz = g.o[at[2]], ox = g.o[at[0]], oy = g.o[at[1]];
    g.o[0] = oz;
    g.o[1] = ox;
    g.o[2] = oy;
    g.xy_shared = 1;
  }
  for (int g0 = 0; g0 < ng; g0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, ng - g0);
    ZRegArgs<C2> a{};
    a.map.nxh = P.nxh;
    a.map.nother = P.ny;
    a.map.so = P.nxh;
    a.sf = (long)P.ny * P.nxh;
    a.nx = P.nx;
    a.ny = P.ny;
    a.nz = P.nz;
    a.dsym = dsym_of<C2>(h);
    a.tw = twid<C2>(P.az);
    a.box = h->box;
    for (int i = 0; i < nb; i++) a.g[i] = groups[g0 + i];
    const long total = (long)P.nxh * P.ny;
    bool single = true;
    for (int i = 0; i < nb; i++) single = single && (a.g[i].nout == 1);
    HE4_REG_SWITCH(P.nz, P.n1[2], {
      constexpr int W = kRegThreads / N1_;
      a.map.W = W;
      const long ntiles = (total + W - 1) / W;
      static std::atomic<int> per_sm[kMaxDevices][2];  // per instantiation and device
      const int dev = h->dev;
      int ps = per_sm[dev][single ? 1 : 0].load(std::memory_order_relaxed);
      if (ps == 0) {
        int nsm = 0, occ = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (single)
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_zconv_pipe<NN, N1_, true, C2>, kRegThreads,
                                                        smem_zpipe<NN, N1_, C2>());
        else
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_zconv_pipe<NN, N1_, false, C2>, kRegThreads,
                                                        smem_zpipe<NN, N1_, C2>());
        ps = std::max(1, occ) * std::max(1, nsm);
        per_sm[dev][single ? 1 : 0].store(ps, std::memory_order_relaxed);
      }
      dim3 grid(nb, (unsigned)std::min<long>(ntiles, std::max(1, ps / nb)));
      if (single) {
        k_zconv_pipe<NN, N1_, true, C2><<<grid, kRegThreads, smem_zpipe<NN, N1_, C2>(), h->stream>>>(a);
      } else if (sizeof(C2) == 16) {
        k_zconv_pipe<NN, N1_, false, C2><<<grid, kRegThreads, smem_zpipe<NN, N1_, C2>(), h->stream>>>(a);
      } else {
        // FP32 with several outputs: the pipelined form's registers (two
        // tiles, two kernel sets) leave one CTA per SM; the one-tile form
        // with shared-memory kernel tiles is faster there
        dim3 g1(nb, (unsigned)ntiles);
        k_zconv_reg<NN, N1_, false, C2><<<g1, kRegThreads, smem_zconv<NN, N1_, false, C2>(), h->stream>>>(a);
      }
    });
    HE4_LAUNCHED(h);
  }
  return HE4_OK;
}

int fft_z_conv(Handle *h, int n, const ZOp *ops) {
  const FftPlan &P = h->fft;
  if (n <= 0) return HE4_OK;
  const bool plain = ops[0].mode != 0;
  if (reg_ok(P.nz) && !plain) return h->fp32 ? zconv_reg<float2>(h, n, ops) : zconv_reg<double2>(h, n, ops);
  if (reg_ok(P.nz) && plain) {
    for (int i = 0; i < n; i++) {
      double2 *b[1] = {ops[i].out};
      if (ops[i].out != ops[i].in) {
        set_error("plain z transforms are in place");
        return HE4_E_ARG;
      }
      HE4_TRY(strided_pass(h, 1, b, 2, ops[i].mode == 2));
    }
    return HE4_OK;
  }
  if (h->fp32) {
    set_error("FP32 spectra need register-path axis lengths");
    return HE4_E_UNSUPPORTED;
  }
  for (int b0 = 0; b0 < n; b0 += kMaxBatch) {
    int nb = std::min(kMaxBatch, n - b0);
    ZArgs a{};
    a.az = P.az;
    a.map.nxh = P.nxh;
    a.map.nother = P.ny;
    a.map.W = P.wz;
    a.map.so = P.nxh;
    a.sf = (long)P.ny * P.nxh;
    a.nx = P.nx;
    a.ny = P.ny;
    a.nz = P.nz;
    a.dsym = h->dsym;
    for (int i = 0; i < nb; i++) a.ops[i] = ops[b0 + i];
    long total = (long)P.nxh * P.ny;
    dim3 grid(nb, (unsigned)((total + P.wz - 1) / P.wz));
    k_fft_z_conv<<<grid, kThreads, smem_yz(P.nz, P.wz), h->stream>>>(a);
    HE4_LAUNCHED(h);
  }
  return HE4_OK;
}

template <typename C2>
static int zsum_reg(Handle *h, int nterm, const ZTerm *terms, double2 *out) {
  const FftPlan &P = h->fft;
  ZSumArgs<C2> a{};
  a.map.nxh = P.nxh;
  a.map.nother = P.ny;
  a.map.so = P.nxh;
  a.sf = (long)P.ny * P.nxh;
  a.tw = twid<C2>(P.az);
  a.nterm = nterm;
  for (int j = 0; j < nterm; j++) {
    a.t[j].in = reinterpret_cast<const C2 *>(terms[j].in);
    a.t[j].kern = kern_of<C2>(h, terms[j].kern);
    a.t[j].coef = terms[j].coef;
    if (!a.t[j].kern) {
      set_error("z-pass sum term without a kernel");
      return HE4_E_ARG;
    }
  }
  a.out = reinterpret_cast<C2 *>(out);
  const long total = (long)P.nxh * P.ny;
  HE4_REG_SWITCH(P.nz, P.n1[2], {
    constexpr int W = kRegThreads / N1_;
    a.map.W = W;
    k_zsum_reg<NN, N1_, C2><<<(unsigned)((total + W - 1) / W), kRegThreads, smem_zsum<NN, N1_, C2>(),
                             h->stream>>>(a);
  });
  HE4_LAUNCHED(h);
  return HE4_OK;
}

bool fft_z_sum_ok(const Handle *h) { return reg_ok(h->fft.nz); }

int fft_z_sum(Handle *h, int nterm, const ZTerm *terms, double2 *out) {
  if (nterm < 1 || nterm > kMaxTerms || !fft_z_sum_ok(h)) {
    set_error("fft_z_sum: %d terms, z length %d", nterm, h->fft.nz);
    return HE4_E_ARG;
  }
  return h->fp32 ? zsum_reg<float2>(h, nterm, terms, out) : zsum_reg<double2>(h, nterm, terms, out);
}

int fft_z_only(Handle *h, double2 *buf, bool inverse) {
  ZOp op{buf, buf, nullptr, 1.0, -1, inverse ? 2 : 1};
  return fft_z_conv(h, 1, &op);
}

// the inverse x pass alone with float output rows (FP32-convolution form)
int fft_x_c2r_f32_only(Handle *h, const double2 *cin, float *rout) {
  double2 *ci[1] = {const_cast<double2 *>(cin)};
  void *ro[1] = {rout};
  return x_pass_v(h, 1, nullptr, nullptr, ci, ro, true, nullptr, XLoad(), true);
}

int fft_x_only(Handle *h, const double *rin, double2 *cout, const double2 *cin, double *rout, bool inverse) {
  const double *ri[1] = {rin};
  double2 *co[1] = {cout};
  double2 *ci[1] = {const_cast<double2 *>(cin)};
  double *ro[1] = {rout};
  return x_pass(h, 1, ri, co, ci, ro, inverse);
}

}  // namespace he4

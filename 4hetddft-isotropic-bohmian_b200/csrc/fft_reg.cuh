// fft_reg.cuh -- register-resident pencil FFTs for lengths 16..256 (powers
// of two), used by the x, y and z passes when the axis length allows, in
// FP64 (double2) or FP32 (float2).
//
// A length-N transform is split N = N1 * N2 (four-step form).  With
// j = j1 + N1 j2 and k = k2 + N2 k1:
//   X[k2 + N2 k1] = sum_j1 w_N1^(j1 k1) w_N^(j1 k2) sum_j2 x[j1 + N1 j2] w_N2^(j2 k2)
// Thread "j1" of a pencil holds x[j1 + N1 j2] (j2 < N2) in registers, runs
// the N2-point DFT, applies w_N^(j1 k2) and writes to shared memory; after a
// barrier thread "q" reads the N1 values of its k2 = q + N1 c (c < N2/N1),
// runs the N1-point DFTs and holds X[k2 + N2 k1] in registers.  The inverse
// runs the same steps backwards from that register layout, so a
// forward transform, a pointwise multiply and an inverse transform need two
// shared-memory exchanges and no global round trip.
#pragma once
#include "common.cuh"

namespace he4 {
namespace regfft {

// complex type of a real type
template <typename T>
struct Cx;
template <>
struct Cx<double> {
  using type = double2;
};
template <>
struct Cx<float> {
  using type = float2;
};

template <typename C2>
struct Re;
template <>
struct Re<double2> {
  using type = double;
};
template <>
struct Re<float2> {
  using type = float;
};

template <typename C2>
__device__ __forceinline__ C2 mk(typename Re<C2>::type a, typename Re<C2>::type b) {
  C2 r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename C2>
__device__ __forceinline__ C2 add(C2 a, C2 b) { return mk<C2>(a.x + b.x, a.y + b.y); }
template <typename C2>
__device__ __forceinline__ C2 sub(C2 a, C2 b) { return mk<C2>(a.x - b.x, a.y - b.y); }
// FP32: both components in one packed instruction (sm_100 f32x2 arithmetic;
// the same round-to-nearest sums as the scalar form)
template <>
__device__ __forceinline__ float2 add<float2>(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0,%1}, rd;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template <>
__device__ __forceinline__ float2 sub<float2>(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2,%3};\n\tmov.b64 rb, {%4,%5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0,%1}, rd;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template <typename C2>
__device__ __forceinline__ C2 scale(C2 a, typename Re<C2>::type s) { return mk<C2>(a.x * s, a.y * s); }
template <typename C2>
__device__ __forceinline__ C2 mul(C2 a, C2 b) { return mk<C2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

constexpr double kR2 = 0.70710678118654752440;   // cos(pi/4)
constexpr double kC1 = 0.92387953251128675613;   // cos(pi/8)
constexpr double kS1 = 0.38268343236508977173;   // sin(pi/8)

// v * w_16^m for compile-time m (forward root exp(-2 pi i m / 16))
template <int M, bool INV, typename C2>
__device__ __forceinline__ C2 rot16(C2 v) {
  using T = typename Re<C2>::type;
  constexpr int m = M & 15;
  if (m == 0) return v;
  if (m == 4) return INV ? mk<C2>(-v.y, v.x) : mk<C2>(v.y, -v.x);
  if (m == 8) return mk<C2>(-v.x, -v.y);
  if (m == 12) return INV ? mk<C2>(v.y, -v.x) : mk<C2>(-v.y, v.x);
  double cd, sd;
  switch (m) {
    case 1: cd = kC1; sd = kS1; break;
    case 2: cd = kR2; sd = kR2; break;
    case 3: cd = kS1; sd = kC1; break;
    case 5: cd = -kS1; sd = kC1; break;
    case 6: cd = -kR2; sd = kR2; break;
    case 7: cd = -kC1; sd = kS1; break;
    case 9: cd = -kC1; sd = -kS1; break;
    case 10: cd = -kR2; sd = -kR2; break;
    case 11: cd = -kS1; sd = -kC1; break;
    case 13: cd = kS1; sd = -kC1; break;
    case 14: cd = kR2; sd = -kR2; break;
    default: cd = kC1; sd = -kS1; break;  // 15
  }
  const T c = (T)cd, s = (T)sd;
  // forward root: c - i s ; inverse: c + i s
  if (INV) return mk<C2>(v.x * c - v.y * s, v.x * s + v.y * c);
  return mk<C2>(v.x * c + v.y * s, v.y * c - v.x * s);
}

template <bool INV, typename C2>
__device__ __forceinline__ C2 muli(C2 a) {  // -i a (fwd), +i a (inv)
  return INV ? mk<C2>(-a.y, a.x) : mk<C2>(a.y, -a.x);
}

template <bool INV, typename C2>
__device__ __forceinline__ void dft4(C2 &x0, C2 &x1, C2 &x2, C2 &x3) {
  const C2 a = add(x0, x2), b = sub(x0, x2), c = add(x1, x3), d = muli<INV>(sub(x1, x3));
  x0 = add(a, c);
  x2 = sub(a, c);
  x1 = add(b, d);
  x3 = sub(b, d);
}

// in-place DFT of R points held in v[0..R-1] (natural order in and out)
template <int R, bool INV, typename C2>
struct Dft;

template <bool INV, typename C2>
struct Dft<2, INV, C2> {
  static __device__ __forceinline__ void run(C2 *v) {
    const C2 t = v[0];
    v[0] = add(t, v[1]);
    v[1] = sub(t, v[1]);
  }
};

template <bool INV, typename C2>
struct Dft<4, INV, C2> {
  static __device__ __forceinline__ void run(C2 *v) { dft4<INV>(v[0], v[1], v[2], v[3]); }
};

template <bool INV, typename C2>
struct Dft<8, INV, C2> {
  // j = j1 + 2 j2: DFT4 over j2 for j1 = 0, 1; twiddle w_8^(j1 k2); DFT2
  static __device__ __forceinline__ void run(C2 *v) {
    C2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
    C2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
    dft4<INV>(a0, a1, a2, a3);
    dft4<INV>(b0, b1, b2, b3);
    b1 = rot16<2, INV>(b1);
    b2 = rot16<4, INV>(b2);
    b3 = rot16<6, INV>(b3);
    v[0] = add(a0, b0);
    v[4] = sub(a0, b0);
    v[1] = add(a1, b1);
    v[5] = sub(a1, b1);
    v[2] = add(a2, b2);
    v[6] = sub(a2, b2);
    v[3] = add(a3, b3);
    v[7] = sub(a3, b3);
  }
};

template <bool INV, typename C2>
struct Dft<16, INV, C2> {
  // j = j1 + 4 j2: DFT4 over j2 for each j1; twiddle w_16^(j1 k2); DFT4 over j1
  static __device__ __forceinline__ void run(C2 *v) {
    C2 y[4][4];
#pragma unroll
    for (int j1 = 0; j1 < 4; j1++) {
      y[j1][0] = v[j1];
      y[j1][1] = v[j1 + 4];
      y[j1][2] = v[j1 + 8];
      y[j1][3] = v[j1 + 12];
      dft4<INV>(y[j1][0], y[j1][1], y[j1][2], y[j1][3]);
    }
    y[1][1] = rot16<1, INV>(y[1][1]);
    y[1][2] = rot16<2, INV>(y[1][2]);
    y[1][3] = rot16<3, INV>(y[1][3]);
    y[2][1] = rot16<2, INV>(y[2][1]);
    y[2][2] = rot16<4, INV>(y[2][2]);
    y[2][3] = rot16<6, INV>(y[2][3]);
    y[3][1] = rot16<3, INV>(y[3][1]);
    y[3][2] = rot16<6, INV>(y[3][2]);
    y[3][3] = rot16<9, INV>(y[3][3]);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) {
      C2 a = y[0][k2], b = y[1][k2], c = y[2][k2], d = y[3][k2];
      dft4<INV>(a, b, c, d);
      v[k2] = a;
      v[k2 + 4] = b;
      v[k2 + 8] = c;
      v[k2 + 12] = d;
    }
  }
};

// shared-memory layouts of the exchange buffer
// pencil-minor (y/z passes): element (k2, j1) of pencil w at (k2*N1+j1)*W+w
struct LayoutYZ {
  int W, w;
  __device__ __forceinline__ int at(int k2, int j1, int N1) const { return (k2 * N1 + j1) * W + w; }
};
// pencil-major with a pad of one per N1 (x pass): conflict-free for both the
// write (consecutive j1) and the read (consecutive k2) of 16-byte elements
struct LayoutX {
  int base;  // p * N2 * (N1 + 1)
  __device__ __forceinline__ int at(int k2, int j1, int N1) const { return base + k2 * (N1 + 1) + j1; }
};

// forward: a[j2] = x[j1 + N1 j2]  ->  a[c N1 + k1] = X[(q + N1 c) + N2 k1], q = j1
template <int N, int N1, bool INV, typename L, typename C2>
__device__ __forceinline__ void fwd2(C2 (&a)[N / N1], C2 *S, const L &lay, int j1, const C2 *__restrict__ tw) {
  constexpr int N2 = N / N1;
  static_assert(N2 % N1 == 0, "N2 must be a multiple of N1");
  Dft<N2, INV, C2>::run(a);
#pragma unroll
  for (int k2 = 1; k2 < N2; k2++) {
    C2 t = tw[j1 * k2];
    if (INV) t.y = -t.y;
    a[k2] = mul(a[k2], t);
  }
#pragma unroll
  for (int k2 = 0; k2 < N2; k2++) S[lay.at(k2, j1, N1)] = a[k2];
  __syncthreads();
#pragma unroll
  for (int c = 0; c < N2 / N1; c++) {
    const int k2 = j1 + N1 * c;
    C2 b[N1];
#pragma unroll
    for (int jj = 0; jj < N1; jj++) b[jj] = S[lay.at(k2, jj, N1)];
    Dft<N1, INV, C2>::run(b);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) a[c * N1 + k1] = b[k1];
  }
  __syncthreads();
}

// inverse of fwd2's layout: a[c N1 + k1] = X[(q + N1 c) + N2 k1]  ->
// a[n2] = x[j1 + N1 n2] (unnormalised; INV selects the root direction)
template <int N, int N1, bool INV, typename L, typename C2>
__device__ __forceinline__ void bwd2(C2 (&a)[N / N1], C2 *S, const L &lay, int j1, const C2 *__restrict__ tw) {
  constexpr int N2 = N / N1;
#pragma unroll
  for (int c = 0; c < N2 / N1; c++) {
    const int k2 = j1 + N1 * c;
    C2 b[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) b[k1] = a[c * N1 + k1];
    Dft<N1, INV, C2>::run(b);
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) {
      C2 t = tw[n1 * k2];
      if (INV) t.y = -t.y;
      S[lay.at(k2, n1, N1)] = (n1 == 0 || k2 == 0) ? b[n1] : mul(b[n1], t);
    }
  }
  __syncthreads();
#pragma unroll
  for (int k2 = 0; k2 < N2; k2++) a[k2] = S[lay.at(k2, j1, N1)];
  Dft<N2, INV, C2>::run(a);
  __syncthreads();
}

}  // namespace regfft
}  // namespace he4

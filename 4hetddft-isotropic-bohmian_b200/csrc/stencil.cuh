// stencil.cuh -- npd-point finite differences on the device.
//
// Restates Deriv3D_p / Deriv3D_pc (init_deriv_parallel.f90:1100-1205,
// 373-655): df(i) = sum_{t=-m..m} Cd(ko2p1, t) f(i+t), Cd = centre row of the
// Bickley matrix times 1/h^id.  icon=8: indices wrap periodically.  icon=13:
// Redef (redef.f:133-170) makes each of the ko2 boundary rows at either end
// the centre row shifted by one more place, its taps past the end dropped,
// which is the same sum with f = 0 outside the grid (Geo::zpad = 1).
// icon=12: Redef shifts only the rows after the centre, so the last ko2
// points see the zero-padded centred stencil and the first ko2 points keep
// the one-sided rows of the Bickley matrix, df(i) = sum_j Cd(i, j) f(j) over
// the first npd points (init_deriv_parallel.f90:429-435; Geo::zpad = 2, the
// rows in Stencil::lo).
#pragma once
#include "common.cuh"

namespace he4 {

struct Geo {
  int nx, ny, nz;
  // 0: icon=8, periodic; 1: icon=13, taps outside the grid dropped; 2:
  // icon=12, the same at the upper end, one-sided rows at the lower end
  int zpad = 0;
};

inline int zpad_of(int icon) { return icon == 13 ? 1 : (icon == 12 ? 2 : 0); }

// weights of derivative order `ord` along `axis`
__device__ __forceinline__ const double *stencil_w(const Stencil &st, int ord, int axis) {
  return ord == 1 ? st.w1[axis] : st.w2[axis];
}
// one-sided row of point c < m (icon=12): taps on the first 2m+1 points
__device__ __forceinline__ const double *stencil_lo(const Stencil &st, int ord, int axis, int c) {
  return st.lo + ((size_t)((ord - 1) * 3 + axis) * st.m + c) * (2 * st.m + 1);
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// sum_t w[t] * f(i + t e_axis), sequential order t = -m..m; ZPAD: taps
// outside the grid dropped (icon=13, 12), one-sided rows at the lower end
// (icon=12), else indices wrapped (icon=8)
template <bool ZPAD>
__device__ __forceinline__ double stencil_axis_t(const double *__restrict__ f, const Stencil &s, int ord,
                                                 const Geo &g, int i, int j, int k, int axis) {
  const double *w = stencil_w(s, ord, axis);
  const int m = s.m;
  double acc = 0.0;
  if constexpr (ZPAD) {
    const int c = (axis == 0) ? i : (axis == 1) ? j : k, n = (axis == 0) ? g.nx : (axis == 1) ? g.ny : g.nz;
    const size_t st = (axis == 0) ? 1 : (axis == 1) ? (size_t)g.nx : (size_t)g.nx * g.ny;
    const double *p0 = f + ((size_t)k * g.ny + j) * g.nx + i;
    if (g.zpad == 2 && c < m) {
      const double *L = stencil_lo(s, ord, axis, c);
      for (int t = 0; t <= 2 * m; t++) acc += L[t] * __ldg(p0 + (long)(t - c) * (long)st);
      return acc;
    }
    for (int t = -m; t <= m; t++)
      if (c + t >= 0 && c + t < n) acc += w[t + m] * __ldg(p0 + (long)t * (long)st);
    return acc;
  }
  if (axis == 0) {
    const double *row = f + ((size_t)k * g.ny + j) * g.nx;
    for (int t = -m; t <= m; t++) acc += w[t + m] * __ldg(row + wrap(i + t, g.nx));
  } else if (axis == 1) {
    const double *col = f + (size_t)k * g.ny * g.nx + i;
    for (int t = -m; t <= m; t++) acc += w[t + m] * __ldg(col + (size_t)wrap(j + t, g.ny) * g.nx);
  } else {
    const double *col = f + (size_t)j * g.nx + i;
    const size_t ps = (size_t)g.ny * g.nx;
    for (int t = -m; t <= m; t++) acc += w[t + m] * __ldg(col + (size_t)wrap(k + t, g.nz) * ps);
  }
  return acc;
}

// the periodic or boundary-row form as the grid says
__device__ __forceinline__ double stencil_axis(const double *__restrict__ f, const Stencil &s, int ord, const Geo &g,
                                               int i, int j, int k, int axis) {
  return g.zpad ? stencil_axis_t<true>(f, s, ord, g, i, j, k, axis) : stencil_axis_t<false>(f, s, ord, g, i, j, k, axis);
}

template <bool ZPAD>
__device__ __forceinline__ double2 stencil_axis_c_t(const double2 *__restrict__ f, const Stencil &s, int ord,
                                                    const Geo &g, int i, int j, int k, int axis) {
  const double *w = stencil_w(s, ord, axis);
  const int m = s.m;
  double ar = 0.0, ai = 0.0;
  if constexpr (ZPAD) {
    const int c = (axis == 0) ? i : (axis == 1) ? j : k, n = (axis == 0) ? g.nx : (axis == 1) ? g.ny : g.nz;
    const size_t st = (axis == 0) ? 1 : (axis == 1) ? (size_t)g.nx : (size_t)g.nx * g.ny;
    const double2 *p0 = f + ((size_t)k * g.ny + j) * g.nx + i;
    if (g.zpad == 2 && c < m) {
      const double *L = stencil_lo(s, ord, axis, c);
      for (int t = 0; t <= 2 * m; t++) {
        const double2 v = __ldg(p0 + (long)(t - c) * (long)st);
        ar += L[t] * v.x;
        ai += L[t] * v.y;
      }
      return make_double2(ar, ai);
    }
    for (int t = -m; t <= m; t++)
      if (c + t >= 0 && c + t < n) {
        const double2 v = __ldg(p0 + (long)t * (long)st);
        ar += w[t + m] * v.x;
        ai += w[t + m] * v.y;
      }
    return make_double2(ar, ai);
  }
  if (axis == 0) {
    const double2 *row = f + ((size_t)k * g.ny + j) * g.nx;
    for (int t = -m; t <= m; t++) {
      double2 v = __ldg(row + wrap(i + t, g.nx));
      ar += w[t + m] * v.x;
      ai += w[t + m] * v.y;
    }
  } else if (axis == 1) {
    const double2 *col = f + (size_t)k * g.ny * g.nx + i;
    for (int t = -m; t <= m; t++) {
      double2 v = __ldg(col + (size_t)wrap(j + t, g.ny) * g.nx);
      ar += w[t + m] * v.x;
      ai += w[t + m] * v.y;
    }
  } else {
    const double2 *col = f + (size_t)j * g.nx + i;
    const size_t ps = (size_t)g.ny * g.nx;
    for (int t = -m; t <= m; t++) {
      double2 v = __ldg(col + (size_t)wrap(k + t, g.nz) * ps);
      ar += w[t + m] * v.x;
      ai += w[t + m] * v.y;
    }
  }
  return make_double2(ar, ai);
}

__device__ __forceinline__ double2 stencil_axis_c(const double2 *__restrict__ f, const Stencil &s, int ord,
                                                  const Geo &g, int i, int j, int k, int axis) {
  return g.zpad ? stencil_axis_c_t<true>(f, s, ord, g, i, j, k, axis)
                : stencil_axis_c_t<false>(f, s, ord, g, i, j, k, axis);
}

// complex Laplacian (sum of the three second derivatives, x + y + z)
template <bool ZPAD>
__device__ __forceinline__ double2 lap_c_t(const double2 *__restrict__ f, const Stencil &st, const Geo &g, int i,
                                           int j, int k) {
  double2 a = stencil_axis_c_t<ZPAD>(f, st, 2, g, i, j, k, 0);
  double2 b = stencil_axis_c_t<ZPAD>(f, st, 2, g, i, j, k, 1);
  double2 c = stencil_axis_c_t<ZPAD>(f, st, 2, g, i, j, k, 2);
  return make_double2((a.x + b.x) + c.x, (a.y + b.y) + c.y);
}

// launch geometry helpers: blocks of 32 x 8 points, grid over (x, y, z)
inline dim3 grid3(const Geo &g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }
inline dim3 block3() { return dim3(32, 8, 1); }

#define HE4_IJK(g)                                   \
  const int i = blockIdx.x * 32 + threadIdx.x;       \
  const int j = blockIdx.y * 8 + threadIdx.y;        \
  const int k = blockIdx.z;                          \
  if (i >= (g).nx || j >= (g).ny) return;            \
  const size_t t = ((size_t)k * (g).ny + j) * (g).nx + i;

}  // namespace he4

// stencil.cuh -- periodic npd-point finite differences on the device.
//
// Restates Deriv3D_p / Deriv3D_pc for icon=8 (init_deriv_parallel.f90:
// 1100-1205, 475-650): df(i) = sum_{t=-m..m} Cd(ko2p1, t) f(i+t) with indices
// wrapped periodically, Cd = centre row of the Bickley matrix times 1/h^id.
#pragma once
#include "common.cuh"

namespace he4 {

struct Geo {
  int nx, ny, nz;
};

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// sum_t w[t] * f(i + t e_axis), periodic; sequential order t = -m..m
__device__ __forceinline__ double stencil_axis(const double *__restrict__ f, const double *w, int m, const Geo &g,
                                               int i, int j, int k, int axis) {
  double acc = 0.0;
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

__device__ __forceinline__ double2 stencil_axis_c(const double2 *__restrict__ f, const double *w, int m,
                                                  const Geo &g, int i, int j, int k, int axis) {
  double ar = 0.0, ai = 0.0;
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

// complex Laplacian (sum of the three second derivatives, x + y + z)
__device__ __forceinline__ double2 lap_c(const double2 *__restrict__ f, const Stencil &st, const Geo &g, int i,
                                         int j, int k) {
  double2 a = stencil_axis_c(f, st.w2[0], st.m, g, i, j, k, 0);
  double2 b = stencil_axis_c(f, st.w2[1], st.m, g, i, j, k, 1);
  double2 c = stencil_axis_c(f, st.w2[2], st.m, g, i, j, k, 2);
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

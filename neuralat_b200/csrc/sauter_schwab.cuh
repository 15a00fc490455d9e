// Sauter-Schwab quadrature of touching triangle pairs, shared by the generic
// and Burton-Miller assembly kernels.  The published method in the
// reference's parametrisation (src/bem/cuda/include/integrand.h:117-152):
// both triangles mapped to the reference triangle (0,0),(1,0),(1,1) with the
// shared vertices first (integrand.h:351-387), a 4-D Gauss-Legendre rule on
// [0,1]^4, and per coincidence type the sub-regions below.
#pragma once

#include "bem_common.cuh"

namespace bemb {

// Gauss-Legendre points on [-1,1] for 2 and 4 points.
template <int LN>
__host__ __device__ constexpr double gl_x(int i) {
  return LN == 4 ? gl4_x(i) : (i == 0 ? 0.57735026918962576 : -0.57735026918962576);
}
template <int LN>
__host__ __device__ constexpr double gl_w(int i) {
  return LN == 4 ? gl4_w(i) : 1.0;
}

// Local vertex order of a touching pair with the shared vertices first:
// test slot c holds local vertex i_c, trial slot c holds j_c.
struct Perm6 {
  int i0, i1, i2, j0, j1, j2;
};
__device__ __forceinline__ int sel3(int a0, int a1, int a2, int idx) { return idx == 0 ? a0 : (idx == 1 ? a1 : a2); }

template <int NCOMMON>
__device__ __forceinline__ Perm6 reorder6(int s0, int s1, int s2, int t0, int t1, int t2) {
  Perm6 p{0, 1, 2, 0, 1, 2};
  const int si[3] = {s0, s1, s2}, sj[3] = {t0, t1, t2};
  if (NCOMMON == 2) {
    int mi0 = 0, mj0 = 0, mi1 = 1, mj1 = 1, cnt = 0;
#pragma unroll
    for (int jj = 0; jj < 3; jj++)
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const bool eq = si[ii] == sj[jj];
        if (eq && cnt == 0) { mi0 = ii; mj0 = jj; }
        if (eq && cnt == 1) { mi1 = ii; mj1 = jj; }
        cnt += eq ? 1 : 0;
      }
    p = Perm6{mi0, mi1, 3 - mi0 - mi1, mj0, mj1, 3 - mj0 - mj1};
  } else if (NCOMMON == 1) {
    int ci = 0, cj = 0;
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++)
        if (si[ii] == sj[jj]) { ci = ii; cj = jj; }
    p = Perm6{ci, ci == 1 ? 0 : 1, ci == 2 ? 0 : 2, cj, cj == 1 ? 0 : 1, cj == 2 ? 0 : 2};
  }
  return p;
}

// Calls region(x1, x2, y1, y2, weight) for every sub-region of one point
// (xi, e1, e2, e3) of the 4-D rule with weight w0; (x1, x2) and (y1, y2)
// are points of the reference triangle for the test and trial triangle.
template <int NCOMMON, typename R, typename F>
__device__ __forceinline__ void ss_regions(R xi, R e1, R e2, R e3, R w0, F& region) {
  const R e12 = e1 * e2, e123 = e12 * e3;
  if (NCOMMON == 3) {
    const R sc = xi * xi * xi * e1 * e1 * e2 * w0;
    region(xi, xi * (R(1) - e1 + e12), xi * (R(1) - e123), xi * (R(1) - e1), sc);
    region(xi * (R(1) - e123), xi * (R(1) - e1), xi, xi * (R(1) - e1 + e12), sc);
    region(xi, xi * (e1 - e12 + e123), xi * (R(1) - e12), xi * (e1 - e12), sc);
    region(xi * (R(1) - e12), xi * (e1 - e12), xi, xi * (e1 - e12 + e123), sc);
    region(xi * (R(1) - e123), xi * (e1 - e123), xi, xi * (e1 - e12), sc);
    region(xi, xi * (e1 - e12), xi * (R(1) - e123), xi * (e1 - e123), sc);
  } else if (NCOMMON == 2) {
    const R sc = xi * xi * xi * e1 * e1 * w0;
    region(xi, xi * e1 * e3, xi * (R(1) - e12), xi * e1 * (R(1) - e2), sc);
    region(xi, xi * e1, xi * (R(1) - e123), xi * e1 * e2 * (R(1) - e3), e2 * sc);
    region(xi * (R(1) - e12), xi * e1 * (R(1) - e2), xi, xi * e123, e2 * sc);
    region(xi * (R(1) - e123), xi * e12 * (R(1) - e3), xi, xi * e1, e2 * sc);
    region(xi * (R(1) - e123), xi * e1 * (R(1) - e2 * e3), xi, xi * e12, e2 * sc);
  } else {
    const R sc = xi * xi * xi * e2 * w0;
    region(xi, xi * e1, xi * e2, xi * e2 * e3, sc);
    region(xi * e2, xi * e2 * e3, xi, xi * e1, sc);
  }
}

}  // namespace bemb

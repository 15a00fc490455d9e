// Hand-written adjoint of the listener pressures p = -S g + D u with
// (1/2 M - K) u = -V g (src/bem/solver.py:97-104,140-147).
//
// For a loss with gradient pbar = dL/dp* (PyTorch's convention),
//   lambda = (1/2 M - K)^{-H} D^H pbar                      (adjoint solve)
//   dL/dg* = -S^H pbar - V^H lambda
//   dL/dx  = Re[ -pbar^H dS g + pbar^H dD u - lambda^H dV g
//                - 1/2 lambda^H dM u + lambda^H dK u ]       (vertex coordinates)
// The second line needs only conjugate-transposed applications; the last is
// a "kernel-derivative assembly": one pass over every triangle pair (and
// listener-triangle pair) differentiates the quadrature sum through the
// quadrature points, the areas and the trial normals, contracted with the
// vectors on the fly, so no derivative matrix is ever stored.
//
// With G = e^{ikr}/(4 pi r), d = y - x, f = G'(r)/r, the double-layer kernel
// is K = f (d.n_y) and, for a pair term F = a (bV G + bK K):
//   grad_y F = (a bV f + a bK f' (d.n)/r) d + a bK f n,  grad_x F = -grad_y F,
//   grad_n F = a bK f d,
// with the reference's clamp r -> max(r, 1e-3) (potential.h:21-23): inside it
// G and K's radial factor are constant, so their r-derivatives vanish.

#include <cmath>

#include "bem_common.cuh"

namespace bemb {

int geom_view(const void* geom, GeomView* v, GeomHeader* out_hdr);

namespace {

template <typename R>
__device__ __forceinline__ void sincos_a(R x, R* s, R* c);
template <>
__device__ __forceinline__ void sincos_a<double>(double x, double* s, double* c) {
  sincos(x, s, c);
}
template <>
__device__ __forceinline__ void sincos_a<float>(float x, float* s, float* c) {
  sincosf(x, s, c);
}

// One quadrature-point pair.  Accumulates (all times W):
//   F  += Re(a (bV G + bK K))
//   gy += grad_y Re(...)     (grad_x is its negative)
//   gn += grad_n Re(...)
template <typename R>
__device__ __forceinline__ void point_grad(const R d[3], const R n[3], R k, R ar, R ai, R bvr, R bvi, R bkr, R bki,
                                           R W, R& F, R gy[3], R gn[3]) {
  R r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const bool clamped = r < R(kEps);
  if (clamped) r = R(kEps);
  const R u = R(1) / r;
  R s, c;
  sincos_a<R>(k * r, &s, &c);
  const R Gr = u * c, Gi = u * s;                                     // G (without 1/4pi)
  const R Gpr = u * (-u * c - k * s), Gpi = u * (-u * s + k * c);     // G'
  const R fr = Gpr * u, fi = Gpi * u;                                 // f = G'/r
  const R t1 = R(2) * u * u - k * k, t2 = R(-2) * k * u;
  const R Gppr = Gr * t1 - Gi * t2, Gppi = Gr * t2 + Gi * t1;         // G''
  const R fpr = (Gppr - Gpr * u) * u, fpi = (Gppi - Gpi * u) * u;     // f'
  const R dn = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
  const R aVr = ar * bvr - ai * bvi, aVi = ar * bvi + ai * bvr;       // a bV
  const R aKr = ar * bkr - ai * bki, aKi = ar * bki + ai * bkr;       // a bK
  const R ReG = aVr * Gr - aVi * Gi;
  const R ReK = (aKr * fr - aKi * fi) * dn;
  F += W * (ReG + ReK);
  const R ReAVf = clamped ? R(0) : (aVr * fr - aVi * fi);
  const R ReAKfp = clamped ? R(0) : (aKr * fpr - aKi * fpi);
  const R c1 = W * (ReAVf + ReAKfp * dn * u);
  const R c2 = W * (aKr * fr - aKi * fi);
#pragma unroll
  for (int e = 0; e < 3; e++) {
    gy[e] += c1 * d[e] + c2 * n[e];
    gn[e] += c2 * d[e];
  }
}

template <typename R>
struct V3R {
  R x[3];
};

// d(area)/d(v_c) = 1/2 n x (v_{c+2} - v_{c+1});   normal chain:
// d(E)/d(v_c) += (v_{c+1} - v_{c+2}) x t,  t = (I - n n^T) dE/dn / |c|.
template <typename R>
__device__ __forceinline__ void area_normal_grad(const R v[3][3], R dE_dA_over, const R dEdn[3], bool use_n,
                                                 R out[3][3]) {
  const R e1[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
  const R e2[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
  const R cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  const R cn = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  const R n[3] = {cr[0] / cn, cr[1] / cn, cr[2] / cn};
  R t[3] = {0, 0, 0};
  if (use_n) {
    const R nd = n[0] * dEdn[0] + n[1] * dEdn[1] + n[2] * dEdn[2];
    for (int e = 0; e < 3; e++) t[e] = (dEdn[e] - nd * n[e]) / cn;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
    const R ea[3] = {v[c2][0] - v[c1][0], v[c2][1] - v[c1][1], v[c2][2] - v[c1][2]};  // v_{c+2} - v_{c+1}
    // 1/2 n x ea, scaled by dE/dA
    const R ag[3] = {R(0.5) * (n[1] * ea[2] - n[2] * ea[1]), R(0.5) * (n[2] * ea[0] - n[0] * ea[2]),
                     R(0.5) * (n[0] * ea[1] - n[1] * ea[0])};
    const R eb[3] = {-ea[0], -ea[1], -ea[2]};  // v_{c+1} - v_{c+2}
    const R ng[3] = {eb[1] * t[2] - eb[2] * t[1], eb[2] * t[0] - eb[0] * t[2], eb[0] * t[1] - eb[1] * t[0]};
#pragma unroll
    for (int e = 0; e < 3; e++) out[c][e] = dE_dA_over * ag[e] + ng[e];
  }
}

__device__ __forceinline__ double2 lerp3(const float2* vec, int v0, int v1, int v2, double l0, double l1, double l2) {
  const float2 a = vec[v0], b = vec[v1], c = vec[v2];
  return make_double2(l0 * a.x + l1 * b.x + l2 * c.x, l0 * a.y + l1 * b.y + l2 * c.y);
}

// ---------------------------------------------------------------------------
// Regular pairs (touching pairs masked).  Thread = test triangle (input
// order), loops over all trial triangles; test-side gradient in registers,
// trial-side per pair through warp shuffles (all lanes share the trial
// triangle) and one set of atomics.
// ---------------------------------------------------------------------------
constexpr int kAdjThreads = 128;

__global__ void __launch_bounds__(kAdjThreads)
    grad_regular_kernel(GeomView g, float k, const float2* __restrict__ lam, const float2* __restrict__ gvec,
                        const float2* __restrict__ uvec, double* __restrict__ grad, int jchunk) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * 32 + lane;  // each warp of the block takes a quarter of the trial range
  const int warp = threadIdx.x >> 5;
  const bool valid_i = i < g.nt;
  const TriRec& ri = g.rec_orig[valid_i ? i : 0];
  const int iv[3] = {ri.v[0], ri.v[1], ri.v[2]};
  // conj(lambda) at the 6 test points
  float ar[6], ai[6];
#pragma unroll
  for (int p = 0; p < 6; p++) {
    const double2 l = lerp3(lam, iv[0], iv[1], iv[2], tri6_phi(p, 0), tri6_phi(p, 1), tri6_phi(p, 2));
    ar[p] = (float)l.x;
    ai[p] = -(float)l.y;
  }
  float gi[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  float Fi = 0.f;
  const int j0 = blockIdx.y * jchunk + warp;
  const int j1 = min(g.nt, (blockIdx.y + 1) * jchunk);
  for (int j = j0; j < j1; j += kAdjThreads / 32) {
    const TriRec& rj = g.rec_orig[j];
    const bool touching = (iv[0] == rj.v[0]) | (iv[0] == rj.v[1]) | (iv[0] == rj.v[2]) | (iv[1] == rj.v[0]) |
                          (iv[1] == rj.v[1]) | (iv[1] == rj.v[2]) | (iv[2] == rj.v[0]) | (iv[2] == rj.v[1]) |
                          (iv[2] == rj.v[2]);
    const float W0 = (valid_i && !touching) ? ri.area * rj.area * kInv4Pi : 0.f;
    float Fp = 0.f, Nsum[3] = {0, 0, 0};
    float U[6][3];
#pragma unroll
    for (int q = 0; q < 6; q++) U[q][0] = U[q][1] = U[q][2] = 0.f;
    float bvr[6], bvi[6], bkr[6], bki[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const double2 gq = lerp3(gvec, rj.v[0], rj.v[1], rj.v[2], tri6_phi(q, 0), tri6_phi(q, 1), tri6_phi(q, 2));
      const double2 uq = lerp3(uvec, rj.v[0], rj.v[1], rj.v[2], tri6_phi(q, 0), tri6_phi(q, 1), tri6_phi(q, 2));
      bvr[q] = -(float)gq.x;
      bvi[q] = -(float)gq.y;
      bkr[q] = (float)uq.x;
      bki[q] = (float)uq.y;
    }
    const float n[3] = {rj.n[0], rj.n[1], rj.n[2]};
#pragma unroll
    for (int p = 0; p < 6; p++) {
      float T[3] = {0, 0, 0};
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const float d[3] = {rj.qp[3 * q] - ri.qp[3 * p], rj.qp[3 * q + 1] - ri.qp[3 * p + 1],
                            rj.qp[3 * q + 2] - ri.qp[3 * p + 2]};
        float gy[3] = {0, 0, 0};
        const float W = W0 * (float)(tri6_w(p) * tri6_w(q));
        point_grad<float>(d, n, k, ar[p], ai[p], bvr[q], bvi[q], bkr[q], bki[q], W, Fp, gy, Nsum);
#pragma unroll
        for (int e = 0; e < 3; e++) {
          T[e] += gy[e];
          U[q][e] += gy[e];
        }
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float l = (float)tri6_phi(p, c);
#pragma unroll
        for (int e = 0; e < 3; e++) gi[c][e] -= l * T[e];  // grad_x = -grad_y
      }
    }
    Fi += Fp;
    // trial side: reduce over the warp's test triangles
    float gj[3][3];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) {
        float s = 0.f;
#pragma unroll
        for (int q = 0; q < 6; q++) s += (float)tri6_phi(q, c) * U[q][e];
        gj[c][e] = s;
      }
    float red[13];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) red[3 * c + e] = gj[c][e];
    red[9] = Fp;
    red[10] = Nsum[0];
    red[11] = Nsum[1];
    red[12] = Nsum[2];
#pragma unroll
    for (int e = 0; e < 13; e++) {
      float v = red[e];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      red[e] = v;
    }
    if (lane == 0) {
      float vj[3][3];
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int e = 0; e < 3; e++) vj[c][e] = g.vertices[3 * rj.v[c] + e];
      float out[3][3];
      const float dEdn[3] = {red[10], red[11], red[12]};
      area_normal_grad<float>(vj, red[9] / rj.area, dEdn, true, out);
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int e = 0; e < 3; e++) atomicAdd(&grad[3 * rj.v[c] + e], (double)(red[3 * c + e] + out[c][e]));
    }
  }
  if (valid_i) {
    float vi[3][3];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) vi[c][e] = g.vertices[3 * iv[c] + e];
    float out[3][3];
    const float zero[3] = {0, 0, 0};
    area_normal_grad<float>(vi, Fi / ri.area, zero, false, out);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) atomicAdd(&grad[3 * iv[c] + e], (double)(gi[c][e] + out[c][e]));
  }
}

// ---------------------------------------------------------------------------
// Touching pairs: Sauter-Schwab points (integrand.h:63-185) with the same
// per-point gradient, one warp per pair.
// ---------------------------------------------------------------------------
struct PermA {
  int i0, i1, i2, j0, j1, j2;
};
__device__ __forceinline__ int pk3(int a0, int a1, int a2, int idx) { return idx == 0 ? a0 : (idx == 1 ? a1 : a2); }

template <int NCOMMON>
__device__ __forceinline__ PermA reorderA(int s0, int s1, int s2, int t0, int t1, int t2) {
  PermA p{0, 1, 2, 0, 1, 2};
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
    p = PermA{mi0, mi1, 3 - mi0 - mi1, mj0, mj1, 3 - mj0 - mj1};
  } else if (NCOMMON == 1) {
    int ci = 0, cj = 0;
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++)
        if (si[ii] == sj[jj]) { ci = ii; cj = jj; }
    p = PermA{ci, ci == 1 ? 0 : 1, ci == 2 ? 0 : 2, cj, cj == 1 ? 0 : 1, cj == 2 ? 0 : 2};
  }
  return p;
}

template <typename R, int NCOMMON>
__global__ void __launch_bounds__(128)
    grad_singular_kernel(GeomView g, const int2* __restrict__ pairs, int npairs, float k, const float2* __restrict__ lam,
                         const float2* __restrict__ gvec, const float2* __restrict__ uvec, double* __restrict__ grad) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pair >= npairs) return;
  const int ti = NCOMMON == 3 ? pair : pairs[pair].x;
  const int tj = NCOMMON == 3 ? pair : pairs[pair].y;
  const int s0 = g.triangles[3 * ti], s1 = g.triangles[3 * ti + 1], s2 = g.triangles[3 * ti + 2];
  const int t0 = g.triangles[3 * tj], t1 = g.triangles[3 * tj + 1], t2 = g.triangles[3 * tj + 2];
  const PermA pm = reorderA<NCOMMON>(s0, s1, s2, t0, t1, t2);
  const int pi_[3] = {pm.i0, pm.i1, pm.i2}, pj_[3] = {pm.j0, pm.j1, pm.j2};
  int va[3], vb[3];
  R a[3][3], b[3][3], oa[3][3], ob[3][3];
  const int sv[3] = {s0, s1, s2}, tv[3] = {t0, t1, t2};
  R lr[3], li[3], gr[3], gim[3], ur[3], uim[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    va[c] = pk3(s0, s1, s2, pi_[c]);
    vb[c] = pk3(t0, t1, t2, pj_[c]);
#pragma unroll
    for (int e = 0; e < 3; e++) {
      a[c][e] = (R)g.vertices[3 * va[c] + e];
      b[c][e] = (R)g.vertices[3 * vb[c] + e];
      oa[c][e] = (R)g.vertices[3 * sv[c] + e];
      ob[c][e] = (R)g.vertices[3 * tv[c] + e];
    }
    lr[c] = (R)lam[va[c]].x;
    li[c] = -(R)lam[va[c]].y;  // conjugated
    gr[c] = -(R)gvec[vb[c]].x;
    gim[c] = -(R)gvec[vb[c]].y;
    ur[c] = (R)uvec[vb[c]].x;
    uim[c] = (R)uvec[vb[c]].y;
  }
  R nj[3], Ji, Jj;
  {
    const R e1[3] = {oa[1][0] - oa[0][0], oa[1][1] - oa[0][1], oa[1][2] - oa[0][2]};
    const R e2[3] = {oa[2][0] - oa[0][0], oa[2][1] - oa[0][1], oa[2][2] - oa[0][2]};
    const R cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    Ji = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  }
  {
    const R e1[3] = {ob[1][0] - ob[0][0], ob[1][1] - ob[0][1], ob[1][2] - ob[0][2]};
    const R e2[3] = {ob[2][0] - ob[0][0], ob[2][1] - ob[0][1], ob[2][2] - ob[0][2]};
    const R cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    Jj = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int e = 0; e < 3; e++) nj[e] = cr[e] / Jj;
  }
  R F = 0, N[3] = {0, 0, 0}, GA[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, GB[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  const R kk = (R)k;
  auto region = [&](R x1, R x2, R y1, R y2, R ww) {
    const R lx[3] = {R(1) - x1, x1 - x2, x2};
    const R ly[3] = {R(1) - y1, y1 - y2, y2};
    R d[3];
#pragma unroll
    for (int e = 0; e < 3; e++)
      d[e] = (ly[0] * b[0][e] + ly[1] * b[1][e] + ly[2] * b[2][e]) - (lx[0] * a[0][e] + lx[1] * a[1][e] + lx[2] * a[2][e]);
    const R ar = lx[0] * lr[0] + lx[1] * lr[1] + lx[2] * lr[2];
    const R ai = lx[0] * li[0] + lx[1] * li[1] + lx[2] * li[2];
    const R bvr = ly[0] * gr[0] + ly[1] * gr[1] + ly[2] * gr[2];
    const R bvi = ly[0] * gim[0] + ly[1] * gim[1] + ly[2] * gim[2];
    const R bkr = ly[0] * ur[0] + ly[1] * ur[1] + ly[2] * ur[2];
    const R bki = ly[0] * uim[0] + ly[1] * uim[1] + ly[2] * uim[2];
    R gy[3] = {0, 0, 0};
    point_grad<R>(d, nj, kk, ar, ai, bvr, bvi, bkr, bki, ww, F, gy, N);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) {
        GA[c][e] -= lx[c] * gy[e];
        GB[c][e] += ly[c] * gy[e];
      }
  };
  const R jw = Ji * Jj / R(16) * R(kInv4Pi);
#pragma unroll 1
  for (int pt = lane; pt < 256; pt += 32) {
    const int i0 = pt >> 6, i1 = (pt >> 4) & 3, i2 = (pt >> 2) & 3, i3 = pt & 3;
    const R xi = R(0.5) * (R(gl4_x(i0)) + R(1)), e1 = R(0.5) * (R(gl4_x(i1)) + R(1));
    const R e2 = R(0.5) * (R(gl4_x(i2)) + R(1)), e3 = R(0.5) * (R(gl4_x(i3)) + R(1));
    const R w0 = R(gl4_w(i0)) * R(gl4_w(i1)) * R(gl4_w(i2)) * R(gl4_w(i3)) * jw;
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
  // reduce the 22 accumulators over the warp
  R acc[22];
  acc[0] = F;
  for (int e = 0; e < 3; e++) acc[1 + e] = N[e];
  for (int c = 0; c < 3; c++)
    for (int e = 0; e < 3; e++) {
      acc[4 + 3 * c + e] = GA[c][e];
      acc[13 + 3 * c + e] = GB[c][e];
    }
#pragma unroll
  for (int e = 0; e < 22; e++) {
    R v = acc[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[e] = v;
  }
  if (lane == 0) {
    // point terms on the re-ordered slots
    for (int c = 0; c < 3; c++)
      for (int e = 0; e < 3; e++) {
        atomicAdd(&grad[3 * va[c] + e], (double)acc[4 + 3 * c + e]);
        atomicAdd(&grad[3 * vb[c] + e], (double)acc[13 + 3 * c + e]);
      }
    // weight J_i J_j: d log(J_i J_j) = dA_i / A_i + dA_j / A_j; trial normal chain
    R out[3][3];
    const R zero[3] = {0, 0, 0};
    area_normal_grad<R>(oa, acc[0] / (R(0.5) * Ji), zero, false, out);
    for (int c = 0; c < 3; c++)
      for (int e = 0; e < 3; e++) atomicAdd(&grad[3 * sv[c] + e], (double)out[c][e]);
    const R dEdn[3] = {acc[1], acc[2], acc[3]};
    area_normal_grad<R>(ob, acc[0] / (R(0.5) * Jj), dEdn, true, out);
    for (int c = 0; c < 3; c++)
      for (int e = 0; e < 3; e++) atomicAdd(&grad[3 * tv[c] + e], (double)out[c][e]);
  }
}

// Listener terms Re[-pbar^H dS g + pbar^H dD u]: thread per triangle, loop
// over listeners (x fixed): only the trial side, its area and its normal.
__global__ void grad_listener_kernel(GeomView g, float k, const float* __restrict__ pts, int np,
                                     const float2* __restrict__ pbar, const float2* __restrict__ gvec,
                                     const float2* __restrict__ uvec, double* __restrict__ grad) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.nt) return;
  const TriRec& rj = g.rec_orig[j];
  float bvr[6], bvi[6], bkr[6], bki[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const double2 gq = lerp3(gvec, rj.v[0], rj.v[1], rj.v[2], tri6_phi(q, 0), tri6_phi(q, 1), tri6_phi(q, 2));
    const double2 uq = lerp3(uvec, rj.v[0], rj.v[1], rj.v[2], tri6_phi(q, 0), tri6_phi(q, 1), tri6_phi(q, 2));
    bvr[q] = -(float)gq.x;
    bvi[q] = -(float)gq.y;
    bkr[q] = (float)uq.x;
    bki[q] = (float)uq.y;
  }
  const float n[3] = {rj.n[0], rj.n[1], rj.n[2]};
  float F = 0.f, N[3] = {0, 0, 0}, U[6][3];
#pragma unroll
  for (int q = 0; q < 6; q++) U[q][0] = U[q][1] = U[q][2] = 0.f;
  for (int p = 0; p < np; p++) {
    const float ar = pbar[p].x, ai = -pbar[p].y;  // conj(pbar)
    const float x0 = pts[3 * p], x1 = pts[3 * p + 1], x2 = pts[3 * p + 2];
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const float d[3] = {rj.qp[3 * q] - x0, rj.qp[3 * q + 1] - x1, rj.qp[3 * q + 2] - x2};
      float gy[3] = {0, 0, 0};
      const float W = rj.area * kInv4Pi * (float)tri6_w(q);
      point_grad<float>(d, n, k, ar, ai, bvr[q], bvi[q], bkr[q], bki[q], W, F, gy, N);
#pragma unroll
      for (int e = 0; e < 3; e++) U[q][e] += gy[e];
    }
  }
  float vj[3][3];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int e = 0; e < 3; e++) vj[c][e] = g.vertices[3 * rj.v[c] + e];
  float out[3][3];
  area_normal_grad<float>(vj, F / rj.area, N, true, out);
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int e = 0; e < 3; e++) {
      float s = out[c][e];
#pragma unroll
      for (int q = 0; q < 6; q++) s += (float)tri6_phi(q, c) * U[q][e];
      atomicAdd(&grad[3 * rj.v[c] + e], (double)s);
    }
}

// Mass term -1/2 Re[lambda^H dM u]: M_ab = A (1 + delta_ab)/12 per triangle.
__global__ void grad_mass_kernel(GeomView g, float mass_coeff, const float2* __restrict__ lam,
                                 const float2* __restrict__ uvec, double* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nt) return;
  const TriRec& r = g.rec_orig[i];
  double e = 0.0;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      const float2 la = lam[r.v[a]], ub = uvec[r.v[b]];
      const double m = (a == b ? 2.0 : 1.0) / 12.0;
      e += m * ((double)la.x * ub.x + (double)la.y * ub.y);  // Re(conj(l) u)
    }
  double v[3][3];
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 3; d++) v[c][d] = g.vertices[3 * r.v[c] + d];
  double out[3][3];
  const double zero[3] = {0, 0, 0};
  area_normal_grad<double>(v, (double)mass_coeff * e, zero, false, out);  // dE/dA = coeff * e
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 3; d++) atomicAdd(&grad[3 * r.v[c] + d], out[c][d]);
}

// Y = A^H X (A: n x n complex64 row-major), m columns, Y overwritten.
__global__ void cmatmul_h_kernel(const float2* __restrict__ A, int n, const float2* __restrict__ X, int m,
                                 float2* __restrict__ Y, int rows_per_block) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  const int r0 = blockIdx.y * rows_per_block, r1 = min(n, r0 + rows_per_block);
  for (int s = 0; s < m; s++) {
    double ar = 0.0, ai = 0.0;
    for (int r = r0; r < r1; r++) {
      const float2 a = A[(size_t)r * n + col];
      const float2 x = X[(size_t)r * m + s];
      ar += (double)a.x * x.x + (double)a.y * x.y;  // conj(a) x
      ai += (double)a.x * x.y - (double)a.y * x.x;
    }
    atomicAdd(&Y[(size_t)col * m + s], make_float2((float)ar, (float)ai));
  }
}

// out = conj(A)^T, tiled through shared memory.
__global__ void conj_transpose_kernel(const float2* __restrict__ A, int n, float2* __restrict__ out) {
  __shared__ float2 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int row = by + r, col = bx + threadIdx.x;
    if (row < n && col < n) tile[r][threadIdx.x] = A[(size_t)row * n + col];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int row = bx + r, col = by + threadIdx.x;  // out[row][col] = conj(A[col][row])
    if (row < n && col < n) {
      const float2 v = tile[threadIdx.x][r];
      out[(size_t)row * n + col] = make_float2(v.x, -v.y);
    }
  }
}

// S^H pbar and D^H pbar: thread per trial quadrature point, loop over listeners.
__global__ void b2p_adjoint_kernel(GeomView g, const float* __restrict__ pts, int np, float k,
                                   const float2* __restrict__ pbar, float2* __restrict__ out_s,
                                   float2* __restrict__ out_d) {
  const int jq = blockIdx.x * blockDim.x + threadIdx.x;
  if (jq >= 6 * g.nt) return;
  const int j = jq / 6, q = jq - 6 * j;
  const TriRec& r = g.rec_orig[j];
  float zsr = 0.f, zsi = 0.f, zdr = 0.f, zdi = 0.f;
  for (int p = 0; p < np; p++) {
    const float dx = r.qp[3 * q] - pts[3 * p], dy = r.qp[3 * q + 1] - pts[3 * p + 1], dz = r.qp[3 * q + 2] - pts[3 * p + 2];
    float rr = sqrtf(dx * dx + dy * dy + dz * dz);
    rr = fmaxf(rr, kEps);
    float s, c;
    sincosf(k * rr, &s, &c);
    const float u = 1.f / rr;
    const float gr = c * u, gi = s * u;
    const float dn = dx * r.n[0] + dy * r.n[1] + dz * r.n[2];
    const float f = -dn * u * u * u, kr = k * rr;
    const float dr = (c + kr * s) * f, di = (s - kr * c) * f;
    const float2 pb = pbar[p];
    // conj(kernel) * pbar
    zsr += gr * pb.x + gi * pb.y;
    zsi += gr * pb.y - gi * pb.x;
    zdr += dr * pb.x + di * pb.y;
    zdi += dr * pb.y - di * pb.x;
  }
  const float w = (float)tri6_w(q) * r.area * kInv4Pi;
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const float f = w * (float)tri6_phi(q, b);
    if (out_s) atomicAdd(&out_s[r.v[b]], make_float2(f * zsr, f * zsi));
    if (out_d) atomicAdd(&out_d[r.v[b]], make_float2(f * zdr, f * zdi));
  }
}

}  // namespace

}  // namespace bemb

using namespace bemb;

extern "C" int bem_cmatmul_adjoint(const void* A, int n, const void* X, int m, void* Y, bem_stream_t stream) {
  if (n <= 0 || m <= 0 || !A || !X || !Y) return BEM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  BEM_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(float2) * (size_t)n * m, s));
  const int rpb = 128;
  dim3 grid((n + 127) / 128, (n + rpb - 1) / rpb);
  (cmatmul_h_kernel<<<grid, 128, 0, s>>>((const float2*)A, n, (const float2*)X, m, (float2*)Y, rpb), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

extern "C" int bem_conj_transpose(const void* A, int n, void* out, bem_stream_t stream) {
  if (n <= 0 || !A || !out || A == out) return BEM_ERR_INVALID_ARGUMENT;
  dim3 grid((n + 31) / 32, (n + 31) / 32);
  (conj_transpose_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const float2*)A, n, (float2*)out),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

extern "C" int bem_boundary2potential_adjoint(const void* geom, const float* points, int np, float k,
                                              const void* pbar, void* out_s, void* out_d, bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (np <= 0 || !points || !pbar || (!out_s && !out_d)) return BEM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  if (out_s) BEM_CUDA_TRY(cudaMemsetAsync(out_s, 0, sizeof(float2) * (size_t)g.nv, s));
  if (out_d) BEM_CUDA_TRY(cudaMemsetAsync(out_d, 0, sizeof(float2) * (size_t)g.nv, s));
  (b2p_adjoint_kernel<<<(6 * g.nt + 127) / 128, 128, 0, s>>>(g, points, np, k, (const float2*)pbar, (float2*)out_s,
                                                              (float2*)out_d),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

extern "C" int bem_vertex_gradient(const void* geom, float k, const void* lambda, const void* neumann,
                                   const void* dirichlet, const float* points, int np, const void* pbar, double* grad,
                                   bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (!lambda || !neumann || !dirichlet || !grad || np < 0 || (np > 0 && (!points || !pbar)))
    return BEM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const float2* lam = (const float2*)lambda;
  const float2* gv = (const float2*)neumann;
  const float2* uv = (const float2*)dirichlet;
  BEM_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(double) * 3 * (size_t)g.nv, s));
  // regular pairs: blocks of 4 warps share 32 test triangles, split the trial range
  const int jchunk = 512;
  dim3 rg((g.nt + 31) / 32, (g.nt + jchunk - 1) / jchunk);
  (grad_regular_kernel<<<rg, kAdjThreads, 0, s>>>(g, k, lam, gv, uv, grad, jchunk), count_launch());
  const int wpb = 4;
  (grad_singular_kernel<double, 3><<<(g.nt + wpb - 1) / wpb, 32 * wpb, 0, s>>>(g, nullptr, g.nt, k, lam, gv, uv, grad),
   count_launch());
  if (g.n_edge)
    (grad_singular_kernel<double, 2><<<(g.n_edge + wpb - 1) / wpb, 32 * wpb, 0, s>>>(g, g.edge_pairs, g.n_edge, k, lam,
                                                                                    gv, uv, grad),
     count_launch());
  if (g.n_vert)
    (grad_singular_kernel<float, 1><<<(g.n_vert + wpb - 1) / wpb, 32 * wpb, 0, s>>>(g, g.vert_pairs, g.n_vert, k, lam,
                                                                                   gv, uv, grad),
     count_launch());
  (grad_mass_kernel<<<(g.nt + 127) / 128, 128, 0, s>>>(g, -0.5f, lam, uv, grad), count_launch());
  if (np > 0)
    (grad_listener_kernel<<<(g.nt + 127) / 128, 128, 0, s>>>(g, k, points, np, (const float2*)pbar, gv, uv, grad),
     count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

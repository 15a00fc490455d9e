// FP64 CPU oracle for the NeuralAT boundary-element hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain double precision,
// the quadrature the reference's `src/bem` CUDA extension applies, so that the
// CUDA product path can be checked against it.  Only `tests/`, the smoke test
// and the benchmark's CPU-baseline leg load it; the product never does.
//
// What is restated (reference file:line, paths inside the NeuralAT project):
//   * Green's function and its normal derivatives, with the r >= 1e-3 clamp
//       src/bem/cuda/include/potential.h:16-52 (BM_LHS split: :55-65)
//   * Gauss-Legendre line rules (1..4 points) and the 1/3/4/6-point triangle
//     rules on the unit triangle               src/bem/cuda/include/gauss.h:5-127
//   * regular triangle-pair integrand, weight J1*J2/4
//                                              src/bem/cuda/include/integrand.h:187-235
//   * Sauter-Schwab singular quadrature on the reference triangle
//     (0,0),(1,0),(1,1): coincident / common-edge / common-vertex regions,
//     GL map [-1,1]->[0,1], weight J1*J2/16   src/bem/cuda/include/integrand.h:54-185
//   * vertex re-ordering so shared vertices come first, un-permutation
//                                              src/bem/cuda/include/integrand.h:331-394
//   * hypersingular / Burton-Miller curl-product combination
//                                              src/bem/cuda/include/integrand.h:296-323,
//                                              src/bem/cuda/bind.cu:128-143
//   * surface curls (n x grad phi) from (J^T J)^-1  src/bem/solver.py:40-58
//   * P1 mass matrix                          src/bem/cuda/include/integrand.h:257-278
//   * listener potential integrand            src/bem/cuda/include/integrand.h:237-255,396-406
//   * triangle -> vertex averaging            src/bem/cuda/bind.cu:23-48
// Row index = vertex of the test ("src") triangle, column = vertex of the
// trial ("trg") triangle, exactly as the reference scatters
// (src/bem/cuda/include/integrand.h:301-328).
//
// Quadrature constants are evaluated here from the closed forms of the
// published rules (Gauss-Legendre; Dunavant's degree-4 six-point triangle
// rule; Strang-Fix 3/4-point rules), not copied as literals.
//
// Built by oracle/Makefile into oracle/_build/libbem_oracle.so.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

enum Layer { SINGLE = 0, DOUBLE = 1, ADJOINT_DOUBLE = 2, HYPERSINGULAR = 3, BM_LHS = 4, BM_RHS = 5 };

const double kPi = 3.14159265358979323846;
const double kEps = 1e-3;  // potential.h:16 clamp on r

// ---- quadrature rules -----------------------------------------------------

// Gauss-Legendre nodes/weights on [-1, 1] (gauss.h:5-54 uses the same rules).
bool line_rule(int n, double* pts, double* wts) {
  switch (n) {
    case 1:
      pts[0] = 0.0;
      wts[0] = 2.0;
      return true;
    case 2: {
      double a = 1.0 / std::sqrt(3.0);
      pts[0] = a; pts[1] = -a;
      wts[0] = wts[1] = 1.0;
      return true;
    }
    case 3: {
      double a = std::sqrt(3.0 / 5.0);
      pts[0] = a; pts[1] = 0.0; pts[2] = -a;
      wts[0] = 5.0 / 9.0; wts[1] = 8.0 / 9.0; wts[2] = 5.0 / 9.0;
      return true;
    }
    case 4: {
      double s = 2.0 / 7.0 * std::sqrt(6.0 / 5.0);
      double a = std::sqrt(3.0 / 7.0 + s);  // outer node
      double b = std::sqrt(3.0 / 7.0 - s);  // inner node
      double wa = (18.0 - std::sqrt(30.0)) / 36.0;
      double wb = (18.0 + std::sqrt(30.0)) / 36.0;
      pts[0] = a; pts[1] = b; pts[2] = -b; pts[3] = -a;
      wts[0] = wa; wts[1] = wb; wts[2] = wb; wts[3] = wa;
      return true;
    }
  }
  return false;
}

// Triangle rules on the unit triangle (0,0),(1,0),(0,1); weights sum to 1.
// pts holds (x1, x2) pairs; barycentrics are (1-x1-x2, x1, x2).
bool tri_rule(int n, double* pts, double* wts) {
  switch (n) {
    case 1:
      pts[0] = pts[1] = 1.0 / 3.0;
      wts[0] = 1.0;
      return true;
    case 3: {
      // Strang-Fix degree-2 interior rule: (2/3, 1/6, 1/6) and permutations.
      const double a = 1.0 / 6.0, b = 2.0 / 3.0;
      const double P[3][2] = {{a, a}, {b, a}, {a, b}};
      for (int i = 0; i < 3; i++) { pts[2 * i] = P[i][0]; pts[2 * i + 1] = P[i][1]; wts[i] = 1.0 / 3.0; }
      return true;
    }
    case 4: {
      // Strang-Fix degree-3 rule: centroid (-27/48) and (3/5, 1/5, 1/5) orbit (25/48).
      const double P[4][2] = {{1.0 / 3.0, 1.0 / 3.0}, {0.2, 0.2}, {0.6, 0.2}, {0.2, 0.6}};
      const double W[4] = {-27.0 / 48.0, 25.0 / 48.0, 25.0 / 48.0, 25.0 / 48.0};
      for (int i = 0; i < 4; i++) { pts[2 * i] = P[i][0]; pts[2 * i + 1] = P[i][1]; wts[i] = W[i]; }
      return true;
    }
    case 6: {
      // Dunavant degree-4 rule: two orbits (a, a, 1-2a), closed forms below.
      const double r10 = std::sqrt(10.0);
      const double t = std::sqrt(38.0 - 44.0 * std::sqrt(2.0 / 5.0));
      const double a1 = (8.0 - r10 + t) / 18.0;  // ~0.44594849
      const double a2 = (8.0 - r10 - t) / 18.0;  // ~0.09157621
      const double w1 = (620.0 + std::sqrt(213125.0 - 53320.0 * r10)) / 3720.0;  // ~0.22338159
      const double w2 = (620.0 - std::sqrt(213125.0 - 53320.0 * r10)) / 3720.0;  // ~0.10995174
      const double P[6][2] = {{a1, a1}, {1 - 2 * a1, a1}, {a1, 1 - 2 * a1},
                              {a2, a2}, {1 - 2 * a2, a2}, {a2, 1 - 2 * a2}};
      const double W[6] = {w1, w1, w1, w2, w2, w2};
      for (int i = 0; i < 6; i++) { pts[2 * i] = P[i][0]; pts[2 * i + 1] = P[i][1]; wts[i] = W[i]; }
      return true;
    }
  }
  return false;
}

// ---- kernels (potential.h:18-65) -----------------------------------------
// Evaluates the integrand at (x, y).  `aux` is what the reference adds to the
// unweighted slot result[9]: for BM_LHS the (i/k) G term, otherwise `main`.
inline void kernel_eval(int layer, V3 x, V3 y, V3 xn, V3 yn, double k, cplx& main, cplx& aux) {
  V3 d = x - y;
  double r = norm(d);
  if (r < kEps) r = kEps;
  const cplx I(0.0, 1.0);
  cplx ikr = I * (r * k);
  cplx e = std::exp(ikr);
  switch (layer) {
    case SINGLE:
    case HYPERSINGULAR:  // hypersingular integrates G and recombines with curls
      main = e / (4.0 * kPi * r);
      break;
    case DOUBLE:
      main = -e / (4.0 * kPi * r * r * r) * (1.0 - ikr) * dot(y - x, yn);
      break;
    case ADJOINT_DOUBLE:
      main = -e / (4.0 * kPi * r * r * r) * (1.0 - ikr) * dot(x - y, xn);
      break;
    case BM_LHS: {
      cplx sp = e / (4.0 * kPi * r);
      main = (-I * k * dot(xn, yn) + 1.0 / (r * r) * (1.0 - ikr) * dot(y - x, yn)) * sp;
      aux = I / k * sp;
      return;
    }
    case BM_RHS: {
      cplx sp = e / (4.0 * kPi * r);
      main = -sp + I / k * sp / (r * r) * (1.0 - ikr) * dot(x - y, xn);
      break;
    }
  }
  aux = main;
}

struct Mesh {
  const double* v;
  const int* t;
  int nv, nt;
  V3 vert(int i) const { return {v[3 * i], v[3 * i + 1], v[3 * i + 2]}; }
  void tri(int i, int idx[3], V3 p[3]) const {
    for (int a = 0; a < 3; a++) { idx[a] = t[3 * i + a]; p[a] = vert(idx[a]); }
  }
};

inline V3 tri_normal(const V3 p[3]) {
  V3 n = cross(p[1] - p[0], p[2] - p[0]);
  return (1.0 / norm(n)) * n;
}
inline double tri_jac(const V3 p[3]) { return norm(cross(p[1] - p[0], p[2] - p[0])); }

// surface curls (n x grad phi_b), rows b = 0..2 (solver.py:40-58)
void surface_curls(const V3 p[3], double out[9]) {
  V3 e1 = p[1] - p[0], e2 = p[2] - p[0];
  V3 n = tri_normal(p);
  double g11 = dot(e1, e1), g12 = dot(e1, e2), g22 = dot(e2, e2);
  double det = g11 * g22 - g12 * g12;
  double i11 = g22 / det, i12 = -g12 / det, i22 = g11 / det;
  // J (J^T J)^-1 : columns c1, c2
  V3 c1 = i11 * e1 + i12 * e2;
  V3 c2 = i12 * e1 + i22 * e2;
  // reference gradients of phi: phi0 (-1,-1), phi1 (1,0), phi2 (0,1)
  V3 g[3] = {-1.0 * (c1 + c2), c1, c2};
  for (int b = 0; b < 3; b++) {
    V3 c = cross(n, g[b]);
    out[3 * b] = c.x; out[3 * b + 1] = c.y; out[3 * b + 2] = c.z;
  }
}

int common_vertices(const int a[3], const int b[3]) {
  int c = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) c += (a[i] == b[j]);
  return c;
}

// Regular pair integrand (integrand.h:187-235): result[0..8] (test a, trial b), result[9].
void regular_block(int layer, int tri_n, const V3 ti[3], const V3 tj[3], double k, cplx res[10]) {
  double pts[12], wts[6];
  tri_rule(tri_n, pts, wts);
  V3 ni = tri_normal(ti), nj = tri_normal(tj);
  double w1 = 0.25 * tri_jac(ti) * tri_jac(tj);
  for (int c = 0; c < 10; c++) res[c] = 0.0;
  for (int p = 0; p < tri_n; p++) {
    double lp[3] = {1 - pts[2 * p] - pts[2 * p + 1], pts[2 * p], pts[2 * p + 1]};
    V3 x = lp[0] * ti[0] + lp[1] * ti[1] + lp[2] * ti[2];
    for (int q = 0; q < tri_n; q++) {
      double lq[3] = {1 - pts[2 * q] - pts[2 * q + 1], pts[2 * q], pts[2 * q + 1]};
      V3 y = lq[0] * tj[0] + lq[1] * tj[1] + lq[2] * tj[2];
      double w2 = w1 * wts[p] * wts[q];
      cplx m, a;
      kernel_eval(layer, x, y, ni, nj, k, m, a);
      for (int ii = 0; ii < 3; ii++)
        for (int jj = 0; jj < 3; jj++) res[3 * ii + jj] += m * (w2 * lp[ii] * lq[jj]);
      res[9] += a * w2;
    }
  }
}

// Sauter-Schwab singular pair integrand (integrand.h:63-185, 331-394).
void singular_block(int layer, int line_n, const int si[3], const V3 ti[3], const int sj[3],
                    const V3 tj[3], double k, cplx res[10]) {
  int ncommon = common_vertices(si, sj);
  int pi[3] = {0, 1, 2}, pj[3] = {0, 1, 2};
  if (ncommon == 2) {
    int idx = 0;
    for (int jj = 0; jj < 3; jj++)
      for (int ii = 0; ii < 3; ii++)
        if (si[ii] == sj[jj] && idx < 2) { pi[idx] = ii; pj[idx] = jj; idx++; }
    pi[2] = 3 - pi[0] - pi[1];
    pj[2] = 3 - pj[0] - pj[1];
  } else if (ncommon == 1) {
    for (int ii = 0; ii < 3; ii++)
      for (int jj = 0; jj < 3; jj++)
        if (si[ii] == sj[jj]) {
          if (ii != 0) { pi[0] = ii; pi[ii] = 0; }
          if (jj != 0) { pj[0] = jj; pj[jj] = 0; }
        }
  }
  V3 a[3], b[3];
  for (int c = 0; c < 3; c++) { a[c] = ti[pi[c]]; b[c] = tj[pj[c]]; }
  V3 ni = tri_normal(ti), nj = tri_normal(tj);  // normals of the un-permuted triangles
  double jac = tri_jac(ti) * tri_jac(tj);

  double gp[4], gw[4];
  line_rule(line_n, gp, gw);
  cplx loc[10];
  for (int c = 0; c < 10; c++) loc[c] = 0.0;

  for (int i0 = 0; i0 < line_n; i0++)
    for (int i1 = 0; i1 < line_n; i1++)
      for (int i2 = 0; i2 < line_n; i2++)
        for (int i3 = 0; i3 < line_n; i3++) {
          double xi = 0.5 * (gp[i0] + 1), e1 = 0.5 * (gp[i1] + 1);
          double e2 = 0.5 * (gp[i2] + 1), e3 = 0.5 * (gp[i3] + 1);
          double weight = gw[i0] * gw[i1] * gw[i2] * gw[i3] * jac / 16.0;
          double e12 = e1 * e2, e123 = e1 * e2 * e3;
          cplx acc[10];
          for (int c = 0; c < 10; c++) acc[c] = 0.0;
          // one Sauter-Schwab region: points (x1,x2) on test, (y1,y2) on trial,
          // reference triangle (0,0),(1,0),(1,1) with shape (1-s, s-t, t)
          auto region = [&](double x1, double x2, double y1, double y2, double ww) {
            double lx[3] = {1 - x1, x1 - x2, x2};
            double ly[3] = {1 - y1, y1 - y2, y2};
            V3 x = lx[0] * a[0] + lx[1] * a[1] + lx[2] * a[2];
            V3 y = ly[0] * b[0] + ly[1] * b[1] + ly[2] * b[2];
            cplx m, au;
            kernel_eval(layer, x, y, ni, nj, k, m, au);
            m *= ww;
            au *= ww;
            for (int ii = 0; ii < 3; ii++)
              for (int jj = 0; jj < 3; jj++) acc[3 * ii + jj] += m * (lx[ii] * ly[jj]);
            acc[9] += au;
          };
          double w = 0.0;
          if (ncommon == 3) {
            w = xi * xi * xi * e1 * e1 * e2;
            region(xi, xi * (1.0 - e1 + e12), xi * (1.0 - e123), xi * (1.0 - e1), 1.0);
            region(xi * (1.0 - e123), xi * (1.0 - e1), xi, xi * (1.0 - e1 + e12), 1.0);
            region(xi, xi * (e1 - e12 + e123), xi * (1.0 - e12), xi * (e1 - e12), 1.0);
            region(xi * (1.0 - e12), xi * (e1 - e12), xi, xi * (e1 - e12 + e123), 1.0);
            region(xi * (1.0 - e123), xi * (e1 - e123), xi, xi * (e1 - e12), 1.0);
            region(xi, xi * (e1 - e12), xi * (1.0 - e123), xi * (e1 - e123), 1.0);
          } else if (ncommon == 2) {
            w = xi * xi * xi * e1 * e1;
            region(xi, xi * e1 * e3, xi * (1.0 - e12), xi * e1 * (1.0 - e2), 1.0);
            region(xi, xi * e1, xi * (1.0 - e123), xi * e1 * e2 * (1 - e3), e2);
            region(xi * (1.0 - e12), xi * e1 * (1.0 - e2), xi, xi * e123, e2);
            region(xi * (1.0 - e123), xi * e12 * (1.0 - e3), xi, xi * e1, e2);
            region(xi * (1.0 - e123), xi * e1 * (1.0 - e2 * e3), xi, xi * e12, e2);
          } else if (ncommon == 1) {
            w = xi * xi * xi * e2;
            region(xi, xi * e1, xi * e2, xi * e2 * e3, 1.0);
            region(xi * e2, xi * e2 * e3, xi, xi * e1, 1.0);
          }
          for (int c = 0; c < 10; c++) loc[c] += acc[c] * (w * weight);
        }
  for (int c = 0; c < 10; c++) res[c] = 0.0;
  for (int ii = 0; ii < 3; ii++)
    for (int jj = 0; jj < 3; jj++) res[3 * pi[ii] + pj[jj]] = loc[3 * ii + jj];
  res[9] = loc[9];
}

void combine_curls(int layer, cplx res[10], const double ci[9], const double cj[9], double nn, double k) {
  if (layer != HYPERSINGULAR && layer != BM_LHS) return;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      double cp = ci[3 * a] * cj[3 * b] + ci[3 * a + 1] * cj[3 * b + 1] + ci[3 * a + 2] * cj[3 * b + 2];
      if (layer == HYPERSINGULAR)
        res[3 * a + b] = res[9] * cp - res[3 * a + b] * (nn * k * k);
      else
        res[3 * a + b] = res[9] * cp + res[3 * a + b];
    }
}

inline void atomic_add(double* p, double v) {
#pragma omp atomic
  *p += v;
}

}  // namespace

extern "C" {

// Dense Galerkin boundary matrix of `layer` with line rule `line_n` (singular)
// and triangle rule `tri_n` (regular), bind.cu:49-154.
// vertices (nv,3) f64, triangles (nt,3) i32.  Output: complex128 interleaved,
// `nrows` x nv where row r is vertex rows[r] (rows == NULL: all nv rows).
int oracle_boundary_matrix(int layer, int line_n, int tri_n, const double* vertices, int nv,
                           const int* triangles, int nt, double k, const int* rows, int nrows,
                           double* out) {
  double tmp[12];
  if (!line_rule(line_n, tmp, tmp + 6) || !tri_rule(tri_n, tmp, tmp + 6)) return 1;
  Mesh m{vertices, triangles, nv, nt};
  std::vector<int> slot(nv, -1);
  if (rows) {
    for (int r = 0; r < nrows; r++) slot[rows[r]] = r;
  } else {
    nrows = nv;
    for (int r = 0; r < nv; r++) slot[r] = r;
  }
  std::memset(out, 0, sizeof(double) * 2 * (size_t)nrows * nv);
  std::vector<double> curls(9 * (size_t)nt);
  for (int i = 0; i < nt; i++) {
    int id[3];
    V3 p[3];
    m.tri(i, id, p);
    surface_curls(p, &curls[9 * (size_t)i]);
  }
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nt; i++) {
    int si[3];
    V3 ti[3];
    m.tri(i, si, ti);
    if (slot[si[0]] < 0 && slot[si[1]] < 0 && slot[si[2]] < 0) continue;
    V3 ni = tri_normal(ti);
    std::vector<cplx> rowacc(3 * (size_t)nv, cplx(0.0, 0.0));
    for (int j = 0; j < nt; j++) {
      int sj[3];
      V3 tj[3];
      m.tri(j, sj, tj);
      cplx res[10];
      if (common_vertices(si, sj) == 0)
        regular_block(layer, tri_n, ti, tj, k, res);
      else
        singular_block(layer, line_n, si, ti, sj, tj, k, res);
      combine_curls(layer, res, &curls[9 * (size_t)i], &curls[9 * (size_t)j], dot(ni, tri_normal(tj)), k);
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) rowacc[(size_t)a * nv + sj[b]] += res[3 * a + b];
    }
    for (int a = 0; a < 3; a++) {
      int r = slot[si[a]];
      if (r < 0) continue;
      double* o = out + 2 * (size_t)r * nv;
      for (int b = 0; b < nv; b++) {
        cplx v = rowacc[(size_t)a * nv + b];
        if (v.real() != 0.0 || v.imag() != 0.0) {
          atomic_add(o + 2 * b, v.real());
          atomic_add(o + 2 * b + 1, v.imag());
        }
      }
    }
  }
  return 0;
}

// Selected COLUMNS of the same matrix: output complex128 interleaved, nv x
// ncols, column c = vertex cols[c] (the trial-vertex side, bind.cu:144-151).
// Only trial triangles touching a selected vertex contribute, so a few
// columns cost a few rows' worth of work (used by the finite-difference
// checker of the vertex gradient, which updates the rows and columns a
// moved vertex touches).
int oracle_boundary_matrix_cols(int layer, int line_n, int tri_n, const double* vertices, int nv,
                                const int* triangles, int nt, double k, const int* cols, int ncols, double* out) {
  double tmp[12];
  if (!line_rule(line_n, tmp, tmp + 6) || !tri_rule(tri_n, tmp, tmp + 6)) return 1;
  if (!cols || ncols <= 0) return 2;
  Mesh m{vertices, triangles, nv, nt};
  std::vector<int> slot(nv, -1);
  for (int c = 0; c < ncols; c++) slot[cols[c]] = c;
  std::memset(out, 0, sizeof(double) * 2 * (size_t)nv * ncols);
  std::vector<double> curls(9 * (size_t)nt);
  std::vector<int> trial;
  for (int j = 0; j < nt; j++) {
    int id[3];
    V3 p[3];
    m.tri(j, id, p);
    surface_curls(p, &curls[9 * (size_t)j]);
    if (slot[id[0]] >= 0 || slot[id[1]] >= 0 || slot[id[2]] >= 0) trial.push_back(j);
  }
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    int si[3];
    V3 ti[3];
    m.tri(i, si, ti);
    V3 ni = tri_normal(ti);
    for (int j : trial) {
      int sj[3];
      V3 tj[3];
      m.tri(j, sj, tj);
      cplx res[10];
      if (common_vertices(si, sj) == 0)
        regular_block(layer, tri_n, ti, tj, k, res);
      else
        singular_block(layer, line_n, si, ti, sj, tj, k, res);
      combine_curls(layer, res, &curls[9 * (size_t)i], &curls[9 * (size_t)j], dot(ni, tri_normal(tj)), k);
      for (int b = 0; b < 3; b++) {
        const int c = slot[sj[b]];
        if (c < 0) continue;
        for (int a = 0; a < 3; a++) {
          double* o = out + 2 * ((size_t)si[a] * ncols + c);
          atomic_add(o, res[3 * a + b].real());
          atomic_add(o + 1, res[3 * a + b].imag());
        }
      }
    }
  }
  return 0;
}

// One 3x3 pair block (plus the unweighted slot 9), for unit tests of the
// quadrature itself.  Triangles i and j of the mesh; output 10 complex.
int oracle_pair_block(int layer, int line_n, int tri_n, const double* vertices, int nv,
                      const int* triangles, int nt, int i, int j, double k, double* out) {
  if (i < 0 || j < 0 || i >= nt || j >= nt) return 1;
  Mesh m{vertices, triangles, nv, nt};
  int si[3], sj[3];
  V3 ti[3], tj[3];
  m.tri(i, si, ti);
  m.tri(j, sj, tj);
  cplx res[10];
  if (common_vertices(si, sj) == 0)
    regular_block(layer, tri_n, ti, tj, k, res);
  else
    singular_block(layer, line_n, si, ti, sj, tj, k, res);
  double ci[9], cj[9];
  surface_curls(ti, ci);
  surface_curls(tj, cj);
  combine_curls(layer, res, ci, cj, dot(tri_normal(ti), tri_normal(tj)), k);
  for (int c = 0; c < 10; c++) { out[2 * c] = res[c].real(); out[2 * c + 1] = res[c].imag(); }
  return 0;
}

// P1 mass matrix, dense nv x nv complex128 (integrand.h:257-278).
int oracle_identity_matrix(const double* vertices, int nv, const int* triangles, int nt, double* out) {
  Mesh m{vertices, triangles, nv, nt};
  double pts[12], wts[6];
  tri_rule(6, pts, wts);
  std::memset(out, 0, sizeof(double) * 2 * (size_t)nv * nv);
  for (int i = 0; i < nt; i++) {
    int s[3];
    V3 p[3];
    m.tri(i, s, p);
    double w = 0.5 * tri_jac(p);
    for (int q = 0; q < 6; q++) {
      double l[3] = {1 - pts[2 * q] - pts[2 * q + 1], pts[2 * q], pts[2 * q + 1]};
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) out[2 * ((size_t)s[a] * nv + s[b])] += wts[q] * w * l[a] * l[b];
    }
  }
  return 0;
}

// Listener potential matrix (np x nv complex128) for SINGLE or DOUBLE,
// six-point rule per triangle, no singular treatment (bind.cu:156-176).
int oracle_potential_matrix(int layer, const double* vertices, int nv, const int* triangles, int nt,
                            const double* points, int np, double k, double* out) {
  if (layer != SINGLE && layer != DOUBLE) return 1;
  Mesh m{vertices, triangles, nv, nt};
  double pts[12], wts[6];
  tri_rule(6, pts, wts);
  std::memset(out, 0, sizeof(double) * 2 * (size_t)np * nv);
#pragma omp parallel for schedule(static)
  for (int p = 0; p < np; p++) {
    V3 x{points[3 * p], points[3 * p + 1], points[3 * p + 2]};
    V3 zero{0, 0, 0};
    double* row = out + 2 * (size_t)p * nv;
    for (int j = 0; j < nt; j++) {
      int s[3];
      V3 t[3];
      m.tri(j, s, t);
      V3 n = tri_normal(t);
      double w1 = 0.5 * tri_jac(t);
      for (int q = 0; q < 6; q++) {
        double l[3] = {1 - pts[2 * q] - pts[2 * q + 1], pts[2 * q], pts[2 * q + 1]};
        V3 y = l[0] * t[0] + l[1] * t[1] + l[2] * t[2];
        cplx g, aux;
        kernel_eval(layer, x, y, zero, n, k, g, aux);
        g *= w1 * wts[q];
        for (int a = 0; a < 3; a++) {
          row[2 * s[a]] += g.real() * l[a];
          row[2 * s[a] + 1] += g.imag() * l[a];
        }
      }
    }
  }
  return 0;
}

// Per-triangle complex values averaged onto vertices (bind.cu:23-48).
int oracle_triangle2vertex(int nv, const int* triangles, int nt, const double* tri_values, double* out) {
  std::vector<int> count(nv, 0);
  std::memset(out, 0, sizeof(double) * 2 * (size_t)nv);
  for (int i = 0; i < nt; i++)
    for (int a = 0; a < 3; a++) {
      int v = triangles[3 * i + a];
      out[2 * v] += tri_values[2 * i];
      out[2 * v + 1] += tri_values[2 * i + 1];
      count[v]++;
    }
  for (int v = 0; v < nv; v++) {
    // the reference divides by the count unconditionally; an isolated vertex gives 0/0
    out[2 * v] /= count[v];
    out[2 * v + 1] /= count[v];
  }
  return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

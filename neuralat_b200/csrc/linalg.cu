// Dense complex linear algebra for the BEM solve.
//
// Replaces, for this path, the torch/cuBLAS complex gemv the reference calls
// (src/bem/solver.py:103,147) and the host-driven Python BiCGSTAB loop with
// two device->host syncs per iteration (src/bem/BiCGSTAB.py:48-107).
//
//  * cmatmul_kernel: Y = A X (or R = B - A X with column norms) for an n x n
//    complex64 matrix and m <= 8 right-hand sides per pass, HBM-streaming:
//    each warp owns 4 rows, the X tile is staged in shared memory and reused
//    by the 4 rows, lanes read A rows coalesced.  Accumulation in float or
//    double (the latter is the FP64 refinement residual).
//  * restarted GMRES, one Krylov space per right-hand side sharing every
//    operator application: Arnoldi in FP64 with classical Gram-Schmidt and
//    re-orthogonalisation (CGS2), complex Givens rotations in FP64, all state
//    on the device; the host only watches a convergence flag through events,
//    without stalling the GPU.  Outer FP64 iterative refinement
//    r = b - A x against the FP32 matrix.

#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "bem_common.cuh"

namespace bemb {

// tensor-core operator (tc_matvec.cu)
int tc_operator_prepare(const float2* A, int n, int precision, void* ws, cudaStream_t s);
int tc_matvec(const void* ws, int n, int precision, const float2* X, int m, float2* Y, const int* skip,
              cudaStream_t s);
int tc_error(const void* ws, int* err_host, cudaStream_t s);
size_t tc_workspace_bytes(int n, int m, int precision);

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

template <typename T>
struct C2;
template <>
struct C2<float> {
  typedef float2 type;
};
template <>
struct C2<double> {
  typedef double2 type;
};

constexpr int kMMThreads = 256;
constexpr int kMMColTile = 128;
// rows per warp: 4 in FP32 (X tile reused 4x), 2 in FP64 (register budget)
template <typename T>
struct MMRows {
  static constexpr int kPerWarp = sizeof(T) == 4 ? 4 : 2;
  static constexpr int kPerBlock = kPerWarp * (kMMThreads / 32);
};

// MODE 0: Y[i, s] = sum_j A[i, j] X[j, s]
// MODE 1: Y[i, s] = B[i, s] - sum_j A[i, j] X[j, s], norm2[s] += |Y[i,s]|^2
// X, Y, B are (n, ldx/ldy) row-major; MR right-hand sides per pass.
template <typename T, int MR, int MODE>
__global__ void __launch_bounds__(kMMThreads)
    cmatmul_kernel(const float2* __restrict__ A, int n, const typename C2<T>::type* __restrict__ X, int ldx,
                   int m, typename C2<T>::type* __restrict__ Y, int ldy, const float2* __restrict__ B, int ldb,
                   double* __restrict__ norm2, const int* __restrict__ skip) {
  typedef typename C2<T>::type CT;
  constexpr int kMMRowsPerWarp = MMRows<T>::kPerWarp;
  constexpr int kMMRows = MMRows<T>::kPerBlock;
  if (skip && *skip) return;
  __shared__ CT xs[MR][kMMColTile];  // [rhs][column]: lanes read consecutive columns
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row0 = blockIdx.x * kMMRows + warp * kMMRowsPerWarp;
  const int s0 = blockIdx.y * MR;
  const int ms = min(MR, m - s0);
  T acc[kMMRowsPerWarp][MR][2];
#pragma unroll
  for (int r = 0; r < kMMRowsPerWarp; r++)
#pragma unroll
    for (int s = 0; s < MR; s++) acc[r][s][0] = acc[r][s][1] = T(0);

  for (int c0 = 0; c0 < n; c0 += kMMColTile) {
    __syncthreads();
    for (int e = threadIdx.x; e < kMMColTile * MR; e += kMMThreads) {
      const int c = e / MR, s = e - (e / MR) * MR;
      CT v;
      v.x = T(0);
      v.y = T(0);
      if (c0 + c < n && s < ms) v = X[(size_t)(c0 + c) * ldx + s0 + s];
      xs[s][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kMMColTile / 32; u++) {
      const int c = u * 32 + lane;
      const int col = c0 + c;
      float2 a[kMMRowsPerWarp];
#pragma unroll
      for (int r = 0; r < kMMRowsPerWarp; r++) {
        const int row = row0 + r;
        a[r] = (row < n && col < n) ? __ldcs(&A[(size_t)row * n + col]) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int s = 0; s < MR; s++) {
        const CT x = xs[s][c];
#pragma unroll
        for (int r = 0; r < kMMRowsPerWarp; r++) {
          const T ar = (T)a[r].x, ai = (T)a[r].y;
          acc[r][s][0] = fma(ar, x.x, fma(-ai, x.y, acc[r][s][0]));
          acc[r][s][1] = fma(ar, x.y, fma(ai, x.x, acc[r][s][1]));
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kMMRowsPerWarp; r++)
#pragma unroll
    for (int s = 0; s < MR; s++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        T v = acc[r][s][h];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[r][s][h] = v;
      }
  // lane (r * MR + s) writes entry (row0 + r, s0 + s)
#pragma unroll
  for (int r = 0; r < kMMRowsPerWarp; r++)
#pragma unroll
    for (int s = 0; s < MR; s++) {
      if (lane == r * MR + s) {
        const int row = row0 + r;
        if (row < n && s < ms) {
          CT out;
          if (MODE == 0) {
            out.x = acc[r][s][0];
            out.y = acc[r][s][1];
          } else {
            const float2 b = B[(size_t)row * ldb + s0 + s];
            out.x = (T)b.x - acc[r][s][0];
            out.y = (T)b.y - acc[r][s][1];
            atomicAdd(&norm2[s0 + s], (double)out.x * (double)out.x + (double)out.y * (double)out.y);
          }
          Y[(size_t)row * ldy + s0 + s] = out;
        }
      }
    }
}

template <typename T, int MODE>
int launch_cmatmul(const float2* A, int n, const typename C2<T>::type* X, int ldx, int m, typename C2<T>::type* Y,
                   int ldy, const float2* B, int ldb, double* norm2, const int* skip, cudaStream_t s) {
  const int rb = (n + MMRows<T>::kPerBlock - 1) / MMRows<T>::kPerBlock;
  if (m == 1) {
    (cmatmul_kernel<T, 1, MODE><<<dim3(rb, 1), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2, skip), count_launch());
  } else if (m == 2) {
    (cmatmul_kernel<T, 2, MODE><<<dim3(rb, 1), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2, skip), count_launch());
  } else if (m <= 4) {
    (cmatmul_kernel<T, 4, MODE><<<dim3(rb, 1), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2, skip), count_launch());
  } else {
    (cmatmul_kernel<T, 8, MODE><<<dim3(rb, (m + 7) / 8), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2,
                                                                          skip), count_launch());
  }
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// GMRES state and kernels
// ---------------------------------------------------------------------------
struct GmState {
  int k;           // Arnoldi step inside the current cycle (same for all active columns)
  int any_active;  // 0 when every column has converged (matvec early-out)
  int skip;        // == !any_active, read by the matvec kernel
  int pad;
  int any_count;   // scratch counters of gm_finalize_kernel (zero between launches)
  int done_blocks;
  int act_count;   // columns active when the step started (scratch)
  int iters_done;  // Arnoldi steps executed with at least one active column
};

struct GmPtrs {
  int n, m, R;
  float2* Vb;      // [m][R+1][n]  Krylov basis, complex64 storage
  double2* H;      // [m][R][R+1]  column k, rows 0..k+1
  double* cs;      // [m][R]
  double2* sn;     // [m][R]
  double2* g;      // [m][R+1]
  double2* h;      // [2][m][R+1]  dots of the two CGS passes
  double2* w;      // [m][n]
  double2* d;      // [m][n]  inner correction
  double2* x;      // [n][m]  solution (FP64)
  double2* r;      // [n][m]  outer residual (FP64)
  float2* X;       // [n][m]  matvec input
  float2* Y;       // [n][m]  matvec output
  double* norm2;   // [m]  |w|^2 accumulator of the current step
  double* winv;    // [m]  1 / h_{k+1,k} of the previous step
  double* beta;    // [m]
  double* tol;     // [m] inner absolute tolerance
  double* resid;   // [m]
  int* active;     // [m]
  int* kend;       // [m]  basis size used by each column in this cycle
  double* y;       // [m][R]
  GmState* st;
  double* bnorm2;  // [m]
};

// X[:, s] = float(V[s][k]) after normalising w into V[s][k] (k > 0).
__global__ void gm_pack_kernel(GmPtrs P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  const int k = P.st->k;
  float2* vk = P.Vb + ((size_t)s * (P.R + 1) + k) * P.n;
  if (P.active[s]) {
    float2 v;
    if (k > 0) {
      const double inv = P.winv[s];
      const double2 ww = P.w[(size_t)s * P.n + i];
      v = make_float2((float)(ww.x * inv), (float)(ww.y * inv));
      vk[i] = v;
    } else {
      v = vk[i];
    }
    P.X[(size_t)i * P.m + s] = v;
  } else {
    P.X[(size_t)i * P.m + s] = make_float2(0.f, 0.f);
  }
}

// w_s = double(Y[:, s]) for active columns (Y is (n, m) row-major; w is
// column-major, so both Gram-Schmidt passes read contiguous vectors).
__global__ void gm_y2w_kernel(GmPtrs P) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)P.n * P.m) return;
  const int i = (int)(idx / P.m), s = (int)(idx - (long long)i * P.m);
  if (!P.active[s]) return;
  const float2 y = P.Y[idx];
  P.w[(size_t)s * P.n + i] = make_double2(y.x, y.y);
}

// h[pass][s][l] += <V[s][l], w_s> over one chunk of rows, for a group of
// kDotL basis vectors: every thread keeps 8 rows of w in registers and issues
// 8 x kDotL independent loads; partial sums reach h through FP64 atomics
// (h is zeroed at the start of a cycle and after each use).
constexpr int kDotThreads = 256;
constexpr int kDotRowsPerThread = 8;
constexpr int kDotRows = kDotThreads * kDotRowsPerThread;  // 2048
constexpr int kDotL = 8;
__global__ void __launch_bounds__(kDotThreads) gm_dots_kernel(GmPtrs P, int pass) {
  const int s = blockIdx.z;
  if (!P.active[s]) return;
  const int k = P.st->k;
  const int l0 = blockIdx.y * kDotL;
  if (l0 > k) return;
  const int nl = min(kDotL, k + 1 - l0);
  const int row0 = blockIdx.x * kDotRows;
  double2 src[kDotRowsPerThread];
#pragma unroll
  for (int u = 0; u < kDotRowsPerThread; u++) {
    const int i = row0 + threadIdx.x + u * kDotThreads;
    src[u] = i < P.n ? P.w[(size_t)s * P.n + i] : make_double2(0.0, 0.0);
  }
  double re[kDotL], im[kDotL];
#pragma unroll
  for (int ll = 0; ll < kDotL; ll++) {
    re[ll] = 0.0;
    im[ll] = 0.0;
    if (ll < nl) {
      const float2* v = P.Vb + ((size_t)s * (P.R + 1) + l0 + ll) * P.n;
#pragma unroll
      for (int u = 0; u < kDotRowsPerThread; u++) {
        const int i = row0 + threadIdx.x + u * kDotThreads;
        if (i < P.n) {
          const float2 vv = v[i];
          re[ll] += (double)vv.x * src[u].x + (double)vv.y * src[u].y;  // conj(v) w
          im[ll] += (double)vv.x * src[u].y - (double)vv.y * src[u].x;
        }
      }
    }
  }
  __shared__ double red[kDotThreads / 32][kDotL][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int ll = 0; ll < kDotL; ll++) {
    double a = re[ll], b = im[ll];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
      red[warp][ll][0] = a;
      red[warp][ll][1] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * nl) {
    const int ll = threadIdx.x >> 1, c = threadIdx.x & 1;
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kDotThreads / 32; w++) t += red[w][ll][c];
    double* h = (double*)(P.h + ((size_t)pass * P.m + s) * (P.R + 1) + l0 + ll);
    atomicAdd(h + c, t);
  }
}

// w_s = src_s - sum_{l<=k} V[s][l] h[pass][s][l]; pass 1 also accumulates |w|^2.
__global__ void gm_update_kernel(GmPtrs P, int pass) {
  const int s = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = P.st->k;
  if (!P.active[s]) return;
  __shared__ double2 hs[256];
  for (int l = threadIdx.x; l <= k; l += blockDim.x) hs[l] = P.h[((size_t)pass * P.m + s) * (P.R + 1) + l];
  __syncthreads();
  double n2 = 0.0;
  if (i < P.n) {
    double2 acc = P.w[(size_t)s * P.n + i];
    const float2* v = P.Vb + (size_t)s * (P.R + 1) * P.n + i;
    // batches of 8 independent loads, two accumulators
    double2 acc2 = make_double2(0.0, 0.0);
    int l = 0;
    for (; l + 8 <= k + 1; l += 8) {
      float2 vv[8];
#pragma unroll
      for (int u = 0; u < 8; u++) vv[u] = v[(size_t)(l + u) * P.n];
#pragma unroll
      for (int u = 0; u < 8; u += 2) {
        const double2 t0 = cmul(make_double2(vv[u].x, vv[u].y), hs[l + u]);
        const double2 t1 = cmul(make_double2(vv[u + 1].x, vv[u + 1].y), hs[l + u + 1]);
        acc.x -= t0.x;
        acc.y -= t0.y;
        acc2.x -= t1.x;
        acc2.y -= t1.y;
      }
    }
    for (; l <= k; l++) {
      const float2 vv = v[(size_t)l * P.n];
      const double2 t = cmul(make_double2(vv.x, vv.y), hs[l]);
      acc.x -= t.x;
      acc.y -= t.y;
    }
    acc.x += acc2.x;
    acc.y += acc2.y;
    P.w[(size_t)s * P.n + i] = acc;
    n2 = acc.x * acc.x + acc.y * acc.y;
  }
  if (pass == 1) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    if ((threadIdx.x & 31) == 0 && n2 != 0.0) atomicAdd(&P.norm2[s], n2);
  }
}

// Hessenberg column, Givens rotations, residual estimate, convergence.  One
// warp per column: the lanes stage the new column and the previous rotations
// in shared memory, lane 0 applies the rotations (inherently sequential); the
// last block to finish advances k.  One block per kFinWarps columns.
constexpr int kFinWarps = 4;  // 40 KB of static shared memory
constexpr int kMaxRestart = 256;
__global__ void __launch_bounds__(32 * kFinWarps) gm_finalize_kernel(GmPtrs P, int* __restrict__ any_count,
                                                                     int* __restrict__ done_blocks) {
  __shared__ double2 hcol[kFinWarps][kMaxRestart + 1];
  __shared__ double csv[kFinWarps][kMaxRestart];
  __shared__ double2 snv[kFinWarps][kMaxRestart];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int s = blockIdx.x * kFinWarps + wl;
  const int k = P.st->k;
  if (s < P.m && P.active[s] && lane == 0) atomicAdd(&P.st->act_count, 1);
  if (s < P.m && P.active[s]) {
    const double2* h0 = P.h + ((size_t)0 * P.m + s) * (P.R + 1);
    const double2* h1 = P.h + ((size_t)1 * P.m + s) * (P.R + 1);
    for (int l = lane; l <= k; l += 32) {
      hcol[wl][l] = make_double2(h0[l].x + h1[l].x, h0[l].y + h1[l].y);
      if (l < k) {
        csv[wl][l] = P.cs[s * P.R + l];
        snv[wl][l] = P.sn[s * P.R + l];
      }
    }
    __syncwarp();
    double2* Hk = P.H + ((size_t)s * P.R + k) * (P.R + 1);
    const double hn = sqrt(P.norm2[s]);
    if (lane == 0) {
      double2* hc = hcol[wl];
      hc[k + 1] = make_double2(hn, 0.0);
      for (int l = 0; l < k; l++) {
        const double c = csv[wl][l];
        const double2 sn = snv[wl][l];
        const double2 a = hc[l], b = hc[l + 1];
        const double2 sb = cmul(sn, b);
        const double2 t = cmul(make_double2(-sn.x, sn.y), a);  // -conj(sn) a
        hc[l] = make_double2(c * a.x + sb.x, c * a.y + sb.y);
        hc[l + 1] = make_double2(t.x + c * b.x, t.y + c * b.y);
      }
      const double2 a = hc[k], b = hc[k + 1];
      const double na = sqrt(a.x * a.x + a.y * a.y), nb = sqrt(b.x * b.x + b.y * b.y);
      const double rho = sqrt(na * na + nb * nb);
      double c;
      double2 sn;
      if (rho == 0.0) {
        c = 1.0;
        sn = make_double2(0.0, 0.0);
      } else if (na == 0.0) {
        c = 0.0;
        sn = make_double2(b.x / nb, -b.y / nb);  // conj(b)/|b|
        hc[k] = make_double2(nb, 0.0);
      } else {
        c = na / rho;
        const double2 ph = make_double2(a.x / na, a.y / na);
        sn = cmul(ph, make_double2(b.x / rho, -b.y / rho));
        hc[k] = make_double2(ph.x * rho, ph.y * rho);
      }
      hc[k + 1] = make_double2(0.0, 0.0);
      P.cs[s * P.R + k] = c;
      P.sn[s * P.R + k] = sn;
      double2* gs = P.g + (size_t)s * (P.R + 1);
      const double2 gk = gs[k];
      gs[k + 1] = cmul(make_double2(-sn.x, sn.y), gk);
      gs[k] = make_double2(c * gk.x, c * gk.y);
      const double res = sqrt(gs[k + 1].x * gs[k + 1].x + gs[k + 1].y * gs[k + 1].y);
      P.resid[s] = res;
      P.kend[s] = k + 1;
      P.winv[s] = hn > 0.0 ? 1.0 / hn : 0.0;
      const bool breakdown = !(hn > 1e-300) || !(hn > 1e-14 * rho);
      if (res <= P.tol[s] || breakdown || k + 1 >= P.R) {
        P.active[s] = 0;
      } else {
        atomicAdd(any_count, 1);
      }
    }
    __syncwarp();
    for (int l = lane; l <= k + 1; l += 32) Hk[l] = hcol[wl][l];
    double2* h0w = P.h + ((size_t)0 * P.m + s) * (P.R + 1);
    double2* h1w = P.h + ((size_t)1 * P.m + s) * (P.R + 1);
    for (int l = lane; l <= k; l += 32) {
      h0w[l] = make_double2(0.0, 0.0);
      h1w[l] = make_double2(0.0, 0.0);
    }
  }
  if (s < P.m && lane == 0) P.norm2[s] = 0.0;
  // the last block to finish publishes k + 1 and the activity flag
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const int done = atomicAdd(done_blocks, 1);
    if (done == (int)gridDim.x - 1) {
      __threadfence();
      const int any = atomicAdd(any_count, 0);
      if (atomicAdd(&P.st->act_count, 0) > 0) P.st->iters_done += 1;
      P.st->act_count = 0;
      P.st->k = k + 1;
      P.st->any_active = any;
      P.st->skip = any ? 0 : 1;
      *any_count = 0;
      *done_blocks = 0;
    }
  }
}

// Back substitution H y = g on the Givens-reduced Hessenberg matrix, one
// warp per column, column-oriented: y_j = g_j / H_jj, then the lanes update
// g_0..g_{j-1} -= y_j H_{0..j-1, j} (column j of H is contiguous).
constexpr int kSolveWarps = 4;
__global__ void __launch_bounds__(32 * kSolveWarps) gm_solve_kernel(GmPtrs P) {
  __shared__ double2 gsh[kSolveWarps][kMaxRestart + 1];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int s = blockIdx.x * kSolveWarps + wl;
  if (s >= P.m) return;
  const int kk = P.kend[s];
  const double2* gs = P.g + (size_t)s * (P.R + 1);
  double2* y = (double2*)(P.y) + (size_t)s * P.R;
  for (int l = lane; l < kk; l += 32) gsh[wl][l] = gs[l];
  __syncwarp();
  for (int j = kk - 1; j >= 0; j--) {
    const double2* Hj = P.H + ((size_t)s * P.R + j) * (P.R + 1);  // column j, rows 0..j
    const double2 hd = Hj[j];
    const double den = hd.x * hd.x + hd.y * hd.y;
    const double2 gj = gsh[wl][j];
    const double2 yj = den > 0.0 ? make_double2((gj.x * hd.x + gj.y * hd.y) / den, (gj.y * hd.x - gj.x * hd.y) / den)
                                 : make_double2(0.0, 0.0);
    if (lane == 0) y[j] = yj;
    for (int l = lane; l < j; l += 32) {
      const double2 t = cmul(Hj[l], yj);
      gsh[wl][l].x -= t.x;
      gsh[wl][l].y -= t.y;
    }
    __syncwarp();
  }
}

__global__ void gm_xupdate_kernel(GmPtrs P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  const int kk = P.kend[s];
  const double2* y = (const double2*)(P.y) + (size_t)s * P.R;
  double2 acc = P.d[(size_t)s * P.n + i];
  const float2* v = P.Vb + (size_t)s * (P.R + 1) * P.n + i;
  for (int l = 0; l < kk; l++) {
    const float2 vv = v[(size_t)l * P.n];
    const double2 t = cmul(make_double2(vv.x, vv.y), y[l]);
    acc.x += t.x;
    acc.y += t.y;
  }
  P.d[(size_t)s * P.n + i] = acc;
}

// Cycle start: r_in = r_out (first cycle) or r_out - Y (later cycles);
// V[s][0] = r_in / ||r_in||, g = (beta, 0, ...).  norm2 holds ||r_in||^2.
__global__ void gm_start_vec_kernel(GmPtrs P, int use_y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  double2 r = P.r[(size_t)i * P.m + s];
  if (use_y) {
    const float2 y = P.Y[(size_t)i * P.m + s];
    r.x -= y.x;
    r.y -= y.y;
  }
  P.w[(size_t)s * P.n + i] = r;
  double n2 = r.x * r.x + r.y * r.y;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if ((threadIdx.x & 31) == 0 && n2 != 0.0) atomicAdd(&P.norm2[s], n2);
}

__global__ void gm_start_scalar_kernel(GmPtrs P, const double* __restrict__ outer_norm2, double inner_rtol,
                                       double floor_abs_rtol) {
  const int s = threadIdx.x;
  __shared__ int any;
  if (s == 0) any = 0;
  __syncthreads();
  if (s < P.m) {
    const double beta = sqrt(P.norm2[s]);
    P.beta[s] = beta;
    const double rout = sqrt(outer_norm2[s]);
    const double target = fmax(inner_rtol * rout, floor_abs_rtol * sqrt(P.bnorm2[s]));
    P.tol[s] = target;
    double2* gs = P.g + (size_t)s * (P.R + 1);
    gs[0] = make_double2(beta, 0.0);
    P.kend[s] = 0;
    P.resid[s] = beta;
    const int act = beta > target && beta > 0.0;
    P.active[s] = act;
    if (act) atomicAdd(&any, 1);
    P.norm2[s] = 0.0;
  }
  __syncthreads();
  if (s == 0) {
    P.st->k = 0;
    P.st->any_active = any;
    P.st->skip = any ? 0 : 1;
  }
}

// V[s][0] = w_s / beta_s
__global__ void gm_start_norm_kernel(GmPtrs P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  const double b = P.beta[s];
  const double inv = b > 0.0 ? 1.0 / b : 0.0;
  const double2 w = P.w[(size_t)s * P.n + i];
  P.Vb[(size_t)s * (P.R + 1) * P.n + i] = make_float2((float)(w.x * inv), (float)(w.y * inv));
}

// X = float(d) (for r_out - A_lp d), or X = 0
__global__ void gm_pack_d_kernel(GmPtrs P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  const double2 v = P.d[(size_t)s * P.n + i];
  P.X[(size_t)i * P.m + s] = make_float2((float)v.x, (float)v.y);
}

// x += d, d = 0
__global__ void gm_accept_kernel(GmPtrs P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  double2& dd = P.d[(size_t)s * P.n + i];
  double2& xx = P.x[(size_t)i * P.m + s];
  xx.x += dd.x;
  xx.y += dd.y;
  dd = make_double2(0.0, 0.0);
}

__global__ void gm_init_x_kernel(GmPtrs P, const float2* __restrict__ X0, int use_x0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  double2 v = make_double2(0.0, 0.0);
  if (use_x0) {
    const float2 x0 = X0[(size_t)i * P.m + s];
    v = make_double2(x0.x, x0.y);
  }
  P.x[(size_t)i * P.m + s] = v;
  P.d[(size_t)s * P.n + i] = make_double2(0.0, 0.0);
}

__global__ void gm_bnorm_kernel(GmPtrs P, const float2* __restrict__ B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  double n2 = 0.0;
  if (i < P.n) {
    const float2 b = B[(size_t)i * P.m + s];
    n2 = (double)b.x * b.x + (double)b.y * b.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if ((threadIdx.x & 31) == 0 && n2 != 0.0) atomicAdd(&P.bnorm2[s], n2);
}

// r = b (zero initial guess), rnorm2 += |b|^2
__global__ void gm_copy_b_kernel(GmPtrs P, const float2* __restrict__ B, double* __restrict__ rnorm2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  double n2 = 0.0;
  if (i < P.n) {
    const float2 b = B[(size_t)i * P.m + s];
    P.r[(size_t)i * P.m + s] = make_double2(b.x, b.y);
    n2 = (double)b.x * b.x + (double)b.y * b.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if ((threadIdx.x & 31) == 0 && n2 != 0.0) atomicAdd(&rnorm2[s], n2);
}

__global__ void gm_store_x_kernel(GmPtrs P, float2* __restrict__ X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= P.n) return;
  const double2 v = P.x[(size_t)i * P.m + s];
  X[(size_t)i * P.m + s] = make_float2((float)v.x, (float)v.y);
}

inline size_t al(size_t x) { return (x + 255) / 256 * 256; }

struct Layout {
  size_t Vb, H, cs, sn, g, h, w, d, x, r, X, Y, norm2, winv, rnorm2, beta, tol, resid, active, kend, y, st, bnorm2, tc,
      total;
};

Layout layout(int n, int m, int R, int precision) {
  Layout L;
  size_t o = 0;
  auto take = [&](size_t b) {
    size_t r = o;
    o = al(o + b);
    return r;
  };
  L.st = take(sizeof(GmState));
  L.Vb = take(sizeof(float2) * (size_t)m * (R + 1) * n);
  L.H = take(sizeof(double2) * (size_t)m * R * (R + 1));
  L.cs = take(sizeof(double) * (size_t)m * R);
  L.sn = take(sizeof(double2) * (size_t)m * R);
  L.g = take(sizeof(double2) * (size_t)m * (R + 1));
  L.h = take(sizeof(double2) * 2 * (size_t)m * (R + 1));
  L.w = take(sizeof(double2) * (size_t)m * n);
  L.d = take(sizeof(double2) * (size_t)m * n);
  L.x = take(sizeof(double2) * (size_t)m * n);
  L.r = take(sizeof(double2) * (size_t)m * n);
  L.X = take(sizeof(float2) * (size_t)m * n);
  L.Y = take(sizeof(float2) * (size_t)m * n);
  L.norm2 = take(sizeof(double) * m);
  L.winv = take(sizeof(double) * m);
  L.rnorm2 = take(sizeof(double) * m);
  L.beta = take(sizeof(double) * m);
  L.tol = take(sizeof(double) * m);
  L.resid = take(sizeof(double) * m);
  L.active = take(sizeof(int) * m);
  L.kend = take(sizeof(int) * m);
  L.y = take(sizeof(double2) * (size_t)m * R);
  L.bnorm2 = take(sizeof(double) * m);
  L.tc = take(precision == BEM_PREC_FP32 ? 0 : tc_workspace_bytes(n, m, precision));
  L.total = o;
  return L;
}

bool params_ok(const bem_solver_params* p) {
  return p && p->restart >= 1 && p->restart < kMaxRestart && p->max_iters >= 1 && p->max_refine >= 1 && p->rtol >= 0.0 &&
         (p->precision == BEM_PREC_FP32 || p->precision == BEM_PREC_BF16X3 || p->precision == BEM_PREC_BF16);
}

// Pinned host snapshots of the solver state, one per Arnoldi step in a ring,
// each with an event.  The host runs at most kLookahead steps ahead of the
// GPU: it blocks on the event of step it - kLookahead (the GPU still has that
// many steps queued) and stops enqueueing once a snapshot shows every column
// converged, so at most kLookahead no-op steps follow convergence.
constexpr int kRing = 8;
constexpr int kLookahead = 4;
struct HostRing {
  GmState* snap = nullptr;
  cudaEvent_t ev[kRing] = {};
  ~HostRing() {
    if (snap) cudaFreeHost(snap);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};
thread_local HostRing t_ring;

// One Arnoldi step (every kernel reads the step index from device memory) is
// captured once per solve on a private stream and replayed with one graph
// launch per step on the caller's stream.
thread_local cudaStream_t t_capture_stream = nullptr;

int capture_graph(const std::function<int(cudaStream_t)>& body, cudaGraphExec_t* exec, unsigned long long* nkern) {
  if (!t_capture_stream) BEM_CUDA_TRY(cudaStreamCreateWithFlags(&t_capture_stream, cudaStreamNonBlocking));
  const unsigned long long l0 = launch_count();
  BEM_CUDA_TRY(cudaStreamBeginCapture(t_capture_stream, cudaStreamCaptureModeThreadLocal));
  const int rc = body(t_capture_stream);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(t_capture_stream, &graph);
  if (rc != BEM_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc != BEM_OK ? rc : BEM_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) return BEM_ERR_CUDA;
  *nkern = launch_count() - l0;
  return BEM_OK;
}

int host_ring(HostRing** r) {
  if (!t_ring.snap) {
    BEM_CUDA_TRY(cudaHostAlloc((void**)&t_ring.snap, sizeof(GmState) * kRing, cudaHostAllocDefault));
    for (auto& e : t_ring.ev) BEM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  *r = &t_ring;
  return BEM_OK;
}

}  // namespace

int cmatmul(const float2* A, int n, const float2* X, int m, float2* Y, cudaStream_t s) {
  return launch_cmatmul<float, 0>(A, n, X, m, m, Y, m, nullptr, 0, nullptr, nullptr, s);
}

}  // namespace bemb

using namespace bemb;

extern "C" int bem_cmatmul(const void* A, int n, const void* X, int m, void* Y, bem_stream_t stream) {
  if (n < 0 || m < 0) return BEM_ERR_INVALID_ARGUMENT;
  if (n == 0 || m == 0) return BEM_OK;
  if (!A || !X || !Y) return BEM_ERR_INVALID_ARGUMENT;
  return cmatmul((const float2*)A, n, (const float2*)X, m, (float2*)Y, (cudaStream_t)stream);
}

extern "C" size_t bem_gmres_workspace_bytes(int n, int m, const bem_solver_params* params) {
  if (n <= 0 || m <= 0 || !params_ok(params)) return 0;
  return layout(n, m, params->restart, params->precision).total;
}

extern "C" int bem_gmres_solve(const void* A, int n, const void* B, int m, void* X, int use_x0,
                               const bem_solver_params* params, void* workspace, size_t workspace_bytes,
                               bem_solver_info* info, bem_stream_t stream) {
  if (info) std::memset(info, 0, sizeof(*info));
  if (n <= 0 || m <= 0 || !A || !B || !X || !params_ok(params)) return BEM_ERR_INVALID_ARGUMENT;
  if (m > 1024 || (params->precision != BEM_PREC_FP32 && m > 128)) return BEM_ERR_UNSUPPORTED;
  const int R = params->restart;
  const Layout L = layout(n, m, R, params->precision);
  if (!workspace || workspace_bytes < L.total) return BEM_ERR_WORKSPACE;
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  GmPtrs P;
  P.n = n;
  P.m = m;
  P.R = R;
  P.Vb = (float2*)(w + L.Vb);
  P.H = (double2*)(w + L.H);
  P.cs = (double*)(w + L.cs);
  P.sn = (double2*)(w + L.sn);
  P.g = (double2*)(w + L.g);
  P.h = (double2*)(w + L.h);
  P.w = (double2*)(w + L.w);
  P.d = (double2*)(w + L.d);
  P.x = (double2*)(w + L.x);
  P.r = (double2*)(w + L.r);
  P.X = (float2*)(w + L.X);
  P.Y = (float2*)(w + L.Y);
  P.norm2 = (double*)(w + L.norm2);
  P.winv = (double*)(w + L.winv);
  P.beta = (double*)(w + L.beta);
  P.tol = (double*)(w + L.tol);
  P.resid = (double*)(w + L.resid);
  P.active = (int*)(w + L.active);
  P.kend = (int*)(w + L.kend);
  P.y = (double*)(w + L.y);
  P.st = (GmState*)(w + L.st);
  P.bnorm2 = (double*)(w + L.bnorm2);
  double* rnorm2 = (double*)(w + L.rnorm2);
  void* tcws = w + L.tc;
  const int prec = params->precision;
  if (prec != BEM_PREC_FP32) {
    int rc = tc_operator_prepare((const float2*)A, n, prec, tcws, s);
    if (rc) return rc;
  }
  auto inner_matvec_on = [&](cudaStream_t st) -> int {
    if (prec == BEM_PREC_FP32)
      return launch_cmatmul<float, 0>((const float2*)A, n, P.X, m, m, P.Y, m, nullptr, 0, nullptr, &P.st->skip, st);
    return tc_matvec(tcws, n, prec, P.X, m, P.Y, &P.st->skip, st);
  };
  auto inner_matvec = [&]() -> int { return inner_matvec_on(s); };

  const dim3 gv((n + 255) / 256, m);
  const dim3 dots_grid((n + kDotRows - 1) / kDotRows, (R + 1 + kDotL - 1) / kDotL, m);
  auto arnoldi_step = [&](cudaStream_t st) -> int {
    (gm_pack_kernel<<<gv, 256, 0, st>>>(P), count_launch());
    int r2 = inner_matvec_on(st);
    if (r2) return r2;
    (gm_y2w_kernel<<<(unsigned)(((long long)n * m + 255) / 256), 256, 0, st>>>(P), count_launch());
    (gm_dots_kernel<<<dots_grid, kDotThreads, 0, st>>>(P, 0), count_launch());
    (gm_update_kernel<<<gv, 256, 0, st>>>(P, 0), count_launch());
    (gm_dots_kernel<<<dots_grid, kDotThreads, 0, st>>>(P, 1), count_launch());
    (gm_update_kernel<<<gv, 256, 0, st>>>(P, 1), count_launch());
    (gm_finalize_kernel<<<(m + kFinWarps - 1) / kFinWarps, 32 * kFinWarps, 0, st>>>(P, &P.st->any_count,
                                                                                   &P.st->done_blocks),
     count_launch());
    BEM_CUDA_TRY(cudaGetLastError());
    return BEM_OK;
  };
  cudaGraphExec_t step_exec = nullptr;
  unsigned long long step_kernels = 0;
  bool step_direct_done = false;  // the first step runs uncaptured (sets kernel attributes)
  HostRing* ring;
  int rc = host_ring(&ring);
  if (rc) return rc;
  std::vector<double> hres(m), hb(m);

  BEM_CUDA_TRY(cudaMemsetAsync(P.st, 0, sizeof(GmState), s));
  BEM_CUDA_TRY(cudaMemsetAsync(P.bnorm2, 0, sizeof(double) * m, s));
  BEM_CUDA_TRY(cudaMemsetAsync(P.norm2, 0, sizeof(double) * m, s));
  (gm_bnorm_kernel<<<gv, 256, 0, s>>>(P, (const float2*)B), count_launch());
  (gm_init_x_kernel<<<gv, 256, 0, s>>>(P, (const float2*)X, use_x0), count_launch());
  BEM_CUDA_TRY(cudaMemcpyAsync(hb.data(), P.bnorm2, sizeof(double) * m, cudaMemcpyDeviceToHost, s));

  int total_iters = 0, matvecs = 0, refinements = 0;
  double max_rel = 0.0;
  int status = BEM_ERR_NOT_CONVERGED;
  bool x_nonzero = use_x0 != 0;
  for (int outer = 0; outer <= params->max_refine; outer++) {
    // outer FP64 residual r = b - A x against the FP32 matrix
    BEM_CUDA_TRY(cudaMemsetAsync(rnorm2, 0, sizeof(double) * m, s));
    if (x_nonzero) {
      rc = launch_cmatmul<double, 1>((const float2*)A, n, P.x, m, m, P.r, m, (const float2*)B, m, rnorm2, nullptr, s);
      if (rc) return rc;
      matvecs++;
    } else {
      (gm_copy_b_kernel<<<gv, 256, 0, s>>>(P, (const float2*)B, rnorm2), count_launch());
    }
    BEM_CUDA_TRY(cudaMemcpyAsync(hres.data(), rnorm2, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    BEM_CUDA_TRY(cudaStreamSynchronize(s));
    bool done = true;
    max_rel = 0.0;
    for (int c = 0; c < m; c++) {
      const double bn = std::sqrt(hb[c]), rn = std::sqrt(hres[c]);
      const double rel = bn > 0.0 ? rn / bn : (rn > 0.0 ? INFINITY : 0.0);
      if (!std::isfinite(rel)) {
        status = BEM_ERR_NONFINITE;
        done = true;
        max_rel = rel;
        break;
      }
      max_rel = std::max(max_rel, rel);
      if (!(rn <= params->rtol * bn || rn <= params->atol)) done = false;
    }
    if (status == BEM_ERR_NONFINITE) break;
    if (done) {
      status = BEM_OK;
      break;
    }
    if (outer == params->max_refine || total_iters >= params->max_iters) break;
    refinements = outer + 1;

    // inner restarted GMRES on A_lp d = r
    const double inner_rtol = prec == BEM_PREC_FP32 ? 0.0 : params->inner_rtol;
    bool first_cycle = true;
    while (total_iters < params->max_iters) {
      BEM_CUDA_TRY(cudaMemsetAsync(P.norm2, 0, sizeof(double) * m, s));
      if (!first_cycle) {
        (gm_pack_d_kernel<<<gv, 256, 0, s>>>(P), count_launch());
        BEM_CUDA_TRY(cudaMemsetAsync(&P.st->skip, 0, sizeof(int), s));
        if ((rc = inner_matvec())) return rc;
        matvecs++;
      }
      BEM_CUDA_TRY(cudaMemsetAsync(P.h, 0, sizeof(double2) * 2 * (size_t)m * (R + 1), s));
      (gm_start_vec_kernel<<<gv, 256, 0, s>>>(P, first_cycle ? 0 : 1), count_launch());
      // absolute inner target: inner_rtol * ||r_out|| but never below rtol * ||b|| / 2
      (gm_start_scalar_kernel<<<1, ((m + 31) / 32) * 32, 0, s>>>(P, rnorm2, inner_rtol, 0.5 * params->rtol), count_launch());
      (gm_start_norm_kernel<<<gv, 256, 0, s>>>(P), count_launch());
      first_cycle = false;
      int it = 0;
      bool cycle_done = false;
      while (it < R && total_iters < params->max_iters) {
        if (!step_direct_done || !step_exec) {
          if ((rc = arnoldi_step(s))) return rc;
          if (!step_direct_done) {
            step_direct_done = true;
            if (capture_graph(arnoldi_step, &step_exec, &step_kernels) != BEM_OK) step_exec = nullptr;
          }
        } else {
          BEM_CUDA_TRY(cudaGraphLaunch(step_exec, s));
          count_launches(step_kernels);
        }
        BEM_CUDA_TRY(cudaMemcpyAsync(&ring->snap[it % kRing], P.st, sizeof(GmState), cudaMemcpyDeviceToHost, s));
        BEM_CUDA_TRY(cudaEventRecord(ring->ev[it % kRing], s));
        it++;
        total_iters++;
        if (it > kLookahead) {
          const int old = (it - 1 - kLookahead) % kRing;
          BEM_CUDA_TRY(cudaEventSynchronize(ring->ev[old]));
          if (ring->snap[old].any_active == 0) cycle_done = true;
        }
        if (cycle_done) break;
      }
      (gm_solve_kernel<<<(m + kSolveWarps - 1) / kSolveWarps, 32 * kSolveWarps, 0, s>>>(P), count_launch());
      (gm_xupdate_kernel<<<gv, 256, 0, s>>>(P), count_launch());
      // converged when no column is active at the end of the cycle with
      // resid <= tol (columns that stopped at the restart length restart)
      BEM_CUDA_TRY(cudaMemcpyAsync(hres.data(), P.resid, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
      std::vector<double> htol(m);
      BEM_CUDA_TRY(cudaMemcpyAsync(htol.data(), P.tol, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
      BEM_CUDA_TRY(cudaStreamSynchronize(s));
      bool all = true;
      for (int c = 0; c < m; c++)
        if (hres[c] > htol[c]) all = false;
      if (all) break;
    }
    (gm_accept_kernel<<<gv, 256, 0, s>>>(P), count_launch());
    x_nonzero = true;
  }
  (gm_store_x_kernel<<<gv, 256, 0, s>>>(P, (float2*)X), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  if (prec != BEM_PREC_FP32) {
    int tc_err = 0;
    if (tc_error(tcws, &tc_err, s) != BEM_OK || tc_err) status = BEM_ERR_CUDA;
  }
  if (step_exec) cudaGraphExecDestroy(step_exec);
  GmState fin;
  BEM_CUDA_TRY(cudaMemcpy(&fin, P.st, sizeof(GmState), cudaMemcpyDeviceToHost));
  (void)total_iters;  // steps enqueued; fin.iters_done counts the executed ones
  matvecs += fin.iters_done;
  if (info) {
    info->status = status;
    info->iterations = fin.iters_done;
    info->refinements = refinements;
    info->matvecs = matvecs;
    info->rel_residual = max_rel;
  }
  return status;
}

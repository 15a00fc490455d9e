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
//    operator application: Arnoldi with classical Gram-Schmidt in FP64 (one
//    pass by default, re-orthogonalisation on request), complex Givens
//    rotations in FP64, all state
//    on the device; the host only watches a convergence flag through events,
//    without stalling the GPU.  Outer FP64 iterative refinement
//    r = b - A x against the FP32 matrix.

#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <future>
#include <mutex>
#include <vector>

#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "async_copy.cuh"
#include "bem_common.cuh"

namespace bemb {

namespace cg = cooperative_groups;

int g_gmres_reorth = 0;     // Gram-Schmidt passes: 0 automatic, 1 one pass (CGS), 2 two passes (CGS2); a tuning knob
int g_arn_max_cluster = 0;  // largest Arnoldi cluster size tried (0: 16); a tuning knob
int g_arn_mode = 0;         // Arnoldi step: 0 automatic (the cluster kernel), 1 cluster kernel, 2 streamed
                            // kernels, 3 cooperative kernel; a tuning knob
int g_gmres_block = 0;      // 0: one block Krylov space for 2..16 right-hand sides, 1: separate spaces; a tuning knob

// tensor-core operator (tc_matvec.cu)
int tc_operator_prepare(const float2* A, int n, int precision, void* ws, cudaStream_t s);
int tc_matvec(const void* ws, int n, int precision, const float2* X, int m, float2* Y, const int* active,
              cudaStream_t s);
int tc_error(const void* ws, int* err_host, cudaStream_t s, bool clear);
size_t tc_workspace_bytes(int n, int m, int precision);
int tc_b_planes(void* ws, int n, int m, int precision, __nv_bfloat16** bh, __nv_bfloat16** bl, int* ldb, int* nb,
                float** cinv);
int encode_map_2d_f32(CUtensorMap* map, const void* ptr, unsigned long long cols, unsigned long long rows,
                      unsigned long long ld_bytes, unsigned box_cols, unsigned box_rows);
int encode_map_2d_f32_sw128(CUtensorMap* map, const void* ptr, unsigned long long cols, unsigned long long rows,
                            unsigned long long ld_bytes, unsigned box_cols, unsigned box_rows);
int tc_gemm(const void* ws, int n, int precision, int m, float2* Y, const int* active, cudaStream_t s);

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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
__global__ void __launch_bounds__(kMMThreads, 2)
    cmatmul_kernel(const float2* __restrict__ A, int n, const typename C2<T>::type* __restrict__ X, int ldx,
                   int m, typename C2<T>::type* __restrict__ Y, int ldy, const float2* __restrict__ B, int ldb,
                   double* __restrict__ norm2, const int* __restrict__ active) {
  typedef typename C2<T>::type CT;
  constexpr int kMMRowsPerWarp = MMRows<T>::kPerWarp;
  constexpr int kMMRows = MMRows<T>::kPerBlock;
  if (active) {  // GMRES: nothing to do once every column has converged
    int any = 0;
    for (int c = 0; c < m; c++) any |= active[c];
    if (!any) return;
  }
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
                   int ldy, const float2* B, int ldb, double* norm2, const int* active, cudaStream_t s) {
  const int rb = (n + MMRows<T>::kPerBlock - 1) / MMRows<T>::kPerBlock;
  if (m == 1) {
    (cmatmul_kernel<T, 1, MODE><<<dim3(rb, 1), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2, active), count_launch());
  } else if (m == 2) {
    (cmatmul_kernel<T, 2, MODE><<<dim3(rb, 1), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2, active), count_launch());
  } else if (m <= 4) {
    (cmatmul_kernel<T, 4, MODE><<<dim3(rb, 1), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2, active), count_launch());
  } else {
    (cmatmul_kernel<T, 8, MODE><<<dim3(rb, (m + 7) / 8), kMMThreads, 0, s>>>(A, n, X, ldx, m, Y, ldy, B, ldb, norm2,
                                                                          active), count_launch());
  }
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// FP64 residual R = B - A X (A complex64, X and R complex128) for the outer
// refinement, FP64 products and sums.  The work is FP64-bound (4 DFMA per
// complex product, n^2 m of them), so the layout keeps the FP64 pipe fed:
// thread = row, A read 16 complex (one 128-byte line) per lane per step, the
// CTA's X columns staged in shared memory and read as warp broadcasts (one
// wavefront per 16 bytes for all 32 rows), 8 right-hand sides accumulated
// per thread.  CTAs cover 256 rows x kRsCols columns; the column ranges'
// partial sums meet in R by FP64 atomics (R zeroed first), then
// resid_finish_kernel forms B - R and the squared norms.  n even (16-byte
// rows); odd n takes cmatmul_kernel.
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsCols = 320;  // columns per CTA (multiple of 16)
constexpr int kRsRhs = 8;     // right-hand sides per CTA (blockIdx.z groups)

__global__ void __launch_bounds__(kRsThreads, 2)
    resid_f64_kernel(const float2* __restrict__ A, int n, const double2* __restrict__ X, int m,
                     double2* __restrict__ R) {
  __shared__ double2 xs[kRsCols * kRsRhs];  // [column][rhs]
  const int c0 = blockIdx.y * kRsCols;
  const int cn = min(kRsCols, n - c0);
  const int s0 = blockIdx.z * kRsRhs;
  const int ms = min(kRsRhs, m - s0);
  for (int e = threadIdx.x; e < kRsCols * kRsRhs; e += kRsThreads) {
    const int c = e / kRsRhs, s = e - c * kRsRhs;
    xs[e] = (c < cn && s < ms) ? X[(size_t)(c0 + c) * m + s0 + s] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const int row = blockIdx.x * kRsThreads + threadIdx.x;
  if (row >= n) return;  // after the only barrier
  const float4* a4 = reinterpret_cast<const float4*>(A + (size_t)row * n + c0);  // n even: 16-byte aligned
  double acc[kRsRhs][2];
#pragma unroll
  for (int s = 0; s < kRsRhs; s++) acc[s][0] = acc[s][1] = 0.0;
  const int cfull = cn & ~15;
  for (int c = 0; c < cfull; c += 16) {
    float4 v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = __ldcs(a4 + c / 2 + k);
#pragma unroll
    for (int k = 0; k < 8; k++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const double ar = h ? v[k].z : v[k].x, ai = h ? v[k].w : v[k].y;
        const double2* xc = xs + (size_t)(c + 2 * k + h) * kRsRhs;
#pragma unroll
        for (int s = 0; s < kRsRhs; s++) {
          const double2 x = xc[s];
          acc[s][0] = fma(ar, x.x, fma(-ai, x.y, acc[s][0]));
          acc[s][1] = fma(ar, x.y, fma(ai, x.x, acc[s][1]));
        }
      }
    }
  }
  const float2* a2 = A + (size_t)row * n + c0;
  for (int c = cfull; c < cn; c++) {
    const float2 v = __ldcs(a2 + c);
    const double ar = v.x, ai = v.y;
#pragma unroll
    for (int s = 0; s < kRsRhs; s++) {
      const double2 x = xs[(size_t)c * kRsRhs + s];
      acc[s][0] = fma(ar, x.x, fma(-ai, x.y, acc[s][0]));
      acc[s][1] = fma(ar, x.y, fma(ai, x.x, acc[s][1]));
    }
  }
#pragma unroll
  for (int s = 0; s < kRsRhs; s++) {
    if (s < ms) {
      double* r = reinterpret_cast<double*>(R + (size_t)row * m + s0 + s);
      atomicAdd(r, acc[s][0]);
      atomicAdd(r + 1, acc[s][1]);
    }
  }
}

// R = B - R (R holding A X) and norm2[s] += |R[:, s]|^2.
__global__ void __launch_bounds__(256) resid_finish_kernel(const float2* __restrict__ B, int n, int m,
                                                           double2* __restrict__ R, double* __restrict__ norm2) {
  __shared__ double red[256];
  const int s = blockIdx.y;
  double sum = 0.0;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
    const size_t e = (size_t)i * m + s;
    const float2 b = B[e];
    double2 r = R[e];
    r.x = (double)b.x - r.x;
    r.y = (double)b.y - r.y;
    R[e] = r;
    sum += r.x * r.x + r.y * r.y;
  }
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(&norm2[s], red[0]);
}

// ---------------------------------------------------------------------------
// resid_tma_kernel: the same R = A X (FP64 products and sums) with the
// matrix streamed through shared memory, so that the rows are read from HBM
// coalesced instead of one 128-byte line per lane.  A producer warp loads
// 256-row x 16-column tiles of A (2-D tensor map over the matrix as FP32
// pairs, 128-byte swizzle, no multicast; rows and columns past n arrive
// zero-filled) into a ring of kRtStages stages; compute threads t and
// t + 256 own row r0 + t, each for 4 of the 8 right-hand sides (16 compute
// warps to cover the FP64 and shared-memory latencies), and read the row's
// 128-byte slice as 8 float4 chunks (chunk k at k ^ (t & 7): the 32 lanes of
// a warp read 512 bytes in 4 wavefronts); the item's X columns are staged
// once in shared memory and read as broadcasts.
// Items (256-row block, group of cb columns, 8 right-hand sides) are taken
// from blockIdx.x on, gridDim.x apart; every wait is bounded (err).
// ---------------------------------------------------------------------------
inline int device_sms() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

constexpr int kRtRows = 256;                                            // rows per item
constexpr int kRtSplit = 1;                                             // compute threads per row
constexpr int kRtRhs = kRsRhs / kRtSplit;                               // right-hand sides per thread
constexpr int kRtThreads = kRtSplit * kRtRows + 32;                     // + the producer warp
constexpr int kRtTileCols = 16;                                         // complex columns per stage: 128 B per row
constexpr int kRtStages = 4;
constexpr size_t kRtStageBytes = sizeof(float2) * kRtRows * kRtTileCols;  // 32 KB
constexpr int kRtMaxCols = 640;                                         // columns per item (multiple of 16)
constexpr size_t kRtXBytes = sizeof(double2) * kRtMaxCols * kRsRhs;     // 80 KB
constexpr size_t kRtSmem = kRtStageBytes * kRtStages + kRtXBytes + 2 * kRtStages * sizeof(uint64_t);

__global__ void __launch_bounds__(kRtThreads, 1)
    resid_tma_kernel(const __grid_constant__ CUtensorMap amap, int n, const double2* __restrict__ X, int m,
                     double2* __restrict__ R, int cb, int n_cg, int n_items, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char rt_raw[];
  const float4* ring = reinterpret_cast<const float4*>(rt_raw);                     // [stage][row][8 chunks]
  double2* xs = reinterpret_cast<double2*>(rt_raw + kRtStageBytes * kRtStages);       // [column][rhs]
  uint64_t* full = reinterpret_cast<uint64_t*>(rt_raw + kRtStageBytes * kRtStages + kRtXBytes);
  uint64_t* empty = full + kRtStages;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int kComputeWarps = kRtSplit * kRtRows / 32;
  if ((smem_u32(rt_raw) & 1023u) != 0u) {  // the swizzled tiles need 1024-byte alignment (uniform)
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (tid == 0) {
    for (int st = 0; st < kRtStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kComputeWarps);
    }
    mbar_init_fence();
  }
  __syncthreads();
  const int n_rb = (n + kRtRows - 1) / kRtRows;
  unsigned g = 0;  // ring stages used so far (producer and consumers count alike)
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int sg = item / (n_rb * n_cg);
    const int rem = item - sg * n_rb * n_cg;
    const int cg = rem / n_rb, rb = rem - cg * n_rb;
    const int r0 = rb * kRtRows, c0 = cg * cb;
    const int cn = min(cb, n - c0);
    const int s0 = sg * kRsRhs, ms = min(kRsRhs, m - s0);
    const int ntiles = (cn + kRtTileCols - 1) / kRtTileCols;
    __syncthreads();  // the previous item's readers are done with xs
    for (int e = tid; e < ntiles * kRtTileCols * kRsRhs; e += kRtThreads) {
      const int c = e / kRsRhs, sl = e - c * kRsRhs;
      xs[e] = (c < cn && sl < ms) ? X[(size_t)(c0 + c) * m + s0 + sl] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (warp == kComputeWarps) {  // producer
      if (lane == 0) {
        const uint64_t pol = l2_evict_first_policy();
        for (int t = 0; t < ntiles; t++) {
          const unsigned gi = g + t;
          const int st = (int)(gi % kRtStages);
          if (gi >= kRtStages && !mbar_wait(&empty[st], (gi / kRtStages - 1u) & 1u, err)) break;
          mbar_expect_tx(&full[st], (uint32_t)kRtStageBytes);
          tma_load_2d_hint(rt_raw + (size_t)st * kRtStageBytes, &amap, 2 * (c0 + t * kRtTileCols), r0, &full[st],
                           pol);
        }
      }
    } else {
      const int rl = tid % kRtRows, sh = (tid / kRtRows) * kRtRhs;  // row in the item, first right-hand side
      const int row = r0 + rl;
      double acc[kRtRhs][2];
#pragma unroll
      for (int sl = 0; sl < kRtRhs; sl++) acc[sl][0] = acc[sl][1] = 0.0;
      for (int t = 0; t < ntiles; t++) {
        const unsigned gi = g + t;
        const int st = (int)(gi % kRtStages);
        mbar_wait(&full[st], (gi / kRtStages) & 1u, err);
        if (row < n) {
          const float4* rp = ring + ((size_t)st * kRtRows + rl) * 8;
          const double2* xt = xs + (size_t)t * kRtTileCols * kRsRhs + sh;
#pragma unroll 4
          for (int k = 0; k < 8; k++) {
            const float4 v = rp[k ^ (rl & 7)];  // columns 2k, 2k + 1 of the tile
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const double ar = h ? v.z : v.x, ai = h ? v.w : v.y;
              const double2* xc = xt + (size_t)(2 * k + h) * kRsRhs;
#pragma unroll
              for (int sl = 0; sl < kRtRhs; sl++) {
                const double2 x = xc[sl];
                acc[sl][0] = fma(ar, x.x, fma(-ai, x.y, acc[sl][0]));
                acc[sl][1] = fma(ar, x.y, fma(ai, x.x, acc[sl][1]));
              }
            }
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[st]);
      }
      if (row < n) {
#pragma unroll
        for (int sl = 0; sl < kRtRhs; sl++) {
          if (sh + sl < ms) {
            double* r = reinterpret_cast<double*>(R + (size_t)row * m + s0 + sh + sl);
            atomicAdd(r, acc[sl][0]);
            atomicAdd(r + 1, acc[sl][1]);
          }
        }
      }
    }
    g += (unsigned)ntiles;
  }
  // every issued copy has landed before the CTA exits (a wait above may have
  // given up after an error): the last use of each slot
  __syncthreads();
  if (tid == 0)
    for (int st = 0; st < kRtStages; st++)
      if (g > (unsigned)st) mbar_wait_drain(&full[st], ((g - 1u - (unsigned)st) / kRtStages) & 1u);
}

// R = B - A X, norm2[s] += |R[:, s]|^2 (X, R: n x m row-major complex128; B: complex64).
// err (device int, raised when a bounded wait expires) selects the streamed
// kernel for n even and a 16-byte aligned A; else the row-per-thread kernel.
int launch_resid_f64(const float2* A, int n, const double2* X, int m, double2* R, const float2* B, double* norm2,
                     cudaStream_t s, int* err = nullptr) {
  if (n & 1) return launch_cmatmul<double, 1>(A, n, X, m, m, R, m, B, m, norm2, nullptr, s);
  BEM_CUDA_TRY(cudaMemsetAsync(R, 0, sizeof(double2) * (size_t)n * m, s));
  if (err && ((uintptr_t)A & 15) == 0) {
    static std::atomic<bool> attr{false};
    if (!attr.load(std::memory_order_acquire)) {
      BEM_CUDA_TRY(cudaFuncSetAttribute(resid_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRtSmem));
      attr.store(true, std::memory_order_release);
    }
    CUtensorMap map;
    int rc = encode_map_2d_f32_sw128(&map, A, 2ull * n, (unsigned long long)n, 8ull * n, 2 * kRtTileCols, kRtRows);
    if (rc) return rc;
    const int n_cg = (n + kRtMaxCols - 1) / kRtMaxCols;
    const int cb = ((n + n_cg - 1) / n_cg + kRtTileCols - 1) / kRtTileCols * kRtTileCols;
    const long long n_items = (long long)((n + kRtRows - 1) / kRtRows) * n_cg * ((m + kRsRhs - 1) / kRsRhs);
    const int grid = (int)std::min<long long>(n_items, device_sms());
    (resid_tma_kernel<<<grid, kRtThreads, kRtSmem, s>>>(map, n, X, m, R, cb, n_cg, (int)n_items, err),
     count_launch());
  } else {
    const dim3 grid((n + kRsThreads - 1) / kRsThreads, (n + kRsCols - 1) / kRsCols, (m + kRsRhs - 1) / kRsRhs);
    (resid_f64_kernel<<<grid, kRsThreads, 0, s>>>(A, n, X, m, R), count_launch());
  }
  BEM_CUDA_TRY(cudaGetLastError());
  (resid_finish_kernel<<<dim3(std::min(148, (n + 255) / 256), m), 256, 0, s>>>(B, n, m, R, norm2), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// FP32 complex matvec Y += A X (HBM-streaming, CUDA cores, 4 FMA per complex
// product), for the FP32 precision mode and the right-hand side -V g.
//
// Split over 1024-column chunks of A (blockIdx.x), row ranges (blockIdx.y)
// and groups of MR <= 8 right-hand sides (blockIdx.z).  The CTA stages its X
// chunk transposed in shared memory ([rhs][column]: lanes reading
// consecutive columns hit consecutive banks); each warp owns 4 rows at a
// time and meets every A value with MR right-hand sides.  Lane partial sums
// are combined with a warp reduce-scatter and added to Y with one vector
// atomic per entry, so Y must hold zero (or the sum to add to) beforehand.
//  * cgemv_tma_kernel (n even, rows 16-byte aligned): a producer warp streams
//    32-row x 128-column tiles of A (2-D tensor map over the matrix as FP32
//    pairs, no multicast; rows / columns past n arrive zero-filled) through a
//    4-stage shared-memory ring, so memory-level parallelism does not depend
//    on registers; 8 compute warps read A and X from shared memory.
//  * cgemv_kernel (any n): lanes stream A rows from global memory.
// ---------------------------------------------------------------------------
constexpr int kGvThreads = 256;
constexpr int kGvRows = 4;       // rows per warp
constexpr int kGvChunk = 1024;   // columns per CTA

// Warp reduce-scatter of NC complex values held as 2*NC floats (NC a power
// of two, 1..32): lane L returns the warp total of complex value
// L >> (5 - log2 NC).
template <int NC>
__device__ __forceinline__ float2 warp_rs_complex(float (&v)[2 * NC], int lane) {
#pragma unroll
  for (int half = NC / 2, off = 16; half >= 1; half >>= 1, off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int j = 0; j < half; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const float send = upper ? v[2 * j + h] : v[2 * (j + half) + h];
        const float keep = upper ? v[2 * (j + half) + h] : v[2 * j + h];
        v[2 * j + h] = keep + __shfl_xor_sync(0xffffffffu, send, off);
      }
    }
  }
  float re = v[0], im = v[1];
#pragma unroll
  for (int off = 16 / NC; off >= 1; off >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, off);
    im += __shfl_xor_sync(0xffffffffu, im, off);
  }
  return make_float2(re, im);
}

// acc[2(r MR + s)] += A row r (columns c, c+1) * X (columns c, c+1, rhs s)
template <int MR>
__device__ __forceinline__ void cgemv_fma2(float (&acc)[2 * kGvRows * MR], const float4 (&a)[kGvRows],
                                           const float2* xs, int c) {
#pragma unroll
  for (int sl = 0; sl < MR; sl++) {
    const float4 x = *reinterpret_cast<const float4*>(&xs[sl * kGvChunk + c]);
#pragma unroll
    for (int r = 0; r < kGvRows; r++) {
      float& re = acc[2 * (r * MR + sl)];
      float& im = acc[2 * (r * MR + sl) + 1];
      re = fmaf(a[r].x, x.x, re);
      re = fmaf(-a[r].y, x.y, re);
      re = fmaf(a[r].z, x.z, re);
      re = fmaf(-a[r].w, x.w, re);
      im = fmaf(a[r].x, x.y, im);
      im = fmaf(a[r].y, x.x, im);
      im = fmaf(a[r].z, x.w, im);
      im = fmaf(a[r].w, x.z, im);
    }
  }
}

// X chunk [c0, c0 + cn) x [s0, s0 + MR) -> xs[rhs][column], zero-padded.
template <int MR>
__device__ __forceinline__ void cgemv_stage_x(const float2* __restrict__ X, int m, int c0, int cn, int s0,
                                              float2* xs, int nthreads) {
  for (int e = threadIdx.x; e < MR * kGvChunk; e += nthreads) {
    const int c = e / MR, sl = e - c * MR;
    float2 v = make_float2(0.f, 0.f);
    if (c < cn && s0 + sl < m) v = X[(size_t)(c0 + c) * m + s0 + sl];
    xs[sl * kGvChunk + c] = v;
  }
}

// Reduce a warp's 4 x MR partial sums and add them to Y (rows row0..row0+3).
template <int MR>
__device__ __forceinline__ void cgemv_flush(float (&acc)[2 * kGvRows * MR], int lane, int row0, int r_end, int s0,
                                            int m, float2* __restrict__ Y) {
  constexpr int NC = kGvRows * MR;
  const float2 t = warp_rs_complex<NC>(acc, lane);
  constexpr int kShift = NC >= 32 ? 0 : (NC == 16 ? 1 : (NC == 8 ? 2 : (NC == 4 ? 3 : 4)));
  if ((lane & ((1 << kShift) - 1)) == 0) {
    const int idx = lane >> kShift;
    const int r = idx / MR, sl = idx - r * MR;
    if (row0 + r < r_end && s0 + sl < m) atomicAdd(&Y[(size_t)(row0 + r) * m + s0 + sl], t);
  }
}

template <int MR>
__global__ void __launch_bounds__(kGvThreads, 2)
    cgemv_kernel(const float2* __restrict__ A, int n, const float2* __restrict__ X, int m, float2* __restrict__ Y,
                 int rows_per_cta, const int* __restrict__ active) {
  extern __shared__ __align__(16) float2 xs[];  // [MR][kGvChunk]
  if (active) {  // GMRES: nothing to do once every column has converged
    int any = 0;
    for (int c = 0; c < m; c++) any |= active[c];
    if (!any) return;
  }
  const int c0 = blockIdx.x * kGvChunk;
  const int cn = min(kGvChunk, n - c0);
  const int s0 = blockIdx.z * MR;
  cgemv_stage_x<MR>(X, m, c0, cn, s0, xs, kGvThreads);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r_begin = blockIdx.y * rows_per_cta;
  const int r_end = min(n, r_begin + rows_per_cta);
  for (int rb = r_begin + warp * kGvRows; rb < r_end; rb += kGvRows * (kGvThreads / 32)) {
    float acc[2 * kGvRows * MR];
#pragma unroll
    for (int q = 0; q < 2 * kGvRows * MR; q++) acc[q] = 0.f;
    const float2* arow[kGvRows];
#pragma unroll
    for (int r = 0; r < kGvRows; r++) arow[r] = A + (size_t)min(rb + r, n - 1) * n + c0;
#pragma unroll 4
    for (int c = lane; c < cn; c += 32) {
      float2 a[kGvRows];
#pragma unroll
      for (int r = 0; r < kGvRows; r++) a[r] = __ldcs(arow[r] + c);
#pragma unroll
      for (int sl = 0; sl < MR; sl++) {
        const float2 x = xs[sl * kGvChunk + c];
#pragma unroll
        for (int r = 0; r < kGvRows; r++) {
          float& re = acc[2 * (r * MR + sl)];
          float& im = acc[2 * (r * MR + sl) + 1];
          re = fmaf(a[r].x, x.x, re);
          re = fmaf(-a[r].y, x.y, re);
          im = fmaf(a[r].x, x.y, im);
          im = fmaf(a[r].y, x.x, im);
        }
      }
    }
    cgemv_flush<MR>(acc, lane, rb, r_end, s0, m, Y);
  }
}

constexpr int kGtComputeWarps = 8;
constexpr int kGtThreads = 32 * (kGtComputeWarps + 1);
constexpr int kGtBlockRows = kGvRows * kGtComputeWarps;  // 32
constexpr int kGtTileCols = 128;                          // complex columns per stage
constexpr int kGtStages = 4;
constexpr size_t kGtStageBytes = sizeof(float2) * kGtBlockRows * kGtTileCols;  // 32 KB

template <int MR>
__host__ __device__ constexpr size_t gt_smem_bytes() {
  return kGtStageBytes * kGtStages + sizeof(float2) * MR * kGvChunk + 2 * kGtStages * sizeof(uint64_t);
}

template <int MR>
__global__ void __launch_bounds__(kGtThreads, 1)
    cgemv_tma_kernel(const __grid_constant__ CUtensorMap amap, int n, const float2* __restrict__ X, int m,
                     float2* __restrict__ Y, int rows_per_cta, const int* __restrict__ active, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char gt_raw[];
  float2* tiles = reinterpret_cast<float2*>(gt_raw);                           // [stage][32][128]
  float2* xs = reinterpret_cast<float2*>(gt_raw + kGtStageBytes * kGtStages);  // [MR][kGvChunk]
  uint64_t* full = reinterpret_cast<uint64_t*>(gt_raw + kGtStageBytes * kGtStages + sizeof(float2) * MR * kGvChunk);
  uint64_t* empty = full + kGtStages;
  if (active) {  // GMRES: nothing to do once every column has converged
    int any = 0;
    for (int c = 0; c < m; c++) any |= active[c];
    if (!any) return;
  }
  const int c0 = blockIdx.x * kGvChunk;
  const int cn = min(kGvChunk, n - c0);
  const int ntiles = (cn + kGtTileCols - 1) / kGtTileCols;
  const int s0 = blockIdx.z * MR;
  const int r_begin = blockIdx.y * rows_per_cta;
  const int r_end = min(n, r_begin + rows_per_cta);
  const int nblocks = r_end > r_begin ? (r_end - r_begin + kGtBlockRows - 1) / kGtBlockRows : 0;
  const int total = nblocks * ntiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    for (int st = 0; st < kGtStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kGtComputeWarps);
    }
    mbar_init_fence();
  }
  cgemv_stage_x<MR>(X, m, c0, cn, s0, xs, kGtThreads);
  __syncthreads();

  if (warp == kGtComputeWarps) {  // producer
    if (lane == 0) {
      const uint64_t pol = l2_evict_first_policy();
      for (int g = 0; g < total; g++) {
        const int st = g % kGtStages;
        if (g >= kGtStages && !mbar_wait(&empty[st], ((uint32_t)(g / kGtStages) - 1u) & 1u, err)) break;
        const int b = g / ntiles, t = g - b * ntiles;
        mbar_expect_tx(&full[st], (uint32_t)kGtStageBytes);
        tma_load_2d_hint(tiles + (size_t)st * kGtBlockRows * kGtTileCols, &amap, 2 * (c0 + t * kGtTileCols),
                         r_begin + b * kGtBlockRows, &full[st], pol);
      }
    }
    return;
  }

  for (int b = 0; b < nblocks; b++) {
    float acc[2 * kGvRows * MR];
#pragma unroll
    for (int q = 0; q < 2 * kGvRows * MR; q++) acc[q] = 0.f;
    for (int t = 0; t < ntiles; t++) {
      const int g = b * ntiles + t;
      const int st = g % kGtStages;
      mbar_wait(&full[st], (uint32_t)(g / kGtStages) & 1u, err);
      const float2* tile = tiles + (size_t)st * kGtBlockRows * kGtTileCols + (size_t)warp * kGvRows * kGtTileCols;
#pragma unroll
      for (int j = 0; j < kGtTileCols / 64; j++) {
        const int col = 2 * lane + 64 * j;
        float4 a[kGvRows];
#pragma unroll
        for (int r = 0; r < kGvRows; r++) a[r] = *reinterpret_cast<const float4*>(tile + r * kGtTileCols + col);
        cgemv_fma2<MR>(acc, a, xs, t * kGtTileCols + col);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
    }
    cgemv_flush<MR>(acc, lane, r_begin + b * kGtBlockRows + warp * kGvRows, r_end, s0, m, Y);
  }
}

template <int MR>
int launch_cgemv_mr(const float2* A, int n, const float2* X, int m, float2* Y, const int* active, cudaStream_t s) {
  static std::atomic<bool> attr{false};
  const int smem = (int)(sizeof(float2) * MR * kGvChunk);
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(cgemv_kernel<MR>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr.store(true, std::memory_order_release);
  }
  int occ = 0;
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, cgemv_kernel<MR>, kGvThreads, smem));
  const int kc = (n + kGvChunk - 1) / kGvChunk;
  const int groups = (m + MR - 1) / MR;
  long long rg = (long long)device_sms() * (occ > 0 ? occ : 1) / ((long long)kc * groups);
  if (rg < 1) rg = 1;
  const int step = kGvRows * (kGvThreads / 32);
  const int rows = (int)(((n + rg - 1) / rg + step - 1) / step * step);
  rg = (n + rows - 1) / rows;
  (cgemv_kernel<MR><<<dim3((unsigned)kc, (unsigned)rg, (unsigned)groups), kGvThreads, smem, s>>>(A, n, X, m, Y, rows,
                                                                                               active),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

template <int MR>
int launch_cgemv_tma(const float2* A, int n, const float2* X, int m, float2* Y, const int* active, int* err,
                     cudaStream_t s) {
  static std::atomic<bool> attr{false};
  const int smem = (int)gt_smem_bytes<MR>();
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(cgemv_tma_kernel<MR>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr.store(true, std::memory_order_release);
  }
  CUtensorMap map;
  int rc = encode_map_2d_f32(&map, A, 2ull * n, (unsigned long long)n, 8ull * n, 2 * kGtTileCols, kGtBlockRows);
  if (rc) return rc;
  const int kc = (n + kGvChunk - 1) / kGvChunk;
  const int groups = (m + MR - 1) / MR;
  long long rg = (long long)device_sms() / ((long long)kc * groups);
  if (rg < 1) rg = 1;
  const int rows = (int)(((n + rg - 1) / rg + kGtBlockRows - 1) / kGtBlockRows * kGtBlockRows);
  rg = (n + rows - 1) / rows;
  (cgemv_tma_kernel<MR><<<dim3((unsigned)kc, (unsigned)rg, (unsigned)groups), kGtThreads, smem, s>>>(
       map, n, X, m, Y, rows, active, err),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// Y += A X for an n x n complex64 A and m right-hand sides (row-major
// (n, m)).  err: device int raised if a bounded wait of the TMA variant
// expired; NULL selects the register variant.
int launch_cgemv(const float2* A, int n, const float2* X, int m, float2* Y, const int* active, cudaStream_t s,
                 int* err = nullptr) {
  if (n <= 0 || m <= 0) return BEM_OK;
  if ((n & 1) == 0 && err && ((uintptr_t)A & 15) == 0) {
    if (m == 1) return launch_cgemv_tma<1>(A, n, X, m, Y, active, err, s);
    if (m == 2) return launch_cgemv_tma<2>(A, n, X, m, Y, active, err, s);
    if (m <= 4) return launch_cgemv_tma<4>(A, n, X, m, Y, active, err, s);
    return launch_cgemv_tma<8>(A, n, X, m, Y, active, err, s);
  }
  if (m == 1) return launch_cgemv_mr<1>(A, n, X, m, Y, active, s);
  if (m == 2) return launch_cgemv_mr<2>(A, n, X, m, Y, active, s);
  if (m <= 4) return launch_cgemv_mr<4>(A, n, X, m, Y, active, s);
  return launch_cgemv_mr<8>(A, n, X, m, Y, active, s);
}

// ---------------------------------------------------------------------------
// GMRES state and kernels
// ---------------------------------------------------------------------------
struct GmState {
  int err;             // a bounded wait of an Arnoldi kernel expired
  unsigned bar_count;  // grid barrier of the cooperative step: arrivals
  unsigned bar_gen;    // and generation
  int pad;
};

// Host-mapped ring of per-step column activity (kSnapRing steps x m ints),
// written by the Arnoldi kernel and read by the host after the step's event.
constexpr int kSnapRing = 8;

struct GmPtrs {
  int n, m, R;
  int ldv;         // basis row stride (n rounded up to even: 16-byte pairs)
  int ldb;         // row stride of the tensor-core B planes
  float2* Vb;      // [m][R+1][ldv]  orthonormal Krylov basis, complex64 storage
  __nv_bfloat16* bh;  // tensor-core B planes (hi, lo) of the matvec operand, or NULL (FP32 matvec on X)
  __nv_bfloat16* bl;
  float* cinv;     // fp16 planes: inverse per-column scale read by the GEMM epilogue
  int f16;         // B planes hold fp16 scaled by kF16VecScale (normalised vectors)
  double2* H;      // [m][R][R+1]  column k, rows 0..k+1
  double* cs;      // [m][R]
  double2* sn;     // [m][R]
  double2* g;      // [m][R+1]
  double2* w;      // [m][n]
  double2* d;      // [m][n]  inner correction
  double2* x;      // [n][m]  solution (FP64)
  double2* r;      // [n][m]  outer residual (FP64)
  float2* X;       // [n][m]  matvec input
  float2* Y;       // [n][m]  matvec output
  double* norm2;   // [m]  |w|^2 accumulator of the current step
  double* beta;    // [m]
  double* tol;     // [m] inner absolute tolerance
  double* resid;   // [m]
  int* active;     // [m]
  int* kend;       // [m]  basis size used by each column in this cycle
  int* kcol;       // [m]  Arnoldi step of each column inside the current cycle
  int* colstep;    // [m]  Arnoldi launches so far in this solve (snapshot slot)
  int* snap;       // device view of the host-mapped activity ring
  double* y;       // [m][R]
  GmState* st;
  double* bnorm2;  // [m]
  double* hacc;    // [2][m][2][2 (R+1)]  streamed step: h sums of the two passes, by step parity
  double* nacc;    // [2][m][3]           streamed step: |w|^2 before and after each pass, by parity
};

// ---------------------------------------------------------------------------
// Arnoldi step = the matvec plus ONE launch of gm_arnoldi_kernel.
//
// A thread-block cluster (up to 16 CTAs) owns one right-hand-side column;
// its CTAs split the unknowns and keep their slice of w in shared memory for
// the whole step:
//   w = Y (Y cleared for the next accumulating matvec)
//   h1 = V^H w                 classical Gram-Schmidt, FP64 sums
//   w' = w - V h1            (one pass by default; with re-orthogonalisation
//   h2 = V^H w', w'' = w' - V h2   also this second pass, CGS2)
//   h_{k+1,k} = |w''|
//   v_{k+1} = w'' / h_{k+1,k} -> basis (complex64) and the next matvec operand
//   Givens rotation of the new Hessenberg column (CTA 0 of the cluster)
// Partial sums of each CTA are combined across the cluster through
// distributed shared memory after a cluster barrier (no global atomics);
// every CTA forms the same totals.  Each of the four passes streams the CTA's
// slice of basis vectors 0..k through a ring of shared-memory stages with
// 1-D bulk async copies (mbarrier completion, bounded waits), so the copy
// engine keeps a whole pass in flight while the threads compute from shared
// memory.  Threads own pairs of consecutive unknowns; per-basis-vector sums
// are reduced with a warp reduce-scatter.  The last column to finish
// publishes k + 1 and the activity flag for the host and the matvec.
// ---------------------------------------------------------------------------
constexpr int kArnConsumerWarps = 12;
constexpr int kArnConsumers = 32 * kArnConsumerWarps;
constexpr int kArnThreads = kArnConsumers + 32;  // + one producer warp (bulk copies)
constexpr int kArnWarps = kArnThreads / 32;
constexpr int kChunkMax = 8;     // basis vectors per staged chunk (<= consumer warps)
constexpr int kRingStages = 4;   // shared-memory stages of the basis stream
constexpr int kMaxRestart = 256;
constexpr int kArnMaxCluster = 16;

__device__ __forceinline__ const float2* vrow(const GmPtrs& P, int s, int l) {
  return P.Vb + ((size_t)s * (P.R + 1) + l) * P.ldv;
}

// Warp reduce-scatter of NV doubles (NV a power of two, 2..32): afterwards
// the returned value of lane L is the warp total of value L >> (5 - log2 NV).
template <int NV, typename T>
__device__ __forceinline__ T warp_reduce_scatter(T (&v)[NV], int lane) {
#pragma unroll
  for (int half = NV / 2, off = 16; half >= 1; half >>= 1, off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int j = 0; j < half; j++) {
      const T send = upper ? v[j] : v[j + half];
      const T keep = upper ? v[j + half] : v[j];
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  T t = v[0];
#pragma unroll
  for (int off = 16 / NV; off >= 1; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
  return t;
}

// Matvec operand for unknowns j, j+1 of column s: complex64 X (FP32 matvec)
// or the hi/lo B planes of the tensor-core GEMM (rows 2s: (re, -im),
// 2s+1: (im, re) per unknown, as the tensor-core pack kernels write them):
// bf16, or fp16 scaled by kF16VecScale (the vectors are normalised, so
// |component| <= 1).  x1 is zero when j+1 is the padding entry.
constexpr float kF16VecScale = 16384.f;
__device__ __forceinline__ void store_operand(const GmPtrs& P, int j, int s, float2 x0, float2 x1) {
  if (!P.bh) {
    P.X[(size_t)j * P.m + s] = x0;
    if (j + 1 < P.n) P.X[(size_t)(j + 1) * P.m + s] = x1;
    return;
  }
  const float e[2][4] = {{x0.x, -x0.y, x1.x, -x1.y}, {x0.y, x0.x, x1.y, x1.x}};
  if (P.f16) {
#pragma unroll
    for (int r = 0; r < 2; r++) {
      __align__(8) __half hi[4], lo[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float v = e[r][q] * kF16VecScale;
        hi[q] = __float2half_rn(v);
        lo[q] = __float2half_rn(v - __half2float(hi[q]));
      }
      const size_t o = (size_t)(2 * s + r) * P.ldb + 2 * j;
      *reinterpret_cast<uint2*>(P.bh + o) = *reinterpret_cast<const uint2*>(hi);
      *reinterpret_cast<uint2*>(P.bl + o) = *reinterpret_cast<const uint2*>(lo);
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < 2; r++) {
    __align__(8) __nv_bfloat16 hi[4], lo[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      hi[q] = __float2bfloat16_rn(e[r][q]);
      lo[q] = __float2bfloat16_rn(e[r][q] - __bfloat162float(hi[q]));
    }
    const size_t o = (size_t)(2 * s + r) * P.ldb + 2 * j;
    *reinterpret_cast<uint2*>(P.bh + o) = *reinterpret_cast<const uint2*>(hi);
    *reinterpret_cast<uint2*>(P.bl + o) = *reinterpret_cast<const uint2*>(lo);
  }
}

struct ArnSmem {
  uint64_t full[kRingStages];     // bulk-copy completion of each ring stage
  uint64_t empty[kRingStages];    // consumer warps done with the stage
  double red[kArnWarps][2 * kChunkMax];
  double part1[2 * kMaxRestart];  // this CTA's partial h1 (re, im), read by the whole cluster; atomics
  double part2[2 * kMaxRestart];  // partial h2
  double part3[2];                // partial |w''|^2
  double2 c1[kMaxRestart];        // cluster totals h1, h2
  double2 c2[kMaxRestart];
  double2 hcol[kMaxRestart + 1];  // Givens scratch (CTA 0)
  double2 snv[kMaxRestart];
  double csv[kMaxRestart];
  double hn2;
  double tol;   // this column's inner tolerance (CTA 0)
  double2 gk;   // g[k] of this column (CTA 0)
};

// Row li, unknowns 2p, 2p+1 of a staged chunk; the padding entry of an odd n
// reads as zero.
__device__ __forceinline__ float4 staged_pair(const float2* rows, int li, int units, int p, bool pad) {
  float4 v = *reinterpret_cast<const float4*>(rows + (size_t)li * units + 2 * p);
  if (pad) {
    v.z = 0.f;
    v.w = 0.f;
  }
  return v;
}

// The basis stream of one launch: every pass reads rows 0..k of this CTA's
// slice (ucta unknowns from i0) in nch chunks of `chunk` rows; chunk c of
// pass q is ring position g = q * nch + c, stage g % kRingStages.
struct ArnStream {
  const GmPtrs* P;
  ArnSmem* S;
  float2* ring;
  int s, k, i0, ucta, units, chunk, nch;
  __device__ float2* stage_rows(uint32_t g) const { return ring + (size_t)(g % kRingStages) * chunk * units; }
  // producer (one thread): wait until the stage is free, then bulk-copy the rows
  __device__ void produce(int pass, int c) const {
    const uint32_t g = (uint32_t)(pass * nch + c);
    const int st = (int)(g % kRingStages);
    if (g >= (uint32_t)kRingStages) mbar_wait(&S->empty[st], ((g / kRingStages) - 1u) & 1u, &P->st->err);
    const int l0 = c * chunk, nl = min(chunk, k + 1 - l0);
    const uint32_t row_bytes = (uint32_t)ucta * 8u;
    mbar_expect_tx(&S->full[st], row_bytes * (uint32_t)nl);
    float2* dst = stage_rows(g);
    // the basis is re-read every step: keep it in L2 while the matvec streams
    // the matrix evict-first
    const uint64_t pol = l2_evict_last_policy();
    for (int li = 0; li < nl; li++)
      bulk_load_hint(dst + (size_t)li * units, vrow(*P, s, l0 + li) + i0, row_bytes, &S->full[st], pol);
  }
  // consumer warps: wait for the chunk's rows
  __device__ const float2* acquire(int pass, int c) const {
    const uint32_t g = (uint32_t)(pass * nch + c);
    if (ucta > 0) mbar_wait(&S->full[g % kRingStages], (g / kRingStages) & 1u, &P->st->err);
    return stage_rows(g);
  }
  // consumer warps: the warp is done with the chunk's stage
  __device__ void release(int pass, int c) const {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&S->empty[(uint32_t)(pass * nch + c) % kRingStages]);
  }
};

// Dots pass (consumer threads own pairs, as in the update pass):
// part[2l + c] = sum over this CTA's unknowns of conj(V[l]) w.  Each thread
// forms its pairs' products for every row of the chunk in FP64 (exact for the
// FP32 basis: the projections carry no rounding that the Gram-Schmidt
// cancellation ||w|| / ||w'|| would amplify into lost orthogonality), a warp
// reduce-scatter sums the lanes, and
// each warp adds its partials to `part` (zeroed at launch) with FP64
// shared-memory atomics: no barrier between the consumer warps, which run
// through the chunks independently (the cluster barrier after the pass
// orders the atomics before the totals are read).

__device__ __forceinline__ void arn_dots(const ArnStream& T, int pass, const double2* __restrict__ wsl, int npairs,
                                         double* part) {
  const int tid = threadIdx.x, lane = tid & 31;
  for (int c = 0; c < T.nch; c++) {
    const float2* rows = T.acquire(pass, c);
    const int l0 = c * T.chunk, nl = min(T.chunk, T.k + 1 - l0);
    double v[2 * kChunkMax];
#pragma unroll
    for (int q = 0; q < 2 * kChunkMax; q++) v[q] = 0.0;
    for (int p = tid; p < npairs; p += kArnConsumers) {
      const bool pad = T.i0 + 2 * p + 1 >= T.P->n;
      const double2 w0 = wsl[2 * p], w1 = wsl[2 * p + 1];
#pragma unroll
      for (int li = 0; li < kChunkMax; li++) {
        if (li < nl) {
          const float4 a = staged_pair(rows, li, T.units, p, pad);
          const double ax = a.x, ay = a.y, az = a.z, aw = a.w;
          v[2 * li] = fma(ax, w0.x, fma(ay, w0.y, fma(az, w1.x, fma(aw, w1.y, v[2 * li]))));
          v[2 * li + 1] = fma(ax, w0.y, fma(-ay, w0.x, fma(az, w1.y, fma(-aw, w1.x, v[2 * li + 1]))));
        }
      }
    }
    const double t = warp_reduce_scatter<2 * kChunkMax>(v, lane);
    T.release(pass, c);  // this warp is done with the stage
    if ((lane & 1) == 0 && (lane >> 1) < 2 * nl) atomicAdd(&part[2 * l0 + (lane >> 1)], t);
  }
}

// Update pass (consumer threads own pairs): w -= V coef over this CTA's unknowns.
__device__ __forceinline__ void arn_update(const ArnStream& T, int pass, const double2* __restrict__ coef,
                                           double2* __restrict__ wsl, int npairs) {
  for (int c = 0; c < T.nch; c++) {
    const float2* rows = T.acquire(pass, c);
    const int l0 = c * T.chunk, nl = min(T.chunk, T.k + 1 - l0);
    for (int p = threadIdx.x; p < npairs; p += kArnConsumers) {
      const bool pad = T.i0 + 2 * p + 1 >= T.P->n;
      double2 a0 = wsl[2 * p], a1 = wsl[2 * p + 1];
#pragma unroll
      for (int li = 0; li < kChunkMax; li++) {
        if (li < nl) {
          const float4 v = staged_pair(rows, li, T.units, p, pad);
          const double2 cc = coef[l0 + li];
          a0.x -= (double)v.x * cc.x - (double)v.y * cc.y;
          a0.y -= (double)v.x * cc.y + (double)v.y * cc.x;
          a1.x -= (double)v.z * cc.x - (double)v.w * cc.y;
          a1.y -= (double)v.z * cc.y + (double)v.w * cc.x;
        }
      }
      wsl[2 * p] = a0;
      wsl[2 * p + 1] = a1;
    }
    T.release(pass, c);
  }
}

// dst[t] = sum over the cluster's CTAs of src[t], t < count (after a cluster barrier).
__device__ __forceinline__ void cluster_sum(cg::cluster_group& cluster, double* src, double* dst, int count) {
  const int nb = (int)cluster.num_blocks();
  for (int t = threadIdx.x; t < count; t += kArnThreads) {
    double v[kArnMaxCluster];
#pragma unroll
    for (int r = 0; r < kArnMaxCluster; r++) v[r] = r < nb ? cluster.map_shared_rank(src, r)[t] : 0.0;
    double sum = 0.0;
#pragma unroll
    for (int r = 0; r < kArnMaxCluster; r++) sum += v[r];
    dst[t] = sum;
  }
}

// One column's step record (one thread per column): the new step index
// and whether the column is still active, the latter also into the
// host-mapped ring slot of this launch.
__device__ __forceinline__ void column_done(const GmPtrs& P, int s, int k_next, bool still_active) {
  P.kcol[s] = k_next;
  const int step = P.colstep[s];
  P.colstep[s] = step + 1;
  reinterpret_cast<volatile int*>(P.snap)[(step % kSnapRing) * P.m + s] = still_active ? 1 : 0;
}

// Hessenberg column k of column s (hcol = h1 + h2, hcol[k+1] = hn), the
// previous rotations applied, the new complex Givens rotation, residual
// estimate and convergence (one warp; lane 0 applies the rotations, which is
// inherently sequential).  Returns on every lane whether s stays active.
__device__ __forceinline__ bool arn_givens(const GmPtrs& P, ArnSmem& S, int s, int k, double hn) {
  const int lane = threadIdx.x & 31;
  for (int l = lane; l <= k; l += 32) S.hcol[l] = make_double2(S.c1[l].x + S.c2[l].x, S.c1[l].y + S.c2[l].y);
  __syncwarp();
  int still = 0;
  if (lane == 0) {
    double2* hc = S.hcol;
    hc[k + 1] = make_double2(hn, 0.0);
    for (int l = 0; l < k; l++) {
      const double c = S.csv[l];
      const double2 sn = S.snv[l];
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
    const double2 gk = S.gk;
    const double2 gk1 = cmul(make_double2(-sn.x, sn.y), gk);
    gs[k + 1] = gk1;
    gs[k] = make_double2(c * gk.x, c * gk.y);
    const double res = sqrt(gk1.x * gk1.x + gk1.y * gk1.y);
    P.resid[s] = res;
    P.kend[s] = k + 1;
    const bool breakdown = !(hn > 1e-300) || !(hn > 1e-14 * rho);
    if (res <= S.tol || breakdown || k + 1 >= P.R) {
      P.active[s] = 0;
    } else {
      still = 1;
    }
  }
  __syncwarp();
  double2* Hk = P.H + ((size_t)s * P.R + k) * (P.R + 1);
  for (int l = lane; l <= k + 1; l += 32) Hk[l] = S.hcol[l];
  return __shfl_sync(0xffffffffu, still, 0) != 0;
}

// Dynamic shared memory of gm_arnoldi_kernel: ArnSmem, the CTA's slice of w
// (units complex doubles), the ring (kRingStages x chunk x units complex64).
__host__ __device__ constexpr size_t arn_ring_offset(int units) {
  return ((sizeof(ArnSmem) + sizeof(double2) * (size_t)units) + 127) / 128 * 128;
}
__host__ __device__ constexpr size_t arn_smem_bytes(int units, int chunk) {
  return arn_ring_offset(units) + sizeof(float2) * (size_t)kRingStages * chunk * units;
}

// grid (cluster size, m), cluster (cluster size, 1, 1).  reorth != 0 adds the
// second Gram-Schmidt pass (CGS2); without it the step is classical
// Gram-Schmidt (enough when a cycle only reduces the residual by ~1e-3 and the
// basis is stored in complex64).
__global__ void __launch_bounds__(kArnThreads, 1) gm_arnoldi_kernel(GmPtrs P, int units, int chunk, int reorth) {
  extern __shared__ __align__(128) unsigned char arn_raw[];
  ArnSmem& S = *reinterpret_cast<ArnSmem*>(arn_raw);
  double2* wsl = reinterpret_cast<double2*>(arn_raw + sizeof(ArnSmem));
  float2* ring = reinterpret_cast<float2*>(arn_raw + arn_ring_offset(units));
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const int s = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool producer = warp == kArnConsumerWarps;
  const int k = P.kcol[s];
  if (!P.active[s]) {  // uniform over the cluster: nobody waits for this column
    if (rank == 0 && tid == 0) column_done(P, s, k, false);
    return;
  }
  const int i0 = (int)rank * units;
  const int i1 = min(P.n, i0 + units);
  const int npairs = i1 > i0 ? (i1 - i0 + 1) / 2 : 0;
  ArnStream T;
  T.P = &P;
  T.S = &S;
  T.ring = ring;
  T.s = s;
  T.k = k;
  T.i0 = i0;
  T.ucta = 2 * npairs;
  T.units = units;
  T.chunk = chunk;
  T.nch = (k + chunk) / chunk;
  if (tid == 0) {
    for (int st = 0; st < kRingStages; st++) {
      mbar_init(&S.full[st], 1);
      mbar_init(&S.empty[st], kArnConsumerWarps);
    }
    mbar_init_fence();
  }
  if (rank == 0 && warp == 0) {  // Givens inputs, loaded while the passes run
    for (int l = lane; l < k; l += 32) {
      S.csv[l] = P.cs[s * P.R + l];
      S.snv[l] = P.sn[s * P.R + l];
    }
    if (lane == 0) {
      S.gk = P.g[(size_t)s * (P.R + 1) + k];
      S.tol = P.tol[s];
    }
  }

  // w = Y over this CTA's unknowns; Y = 0 for the next accumulating matvec
  for (int p = tid; p < npairs; p += kArnThreads) {
    const int i = i0 + 2 * p;
    float2* y0 = P.Y + (size_t)i * P.m + s;
    wsl[2 * p] = make_double2(y0->x, y0->y);
    *y0 = make_float2(0.f, 0.f);
    double2 w1 = make_double2(0.0, 0.0);
    if (i + 1 < P.n) {
      float2* y1 = P.Y + (size_t)(i + 1) * P.m + s;
      w1 = make_double2(y1->x, y1->y);
      *y1 = make_float2(0.f, 0.f);
    }
    wsl[2 * p + 1] = w1;
  }
  for (int t = tid; t < 2 * (k + 1); t += kArnThreads) {  // the dots passes accumulate into these
    S.part1[t] = 0.0;
    S.part2[t] = 0.0;
  }
  __syncthreads();

  // passes: dots h1, update; with reorth also dots h2, update.  The producer
  // issues each pass's chunks and, before the pass boundary, the first
  // stages of the next pass (their stages are freed within this pass).
  const int npass = reorth ? 4 : 2;
  int first = 0;
  for (int pass = 0; pass < npass; pass++) {
    const bool dots = (pass & 1) == 0;
    double* part = pass == 0 ? S.part1 : S.part2;
    double2* coef = pass == 1 ? S.c1 : S.c2;
    if (producer) {
      if (lane == 0 && T.ucta > 0) {
        for (int c = first; c < T.nch; c++) T.produce(pass, c);
        if (pass + 1 < npass)
          for (int c = 0; c < min(kRingStages, T.nch); c++) T.produce(pass + 1, c);
      }
      first = min(kRingStages, T.nch);
      __syncwarp();
    } else if (dots) {
      arn_dots(T, pass, wsl, npairs, part);
    } else {
      arn_update(T, pass, coef, wsl, npairs);
    }
    if (dots) {
      cluster.sync();
      cluster_sum(cluster, part, reinterpret_cast<double*>(pass == 0 ? S.c1 : S.c2), 2 * (k + 1));
    }
    __syncthreads();
  }
  if (!reorth)
    for (int t = tid; t <= k; t += kArnThreads) S.c2[t] = make_double2(0.0, 0.0);
  if (npairs > 0 && *(volatile int*)&P.st->err && producer && lane == 0) {
    // a wait expired: let the copies of the last chunks land before leaving
    const uint32_t gc = (uint32_t)(npass * T.nch);
    for (uint32_t g = gc > kRingStages ? gc - kRingStages : 0; g < gc; g++)
      mbar_wait_drain(&S.full[g % kRingStages], (g / kRingStages) & 1u);
  }
  double n2 = 0.0;
  for (int p = tid; p < npairs; p += kArnThreads) {
    const double2 a0 = wsl[2 * p], a1 = wsl[2 * p + 1];
    n2 += a0.x * a0.x + a0.y * a0.y + a1.x * a1.x + a1.y * a1.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if (lane == 0) S.red[warp][0] = n2;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kArnWarps; w++) t += S.red[w][0];
    S.part3[0] = t;
  }
  cluster.sync();
  if (tid == 0) {
    double t = 0.0;
    for (unsigned r = 0; r < cluster.num_blocks(); r++) t += cluster.map_shared_rank(S.part3, r)[0];
    S.hn2 = t;
  }
  cluster.sync();  // remote reads done before any CTA leaves; publishes hn2 in the CTA
  const double hn = sqrt(S.hn2);
  const double inv = hn > 0.0 ? 1.0 / hn : 0.0;

  // v_{k+1} and the next matvec operand
  float2* vk1 = P.Vb + ((size_t)s * (P.R + 1) + k + 1) * P.ldv;
  for (int p = tid; p < npairs; p += kArnThreads) {
    const int i = i0 + 2 * p;
    const double2 a0 = wsl[2 * p], a1 = wsl[2 * p + 1];
    const float2 f0 = make_float2((float)(a0.x * inv), (float)(a0.y * inv));
    const float2 f1 = i + 1 < P.n ? make_float2((float)(a1.x * inv), (float)(a1.y * inv)) : make_float2(0.f, 0.f);
    *reinterpret_cast<float4*>(vk1 + i) = make_float4(f0.x, f0.y, f1.x, f1.y);
    store_operand(P, i, s, f0, f1);
  }
  if (rank == 0 && warp == 0) {
    const bool still = arn_givens(P, S, s, k, hn);
    if (lane == 0) column_done(P, s, k + 1, still);
  }
}

// ---------------------------------------------------------------------------
// Streamed Arnoldi step: launches over all SMs, no clusters, classical
// Gram-Schmidt with selective reorthogonalisation (the criterion of Daniel,
// Gragg, Kaufman and Stewart): a column gets a second pass only when the
// first one removed most of w, |w'|^2 < |w|^2 / 2.
//   gm_st_dots_kernel<0>    h1 = V^H Y (Y = this step's matvec output) and |Y|^2:
//                           FP32 products per thread, FP64 block sums, FP64 atomics
//   gm_st_update_kernel<0>  w' = Y - V h1 in FP64 -> P.w, Y cleared, |w'|^2
//   gm_st_dots_kernel<1>,   for the columns that need it: h2 = V^H w',
//   gm_st_update_kernel<1>  w'' = w' - V h2 -> P.w, |w''|^2
//   gm_st_finish_kernel     v_{k+1} = w / |w| -> basis and the next matvec operand
//   gm_st_givens_kernel     one warp per column: Givens rotation of h1 + h2 and
//                           the step record (k + 1, activity); a separate
//                           launch because every block of the other kernels
//                           reads k and the activity flag that it advances
// The sums are double-buffered by the column's step parity: a step's finish
// kernel clears the other buffer for the next step (the cycle start clears
// both).
// ---------------------------------------------------------------------------
constexpr int kStThreads = 256;
constexpr int kStRows = 8;  // basis rows per register chunk of the dots pass

__device__ __forceinline__ double* st_hacc(const GmPtrs& P, int buf, int s, int pass) {
  return P.hacc + (((size_t)buf * P.m + s) * 2 + pass) * 2 * (P.R + 1);
}
// j = 0: |w|^2 before the first pass, 1: after it, 2: after the second
__device__ __forceinline__ double* st_nacc(const GmPtrs& P, int buf, int s, int j) {
  return P.nacc + ((size_t)buf * P.m + s) * 3 + j;
}
__device__ __forceinline__ bool st_reorth(const GmPtrs& P, int buf, int s) {
  return *st_nacc(P, buf, s, 1) < 0.5 * *st_nacc(P, buf, s, 0);
}

// Block sum of v (all threads), added to *dst by thread 0; red: kStThreads / 32 doubles.
__device__ __forceinline__ void st_block_add(double v, double* red, double* dst) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kStThreads / 32; w++) t += red[w];
    atomicAdd(dst, t);
  }
}

// Row l, unknowns i, i+1 of column s's basis; the padding entry of an odd n reads as zero.
__device__ __forceinline__ float4 st_pair(const GmPtrs& P, int s, int l, int i) {
  float4 v = *reinterpret_cast<const float4*>(vrow(P, s, l) + i);
  if (i + 1 >= P.n) {
    v.z = 0.f;
    v.w = 0.f;
  }
  return v;
}

// Work item q of a streamed kernel: column q / nb, pairs [b span, (b+1) span)
// of it, b = q % nb; persistent grids loop over the items.
template <int PASS>
__global__ void __launch_bounds__(kStThreads) gm_st_dots_kernel(GmPtrs P, int span, int nb) {
  extern __shared__ __align__(16) double4 wst[];  // the item's w, span pairs
  __shared__ double hs[2 * kMaxRestart];
  __shared__ double red[kStThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31;
  const int npairs = (P.n + 1) / 2;
  for (int q = blockIdx.x; q < P.m * nb; q += gridDim.x) {  // uniform over the block
    const int s = q / nb, p0 = (q - s * nb) * span, p1 = min(npairs, p0 + span);
    if (!P.active[s] || p0 >= p1) continue;
    const int k = P.kcol[s];
    if (PASS == 1 && !st_reorth(P, k & 1, s)) continue;
    __syncthreads();  // the previous item is done with hs, red and wst
    for (int t = tid; t < 2 * (k + 1); t += kStThreads) hs[t] = 0.0;
    double n2 = 0.0;
    for (int p = p0 + tid; p < p1; p += kStThreads) {
      const int i = 2 * p;
      double4 w;
      if (PASS == 0) {
        const float2 y0 = P.Y[(size_t)i * P.m + s];
        const float2 y1 = i + 1 < P.n ? P.Y[(size_t)(i + 1) * P.m + s] : make_float2(0.f, 0.f);
        w = make_double4(y0.x, y0.y, y1.x, y1.y);
        n2 += w.x * w.x + w.y * w.y + w.z * w.z + w.w * w.w;
      } else {
        const double2 a0 = P.w[(size_t)s * P.n + i];
        const double2 a1 = i + 1 < P.n ? P.w[(size_t)s * P.n + i + 1] : make_double2(0.0, 0.0);
        w = make_double4(a0.x, a0.y, a1.x, a1.y);
      }
      wst[p - p0] = w;
    }
    if (PASS == 0) st_block_add(n2, red, st_nacc(P, k & 1, s, 0));  // syncs the block
    __syncthreads();
    for (int c0 = 0; c0 <= k; c0 += kStRows) {
      const int nl = min(kStRows, k + 1 - c0);
      double v[2 * kStRows];
#pragma unroll
      for (int r = 0; r < 2 * kStRows; r++) v[r] = 0.0;
      for (int p = p0 + tid; p < p1; p += kStThreads) {
        const double4 w = wst[p - p0];
#pragma unroll
        for (int li = 0; li < kStRows; li++) {
          if (li < nl) {
            const float4 a = st_pair(P, s, c0 + li, 2 * p);
            const double ax = a.x, ay = a.y, az = a.z, aw = a.w;
            v[2 * li] = fma(ax, w.x, fma(ay, w.y, fma(az, w.z, fma(aw, w.w, v[2 * li]))));
            v[2 * li + 1] = fma(ax, w.y, fma(-ay, w.x, fma(az, w.w, fma(-aw, w.z, v[2 * li + 1]))));
          }
        }
      }
      const double t = warp_reduce_scatter<2 * kStRows>(v, lane);
      if ((lane & 1) == 0 && (lane >> 1) < 2 * nl) atomicAdd(&hs[2 * c0 + (lane >> 1)], t);
    }
    __syncthreads();
    double* hacc = st_hacc(P, k & 1, s, PASS);
    for (int t = tid; t < 2 * (k + 1); t += kStThreads) atomicAdd(&hacc[t], hs[t]);
  }
}

template <int PASS>
__global__ void __launch_bounds__(kStThreads) gm_st_update_kernel(GmPtrs P, int span, int nb) {
  __shared__ double2 h[kMaxRestart];
  __shared__ double red[kStThreads / 32];
  const int tid = threadIdx.x;
  const int npairs = (P.n + 1) / 2;
  for (int q = blockIdx.x; q < P.m * nb; q += gridDim.x) {  // uniform over the block
    const int s = q / nb, p0 = (q - s * nb) * span, p1 = min(npairs, p0 + span);
    if (!P.active[s] || p0 >= p1) continue;
    const int k = P.kcol[s];
    if (PASS == 1 && !st_reorth(P, k & 1, s)) continue;
    const double* hacc = st_hacc(P, k & 1, s, PASS);
    __syncthreads();  // the previous item is done with h and red
    for (int l = tid; l <= k; l += kStThreads) h[l] = make_double2(hacc[2 * l], hacc[2 * l + 1]);
    __syncthreads();
    double n2 = 0.0;
    for (int p = p0 + tid; p < p1; p += kStThreads) {
      const int i = 2 * p;
      double2 a0, a1;
      if (PASS == 0) {
        float2* y0p = P.Y + (size_t)i * P.m + s;
        const float2 y0 = *y0p;
        *y0p = make_float2(0.f, 0.f);
        float2 y1 = make_float2(0.f, 0.f);
        if (i + 1 < P.n) {
          float2* y1p = P.Y + (size_t)(i + 1) * P.m + s;
          y1 = *y1p;
          *y1p = make_float2(0.f, 0.f);
        }
        a0 = make_double2(y0.x, y0.y);
        a1 = make_double2(y1.x, y1.y);
      } else {
        a0 = P.w[(size_t)s * P.n + i];
        a1 = i + 1 < P.n ? P.w[(size_t)s * P.n + i + 1] : make_double2(0.0, 0.0);
      }
#pragma unroll 4
      for (int l = 0; l <= k; l++) {
        const float4 v = st_pair(P, s, l, i);
        const double2 cc = h[l];
        a0.x -= (double)v.x * cc.x - (double)v.y * cc.y;
        a0.y -= (double)v.x * cc.y + (double)v.y * cc.x;
        a1.x -= (double)v.z * cc.x - (double)v.w * cc.y;
        a1.y -= (double)v.z * cc.y + (double)v.w * cc.x;
      }
      P.w[(size_t)s * P.n + i] = a0;
      if (i + 1 < P.n) P.w[(size_t)s * P.n + i + 1] = a1;
      n2 += a0.x * a0.x + a0.y * a0.y + a1.x * a1.x + a1.y * a1.y;
    }
    st_block_add(n2, red, st_nacc(P, k & 1, s, 1 + PASS));
  }
}

__global__ void __launch_bounds__(kStThreads) gm_st_finish_kernel(GmPtrs P, int span, int nb) {
  const int tid = threadIdx.x;
  const int npairs = (P.n + 1) / 2;
  for (int q = blockIdx.x; q < P.m * nb; q += gridDim.x) {
    const int s = q / nb, b = q - s * nb, p0 = b * span, p1 = min(npairs, p0 + span);
    if (!P.active[s]) continue;
    const int k = P.kcol[s];
    const int buf = k & 1;
    const double hn = sqrt(*st_nacc(P, buf, s, st_reorth(P, buf, s) ? 2 : 1));
    const double inv = hn > 0.0 ? 1.0 / hn : 0.0;
    float2* vk1 = P.Vb + ((size_t)s * (P.R + 1) + k + 1) * P.ldv;
    for (int p = p0 + tid; p < p1; p += kStThreads) {
      const int i = 2 * p;
      const double2 a0 = P.w[(size_t)s * P.n + i];
      const double2 a1 = i + 1 < P.n ? P.w[(size_t)s * P.n + i + 1] : make_double2(0.0, 0.0);
      const float2 f0 = make_float2((float)(a0.x * inv), (float)(a0.y * inv));
      const float2 f1 =
          i + 1 < P.n ? make_float2((float)(a1.x * inv), (float)(a1.y * inv)) : make_float2(0.f, 0.f);
      *reinterpret_cast<float4*>(vk1 + i) = make_float4(f0.x, f0.y, f1.x, f1.y);
      store_operand(P, i, s, f0, f1);
    }
    if (b == 0) {  // the next step's sums start from zero (nobody reads that buffer now)
      double* hnext = st_hacc(P, buf ^ 1, s, 0);  // both passes, contiguous
      for (int t = tid; t < 4 * (P.R + 1); t += kStThreads) hnext[t] = 0.0;
      if (tid < 3) *st_nacc(P, buf ^ 1, s, tid) = 0.0;
    }
  }
}

// One warp (block) per column, after gm_st_finish_kernel.
__global__ void __launch_bounds__(32) gm_st_givens_kernel(GmPtrs P) {
  extern __shared__ __align__(16) unsigned char st_raw[];  // ArnSmem
  const int s = blockIdx.x, lane = threadIdx.x;
  const int k = P.kcol[s];
  if (!P.active[s]) {
    if (lane == 0) column_done(P, s, k, false);
    return;
  }
  const int buf = k & 1;
  const bool two = st_reorth(P, buf, s);
  const double hn = sqrt(*st_nacc(P, buf, s, two ? 2 : 1));
  ArnSmem& S = *reinterpret_cast<ArnSmem*>(st_raw);
  const double* h1 = st_hacc(P, buf, s, 0);
  const double* h2 = st_hacc(P, buf, s, 1);
  for (int l = lane; l <= k; l += 32) {
    S.c1[l] = make_double2(h1[2 * l], h1[2 * l + 1]);
    S.c2[l] = two ? make_double2(h2[2 * l], h2[2 * l + 1]) : make_double2(0.0, 0.0);
  }
  for (int l = lane; l < k; l += 32) {
    S.csv[l] = P.cs[s * P.R + l];
    S.snv[l] = P.sn[s * P.R + l];
  }
  if (lane == 0) {
    S.gk = P.g[(size_t)s * (P.R + 1) + k];
    S.tol = P.tol[s];
  }
  __syncwarp();
  const bool still = arn_givens(P, S, s, k, hn);
  if (lane == 0) column_done(P, s, k + 1, still);
}

// ---------------------------------------------------------------------------
// Cooperative Arnoldi step (one classical Gram-Schmidt pass): ONE launch of a
// cooperative grid over all SMs, every CTA resident and owning a contiguous
// range of unknowns for every column, with two grid-wide barriers:
//   load    w = Y over the CTA's unknowns (FP64, shared memory); Y = 0 for
//           the next accumulating matvec
//   dots    h = V^H w.  Work items are (column, 4 basis rows); each compute
//           warp takes every 8th item and streams its rows of the CTA's
//           unknowns through its own ring of shared-memory slots with 1-D
//           bulk async copies (mbarrier completion, bounded waits), its lane
//           0 issuing ahead, so a whole ring of copies is in flight per warp.
//           Lanes own unknown pairs: FP64 products (exact for the FP32
//           basis), a warp reduce-scatter, FP64 atomics into the column's h
//           (P.hacc, by the column's step parity).
//   == grid barrier ==  (the ring already holds the first rows of the next pass)
//   update  w' = w - V h, the same items and ring (h read from L2, every
//           lane the same address), contributions subtracted from w in
//           shared memory with FP64 shared atomics; |w'|^2 per column, FP64
//           atomics (P.nacc).  Meanwhile the Givens warp of the CTA that owns
//           the column (CTA c: columns c, c + G, ...) applies its previous
//           rotations to h, which is inherently sequential.
//   == grid barrier ==
//   finish  v_{k+1} = w' / |w'| -> basis and the next matvec operand; the
//           Givens warp adds the new rotation, the residual estimate and the
//           step record (k + 1, activity, host-mapped snapshot)
// Every CTA streams the same number of basis bytes; a step costs one launch
// and two barriers.  Barrier and copy waits are bounded (P.st->err on expiry;
// copies still in flight are drained before the CTA exits).
// ---------------------------------------------------------------------------
constexpr int kCoComputeWarps = 8;
constexpr int kCoCompute = 32 * kCoComputeWarps;  // 256 compute threads
constexpr int kCoThreads = kCoCompute + 32;       // + the Givens warp
constexpr int kCoRows = 4;                        // basis rows per work item
constexpr int kCoMaxColsPerCta = 4;               // columns whose rotations one CTA applies
constexpr unsigned long long kCoWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier of the cooperative step (all CTAs resident).  Thread 0
// of each CTA arrives; the last one resets the count and advances the
// generation.  The wait is bounded: on expiry (or once anyone raised the
// error flag) the CTA goes on and P.st->err is set, so the solve reports
// BEM_ERR_CUDA instead of hanging.
__device__ __forceinline__ void co_grid_sync(GmState* st) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_acquire_u32(&st->bar_gen);
    __threadfence();  // this CTA's writes and atomics before the arrival
    const unsigned arrived = atomicAdd(&st->bar_count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      const unsigned long long t0 = globaltimer();
      for (unsigned it = 0;; it++) {
        if (ld_acquire_u32(&st->bar_gen) != gen) break;
        if ((it & 31u) == 0u) {
          if (*(volatile int*)&st->err) break;
          if (globaltimer() - t0 > kCoWaitNs) {
            atomicExch(&st->err, 1);
            break;
          }
        }
        __nanosleep(64);
      }
    }
    __threadfence();  // the other CTAs' writes are visible after the barrier
  }
  __syncthreads();
}

__device__ __forceinline__ void co_compute_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kCoCompute) : "memory"); }

// Dynamic shared memory: ks[m] act[m] | wsm[m][2 npc] | nsm[m] | full[8][slots]
// | ring[8][slots][kCoRows][2 npc] | per owned column: hc[R+1], snv[R]
// (double2), csv[R], misc[2] (double2, 16-byte aligned).
struct CoLayout {
  size_t ks, act, wsm, nsm, full, ring, giv, total;
  int giv_stride;  // bytes of one column's Givens scratch
  int slot_floats;  // float2 entries of one ring slot
};
__host__ __device__ inline CoLayout co_layout(int m, int npc, int R, int cpc, int slots) {
  CoLayout L;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t r = o;
    o = (o + b + 15) / 16 * 16;
    return r;
  };
  L.ks = take(sizeof(int) * m);
  L.act = take(sizeof(int) * m);
  L.wsm = take(sizeof(double2) * (size_t)m * 2 * npc);
  L.nsm = take(sizeof(double) * m);
  L.full = take(sizeof(uint64_t) * kCoComputeWarps * slots);
  L.slot_floats = kCoRows * 2 * npc;
  L.ring = take(sizeof(float2) * (size_t)L.slot_floats * kCoComputeWarps * slots);
  L.giv_stride = (int)((sizeof(double2) * (R + 1) + sizeof(double2) * R + sizeof(double) * R + 16 +
                        2 * sizeof(double2) + 15) / 16 * 16);
  L.giv = take((size_t)L.giv_stride * cpc);
  L.total = o;
  return L;
}

__device__ __forceinline__ double2* co_misc(double* csv, int R) {
  return reinterpret_cast<double2*>(((uintptr_t)(csv + R) + 15) & ~(uintptr_t)15);
}

// The work items of a pass: (column s, rows 4c .. 4c+3), it = s nch + c,
// present when the column is active and 4c <= k_s.
struct CoItems {
  const int* ks;
  const int* act;
  int nch, total;
  __device__ bool valid(int it) const {
    const int s = it / nch, c = it - s * nch;
    return act[s] && kCoRows * c <= ks[s];
  }
  // the first valid item at or after `it` in this warp's sequence (stride 8)
  __device__ int next(int it) const {
    while (it < total && !valid(it)) it += kCoComputeWarps;
    return it;
  }
};

__global__ void __launch_bounds__(kCoThreads, 1)
    gm_arnoldi_coop_kernel(GmPtrs P, int npc, int cpc, int slots) {
  extern __shared__ __align__(16) unsigned char co_raw[];
  const int m = P.m, R = P.R;
  const CoLayout Lo = co_layout(m, npc, R, cpc, slots);
  int* ks = reinterpret_cast<int*>(co_raw + Lo.ks);
  int* act = reinterpret_cast<int*>(co_raw + Lo.act);
  double2* wsm = reinterpret_cast<double2*>(co_raw + Lo.wsm);
  double* nsm = reinterpret_cast<double*>(co_raw + Lo.nsm);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool giv_warp = warp == kCoComputeWarps;
  const int npairs_all = (P.n + 1) / 2;
  const int p_begin = blockIdx.x * npc;
  const int nvp = max(0, min(npc, npairs_all - p_begin));  // valid pairs of this CTA
  const int i0 = 2 * p_begin;
  const int rows = 2 * npc;  // wsm row stride and ring row stride (float2)

  for (int s = tid; s < m; s += kCoThreads) {
    ks[s] = P.kcol[s];
    act[s] = P.active[s];
  }
  if (tid < kCoComputeWarps * slots) mbar_init(reinterpret_cast<uint64_t*>(co_raw + Lo.full) + tid, 1);
  mbar_init_fence();
  __syncthreads();
  int kmax = -1;
  for (int s = 0; s < m; s++)
    if (act[s]) kmax = max(kmax, ks[s]);
  CoItems items;
  items.ks = ks;
  items.act = act;
  items.nch = kmax >= 0 ? kmax / kCoRows + 1 : 1;
  items.total = (kmax >= 0 && nvp > 0) ? m * items.nch : 0;

  // this warp's ring: slot q holds kCoRows rows of 2 nvp unknowns (row stride 2 npc)
  uint64_t* full = reinterpret_cast<uint64_t*>(co_raw + Lo.full) + (giv_warp ? 0 : warp) * slots;
  float2* ring = reinterpret_cast<float2*>(co_raw + Lo.ring) + (size_t)(giv_warp ? 0 : warp) * slots * Lo.slot_floats;
  const uint64_t pol = l2_evict_last_policy();
  const uint32_t row_bytes = (uint32_t)nvp * 16u;
  // the warp's sequence: its items of the dots pass, then the same items again for the update pass
  // next item to issue and its pass (2: nothing left); a warp without items
  // in the dots pass has none in the update pass either
  int iss = giv_warp ? items.total : items.next(warp);
  int iss_pass = iss < items.total ? 0 : 2;
  unsigned nissued = 0, nconsumed = 0;
  auto issue = [&]() {  // lane 0: bulk-copy the next item of the sequence into its slot
    if (iss_pass > 1) return;
    if (lane == 0) {
      const int s = iss / items.nch, c = iss - s * items.nch;
      const int l0 = kCoRows * c, nl = min(kCoRows, ks[s] + 1 - l0);
      uint64_t* bar = &full[nissued % slots];
      float2* dst = ring + (size_t)(nissued % slots) * Lo.slot_floats;
      mbar_expect_tx(bar, row_bytes * (uint32_t)nl);
      for (int li = 0; li < nl; li++) bulk_load_hint(dst + (size_t)li * rows, vrow(P, s, l0 + li) + i0, row_bytes, bar, pol);
    }
    nissued++;
    iss = items.next(iss + kCoComputeWarps);
    if (iss >= items.total && iss_pass == 0) {
      iss_pass = 1;
      iss = items.next(warp);
    } else if (iss >= items.total) {
      iss_pass = 2;
    }
  };
  // consumer: wait for the next slot.  If the bounded wait expires (the error
  // flag is raised) it still lets the copy land, so the slot accounting stays
  // in step and no copy is left in flight; false only if that drain expires too.
  auto acquire = [&](const float2** rowsp) -> bool {
    const unsigned q = nconsumed % slots;
    const uint32_t par = (nconsumed / slots) & 1u;
    bool ok = mbar_wait(&full[q], par, &P.st->err);
    if (!ok) ok = mbar_wait_drain(&full[q], par);
    *rowsp = ring + (size_t)q * Lo.slot_floats;
    return ok;
  };

  // ---- load w = Y (all columns; Y cleared), clear the next step's sums ----
  if (!giv_warp) {
    for (int d = 0; d < slots && iss_pass < 2 && items.total > 0; d++) issue();  // rows start landing now
    for (int t = tid; t < 2 * npc * m; t += kCoCompute) {
      const int il = t / m, s = t - il * m;
      const int i = i0 + il;
      double2 w = make_double2(0.0, 0.0);
      if (il < 2 * nvp && i < P.n) {
        float2* y = P.Y + (size_t)i * m + s;
        const float2 yv = *y;
        w = make_double2(yv.x, yv.y);
        *y = make_float2(0.f, 0.f);
      }
      wsm[(size_t)s * rows + il] = w;
    }
    // the sums of the next step (other parity) start from zero; nobody reads them now
    const size_t per = 2 * (size_t)(R + 1);
    for (size_t t = (size_t)blockIdx.x * kCoCompute + tid; t < (size_t)m * (per + 1);
         t += (size_t)gridDim.x * kCoCompute) {
      const int s = (int)(t / (per + 1));
      const size_t j = t - (size_t)s * (per + 1);
      const int nb = (ks[s] & 1) ^ 1;
      if (j < per)
        st_hacc(P, nb, s, 0)[j] = 0.0;
      else
        *st_nacc(P, nb, s, 1) = 0.0;
    }
  }
  __syncthreads();

  // ---- dots: h += V^H w over this CTA's unknowns ----
  if (!giv_warp) {
    for (int it = items.next(warp); it < items.total; it = items.next(it + kCoComputeWarps)) {
      const int s = it / items.nch, c = it - s * items.nch;
      const int l0 = kCoRows * c, nl = min(kCoRows, ks[s] + 1 - l0);
      const float2* rw;
      const bool ok = acquire(&rw);
      double v[2 * kCoRows];
#pragma unroll
      for (int q = 0; q < 2 * kCoRows; q++) v[q] = 0.0;
      if (ok) {
        const double2* ws = wsm + (size_t)s * rows;
        for (int p = lane; p < nvp; p += 32) {
          const bool pad = i0 + 2 * p + 1 >= P.n;
          const double2 w0 = ws[2 * p], w1 = ws[2 * p + 1];
#pragma unroll
          for (int li = 0; li < kCoRows; li++) {
            if (li < nl) {
              float4 a = *reinterpret_cast<const float4*>(rw + (size_t)li * rows + 2 * p);
              if (pad) {
                a.z = 0.f;
                a.w = 0.f;
              }
              const double ax = a.x, ay = a.y, az = a.z, aw = a.w;
              v[2 * li] = fma(ax, w0.x, fma(ay, w0.y, fma(az, w1.x, fma(aw, w1.y, v[2 * li]))));
              v[2 * li + 1] = fma(ax, w0.y, fma(-ay, w0.x, fma(az, w1.y, fma(-aw, w1.x, v[2 * li + 1]))));
            }
          }
        }
      }
      __syncwarp();  // every lane is done with the slot
      nconsumed++;
      issue();
      const double tsum = warp_reduce_scatter<2 * kCoRows>(v, lane);
      if ((lane & 3) == 0 && (lane >> 2) < 2 * nl && tsum != 0.0)
        atomicAdd(st_hacc(P, ks[s] & 1, s, 0) + 2 * l0 + (lane >> 2), tsum);
    }
  }
  co_grid_sync(P.st);

  // ---- update (compute warps) and the previous rotations (Givens warp) ----
  if (!giv_warp) {
    for (int it = items.next(warp); it < items.total; it = items.next(it + kCoComputeWarps)) {
      const int s = it / items.nch, c = it - s * items.nch;
      const int l0 = kCoRows * c, nl = min(kCoRows, ks[s] + 1 - l0);
      const double* hp = st_hacc(P, ks[s] & 1, s, 0) + 2 * l0;
      double2 h[kCoRows];
#pragma unroll
      for (int li = 0; li < kCoRows; li++)
        h[li] = li < nl ? make_double2(__ldcg(hp + 2 * li), __ldcg(hp + 2 * li + 1)) : make_double2(0.0, 0.0);
      const float2* rw;
      const bool ok = acquire(&rw);
      if (ok) {
        double2* ws = wsm + (size_t)s * rows;
        for (int p = lane; p < nvp; p += 32) {
          const bool pad = i0 + 2 * p + 1 >= P.n;
          double2 d0 = make_double2(0.0, 0.0), d1 = make_double2(0.0, 0.0);
#pragma unroll
          for (int li = 0; li < kCoRows; li++) {
            if (li < nl) {
              float4 v = *reinterpret_cast<const float4*>(rw + (size_t)li * rows + 2 * p);
              if (pad) {
                v.z = 0.f;
                v.w = 0.f;
              }
              const double2 cc = h[li];
              d0.x = fma((double)v.x, cc.x, fma(-(double)v.y, cc.y, d0.x));
              d0.y = fma((double)v.x, cc.y, fma((double)v.y, cc.x, d0.y));
              d1.x = fma((double)v.z, cc.x, fma(-(double)v.w, cc.y, d1.x));
              d1.y = fma((double)v.z, cc.y, fma((double)v.w, cc.x, d1.y));
            }
          }
          atomicAdd(&ws[2 * p].x, -d0.x);
          atomicAdd(&ws[2 * p].y, -d0.y);
          atomicAdd(&ws[2 * p + 1].x, -d1.x);
          atomicAdd(&ws[2 * p + 1].y, -d1.y);
        }
      }
      __syncwarp();
      nconsumed++;
      issue();
    }
    for (int s = tid; s < m; s += kCoCompute) nsm[s] = 0.0;
    co_compute_sync();  // every update of wsm is done
    for (int u = tid; u < m * npc; u += kCoCompute) {
      const int s = u / npc, p = u - s * npc;
      if (!act[s] || p >= nvp) continue;
      const double2 a0 = wsm[(size_t)s * rows + 2 * p], a1 = wsm[(size_t)s * rows + 2 * p + 1];
      atomicAdd(&nsm[s], a0.x * a0.x + a0.y * a0.y + a1.x * a1.x + a1.y * a1.y);
    }
    co_compute_sync();
    for (int s = tid; s < m; s += kCoCompute)
      if (act[s] && nsm[s] != 0.0) atomicAdd(st_nacc(P, ks[s] & 1, s, 1), nsm[s]);
    if (lane == 0) {  // every issued copy was consumed; make sure the last use of each slot has landed
      for (unsigned q = nissued > (unsigned)slots ? nissued - slots : 0u; q < nissued; q++)
        mbar_wait_drain(&full[q % slots], (q / slots) & 1u);
    }
  } else {
    // Givens warp: columns s = blockIdx.x + q gridDim.x
    for (int q = 0; q < cpc; q++) {
      const int s = blockIdx.x + q * gridDim.x;
      if (s >= m || !act[s]) continue;
      unsigned char* gv = co_raw + Lo.giv + (size_t)q * Lo.giv_stride;
      double2* hc = reinterpret_cast<double2*>(gv);
      double2* snv = hc + (R + 1);
      double* csv = reinterpret_cast<double*>(snv + R);
      double2* misc = co_misc(csv, R);  // [0] = g_k, [1].x = tol
      const int k = ks[s];
      const double* h = st_hacc(P, k & 1, s, 0);
      for (int l = lane; l <= k; l += 32) hc[l] = make_double2(__ldcg(h + 2 * l), __ldcg(h + 2 * l + 1));
      for (int l = lane; l < k; l += 32) {
        csv[l] = P.cs[s * R + l];
        snv[l] = P.sn[s * R + l];
      }
      if (lane == 0) {
        misc[0] = P.g[(size_t)s * (R + 1) + k];
        misc[1] = make_double2(P.tol[s], 0.0);
      }
      __syncwarp();
      if (lane == 0) {
        // previous rotations, sequential: hc[l], hc[l+1] <- (c a + sn b, -conj(sn) a + c b)
        double2 a = hc[0];
        for (int l = 0; l < k; l++) {
          const double c = csv[l];
          const double2 sn = snv[l];
          const double2 b = hc[l + 1];
          const double2 sb = cmul(sn, b);
          const double2 t = cmul(make_double2(-sn.x, sn.y), a);
          hc[l] = make_double2(c * a.x + sb.x, c * a.y + sb.y);
          a = make_double2(t.x + c * b.x, t.y + c * b.y);
        }
        hc[k] = a;
      }
      __syncwarp();
    }
  }
  co_grid_sync(P.st);

  // ---- finish: v_{k+1} = w' / |w'| and the next operand ----
  if (!giv_warp) {
    for (int u = tid; u < m * npc; u += kCoCompute) {
      const int s = u / npc, p = u - s * npc;
      if (!act[s] || p >= nvp) continue;
      const int k = ks[s];
      const double hn = sqrt(__ldcg(st_nacc(P, k & 1, s, 1)));
      const double inv = hn > 0.0 ? 1.0 / hn : 0.0;
      const int i = i0 + 2 * p;
      const double2 a0 = wsm[(size_t)s * rows + 2 * p], a1 = wsm[(size_t)s * rows + 2 * p + 1];
      const float2 f0 = make_float2((float)(a0.x * inv), (float)(a0.y * inv));
      const float2 f1 = i + 1 < P.n ? make_float2((float)(a1.x * inv), (float)(a1.y * inv)) : make_float2(0.f, 0.f);
      *reinterpret_cast<float4*>(P.Vb + ((size_t)s * (R + 1) + k + 1) * P.ldv + i) = make_float4(f0.x, f0.y, f1.x, f1.y);
      store_operand(P, i, s, f0, f1);
    }
  } else {
    for (int q = 0; q < cpc; q++) {
      const int s = blockIdx.x + q * gridDim.x;
      if (s >= m) continue;
      const int k = ks[s];
      if (!act[s]) {
        if (lane == 0) column_done(P, s, k, false);
        continue;
      }
      unsigned char* gv = co_raw + Lo.giv + (size_t)q * Lo.giv_stride;
      double2* hc = reinterpret_cast<double2*>(gv);
      double2* snv = hc + (R + 1);
      double* csv = reinterpret_cast<double*>(snv + R);
      double2* misc = co_misc(csv, R);
      const double hn = sqrt(__ldcg(st_nacc(P, k & 1, s, 1)));
      int still = 0;
      if (lane == 0) {
        const double2 a = hc[k];
        const double na = sqrt(a.x * a.x + a.y * a.y), nb = hn;
        const double rho = sqrt(na * na + nb * nb);
        double c;
        double2 sn;
        if (rho == 0.0) {
          c = 1.0;
          sn = make_double2(0.0, 0.0);
        } else if (na == 0.0) {
          c = 0.0;
          sn = make_double2(1.0, 0.0);  // conj(hn)/|hn|, hn real and positive
          hc[k] = make_double2(nb, 0.0);
        } else {
          c = na / rho;
          const double2 ph = make_double2(a.x / na, a.y / na);
          sn = make_double2(ph.x * nb / rho, ph.y * nb / rho);  // ph conj(b)/rho, b = hn real
          hc[k] = make_double2(ph.x * rho, ph.y * rho);
        }
        hc[k + 1] = make_double2(0.0, 0.0);
        P.cs[s * R + k] = c;
        P.sn[s * R + k] = sn;
        double2* gs = P.g + (size_t)s * (R + 1);
        const double2 gk = misc[0];
        const double2 gk1 = cmul(make_double2(-sn.x, sn.y), gk);
        gs[k + 1] = gk1;
        gs[k] = make_double2(c * gk.x, c * gk.y);
        const double res = sqrt(gk1.x * gk1.x + gk1.y * gk1.y);
        P.resid[s] = res;
        P.kend[s] = k + 1;
        const bool breakdown = !(hn > 1e-300) || !(hn > 1e-14 * rho);
        if (res <= misc[1].x || breakdown || k + 1 >= R)
          P.active[s] = 0;
        else
          still = 1;
      }
      __syncwarp();
      double2* Hk = P.H + ((size_t)s * R + k) * (R + 1);
      for (int l = lane; l <= k + 1; l += 32) Hk[l] = hc[l];
      still = __shfl_sync(0xffffffffu, still, 0);
      if (lane == 0) column_done(P, s, k + 1, still != 0);
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Block GMRES step (2 <= m <= kBkMaxP right-hand sides sharing ONE block
// Krylov space).  On the BEM operators the block space converges in about a
// quarter of the operator applications of m separate Krylov spaces (30
// against 118 at s4 with 8 right-hand sides), because each application
// extends the space by m directions.  Per step, one cooperative launch over
// all SMs (CTAs own nr unknowns of every column; the block size p is padded
// to PP = 4, 8 or 16 columns):
//   W = Y (this step's matvec output, FP64 in shared memory; Y cleared)
//   H = Q^H W   the basis rows over this CTA's unknowns stream through a ring
//               of 32-vector stages (1-D bulk copies of the complex64 rows,
//               converted to FP64 on use); thread (vector, 4 columns,
//               unknown slice), slices reduced by shuffles; FP64 atomics into
//               one of kBkCopies copies of the step's H block column, the
//               tiles taken in a CTA-dependent order so that the CTAs' atomics
//               spread over many L2 lines
//   == grid barrier ==
//   W' = W - Q H (second pass over the ring, H staged once; thread (unknown,
//               4 columns, vector slice), slices summed at the end), Gram
//               G = W'^H W' (FP64 atomics, copies as for H)
//   == grid barrier ==
//   CholQR: G = R^H R and R^{-1} (one warp, every CTA identically),
//               Q_{j+1} = W' R^{-1} -> basis (complex64) and the next matvec
//               operand; CTA 0 writes H and R_{j+1} to host-mapped memory
// The small block least-squares problem (incremental Householder QR of the
// block Hessenberg matrix and the residual estimate per right-hand side)
// runs on the host, a few steps behind the GPU, so it never stalls the step.
// A column that is dependent on the earlier ones (Cholesky pivot <= 1e-10 of
// its own squared norm) or vanishes is reported as a breakdown: the cycle
// ends with the steps before it (at the start block: per-column spaces).
// ---------------------------------------------------------------------------
constexpr int kBkThreads = 512;
constexpr int kBkTileMax = 32;  // basis vectors per ring stage: 32, or 16 when a CTA's unknowns are many
constexpr int kBkMaxP = 16;
constexpr int kBkMaxGroups = 4;                    // 17 .. 64 right-hand sides: groups of <= 16 columns,
constexpr int kBkMaxRhs = kBkMaxP * kBkMaxGroups;  // each its own block space, one shared matvec per step
constexpr int kBkVectors = 384;  // basis vectors per cycle: kBkVectors / m block steps (at most the restart length)
constexpr int kBkCopies = 4;     // copies of the H and Gram sums (CTA c adds into copy c % kBkCopies)
constexpr int kBkHostRing = 4;   // host-mapped H column blocks in flight (the host is at most 2 steps behind)
constexpr int kBkStreamVectors = 1600;  // basis vectors per group and cycle with streamed H
constexpr int kBkMaxStages = 4;

// Block steps per cycle for blocks of p columns and restart length R.
__host__ __device__ inline int bk_steps(int p, int R) {
  const int nb = kBkVectors / p;
  return nb < R ? nb : R;
}

// Device sums and least-squares solution of group g (doubles / double2),
// sized for both step modes: staged H (kBkCopies copies, kBkVectors per
// cycle) and streamed H (one copy, kBkStreamVectors per cycle).
inline void bk_group_sizes(int p, int R, size_t* nh, size_t* ng, size_t* ny) {
  const int nb_staged = std::min(kBkVectors / p, R), nb_stream = std::min(kBkStreamVectors / p, R);
  const size_t hs = std::max((size_t)kBkCopies * (nb_staged + 1), (size_t)(nb_stream + 1));
  *nh = 2 * hs * p * p * 2;
  *ng = 2 * (size_t)kBkCopies * p * p * 2;
  *ny = (size_t)std::max(nb_staged, nb_stream) * p * p;
}

// Groups of m right-hand sides (2 <= m <= kBkMaxRhs): ceil(m / 16) groups,
// sizes as equal as possible (each >= 2).
inline int bk_groups(int m, int* size, int* col0) {
  const int G = (m + kBkMaxP - 1) / kBkMaxP;
  int c = 0;
  for (int g = 0; g < G; g++) {
    size[g] = m / G + (g < m % G ? 1 : 0);
    col0[g] = c;
    c += size[g];
  }
  return G;
}

// Shape of the per-CTA work (host-computed, see bk_geom).
struct BkGeom {
  int hstream; // H streamed per tile (double-buffered [2][tile][pp]) instead of staged whole
  int tile;    // basis vectors per ring stage (16 or 32)
  int pp;      // padded block size: 4, 8 or 16
  int hs;      // unknown slices of the dots (16 / (pp / 4))
  int L;       // unknowns per slice (odd)
  int lw;      // L * hs >= nr: padded unknowns of a W row
  int rs;      // ring row stride in complex64 (>= lw, == hs mod 16, even)
  int as;      // vector slices of the update
  int stages;  // ring stages
};

struct BkPtrs {
  int p;           // block size (the right-hand sides of this group)
  int col0;        // first right-hand side (column) of the group
  int vbase;       // first basis row of the group in P.Vb
  int nb;          // block steps per cycle
  int nr;          // unknowns per CTA (even)
  int ncopy;       // copies of the H and Gram sums (kBkCopies; 1 with streamed H)
  int hstream;     // 1: H read per tile from the (single) sums, 0: the step's H staged whole in shared memory
  BkGeom g;
  double* hacc;    // [2][ncopy][(nb + 1) p][p][re, im]: H column block of the step, by step parity
  double* gacc;    // [2][ncopy][p][p][re, im]: Gram matrix of the step (parity 1 also serves the cycle start)
  double2* Yb;     // [nb p][p]: least-squares solution uploaded by the host
  int* step;       // block step j of the cycle (device)
  double2* hostH;  // host-mapped [kBkHostRing][(nb + 1) p][p]: H column block j (slot j % ring) incl. R_{j+1}
  double2* hostR0; // host-mapped [p][p]: R_0 of the cycle's start block
  int* hostS;      // host-mapped [nb + 1]: 1 step done, 2 breakdown (index nb: the start)
};

__device__ __forceinline__ double* bk_hacc(const BkPtrs& K, int par, int copy) {
  return K.hacc + ((size_t)par * K.ncopy + copy) * (K.nb + 1) * K.p * K.p * 2;
}
__device__ __forceinline__ double* bk_gacc(const BkPtrs& K, int par, int copy) {
  return K.gacc + ((size_t)par * K.ncopy + copy) * K.p * K.p * 2;
}

// Unknown slices of the dots for padded block size pp (the host geometry and
// the kernel's compile-time lane layout both take it from here).
__host__ __device__ constexpr int bk_slices(int pp, int tile) { return kBkThreads / (tile * (pp / 4)); }

__host__ __device__ inline BkGeom bk_geom(int p, int nr, int tile) {
  BkGeom g;
  g.tile = tile;
  g.hstream = 0;
  g.pp = p <= 4 ? 4 : (p <= 8 ? 8 : 16);
  const int cg = g.pp / 4;
  g.hs = bk_slices(g.pp, tile);
  g.L = ((nr + g.hs - 1) / g.hs) | 1;
  g.lw = g.L * g.hs;
  // rows rs apart with rs == hs (mod 16) and odd L: the dots' 8-byte loads
  // (hs slices x 32 / hs vectors per warp) hit every bank pair exactly twice
  const int r = g.hs & 15;
  g.rs = g.lw + ((r - g.lw % 16) + 16) % 16;
  g.as = kBkThreads / (nr * cg);
  if (g.as < 1) g.as = 1;
  if (g.as > 32) g.as = 32;
  g.stages = 0;
  return g;
}

// Dynamic shared memory of gm_block_kernel.
struct BkLayout {
  size_t ring, W, Hs, G, bars, total;
};
__host__ __device__ inline BkLayout bk_layout(int p, int nr, const BkGeom& g, int na_max) {
  BkLayout L;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t r = o;
    o = (o + b + 15) / 16 * 16;
    return r;
  };
  const size_t ring = sizeof(float2) * (size_t)g.stages * g.tile * g.rs;
  const size_t part = sizeof(double2) * (size_t)(g.as - 1) * g.pp * nr;  // update slices, after the ring is drained
  L.ring = take(ring > part ? ring : part);
  L.W = take(sizeof(double2) * (size_t)g.pp * g.lw);
  L.Hs = take(sizeof(double2) * (size_t)(g.hstream ? 2 * g.tile : na_max) * g.pp);
  L.G = take(sizeof(double2) * 2 * (size_t)p * p + sizeof(double) * p);  // G / R^{-1}, R, 1 / R_cc
  L.bars = take(sizeof(uint64_t) * kBkMaxStages);
  L.total = o;
  return L;
}

// Sum of 8 values over HS lanes (xor partners, lane bits below HS): lanes
// first fold whole sets while HS > 8, then exchange halves (transpose-
// reduce); afterwards lane h holds value h & 7 (HS >= 8) or values 2h, 2h + 1
// (HS == 4) in v[0] (and v[1]).
template <int HS>
__device__ __forceinline__ void bk_reduce8(double (&v)[8], int h) {
#pragma unroll
  for (int o = HS / 2; o >= 8; o >>= 1)
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  constexpr int top = HS >= 8 ? 4 : HS / 2;
#pragma unroll
  for (int o = top, half = 4; o >= 1; o >>= 1, half >>= 1) {
    const bool hi = (h & o) != 0;
#pragma unroll
    for (int k = 0; k < half; k++) {
      const double send = hi ? v[k] : v[k + half];
      const double keep = hi ? v[k + half] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
}

// Ring stage s: tile (rot + s) mod T of the basis rows over unknowns
// [i0, i0 + nvc) (nvc even: 16-byte rows), issued by the lanes of warp 0.
__device__ __forceinline__ void bk_issue(const GmPtrs& P, const BkPtrs& K, float2* ring, uint64_t* bars, int s, int T,
                                         int rot, int na_all, int i0, int nvc) {
  const BkGeom& g = K.g;
  const int slot = s % g.stages;
  const int tile = (rot + s) % T;
  const int a0 = tile * g.tile, na = min(g.tile, na_all - a0);
  const int lane = threadIdx.x & 31;
  const uint32_t bytes = (uint32_t)nvc * sizeof(float2);
  if (lane == 0) mbar_expect_tx(&bars[slot], bytes * (uint32_t)na);
  __syncwarp();
  if (lane < na)
    bulk_load(ring + ((size_t)slot * g.tile + lane) * g.rs, P.Vb + (size_t)(K.vbase + a0 + lane) * P.ldv + i0, bytes,
              &bars[slot]);
}

// mode 0: cycle start (W = r_in from P.w, CholQR -> Q_0, R_0); mode 1: step j.
template <int PP, int TILE>
__global__ void __launch_bounds__(kBkThreads, 1) gm_block_kernel(GmPtrs P, BkPtrs K, int mode) {
  constexpr int CG = PP / 4, HS = bk_slices(PP, TILE);
  extern __shared__ __align__(16) unsigned char bk_raw[];
  const int p = K.p, nr = K.nr, n = P.n;
  const BkGeom& g = K.g;
  const int j = mode == 0 ? -1 : *K.step;  // read before any CTA can pass the second barrier
  const int na_all = (j + 1) * p;          // basis vectors 0 .. na_all - 1 exist
  const BkLayout Lo = bk_layout(p, nr, g, K.nb * p);
  float2* ring = reinterpret_cast<float2*>(bk_raw + Lo.ring);  // [stages][TILE][rs]
  double2* W = reinterpret_cast<double2*>(bk_raw + Lo.W);      // [PP][lw]
  double2* Hs = reinterpret_cast<double2*>(bk_raw + Lo.Hs);    // [na_all][PP], or [2][TILE][PP] with streamed H
  double2* G = reinterpret_cast<double2*>(bk_raw + Lo.G);      // [p][p]: G, then R^{-1}
  double2* Rm = G + p * p;                                      // [p][p]: R
  double* rinv = reinterpret_cast<double*>(Rm + p * p);         // [p]: 1 / R_cc
  uint64_t* bars = reinterpret_cast<uint64_t*>(bk_raw + Lo.bars);
  const int tid = threadIdx.x, lane = tid & 31, wq = tid >> 5;
  const int i0 = blockIdx.x * nr;
  const int nvr = max(0, min(nr, n - i0));  // valid unknowns of this CTA
  const int nvc = (nvr + 1) & ~1;           // copied unknowns (the basis rows are zero-padded to even)
  const int par = j & 1;                    // this step's sums (the start uses parity 1)
  const int copy = blockIdx.x % K.ncopy;
  const int T = (na_all + TILE - 1) / TILE;  // basis tiles
  // update units (unknown, 4-column group): if they fit the CTA's threads,
  // register accumulators over all tiles (slices of the vectors share out
  // the spare threads); else every tile updates W in shared memory unit by
  // unit (a unit belongs to one thread within a tile)
  const int nunits = nr * CG;
  const bool inplace = nunits > kBkThreads;
  const int ST = 2 * T;  // ring stages of the step: dots, then the update
  const int rot = T > 0 ? (int)(blockIdx.x % T) : 0;
  int* err = &P.st->err;
  if (g.hs != HS || g.tile != TILE) {  // host geometry built for another lane layout (uniform over the grid)
    if (tid == 0) atomicExch(err, 1);
    return;
  }

  // ---- ring start, W, clear the next step's sums ----
  if (mode == 1) {
    if (tid == 0) {
      for (int s = 0; s < g.stages; s++) mbar_init(&bars[s], 1);
      mbar_init_fence();
    }
    __syncthreads();
    if (wq == 0)
      for (int s = 0; s < min(g.stages, ST); s++) bk_issue(P, K, ring, bars, s, T, rot, na_all, i0, nvc);
    // the unknowns [nvc, lw) of every ring row stay zero (never written by the copies)
    const int padw = g.lw - nvc;
    for (int t = tid; t < g.stages * TILE * padw; t += kBkThreads) {
      const int row = t / padw;
      ring[(size_t)row * g.rs + nvc + (t - row * padw)] = make_float2(0.f, 0.f);
    }
  }
  if (mode == 0) {
    if (P.f16 && blockIdx.x == 0 && tid < p) P.cinv[K.col0 + tid] = 1.f / kF16VecScale;  // operand scale of Q_0, Q_1, ...
    for (int t = tid; t < PP * g.lw; t += kBkThreads) {
      const int b = t / g.lw, i = t - b * g.lw;
      W[t] = (b < p && i < nvr) ? P.w[(size_t)(K.col0 + b) * n + i0 + i] : make_double2(0.0, 0.0);
    }
  } else {
    for (int t = tid; t < PP * g.lw; t += kBkThreads) {
      const int i = t / PP, b = t - i * PP;
      double2 w = make_double2(0.0, 0.0);
      if (i < nvr && b < p) {
        float2* y = P.Y + (size_t)(i0 + i) * P.m + K.col0 + b;
        const float2 yv = *y;
        w = make_double2(yv.x, yv.y);
        *y = make_float2(0.f, 0.f);
      }
      W[b * g.lw + i] = w;
    }
  }
  {
    const int np = par ^ 1;
    const size_t nh = (size_t)(K.nb + 1) * p * p * 2, ng = (size_t)p * p * 2;
    for (size_t t = (size_t)blockIdx.x * kBkThreads + tid; t < (size_t)K.ncopy * (nh + ng);
         t += (size_t)gridDim.x * kBkThreads) {
      const int c = (int)(t / (nh + ng));
      const size_t u = t - (size_t)c * (nh + ng);
      if (u < nh)
        bk_hacc(K, np, c)[u] = 0.0;
      else
        bk_gacc(K, np, c)[u - nh] = 0.0;
    }
  }
  __syncthreads();

  if (mode == 1) {
    double* hacc = bk_hacc(K, par, copy);
    // ---- H = Q^H W: thread (vector, 4 columns, unknown slice) ----
    const int d_cg = wq % CG;
    const int d_al = (wq / CG) * (32 / HS) + lane / HS;
    const int d_hs = lane % HS;
    for (int s = 0; s < T; s++) {
      const int slot = s % g.stages;
      const int a0 = ((rot + s) % T) * TILE, na = min(TILE, na_all - a0);
      mbar_wait(&bars[slot], (uint32_t)(s / g.stages) & 1u, err);
      const float2* q = ring + ((size_t)slot * TILE + d_al) * g.rs + d_hs * g.L;
      const double2* w = W + (size_t)(d_cg * 4) * g.lw + d_hs * g.L;
      double v[8];
#pragma unroll
      for (int k = 0; k < 8; k++) v[k] = 0.0;
      for (int e = 0; e < g.L; e++) {  // conj(q) w
        const float2 qf = q[e];
        const double qx = qf.x, qy = qf.y;
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const double2 wv = w[(size_t)c * g.lw + e];
          v[2 * c] = fma(qx, wv.x, fma(qy, wv.y, v[2 * c]));
          v[2 * c + 1] = fma(qx, wv.y, fma(-qy, wv.x, v[2 * c + 1]));
        }
      }
      bk_reduce8<HS>(v, d_hs);
      if (d_al < na) {
        if constexpr (HS >= 8) {
          const int b = d_cg * 4 + ((d_hs & 7) >> 1);
          if (d_hs < 8 && b < p && v[0] != 0.0) atomicAdd(hacc + ((size_t)(a0 + d_al) * p + b) * 2 + (d_hs & 1), v[0]);
        } else {
          const int b = d_cg * 4 + d_hs;
          if (b < p) {
            double* hp = hacc + ((size_t)(a0 + d_al) * p + b) * 2;
            if (v[0] != 0.0) atomicAdd(hp, v[0]);
            if (v[1] != 0.0) atomicAdd(hp + 1, v[1]);
          }
        }
      }
      __syncthreads();  // stage consumed by every warp
      if (wq == 0 && s + g.stages < ST) bk_issue(P, K, ring, bars, s + g.stages, T, rot, na_all, i0, nvc);
    }
    co_grid_sync(P.st);

    // ---- stage H (sum of the copies), unless it is streamed per tile ----
    for (int t = tid; t < (g.hstream ? 0 : na_all * PP); t += kBkThreads) {
      const int a = t / PP, b = t - a * PP;
      double2 h = make_double2(0.0, 0.0);
      if (b < p) {
#pragma unroll
        for (int c = 0; c < K.ncopy; c++) {
          const double* hp = bk_hacc(K, par, c) + ((size_t)a * p + b) * 2;
          h.x += __ldcg(hp);
          h.y += __ldcg(hp + 1);
        }
      }
      Hs[t] = h;
    }
    __syncthreads();

    // ---- W' = W - Q H ----
    const int uas = inplace ? 1 : g.as;  // vector slices (register mode)
    const int u_as = inplace ? 0 : tid / nunits;
    double2 acc[4];
#pragma unroll
    for (int c = 0; c < 4; c++) acc[c] = make_double2(0.0, 0.0);
    // streamed H: thread t < TILE * PP carries entry (t / PP, t % PP) of the
    // next tile's rows in a register, stored after the current tile
    const double2* Hg = reinterpret_cast<const double2*>(bk_hacc(K, par, 0));  // one copy when streamed
    auto h_fetch = [&](int s2) -> double2 {
      if (!g.hstream || tid >= TILE * PP || s2 >= 2 * T) return make_double2(0.0, 0.0);
      const int a = ((rot + s2) % T) * TILE + tid / PP, b = tid % PP;
      return (a < na_all && b < p) ? __ldcg(Hg + (size_t)a * p + b) : make_double2(0.0, 0.0);
    };
    double2 hnext = h_fetch(T);
    for (int s = T; s < 2 * T; s++) {
      const int slot = s % g.stages;
      const int a0 = ((rot + s) % T) * TILE, na = min(TILE, na_all - a0);
      if (g.hstream) {  // this tile's H rows into buffer s & 1 (its previous readers passed the last barrier)
        if (tid < TILE * PP) Hs[(size_t)(s & 1) * TILE * PP + tid] = hnext;
        hnext = h_fetch(s + 1);
        __syncthreads();
      }
      mbar_wait(&bars[slot], (uint32_t)(s / g.stages) & 1u, err);
      const double2* hbase = g.hstream ? Hs + (size_t)(s & 1) * TILE * PP : Hs + (size_t)a0 * PP;
      for (int unit = inplace ? tid : tid % nunits; unit < (inplace ? nunits : tid % nunits + 1);
           unit += kBkThreads) {
        const int u_cg = unit / nr, u_i = unit - u_cg * nr;
        if (u_as >= uas || u_i >= nvr) continue;
        if (inplace)
#pragma unroll
          for (int c = 0; c < 4; c++) acc[c] = make_double2(0.0, 0.0);
        const float2* q = ring + (size_t)slot * TILE * g.rs + u_i;
        const double2* h = hbase + u_cg * 4;
        for (int al = u_as; al < na; al += uas) {
          const float2 qf = q[(size_t)al * g.rs];
          const double qx = qf.x, qy = qf.y;
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const double2 hv = h[(size_t)al * PP + c];
            acc[c].x = fma(qx, hv.x, fma(-qy, hv.y, acc[c].x));
            acc[c].y = fma(qx, hv.y, fma(qy, hv.x, acc[c].y));
          }
        }
        if (inplace)
#pragma unroll
          for (int c = 0; c < 4; c++) {
            double2* wp = W + (size_t)(u_cg * 4 + c) * g.lw + u_i;
            wp->x -= acc[c].x;
            wp->y -= acc[c].y;
          }
      }
      __syncthreads();
      if (wq == 0 && s + g.stages < ST) bk_issue(P, K, ring, bars, s + g.stages, T, rot, na_all, i0, nvc);
    }
    // every issued stage has been waited for (after an error, a wait may have
    // given up: the last stage issued into each slot is drained before the
    // ring is reused for the slice sums)
    if (tid == 0)
      for (int sl = 0; sl < min(g.stages, ST); sl++) {
        const int s_last = sl + ((ST - 1 - sl) / g.stages) * g.stages;
        mbar_wait_drain(&bars[sl], (uint32_t)(s_last / g.stages) & 1u);
      }
    __syncthreads();
    if (!inplace) {
      const int unit = tid % nunits;
      const int u_cg = unit / nr, u_i = unit - u_cg * nr;
      const bool u_on = u_as < uas && u_i < nvr;
      if (uas > 1) {  // slice sums through the (drained) ring
        double2* part = reinterpret_cast<double2*>(ring);  // [as - 1][CG][nr][4]
        if (u_on && u_as > 0) {
          double2* dst = part + (((size_t)(u_as - 1) * CG + u_cg) * nr + u_i) * 4;
#pragma unroll
          for (int c = 0; c < 4; c++) dst[c] = acc[c];
        }
        __syncthreads();
        if (u_on && u_as == 0)
          for (int a = 1; a < uas; a++) {
            const double2* src = part + (((size_t)(a - 1) * CG + u_cg) * nr + u_i) * 4;
#pragma unroll
            for (int c = 0; c < 4; c++) {
              acc[c].x += src[c].x;
              acc[c].y += src[c].y;
            }
          }
      }
      if (u_on && u_as == 0)
#pragma unroll
        for (int c = 0; c < 4; c++) {
          double2* wp = W + (size_t)(u_cg * 4 + c) * g.lw + u_i;
          wp->x -= acc[c].x;
          wp->y -= acc[c].y;
        }
    }
    __syncthreads();
  }

  // ---- Gram G = W^H W (FP64 atomics): 16 lanes per upper-triangle entry ----
  {
    double* gacc = bk_gacc(K, par, copy);
    const int nent = p * (p + 1) / 2;
    const int nu = (16 * nent + 31) & ~31;  // whole warps: every lane takes part in the shuffles
    for (int u = tid; u < nu; u += kBkThreads) {
      const int e = u >> 4, k = u & 15;  // entry, row slice
      int b1 = 0, b2 = 0;
      double re = 0.0, im = 0.0;
      if (e < nent) {
        int rem = e;
        while (rem >= p - b1) {  // e -> (b1, b2), b2 >= b1
          rem -= p - b1;
          b1++;
        }
        b2 = b1 + rem;
        const double2* w1 = W + (size_t)b1 * g.lw;
        const double2* w2 = W + (size_t)b2 * g.lw;
        for (int i = k; i < nvr; i += 16) {  // conj(w1) w2
          const double2 x = w1[i], y = w2[i];
          re = fma(x.x, y.x, fma(x.y, y.y, re));
          im = fma(x.x, y.y, fma(-x.y, y.x, im));
        }
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
      }
      if (k == 0 && e < nent) {
        const int v = b1 * p + b2;
        if (re != 0.0) atomicAdd(gacc + 2 * v, re);
        if (im != 0.0) atomicAdd(gacc + 2 * v + 1, im);
      }
    }
  }
  co_grid_sync(P.st);

  // ---- CholQR: G = R^H R (R upper triangular), R^{-1}; warp 0, lane b owns column b ----
  __shared__ int s_breakdown;
  if (wq == 0) {
    for (int u = lane; u < p * p; u += 32) {
      const int b1 = u / p, b2 = u - b1 * p;
      const int v = b2 >= b1 ? u : b2 * p + b1;  // lower triangle from the upper one
      double2 gv = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < K.ncopy; c++) {
        const double* gp = bk_gacc(K, par, c) + 2 * v;
        gv.x += __ldcg(gp);
        gv.y += __ldcg(gp + 1);
      }
      if (b2 < b1) gv.y = -gv.y;
      G[u] = gv;
      Rm[u] = make_double2(0.0, 0.0);
    }
    __syncwarp();
    const double gown = lane < p ? G[lane * p + lane].x : 0.0;  // the column's own squared norm
    double dmax = gown;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    int bd = !(dmax > 0.0);
    // right-looking: row c of R from the updated row c of G, then the trailing update
    for (int c = 0; c < p && !bd; c++) {
      const double d = G[c * p + c].x;
      const double gcc = __shfl_sync(0xffffffffu, gown, c);
      // a column dependent on the earlier ones to within 1e-5 in angle (the
      // pivot relative to the column's own norm), or a vanishing column:
      // CholQR would lose orthogonality (its error grows like the square of that ratio)
      if (!(gcc > 1e-30 * dmax) || !(d > 1e-10 * gcc)) {
        bd = 1;
        break;
      }
      const double rc = sqrt(d), ri = 1.0 / rc;
      double2 rcb = make_double2(0.0, 0.0);
      if (lane == c) {
        Rm[c * p + c] = make_double2(rc, 0.0);
        rinv[c] = ri;
      } else if (lane > c && lane < p) {
        const double2 x = G[c * p + lane];
        rcb = make_double2(x.x * ri, x.y * ri);
        Rm[c * p + lane] = rcb;
      }
      __syncwarp();
      if (lane > c && lane < p) {  // G[b1][lane] -= conj(R[c][b1]) R[c][lane], c < b1 <= lane
        for (int b1 = c + 1; b1 <= lane; b1++) {
          const double2 a = Rm[c * p + b1];
          double2* gp = &G[b1 * p + lane];
          gp->x -= a.x * rcb.x + a.y * rcb.y;
          gp->y -= a.x * rcb.y - a.y * rcb.x;
        }
      }
      __syncwarp();
    }
    if (!bd && lane < p) {
      // column b = lane of R^{-1} by back substitution (into G, which is no longer needed)
      const int b = lane;
      for (int c = p - 1; c > b; c--) G[c * p + b] = make_double2(0.0, 0.0);
      for (int c = b; c >= 0; c--) {
        double2 x = make_double2(c == b ? 1.0 : 0.0, 0.0);
        for (int k = c + 1; k <= b; k++) {  // x -= R[c][k] Ri[k][b]
          const double2 r = Rm[c * p + k], y = G[k * p + b];
          x.x -= r.x * y.x - r.y * y.y;
          x.y -= r.x * y.y + r.y * y.x;
        }
        G[c * p + b] = make_double2(x.x * rinv[c], x.y * rinv[c]);
      }
    }
    if (lane == 0) s_breakdown = bd;
  }
  __syncthreads();
  const bool breakdown = s_breakdown != 0;

  // ---- Q_{j+1} = W R^{-1}: thread per (unknown pair, column) ----
  if (!breakdown) {
    const int qa0 = (j + 1) * p;  // first basis vector of the new block
    const int np2 = (nr + 1) / 2;
    for (int u = tid; u < p * np2; u += kBkThreads) {
      const int b = u / np2, il = 2 * (u - b * np2);
      if (il >= nvr) continue;
      const int i = i0 + il;
      double2 q0 = make_double2(0.0, 0.0), q1 = make_double2(0.0, 0.0);
      for (int c = 0; c <= b; c++) {
        const double2 r = G[c * p + b], x0 = W[(size_t)c * g.lw + il], x1 = W[(size_t)c * g.lw + il + 1];
        q0.x += x0.x * r.x - x0.y * r.y;
        q0.y += x0.x * r.y + x0.y * r.x;
        q1.x += x1.x * r.x - x1.y * r.y;
        q1.y += x1.x * r.y + x1.y * r.x;
      }
      const float2 f0 = make_float2((float)q0.x, (float)q0.y);
      const float2 f1 = i + 1 < n ? make_float2((float)q1.x, (float)q1.y) : make_float2(0.f, 0.f);
      *reinterpret_cast<float4*>(P.Vb + (size_t)(K.vbase + qa0 + b) * P.ldv + i) = make_float4(f0.x, f0.y, f1.x, f1.y);
      store_operand(P, i, K.col0 + b, f0, f1);
    }
  }

  // ---- CTA 0: H column block and R to the host, step record ----
  if (blockIdx.x == 0) {
    if (mode == 0) {
      for (int u = tid; u < p * p; u += kBkThreads) K.hostR0[u] = Rm[u];
    } else {
      double2* hj = K.hostH + (size_t)(j % kBkHostRing) * (K.nb + 1) * p * p;
      const double2* Hg = reinterpret_cast<const double2*>(bk_hacc(K, par, 0));
      for (int u = tid; u < (na_all + p) * p; u += kBkThreads) {
        const int a = u / p;
        hj[u] = a < na_all ? (g.hstream ? __ldcg(Hg + u) : Hs[(size_t)a * PP + (u - a * p)]) : Rm[u - na_all * p];
      }
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence_system();
      reinterpret_cast<volatile int*>(K.hostS)[mode == 0 ? K.nb : j] = breakdown ? 2 : 1;
      *K.step = j + 1;
    }
  }
}

// D(:, s) += sum_{a < na} Q_a Y[a][s] for the block solution of the cycle.
// Thread = unknown i, all PP (>= p) columns of the group, so every basis
// element is read once; blockIdx.y takes one of gridDim.y slices of the basis
// vectors (the slices meet in D by FP64 atomics); Y staged in shared memory
// chunk by chunk, the basis loads unrolled so that several are in flight.
constexpr int kXuThreads = 128;
constexpr int kXuChunk = 64;  // basis vectors per shared-memory chunk of Y
template <int PP>
__global__ void __launch_bounds__(kXuThreads) gm_block_xupdate_kernel(GmPtrs P, BkPtrs K, int na) {
  __shared__ double2 ys[kXuChunk][PP];
  const int i = blockIdx.x * kXuThreads + threadIdx.x;
  const int p = K.p;
  const int per = (na + gridDim.y - 1) / gridDim.y;
  const int a_begin = blockIdx.y * per, a_end = min(na, a_begin + per);
  double2 acc[PP];
#pragma unroll
  for (int c = 0; c < PP; c++) acc[c] = make_double2(0.0, 0.0);
  for (int a0 = a_begin; a0 < a_end; a0 += kXuChunk) {
    const int nc = min(kXuChunk, a_end - a0);
    __syncthreads();  // the previous chunk's readers are done
    for (int e = threadIdx.x; e < kXuChunk * PP; e += kXuThreads) {
      const int a = e / PP, c = e - a * PP;
      ys[a][c] = (a < nc && c < p) ? K.Yb[(size_t)(a0 + a) * p + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (i < P.n) {
      const float2* q = P.Vb + (size_t)(K.vbase + a0) * P.ldv + i;
#pragma unroll 8
      for (int a = 0; a < nc; a++) {
        const float2 v = q[(size_t)a * P.ldv];
        const double vx = v.x, vy = v.y;
#pragma unroll
        for (int c = 0; c < PP; c++) {
          const double2 y = ys[a][c];
          acc[c].x = fma(vx, y.x, fma(-vy, y.y, acc[c].x));
          acc[c].y = fma(vx, y.y, fma(vy, y.x, acc[c].y));
        }
      }
    }
  }
  if (i < P.n && a_begin < a_end) {
#pragma unroll
    for (int c = 0; c < PP; c++)
      if (c < p) {
        double* d = reinterpret_cast<double*>(P.d + (size_t)(K.col0 + c) * P.n + i);
        atomicAdd(d, acc[c].x);
        atomicAdd(d + 1, acc[c].y);
      }
  }
}

// D(:, col0 + c) += sum_{a < na} Q_a Y[a][c] for the p columns of group K.
int launch_block_xupdate(const GmPtrs& P, const BkPtrs& K, int na, cudaStream_t s) {
  if (na <= 0) return BEM_OK;
  const int bx = (P.n + kXuThreads - 1) / kXuThreads;
  int by = (2 * device_sms() + bx - 1) / bx;  // about two CTAs per SM in all
  by = std::max(1, std::min(by, (na + kXuChunk - 1) / kXuChunk));
  const dim3 grid(bx, by);
  if (K.p <= 4)
    (gm_block_xupdate_kernel<4><<<grid, kXuThreads, 0, s>>>(P, K, na), count_launch());
  else if (K.p <= 8)
    (gm_block_xupdate_kernel<8><<<grid, kXuThreads, 0, s>>>(P, K, na), count_launch());
  else
    (gm_block_xupdate_kernel<16><<<grid, kXuThreads, 0, s>>>(P, K, na), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
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
  const float2* v = P.Vb + (size_t)s * (P.R + 1) * P.ldv + i;
  for (int l = 0; l < kk; l++) {
    const float2 vv = v[(size_t)l * P.ldv];
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
    P.active[s] = beta > target && beta > 0.0;
    P.kcol[s] = 0;
    P.norm2[s] = 0.0;
  }
}

// V[s][0] = w_s / beta_s and the first matvec operand; two unknowns per thread
constexpr int kPairThreads = 256;
__global__ void __launch_bounds__(kPairThreads) gm_start_norm_kernel(GmPtrs P) {
  const int i = blockIdx.x * 2 * kPairThreads + 2 * threadIdx.x;
  const int s = blockIdx.y;
  if (P.f16 && blockIdx.x == 0 && threadIdx.x == 0) P.cinv[s] = 1.f / kF16VecScale;
  if (i >= P.n) return;
  const double b = P.beta[s];
  const double inv = b > 0.0 ? 1.0 / b : 0.0;
  const double2 w0 = P.w[(size_t)s * P.n + i];
  const double2 w1 = i + 1 < P.n ? P.w[(size_t)s * P.n + i + 1] : make_double2(0.0, 0.0);
  const float2 f0 = make_float2((float)(w0.x * inv), (float)(w0.y * inv));
  const float2 f1 = make_float2((float)(w1.x * inv), (float)(w1.y * inv));
  *reinterpret_cast<float4*>(P.Vb + (size_t)s * (P.R + 1) * P.ldv + i) = make_float4(f0.x, f0.y, f1.x, f1.y);
  store_operand(P, i, s, f0, f1);
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
  size_t Vb, H, cs, sn, g, w, d, x, r, X, Y, norm2, rnorm2, beta, tol, resid, active, kend, kcol, colstep, y, st,
      bnorm2, hacc, nacc, bk_hacc, bk_gacc, bk_y, bk_step, tc, total;
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
  L.Vb = take(sizeof(float2) * (size_t)m * (R + 1) * (size_t)((n + 1) & ~1));
  L.H = take(sizeof(double2) * (size_t)m * R * (R + 1));
  L.cs = take(sizeof(double) * (size_t)m * R);
  L.sn = take(sizeof(double2) * (size_t)m * R);
  L.g = take(sizeof(double2) * (size_t)m * (R + 1));
  L.w = take(sizeof(double2) * (size_t)m * n);
  L.d = take(sizeof(double2) * (size_t)m * n);
  L.x = take(sizeof(double2) * (size_t)m * n);
  L.r = take(sizeof(double2) * (size_t)m * n);
  L.X = take(sizeof(float2) * (size_t)m * n);
  L.Y = take(sizeof(float2) * (size_t)m * n);
  L.norm2 = take(sizeof(double) * m);
  L.rnorm2 = take(sizeof(double) * m);
  L.beta = take(sizeof(double) * m);
  L.tol = take(sizeof(double) * m);
  L.resid = take(sizeof(double) * m);
  L.active = take(sizeof(int) * m);
  L.kend = take(sizeof(int) * m);
  L.kcol = take(sizeof(int) * m);
  L.colstep = take(sizeof(int) * m);
  L.y = take(sizeof(double2) * (size_t)m * R);
  L.bnorm2 = take(sizeof(double) * m);
  L.hacc = take(sizeof(double) * 2 * (size_t)m * 4 * (R + 1));
  L.nacc = take(sizeof(double) * 2 * (size_t)m * 3);
  // block solver state (used when 2 <= m <= kBkMaxP)
  const bool bk = m >= 2 && m <= kBkMaxRhs;
  size_t sh = 0, sg = 0, sy = 0;
  if (bk) {
    int gsz[kBkMaxGroups], gc0[kBkMaxGroups];
    const int G = bk_groups(m, gsz, gc0);
    for (int g = 0; g < G; g++) {
      size_t a, b, c;
      bk_group_sizes(gsz[g], R, &a, &b, &c);
      sh += a;
      sg += b;
      sy += c;
    }
  }
  L.bk_hacc = take(sizeof(double) * sh);
  L.bk_gacc = take(sizeof(double) * sg);
  L.bk_y = take(sizeof(double2) * sy);
  L.bk_step = take(bk ? sizeof(int) * kBkMaxGroups : 0);
  L.tc = take(precision == BEM_PREC_FP32 ? 0 : tc_workspace_bytes(n, m, precision));
  L.total = o;
  return L;
}

bool params_ok(const bem_solver_params* p) {
  return p && p->restart >= 1 && p->restart < kMaxRestart && p->max_iters >= 1 && p->max_refine >= 1 && p->rtol >= 0.0 &&
         (p->precision == BEM_PREC_FP32 || p->precision == BEM_PREC_BF16X3 || p->precision == BEM_PREC_BF16 ||
          p->precision == BEM_PREC_FP16X3);
}

// Per-step column activity in host-mapped pinned memory (kSnapRing slots of
// m ints, written by the Arnoldi kernel) and one event per slot.  The host
// runs at most kLookahead steps ahead of the GPU: before enqueueing step
// j + kLookahead + 1 it waits for the event of step j and reads its slot, and
// it stops enqueueing once a slot shows every column converged, so at most
// kLookahead no-op steps follow convergence.  No copy is enqueued per step.
constexpr int kLookahead = 4;
static_assert(kLookahead < kSnapRing, "a slot is read before it is reused");
struct HostRing {
  int* snap = nullptr;  // [kSnapRing][cap] host view
  int* dsnap = nullptr;  // device view
  int cap = 0;
  cudaEvent_t ev[kSnapRing] = {};
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

// Host-mapped buffers of the block solver (H column blocks, R_0, step
// status), one set per host thread, grown on demand.
struct BlockHost {
  double2* H = nullptr;  // host view [kBkHostRing][(nb + 1) p][p]
  double2* dH = nullptr;  // device view
  double2* R0 = nullptr;
  double2* dR0 = nullptr;
  int* S = nullptr;
  int* dS = nullptr;
  size_t cap = 0;  // H entries the buffers hold
  ~BlockHost() {
    if (H) cudaFreeHost(H);
    if (R0) cudaFreeHost(R0);
    if (S) cudaFreeHost(S);
  }
};
thread_local BlockHost t_blocks[kBkMaxGroups];

int block_host(int group, int p, int nb, BlockHost** out) {
  BlockHost& t_block = t_blocks[group];
  // H column blocks of the steps in flight (slot j % kBkHostRing), and the step records
  const size_t need = std::max((size_t)kBkHostRing * (nb + 1) * p * p, (size_t)nb + 1);
  if (t_block.cap < need) {
    if (t_block.H) cudaFreeHost(t_block.H);
    if (t_block.R0) cudaFreeHost(t_block.R0);
    if (t_block.S) cudaFreeHost(t_block.S);
    t_block.H = t_block.R0 = nullptr;
    t_block.S = nullptr;
    t_block.cap = 0;
    BEM_CUDA_TRY(cudaHostAlloc((void**)&t_block.H, sizeof(double2) * need, cudaHostAllocMapped));
    BEM_CUDA_TRY(cudaHostAlloc((void**)&t_block.R0, sizeof(double2) * kBkMaxP * kBkMaxP, cudaHostAllocMapped));
    BEM_CUDA_TRY(cudaHostAlloc((void**)&t_block.S, sizeof(int) * need, cudaHostAllocMapped));
    BEM_CUDA_TRY(cudaHostGetDevicePointer((void**)&t_block.dH, t_block.H, 0));
    BEM_CUDA_TRY(cudaHostGetDevicePointer((void**)&t_block.dR0, t_block.R0, 0));
    BEM_CUDA_TRY(cudaHostGetDevicePointer((void**)&t_block.dS, t_block.S, 0));
    t_block.cap = need;
  }
  *out = &t_block;
  return BEM_OK;
}

// Reflection of rows r .. r + p of the columns [t0, t1) of a row-major
// [row][p] (re, im) pair of arrays: y -= f u (u^H y).  The loops run over the
// columns, contiguous in memory, so that they vectorise; the body is stamped
// twice, for x86-64 CPUs with AVX2 and FMA and for any other.
#define BK_REFLECT_BODY                                         \
  double dr[kBkMaxP], di[kBkMaxP];                              \
  for (int t = t0; t < t1; t++) dr[t] = di[t] = 0.0;            \
  for (int e = 0; e <= p; e++) {                                \
    const double a = ur[e], b = ui[e];                          \
    const double* xr = yr + (size_t)e * p;                      \
    const double* xi = yi + (size_t)e * p;                      \
    _Pragma("GCC ivdep") for (int t = t0; t < t1; t++) {        \
      dr[t] += a * xr[t] + b * xi[t];                           \
      di[t] += a * xi[t] - b * xr[t];                           \
    }                                                           \
  }                                                             \
  for (int t = t0; t < t1; t++) {                               \
    dr[t] *= f;                                                 \
    di[t] *= f;                                                 \
  }                                                             \
  for (int e = 0; e <= p; e++) {                                \
    const double a = ur[e], b = ui[e];                          \
    double* xr = yr + (size_t)e * p;                            \
    double* xi = yi + (size_t)e * p;                            \
    _Pragma("GCC ivdep") for (int t = t0; t < t1; t++) {        \
      xr[t] -= a * dr[t] - b * di[t];                           \
      xi[t] -= a * di[t] + b * dr[t];                           \
    }                                                           \
  }

__attribute__((target("avx2,fma"))) void bk_reflect_avx2(const double* __restrict ur, const double* __restrict ui,
                                                          double f, int p, int t0, int t1, double* __restrict yr,
                                                          double* __restrict yi) {
  BK_REFLECT_BODY
}
void bk_reflect_generic(const double* __restrict ur, const double* __restrict ui, double f, int p, int t0, int t1,
                        double* __restrict yr, double* __restrict yi) {
  BK_REFLECT_BODY
}
#undef BK_REFLECT_BODY
typedef void (*BkReflectFn)(const double*, const double*, double, int, int, int, double*, double*);
BkReflectFn bk_reflect() {
  static const BkReflectFn fn =
      (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) ? bk_reflect_avx2 : bk_reflect_generic;
  return fn;
}

// The block least-squares problem min || E1 R_0 - H_k Y || of block GMRES,
// solved incrementally on the host: Householder reflections triangularise
// the block Hessenberg matrix one block column at a time (column c has
// nonzeros down to row c + p, so each reflection acts on p + 1 rows) and are
// applied to the right-hand side Z = E1 R_0; the residual of right-hand side
// b is the norm of Z's rows (k+1)p .. (k+2)p-1 below the triangle.
// Each new block column is reflected by every earlier reflection across all
// its p columns at once (row-major [row][column] working copy, vectorised).
struct BlockLS {
  int p = 0, ld = 0, ncols = 0;
  std::vector<double> Tre, Tim;  // triangular factor, column-major: [column][row], ld rows
  std::vector<double> Zre, Zim;  // rotated right-hand side, row-major: [row][p]
  std::vector<double> Ure, Uim;  // reflections, p + 1 entries each
  std::vector<double> fac;       // 2 / (u^H u) of each reflection (0: identity)
  std::vector<double> Xre, Xim;  // the new block column, row-major: [row][p]
  BkReflectFn refl = nullptr;
  void init(int p_, int nb, const double2* R0) {
    p = p_;
    ld = (nb + 1) * p;
    ncols = 0;
    refl = bk_reflect();
    Tre.assign((size_t)ld * nb * p, 0.0);
    Tim.assign((size_t)ld * nb * p, 0.0);
    Zre.assign((size_t)ld * p, 0.0);
    Zim.assign((size_t)ld * p, 0.0);
    Ure.assign((size_t)nb * p * (p + 1), 0.0);
    Uim.assign((size_t)nb * p * (p + 1), 0.0);
    fac.assign((size_t)nb * p, 0.0);
    Xre.assign((size_t)ld * p, 0.0);
    Xim.assign((size_t)ld * p, 0.0);
    for (int c = 0; c < p; c++)
      for (int b = 0; b < p; b++) {
        Zre[(size_t)c * p + b] = R0[c * p + b].x;
        Zim[(size_t)c * p + b] = R0[c * p + b].y;
      }
  }
  // block column j: hj[a][b], rows a < (j + 2) p; residual estimate per right-hand side.
  // Returns false if the triangular factor is singular (a lost direction).
  bool add(int j, const double2* hj, double* resid) {
    const int c0 = j * p, nrow = (j + 2) * p;
    for (int a = 0; a < nrow; a++)
      for (int t = 0; t < p; t++) {
        Xre[(size_t)a * p + t] = hj[a * p + t].x;
        Xim[(size_t)a * p + t] = hj[a * p + t].y;
      }
    // the reflections of the earlier block columns, each to all p new columns
    for (int r = 0; r < c0; r++)
      if (fac[r] != 0.0)
        refl(&Ure[(size_t)r * (p + 1)], &Uim[(size_t)r * (p + 1)], fac[r], p, 0, p, &Xre[(size_t)r * p],
             &Xim[(size_t)r * p]);
    for (int t = 0; t < p; t++) {
      const int cc = c0 + t;  // reflection for rows cc .. cc + p of column cc
      double nrm2 = 0.0;
      for (int e = 0; e <= p; e++) {
        const double xr = Xre[(size_t)(cc + e) * p + t], xi = Xim[(size_t)(cc + e) * p + t];
        nrm2 += xr * xr + xi * xi;
      }
      const double nrm = std::sqrt(nrm2);
      if (!(nrm > 0.0)) return false;
      const double ax = Xre[(size_t)cc * p + t], ay = Xim[(size_t)cc * p + t];
      const double aa = std::sqrt(ax * ax + ay * ay);
      const double phx = aa > 0.0 ? ax / aa : 1.0, phy = aa > 0.0 ? ay / aa : 0.0;
      double* ur = &Ure[(size_t)cc * (p + 1)];
      double* ui = &Uim[(size_t)cc * (p + 1)];
      for (int e = 0; e <= p; e++) {
        ur[e] = Xre[(size_t)(cc + e) * p + t];
        ui[e] = Xim[(size_t)(cc + e) * p + t];
      }
      ur[0] += phx * nrm;
      ui[0] += phy * nrm;
      double uu = 0.0;
      for (int e = 0; e <= p; e++) uu += ur[e] * ur[e] + ui[e] * ui[e];
      fac[cc] = uu > 0.0 ? 2.0 / uu : 0.0;
      Xre[(size_t)cc * p + t] = -phx * nrm;
      Xim[(size_t)cc * p + t] = -phy * nrm;
      for (int e = 1; e <= p; e++) {
        Xre[(size_t)(cc + e) * p + t] = 0.0;
        Xim[(size_t)(cc + e) * p + t] = 0.0;
      }
      if (fac[cc] != 0.0) {  // the block's later columns and Z
        if (t + 1 < p) refl(ur, ui, fac[cc], p, t + 1, p, &Xre[(size_t)cc * p], &Xim[(size_t)cc * p]);
        refl(ur, ui, fac[cc], p, 0, p, &Zre[(size_t)cc * p], &Zim[(size_t)cc * p]);
      }
    }
    for (int t = 0; t < p; t++)
      for (int a = 0; a < nrow; a++) {
        Tre[(size_t)(c0 + t) * ld + a] = Xre[(size_t)a * p + t];
        Tim[(size_t)(c0 + t) * ld + a] = Xim[(size_t)a * p + t];
      }
    ncols = c0 + p;
    for (int b = 0; b < p; b++) {
      double r2 = 0.0;
      for (int a = (j + 1) * p; a < (j + 2) * p; a++) {
        const double zr = Zre[(size_t)a * p + b], zi = Zim[(size_t)a * p + b];
        r2 += zr * zr + zi * zi;
      }
      resid[b] = std::sqrt(r2);
    }
    return true;
  }
  // Y (kk p x p, row a col b -> Y[a p + b]) solving T[0:kk p, 0:kk p] Y = Z[0:kk p, :]
  void solve(int kk, std::vector<double2>& Y) const {
    const int nc = kk * p;
    Y.assign((size_t)nc * p, make_double2(0.0, 0.0));
    std::vector<double> yr(nc), yi(nc);
    for (int b = 0; b < p; b++) {
      for (int a = 0; a < nc; a++) {
        yr[a] = Zre[(size_t)a * p + b];
        yi[a] = Zim[(size_t)a * p + b];
      }
      for (int c = nc - 1; c >= 0; c--) {
        const double dx = Tre[(size_t)c * ld + c], dy = Tim[(size_t)c * ld + c];
        const double dd = dx * dx + dy * dy;
        const double vx = (yr[c] * dx + yi[c] * dy) / dd, vy = (yi[c] * dx - yr[c] * dy) / dd;
        yr[c] = vx;
        yi[c] = vy;
        const double* cr = &Tre[(size_t)c * ld];
        const double* ci = &Tim[(size_t)c * ld];
        for (int a = 0; a < c; a++) {
          yr[a] -= cr[a] * vx - ci[a] * vy;
          yi[a] -= cr[a] * vy + ci[a] * vx;
        }
      }
      for (int a = 0; a < nc; a++) Y[(size_t)a * p + b] = make_double2(yr[a], yi[a]);
    }
  }
};

int host_ring(int m, HostRing** r) {
  if (!t_ring.ev[0])
    for (auto& e : t_ring.ev) BEM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (t_ring.cap < m) {
    if (t_ring.snap) cudaFreeHost(t_ring.snap);
    t_ring.snap = nullptr;
    t_ring.cap = 0;
    BEM_CUDA_TRY(cudaHostAlloc((void**)&t_ring.snap, sizeof(int) * kSnapRing * (size_t)m, cudaHostAllocMapped));
    BEM_CUDA_TRY(cudaHostGetDevicePointer((void**)&t_ring.dsnap, t_ring.snap, 0));
    t_ring.cap = m;
  }
  *r = &t_ring;
  return BEM_OK;
}

// Launch shape of gm_arnoldi_kernel for n unknowns and m columns.  One
// cluster (<= 16 CTAs, any size) per column; each CTA holds `units` unknowns.
// The step streams the basis once per pass through every CTA, so more CTAs
// per column means fewer bytes per SM, but a cluster must fit in one GPC and
// not every size lets all m clusters be resident at once: the shape
// minimises waves x (units + a fixed-cost allowance), with the number of
// co-resident clusters from cudaOccupancyMaxActiveClusters.
struct ArnShape {
  int cluster = 1;
  int units = 0;
  int chunk = 0;
  size_t smem = 0;
};

int sm_count_linalg() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

int arnoldi_shape(int n, int m, ArnShape* out) {
  static std::atomic<bool> attr{false};
  int dev = 0, smem_optin = 0;
  BEM_CUDA_TRY(cudaGetDevice(&dev));
  BEM_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(gm_arnoldi_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    BEM_CUDA_TRY(cudaFuncSetAttribute(gm_arnoldi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin));
    attr.store(true, std::memory_order_release);
  }
  const int max_cl = g_arn_max_cluster > 0 && g_arn_max_cluster < kArnMaxCluster ? g_arn_max_cluster : kArnMaxCluster;
  int cl = 1;
  while (cl < max_cl && (long long)cl * 2 * kArnThreads < n) cl++;
  long long best_cost = -1;
  for (; cl >= 1; cl--) {
    const int units = (((n + cl - 1) / cl) + 1) & ~1;
    int chunk = kChunkMax;
    while (chunk > 1 && arn_smem_bytes(units, chunk) > (size_t)smem_optin) chunk--;
    const size_t smem = arn_smem_bytes(units, chunk);
    if (smem > (size_t)smem_optin) break;  // smaller clusters need even more
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cl, 1, 1);
    cfg.blockDim = dim3(kArnThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, gm_arnoldi_kernel, &cfg) != cudaSuccess || nclusters <= 0) {
      cudaGetLastError();
      continue;
    }
    const long long waves = (m + nclusters - 1) / nclusters;
    const long long cost = waves * ((long long)units + 512);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      out->cluster = cl;
      out->units = units;
      out->chunk = chunk;
      out->smem = smem;
    }
  }
  return best_cost < 0 ? BEM_ERR_UNSUPPORTED : BEM_OK;
}

// Launch shape of gm_arnoldi_coop_kernel: npc unknown pairs per CTA (at
// least 16, enough CTAs to cover every SM once), one CTA per SM at most, all
// resident (cooperative launch); every column's rotations owned by one CTA.
struct CoShape {
  int npc = 0, grid = 0, cpc = 0, slots = 0;
  size_t smem = 0;
};

int coop_shape(int n, int m, int R, CoShape* out) {
  static std::atomic<bool> attr{false};
  int dev = 0, coop_ok = 0, smem_optin = 0;
  BEM_CUDA_TRY(cudaGetDevice(&dev));
  BEM_CUDA_TRY(cudaDeviceGetAttribute(&coop_ok, cudaDevAttrCooperativeLaunch, dev));
  BEM_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (!coop_ok) return BEM_ERR_UNSUPPORTED;
  const int sms = sm_count_linalg();
  const int npairs = (n + 1) / 2;
  int npc = std::max(16, (npairs + sms - 1) / sms);
  const int grid = (npairs + npc - 1) / npc;
  const int cpc = (m + grid - 1) / grid;  // columns whose rotations one CTA applies
  if (cpc > kCoMaxColsPerCta) return BEM_ERR_UNSUPPORTED;
  // ring slots per warp: 4, fewer when shared memory is short (half the
  // opt-in maximum, leaving room for a concurrent solve's kernels)
  int slots = 4;
  while (slots > 2 && co_layout(m, npc, R, cpc, slots).total > (size_t)smem_optin / 2) slots--;
  const size_t smem = co_layout(m, npc, R, cpc, slots).total;
  if (smem > (size_t)smem_optin / 2) return BEM_ERR_UNSUPPORTED;
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(gm_arnoldi_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem_optin / 2));
    attr.store(true, std::memory_order_release);
  }
  int occ = 0;
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, gm_arnoldi_coop_kernel, kCoThreads, smem));
  if (occ < 1 || grid > occ * sms) return BEM_ERR_UNSUPPORTED;
  out->npc = npc;
  out->grid = grid;
  out->cpc = cpc;
  out->slots = slots;
  out->smem = smem;
  return BEM_OK;
}

// Launch shape of gm_block_kernel: nr unknowns per CTA (even), one CTA per
// SM at most, all resident (cooperative launch).  Preference, first fit in
// shared memory: the full cycle length, 32-vector ring stages, more stages;
// with many unknowns per CTA the stages shrink to 16 vectors and then the
// cycle shortens.  One geometry per group (the groups differ in p by <= 1).
struct BkShape {
  int nr = 0, grid = 0, nb = 0, groups = 0;
  int p[kBkMaxGroups] = {}, col0[kBkMaxGroups] = {}, vbase[kBkMaxGroups] = {};
  BkGeom g[kBkMaxGroups] = {};
  size_t smem[kBkMaxGroups] = {};
};

template <typename F>
int block_dispatch(int pp, int tile, F&& f) {
  if (tile == 32) {
    if (pp == 4) return f(gm_block_kernel<4, 32>);
    if (pp == 8) return f(gm_block_kernel<8, 32>);
    return f(gm_block_kernel<16, 32>);
  }
  if (pp == 4) return f(gm_block_kernel<4, 16>);
  if (pp == 8) return f(gm_block_kernel<8, 16>);
  return f(gm_block_kernel<16, 16>);
}

int block_shape(int n, int m, int R, BkShape* out) {
  static std::mutex mu;
  static bool attr_set[2][3] = {};
  int dev = 0, coop_ok = 0, smem_optin = 0;
  BEM_CUDA_TRY(cudaGetDevice(&dev));
  BEM_CUDA_TRY(cudaDeviceGetAttribute(&coop_ok, cudaDevAttrCooperativeLaunch, dev));
  BEM_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (!coop_ok || m < 2 || m > kBkMaxRhs) return BEM_ERR_UNSUPPORTED;
  const int sms = sm_count_linalg();
  int nr = (n + sms - 1) / sms;
  nr = std::max(16, (nr + 1) & ~1);
  if (nr > 320) return BEM_ERR_UNSUPPORTED;
  const int grid = (n + nr - 1) / nr;
  BkShape sh;
  sh.groups = bk_groups(m, sh.p, sh.col0);
  // staged H at the full cycle length; else H streamed per tile (one copy of
  // its sums, the cycle up to kBkStreamVectors basis vectors per group)
  bool fit = false;
  for (int hstream = 0; hstream <= 1 && !fit; hstream++) {
    const int nb = hstream ? std::min(kBkStreamVectors / sh.p[0], R) : bk_steps(sh.p[0], R);
    for (int tile = kBkTileMax; tile >= 16 && !fit; tile /= 2) {
      for (int stages = kBkMaxStages; stages >= 2 && !fit; stages--) {
        bool ok = true;
        for (int g = 0; g < sh.groups && ok; g++) {
          sh.g[g] = bk_geom(sh.p[g], nr, tile);
          sh.g[g].stages = stages;
          sh.g[g].hstream = hstream;
          sh.smem[g] = bk_layout(sh.p[g], nr, sh.g[g], nb * sh.p[g]).total;
          ok = sh.smem[g] + 1024 <= (size_t)smem_optin;
        }
        if (ok) {
          fit = true;
          sh.nb = nb;
        }
      }
    }
  }
  if (!fit) return BEM_ERR_UNSUPPORTED;
  for (int g = 0, row = 0; g < sh.groups; g++) {
    sh.vbase[g] = row;
    row += (sh.nb + 1) * sh.p[g];
    const int pi = sh.g[g].pp == 4 ? 0 : sh.g[g].pp == 8 ? 1 : 2, ti = sh.g[g].tile == 32 ? 0 : 1;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (!attr_set[ti][pi]) {
        int rc = block_dispatch(sh.g[g].pp, sh.g[g].tile, [&](auto kern) -> int {
          BEM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin - 1024));
          return BEM_OK;
        });
        if (rc) return rc;
        attr_set[ti][pi] = true;
      }
    }
    int occ = 0;
    int rc = block_dispatch(sh.g[g].pp, sh.g[g].tile, [&](auto kern) -> int {
      BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kBkThreads, sh.smem[g]));
      return BEM_OK;
    });
    if (rc) return rc;
    if (occ < 1 || grid > occ * sms) return BEM_ERR_UNSUPPORTED;
  }
  sh.nr = nr;
  sh.grid = grid;
  *out = sh;
  return BEM_OK;
}

int launch_block(const GmPtrs& P, const BkPtrs& K, const BkShape& sh, int group, int mode, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)sh.grid, 1, 1);
  cfg.blockDim = dim3(kBkThreads, 1, 1);
  cfg.dynamicSmemBytes = sh.smem[group];
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int rc = block_dispatch(sh.g[group].pp, sh.g[group].tile, [&](auto kern) -> int {
    BEM_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, P, K, mode));
    return BEM_OK;
  });
  if (rc) return rc;
  count_launch();
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

}  // namespace

int cmatmul(const float2* A, int n, const float2* X, int m, float2* Y, cudaStream_t s) {
  BEM_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(float2) * (size_t)n * m, s));
  return launch_cgemv(A, n, X, m, Y, nullptr, s);
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
  P.w = (double2*)(w + L.w);
  P.d = (double2*)(w + L.d);
  P.x = (double2*)(w + L.x);
  P.r = (double2*)(w + L.r);
  P.X = (float2*)(w + L.X);
  P.Y = (float2*)(w + L.Y);
  P.norm2 = (double*)(w + L.norm2);
  P.ldv = (n + 1) & ~1;
  P.bh = nullptr;
  P.bl = nullptr;
  P.ldb = 0;
  P.cinv = nullptr;
  P.f16 = 0;
  P.beta = (double*)(w + L.beta);
  P.tol = (double*)(w + L.tol);
  P.resid = (double*)(w + L.resid);
  P.active = (int*)(w + L.active);
  P.kend = (int*)(w + L.kend);
  P.kcol = (int*)(w + L.kcol);
  P.colstep = (int*)(w + L.colstep);
  P.y = (double*)(w + L.y);
  P.st = (GmState*)(w + L.st);
  P.bnorm2 = (double*)(w + L.bnorm2);
  P.hacc = (double*)(w + L.hacc);
  P.nacc = (double*)(w + L.nacc);
  double* rnorm2 = (double*)(w + L.rnorm2);
  void* tcws = w + L.tc;
  const int prec = params->precision;
  // block Krylov spaces (see gm_block_kernel): one for 2..16 right-hand
  // sides, groups of <= 16 columns for up to 64, one shared matvec per step
  BkPtrs K[kBkMaxGroups] = {};
  BkShape bshape;
  BlockHost* bh[kBkMaxGroups] = {};
  bool block = g_gmres_block == 0 && m >= 2 && m <= kBkMaxRhs && block_shape(n, m, R, &bshape) == BEM_OK;
  const int nbk = bshape.nb, ngr = block ? bshape.groups : 0;
  {
    size_t oh = 0, og = 0, oy = 0;
    for (int g = 0; g < ngr; g++) {
      const int pg = bshape.p[g];
      int rcb = block_host(g, pg, nbk, &bh[g]);
      if (rcb) return rcb;
      K[g].p = pg;
      K[g].col0 = bshape.col0[g];
      K[g].vbase = bshape.vbase[g];
      K[g].nb = nbk;
      K[g].nr = bshape.nr;
      K[g].g = bshape.g[g];
      K[g].hstream = bshape.g[g].hstream;
      K[g].ncopy = K[g].hstream ? 1 : kBkCopies;
      K[g].hacc = (double*)(w + L.bk_hacc) + oh;
      K[g].gacc = (double*)(w + L.bk_gacc) + og;
      K[g].Yb = (double2*)(w + L.bk_y) + oy;
      K[g].step = (int*)(w + L.bk_step) + g;
      K[g].hostH = bh[g]->dH;
      K[g].hostR0 = bh[g]->dR0;
      K[g].hostS = bh[g]->dS;
      size_t a, b, c;
      bk_group_sizes(pg, R, &a, &b, &c);
      oh += a;
      og += b;
      oy += c;
    }
  }
  if (prec != BEM_PREC_FP32) {
    int rc = tc_operator_prepare((const float2*)A, n, prec, tcws, s);
    if (rc) return rc;
    int nb = 0;
    if ((rc = tc_b_planes(tcws, n, m, prec, &P.bh, &P.bl, &P.ldb, &nb, &P.cinv))) return rc;
    P.f16 = prec == BEM_PREC_FP16X3;
    // rows 2m..nb-1 of the B planes stay zero; the step kernels write rows < 2m
    BEM_CUDA_TRY(cudaMemsetAsync(P.bh, 0, sizeof(__nv_bfloat16) * (size_t)nb * P.ldb, s));
    BEM_CUDA_TRY(cudaMemsetAsync(P.bl, 0, sizeof(__nv_bfloat16) * (size_t)nb * P.ldb, s));
  } else {
    BEM_CUDA_TRY(cudaMemsetAsync(P.X, 0, sizeof(float2) * (size_t)n * m, s));
  }
  auto inner_matvec_on = [&](cudaStream_t st) -> int {
    if (prec == BEM_PREC_FP32) {
      BEM_CUDA_TRY(cudaMemsetAsync(P.Y, 0, sizeof(float2) * (size_t)n * m, st));
      return launch_cgemv((const float2*)A, n, P.X, m, P.Y, nullptr, st, &P.st->err);
    }
    return tc_matvec(tcws, n, prec, P.X, m, P.Y, nullptr, st);
  };
  auto inner_matvec = [&]() -> int { return inner_matvec_on(s); };

  const dim3 gv((n + 255) / 256, m);
  const dim3 pair_grid((n + 2 * kPairThreads - 1) / (2 * kPairThreads), m);
  // FP32-level matvec: CUDA-core FP32, or fp16x3 up to 64 right-hand sides
  // (wider tensor-core tiles accumulate whole rows in tensor memory, ~3e-5)
  const bool full_cycle = prec == BEM_PREC_FP32 || (prec == BEM_PREC_FP16X3 && m <= 64);
  // one classical Gram-Schmidt pass by default: with FP64 dot products and the
  // FP64-refined outer loop it converged exactly like CGS2 here (same
  // iterations and residuals at 4 and 10 kHz) for half the basis traffic
  const int reorth = g_gmres_reorth == 2 ? 1 : 0;
  ArnShape shape;
  {
    int rc0 = arnoldi_shape(n, m, &shape);
    if (rc0) return rc0;
  }
  // The streamed step (launches over all SMs, selective second pass) when
  // the mode key asks for it; the cluster kernel is faster at s5 and s6.
  const bool streamed = reorth == 0 && g_arn_mode == 2;
  // The cooperative step (one launch over all SMs, two grid barriers) when the
  // mode key asks for it.  Measured on the s5 workload (8 right-hand sides)
  // it is slower than the cluster kernel (solve 28.6 ms against 25.2 ms):
  // both are bound by FP64 work per basis element (two float->double
  // conversions and two complex FP64 multiply-adds per element and step), and
  // with ~70 unknowns per CTA its lanes diverge and its bulk copies are small.
  CoShape co;
  const bool coop = reorth == 0 && g_arn_mode == 3 && coop_shape(n, m, R, &co) == BEM_OK;
  const int npairs_all = (n + 1) / 2;
  // about 8 work items per SM over all columns, each of 128 to 4096 pairs
  // (w of an item in FP64: at most 128 KB of shared memory)
  const long long st_target = (long long)npairs_all * m / (8LL * sm_count_linalg());
  const int st_span = (int)std::max(128LL, std::min(4096LL, st_target));
  const int st_nb = (npairs_all + st_span - 1) / st_span;
  const int st_grid = std::min(m * st_nb, 3 * sm_count_linalg());  // persistent: up to 3 blocks per SM
  if (streamed) {
    static std::atomic<bool> st_attr{false};
    if (!st_attr.load(std::memory_order_acquire)) {
      BEM_CUDA_TRY(cudaFuncSetAttribute(gm_st_dots_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(sizeof(double4) * 4096)));
      BEM_CUDA_TRY(cudaFuncSetAttribute(gm_st_dots_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(sizeof(double4) * 4096)));
      st_attr.store(true, std::memory_order_release);
    }
  }
  // one Arnoldi step: the matvec reads the operand that gm_arnoldi_kernel (or
  // gm_start_norm_kernel) wrote and accumulates into Y, which
  // gm_arnoldi_kernel clears again after reading it
  auto arnoldi_step = [&](cudaStream_t st) -> int {
    int r2 = prec == BEM_PREC_FP32
                 ? launch_cgemv((const float2*)A, n, P.X, m, P.Y, P.active, st, &P.st->err)
                 : tc_gemm(tcws, n, prec, m, P.Y, P.active, st);
    if (r2) return r2;
    if (coop) {
      cudaLaunchConfig_t ccfg = {};
      ccfg.gridDim = dim3((unsigned)co.grid, 1, 1);
      ccfg.blockDim = dim3(kCoThreads, 1, 1);
      ccfg.dynamicSmemBytes = co.smem;
      ccfg.stream = st;
      cudaLaunchAttribute cat[1];
      cat[0].id = cudaLaunchAttributeCooperative;
      cat[0].val.cooperative = 1;
      ccfg.attrs = cat;
      ccfg.numAttrs = 1;
      BEM_CUDA_TRY(cudaLaunchKernelEx(&ccfg, gm_arnoldi_coop_kernel, P, co.npc, co.cpc, co.slots));
      count_launch();
      BEM_CUDA_TRY(cudaGetLastError());
      return BEM_OK;
    }
    if (streamed) {
      (gm_st_dots_kernel<0><<<st_grid, kStThreads, sizeof(double4) * st_span, st>>>(P, st_span, st_nb),
       count_launch());
      (gm_st_update_kernel<0><<<st_grid, kStThreads, 0, st>>>(P, st_span, st_nb), count_launch());
      (gm_st_dots_kernel<1><<<st_grid, kStThreads, sizeof(double4) * st_span, st>>>(P, st_span, st_nb),
       count_launch());
      (gm_st_update_kernel<1><<<st_grid, kStThreads, 0, st>>>(P, st_span, st_nb), count_launch());
      (gm_st_finish_kernel<<<st_grid, kStThreads, 0, st>>>(P, st_span, st_nb), count_launch());
      (gm_st_givens_kernel<<<m, 32, sizeof(ArnSmem), st>>>(P), count_launch());
      BEM_CUDA_TRY(cudaGetLastError());
      return BEM_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)shape.cluster, (unsigned)m, 1);
    cfg.blockDim = dim3(kArnThreads, 1, 1);
    cfg.dynamicSmemBytes = shape.smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)shape.cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    BEM_CUDA_TRY(cudaLaunchKernelEx(&cfg, gm_arnoldi_kernel, P, shape.units, shape.chunk, reorth));
    count_launch();
    BEM_CUDA_TRY(cudaGetLastError());
    return BEM_OK;
  };
  // the captured step is destroyed on every return path (early error returns included)
  struct ExecGuard {
    cudaGraphExec_t e = nullptr;
    ~ExecGuard() {
      if (e) cudaGraphExecDestroy(e);
    }
  } step_guard;
  cudaGraphExec_t& step_exec = step_guard.e;
  unsigned long long step_kernels = 0;
  bool step_direct_done = false;  // the first step runs uncaptured (sets kernel attributes)
  // block step: the matvec of the block Q_j, then gm_block_kernel
  auto block_step = [&](cudaStream_t st) -> int {
    int r2 = prec == BEM_PREC_FP32 ? launch_cgemv((const float2*)A, n, P.X, m, P.Y, nullptr, st, &P.st->err)
                                   : tc_gemm(tcws, n, prec, m, P.Y, nullptr, st);
    if (r2) return r2;
    for (int g = 0; g < ngr; g++)
      if ((r2 = launch_block(P, K[g], bshape, g, 1, st))) return r2;
    return BEM_OK;
  };
  ExecGuard block_guard;
  cudaGraphExec_t& block_exec = block_guard.e;
  unsigned long long block_kernels = 0;
  bool block_direct_done = false;
  BlockLS ls[kBkMaxGroups];
  std::vector<double> bres(m), btol(m);
  std::vector<double2> bY;
  constexpr int kBkLookahead = 1;  // one step queued behind the one the host examines
  HostRing* ring;
  int rc = host_ring(m, &ring);
  if (rc) return rc;
  P.snap = ring->dsnap;
  std::vector<double> hres(m), hb(m);

  BEM_CUDA_TRY(cudaMemsetAsync(P.st, 0, sizeof(GmState), s));
  BEM_CUDA_TRY(cudaMemsetAsync(P.colstep, 0, sizeof(int) * m, s));
  BEM_CUDA_TRY(cudaMemsetAsync(P.bnorm2, 0, sizeof(double) * m, s));
  BEM_CUDA_TRY(cudaMemsetAsync(P.norm2, 0, sizeof(double) * m, s));
  (gm_bnorm_kernel<<<gv, 256, 0, s>>>(P, (const float2*)B), count_launch());
  (gm_init_x_kernel<<<gv, 256, 0, s>>>(P, (const float2*)X, use_x0), count_launch());
  BEM_CUDA_TRY(cudaMemcpyAsync(hb.data(), P.bnorm2, sizeof(double) * m, cudaMemcpyDeviceToHost, s));

  int total_iters = 0, matvecs = 0, refinements = 0, iters_done = 0;
  long long launched = 0;  // Arnoldi launches in this solve (snapshot slot = launched % kSnapRing)
  double max_rel = 0.0;
  int status = BEM_ERR_NOT_CONVERGED;
  bool x_nonzero = use_x0 != 0;
  for (int outer = 0; outer <= params->max_refine; outer++) {
    // outer FP64 residual r = b - A x against the FP32 matrix
    BEM_CUDA_TRY(cudaMemsetAsync(rnorm2, 0, sizeof(double) * m, s));
    if (x_nonzero) {
      rc = launch_resid_f64((const float2*)A, n, P.x, m, P.r, (const float2*)B, rnorm2, s, &P.st->err);
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
      // a NaN or Inf anywhere in b or in the residual makes its norm non-finite
      const double rel = !(std::isfinite(bn) && std::isfinite(rn)) ? NAN
                                                                     : (bn > 0.0 ? rn / bn : (rn > 0.0 ? INFINITY : 0.0));
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
    // FP32-level matvecs: one cycle to the target unless it is below their
    // accuracy (~4e-7 relative); then refinement takes over
    const double inner_rtol = full_cycle ? 3e-7 : params->inner_rtol;
    bool first_cycle = true;
    while (total_iters < params->max_iters) {
      BEM_CUDA_TRY(cudaMemsetAsync(P.norm2, 0, sizeof(double) * m, s));
      if (streamed || coop) {  // both parity buffers of the step's sums
        BEM_CUDA_TRY(cudaMemsetAsync(P.hacc, 0, sizeof(double) * 2 * (size_t)m * 4 * (R + 1), s));
        BEM_CUDA_TRY(cudaMemsetAsync(P.nacc, 0, sizeof(double) * 2 * (size_t)m * 3, s));
      }
      if (!first_cycle) {
        (gm_pack_d_kernel<<<gv, 256, 0, s>>>(P), count_launch());
        if ((rc = inner_matvec())) return rc;
        matvecs++;
      }
      (gm_start_vec_kernel<<<gv, 256, 0, s>>>(P, first_cycle ? 0 : 1), count_launch());
      // absolute inner target: inner_rtol * ||r_out|| but never below rtol * ||b|| / 2
      (gm_start_scalar_kernel<<<1, ((m + 31) / 32) * 32, 0, s>>>(P, rnorm2, inner_rtol, 0.5 * params->rtol), count_launch());
      BEM_CUDA_TRY(cudaMemsetAsync(P.Y, 0, sizeof(float2) * (size_t)n * m, s));
      if (block) {
        // ---- block Krylov spaces: start blocks Q_0 R_0 = r_in (CholQR), one per group ----
        first_cycle = false;
        for (int g = 0; g < ngr; g++) {
          const int pg = bshape.p[g];
          BEM_CUDA_TRY(cudaMemsetAsync(K[g].hacc, 0, sizeof(double) * 2 * K[g].ncopy * (size_t)(nbk + 1) * pg * pg * 2, s));
          BEM_CUDA_TRY(cudaMemsetAsync(K[g].gacc, 0, sizeof(double) * 2 * K[g].ncopy * (size_t)pg * pg * 2, s));
          for (int q = 0; q <= nbk; q++) bh[g]->S[q] = 0;  // no step of this solve is in flight here
          if ((rc = launch_block(P, K[g], bshape, g, 0, s))) return rc;
        }
        BEM_CUDA_TRY(cudaMemcpyAsync(btol.data(), P.tol, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        BEM_CUDA_TRY(cudaStreamSynchronize(s));
        bool start_ok = true;
        for (int g = 0; g < ngr; g++) start_ok &= reinterpret_cast<volatile int*>(bh[g]->S)[nbk] == 1;
        if (!start_ok) {
          // a residual block has lost rank (e.g. equal or zero columns):
          // separate Krylov spaces for the rest of this solve
          block = false;
        } else {
          int kk[kBkMaxGroups] = {};
          bool gstop[kBkMaxGroups] = {}, gconv[kBkMaxGroups] = {};
          for (int g = 0; g < ngr; g++) ls[g].init(bshape.p[g], nbk, bh[g]->R0);
          int launched_c = 0, checked_c = 0;
          bool stop = false;
          const long long bbase = launched;
          // step jj of every group: a group stops at a breakdown (keeping the
          // steps before it) or when all its columns meet their tolerance
          // one group's least-squares step (groups touch disjoint state)
          auto group_step = [&](int g, int jj) -> bool {
            const int pg = bshape.p[g], c0 = bshape.col0[g];
            if (reinterpret_cast<volatile int*>(bh[g]->S)[jj] != 1 ||
                !ls[g].add(jj, bh[g]->H + (size_t)(jj % kBkHostRing) * (nbk + 1) * pg * pg, bres.data() + c0)) {
              gstop[g] = true;
              return false;
            }
            kk[g] = jj + 1;
            bool all = true;
            for (int c = c0; c < c0 + pg; c++)
              if (!(bres[c] <= btol[c])) all = false;
            if (all) gconv[g] = gstop[g] = true;
            return true;
          };
          auto process = [&](int jj) -> int {
            BEM_CUDA_TRY(cudaEventSynchronize(ring->ev[(bbase + jj) % kSnapRing]));
            if (stop) return BEM_OK;
            bool accepted = false;
            const double work = (double)(jj + 1) * bshape.p[0] * bshape.p[0] * bshape.p[0];
            if (ngr > 1 && work >= 65536.0) {  // the block QR grows with the cycle: groups on their own threads
              std::future<bool> f[kBkMaxGroups];
              for (int g = 1; g < ngr; g++)
                if (!gstop[g]) f[g] = std::async(std::launch::async, group_step, g, jj);
              if (!gstop[0]) accepted |= group_step(0, jj);
              for (int g = 1; g < ngr; g++)
                if (f[g].valid()) accepted |= f[g].get();
            } else {
              for (int g = 0; g < ngr; g++)
                if (!gstop[g]) accepted |= group_step(g, jj);
            }
            bool all_stopped = true;
            for (int g = 0; g < ngr; g++) all_stopped &= gstop[g];
            if (accepted) iters_done++;
            if (all_stopped) stop = true;
            return BEM_OK;
          };
          while (launched_c < nbk && total_iters < params->max_iters && !stop) {
            if (!block_direct_done || !block_exec) {
              if ((rc = block_step(s))) return rc;
              if (!block_direct_done) {
                block_direct_done = true;
                if (capture_graph(block_step, &block_exec, &block_kernels) != BEM_OK) block_exec = nullptr;
              }
            } else {
              BEM_CUDA_TRY(cudaGraphLaunch(block_exec, s));
              count_launches(block_kernels);
            }
            BEM_CUDA_TRY(cudaEventRecord(ring->ev[launched % kSnapRing], s));
            launched++;
            launched_c++;
            total_iters++;
            while (checked_c < launched_c - kBkLookahead)
              if ((rc = process(checked_c++))) return rc;
          }
          while (checked_c < launched_c)  // every launched step has finished after this
            if ((rc = process(checked_c++))) return rc;
          bool conv = true, none = true;
          for (int g = 0; g < ngr; g++) {
            conv &= gconv[g];
            if (kk[g] == 0) continue;
            none = false;
            ls[g].solve(kk[g], bY);
            BEM_CUDA_TRY(cudaMemcpyAsync(K[g].Yb, bY.data(), sizeof(double2) * bY.size(), cudaMemcpyHostToDevice, s));
            // bY is reused by the next group: the copy must have read it
            BEM_CUDA_TRY(cudaStreamSynchronize(s));
            if ((rc = launch_block_xupdate(P, K[g], kk[g] * bshape.p[g], s))) return rc;
          }
          if (conv) break;
          if (none) {  // broke down at the first step: separate Krylov spaces instead
            block = false;
          }
          continue;
        }
      }
      (gm_start_norm_kernel<<<pair_grid, kPairThreads, 0, s>>>(P), count_launch());
      first_cycle = false;
      int it = 0, checked = 0;
      bool cycle_done = false;
      const long long base = launched;
      // step j of the cycle ran with at least one active column unless an
      // earlier step's slot already showed all converged
      auto examine = [&](int j) -> int {
        const int slot = (int)((base + j) % kSnapRing);
        BEM_CUDA_TRY(cudaEventSynchronize(ring->ev[slot]));
        if (!cycle_done) {
          iters_done++;
          bool any = false;
          for (int c = 0; c < m; c++) any |= ring->snap[(size_t)slot * m + c] != 0;
          if (!any) cycle_done = true;
        }
        return BEM_OK;
      };
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
        BEM_CUDA_TRY(cudaEventRecord(ring->ev[launched % kSnapRing], s));
        launched++;
        it++;
        total_iters++;
        while (checked < it - kLookahead) {
          if ((rc = examine(checked++))) return rc;
        }
        if (cycle_done) break;
      }
      while (checked < it)
        if ((rc = examine(checked++))) return rc;
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
    if (tc_error(tcws, &tc_err, s, false) != BEM_OK || tc_err) status = BEM_ERR_CUDA;
  }
  GmState fin;
  BEM_CUDA_TRY(cudaMemcpyAsync(&fin, P.st, sizeof(GmState), cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  if (fin.err) status = BEM_ERR_CUDA;  // a bounded wait in gm_arnoldi_kernel expired
  (void)total_iters;  // steps enqueued; iters_done counts those with an active column
  matvecs += iters_done;
  if (info) {
    info->status = status;
    info->iterations = iters_done;
    info->refinements = refinements;
    info->matvecs = matvecs;
    info->rel_residual = max_rel;
  }
  return status;
}

// Tensor-core (tcgen05) multi-right-hand-side complex matvec for the Krylov
// solver: Y = A X with A an n x n complex64 matrix held as bf16 planes.
//
// The complex product is one real GEMM.  Row i of A, read as 2n reals
// (re, im interleaved -- exactly the complex64 memory layout), is the K-major
// A operand.  Each right-hand side s becomes two K-major B rows,
//     row 2s   = (xr_0, -xi_0, xr_1, -xi_1, ...)  ->  D[i][2s]   = Re (A x)_i
//     row 2s+1 = (xi_0,  xr_0, xi_1,  xr_1, ...)  ->  D[i][2s+1] = Im (A x)_i
// so D (n x 2m, fp32) is Y in complex64 layout.  Precision modes:
//   BF16X3: A = Ah + Al, x = xh + xl (bf16 hi/lo splits), D = Ah xh + Ah xl + Al xh
//   BF16:   A = Ah only (half the HBM bytes), D = Ah xh + Ah xl
// with FP32 accumulation in tensor memory; the solver's FP64 refinement
// against the FP32 matrix recovers full accuracy.
//
// Kernel: one CTA per SM, stream-K over (128-row block, 64-wide K block)
// units so every SM streams the same number of A bytes; warp 0 issues TMA
// loads (128B swizzle, no multicast) into a ring of stages, warp 1 issues
// tcgen05.mma (M=128, N=2m rounded to 16, K=16) into one of two TMEM
// accumulators, warps 2-5 drain a finished accumulator with tcgen05.ld and add
// it to Y with vector atomics while the next row block accumulates.  Every
// mbarrier wait is bounded in time; on expiry the kernel raises an error flag
// and unwinds instead of spinning.

#include <atomic>
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstring>

#include "async_copy.cuh"
#include "bem_common.cuh"

namespace bemb {

namespace {

constexpr int kBM = 128;            // rows per tile (UMMA M)
constexpr int kBK = 64;             // K elements per stage: one 128-byte swizzle row
constexpr int kTcThreads = 192;     // warp 0 TMA, warp 1 MMA + TMEM owner, warps 2..5 epilogue
constexpr int kSmemBudget = 200 * 1024;
struct TcArgs {
  int n;          // matrix order
  int n_rb;       // row blocks
  int n_kb;       // K blocks (of 64 reals)
  long long units;  // n_rb * n_kb
  int m2;         // 2 * (right-hand sides), valid D columns
  float* Y;       // (n, m2) fp32 = (n, m) complex64
  const int* active;  // if set: nothing to do unless some active[c] != 0, c < nact
  int nact;
  int* err;       // set to 1 when a wait expired
};

// 2-D tiled TMA load (no multicast) completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Same, with an L2 eviction-priority policy (used to stream the matrix
// evict-first so that the small, re-read Krylov basis stays in L2).
__device__ __forceinline__ void tma_load_2d_hint(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar,
                                                 uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, "
      "%3}], [%4], %5;" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// Shared-memory matrix descriptor: K-major tile with 128-byte swizzle, rows
// of 128 bytes, 8-row core groups 1024 bytes apart (SBO), sm100 version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset
  d |= (uint64_t)1 << 46;             // descriptor version
  d |= (uint64_t)2 << 61;             // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::f16: bf16 x bf16 -> f32, both K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int NB, bool X3>
struct TcSmem {
  static constexpr int kABytes = kBM * kBK * 2;  // 16 KB per A plane
  static constexpr int kBBytes = NB * kBK * 2;
  static constexpr int kStageBytes = (X3 ? 2 : 1) * kABytes + 2 * kBBytes;
  static constexpr int kStages = (kSmemBudget / kStageBytes) > 8 ? 8 : (kSmemBudget / kStageBytes);
  static constexpr int kTmemCols =
      (2 * NB <= 32) ? 32 : (2 * NB <= 64 ? 64 : (2 * NB <= 128 ? 128 : (2 * NB <= 256 ? 256 : 512)));
  static constexpr int kBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
};

template <int NB, bool X3>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                   const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl, TcArgs p) {
  using S = TcSmem<NB, X3>;
  if (p.active) {  // uniform: every thread reads the same flags
    int any = 0;
    for (int c = 0; c < p.nact; c++) any |= p.active[c];
    if (!any) return;
  }
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(base + S::kStages * S::kStageBytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + S::kStages;
  uint64_t* accf = bars + 2 * S::kStages;
  uint64_t* acce = accf + 2;
  uint32_t* tmem_slot = (uint32_t*)(acce + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this CTA's contiguous range of (row block, K block) units
  const long long u0 = p.units * blockIdx.x / gridDim.x;
  const long long u1 = p.units * (blockIdx.x + 1) / gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S::kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4 * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)S::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    int stage = 0;
    uint32_t phase = 0;
    const uint64_t stream_policy = l2_evict_first_policy();
    for (long long u = u0; u < u1; u++) {
      const int rb = (int)(u / p.n_kb), kb = (int)(u % p.n_kb);
      if (!mbar_wait(&empty[stage], phase ^ 1u, p.err)) break;
      unsigned char* st = base + stage * S::kStageBytes;
      mbar_expect_tx(&full[stage], S::kStageBytes);
      tma_load_2d_hint(st, &tmAh, kb * kBK, rb * kBM, &full[stage], stream_policy);
      if (X3) tma_load_2d_hint(st + S::kABytes, &tmAl, kb * kBK, rb * kBM, &full[stage], stream_policy);
      unsigned char* bst = st + (X3 ? 2 : 1) * S::kABytes;
      tma_load_2d(bst, &tmBh, kb * kBK, 0, &full[stage]);
      tma_load_2d(bst + S::kBBytes, &tmBl, kb * kBK, 0, &full[stage]);
      if (++stage == S::kStages) {
        stage = 0;
        phase ^= 1u;
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc = instr_desc(kBM, NB);
    int stage = 0;
    uint32_t phase = 0;
    int buf = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    long long u = u0;
    while (u < u1 && ok) {
      const int rb = (int)(u / p.n_kb);
      const long long seg_end = (long long)(rb + 1) * p.n_kb < u1 ? (long long)(rb + 1) * p.n_kb : u1;
      if (!mbar_wait(&acce[buf], acc_phase ^ 1u, p.err)) break;
      tc_fence_after();
      const uint32_t dt = tmem_base + (uint32_t)(buf * NB);
      bool first = true;
      for (; u < seg_end; u++) {
        if (!mbar_wait(&full[stage], phase, p.err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        unsigned char* st = base + stage * S::kStageBytes;
        const uint32_t ah = smem_u32(st);
        const uint32_t al = ah + S::kABytes;
        const uint32_t bh = ah + (X3 ? 2 : 1) * S::kABytes;
        const uint32_t bl = bh + S::kBBytes;
#pragma unroll
        for (int kk = 0; kk < kBK / 16; kk++) {
          const uint32_t off = kk * 32;  // 16 bf16 along the swizzled 128-byte row
          umma_bf16(dt, smem_desc(ah + off), smem_desc(bh + off), idesc, first ? 0u : 1u);
          umma_bf16(dt, smem_desc(ah + off), smem_desc(bl + off), idesc, 1u);
          if (X3) umma_bf16(dt, smem_desc(al + off), smem_desc(bh + off), idesc, 1u);
          first = false;
        }
        umma_commit(&empty[stage]);  // stage reusable once these MMAs have read it
        if (++stage == S::kStages) {
          stage = 0;
          phase ^= 1u;
        }
      }
      umma_commit(&accf[buf]);  // accumulator complete (also on a failed wait: unwinds the epilogue)
      if (++buf == 2) {
        buf = 0;
        acc_phase ^= 1u;
      }
    }
  } else if (warp >= 2) {
    // ---------------- epilogue: TMEM -> registers -> atomics into Y ----------------
    const int quarter = warp & 3;  // TMEM lanes this warp may access
    int buf = 0;
    uint32_t acc_phase = 0;
    long long u = u0;
    while (u < u1) {
      const int rb = (int)(u / p.n_kb);
      const long long seg_end = (long long)(rb + 1) * p.n_kb < u1 ? (long long)(rb + 1) * p.n_kb : u1;
      u = seg_end;
      if (!mbar_wait(&accf[buf], acc_phase, p.err)) break;
      tc_fence_after();
      const int row = rb * kBM + quarter * 32 + lane;
      float* yr = p.Y + (size_t)row * p.m2;
#pragma unroll 1
      for (int c = 0; c < NB; c += 16) {
        float t[16];
        tmem_ld16(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * NB + c), t);
        if (row < p.n) {
#pragma unroll
          for (int i = 0; i < 16; i += 2)
            if (c + i < p.m2) atomicAdd((float2*)(yr + c + i), make_float2(t[i], t[i + 1]));
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
      if (++buf == 2) {
        buf = 0;
        acc_phase ^= 1u;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                 "r"((uint32_t)S::kTmemCols));
  }
}

// A (complex64, n x n) -> bf16 hi (and lo) planes, n x ld, zero padded.
__global__ void tc_split_a_kernel(const float* __restrict__ A, int n, int ld, __nv_bfloat16* __restrict__ Ah,
                                  __nv_bfloat16* __restrict__ Al) {
  const long long total = (long long)n * ld;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx / ld), c = (int)(idx - (long long)r * ld);
    const float a = c < 2 * n ? A[(size_t)r * 2 * n + c] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(a);
    Ah[idx] = h;
    if (Al) Al[idx] = __float2bfloat16_rn(a - __bfloat162float(h));
  }
}

// X (n x m complex64) -> B planes (nb x ld bf16): rows 2s, 2s+1 as in the header.
__global__ void tc_pack_b_kernel(const float2* __restrict__ X, int n, int m, int ld, int nb,
                                 __nv_bfloat16* __restrict__ Bh, __nv_bfloat16* __restrict__ Bl) {
  const long long total = (long long)nb * n;  // one thread per (B row, unknown)
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(idx / n), j = (int)(idx - (long long)row * n);
    const int s = row >> 1;
    float e0 = 0.f, e1 = 0.f;
    if (s < m) {
      const float2 x = X[(size_t)j * m + s];
      if ((row & 1) == 0) {
        e0 = x.x;
        e1 = -x.y;
      } else {
        e0 = x.y;
        e1 = x.x;
      }
    }
    const __nv_bfloat16 h0 = __float2bfloat16_rn(e0), h1 = __float2bfloat16_rn(e1);
    const size_t o = (size_t)row * ld + 2 * j;
    Bh[o] = h0;
    Bh[o + 1] = h1;
    Bl[o] = __float2bfloat16_rn(e0 - __bfloat162float(h0));
    Bl[o + 1] = __float2bfloat16_rn(e1 - __bfloat162float(h1));
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn lookup_encode_fn() {
  void* ptr = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    return (EncodeTiledFn)ptr;
  return nullptr;
}

EncodeTiledFn encode_fn() {
  static const EncodeTiledFn fn = lookup_encode_fn();  // initialised once, thread-safe
  return fn;
}

// bf16 matrix of `rows` x `kext` (row stride ld elements), box kBK x box_rows.
int make_map(CUtensorMap* map, const void* ptr, int kext, int rows, int ld, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return BEM_ERR_CUDA;
  if (((uintptr_t)ptr & 15) || (ld % 8)) return BEM_ERR_INVALID_ARGUMENT;
  cuuint64_t dims[2] = {(cuuint64_t)kext, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? BEM_OK : BEM_ERR_CUDA;
}

inline size_t al256(size_t x) { return (x + 255) / 256 * 256; }

// Workspace: [header: error flag, zero flag][A hi][A lo (bf16x3)][B hi][B lo].
// The A offsets do not depend on m.
struct TcLayout {
  int ld, nb;
  size_t hdr, ah, alo, bh, bl, total;
};

TcLayout tc_layout(int n, int m, int precision) {
  TcLayout L;
  L.ld = ((2 * n + kBK - 1) / kBK) * kBK;
  int nb = ((2 * m + 15) / 16) * 16;
  L.nb = nb <= 16 ? 16 : nb <= 32 ? 32 : nb <= 64 ? 64 : nb <= 128 ? 128 : 256;
  size_t o = 0;
  L.hdr = o;
  o = al256(o + 256);
  L.ah = o;
  o = al256(o + (size_t)n * L.ld * 2);
  L.alo = o;
  if (precision == BEM_PREC_BF16X3) o = al256(o + (size_t)n * L.ld * 2);
  L.bh = o;
  o = al256(o + (size_t)L.nb * L.ld * 2);
  L.bl = o;
  o = al256(o + (size_t)L.nb * L.ld * 2);
  L.total = o;
  return L;
}

template <int NB, bool X3>
int launch_tc(const TcLayout& L, char* ws, int n, const int* active, int nact, float* Y, int m2, cudaStream_t s) {
  using S = TcSmem<NB, X3>;
  static std::atomic<bool> attr{false};
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel<NB, X3>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes));
    attr.store(true, std::memory_order_release);
  }
  CUtensorMap mah, mal, mbh, mbl;
  int rc;
  if ((rc = make_map(&mah, ws + L.ah, 2 * n, n, L.ld, kBM))) return rc;
  if ((rc = make_map(&mal, ws + (X3 ? L.alo : L.ah), 2 * n, n, L.ld, kBM))) return rc;
  if ((rc = make_map(&mbh, ws + L.bh, 2 * n, NB, L.ld, NB))) return rc;
  if ((rc = make_map(&mbl, ws + L.bl, 2 * n, NB, L.ld, NB))) return rc;
  TcArgs a;
  a.n = n;
  a.n_rb = (n + kBM - 1) / kBM;
  a.n_kb = (2 * n + kBK - 1) / kBK;
  a.units = (long long)a.n_rb * a.n_kb;
  a.m2 = m2;
  a.Y = Y;
  a.err = (int*)(ws + L.hdr);
  a.active = active;
  a.nact = nact;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (long long)sms < a.units ? sms : (int)a.units;
  (tc_gemm_kernel<NB, X3><<<grid, kTcThreads, S::kBytes, s>>>(mah, mal, mbh, mbl, a), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

}  // namespace

size_t tc_workspace_bytes(int n, int m, int precision) {
  if ((precision != BEM_PREC_BF16X3 && precision != BEM_PREC_BF16) || n <= 0 || m <= 0 || m > 128) return 0;
  return tc_layout(n, m, precision).total;
}

int tc_operator_prepare(const float2* A, int n, int precision, void* ws, cudaStream_t s) {
  const TcLayout L = tc_layout(n, 1, precision);
  char* w = (char*)ws;
  BEM_CUDA_TRY(cudaMemsetAsync(w + L.hdr, 0, 256, s));
  (tc_split_a_kernel<<<1184, 256, 0, s>>>((const float*)A, n, L.ld, (__nv_bfloat16*)(w + L.ah),
                                          precision == BEM_PREC_BF16X3 ? (__nv_bfloat16*)(w + L.alo) : nullptr),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

int tc_gemm(const void* ws_, int n, int precision, int m, float2* Y, const int* active, cudaStream_t s);

// Y = A X for m <= 128 right-hand sides; `active` (device ints, one per
// right-hand side, may be NULL) turns the launch into a no-op when all are 0.
int tc_matvec(const void* ws_, int n, int precision, const float2* X, int m, float2* Y, const int* active,
              cudaStream_t s) {
  if (m <= 0 || m > 128) return BEM_ERR_UNSUPPORTED;
  char* ws = (char*)ws_;
  const TcLayout L = tc_layout(n, m, precision);
  (tc_pack_b_kernel<<<1184, 256, 0, s>>>(X, n, m, L.ld, L.nb, (__nv_bfloat16*)(ws + L.bh),
                                         (__nv_bfloat16*)(ws + L.bl)),
   count_launch());
  BEM_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(float2) * (size_t)n * m, s));
  return tc_gemm(ws_, n, precision, m, Y, active, s);
}

// B operand planes, for producers that write them directly: element (j, s)
// of X occupies columns 2j, 2j+1 of rows 2s, 2s+1 (row stride ldb), as
// written by tc_pack_b_kernel.  Rows 2m..nb-1 must be zero.
int tc_b_planes(void* ws_, int n, int m, int precision, __nv_bfloat16** bh, __nv_bfloat16** bl, int* ldb,
                int* nb) {
  if (m <= 0 || m > 128) return BEM_ERR_UNSUPPORTED;
  char* ws = (char*)ws_;
  const TcLayout L = tc_layout(n, m, precision);
  *bh = (__nv_bfloat16*)(ws + L.bh);
  *bl = (__nv_bfloat16*)(ws + L.bl);
  *ldb = L.ld;
  *nb = L.nb;
  return BEM_OK;
}

// Y += A_lp B with the B planes already in the workspace.
int tc_gemm(const void* ws_, int n, int precision, int m, float2* Y, const int* active, cudaStream_t s) {
  if (m <= 0 || m > 128) return BEM_ERR_UNSUPPORTED;
  char* ws = (char*)ws_;
  const TcLayout L = tc_layout(n, m, precision);
  const bool x3 = precision == BEM_PREC_BF16X3;
  float* y = (float*)Y;
  switch (L.nb) {
    case 16: return x3 ? launch_tc<16, true>(L, ws, n, active, m, y, 2 * m, s) : launch_tc<16, false>(L, ws, n, active, m, y, 2 * m, s);
    case 32: return x3 ? launch_tc<32, true>(L, ws, n, active, m, y, 2 * m, s) : launch_tc<32, false>(L, ws, n, active, m, y, 2 * m, s);
    case 64: return x3 ? launch_tc<64, true>(L, ws, n, active, m, y, 2 * m, s) : launch_tc<64, false>(L, ws, n, active, m, y, 2 * m, s);
    case 128: return x3 ? launch_tc<128, true>(L, ws, n, active, m, y, 2 * m, s) : launch_tc<128, false>(L, ws, n, active, m, y, 2 * m, s);
    default: return x3 ? launch_tc<256, true>(L, ws, n, active, m, y, 2 * m, s) : launch_tc<256, false>(L, ws, n, active, m, y, 2 * m, s);
  }
}

// Error flag of the tensor-core kernels that used this workspace (syncs).
int tc_error(const void* ws_, int* err_host, cudaStream_t s) {
  BEM_CUDA_TRY(cudaMemcpyAsync(err_host, ws_, sizeof(int), cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  return BEM_OK;
}

}  // namespace bemb

using namespace bemb;

extern "C" size_t bem_tc_operator_bytes(int n, int m, int precision) { return tc_workspace_bytes(n, m, precision); }

extern "C" int bem_tc_operator_prepare(const void* A, int n, int precision, void* ws, size_t ws_bytes,
                                       bem_stream_t stream) {
  if (!A || !ws || n <= 0) return BEM_ERR_INVALID_ARGUMENT;
  if (precision != BEM_PREC_BF16X3 && precision != BEM_PREC_BF16) return BEM_ERR_INVALID_ARGUMENT;
  if (ws_bytes < tc_workspace_bytes(n, 1, precision)) return BEM_ERR_WORKSPACE;
  return tc_operator_prepare((const float2*)A, n, precision, ws, (cudaStream_t)stream);
}

extern "C" int bem_tc_matmul(const void* ws, size_t ws_bytes, int n, int precision, const void* X, int m, void* Y,
                             bem_stream_t stream) {
  if (!ws || !X || !Y || n <= 0 || m <= 0) return BEM_ERR_INVALID_ARGUMENT;
  if (m > 128) return BEM_ERR_UNSUPPORTED;
  if (ws_bytes < tc_workspace_bytes(n, m, precision)) return BEM_ERR_WORKSPACE;
  return tc_matvec(ws, n, precision, (const float2*)X, m, (float2*)Y, nullptr, (cudaStream_t)stream);
}

extern "C" int bem_tc_status(const void* ws, bem_stream_t stream) {
  if (!ws) return BEM_ERR_INVALID_ARGUMENT;
  int err = 0;
  int rc = tc_error(ws, &err, (cudaStream_t)stream);
  if (rc) return rc;
  return err ? BEM_ERR_CUDA : BEM_OK;
}

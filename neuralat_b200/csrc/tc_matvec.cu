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
//   FP16X3: as BF16X3 with fp16 hi/lo planes.  fp16 keeps 11 significant
//           bits, so the two-term split is accurate to 2^-24 (FP32 level,
//           against 2^-16 for bf16) at the same 4 bytes per real.  Its range
//           is narrow, so every row of A is scaled by a power of two that puts
//           the row maximum below 2^14 (kept as rinv), every right-hand side
//           likewise (cinv; normalised Krylov vectors use the fixed 2^14), and
//           the epilogue multiplies D back by rinv[row] * cinv[s].
// with FP32 accumulation in tensor memory; the solver's FP64 refinement
// against the FP32 matrix recovers full accuracy.
//
// Accumulation: the tensor core's in-place FP32 accumulation over a long K
// range loses precision (measured: ~3e-5 relative on the BEM matrix whatever
// the operand split), so accumulator segments are short (`promote` K blocks,
// two by default for N <= 128, i.e. up to 64 right-hand sides): after each
// segment the epilogue adds the tensor-memory sum to per-row registers with
// round-to-nearest FP32 adds and writes Y once per row block (fp16x3 then
// matches an FP32 matvec, ~5e-7).
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
#include <cuda_fp16.h>

#include <cstring>

#include "async_copy.cuh"
#include "bem_common.cuh"

namespace bemb {

int g_tc_promote = 0;  // accumulator segment length in K blocks (0: automatic); a tuning knob
int g_tc_wait_us = 0;  // limit of the bounded waits of the tensor-core kernels in microseconds (0: 2 s)
std::atomic<int> g_tc_skip_fill{0};  // test hook, one launch: fill (value - 1) of CTA 0 is not issued

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
  const float* rinv;  // FP16X3: per-row and per-right-hand-side inverse scales
  const float* cinv;
  long long promote;  // K blocks per accumulator segment
  unsigned long long wait_ns;  // limit of every bounded wait
  int skip_fill;  // test hook: CTA 0's producer leaves its fill number skip_fill (>= 0) unissued, so the
                  // consumer's bounded wait on that stage expires; -1 = off
};

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

// Instruction descriptor, kind::f16 -> f32 accumulate, both operands K-major
// and of the same type: bf16 x bf16 (formats 1) or f16 x f16 (formats 0).
__host__ __device__ constexpr uint32_t instr_desc(int M, int N, bool f16) {
  return (1u << 4) | (f16 ? 0u : ((1u << 7) | (1u << 10))) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
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
  // tensor-memory accumulators in flight: with one-K-block segments the MMA
  // issuer runs up to kAccBufs segments ahead of the epilogue
  static constexpr int kAccBufs = NB <= 128 ? 4 : 2;
  static constexpr int kTmemCols = (kAccBufs * NB <= 32)    ? 32
                                   : (kAccBufs * NB <= 64)  ? 64
                                   : (kAccBufs * NB <= 128) ? 128
                                   : (kAccBufs * NB <= 256) ? 256
                                                            : 512;
  static constexpr int kBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
  static_assert((2 * kStages + 2 * kAccBufs) * 8 + 8 + 8 <= 256, "barriers, TMEM slot and done barrier fit");
};

// End of the accumulator segment that starts at unit u: the row block's end,
// the CTA's end, or `promote` K blocks, whichever comes first (the MMA issuer
// and the epilogue walk the same segments).
__device__ __forceinline__ long long segment_end(long long u, long long u1, const TcArgs& p) {
  const long long rb_end = (u / p.n_kb + 1) * p.n_kb;
  long long e = rb_end < u1 ? rb_end : u1;
  if (u + p.promote < e) e = u + p.promote;
  return e;
}

template <int NB, bool X3, bool F16>
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
  uint64_t* acce = accf + S::kAccBufs;
  uint64_t* mma_done = acce + S::kAccBufs;  // all MMAs of this CTA complete (checked before TMEM is released)
  uint32_t* tmem_slot = (uint32_t*)(mma_done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this CTA's contiguous range of (row block, K block) units
  const long long u0 = p.units * blockIdx.x / gridDim.x;
  const long long u1 = p.units * (blockIdx.x + 1) / gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S::kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < S::kAccBufs; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4 * 32);
    }
    mbar_init(mma_done, 1);
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
    int armed[S::kStages];  // phase of each stage's last issued fill, -1: none
#pragma unroll
    for (int q = 0; q < S::kStages; q++) armed[q] = -1;
    const uint64_t stream_policy = l2_evict_first_policy();
    long long fill = 0;
    for (long long u = u0; u < u1; u++, fill++) {
      const int rb = (int)(u / p.n_kb), kb = (int)(u % p.n_kb);
      if (!mbar_wait(&empty[stage], phase ^ 1u, p.err, p.wait_ns)) break;
      if (!(blockIdx.x == 0 && fill == p.skip_fill)) {
        unsigned char* st = base + stage * S::kStageBytes;
        mbar_expect_tx(&full[stage], S::kStageBytes);
        tma_load_2d_hint(st, &tmAh, kb * kBK, rb * kBM, &full[stage], stream_policy);
        if (X3) tma_load_2d_hint(st + S::kABytes, &tmAl, kb * kBK, rb * kBM, &full[stage], stream_policy);
        unsigned char* bst = st + (X3 ? 2 : 1) * S::kABytes;
        tma_load_2d(bst, &tmBh, kb * kBK, 0, &full[stage]);
        tma_load_2d(bst + S::kBBytes, &tmBl, kb * kBK, 0, &full[stage]);
        armed[stage] = (int)phase;
      }
      if (++stage == S::kStages) {
        stage = 0;
        phase ^= 1u;
      }
    }
    if (*(volatile int*)p.err) {
      // a wait expired: the consumer may have stopped; let every issued copy
      // land before the CTA exits (the last fill of each stage is the newest)
#pragma unroll 1
      for (int q = 0; q < S::kStages; q++)
        if (armed[q] >= 0) mbar_wait_drain(&full[q], (uint32_t)armed[q], p.wait_ns);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc = instr_desc(kBM, NB, F16);
    int stage = 0;
    uint32_t phase = 0;
    int buf = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    long long u = u0;
    while (u < u1 && ok) {
      const long long seg_end = segment_end(u, u1, p);
      if (!mbar_wait(&acce[buf], acc_phase ^ 1u, p.err, p.wait_ns)) break;
      tc_fence_after();
      const uint32_t dt = tmem_base + (uint32_t)(buf * NB);
      bool first = true;
      for (; u < seg_end; u++) {
        if (!mbar_wait(&full[stage], phase, p.err, p.wait_ns)) {
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
      if (++buf == S::kAccBufs) {
        buf = 0;
        acc_phase ^= 1u;
      }
    }
    // every MMA issued here has finished reading shared memory and writing
    // tensor memory before the CTA releases either (the epilogue may have
    // stopped waiting after an expired wait)
    umma_commit(mma_done);
    mbar_wait_drain(mma_done, 0u, p.wait_ns);
  } else if (warp >= 2) {
    // ---------------- epilogue: TMEM -> registers -> atomics into Y ----------------
    // Each lane owns one row.  With NB <= 128 the segment sums are added in
    // registers (round-to-nearest FP32) and Y receives one atomic per entry
    // when the row block (or this CTA's range) ends; wider tiles add every
    // segment to Y directly.
    constexpr bool kRegAcc = NB <= 128;
    const int quarter = warp & 3;  // TMEM lanes this warp may access
    int buf = 0;
    uint32_t acc_phase = 0;
    long long u = u0;
    float racc[kRegAcc ? NB : 1];
#pragma unroll
    for (int i = 0; i < (kRegAcc ? NB : 1); i++) racc[i] = 0.f;
    while (u < u1) {
      const int rb = (int)(u / p.n_kb);
      const long long seg_end = segment_end(u, u1, p);
      u = seg_end;
      const bool row_done = u == u1 || u % p.n_kb == 0;
      if (!mbar_wait(&accf[buf], acc_phase, p.err, p.wait_ns)) break;
      tc_fence_after();
      const int row = rb * kBM + quarter * 32 + lane;
      float* yr = p.Y + (size_t)row * p.m2;
      const float ri = (F16 && row < p.n) ? p.rinv[row] : 1.f;
      if (kRegAcc) {
#pragma unroll
        for (int c = 0; c < (kRegAcc ? NB : 16); c += 16) {
          float t[16];
          tmem_ld16(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * NB + c), t);
#pragma unroll
          for (int i = 0; i < 16; i++) racc[c + i] += t[i];
        }
      } else {
#pragma unroll 1
        for (int c = 0; c < NB; c += 16) {
          float t[16];
          tmem_ld16(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * NB + c), t);
          if (row < p.n) {
#pragma unroll
            for (int i = 0; i < 16; i += 2)
              if (c + i < p.m2) {
                const float sc = F16 ? ri * p.cinv[(c + i) >> 1] : 1.f;
                atomicAdd((float2*)(yr + c + i), make_float2(t[i] * sc, t[i + 1] * sc));
              }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
      if (++buf == S::kAccBufs) {
        buf = 0;
        acc_phase ^= 1u;
      }
      if (kRegAcc && row_done) {
        if (row < p.n) {
#pragma unroll
          for (int i = 0; i < (kRegAcc ? NB : 1); i += 2)
            if (i < p.m2) {
              const float sc = F16 ? ri * p.cinv[i >> 1] : 1.f;
              atomicAdd((float2*)(yr + i), make_float2(racc[i] * sc, racc[i + 1] * sc));
            }
        }
#pragma unroll
        for (int i = 0; i < (kRegAcc ? NB : 1); i++) racc[i] = 0.f;
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

// Power of two q with |v| * q < 2^14 for |v| <= mx (1 for mx == 0).
__device__ __forceinline__ float f16_scale(float mx) {
  if (!(mx > 0.f)) return 1.f;
  int e;
  frexpf(mx, &e);  // mx < 2^e
  return ldexpf(1.f, 14 - e);
}

// A -> fp16 hi/lo planes, row r scaled by a power of two (rinv[r] = 1/scale).
// One block per row at a time: a max reduction, then the split.
__global__ void __launch_bounds__(256) tc_split_a_f16_kernel(const float* __restrict__ A, int n, int ld,
                                                            __half* __restrict__ Ah, __half* __restrict__ Al,
                                                            float* __restrict__ rinv) {
  __shared__ float red[8];
  // n even: rows start 16-byte aligned (float4 reads) and ld is a multiple of
  // 4 (8-byte stores of four halves per plane)
  const bool vec = (n & 1) == 0 && (ld & 3) == 0;
  for (int r = blockIdx.x; r < n; r += gridDim.x) {
    const float* row = A + (size_t)r * 2 * n;
    float mx = 0.f;
    if (vec) {
      const float4* row4 = reinterpret_cast<const float4*>(row);
#pragma unroll 4
      for (int c = threadIdx.x; c < n / 2; c += 256) {
        const float4 v = row4[c];
        mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
      }
    } else {
      for (int c = threadIdx.x; c < 2 * n; c += 256) mx = fmaxf(mx, fabsf(row[c]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    float rmx = 0.f;
#pragma unroll
    for (int w = 0; w < 8; w++) rmx = fmaxf(rmx, red[w]);
    const float q = f16_scale(rmx);
    if (threadIdx.x == 0) rinv[r] = 1.f / q;
    if (vec) {
      const float4* row4 = reinterpret_cast<const float4*>(row);
      uint2* h4 = reinterpret_cast<uint2*>(Ah + (size_t)r * ld);
      uint2* l4 = reinterpret_cast<uint2*>(Al + (size_t)r * ld);
#pragma unroll 4
      for (int c = threadIdx.x; c < ld / 4; c += 256) {
        float a[4] = {0.f, 0.f, 0.f, 0.f};
        if (c < n / 2) {
          const float4 v = row4[c];
          a[0] = v.x * q;
          a[1] = v.y * q;
          a[2] = v.z * q;
          a[3] = v.w * q;
        }
        __align__(8) __half hi[4], lo[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          hi[e] = __float2half_rn(a[e]);
          lo[e] = __float2half_rn(a[e] - __half2float(hi[e]));
        }
        h4[c] = *reinterpret_cast<const uint2*>(hi);
        l4[c] = *reinterpret_cast<const uint2*>(lo);
      }
    } else {
      for (int c = threadIdx.x; c < ld; c += 256) {
        const float a = c < 2 * n ? row[c] * q : 0.f;
        const __half h = __float2half_rn(a);
        Ah[(size_t)r * ld + c] = h;
        Al[(size_t)r * ld + c] = __float2half_rn(a - __half2float(h));
      }
    }
    __syncthreads();  // red is reused by the next row
  }
}

// The same split with the row staged in shared memory (n even, ld a
// multiple of 4, n / 2 float4 per row in dynamic shared memory): the matrix
// is read from HBM once, for the maximum, and split from shared memory.
__global__ void __launch_bounds__(256) tc_split_a_f16_smem_kernel(const float* __restrict__ A, int n, int ld,
                                                                 __half* __restrict__ Ah, __half* __restrict__ Al,
                                                                 float* __restrict__ rinv) {
  extern __shared__ float4 rowbuf[];  // [n / 2]
  __shared__ float red[8];
  const int nv = n / 2;
  for (int r = blockIdx.x; r < n; r += gridDim.x) {
    const float4* row4 = reinterpret_cast<const float4*>(A + (size_t)r * 2 * n);
    float mx = 0.f;
#pragma unroll 4
    for (int c = threadIdx.x; c < nv; c += 256) {
      const float4 v = __ldcs(row4 + c);
      rowbuf[c] = v;
      mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();  // also: rowbuf complete
    float rmx = 0.f;
#pragma unroll
    for (int w = 0; w < 8; w++) rmx = fmaxf(rmx, red[w]);
    const float q = f16_scale(rmx);
    if (threadIdx.x == 0) rinv[r] = 1.f / q;
    uint2* h4 = reinterpret_cast<uint2*>(Ah + (size_t)r * ld);
    uint2* l4 = reinterpret_cast<uint2*>(Al + (size_t)r * ld);
#pragma unroll 4
    for (int c = threadIdx.x; c < ld / 4; c += 256) {
      float a[4] = {0.f, 0.f, 0.f, 0.f};
      if (c < nv) {
        const float4 v = rowbuf[c];
        a[0] = v.x * q;
        a[1] = v.y * q;
        a[2] = v.z * q;
        a[3] = v.w * q;
      }
      __align__(8) __half hi[4], lo[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        hi[e] = __float2half_rn(a[e]);
        lo[e] = __float2half_rn(a[e] - __half2float(hi[e]));
      }
      h4[c] = *reinterpret_cast<const uint2*>(hi);
      l4[c] = *reinterpret_cast<const uint2*>(lo);
    }
    __syncthreads();  // red and rowbuf are reused by the next row
  }
}

// Column maxima of X (n x m complex64) for the fp16 scales: grid (blocks, m).
__global__ void tc_colmax_kernel(const float2* __restrict__ X, int n, int m, unsigned* __restrict__ cmax) {
  const int s = blockIdx.y;
  float mx = 0.f;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const float2 x = X[(size_t)j * m + s];
    mx = fmaxf(mx, fmaxf(fabsf(x.x), fabsf(x.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&cmax[s], __float_as_uint(mx));  // non-negative floats order as uints
}

// X -> fp16 B planes with the per-column scales (rows 2s, 2s+1 as for bf16).
__global__ void tc_pack_b_f16_kernel(const float2* __restrict__ X, int n, int m, int ld, int nb,
                                     const unsigned* __restrict__ cmax, __half* __restrict__ Bh,
                                     __half* __restrict__ Bl, float* __restrict__ cinv) {
  const long long total = (long long)nb * n;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(idx / n), j = (int)(idx - (long long)row * n);
    const int s = row >> 1;
    float e0 = 0.f, e1 = 0.f;
    if (s < m) {
      const float q = f16_scale(__uint_as_float(cmax[s]));
      if (j == 0 && (row & 1) == 0) cinv[s] = 1.f / q;
      const float2 x = X[(size_t)j * m + s];
      if ((row & 1) == 0) {
        e0 = x.x * q;
        e1 = -x.y * q;
      } else {
        e0 = x.y * q;
        e1 = x.x * q;
      }
    }
    const __half h0 = __float2half_rn(e0), h1 = __float2half_rn(e1);
    const size_t o = (size_t)row * ld + 2 * j;
    Bh[o] = h0;
    Bh[o + 1] = h1;
    Bl[o] = __float2half_rn(e0 - __half2float(h0));
    Bl[o + 1] = __float2half_rn(e1 - __half2float(h1));
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

}  // namespace

// 2-D FP32 tensor map (no swizzle, zero fill outside the tensor) over a
// row-major matrix of `rows` rows of `cols` floats, `ld_bytes` apart.
int encode_map_2d_f32(CUtensorMap* map, const void* ptr, unsigned long long cols, unsigned long long rows,
                      unsigned long long ld_bytes, unsigned box_cols, unsigned box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return BEM_ERR_CUDA;
  if (((uintptr_t)ptr & 15) || (ld_bytes & 15)) return BEM_ERR_INVALID_ARGUMENT;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld_bytes};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? BEM_OK : BEM_ERR_CUDA;
}

// Same with the 128-byte swizzle (box_cols * 4 bytes must be 128): 16-byte
// chunk k of box row r lands at chunk k ^ (r & 7) of its 128-byte row, so
// lanes that read one chunk each of consecutive rows hit distinct banks.
int encode_map_2d_f32_sw128(CUtensorMap* map, const void* ptr, unsigned long long cols, unsigned long long rows,
                            unsigned long long ld_bytes, unsigned box_cols, unsigned box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return BEM_ERR_CUDA;
  if (((uintptr_t)ptr & 15) || (ld_bytes & 15) || box_cols * 4 != 128) return BEM_ERR_INVALID_ARGUMENT;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld_bytes};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? BEM_OK : BEM_ERR_CUDA;
}

namespace {

// Workspace: [header: error flag][column maxima (m)][cinv (m)][rinv (n)]
// [A hi][A lo (bf16x3, fp16x3)][B hi][B lo].  The A offsets do not depend on m.
struct TcLayout {
  int ld, nb;
  size_t hdr, cmax, cinv, rinv, ah, alo, bh, bl, total;
};

TcLayout tc_layout(int n, int m, int precision) {
  TcLayout L;
  L.ld = ((2 * n + kBK - 1) / kBK) * kBK;
  int nb = ((2 * m + 15) / 16) * 16;
  L.nb = nb <= 16 ? 16 : nb <= 32 ? 32 : nb <= 64 ? 64 : nb <= 128 ? 128 : 256;
  size_t o = 0;
  L.hdr = o;
  o = al256(o + 256);
  L.cmax = o;
  o = al256(o + 128 * sizeof(unsigned));
  L.cinv = o;
  o = al256(o + 128 * sizeof(float));
  L.rinv = o;
  o = al256(o + sizeof(float) * (size_t)n);
  L.ah = o;
  o = al256(o + (size_t)n * L.ld * 2);
  L.alo = o;
  if (precision == BEM_PREC_BF16X3 || precision == BEM_PREC_FP16X3) o = al256(o + (size_t)n * L.ld * 2);
  L.bh = o;
  o = al256(o + (size_t)L.nb * L.ld * 2);
  L.bl = o;
  o = al256(o + (size_t)L.nb * L.ld * 2);
  L.total = o;
  return L;
}

template <int NB, bool X3, bool F16>
int launch_tc(const TcLayout& L, char* ws, int n, const int* active, int nact, float* Y, int m2, cudaStream_t s) {
  using S = TcSmem<NB, X3>;
  static std::atomic<bool> attr{false};
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(
        cudaFuncSetAttribute(tc_gemm_kernel<NB, X3, F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes));
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
  a.rinv = F16 ? (const float*)(ws + L.rinv) : nullptr;
  a.cinv = F16 ? (const float*)(ws + L.cinv) : nullptr;
  // two K blocks per segment: fp16x3 error 6e-7 on the BEM matrix (one block:
  // 4e-7 but 18% slower; 16 blocks: 4e-6; a whole row block: 3e-5)
  a.promote = g_tc_promote > 0 ? g_tc_promote : (NB <= 128 ? 2 : (1ll << 40));
  a.wait_ns = g_tc_wait_us > 0 ? 1000ull * (unsigned long long)g_tc_wait_us : kWaitLimitNs;
  a.skip_fill = g_tc_skip_fill.exchange(0) - 1;  // consumed by this launch
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (long long)sms < a.units ? sms : (int)a.units;
  (tc_gemm_kernel<NB, X3, F16><<<grid, kTcThreads, S::kBytes, s>>>(mah, mal, mbh, mbl, a), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

}  // namespace

size_t tc_workspace_bytes(int n, int m, int precision) {
  if ((precision != BEM_PREC_BF16X3 && precision != BEM_PREC_BF16 && precision != BEM_PREC_FP16X3) || n <= 0 ||
      m <= 0 || m > 128)
    return 0;
  return tc_layout(n, m, precision).total;
}

int tc_operator_prepare(const float2* A, int n, int precision, void* ws, cudaStream_t s) {
  const TcLayout L = tc_layout(n, 1, precision);
  char* w = (char*)ws;
  BEM_CUDA_TRY(cudaMemsetAsync(w + L.hdr, 0, 256, s));
  if (precision == BEM_PREC_FP16X3) {
    // a row of up to 96 KB staged in shared memory (two CTAs per SM), else two reads of it
    const size_t row_bytes = sizeof(float4) * (size_t)(n / 2);
    const bool staged = (n & 1) == 0 && (L.ld & 3) == 0 && ((uintptr_t)A & 15) == 0 && row_bytes <= 96 * 1024;
    if (staged) {
      static std::atomic<bool> attr{false};
      if (!attr.load(std::memory_order_acquire)) {
        BEM_CUDA_TRY(cudaFuncSetAttribute(tc_split_a_f16_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          96 * 1024));
        attr.store(true, std::memory_order_release);
      }
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const int grid = std::min(n, 2 * sms);
      (tc_split_a_f16_smem_kernel<<<grid, 256, row_bytes, s>>>((const float*)A, n, L.ld, (__half*)(w + L.ah),
                                                               (__half*)(w + L.alo), (float*)(w + L.rinv)),
       count_launch());
    } else {
      (tc_split_a_f16_kernel<<<n < 1184 ? n : 1184, 256, 0, s>>>((const float*)A, n, L.ld, (__half*)(w + L.ah),
                                                                  (__half*)(w + L.alo), (float*)(w + L.rinv)),
       count_launch());
    }
  } else {
    (tc_split_a_kernel<<<1184, 256, 0, s>>>((const float*)A, n, L.ld, (__nv_bfloat16*)(w + L.ah),
                                            precision == BEM_PREC_BF16X3 ? (__nv_bfloat16*)(w + L.alo) : nullptr),
     count_launch());
  }
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
  if (precision == BEM_PREC_FP16X3) {
    BEM_CUDA_TRY(cudaMemsetAsync(ws + L.cmax, 0, sizeof(unsigned) * m, s));
    (tc_colmax_kernel<<<dim3(n < 8192 ? (n + 255) / 256 : 32, m), 256, 0, s>>>(X, n, m, (unsigned*)(ws + L.cmax)),
     count_launch());
    (tc_pack_b_f16_kernel<<<1184, 256, 0, s>>>(X, n, m, L.ld, L.nb, (const unsigned*)(ws + L.cmax),
                                               (__half*)(ws + L.bh), (__half*)(ws + L.bl), (float*)(ws + L.cinv)),
     count_launch());
  } else {
    (tc_pack_b_kernel<<<1184, 256, 0, s>>>(X, n, m, L.ld, L.nb, (__nv_bfloat16*)(ws + L.bh),
                                           (__nv_bfloat16*)(ws + L.bl)),
     count_launch());
  }
  BEM_CUDA_TRY(cudaMemsetAsync(Y, 0, sizeof(float2) * (size_t)n * m, s));
  return tc_gemm(ws_, n, precision, m, Y, active, s);
}

// B operand planes, for producers that write them directly: element (j, s)
// of X occupies columns 2j, 2j+1 of rows 2s, 2s+1 (row stride ldb), as
// written by tc_pack_b_kernel (bf16) or tc_pack_b_f16_kernel (fp16, scaled:
// the producer also sets cinv[s]).  Rows 2m..nb-1 must be zero.
int tc_b_planes(void* ws_, int n, int m, int precision, __nv_bfloat16** bh, __nv_bfloat16** bl, int* ldb,
                int* nb, float** cinv) {
  if (m <= 0 || m > 128) return BEM_ERR_UNSUPPORTED;
  char* ws = (char*)ws_;
  const TcLayout L = tc_layout(n, m, precision);
  *bh = (__nv_bfloat16*)(ws + L.bh);
  *bl = (__nv_bfloat16*)(ws + L.bl);
  *ldb = L.ld;
  *nb = L.nb;
  *cinv = (float*)(ws + L.cinv);
  return BEM_OK;
}

// Y += A_lp B with the B planes already in the workspace.
int tc_gemm(const void* ws_, int n, int precision, int m, float2* Y, const int* active, cudaStream_t s) {
  if (m <= 0 || m > 128) return BEM_ERR_UNSUPPORTED;
  char* ws = (char*)ws_;
  const TcLayout L = tc_layout(n, m, precision);
  float* y = (float*)Y;
#define BEM_TC_CASE(NBV)                                                                                  \
  case NBV:                                                                                               \
    if (precision == BEM_PREC_FP16X3) return launch_tc<NBV, true, true>(L, ws, n, active, m, y, 2 * m, s); \
    if (precision == BEM_PREC_BF16X3) return launch_tc<NBV, true, false>(L, ws, n, active, m, y, 2 * m, s); \
    return launch_tc<NBV, false, false>(L, ws, n, active, m, y, 2 * m, s);
  switch (L.nb) {
    BEM_TC_CASE(16)
    BEM_TC_CASE(32)
    BEM_TC_CASE(64)
    BEM_TC_CASE(128)
    BEM_TC_CASE(256)
  }
#undef BEM_TC_CASE
  return BEM_ERR_UNSUPPORTED;
}

// Error flag of the tensor-core kernels that used this workspace (syncs);
// with `clear` it is reset for the next launches.
int tc_error(const void* ws_, int* err_host, cudaStream_t s, bool clear) {
  BEM_CUDA_TRY(cudaMemcpyAsync(err_host, ws_, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (clear) BEM_CUDA_TRY(cudaMemsetAsync(const_cast<void*>(ws_), 0, sizeof(int), s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  return BEM_OK;
}

}  // namespace bemb

using namespace bemb;

extern "C" size_t bem_tc_operator_bytes(int n, int m, int precision) { return tc_workspace_bytes(n, m, precision); }

extern "C" int bem_tc_operator_prepare(const void* A, int n, int precision, void* ws, size_t ws_bytes,
                                       bem_stream_t stream) {
  if (!A || !ws || n <= 0) return BEM_ERR_INVALID_ARGUMENT;
  if (precision != BEM_PREC_BF16X3 && precision != BEM_PREC_BF16 && precision != BEM_PREC_FP16X3)
    return BEM_ERR_INVALID_ARGUMENT;
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
  int rc = tc_error(ws, &err, (cudaStream_t)stream, true);
  if (rc) return rc;
  return err ? BEM_ERR_CUDA : BEM_OK;
}

// Boundary-to-listener evaluation and triangle -> vertex averaging.
//
// Reference: src/bem/cuda/bind.cu:156-176 (explicit P x N potential matrix,
// one block per listener, 3 scalar atomics per (listener, triangle)),
// integrand.h:237-255,396-406 (6-point rule, target normal 0, trial normal),
// src/bem/solver.py:128-147 (matrix times vector), bind.cu:23-48
// (triangle2vertex).
//
// B200 design: `boundary2potential` never materialises the P x N matrices.
// The P1 densities are first interpolated onto the 6T quadrature points
// (one small pass), after which the listener sum is a dense, atomic-free
// "N-body" contraction: each lane owns a listener, warps stream quadrature
// points, and S and D share one distance and one sincos.

#include "bem_common.cuh"

namespace bemb {

int geom_view(const void* geom, GeomView* v, GeomHeader* out_hdr);

namespace {

// Explicit potential matrix: thread = (listener p, triangle j).
template <int LAYER>
__global__ void potential_matrix_kernel(GeomView g, const float* __restrict__ pts, int np, float k,
                                        float2* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = blockIdx.y;
  if (j >= g.nt || p >= np) return;
  const TriRec& r = g.rec_orig[j];
  const float px = pts[3 * p], py = pts[3 * p + 1], pz = pts[3 * p + 2];
  float2 acc[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const float dx = r.qp[3 * q] - px, dy = r.qp[3 * q + 1] - py, dz = r.qp[3 * q + 2] - pz;
    float rr = sqrtf(dx * dx + dy * dy + dz * dz);
    rr = fmaxf(rr, kEps);
    float s, c;
    sincosf(k * rr, &s, &c);
    float gr, gi;
    if (LAYER == BEM_SINGLE_LAYER) {
      gr = c / rr;
      gi = s / rr;
    } else {
      const float dn = dx * r.n[0] + dy * r.n[1] + dz * r.n[2];  // (y - x) . n_y
      const float f = -dn / (rr * rr * rr);
      const float kr = k * rr;
      gr = (c + kr * s) * f;
      gi = (s - kr * c) * f;
    }
#pragma unroll
    for (int b = 0; b < 3; b++) {
      const float w = (float)(tri6_w(q) * tri6_phi(q, b));
      acc[b].x = fmaf(w, gr, acc[b].x);
      acc[b].y = fmaf(w, gi, acc[b].y);
    }
  }
  const float sc = r.area * kInv4Pi;
#pragma unroll
  for (int b = 0; b < 3; b++)
    atomicAdd(&out[(size_t)p * g.nv + r.v[b]], make_float2(acc[b].x * sc, acc[b].y * sc));
}

// Densities on quadrature points: dens[(6 j + q) * nrhs + s] =
//   area_j w_q sum_b phi_b(q) u[v_b(j), s]   for u = neumann (slot 0) and dirichlet (slot 1).
__global__ void b2p_density_kernel(GeomView g, const float2* __restrict__ neu, const float2* __restrict__ dir,
                                   int nrhs, float2* __restrict__ dn_out, float2* __restrict__ dd_out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)g.nt * 6 * nrhs;
  if (idx >= total) return;
  const int s = (int)(idx % nrhs);
  const int jq = (int)(idx / nrhs);
  const int j = jq / 6, q = jq - 6 * (jq / 6);
  const TriRec& r = g.rec_orig[j];
  float2 an = make_float2(0.f, 0.f), ad = make_float2(0.f, 0.f);
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const float f = (float)tri6_phi(q, b);
    if (neu) {
      const float2 u = neu[(size_t)r.v[b] * nrhs + s];
      an.x = fmaf(f, u.x, an.x);
      an.y = fmaf(f, u.y, an.y);
    }
    if (dir) {
      const float2 u = dir[(size_t)r.v[b] * nrhs + s];
      ad.x = fmaf(f, u.x, ad.x);
      ad.y = fmaf(f, u.y, ad.y);
    }
  }
  const float w = (float)tri6_w(q) * r.area * kInv4Pi;
  dn_out[idx] = make_float2(-an.x * w, -an.y * w);  // -S applied to neumann
  dd_out[idx] = make_float2(ad.x * w, ad.y * w);
}

constexpr int kB2PThreads = 256;

// out[p, s] += sum_{jq in chunk} G(x_p, y_jq) dn[jq, s] + D(x_p, y_jq) dd[jq, s]
// (the -1, the weights and 1/(4 pi) are inside dn/dd).  Block = 32 listeners
// (lanes) x one chunk of quadrature points split over 8 warps; kB2PRhs
// right-hand sides per pass (8, or 16 for more than 8 right-hand sides: the
// distances and sin/cos are computed once per pass).
template <int kB2PRhs>
__global__ void __launch_bounds__(kB2PThreads)
    b2p_eval_kernel(GeomView g, const float* __restrict__ pts, int np, float k, const float2* __restrict__ dn,
                    const float2* __restrict__ dd, int nrhs, int rhs0, int chunk, float2* __restrict__ out) {
  __shared__ float2 red[kB2PThreads / 32][32][kB2PRhs];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int p = blockIdx.x * 32 + lane;
  const bool valid = p < np;
  const float px = valid ? pts[3 * p] : 0.f, py = valid ? pts[3 * p + 1] : 0.f, pz = valid ? pts[3 * p + 2] : 0.f;
  const int nq = 6 * g.nt;
  const int q0 = blockIdx.y * chunk, q1 = min(q0 + chunk, nq);
  const int ns = min(kB2PRhs, nrhs - rhs0);
  float2 acc[kB2PRhs];
#pragma unroll
  for (int s = 0; s < kB2PRhs; s++) acc[s] = make_float2(0.f, 0.f);
  for (int jq = q0 + warp; jq < q1; jq += kB2PThreads / 32) {
    const int j = jq / 6, q = jq - 6 * j;
    const TriRec& r = g.rec_orig[j];
    const float dx = r.qp[3 * q] - px, dy = r.qp[3 * q + 1] - py, dz = r.qp[3 * q + 2] - pz;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float rinv = fminf(rsqrtf(r2), 1.0f / kEps);
    const float rr = fmaxf(r2 * rinv, kEps);
    // hardware sin/cos: the FP32 phase k r carries a relative error of ~2^-24,
    // which the hardware evaluation keeps (a few 1e-6 rad at k r ~ 100)
    float sn, cs;
    __sincosf(k * rr, &sn, &cs);
    const float gr = cs * rinv, gi = sn * rinv;
    const float dnv = dx * r.n[0] + dy * r.n[1] + dz * r.n[2];
    const float f = -dnv * rinv * rinv;
    const float kr = k * rr;
    const float dr = (cs + kr * sn) * rinv * f, di = (sn - kr * cs) * rinv * f;
    const float2* pn = dn + (size_t)jq * nrhs + rhs0;
    const float2* pd = dd + (size_t)jq * nrhs + rhs0;
#pragma unroll
    for (int s = 0; s < kB2PRhs; s++) {
      if (s < ns) {
        const float2 a = pn[s], b = pd[s];
        acc[s].x += gr * a.x - gi * a.y + dr * b.x - di * b.y;
        acc[s].y += gr * a.y + gi * a.x + dr * b.y + di * b.x;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < kB2PRhs; s++) red[warp][lane][s] = acc[s];
  __syncthreads();
  if (warp == 0 && valid) {
    for (int s = 0; s < ns; s++) {
      float2 t = make_float2(0.f, 0.f);
#pragma unroll
      for (int w = 0; w < kB2PThreads / 32; w++) {
        t.x += red[w][lane][s].x;
        t.y += red[w][lane][s].y;
      }
      atomicAdd(&out[(size_t)p * nrhs + rhs0 + s], t);
    }
  }
}

__global__ void t2v_scatter_kernel(GeomView g, const float2* __restrict__ tv, float2* __restrict__ out,
                                   int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nt) return;
  const float2 v = tv[i];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int vid = g.triangles[3 * i + a];
    atomicAdd(&out[vid], v);
    atomicAdd(&cnt[vid], 1);
  }
}

__global__ void t2v_divide_kernel(int nv, float2* __restrict__ out, const int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  // an isolated vertex gives 0/0 = NaN, as in the reference (bind.cu:46)
  const float c = (float)cnt[i];
  out[i] = make_float2(out[i].x / c, out[i].y / c);
}

}  // namespace

}  // namespace bemb

using namespace bemb;

extern "C" int bem_potential_matrix(const void* geom, int layer, const float* points, int np, float k, void* out,
                                    bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (np < 0 || (np > 0 && (!points || !out))) return BEM_ERR_INVALID_ARGUMENT;
  if (layer != BEM_SINGLE_LAYER && layer != BEM_DOUBLE_LAYER) return BEM_ERR_UNSUPPORTED;
  if (np == 0) return BEM_OK;
  cudaStream_t s = (cudaStream_t)stream;
  BEM_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * (size_t)np * g.nv, s));
  dim3 grid((g.nt + 127) / 128, np);
  if (layer == BEM_SINGLE_LAYER)
    (potential_matrix_kernel<BEM_SINGLE_LAYER><<<grid, 128, 0, s>>>(g, points, np, k, (float2*)out), count_launch());
  else
    (potential_matrix_kernel<BEM_DOUBLE_LAYER><<<grid, 128, 0, s>>>(g, points, np, k, (float2*)out), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

extern "C" size_t bem_boundary2potential_scratch_bytes(int nt, int nrhs) {
  if (nt <= 0 || nrhs <= 0) return 0;
  return 2 * sizeof(float2) * (size_t)nt * 6 * (size_t)nrhs;
}

namespace bemb {
// The densities of both layers at every quadrature point (into dn, dd: 6 nt
// nrhs complex64 each), then the listener sums: the work of
// bem_boundary2potential and bem_boundary2potential_noalloc, which differ
// only in where dn and dd live.
int b2p_enqueue(const GeomView& g, const float* points, int np, float k, const void* neumann, const void* dirichlet,
                int nrhs, void* out, float2* dn, float2* dd, cudaStream_t s) {
  const long long total = (long long)g.nt * 6 * nrhs;
  (b2p_density_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(g, (const float2*)neumann,
                                                                      (const float2*)dirichlet, nrhs, dn, dd),
   count_launch());
  BEM_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * (size_t)np * nrhs, s));
  const int nq = 6 * g.nt;
  const int ptiles = (np + 31) / 32;
  // enough quadrature chunks to fill the GPU ~4 times
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int nchunks = (4 * sms * 4 + ptiles - 1) / ptiles;
  int chunk = (nq + nchunks - 1) / nchunks;
  chunk = chunk < 256 ? 256 : chunk;
  nchunks = (nq + chunk - 1) / chunk;
  if (nrhs <= 8) {
    (b2p_eval_kernel<8><<<dim3(ptiles, nchunks), kB2PThreads, 0, s>>>(g, points, np, k, dn, dd, nrhs, 0, chunk,
                                                                      (float2*)out), count_launch());
  } else {
    for (int r0 = 0; r0 < nrhs; r0 += 16)
      (b2p_eval_kernel<16><<<dim3(ptiles, nchunks), kB2PThreads, 0, s>>>(g, points, np, k, dn, dd, nrhs, r0, chunk,
                                                                         (float2*)out), count_launch());
  }
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}
}  // namespace bemb

extern "C" int bem_boundary2potential(const void* geom, const float* points, int np, float k, const void* neumann,
                                      const void* dirichlet, int nrhs, void* out, void* scratch, size_t scratch_bytes,
                                      bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (np < 0 || nrhs <= 0 || (np > 0 && (!points || !out))) return BEM_ERR_INVALID_ARGUMENT;
  if (np == 0) return BEM_OK;
  if (!scratch || scratch_bytes < bem_boundary2potential_scratch_bytes(g.nt, nrhs)) return BEM_ERR_WORKSPACE;
  float2* dn = (float2*)scratch;
  float2* dd = dn + (size_t)g.nt * 6 * nrhs;
  return b2p_enqueue(g, points, np, k, neumann, dirichlet, nrhs, out, dn, dd, (cudaStream_t)stream);
}

extern "C" int bem_triangle2vertex(const void* geom, const void* tri_values, void* out, int* counts,
                                   bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (!tri_values || !out || !counts) return BEM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  BEM_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * (size_t)g.nv, s));
  BEM_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)g.nv, s));
  (t2v_scatter_kernel<<<(g.nt + 255) / 256, 256, 0, s>>>(g, (const float2*)tri_values, (float2*)out, counts), count_launch());
  (t2v_divide_kernel<<<(g.nv + 255) / 256, 256, 0, s>>>(g.nv, (float2*)out, counts), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// Listener evaluation for callers that cannot allocate device memory.
//
// Some hosts of this library never call cudaMalloc while they run: real-time
// audio or rendering loops that synthesise sound from listener pressures
// must not block on the allocator (an allocation may synchronise the device
// and miss the callback deadline), and plug-ins embedded through a plain C
// FFI often have no device allocator of their own.  This entry point is the
// same computation as bem_boundary2potential, with the quadrature-point
// densities kept in a fixed array of this library's own device memory
// instead of a caller-provided scratch buffer.
//
// Contract:
//  * the array holds 2 x kNoAllocQuadRhs complex64 values (16 MiB); every GPU
//    that loads the library reserves it until the process exits;
//  * requests with 6 * nt * nrhs > kNoAllocQuadRhs are rejected with
//    BEM_ERR_WORKSPACE before any work is enqueued;
//  * the first call on a device, with that device current, looks up the
//    array's device address (cudaGetSymbolAddress) and caches it; make that
//    first call before any stream capture;
//  * all calls share the array and it keeps the last call's contents: each
//    call overwrites every density it reads before reading it, so nothing
//    needs clearing, but calls that overlap on the GPU (different streams,
//    or different host threads) race on it and must be serialised by the
//    caller;
//  * no cudaMalloc, cudaFree or allocating library routine is called.
// ---------------------------------------------------------------------------
#include <mutex>

namespace bemb {
namespace {
constexpr long long kNoAllocQuadRhs = 1LL << 20;
static __device__ __align__(256) float2 g_noalloc_density[2 * kNoAllocQuadRhs];
std::mutex g_noalloc_mu;
constexpr int kNoAllocMaxDevices = 64;
float2* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_density on the current device (set-up once per
// device; the name itself is only a host-side handle for the symbol).
int noalloc_density(float2** out) {
  int dev = 0;
  BEM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return BEM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_density);
    if (e != cudaSuccess || !p) return BEM_ERR_CUDA;
    g_noalloc_addr[dev] = (float2*)p;
  }
  *out = g_noalloc_addr[dev];
  return BEM_OK;
}
}  // namespace
}  // namespace bemb

extern "C" long long bem_boundary2potential_noalloc_max(void) { return bemb::kNoAllocQuadRhs; }

extern "C" int bem_boundary2potential_noalloc(const void* geom, const float* points, int np, float k,
                                              const void* neumann, const void* dirichlet, int nrhs, void* out,
                                              bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (np < 0 || nrhs <= 0 || (np > 0 && (!points || !out))) return BEM_ERR_INVALID_ARGUMENT;
  if ((long long)6 * g.nt * nrhs > kNoAllocQuadRhs) return BEM_ERR_WORKSPACE;
  if (np == 0) return BEM_OK;
  float2* base = nullptr;
  if ((rc = noalloc_density(&base))) return rc;
  return b2p_enqueue(g, points, np, k, neumann, dirichlet, nrhs, out, base, base + kNoAllocQuadRhs,
                     (cudaStream_t)stream);
}

// Dense Galerkin assembly of the Helmholtz single-layer (V) and double-layer
// (K) matrices in the P1 vertex basis, plus the P1 mass matrix.
//
// Reference behaviour (file:line inside the NeuralAT project):
//   regular pairs     src/bem/cuda/bind.cu:67-79, integrand.h:187-235,280-329
//   singular pairs    src/bem/cuda/bind.cu:81-152, integrand.h:63-185,331-394
//   kernels           src/bem/cuda/include/potential.h:18-32 (r >= 1e-3 clamp)
//   mass matrix       src/bem/cuda/bind.cu:10-21, integrand.h:257-278
//
// Design (B200): the reference launches one block per test triangle, sweeps
// every trial triangle with one thread each, recomputes r and exp(ikr)
// separately for V and for K, and scatters 18 float atomics per pair into the
// N x N matrix.  Here:
//   * one pass evaluates each quadrature-point pair once for BOTH operators
//     (shared r, rsqrt and sincos), with the 6-point rule's constant weights
//     folded into immediate FMA operands;
//   * V and K together (regular_sym_kernel): each unordered pair once, a
//     CTA owns one 16-triangle test tile (lane & 15) and sweeps the trial
//     tiles at or after it, two trial triangles per warp, tiles
//     double-buffered by bulk copies, two CTAs per SM; one operator alone
//     (regular_vk_kernel): a CTA owns 32 test triangles (one per lane) x one
//     16-triangle trial tile, the 8 warps broadcasting their trial triangles
//     from shared memory;
//   * pair blocks go to a shared-memory "corner" slab (test corner x trial
//     corner) and are reduced on chip onto the tile's distinct vertices, so
//     each matrix entry receives ~0.8 vector atomics per triangle pair instead
//     of the reference's 18 scalar atomics;
//   * touching pairs are masked out of the regular pass and integrated by
//     separate Sauter-Schwab kernels (coincident pairs in FP64), one warp per
//     pair over a precomputed pair list (no O(T^2) adjacency scan).

#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "async_copy.cuh"
#include "bem_common.cuh"

namespace bemb {

int geom_view(const void* geom, GeomView* v, GeomHeader* out_hdr);

extern int g_tc_promote;    // tensor-core matvec accumulator segment (tc_matvec.cu)
extern int g_gmres_reorth;  // Gram-Schmidt passes of the Arnoldi step (linalg.cu)
extern int g_arn_max_cluster;  // largest Arnoldi cluster size (linalg.cu)
extern int g_arn_mode;         // Arnoldi step variant (linalg.cu)
extern int g_gmres_block;      // block Krylov space for several right-hand sides (linalg.cu)
extern int g_tc_wait_us;       // bounded-wait limit of the tensor-core kernels (tc_matvec.cu)
extern std::atomic<int> g_tc_skip_fill;  // test hook of the tensor-core kernel (tc_matvec.cu)

namespace {
extern int g_tune_chunk;
extern int g_tune_ctas_per_sm;
}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Regular triangle pairs.
// ---------------------------------------------------------------------------
constexpr int kRegThreads = 256;
constexpr int kRegWarps = kRegThreads / 32;
constexpr int kTestTris = 32;                  // one test triangle per lane
constexpr int kTestCorners = 3 * kTestTris;     // 96
constexpr int kSlotStride = kTileCorners + 1;   // 49 float2: conflict-free column writes

template <bool DO_V, bool DO_K>
struct RegSmem {
  float2 slotV[DO_V ? kTestCorners : 1][kSlotStride];
  float2 slotK[DO_K ? kTestCorners : 1][kSlotStride];
  TriRec trial[kTile];
  TileRec tileJ;
  TileRec tileI[2];
};

// 3x3 P1 blocks of one (test, trial) pair under the 6x6 point rule:
//   aV[3a+b] = sum_pq C_ap C_bq e^{ikr}/r,
//   aK[3a+b] = sum_pq C_ap C_bq dn_p (c + kr s + i(s - kr c)) / r^3,
// with C_aq = w_q phi_a(q), dn_p = n_j . (y - x_p) (constant over the trial
// plane), r clamped to >= 1e-3 (potential.h:21-23).  The 1/(4 pi), the
// areas and the double layer's minus sign are applied by the caller.
template <bool DO_V, bool DO_K>
__device__ __forceinline__ void pair_block(const float (&xq)[18], const float (&yq)[18], float njx, float njy,
                                           float njz, float cjx, float cjy, float cjz, float k, float2 (&aV)[9],
                                           float2 (&aK)[9]) {
#pragma unroll
  for (int e = 0; e < 9; e++) {
    aV[e] = make_float2(0.f, 0.f);
    aK[e] = make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int p = 0; p < 6; p++) {
    const float px = xq[3 * p], py = xq[3 * p + 1], pz = xq[3 * p + 2];
    const float dn = njx * (cjx - px) + njy * (cjy - py) + njz * (cjz - pz);
    float2 tV[3], tK[3];
#pragma unroll
    for (int b = 0; b < 3; b++) {
      tV[b] = make_float2(0.f, 0.f);
      tK[b] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const float dx = yq[3 * q] - px, dy = yq[3 * q + 1] - py, dz = yq[3 * q + 2] - pz;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const float rinv = fminf(rsqrtf(r2), 1.0f / kEps);
      const float r = fmaxf(r2 * rinv, kEps);
      float s, c;
      __sincosf(k * r, &s, &c);
      const float gvr = c * rinv, gvi = s * rinv;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        const float w = (float)(tri6_w(q) * tri6_phi(q, b));
        if (DO_V) {
          tV[b].x = fmaf(w, gvr, tV[b].x);
          tV[b].y = fmaf(w, gvi, tV[b].y);
        }
      }
      if (DO_K) {
        const float rinv2 = rinv * rinv;
        const float gkr = fmaf(k, s, gvr) * rinv2;   // (c + kr s) / r^3
        const float gki = fmaf(-k, c, gvi) * rinv2;  // (s - kr c) / r^3
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const float w = (float)(tri6_w(q) * tri6_phi(q, b));
          tK[b].x = fmaf(w, gkr, tK[b].x);
          tK[b].y = fmaf(w, gki, tK[b].y);
        }
      }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float wa = (float)(tri6_w(p) * tri6_phi(p, a));
      const float wk = wa * dn;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        if (DO_V) {
          aV[3 * a + b].x = fmaf(wa, tV[b].x, aV[3 * a + b].x);
          aV[3 * a + b].y = fmaf(wa, tV[b].y, aV[3 * a + b].y);
        }
        if (DO_K) {
          aK[3 * a + b].x = fmaf(wk, tK[b].x, aK[3 * a + b].x);
          aK[3 * a + b].y = fmaf(wk, tK[b].y, aK[3 * a + b].y);
        }
      }
    }
  }
}

__device__ __forceinline__ void copy_words(void* dst, const void* src, int bytes, int tid, int nthreads) {
  const int4* s = (const int4*)src;
  int4* d = (int4*)dst;
  for (int i = tid; i < bytes / 16; i += nthreads) d[i] = s[i];
}

// Work item = (group of 32 test triangles = 2 tiles) x (chunk of `chunk`
// trial tiles).  Items are dealt round-robin to a persistent grid.
// One work item: test group `grp` (32 triangles = 2 tiles) against the trial
// tiles [ch * chunk, ch * chunk + chunk).
template <bool DO_V, bool DO_K>
__device__ __forceinline__ void regular_item(RegSmem<DO_V, DO_K>& sm, const GeomView& g, float k,
                                             float2* __restrict__ V, float2* __restrict__ K, float v_scale,
                                             float k_scale, int grp, int ch, int chunk) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nt = g.nt, nv = g.nv;
  {
    const int tile0 = 2 * grp;
    const bool has_t1 = tile0 + 1 < g.ntiles;

    // test triangle of this lane (all warps hold the same 32)
    const int ti = grp * kTestTris + lane;
    const bool valid_i = ti < nt;
    const TriRec& ri = g.rec[valid_i ? ti : nt - 1];
    float xq[18];
#pragma unroll
    for (int e = 0; e < 18; e++) xq[e] = ri.qp[e];
    const float area_i = ri.area;
    const int iv0 = ri.v[0], iv1 = ri.v[1], iv2 = ri.v[2];

    __syncthreads();  // previous item's gather has finished with tileI
    copy_words(&sm.tileI[0], &g.tiles[tile0], sizeof(TileRec), tid, kRegThreads);
    if (has_t1) copy_words(&sm.tileI[1], &g.tiles[tile0 + 1], sizeof(TileRec), tid, kRegThreads);

    const int jt_begin = ch * chunk;
    const int jt_end = min(jt_begin + chunk, g.ntiles);
    for (int jt = jt_begin; jt < jt_end; jt++) {
      __syncthreads();  // gather of the previous trial tile is done with the slots
      copy_words(&sm.tileJ, &g.tiles[jt], sizeof(TileRec), tid, kRegThreads);
      const int ntriJ = min(kTile, nt - jt * kTile);
      copy_words(sm.trial, &g.rec[jt * kTile], ntriJ * (int)sizeof(TriRec), tid, kRegThreads);
      __syncthreads();

      // ---- compute: each warp takes trial triangles warp and warp + 8 ----
#pragma unroll 1
      for (int tt = warp; tt < ntriJ; tt += kRegWarps) {
        const TriRec& rj = sm.trial[tt];
        float yq[18];
#pragma unroll
        for (int e = 0; e < 18; e++) yq[e] = rj.qp[e];
        float2 aV[9], aK[9];
        pair_block<DO_V, DO_K>(xq, yq, rj.n[0], rj.n[1], rj.n[2], rj.c[0], rj.c[1], rj.c[2], k, aV, aK);
        const int j0 = rj.v[0], j1 = rj.v[1], j2 = rj.v[2];
        const bool touching = (iv0 == j0) | (iv0 == j1) | (iv0 == j2) | (iv1 == j0) | (iv1 == j1) | (iv1 == j2) |
                              (iv2 == j0) | (iv2 == j1) | (iv2 == j2);
        const float aa = (valid_i && !touching) ? area_i * rj.area : 0.f;
        const float sv = aa * v_scale, sk = aa * k_scale;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++) {
            if (DO_V) sm.slotV[3 * lane + a][3 * tt + b] = make_float2(aV[3 * a + b].x * sv, aV[3 * a + b].y * sv);
            if (DO_K) sm.slotK[3 * lane + a][3 * tt + b] = make_float2(aK[3 * a + b].x * sk, aK[3 * a + b].y * sk);
          }
      }
      __syncthreads();

      // ---- reduce corner slots onto distinct vertices, one atomic per entry ----
      // Pass 1, in place: for every trial corner column, the row of test
      // vertex A's first corner gets the sum over A's test corners (corner
      // rows of different vertices are disjoint); pass 2: entry (A, B) sums
      // B's trial corners along that row.
      const int nI0 = sm.tileI[0].nlv;
      const int nI1 = has_t1 ? sm.tileI[1].nlv : 0;
      const int nJ = sm.tileJ.nlv;
      const int ncol = 3 * ntriJ;
      const float rcol = 1.f / (float)ncol, rJ = 1.f / (float)(nJ > 0 ? nJ : 1);
      for (int e = tid; e < (nI0 + nI1) * ncol; e += kRegThreads) {
        const int ai = div_by(e, ncol, rcol);
        const int col = e - ai * ncol;
        const int s = ai >= nI0;
        const int a = ai - s * nI0;
        const TileRec& TI = sm.tileI[s];
        const int ca0 = TI.lv_ptr[a], ca1 = TI.lv_ptr[a + 1];
        const int rep = s * kTileCorners + TI.lv_corner[ca0];
        float2 v = make_float2(0.f, 0.f), kk = make_float2(0.f, 0.f);
        if (DO_V) v = sm.slotV[rep][col];
        if (DO_K) kk = sm.slotK[rep][col];
        for (int ca = ca0 + 1; ca < ca1; ca++) {
          const int row = s * kTileCorners + TI.lv_corner[ca];
          if (DO_V) {
            v.x += sm.slotV[row][col].x;
            v.y += sm.slotV[row][col].y;
          }
          if (DO_K) {
            kk.x += sm.slotK[row][col].x;
            kk.y += sm.slotK[row][col].y;
          }
        }
        if (DO_V) sm.slotV[rep][col] = v;
        if (DO_K) sm.slotK[rep][col] = kk;
      }
      __syncthreads();
      for (int e = tid; e < (nI0 + nI1) * nJ; e += kRegThreads) {
        const int ai = div_by(e, nJ, rJ);
        const int b = e - ai * nJ;
        const int s = ai >= nI0;
        const int a = ai - s * nI0;
        const TileRec& TI = sm.tileI[s];
        const int rep = s * kTileCorners + TI.lv_corner[TI.lv_ptr[a]];
        float2 acc_v = make_float2(0.f, 0.f), acc_k = make_float2(0.f, 0.f);
        const int cb0 = sm.tileJ.lv_ptr[b], cb1 = sm.tileJ.lv_ptr[b + 1];
        for (int cb = cb0; cb < cb1; cb++) {
          const int col = sm.tileJ.lv_corner[cb];
          if (DO_V) {
            acc_v.x += sm.slotV[rep][col].x;
            acc_v.y += sm.slotV[rep][col].y;
          }
          if (DO_K) {
            acc_k.x += sm.slotK[rep][col].x;
            acc_k.y += sm.slotK[rep][col].y;
          }
        }
        const size_t idx = (size_t)TI.vid[a] * nv + sm.tileJ.vid[b];
        if (DO_V) atomicAdd(&V[idx], acc_v);
        if (DO_K) atomicAdd(&K[idx], acc_k);
      }
    }
  }
}

// Single problem: items dealt round-robin to a persistent grid.
template <bool DO_V, bool DO_K>
__global__ void __launch_bounds__(kRegThreads, 2)
    regular_vk_kernel(GeomView g, float k, float2* __restrict__ V, float2* __restrict__ K, float v_scale,
                      float k_scale, int chunk, int n_chunks, int n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RegSmem<DO_V, DO_K>& sm = *reinterpret_cast<RegSmem<DO_V, DO_K>*>(smem_raw);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int grp = item / n_chunks;
    regular_item<DO_V, DO_K>(sm, g, k, V, K, v_scale, k_scale, grp, item - grp * n_chunks, chunk);
  }
}

// ---------------------------------------------------------------------------
// Symmetric evaluation of the regular pairs (V and K together).  G(|x - y|)
// is symmetric, so each unordered non-touching pair {i, j} is evaluated once
// and scattered both ways:
//   V_ji = V_ij^T,
//   K_ij uses the trial plane of j (dn_j(p) = n_j . (c_j - x_p)),
//   K_ji uses the plane of i at the trial points (dn_i(q) = n_i . (c_i - y_q)),
// both from the same r, sincos and kernel values.  A work item is one test
// tile (16 triangles, test triangle = lane & 15) against a chunk of trial
// tiles at or after it; on the test tile itself only pairs j > i.  Each of
// the 8 warps takes two trial triangles (one per half-warp); the test points
// are staged structure-of-arrays in shared memory.  The slabs fit two CTAs
// per SM, so one CTA's reduction and barriers overlap the other's evaluation.
// ---------------------------------------------------------------------------
constexpr int kSymThreads = 16 * kTile;         // 256: warp w takes trial triangles 2w, 2w + 1
constexpr int kSymTest = kTile;                 // test triangles per CTA (one tile)
constexpr int kSymCorners = 3 * kSymTest;       // 48

struct SymSmem {
  float2 slotV[kSymCorners][kSlotStride];
  float2 slotK[kSymCorners][kSlotStride];
  float2 slotM[kSymCorners][kSlotStride];  // K_ji^T, indexed like slotK
  float xs[18][kSymTest];                  // test quadrature points, [coordinate][tl]
  TriRec trial[2][kTile];                  // trial tile records, double-buffered
  TileRec tileJ[2];
  TileRec tileI;
  uint64_t tile_full[2];                   // bulk-copy completion of each trial buffer
};

// A bounded wait of the assembly kernels expired somewhere in this process
// (read and cleared by bem_assembly_status).  The waits themselves check the
// status word of the geometry they assemble (GeomView::err), so an expiry on
// one geometry does not affect assemblies of other geometries.
__device__ int g_asm_err;

// Thread 0: bulk-copy trial tile jt (records and vertex table) into buffer b.
__device__ __forceinline__ void sym_fetch_tile(SymSmem& sm, const GeomView& g, int jt, int b) {
  const int ntri = min(kTile, g.nt - jt * kTile);
  const uint32_t rec_bytes = (uint32_t)(ntri * sizeof(TriRec));
  mbar_expect_tx(&sm.tile_full[b], rec_bytes + (uint32_t)sizeof(TileRec));
  bulk_load(sm.trial[b], &g.rec[jt * kTile], rec_bytes, &sm.tile_full[b]);
  bulk_load(&sm.tileJ[b], &g.tiles[jt], (uint32_t)sizeof(TileRec), &sm.tile_full[b]);
}

// aV, aK as pair_block; aM[3a+b] = sum_pq C_ap C_bq dn_i(q) Gk(r_pq) = K_ji[b][a].
// The arithmetic runs on packed FP32 pairs: the complex accumulations as
// (re, im) pairs and the distance computation for two trial points at once,
// with the same operations and rounding as the scalar form (bit-identical),
// in about half the issued instructions; rsqrt and sin/cos stay scalar.
__device__ __forceinline__ void pair_block_sym(const float (*xs)[kSymTest], int tl, const float (&yq)[18],
                                               const float (&dq)[6], float njx, float njy, float njz, float cjx,
                                               float cjy, float cjz, float k, float2 (&aV)[9], float2 (&aK)[9],
                                               float2 (&aM)[9]) {
#pragma unroll
  for (int e = 0; e < 9; e++) {
    aV[e] = make_float2(0.f, 0.f);
    aK[e] = make_float2(0.f, 0.f);
    aM[e] = make_float2(0.f, 0.f);
  }
  // trial points in pairs (2h, 2h + 1), one float2 per coordinate
  float2 Yx[3], Yy[3], Yz[3];
#pragma unroll
  for (int h = 0; h < 3; h++) {
    Yx[h] = make_float2(yq[6 * h], yq[6 * h + 3]);
    Yy[h] = make_float2(yq[6 * h + 1], yq[6 * h + 4]);
    Yz[h] = make_float2(yq[6 * h + 2], yq[6 * h + 5]);
  }
  const float2 kk = make_float2(k, -k);
#pragma unroll
  for (int p = 0; p < 6; p++) {
    const float px = xs[3 * p][tl], py = xs[3 * p + 1][tl], pz = xs[3 * p + 2][tl];
    const float dn = njx * (cjx - px) + njy * (cjy - py) + njz * (cjz - pz);
    // the rule is symmetric: phi_b(q) = a_q + (1 - 3 a_q) [b = own vertex of
    // q], so each point adds its own-vertex excess to one trial sum and its
    // common weight to c*, which all three sums receive at the end
    float2 tV[3], tK[3], uK[3];
    float2 cV = make_float2(0.f, 0.f), cK = cV, cU = cV;
#pragma unroll
    for (int b = 0; b < 3; b++) {
      tV[b] = make_float2(0.f, 0.f);
      tK[b] = make_float2(0.f, 0.f);
      uK[b] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int h = 0; h < 3; h++) {
      const float2 dx = f2_sub(Yx[h], f2(px)), dy = f2_sub(Yy[h], f2(py)), dz = f2_sub(Yz[h], f2(pz));
      const float2 r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
      const float2 rinv = make_float2(fminf(rsqrtf(r2.x), 1.0f / kEps), fminf(rsqrtf(r2.y), 1.0f / kEps));
      float2 r = f2_mul(r2, rinv);
      r.x = fmaxf(r.x, kEps);
      r.y = fmaxf(r.y, kEps);
      const float2 kr = f2_mul(f2(k), r);
      const float2 rinv2 = f2_mul(rinv, rinv);
      float sc[2][2];  // [point][sin, cos]
      __sincosf(kr.x, &sc[0][0], &sc[0][1]);
      __sincosf(kr.y, &sc[1][0], &sc[1][1]);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int q = 2 * h + j;
        const float ri = j == 0 ? rinv.x : rinv.y, ri2 = j == 0 ? rinv2.x : rinv2.y;
        const float2 gv = f2_mul(make_float2(sc[j][1], sc[j][0]), f2(ri));                  // (c, s) / r
        const float2 gk = f2_mul(f2_fma(kk, make_float2(sc[j][0], sc[j][1]), gv), f2(ri2));  // (c + kr s, s - kr c) / r^3
        const float2 mk = f2_mul(f2(dq[q]), gk);
        const int b = tri6_own(q);
        const float2 wo = f2((float)tri6_w_own(q)), wc = f2((float)tri6_w_common(q));
        tV[b] = f2_fma(wo, gv, tV[b]);
        tK[b] = f2_fma(wo, gk, tK[b]);
        uK[b] = f2_fma(wo, mk, uK[b]);
        cV = f2_fma(wc, gv, cV);
        cK = f2_fma(wc, gk, cK);
        cU = f2_fma(wc, mk, cU);
      }
    }
#pragma unroll
    for (int b = 0; b < 3; b++) {
      tV[b] = f2_fma(f2(1.f), cV, tV[b]);
      tK[b] = f2_fma(f2(1.f), cK, tK[b]);
      uK[b] = f2_fma(f2(1.f), cU, uK[b]);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float wa = (float)(tri6_w(p) * tri6_phi(p, a));
      const float2 wa2 = f2(wa), wk2 = f2(wa * dn);
#pragma unroll
      for (int b = 0; b < 3; b++) {
        aV[3 * a + b] = f2_fma(wa2, tV[b], aV[3 * a + b]);
        aK[3 * a + b] = f2_fma(wk2, tK[b], aK[3 * a + b]);
        aM[3 * a + b] = f2_fma(wa2, uK[b], aM[3 * a + b]);
      }
    }
  }
}

// `uses` counts the trial tiles this CTA has processed (buffer = uses & 1,
// mbarrier parity = (uses >> 1) & 1).
__device__ __forceinline__ void regular_sym_item(SymSmem& sm, const GeomView& g, float k, float2* __restrict__ V,
                                                 float2* __restrict__ K, float v_scale, float k_scale, int grp,
                                                 int jt_begin, int jt_end, unsigned& uses) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tl = lane & 15;               // test triangle of this lane
  const int tt = 2 * warp + (lane >> 4);  // trial triangle of this half-warp
  const int nt = g.nt, nv = g.nv;
  const int ti = grp * kSymTest + tl;
  const bool valid_i = ti < nt;
  const TriRec& ri = g.rec[valid_i ? ti : nt - 1];
  const float area_i = ri.area;
  const float nix = ri.n[0], niy = ri.n[1], niz = ri.n[2], cix = ri.c[0], ciy = ri.c[1], ciz = ri.c[2];
  const int iv0 = ri.v[0], iv1 = ri.v[1], iv2 = ri.v[2];

  __syncthreads();  // the previous item is done with tileI, xs and both trial buffers
  if (tid == 0) sym_fetch_tile(sm, g, jt_begin, uses & 1);
  copy_words(&sm.tileI, &g.tiles[grp], sizeof(TileRec), tid, kSymThreads);
  for (int e = tid; e < 18 * kSymTest; e += kSymThreads) {
    const int c = e / kSymTest, l = e - c * kSymTest;
    const int t = min(grp * kSymTest + l, nt - 1);
    sm.xs[c][l] = g.rec[t].qp[c];
  }

  for (int jt = jt_begin; jt < jt_end; jt++, uses++) {
    const int bf = uses & 1;
    __syncthreads();  // the previous tile's gather is done with the slots and with buffer bf ^ 1
    if (tid == 0 && jt + 1 < jt_end) sym_fetch_tile(sm, g, jt + 1, bf ^ 1);
    if (!mbar_wait(&sm.tile_full[bf], (uses >> 1) & 1u, g.err)) {
      // expired (this geometry's status word raised): record it process-wide
      // too, and let the copy land before the buffer is reused
      if (tid == 0) atomicExch(&g_asm_err, 1);
      mbar_wait_drain(&sm.tile_full[bf], (uses >> 1) & 1u);
    }
    const TriRec* trial = sm.trial[bf];
    const TileRec& tileJ = sm.tileJ[bf];
    const int ntriJ = min(kTile, nt - jt * kTile);

    // ---- compute: half-warp h of warp w takes trial triangle 2w + h ----
    const int tj = jt * kTile + tt;
    float aa = 0.f;
    if (tt < ntriJ) {
      const TriRec& rj = trial[tt];
      const int j0 = rj.v[0], j1 = rj.v[1], j2 = rj.v[2];
      const bool touching = (iv0 == j0) | (iv0 == j1) | (iv0 == j2) | (iv1 == j0) | (iv1 == j1) | (iv1 == j2) |
                            (iv2 == j0) | (iv2 == j1) | (iv2 == j2);
      // on the test tile itself each unordered pair once (j > i)
      const bool once = jt > grp || tj > ti;
      aa = (valid_i && !touching && once) ? area_i * rj.area : 0.f;
    }
    const bool any = __any_sync(0xffffffffu, aa != 0.f);  // every lane, before the half-warp branch
    if (tt < ntriJ && any) {
      const TriRec& rj = trial[tt];
      float yq[18];
#pragma unroll
      for (int e = 0; e < 18; e++) yq[e] = rj.qp[e];
      float dq[6];
#pragma unroll
      for (int q = 0; q < 6; q++)
        dq[q] = nix * (cix - yq[3 * q]) + niy * (ciy - yq[3 * q + 1]) + niz * (ciz - yq[3 * q + 2]);
      float2 aV[9], aK[9], aM[9];
      pair_block_sym(sm.xs, tl, yq, dq, rj.n[0], rj.n[1], rj.n[2], rj.c[0], rj.c[1], rj.c[2], k, aV, aK, aM);
      const float sv = aa * v_scale, sk = aa * k_scale;
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          sm.slotV[3 * tl + a][3 * tt + b] = make_float2(aV[3 * a + b].x * sv, aV[3 * a + b].y * sv);
          sm.slotK[3 * tl + a][3 * tt + b] = make_float2(aK[3 * a + b].x * sk, aK[3 * a + b].y * sk);
          sm.slotM[3 * tl + a][3 * tt + b] = make_float2(aM[3 * a + b].x * sk, aM[3 * a + b].y * sk);
        }
    } else if (tt < ntriJ) {
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          sm.slotV[3 * tl + a][3 * tt + b] = make_float2(0.f, 0.f);
          sm.slotK[3 * tl + a][3 * tt + b] = make_float2(0.f, 0.f);
          sm.slotM[3 * tl + a][3 * tt + b] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();

    // ---- reduce corner slots onto distinct vertices: (A, B) and (B, A) ----
    // Pass 1, in place: for every trial corner column, the row of test
    // vertex A's first corner gets the sum over A's test corners (the corner
    // rows of different vertices are disjoint).  Pass 2: entry (A, B) is the
    // sum over B's trial corners along that row.  Short independent chains
    // instead of one (corner x corner) loop per entry.
    const TileRec& TI = sm.tileI;
    const int nI = TI.nlv, nJ = tileJ.nlv;
    const int ncol = 3 * ntriJ;
    const float rcol = 1.f / (float)ncol, rJ = 1.f / (float)(nJ > 0 ? nJ : 1);
    for (int e = tid; e < nI * ncol; e += kSymThreads) {
      const int a = div_by(e, ncol, rcol);
      const int col = e - a * ncol;
      const int ca0 = TI.lv_ptr[a], ca1 = TI.lv_ptr[a + 1];
      const int rep = TI.lv_corner[ca0];
      float2 v = sm.slotV[rep][col], kk = sm.slotK[rep][col], mm = sm.slotM[rep][col];
#pragma unroll 4
      for (int ca = ca0 + 1; ca < ca1; ca++) {
        const int row = TI.lv_corner[ca];
        const float2 v1 = sm.slotV[row][col], k1 = sm.slotK[row][col], m1 = sm.slotM[row][col];
        v.x += v1.x;
        v.y += v1.y;
        kk.x += k1.x;
        kk.y += k1.y;
        mm.x += m1.x;
        mm.y += m1.y;
      }
      sm.slotV[rep][col] = v;
      sm.slotK[rep][col] = kk;
      sm.slotM[rep][col] = mm;
    }
    __syncthreads();
    for (int e = tid; e < nI * nJ; e += kSymThreads) {
      const int a = div_by(e, nJ, rJ);
      const int b = e - a * nJ;
      const int rep = TI.lv_corner[TI.lv_ptr[a]];
      const int cb0 = tileJ.lv_ptr[b], cb1 = tileJ.lv_ptr[b + 1];
      float2 acc_v = make_float2(0.f, 0.f), acc_k = make_float2(0.f, 0.f), acc_m = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int cb = cb0; cb < cb1; cb++) {
        const int col = tileJ.lv_corner[cb];
        const float2 v1 = sm.slotV[rep][col], k1 = sm.slotK[rep][col], m1 = sm.slotM[rep][col];
        acc_v.x += v1.x;
        acc_v.y += v1.y;
        acc_k.x += k1.x;
        acc_k.y += k1.y;
        acc_m.x += m1.x;
        acc_m.y += m1.y;
      }
      const int A = TI.vid[a], B = tileJ.vid[b];
      if (acc_v.x != 0.f || acc_v.y != 0.f || acc_k.x != 0.f || acc_k.y != 0.f || acc_m.x != 0.f ||
          acc_m.y != 0.f) {
        atomicAdd(&V[(size_t)A * nv + B], acc_v);
        atomicAdd(&V[(size_t)B * nv + A], acc_v);
        atomicAdd(&K[(size_t)A * nv + B], acc_k);
        atomicAdd(&K[(size_t)B * nv + A], acc_m);
      }
    }
  }
}

// Splits units [pos, end) of one problem at test-tile boundaries.
__device__ __forceinline__ void regular_sym_units(SymSmem& sm, const GeomView& g, float k, float2* V, float2* K,
                                                  float v_scale, float k_scale, long long pos, long long end,
                                                  unsigned& uses) {
  while (pos < end) {  // uniform over the block
    const int grp = tile_group_of(pos, g.ntiles);
    const long long base = tile_units_before(grp, g.ntiles);
    const long long gend = base + (g.ntiles - grp);
    const long long stop = end < gend ? end : gend;
    const int jt0 = grp + (int)(pos - base);
    regular_sym_item(sm, g, k, V, K, v_scale, k_scale, grp, jt0, jt0 + (int)(stop - pos), uses);
    pos = stop;
  }
}

// The (test tile, trial tile >= it) units in order (tile_units_before).
// Items are equal runs of `chunk` consecutive units (a run crossing a test
// tile is split), dealt round-robin to a persistent grid: every CTA gets the
// same amount of work.
__global__ void __launch_bounds__(kSymThreads, 2)
    regular_sym_kernel(GeomView g, float k, float2* __restrict__ V, float2* __restrict__ K, float v_scale,
                       float k_scale, long long chunk, long long n_units, int n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SymSmem& sm = *reinterpret_cast<SymSmem*>(smem_raw);
  if (threadIdx.x == 0) {
    mbar_init(&sm.tile_full[0], 1);
    mbar_init(&sm.tile_full[1], 1);
    mbar_init_fence();
  }
  unsigned uses = 0;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const long long pos = (long long)item * chunk;
    const long long end = pos + chunk < n_units ? pos + chunk : n_units;
    regular_sym_units(sm, g, k, V, K, v_scale, k_scale, pos, end, uses);
  }
}

// ---------------------------------------------------------------------------
// Singular (touching) pairs: Sauter-Schwab quadrature on the reference
// triangle (0,0),(1,0),(1,1) (integrand.h:54-185), after re-ordering so the
// shared vertices come first (integrand.h:351-387).  One warp per pair; the
// lanes split the 4^4 Gauss-Legendre points; blocks are reduced with
// shuffles and added with one atomic per entry.
// ---------------------------------------------------------------------------

template <typename R>
struct R3 {
  R x, y, z;
};

// Re-ordering of the reference (integrand.h:351-387): for a common edge the
// shared vertices take local slots 0,1 in trial order; for a common vertex it
// is swapped into slot 0 on both triangles.  Kept in scalar registers (no
// runtime-indexed local arrays): p.i[c] / p.j[c] is the original local index
// of re-ordered slot c.
struct Perm {
  int i0, i1, i2, j0, j1, j2;
};

__device__ __forceinline__ int pick3(int a0, int a1, int a2, int idx) { return idx == 0 ? a0 : (idx == 1 ? a1 : a2); }

template <int NCOMMON>
__device__ __forceinline__ Perm reorder_pair(int s0, int s1, int s2, int t0, int t1, int t2) {
  Perm p{0, 1, 2, 0, 1, 2};
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
    p = Perm{mi0, mi1, 3 - mi0 - mi1, mj0, mj1, 3 - mj0 - mj1};
  } else if (NCOMMON == 1) {
    int ci = 0, cj = 0;
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++)
        if (si[ii] == sj[jj]) { ci = ii; cj = jj; }
    p = Perm{ci, ci == 1 ? 0 : 1, ci == 2 ? 0 : 2, cj, cj == 1 ? 0 : 1, cj == 2 ? 0 : 2};
  }
  return p;
}

template <typename R, int NCOMMON, bool DO_V, bool DO_K>
struct SingularAcc {
  R v[18];  // 9 complex, (re, im) pairs, index 3 * test + trial (re-ordered)
  R kk[18];
  R3<R> a[3];  // re-ordered test vertices
  R3<R> b[3];  // re-ordered trial vertices
  R3<R> nj;    // unit normal of the trial triangle
  R k;

  // One Sauter-Schwab region: point (x1, x2) on the test triangle and (y1, y2)
  // on the trial triangle, shape functions (1 - s, s - t, t), weight ww.
  __device__ __forceinline__ void region(R x1, R x2, R y1, R y2, R ww) {
    const R lx0 = R(1) - x1, lx1 = x1 - x2, lx2 = x2;
    const R ly0 = R(1) - y1, ly1 = y1 - y2, ly2 = y2;
    const R xx = lx0 * a[0].x + lx1 * a[1].x + lx2 * a[2].x;
    const R xy = lx0 * a[0].y + lx1 * a[1].y + lx2 * a[2].y;
    const R xz = lx0 * a[0].z + lx1 * a[1].z + lx2 * a[2].z;
    const R yx = ly0 * b[0].x + ly1 * b[1].x + ly2 * b[2].x;
    const R yy = ly0 * b[0].y + ly1 * b[1].y + ly2 * b[2].y;
    const R yz = ly0 * b[0].z + ly1 * b[1].z + ly2 * b[2].z;
    const R dx = yx - xx, dy = yy - xy, dz = yz - xz;
    R r, inv_r;
    inv_dist<R>(dx * dx + dy * dy + dz * dz, &r, &inv_r);
    R s, c;
    const R kr = k * r;
    sincos_t<R>(kr, &s, &c);
    const R gvr = c * inv_r * ww, gvi = s * inv_r * ww;
    R gkr = 0, gki = 0;
    if (DO_K) {
      const R dn = dx * nj.x + dy * nj.y + dz * nj.z;  // (y - x) . n_trial
      const R f = dn * inv_r * inv_r * inv_r * ww;
      gkr = (c + kr * s) * f;
      gki = (s - kr * c) * f;
    }
    const R lx[3] = {lx0, lx1, lx2}, ly[3] = {ly0, ly1, ly2};
    if constexpr (std::is_same<R, float>::value) {
      // packed FP32: (re, im) pairs, the trial weight applied first (3 + 3
      // multiplies, then one packed FMA per entry and kernel)
      float2 gy[3], ky[3];
#pragma unroll
      for (int jj = 0; jj < 3; jj++) {
        gy[jj] = f2_mul(f2(ly[jj]), make_float2(gvr, gvi));
        ky[jj] = f2_mul(f2(ly[jj]), make_float2(gkr, gki));
      }
#pragma unroll
      for (int ii = 0; ii < 3; ii++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          const int e = 3 * ii + jj;
          if (DO_V) {
            const float2 t = f2_fma(f2(lx[ii]), gy[jj], make_float2(v[2 * e], v[2 * e + 1]));
            v[2 * e] = t.x;
            v[2 * e + 1] = t.y;
          }
          if (DO_K) {
            const float2 t = f2_fma(f2(lx[ii]), ky[jj], make_float2(kk[2 * e], kk[2 * e + 1]));
            kk[2 * e] = t.x;
            kk[2 * e + 1] = t.y;
          }
        }
    } else {
#pragma unroll
      for (int ii = 0; ii < 3; ii++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          const R f = lx[ii] * ly[jj];
          if (DO_V) {
            v[2 * (3 * ii + jj)] += gvr * f;
            v[2 * (3 * ii + jj) + 1] += gvi * f;
          }
          if (DO_K) {
            kk[2 * (3 * ii + jj)] += gkr * f;
            kk[2 * (3 * ii + jj) + 1] += gki * f;
          }
        }
    }
  }

  // One 4D Gauss point (xi, e1, e2, e3 on [0,1]) of weight w0; the region
  // Jacobian w (integrand.h:121,134,146) is applied to every region.
  __device__ __forceinline__ void point(R xi, R e1, R e2, R e3, R w0) {
    const R e12 = e1 * e2, e123 = e1 * e2 * e3;
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
};

template <typename R>
__device__ __forceinline__ R warp_sum(R x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// NCOMMON = 3: pairs (i, i), i = pair index; otherwise pairs from the list.
template <typename R, int NCOMMON, bool DO_V, bool DO_K>
__device__ __forceinline__ void singular_pair(const GeomView& g, int ti, int tj, float k, float2* __restrict__ V,
                                              float2* __restrict__ K, float v_scale, float k_scale,
                                              float mass_coeff) {
  const int lane = threadIdx.x & 31;
  const int s0 = g.triangles[3 * ti], s1 = g.triangles[3 * ti + 1], s2 = g.triangles[3 * ti + 2];
  const int t0 = g.triangles[3 * tj], t1 = g.triangles[3 * tj + 1], t2 = g.triangles[3 * tj + 2];
  const Perm pm = reorder_pair<NCOMMON>(s0, s1, s2, t0, t1, t2);
  const int pi_[3] = {pm.i0, pm.i1, pm.i2}, pj_[3] = {pm.j0, pm.j1, pm.j2};
  R3<R> pa[3], pb[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int va = pick3(s0, s1, s2, pi_[c]), vb = pick3(t0, t1, t2, pj_[c]);
    pa[c] = {(R)g.vertices[3 * va], (R)g.vertices[3 * va + 1], (R)g.vertices[3 * va + 2]};
    pb[c] = {(R)g.vertices[3 * vb], (R)g.vertices[3 * vb + 1], (R)g.vertices[3 * vb + 2]};
  }
  const int si[3] = {s0, s1, s2}, sj[3] = {t0, t1, t2};
  // Jacobians and the trial normal of the un-permuted triangles
  auto jac_normal = [](const R3<R>* p, R3<R>* n) {
    const R e1x = p[1].x - p[0].x, e1y = p[1].y - p[0].y, e1z = p[1].z - p[0].z;
    const R e2x = p[2].x - p[0].x, e2y = p[2].y - p[0].y, e2z = p[2].z - p[0].z;
    const R cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
    const R J = sqrt(cx * cx + cy * cy + cz * cz);
    if (n) *n = {cx / J, cy / J, cz / J};
    return J;
  };
  R3<R> oa[3], ob[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    oa[c] = {(R)g.vertices[3 * si[c]], (R)g.vertices[3 * si[c] + 1], (R)g.vertices[3 * si[c] + 2]};
    ob[c] = {(R)g.vertices[3 * sj[c]], (R)g.vertices[3 * sj[c] + 1], (R)g.vertices[3 * sj[c] + 2]};
  }
  R3<R> nj;
  const R Ji = jac_normal(oa, nullptr);
  const R Jj = jac_normal(ob, &nj);

  SingularAcc<R, NCOMMON, DO_V, DO_K> acc;
#pragma unroll
  for (int e = 0; e < 18; e++) {
    acc.v[e] = 0;
    acc.kk[e] = 0;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc.a[c] = pa[c];
    acc.b[c] = pb[c];
  }
  acc.nj = nj;
  acc.k = (R)k;
  const R jw = Ji * Jj / R(16);
#pragma unroll 1
  for (int pt = lane; pt < 256; pt += 32) {
    const int i0 = pt >> 6, i1 = (pt >> 4) & 3, i2 = (pt >> 2) & 3, i3 = pt & 3;
    const R xi = R(0.5) * (R(gl4_x(i0)) + R(1));
    const R e1 = R(0.5) * (R(gl4_x(i1)) + R(1));
    const R e2 = R(0.5) * (R(gl4_x(i2)) + R(1));
    const R e3 = R(0.5) * (R(gl4_x(i3)) + R(1));
    const R w0 = R(gl4_w(i0)) * R(gl4_w(i1)) * R(gl4_w(i2)) * R(gl4_w(i3)) * jw;
    acc.point(xi, e1, e2, e3, w0);
  }
  // reduce: values 0..31 by a transpose-reduce (lane L ends with the warp
  // total of value L), values 32..35 by plain sums; then lane e (< 9) takes
  // V entry e, lane 9 + e K entry e
  constexpr int NV = (DO_V ? 18 : 0) + (DO_K ? 18 : 0);
  R t[32];
#pragma unroll
  for (int i = 0; i < 32; i++) {
    const int vi = i, ki = DO_V ? i - 18 : i;
    t[i] = (DO_V && vi < 18) ? acc.v[vi] : ((DO_K && ki >= 0 && ki < 18) ? acc.kk[ki] : R(0));
  }
  R extra[4] = {R(0), R(0), R(0), R(0)};
  if (NV > 32) {
#pragma unroll
    for (int i = 0; i < 4; i++) extra[i] = warp_sum(acc.kk[14 + i]);
  }
#pragma unroll
  for (int o = 16, half = 16; o >= 1; o >>= 1, half >>= 1) {
    const bool hi = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < half; i++) {
      const R send = hi ? t[i] : t[i + half];
      const R keep = hi ? t[i + half] : t[i];
      t[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  const R mine = t[0];  // warp total of value `lane`
  // value indices of this lane's entry (re, im)
  const int e = lane < 9 ? lane : lane - 9;
  const int base = lane < 9 ? 0 : (DO_V ? 18 : 0);
  const int ire = base + 2 * e, iim = ire + 1;
  const R vre = __shfl_sync(0xffffffffu, mine, ire & 31), vim = __shfl_sync(0xffffffffu, mine, iim & 31);
  R re = ire < 32 ? vre : extra[ire - 32 < 4 ? ire - 32 : 0];
  R im = iim < 32 ? vim : extra[iim - 32 < 4 ? iim - 32 : 0];
  float out_re = 0.f, out_im = 0.f;
  int out_row = -1, out_col = -1;
  if (lane < 18) {
    const R sc = lane < 9 ? R(v_scale) : R(k_scale);
    out_re = (float)(re * sc);
    out_im = (float)(im * sc);
    out_row = pick3(s0, s1, s2, pi_[e / 3]);
    out_col = pick3(t0, t1, t2, pj_[e % 3]);
  }
  const size_t nv = (size_t)g.nv;
  if (lane < 9 && DO_V) atomicAdd(&V[out_row * nv + out_col], make_float2(out_re, out_im));
  if (lane >= 9 && lane < 18 && DO_K) {
    float add_re = out_re;
    if (NCOMMON == 3 && mass_coeff != 0.f) {
      // P1 mass block of a coincident pair (integrand.h:257-278): area * sum_q w_q phi_a phi_b
      const int e = lane - 9, a = pick3(pm.i0, pm.i1, pm.i2, e / 3), b = pick3(pm.j0, pm.j1, pm.j2, e % 3);
      double m = 0.0;
#pragma unroll
      for (int q = 0; q < 6; q++) m += tri6_w(q) * tri6_phi(q, a) * tri6_phi(q, b);
      add_re += (float)(mass_coeff * 0.5 * (double)Ji * m);
    }
    atomicAdd(&K[out_row * nv + out_col], make_float2(add_re, out_im));
  }
}

template <typename R, int NCOMMON, bool DO_V, bool DO_K>
__global__ void __launch_bounds__(128)
    singular_vk_kernel(GeomView g, const int2* __restrict__ pairs, int npairs, float k, float2* __restrict__ V,
                       float2* __restrict__ K, float v_scale, float k_scale, float mass_coeff) {
  const int pair = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pair >= npairs) return;
  const int ti = NCOMMON == 3 ? pair : pairs[pair].x;
  const int tj = NCOMMON == 3 ? pair : pairs[pair].y;
  singular_pair<R, NCOMMON, DO_V, DO_K>(g, ti, tj, k, V, K, v_scale, k_scale, mass_coeff);
}

// ---------------------------------------------------------------------------
// Batched assembly: many problems (meshes of uneven size, wavenumbers) in one
// persistent launch.  Regular work items of all problems (runs of used
// (test group, trial tile) units, each unordered pair once) form one queue
// that CTAs drain with an atomic counter (dynamic load balance); touching
// pairs of all problems are concatenated per type.
// ---------------------------------------------------------------------------
struct BatchProblem {
  GeomView g;
  float k;
  int chunk, n_chunks;      // units per item, items
  long long n_units;        // used (test group, trial tile) units
  float2* V;
  float2* K;
  long long item_begin;   // prefix sum of regular items
  long long pair_begin[3];  // prefix sums of coincident / edge / vertex pairs
};

struct BatchHeader {
  unsigned long long next_item;  // queue head (zeroed before each launch)
  int nproblems;
  int pad;
  long long total_items;
  long long total_pairs[3];
};

__device__ __forceinline__ int find_problem(const BatchProblem* probs, int np, long long x, int which) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const long long b = which < 0 ? probs[mid].item_begin : probs[mid].pair_begin[which];
    if (b <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Each unordered regular pair of every problem once (the symmetric item of
// regular_sym_kernel); items are runs of `chunk` units of one problem.
__global__ void __launch_bounds__(kSymThreads, 2)
    regular_sym_batch_kernel(BatchHeader* __restrict__ hdr, const BatchProblem* __restrict__ probs, float v_scale,
                             float k_scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SymSmem& sm = *reinterpret_cast<SymSmem*>(smem_raw);
  __shared__ long long s_item;
  if (threadIdx.x == 0) {
    mbar_init(&sm.tile_full[0], 1);
    mbar_init(&sm.tile_full[1], 1);
    mbar_init_fence();
  }
  const int np = hdr->nproblems;
  const long long total = hdr->total_items;
  unsigned uses = 0;
  for (;;) {
    __syncthreads();  // everyone has read s_item of the previous round
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(&hdr->next_item, 1ull);
    __syncthreads();
    const long long item = s_item;
    if (item >= total) break;
    const BatchProblem& P = probs[find_problem(probs, np, item, -1)];
    const long long pos = (item - P.item_begin) * P.chunk;
    const long long end = pos + P.chunk < P.n_units ? pos + P.chunk : P.n_units;
    regular_sym_units(sm, P.g, P.k, P.V, P.K, v_scale, k_scale, pos, end, uses);
  }
}

template <typename R, int NCOMMON>
__global__ void __launch_bounds__(128)
    singular_vk_batch_kernel(const BatchHeader* __restrict__ hdr, const BatchProblem* __restrict__ probs,
                             float v_scale, float k_scale, float mass_coeff) {
  const int which = NCOMMON == 3 ? 0 : (NCOMMON == 2 ? 1 : 2);
  const long long pair = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pair >= hdr->total_pairs[which]) return;
  const int pi = find_problem(probs, hdr->nproblems, pair, which);
  const BatchProblem& P = probs[pi];
  const int local = (int)(pair - P.pair_begin[which]);
  int ti = local, tj = local;
  if (NCOMMON == 2) {
    ti = P.g.edge_pairs[local].x;
    tj = P.g.edge_pairs[local].y;
  } else if (NCOMMON == 1) {
    ti = P.g.vert_pairs[local].x;
    tj = P.g.vert_pairs[local].y;
  }
  singular_pair<R, NCOMMON, true, true>(P.g, ti, tj, P.k, P.V, P.K, v_scale, k_scale, mass_coeff);
}

// Dense P1 mass matrix, one thread per triangle (bind.cu:10-21).
__global__ void mass_kernel(GeomView g, float2* __restrict__ M, float coeff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nt) return;
  const TriRec& r = g.rec_orig[i];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      double m = 0.0;
#pragma unroll
      for (int q = 0; q < 6; q++) m += tri6_w(q) * tri6_phi(q, a) * tri6_phi(q, b);
      atomicAdd(&M[(size_t)r.v[a] * g.nv + r.v[b]], make_float2((float)(coeff * r.area * m), 0.f));
    }
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

template <bool DO_V, bool DO_K>
int launch_regular(const GeomView& g, float k, float2* V, float2* K, float v_scale, float k_scale, cudaStream_t s) {
  const int smem = (int)sizeof(RegSmem<DO_V, DO_K>);
  static std::atomic<bool> attr_set{false};
  if (!attr_set.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(regular_vk_kernel<DO_V, DO_K>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set.store(true, std::memory_order_release);
  }
  const int n_groups = (g.nt + kTestTris - 1) / kTestTris;
  int occ = 0;
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, regular_vk_kernel<DO_V, DO_K>, kRegThreads, smem));
  if (g_tune_ctas_per_sm > 0 && g_tune_ctas_per_sm < occ) occ = g_tune_ctas_per_sm;
  const int grid = sm_count() * (occ > 0 ? occ : 1);
  // chunk of trial tiles per work item: enough items to balance the grid
  int chunk = (int)((long long)n_groups * g.ntiles / (8LL * grid));
  chunk = chunk < 1 ? 1 : (chunk > 64 ? 64 : chunk);
  if (g_tune_chunk > 0) chunk = g_tune_chunk;
  const int n_chunks = (g.ntiles + chunk - 1) / chunk;
  const int n_items = n_groups * n_chunks;
  (regular_vk_kernel<DO_V, DO_K><<<grid < n_items ? grid : n_items, kRegThreads, smem, s>>>(
      g, k, V, K, v_scale, k_scale, chunk, n_chunks, n_items), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

template <bool DO_V, bool DO_K>
int launch_singular(const GeomView& g, float k, float2* V, float2* K, float v_scale, float k_scale, float mass_coeff,
                    cudaStream_t s) {
  const int wpb = 4;  // warps per block
  (singular_vk_kernel<double, 3, DO_V, DO_K><<<(g.nt + wpb - 1) / wpb, 32 * wpb, 0, s>>>(
      g, nullptr, g.nt, k, V, K, v_scale, k_scale, mass_coeff), count_launch());
  if (g.n_edge)
    (singular_vk_kernel<float, 2, DO_V, DO_K><<<(g.n_edge + wpb - 1) / wpb, 32 * wpb, 0, s>>>(
        g, g.edge_pairs, g.n_edge, k, V, K, v_scale, k_scale, 0.f), count_launch());
  if (g.n_vert)
    (singular_vk_kernel<float, 1, DO_V, DO_K><<<(g.n_vert + wpb - 1) / wpb, 32 * wpb, 0, s>>>(
        g, g.vert_pairs, g.n_vert, k, V, K, v_scale, k_scale, 0.f), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

}  // namespace

// V and/or (mass_coeff M + k_coeff K), both overwritten.
int launch_regular_sym(const GeomView& g, float k, float2* V, float2* K, float v_scale, float k_scale,
                       cudaStream_t s) {
  const int smem = (int)sizeof(SymSmem);
  static std::atomic<bool> attr_set{false};
  if (!attr_set.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(regular_sym_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set.store(true, std::memory_order_release);
  }
  int occ = 0;
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, regular_sym_kernel, kSymThreads, smem));
  const int grid = sm_count() * (occ > 0 ? occ : 1);
  const long long n_units = (long long)g.ntiles * (g.ntiles + 1) / 2;
  // 8 equal items per CTA (a tuned chunk overrides)
  long long chunk = (n_units + 8LL * grid - 1) / (8LL * grid);
  if (chunk < 1) chunk = 1;
  if (g_tune_chunk > 0) chunk = g_tune_chunk;
  const long long n_items = (n_units + chunk - 1) / chunk;
  (regular_sym_kernel<<<grid < n_items ? grid : (int)n_items, kSymThreads, smem, s>>>(g, k, V, K, v_scale, k_scale,
                                                                                       chunk, n_units, (int)n_items),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

int assemble_vk(const GeomView& g, float k, float2* V, float2* Kout, float mass_coeff, float k_coeff, cudaStream_t s) {
  const size_t bytes = sizeof(float2) * (size_t)g.nv * g.nv;
  if (V) BEM_CUDA_TRY(cudaMemsetAsync(V, 0, bytes, s));
  if (Kout) BEM_CUDA_TRY(cudaMemsetAsync(Kout, 0, bytes, s));
  const float v_scale = kInv4Pi;
  const float k_scale = -kInv4Pi * k_coeff;  // K = -(...)/(4 pi)
  int rc;
  if (V && Kout) {
    if ((rc = launch_regular_sym(g, k, V, Kout, v_scale, k_scale, s))) return rc;
    return launch_singular<true, true>(g, k, V, Kout, v_scale, k_scale, mass_coeff, s);
  } else if (V) {
    if ((rc = launch_regular<true, false>(g, k, V, nullptr, v_scale, 0.f, s))) return rc;
    return launch_singular<true, false>(g, k, V, nullptr, v_scale, 0.f, 0.f, s);
  } else if (Kout) {
    if ((rc = launch_regular<false, true>(g, k, nullptr, Kout, 0.f, k_scale, s))) return rc;
    return launch_singular<false, true>(g, k, nullptr, Kout, 0.f, k_scale, mass_coeff, s);
  }
  return BEM_OK;
}

int assemble_mass(const GeomView& g, float2* M, float coeff, bool zero, cudaStream_t s) {
  if (zero) BEM_CUDA_TRY(cudaMemsetAsync(M, 0, sizeof(float2) * (size_t)g.nv * g.nv, s));
  (mass_kernel<<<(g.nt + 127) / 128, 128, 0, s>>>(g, M, coeff), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

}  // namespace bemb

// ---------------------------------------------------------------------------
// Batched assembly host side and tuning knobs.
// ---------------------------------------------------------------------------
#include <vector>

namespace bemb {

namespace {
int g_tune_chunk = 0;        // trial tiles per regular work item (0: automatic)
int g_tune_ctas_per_sm = 0;  // persistent CTAs per SM (0: occupancy limit)

struct PinnedStage {
  void* buf = nullptr;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
  ~PinnedStage() {
    if (buf) cudaFreeHost(buf);
    if (ev) cudaEventDestroy(ev);
  }
};
thread_local PinnedStage t_stage;

inline size_t al256b(size_t x) { return (x + 255) / 256 * 256; }
}  // namespace

// Reads and clears the flag that an assembly kernel's bounded wait expired
// (synchronises the stream).
int assembly_status(int* err_host, cudaStream_t s) {
  int zero = 0;
  BEM_CUDA_TRY(cudaMemcpyFromSymbolAsync(err_host, g_asm_err, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaMemcpyToSymbolAsync(g_asm_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  return BEM_OK;
}

int set_tuning(int key, int value) {
  if (value < 0) return BEM_ERR_INVALID_ARGUMENT;
  switch (key) {
    case BEM_TUNE_ASSEMBLY_CHUNK: g_tune_chunk = value; return BEM_OK;
    case BEM_TUNE_ASSEMBLY_CTAS_PER_SM: g_tune_ctas_per_sm = value; return BEM_OK;
    case BEM_TUNE_TC_PROMOTE: g_tc_promote = value; return BEM_OK;
    case BEM_TUNE_GMRES_REORTH:
      if (value > 2) return BEM_ERR_INVALID_ARGUMENT;
      g_gmres_reorth = value;
      return BEM_OK;
    case BEM_TUNE_ARNOLDI_CLUSTER:
      if (value > 16) return BEM_ERR_INVALID_ARGUMENT;
      g_arn_max_cluster = value;
      return BEM_OK;
    case BEM_TUNE_ARNOLDI_MODE:
      if (value > 3) return BEM_ERR_INVALID_ARGUMENT;
      g_arn_mode = value;
      return BEM_OK;
    case BEM_TUNE_TC_WAIT_US:
      g_tc_wait_us = value;
      return BEM_OK;
    case BEM_TUNE_TC_TEST_SKIP_FILL:
      g_tc_skip_fill.store(value);
      return BEM_OK;
    case BEM_TUNE_GMRES_BLOCK:
      if (value > 1) return BEM_ERR_INVALID_ARGUMENT;
      g_gmres_block = value;
      return BEM_OK;
  }
  return BEM_ERR_INVALID_ARGUMENT;
}

int get_tuning(int key) {
  switch (key) {
    case BEM_TUNE_ASSEMBLY_CHUNK: return g_tune_chunk;
    case BEM_TUNE_ASSEMBLY_CTAS_PER_SM: return g_tune_ctas_per_sm;
    case BEM_TUNE_TC_PROMOTE: return g_tc_promote;
    case BEM_TUNE_GMRES_REORTH: return g_gmres_reorth;
    case BEM_TUNE_ARNOLDI_CLUSTER: return g_arn_max_cluster;
    case BEM_TUNE_ARNOLDI_MODE: return g_arn_mode;
    case BEM_TUNE_TC_WAIT_US: return g_tc_wait_us;
    case BEM_TUNE_TC_TEST_SKIP_FILL: return g_tc_skip_fill.load();
    case BEM_TUNE_GMRES_BLOCK: return g_gmres_block;
  }
  return -1;
}

size_t batch_workspace_bytes(int np) {
  return al256b(sizeof(BatchHeader)) + al256b(sizeof(BatchProblem) * (size_t)(np > 0 ? np : 1));
}

int assemble_vk_batch(const GeomView* views, const float* ks, float2* const* Vs, float2* const* Ks, int np,
                      float mass_coeff, float k_coeff, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (np <= 0) return BEM_ERR_INVALID_ARGUMENT;
  if (!ws || ws_bytes < batch_workspace_bytes(np)) return BEM_ERR_WORKSPACE;
  const int smem = (int)sizeof(SymSmem);
  static std::atomic<bool> attr{false};
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(regular_sym_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr.store(true, std::memory_order_release);
  }
  // host descriptors
  const size_t hbytes = al256b(sizeof(BatchHeader)), pbytes = sizeof(BatchProblem) * (size_t)np;
  if (!t_stage.ev) BEM_CUDA_TRY(cudaEventCreateWithFlags(&t_stage.ev, cudaEventDisableTiming));
  BEM_CUDA_TRY(cudaEventSynchronize(t_stage.ev));  // previous upload from the staging buffer is done
  if (t_stage.cap < hbytes + pbytes) {
    if (t_stage.buf) cudaFreeHost(t_stage.buf);
    t_stage.cap = 2 * (hbytes + pbytes);
    BEM_CUDA_TRY(cudaHostAlloc(&t_stage.buf, t_stage.cap, cudaHostAllocDefault));
  }
  BatchHeader* hh = (BatchHeader*)t_stage.buf;
  BatchProblem* hp = (BatchProblem*)((char*)t_stage.buf + hbytes);
  std::memset(hh, 0, sizeof(BatchHeader));
  hh->nproblems = np;
  long long items = 0, pairs[3] = {0, 0, 0};
  const size_t elem = sizeof(float2);
  for (int p = 0; p < np; p++) {
    const GeomView& g = views[p];
    if (!Vs[p] || !Ks[p]) return BEM_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(ks[p])) return BEM_ERR_NONFINITE;
    BEM_CUDA_TRY(cudaMemsetAsync(Vs[p], 0, elem * (size_t)g.nv * g.nv, s));
    BEM_CUDA_TRY(cudaMemsetAsync(Ks[p], 0, elem * (size_t)g.nv * g.nv, s));
    BatchProblem& P = hp[p];
    P.g = g;
    P.k = ks[p];
    P.n_units = (long long)g.ntiles * (g.ntiles + 1) / 2;
    int chunk = g_tune_chunk > 0 ? g_tune_chunk : (g.ntiles / 8 < 1 ? 1 : (g.ntiles / 8 > 64 ? 64 : g.ntiles / 8));
    P.chunk = chunk;
    P.n_chunks = (int)((P.n_units + chunk - 1) / chunk);
    P.V = Vs[p];
    P.K = Ks[p];
    P.item_begin = items;
    items += P.n_chunks;
    P.pair_begin[0] = pairs[0];
    P.pair_begin[1] = pairs[1];
    P.pair_begin[2] = pairs[2];
    pairs[0] += g.nt;
    pairs[1] += g.n_edge;
    pairs[2] += g.n_vert;
  }
  hh->total_items = items;
  for (int t = 0; t < 3; t++) hh->total_pairs[t] = pairs[t];
  BatchHeader* dh = (BatchHeader*)ws;
  BatchProblem* dp = (BatchProblem*)((char*)ws + hbytes);
  BEM_CUDA_TRY(cudaMemcpyAsync(ws, t_stage.buf, hbytes + pbytes, cudaMemcpyHostToDevice, s));
  BEM_CUDA_TRY(cudaEventRecord(t_stage.ev, s));
  const float v_scale = kInv4Pi, k_scale = -kInv4Pi * k_coeff;
  int occ = 0;
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, regular_sym_batch_kernel, kSymThreads, smem));
  if (g_tune_ctas_per_sm > 0 && g_tune_ctas_per_sm < occ) occ = g_tune_ctas_per_sm;
  const long long grid = (long long)sm_count() * (occ > 0 ? occ : 1);
  if (items > 0)
    (regular_sym_batch_kernel<<<(unsigned)(grid < items ? grid : items), kSymThreads, smem, s>>>(dh, dp, v_scale,
                                                                                                 k_scale),
     count_launch());
  const int wpb = 4;
  if (pairs[0])
    (singular_vk_batch_kernel<double, 3><<<(unsigned)((pairs[0] + wpb - 1) / wpb), 32 * wpb, 0, s>>>(
         dh, dp, v_scale, k_scale, mass_coeff),
     count_launch());
  if (pairs[1])
    (singular_vk_batch_kernel<float, 2><<<(unsigned)((pairs[1] + wpb - 1) / wpb), 32 * wpb, 0, s>>>(
         dh, dp, v_scale, k_scale, mass_coeff),
     count_launch());
  if (pairs[2])
    (singular_vk_batch_kernel<float, 1><<<(unsigned)((pairs[2] + wpb - 1) / wpb), 32 * wpb, 0, s>>>(
         dh, dp, v_scale, k_scale, mass_coeff),
     count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

}  // namespace bemb

// Fused Burton-Miller assembly: both matrices of the reference's
// neumann2dirichlet (src/bem/solver.py:118-126) in one pass,
//   lhs = BM_LHS + 1/2 M,     rhs = BM_RHS - (i / (2k)) M,
// at the <2,3> rules of its "_approx" bindings (bind.cu:204-215): the 3-point
// degree-2 triangle rule for regular pairs, 2-point Gauss-Legendre
// Sauter-Schwab quadrature for touching pairs.  At the exact <4,6> rules the
// same pair is the reference's HBIE system (solver.py:106-116):
//   1/2 M - K + (i/k) W = BM_LHS + 1/2 M   (W = curl term - k^2 n.n G),
//   -V - (i/k)(K' + 1/2 M) = BM_RHS - (i/(2k)) M,
// so the kernels are templated on the rule (TN points per triangle, LN
// Gauss-Legendre points per Sauter-Schwab axis).
//
// Kernels (potential.h:42-65, integrand.h:94-101,216-221,314-322), x on the
// test triangle i, y on the trial triangle j, G = e^{ikr}/r and
// H = (1 - ikr) e^{ikr} / r^3 (the 1/(4 pi) applied last):
//   BM_LHS(i,j) = -ik (n_i.n_j) G + H (y - x).n_j + (i/k) G (curl_i . curl_j)
//   BM_RHS(i,j) = -G + (i/k) H (x - y).n_i
// The curl term uses the P1 surface curls, constant per triangle, so the
// Galerkin block needs only the weight sum of G over the pair.
//
// Regular pairs: G, H (y-x).n_j and H (x-y).n_i are symmetric / swapped under
// i <-> j, so one evaluation of r and sincos per quadrature-point pair of an
// UNORDERED pair gives all four blocks lhs_ij, lhs_ji, rhs_ij, rhs_ji:
//   S = sum C C G,  T = sum C C H (y-x).n_j,  U = sum C C H (x-y).n_i
//   lhs_ij = -ik nn S + T + (i/k) s cc      lhs_ji^T = -ik nn S + U + (i/k) s cc
//   rhs_ij = -S + (i/k) U                   rhs_ji^T = -S + (i/k) T
// with s = sum_ab S_ab (the P1 functions sum to one) and cc_ab the curl
// products.  Work decomposition: a CTA of 8 warps owns one 16-triangle test
// tile (test triangle = lane & 15) and sweeps 16-triangle trial tiles,
// double-buffered in shared memory by bulk copies, each warp taking two trial
// triangles (one per half-warp); the 3x3 blocks go to corner slabs that are
// reduced on chip onto the tiles' distinct vertices, four vector atomics per
// entry.  The slabs are small enough for three CTAs per SM, so one CTA's
// reduction and barriers overlap the others' evaluation.
// Touching pairs: one warp per pair evaluates both kernels at each
// Sauter-Schwab point (shared r and sincos); the coincident pass (FP64) adds
// the mass terms.  A batch (meshes, wavenumbers) uses the same kernels with a
// work queue over all problems.

#include <atomic>
#include <cmath>
#include <cstring>

#include "async_copy.cuh"
#include "bem_common.cuh"
#include "sauter_schwab.cuh"

namespace bemb {

namespace {

constexpr int kBmThreads = 16 * kTile;       // 256: warp w takes trial triangles 2w, 2w + 1
constexpr int kBmTest = kTile;               // test triangles per CTA (one tile), lane & 15
constexpr int kBmCorners = 3 * kBmTest;      // 48
constexpr int kBmStride = kTileCorners + 1;  // 49 float2: conflict-free column writes

// C(q, b) = w_q phi_b(q): centroid rule 1/3; 3-point rule 1/3 * (q == b ?
// 2/3 : 1/6); 6-point rule as the V/K assembly.
template <int TN>
__host__ __device__ constexpr float bm_c(int q, int b) {
  return TN == 1 ? 1.0f / 3.0f
                 : (TN == 3 ? (q == b ? 2.0f / 9.0f : 1.0f / 18.0f) : (float)(tri6_w(q) * tri6_phi(q, b)));
}

// Coordinate c of the rule's points of a triangle (records in sorted order).
template <int TN>
__device__ __forceinline__ float bm_point(const TriRec& r, const BmRec& b, int c) {
  return TN == 3 ? b.qp[c] : (TN == 6 ? r.qp[c] : r.c[c]);
}

struct BmSmem {
  // rhs_ji[b][a] is not stored: rhs_ji^T - rhs_ij = (i/k)(T - U) =
  // (i/k)(lhs_ij - lhs_ji^T) entry by entry, so it follows from the three
  // reduced slots of each vertex pair.
  float2 slotL[kBmCorners][kBmStride];   // lhs_ij[a][b] at [3 tl + a][3 tt + b]
  float2 slotLT[kBmCorners][kBmStride];  // lhs_ji[b][a], same indexing
  float2 slotR[kBmCorners][kBmStride];
  float xs[18][kBmTest];                 // test quadrature points [coordinate][tl]
  float xc[9][kBmTest];                  // test curls [3 a + d][tl]
  TriRec trial[2][kTile];                // trial tile, double-buffered
  BmRec trialB[2][kTile];
  TileRec tileJ[2];
  TileRec tileI;
  uint64_t tile_full[2];
};

// A bounded wait of the Burton-Miller kernels expired (read by bm_status).
__device__ int g_bm_err;

__device__ __forceinline__ void bm_copy_words(void* dst, const void* src, int bytes, int tid) {
  const int4* s = (const int4*)src;
  int4* d = (int4*)dst;
  for (int i = tid; i < bytes / 16; i += kBmThreads) d[i] = s[i];
}

// Thread 0: bulk-copy trial tile jt (records, Burton-Miller records, vertex
// table) into buffer b.
__device__ __forceinline__ void bm_fetch_tile(BmSmem& sm, const GeomView& g, int jt, int b) {
  const int ntri = min(kTile, g.nt - jt * kTile);
  const uint32_t rb = (uint32_t)(ntri * sizeof(TriRec)), mb = (uint32_t)(ntri * sizeof(BmRec));
  mbar_expect_tx(&sm.tile_full[b], rb + mb + (uint32_t)sizeof(TileRec));
  bulk_load(sm.trial[b], &g.rec[jt * kTile], rb, &sm.tile_full[b]);
  bulk_load(sm.trialB[b], &g.bm[jt * kTile], mb, &sm.tile_full[b]);
  bulk_load(&sm.tileJ[b], &g.tiles[jt], (uint32_t)sizeof(TileRec), &sm.tile_full[b]);
}

// S, T, U blocks of one unordered pair under the TN x TN point rule (test
// triangle tl, points in xs; trial points yq, dq[q] = n_i . (c_i - y_q)).
// Packed FP32 pairs (f32x2): complex sums as (re, im) pairs, distances for two
// trial points at once; same operations and rounding as the scalar form.
template <int TN>
__device__ __forceinline__ void bm_pair_block(const float (*xs)[kBmTest], int tl, const float (&yq)[3 * TN],
                                              const float (&dq)[TN], float njx, float njy, float njz, float cjx,
                                              float cjy, float cjz, float k, float2 (&aS)[9], float2 (&aT)[9],
                                              float2 (&aU)[9]) {
#pragma unroll
  for (int e = 0; e < 9; e++) {
    aS[e] = make_float2(0.f, 0.f);
    aT[e] = make_float2(0.f, 0.f);
    aU[e] = make_float2(0.f, 0.f);
  }
  const float2 kk = make_float2(k, -k);
#pragma unroll
  for (int p = 0; p < TN; p++) {
    const float px = xs[3 * p][tl], py = xs[3 * p + 1][tl], pz = xs[3 * p + 2][tl];
    const float dn = njx * (cjx - px) + njy * (cjy - py) + njz * (cjz - pz);  // (y - x).n_j on plane j
    float2 tS[3], tT[3], tU[3];
#pragma unroll
    for (int b = 0; b < 3; b++) {
      tS[b] = make_float2(0.f, 0.f);
      tT[b] = make_float2(0.f, 0.f);
      tU[b] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int q0 = 0; q0 < TN; q0 += 2) {
      constexpr int kLast = TN - 1;
      const int q1 = q0 + 1 < TN ? q0 + 1 : kLast;  // an odd rule repeats its last point in the idle lane
      const float2 dx = f2_sub(make_float2(yq[3 * q0], yq[3 * q1]), f2(px));
      const float2 dy = f2_sub(make_float2(yq[3 * q0 + 1], yq[3 * q1 + 1]), f2(py));
      const float2 dz = f2_sub(make_float2(yq[3 * q0 + 2], yq[3 * q1 + 2]), f2(pz));
      const float2 r2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_mul(dz, dz)));
      const float2 rinv = make_float2(fminf(rsqrtf(r2.x), 1.0f / kEps), fminf(rsqrtf(r2.y), 1.0f / kEps));
      float2 r = f2_mul(r2, rinv);
      r.x = fmaxf(r.x, kEps);
      r.y = fmaxf(r.y, kEps);
      const float2 kr = f2_mul(f2(k), r);
      const float2 rinv2 = f2_mul(rinv, rinv);
      float sc[2][2];  // [point][sin, cos]
      __sincosf(kr.x, &sc[0][0], &sc[0][1]);
      if (q0 + 1 < TN) __sincosf(kr.y, &sc[1][0], &sc[1][1]);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        if (q0 + j < TN) {
          const int q = q0 + j;
          const float ri = j == 0 ? rinv.x : rinv.y, ri2 = j == 0 ? rinv2.x : rinv2.y;
          const float2 g = f2_mul(make_float2(sc[j][1], sc[j][0]), f2(ri));                  // (c, s) / r
          const float2 h = f2_mul(f2_fma(kk, make_float2(sc[j][0], sc[j][1]), g), f2(ri2));  // (c + kr s, s - kr c) / r^3
          const float2 u = f2_mul(f2(dq[q]), h);
#pragma unroll
          for (int b = 0; b < 3; b++) {
            const float2 w = f2(bm_c<TN>(q, b));
            tS[b] = f2_fma(w, g, tS[b]);
            tT[b] = f2_fma(w, h, tT[b]);
            tU[b] = f2_fma(w, u, tU[b]);
          }
        }
      }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float wa = bm_c<TN>(p, a);
      const float2 wa2 = f2(wa), wt2 = f2(wa * dn);
#pragma unroll
      for (int b = 0; b < 3; b++) {
        aS[3 * a + b] = f2_fma(wa2, tS[b], aS[3 * a + b]);
        aT[3 * a + b] = f2_fma(wt2, tT[b], aT[3 * a + b]);
        aU[3 * a + b] = f2_fma(wa2, tU[b], aU[3 * a + b]);
      }
    }
  }
}

// One work item: test tile grp against trial tiles [jt_begin, jt_end), all
// at or after grp.  `uses` counts the trial tiles this CTA has processed
// (buffer = uses & 1, mbarrier parity = (uses >> 1) & 1).
template <int TN>
__device__ __forceinline__ void bm_item(BmSmem& sm, const GeomView& g, float k, float2* __restrict__ L,
                                        float2* __restrict__ Rm, int grp, int jt_begin, int jt_end,
                                        unsigned& uses) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tl = lane & 15;               // test triangle of this lane
  const int tt = 2 * warp + (lane >> 4);  // trial triangle of this half-warp
  const int nt = g.nt, nv = g.nv;
  const int ti = grp * kBmTest + tl;
  const bool valid_i = ti < nt;
  const TriRec& ri = g.rec[valid_i ? ti : nt - 1];
  const float area_i = ri.area;
  const float nix = ri.n[0], niy = ri.n[1], niz = ri.n[2], cix = ri.c[0], ciy = ri.c[1], ciz = ri.c[2];
  const int iv0 = ri.v[0], iv1 = ri.v[1], iv2 = ri.v[2];
  const float kinv = 1.0f / k;

  __syncthreads();  // the previous item is done with tileI, xs, xc and both trial buffers
  if (tid == 0) bm_fetch_tile(sm, g, jt_begin, uses & 1);
  bm_copy_words(&sm.tileI, &g.tiles[grp], sizeof(TileRec), tid);
  for (int e = tid; e < (3 * TN + 9) * kBmTest; e += kBmThreads) {
    const int c = e / kBmTest, l = e - c * kBmTest;
    const int t = min(grp * kBmTest + l, nt - 1);
    if (c < 3 * TN)
      sm.xs[c][l] = bm_point<TN>(g.rec[t], g.bm[t], c);
    else
      sm.xc[c - 3 * TN][l] = g.bm[t].curl[c - 3 * TN];
  }

  for (int jt = jt_begin; jt < jt_end; jt++, uses++) {
    const int bf = uses & 1;
    __syncthreads();  // the previous tile's gather is done with the slots and with buffer bf ^ 1
    if (tid == 0 && jt + 1 < jt_end) bm_fetch_tile(sm, g, jt + 1, bf ^ 1);
    if (!mbar_wait(&sm.tile_full[bf], (uses >> 1) & 1u, g.err)) {
      // expired (this geometry's status word raised): record it process-wide
      // too, and let the copy land before the buffer is reused
      if (threadIdx.x == 0) atomicExch(&g_bm_err, 1);
      mbar_wait_drain(&sm.tile_full[bf], (uses >> 1) & 1u);
    }
    const TileRec& tileJ = sm.tileJ[bf];
    const int ntriJ = min(kTile, nt - jt * kTile);

    // ---- compute: half-warp h of warp w takes trial triangle 2w + h ----
    const int tj = jt * kTile + tt;
    float aa = 0.f;
    if (tt < ntriJ) {
      const TriRec& rj = sm.trial[bf][tt];
      const int j0 = rj.v[0], j1 = rj.v[1], j2 = rj.v[2];
      const bool touching = (iv0 == j0) | (iv0 == j1) | (iv0 == j2) | (iv1 == j0) | (iv1 == j1) | (iv1 == j2) |
                            (iv2 == j0) | (iv2 == j1) | (iv2 == j2);
      const bool once = jt > grp || tj > ti;  // on the test tile itself each unordered pair once
      aa = (valid_i && !touching && once) ? area_i * rj.area : 0.f;
    }
    const bool any = __any_sync(0xffffffffu, aa != 0.f);  // every lane, before the half-warp branch
    if (tt < ntriJ && any) {
      const TriRec& rj = sm.trial[bf][tt];
      const BmRec& bj = sm.trialB[bf][tt];
      float yq[3 * TN];
#pragma unroll
      for (int e = 0; e < 3 * TN; e++) yq[e] = bm_point<TN>(rj, bj, e);
      float dq[TN];
#pragma unroll
      for (int q = 0; q < TN; q++)
        dq[q] = nix * (cix - yq[3 * q]) + niy * (ciy - yq[3 * q + 1]) + niz * (ciz - yq[3 * q + 2]);
      float2 aS[9], aT[9], aU[9];
      bm_pair_block<TN>(sm.xs, tl, yq, dq, rj.n[0], rj.n[1], rj.n[2], rj.c[0], rj.c[1], rj.c[2], k, aS, aT, aU);
      const float sc = aa * kInv4Pi;
      float2 s9 = make_float2(0.f, 0.f);
#pragma unroll
      for (int e = 0; e < 9; e++) {
        s9.x += aS[e].x;
        s9.y += aS[e].y;
      }
      s9.x *= sc * kinv;  // (i/k) s = (-s.y / k, s.x / k), scaled
      s9.y *= sc * kinv;
      const float knn = k * (nix * rj.n[0] + niy * rj.n[1] + niz * rj.n[2]);
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const float cc = sm.xc[3 * a][tl] * bj.curl[3 * b] + sm.xc[3 * a + 1][tl] * bj.curl[3 * b + 1] +
                           sm.xc[3 * a + 2][tl] * bj.curl[3 * b + 2];
          const float Sx = aS[3 * a + b].x * sc, Sy = aS[3 * a + b].y * sc;
          const float Tx = aT[3 * a + b].x * sc, Ty = aT[3 * a + b].y * sc;
          const float Ux = aU[3 * a + b].x * sc, Uy = aU[3 * a + b].y * sc;
          const float lx = fmaf(knn, Sy, -s9.y * cc), ly = fmaf(-knn, Sx, s9.x * cc);
          sm.slotL[3 * tl + a][3 * tt + b] = make_float2(lx + Tx, ly + Ty);
          sm.slotLT[3 * tl + a][3 * tt + b] = make_float2(lx + Ux, ly + Uy);
          sm.slotR[3 * tl + a][3 * tt + b] = make_float2(fmaf(-Uy, kinv, -Sx), fmaf(Ux, kinv, -Sy));
        }
    } else if (tt < ntriJ) {
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          sm.slotL[3 * tl + a][3 * tt + b] = make_float2(0.f, 0.f);
          sm.slotLT[3 * tl + a][3 * tt + b] = make_float2(0.f, 0.f);
          sm.slotR[3 * tl + a][3 * tt + b] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();

    // ---- reduce corner slots onto distinct vertices: (A, B) and (B, A) ----
    // Pass 1, in place: for every trial corner column, the row of test
    // vertex A's first corner gets the sum over A's test corners (corner rows
    // of different vertices are disjoint); pass 2: entry (A, B) sums B's
    // trial corners along that row.
    const TileRec& TI = sm.tileI;
    const int nI = TI.nlv, nJ = tileJ.nlv;
    const int ncol = 3 * ntriJ;
    const float rcol = 1.f / (float)ncol, rJ = 1.f / (float)(nJ > 0 ? nJ : 1);
    for (int e = tid; e < nI * ncol; e += kBmThreads) {
      const int a = div_by(e, ncol, rcol);
      const int col = e - a * ncol;
      const int ca0 = TI.lv_ptr[a], ca1 = TI.lv_ptr[a + 1];
      const int rep = TI.lv_corner[ca0];
      float2 l = sm.slotL[rep][col], lt = sm.slotLT[rep][col], rr = sm.slotR[rep][col];
#pragma unroll 4
      for (int ca = ca0 + 1; ca < ca1; ca++) {
        const int row = TI.lv_corner[ca];
        const float2 l1 = sm.slotL[row][col], lt1 = sm.slotLT[row][col], r1 = sm.slotR[row][col];
        l.x += l1.x;
        l.y += l1.y;
        lt.x += lt1.x;
        lt.y += lt1.y;
        rr.x += r1.x;
        rr.y += r1.y;
      }
      sm.slotL[rep][col] = l;
      sm.slotLT[rep][col] = lt;
      sm.slotR[rep][col] = rr;
    }
    __syncthreads();
    for (int e = tid; e < nI * nJ; e += kBmThreads) {
      const int a = div_by(e, nJ, rJ);
      const int b = e - a * nJ;
      const int rep = TI.lv_corner[TI.lv_ptr[a]];
      const int cb0 = tileJ.lv_ptr[b], cb1 = tileJ.lv_ptr[b + 1];
      float2 l = make_float2(0.f, 0.f), lt = l, rr = l;
#pragma unroll 4
      for (int cb = cb0; cb < cb1; cb++) {
        const int col = tileJ.lv_corner[cb];
        const float2 l1 = sm.slotL[rep][col], lt1 = sm.slotLT[rep][col], r1 = sm.slotR[rep][col];
        l.x += l1.x;
        l.y += l1.y;
        lt.x += lt1.x;
        lt.y += lt1.y;
        rr.x += r1.x;
        rr.y += r1.y;
      }
      const float2 rt = make_float2(fmaf(lt.y - l.y, kinv, rr.x), fmaf(l.x - lt.x, kinv, rr.y));
      const int A = TI.vid[a], B = tileJ.vid[b];
      if (l.x != 0.f || l.y != 0.f || lt.x != 0.f || lt.y != 0.f || rr.x != 0.f || rr.y != 0.f) {
        atomicAdd(&L[(size_t)A * nv + B], l);
        atomicAdd(&L[(size_t)B * nv + A], lt);
        atomicAdd(&Rm[(size_t)A * nv + B], rr);
        atomicAdd(&Rm[(size_t)B * nv + A], rt);
      }
    }
  }
}

// Splits units [pos, end) of one problem at test-tile boundaries.
template <int TN>
__device__ __forceinline__ void bm_units(BmSmem& sm, const GeomView& g, float k, float2* L, float2* Rm,
                                         long long pos, long long end, unsigned& uses) {
  while (pos < end) {  // uniform over the block
    const int grp = tile_group_of(pos, g.ntiles);
    const long long base = tile_units_before(grp, g.ntiles);
    const long long gend = base + (g.ntiles - grp);
    const long long stop = end < gend ? end : gend;
    const int jt0 = grp + (int)(pos - base);
    bm_item<TN>(sm, g, k, L, Rm, grp, jt0, jt0 + (int)(stop - pos), uses);
    pos = stop;
  }
}

// ---- problem descriptors (one problem, or a batch) ----
struct BmProblem {
  GeomView g;
  float k;
  int chunk;                // units per work item
  long long n_units;        // used (test group, trial tile) units
  long long item_begin;     // prefix sum of work items
  long long pair_begin[3];  // prefix sums of coincident / edge / vertex pairs
  float2* L;
  float2* R;
};

struct BmHeader {
  unsigned long long next_item;  // queue head (zeroed before each launch)
  int nproblems;
  int pad;
  long long total_items;
  long long total_pairs[3];
};

__device__ __forceinline__ int bm_find(const BmProblem* probs, int np, long long x, int which) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const long long b = which < 0 ? probs[mid].item_begin : probs[mid].pair_begin[which];
    if (b <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void bm_init_barriers(BmSmem& sm) {
  if (threadIdx.x == 0) {
    mbar_init(&sm.tile_full[0], 1);
    mbar_init(&sm.tile_full[1], 1);
    mbar_init_fence();
  }
}

// CTAs per SM of the regular kernels: three at the 1- and 3-point rules
// (80 registers, the slabs of three CTAs fit in shared memory: the barriers
// and the on-chip reduction of one CTA overlap two others' evaluation), two at
// the 6-point rule (whose accumulators would spill at 80 registers).
__host__ __device__ constexpr int bm_min_ctas(int tn) { return tn == 6 ? 2 : 3; }

// Regular pairs of one problem: equal work items dealt round-robin to a
// persistent grid.
template <int TN>
__global__ void __launch_bounds__(kBmThreads, bm_min_ctas(TN))
    regular_bm_kernel(const __grid_constant__ BmProblem P, int n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BmSmem& sm = *reinterpret_cast<BmSmem*>(smem_raw);
  bm_init_barriers(sm);
  unsigned uses = 0;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const long long pos = (long long)item * P.chunk;
    const long long end = pos + P.chunk < P.n_units ? pos + P.chunk : P.n_units;
    bm_units<TN>(sm, P.g, P.k, P.L, P.R, pos, end, uses);
  }
}

// Regular pairs of a batch: CTAs drain one queue of work items.
template <int TN>
__global__ void __launch_bounds__(kBmThreads, bm_min_ctas(TN))
    regular_bm_batch_kernel(BmHeader* __restrict__ hdr, const BmProblem* __restrict__ probs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BmSmem& sm = *reinterpret_cast<BmSmem*>(smem_raw);
  __shared__ long long s_item;
  bm_init_barriers(sm);
  const int np = hdr->nproblems;
  const long long total = hdr->total_items;
  unsigned uses = 0;
  for (;;) {
    __syncthreads();  // everyone has read s_item of the previous round
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(&hdr->next_item, 1ull);
    __syncthreads();
    const long long item = s_item;
    if (item >= total) break;
    const BmProblem& P = probs[bm_find(probs, np, item, -1)];
    const long long pos = (item - P.item_begin) * P.chunk;
    const long long end = pos + P.chunk < P.n_units ? pos + P.chunk : P.n_units;
    bm_units<TN>(sm, P.g, P.k, P.L, P.R, pos, end, uses);
  }
}

// Both Burton-Miller kernels at d = y - x, without the 1/(4 pi):
// lhs_main = -ik nn G + H d.n_j, aux = (i/k) G, rhs = -G + (i/k) H (-d).n_i.
template <typename R>
__device__ __forceinline__ void bm_eval(R dx, R dy, R dz, const R (&ni)[3], const R (&nj)[3], R nn, R k, R kinv,
                                        R& lr, R& li, R& ar, R& ai, R& rr, R& ri) {
  R r, ir;
  inv_dist<R>(dx * dx + dy * dy + dz * dz, &r, &ir);
  const R kr = k * r;
  R s, c;
  sincos_t<R>(kr, &s, &c);
  const R gr = c * ir, gi = s * ir;
  const R ir2 = ir * ir;
  const R hr = (c + kr * s) * ir * ir2, hi = (s - kr * c) * ir * ir2;
  const R dnj = dx * nj[0] + dy * nj[1] + dz * nj[2];     // (y - x).n_j
  const R dni = -(dx * ni[0] + dy * ni[1] + dz * ni[2]);  // (x - y).n_i
  lr = k * nn * gi + hr * dnj;
  li = -k * nn * gr + hi * dnj;
  ar = -gi * kinv;
  ai = gr * kinv;
  rr = -gr - hi * dni * kinv;
  ri = -gi + hr * dni * kinv;
}

// Lanes per touching pair: the LN^4 Gauss points of the 4-D rule are split
// over 16 lanes when there are at most 16 of them (two pairs per warp, at
// the 2-point rule of the <2,3> orders), else over the whole warp.
template <int LN>
struct BmSingLanes {
  static constexpr int kPoints = LN * LN * LN * LN;
  static constexpr int kW = kPoints <= 16 ? 16 : 32;
  static constexpr int kPairsPerWarp = 32 / kW;
};

// One touching pair (index `local` of its type) on W = BmSingLanes<LN>::kW
// lanes (lane `sub` of them); the coincident pass also adds 1/2 M to lhs and
// -(i/(2k)) M to rhs.  `store` is false for the idle half of a warp whose
// last pair is missing (it computes a copy of a valid pair, for the
// shuffles, and adds nothing).
template <typename R, int NCOMMON, int LN>
__device__ __forceinline__ void singular_bm_pair(const BmProblem& P, int local, int sub, bool store) {
  constexpr int W = BmSingLanes<LN>::kW;
  const GeomView& g = P.g;
  int ti = local, tj = local;
  if (NCOMMON == 2) {
    ti = g.edge_pairs[local].x;
    tj = g.edge_pairs[local].y;
  } else if (NCOMMON == 1) {
    ti = g.vert_pairs[local].x;
    tj = g.vert_pairs[local].y;
  }
  const int s0 = g.triangles[3 * ti], s1 = g.triangles[3 * ti + 1], s2 = g.triangles[3 * ti + 2];
  const int t0 = g.triangles[3 * tj], t1 = g.triangles[3 * tj + 1], t2 = g.triangles[3 * tj + 2];
  const Perm6 pm = reorder6<NCOMMON>(s0, s1, s2, t0, t1, t2);
  const int pi_[3] = {pm.i0, pm.i1, pm.i2}, pj_[3] = {pm.j0, pm.j1, pm.j2};
  const int sv[3] = {s0, s1, s2}, tv[3] = {t0, t1, t2};
  R a[3][3], b[3][3], oa[3][3], ob[3][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int va = sel3(s0, s1, s2, pi_[c]), vb = sel3(t0, t1, t2, pj_[c]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      a[c][d] = (R)g.vertices[3 * va + d];
      b[c][d] = (R)g.vertices[3 * vb + d];
      oa[c][d] = (R)g.vertices[3 * sv[c] + d];
      ob[c][d] = (R)g.vertices[3 * tv[c] + d];
    }
  }
  R ni[3], nj[3], Ji, Jj;
  {
    const R e1[3] = {oa[1][0] - oa[0][0], oa[1][1] - oa[0][1], oa[1][2] - oa[0][2]};
    const R e2[3] = {oa[2][0] - oa[0][0], oa[2][1] - oa[0][1], oa[2][2] - oa[0][2]};
    const R cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    Ji = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int d = 0; d < 3; d++) ni[d] = cr[d] / Ji;
  }
  {
    const R e1[3] = {ob[1][0] - ob[0][0], ob[1][1] - ob[0][1], ob[1][2] - ob[0][2]};
    const R e2[3] = {ob[2][0] - ob[0][0], ob[2][1] - ob[0][1], ob[2][2] - ob[0][2]};
    const R cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    Jj = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int d = 0; d < 3; d++) nj[d] = cr[d] / Jj;
  }
  const R kk = (R)P.k, kinv = R(1) / kk;
  const R nn = ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2];
  // t[4 e + (0, 1, 2, 3)] = (lhs re, lhs im, rhs re, rhs im) of block entry
  // e = 3 ii + jj (re-ordered slots), t[36], t[37] = the weight sum of the
  // curl term's (i/k) G; t[38..63] stay zero (padding for the reduction)
  R t[64];
#pragma unroll
  for (int e = 0; e < 64; e++) t[e] = 0;
  auto region = [&](R x1, R x2, R y1, R y2, R ww) {
    const R lx[3] = {R(1) - x1, x1 - x2, x2};
    const R ly[3] = {R(1) - y1, y1 - y2, y2};
    R xp[3], yp[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      xp[d] = lx[0] * a[0][d] + lx[1] * a[1][d] + lx[2] * a[2][d];
      yp[d] = ly[0] * b[0][d] + ly[1] * b[1][d] + ly[2] * b[2][d];
    }
    R lr, li, ar, ai, rr, ri;
    bm_eval<R>(yp[0] - xp[0], yp[1] - xp[1], yp[2] - xp[2], ni, nj, nn, kk, kinv, lr, li, ar, ai, rr, ri);
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++) {
        const R f = lx[ii] * ly[jj] * ww;
        const int e = 3 * ii + jj;
        t[4 * e] += lr * f;
        t[4 * e + 1] += li * f;
        t[4 * e + 2] += rr * f;
        t[4 * e + 3] += ri * f;
      }
    t[36] += ar * ww;
    t[37] += ai * ww;
  };
  const R jw = Ji * Jj / R(16);
  constexpr int NPT = BmSingLanes<LN>::kPoints;
#pragma unroll 1
  for (int pt = sub; pt < NPT; pt += W) {
    const int i0 = pt / (LN * LN * LN), i1 = (pt / (LN * LN)) % LN, i2 = (pt / LN) % LN, i3 = pt % LN;
    const R xi = R(0.5) * (R(gl_x<LN>(i0)) + R(1)), e1 = R(0.5) * (R(gl_x<LN>(i1)) + R(1));
    const R e2 = R(0.5) * (R(gl_x<LN>(i2)) + R(1)), e3 = R(0.5) * (R(gl_x<LN>(i3)) + R(1));
    const R w0 = R(gl_w<LN>(i0)) * R(gl_w<LN>(i1)) * R(gl_w<LN>(i2)) * R(gl_w<LN>(i3)) * jw;
    ss_regions<NCOMMON, R>(xi, e1, e2, e3, w0, region);
  }
  // transpose-reduce over the W lanes (xor offsets < W stay inside the
  // pair's lanes): every round halves the values a lane keeps, so lane `sub`
  // ends with the totals of values (64 / W) sub + i in t[i]
#pragma unroll
  for (int o = W / 2, half = 32; o >= 1; o >>= 1, half >>= 1) {
    const bool hi = (sub & o) != 0;
#pragma unroll
    for (int i = 0; i < half; i++) {
      const R send = hi ? t[i] : t[i + half];
      const R keep = hi ? t[i + half] : t[i];
      t[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  // W = 16: lane e (< 9) holds entry e (lhs re, im, rhs re, im), lane 9 the
  // curl sums; W = 32: lane 2e holds entry e's lhs, lane 2e + 1 its rhs,
  // lane 18 the curl sums
  constexpr int kAuxLane = W == 16 ? 9 : 18;
  const R aux_re = __shfl_sync(0xffffffffu, t[0], kAuxLane, W);
  const R aux_im = __shfl_sync(0xffffffffu, t[1], kAuxLane, W);
  const int e = W == 16 ? sub : (sub >> 1);
  const bool do_lhs = W == 16 ? sub < 9 : (sub < 18 && (sub & 1) == 0);
  const bool do_rhs = W == 16 ? sub < 9 : (sub < 18 && (sub & 1) == 1);
  if (!store || !(do_lhs || do_rhs)) return;
  const int ii = e / 3, jj = e % 3;      // re-ordered slots
  const int ia = pi_[ii], jb = pj_[jj];  // original local vertices
  const R sc = R(kInv4Pi);
  const R m = NCOMMON == 3 ? R(0.5) * Ji * (ia == jb ? R(2) : R(1)) / R(12) : R(0);  // P1 mass: area (1 + [a == b]) / 12
  const size_t at = (size_t)sel3(s0, s1, s2, ia) * g.nv + sel3(t0, t1, t2, jb);
  if (do_lhs) {
    R cp = 0;
    for (int d = 0; d < 3; d++) cp += (R)g.curls[9 * ti + 3 * ia + d] * (R)g.curls[9 * tj + 3 * jb + d];
    R lre = (t[0] + aux_re * cp) * sc, lim = (t[1] + aux_im * cp) * sc;
    if (NCOMMON == 3) lre += R(0.5) * m;
    atomicAdd(&P.L[at], make_float2((float)lre, (float)lim));
  }
  if (do_rhs) {
    const int o = W == 16 ? 2 : 0;
    R rre = t[o] * sc, rim = t[o + 1] * sc;
    if (NCOMMON == 3) rim -= R(0.5) * kinv * m;
    atomicAdd(&P.R[at], make_float2((float)rre, (float)rim));
  }
}

// Pair index of this warp's lanes (kPairsPerWarp pairs per warp): `first` is
// the warp's first pair, `sub` the lane within the pair.
template <int LN>
__device__ __forceinline__ long long bm_sing_pair_index(long long* first, int* sub) {
  constexpr int W = BmSingLanes<LN>::kW, PPW = BmSingLanes<LN>::kPairsPerWarp;
  const int lane = threadIdx.x & 31;
  *first = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * PPW;
  *sub = lane & (W - 1);
  return *first + lane / W;
}

template <typename R, int NCOMMON, int LN>
__global__ void __launch_bounds__(128) singular_bm_kernel(const __grid_constant__ BmProblem P, int npairs) {
  long long first;
  int sub;
  const long long pair = bm_sing_pair_index<LN>(&first, &sub);
  if (first >= npairs) return;  // uniform over the warp
  const bool store = pair < npairs;
  singular_bm_pair<R, NCOMMON, LN>(P, (int)(store ? pair : first), sub, store);
}

template <typename R, int NCOMMON, int LN>
__global__ void __launch_bounds__(128)
    singular_bm_batch_kernel(const BmHeader* __restrict__ hdr, const BmProblem* __restrict__ probs) {
  constexpr int which = NCOMMON == 3 ? 0 : (NCOMMON == 2 ? 1 : 2);
  long long first;
  int sub;
  long long pair = bm_sing_pair_index<LN>(&first, &sub);
  const long long total = hdr->total_pairs[which];
  if (first >= total) return;  // uniform over the warp
  const bool store = pair < total;
  if (!store) pair = first;
  const BmProblem& P = probs[bm_find(probs, hdr->nproblems, pair, which)];
  singular_bm_pair<R, NCOMMON, LN>(P, (int)(pair - P.pair_begin[which]), sub, store);
}

inline size_t al256(size_t x) { return (x + 255) / 256 * 256; }

int bm_sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

// Host staging of the batch descriptors (pinned, reused; one per host thread).
struct BmStage {
  void* buf = nullptr;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
  ~BmStage() {
    if (buf) cudaFreeHost(buf);
    if (ev) cudaEventDestroy(ev);
  }
};
thread_local BmStage t_bm_stage;

int bm_check(float k, const float2* L, const float2* R) {
  if (!L || !R) return BEM_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(k)) return BEM_ERR_NONFINITE;
  if (k == 0.f) return BEM_ERR_INVALID_ARGUMENT;  // the Burton-Miller coupling i/k
  return BEM_OK;
}

// Persistent grid of a regular kernel (shared-memory attribute set once).
template <typename KernelT>
int bm_grid(KernelT kernel, std::atomic<bool>& attr, long long* grid) {
  const int smem = (int)sizeof(BmSmem);
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr.store(true, std::memory_order_release);
  }
  int occ = 0;
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBmThreads, smem));
  *grid = (long long)bm_sm_count() * (occ > 0 ? occ : 1);
  return BEM_OK;
}

long long bm_units_of(const GeomView& g) { return (long long)g.ntiles * (g.ntiles + 1) / 2; }

}  // namespace

size_t bm_workspace_bytes(int np) {
  return al256(sizeof(BmHeader)) + al256(sizeof(BmProblem) * (size_t)(np > 0 ? np : 1));
}

namespace {

template <int TN>
int bm_single_grid(long long* grid) {
  static std::atomic<bool> attr{false};
  return bm_grid(regular_bm_kernel<TN>, attr, grid);
}

template <int TN>
int bm_batch_grid(long long* grid) {
  static std::atomic<bool> attr{false};
  return bm_grid(regular_bm_batch_kernel<TN>, attr, grid);
}

int bm_rule(int order, int* tn) {
  if (order == BEM_ORDER_EXACT) *tn = 6;
  else if (order == BEM_ORDER_APPROX) *tn = 3;
  else if (order == BEM_ORDER_APPROX_1) *tn = 1;
  else return BEM_ERR_INVALID_ARGUMENT;
  return BEM_OK;
}

template <int TN, int LN>
void bm_single_launch(const BmProblem& P, long long grid, long long items, cudaStream_t s) {
  const GeomView& g = P.g;
  if (items > 0)
    (regular_bm_kernel<TN><<<(unsigned)(grid < items ? grid : items), kBmThreads, sizeof(BmSmem), s>>>(P, (int)items),
     count_launch());
  const int wpb = 4, ppb = wpb * BmSingLanes<LN>::kPairsPerWarp;  // warps, pairs per block
  (singular_bm_kernel<double, 3, LN><<<(g.nt + ppb - 1) / ppb, 32 * wpb, 0, s>>>(P, g.nt), count_launch());
  if (g.n_edge)
    (singular_bm_kernel<float, 2, LN><<<(g.n_edge + ppb - 1) / ppb, 32 * wpb, 0, s>>>(P, g.n_edge),
     count_launch());
  if (g.n_vert)
    (singular_bm_kernel<float, 1, LN><<<(g.n_vert + ppb - 1) / ppb, 32 * wpb, 0, s>>>(P, g.n_vert),
     count_launch());
}

template <int TN, int LN>
void bm_batch_launch(BmHeader* dh, BmProblem* dp, long long grid, long long items, const long long* pairs,
                     cudaStream_t s) {
  if (items > 0)
    (regular_bm_batch_kernel<TN><<<(unsigned)(grid < items ? grid : items), kBmThreads, sizeof(BmSmem), s>>>(dh, dp),
     count_launch());
  const int wpb = 4, ppb = wpb * BmSingLanes<LN>::kPairsPerWarp;  // warps, pairs per block
  if (pairs[0])
    (singular_bm_batch_kernel<double, 3, LN><<<(unsigned)((pairs[0] + ppb - 1) / ppb), 32 * wpb, 0, s>>>(dh, dp),
     count_launch());
  if (pairs[1])
    (singular_bm_batch_kernel<float, 2, LN><<<(unsigned)((pairs[1] + ppb - 1) / ppb), 32 * wpb, 0, s>>>(dh, dp),
     count_launch());
  if (pairs[2])
    (singular_bm_batch_kernel<float, 1, LN><<<(unsigned)((pairs[2] + ppb - 1) / ppb), 32 * wpb, 0, s>>>(dh, dp),
     count_launch());
}

}  // namespace

// lhs = BM_LHS + 1/2 M and rhs = BM_RHS - (i/(2k)) M of one problem (both
// nv x nv complex64, overwritten) at `order` (the reference's <2,3> for
// neumann2dirichlet; <4,6> gives its HBIE system).
int assemble_bm(const GeomView& g, int order, float k, float2* L, float2* R, cudaStream_t s) {
  int rc = bm_check(k, L, R), tn = 0;
  if (rc) return rc;
  if ((rc = bm_rule(order, &tn))) return rc;
  long long grid = 0;
  rc = tn == 6 ? bm_single_grid<6>(&grid) : (tn == 3 ? bm_single_grid<3>(&grid) : bm_single_grid<1>(&grid));
  if (rc) return rc;
  BEM_CUDA_TRY(cudaMemsetAsync(L, 0, sizeof(float2) * (size_t)g.nv * g.nv, s));
  BEM_CUDA_TRY(cudaMemsetAsync(R, 0, sizeof(float2) * (size_t)g.nv * g.nv, s));
  BmProblem P;
  std::memset(&P, 0, sizeof(P));
  P.g = g;
  P.k = k;
  P.n_units = bm_units_of(g);
  const long long chunk = (P.n_units + 8 * grid - 1) / (8 * grid);  // 8 equal items per CTA
  P.chunk = (int)(chunk < 1 ? 1 : chunk);
  P.L = L;
  P.R = R;
  const long long items = (P.n_units + P.chunk - 1) / P.chunk;
  if (tn == 6)
    bm_single_launch<6, 4>(P, grid, items, s);
  else if (tn == 3)
    bm_single_launch<3, 2>(P, grid, items, s);
  else
    bm_single_launch<1, 2>(P, grid, items, s);
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// The same for many problems: one queue-driven launch over every problem's
// regular pairs, one launch per touching-pair type.
int assemble_bm_batch(const GeomView* views, const float* ks, float2* const* Ls, float2* const* Rs, int np, int order,
                      void* ws, size_t ws_bytes, cudaStream_t s) {
  if (np <= 0 || !views || !ks || !Ls || !Rs) return BEM_ERR_INVALID_ARGUMENT;
  if (!ws || ws_bytes < bm_workspace_bytes(np)) return BEM_ERR_WORKSPACE;
  int rc, tn = 0;
  for (int p = 0; p < np; p++)
    if ((rc = bm_check(ks[p], Ls[p], Rs[p]))) return rc;
  if ((rc = bm_rule(order, &tn))) return rc;
  long long grid = 0;
  rc = tn == 6 ? bm_batch_grid<6>(&grid) : (tn == 3 ? bm_batch_grid<3>(&grid) : bm_batch_grid<1>(&grid));
  if (rc) return rc;

  const size_t hbytes = al256(sizeof(BmHeader)), pbytes = sizeof(BmProblem) * (size_t)np;
  BmStage& st = t_bm_stage;
  if (!st.ev) BEM_CUDA_TRY(cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming));
  BEM_CUDA_TRY(cudaEventSynchronize(st.ev));  // the previous upload from the staging buffer is done
  if (st.cap < hbytes + pbytes) {
    if (st.buf) cudaFreeHost(st.buf);
    st.buf = nullptr;
    st.cap = 0;
    BEM_CUDA_TRY(cudaHostAlloc(&st.buf, 2 * (hbytes + pbytes), cudaHostAllocDefault));
    st.cap = 2 * (hbytes + pbytes);
  }
  BmHeader* hh = (BmHeader*)st.buf;
  BmProblem* hp = (BmProblem*)((char*)st.buf + hbytes);
  std::memset(hh, 0, sizeof(BmHeader));
  std::memset(hp, 0, pbytes);
  hh->nproblems = np;
  long long units_all = 0;
  for (int p = 0; p < np; p++) units_all += bm_units_of(views[p]);
  // about 8 items per CTA over the whole batch, at most 64 units per item
  long long chunk = (units_all + 8 * grid - 1) / (8 * grid);
  chunk = chunk < 1 ? 1 : (chunk > 64 ? 64 : chunk);
  long long items = 0, pairs[3] = {0, 0, 0};
  for (int p = 0; p < np; p++) {
    const GeomView& g = views[p];
    BEM_CUDA_TRY(cudaMemsetAsync(Ls[p], 0, sizeof(float2) * (size_t)g.nv * g.nv, s));
    BEM_CUDA_TRY(cudaMemsetAsync(Rs[p], 0, sizeof(float2) * (size_t)g.nv * g.nv, s));
    BmProblem& P = hp[p];
    P.g = g;
    P.k = ks[p];
    P.n_units = bm_units_of(g);
    P.chunk = (int)chunk;
    P.item_begin = items;
    items += (P.n_units + P.chunk - 1) / P.chunk;
    P.pair_begin[0] = pairs[0];
    P.pair_begin[1] = pairs[1];
    P.pair_begin[2] = pairs[2];
    pairs[0] += g.nt;
    pairs[1] += g.n_edge;
    pairs[2] += g.n_vert;
    P.L = Ls[p];
    P.R = Rs[p];
  }
  hh->total_items = items;
  for (int t = 0; t < 3; t++) hh->total_pairs[t] = pairs[t];
  BmHeader* dh = (BmHeader*)ws;
  BmProblem* dp = (BmProblem*)((char*)ws + hbytes);
  BEM_CUDA_TRY(cudaMemcpyAsync(ws, st.buf, hbytes + pbytes, cudaMemcpyHostToDevice, s));
  BEM_CUDA_TRY(cudaEventRecord(st.ev, s));
  if (tn == 6)
    bm_batch_launch<6, 4>(dh, dp, grid, items, pairs, s);
  else if (tn == 3)
    bm_batch_launch<3, 2>(dh, dp, grid, items, pairs, s);
  else
    bm_batch_launch<1, 2>(dh, dp, grid, items, pairs, s);
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

// Reads and clears the flag that a Burton-Miller kernel's bounded wait
// expired (synchronises the stream).
int bm_status(int* err_host, cudaStream_t s) {
  int zero = 0;
  BEM_CUDA_TRY(cudaMemcpyFromSymbolAsync(err_host, g_bm_err, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaMemcpyToSymbolAsync(g_bm_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  return BEM_OK;
}

}  // namespace bemb

// Assembly of the remaining operator types and quadrature orders:
// adjoint double layer, hypersingular, Burton-Miller left/right-hand sides,
// at the <4,6>, <2,3> and <2,1> (singular GL points, triangle-rule points)
// orders of the reference bindings (src/bem/cuda/bind.cu:180-215).
//
// Kernels (potential.h:33-65), with x on the test triangle (normal n_x) and y
// on the trial triangle (normal n_y):
//   ADJOINT_DOUBLE  -e^{ikr}(1-ikr)(x-y).n_x / (4 pi r^3)
//   HYPERSINGULAR   G, recombined per pair as  s9 * (curl_i . curl_j) - s_ab (n_i.n_j) k^2
//   BM_LHS          (-ik n_x.n_y + (1-ikr)(y-x).n_y / r^2) G, plus (i/k) G in slot 9,
//                   recombined as s9 * (curl_i . curl_j) + s_ab
//   BM_RHS          -G + (i/k) G (1-ikr)(x-y).n_x / r^2
// (integrand.h:94-115,216-233,296-323; bind.cu:128-143).  Single and double
// layer at these orders use the same generic path.
//
// Same structure as the fused V/K kernel (32 test triangles per CTA, trial
// tiles of 16 in shared memory, on-chip reduction onto distinct vertices,
// touching pairs masked and integrated by Sauter-Schwab kernels, coincident
// pairs in FP64), with one output and the quadrature points computed from the
// vertices for any rule.

#include <atomic>
#include <cmath>

#include "bem_common.cuh"
#include "sauter_schwab.cuh"

namespace bemb {

namespace {

// ---- triangle rules on the unit triangle, point q dominant at vertex q ----
template <int TN>
__host__ __device__ constexpr double trule_phi(int q, int b);
template <>
__host__ __device__ constexpr double trule_phi<6>(int q, int b) {
  return tri6_phi(q, b);
}
template <>
__host__ __device__ constexpr double trule_phi<3>(int q, int b) {
  return q == b ? 2.0 / 3.0 : 1.0 / 6.0;  // Strang-Fix degree-2 rule
}
template <>
__host__ __device__ constexpr double trule_phi<1>(int, int) {
  return 1.0 / 3.0;  // centroid
}
template <int TN>
__host__ __device__ constexpr double trule_w(int q) {
  return TN == 6 ? tri6_w(q) : (TN == 3 ? 1.0 / 3.0 : 1.0);
}

template <typename R>
__device__ __forceinline__ void sincos_r(R x, R* s, R* c);
template <>
__device__ __forceinline__ void sincos_r<double>(double x, double* s, double* c) {
  sincos(x, s, c);
}
template <>
__device__ __forceinline__ void sincos_r<float>(float x, float* s, float* c) {
  sincosf(x, s, c);
}

// Kernel value (main, aux) without the 1/(4 pi), at d = y - x.
template <int LAYER, typename R>
__device__ __forceinline__ void eval_kernel(R dx, R dy, R dz, R xnx, R xny, R xnz, R ynx, R yny, R ynz, R k,
                                            R& mr, R& mi, R& ar, R& ai) {
  R r = sqrt(dx * dx + dy * dy + dz * dz);
  if (r < R(kEps)) r = R(kEps);
  R s, c;
  sincos_r<R>(k * r, &s, &c);
  const R ir = R(1) / r;
  const R kr = k * r;
  const R A = c + kr * s, B = s - kr * c;  // (1 - ikr) e^{ikr}
  if (LAYER == BEM_SINGLE_LAYER || LAYER == BEM_HYPERSINGULAR) {
    mr = c * ir;
    mi = s * ir;
  } else if (LAYER == BEM_DOUBLE_LAYER) {
    const R f = -(dx * ynx + dy * yny + dz * ynz) * ir * ir * ir;  // (y-x).n_y
    mr = A * f;
    mi = B * f;
  } else if (LAYER == BEM_ADJOINT_DOUBLE_LAYER) {
    const R f = (dx * xnx + dy * xny + dz * xnz) * ir * ir * ir;  // -(x-y).n_x = (y-x).n_x
    mr = A * f;
    mi = B * f;
  } else if (LAYER == BEM_BM_LHS) {
    const R nn = xnx * ynx + xny * yny + xnz * ynz;
    const R f = (dx * ynx + dy * yny + dz * ynz) * ir * ir * ir;  // (y-x).n_y / r^3
    mr = k * nn * s * ir + A * f;
    mi = -k * nn * c * ir + B * f;
    ar = -s * ir / k;  // (i/k) e^{ikr}/r
    ai = c * ir / k;
    return;
  } else {  // BM_RHS
    const R f = -(dx * xnx + dy * xny + dz * xnz) * ir * ir * ir / k;  // (x-y).n_x / (k r^3)
    mr = -c * ir - B * f;
    mi = -s * ir + A * f;
  }
  ar = mr;
  ai = mi;
}

constexpr int kGenThreads = 256;
constexpr int kGenWarps = kGenThreads / 32;
constexpr int kGenSlot = kTileCorners + 1;

struct GenSmem {
  float2 slot[96][kGenSlot];
  TriRec trial[kTile];
  float tverts[kTile][9];
  float tcurl[kTile][9];
  float tnrm[kTile][3];
  TileRec tileJ;
  TileRec tileI[2];
};

__device__ __forceinline__ void copy_words16(void* dst, const void* src, int bytes, int tid, int nthreads) {
  const int4* s = (const int4*)src;
  int4* d = (int4*)dst;
  for (int i = tid; i < bytes / 16; i += nthreads) d[i] = s[i];
}

template <int LAYER, int TN>
__global__ void __launch_bounds__(kGenThreads, 2)
    regular_generic_kernel(GeomView g, float k, const float* __restrict__ normals, const float* __restrict__ curls,
                           float2* __restrict__ out, int chunk, int n_chunks, int n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GenSmem& sm = *reinterpret_cast<GenSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nt = g.nt, nv = g.nv;
  constexpr bool kCurl = (LAYER == BEM_HYPERSINGULAR || LAYER == BEM_BM_LHS);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int grp = item / n_chunks;
    const int ch = item - grp * n_chunks;
    const int tile0 = 2 * grp;
    const bool has_t1 = tile0 + 1 < g.ntiles;
    const int ti = grp * 32 + lane;
    const bool valid_i = ti < nt;
    const TriRec& ri = g.rec[valid_i ? ti : nt - 1];
    const int oi = g.perm[valid_i ? ti : nt - 1];
    float xv[9];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int c = 0; c < 3; c++) xv[3 * a + c] = g.vertices[3 * ri.v[a] + c];
    float ci[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, nip[3] = {0, 0, 0};
    if (kCurl) {
#pragma unroll
      for (int e = 0; e < 9; e++) ci[e] = curls[9 * oi + e];
#pragma unroll
      for (int e = 0; e < 3; e++) nip[e] = normals[3 * oi + e];
    }
    const float area_i = ri.area;
    const int iv0 = ri.v[0], iv1 = ri.v[1], iv2 = ri.v[2];
    __syncthreads();
    copy_words16(&sm.tileI[0], &g.tiles[tile0], sizeof(TileRec), tid, kGenThreads);
    if (has_t1) copy_words16(&sm.tileI[1], &g.tiles[tile0 + 1], sizeof(TileRec), tid, kGenThreads);
    const int jt_begin = ch * chunk;
    const int jt_end = min(jt_begin + chunk, g.ntiles);
    for (int jt = jt_begin; jt < jt_end; jt++) {
      __syncthreads();
      copy_words16(&sm.tileJ, &g.tiles[jt], sizeof(TileRec), tid, kGenThreads);
      const int ntriJ = min(kTile, nt - jt * kTile);
      copy_words16(sm.trial, &g.rec[jt * kTile], ntriJ * (int)sizeof(TriRec), tid, kGenThreads);
      __syncthreads();
      for (int e = tid; e < ntriJ * 9; e += kGenThreads) {
        const int t = e / 9, c = e - 9 * t;
        sm.tverts[t][c] = g.vertices[3 * sm.trial[t].v[c / 3] + c % 3];
        if (kCurl) sm.tcurl[t][c] = curls[9 * g.perm[jt * kTile + t] + c];
      }
      if (kCurl)
        for (int e = tid; e < ntriJ * 3; e += kGenThreads)
          sm.tnrm[e / 3][e % 3] = normals[3 * g.perm[jt * kTile + e / 3] + e % 3];
      __syncthreads();
#pragma unroll 1
      for (int tt = warp; tt < ntriJ; tt += kGenWarps) {
        const TriRec& rj = sm.trial[tt];
        float res[20];
#pragma unroll
        for (int e = 0; e < 20; e++) res[e] = 0.f;
#pragma unroll
        for (int p = 0; p < TN; p++) {
          float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll
          for (int b = 0; b < 3; b++) {
            const float f = (float)trule_phi<TN>(p, b);
            px += f * xv[3 * b];
            py += f * xv[3 * b + 1];
            pz += f * xv[3 * b + 2];
          }
#pragma unroll
          for (int q = 0; q < TN; q++) {
            float qx = 0.f, qy = 0.f, qz = 0.f;
#pragma unroll
            for (int b = 0; b < 3; b++) {
              const float f = (float)trule_phi<TN>(q, b);
              qx += f * sm.tverts[tt][3 * b];
              qy += f * sm.tverts[tt][3 * b + 1];
              qz += f * sm.tverts[tt][3 * b + 2];
            }
            float mr, mi, ar, ai;
            eval_kernel<LAYER, float>(qx - px, qy - py, qz - pz, ri.n[0], ri.n[1], ri.n[2], rj.n[0], rj.n[1],
                                      rj.n[2], k, mr, mi, ar, ai);
            const float w = (float)(trule_w<TN>(p) * trule_w<TN>(q));
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
              for (int b = 0; b < 3; b++) {
                const float f = w * (float)(trule_phi<TN>(p, a) * trule_phi<TN>(q, b));
                res[2 * (3 * a + b)] += f * mr;
                res[2 * (3 * a + b) + 1] += f * mi;
              }
            res[18] += w * ar;
            res[19] += w * ai;
          }
        }
        if (kCurl) {
          float nn = nip[0] * sm.tnrm[tt][0] + nip[1] * sm.tnrm[tt][1] + nip[2] * sm.tnrm[tt][2];
#pragma unroll
          for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
              const float cp = ci[3 * a] * sm.tcurl[tt][3 * b] + ci[3 * a + 1] * sm.tcurl[tt][3 * b + 1] +
                               ci[3 * a + 2] * sm.tcurl[tt][3 * b + 2];
              float& re = res[2 * (3 * a + b)];
              float& im = res[2 * (3 * a + b) + 1];
              if (LAYER == BEM_HYPERSINGULAR) {
                re = res[18] * cp - re * nn * k * k;
                im = res[19] * cp - im * nn * k * k;
              } else {
                re = res[18] * cp + re;
                im = res[19] * cp + im;
              }
            }
        }
        const int j0 = rj.v[0], j1 = rj.v[1], j2 = rj.v[2];
        const bool touching = (iv0 == j0) | (iv0 == j1) | (iv0 == j2) | (iv1 == j0) | (iv1 == j1) | (iv1 == j2) |
                              (iv2 == j0) | (iv2 == j1) | (iv2 == j2);
        const float sc = (valid_i && !touching) ? area_i * rj.area * kInv4Pi : 0.f;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++)
            sm.slot[3 * lane + a][3 * tt + b] = make_float2(res[2 * (3 * a + b)] * sc, res[2 * (3 * a + b) + 1] * sc);
      }
      __syncthreads();
      const int nI0 = sm.tileI[0].nlv;
      const int nI1 = has_t1 ? sm.tileI[1].nlv : 0;
      const int nJ = sm.tileJ.nlv;
      const int total = (nI0 + nI1) * nJ;
      for (int e = tid; e < total; e += kGenThreads) {
        const int ai = e / nJ;
        const int b = e - ai * nJ;
        const int s = ai >= nI0;
        const int a = ai - s * nI0;
        const TileRec& TI = sm.tileI[s];
        float2 acc = make_float2(0.f, 0.f);
        for (int ca = TI.lv_ptr[a]; ca < TI.lv_ptr[a + 1]; ca++) {
          const int row = s * kTileCorners + TI.lv_corner[ca];
          for (int cb = sm.tileJ.lv_ptr[b]; cb < sm.tileJ.lv_ptr[b + 1]; cb++) {
            const float2 v = sm.slot[row][sm.tileJ.lv_corner[cb]];
            acc.x += v.x;
            acc.y += v.y;
          }
        }
        atomicAdd(&out[(size_t)TI.vid[a] * nv + sm.tileJ.vid[b]], acc);
      }
    }
  }
}

// Sauter-Schwab singular pairs for a generic kernel (integrand.h:63-185),
// re-ordering as in the fused V/K kernel; 10 slots; curl recombination.
template <typename R, int LAYER, int LN, int NCOMMON>
__global__ void __launch_bounds__(128)
    singular_generic_kernel(GeomView g, const int2* __restrict__ pairs, int npairs, float k,
                            const float* __restrict__ normals, const float* __restrict__ curls,
                            float2* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pair >= npairs) return;
  const int ti = NCOMMON == 3 ? pair : pairs[pair].x;
  const int tj = NCOMMON == 3 ? pair : pairs[pair].y;
  const int s0 = g.triangles[3 * ti], s1 = g.triangles[3 * ti + 1], s2 = g.triangles[3 * ti + 2];
  const int t0 = g.triangles[3 * tj], t1 = g.triangles[3 * tj + 1], t2 = g.triangles[3 * tj + 2];
  const Perm6 pm = reorder6<NCOMMON>(s0, s1, s2, t0, t1, t2);
  const int pi_[3] = {pm.i0, pm.i1, pm.i2}, pj_[3] = {pm.j0, pm.j1, pm.j2};
  R a[3][3], b[3][3], oa[3][3], ob[3][3];
  const int sv[3] = {s0, s1, s2}, tv[3] = {t0, t1, t2};
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
  R acc[20];
#pragma unroll
  for (int e = 0; e < 20; e++) acc[e] = 0;
  const R kk = (R)k;
  constexpr int NPT = LN * LN * LN * LN;
  auto region = [&](R x1, R x2, R y1, R y2, R ww) {
    const R lx[3] = {R(1) - x1, x1 - x2, x2};
    const R ly[3] = {R(1) - y1, y1 - y2, y2};
    R xp[3], yp[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      xp[d] = lx[0] * a[0][d] + lx[1] * a[1][d] + lx[2] * a[2][d];
      yp[d] = ly[0] * b[0][d] + ly[1] * b[1][d] + ly[2] * b[2][d];
    }
    R mr, mi, ar, ai;
    eval_kernel<LAYER, R>(yp[0] - xp[0], yp[1] - xp[1], yp[2] - xp[2], ni[0], ni[1], ni[2], nj[0], nj[1], nj[2], kk,
                          mr, mi, ar, ai);
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++) {
        const R f = lx[ii] * ly[jj] * ww;
        acc[2 * (3 * ii + jj)] += mr * f;
        acc[2 * (3 * ii + jj) + 1] += mi * f;
      }
    acc[18] += ar * ww;
    acc[19] += ai * ww;
  };
  const R jw = Ji * Jj / R(16);
#pragma unroll 1
  for (int pt = lane; pt < NPT; pt += 32) {
    const int i0 = pt / (LN * LN * LN), i1 = (pt / (LN * LN)) % LN, i2 = (pt / LN) % LN, i3 = pt % LN;
    const R xi = R(0.5) * (R(gl_x<LN>(i0)) + R(1)), e1 = R(0.5) * (R(gl_x<LN>(i1)) + R(1));
    const R e2 = R(0.5) * (R(gl_x<LN>(i2)) + R(1)), e3 = R(0.5) * (R(gl_x<LN>(i3)) + R(1));
    const R w0 = R(gl_w<LN>(i0)) * R(gl_w<LN>(i1)) * R(gl_w<LN>(i2)) * R(gl_w<LN>(i3)) * jw;
    ss_regions<NCOMMON, R>(xi, e1, e2, e3, w0, region);
  }
#pragma unroll
  for (int e = 0; e < 20; e++) {
    R v = acc[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[e] = v;
  }
  if (lane < 9) {
    const int ii = lane / 3, jj = lane % 3;  // re-ordered slots
    const int ia = pi_[ii], jb = pj_[jj];    // original local vertices
    R re = acc[2 * lane], im = acc[2 * lane + 1];
    if (LAYER == BEM_HYPERSINGULAR || LAYER == BEM_BM_LHS) {
      R cp = 0, nn = 0;
      for (int d = 0; d < 3; d++) {
        cp += (R)curls[9 * ti + 3 * ia + d] * (R)curls[9 * tj + 3 * jb + d];
        nn += (R)normals[3 * ti + d] * (R)normals[3 * tj + d];
      }
      if (LAYER == BEM_HYPERSINGULAR) {
        re = acc[18] * cp - re * nn * kk * kk;
        im = acc[19] * cp - im * nn * kk * kk;
      } else {
        re = acc[18] * cp + re;
        im = acc[19] * cp + im;
      }
    }
    const R sc = R(kInv4Pi);
    atomicAdd(&out[(size_t)sel3(s0, s1, s2, ia) * g.nv + sel3(t0, t1, t2, jb)],
              make_float2((float)(re * sc), (float)(im * sc)));
  }
}

template <int LAYER, int TN>
int launch_regular_generic(const GeomView& g, float k, const float* normals, const float* curls, float2* out,
                           cudaStream_t s) {
  const int smem = (int)sizeof(GenSmem);
  static std::atomic<bool> attr{false};
  if (!attr.load(std::memory_order_acquire)) {
    BEM_CUDA_TRY(cudaFuncSetAttribute(regular_generic_kernel<LAYER, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    attr.store(true, std::memory_order_release);
  }
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  BEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, regular_generic_kernel<LAYER, TN>, kGenThreads,
                                                             smem));
  const int grid = sms * (occ > 0 ? occ : 1);
  const int n_groups = (g.nt + 31) / 32;
  int chunk = (int)((long long)n_groups * g.ntiles / (8LL * grid));
  chunk = chunk < 1 ? 1 : (chunk > 64 ? 64 : chunk);
  const int n_chunks = (g.ntiles + chunk - 1) / chunk;
  const int n_items = n_groups * n_chunks;
  (regular_generic_kernel<LAYER, TN><<<grid < n_items ? grid : n_items, kGenThreads, smem, s>>>(
       g, k, normals, curls, out, chunk, n_chunks, n_items),
   count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

template <int LAYER, int LN>
int launch_singular_generic(const GeomView& g, float k, const float* normals, const float* curls, float2* out,
                            cudaStream_t s) {
  const int wpb = 4;
  (singular_generic_kernel<double, LAYER, LN, 3><<<(g.nt + wpb - 1) / wpb, 32 * wpb, 0, s>>>(g, nullptr, g.nt, k,
                                                                                              normals, curls, out),
   count_launch());
  if (g.n_edge)
    (singular_generic_kernel<float, LAYER, LN, 2><<<(g.n_edge + wpb - 1) / wpb, 32 * wpb, 0, s>>>(
         g, g.edge_pairs, g.n_edge, k, normals, curls, out),
     count_launch());
  if (g.n_vert)
    (singular_generic_kernel<float, LAYER, LN, 1><<<(g.n_vert + wpb - 1) / wpb, 32 * wpb, 0, s>>>(
         g, g.vert_pairs, g.n_vert, k, normals, curls, out),
     count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  return BEM_OK;
}

template <int LAYER>
int assemble_layer(const GeomView& g, int order, float k, const float* normals, const float* curls, float2* out,
                   cudaStream_t s) {
  int rc;
  if (order == BEM_ORDER_EXACT) {
    if ((rc = launch_regular_generic<LAYER, 6>(g, k, normals, curls, out, s))) return rc;
    return launch_singular_generic<LAYER, 4>(g, k, normals, curls, out, s);
  }
  if (order == BEM_ORDER_APPROX) {
    if ((rc = launch_regular_generic<LAYER, 3>(g, k, normals, curls, out, s))) return rc;
  } else {
    if ((rc = launch_regular_generic<LAYER, 1>(g, k, normals, curls, out, s))) return rc;
  }
  return launch_singular_generic<LAYER, 2>(g, k, normals, curls, out, s);
}

}  // namespace

int assemble_generic(const GeomView& g, int layer, int order, float k, const float* normals, const float* curls,
                     float2* out, cudaStream_t s) {
  if (!normals) normals = g.normals;
  if (!curls) curls = g.curls;
  BEM_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * (size_t)g.nv * g.nv, s));
  switch (layer) {
    case BEM_SINGLE_LAYER: return assemble_layer<BEM_SINGLE_LAYER>(g, order, k, normals, curls, out, s);
    case BEM_DOUBLE_LAYER: return assemble_layer<BEM_DOUBLE_LAYER>(g, order, k, normals, curls, out, s);
    case BEM_ADJOINT_DOUBLE_LAYER: return assemble_layer<BEM_ADJOINT_DOUBLE_LAYER>(g, order, k, normals, curls, out, s);
    case BEM_HYPERSINGULAR: return assemble_layer<BEM_HYPERSINGULAR>(g, order, k, normals, curls, out, s);
    case BEM_BM_LHS: return assemble_layer<BEM_BM_LHS>(g, order, k, normals, curls, out, s);
    case BEM_BM_RHS: return assemble_layer<BEM_BM_RHS>(g, order, k, normals, curls, out, s);
  }
  return BEM_ERR_INVALID_ARGUMENT;
}

}  // namespace bemb

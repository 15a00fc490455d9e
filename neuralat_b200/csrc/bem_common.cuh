// Shared definitions for the B200 boundary-element kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/bem_b200.h"

namespace bemb {

// ---- quadrature ---------------------------------------------------------
// Six-point degree-4 triangle rule (Dunavant), the rule the reference uses for
// regular pairs, the mass matrix and listener potentials
// (src/bem/cuda/include/gauss.h:106-126).  Points are given by barycentric
// orbits (a, a, 1-2a); weights sum to one.  Point q has its dominant
// barycentric weight at local vertex q % 3, which the kernels exploit.
constexpr double kTriA1 = 0.44594849091596489;   // orbit 1: (1-2a1) on the dominant vertex
constexpr double kTriA2 = 0.091576213509770743;  // orbit 2
constexpr double kTriW1 = 0.22338158967801147;
constexpr double kTriW2 = 0.10995174365532187;

// barycentric coordinate of quadrature point q (0..5) at local vertex b (0..2)
__host__ __device__ constexpr double tri6_phi(int q, int b) {
  return (q < 3) ? ((q == b) ? 1.0 - 2.0 * kTriA1 : kTriA1) : ((q - 3 == b) ? 1.0 - 2.0 * kTriA2 : kTriA2);
}
__host__ __device__ constexpr double tri6_w(int q) { return q < 3 ? kTriW1 : kTriW2; }
// The rule is symmetric: w_q phi_b(q) = tri6_w_common(q) + tri6_w_own(q) [b == tri6_own(q)].
__host__ __device__ constexpr int tri6_own(int q) { return q < 3 ? q : q - 3; }
__host__ __device__ constexpr double tri6_w_common(int q) { return tri6_w(q) * (q < 3 ? kTriA1 : kTriA2); }
__host__ __device__ constexpr double tri6_w_own(int q) { return tri6_w(q) * (1.0 - 3.0 * (q < 3 ? kTriA1 : kTriA2)); }

// Gauss-Legendre 4-point rule on [-1, 1] (gauss.h:44-54).
constexpr double kGL4x0 = 0.86113631159405258, kGL4x1 = 0.33998104358485626;
constexpr double kGL4w0 = 0.34785484513745385, kGL4w1 = 0.65214515486254614;
__host__ __device__ constexpr double gl4_x(int i) {
  return i == 0 ? kGL4x0 : i == 1 ? kGL4x1 : i == 2 ? -kGL4x1 : -kGL4x0;
}
__host__ __device__ constexpr double gl4_w(int i) { return (i == 0 || i == 3) ? kGL4w0 : kGL4w1; }

constexpr float kEps = 1e-3f;  // r clamp of the reference kernels (potential.h:16-23)

// ---- packed FP32 pairs (sm_100 f32x2 arithmetic) ---------------------------
// One instruction applies the same IEEE round-to-nearest operation to both
// lanes of a float2, so a packed expression gives bit-identical results to
// the two scalar ones while issuing half the instructions.
// e / d for 0 <= e < 2^24 and d >= 1, with rd = 1.f / d computed once by the
// caller: a float multiply and one correction step instead of an integer
// division sequence in the inner loops.
__device__ __forceinline__ int div_by(int e, int d, float rd) {
  int q = __float2int_rz((float)e * rd);
  const int r = e - q * d;
  q += (r >= d) - (r < 0);
  return q;
}

__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
constexpr double kPi = 3.14159265358979323846;
constexpr float kInv4Pi = (float)(1.0 / (4.0 * kPi));

// ---- geometry -------------------------------------------------------------
// One record per triangle, 32 words.  Quadrature points in rule order
// (q = 0..5), unit normal, centroid, area = J/2, and the three vertex ids.
struct __align__(16) TriRec {
  float qp[18];
  float n[3];
  float c[3];
  float area;
  int v[3];
  float h;  // n . v0 (plane offset)
  float pad;
};
static_assert(sizeof(TriRec) == 128, "TriRec must be 128 bytes");

// Burton-Miller companion record, sorted order: the points of the 3-point
// degree-2 triangle rule (phi = 2/3 at the point's own vertex, 1/6 at the
// others; weights 1/3) used by the <2,3> Burton-Miller bindings, and the
// surface curls n x grad(phi_b) of the three P1 functions (rows b).
struct __align__(16) BmRec {
  float qp[9];
  float curl[9];
  float pad[2];
};
static_assert(sizeof(BmRec) == 80, "BmRec must be 80 bytes");

constexpr int kTile = 16;               // triangles per geometry tile
constexpr int kTileCorners = 3 * kTile;  // 48

// Per-tile local-vertex tables, one per 16-triangle tile of the sorted order.
struct __align__(16) TileRec {
  int nlv;                       // number of distinct vertices in the tile
  int ntri;                      // triangles in the tile (last tile may be short)
  int pad0, pad1;
  int vid[kTileCorners];         // global vertex id of each local vertex (ascending)
  uint8_t corner_lv[kTileCorners];     // local vertex of corner (3*t + a)
  uint8_t lv_ptr[kTileCorners + 4];    // CSR: corners of local vertex l are lv_corner[lv_ptr[l]..lv_ptr[l+1])
  uint8_t lv_corner[kTileCorners];
  uint8_t pad2[12];
};
static_assert(sizeof(TileRec) % 16 == 0, "TileRec alignment");

// Header at the start of the geometry workspace.  All offsets in bytes from
// the start of the workspace.
struct GeomHeader {
  uint32_t magic;
  int nv, nt, ntiles;
  int n_edge, n_vert;  // ordered singular pairs sharing 2 / 1 vertices
  int max_valence;
  int err;  // status word: set to 1 by an assembly kernel whose bounded wait expired on this geometry
  uint64_t off_vertices;   // float[nv*3] (copy of the input)
  uint64_t off_triangles;  // int[nt*3] (copy of the input)
  uint64_t off_perm;       // int[nt]  sorted position -> triangle id
  uint64_t off_trirec;     // TriRec[nt] in sorted order
  uint64_t off_trirec_orig;  // TriRec[nt] in input order
  uint64_t off_tiles;      // TileRec[ntiles]
  uint64_t off_edge_pairs;  // int2[n_edge]  (test tri, trial tri), input ids
  uint64_t off_vert_pairs;  // int2[n_vert]
  uint64_t off_normals;    // float[nt*3]
  uint64_t off_curls;      // float[nt*9]   rows: n x grad(phi_b)
  uint64_t off_bmrec;      // BmRec[nt] in sorted order
  uint64_t bytes;
};
constexpr uint32_t kGeomMagic = 0x42454D33u;  // "BEM3"

// Device-side view of a built geometry.
struct GeomView {
  int nv, nt, ntiles, n_edge, n_vert;
  const float* vertices;
  const int* triangles;
  const int* perm;
  const TriRec* rec;       // sorted order
  const TriRec* rec_orig;  // input order
  const TileRec* tiles;
  const int2* edge_pairs;
  const int2* vert_pairs;
  const float* normals;
  const float* curls;
  const BmRec* bm;         // sorted order
  int* err;                // the header's status word (GeomHeader::err)
};

// Symmetric regular-pair work units (test tile g, trial tile jt >= g) in
// order: test tile g owns the ntiles - g trial tiles from itself on, so
// U(g) = g ntiles - g (g - 1) / 2 units come before it.
__device__ __forceinline__ long long tile_units_before(long long g, long long n) { return g * n - g * (g - 1) / 2; }

__device__ __forceinline__ int tile_group_of(long long pos, int n) {
  const double b = 2.0 * n + 1.0;
  const double disc = b * b - 8.0 * (double)pos;
  long long g = (long long)((b - sqrt(disc > 0.0 ? disc : 0.0)) * 0.5);
  if (g < 0) g = 0;
  if (g > n - 1) g = n - 1;
  while (g + 1 < n && tile_units_before(g + 1, n) <= pos) g++;
  while (g > 0 && tile_units_before(g, n) > pos) g--;
  return (int)g;
}

// ---- small math -------------------------------------------------------------
// sine and cosine of one argument: the library sincos in FP64
template <typename R>
__device__ __forceinline__ void sincos_t(R x, R* s, R* c);
template <>
__device__ __forceinline__ void sincos_t<double>(double x, double* s, double* c) {
  sincos(x, s, c);
}
// FP32 (edge and vertex pairs of the touching-pair kernels): the hardware
// approximation, accurate to a few 1e-7 absolute for the |k r| <= ~1 of
// touching triangles (the regular kernels use it at larger arguments).
template <>
__device__ __forceinline__ void sincos_t<float>(float x, float* s, float* c) {
  __sincosf(x, s, c);
}

// 1 / r and r from r^2 (r clamped to kEps as in potential.h): rsqrt in FP32, a
// correctly rounded sqrt and division in FP64.
template <typename R>
__device__ __forceinline__ void inv_dist(R r2, R* r, R* inv_r);
template <>
__device__ __forceinline__ void inv_dist<double>(double r2, double* r, double* inv_r) {
  double rr = sqrt(r2);
  if (rr < kEps) rr = kEps;
  *r = rr;
  *inv_r = 1.0 / rr;
}
template <>
__device__ __forceinline__ void inv_dist<float>(float r2, float* r, float* inv_r) {
  const float ri = fminf(rsqrtf(r2), 1.0f / kEps);
  *inv_r = ri;
  *r = fmaxf(r2 * ri, kEps);
}

struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 make3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct d3 {
  double x, y, z;
};
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross3(d3 a, d3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

__device__ __forceinline__ void atomic_add_c64(float2* p, float re, float im) {
  atomicAdd(p, make_float2(re, im));  // vector red.global.add.v2.f32 (sm_90+)
}

}  // namespace bemb

namespace bemb {
// process-wide count of kernel launches issued by this library (host side)
void count_launch();
void count_launches(unsigned long long n);
unsigned long long launch_count();
}  // namespace bemb

// error-checking helper for host code inside the library
#define BEM_CUDA_TRY(expr)                          \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) return BEM_ERR_CUDA;     \
  } while (0)

// Geometry set-up: validation, per-triangle quadrature records, locality
// sorted 16-triangle tiles and touching-pair lists.
//
// The reference recomputes everything per assembly call and discovers the
// touching pairs of every triangle with an O(T) scan per block
// (src/bem/cuda/bind.cu:81-97, capped at 64 neighbours by `adj[64]`).  Here
// the combinatorics are done once, exactly, on the host (no cap), and the
// floating-point records are computed on the device in FP64 and rounded.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "bem_common.cuh"

namespace bemb {

namespace {

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Spread the low 10 bits of v so that there are two zero bits between each.
inline uint32_t part1by2(uint32_t v) {
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000FF;
  v = (v | (v << 8)) & 0x0300F00F;
  v = (v | (v << 4)) & 0x030C30C3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}

struct HostGeom {
  int nv = 0, nt = 0, ntiles = 0;
  std::vector<float> vertices;
  std::vector<int> triangles;
  std::vector<int> perm;
  std::vector<TileRec> tiles;
  std::vector<int2> edge_pairs, vert_pairs;
  int max_valence = 0;
  GeomHeader hdr{};
};

int analyse_host(HostGeom& g);

// The most recent analysis of this host thread: bem_geometry_bytes followed by
// bem_geometry_build on an unchanged mesh analyses it once, and a rebuild of
// an unchanged mesh re-uploads its staged integer tables.
thread_local HostGeom t_last;
thread_local bool t_last_valid = false;

// Pinned host buffer of this thread (grown on demand).
struct PinnedBuf {
  char* p = nullptr;
  size_t cap = 0;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
  int ensure(size_t n) {
    if (cap >= n) return BEM_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    BEM_CUDA_TRY(cudaHostAlloc((void**)&p, n, cudaHostAllocDefault));
    cap = n;
    return BEM_OK;
  }
};
thread_local PinnedBuf t_download;  // the mesh read back for the comparison with t_last
thread_local PinnedBuf t_stage;     // t_last's integer tables as uploaded (valid if t_stage_ok)
thread_local bool t_stage_ok = false;

// Analysis of the mesh on the device (t_last; valid until the next call on
// this thread).
int analyse(const float* d_vertices, int nv, const int* d_triangles, int nt, cudaStream_t s, const HostGeom** out) {
  if (nv <= 0 || nt <= 0 || !d_vertices || !d_triangles) return BEM_ERR_INVALID_ARGUMENT;
  const size_t vb = sizeof(float) * 3 * (size_t)nv, tb = sizeof(int) * 3 * (size_t)nt;
  int rc = t_download.ensure(vb + tb);
  if (rc) return rc;
  BEM_CUDA_TRY(cudaMemcpyAsync(t_download.p, d_vertices, vb, cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaMemcpyAsync(t_download.p + vb, d_triangles, tb, cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  if (t_last_valid && t_last.nv == nv && t_last.nt == nt && std::memcmp(t_last.vertices.data(), t_download.p, vb) == 0 &&
      std::memcmp(t_last.triangles.data(), t_download.p + vb, tb) == 0) {
    *out = &t_last;
    return BEM_OK;
  }
  t_last_valid = false;
  t_stage_ok = false;
  t_last = HostGeom{};
  t_last.nv = nv;
  t_last.nt = nt;
  t_last.vertices.assign((const float*)t_download.p, (const float*)t_download.p + 3 * (size_t)nv);
  t_last.triangles.assign((const int*)(t_download.p + vb), (const int*)(t_download.p + vb) + 3 * (size_t)nt);
  rc = analyse_host(t_last);
  if (rc) return rc;
  t_last_valid = true;
  *out = &t_last;
  return BEM_OK;
}

int analyse_host(HostGeom& g) {
  const int nv = g.nv, nt = g.nt;

  for (size_t i = 0; i < g.vertices.size(); i++)
    if (!std::isfinite(g.vertices[i])) return BEM_ERR_NONFINITE;
  for (int i = 0; i < nt; i++) {
    const int* t = &g.triangles[3 * (size_t)i];
    for (int a = 0; a < 3; a++)
      if (t[a] < 0 || t[a] >= nv) return BEM_ERR_INDEX;
    if (t[0] == t[1] || t[1] == t[2] || t[0] == t[2]) return BEM_ERR_DEGENERATE;
    double p[3][3];
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) p[a][c] = g.vertices[3 * (size_t)t[a] + c];
    double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
    if (!(cx * cx + cy * cy + cz * cz > 0.0)) return BEM_ERR_DEGENERATE;
  }

  // Morton order of centroids (10 bits per axis over the bounding box).
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int v = 0; v < nv; v++)
    for (int c = 0; c < 3; c++) {
      lo[c] = std::min(lo[c], (double)g.vertices[3 * (size_t)v + c]);
      hi[c] = std::max(hi[c], (double)g.vertices[3 * (size_t)v + c]);
    }
  double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-30});
  std::vector<uint64_t> key(nt);
  for (int i = 0; i < nt; i++) {
    uint32_t q[3];
    for (int c = 0; c < 3; c++) {
      double m = 0.0;
      for (int a = 0; a < 3; a++) m += g.vertices[3 * (size_t)g.triangles[3 * (size_t)i + a] + c];
      m = (m / 3.0 - lo[c]) / ext;
      q[c] = (uint32_t)std::min(1023.0, std::max(0.0, std::floor(m * 1024.0)));
    }
    uint64_t code = part1by2(q[0]) | (part1by2(q[1]) << 1) | (part1by2(q[2]) << 2);
    key[i] = (code << 32) | (uint32_t)i;
  }
  std::sort(key.begin(), key.end());
  g.perm.resize(nt);
  for (int s2 = 0; s2 < nt; s2++) g.perm[s2] = (int)(key[s2] & 0xffffffffu);

  // 16-triangle tiles with local vertex tables.
  g.ntiles = (nt + kTile - 1) / kTile;
  g.tiles.assign(g.ntiles, TileRec{});
  for (int t = 0; t < g.ntiles; t++) {
    TileRec& tr = g.tiles[t];
    std::memset(&tr, 0, sizeof(TileRec));
    int ntri = std::min(kTile, nt - t * kTile);
    tr.ntri = ntri;
    int ids[kTileCorners];
    int nc = 3 * ntri;
    for (int c = 0; c < nc; c++) ids[c] = g.triangles[3 * (size_t)g.perm[t * kTile + c / 3] + c % 3];
    int uniq[kTileCorners];
    std::copy(ids, ids + nc, uniq);
    std::sort(uniq, uniq + nc);
    int nl = (int)(std::unique(uniq, uniq + nc) - uniq);
    tr.nlv = nl;
    for (int l = 0; l < nl; l++) tr.vid[l] = uniq[l];
    int count[kTileCorners] = {0};
    for (int c = 0; c < nc; c++) {
      int l = (int)(std::lower_bound(uniq, uniq + nl, ids[c]) - uniq);
      tr.corner_lv[c] = (uint8_t)l;
      count[l]++;
    }
    tr.lv_ptr[0] = 0;
    for (int l = 0; l < nl; l++) tr.lv_ptr[l + 1] = (uint8_t)(tr.lv_ptr[l] + count[l]);
    int fill[kTileCorners] = {0};
    for (int c = 0; c < nc; c++) {
      int l = tr.corner_lv[c];
      tr.lv_corner[tr.lv_ptr[l] + fill[l]++] = (uint8_t)c;
    }
  }

  // Vertex stars and touching pairs (exact, no neighbour cap).
  std::vector<int> vptr(nv + 1, 0), vtri(3 * (size_t)nt);
  for (int i = 0; i < 3 * nt; i++) vptr[g.triangles[i] + 1]++;
  for (int v = 0; v < nv; v++) {
    g.max_valence = std::max(g.max_valence, vptr[v + 1]);
    vptr[v + 1] += vptr[v];
  }
  {
    std::vector<int> fill(vptr.begin(), vptr.end() - 1);
    for (int i = 0; i < nt; i++)
      for (int a = 0; a < 3; a++) vtri[fill[g.triangles[3 * (size_t)i + a]]++] = i;
  }
  std::vector<int> seen(nt, -1);
  for (int i = 0; i < nt; i++) {
    const int* ti = &g.triangles[3 * (size_t)i];
    seen[i] = i;
    for (int a = 0; a < 3; a++)
      for (int p = vptr[ti[a]]; p < vptr[ti[a] + 1]; p++) {
        int j = vtri[p];
        if (seen[j] == i) continue;
        seen[j] = i;
        const int* tj = &g.triangles[3 * (size_t)j];
        int common = 0;
        for (int x = 0; x < 3; x++)
          for (int y = 0; y < 3; y++) common += (ti[x] == tj[y]);
        if (common >= 3) return BEM_ERR_DEGENERATE;  // duplicated triangle
        if (common == 2)
          g.edge_pairs.push_back(make_int2(i, j));
        else
          g.vert_pairs.push_back(make_int2(i, j));
      }
  }

  // workspace layout
  GeomHeader& h = g.hdr;
  std::memset(&h, 0, sizeof(h));
  h.magic = kGeomMagic;
  h.nv = nv;
  h.nt = nt;
  h.ntiles = g.ntiles;
  h.n_edge = (int)g.edge_pairs.size();
  h.n_vert = (int)g.vert_pairs.size();
  h.max_valence = g.max_valence;
  uint64_t off = align_up(sizeof(GeomHeader), 256);
  auto take = [&](uint64_t bytes) {
    uint64_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  // host-built tables first (one upload), device-computed records after
  h.off_vertices = take(sizeof(float) * 3 * (size_t)nv);
  h.off_triangles = take(sizeof(int) * 3 * (size_t)nt);
  h.off_perm = take(sizeof(int) * (size_t)nt);
  h.off_tiles = take(sizeof(TileRec) * (size_t)g.ntiles);
  h.off_edge_pairs = take(sizeof(int2) * (size_t)std::max(1, h.n_edge));
  h.off_vert_pairs = take(sizeof(int2) * (size_t)std::max(1, h.n_vert));
  h.off_trirec = take(sizeof(TriRec) * (size_t)nt);
  h.off_trirec_orig = take(sizeof(TriRec) * (size_t)nt);
  h.off_normals = take(sizeof(float) * 3 * (size_t)nt);
  h.off_curls = take(sizeof(float) * 9 * (size_t)nt);
  h.off_bmrec = take(sizeof(BmRec) * (size_t)nt);
  h.bytes = off;
  return BEM_OK;
}

// FP64 per-triangle records; launched over sorted positions.
__global__ void geom_records_kernel(int nt, const float* __restrict__ verts, const int* __restrict__ tris,
                                    const int* __restrict__ perm, TriRec* __restrict__ rec_sorted,
                                    TriRec* __restrict__ rec_orig, float* __restrict__ normals,
                                    float* __restrict__ curls, BmRec* __restrict__ bm) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nt) return;
  int i = perm[s];
  int id[3];
  d3 p[3];
  for (int a = 0; a < 3; a++) {
    id[a] = tris[3 * i + a];
    p[a] = {(double)verts[3 * id[a]], (double)verts[3 * id[a] + 1], (double)verts[3 * id[a] + 2]};
  }
  d3 e1 = sub(p[1], p[0]), e2 = sub(p[2], p[0]);
  d3 cr = cross3(e1, e2);
  double J = sqrt(dot3(cr, cr));
  d3 n = {cr.x / J, cr.y / J, cr.z / J};
  TriRec r;
  for (int q = 0; q < 6; q++) {
    double x = 0, y = 0, z = 0;
    for (int b = 0; b < 3; b++) {
      double f = tri6_phi(q, b);
      x += f * p[b].x;
      y += f * p[b].y;
      z += f * p[b].z;
    }
    r.qp[3 * q] = (float)x;
    r.qp[3 * q + 1] = (float)y;
    r.qp[3 * q + 2] = (float)z;
  }
  r.n[0] = (float)n.x;
  r.n[1] = (float)n.y;
  r.n[2] = (float)n.z;
  r.c[0] = (float)((p[0].x + p[1].x + p[2].x) / 3.0);
  r.c[1] = (float)((p[0].y + p[1].y + p[2].y) / 3.0);
  r.c[2] = (float)((p[0].z + p[1].z + p[2].z) / 3.0);
  r.area = (float)(0.5 * J);
  r.v[0] = id[0];
  r.v[1] = id[1];
  r.v[2] = id[2];
  r.h = (float)dot3(n, p[0]);
  r.pad = 0.f;
  rec_sorted[s] = r;
  rec_orig[i] = r;
  normals[3 * i] = r.n[0];
  normals[3 * i + 1] = r.n[1];
  normals[3 * i + 2] = r.n[2];
  // surface curls n x grad(phi_b) via (J^T J)^-1 (src/bem/solver.py:40-58)
  double g11 = dot3(e1, e1), g12 = dot3(e1, e2), g22 = dot3(e2, e2);
  double det = g11 * g22 - g12 * g12;
  double i11 = g22 / det, i12 = -g12 / det, i22 = g11 / det;
  d3 c1 = {i11 * e1.x + i12 * e2.x, i11 * e1.y + i12 * e2.y, i11 * e1.z + i12 * e2.z};
  d3 c2 = {i12 * e1.x + i22 * e2.x, i12 * e1.y + i22 * e2.y, i12 * e1.z + i22 * e2.z};
  d3 gr[3] = {{-(c1.x + c2.x), -(c1.y + c2.y), -(c1.z + c2.z)}, c1, c2};
  BmRec m;
  for (int b = 0; b < 3; b++) {
    d3 c = cross3(n, gr[b]);
    curls[9 * i + 3 * b] = m.curl[3 * b] = (float)c.x;
    curls[9 * i + 3 * b + 1] = m.curl[3 * b + 1] = (float)c.y;
    curls[9 * i + 3 * b + 2] = m.curl[3 * b + 2] = (float)c.z;
  }
  // 3-point degree-2 rule: point q = 2/3 vertex q + 1/6 (each other vertex)
  for (int q = 0; q < 3; q++) {
    const double own = 2.0 / 3.0 - 1.0 / 6.0, all = 1.0 / 6.0;
    m.qp[3 * q] = (float)(all * (p[0].x + p[1].x + p[2].x) + own * p[q].x);
    m.qp[3 * q + 1] = (float)(all * (p[0].y + p[1].y + p[2].y) + own * p[q].y);
    m.qp[3 * q + 2] = (float)(all * (p[0].z + p[1].z + p[2].z) + own * p[q].z);
  }
  m.pad[0] = m.pad[1] = 0.f;
  bm[s] = m;
}

}  // namespace

// Host-side copies of the headers of geometries built in this process, so
// that assembly calls need not read the header back from the device.
static std::mutex g_cache_mu;
static std::unordered_map<const void*, GeomHeader> g_cache;

static void cache_put(const void* geom, const GeomHeader& h) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_cache[geom] = h;
}

static void cache_drop(const void* geom) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_cache.erase(geom);
}

// Reads the header of a built geometry into a device view (host side).  A
// geometry built elsewhere (copied buffer) is read back with a blocking copy.
int geom_view(const void* geom, GeomView* v, GeomHeader* out_hdr) {
  if (!geom) return BEM_ERR_WORKSPACE;
  GeomHeader h;
  bool hit = false;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find(geom);
    if (it != g_cache.end()) {
      h = it->second;
      hit = true;
    }
  }
  if (!hit) {
    if (cudaMemcpy(&h, geom, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return BEM_ERR_CUDA;
    if (h.magic == kGeomMagic) cache_put(geom, h);
  }
  if (h.magic != kGeomMagic) return BEM_ERR_WORKSPACE;
  const char* b = (const char*)geom;
  v->nv = h.nv;
  v->nt = h.nt;
  v->ntiles = h.ntiles;
  v->n_edge = h.n_edge;
  v->n_vert = h.n_vert;
  v->vertices = (const float*)(b + h.off_vertices);
  v->triangles = (const int*)(b + h.off_triangles);
  v->perm = (const int*)(b + h.off_perm);
  v->rec = (const TriRec*)(b + h.off_trirec);
  v->rec_orig = (const TriRec*)(b + h.off_trirec_orig);
  v->tiles = (const TileRec*)(b + h.off_tiles);
  v->edge_pairs = (const int2*)(b + h.off_edge_pairs);
  v->vert_pairs = (const int2*)(b + h.off_vert_pairs);
  v->normals = (const float*)(b + h.off_normals);
  v->curls = (const float*)(b + h.off_curls);
  v->bm = (const BmRec*)(b + h.off_bmrec);
  v->err = (int*)((char*)geom + offsetof(GeomHeader, err));
  if (out_hdr) *out_hdr = h;
  return BEM_OK;
}

}  // namespace bemb

using namespace bemb;

extern "C" int bem_geometry_bytes(const float* vertices, int nv, const int* triangles, int nt, size_t* bytes,
                                  bem_stream_t stream) {
  if (!bytes) return BEM_ERR_INVALID_ARGUMENT;
  const HostGeom* g = nullptr;
  int rc = analyse(vertices, nv, triangles, nt, (cudaStream_t)stream, &g);
  if (rc) return rc;
  *bytes = (size_t)g->hdr.bytes;
  return BEM_OK;
}

extern "C" int bem_geometry_build(const float* vertices, int nv, const int* triangles, int nt, void* geom,
                                  size_t geom_bytes, bem_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const HostGeom* gp = nullptr;
  int rc = analyse(vertices, nv, triangles, nt, s, &gp);
  if (rc) return rc;
  const HostGeom& g = *gp;
  if (!geom || geom_bytes < g.hdr.bytes) return BEM_ERR_WORKSPACE;
  const GeomHeader& h = g.hdr;
  // the integer tables in one pinned staging buffer (kept while the mesh is
  // unchanged), then one upload
  const size_t nstage = h.off_trirec;
  if (!t_stage_ok) {
    if ((rc = t_stage.ensure(nstage))) return rc;
    char* st = t_stage.p;
    std::memset(st, 0, nstage);
    std::memcpy(st, &h, sizeof(h));
    std::memcpy(st + h.off_vertices, g.vertices.data(), sizeof(float) * 3 * (size_t)nv);
    std::memcpy(st + h.off_triangles, g.triangles.data(), sizeof(int) * 3 * (size_t)nt);
    std::memcpy(st + h.off_perm, g.perm.data(), sizeof(int) * (size_t)nt);
    std::memcpy(st + h.off_tiles, g.tiles.data(), sizeof(TileRec) * (size_t)g.ntiles);
    if (h.n_edge) std::memcpy(st + h.off_edge_pairs, g.edge_pairs.data(), sizeof(int2) * h.n_edge);
    if (h.n_vert) std::memcpy(st + h.off_vert_pairs, g.vert_pairs.data(), sizeof(int2) * h.n_vert);
    t_stage_ok = true;
  }
  BEM_CUDA_TRY(cudaMemcpyAsync(geom, t_stage.p, nstage, cudaMemcpyHostToDevice, s));
  char* b = (char*)geom;
  (geom_records_kernel<<<(nt + 127) / 128, 128, 0, s>>>(
      nt, (const float*)(b + h.off_vertices), (const int*)(b + h.off_triangles), (const int*)(b + h.off_perm),
      (TriRec*)(b + h.off_trirec), (TriRec*)(b + h.off_trirec_orig), (float*)(b + h.off_normals),
      (float*)(b + h.off_curls), (BmRec*)(b + h.off_bmrec)), count_launch());
  BEM_CUDA_TRY(cudaGetLastError());
  BEM_CUDA_TRY(cudaStreamSynchronize(s));  // the staging buffer serves the next build of this thread
  cache_put(geom, h);
  return BEM_OK;
}

extern "C" int bem_geometry_status(const void* geom, bem_stream_t stream) {
  GeomView v;
  int rc = geom_view(geom, &v, nullptr);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int err = 0;
  const int zero = 0;
  BEM_CUDA_TRY(cudaMemcpyAsync(&err, v.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  BEM_CUDA_TRY(cudaMemcpyAsync(v.err, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
  BEM_CUDA_TRY(cudaStreamSynchronize(s));
  return err ? BEM_ERR_CUDA : BEM_OK;
}

extern "C" int bem_geometry_release(const void* geom) {
  if (!geom) return BEM_ERR_INVALID_ARGUMENT;
  cache_drop(geom);
  return BEM_OK;
}

extern "C" int bem_geometry_normals(const void* geom, float* normals, float* curls, bem_stream_t stream) {
  GeomView v;
  int rc = geom_view(geom, &v, nullptr);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (normals)
    BEM_CUDA_TRY(cudaMemcpyAsync(normals, v.normals, sizeof(float) * 3 * (size_t)v.nt, cudaMemcpyDeviceToDevice, s));
  if (curls)
    BEM_CUDA_TRY(cudaMemcpyAsync(curls, v.curls, sizeof(float) * 9 * (size_t)v.nt, cudaMemcpyDeviceToDevice, s));
  return BEM_OK;
}

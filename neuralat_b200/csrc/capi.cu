// extern "C" entry points for assembly, plus status strings.

#include <atomic>
#include <cmath>
#include <vector>

#include "bem_common.cuh"

namespace bemb {
int assembly_status(int* err_host, cudaStream_t s);
int geom_view(const void* geom, GeomView* v, GeomHeader* out_hdr);
int assemble_vk(const GeomView& g, float k, float2* V, float2* Kout, float mass_coeff, float k_coeff, cudaStream_t s);
int assemble_mass(const GeomView& g, float2* M, float coeff, bool zero, cudaStream_t s);
int assemble_generic(const GeomView& g, int layer, int order, float k, const float* normals, const float* curls,
                     float2* out, cudaStream_t s);
int set_tuning(int key, int value);
int get_tuning(int key);
size_t batch_workspace_bytes(int np);
int assemble_vk_batch(const GeomView* views, const float* ks, float2* const* Vs, float2* const* Ks, int np,
                      float mass_coeff, float k_coeff, void* ws, size_t ws_bytes, cudaStream_t s);
int assemble_bm(const GeomView& g, int order, float k, float2* L, float2* R, cudaStream_t s);
size_t bm_workspace_bytes(int np);
int assemble_bm_batch(const GeomView* views, const float* ks, float2* const* Ls, float2* const* Rs, int np, int order,
                      void* ws, size_t ws_bytes, cudaStream_t s);
int bm_status(int* err_host, cudaStream_t s);
}  // namespace bemb

namespace bemb {
static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace bemb

using namespace bemb;

extern "C" unsigned long long bem_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" const char* bem_status_string(int status) {
  switch (status) {
    case BEM_OK: return "ok";
    case BEM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BEM_ERR_INDEX: return "triangle vertex index out of range";
    case BEM_ERR_DEGENERATE: return "degenerate mesh (zero-area, repeated-vertex or duplicated triangle)";
    case BEM_ERR_WORKSPACE: return "workspace missing, too small or not a built geometry";
    case BEM_ERR_NONFINITE: return "non-finite value";
    case BEM_ERR_NOT_CONVERGED: return "iterative solver did not converge";
    case BEM_ERR_BREAKDOWN: return "iterative solver breakdown";
    case BEM_ERR_CUDA: return "CUDA error";
    case BEM_ERR_UNSUPPORTED: return "unsupported request";
  }
  return "unknown status";
}

extern "C" const char* bem_version(void) { return "bemb200 0.1 sm_100a"; }

extern "C" int bem_boundary_matrices_vk(const void* geom, float k, void* v_out, void* k_out, float mass_coeff,
                                        float k_coeff, bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (!std::isfinite(k)) return BEM_ERR_NONFINITE;
  return assemble_vk(g, k, (float2*)v_out, (float2*)k_out, mass_coeff, k_coeff, (cudaStream_t)stream);
}

extern "C" int bem_boundary_matrix(const void* geom, int layer, int order, float k, const float* normals,
                                   const float* curls, void* out, bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (!out) return BEM_ERR_INVALID_ARGUMENT;
  if (layer < BEM_SINGLE_LAYER || layer > BEM_BM_RHS || order < BEM_ORDER_EXACT || order > BEM_ORDER_APPROX_1)
    return BEM_ERR_INVALID_ARGUMENT;
  if (!std::isfinite(k)) return BEM_ERR_NONFINITE;
  cudaStream_t s = (cudaStream_t)stream;
  if (order == BEM_ORDER_EXACT && layer == BEM_SINGLE_LAYER)
    return assemble_vk(g, k, (float2*)out, nullptr, 0.f, 0.f, s);
  if (order == BEM_ORDER_EXACT && layer == BEM_DOUBLE_LAYER)
    return assemble_vk(g, k, nullptr, (float2*)out, 0.f, 1.f, s);
  return assemble_generic(g, layer, order, k, normals, curls, (float2*)out, s);
}

extern "C" int bem_identity_matrix(const void* geom, void* out, bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  if (!out) return BEM_ERR_INVALID_ARGUMENT;
  return assemble_mass(g, (float2*)out, 1.f, true, (cudaStream_t)stream);
}

extern "C" int bem_set_tuning(int key, int value) { return set_tuning(key, value); }
extern "C" int bem_get_tuning(int key) { return get_tuning(key); }
extern "C" size_t bem_batch_workspace_bytes(int nproblems) {
  const size_t a = batch_workspace_bytes(nproblems), b = bm_workspace_bytes(nproblems);
  return a > b ? a : b;
}

extern "C" int bem_boundary_matrices_bm(const void* geom, int order, float k, void* lhs_out, void* rhs_out,
                                        bem_stream_t stream) {
  GeomView g;
  int rc = geom_view(geom, &g, nullptr);
  if (rc) return rc;
  return assemble_bm(g, order, k, (float2*)lhs_out, (float2*)rhs_out, (cudaStream_t)stream);
}

extern "C" int bem_batch_matrices_bm(const bem_bm_problem* problems, int nproblems, int order, void* workspace,
                                     size_t workspace_bytes, bem_stream_t stream) {
  if (!problems || nproblems <= 0) return BEM_ERR_INVALID_ARGUMENT;
  std::vector<GeomView> views(nproblems);
  std::vector<float> ks(nproblems);
  std::vector<float2*> Ls(nproblems), Rs(nproblems);
  for (int p = 0; p < nproblems; p++) {
    int rc = geom_view(problems[p].geom, &views[p], nullptr);
    if (rc) return rc;
    ks[p] = problems[p].k;
    Ls[p] = (float2*)problems[p].lhs_out;
    Rs[p] = (float2*)problems[p].rhs_out;
  }
  return assemble_bm_batch(views.data(), ks.data(), Ls.data(), Rs.data(), nproblems, order, workspace,
                           workspace_bytes, (cudaStream_t)stream);
}

extern "C" int bem_batch_matrices_vk(const bem_batch_problem* problems, int nproblems, float mass_coeff, float k_coeff,
                                     void* workspace, size_t workspace_bytes, bem_stream_t stream) {
  if (!problems || nproblems <= 0) return BEM_ERR_INVALID_ARGUMENT;
  std::vector<GeomView> views(nproblems);
  std::vector<float> ks(nproblems);
  std::vector<float2*> Vs(nproblems), Ks(nproblems);
  for (int p = 0; p < nproblems; p++) {
    int rc = geom_view(problems[p].geom, &views[p], nullptr);
    if (rc) return rc;
    ks[p] = problems[p].k;
    Vs[p] = (float2*)problems[p].v_out;
    Ks[p] = (float2*)problems[p].k_out;
  }
  return assemble_vk_batch(views.data(), ks.data(), Vs.data(), Ks.data(), nproblems, mass_coeff, k_coeff, workspace,
                           workspace_bytes, (cudaStream_t)stream);
}

extern "C" int bem_assembly_status(bem_stream_t stream) {
  int err = 0, err_bm = 0;
  int rc = assembly_status(&err, (cudaStream_t)stream);
  if (rc) return rc;
  if ((rc = bm_status(&err_bm, (cudaStream_t)stream))) return rc;
  return (err || err_bm) ? BEM_ERR_CUDA : BEM_OK;
}

// placeholder for the remaining operator types / quadrature orders
#include "bem_common.cuh"
namespace bemb {
int assemble_generic(const GeomView&, int, int, float, const float*, const float*, float2*, cudaStream_t) {
  return BEM_ERR_UNSUPPORTED;
}
}  // namespace bemb

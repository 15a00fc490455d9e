// placeholder, replaced by the tensor-core operator
#include "bem_common.cuh"
namespace bemb {
size_t tc_workspace_bytes(int, int, int) { return 0; }
int tc_operator_prepare(const float2*, int, int, void*, cudaStream_t) { return BEM_ERR_UNSUPPORTED; }
int tc_matvec(const void*, int, int, const float2*, int, float2*, cudaStream_t) { return BEM_ERR_UNSUPPORTED; }
}  // namespace bemb

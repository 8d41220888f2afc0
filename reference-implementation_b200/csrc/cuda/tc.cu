// Tensor-core path (pack pre-pass + tcgen05 GEMM). Placeholder until the
// kernels land: routes to the CUDA-core kernels.
#include "tb_common.cuh"

namespace tb {
cudaError_t launch_generic(const tb_plan* P, const tb_ptrs* d, cudaStream_t s);

cudaError_t launch_tc(const tb_plan* P, const tb_ptrs* d, int num, cudaStream_t s, int* kernels)
{
    tb_plan q = *P;
    q.path = TB_PATH_GENERIC;
    for (int i = 0; i < num; i++) {
        cudaError_t e = launch_generic(&q, &d[i], s);
        if (e != cudaSuccess) return e;
    }
    *kernels = num;
    return cudaSuccess;
}
}  // namespace tb

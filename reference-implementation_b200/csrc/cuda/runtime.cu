// C ABI of the CUDA layer (tb_cuda.h): pointer queries, stream-ordered
// device memory, copies, timing, launch counting and the dispatch of a launch
// plan to its kernels.
#include <atomic>
#include <cstdio>

#include "../tb_cuda.h"
#include "tb_common.cuh"

namespace tb {

static std::atomic<long long> g_launches{0};

void count_launch(int n) { g_launches += n; }

cudaError_t launch_generic(const tb_plan* P, const tb_ptrs* d, cudaStream_t s);
cudaError_t launch_tc(const tb_plan* P, const tb_ptrs* d, int num, cudaStream_t s, int* kernels);

}  // namespace tb

extern "C" {

int tbk_device_count(int* count)
{
    return (int)cudaGetDeviceCount(count);
}

int tbk_pointer_kind(const void* p, int* kind, int* device)
{
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        // no usable driver/device: report the error
        return (int)e;
    }
    *device = a.device;
    switch (a.type) {
    case cudaMemoryTypeDevice: *kind = TBK_PTR_DEVICE; break;
    case cudaMemoryTypeManaged: *kind = TBK_PTR_MANAGED; break;
    case cudaMemoryTypeHost: *kind = TBK_PTR_HOST_PINNED; break;
    default: *kind = TBK_PTR_HOST; break;
    }
    return 0;
}

int tbk_get_device(int* dev) { return (int)cudaGetDevice(dev); }
int tbk_set_device(int dev) { return (int)cudaSetDevice(dev); }

int tbk_malloc(void** p, size_t bytes, void* stream)
{
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(p, bytes, (cudaStream_t)stream);
    if (e != cudaSuccess) (void)cudaGetLastError();
    return (int)e;
}

int tbk_free(void* p, void* stream)
{
    return (int)cudaFreeAsync(p, (cudaStream_t)stream);
}

int tbk_memcpy(void* dst, const void* src, size_t bytes, int dir, void* stream)
{
    cudaMemcpyKind k = dir == TBK_H2D ? cudaMemcpyHostToDevice : dir == TBK_D2H ? cudaMemcpyDeviceToHost
                                                                              : cudaMemcpyDeviceToDevice;
    return (int)cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream);
}

int tbk_stream_sync(void* stream)
{
    return (int)cudaStreamSynchronize((cudaStream_t)stream);
}

struct tb_timer {
    cudaEvent_t a, b;
};

int tbk_timer_begin(void* stream, void** timer)
{
    tb_timer* t = new tb_timer;
    cudaEventCreate(&t->a);
    cudaEventCreate(&t->b);
    *timer = t;
    return (int)cudaEventRecord(t->a, (cudaStream_t)stream);
}

int tbk_timer_end(void* stream, void* timer)
{
    return (int)cudaEventRecord(((tb_timer*)timer)->b, (cudaStream_t)stream);
}

int tbk_timer_elapsed_us(void* timer, double* us)
{
    tb_timer* t = (tb_timer*)timer;
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(t->b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t->a, t->b);
    *us = 1000.0 * ms;
    cudaEventDestroy(t->a);
    cudaEventDestroy(t->b);
    delete t;
    return (int)e;
}

int tbk_run_plan(const tb_plan* plan, const tb_ptrs* ptrs, void* stream, int* kernels)
{
    cudaStream_t s = (cudaStream_t)stream;
    *kernels = 0;
    cudaError_t e = cudaSuccess;
    switch (plan->path) {
    case TB_PATH_NOOP: return 0;
    case TB_PATH_TC: e = tb::launch_tc(plan, ptrs, 1, s, kernels); break;
    default:
        e = tb::launch_generic(plan, ptrs, s);
        *kernels = 1;
        break;
    }
    return (int)e;
}

int tbk_run_plan_batched(const tb_plan* plan, const tb_ptrs* ptrs, int num, void* stream, int* kernels)
{
    cudaStream_t s = (cudaStream_t)stream;
    *kernels = 0;
    if (plan->path == TB_PATH_TC) return (int)tb::launch_tc(plan, ptrs, num, s, kernels);
    for (int i = 0; i < num; i++) {
        int k = 0;
        int e = tbk_run_plan(plan, &ptrs[i], stream, &k);
        *kernels += k;
        if (e) return e;
    }
    return 0;
}

long long tbk_launch_count(void) { return tb::g_launches.load(); }

const char* tbk_error_string(int err) { return cudaGetErrorString((cudaError_t)err); }

}  // extern "C"

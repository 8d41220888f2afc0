// C ABI of the CUDA layer (tb_cuda.h): pointer queries, stream-ordered
// device memory, copies, timing, launch counting and the dispatch of a launch
// plan to its kernels.
#include <cuda.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "../tb_cuda.h"
#include "tb_common.cuh"

namespace tb {

static std::atomic<long long> g_launches{0};
static std::atomic<long long> g_allocations{0};

void count_launch(int n) { g_launches += n; }
void count_allocation() { g_allocations++; }

// One device word per GPU that kernels set when a bounded wait expires; the
// host reads and clears it after synchronous executions.
static int* g_err_word[64];
static std::mutex g_err_mutex;

int* device_error_word()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_err_mutex);
    if (!g_err_word[dev]) {
        int* p = nullptr;
        count_allocation();
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) return nullptr;
        g_err_word[dev] = p;
    }
    return g_err_word[dev];
}

// The library's own stream-ordered memory pool per GPU. Its release
// threshold is unlimited, so scratch and staging buffers freed by one call
// are reused by the next instead of being unmapped at every synchronisation
// (the device default pool's threshold of 0 would do that).
static cudaMemPool_t g_pool[64];
static std::mutex g_pool_mutex;

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    count_allocation();
    if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, s);
    {
        std::lock_guard<std::mutex> lk(g_pool_mutex);
        if (!g_pool[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t pool;
            e = cudaMemPoolCreate(&pool, &props);
            if (e != cudaSuccess) return e;
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            g_pool[dev] = pool;
        }
    }
    return cudaMallocFromPoolAsync(p, bytes, g_pool[dev], s);
}

// Small host-to-device copies of launch descriptors (pointer arrays) through
// a page-locked ring per device, so that they are truly asynchronous: slot i
// is reused only after the copy that last read it has run (an event per
// slot). Larger blocks go through pageable memory.
constexpr int RING_SLOTS = 64;
constexpr size_t RING_SLOT_BYTES = 64 << 10;
struct StageRing {
    char* host = nullptr;
    cudaEvent_t ev[RING_SLOTS];
    bool used[RING_SLOTS];
    int next = 0;
};
static StageRing g_ring[64];
static std::mutex g_ring_mutex;

cudaError_t stage_copy(void* dev_dst, const void* src, size_t bytes, cudaStream_t s)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (bytes > RING_SLOT_BYTES || dev < 0 || dev >= 64)
        return cudaMemcpyAsync(dev_dst, src, bytes, cudaMemcpyHostToDevice, s);
    std::lock_guard<std::mutex> lk(g_ring_mutex);
    StageRing& r = g_ring[dev];
    if (!r.host) {
        count_allocation();
        e = cudaMallocHost((void**)&r.host, RING_SLOTS * RING_SLOT_BYTES);
        if (e != cudaSuccess) {
            r.host = nullptr;
            return cudaMemcpyAsync(dev_dst, src, bytes, cudaMemcpyHostToDevice, s);
        }
        for (int i = 0; i < RING_SLOTS; i++) {
            cudaEventCreateWithFlags(&r.ev[i], cudaEventDisableTiming);
            r.used[i] = false;
        }
    }
    const int i = r.next;
    r.next = (r.next + 1) % RING_SLOTS;
    if (r.used[i]) {
        e = cudaEventSynchronize(r.ev[i]);
        if (e != cudaSuccess) return e;
    }
    char* slot = r.host + (size_t)i * RING_SLOT_BYTES;
    memcpy(slot, src, bytes);
    e = cudaMemcpyAsync(dev_dst, slot, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(r.ev[i], s);
    r.used[i] = e == cudaSuccess;
    return e;
}

cudaError_t launch_generic(const tb_plan* P, const tb_ptrs* d, cudaStream_t s, int* kernels);
cudaError_t launch_simt(const tb_plan* P, const tb_ptrs* d, cudaStream_t s);
cudaError_t launch_tc(const tb_plan* P, const tb_ptrs* d, int num, cudaStream_t s, int* kernels, void** main_timer);
size_t group_descriptor_bytes(int n);
size_t simt_scratch_bytes(const tb_plan* P);
size_t sliced_scratch_bytes(const tb_plan* P);
cudaError_t launch_sliced(const tb_plan* P, const tb_ptrs* d, cudaStream_t s, int* kernels, void** main_timer);
size_t reduce_scratch_bytes(const tb_plan* P, size_t real_bytes);
cudaError_t launch_generic_group(const tb_plan* const* P, const tb_ptrs* d, int n, void* host, void* dev,
                                 cudaStream_t s);
size_t group_tc_bytes(int n);
size_t loop_slot_bytes();
void loop_fill(void* slot, const tb_plan* P, const tb_ptrs* d);
size_t loop_state_bytes(int nslots, int blocks);
cudaError_t loop_launch(void* slots_dev, void* state, int nslots, int blocks, unsigned long long idle_ns,
                        cudaStream_t s);
cudaError_t launch_group_tc(const tb_plan* const* P, const tb_ptrs* d, int n, void* host, void* dev, int tile,
                            cudaStream_t s, int64_t* tiles_out);

static void CUDART_CB free_host_buffer(void* p) { free(p); }

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

typedef CUresult (*PointerAttrFn)(void*, CUpointer_attribute, CUdeviceptr);

static PointerAttrFn pointer_attr_fn()
{
    static PointerAttrFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PointerAttrFn)p;
    });
    return fn;
}

int tbk_pointer_range(const void* p, int* kind, int* device, uintptr_t* start, size_t* size)
{
    int e = tbk_pointer_kind(p, kind, device);
    *start = (uintptr_t)p;
    *size = 1;
    if (e || (*kind != TBK_PTR_DEVICE && *kind != TBK_PTR_MANAGED)) return e;
    PointerAttrFn fn = pointer_attr_fn();
    CUdeviceptr st = 0;
    size_t sz = 0;
    if (fn && fn(&st, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, (CUdeviceptr)p) == CUDA_SUCCESS &&
        fn(&sz, CU_POINTER_ATTRIBUTE_RANGE_SIZE, (CUdeviceptr)p) == CUDA_SUCCESS && sz > 0) {
        *start = (uintptr_t)st;
        *size = sz;
    }
    return 0;
}

int tbk_get_device(int* dev) { return (int)cudaGetDevice(dev); }
int tbk_set_device(int dev) { return (int)cudaSetDevice(dev); }

int tbk_malloc(void** p, size_t bytes, void* stream)
{
    if (bytes == 0) bytes = 16;
    cudaError_t e = tb::pool_alloc(p, bytes, (cudaStream_t)stream);
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

int tbk_run_plan(const tb_plan* plan, const tb_ptrs* ptrs, void* stream, int* kernels, void** main_timer)
{
    cudaStream_t s = (cudaStream_t)stream;
    *kernels = 0;
    cudaError_t e = cudaSuccess;
    switch (plan->path) {
    case TB_PATH_NOOP: return 0;
    case TB_PATH_TC: e = tb::launch_tc(plan, ptrs, 1, s, kernels, main_timer); break;
    case TB_PATH_SLICED: e = tb::launch_sliced(plan, ptrs, s, kernels, main_timer); break;
    case TB_PATH_SIMT:
        if (main_timer) tbk_timer_begin(stream, main_timer);
        e = tb::launch_simt(plan, ptrs, s);
        if (main_timer) tbk_timer_end(stream, *main_timer);
        *kernels = 1;
        break;
    default:
        if (main_timer) tbk_timer_begin(stream, main_timer);
        e = tb::launch_generic(plan, ptrs, s, kernels);
        if (main_timer) tbk_timer_end(stream, *main_timer);
        break;
    }
    return (int)e;
}

int tbk_run_plan_batched(const tb_plan* plan, const tb_ptrs* ptrs, int num, void* stream, int* kernels)
{
    cudaStream_t s = (cudaStream_t)stream;
    *kernels = 0;
    if (plan->path == TB_PATH_TC) return (int)tb::launch_tc(plan, ptrs, num, s, kernels, nullptr);
    if (plan->path == TB_PATH_GENERIC && num > 1) {
        // one grouped launch; the descriptors go through a host buffer that a
        // stream callback frees once the copy has run
        const size_t bytes = tb::group_descriptor_bytes(num);
        void* host = malloc(bytes);
        const tb_plan** plans = (const tb_plan**)malloc(sizeof(tb_plan*) * (size_t)num);
        if (!host || !plans) {
            free(host);
            free(plans);
            return (int)cudaErrorMemoryAllocation;
        }
        for (int i = 0; i < num; i++) plans[i] = plan;
        void* dev = nullptr;
        cudaError_t e = tb::pool_alloc(&dev, bytes, s);
        if (e == cudaSuccess) {
            e = tb::launch_generic_group(plans, ptrs, num, host, dev, s);
            cudaFreeAsync(dev, s);
        }
        free(plans);
        if (e == cudaSuccess) e = cudaLaunchHostFunc(s, tb::free_host_buffer, host);
        else {
            cudaStreamSynchronize(s);
            free(host);
        }
        *kernels = 1;
        return (int)e;
    }
    for (int i = 0; i < num; i++) {
        int k = 0;
        int e = tbk_run_plan(plan, &ptrs[i], stream, &k, nullptr);
        *kernels += k;
        if (e) return e;
    }
    return 0;
}

int tbk_stream_create(void** stream)
{
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    *stream = s;
    return (int)e;
}

int tbk_stream_destroy(void* stream) { return (int)cudaStreamDestroy((cudaStream_t)stream); }

int tbk_host_func(void* stream, void (*fn)(void*), void* arg)
{
    return (int)cudaLaunchHostFunc((cudaStream_t)stream, fn, arg);
}

int tbk_event_create(void** ev)
{
    cudaEvent_t e = nullptr;
    cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    *ev = e;
    return (int)r;
}

int tbk_event_record(void* ev, void* stream) { return (int)cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream); }

int tbk_host_alloc(void** p, size_t bytes)
{
    tb::count_allocation();
    return (int)cudaMallocHost(p, bytes);
}
int tbk_host_free(void* p) { return (int)cudaFreeHost(p); }

size_t tbk_group_bytes(int n) { return tb::group_descriptor_bytes(n); }

size_t tbk_scratch_bytes(const tb_plan* plan)
{
    switch (plan->path) {
    case TB_PATH_TC: return tbk_tc_scratch_bytes(plan);
    case TB_PATH_SIMT: return tb::simt_scratch_bytes(plan);
    case TB_PATH_SLICED: return tb::sliced_scratch_bytes(plan);
    case TB_PATH_REDUCE:
        return tb::reduce_scratch_bytes(plan, plan->compute == TB_R32 || plan->compute == TB_C32 ? 4 : 8);
    default: return 0;
    }
}

size_t tbk_group_tc_bytes(int n) { return tb::group_tc_bytes(n); }

int tbk_run_group_tc(const tb_plan* const* plans, const tb_ptrs* ptrs, int n, void* host_desc, void* dev_desc, int tile,
                     void* stream, int64_t* tiles)
{
    return (int)tb::launch_group_tc(plans, ptrs, n, host_desc, dev_desc, tile, (cudaStream_t)stream, tiles);
}

// One grouped tensor-core launch with descriptor buffers of its own: a host
// buffer freed by a stream callback once its copy has run, device memory
// from the pool.
int tbk_run_group_tc_owned(const tb_plan* const* plans, const tb_ptrs* ptrs, int n, int tile, void* stream,
                           int64_t* tiles)
{
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = tb::group_tc_bytes(n);
    void* host = malloc(bytes);
    if (!host) return (int)cudaErrorMemoryAllocation;
    void* dev = nullptr;
    cudaError_t e = tb::pool_alloc(&dev, bytes, s);
    if (e == cudaSuccess) {
        e = tb::launch_group_tc(plans, ptrs, n, host, dev, tile, s, tiles);
        cudaFreeAsync(dev, s);
    }
    if (e == cudaSuccess) e = cudaLaunchHostFunc(s, tb::free_host_buffer, host);
    else {
        cudaStreamSynchronize(s);
        free(host);
    }
    return (int)e;
}

int tbk_run_group(const tb_plan* const* plans, const tb_ptrs* ptrs, int n, void* host_desc, void* dev_desc,
                  void* stream)
{
    for (int i = 0; i < n; i++)
        if (plans[i]->path != TB_PATH_GENERIC || plans[i]->compute != plans[0]->compute)
            return (int)cudaErrorInvalidValue;
    return (int)tb::launch_generic_group(plans, ptrs, n, host_desc, dev_desc, (cudaStream_t)stream);
}

// ---- device-resident request loop (host/loop.c) ----
size_t tbk_loop_slot_bytes(void) { return tb::loop_slot_bytes(); }
void tbk_loop_fill(void* slot, const tb_plan* P, const tb_ptrs* d) { tb::loop_fill(slot, P, d); }

// page-locked host memory mapped into the device's address space
int tbk_host_alloc_mapped(void** host, void** dev, size_t bytes)
{
    tb::count_allocation();
    cudaError_t e = cudaHostAlloc(host, bytes, cudaHostAllocMapped);
    if (e != cudaSuccess) return (int)e;
    memset(*host, 0, bytes);
    e = cudaHostGetDevicePointer(dev, *host, 0);
    if (e != cudaSuccess) {
        cudaFreeHost(*host);
        *host = nullptr;
    }
    return (int)e;
}

// the device state of a loop (tb::loop_state_bytes), zeroed
int tbk_loop_state(void** state, int nslots, int blocks)
{
    tb::count_allocation();
    const size_t bytes = tb::loop_state_bytes(nslots, blocks);
    cudaError_t e = cudaMalloc(state, bytes);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaMemset(*state, 0, bytes);
}

// launches the loop on `stream` and records `*event` (created on first use) after it
int tbk_loop_launch(void* slots_dev, void* state, int nslots, int blocks, unsigned long long idle_ns, void* stream,
                    void** event)
{
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (!*event) e = cudaEventCreateWithFlags((cudaEvent_t*)event, cudaEventDisableTiming);
    if (e == cudaSuccess) e = tb::loop_launch(slots_dev, state, nslots, blocks, idle_ns, s);
    if (e == cudaSuccess) e = cudaEventRecord((cudaEvent_t)*event, s);
    return (int)e;
}

// 1 when the work before the event has run, 0 while it runs, a negative code on error
int tbk_event_done(void* event)
{
    cudaError_t e = cudaEventQuery((cudaEvent_t)event);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) {
        (void)cudaGetLastError();
        return 0;
    }
    return -(int)e;
}

void tbk_event_destroy(void* event)
{
    if (event) cudaEventDestroy((cudaEvent_t)event);
}

int tbk_dev_free(void* p) { return (int)cudaFree(p); }

long long tbk_launch_count(void) { return tb::g_launches.load(); }
long long tbk_allocation_count(void) { return tb::g_allocations.load(); }

int tbk_check_device_error(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || !tb::g_err_word[dev]) return 0;
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, tb::g_err_word[dev], sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    if (v) {
        cudaMemset(tb::g_err_word[dev], 0, sizeof(int));
        return (int)cudaErrorLaunchTimeout;
    }
    return 0;
}

const char* tbk_error_string(int err) { return cudaGetErrorString((cudaError_t)err); }

}  // extern "C"

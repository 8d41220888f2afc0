/*
 * C ABI of the CUDA layer. The host library (C) calls only these functions;
 * they are implemented in the .cu translation units. Return values are 0 on
 * success or a cudaError_t value.
 */
#ifndef TB_CUDA_H_
#define TB_CUDA_H_

#include <stddef.h>
#include <stdint.h>

#include "tb_plan.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { TBK_PTR_HOST = 0, TBK_PTR_HOST_PINNED = 1, TBK_PTR_DEVICE = 2, TBK_PTR_MANAGED = 3 };
enum { TBK_H2D = 0, TBK_D2H = 1, TBK_D2D = 2 };
enum { TBK_ERR_NOMEM = 2 };  /* cudaErrorMemoryAllocation */

int tbk_device_count(int* count);
int tbk_wait_selftest(unsigned long long limit_ns, int* out);
int tbk_simt_kernel(const tb_plan* P);
int tbk_generic_kernel(const tb_plan* P);
int tbk_tc_split_in_place(const tb_plan* P);
int tbk_pointer_kind(const void* p, int* kind, int* device);
/* as tbk_pointer_kind; for device and managed memory also the allocation
 * holding p, [start, start + size) */
int tbk_pointer_range(const void* p, int* kind, int* device, uintptr_t* start, size_t* size);
int tbk_get_device(int* dev);
int tbk_set_device(int dev);
int tbk_malloc(void** p, size_t bytes, void* stream);
int tbk_free(void* p, void* stream);
int tbk_memcpy(void* dst, const void* src, size_t bytes, int dir, void* stream);
int tbk_stream_sync(void* stream);

/* Device time between two points on a stream: begin records an event pair
 * slot, end records the second event; elapsed waits for it. */
int tbk_timer_begin(void* stream, void** timer);
int tbk_timer_end(void* stream, void* timer);
int tbk_timer_elapsed_us(void* timer, double* us);   /* frees the timer */

/* Runs the plan on device-accessible operands. kernels receives the number
 * of kernels launched. When main_timer is not NULL, a timer (see
 * tbk_timer_*) around the dominant kernel is returned through it. */
int tbk_run_plan(const tb_plan* plan, const tb_ptrs* ptrs, void* stream, int* kernels, void** main_timer);

/* Runs the plan on num independent operand sets in one grouped launch
 * where the path allows it. */
int tbk_run_plan_batched(const tb_plan* plan, const tb_ptrs* ptrs, int num, void* stream, int* kernels);

/* Streams (non-blocking) and host callbacks ordered on a stream; fn runs on
 * a driver thread once the work before it has completed and must not call
 * CUDA. */
int tbk_stream_create(void** stream);
int tbk_stream_destroy(void* stream);
int tbk_host_func(void* stream, void (*fn)(void*), void* arg);
/* Completion events (no timing): recorded on a stream, polled with
 * tbk_event_done and freed with tbk_event_destroy (below). */
int tbk_event_create(void** ev);
int tbk_event_record(void* ev, void* stream);
int tbk_host_alloc(void** p, size_t bytes);   /* page-locked host memory */
int tbk_host_free(void* p);

/* One launch for n products of the CUDA-core element path that share a
 * compute domain (tb_plan.compute). host_desc (page-locked) and dev_desc hold
 * tbk_group_bytes(n) bytes each and must stay valid until the launch has run. */
size_t tbk_group_bytes(int n);
/* device scratch one execution of the plan allocates from the pool */
size_t tbk_scratch_bytes(const tb_plan* plan);
int tbk_run_group(const tb_plan* const* plans, const tb_ptrs* ptrs, int n, void* host_desc, void* dev_desc,
                  void* stream);

/* Grouped tensor-core products (group.cu): n products of different plans,
 * each a real binary32 product of the tensor-core path (16-bit precisions or
 * split bfloat16) whose A and B the converter warps read in place
 * (tbk_tc_groupable), run in one launch with tile shape `tile` (1: 256 x 256
 * on CTA pairs, 2: 128 x 128). host_desc is host memory of
 * tbk_group_tc_bytes(n) that must stay untouched until the stream has run the
 * copy; dev_desc device memory of the same size. *tiles receives the number
 * of tiles launched. The _owned form allocates and frees both itself. */
size_t tbk_group_tc_bytes(int n);
int tbk_tc_groupable(const tb_plan* plan, const void* A, const void* B);
int tbk_tc_group_same_as_solo(const tb_plan* plan);
int tbk_run_group_tc(const tb_plan* const* plans, const tb_ptrs* ptrs, int n, void* host_desc, void* dev_desc, int tile,
                     void* stream, int64_t* tiles);
int tbk_run_group_tc_owned(const tb_plan* const* plans, const tb_ptrs* ptrs, int n, int tile, void* stream,
                           int64_t* tiles);

/* Device-resident request loop (generic.cu: k_request_loop; host/loop.c):
 * slots of tbk_loop_slot_bytes() in mapped host memory, the loop's state in
 * device memory (ring copy, sequence words, arrival counters, per-block
 * tickets), launch + completion event. */
size_t tbk_loop_slot_bytes(void);
void tbk_loop_fill(void* slot, const tb_plan* plan, const tb_ptrs* ptrs);
int tbk_host_alloc_mapped(void** host, void** dev, size_t bytes);
int tbk_loop_state(void** state, int nslots, int blocks);
int tbk_loop_launch(void* slots_dev, void* state, int nslots, int blocks, unsigned long long idle_ns, void* stream,
                    void** event);
int tbk_event_done(void* event);
void tbk_event_destroy(void* event);
int tbk_dev_free(void* p);

long long tbk_launch_count(void);
long long tbk_allocation_count(void);

/* Reads (and clears) the word kernels set when one of their bounded waits
 * expired; returns 0 or a cudaError_t value. Synchronises the device. */
int tbk_check_device_error(void);
const char* tbk_error_string(int err);

/* Allocation-free tensor-core product: scratch from a fixed device array of
 * the library (tbk_noalloc_capacity() bytes); see tc.cu. */
size_t tbk_noalloc_capacity(void);
size_t tbk_tc_scratch_bytes(const tb_plan* plan);
int tbk_run_plan_tc_noalloc(const tb_plan* plan, const tb_ptrs* ptrs, void* stream, int* kernels);
int tbk_noalloc_check_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TB_CUDA_H_ */

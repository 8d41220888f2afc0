/*
 * tapp_b200_execute_product_noalloc: the tensor product for callers that
 * cannot allocate device memory while they run it (a memory manager or an
 * allocator callback that calls into the library, or a program that has
 * handed the whole device to its own pool). It has no counterpart in the
 * reference.
 *
 * It runs the same tensor-core kernels as TAPP_execute_product, but takes the
 * packed operand panels from a fixed 32 MiB device array that the library
 * owns; this path of the library calls neither cudaMalloc, cudaFree nor any
 * other device or host allocator (validation included: the self-aliasing
 * check needs no temporaries). Consequences:
 *   - all four operand pointers must be device pointers (host operands would
 *     need staging buffers);
 *   - only products that the tensor cores run qualify (BF16BF16_ACCUM_F32,
 *     F16F16_ACCUM_F32/F16, or F32 in split-bfloat16 mode);
 *   - a product whose panels need more than the array holds is rejected with
 *     TAPP_B200_ERR_SCRATCH before any launch;
 *   - the first call on a device looks the array's device address up (make
 *     it before any stream capture), and calls whose work overlaps on the GPU
 *     share the array and race on it;
 *   - a synchronous call reports a bounded wait that expired in its kernels
 *     (TAPP_B200_ERR_CUDA); an asynchronous call returns before they run, so
 *     such an expiry is reported by the next synchronous call on the device.
 */
#include <string.h>

#include "tb_internal.h"

TAPP_error tapp_b200_execute_product_noalloc(TAPP_tensor_product plan, TAPP_executor exec, const void* alpha,
                                             const void* A, const void* B, const void* beta, const void* C, void* D)
{
    struct tb_product* p = (struct tb_product*)plan;
    if (!p || p->magic != TB_MAGIC_PRODUCT) return TAPP_B200_ERR_INVALID;
    tb_tensor_view v[4];
    for (int k = 0; k < 4; k++) {
        const struct tb_info* t = (const struct tb_info*)p->info[k];
        if (t->nmode > p->nidx[k]) return TAPP_B200_ERR_LABELS;
        v[k].type = t->type;
        v[k].nmode = t->nmode;
        v[k].op = p->op[k];
        v[k].extents = t->extents;
        v[k].strides = t->strides;
        v[k].idx = p->idx[k];
    }
    int err = tb_validate(&v[0], &v[1], &v[2], &v[3], beta, C != NULL);
    if (err) return err;

    /* executor (the reference's code 33 for NULL or unknown ids) */
    void* stream = NULL;
    int async = 0, f32_mode = 0;
    if (!exec) return 33;
    if (tb_executor_is_ours(exec)) {
        const struct tb_executor* e = (const struct tb_executor*)exec;
        stream = e->stream;
        async = e->async;
        f32_mode = e->f32_mode;
    } else {
        int id = *(const int*)exec;
        if (id != 1 && id != 2 && id != 12) return 33;
    }

    tb_plan P;
    tb_plan_options opt = {f32_mode, TB_PATH_TC, 0};
    err = tb_build_plan(&v[0], &v[1], &v[2], &v[3], p->prec, alpha, beta, &opt, &P);
    if (err) return err;
    if (P.path == TB_PATH_NOOP) return 0;
    if (P.path != TB_PATH_TC) return TAPP_B200_ERR_UNSUPPORTED;

    const void* ptr[4] = {A, B, C, D};
    int device = -1;
    for (int k = 0; k < 4; k++) {
        if (!ptr[k] || (k == 2 && P.beta_zero)) continue;
        int kind = 0, d = -1;
        int e = tbk_pointer_kind(ptr[k], &kind, &d);
        if (e) return TAPP_B200_ERR_CUDA;
        if (kind != TBK_PTR_DEVICE && kind != TBK_PTR_MANAGED) return TAPP_B200_ERR_INVALID;
        if (device < 0) device = d;
    }
    if (device >= 0 && tbk_set_device(device)) return TAPP_B200_ERR_CUDA;
    if (tbk_tc_scratch_bytes(&P) > tbk_noalloc_capacity()) return TAPP_B200_ERR_SCRATCH;

    tb_ptrs dp = {A, B, P.beta_zero ? NULL : C, D};
    int kernels = 0;
    int e = tbk_run_plan_tc_noalloc(&P, &dp, stream, &kernels);
    if (e) return e == TBK_ERR_NOMEM ? TAPP_B200_ERR_SCRATCH : TAPP_B200_ERR_CUDA;
    if (!async) {
        if (tbk_stream_sync(stream)) return TAPP_B200_ERR_CUDA;
        if (tbk_noalloc_check_error()) return TAPP_B200_ERR_CUDA;
    }
    return 0;
}

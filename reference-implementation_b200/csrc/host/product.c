/*
 * Tensor products: TAPP_create_tensor_product, TAPP_destroy_tensor_product,
 * TAPP_execute_product and TAPP_execute_batched_product.
 *
 * create/destroy follow reference_implementation/src/product.c:66-128: the
 * product copies the four label arrays and keeps the four tensor infos by
 * reference, so execute sees their contents at call time; nothing is checked
 * at creation. execute follows product.c:130-465 up to the point where the
 * reference starts its element loop: the same validation chain and codes,
 * then the product runs on the GPU from a launch plan cached on the product.
 *
 * Operand pointers may be device pointers (used in place) or host pointers
 * (each addressed span is copied to the device, and D's span copied back).
 */
#include <stdlib.h>
#include <string.h>

#include "tb_internal.h"

static int64_t* dup_labels(const int64_t* idx, int n)
{
    int64_t* p = malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (p && n > 0) memcpy(p, idx, sizeof(int64_t) * (size_t)n);
    return p;
}

/* product.c:66-117 */
TAPP_error TAPP_create_tensor_product(TAPP_tensor_product* plan, TAPP_handle handle,
                                      TAPP_element_op op_A, TAPP_tensor_info A, const int64_t* idx_A,
                                      TAPP_element_op op_B, TAPP_tensor_info B, const int64_t* idx_B,
                                      TAPP_element_op op_C, TAPP_tensor_info C, const int64_t* idx_C,
                                      TAPP_element_op op_D, TAPP_tensor_info D, const int64_t* idx_D,
                                      TAPP_prectype prec)
{
    struct tb_product* p = calloc(1, sizeof(*p));
    if (!p) return TAPP_B200_ERR_NOMEM;
    p->magic = TB_MAGIC_PRODUCT;
    p->handle = handle;
    TAPP_element_op ops[4] = {op_A, op_B, op_C, op_D};
    TAPP_tensor_info infos[4] = {A, B, C, D};
    const int64_t* idx[4] = {idx_A, idx_B, idx_C, idx_D};
    for (int k = 0; k < 4; k++) {
        p->op[k] = ops[k];
        p->info[k] = infos[k];
        p->nidx[k] = ((struct tb_info*)infos[k])->nmode;
        p->idx[k] = dup_labels(idx[k], p->nidx[k]);
    }
    p->prec = prec;
    pthread_mutex_init(&p->lock, NULL);
    *plan = (TAPP_tensor_product)p;
    return 0;
}

/* product.c:119-128 */
TAPP_error TAPP_destroy_tensor_product(TAPP_tensor_product plan)
{
    struct tb_product* p = (struct tb_product*)plan;
    if (!p) return 0;
    for (int k = 0; k < 4; k++) free(p->idx[k]);
    free(p->cache.key);
    pthread_mutex_destroy(&p->lock);
    p->magic = 0;
    free(p);
    return 0;
}

/* check_executor_existence, product.c:878-885 (code 33) */
static int resolve_executor(TAPP_executor exec, tb_exec_settings* s)
{
    memset(s, 0, sizeof(*s));
    if (!exec) return 33;
    if (tb_executor_is_ours(exec)) {
        const struct tb_executor* e = (const struct tb_executor*)exec;
        s->stream = e->stream;
        s->async = e->async;
        s->f32_mode = e->f32_mode;
        s->force_path = e->force_path;
        s->want_status = e->want_status;
        s->server = e->server;
        s->f64_mode = e->f64_mode;
        s->tile = e->tile;
        return 0;
    }
    int id = *(const int*)exec;
    return (id == 1 || id == 2 || id == 12) ? 0 : 33;
}

int tb_product_views(struct tb_product* p, tb_tensor_view v[4])
{
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
    return 0;
}

/* Launch plans depend on the infos' contents, the scalars (rounded per
 * precision) and the executor's options; a cached plan is reused when all
 * of them match. */
int tb_product_plan(struct tb_product* p, const tb_tensor_view v[4], const void* alpha, const void* beta,
                    const tb_exec_settings* s, tb_plan* out)
{
    int64_t key[4 * (3 * 64 + 2) + 8];
    int n = 0, fits = 1;
    for (int k = 0; k < 4 && fits; k++) {
        if (v[k].nmode > 64) { fits = 0; break; }
        key[n++] = v[k].type;
        key[n++] = v[k].nmode;
        for (int i = 0; i < v[k].nmode; i++) {
            key[n++] = v[k].extents[i];
            key[n++] = v[k].strides[i];
        }
    }
    tb_plan_options opt = {s->f32_mode, s->force_path, s->f64_mode};
    int err;
    if (fits) {
        pthread_mutex_lock(&p->lock);
        struct tb_plan_cache* c = &p->cache;
        if (c->valid && c->key_len == n && !memcmp(c->key, key, sizeof(int64_t) * (size_t)n) &&
            c->f32_mode == s->f32_mode && c->force_path == s->force_path && c->f64_mode == s->f64_mode) {
            *out = c->plan;
            pthread_mutex_unlock(&p->lock);
            /* scalars may change per call; beta's zero-ness changes the plan */
            if (!tb_plan_set_scalars(out, alpha, beta)) return 0;
            return tb_build_plan(&v[0], &v[1], &v[2], &v[3], p->prec, alpha, beta, &opt, out);
        }
        pthread_mutex_unlock(&p->lock);
    }
    err = tb_build_plan(&v[0], &v[1], &v[2], &v[3], p->prec, alpha, beta, &opt, out);
    if (err || !fits) return err;
    pthread_mutex_lock(&p->lock);
    struct tb_plan_cache* c = &p->cache;
    int64_t* k2 = realloc(c->key, sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (k2) {
        c->key = k2;
        memcpy(c->key, key, sizeof(int64_t) * (size_t)n);
        c->key_len = n;
        c->f32_mode = s->f32_mode;
        c->force_path = s->force_path;
        c->f64_mode = s->f64_mode;
        c->plan = *out;
        c->valid = 1;
    }
    pthread_mutex_unlock(&p->lock);
    return 0;
}

/* lowest and highest element offset a layout addresses; 0 if it addresses none */
int tb_span_of(const tb_tensor_view* t, int64_t* lo, int64_t* hi)
{
    *lo = *hi = 0;
    for (int i = 0; i < t->nmode; i++) {
        if (t->extents[i] == 0) return 0;
        int64_t r = t->strides[i] * (t->extents[i] - 1);
        if (r < 0) *lo += r; else *hi += r;
    }
    return 1;
}

/* whether every element of the span is addressed (no holes) */
int tb_span_dense(const tb_tensor_view* t, int64_t lo, int64_t hi)
{
    int64_t count = 1;
    for (int i = 0; i < t->nmode; i++) count *= t->extents[i];
    /* repeated labels address a diagonal only */
    for (int i = 0; i < t->nmode; i++)
        for (int j = 0; j < i; j++)
            if (t->idx[i] == t->idx[j]) return 0;
    return count == hi - lo + 1;
}

static int cuda_err(int e) { return e == TBK_ERR_NOMEM ? TAPP_B200_ERR_NOMEM : TAPP_B200_ERR_CUDA; }

typedef struct {
    void* dev[4];        /* device staging buffers (NULL when the pointer is used in place) */
    int64_t lo[4], hi[4];
    const void* host[4];
    int staged_any;
} staging;

/* Copies host operands to the device; fills ptrs with device-accessible
 * pointers to coordinate 0 of each tensor. */
static int stage_in(const tb_plan* P, const tb_tensor_view v[4], const void* ptr[4], staging* st,
                    tb_ptrs* out, void* stream, int* device)
{
    memset(st, 0, sizeof(*st));
    int kinds[4], dev = -1;
    for (int k = 0; k < 4; k++) {
        kinds[k] = TBK_PTR_HOST;
        if (!ptr[k]) continue;
        int kind = 0, d = -1;
        int e = tbk_pointer_kind(ptr[k], &kind, &d);
        if (e) return cuda_err(e);
        kinds[k] = kind;
        if ((kind == TBK_PTR_DEVICE || kind == TBK_PTR_MANAGED) && dev < 0 && d >= 0) dev = d;
    }
    if (dev >= 0) {
        int e = tbk_set_device(dev);
        if (e) return cuda_err(e);
    }
    *device = dev;
    void* outp[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; k++) {
        if (!ptr[k]) continue;
        const int needed = k < 2 || (k == 2 && !P->beta_zero) || k == 3;
        if (kinds[k] == TBK_PTR_DEVICE || kinds[k] == TBK_PTR_MANAGED || !needed) {
            outp[k] = (void*)ptr[k];
            continue;
        }
        int64_t lo, hi;
        if (!tb_span_of(&v[k], &lo, &hi)) { outp[k] = (void*)ptr[k]; continue; }
        const int eb = tb_elem_bytes(v[k].type);
        const size_t bytes = (size_t)(hi - lo + 1) * (size_t)eb;
        void* d = NULL;
        int e = tbk_malloc(&d, bytes, stream);
        if (e) return cuda_err(e);
        st->dev[k] = d;
        st->lo[k] = lo;
        st->hi[k] = hi;
        st->host[k] = ptr[k];
        st->staged_any = 1;
        const char* hsrc = (const char*)ptr[k] + lo * eb;
        if (k < 3 || !tb_span_dense(&v[k], lo, hi)) {
            e = tbk_memcpy(d, hsrc, bytes, TBK_H2D, stream);
            if (e) return cuda_err(e);
        }
        outp[k] = (char*)d - lo * eb;
    }
    out->A = outp[0];
    out->B = outp[1];
    out->C = outp[2];
    out->D = outp[3];
    return 0;
}

static int stage_out(const tb_tensor_view v[4], staging* st, void* stream)
{
    int err = 0;
    if (st->dev[3]) {
        const int eb = tb_elem_bytes(v[3].type);
        const size_t bytes = (size_t)(st->hi[3] - st->lo[3] + 1) * (size_t)eb;
        int e = tbk_memcpy((char*)st->host[3] + st->lo[3] * eb, st->dev[3], bytes, TBK_D2H, stream);
        if (e) err = cuda_err(e);
    }
    for (int k = 0; k < 4; k++)
        if (st->dev[k]) tbk_free(st->dev[k], stream);
    return err;
}

static int run(struct tb_product* p, TAPP_executor exec, TAPP_status* status, const void* alpha,
               const void* A, const void* B, const void* beta, const void* C, void* D)
{
    tb_tensor_view v[4];
    int err = tb_product_views(p, v);
    if (err) return err;
    err = tb_validate(&v[0], &v[1], &v[2], &v[3], beta, C != NULL);
    if (err) return err;
    tb_exec_settings s;
    err = resolve_executor(exec, &s);
    if (err) return err;
    if (s.server) {
        if (!tb_server_is_live(s.server)) return TAPP_B200_ERR_INVALID;
        /* the executor routes its products through a server: queue, then
         * wait for this product's completion */
        int64_t ticket = -1;
        err = tb_server_enqueue(s.server, p, v, &s, alpha, A, B, beta, C, D, &ticket);
        if (!err && ticket >= 0) err = tapp_b200_server_wait((TAPP_b200_server)s.server, ticket);
        return err;
    }

    tb_plan P;
    err = tb_product_plan(p, v, alpha, beta, &s, &P);
    if (err) return err;

    int kernels = 0;
    double dev_us = 0.0, main_us = 0.0;
    if (P.path != TB_PATH_NOOP) {
        const void* ptr[4] = {A, B, C, D};
        staging st;
        tb_ptrs dp;
        int device = -1;
        err = stage_in(&P, v, ptr, &st, &dp, s.stream, &device);
        void* timer = NULL;
        void* main_timer = NULL;
        const int timed = !err && s.want_status && !s.async;
        if (timed) tbk_timer_begin(s.stream, &timer);
        if (!err) {
            int e = tbk_run_plan(&P, &dp, s.stream, &kernels, timed ? &main_timer : NULL);
            if (e) err = cuda_err(e);
        }
        if (timer) tbk_timer_end(s.stream, timer);
        int e2 = stage_out(v, &st, s.stream);
        if (!err) err = e2;
        if (!s.async || st.staged_any) {
            int e = tbk_stream_sync(s.stream);
            if (!err && e) err = cuda_err(e);
            if (!err && (P.path == TB_PATH_TC || P.path == TB_PATH_SLICED) && (e = tbk_check_device_error())) err = cuda_err(e);
        }
        if (timer) tbk_timer_elapsed_us(timer, &dev_us);
        if (main_timer) tbk_timer_elapsed_us(main_timer, &main_us);
    }
    if (s.want_status && status) {
        struct tb_status* so = calloc(1, sizeof(*so));
        if (so) {
            so->magic = TB_MAGIC_STATUS;
            so->path = P.path;
            so->kernels = kernels;
            so->tc_mode = P.tc_mode;
            so->flops = tb_plan_flops(&P);
            so->err_bound = tb_plan_error_bound(&P);
            so->device_us = dev_us;
            so->main_us = main_us;
            *status = (TAPP_status)so;
        }
    }
    return err;
}

/* product.c:130-465 */
TAPP_error TAPP_execute_product(TAPP_tensor_product plan, TAPP_executor exec, TAPP_status* status,
                                const void* alpha, const void* A, const void* B,
                                const void* beta, const void* C, void* D)
{
    struct tb_product* p = (struct tb_product*)plan;
    if (!p || p->magic != TB_MAGIC_PRODUCT) return TAPP_B200_ERR_INVALID;
    return run(p, exec, status, alpha, A, B, beta, C, D);
}

/* product.h:66-75 (no implementation in the reference). Each batch is
 * validated like a single product; device-resident batches of a path that
 * supports grouping run as one launch. */
TAPP_error TAPP_execute_batched_product(TAPP_tensor_product plan, TAPP_executor exec, TAPP_status* status,
                                        int num_batches, const void* alpha, const void** A, const void** B,
                                        const void* beta, const void** C, void** D)
{
    struct tb_product* p = (struct tb_product*)plan;
    if (!p || p->magic != TB_MAGIC_PRODUCT) return TAPP_B200_ERR_INVALID;
    if (num_batches < 0 || (num_batches > 0 && (!A || !B || !D))) return TAPP_B200_ERR_INVALID;
    if (num_batches == 0) return 0;
    tb_tensor_view v[4];
    int err = tb_product_views(p, v);
    if (err) return err;
    for (int i = 0; i < num_batches; i++) {
        err = tb_validate(&v[0], &v[1], &v[2], &v[3], beta, C && C[i] != NULL);
        if (err) return err;
    }
    tb_exec_settings s;
    err = resolve_executor(exec, &s);
    if (err) return err;
    tb_plan P;
    err = tb_product_plan(p, v, alpha, beta, &s, &P);
    if (err) return err;
    if (P.path == TB_PATH_NOOP) return 0;

    /* all operands on the device: one grouped launch */
    /* batches are often slices of a few allocations: a pointer inside an
     * allocation already found to be device memory needs no query */
    int all_dev = 1;
    enum { NR = 16 };
    uintptr_t r_lo[NR], r_hi[NR];
    int nr = 0, next = 0;
    for (int i = 0; i < num_batches && all_dev; i++) {
        const void* q[4] = {A[i], B[i], C ? C[i] : NULL, D[i]};
        for (int k = 0; k < 4; k++) {
            if (!q[k]) continue;
            const uintptr_t a = (uintptr_t)q[k];
            int known = 0;
            for (int j = 0; j < nr && !known; j++) known = a >= r_lo[j] && a < r_hi[j];
            if (known) continue;
            int kind = 0, d = -1;
            uintptr_t st = 0;
            size_t sz = 0;
            if (tbk_pointer_range(q[k], &kind, &d, &st, &sz) || (kind != TBK_PTR_DEVICE && kind != TBK_PTR_MANAGED)) {
                all_dev = 0;
                break;
            }
            r_lo[next] = st;
            r_hi[next] = st + sz;
            next = (next + 1) % NR;
            if (nr < NR) nr++;
        }
    }
    if (all_dev) {
        tb_ptrs* dp = malloc(sizeof(tb_ptrs) * (size_t)num_batches);
        if (!dp) return TAPP_B200_ERR_NOMEM;
        for (int i = 0; i < num_batches; i++) {
            dp[i].A = A[i];
            dp[i].B = B[i];
            dp[i].C = C ? C[i] : NULL;
            dp[i].D = D[i];
        }
        int kernels = 0;
        int e = tbk_run_plan_batched(&P, dp, num_batches, s.stream, &kernels);
        free(dp);
        if (e) return cuda_err(e);
        if (!s.async) {
            e = tbk_stream_sync(s.stream);
            if (e) return cuda_err(e);
            if ((P.path == TB_PATH_TC || P.path == TB_PATH_SLICED) && (e = tbk_check_device_error())) return cuda_err(e);
        }
        if (s.want_status && status) {
            struct tb_status* so = calloc(1, sizeof(*so));
            if (so) {
                so->magic = TB_MAGIC_STATUS;
                so->path = P.path;
                so->kernels = kernels;
                so->tc_mode = P.tc_mode;
                so->flops = tb_plan_flops(&P) * num_batches;
                so->err_bound = tb_plan_error_bound(&P);
                *status = (TAPP_status)so;
            }
        }
        return 0;
    }
    for (int i = 0; i < num_batches; i++) {
        err = run(p, exec, NULL, alpha, A[i], B[i], beta, C ? C[i] : NULL, D[i]);
        if (err) return err;
    }
    return 0;
}

size_t tapp_b200_describe_plan(TAPP_tensor_product plan, TAPP_executor exec, size_t maxlen, char* out)
{
    struct tb_product* p = (struct tb_product*)plan;
    if (!p || p->magic != TB_MAGIC_PRODUCT) return 0;
    tb_tensor_view v[4];
    if (tb_product_views(p, v)) return 0;
    tb_exec_settings s;
    memset(&s, 0, sizeof(s));
    if (exec) resolve_executor(exec, &s);
    /* beta = 1 in D's type so that C counts as read */
    union { float f[4]; double d[2]; uint16_t h[8]; } one;
    memset(&one, 0, sizeof one);
    switch (v[3].type) {
    case TAPP_F32: case TAPP_C32: one.f[0] = 1.0f; break;
    case TAPP_F64: case TAPP_C64: one.d[0] = 1.0; break;
    case TAPP_F16: one.h[0] = 0x3c00; break;
    case TAPP_BF16: one.h[0] = 0x3f80; break;
    default: break;
    }
    tb_plan P;
    tb_plan_options opt = {s.f32_mode, s.force_path, s.f64_mode};
    if (tb_build_plan(&v[0], &v[1], &v[2], &v[3], p->prec, &one, &one, &opt, &P)) return 0;
    return tb_describe(&P, maxlen, out);
}

/* A chain of products on one stream: step i may read the D of step i - 1 as
 * its A or B (a NULL pointer), and a NULL D before the last step is an
 * intermediate in device memory from the library's pool. Host operands are
 * staged per step as TAPP_execute_product stages them; the host waits once,
 * at the end. The products are validated step by step with the codes of
 * TAPP_execute_product. */
TAPP_error tapp_b200_execute_chain(int n, const TAPP_tensor_product* plans, TAPP_executor exec,
                                   const void* const* alphas, const void* const* betas, const void* const* A,
                                   const void* const* B, const void* const* C, void* const* D)
{
    if (n <= 0 || !plans || !alphas || !betas || !A || !B || !D || !D[n - 1]) return TAPP_B200_ERR_INVALID;
    tb_exec_settings s;
    int err = resolve_executor(exec, &s);
    if (err) return err;
    if (s.server) return TAPP_B200_ERR_INVALID;
    void** inter = calloc((size_t)n, sizeof(void*));   /* intermediates to free */
    void** dout = calloc((size_t)n, sizeof(void*));    /* coordinate 0 of each step's D */
    if (!inter || !dout) {
        free(inter);
        free(dout);
        return TAPP_B200_ERR_NOMEM;
    }
    int any_tc = 0;
    for (int i = 0; i < n && !err; i++) {
        struct tb_product* p = (struct tb_product*)plans[i];
        if (!p || p->magic != TB_MAGIC_PRODUCT) {
            err = TAPP_B200_ERR_INVALID;
            break;
        }
        const void* a = A[i] ? A[i] : (i > 0 ? dout[i - 1] : NULL);
        const void* b = B[i] ? B[i] : (i > 0 ? dout[i - 1] : NULL);
        const void* c = C ? C[i] : NULL;
        if (!a || !b) {
            err = TAPP_B200_ERR_INVALID;
            break;
        }
        tb_tensor_view v[4];
        err = tb_product_views(p, v);
        if (!err) err = tb_validate(&v[0], &v[1], &v[2], &v[3], betas[i], c != NULL);
        tb_plan P;
        if (!err) err = tb_product_plan(p, v, alphas[i], betas[i], &s, &P);
        if (err) break;
        void* d = D[i];
        if (!d) {
            int64_t lo, hi;
            if (!tb_span_of(&v[3], &lo, &hi)) {
                lo = 0;
                hi = 0;
            }
            const int eb = tb_elem_bytes(v[3].type);
            void* buf = NULL;
            const int e = tbk_malloc(&buf, (size_t)(hi - lo + 1) * (size_t)eb, s.stream);
            if (e) {
                err = cuda_err(e);
                break;
            }
            inter[i] = buf;
            d = (char*)buf - lo * eb;
        }
        dout[i] = d;
        if (P.path == TB_PATH_NOOP) continue;
        const void* ptr[4] = {a, b, c, d};
        staging st;
        tb_ptrs dp;
        int device = -1;
        err = stage_in(&P, v, ptr, &st, &dp, s.stream, &device);
        int kernels = 0;
        if (!err) {
            const int e = tbk_run_plan(&P, &dp, s.stream, &kernels, NULL);
            if (e) err = cuda_err(e);
        }
        const int e2 = stage_out(v, &st, s.stream);
        if (!err) err = e2;
        if (P.path == TB_PATH_TC || P.path == TB_PATH_SLICED) any_tc = 1;
    }
    for (int i = 0; i < n; i++)
        if (inter[i]) tbk_free(inter[i], s.stream);
    if (!s.async) {
        int e = tbk_stream_sync(s.stream);
        if (!err && e) err = cuda_err(e);
        if (!err && any_tc && (e = tbk_check_device_error())) err = cuda_err(e);
    }
    free(inter);
    free(dout);
    return err;
}

/* Products of different plans in one call. Products whose plans run on the
 * tensor cores from binary32 storage, with all operands on the device and
 * operands the converter warps read in place, run in grouped launches (one
 * per tile shape, tiles.c); every other product runs as TAPP_execute_product
 * runs it, on the same stream. Every product is validated before anything
 * runs (the first failing product's code is returned). The products must be
 * independent: no D may overlap another product's operands. */
TAPP_error tapp_b200_execute_group(int n, const TAPP_tensor_product* plans, TAPP_executor exec,
                                   const void* const* alphas, const void* const* betas, const void* const* A,
                                   const void* const* B, const void* const* C, void* const* D)
{
    if (n < 0 || (n > 0 && (!plans || !alphas || !betas || !A || !B || !D))) return TAPP_B200_ERR_INVALID;
    if (n == 0) return 0;
    tb_exec_settings s;
    int err = resolve_executor(exec, &s);
    if (err) return err;
    if (s.server) return TAPP_B200_ERR_INVALID;
    tb_plan* P = malloc(sizeof(tb_plan) * (size_t)n);
    int* tile = malloc(sizeof(int) * (size_t)n);
    const tb_plan** gp = malloc(sizeof(tb_plan*) * (size_t)n);
    tb_ptrs* gd = malloc(sizeof(tb_ptrs) * (size_t)n);
    int any_tc = 0;
    if (!P || !tile || !gp || !gd) {
        err = TAPP_B200_ERR_NOMEM;
        goto done;
    }
    for (int i = 0; i < n && !err; i++) {
        struct tb_product* p = (struct tb_product*)plans[i];
        tile[i] = 0;
        if (!p || p->magic != TB_MAGIC_PRODUCT || !A[i] || !B[i] || !D[i] || !alphas[i] || !betas[i]) {
            err = TAPP_B200_ERR_INVALID;
            break;
        }
        tb_tensor_view v[4];
        err = tb_product_views(p, v);
        if (!err) err = tb_validate(&v[0], &v[1], &v[2], &v[3], betas[i], C && C[i] != NULL);
        if (!err) err = tb_product_plan(p, v, alphas[i], betas[i], &s, &P[i]);
        if (err || P[i].path != TB_PATH_TC || !tbk_tc_groupable(&P[i], A[i], B[i])) continue;
        const void* q[4] = {A[i], B[i], C ? C[i] : NULL, D[i]};
        int on_device = 1;
        for (int k = 0; k < 4 && on_device; k++) {
            if (!q[k] || (k == 2 && P[i].beta_zero)) continue;
            int kind = 0, dev = -1;
            on_device = !tbk_pointer_kind(q[k], &kind, &dev) && (kind == TBK_PTR_DEVICE || kind == TBK_PTR_MANAGED);
        }
        if (on_device) tile[i] = s.tile ? s.tile : tb_tile_choice(&P[i]);
    }
    if (err) goto done;
    for (int t = 1; t <= 2 && !err; t++) {
        int m = 0;
        for (int i = 0; i < n; i++)
            if (tile[i] == t) {
                gp[m] = &P[i];
                gd[m].A = A[i];
                gd[m].B = B[i];
                gd[m].C = P[i].beta_zero ? NULL : (C ? C[i] : NULL);
                gd[m].D = D[i];
                m++;
            }
        if (!m) continue;
        any_tc = 1;
        int64_t tiles = 0;
        const int e = tbk_run_group_tc_owned(gp, gd, m, t, s.stream, &tiles);
        if (e) err = cuda_err(e);
    }
    for (int i = 0; i < n && !err; i++)
        if (!tile[i])
            err = run((struct tb_product*)plans[i], exec, NULL, alphas[i], A[i], B[i], betas[i], C ? C[i] : NULL,
                      D[i]);
    if (!err && !s.async) {
        int e = tbk_stream_sync(s.stream);
        if (e) err = cuda_err(e);
        if (!err && any_tc && (e = tbk_check_device_error())) err = cuda_err(e);
    }
done:
    free(P);
    free(tile);
    free(gp);
    free(gd);
    return err;
}

/*
 * Device-resident request loop: tapp_b200_loop_*.
 *
 * The reference reserves its handle and executor for such state
 * (reference_implementation/src/handle.c:9-17, executor.c:9-23 allocate
 * placeholders only) and runs every product on the calling thread. Here a
 * persistent kernel of a few blocks (generic.cu: k_request_loop) stays on
 * the GPU and serves small products as they are submitted, with no kernel
 * launch, stream callback or host thread hand-over per product:
 *
 *   submit   validates and plans the product as TAPP_execute_product does,
 *            writes its descriptor into slot t % slots of a ring in mapped
 *            page-locked memory and then the slot's sequence word; launches
 *            the loop if it is not running (it returns after idle_ms without
 *            products, so it never spins without a bound);
 *   device   block 0 polls the sequence word and relays the descriptor
 *            through device memory; every block computes its share of D
 *            with the element kernel's per-output function; the last one to
 *            finish writes the slot's completion word;
 *   wait     polls the completion word; if the loop has returned meanwhile
 *            (it went idle just before the product was posted), relaunches
 *            it. A wait gives up after 30 s with TAPP_B200_ERR_CUDA.
 *
 * Products must plan to the element path (small products: the planner's
 * generic path) and have device operands; others get
 * TAPP_B200_ERR_UNSUPPORTED / TAPP_B200_ERR_INVALID. Results equal
 * TAPP_execute_product's bit for bit. Latency per product (submission to the
 * wait that sees it done) is counted for p50/p99.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "tb_internal.h"

#define LOOP_MAGIC 0x54420009
#define LOOP_LAT 65536

struct tb_loop {
    int magic;
    int device;
    int blocks, nslots;
    unsigned long long idle_ns;
    tb_exec_settings settings;
    void* stream;
    void* event;
    int launched;
    char* ring;        /* host view of the slots */
    void* ring_dev;    /* device view */
    size_t slot_bytes;
    void* state;       /* device: ring copy, sequence words, arrival counters, per-block tickets */
    int64_t next_ticket;
    double* t_submit;  /* per slot: submission time of its ticket */
    int64_t submitted, completed, launches;
    double lat[LOOP_LAT];
    int64_t n_lat;
    pthread_mutex_t lock;
};

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static struct tb_loop* as_loop(TAPP_b200_loop h)
{
    struct tb_loop* l = (struct tb_loop*)h;
    return l && l->magic == LOOP_MAGIC ? l : NULL;
}

/* the slot's words as the device writes them (offsets inside the slot:
 * seq and done are the two int64 words after the descriptor) */
static volatile int64_t* seq_word(struct tb_loop* l, int64_t slot, int which)
{
    char* s = l->ring + (size_t)slot * l->slot_bytes;
    /* LoopSlot ends with seq, done and 6 words of padding */
    return (volatile int64_t*)(s + l->slot_bytes - 8 * 8 + 8 * which);
}

/* launches the loop unless a launch is still running; call with the lock */
static int ensure_running(struct tb_loop* l)
{
    if (l->launched) {
        const int d = tbk_event_done(l->event);
        if (d < 0) return TAPP_B200_ERR_CUDA;
        if (d == 0) return 0;
    }
    if (tbk_set_device(l->device) ||
        tbk_loop_launch(l->ring_dev, l->state, l->nslots, l->blocks, l->idle_ns, l->stream, &l->event))
        return TAPP_B200_ERR_CUDA;
    l->launched = 1;
    l->launches++;
    return 0;
}

TAPP_error tapp_b200_loop_create(TAPP_b200_loop* loop, TAPP_executor exec, int blocks, int slots, double idle_ms)
{
    if (!loop || blocks < 1 || blocks > 256 || slots < blocks || slots > 4096 || !(idle_ms > 0.0) || idle_ms > 10000.0)
        return TAPP_B200_ERR_INVALID;
    *loop = 0;
    struct tb_loop* l = calloc(1, sizeof(*l));
    if (!l) return TAPP_B200_ERR_NOMEM;
    l->magic = LOOP_MAGIC;
    l->blocks = blocks;
    l->nslots = slots;
    l->idle_ns = (unsigned long long)(idle_ms * 1e6);
    if (exec && tb_executor_is_ours(exec)) {
        const struct tb_executor* x = (const struct tb_executor*)exec;
        l->settings.f32_mode = x->f32_mode;
        l->settings.force_path = x->force_path;
    }
    pthread_mutex_init(&l->lock, NULL);
    l->slot_bytes = tbk_loop_slot_bytes();
    int err = 0;
    if (tbk_get_device(&l->device)) err = TAPP_B200_ERR_CUDA;
    if (!err && tbk_stream_create(&l->stream)) err = TAPP_B200_ERR_CUDA;
    if (!err && tbk_host_alloc_mapped((void**)&l->ring, &l->ring_dev, l->slot_bytes * (size_t)slots))
        err = TAPP_B200_ERR_NOMEM;
    if (!err && tbk_loop_state(&l->state, slots, blocks)) err = TAPP_B200_ERR_NOMEM;
    if (!err && !(l->t_submit = calloc((size_t)slots, sizeof(double)))) err = TAPP_B200_ERR_NOMEM;
    if (err) {
        tapp_b200_loop_destroy((TAPP_b200_loop)l);
        return err;
    }
    *loop = (TAPP_b200_loop)l;
    return 0;
}

TAPP_error tapp_b200_loop_submit(TAPP_b200_loop loop, TAPP_tensor_product plan, const void* alpha, const void* A,
                                 const void* B, const void* beta, const void* C, void* D, int64_t* ticket)
{
    struct tb_loop* l = as_loop(loop);
    struct tb_product* p = (struct tb_product*)plan;
    if (!l || !ticket || !p || p->magic != TB_MAGIC_PRODUCT) return TAPP_B200_ERR_INVALID;
    *ticket = -1;
    tb_tensor_view v[4];
    int err = tb_product_views(p, v);
    if (!err) err = tb_validate(&v[0], &v[1], &v[2], &v[3], beta, C != NULL);
    if (err) return err;
    tb_plan P;
    err = tb_product_plan(p, v, alpha, beta, &l->settings, &P);
    if (err) return err;
    if (P.path != TB_PATH_GENERIC && P.path != TB_PATH_NOOP) return TAPP_B200_ERR_UNSUPPORTED;
    const void* q[4] = {A, B, C, D};
    for (int k = 0; k < 4 && P.path != TB_PATH_NOOP; k++) {
        if (k == 2 && P.beta_zero) continue;
        int kind = 0, dev = -1;
        if (!q[k] || tbk_pointer_kind(q[k], &kind, &dev) || (kind != TBK_PTR_DEVICE && kind != TBK_PTR_MANAGED))
            return TAPP_B200_ERR_INVALID;
    }
    tb_ptrs dp = {A, B, P.beta_zero ? NULL : C, D};
    pthread_mutex_lock(&l->lock);
    const int64_t t = l->next_ticket;
    const int64_t slot = t % l->nslots;
    /* the slot is free once the ticket that used it last is done */
    const double t0 = now_s();
    while (t >= l->nslots && *seq_word(l, slot, 1) < t - l->nslots + 1) {
        if ((err = ensure_running(l))) break;
        if (now_s() - t0 > 30.0) {
            err = TAPP_B200_ERR_CUDA;
            break;
        }
    }
    if (!err) {
        tbk_loop_fill(l->ring + (size_t)slot * l->slot_bytes, &P, &dp);
        l->t_submit[slot] = now_s();
        __atomic_thread_fence(__ATOMIC_RELEASE);
        __atomic_store_n((int64_t*)seq_word(l, slot, 0), t + 1, __ATOMIC_RELEASE);
        l->next_ticket++;
        l->submitted++;
        err = ensure_running(l);
    }
    pthread_mutex_unlock(&l->lock);
    if (!err) *ticket = t;
    return err;
}

TAPP_error tapp_b200_loop_wait(TAPP_b200_loop loop, int64_t ticket)
{
    struct tb_loop* l = as_loop(loop);
    if (!l || ticket < 0 || ticket >= l->next_ticket) return TAPP_B200_ERR_INVALID;
    const int64_t slot = ticket % l->nslots;
    const double t0 = now_s();
    for (uint64_t i = 0;; i++) {
        if (__atomic_load_n((const int64_t*)seq_word(l, slot, 1), __ATOMIC_ACQUIRE) >= ticket + 1) break;
        if ((i & 1023) == 1023) {
            pthread_mutex_lock(&l->lock);
            const int e = ensure_running(l);   /* the loop went idle before this product was posted */
            pthread_mutex_unlock(&l->lock);
            if (e) return e;
            if (now_s() - t0 > 30.0) return TAPP_B200_ERR_CUDA;
        }
    }
    const double t1 = now_s();
    pthread_mutex_lock(&l->lock);
    if (ticket + l->nslots >= l->next_ticket) {  /* the slot still holds this ticket's time */
        l->lat[l->n_lat % LOOP_LAT] = t1 - l->t_submit[slot];
        l->n_lat++;
    }
    l->completed++;
    pthread_mutex_unlock(&l->lock);
    return 0;
}

static int cmp_d(const void* a, const void* b)
{
    const double x = *(const double*)a, y = *(const double*)b;
    return x < y ? -1 : x > y;
}

TAPP_error tapp_b200_loop_stats(TAPP_b200_loop loop, tapp_b200_loop_counters* out)
{
    struct tb_loop* l = as_loop(loop);
    if (!l || !out) return TAPP_B200_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    pthread_mutex_lock(&l->lock);
    out->submitted = l->submitted;
    out->completed = l->completed;
    out->launches = l->launches;
    out->running = l->launched && tbk_event_done(l->event) == 0;
    const int64_t n = l->n_lat < LOOP_LAT ? l->n_lat : LOOP_LAT;
    double* v = n ? malloc(sizeof(double) * (size_t)n) : NULL;
    if (v) {
        memcpy(v, l->lat, sizeof(double) * (size_t)n);
        qsort(v, (size_t)n, sizeof(double), cmp_d);
        double sum = 0;
        for (int64_t i = 0; i < n; i++) sum += v[i];
        out->p50_us = 1e6 * v[(n - 1) / 2];
        out->p99_us = 1e6 * v[(int64_t)((double)(n - 1) * 0.99)];
        out->mean_us = 1e6 * sum / (double)n;
        out->max_us = 1e6 * v[n - 1];
        free(v);
    }
    pthread_mutex_unlock(&l->lock);
    return 0;
}

TAPP_error tapp_b200_loop_reset_stats(TAPP_b200_loop loop)
{
    struct tb_loop* l = as_loop(loop);
    if (!l) return TAPP_B200_ERR_INVALID;
    pthread_mutex_lock(&l->lock);
    l->n_lat = 0;
    l->submitted = l->completed = l->launches = 0;
    pthread_mutex_unlock(&l->lock);
    return 0;
}

/* Waits for the loop to return (at most its idle limit after the last
 * product), then frees it. */
TAPP_error tapp_b200_loop_destroy(TAPP_b200_loop loop)
{
    struct tb_loop* l = as_loop(loop);
    if (!l) return TAPP_B200_ERR_INVALID;
    int err = 0;
    if (l->launched) {
        const double t0 = now_s();
        int d;
        while ((d = tbk_event_done(l->event)) == 0)
            if (now_s() - t0 > 60.0) break;
        if (d != 1) err = TAPP_B200_ERR_CUDA;
    }
    if (err) return err;   /* the kernel may still read the ring: keep it */
    tbk_event_destroy(l->event);
    if (l->state) tbk_dev_free(l->state);
    if (l->ring) tbk_host_free(l->ring);
    if (l->stream) tbk_stream_destroy(l->stream);
    free(l->t_submit);
    pthread_mutex_destroy(&l->lock);
    l->magic = 0;
    free(l);
    return 0;
}

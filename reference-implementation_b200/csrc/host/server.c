/*
 * Serving: the tapp_b200_server_* functions and executors that carry
 * TAPP_B200_ATTR_SERVER. The reference reserves its handle and executor for
 * such state (reference_implementation/src/handle.c:9-17 and executor.c:9-23
 * allocate placeholders only) and runs every product synchronously on the
 * calling thread (product.c:130-465); this file adds what a service needs
 * on one GPU.
 *
 * Flow of a product:
 *   submit     (caller's thread) the product is validated and planned
 *              exactly as TAPP_execute_product does it, the device memory it
 *              needs is computed (staging of host operands, tensor-core
 *              panels), and it is queued with a ticket;
 *   admission  (scheduler thread) queued products are taken in arrival
 *              order while their memory fits the remaining HBM budget and
 *              fewer than max_in_flight are running;
 *   issue      admitted products of the CUDA-core element path with modest
 *              work are packed into one grouped launch per compute domain
 *              (tbk_run_group); admitted tensor-core products of binary32
 *              storage into one grouped tensor-core launch per tile shape
 *              (tbk_run_group_tc, operands read in place), where that
 *              launch gives the same bits as the product alone; every other
 *              product is a unit of its own.
 *              Units are spread round-robin over the server's streams, each
 *              as: staging copies in, kernel(s), copy of D out, frees, and a
 *              completion event;
 *   completion the completion thread polls the oldest pending unit of each
 *              stream; once its event has passed it stamps the products'
 *              completion time, returns their budget and slots and wakes the
 *              scheduler and waiters.
 * Admission therefore runs whenever work completes or arrives, so products
 * join the device while others are still running (continuous batching).
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <sched.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "tb_internal.h"

#define SRV_MAGIC 0x54420007
#define SRV_MAX_STREAMS 16
#define SRV_GROUP_MAX 64          /* products per grouped launch */
#define SRV_SLABS_PER_STREAM 4    /* page-locked descriptor buffers */
#define SRV_GROUP_MAX_OUT (1 << 20)   /* grouped products: at most this many outputs */
#define SRV_GROUP_MAX_WORK (1 << 26)  /* ... and outputs x contracted size */
#define SRV_MAX_LIVE 256

enum { RQ_QUEUED = 0, RQ_RUNNING = 1, RQ_DONE = 2 };

typedef struct srv_req {
    int64_t ticket;
    tb_plan P;
    const void* ptr[4];
    int staged[4];   /* operand k goes through a device copy */
    int copy_in[4];  /* ... whose span is copied in first */
    int64_t lo[4], hi[4];
    int eb[4];
    int64_t need;    /* bytes charged against the budget */
    void* dev[4];
    struct srv_req* next;
} srv_req;

typedef struct srv_rec {
    double t_submit, t_done, flops;
    int state, err, tc;
} srv_rec;

struct tb_server {
    int magic;
    int device;
    int n_streams, max_in_flight;
    void* streams[SRV_MAX_STREAMS];
    int rr;
    tb_exec_settings settings;

    pthread_mutex_t lock;
    pthread_cond_t cv_sched;  /* queue, budget or slots changed */
    pthread_cond_t cv_done;   /* a product completed */
    pthread_cond_t cv_reap;   /* a unit was issued (the completion thread's wake-up) */
    pthread_t thread;
    pthread_t reaper;         /* completion thread: polls the issued units' events */
    int stop, reap_stop;

    /* issued units not yet complete, per stream in issue order (a stream
     * completes its units in that order) */
    struct srv_unit *pend_head[SRV_MAX_STREAMS], *pend_tail[SRV_MAX_STREAMS];
    int64_t n_pend;

    srv_req *head, *tail;

    srv_rec* rec;             /* rec[t - rec_base] for ticket t */
    int64_t rec_base, n_rec, cap_rec;

    int64_t budget, reserved, peak_reserved;
    int64_t in_flight, peak_in_flight;
    int64_t submitted, completed, failed, units, grouped, budget_waits;
    double t_first, t_last;
    int first_err, tc_ran;
    int64_t last_blocked;     /* ticket of the last product counted in budget_waits */

    int n_slabs;
    size_t slab_bytes;
    void* slab[SRV_MAX_STREAMS * SRV_SLABS_PER_STREAM];
    int slab_free[SRV_MAX_STREAMS * SRV_SLABS_PER_STREAM];
};

typedef struct srv_unit {
    struct tb_server* srv;
    int n, slab, err;
    int tc_tile;     /* grouped tensor-core unit: its tile shape (1, 2); 0 otherwise */
    void* ev;        /* recorded on the unit's stream after its work */
    struct srv_unit* next_pend;
    srv_req* req[SRV_GROUP_MAX];
} srv_unit;

/* ---- registry of live servers (attribute values are checked against it) ---- */

static pthread_mutex_t live_lock = PTHREAD_MUTEX_INITIALIZER;
static const struct tb_server* live[SRV_MAX_LIVE];
static int n_live;

int tb_server_is_live(const struct tb_server* srv)
{
    int found = 0;
    pthread_mutex_lock(&live_lock);
    for (int i = 0; i < n_live; i++)
        if (live[i] == srv) { found = 1; break; }
    pthread_mutex_unlock(&live_lock);
    return found;
}

static int live_add(const struct tb_server* srv)
{
    int ok = 0;
    pthread_mutex_lock(&live_lock);
    if (n_live < SRV_MAX_LIVE) { live[n_live++] = srv; ok = 1; }
    pthread_mutex_unlock(&live_lock);
    return ok;
}

static void live_remove(const struct tb_server* srv)
{
    pthread_mutex_lock(&live_lock);
    for (int i = 0; i < n_live; i++)
        if (live[i] == srv) { live[i] = live[--n_live]; break; }
    pthread_mutex_unlock(&live_lock);
}

static struct tb_server* as_server(TAPP_b200_server h)
{
    struct tb_server* s = (struct tb_server*)h;
    return s && tb_server_is_live(s) && s->magic == SRV_MAGIC ? s : NULL;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int cuda_code(int e) { return e == TBK_ERR_NOMEM ? TAPP_B200_ERR_NOMEM : TAPP_B200_ERR_CUDA; }

static int64_t round512(int64_t b) { return (b + 511) & ~(int64_t)511; }

/* ---- completion (completion thread) ---- */

static void unit_done(void* arg)
{
    srv_unit* u = (srv_unit*)arg;
    struct tb_server* s = u->srv;
    const double t = now_s();
    pthread_mutex_lock(&s->lock);
    for (int i = 0; i < u->n; i++) {
        const srv_req* r = u->req[i];
        srv_rec* rc = &s->rec[r->ticket - s->rec_base];
        rc->t_done = t;
        rc->err = u->err;
        rc->state = RQ_DONE;
        s->reserved -= r->need;
        s->in_flight--;
        s->completed++;
        if (u->err) {
            s->failed++;
            if (!s->first_err) s->first_err = u->err;
        }
    }
    if (u->slab >= 0) s->slab_free[u->slab] = 1;
    s->t_last = t;
    pthread_cond_broadcast(&s->cv_done);
    pthread_cond_broadcast(&s->cv_sched);
    pthread_mutex_unlock(&s->lock);
    for (int i = 0; i < u->n; i++) free(u->req[i]);
    free(u);
}

/* ---- issue (scheduler thread) ---- */

static int stage_in(srv_req* r, void* stream, tb_ptrs* out)
{
    void* p[4];
    for (int k = 0; k < 4; k++) {
        p[k] = (void*)r->ptr[k];
        if (!r->staged[k]) continue;
        const size_t bytes = (size_t)(r->hi[k] - r->lo[k] + 1) * (size_t)r->eb[k];
        void* d = NULL;
        int e = tbk_malloc(&d, bytes, stream);
        if (e) return e;
        r->dev[k] = d;
        if (r->copy_in[k]) {
            e = tbk_memcpy(d, (const char*)r->ptr[k] + r->lo[k] * r->eb[k], bytes, TBK_H2D, stream);
            if (e) return e;
        }
        p[k] = (char*)d - r->lo[k] * r->eb[k];
    }
    out->A = p[0];
    out->B = p[1];
    out->C = p[2];
    out->D = p[3];
    return 0;
}

static int stage_out(srv_req* r, void* stream, int copy)
{
    int err = 0;
    if (copy && r->dev[3]) {
        const size_t bytes = (size_t)(r->hi[3] - r->lo[3] + 1) * (size_t)r->eb[3];
        err = tbk_memcpy((char*)r->ptr[3] + r->lo[3] * r->eb[3], r->dev[3], bytes, TBK_D2H, stream);
    }
    for (int k = 0; k < 4; k++)
        if (r->dev[k]) {
            tbk_free(r->dev[k], stream);
            r->dev[k] = NULL;
        }
    return err;
}

static int take_slab(struct tb_server* s)
{
    pthread_mutex_lock(&s->lock);
    int got = -1;
    for (;;) {
        for (int i = 0; i < s->n_slabs; i++)
            if (s->slab_free[i]) { got = i; break; }
        if (got >= 0) break;
        pthread_cond_wait(&s->cv_sched, &s->lock);
    }
    s->slab_free[got] = 0;
    pthread_mutex_unlock(&s->lock);
    return got;
}

static void issue(struct tb_server* s, srv_unit* u)
{
    const int si = s->rr++ % s->n_streams;
    void* stream = s->streams[si];
    tb_ptrs dp[SRV_GROUP_MAX];
    int e = 0;
    for (int i = 0; i < u->n && !e; i++) e = stage_in(u->req[i], stream, &dp[i]);
    if (!e) {
        if (u->n == 1) {
            int kernels = 0;
            e = tbk_run_plan(&u->req[0]->P, &dp[0], stream, &kernels, NULL);
        } else {
            const tb_plan* plans[SRV_GROUP_MAX];
            for (int i = 0; i < u->n; i++) plans[i] = &u->req[i]->P;
            u->slab = take_slab(s);
            void* ddesc = NULL;
            const size_t bytes = u->tc_tile ? tbk_group_tc_bytes(u->n) : tbk_group_bytes(u->n);
            e = tbk_malloc(&ddesc, bytes, stream);
            if (!e) {
                int64_t tiles = 0;
                e = u->tc_tile ? tbk_run_group_tc(plans, dp, u->n, s->slab[u->slab], ddesc, u->tc_tile, stream, &tiles)
                               : tbk_run_group(plans, dp, u->n, s->slab[u->slab], ddesc, stream);
                tbk_free(ddesc, stream);
            }
        }
    }
    for (int i = 0; i < u->n; i++) {
        int e2 = stage_out(u->req[i], stream, !e);
        if (!e) e = e2;
    }
    u->err = e ? cuda_code(e) : 0;
    pthread_mutex_lock(&s->lock);
    s->units++;
    if (u->n > 1) s->grouped += u->n;
    for (int i = 0; i < u->n; i++)
        if (u->req[i]->P.path == TB_PATH_TC || u->req[i]->P.path == TB_PATH_SLICED) s->tc_ran = 1;
    pthread_mutex_unlock(&s->lock);
    void* ev = NULL;
    if (!tbk_event_create(&ev) && !tbk_event_record(ev, stream)) {
        u->ev = ev;
        u->next_pend = NULL;
        pthread_mutex_lock(&s->lock);
        if (s->pend_tail[si]) s->pend_tail[si]->next_pend = u;
        else s->pend_head[si] = u;
        s->pend_tail[si] = u;
        s->n_pend++;
        pthread_cond_signal(&s->cv_reap);
        pthread_mutex_unlock(&s->lock);
    } else {
        if (ev) tbk_event_destroy(ev);
        tbk_stream_sync(stream);
        if (!u->err) u->err = TAPP_B200_ERR_CUDA;
        unit_done(u);
    }
}

/* Completion thread: polls the issued units of every stream in issue order
 * (a stream completes them in that order) and completes each run of units
 * whose events have passed. Polling (a yield between sweeps, a 20 us sleep
 * once sweeps have found nothing for a while) answers within microseconds
 * of a unit's end, where a stream callback waits for the driver's callback
 * thread and holds its stream until it returns; it keeps a host core busy
 * while units are in flight and sleeps on cv_reap when none are. */
#define SRV_REAP_MAX 32  /* units of one stream looked at per sweep */
static void* reaper(void* arg)
{
    struct tb_server* s = (struct tb_server*)arg;
    tbk_set_device(s->device);
    int idle = 0;
    srv_unit* seen[SRV_MAX_STREAMS][SRV_REAP_MAX];
    int nseen[SRV_MAX_STREAMS], ndone[SRV_MAX_STREAMS];
    pthread_mutex_lock(&s->lock);
    for (;;) {
        while (!s->n_pend && !s->reap_stop) {
            idle = 0;
            pthread_cond_wait(&s->cv_reap, &s->lock);
        }
        if (!s->n_pend) break;  /* stopping, nothing in flight */
        const int ns = s->n_streams;
        for (int i = 0; i < ns; i++) {
            nseen[i] = 0;
            for (srv_unit* u = s->pend_head[i]; u && nseen[i] < SRV_REAP_MAX; u = u->next_pend) seen[i][nseen[i]++] = u;
        }
        pthread_mutex_unlock(&s->lock);
        /* only this thread removes units, so the ones seen stay valid unlocked */
        int total = 0;
        for (int i = 0; i < ns; i++) {
            ndone[i] = 0;
            for (int j = 0; j < nseen[i]; j++) {
                srv_unit* u = seen[i][j];
                const int q = tbk_event_done(u->ev);
                if (q == 0) break;
                if (q < 0 && !u->err) u->err = TAPP_B200_ERR_CUDA;
                ndone[i]++;
            }
            total += ndone[i];
        }
        if (total) {
            pthread_mutex_lock(&s->lock);
            for (int i = 0; i < ns; i++) {
                if (!ndone[i]) continue;
                s->pend_head[i] = seen[i][ndone[i] - 1]->next_pend;
                if (!s->pend_head[i]) s->pend_tail[i] = NULL;
            }
            s->n_pend -= total;
            pthread_mutex_unlock(&s->lock);
            for (int i = 0; i < ns; i++)
                for (int j = 0; j < ndone[i]; j++) {
                    tbk_event_destroy(seen[i][j]->ev);
                    unit_done(seen[i][j]);
                }
            idle = 0;
        } else if (++idle < 256) {
            sched_yield();
        } else {
            const struct timespec ts = {0, 20000};
            nanosleep(&ts, NULL);
        }
        pthread_mutex_lock(&s->lock);
    }
    pthread_mutex_unlock(&s->lock);
    return NULL;
}

/* a tensor-core product that a grouped launch runs with the same result as
 * alone: its tile shape (1, 2), else 0 */
static int tc_groupable(const struct tb_server* s, const srv_req* r)
{
    const tb_plan* P = &r->P;
    if (P->path != TB_PATH_TC || !tbk_tc_groupable(P, r->ptr[0], r->ptr[1]) || !tbk_tc_group_same_as_solo(P))
        return 0;
    return s->settings.tile ? s->settings.tile : tb_tile_choice(P);
}

/* element-path products of modest work: the grouped element kernel runs
 * each with its own launch's per-output function (a thread, or a warp, per
 * output), so the bits are those of its own launch */
static int groupable(const tb_plan* P)
{
    return P->path == TB_PATH_GENERIC && P->F.size <= SRV_GROUP_MAX_OUT &&
           (double)P->F.size * (double)P->K.size * (double)(P->UA.size + P->UB.size) <= (double)SRV_GROUP_MAX_WORK;
}

static srv_unit* new_unit(struct tb_server* s)
{
    srv_unit* u = calloc(1, sizeof(*u));
    if (u) {
        u->srv = s;
        u->slab = -1;
    }
    return u;
}

/* completes one product that could not be issued (no host memory for its unit) */
static void fail_now(struct tb_server* s, srv_req* r, int err)
{
    const double t = now_s();
    pthread_mutex_lock(&s->lock);
    srv_rec* rc = &s->rec[r->ticket - s->rec_base];
    rc->t_done = t;
    rc->err = err;
    rc->state = RQ_DONE;
    s->reserved -= r->need;
    s->in_flight--;
    s->completed++;
    s->failed++;
    if (!s->first_err) s->first_err = err;
    s->t_last = t;
    pthread_cond_broadcast(&s->cv_done);
    pthread_cond_broadcast(&s->cv_sched);
    pthread_mutex_unlock(&s->lock);
    free(r);
}

static void dispatch(struct tb_server* s, srv_req* batch)
{
    srv_unit* group[4] = {NULL, NULL, NULL, NULL};
    srv_unit* tcg[3] = {NULL, NULL, NULL};  /* grouped tensor-core units by tile shape */
    while (batch) {
        srv_req* r = batch;
        batch = r->next;
        r->next = NULL;
        const int tile = tc_groupable(s, r);
        if (tile) {
            if (!tcg[tile] && !(tcg[tile] = new_unit(s))) {
                fail_now(s, r, TAPP_B200_ERR_NOMEM);
                continue;
            }
            tcg[tile]->tc_tile = tile;
            tcg[tile]->req[tcg[tile]->n++] = r;
            if (tcg[tile]->n == SRV_GROUP_MAX) {
                issue(s, tcg[tile]);
                tcg[tile] = NULL;
            }
            continue;
        }
        if (groupable(&r->P)) {
            const int c = r->P.compute & 3;
            if (!group[c] && !(group[c] = new_unit(s))) {
                fail_now(s, r, TAPP_B200_ERR_NOMEM);
                continue;
            }
            group[c]->req[group[c]->n++] = r;
            if (group[c]->n == SRV_GROUP_MAX) {
                issue(s, group[c]);
                group[c] = NULL;
            }
            continue;
        }
        srv_unit* u = new_unit(s);
        if (!u) {
            fail_now(s, r, TAPP_B200_ERR_NOMEM);
            continue;
        }
        u->req[u->n++] = r;
        issue(s, u);
    }
    for (int c = 0; c < 4; c++)
        if (group[c]) issue(s, group[c]);
    for (int t = 1; t <= 2; t++)
        if (tcg[t]) issue(s, tcg[t]);
}

static int admissible(const struct tb_server* s)
{
    return s->head && s->in_flight < s->max_in_flight && s->reserved + s->head->need <= s->budget;
}

/* counts each queued product that had to wait for memory, once */
static void note_budget_wait(struct tb_server* s)
{
    if (s->head && s->in_flight < s->max_in_flight && s->reserved + s->head->need > s->budget &&
        s->head->ticket != s->last_blocked) {
        s->budget_waits++;
        s->last_blocked = s->head->ticket;
    }
}

static void* scheduler(void* arg)
{
    struct tb_server* s = (struct tb_server*)arg;
    tbk_set_device(s->device);
    pthread_mutex_lock(&s->lock);
    for (;;) {
        while (!s->stop && !admissible(s)) {
            note_budget_wait(s);
            pthread_cond_wait(&s->cv_sched, &s->lock);
        }
        if (!admissible(s)) break;  /* stopping, nothing admissible */
        srv_req* batch = NULL;
        srv_req** tail = &batch;
        while (admissible(s)) {
            srv_req* r = s->head;
            s->head = r->next;
            if (!s->head) s->tail = NULL;
            r->next = NULL;
            *tail = r;
            tail = &r->next;
            s->reserved += r->need;
            s->in_flight++;
            s->rec[r->ticket - s->rec_base].state = RQ_RUNNING;
        }
        note_budget_wait(s);
        if (s->reserved > s->peak_reserved) s->peak_reserved = s->reserved;
        if (s->in_flight > s->peak_in_flight) s->peak_in_flight = s->in_flight;
        pthread_mutex_unlock(&s->lock);
        dispatch(s, batch);
        pthread_mutex_lock(&s->lock);
    }
    pthread_mutex_unlock(&s->lock);
    return NULL;
}

/* ---- submission ---- */

int tb_server_enqueue(struct tb_server* s, struct tb_product* p, const tb_tensor_view v[4],
                      const tb_exec_settings* set, const void* alpha, const void* A, const void* B,
                      const void* beta, const void* C, void* D, int64_t* ticket)
{
    *ticket = -1;
    srv_req* r = calloc(1, sizeof(*r));
    if (!r) return TAPP_B200_ERR_NOMEM;
    int err = tb_product_plan(p, v, alpha, beta, set, &r->P);
    if (err) {
        free(r);
        return err;
    }
    const void* ptr[4] = {A, B, C, D};
    for (int k = 0; k < 4 && r->P.path != TB_PATH_NOOP; k++) {
        r->ptr[k] = ptr[k];
        if (!ptr[k]) continue;
        const int needed = k < 2 || (k == 2 && !r->P.beta_zero) || k == 3;
        int kind = 0, dev = -1;
        int e = tbk_pointer_kind(ptr[k], &kind, &dev);
        if (e) {
            free(r);
            return cuda_code(e);
        }
        if (kind == TBK_PTR_DEVICE || kind == TBK_PTR_MANAGED) {
            if (kind == TBK_PTR_DEVICE && dev != s->device) {
                free(r);
                return TAPP_B200_ERR_INVALID;
            }
            continue;
        }
        int64_t lo, hi;
        if (!needed || !tb_span_of(&v[k], &lo, &hi)) continue;
        r->staged[k] = 1;
        r->copy_in[k] = k < 3 || !tb_span_dense(&v[k], lo, hi);
        r->lo[k] = lo;
        r->hi[k] = hi;
        r->eb[k] = tb_elem_bytes(v[k].type);
        r->need += round512((hi - lo + 1) * r->eb[k]);
    }
    r->need += round512((int64_t)tbk_scratch_bytes(&r->P));
    if (r->need > s->budget) {
        free(r);
        return TAPP_B200_ERR_BUDGET;
    }

    const double t = now_s();
    pthread_mutex_lock(&s->lock);
    if (s->n_rec == s->cap_rec) {
        const int64_t cap = s->cap_rec ? 2 * s->cap_rec : 1024;
        srv_rec* nr = realloc(s->rec, sizeof(srv_rec) * (size_t)cap);
        if (!nr) {
            pthread_mutex_unlock(&s->lock);
            free(r);
            return TAPP_B200_ERR_NOMEM;
        }
        s->rec = nr;
        s->cap_rec = cap;
    }
    r->ticket = s->rec_base + s->n_rec;
    srv_rec* rc = &s->rec[s->n_rec++];
    memset(rc, 0, sizeof(*rc));
    rc->t_submit = t;
    rc->flops = tb_plan_flops(&r->P);
    rc->tc = r->P.path == TB_PATH_TC || r->P.path == TB_PATH_SLICED;
    if (!s->submitted) s->t_first = t;
    s->submitted++;
    *ticket = r->ticket;
    if (r->P.path == TB_PATH_NOOP) {
        /* nothing to run (empty D, or the 16-bit complex D the reference leaves alone) */
        rc->state = RQ_DONE;
        rc->t_done = t;
        s->completed++;
        s->t_last = t;
        pthread_cond_broadcast(&s->cv_done);
        pthread_mutex_unlock(&s->lock);
        free(r);
        return 0;
    }
    rc->state = RQ_QUEUED;
    if (s->tail) s->tail->next = r;
    else s->head = r;
    s->tail = r;
    pthread_cond_signal(&s->cv_sched);
    pthread_mutex_unlock(&s->lock);
    return 0;
}

/* ---- public functions ---- */

TAPP_error tapp_b200_server_create(TAPP_b200_server* server, TAPP_executor exec, int64_t hbm_budget_bytes,
                                   int n_streams, int max_in_flight)
{
    if (!server || hbm_budget_bytes <= 0 || n_streams < 1 || n_streams > SRV_MAX_STREAMS || max_in_flight < 1)
        return TAPP_B200_ERR_INVALID;
    *server = 0;
    int dev = 0, e = tbk_get_device(&dev);
    if (e) return cuda_code(e);
    struct tb_server* s = calloc(1, sizeof(*s));
    if (!s) return TAPP_B200_ERR_NOMEM;
    s->magic = SRV_MAGIC;
    s->device = dev;
    s->n_streams = n_streams;
    s->max_in_flight = max_in_flight;
    s->budget = hbm_budget_bytes;
    s->last_blocked = -1;
    if (exec && tb_executor_is_ours(exec)) {
        const struct tb_executor* x = (const struct tb_executor*)exec;
        s->settings.f32_mode = x->f32_mode;
        s->settings.force_path = x->force_path;
        s->settings.tile = x->tile;
    }
    pthread_mutex_init(&s->lock, NULL);
    pthread_cond_init(&s->cv_sched, NULL);
    pthread_cond_init(&s->cv_done, NULL);
    pthread_cond_init(&s->cv_reap, NULL);
    int err = 0;
    for (int i = 0; i < n_streams && !err; i++)
        if ((e = tbk_stream_create(&s->streams[i]))) err = cuda_code(e);
    s->slab_bytes = tbk_group_bytes(SRV_GROUP_MAX);
    if (tbk_group_tc_bytes(SRV_GROUP_MAX) > s->slab_bytes) s->slab_bytes = tbk_group_tc_bytes(SRV_GROUP_MAX);
    s->n_slabs = n_streams * SRV_SLABS_PER_STREAM;
    for (int i = 0; i < s->n_slabs && !err; i++) {
        if ((e = tbk_host_alloc(&s->slab[i], s->slab_bytes))) err = cuda_code(e);
        s->slab_free[i] = 1;
    }
    int reaper_on = 0;
    if (!err) {
        if (pthread_create(&s->reaper, NULL, reaper, s)) err = TAPP_B200_ERR_NOMEM;
        else reaper_on = 1;
    }
    if (!err && pthread_create(&s->thread, NULL, scheduler, s)) err = TAPP_B200_ERR_NOMEM;
    if (!err && !live_add(s)) {
        pthread_mutex_lock(&s->lock);
        s->stop = 1;
        pthread_cond_broadcast(&s->cv_sched);
        pthread_mutex_unlock(&s->lock);
        pthread_join(s->thread, NULL);
        err = TAPP_B200_ERR_LIMIT;
    }
    if (err && reaper_on) {
        pthread_mutex_lock(&s->lock);
        s->reap_stop = 1;
        pthread_cond_broadcast(&s->cv_reap);
        pthread_mutex_unlock(&s->lock);
        pthread_join(s->reaper, NULL);
    }
    if (err) {
        for (int i = 0; i < s->n_slabs; i++)
            if (s->slab[i]) tbk_host_free(s->slab[i]);
        for (int i = 0; i < n_streams; i++)
            if (s->streams[i]) tbk_stream_destroy(s->streams[i]);
        pthread_mutex_destroy(&s->lock);
        pthread_cond_destroy(&s->cv_sched);
        pthread_cond_destroy(&s->cv_done);
        pthread_cond_destroy(&s->cv_reap);
        free(s);
        return err;
    }
    *server = (TAPP_b200_server)s;
    return 0;
}

TAPP_error tapp_b200_server_submit(TAPP_b200_server server, TAPP_tensor_product plan, const void* alpha,
                                   const void* A, const void* B, const void* beta, const void* C, void* D,
                                   int64_t* ticket)
{
    struct tb_server* s = as_server(server);
    struct tb_product* p = (struct tb_product*)plan;
    if (!s || !ticket || !p || p->magic != TB_MAGIC_PRODUCT) return TAPP_B200_ERR_INVALID;
    tb_tensor_view v[4];
    int err = tb_product_views(p, v);
    if (err) return err;
    err = tb_validate(&v[0], &v[1], &v[2], &v[3], beta, C != NULL);
    if (err) return err;
    return tb_server_enqueue(s, p, v, &s->settings, alpha, A, B, beta, C, D, ticket);
}

/* the device word kernels set when a bounded wait expired, read with the
 * server's device current */
static int device_word(const struct tb_server* s)
{
    int prev = -1;
    tbk_get_device(&prev);
    if (prev != s->device) tbk_set_device(s->device);
    int e = tbk_check_device_error();
    if (prev >= 0 && prev != s->device) tbk_set_device(prev);
    return e ? cuda_code(e) : 0;
}

TAPP_error tapp_b200_server_wait(TAPP_b200_server server, int64_t ticket)
{
    struct tb_server* s = as_server(server);
    if (!s) return TAPP_B200_ERR_INVALID;
    pthread_mutex_lock(&s->lock);
    if (ticket < s->rec_base || ticket >= s->rec_base + s->n_rec) {
        pthread_mutex_unlock(&s->lock);
        return TAPP_B200_ERR_INVALID;
    }
    while (s->rec[ticket - s->rec_base].state != RQ_DONE) pthread_cond_wait(&s->cv_done, &s->lock);
    const int err = s->rec[ticket - s->rec_base].err;
    const int tc = s->rec[ticket - s->rec_base].tc;
    pthread_mutex_unlock(&s->lock);
    if (!err && tc) return device_word(s);
    return err;
}

TAPP_error tapp_b200_server_drain(TAPP_b200_server server)
{
    struct tb_server* s = as_server(server);
    if (!s) return TAPP_B200_ERR_INVALID;
    pthread_mutex_lock(&s->lock);
    while (s->completed < s->submitted) pthread_cond_wait(&s->cv_done, &s->lock);
    int err = s->first_err;
    s->first_err = 0;
    const int tc = s->tc_ran;
    pthread_mutex_unlock(&s->lock);
    if (!err && tc) err = device_word(s);
    return err;
}

static int cmp_double(const void* a, const void* b)
{
    const double x = *(const double*)a, y = *(const double*)b;
    return x < y ? -1 : x > y;
}

TAPP_error tapp_b200_server_stats(TAPP_b200_server server, tapp_b200_server_counters* out)
{
    struct tb_server* s = as_server(server);
    if (!s || !out) return TAPP_B200_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    pthread_mutex_lock(&s->lock);
    double* lat = malloc(sizeof(double) * (size_t)(s->n_rec > 0 ? s->n_rec : 1));
    int64_t n = 0;
    double sum = 0.0, flops = 0.0;
    for (int64_t i = 0; i < s->n_rec; i++) {
        const srv_rec* rc = &s->rec[i];
        if (rc->state != RQ_DONE) continue;
        const double us = 1e6 * (rc->t_done - rc->t_submit);
        if (lat) lat[n] = us;
        n++;
        sum += us;
        if (!rc->err) flops += rc->flops;
    }
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->units = s->units;
    out->grouped = s->grouped;
    out->budget_waits = s->budget_waits;
    out->peak_in_flight = s->peak_in_flight;
    out->budget_bytes = s->budget;
    out->peak_reserved = s->peak_reserved;
    out->flops = flops;
    out->span_s = s->completed ? s->t_last - s->t_first : 0.0;
    pthread_mutex_unlock(&s->lock);
    if (n > 0 && lat) {
        qsort(lat, (size_t)n, sizeof(double), cmp_double);
        /* nearest-rank percentiles */
        int64_t i50 = (int64_t)(0.50 * (double)n + 0.999999) - 1;
        int64_t i99 = (int64_t)(0.99 * (double)n + 0.999999) - 1;
        if (i50 < 0) i50 = 0;
        if (i99 < 0) i99 = 0;
        out->p50_us = lat[i50];
        out->p99_us = lat[i99];
        out->max_us = lat[n - 1];
        out->mean_us = sum / (double)n;
    }
    if (out->span_s > 0) out->requests_per_s = (double)out->completed / out->span_s;
    free(lat);
    return 0;
}

TAPP_error tapp_b200_server_reset_stats(TAPP_b200_server server)
{
    struct tb_server* s = as_server(server);
    if (!s) return TAPP_B200_ERR_INVALID;
    int err = tapp_b200_server_drain(server);
    pthread_mutex_lock(&s->lock);
    s->rec_base += s->n_rec;
    s->n_rec = 0;
    s->submitted = s->completed = s->failed = s->units = s->grouped = s->budget_waits = 0;
    s->peak_reserved = s->reserved;
    s->peak_in_flight = s->in_flight;
    s->t_first = s->t_last = 0.0;
    s->tc_ran = 0;
    pthread_mutex_unlock(&s->lock);
    return err;
}

TAPP_error tapp_b200_server_destroy(TAPP_b200_server server)
{
    struct tb_server* s = as_server(server);
    if (!s) return TAPP_B200_ERR_INVALID;
    int err = tapp_b200_server_drain(server);
    live_remove(s);
    pthread_mutex_lock(&s->lock);
    s->stop = 1;
    pthread_cond_broadcast(&s->cv_sched);
    pthread_mutex_unlock(&s->lock);
    pthread_join(s->thread, NULL);
    pthread_mutex_lock(&s->lock);
    s->reap_stop = 1;  /* the reaper ends once the issued units have completed */
    pthread_cond_broadcast(&s->cv_reap);
    pthread_mutex_unlock(&s->lock);
    pthread_join(s->reaper, NULL);
    for (int i = 0; i < s->n_streams; i++) {
        tbk_stream_sync(s->streams[i]);
        tbk_stream_destroy(s->streams[i]);
    }
    for (int i = 0; i < s->n_slabs; i++)
        if (s->slab[i]) tbk_host_free(s->slab[i]);
    free(s->rec);
    pthread_mutex_destroy(&s->lock);
    pthread_cond_destroy(&s->cv_sched);
    pthread_cond_destroy(&s->cv_done);
    pthread_cond_destroy(&s->cv_reap);
    s->magic = 0;
    free(s);
    return err;
}

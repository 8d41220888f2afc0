/*
 * Handles, executors, status objects and attributes.
 *
 * Executors: TAPP_create_executor returns a pointer whose first int is 1, the
 * id of the reference's executor (reference_implementation/src/executor.c:
 * 9-18), followed by this library's execution settings. Executors this
 * library created are kept in a registry; any other non-NULL executor is
 * accepted when it points at an int 1, 2 or 12, as the reference accepts it
 * (product.c:878-885), and runs with default settings.
 *
 * Handles: the reference's handle is an unused placeholder (handle.c:9-17)
 * and its callers sometimes pass one that was never created; the product
 * only trusts a handle found in this library's registry.
 *
 * Attributes (declared by the reference in attributes.h:14-18, never
 * implemented there): an attribute object is an executor or a status; keys
 * are listed in tapp_b200.h.
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "tb_internal.h"

#define REG_MAX 4096

static pthread_mutex_t reg_lock = PTHREAD_MUTEX_INITIALIZER;
static TAPP_executor exec_reg[REG_MAX];
static int exec_n;
static TAPP_handle handle_reg[REG_MAX];
static int handle_n;

static void reg_add(intptr_t* arr, int* n, intptr_t v)
{
    pthread_mutex_lock(&reg_lock);
    if (*n < REG_MAX) arr[(*n)++] = v;
    pthread_mutex_unlock(&reg_lock);
}

static void reg_remove(intptr_t* arr, int* n, intptr_t v)
{
    pthread_mutex_lock(&reg_lock);
    for (int i = 0; i < *n; i++)
        if (arr[i] == v) { arr[i] = arr[--(*n)]; break; }
    pthread_mutex_unlock(&reg_lock);
}

static int reg_has(const intptr_t* arr, const int* n, intptr_t v)
{
    int found = 0;
    pthread_mutex_lock(&reg_lock);
    for (int i = 0; i < *n; i++)
        if (arr[i] == v) { found = 1; break; }
    pthread_mutex_unlock(&reg_lock);
    return found;
}

int tb_executor_is_ours(TAPP_executor e) { return e && reg_has(exec_reg, &exec_n, e); }
int tb_handle_is_ours(TAPP_handle h) { return h && reg_has(handle_reg, &handle_n, h); }

/* handle.c:9-12 */
TAPP_error TAPP_create_handle(TAPP_handle* handle)
{
    struct tb_handle* h = calloc(1, sizeof(*h));
    if (!h) return TAPP_B200_ERR_NOMEM;
    h->magic = TB_MAGIC_HANDLE;
    h->device = -1;
    *handle = (TAPP_handle)h;
    reg_add(handle_reg, &handle_n, *handle);
    return 0;
}

/* handle.c:14-17 */
TAPP_error TAPP_destroy_handle(TAPP_handle handle)
{
    if (!handle) return 0;
    reg_remove(handle_reg, &handle_n, handle);
    free((void*)handle);
    return 0;
}

static int env_int(const char* name, int dflt)
{
    const char* v = getenv(name);
    if (!v || !*v) return dflt;
    if (!strcmp(v, "split") || !strcmp(v, "split_bf16")) return 1;
    if (!strcmp(v, "plain")) return 0;
    return atoi(v);
}

/* executor.c:9-18 */
TAPP_error TAPP_create_executor(TAPP_executor* exec)
{
    struct tb_executor* e = calloc(1, sizeof(*e));
    if (!e) return TAPP_B200_ERR_NOMEM;
    e->id = 1;
    e->f32_mode = env_int("TAPP_B200_F32_MODE", 0);
    e->force_path = env_int("TAPP_B200_PATH", 0);
    e->f64_mode = env_int("TAPP_B200_F64_MODE", 0);
    if (e->f64_mode < 2 || e->f64_mode > 16) e->f64_mode = 0;
    *exec = (TAPP_executor)e;
    reg_add(exec_reg, &exec_n, *exec);
    return 0;
}

/* executor.c:20-23 */
TAPP_error TAPP_destroy_executor(TAPP_executor exec)
{
    if (!exec) return 0;
    reg_remove(exec_reg, &exec_n, exec);
    free((void*)exec);
    return 0;
}

/* status.h:17 (declared, not implemented, by the reference) */
TAPP_error TAPP_destroy_status(TAPP_status status)
{
    struct tb_status* s = (struct tb_status*)status;
    if (!s) return 0;
    if (s->magic != TB_MAGIC_STATUS) return TAPP_B200_ERR_INVALID;
    s->magic = 0;
    free(s);
    return 0;
}

static struct tb_status* as_status(TAPP_attr a)
{
    struct tb_status* s = (struct tb_status*)a;
    if (!s || tb_executor_is_ours((TAPP_executor)a)) return NULL;
    return s->magic == TB_MAGIC_STATUS ? s : NULL;
}

/* attributes.h:14 */
TAPP_error TAPP_attr_set(TAPP_attr attr, TAPP_key key, void* value)
{
    if (!tb_executor_is_ours((TAPP_executor)attr)) return TAPP_B200_ERR_INVALID;
    struct tb_executor* e = (struct tb_executor*)attr;
    switch (key) {
    case TAPP_B200_ATTR_STREAM: e->stream = value; return 0;
    case TAPP_B200_ATTR_ASYNC: e->async = value ? *(int*)value : 0; return 0;
    case TAPP_B200_ATTR_F32_MODE: e->f32_mode = value ? *(int*)value : 0; return 0;
    case TAPP_B200_ATTR_PATH: e->force_path = value ? *(int*)value : 0; return 0;
    case TAPP_B200_ATTR_WANT_STATUS: e->want_status = value ? *(int*)value : 0; return 0;
    case TAPP_B200_ATTR_F64_MODE: {
        const int v = value ? *(int*)value : 0;
        if (v != 0 && (v < 2 || v > 16)) return TAPP_B200_ERR_INVALID;
        e->f64_mode = v;
        return 0;
    }
    case TAPP_B200_ATTR_TILE: {
        const int v = value ? *(int*)value : 0;
        if (v < 0 || v > 2) return TAPP_B200_ERR_INVALID;
        e->tile = v;
        return 0;
    }
    case TAPP_B200_ATTR_SERVER:
        if (value && !tb_server_is_live((const struct tb_server*)value)) return TAPP_B200_ERR_INVALID;
        e->server = (struct tb_server*)value;
        return 0;
    default: return TAPP_B200_ERR_INVALID;
    }
}

/* attributes.h:16. Executor keys store their value into *value (the stream
 * itself for TAPP_B200_ATTR_STREAM, else an int); status keys write an int
 * or a double into the memory *value points at. */
TAPP_error TAPP_attr_get(TAPP_attr attr, TAPP_key key, void** value)
{
    if (!value) return TAPP_B200_ERR_INVALID;
    if (tb_executor_is_ours((TAPP_executor)attr)) {
        struct tb_executor* e = (struct tb_executor*)attr;
        switch (key) {
        case TAPP_B200_ATTR_STREAM: *value = e->stream; return 0;
        case TAPP_B200_ATTR_ASYNC: *(int*)*value = e->async; return 0;
        case TAPP_B200_ATTR_F32_MODE: *(int*)*value = e->f32_mode; return 0;
        case TAPP_B200_ATTR_PATH: *(int*)*value = e->force_path; return 0;
        case TAPP_B200_ATTR_WANT_STATUS: *(int*)*value = e->want_status; return 0;
        case TAPP_B200_ATTR_SERVER: *value = e->server; return 0;
        case TAPP_B200_ATTR_F64_MODE: *(int*)*value = e->f64_mode; return 0;
        case TAPP_B200_ATTR_TILE: *(int*)*value = e->tile; return 0;
        default: return TAPP_B200_ERR_INVALID;
        }
    }
    struct tb_status* s = as_status(attr);
    if (!s || !*value) return TAPP_B200_ERR_INVALID;
    switch (key) {
    case TAPP_B200_STATUS_PATH: *(int*)*value = s->path; return 0;
    case TAPP_B200_STATUS_KERNELS: *(int*)*value = s->kernels; return 0;
    case TAPP_B200_STATUS_TC_MODE: *(int*)*value = s->tc_mode; return 0;
    case TAPP_B200_STATUS_FLOPS: *(double*)*value = s->flops; return 0;
    case TAPP_B200_STATUS_DEVICE_US: *(double*)*value = s->device_us; return 0;
    case TAPP_B200_STATUS_MAIN_US: *(double*)*value = s->main_us; return 0;
    case TAPP_B200_STATUS_ERR_BOUND: *(double*)*value = s->err_bound; return 0;
    default: return TAPP_B200_ERR_INVALID;
    }
}

/* attributes.h:18: restores an executor key to its default */
TAPP_error TAPP_attr_clear(TAPP_attr attr, TAPP_key key)
{
    if (!tb_executor_is_ours((TAPP_executor)attr)) return TAPP_B200_ERR_INVALID;
    struct tb_executor* e = (struct tb_executor*)attr;
    switch (key) {
    case TAPP_B200_ATTR_STREAM: e->stream = NULL; return 0;
    case TAPP_B200_ATTR_ASYNC: e->async = 0; return 0;
    case TAPP_B200_ATTR_F32_MODE: e->f32_mode = 0; return 0;
    case TAPP_B200_ATTR_PATH: e->force_path = 0; return 0;
    case TAPP_B200_ATTR_WANT_STATUS: e->want_status = 0; return 0;
    case TAPP_B200_ATTR_SERVER: e->server = NULL; return 0;
    case TAPP_B200_ATTR_F64_MODE: e->f64_mode = 0; return 0;
    case TAPP_B200_ATTR_TILE: e->tile = 0; return 0;
    default: return TAPP_B200_ERR_INVALID;
    }
}

long long tapp_b200_kernel_launches(void)
{
    return tbk_launch_count();
}

long long tapp_b200_device_allocations(void)
{
    return tbk_allocation_count();
}

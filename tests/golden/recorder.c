/*
 * Recording shim for golden fixtures (test infrastructure).
 *
 * Exports the TAPP C ABI, forwards every call to the library named by
 * $TAPP_RECORD_TARGET (loaded with dlopen) and appends one JSON object per
 * TAPP_execute_product call to $TAPP_RECORD_OUT: the layouts, labels, ops,
 * precision, scalars, every element each operand addresses, D before and
 * after the call, and the returned code. Linking the reference's own
 * example programs against this shim turns their hand-written cases into
 * fixtures that a GPU test can replay without the reference present.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int TAPP_error;
typedef intptr_t TAPP_tensor_info, TAPP_tensor_product, TAPP_handle, TAPP_executor, TAPP_status;

static void* target;
static int call_no;

static void* sym(const char* name)
{
    if (!target) {
        const char* path = getenv("TAPP_RECORD_TARGET");
        target = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!target) { fprintf(stderr, "recorder: %s\n", dlerror()); exit(3); }
    }
    void* f = dlsym(target, name);
    if (!f) { fprintf(stderr, "recorder: missing %s\n", name); exit(3); }
    return f;
}

/* -------- bookkeeping of infos and plans -------- */
#define MAXOBJ 4096
typedef struct { TAPP_tensor_info h; int type; } info_rec;
typedef struct { TAPP_tensor_product h; int ops[4]; TAPP_tensor_info t[4]; int64_t* idx[4]; int prec; } plan_rec;
static info_rec infos[MAXOBJ];
static int n_infos;
static plan_rec plans[MAXOBJ];
static int n_plans;

static int info_type(TAPP_tensor_info h)
{
    for (int i = n_infos - 1; i >= 0; i--) if (infos[i].h == h) return infos[i].type;
    return -1;
}

/* -------- forwarded API -------- */
#define FWD(ret, name, params, args) \
    ret name params { return ((ret(*)params)sym(#name)) args; }

TAPP_error TAPP_create_tensor_info(TAPP_tensor_info* info, int type, int nmode, const int64_t* ext, const int64_t* str)
{
    TAPP_error e = ((TAPP_error(*)(TAPP_tensor_info*, int, int, const int64_t*, const int64_t*))
                    sym("TAPP_create_tensor_info"))(info, type, nmode, ext, str);
    if (e == 0 && n_infos < MAXOBJ) { infos[n_infos].h = *info; infos[n_infos].type = type; n_infos++; }
    return e;
}
FWD(TAPP_error, TAPP_destroy_tensor_info, (TAPP_tensor_info i), (i))
FWD(int, TAPP_get_nmodes, (TAPP_tensor_info i), (i))
FWD(TAPP_error, TAPP_set_nmodes, (TAPP_tensor_info i, int n), (i, n))
FWD(void, TAPP_get_extents, (TAPP_tensor_info i, int64_t* e), (i, e))
FWD(TAPP_error, TAPP_set_extents, (TAPP_tensor_info i, const int64_t* e), (i, e))
FWD(void, TAPP_get_strides, (TAPP_tensor_info i, int64_t* s), (i, s))
FWD(TAPP_error, TAPP_set_strides, (TAPP_tensor_info i, const int64_t* s), (i, s))
FWD(TAPP_error, TAPP_create_handle, (TAPP_handle* h), (h))
FWD(TAPP_error, TAPP_destroy_handle, (TAPP_handle h), (h))
FWD(TAPP_error, TAPP_create_executor, (TAPP_executor* e), (e))
FWD(TAPP_error, TAPP_destroy_executor, (TAPP_executor e), (e))
FWD(bool, TAPP_check_success, (TAPP_error e), (e))
FWD(size_t, TAPP_explain_error, (TAPP_error e, size_t n, char* m), (e, n, m))

TAPP_error TAPP_create_tensor_product(TAPP_tensor_product* plan, TAPP_handle handle,
                                      int opA, TAPP_tensor_info A, const int64_t* iA,
                                      int opB, TAPP_tensor_info B, const int64_t* iB,
                                      int opC, TAPP_tensor_info C, const int64_t* iC,
                                      int opD, TAPP_tensor_info D, const int64_t* iD, int prec)
{
    TAPP_error e = ((TAPP_error(*)(TAPP_tensor_product*, TAPP_handle, int, TAPP_tensor_info, const int64_t*,
                                   int, TAPP_tensor_info, const int64_t*, int, TAPP_tensor_info, const int64_t*,
                                   int, TAPP_tensor_info, const int64_t*, int))sym("TAPP_create_tensor_product"))(
        plan, handle, opA, A, iA, opB, B, iB, opC, C, iC, opD, D, iD, prec);
    if (n_plans < MAXOBJ) {
        plan_rec* p = &plans[n_plans++];
        p->h = *plan;
        int ops[4] = {opA, opB, opC, opD};
        TAPP_tensor_info t[4] = {A, B, C, D};
        const int64_t* ix[4] = {iA, iB, iC, iD};
        for (int k = 0; k < 4; k++) {
            p->ops[k] = ops[k];
            p->t[k] = t[k];
            int n = TAPP_get_nmodes(t[k]);
            p->idx[k] = malloc(sizeof(int64_t) * (n > 0 ? n : 1));
            memcpy(p->idx[k], ix[k], sizeof(int64_t) * (n > 0 ? n : 0));
        }
        p->prec = prec;
    }
    return e;
}
FWD(TAPP_error, TAPP_destroy_tensor_product, (TAPP_tensor_product p), (p))

static int elem_bytes(int t)
{
    switch (t) { case 0: return 4; case 1: return 8; case 2: return 8; case 3: return 16; case 4: case 5: return 2; }
    return 0;
}

static void dump_scalar(FILE* f, int type, const void* p)
{
    if (!p) { fprintf(f, "null"); return; }
    switch (type) {
    case 0: fprintf(f, "[%.17g,0]", (double)*(const float*)p); break;
    case 1: fprintf(f, "[%.17g,0]", *(const double*)p); break;
    case 2: fprintf(f, "[%.17g,%.17g]", (double)((const float*)p)[0], (double)((const float*)p)[1]); break;
    case 3: fprintf(f, "[%.17g,%.17g]", ((const double*)p)[0], ((const double*)p)[1]); break;
    default: fprintf(f, "null");
    }
}

/* Every element between the lowest and highest addressed offset. */
static void dump_span(FILE* f, int type, int n, const int64_t* ext, const int64_t* str, const void* base)
{
    int64_t lo = 0, hi = 0;
    for (int i = 0; i < n; i++) {
        if (ext[i] == 0) { fprintf(f, "{\"lo\":0,\"data\":[]}"); return; }
        if (str[i] < 0) lo += str[i] * (ext[i] - 1); else hi += str[i] * (ext[i] - 1);
    }
    fprintf(f, "{\"lo\":%lld,\"data\":[", (long long)lo);
    int b = elem_bytes(type);
    for (int64_t o = lo; o <= hi && base; o++) {
        if (o != lo) fputc(',', f);
        dump_scalar(f, type, (const char*)base + o * b);
    }
    fprintf(f, "]}");
}

TAPP_error TAPP_execute_product(TAPP_tensor_product plan, TAPP_executor exec, TAPP_status* status,
                                const void* alpha, const void* A, const void* B,
                                const void* beta, const void* C, void* D)
{
    plan_rec* p = NULL;
    for (int i = n_plans - 1; i >= 0; i--) if (plans[i].h == plan) { p = &plans[i]; break; }
    const char* out = getenv("TAPP_RECORD_OUT");
    FILE* f = (p && out) ? fopen(out, "a") : NULL;
    int n[4], type[4];
    int64_t ext[4][64], str[4][64];
    const void* ptr[4] = {A, B, C, D};
    if (f) {
        for (int k = 0; k < 4; k++) {
            n[k] = TAPP_get_nmodes(p->t[k]);
            TAPP_get_extents(p->t[k], ext[k]);
            TAPP_get_strides(p->t[k], str[k]);
            type[k] = info_type(p->t[k]);
        }
        const char* prog = getenv("TAPP_RECORD_PROGRAM");
        fprintf(f, "{\"program\":\"%s\",\"call\":%d,\"prec\":%d,\"alpha\":", prog ? prog : "", call_no, p->prec);
        dump_scalar(f, type[3], alpha);
        fprintf(f, ",\"beta\":");
        dump_scalar(f, type[3], beta);
        fprintf(f, ",\"tensors\":[");
        for (int k = 0; k < 4; k++) {
            fprintf(f, "%s{\"type\":%d,\"op\":%d,\"extents\":[", k ? "," : "", type[k], p->ops[k]);
            for (int i = 0; i < n[k]; i++) fprintf(f, "%s%lld", i ? "," : "", (long long)ext[k][i]);
            fprintf(f, "],\"strides\":[");
            for (int i = 0; i < n[k]; i++) fprintf(f, "%s%lld", i ? "," : "", (long long)str[k][i]);
            fprintf(f, "],\"idx\":[");
            for (int i = 0; i < n[k]; i++) fprintf(f, "%s%lld", i ? "," : "", (long long)p->idx[k][i]);
            fprintf(f, "],\"null\":%s,\"span\":", ptr[k] ? "false" : "true");
            dump_span(f, type[k], n[k], ext[k], str[k], ptr[k]);
            fprintf(f, "}");
        }
        fprintf(f, "]");
    }
    TAPP_error e = ((TAPP_error(*)(TAPP_tensor_product, TAPP_executor, TAPP_status*, const void*, const void*,
                                   const void*, const void*, const void*, void*))sym("TAPP_execute_product"))(
        plan, exec, status, alpha, A, B, beta, C, D);
    if (f) {
        fprintf(f, ",\"error\":%d,\"D_after\":", e);
        dump_span(f, type[3], n[3], ext[3], str[3], D);
        fprintf(f, "}\n");
        fclose(f);
    }
    call_no++;
    return e;
}

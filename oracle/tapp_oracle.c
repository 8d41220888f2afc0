/*
 * CPU oracle for the TAPP tensor product — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's TAPP_execute_product
 * (reference_implementation/src/product.c). The GPU library does not link,
 * load or call this code; tests, the smoke check and the benchmark's CPU
 * baseline leg use it as the checker.
 *
 * Scalar arithmetic of the reference is reproduced with a small value type
 * that carries the precision an expression is evaluated in. Every operation
 * is done in binary64 and rounded to that precision. For binary32 operands
 * this gives the binary32 result exactly: binary64 has 53 >= 2*24+2 bits, so
 * the double rounding of +, -, * is innocuous (S. A. Figueroa, "When is double
 * rounding innocuous?", SIGNUM Newsletter 30(3), 1995). binary16 and bfloat16
 * operands are evaluated in binary32 and rounded when stored, which is what
 * ISO C's excess-precision rule (FLT_EVAL_METHOD for _Float16 on x86-64)
 * prescribes for the reference's -std=c99 build.
 */
#include "tapp_oracle.h"

#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

enum { T_F32 = 0, T_F64 = 1, T_C32 = 2, T_C64 = 3, T_F16 = 4, T_BF16 = 5 };
enum { PR_DEFAULT = -1, PR_F32 = 0, PR_F64 = 1, PR_F16 = 4, PR_F16_F32 = 5, PR_BF16_F32 = 6 };

/* ------------------------------------------------------------------ */
/* scalar formats                                                      */
/* ------------------------------------------------------------------ */

typedef enum { P_H = 0, P_BH = 1, P_S = 2, P_D = 3 } pr_t;  /* f16, bf16, f32, f64 */
typedef struct { pr_t p; int c; } vtype;
typedef struct { pr_t p; int c; double re, im; } val;

/* Round x to a binary format with `p` significand bits, minimum normal
 * exponent `emin` (value 2^emin) and largest finite value `maxv`,
 * round-to-nearest-even, overflow to infinity, gradual underflow. */
static double rnd_fmt(double x, int p, int emin, double maxv)
{
    if (x == 0.0 || !isfinite(x)) return x;
    int e;
    (void)frexp(x, &e);               /* x = m * 2^e, 0.5 <= |m| < 1 */
    int q = e - p;                    /* exponent of one unit in the last place */
    if (q < emin + 1 - p) q = emin + 1 - p;
    double y = ldexp(nearbyint(ldexp(x, -q)), q);
    if (fabs(y) > maxv) return copysign(INFINITY, x);
    return y;
}

#define F16_MAX 65504.0
#define BF16_MAX 3.3895313892515355e38  /* (2 - 2^-7) * 2^127 */

static double rp(pr_t p, double x)
{
    switch (p) {
    case P_D: return x;
    case P_S: return (double)(float)x;
    case P_H: return rnd_fmt(x, 11, -14, F16_MAX);
    case P_BH: return rnd_fmt(x, 8, -126, BF16_MAX);
    }
    return x;
}

/* Precision an operation on two operands is evaluated in: the wider one,
 * and never narrower than binary32 (excess precision of 16-bit types). */
static pr_t evp(pr_t a, pr_t b)
{
    pr_t m = a > b ? a : b;
    return m < P_S ? P_S : m;
}

static val vzero(vtype t) { val v = {t.p, t.c, 0.0, 0.0}; return v; }

static val vconv(val v, vtype t)
{
    val r;
    r.p = t.p;
    r.c = t.c;
    r.re = rp(t.p, v.re);
    r.im = t.c ? (v.c ? rp(t.p, v.im) : 0.0) : 0.0;
    return r;
}

static val vconj(val v)
{
    if (v.c) v.im = -v.im;
    return v;
}

static val vmul(val a, val b)
{
    val r;
    r.p = evp(a.p, b.p);
    r.c = a.c || b.c;
    if (!a.c && !b.c) {
        r.re = rp(r.p, a.re * b.re);
        r.im = 0.0;
    } else if (a.c && !b.c) {
        r.re = rp(r.p, a.re * b.re);
        r.im = rp(r.p, a.im * b.re);
    } else if (!a.c && b.c) {
        r.re = rp(r.p, a.re * b.re);
        r.im = rp(r.p, a.re * b.im);
    } else {
        double ac = rp(r.p, a.re * b.re), bd = rp(r.p, a.im * b.im);
        double ad = rp(r.p, a.re * b.im), bc = rp(r.p, a.im * b.re);
        r.re = rp(r.p, ac - bd);
        r.im = rp(r.p, ad + bc);
    }
    return r;
}

static val vadd(val a, val b)
{
    val r;
    r.p = evp(a.p, b.p);
    r.c = a.c || b.c;
    r.re = rp(r.p, a.re + b.re);
    if (a.c && b.c) r.im = rp(r.p, a.im + b.im);
    else if (a.c) r.im = a.im;
    else if (b.c) r.im = b.im;
    else r.im = 0.0;
    return r;
}

static int is_cplx(int t) { return t == T_C32 || t == T_C64; }

static vtype storage_vt(int t)
{
    vtype v = {P_S, 0};
    switch (t) {
    case T_F32: v.p = P_S; break;
    case T_F64: v.p = P_D; break;
    case T_C32: v.p = P_S; v.c = 1; break;
    case T_C64: v.p = P_D; v.c = 1; break;
    case T_F16: v.p = P_H; break;
    case T_BF16: v.p = P_BH; break;
    }
    return v;
}

/* Internal operand type for a precision (alloc_val, product.c:1104-1230). */
static vtype prec_vt(int prec, int t)
{
    vtype v;
    v.c = is_cplx(t);
    switch (prec) {
    case PR_F32: v.p = P_S; break;
    case PR_F64: v.p = P_D; break;
    case PR_F16: case PR_F16_F32: v.p = P_H; break;
    case PR_BF16_F32: v.p = P_BH; break;
    default: return storage_vt(t);
    }
    return v;
}

/* Accumulator type (alloc_accum, product.c:1012-1102). */
static vtype acc_vt(int prec, int tD)
{
    vtype v;
    v.c = is_cplx(tD);
    switch (prec) {
    case PR_F32: case PR_F16_F32: case PR_BF16_F32: v.p = P_S; break;
    case PR_F64: v.p = P_D; break;
    case PR_F16: v.p = P_H; break;
    default: return storage_vt(tD);
    }
    return v;
}

static double f16_decode(uint16_t h)
{
    int s = h >> 15, e = (h >> 10) & 0x1f, m = h & 0x3ff;
    double v;
    if (e == 0) v = ldexp((double)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexp((double)(m | 0x400), e - 25);
    return s ? -v : v;
}

static uint16_t f16_encode(double x)  /* x already on the binary16 grid */
{
    uint16_t s = signbit(x) ? 0x8000 : 0;
    double a = fabs(x);
    if (isnan(x)) return 0x7e00;
    if (isinf(a)) return s | 0x7c00;
    if (a == 0.0) return s;
    int e;
    (void)frexp(a, &e);                /* a = m * 2^e, m in [0.5,1) */
    int ub = e - 1 + 15;               /* biased exponent */
    if (ub <= 0) return s | (uint16_t)ldexp(a, 24);
    uint16_t m = (uint16_t)(ldexp(a, 11 - e) - 1024.0);
    return s | (uint16_t)(ub << 10) | m;
}

static double bf16_decode(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

static uint16_t bf16_encode(double x)  /* x already on the bfloat16 grid */
{
    float f = (float)x;
    uint32_t u;
    memcpy(&u, &f, 4);
    return (uint16_t)(u >> 16);
}

static val load_elem(const void* base, int64_t off, int t)
{
    val v = {P_S, 0, 0.0, 0.0};
    switch (t) {
    case T_F32: v.p = P_S; v.re = ((const float*)base)[off]; break;
    case T_F64: v.p = P_D; v.re = ((const double*)base)[off]; break;
    case T_C32: v.p = P_S; v.c = 1; v.re = ((const float*)base)[2 * off]; v.im = ((const float*)base)[2 * off + 1]; break;
    case T_C64: v.p = P_D; v.c = 1; v.re = ((const double*)base)[2 * off]; v.im = ((const double*)base)[2 * off + 1]; break;
    case T_F16: v.p = P_H; v.re = f16_decode(((const uint16_t*)base)[off]); break;
    case T_BF16: v.p = P_BH; v.re = bf16_decode(((const uint16_t*)base)[off]); break;
    }
    return v;
}

static void store_elem(void* base, int64_t off, int t, val v)
{
    v = vconv(v, storage_vt(t));
    switch (t) {
    case T_F32: ((float*)base)[off] = (float)v.re; break;
    case T_F64: ((double*)base)[off] = v.re; break;
    case T_C32: ((float*)base)[2 * off] = (float)v.re; ((float*)base)[2 * off + 1] = (float)v.im; break;
    case T_C64: ((double*)base)[2 * off] = v.re; ((double*)base)[2 * off + 1] = v.im; break;
    case T_F16: ((uint16_t*)base)[off] = f16_encode(v.re); break;
    case T_BF16: ((uint16_t*)base)[off] = bf16_encode(v.re); break;
    }
}

/* ------------------------------------------------------------------ */
/* validation chain (product.c:199-206, helpers :757-885)              */
/* ------------------------------------------------------------------ */

/* check_idx_occurrence, product.c:757-784 */
static int chk_occurrence(int n, const int64_t* idx, int na, const int64_t* ia, int nb, const int64_t* ib, int code)
{
    for (int i = 0; i < n; i++) {
        int found = 0;
        for (int j = 0; j < na; j++) if (idx[i] == ia[j]) { found = 1; break; }
        for (int j = 0; j < nb && !found; j++) if (idx[i] == ib[j]) { found = 1; break; }
        if (!found) return code;
    }
    return 0;
}

/* check_extents, product.c:786-813 */
static int chk_extents(int na, const int64_t* ia, const int64_t* ea,
                       int nb, const int64_t* ib, const int64_t* eb,
                       int nd, const int64_t* id, const int64_t* ed,
                       int c_aa, int c_ab, int c_ad)
{
    for (int i = 0; i < na; i++) {
        for (int j = 0; j < na; j++) if (ia[i] == ia[j] && ea[i] != ea[j]) return c_aa;
        for (int j = 0; j < nb; j++) if (ia[i] == ib[j] && ea[i] != eb[j]) return c_ab;
        for (int j = 0; j < nd; j++) if (ia[i] == id[j] && ea[i] != ed[j]) return c_ad;
    }
    return 0;
}

/* check_same_structure, product.c:815-834 (C first, D second) */
static int chk_structure(int nc, const int64_t* ic, const int64_t* ec, int nd, const int64_t* id, const int64_t* ed)
{
    if (nc != nd) return 5;
    for (int i = 0; i < nd; i++) {
        if (id[i] != ic[i]) return 6;
        if (ed[i] != ec[i]) return 7;
    }
    return 0;
}

/* check_self_aliasing, product.c:836-870: sort (|stride|, extent) pairs by
 * stride, ties by extent, and require each stride to clear the span of the
 * previous mode. The reference's merge sort copies through int arrays
 * (:923-926); strides here stay 64-bit. */
static int chk_aliasing(int n, const int64_t* ext, const int64_t* str)
{
    if (n <= 1) return 0;
    for (int i = 0; i < n; i++) if (str[i] == 0) return 8;
    int64_t* s = malloc(sizeof(int64_t) * n);
    int64_t* e = malloc(sizeof(int64_t) * n);
    for (int i = 0; i < n; i++) { s[i] = str[i] < 0 ? -str[i] : str[i]; e[i] = ext[i]; }
    for (int i = 1; i < n; i++) {  /* stable insertion sort, same order as the merge */
        int64_t ks = s[i], ke = e[i];
        int j = i - 1;
        while (j >= 0 && (s[j] > ks || (s[j] == ks && e[j] > ke))) { s[j + 1] = s[j]; e[j + 1] = e[j]; j--; }
        s[j + 1] = ks; e[j + 1] = ke;
    }
    int r = 0;
    for (int i = 0; i < n - 1; i++) if (s[i + 1] < s[i] * e[i]) { r = 8; break; }
    free(s);
    free(e);
    return r;
}

static int scalar_is_zero(const void* s, int t)
{
    val v = load_elem(s, 0, t);
    return v.re == 0.0 && v.im == 0.0;
}

int oracle_validate(const oracle_tensor* A, const oracle_tensor* B,
                    const oracle_tensor* C, const oracle_tensor* D,
                    const void* beta, int C_present)
{
    int e = chk_occurrence(D->nmode, D->idx, A->nmode, A->idx, B->nmode, B->idx, 4);
    if (!e) e = chk_extents(A->nmode, A->idx, A->extents, B->nmode, B->idx, B->extents, D->nmode, D->idx, D->extents, 9, 1, 2);
    if (!e) e = chk_extents(B->nmode, B->idx, B->extents, A->nmode, A->idx, A->extents, D->nmode, D->idx, D->extents, 10, 1, 3);
    if (!e) e = chk_extents(D->nmode, D->idx, D->extents, A->nmode, A->idx, A->extents, B->nmode, B->idx, B->extents, 11, 2, 3);
    if (!e) e = chk_structure(C->nmode, C->idx, C->extents, D->nmode, D->idx, D->extents);
    if (!e) e = chk_aliasing(D->nmode, D->extents, D->strides);
    if (!e && !C_present && !scalar_is_zero(beta, D->type)) e = 12;
    return e;
}

/* ------------------------------------------------------------------ */
/* index planning (product.c:265-310, helpers :538-735, :969-1010)     */
/* ------------------------------------------------------------------ */

#define OMAX 64

typedef struct { int n; int64_t idx[OMAX], ext[OMAX], str[OMAX]; } folded;

/* compress_repeated_indices, product.c:969-1010: one mode per distinct
 * label, its stride the sum of the strides of the repeats. */
static void fold(const oracle_tensor* t, folded* f)
{
    f->n = 0;
    for (int i = 0; i < t->nmode; i++) {
        int seen = 0;
        for (int j = 0; j < f->n; j++) if (f->idx[j] == t->idx[i]) seen = 1;
        if (seen) continue;
        int k = f->n++;
        f->idx[k] = t->idx[i];
        f->ext[k] = t->extents[i];
        f->str[k] = 0;
        for (int j = 0; j < t->nmode; j++) if (t->idx[j] == t->idx[i]) f->str[k] += t->strides[j];
    }
}

static int find(const folded* f, int64_t label)
{
    for (int i = 0; i < f->n; i++) if (f->idx[i] == label) return i;
    return -1;
}

typedef struct {
    folded A, B, C, D;
    int nfree;                               /* D's modes */
    int64_t free_ext[OMAX], sfA[OMAX], sfB[OMAX], sC[OMAX], sD[OMAX];
    int nbin;                                /* in A and B, not in D (A's order) */
    int64_t bin_ext[OMAX], sbA[OMAX], sbB[OMAX];
    int nuA, nuB;                            /* only in A / only in B */
    int64_t uA_ext[OMAX], suA[OMAX], uB_ext[OMAX], suB[OMAX];
} layout;

static void plan_layout(const oracle_tensor* A, const oracle_tensor* B,
                        const oracle_tensor* C, const oracle_tensor* D, layout* L)
{
    fold(A, &L->A); fold(B, &L->B); fold(C, &L->C); fold(D, &L->D);
    L->nfree = L->D.n;
    for (int j = 0; j < L->D.n; j++) {
        int a = find(&L->A, L->D.idx[j]), b = find(&L->B, L->D.idx[j]);
        L->free_ext[j] = L->D.ext[j];
        L->sfA[j] = a >= 0 ? L->A.str[a] : 0;   /* extract_free_strides :621-641 */
        L->sfB[j] = b >= 0 ? L->B.str[b] : 0;
        L->sC[j] = j < L->C.n ? L->C.str[j] : 0;
        L->sD[j] = L->D.str[j];
    }
    L->nbin = L->nuA = L->nuB = 0;
    for (int i = 0; i < L->A.n; i++) {
        int b = find(&L->B, L->A.idx[i]), d = find(&L->D, L->A.idx[i]);
        if (b >= 0 && d < 0) {                  /* :538-570 */
            L->bin_ext[L->nbin] = L->A.ext[i];
            L->sbA[L->nbin] = L->A.str[i];
            L->sbB[L->nbin] = L->B.str[b];
            L->nbin++;
        } else if (b < 0 && d < 0) {            /* :588-619 */
            L->uA_ext[L->nuA] = L->A.ext[i];
            L->suA[L->nuA] = L->A.str[i];
            L->nuA++;
        }
    }
    for (int i = 0; i < L->B.n; i++) {
        if (find(&L->A, L->B.idx[i]) < 0 && find(&L->D, L->B.idx[i]) < 0) {
            L->uB_ext[L->nuB] = L->B.ext[i];
            L->suB[L->nuB] = L->B.str[i];
            L->nuB++;
        }
    }
}

static int64_t size_of(int n, const int64_t* e)
{
    int64_t s = 1;
    for (int i = 0; i < n; i++) s *= e[i];
    return s;
}

/* increment_coordinates, product.c:702-715: first coordinate fastest. */
static void incr(int64_t* c, int n, const int64_t* e)
{
    for (int k = 0; k < n; k++) {
        c[k]++;
        if (c[k] < e[k]) return;
        c[k] = 0;
    }
}

static int64_t dot(int n, const int64_t* c, const int64_t* s)
{
    int64_t r = 0;
    for (int i = 0; i < n; i++) r += c[i] * s[i];
    return r;
}

/* Whether op_A / op_B conjugation is applied (sum_unary_contractions,
 * product.c:1863-2020: only the DEFAULT, F32 and F64 branches conjugate). */
static int conj_applies(int prec)
{
    return prec == PR_DEFAULT || prec == PR_F32 || prec == PR_F64;
}

/* ------------------------------------------------------------------ */
/* reference-faithful loop (product.c:312-422)                          */
/* ------------------------------------------------------------------ */

int oracle_execute(int prec,
                   const oracle_tensor* A, const oracle_tensor* B,
                   const oracle_tensor* C, const oracle_tensor* D,
                   const void* alpha, const void* A_data, const void* B_data,
                   const void* beta, const void* C_data, void* D_data)
{
    int err = oracle_validate(A, B, C, D, beta, C_data != NULL);
    if (err) return err;
    if (prec != PR_DEFAULT && prec != PR_F32 && prec != PR_F64 && prec != PR_F16 &&
        prec != PR_F16_F32 && prec != PR_BF16_F32)
        return 0;  /* unknown precision: every switch of the reference falls through */

    layout* L = malloc(sizeof(layout));
    plan_layout(A, B, C, D, L);
    const int tA = A->type, tB = B->type, tC = C->type, tD = D->type;
    const vtype accT = acc_vt(prec, tD), sAT = prec_vt(prec, tA), sBT = prec_vt(prec, tB);
    const vtype cT = prec_vt(prec, tC), scT = prec_vt(prec, tD);
    const val alpha_p = vconv(load_elem(alpha, 0, tD), scT);   /* create_prec_scalar :1232 */
    const val beta_p = vconv(load_elem(beta, 0, tD), scT);
    const int beta_zero = scalar_is_zero(beta, tD);
    const int cj = conj_applies(prec);
    const int cplxD = is_cplx(tD);

    int64_t cf[OMAX] = {0}, cb[OMAX] = {0}, cua[OMAX] = {0}, cub[OMAX] = {0};
    const int64_t size_free = size_of(L->nfree, L->free_ext);
    const int64_t size_bin = size_of(L->nbin, L->bin_ext);
    const int64_t size_uA = size_of(L->nuA, L->uA_ext);
    const int64_t size_uB = size_of(L->nuB, L->uB_ext);

    for (int64_t i = 0; i < size_free; i++) {
        const int64_t oA = dot(L->nfree, cf, L->sfA), oB = dot(L->nfree, cf, L->sfB);
        const int64_t oC = dot(L->nfree, cf, L->sC), oD = dot(L->nfree, cf, L->sD);
        val acc;
        if (!beta_zero) {                                        /* :351-360 */
            val vc = vconv(load_elem(C_data, oC, tC), cT);       /* get_val :10830 */
            if (prec == PR_DEFAULT) {                            /* calculate_beta_C_default :2034 */
                if (is_cplx(tC) && C->op == 1) vc = vconj(vc);
                acc = vconv(vmul(beta_p, vc), accT);
            } else {                                             /* _prec :3156 ignores op_C */
                acc = vconv(vmul(beta_p, vc), accT);
            }
        } else {
            acc = vzero(accT);
        }
        for (int64_t j = 0; j < size_bin; j++) {                 /* :361-395 */
            const int64_t bA = oA + dot(L->nbin, cb, L->sbA), bB = oB + dot(L->nbin, cb, L->sbB);
            val sA = vzero(sAT);
            for (int64_t k = 0; k < size_uA; k++) {
                val e = load_elem(A_data, bA + dot(L->nuA, cua, L->suA), tA);
                if (cj && is_cplx(tA) && A->op == 1) e = vconj(e);
                sA = vconv(vadd(sA, e), sAT);
                incr(cua, L->nuA, L->uA_ext);
            }
            val sB = vzero(sBT);
            for (int64_t k = 0; k < size_uB; k++) {
                val e = load_elem(B_data, bB + dot(L->nuB, cub, L->suB), tB);
                if (cj && is_cplx(tB) && B->op == 1) e = vconj(e);
                sB = vconv(vadd(sB, e), sBT);
                incr(cub, L->nuB, L->uB_ext);
            }
            acc = vconv(vadd(acc, vmul(vmul(alpha_p, sA), sB)), accT);  /* calculate_alpha_A_B :3431 */
            incr(cb, L->nbin, L->bin_ext);
        }
        if (cplxD && D->op == 1) {                               /* calculate_op_D :10737 */
            if (prec == PR_F64) {
                vtype cf32 = {P_S, 1};                           /* conjf on complex double, :10814 */
                acc = vconv(vconj(vconv(acc, cf32)), accT);
            } else if (prec != PR_F16) {
                acc = vconj(acc);
            }
        }
        if (!(prec == PR_F16 && cplxD))                          /* assign_D :10989; no-op there */
            store_elem(D_data, oD, tD, acc);
        incr(cf, L->nfree, L->free_ext);
    }
    free(L);
    return 0;
}

/* ------------------------------------------------------------------ */
/* binary64 evaluation                                                  */
/* ------------------------------------------------------------------ */

typedef struct { double re, im; } c64;

static c64 cmul(c64 a, c64 b) { c64 r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static double cabs64(c64 a) { return hypot(a.re, a.im); }

static c64 to_c64(val v) { c64 r = {v.re, v.c ? v.im : 0.0}; return r; }

int64_t oracle_folded_size(const oracle_tensor* D)
{
    folded f;
    fold(D, &f);
    return size_of(f.n, f.ext);
}

int oracle_execute_f64(int prec,
                       const oracle_tensor* A, const oracle_tensor* B,
                       const oracle_tensor* C, const oracle_tensor* D,
                       const void* alpha, const void* A_data, const void* B_data,
                       const void* beta, const void* C_data,
                       int64_t n_samples, const int64_t* samples,
                       double* D64, double* scale, int64_t* D_offsets)
{
    int err = oracle_validate(A, B, C, D, beta, C_data != NULL);
    if (err) return err;
    layout* L = malloc(sizeof(layout));
    plan_layout(A, B, C, D, L);
    const int tA = A->type, tB = B->type, tC = C->type, tD = D->type;
    const vtype sAT = prec_vt(prec, tA), sBT = prec_vt(prec, tB), cT = prec_vt(prec, tC), scT = prec_vt(prec, tD);
    const c64 al = to_c64(vconv(load_elem(alpha, 0, tD), scT));
    const c64 be = to_c64(vconv(load_elem(beta, 0, tD), scT));
    const int beta_zero = scalar_is_zero(beta, tD);
    const int cj = conj_applies(prec);
    const int cplxD = is_cplx(tD);
    const int64_t size_free = size_of(L->nfree, L->free_ext);
    const int64_t size_bin = size_of(L->nbin, L->bin_ext);
    const int64_t size_uA = size_of(L->nuA, L->uA_ext);
    const int64_t size_uB = size_of(L->nuB, L->uB_ext);
    const int64_t count = n_samples < 0 ? size_free : n_samples;

    for (int64_t s = 0; s < count; s++) {
        int64_t cf[OMAX] = {0}, cb[OMAX] = {0}, cua[OMAX] = {0}, cub[OMAX] = {0};
        int64_t lin = n_samples < 0 ? s : samples[s];
        for (int j = 0; j < L->nfree; j++) { cf[j] = lin % L->free_ext[j]; lin /= L->free_ext[j]; }
        const int64_t oA = dot(L->nfree, cf, L->sfA), oB = dot(L->nfree, cf, L->sfB);
        const int64_t oC = dot(L->nfree, cf, L->sC), oD = dot(L->nfree, cf, L->sD);
        c64 acc = {0.0, 0.0};
        double sc = 0.0;
        if (!beta_zero) {
            val vc = vconv(load_elem(C_data, oC, tC), cT);
            if (prec == PR_DEFAULT && is_cplx(tC) && C->op == 1) vc = vconj(vc);
            acc = cmul(be, to_c64(vc));
            sc = cabs64(be) * cabs64(to_c64(vc));
        }
        c64 sum = {0.0, 0.0};
        double ssum = 0.0;
        for (int64_t j = 0; j < size_bin; j++) {
            const int64_t bA = oA + dot(L->nbin, cb, L->sbA), bB = oB + dot(L->nbin, cb, L->sbB);
            c64 sa = {0.0, 0.0}, sb = {0.0, 0.0};
            double aa = 0.0, ab = 0.0;
            for (int64_t k = 0; k < size_uA; k++) {
                val e = vconv(load_elem(A_data, bA + dot(L->nuA, cua, L->suA), tA), sAT);
                if (cj && is_cplx(tA) && A->op == 1) e = vconj(e);
                c64 x = to_c64(e);
                sa.re += x.re; sa.im += x.im; aa += cabs64(x);
                incr(cua, L->nuA, L->uA_ext);
            }
            for (int64_t k = 0; k < size_uB; k++) {
                val e = vconv(load_elem(B_data, bB + dot(L->nuB, cub, L->suB), tB), sBT);
                if (cj && is_cplx(tB) && B->op == 1) e = vconj(e);
                c64 x = to_c64(e);
                sb.re += x.re; sb.im += x.im; ab += cabs64(x);
                incr(cub, L->nuB, L->uB_ext);
            }
            c64 p = cmul(sa, sb);
            sum.re += p.re; sum.im += p.im;
            ssum += aa * ab;
            incr(cb, L->nbin, L->bin_ext);
        }
        c64 t = cmul(al, sum);
        acc.re += t.re; acc.im += t.im;
        sc += cabs64(al) * ssum;
        if (!cplxD) acc.im = 0.0;
        if (cplxD && D->op == 1) {
            if (prec == PR_F64) {              /* conjf on complex double rounds to binary32, product.c:10814 */
                acc.re = (double)(float)acc.re;
                acc.im = -(double)(float)acc.im;
            } else if (prec != PR_F16) {
                acc.im = -acc.im;
            }
        }
        const int untouched = (prec == PR_F16 && cplxD);
        if (n_samples < 0) {
            if (!untouched) { D64[2 * oD] = acc.re; D64[2 * oD + 1] = acc.im; }
            scale[oD] = untouched ? 0.0 : sc;
        } else {
            D64[2 * s] = untouched ? NAN : acc.re;
            D64[2 * s + 1] = untouched ? NAN : acc.im;
            scale[s] = sc;
            if (D_offsets) D_offsets[s] = oD;
        }
    }
    free(L);
    return 0;
}

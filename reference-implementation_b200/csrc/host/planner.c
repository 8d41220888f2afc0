/*
 * Host planner: turns a validated TAPP product into a launch plan.
 *
 * The index analysis is the reference's (reference_implementation/src/
 * product.c:265-310 with helpers :538-735, :969-1010), done once on the host
 * instead of per element:
 *   - repeated labels in one tensor merge into one mode whose stride is the
 *     sum of the repeats' strides (compress_repeated_indices :969-1010);
 *   - D's modes are the free modes; their stride in A or B is 0 where that
 *     operand lacks the label (extract_free_strides :621-641);
 *   - labels in A and B but not D are contracted (:538-570), taking their
 *     extents from A;
 *   - labels only in A (only in B) are unary and are summed before the
 *     multiplication (:588-619, sum_unary_contractions :1863).
 * Beyond the reference: extent-1 modes are dropped, modes are ordered by
 * stride, neighbours that are contiguous in every tensor are merged, and the
 * free modes are split into the batch/M/N view the GEMM kernels use.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tb_internal.h"

int tb_elem_bytes(TAPP_datatype t)
{
    switch (t) {
    case TAPP_F32: return 4;
    case TAPP_F64: return 8;
    case TAPP_C32: return 8;
    case TAPP_C64: return 16;
    case TAPP_F16: case TAPP_BF16: return 2;
    default: return 0;
    }
}

int tb_is_complex(TAPP_datatype t) { return t == TAPP_C32 || t == TAPP_C64; }
static int is_wide(TAPP_datatype t) { return t == TAPP_F64 || t == TAPP_C64; }

#define FOLD_MAX 256
typedef struct { int n; int64_t idx[FOLD_MAX], ext[FOLD_MAX], str[FOLD_MAX]; } folded;

/* compress_repeated_indices, product.c:969-1010 */
static int fold(const tb_tensor_view* t, folded* f)
{
    f->n = 0;
    for (int i = 0; i < t->nmode; i++) {
        int k = -1;
        for (int j = 0; j < f->n; j++)
            if (f->idx[j] == t->idx[i]) { k = j; break; }
        if (k < 0) {
            if (f->n >= FOLD_MAX) return TAPP_B200_ERR_LIMIT;
            k = f->n++;
            f->idx[k] = t->idx[i];
            f->ext[k] = t->extents[i];
            f->str[k] = 0;
        }
        f->str[k] += t->strides[i];
    }
    return 0;
}

static int find(const folded* f, int64_t label)
{
    for (int i = 0; i < f->n; i++)
        if (f->idx[i] == label) return i;
    return -1;
}

/* a working list of modes before compaction into tb_modes */
typedef struct { int n; int64_t ext[FOLD_MAX], s[4][FOLD_MAX]; } mlist;

static void ml_push(mlist* m, int64_t e, int64_t a, int64_t b, int64_t c, int64_t d)
{
    int k = m->n++;
    m->ext[k] = e;
    m->s[0][k] = a; m->s[1][k] = b; m->s[2][k] = c; m->s[3][k] = d;
}

static int64_t iabs64(int64_t x) { return x < 0 ? -x : x; }

/* Drops extent-1 modes, sorts by |stride of tensor `key`| (stable), and
 * merges neighbours j, j+1 with s[j+1] == s[j] * ext[j] in every tensor. */
static void simplify(mlist* m, int key)
{
    int w = 0;
    for (int i = 0; i < m->n; i++) {
        if (m->ext[i] == 1) continue;
        m->ext[w] = m->ext[i];
        for (int t = 0; t < 4; t++) m->s[t][w] = m->s[t][i];
        w++;
    }
    m->n = w;
    for (int i = 1; i < m->n; i++) {
        int64_t e = m->ext[i], s[4];
        for (int t = 0; t < 4; t++) s[t] = m->s[t][i];
        int j = i - 1;
        while (j >= 0 && iabs64(m->s[key][j]) > iabs64(s[key])) {
            m->ext[j + 1] = m->ext[j];
            for (int t = 0; t < 4; t++) m->s[t][j + 1] = m->s[t][j];
            j--;
        }
        m->ext[j + 1] = e;
        for (int t = 0; t < 4; t++) m->s[t][j + 1] = s[t];
    }
    w = 0;
    for (int i = 0; i < m->n; i++) {
        if (w > 0) {
            int ok = 1;
            for (int t = 0; t < 4; t++)
                if (m->s[t][i] != m->s[t][w - 1] * m->ext[w - 1]) ok = 0;
            if (ok) { m->ext[w - 1] *= m->ext[i]; continue; }
        }
        m->ext[w] = m->ext[i];
        for (int t = 0; t < 4; t++) m->s[t][w] = m->s[t][i];
        w++;
    }
    m->n = w;
}

static void reorder_by(tb_modes* F, const int64_t* s);

/* Element path: one thread per output, consecutive threads on consecutive
 * outputs in F order (D's stride order). When the larger operand holds more
 * than twice as many elements as D and is contiguous along an output mode
 * (stride +-1), F is put in that operand's stride order instead (modes it
 * lacks last, stable), so that a warp reads it in whole lines rather than
 * one line per lane. Every output is computed the same way in either order. */
static void order_outputs(tb_plan* P)
{
    tb_modes* F = &P->F;
    double nA = (double)P->K.size * (double)P->UA.size, nB = (double)P->K.size * (double)P->UB.size;
    for (int i = 0; i < F->n; i++) {
        if (F->sA[i]) nA *= (double)F->ext[i];
        if (F->sB[i]) nB *= (double)F->ext[i];
    }
    const int useA = nA >= nB;
    const int64_t* s = useA ? F->sA : F->sB;
    if ((useA ? nA : nB) <= 2.0 * (double)F->size) return;
    int unit = 0;
    for (int i = 0; i < F->n; i++)
        if (s[i] == 1 || s[i] == -1) unit = 1;
    if (!unit) return;
    reorder_by(F, s);
    /* The other operand, when consecutive outputs would read it far apart
     * (one line per lane) and it is at most half the size of the walked one
     * and at least 64 Ki elements: copied once into the walk's order before
     * the element kernel runs (its values, and so every output, unchanged). */
    const int64_t* o = useA ? F->sB : F->sA;
    const double nO = useA ? nB : nA;
    if (F->n >= 1 && o[0] != 0 && o[0] != 1 && o[0] != -1 && nO * 2.0 <= (useA ? nA : nB) && nO >= 65536.0 &&
        nO < 2147483648.0)
        P->elem_stage = useA ? 2 : 1;
}

/* stable sort of F's modes by |s| (modes with s = 0 last) */
static void reorder_by(tb_modes* F, const int64_t* s)
{
    int64_t key[TB_MAXMODES];
    for (int i = 0; i < F->n; i++) key[i] = s[i] ? iabs64(s[i]) : INT64_MAX;
    for (int i = 1; i < F->n; i++) {
        const int64_t k = key[i], e = F->ext[i], a = F->sA[i], b = F->sB[i], c = F->sC[i], d = F->sD[i];
        int j = i - 1;
        while (j >= 0 && key[j] > k) {
            key[j + 1] = key[j];
            F->ext[j + 1] = F->ext[j];
            F->sA[j + 1] = F->sA[j];
            F->sB[j + 1] = F->sB[j];
            F->sC[j + 1] = F->sC[j];
            F->sD[j + 1] = F->sD[j];
            j--;
        }
        key[j + 1] = k;
        F->ext[j + 1] = e;
        F->sA[j + 1] = a;
        F->sB[j + 1] = b;
        F->sC[j + 1] = c;
        F->sD[j + 1] = d;
    }
}

static int to_modes(const mlist* m, tb_modes* out)
{
    memset(out, 0, sizeof(*out));
    if (m->n > TB_MAXMODES) return TAPP_B200_ERR_LIMIT;
    out->n = m->n;
    out->size = 1;
    for (int i = 0; i < m->n; i++) {
        out->ext[i] = m->ext[i];
        out->sA[i] = m->s[0][i];
        out->sB[i] = m->s[1][i];
        out->sC[i] = m->s[2][i];
        out->sD[i] = m->s[3][i];
        out->size *= m->ext[i];
    }
    return 0;
}

static double read_re(const void* s, TAPP_datatype t);
static double read_im(const void* s, TAPP_datatype t);

/* Round to a binary format with p significand bits and minimum normal
 * exponent emin, nearest-even, overflow to infinity. */
static double round_fmt(double x, int p, int emin, double maxv)
{
    if (x == 0.0 || !isfinite(x)) return x;
    int e;
    (void)frexp(x, &e);
    int q = e - p;
    if (q < emin + 1 - p) q = emin + 1 - p;
    double y = ldexp(nearbyint(ldexp(x, -q)), q);
    return fabs(y) > maxv ? copysign(INFINITY, x) : y;
}

static double round_to(int mode, double x)
{
    switch (mode) {
    case TB_ROUND_F32: return (double)(float)x;
    case TB_ROUND_F16: return round_fmt(x, 11, -14, 65504.0);
    case TB_ROUND_BF16: return round_fmt(x, 8, -126, 3.3895313892515355e38);
    default: return x;
    }
}

static double f16_val(uint16_t h)
{
    int s = h >> 15, e = (h >> 10) & 0x1f, m = h & 0x3ff;
    double v = e == 0 ? ldexp((double)m, -24) : e == 31 ? (m ? NAN : INFINITY) : ldexp((double)(m | 0x400), e - 25);
    return s ? -v : v;
}

static double bf16_val(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static double read_re(const void* s, TAPP_datatype t)
{
    switch (t) {
    case TAPP_F32: case TAPP_C32: return ((const float*)s)[0];
    case TAPP_F64: case TAPP_C64: return ((const double*)s)[0];
    case TAPP_F16: return f16_val(*(const uint16_t*)s);
    case TAPP_BF16: return bf16_val(*(const uint16_t*)s);
    default: return 0.0;
    }
}

static double read_im(const void* s, TAPP_datatype t)
{
    switch (t) {
    case TAPP_C32: return ((const float*)s)[1];
    case TAPP_C64: return ((const double*)s)[1];
    default: return 0.0;
    }
}

/* Whether op_A / op_B conjugation is applied: only the DEFAULT, F32 and F64
 * branches of sum_unary_contractions conjugate (product.c:1863-2020). */
static int conj_operands(TAPP_prectype prec)
{
    return prec == TAPP_DEFAULT_PREC || prec == TAPP_F32F32_ACCUM_F32 || prec == TAPP_F64F64_ACCUM_F64;
}

static int known_prec(TAPP_prectype p)
{
    return p == TAPP_DEFAULT_PREC || p == TAPP_F32F32_ACCUM_F32 || p == TAPP_F64F64_ACCUM_F64 ||
           p == TAPP_F16F16_ACCUM_F16 || p == TAPP_F16F16_ACCUM_F32 || p == TAPP_BF16BF16_ACCUM_F32;
}

/* alpha and beta as scalars of the precision's type (create_prec_scalar,
 * product.c:1232). Returns 1 when beta's zero-ness differs from the plan's
 * (the plan must then be rebuilt: C's strides entered the mode merging). */
int tb_plan_set_scalars(tb_plan* P, const void* alpha, const void* beta)
{
    const int bz = tb_scalar_is_zero(beta, P->tD);
    P->alpha_re = round_to(P->round_scalars, read_re(alpha, P->tD));
    P->alpha_im = round_to(P->round_scalars, read_im(alpha, P->tD));
    P->beta_re = bz ? 0.0 : round_to(P->round_scalars, read_re(beta, P->tD));
    P->beta_im = bz ? 0.0 : round_to(P->round_scalars, read_im(beta, P->tD));
    return bz != P->beta_zero;
}

/* A-priori bound on the error of the plan's arithmetic (see tapp_b200.h,
 * TAPP_B200_STATUS_ERR_BOUND): n terms summed in a format with unit
 * roundoff u err by at most gamma_n = n u / (1 - n u) times the sum of their
 * magnitudes (Higham, Accuracy and Stability of Numerical Algorithms, 3.1). */
double tb_plan_error_bound(const tb_plan* p)
{
    const int cplx = p->compute == TB_C32 || p->compute == TB_C64;
    const double K = (double)p->K.size, UA = (double)p->UA.size, UB = (double)p->UB.size;
    if (p->path == TB_PATH_SLICED) {
        const double kreal = K * (cplx ? 2.0 : 1.0);
        return kreal * (p->slices + 4) * ldexp(1.0, -7 * p->slices);
    }
    const double u = (p->compute == TB_R64 || p->compute == TB_C64) ? ldexp(1.0, -53) : ldexp(1.0, -24);
    const double n = K * (UA > 1 ? UA : 1) + UA + UB + 8;
    double g = n * u / (1.0 - n * u);
    if (p->path == TB_PATH_TC && p->tc_mode == TB_TC_SPLIT_BF16) g += ldexp(1.0, -16);
    if (p->round_in == TB_ROUND_BF16 || p->round_in == TB_ROUND_F16) {
        /* the 16-bit precisions keep running unary sums in 16 bits */
        const double u16 = p->round_in == TB_ROUND_BF16 ? ldexp(1.0, -8) : ldexp(1.0, -11);
        if (UA > 1 || UB > 1) g += (UA + UB) * u16;
    }
    return g;
}

double tb_plan_flops(const tb_plan* p)
{
    double f = (double)p->F.size * (double)p->K.size;
    return (p->compute == TB_C32 || p->compute == TB_C64) ? 8.0 * f : 2.0 * f;
}

int tb_build_plan(const tb_tensor_view* A, const tb_tensor_view* B,
                  const tb_tensor_view* C, const tb_tensor_view* D,
                  TAPP_prectype prec, const void* alpha, const void* beta,
                  const tb_plan_options* opt, tb_plan* P)
{
    memset(P, 0, sizeof(*P));
    P->tA = A->type; P->tB = B->type; P->tC = C->type; P->tD = D->type;
    P->prec = prec;
    for (int k = 0; k < 4; k++) {
        const tb_tensor_view* t = k == 0 ? A : k == 1 ? B : k == 2 ? C : D;
        if (tb_elem_bytes(t->type) == 0) return TAPP_B200_ERR_UNSUPPORTED;
    }
    P->beta_zero = tb_scalar_is_zero(beta, D->type);

    static __thread folded fA, fB, fC, fD;
    int err = fold(A, &fA);
    if (!err) err = fold(B, &fB);
    if (!err) err = fold(C, &fC);
    if (!err) err = fold(D, &fD);
    if (err) return err;

    static __thread mlist F, K, UA, UB;
    F.n = K.n = UA.n = UB.n = 0;
    int empty_D = 0, empty_sum = 0;
    for (int j = 0; j < fD.n; j++) {
        int a = find(&fA, fD.idx[j]), b = find(&fB, fD.idx[j]);
        int64_t sC = j < fC.n ? fC.str[j] : 0;
        if (P->beta_zero) sC = fD.str[j];   /* C unread: let it follow D */
        if (fD.ext[j] == 0) empty_D = 1;
        ml_push(&F, fD.ext[j], a >= 0 ? fA.str[a] : 0, b >= 0 ? fB.str[b] : 0, sC, fD.str[j]);
    }
    for (int i = 0; i < fA.n; i++) {
        int b = find(&fB, fA.idx[i]), d = find(&fD, fA.idx[i]);
        if (d >= 0) continue;
        if (fA.ext[i] == 0) empty_sum = 1;
        if (b >= 0) ml_push(&K, fA.ext[i], fA.str[i], fB.str[b], 0, 0);
        else ml_push(&UA, fA.ext[i], fA.str[i], 0, 0, 0);
    }
    for (int i = 0; i < fB.n; i++) {
        if (find(&fA, fB.idx[i]) >= 0 || find(&fD, fB.idx[i]) >= 0) continue;
        if (fB.ext[i] == 0) empty_sum = 1;
        ml_push(&UB, fB.ext[i], 0, fB.str[i], 0, 0);
    }

    /* precision and compute domain (alloc_accum :1012, alloc_val :1104) */
    const int read_C = !P->beta_zero;
    int cplx = tb_is_complex(A->type) || tb_is_complex(B->type) || tb_is_complex(D->type) ||
               (read_C && tb_is_complex(C->type));
    int wide;
    switch (prec) {
    case TAPP_F64F64_ACCUM_F64: wide = 1; break;
    case TAPP_DEFAULT_PREC:
        wide = is_wide(A->type) || is_wide(B->type) || is_wide(D->type) || (read_C && is_wide(C->type));
        break;
    default: wide = 0; break;
    }
    P->compute = cplx ? (wide ? TB_C64 : TB_C32) : (wide ? TB_R64 : TB_R32);
    P->round_in = prec == TAPP_F16F16_ACCUM_F16 || prec == TAPP_F16F16_ACCUM_F32 ? TB_ROUND_F16
                  : prec == TAPP_BF16BF16_ACCUM_F32 ? TB_ROUND_BF16 : TB_ROUND_NONE;
    /* alpha/beta become scalars of the precision's type (create_prec_scalar :1232) */
    P->round_scalars = P->round_in != TB_ROUND_NONE ? P->round_in
                       : (prec == TAPP_F32F32_ACCUM_F32 ? TB_ROUND_F32 : TB_ROUND_NONE);
    tb_plan_set_scalars(P, alpha, beta);
    P->conjA = A->op == TAPP_CONJUGATE && tb_is_complex(A->type) && conj_operands(prec);
    P->conjB = B->op == TAPP_CONJUGATE && tb_is_complex(B->type) && conj_operands(prec);
    /* op_C is applied only by the DEFAULT branch (calculate_beta_C_prec :3156 has no op) */
    P->conjC = C->op == TAPP_CONJUGATE && tb_is_complex(C->type) && prec == TAPP_DEFAULT_PREC;
    /* calculate_op_D :10737: no conjugation under F16F16_ACCUM_F16; under
     * F64F64_ACCUM_F64 it goes through conjf and rounds to binary32 (:10814) */
    P->conjD = D->op == TAPP_CONJUGATE && tb_is_complex(D->type) && prec != TAPP_F16F16_ACCUM_F16;
    P->conjD_round_f32 = P->conjD && prec == TAPP_F64F64_ACCUM_F64;
    /* assign_D :10989: complex D is not written under F16F16_ACCUM_F16 */
    P->skip_store = prec == TAPP_F16F16_ACCUM_F16 && tb_is_complex(D->type);

    simplify(&F, 3);
    /* Contracted modes are ordered by the strides of the operand that is
     * contiguous along a contracted mode (K-major), so that the operand
     * packing reads it along its fastest mode; an operand contiguous along a
     * free mode is read along that mode whatever the contracted order. */
    int64_t minKA = INT64_MAX, minKB = INT64_MAX, minFA = INT64_MAX;
    for (int i = 0; i < K.n; i++) {
        if (K.ext[i] == 1) continue;
        if (K.s[0][i] && iabs64(K.s[0][i]) < minKA) minKA = iabs64(K.s[0][i]);
        if (K.s[1][i] && iabs64(K.s[1][i]) < minKB) minKB = iabs64(K.s[1][i]);
    }
    for (int i = 0; i < F.n; i++)
        if (F.s[0][i] && F.s[1][i] == 0 && iabs64(F.s[0][i]) < minFA) minFA = iabs64(F.s[0][i]);
    const int A_kmajor = minKA < minFA;
    simplify(&K, (!A_kmajor && minKB != INT64_MAX) ? 1 : 0);
    simplify(&UA, 0);
    simplify(&UB, 1);
    if ((err = to_modes(&F, &P->F)) || (err = to_modes(&K, &P->K)) ||
        (err = to_modes(&UA, &P->UA)) || (err = to_modes(&UB, &P->UB)))
        return err;
    if (empty_sum) { P->K.n = 0; P->K.size = 0; }

    /* GEMM view: batch modes use both operands, M only A, N only B */
    mlist Lm, Mm, Nm;
    Lm.n = Mm.n = Nm.n = 0;
    for (int i = 0; i < P->F.n; i++) {
        mlist* dst = P->F.sB[i] == 0 ? &Mm : (P->F.sA[i] == 0 ? &Nm : &Lm);
        ml_push(dst, P->F.ext[i], P->F.sA[i], P->F.sB[i], P->F.sC[i], P->F.sD[i]);
    }
    simplify(&Mm, 0);
    simplify(&Nm, 1);
    simplify(&Lm, 3);
    if ((err = to_modes(&Lm, &P->L)) || (err = to_modes(&Mm, &P->M)) || (err = to_modes(&Nm, &P->N)))
        return err;

    /* path */
    if (!known_prec(prec) || empty_D || P->skip_store) {
        P->path = TB_PATH_NOOP;   /* every branch of the reference falls through: D untouched */
        return 0;
    }
    const int64_t outs = P->F.size, ksz = P->K.size;
    const double macs = (double)outs * (double)(ksz > 0 ? ksz : 1) * (double)P->UA.size * (double)P->UB.size;
    int path = TB_PATH_GENERIC;
    /* few outputs and a long contraction: one block per output instead of
     * one thread; also wherever one thread per output would make about one
     * wave of threads or less (under 148 x 1024 outputs) and each would loop
     * over >= 1024 terms */
    if ((outs < 4096 && ksz >= 512 && outs * 16 < ksz) || (outs < 148 * 1024 && ksz >= 1024))
        path = TB_PATH_REDUCE;

    int tc_ok = 0;
    if ((P->compute == TB_R32 || P->compute == TB_C32) && ksz > 0) {
        if (prec == TAPP_BF16BF16_ACCUM_F32) { tc_ok = 1; P->tc_mode = TB_TC_BF16; }
        else if (prec == TAPP_F16F16_ACCUM_F32 || prec == TAPP_F16F16_ACCUM_F16) { tc_ok = 1; P->tc_mode = TB_TC_F16; }
        else if (opt && opt->f32_mode >= 1 && opt->f32_mode <= 3) {
            tc_ok = 1;
            P->tc_mode = TB_TC_SPLIT_BF16;
            P->split_route = opt->f32_mode;
        }
    }
    /* launch limits of the pack grid (z = batch, y = contraction tiles) and the tile count */
    const int64_t kcols = ksz * (P->compute == TB_C32 ? 2 : 1);
    if (P->L.size > 65535 || (kcols + 31) / 32 > 65535 ||
        (double)((P->M.size + 127) / 128) * (double)((P->N.size * 2 + 255) / 256) * (double)P->L.size > 1e9 ||
        P->UA.n > TB_MAXMODES || P->UB.n > TB_MAXMODES)
        tc_ok = 0;
    const int big = P->M.size >= 64 && P->N.size >= 64 && ksz >= 64 && macs >= 16.0 * 1024 * 1024;
    /* tiled CUDA-core GEMM: products without unary modes */
    const int simt_ok = P->UA.n == 0 && P->UB.n == 0 && ksz > 0 && P->UA.size == 1 && P->UB.size == 1;
    /* the GEMM is turned so that its rows are the longer side; a long side of
     * 16 fills its narrowest tile, a short side of 1 (matrix-vector) is fine */
    const int64_t long_side = P->M.size > P->N.size ? P->M.size : P->N.size;
    const int64_t short_side = P->M.size > P->N.size ? P->N.size : P->M.size;
    /* many small batches of matrix-vector products fill tiles poorly: those
     * stay on the element kernel */
    const int simt_big = long_side >= 16 && ksz >= 8 && macs >= 1024.0 * 1024 &&
                         (short_side >= 4 || P->L.size == 1);
    if (simt_ok && simt_big) path = TB_PATH_SIMT;
    if (tc_ok && big) path = TB_PATH_TC;
    /* sliced binary64: digit panels must fit the slicing grid (batch in
     * grid.z, 64-byte column tiles in grid.y) */
    const int64_t kreal = ksz * (P->compute == TB_C64 ? 2 : 1);
    const int sliced_ok = (P->compute == TB_R64 || P->compute == TB_C64) && opt && opt->f64_mode >= 2 &&
                          opt->f64_mode <= 16 && simt_ok && P->L.size <= 65535 && (kreal + 15) / 16 * 16 / 64 < 65535 &&
                          (double)((P->M.size + 255) / 256) * (double)((P->N.size * 2 + 255) / 256) * (double)P->L.size < 1e9;
    if (sliced_ok) P->slices = opt->f64_mode;
    if (sliced_ok && big) {
        path = TB_PATH_SLICED;
        P->tc_mode = TB_TC_SLICED_I8;
    }
    if (opt && opt->force_path) {
        int f = opt->force_path;
        if (f == TB_PATH_TC && tc_ok) path = TB_PATH_TC;
        else if (f == TB_PATH_SIMT && simt_ok) path = TB_PATH_SIMT;
        else if (f == TB_PATH_SLICED && sliced_ok) {
            path = TB_PATH_SLICED;
            P->tc_mode = TB_TC_SLICED_I8;
        }
        else if (f == TB_PATH_GENERIC || f == TB_PATH_REDUCE) path = f;
    }
    P->path = path;
    if (path == TB_PATH_GENERIC) order_outputs(P);
    return 0;
}

static size_t put(char* out, size_t maxlen, size_t at, const char* fmt, ...)
    __attribute__((format(printf, 4, 5)));

#include <stdarg.h>
static size_t put(char* out, size_t maxlen, size_t at, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    char tmp[512];
    int n = vsnprintf(tmp, sizeof tmp, fmt, ap);
    va_end(ap);
    if (n < 0) return at;
    for (int i = 0; i < n; i++, at++)
        if (out && at + 1 < maxlen) out[at] = tmp[i];
    return at;
}

static size_t put_modes(char* out, size_t maxlen, size_t at, const char* name, const tb_modes* m)
{
    at = put(out, maxlen, at, " %s=[", name);
    for (int i = 0; i < m->n; i++)
        at = put(out, maxlen, at, "%s(%lld:%lld,%lld,%lld,%lld)", i ? "," : "", (long long)m->ext[i],
                 (long long)m->sA[i], (long long)m->sB[i], (long long)m->sC[i], (long long)m->sD[i]);
    return put(out, maxlen, at, "]");
}

/* Text form of a plan; modes print as (extent:strideA,strideB,strideC,strideD). */
size_t tb_describe(const tb_plan* p, size_t maxlen, char* out)
{
    static const char* paths[] = {"noop", "generic", "reduce", "simt", "tc", "sliced"};
    static const char* comp[] = {"r32", "r64", "c32", "c64"};
    static const char* tcm[] = {"bf16", "f16", "split_bf16", "sliced_i8"};
    size_t at = 0;
    at = put(out, maxlen, at, "path=%s compute=%s prec=%d round_in=%d conj=%d%d%d%d beta_zero=%d",
             paths[p->path], comp[p->compute], p->prec, p->round_in, p->conjA, p->conjB, p->conjC, p->conjD,
             p->beta_zero);
    if (p->path == TB_PATH_TC) at = put(out, maxlen, at, " tc_mode=%s", tcm[p->tc_mode]);
    if (p->path == TB_PATH_TC && p->tc_mode == TB_TC_SPLIT_BF16)
        at = put(out, maxlen, at, " operands=%s", tbk_tc_split_in_place(p) ? "in_place" : "packed");
    if (p->path == TB_PATH_SLICED) at = put(out, maxlen, at, " slices=%d", p->slices);
    if (p->path == TB_PATH_GENERIC) {
        const int warp = tbk_generic_kernel(p);
        at = put(out, maxlen, at, " kernel=%s", warp ? "warpdot" : "element");
        if (!warp && p->elem_stage) at = put(out, maxlen, at, " staged=%s", p->elem_stage == 1 ? "A" : "B");
    }
    if (p->path == TB_PATH_SIMT) {
        static const char* kern[] = {"tiled", "narrow", "narrow_stream", "narrow_coop", "narrow_cstream", "narrow_vec",
                                     "narrow_cvec", "narrow_kt"};
        const int k = tbk_simt_kernel(p);
        if (k >= 0 && k <= 7) at = put(out, maxlen, at, " kernel=%s", kern[k]);
    }
    at = put_modes(out, maxlen, at, "F", &p->F);
    at = put_modes(out, maxlen, at, "K", &p->K);
    at = put_modes(out, maxlen, at, "UA", &p->UA);
    at = put_modes(out, maxlen, at, "UB", &p->UB);
    at = put_modes(out, maxlen, at, "L", &p->L);
    at = put_modes(out, maxlen, at, "M", &p->M);
    at = put_modes(out, maxlen, at, "N", &p->N);
    if (out && maxlen) out[at < maxlen ? at : maxlen - 1] = '\0';
    return at;
}

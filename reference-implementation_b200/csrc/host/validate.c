/*
 * The reference's validation chain, in its order and with its codes
 * (reference_implementation/src/product.c:199-206; helpers :757-885).
 * The first failing check wins:
 *   4  a label of D is in neither A nor B            (check_idx_occurrence :757)
 *   9 / 1 / 2   A's labels against A, B, D extents   (check_extents :786)
 *   10 / 1 / 3  B's labels against B, A, D
 *   11 / 2 / 3  D's labels against D, A, B
 *   5 / 6 / 7   C against D: mode count, then per position label, extent
 *                                                    (check_same_structure :815)
 *   8  D aliases itself                               (check_self_aliasing :836)
 *   12 C is NULL while beta != 0                      (check_tensor_existence :872)
 * The executor check (33) is done by the caller.
 */
#include <stdlib.h>

#include "tb_internal.h"

static int occurrence(const tb_tensor_view* D, const tb_tensor_view* A, const tb_tensor_view* B)
{
    for (int i = 0; i < D->nmode; i++) {
        int found = 0;
        for (int j = 0; j < A->nmode && !found; j++) found = D->idx[i] == A->idx[j];
        for (int j = 0; j < B->nmode && !found; j++) found = D->idx[i] == B->idx[j];
        if (!found) return 4;
    }
    return 0;
}

static int extents(const tb_tensor_view* X, const tb_tensor_view* Y, const tb_tensor_view* Z,
                   int c_xx, int c_xy, int c_xz)
{
    for (int i = 0; i < X->nmode; i++) {
        for (int j = 0; j < X->nmode; j++)
            if (X->idx[i] == X->idx[j] && X->extents[i] != X->extents[j]) return c_xx;
        for (int j = 0; j < Y->nmode; j++)
            if (X->idx[i] == Y->idx[j] && X->extents[i] != Y->extents[j]) return c_xy;
        for (int j = 0; j < Z->nmode; j++)
            if (X->idx[i] == Z->idx[j] && X->extents[i] != Z->extents[j]) return c_xz;
    }
    return 0;
}

static int structure(const tb_tensor_view* C, const tb_tensor_view* D)
{
    if (C->nmode != D->nmode) return 5;
    for (int i = 0; i < D->nmode; i++) {
        if (D->idx[i] != C->idx[i]) return 6;
        if (D->extents[i] != C->extents[i]) return 7;
    }
    return 0;
}

/* Modes sorted by |stride| (ties: smaller extent first, the order the
 * reference's merge sort produces); each stride must reach past the span of
 * the previous mode. A zero stride aliases when there are two or more modes.
 * The reference sorts through int temporaries (:923-926); this keeps 64 bits.
 * No sorted copy is made: for every mode, its successor in that order (the
 * smallest (|stride|, extent, position) above its own) is found by a scan,
 * which compares the same neighbouring pairs as a sort would, in O(n^2) time
 * and no memory (the allocation-free entry point validates through here). */
static int aliasing(const tb_tensor_view* D)
{
    int n = D->nmode;
    if (n <= 1) return 0;
    for (int i = 0; i < n; i++)
        if (D->strides[i] == 0) return 8;
    for (int i = 0; i < n; i++) {
        const int64_t vi = D->strides[i] < 0 ? -D->strides[i] : D->strides[i], xi = D->extents[i];
        int next = -1;
        int64_t vn = 0, xn = 0;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            const int64_t vj = D->strides[j] < 0 ? -D->strides[j] : D->strides[j], xj = D->extents[j];
            const int above = vj > vi || (vj == vi && (xj > xi || (xj == xi && j > i)));
            if (!above) continue;
            if (next < 0 || vj < vn || (vj == vn && (xj < xn || (xj == xn && j < next)))) {
                next = j;
                vn = vj;
                xn = xj;
            }
        }
        if (next >= 0 && vn < vi * xi) return 8;
    }
    return 0;
}

int tb_scalar_is_zero(const void* s, TAPP_datatype t)
{
    if (!s) return 1;
    switch (t) {
    case TAPP_F32: return *(const float*)s == 0.0f;
    case TAPP_F64: return *(const double*)s == 0.0;
    case TAPP_C32: return ((const float*)s)[0] == 0.0f && ((const float*)s)[1] == 0.0f;
    case TAPP_C64: return ((const double*)s)[0] == 0.0 && ((const double*)s)[1] == 0.0;
    case TAPP_F16:
    case TAPP_BF16: return (*(const uint16_t*)s & 0x7fff) == 0;
    default: return 0;
    }
}

int tb_validate(const tb_tensor_view* A, const tb_tensor_view* B,
                const tb_tensor_view* C, const tb_tensor_view* D,
                const void* beta, int C_present)
{
    int e = occurrence(D, A, B);
    if (!e) e = extents(A, B, D, 9, 1, 2);
    if (!e) e = extents(B, A, D, 10, 1, 3);
    if (!e) e = extents(D, A, B, 11, 2, 3);
    if (!e) e = structure(C, D);
    if (!e) e = aliasing(D);
    if (!e && !C_present && !tb_scalar_is_zero(beta, D->type)) e = 12;
    return e;
}

/*
 * Tensor infos: TAPP_create_tensor_info and its getters and setters.
 * Behaviour follows reference_implementation/src/tensor.c:11-101: the info
 * owns copies of extents and strides; a negative mode count returns 14 and a
 * negative extent 15, both before anything is allocated.
 */
#include <stdlib.h>
#include <string.h>

#include "tb_internal.h"

static int64_t* dup_i64(const int64_t* src, int n)
{
    int64_t* p = malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (p && n > 0 && src) memcpy(p, src, sizeof(int64_t) * (size_t)n);
    return p;
}

/* tensor.c:11-39 */
TAPP_error TAPP_create_tensor_info(TAPP_tensor_info* info, TAPP_datatype type, int nmode,
                                   const int64_t* extents, const int64_t* strides)
{
    if (nmode < 0) return 14;
    for (int i = 0; i < nmode; i++)
        if (extents[i] < 0) return 15;
    struct tb_info* t = malloc(sizeof(*t));
    if (!t) return TAPP_B200_ERR_NOMEM;
    t->magic = TB_MAGIC_INFO;
    t->type = type;
    t->nmode = nmode;
    t->extents = dup_i64(extents, nmode);
    t->strides = dup_i64(strides, nmode);
    *info = (TAPP_tensor_info)t;
    return 0;
}

/* tensor.c:41-48 */
TAPP_error TAPP_destroy_tensor_info(TAPP_tensor_info info)
{
    struct tb_info* t = (struct tb_info*)info;
    if (!t) return 0;
    t->magic = 0;
    free(t->extents);
    free(t->strides);
    free(t);
    return 0;
}

/* tensor.c:50-53 */
int TAPP_get_nmodes(TAPP_tensor_info info)
{
    return ((struct tb_info*)info)->nmode;
}

/* tensor.c:55-66: resizes both arrays; new entries are unspecified until set
 * (zero here). */
TAPP_error TAPP_set_nmodes(TAPP_tensor_info info, int nmodes)
{
    if (nmodes < 0) return 14;
    struct tb_info* t = (struct tb_info*)info;
    int64_t* e = realloc(t->extents, sizeof(int64_t) * (size_t)(nmodes > 0 ? nmodes : 1));
    int64_t* s = realloc(t->strides, sizeof(int64_t) * (size_t)(nmodes > 0 ? nmodes : 1));
    if (e) t->extents = e;
    if (s) t->strides = s;
    if (!e || !s) return TAPP_B200_ERR_NOMEM;
    for (int i = t->nmode; i < nmodes; i++) { t->extents[i] = 0; t->strides[i] = 0; }
    t->nmode = nmodes;
    return 0;
}

/* tensor.c:68-72 */
void TAPP_get_extents(TAPP_tensor_info info, int64_t* extents)
{
    struct tb_info* t = (struct tb_info*)info;
    if (t->nmode > 0) memcpy(extents, t->extents, sizeof(int64_t) * (size_t)t->nmode);
}

/* tensor.c:74-88: rejects a negative extent with 15 and changes nothing */
TAPP_error TAPP_set_extents(TAPP_tensor_info info, const int64_t* extents)
{
    struct tb_info* t = (struct tb_info*)info;
    for (int i = 0; i < t->nmode; i++)
        if (extents[i] < 0) return 15;
    if (t->nmode > 0) memcpy(t->extents, extents, sizeof(int64_t) * (size_t)t->nmode);
    return 0;
}

/* tensor.c:90-94 */
void TAPP_get_strides(TAPP_tensor_info info, int64_t* strides)
{
    struct tb_info* t = (struct tb_info*)info;
    if (t->nmode > 0) memcpy(strides, t->strides, sizeof(int64_t) * (size_t)t->nmode);
}

/* tensor.c:96-101 */
TAPP_error TAPP_set_strides(TAPP_tensor_info info, const int64_t* strides)
{
    struct tb_info* t = (struct tb_info*)info;
    if (t->nmode > 0) memcpy(t->strides, strides, sizeof(int64_t) * (size_t)t->nmode);
    return 0;
}

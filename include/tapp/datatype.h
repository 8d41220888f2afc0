/*
 * Storage data types and computational precisions of the TAPP C ABI.
 * Replaces api/include/tapp/datatype.h:15-95 of the reference; the numeric
 * values are part of the ABI and are the reference's.
 */
#ifndef TAPP_DATATYPE_H_
#define TAPP_DATATYPE_H_

#include "util.h"

/* datatype.h:15-42: element storage formats. */
typedef int TAPP_datatype;

enum
{
    TAPP_F32 = 0,   /* IEEE binary32 */
    TAPP_F64 = 1,   /* IEEE binary64 */
    TAPP_C32 = 2,   /* two binary32, real then imaginary (8 bytes) */
    TAPP_C64 = 3,   /* two binary64, real then imaginary (16 bytes) */
    TAPP_F16 = 4,   /* IEEE binary16 */
    TAPP_BF16 = 5,  /* bfloat16 */

    TAPP_FLOAT = TAPP_F32,
    TAPP_DOUBLE = TAPP_F64,
    TAPP_SCOMPLEX = TAPP_C32,
    TAPP_DCOMPLEX = TAPP_C64,
};

/*
 * datatype.h:71-95: precision of the multiply-accumulate. The value of
 * TAPP_F16F16_ACCUM_F16 is TAPP_F16, i.e. 4 (the reference's comment there
 * says 3, its enum value is 4).
 */
typedef int TAPP_prectype;

enum
{
    TAPP_DEFAULT_PREC = -1,
    TAPP_F32F32_ACCUM_F32 = TAPP_F32,
    TAPP_F64F64_ACCUM_F64 = TAPP_F64,
    TAPP_F16F16_ACCUM_F16 = TAPP_F16,
    TAPP_F16F16_ACCUM_F32 = 5,
    TAPP_BF16BF16_ACCUM_F32 = 6,
};

#endif /* TAPP_DATATYPE_H_ */

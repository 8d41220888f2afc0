/*
 * Launch plan shared by the host planner (C) and the CUDA layer (C++).
 *
 * The planner turns one TAPP product into index classes over the modes left
 * after repeated labels are merged (the stride-summing fold of
 * reference_implementation/src/product.c:969-1010):
 *   F  free modes = D's modes, each with its stride in A (0 when A lacks the
 *      label), in B, in C and in D; a free mode present in A and B is a
 *      Hadamard (batch) mode
 *   K  binary-contracted modes (labels in A and B, not in D)
 *   UA unary modes of A (only in A), UB unary modes of B (only in B)
 * and, for the tensor-core path, the GEMM view
 *   D[l,m,n] = alpha * sum_k A'[l,m,k] B'[l,k,n] + beta * C[l,m,n]
 * where A' = sum over UA of op_A(A), B' = sum over UB of op_B(B), L = free
 * modes in A and B, M = free modes only in A, N = free modes only in B.
 * Plain C, no CUDA types: the struct travels by value as a kernel argument.
 */
#ifndef TB_PLAN_H_
#define TB_PLAN_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TB_MAXMODES 16

/* compute domains */
enum { TB_R32 = 0, TB_R64 = 1, TB_C32 = 2, TB_C64 = 3 };
/* rounding applied to operands before they are multiplied */
enum { TB_ROUND_NONE = 0, TB_ROUND_F16 = 1, TB_ROUND_BF16 = 2, TB_ROUND_F32 = 3 };
/* execution paths */
enum {
    TB_PATH_NOOP = 0,      /* nothing to write (empty D, or a no-op precision) */
    TB_PATH_GENERIC = 1,   /* CUDA-core kernel, one thread per element of D */
    TB_PATH_REDUCE = 2,    /* CUDA-core kernel, one block per element of D (long K) */
    TB_PATH_SIMT = 3,      /* tiled CUDA-core GEMM over the L/M/N/K view */
    TB_PATH_TC = 4,        /* pack pre-pass + tcgen05 GEMM + fused epilogue */
    TB_PATH_SLICED = 5,    /* binary64 as 8-bit digit slices on the integer tensor cores */
};
/* tensor-core operand modes */
enum { TB_TC_BF16 = 0, TB_TC_F16 = 1, TB_TC_SPLIT_BF16 = 2, TB_TC_SLICED_I8 = 3 };

typedef struct tb_modes {
    int32_t n;
    int32_t reserved;
    int64_t size;                 /* product of extents */
    int64_t ext[TB_MAXMODES];
    int64_t sA[TB_MAXMODES];      /* stride in A (elements), 0 if absent */
    int64_t sB[TB_MAXMODES];
    int64_t sC[TB_MAXMODES];
    int64_t sD[TB_MAXMODES];
} tb_modes;

typedef struct tb_plan {
    int32_t tA, tB, tC, tD;       /* storage types (TAPP_datatype) */
    int32_t prec;                 /* TAPP_prectype */
    int32_t compute;              /* TB_R32 .. TB_C64 */
    int32_t round_in;             /* TB_ROUND_* applied to A, B (and C) elements */
    int32_t round_scalars;        /* TB_ROUND_* applied to alpha and beta */
    int32_t conjA, conjB, conjC, conjD;
    int32_t conjD_round_f32;      /* op_D conjugation rounds to binary32 (F64 precision) */
    int32_t skip_store;           /* D is left untouched */
    int32_t beta_zero;            /* C is not read */
    int32_t path;
    int32_t tc_mode;              /* TB_TC_* */
    int32_t slices;               /* TB_PATH_SLICED: digit slices per operand */
    int32_t split_route;          /* TB_TC_SPLIT_BF16 operands: 1 automatic, 2 packed hi/lo panels,
                                   * 3 read in place by converter warps */
    int32_t elem_stage;           /* element path: 1 (2) when A (B) is first copied into the
                                   * order in which the outputs are walked */
    double alpha_re, alpha_im;    /* scalars, already rounded per precision */
    double beta_re, beta_im;
    tb_modes F;                   /* free modes, sorted by |stride in D| */
    tb_modes K;
    tb_modes UA;
    tb_modes UB;
    tb_modes L, M, N;             /* GEMM view (sub-lists of F) */
} tb_plan;

/* Operand pointers of one product, all device-accessible. */
typedef struct tb_ptrs {
    const void* A;
    const void* B;
    const void* C;
    void* D;
} tb_ptrs;

#ifdef __cplusplus
}
#endif

#endif /* TB_PLAN_H_ */

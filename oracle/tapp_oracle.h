/*
 * CPU oracle for the TAPP tensor product — TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C, what the reference implementation's
 * TAPP_execute_product computes (reference_implementation/src/product.c).
 * It exists to check the GPU library: only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it. The GPU library never calls it.
 *
 * Three entry points:
 *   oracle_validate      the reference's error-code chain (product.c:199-206)
 *   oracle_execute       the reference's brute-force loop with its scalar types,
 *                        operation order and rounding per precision; meant to
 *                        reproduce the reference's output bit for bit
 *   oracle_execute_f64   the same product evaluated in binary64 on the inputs
 *                        rounded to the precision's operand type, plus a
 *                        per-element error scale |alpha|*sum|a||b| + |beta||c|;
 *                        optionally only on a sample of output elements
 */
#ifndef TAPP_ORACLE_H_
#define TAPP_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_tensor {
    int32_t type;          /* TAPP_datatype */
    int32_t nmode;
    int32_t op;            /* TAPP_element_op */
    int32_t reserved;
    const int64_t* extents;
    const int64_t* strides;  /* in elements */
    const int64_t* idx;      /* labels */
} oracle_tensor;

/* Error code the reference returns for this product, or 0. C_present tells
 * whether the C pointer is non-NULL. */
int oracle_validate(const oracle_tensor* A, const oracle_tensor* B,
                    const oracle_tensor* C, const oracle_tensor* D,
                    const void* beta, int C_present);

/* Reference-faithful product. Writes D in D's storage type. Returns the
 * error code (0 on success). */
int oracle_execute(int prec,
                   const oracle_tensor* A, const oracle_tensor* B,
                   const oracle_tensor* C, const oracle_tensor* D,
                   const void* alpha, const void* A_data, const void* B_data,
                   const void* beta, const void* C_data, void* D_data);

/* Binary64 product. If n_samples < 0 every element of D is computed and
 * D64 / scale are laid out like D (same element offsets, element = 2 doubles
 * for D64 (re, im) and 1 double for scale, pointers at coordinate 0).
 * If n_samples >= 0, `samples` lists linear indices over D's modes after
 * repeated labels are merged (first mode fastest); D64 receives 2 doubles per
 * sample, scale one double per sample and D_offsets the element offset of
 * that sample in D. Returns the error code. */
int oracle_execute_f64(int prec,
                       const oracle_tensor* A, const oracle_tensor* B,
                       const oracle_tensor* C, const oracle_tensor* D,
                       const void* alpha, const void* A_data, const void* B_data,
                       const void* beta, const void* C_data,
                       int64_t n_samples, const int64_t* samples,
                       double* D64, double* scale, int64_t* D_offsets);

/* Number of elements of D after repeated labels are merged. */
int64_t oracle_folded_size(const oracle_tensor* D);

#ifdef __cplusplus
}
#endif

#endif /* TAPP_ORACLE_H_ */

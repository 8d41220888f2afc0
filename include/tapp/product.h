/*
 * The tensor product of the TAPP C ABI:
 *     D <- op_D( alpha * sum op_A(A) * op_B(B) + beta * op_C(C) )
 * Replaces api/include/tapp/product.h:15-75 of the reference.
 *
 * Data pointers address the element at coordinate 0 of each tensor; negative
 * strides reach below it. They may be device pointers (used in place) or host
 * pointers (staged through device memory by the library). alpha and beta are
 * host scalars of D's storage type. C may be NULL when beta == 0, and C may
 * equal D.
 */
#ifndef TAPP_PRODUCT_H_
#define TAPP_PRODUCT_H_

#include <stdint.h>

#include "util.h"
#include "error.h"
#include "handle.h"
#include "executor.h"
#include "datatype.h"
#include "status.h"
#include "tensor.h"

/* product.h:15-21 */
typedef int TAPP_element_op;

enum
{
    TAPP_IDENTITY = 0,
    TAPP_CONJUGATE = 1,
};

/* product.h:24 */
#define TAPP_IN_PLACE NULL

/* product.h:31 */
typedef intptr_t TAPP_tensor_product;

/*
 * product.h:33-47. Copies the four label arrays and keeps references to the
 * four tensor infos; nothing is checked here, every error surfaces at execute
 * (as in reference_implementation/src/product.c:66-117).
 */
TAPP_EXPORT TAPP_error TAPP_create_tensor_product(TAPP_tensor_product* plan,
                                                  TAPP_handle handle,
                                                  TAPP_element_op op_A,
                                                  TAPP_tensor_info A,
                                                  const int64_t* idx_A,
                                                  TAPP_element_op op_B,
                                                  TAPP_tensor_info B,
                                                  const int64_t* idx_B,
                                                  TAPP_element_op op_C,
                                                  TAPP_tensor_info C,
                                                  const int64_t* idx_C,
                                                  TAPP_element_op op_D,
                                                  TAPP_tensor_info D,
                                                  const int64_t* idx_D,
                                                  TAPP_prectype prec);

/* product.h:49 */
TAPP_EXPORT TAPP_error TAPP_destroy_tensor_product(TAPP_tensor_product plan);

/*
 * product.h:53-61. Validates in the reference's order (product.c:199-206) and
 * runs the product on the GPU. Returns once D holds the result unless the
 * executor was switched to asynchronous mode (tapp_b200.h).
 */
TAPP_EXPORT TAPP_error TAPP_execute_product(TAPP_tensor_product plan,
                                            TAPP_executor exec,
                                            TAPP_status* status,
                                            const void* alpha,
                                            const void* A,
                                            const void* B,
                                            const void* beta,
                                            const void* C,
                                                  void* D);

/*
 * product.h:66-75 (declared by the reference, not implemented there).
 * Runs the same product on num_batches independent sets of operands; all
 * batches share the plan's layouts, alpha and beta. The batches run as one
 * grouped launch.
 */
TAPP_EXPORT TAPP_error TAPP_execute_batched_product(TAPP_tensor_product plan,
                                                    TAPP_executor exec,
                                                    TAPP_status* status,
                                                    int num_batches,
                                                    const void* alpha,
                                                    const void** A,
                                                    const void** B,
                                                    const void* beta,
                                                    const void** C,
                                                          void** D);

#endif /* TAPP_PRODUCT_H_ */

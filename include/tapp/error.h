/*
 * Error codes of the TAPP C ABI.
 * Replaces api/include/tapp/error.h:9-26 of the reference.
 *
 * A TAPP_error is a plain int; 0 means success. The codes that
 * TAPP_execute_product and TAPP_create_tensor_info return are the reference's
 * (reference_implementation/src/product.c:199-206, tensor.c:16-23):
 *   1  A/B extent mismatch        2  A/D extent mismatch    3  B/D extent mismatch
 *   4  label of D in neither A nor B                          5  C/D mode count differ
 *   6  C/D labels differ          7  C/D extents differ     8  D aliases itself
 *   9  A repeated-label extents  10  same for B            11  same for D
 *  12  C is NULL while beta != 0 14  negative mode count   15  negative extent
 *  33  NULL or unknown executor
 * Codes at or above 0x1000 are this implementation's own (device errors).
 */
#ifndef TAPP_ERROR_H_
#define TAPP_ERROR_H_

#include <stddef.h>
#include <stdbool.h>

#include "util.h"

typedef int TAPP_error;

/* error.h:12 — true iff error == 0. */
TAPP_EXPORT bool TAPP_check_success(TAPP_error error);

/*
 * error.h:24-26 — writes at most maxlen-1 characters of the explanation of
 * `error` plus a terminating NUL into `message` and returns the number of
 * characters written; with maxlen == 0 nothing is written and the length of
 * the whole explanation is returned.
 */
TAPP_EXPORT size_t TAPP_explain_error(TAPP_error error,
                                      size_t maxlen,
                                      char* message);

#endif /* TAPP_ERROR_H_ */

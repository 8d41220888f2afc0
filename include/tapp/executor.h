/*
 * Executor of the TAPP C ABI.
 * Replaces api/include/tapp/executor.h:9-18 of the reference. An executor
 * created here points at an int holding 1 (the id the reference's own
 * executor carries, reference_implementation/src/executor.c:11), followed by
 * this library's execution settings; executors that point at a bare int 1, 2
 * or 12 are accepted too, as by the reference (product.c:878-885).
 */
#ifndef TAPP_EXECUTOR_H_
#define TAPP_EXECUTOR_H_

#include <stdint.h>

#include "util.h"
#include "error.h"

typedef intptr_t TAPP_executor;

/* executor.h:11 */
TAPP_EXPORT TAPP_error TAPP_create_executor(TAPP_executor* exec);

/* executor.h:18 */
TAPP_EXPORT TAPP_error TAPP_destroy_executor(TAPP_executor exec);

#endif /* TAPP_EXECUTOR_H_ */

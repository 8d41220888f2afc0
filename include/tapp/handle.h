/*
 * Library handle of the TAPP C ABI.
 * Replaces api/include/tapp/handle.h:9-24 of the reference. The handle owns the
 * device and stream state used by products created with it; products whose
 * handle was never created (as some reference callers do) use the library's
 * per-device default state.
 */
#ifndef TAPP_HANDLE_H_
#define TAPP_HANDLE_H_

#include <stdint.h>

#include "util.h"
#include "error.h"

typedef intptr_t TAPP_handle;

/* handle.h:11 */
TAPP_EXPORT TAPP_error TAPP_create_handle(TAPP_handle* handle);

/* handle.h:24 */
TAPP_EXPORT TAPP_error TAPP_destroy_handle(TAPP_handle handle);

#endif /* TAPP_HANDLE_H_ */

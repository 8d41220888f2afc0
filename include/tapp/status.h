/*
 * Status objects of the TAPP C ABI.
 * Replaces api/include/tapp/status.h:9-17 of the reference (declared there,
 * never implemented). A status object is written by TAPP_execute_product only
 * when the executor asks for one (key TAPP_B200_ATTR_WANT_STATUS in
 * tapp_b200.h); it is then read with TAPP_attr_get and released here.
 */
#ifndef TAPP_STATUS_H_
#define TAPP_STATUS_H_

#include <stdint.h>

#include "util.h"
#include "error.h"

typedef intptr_t TAPP_status;

/* status.h:17 */
TAPP_EXPORT TAPP_error TAPP_destroy_status(TAPP_status status);

#endif /* TAPP_STATUS_H_ */

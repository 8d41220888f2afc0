/*
 * TAPP C ABI, B200 implementation. Same umbrella as the reference's
 * api/include/tapp.h:1-21: including this header declares the whole API.
 */
#ifndef TAPP_TAPP_H_
#define TAPP_TAPP_H_

#ifdef __cplusplus
extern "C" {
#endif

#include "tapp/error.h"
#include "tapp/attributes.h"
#include "tapp/datatype.h"
#include "tapp/handle.h"
#include "tapp/executor.h"
#include "tapp/status.h"
#include "tapp/tensor.h"
#include "tapp/product.h"

#ifdef __cplusplus
}
#endif

#endif /* TAPP_TAPP_H_ */

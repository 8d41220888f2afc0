/*
 * Tensor layout descriptions of the TAPP C ABI.
 * Replaces api/include/tapp/tensor.h:10-44 of the reference.
 *
 * A tensor info holds a storage type, a mode count and, per mode, an extent
 * and a stride counted in elements (any sign, zero allowed). The info owns
 * copies of both arrays. Products keep a reference to the info, so a change
 * made through the setters is seen by the next TAPP_execute_product.
 */
#ifndef TAPP_TENSOR_H_
#define TAPP_TENSOR_H_

#include <stdint.h>

#include "util.h"
#include "error.h"
#include "datatype.h"

typedef intptr_t TAPP_tensor_info;

/* tensor.h:22-26; returns 14 for nmode < 0 and 15 for a negative extent. */
TAPP_EXPORT TAPP_error TAPP_create_tensor_info(TAPP_tensor_info* info,
                                               TAPP_datatype type,
                                               int nmode,
                                               const int64_t* extents,
                                               const int64_t* strides);

/* tensor.h:28 */
TAPP_EXPORT TAPP_error TAPP_destroy_tensor_info(TAPP_tensor_info info);

/* tensor.h:30 */
TAPP_EXPORT int TAPP_get_nmodes(TAPP_tensor_info info);

/* tensor.h:32-33; returns 14 for nmodes < 0. */
TAPP_EXPORT TAPP_error TAPP_set_nmodes(TAPP_tensor_info info,
                                       int nmodes);

/* tensor.h:35-36 */
TAPP_EXPORT void TAPP_get_extents(TAPP_tensor_info info,
                                  int64_t* extents);

/* tensor.h:38-39; returns 15 for a negative extent. */
TAPP_EXPORT TAPP_error TAPP_set_extents(TAPP_tensor_info info,
                                        const int64_t* extents);

/* tensor.h:41-42 */
TAPP_EXPORT void TAPP_get_strides(TAPP_tensor_info info,
                                  int64_t* strides);

/* tensor.h:44-45 */
TAPP_EXPORT TAPP_error TAPP_set_strides(TAPP_tensor_info info,
                                        const int64_t* strides);

#endif /* TAPP_TENSOR_H_ */

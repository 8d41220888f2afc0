/*
 * Attribute objects of the TAPP C ABI.
 * Replaces api/include/tapp/attributes.h:9-18 of the reference (declared there,
 * never implemented by it). Here an attribute object is a TAPP_handle or a
 * TAPP_executor; the keys are listed in tapp_b200.h.
 */
#ifndef TAPP_ATTRIBUTES_H_
#define TAPP_ATTRIBUTES_H_

#include <stdint.h>

#include "util.h"
#include "error.h"

typedef intptr_t TAPP_attr;
typedef int TAPP_key;

/* attributes.h:14 */
TAPP_EXPORT TAPP_error TAPP_attr_set(TAPP_attr attr, TAPP_key key, void* value);

/* attributes.h:16 */
TAPP_EXPORT TAPP_error TAPP_attr_get(TAPP_attr attr, TAPP_key key, void** value);

/* attributes.h:18 */
TAPP_EXPORT TAPP_error TAPP_attr_clear(TAPP_attr attr, TAPP_key key);

#endif /* TAPP_ATTRIBUTES_H_ */

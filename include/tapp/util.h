/*
 * Export macro of the TAPP C ABI.
 * Mirrors api/include/tapp/util.h:5-9 of the reference: every entry point has
 * default ELF visibility, and C++ includers see C linkage.
 */
#ifndef TAPP_UTIL_H_
#define TAPP_UTIL_H_

#ifdef __cplusplus
#define TAPP_EXPORT extern "C" __attribute__((visibility("default")))
#else
#define TAPP_EXPORT __attribute__((visibility("default")))
#endif

#endif /* TAPP_UTIL_H_ */

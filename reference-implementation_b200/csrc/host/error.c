/*
 * Error codes: TAPP_check_success and TAPP_explain_error.
 * Behaviour follows reference_implementation/src/error.c:10-76; the texts of
 * codes 0-14 are the reference's, byte for byte, because callers print them
 * (the reference's example programs do). Codes the reference leaves without
 * text (15, 33, its own debug code 137, and this library's codes >= 0x1000)
 * get a text here instead of the reference's undefined behaviour.
 */
#include <string.h>

#include "tb_internal.h"

/* error.c:10-12 */
bool TAPP_check_success(TAPP_error error)
{
    return error == 0;
}

static const char* message_of(TAPP_error error)
{
    switch (error) {
    /* error.c:21-64 */
    case 0: return "Success.";
    case 1: return "The extents for the indices shared between tensor A and B does not match.";
    case 2: return "The extents for the indices shared between tensor A and D does not match.";
    case 3: return "The extents for the indices shared between tensor B and D does not match.";
    case 4: return "Tensor D has indices not shared with tensor A or B.";
    case 5: return "The tensors C and D have different amount of dimensions.";
    case 6: return "The indices of tensor C and D does not line up.";
    case 7: return "The extents for the indices shared between tensor C and D does not match.";
    case 8: return "Aliasing found within tensor D.";
    case 9: return "An idx in tensor A has two different extents.";
    case 10: return "An idx in tensor B has two different extents.";
    case 11: return "An idx in tensor D has two different extents.";
    case 12: return "C should not be NULL while beta is not zero.";
    case 13: return "Nmode can not be negative.";
    case 14: return "Extents can not be negative.";
    /* codes returned by the reference without a text */
    case 15: return "A tensor extent is negative.";
    case 33: return "The executor is NULL or not a known executor.";
    case 137: return "Results of two executors differ.";
    /* this library */
    case TAPP_B200_ERR_CUDA: return "A CUDA call failed (no usable GPU, or a launch error).";
    case TAPP_B200_ERR_LIMIT: return "The product has more index modes than the B200 planner supports.";
    case TAPP_B200_ERR_UNSUPPORTED: return "Storage type, precision or option not supported by the B200 library.";
    case TAPP_B200_ERR_NOMEM: return "Device memory allocation failed.";
    case TAPP_B200_ERR_INVALID: return "Invalid object or argument.";
    case TAPP_B200_ERR_LABELS: return "A tensor has more modes than when the product was created.";
    case TAPP_B200_ERR_SCRATCH:
        return "The product needs more scratch memory than the 32 MiB array of the allocation-free entry point.";
    case TAPP_B200_ERR_BUDGET: return "The product needs more device memory than the server's whole HBM budget.";
    default: return "Unknown error code.";
    }
}

/* error.c:69-76 */
size_t TAPP_explain_error(TAPP_error error, size_t maxlen, char* message)
{
    const char* m = message_of(error);
    size_t len = strlen(m);
    if (maxlen == 0) return len;
    size_t w = maxlen - 1 < len ? maxlen - 1 : len;
    memcpy(message, m, w);
    message[w] = '\0';
    return w;
}

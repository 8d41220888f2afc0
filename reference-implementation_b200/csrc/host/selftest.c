/*
 * tapp_b200_selftest_waits: shows that the kernels' bounded waits end. A
 * kernel waits, with the same device functions the tensor-core kernels use,
 * on a flag and an mbarrier phase that nothing completes; each wait gives up
 * after limit_ms, raises the kernel's abort word and returns. No
 * counterpart in the reference.
 */
#include "tb_internal.h"

TAPP_error tapp_b200_selftest_waits(double limit_ms, int* flag_wait_expired, int* barrier_wait_expired)
{
    if (!flag_wait_expired || !barrier_wait_expired || !(limit_ms > 0.0) || limit_ms > 10000.0)
        return TAPP_B200_ERR_INVALID;
    int out[4] = {0, 0, 0, 0};
    if (tbk_wait_selftest((unsigned long long)(limit_ms * 1e6), out) != 0) return TAPP_B200_ERR_CUDA;
    /* a wait that gave up returned false and left the abort word raised */
    *flag_wait_expired = out[0] == 0 && out[1] == 1;
    *barrier_wait_expired = out[2] == 0 && out[3] == 1;
    return 0;
}

"""Failure detection without a GPU fault. Every wait in the library's kernels
is bounded: a wait that runs out raises the kernel's abort word and returns,
so a stalled product ends with an error instead of a hang. The self-test
kernel waits, with those same device functions, on a flag that nothing
raises and on an mbarrier phase that nothing completes; both waits must give
up after their limit, and the context must stay usable afterwards."""
import ctypes as C
import time

import numpy as np
import pytest

import tapp_b200
from test_gpu_parity import check_against_f64

pytestmark = pytest.mark.gpu


def _selftest(tapp):
    f = tapp.lib.tapp_b200_selftest_waits
    f.restype = C.c_int
    f.argtypes = [C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return f


def test_bounded_waits_expire_and_context_stays_usable(tapp, oracle, gpu):
    f = _selftest(tapp)
    flag, barrier = C.c_int(-1), C.c_int(-1)
    t0 = time.perf_counter()
    assert f(200.0, C.byref(flag), C.byref(barrier)) == 0
    dt = time.perf_counter() - t0
    assert flag.value == 1 and barrier.value == 1
    assert 0.35 < dt < 10.0  # two waits of 0.2 s, one after the other
    # the same context runs products correctly right after
    from tapp_b200.workloads import dense_contraction_case
    check_against_f64(tapp, oracle, dense_contraction_case(np.random.default_rng(5), extent=8), device=True)
    check_against_f64(tapp, oracle, dense_contraction_case(np.random.default_rng(6), extent=16), device=True)

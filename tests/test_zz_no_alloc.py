"""The allocation-free entry point, tapp_b200_execute_product_noalloc.

Callers that cannot allocate device memory while a product runs (code inside
an allocator or memory manager, or a program that has given the whole device
to its own pool) use this entry point: it runs the tensor-core product with
its operand scratch in a fixed 32 MiB device array of the library and calls
no allocator. These tests call it through the C ABI and compare its D with
what TAPP_execute_product writes for the same product, within the bound the
other GPU tests use, on two calls in a row (the second reuses the array the
first left behind). The file is named to be collected last, so that a run
that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

import tapp_b200
from tapp_b200.workloads import large_dense_case
from helpers import error_bound, d_values

pytestmark = pytest.mark.gpu


def _noalloc(tapp):
    f = tapp.lib.tapp_b200_execute_product_noalloc
    f.restype = C.c_int
    f.argtypes = [tapp_b200.intptr, tapp_b200.intptr] + [C.c_void_p] * 6
    return f


def _plan(tapp, case):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    err, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                    [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    assert err == 0
    return plan, infos


def _device(case, torch):
    out = []
    for t in (case.A, case.B, case.C, case.D):
        x = torch.from_numpy(t.buf.view(np.uint8).copy()).cuda()
        out.append((x, x.data_ptr() + t.base * t.itemsize))
    return out


@pytest.mark.parametrize("prec,split", [(tapp_b200.TAPP_BF16BF16_ACCUM_F32, 0), (tapp_b200.TAPP_F32F32_ACCUM_F32, 1)])
def test_noalloc_matches_execute_product(tapp, oracle, gpu, prec, split):
    import torch
    case = large_dense_case(np.random.default_rng(21), prec, tapp_b200.TAPP_F32, extent=16)
    _, D64, scale = oracle.execute_f64(case.copy())
    bound = error_bound(case, scale, D64, 2.0 ** -16 if split else 0.0)
    plan, infos = _plan(tapp, case)
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, split)
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_TC)
    dev = _device(case, torch)
    D0 = dev[3][0].clone()
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), case.alpha.ctypes.data, dev[0][1], dev[1][1],
                                        case.beta.ctypes.data, dev[2][1], dev[3][1])
    assert err == 0
    want = dev[3][0].cpu().numpy().view(np.float32).astype(np.complex128)
    noalloc = _noalloc(tapp)
    for call in range(2):
        dev[3][0].copy_(D0)
        err = noalloc(plan, ex, case.alpha.ctypes.data, dev[0][1], dev[1][1], case.beta.ctypes.data,
                      dev[2][1], dev[3][1])
        assert err == 0, tapp.explain(err)
        got = dev[3][0].cpu().numpy().view(np.float32).astype(np.complex128)
        assert (np.abs(got - want) <= bound).all(), call
        assert (np.abs(got - D64) <= bound).all(), call
    tapp.lib.TAPP_destroy_executor(ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        tapp.lib.TAPP_destroy_tensor_info(h)


def test_noalloc_rejects_products_beyond_its_array(tapp, gpu):
    """M = N = K = 4096 needs 64 MiB of operand panels: refused, nothing launched."""
    import torch
    case = large_dense_case(np.random.default_rng(22), tapp_b200.TAPP_BF16BF16_ACCUM_F32, tapp_b200.TAPP_F32,
                            extent=64)
    plan, infos = _plan(tapp, case)
    ex = tapp.create_executor()
    dev = _device(case, torch)
    n0 = tapp.launches()
    err = _noalloc(tapp)(plan, ex, case.alpha.ctypes.data, dev[0][1], dev[1][1], case.beta.ctypes.data,
                         dev[2][1], dev[3][1])
    assert err == 0x1007 and "32 MiB" in tapp.explain(err)
    assert tapp.launches() == n0
    tapp.lib.TAPP_destroy_executor(ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)


def test_noalloc_rejects_host_operands(tapp, gpu):
    case = large_dense_case(np.random.default_rng(23), tapp_b200.TAPP_BF16BF16_ACCUM_F32, tapp_b200.TAPP_F32,
                            extent=16)
    plan, infos = _plan(tapp, case)
    ex = tapp.create_executor()
    err = _noalloc(tapp)(plan, ex, case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(), case.beta.ctypes.data,
                         case.C.ptr(), case.D.ptr())
    assert err == tapp_b200.ERR_INVALID
    tapp.lib.TAPP_destroy_executor(ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)

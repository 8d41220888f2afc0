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


def _matmul_case(rng, m, n, k, prec):
    """D[m,n] = 1.3 sum_k A[m,k] B[k,n] + 0.7 C, binary32 storage, ragged
    sizes (not multiples of the 128 x 256 tiles nor of the 64-deep
    contraction blocks)."""
    from tapp_b200.case import Case, alloc, fill_uniform, scalar
    from tapp_b200.workloads import colmajor
    T = lambda ext, idx: fill_uniform(alloc(tapp_b200.TAPP_F32, ext, colmajor(ext), [ord(c) for c in idx]), rng)
    return Case(T([m, k], "mk"), T([k, n], "kn"), T([m, n], "mn"), T([m, n], "mn"),
                scalar(tapp_b200.TAPP_F32, 1.3), scalar(tapp_b200.TAPP_F32, 0.7), prec, False, f"matmul_{m}x{n}x{k}")


def _cases():
    from tapp_b200.workloads import dense_contraction_case
    F32, BF16P, F16P = tapp_b200.TAPP_F32F32_ACCUM_F32, tapp_b200.TAPP_BF16BF16_ACCUM_F32, 5
    return [
        ("dense16_bf16", lambda: large_dense_case(np.random.default_rng(21), BF16P, tapp_b200.TAPP_F32, extent=16), 0),
        ("dense16_split", lambda: large_dense_case(np.random.default_rng(21), F32, tapp_b200.TAPP_F32, extent=16), 1),
        ("matmul_ragged_f16", lambda: _matmul_case(np.random.default_rng(24), 200, 300, 150, F16P), 0),
        ("matmul_ragged_split", lambda: _matmul_case(np.random.default_rng(25), 333, 129, 517, F32), 1),
        ("complex_bf16", lambda: dense_contraction_case(np.random.default_rng(26), extent=12,
                                                        dtype=tapp_b200.TAPP_C32, prec=BF16P), 0),
    ]


@pytest.mark.parametrize("name,make,split", _cases(), ids=[c[0] for c in _cases()])
def test_noalloc_matches_execute_product(tapp, oracle, gpu, name, make, split):
    """Two calls in a row through the allocation-free entry point give the D
    that TAPP_execute_product gives (within the bound of the GPU tests), and
    the library asks CUDA for no memory during them."""
    import torch
    case = make()
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
    # D is dense in every case: its buffer holds exactly its elements
    read_d = lambda: dev[3][0].cpu().numpy().view(case.D.buf.dtype).astype(np.complex128)
    want = read_d()
    noalloc = _noalloc(tapp)
    for call in range(2):
        dev[3][0].copy_(D0)
        torch.cuda.synchronize()
        a0 = tapp.allocations()
        err = noalloc(plan, ex, case.alpha.ctypes.data, dev[0][1], dev[1][1], case.beta.ctypes.data,
                      dev[2][1], dev[3][1])
        assert err == 0, tapp.explain(err)
        assert tapp.allocations() == a0, "the allocation-free entry point asked CUDA for memory"
        got = read_d()
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

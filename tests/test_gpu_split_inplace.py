"""GPU parity of the two operand routes of the split-bfloat16 product
(float32 products on the tensor cores: hi*hi + hi*lo + lo*hi of bfloat16
parts, accumulated in binary32):

  in place (TAPP_B200_ATTR_F32_MODE = 3): the GEMM's converter warps load A
    and B from their own strided layouts and split each value in shared
    memory; no pack launch, no operand panels (one kernel per product).
    Operands qualify when their contiguous mode (stride 1, extent divisible
    by 8) is a row or a contracted mode, every other stride is divisible by
    4 and the base is 16-byte aligned; A has at least 256 rows.
  panels (TAPP_B200_ATTR_F32_MODE = 2, and the automatic mode 1): one pass
    per operand writes [hi | lo] bfloat16 panels, the GEMM's TMA loads bring
    both parts of a 64-deep block into one stage (three launches).

Each case checks the route (the plan description and the kernel count) and
the result against the oracle's binary64 evaluation with the split-bfloat16
bound (tests/helpers: error_bound with 2^-16 relative to |alpha| sum |a||b|).
"""
import ctypes as C
import zlib

import numpy as np
import pytest

import tapp_b200
from tapp_b200.case import Case, alloc, fill_uniform, scalar
from tapp_b200.workloads import large_dense_case
from helpers import error_bound, d_values, run_on_device

pytestmark = pytest.mark.gpu
SPLIT_REL = 2.0 ** -16
F32, F64 = tapp_b200.TAPP_F32, tapp_b200.TAPP_F64


def _t(rng, ext, idx, strides=None, dtype=F32, fill=True):
    if strides is None:
        strides, acc = [], 1
        for e in ext:
            strides.append(acc)
            acc *= e
    T = alloc(dtype, ext, strides, [ord(c) for c in idx])
    return fill_uniform(T, rng) if fill else T


def _matmul(rng, m, n, k, a_km=False, b_nk=False, beta=0.7, cd=F32, lead_pad=0):
    """D[m,n] = 1.1 sum_k A[m,k] B[k,n] + beta C; A stored k-fastest when
    a_km, B stored n-fastest when b_nk; lead_pad pads A's leading dimension."""
    if a_km:
        A = _t(rng, [m, k], "mk", [k + lead_pad, 1])
    else:
        A = _t(rng, [m, k], "mk", [1, m + lead_pad])
    B = _t(rng, [k, n], "kn", [n, 1] if b_nk else None)
    Cc = _t(rng, [m, n], "mn", dtype=cd)
    D = _t(rng, [m, n], "mn", dtype=cd)
    return Case(A, B, Cc, D, scalar(cd, 1.1), scalar(cd, beta), tapp_b200.TAPP_F32F32_ACCUM_F32, beta == 0.0,
                f"matmul_{m}x{n}x{k}")


def _batched(rng, m, n, k, h):
    A = _t(rng, [m, k, h], "mkh")
    B = _t(rng, [k, n, h], "knh")
    Cc = _t(rng, [m, n, h], "mnh")
    D = _t(rng, [m, n, h], "mnh")
    return Case(A, B, Cc, D, scalar(F32, 0.9), scalar(F32, -0.4), 0, False, "batched")


CASES = {
    "dense4_extent32": lambda r: large_dense_case(r, 0, 0, extent=32),
    "mk_kn": lambda r: _matmul(r, 512, 384, 320),
    "km_nk_ragged": lambda r: _matmul(r, 264, 200, 136, a_km=True, b_nk=True),
    "km_kn_padded_lead": lambda r: _matmul(r, 304, 136, 200, a_km=True, lead_pad=8),
    "beta_zero": lambda r: _matmul(r, 256, 256, 64, beta=0.0),
    "c_d_binary64": lambda r: _matmul(r, 288, 72, 96, cd=F64),
    "batched_hadamard": lambda r: _batched(r, 320, 96, 72, 3),
}


def _executor(tapp, mode=3):
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_TC)
    tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, mode)
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    return ex


def _describe(tapp, case, ex):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    d = tapp.describe(plan, ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        tapp.lib.TAPP_destroy_tensor_info(h)
    return d


@pytest.mark.parametrize("mode", [3, 2, 1], ids=["in_place", "panels", "automatic"])
@pytest.mark.parametrize("name", list(CASES))
def test_split_routes(tapp, oracle, gpu, name, mode):
    import torch
    case = CASES[name](np.random.default_rng(zlib.crc32(name.encode())))
    ex = _executor(tapp, mode)
    in_place = mode == 3
    assert ("operands=in_place" if in_place else "operands=packed") in _describe(tapp, case, ex)
    run = case.copy()
    dev, ptrs = [], []
    for t in (run.A, run.B, run.C, run.D):
        x = torch.from_numpy(t.buf.view(np.uint8).copy()).cuda()
        dev.append(x)
        ptrs.append(x.data_ptr() + t.base * t.itemsize)
    st = tapp_b200.intptr(0)
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (run.A, run.B, run.C, run.D)]
    _, plan = tapp.create_product(0, [t.op for t in (run.A, run.B, run.C, run.D)], infos,
                                  [run.A.idx, run.B.idx, run.C.idx, run.D.idx], run.prec)
    err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), run.alpha.ctypes.data, ptrs[0], ptrs[1],
                                        run.beta.ctypes.data, None if run.C_is_null else ptrs[2], ptrs[3])
    torch.cuda.synchronize()
    assert err == 0, tapp.explain(err)
    # in place: the GEMM alone; panels: a pack per operand and the GEMM
    assert tapp.status_value(st.value, tapp_b200.STATUS_KERNELS) == (1 if in_place else 3)
    tapp.lib.TAPP_destroy_status(st.value)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        tapp.lib.TAPP_destroy_tensor_info(h)
    tapp.lib.TAPP_destroy_executor(ex)
    run.D.buf[:] = dev[3].cpu().numpy().view(run.D.buf.dtype)
    e64, D64, scale = oracle.execute_f64(case.copy())
    assert e64 == 0
    bound = error_bound(case, scale, D64, SPLIT_REL)
    got = d_values(run.D)
    bad = np.abs(got - D64) > bound
    assert not bad.any(), (name, int(bad.sum()), got[bad][:4], D64[bad][:4], bound[bad][:4])


@pytest.mark.parametrize("name", list(CASES))
def test_split_routes_same_bits(tapp, gpu, name):
    """The two routes split every value the same way (hi = bf16(x), lo =
    bf16(x - hi)) and issue the same three MMAs per 16-deep step: the panels
    written by the pack pass and the tiles written by the converter warps
    give the same D bit for bit."""
    case = CASES[name](np.random.default_rng(zlib.crc32(name.encode()) + 1))
    outs = []
    for mode in (3, 2):
        ex = _executor(tapp, mode)
        run = case.copy()
        assert run_on_device(tapp, run, ex) == 0
        tapp.lib.TAPP_destroy_executor(ex)
        outs.append(run.D.buf.view(np.uint8).copy())
    assert np.array_equal(outs[0], outs[1]), name


def test_split_packed_when_layout_does_not_qualify(tapp, oracle, gpu):
    """A contiguous contracted mode of extent 12 (not a multiple of 8): the
    operands are packed first (three launches), same bound."""
    rng = np.random.default_rng(77)
    case = _matmul(rng, 256, 128, 12, a_km=True)
    ex = _executor(tapp)
    assert "operands=packed" in _describe(tapp, case, ex)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    tapp.lib.TAPP_destroy_executor(ex)
    e64, D64, scale = oracle.execute_f64(case.copy())
    bound = error_bound(case, scale, D64, SPLIT_REL)
    assert (np.abs(d_values(run.D) - D64) <= bound).all()


@pytest.mark.parametrize("mode", [3, 2])
def test_split_repeatable(tapp, gpu, mode):
    """The summation order is fixed: two runs of the same product give the
    same bits (either route)."""
    case = _matmul(np.random.default_rng(5), 512, 256, 512)
    ex = _executor(tapp, mode)
    outs = []
    for _ in range(2):
        run = case.copy()
        assert run_on_device(tapp, run, ex) == 0
        outs.append(run.D.buf.copy())
    tapp.lib.TAPP_destroy_executor(ex)
    assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))

"""GPU parity of the sliced binary64 path (TAPP_B200_ATTR_F64_MODE = S):
binary64 and complex-double products as exact 8-bit integer digit products
on the tensor cores, added up in binary64.

Bound per output (derivation in csrc/cuda/sliced.cu): with |A[r,:]| < 2^E_r
and |B[:,c]| < 2^F_c, dropping the digit pairs of order >= S and the digits
beyond the S-th errs by at most |alpha| K (S + 4) 2^(-7S) 2^(E_r + F_c), K the
number of real products per output (2x the contracted size for complex). The
tests bound 2^(E_r + F_c) by 4 max|A| max|B| (the largest elements of the
operands) and add the binary64 roundings of the epilogue, so a wrong digit,
scale or level shows up as an error of order max|A| max|B| instead.
"""
import ctypes as C

import numpy as np
import pytest

import tapp_b200
from tapp_b200.workloads import double_case
from families import bounded_case
from helpers import run_on_device, folded_sizes, d_values

pytestmark = pytest.mark.gpu

F64_MODE = 0x1007
PATH_SLICED = 5


def sliced_executor(tapp, slices):
    ex = tapp.create_executor()
    assert tapp.set_int(ex, F64_MODE, slices) == 0
    return ex


def describe(tapp, case, ex):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    d = tapp.describe(plan, ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    return d


def maxabs(t):
    v = t.buf
    return float(np.max(np.abs(v))) if v.size else 0.0


def sliced_bound(case, slices, scale, D64):
    K, UA, UB = folded_sizes(case)
    cplx = case.D.dtype in (tapp_b200.TAPP_C32, tapp_b200.TAPP_C64)
    kreal = K * (2 if cplx else 1)
    alpha = abs(complex(case.alpha[0]))
    digits = alpha * kreal * (slices + 4) * 2.0 ** (-7 * slices) * 4 * maxabs(case.A) * maxabs(case.B)
    u = 2.0 ** -53
    return digits + 8 * u * scale + 2 * u * np.abs(D64) + 1e-300


def check(tapp, oracle, case, slices, samples=None, device=True):
    ex = sliced_executor(tapp, slices)
    assert f"path=sliced" in describe(tapp, case, ex) and f"slices={slices}" in describe(tapp, case, ex)
    run = case.copy()
    err = run_on_device(tapp, run, ex) if device else run.run(tapp, executor=ex)
    assert err == 0, tapp.explain(err)
    tapp.lib.TAPP_destroy_executor(ex)
    if samples is None:
        e64, D64, scale = oracle.execute_f64(case.copy())
        got = d_values(run.D)
    else:
        e64, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
        got = run.D.buf[run.D.base + offs].astype(np.complex128)
    assert e64 == 0
    bound = sliced_bound(case, slices, scale, D64)
    bad = np.abs(got - D64) > bound
    assert not bad.any(), (case.name, slices, int(bad.sum()), (got - D64)[bad][:4], bound[bad][:4])
    return np.max(np.abs(got - D64) / np.maximum(scale, 1e-300))


@pytest.mark.parametrize("slices", [3, 5, 8])
@pytest.mark.parametrize("cplx", [False, True])
def test_four_index_contraction(tapp, oracle, gpu, slices, cplx):
    """D[a,b,i,j] = sum_{e,f} A[a,b,e,f] B[e,f,i,j] + C with extents 24 and 12
    (M = 576, N = 144, K = 576), log-uniform magnitudes over 8 decades;
    complex double with conj(A)."""
    case = double_case(np.random.default_rng(120 + slices + 10 * cplx), cplx=cplx, ab=24, ij=12)
    check(tapp, oracle, case, slices)


def test_eight_slices_reach_binary64_accuracy(tapp, oracle, gpu):
    """With S = 8 the error relative to sum |alpha a b| + |beta c| stays at the
    level of native binary64 arithmetic on the log-uniform data."""
    case = double_case(np.random.default_rng(131), cplx=False, ab=24, ij=12)
    rel = check(tapp, oracle, case, 8)
    assert rel < 1e-13, rel


@pytest.mark.parametrize("seed", range(4))
def test_strided_batched_and_mixed_types(tapp, oracle, gpu, seed):
    """Hadamard (batch) modes, subtensor views with mixed-sign strides,
    permuted D, element ops, binary32 operands under binary64 arithmetic."""
    rng = np.random.default_rng(140 + seed)
    types = [(1, 1, 1, 1), (0, 1, 1, 1), (3, 3, 3, 3), (2, 3, 3, 3)][seed]
    case = bounded_case(rng, types=types, prec=-1, n_contracted=2, n_hadamard=1, n_freeA=2, n_freeB=2,
                        ext_choices=[11, 13], subtensor=bool(seed & 1), mixed=bool(seed & 2),
                        ops=[seed & 1, (seed >> 1) & 1, 0, seed & 1], max_work=1e9)
    check(tapp, oracle, case, 6, device=bool(seed & 1))


def long_contraction_case(rng, k1, k2, m=64, n=64):
    """D[a,i] = sum_{e,f} A[a,e,f] B[e,f,i] + C in binary64, log-uniform values."""
    from tapp_b200.workloads import RequestSpec, case_from_spec, loguniform
    spec = RequestSpec("long", tapp_b200.TAPP_F64, -1, ([m, k1, k2], [k1, k2, n], [m, n], [m, n]),
                       ([0, 1, 2], [1, 2, 3], [0, 3], [0, 3]), 1.0, 0.5)
    case = case_from_spec(rng, spec)
    for t in (case.A, case.B, case.C):
        t.buf[:] = loguniform(rng, t.buf.size, False)
    return case


def test_levels_split_by_integer_range(tapp, oracle, gpu):
    """K = 40,000 terms: at most 3 digit pairs fit one 32-bit sum, so the
    higher levels run as several GEMMs."""
    check(tapp, oracle, long_contraction_case(np.random.default_rng(150), 200, 200), 6)


def test_contraction_chunks(tapp, oracle, gpu):
    """K = 140,000 terms: even one digit pair could pass 2^31, so every pair
    runs over K chunks of 133,120."""
    check(tapp, oracle, long_contraction_case(np.random.default_rng(151), 350, 400), 3)


def test_zero_and_nonfinite_rows(tapp, oracle, gpu):
    """A row of zeros gives beta*C exactly; a row holding inf gives NaN (the
    scheme needs finite inputs; the native path is the one that propagates
    infinities the reference's way)."""
    case = double_case(np.random.default_rng(160), cplx=False, ab=16, ij=16)
    A = case.A.buf.reshape(16 * 16, 16 * 16, order="F")  # rows (a,b), columns (e,f)
    A[3, :] = 0.0
    A[7, 5] = np.inf
    ex = sliced_executor(tapp, 6)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    tapp.lib.TAPP_destroy_executor(ex)
    D = run.D.buf.reshape(256, 256, order="F")
    Cm = case.C.buf.reshape(256, 256, order="F")
    assert np.array_equal(D[3, :], float(case.beta[0]) * Cm[3, :])
    assert np.isnan(D[7, :]).all()
    assert np.isfinite(np.delete(D, 7, axis=0)).all()


def test_status_reports_sliced_mode(tapp, gpu):
    case = double_case(np.random.default_rng(170), cplx=False, ab=16, ij=16)
    ex = sliced_executor(tapp, 7)
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [case.A.idx, case.B.idx, case.C.idx, case.D.idx], -1)
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(),
                                        case.beta.ctypes.data, case.C.ptr(), case.D.ptr())
    assert err == 0
    assert tapp.status_value(st.value, tapp_b200.STATUS_PATH) == PATH_SLICED
    assert tapp.status_value(st.value, tapp_b200.STATUS_TC_MODE) == 3
    assert tapp.status_value(st.value, tapp_b200.STATUS_KERNELS) >= 6
    tapp.lib.TAPP_destroy_status(st.value)
    tapp.lib.TAPP_destroy_executor(ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)


def test_status_error_bound_sliced(tapp, oracle, gpu):
    """The sliced path's reported bound, times |alpha| 2^(E+F) <= 4 |alpha|
    max|A| max|B|, covers the measured error."""
    case = double_case(np.random.default_rng(171), cplx=False, ab=24, ij=12)
    ex = sliced_executor(tapp, 5)
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [case.A.idx, case.B.idx, case.C.idx, case.D.idx], -1)
    run = case.copy()
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), run.alpha.ctypes.data, run.A.ptr(), run.B.ptr(),
                                        run.beta.ctypes.data, run.C.ptr(), run.D.ptr())
    assert err == 0
    bound = tapp.status_value(st.value, tapp_b200.STATUS_ERR_BOUND)
    tapp.lib.TAPP_destroy_status(st.value)
    K, _, _ = folded_sizes(case)
    assert bound == pytest.approx(K * 9 * 2.0 ** -35)
    _, D64, scale = oracle.execute_f64(case.copy())
    lim = bound * 4 * maxabs(case.A) * maxabs(case.B) + 8 * 2.0 ** -53 * scale + 2 * 2.0 ** -53 * np.abs(D64)
    assert (np.abs(d_values(run.D) - D64) <= lim).all()
    tapp.lib.TAPP_destroy_executor(ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)

"""GPU parity: the CUDA library against the reference's outputs and the oracle.

Every product runs through the C ABI (TAPP_execute_product) of
lib/libtapp-b200.so on cuda:0, with host pointers (the drop-in path the
reference's callers use) and with device pointers. Results are compared:
  - with the reference's own recorded outputs (golden/ fixtures), and
  - with the oracle's binary64 evaluation, element by element, within the
    bound of helpers.error_bound: gamma_n * (|alpha| sum|a||b| + |beta||c|)
    plus the rounding of the result to D's type, with n the number of
    accumulated terms and the unit roundoff of the product's arithmetic
    (2^-24 binary32, 2^-53 binary64). 16-bit precisions round their operands
    exactly as the oracle does, so the same bound applies.
Elements of D's buffer that the layout does not address must be untouched.
"""
import numpy as np
import pytest

import tapp_b200
from tapp_b200.case import bf16_to_f32
from families import family_cases, random_case, bounded_case
from helpers import case_from_record, golden_records, error_bound, d_values, run_on_device, folded_sizes

pytestmark = pytest.mark.gpu


def check_against_f64(tapp, oracle, case, device=False, executor=None, extra_rel=0.0):
    ref = case.copy()
    err64, D64, scale = oracle.execute_f64(ref)
    assert err64 == 0
    run = case.copy()
    err = run_on_device(tapp, run, executor) if device else run.run(tapp, executor=executor)
    assert err == 0, (case.name, err, tapp.explain(err))
    got = d_values(run.D)
    bound = error_bound(case, scale, D64, extra_rel)
    bad = np.abs(got - D64) > bound
    assert not bad.any(), (case.name, int(bad.sum()), got[bad][:4], D64[bad][:4], bound[bad][:4])
    return run


RECORDS = [r for r in golden_records() if r["error"] == 0]


@pytest.mark.parametrize("device", [False, True], ids=["host_ptrs", "device_ptrs"])
@pytest.mark.parametrize("rec", RECORDS, ids=lambda r: f"{r['program']}#{r['call']}")
def test_reference_programs(tapp, oracle, gpu, rec, device):
    """The reference's example programs' products reproduce the reference's
    recorded D (within the binary32/64 bound)."""
    case, after = case_from_record(rec)
    run = check_against_f64(tapp, oracle, case, device=device)
    got = d_values(run.D)[:after.size]
    want = after.astype(np.complex128)
    _, D64, scale = oracle.execute_f64(case.copy())
    bound = 2 * error_bound(case, scale, D64)[:after.size]
    assert (np.abs(got - want) <= bound).all()


def test_reference_program_errors_propagate(tapp, gpu):
    for rec in golden_records():
        if rec["error"]:
            case, _ = case_from_record(rec)
            assert case.run(tapp) == rec["error"]


@pytest.mark.parametrize("prec", [-1, 0, 1, 4, 5, 6])
def test_families(tapp, oracle, gpu, prec):
    n = 0
    for fam, case in family_cases(2000 + prec, 2):
        case.prec = prec
        check_against_f64(tapp, oracle, case, device=(n % 2 == 1))
        n += 1
    assert n > 30


@pytest.mark.parametrize("prec", [-1, 0, 1, 5, 6])
def test_mixed_and_half_storage(tapp, oracle, gpu, prec):
    rng = np.random.default_rng(40 + prec)
    type_sets = [(0, 1, 0, 1), (1, 0, 1, 0), (2, 3, 2, 3), (3, 2, 2, 2), (0, 2, 0, 2), (4, 4, 4, 4),
                 (5, 5, 0, 0), (4, 0, 4, 0), (5, 5, 5, 5), (0, 0, 4, 4)]
    for types in type_sets:
        if prec != -1 and types[0] in (0, 1, 4, 5) and types[1] in (2, 3):
            continue
        for i in range(3):
            case = random_case(rng, types=types, prec=prec, n_isoA=i % 2, n_repA=(i // 2) % 2,
                               subtensor=True, mixed=(i == 2))
            check_against_f64(tapp, oracle, case, device=bool(i % 2))


def test_dense_contraction_config(tapp, oracle, gpu):
    """D[a,b,c,d] = 1.3 sum_{e,f} A[a,e,b,f] B[f,c,e,d] + 0.7 C, all extents 16, float32."""
    from tapp_b200.workloads import dense_contraction_case
    case = dense_contraction_case(np.random.default_rng(1), extent=16)
    check_against_f64(tapp, oracle, case, device=True)
    check_against_f64(tapp, oracle, case, device=False)


def test_mixed_classes_config(tapp, oracle, gpu):
    """Hadamard h, diagonal k, unary u (stride 0) and v, conj(B), negative
    stride, permuted D; complex float, default precision."""
    from tapp_b200.workloads import mixed_classes_case
    case = mixed_classes_case(np.random.default_rng(2))
    check_against_f64(tapp, oracle, case, device=True)
    check_against_f64(tapp, oracle, case, device=False)


def test_empty_extents_leave_D_untouched(tapp, oracle, gpu):
    """A zero extent on a free label: nothing to write, D stays as it was."""
    rng = np.random.default_rng(3)
    case = random_case(rng, dtype=0, n_contracted=1, n_freeA=1, n_freeB=1, n_hadamard=0)
    lab = case.D.idx[0]
    for t in (case.A, case.B, case.C, case.D):
        for j, l in enumerate(t.idx):
            if l == lab:
                t.extents[j] = 0
    before = case.D.buf.copy()
    assert case.run(tapp) == 0
    assert np.array_equal(before, case.D.buf)


def test_zero_extent_contraction_gives_beta_C(tapp, oracle, gpu):
    rng = np.random.default_rng(4)
    case = random_case(rng, dtype=1, n_contracted=1, n_freeA=1, n_freeB=1, n_hadamard=0, min_ext=2)
    k = [l for l in case.A.idx if l in case.B.idx][0]
    case.A.extents[case.A.idx.index(k)] = 0
    case.B.extents[case.B.idx.index(k)] = 0
    check_against_f64(tapp, oracle, case)


def test_C_equals_D_in_place(tapp, oracle, gpu):
    rng = np.random.default_rng(5)
    case = random_case(rng, dtype=0, n_contracted=2, n_freeA=2, n_freeB=1)
    case.C = case.D  # same buffer and layout
    ref = case.copy()
    ref.C = ref.D
    _, D64, scale = oracle.execute_f64(ref)
    assert case.run(tapp) == 0
    assert (np.abs(d_values(case.D) - D64) <= error_bound(case, scale, D64)).all()


def test_beta_zero_with_null_C(tapp, oracle, gpu):
    rng = np.random.default_rng(6)
    for dt in (0, 1, 2, 3):
        case = random_case(rng, dtype=dt, beta_zero=True, C_null=True, n_contracted=1)
        check_against_f64(tapp, oracle, case)


def test_zero_and_negative_strides(tapp, oracle, gpu):
    rng = np.random.default_rng(7)
    for i in range(12):
        case = random_case(rng, dtype=i % 4, zero_stride="AB"[i % 2], neg=bool(i % 3 == 0),
                           mixed=bool(i % 3 == 1), subtensor=True, n_contracted=2)
        check_against_f64(tapp, oracle, case, device=bool(i % 2))


def test_larger_random_products(tapp, oracle, gpu):
    rng = np.random.default_rng(8)
    for i in range(8):
        case = bounded_case(rng, dtype=i % 4, n_contracted=2, n_freeA=2, n_freeB=2, n_hadamard=i % 2,
                            min_ext=5, max_ext=12, subtensor=bool(i % 2), mixed=bool(i % 3 == 0),
                            n_isoA=int(i == 5), n_isoB=int(i == 6))
        check_against_f64(tapp, oracle, case, device=True)


def test_long_contraction_reduce_path(tapp, oracle, gpu):
    """Few outputs, long contraction: one block per output."""
    rng = np.random.default_rng(9)
    for dt in (0, 1, 2, 3):
        case = random_case(rng, dtype=dt, n_contracted=3, n_freeA=1, n_freeB=0, n_hadamard=0,
                           ext_choices=[16, 20, 24])
        run = check_against_f64(tapp, oracle, case, device=True)
        K, _, _ = folded_sizes(case)
        assert K >= 4096


def test_status_object(tapp, gpu):
    from tapp_b200.workloads import dense_contraction_case
    import ctypes as C
    case = dense_contraction_case(np.random.default_rng(1), extent=8)
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(),
                                        case.beta.ctypes.data, case.C.ptr(), case.D.ptr())
    assert err == 0 and st.value != 0
    assert tapp.status_value(st.value, tapp_b200.STATUS_KERNELS) >= 1
    assert tapp.status_value(st.value, tapp_b200.STATUS_FLOPS) == 2.0 * 8 ** 4 * 8 ** 2
    assert tapp.status_value(st.value, tapp_b200.STATUS_DEVICE_US) > 0
    assert tapp.lib.TAPP_destroy_status(st.value) == 0
    tapp.lib.TAPP_destroy_executor(ex)


def test_batched_product_matches_single(tapp, oracle, gpu):
    import ctypes as C
    import torch
    from tapp_b200.workloads import dense_contraction_case
    rng = np.random.default_rng(10)
    cases = [dense_contraction_case(rng, extent=6) for _ in range(5)]
    c0 = cases[0]
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (c0.A, c0.B, c0.C, c0.D)]
    _, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [c0.A.idx, c0.B.idx, c0.C.idx, c0.D.idx], c0.prec)
    dev = []
    arrs = {k: (C.c_void_p * 5)() for k in "ABCD"}
    for i, c in enumerate(cases):
        for k in "ABCD":
            t = getattr(c, k)
            x = torch.from_numpy(t.buf.view(np.uint8).copy()).cuda()
            dev.append((k, i, x, t))
            arrs[k][i] = x.data_ptr() + t.base * t.itemsize
    ex = tapp.create_executor()
    err = tapp.lib.TAPP_execute_batched_product(plan, ex, None, 5, c0.alpha.ctypes.data, arrs["A"], arrs["B"],
                                                c0.beta.ctypes.data, arrs["C"], arrs["D"])
    torch.cuda.synchronize()
    assert err == 0
    for k, i, x, t in dev:
        if k == "D":
            got = x.cpu().numpy().view(t.buf.dtype).astype(np.complex128)
            _, D64, scale = oracle.execute_f64(cases[i].copy())
            assert (np.abs(got - D64) <= error_bound(cases[i], scale, D64)).all()
    tapp.lib.TAPP_destroy_executor(ex)


def _run_with_status(tapp, case, ex):
    import ctypes as C
    import torch
    dev = [torch.from_numpy(t.buf.view(np.uint8).copy()).cuda() for t in (case.A, case.B, case.C, case.D)]
    ptr = [d.data_ptr() + t.base * t.itemsize for d, t in zip(dev, (case.A, case.B, case.C, case.D))]
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), case.alpha.ctypes.data, ptr[0], ptr[1],
                                        case.beta.ctypes.data, None if case.C_is_null else ptr[2], ptr[3])
    assert err == 0
    bound = tapp.status_value(st.value, tapp_b200.STATUS_ERR_BOUND)
    tapp.lib.TAPP_destroy_status(st.value)
    case.D.buf[:] = dev[3].cpu().numpy().view(case.D.buf.dtype)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    return bound


@pytest.mark.parametrize("label", ["plain_f32", "bf16_tc", "split_bf16", "f64", "c32_generic"])
def test_status_error_bound_holds(tapp, oracle, gpu, label):
    """The error bound a status reports covers the measured error against
    the binary64 evaluation of the (precision-rounded) operands."""
    from tapp_b200.workloads import large_dense_case, dense_contraction_case
    rng = np.random.default_rng(300)
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    if label == "plain_f32":
        case = dense_contraction_case(rng, extent=16)
    elif label == "bf16_tc":
        case = large_dense_case(rng, 6, 0, extent=16)
    elif label == "split_bf16":
        case = large_dense_case(rng, 0, 0, extent=16)
        tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, 1)
    elif label == "f64":
        case = dense_contraction_case(rng, extent=12, dtype=1, prec=1)
    else:
        case = bounded_case(rng, dtype=2, prec=-1, n_contracted=2, n_freeA=1, n_freeB=1, n_isoA=1, max_ext=6)
    run = case.copy()
    bound = _run_with_status(tapp, run, ex)
    _, D64, scale = oracle.execute_f64(case.copy())
    got = d_values(run.D)
    u_d = 2.0 ** -53 if run.D.dtype in (1, 3) else 2.0 ** -24
    assert 0 < bound < 1e-2
    assert (np.abs(got - D64) <= bound * scale + 2 * u_d * np.abs(D64) + 1e-300).all()
    tapp.lib.TAPP_destroy_executor(ex)

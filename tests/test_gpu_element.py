"""GPU parity of the element path's warp-per-output kernel (k_warpdot):
products whose contraction runs along an operand's contiguous mode while
consecutive outputs step that operand by a whole row (batched
matrix-vector and Hadamard products with A stored contraction-fastest).
Each case checks the kernel choice in the plan description, the result
against the oracle's binary64 bound, and that two runs give the same bits.
"""
import numpy as np
import pytest

import tapp_b200
from tapp_b200.case import Case, alloc, fill_uniform, scalar
from helpers import run_on_device, error_bound, d_values

pytestmark = pytest.mark.gpu


def _t(rng, dtype, ext, idx, order):
    strides = [0] * len(ext)
    acc = 1
    for i in order:
        strides[i] = acc
        acc *= ext[i]
    return fill_uniform(alloc(dtype, ext, strides, [ord(c) for c in idx]), rng)


def _matvec(rng, dtype, prec, k=300, m=70, h=9, unary=0, conj=False):
    """D[m,h] = alpha sum_k (sum_u A[k,m,h,u]) B[k,h] + beta C, A contiguous along k."""
    if unary:
        A = _t(rng, dtype, [k, m, h, unary], "kmhu", [0, 1, 2, 3])
    else:
        A = _t(rng, dtype, [k, m, h], "kmh", [0, 1, 2])
    B = _t(rng, dtype, [k, h], "kh", [0, 1])
    if conj:
        B.op = tapp_b200.TAPP_CONJUGATE
    Cc = _t(rng, dtype, [m, h], "mh", [0, 1])
    D = _t(rng, dtype, [m, h], "mh", [0, 1])
    cplx = dtype in (tapp_b200.TAPP_C32, tapp_b200.TAPP_C64)
    al = complex(0.8, -0.3) if cplx else 0.8
    be = complex(-0.4, 0.2) if cplx else -0.4
    return Case(A, B, Cc, D, scalar(dtype, al), scalar(dtype, be), prec, False, "matvec")


CASES = [
    ("f32", tapp_b200.TAPP_F32, 0, {}),
    ("f64", tapp_b200.TAPP_F64, 1, {}),
    ("c32_conj", tapp_b200.TAPP_C32, -1, {"conj": True}),
    ("f32_unary", tapp_b200.TAPP_F32, -1, {"unary": 3}),
    ("bf16_prec", tapp_b200.TAPP_F32, tapp_b200.TAPP_BF16BF16_ACCUM_F32, {"k": 97}),
]


def _describe(tapp, case):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    d = tapp.describe(plan)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        tapp.lib.TAPP_destroy_tensor_info(h)
    return d


@pytest.mark.parametrize("name,dtype,prec,kw", CASES, ids=[c[0] for c in CASES])
def test_warpdot(tapp, oracle, gpu, name, dtype, prec, kw):
    case = _matvec(np.random.default_rng(len(name) * 7 + dtype), dtype, prec, **kw)
    d = _describe(tapp, case)
    assert "path=generic" in d and "kernel=warpdot" in d, d
    runs = []
    for _ in range(2):
        run = case.copy()
        assert run_on_device(tapp, run) == 0
        runs.append(run)
    assert np.array_equal(runs[0].D.buf.view(np.uint8), runs[1].D.buf.view(np.uint8))
    e64, D64, scale = oracle.execute_f64(case.copy())
    assert e64 == 0
    bound = error_bound(case, scale, D64)
    bad = np.abs(d_values(runs[0].D) - D64) > bound
    assert not bad.any(), (name, int(bad.sum()))


def _hadamard(rng, d_order, ext=(72, 8, 20, 30, 16)):
    """D[l3,l2,l1,l0] = 0.9 sum_k A[l0,l1,k,l2,l3] B[l2,k,l0,l1] - 0.3 C (the
    served mix's batched matrix-vector Hadamard kind): A contiguous along l0;
    D's modes stored in the order d_order (labels)."""
    e0, e1, ek, e2, e3 = ext
    A = _t(rng, tapp_b200.TAPP_F32, [e0, e1, ek, e2, e3], "abkcd", [0, 1, 2, 3, 4])
    B = _t(rng, tapp_b200.TAPP_F32, [e2, ek, e0, e1], "ckab", [0, 1, 2, 3])
    ext_of = {"a": e0, "b": e1, "c": e2, "d": e3}
    idx = "".join(d_order)
    Cc = _t(rng, tapp_b200.TAPP_F32, [ext_of[c] for c in idx], idx, list(range(4)))
    D = _t(rng, tapp_b200.TAPP_F32, [ext_of[c] for c in idx], idx, list(range(4)))
    return Case(A, B, Cc, D, scalar(tapp_b200.TAPP_F32, 0.9), scalar(tapp_b200.TAPP_F32, -0.3), 0, False, "hadamard")


def _logical(t, order):
    """t's values as an array indexed in the label order `order`."""
    import itertools
    pos = {c: i for i, c in enumerate("".join(chr(x) for x in t.idx))}
    out = np.empty([t.extents[pos[c]] for c in order], dtype=t.buf.dtype)
    for coords in itertools.product(*[range(n) for n in out.shape]):
        off = t.base + sum(coords[k] * t.strides[pos[c]] for k, c in enumerate(order))
        out[coords] = t.buf[off]
    return out


def test_element_path_walks_the_larger_operand(tapp, oracle, gpu):
    """Outputs walked in A's stride order (A contiguous along a batch mode, D
    along another): within the oracle bound, and bit-identical to the same
    product with D stored in A's order (outputs walked in D's order)."""
    ext = (72, 8, 6, 10, 5)
    walked = _hadamard(np.random.default_rng(91), "dcba", ext)
    plain = _hadamard(np.random.default_rng(91), "abcd", ext)
    # the same values in both (A and B are drawn alike; C copied in logical order)
    plain.C.buf[plain.C.base + plain.C.offsets()] = _logical(walked.C, "abcd").reshape(-1, order="F")
    assert "kernel=element" in _describe(tapp, walked) and " F=[(72:1," in _describe(tapp, walked)
    runs = {}
    for name, case in (("walked", walked), ("plain", plain)):
        run = case.copy()
        assert run_on_device(tapp, run) == 0
        runs[name] = _logical(run.D, "abcd")
    assert np.array_equal(runs["walked"].view(np.uint8), runs["plain"].view(np.uint8))
    e64, D64, scale = oracle.execute_f64(walked.copy())
    assert e64 == 0
    run = walked.copy()
    assert run_on_device(tapp, run) == 0
    bound = error_bound(walked, scale, D64)
    assert not (np.abs(d_values(run.D) - D64) > bound).any()


def test_small_grid_runs_a_warp_per_output(tapp, oracle, gpu):
    """The mixed-class complex product (17,280 outputs, less than a wave of
    threads; 24 diagonal terms with unary sums of 6 and 5 values each): one
    warp per output, lanes over the terms. Within the oracle bound, and the
    same bits in two runs."""
    from tapp_b200.workloads import mixed_classes_case
    case = mixed_classes_case(np.random.default_rng(0x7A990002))
    assert "kernel=warpdot" in _describe(tapp, case)
    runs = []
    for _ in range(2):
        run = case.copy()
        assert run_on_device(tapp, run) == 0
        runs.append(run)
    assert np.array_equal(runs[0].D.buf.view(np.uint8), runs[1].D.buf.view(np.uint8))
    e64, D64, scale = oracle.execute_f64(case.copy())
    assert e64 == 0
    bound = error_bound(case, scale, D64)
    assert not (np.abs(d_values(runs[0].D) - D64) > bound).any()


def test_element_path_stages_the_small_operand(tapp, oracle, gpu):
    """Batched Hadamard product whose small operand B would be read 600
    elements apart by consecutive outputs: B is first copied into the order
    of the output walk (plan: staged=B). Within the oracle bound, and the same
    bits as the grouped element launch of a batched product, which reads B in
    place."""
    from test_gpu_tc import _batched_against_single
    case = _hadamard(np.random.default_rng(93), "dcba", (72, 8, 20, 30, 16))
    d = _describe(tapp, case)
    assert "kernel=element staged=B" in d, d
    run = case.copy()
    assert run_on_device(tapp, run) == 0
    e64, D64, scale = oracle.execute_f64(case.copy())
    assert e64 == 0
    bound = error_bound(case, scale, D64)
    assert not (np.abs(d_values(run.D) - D64) > bound).any()
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    _batched_against_single(tapp, [case, case.copy()], ex)
    tapp.lib.TAPP_destroy_executor(ex)

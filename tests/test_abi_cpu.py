"""Host-side behaviour of the B200 library, without a GPU.

Everything that happens before the first CUDA call is checked here against
the reference's codes: tensor-info creation, the validation chain and its
precedence, the executor check, error texts, attributes and the planner's
index classification. The library must load, and export every entry point
its headers declare.
"""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import tapp_b200
from tapp_b200.case import alloc, scalar, Case
from helpers import GOLDEN
from families import random_case

INCLUDE = tapp_b200.INCLUDE_DIR


def declared_symbols():
    names = set()
    for root, _, files in os.walk(INCLUDE):
        for fn in files:
            if fn.endswith(".h"):
                src = open(os.path.join(root, fn)).read()
                names |= set(re.findall(r"TAPP_EXPORT[^;]*?\b((?:TAPP|tapp_b200)_\w+)\s*\(", src, re.S))
    return names


def test_library_loads_and_exports_every_declared_symbol(tapp):
    names = declared_symbols()
    assert len(names) >= 24
    for n in sorted(names):
        assert hasattr(tapp.lib, n), n


def test_exports_match_reference_abi(tapp):
    """Every entry point the reference exports (its symbol table; the API
    part of it) is exported here with the same name."""
    ref_api = ["TAPP_check_success", "TAPP_create_executor", "TAPP_create_handle", "TAPP_create_tensor_info",
               "TAPP_create_tensor_product", "TAPP_destroy_executor", "TAPP_destroy_handle",
               "TAPP_destroy_tensor_info", "TAPP_destroy_tensor_product", "TAPP_execute_product",
               "TAPP_explain_error", "TAPP_get_extents", "TAPP_get_nmodes", "TAPP_get_strides",
               "TAPP_set_extents", "TAPP_set_nmodes", "TAPP_set_strides"]
    for n in ref_api:
        assert hasattr(tapp.lib, n)


def test_tensor_info_codes(tapp):
    err, _ = tapp.tensor_info(0, [2, 3], [1, 2])
    assert err == 0
    h = C.c_ssize_t(0)
    assert tapp.lib.TAPP_create_tensor_info(C.byref(h), 0, -1, None, None) == 14
    assert tapp.tensor_info(0, [2, -1], [1, 2])[0] == 15
    err, info = tapp.tensor_info(1, [4, 5, 6], [1, 4, 20])
    assert tapp.lib.TAPP_get_nmodes(info) == 3
    e = (C.c_int64 * 3)()
    s = (C.c_int64 * 3)()
    tapp.lib.TAPP_get_extents(info, e)
    tapp.lib.TAPP_get_strides(info, s)
    assert list(e) == [4, 5, 6] and list(s) == [1, 4, 20]
    assert tapp.lib.TAPP_set_extents(info, tapp.i64([1, -2, 3])) == 15
    tapp.lib.TAPP_get_extents(info, e)
    assert list(e) == [4, 5, 6]
    assert tapp.lib.TAPP_set_nmodes(info, -3) == 14
    assert tapp.lib.TAPP_set_nmodes(info, 2) == 0
    assert tapp.lib.TAPP_get_nmodes(info) == 2
    assert tapp.lib.TAPP_set_strides(info, tapp.i64([7, 8])) == 0
    tapp.lib.TAPP_get_strides(info, s)
    assert list(s)[:2] == [7, 8]
    assert tapp.lib.TAPP_destroy_tensor_info(info) == 0


def test_explain_error_texts_match_reference(tapp):
    with open(os.path.join(GOLDEN, "explain_error.json")) as f:
        texts = json.load(f)
    for code, text in texts.items():
        assert tapp.explain(int(code)) == text
    # truncation and measuring (error.h:15-23)
    n = tapp.lib.TAPP_explain_error(8, 0, None)
    assert n == len(texts["8"])
    buf = C.create_string_buffer(10)
    w = tapp.lib.TAPP_explain_error(8, 5, buf)
    assert w == 4 and buf.value.decode() == texts["8"][:4]
    for code in (15, 33, 137, tapp_b200.ERR_CUDA, 12345):
        assert len(tapp.explain(code)) > 0
    assert tapp.lib.TAPP_check_success(0) and not tapp.lib.TAPP_check_success(3)


def _case_from_spec(c):
    ts = [alloc(0, t["extents"], t["strides"], t["idx"]) for t in c["tensors"]]
    return Case(*ts, scalar(0, 1.0), scalar(0, c["beta"]), -1, c["C_null"])


def test_validation_codes_match_reference_fixture(tapp):
    with open(os.path.join(GOLDEN, "error_cases.json")) as f:
        cases = json.load(f)
    checked = 0
    for c in cases:
        if c["expected"] == 0:
            continue
        case = _case_from_spec(c)
        assert case.run(tapp) == c["expected"], c
        checked += 1
    assert checked > 300


def test_validation_matches_oracle_on_random_products(tapp, oracle):
    rng = np.random.default_rng(5)
    for i in range(300):
        case = random_case(rng, dtype=int(rng.integers(0, 4)), n_contracted=int(rng.integers(0, 3)),
                           n_repA=int(rng.integers(0, 2)), n_repB=int(rng.integers(0, 2)),
                           n_repD=int(rng.integers(0, 2)))
        t = [case.A, case.B, case.C, case.D][int(rng.integers(0, 4))]
        if t.nmode and rng.random() < 0.7:
            j = int(rng.integers(0, t.nmode))
            what = rng.integers(0, 3)
            if what == 0:
                t.extents[j] += 1
            elif what == 1:
                t.strides[j] = 0
            else:
                t.idx[j] = int(rng.integers(0, 10**6))
            t.buf = np.zeros(10**4, dtype=t.buf.dtype)
            t.base = 5000
        want = oracle.validate(case)
        if want == 0:
            continue
        assert case.run(tapp) == want


def test_executor_check(tapp):
    case = _case_from_spec({"beta": 0.0, "C_null": False, "tensors": [
        {"extents": [2], "strides": [1], "idx": [1]}, {"extents": [2], "strides": [1], "idx": [1]},
        {"extents": [], "strides": [], "idx": []}, {"extents": [], "strides": [], "idx": []}]})
    assert case.run(tapp, executor=0) == 33  # NULL executor (product.c:878-885)
    bogus = C.c_int(7)
    assert case.run(tapp, executor=C.addressof(bogus)) == 33
    foreign = C.c_int(1)  # a bare int 1, as the reference's demo.c comments suggest
    err = case.run(tapp, executor=C.addressof(foreign))
    assert err in (0, tapp_b200.ERR_CUDA)


def test_executor_attributes(tapp):
    ex = tapp.create_executor()
    assert C.c_int.from_address(ex).value == 1  # reference executor id first
    assert tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, 1) == 0
    box = C.c_int(0)
    p = C.c_void_p(C.addressof(box))
    assert tapp.lib.TAPP_attr_get(ex, tapp_b200.ATTR_F32_MODE, C.byref(p)) == 0 and box.value == 1
    assert tapp.lib.TAPP_attr_clear(ex, tapp_b200.ATTR_F32_MODE) == 0
    assert tapp.lib.TAPP_attr_get(ex, tapp_b200.ATTR_F32_MODE, C.byref(p)) == 0 and box.value == 0
    assert tapp.set_int(ex, 0x7777, 1) == tapp_b200.ERR_INVALID
    assert tapp.lib.TAPP_attr_set(12345, tapp_b200.ATTR_ASYNC, None) == tapp_b200.ERR_INVALID
    tapp.lib.TAPP_destroy_executor(ex)


def _plan(tapp, case):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    err, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                    [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    return plan, infos


def test_planner_classification_config_mixed_classes(tapp):
    """The mixed index-class product D[a,h,c] = sum_{k,u,v} A[a,h,k,k,u] conj(B[k,h,c,v])
    classifies h as batch, a as M, c as N, the repeated k as one contracted mode
    with summed stride, u as unary-A (stride 0) and v as unary-B."""
    from tapp_b200.workloads import mixed_classes_case
    case = mixed_classes_case(np.random.default_rng(0))
    plan, infos = _plan(tapp, case)
    d = tapp.describe(plan)
    assert "compute=c32" in d and "conj=0100" in d
    ua = re.search(r" UA=\[(.*?)\]", d).group(1)
    ub = re.search(r" UB=\[(.*?)\]", d).group(1)
    k = re.search(r" K=\[(.*?)\]", d).group(1)
    assert ua.startswith("(6:0,") and ub.startswith("(5:")
    a = case.A
    kstride = sum(s for s, l in zip(a.strides, a.idx) if l == ord("k"))
    assert k.startswith(f"(24:{kstride},")
    assert re.search(r" L=\[\(12:", d) and re.search(r" M=\[\(40:", d) and re.search(r" N=\[\(36:", d)


def test_planner_dense_contraction_modes(tapp):
    """All-16 dense contraction D[a,b,c,d] = sum_{e,f} A[a,e,b,f] B[f,c,e,d]:
    a,b are M (absent from B), c,d are N; no pair is contiguous in every
    tensor that holds it (e sits between a and b in A, and between c and d
    in B), so nothing merges. A is contiguous along a free mode (a) and B
    along a contracted one (f), so the contracted modes follow B's strides:
    K = (f, e) with strides (4096, 16) in A and (1, 256) in B."""
    from tapp_b200.workloads import dense_contraction_case
    case = dense_contraction_case(np.random.default_rng(0), extent=16, dtype=0)
    plan, infos = _plan(tapp, case)
    d = tapp.describe(plan)
    assert " M=[(16:1,0,1,1),(16:256,0,16,16)]" in d, d
    assert " N=[(16:0,16,256,256),(16:0,4096,4096,4096)]" in d, d
    assert " K=[(16:4096,1,0,0),(16:16,256,0,0)]" in d, d
    assert " L=[]" in d and " UA=[]" in d


def test_planner_merges_contiguous_modes(tapp):
    """A plain matrix product written with split modes: D[a,b,c] = sum_k
    A[a,b,k] B[k,c] with A, C, D dense column-major: (a, b) is contiguous in
    A, C and D and merges into one M mode of 12."""
    A = alloc(0, [3, 4, 5], [1, 3, 12], [1, 2, 9])
    B = alloc(0, [5, 6], [1, 5], [9, 3])
    Cc = alloc(0, [3, 4, 6], [1, 3, 12], [1, 2, 3])
    D = alloc(0, [3, 4, 6], [1, 3, 12], [1, 2, 3])
    case = Case(A, B, Cc, D, scalar(0, 1.0), scalar(0, 1.0), -1)
    plan, infos = _plan(tapp, case)
    d = tapp.describe(plan)
    assert " M=[(12:1,0,1,1)]" in d, d
    assert " N=[(6:0,5,12,12)]" in d, d
    assert " K=[(5:12,1,0,0)]" in d, d


@pytest.mark.parametrize("dims,path", [
    # D[a,h] = sum_{b,c,e} A[a,b,c,h,e] B[e,b,h,c]: 4565 outputs x 17,172 terms
    (([55, 54, 53, 83, 6], [6, 54, 83, 53], [55, 83]), "reduce"),
    # 666 outputs x 5160 terms
    (([18, 86, 37, 60], [86, 60, 37], [18, 37]), "reduce"),
    # D[a,h] = sum_k A[a,k,h] B[k,h]: 31 x 1794 outputs x 3634 terms (batched matrix-vector)
    (([31, 3634, 1794], [3634, 1794], [31, 1794]), "reduce"),
    # 200 x 40 outputs x 30 terms: short contractions stay one thread per output
    (([200, 30, 40], [30, 40], [200, 40]), "generic"),
])
def test_planner_long_contraction_few_outputs(tapp, dims, path):
    """Hadamard products with few outputs for one thread each and a long
    contraction take the block-per-output reduction path."""
    from tapp_b200.workloads import colmajor
    ea, eb, ed = dims
    if len(ea) == 5:
        ia, ib, idd = [0, 1, 2, 3, 4], [4, 1, 3, 2], [0, 3]
    elif len(ea) == 4:
        ia, ib, idd = [0, 1, 2, 3], [1, 3, 2], [0, 2]
    else:
        ia, ib, idd = [0, 1, 2], [1, 2], [0, 2]
    ts = [alloc(0, e, colmajor(e), i) for e, i in ((ea, ia), (eb, ib), (ed, idd), (ed, idd))]
    case = Case(*ts, scalar(0, 1.0), scalar(0, 1.0), -1)
    plan, infos = _plan(tapp, case)
    assert f"path={path}" in tapp.describe(plan), tapp.describe(plan)
    tapp.lib.TAPP_destroy_tensor_product(plan)


def test_wait_selftest_argument_checks(tapp):
    """tapp_b200_selftest_waits refuses NULL outputs and limits outside
    (0, 10 s] before touching a device."""
    f = tapp.lib.tapp_b200_selftest_waits
    f.restype = C.c_int
    f.argtypes = [C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    a, b = C.c_int(0), C.c_int(0)
    assert f(100.0, None, C.byref(b)) == tapp_b200.ERR_INVALID
    assert f(100.0, C.byref(a), None) == tapp_b200.ERR_INVALID
    for bad in (0.0, -1.0, 1e9, float("nan")):
        assert f(bad, C.byref(a), C.byref(b)) == tapp_b200.ERR_INVALID


@pytest.mark.parametrize("core,mode,rank,storage,prec,kernel", [
    ([64, 40, 32, 32], 1, 38, 0, 0, "narrow_vec"),        # rows contiguous in A, C and D: 4-row vectors
    ([62, 40, 32, 32], 1, 38, 0, 0, "narrow_vec"),        # row extent even: 2-row vectors
    ([63, 40, 32, 32], 1, 38, 0, 0, "narrow_stream"),     # odd row extent: a row per thread
    ([64, 40, 32, 32], 0, 38, 0, 0, "narrow_kt"),         # A along the contraction in 16-byte runs
    ([62, 40, 32, 32], 0, 38, 0, 0, "narrow_coop"),       # A along the contraction, D along the rank
    ([64, 40, 32, 32], 0, 8, 0, 0, "narrow_coop"),        # too narrow for the register tiles
    ([64, 40, 32, 32], 1, 24, 0, 6, "narrow_vec"),        # bf16 precision: rounding after the copy
    ([63, 40, 32, 32], 1, 24, 0, 6, "narrow_stream"),
    ([64, 40, 32, 32], 1, 24, 1, -1, "narrow_vec"),       # binary64, rows contiguous
    ([63, 40, 32, 32], 1, 24, 1, -1, "narrow_stream"),
    ([64, 40, 32, 32], 0, 38, 1, -1, "narrow"),           # binary64 with D along the rank
    ([64, 40, 32, 32], 1, 60, 1, -1, "narrow_vec"),       # binary64 wider than 48
    ([63, 40, 32, 32], 1, 60, 1, -1, "narrow"),
    ([64, 40, 32, 32], 1, 24, 2, -1, "narrow_cvec"),      # complex float, rows in 2-row vectors
    ([63, 40, 32, 32], 1, 24, 2, -1, "narrow_cstream"),   # complex float, odd row extent
    ([64, 40, 32, 32], 1, 24, 3, -1, "tiled"),            # complex double
])
def test_planner_reports_the_cuda_core_kernel(tapp, core, mode, rank, storage, prec, kernel):
    """tapp_b200_describe_plan names the CUDA-core kernel a mode-n product of
    the simt path runs, from its layout, types and width."""
    from tapp_b200.workloads import RequestSpec, case_from_spec
    o = len(core)
    d_ext = list(core)
    d_ext[mode] = rank
    d_idx = list(range(o))
    d_idx[mode] = o
    case = case_from_spec(np.random.default_rng(0), RequestSpec("tucker", storage, prec, (core, [rank, core[mode]], d_ext, d_ext),
                                                                (list(range(o)), [o, mode], d_idx, d_idx), 0.7, 0.3))
    plan, infos = _plan(tapp, case)
    d = tapp.describe(plan)
    assert "path=simt" in d and f" kernel={kernel} " in d, d
    tapp.lib.TAPP_destroy_tensor_product(plan)


def test_planner_reports_tiled_kernel_for_wide_products(tapp):
    A = alloc(0, [512, 256], [1, 512], [0, 2])
    B = alloc(0, [256, 384], [1, 256], [2, 1])
    Cc = alloc(0, [512, 384], [1, 512], [0, 1])
    D = alloc(0, [512, 384], [1, 512], [0, 1])
    plan, infos = _plan(tapp, Case(A, B, Cc, D, scalar(0, 1.0), scalar(0, 1.0), 0))
    assert " kernel=tiled " in tapp.describe(plan)
    tapp.lib.TAPP_destroy_tensor_product(plan)


def test_element_path_walks_the_larger_operand(tapp):
    """Element-path Hadamard product whose A (5x D's size) is contiguous along
    a batch mode while D is contiguous along A's last free mode: the plan
    orders the outputs by A's strides (A's stride-1 mode first), so that
    consecutive threads read consecutive elements of A."""
    A = alloc(0, [8, 4, 5, 6, 7], [1, 8, 32, 160, 960], [0, 1, 4, 2, 3])
    B = alloc(0, [6, 5, 8, 4], [1, 6, 30, 240], [2, 4, 0, 1])
    Cc = alloc(0, [7, 6, 4, 8], [1, 7, 42, 168], [3, 2, 1, 0])
    D = alloc(0, [7, 6, 4, 8], [1, 7, 42, 168], [3, 2, 1, 0])
    plan, infos = _plan(tapp, Case(A, B, Cc, D, scalar(0, 1.0), scalar(0, 0.5), 0))
    d = tapp.describe(plan)
    assert "path=generic" in d and "kernel=element" in d, d
    assert " F=[(8:1,30," in d, d
    tapp.lib.TAPP_destroy_tensor_product(plan)

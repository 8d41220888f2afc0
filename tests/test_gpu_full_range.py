"""Inputs over the whole finite range of their type, on the GPU.

The reference's randomized tests draw tensor values, alpha and beta uniformly
over [-max, max] of the storage type (test/test.cpp:1088-1098, scalars at
:358-359), so almost every product of two operands overflows and the
outputs are infinities and NaNs. These tests run the same kind of inputs
through the CUDA library and through the reference itself (built from its
sources into oracle/_ref; the F16 build for the F16 precision, the oracle's
restatement for TAPP_BF16BF16_ACCUM_F32, which the reference cannot build)
and require per element of a real D:

  reference +-inf   the same signed infinity;
  reference NaN     NaN or an infinity. The reference rounds every product
                    before adding it, so two overflowing products of
                    opposite signs meet as +inf and -inf in a NaN. The
                    kernels' fused multiply-adds (and the tensor cores'
                    accumulation) keep a product exact until the sum is
                    rounded: +inf + (-1e76) stays +inf;
  reference finite  finite, within the reference's own relative tolerance
                    5e-5 (compare_tensors, test.cpp:238-265).

For a complex D the element (both parts) must be non-finite exactly where
the reference's is: the reference multiplies complex numbers with C99's
`*`, which recovers an infinity from some NaN results (C11 Annex G), so the
kind of non-finite value differs as well.

IEEE half storage is left out: its range keeps products finite in binary32,
and the overflow of the final rounding is then order-dependent, as for any
finite sum; the ordinary tests cover it with their error bounds.
"""
import numpy as np
import pytest

import oracle as oracle_mod
import tapp_b200
from tapp_b200.abi import TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_BF16
from tapp_b200.case import bf16_from_f32, is_complex
from tapp_b200.workloads import large_dense_case
from families import family_cases, bounded_case
from helpers import run_on_device, d_values
from test_gpu_simt import spec_case, describe

pytestmark = pytest.mark.gpu

TYPE_MAX = {TAPP_F32: float(np.finfo(np.float32).max), TAPP_C32: float(np.finfo(np.float32).max),
            TAPP_F64: float(np.finfo(np.float64).max), TAPP_C64: float(np.finfo(np.float64).max),
            TAPP_BF16: float(np.finfo(np.float32).max)}


def _uniform_full(rng, dtype, n):
    """n values uniform over [-max, max] of dtype (complex: each part)."""
    m = TYPE_MAX[dtype]
    if dtype in (TAPP_C32, TAPP_C64):
        return rng.uniform(-1, 1, n) * m + 1j * (rng.uniform(-1, 1, n) * m)
    v = rng.uniform(-1, 1, n) * m
    if dtype == TAPP_F32:
        return v.astype(np.float32)
    if dtype == TAPP_BF16:
        # values at the top of binary32's range round to infinity in
        # bfloat16: keep them below its largest finite value
        return bf16_from_f32((v * 0.99).astype(np.float32))
    return v


def full_range(case, rng):
    """The case with A, B, C, D (D's elements outside its layout included)
    and alpha, beta (beta = 0 kept) drawn over the full range."""
    c = case.copy()
    for t in (c.A, c.B, c.C, c.D):
        t.buf[:] = _uniform_full(rng, t.dtype, t.buf.size)
    tD = c.D.dtype
    c.alpha = c.alpha.copy()
    c.alpha[:] = _uniform_full(rng, tD, 1)
    beta = d_values_scalar(c.beta, tD)
    if beta != 0:
        c.beta = c.beta.copy()
        c.beta[:] = _uniform_full(rng, tD, 1)
    return c


def d_values_scalar(a, dtype):
    from tapp_b200.case import bf16_to_f32
    return complex(bf16_to_f32(a)[0]) if dtype == TAPP_BF16 else complex(a[0])


def _reference_for(case):
    """(library, name) that gives the reference's result for this case."""
    if case.prec == 6:
        return None, "oracle"
    ref = oracle_mod.reference_lib(f16=case.prec in (4, 5))
    if ref is None:
        pytest.skip("the reference was not built from its sources into oracle/_ref")
    return ref, "reference"


def check_classes(tapp, oracle, case, executor=None, device=True, want_path=None):
    if want_path is not None:
        ex = executor if executor is not None else tapp.create_executor()
        assert f"path={want_path}" in describe(tapp, case, ex), describe(tapp, case, ex)
        if executor is None:
            tapp.lib.TAPP_destroy_executor(ex)
    ref, _ = _reference_for(case)
    want_case = case.copy()
    if ref is None:
        assert oracle.execute(want_case) == 0
    else:
        assert want_case.run(ref) == 0
    run = case.copy()
    with np.errstate(all="ignore"):
        err = run_on_device(tapp, run, executor) if device else run.run(tapp, executor=executor)
        assert err == 0, (case.name, err, tapp.explain(err))
        got, want = d_values(run.D), d_values(want_case.D)
        if is_complex(case.D.dtype):
            fin_w = np.isfinite(want)
            assert (np.isfinite(got) == fin_w).all(), (case.name, int((np.isfinite(got) != fin_w).sum()))
        else:
            got, want = got.real, want.real
            fin_w = np.isfinite(want)
            inf = np.isinf(want)
            assert (got[inf] == want[inf]).all(), (case.name, "not the reference's infinity",
                                                   got[inf][got[inf] != want[inf]][:4])
            assert not np.isfinite(got[np.isnan(want)]).any(), (case.name, "finite where the reference has NaN")
            assert np.isfinite(got[fin_w]).all(), (case.name, "non-finite where the reference is finite")
        g, w = got[fin_w], want[fin_w]
        rel = np.abs(g - w) / np.maximum(np.abs(w), np.finfo(np.float64).tiny)
        assert (rel <= 5e-5).all(), (case.name, float(rel.max()))
    return int(fin_w.size - fin_w.sum())


@pytest.mark.parametrize("dtype", [TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64])
def test_full_range_families(tapp, oracle, gpu, dtype):
    """Every family of the randomized tests (Hadamard, contraction, outer,
    full contraction, zero- and one-mode, subtensors, negative and zero
    strides, unary and repeated indices, beta = 0 with C null) at the full
    range, on the kernels the planner picks; host pointers as the reference's
    callers pass them."""
    rng = np.random.default_rng(900 + dtype)
    nonfinite = 0
    for name, case in family_cases(910 + dtype, count_per_family=2, dtypes=(dtype,), max_ext=4):
        nonfinite += check_classes(tapp, oracle, full_range(case, rng), device=False)
    assert nonfinite > 0


@pytest.mark.parametrize("storage,prec", [(TAPP_F32, -1), (TAPP_F32, 0), (TAPP_F64, -1), (TAPP_C32, -1),
                                          (TAPP_C64, -1)])
def test_full_range_cuda_core_kernels(tapp, oracle, gpu, storage, prec):
    """The CUDA-core kernels past the element path: the tiled GEMM, the
    narrow (mode-n) kernels on each mode, the block-per-output reduction."""
    rng = np.random.default_rng(950 + storage * 7 + prec)
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_SIMT)
    case = bounded_case(rng, dtype=storage, prec=prec, n_contracted=2, n_freeA=1, n_freeB=1, n_hadamard=0,
                        ext_choices=[17, 40], max_work=2e6)
    check_classes(tapp, oracle, full_range(case, rng), executor=ex, want_path="simt")
    tapp.lib.TAPP_destroy_executor(ex)
    core = [101, 61, 43]
    for mode in range(3):
        d_ext = list(core)
        d_ext[mode] = 24
        d_idx = [0, 1, 2]
        d_idx[mode] = 3
        case = spec_case(rng, storage, prec, (core, [24, core[mode]], d_ext, d_ext),
                         ([0, 1, 2], [3, mode], d_idx, d_idx), "tucker")
        check_classes(tapp, oracle, full_range(case, rng), want_path="simt")
    case = spec_case(rng, storage, prec, ([30, 5, 40, 30], [30, 30, 40], [5], [5]),
                     ([0, 4, 1, 2], [2, 0, 1], [4], [4]))
    check_classes(tapp, oracle, full_range(case, rng), want_path="reduce")


@pytest.mark.parametrize("storage,prec", [(TAPP_F32, 6), (TAPP_F32, 5), (TAPP_BF16, 6)])
def test_full_range_tensor_cores(tapp, oracle, gpu, storage, prec):
    """The tensor-core GEMM under the 16-bit precisions: operands rounded to
    bfloat16 / half (out-of-range half operands become infinities), products
    accumulated in binary32 on the tensor cores."""
    rng = np.random.default_rng(980 + storage + prec)
    case = large_dense_case(rng, prec, storage=storage, extent=16)
    check_classes(tapp, oracle, full_range(case, rng), want_path="tc")

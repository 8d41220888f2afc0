"""The CUDA library against the reference itself, on the same seeded inputs.

The reference is built from its own sources into oracle/_ref (the default
build, and the F16 build for the 16-bit precisions). Each product runs
through both libraries' TAPP_execute_product; the codes must be equal and
every element of D within the sum of both results' rounding bounds from the
binary64 evaluation (gamma_n times the sum of term magnitudes, plus the
rounding to D's type: helpers.error_bound for the kernels' arithmetic,
reference_bound below for the reference's), so |D_gpu - D_ref| is bounded
element by element, not only each against binary64. Elements of D's buffer
outside its layout stay as they were in both. The cases are the test
families of the oracle's bit-exact pinning (tests/test_oracle_reference.py)
on the planner's own kernels, plus shapes that reach the tiled CUDA-core
GEMM, the narrow kernels and the reduction path.
"""
import itertools

import numpy as np
import pytest

import oracle as oracle_mod
import tapp_b200
from families import family_cases, random_case, bounded_case
from tapp_b200.abi import TAPP_F32, TAPP_C32, TAPP_F16, TAPP_BF16
from helpers import error_bound, d_values, run_on_device, folded_sizes, output_unit, UNIT
from test_gpu_simt import spec_case

pytestmark = pytest.mark.gpu

REF = oracle_mod.reference_lib()
REF16 = oracle_mod.reference_lib(f16=True)


def reference_bound(case, scale, D64):
    """Rounding bound of the reference's own arithmetic: error_bound with the
    unit roundoff of the narrowest type it computes in. Under DEFAULT the
    reference multiplies and adds in the operands' own C types (a product of
    two binary32 values is rounded to binary32 even when D is binary64, and
    IEEE-half storage computes in half), F16F16_ACCUM_F16 keeps its sums in
    half, and the 16-bit precisions keep running unary sums in 16 bits
    (product.c:1958-2017); the CUDA kernels compute these in binary32 or binary64, so the
    two results differ by up to the reference's rounding, not only by the
    kernels'."""
    types = [case.A.dtype, case.B.dtype, case.D.dtype] + ([] if case.C_is_null else [case.C.dtype])
    if case.prec == 4 or (case.prec == -1 and TAPP_F16 in types):
        u = UNIT["f16"]
    elif case.prec in (0, 5, 6) or (case.prec == -1 and any(t in (TAPP_F32, TAPP_C32, TAPP_BF16) for t in types)):
        u = UNIT["f32"]
    else:
        u = UNIT["f64"]
    K, UA, UB = folded_sizes(case)
    n = K * max(UA, 1) + UA + UB + 8
    gamma = n * u / (1 - n * u)
    if max(UA, UB) > 1 and (case.prec in (4, 5, 6) or u == UNIT["f16"]):
        # running unary sums kept in 16 bits, rounded after every addition
        gamma += (UA + UB) * (UNIT["bf16"] if case.prec == 6 else UNIT["f16"])
    return gamma * scale + 2 * output_unit(case.D.dtype) * np.abs(D64) + 1e-300


def against_reference(tapp, oracle, case, ref, device=False, executor=None):
    if ref is None:
        pytest.skip("the reference was not built from its sources into oracle/_ref")
    r = case.copy()
    e_ref = r.run(ref)
    g = case.copy()
    e_gpu = run_on_device(tapp, g, executor) if device else g.run(tapp, executor=executor)
    assert e_gpu == e_ref, (case.name, e_gpu, e_ref)
    if e_ref:
        return
    e64, D64, scale = oracle.execute_f64(case.copy())
    assert e64 == 0
    bound = error_bound(case, scale, D64) + reference_bound(case, scale, D64)
    got, want = d_values(g.D), d_values(r.D)
    bad = np.abs(got - want) > bound
    assert not bad.any(), (case.name, int(bad.sum()), got[bad][:3], want[bad][:3], bound[bad][:3])


@pytest.mark.parametrize("prec", [-1, 0, 1])
def test_families_against_reference(tapp, oracle, gpu, prec):
    for i, (fam, case) in enumerate(family_cases(1000 + prec, 3)):
        case.prec = prec
        against_reference(tapp, oracle, case, REF, device=bool(i % 2))


@pytest.mark.parametrize("prec", [-1, 0, 1])
def test_mixed_storage_types_against_reference(tapp, oracle, gpu, prec):
    rng = np.random.default_rng(77 + prec)
    for types in itertools.product((0, 1, 2, 3), repeat=4):
        if prec != -1 and types[0] in (0, 1) and types[1] in (2, 3):
            continue  # the reference leaves B's imaginary sum uninitialised there (product.c:381)
        case = random_case(rng, types=types, prec=prec, n_isoA=int(rng.integers(0, 2)),
                           n_isoB=int(rng.integers(0, 2)), n_repA=int(rng.integers(0, 2)),
                           subtensor=True, mixed=True)
        against_reference(tapp, oracle, case, REF)


@pytest.mark.parametrize("prec", [4, 5])
def test_half_precisions_against_reference(tapp, oracle, gpu, prec):
    rng = np.random.default_rng(300 + prec)
    for types in [(0, 0, 0, 0), (1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3), (4, 4, 4, 4), (4, 0, 4, 0), (0, 4, 0, 4)]:
        for i in range(4):
            case = random_case(rng, types=types, prec=prec, n_isoA=i % 2, n_repA=(i // 2) % 2,
                               mixed=(i == 3), subtensor=True)
            against_reference(tapp, oracle, case, REF16)


def test_binary16_storage_default_precision_against_reference(tapp, oracle, gpu):
    rng = np.random.default_rng(11)
    for i in range(12):
        case = random_case(rng, types=(4, 4, 4, 4), prec=-1, n_isoA=i % 2, subtensor=True)
        against_reference(tapp, oracle, case, REF16)


@pytest.mark.parametrize("storage,prec", [(0, -1), (0, 0), (1, -1), (2, -1), (3, -1), (0, 1)])
def test_cuda_core_kernels_against_reference(tapp, oracle, gpu, storage, prec):
    """The tiled CUDA-core GEMM (forced), the narrow kernels on each mode of
    a Tucker product and the reduction path, each against the reference."""
    rng = np.random.default_rng(500 + 7 * storage + prec)
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_SIMT)
    case = bounded_case(rng, dtype=storage, prec=prec, n_contracted=2, n_freeA=1, n_freeB=1, n_hadamard=1,
                        ext_choices=[9, 24], max_work=4e5)
    against_reference(tapp, oracle, case, REF, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)
    core = [64, 40, 33]
    for mode in range(3):
        d_ext = list(core)
        d_ext[mode] = 12
        d_idx = [0, 1, 2]
        d_idx[mode] = 3
        case = spec_case(rng, storage, prec, (core, [12, core[mode]], d_ext, d_ext),
                         ([0, 1, 2], [3, mode], d_idx, d_idx), "tucker")
        against_reference(tapp, oracle, case, REF, device=True)
    case = spec_case(rng, storage, prec, ([12, 5, 20, 12], [12, 12, 20], [5], [5]),
                     ([0, 4, 1, 2], [2, 0, 1], [4], [4]))
    against_reference(tapp, oracle, case, REF, device=True)

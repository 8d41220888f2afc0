"""GPU parity of the tensor-core path (pack pre-pass + tcgen05 GEMM).

Products are forced onto the tensor cores with the executor attribute
TAPP_B200_ATTR_PATH = 4; binary32 products use the split-bfloat16 mode
(TAPP_B200_ATTR_F32_MODE = 1). Bounds (helpers.error_bound):
  BF16BF16_ACCUM_F32 / F16F16_ACCUM_F32: operands are rounded to 16 bits
    exactly as the oracle rounds them, products are exact in binary32, so
    the binary32 summation bound gamma_n applies unchanged;
  split bfloat16: x = hi + lo + r with |r| <= 2^-18 |x|, and the dropped
    lo*lo term, give at most 3 * 2^-18 |a||b| per product; the tests add
    2^-16 relative to |alpha| sum|a||b|.
"""
import numpy as np
import pytest

import tapp_b200
from tapp_b200.workloads import large_dense_case, dense_contraction_case
from families import bounded_case
from helpers import error_bound, d_values, run_on_device
from test_gpu_parity import check_against_f64

pytestmark = pytest.mark.gpu
SPLIT_REL = 2.0 ** -16


def tc_executor(tapp, split=False):
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_TC)
    tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
    if split:
        tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, 1)
    return ex


def path_of(tapp, case, ex):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    d = tapp.describe(plan, ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    return d


@pytest.mark.parametrize("prec,storage", [(6, 0), (5, 0), (6, 5), (5, 4), (4, 0)])
def test_dense_4index_contraction(tapp, oracle, gpu, prec, storage):
    """D[a,b,i,j] = sum_{c,d} A[a,c,i,d] B[d,b,c,j] + 0.5 C with extents 16
    (M = N = K = 256), N(0,1) with 1% outliers x1e3."""
    case = large_dense_case(np.random.default_rng(prec * 10 + storage), prec, storage, extent=16)
    ex = tc_executor(tapp)
    assert "path=tc" in path_of(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


def test_split_bf16_float32(tapp, oracle, gpu):
    case = large_dense_case(np.random.default_rng(3), 0, 0, extent=16)
    ex = tc_executor(tapp, split=True)
    assert "tc_mode=split_bf16" in path_of(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex, extra_rel=SPLIT_REL)
    tapp.lib.TAPP_destroy_executor(ex)


def test_ragged_sizes_and_tails(tapp, oracle, gpu):
    """Sizes that are not multiples of the 128x256x64 tile, with a batch mode."""
    rng = np.random.default_rng(4)
    for prec in (6, 5):
        for i in range(4):
            case = bounded_case(rng, dtype=0, prec=prec, n_contracted=2, n_freeA=1, n_freeB=2, n_hadamard=i % 2,
                                ext_choices=[3, 13, 37, 70, 129], subtensor=bool(i % 2), mixed=(i == 3))
            ex = tc_executor(tapp)
            check_against_f64(tapp, oracle, case, device=bool(i % 2), executor=ex)
            tapp.lib.TAPP_destroy_executor(ex)


def test_unary_and_diagonal_in_pack(tapp, oracle, gpu):
    rng = np.random.default_rng(5)
    for prec in (6, 5):
        case = bounded_case(rng, dtype=0, prec=prec, n_contracted=1, n_freeA=1, n_freeB=1, n_isoA=1, n_isoB=1,
                            n_repA=1, ext_choices=[3, 67, 130])
        ex = tc_executor(tapp)
        check_against_f64(tapp, oracle, case, device=True, executor=ex)
        tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("mode", ["split", "bf16", "f16"])
def test_complex_4m(tapp, oracle, gpu, mode):
    """Complex float products as one real GEMM (4M form), with conj(A)."""
    rng = np.random.default_rng(6)
    prec = {"split": 0, "bf16": 6, "f16": 5}[mode]
    for i in range(3):
        case = bounded_case(rng, dtype=2, prec=prec, n_contracted=2, n_freeA=2, n_freeB=1, n_hadamard=i % 2,
                            ext_choices=[9, 33, 65], ops=[1, 0, int(i == 2), int(i == 1)], mixed=(i == 1))
        ex = tc_executor(tapp, split=(mode == "split"))
        assert "compute=c32" in path_of(tapp, case, ex)
        check_against_f64(tapp, oracle, case, device=True, executor=ex,
                          extra_rel=SPLIT_REL if mode == "split" else 0.0)
        tapp.lib.TAPP_destroy_executor(ex)


def test_tc_chosen_automatically_for_16bit_precisions(tapp, gpu):
    case = large_dense_case(np.random.default_rng(7), 6, 0, extent=16)
    ex = tapp.create_executor()
    assert "path=tc" in path_of(tapp, case, ex)
    tapp.lib.TAPP_destroy_executor(ex)


def test_full_size_dense_sampled(tapp, oracle, gpu):
    """The 64^4 contraction (M = N = K = 4096) in BF16BF16_ACCUM_F32: 4096
    outputs sampled across the whole tensor checked against binary64."""
    case = large_dense_case(np.random.default_rng(8), 6, 0, extent=64)
    run = case.copy()
    assert run_on_device(tapp, run) == 0
    rng = np.random.default_rng(9)
    samples = rng.integers(0, 64 ** 4, 4096)
    err, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
    got = run.D.buf[run.D.base + offs].astype(np.complex128)
    n = 4096 + 8
    bound = (n * 2.0 ** -24) * scale + 2 * 2.0 ** -24 * np.abs(D64)
    assert (np.abs(got - D64) <= bound).all()


def _matmul_case(rng, a, b, k, h, prec, beta=0.7, permute_C=False):
    """D[a,b,h] = sum_k A[a,k,h] B[k,b,h] + beta C, dense column-major."""
    from tapp_b200.case import alloc, fill_uniform, scalar, Case
    L = {c: ord(c) for c in "abkh"}
    def t(idx, ext, strides=None):
        if strides is None:
            strides, acc = [], 1
            for e in ext:
                strides.append(acc)
                acc *= e
        T = alloc(0, ext, strides, [L[c] for c in idx])
        fill_uniform(T, rng)
        return T
    A = t("akh", [a, k, h])
    B = t("kbh", [k, b, h])
    D = t("abh", [a, b, h])
    Cc = t("abh", [a, b, h], [h * b, h, 1] if permute_C else None)
    return Case(A, B, Cc, D, scalar(0, 1.1), scalar(0, beta), prec, beta == 0.0, "matmul")


@pytest.mark.parametrize("beta,permute_C", [(0.7, False), (0.0, False), (0.7, True)])
def test_tma_epilogue_batched(tapp, oracle, gpu, beta, permute_C):
    """First M and N modes multiple of 32 (the TMA epilogue), a batch mode,
    ragged tiles; beta = 0 skips C; a permuted C falls back to per-thread
    epilogue loads."""
    rng = np.random.default_rng(11)
    for prec in (6, 5):
        case = _matmul_case(rng, 64, 96, 80, 3, prec, beta, permute_C)
        ex = tc_executor(tapp)
        check_against_f64(tapp, oracle, case, device=True, executor=ex)
        tapp.lib.TAPP_destroy_executor(ex)


def test_tma_epilogue_4index_sampled(tapp, oracle, gpu):
    """D[a,b,i,j] = sum_{c,d} A[a,c,i,d] B[d,b,c,j] + 0.5 C, extents 32
    (M = N = K = 1024), split bfloat16: 4096 outputs against binary64."""
    case = large_dense_case(np.random.default_rng(12), 0, 0, extent=32)
    ex = tc_executor(tapp, split=True)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    samples = np.random.default_rng(13).integers(0, 32 ** 4, 4096)
    err, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
    got = run.D.buf[run.D.base + offs].astype(np.complex128)
    n = 1024 * 3 + 8
    bound = (n * 2.0 ** -24 + SPLIT_REL) * scale + 2 * 2.0 ** -24 * np.abs(D64)
    assert (np.abs(got - D64) <= bound).all()
    tapp.lib.TAPP_destroy_executor(ex)

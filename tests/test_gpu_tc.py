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


def _batched_against_single(tapp, cases, ex, shared=(), misalign=0):
    """Runs TAPP_execute_batched_product over the cases (device operands,
    batch i = cases[i]; operands named in `shared` all point at case 0's
    buffers; `misalign` elements of padding shift every base) and compares
    each D bit for bit with a solo TAPP_execute_product of the same batch."""
    import ctypes as C
    import torch
    c0 = cases[0]
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (c0.A, c0.B, c0.C, c0.D)]
    _, plan = tapp.create_product(0, [t.op for t in (c0.A, c0.B, c0.C, c0.D)], infos,
                                  [c0.A.idx, c0.B.idx, c0.C.idx, c0.D.idx], c0.prec)
    n = len(cases)
    keep = []

    def dev(t):
        raw = np.zeros(t.buf.nbytes + misalign * t.itemsize, dtype=np.uint8)
        raw[misalign * t.itemsize:] = t.buf.view(np.uint8)
        x = torch.from_numpy(raw).cuda()
        keep.append(x)
        return x, x.data_ptr() + (misalign + t.base) * t.itemsize

    arrs = {k: (C.c_void_p * n)() for k in "ABCD"}
    outs = []
    for i, c in enumerate(cases):
        for k in "ABCD":
            src = c0 if k in shared else c
            t = getattr(src, k)
            if k in shared and i > 0:
                arrs[k][i] = arrs[k][0]
                continue
            x, ptr = dev(t)
            arrs[k][i] = ptr
            if k == "D":
                outs.append((x, t))
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_batched_product(plan, ex, C.byref(st), n, c0.alpha.ctypes.data, arrs["A"],
                                                arrs["B"], c0.beta.ctypes.data,
                                                None if c0.C_is_null else arrs["C"], arrs["D"])
    torch.cuda.synchronize()
    assert err == 0, tapp.explain(err)
    kernels = tapp.status_value(st.value, tapp_b200.STATUS_KERNELS)
    tapp.lib.TAPP_destroy_status(st.value)
    solos = {}
    for i, c in enumerate(cases):
        if id(c) not in solos:
            solo = c.copy()
            for k in shared:
                setattr(solo, k, getattr(cases[0], k).copy())
            assert run_on_device(tapp, solo, ex) == 0
            solos[id(c)] = solo.D.buf
        x, t = outs[i]
        got = x.cpu().numpy()[misalign * t.itemsize:].view(t.buf.dtype)
        assert np.array_equal(got.view(np.uint8), solos[id(c)].view(np.uint8)), i
    tapp.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        tapp.lib.TAPP_destroy_tensor_info(h)
    return kernels


@pytest.mark.parametrize("prec,split,misalign", [(6, False, 0), (6, False, 1), (5, False, 0), (0, True, 0)])
def test_batched_product_one_gemm(tapp, gpu, prec, split, misalign):
    """Seven batches of the 4-index contraction (extent 16) run as one pack
    launch per operand and one GEMM launch; every batch equals its solo run.
    misalign = 1 moves every base off 16-byte alignment (scalar pack loads)."""
    rng = np.random.default_rng(60 + prec)
    cases = [large_dense_case(rng, prec, 0, extent=16) for _ in range(7)]
    ex = tc_executor(tapp, split=split)
    kernels = _batched_against_single(tapp, cases, ex, misalign=misalign)
    assert kernels == 3
    tapp.lib.TAPP_destroy_executor(ex)


def test_batched_split_in_place_one_launch(tapp, gpu):
    """Split bfloat16 with the operands read in place (TAPP_B200_ATTR_F32_MODE
    = 3): seven batches in one GEMM launch (no pack), each equal to its solo
    run."""
    rng = np.random.default_rng(66)
    cases = [large_dense_case(rng, 0, 0, extent=16) for _ in range(7)]
    ex = tc_executor(tapp)
    tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, 3)
    assert _batched_against_single(tapp, cases, ex) == 1
    tapp.lib.TAPP_destroy_executor(ex)


def test_batched_complex_hadamard_misaligned(tapp, gpu):
    """Complex float with a Hadamard (batch) mode, conj(B), beta = 0 with C
    absent, and base pointers off 16-byte alignment (scalar loads in the
    pack): five batches against their solo runs."""
    rng = np.random.default_rng(64)
    cases = [bounded_case(rng, dtype=2, prec=6, n_contracted=1, n_hadamard=1, n_freeA=1, n_freeB=1,
                          ext_choices=[67, 70], ops=[0, 1, 0, 0], beta_zero=True, C_null=True, max_work=1e9)
             for _ in range(1)]
    base = cases[0]
    cases = [base] + [base.copy() for _ in range(4)]
    for c in cases[1:]:
        for t in (c.A, c.B):
            t.buf[:] = (rng.uniform(-1, 1, t.buf.size) + 1j * rng.uniform(-1, 1, t.buf.size)).astype(t.buf.dtype)
    ex = tc_executor(tapp)
    assert "path=tc" in path_of(tapp, base, ex)
    _batched_against_single(tapp, cases, ex, misalign=1)
    tapp.lib.TAPP_destroy_executor(ex)


def test_batched_groups_split_by_grid_limit(tapp, gpu):
    """2048 batch modes per product x 40 products exceed grid.z = 65535, so
    the batches run in groups (31 + 9); A, B and C are shared, D is not."""
    rng = np.random.default_rng(65)
    base = _matmul_case(rng, 64, 64, 64, 2048, 6, beta=0.5)
    cases = [base] * 40
    ex = tc_executor(tapp)
    kernels = _batched_against_single(tapp, cases, ex, shared=("A", "B", "C"))
    assert kernels == 6
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("beta", [0.5, 0.0])
def test_batched_tma_epilogue_per_batch_maps(tapp, gpu, beta):
    """Dense D[a,b] = sum_k A[a,k] B[k,b] + beta C batches (a = b = k = 256):
    the epilogue moves each batch's C and D through that batch's own tensor
    maps; beta = 0 leaves C out. Every batch equals its solo run."""
    rng = np.random.default_rng(66)
    cases = [_matmul_case(rng, 256, 256, 256, 1, 6, beta) for _ in range(9)]
    ex = tc_executor(tapp)
    assert _batched_against_single(tapp, cases, ex) == 3
    tapp.lib.TAPP_destroy_executor(ex)


def _mm16(rng, n, storage, prec, a_t, b_t):
    """D[a,b] = sum_k A B + 0.5 C with 16-bit A and B (storage), binary32 C
    and D; a_t / b_t store A as [k,a] and B as [b,k] instead of [a,k], [k,b]."""
    from tapp_b200.case import alloc, fill_uniform, scalar, Case
    ak = [ord("k"), ord("a")] if a_t else [ord("a"), ord("k")]
    bk = [ord("b"), ord("k")] if b_t else [ord("k"), ord("b")]
    def t(dtype, idx):
        T = alloc(dtype, [n, n], [1, n], idx)
        fill_uniform(T, rng)
        return T
    A, B = t(storage, ak), t(storage, bk)
    Cc, D = t(0, [ord("a"), ord("b")]), t(0, [ord("a"), ord("b")])
    return Case(A, B, Cc, D, scalar(0, 1.0), scalar(0, 0.5), prec, False, "mm16")


@pytest.mark.parametrize("storage,prec", [(5, 6), (4, 5)])
@pytest.mark.parametrize("a_t,b_t", [(False, False), (True, True), (True, False), (False, True)])
def test_16bit_operands_read_in_place(tapp, oracle, gpu, storage, prec, a_t, b_t):
    """16-bit operands of the product's own type are read by the GEMM in place
    through 5-d tensor maps (MN-major tiles when rows are contiguous, K-major
    when the contraction is): no pack launch, same result bound."""
    from test_gpu_parity import _run_with_status
    rng = np.random.default_rng(500 + storage + 2 * a_t + b_t)
    case = _mm16(rng, 256, storage, prec, a_t, b_t)
    ex = tc_executor(tapp)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    import ctypes as C
    import torch
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [case.A.idx, case.B.idx, case.C.idx, case.D.idx], prec)
    dev = [torch.from_numpy(t.buf.view(np.uint8).copy()).cuda() for t in (case.A, case.B, case.C, case.D)]
    st = tapp_b200.intptr(0)
    assert tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), case.alpha.ctypes.data, dev[0].data_ptr(),
                                         dev[1].data_ptr(), case.beta.ctypes.data, dev[2].data_ptr(),
                                         dev[3].data_ptr()) == 0
    assert tapp.status_value(st.value, tapp_b200.STATUS_KERNELS) == 1   # the GEMM alone
    tapp.lib.TAPP_destroy_status(st.value)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("storage,prec", [(5, 6), (4, 5)])
def test_16bit_4index_in_place_sampled(tapp, oracle, gpu, storage, prec):
    """The 64^4 contraction with 16-bit A and B: A[a,c,i,d] is read MN-major
    (a contiguous), B[d,b,c,j] K-major (d contiguous), both as 64 x 64 boxes of
    5-d maps; 4096 sampled outputs against binary64."""
    case = large_dense_case(np.random.default_rng(510 + prec), prec, storage, extent=64)
    ex = tc_executor(tapp)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    samples = np.random.default_rng(511).integers(0, 64 ** 4, 4096)
    err, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
    got = run.D.buf[run.D.base + offs].astype(np.complex128)
    n = 4096 + 8
    bound = n * 2.0 ** -24 / (1 - n * 2.0 ** -24) * scale + 2 * 2.0 ** -24 * np.abs(D64)
    assert (np.abs(got - D64) <= bound).all()
    tapp.lib.TAPP_destroy_executor(ex)

"""GPU parity of the tiled CUDA-core GEMM (the plain path for large real
products: binary32 and binary64, one launch per product).

Products are forced onto it with TAPP_B200_ATTR_PATH = 3 where the planner
would choose another path; the bound is helpers.error_bound (binary32 or
binary64 summation, 16-bit operand rounding identical to the oracle's).
"""
import numpy as np
import pytest

import tapp_b200
from tapp_b200.workloads import dense_contraction_case, large_dense_case
from families import bounded_case
from test_gpu_parity import check_against_f64
from helpers import run_on_device

pytestmark = pytest.mark.gpu


def simt_executor(tapp):
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_SIMT)
    return ex


def describe(tapp, case, ex):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    d = tapp.describe(plan, ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    return d


def test_dense_contraction_float32_chooses_simt(tapp, oracle, gpu):
    """D[a,b,c,d] = 1.3 sum_{e,f} A[a,e,b,f] B[f,c,e,d] + 0.7 C, extents 16, F32F32_ACCUM_F32."""
    case = dense_contraction_case(np.random.default_rng(31), extent=16)
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("dtype,prec", [(0, -1), (0, 0), (1, -1), (1, 1), (0, 1), (1, 0), (0, 6), (0, 5)])
def test_random_real_products(tapp, oracle, gpu, dtype, prec):
    rng = np.random.default_rng(40 + dtype * 10 + prec)
    for i in range(4):
        case = bounded_case(rng, dtype=dtype, prec=prec, n_contracted=1 + i % 2, n_freeA=1 + (i % 2),
                            n_freeB=1 + (i // 2), n_hadamard=i % 2, ext_choices=[3, 17, 40, 129],
                            subtensor=bool(i % 2), mixed=(i == 3), n_repA=int(i == 2), max_work=2e6)
        ex = simt_executor(tapp)
        check_against_f64(tapp, oracle, case, device=bool(i % 2), executor=ex)
        tapp.lib.TAPP_destroy_executor(ex)


def test_mixed_storage_types(tapp, oracle, gpu):
    rng = np.random.default_rng(50)
    for types in [(0, 1, 0, 1), (1, 0, 1, 0), (4, 4, 0, 0), (5, 0, 0, 4)]:
        case = bounded_case(rng, types=types, prec=-1, n_contracted=2, n_freeA=1, n_freeB=1, n_hadamard=0,
                            ext_choices=[33, 70], max_work=2e6)
        ex = simt_executor(tapp)
        check_against_f64(tapp, oracle, case, device=True, executor=ex)
        tapp.lib.TAPP_destroy_executor(ex)


def test_double_4index_sampled(tapp, oracle, gpu):
    """D[a,b,i,j] = sum_{e,f} A[a,b,e,f] B[e,f,i,j] + C in binary64 at extents 40/12
    (M = 1600, N = 144, K = 1600), log-uniform magnitudes: sampled outputs."""
    from tapp_b200.workloads import double_case
    from helpers import run_on_device
    case = double_case(np.random.default_rng(51), cplx=False, ab=40, ij=12)
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    samples = np.random.default_rng(52).integers(0, 40 * 40 * 12 * 12, 2048)
    err, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
    got = run.D.buf[run.D.base + offs].astype(np.complex128)
    n = 1600 + 8
    bound = n * 2.0 ** -53 * scale * 4 + 2 * 2.0 ** -53 * np.abs(D64)
    assert (np.abs(got - D64) <= bound).all()
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("dtype,prec", [(2, -1), (3, -1), (2, 0), (3, 1), (3, 0), (2, 1)])
def test_complex_products(tapp, oracle, gpu, dtype, prec):
    """Complex float and double with every element op (op_C only under DEFAULT,
    op_D under F64 rounding through binary32, as the reference does)."""
    rng = np.random.default_rng(60 + dtype * 10 + prec)
    for i in range(4):
        case = bounded_case(rng, dtype=dtype, prec=prec, n_contracted=1 + i % 2, n_freeA=1, n_freeB=1 + i % 2,
                            n_hadamard=i % 2, ext_choices=[5, 33, 70], ops=[i & 1, (i >> 1) & 1, 1, int(i == 3)],
                            subtensor=bool(i % 2), mixed=(i == 2), max_work=1e6)
        ex = simt_executor(tapp)
        check_against_f64(tapp, oracle, case, device=bool(i % 2), executor=ex)
        tapp.lib.TAPP_destroy_executor(ex)


def test_complex_double_4index_sampled(tapp, oracle, gpu):
    """The complex-double form of the 4-index contraction with conj(A), extents
    40/12, random phases, log-uniform magnitudes: sampled outputs."""
    from tapp_b200.workloads import double_case
    from helpers import run_on_device
    case = double_case(np.random.default_rng(61), cplx=True, ab=40, ij=12)
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex) and "compute=c64" in describe(tapp, case, ex)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    samples = np.random.default_rng(62).integers(0, 40 * 40 * 12 * 12, 2048)
    err, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
    got = run.D.buf[run.D.base + offs].astype(np.complex128)
    n = 1600 + 8
    bound = n * 2.0 ** -53 * scale * 4 + 2 * 2.0 ** -53 * np.abs(D64)
    assert (np.abs(got - D64) <= bound).all()
    tapp.lib.TAPP_destroy_executor(ex)


def spec_case(rng, storage, prec, extents, idx, kind="shape"):
    from tapp_b200.workloads import RequestSpec, case_from_spec
    cplx = storage in (2, 3)
    a = complex(rng.uniform(-1, 1), rng.uniform(-1, 1)) if cplx else float(rng.uniform(-1, 1))
    b = complex(rng.uniform(-1, 1), rng.uniform(-1, 1)) if cplx else float(rng.uniform(-1, 1))
    return case_from_spec(rng, RequestSpec(kind, storage, prec, extents, idx, a, b))


@pytest.mark.parametrize("storage,prec", [(0, 0), (0, 6), (1, -1), (2, -1), (3, -1)])
@pytest.mark.parametrize("rank", [4, 12, 24, 40])
def test_mode_n_products_narrow_tiles(tapp, oracle, gpu, storage, prec, rank):
    """Tucker mode-n products D[i,r,k] = sum_j core[i,j,k] U[r,j] (and on the
    first and last mode): N is the factor rank, so the narrow 128x16 and
    128x32 tiles and the square tile all appear."""
    rng = np.random.default_rng(70 + rank + 7 * storage + prec)
    core = [101, 61, 43]
    for mode in range(3):
        d_ext = list(core)
        d_ext[mode] = rank
        d_idx = [0, 1, 2]
        d_idx[mode] = 3
        case = spec_case(rng, storage, prec, ([*core], [rank, core[mode]], d_ext, d_ext),
                         ([0, 1, 2], [3, mode], d_idx, d_idx), "tucker")
        ex = tapp.create_executor()
        assert "path=simt" in describe(tapp, case, ex)
        check_against_f64(tapp, oracle, case, device=bool(mode % 2), executor=ex)
        tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("storage,prec", [(0, 0), (1, -1), (2, -1), (0, 6)])
@pytest.mark.parametrize("turned", [False, True])
def test_long_contraction_split(tapp, oracle, gpu, storage, prec, turned):
    """Few output tiles and a long contraction: the contraction is split over
    the grid and the splits are added by the final kernel. turned=True puts
    the long side on B (the view is turned so that M >= N)."""
    rng = np.random.default_rng(90 + storage + 3 * prec + int(turned))
    A = ([12, 10, 30, 24], [0, 1, 4, 2])
    B = ([14, 12, 24, 10], [3, 0, 2, 1])
    D = ([14, 30], [3, 4])
    if turned:
        A, B = B, A
    case = spec_case(rng, storage, prec, (A[0], B[0], D[0], D[0]), (A[1], B[1], D[1], D[1]))
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("storage,prec", [(0, 0), (1, -1), (2, -1), (3, -1), (0, 6)])
def test_few_outputs_split_reduction(tapp, oracle, gpu, storage, prec):
    """D[x] = sum_{a,b,c} A[a,x,b,c] B[c,a,b] with 5 outputs and 36000 terms
    each: the reduction path with the contraction split over blocks."""
    rng = np.random.default_rng(110 + storage + prec)
    case = spec_case(rng, storage, prec, ([30, 5, 40, 30], [30, 30, 40], [5], [5]),
                     ([0, 4, 1, 2], [2, 0, 1], [4], [4]))
    ex = tapp.create_executor()
    assert "path=reduce" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=False, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("storage,prec", [(0, 0), (1, -1), (2, -1), (3, -1), (0, 6)])
def test_hadamard_long_contraction_reduction(tapp, oracle, gpu, storage, prec):
    """D[a,h] = sum_{b,c,e} A[a,b,c,h,e] B[e,b,h,c]: 1200 outputs (a Hadamard
    mode of 40) of 2880 terms each, too few outputs to give each a thread:
    one block per output on the reduction path."""
    rng = np.random.default_rng(130 + storage + prec)
    case = spec_case(rng, storage, prec, ([30, 24, 20, 40, 6], [6, 24, 40, 20], [30, 40], [30, 40]),
                     ([0, 1, 2, 3, 4], [4, 1, 3, 2], [0, 3], [0, 3]), kind="hadamard")
    ex = tapp.create_executor()
    assert "path=reduce" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("prec", [0, 6])
@pytest.mark.parametrize("rank", [8, 24, 40, 60])
def test_first_mode_products_beta_zero_and_aliased_c(tapp, oracle, gpu, prec, rank):
    """Mode-n products on the first mode (A contiguous along the contraction,
    D along the rank: the cooperative streaming kernel) with beta = 0, and
    with C given as D's own buffer, whose result must equal the one from a
    separate copy of C bit for bit (rows are read and written by one warp)."""
    import ctypes as C
    import torch
    from tapp_b200.case import scalar
    rng = np.random.default_rng(200 + rank + prec)
    core = [60, 77, 43]
    d_ext = [rank, 77, 43]
    case = spec_case(rng, 0, prec, (core, [rank, 60], d_ext, d_ext), ([0, 1, 2], [3, 0], [3, 1, 2], [3, 1, 2]),
                     "tucker")
    zero = case.copy()
    zero.beta = scalar(0, 0.0)
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, zero, device=True, executor=ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [case.A.idx, case.B.idx, case.C.idx, case.D.idx], prec)
    dev = [torch.from_numpy(t.buf.view(np.uint8).copy()).cuda() for t in (case.A, case.B, case.C, case.D)]
    aliased = dev[2].clone()  # D's buffer holding C's values
    st = tapp_b200.intptr(0)
    call = lambda Cp, Dp: tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), case.alpha.ctypes.data, dev[0].data_ptr(),
                                                        dev[1].data_ptr(), case.beta.ctypes.data, Cp, Dp)
    assert call(dev[2].data_ptr(), dev[3].data_ptr()) == 0
    assert call(aliased.data_ptr(), aliased.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.equal(aliased, dev[3])
    tapp.lib.TAPP_destroy_tensor_product(plan)
    tapp.lib.TAPP_destroy_executor(ex)


def _padded_rows(case):
    """The same product with every tensor's first mode padded by one element
    (leading stride extent + 1): values unchanged, row vectors impossible."""
    from tapp_b200.case import alloc
    out = case.copy()
    for name in ("A", "C", "D"):
        t = getattr(case, name)
        if t.strides[0] != 1:
            continue
        strides, acc = [], 1
        for j, e in enumerate(t.extents):
            strides.append(acc)
            acc *= e + 1 if j == 0 else e
        u = alloc(t.dtype, list(t.extents), strides, list(t.idx))
        u.op = t.op
        u.buf[u.base + u.offsets()] = t.buf[t.base + t.offsets()]
        setattr(out, name, u)
    return out


@pytest.mark.parametrize("prec", [0, 6])
@pytest.mark.parametrize("rank", [24, 40, 60])
def test_first_mode_products_contraction_runs(tapp, oracle, gpu, prec, rank):
    """Mode-n products on the first mode with A's rows read in 16-byte runs
    along the contraction (the register-tiled kernel with a swizzled ring):
    within the binary64 bound, and bit-identical to the same product with A's
    first mode padded, which runs the cooperative kernel with the same
    summation order."""
    rng = np.random.default_rng(500 + rank + prec)
    core = [60, 77, 43]
    d_ext = [rank, 77, 43]
    case = spec_case(rng, 0, prec, (core, [rank, 60], d_ext, d_ext), ([0, 1, 2], [3, 0], [3, 1, 2], [3, 1, 2]),
                     "tucker")
    ex = tapp.create_executor()
    assert "kernel=narrow_kt" in describe(tapp, case, ex), describe(tapp, case, ex)
    padded = _padded_rows(case)
    assert "kernel=narrow_coop" in describe(tapp, padded, ex), describe(tapp, padded, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    runs = []
    for c in (case, padded):
        run = c.copy()
        assert run_on_device(tapp, run, ex) == 0
        runs.append(run.D.buf[run.D.base + run.D.offsets()].copy())
    assert np.array_equal(runs[0].view(np.uint8), runs[1].view(np.uint8))
    tapp.lib.TAPP_destroy_executor(ex)


WIDE_CASES = [(st, pr, core, mode, rank)
              for st, pr in ((0, 0), (0, 6), (2, -1))
              for core, mode, rank in (([64, 100, 36], 1, 60), ([48, 40, 130], 2, 52), ([128, 40, 64], 0, 56))
              if not (mode == 0 and st == 2)]  # complex first-mode products have no register-tiled form


@pytest.mark.parametrize("storage,prec,core,mode,rank", WIDE_CASES)
def test_wide_mode_n_products_row_vectors(tapp, oracle, gpu, storage, prec, core, mode, rank):
    """Mode-n products with more than 48 columns and a contraction over more
    than 64 terms: the register-tiled kernels (rows contiguous in A, C and D,
    real and complex; binary32 A contiguous along the contraction on the
    first mode) take them, within the binary64 bound."""
    rng = np.random.default_rng(700 + rank + 7 * storage + prec + mode)
    d_ext = list(core)
    d_ext[mode] = rank
    d_idx = [0, 1, 2]
    d_idx[mode] = 3
    case = spec_case(rng, storage, prec, ([*core], [rank, core[mode]], d_ext, d_ext),
                     ([0, 1, 2], [3, mode], d_idx, d_idx), "tucker")
    ex = tapp.create_executor()
    want = "kernel=narrow_cvec" if storage == 2 else ("kernel=narrow_kt" if mode == 0 else "kernel=narrow_vec")
    assert want in describe(tapp, case, ex), describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("ops", [(0, 0, 0, 0), (1, 1, 1, 1), (0, 1, 0, 1)])
@pytest.mark.parametrize("core,mode,rank", [([64, 40, 36], 1, 24), ([62, 33, 80], 1, 8), ([64, 40, 36], 2, 30)])
def test_complex_mode_n_products_row_vectors(tapp, oracle, gpu, ops, core, mode, rank):
    """Complex-float mode-n products with A, C and D contiguous along their
    rows (the complex register-tiled kernel, 2-row vectors), with op_A, op_B,
    op_C and op_D: within the binary64 bound, and bit-identical to the same
    product with padded rows (the complex streaming kernel, the same
    multiply-add order)."""
    rng = np.random.default_rng(600 + rank + 7 * sum(ops) + mode)
    d_ext = list(core)
    d_ext[mode] = rank
    d_idx = [0, 1, 2]
    d_idx[mode] = 3
    case = spec_case(rng, 2, -1, ([*core], [rank, core[mode]], d_ext, d_ext), ([0, 1, 2], [3, mode], d_idx, d_idx),
                     "tucker")
    for t, o in zip((case.A, case.B, case.C, case.D), ops):
        t.op = o
    ex = tapp.create_executor()
    assert "kernel=narrow_cvec" in describe(tapp, case, ex), describe(tapp, case, ex)
    padded = _padded_rows(case)
    assert "kernel=narrow_cstream" in describe(tapp, padded, ex), describe(tapp, padded, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    runs = []
    for c in (case, padded):
        run = c.copy()
        assert run_on_device(tapp, run, ex) == 0
        runs.append(run.D.buf[run.D.base + run.D.offsets()].copy())
    assert np.array_equal(runs[0].view(np.uint8), runs[1].view(np.uint8))
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("storage,prec", [(0, 0), (0, 6), (1, -1)])
@pytest.mark.parametrize("core,mode,rank", [([64, 40, 36], 1, 38), ([64, 40, 36], 2, 24), ([62, 33, 80], 1, 8),
                                            ([62, 33, 40], 2, 60), ([32, 48, 64], 1, 64)])
def test_mode_n_products_row_vectors(tapp, oracle, gpu, storage, prec, core, mode, rank):
    """Mode-n products on an inner mode with A, C and D contiguous along their
    rows (the register-tiled kernel, 4- or 2-row vectors; widths 8 to 64,
    beta = 0 too): within the binary64 bound, and bit-identical to the same
    product with padded rows, which runs a one-row-per-thread kernel with the
    same summation order."""
    from tapp_b200.case import scalar
    rng = np.random.default_rng(400 + rank + 7 * storage + prec + mode)
    d_ext = list(core)
    d_ext[mode] = rank
    d_idx = [0, 1, 2]
    d_idx[mode] = 3
    case = spec_case(rng, storage, prec, ([*core], [rank, core[mode]], d_ext, d_ext),
                     ([0, 1, 2], [3, mode], d_idx, d_idx), "tucker")
    if rank == 8:
        case.beta = scalar(case.D.dtype, 0.0)
    ex = tapp.create_executor()
    assert "kernel=narrow_vec" in describe(tapp, case, ex), describe(tapp, case, ex)
    padded = _padded_rows(case)
    assert "kernel=narrow_vec" not in describe(tapp, padded, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    runs = []
    for c in (case, padded):
        run = c.copy()
        assert run_on_device(tapp, run, ex) == 0
        runs.append(run.D.buf[run.D.base + run.D.offsets()].copy())
    assert np.array_equal(runs[0].view(np.uint8), runs[1].view(np.uint8))
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("ops", [(0, 0, 0, 0), (1, 1, 1, 1), (1, 0, 0, 1)])
@pytest.mark.parametrize("rank", [6, 12, 30])
def test_complex_mode_n_products_streaming(tapp, oracle, gpu, ops, rank):
    """Complex-float mode-n products on an inner mode (rows contiguous in A and
    D, at most 32 columns: the complex streaming kernel), with op_A, op_B,
    op_C and op_D conjugation under the DEFAULT precision."""
    rng = np.random.default_rng(300 + rank + 7 * sum(ops))
    core = [70, 45, 60]
    d_ext = [70, rank, 60]
    case = spec_case(rng, 2, -1, (core, [rank, 45], d_ext, d_ext), ([0, 1, 2], [3, 1], [0, 3, 2], [0, 3, 2]), "tucker")
    for t, o in zip((case.A, case.B, case.C, case.D), ops):
        t.op = o
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    check_against_f64(tapp, oracle, case, device=False, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)


@pytest.mark.parametrize("storage,prec", [(0, 0), (1, -1)])
@pytest.mark.parametrize("a_t,b_t", [(False, False), (True, False), (False, True), (True, True)])
def test_gemm_vector_loads(tapp, oracle, gpu, storage, prec, a_t, b_t):
    """Binary32 and binary64 matrix products D[m,n] = A B + C whose operands
    are dense with extents divisible by 4 (the tiled kernel reads them 16
    bytes at a time, along rows or along the contraction), with ragged tiles
    (600 rows, 200 columns) and a contraction of 1000."""
    rng = np.random.default_rng(400 + 2 * a_t + b_t + 10 * storage)
    M, N, K = 600, 200, 1000
    A = ([K, M], [2, 0]) if a_t else ([M, K], [0, 2])
    B = ([N, K], [1, 2]) if b_t else ([K, N], [2, 1])
    case = spec_case(rng, storage, prec, (A[0], B[0], [M, N], [M, N]), (A[1], B[1], [0, 1], [0, 1]))
    ex = tapp.create_executor()
    assert "path=simt" in describe(tapp, case, ex)
    check_against_f64(tapp, oracle, case, device=True, executor=ex)
    tapp.lib.TAPP_destroy_executor(ex)

"""The benchmark configurations on the GPU at their stated sizes, and the two
small ones against the reference itself.

  c1  D[a,b,c,d] = 1.3 sum_{e,f} A[a,e,b,f] B[f,c,e,d] + 0.7 C, float32,
      every extent 16: plain CUDA-core float32 and split bfloat16, compared
      element by element with the D the reference's own TAPP_execute_product
      (built from its sources into oracle/_ref) writes for the same inputs.
  c2  complex float, DEFAULT precision, Hadamard + diagonal + unary modes,
      conj(B), a view with negative and zero strides, D permuted against C:
      against the reference likewise.
  c3  the 64^4 contraction (M = N = K = 4096) in F16F16_ACCUM_F32, split
      bfloat16 and plain float32: 4096 outputs sampled over D against the
      oracle's binary64 evaluation.
  c4  D[a,b,i,j] = sum_{e,f} A[a,b,e,f] B[e,f,i,j] + C with a=b=e=f=160,
      i=j=40 (M = K = 25600, N = 1600), binary64 and complex double with
      conj(A), magnitudes log-uniform in [1e-8, 1]: native CUDA-core and
      sliced (7 and 8 digit slices) against the oracle's binary64 evaluation
      of 64 x 64 sampled outputs.

Against the reference, the GPU's D and the reference's D each lie within the
rounding bound of their arithmetic (tests/helpers.error_bound) of the exact
binary64 result, so they differ by at most the sum of the two bounds.
"""
import math

import numpy as np
import pytest

import oracle as oracle_mod
import tapp_b200
from tapp_b200.case import Case, Tensor, scalar
from tapp_b200.workloads import dense_contraction_case, mixed_classes_case, large_dense_case
from helpers import run_on_device, error_bound, d_values
from test_gpu_sliced import sliced_bound

pytestmark = pytest.mark.gpu

SPLIT_REL = 2.0 ** -16
F64_MODE = 0x1007


def _reference():
    ref = oracle_mod.reference_lib()
    if ref is None:
        pytest.skip("the reference was not built from its sources into oracle/_ref")
    return ref


def _executor(tapp, f32_mode=0, path=0, f64_mode=0):
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, f32_mode)
    tapp.set_int(ex, tapp_b200.ATTR_PATH, path)
    if f64_mode:
        assert tapp.set_int(ex, F64_MODE, f64_mode) == 0
    return ex


def _path(tapp, case, ex):
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
    d = tapp.describe(plan, ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        tapp.lib.TAPP_destroy_tensor_info(h)
    return d


def _against_reference(tapp, oracle, case, f32_mode, extra_rel, want_path):
    ref = _reference()
    rc = case.copy()
    assert rc.run(ref) == 0
    e64, D64, scale = oracle.execute_f64(case.copy())
    assert e64 == 0
    b_ref = error_bound(case, scale, D64)
    b_gpu = error_bound(case, scale, D64, extra_rel)
    d_ref = d_values(rc.D)
    assert (np.abs(d_ref - D64) <= b_ref).all(), "the reference itself outside its rounding bound"
    ex = _executor(tapp, f32_mode)
    assert f"path={want_path}" in _path(tapp, case, ex)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    tapp.lib.TAPP_destroy_executor(ex)
    got = d_values(run.D)
    diff = np.abs(got - d_ref)
    bad = diff > b_gpu + b_ref
    assert not bad.any(), (int(bad.sum()), diff[bad][:4], (b_gpu + b_ref)[bad][:4])
    return float(diff.max() / np.abs(d_ref).max())


@pytest.mark.parametrize("mode,f32_mode,extra,path", [("plain_f32", 0, 0.0, "simt"),
                                                      ("split_bf16", 1, SPLIT_REL, "tc")])
def test_c1_against_reference(tapp, oracle, gpu, mode, f32_mode, extra, path):
    case = dense_contraction_case(np.random.default_rng(0x7A990001), extent=16)
    rel = _against_reference(tapp, oracle, case, f32_mode, extra, path)
    assert rel < (1e-5 if f32_mode else 1e-6)


def test_c2_against_reference(tapp, oracle, gpu):
    case = mixed_classes_case(np.random.default_rng(0x7A990002))
    rel = _against_reference(tapp, oracle, case, 0, 0.0, "generic")
    assert rel < 1e-6


@pytest.mark.parametrize("mode,prec,f32_mode,extra,path", [
    ("f16_from_f32", tapp_b200.TAPP_F16F16_ACCUM_F32, 0, 0.0, "tc"),
    ("split_bf16", 0, 1, SPLIT_REL, "tc"),
    ("plain_f32", 0, 0, 0.0, "simt"),
])
def test_c3_full_size_sampled(tapp, oracle, gpu, mode, prec, f32_mode, extra, path):
    """64^4 (M = N = K = 4096), float32 storage, N(0,1) with 1% x1e3
    outliers, beta = 0.5: 4096 outputs sampled over D against binary64."""
    case = large_dense_case(np.random.default_rng(0x7A990003), prec, 0, extent=64)
    ex = _executor(tapp, f32_mode)
    assert f"path={path}" in _path(tapp, case, ex)
    run = case.copy()
    assert run_on_device(tapp, run, ex) == 0
    tapp.lib.TAPP_destroy_executor(ex)
    samples = np.random.default_rng(0x7A990103).integers(0, 64 ** 4, 4096)
    err, D64, scale, offs = oracle.execute_f64(case.copy(), samples=samples)
    assert err == 0
    got = run.D.buf[run.D.base + offs].astype(np.complex128)
    n = 4096 + 8
    bound = (n * 2.0 ** -24 + extra) * scale + 2 * 2.0 ** -24 * np.abs(D64)
    assert (np.abs(got - D64) <= bound).all()


# ---------------------------------------------------------------------------
# c4 at full size

C4_AB, C4_IJ = 160, 40


def _c4_device(torch, cplx, seed):
    """A, B, C (and a zeroed D) of the binary64 configuration on the GPU,
    magnitudes log-uniform in [1e-8, 1], random sign (phase), seeded."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)

    def logu(n):
        mag = torch.pow(10.0, torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 8 - 8)
        if cplx:
            ph = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * (2 * math.pi)
            return torch.polar(mag, ph)
        sign = torch.where(torch.rand(n, device="cuda", generator=g) < 0.5, -1.0, 1.0).to(torch.float64)
        return mag * sign
    M, N, K = C4_AB * C4_AB, C4_IJ * C4_IJ, C4_AB * C4_AB
    A, B, Cc = logu(M * K), logu(K * N), logu(M * N)
    D = torch.zeros(M * N, dtype=A.dtype, device="cuda")
    return A, B, Cc, D


def _c4_case(ty, ext_idx, bufs=None):
    ts = []
    for k, (ext, idx, op) in enumerate(ext_idx):
        st, acc = [], 1
        for e in ext:
            st.append(acc)
            acc *= e
        ts.append(Tensor(ty, list(ext), st, [ord(c) for c in idx], op, None if bufs is None else bufs[k], 0))
    return Case(ts[0], ts[1], ts[2], ts[3], scalar(ty, 1.0), scalar(ty, 1.0), -1, False, "c4")


@pytest.mark.parametrize("slices", [0, 7, 8])
@pytest.mark.parametrize("cplx", [False, True])
def test_c4_full_size_sampled(tapp, oracle, gpu, cplx, slices):
    """Full size: the product runs on the whole tensors; 64 rows (a,b) x 64
    columns (i,j) of D are checked against the oracle's binary64 evaluation
    of the same outputs (the product restricted to those rows of A and
    columns of B, which is the same sum)."""
    import torch
    ty = tapp_b200.TAPP_C64 if cplx else tapp_b200.TAPP_F64
    conj = tapp_b200.TAPP_CONJUGATE if cplx else 0
    ab, ij = C4_AB, C4_IJ
    M, N, K = ab * ab, ij * ij, ab * ab
    A, B, Cc, D = _c4_device(torch, cplx, 0x7A990004 + int(cplx))
    full = _c4_case(ty, [([ab] * 4, "abef", conj), ([ab, ab, ij, ij], "efij", 0),
                         ([ab, ab, ij, ij], "abij", 0), ([ab, ab, ij, ij], "abij", 0)])
    ex = _executor(tapp, f64_mode=slices)
    assert ("path=sliced" if slices else "path=simt") in _path(tapp, full, ex)
    err = full.run(tapp, executor=ex, A_ptr=A.data_ptr(), B_ptr=B.data_ptr(), C_ptr=Cc.data_ptr(),
                   D_ptr=D.data_ptr())
    torch.cuda.synchronize()
    tapp.lib.TAPP_destroy_executor(ex)
    assert err == 0, tapp.explain(err)

    rng = np.random.default_rng(0x7A990104 + int(cplx))
    ms = torch.from_numpy(np.sort(rng.choice(M, 64, replace=False))).cuda()
    ns = torch.from_numpy(np.sort(rng.choice(N, 64, replace=False))).cuda()
    # column-major A[a,b,e,f]: element (m, k) at m + M k; B[e,f,i,j]: (k, n) at k + K n
    a_sub = A.view(K, M)[:, ms].contiguous().cpu().numpy().reshape(-1)   # [p fastest, then e, f]
    b_sub = B.view(N, K)[ns, :].contiguous().cpu().numpy().reshape(-1)   # [e, f fastest, then q]
    c_sub = Cc.view(N, M)[ns][:, ms].contiguous().cpu().numpy().reshape(-1)
    got = D.view(N, M)[ns][:, ms].contiguous().cpu().numpy().reshape(-1).astype(np.complex128)
    del A, B, Cc, D
    torch.cuda.empty_cache()
    sub = _c4_case(ty, [([64, ab, ab], "pef", conj), ([ab, ab, 64], "efq", 0), ([64, 64], "pq", 0),
                        ([64, 64], "pq", 0)],
                   [a_sub, b_sub, c_sub, np.zeros_like(c_sub)])
    e64, D64, scale = oracle.execute_f64(sub.copy())
    assert e64 == 0
    if slices:
        bound = sliced_bound(sub, slices, scale, D64)
    else:
        bound = error_bound(sub, scale, D64)
    diff = np.abs(got - D64)
    bad = diff > bound
    assert not bad.any(), (int(bad.sum()), diff[bad][:4], bound[bad][:4])
    # the accuracy the benchmark reports (max error over max |D|): native
    # binary64 about 1e-14, 7 slices about 1e-13, 8 slices about 1e-15
    rel = float(diff.max() / np.abs(D64).max())
    assert rel < {0: 1e-13, 7: 1e-12, 8: 1e-14}[slices]

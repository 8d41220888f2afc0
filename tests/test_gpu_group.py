"""GPU tests of grouped tensor-core products (tapp_b200_execute_group): many
products of different shapes, layouts and precision modes in one
persistent launch per tile shape, operands read in place.

Every grouped product must give the same bits as the same product run on
its own through TAPP_execute_product (same operand rounding or splitting,
same order of the contraction, same epilogue formula), and lie within the
binary64 oracle's bound. Products that cannot join a group (plain binary32
on the CUDA cores, host operands) run as TAPP_execute_product runs them,
inside the same call.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import tapp_b200
from tapp_b200.case import Case, alloc, fill_uniform, scalar
from helpers import error_bound

pytestmark = pytest.mark.gpu
F32 = tapp_b200.TAPP_F32
SPLIT_REL = 2.0 ** -16


def _t(rng, ext, idx, order, pad=0):
    """Tensor with modes `idx` of extents `ext`, stored with the modes in
    `order` from fastest to slowest; pad widens the fastest mode's span."""
    strides = [0] * len(ext)
    acc = 1
    for n, i in enumerate(order):
        strides[i] = acc
        acc *= ext[i] + (pad if n == 0 else 0)
    return fill_uniform(alloc(F32, ext, strides, [ord(c) for c in idx]), rng)


def _product(rng, prec, ragged=False):
    """A matrix or batched matrix product with random sizes and layouts; the
    float32 (split) products keep at least 256 rows, where their solo run
    takes the same three-MMA kernel."""
    split = prec == tapp_b200.TAPP_F32F32_ACCUM_F32
    ms = [256, 264, 384, 520, 1024] if split else [128, 136, 256, 264, 384, 520, 1024]
    m = int(rng.choice(ms))
    n = int(rng.choice([64, 72, 128, 200, 256, 384, 512]))
    k = int(rng.choice([64, 96, 136, 256, 512]))
    if ragged:  # extents that are not multiples of 8: element-wise operand loads
        m, n, k = m + 3, n + 5, k + 7
    h = int(rng.choice([1, 1, 2, 3]))
    a_kmajor, b_nmajor, beta0 = rng.random() < 0.5, rng.random() < 0.5, rng.random() < 0.25
    if h > 1:
        A = _t(rng, [m, k, h], "mkh", [1, 0, 2] if a_kmajor else [0, 1, 2])
        B = _t(rng, [k, n, h], "knh", [1, 0, 2] if b_nmajor else [0, 1, 2])
        Cc = _t(rng, [m, n, h], "mnh", [0, 1, 2])
        D = _t(rng, [m, n, h], "mnh", [0, 1, 2])
    else:
        A = _t(rng, [m, k], "mk", [1, 0] if a_kmajor else [0, 1])
        B = _t(rng, [k, n], "kn", [1, 0] if b_nmajor else [0, 1])
        Cc = _t(rng, [m, n], "mn", [0, 1])
        D = _t(rng, [m, n], "mn", [0, 1])
    beta = 0.0 if beta0 else float(rng.uniform(-1, 1))
    return Case(A, B, Cc, D, scalar(F32, float(rng.uniform(0.5, 1.5))), scalar(F32, beta), prec, beta0,
                f"p{m}x{n}x{k}x{h}")


PRECS = [tapp_b200.TAPP_BF16BF16_ACCUM_F32, tapp_b200.TAPP_F16F16_ACCUM_F32, tapp_b200.TAPP_F32F32_ACCUM_F32]


def _mix(seed, count=18, ragged=False):
    rng = np.random.default_rng(seed)
    return [_product(rng, PRECS[i % 3], ragged) for i in range(count)]


class _Dev:
    """A case's buffers on the GPU and its plan."""

    def __init__(self, tapp, case):
        import torch
        self.case = case
        ts = (case.A, case.B, case.C, case.D)
        self.bufs = [torch.from_numpy(t.buf.view(np.uint8).copy()).cuda() for t in ts]
        self.ptr = [b.data_ptr() + t.base * t.itemsize for b, t in zip(self.bufs, ts)]
        self.D0 = self.bufs[3].clone()
        self.infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in ts]
        err, self.plan = tapp.create_product(0, [0, 0, 0, 0], self.infos, [t.idx for t in ts], case.prec)
        assert err == 0

    def reset(self):
        self.bufs[3].copy_(self.D0)

    def d(self):
        return self.bufs[3].cpu().numpy().view(np.float32).copy()

    def close(self, tapp):
        tapp.lib.TAPP_destroy_tensor_product(self.plan)
        for h in self.infos:
            tapp.lib.TAPP_destroy_tensor_info(h)


def _executor(tapp, tile):
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_PATH, tapp_b200.PATH_TC)
    tapp.set_int(ex, tapp_b200.ATTR_F32_MODE, 1)
    tapp.set_int(ex, tapp_b200.ATTR_TILE, tile)
    return ex


def _solo(tapp, devs, ex):
    import torch
    out = []
    for d in devs:
        d.reset()
        st = tapp_b200.intptr(0)
        c = d.case
        err = tapp.lib.TAPP_execute_product(d.plan, ex, C.byref(st), c.alpha.ctypes.data, d.ptr[0], d.ptr[1],
                                            c.beta.ctypes.data, None if c.C_is_null else d.ptr[2], d.ptr[3])
        assert err == 0, tapp.explain(err)
        torch.cuda.synchronize()
        out.append(d.d())
    return out


def _group(tapp, devs, ex):
    for d in devs:
        d.reset()
    n0 = tapp.launches()
    err = tapp.execute_group([d.plan for d in devs], ex, [d.case.alpha.ctypes.data for d in devs],
                             [d.case.beta.ctypes.data for d in devs], [d.ptr[0] for d in devs],
                             [d.ptr[1] for d in devs], [None if d.case.C_is_null else d.ptr[2] for d in devs],
                             [d.ptr[3] for d in devs])
    assert err == 0, tapp.explain(err)
    return [d.d() for d in devs], tapp.launches() - n0


def _check_bound(oracle, c, got):
    e64, D64, scale = oracle.execute_f64(c.copy())
    assert e64 == 0
    bound = error_bound(c, scale, D64, SPLIT_REL if c.prec == 0 else 0.0)
    bad = np.abs(got.astype(np.complex128) - D64) > bound
    assert not bad.any(), (c.name, int(bad.sum()))


@pytest.mark.parametrize("tile", [1, 2])
def test_group_matches_solo_runs(tapp, oracle, gpu, tile):
    """18 uneven products (bfloat16, f16 and split-bfloat16 modes; row- and
    contraction-major operands; batch modes; beta = 0 with C absent) in ONE
    launch: each equals its solo run bit for bit and lies within the
    oracle's bound."""
    cases = _mix(100 + tile)
    devs = [_Dev(tapp, c) for c in cases]
    ex = _executor(tapp, tile)
    solo = _solo(tapp, devs, ex)
    grouped, launches = _group(tapp, devs, ex)
    assert launches == 1
    same = [np.array_equal(s.view(np.uint32), g.view(np.uint32)) for s, g in zip(solo, grouped)]
    for c, g in zip(cases, grouped):
        _check_bound(oracle, c, g)
    assert all(same), [c.name for c, ok in zip(cases, same) if not ok]
    tapp.lib.TAPP_destroy_executor(ex)
    for d in devs:
        d.close(tapp)


@pytest.mark.parametrize("tile", [1, 2])
def test_group_ragged_layouts(tapp, oracle, gpu, tile):
    """Extents that are not multiples of 8 (operands loaded element by element
    through offset tables) in one launch, within the oracle's bound."""
    cases = _mix(300 + tile, count=12, ragged=True)
    devs = [_Dev(tapp, c) for c in cases]
    ex = _executor(tapp, tile)
    grouped, launches = _group(tapp, devs, ex)
    assert launches == 1
    for c, g in zip(cases, grouped):
        _check_bound(oracle, c, g)
    tapp.lib.TAPP_destroy_executor(ex)
    for d in devs:
        d.close(tapp)


def test_group_with_products_that_cannot_join(tapp, oracle, gpu):
    """Plain binary32 products (CUDA-core path) and a product with host
    operands run inside the same call, as TAPP_execute_product runs them."""
    rng = np.random.default_rng(7)
    cases = _mix(8, count=6)
    ex = tapp.create_executor()
    tapp.set_int(ex, tapp_b200.ATTR_TILE, 2)   # float32 mode 0: the float32 products stay on the CUDA cores
    devs = [_Dev(tapp, c) for c in cases]
    hc = _product(rng, tapp_b200.TAPP_BF16BF16_ACCUM_F32)
    hinfos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (hc.A, hc.B, hc.C, hc.D)]
    _, hplan = tapp.create_product(0, [0, 0, 0, 0], hinfos, [hc.A.idx, hc.B.idx, hc.C.idx, hc.D.idx], hc.prec)
    ref_h = hc.copy()
    err = tapp.execute_group([d.plan for d in devs] + [hplan], ex,
                             [c.alpha.ctypes.data for c in cases] + [hc.alpha.ctypes.data],
                             [c.beta.ctypes.data for c in cases] + [hc.beta.ctypes.data],
                             [d.ptr[0] for d in devs] + [hc.A.ptr()], [d.ptr[1] for d in devs] + [hc.B.ptr()],
                             [None if d.case.C_is_null else d.ptr[2] for d in devs] +
                             [None if hc.C_is_null else hc.C.ptr()],
                             [d.ptr[3] for d in devs] + [hc.D.ptr()])
    assert err == 0, tapp.explain(err)
    for c, dv in zip(cases, devs):
        e64, D64, scale = oracle.execute_f64(c.copy())
        assert (np.abs(dv.d().astype(np.complex128) - D64) <= error_bound(c, scale, D64)).all(), c.name
    e64, D64, scale = oracle.execute_f64(ref_h)
    assert (np.abs(hc.D.buf.astype(np.complex128) - D64) <= error_bound(hc, scale, D64)).all()
    tapp.lib.TAPP_destroy_executor(ex)
    tapp.lib.TAPP_destroy_tensor_product(hplan)
    for h in hinfos:
        tapp.lib.TAPP_destroy_tensor_info(h)
    for d in devs:
        d.close(tapp)


def test_group_validates_every_product_first(tapp, gpu):
    """A failing product (C absent with beta != 0: code 12) stops the call
    before anything runs; no kernel is launched."""
    cases = _mix(9, count=4)
    devs = [_Dev(tapp, c) for c in cases]
    ex = _executor(tapp, 1)
    bad = next(i for i, c in enumerate(cases) if not c.C_is_null)
    n0 = tapp.launches()
    err = tapp.execute_group([d.plan for d in devs], ex, [c.alpha.ctypes.data for c in cases],
                             [c.beta.ctypes.data for c in cases], [d.ptr[0] for d in devs],
                             [d.ptr[1] for d in devs],
                             [None if (i == bad or d.case.C_is_null) else d.ptr[2] for i, d in enumerate(devs)],
                             [d.ptr[3] for d in devs])
    assert err == 12
    assert tapp.launches() == n0
    tapp.lib.TAPP_destroy_executor(ex)
    for d in devs:
        d.close(tapp)


def test_tile_table_and_tuner(tapp, gpu):
    """The tuner times both tile shapes on synthetic products of two shape
    classes and writes its table; with a table that puts two classes on
    different shapes, TAPP_B200_ATTR_TILE = 0 runs a mix of them as two
    launches."""
    from tapp_b200 import tuner
    bf16 = tapp_b200.TAPP_BF16BF16_ACCUM_F32
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "tiles.txt")
        rows = tuner.tune(tapp, [(bf16, 128, 64, 256), (bf16, 1024, 512, 256)], path, products_per_class=8, reps=3)
        assert len(rows) == 2 and all(r["tile"] in (1, 2) and min(r["us"]) > 0 for r in rows)
        assert tapp.load_tile_table(path) == 0
        with open(path, "w") as f:
            f.write("# mode m n k tile\n0 7 6 8 2\n0 10 9 8 1\n")
        assert tapp.load_tile_table(path) == 0
        rng = np.random.default_rng(3)
        cases = []
        for m, n, k in [(128, 64, 256), (1024, 512, 256)]:
            T = lambda ext, idx: fill_uniform(alloc(F32, ext, [1, ext[0]], [ord(c) for c in idx]), rng)
            cases.append(Case(T([m, k], "mk"), T([k, n], "kn"), T([m, n], "mn"), T([m, n], "mn"), scalar(F32, 1.0),
                              scalar(F32, 0.5), bf16, False, "t"))
        devs = [_Dev(tapp, c) for c in cases]
        ex = _executor(tapp, 0)
        _, launches = _group(tapp, devs, ex)
        assert launches == 2
        tapp.lib.TAPP_destroy_executor(ex)
        for dv in devs:
            dv.close(tapp)
        assert tapp.load_tile_table(None) == 0

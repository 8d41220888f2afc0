"""GPU tests of the device-resident request loop (tapp_b200_loop_*): a
persistent kernel that serves small products as they are submitted, polls a
ring in mapped host memory with a time limit, and returns when idle.

  - every product served by the loop equals TAPP_execute_product's D bit for
    bit (the loop computes each output with the element kernel's function);
  - the loop returns after its idle limit (no kernel left on the GPU) and is
    launched again by the next submission;
  - products that are not small (other paths) or have host operands are
    refused, with nothing written.
"""
import ctypes as C
import time

import numpy as np
import pytest

import tapp_b200
from tapp_b200.workloads import dense_contraction_case, mixed_classes_case
from families import bounded_case
from test_gpu_element import _matvec

pytestmark = pytest.mark.gpu


def _small_cases():
    rng = np.random.default_rng(41)
    cases = [mixed_classes_case(np.random.default_rng(0x7A990002))]
    for e in (3, 4, 5):
        for dt, prec in ((tapp_b200.TAPP_F32, 0), (tapp_b200.TAPP_F64, 1), (tapp_b200.TAPP_C32, -1)):
            cases.append(dense_contraction_case(rng, extent=e, dtype=dt, prec=prec))
    for i in range(20):
        cases.append(bounded_case(rng, max_work=2e5))
    # contraction-contiguous products: TAPP_execute_product runs them one warp per output
    cases.append(_matvec(rng, tapp_b200.TAPP_F32, 0, k=200, m=40, h=5))
    cases.append(_matvec(rng, tapp_b200.TAPP_C32, -1, k=96, m=30, h=4, conj=True))
    return cases


class _Dev:
    def __init__(self, tapp, case):
        import torch
        self.case = case
        ts = (case.A, case.B, case.C, case.D)
        self.bufs = [torch.from_numpy(t.buf.view(np.uint8).copy()).cuda() for t in ts]
        self.ptr = [b.data_ptr() + t.base * t.itemsize for b, t in zip(self.bufs, ts)]
        self.D0 = self.bufs[3].clone()
        self.infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in ts]
        err, self.plan = tapp.create_product(0, [t.op for t in ts], self.infos, [t.idx for t in ts], case.prec)
        assert err == 0

    def args(self):
        c = self.case
        return (c.alpha.ctypes.data, self.ptr[0], self.ptr[1], c.beta.ctypes.data,
                None if c.C_is_null else self.ptr[2], self.ptr[3])

    def close(self, tapp):
        tapp.lib.TAPP_destroy_tensor_product(self.plan)
        for h in self.infos:
            tapp.lib.TAPP_destroy_tensor_info(h)


def _plain(tapp, devs):
    import torch
    out = []
    ex = tapp.create_executor()
    for d in devs:
        d.bufs[3].copy_(d.D0)
        a, A, B, b, Cp, D = d.args()
        st = tapp_b200.intptr(0)
        assert tapp.lib.TAPP_execute_product(d.plan, ex, C.byref(st), a, A, B, b, Cp, D) == 0
        torch.cuda.synchronize()
        out.append(d.bufs[3].cpu().numpy().copy())
    tapp.lib.TAPP_destroy_executor(ex)
    return out


@pytest.mark.parametrize("blocks", [4, "sms"])
def test_loop_matches_execute_product(tapp, gpu, blocks):
    """Products of every compute domain, small enough for the element path,
    submitted back to back (tickets in flight together over 4 blocks, and
    over one block per SM); each D equals TAPP_execute_product's bit for
    bit."""
    import torch
    if blocks == "sms":
        blocks = torch.cuda.get_device_properties(0).multi_processor_count
    devs = [_Dev(tapp, c) for c in _small_cases()]
    want = _plain(tapp, devs)
    err, loop = tapp.loop_create(0, blocks=blocks, slots=max(16, blocks), idle_ms=200.0)
    assert err == 0
    for d in devs:
        d.bufs[3].copy_(d.D0)
    import torch
    torch.cuda.synchronize()
    tickets = []
    for d in devs:
        err, t = tapp.loop_submit(loop, d.plan, *d.args())
        assert err == 0, tapp.explain(err)
        tickets.append(t)
    for t in tickets:
        assert tapp.lib.tapp_b200_loop_wait(loop, t) == 0
    for d, w in zip(devs, want):
        got = d.bufs[3].cpu().numpy()
        assert np.array_equal(got, w), d.case.name
    st = tapp.loop_stats(loop)
    assert st["submitted"] == len(devs) and st["completed"] == len(devs) and st["p50_us"] > 0
    assert tapp.lib.tapp_b200_loop_destroy(loop) == 0
    for d in devs:
        d.close(tapp)


def test_loop_returns_when_idle_and_restarts(tapp, gpu):
    """After its idle limit the loop's kernel returns (nothing left running);
    the next submission launches it again and is served."""
    devs = [_Dev(tapp, c) for c in _small_cases()[:3]]
    want = _plain(tapp, devs)
    err, loop = tapp.loop_create(0, blocks=2, slots=8, idle_ms=50.0)
    assert err == 0
    for i, d in enumerate(devs):
        d.bufs[3].copy_(d.D0)
        import torch
        torch.cuda.synchronize()
        err, t = tapp.loop_submit(loop, d.plan, *d.args())
        assert err == 0
        assert tapp.lib.tapp_b200_loop_wait(loop, t) == 0
        assert np.array_equal(d.bufs[3].cpu().numpy(), want[i])
        t0 = time.time()
        while tapp.loop_stats(loop)["running"] and time.time() - t0 < 2.0:
            time.sleep(0.01)
        st = tapp.loop_stats(loop)
        assert st["running"] == 0, "the loop did not return within 2 s of a 50 ms idle limit"
        assert st["launches"] == i + 1
    assert tapp.lib.tapp_b200_loop_destroy(loop) == 0
    for d in devs:
        d.close(tapp)


def test_loop_refuses_large_products_and_host_operands(tapp, gpu):
    err, loop = tapp.loop_create(0, blocks=1, slots=4, idle_ms=20.0)
    assert err == 0
    big = _Dev(tapp, dense_contraction_case(np.random.default_rng(2), extent=16))   # tiled CUDA-core GEMM
    err, t = tapp.loop_submit(loop, big.plan, *big.args())
    assert err == tapp_b200.ERR_UNSUPPORTED and t == -1
    small = dense_contraction_case(np.random.default_rng(3), extent=3)
    sd = _Dev(tapp, small)
    c = small
    err, t = tapp.loop_submit(loop, sd.plan, c.alpha.ctypes.data, c.A.ptr(), c.B.ptr(), c.beta.ctypes.data,
                              c.C.ptr(), c.D.ptr())
    assert err == tapp_b200.ERR_INVALID and t == -1
    st = tapp.loop_stats(loop)
    assert st["submitted"] == 0 and st["launches"] == 0
    assert tapp.lib.tapp_b200_loop_destroy(loop) == 0
    big.close(tapp)
    sd.close(tapp)

"""Serving: tapp_b200_server_* and executors carrying TAPP_B200_ATTR_SERVER.

The central property is that a product gives the same D when it runs alone
(TAPP_execute_product) and when it runs inside a mix that the server admits
against its HBM budget, packs into grouped launches and overlaps on several
streams: every product runs the same kernels with the same arguments either
way, so D is compared bit for bit. The other tests cover refusal of a
product larger than the budget, back-pressure (products wait for memory and
all complete), the validation codes of submission, the executor attribute
with concurrent callers, and the latency counters.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

import tapp_b200
from tapp_b200.server import Server, Prepared, ERR_BUDGET, ATTR_SERVER
from tapp_b200.case import alloc
from tapp_b200.workloads import dense_contraction_case, large_dense_case
from families import bounded_case

pytestmark = pytest.mark.gpu

GB = 1 << 30


def mixed_cases(seed: int, n: int):
    """Products of every path: small element-path products in all four
    compute domains (several index classes, strided views), tiled CUDA-core
    GEMMs and tensor-core products."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = i % 7
        if k == 4:
            out.append(dense_contraction_case(rng, extent=16))
        elif k == 5:
            out.append(large_dense_case(rng, tapp_b200.TAPP_BF16BF16_ACCUM_F32, tapp_b200.TAPP_F32, extent=16))
        elif k == 6:
            out.append(bounded_case(rng, n_contracted=1, n_hadamard=1, n_freeA=1, n_freeB=1, n_isoA=1,
                                    n_repB=1, subtensor=True, mixed=True, max_ext=8, max_work=2e5))
        else:
            dt = (tapp_b200.TAPP_F32, tapp_b200.TAPP_C32, tapp_b200.TAPP_F64, tapp_b200.TAPP_C64)[k]
            out.append(bounded_case(rng, dtype=dt, n_contracted=2, n_freeA=2, n_freeB=1, max_ext=12,
                                    max_work=3e5))
    return out


def alone(tapp, case):
    c = case.copy()
    err = c.run(tapp)
    assert err == 0, (case.name, tapp.explain(err))
    return c.D.buf.copy()


class DeviceCopy:
    """The four buffers of a case on the GPU (torch), addressed like the host ones."""

    def __init__(self, case):
        import torch
        self.case = case
        self.t = [torch.from_numpy(x.buf.view(np.uint8).copy()).cuda() for x in (case.A, case.B, case.C, case.D)]
        self.ptr = [t.data_ptr() + x.base * x.itemsize for t, x in zip(self.t, (case.A, case.B, case.C, case.D))]

    def D(self):
        return self.t[3].cpu().numpy().view(self.case.D.buf.dtype)


def submit(srv, prep, case, ptrs=None):
    A, B, Cp, D = ptrs if ptrs is not None else (case.A.ptr(), case.B.ptr(), case.C.ptr(), case.D.ptr())
    err, t = srv.submit(prep.plan, case.alpha.ctypes.data, A, B, case.beta.ctypes.data,
                        None if case.C_is_null else Cp, D)
    assert err == 0, (case.name, srv.tapp.explain(err))
    return t


def test_mix_matches_alone(tapp, gpu):
    cases = mixed_cases(101, 42)
    want = [alone(tapp, c) for c in cases]
    work = [c.copy() for c in cases]
    preps = [Prepared(tapp, c) for c in work]
    dev = {i: DeviceCopy(work[i]) for i in range(0, len(work), 2)}  # half on the device, half staged
    with Server(tapp, 8 * GB, n_streams=4, max_in_flight=16) as srv:
        tickets = [submit(srv, p, c, dev[i].ptr if i in dev else None) for i, (p, c) in enumerate(zip(preps, work))]
        for t in tickets:
            assert srv.wait(t) == 0
        assert srv.drain() == 0
        st = srv.stats()
    for i, c in enumerate(work):
        got = dev[i].D() if i in dev else c.D.buf
        assert np.array_equal(got.view(np.uint8), want[i].view(np.uint8)), c.name
    assert st["completed"] == st["submitted"] == len(cases)
    assert st["failed"] == 0 and st["peak_reserved"] <= st["budget_bytes"]
    for p in preps:
        p.release()


def test_budget_backpressure_and_grouping(tapp, gpu):
    """Two large products with host operands each need most of the budget,
    so the second waits for the first; the small device-resident products
    queued behind it are admitted together when memory frees up and run as
    grouped launches. Every result still matches its solo run."""
    rng = np.random.default_rng(7)
    big = [large_dense_case(rng, tapp_b200.TAPP_BF16BF16_ACCUM_F32, tapp_b200.TAPP_F32, extent=48) for _ in range(2)]
    small = [bounded_case(rng, dtype=tapp_b200.TAPP_F32, n_contracted=1, n_freeA=2, n_freeB=1, max_ext=10,
                          max_work=1e5) for _ in range(24)]
    cases = big + small
    want = [alone(tapp, c) for c in cases]
    work = [c.copy() for c in cases]
    preps = [Prepared(tapp, c) for c in work]
    dev = {i: DeviceCopy(work[i]) for i in range(2, len(work))}
    # host spans of one big product (A, B, C, D in binary32) plus its bfloat16 panels
    n = 48 ** 4
    need = 4 * n * 4 + 2 * (48 * 48) ** 2 * 2 * 2
    budget = need + need // 2
    with Server(tapp, budget, n_streams=4, max_in_flight=64) as srv:
        tickets = [submit(srv, p, c, dev[i].ptr if i in dev else None) for i, (p, c) in enumerate(zip(preps, work))]
        assert srv.drain() == 0
        st = srv.stats()
        for t in tickets:
            assert srv.wait(t) == 0
    for i, c in enumerate(work):
        got = dev[i].D() if i in dev else c.D.buf
        assert np.array_equal(got.view(np.uint8), want[i].view(np.uint8)), c.name
    assert st["budget_waits"] >= 1
    assert st["peak_reserved"] <= budget
    assert st["grouped"] >= 2
    assert st["units"] < len(cases)
    for p in preps:
        p.release()


def test_refuses_product_beyond_budget(tapp, gpu):
    rng = np.random.default_rng(8)
    # four 256 KiB host operands to stage, plus 1 MiB of split-contraction
    # sums: 2 MiB in all, more than the budget; from device memory only the
    # split sums count, and they fit
    case = dense_contraction_case(rng, extent=16)
    prep = Prepared(tapp, case)
    with Server(tapp, 1536 * 1024) as srv:
        err, t = srv.submit(prep.plan, case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(), case.beta.ctypes.data,
                            case.C.ptr(), case.D.ptr())
        assert err == ERR_BUDGET and t == -1
        assert "budget" in tapp.explain(err)
        assert srv.stats()["submitted"] == 0
        # the same product from device memory needs no budget
        d = DeviceCopy(case)
        t = submit(srv, prep, case, d.ptr)
        assert srv.wait(t) == 0
    assert np.array_equal(d.D().view(np.uint8), alone(tapp, case).view(np.uint8))
    prep.release()


def test_submit_returns_validation_codes(tapp, gpu):
    """Submission checks like TAPP_execute_product: same code, nothing queued."""
    rng = np.random.default_rng(9)
    case = dense_contraction_case(rng, extent=4)
    case.B.extents[0] += 1          # a contracted extent that differs between A and B
    case.B = alloc(case.B.dtype, case.B.extents, case.B.strides, case.B.idx)
    want = case.copy().run(tapp)
    assert want != 0
    prep = Prepared(tapp, case)
    with Server(tapp, GB) as srv:
        err, t = srv.submit(prep.plan, case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(), case.beta.ctypes.data,
                            case.C.ptr(), case.D.ptr())
        assert err == want and t == -1
        assert srv.stats()["submitted"] == 0
    prep.release()


def test_executor_attribute_with_concurrent_callers(tapp, gpu):
    """Threads calling TAPP_execute_product with an executor that carries the
    server are served together; each gets its own product's result."""
    cases = mixed_cases(202, 28)
    want = [alone(tapp, c) for c in cases]
    work = [c.copy() for c in cases]
    with Server(tapp, 8 * GB, n_streams=4, max_in_flight=32) as srv:
        ex = tapp.create_executor()
        import ctypes
        assert tapp.lib.TAPP_attr_set(ex, ATTR_SERVER, ctypes.c_void_p(srv.handle)) == 0
        errs = [None] * len(work)

        def worker(j):
            for i in range(j, len(work), 4):
                errs[i] = work[i].run(tapp, executor=ex)

        th = [threading.Thread(target=worker, args=(j,)) for j in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        st = srv.stats()
        assert tapp.lib.TAPP_attr_clear(ex, ATTR_SERVER) == 0
        tapp.lib.TAPP_destroy_executor(ex)
    assert errs == [0] * len(work)
    for i, c in enumerate(work):
        assert np.array_equal(c.D.buf.view(np.uint8), want[i].view(np.uint8)), c.name
    assert st["completed"] == len(work)


def test_latency_counters(tapp, gpu):
    cases = mixed_cases(303, 21)
    preps = [Prepared(tapp, c) for c in cases]
    with Server(tapp, 8 * GB) as srv:
        for p, c in zip(preps, cases):
            submit(srv, p, c)
        assert srv.drain() == 0
        st = srv.stats()
        assert st["completed"] == 21 and st["failed"] == 0
        assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
        assert st["requests_per_s"] > 0 and st["span_s"] > 0
        flops = 0.0
        for p in preps:
            ex = tapp.create_executor()
            tapp.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1)
            flops += plan_flops(tapp, p, ex)
            tapp.lib.TAPP_destroy_executor(ex)
        assert st["flops"] == pytest.approx(flops, rel=1e-12)
        assert srv.reset_stats() == 0
        st = srv.stats()
        assert st["completed"] == 0 and st["submitted"] == 0
    for p in preps:
        p.release()


def plan_flops(tapp, prep, ex):
    """Algorithmic flops of one product, from the status of a solo run."""
    import ctypes
    c = prep.case.copy()
    st = tapp_b200.intptr(0)
    err = tapp.lib.TAPP_execute_product(prep.plan, ex, ctypes.byref(st), c.alpha.ctypes.data, c.A.ptr(), c.B.ptr(),
                                        c.beta.ctypes.data, None if c.C_is_null else c.C.ptr(), c.D.ptr())
    assert err == 0
    f = tapp.status_value(st.value, tapp_b200.STATUS_FLOPS)
    tapp.lib.TAPP_destroy_status(st.value)
    return f


def test_served_stream_matches_plain_run(tapp, gpu):
    """A reduced stream of the served mix (Tucker mode-n, binary and
    Hadamard-plus-contraction products; f32, bf16-accum-f32, f64 and complex
    float), small shapes: every request's D from the server (all submitted at
    once, then at Poisson arrival times) equals its D from a solo synchronous
    TAPP_execute_product, bit for bit."""
    import torch
    from tapp_b200.workloads import served_stream
    from tapp_b200.served import StreamRunner
    specs = served_stream(np.random.default_rng(11), 120, max_tensor_bytes=8 << 20)
    run = StreamRunner(tapp, specs, torch, seed=3, distinct_outputs=True)
    ex = tapp.create_executor()
    run.run_plain(ex)
    torch.cuda.synchronize()
    want = [run.output(i).copy() for i in range(len(specs))]
    with Server(tapp, 64 * GB, n_streams=4, max_in_flight=32) as srv:
        for arrivals in (None, np.cumsum(np.random.default_rng(4).exponential(2e-4, len(specs)))):
            run.clear_outputs()
            st = run.run_served(srv, arrivals)
            assert st["completed"] == len(specs) and st["failed"] == 0
            for i in range(len(specs)):
                assert np.array_equal(run.output(i), want[i]), (i, specs[i])
    tapp.lib.TAPP_destroy_executor(ex)
    run.close()

"""Host-side behaviour of the serving entry points, without a GPU: argument
checks, refusal of unknown server handles (by the functions and by the
executor attribute), and the error text of the budget code. Creating a
server needs a CUDA device, so here it must fail with TAPP_B200_ERR_CUDA and
leave nothing behind."""
from __future__ import annotations

import ctypes as C

import pytest

import tapp_b200
from tapp_b200.server import bind, Counters, ERR_BUDGET, ATTR_SERVER


@pytest.fixture()
def lib(tapp):
    bind(tapp.lib)
    return tapp.lib


def test_create_checks_arguments(lib):
    h = tapp_b200.intptr(0)
    assert lib.tapp_b200_server_create(None, 0, 1 << 30, 4, 8) == tapp_b200.ERR_INVALID
    assert lib.tapp_b200_server_create(C.byref(h), 0, 0, 4, 8) == tapp_b200.ERR_INVALID
    assert lib.tapp_b200_server_create(C.byref(h), 0, 1 << 30, 0, 8) == tapp_b200.ERR_INVALID
    assert lib.tapp_b200_server_create(C.byref(h), 0, 1 << 30, 17, 8) == tapp_b200.ERR_INVALID
    assert lib.tapp_b200_server_create(C.byref(h), 0, 1 << 30, 4, 0) == tapp_b200.ERR_INVALID


def test_create_without_device_fails_cleanly(lib, tapp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = tapp_b200.intptr(0)
    assert lib.tapp_b200_server_create(C.byref(h), 0, 1 << 30, 4, 8) == tapp_b200.ERR_CUDA
    assert h.value == 0


def test_unknown_handles_are_refused(lib, tapp):
    bogus = C.create_string_buffer(4096)      # readable memory that is not a server
    hb = C.addressof(bogus)
    t = C.c_int64(0)
    for h in (0, hb):
        assert lib.tapp_b200_server_submit(h, 0, None, None, None, None, None, None, C.byref(t)) == tapp_b200.ERR_INVALID
        assert lib.tapp_b200_server_wait(h, 0) == tapp_b200.ERR_INVALID
        assert lib.tapp_b200_server_drain(h) == tapp_b200.ERR_INVALID
        assert lib.tapp_b200_server_stats(h, C.byref(Counters())) == tapp_b200.ERR_INVALID
        assert lib.tapp_b200_server_reset_stats(h) == tapp_b200.ERR_INVALID
        assert lib.tapp_b200_server_destroy(h) == tapp_b200.ERR_INVALID
    ex = tapp.create_executor()
    assert lib.TAPP_attr_set(ex, ATTR_SERVER, C.c_void_p(hb)) == tapp_b200.ERR_INVALID
    assert lib.TAPP_attr_set(ex, ATTR_SERVER, None) == 0          # detaching is always allowed
    box = C.c_void_p(1)
    assert lib.TAPP_attr_get(ex, ATTR_SERVER, C.byref(box)) == 0 and not box.value
    assert lib.TAPP_attr_clear(ex, ATTR_SERVER) == 0
    lib.TAPP_destroy_executor(ex)


def test_budget_code_text(tapp):
    assert "budget" in tapp.explain(ERR_BUDGET)
    assert not tapp.lib.TAPP_check_success(ERR_BUDGET)


def test_f64_mode_attribute(tapp):
    """TAPP_B200_ATTR_F64_MODE: 0 or 2..16 slices; the planner takes the sliced
    path for large binary64 products only when it is set."""
    import numpy as np
    from tapp_b200.workloads import double_case
    ex = tapp.create_executor()
    for bad in (1, 17, -3):
        assert tapp.set_int(ex, 0x1007, bad) == tapp_b200.ERR_INVALID
    case = double_case(np.random.default_rng(0), cplx=True, ab=16, ij=16)
    infos = [tapp.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
    _, plan = tapp.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], infos,
                                  [case.A.idx, case.B.idx, case.C.idx, case.D.idx], -1)
    assert "path=simt" in tapp.describe(plan, ex)
    assert tapp.set_int(ex, 0x1007, 8) == 0
    d = tapp.describe(plan, ex)
    assert "path=sliced" in d and "slices=8" in d and "compute=c64" in d
    box = C.c_int(0)
    p = C.c_void_p(C.addressof(box))
    assert tapp.lib.TAPP_attr_get(ex, 0x1007, C.byref(p)) == 0 and box.value == 8
    assert tapp.lib.TAPP_attr_clear(ex, 0x1007) == 0
    assert "path=simt" in tapp.describe(plan, ex)
    tapp.lib.TAPP_destroy_tensor_product(plan)
    tapp.lib.TAPP_destroy_executor(ex)

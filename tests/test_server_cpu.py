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

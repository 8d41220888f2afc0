"""Argument checks of tapp_b200_execute_chain that run before any device
work (no GPU needed): an empty chain, missing arrays, a missing final D,
and the reference's executor code."""
import ctypes as C

import tapp_b200


def test_chain_rejects_bad_arguments(tapp):
    f = tapp.lib.tapp_b200_execute_chain
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.POINTER(tapp_b200.intptr), tapp_b200.intptr] + [C.POINTER(C.c_void_p)] * 6
    ex = tapp.create_executor()
    plans = (tapp_b200.intptr * 1)(1)
    one = (C.c_void_p * 1)(1)
    none = (C.c_void_p * 1)(None)
    assert f(0, plans, ex, one, one, one, one, None, one) == tapp_b200.ERR_INVALID
    assert f(1, None, ex, one, one, one, one, None, one) == tapp_b200.ERR_INVALID
    assert f(1, plans, ex, one, one, one, one, None, none) == tapp_b200.ERR_INVALID
    assert f(1, plans, 0, one, one, one, one, None, one) == 33
    # a pointer that is not a product of this library
    bogus = C.create_string_buffer(256)
    plans[0] = C.addressof(bogus)
    assert f(1, plans, ex, one, one, one, one, None, one) == tapp_b200.ERR_INVALID
    tapp.lib.TAPP_destroy_executor(ex)

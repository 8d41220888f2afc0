"""ctypes binding of the TAPP C ABI.

The argument types follow the reference's own Python binding
(test/test.py:14-120 of the reference): handles are intptr_t, extents,
strides and labels int64 arrays, alpha/beta `void*` to a scalar of D's
storage type. Any shared library that exports the TAPP ABI can be bound —
this repository's GPU library, or the reference built from source.
"""
from __future__ import annotations

import ctypes as C
from ctypes import POINTER, c_int, c_int64, c_size_t, c_void_p, c_char_p, c_bool

intptr = C.c_ssize_t

TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16 = 0, 1, 2, 3, 4, 5
TAPP_DEFAULT_PREC = -1
TAPP_F32F32_ACCUM_F32 = 0
TAPP_F64F64_ACCUM_F64 = 1
TAPP_F16F16_ACCUM_F16 = 4
TAPP_F16F16_ACCUM_F32 = 5
TAPP_BF16BF16_ACCUM_F32 = 6
TAPP_IDENTITY, TAPP_CONJUGATE = 0, 1

ELEM_BYTES = {TAPP_F32: 4, TAPP_F64: 8, TAPP_C32: 8, TAPP_C64: 16, TAPP_F16: 2, TAPP_BF16: 2}


class TappLib:
    """Binds the TAPP entry points of one shared library."""

    def __init__(self, path: str, mode: int = C.RTLD_LOCAL):
        self.path = path
        self.lib = C.CDLL(path, mode=mode)
        L = self.lib
        L.TAPP_create_tensor_info.restype = c_int
        L.TAPP_create_tensor_info.argtypes = [POINTER(intptr), c_int, c_int, POINTER(c_int64), POINTER(c_int64)]
        L.TAPP_destroy_tensor_info.restype = c_int
        L.TAPP_destroy_tensor_info.argtypes = [intptr]
        L.TAPP_get_nmodes.restype = c_int
        L.TAPP_get_nmodes.argtypes = [intptr]
        L.TAPP_set_nmodes.restype = c_int
        L.TAPP_set_nmodes.argtypes = [intptr, c_int]
        L.TAPP_get_extents.restype = None
        L.TAPP_get_extents.argtypes = [intptr, POINTER(c_int64)]
        L.TAPP_set_extents.restype = c_int
        L.TAPP_set_extents.argtypes = [intptr, POINTER(c_int64)]
        L.TAPP_get_strides.restype = None
        L.TAPP_get_strides.argtypes = [intptr, POINTER(c_int64)]
        L.TAPP_set_strides.restype = c_int
        L.TAPP_set_strides.argtypes = [intptr, POINTER(c_int64)]
        L.TAPP_create_tensor_product.restype = c_int
        L.TAPP_create_tensor_product.argtypes = [
            POINTER(intptr), intptr,
            c_int, intptr, POINTER(c_int64),
            c_int, intptr, POINTER(c_int64),
            c_int, intptr, POINTER(c_int64),
            c_int, intptr, POINTER(c_int64),
            c_int]
        L.TAPP_destroy_tensor_product.restype = c_int
        L.TAPP_destroy_tensor_product.argtypes = [intptr]
        L.TAPP_execute_product.restype = c_int
        L.TAPP_execute_product.argtypes = [intptr, intptr, POINTER(intptr),
                                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        L.TAPP_create_executor.restype = c_int
        L.TAPP_create_executor.argtypes = [POINTER(intptr)]
        L.TAPP_destroy_executor.restype = c_int
        L.TAPP_destroy_executor.argtypes = [intptr]
        L.TAPP_create_handle.restype = c_int
        L.TAPP_create_handle.argtypes = [POINTER(intptr)]
        L.TAPP_destroy_handle.restype = c_int
        L.TAPP_destroy_handle.argtypes = [intptr]
        L.TAPP_check_success.restype = c_bool
        L.TAPP_check_success.argtypes = [c_int]
        L.TAPP_explain_error.restype = c_size_t
        L.TAPP_explain_error.argtypes = [c_int, c_size_t, c_char_p]
        self.has_batched = hasattr(L, "TAPP_execute_batched_product")
        if self.has_batched:
            L.TAPP_execute_batched_product.restype = c_int
            L.TAPP_execute_batched_product.argtypes = [
                intptr, intptr, POINTER(intptr), c_int, c_void_p,
                POINTER(c_void_p), POINTER(c_void_p), c_void_p, POINTER(c_void_p), POINTER(c_void_p)]

    # -- small helpers -------------------------------------------------
    @staticmethod
    def i64(vals):
        vals = [int(v) for v in vals]
        return (c_int64 * max(1, len(vals)))(*vals)

    def tensor_info(self, dtype: int, extents, strides) -> tuple[int, int]:
        h = intptr(0)
        err = self.lib.TAPP_create_tensor_info(C.byref(h), dtype, len(extents),
                                               self.i64(extents), self.i64(strides))
        return err, h.value

    def explain(self, err: int) -> str:
        n = self.lib.TAPP_explain_error(err, 0, None)
        buf = C.create_string_buffer(int(n) + 1)
        self.lib.TAPP_explain_error(err, n + 1, buf)
        return buf.value.decode()

    def create_executor(self) -> int:
        e = intptr(0)
        self.lib.TAPP_create_executor(C.byref(e))
        return e.value

    def create_handle(self) -> int:
        h = intptr(0)
        self.lib.TAPP_create_handle(C.byref(h))
        return h.value

    def create_product(self, handle, ops, infos, idxs, prec) -> tuple[int, int]:
        p = intptr(0)
        args = []
        for op, info, idx in zip(ops, infos, idxs):
            args += [op, info, self.i64(idx)]
        err = self.lib.TAPP_create_tensor_product(C.byref(p), handle, *args, prec)
        return err, p.value

    def execute(self, plan, executor, alpha_ptr, A, B, beta_ptr, Cp, D) -> int:
        st = intptr(0)
        return self.lib.TAPP_execute_product(plan, executor, C.byref(st), alpha_ptr, A, B, beta_ptr, Cp, D)

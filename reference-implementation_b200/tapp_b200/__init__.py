"""B200 implementation of the TAPP tensor product — Python side.

The product itself is the shared library lib/libtapp-b200.so (C host code
plus CUDA kernels for sm_100a). This package binds its C ABI with ctypes the
way the reference's own Python test does (test/test.py:14-185 of the
reference), and adds helpers for device buffers (torch tensors) and for the
benchmark workloads. There is no CPU fallback: without the built library,
`load()` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from .abi import (TappLib, TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16,  # noqa: F401
                  TAPP_DEFAULT_PREC, TAPP_F32F32_ACCUM_F32, TAPP_F64F64_ACCUM_F64,
                  TAPP_F16F16_ACCUM_F16, TAPP_F16F16_ACCUM_F32, TAPP_BF16BF16_ACCUM_F32,
                  TAPP_IDENTITY, TAPP_CONJUGATE, ELEM_BYTES, intptr)

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "lib", "libtapp-b200.so")
INCLUDE_DIR = os.path.join(REPO_DIR, "include")

# implementation-defined keys and codes (include/tapp_b200.h)
ERR_CUDA, ERR_LIMIT, ERR_UNSUPPORTED, ERR_NOMEM, ERR_INVALID, ERR_LABELS = 0x1001, 0x1002, 0x1003, 0x1004, 0x1005, 0x1006
ATTR_STREAM, ATTR_ASYNC, ATTR_F32_MODE, ATTR_PATH, ATTR_WANT_STATUS = 0x1000, 0x1001, 0x1002, 0x1004, 0x1005
ATTR_F64_MODE, ATTR_TILE = 0x1007, 0x1008
STATUS_PATH, STATUS_KERNELS, STATUS_FLOPS, STATUS_DEVICE_US, STATUS_TC_MODE, STATUS_MAIN_US = (
    0x1100, 0x1101, 0x1102, 0x1103, 0x1104, 0x1105)
STATUS_ERR_BOUND = 0x1106
PATH_NOOP, PATH_GENERIC, PATH_REDUCE, PATH_SIMT, PATH_TC = 0, 1, 2, 3, 4

_lib: "B200Lib | None" = None


def build(jobs: int = 8) -> str:
    """Compiles the library in-tree (make) and returns its path."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", PKG_DIR], check=True)
    return LIB_PATH


class LoopCounters(C.Structure):
    """tapp_b200_loop_counters (include/tapp_b200.h)."""
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("launches", C.c_int64),
                ("running", C.c_int32), ("pad", C.c_int32), ("p50_us", C.c_double), ("p99_us", C.c_double),
                ("mean_us", C.c_double), ("max_us", C.c_double)]


class B200Lib(TappLib):
    """TappLib plus the implementation-defined entry points."""

    def __init__(self, path: str = LIB_PATH):
        super().__init__(path)
        L = self.lib
        L.tapp_b200_describe_plan.restype = C.c_size_t
        L.tapp_b200_describe_plan.argtypes = [intptr, intptr, C.c_size_t, C.c_char_p]
        L.tapp_b200_kernel_launches.restype = C.c_longlong
        L.tapp_b200_kernel_launches.argtypes = []
        L.tapp_b200_device_allocations.restype = C.c_longlong
        L.tapp_b200_device_allocations.argtypes = []
        L.tapp_b200_execute_group.restype = C.c_int
        L.tapp_b200_execute_group.argtypes = [C.c_int, C.POINTER(intptr), intptr] + [C.POINTER(C.c_void_p)] * 6
        L.tapp_b200_load_tile_table.restype = C.c_int
        L.tapp_b200_load_tile_table.argtypes = [C.c_char_p]
        for name, args in (("tapp_b200_loop_create", [C.POINTER(intptr), intptr, C.c_int, C.c_int, C.c_double]),
                           ("tapp_b200_loop_submit", [intptr, intptr] + [C.c_void_p] * 6 + [C.POINTER(C.c_int64)]),
                           ("tapp_b200_loop_wait", [intptr, C.c_int64]),
                           ("tapp_b200_loop_stats", [intptr, C.POINTER(LoopCounters)]),
                           ("tapp_b200_loop_reset_stats", [intptr]),
                           ("tapp_b200_loop_destroy", [intptr])):
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = args
        L.TAPP_attr_set.restype = C.c_int
        L.TAPP_attr_set.argtypes = [intptr, C.c_int, C.c_void_p]
        L.TAPP_attr_get.restype = C.c_int
        L.TAPP_attr_get.argtypes = [intptr, C.c_int, C.POINTER(C.c_void_p)]
        L.TAPP_attr_clear.restype = C.c_int
        L.TAPP_attr_clear.argtypes = [intptr, C.c_int]
        L.TAPP_destroy_status.restype = C.c_int
        L.TAPP_destroy_status.argtypes = [intptr]

    def set_int(self, executor: int, key: int, value: int) -> int:
        v = C.c_int(value)
        return self.lib.TAPP_attr_set(executor, key, C.cast(C.byref(v), C.c_void_p))

    def set_stream(self, executor: int, stream_handle: int) -> int:
        return self.lib.TAPP_attr_set(executor, ATTR_STREAM, C.c_void_p(stream_handle))

    def status_value(self, status: int, key: int):
        if key in (STATUS_FLOPS, STATUS_DEVICE_US, STATUS_MAIN_US, STATUS_ERR_BOUND):
            box = C.c_double(0.0)
        else:
            box = C.c_int(0)
        p = C.c_void_p(C.addressof(box))
        err = self.lib.TAPP_attr_get(status, key, C.byref(p))
        if err:
            raise RuntimeError(f"TAPP_attr_get({key:#x}) failed: {err}")
        return box.value

    def describe(self, plan: int, executor: int = 0) -> str:
        n = self.lib.tapp_b200_describe_plan(plan, executor, 0, None)
        buf = C.create_string_buffer(int(n) + 1)
        self.lib.tapp_b200_describe_plan(plan, executor, n + 1, buf)
        return buf.value.decode()

    def launches(self) -> int:
        return int(self.lib.tapp_b200_kernel_launches())

    def allocations(self) -> int:
        return int(self.lib.tapp_b200_device_allocations())

    def execute_group(self, plans, executor, alphas, betas, A, B, Cs, D) -> int:
        """tapp_b200_execute_group over lists (pointers as ints, Cs may hold None)."""
        n = len(plans)
        arr = lambda v: (C.c_void_p * n)(*v)
        return int(self.lib.tapp_b200_execute_group(n, (intptr * n)(*plans), executor, arr(alphas), arr(betas),
                                                    arr(A), arr(B), arr(Cs), arr(D)))

    def loop_create(self, executor=0, blocks=4, slots=256, idle_ms=100.0) -> tuple[int, int]:
        h = intptr(0)
        err = self.lib.tapp_b200_loop_create(C.byref(h), executor, blocks, slots, idle_ms)
        return err, h.value

    def loop_submit(self, loop, plan, alpha_ptr, A, B, beta_ptr, Cp, D) -> tuple[int, int]:
        t = C.c_int64(-1)
        err = self.lib.tapp_b200_loop_submit(loop, plan, alpha_ptr, A, B, beta_ptr, Cp, D, C.byref(t))
        return err, t.value

    def loop_stats(self, loop) -> dict:
        c = LoopCounters()
        assert self.lib.tapp_b200_loop_stats(loop, C.byref(c)) == 0
        return {f: getattr(c, f) for f, _ in LoopCounters._fields_ if f != "pad"}

    def load_tile_table(self, path: str | None) -> int:
        return int(self.lib.tapp_b200_load_tile_table(None if path is None else path.encode()))


def load() -> B200Lib:
    """The process-wide binding of lib/libtapp-b200.so. Raises if the library
    has not been built (there is no other implementation to fall back to)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                               "(or __graft_entry__.build())")
        _lib = B200Lib(LIB_PATH)
    return _lib

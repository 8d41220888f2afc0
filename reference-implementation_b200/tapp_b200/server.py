"""ctypes binding of the serving entry points (tapp_b200_server_*).

A `Server` queues products on one GPU and runs them as they arrive: see
include/tapp_b200.h for the semantics (HBM-budget admission, streams,
grouped launches, latency counters). `Prepared` holds the tensor infos and
the product object of one `Case`, so that the same product can be submitted
many times without re-creating them.
"""
from __future__ import annotations

import ctypes as C

from .abi import intptr

ERR_BUDGET = 0x1008
ATTR_SERVER = 0x1006


class Counters(C.Structure):
    """tapp_b200_server_counters"""
    _fields_ = [
        ("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
        ("units", C.c_int64), ("grouped", C.c_int64), ("budget_waits", C.c_int64),
        ("peak_in_flight", C.c_int64), ("budget_bytes", C.c_int64), ("peak_reserved", C.c_int64),
        ("p50_us", C.c_double), ("p99_us", C.c_double), ("mean_us", C.c_double), ("max_us", C.c_double),
        ("span_s", C.c_double), ("requests_per_s", C.c_double), ("flops", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def bind(lib) -> None:
    """Declares the argument types of the server entry points on a CDLL."""
    if getattr(lib, "_server_bound", False):
        return
    lib.tapp_b200_server_create.restype = C.c_int
    lib.tapp_b200_server_create.argtypes = [C.POINTER(intptr), intptr, C.c_int64, C.c_int, C.c_int]
    lib.tapp_b200_server_submit.restype = C.c_int
    lib.tapp_b200_server_submit.argtypes = [intptr, intptr] + [C.c_void_p] * 6 + [C.POINTER(C.c_int64)]
    lib.tapp_b200_server_wait.restype = C.c_int
    lib.tapp_b200_server_wait.argtypes = [intptr, C.c_int64]
    lib.tapp_b200_server_drain.restype = C.c_int
    lib.tapp_b200_server_drain.argtypes = [intptr]
    lib.tapp_b200_server_stats.restype = C.c_int
    lib.tapp_b200_server_stats.argtypes = [intptr, C.POINTER(Counters)]
    lib.tapp_b200_server_reset_stats.restype = C.c_int
    lib.tapp_b200_server_reset_stats.argtypes = [intptr]
    lib.tapp_b200_server_destroy.restype = C.c_int
    lib.tapp_b200_server_destroy.argtypes = [intptr]
    lib._server_bound = True


class Server:
    def __init__(self, tapp, budget_bytes: int, n_streams: int = 4, max_in_flight: int = 64, executor: int = 0):
        self.tapp = tapp
        self.lib = tapp.lib
        bind(self.lib)
        h = intptr(0)
        err = self.lib.tapp_b200_server_create(C.byref(h), executor, int(budget_bytes), n_streams, max_in_flight)
        if err:
            raise RuntimeError(f"tapp_b200_server_create: {err:#x} {tapp.explain(err)}")
        self.handle = h.value

    def submit(self, plan: int, alpha_ptr, A, B, beta_ptr, Cp, D) -> tuple[int, int]:
        """(code, ticket); ticket is -1 when the code is not 0."""
        t = C.c_int64(-1)
        err = self.lib.tapp_b200_server_submit(self.handle, plan, alpha_ptr, A, B, beta_ptr, Cp, D, C.byref(t))
        return err, t.value

    def wait(self, ticket: int) -> int:
        return self.lib.tapp_b200_server_wait(self.handle, ticket)

    def drain(self) -> int:
        return self.lib.tapp_b200_server_drain(self.handle)

    def stats(self) -> dict:
        c = Counters()
        err = self.lib.tapp_b200_server_stats(self.handle, C.byref(c))
        if err:
            raise RuntimeError(f"tapp_b200_server_stats: {err:#x}")
        return c.as_dict()

    def reset_stats(self) -> int:
        return self.lib.tapp_b200_server_reset_stats(self.handle)

    def close(self) -> int:
        if not self.handle:
            return 0
        err = self.lib.tapp_b200_server_destroy(self.handle)
        self.handle = 0
        return err

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Prepared:
    """Tensor infos and product object of a Case, kept for repeated use."""

    def __init__(self, tapp, case, handle: int = 0):
        self.tapp = tapp
        self.case = case
        self.infos = []
        for t in (case.A, case.B, case.C, case.D):
            err, h = tapp.tensor_info(t.dtype, t.extents, t.strides)
            if err:
                raise RuntimeError(f"TAPP_create_tensor_info: {err}")
            self.infos.append(h)
        err, self.plan = tapp.create_product(handle, [case.A.op, case.B.op, case.C.op, case.D.op], self.infos,
                                             [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
        if err:
            raise RuntimeError(f"TAPP_create_tensor_product: {err}")

    def release(self) -> None:
        if self.plan:
            self.tapp.lib.TAPP_destroy_tensor_product(self.plan)
            for h in self.infos:
                self.tapp.lib.TAPP_destroy_tensor_info(h)
            self.plan = 0

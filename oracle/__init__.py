"""ctypes binding of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loaded by the tests, the smoke check and the CPU-baseline leg of the
benchmark, never by the GPU library. `Oracle` wraps build/liboracle.so (this
repository's C restatement of the reference's product); `reference_lib()`
binds the reference itself when it was built from its sources into _ref/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libtapp-reference.so")
REF_LIB_F16 = os.path.join(HERE, "_ref", "libtapp-reference-f16.so")


class _OTensor(C.Structure):
    _fields_ = [("type", C.c_int32), ("nmode", C.c_int32), ("op", C.c_int32), ("reserved", C.c_int32),
                ("extents", C.POINTER(C.c_int64)), ("strides", C.POINTER(C.c_int64)),
                ("idx", C.POINTER(C.c_int64))]


def build(reference_dir: str | None = None) -> None:
    """Compile the oracle; with `reference_dir` (or TAPP_REFERENCE_DIR) naming
    a checkout of the reference whose sources are present, also build the
    reference itself into _ref/."""
    targets = ["all"]
    env = dict(os.environ)
    ref = reference_dir or env.get("TAPP_REFERENCE_DIR")
    if ref and os.path.isfile(os.path.join(ref, "reference_implementation", "src", "product.c")):
        targets.append("ref")
        env["REF"] = ref
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True, env=env)


def _arr(vals):
    vals = [int(v) for v in vals]
    return (C.c_int64 * max(1, len(vals)))(*vals)


class Oracle:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        P = C.POINTER(_OTensor)
        self.lib.oracle_validate.restype = C.c_int
        self.lib.oracle_validate.argtypes = [P, P, P, P, C.c_void_p, C.c_int]
        self.lib.oracle_execute.restype = C.c_int
        self.lib.oracle_execute.argtypes = [C.c_int, P, P, P, P] + [C.c_void_p] * 6
        self.lib.oracle_execute_f64.restype = C.c_int
        self.lib.oracle_execute_f64.argtypes = [C.c_int, P, P, P, P] + [C.c_void_p] * 5 + [
            C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.oracle_folded_size.restype = C.c_int64
        self.lib.oracle_folded_size.argtypes = [P]

    @staticmethod
    def _t(t):
        keep = (_arr(t.extents), _arr(t.strides), _arr(t.idx))
        s = _OTensor(t.dtype, t.nmode, t.op, 0, keep[0], keep[1], keep[2])
        return s, keep

    def _four(self, case):
        out, keep = [], []
        for t in (case.A, case.B, case.C, case.D):
            s, k = self._t(t)
            out.append(s)
            keep.append(k)
        return out, keep

    def validate(self, case) -> int:
        (a, b, c, d), _k = self._four(case)
        return self.lib.oracle_validate(C.byref(a), C.byref(b), C.byref(c), C.byref(d),
                                        case.beta.ctypes.data, 0 if case.C_is_null else 1)

    def execute(self, case) -> int:
        """Reference-faithful product; writes case.D.buf in place."""
        (a, b, c, d), _k = self._four(case)
        return self.lib.oracle_execute(case.prec, C.byref(a), C.byref(b), C.byref(c), C.byref(d),
                                       case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(),
                                       case.beta.ctypes.data, None if case.C_is_null else case.C.ptr(),
                                       case.D.ptr())

    def folded_size(self, case) -> int:
        d, _k = self._t(case.D)
        return int(self.lib.oracle_folded_size(C.byref(d)))

    def execute_f64(self, case, samples=None):
        """Binary64 product. Without samples: (err, D64, scale), both laid out
        like case.D.buf (complex128 / float64 buffers with the same base).
        With samples (linear indices over D's merged modes): (err, D64[n],
        scale[n], D_offsets[n])."""
        (a, b, c, d), _k = self._four(case)
        args = (case.prec, C.byref(a), C.byref(b), C.byref(c), C.byref(d),
                case.alpha.ctypes.data, case.A.ptr(), case.B.ptr(),
                case.beta.ctypes.data, None if case.C_is_null else case.C.ptr())
        if samples is None:
            n = case.D.buf.size
            D64 = np.zeros(n, dtype=np.complex128)
            cur = case.D.buf
            if cur.dtype == np.uint16:
                from tapp_b200.case import bf16_to_f32
                D64[:] = bf16_to_f32(cur)
            else:
                D64[:] = cur
            scale = np.zeros(n, dtype=np.float64)
            base = case.D.base
            err = self.lib.oracle_execute_f64(*args, -1, None,
                                              D64.ctypes.data + 16 * base, scale.ctypes.data + 8 * base, None)
            return err, D64, scale
        samples = np.ascontiguousarray(samples, dtype=np.int64)
        n = samples.size
        D64 = np.zeros(n, dtype=np.complex128)
        scale = np.zeros(n, dtype=np.float64)
        offs = np.zeros(n, dtype=np.int64)
        err = self.lib.oracle_execute_f64(*args, n, samples.ctypes.data, D64.ctypes.data,
                                          scale.ctypes.data, offs.ctypes.data)
        return err, D64, scale, offs


def reference_lib(f16: bool = False):
    """TappLib bound to the reference built from its sources, or None."""
    path = REF_LIB_F16 if f16 else REF_LIB
    if not os.path.exists(path):
        return None
    from tapp_b200.abi import TappLib
    return TappLib(path)

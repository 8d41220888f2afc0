"""Host-side description of one tensor product and its operand buffers.

A `Tensor` is a TAPP tensor info (storage type, extents, strides in
elements, labels, element op) together with a flat numpy buffer that covers
every element the strides address; `base` is the element index of
coordinate 0 inside that buffer, so negative strides reach below it, as the
reference's own tests do (test/test.cpp:996-1031, test/demo.c:1043-1044).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from .abi import (TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16,
                  ELEM_BYTES)

NP_DTYPE = {
    TAPP_F32: np.float32,
    TAPP_F64: np.float64,
    TAPP_C32: np.complex64,
    TAPP_C64: np.complex128,
    TAPP_F16: np.float16,
    TAPP_BF16: np.uint16,  # raw bfloat16 bit patterns
}


def is_complex(dtype: int) -> bool:
    return dtype in (TAPP_C32, TAPP_C64)


def span(extents, strides) -> tuple[int, int, bool]:
    """(lowest, highest) element offset a layout addresses, and whether it
    addresses any element at all."""
    lo = hi = 0
    for e, s in zip(extents, strides):
        if e == 0:
            return 0, 0, False
        if s < 0:
            lo += s * (e - 1)
        else:
            hi += s * (e - 1)
    return lo, hi, True


def bf16_from_f32(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 bit patterns (nearest, ties to even)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    nan = np.isnan(x)
    out = rounded.astype(np.uint16)
    out[nan] = 0x7FC0
    return out


def bf16_to_f32(h: np.ndarray) -> np.ndarray:
    return (np.asarray(h, dtype=np.uint32) << 16).view(np.float32)


@dataclass
class Tensor:
    dtype: int
    extents: list
    strides: list
    idx: list
    op: int = 0
    buf: np.ndarray | None = None
    base: int = 0

    @property
    def nmode(self) -> int:
        return len(self.extents)

    @property
    def itemsize(self) -> int:
        return ELEM_BYTES[self.dtype]

    def ptr(self) -> int | None:
        """Host address of coordinate 0 (None when there is no buffer)."""
        if self.buf is None:
            return None
        return self.buf.ctypes.data + self.base * self.itemsize

    def offsets(self) -> np.ndarray:
        """Element offsets (relative to coordinate 0) of every coordinate,
        first mode fastest."""
        off = np.zeros(1, dtype=np.int64)
        for e, s in zip(self.extents, self.strides):
            # each later mode varies slower than all earlier ones
            off = ((np.arange(e, dtype=np.int64) * s)[:, None] + off[None, :]).reshape(-1)
        return off

    def copy(self) -> "Tensor":
        return Tensor(self.dtype, list(self.extents), list(self.strides), list(self.idx), self.op,
                      None if self.buf is None else self.buf.copy(), self.base)


def alloc(dtype: int, extents, strides, idx, op=0, pad_lo=0, pad_hi=0) -> Tensor:
    """Zero buffer covering the addressed span plus optional padding."""
    lo, hi, any_ = span(extents, strides)
    n = (hi - lo + 1 if any_ else 1) + pad_lo + pad_hi
    buf = np.zeros(n, dtype=NP_DTYPE[dtype])
    return Tensor(dtype, list(extents), list(strides), list(idx), op, buf, -lo + pad_lo)


def fill_uniform(t: Tensor, rng: np.random.Generator, lo=-1.0, hi=1.0) -> Tensor:
    n = t.buf.size
    if t.dtype in (TAPP_C32, TAPP_C64):
        t.buf[:] = rng.uniform(lo, hi, n) + 1j * rng.uniform(lo, hi, n)
    elif t.dtype == TAPP_BF16:
        t.buf[:] = bf16_from_f32(rng.uniform(lo, hi, n).astype(np.float32))
    else:
        t.buf[:] = rng.uniform(lo, hi, n)
    return t


def scalar(dtype: int, value) -> np.ndarray:
    """A one-element array of `dtype` holding `value` (alpha / beta)."""
    if dtype == TAPP_BF16:
        return bf16_from_f32(np.array([np.real(value)], dtype=np.float32))
    a = np.zeros(1, dtype=NP_DTYPE[dtype])
    a[0] = value if is_complex(dtype) else np.real(value)
    return a


@dataclass
class Case:
    """One call of TAPP_execute_product: four tensors, scalars, precision."""
    A: Tensor
    B: Tensor
    C: Tensor
    D: Tensor
    alpha: np.ndarray
    beta: np.ndarray
    prec: int = -1
    C_is_null: bool = False
    name: str = ""

    def copy(self) -> "Case":
        return Case(self.A.copy(), self.B.copy(), self.C.copy(), self.D.copy(),
                    self.alpha.copy(), self.beta.copy(), self.prec, self.C_is_null, self.name)

    def run(self, tapp, executor=None, handle=0, D_ptr=None, A_ptr=None, B_ptr=None, C_ptr=None):
        """Execute through any TAPP library binding (`abi.TappLib`); the
        result lands in self.D.buf unless other pointers are given."""
        infos = []
        for t in (self.A, self.B, self.C, self.D):
            err, h = tapp.tensor_info(t.dtype, t.extents, t.strides)
            assert err == 0, err
            infos.append(h)
        err, plan = tapp.create_product(handle, [self.A.op, self.B.op, self.C.op, self.D.op], infos,
                                        [self.A.idx, self.B.idx, self.C.idx, self.D.idx], self.prec)
        assert err == 0
        own_exec = executor is None
        if own_exec:
            executor = tapp.create_executor()
        try:
            err = tapp.execute(plan, executor,
                               self.alpha.ctypes.data,
                               A_ptr if A_ptr is not None else self.A.ptr(),
                               B_ptr if B_ptr is not None else self.B.ptr(),
                               self.beta.ctypes.data,
                               None if self.C_is_null else (C_ptr if C_ptr is not None else self.C.ptr()),
                               D_ptr if D_ptr is not None else self.D.ptr())
        finally:
            if own_exec:
                tapp.lib.TAPP_destroy_executor(executor)
            tapp.lib.TAPP_destroy_tensor_product(plan)
            for h in infos:
                tapp.lib.TAPP_destroy_tensor_info(h)
        return err

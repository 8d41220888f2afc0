"""Shared test helpers: golden-record decoding, error bounds, device runs."""
from __future__ import annotations

import json
import os

import numpy as np

from tapp_b200.abi import TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16
from tapp_b200.case import Case, Tensor, NP_DTYPE, is_complex, bf16_to_f32

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_records():
    with open(os.path.join(GOLDEN, "reference_programs.jsonl")) as f:
        return [json.loads(l) for l in f]


def _values(dtype, data):
    if dtype in (TAPP_C32, TAPP_C64):
        return np.array([complex(re, im) for re, im in data], dtype=NP_DTYPE[dtype])
    return np.array([re for re, _ in data], dtype=NP_DTYPE[dtype])


def case_from_record(rec) -> tuple[Case, np.ndarray]:
    """Rebuilds the call a golden record describes; returns the case (D as it
    was before the call) and the reference's D span after the call."""
    ts = []
    for t in rec["tensors"]:
        span = t["span"]
        data = span["data"]
        buf = _values(t["type"], data) if data else np.zeros(1, dtype=NP_DTYPE[t["type"]])
        ts.append(Tensor(t["type"], t["extents"], t["strides"], t["idx"], t["op"], buf, -span["lo"]))
    tD = rec["tensors"][3]["type"]
    def scal(v):
        a = np.zeros(1, dtype=NP_DTYPE[tD])
        a[0] = complex(v[0], v[1]) if is_complex(tD) else v[0]
        return a
    case = Case(*ts, scal(rec["alpha"]), scal(rec["beta"]), rec["prec"], rec["tensors"][2]["null"],
                f"{rec['program']}#{rec['call']}")
    after = _values(tD, rec["D_after"]["data"]) if rec["D_after"]["data"] else np.zeros(0, dtype=NP_DTYPE[tD])
    return case, after


def folded_sizes(case: Case) -> tuple[int, int, int]:
    """(contracted, unary-A, unary-B) sizes after repeated labels merge."""
    def fold(t):
        d = {}
        for l, e in zip(t.idx, t.extents):
            d[l] = e
        return d
    a, b, d = fold(case.A), fold(case.B), fold(case.D)
    K = int(np.prod([e for l, e in a.items() if l in b and l not in d], dtype=np.int64))
    UA = int(np.prod([e for l, e in a.items() if l not in b and l not in d], dtype=np.int64))
    UB = int(np.prod([e for l, e in b.items() if l not in a and l not in d], dtype=np.int64))
    return K, UA, UB


UNIT = {"f64": 2.0 ** -53, "f32": 2.0 ** -24, "f16": 2.0 ** -11, "bf16": 2.0 ** -8}


def compute_unit(case: Case) -> float:
    """Unit roundoff of the arithmetic the product runs in."""
    types = [case.A.dtype, case.B.dtype, case.D.dtype] + ([] if case.C_is_null else [case.C.dtype])
    if case.prec == 1 or (case.prec == -1 and any(t in (TAPP_F64, TAPP_C64) for t in types)):
        return UNIT["f64"]
    return UNIT["f32"]


def output_unit(dtype: int) -> float:
    return {TAPP_F32: UNIT["f32"], TAPP_C32: UNIT["f32"], TAPP_F64: UNIT["f64"], TAPP_C64: UNIT["f64"],
            TAPP_F16: UNIT["f16"], TAPP_BF16: UNIT["bf16"]}[dtype]


def error_bound(case: Case, scale: np.ndarray, D64: np.ndarray, extra_rel: float = 0.0) -> np.ndarray:
    """Per-element bound on |D_gpu - D_64|.

    Summation of n terms in any order in a format with unit roundoff u errs
    by at most gamma_n * sum|terms| with gamma_n = n u / (1 - n u)
    (N. J. Higham, Accuracy and Stability of Numerical Algorithms, 2nd ed.,
    section 3.1 and 4.2); `scale` is |alpha| sum|a||b| + |beta||c| from the
    oracle. n counts the contracted and unary terms plus the alpha/beta
    operations and a complex multiply; the result is then rounded to D's
    type. `extra_rel` adds a relative term for operand splitting (split
    bfloat16) or 16-bit unary sums."""
    K, UA, UB = folded_sizes(case)
    n = K * max(UA, 1) + UA + UB + 8
    u = compute_unit(case)
    gamma = n * u / (1 - n * u)
    if case.prec in (4, 5, 6) and max(UA, UB) > 1:
        # the 16-bit precisions keep running unary sums in 16 bits, rounding
        # after every addition (product.c:1958-2017); each rounding errs by at
        # most u16 times the sum of magnitudes seen so far
        u16 = UNIT["bf16"] if case.prec == 6 else UNIT["f16"]
        extra_rel += (UA + UB) * u16
    return (gamma + extra_rel) * scale + 2 * output_unit(case.D.dtype) * np.abs(D64) + 1e-300


def d_values(t: Tensor) -> np.ndarray:
    """D buffer as complex128 (bf16 decoded)."""
    if t.dtype == TAPP_BF16:
        return bf16_to_f32(t.buf).astype(np.complex128)
    return t.buf.astype(np.complex128)


def run_on_device(tapp, case: Case, executor=None):
    """Copies the case's buffers to the GPU, runs through the C ABI with
    device pointers, and copies D back into case.D.buf. Returns the code."""
    import torch
    dev = []
    ptrs = []
    for t in (case.A, case.B, case.C, case.D):
        raw = torch.from_numpy(t.buf.view(np.uint8).copy()).cuda()
        dev.append(raw)
        ptrs.append(raw.data_ptr() + t.base * t.itemsize)
    err = case.run(tapp, executor=executor, A_ptr=ptrs[0], B_ptr=ptrs[1], C_ptr=ptrs[2], D_ptr=ptrs[3])
    torch.cuda.synchronize()
    case.D.buf[:] = dev[3].cpu().numpy().view(case.D.buf.dtype)
    return err

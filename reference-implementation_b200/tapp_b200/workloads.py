"""Synthetic benchmark workloads (seeded), one builder per configuration.

  dense_contraction_case  D[a,b,c,d] = 1.3 sum_{e,f} A[a,e,b,f] B[f,c,e,d] + 0.7 C,
                          all extents 16, dense column-major, U[-1,1]
  mixed_classes_case      D[a,h,c] = alpha sum_{k,u,v} A[a,h,k,k,u] conj(B[k,h,c,v]) + beta C,
                          complex float; a=40 h=12 k=24 u=6 c=36 v=5; A a strided
                          view with a negative stride on a and a zero stride on u;
                          D permuted relative to C
  large_dense_case        D[a,b,i,j] = sum_{c,d} A[a,c,i,d] B[d,b,c,j] + 0.5 C, all
                          extents 64 (M = N = K = 4096); N(0,1) with 1% of the
                          entries scaled by 1e3
  double_case             D[a,b,i,j] = sum_{e,f} A[a,b,e,f] B[e,f,i,j] + C,
                          a=b=e=f=160, i=j=40; |x| log-uniform in [1e-8, 1], random
                          sign (float64) or phase (complex double, conj(A))
The data are synthetic stand-ins with the shapes and value distributions the
benchmark configurations specify; nothing is read from disk.
"""
from __future__ import annotations

import numpy as np

from .abi import TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16, TAPP_CONJUGATE
from .case import Case, Tensor, alloc, scalar, bf16_from_f32, NP_DTYPE

L = {ch: ord(ch) for ch in "abcdefhijkuv"}


def colmajor(extents):
    s, acc = [], 1
    for e in extents:
        s.append(acc)
        acc *= e
    return s


def dense_contraction_case(rng, extent=16, dtype=TAPP_F32, prec=TAPP_F32, alpha=1.3, beta=0.7) -> Case:
    e = extent
    def t(idx, ty=dtype):
        ext = [e] * len(idx)
        T = alloc(ty, ext, colmajor(ext), [L[c] for c in idx])
        n = T.buf.size
        if ty in (TAPP_C32, TAPP_C64):
            T.buf[:] = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        else:
            T.buf[:] = rng.uniform(-1, 1, n)
        return T
    A, B, C, D = t("aebf"), t("fced"), t("abcd"), t("abcd")
    return Case(A, B, C, D, scalar(dtype, alpha), scalar(dtype, beta), prec, False, f"dense_contraction_{e}")


def mixed_classes_case(rng) -> Case:
    a, h, k, u, c, v = 40, 12, 24, 6, 36, 5
    cplx = lambda n: (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
    # A[a,h,k,k,u]: view into a [44,12,24,24] buffer, a running downwards,
    # u broadcast (stride 0), k taken on its diagonal
    a_out = a + 4
    sA = [-1, a_out, a_out * h, a_out * h * k, 0]
    A = alloc(TAPP_C32, [a, h, k, k, u], sA, [L["a"], L["h"], L["k"], L["k"], L["u"]], 0, pad_lo=2, pad_hi=0)
    A.buf[:] = cplx(A.buf.size)
    eB = [k, h, c, v]
    B = alloc(TAPP_C32, eB, colmajor(eB), [L["k"], L["h"], L["c"], L["v"]], TAPP_CONJUGATE)
    B.buf[:] = cplx(B.buf.size)
    eD = [a, h, c]
    C = alloc(TAPP_C32, eD, colmajor(eD), [L["a"], L["h"], L["c"]])
    C.buf[:] = cplx(C.buf.size)
    # D stored with c fastest, then a, then h
    sD = [c, c * a, 1]
    D = alloc(TAPP_C32, eD, sD, [L["a"], L["h"], L["c"]])
    D.buf[:] = cplx(D.buf.size)
    al = complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
    be = complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
    return Case(A, B, C, D, scalar(TAPP_C32, al), scalar(TAPP_C32, be), -1, False, "mixed_classes")


def outlier_normal(rng, n, frac=0.01, scale=1e3):
    x = rng.standard_normal(n).astype(np.float32)
    m = rng.random(n) < frac
    x[m] *= scale
    return x


def large_dense_case(rng, prec, storage=TAPP_F32, extent=64, beta=0.5) -> Case:
    """storage: TAPP_F32 (operands rounded per precision inside the product)
    or TAPP_BF16 / TAPP_F16 (16-bit A and B, binary32 C and D)."""
    e = extent
    def t(idx, ty):
        ext = [e] * 4
        T = alloc(ty, ext, colmajor(ext), [L[c] for c in idx])
        x = outlier_normal(rng, T.buf.size)
        if ty == TAPP_BF16:
            T.buf[:] = bf16_from_f32(x)
        else:
            T.buf[:] = x.astype(NP_DTYPE[ty])
        return T
    A = t("acid", storage)
    B = t("dbcj", storage)
    C = t("abij", TAPP_F32)
    D = alloc(TAPP_F32, [e] * 4, colmajor([e] * 4), [L[c] for c in "abij"])
    return Case(A, B, C, D, scalar(TAPP_F32, 1.0), scalar(TAPP_F32, beta), prec, False, f"large_dense_{e}")


def loguniform(rng, n, cplx):
    mag = 10.0 ** rng.uniform(-8, 0, n)
    if cplx:
        return mag * np.exp(2j * np.pi * rng.random(n))
    return mag * rng.choice([-1.0, 1.0], n)


def double_case(rng, cplx=False, ab=160, ij=40, beta=1.0) -> Case:
    ty = TAPP_C64 if cplx else TAPP_F64
    def t(idx, ext, op=0):
        T = alloc(ty, ext, colmajor(ext), [L[c] for c in idx], op)
        T.buf[:] = loguniform(rng, T.buf.size, cplx)
        return T
    A = t("abef", [ab, ab, ab, ab], TAPP_CONJUGATE if cplx else 0)
    B = t("efij", [ab, ab, ij, ij])
    C = t("abij", [ab, ab, ij, ij])
    D = alloc(ty, [ab, ab, ij, ij], colmajor([ab, ab, ij, ij]), [L[c] for c in "abij"])
    return Case(A, B, C, D, scalar(ty, 1.0), scalar(ty, beta), -1, False, "double_" + ("c64" if cplx else "f64"))

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
  served_stream           the request mix of the served configuration: 50% Tucker
                          mode-n products (order-3/4 core, extents 8..256, factor
                          rank 4..64, random mode), 30% binary contractions with
                          2..6 indices of extent 4..96, 20% Hadamard plus
                          contraction; 40% f32, 30% bf16-accum-f32, 20% f64, 10%
                          complex float; specifications only (shapes, labels,
                          scalars), the data come from the runner
The data are synthetic stand-ins with the shapes and value distributions the
benchmark configurations specify; nothing is read from disk.
"""
from __future__ import annotations

import numpy as np

from dataclasses import dataclass

from .abi import (TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16, TAPP_CONJUGATE, ELEM_BYTES,
                  TAPP_DEFAULT_PREC, TAPP_F32F32_ACCUM_F32, TAPP_BF16BF16_ACCUM_F32)
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


@dataclass
class RequestSpec:
    """One served product: storage type of all four tensors, precision,
    extents and labels of A, B, C, D (dense column-major), scalars."""
    kind: str
    storage: int
    prec: int
    extents: tuple
    idx: tuple
    alpha: complex
    beta: complex

    def elems(self, k: int) -> int:
        return int(np.prod(self.extents[k], dtype=np.int64))

    def nbytes(self, k: int) -> int:
        return self.elems(k) * ELEM_BYTES[self.storage]

    def flops(self) -> float:
        """2 |D| |K| (8 |D| |K| complex): the algorithmic count of the product."""
        ext = {}
        for e_list, i_list in zip(self.extents, self.idx):
            for e, l in zip(e_list, i_list):
                ext[l] = e
        K = [l for l in set(self.idx[0]) & set(self.idx[1]) if l not in self.idx[3]]
        k = float(np.prod([ext[l] for l in K])) if K else 1.0
        f = 2.0 * self.elems(3) * k
        return 4.0 * f if self.storage in (TAPP_C32, TAPP_C64) else f


# (storage, precision) of the served mix, with its shares
SERVED_TYPES = ((0.4, TAPP_F32, TAPP_F32F32_ACCUM_F32), (0.3, TAPP_F32, TAPP_BF16BF16_ACCUM_F32),
                (0.2, TAPP_F64, TAPP_DEFAULT_PREC), (0.1, TAPP_C32, TAPP_DEFAULT_PREC))


def _tucker(rng):
    o = int(rng.integers(3, 5))
    ext = [int(x) for x in rng.integers(8, 257, o)]
    R = int(rng.integers(4, 65))
    n = int(rng.integers(0, o))
    core = list(range(o))
    d_idx = list(core)
    d_idx[n] = o
    d_ext = list(ext)
    d_ext[n] = R
    return (ext, [R, ext[n]], d_ext, d_ext), (core, [o, n], d_idx, d_idx)


def _three_way(rng, labels, nK, nH):
    """Splits labels into contracted, Hadamard and free-in-A/B classes and
    orders every tensor's labels at random."""
    labels = list(labels)
    rng.shuffle(labels)
    K, H, rest = labels[:nK], labels[nK:nK + nH], labels[nK + nH:]
    FA = [l for l in rest if rng.random() < 0.5]
    FB = [l for l in rest if l not in FA]
    A, B, D = K + H + FA, K + H + FB, H + FA + FB
    for x in (A, B, D):
        rng.shuffle(x)
    return A, B, D


def _binary(rng, hadamard: bool):
    if hadamard:
        nl = int(rng.integers(3, 7))
        nH = int(rng.integers(1, nl - 1))
        nK = int(rng.integers(1, nl - nH))
    else:
        nl = int(rng.integers(2, 7))
        nH = 0
        nK = int(rng.integers(1, nl))
    ext = {l: int(rng.integers(4, 97)) for l in range(nl)}
    A, B, D = _three_way(rng, range(nl), nK, nH)
    e = lambda idx: [ext[l] for l in idx]
    return (e(A), e(B), e(D), e(D)), (A, B, D, D)


def served_stream(rng, n: int = 20000, max_tensor_bytes: int = 64 << 30) -> list:
    """n request specifications of the served mix; shapes are redrawn until
    every tensor of the request fits max_tensor_bytes."""
    out = []
    shares = np.cumsum([t[0] for t in SERVED_TYPES])
    for _ in range(n):
        u = rng.random()
        kind = "tucker" if u < 0.5 else ("binary" if u < 0.8 else "hadamard")
        v = rng.random()
        _, storage, prec = SERVED_TYPES[int(np.searchsorted(shares, v, side="right"))]
        eb = ELEM_BYTES[storage]
        for _attempt in range(10000):
            ext, idx = _tucker(rng) if kind == "tucker" else _binary(rng, kind == "hadamard")
            if max(int(np.prod(e, dtype=np.int64)) for e in ext) * eb <= max_tensor_bytes:
                break
        if storage in (TAPP_C32, TAPP_C64):
            a = complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
            b = complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
        else:
            a, b = float(rng.uniform(-1, 1)), float(rng.uniform(-1, 1))
        out.append(RequestSpec(kind, storage, prec, tuple(list(e) for e in ext), tuple(list(i) for i in idx), a, b))
    return out


def case_from_spec(rng, spec: RequestSpec) -> Case:
    """A Case with the spec's shapes (dense column-major) and values uniform
    in [-1, 1] (real and imaginary parts for complex storage)."""
    ts = []
    for k in range(4):
        ext = list(spec.extents[k])
        T = alloc(spec.storage, ext, colmajor(ext), list(spec.idx[k]))
        n = T.buf.size
        if spec.storage in (TAPP_C32, TAPP_C64):
            T.buf[:] = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        else:
            T.buf[:] = rng.uniform(-1, 1, n)
        ts.append(T)
    return Case(*ts, scalar(spec.storage, spec.alpha), scalar(spec.storage, spec.beta), spec.prec, False,
                f"{spec.kind}")

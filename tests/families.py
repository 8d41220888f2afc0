"""Seeded generators of tensor products for the parity tests.

The families cover what the reference's randomized suites exercise
(test/test.cpp:1285-3355 and test/test.py:206-541): Hadamard products,
contractions, commuted operands, permuted D, equal extents, outer products,
full contractions, 0- and 1-mode tensors, subtensor views (same and fewer
modes), negative and mixed-sign strides, zero strides on A or B, isolated
(unary) labels, repeated (diagonal) labels, Hadamard plus free and Hadamard
plus contracted labels, every storage type and element op. The generator is
this repository's own; only the list of families follows the reference.
"""
from __future__ import annotations

import numpy as np

from tapp_b200.abi import (TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, TAPP_F16, TAPP_BF16)
from tapp_b200.case import Case, Tensor, alloc, fill_uniform, scalar, is_complex

ALL_TYPES = (TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64)


def _labels(rng, n):
    # labels are arbitrary int64 values in the ABI; mix letters and large values
    if rng.random() < 0.5:
        pool = list(range(ord("a"), ord("a") + 26)) + list(range(ord("A"), ord("A") + 26))
        return [int(x) for x in rng.choice(pool, size=n, replace=False)]
    out = set()
    while len(out) < n:
        out.add(int(rng.integers(-10**12, 10**12)))
    return list(out)


def _layout(rng, extents, *, subtensor=False, neg=False, mixed=False, extra_modes=False):
    """Strides (elements) of a column-major layout over a random mode order,
    optionally embedded in a larger tensor, with sign flips. Returns
    (strides, pad_lo, pad_hi)."""
    n = len(extents)
    order = rng.permutation(n) if n else []
    strides = [0] * n
    acc = 1
    if extra_modes and n:
        acc *= int(rng.integers(1, 3))
    for k in order:
        strides[k] = acc
        outer = extents[k] + (int(rng.integers(0, 3)) if subtensor else 0)
        acc *= max(outer, 1)
    if neg or mixed:
        for k in range(n):
            if neg and not mixed:
                strides[k] = -strides[k]
            elif rng.random() < 0.5:
                strides[k] = -strides[k]
    pad_lo = int(rng.integers(0, 4)) if subtensor else 0
    pad_hi = int(rng.integers(0, 4)) if subtensor else 0
    return strides, pad_lo, pad_hi


def random_case(rng: np.random.Generator, *, dtype=None, types=None, prec=-1,
                n_contracted=None, n_hadamard=None, n_freeA=None, n_freeB=None,
                n_isoA=0, n_isoB=0, n_repA=0, n_repB=0, n_repD=0,
                min_ext=1, max_ext=4, ext_choices=None,
                subtensor=False, neg=False, mixed=False, zero_stride=None,
                ops=None, C_null=False, beta_zero=False, name="", max_work=None) -> Case:
    if types is None:
        if dtype is None:
            dtype = int(rng.choice(ALL_TYPES))
        types = (dtype,) * 4
    tA, tB, tC, tD = types
    r = lambda lo, hi: int(rng.integers(lo, hi + 1))
    nK = r(0, 2) if n_contracted is None else n_contracted
    nH = r(0, 1) if n_hadamard is None else n_hadamard
    nFA = r(0, 2) if n_freeA is None else n_freeA
    nFB = r(0, 2) if n_freeB is None else n_freeB
    total = nK + nH + nFA + nFB + n_isoA + n_isoB
    labs = _labels(rng, total)
    it = iter(labs)
    K = [next(it) for _ in range(nK)]
    H = [next(it) for _ in range(nH)]
    FA = [next(it) for _ in range(nFA)]
    FB = [next(it) for _ in range(nFB)]
    UA = [next(it) for _ in range(n_isoA)]
    UB = [next(it) for _ in range(n_isoB)]
    ext = {}
    for attempt in range(1000):
        for l in labs:
            ext[l] = int(rng.choice(ext_choices)) if ext_choices is not None else r(min_ext, max_ext)
        work = float(np.prod([ext[l] for l in labs], dtype=np.float64))
        if max_work is None or work <= max_work:
            break
    else:
        raise RuntimeError("no extents under the work bound")

    def shuffled(x):
        x = list(x)
        rng.shuffle(x)
        return x

    idx_A = shuffled(K + H + FA + UA)
    idx_B = shuffled(K + H + FB + UB)
    idx_D = shuffled(H + FA + FB)
    for _ in range(n_repA):
        if idx_A:
            idx_A.insert(r(0, len(idx_A)), idx_A[r(0, len(idx_A) - 1)])
    for _ in range(n_repB):
        if idx_B:
            idx_B.insert(r(0, len(idx_B)), idx_B[r(0, len(idx_B) - 1)])
    for _ in range(n_repD):
        if idx_D:
            idx_D.insert(r(0, len(idx_D)), idx_D[r(0, len(idx_D) - 1)])
    idx_C = list(idx_D)

    if ops is None:
        ops = [int(rng.integers(0, 2)) for _ in range(4)]
    tensors = []
    for t, idx, op, which in ((tA, idx_A, ops[0], "A"), (tB, idx_B, ops[1], "B"),
                              (tC, idx_C, ops[2], "C"), (tD, idx_D, ops[3], "D")):
        e = [ext[l] for l in idx]
        if which == "C" and tensors:
            # C is laid out independently of D (a permutation of its storage)
            pass
        s, plo, phi = _layout(rng, e, subtensor=subtensor, neg=neg, mixed=mixed)
        if zero_stride is not None and which in zero_stride and len(e) > 0:
            s[r(0, len(e) - 1)] = 0
        T = alloc(t, e, s, idx, op, plo, phi)
        fill_uniform(T, rng)
        tensors.append(T)
    A, B, Cc, D = tensors
    if is_complex(tD):
        a = complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
        b = 0.0 if beta_zero else complex(rng.uniform(-1, 1), rng.uniform(-1, 1))
    else:
        a = float(rng.uniform(-1, 1))
        b = 0.0 if beta_zero else float(rng.uniform(-1, 1))
    return Case(A, B, Cc, D, scalar(tD, a), scalar(tD, b), prec, C_null, name)


def family_cases(seed: int, count_per_family: int = 4, dtypes=ALL_TYPES, max_ext=4):
    """Yields (family_name, case) for every family."""
    rng = np.random.default_rng(seed)
    fams = {
        "hadamard": dict(n_contracted=0, n_hadamard=2, n_freeA=0, n_freeB=0),
        "contraction": dict(n_contracted=2, n_hadamard=0, n_freeA=2, n_freeB=1),
        "outer": dict(n_contracted=0, n_hadamard=0, n_freeA=2, n_freeB=2),
        "full_contraction": dict(n_contracted=3, n_hadamard=0, n_freeA=0, n_freeB=0),
        "zero_dim": dict(n_contracted=0, n_hadamard=0, n_freeA=0, n_freeB=0),
        "one_dim": dict(n_contracted=1, n_hadamard=0, n_freeA=1, n_freeB=0),
        "equal_extents": dict(ext_choices=[3]),
        "subtensor": dict(subtensor=True),
        "negative_strides": dict(neg=True),
        "mixed_strides": dict(mixed=True, subtensor=True),
        "zero_stride_A": dict(zero_stride="A"),
        "zero_stride_B": dict(zero_stride="B"),
        "isolated": dict(n_isoA=1, n_isoB=1),
        "repeated": dict(n_repA=1, n_repB=1),
        "repeated_D": dict(n_repD=1),
        "hadamard_free": dict(n_contracted=0, n_hadamard=1, n_freeA=1, n_freeB=1),
        "hadamard_contraction": dict(n_contracted=1, n_hadamard=1, n_freeA=1, n_freeB=1),
        "beta_zero_C_null": dict(beta_zero=True, C_null=True),
        "everything": dict(n_contracted=2, n_hadamard=1, n_freeA=1, n_freeB=1, n_isoA=1, n_isoB=1,
                           n_repA=1, subtensor=True, mixed=True),
    }
    for name, kw in fams.items():
        for i in range(count_per_family):
            dt = int(dtypes[(i + len(name)) % len(dtypes)])
            kw2 = dict(kw)
            kw2.setdefault("max_ext", max_ext)
            yield name, random_case(rng, dtype=dt, name=f"{name}-{i}", **kw2)


def bounded_case(rng, max_work=3e6, **kw):
    """random_case with extents redrawn until the product of all label
    extents (|D| * |K| * |UA| * |UB|, the oracle's work) stays below
    max_work, so that the binary64 oracle finishes in well under a second."""
    return random_case(rng, max_work=max_work, **kw)

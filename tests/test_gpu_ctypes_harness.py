"""The reference's Python callers, unchanged but for the library path.

The reference's Python test harness (test/test.py) binds the library with
ctypes: `CDLL(path)` and the argument types of test/test.py:16-120 (handles
as 64-bit integers, label and extent arrays as int64 pointers, data as void
pointers), builds every product from numpy arrays (extents and element
strides from the array, type TAPP_F64 or TAPP_C64, DEFAULT precision, host
pointers: :122-185) and checks D against numpy.einsum with np.allclose
(:187-204). This file declares the same binding against
lib/libtapp-b200.so and runs the harness's thirteen kinds of products
(:206-541: Hadamard, contraction, commutativity, permutations, equal
extents, outer product, full contraction, zero- and one-mode operands,
subtensors with the same and with fewer modes, unique and repeated labels)
from seeded generators of its own, host numpy arrays in and out.

One deliberate difference: the harness passes alpha and beta as a c_double
for complex products too, so the library reads the imaginary part from
whatever follows it in memory; here complex scalars are two doubles.
"""
import ctypes as C
import itertools
import os

import numpy as np
import pytest

import tapp_b200

pytestmark = pytest.mark.gpu

H = C.c_int64          # handle type of a 64-bit build, as the harness picks it


def bind(path):
    """CDLL with the argument types of the reference harness."""
    L = C.CDLL(path)
    sig = {
        "TAPP_create_tensor_product": [C.POINTER(H), H, C.c_int, H, C.POINTER(C.c_int64), C.c_int, H,
                                       C.POINTER(C.c_int64), C.c_int, H, C.POINTER(C.c_int64), C.c_int, H,
                                       C.POINTER(C.c_int64), C.c_int],
        "TAPP_destroy_tensor_product": [H],
        "TAPP_execute_product": [H, H, C.POINTER(H), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p],
        "TAPP_create_tensor_info": [C.POINTER(H), C.c_int, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
        "TAPP_destroy_tensor_info": [H],
        "TAPP_create_executor": [C.POINTER(H)],
        "TAPP_destroy_executor": [H],
        "TAPP_create_handle": [C.POINTER(H)],
        "TAPP_destroy_handle": [H],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.restype = C.c_int
        f.argtypes = args
    return L


@pytest.fixture(scope="module")
def L():
    tapp_b200.load()                     # builds nothing; fails loudly if the library is missing
    return bind(os.path.join(os.path.dirname(tapp_b200.__file__), "..", "lib", "libtapp-b200.so"))


def product(L, alpha, A, B, beta, C_, D, idx_A, idx_B, idx_C, idx_D, ops):
    """One TAPP_execute_product on numpy arrays, the way the harness builds it."""
    ty = 1 if A.dtype == np.float64 else 3
    infos = []
    for T in (A, B, C_, D):
        ext = (C.c_int64 * T.ndim)(*T.shape)
        st = (C.c_int64 * T.ndim)(*[s // T.itemsize for s in T.strides])
        h = H(0)
        assert L.TAPP_create_tensor_info(C.byref(h), ty, T.ndim, ext, st) == 0
        infos.append(h)
    idx = [(C.c_int64 * max(len(i), 1))(*i) for i in (idx_A, idx_B, idx_C, idx_D)]
    handle, plan, ex, status = H(0), H(0), H(0), H(0)
    assert L.TAPP_create_handle(C.byref(handle)) == 0
    assert L.TAPP_create_tensor_product(C.byref(plan), handle, ops[0], infos[0], idx[0], ops[1], infos[1], idx[1],
                                        ops[2], infos[2], idx[2], ops[3], infos[3], idx[3], -1) == 0
    assert L.TAPP_create_executor(C.byref(ex)) == 0
    scal = (lambda v: C.byref((C.c_double * 2)(v.real, v.imag))) if ty == 3 else (lambda v: C.byref(C.c_double(v)))
    err = L.TAPP_execute_product(plan, ex, C.byref(status), scal(alpha), A.ctypes.data, B.ctypes.data, scal(beta),
                                 C_.ctypes.data, D.ctypes.data)
    L.TAPP_destroy_handle(handle)
    L.TAPP_destroy_executor(ex)
    L.TAPP_destroy_tensor_product(plan)
    for h in infos:
        L.TAPP_destroy_tensor_info(h)
    assert err == 0, err
    return D


def einsum(alpha, A, B, beta, C_, D, idx_A, idx_B, idx_D, ops):
    """D <- op_D(alpha * einsum(op_A(A), op_B(B)) + beta * op_C(C)), numpy."""
    A = np.conjugate(A) if ops[0] else A
    B = np.conjugate(B) if ops[1] else B
    C_ = np.conjugate(C_) if ops[2] else C_
    spec = "".join(map(chr, idx_A)) + "," + "".join(map(chr, idx_B)) + "->" + "".join(map(chr, idx_D))
    out = alpha * np.einsum(spec, A, B) + beta * C_
    D[...] = np.conjugate(out) if ops[3] else out
    return D


def rand_array(rng, shape, cplx):
    a = np.array(rng.random(shape))
    return np.array(a + 1j * rng.random(shape)) if cplx else a


def view(rng, base_shape, cplx, drop=()):
    """A strided subtensor of a larger array: every mode sliced with an
    offset and a step; modes in `drop` indexed away (fewer modes)."""
    big = rand_array(rng, [2 * e + 2 for e in base_shape], cplx)
    sl = []
    for m, e in enumerate(base_shape):
        off = int(rng.integers(0, 2))
        sl.append(off if m in drop else slice(off, off + 2 * e, 2))
    return big[tuple(sl)]


class Gen:
    """Labels and extents of one product: contracted labels (in A and B),
    free labels of A and of B (in D), Hadamard labels (in A, B and D),
    unique labels (only in A or only in B), one repeated label per operand."""

    def __init__(self, rng, *, n_con=None, n_fa=None, n_fb=None, n_had=0, n_ua=0, n_ub=0, rep=False,
                 ext=None, cplx=None):
        r = lambda lo, hi: int(rng.integers(lo, hi + 1))
        self.rng = rng
        self.cplx = bool(rng.integers(0, 2)) if cplx is None else cplx
        counts = [r(0, 3) if n_con is None else n_con, r(0, 2) if n_fa is None else n_fa,
                  r(0, 2) if n_fb is None else n_fb, n_had, n_ua, n_ub]
        labels = iter(range(97, 97 + 26))
        con, fa, fb, had, ua, ub = ([next(labels) for _ in range(c)] for c in counts)
        self.ext = {l: (ext if ext is not None else r(1, 4)) for l in con + fa + fb + had + ua + ub}
        self.idx_A = list(rng.permutation(con + fa + had + ua))
        self.idx_B = list(rng.permutation(con + fb + had + ub))
        self.idx_D = list(rng.permutation(fa + fb + had))
        if rep:
            for lst in (self.idx_A, self.idx_B):
                if lst:
                    lst.insert(r(0, len(lst)), lst[r(0, len(lst) - 1)])
        self.idx_A = [int(x) for x in self.idx_A]
        self.idx_B = [int(x) for x in self.idx_B]
        self.idx_D = [int(x) for x in self.idx_D]

    def shape(self, idx):
        return [self.ext[l] for l in idx]

    def run(self, L, A=None, B=None, C_=None, D=None, idx_D=None, swap=False):
        rng = self.rng
        idx_D = self.idx_D if idx_D is None else idx_D
        A = rand_array(rng, self.shape(self.idx_A), self.cplx) if A is None else A
        B = rand_array(rng, self.shape(self.idx_B), self.cplx) if B is None else B
        C_ = rand_array(rng, self.shape(idx_D), self.cplx) if C_ is None else C_
        D = rand_array(rng, self.shape(idx_D), self.cplx) if D is None else D
        alpha = complex(rng.random(), rng.random()) if self.cplx else float(rng.random())
        beta = complex(rng.random(), rng.random()) if self.cplx else float(rng.random())
        ops = [int(x) for x in rng.integers(0, 2, 4)]
        E = np.array(D)
        ia, ib = (self.idx_B, self.idx_A) if swap else (self.idx_A, self.idx_B)
        a, b = (B, A) if swap else (A, B)
        oa = [ops[1], ops[0], ops[2], ops[3]] if swap else ops
        product(L, alpha, a, b, beta, C_, D, ia, ib, idx_D, idx_D, oa)
        einsum(alpha, a, b, beta, C_, E, ia, ib, idx_D, oa)
        assert np.allclose(D, E), (ia, ib, idx_D, float(np.abs(D - E).max()))
        return D


N = 12      # products per kind


def test_hadamard_product(L):
    rng = np.random.default_rng(1)
    for _ in range(N):
        Gen(rng, n_con=0, n_fa=0, n_fb=0, n_had=int(rng.integers(1, 5))).run(L)


def test_contraction(L):
    rng = np.random.default_rng(2)
    for _ in range(N):
        Gen(rng).run(L)


def test_commutativity(L):
    """A B and B A (labels and ops swapped with them) give the same D."""
    rng = np.random.default_rng(3)
    for _ in range(N):
        g = Gen(rng, n_con=int(rng.integers(1, 3)), n_fa=1, n_fb=1)
        A = rand_array(rng, g.shape(g.idx_A), g.cplx)
        B = rand_array(rng, g.shape(g.idx_B), g.cplx)
        C_ = rand_array(rng, g.shape(g.idx_D), g.cplx)
        state = rng.bit_generator.state
        d1 = g.run(L, A, B, C_, np.zeros_like(C_))
        rng.bit_generator.state = state
        d2 = g.run(L, A, B, C_, np.zeros_like(C_), swap=True)
        assert np.allclose(d1, d2)


def test_permutations(L):
    """Every order of D's labels (C laid out in the same order)."""
    rng = np.random.default_rng(4)
    g = Gen(rng, n_con=1, n_fa=2, n_fb=1)
    for perm in itertools.permutations(g.idx_D):
        g.run(L, idx_D=list(perm))


def test_equal_extents(L):
    rng = np.random.default_rng(5)
    for _ in range(N):
        Gen(rng, ext=int(rng.integers(1, 5))).run(L)


def test_outer_product(L):
    rng = np.random.default_rng(6)
    for _ in range(N):
        Gen(rng, n_con=0, n_fa=int(rng.integers(1, 3)), n_fb=int(rng.integers(1, 3))).run(L)


def test_full_contraction(L):
    rng = np.random.default_rng(7)
    for _ in range(N):
        Gen(rng, n_con=int(rng.integers(1, 4)), n_fa=0, n_fb=0).run(L)


def test_zero_mode_operand(L):
    """A is a scalar (0 modes): D = alpha a B + beta C."""
    rng = np.random.default_rng(8)
    for _ in range(N):
        Gen(rng, n_con=0, n_fa=0, n_fb=int(rng.integers(0, 4))).run(L)


def test_one_mode_operand(L):
    rng = np.random.default_rng(9)
    for _ in range(N):
        con = int(rng.integers(0, 2))
        Gen(rng, n_con=con, n_fa=1 - con, n_fb=int(rng.integers(0, 3))).run(L)


def test_subtensor_same_modes(L):
    """Every operand a strided view (offset and step 2 on each mode) of a
    larger array, with as many modes as the array."""
    rng = np.random.default_rng(10)
    for _ in range(N):
        g = Gen(rng, n_con=int(rng.integers(1, 3)), n_fa=1, n_fb=1)
        A = view(rng, g.shape(g.idx_A), g.cplx)
        B = view(rng, g.shape(g.idx_B), g.cplx)
        C_ = view(rng, g.shape(g.idx_D), g.cplx)
        D = view(rng, g.shape(g.idx_D), g.cplx)
        g.run(L, A, B, C_, D)


def test_subtensor_fewer_modes(L):
    """Operands that are views with one mode of a larger array indexed away."""
    rng = np.random.default_rng(11)
    for _ in range(N):
        g = Gen(rng, n_con=int(rng.integers(1, 3)), n_fa=1, n_fb=1)
        sA = g.shape(g.idx_A)
        A = view(rng, sA[:1] + [3] + sA[1:], g.cplx, drop=(1,))
        sD = g.shape(g.idx_D)
        D = view(rng, [3] + sD, g.cplx, drop=(0,))
        g.run(L, A, None, None, D)


def test_unique_labels(L):
    """Labels only in A or only in B are summed over before the product."""
    rng = np.random.default_rng(12)
    for _ in range(N):
        Gen(rng, n_ua=int(rng.integers(1, 3)), n_ub=int(rng.integers(1, 3))).run(L)


def test_repeated_labels(L):
    """A label repeated in an operand takes its diagonal."""
    rng = np.random.default_rng(13)
    for _ in range(N):
        Gen(rng, n_con=int(rng.integers(1, 3)), n_fa=1, n_fb=1, rep=True).run(L)

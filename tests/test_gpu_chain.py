"""tapp_b200_execute_chain: the mode-n products that rebuild a tensor from
its Tucker core and factor matrices (X = G x1 U1 x2 U2 x3 U3, as the
reference's Tucker exercise computes it one product at a time), run as one
chain with the intermediates kept in device memory. Each chain result equals
the same products run one by one with TAPP_execute_product (same kernels,
same arguments: bit for bit), with host or device operands, and matches a
binary64 evaluation within the binary32 bound."""
import ctypes as C

import numpy as np
import pytest

import tapp_b200
from tapp_b200.case import alloc, scalar
from tapp_b200.workloads import colmajor

pytestmark = pytest.mark.gpu


def _chain_fn(tapp):
    f = tapp.lib.tapp_b200_execute_chain
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.POINTER(tapp_b200.intptr), tapp_b200.intptr] + [C.POINTER(C.c_void_p)] * 6
    return f


class Tucker:
    """Core G[i,j,k], factors U1[a,i], U2[b,j], U3[c,k] and the three steps
    T1[a,j,k] = sum_i G U1, T2[a,b,k] = sum_j T1 U2, X[a,b,c] = sum_k T2 U3."""

    def __init__(self, tapp, rng, dtype=0, prec=0, r=(24, 20, 16), n=(64, 48, 40)):
        self.tapp = tapp
        self.dtype, self.prec = dtype, prec
        i, j, k = ord("i"), ord("j"), ord("k")
        a, b, c = ord("a"), ord("b"), ord("c")
        self.shapes = [
            # (A extents, A idx, B extents, B idx, D extents, D idx)
            ([r[0], r[1], r[2]], [i, j, k], [n[0], r[0]], [a, i], [n[0], r[1], r[2]], [a, j, k]),
            ([n[0], r[1], r[2]], [a, j, k], [n[1], r[1]], [b, j], [n[0], n[1], r[2]], [a, b, k]),
            ([n[0], n[1], r[2]], [a, b, k], [n[2], r[2]], [c, k], [n[0], n[1], n[2]], [a, b, c]),
        ]
        def t(ext, idx):
            T = alloc(dtype, ext, colmajor(ext), idx)
            T.buf[:] = rng.uniform(-1, 1, T.buf.size)
            return T
        self.G = t(self.shapes[0][0], self.shapes[0][1])
        self.U = [t(s[2], s[3]) for s in self.shapes]
        self.alpha = scalar(dtype, 1.0)
        self.beta = scalar(dtype, 0.0)
        self.plans, self.infos = [], []
        for ae, ai, be, bi, de, di in self.shapes:
            inf = [tapp.tensor_info(dtype, e, colmajor(e))[1] for e in (ae, be, de, de)]
            _, plan = tapp.create_product(0, [0, 0, 0, 0], inf, [ai, bi, di, di], prec)
            self.plans.append(plan)
            self.infos += inf

    def outputs(self):
        return [alloc(self.dtype, s[4], colmajor(s[4]), s[5]) for s in self.shapes]

    def release(self):
        for p in self.plans:
            self.tapp.lib.TAPP_destroy_tensor_product(p)
        for h in self.infos:
            self.tapp.lib.TAPP_destroy_tensor_info(h)


def _arr(vals):
    return (C.c_void_p * len(vals))(*vals)


def run_chain(tapp, tk, ex, G, U, X):
    n = 3
    plans = (tapp_b200.intptr * n)(*tk.plans)
    al = _arr([tk.alpha.ctypes.data] * n)
    be = _arr([tk.beta.ctypes.data] * n)
    return _chain_fn(tapp)(n, plans, ex, al, be, _arr([G, None, None]), _arr(U), None, _arr([None, None, X]))


def sequential(tapp, tk, ex):
    """The three products one by one on the host buffers."""
    outs = tk.outputs()
    A = tk.G
    for s, (plan, U, D) in enumerate(zip(tk.plans, tk.U, outs)):
        st = tapp_b200.intptr(0)
        err = tapp.lib.TAPP_execute_product(plan, ex, C.byref(st), tk.alpha.ctypes.data, A.ptr(), U.ptr(),
                                            tk.beta.ctypes.data, None, D.ptr())
        assert err == 0
        A = D
    return outs[-1]


@pytest.mark.parametrize("dtype,prec", [(0, 0), (0, 6), (1, 1)])
@pytest.mark.parametrize("where", ["host", "device"])
def test_tucker_chain_matches_steps(tapp, gpu, dtype, prec, where):
    import torch
    rng = np.random.default_rng(400 + dtype + prec)
    tk = Tucker(tapp, rng, dtype, prec)
    ex = tapp.create_executor()
    want = sequential(tapp, tk, ex)
    X = tk.outputs()[-1]
    if where == "host":
        err = run_chain(tapp, tk, ex, tk.G.ptr(), [U.ptr() for U in tk.U], X.ptr())
        got = X.buf
    else:
        dev = [torch.from_numpy(t.buf.copy()).cuda() for t in [tk.G] + tk.U + [X]]
        err = run_chain(tapp, tk, ex, dev[0].data_ptr(), [d.data_ptr() for d in dev[1:4]], dev[4].data_ptr())
        torch.cuda.synchronize()
        got = dev[4].cpu().numpy()
    assert err == 0, tapp.explain(err)
    assert np.array_equal(got.view(np.uint8), want.buf.view(np.uint8))
    # against binary64 (einsum of the 16-bit-rounded operands for prec 6 is
    # not what the steps compute, so only the plain precisions are compared)
    if prec in (0, 1):
        r = tk.shapes
        Gm = tk.G.buf.reshape(r[0][0], order="F").astype(np.float64)
        U1, U2, U3 = [u.buf.reshape(s[2], order="F").astype(np.float64) for u, s in zip(tk.U, r)]
        ref = np.einsum("ijk,ai,bj,ck->abc", Gm, U1, U2, U3).reshape(-1, order="F")
        tol = 1e-4 if dtype == 0 else 1e-12
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    tapp.lib.TAPP_destroy_executor(ex)
    tk.release()


def test_chain_argument_and_validation_codes(tapp, gpu):
    rng = np.random.default_rng(410)
    tk = Tucker(tapp, rng)
    ex = tapp.create_executor()
    X = tk.outputs()[-1]
    f = _chain_fn(tapp)
    plans = (tapp_b200.intptr * 3)(*tk.plans)
    al = _arr([tk.alpha.ctypes.data] * 3)
    be = _arr([tk.beta.ctypes.data] * 3)
    U = _arr([u.ptr() for u in tk.U])
    # step 0 has nothing to read from; the last D must be given
    assert f(3, plans, ex, al, be, _arr([None, None, None]), U, None, _arr([None, None, X.ptr()])) == tapp_b200.ERR_INVALID
    assert f(3, plans, ex, al, be, _arr([tk.G.ptr(), None, None]), U, None, _arr([None, None, None])) == tapp_b200.ERR_INVALID
    # NULL executor: the reference's code 33
    assert f(3, plans, 0, al, be, _arr([tk.G.ptr(), None, None]), U, None, _arr([None, None, X.ptr()])) == 33
    # a step whose D layout disagrees with its labels returns that step's validation code
    bad = tapp.tensor_info(0, [5, 5], [1, 5])[1]
    _, pbad = tapp.create_product(0, [0, 0, 0, 0], [tk.infos[3], tk.infos[4], bad, bad],
                                  [tk.shapes[1][1], tk.shapes[1][3], tk.shapes[1][5], tk.shapes[1][5]], 0)
    want = tapp.lib.TAPP_execute_product(pbad, ex, None, tk.alpha.ctypes.data, tk.G.ptr(), tk.U[1].ptr(),
                                         tk.beta.ctypes.data, None, X.ptr())
    assert want != 0
    plans2 = (tapp_b200.intptr * 3)(tk.plans[0], pbad, tk.plans[2])
    assert f(3, plans2, ex, al, be, _arr([tk.G.ptr(), None, None]), U, None, _arr([None, None, X.ptr()])) == want
    tapp.lib.TAPP_destroy_tensor_product(pbad)
    tapp.lib.TAPP_destroy_tensor_info(bad)
    tapp.lib.TAPP_destroy_executor(ex)
    tk.release()

"""Tile-shape tuner for grouped tensor-core products.

A grouped launch (tapp_b200_execute_group, the server's grouped units) runs
its tiles either as 256 x 256 tiles on SM pairs or as 128 x 128 tiles on
single SMs. For every shape class (operand mode, floor(log2 M),
floor(log2 N), floor(log2 K)) the tuner builds a group of synthetic products
of that size, times one grouped launch with each shape on the GPU (CUDA
events, median of several runs), and writes the faster shape per class to a
text table ("mode m n k tile" per line) that the library loads with
tapp_b200_load_tile_table or from TAPP_B200_TILE_TABLE.

    python -m tapp_b200.tuner --out tiles.txt              # the served mix's classes
    python -m tapp_b200.tuner --out t.txt --class 6,512,128,256

The candidate classes are chosen on the CPU (the classes a workload has);
only their timing runs on the GPU.
"""
from __future__ import annotations

import argparse
import math
import os
import statistics

import numpy as np

from .abi import TAPP_F32, TAPP_BF16BF16_ACCUM_F32, TAPP_F16F16_ACCUM_F32, TAPP_F32F32_ACCUM_F32

ATTR_ASYNC, ATTR_F32_MODE, ATTR_PATH, ATTR_TILE = 0x1001, 0x1002, 0x1004, 0x1008
PATH_TC = 4
MODE_OF_PREC = {TAPP_BF16BF16_ACCUM_F32: 0, TAPP_F16F16_ACCUM_F32: 1, TAPP_F32F32_ACCUM_F32: 2}


def class_key(prec: int, m: int, n: int, k: int) -> tuple:
    """(mode, floor(log2 M), floor(log2 N), floor(log2 K)) as the library keys its table."""
    lg = lambda x: int(math.floor(math.log2(max(int(x), 1))))
    return MODE_OF_PREC[prec], lg(m), lg(n), lg(k)


def _products(tapp, torch, prec, m, n, k, count, seed):
    """count products D[m,n] = sum_k A[m,k] B[k,n] + 0.5 C, binary32 on the
    GPU, A contiguous along m and B along k."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    out = []
    for _ in range(count):
        A = torch.rand(m * k, device="cuda", generator=g) * 2 - 1
        B = torch.rand(k * n, device="cuda", generator=g) * 2 - 1
        Cc = torch.rand(m * n, device="cuda", generator=g) * 2 - 1
        D = torch.zeros(m * n, device="cuda")
        infos = [tapp.tensor_info(TAPP_F32, e, [1, e[0]])[1] for e in ([m, k], [k, n], [m, n], [m, n])]
        err, plan = tapp.create_product(0, [0, 0, 0, 0], infos, [[109, 107], [107, 110], [109, 110], [109, 110]], prec)
        assert err == 0
        out.append((plan, infos, (A, B, Cc, D)))
    return out


def _time_group(tapp, torch, prods, alpha, beta, tile, f32_mode, reps):
    ex = tapp.create_executor()
    tapp.set_int(ex, ATTR_PATH, PATH_TC)
    tapp.set_int(ex, ATTR_F32_MODE, f32_mode)
    tapp.set_int(ex, ATTR_TILE, tile)
    stream = torch.cuda.current_stream()
    tapp.set_stream(ex, stream.cuda_stream)
    tapp.set_int(ex, ATTR_ASYNC, 1)
    n = len(prods)
    args = ([p[0] for p in prods], ex, [alpha.ctypes.data] * n, [beta.ctypes.data] * n,
            [p[2][0].data_ptr() for p in prods], [p[2][1].data_ptr() for p in prods],
            [p[2][2].data_ptr() for p in prods], [p[2][3].data_ptr() for p in prods])
    assert tapp.execute_group(*args) == 0   # warm-up (first launch, pool growth)
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert tapp.execute_group(*args) == 0
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e3)
    tapp.lib.TAPP_destroy_executor(ex)
    return statistics.median(times)


def tune(tapp, classes, path, products_per_class=16, reps=5, seed=0):
    """Times both tile shapes for each class (precision, M, N, K) and writes
    the table to `path`. Returns one dict per class: its key, both times in
    microseconds (tile 1, tile 2) and the chosen tile."""
    import torch
    rows = []
    alpha = np.array([1.0], dtype=np.float32)
    beta = np.array([0.5], dtype=np.float32)
    for i, (prec, m, n, k) in enumerate(classes):
        prods = _products(tapp, torch, prec, m, n, k, products_per_class, seed + i)
        f32_mode = 1 if prec == TAPP_F32F32_ACCUM_F32 else 0
        t1 = _time_group(tapp, torch, prods, alpha, beta, 1, f32_mode, reps)
        t2 = _time_group(tapp, torch, prods, alpha, beta, 2, f32_mode, reps)
        rows.append({"class": (prec, m, n, k), "key": class_key(prec, m, n, k), "us": (t1, t2),
                     "tile": 1 if t1 <= t2 else 2})
        for plan, infos, _ in prods:
            tapp.lib.TAPP_destroy_tensor_product(plan)
            for h in infos:
                tapp.lib.TAPP_destroy_tensor_info(h)
        del prods
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    seen = set()
    with open(path, "w") as f:
        f.write("# tapp_b200 tile table: mode log2(M) log2(N) log2(K) tile (1: 256x256 pairs, 2: 128x128)\n")
        for r in rows:
            if r["key"] in seen:
                continue
            seen.add(r["key"])
            f.write("%d %d %d %d %d\n" % (*r["key"], r["tile"]))
            f.write("# %s: %.1f us with 256x256, %.1f us with 128x128\n" % (r["class"], *r["us"]))
    return rows


def served_classes(seed=5, n=2000, max_per_class_bytes=2 << 30):
    """Shape classes of the served mix's tensor-core products (binary32
    storage, bfloat16 precision), one representative size per class, chosen
    on the CPU from the stream's specs and plan descriptions."""
    from .workloads import served_stream
    import tapp_b200
    lib = tapp_b200.load()
    reps = {}
    for s in served_stream(np.random.default_rng(seed), n, max_tensor_bytes=1 << 30):
        if s.prec != TAPP_BF16BF16_ACCUM_F32 or s.storage != TAPP_F32:
            continue
        infos = [lib.tensor_info(s.storage, s.extents[j], _colmajor(s.extents[j]))[1] for j in range(4)]
        _, plan = lib.create_product(0, [0, 0, 0, 0], infos, list(s.idx), s.prec)
        d = lib.describe(plan)
        lib.lib.TAPP_destroy_tensor_product(plan)
        for h in infos:
            lib.lib.TAPP_destroy_tensor_info(h)
        if "path=tc" not in d:
            continue
        m, n_, k = _mode_size(d, "M"), _mode_size(d, "N"), _mode_size(d, "K")
        if 4 * (m * k + k * n_ + 2 * m * n_) > max_per_class_bytes:
            continue
        reps.setdefault(class_key(s.prec, m, n_, k), (s.prec, m, n_, k))
    return list(reps.values())


def _colmajor(ext):
    st, acc = [], 1
    for e in ext:
        st.append(acc)
        acc *= e
    return st


def _mode_size(desc: str, name: str) -> int:
    """Product of the extents of mode list `name` in a plan description."""
    i = desc.index(" " + name + "=[") + len(name) + 3
    j = desc.index("]", i)
    size = 1
    for part in desc[i:j].split("),("):
        part = part.strip("()")
        if part:
            size *= int(part.split(":")[0])
    return size


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", required=True)
    ap.add_argument("--class", dest="classes", action="append", default=[],
                    help="prec,M,N,K (repeatable); default: the served mix's classes")
    ap.add_argument("--products", type=int, default=8)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    import tapp_b200
    lib = tapp_b200.load()
    classes = [tuple(int(x) for x in c.split(",")) for c in a.classes] or served_classes()
    for r in tune(lib, classes, a.out, a.products, a.reps):
        print(r)


if __name__ == "__main__":
    main()

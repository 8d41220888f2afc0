"""Runs a stream of served products (workloads.served_stream) on one GPU, in
two ways, on the same device-resident operands:

  plain   one synchronous TAPP_execute_product per request, in arrival order
          (one launch sequence per contraction, nothing overlapped)
  served  the requests submitted to a server (tapp_b200_server_*) as they
          arrive, either at Poisson arrival times or all at once

Operands live in HBM for the whole run: A, B and C of every request point
into one random pool per storage type (uniform in [-1, 1]); D points into
an output arena, either one region per request (distinct_outputs, for
checking results) or a ring that requests share (for timing only).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from .abi import TAPP_F32, TAPP_F64, TAPP_C32, TAPP_C64, ELEM_BYTES, intptr
from .server import Server

ALIGN = 256


def _scalar_buf(storage, v):
    dt = {TAPP_F32: np.float32, TAPP_F64: np.float64, TAPP_C32: np.complex64, TAPP_C64: np.complex128}[storage]
    a = np.zeros(1, dtype=dt)
    a[0] = v if storage in (TAPP_C32, TAPP_C64) else np.real(v)
    return a


def _colmajor(ext):
    s, acc = [], 1
    for e in ext:
        s.append(acc)
        acc *= e
    return s


class StreamRunner:
    def __init__(self, tapp, specs, torch, seed=0, distinct_outputs=False, ring_bytes=4 << 30):
        self.tapp = tapp
        self.specs = specs
        self.torch = torch
        rng = np.random.default_rng(seed)
        L = tapp.lib
        # input pools, one per real base type, large enough for the largest operand
        need = {TAPP_F32: 0, TAPP_F64: 0}
        base = {TAPP_F32: TAPP_F32, TAPP_C32: TAPP_F32, TAPP_F64: TAPP_F64, TAPP_C64: TAPP_F64}
        for s in specs:
            for k in range(3):
                need[base[s.storage]] = max(need[base[s.storage]], s.nbytes(k))
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        self.pool = {}
        for t, nbytes in need.items():
            if nbytes == 0:
                continue
            dt = torch.float32 if t == TAPP_F32 else torch.float64
            n = (nbytes + ALIGN) // ELEM_BYTES[t] + 1
            self.pool[t] = torch.rand(n, dtype=dt, device="cuda", generator=g) * 2 - 1
        out_bytes = [(s.nbytes(3) + ALIGN - 1) // ALIGN * ALIGN for s in specs]
        total_out = sum(out_bytes) if distinct_outputs else max(ring_bytes, max(out_bytes))
        self.arena = torch.zeros(total_out // 4 + 1, dtype=torch.float32, device="cuda")
        self.infos, self.plans, self.ptrs, self.scalars, self.d_off = [], [], [], [], []
        ring = 0
        for s, ob in zip(specs, out_bytes):
            infos = []
            for k in range(4):
                err, h = tapp.tensor_info(s.storage, s.extents[k], _colmajor(s.extents[k]))
                assert err == 0
                infos.append(h)
            err, plan = tapp.create_product(0, [0, 0, 0, 0], infos, list(s.idx), s.prec)
            assert err == 0
            pool = self.pool[base[s.storage]]
            pbytes = pool.numel() * pool.element_size()
            p = []
            for k in range(3):
                hi = (pbytes - s.nbytes(k) - ALIGN) // ALIGN
                off = int(rng.integers(0, max(hi, 0) + 1)) * ALIGN
                p.append(pool.data_ptr() + off)
            if distinct_outputs:
                d = ring
                ring += ob
            else:
                if ring + ob > total_out:
                    ring = 0
                d = ring
                ring += ob
            self.d_off.append(d)
            p.append(self.arena.data_ptr() + d)
            self.infos.append(infos)
            self.plans.append(plan)
            self.ptrs.append(p)
            self.scalars.append((_scalar_buf(s.storage, s.alpha), _scalar_buf(s.storage, s.beta)))
        self.flops = np.array([s.flops() for s in specs])

    def output(self, i):
        """D of request i as a numpy array (distinct_outputs runs)."""
        s = self.specs[i]
        n = s.nbytes(3)
        raw = self.arena.view(self.torch.uint8)[self.d_off[i]:self.d_off[i] + n].cpu().numpy()
        return raw

    def clear_outputs(self):
        self.arena.zero_()
        self.torch.cuda.synchronize()

    # ------------------------------------------------------------------
    def run_plain(self, executor, order=None):
        """Runs every request alone, synchronously; returns per-request
        service times in seconds (wall clock around each call)."""
        L = self.tapp.lib
        st = intptr(0)
        order = range(len(self.specs)) if order is None else order
        times = np.zeros(len(self.specs))
        for i in order:
            a, b = self.scalars[i]
            A, B, Cp, D = self.ptrs[i]
            t0 = time.perf_counter()
            err = L.TAPP_execute_product(self.plans[i], executor, C.byref(st), a.ctypes.data, A, B,
                                         b.ctypes.data, Cp, D)
            times[i] = time.perf_counter() - t0
            if err:
                raise RuntimeError(f"request {i}: {err:#x} {self.tapp.explain(err)}")
        return times

    def run_plain_arrivals(self, executor, arrivals):
        """The plain path under arrivals: one caller runs the requests
        synchronously in arrival order, each started no earlier than its
        arrival time (a FIFO queue fed at `arrivals` seconds). Returns the
        measured latency of every request (completion minus arrival, seconds)
        and the span from the first arrival to the last completion."""
        L = self.tapp.lib
        st = intptr(0)
        n = len(self.specs)
        done = np.zeros(n)
        t_start = time.perf_counter()
        for i in range(n):
            target = t_start + arrivals[i]
            wait = target - time.perf_counter()
            if wait > 2e-4:
                time.sleep(wait - 1e-4)
            while time.perf_counter() < target:
                pass
            a, b = self.scalars[i]
            A, B, Cp, D = self.ptrs[i]
            err = L.TAPP_execute_product(self.plans[i], executor, C.byref(st), a.ctypes.data, A, B,
                                         b.ctypes.data, Cp, D)
            done[i] = time.perf_counter() - t_start
            if err:
                raise RuntimeError(f"request {i}: {err:#x} {self.tapp.explain(err)}")
        return done - np.asarray(arrivals), float(done[-1] - arrivals[0])

    def run_served(self, server: Server, arrivals=None):
        """Submits every request (at arrivals[i] seconds after the start,
        or all at once) and waits for all; returns the server's counters."""
        server.reset_stats()
        t_start = time.perf_counter()
        for i in range(len(self.specs)):
            if arrivals is not None:
                wait = t_start + arrivals[i] - time.perf_counter()
                if wait > 2e-4:
                    time.sleep(wait - 1e-4)
                while time.perf_counter() < t_start + arrivals[i]:
                    pass
            a, b = self.scalars[i]
            A, B, Cp, D = self.ptrs[i]
            err, _ = server.submit(self.plans[i], a.ctypes.data, A, B, b.ctypes.data, Cp, D)
            if err:
                raise RuntimeError(f"request {i}: {err:#x} {self.tapp.explain(err)}")
        err = server.drain()
        if err:
            raise RuntimeError(f"drain: {err:#x} {self.tapp.explain(err)}")
        return server.stats()

    def close(self):
        L = self.tapp.lib
        for plan, infos in zip(self.plans, self.infos):
            L.TAPP_destroy_tensor_product(plan)
            for h in infos:
                L.TAPP_destroy_tensor_info(h)
        self.plans, self.infos = [], []


def fifo_latencies(arrivals, service):
    """Latency of each request when one server takes them in arrival order
    with the given service times (a single FIFO queue)."""
    done = 0.0
    lat = np.zeros(len(arrivals))
    for i, (a, s) in enumerate(zip(arrivals, service)):
        start = max(a, done)
        done = start + s
        lat[i] = done - a
    return lat

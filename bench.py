#!/usr/bin/env python3
"""Benchmark of the TAPP tensor product on B200 (one JSON line on stdout).

Workload (one step = one TAPP_execute_product): the dense 4-index
contraction D[a,b,i,j] = sum_{c,d} A[a,c,i,d] B[d,b,c,j] + 0.5 C with every
extent 64 (M = N = K = 4096), float32 storage, inputs N(0,1) with 1% of the
entries scaled by 1e3, synthetic and seeded. The headline is the float32
product (TAPP_F32F32_ACCUM_F32) in the library's split-bfloat16 mode: each
operand split into a bfloat16 high and low part, three products accumulated
in binary32 on the tensor cores; its error against a binary64 evaluation is
on the line. The other precision modes of the same product (bfloat16, f16,
16-bit storage, the plain CUDA-core float32 path) are reported under
"modes", each with its error.

  value      TFLOP/s with all operands resident in HBM (2*M*N*K flops per
             step, CUDA events on the launching stream, max over ranks)
  e2e        the same through the C ABI with pinned HOST buffers: each step
             copies A, B, C to the device and D back (inside the timed region)
  roofline   the dominant kernel (the tcgen05 GEMM): useful flops per launch
             / its measured duration, against the measured bf16 peak; the
             tensor pipe runs three products per useful one (pipe_frac)
  cpu_baseline  the reference's own CPU product (built from its sources into
             oracle/_ref) on this host's cores, on a bounded slab of D

`--impl reference` times only the reference's CPU product (all host threads)
on the same workload, metric and precision (float32) and prints its line.
Multi-GPU runs (torchrun) are replicas: every rank runs the whole product on
its own GPU, no collective on the data path; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for p in (REPO, os.path.join(REPO, "reference-implementation_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

EXTENT = 64
FLOPS = 2.0 * (EXTENT ** 2) ** 3          # 2 * M * N * K
WORKLOAD = "dense_4index_contraction_64^4"
METRIC = f"TFLOP/s ({WORKLOAD}, F32)"     # the same string on both arms
HEADLINE = "split_bf16_f32"
STEP_DESCRIPTION = ("a pass per operand writes [hi | lo] bfloat16 panels, then one tcgen05 GEMM "
                    "(three MMAs per 16-deep step on TMA-loaded hi/lo tiles) with the fused epilogue")
MODES = {
    # name: (precision, storage of A and B, f32_mode, forced path)
    "split_bf16_f32": (0, 0, 1, 0),
    "split_bf16_f32_in_place": (0, 0, 3, 0),
    "bf16": (6, 0, 0, 0),
    "f16": (5, 0, 0, 0),
    "bf16_storage": (6, 5, 0, 0),
    "f16_storage": (5, 4, 0, 0),
    "plain_f32": (0, 0, 0, 3),
}


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-modes", action="store_true", help="skip the non-headline precision modes")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--served", type=int, default=20000,
                    help="requests in the served-stream measurement (0 skips it)")
    ap.add_argument("--only-served", action="store_true", help="print only the served-stream measurement")
    ap.add_argument("--no-double", action="store_true", help="skip the binary64 / complex-double measurement")
    ap.add_argument("--only-double", action="store_true", help="print only the binary64 / complex-double measurement")
    ap.add_argument("--only-batched", action="store_true", help="print only the batched-product measurement")
    ap.add_argument("--only-chain", action="store_true", help="print only the Tucker-chain measurement")
    ap.add_argument("--only-tucker", action="store_true", help="print only the Tucker mode-n measurement")
    ap.add_argument("--only-tiny", action="store_true", help="print only the small-product latency measurement")
    ap.add_argument("--only-small", action="store_true",
                    help="print only the small configurations and the element-path measurement")
    ap.add_argument("--only-element", action="store_true", help="print only the element-path measurement")
    ap.add_argument("--slices", type=str, default="7,8", help="digit slices of the sliced binary64 runs")
    ap.add_argument("--double-ab", type=int, default=160, help="extent of a, b, e, f in the binary64 workload")
    ap.add_argument("--double-ij", type=int, default=40, help="extent of i, j in the binary64 workload")
    ap.add_argument("--only-headline", action="store_true",
                    help="run only the timed headline steps (for profiling); prints its timing")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


# --------------------------------------------------------------------------
# CPU reference product (the reference built from its sources, else the
# oracle's restatement of it)

def cpu_reference_run(threads: int | None = None, i_slab: int = 16):
    """Times the reference's CPU product on `threads` disjoint slabs of D
    (D[:, :, 0:i_slab, t] for thread t, views into the same tensors), in
    TAPP_F32F32_ACCUM_F32, the precision of the headline. Returns a dict."""
    import oracle
    from tapp_b200.workloads import large_dense_case
    from tapp_b200.case import Tensor, Case
    threads = threads or os.cpu_count() or 1
    threads = min(threads, EXTENT)
    ref = oracle.reference_lib()
    kind = "reference" if ref is not None else "port"
    case = large_dense_case(np.random.default_rng(0), 0, 0, extent=EXTENT)
    ora = None if ref is not None else oracle.Oracle()

    def slab(t):
        D = case.D
        ext = [EXTENT, EXTENT, i_slab, 1]
        sub = Tensor(D.dtype, ext, list(D.strides), list(D.idx), 0, D.buf, D.base + t * D.strides[3])
        Cs = Tensor(case.C.dtype, ext, list(case.C.strides), list(case.C.idx), 0, case.C.buf,
                    case.C.base + t * case.C.strides[3])
        B = case.B
        Bs = Tensor(B.dtype, [EXTENT, EXTENT, EXTENT, 1], list(B.strides), list(B.idx), 0, B.buf,
                    B.base + t * B.strides[3])
        A = case.A
        As = Tensor(A.dtype, [EXTENT, EXTENT, i_slab, EXTENT], list(A.strides), list(A.idx), 0, A.buf, A.base)
        return Case(As, Bs, Cs, sub, case.alpha, case.beta, 0, False, "slab")

    slabs = [slab(t) for t in range(threads)]
    errs = [None] * threads

    def work(t):
        errs[t] = slabs[t].run(ref) if ref is not None else ora.execute(slabs[t])

    ths = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    wall = time.perf_counter() - t0
    assert all(e == 0 for e in errs), errs
    flops = 2.0 * (EXTENT * EXTENT * i_slab) * EXTENT ** 2 * threads
    return {"value": flops / wall / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": kind, "flops": flops,
            "sample": f"{threads} threads x D[:,:,0:{i_slab},t] slab ({EXTENT * EXTENT * i_slab} outputs x "
                      f"K={EXTENT ** 2} each), F32F32_ACCUM_F32; {wall:.2f} s wall",
            "seconds": wall}


def run_reference(args):
    """The reference arm: the reference's own CPU product on all host
    threads, each step one bounded slab of the workload's D (16 threads x
    D[:,:,0:2,t]); value = the slab's flops / its wall time, ms_per_step =
    that wall time (a time that ran). The reference's cost is linear in the
    number of D elements (product.c:338), so the whole step's time is the
    slab's times the ratio of flops, reported beside it."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    vals, walls = [], []
    for _ in range(min(max(args.warmup, 0), 3)):
        cpu_reference_run(i_slab=1)
    info = None
    total = 0.0
    for _ in range(max(args.steps, 1)):
        info = cpu_reference_run(i_slab=2)
        vals.append(info["value"])
        walls.append(info["seconds"])
        total += info["seconds"]
        if total > 90.0:  # keep the whole run within a few minutes
            break
    value = statistics.median(vals)
    slab_ms = statistics.median(walls) * 1e3
    slab_flops = info["flops"]
    line = {"metric": METRIC, "value": value, "unit": "TFLOP/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": len(vals), "warmup": args.warmup,
            "ms_per_step": slab_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "extents": EXTENT, "M": EXTENT ** 2, "N": EXTENT ** 2,
                       "K": EXTENT ** 2, "precision": "F32F32_ACCUM_F32",
                       "step": "one bounded slab of D on all host threads (the sample below)"},
            "extrapolation": {"slab_flops": slab_flops, "full_step_flops": FLOPS,
                              "factor": FLOPS / slab_flops, "full_step_ms_est": slab_ms * FLOPS / slab_flops},
            "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": info["cores"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GPU

class ClockSampler:
    """SM clock and clock-event (throttle) reasons of one GPU, sampled by a
    thread through NVML every `period` seconds while the block runs (read
    only; nothing is set). summary() keeps the samples inside the timed
    region's wall-clock window."""
    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("hw_power_brake_slowdown", 0x80), ("sw_power_cap", 0x4))

    def __init__(self, device: int, period: float = 0.001):
        self.device = device
        self.period = period
        self.rows = []
        self._stop = threading.Event()
        self._th = None

    def _handle(self, nv):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            return nv.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def _run(self, nv, h):
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.rows.append((time.time(), float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                  float(self.max_mhz), int(get_reasons(h))))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._th = threading.Thread(target=self._run, args=(nv, h), daemon=True)
            self._th.start()
        except Exception:
            self._th = None
        time.sleep(0.05)
        return self

    def __exit__(self, *a):
        time.sleep(0.05)
        self._stop.set()
        if self._th is not None:
            self._th.join(timeout=5)

    def summary(self, t0=None, t1=None):
        """Median SM clock and the reasons seen in [t0, t1] (wall clock); all
        samples when the window holds none."""
        rows = list(self.rows)
        inside = [r for r in rows if t0 is not None and t0 <= r[0] <= t1]
        use = inside or rows
        reasons = set()
        for r in use:
            for name, bit in self.REASONS:
                if r[3] & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median([r[1] for r in use]) if use else None,
                "sm_max_mhz": use[-1][2] if use else None, "reasons": sorted(reasons),
                "samples": len(use), "samples_in_timed_region": len(inside), "source": "NVML"}


def max_sm_mhz(device=0):
    """The GPU's maximum SM clock from NVML (read only); 1965 MHz, B200's
    maximum, when NVML cannot be read."""
    try:
        import pynvml as nv
        nv.nvmlInit()
        return float(nv.nvmlDeviceGetMaxClockInfo(nv.nvmlDeviceGetHandleByIndex(device), nv.NVML_CLOCK_SM))
    except Exception:
        return 1965.0


def nominal_cuda_core_tflops(torch, fma_lanes_per_sm):
    """Nominal CUDA-core peak in TFLOP/s: SMs x FMA lanes per SM x 2 flops x
    maximum SM clock (B200: 128 binary32 and 64 binary64 FMA lanes per SM).
    A nominal figure: the plain comparators' fractions are quoted against
    it ("of nominal"), since no measured CUDA-core peak exists here."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return sms * fma_lanes_per_sm * 2 * max_sm_mhz() * 1e6 / 1e12


INT8_DENSE_NOMINAL_TOPS = 4500.0   # B200 dense int8 tensor rate, nominal


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["bf16_tflops"], "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def profiled_traffic():
    """dram bytes per launch of the headline's GEMM (split bfloat16, panels) from
    the committed ncu summary, if any."""
    path = os.path.join(REPO, "profiles", "k_gemm_split_panels_64.md")  # written from an ncu capture
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Product:
    """One TAPP product bound to device (or host) buffers."""

    def __init__(self, lib, case, tensors, executor):
        self.lib = lib
        self.case = case
        self.ex = executor
        self.infos = [lib.tensor_info(t.dtype, t.extents, t.strides)[1] for t in (case.A, case.B, case.C, case.D)]
        err, self.plan = lib.create_product(0, [t.op for t in (case.A, case.B, case.C, case.D)], self.infos,
                                            [case.A.idx, case.B.idx, case.C.idx, case.D.idx], case.prec)
        assert err == 0
        self.ptrs = tensors

    def __call__(self, status=None):
        st = C.c_ssize_t(0)
        err = self.lib.lib.TAPP_execute_product(self.plan, self.ex, C.byref(st), self.case.alpha.ctypes.data,
                                                self.ptrs[0], self.ptrs[1], self.case.beta.ctypes.data,
                                                self.ptrs[2], self.ptrs[3])
        if err:
            raise RuntimeError(f"TAPP_execute_product failed: {err} {self.lib.explain(err)}")
        if status is not None:
            status.append(st.value)

    def close(self):
        self.lib.lib.TAPP_destroy_tensor_product(self.plan)
        for h in self.infos:
            self.lib.lib.TAPP_destroy_tensor_info(h)


def to_device(t, torch):
    x = torch.from_numpy(t.buf.view(np.uint8)).cuda()
    return x, x.data_ptr() + t.base * t.itemsize


def make_executor(lib, stream, f32_mode=0, path=0, async_=True, status=False):
    import tapp_b200
    ex = lib.create_executor()
    if stream is not None:
        lib.set_stream(ex, stream)
    lib.set_int(ex, tapp_b200.ATTR_ASYNC, 1 if async_ else 0)
    lib.set_int(ex, tapp_b200.ATTR_F32_MODE, f32_mode)
    lib.set_int(ex, tapp_b200.ATTR_PATH, path)
    lib.set_int(ex, tapp_b200.ATTR_WANT_STATUS, 1 if status else 0)
    return ex


def replica_max(dist, value, device):
    """The largest of a per-rank scalar over the ranks (the slowest replica's
    time); the value itself with one rank (dist None)."""
    if dist is None:
        return value
    import torch
    x = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())


def replica_tflops(world, flops_per_rank, seconds):
    """Whole-job throughput of `world` replicas that each did `flops_per_rank`
    in at most `seconds` (weak scaling: the work per rank is fixed)."""
    return world * flops_per_rank / seconds / 1e12


def time_device(torch, fn, steps, warmup, barrier, window=None):
    """Mean device time of one step in ms: `warmup` untimed steps, then
    `steps` steps between CUDA events on the current stream, bracketed by a
    barrier and a device synchronisation on both sides."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(s)
    for _ in range(steps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    w1 = time.time()
    barrier()
    if window is not None:
        window[:] = [w0, w1]
    return e0.elapsed_time(e1) / steps  # ms


def mode_case(name, rng_seed=1):
    from tapp_b200.workloads import large_dense_case
    prec, storage, _, _ = MODES[name]
    return large_dense_case(np.random.default_rng(rng_seed), prec, storage, extent=EXTENT)


def f64_slab_reference(lib, torch, case, j_count=2):
    """Binary64 evaluation, on the GPU through the library's own F64F64
    path, of D[:, :, :, 0:j_count] for the exact stored inputs of `case`."""
    from tapp_b200.case import Tensor, Case, alloc, scalar, bf16_to_f32
    from tapp_b200.abi import TAPP_F64, TAPP_BF16

    def f64(t, ext=None):
        vals = bf16_to_f32(t.buf) if t.dtype == TAPP_BF16 else t.buf
        T = Tensor(TAPP_F64, list(ext or t.extents), list(t.strides), list(t.idx), 0,
                   np.asarray(vals, dtype=np.float64).copy(), t.base)
        return T
    e = EXTENT
    A = f64(case.A)
    B = f64(case.B, [e, e, e, j_count])
    Cc = f64(case.C, [e, e, e, j_count])
    D = f64(case.D, [e, e, e, j_count])
    c64 = Case(A, B, Cc, D, scalar(TAPP_F64, float(case.alpha[0])), scalar(TAPP_F64, float(case.beta[0])), 1)
    dev = [to_device(t, torch) for t in (A, B, Cc, D)]
    ex = make_executor(lib, None, async_=False)
    prod = Product(lib, c64, [d[1] for d in dev], ex)
    prod()
    prod.close()
    lib.lib.TAPP_destroy_executor(ex)
    out = dev[3][0].cpu().numpy().view(np.float64)
    offs = D.offsets()
    return out[D.base + offs]


def slab_values(case_D, dbuf, j_count=2):
    from tapp_b200.case import Tensor
    e = EXTENT
    sub = Tensor(case_D.dtype, [e, e, e, j_count], list(case_D.strides), list(case_D.idx), 0, None, case_D.base)
    return dbuf[case_D.base + sub.offsets()].astype(np.float64)


C4_AB, C4_IJ = 160, 40


def batched_measure(lib, torch, batches=64, n=512, steps=20):
    """TAPP_execute_batched_product against one TAPP_execute_product per batch:
    `batches` products D[a,b] = sum_k A[a,k] B[k,b] + 0.5 C with a = b = k = n,
    float32 storage, BF16BF16_ACCUM_F32, operands resident in HBM (synthetic,
    uniform in [-1, 1]). The batched call runs one pack launch per operand and
    one GEMM for all batches."""
    import ctypes as Cty
    from tapp_b200.case import Case, Tensor, scalar
    T = lambda ext, idx: Tensor(0, ext, [1, ext[0]], [ord(c) for c in idx], 0, None, 0)
    case = Case(T([n, n], "ak"), T([n, n], "kb"), T([n, n], "ab"), T([n, n], "ab"), scalar(0, 1.0), scalar(0, 0.5), 6)
    bufs = {k: torch.rand(batches, n * n, device="cuda") * 2 - 1 for k in "ABCD"}
    arrs = {k: (Cty.c_void_p * batches)(*[bufs[k][i].data_ptr() for i in range(batches)]) for k in "ABCD"}
    ex = make_executor(lib, torch.cuda.current_stream().cuda_stream)
    prod = Product(lib, case, [bufs[k][0].data_ptr() for k in "ABCD"], ex)

    def batched():
        st = Cty.c_ssize_t(0)
        err = lib.lib.TAPP_execute_batched_product(prod.plan, ex, Cty.byref(st), batches, case.alpha.ctypes.data,
                                                   arrs["A"], arrs["B"], case.beta.ctypes.data, arrs["C"], arrs["D"])
        if err:
            raise RuntimeError(f"TAPP_execute_batched_product: {err}")

    def singles():
        for i in range(batches):
            prod.ptrs = [bufs[k][i].data_ptr() for k in "ABCD"]
            prod()

    flops = 2.0 * n ** 3 * batches
    n0 = lib.launches()
    t_b = time_device(torch, batched, steps, 3, lambda: None)
    l_b = (lib.launches() - n0) // (steps + 3)
    n0 = lib.launches()
    t_s = time_device(torch, singles, steps, 3, lambda: None)
    l_s = (lib.launches() - n0) // (steps + 3)
    prod.close()
    lib.lib.TAPP_destroy_executor(ex)
    return {"workload": f"{batches} x D[a,b] = sum_k A[a,k] B[k,b] + 0.5 C, a=b=k={n}, f32 storage, BF16BF16_ACCUM_F32",
            "batched": {"tflops": flops / (t_b * 1e-3) / 1e12, "ms": t_b, "launches": l_b},
            "one_call_per_batch": {"tflops": flops / (t_s * 1e-3) / 1e12, "ms": t_s, "launches": l_s},
            "speedup": t_s / t_b}


def small_configs_measure(lib, torch, with_cpu=True, steps=200, e2e_calls=50):
    """The reference's own small cases, through the C ABI:
      c1  D[a,b,c,d] = 1.3 sum_{e,f} A[a,e,b,f] B[f,c,e,d] + 0.7 C, float32,
          F32F32_ACCUM_F32, every extent 16, dense column-major, U[-1, 1]:
          plain CUDA-core float32 and split bfloat16;
      c2  D[a,h,c] = alpha sum_{k,u,v} A[a,h,k,k,u] conj(B[k,h,c,v]) + beta C,
          complex float, DEFAULT precision (Hadamard h, diagonal k, unary u and
          v; A a view with a negative and a zero stride; D permuted against C).
    Per call: device time with operands in HBM (CUDA events, `steps` calls)
    and end-to-end time from pinned host buffers (synchronous calls, wall
    clock). With with_cpu, the reference's CPU product runs the same inputs
    (one call, one thread, best of 3) and the GPU results are compared with
    its D: max |D_gpu - D_ref| / max |D_ref|."""
    from tapp_b200.workloads import dense_contraction_case, mixed_classes_case
    ref = None
    if with_cpu:
        import oracle
        ref = oracle.reference_lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = {"c1": (dense_contraction_case(np.random.default_rng(0x7A990001), extent=16), 2.0 * 16 ** 6,
                    [("plain_f32", 0), ("split_bf16_f32", 1)]),
             "c2": (mixed_classes_case(np.random.default_rng(0x7A990002)), 8.0 * 40 * 36 * 24 * 12,
                    [("default_c32", 0)])}
    out = {}
    for key, (case, flops, variants) in cases.items():
        res = {"flops": flops}
        d_ref = None
        if ref is not None:
            walls = []
            for _ in range(3):
                rc = case.copy()
                t0 = time.perf_counter()
                assert rc.run(ref) == 0
                walls.append(time.perf_counter() - t0)
            d_ref = rc.D.buf[rc.D.base + rc.D.offsets()].astype(np.complex128)
            res["reference_cpu"] = {"ms": min(walls) * 1e3, "cores": 1, "gflops": flops / min(walls) / 1e9,
                                    "kind": "reference"}
        for name, f32_mode in variants:
            dev = [to_device(t, torch) for t in (case.A, case.B, case.C, case.D)]
            ex = make_executor(lib, stream, f32_mode=f32_mode)
            prod = Product(lib, case, [d[1] for d in dev], ex)
            ms = time_device(torch, prod, steps, 10, lambda: None)
            got = dev[3][0].cpu().numpy().view(case.D.buf.dtype)
            prod.close()
            lib.lib.TAPP_destroy_executor(ex)
            # from pinned host buffers, D copied back every call
            pinned = []
            for t in (case.A, case.B, case.C, case.D):
                h = torch.from_numpy(t.buf.view(np.uint8).copy()).pin_memory()
                pinned.append((h, h.data_ptr() + t.base * t.itemsize))
            ex_h = make_executor(lib, None, f32_mode=f32_mode, async_=False)
            prod_h = Product(lib, case, [q[1] for q in pinned], ex_h)
            for _ in range(3):
                prod_h()
            t0 = time.perf_counter()
            for _ in range(e2e_calls):
                prod_h()
            e2e_us = (time.perf_counter() - t0) / e2e_calls * 1e6
            prod_h.close()
            lib.lib.TAPP_destroy_executor(ex_h)
            v = {"device_us": ms * 1e3, "tflops": flops / (ms * 1e-3) / 1e12, "e2e_us": e2e_us,
                 "h2d_bytes": sum(t.buf.nbytes for t in (case.A, case.B, case.C)), "d2h_bytes": case.D.buf.nbytes}
            if d_ref is not None:
                # repeated steps apply beta * C to the same C, so D is the same every step
                g = got[case.D.base + case.D.offsets()].astype(np.complex128)
                v["max_abs_err_vs_reference_rel_to_max"] = float(np.abs(g - d_ref).max() / np.abs(d_ref).max())
                v["speedup_vs_reference_cpu_e2e"] = res["reference_cpu"]["ms"] * 1e3 / e2e_us
            res[name] = v
            del dev, pinned
        out[key] = res
    out["c1"]["split_vs_plain_device"] = out["c1"]["plain_f32"]["device_us"] / out["c1"]["split_bf16_f32"]["device_us"]
    return out


def element_measure(lib, torch, steps=20, warmup=3):
    """Element-path products through the C ABI, operands in HBM; device time
    per product (CUDA events) and algorithmic bytes (A + B + C + D spans):
      hadamard  the served mix's largest batched Hadamard product of the first
                140 requests: D[l3,l2,l1,l0] = sum_k A[l0,l1,k,l2,l3]
                B[l2,k,l0,l1] + C, extents l0..l3 = 72, 8, 74, 67, k = 69,
                float32 (A 790 MB, contiguous along l0; D along l3): the
                outputs are walked in A's stride order;
      matvec    batched matrix-vector D[m,h] = sum_k A[k,m,h] B[k,h] + C,
                k = 300, m = 2000, h = 64, A contiguous along k: one warp per
                output (k_warpdot);
      c2        the mixed-class complex product (element kernel)."""
    from tapp_b200.workloads import RequestSpec, case_from_spec, mixed_classes_case
    stream = torch.cuda.current_stream().cuda_stream
    specs = {
        "hadamard": RequestSpec("hadamard", 0, 0, ([72, 8, 69, 74, 67], [74, 69, 72, 8], [67, 74, 8, 72], [67, 74, 8, 72]),
                                ([0, 1, 4, 2, 3], [2, 4, 0, 1], [3, 2, 1, 0], [3, 2, 1, 0]), 0.9, -0.3),
        "matvec": RequestSpec("hadamard", 0, 0, ([300, 2000, 64], [300, 64], [2000, 64], [2000, 64]),
                              ([0, 1, 2], [0, 2], [1, 2], [1, 2]), 0.9, -0.3),
    }
    out = {}
    for name in ("hadamard", "matvec", "c2"):
        if name == "c2":
            case = mixed_classes_case(np.random.default_rng(0x7A990002))
            nbytes = sum(t.buf.nbytes for t in (case.A, case.B, case.C, case.D))
        else:
            case = case_from_spec(np.random.default_rng(11), specs[name])
            nbytes = sum(specs[name].nbytes(k) for k in range(4))
        dev = [to_device(t, torch) for t in (case.A, case.B, case.C, case.D)]
        ex = make_executor(lib, stream)
        prod = Product(lib, case, [d[1] for d in dev], ex)
        desc = lib.describe(prod.plan)
        ms = time_device(torch, prod, steps, warmup, lambda: None)
        out[name] = {"kernel": desc.split("kernel=")[1].split()[0] if "kernel=" in desc else desc.split()[0],
                     "us": ms * 1e3, "bytes": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9}
        prod.close()
        lib.lib.TAPP_destroy_executor(ex)
        del dev
    return out


def tiny_latency_measure(lib, torch, n=2000):
    """Latency of small products (the element path: the mixed-class
    configuration, complex float with Hadamard, diagonal and unary modes, and
    4-index contractions with extents 4, binary32 and binary64), operands in
    HBM, one product at a time (submit, then wait for it):
      plain   synchronous TAPP_execute_product (a launch and a stream wait)
      server  tapp_b200_server_submit + wait (host scheduler thread, streams,
              stream callbacks)
      loop    tapp_b200_loop_submit + wait (the device-resident loop: no
              launch per product)
    and the throughput of `n` products submitted back to back then waited."""
    from tapp_b200.workloads import dense_contraction_case, mixed_classes_case
    from tapp_b200.server import Server
    rng = np.random.default_rng(17)
    cases = [mixed_classes_case(np.random.default_rng(0x7A990002)),
             dense_contraction_case(rng, extent=4), dense_contraction_case(rng, extent=4, dtype=1, prec=1)]
    devs = []
    for c in cases:
        ts = (c.A, c.B, c.C, c.D)
        bufs = [to_device(t, torch) for t in ts]
        infos = [lib.tensor_info(t.dtype, t.extents, t.strides)[1] for t in ts]
        err, plan = lib.create_product(0, [t.op for t in ts], infos, [t.idx for t in ts], c.prec)
        assert err == 0
        devs.append((c, bufs, infos, plan))
    args = lambda d: (d[0].alpha.ctypes.data, d[1][0][1], d[1][1][1], d[0].beta.ctypes.data, d[1][2][1], d[1][3][1])
    order = [devs[i % len(devs)] for i in range(n)]
    out = {"workload": "small element-path products (mixed-class complex float; 4-index contractions, extents 4, "
                       "f32 and f64), operands in HBM", "products": n}
    # plain
    ex = lib.create_executor()
    lat = []
    for d in order[:200]:
        a = args(d)
        st = C.c_ssize_t(0)
        lib.lib.TAPP_execute_product(d[3], ex, C.byref(st), *a)
    for d in order:
        a = args(d)
        st = C.c_ssize_t(0)
        t0 = time.perf_counter()
        lib.lib.TAPP_execute_product(d[3], ex, C.byref(st), *a)
        lat.append(time.perf_counter() - t0)
    lib.lib.TAPP_destroy_executor(ex)
    lat = np.array(lat) * 1e6
    out["plain"] = {"p50_us": float(np.percentile(lat, 50)), "p99_us": float(np.percentile(lat, 99))}
    # server, one at a time, then all at once
    with Server(lib, 8 << 30, n_streams=4, max_in_flight=64) as srv:
        for d in order[:200]:
            srv.wait(srv.submit(d[3], *args(d))[1])
        srv.reset_stats()
        for d in order:
            err, t = srv.submit(d[3], *args(d))
            srv.wait(t)
        one = srv.stats()
        srv.reset_stats()
        t0 = time.perf_counter()
        for d in order:
            srv.submit(d[3], *args(d))
        srv.drain()
        burst_s = time.perf_counter() - t0
    out["server"] = {"p50_us": one["p50_us"], "p99_us": one["p99_us"], "burst_products_per_s": n / burst_s}
    # device loop
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    err, loop = lib.loop_create(0, blocks=sms, slots=256, idle_ms=100.0)
    assert err == 0
    for d in order[:200]:
        lib.lib.tapp_b200_loop_wait(loop, lib.loop_submit(loop, d[3], *args(d))[1])
    lib.lib.tapp_b200_loop_reset_stats(loop)
    for d in order:
        err, t = lib.loop_submit(loop, d[3], *args(d))
        lib.lib.tapp_b200_loop_wait(loop, t)
    one = lib.loop_stats(loop)
    lib.lib.tapp_b200_loop_reset_stats(loop)
    t0 = time.perf_counter()
    tickets = [lib.loop_submit(loop, d[3], *args(d))[1] for d in order]
    for t in tickets:
        lib.lib.tapp_b200_loop_wait(loop, t)
    burst_s = time.perf_counter() - t0
    out["loop"] = {"p50_us": one["p50_us"], "p99_us": one["p99_us"], "burst_products_per_s": n / burst_s,
                   "launches": one["launches"]}
    lib.lib.tapp_b200_loop_destroy(loop)
    out["loop_vs_server_p50"] = out["server"]["p50_us"] / out["loop"]["p50_us"]
    for c, bufs, infos, plan in devs:
        lib.lib.TAPP_destroy_tensor_product(plan)
        for h in infos:
            lib.lib.TAPP_destroy_tensor_info(h)
    return out


def hbm_peak():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


TUCKER_CASES = [  # (core extents, contracted mode, rank, storage, precision)
    ([128, 40, 128, 128], 1, 38, 0, 0),
    ([128, 40, 128, 128], 0, 38, 0, 0),
    ([128, 40, 128, 128], 1, 38, 0, 6),
    ([77, 190, 133, 61], 2, 33, 0, 0),
    ([96, 200, 90, 64], 3, 24, 1, -1),
    ([128, 40, 128, 128], 1, 24, 2, -1),
]


def tucker_measure(lib, torch, steps=10, warmup=3):
    """Tucker mode-n products D = 0.7 core x_n U + 0.3 C (the served mix's most common kind:
    U is rank x extent, D has the rank at mode n), operands resident in HBM, uniform in [-1, 1].
    Device time per product with CUDA events; algorithmic bytes = A + B + C + D."""
    from tapp_b200.workloads import RequestSpec, case_from_spec
    peak, peak_kind = hbm_peak()
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for core, mode, R, storage, prec in TUCKER_CASES:
        o = len(core)
        d_ext = list(core)
        d_ext[mode] = R
        d_idx = list(range(o))
        d_idx[mode] = o
        spec = RequestSpec("tucker", storage, prec, (core, [R, core[mode]], d_ext, d_ext),
                           (list(range(o)), [o, mode], d_idx, d_idx), 0.7, 0.3)
        case = case_from_spec(np.random.default_rng(3), spec)
        dev = [to_device(t, torch) for t in (case.A, case.B, case.C, case.D)]
        ex = make_executor(lib, stream)
        prod = Product(lib, case, [d[1] for d in dev], ex)
        ms = time_device(torch, prod, steps, warmup, lambda: None)
        nbytes = sum(spec.nbytes(k) for k in range(4))
        gbs = nbytes / (ms * 1e-3) / 1e9
        out.append({"core": core, "mode": mode, "rank": R, "storage": ["f32", "f64", "c32", "c64"][storage], "precision": prec,
                    "us": ms * 1e3, "gbs": gbs, "hbm_frac": gbs / peak, "tflops": spec.flops() / (ms * 1e-3) / 1e12})
        prod.close()
        lib.lib.TAPP_destroy_executor(ex)
        del dev
    return {"workload": "Tucker mode-n products D = 0.7 core x_n U + 0.3 C, operands in HBM (> L2)",
            "hbm_peak_gbs": peak, "peak_kind": peak_kind, "cases": out}


def chain_measure(lib, torch, r=64, n=256, reps=10):
    """Tucker reconstruction X[a,b,c] = sum_{i,j,k} G[i,j,k] U1[a,i] U2[b,j] U3[c,k] (core r^3,
    factors n x r, float32, F32F32_ACCUM_F32; synthetic, uniform in [-1, 1]) from pinned HOST
    buffers: tapp_b200_execute_chain (intermediates stay on the device, one host wait) against
    three TAPP_execute_product calls (each intermediate copied back and forth). Wall clock."""
    import ctypes as Cty
    from tapp_b200.case import Tensor, scalar
    i_, j_, k_, a_, b_, c_ = (ord(x) for x in "ijkabc")
    shapes = [([r, r, r], [i_, j_, k_], [n, r], [a_, i_], [n, r, r], [a_, j_, k_]),
              ([n, r, r], [a_, j_, k_], [n, r], [b_, j_], [n, n, r], [a_, b_, k_]),
              ([n, n, r], [a_, b_, k_], [n, r], [c_, k_], [n, n, n], [a_, b_, c_])]

    def colmajor(e):
        st, acc = [], 1
        for x in e:
            st.append(acc)
            acc *= x
        return st

    def pinned(numel):
        t = torch.empty(numel, dtype=torch.float32).pin_memory()
        t.uniform_(-1, 1)
        return t

    G = pinned(r ** 3)
    U = [pinned(n * r) for _ in range(3)]
    outs = [pinned(int(np.prod(s[4]))) for s in shapes]
    alpha, beta = scalar(0, 1.0), scalar(0, 0.0)
    plans, infos = [], []
    for ae, ai, be, bi, de, di in shapes:
        inf = [lib.tensor_info(0, e, colmajor(e))[1] for e in (ae, be, de, de)]
        _, plan = lib.create_product(0, [0, 0, 0, 0], inf, [ai, bi, di, di], 0)
        plans.append(plan)
        infos += inf
    ex = lib.create_executor()
    f = lib.lib.tapp_b200_execute_chain
    f.restype = Cty.c_int
    f.argtypes = [Cty.c_int, Cty.POINTER(Cty.c_ssize_t), Cty.c_ssize_t] + [Cty.POINTER(Cty.c_void_p)] * 6
    arr = lambda v: (Cty.c_void_p * len(v))(*v)
    P = (Cty.c_ssize_t * 3)(*plans)
    al, be_ = arr([alpha.ctypes.data] * 3), arr([beta.ctypes.data] * 3)
    A = arr([G.data_ptr(), None, None])
    B = arr([u.data_ptr() for u in U])
    D = arr([None, None, outs[2].data_ptr()])

    def chain():
        if f(3, P, ex, al, be_, A, B, None, D):
            raise RuntimeError("tapp_b200_execute_chain failed")

    def steps():
        src = G
        for s_, (plan, u, o) in enumerate(zip(plans, U, outs)):
            st = Cty.c_ssize_t(0)
            if lib.lib.TAPP_execute_product(plan, ex, Cty.byref(st), alpha.ctypes.data, src.data_ptr(), u.data_ptr(),
                                            beta.ctypes.data, None, o.data_ptr()):
                raise RuntimeError("TAPP_execute_product failed")
            src = o

    def wall(fn):
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts) * 1e3

    t_chain, t_steps = wall(chain), wall(steps)
    for plan in plans:
        lib.lib.TAPP_destroy_tensor_product(plan)
    for h in infos:
        lib.lib.TAPP_destroy_tensor_info(h)
    lib.lib.TAPP_destroy_executor(ex)
    flops = 2.0 * (n * r ** 3 + n * n * r ** 2 + n ** 3 * r)
    return {"workload": f"Tucker reconstruction, core {r}^3, factors {n}x{r}, float32, pinned host operands",
            "chain_ms": t_chain, "three_calls_ms": t_steps, "speedup": t_steps / t_chain,
            "chain_tflops_e2e": flops / (t_chain * 1e-3) / 1e12,
            "h2d_bytes": 4 * (r ** 3 + 3 * n * r), "d2h_bytes": 4 * n ** 3}


def double_measure(lib, torch, slices_list=(7, 8), steps=2, samples=256, ab=C4_AB, ij=C4_IJ):
    """The binary64 configuration: D[a,b,i,j] = sum_{e,f} A[a,b,e,f] B[e,f,i,j] + C
    with a = b = e = f = 160 and i = j = 40 (M = K = 25600, N = 1600), once in
    binary64 and once in complex double with conj(A); |x| log-uniform in
    [1e-8, 1] with random sign (phase), beta = 1; synthetic, generated on the
    GPU. Native binary64 CUDA-core path against the sliced path (S 8-bit digit
    slices on the integer tensor cores). Error: max |D - D_ref| / max |D_ref|
    over sampled outputs, D_ref accumulated in extended precision (numpy
    longdouble) from the same inputs."""
    import math
    import tapp_b200
    from tapp_b200.case import Case, Tensor, scalar
    from tapp_b200.abi import TAPP_F64, TAPP_C64, TAPP_CONJUGATE
    M, N, K = ab * ab, ij * ij, ab * ab
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    rng = np.random.default_rng(44)
    out = {}
    for cplx in (False, True):
        dt = torch.complex128 if cplx else torch.float64

        def logu(n):
            mag = torch.pow(10.0, torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 8 - 8)
            if cplx:
                ph = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * (2 * math.pi)
                return torch.polar(mag, ph)
            return mag * torch.where(torch.rand(n, device="cuda", generator=g) < 0.5, -1.0, 1.0).to(torch.float64)

        A, B, Cc = logu(M * K), logu(K * N), logu(M * N)
        D = torch.zeros(M * N, dtype=dt, device="cuda")
        ty = TAPP_C64 if cplx else TAPP_F64

        def T(ext, idx, op=0):
            st, acc = [], 1
            for e_ in ext:
                st.append(acc)
                acc *= e_
            return Tensor(ty, ext, st, [ord(c) for c in idx], op, None, 0)

        case = Case(T([ab] * 4, "abef", TAPP_CONJUGATE if cplx else 0), T([ab, ab, ij, ij], "efij"),
                    T([ab, ab, ij, ij], "abij"), T([ab, ab, ij, ij], "abij"), scalar(ty, 1.0), scalar(ty, 1.0), -1)
        ptrs = [A.data_ptr(), B.data_ptr(), Cc.data_ptr(), D.data_ptr()]
        flops = 2.0 * M * N * K * (4 if cplx else 1)
        ms = rng.integers(0, M, samples)
        ns = rng.integers(0, N, samples)
        a_rows = A.view(K, M)[:, torch.from_numpy(ms).cuda()].cpu().numpy()        # [k, sample]
        b_cols = B.view(N, K)[torch.from_numpy(ns).cuda(), :].cpu().numpy()        # [sample, k]
        c_vals = Cc.view(N, M)[torch.from_numpy(ns).cuda(), torch.from_numpy(ms).cuda()].cpu().numpy()
        ld = np.clongdouble if cplx else np.longdouble
        ref = np.empty(samples, dtype=ld)
        for i in range(samples):
            a = a_rows[:, i].astype(ld)
            if cplx:
                a = np.conj(a)
            ref[i] = np.sum(a * b_cols[i].astype(ld)) + ld(c_vals[i])
        ref_max = float(np.max(np.abs(ref)))

        def run(label, f64_mode):
            ex = make_executor(lib, torch.cuda.current_stream().cuda_stream)
            lib.set_int(ex, 0x1007, f64_mode)
            prod = Product(lib, case, ptrs, ex)
            t_ms = time_device(torch, prod, steps, 1, lambda: None)
            ex_s = make_executor(lib, torch.cuda.current_stream().cuda_stream, async_=False, status=True)
            lib.set_int(ex_s, 0x1007, f64_mode)
            prod_s = Product(lib, case, ptrs, ex_s)
            st = []
            prod_s(st)
            path = lib.status_value(st[0], tapp_b200.STATUS_PATH)
            main_us = lib.status_value(st[0], tapp_b200.STATUS_MAIN_US)
            kernels = lib.status_value(st[0], tapp_b200.STATUS_KERNELS)
            lib.lib.TAPP_destroy_status(st[0])
            got = D.view(N, M)[torch.from_numpy(ns).cuda(), torch.from_numpy(ms).cuda()].cpu().numpy()
            err = float(np.max(np.abs(got.astype(ld) - ref))) / ref_max
            r = {"tflops": flops / (t_ms * 1e-3) / 1e12, "ms": t_ms, "path": ["noop", "generic", "reduce", "simt",
                 "tc", "sliced"][path], "kernels": kernels, "max_abs_err_rel_to_max": err}
            if f64_mode:
                levels = f64_mode * (f64_mode + 1) // 2
                int8_ops = 2.0 * M * N * (2 if cplx else 1) * K * (2 if cplx else 1) * levels
                r["slices"] = f64_mode
                r["int8_gemm_ms"] = main_us / 1e3
                r["int8_tops"] = int8_ops / (main_us * 1e-6) / 1e12
                r["int8_frac_of_nominal"] = r["int8_tops"] / INT8_DENSE_NOMINAL_TOPS
            prod.close()
            prod_s.close()
            lib.lib.TAPP_destroy_executor(ex)
            lib.lib.TAPP_destroy_executor(ex_s)
            return r

        res = {"native": run("native", 0)}
        res["native"]["fp64_pipe_frac_of_nominal"] = res["native"]["tflops"] / nominal_cuda_core_tflops(torch, 64)
        for S in slices_list:
            res[f"sliced_{S}"] = run(f"sliced_{S}", S)
            res[f"sliced_{S}"]["vs_native"] = res[f"sliced_{S}"]["tflops"] / res["native"]["tflops"]
        # the headline point: 8 slices (error at or below the native path's; 7 slices trade accuracy)
        hs = 8 if 8 in slices_list else max(slices_list, default=0)
        if hs:
            res["headline"] = {"slices": hs, "tflops": res[f"sliced_{hs}"]["tflops"],
                               "vs_native": res[f"sliced_{hs}"]["vs_native"],
                               "max_abs_err_rel_to_max": res[f"sliced_{hs}"]["max_abs_err_rel_to_max"],
                               "native_max_abs_err_rel_to_max": res["native"]["max_abs_err_rel_to_max"]}
        out["c64_conjA" if cplx else "f64"] = res
        del A, B, Cc, D
        torch.cuda.empty_cache()
    out["config"] = (f"D[a,b,i,j] = sum_{{e,f}} A[a,b,e,f] B[e,f,i,j] + C, a=b=e=f={ab}, i=j={ij}; "
                     "|x| log-uniform [1e-8,1], random sign / phase, beta=1")
    out["error_reference"] = f"{samples} sampled outputs accumulated in numpy longdouble"
    return out


def served_measure(lib, torch, n, seed=5, max_tensor_bytes=1 << 30, load=1.05):
    """The served configuration: n requests (20,000 by default) of the served
    mix with every tensor at most max_tensor_bytes (with tensors up to the
    64 GB budget the configuration moves about 34 TB, hours of HBM traffic),
    operands resident in HBM. A first
    plain pass measures each request's service time; Poisson arrivals at
    `load` times the plain path's capacity (past its saturation) then drive
    both arms, and both arms' latencies are measured:
      plain   one caller runs synchronous TAPP_execute_product calls in
              arrival order (a FIFO queue: a request starts at its arrival or
              when the previous one ends);
      served  the same requests submitted to a server at their arrivals.
    The served arm also runs all requests at once (its capacity)."""
    from tapp_b200.workloads import served_stream
    from tapp_b200.served import StreamRunner
    from tapp_b200.server import Server
    rng = np.random.default_rng(seed)
    specs = served_stream(rng, n, max_tensor_bytes=max_tensor_bytes)
    run = StreamRunner(lib, specs, torch, seed=seed)
    ex = make_executor(lib, None, async_=False)
    run.run_plain(ex)      # warm-up over the whole stream: first-use kernel loads, pool growth
    service = run.run_plain(ex)
    t_plain = float(service.sum())
    capacity = n / t_plain
    rate = load * capacity
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    plain_lat, plain_span = run.run_plain_arrivals(ex, arrivals)
    lib.lib.TAPP_destroy_executor(ex)
    flops = float(run.flops.sum())
    with Server(lib, 64 << 30, n_streams=8, max_in_flight=64) as srv:
        run.run_served(srv, arrivals=None)               # warm-up of the served path
        burst = run.run_served(srv, arrivals=None)
        poisson = run.run_served(srv, arrivals=arrivals)
    run.close()

    def served_summary(st):
        return {"req_per_s": st["requests_per_s"], "tflops": flops / st["span_s"] / 1e12,
                "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3, "span_s": st["span_s"],
                "units": st["units"], "grouped_requests": st["grouped"], "peak_in_flight": st["peak_in_flight"],
                "failed": st["failed"]}
    kinds = {}
    for s_ in specs:
        kinds[s_.kind] = kinds.get(s_.kind, 0) + 1
    srv_p = served_summary(poisson)
    plain = {"req_per_s": n / plain_span, "capacity_req_per_s": capacity, "tflops": flops / plain_span / 1e12,
             "service_mean_ms": 1e3 * t_plain / n,
             "p50_ms": 1e3 * float(np.percentile(plain_lat, 50)), "p99_ms": 1e3 * float(np.percentile(plain_lat, 99)),
             "how": "synchronous TAPP_execute_product per request, run in arrival order as they arrive (measured)"}
    return {
        "workload": "served stream: 50% Tucker mode-n, 30% binary, 20% Hadamard+contraction; "
                    "40% f32, 30% bf16-accum-f32, 20% f64, 10% c32; HBM budget 64 GB",
        "requests": n, "requests_by_kind": kinds, "max_tensor_bytes": max_tensor_bytes,
        "total_gflop": flops / 1e9,
        "reduction": (f"{n} of 20000 requests; " if n < 20000 else "all 20000 requests; ") +
                     f"every tensor <= {max_tensor_bytes >> 20} MiB (the configuration as stated, with tensors up "
                     "to the 64 GB budget, moves ~34 TB, 1.5 h or more at HBM speed)",
        "arrival_rate_per_s": rate, "load_vs_plain_capacity": load,
        "plain": plain,
        "served_poisson": srv_p,
        "served_burst": served_summary(burst),
        "burst_vs_plain_capacity": burst["requests_per_s"] / capacity,
        "served_vs_plain_p99": plain["p99_ms"] / srv_p["p99_ms"] if srv_p["p99_ms"] else None,
    }


def run_b200(args):
    import torch
    import tapp_b200
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    lib = tapp_b200.load()
    stream = torch.cuda.current_stream().cuda_stream
    if args.only_served:
        if rank == 0:
            print(json.dumps(served_measure(lib, torch, max(args.served, 1))), flush=True)
        return
    slices = tuple(int(x) for x in args.slices.split(",") if x)
    if args.only_chain:
        if rank == 0:
            print(json.dumps(chain_measure(lib, torch)), flush=True)
        return
    if args.only_tucker:
        if rank == 0:
            print(json.dumps(tucker_measure(lib, torch)), flush=True)
        return
    if args.only_tiny:
        if rank == 0:
            print(json.dumps(tiny_latency_measure(lib, torch)), flush=True)
        return
    if args.only_element:
        if rank == 0:
            print(json.dumps(element_measure(lib, torch)), flush=True)
        return
    if args.only_small:
        if rank == 0:
            print(json.dumps({"small_configs": small_configs_measure(lib, torch, with_cpu=False),
                              "element": element_measure(lib, torch)}), flush=True)
        return
    if args.only_batched:
        if rank == 0:
            print(json.dumps(batched_measure(lib, torch)), flush=True)
        return
    if args.only_double:
        if rank == 0:
            print(json.dumps(double_measure(lib, torch, slices, ab=args.double_ab, ij=args.double_ij)), flush=True)
        return

    # ---------------- headline: float32 in split-bfloat16 mode, operands in HBM ----------------
    case = mode_case(HEADLINE)
    _, _, head_f32_mode, _ = MODES[HEADLINE]
    dev = [to_device(t, torch) for t in (case.A, case.B, case.C, case.D)]
    ex = make_executor(lib, stream, f32_mode=head_f32_mode)
    prod = Product(lib, case, [d[1] for d in dev], ex)
    n0 = lib.launches()
    window = [None, None]
    with ClockSampler(local_rank) as clk:
        t_ms = time_device(torch, prod, args.steps, args.warmup, barrier, window)
    launches = lib.launches() - n0
    gpu_launches = launches * args.steps // (args.steps + args.warmup)
    clocks = clk.summary(*window)
    if args.only_headline:
        if rank == 0:
            print(json.dumps({"ms_per_step": t_ms, "tflops": FLOPS / (t_ms * 1e-3) / 1e12,
                              "gpu_launches": gpu_launches, "clocks": clocks}), flush=True)
        prod.close()
        lib.lib.TAPP_destroy_executor(ex)
        if dist is not None:
            dist.destroy_process_group()
        return
    t_max = replica_max(dist, t_ms, "cuda")
    value = replica_tflops(world, FLOPS, t_max * 1e-3)

    # ---------------- dominant kernel: GEMM duration per launch ----------------
    ex_s = make_executor(lib, stream, f32_mode=head_f32_mode, async_=False, status=True)
    prod_s = Product(lib, case, [d[1] for d in dev], ex_s)
    mains, devs = [], []
    for i in range(min(max(args.steps, 3), 20)):
        st = []
        prod_s(st)
        mains.append(lib.status_value(st[0], tapp_b200.STATUS_MAIN_US))
        devs.append(lib.status_value(st[0], tapp_b200.STATUS_DEVICE_US))
        lib.lib.TAPP_destroy_status(st[0])
    main_us = statistics.median(mains[1:] if len(mains) > 1 else mains)
    dev_us = statistics.median(devs[1:] if len(devs) > 1 else devs)
    peak, peak_kind = measured_peaks()
    achieved = FLOPS / (main_us * 1e-6) / 1e12
    traffic = profiled_traffic()
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} bf16 dense burst",
                "kernel": "tb::tc::k_gemm (split bfloat16)", "kernel_us": main_us, "step_device_us": dev_us,
                "flops_per_launch": FLOPS, "pipe_flops_per_launch": 3 * FLOPS,
                "pipe_frac": 3 * achieved / peak, "step_frac": FLOPS / (dev_us * 1e-6) / 1e12 / peak,
                "note": "achieved counts useful flops (2*M*N*K); the tensor pipe runs the three bfloat16 "
                        "products hi*hi + hi*lo + lo*hi, 3x that (pipe_frac)"}
    prod_s.close()
    lib.lib.TAPP_destroy_executor(ex_s)

    # ---------------- error of the headline and the other precision modes ----------------
    modes = {}
    ref64 = f64_slab_reference(lib, torch, case)
    D_head = dev[3][0].cpu().numpy().view(np.float32)
    head_err = float(np.abs(slab_values(case.D, D_head) - ref64).max() / np.abs(ref64).max())
    modes[HEADLINE] = {"tflops": value / world, "ms": t_ms, "max_abs_err_rel_to_max": head_err}
    if not args.no_modes:
        for name, (prec, storage, f32_mode, path) in MODES.items():
            if name == HEADLINE:
                continue
            mc = mode_case(name)
            mdev = [to_device(t, torch) for t in (mc.A, mc.B, mc.C, mc.D)]
            mex = make_executor(lib, stream, f32_mode=f32_mode, path=path)
            mp = Product(lib, mc, [d[1] for d in mdev], mex)
            steps = max(3, min(args.steps, 50)) if path == 3 else args.steps
            mt = time_device(torch, mp, steps, 3 if path == 3 else args.warmup, barrier)
            mref = ref64 if storage == 0 else f64_slab_reference(lib, torch, mc)
            Dm = mdev[3][0].cpu().numpy().view(np.float32)
            merr = np.abs(slab_values(mc.D, Dm) - mref)
            modes[name] = {"tflops": FLOPS / (mt * 1e-3) / 1e12, "ms": mt,
                           "max_abs_err_rel_to_max": float(merr.max() / np.abs(mref).max())}
            mp.close()
            lib.lib.TAPP_destroy_executor(mex)
            del mdev
    plain = modes.get("plain_f32", {}).get("tflops")
    if plain:
        modes["plain_f32"]["fp32_pipe_frac_of_nominal"] = plain / nominal_cuda_core_tflops(torch, 128)

    # ---------------- end to end through host buffers ----------------
    pinned = []
    for t in (case.A, case.B, case.C, case.D):
        h = torch.from_numpy(t.buf.view(np.uint8)).pin_memory()
        pinned.append((h, h.data_ptr() + t.base * t.itemsize))
    ex_h = make_executor(lib, None, f32_mode=head_f32_mode, async_=False)
    prod_h = Product(lib, case, [p[1] for p in pinned], ex_h)
    e2e_steps = max(3, min(args.steps, 20))
    for _ in range(2):
        prod_h()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        prod_h()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = replica_max(dist, e2e_s, "cuda")
    h2d = sum(t.buf.nbytes for t in (case.A, case.B, case.C))
    d2h = case.D.buf.nbytes
    e2e = {"value": replica_tflops(world, FLOPS, e2e_s), "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3,
           "how": "TAPP_execute_product on pinned host buffers, synchronous; wall clock per call"}
    prod_h.close()
    lib.lib.TAPP_destroy_executor(ex_h)

    small = small_configs_measure(lib, torch, with_cpu=(rank == 0 and not args.no_cpu)) \
        if world == 1 and not args.no_modes else None
    element = element_measure(lib, torch) if world == 1 and not args.no_modes else None

    served = None
    if world == 1 and args.served > 0:
        served = served_measure(lib, torch, args.served)
    batched = batched_measure(lib, torch) if world == 1 and not args.no_modes else None
    chain = chain_measure(lib, torch) if world == 1 and not args.no_modes else None
    tucker = tucker_measure(lib, torch) if world == 1 and not args.no_modes else None
    tiny = tiny_latency_measure(lib, torch) if world == 1 and not args.no_modes else None
    double = None
    if world == 1 and not args.no_double:
        double = double_measure(lib, torch, slices)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_run()
        cpu.pop("seconds", None)
        cpu.pop("flops", None)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "TFLOP/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "extents": EXTENT, "M": EXTENT ** 2, "N": EXTENT ** 2,
                           "K": EXTENT ** 2, "storage": "f32 A,B,C,D", "precision": "F32F32_ACCUM_F32",
                           "f32_mode": "split bfloat16 (TAPP_B200_ATTR_F32_MODE = 1)",
                           "parallelism": f"replicas x{world}",
                           "l2": "inputs 256 MiB > 126 MB L2 (A,B,C,D 64 MiB each)",
                           "step": STEP_DESCRIPTION},
                "max_abs_err_rel_to_max": head_err,
                "error_reference": "binary64 evaluation of D[:,:,:,0:2] from the same stored inputs",
                "vs_plain_gpu": (value / world / plain) if plain else None,
                "modes": modes, "small_configs": small, "element": element, "batched": batched, "tucker_chain": chain,
                "tucker": tucker, "tiny_latency": tiny, "double": double, "served": served, "roofline": roofline, "e2e": e2e,
                "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": gpu_launches}
        print(json.dumps(line), flush=True)
    prod.close()
    lib.lib.TAPP_destroy_executor(ex)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()

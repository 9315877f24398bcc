#!/usr/bin/env python
"""SpMV benchmark of the B200 engine (one JSON line on stdout, rank 0).

Default workload: FP64 SpMV in the K1 format (the engine's fastest FP64 format here; the
CSR and AXT formats and cuSPARSE are timed in the same run under "formats") on the
power-law matrix -- 4,194,304 rows, 67,108,864 nnz, lognormal(2.5, 1.2) row
lengths clipped to [1, 10000] and rescaled, columns uniform without replacement, values
N(0,1), x uniform[-1,1], seed 1.  A step is one SpMV of the whole matrix (one kernel
launch).  The value/column streams (805 MB) are larger than the 126 MB L2, so no L2 flush
is inserted between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--workload powerlaw|laplacian|stencil27|powerlaw-small]
                  [--variant axt-com-th1|axt-unc-th1-hw4|csr|k1|axc|...] [--sweep]

Under torchrun (N > 1) every rank owns an independent partition of the same size (its own
power-law block, seed 1 + rank: a block-diagonal operator, no exchange on the data path),
so per-GPU work is fixed ("weak" scaling); the time is the max over ranks.  Beside it the
line's "dist" object times the partitioned product of ONE shared matrix (DistSpMV:
nnz-balanced row blocks, x all-gathered over NCCL, each block in K1), µs per product as the
max over ranks ("strong" scaling).
``--impl reference`` times the reference's own CPU CSR SpMV (ncsr, cudaSpmv.cu:451,
compiled unchanged into oracle/_ref) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV GFLOP/s & HBM GB/s (% of 8 TB/s), FP64 vs mixed/batched/adjoint, 1 B200"

WORKLOADS = {
    "powerlaw": dict(desc="power-law 4194304 rows x 67108864 nnz, lognormal(2.5,1.2) "
                          "lengths clipped [1,10000], FP64, x U[-1,1]",
                     seed=1, xseed=1),
    "powerlaw-small": dict(desc="power-law 1048576 rows x 16777216 nnz (profiling case), "
                                "FP64", seed=1, xseed=1),
    "laplacian": dict(desc="2D 5-point Laplacian 512x512 (262144 rows, 1308672 nnz), FP64, "
                           "x U[-1,1]", seed=0, xseed=0),
    "stencil27": dict(desc="3D 27-point stencil 160^3 (4096000 rows, 109215352 nnz), FP64, "
                           "x N(0,1)", seed=2, xseed=2),
    "stencil27-small": dict(desc="3D 27-point stencil 100^3 (1000000 rows, 26463592 nnz, "
                                 "profiling case), x N(0,1)", seed=2, xseed=2),
}

VARIANTS = {
    "csr": dict(fmt="CSR"),
    "k1": dict(fmt="K1"),
    "axc": dict(fmt="AXC", hbs=32),
    "axt-com-th1": dict(fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=256),
    "axt-com-th2": dict(fmt="AXT", mode="COM", tileH=2, tileHW=32, bs=256),
    "axt-com-th4": dict(fmt="AXT", mode="COM", tileH=4, tileHW=32, bs=256),
    "axt-com-th8": dict(fmt="AXT", mode="COM", tileH=8, tileHW=32, bs=256),
    "axt-unc-th1-hw4": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=4),
    "axt-unc-th1-hw8": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=8),
    "axt-unc-th1-hw16": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=16),
    "axt-com-th16": dict(fmt="AXT", mode="COM", tileH=16, tileHW=32, bs=256),
    "axt-unc-th2": dict(fmt="AXT", mode="UNC", tileH=2, tileHW=32),
    "axt-unc-th4": dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32),
    "axt-unc-th8": dict(fmt="AXT", mode="UNC", tileH=8, tileHW=32),
    # the first generation's brick formats with x gathered at run time: AXCv0 = AXC with
    # half-bricks of 16, AXCv1 = AXT UNC tileH 1 tileHW 16, AXBv0 = AXT COM tileH 1 tileHW 16
    # with a header every 32 positions
    "axcv0": dict(fmt="AXC", hbs=16),
    "axcv1": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=16),
    "axbv0": dict(fmt="AXT", mode="COM", tileH=1, tileHW=16, bs=32),
    # kernel variants of the same layouts (comparison / tuning)
    "axt-com-th8-tma": dict(fmt="AXT", mode="COM", tileH=8, tileHW=32, bs=256, tma=True),
    "axt-unc-th4-tma": dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32, tma=True),
    "axt-com-th1-striped": dict(fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=256,
                                striped=True),
    # mixed precision: FP32 / BF16 values, 32-bit or 16-bit column offsets, FP32 x;
    # products and sums in FP32, or the sums in FP64 (acc64, FP64 y)
    "k1-f32": dict(fmt="K1", vtype="f32"),
    "k1-f32-u16": dict(fmt="K1", vtype="f32", itype="u16"),
    "k1-f32-u16-acc64": dict(fmt="K1", vtype="f32", itype="u16", acc64=True),
    "k1-bf16-u16": dict(fmt="K1", vtype="bf16", itype="u16"),
    "k1-bf16": dict(fmt="K1", vtype="bf16"),
    "csr-f32": dict(fmt="CSR", vtype="f32"),
    "csr-f32-u16": dict(fmt="CSR", vtype="f32", itype="u16"),
    "csr-f32-u16-acc64": dict(fmt="CSR", vtype="f32", itype="u16", acc64=True),
    "csr-bf16-u16": dict(fmt="CSR", vtype="bf16", itype="u16"),
    "axt-com-th1-f32-u16": dict(fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=256,
                                vtype="f32", itype="u16"),
    "axt-unc-th1-hw8-f32-u16": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=8, vtype="f32",
                                    itype="u16"),
    "axt-unc-th1-hw8-bf16-u16": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=8, vtype="bf16",
                                     itype="u16"),
}
RUN_KEYS = ("tma", "striped", "acc64")


def split_variant(vname: str):
    """(Matrix kwargs, spmv kwargs) of a variant."""
    kw = dict(VARIANTS[vname])
    run = {k: kw.pop(k) for k in RUN_KEYS if k in kw}
    return kw, run


def variant_bytes(n: int, nnz: int, kw: dict, run: dict) -> float:
    from gpu_spmv_b200 import engine as E

    vt = kw.get("vtype", "f64")
    s_v = {"f64": 8, "f32": 4, "bf16": 2}[vt]
    s_i = 2 if kw.get("itype") == "u16" else 4
    s_x = 8 if vt == "f64" else 4
    s_y = 8 if (vt == "f64" or run.get("acc64")) else 4
    return E.algorithmic_bytes(n, n, nnz, 1, s_v, s_i, s_x, s_y)
DEFAULT_VARIANT = "k1"
# formats timed beside the headline (µs per product), same matrix and x
COMPARE = ("csr", "axt-com-th1", "axt-com-th4", "axt-unc-th1-hw4", "axt-unc-th2", "axt-unc-th4",
           "axt-unc-th8", "axc", "axcv0", "axcv1", "axbv0")


def make_matrix(workload: str, rank: int, matgen=None):
    """The workload's CSR arrays and x.  `matgen` is the generator module: the engine's
    (gpu_spmv_b200.matgen) for this engine's arm, the same source built apart from the engine
    (oracle.workload) for the reference arm; both give the same bytes for a seed."""
    if matgen is None:
        from gpu_spmv_b200 import matgen

    w = WORKLOADS[workload]
    if workload == "powerlaw":
        row, col, val = matgen.powerlaw(seed=w["seed"] + rank)
        x = matgen.vector(len(row) - 1, "uniform", -1.0, 1.0, seed=w["xseed"] + 1000 + rank)
    elif workload == "powerlaw-small":
        row, col, val = matgen.powerlaw(nrows=1048576, nnz=16777216, seed=w["seed"] + rank)
        x = matgen.vector(len(row) - 1, "uniform", -1.0, 1.0, seed=w["xseed"] + 1000 + rank)
    elif workload == "laplacian":
        row, col, val = matgen.laplacian2d(512)
        x = matgen.vector(len(row) - 1, "uniform", -1.0, 1.0, seed=w["xseed"] + rank)
    elif workload in ("stencil27", "stencil27-small"):
        g = 160 if workload == "stencil27" else 100
        row, col, val = matgen.stencil27(g, seed=w["seed"] + rank)
        x = matgen.vector(len(row) - 1, "normal", seed=w["xseed"] + rank)
    else:
        raise KeyError(workload)
    return row, col, val, x


def loaded_repo_libraries() -> list:
    """Shared libraries of this repository mapped into this process (from /proc/self/maps)."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") and os.path.realpath(path).startswith(os.path.realpath(ROOT)):
                    out.add(os.path.relpath(os.path.realpath(path), os.path.realpath(ROOT)))
    except OSError:
        pass
    return sorted(out)


def workload_config(workload: str, n: int, nnz: int, world: int) -> dict:
    """The `config` object of the JSON line, the same for both arms on one workload."""
    return {"workload": WORKLOADS[workload]["desc"], "nrows": n, "nnz": nnz,
            "l2": "value/column streams > 126 MB L2 each step; no flush",
            "per_rank": ("independent partition of the same size (block-diagonal)"
                         if world > 1 else "one matrix")}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_lookup(key: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(p)).get(key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.lines: list[str] = []
        self.proc = None
        self.dev = device_index

    def start(self):
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            ident = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", ident], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [s.strip() for s in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_spmv(row, col, val, x, budget_s=15.0, threads=None):
    """The reference's ncsr (OpenMP) on the host cores; returns (GFLOP/s, sample text)."""
    from oracle.oracle import Ref

    R = Ref()
    threads = threads or os.cpu_count() or 1
    t0 = time.perf_counter()
    R.ncsr(row, col, val, x, threads=threads)  # warm-up (page-in)
    t1 = time.perf_counter()
    reps = max(1, min(50, int(budget_s / max(t1 - t0, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(reps):
        R.ncsr(row, col, val, x, threads=threads)
    dt = (time.perf_counter() - t0) / reps
    nnz = len(col)
    return 2.0 * nnz / dt / 1e9, f"{reps} full SpMVs of the workload ({nnz} nnz)", threads


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_details(row, col, val, x, block_rows: int = 1 << 18, reps: int = 5):
    """Single-core figures on a bounded sample (the first `block_rows` rows): the
    reference's ncsr on 1 thread and its serial cpuSpmvCSR (spmv_header.h), and the oracle's
    restatement of the CPU AXT loop (UNC tileH=1, tileHW=16, column stream); median of
    `reps` runs, GFLOP/s."""
    from oracle.oracle import Port, Ref

    R, P = Ref(), Port()
    r1 = min(block_rows, len(row) - 1)
    rr = np.ascontiguousarray(row[:r1 + 1])
    cc, vv = col[:int(rr[-1])], val[:int(rr[-1])]
    nnz = len(cc)

    def med(fn):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return 2.0 * nnz / statistics.median(ts) / 1e9

    a = P.axt(rr, cc, vv, 16, 1, "UNC")
    out = {"sample": f"first {r1} rows ({nnz} nnz), median of {reps}",
           "ncsr_1_thread": med(lambda: R.ncsr(rr, cc, vv, x, threads=1)),
           "axt_unc_th1_hw16_restated_1_thread": med(lambda: P.axt_spmv(a, x))}
    if R.lib_spmv is not None:
        out["cpuSpmvCSR_serial"] = med(lambda: R.cpu_spmv_csr(rr, cc, vv, x))
    return out


def error_vs_fp64(row, col, val, x, y) -> float:
    """max_i |y_i - y64_i| / (|A||x|)_i of a product y against an FP64 product computed
    outside this engine (torch's sparse CSR product, cuSPARSE, on the same device), with
    (|A||x|)_i from the same library on |A| and |x|."""
    import torch

    n = len(row) - 1
    dev = y.device
    crow = torch.from_numpy(row.astype(np.int64)).to(dev)
    cols = torch.from_numpy(col.astype(np.int64)).to(dev)
    v = torch.from_numpy(val).to(dev)
    dx = torch.from_numpy(x).to(dev)
    A = torch.sparse_csr_tensor(crow, cols, v, size=(n, len(x)))
    y64 = (A @ dx[:, None])[:, 0]
    Aa = torch.sparse_csr_tensor(crow, cols, v.abs(), size=(n, len(x)))
    mag = (Aa @ dx.abs()[:, None])[:, 0]
    r = (y.double() - y64).abs() / mag.clamp_min(1e-300)
    out = float(r.max())
    del A, Aa, crow, cols, v
    torch.cuda.empty_cache()
    return out


def _time_us(fn, steps: int, warm: int = 5) -> float:
    """Mean µs of fn() over `steps` calls, CUDA events around each call (current stream)."""
    import torch

    for _ in range(warm):
        fn()
    evs = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        evs.append((a, b))
    torch.cuda.synchronize()
    return 1e3 * sum(a.elapsed_time(b) for a, b in evs) / steps


def time_mixed(steps: int):
    """27-point stencil 160^3: FP64 K1 against reduced-precision K1 (µs per product, GFLOP/s,
    max_i |y - y64|_i / (|A||x|)_i)."""
    import torch

    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.stencil27(160, seed=2)
    n, nnz = len(row) - 1, len(col)
    x = matgen.vector(n, "normal", seed=2)
    out = {"workload": "27-point stencil 160^3 (4096000 rows, %d nnz), x N(0,1), seed 2" % nnz}
    dx64 = torch.from_numpy(x).cuda()
    for name, kw, acc in (("k1-f64", {}, False), ("k1-f32", dict(vtype="f32"), False),
                          ("k1-f32-u16", dict(vtype="f32", itype="u16"), False),
                          ("k1-f32-acc64", dict(vtype="f32"), True),
                          ("k1-bf16", dict(vtype="bf16"), False),
                          ("k1-bf16-u16", dict(vtype="bf16", itype="u16"), False)):
        A = E.Matrix(row, col, val, ncols=n, fmt="K1", **kw)
        dx = dx64 if not kw else dx64.float()
        y = torch.empty(n, dtype=torch.float64 if (not kw or acc) else torch.float32,
                        device="cuda")
        us = _time_us(lambda: A.spmv(dx, y, acc64=acc), steps)
        err = error_vs_fp64(row, col, val, x, y)
        out[name] = {"us": round(us, 2), "gflops": round(2.0 * nnz / us / 1e3, 1),
                     "error_vs_fp64": err}
        A.close()
    ok = [k for k, v in out.items() if isinstance(v, dict) and k != "k1-f64"
          and v["error_vs_fp64"] <= 1e-6]
    best = min(ok, key=lambda k: out[k]["us"])
    out["best_within_1e-6"] = best
    out["speedup_vs_f64"] = round(out["k1-f64"]["us"] / out[best]["us"], 3)
    return out


def time_adjoint(steps: int):
    """Differentiable product Y = A(v) X, FP32, 8 right-hand sides, on a power-law matrix of
    1,048,576 rows and 16,777,216 nnz (lognormal(2.5, 1.2) lengths, seed 4): forward,
    adjoint (Xbar and vbar) in both modes, and the (forward + adjoint) / forward ratio."""
    import torch

    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.powerlaw(nrows=1048576, nnz=16777216, seed=4)
    n, nnz, k = len(row) - 1, len(col), 8
    g = torch.Generator(device="cuda").manual_seed(4)
    A = E.Matrix(row, col, val, ncols=n, fmt="K1", vtype="f32", adjoint=True)
    X = torch.randn(n, k, device="cuda", generator=g)
    B = torch.randn(n, k, device="cuda", generator=g)
    Y = torch.empty(n, k, device="cuda")
    Xbar = torch.empty(n, k, device="cuda")
    vbar = torch.empty(nnz, device="cuda")
    Yb = A.spmm(X) - B
    from gpu_spmv_b200 import _lib as L

    lib, sh = L.lib(), E.stream_handle()

    def fwd():
        L.check(lib.gs_spmm(A._h, X.data_ptr(), Y.data_ptr(), L.GS_F32, k, sh), "spmm")

    vslots = torch.empty(A.value_slots(), device="cuda")

    def adj(mode, order, want_vbar=True):
        vb = vslots if order == L.GS_VALUES_SLOTS else vbar
        L.check(lib.gs_spmm_adjoint(A._h, Yb.data_ptr(), X.data_ptr(), Xbar.data_ptr(),
                                    vb.data_ptr() if want_vbar else None, L.GS_F32, k, mode,
                                    order, sh), "adjoint")

    vals = torch.from_numpy(val.astype(np.float32)).cuda()
    vals_slots = A.convert_values(vals, to="slots")
    f = _time_us(fwd, steps)
    ads = _time_us(lambda: adj(L.GS_ADJ_DETERMINISTIC, L.GS_VALUES_SLOTS), steps)
    adc = _time_us(lambda: adj(L.GS_ADJ_DETERMINISTIC, L.GS_VALUES_CSR), steps)
    aa = _time_us(lambda: adj(L.GS_ADJ_ATOMIC, L.GS_VALUES_CSR), steps)
    aas = _time_us(lambda: adj(L.GS_ADJ_ATOMIC, L.GS_VALUES_SLOTS), steps)
    ax_d = _time_us(lambda: adj(L.GS_ADJ_DETERMINISTIC, L.GS_VALUES_CSR, False), steps)
    ax_a = _time_us(lambda: adj(L.GS_ADJ_ATOMIC, L.GS_VALUES_CSR, False), steps)
    svs = _time_us(lambda: A.set_values(vals_slots, "slots"), steps)
    svc = _time_us(lambda: A.set_values(vals, "csr"), steps)
    A.close()
    return {"workload": "power-law 1048576 rows x %d nnz, FP32 values, 8 RHS, seed 4" % nnz,
            "forward_us": round(f, 2), "forward_gflops": round(2.0 * nnz * k / f / 1e3, 1),
            "adjoint_deterministic_slots_us": round(ads, 2),
            "adjoint_deterministic_csr_us": round(adc, 2),
            "adjoint_atomic_csr_us": round(aa, 2),
            "adjoint_atomic_slots_us": round(aas, 2),
            "xbar_only_deterministic_us": round(ax_d, 2),
            "xbar_only_atomic_us": round(ax_a, 2),
            "set_values_slots_us": round(svs, 2), "set_values_csr_us": round(svc, 2),
            "fwd_plus_adj_over_fwd": round((f + ads) / f, 3),
            "fwd_plus_adj_over_fwd_csr_order": round((f + adc) / f, 3),
            "fwd_plus_adj_over_fwd_atomic": round((f + aa) / f, 3),
            "fwd_plus_xbar_over_fwd_atomic": round((f + ax_a) / f, 3),
            "note": "adjoint = Xbar = A^T Ybar and vbar (value gradient) in one launch; "
                    "slots = values kept in the adjoint layout's order"}


def time_batched(steps: int, count: int = 256):
    """256 banded matrices (rows log-uniform in [1000, 200000], half-bandwidth U[16, 256],
    U[5, 60] entries per row in the band, FP32 values N(0,1)), each with U[1, 32]
    right-hand sides N(0,1), seed 3: one persistent launch replayed from a CUDA graph (row
    blocks with the X band in shared memory), block widths from the autotuner; beside it
    the same batch on K1 units.  The plain FP64 form is the same work as single-RHS FP64 K1
    products, one per matrix and right-hand side (device time per product x k_i)."""
    import torch

    from gpu_spmv_b200 import autotune
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    nm = count
    work = matgen.banded_batch(nm, seed=3)
    ks = [w[3] for w in work]
    mats, plain_us, nnz_tot, nrows_tot = [], 0.0, 0, 0
    for i, (row, col, val, _) in enumerate(work):
        n = len(row) - 1
        nrows_tot += n
        nnz_tot += len(col)
        mats.append(E.Matrix(row, col, val, ncols=n, fmt="K1", vtype="f32"))
        A64 = E.Matrix(row, col, val, ncols=n, fmt="K1")
        x = torch.randn(n, dtype=torch.float64, device="cuda")
        y = torch.empty(n, dtype=torch.float64, device="cuda")
        plain_us += ks[i] * _time_us(lambda: A64.spmv(x, y), 5, warm=2)
        A64.close()
    B = E.Batch(mats, ks)
    B.make_operands([matgen.batch_rhs(i, A.ncols, k, seed=3) for i, (A, k) in
                     enumerate(zip(mats, ks))])
    tune = autotune.tune(B, reps=5)
    tuned = tune["config"]
    us = _time_us(lambda: B.run(graph=True), steps, warm=3)
    paths = B.paths
    row_blocks = B.row_blocks
    # untuned: every matrix at its full width, the default path and 4096-row blocks
    autotune.apply_config(B, {"kb": list(B.kpad), "path": ["auto"] * nm, "rows": [4096] * nm})
    us_default = _time_us(lambda: B.run(graph=True), max(5, steps // 4), warm=2)
    autotune.apply_config(B, {"kb": tuned["kb"], "path": ["k1"] * nm, "rows": tuned["rows"]})
    us_k1 = _time_us(lambda: B.run(graph=True), max(5, steps // 4), warm=2)  # K1 units only
    autotune.apply_config(B, tuned)
    # error of every matrix's FP32 result against the FP64 product of the same FP32 values and
    # right-hand sides (torch's sparse CSR product, outside this engine), per row over
    # (|A||X|)_i: the largest over all matrices and columns
    B.run(graph=True)
    torch.cuda.synchronize()
    err = 0.0
    for (row, col, val, k), Y, X in zip(work, B.results(), B.X):
        n = len(row) - 1
        crow = torch.from_numpy(row.astype(np.int64)).cuda()
        cols = torch.from_numpy(col.astype(np.int64)).cuda()
        v = torch.from_numpy(val.astype(np.float32).astype(np.float64)).cuda()
        X64 = X[:, :k].double()
        y64 = torch.sparse_csr_tensor(crow, cols, v, size=(n, n)) @ X64
        mag = torch.sparse_csr_tensor(crow, cols, v.abs(), size=(n, n)) @ X64.abs()
        err = max(err, float(((Y.double() - y64).abs() / mag.clamp_min(1e-300)).max()))
    flops = B.flops
    out = {"workload": "%d banded FP32 matrices, %d rows, %d nnz, 1-32 RHS (sum %d), seed 3"
                       % (nm, nrows_tot, nnz_tot, sum(ks)),
           "us_per_run": round(us, 1), "gflops": round(flops / us / 1e3, 1),
           "us_per_run_untuned": round(us_default, 1),
           "work_items": B.nitems,
           "row_block_matrices": paths.count("band"),
           "us_per_run_k1_units": round(us_k1, 1),
           "plain_fp64_us": round(plain_us, 1),
           "plain_fp64_gflops": round(flops / plain_us / 1e3, 1),
           "speedup_vs_plain_fp64": round(plain_us / us, 2),
           "error_vs_fp64": err,
           "error_note": "max over all matrices, rows and columns of |Y - Y64| / (|A||X|)_i, "
                         "Y64 = torch sparse CSR FP64 product of the same FP32 numbers",
           "autotune": tune["choices"],
           "row_blocks": sum(b for _, b in row_blocks),
           "autotune_ms": {k: round(v, 3) for k, v in tune["timings"].items()}}
    B.close()
    for A in mats:
        A.close()
    return out


def time_dropin(workload: str, steps: int):
    """The drop-in API the way the reference's main() drives it (cudaSpmv.cu:2319-2417): per
    format, its getFormatData* converter (the reference's layouts, x baked into AXC / AXT as
    the reference does) and its test_* entry point, `steps` launches (gs_set_num_ite).  Each
    row: the converter's mfp / beta / conversion seconds and the product's mean device time,
    with the reference's error summary against the drop-in ncsr (on the GPU here)."""
    import ctypes as Cc

    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import refapi as R

    row, col, val, x = make_matrix(workload, 0)
    n = len(row) - 1
    lib = L.lib()
    lib.gs_set_num_ite(max(1, steps))
    h = R.csr_struct(row, col, val, name=workload + ".bin")
    y_ref = np.zeros(n)
    lib.ncsr(os.cpu_count() or 1, h.s, R.f64p(x), R.f64p(y_ref))
    out = {}

    def put(fd, res):
        out[res.name.decode()] = dict(
            format=fd.name.decode() if fd is not None else "fcsr", mfp=fd.mfp if fd else None,
            beta=fd.beta if fd else None, conversion_s=fd.ct if fd else None,
            us=round(res.et * 1e6, 2), gflops=round(res.flops / 1e9, 1),
            abs_err=res.sErr.aErr, rel_err=res.sErr.rErr)

    put(None, lib.test_gcsr(256, h.s, R.f64p(x), R.f64p(y_ref)))
    k = L.StrMatK1()
    fd = lib.getFormatDataK1(32, h.s, R.f64p(x), Cc.byref(k))
    put(fd, lib.test_gk1(256, k, R.f64p(x), R.f64p(y_ref)))
    R.free_struct_arrays(k, ("permi", "nmc", "chp", "val", "col"))
    a = L.StrMatAXC()
    fd = lib.getFormatDataAXC(os.cpu_count() or 1, 32, h.s, R.f64p(x), Cc.byref(a))
    put(fd, lib.test_gaxc(256, a, R.f64p(y_ref)))
    R.free_struct_arrays(a, ("ax", "brp", "mapx"))
    for mode, th, thw, fn in (("UNC", 1, 16, lambda t: lib.test_gaxtuh1hw16w(128, 256, t, R.f64p(y_ref))),
                              ("UNC", 1, 8, lambda t: lib.test_gaxtuh1hw08w(64, 256, t, R.f64p(y_ref))),
                              ("UNC", 1, 4, lambda t: lib.test_gaxtuh1hw04w(32, 256, t, R.f64p(y_ref))),
                              ("UNC", 4, 32, lambda t: lib.test_gaxtuh(4, 256, t, R.f64p(y_ref))),
                              ("UNC", 8, 32, lambda t: lib.test_gaxtuh(4, 256, t, R.f64p(y_ref))),
                              ("COM", 1, 32, lambda t: lib.test_gaxtch1(256, t, R.f64p(y_ref)))):
        t = L.StrMatAXT()
        fd = lib.getFormatDataAXT(os.cpu_count() or 1, 256, thw, th, mode.encode(), h.s,
                                  R.f64p(x), Cc.byref(t))
        put(fd, fn(t))
        R.free_struct_arrays(t, ("ax", "sec", "con"))
    lib.gs_set_num_ite(250)
    return {"workload": WORKLOADS[workload]["desc"], "launches_per_entry_point": steps,
            "entry_points": out}


PROBE_SO = os.path.join(ROOT, "gpu_spmv_b200", "lib", "libgs_bench_probe.so")
_probe = None


def probe_lib():
    """The benchmark's measurement helpers (gs_bench_probe.cu), not part of the engine."""
    global _probe
    if _probe is None:
        import ctypes as Cc

        lib = Cc.CDLL(PROBE_SO)
        lib.gsp_last_error.restype = Cc.c_char_p
        lib.gsp_gather_rate.restype = Cc.c_int
        lib.gsp_gather_rate.argtypes = [Cc.c_void_p, Cc.c_uint32, Cc.c_uint32,
                                        Cc.POINTER(Cc.c_double), Cc.c_void_p]
        lib.gsp_gather4_rate.restype = Cc.c_int
        lib.gsp_gather4_rate.argtypes = [Cc.c_void_p, Cc.c_uint32, Cc.c_uint32, Cc.c_uint32,
                                         Cc.c_uint32, Cc.c_uint32, Cc.POINTER(Cc.c_double),
                                         Cc.POINTER(Cc.c_uint32), Cc.c_void_p]
        _probe = lib
    return _probe


def gather_rate(dx, n) -> float:
    """Random 8-byte reads per second from dx[0..n) through the SM load path."""
    import ctypes as Cc

    rate = Cc.c_double()
    lib = probe_lib()
    if lib.gsp_gather_rate(dx.data_ptr(), n, 256, Cc.byref(rate), None):
        raise RuntimeError(f"gsp_gather_rate: {lib.gsp_last_error().decode()}")
    return rate.value


def gather4_rates(dx, n, per_lane: int = 256):
    """Random reads per second from dx when issued as TMA tile::gather4 loads (four 16-byte
    rows per instruction into shared memory), alone and beside load-path gathers in the same
    blocks: {config: reads/s}.  Raises if a bounded wait gave up."""
    import ctypes as Cc

    lib = probe_lib()
    out = {}
    n2 = n & ~1
    # (warps per block, of which load-path warps, blocks per SM): 16 KB of stages per
    # gather4 warp, so at most 12 gather4 warps per SM
    for warps, lsu, bps in ((4, 0, 3), (8, 0, 1), (4, 0, 2), (4, 2, 3), (8, 4, 1), (8, 4, 2),
                            (8, 8, 2)):
        rate, to = Cc.c_double(), Cc.c_uint32()
        if lib.gsp_gather4_rate(dx.data_ptr(), n2, per_lane, warps, lsu, bps, Cc.byref(rate),
                                Cc.byref(to), None):
            raise RuntimeError(f"gsp_gather4_rate: {lib.gsp_last_error().decode()}")
        if to.value:
            raise RuntimeError("gsp_gather4_rate: " + ("a destination was not 128-byte aligned"
                                                       if to.value & 2 else
                                                       "a bounded wait gave up"))
        out[f"{bps}x{warps}warps_{lsu}lsu"] = rate.value
    return out


def time_gathers(workload: str):
    """Random-read rates from the workload's x (n doubles): the load path alone, and TMA
    tile::gather4 loads alone and beside load-path gathers in the same blocks."""
    import torch

    from gpu_spmv_b200 import matgen

    n = {"powerlaw": 4194304, "powerlaw-small": 1048576, "stencil27": 4096000}.get(workload,
                                                                                    4194304)
    dx = torch.from_numpy(matgen.vector(n, "uniform", -1.0, 1.0, seed=1001)).cuda()
    out = {"n": n, "bytes": 8 * n, "load_path_reads_per_s": gather_rate(dx, n)}
    out["tma_gather4_reads_per_s"] = gather4_rates(dx, n)
    return out


def gather_ceiling(A, n, nnz, kw, dx, kern_ms, rate_per_s=None):
    """The product's line requests per launch against this GPU's measured rate of random
    8-byte reads from x (gsp_gather_rate on the workload's own x, or `rate_per_s` when it was
    measured already): one request per x gather (nnz), the value and column streams (slots x
    bytes / 128), and y (one request per row when K1 scatters it by its permutation, else
    streamed).  frac = ceiling time / kernel time."""
    import ctypes as Cc

    rate = Cc.c_double(rate_per_s if rate_per_s else gather_rate(dx, n))
    slots = nnz / A.info.beta if A.info.beta > 0 else nnz
    sv = {"f64": 8, "f32": 4, "bf16": 2}[kw.get("vtype", "f64")]
    si = 2 if kw.get("itype") == "u16" else 4
    k1 = kw.get("fmt") == "K1"
    lines = nnz + slots * (sv + si) / 128.0 + (n if k1 else n * 8 / 128.0)
    ceiling_us = lines / rate.value * 1e6
    return {"reads_per_s_measured": rate.value, "line_requests_per_launch": lines,
            "ceiling_us": ceiling_us, "frac": ceiling_us / (kern_ms * 1e3),
            "note": "random 8-byte reads from x through the SM load path: the bound of an SpMV "
                    "whose columns are uniformly random"}


def pcie_bandwidth(hx, hy, dx, dy, reps: int = 10):
    """GB/s of pinned host -> device and device -> host copies of these buffers, alone and
    both at once (two streams), timed on the host around synchronised batches of copies."""
    import torch

    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def run(h2d, d2h):
        for _ in range(2):
            with torch.cuda.stream(s1):
                if h2d:
                    dx.copy_(hx, non_blocking=True)
            with torch.cuda.stream(s2):
                if d2h:
                    hy.copy_(dy, non_blocking=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            with torch.cuda.stream(s1):
                if h2d:
                    dx.copy_(hx, non_blocking=True)
            with torch.cuda.stream(s2):
                if d2h:
                    hy.copy_(dy, non_blocking=True)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    bx, by = hx.numel() * hx.element_size(), hy.numel() * hy.element_size()
    t_in, t_out, t_both = run(True, False), run(False, True), run(True, True)
    return {"h2d_gbs": round(bx / t_in / 1e9, 1), "d2h_gbs": round(by / t_out / 1e9, 1),
            "h2d_gbs_concurrent": round(bx / t_both / 1e9, 1),
            "d2h_gbs_concurrent": round(by / t_both / 1e9, 1)}


def time_formats(row, col, val, x, steps: int):
    """µs per product of the other formats and of cuSPARSE CSR on the same matrix and x
    (per-launch CUDA events, mean over `steps` launches after warm-up), and each format's
    max_i |y - y64|_i / (|A||x|)_i against torch's FP64 sparse CSR product."""
    import torch

    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import refapi as R

    n = len(row) - 1
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    out, errs, fracs = {}, {}, {}
    rate = gather_rate(dx, n)
    for vname in COMPARE:
        kw = dict(VARIANTS[vname])
        A = E.Matrix(row, col, val, ncols=n, **kw)
        for _ in range(5):
            A.spmv(dx, dy)
        ts = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            A.spmv(dx, dy)
            b.record()
            ts.append((a, b))
        torch.cuda.synchronize()
        out[vname] = round(1e3 * sum(a.elapsed_time(b) for a, b in ts) / steps, 2)
        if kw.get("vtype", "f64") == "f64":
            fracs[vname] = round(gather_ceiling(A, n, len(col), kw, dx, out[vname] * 1e-3,
                                                rate)["frac"], 3)
        A.close()
        errs[vname] = error_vs_fp64(row, col, val, x, dy)
    # cuSPARSE generic CSR SpMV through the drop-in test_gcucsr (per-launch events)
    h = R.csr_struct(row, col, val)
    ref = dy.cpu().numpy()
    old = L.lib().gs_get_num_ite()
    L.lib().gs_set_num_ite(max(20, steps // 2))
    try:
        L.lib().test_gcucsr(h.s, R.f64p(x), R.f64p(ref))  # warm-up: the library's first call
        r = L.lib().test_gcucsr(h.s, R.f64p(x), R.f64p(ref))
        out["cusparse-csr"] = round(r.et * 1e6, 2) if r.name == b"gcucsr" else None
    finally:
        L.lib().gs_set_num_ite(old)
    out["error_vs_fp64"] = errs
    out["gather_ceiling_frac"] = fracs
    return out


def time_dist(row, col, val, x, steps: int, warmup: int, device, local_factory=None,
              group=None):
    """The distributed product of ONE matrix shared by every rank
    (gpu_spmv_b200.distributed.DistSpMV: nnz-balanced row blocks, x all-gathered over the
    process group, each rank's block multiplied on its own device): µs per product, the max
    over ranks, timed with CUDA events on CUDA devices (the wall clock on CPU ranks).  Before
    any timed collective every rank reports whether it built its block (one all-reduce), so
    that no rank enters the timed all-gathers alone; on a failure every rank returns
    {"error": ...}.  `row` None stands for a matrix this rank could not build."""
    import torch
    import torch.distributed as dist

    from gpu_spmv_b200.distributed import DistSpMV

    err, D, xl = None, None, None
    try:
        if row is None:
            raise RuntimeError("no matrix")
        D = DistSpMV(row, col, val, len(row) - 1, group=group, device=device,
                     local_factory=local_factory)
        xl = torch.from_numpy(np.ascontiguousarray(x[D.r0:D.r1])).to(device)
    except Exception as e:
        err = f"{type(e).__name__}: {e}"
    flag = torch.tensor([0 if err else 1], dtype=torch.int32, device=device)
    dist.all_reduce(flag, op=dist.ReduceOp.MIN, group=group)
    if int(flag.item()) == 0:
        return {"error": err or "another rank could not build its row block"}
    cuda = torch.device(device).type == "cuda"
    for _ in range(warmup):
        D.spmv(xl)
    if cuda:
        torch.cuda.synchronize()
    dist.barrier(group=group)
    if cuda:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            D.spmv(xl)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    else:
        t0 = time.perf_counter()
        for _ in range(steps):
            D.spmv(xl)
        ms = (time.perf_counter() - t0) * 1e3
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    us = float(t.item()) * 1e3 / steps
    nnz = len(col)
    row64 = np.asarray(row, dtype=np.int64)
    return {"us_per_product": round(us, 2), "gflops": round(2.0 * nnz / (us * 1e-6) / 1e9, 1),
            "ranks": D.world, "rows_per_rank": D.sizes,
            "nnz_per_rank": [int(row64[D.bounds[k + 1]] - row64[D.bounds[k]])
                             for k in range(D.world)],
            "allgather_bytes_per_product": D.pad * D.world * xl.element_size(),
            "local_format": "K1", "scaling": "strong", "steps": steps, "warmup": warmup}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        from oracle.oracle import Ref

        if not Ref.available():
            raise FileNotFoundError("oracle/_ref not built")
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build missing: {e}"}))
        return 0
    from oracle import workload as oracle_workload

    row, col, val, x = make_matrix(args.workload, 0, oracle_workload)
    from oracle.oracle import Ref

    R = Ref()
    threads = os.cpu_count() or 1
    n, nnz = len(row) - 1, len(col)
    # each step is a bounded sample: a rotating block of rows sized so that the whole run
    # stays within ~2 minutes
    t0 = time.perf_counter()
    R.ncsr(row, col, val, x, threads=threads)
    t_full = time.perf_counter() - t0
    total_steps = args.steps + args.warmup
    frac = min(1.0, 120.0 / max(total_steps * t_full, 1e-9))
    nb = max(1, int(round(1.0 / frac)))
    blocks = np.linspace(0, n, nb + 1).astype(np.int64)
    subs = []
    for b in range(nb):
        r0, r1 = blocks[b], blocks[b + 1]
        rr = (row[r0:r1 + 1] - row[r0]).astype(np.uint32)
        subs.append((rr, col[row[r0]:row[r1]], val[row[r0]:row[r1]]))
    for s in range(args.warmup):
        rr, cc, vv = subs[s % nb]
        R.ncsr(rr, cc, vv, x, threads=threads)
    done_nnz, t = 0, 0.0
    for s in range(args.steps):
        rr, cc, vv = subs[s % nb]
        t0 = time.perf_counter()
        R.ncsr(rr, cc, vv, x, threads=threads)
        t += time.perf_counter() - t0
        done_nnz += len(cc)
    value = 2.0 * done_nnz / t / 1e9
    sample = (f"each step: one of {nb} row blocks (~{nnz // nb} nnz) of the workload, "
              f"full SpMV takes {t_full:.3f} s on {threads} threads")
    line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(args.workload, n, nnz, args.gpus),
            "path": {"impl": "reference ncsr (cudaSpmv.cu:451-466, OpenMP, compiled "
                             "unchanged into oracle/_ref)", "threads": threads,
                     "inputs": "oracle/_build/libgs_workload.so (the benchmark generator "
                               "built apart from the engine)"},
            "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "loaded_libraries": loaded_repo_libraries()}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch

    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import engine as E

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    row, col, val, x = make_matrix(args.workload, rank)
    n, nnz = len(row) - 1, len(col)
    variants = list(VARIANTS) if args.sweep else [args.variant]
    results = {}
    for vname in variants:
        kw, run = split_variant(vname)
        try:
            A = E.Matrix(row, col, val, ncols=n, **kw)
        except L.GSError as e:
            if not args.sweep or e.status != L.GS_ERR_UNSUPPORTED:
                raise
            print(f"[sweep] {vname:18s} skipped: {e}", file=sys.stderr, flush=True)
            continue
        f64 = kw.get("vtype", "f64") == "f64"
        dx = torch.from_numpy(x).cuda()
        if not f64:
            dx = dx.float()
        dy = torch.empty(n, dtype=torch.float64 if (f64 or run.get("acc64")) else torch.float32,
                         device="cuda")
        stream = torch.cuda.current_stream()
        for _ in range(args.warmup):
            A.spmv(dx, dy, **run)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        K = args.steps
        sampler = ClockSampler(local) if (rank == 0 and not args.sweep and not args.no_clocks) else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eb = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        ea = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        torch.cuda.synchronize()
        ev0.record(stream)
        for k in range(K):
            eb[k].record(stream)
            A.spmv(dx, dy, **run)
            ea[k].record(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        if sampler:
            sampler.stop()
        if A.device_status():
            raise RuntimeError(f"{vname}: a kernel reported a timed-out wait")
        elapsed = ev0.elapsed_time(ev1)  # ms
        kern = sum(b.elapsed_time(a) for b, a in zip(eb, ea)) / K
        if dist:
            t = torch.tensor([elapsed, kern], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            elapsed, kern = float(t[0]), float(t[1])
        results[vname] = (A, elapsed, kern, sampler, dx, dy, run)
        if args.sweep and rank == 0:
            gf = 2.0 * nnz * K / (elapsed * 1e-3) / 1e9
            B = variant_bytes(n, nnz, kw, run)
            err = error_vs_fp64(row, col, val, x, dy)
            print(f"[sweep] {vname:18s} {elapsed / K * 1e3:9.1f} us/step  {gf:8.1f} GFLOP/s  "
                  f"{B / (kern * 1e-3) / 1e9:8.1f} GB/s alg  beta={A.info.beta:.3f} "
                  f"conv={A.info.conv_ms:.1f} ms  err={err:.2e}", file=sys.stderr, flush=True)
        if args.sweep:
            A.close()
    if args.sweep:
        return 0
    A, elapsed, kern, sampler, dx, dy, run = results[args.variant]
    kw, _ = split_variant(args.variant)
    spmv_flags = ((L.GS_FLAG_TMA if run.get("tma") else 0) |
                  (L.GS_FLAG_STRIPED if run.get("striped") else 0) |
                  (L.GS_FLAG_ACC_F64 if run.get("acc64") else 0))
    K = args.steps
    nnz_all = float(nnz)  # stored elements of all ranks' blocks (each rank its own seed)
    if dist:
        t = torch.tensor([nnz_all], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        nnz_all = float(t[0])
    value = 2.0 * nnz_all * K / (elapsed * 1e-3) / 1e9
    B = variant_bytes(n, nnz, kw, run)
    peak, peak_kind = measured_peak()
    achieved = B / (kern * 1e-3) / 1e9
    tkey = f"{args.workload}/{args.variant}"
    traffic = traffic_lookup(tkey)
    gather = gather_ceiling(A, n, nnz, kw, dx, kern) if dx.dtype == torch.float64 else None

    # ---- end to end through the C ABI with host buffers: H2D x, SpMV, D2H y per step
    e2e = None
    if not args.no_e2e:
        hx = torch.from_numpy(x).to(dx.dtype).pin_memory()
        hy = torch.empty(n, dtype=dy.dtype).pin_memory()
        xcode = L.GS_F64 if dx.dtype == torch.float64 else L.GS_F32
        ycode = L.GS_F64 if dy.dtype == torch.float64 else L.GS_F32
        Ke = min(K, args.e2e_steps)
        lib = L.lib()
        sh = E.stream_handle()
        for _ in range(3):
            L.check(lib.gs_spmv_host(A._h, hx.data_ptr(), dx.data_ptr(), xcode,
                                     hy.data_ptr(), dy.data_ptr(), ycode, spmv_flags, sh), "e2e")
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(Ke):
            L.check(lib.gs_spmv_host(A._h, hx.data_ptr(), dx.data_ptr(), xcode,
                                     hy.data_ptr(), dy.data_ptr(), ycode, spmv_flags, sh), "e2e")
        te_serial = time.perf_counter() - t0
        # streamed: the same per-step copies, consecutive steps overlapped (3 streams)
        L.check(lib.gs_spmv_host_stream(A._h, hx.data_ptr(), 0, xcode, hy.data_ptr(), 0, ycode,
                                        3, spmv_flags, sh), "e2e stream")
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(lib.gs_spmv_host_stream(A._h, hx.data_ptr(), 0, xcode, hy.data_ptr(), 0, ycode,
                                        Ke, spmv_flags, sh), "e2e stream")
        te = time.perf_counter() - t0
        if dist:
            t = torch.tensor([te, te_serial], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te, te_serial = float(t[0]), float(t[1])
        # the link's ceiling for these copies: pinned host <-> device, both directions at
        # once on two streams, as the streamed steps run them
        pcie = pcie_bandwidth(hx, hy, dx, dy)
        step_s = max(hx.element_size() * n / (pcie["h2d_gbs_concurrent"] * 1e9),
                     hy.element_size() * n / (pcie["d2h_gbs_concurrent"] * 1e9))
        ceiling = 2.0 * nnz_all / step_s / 1e9
        e2e = {"value": 2.0 * nnz_all * Ke / te / 1e9, "unit": "GFLOP/s",
               "pcie": pcie, "pcie_ceiling": round(ceiling, 1),
               "frac_of_pcie_ceiling": round(2.0 * nnz_all * Ke / te / 1e9 / ceiling, 3),
               "h2d_bytes_per_step": hx.element_size() * n,
               "d2h_bytes_per_step": hy.element_size() * n, "steps": Ke,
               "path": "gs_spmv_host_stream (C ABI): per step, pinned host x -> device, "
                       "SpMV, y -> host; consecutive steps overlap on three streams",
               "serial_value": 2.0 * nnz_all * Ke / te_serial / 1e9,
               "serial_path": "gs_spmv_host, one synchronous call per step"}

    formats = None
    if rank == 0 and world == 1 and not args.no_formats:
        formats = {"unit": "us per product", "headline": args.variant,
                   args.variant: round(1e3 * kern, 2)}
        formats.update(time_formats(row, col, val, x, args.format_steps))

    mixed = adjoint = batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = time_batched(max(10, args.format_steps // 4))
    if rank == 0 and world == 1 and not args.no_mixed:
        mixed = time_mixed(args.format_steps)
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = time_adjoint(args.format_steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, sample, threads = cpu_reference_spmv(row, col, val, x)
            cpu = {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "reference",
                   "sample": sample + "; reference ncsr compiled unchanged (oracle/_ref)",
                   "cpu_model": cpu_model(), "one_core": cpu_details(row, col, val, x)}
        except Exception as e:  # the checker library is absent: report it
            cpu = {"value": None, "unit": "GFLOP/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    # the partitioned product of one shared matrix (x all-gather over NCCL), beside the
    # independent per-rank blocks of the headline
    dres = None
    if dist and not args.no_dist:
        try:
            drow, dcol, dval, dxv = make_matrix(args.workload, 0)
        except Exception:
            drow = dcol = dval = dxv = None
        dres = time_dist(drow, dcol, dval, dxv, K, args.warmup, torch.device("cuda", local))
        if drow is not None:
            dres["workload"] = (f"{WORKLOADS[args.workload]['desc']}, seed "
                                f"{WORKLOADS[args.workload]['seed']}, one matrix shared by "
                                f"the {world} ranks")
        del drow, dcol, dval, dxv

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    clocks = sampler.summary() if sampler else None
    info = A.info
    line = {
        "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": elapsed / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": kw.get("vtype", "f64"),
        "data": "synthetic",
        "config": workload_config(args.workload, n, nnz, world),
        "path": {"format": args.variant, "beta": info.beta,
                 "error_vs_fp64": error_vs_fp64(row, col, val, x, dy)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "frac_of_8TBs": achieved / 8000.0, "traffic": traffic,
                     "algorithmic_bytes_per_launch": B, "kernel_ms": kern,
                     "gather_ceiling": gather},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "formats": formats,
        "mixed": mixed,
        "adjoint": adjoint,
        "batched": batched,
        "dist": dres,
        "gpu_launches": K,
        "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="powerlaw", choices=list(WORKLOADS))
    ap.add_argument("--variant", default=DEFAULT_VARIANT, choices=list(VARIANTS))
    ap.add_argument("--sweep", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-dist", action="store_true",
                    help="under torchrun: skip the partitioned product of one shared matrix")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-formats", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--only", choices=["mixed", "adjoint", "batched", "batched-small", "dropin",
                                       "gathers"],
                    help="run one section alone and print its object (dropin: the reference's "
                         "converters and test_* entry points, through this library, on --workload)")
    ap.add_argument("--format-steps", type=int, default=200)
    ap.add_argument("--no-clocks", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.only:
        # one section alone (profiling): its JSON object, `--steps` timed launches
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        fn = {"mixed": lambda: time_mixed(args.steps),
              "adjoint": lambda: time_adjoint(args.steps),
              "batched": lambda: time_batched(args.steps),
              "batched-small": lambda: time_batched(args.steps, count=32),
              "dropin": lambda: time_dropin(args.workload, args.steps),
              "gathers": lambda: time_gathers(args.workload)}[args.only]
        print(json.dumps({args.only: fn()}))
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

"""Autotuners: the layout of a single matrix (choose_format), and each matrix's
right-hand-side block width in a batched multi-RHS product (tune).

A matrix with kpad right-hand sides runs as kpad/kb passes of kb columns.  Wide blocks
gather each stored element's x row once for all columns; narrow ones re-read the value and
column streams per pass but need fewer registers.  The batch kernel is instantiated for its
widest block, so one wide matrix sets the register budget, and hence the occupancy, of the
whole launch.  The tuner therefore times whole-batch runs (CUDA events, median of `reps`
after warm-up):

  1. a global cap C in (32, 16, 8, 4): kb_i = min(kpad_i, C);
  2. one pass over the groups of matrices with the same (kpad, row-length class), trying
     half the group's width and keeping it when the batch gets faster by more than 1 %.

The choice is stored per group key "<dtype>/kpad<k>/len<class>" in an optional JSON cache,
which later batches apply without timing.
"""
from __future__ import annotations

import json
import os
import statistics

import torch

from . import engine as E


def _len_class(A) -> int:
    avg = A.nnz / max(1, A.nrows)
    return 0 if avg < 16 else (1 if avg < 48 else 2)


def _time_batch(B: E.Batch, reps: int) -> float:
    for _ in range(2):
        B.run(graph=False)
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        B.run(graph=False)
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def tune(batch: E.Batch, reps: int = 5, cache_path: str | None = None) -> dict:
    """Choose and apply a block width per matrix of `batch` (operands must be set).
    Returns {"choices": {group key: kb}, "timings": {candidate: ms}}."""
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    dt = "f64" if batch.dtype == torch.float64 else "f32"
    keys = [f"{dt}/kpad{kp}/len{_len_class(A)}" for A, kp in zip(batch.mats, batch.kpad)]
    groups: dict[str, list[int]] = {}
    for i, key in enumerate(keys):
        groups.setdefault(key, []).append(i)
    if all(k in cache for k in groups):
        choices = {k: int(cache[k]) for k in groups}
        batch.set_blocking([choices[k] for k in keys])
        return {"choices": choices, "timings": {}}

    timings = {}
    best_kb, best_t = None, float("inf")
    for cap in (32, 16, 8, 4):
        kb = [min(kp, cap) for kp in batch.kpad]
        if kb == best_kb:
            continue
        batch.set_blocking(kb)
        t = _time_batch(batch, reps)
        timings[f"cap{cap}"] = t
        if t < best_t:
            best_kb, best_t = kb, t
    kb = list(best_kb)
    for key, idx in groups.items():
        w = kb[idx[0]]
        if w == 1 or w * 8 < batch.kpad[idx[0]] * 2:
            continue
        trial = list(kb)
        for i in idx:
            trial[i] = w // 2
        batch.set_blocking(trial)
        t = _time_batch(batch, reps)
        timings[f"{key}:kb{w // 2}"] = t
        if t < 0.99 * best_t:
            kb, best_t = trial, t
    batch.set_blocking(kb)
    choices = {key: kb[idx[0]] for key, idx in groups.items()}
    if cache_path:
        cache.update(choices)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return {"choices": choices, "timings": timings}


# ----------------------------------------------------------------------------- formats
# Candidate layouts for one matrix (the reference sweeps these by hand: its job scripts run
# every format and tile parameter and compare the timings).
FORMAT_CANDIDATES = {
    "k1": dict(fmt="K1"),
    "csr": dict(fmt="CSR"),
    "axt-unc-th4": dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32),
    "axt-unc-th8": dict(fmt="AXT", mode="UNC", tileH=8, tileHW=32),
    "axt-unc-th1-hw4": dict(fmt="AXT", mode="UNC", tileH=1, tileHW=4),
    "axt-com-th1": dict(fmt="AXT", mode="COM", tileH=1, tileHW=32),
}


def matrix_key(row, vtype: str = "f64") -> str:
    """Shape class of a CSR matrix: dtype, log2 rows, log2 nnz, row-length spread."""
    import numpy as np

    row = np.asarray(row, dtype=np.int64)
    n = len(row) - 1
    nnz = int(row[-1])
    lens = np.diff(row)
    cv = float(lens.std() / max(lens.mean(), 1e-9)) if n else 0.0
    spread = 0 if cv < 0.25 else (1 if cv < 1.0 else 2)
    return f"{vtype}/n2^{max(n, 1).bit_length()}/nnz2^{max(nnz, 1).bit_length()}/cv{spread}"


def choose_format(row, col, val, ncols=None, vtype: str = "f64", candidates=None,
                  reps: int = 20, cache_path: str | None = None, device="cuda"):
    """Convert the matrix into each candidate layout, time its product (CUDA events,
    median of `reps` after warm-up) and return (best Matrix, {name: µs}); the others are
    released.  With a cache holding this matrix's key, only the cached choice is built."""
    from . import _lib as L
    from . import engine as E

    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    key = matrix_key(row, vtype)
    names = list(candidates or FORMAT_CANDIDATES)
    if key in cache and cache[key] in FORMAT_CANDIDATES:
        names = [cache[key]]
    n = len(row) - 1
    nc = ncols if ncols is not None else n
    dt = torch.float64 if vtype == "f64" else torch.float32
    x = torch.rand(nc, dtype=dt, device=device)
    best, best_t, timings = None, float("inf"), {}
    for name in names:
        kw = dict(FORMAT_CANDIDATES[name])
        try:
            A = E.Matrix(row, col, val, ncols=nc, vtype=vtype, device=device, **kw)
        except L.GSError as e:  # a layout this matrix or value type cannot take
            if e.status != L.GS_ERR_UNSUPPORTED:
                raise
            continue
        y = A.spmv(x)
        for _ in range(3):
            A.spmv(x, y)
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            A.spmv(x, y)
            b.record()
            ts.append((a, b))
        torch.cuda.synchronize()
        t = statistics.median(a.elapsed_time(b) for a, b in ts) * 1e3
        timings[name] = t
        if t < best_t:
            if best is not None:
                best.close()
            best, best_t = A, t
            best.autotuned_format = name
        else:
            A.close()
    if best is None:
        raise RuntimeError("no candidate layout accepted the matrix")
    if cache_path and len(names) > 1:
        cache[key] = best.autotuned_format
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return best, timings

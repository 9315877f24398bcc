"""Autotuners: the layout of a single matrix (choose_format), and the launch shape of each
matrix in a batched multi-RHS product (tune).

A batched matrix has three knobs, the batched counterparts of the reference's sweep over
tileHeight, threads (warps) per row and block size (cudaSpmv.cu:2349-2417):

  * the right-hand-side block width kb: kpad/kb passes of kb columns.  Wide blocks gather
    each stored element's X row once for all columns; narrow ones re-read the value and
    column streams per pass but need fewer registers.  On row blocks kb also sets the lanes
    per row (16 bytes of the row's kb values per lane: 8 lanes at kb = 32 in FP32);
  * the path: K1 units (a warp per 32-row unit, X gathered through L1 / L2) or row blocks
    (a thread block per block of rows, X band staged in shared memory);
  * the row-block height (rows per block, 32..4096): smaller blocks make more, smaller work
    items for the persistent kernel to balance.

The batch kernels are instantiated for the widest block, so one wide matrix sets the
register budget, and hence the occupancy, of the whole launch.  The tuner therefore times
whole-batch runs (CUDA events, median of `reps` after warm-up):

  1. a global cap C in (32, 16, 8, 4): kb_i = min(kpad_i, C);
  2. one pass over the groups of matrices with the same (kpad, row-length class, size
     class), trying for each group half its width, the other path, and row-block heights
     of 1024 and 256, keeping a change when the batch gets faster by more than 1 %.

The choices are stored per group key "<dtype>/kpad<k>/len<class>/n<class>" in an optional
JSON cache, which later batches apply without timing.  None of the knobs changes the sums or
their order: every choice gives the same bits.
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


def _size_class(A) -> int:
    return 0 if A.nrows < 20000 else (1 if A.nrows < 100000 else 2)


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


class _Config:
    """kb, requested path and row-block height of every matrix of a batch."""

    def __init__(self, kb, path, rows):
        self.kb, self.path, self.rows = list(kb), list(path), list(rows)

    def copy(self):
        return _Config(self.kb, self.path, self.rows)

    def apply(self, batch: E.Batch) -> bool:
        """Set it on the batch; False (batch unchanged) when a matrix cannot take it."""
        from . import _lib as L

        try:
            batch.set_row_blocks(self.rows)
            batch.set_paths(self.path)
            batch.set_blocking(self.kb)
        except L.GSError as e:
            if e.status != L.GS_ERR_UNSUPPORTED:
                raise
            return False
        return True


def tune(batch: E.Batch, reps: int = 5, cache_path: str | None = None) -> dict:
    """Choose and apply each matrix's right-hand-side block width, path and row-block height
    (operands must be set).  Returns {"choices": {group key: {"kb", "path", "rows"}},
    "timings": {candidate: ms}, "untuned_ms", "tuned_ms"}."""
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    dt = "f64" if batch.dtype == torch.float64 else "f32"
    keys = [f"{dt}/kpad{kp}/len{_len_class(A)}/n{_size_class(A)}"
            for A, kp in zip(batch.mats, batch.kpad)]
    groups: dict[str, list[int]] = {}
    for i, key in enumerate(keys):
        groups.setdefault(key, []).append(i)
    n = len(batch.mats)
    if all(isinstance(cache.get(k), dict) for k in groups):
        cfg = _Config([cache[k]["kb"] for k in keys], [cache[k]["path"] for k in keys],
                      [cache[k]["rows"] for k in keys])
        if cfg.apply(batch):
            return {"choices": {k: cache[k] for k in groups}, "timings": {},
                    "config": {"kb": cfg.kb, "path": cfg.path, "rows": cfg.rows}}

    timings = {}
    base = _Config(batch.kpad, ["auto"] * n, [4096] * n)
    base.apply(batch)
    untuned = _time_batch(batch, reps)
    timings["untuned"] = untuned
    best, best_t = base, untuned
    for cap in (16, 8, 4):
        cfg = best.copy()
        cfg.kb = [min(kp, cap) for kp in batch.kpad]
        if cfg.kb == best.kb or not cfg.apply(batch):
            continue
        t = _time_batch(batch, reps)
        timings[f"cap{cap}"] = t
        if t < 0.99 * best_t:
            best, best_t = cfg, t
    for key, idx in groups.items():
        trials = []
        w = best.kb[idx[0]]
        if w > 1:
            trials.append(("kb%d" % (w // 2), "kb", w // 2))
        trials.append(("k1" if best.path[idx[0]] != "k1" else "band", "path",
                       "k1" if best.path[idx[0]] != "k1" else "auto"))
        for rows in (1024, 256):
            trials.append(("rows%d" % rows, "rows", rows))
        for name, knob, value in trials:
            cfg = best.copy()
            for i in idx:
                getattr(cfg, knob)[i] = value
            if not cfg.apply(batch):
                continue
            t = _time_batch(batch, reps)
            timings[f"{key}:{name}"] = t
            if t < 0.99 * best_t:
                best, best_t = cfg, t
    best.apply(batch)
    choices = {key: {"kb": best.kb[idx[0]], "path": best.path[idx[0]],
                     "rows": best.rows[idx[0]]} for key, idx in groups.items()}
    if cache_path:
        cache.update(choices)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return {"choices": choices, "timings": timings, "untuned_ms": untuned, "tuned_ms": best_t,
            "config": {"kb": best.kb, "path": best.path, "rows": best.rows}}


def apply_config(batch: E.Batch, config: dict) -> bool:
    """Set a configuration returned by tune() ({"kb", "path", "rows"} lists) on a batch."""
    return _Config(config["kb"], config["path"], config["rows"]).apply(batch)


# ----------------------------------------------------------------------------- formats
# Candidate layouts for one matrix (the reference sweeps these by hand: its job scripts run
# every format and tile parameter and compare the timings).
FORMAT_CANDIDATES = {
    "k1": dict(fmt="K1"),
    "csr": dict(fmt="CSR"),
    "axt-unc-th2": dict(fmt="AXT", mode="UNC", tileH=2, tileHW=32),
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

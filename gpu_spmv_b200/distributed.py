"""Row-partitioned SpMV over several GPUs (one process per GPU, torch.distributed).

The matrix is cut into contiguous row blocks of about equal nnz (nnz_balanced_rows), one per
rank; x and y are distributed the same way (rank r owns entries rows[r]:rows[r+1]), as an
iterative solver needs for a square operator.  One product is

    x_full = all_gather(x_local)          (NCCL over NVLink; the one exchange step)
    y_local = A[rows_r, :] x_full          (the engine's K1 kernel on this rank's GPU)

and the adjoint of y = A x is

    xbar = reduce_scatter(A[rows_r, :]^T ybar_local)   (each rank's partial over all columns)

Uneven blocks are padded to the largest block for the collectives.  The local operator is
the engine's K1 matrix (gpu_spmv_b200.engine.Matrix); `local_factory` replaces it, which
the CPU tests use to run the exchange logic under the gloo backend with the oracle as the
local product.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def nnz_balanced_rows(row, parts: int) -> list[int]:
    """Row boundaries b[0]=0 <= ... <= b[parts]=n cutting the CSR row pointer `row` into
    `parts` blocks of about nnz/parts entries each (cut at the first row whose start
    reaches k*nnz/parts; empty blocks only when there are fewer rows than parts)."""
    row = np.asarray(row, dtype=np.int64)
    n, nnz = len(row) - 1, int(row[-1])
    b = [0]
    for k in range(1, parts):
        target = (nnz * k + parts - 1) // parts
        r = int(np.searchsorted(row, target, side="left"))
        b.append(min(max(r, b[-1]), n))
    b.append(n)
    return b


def _engine_factory(row, col, val, ncols, device, adjoint):
    from . import engine as E

    return E.Matrix(row, col, val, ncols=ncols, fmt="K1", device=device, adjoint=adjoint)


class DistSpMV:
    """This rank's row block of a square sparse matrix, with distributed products."""

    def __init__(self, row, col, val, ncols=None, group=None, device=None, adjoint=False,
                 local_factory=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        row = np.asarray(row, dtype=np.uint32)
        n = len(row) - 1
        self.n = n
        self.ncols = int(ncols if ncols is not None else n)
        if self.ncols != n:
            raise ValueError("distributed products take square matrices (x split like y)")
        self.bounds = nnz_balanced_rows(row, self.world)
        self.r0, self.r1 = self.bounds[self.rank], self.bounds[self.rank + 1]
        self.sizes = [self.bounds[k + 1] - self.bounds[k] for k in range(self.world)]
        self.pad = max(self.sizes) if self.sizes else 0
        e0, e1 = int(row[self.r0]), int(row[self.r1])
        lrow = (row[self.r0:self.r1 + 1] - row[self.r0]).astype(np.uint32)
        lcol = np.asarray(col)[e0:e1]
        lval = np.asarray(val)[e0:e1]
        self.device = torch.device(device) if device is not None else (
            torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available()
            else torch.device("cpu"))
        factory = local_factory or _engine_factory
        self.local = factory(lrow, lcol, lval, self.ncols, self.device, adjoint)

    # -------------------------------------------------------------- collectives
    def _gather_x(self, x_local: torch.Tensor) -> torch.Tensor:
        """Full x from every rank's block (padded all-gather)."""
        tail = tuple(x_local.shape[1:])
        buf = torch.zeros((self.pad,) + tail, dtype=x_local.dtype, device=x_local.device)
        buf[:x_local.shape[0]] = x_local
        parts = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(parts, buf, group=self.group)
        return torch.cat([p[:s] for p, s in zip(parts, self.sizes)], 0)

    def _scatter_sum(self, full: torch.Tensor) -> torch.Tensor:
        """Sum of every rank's `full` (ncols rows), this rank's block of it."""
        tail = tuple(full.shape[1:])
        if dist.get_backend(self.group) == "nccl":
            chunks = torch.zeros((self.world, self.pad) + tail, dtype=full.dtype,
                                 device=full.device)
            for k in range(self.world):
                chunks[k, :self.sizes[k]] = full[self.bounds[k]:self.bounds[k + 1]]
            out = torch.empty((self.pad,) + tail, dtype=full.dtype, device=full.device)
            dist.reduce_scatter_tensor(out, chunks.reshape((-1,) + tail), group=self.group)
            return out[:self.sizes[self.rank]]
        t = full.clone()  # backends without reduce-scatter: all-reduce, keep own block
        dist.all_reduce(t, group=self.group)
        return t[self.r0:self.r1]

    # -------------------------------------------------------------- products
    def spmv(self, x_local: torch.Tensor) -> torch.Tensor:
        """y_local = (A x)[rows of this rank], from this rank's block of x."""
        if x_local.shape[0] != self.r1 - self.r0:
            raise ValueError(f"rank {self.rank} owns {self.r1 - self.r0} entries of x")
        x_full = self._gather_x(x_local)
        return self.local.spmm(x_full) if x_full.dim() == 2 else self.local.spmv(x_full)

    def adjoint(self, ybar_local: torch.Tensor) -> torch.Tensor:
        """xbar_local = (A^T ybar)[rows of this rank], from this rank's block of ybar."""
        part, _ = self.local.adjoint(ybar_local.contiguous(), None, want_vbar=False)
        return self._scatter_sum(part)

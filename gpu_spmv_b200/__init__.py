"""gpu_spmv_b200 -- a B200 (sm_100a) SpMV engine with the host API of edoardoCB/gpu_spmv.

Layers:
  * ``include/gpuspmv_b200.h`` / ``lib/libgpuspmv_b200.so``: the C ABI -- the reference's
    format structs, converters and per-format entry points (drop-in), and the native
    device API (gs_*);
  * ``engine``: device-resident matrices (CSR / K1 / AXC / AXT) and SpMV from Python;
  * ``matgen``: seeded synthetic workloads;
  * ``refapi``: ctypes helpers for the drop-in layer;
  * ``autograd``: Y = A(v) X as a torch.autograd.Function over the hand-written adjoint;
  * ``autotune``: right-hand-side block widths for batched products (``engine.Batch``).
"""
from . import _lib
from ._lib import GSError, lib

__all__ = ["GSError", "lib", "engine", "matgen", "refapi", "autograd", "autotune", "version"]


def version() -> str:
    return lib().gs_version().decode()


def __getattr__(name):
    if name in ("engine", "matgen", "refapi", "autograd", "autotune"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)

"""gs_k1_spmv_f64_static, the K1 SpMV whose scratch is a static device array, for callers
that cannot allocate device memory: on the reference's K1 arrays (oracle-built, on the
device) two consecutive calls give y within the FP64 bound 1e-13 (|A||x|)_i of the oracle's
CPU loop and of the matrix-handle entry point (gs_spmv on a GS_FMT_K1 matrix), calls take
no device memory, and the size limit is refused on the host.  The two entry points cut long
rows into pieces of different lengths (256 and 128 steps), so they are compared within the
bound, not bit for bit."""
import ctypes as C

import numpy as np
import pytest
import torch

from mats import case, csr_from_lengths, within_bound


def _long_rows(rng):
    """Many chunks longer than one 256-step piece: 300 rows of 257..3000 entries."""
    n = 2048
    lens = rng.integers(0, 40, n)
    lens[rng.choice(n, 300, replace=False)] = rng.integers(257, 3000, 300)
    return csr_from_lengths(lens, 4096, rng) + (4096,)


def _matrix(name, rng):
    if name == "long_rows":
        return _long_rows(rng)
    row, col, val = case(name, rng)
    n = len(row) - 1
    return row, col, val, max(n, int(col.max()) + 1 if len(col) else n)


def _device_k1(k):
    from gpu_spmv_b200 import engine as E

    dev = torch.device("cuda")
    return {key: E.to_device_u32(k[key], dev) for key in ("col", "nmc", "chp", "permi")} | \
        {"val": torch.from_numpy(k["val"]).to(dev)}


def _static_spmv(k, d, x):
    from gpu_spmv_b200 import _lib as L

    y = torch.full((k["nrows"],), float("nan"), dtype=torch.float64, device=x.device)
    L.check(L.lib().gs_k1_spmv_f64_static(
        k["nrows"], k["chunkNum"], k["lenVC"], d["val"].data_ptr(), d["col"].data_ptr(),
        d["nmc"].data_ptr(), d["chp"].data_ptr(), d["permi"].data_ptr(), x.data_ptr(),
        y.data_ptr(), torch.cuda.current_stream().cuda_stream), "gs_k1_spmv_f64_static")
    return y


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mixed", "k1_empty_chunk", "single_row", "dense_row",
                                  "powerlaw_small", "long_rows"])
def test_static_matches_matrix_entry_point(port, name):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, name)) + 91)
    row, col, val, ncols = _matrix(name, rng)
    xh = rng.uniform(-1, 1, ncols)
    x = torch.from_numpy(xh).cuda()
    A = E.Matrix(row, col, val, ncols=ncols, fmt="K1")
    y_mat = A.spmv(x).cpu().numpy()
    k = port.k1(row, col, val)  # the reference's K1 arrays
    d = _device_k1(k)
    y_ref = port.csr_spmv(row, col, val, xh)
    _, mag = port.csr_truth(row, col, val, xh)
    for _ in range(2):  # the second call relies on the counters the first left at zero
        y = _static_spmv(k, d, x).cpu().numpy()
        assert within_bound(y, y_ref, mag), np.max(np.abs(y - y_ref) / np.maximum(mag, 1e-300))
        assert within_bound(y, y_mat, mag), np.max(np.abs(y - y_mat) / np.maximum(mag, 1e-300))
    A.close()


@pytest.mark.gpu
def test_static_unsorted_chunks_still_exact(port):
    """Full chunks in reverse (increasing nmc) order: the bisection's prefix no longer holds
    the long chunks, so long chunks past it run whole in one warp, and the products stay
    within the bound of the oracle's CPU loop."""
    rng = np.random.default_rng(3)
    row, col, val, ncols = _long_rows(rng)
    k = port.k1(row, col, val)
    nc = k["chunkNum"]
    full = nc - 1 if k["nrows"] % 32 else nc
    order = np.concatenate([np.arange(full)[::-1], np.arange(full, nc)])
    k2 = dict(k)
    k2["nmc"] = k["nmc"][order].copy()
    k2["chp"] = k["chp"][order].copy()
    permi = k["permi"].copy()
    permi[:nc * 32] = k["permi"][:nc * 32].reshape(nc, 32)[order].reshape(-1)
    k2["permi"] = permi
    xh = rng.uniform(-1, 1, ncols)
    x = torch.from_numpy(xh).cuda()
    y = _static_spmv(k2, _device_k1(k2), x).cpu().numpy()
    _, mag = port.csr_truth(row, col, val, xh)
    assert within_bound(y, port.csr_spmv(row, col, val, xh), mag)


@pytest.mark.gpu
def test_static_calls_take_no_device_memory(port):
    rng = np.random.default_rng(11)
    row, col, val, ncols = _long_rows(rng)
    k = port.k1(row, col, val)
    d = _device_k1(k)
    x = torch.from_numpy(rng.uniform(-1, 1, ncols)).cuda()
    _static_spmv(k, d, x)  # first call on the device: symbol look-up
    y = torch.empty(k["nrows"], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]  # after every buffer of the test exists
    from gpu_spmv_b200 import _lib as L
    for _ in range(3):
        L.check(L.lib().gs_k1_spmv_f64_static(
            k["nrows"], k["chunkNum"], k["lenVC"], d["val"].data_ptr(), d["col"].data_ptr(),
            d["nmc"].data_ptr(), d["chp"].data_ptr(), d["permi"].data_ptr(), x.data_ptr(),
            y.data_ptr(), torch.cuda.current_stream().cuda_stream), "gs_k1_spmv_f64_static")
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    yh = y.cpu().numpy()
    _, mag = port.csr_truth(row, col, val, x.cpu().numpy())
    assert within_bound(yh, port.csr_spmv(row, col, val, x.cpu().numpy()), mag)


def test_static_size_limit_refused_on_host():
    """Argument and size checks come before any CUDA call (runs without a GPU)."""
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import _lib as L

    f = L.lib().gs_k1_spmv_f64_static
    fake = [C.c_void_p(256)] * 7
    nrows = 1 << 20
    st = f(nrows, nrows // 32, L.GS_K1_STATIC_MAX_SLOTS + 1, *fake, None)
    assert st == L.GS_ERR_UNSUPPORTED
    assert "static scratch" in L.lib().gs_last_error().decode()
    with pytest.raises(GSError, match="GS_ERR_INVALID"):
        L.check(f(nrows, nrows // 32 + 1, 1000, *fake, None), "chunkNum")
    with pytest.raises(GSError, match="GS_ERR_INVALID"):
        L.check(f(nrows, nrows // 32, 1000, None, *fake[1:], None), "NULL")
    assert f(0, 0, 0, *([None] * 7), None) == L.GS_OK

"""Python front end of the native layer: device-resident matrices and SpMV.

PyTorch is used only for device memory and streams; every product runs in the engine's
sm_100a kernels through the C ABI (``gs_matrix_create`` / ``gs_spmv``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L

DTYPES = {"f64": L.GS_F64, "f32": L.GS_F32, "bf16": L.GS_BF16}
TORCH_DTYPES = {L.GS_F64: torch.float64, L.GS_F32: torch.float32, L.GS_BF16: torch.bfloat16}
FORMATS = {"CSR": L.GS_FMT_CSR, "K1": L.GS_FMT_K1, "AXC": L.GS_FMT_AXC, "AXT": L.GS_FMT_AXT}
MODES = {"UNC": L.GS_AXT_UNC, "NOC": L.GS_AXT_UNC, "COM": L.GS_AXT_COM}


def stream_handle(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def to_device_u32(a, device) -> torch.Tensor:
    """uint32 host/device array -> contiguous int32-typed device tensor (same bits)."""
    if isinstance(a, torch.Tensor):
        t = a
        if t.dtype == torch.uint32:
            t = t.view(torch.int32)
        return t.to(device=device).contiguous()
    arr = np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)
    return torch.from_numpy(arr).to(device)


def to_device(a, device, dtype) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


class Matrix:
    """A sparse matrix converted on the GPU into one of the engine's formats.

    fmt: "CSR", "K1", "AXC" (hbs) or "AXT" (tileHW, tileH, mode "UNC"/"COM", bs) -- the
    parameters of the reference converters getFormatData{K1,AXC,AXT}.  vtype "f64" / "f32"
    / "bf16" is the stored value type, itype "u32" or "u16" (16-bit column offsets).
    """

    def __init__(self, row, col, val, ncols=None, fmt="CSR", tileHW=32, tileH=1, bs=256,
                 mode="COM", hbs=32, vtype="f64", itype="u32", keep_layout=False,
                 device="cuda", stream=None):
        self._h = None
        dev = torch.device(device)
        row_t = to_device_u32(row, dev)
        col_t = to_device_u32(col, dev)
        vin = torch.float64 if (not isinstance(val, torch.Tensor) or val.dtype == torch.float64) \
            else torch.float32
        val_t = to_device(val, dev, vin)
        self.nrows = int(row_t.numel() - 1)
        self.nnz = int(col_t.numel())
        self.ncols = int(ncols if ncols is not None else self.nrows)
        self.fmt = fmt
        self.vtype = DTYPES[vtype]
        self.itype = L.GS_IDX_U16 if itype == "u16" else L.GS_IDX_U32
        p = L.ConvertParams(FORMATS[fmt], tileHW, tileH, bs, MODES[mode], hbs, self.vtype,
                            self.itype, 1 if keep_layout else 0)
        h = C.c_void_p()
        with torch.cuda.device(dev):
            st = L.lib().gs_matrix_create(
                C.byref(h), C.byref(p), self.nrows, self.ncols, self.nnz, row_t.data_ptr(),
                col_t.data_ptr(), val_t.data_ptr(),
                L.GS_F64 if vin == torch.float64 else L.GS_F32, stream_handle(stream))
        L.check(st, f"gs_matrix_create({fmt})")
        self._h = h
        self.device = dev
        self.info = self._info()

    def _info(self) -> L.MatrixInfo:
        i = L.MatrixInfo()
        L.check(L.lib().gs_matrix_get_info(self._h, C.byref(i)), "gs_matrix_get_info")
        return i

    # ---------------------------------------------------------------- products
    def spmv(self, x: torch.Tensor, y: torch.Tensor | None = None, acc64: bool = False,
             out_dtype=None, stream=None, tma: bool = False,
             striped: bool = False) -> torch.Tensor:
        """y = A x on the device (x: ncols entries; FP64 for FP64 matrices, else FP32).
        Kernel variants: tma=True stages 32-wide tileH>1 tiles with TMA bulk copies;
        striped=True maps one position per lane per 32-position chunk (CSR / COM
        tileH=1) instead of 8 consecutive positions per lane."""
        xt = torch.float64 if self.vtype == L.GS_F64 else torch.float32
        if x.dtype != xt or not x.is_cuda or not x.is_contiguous():
            raise TypeError(f"x must be a contiguous CUDA {xt} tensor")
        if y is None:
            ydt = out_dtype or (torch.float64 if (self.vtype == L.GS_F64 or acc64) else torch.float32)
            y = torch.empty(self.nrows, dtype=ydt, device=x.device)
        ycode = L.GS_F64 if y.dtype == torch.float64 else L.GS_F32
        xcode = L.GS_F64 if xt == torch.float64 else L.GS_F32
        flags = ((L.GS_FLAG_ACC_F64 if acc64 else 0) | (L.GS_FLAG_TMA if tma else 0) |
                 (L.GS_FLAG_STRIPED if striped else 0))
        L.check(L.lib().gs_spmv(self._h, x.data_ptr(), xcode, y.data_ptr(), ycode, flags,
                                stream_handle(stream)), "gs_spmv")
        return y

    def device_status(self, reset: bool = True) -> int:
        """Status word of the kernels (bit 0: a bounded wait timed out); synchronises."""
        w = L.UIN()
        L.check(L.lib().gs_matrix_device_status(self._h, C.byref(w), 1 if reset else 0),
                "gs_matrix_device_status")
        return w.value

    # ---------------------------------------------------------------- layout readback
    def layout(self) -> dict:
        """Copy the stored arrays back to the host (numpy), for parity checks."""
        i = self.info
        out = {}

        def grab(ptr, n, dt):
            if not ptr or n == 0:
                return np.zeros(0, dt)
            h = np.empty(n, dt)
            L.check(L.lib().gs_copy_to_host(h.ctypes.data, ptr, h.nbytes), "gs_copy_to_host")
            return h

        vdt = {L.GS_F64: np.float64, L.GS_F32: np.float32, L.GS_BF16: np.uint16}[i.vtype]
        idt = np.uint16 if i.itype == L.GS_IDX_U16 else np.uint32
        n = i.nrows
        out["val"] = grab(i.d_val, i.nslots, vdt)
        out["col"] = grab(i.d_col, i.nslots, idt)
        out["rpos"] = grab(i.d_rpos, n + 1, np.uint32)
        out["rlen"] = grab(i.d_rlen, n, np.uint32)
        if i.format == L.GS_FMT_AXT:
            out["sec"] = grab(i.d_sec, i.lenSEC, np.uint32)
            out["con"] = grab(i.d_con, i.lenCON + 1, np.uint32)
        if i.format == L.GS_FMT_AXC:
            out["brp"] = grab(i.d_brp, i.lenBRP, np.uint32)
            out["mapx"] = grab(i.d_mapx, i.lenMAPX, np.uint32)
        if i.format == L.GS_FMT_K1:
            out["permi"] = grab(i.d_permi, (i.chunkNum + 1) * 32, np.uint32)
            out["nmc"] = grab(i.d_nmc, i.chunkNum, np.uint32)
            out["chp"] = grab(i.d_chp, i.chunkNum, np.uint32)
        return out

    def close(self):
        if self._h:
            L.lib().gs_matrix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def csr_spmv_f64(row: torch.Tensor, col: torch.Tensor, val: torch.Tensor, x: torch.Tensor,
                 y: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """y = A x straight from device CSR arrays (row/col int32-typed views of uint32)."""
    n = row.numel() - 1
    if y is None:
        y = torch.empty(n, dtype=torch.float64, device=x.device)
    L.check(L.lib().gs_csr_spmv_f64(n, x.numel(), col.numel(), row.data_ptr(), col.data_ptr(),
                                    val.data_ptr(), x.data_ptr(), y.data_ptr(),
                                    stream_handle(stream)), "gs_csr_spmv_f64")
    return y


def algorithmic_bytes(nrows, ncols, nnz, k=1, s_v=8, s_i=4, s_x=8, s_y=8) -> float:
    return L.lib().gs_algorithmic_bytes(nrows, ncols, nnz, k, s_v, s_i, s_x, s_y)

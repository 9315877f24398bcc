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
                 device="cuda", stream=None, adjoint=False):
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
        self._values_key = None
        if adjoint:
            with torch.cuda.device(dev):
                L.check(L.lib().gs_matrix_prepare_adjoint(h, row_t.data_ptr(), col_t.data_ptr(),
                                                          stream_handle(stream)),
                        "gs_matrix_prepare_adjoint")

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

    # ---------------------------------------------------------------- multi-RHS / adjoint
    MM_K = (1, 2, 4, 8, 16, 32)

    def _value_dtype(self):
        if self.vtype not in (L.GS_F64, L.GS_F32):
            raise TypeError("multi-RHS products take FP64 or FP32 matrices")
        return TORCH_DTYPES[self.vtype]

    @classmethod
    def _blocks(cls, k: int):
        """Column blocks of at most 32 right-hand sides, each padded to a supported width."""
        out, c0 = [], 0
        while c0 < k:
            w = min(32, k - c0)
            kp = next(q for q in cls.MM_K if q >= w)
            out.append((c0, w, kp))
            c0 += w
        return out

    def spmm(self, X: torch.Tensor, stream=None) -> torch.Tensor:
        """Y = A X for X of shape [ncols, k] (any k; run in blocks of up to 32 columns)."""
        dt = self._value_dtype()
        if X.dim() == 1:
            return self.spmm(X[:, None], stream)[:, 0]
        if X.dtype != dt or not X.is_cuda or X.shape[0] != self.ncols:
            raise TypeError(f"X must be a CUDA {dt} tensor with {self.ncols} rows")
        k = X.shape[1]
        Y = torch.empty(self.nrows, k, dtype=dt, device=X.device)
        for c0, w, kp in self._blocks(k):
            Xb = X[:, c0:c0 + w]
            if kp != w or not Xb.is_contiguous() or Xb.data_ptr() % 32:
                Xp = torch.zeros(self.ncols, kp, dtype=dt, device=X.device)
                Xp[:, :w] = Xb
                Xb = Xp
            Yb = Y[:, c0:c0 + w] if (kp == w and w == k) else \
                torch.empty(self.nrows, kp, dtype=dt, device=X.device)
            L.check(L.lib().gs_spmm(self._h, Xb.data_ptr(), Yb.data_ptr(), self.vtype, kp,
                                    stream_handle(stream)), "gs_spmm")
            if Yb.data_ptr() != Y.data_ptr():
                Y[:, c0:c0 + w] = Yb[:, :w]
        return Y

    ORDERS = {"csr": L.GS_VALUES_CSR, "slots": L.GS_VALUES_SLOTS}

    def value_slots(self) -> int:
        """Length of a value array in "slots" order (the adjoint layout's slots)."""
        n = L.UIN()
        L.check(L.lib().gs_matrix_value_slots(self._h, C.byref(n)), "gs_matrix_value_slots")
        return n.value

    def _order_len(self, order: str) -> int:
        return self.nnz if order == "csr" else self.value_slots()

    def set_values(self, values: torch.Tensor, order: str = "csr", stream=None):
        """Replace the stored values by `values`: nnz entries in the CSR order of creation
        ("csr") or value_slots() entries in the adjoint layout's order ("slots"); needs a
        matrix created with adjoint=True."""
        dt = self._value_dtype()
        if values.dtype != dt or not values.is_cuda or values.numel() != self._order_len(order):
            raise TypeError(f"values must be {self._order_len(order)} CUDA {dt} entries")
        v = values.contiguous()
        L.check(L.lib().gs_matrix_set_values(self._h, v.data_ptr(), self.vtype,
                                             self.ORDERS[order], stream_handle(stream)),
                "gs_matrix_set_values")
        self._values_key = (v.data_ptr(), getattr(values, "_version", None), order)

    def convert_values(self, values: torch.Tensor, to: str, stream=None) -> torch.Tensor:
        """The same values in the other order ("csr" <-> "slots")."""
        src = "slots" if to == "csr" else "csr"
        dt = self._value_dtype()
        v = values.contiguous()
        if v.dtype != dt or v.numel() != self._order_len(src):
            raise TypeError(f"expected {self._order_len(src)} {dt} values in {src} order")
        out = torch.zeros(self._order_len(to), dtype=dt, device=v.device)
        L.check(L.lib().gs_matrix_convert_values(self._h, v.data_ptr(), self.ORDERS[src],
                                                 out.data_ptr(), self.vtype,
                                                 stream_handle(stream)),
                "gs_matrix_convert_values")
        return out

    def adjoint(self, Ybar: torch.Tensor, X: torch.Tensor | None = None, mode="deterministic",
                want_vbar: bool = True, order: str = "csr", stream=None):
        """(Xbar, vbar): Xbar = A^T Ybar, vbar[e] = Ybar[row_e] . X[col_e] in `order` ("csr"
        or "slots"; None unless want_vbar).  mode "deterministic" (transposed layout) or
        "atomic"."""
        dt = self._value_dtype()
        if Ybar.dim() == 1:
            Xb, vb = self.adjoint(Ybar[:, None], None if X is None else X[:, None], mode,
                                  want_vbar, order, stream)
            return Xb[:, 0], vb
        k = Ybar.shape[1]
        m = L.GS_ADJ_ATOMIC if mode == "atomic" else L.GS_ADJ_DETERMINISTIC
        if want_vbar and X is None:
            raise TypeError("vbar needs X")
        Xbar = torch.empty(self.ncols, k, dtype=dt, device=Ybar.device)
        nv = self._order_len(order)
        vbar = torch.zeros(nv, dtype=dt, device=Ybar.device) if want_vbar else None
        part = torch.zeros(nv, dtype=dt, device=Ybar.device) if want_vbar else None
        blocks = self._blocks(k)
        for i, (c0, w, kp) in enumerate(blocks):
            def padded(T, rows):
                Tb = T[:, c0:c0 + w]
                if kp == w and Tb.is_contiguous() and Tb.data_ptr() % 32 == 0:
                    return Tb
                P = torch.zeros(rows, kp, dtype=dt, device=Ybar.device)
                P[:, :w] = Tb
                return P
            Yb = padded(Ybar, self.nrows)
            Xin = padded(X, self.ncols) if want_vbar else None
            Xo = torch.empty(self.ncols, kp, dtype=dt, device=Ybar.device)
            vout = (vbar if len(blocks) == 1 else part) if want_vbar else None
            L.check(L.lib().gs_spmm_adjoint(
                self._h, Yb.data_ptr(), Xin.data_ptr() if Xin is not None else None,
                Xo.data_ptr(), vout.data_ptr() if vout is not None else None, self.vtype, kp,
                m, self.ORDERS[order], stream_handle(stream)), "gs_spmm_adjoint")
            Xbar[:, c0:c0 + w] = Xo[:, :w]
            if want_vbar and len(blocks) > 1:
                vbar += part
        return Xbar, vbar

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


class Batch:
    """Y_i = A_i X_i for many K1 matrices (FP64 or FP32) in one persistent launch.

    mats: K1 Matrix objects of one value type; ks: right-hand sides per matrix (1..32).
    Operands are [ncols_i, kpad_i] / [nrows_i, kpad_i] tensors (kpad_i = next power of two
    >= k_i; make_operands builds them, zero in the padding columns).
    """

    def __init__(self, mats, ks, stream=None):
        self.mats = list(mats)
        self.ks = [int(k) for k in ks]
        n = len(self.mats)
        arr_m = (C.c_void_p * max(1, n))(*[m._h for m in self.mats])
        arr_k = (L.UIN * max(1, n))(*self.ks)
        h = C.c_void_p()
        L.check(L.lib().gs_batch_create(C.byref(h), n, arr_m, arr_k, stream_handle(stream)),
                "gs_batch_create")
        self._h = h
        kp = (L.UIN * max(1, n))()
        nitems = L.UIN()
        flops = C.c_double()
        L.check(L.lib().gs_batch_info(h, C.byref(nitems), kp, C.byref(flops)), "gs_batch_info")
        self.kpad = [int(kp[i]) for i in range(n)]
        self.flops = flops.value
        self.blocking = list(self.kpad)
        self.dtype = TORCH_DTYPES[self.mats[0].vtype] if n else torch.float64
        self.X = self.Y = None

    @property
    def nitems(self) -> int:
        v = L.UIN()
        L.check(L.lib().gs_batch_info(self._h, C.byref(v), None, None), "gs_batch_info")
        return v.value

    def make_operands(self, Xs):
        """Padded device copies of the right-hand sides Xs[i] ([ncols_i, k_i]) and output
        buffers; registers them with the batch and returns (X list, Y list)."""
        dev = torch.device("cuda")
        X, Y = [], []
        for A, kp, k, x in zip(self.mats, self.kpad, self.ks, Xs):
            xp = torch.zeros(A.ncols, kp, dtype=self.dtype, device=dev)
            xp[:, :k] = torch.as_tensor(x, dtype=self.dtype).reshape(A.ncols, k).to(dev)
            X.append(xp)
            Y.append(torch.empty(A.nrows, kp, dtype=self.dtype, device=dev))
        self.set_operands(X, Y)
        return X, Y

    def set_operands(self, X, Y, stream=None):
        n = len(self.mats)
        ax = (C.c_void_p * max(1, n))(*[t.data_ptr() for t in X])
        ay = (C.c_void_p * max(1, n))(*[t.data_ptr() for t in Y])
        L.check(L.lib().gs_batch_set_operands(self._h, ax, ay, stream_handle(stream)),
                "gs_batch_set_operands")
        self.X, self.Y = X, Y

    def set_blocking(self, kb, stream=None):
        n = len(self.mats)
        arr = (L.UIN * max(1, n))(*[int(b) for b in kb])
        L.check(L.lib().gs_batch_set_blocking(self._h, arr, stream_handle(stream)),
                "gs_batch_set_blocking")
        self.blocking = [int(b) for b in kb]

    PATHS = {"auto": L.GS_BATCH_AUTO, "k1": L.GS_BATCH_K1, "band": L.GS_BATCH_BAND}

    def set_paths(self, paths, stream=None):
        """How each matrix runs: "k1" (warps over K1 units), "band" (thread blocks over row
        blocks with the X band staged in shared memory) or "auto" (band where it fits)."""
        n = len(self.mats)
        arr = (L.UIN * max(1, n))(*[self.PATHS[p] for p in paths])
        L.check(L.lib().gs_batch_set_paths(self._h, arr, stream_handle(stream)),
                "gs_batch_set_paths")

    def set_row_blocks(self, rows_max, stream=None):
        """Height of each matrix's row blocks (32..4096 rows; the row-block path's
        tileHeight)."""
        n = len(self.mats)
        arr = (L.UIN * max(1, n))(*[int(r) for r in rows_max])
        L.check(L.lib().gs_batch_set_row_blocks(self._h, arr, stream_handle(stream)),
                "gs_batch_set_row_blocks")

    @property
    def row_blocks(self):
        """(height, number of row blocks) per matrix; 0 blocks for a matrix on K1 units."""
        n = len(self.mats)
        h = (L.UIN * max(1, n))()
        b = (L.UIN * max(1, n))()
        L.check(L.lib().gs_batch_row_blocks(self._h, h, b), "gs_batch_row_blocks")
        return [(int(h[i]), int(b[i])) for i in range(n)]

    @property
    def paths(self):
        """The path each matrix runs on: "k1" or "band"."""
        n = len(self.mats)
        arr = (L.UIN * max(1, n))()
        L.check(L.lib().gs_batch_paths(self._h, arr), "gs_batch_paths")
        return ["band" if arr[i] == L.GS_BATCH_BAND else "k1" for i in range(n)]

    def status(self, stream=None) -> int:
        """Reads and clears the device status word (bit 0: a bounded wait timed out)."""
        v = L.UIN()
        L.check(L.lib().gs_batch_status(self._h, C.byref(v), stream_handle(stream)),
                "gs_batch_status")
        return v.value

    def run(self, graph: bool = True, stream=None):
        f = L.lib().gs_batch_run_graph if graph else L.lib().gs_batch_run
        L.check(f(self._h, stream_handle(stream)), "gs_batch_run")

    def results(self):
        """Y_i[:, :k_i] views."""
        return [y[:, :k] for y, k in zip(self.Y, self.ks)]

    def close(self):
        if getattr(self, "_h", None):
            L.lib().gs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""ORACLE TEST INFRASTRUCTURE -- ctypes front end for the two CPU oracles.

* ``Port``: the plain-C restatement in ``spmv_oracle.c`` (built by ``make -C oracle port``
  with gcc; always available, builds itself on first use if the library is missing).
* ``Ref``: the reference's own host code (cudaSpmv.cu / spmv_header.h) compiled unchanged
  into ``oracle/_ref/`` (``make -C oracle ref``; needs the reference tree at build time,
  the prebuilt libraries travel with the repository).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import
this module, and only as the checker / reported CPU baseline.  The product
(``gpu_spmv_b200``) never imports it.

All arrays are numpy; indices are uint32 (the reference's ``UIN``), values float64 (the
reference's ``FPT`` with ``FP_TYPE=FP_DOUBLE``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "libref_oracle.so")
REF_SPMV_SO = os.path.join(HERE, "_ref", "libref_spmv.so")
REF_GEN2_SO = os.path.join(HERE, "_ref", "libref_gen2.so")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_lock = threading.Lock()


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def build_port(force: bool = False) -> str:
    if force or not os.path.exists(PORT_SO):
        subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return PORT_SO


def build_ref(ref_dir: str | None = None) -> bool:
    """Compile the reference into oracle/_ref/ (``make -C oracle ref``) from the source tree
    named by `ref_dir`, the GS_REFERENCE_DIR environment variable, or the recipe's REF_DIR.
    A directory named here that holds no cudaSpmv.cu is an error; when the recipe's own
    directory is absent (a machine without the reference), the prebuilt libraries are kept
    and the result says whether they exist."""
    ref_dir = ref_dir or os.environ.get("GS_REFERENCE_DIR")
    cmd = ["make", "-s", "-C", HERE, "ref"]
    if ref_dir:
        if not os.path.exists(os.path.join(ref_dir, "cudaSpmv.cu")):
            raise FileNotFoundError(f"reference directory {ref_dir} holds no cudaSpmv.cu")
        cmd.append(f"REF_DIR={ref_dir}")
        subprocess.run(cmd, check=True)
        return True
    if subprocess.run(cmd, stderr=subprocess.DEVNULL).returncode != 0:
        return os.path.exists(REF_SO)
    return True


@dataclass
class AxtDims:
    tileN: int
    lenAX: int
    lenSEC: int
    lenCON: int
    log: int
    logTH: int


class _OrcAxtDims(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("tileN", "lenAX", "lenSEC", "lenCON", "log", "logTH")]


class Port:
    """The C restatement (spmv_oracle.c)."""

    _lib = None

    def __init__(self):
        with _lock:
            if Port._lib is None:
                lib = C.CDLL(build_port())
                u32, i32 = C.c_uint32, C.c_int
                sig = {
                    "orc_csr_spmv": (None, [u32, _u32p, _u32p, _f64p, _f64p, _f64p]),
                    "orc_csr_spmv_truth": (None, [u32, _u32p, _u32p, _f64p, _f64p, _f64p, _f64p]),
                    "orc_csr_spmm": (None, [u32, u32, _u32p, _u32p, _f64p, _f64p, _f64p]),
                    "orc_row_stats": (None, [u32, _u32p, _u32p, _u32p, _f64p]),
                    "orc_get_errors": (None, [u32, _f64p, _f64p, C.POINTER(C.c_double),
                                              C.POINTER(C.c_double), C.POINTER(u32)]),
                    "orc_k1_chunknum": (u32, [u32]),
                    "orc_k1_perm": (None, [u32, _u32p, _u32p]),
                    "orc_k1_nmc_chp": (u32, [u32, _u32p, _u32p, _u32p, _u32p]),
                    "orc_k1_fill": (None, [u32, _u32p, _u32p, _f64p, _u32p, _u32p, _f64p, _u32p]),
                    "orc_k1_spmv": (None, [u32, _u32p, _u32p, _u32p, _f64p, _u32p, _f64p, _f64p]),
                    "orc_axc_brp": (u32, [u32, u32, _u32p, _u32p]),
                    "orc_axc_fill": (None, [u32, u32, _u32p, _u32p, _f64p, C.c_void_p, _u32p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
                    "orc_axt_dims_con": (i32, [u32, _u32p, u32, u32, u32, i32, _u32p,
                                               C.POINTER(_OrcAxtDims)]),
                    "orc_axt_fill": (None, [u32, _u32p, _u32p, _f64p, C.c_void_p, u32, u32, u32,
                                            i32, _u32p, C.POINTER(_OrcAxtDims), C.c_void_p,
                                            C.c_void_p, C.c_void_p, _u32p]),
                    "orc_axt_spmv": (i32, [u32, u32, u32, u32, i32, C.POINTER(_OrcAxtDims),
                                           _u32p, _f64p, _u32p, _f64p, _f64p]),
                    "orc_axt_spmv_baked": (i32, [u32, u32, u32, u32, i32,
                                                 C.POINTER(_OrcAxtDims), _u32p, _f64p, _f64p]),
                }
                for name, (res, args) in sig.items():
                    f = getattr(lib, name)
                    f.restype = res
                    f.argtypes = args
                Port._lib = lib
        self.lib = Port._lib

    # --- CSR
    def csr_spmv(self, row, col, val, x):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        y = np.empty(n, np.float64)
        self.lib.orc_csr_spmv(n, row, col, val, x, y)
        return y

    def csr_truth(self, row, col, val, x):
        """(y in long-double accumulation, sum_j |a_ij||x_j|) per row."""
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        y = np.empty(n, np.float64)
        m = np.empty(n, np.float64)
        self.lib.orc_csr_spmv_truth(n, row, col, val, x, y, m)
        return y, m

    def csr_spmm(self, row, col, val, X):
        row, col, val = _u32(row), _u32(col), _f64(val)
        X = _f64(X)
        n, k = len(row) - 1, X.shape[1]
        Y = np.empty((n, k), np.float64)
        self.lib.orc_csr_spmm(n, k, row, col, val, X, Y)
        return Y

    def row_stats(self, row, col):
        row, col = _u32(row), _u32(col)
        n = len(row) - 1
        rl = np.empty(n, np.uint32)
        out = np.empty(5, np.float64)
        self.lib.orc_row_stats(n, row, col, rl, out)
        return rl, dict(rmin=int(out[0]), rave=out[1], rmax=int(out[2]), rsd=out[3],
                        bw=int(out[4]))

    def get_errors(self, ar, ac):
        a, r, p = C.c_double(), C.c_double(), C.c_uint32()
        self.lib.orc_get_errors(len(ar), _f64(ar), _f64(ac), C.byref(a), C.byref(r),
                                C.byref(p))
        return a.value, r.value, p.value

    # --- K1
    def k1(self, row, col, val):
        row, col, val = _u32(row), _u32(col), _f64(val)
        n = len(row) - 1
        rl = np.diff(row).astype(np.uint32)
        nc = self.lib.orc_k1_chunknum(n)
        permi = np.zeros((nc + 1) * 32, np.uint32)
        self.lib.orc_k1_perm(n, rl, permi)
        nmc = np.zeros(nc, np.uint32)
        chp = np.zeros(nc, np.uint32)
        lenvc = self.lib.orc_k1_nmc_chp(n, rl, permi, nmc, chp)
        kval = np.zeros(lenvc, np.float64)
        kcol = np.zeros(lenvc, np.uint32)
        self.lib.orc_k1_fill(n, row, col, val, permi, chp, kval, kcol)
        return dict(nrows=n, chunkNum=nc, lenVC=lenvc, permi=permi, nmc=nmc, chp=chp,
                    val=kval, col=kcol)

    def k1_spmv(self, k, x):
        y = np.empty(k["nrows"], np.float64)
        self.lib.orc_k1_spmv(k["nrows"], k["permi"], k["nmc"], k["chp"], k["val"], k["col"],
                             _f64(x), y)
        return y

    # --- AXC
    def axc(self, row, col, val, x=None, hbs=32):
        row, col, val = _u32(row), _u32(col), _f64(val)
        n = len(row) - 1
        rl = np.diff(row).astype(np.uint32)
        brp = np.zeros(n + 1, np.uint32)
        lenax = self.lib.orc_axc_brp(n, hbs, rl, brp)
        ax = np.zeros(lenax, np.float64) if x is not None else None
        xx = _f64(x) if x is not None else None
        nval = np.zeros(lenax // 2, np.float64)
        ncol = np.zeros(lenax // 2, np.uint32)
        mapx = np.zeros(lenax // 2 + 8, np.uint32)
        self.lib.orc_axc_fill(n, hbs, row, col, val, _ptr(xx), brp, _ptr(ax), _ptr(nval),
                              _ptr(ncol), _ptr(mapx))
        return dict(nrows=n, hbs=hbs, lenAX=lenax, lenBRP=n + 1, lenMAPX=lenax // 2 + 8,
                    brp=brp, ax=ax, val=nval, col=ncol, mapx=mapx)

    # --- AXT
    def axt(self, row, col, val, thw, th, mode, bs=256, x=None):
        """mode: 'UNC' (or 'NOC') / 'COM'."""
        row, col, val = _u32(row), _u32(col), _f64(val)
        n = len(row) - 1
        rl = np.diff(row).astype(np.uint32)
        m = 0 if mode in ("UNC", "NOC") else 1
        con = np.zeros(n + 1, np.uint32)
        d = _OrcAxtDims()
        if self.lib.orc_axt_dims_con(n, rl, thw, th, bs, m, con, C.byref(d)) != 0:
            raise ValueError("invalid AXT parameters")
        ax = np.zeros(d.lenAX, np.float64) if x is not None else None
        xx = _f64(x) if x is not None else None
        nval = np.zeros(d.lenAX // 2, np.float64)
        ncol = np.zeros(d.lenAX // 2, np.uint32)
        sec = np.zeros(d.lenSEC, np.uint32)
        self.lib.orc_axt_fill(n, row, col, val, _ptr(xx), thw, th, bs, m, con, C.byref(d),
                              _ptr(ax), _ptr(nval), _ptr(ncol), sec)
        dims = AxtDims(d.tileN, d.lenAX, d.lenSEC, d.lenCON, d.log, d.logTH)
        return dict(nrows=n, nnz=int(row[-1]), thw=thw, th=th, bs=bs, mode=m, dims=dims,
                    _d=d, con=con, ax=ax, val=nval, col=ncol, sec=sec)

    def axt_spmv(self, a, x):
        y = np.empty(a["nrows"], np.float64)
        rc = self.lib.orc_axt_spmv(a["nrows"], a["thw"], a["th"], a["bs"], a["mode"],
                                   C.byref(a["_d"]), a["sec"], a["val"], a["col"], _f64(x), y)
        if rc != 0:
            raise ValueError("malformed AXT metadata")
        return y

    def axt_spmv_baked(self, a):
        y = np.empty(a["nrows"], np.float64)
        rc = self.lib.orc_axt_spmv_baked(a["nrows"], a["thw"], a["th"], a["bs"], a["mode"],
                                         C.byref(a["_d"]), a["sec"], a["ax"], y)
        if rc != 0:
            raise ValueError("malformed AXT metadata")
        return y


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Ref:
    """The reference's own compiled host code (oracle/_ref)."""

    _lib = None
    _lib_spmv = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self):
        with _lock:
            if Ref._lib is None:
                if not os.path.exists(REF_SO):
                    raise FileNotFoundError(
                        f"{REF_SO} missing: build it with `make -C oracle ref` where the "
                        "reference sources are present")
                lib = C.CDLL(REF_SO)
                u32, vp = C.c_uint32, C.c_void_p
                sig = {
                    "ref_ncsr": (None, [u32, u32, u32, _f64p, _u32p, _u32p, _f64p, _f64p]),
                    "ref_init_vec": (None, [u32, u32, _f64p]),
                    "ref_get_errors": (None, [u32, _f64p, _f64p, C.POINTER(C.c_double),
                                              C.POINTER(C.c_double), C.POINTER(u32)]),
                    "ref_stats": (None, [C.c_char_p, u32, u32, _f64p, _u32p, _u32p, _u32p,
                                         _f64p]),
                    "ref_k1": (vp, [u32, u32, _f64p, _u32p, _u32p, _f64p, _f64p]),
                    "ref_k1_dims": (None, [vp, _u32p]),
                    "ref_k1_copy": (None, [vp, _u32p, _u32p, _u32p, _f64p, _u32p]),
                    "ref_k1_free": (None, [vp]),
                    "ref_axc": (vp, [u32, u32, u32, u32, _f64p, _u32p, _u32p, _f64p, _f64p]),
                    "ref_axc_dims": (None, [vp, _u32p]),
                    "ref_axc_copy": (None, [vp, _f64p, _u32p, _u32p]),
                    "ref_axc_free": (None, [vp]),
                    "ref_axt": (vp, [u32, u32, u32, u32, C.c_char_p, u32, u32, _f64p, _u32p,
                                     _u32p, _f64p, _f64p, C.c_char_p]),
                    "ref_axt_dims": (None, [vp, _u32p]),
                    "ref_axt_copy": (None, [vp, _f64p, _u32p, _u32p]),
                    "ref_axt_free": (None, [vp]),
                    "ref_gpu_csr": (C.c_double, [u32, u32, u32, _f64p, _u32p, _u32p, _f64p,
                                                 _f64p, _f64p]),
                    "ref_gpu_k1": (C.c_double, [vp, u32, _f64p, _f64p, _f64p]),
                    "ref_gpu_axc": (C.c_double, [vp, u32, _f64p, _f64p]),
                    "ref_gpu_axt_uh": (C.c_double, [vp, u32, u32, _f64p, _f64p]),
                    "ref_gpu_axt_uh1hw16": (C.c_double, [vp, u32, u32, _f64p, _f64p]),
                    "ref_gpu_axt_ch1": (C.c_double, [vp, _f64p, _f64p]),
                    "ref_gpu_axt_ch": (C.c_double, [vp, u32, _f64p, _f64p]),
                }
                for name, (res, args) in sig.items():
                    f = getattr(lib, name)
                    f.restype = res
                    f.argtypes = args
                Ref._lib = lib
                if os.path.exists(REF_SPMV_SO):
                    l2 = C.CDLL(REF_SPMV_SO)
                    l2.ref_cpuSpmvCSR.restype = None
                    l2.ref_cpuSpmvCSR.argtypes = [u32, u32, _f64p, _u32p, _u32p, _f64p, _f64p]
                    if hasattr(l2, "ref0_convert"):
                        PP = C.POINTER
                        l2.ref0_convert.restype = None
                        l2.ref0_convert.argtypes = [C.c_int, u32, u32, u32, _f64p, _u32p,
                                                    _u32p, _f64p, _f64p,
                                                    PP(PP(C.c_double)), PP(PP(u32)),
                                                    PP(PP(u32)), _u32p, C.c_char_p]
                        l2.ref0_free.restype = None
                        l2.ref0_free.argtypes = [C.c_void_p]
                    Ref._lib_spmv = l2
        self.lib = Ref._lib
        self.lib_spmv = Ref._lib_spmv

    def ncsr(self, row, col, val, x, threads=None):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        y = np.empty(n, np.float64)
        self.lib.ref_ncsr(threads or os.cpu_count() or 1, n, int(row[-1]), val, col, row, x, y)
        return y

    GEN0_KINDS = {"AXCv0": 0, "AXCv1": 1, "AXBv0": 2, "AXBv1": 3}

    def gen0(self, kind, row, col, val, x, cbs=256):
        """A brick format of the first generation (spmv_header.h: getFormatDataAXCv0,
        AXCv1, AXBv0, AXBv1) as the reference's own converter builds it: dict with ax, the
        index arrays (brp / rwp / hdr), blockLog (AXBv1), fd (mfp, beta, ct) and name."""
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        fd = np.zeros(3, np.float64)
        lens = np.zeros(4, np.uint32)
        name = C.create_string_buffer(16)
        pax = C.POINTER(C.c_double)()
        p1 = C.POINTER(C.c_uint32)()
        p2 = C.POINTER(C.c_uint32)()
        lib = self.lib_spmv
        lib.ref0_convert(self.GEN0_KINDS[kind], cbs, n, int(row[-1]), val, col, row, x, fd,
                         C.byref(pax), C.byref(p1), C.byref(p2), lens, name)

        def take(p, k, dt):
            if not p or k == 0:
                out = np.zeros(0, dt)
            else:
                out = np.ctypeslib.as_array(p, shape=(int(k),)).copy()
            if p:
                lib.ref0_free(C.cast(p, C.c_void_p))
            return out

        out = dict(ax=take(pax, lens[0], np.float64), fd=fd, name=name.value.decode(),
                   blockLog=int(lens[3]))
        i1 = take(p1, lens[1], np.uint32)
        i2 = take(p2, lens[2], np.uint32)
        if kind in ("AXCv0", "AXCv1"):
            out["brp"] = i1
        if kind == "AXCv1":
            out["rwp"] = i2
        if kind in ("AXBv0", "AXBv1"):
            out["hdr"] = i1
        return out

    def cpu_spmv_csr(self, row, col, val, x):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        y = np.empty(n, np.float64)
        self.lib_spmv.ref_cpuSpmvCSR(n, int(row[-1]), val, col, row, x, y)
        return y

    def init_vec(self, n):
        v = np.empty(n, np.float64)
        self.lib.ref_init_vec(1, n, v)
        return v

    def get_errors(self, ar, ac):
        a, r, p = C.c_double(), C.c_double(), C.c_uint32()
        self.lib.ref_get_errors(len(ar), _f64(ar), _f64(ac), C.byref(a), C.byref(r),
                                C.byref(p))
        return a.value, r.value, p.value

    def stats(self, path, row, col, val):
        row, col, val = _u32(row), _u32(col), _f64(val)
        n = len(row) - 1
        rl = np.zeros(n, np.uint32)
        out = np.zeros(5, np.float64)
        self.lib.ref_stats(path.encode(), n, int(row[-1]), val, col, row, rl, out)
        return rl, dict(rmin=int(out[0]), rave=out[1], rmax=int(out[2]), rsd=out[3],
                        bw=int(out[4]))

    def k1(self, row, col, val, x):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        fd = np.zeros(3, np.float64)
        h = self.lib.ref_k1(n, int(row[-1]), val, col, row, x, fd)
        d = np.zeros(4, np.uint32)
        self.lib.ref_k1_dims(h, d)
        nc, lenvc = int(d[2]), int(d[3])
        out = dict(nrows=n, chunkNum=nc, lenVC=lenvc,
                   permi=np.zeros((nc + 1) * 32, np.uint32), nmc=np.zeros(nc, np.uint32),
                   chp=np.zeros(nc, np.uint32), val=np.zeros(lenvc, np.float64),
                   col=np.zeros(lenvc, np.uint32), fd=fd)
        self.lib.ref_k1_copy(h, out["permi"], out["nmc"], out["chp"], out["val"], out["col"])
        self.lib.ref_k1_free(h)
        return out

    def axc(self, row, col, val, x, hbs=32, threads=1):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        fd = np.zeros(3, np.float64)
        h = self.lib.ref_axc(threads, hbs, n, int(row[-1]), val, col, row, x, fd)
        d = np.zeros(6, np.uint32)
        self.lib.ref_axc_dims(h, d)
        out = dict(nrows=n, hbs=int(d[2]), lenAX=int(d[3]), lenBRP=int(d[4]),
                   lenMAPX=int(d[5]), ax=np.zeros(int(d[3]), np.float64),
                   brp=np.zeros(int(d[4]), np.uint32), mapx=np.zeros(int(d[5]), np.uint32),
                   fd=fd)
        self.lib.ref_axc_copy(h, out["ax"], out["brp"], out["mapx"])
        self.lib.ref_axc_free(h)
        return out

    def axt(self, row, col, val, x, thw, th, mode, bs=256, threads=1):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        fd = np.zeros(3, np.float64)
        name = C.create_string_buffer(48)
        h = self.lib.ref_axt(threads, bs, thw, th, mode.encode(), n, int(row[-1]), val, col,
                             row, x, fd, name)
        d = np.zeros(11, np.uint32)
        self.lib.ref_axt_dims(h, d)
        keys = ("nrows", "nnz", "tileHW", "tileH", "logTH", "tileN", "lenAX", "lenSEC",
                "lenCON", "log", "bs")
        out = {k: int(v) for k, v in zip(keys, d)}
        out["ax"] = np.zeros(out["lenAX"], np.float64)
        out["sec"] = np.zeros(out["lenSEC"], np.uint32)
        out["con"] = np.zeros(out["lenCON"] + 1, np.uint32)
        out["fd"] = fd
        out["name"] = name.value.decode()
        self.lib.ref_axt_copy(h, out["ax"], out["sec"], out["con"])
        self.lib.ref_axt_free(h)
        return out


    # ---- the reference's own GPU products (its kernels compiled for sm_100a; GPU needed)
    def gpu_products(self, row, col, val, x, ref, cbs=256, tpw=4, th=4, reps=5):
        """Device seconds of one launch (median of `reps` calls) of the reference's gcsr,
        gk1, gaxc (hbs 32), gaxtuh (tileH th, tileHW 32, tpw tiles per warp), gaxtuh1hw16w
        (tileH 1, tileHW 16, 128 slots per warp), gaxtch1 (COM tileH 1, tileHW 32, header
        block = cbs) and gaxtch (COM tileH th, tileHW 32) on this matrix, and each one's get_errors
        summary against `ref`.  x is baked into the AXC / AXT layouts, as the reference does.
        The matrix must have no all-empty 32-row chunk (gk1 reads a chunk's first slot
        unconditionally)."""
        import statistics

        row, col, val, x, ref = _u32(row), _u32(col), _f64(val), _f64(x), _f64(ref)
        n, nnz = len(row) - 1, int(row[-1])
        out = {}

        def run(name, fn):
            ts, err = [], np.zeros(3, np.float64)
            for _ in range(reps):
                ts.append(fn(err))
            out[name] = dict(seconds=statistics.median(ts), aErr=err[0], rErr=err[1])

        run("gcsr", lambda e: self.lib.ref_gpu_csr(cbs, n, nnz, val, col, row, x, ref, e))
        fd = np.zeros(3, np.float64)
        h = self.lib.ref_k1(n, nnz, val, col, row, x, fd)
        run("gk1", lambda e: self.lib.ref_gpu_k1(h, cbs, x, ref, e))
        self.lib.ref_k1_free(h)
        threads = os.cpu_count() or 1
        h = self.lib.ref_axc(threads, 32, n, nnz, val, col, row, x, fd)
        run("gaxc", lambda e: self.lib.ref_gpu_axc(h, cbs, ref, e))
        self.lib.ref_axc_free(h)
        h = self.lib.ref_axt(threads, 256, 32, th, b"UNC", n, nnz, val, col, row, x, fd, None)
        run(f"gaxtuh{th}", lambda e: self.lib.ref_gpu_axt_uh(h, tpw, cbs, ref, e))
        self.lib.ref_axt_free(h)
        h = self.lib.ref_axt(threads, 256, 16, 1, b"UNC", n, nnz, val, col, row, x, fd, None)
        run("gaxtuh1hw16", lambda e: self.lib.ref_gpu_axt_uh1hw16(h, 128, cbs, ref, e))
        self.lib.ref_axt_free(h)
        h = self.lib.ref_axt(threads, cbs, 32, 1, b"COM", n, nnz, val, col, row, x, fd, None)
        run("gaxtch1", lambda e: self.lib.ref_gpu_axt_ch1(h, ref, e))
        self.lib.ref_axt_free(h)
        h = self.lib.ref_axt(threads, 256, 32, th, b"COM", n, nnz, val, col, row, x, fd, None)
        run(f"gaxtch{th}", lambda e: self.lib.ref_gpu_axt_ch(h, cbs, ref, e))
        self.lib.ref_axt_free(h)
        return out


class Ref2:
    """The reference's second API generation (gpuSpmv_header.h), compiled unchanged
    (oracle/_ref/libref_gen2.so)."""

    _lib = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_GEN2_SO)

    def __init__(self):
        with _lock:
            if Ref2._lib is None:
                if not os.path.exists(REF_GEN2_SO):
                    raise FileNotFoundError(f"{REF_GEN2_SO} missing: `make -C oracle ref`")
                lib = C.CDLL(REF_GEN2_SO)
                u32 = C.c_uint32
                sig = {
                    "ref2_stats": (None, [C.c_char_p, u32, u32, _f64p, _u32p, _u32p, _u32p, _f64p]),
                    "ref2_cf_csr": (None, [u32, u32, _f64p, _u32p, _u32p, _f64p, _f64p]),
                    "ref2_fd": (None, [C.c_char_p, _f64p]),
                    "ref2_axc": (None, [u32, u32, u32, _f64p, _u32p, _u32p, _f64p, _u32p]),
                    "ref2_axc_copy": (None, [_f64p, _u32p]),
                    "ref2_k1": (None, [u32, u32, u32, _f64p, _u32p, _u32p, _f64p, _u32p]),
                    "ref2_k1_copy": (None, [_u32p, _u32p, _u32p, _f64p, _u32p]),
                    "ref2_axt": (None, [u32, u32, u32, u32, C.c_char_p, u32, u32, _f64p,
                                        _u32p, _u32p, _f64p, _u32p]),
                    "ref2_axt_copy": (None, [_f64p, _u32p, _u32p]),
                }
                for name, (res, args) in sig.items():
                    f = getattr(lib, name)
                    f.restype = res
                    f.argtypes = args
                Ref2._lib = lib
        self.lib = Ref2._lib

    def _fd(self):
        name = C.create_string_buffer(18)
        mb = np.zeros(2)
        self.lib.ref2_fd(name, mb)
        return {"name": name.value.decode(), "mfp": mb[0], "beta": mb[1]}

    def stats(self, path, row, col, val):
        row, col, val = _u32(row), _u32(col), _f64(val)
        n = len(row) - 1
        rl = np.zeros(max(n, 1), np.uint32)
        out = np.zeros(5)
        self.lib.ref2_stats(path.encode(), n, len(col), val, col, row, rl, out)
        return rl[:n], dict(zip(("rmin", "rave", "rmax", "rsd", "bw"), out))

    def cf_csr(self, row, col, val, x):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        y = np.empty(n)
        self.lib.ref2_cf_csr(n, len(col), val, col, row, x, y)
        return y

    def axc(self, row, col, val, x, threads=1):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        dims = np.zeros(2, np.uint32)
        self.lib.ref2_axc(threads, n, len(col), val, col, row, x, dims)
        ax = np.zeros(int(dims[0]))
        brp = np.zeros(int(dims[1]), np.uint32)
        self.lib.ref2_axc_copy(ax, brp)
        return {"lenAX": int(dims[0]), "lenBRP": int(dims[1]), "ax": ax, "brp": brp,
                "fd": self._fd()}

    def k1(self, row, col, val, x, cbs=32):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        dims = np.zeros(2, np.uint32)
        self.lib.ref2_k1(cbs, n, len(col), val, col, row, x, dims)
        nc, lv = int(dims[0]), int(dims[1])
        out = {"chunkNum": nc, "lenVC": lv, "permi": np.zeros(nc * 32, np.uint32),
               "nmc": np.zeros(nc, np.uint32), "chp": np.zeros(nc, np.uint32),
               "val": np.zeros(lv), "col": np.zeros(lv, np.uint32)}
        self.lib.ref2_k1_copy(out["permi"], out["nmc"], out["chp"], out["val"], out["col"])
        out["fd"] = self._fd()
        return out

    def axt(self, row, col, val, x, thw, th, mode, bs=256, threads=1):
        row, col, val, x = _u32(row), _u32(col), _f64(val), _f64(x)
        n = len(row) - 1
        dims = np.zeros(6, np.uint32)
        self.lib.ref2_axt(threads, bs, thw, th, mode.encode(), n, len(col), val, col, row, x,
                          dims)
        keys = ("tileN", "lenAX", "lenSEC", "lenCON", "logTH", "log")
        out = {k: int(v) for k, v in zip(keys, dims)}
        out["ax"] = np.zeros(out["lenAX"])
        out["sec"] = np.zeros(out["lenSEC"], np.uint32)
        out["con"] = np.zeros(out["lenCON"], np.uint32)
        self.lib.ref2_axt_copy(out["ax"], out["sec"], out["con"])
        out["fd"] = self._fd()
        return out

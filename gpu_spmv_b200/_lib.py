"""ctypes bindings of ``libgpuspmv_b200.so`` (the C ABI declared in include/gpuspmv_b200.h).

The shared library is built in-tree (``python -m gpu_spmv_b200.build``).  Nothing here
falls back to another implementation: if the library is missing, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgpuspmv_b200.so")

UIN = C.c_uint32
FPT = C.c_double
UINp = C.POINTER(UIN)
FPTp = C.POINTER(FPT)

# status codes
GS_OK, GS_ERR_INVALID, GS_ERR_CUDA, GS_ERR_ALLOC, GS_ERR_OVERFLOW, GS_ERR_UNSUPPORTED, \
    GS_ERR_DEVICE = range(7)
# enums
GS_F64, GS_F32, GS_BF16 = 0, 1, 2
GS_IDX_U32, GS_IDX_U16 = 0, 1
GS_FMT_CSR, GS_FMT_K1, GS_FMT_AXC, GS_FMT_AXT = 0, 1, 2, 3
GS_AXT_UNC, GS_AXT_COM = 0, 1
GS_FLAG_NONE, GS_FLAG_ACC_F64, GS_FLAG_TMA, GS_FLAG_STRIPED = 0, 1, 2, 4
GS_K1_STATIC_MAX_SLOTS = 134217728
GS_ADJ_DETERMINISTIC, GS_ADJ_ATOMIC = 0, 1
GS_VALUES_CSR, GS_VALUES_SLOTS = 0, 1
GS_BATCH_AUTO, GS_BATCH_K1, GS_BATCH_BAND = 0, 1, 2


# ------------------------------------------------------------------ drop-in structs
class StrMatCSR(C.Structure):  # cudaSpmv.cu:261
    _fields_ = [("name", C.c_char * 48), ("nrows", UIN), ("nnz", UIN), ("rmin", UIN),
                ("rave", FPT), ("rmax", UIN), ("rsd", FPT), ("bw", UIN), ("val", FPTp),
                ("row", UINp), ("rowStart", UINp), ("rowEnd", UINp), ("col", UINp),
                ("rl", UINp)]


class StrFormatData(C.Structure):  # cudaSpmv.cu:385
    _fields_ = [("name", C.c_char * 48), ("mfp", C.c_double), ("beta", C.c_double),
                ("ct", C.c_double)]


class StrErr(C.Structure):  # cudaSpmv.cu:470
    _fields_ = [("aErr", C.c_double), ("rErr", C.c_double), ("pos", UIN)]


class StrRes(C.Structure):  # cudaSpmv.cu:499
    _fields_ = [("name", C.c_char * 48), ("et", C.c_double), ("ot", C.c_double),
                ("flops", C.c_double), ("sErr", StrErr)]


class StrMatK1(C.Structure):  # cudaSpmv.cu:712
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("chunkNum", UIN), ("lenVC", UIN),
                ("permi", UINp), ("nmc", UINp), ("chp", UINp), ("val", FPTp), ("col", UINp)]


class StrMatAXC(C.Structure):  # cudaSpmv.cu:933
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("hbs", UIN), ("lenAX", UIN), ("lenBRP", UIN),
                ("lenMAPX", UIN), ("ax", FPTp), ("brp", UINp), ("mapx", UINp)]


class StrMatAXT(C.Structure):  # cudaSpmv.cu:1154
    _fields_ = [("name", C.c_char * 48), ("nrows", UIN), ("nnz", UIN), ("mode", C.c_char * 8),
                ("tileHW", UIN), ("tileH", UIN), ("logTH", UIN), ("tileN", UIN),
                ("lenAX", UIN), ("lenSEC", UIN), ("lenCON", UIN), ("log", UIN), ("bs", UIN),
                ("ax", FPTp), ("sec", UINp), ("con", UINp)]


# ------------------------------------------------------------------ second API generation
class Gen0MatCSR(C.Structure):  # spmv_header.h:247
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("rmin", UIN), ("rave", FPT), ("rmax", UIN),
                ("rsd", FPT), ("bw", UIN), ("val", FPTp), ("row", UINp), ("col", UINp),
                ("rl", UINp)]


class Gen0FormatData(C.Structure):  # spmv_header.h:370
    _fields_ = [("name", C.c_char * 12), ("mfp", C.c_double), ("beta", C.c_double),
                ("ct", C.c_double)]


class Gen0Err(C.Structure):  # spmv_header.h:435
    _fields_ = [("aErr", C.c_double), ("rErr", C.c_double), ("pos", UIN)]


class Gen0Res(C.Structure):  # spmv_header.h:464
    _fields_ = [("name", C.c_char * 24), ("et", C.c_double), ("flops", C.c_double),
                ("sErr", Gen0Err)]


class Gen0MatAXCv0(C.Structure):  # spmv_header.h:665
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("lenAX", UIN), ("lenBRP", UIN), ("ax", FPTp),
                ("brp", UINp)]


class Gen0MatAXCv1(C.Structure):  # spmv_header.h:851
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("lenAX", UIN), ("lenBRP", UIN), ("lenRWP", UIN),
                ("ax", FPTp), ("brp", UINp), ("rwp", UINp)]


class Gen0MatAXBv0(C.Structure):  # spmv_header.h:1649
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("brickNum", UIN), ("lenAX", UIN),
                ("lenHDR", UIN), ("ax", FPTp), ("hdr0", UINp)]


class Gen0MatAXBv1(C.Structure):  # spmv_header.h:2299
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("brickNum", UIN), ("lenAX", UIN),
                ("lenHDR", UIN), ("blockLog", UIN), ("ax", FPTp), ("hdr1", UINp)]


class Gen2MatCSR(C.Structure):  # gpuSpmv_header.h:252
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("rmin", UIN), ("rave", FPT), ("rmax", UIN),
                ("rsd", FPT), ("bw", UIN), ("val", FPTp), ("row", UINp), ("col", UINp),
                ("rl", UINp)]


class Gen2FormatData(C.Structure):  # gpuSpmv_header.h:375
    _fields_ = [("name", C.c_char * 18), ("mfp", C.c_double), ("beta", C.c_double),
                ("ct", C.c_double)]


class Gen2Res(C.Structure):  # gpuSpmv_header.h:469
    _fields_ = [("name", C.c_char * 24), ("et", C.c_double), ("flops", C.c_double),
                ("sErr", StrErr)]


class Gen2MatAXC(C.Structure):  # gpuSpmv_header.h:675
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("lenAX", UIN), ("lenBRP", UIN), ("ax", FPTp),
                ("brp", UINp)]


class Gen2MatAXT(C.Structure):  # gpuSpmv_header.h:1082
    _fields_ = [("nrows", UIN), ("nnz", UIN), ("mode", C.c_char * 8), ("tileHW", UIN),
                ("tileH", UIN), ("logTH", UIN), ("tileN", UIN), ("lenAX", UIN),
                ("lenSEC", UIN), ("lenCON", UIN), ("log", UIN), ("ax", FPTp), ("sec", UINp),
                ("con", UINp)]


# ------------------------------------------------------------------ native structs
class ConvertParams(C.Structure):
    _fields_ = [("format", C.c_int), ("tileHW", UIN), ("tileH", UIN), ("bs", UIN),
                ("mode", C.c_int), ("hbs", UIN), ("vtype", C.c_int), ("itype", C.c_int),
                ("keep_layout", UIN)]


class MatrixInfo(C.Structure):
    _fields_ = [("format", C.c_int), ("nrows", UIN), ("ncols", UIN), ("nnz", UIN),
                ("tileHW", UIN), ("tileH", UIN), ("logTH", UIN), ("tileN", UIN),
                ("lenAX", UIN), ("lenSEC", UIN), ("lenCON", UIN), ("log", UIN), ("bs", UIN),
                ("mode", C.c_int), ("hbs", UIN), ("lenBRP", UIN), ("lenMAPX", UIN),
                ("chunkNum", UIN), ("lenVC", UIN), ("nslots", UIN), ("vtype", C.c_int),
                ("itype", C.c_int), ("d_val", C.c_void_p), ("d_col", C.c_void_p),
                ("d_colbase", C.c_void_p), ("d_sec", C.c_void_p), ("d_con", C.c_void_p),
                ("d_brp", C.c_void_p), ("d_mapx", C.c_void_p), ("d_permi", C.c_void_p),
                ("d_nmc", C.c_void_p), ("d_chp", C.c_void_p), ("d_rpos", C.c_void_p),
                ("d_rlen", C.c_void_p), ("conv_ms", C.c_double), ("mfp", C.c_double),
                ("beta", C.c_double), ("lane_positions", UIN), ("tiles_per_step", UIN)]


_vp = C.c_void_p
_st = C.c_int
SIGNATURES = {
    # drop-in layer
    "matrixReading": (StrMatCSR, [C.c_char_p]),
    "printMatrixStats": (None, [C.c_char_p, C.POINTER(StrMatCSR)]),
    "matrixWritingBin": (C.c_int, [C.c_char_p, C.POINTER(StrMatCSR)]),
    "getFormatDataCSR": (StrFormatData, [C.POINTER(StrMatCSR)]),
    "init_vec": (None, [UIN, UIN, FPTp]),
    "ncsr": (None, [UIN, StrMatCSR, FPTp, FPTp]),
    "get_errors": (None, [UIN, FPTp, FPTp, C.POINTER(StrErr)]),
    "getFormatDataK1": (StrFormatData, [UIN, StrMatCSR, FPTp, C.POINTER(StrMatK1)]),
    "getFormatDataAXC": (StrFormatData, [UIN, UIN, StrMatCSR, FPTp, C.POINTER(StrMatAXC)]),
    "getFormatDataAXT": (StrFormatData, [UIN, UIN, UIN, UIN, C.c_char_p, StrMatCSR, FPTp,
                                         C.POINTER(StrMatAXT)]),
    "test_gcsr": (StrRes, [UIN, StrMatCSR, FPTp, FPTp]),
    "test_gcucsr": (StrRes, [StrMatCSR, FPTp, FPTp]),
    "test_gk1": (StrRes, [UIN, StrMatK1, FPTp, FPTp]),
    "test_gaxc": (StrRes, [UIN, StrMatAXC, FPTp]),
    "test_gaxtuh1hw16w": (StrRes, [UIN, UIN, StrMatAXT, FPTp]),
    "test_gaxtuh1hw08w": (StrRes, [UIN, UIN, StrMatAXT, FPTp]),
    "test_gaxtuh1hw04w": (StrRes, [UIN, UIN, StrMatAXT, FPTp]),
    "test_gaxtuh": (StrRes, [UIN, UIN, StrMatAXT, FPTp]),
    "test_gaxtch1": (StrRes, [UIN, StrMatAXT, FPTp]),
    "test_gaxtch": (StrRes, [UIN, StrMatAXT, FPTp]),
    # second API generation (gpuspmv_b200_gen2.h)
    "gs2_matrixReading": (Gen2MatCSR, [C.c_char_p]),
    "gs2_printMatrixStats": (None, [C.c_char_p, C.POINTER(Gen2MatCSR)]),
    "gs2_getFormatDataCSR": (Gen2FormatData, [Gen2MatCSR]),
    "gs2_initVec": (None, [UIN, FPTp]),
    "gs2_cf_CSR": (None, [Gen2MatCSR, FPTp, FPTp]),
    "gs2_getErrors": (None, [UIN, FPTp, FPTp, C.POINTER(StrErr)]),
    "gs2_test_cf_CSR": (Gen2Res, [Gen2MatCSR, FPTp, FPTp]),
    "gs2_test_gk_CSR": (Gen2Res, [UIN, Gen2MatCSR, FPTp, FPTp]),
    "gs2_test_gcu_CSR": (Gen2Res, [Gen2MatCSR, FPTp, FPTp]),
    "gs2_getFormatDataAXC": (Gen2FormatData, [UIN, Gen2MatCSR, FPTp, C.POINTER(Gen2MatAXC)]),
    "gs2_test_gk_AXC": (Gen2Res, [UIN, Gen2MatAXC, FPTp]),
    "gs2_getFormatDataK1": (Gen2FormatData, [UIN, Gen2MatCSR, FPTp, C.POINTER(StrMatK1)]),
    "gs2_test_gk_K1": (Gen2Res, [UIN, StrMatK1, FPTp, FPTp]),
    "gs2_getFormatDataAXT": (Gen2FormatData, [UIN, UIN, UIN, UIN, C.c_char_p, Gen2MatCSR, FPTp,
                                              C.POINTER(Gen2MatAXT)]),
    "gs2_test_gk_AXT_NOC_H1": (Gen2Res, [UIN, Gen2MatAXT, FPTp]),
    "gs2_test_gk_AXT_NOC": (Gen2Res, [UIN, Gen2MatAXT, FPTp]),
    "gs2_test_gk_AXT_COM_H1": (Gen2Res, [UIN, Gen2MatAXT, FPTp]),
    # native layer
    "gs_status_string": (C.c_char_p, [_st]),
    "gs_last_error": (C.c_char_p, []),
    "gs_version": (C.c_char_p, []),
    "gs_set_num_ite": (None, [UIN]),
    "gs_get_num_ite": (UIN, []),
    "gs_matrix_create": (_st, [C.POINTER(_vp), C.POINTER(ConvertParams), UIN, UIN, UIN, _vp,
                               _vp, _vp, C.c_int, _vp]),
    "gs_matrix_create_host": (_st, [C.POINTER(_vp), C.POINTER(ConvertParams), UIN, UIN, UIN,
                                    _vp, _vp, _vp, C.c_int, _vp]),
    "gs_matrix_destroy": (_st, [_vp]),
    "gs_matrix_get_info": (_st, [_vp, C.POINTER(MatrixInfo)]),
    "gs_dropin_last_y": (UIN, [FPTp, UIN]),
    "gs0_getFormatDataAXCv0": (Gen0FormatData, [UIN, Gen0MatCSR, FPTp, C.POINTER(Gen0MatAXCv0)]),
    "gs0_getFormatDataAXCv1": (Gen0FormatData, [UIN, Gen0MatCSR, FPTp, C.POINTER(Gen0MatAXCv1)]),
    "gs0_getFormatDataAXBv0": (Gen0FormatData, [Gen0MatCSR, FPTp, C.POINTER(Gen0MatAXBv0)]),
    "gs0_getFormatDataAXBv1": (Gen0FormatData, [UIN, Gen0MatCSR, FPTp, C.POINTER(Gen0MatAXBv1)]),
    "gs0_testGpuSpmvAXCv0": (Gen0Res, [UIN, Gen0MatAXCv0, FPTp]),
    "gs0_testGpuSpmvAXCv1_0": (Gen0Res, [UIN, Gen0MatAXCv1, FPTp]),
    "gs0_testGpuSpmvAXCv1_1": (Gen0Res, [UIN, Gen0MatAXCv1, FPTp]),
    "gs0_testGpuSpmvAXCv1_2": (Gen0Res, [UIN, Gen0MatAXCv1, FPTp]),
    "gs0_testGpuSpmvAXCv1_3": (Gen0Res, [UIN, Gen0MatAXCv1, FPTp]),
    "gs0_testGpuSpmvAXCv1_4": (Gen0Res, [UIN, Gen0MatAXCv1, FPTp]),
    "gs0_testGpuSpmvAXBv0_0": (Gen0Res, [UIN, Gen0MatAXBv0, FPTp]),
    "gs0_testGpuSpmvAXBv0_1": (Gen0Res, [UIN, Gen0MatAXBv0, FPTp]),
    "gs0_testGpuSpmvAXBv0_2": (Gen0Res, [UIN, Gen0MatAXBv0, FPTp]),
    "gs0_testGpuSpmvAXBv0_3": (Gen0Res, [UIN, Gen0MatAXBv0, FPTp]),
    "gs0_testGpuSpmvAXBv1_0": (Gen0Res, [UIN, Gen0MatAXBv1, FPTp]),
    "gs_algorithmic_bytes": (C.c_double, [UIN, UIN, UIN, UIN, UIN, UIN, UIN, UIN]),
    "gs_spmv": (_st, [_vp, _vp, C.c_int, _vp, C.c_int, UIN, _vp]),
    "gs_spmv_host": (_st, [_vp, _vp, _vp, C.c_int, _vp, _vp, C.c_int, UIN, _vp]),
    "gs_spmv_host_stream": (_st, [_vp, _vp, C.c_size_t, C.c_int, _vp, C.c_size_t, C.c_int, UIN,
                                  UIN, _vp]),
    "gs_csr_spmv_f64": (_st, [UIN, UIN, UIN, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gs_k1_spmv_f64_static": (_st, [UIN, UIN, UIN, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gs_spmm": (_st, [_vp, _vp, _vp, C.c_int, UIN, _vp]),
    "gs_matrix_prepare_adjoint": (_st, [_vp, _vp, _vp, _vp]),
    "gs_matrix_set_values": (_st, [_vp, _vp, C.c_int, C.c_int, _vp]),
    "gs_matrix_value_slots": (_st, [_vp, C.POINTER(UIN)]),
    "gs_matrix_convert_values": (_st, [_vp, _vp, C.c_int, _vp, C.c_int, _vp]),
    "gs_spmm_adjoint": (_st, [_vp, _vp, _vp, _vp, _vp, C.c_int, UIN, C.c_int, C.c_int, _vp]),
    "gs_batch_create": (_st, [C.POINTER(_vp), UIN, C.POINTER(_vp), C.POINTER(UIN), _vp]),
    "gs_batch_destroy": (_st, [_vp]),
    "gs_batch_info": (_st, [_vp, C.POINTER(UIN), C.POINTER(UIN), C.POINTER(C.c_double)]),
    "gs_batch_set_operands": (_st, [_vp, C.POINTER(_vp), C.POINTER(_vp), _vp]),
    "gs_batch_set_blocking": (_st, [_vp, C.POINTER(UIN), _vp]),
    "gs_batch_set_paths": (_st, [_vp, C.POINTER(UIN), _vp]),
    "gs_batch_paths": (_st, [_vp, C.POINTER(UIN)]),
    "gs_batch_set_row_blocks": (_st, [_vp, C.POINTER(UIN), _vp]),
    "gs_batch_row_blocks": (_st, [_vp, C.POINTER(UIN), C.POINTER(UIN)]),
    "gs_batch_status": (_st, [_vp, C.POINTER(UIN), _vp]),
    "gs_batch_run": (_st, [_vp, _vp]),
    "gs_batch_run_graph": (_st, [_vp, _vp]),
    "gs_copy_to_host": (_st, [_vp, _vp, C.c_size_t]),
    "gs_matrix_device_status": (_st, [_vp, C.POINTER(UIN), C.c_int]),
    "gs_gen_laplacian2d": (_st, [UIN, C.POINTER(UINp), C.POINTER(UINp), C.POINTER(FPTp),
                                 C.POINTER(UIN), C.POINTER(UIN)]),
    "gs_gen_powerlaw": (_st, [UIN, C.c_uint64, C.c_double, C.c_double, UIN, C.c_uint64,
                              C.POINTER(UINp), C.POINTER(UINp), C.POINTER(FPTp),
                              C.POINTER(UIN)]),
    "gs_gen_stencil27": (_st, [UIN, C.c_uint64, C.POINTER(UINp), C.POINTER(UINp),
                               C.POINTER(FPTp), C.POINTER(UIN), C.POINTER(UIN)]),
    "gs_gen_banded": (_st, [UIN, UIN, UIN, UIN, C.c_uint64, C.POINTER(UINp), C.POINTER(UINp),
                            C.POINTER(FPTp), C.POINTER(UIN)]),
    "gs_gen_vector": (_st, [C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_uint64, FPTp]),
    "gs_free_host": (None, [_vp]),
}

_lib = None
_lock = threading.Lock()


class GSError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {_status_name(status)}: {detail}")


def _status_name(s):
    names = {0: "GS_OK", 1: "GS_ERR_INVALID", 2: "GS_ERR_CUDA", 3: "GS_ERR_ALLOC",
             4: "GS_ERR_OVERFLOW", 5: "GS_ERR_UNSUPPORTED", 6: "GS_ERR_DEVICE"}
    return names.get(s, f"status {s}")


def lib() -> C.CDLL:
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        f"{LIB_PATH} is missing: build the CUDA engine with "
                        "`python -m gpu_spmv_b200.build` (no CPU fallback exists)")
                L = C.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def check(status: int, where: str):
    if status != GS_OK:
        raise GSError(status, where, lib().gs_last_error().decode(errors="replace"))

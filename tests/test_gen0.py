"""The first API generation's brick formats (spmv_header.h: AXCv0, AXCv1, AXBv0, AXBv1)
through the drop-in gs0_* layer (include/gpuspmv_b200_gen0.h).

CPU: the header's structs have the sizes and field offsets of the reference's own (compiled
unchanged into oracle/_ref/libref_spmv.so), every declared symbol is exported, and a C
program written against the first generation's names compiles and links.
GPU: each converter returns the reference converter's arrays bit for bit with the same format
data (name, mfp, beta), and every entry point's y, read back row by row, is within
1e-13 (|A||x|)_i of the oracle's CPU loop."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from mats import CASES, case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER0 = os.path.join(ROOT, "include", "gpuspmv_b200_gen0.h")
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


def test_gen0_symbols_exported():
    from gpu_spmv_b200 import _lib as L

    src = re.sub(r"/\*.*?\*/", "", open(HEADER0).read(), flags=re.S)
    names = re.findall(r"\b(gs0_\w+)\s*\(", src)
    assert len(names) == 15
    lib = L.lib()
    for n in names:
        assert hasattr(lib, n), n


def test_gen0_struct_layouts_match_reference(tmp_path):
    from oracle.oracle import REF_SPMV_SO

    if not os.path.exists(REF_SPMV_SO):
        pytest.skip("first-generation oracle library not built")
    ref = C.CDLL(REF_SPMV_SO)
    if not hasattr(ref, "ref0_struct_layout"):
        pytest.skip("first-generation oracle library predates the layout export")
    ref.ref0_struct_layout.restype = C.c_size_t
    ref.ref0_struct_layout.argtypes = [C.c_char_p, C.c_size_t]
    buf = C.create_string_buffer(1 << 14)
    assert ref.ref0_struct_layout(buf, len(buf)) > 0
    want = dict(l.split() for l in buf.value.decode().splitlines())
    prog = tmp_path / "lay0.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER0}"',
             "int main(int argc, char **argv){"]
    for key in want:
        if "." in key:
            t, f = key.split(".")
            lines.append(f'printf("{key} %zu\\n", offsetof({t}, {f}));')
        else:
            lines.append(f'printf("{key} %zu\\n", sizeof({key}));')
    # never taken: only makes the first generation's names link
    lines += ["if (argc > 5) { str_matCSR m = {0}; FPT v[1]; str_matAXBv1 b;",
              "  str_formatData fd = getFormatDataAXBv1(256, m, v, &b);",
              "  str_res r = testGpuSpmvAXBv1_0(256, b, v); printf(\"%s %s\", fd.name, r.name); }",
              "return 0;}"]
    prog.write_text("\n".join(lines))
    exe = tmp_path / "lay0"
    from gpu_spmv_b200 import _lib as L

    lib = os.path.dirname(L.LIB_PATH)
    subprocess.run(["gcc", str(prog), "-o", str(exe), f"-L{lib}", "-lgpuspmv_b200",
                    f"-Wl,-rpath,{lib}"], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    assert len(want) == 59  # 8 sizes, 51 field offsets
    assert got == want


def _inputs(name):
    rng = np.random.default_rng(sum(map(ord, os.path.basename(name))) + 3)
    if name.endswith(".npz"):
        g = np.load(name)
        row, col, val = g["row"], g["col"], g["val"]
        x = np.arange(len(row) - 1, dtype=np.float64)
    else:
        row, col, val = case(name, rng)
        x = rng.uniform(-1, 1, len(row) - 1)
    return row, col, val, x


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES + GOLDEN,
                         ids=CASES + [os.path.basename(p) for p in GOLDEN])
def test_gen0_converters_and_products(port, ref, name):
    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import refapi as R

    if ref.lib_spmv is None or not hasattr(ref.lib_spmv, "ref0_convert"):
        pytest.skip("first-generation oracle library not built")
    row, col, val, x = _inputs(name)
    n = len(row) - 1
    if len(x) < n or (len(col) and int(col.max()) >= len(x)):
        pytest.skip("square matrices only")
    lib = L.lib()
    lib.gs_set_num_ite(3)
    h = R.csr_struct(row, col, val)
    m = L.Gen0MatCSR(nrows=n, nnz=len(col), val=h.s.val, row=h.s.row, col=h.s.col, rl=h.s.rl)
    xp = R.f64p(np.ascontiguousarray(x))
    y_ref = port.csr_spmv(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)
    yp = R.f64p(y_ref)

    def check_y(res, what):
        assert res.name != b"error", (what, lib.gs_last_error())
        y = R.last_y(n)
        err = np.abs(y - y_ref)
        assert np.all(err <= 1e-13 * mag), (what, float(np.max(err / np.maximum(mag, 1e-300))))

    def same_fd(fd, r, kind):
        assert fd.name.decode() == r["name"] == kind
        assert (fd.mfp, fd.beta) == (r["fd"][0], r["fd"][1]), kind

    a0 = L.Gen0MatAXCv0()
    fd = lib.gs0_getFormatDataAXCv0(1, m, xp, C.byref(a0))
    r = ref.gen0("AXCv0", row, col, val, x)
    same_fd(fd, r, "AXCv0")
    assert np.array_equal(R.arr_f64(a0.ax, a0.lenAX), r["ax"])
    assert np.array_equal(R.arr_u32(a0.brp, a0.lenBRP), r["brp"])
    res = lib.gs0_testGpuSpmvAXCv0(256, a0, yp)
    assert res.name == b"gk_AXCv0"
    check_y(res, "AXCv0")
    R.free_struct_arrays(a0, ("ax", "brp"))

    a1 = L.Gen0MatAXCv1()
    fd = lib.gs0_getFormatDataAXCv1(1, m, xp, C.byref(a1))
    r = ref.gen0("AXCv1", row, col, val, x)
    same_fd(fd, r, "AXCv1")
    assert np.array_equal(R.arr_f64(a1.ax, a1.lenAX), r["ax"])
    assert np.array_equal(R.arr_u32(a1.brp, a1.lenBRP), r["brp"])
    assert np.array_equal(R.arr_u32(a1.rwp, a1.lenRWP), r["rwp"])
    for k in range(5):
        res = getattr(lib, f"gs0_testGpuSpmvAXCv1_{k}")(256, a1, yp)
        assert res.name == f"gk_AXCv1_{k}".encode()
        check_y(res, f"AXCv1_{k}")
    R.free_struct_arrays(a1, ("ax", "brp", "rwp"))

    b0 = L.Gen0MatAXBv0()
    fd = lib.gs0_getFormatDataAXBv0(m, xp, C.byref(b0))
    r = ref.gen0("AXBv0", row, col, val, x)
    same_fd(fd, r, "AXBv0")
    assert b0.brickNum == (len(col) + 15) // 16
    assert np.array_equal(R.arr_f64(b0.ax, b0.lenAX), r["ax"])
    assert np.array_equal(R.arr_u32(b0.hdr0, b0.lenHDR), r["hdr"])
    for k in range(4):
        res = getattr(lib, f"gs0_testGpuSpmvAXBv0_{k}")(256, b0, yp)
        assert res.name == f"gk_AXBv0_{k}".encode()
        check_y(res, f"AXBv0_{k}")
    R.free_struct_arrays(b0, ("ax", "hdr0"))

    for cbs in (32, 256, 1024):
        b1 = L.Gen0MatAXBv1()
        fd = lib.gs0_getFormatDataAXBv1(cbs, m, xp, C.byref(b1))
        r = ref.gen0("AXBv1", row, col, val, x, cbs=cbs)
        same_fd(fd, r, "AXBv1")
        assert b1.blockLog == r["blockLog"]
        assert np.array_equal(R.arr_f64(b1.ax, b1.lenAX), r["ax"])
        assert np.array_equal(R.arr_u32(b1.hdr1, b1.lenHDR), r["hdr"])
        res = lib.gs0_testGpuSpmvAXBv1_0(cbs, b1, yp)
        assert res.name == b"gk_AXBv1_0"
        check_y(res, f"AXBv1 cbs {cbs}")
        R.free_struct_arrays(b1, ("ax", "hdr1"))
    b1 = L.Gen0MatAXBv1()
    fd = lib.gs0_getFormatDataAXBv1(96, m, xp, C.byref(b1))
    assert fd.name == b"error" and b"power of two" in lib.gs_last_error()
    lib.gs_set_num_ite(250)

"""The C ABI library loads here (no GPU), exports every function include/gpuspmv_b200.h
declares, and its struct layouts match the header (checked with a host C compiler)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from gpu_spmv_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpuspmv_b200.h")
HEADER2 = os.path.join(ROOT, "include", "gpuspmv_b200_gen2.h")


def declared_functions(header=HEADER):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    src = re.sub(r"#[^\n]*", "", src)
    src = re.sub(r"typedef\s+struct\s*\{.*?\}\s*\w+\s*;", "", src, flags=re.S)
    src = re.sub(r"typedef[^;]*;", "", src)
    names = re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions() + declared_functions(HEADER2)
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(L.SIGNATURES), set(names) - set(L.SIGNATURES)


def test_version_and_status_strings():
    lib = L.lib()
    assert b"sm_100a" in lib.gs_version()
    assert lib.gs_status_string(L.GS_ERR_OVERFLOW) == b"GS_ERR_OVERFLOW"
    lib.gs_set_num_ite(7)
    assert lib.gs_get_num_ite() == 7
    lib.gs_set_num_ite(250)


def test_argument_errors_need_no_gpu():
    lib = L.lib()
    h = C.c_void_p()
    assert lib.gs_matrix_create(C.byref(h), None, 1, 1, 0, None, None, None, 0, None) == \
        L.GS_ERR_INVALID
    assert lib.gs_spmv(None, None, 0, None, 0, 0, None) == L.GS_ERR_INVALID
    assert lib.gs_matrix_get_info(None, None) == L.GS_ERR_INVALID
    assert b"NULL" in lib.gs_last_error()


@pytest.mark.parametrize("case,expect", [
    # algorithmic bytes of one product: nnz(s_v+s_i) + 4(n+1) + s_x n k + s_y n k
    ((262144, 262144, 1308672, 1, 8, 4, 8, 8), 20946948),
    ((4194304, 4194304, 67108864, 1, 8, 4, 8, 8), 889192452),
    ((4096000, 4096000, 109215352, 1, 8, 4, 8, 8), 1392504228),
    ((4096000, 4096000, 109215352, 1, 4, 4, 4, 4), 922874820),
    ((4096000, 4096000, 109215352, 1, 2, 2, 4, 4), 486013412),
    ((1048576, 1048576, 16777216, 8, 4, 4, 4, 4), 205520900),
])
def test_algorithmic_bytes(case, expect):
    assert L.lib().gs_algorithmic_bytes(*case) == expect


def test_struct_layouts_match_header(tmp_path):
    prog = tmp_path / "sz.c"
    structs = ["str_matCSR", "str_formatData", "str_err", "str_res", "str_matK1",
               "str_matAXC", "str_matAXT", "gs_convert_params", "gs_matrix_info"]
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             "int main(void){"]
    for s in structs:
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
    lines.append('printf("axt_ax %zu\\n", offsetof(str_matAXT, ax));')
    lines.append('printf("res_sErr %zu\\n", offsetof(str_res, sErr));')
    lines.append('printf("info_conv %zu\\n", offsetof(gs_matrix_info, conv_ms));')
    lines.append("return 0;}")
    prog.write_text("\n".join(lines))
    exe = tmp_path / "sz"
    subprocess.run(["gcc", str(prog), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    ct = {"str_matCSR": L.StrMatCSR, "str_formatData": L.StrFormatData, "str_err": L.StrErr,
          "str_res": L.StrRes, "str_matK1": L.StrMatK1, "str_matAXC": L.StrMatAXC,
          "str_matAXT": L.StrMatAXT, "gs_convert_params": L.ConvertParams,
          "gs_matrix_info": L.MatrixInfo}
    for s, cls in ct.items():
        assert int(out[s]) == C.sizeof(cls), s
    assert int(out["axt_ax"]) == L.StrMatAXT.ax.offset
    assert int(out["res_sErr"]) == L.StrRes.sErr.offset
    assert int(out["info_conv"]) == L.MatrixInfo.conv_ms.offset


def test_gen2_struct_layouts_and_names(tmp_path):
    """The second-generation header compiles (alone, and through GS_API_GEN2), its structs
    match the ctypes mirror, and a program using that API's names links."""
    prog = tmp_path / "g2.c"
    prog.write_text("\n".join([
        "#include <stdio.h>", "#include <stddef.h>", "#define GS_API_GEN2",
        f'#include "{HEADER}"',
        "int main(int argc, char **argv){",
        'printf("csr %zu\\n", sizeof(str_matCSR));',
        'printf("fd %zu\\n", sizeof(str_formatData));',
        'printf("res %zu\\n", sizeof(str_res));',
        'printf("axc %zu\\n", sizeof(str_matAXC));',
        'printf("axt %zu\\n", sizeof(str_matAXT));',
        'printf("axt_con %zu\\n", offsetof(str_matAXT, con));',
        "if (argc > 5) {",  # never taken: only makes the names link
        "  str_matCSR m = matrixReading(argv[1]); printMatrixStats(argv[1], &m);",
        "  FPT v[4]; initVec(4, v); str_matAXT a;",
        "  str_formatData fd = getFormatDataAXT(1, 256, 32, 1, \"NOC\", m, v, &a);",
        "  str_res r = test_gk_AXT_NOC_H1(256, a, v); printf(\"%s %s\", fd.name, r.name); }",
        "return 0;}"]))
    exe = tmp_path / "g2"
    lib = os.path.dirname(L.LIB_PATH)
    subprocess.run(["gcc", str(prog), "-o", str(exe), f"-L{lib}", "-lgpuspmv_b200",
                    f"-Wl,-rpath,{lib}"], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    assert int(out["csr"]) == C.sizeof(L.Gen2MatCSR)
    assert int(out["fd"]) == C.sizeof(L.Gen2FormatData)
    assert int(out["res"]) == C.sizeof(L.Gen2Res)
    assert int(out["axc"]) == C.sizeof(L.Gen2MatAXC)
    assert int(out["axt"]) == C.sizeof(L.Gen2MatAXT)
    assert int(out["axt_con"]) == L.Gen2MatAXT.con.offset


def test_reference_arm_loads_no_engine_code():
    """bench.py --impl reference times the reference's own CPU SpMV on inputs from the
    oracle-side generator: no library of the engine package may be mapped into it."""
    import json
    import subprocess
    import sys

    from oracle.oracle import Ref

    if not Ref.available():
        pytest.skip("reference oracle library oracle/_ref not built")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--workload", "laplacian", "--steps", "3", "--warmup", "3"],
                         capture_output=True, text=True, check=True, timeout=600)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    libs = line["loaded_libraries"]
    assert any(p.startswith("oracle/") for p in libs), libs
    assert not any(p.startswith("gpu_spmv_b200/") for p in libs), libs


def test_struct_layouts_match_compiled_reference(tmp_path):
    """sizeof and every field offset of the drop-in header's str_matCSR, str_formatData,
    str_err, str_res, str_matK1, str_matAXC and str_matAXT equal those of the reference's own
    structs (cudaSpmv.cu:261, 385, 470, 499, 712, 933, 1154) as its compiled source lays them
    out (oracle/_ref/libref_oracle.so)."""
    from oracle.oracle import REF_SO, Ref

    if not Ref.available():
        pytest.skip("reference oracle library oracle/_ref not built")
    ref = C.CDLL(REF_SO)
    ref.ref_struct_layout.restype = C.c_size_t
    ref.ref_struct_layout.argtypes = [C.c_char_p, C.c_size_t]
    buf = C.create_string_buffer(1 << 14)
    assert ref.ref_struct_layout(buf, len(buf)) > 0
    want = dict(l.split() for l in buf.value.decode().splitlines())
    prog = tmp_path / "lay.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             "int main(void){"]
    for key in want:
        if "." in key:
            t, f = key.split(".")
            lines.append(f'printf("{key} %zu\\n", offsetof({t}, {f}));')
        else:
            lines.append(f'printf("{key} %zu\\n", sizeof({key}));')
    lines.append("return 0;}")
    prog.write_text("\n".join(lines))
    exe = tmp_path / "lay"
    subprocess.run(["gcc", str(prog), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    assert len(want) == 67  # 7 sizes, 60 field offsets
    assert got == want

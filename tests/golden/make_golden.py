"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own compiled host code
(oracle/_ref, built from cudaSpmv.cu / spmv_header.h unchanged).

    python tests/golden/make_golden.py

For each small seeded matrix it records the reference's outputs:
  * ncsr / cpuSpmvCSR y for x uniform[-1,1] and for x[i] = i (init_vec),
  * getFormatDataK1 arrays (permi, nmc, chp, val, col),
  * getFormatDataAXC arrays (brp, ax, mapx) for x[i] = i,
  * getFormatDataAXT arrays (ax, sec, con) and dimensions for every (mode, tileH, tileHW,
    bs) of the reference's main (cudaSpmv.cu:2349-2360) plus tileH 2 / 8 / 16,
  * printMatrixStats statistics and rl.
The fixtures pin the CPU restatement (oracle/spmv_oracle.c) and the engine without the
reference tree present.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import Ref, build_ref  # noqa: E402
from mats import AXT_PARAMS, csr_from_lengths  # noqa: E402


def golden_cases():
    rng = np.random.default_rng(2024)
    out = {}
    lens = rng.integers(0, 41, 150)
    lens[0] = 1
    lens[4] = 0
    lens[20] = 32
    lens[21] = 96
    lens[-1] = 0
    out["g_mixed"] = csr_from_lengths(lens, 150, rng)
    lens = rng.integers(0, 9, 100)
    lens[:3] = 0
    out["g_row0_empty"] = csr_from_lengths(lens, 100, rng)
    lens = np.clip(np.rint(np.clip(rng.lognormal(2.5, 1.2, 200), 1, 300) * 0.64), 1, 190)
    out["g_powerlaw"] = csr_from_lengths(lens.astype(np.int64), 200, rng)
    return out


def main():
    build_ref()
    R = Ref()
    for name, (row, col, val) in golden_cases().items():
        n = len(row) - 1
        rng = np.random.default_rng(7)
        x = rng.uniform(-1, 1, n)
        xi = R.init_vec(n)
        rec = dict(row=row, col=col, val=val, x=x,
                   y_ncsr=R.ncsr(row, col, val, x), y_ncsr_xi=R.ncsr(row, col, val, xi),
                   y_cpuSpmvCSR=R.cpu_spmv_csr(row, col, val, x))
        with tempfile.TemporaryDirectory() as td:
            rl, st = R.stats(os.path.join(td, "m.bin"), row, col, val)
        rec["rl"] = rl
        rec["stats"] = np.array([st["rmin"], st["rave"], st["rmax"], st["rsd"], st["bw"]])
        k = R.k1(row, col, val, xi)
        for f in ("permi", "nmc", "chp", "val", "col"):
            rec[f"k1_{f}"] = k[f]
        a = R.axc(row, col, val, xi, hbs=32)
        for f in ("brp", "ax", "mapx"):
            rec[f"axc_{f}"] = a[f]
        for (mode, th, thw, bs) in AXT_PARAMS:
            t = R.axt(row, col, val, xi, thw, th, mode, bs=bs)
            key = f"axt_{mode}_{th}_{thw}_{bs}"
            rec[key + "_ax"] = t["ax"]
            rec[key + "_sec"] = t["sec"]
            rec[key + "_con"] = t["con"]
            rec[key + "_dims"] = np.array([t[k] for k in ("tileN", "lenAX", "lenSEC", "lenCON",
                                                          "log", "logTH")], np.uint32)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print(name, n, len(col))


if __name__ == "__main__":
    main()

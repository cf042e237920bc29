"""Generate the golden fixtures in this folder from the CPU oracle.

The reference (EFDC+ 8.5, Intel Fortran) ships no tests, golden vectors or
result files for the external mode and cannot be compiled here, so these
fixtures are outputs of the oracle restatement itself: they pin the oracle
(and, on the GPU, the CUDA library) against drift.  Each case is a seeded
scenario run for a few CALPUV2C steps; the fixture stores the input seed
parameters, the per-step statistics and the final state.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "efdcplus8.5_b200"))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "tests"))

import cases  # noqa: E402
import oracle as O  # noqa: E402

KEYS = ("p", "hp", "h1p", "hu", "hv", "uhdye", "vhdxe", "uhe", "vhe", "sub", "svb", "sbx",
        "sby", "lmaskdry", "iscdry", "lopenbcdry", "natdry", "qdwaste", "vdwaste")


def main():
    for name in cases.GOLDEN:
        scn, steps, tmul = cases.build(name)
        st, stats = O.run(scn, steps, nthreads=1, lists=True, tn_mul=tmul)
        out = {f"state_{k}": st[k] for k in KEYS}
        out["lwet"] = st["lwet"]
        out["ldry"] = st["ldry"]
        for k in ("status", "iters_total", "solves", "lawet", "ladry", "n_negdep", "n_wasted"):
            out[f"stat_{k}"] = np.array([s[k] for s in stats], np.int64)
        out["stat_rsq_last"] = np.array([s["rsq_last"] for s in stats])
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, "la", scn.la, "steps", steps, "iters", out["stat_iters_total"].sum())


if __name__ == "__main__":
    main()

"""Fixtures of the reference's three sample models (run here, where the
reference tree is present; the GPU box reads only the .npz files it writes).

    python tests/golden/make_sample_models.py [REFERENCE_ROOT]

For each of SampleModels/{Lake_T_HYD_WQ, Lake_Washington, Ohio_River_4} it
reads
  * cell.inp   the cell-type map IJCT (5 water, 9 land, 0 outside),
  * dxdy.inp   per water cell I, J, DX, DY, DEPTH, bottom ELEV, ZROUGH,
  * efdc.inp   C3 (RSQM, ITERM), C5 (ISDRY, the sign only selects a report),
               C7 (NTSPTC, NDRYSTP), C8 (TCON, TBEGIN), C11 (HDRY), C19 (the
               west elevation-boundary cells and their ISPBW), C24 (the flow
               source cells, their series and QSFACTOR),
  * qser.inp   each flow series, interpolated at TBEGIN, times QSFACTOR,
  * pser.inp   the first elevation series at TBEGIN (the west boundary head),
and writes tests/golden/sample_<model>.npz with those values.  The arrays
are the models' own grids and bathymetry: irregular shorelines, islands and
a long narrow reach, which the seeded rectangles of the other tests do not
have.  What the step needs beyond them (time step, wind) is set by
scenario.sample_model, and the tests say so.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
MODELS = ("Lake_T_HYD_WQ", "Lake_Washington", "Ohio_River_4")


def _data_lines(path):
    return [ln for ln in Path(path).read_text(errors="replace").splitlines()
            if ln.strip() and not ln.lstrip().upper().startswith("C ") and ln[:1] not in "Cc*-"]


def read_cell(path):
    """cell.inp: 'C' header lines, then one line per row J (top first):
    J in columns 1-3, the IC cell types from column 6 on."""
    lines = Path(path).read_text().splitlines()
    rows = {}
    ic = 0
    for ln in lines:
        if not ln.strip() or ln[0] in "Cc":
            continue
        j = int(ln[:3])
        t = ln[5:].rstrip()
        rows[j] = t
        ic = max(ic, len(t))
    jc = max(rows)
    ijct = np.zeros((jc, ic), np.int8)
    for j, t in rows.items():
        ijct[j - 1, :len(t)] = [int(c) for c in t]
    return ijct


def read_dxdy(path):
    """dxdy.inp: I J DX DY DEPTH ELEV ZROUGH [TYPE]."""
    out = []
    for ln in Path(path).read_text().splitlines():
        if not ln.strip() or ln[0] in "Cc":
            continue
        v = ln.split()
        out.append((int(v[0]), int(v[1]), float(v[2]), float(v[3]), float(v[4]), float(v[5]),
                    float(v[6])))
    return out


def card(lines, name, nrows=1):
    """The first `nrows` data rows that follow the header line of card `name`
    (its last line starting with the card name: the column titles; the first
    one is the card's description)."""
    k = max(i for i, ln in enumerate(lines) if ln.split()[:1] == [name])
    rows = []
    for ln in lines[k + 1:]:
        if ln.startswith("C") or ln.startswith("-"):
            if rows or ln.startswith("C"):
                break
            continue
        if ln.startswith("*"):
            continue
        rows.append(ln.split("!")[0].split())
        if len(rows) == nrows:
            break
    return rows


def read_series(path, kc):
    """qser.inp / pser.inp: per series a header 'InType M TC TA RMUL ADD ...',
    (InType 1: a line of KC depth weights), then M lines of time and value(s).
    Returns a list of (times in days, values summed over layers)."""
    toks = [ln.split("!")[0].split() for ln in Path(path).read_text().splitlines()
            if ln.strip() and ln.lstrip()[:1] not in "Cc"]
    out, k = [], 0
    while k < len(toks):
        h = toks[k]
        intype, m, tc, ta = int(h[0]), int(h[1]), float(h[2]), float(h[3])
        rmul, add = float(h[4]), float(h[5])
        k += 1
        if intype == 1 and "pser" not in Path(path).name:
            k += 1  # depth weights
        t = np.empty(m)
        v = np.empty(m)
        for i in range(m):
            row = [float(x) for x in toks[k + i]]
            t[i] = (row[0] + ta) * tc / 86400.0
            v[i] = (sum(row[1:]) if intype == 0 and len(row) > 2 else row[1]) * rmul + add
        k += m
        out.append((t, v))
    return out


def at(series, day):
    t, v = series
    return float(np.interp(day, t, v))


def make(ref: Path, model: str) -> dict:
    d = ref / "SampleModels" / model
    ijct = read_cell(d / "cell.inp")
    jc, ic = ijct.shape
    cells = read_dxdy(d / "dxdy.inp")
    dxp = np.zeros((jc, ic))
    dyp = np.zeros((jc, ic))
    dep = np.zeros((jc, ic))
    elev = np.zeros((jc, ic))
    zr = np.zeros((jc, ic))
    for i, j, dx, dy, h, e, z in cells:
        dxp[j - 1, i - 1], dyp[j - 1, i - 1] = dx, dy
        dep[j - 1, i - 1], elev[j - 1, i - 1], zr[j - 1, i - 1] = h, e, z
    lines = (d / "efdc.inp").read_text(errors="replace").splitlines()
    c3 = card(lines, "C3")[0]
    c5 = card(lines, "C5")[0]
    c7 = card(lines, "C7")[0]
    c8 = card(lines, "C8")[0]
    c9 = card(lines, "C9")[0]
    c11 = card(lines, "C11")[0]
    c16 = card(lines, "C16")[0]
    npbw = int(c16[1])
    west = card(lines, "C19", npbw) if npbw else []
    c23 = card(lines, "C23")[0]
    nqsij = int(c23[0])
    src = card(lines, "C24", nqsij) if nqsij else []
    tcon, tbegin = float(c8[0]), float(c8[1])
    ntsptc = int(c7[1])
    kc = 1
    qser = read_series(d / "qser.inp", kc) if (d / "qser.inp").exists() else []
    q = []
    for r in src:
        i, j, ns, fac = int(r[0]), int(r[1]), int(r[5]), float(r[14])
        q.append((i, j, at(qser[ns - 1], tbegin) * fac if ns > 0 else float(r[2])))
    head = np.nan
    if npbw and (d / "pser.inp").exists():
        head = at(read_series(d / "pser.inp", kc)[0], tbegin)
    for i, j, _q in q:
        assert ijct[j - 1, i - 1] == 5, (model, i, j)
    return dict(
        ijct=ijct, dxp=dxp, dyp=dyp, depth=dep, belv=elev, zrough=zr,
        rsqm=float(c3[1]), iterm=int(c3[2]), isdry=abs(int(c5[4])), hdry=float(c11[9]),
        ndrystp=int(c7[10]), dt_reference=tcon / ntsptc, tbegin=tbegin,
        lc_reference=int(c9[2]),
        west=np.array([[int(r[0]), int(r[1]), int(r[2])] for r in west], np.int32).reshape(-1, 3),
        west_head=head,
        sources=np.array(q, np.float64).reshape(-1, 3),
    )


def main():
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    for m in MODELS:
        f = make(ref, m)
        nw = int(((f["ijct"] > 0) & (f["ijct"] < 9)).sum())
        assert nw + 2 == f["lc_reference"], (m, nw, f["lc_reference"])
        np.savez_compressed(HERE / f"sample_{m}.npz", **f)
        print(m, f["ijct"].shape, "water cells", nw, "RSQM", f["rsqm"], "ITERM", f["iterm"],
              "ISDRY", f["isdry"], "HDRY", f["hdry"], "sources", len(f["sources"]),
              "west BC", len(f["west"]), "head", f["west_head"])


if __name__ == "__main__":
    main()

"""CPU checks of the oracle (the FP64 C++ restatement of CALPUV2C/CONGRAD).

The reference ships no tests or golden vectors for this path and cannot be
built here, so the oracle is pinned by independent properties instead:
a direct sparse solve of the system it assembles, a lake at rest, mirror
symmetry, the volume budget, thread-count invariance (the reference's own
claim, docs/computer_implementation/started/running.rst:37), and regression
against the committed fixtures in tests/golden/.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import cases
import efdc_xm as X
import oracle as O
import scenario as S


def assemble_matrix(grid, st, la):
    """Sparse A and b of the scaled system CONGRAD solves (congrad.f90:54-77)."""
    n = la - 1
    rows, cols, vals = [], [], []
    for key, nb in (("ccc", None), ("ccs", "lsc"), ("ccn", "lnc"), ("ccw", "lwc"), ("cce", "lec")):
        v = st[key][1:la]
        r = np.arange(n)
        if nb is None:
            c = r
        else:
            c = grid[nb][1:la] - 2
        ok = (c >= 0) & (c < n) & (v != 0)
        rows.append(r[ok]); cols.append(c[ok]); vals.append(v[ok])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    return A, st["fptmp"][1:la].copy()


@pytest.mark.parametrize("name", cases.GOLDEN)
def test_golden_regression(name):
    scn, steps, tm = cases.build(name)
    st, stats = O.run(scn, steps, lists=True, tn_mul=tm)
    g = np.load(cases_path(name))
    for k in g.files:
        if k.startswith("state_"):
            np.testing.assert_array_equal(st[k[6:]], g[k], err_msg=f"{name}:{k}")
    np.testing.assert_array_equal([s["iters_total"] for s in stats], g["stat_iters_total"])
    np.testing.assert_array_equal([s["solves"] for s in stats], g["stat_solves"])
    np.testing.assert_array_equal(st["lwet"][: stats[-1]["lawet"]], g["lwet"][: stats[-1]["lawet"]])


def cases_path(name):
    from pathlib import Path
    return Path(__file__).resolve().parent / "golden" / f"{name}.npz"


@pytest.mark.parametrize("name", ["basin_fp64", "radiation_all_sides", "noise_forcing"])
def test_cg_agrees_with_direct_solve(name):
    """CONGRAD's result satisfies RSQ <= RSQM and matches spsolve of the same
    assembled system to the accuracy that RSQM allows."""
    scn, _, tm = cases.build(name)
    st = scn.copy_state()
    orc = O.Oracle(scn.grid)
    p_in = st["p"].copy()
    prm = X.make_params(scn.params, n=1, tn=scn.tn(1) * tm)
    orc.step(prm, st, diag=True)
    A, b = assemble_matrix(scn.grid, st, scn.la)
    x_direct = spla.spsolve(A.tocsc(), b)
    ccci = np.zeros_like(st["ccc"])
    ccci[1:scn.la] = 1.0 / st["ccc"][1:scn.la]
    p = p_in.copy()
    rc, it, rsq = orc.congrad(st["ccc"], st["ccs"], st["ccn"], st["ccw"], st["cce"], ccci,
                              st["fptmp"], p, scn.params["rsqm"], scn.params["iterm"])
    assert rc == 0 and it > 0
    x = p[1:scn.la]
    res = b - A @ x
    assert float(res @ res) <= scn.params["rsqm"] * 1.000001
    # |x - x*| <= |A^-1| |r|; the scaled operator has smallest eigenvalue >= ~0.1 here
    lam_min = spla.eigsh(A.tocsc(), k=1, sigma=0, which="LM", return_eigenvectors=False)[0] \
        if (A != A.T).nnz == 0 else 0.1
    bound = np.sqrt(scn.params["rsqm"]) / max(lam_min, 1e-3)
    assert np.abs(x - x_direct).max() <= bound


def test_lake_at_rest_stays_at_rest():
    """Flat surface, no forcing, open boundary at the same level: nothing moves
    and CONGRAD returns at RPCG == 0 (congrad.f90:88)."""
    scn = S.make_scenario(40, 30, seed=21, amp=0.0, manning=0.0, datum=0.0, dt=10.0)
    st = scn.copy_state()
    p0 = st["p"].copy()
    out, stats = O.run(scn, 5, state=st)
    assert all(s["iters_total"] == 0 for s in stats)
    np.testing.assert_array_equal(out["p"], p0)
    assert np.all(out["uhdye"] == 0) and np.all(out["vhdxe"] == 0)


def test_lake_at_rest_with_datum():
    """Same at a 120 m datum: rounding of P=G*(HP+BELV) may leave a residual,
    but the surface stays flat to 1e-9 m."""
    scn = S.make_scenario(40, 30, seed=22, amp=0.0, manning=0.0, datum=120.0, dt=10.0)
    out, _ = O.run(scn, 5)
    eta = out["p"][1:scn.la] / S.G
    assert np.abs(eta - 120.0).max() < 1e-9


def test_mirror_symmetry():
    """A basin symmetric about its middle row stays symmetric (to roundoff of
    the differently ordered sums)."""
    nx, ny = 50, 31
    rng = np.random.default_rng(5)
    half = rng.random((ny // 2 + 1, nx)) < 0.05
    land = np.concatenate([half, half[-2::-1]], axis=0)
    f = rng.random((ny // 2 + 1, nx))
    dep = 3.0 + 20.0 * np.concatenate([f, f[-2::-1]], axis=0)
    belv = np.zeros((ny + 2, nx + 2))
    belv[1:-1, 1:-1] = -dep
    belv[0, 1:-1] = belv[1, 1:-1]
    belv[-1, 1:-1] = belv[-2, 1:-1]
    belv[:, 0] = belv[:, 1]
    belv[:, -1] = belv[:, -2]
    scn = S.make_scenario(nx, ny, seed=23, land_mask=land, belv2d=belv, amp=0.5, manning=0.0,
                          dt=20.0)
    out, _ = O.run(scn, 20, tn_mul=10.0)
    jc, ic = scn.jc, scn.ic
    eta = np.full((jc, ic), np.nan)
    il, jl = scn.grid["il"][1:scn.la] - 1, scn.grid["jl"][1:scn.la] - 1
    eta[jl, il] = out["p"][1:scn.la] / S.G
    mirrored = eta[::-1, :]
    ok = ~np.isnan(eta)
    assert np.array_equal(ok, ~np.isnan(mirrored))
    assert np.abs(eta[ok] - mirrored[ok]).max() < 1e-10


def test_volume_budget_closed_basin():
    """No open boundary: the change of sum(DXYP*HP) equals DT*sum(QSUME)
    (the continuity of calpuv2c.f90:466-486 telescopes), 1e-10 relative."""
    scn = S.make_scenario(60, 40, seed=24, obc_sides=(), manning=0.02, dt=10.0,
                          explicit_noise=1e-4)
    st = scn.copy_state()
    dxyp = scn.grid["dxyp"][1:scn.la]
    v0 = float(np.sum(dxyp * st["hp"][1:scn.la]))
    src = 0.0
    orc = O.Oracle(scn.grid)
    for n in range(1, 21):
        orc.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), st)
        src += scn.params["dt"] * float(np.sum(st["qsume"][1:scn.la]))
    v1 = float(np.sum(dxyp * st["hp"][1:scn.la]))
    assert abs((v1 - v0) - src) / v0 < 1e-10


def test_thread_count_invariance():
    """Results are bit-identical for 1 and 4 OpenMP threads (serial dots)."""
    scn, steps, tm = cases.build("noise_forcing")
    a, sa = O.run(scn, steps, nthreads=1, tn_mul=tm)
    b, sb = O.run(scn, steps, nthreads=4, tn_mul=tm)
    for k in ("p", "hp", "uhdye", "vhdxe", "hu", "hv"):
        np.testing.assert_array_equal(a[k], b[k])
    assert sa == sb
    scn, steps, tm = cases.build("tidal_flat_99")
    a, sa = O.run(scn, steps, nthreads=1, tn_mul=tm)
    b, sb = O.run(scn, steps, nthreads=3, tn_mul=tm)
    for k in ("p", "hp", "sub", "svb", "lmaskdry", "iscdry"):
        np.testing.assert_array_equal(a[k], b[k])


def test_noptimal_rule():
    """NOPTIMAL = MIN(NTHREADS, 8, MAX(LA/100,1)) (calpuv2c.f90:61)."""
    scn = S.config1()
    assert O.Oracle(scn.grid, nthreads=16).noptimal == 8
    assert O.Oracle(scn.grid, nthreads=3).noptimal == 3
    small = S.make_scenario(10, 8, seed=1)
    assert O.Oracle(small.grid, nthreads=8).noptimal == max(small.la // 100, 1)


def test_cg_maxiter_status():
    """ITERM exceeded is reported (the reference STOPs, congrad.f90:171-184)."""
    scn, _, tm = cases.build("basin_fp64")
    scn.params["iterm"] = 2
    _, stats = O.run(scn, 1, tn_mul=tm)
    assert stats[0]["status"] == X.CG_MAXITER


def test_wetdry_flat_toggles_and_closes_faces():
    scn, steps, tm = cases.build("tidal_flat_99")
    st, stats = O.run(scn, steps, tn_mul=tm)
    assert max(s["solves"] for s in stats) > 1  # wet/dry re-solves happened
    dry = st["lmaskdry"][1:scn.la] == 0
    assert 0 < dry.sum() < scn.la - 1
    # a dry cell has all four faces closed
    L = np.nonzero(dry)[0] + 2
    lec = scn.grid["lec"][L - 1]
    lnc = scn.grid["lnc"][L - 1]
    assert np.all(st["sub"][L - 1] < 0.5) and np.all(st["sub"][lec - 1] < 0.5)
    assert np.all(st["svb"][L - 1] < 0.5) and np.all(st["svb"][lnc - 1] < 0.5)

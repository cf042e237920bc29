"""Explicit momentum producer: CALEXP2T's external-mode terms on the device
(efdc_xm_set_momentum / efdc_xm_explicit_batch) against the oracle's
restatement of calexp2t.f90:129-956.

CPU tests pin properties of the oracle's restatement (no flow gives no
forcing, a uniform flow gives no flux divergence away from the edges, cells
outside the wet set hold zero, the type-2 forms replace the interior ones).
GPU tests: every output bit for bit against the oracle (the device kernels
round in the reference's operand order without FMA), over one and several
layers, triangular cells, momentum diffusion, source momentum, type-2 open
boundaries, flow-boundary edges, wet sets that change between calls, and a
batch; and the sums left on the device feed the next step as the host's
arrays would.
"""
import numpy as np
import pytest

import cases
import efdc_xm as X
import oracle as O
import scenario as S

LAYER = ("fcax", "fcay", "fx", "fy", "cac")
SUMS = ("fcaxe", "fcaye", "fxe", "fye")


def setup(name="noise_forcing", kc=1, **kw):
    scn = cases.build(name)[0]
    S.add_momentum(scn, kc=kc, seed=kc, **kw)
    return scn


def oracle_call(scn, f, prm):
    o = O.Oracle(scn.grid)
    o.set_momentum(scn.momentum)
    assert o.explicit(prm, f) == 0
    o.close()
    return f


# ---------------------------------------------------------------- CPU, oracle
def test_oracle_no_flow_no_forcing():
    scn = setup(kc=2)
    f = S.momentum_fields(scn, u_scale=0.0)
    oracle_call(scn, f, X.make_explicit_params(1.0, 1, 0))
    for k in SUMS + ("fx", "fy", "fcax", "fcay"):
        assert np.abs(f[k]).max() == 0.0, k
    # the Coriolis coefficient itself is FCORC*DXYP*HP
    la = scn.la
    want = scn.momentum["fcorc"][1:la] * scn.grid["dxyp"][1:la] * scn.state["hp"][1:la]
    np.testing.assert_allclose(f["cac"][0, 1:la], want, rtol=1e-15)


def test_oracle_uniform_flow_no_divergence_inside():
    """U uniform, V = 0, UHDY uniform: FUHU is the same on both faces of an
    interior cell and FVHU vanishes, so FX is 0 where all four neighbours and
    the diagonals are wet water cells."""
    scn = setup(kc=1, nbcs=0)
    f = S.momentum_fields(scn, u_scale=0.0)
    la = scn.la
    f["u"][:, 1:la] = 0.3
    f["uhdy"][:, 1:la] = 0.3 * 100.0 * 5.0
    oracle_call(scn, f, X.make_explicit_params(1.0, 0, 0))
    g = scn.grid
    inner = [L for L in range(2, la + 1)
             if all(2 <= g[k][L - 1] <= la for k in ("lec", "lwc", "lnc", "lsc"))
             and all(2 <= g[k][g[j][L - 1] - 1] <= la
                     for k in ("lec", "lwc", "lnc", "lsc") for j in ("lec", "lwc", "lnc", "lsc"))]
    assert len(inner) > 100
    idx = np.array(inner) - 1
    assert np.abs(f["fx"][0, idx]).max() == 0.0
    assert np.abs(f["fxe"][idx]).max() == 0.0


def test_oracle_dry_cells_hold_zero():
    scn = setup(kc=2, nbcs=0)
    f = S.momentum_fields(scn, seed=3, wet_frac=0.8)
    oracle_call(scn, f, X.make_explicit_params(1.0, 1, 0))
    dry = np.where(f["wet"][1:scn.la] == 0)[0] + 1
    assert dry.size > 10
    for k in SUMS:
        assert np.abs(f[k][dry]).max() == 0.0, k
    for k in LAYER:
        assert np.abs(f[k][:, dry]).max() == 0.0, k


def test_oracle_type2_west_form():
    """A type-2 west boundary: the cell after each boundary cell takes
    FCAX = 0.5*SCAX*CAC*(V(LN)+V(L)) (calexp2t.f90:607-614)."""
    scn = setup(kc=1, type2=("W",), nbcs=0)
    f = S.momentum_fields(scn, seed=4)
    oracle_call(scn, f, X.make_explicit_params(1.0, 1, 0))
    g, mo = scn.grid, scn.momentum
    for LB in g["obc"]["W"]["l"]:
        L = int(LB) + 1
        LN = int(g["lnc"][L - 1])
        want = 0.5 * mo["scax"][L - 1] * f["cac"][0, L - 1] * (f["v"][0, LN - 1] + f["v"][0, L - 1])
        assert f["fcax"][0, L - 1] == want


# ---------------------------------------------------------------- GPU parity
CASES = {
    "one_layer": dict(name="noise_forcing", kc=1, mo={}, fl={}),
    "layers_tri_hdmf_sources": dict(name="noise_forcing", kc=3, mo=dict(tri=True, hdmf=True),
                                    fl=dict(fuhj=True, hdmf=True), ishdmf=1),
    "type2_ew_dry": dict(name="radiation_all_sides", kc=2, mo=dict(type2=("E", "W", "S", "N")),
                         fl=dict(wet_frac=0.85)),
    "flat_no_curvature": dict(name="tidal_flat_99", kc=1, mo={}, fl=dict(wet_frac=0.7), curv=0),
}


def run_gpu(scn, fields, prm, sol=None):
    own = sol is None
    sol = sol or X.Solver(scn.grid)
    if own:
        sol.set_momentum(scn.momentum)
    sol.explicit(prm, fields)
    if own:
        sol.close()
    return fields


def compare(a, b, la, kc):
    for k in SUMS:
        np.testing.assert_array_equal(a[k][1:la], b[k][1:la], err_msg=k)
    for k in LAYER:
        np.testing.assert_array_equal(a[k][:kc, 1:la], b[k][:kc, 1:la], err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_gpu_explicit_bit_exact(case):
    X.load()
    c = CASES[case]
    scn = setup(c["name"], c["kc"], **c["mo"])
    prm = X.make_explicit_params(1.0, c.get("curv", 1), c.get("ishdmf", 0))
    fo = S.momentum_fields(scn, seed=5, **c["fl"])
    fg = {k: v.copy() for k, v in fo.items()}
    oracle_call(scn, fo, prm)
    run_gpu(scn, fg, prm)
    assert np.abs(fo["fxe"][1:scn.la]).max() > 0
    compare(fg, fo, scn.la, c["kc"])


@pytest.mark.gpu
def test_gpu_explicit_calls_with_changing_wet_set():
    """Five calls on one context and one oracle, the wet set redrawn each
    time (newly dry cells are zeroed, rewetted cells recomputed)."""
    X.load()
    scn = setup("noise_forcing", 2, hdmf=True)
    prm = X.make_explicit_params(1.0, 1, 1)
    sol = X.Solver(scn.grid)
    sol.set_momentum(scn.momentum)
    o = O.Oracle(scn.grid)
    o.set_momentum(scn.momentum)
    fo = S.momentum_fields(scn, seed=0, wet_frac=0.8, hdmf=True)
    fg = {k: v.copy() for k, v in fo.items()}
    for n in range(5):
        new = S.momentum_fields(scn, seed=n, wet_frac=0.8, hdmf=True)
        for k in ("u", "v", "uhdy", "vhdx", "wet", "fmdux", "fmduy", "fmdvx", "fmdvy"):
            fo[k] = new[k]
            fg[k] = new[k].copy()
        assert o.explicit(prm, fo) == 0
        sol.explicit(prm, fg)
        compare(fg, fo, scn.la, 2)
    sol.close()
    o.close()


@pytest.mark.gpu
def test_gpu_explicit_batch_equals_oracle_per_member():
    X.load()
    scns = [setup("noise_forcing", 2, tri=True), setup("radiation_all_sides", 2, type2=("E",))]
    prm = [X.make_explicit_params(1.0, 1, 0), X.make_explicit_params(0.5, 1, 0)]
    fo = [S.momentum_fields(s, seed=7 + m, wet_frac=0.9, fuhj=True) for m, s in enumerate(scns)]
    fg = [{k: v.copy() for k, v in f.items()} for f in fo]
    for s, f, p in zip(scns, fo, prm):
        oracle_call(s, f, p)
    bs = X.BatchSolver([s.grid for s in scns])
    for m, s in enumerate(scns):
        bs.set_momentum(s.momentum, m)
    bs.explicit(prm, fg)
    bs.close()
    for s, a, b in zip(scns, fg, fo):
        compare(a, b, s.la, 2)


@pytest.mark.gpu
def test_gpu_sums_stay_on_device_for_the_step():
    """The producer's sums kept on the device (outputs NULL) and a step given
    no FCAXE, FCAYE, FXE, FYE step exactly as the host arrays would: the same
    CG iterations and surface as the oracle fed the oracle's sums."""
    X.load()
    scn = setup("noise_forcing", 1)
    prm = X.make_explicit_params(1.0, 1, 0)
    sol = X.Solver(scn.grid)
    sol.set_momentum(scn.momentum)
    o = O.Oracle(scn.grid)
    o.set_momentum(scn.momentum)
    so = cases.copy_state(scn.state)
    sol.upload(scn.state)
    for n in range(1, 6):
        f = S.momentum_fields(scn, seed=n)
        f["hp"] = so["hp"].copy()
        fo = {k: v.copy() for k, v in f.items()}
        for k in SUMS:
            fo[k] = so[k]
        assert o.explicit(prm, fo) == 0
        fg = {k: v for k, v in f.items() if k not in SUMS + LAYER}
        fg.pop("hp")  # the device's HP, which the last step left
        sol.explicit(prm, fg)
        a = sol.step_device(X.make_params(scn.params, n=n, tn=scn.tn(n)))
        b = o.step(X.make_params(scn.params, n=n, tn=scn.tn(n)), so)
        assert a.status == b.status == X.OK
        assert a.iters_total == b.iters_total, n
    out = {"p": np.zeros_like(so["p"])}
    sol.download(out)
    assert np.abs(out["p"][1:scn.la] - so["p"][1:scn.la]).max() / S.G < 1e-9
    sol.close()
    o.close()

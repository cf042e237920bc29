"""Seeded scenario cases shared by the CPU and GPU tests (small sizes)."""
from __future__ import annotations

import numpy as np

import scenario as S

# name -> (builder, steps, tidal-time multiplier)
GOLDEN = ("basin_fp64", "radiation_all_sides", "tidal_flat_99", "legacy_dry_1", "noise_forcing")


def build(name):
    if name == "basin_fp64":  # config-1 layout, 12 steps
        return S.config1(seed=11), 12, 1.0
    if name == "radiation_all_sides":
        scn = S.make_scenario(48, 36, seed=12, obc_sides=("W", "E", "S", "N"), ispb=1,
                              amp=0.3, dt=20.0, land_frac=0.05, explicit_noise=1e-4)
        return scn, 10, 20.0
    if name == "tidal_flat_99":
        return S.tidal_flat(n=48, seed=13, dt=5.0), 40, 60.0
    if name == "legacy_dry_1":
        scn = S.tidal_flat(n=40, seed=14, dt=5.0)
        scn.params["isdry"] = 1
        scn.params["ndrystp"] = 0
        return scn, 30, 60.0
    if name == "noise_forcing":  # clamped W + radiation E, explicit terms
        scn = S.make_scenario(60, 40, seed=15, obc_sides=("W",), amp=0.4, dt=10.0,
                              explicit_noise=3e-4, datum=35.0, snlt=1.0)
        return scn, 10, 10.0
    if name == "radiation_closed_face":  # unsymmetric operator, see unsymmetric()
        return unsymmetric(), 6, 20.0
    raise KeyError(name)


def unsymmetric():
    """A radiation-boundary basin whose operator is unsymmetric: the interior
    faces behind three west boundary cells are closed in the state (SUB = 0,
    as drying leaves them while the static HRUO stays open).  CALPUV2C then
    gives CW(LE) = 0 while SETOPENBC's radiation row keeps CE(L) = -CET
    (setopenbc.f90:67-80), so CE(L) /= CW(LE) at those three faces."""
    scn = S.make_scenario(40, 30, seed=16, obc_sides=("W", "E"), ispb=1, amp=0.3, dt=20.0,
                          land_frac=0.03, explicit_noise=1e-4)
    lw = scn.grid["obc"]["W"]["l"]
    lec = scn.grid["lec"]
    for L in lw[5:8]:
        scn.state["sub"][lec[L - 1] - 1] = 0.0
    return scn


def channels(consistent=0, *, closed=False, qcherr=1.0, n=10, seed=21):
    """A basin with `n` sub-grid channels (x- and y-direction, guests within
    3 cells of their hosts).  With closed=True it has no open boundary and is
    driven by its explicit terms only (its volume is constant).
    `consistent` selects the channel operator (chan_consistent)."""
    scn = S.make_scenario(60, 40, seed=seed, obc_sides=() if closed else ("W",), amp=0.5,
                          dt=10.0, explicit_noise=3e-4)
    S.add_channels(scn, n, seed=3, qcherr=qcherr)
    scn.params["chan_consistent"] = consistent
    return scn


def baroclinic(wetdry=False, *, closed=False, kc=4):
    """A basin with the baroclinic terms (BSC = 1, KC sigma layers, a seeded
    buoyancy front).  wetdry=True: the ISDRY=99 tidal flat instead, so that
    the buoyancy integrals skip the cells that were dry at the last step."""
    if wetdry:
        scn = S.tidal_flat(n=48, seed=13, dt=5.0)
    else:
        scn = S.make_scenario(60, 40, seed=31, obc_sides=() if closed else ("W",), amp=0.3,
                              dt=10.0, explicit_noise=1e-4)
    S.add_baroclinic(scn, kc, seed=2)
    return scn


def copy_state(st):
    return {k: (v.copy() if isinstance(v, np.ndarray) else
                {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
            for k, v in st.items()}


def run_both(scn, steps, tm=1.0, precision=None, same_input=False, lists=False, n0=1,
             nthreads=1, keep=None, oracle_rsqm_scale=1.0):
    """Run the GPU library (efdc_xm_step on host arrays) and the oracle side by
    side for `steps` steps.  Returns one (gpu stats, oracle stats, gpu state,
    oracle state) tuple per step; `keep(n)` selects the steps whose states are
    kept (default: all).  same_input=True starts every GPU step from the
    oracle's state.  oracle_rsqm_scale scales the oracle's RSQM (a tighter
    FP64 solve as the reference solution of the same system)."""
    import efdc_xm as X
    import oracle as O
    precision = X.PREC_FP64 if precision is None else precision
    sol = X.Solver(scn.grid)
    orc = O.Oracle(scn.grid, nthreads=nthreads)
    sg, so = copy_state(scn.state), copy_state(scn.state)
    out = []
    for n in range(n0, n0 + steps):
        if same_input:
            sg = copy_state(so)
        prm = X.make_params(scn.params, n=n, tn=scn.tn(n) * tm, precision=precision)
        a = sol.step(prm, sg, lists=lists)
        po = X.make_params(scn.params, n=n, tn=scn.tn(n) * tm)
        po.rsqm *= oracle_rsqm_scale
        b = orc.step(po, so, lists=lists)
        k = keep is None or keep(n)
        out.append((a.as_dict(), b.as_dict(), copy_state(sg) if k else None,
                    copy_state(so) if k else None))
    sol.close()
    orc.close()
    return out


def state_err(a, b, la, key="p", g=S.G):
    d = np.abs(a[key][1:la] - b[key][1:la])
    return float(d.max() / (g if key == "p" else 1.0))

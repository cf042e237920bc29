"""The FP64 torch reference of the calibration model (oracle/adjoint_ref.py)
against central finite differences of itself (CPU): the reference that the
GPU adjoint is checked against is itself checked here."""
import math

import numpy as np
import pytest
import torch

import adjoint_ref as R
import scenario as S


def small(seed=21):
    scn = S.make_scenario(14, 10, seed=seed, land_frac=0.05, depth=(2.0, 12.0), obc_sides=("W",),
                          amp=0.4, manning=0.0, dt=10.0, isdry=0, fill_dead_ends=True)
    rng = np.random.default_rng(seed)
    log_n = np.full(scn.lc + 1, math.log(0.025))
    log_n[1:scn.la] = rng.normal(math.log(0.025), 0.2, scn.la - 1)
    gauges = np.array([scn.la // 3, scn.la // 2, scn.la - 2], dtype=np.int32)
    return scn, log_n, gauges


def test_reference_gradient_matches_central_differences():
    scn, log_n, gauges = small()
    m = R.RefModel(scn.grid, scn.params, scn.state)
    nb = len(m.bc)
    pcb0 = np.concatenate([np.asarray(scn.grid["obc"][s]["pcb"]).T for s in R.SIDES])
    psb0 = np.concatenate([np.asarray(scn.grid["obc"][s]["psb"]).T for s in R.SIDES])
    assert pcb0.shape == (nb, 1)
    obs = np.zeros((6, len(gauges)))
    k = torch.tensor(log_n, requires_grad=True)
    pc = torch.tensor(pcb0, requires_grad=True)
    ps = torch.tensor(psb0, requires_grad=True)
    loss, _ = m.loss(k, pc, ps, 6, gauges, obs)
    loss.backward()
    rng = np.random.default_rng(3)
    h = 1e-4

    def L(kk, pp):
        with torch.no_grad():
            return float(m.loss(torch.tensor(kk), torch.tensor(pp), torch.tensor(psb0), 6, gauges,
                                obs)[0])

    v = np.zeros_like(log_n)
    v[1:scn.la] = rng.standard_normal(scn.la - 1)
    fd = (L(log_n + h * v, pcb0) - L(log_n - h * v, pcb0)) / (2 * h)
    an = float((k.grad.numpy() * v).sum())
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
    w = rng.standard_normal(pcb0.shape)
    fd = (L(log_n, pcb0 + h * w) - L(log_n, pcb0 - h * w)) / (2 * h)
    an = float((pc.grad.numpy() * w).sum())
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)


def test_reference_rejects_radiation_boundaries():
    scn = S.make_scenario(10, 8, seed=2, obc_sides=("W",), ispb=1, manning=0.0)
    with pytest.raises(ValueError):
        R.RefModel(scn.grid, scn.params, scn.state)

"""Checkpointed forward/reverse runs of the calibration model on one GPU.

The model: EFDC+'s external mode (CALPUV2C, ISDRY=0, clamped open
boundaries) with a Manning bottom drag written each step from a per-cell
log n (see include/efdc_xm.h, "Calibration").  Parameters: log n per cell
and one tidal amplitude per group of open-boundary cells (the constituents'
phases fixed).  Loss: sum over steps and gauges of (eta - eta_observed)^2,
eta = P/G after the step.

Memory: a snapshot of the state every `every` steps during the forward run;
the reverse run recomputes one segment of `every` steps at a time from its
snapshot, keeping one snapshot per step of the segment.
"""
from __future__ import annotations

import numpy as np
import torch

import efdc_xm as X

SIDES = ("W", "E", "S", "N")


def boundary_groups(grid: dict, ngroups: int) -> np.ndarray:
    """Group index of every open-boundary cell (packed W, E, S, N order):
    contiguous runs along the boundary, ngroups of them."""
    n = sum(len(grid["obc"][s]["l"]) for s in SIDES)
    return (np.arange(n) * ngroups) // max(n, 1)


class CalibProblem:
    def __init__(self, scn, gauges, nsteps, *, ngroups=4, every=20, device=0,
                 adj_rel_tol=1e-12, rsqm=None):
        self.scn = scn
        self.gauges = np.ascontiguousarray(gauges, dtype=np.int32)
        self.nsteps = int(nsteps)
        self.every = int(every)
        self.nseg = (self.nsteps + self.every - 1) // self.every
        self.adj_rel_tol = adj_rel_tol
        self.params = dict(scn.params)
        if rsqm is not None:
            self.params["rsqm"] = rsqm
        g = scn.grid
        self.mt = int(g["mtide"])
        self.groups = boundary_groups(g, ngroups)
        self.ngroups = ngroups
        # unit harmonics per boundary cell: PCB = G*a*cos(phase), PSB = G*a*sin(phase)
        pcb = np.concatenate([np.asarray(g["obc"][s]["pcb"]).T for s in SIDES]).reshape(-1, self.mt)
        psb = np.concatenate([np.asarray(g["obc"][s]["psb"]).T for s in SIDES]).reshape(-1, self.mt)
        amp = np.hypot(pcb, psb)
        safe = np.where(amp > 0, amp, 1.0)
        G = float(self.params["g"])
        self.ucos = np.where(amp > 0, pcb / safe, 1.0) * G  # d PCB / d amplitude
        self.usin = np.where(amp > 0, psb / safe, 0.0) * G
        self.sol = X.Solver(g, device=device)
        self.sol.calib_enable(self.nseg + self.every)
        self.obs = None
        self.eta = None

    def harmonics(self, amps):
        a = np.asarray(amps, dtype=np.float64)[self.groups][:, None]
        return a * self.ucos, a * self.usin

    def _prm(self, n):
        return X.make_params(self.params, n=n, tn=self.scn.tn(n))

    def forward(self, log_n, amps, *, keep=True):
        """Run the model; returns gauge elevations [nsteps, ngauges]."""
        self.sol.calib_set_roughness(np.asarray(log_n, dtype=np.float64))
        pcb, psb = self.harmonics(amps)
        self.sol.calib_set_harmonics(pcb.ravel(), psb.ravel())
        self.sol.upload(self.scn.state)
        eta = np.zeros((self.nsteps, len(self.gauges)))
        for k in range(self.nsteps):
            if keep and k % self.every == 0:
                self.sol.calib_snapshot(k // self.every)
            st = self.sol.calib_step(self._prm(k + 1))
            if st.status != X.OK:
                raise RuntimeError(f"calibration forward step {k + 1}: status {st.status}")
            eta[k] = self.sol.calib_gauges(self.gauges) / self.params["g"]
        self.eta = eta
        return eta

    def loss(self, log_n, amps):
        eta = self.forward(log_n, amps)
        return float(((eta - self.obs) ** 2).sum())

    def backward(self):
        """Gradient of the loss of the last forward run: (d/dlog n [LC],
        d/damps [ngroups], d/dBELV [LC], adjoint iterations)."""
        if self.eta is None or self.obs is None:
            raise RuntimeError("run forward() with observations first")
        G = self.params["g"]
        sol = self.sol
        sol.calib_adjoint_reset()
        iters = 0
        for seg in reversed(range(self.nseg)):
            k0 = seg * self.every
            k1 = min(k0 + self.every, self.nsteps)
            sol.calib_restore(seg)
            for k in range(k0, k1):  # one snapshot per step of the segment
                sol.calib_snapshot(self.nseg + (k - k0))
                sol.calib_step(self._prm(k + 1))
            for k in reversed(range(k0, k1)):
                w = 2.0 * (self.eta[k] - self.obs[k]) / G
                sol.calib_add_p_adjoint(self.gauges, w)
                iters += sol.calib_adjoint_step(self._prm(k + 1), self.nseg + (k - k0),
                                                self.adj_rel_tol)
        nb = len(self.groups) * self.mt
        dk, db, dpc, dps, _st, ncl = sol.calib_gradients(nb)
        if ncl:
            raise RuntimeError(f"{ncl} open-boundary targets were dry-clamped")
        dpc = dpc.reshape(-1, self.mt)
        dps = dps.reshape(-1, self.mt)
        da = np.zeros(self.ngroups)
        np.add.at(da, self.groups, (dpc * self.ucos + dps * self.usin).sum(axis=1))
        return dk, da, db, iters

    def close(self):
        self.sol.close()


class CalibLoss(torch.autograd.Function):
    """loss = CalibLoss.apply(log_n, amps, problem): the misfit of the
    calibration model; backward runs the adjoint on the GPU."""

    @staticmethod
    def forward(ctx, log_n, amps, problem):
        loss = problem.loss(log_n.detach().cpu().numpy(), amps.detach().cpu().numpy())
        ctx.problem = problem
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        dk, da, _db, _it = ctx.problem.backward()
        g = float(grad_out)
        return (torch.as_tensor(dk * g), torch.as_tensor(da * g), None)

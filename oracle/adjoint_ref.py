"""FP64 reference gradient of the calibration model (TEST INFRASTRUCTURE).

A restatement in torch (CPU, float64) of the calibration model's step and
its loss, differentiated by torch.autograd; it checks the hand-written
adjoint kernels of libefdc_xm (efdc_xm_calib_*).  Small grids only: the
implicit solve is a dense direct solve.  Only tests import this module.

The step (ISDRY=0, clamped open boundaries ISPB=0, one pass):
  drag      TBX = STBX*SQRT(VU^2+U^2)*U, STBX = G*n_u^2/HU^(1/3) (the form of
            EFDC/hdmt2t.f90:682 with AVCON1=0, Manning drag coefficient)
  begin     EFDC/calpuv2c.f90:214-220 (FUHDYE, FVHDXE), :282-290 (FP1)
  assemble  :306-344 (FP, CS, CW, CE, CN, CC)
  open BCs  EFDC/setopenbc.f90:22-206 (clamped), EFDC/setopenbc2.f90:17-46
  solve     A P' = FP (CONGRAD's system, solved exactly here)
  update    :416-437 (UHDYE, VHDXE), :466-486 (HP), :489-535 (boundary HP),
            :560-570 and :896-906 (P = G*(HP+BELV), HU, HV)
loss = sum over steps and gauges of (P/G - observed)^2.
"""
from __future__ import annotations

import math

import numpy as np
import torch

SIDES = ("W", "E", "S", "N")


class RefModel:
    def __init__(self, grid: dict, params: dict, state: dict):
        T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))  # noqa: E731
        g = grid
        self.la, self.lc = int(g["la"]), int(g["lc"])
        la, lc = self.la, self.lc
        self.W = torch.arange(1, la)  # 0-based indices of L = 2..LA
        ix = lambda name: torch.as_tensor(np.asarray(g[name], dtype=np.int64) - 1)  # noqa: E731
        self.lec, self.lwc, self.lnc, self.lsc = ix("lec"), ix("lwc"), ix("lnc"), ix("lsc")
        for k in ("dxyp", "dxyip", "dxiu", "dyiu", "dxiv", "dyiv", "dxyu", "dxyv", "hruo", "hrvo",
                  "subo", "svbo", "belv"):
            setattr(self, k, T(g[k]))
        n = len(g["belv"])
        self.rcx = torch.zeros(n, dtype=torch.float64)
        self.rcx[self.W] = 1.0
        self.fsgzu = torch.ones(n, dtype=torch.float64)
        self.fsgzv = torch.ones(n, dtype=torch.float64)
        self.fsgzu[self.W] = 0.5 / self.dxyu[self.W]
        self.fsgzv[self.W] = 0.5 / self.dxyv[self.W]
        self.sub, self.svb = T(state["sub"]), T(state["svb"])
        self.p = params
        self.G = float(params["g"])
        self.mtide = int(g["mtide"])
        self.tcp = [float(x) for x in np.asarray(g["tcp"])[: self.mtide]]
        # open-boundary cells in the W, E, S, N order of the lists
        self.bc = []
        for s, side in enumerate(SIDES):
            o = g["obc"][side]
            for ll, L in enumerate(np.asarray(o["l"])):
                L = int(L)
                nb = {0: g["lec"], 1: g["lwc"], 2: g["lnc"], 3: g["lsc"]}[s][L - 1]
                if int(np.asarray(o["ispb"])[ll]) != 0:
                    raise ValueError("the reference covers clamped boundaries only")
                self.bc.append((L - 1, int(nb) - 1, s))
        self.pser = np.concatenate([np.asarray(state["pser"][s], dtype=np.float64)
                                    for s in SIDES]) if self.bc else np.zeros(0)
        self.state0 = {k: T(state[k]) for k in ("p", "hp", "hu", "hv", "uhdye", "vhdxe")}
        isbc = np.zeros(n, bool)
        for L, _, _ in self.bc:
            isbc[L] = True
        self.isbc = torch.as_tensor(isbc)

    def _vel(self, uh, h, dyi):
        v = torch.zeros_like(uh)
        W = self.W
        v = v.index_put((W,), uh[W] * dyi[W] / h[W])
        return v

    def step(self, st, kappa, pcb, psb, n):
        """One step from state dict `st`; pcb/psb [nbc, mtide] tensors."""
        P, HP, HU, HV, UH, VH = st["p"], st["hp"], st["hu"], st["hv"], st["uhdye"], st["vhdxe"]
        W, lec, lwc, lnc, lsc = self.W, self.lec, self.lwc, self.lnc, self.lsc
        pr = self.p
        G = self.G
        delt = float(pr["dt"])
        D2 = 0.5 * delt
        delti = 1.0 / delt
        ritb1 = float(pr.get("ritb1", 1.0))
        sub, svb = self.sub, self.svb
        # drag
        U = self._vel(UH, HU, self.dyiu)
        V = self._vel(VH, HV, self.dxiv)
        Wv = W
        VU = 0.25 * (V[Wv] + V[lnc[Wv]] + V[lwc[Wv]] + V[lnc[lwc[Wv]]])
        UV = 0.25 * (U[Wv] + U[lec[Wv]] + U[lsc[Wv]] + U[lec[lsc[Wv]]])
        en = torch.exp(kappa)
        nu = 0.5 * (en[Wv] + en[lwc[Wv]])
        nv = 0.5 * (en[Wv] + en[lsc[Wv]])
        su = torch.sqrt(torch.clamp(VU * VU + U[Wv] * U[Wv], min=1e-300))
        sv = torch.sqrt(torch.clamp(UV * UV + V[Wv] * V[Wv], min=1e-300))
        tbxw = torch.where(self.subo[Wv] > 0.5, G * nu * nu / HU[Wv] ** (1.0 / 3.0) * su * U[Wv],
                           torch.zeros_like(nu))
        tbyw = torch.where(self.svbo[Wv] > 0.5, G * nv * nv / HV[Wv] ** (1.0 / 3.0) * sv * V[Wv],
                           torch.zeros_like(nv))
        z = torch.zeros_like(P)
        tbx = z.index_put((W,), tbxw)
        tby = z.index_put((W,), tbyw)
        # explicit transports and FP1 (calpuv2c.f90:214-220, 282-290)
        fu = z.index_put((W,), UH[W] - D2 * sub[W] * self.hruo[W] * HU[W] * (P[W] - P[lwc[W]])
                         + sub[W] * delt * self.dxiu[W] * (self.dxyu[W] * (-ritb1 * tbx[W])))
        fv = z.index_put((W,), VH[W] - D2 * svb[W] * self.hrvo[W] * HV[W] * (P[W] - P[lsc[W]])
                         + svb[W] * delt * self.dyiv[W] * (self.dxyv[W] * (-ritb1 * tby[W])))
        fp1 = delti * self.dxyp[W] * P[W] - 0.5 * G * (UH[lec[W]] - UH[W] + VH[lnc[W]] - VH[W])
        # assembly (:306-344)
        fp = fp1 - 0.5 * G * (sub[lec[W]] * fu[lec[W]] - sub[W] * fu[W] +
                              svb[lnc[W]] * fv[lnc[W]] - svb[W] * fv[W])
        C1 = -0.5 * D2 * G
        rc = self.rcx
        cs = C1 * svb[W] * self.hrvo[W] * rc[W] * HV[W]
        cw = C1 * sub[W] * self.hruo[W] * rc[W] * HU[W]
        ce = C1 * sub[lec[W]] * self.hruo[lec[W]] * rc[lec[W]] * HU[lec[W]]
        cn = C1 * svb[lnc[W]] * self.hrvo[lnc[W]] * rc[lnc[W]] * HV[lnc[W]]
        cc = delti * self.dxyp[W] - cs - cw - ce - cn
        full = lambda a: z.index_put((W,), a)  # noqa: E731
        FP, CC, CS, CW, CE, CN = full(fp), full(cc), full(cs), full(cw), full(ce), full(cn)
        # open boundaries (setopenbc.f90, clamped; setopenbc2.f90)
        tn = float(pr["dt"]) * float(n)
        pi2 = float(pr["pi2"])
        cosv = [math.cos(pi2 * math.fmod(tn, t) / t) for t in self.tcp]
        sinv = [math.sin(pi2 * math.fmod(tn, t) / t) for t in self.tcp]
        for k, (L, nb, side) in enumerate(self.bc):
            f = torch.as_tensor(self.pser[k], dtype=torch.float64)
            for m in range(self.mtide):
                f = f + pcb[k, m] * cosv[m] + psb[k, m] * sinv[m]
            one = torch.zeros_like(P)
            one[L] = 1.0
            keep = 1.0 - one
            CC = CC * keep + one * (delti * self.dxyp[L])
            CS, CW, CE, CN = CS * keep, CW * keep, CE * keep, CN * keep
            if side == 0:
                CT = 0.5 * D2 * G * self.hruo[nb] * rc[nb] * HU[nb]
            elif side == 1:
                CT = 0.5 * D2 * G * self.hruo[L] * rc[L] * HU[L]
            elif side == 2:
                CT = 0.5 * D2 * G * self.hrvo[nb] * rc[nb] * HV[nb]
            else:
                CT = 0.5 * D2 * G * self.hrvo[L] * rc[L] * HV[L]
            onb = torch.zeros_like(P)
            onb[nb] = 1.0
            FP = FP + onb * (CT * f)
            FP = FP * keep + one * (delti * self.dxyp[L] * f)
            kill = 1.0 - onb
            if side == 0:
                CW = CW * kill
            elif side == 1:
                CE = CE * kill
            elif side == 2:
                CS = CS * kill
            else:
                CN = CN * kill
        # the implicit solve, exactly (dense)
        nw = self.la - 1
        pos = torch.full((len(P),), -1, dtype=torch.int64)
        pos[W] = torch.arange(nw)
        A = torch.zeros((nw, nw), dtype=torch.float64)
        r = torch.arange(nw)
        A = A.index_put((r, r), CC[W])
        for coef, nbr in ((CS, lsc), (CW, lwc), (CE, lec), (CN, lnc)):
            j = pos[nbr[W]]
            ok = j >= 0
            A = A.index_put((r[ok], j[ok]), coef[W][ok], accumulate=True)
        x = torch.linalg.solve(A, FP[W])
        Pn = P.index_put((W,), x)
        # back-substitution, continuity, boundary depths, refresh
        un = full(sub[W] * (fu[W] - D2 * self.hruo[W] * rc[W] * HU[W] * (Pn[W] - Pn[lwc[W]])))
        vn = full(svb[W] * (fv[W] - D2 * self.hrvo[W] * rc[W] * HV[W] * (Pn[W] - Pn[lsc[W]])))
        # ghost elements keep their values
        un = un + UH * (1.0 - full(torch.ones(len(W), dtype=torch.float64)))
        vn = vn + VH * (1.0 - full(torch.ones(len(W), dtype=torch.float64)))
        hpn_w = HP[W] + D2 * self.dxyip[W] * (-(un[lec[W]] + UH[lec[W]] - un[W] - UH[W] +
                                                vn[lnc[W]] + VH[lnc[W]] - vn[W] - VH[W]))
        bcm = self.isbc[W]
        hpn_w = torch.where(bcm, Pn[W] / G - self.belv[W], hpn_w)
        HPn = HP.index_put((W,), hpn_w)
        Pf = P.index_put((W,), G * (hpn_w + self.belv[W]))
        HUn = HU.index_put((W,), (self.dxyp[W] * hpn_w + self.dxyp[lwc[W]] * HPn[lwc[W]]) *
                           self.fsgzu[W])
        HVn = HV.index_put((W,), (self.dxyp[W] * hpn_w + self.dxyp[lsc[W]] * HPn[lsc[W]]) *
                           self.fsgzv[W])
        return {"p": Pf, "hp": HPn, "hu": HUn, "hv": HVn, "uhdye": un, "vhdxe": vn}

    def loss(self, kappa, pcb, psb, nsteps, gauges, obs, belv=None, state=None):
        """sum_n sum_g (P_g/G - obs[n, g])^2 over steps 1..nsteps; also the
        gauge elevations.  gauges: 1-based L."""
        if belv is not None:
            self.belv = belv
        st = dict(state if state is not None else self.state0)
        gi = torch.as_tensor(np.asarray(gauges, dtype=np.int64) - 1)
        total = torch.zeros((), dtype=torch.float64)
        etas = []
        for n in range(1, nsteps + 1):
            st = self.step(st, kappa, pcb, psb, n)
            eta = st["p"][gi] / self.G
            etas.append(eta.detach().numpy().copy())
            if obs is not None:
                total = total + ((eta - torch.as_tensor(obs[n - 1])) ** 2).sum()
        return total, np.array(etas)

"""Seeded synthetic EFDC+ external-mode scenarios.

Builds, from a handful of scalars and a numpy seed, exactly the set of
MODULE GLOBAL arrays that CALPUV2C reads and writes, in EFDC+'s own
1-based cell order (element L of a Fortran array is at index L-1 here; every
per-cell array has length LCM = LC+1).  The grid set-up restates the
reference's initialisation:

* cell order and neighbour maps: ``EFDC/cellmap.f90:13-28, 80-134``
* land-water face switches SUB/SVB for type-5 cells and the open-boundary
  modifications: ``EFDC/setbcs.f90:25-131, 151-245``
* face widths DXU/DYU/DXV/DYV: ``EFDC/setbcs.f90:343-374``
* permanent switches SUBO/SVBO: ``EFDC/setbcs.f90:1052-1055``
* metrics DXYP, DXYIP, DXIU, HRUO, SBX ...: ``EFDC/aaefdc.f90:2171-2190``
* ghost-cell values DXYP(1), DXYP(LC), BELV(1), BELV(LC): ``EFDC/ainit.f90:21-46``
* tidal constants PCBW = G*A*cos(2*pi*phase/TCP): ``EFDC/input.f90:435-440``
* depths at faces HU/HV: ``EFDC/calpuv2c.f90:898-899``

There is no public dataset for this path; these seeded fields stand in for
the reference's sample models.  Conventions of the generator (not of EFDC+):
the explicit upstream terms (FCAXE, FXE, TSX, QSUME, ...) are held fixed over a
run; the bottom stress TBX = STBX*|u0|*u0 uses Manning's n through
STBX = g n^2 / HU^(1/3) on a seeded, fixed reference velocity u0.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

G = 9.81
PI = 3.1415926535898  # EFDC/aaefdc.f90:650
PI2 = 2.0 * PI
M2_PERIOD = 44712.0

LAND = 9
WATER = 5

SIDES = ("W", "E", "S", "N")


def gaussian_field(rng, shape, corr_cells):
    """Smooth Gaussian random field with a Gaussian spectral filter,
    normalised to [0, 1]."""
    ny, nx = shape
    noise = rng.standard_normal(shape)
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    sigma = max(corr_cells, 1e-6)
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx * kx + ky * ky) * sigma * sigma)
    f = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    f -= f.min()
    mx = f.max()
    return f / mx if mx > 0 else f


@dataclass
class Scenario:
    """One basin: static grid (``grid``), per-step state (``state``) and the
    scalar parameters (``params``).  Arrays follow the Fortran 1-based layout
    (index L-1)."""

    ic: int
    jc: int
    la: int
    lc: int
    grid: dict
    state: dict
    params: dict
    ijct: np.ndarray = field(repr=False, default=None)
    channels: dict = field(repr=False, default=None)  # sub-grid channels (add_channels)
    layers: dict = field(repr=False, default=None)  # sigma layers (add_baroclinic)

    @property
    def ncell(self) -> int:
        return self.la - 1

    def copy_state(self) -> dict:
        return {k: (v.copy() if isinstance(v, np.ndarray) else
                    {s: a.copy() for s, a in v.items()} if isinstance(v, dict) else v)
                for k, v in self.state.items()}

    def tn(self, n: int) -> float:
        """TN of SETOPENBC for step N: DT*FLOAT(N)+TCON*TBEGIN (TBEGIN=0)."""
        return float(self.params["dt"]) * float(n)


def build_grid(ijct, dxp2d, dyp2d, belv2d, *, obc=None, mtide=1, tcp=(M2_PERIOD,),
               dx=None, dy=None):
    """Restate CELLMAP/SETBCS/AAEFDC for type-5 (water) / type-9 (land) cells.

    ijct, dxp2d, dyp2d, belv2d are [JC, IC] arrays (0-based J, I).  ``obc`` maps
    side -> list of (i, j, ispb, amp[mtide], phase[mtide]) with 1-based I, J.
    Returns (la, lc, grid dict, lij)."""
    jc, ic = ijct.shape
    water = (ijct > 0) & (ijct < 9)
    jj, ii = np.nonzero(water)  # C order: J outer, I inner == cellmap.f90:13-24
    nw = jj.size
    la = nw + 1
    lc = la + 1
    lcm = lc + 1
    lij = np.zeros((jc, ic), dtype=np.int64)
    lij[jj, ii] = np.arange(2, la + 1)
    il = np.zeros(lcm, np.int32)
    jl = np.zeros(lcm, np.int32)
    il[1:la] = ii + 1
    jl[1:la] = jj + 1

    def nb(dj, di):
        j2, i2 = jj + dj, ii + di
        inside = (j2 >= 0) & (j2 < jc) & (i2 >= 0) & (i2 < ic)
        out = np.full(nw, lc, np.int32)
        ok = inside.copy()
        ok[inside] = ijct[j2[inside], i2[inside]] != LAND
        out[ok] = lij[j2[ok], i2[ok]]
        return out

    lnc = np.zeros(lcm, np.int32)
    lsc = np.zeros(lcm, np.int32)
    lec = np.zeros(lcm, np.int32)
    lwc = np.zeros(lcm, np.int32)
    # cellmap.f90:80-91, 121-124
    for arr in (lnc, lsc, lec, lwc):
        arr[0] = lc
        arr[lc - 1] = 1
    lnc[1:la] = nb(1, 0)
    lsc[1:la] = nb(-1, 0)
    lec[1:la] = nb(0, 1)
    lwc[1:la] = nb(0, -1)

    # setbcs.f90:100-115 (LCT=5): SUB=1 if west cell is type 3,4,5; SVB=1 if south is 2,3,5
    sub = np.zeros(lcm)
    svb = np.zeros(lcm)
    west_t = np.where(ii - 1 >= 0, ijct[jj, np.maximum(ii - 1, 0)], LAND)
    south_t = np.where(jj - 1 >= 0, ijct[np.maximum(jj - 1, 0), ii], LAND)
    sub[1:la] = np.isin(west_t, (3, 4, 5)).astype(float)
    svb[1:la] = np.isin(south_t, (2, 3, 5)).astype(float)
    sub[0] = svb[0] = sub[lc - 1] = svb[lc - 1] = 0.0

    def F(a, L):  # 1-based accessor
        return a[L - 1]

    obc = obc or {}
    sides = {}
    for s in SIDES:
        cells = obc.get(s, [])
        n = len(cells)
        ls = np.zeros(n, np.int32)
        isp = np.zeros(n, np.int32)
        pcb = np.zeros((mtide, n))
        psb = np.zeros((mtide, n))
        for k, (i, j, ispb, amp, ph) in enumerate(cells):
            L = int(lij[j - 1, i - 1])
            if L < 2:
                raise ValueError(f"open boundary cell ({i},{j}) is not water")
            ls[k] = L
            isp[k] = ispb
            for m in range(mtide):
                rad = PI2 * ph[m] / tcp[m]  # input.f90:435-440
                pcb[m, k] = G * amp[m] * math.cos(rad)
                psb[m, k] = G * amp[m] * math.sin(rad)
        sides[s] = dict(l=ls, ispb=isp, pcb=pcb, psb=psb)

    # setbcs.f90:178-245 water-water boundary switches
    for k, L in enumerate(sides["W"]["l"]):
        sub[L - 1] = 0.0
        svb[L - 1] = 0.0
        svb[F(lnc, L) - 1] = 0.0
        if sides["W"]["ispb"][k] <= 1:
            LE = F(lec, L)
            svb[LE - 1] = 0.0
            svb[F(lnc, LE) - 1] = 0.0
    for k, L in enumerate(sides["E"]["l"]):
        svb[L - 1] = 0.0
        svb[F(lnc, L) - 1] = 0.0
        if sides["E"]["ispb"][k] <= 1:
            LW = F(lwc, L)
            svb[LW - 1] = 0.0
            svb[F(lnc, LW) - 1] = 0.0
    for k, L in enumerate(sides["S"]["l"]):
        LN = F(lnc, L)
        svb[L - 1] = 0.0
        sub[L - 1] = 0.0
        sub[F(lec, L) - 1] = 0.0
        if sides["S"]["ispb"][k] <= 1:
            sub[LN - 1] = 0.0
            sub[F(lec, LN) - 1] = 0.0
    for k, L in enumerate(sides["N"]["l"]):
        LS = F(lsc, L)
        sub[L - 1] = 0.0
        sub[F(lec, L) - 1] = 0.0
        if sides["N"]["ispb"][k] <= 1:
            sub[LS - 1] = 0.0
            sub[F(lec, LS) - 1] = 0.0
    sub[lc - 1] = svb[lc - 1] = 0.0

    dxp = np.zeros(lcm)
    dyp = np.zeros(lcm)
    belv = np.zeros(lcm)
    dxp[1:la] = dxp2d[jj, ii]
    dyp[1:la] = dyp2d[jj, ii]
    belv[1:la] = belv2d[jj, ii]
    dx = float(dx if dx is not None else dxp[1:la].mean())
    dy = float(dy if dy is not None else dyp[1:la].mean())
    # ainit.f90:21-46 ghost cells
    dxp[0] = dxp[lc - 1] = dx
    dyp[0] = dyp[lc - 1] = dy
    belv[0] = belv[1]
    belv[lc - 1] = belv[la - 1]

    # setbcs.f90:343-374 (depends on the final SUB/SVB)
    Ls = np.arange(2, la + 1)
    i0 = Ls - 1
    LW = lwc[i0] - 1
    LE = lec[i0] - 1
    LN = lnc[i0] - 1
    LSv = lsc[i0] - 1
    dxu = np.zeros(lcm)
    dyu = np.zeros(lcm)
    dxv = np.zeros(lcm)
    dyv = np.zeros(lcm)
    s_l = sub[i0]
    s_e = sub[LE]
    c1 = s_l > 0.5
    c2 = (s_l < 0.5) & (s_e > 0.5)
    c3 = (s_l < 0.5) & (s_e < 0.5)
    dxu[i0[c1]] = 0.5 * (dxp[i0[c1]] + dxp[LW[c1]])
    dyu[i0[c1]] = 0.5 * (dyp[i0[c1]] + dyp[LW[c1]])
    ddyddx = 2.0 * (dyp[LE[c2]] - dyp[i0[c2]]) / (dxp[i0[c2]] + dxp[LE[c2]])
    dxu[i0[c2]] = dxp[i0[c2]]
    dyu[i0[c2]] = dyp[i0[c2]] - 0.5 * dxp[i0[c2]] * ddyddx
    dxu[i0[c3]] = dxp[i0[c3]]
    dyu[i0[c3]] = dyp[i0[c3]]
    v_l = svb[i0]
    v_n = svb[LN]
    d1 = v_l > 0.5
    d2 = (v_l < 0.5) & (v_n > 0.5)
    d3 = (v_l < 0.5) & (v_n < 0.5)
    dxv[i0[d1]] = 0.5 * (dxp[i0[d1]] + dxp[LSv[d1]])
    dyv[i0[d1]] = 0.5 * (dyp[i0[d1]] + dyp[LSv[d1]])
    ddxddy = 2.0 * (dxp[LN[d2]] - dxp[i0[d2]]) / (dyp[i0[d2]] + dyp[LN[d2]])
    dxv[i0[d2]] = dxp[i0[d2]] - 0.5 * dyp[i0[d2]] * ddxddy
    dyv[i0[d2]] = dyp[i0[d2]]
    dxv[i0[d3]] = dxp[i0[d3]]
    dyv[i0[d3]] = dyp[i0[d3]]

    subo = sub.copy()
    svbo = svb.copy()
    # aaefdc.f90:2171-2190 (STCAP=1 for type-5 cells)
    z = lambda: np.zeros(lcm)  # noqa: E731
    dxyu, dxyv, dxyp, dxiu, dyiu, dxiv, dyiv, dxyip = (z() for _ in range(8))
    hruo, hrvo, sbx, sby, sbxo, sbyo = (z() for _ in range(6))
    dxyu[i0] = dxu[i0] * dyu[i0]
    dxyv[i0] = dxv[i0] * dyv[i0]
    dxyp[i0] = 1.0 * dxp[i0] * dyp[i0]
    dxiu[i0] = 1.0 / dxu[i0]
    dyiu[i0] = 1.0 / dyu[i0]
    dxiv[i0] = 1.0 / dxv[i0]
    dyiv[i0] = 1.0 / dyv[i0]
    dxyip[i0] = 1.0 / (1.0 * dxp[i0] * dyp[i0])
    hruo[i0] = subo[i0] * dyu[i0] * dxiu[i0]
    hrvo[i0] = svbo[i0] * dxv[i0] * dyiv[i0]
    sbx[i0] = 0.5 * sub[i0] * dyu[i0]
    sby[i0] = 0.5 * svb[i0] * dxv[i0]
    sbxo[i0] = 0.5 * subo[i0] * dyu[i0]
    sbyo[i0] = 0.5 * svbo[i0] * dxv[i0]
    dxyp[0] = dx * dy  # ainit.f90:27,44
    dxyp[lc - 1] = dx * dy

    grid = dict(la=la, lc=lc, il=il, jl=jl, lnc=lnc, lsc=lsc, lec=lec, lwc=lwc,
                dxyp=dxyp, dxyip=dxyip, dxiu=dxiu, dyiu=dyiu, dxiv=dxiv, dyiv=dyiv,
                dxyu=dxyu, dxyv=dxyv, hruo=hruo, hrvo=hrvo, subo=subo, svbo=svbo,
                sbxo=sbxo, sbyo=sbyo, belv=belv, mtide=mtide,
                tcp=np.asarray(tcp, dtype=np.float64)[:mtide], obc=sides,
                dxu=dxu, dyu=dyu, dxv=dxv, dyv=dyv, dxp=dxp, dyp=dyp)
    init = dict(sub=sub, svb=svb, sbx=sbx, sby=sby)
    return la, lc, grid, lij, init


def face_depths(grid, hp):
    """HU/HV/HPI/HUI/HVI from HP exactly as calpuv2c.f90:898-906."""
    la = grid["la"]
    lcm = hp.size
    i0 = np.arange(1, la)
    lw = grid["lwc"][i0] - 1
    ls = grid["lsc"][i0] - 1
    dxyp = grid["dxyp"]
    fsgzu = 0.5 / grid["dxyu"][i0]
    fsgzv = 0.5 / grid["dxyv"][i0]
    hu = np.zeros(lcm)
    hv = np.zeros(lcm)
    hu[i0] = (dxyp[i0] * hp[i0] + dxyp[lw] * hp[lw]) * fsgzu
    hv[i0] = (dxyp[i0] * hp[i0] + dxyp[ls] * hp[ls]) * fsgzv
    with np.errstate(divide="ignore"):
        hpi = np.zeros(lcm)
        hui = np.zeros(lcm)
        hvi = np.zeros(lcm)
        hpi[i0] = 1.0 / hp[i0]
        hui[i0] = 1.0 / hu[i0]
        hvi[i0] = 1.0 / hv[i0]
    return hu, hv, hpi, hui, hvi


def make_scenario(nx=100, ny=60, *, seed=1, dx=100.0, dy=100.0, land_frac=0.07,
                  depth=(2.0, 30.0), corr_len_m=1000.0, curvilinear=None,
                  obc_sides=("W",), amp=0.5, amp_range=None, ispb=0, phase=0.0,
                  mtide=1, tcp=(M2_PERIOD,), manning=0.025, u0=0.1, dt=10.0,
                  rsqm=1e-10, iterm=200, isdry=0, hdry=0.05, ndrystp=0, isbal=1,
                  datum=0.0, eta0=0.0, belv2d=None, land_mask=None, kc=4,
                  explicit_noise=0.0, snlt=0.0, ntstbc=0, fill_dead_ends=False):
    """A basin of nx*ny candidate cells inside a closed land ring.

    The land mask is seeded Bernoulli(land_frac) (the open-boundary column or
    row and its interior neighbour are kept wet); bathymetry is a Gaussian
    random field with correlation length ``corr_len_m`` rescaled to ``depth``.
    ``curvilinear=(lo, hi)`` draws DXP/DYP from a smooth field in [lo, hi] m."""
    rng = np.random.default_rng(seed)
    ic, jc = nx + 2, ny + 2
    ijct = np.full((jc, ic), LAND, np.int32)
    inner = np.ones((ny, nx), bool)
    if land_mask is not None:
        inner &= ~land_mask
    elif land_frac > 0:
        inner &= rng.random((ny, nx)) >= land_frac
    keep = np.zeros((ny, nx), bool)
    if "W" in obc_sides:
        keep[:, :2] = True
    if "E" in obc_sides:
        keep[:, -2:] = True
    if "S" in obc_sides:
        keep[:2, :] = True
    if "N" in obc_sides:
        keep[-2:, :] = True
    inner |= keep
    if fill_dead_ends:
        # water cells with three or four land neighbours (single-cell inlets
        # and lakes) become land, repeatedly, as grid generators do
        while True:
            pad = np.pad(inner, 1, constant_values=False)
            nwet = (pad[:-2, 1:-1].astype(np.int8) + pad[2:, 1:-1] + pad[1:-1, :-2] +
                    pad[1:-1, 2:])
            dead = inner & (nwet <= 1) & ~keep
            if not dead.any():
                break
            inner &= ~dead
    ijct[1:-1, 1:-1] = np.where(inner, WATER, LAND)

    if curvilinear is not None:
        lo, hi = curvilinear
        fx = gaussian_field(rng, (jc, ic), corr_cells=max(nx, ny) / 8.0)
        fy = gaussian_field(rng, (jc, ic), corr_cells=max(nx, ny) / 8.0)
        dxp2d = lo + (hi - lo) * fx
        dyp2d = lo + (hi - lo) * fy
    else:
        dxp2d = np.full((jc, ic), float(dx))
        dyp2d = np.full((jc, ic), float(dy))
    if belv2d is None:
        mean_dx = float(np.mean(dxp2d))
        f = gaussian_field(rng, (jc, ic), corr_cells=corr_len_m / mean_dx)
        dep = depth[0] + (depth[1] - depth[0]) * f
        belv2d = datum - dep
    else:
        belv2d = np.asarray(belv2d, dtype=np.float64)

    # open-boundary cells: the first/last interior column/row
    obc = {}
    mt = mtide
    ph = [phase] * mt
    for s in obc_sides:
        cells = []
        # where two open sides meet, two cells at each corner are left as plain
        # water cells: SETBCS closes the interior faces next to a boundary
        # (setbcs.f90:188-192, 216-220), and a radiation cell whose interior
        # face was closed by the other side's rule has CET=0, hence CC=0 and
        # CCMNM=0 in the reference as well
        if s in ("W", "E"):
            i = 2 if s == "W" else ic - 1
            j0 = 4 if "S" in obc_sides else 2
            j1 = jc - 3 if "N" in obc_sides else jc - 1
            coords = [(i, j) for j in range(j0, j1 + 1)]
        else:
            j = 2 if s == "S" else jc - 1
            i0 = 4 if "W" in obc_sides else 2
            i1 = ic - 3 if "E" in obc_sides else ic - 1
            coords = [(i, j) for i in range(i0, i1 + 1)]
        nb = len(coords)
        for k, (i, j) in enumerate(coords):
            if ijct[j - 1, i - 1] == LAND:
                continue
            if amp_range is not None:
                a = amp_range[0] + (amp_range[1] - amp_range[0]) * (0.5 - 0.5 * math.cos(PI2 * k / max(nb, 1)))
            else:
                a = amp
            cells.append((i, j, ispb, [a] * mt, ph))
        obc[s] = cells

    la, lc, grid, lij, init = build_grid(ijct, dxp2d, dyp2d, belv2d, obc=obc,
                                         mtide=mtide, tcp=tcp, dx=dx, dy=dy)
    lcm = lc + 1
    i0 = np.arange(1, la)
    belv = grid["belv"]
    hp = np.zeros(lcm)
    hp[i0] = np.maximum(datum + eta0 - belv[i0], 0.9 * hdry if isdry else 1e-3)
    p = np.zeros(lcm)
    p[i0] = G * (hp[i0] + belv[i0])
    hu, hv, hpi, hui, hvi = face_depths(grid, hp)
    # explicit upstream terms (fixed over the run; see module docstring)
    tbx = np.zeros(lcm)
    tby = np.zeros(lcm)
    if manning and u0:
        fu = gaussian_field(rng, (jc, ic), corr_cells=max(nx, ny) / 6.0)
        fv = gaussian_field(rng, (jc, ic), corr_cells=max(nx, ny) / 6.0)
        jj = grid["jl"][i0] - 1
        ii = grid["il"][i0] - 1
        u = u0 * (2.0 * fu[jj, ii] - 1.0)
        v = u0 * (2.0 * fv[jj, ii] - 1.0)
        n2 = np.broadcast_to(np.asarray(manning, dtype=np.float64), (la - 1,))
        with np.errstate(divide="ignore", invalid="ignore"):
            stbx = np.where(hu[i0] > 0, G * n2 * n2 / np.cbrt(np.maximum(hu[i0], 1e-3)), 0.0)
            stby = np.where(hv[i0] > 0, G * n2 * n2 / np.cbrt(np.maximum(hv[i0], 1e-3)), 0.0)
        sp = np.sqrt(u * u + v * v)
        tbx[i0] = stbx * sp * u * grid["subo"][i0]
        tby[i0] = stby * sp * v * grid["svbo"][i0]
    zeros = lambda: np.zeros(lcm)  # noqa: E731
    state = dict(
        p=p, hp=hp, h1p=hp.copy(), hu=hu, hv=hv, uhdye=zeros(), vhdxe=zeros(),
        sub=init["sub"], svb=init["svb"], sbx=init["sbx"], sby=init["sby"],
        lmaskdry=np.ones(lcm, np.int32), iscdry=np.zeros(lcm, np.int32),
        lopenbcdry=np.zeros(lcm, np.int32), natdry=np.zeros(lcm, np.int32),
        fcaxe=zeros(), fcaye=zeros(), fxe=zeros(), fye=zeros(),
        tsx=zeros(), tsy=zeros(), tbx=tbx, tby=tby, qsume=zeros(),
        pser={s: np.full(len(grid["obc"][s]["l"]), G * datum) for s in SIDES},
        uhe=zeros(), vhe=zeros(), hpi=hpi, hui=hui, hvi=hvi,
        qdwaste=zeros(), vdwaste=zeros(),
    )
    if explicit_noise > 0:
        for k in ("fcaxe", "fcaye", "fxe", "fye", "tsx", "tsy", "qsume"):
            a = np.zeros(lcm)
            a[i0] = explicit_noise * rng.standard_normal(la - 1)
            if k == "qsume":
                a[i0] *= 1e-3
            state[k] = a
        for k in ("uhdye", "vhdxe"):
            a = np.zeros(lcm)
            a[i0] = 10.0 * explicit_noise * rng.standard_normal(la - 1)
            a[i0] *= grid["subo" if k == "uhdye" else "svbo"][i0]
            state[k] = a
    params = dict(dt=float(dt), g=G, hdry=float(hdry), rsqm=float(rsqm),
                  iterm=int(iterm), isdry=int(isdry), ndrystp=int(ndrystp),
                  isbal=int(isbal), snlt=float(snlt), ritb1=1.0, pi2=PI2,
                  ntstbc=int(ntstbc), max_sweeps=500, kc=int(kc))
    return Scenario(ic=ic, jc=jc, la=la, lc=lc, grid=grid, state=state,
                    params=params, ijct=ijct)


# ---------------------------------------------------------------- configs
def config1(seed=1):
    """100x60 Cartesian basin, dx=dy=100 m, ~5,600 wet cells, 7% seeded land,
    2-30 m depth with 1 km correlation, west open boundary with a 0.5 m M2
    tide, Manning 0.025, dt=10 s, RSQM=1e-10, ISDRY=0."""
    return make_scenario(100, 60, seed=seed, dx=100.0, dy=100.0, land_frac=0.07,
                         depth=(2.0, 30.0), corr_len_m=1000.0, obc_sides=("W",),
                         amp=0.5, dt=10.0, rsqm=1e-10, iterm=200, isdry=0, kc=4)


def config2(seed=2, n=2048):
    """n x n curvilinear-orthogonal basin (DXP/DYP smooth in 50-200 m), depth
    1-60 m, seeded islands (~19% land), west tidal boundary with amplitudes
    0.2-1.5 m along it, dt=5 s, KC=8."""
    rng = np.random.default_rng(seed + 1000)
    f = gaussian_field(rng, (n, n), corr_cells=n / 24.0)
    land = f > np.quantile(f, 0.81)
    return make_scenario(n, n, seed=seed, land_mask=land, land_frac=0.0,
                         curvilinear=(50.0, 200.0), depth=(1.0, 60.0),
                         corr_len_m=20000.0, obc_sides=("W",), amp_range=(0.2, 1.5),
                         dt=5.0, rsqm=1e-10, iterm=500, isdry=0, kc=8)


def config3_sizes(seed=3, members=256, lo=10_000, hi=400_000):
    """Wet-cell counts of the batched ensemble: log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), members)).astype(np.int64)


def config3_member(k, ncell, seed=3):
    """Member k of the batched ensemble: a square-ish basin of ~ncell wet
    cells, depth 1-40 m, Manning 0.015-0.04, M2 amplitude 0.1-1.0 m.

    The members run without wetting/drying (ISDRY=0), where the reference
    STOPs at the first non-positive depth.  So that the seeded members stay
    wet, the shallowest water of a member is 3x its tidal amplitude (at least
    1 m) and dead-end cells (single-cell inlets, in which the tidal standing
    wave amplifies) are land."""
    rng = np.random.default_rng(seed * 100_003 + k)
    n_man = rng.uniform(0.015, 0.04)
    amp = rng.uniform(0.1, 1.0)
    side = int(math.ceil(math.sqrt(ncell / 0.93)))
    ny = max(8, side)
    nx = max(8, int(math.ceil(ncell / 0.93 / ny)))
    return make_scenario(nx, ny, seed=seed * 7919 + k, dx=100.0, dy=100.0,
                         land_frac=0.07, depth=(max(1.0, 3.0 * amp), 40.0),
                         corr_len_m=1500.0, obc_sides=("W",), amp=amp, manning=n_man,
                         dt=10.0, rsqm=1e-10, iterm=500, isdry=0, kc=4,
                         fill_dead_ends=True)


def config4(seed=4, n=512, nsteps=200, ngauges=20):
    """Adjoint calibration basin: n x n cells (~240k wet at n=512), 7% land,
    depth 2-30 m, west M2 boundary 0.5 m, dt=10 s, ISDRY=0, RSQM=1e-10.
    Returns (scenario, gauges, true log n, true boundary amplitudes): the
    per-cell log Manning n ~ N(log 0.025, 0.2), four amplitudes, and 20
    seeded interior gauge cells (1-based L)."""
    scn = make_scenario(n, n, seed=seed, dx=100.0, dy=100.0, land_frac=0.07,
                        depth=(2.0, 30.0), corr_len_m=1000.0, obc_sides=("W",), amp=0.5,
                        manning=0.0, dt=10.0, rsqm=1e-10, iterm=500, isdry=0, kc=4,
                        fill_dead_ends=True)
    rng = np.random.default_rng(seed + 4000)
    log_n = np.full(scn.lc + 1, math.log(0.025))
    log_n[1:scn.la] = rng.normal(math.log(0.025), 0.2, scn.la - 1)
    amps = np.array([0.45, 0.55, 0.5, 0.6])
    bc = set(int(x) for s in SIDES for x in scn.grid["obc"][s]["l"])
    il = scn.grid["il"]
    cand = [L for L in range(2, scn.la + 1) if L not in bc and il[L - 1] > 4]
    gauges = np.sort(rng.choice(cand, size=ngauges, replace=False)).astype(np.int32)
    return scn, gauges, log_n, amps


def tidal_flat(n=1024, *, seed=5, hdry=0.05, amp=2.0, ramp=(-2.0, 15.0 / 4.0),
               noise=0.3, dt=5.0):
    """Wetting/drying tidal flat: bed elevation ramps west->east across the
    basin plus N(0, noise) roughness, 2 m M2 tide on the west boundary,
    ISDRY=99.  The ramp end points are chosen so that 30-45% of the cells
    toggle over a tidal cycle."""
    rng = np.random.default_rng(seed)
    ic, jc = n + 2, n + 2
    x = np.linspace(0.0, 1.0, ic)[None, :]
    belv = ramp[0] + (ramp[1] - ramp[0]) * x + noise * rng.standard_normal((jc, ic))
    belv = np.broadcast_to(belv, (jc, ic)).copy()
    belv[:, :3] = np.minimum(belv[:, :3], -2.0)
    return make_scenario(n, n, seed=seed, land_frac=0.0, belv2d=belv, dx=50.0, dy=50.0,
                         obc_sides=("W",), amp=amp, dt=dt, isdry=99, hdry=hdry,
                         ndrystp=-10, rsqm=1e-10, iterm=500, kc=4)


def add_channels(scn: Scenario, n: int = 6, *, seed: int = 0, types=(1, 2), qcherr: float = 1.0,
                 chanlen=(20.0, 80.0), chanfric=(0.5, 5.0), reach: int = 3,
                 hmin: float = 0.1) -> Scenario:
    """Sub-grid channels (the MDCHH host-guest pairs of subchan.f90) between
    seeded pairs of distinct water cells that are not open-boundary cells, the
    guest within `reach` cells of its host.  Channel k has type
    types[k % len(types)]: 1 = x-direction (guest in LMDCHU, LMDCHV = 1),
    2 = y-direction (guest in LMDCHV, LMDCHU = 1), as input.f90:2576-2588 sets
    them.  Adds the per-channel flows QCHANU, QCHANV, QCHANUN, QCHANVN (zero,
    as input.f90 starts them) to the state, QCHERR to the parameters, and
    HP(1) = HMIN (ainit.f90:91; SUBCHAN's y-direction test reads HP(LMDCHU))."""
    rng = np.random.default_rng(seed)
    g = scn.grid
    bc = set(int(x) for s_ in SIDES for x in g["obc"][s_]["l"])
    lij = {(int(g["il"][L - 1]), int(g["jl"][L - 1])): L for L in range(2, scn.la + 1)}
    used = set(bc)
    host, guest = [], []
    for L in rng.permutation(np.arange(2, scn.la + 1)):
        if len(host) == n:
            break
        L = int(L)
        if L in used:
            continue
        i, j = int(g["il"][L - 1]), int(g["jl"][L - 1])
        near = [lij[(i + di, j + dj)] for di in range(-reach, reach + 1)
                for dj in range(-reach, reach + 1)
                if (di or dj) and (i + di, j + dj) in lij and lij[(i + di, j + dj)] not in used]
        if not near:
            continue
        G_ = int(near[rng.integers(len(near))])
        host.append(L)
        guest.append(G_)
        used.update((L, G_))
    host = np.array(host, dtype=np.int32)
    guest = np.array(guest, dtype=np.int32)
    n = host.size
    typ = np.array([types[k % len(types)] for k in range(n)], dtype=np.int32)
    lu = np.where(typ == 1, guest, 1).astype(np.int32)
    lv = np.where(typ == 2, guest, 1).astype(np.int32)
    scn.channels = dict(type=typ, lhost=host, lu=lu, lv=lv,
                        chanlen=rng.uniform(*chanlen, n), chanfric=rng.uniform(*chanfric, n),
                        dxp=np.asarray(g["dxp"], dtype=np.float64),
                        dyp=np.asarray(g["dyp"], dtype=np.float64))
    for k in ("qchanu", "qchanv", "qchanun", "qchanvn"):
        scn.state[k] = np.zeros(n)
    scn.state["hp"][0] = hmin
    scn.params["qcherr"] = qcherr
    return scn


def add_baroclinic(scn: Scenario, kc: int = 4, *, seed: int = 0, front: float = 2e-3,
                   strat: float = 5e-4, bsc: float = 1.0) -> Scenario:
    """Baroclinic terms on a uniform sigma grid of `kc` layers: DZC = 1/KC and
    ZZ = the layer mid-points (aaefdc.f90:1090, 1237), and a seeded buoyancy
    B(L,K) (a horizontal front of amplitude `front` across the basin plus a
    stable vertical stratification `strat` and small noise).  Adds the
    layers as scn.layers ({"dzc", "zz"}: (KC, LCM)), B to the state
    ((KC, LCM)), and BSC, GP = G to the parameters."""
    rng = np.random.default_rng(seed)
    lcm = scn.lc + 1
    g = scn.grid
    dzc = np.full((kc, lcm), 1.0 / kc)
    zz = np.repeat(((np.arange(kc) + 0.5) / kc)[:, None], lcm, axis=1)
    il = np.zeros(lcm)
    il[1:scn.la] = g["il"][1:scn.la]
    x = (il - il[1:scn.la].min()) / max(1.0, float(np.ptp(il[1:scn.la])))
    b = np.zeros((kc, lcm))
    for k in range(kc):
        b[k, 1:scn.la] = (front * x[1:scn.la] - strat * (kc - 1 - k) / max(kc - 1, 1) +
                          1e-5 * rng.standard_normal(scn.la - 1))
    scn.layers = dict(dzc=dzc, zz=zz)
    scn.state["b"] = b
    scn.params["bsc"] = bsc
    scn.params["gp"] = G
    return scn


def sample_model(f: dict, *, dt: float = 10.0, drawdown: float = 0.0,
                 wind: tuple = (0.0, 0.0), manning: float = 0.025, u0: float = 0.05,
                 seed: int = 0) -> Scenario:
    """A scenario on one of EFDC+'s sample-model grids.

    ``f`` holds the model's own arrays as tests/golden/make_sample_models.py
    extracts them: the cell-type map IJCT (5 water, 9 land, 0 outside), DXP,
    DYP, water depth and bottom elevation per cell (dxdy.inp), RSQM and ITERM
    (card C3), ISDRY (C5), NDRYSTP (C7), HDRY (C11), the west elevation
    boundary cells with their ISPBW (C19) and head (pser.inp at TBEGIN), and
    the flow sources (C24 cells, qser.inp at TBEGIN times QSFACTOR).
    Set here, not by the model files: the time step ``dt`` (the models step
    dynamically or at 10 s), a uniform wind stress ``wind`` = (TSX, TSY), an
    optional ``drawdown`` of the initial surface (so that shallow cells start
    dry), and a bottom stress from Manning's ``manning`` on a seeded velocity
    field of scale ``u0`` (as make_scenario)."""
    rng = np.random.default_rng(seed)
    ijct = np.where(np.asarray(f["ijct"]) == 5, WATER, LAND).astype(np.int32)
    jc, ic = ijct.shape
    dxp2d = np.where(ijct == WATER, f["dxp"], 0.0)
    dyp2d = np.where(ijct == WATER, f["dyp"], 0.0)
    belv2d = np.asarray(f["belv"], np.float64)
    isdry = int(f["isdry"])
    hdry = float(f["hdry"])
    west = np.asarray(f["west"]).reshape(-1, 3)
    obc = {"W": [(int(i), int(j), int(isp), [], []) for i, j, isp in west]}
    wd = dxp2d[ijct == WATER]
    la, lc, grid, lij, init = build_grid(ijct, dxp2d, dyp2d, belv2d, obc=obc, mtide=0, tcp=(),
                                         dx=float(wd.mean()),
                                         dy=float(dyp2d[ijct == WATER].mean()))
    lcm = lc + 1
    i0 = np.arange(1, la)
    jj = grid["jl"][i0] - 1
    ii = grid["il"][i0] - 1
    belv = grid["belv"]
    hp = np.zeros(lcm)
    hp[i0] = np.maximum(np.asarray(f["depth"])[jj, ii] - drawdown,
                        0.9 * hdry if isdry else 1e-3)
    p = np.zeros(lcm)
    p[i0] = G * (hp[i0] + belv[i0])
    hu, hv, hpi, hui, hvi = face_depths(grid, hp)
    tbx = np.zeros(lcm)
    tby = np.zeros(lcm)
    if manning and u0:
        u = u0 * rng.uniform(-1.0, 1.0, la - 1)
        v = u0 * rng.uniform(-1.0, 1.0, la - 1)
        stbx = np.where(hu[i0] > 0, G * manning ** 2 / np.cbrt(np.maximum(hu[i0], 1e-3)), 0.0)
        stby = np.where(hv[i0] > 0, G * manning ** 2 / np.cbrt(np.maximum(hv[i0], 1e-3)), 0.0)
        sp = np.sqrt(u * u + v * v)
        tbx[i0] = stbx * sp * u * grid["subo"][i0]
        tby[i0] = stby * sp * v * grid["svbo"][i0]
    qsume = np.zeros(lcm)
    for i, j, q in np.asarray(f["sources"]).reshape(-1, 3):
        qsume[int(lij[int(j) - 1, int(i) - 1]) - 1] += q
    zeros = lambda: np.zeros(lcm)  # noqa: E731
    tsx = zeros()
    tsy = zeros()
    tsx[i0] = wind[0]
    tsy[i0] = wind[1]
    head = float(f["west_head"]) if west.size else 0.0
    state = dict(
        p=p, hp=hp, h1p=hp.copy(), hu=hu, hv=hv, uhdye=zeros(), vhdxe=zeros(),
        sub=init["sub"], svb=init["svb"], sbx=init["sbx"], sby=init["sby"],
        lmaskdry=np.ones(lcm, np.int32), iscdry=np.zeros(lcm, np.int32),
        lopenbcdry=np.zeros(lcm, np.int32), natdry=np.zeros(lcm, np.int32),
        fcaxe=zeros(), fcaye=zeros(), fxe=zeros(), fye=zeros(),
        tsx=tsx, tsy=tsy, tbx=tbx, tby=tby, qsume=qsume,
        pser={s: np.full(len(grid["obc"][s]["l"]), G * head) for s in SIDES},
        uhe=zeros(), vhe=zeros(), hpi=hpi, hui=hui, hvi=hvi,
        qdwaste=zeros(), vdwaste=zeros(),
    )
    params = dict(dt=float(dt), g=G, hdry=hdry, rsqm=float(f["rsqm"]), iterm=int(f["iterm"]),
                  isdry=isdry, ndrystp=int(f["ndrystp"]), isbal=1, snlt=0.0, ritb1=1.0,
                  pi2=PI2, ntstbc=0, max_sweeps=500, kc=1)
    return Scenario(ic=ic, jc=jc, la=la, lc=lc, grid=grid, state=state, params=params,
                    ijct=ijct)


def add_implicit_drag(scn: Scenario, isitb: int = 1, *, isveg: int = 0, seed: int = 0,
                      u_scale: float = 0.3, manning: float = 0.03,
                      veg: float = 0.0) -> Scenario:
    """The implicit bottom drag of ISITB >= 1 (calpuv2c.f90:222-233) and/or the
    implicit vegetation drag of ISVEG > 0 (:234-242): seeded bottom-layer
    velocities U(L,KSZU(L)), V(L,KSZV(L)) (``ubot``, ``vbot``) and the
    interpolated VU, UV of scale ``u_scale`` m/s, Manning drag coefficients
    STBX = STBY = g n^2 / H^(1/3) on the face depths, vegetative resistances
    FXVEGE, FYVEGE uniform in [0, veg] 1/s, and RITB, RITB1 as CALTBXY sets
    them for ISITB (caltbxy.f90:93-106: 0.55, 0.45 for 1; 1, 0 above).  The
    explicit stresses TBX, TBY stay as they are (weighted by RITB1).  Fixed
    over a run, like the other upstream terms of these scenarios."""
    rng = np.random.default_rng(seed + 7)
    la, lcm = scn.la, scn.lc + 1
    i0 = np.arange(1, la)
    st = scn.state

    def field(scale):
        a = np.zeros(lcm)
        a[i0] = scale * rng.uniform(-1.0, 1.0, la - 1)
        return a

    st["ubot"], st["vbot"] = field(u_scale), field(u_scale)
    st["vu"], st["uv"] = field(u_scale), field(u_scale)
    for k, h in (("stbx", st["hu"]), ("stby", st["hv"])):
        a = np.zeros(lcm)
        a[i0] = G * manning ** 2 / np.cbrt(np.maximum(h[i0], 1e-3))
        st[k] = a
    for k in ("fxvege", "fyvege"):
        a = np.zeros(lcm)
        a[i0] = veg * rng.uniform(0.0, 1.0, la - 1)
        st[k] = a
    if isitb >= 1:
        ritb, ritb1 = (0.55, 0.45) if isitb == 1 else (1.0, 0.0)
    else:
        ritb, ritb1 = 0.0, 1.0
    scn.params.update(isitb=int(isitb), isveg=int(isveg), ritb=ritb, ritb1=ritb1)
    return scn


def add_momentum(scn: Scenario, kc: int = 1, *, seed: int = 0, lat: float = 45.0,
                 tri: bool = False, hdmf: bool = False, nbcs: int = 8,
                 type2: tuple = ()) -> dict:
    """The static part of the explicit momentum producer (efdc_xm_set_momentum)
    for a scenario, as ``scn.momentum``: the f-plane Coriolis parameter at
    ``lat`` times nothing else (FCORC), seeded curvature metrics DYDI, DXDJ of
    a gently curvilinear grid (+-2 % of the cell sizes), SCAX, SCAY = 1 and
    SAAX, SAAY = 1 except on the flow-boundary cells, ``kc`` equal sigma
    layers (SGZU = SGZV = 1/kc, FSGZU = FSGZV = kc), the NW and SE diagonal
    cells LNWC, LSEC from the cell coordinates (LC where land), ``nbcs``
    flow-boundary cells (the open-boundary cells first, then seeded interior
    cells) with their E/W and N/S adjacent cells (1 where none), and, with
    ``tri``, a seeded 0/1 STCUV, with ``hdmf``, SDX, SDY and LHDMF.  The open-
    boundary sides in ``type2`` get ISPBW.. = 2 (their open-boundary cells
    take CALEXP2T's type-2 forms)."""
    rng = np.random.default_rng(seed + 11)
    g = scn.grid
    la, lc, lcm = scn.la, scn.lc, scn.lc + 1
    i0 = np.arange(1, la)
    for side in type2:
        g["obc"][side]["ispb"][:] = 2

    def cellf(vals):
        a = np.zeros(lcm)
        a[i0] = vals
        return a

    il, jl = g["il"][i0].astype(np.int64), g["jl"][i0].astype(np.int64)
    at = np.full((int(il.max()) + 3, int(jl.max()) + 3), lc, np.int32)  # cell (i, j) -> L
    at[il + 1, jl + 1] = np.arange(2, la + 1, dtype=np.int32)
    lnwc = np.full(lcm, lc, np.int32)
    lsec = np.full(lcm, lc, np.int32)
    lnwc[i0] = at[il, jl + 2]
    lsec[i0] = at[il + 2, jl]
    dxp, dyp = g["dxp"], g["dyp"]
    fcor = 2.0 * 7.292e-5 * np.sin(np.radians(lat))
    sgz = np.full((kc, lcm), 1.0 / kc)
    mo = {"kc": kc, "ld": lcm,
          "fcorc": cellf(np.full(la - 1, fcor)),
          "dydi": cellf(0.02 * dyp[i0] * rng.uniform(-1.0, 1.0, la - 1)),
          "dxdj": cellf(0.02 * dxp[i0] * rng.uniform(-1.0, 1.0, la - 1)),
          "scax": cellf(np.ones(la - 1)), "scay": cellf(np.ones(la - 1)),
          "saax": cellf(np.ones(la - 1)), "saay": cellf(np.ones(la - 1)),
          "sgzu": sgz, "sgzv": sgz.copy(), "fsgzu": np.full((kc, lcm), float(kc)),
          "fsgzv": np.full((kc, lcm), float(kc)), "lnwc": lnwc, "lsec": lsec}
    obc_cells = [int(L) for sd in ("W", "E", "S", "N") for L in g["obc"][sd]["l"]]
    extra = [int(L) for L in rng.choice(np.arange(2, la + 1), size=max(0, nbcs), replace=False)]
    lbcs = (obc_cells + extra)[:max(nbcs, 0)]
    lberc = [int(g["lec"][L - 1]) if k % 2 == 0 else int(g["lwc"][L - 1])
             for k, L in enumerate(lbcs)]
    lbnrc = [int(g["lnc"][L - 1]) if k % 3 else 1 for k, L in enumerate(lbcs)]
    lberc = [L if L <= la else 1 for L in lberc]
    lbnrc = [L if L <= la else 1 for L in lbnrc]
    mo["lbcs"] = np.array(lbcs, np.int32)
    mo["lberc"] = np.array(lberc, np.int32)
    mo["lbnrc"] = np.array(lbnrc, np.int32)
    for L in lbcs:
        mo["saax"][L - 1] = 0.0
        mo["saay"][L - 1] = 0.0
    if tri:
        mo["stcuv"] = cellf((rng.uniform(size=la - 1) > 0.1).astype(float))
    if hdmf:
        mo["sdx"] = cellf(g["dyu"][i0] * rng.uniform(0.5, 1.5, la - 1))
        mo["sdy"] = cellf(g["dxv"][i0] * rng.uniform(0.5, 1.5, la - 1))
        lh = np.zeros(lcm, np.int32)
        lh[i0] = (rng.uniform(size=la - 1) > 0.05).astype(np.int32)
        mo["lhdmf"] = lh
    scn.momentum = mo
    return mo


def momentum_fields(scn: Scenario, *, seed: int = 0, u_scale: float = 0.4, wet_frac: float = 1.0,
                    fuhj: bool = False, hdmf: bool = False) -> dict:
    """One call's inputs of the explicit momentum producer for ``scn``: seeded
    layer velocities U, V of scale ``u_scale`` m/s, transports UHDY = U*DYU*HU/kc
    and VHDX = V*DXV*HV/kc, HP from the state, a wet set of ``wet_frac`` of the
    cells (None for all), sparse FUHJ, FVHJ with ``fuhj``, the CALHDMF terms with
    ``hdmf``, and zeroed output arrays (FCAXE.. and the layer outputs)."""
    rng = np.random.default_rng(seed + 13)
    mo = scn.momentum
    kc, lcm = mo["kc"], mo["ld"]
    la = scn.la
    i0 = np.arange(1, la)
    st, g = scn.state, scn.grid

    def lay(scale):
        a = np.zeros((kc, lcm))
        a[:, i0] = scale * rng.uniform(-1.0, 1.0, (kc, la - 1))
        return a

    u, v = lay(u_scale), lay(u_scale)
    f = {"u": u, "v": v, "uhdy": u * (g["dyu"][:lcm] * st["hu"][:lcm]) / kc,
         "vhdx": v * (g["dxv"][:lcm] * st["hv"][:lcm]) / kc,
         "hp": st["hp"].copy()}
    f["uhdy"] = np.ascontiguousarray(f["uhdy"])
    f["vhdx"] = np.ascontiguousarray(f["vhdx"])
    if wet_frac < 1.0:
        w = np.zeros(lcm, np.int32)
        w[i0] = (rng.uniform(size=la - 1) < wet_frac).astype(np.int32)
        f["wet"] = w
    if fuhj:
        for k in ("fuhj", "fvhj"):
            a = np.zeros((kc, lcm))
            pick = rng.choice(i0, size=max(1, (la - 1) // 50), replace=False)
            a[:, pick] = rng.uniform(-5.0, 5.0, (kc, pick.size))
            f[k] = a
    if hdmf:
        for k in ("fmdux", "fmduy", "fmdvx", "fmdvy"):
            f[k] = lay(1e-3)
    for k in ("fcaxe", "fcaye", "fxe", "fye"):
        f[k] = np.zeros(lcm)
    for k in ("fcax", "fcay", "fx", "fy", "cac"):
        f[k] = np.zeros((kc, lcm))
    return f


def add_three_levels(scn: Scenario) -> Scenario:
    """The state of the three-time-level scheme (CALPUV9C) at its start, with
    level n-1 equal to level n: P1 = P, H2P = H1P = HP, UHDY1E = UHDY2E =
    UHDYE, VHDX1E = VHDX2E = VHDXE, H1U = HU, H1V = HV, and the level n-1
    stresses TSX1, TSY1, TBX1, TBY1 equal to TSX, TSY, TBX, TBY.  With
    baroclinic terms FPGXE = FPGYE = 0 (their blend starts from zero)."""
    st = scn.state
    for dst, src in (("p1", "p"), ("h2p", "hp"), ("h1p", "hp"), ("uhdy1e", "uhdye"),
                     ("uhdy2e", "uhdye"), ("vhdx1e", "vhdxe"), ("vhdx2e", "vhdxe"),
                     ("h1u", "hu"), ("h1v", "hv"), ("tsx1", "tsx"), ("tsy1", "tsy"),
                     ("tbx1", "tbx"), ("tby1", "tby")):
        st[dst] = st[src].copy() if src in st else np.zeros_like(st["p"])
    if scn.params.get("bsc", 0.0) > 1e-6:
        st["fpgxe"] = np.zeros_like(st["p"])
        st["fpgye"] = np.zeros_like(st["p"])
    return scn


def three_level_schedule(nsteps: int, ntstbc: int):
    """The CALPUV9C calls of HDMT's time loop for steps 1..nsteps, as
    (N, ISTL, NCTBC, ROLD, RNEW): leapfrog steps (ISTL = 3, ROLD = 0, RNEW = 1)
    and, after the step on which NCTBC reaches NTSTBC, the trapezoidal
    correction of the same step (ISTL = 2, NCTBC = 0, ROLD = RNEW = 0.5)
    (hdmt.f90:299-305, 1009-1029; NCTBC starts at 1, aaefdc.f90:354)."""
    out, n, istl, nctbc = [], 1, 3, 1
    while n <= nsteps:
        out.append((n, istl, nctbc, 0.0 if istl == 3 else 0.5, 1.0 if istl == 3 else 0.5))
        if istl == 3 and nctbc == ntstbc:
            nctbc, istl = 0, 2
        else:
            nctbc, istl, n = nctbc + 1, 3, n + 1
    return out


def three_level_params(params: dict, istl: int, nctbc: int, rold: float, rnew: float) -> dict:
    """The parameters of one CALPUV9C(ISTL) call (DELT = 2*DT for ISTL = 3)."""
    return dict(params, tl3_istl=istl, nctbc=nctbc, rold=rold, rnew=rnew)


def make_bed(scn: Scenario, *, seed: int = 0, kc: int = 1, smooth_frac: float = 0.1,
             zbr=(0.002, 0.05)) -> dict:
    """A seeded bed for the bottom-stress producer (efdc_xm_bed): roughness
    heights ZBR log-uniform in `zbr` with a fraction `smooth_frac` of smooth
    cells (ZBR = 0: the viscous form), drag multipliers STBXO = STBYO = 1,
    DXP/DYP of the grid, and uniform sigma layers (DZC = SGZU = SGZV = 1/KC)."""
    rng = np.random.default_rng(seed)
    lcm = scn.lc + 1
    z = np.exp(rng.uniform(np.log(zbr[0]), np.log(zbr[1]), lcm))
    z[rng.random(lcm) < smooth_frac] = 0.0
    one = np.ones(lcm)
    return dict(zbr=z, stbxo=one.copy(), stbyo=one.copy(), dxp=scn.grid["dxp"].copy(),
                dyp=scn.grid["dyp"].copy(), dzc1=one / kc, sgzu1=one / kc, sgzv1=one / kc,
                kc=kc, avcon=1.0, vismud=1e-6, coeftsbl=4.0)


def drag_inputs(scn: Scenario, st: dict, h1u, h1v, *, seed: int = 0) -> dict:
    """Internal-mode inputs of the bottom-stress producer for the state `st`:
    the depth-averaged face velocities UHDYE/(HU*DYU) as the bottom-layer U, V
    (one layer), and seeded cross-face velocities VU, UV of the same size."""
    rng = np.random.default_rng(seed)
    g = scn.grid
    with np.errstate(all="ignore"):  # ghost elements: HU = 0
        ub = np.nan_to_num(st["uhdye"] * g["dyiu"] / st["hu"], nan=0.0, posinf=0.0, neginf=0.0)
        vb = np.nan_to_num(st["vhdxe"] * g["dxiv"] / st["hv"], nan=0.0, posinf=0.0, neginf=0.0)
    s = max(1e-3, float(np.abs(ub).max()))
    return dict(ub=ub, vb=vb, vu=0.5 * s * rng.standard_normal(ub.size),
                uv=0.5 * s * rng.standard_normal(ub.size), h1u=np.asarray(h1u, float).copy(),
                h1v=np.asarray(h1v, float).copy())

"""Seeded synthetic initial states (problem generators) of the configurations.

C1  2-D dry rising thermal bubble, restated from the reference's
    MeshBlock::ProblemGenerator of examples/2019-Li-snap/robert.cpp:72-114
    (Gaussian bubble: a = 0, s = radius).
C2  3-D moist convection: dry adiabat capped by an isothermal layer, H2O at
    80 % relative humidity, liquid and ice at zero, seeded temperature noise
    near the ground (the moist-adiabat setup of src/snap/
    setup_moist_adiabatic_profile.cpp:7-90 restated for a dry adiabat).
C3  cubed-sphere giant-planet shell: six panels, a dry H2-He adiabat through
    165 K at 1 bar on levels uniform in log pressure from 100 bar to 0.1 bar,
    seeded zonal jets of at most 5 m/s (panel velocities from the eastward
    wind through CubedSphere::GetVyVz, cubed_sphere.cpp:138-151).
C5  batched uneven blocks: C2's column physics on blocks of seeded sizes.

Every generator returns a :class:`Problem`: the block configuration (a
ctypes BlockConfig) and the conserved state u laid out (NV, nc3, nc2, nc1)
with zeroed ghost cells.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import thermo as T
from ._abi import (BC_PERIODIC, BC_REFLECT, FP64, NGHOST, RECON_PLM, RECON_PPM,
                   RS_HLLC, RS_LMARS, BlockConfig, ShellConfig)


@dataclass
class Problem:
    name: str
    cfg: BlockConfig
    x1f: np.ndarray
    u: np.ndarray
    w: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def ny(self):
        return self.cfg.thermo.ny

    @property
    def nv(self):
        return 5 + self.cfg.thermo.ny

    def interior(self, a):
        ng = NGHOST
        nx1, nx2, nx3 = self.cfg.nx1, self.cfg.nx2, self.cfg.nx3
        ks = ng if nx3 > 1 else 0
        js = ng if nx2 > 1 else 0
        return a[..., ks:ks + nx3, js:js + nx2, ng:ng + nx1]


def make_config(nx1, nx2, nx3, x1f, dx2, dx3, th, bc, recon, rsolver,
                implicit_flag=0, satadj=0, cfl=0.8, precision=FP64):
    cfg = BlockConfig()
    cfg.nx1, cfg.nx2, cfg.nx3 = nx1, nx2, nx3
    for q in range(6):
        cfg.bc[q] = bc[q]
    cfg.x2min = 0.0
    cfg.x3min = 0.0
    cfg.dx2, cfg.dx3 = dx2, dx3
    x1f = np.ascontiguousarray(x1f, dtype=np.float64)
    cfg.h_x1f = x1f.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cfg.recon, cfg.rsolver = recon, rsolver
    cfg.implicit_flag, cfg.precision, cfg.satadj = implicit_flag, precision, satadj
    cfg.cfl = cfl
    cfg.thermo = th
    return cfg, x1f


def _shape(nx1, nx2, nx3, nv):
    nc1 = nx1 + 2 * NGHOST
    nc2 = nx2 + 2 * NGHOST if nx2 > 1 else 1
    nc3 = nx3 + 2 * NGHOST if nx3 > 1 else 1
    return (nv, nc3, nc2, nc1)


def _embed(prob_shape, w_int, nx1, nx2, nx3):
    w = np.zeros(prob_shape)
    ks = NGHOST if nx3 > 1 else 0
    js = NGHOST if nx2 > 1 else 0
    w[:, ks:ks + nx3, js:js + nx2, NGHOST:NGHOST + nx1] = w_int
    return w


def bubble2d(nx1=150, nx2=100, x1max=1500.0, x2max=1000.0, dT=0.5, xc=500.0,
             zc=260.0, s=250.0, a=0.0, Ts=300.0, p0=1.0e5, grav=9.81,
             gamma=1.4, cfl=0.4, recon=RECON_PLM, rsolver=RS_LMARS):
    """C1: robert.cpp:72-114 with x1 vertical, nx3 = 1, reflecting walls.

    cfl: the time step is cfl x the per-direction minimum of dx / (|v| + c)
    (patches/21.new_blockdt.patch); the configuration's Courant number 0.8
    is split over the d = 2 directions that carry sound waves, because the
    unsplit RK3 scheme grows grid-scale noise at 0.8 per direction."""
    th = T.dry(gammad=gamma, grav=-grav)
    Rd = th.rd
    cp = gamma / (gamma - 1.0) * Rd
    x1f = np.linspace(0.0, x1max, nx1 + 1)
    x1v = 0.5 * (x1f[1:] + x1f[:-1])
    dx2 = x2max / nx2
    x2v = (np.arange(nx2) + 0.5) * dx2
    z, x = np.meshgrid(x1v, x2v, indexing="ij")  # (nx1, nx2)
    r = np.sqrt((x - xc) ** 2 + (z - zc) ** 2)
    temp = Ts - grav * z / cp
    pres = p0 * (temp / Ts) ** (cp / Rd)
    bub = np.where(r <= a, dT, dT * np.exp(-((r - a) ** 2) / (s * s)))
    temp = temp + bub * (pres / p0) ** (Rd / cp)
    rho = pres / (Rd * temp)
    nv = 5
    w_int = np.zeros((nv, 1, nx2, nx1))
    w_int[0, 0] = rho.T
    w_int[4, 0] = pres.T
    shape = _shape(nx1, nx2, 1, nv)
    w = _embed(shape, w_int, nx1, nx2, 1)
    u = T.prim_to_cons(th, w)
    u[:, :, :, :NGHOST] = 0.0
    u[:, :, :, NGHOST + nx1:] = 0.0
    u = _embed(shape, u[:, 0:1, NGHOST:NGHOST + nx2, NGHOST:NGHOST + nx1], nx1, nx2, 1)
    bc = [BC_REFLECT] * 4 + [BC_PERIODIC] * 2
    cfg, x1f = make_config(nx1, nx2, 1, x1f, dx2, 1.0, th, bc, recon, rsolver,
                           implicit_flag=0, satadj=0, cfl=cfl)
    return Problem("C1-bubble2d", cfg, x1f, u, w, dict(dt_hint=None))


def robert2d(nx1=300, nx2=200, recon=RECON_PPM):
    """The rising-bubble regression run of examples/2019-Li-snap/robert2d.inp:
    300 x 200 cells on 1500 m x 1000 m, Ts = 303.15 K, bubble radius a =
    50 m with a Gaussian skirt s = 100 m centred at (x, z) = (500, 260) m,
    dT = 0.5 K, g = 9.8 m/s^2, p0 = 1e5 Pa, Courant number 0.9 (0.45 per
    direction, see bubble2d), run to tlim = 1080 s with outputs every 180 s.
    The input's fifth-order horizontal reconstruction (xorder = 5) is
    replaced by PPM."""
    p = bubble2d(nx1=nx1, nx2=nx2, x1max=1.5e3, x2max=1.0e3, dT=0.5, xc=500.0, zc=260.0,
                 s=100.0, a=50.0, Ts=303.15, p0=1.0e5, grav=9.8, gamma=1.4, cfl=0.45,
                 recon=recon)
    p.name = "robert2d"
    p.meta.update(tlim=1080.0, out_dt=180.0, p0=1.0e5)
    return p


def straka2d(nx1=64, nx2=256, x1max=6.4e3, x2max=25.6e3, Ts=300.0, p0=1.0e5, dT=-15.0,
             xc=0.0, xr=4.0e3, zc=3.0e3, zr=2.0e3, grav=9.8, K=75.0, cfl=0.45,
             recon=RECON_PPM, rsolver=RS_LMARS):
    """The dense sinking bubble of examples/2019-Li-snap/straka.inp /
    straka.cpp:219-262 (Straka et al. 1993): a dry adiabat from Ts, a cold
    bubble of dT (cos(pi L) + 1) / 2 for L <= 1 centred on the left wall,
    reflecting walls; the dissipation source of diffusivity K (straka.cpp:
    125-190) is turned on by the caller with set_diffusion(meta["K"],
    meta["p0"]).  Courant number 0.9 split over the two directions as in
    bubble2d; fifth-order horizontal reconstruction replaced by PPM."""
    th = T.dry(gammad=1.4, grav=-grav)
    Rd = th.rd
    cp = 1.4 / 0.4 * Rd
    x1f = np.linspace(0.0, x1max, nx1 + 1)
    z = 0.5 * (x1f[1:] + x1f[:-1])
    dx2 = x2max / nx2
    x2v = (np.arange(nx2) + 0.5) * dx2
    zz, xx = np.meshgrid(z, x2v)  # (j, i)
    L = np.sqrt(((xx - xc) / xr) ** 2 + ((zz - zc) / zr) ** 2)
    temp = Ts - grav * zz / cp
    pres = p0 * (temp / Ts) ** (cp / Rd)
    temp = np.where(L <= 1.0, temp + dT * (np.cos(np.pi * L) + 1.0) / 2.0, temp)
    nv = 5
    w_int = np.zeros((nv, 1, nx2, nx1))
    w_int[0, 0] = pres / (Rd * temp)
    w_int[4, 0] = pres
    shape = _shape(nx1, nx2, 1, nv)
    w = _embed(shape, w_int, nx1, nx2, 1)
    u = _embed(shape, T.prim_to_cons(th, w_int), nx1, nx2, 1)
    bc = [BC_REFLECT] * 4 + [BC_PERIODIC] * 2
    cfg, x1f = make_config(nx1, nx2, 1, x1f, dx2, 1.0, th, bc, recon, rsolver,
                           implicit_flag=0, satadj=0, cfl=cfl)
    return Problem("straka2d", cfg, x1f, u, w, dict(tlim=900.0, out_dt=300.0, p0=p0, K=K))


def _solve_T(f, lo, hi, it=60):
    """Bisection of the increasing function f on [lo, hi] (arrays)."""
    lo, hi = np.array(lo, dtype=np.float64), np.array(hi, dtype=np.float64)
    for _ in range(it):
        mid = 0.5 * (lo + hi)
        up = f(mid) > 0.0
        hi = np.where(up, mid, hi)
        lo = np.where(up, lo, mid)
    return 0.5 * (lo + hi)


def bryan2d(nx1=200, nx2=400, x1max=10.0e3, x2max=20.0e3, Ts=289.85, p0=1.0e5, qt=0.0196,
            dT=2.0, xc=10.0e3, zc=2.0e3, xr=2.0e3, zr=2.0e3, grav=9.81, cfl=0.45,
            recon=RECON_PPM, rsolver=RS_LMARS, nsub=16):
    """The moist rising bubble of examples/2019-Li-snap/bryan.inp / bryan.cpp
    (Bryan and Fritsch 2002) on the earth-moist.yaml thermo (dry air, H2O
    vapour and liquid): a saturated reversible moist adiabat of total water
    qt from (Ts, p0) at the ground, and a virtual-temperature bubble of dT
    (cos^2 in the normalised distance L < 1) re-equilibrated at constant
    pressure and total water (bryan.cpp:103-155).  The adiabat keeps the
    moist static energy h + g z of the saturated parcel constant with
    hydrostatic pressure, integrated with nsub midpoint steps per cell from
    the ground to the first cell centre and on from centre to centre.
    Courant number 0.9 split over the two directions as in bubble2d;
    fifth-order horizontal reconstruction replaced by PPM."""
    th = T.moist(("H2O",), ice=False, grav=-grav)
    x1f = np.linspace(0.0, x1max, nx1 + 1)
    z = 0.5 * (x1f[1:] + x1f[:-1])
    dx2 = x2max / nx2
    x2v = (np.arange(nx2) + 0.5) * dx2

    def state(Tk, pk):
        qv, ql = T.sat_split(th, Tk, pk, qt)
        return np.array([qv, ql])

    def rho_of(Tk, pk):
        return pk / (th.rd * T.feps_of(th, state(Tk, pk)) * Tk)

    H0 = T.enthalpy(th, state(Ts, p0), Ts)

    def T_at(pk, zk, Tg):
        return _solve_T(lambda t: T.enthalpy(th, state(t, pk), t) - (H0 - grav * zk),
                        Tg - 30.0, Tg + 5.0)

    Tcol, pcol = np.empty(nx1), np.empty(nx1)
    Tk, pk, zk = Ts, p0, 0.0
    for i in range(nx1):
        h = (z[i] - zk) / nsub
        for _ in range(nsub):
            pm = pk - 0.5 * h * grav * rho_of(Tk, pk)
            Tm = T_at(pm, zk + 0.5 * h, Tk)
            pk = pk - h * grav * rho_of(Tm, pm)
            zk = zk + h
            Tk = T_at(pk, zk, Tk)
        Tcol[i], pcol[i] = Tk, pk
    Tt = np.broadcast_to(Tcol[None, :], (nx2, nx1)).copy()  # (j, i)
    pp = np.broadcast_to(pcol[None, :], (nx2, nx1)).copy()
    # virtual-temperature bubble at constant pressure and total water
    zz, xx = np.meshgrid(z, x2v)
    L = np.sqrt(((xx - xc) / xr) ** 2 + ((zz - zc) / zr) ** 2)
    inb = L < 1.0
    if inb.any():
        t0, p_ = Tt[inb], pp[inb]
        tv = t0 * T.feps_of(th, state(t0, p_)) * (1.0 + dT * np.cos(np.pi * L[inb] / 2.0) ** 2 / 300.0)
        Tt[inb] = _solve_T(lambda t: t * T.feps_of(th, state(t, p_)) - tv, t0, t0 + dT * Ts / 300.0)
    q = state(Tt, pp)
    rho = pp / (th.rd * T.feps_of(th, q) * Tt)
    nv = 5 + th.ny
    w_int = np.zeros((nv, 1, nx2, nx1))
    w_int[0, 0] = rho
    w_int[1, 0], w_int[2, 0] = q[0], q[1]
    w_int[4 + th.ny, 0] = pp
    shape = _shape(nx1, nx2, 1, nv)
    w = _embed(shape, w_int, nx1, nx2, 1)
    u = _embed(shape, T.prim_to_cons(th, w_int), nx1, nx2, 1)
    bc = [BC_REFLECT] * 4 + [BC_PERIODIC] * 2
    cfg, x1f = make_config(nx1, nx2, 1, x1f, dx2, 1.0, th, bc, recon, rsolver,
                           implicit_flag=0, satadj=1, cfl=cfl)
    return Problem("bryan2d", cfg, x1f, u, w,
                   dict(tlim=1000.0, out_dt=100.0, p0=p0, qt=qt))


def moist_profile(th, z, Ts=300.0, Ttop=200.0, ps=1.0e5, rh=0.8, zmoist=10.0e3,
                  nsub=16):
    """Horizontally uniform moist column at heights z (cell centres):
    T = max(Ts - g z / cp_d, Ttop); H2O at `rh` of saturation below zmoist and
    at min(q(zmoist), rh q_sat) above; hydrostatic pressure integrated in
    log p with the gas constant of the moist mixture.  Returns T, p, q_v."""
    g = -th.grav
    cpd = th.rd * th.gammad / (th.gammad - 1.0)
    gam = g / cpd
    imr = th.inv_mu_ratio_m1[0] if th.nvapor else 0.0
    rv = th.rd * (1.0 + imr)

    def temp(zz):
        return np.maximum(Ts - gam * zz, Ttop)

    def qv_rh(tt, pp):
        if not th.nvapor:
            return 0.0 * tt
        e = rh * T.svp(th, 0, tt)
        e = np.minimum(e, 0.5 * pp)
        return (e / rv) / ((pp - e) / th.rd + e / rv)

    # integrate ln p from the ground on a fine grid
    zs = np.concatenate([[0.0], z])
    lnp = np.log(ps)
    p_out = np.empty_like(z)
    q_out = np.empty_like(z)
    q10 = None
    zcur = 0.0
    for n, zt in enumerate(z):
        h = (zt - zcur) / nsub
        for _ in range(nsub):
            zm = zcur + 0.5 * h
            tm = temp(zm)
            pm = np.exp(lnp)
            qm = qv_rh(tm, pm)
            if q10 is not None and zm > zmoist:
                qm = min(qm, q10)
            rm = th.rd * (1.0 + imr * qm)
            lnp -= g * h / (rm * tm)
            zcur += h
        p_out[n] = np.exp(lnp)
        q = qv_rh(temp(zt), p_out[n])
        if zt <= zmoist:
            q10 = q
        elif q10 is not None:
            q = min(q, q10)
        q_out[n] = q
    return temp(z), p_out, q_out


def moist3d(nx1=128, nx2=256, nx3=256, x1max=16.0e3, x2max=64.0e3, x3max=64.0e3,
            seed=20240601, noise=0.1, noise_depth=1.0e3, implicit_flag=1,
            recon=RECON_PPM, rsolver=RS_HLLC, satadj=1, cfl=0.4, th=None, rh=0.8):
    """C2: 3-D moist convection LES initial state.  cfl as in bubble2d: the
    configuration's 0.8 split over the two horizontal directions (the
    implicit x1 direction is limited by |v| only).  rh: relative humidity of
    the moist layer (0.8 in the configuration; 1.0 makes the noise-cooled
    cells condense at the first adjustment)."""
    th = th or T.earth_moist()
    ny = th.ny
    nv = 5 + ny
    x1f = np.linspace(0.0, x1max, nx1 + 1)
    z = 0.5 * (x1f[1:] + x1f[:-1])
    temp, pres, qv = moist_profile(th, z, rh=rh)
    rng = np.random.Generator(np.random.PCG64(seed))
    dtn = rng.uniform(-noise, noise, size=(nx3, nx2, nx1))
    dtn *= (z < noise_depth)[None, None, :]
    tt = temp[None, None, :] + dtn
    q = np.zeros((max(ny, 1), nx3, nx2, nx1))
    if ny:
        q[0] = qv[None, None, :]
    feps = T.feps_of(th, q[:ny]) if ny else 1.0
    pp = np.broadcast_to(pres[None, None, :], tt.shape)
    rho = pp / (th.rd * feps * tt)
    w_int = np.zeros((nv, nx3, nx2, nx1))
    w_int[0] = rho
    for n in range(1, ny + 1):
        w_int[n] = q[n - 1]
    w_int[4 + ny] = pp
    shape = _shape(nx1, nx2, nx3, nv)
    u_int = T.prim_to_cons(th, w_int)
    u = _embed(shape, u_int, nx1, nx2, nx3)
    w = _embed(shape, w_int, nx1, nx2, nx3)
    bc = [BC_REFLECT, BC_REFLECT, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_PERIODIC]
    cfg, x1f = make_config(nx1, nx2, nx3, x1f, x2max / nx2, x3max / nx3, th, bc, recon,
                           rsolver, implicit_flag=implicit_flag, satadj=satadj, cfl=cfl)
    return Problem("C2-moist3d", cfg, x1f, u, w, dict(seed=seed))


def periodic_x1(nx1=48, nx2=8, nx3=4, x1max=4800.0, x2max=800.0, x3max=400.0, moist=False,
                v1=20.0, amp=0.02, seed=20240611, implicit_flag=1, recon=RECON_PPM,
                rsolver=RS_HLLC, cfl=0.4):
    """A box periodic in every direction and without gravity, for the cyclic
    implicit x1 solve (periodic_forward_backward.hpp): uniform 300 K,
    1e5 Pa air moving at v1 along x1, with a seeded density bump and seeded
    velocity noise of relative size amp; moist=True adds H2O vapour at a
    seeded mass fraction near 1e-3 and zero condensates (no saturation
    adjustment)."""
    th = T.earth_moist() if moist else T.dry()
    th.grav = 0.0
    ny = th.ny
    nv = 5 + ny
    x1f = np.linspace(0.0, x1max, nx1 + 1)
    z = 0.5 * (x1f[1:] + x1f[:-1])
    rng = np.random.Generator(np.random.PCG64(seed))
    shp = (nx3, nx2, nx1)
    bump = 1.0 + amp * np.exp(-((z - 0.3 * x1max) / (0.1 * x1max)) ** 2)
    w_int = np.zeros((nv,) + shp)
    q = np.zeros((max(ny, 1),) + shp)
    if ny:
        q[0] = 1.0e-3 * (1.0 + 0.2 * rng.uniform(-1.0, 1.0, shp))
    feps = T.feps_of(th, q[:ny]) if ny else 1.0
    pres = 1.0e5 * (1.0 + 0.1 * amp * rng.uniform(-1.0, 1.0, shp))
    w_int[0] = pres / (th.rd * feps * 300.0) * bump[None, None, :]
    for n in range(1, ny + 1):
        w_int[n] = q[n - 1]
    w_int[1 + ny] = v1 * (1.0 + amp * rng.uniform(-1.0, 1.0, shp))
    w_int[2 + ny] = v1 * amp * rng.uniform(-1.0, 1.0, shp)
    w_int[3 + ny] = v1 * amp * rng.uniform(-1.0, 1.0, shp)
    w_int[4 + ny] = pres
    shape = _shape(nx1, nx2, nx3, nv)
    u = _embed(shape, T.prim_to_cons(th, w_int), nx1, nx2, nx3)
    w = _embed(shape, w_int, nx1, nx2, nx3)
    bc = [BC_PERIODIC] * 6
    cfg, x1f = make_config(nx1, nx2, nx3, x1f, x2max / nx2, x3max / nx3, th, bc, recon,
                           rsolver, implicit_flag=implicit_flag, satadj=0, cfl=cfl)
    return Problem("periodic-x1", cfg, x1f, u, w, dict(seed=seed))


@dataclass
class ShellProblem:
    """A cubed-sphere shell: config, radial faces, conserved and primitive
    state (6, NV, nc3, nc2, nc1) with covariant momenta in u and
    contravariant velocities in w, ghost cells zero."""
    name: str
    cfg: ShellConfig
    x1f: np.ndarray
    u: np.ndarray
    w: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def nv(self):
        return 5 + self.cfg.thermo.ny

    def interior(self, a):
        ng = NGHOST
        n, nx1 = self.cfg.nside, self.cfg.nx1
        return a[..., ng:ng + n, ng:ng + n, ng:ng + nx1]


def shell_c3(nx1=64, nside=96, p_bot=100.0e5, p_top=0.1e5, t1bar=165.0, radius=7.1492e7,
             jet=5.0, nmodes=8, seed=20240607, implicit_flag=1, recon=RECON_PPM, cfl=0.4,
             th=None):
    """C3: dry H2-He shell (g = 24.79 m/s^2, mu = 2.3 g/mol).  Radial faces
    sit at pressures uniform in log p between p_bot and p_top on the dry
    adiabat T = 165 K (p / 1 bar)^(R/cp), mapped to heights by the
    hydrostatic relation dz = -cp dT / g of that adiabat; cell states follow
    the same adiabat in height.  The eastward wind U(lat) sums nmodes seeded
    cosine jets scaled to |U| <= jet; V = 0."""
    from . import cubed_sphere as cs
    th = th or T.giant_planet()
    g = -th.grav
    rd = th.rd
    kappa = (th.gammad - 1.0) / th.gammad
    cp = rd / kappa
    pf = np.exp(np.linspace(np.log(p_bot), np.log(p_top), nx1 + 1))
    tf = t1bar * (pf / 1.0e5) ** kappa
    t_bot = tf[0]
    zf = cp * (t_bot - tf) / g
    x1f = radius + zf
    x1v = 0.5 * (x1f[1:] + x1f[:-1])
    tv = t_bot - g * (x1v - radius) / cp
    pv = 1.0e5 * (tv / t1bar) ** (1.0 / kappa)
    rhov = pv / (rd * tv)
    rng = np.random.Generator(np.random.PCG64(seed))
    amp = rng.uniform(-1.0, 1.0, nmodes)
    amp *= jet / np.abs(amp).sum()
    n = nside + 2 * NGHOST
    nc1 = nx1 + 2 * NGHOST
    nv = 5
    w = np.zeros((6, nv, n, n, nc1))
    u = np.zeros_like(w)
    _, av = cs.panel_angles(nside)
    ing = slice(NGHOST, NGHOST + nside)
    X = np.tan(av[ing])[None, :]     # x2 (j), last axis
    Y = np.tan(av[ing])[:, None]     # x3 (k)
    X, Y = np.broadcast_arrays(X, Y)
    for p in range(6):
        bid = p + 1
        lat, lon = cs.latlon(bid, X, Y)
        U = sum(a * np.cos((2 * m + 1) * lat) for m, a in enumerate(amp))
        v2, v3 = cs.velocity_from_uv(bid, X, Y, U, np.zeros_like(U))
        sl = (p, slice(None), ing, ing, slice(NGHOST, NGHOST + nx1))
        wp = np.zeros((nv, nside, nside, nx1))
        wp[0] = rhov[None, None, :]
        wp[2] = v2[:, :, None]
        wp[3] = v3[:, :, None]
        wp[4] = pv[None, None, :]
        w[sl] = wp
        # PrimitiveToConserved with covariant momenta (patch 26)
        cth = cs.cos_theta(X, Y)[:, :, None]
        m1 = wp[1] * wp[0]
        m2 = wp[2] * wp[0]
        m3 = wp[3] * wp[0]
        m2, m3 = m2 + m3 * cth, m3 + m2 * cth
        up = np.zeros_like(wp)
        up[0] = wp[0]
        up[1], up[2], up[3] = m1, m2, m3
        up[4] = wp[4] / (th.gammad - 1.0) + 0.5 * (m1 * wp[1] + m2 * wp[2] + m3 * wp[3])
        u[sl] = up
    cfg = ShellConfig()
    cfg.nx1, cfg.nside = nx1, nside
    cfg.bc_x1[0], cfg.bc_x1[1] = BC_REFLECT, BC_REFLECT
    x1f = np.ascontiguousarray(x1f, dtype=np.float64)
    cfg.h_x1f = x1f.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cfg.recon, cfg.rsolver = recon, RS_HLLC
    cfg.implicit_flag, cfg.precision = implicit_flag, FP64
    cfg.cfl = cfl
    cfg.thermo = th
    return ShellProblem("C3-shell", cfg, x1f, u, w, dict(jet_amplitudes=amp, seed=seed))


def batch_c5(nblocks=48, seed=20240605, nz=(32, 256), nh=(16, 128), depth=16.0e3, dx=250.0,
             **kw):
    """C5: nblocks independent blocks of C2 physics (moist3d: PPM + HLLC,
    implicit x1, saturation adjustment) with vertical sizes nz and square
    horizontal sizes nh drawn log-uniformly from the seed; every block is
    depth deep with dx horizontal spacing.  Returns a list of Problems."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(nblocks):
        n1 = int(round(np.exp(rng.uniform(np.log(nz[0]), np.log(nz[1])))))
        n2 = int(round(np.exp(rng.uniform(np.log(nh[0]), np.log(nh[1])))))
        p = moist3d(nx1=n1, nx2=n2, nx3=n2, x1max=depth, x2max=n2 * dx, x3max=n2 * dx,
                    seed=seed + 1 + b, **kw)
        p.name = f"C5-block{b}-{n1}x{n2}x{n2}"
        out.append(p)
    return out

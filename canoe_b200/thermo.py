"""Thermodynamic parameter sets of the synthetic configurations.

Species data follow the reference's YAML files
(examples/2019-Li-snap/earth-moist.yaml, earth-dry.yaml, jup-thermo.yaml):
constant-cp species, condensates with zero molar volume, and the "ideal"
saturation vapour pressure p_sat = p3 exp[beta (1 - t3/T) - delta ln(T/t3)].
Consistency of that formula with constant heat capacities fixes the
condensate heat capacity cp_c = cp_v + delta R and the condensate internal
energy u_c(T) = cp_c T - beta R t3 (per mole, gases u = cv T), which is the
relation h0 = -(beta - delta) R T0 stated at earth-moist.yaml:29.
"""
import numpy as np

from ._abi import MAX_NY, MAX_VAPOR, Thermo

RGAS = 8.314462618  # J/mol/K
# atomic weights [g/mol]
AW = {"H": 1.008, "He": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999,
      "S": 32.06, "Ar": 39.948}


def molar_mass(comp):
    """kg/mol of a composition dict like {"O": 0.42, "N": 1.56, "Ar": 0.01}."""
    return sum(AW[e] * n for e, n in comp.items()) * 1e-3


MU_EARTH_DRY = molar_mass({"O": 0.42, "N": 1.56, "Ar": 0.01})  # earth-dry.yaml
MU_H2O = molar_mass({"H": 2, "O": 1})
MU_NH3 = molar_mass({"N": 1, "H": 3})

# "ideal" SVP parameters: jup-thermo.yaml:100-116 / earth-moist.yaml:37
SVP = {
    "H2O": dict(t3=273.16, p3=611.7, beta_l=24.845, delta_l=4.986, beta_s=22.98, delta_s=0.52),
    "NH3": dict(t3=195.4, p3=6060., beta_l=20.08, delta_l=5.62, beta_s=20.64, delta_s=1.43),
}
# vapour molar cp [J/mol/K]: earth-moist.yaml (H2O 21.1, consistent with
# its liquid cp = 21.1 + 4.986 R); jup-thermo.yaml NH3 37.4
CP_VAPOR = {"H2O": 21.1, "NH3": 37.4}


def _new(ny, nvapor, rd, gammad, grav):
    th = Thermo()
    th.ny, th.nvapor = ny, nvapor
    th.rd, th.gammad, th.grav = rd, gammad, grav
    for v in range(MAX_VAPOR):
        th.liq_slot[v] = -1
        th.ice_slot[v] = -1
    return th


def dry(mu=MU_EARTH_DRY, gammad=1.4, grav=-9.81):
    """Dry ideal gas (earth-dry.yaml: cv_R = 2.5, i.e. gamma = 1.4)."""
    return _new(0, 0, RGAS / mu, gammad, grav)


def moist(vapors=("H2O",), ice=True, mu=MU_EARTH_DRY, gammad=1.4, grav=-9.81):
    """Dry air plus condensable vapors, each with a liquid and (optionally) an
    ice phase.  Slots: vapors 1..nv, then the liquids, then the ices."""
    nv = len(vapors)
    ny = nv * (3 if ice else 2)  # vapour + liquid (+ ice) per family
    assert ny <= MAX_NY and nv <= MAX_VAPOR
    rd = RGAS / mu
    th = _new(ny, nv, rd, gammad, grav)
    cvd = rd / (gammad - 1.0)
    mus = {"H2O": MU_H2O, "NH3": MU_NH3}
    for v, name in enumerate(vapors):
        m = mus[name]
        p = SVP[name]
        cp_v = CP_VAPOR[name]
        lslot = 1 + nv + v
        sslot = 1 + 2 * nv + v if ice else -1
        th.liq_slot[v], th.ice_slot[v] = lslot, sslot
        th.t3[v], th.p3[v] = p["t3"], p["p3"]
        th.beta_l[v], th.delta_l[v] = p["beta_l"], p["delta_l"]
        th.beta_s[v], th.delta_s[v] = p["beta_s"], p["delta_s"]
        # vapour: cv = cp - R per mole
        th.cv_ratio_m1[v] = ((cp_v - RGAS) / m) / cvd - 1.0
        th.inv_mu_ratio_m1[v] = mu / m - 1.0
        # liquid: cp_c = cp_v + delta R, u0 = -beta R t3 (per mole)
        cpl = cp_v + p["delta_l"] * RGAS
        th.cv_ratio_m1[lslot - 1] = (cpl / m) / cvd - 1.0
        th.u0[lslot - 1] = -p["beta_l"] * RGAS * p["t3"] / m
        if ice:
            cps = cp_v + p["delta_s"] * RGAS
            th.cv_ratio_m1[sslot - 1] = (cps / m) / cvd - 1.0
            th.u0[sslot - 1] = -p["beta_s"] * RGAS * p["t3"] / m
    return th


def earth_moist():
    """C2 / C5: dry air + H2O vapour, liquid and ice (ny = 3)."""
    return moist(("H2O",), ice=True)


def earth_water_ammonia():
    """C4 learned-warm-start training thermo: H2O and NH3 with liquid and
    ice phases (ny = 6), on the earth-dry air of earth-moist.yaml."""
    return moist(("H2O", "NH3"), ice=True)


def giant_planet(grav=-24.79, mu=2.3e-3, gammad=1.4):
    """C3: dry H2-He shell, mean molecular weight 2.3 g/mol."""
    return dry(mu=mu, gammad=gammad, grav=grav)


def copy(th):
    out = Thermo()
    ctypes_copy = bytes(th)
    import ctypes
    ctypes.memmove(ctypes.addressof(out), ctypes_copy, ctypes.sizeof(Thermo))
    return out


# ---------------------------------------------------------------------------
# numpy restatement of the EOS used by the problem generators (host side)

def gamma_of(th, q):
    """mixture gamma from mass fractions q[n-1] for slots 1..ny (eos.hpp:48-67)."""
    fsig = np.ones_like(q[0]) if th.ny else 1.0
    feps = np.ones_like(q[0]) if th.ny else 1.0
    for n in range(1, th.ny + 1):
        fsig = fsig + q[n - 1] * th.cv_ratio_m1[n - 1]
        if n <= th.nvapor:
            feps = feps + q[n - 1] * th.inv_mu_ratio_m1[n - 1]
        else:
            feps = feps - q[n - 1]
    return 1.0 + (th.gammad - 1.0) * feps / fsig


def feps_of(th, q):
    feps = 1.0
    for n in range(1, th.ny + 1):
        if n <= th.nvapor:
            feps = feps + q[n - 1] * th.inv_mu_ratio_m1[n - 1]
        else:
            feps = feps - q[n - 1]
    return feps


def prim_to_cons(th, w):
    """w: (NV, ...) primitive -> conserved (snapy "W->U", restated)."""
    ny = th.ny
    ivx = 1 + ny
    u = np.empty_like(w)
    rho = w[0]
    q = w[1:1 + ny]
    qsum = q.sum(axis=0) if ny else 0.0
    u[0] = rho * (1.0 - qsum)
    for n in range(1, ny + 1):
        u[n] = rho * w[n]
    v1, v2, v3 = w[ivx], w[ivx + 1], w[ivx + 2]
    u[ivx], u[ivx + 1], u[ivx + 2] = rho * v1, rho * v2, rho * v3
    lat = 0.0
    for n in range(th.nvapor + 1, ny + 1):
        lat = lat + rho * w[n] * th.u0[n - 1]
    gamma = gamma_of(th, q)
    u[ivx + 3] = w[ivx + 3] / (gamma - 1.0) + lat + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3)
    return u


def svp(th, v, T, phase="auto"):
    t3, p3 = th.t3[v], th.p3[v]
    liquid = T >= t3 if phase == "auto" else np.full_like(T, phase == "liquid", dtype=bool)
    beta = np.where(liquid, th.beta_l[v], th.beta_s[v])
    delta = np.where(liquid, th.delta_l[v], th.delta_s[v])
    return p3 * np.exp(beta * (1.0 - t3 / T) - delta * np.log(T / t3))


# ---------------------------------------------------------------------------
# saturated equilibrium of one condensable family (vapour slot 1, liquid slot
# 2, no ice), host side, for the moist problem generators

def sat_split(th, T, p, qt, v=0):
    """Vapour and liquid mass fractions of a parcel with total water mass
    fraction qt in equilibrium at (T, p): the vapour pressure at saturation
    where water condenses, all vapour below it.  With rho q_v R_v T = e_s and
    rho = p / (R_d f_eps T): q_v = (1 - q_t) e_s / ((1 + imr) (p - e_s))."""
    phase = "liquid" if th.ice_slot[v] < 0 else "auto"
    es = svp(th, v, np.asarray(T, dtype=np.float64), phase)
    imr = th.inv_mu_ratio_m1[v]
    qs = (1.0 - qt) * es / ((1.0 + imr) * (p - es))
    qv = np.minimum(qs, qt)
    return qv, qt - qv


def enthalpy(th, q, T):
    """Specific enthalpy e + p / rho of the mixture with mass fractions q
    (slots 1..ny): e = c_v,d (q_d + sum q_n (1 + cv_ratio_m1)) T + sum q_n u0_n,
    p / rho = R_d f_eps T (the energy of prim_to_cons per unit mass)."""
    cvd = th.rd / (th.gammad - 1.0)
    qsum = sum(q[n] for n in range(th.ny))
    cvs = 1.0 - qsum
    lat = 0.0
    for n in range(th.ny):
        cvs = cvs + q[n] * (1.0 + th.cv_ratio_m1[n])
        lat = lat + q[n] * th.u0[n]
    return cvd * cvs * T + lat + th.rd * feps_of(th, q) * T


def theta_e(th, q, T, p, p0=1.0e5, v=0):
    """Equivalent potential temperature, Emanuel (1994) eq. 4.5.11 in the
    reference's form (src/snap/thermodynamics/atm_thermodynamics.hpp:43-98):
    T (p0 / p_d)^(R_d q_d / c_pt) rh^(-R_v q_v / c_pt) exp(L_v q_v / (c_pt T)),
    c_pt = c_pd q_d + c_l q_t, with this thermo's latent heat
    L_v = R_v (beta_l t3 - delta_l T) and liquid c_l."""
    qv = q[v]
    ql = q[th.liq_slot[v] - 1]
    qd = 1.0 - sum(q[n] for n in range(th.ny))
    cvd = th.rd / (th.gammad - 1.0)
    cpd = th.rd + cvd
    rv = th.rd * (1.0 + th.inv_mu_ratio_m1[v])
    cl = cvd * (1.0 + th.cv_ratio_m1[th.liq_slot[v] - 1])
    lv = rv * (th.beta_l[v] * th.t3[v] - th.delta_l[v] * T)
    xd, xv = qd / th.rd, qv / rv  # moles per unit mass times R
    pd = xd / (xd + xv) * p
    e = xv / (xd + xv) * p
    phase = "liquid" if th.ice_slot[v] < 0 else "auto"
    rh = e / svp(th, v, np.asarray(T, dtype=np.float64), phase)
    cpt = cpd * qd + cl * (qv + ql)
    return (T * (p0 / pd) ** (th.rd * qd / cpt) * rh ** (-rv * qv / cpt)
            * np.exp(lv * qv / (cpt * T)))

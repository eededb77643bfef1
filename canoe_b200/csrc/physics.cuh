// physics.cuh -- device-side pointwise physics of the dynamical core:
// mixture gamma, sound speed, PLM / PPM reconstruction of one cell, and the
// LMARS / HLLC Riemann fluxes of one face.  Templated on the arithmetic type
// R (double for the FP64 path, float for the FP32-on-perturbation path) and
// on NY, the number of mass-fraction slots, so that every per-cell array
// lives in registers.
#pragma once

#include <cuda_runtime.h>

#include "../../include/canoe_b200.h"

namespace cb {

constexpr int NG = CANOE_NGHOST;
// Athena++ TINY_NUMBER, the HLLC wave-speed floor (hllc_transform.cpp:152)
constexpr double TINY_NUMBER = 1.0e-20;

template <int NY>
struct Slots {
  static constexpr int IVX = 1 + NY, IVY = 2 + NY, IVZ = 3 + NY, IPR = 4 + NY,
                       NV = 5 + NY;
};

// Division in the FP32 perturbation solvers: the fast reciprocal-based
// __fdividef (2 ulp) for R = float, exact for R = double.  The FP32 path's
// stated error (relative 1e-5 on fluxes) is far above it.
constexpr bool kFastDiv = true;
template <typename R>
__device__ __forceinline__ R pdiv(R a, R b) {
  if constexpr (sizeof(R) == 4 && kFastDiv) return __fdividef(a, b);
  else return a / b;
}

// Mixture adiabatic index from mass fractions w[1..NY]
// (canoe src/interface/eos.hpp:48-67, rho = 1).
template <typename R, int NY>
__device__ __forceinline__ R get_gamma(const canoe_thermo_t &th, const R *w) {
  R fsig = R(1), feps = R(1);
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    fsig += w[n] * R(th.cv_ratio_m1[n - 1]);
    if (n <= th.nvapor)
      feps += w[n] * R(th.inv_mu_ratio_m1[n - 1]);
    else
      feps -= w[n];
  }
  return R(1) + R(th.gammad - 1.) * feps / fsig;
}

// EquationOfState::SoundSpeed (canoe src/snap/eos/ideal_moist_hydro.cpp:87-91)
template <typename R, int NY>
__device__ __forceinline__ R sound_speed(const canoe_thermo_t &th, const R *w) {
  R gamma = get_gamma<R, NY>(th, w);
  return sqrt(gamma * w[Slots<NY>::IPR] / w[0]);
}

// ---------------------------------------------------------------------------
// Reconstruction of one cell: returns the values at its left (wL) and right
// (wR) faces.  Interface states follow as wl(f) = wR(f-1), wr(f) = wL(f).

// PPM slope, Colella & Woodward (1984) eq. 1.7-1.8 (monotonized central)
template <typename R>
__device__ __forceinline__ R ppm_slope(R qm, R q0, R qp) {
  R dwl = q0 - qm, dwr = qp - q0;
  if (dwl * dwr <= R(0)) return R(0);
  R dwc = R(0.5) * (qp - qm);
  R lim = fmin(fabs(dwc), fmin(R(2) * fabs(dwl), R(2) * fabs(dwr)));
  return copysign(lim, dwc);
}

// PPM interface value between cells a and b (eq. 1.6) from their values
// and limited slopes
template <typename R>
__device__ __forceinline__ R ppm_face(R qa, R qb, R dma, R dmb) {
  constexpr R sixth = R(1) / R(6);
  return R(0.5) * (qa + qb) - (dmb - dma) * sixth;
}

// the eq. 1.10 parabola limiter of CW84 on cell value q0 and its
// interface values wL, wR
template <typename R>
__device__ __forceinline__ void ppm_limit(R q0, R &wL, R &wR) {
  if ((wR - q0) * (q0 - wL) <= R(0)) {
    wL = q0;
    wR = q0;
  } else {
    R d = wR - wL;
    R m6 = R(6) * (q0 - R(0.5) * (wL + wR));
    if (d * m6 > d * d)
      wL = R(3) * q0 - R(2) * wR;
    else if (-d * d > d * m6)
      wR = R(3) * q0 - R(2) * wL;
  }
}

// PPM face values of cell c from cells c-2..c+2, uniform spacing: eq. 1.6
// face interpolation and the eq. 1.10 parabola limiter of CW84.
template <typename R>
__device__ __forceinline__ void ppm_cell(R qmm, R qm, R q0, R qp, R qpp, R &wL,
                                         R &wR) {
  R dm_m = ppm_slope(qmm, qm, q0);
  R dm_0 = ppm_slope(qm, q0, qp);
  R dm_p = ppm_slope(q0, qp, qpp);
  wL = ppm_face(qm, q0, dm_m, dm_0);
  wR = ppm_face(q0, qp, dm_0, dm_p);
  ppm_limit(q0, wL, wR);
}

// PLM with the van Leer (1979) harmonic-mean limiter, uniform spacing.
template <typename R>
__device__ __forceinline__ void plm_cell(R qm, R q0, R qp, R &wL, R &wR) {
  R dwl = q0 - qm, dwr = qp - q0;
  R dw2 = dwl * dwr;
  R dwm = dw2 > R(0) ? R(2) * dw2 / (dwl + dwr) : R(0);
  wR = q0 + R(0.5) * dwm;
  wL = q0 - R(0.5) * dwm;
}

// PLM, van Leer limiter, on a nonuniform grid (cell centres xv, faces xf).
template <typename R>
__device__ __forceinline__ void plm_cell_nu(R qm, R q0, R qp, R xvm, R xv0,
                                            R xvp, R xfl, R xfr, R &wL, R &wR) {
  R gl = (q0 - qm) / (xv0 - xvm);
  R gr = (qp - q0) / (xvp - xv0);
  R g2 = gl * gr;
  R g = g2 > R(0) ? R(2) * g2 / (gl + gr) : R(0);
  wR = q0 + g * (xfr - xv0);
  wL = q0 - g * (xv0 - xfl);
}

// ---------------------------------------------------------------------------
// Riemann solvers.  wli, wri, flx are in variable-slot order; DIR = 0, 1, 2
// picks the normal velocity slot ivx = IVX + DIR.

// LMARS (Chen et al. 2013): canoe src/snap/riemann/lmars.cpp:19-85.  The
// kinetic term uses the identity lowering of Cartesian coordinates (the
// reference indexes vec_lower's 3-element result with the variable slot).
template <typename R, int NY, int DIR>
__device__ __forceinline__ void lmars(const canoe_thermo_t &th, const R *wli,
                                      const R *wri, R *flx) {
  using S = Slots<NY>;
  constexpr int ivx = S::IVX + DIR;
  constexpr int ivy = S::IVX + (DIR + 1) % 3;
  constexpr int ivz = S::IVX + (DIR + 2) % 3;
  constexpr int ipr = S::IPR;
  R kappal = R(1) / (get_gamma<R, NY>(th, wli) - R(1));
  R kappar = R(1) / (get_gamma<R, NY>(th, wri) - R(1));
  R hl = wli[ipr] / wli[0] * (kappal + R(1)) +
         R(0.5) * (wli[ivx] * wli[ivx] + wli[ivy] * wli[ivy] + wli[ivz] * wli[ivz]);
  R hr = wri[ipr] / wri[0] * (kappar + R(1)) +
         R(0.5) * (wri[ivx] * wri[ivx] + wri[ivy] * wri[ivy] + wri[ivz] * wri[ivz]);
  R rhobar = R(0.5) * (wli[0] + wri[0]);
  R cbar = sqrt(R(0.5) * (R(1) + (R(1) / kappar + R(1) / kappal) / R(2)) *
                (wli[ipr] + wri[ipr]) / rhobar);
  R pbar = R(0.5) * (wli[ipr] + wri[ipr]) +
           R(0.5) * (rhobar * cbar) * (wli[ivx] - wri[ivx]);
  R ubar = R(0.5) * (wli[ivx] + wri[ivx]) +
           R(0.5) / (rhobar * cbar) * (wli[ipr] - wri[ipr]);
  R rdl = R(1), rdr = R(1);
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    rdl -= wli[n];
    rdr -= wri[n];
  }
  const bool up = ubar > R(0);
  // upwind side (lmars.cpp:69-83)
  R ws[S::NV];
#pragma unroll
  for (int n = 0; n < S::NV; ++n) ws[n] = up ? wli[n] : wri[n];
  R rd = up ? rdl : rdr;
  R h = up ? hl : hr;
  flx[0] = ubar * ws[0] * rd;
#pragma unroll
  for (int n = 1; n <= NY; ++n) flx[n] = ubar * ws[0] * ws[n];
  flx[ivx] = ubar * ws[0] * ws[ivx] + pbar;
  flx[ivy] = ubar * ws[0] * ws[ivy];
  flx[ivz] = ubar * ws[0] * ws[ivz];
  flx[ipr] = ubar * ws[0] * h;
}

// HLLC (Toro 2009, ch. 10): canoe src/snap/riemann/hllc_transform.cpp:
// 25-233.  COVKE: the x1 problem on a cubed-sphere panel, whose kinetic
// energy is contravariant . covariant velocity with the cell's cosine
// ke_cth (hllc_transform.cpp:92-101); the Cartesian branch otherwise.
template <typename R, int NY, int DIR, bool COVKE = false>
__device__ __forceinline__ void hllc(const canoe_thermo_t &th, const R *wl,
                                     const R *wr, R *flx, R ke_cth = R(0)) {
  using S = Slots<NY>;
  constexpr int IVX = S::IVX, IVY = S::IVY, IVZ = S::IVZ, IPR = S::IPR;
  constexpr int ivx = IVX + DIR;
  constexpr int ivy = IVX + (DIR + 1) % 3;
  constexpr int ivz = IVX + (DIR + 2) % 3;
  R wli[S::NV], wri[S::NV];
  // rotate into the face frame: slot IVX holds the normal component
  wli[0] = wl[0];
  wri[0] = wr[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    wli[n] = wl[n];
    wri[n] = wr[n];
  }
  wli[IVX] = wl[ivx];
  wli[IVY] = wl[ivy];
  wli[IVZ] = wl[ivz];
  wri[IVX] = wr[ivx];
  wri[IVY] = wr[ivy];
  wri[IVZ] = wr[ivz];
  wli[IPR] = wl[IPR];
  wri[IPR] = wr[IPR];

  R gammal = get_gamma<R, NY>(th, wli);
  R kappal = R(1) / (gammal - R(1));
  R gammar = get_gamma<R, NY>(th, wri);
  R kappar = R(1) / (gammar - R(1));
  R cl = sqrt(gammal * wli[IPR] / wli[0]);
  R cr = sqrt(gammar * wri[IPR] / wri[0]);
  R KE_l, KE_r;
  if constexpr (COVKE) {
    R vy = wli[IVY] + wli[IVZ] * ke_cth, vz = wli[IVZ] + wli[IVY] * ke_cth;
    KE_l = R(0.5) * wli[0] * (wli[IVX] * wli[IVX] + wli[IVY] * vy + wli[IVZ] * vz);
    vy = wri[IVY] + wri[IVZ] * ke_cth;
    vz = wri[IVZ] + wri[IVY] * ke_cth;
    KE_r = R(0.5) * wri[0] * (wri[IVX] * wri[IVX] + wri[IVY] * vy + wri[IVZ] * vz);
  } else {
    KE_l = R(0.5) * wli[0] * (wli[IVX] * wli[IVX] + wli[IVY] * wli[IVY] + wli[IVZ] * wli[IVZ]);
    KE_r = R(0.5) * wri[0] * (wri[IVX] * wri[IVX] + wri[IVY] * wri[IVY] + wri[IVZ] * wri[IVZ]);
  }
  R el = wli[IPR] * kappal + KE_l;
  R er = wri[IPR] * kappar + KE_r;
  R rhoa = R(.5) * (wli[0] + wri[0]);
  R ca = R(.5) * (cl + cr);
  R pmid = R(.5) * (wli[IPR] + wri[IPR] + (wli[IVX] - wri[IVX]) * rhoa * ca);
  R ql = (pmid <= wli[IPR])
             ? R(1)
             : sqrt(R(1) + (gammal + R(1)) / (R(2) * gammal) * (pmid / wli[IPR] - R(1)));
  R qr = (pmid <= wri[IPR])
             ? R(1)
             : sqrt(R(1) + (gammar + R(1)) / (R(2) * gammar) * (pmid / wri[IPR] - R(1)));
  R al = wli[IVX] - cl * ql;
  R ar = wri[IVX] + cr * qr;
  R bp = ar > R(0) ? ar : R(TINY_NUMBER);
  R bm = al < R(0) ? al : -R(TINY_NUMBER);
  R vxl = wli[IVX] - al;
  R vxr = wri[IVX] - ar;
  R tl = wli[IPR] + vxl * wli[0] * wli[IVX];
  R tr = wri[IPR] + vxr * wri[0] * wri[IVX];
  R ml = wli[0] * vxl;
  R mr = -(wri[0] * vxr);
  R am = (tl - tr) / (ml + mr);
  R cp = (ml * tr + mr * tl) / (ml + mr);
  cp = cp > R(0) ? cp : R(0);
  vxl = wli[IVX] - bm;
  vxr = wri[IVX] - bp;
  R rdl = R(1), rdr = R(1);
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    rdl -= wli[n];
    rdr -= wri[n];
  }
  R sl, sr, sm;
  if (am >= R(0)) {
    sl = am / (am - bm);
    sr = R(0);
    sm = -bm / (am - bm);
  } else {
    sl = R(0);
    sr = -am / (bp - am);
    sm = bp / (bp - am);
  }
  R f[S::NV];
  f[0] = sl * (wli[0] * vxl * rdl) + sr * (wri[0] * vxr * rdr);
#pragma unroll
  for (int n = 1; n <= NY; ++n)
    f[n] = sl * (wli[0] * wli[n] * vxl) + sr * (wri[0] * wri[n] * vxr);
  f[IVX] = sl * (wli[0] * wli[IVX] * vxl + wli[IPR]) +
           sr * (wri[0] * wri[IVX] * vxr + wri[IPR]) + sm * cp;
  f[IVY] = sl * (wli[0] * wli[IVY] * vxl) + sr * (wri[0] * wri[IVY] * vxr);
  f[IVZ] = sl * (wli[0] * wli[IVZ] * vxl) + sr * (wri[0] * wri[IVZ] * vxr);
  f[IPR] = sl * (el * vxl + wli[IPR] * wli[IVX]) +
           sr * (er * vxr + wri[IPR] * wri[IVX]) + sm * cp * am;
  flx[0] = f[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) flx[n] = f[n];
  // rotate back: f[IVX] is the normal component
  flx[ivx] = f[IVX];
  flx[ivy] = f[IVY];
  flx[ivz] = f[IVZ];
  flx[IPR] = f[IPR];
}

template <typename R, int NY, int RS, int DIR>
__device__ __forceinline__ void riemann(const canoe_thermo_t &th, const R *wl,
                                        const R *wr, R *flx) {
  if constexpr (RS == CANOE_RSOLVER_LMARS)
    lmars<R, NY, DIR>(th, wl, wr, flx);
  else
    hllc<R, NY, DIR>(th, wl, wr, flx);
}


// ---------------------------------------------------------------------------
// Perturbation form of the Riemann solvers for the FP32 path.  The pressure
// slot of wl / wr holds p' = p - pref, with pref the FP64 hydrostatic
// reference pressure at the face (the same on both sides).  The returned
// normal-momentum flux excludes pref: F_ivx(p) = F'_ivx + pref exactly for
// LMARS and, since sl + sr + sm = 1, for HLLC.  Absolute pressure enters only
// where the solvers need it in relative terms (sound speeds, enthalpy).

template <typename R, int NY, int DIR>
__device__ __forceinline__ void lmars_pert(const canoe_thermo_t &th, const R *wli,
                                           const R *wri, R pref, R *flx) {
  using S = Slots<NY>;
  constexpr int ivx = S::IVX + DIR;
  constexpr int ivy = S::IVX + (DIR + 1) % 3;
  constexpr int ivz = S::IVX + (DIR + 2) % 3;
  constexpr int ipr = S::IPR;
  const R pl = pref + wli[ipr], pr = pref + wri[ipr];
  R kappal = pdiv(R(1), get_gamma<R, NY>(th, wli) - R(1));
  R kappar = pdiv(R(1), get_gamma<R, NY>(th, wri) - R(1));
  R hl = pdiv(pl, wli[0]) * (kappal + R(1)) +
         R(0.5) * (wli[ivx] * wli[ivx] + wli[ivy] * wli[ivy] + wli[ivz] * wli[ivz]);
  R hr = pdiv(pr, wri[0]) * (kappar + R(1)) +
         R(0.5) * (wri[ivx] * wri[ivx] + wri[ivy] * wri[ivy] + wri[ivz] * wri[ivz]);
  R rhobar = R(0.5) * (wli[0] + wri[0]);
  R cbar = sqrt(pdiv(R(0.5) * (R(1) + (pdiv(R(1), kappar) + pdiv(R(1), kappal)) / R(2)) * (pl + pr), rhobar));
  // pbar - pref and ubar from pressure differences only
  R pbar = R(0.5) * (wli[ipr] + wri[ipr]) + R(0.5) * (rhobar * cbar) * (wli[ivx] - wri[ivx]);
  R ubar = R(0.5) * (wli[ivx] + wri[ivx]) + pdiv(R(0.5), rhobar * cbar) * (wli[ipr] - wri[ipr]);
  R rdl = R(1), rdr = R(1);
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    rdl -= wli[n];
    rdr -= wri[n];
  }
  const bool up = ubar > R(0);
  R ws[S::NV];
#pragma unroll
  for (int n = 0; n < S::NV; ++n) ws[n] = up ? wli[n] : wri[n];
  R rd = up ? rdl : rdr;
  R h = up ? hl : hr;
  flx[0] = ubar * ws[0] * rd;
#pragma unroll
  for (int n = 1; n <= NY; ++n) flx[n] = ubar * ws[0] * ws[n];
  flx[ivx] = ubar * ws[0] * ws[ivx] + pbar;
  flx[ivy] = ubar * ws[0] * ws[ivy];
  flx[ivz] = ubar * ws[0] * ws[ivz];
  flx[ipr] = ubar * ws[0] * h;
}

// COVKE: the covariant kinetic energy of the x1 problem on a cubed-sphere
// panel, as in hllc()
template <typename R, int NY, int DIR, bool COVKE = false>
__device__ __forceinline__ void hllc_pert(const canoe_thermo_t &th, const R *wl, const R *wr,
                                          R pref, R *flx, R ke_cth = R(0)) {
  using S = Slots<NY>;
  constexpr int IVX = S::IVX, IVY = S::IVY, IVZ = S::IVZ, IPR = S::IPR;
  constexpr int ivx = IVX + DIR;
  constexpr int ivy = IVX + (DIR + 1) % 3;
  constexpr int ivz = IVX + (DIR + 2) % 3;
  R wli[S::NV], wri[S::NV];
  wli[0] = wl[0];
  wri[0] = wr[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    wli[n] = wl[n];
    wri[n] = wr[n];
  }
  wli[IVX] = wl[ivx];
  wli[IVY] = wl[ivy];
  wli[IVZ] = wl[ivz];
  wri[IVX] = wr[ivx];
  wri[IVY] = wr[ivy];
  wri[IVZ] = wr[ivz];
  const R dpl = wl[IPR], dpr = wr[IPR];     // p' on each side
  const R pl = pref + dpl, pr = pref + dpr;  // absolute, for relative uses
  R gammal = get_gamma<R, NY>(th, wli);
  R kappal = pdiv(R(1), gammal - R(1));
  R gammar = get_gamma<R, NY>(th, wri);
  R kappar = pdiv(R(1), gammar - R(1));
  R cl = sqrt(pdiv(gammal * pl, wli[0]));
  R cr = sqrt(pdiv(gammar * pr, wri[0]));
  R KE_l, KE_r;
  if constexpr (COVKE) {
    R vy = wli[IVY] + wli[IVZ] * ke_cth, vz = wli[IVZ] + wli[IVY] * ke_cth;
    KE_l = R(0.5) * wli[0] * (wli[IVX] * wli[IVX] + wli[IVY] * vy + wli[IVZ] * vz);
    vy = wri[IVY] + wri[IVZ] * ke_cth;
    vz = wri[IVZ] + wri[IVY] * ke_cth;
    KE_r = R(0.5) * wri[0] * (wri[IVX] * wri[IVX] + wri[IVY] * vy + wri[IVZ] * vz);
  } else {
    KE_l = R(0.5) * wli[0] * (wli[IVX] * wli[IVX] + wli[IVY] * wli[IVY] + wli[IVZ] * wli[IVZ]);
    KE_r = R(0.5) * wri[0] * (wri[IVX] * wri[IVX] + wri[IVY] * wri[IVY] + wri[IVZ] * wri[IVZ]);
  }
  R el = pl * kappal + KE_l;
  R er = pr * kappar + KE_r;
  R rhoa = R(.5) * (wli[0] + wri[0]);
  R ca = R(.5) * (cl + cr);
  R dpmid = R(.5) * (dpl + dpr + (wli[IVX] - wri[IVX]) * rhoa * ca);
  R pmid = pref + dpmid;
  R ql = (dpmid <= dpl) ? R(1) : sqrt(R(1) + pdiv(gammal + R(1), R(2) * gammal) * (pdiv(pmid, pl) - R(1)));
  R qr = (dpmid <= dpr) ? R(1) : sqrt(R(1) + pdiv(gammar + R(1), R(2) * gammar) * (pdiv(pmid, pr) - R(1)));
  R al = wli[IVX] - cl * ql;
  R ar = wri[IVX] + cr * qr;
  R bp = ar > R(0) ? ar : R(TINY_NUMBER);
  R bm = al < R(0) ? al : -R(TINY_NUMBER);
  R vxl = wli[IVX] - al;
  R vxr = wri[IVX] - ar;
  R tl = dpl + vxl * wli[0] * wli[IVX];  // minus pref
  R tr = dpr + vxr * wri[0] * wri[IVX];
  R ml = wli[0] * vxl;
  R mr = -(wri[0] * vxr);
  R am = pdiv(tl - tr, ml + mr);
  R dcp = pdiv(ml * tr + mr * tl, ml + mr);  // contact pressure minus pref
  dcp = dcp > -pref ? dcp : -pref;
  vxl = wli[IVX] - bm;
  vxr = wri[IVX] - bp;
  R rdl = R(1), rdr = R(1);
#pragma unroll
  for (int n = 1; n <= NY; ++n) {
    rdl -= wli[n];
    rdr -= wri[n];
  }
  R sl, sr, sm;
  if (am >= R(0)) {
    sl = pdiv(am, am - bm);
    sr = R(0);
    sm = pdiv(-bm, am - bm);
  } else {
    sl = R(0);
    sr = pdiv(-am, bp - am);
    sm = pdiv(bp, bp - am);
  }
  R f[S::NV];
  f[0] = sl * (wli[0] * vxl * rdl) + sr * (wri[0] * vxr * rdr);
#pragma unroll
  for (int n = 1; n <= NY; ++n)
    f[n] = sl * (wli[0] * wli[n] * vxl) + sr * (wri[0] * wri[n] * vxr);
  f[IVX] = sl * (wli[0] * wli[IVX] * vxl + dpl) + sr * (wri[0] * wri[IVX] * vxr + dpr) + sm * dcp;
  f[IVY] = sl * (wli[0] * wli[IVY] * vxl) + sr * (wri[0] * wri[IVY] * vxr);
  f[IVZ] = sl * (wli[0] * wli[IVZ] * vxl) + sr * (wri[0] * wri[IVZ] * vxr);
  f[IPR] = sl * (el * vxl + pl * wli[IVX]) + sr * (er * vxr + pr * wri[IVX]) +
           sm * (pref + dcp) * am;
  flx[0] = f[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) flx[n] = f[n];
  flx[ivx] = f[IVX];
  flx[ivy] = f[IVY];
  flx[ivz] = f[IVZ];
  flx[IPR] = f[IPR];
}

template <typename R, int NY, int RS, int DIR>
__device__ __forceinline__ void riemann_pert(const canoe_thermo_t &th, const R *wl,
                                             const R *wr, R pref, R *flx) {
  if constexpr (RS == CANOE_RSOLVER_LMARS)
    lmars_pert<R, NY, DIR>(th, wl, wr, pref, flx);
  else
    hllc_pert<R, NY, DIR>(th, wl, wr, pref, flx);
}

// ---------------------------------------------------------------------------
// Ideal-moist EOS (snapy "U->W" / "W->U", restated): conserved u -> prim w.
template <int NY>
__device__ __forceinline__ void cons_to_prim(const canoe_thermo_t &th,
                                             const double *u, double *w) {
  using S = Slots<NY>;
  double rho = u[0];
#pragma unroll
  for (int n = 1; n <= NY; ++n) rho += u[n];
  double di = 1. / rho;
  w[0] = rho;
#pragma unroll
  for (int n = 1; n <= NY; ++n) w[n] = u[n] * di;
  double m1 = u[S::IVX], m2 = u[S::IVY], m3 = u[S::IVZ];
  w[S::IVX] = m1 * di;
  w[S::IVY] = m2 * di;
  w[S::IVZ] = m3 * di;
  double ke = 0.5 * (m1 * w[S::IVX] + m2 * w[S::IVY] + m3 * w[S::IVZ]);
  double lat = 0.;
#pragma unroll
  for (int n = 1; n <= NY; ++n)
    if (n > th.nvapor) lat += u[n] * th.u0[n - 1];
  double gamma = get_gamma<double, NY>(th, w);
  w[S::IPR] = (gamma - 1.) * (u[S::IPR] - ke - lat);
}

}  // namespace cb

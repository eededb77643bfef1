// hydro.cpp -- oracle restatement of the explicit part of one canoe time step.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp for the parity status).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>

#include "oracle.hpp"

namespace oracle {

// Athena++ TINY_NUMBER (athena.hpp of chengcli/athenapp), used by the HLLC
// wave-speed floors at hllc_transform.cpp:152-153.
static constexpr double TINY_NUMBER = 1.0e-20;

void block_init(Block &b, const canoe_block_config_t &cfg) {
  b.cfg = cfg;
  b.th = cfg.thermo;
  b.ny = b.th.ny;
  b.nv = 5 + b.ny;
  b.ivx = 1 + b.ny;
  b.ivy = 2 + b.ny;
  b.ivz = 3 + b.ny;
  b.ipr = 4 + b.ny;
  b.nx1 = cfg.nx1;
  b.nx2 = cfg.nx2;
  b.nx3 = cfg.nx3;
  b.f2 = cfg.nx2 > 1;
  b.f3 = cfg.nx3 > 1;
  b.nc1 = b.nx1 + 2 * NG;
  b.nc2 = b.f2 ? b.nx2 + 2 * NG : 1;
  b.nc3 = b.f3 ? b.nx3 + 2 * NG : 1;
  b.is = NG;
  b.ie = NG + b.nx1 - 1;
  b.js = b.f2 ? NG : 0;
  b.je = b.js + b.nx2 - 1;
  b.ks = b.f3 ? NG : 0;
  b.ke = b.ks + b.nx3 - 1;
  b.x1f.assign(b.nc1 + 1, 0.);
  for (int i = 0; i <= b.nx1; ++i) b.x1f[b.is + i] = cfg.h_x1f[i];
  // ghost faces mirror the interior spacing about the block edges
  for (int g = 1; g <= NG; ++g) {
    b.x1f[b.is - g] = 2. * b.x1f[b.is] - b.x1f[b.is + g];
    b.x1f[b.ie + 1 + g] = 2. * b.x1f[b.ie + 1] - b.x1f[b.ie + 1 - g];
  }
  b.x1v.assign(b.nc1, 0.);
  b.dx1f.assign(b.nc1, 0.);
  for (int i = 0; i < b.nc1; ++i) {
    b.x1v[i] = 0.5 * (b.x1f[i] + b.x1f[i + 1]);
    b.dx1f[i] = b.x1f[i + 1] - b.x1f[i];
  }
  b.dx2 = cfg.dx2;
  b.dx3 = cfg.dx3;
  size_t n = (size_t)b.nv * b.cells();
  b.u.assign(n, 0.);
  b.w.assign(n, 0.);
  b.u1.assign(n, 0.);
  b.du.assign(n, 0.);
  b.flx1.assign((size_t)b.nv * b.nc3 * b.nc2 * (b.nc1 + 1), 0.);
  b.flx2.assign((size_t)b.nv * b.nc3 * (b.nc2 + 1) * b.nc1, 0.);
  b.flx3.assign((size_t)b.nv * (b.nc3 + 1) * b.nc2 * b.nc1, 0.);
  b.psf.assign((size_t)b.nc3 * b.nc2 * (b.nc1 + 1), 0.);
  b.psv.assign(b.cells(), 0.);
  b.gam.assign(b.cells(), 0.);
}

// ---------------------------------------------------------------------------
// thermodynamics

// get_gamma: canoe src/interface/eos.hpp:48-67 (rho = 1: w holds fractions).
double get_gamma(const canoe_thermo_t &th, const double *w) {
  double fsig = 1., feps = 1.;
  for (int n = 1; n <= th.nvapor; ++n) {
    fsig += w[n] * th.cv_ratio_m1[n - 1];
    feps += w[n] * th.inv_mu_ratio_m1[n - 1];
  }
  for (int n = 1 + th.nvapor; n <= th.ny; ++n) {
    fsig += w[n] * th.cv_ratio_m1[n - 1];
    feps -= w[n];
  }
  return 1. + (th.gammad - 1.) * feps / fsig;
}

// EquationOfState::SoundSpeed: canoe src/snap/eos/ideal_moist_hydro.cpp:87-91
double sound_speed(const canoe_thermo_t &th, const double *w) {
  int ipr = 4 + th.ny;
  double gamma = get_gamma(th, w);
  return std::sqrt(gamma * w[ipr] / w[0]);
}

// snapy "U->W" (called at canoe src/snap/eos/ideal_moist_hydro.cpp:52-55),
// restated from the ideal-moist model of Li et al. (2019, ApJS 240, 37):
// rho = sum of all densities, fractions q_n = u_n / rho, and
// p = (gamma - 1) (E - KE - sum_clouds rho_c u0_c) with gamma from get_gamma.
void cons_to_prim_cell(const canoe_thermo_t &th, const double *u, double *w,
                       int64_t s) {
  int ny = th.ny, ivx = 1 + ny, ipr = 4 + ny;
  double rho = u[0];
  for (int n = 1; n <= ny; ++n) rho += u[n * s];
  double di = 1. / rho;
  double wl[CANOE_MAX_NV] = {0.};
  wl[0] = rho;
  for (int n = 1; n <= ny; ++n) wl[n] = u[n * s] * di;
  double m1 = u[ivx * s], m2 = u[(ivx + 1) * s], m3 = u[(ivx + 2) * s];
  wl[ivx] = m1 * di;
  wl[ivx + 1] = m2 * di;
  wl[ivx + 2] = m3 * di;
  double ke = 0.5 * (m1 * wl[ivx] + m2 * wl[ivx + 1] + m3 * wl[ivx + 2]);
  double lat = 0.;
  for (int n = 1 + th.nvapor; n <= ny; ++n) lat += u[n * s] * th.u0[n - 1];
  double gamma = get_gamma(th, wl);
  wl[ipr] = (gamma - 1.) * (u[ipr * s] - ke - lat);
  for (int n = 0; n <= ipr; ++n) w[n * s] = wl[n];
}

// snapy "W->U", the inverse of cons_to_prim_cell.
void prim_to_cons_cell(const canoe_thermo_t &th, const double *w, double *u,
                       int64_t s) {
  int ny = th.ny, ivx = 1 + ny, ipr = 4 + ny;
  double wl[CANOE_MAX_NV] = {0.};
  for (int n = 0; n <= ipr; ++n) wl[n] = w[n * s];
  double rho = wl[0];
  double qsum = 0.;
  for (int n = 1; n <= ny; ++n) qsum += wl[n];
  u[0] = rho * (1. - qsum);
  for (int n = 1; n <= ny; ++n) u[n * s] = rho * wl[n];
  double v1 = wl[ivx], v2 = wl[ivx + 1], v3 = wl[ivx + 2];
  u[ivx * s] = rho * v1;
  u[(ivx + 1) * s] = rho * v2;
  u[(ivx + 2) * s] = rho * v3;
  double lat = 0.;
  for (int n = 1 + th.nvapor; n <= ny; ++n) lat += rho * wl[n] * th.u0[n - 1];
  double gamma = get_gamma(th, wl);
  u[ipr * s] =
      wl[ipr] / (gamma - 1.) + lat + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3);
}

// T = p / (rho Rd feps), feps = 1 + sum_v q_v (mu_d/mu_v - 1) - sum_c q_c
double temperature_of_prim(const canoe_thermo_t &th, const double *w,
                           int64_t s) {
  double feps = 1.;
  for (int n = 1; n <= th.nvapor; ++n) feps += w[n * s] * th.inv_mu_ratio_m1[n - 1];
  for (int n = 1 + th.nvapor; n <= th.ny; ++n) feps -= w[n * s];
  return w[(4 + th.ny) * s] / (w[0] * th.rd * feps);
}

// ---------------------------------------------------------------------------
// Riemann solvers

// LMARS: canoe src/snap/riemann/lmars.cpp:19-85.  The reference forms the
// kinetic energy at :47-53 by indexing the 3-element array returned by
// vec_lower (src/exo3/exo3.hpp:17-20) with the full variable slot ivx, which
// reads past the array; the intended Cartesian lowering is the identity, so
// the kinetic term here is 0.5 (v_ivx^2 + v_ivy^2 + v_ivz^2).
void riemann_lmars(const canoe_thermo_t &th, int ivx, const double *wl,
                   const double *wr, double *flx, int64_t n) {
  int ny = th.ny, IVX = 1 + ny, ipr = 4 + ny, nv = 5 + ny;
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
  for (int64_t i = 0; i < n; ++i) {
    double wli[CANOE_MAX_NV], wri[CANOE_MAX_NV];
    for (int v = 0; v < nv; ++v) {
      wli[v] = wl[v * n + i];
      wri[v] = wr[v * n + i];
    }
    double kappal = 1. / (get_gamma(th, wli) - 1.);
    double kappar = 1. / (get_gamma(th, wri) - 1.);
    double hl = wli[ipr] / wli[0] * (kappal + 1.) +
                0.5 * (wli[ivx] * wli[ivx] + wli[ivy] * wli[ivy] +
                       wli[ivz] * wli[ivz]);
    double hr = wri[ipr] / wri[0] * (kappar + 1.) +
                0.5 * (wri[ivx] * wri[ivx] + wri[ivy] * wri[ivy] +
                       wri[ivz] * wri[ivz]);
    double rhobar = 0.5 * (wli[0] + wri[0]);
    double cbar = std::sqrt(0.5 * (1. + (1. / kappar + 1. / kappal) / 2.) *
                            (wli[ipr] + wri[ipr]) / rhobar);
    double pbar = 0.5 * (wli[ipr] + wri[ipr]) +
                  0.5 * (rhobar * cbar) * (wli[ivx] - wri[ivx]);
    double ubar = 0.5 * (wli[ivx] + wri[ivx]) +
                  0.5 / (rhobar * cbar) * (wli[ipr] - wri[ipr]);
    double rdl = 1., rdr = 1.;
    for (int m = 1; m < IVX; ++m) {
      rdl -= wli[m];
      rdr -= wri[m];
    }
    const double *ws = ubar > 0. ? wli : wri;
    double rd = ubar > 0. ? rdl : rdr;
    double h = ubar > 0. ? hl : hr;
    flx[0 * n + i] = ubar * ws[0] * rd;
    for (int m = 1; m < IVX; ++m) flx[m * n + i] = ubar * ws[0] * ws[m];
    flx[ivx * n + i] = ubar * ws[0] * ws[ivx] + pbar;
    flx[ivy * n + i] = ubar * ws[0] * ws[ivy];
    flx[ivz * n + i] = ubar * ws[0] * ws[ivz];
    flx[ipr * n + i] = ubar * ws[0] * h;
  }
}

// HLLC: canoe src/snap/riemann/hllc_transform.cpp:25-233, Cartesian branch
// (no GENERAL_EOS, no CUBED_SPHERE projection).
void riemann_hllc(const canoe_thermo_t &th, int ivx, const double *wl,
                  const double *wr, double *flx, int64_t n, const double *ke_cth) {
  int ny = th.ny, IVX = 1 + ny, IVY = 2 + ny, IVZ = 3 + ny, IPR = 4 + ny;
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
  for (int64_t i = 0; i < n; ++i) {
    double wli[CANOE_MAX_NV], wri[CANOE_MAX_NV];
    double fl[CANOE_MAX_NV], fr[CANOE_MAX_NV], flxi[CANOE_MAX_NV];
    wli[0] = wl[0 * n + i];
    wli[IVX] = wl[ivx * n + i];
    wli[IVY] = wl[ivy * n + i];
    wli[IVZ] = wl[ivz * n + i];
    wli[IPR] = wl[IPR * n + i];
    wri[0] = wr[0 * n + i];
    wri[IVX] = wr[ivx * n + i];
    wri[IVY] = wr[ivy * n + i];
    wri[IVZ] = wr[ivz * n + i];
    wri[IPR] = wr[IPR * n + i];
    for (int m = 1; m < IVX; ++m) {
      wli[m] = wl[m * n + i];
      wri[m] = wr[m * n + i];
    }
    double gammal = get_gamma(th, wli);
    double kappal = 1. / (gammal - 1.);
    double gammar = get_gamma(th, wri);
    double kappar = 1. / (gammar - 1.);
    double cl = sound_speed(th, wli);
    double cr = sound_speed(th, wri);
    double KE_l, KE_r;
    if (ke_cth) {
      // x1 on a cubed-sphere panel: contravariant . covariant velocity
      // (ContravariantVectorToCovariant, cubed_sphere.cpp:225-238)
      const double cth = *ke_cth;
      double vy = wli[IVY] + wli[IVZ] * cth, vz = wli[IVZ] + wli[IVY] * cth;
      KE_l = 0.5 * wli[0] * (wli[IVX] * wli[IVX] + wli[IVY] * vy + wli[IVZ] * vz);
      vy = wri[IVY] + wri[IVZ] * cth;
      vz = wri[IVZ] + wri[IVY] * cth;
      KE_r = 0.5 * wri[0] * (wri[IVX] * wri[IVX] + wri[IVY] * vy + wri[IVZ] * vz);
    } else {
      KE_l = 0.5 * wli[0] *
             (wli[IVX] * wli[IVX] + wli[IVY] * wli[IVY] + wli[IVZ] * wli[IVZ]);
      KE_r = 0.5 * wri[0] *
             (wri[IVX] * wri[IVX] + wri[IVY] * wri[IVY] + wri[IVZ] * wri[IVZ]);
    }
    double el = wli[IPR] * kappal + KE_l;
    double er = wri[IPR] * kappar + KE_r;
    double rhoa = .5 * (wli[0] + wri[0]);
    double ca = .5 * (cl + cr);
    double pmid = .5 * (wli[IPR] + wri[IPR] + (wli[IVX] - wri[IVX]) * rhoa * ca);
    double ql = (pmid <= wli[IPR])
                    ? 1.0
                    : std::sqrt(1.0 + (gammal + 1) / (2 * gammal) *
                                          (pmid / wli[IPR] - 1.0));
    double qr = (pmid <= wri[IPR])
                    ? 1.0
                    : std::sqrt(1.0 + (gammar + 1) / (2 * gammar) *
                                          (pmid / wri[IPR] - 1.0));
    double al = wli[IVX] - cl * ql;
    double ar = wri[IVX] + cr * qr;
    double bp = ar > 0.0 ? ar : (TINY_NUMBER);
    double bm = al < 0.0 ? al : -(TINY_NUMBER);
    double vxl = wli[IVX] - al;
    double vxr = wri[IVX] - ar;
    double tl = wli[IPR] + vxl * wli[0] * wli[IVX];
    double tr = wri[IPR] + vxr * wri[0] * wri[IVX];
    double ml = wli[0] * vxl;
    double mr = -(wri[0] * vxr);
    double am = (tl - tr) / (ml + mr);
    double cp = (ml * tr + mr * tl) / (ml + mr);
    cp = cp > 0.0 ? cp : 0.0;
    vxl = wli[IVX] - bm;
    vxr = wri[IVX] - bp;
    double rdl = 1., rdr = 1.;
    for (int m = 1; m < IVX; ++m) {
      rdl -= wli[m];
      rdr -= wri[m];
    }
    fl[0] = wli[0] * vxl * rdl;
    fr[0] = wri[0] * vxr * rdr;
    for (int m = 1; m < IVX; ++m) {
      fl[m] = wli[0] * wli[m] * vxl;
      fr[m] = wri[0] * wri[m] * vxr;
    }
    fl[IVX] = wli[0] * wli[IVX] * vxl + wli[IPR];
    fr[IVX] = wri[0] * wri[IVX] * vxr + wri[IPR];
    fl[IVY] = wli[0] * wli[IVY] * vxl;
    fr[IVY] = wri[0] * wri[IVY] * vxr;
    fl[IVZ] = wli[0] * wli[IVZ] * vxl;
    fr[IVZ] = wri[0] * wri[IVZ] * vxr;
    fl[IPR] = el * vxl + wli[IPR] * wli[IVX];
    fr[IPR] = er * vxr + wri[IPR] * wri[IVX];
    double sl, sr, sm;
    if (am >= 0.0) {
      sl = am / (am - bm);
      sr = 0.0;
      sm = -bm / (am - bm);
    } else {
      sl = 0.0;
      sr = -am / (bp - am);
      sm = bp / (bp - am);
    }
    for (int m = 0; m < IVX; ++m) flxi[m] = sl * fl[m] + sr * fr[m];
    flxi[IVX] = sl * fl[IVX] + sr * fr[IVX] + sm * cp;
    flxi[IVY] = sl * fl[IVY] + sr * fr[IVY];
    flxi[IVZ] = sl * fl[IVZ] + sr * fr[IVZ];
    flxi[IPR] = sl * fl[IPR] + sr * fr[IPR] + sm * cp * am;
    for (int m = 0; m < IVX; ++m) flx[m * n + i] = flxi[m];
    flx[ivx * n + i] = flxi[IVX];
    flx[ivy * n + i] = flxi[IVY];
    flx[ivz * n + i] = flxi[IVZ];
    flx[IPR * n + i] = flxi[IPR];
  }
}

// ---------------------------------------------------------------------------
// reconstruction along one line (Athena++ precon, external; restated).
// q[0..m-1] cell values, faces f between cells f-1 and f; fills ql[f] (state
// left of face f, from cell f-1) and qr[f] (right of face f, from cell f)
// for faces lo..hi.

// PLM with the van Leer (1979) harmonic-mean limiter, written with cell
// centres xv and faces xf so it also covers a nonuniform x1 grid.
static void plm_line_nonuniform(const double *q, const double *xv,
                                const double *xf, int lo, int hi, double *ql,
                                double *qr) {
  for (int c = lo - 1; c <= hi; ++c) {
    double gl = (q[c] - q[c - 1]) / (xv[c] - xv[c - 1]);
    double gr = (q[c + 1] - q[c]) / (xv[c + 1] - xv[c]);
    double g2 = gl * gr;
    double g = g2 > 0. ? 2. * g2 / (gl + gr) : 0.;
    if (c + 1 <= hi) ql[c + 1] = q[c] + g * (xf[c + 1] - xv[c]);
    if (c >= lo) qr[c] = q[c] - g * (xv[c] - xf[c]);
  }
}

// PLM, uniform spacing (x2, x3).
void plm_line(const double *q, int lo, int hi, double *ql, double *qr) {
  for (int c = lo - 1; c <= hi; ++c) {
    double dwl = q[c] - q[c - 1];
    double dwr = q[c + 1] - q[c];
    double dw2 = dwl * dwr;
    double dwm = dw2 > 0. ? 2. * dw2 / (dwl + dwr) : 0.;
    if (c + 1 <= hi) ql[c + 1] = q[c] + 0.5 * dwm;
    if (c >= lo) qr[c] = q[c] - 0.5 * dwm;
  }
}

// PPM of Colella & Woodward (1984), uniform spacing: monotonized-central
// slopes (CW84 eq. 1.7-1.8), fourth-order face values (eq. 1.6), and the
// parabola monotonicity limiter (eq. 1.10).  Needs 3 ghost cells.
static inline double ppm_slope(double qm, double q0, double qp) {
  double dwl = q0 - qm, dwr = qp - q0;
  if (dwl * dwr <= 0.) return 0.;
  double dwc = 0.5 * (qp - qm);
  double lim = std::min(std::fabs(dwc), std::min(2. * std::fabs(dwl), 2. * std::fabs(dwr)));
  return std::copysign(lim, dwc);
}

void ppm_line(const double *q, int lo, int hi, double *ql, double *qr) {
  for (int c = lo - 1; c <= hi; ++c) {
    double dm_m = ppm_slope(q[c - 2], q[c - 1], q[c]);
    double dm_0 = ppm_slope(q[c - 1], q[c], q[c + 1]);
    double dm_p = ppm_slope(q[c], q[c + 1], q[c + 2]);
    const double sixth = 1. / 6.;
    double wL = 0.5 * (q[c - 1] + q[c]) - (dm_0 - dm_m) * sixth;
    double wR = 0.5 * (q[c] + q[c + 1]) - (dm_p - dm_0) * sixth;
    double w0 = q[c];
    if ((wR - w0) * (w0 - wL) <= 0.) {
      wL = w0;
      wR = w0;
    } else {
      double d = wR - wL;
      double m6 = 6. * (w0 - 0.5 * (wL + wR));
      if (d * m6 > d * d)
        wL = 3. * w0 - 2. * wR;
      else if (-d * d > d * m6)
        wR = 3. * w0 - 2. * wL;
    }
    if (c + 1 <= hi) ql[c + 1] = wR;
    if (c >= lo) qr[c] = wL;
  }
}

// ---------------------------------------------------------------------------
// ghost cells (Athena reflecting / periodic / outflow conditions, restated)

// A CANOE_BC_BLOCK side is left as it is: its ghosts come from the
// neighbouring block (the exchange of the caller).
void apply_bc(Block &b, std::vector<double> &w) {
  const int *bc = b.cfg.bc;
  // x1 over interior (j, k)
  for (int n = 0; n < b.nv; ++n)
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j)
        for (int g = 1; g <= NG; ++g) {
          double s = (n == b.ivx) ? -1. : 1.;
          size_t lo = b.idx(n, k, j, b.is - g), hi = b.idx(n, k, j, b.ie + g);
          if (bc[0] == CANOE_BC_REFLECT) w[lo] = s * w[b.idx(n, k, j, b.is + g - 1)];
          else if (bc[0] == CANOE_BC_PERIODIC) w[lo] = w[b.idx(n, k, j, b.ie - g + 1)];
          else w[lo] = w[b.idx(n, k, j, b.is)];
          if (bc[1] == CANOE_BC_REFLECT) w[hi] = s * w[b.idx(n, k, j, b.ie - g + 1)];
          else if (bc[1] == CANOE_BC_PERIODIC) w[hi] = w[b.idx(n, k, j, b.is + g - 1)];
          else w[hi] = w[b.idx(n, k, j, b.ie)];
        }
  if (b.f2)
    for (int n = 0; n < b.nv; ++n)
      for (int k = b.ks; k <= b.ke; ++k)
        for (int g = 1; g <= NG; ++g)
          for (int i = 0; i < b.nc1; ++i) {
            double s = (n == b.ivy) ? -1. : 1.;
            size_t lo = b.idx(n, k, b.js - g, i), hi = b.idx(n, k, b.je + g, i);
            const double wlo = w[lo], whi = w[hi];
            if (bc[2] == CANOE_BC_REFLECT) w[lo] = s * w[b.idx(n, k, b.js + g - 1, i)];
            else if (bc[2] == CANOE_BC_PERIODIC) w[lo] = w[b.idx(n, k, b.je - g + 1, i)];
            else w[lo] = w[b.idx(n, k, b.js, i)];
            if (bc[3] == CANOE_BC_REFLECT) w[hi] = s * w[b.idx(n, k, b.je - g + 1, i)];
            else if (bc[3] == CANOE_BC_PERIODIC) w[hi] = w[b.idx(n, k, b.js + g - 1, i)];
            else w[hi] = w[b.idx(n, k, b.je, i)];
            if (bc[2] == CANOE_BC_BLOCK) w[lo] = wlo;
            if (bc[3] == CANOE_BC_BLOCK) w[hi] = whi;
          }
  if (b.f3)
    for (int n = 0; n < b.nv; ++n)
      for (int g = 1; g <= NG; ++g)
        for (int j = 0; j < b.nc2; ++j)
          for (int i = 0; i < b.nc1; ++i) {
            double s = (n == b.ivz) ? -1. : 1.;
            size_t lo = b.idx(n, b.ks - g, j, i), hi = b.idx(n, b.ke + g, j, i);
            const double wlo = w[lo], whi = w[hi];
            if (bc[4] == CANOE_BC_REFLECT) w[lo] = s * w[b.idx(n, b.ks + g - 1, j, i)];
            else if (bc[4] == CANOE_BC_PERIODIC) w[lo] = w[b.idx(n, b.ke - g + 1, j, i)];
            else w[lo] = w[b.idx(n, b.ks, j, i)];
            if (bc[5] == CANOE_BC_REFLECT) w[hi] = s * w[b.idx(n, b.ke - g + 1, j, i)];
            else if (bc[5] == CANOE_BC_PERIODIC) w[hi] = w[b.idx(n, b.ks + g - 1, j, i)];
            else w[hi] = w[b.idx(n, b.ke, j, i)];
            if (bc[4] == CANOE_BC_BLOCK) w[lo] = wlo;
            if (bc[5] == CANOE_BC_BLOCK) w[hi] = whi;
          }
}

void cons_to_prim_block(Block &b) {
  size_t s = b.cells();
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        size_t c = b.idx(0, k, j, i);
        cons_to_prim_cell(b.th, &b.u[c], &b.w[c], s);
      }
  apply_bc(b, b.w);
}

// ---------------------------------------------------------------------------
// Hydro::CalculateFluxes with the canoe hooks (patches/19.calculate_fluxes.
// patch): x1 pencils go through Decomposition::ChangeToTemperature /
// RestoreFromTemperature (src/snap/decomposition/change_to_temperature.cpp:
// 40-167); x2 and x3 reconstruct the primitive state directly.

static void riemann(const Block &b, int ivx, const double *wl, const double *wr,
                    double *flx, int64_t n) {
  if (b.cfg.rsolver == CANOE_RSOLVER_LMARS)
    riemann_lmars(b.th, ivx, wl, wr, flx, n);
  else
    riemann_hllc(b.th, ivx, wl, wr, flx, n);
}

// Decomposition::ChangeToTemperature for column (k, j)
// (change_to_temperature.cpp:40-136): fills the block's psf / psv / gamma_
// for the column and turns the pencil q(n, i) (nv x nc1) into T and p'.
void change_to_temperature_pencil(Block &b, int k, int j, double *q) {
  const int nc1 = b.nc1, ipr = b.ipr;
  const int is = b.is, ie = b.ie;
  const double grav = b.th.grav;
  if (grav == 0.) return;
  double *psf = &b.psf[((size_t)k * b.nc2 + j) * (nc1 + 1)];
  double *psv = &b.psv[b.idx(0, k, j, 0)];
  double *gam = &b.gam[b.idx(0, k, j, 0)];
  double *rho = &q[0], *pre = &q[ipr * nc1];
  // change_to_temperature.cpp:57-64 isothermal extrapolation to the top
  double RdTv = pre[ie] / rho[ie];
  psf[ie + 1] = pre[ie] * std::exp(grav * b.dx1f[ie] / (2 * RdTv));
  // :65 IntegrateDownwards (:30-38)
  for (int i = ie; i >= is; --i) psf[i] = psf[i + 1] - grav * rho[i] * b.dx1f[i];
  // :71-82 ghost psf, reflecting walls integrate with -grav
  double gb = b.cfg.bc[0] == CANOE_BC_REFLECT ? -grav : grav;
  for (int i = is - 1; i >= is - NG; --i) psf[i] = psf[i + 1] - gb * rho[i] * b.dx1f[i];
  double gt = b.cfg.bc[1] == CANOE_BC_REFLECT ? -grav : grav;
  for (int i = ie + 1; i <= ie + NG; ++i) psf[i + 1] = psf[i] + gt * rho[i] * b.dx1f[i];
  // :89-111 per cell: log-mean psv, RovRd, rho -> T, p -> p'
  for (int i = is - NG; i <= ie + NG; ++i) {
    if (std::fabs(psf[i] - psf[i + 1]) < 1.E-6)
      psv[i] = 0.5 * (psf[i] + psf[i + 1]);
    else
      psv[i] = (psf[i] - psf[i + 1]) / std::log(psf[i] / psf[i + 1]);
    double feps = 1.;
    for (int n = 1; n <= b.th.nvapor; ++n)
      feps += q[n * nc1 + i] * b.th.inv_mu_ratio_m1[n - 1];
    gam[i] = b.th.rd * feps;
    rho[i] = pre[i] / (rho[i] * gam[i]);
    pre[i] -= psv[i];
  }
  // :113-127 outflow walls hold T and p' constant into the ghosts
  if (b.cfg.bc[0] == CANOE_BC_OUTFLOW)
    for (int i = is - NG; i < is; ++i) {
      rho[i] = rho[is];
      pre[i] = pre[is];
    }
  if (b.cfg.bc[1] == CANOE_BC_OUTFLOW)
    for (int i = ie + 1; i <= ie + NG; ++i) {
      rho[i] = rho[ie];
      pre[i] = pre[ie];
    }
}

// Decomposition::RestoreFromTemperature for column (k, j)
// (change_to_temperature.cpp:138-167): the pencil q back to rho and p, and
// the face states wl / wr (nv x (nc1 + 1)) of faces lo..hi back to rho and p
// with the hydrostatic face pressure added.
void restore_from_temperature_pencil(Block &b, int k, int j, double *q, double *wl,
                                     double *wr, int lo, int hi) {
  const int nc1 = b.nc1, ipr = b.ipr;
  const int is = b.is, ie = b.ie;
  if (b.th.grav == 0.) return;
  const double *psf = &b.psf[((size_t)k * b.nc2 + j) * (nc1 + 1)];
  const double *psv = &b.psv[b.idx(0, k, j, 0)];
  const double *gam = &b.gam[b.idx(0, k, j, 0)];
  double *rho = &q[0], *pre = &q[ipr * nc1];
  for (int i = is - NG; i <= ie + NG; ++i) {
    pre[i] += psv[i];
    rho[i] = pre[i] / (rho[i] * gam[i]);
  }
  double *lr = &wl[0], *lp = &wl[ipr * (nc1 + 1)];
  double *rr = &wr[0], *rp = &wr[ipr * (nc1 + 1)];
  for (int i = lo; i <= hi; ++i) {
    rp[i] += psf[i];
    if (rp[i] < 0.) rp[i] = psf[i];
    double gamma = std::sqrt(gam[i] * gam[i - 1]);
    rr[i] = rp[i] / (rr[i] * gamma);
    lp[i] += psf[i];
    if (lp[i] < 0.) lp[i] = psf[i];
    lr[i] = lp[i] / (lr[i] * gamma);
  }
}

static void flux_x1_pencil(Block &b, int k, int j, std::vector<double> &q,
                           std::vector<double> &wl, std::vector<double> &wr,
                           std::vector<double> &fx) {
  const int nc1 = b.nc1, nv = b.nv, ipr = b.ipr;
  const int is = b.is, ie = b.ie;
  // pencil copy q(n, i)
  for (int n = 0; n < nv; ++n)
    for (int i = 0; i < nc1; ++i) q[n * nc1 + i] = b.w[b.idx(n, k, j, i)];
  change_to_temperature_pencil(b, k, j, q.data());
  // reconstruct faces is..ie+1
  int lo = is, hi = ie + 1;
  for (int n = 0; n < nv; ++n) {
    const double *qn = &q[n * nc1];
    double *l = &wl[n * (nc1 + 1)], *r = &wr[n * (nc1 + 1)];
    if (b.cfg.recon == CANOE_RECON_PPM)
      ppm_line(qn, lo, hi, l, r);
    else
      plm_line_nonuniform(qn, b.x1v.data(), b.x1f.data(), lo, hi, l, r);
  }
  if (b.th.grav != 0.) {
    restore_from_temperature_pencil(b, k, j, q.data(), wl.data(), wr.data(), lo, hi);
    if (b.fix_roundtrip)
      for (int i = 0; i < nc1; ++i) {
        b.w[b.idx(0, k, j, i)] = q[i];
        b.w[b.idx(ipr, k, j, i)] = q[ipr * nc1 + i];
      }
  }
  // Riemann solver on the packed faces lo..hi
  int nf = hi - lo + 1;
  std::vector<double> pl(nv * nf), pr(nv * nf);
  for (int n = 0; n < nv; ++n)
    for (int f = 0; f < nf; ++f) {
      pl[n * nf + f] = wl[n * (nc1 + 1) + lo + f];
      pr[n * nf + f] = wr[n * (nc1 + 1) + lo + f];
    }
  fx.resize(nv * nf);
  if (b.geo) {
    // cubed-sphere panel: covariant kinetic energy in the x1 Riemann problem
    // (hllc_transform.cpp:92-101) and the contravariant -> covariant
    // projection of the transverse momentum fluxes (:245-272)
    const double x = std::tan(b.geo->x2v[j]), y = std::tan(b.geo->x3v[k]);
    const double Ck = std::sqrt(x * x + 1), Dk = std::sqrt(y * y + 1);
    const double cth_ke = -x * y / (Ck * Dk);
    riemann_hllc(b.th, b.ivx, pl.data(), pr.data(), fx.data(), nf, &cth_ke);
    const double C = std::sqrt(1. + x * x), D = std::sqrt(1. + y * y);
    const double cth = -x * y / C / D;
    for (int f = 0; f < nf; ++f) {
      const double ty = fx[b.ivy * nf + f], tz = fx[b.ivz * nf + f];
      fx[b.ivy * nf + f] = ty + tz * cth;
      fx[b.ivz * nf + f] = tz + ty * cth;
    }
  } else {
    riemann(b, b.ivx, pl.data(), pr.data(), fx.data(), nf);
  }
  for (int n = 0; n < nv; ++n)
    for (int f = 0; f < nf; ++f)
      b.flx1[(((size_t)n * b.nc3 + k) * b.nc2 + j) * (nc1 + 1) + lo + f] =
          fx[n * nf + f];
}

void calculate_fluxes_x1_only(Block &b) {
  const int nv = b.nv;
#pragma omp parallel
  {
    std::vector<double> q(nv * b.nc1), wl(nv * (b.nc1 + 1)), wr(nv * (b.nc1 + 1)), fx;
#pragma omp for collapse(2) schedule(static)
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j) flux_x1_pencil(b, k, j, q, wl, wr, fx);
  }
}

void calculate_fluxes(Block &b) {
  const int nv = b.nv;
  calculate_fluxes_x1_only(b);
  // x2: lines along j for every interior (k, i)
  if (b.f2) {
#pragma omp parallel
    {
      int m = b.nc2;
      std::vector<double> q(m), l((size_t)nv * (m + 1)), r((size_t)nv * (m + 1));
      int nf = b.je + 1 - b.js + 1;
      std::vector<double> pl(nv * nf), pr(nv * nf), fx(nv * nf);
#pragma omp for collapse(2) schedule(static)
      for (int k = b.ks; k <= b.ke; ++k)
        for (int i = b.is; i <= b.ie; ++i) {
          for (int n = 0; n < nv; ++n) {
            for (int j = 0; j < m; ++j) q[j] = b.w[b.idx(n, k, j, i)];
            if (b.cfg.recon == CANOE_RECON_PPM)
              ppm_line(q.data(), b.js, b.je + 1, &l[n * (m + 1)], &r[n * (m + 1)]);
            else
              plm_line(q.data(), b.js, b.je + 1, &l[n * (m + 1)], &r[n * (m + 1)]);
            for (int f = 0; f < nf; ++f) {
              pl[n * nf + f] = l[n * (m + 1) + b.js + f];
              pr[n * nf + f] = r[n * (m + 1) + b.js + f];
            }
          }
          riemann(b, b.ivy, pl.data(), pr.data(), fx.data(), nf);
          for (int n = 0; n < nv; ++n)
            for (int f = 0; f < nf; ++f)
              b.flx2[(((size_t)n * b.nc3 + k) * (b.nc2 + 1) + b.js + f) * b.nc1 + i] =
                  fx[n * nf + f];
        }
    }
  }
  // x3: lines along k for every interior (j, i)
  if (b.f3) {
#pragma omp parallel
    {
      int m = b.nc3;
      std::vector<double> q(m), l((size_t)nv * (m + 1)), r((size_t)nv * (m + 1));
      int nf = b.ke + 1 - b.ks + 1;
      std::vector<double> pl(nv * nf), pr(nv * nf), fx(nv * nf);
#pragma omp for collapse(2) schedule(static)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i) {
          for (int n = 0; n < nv; ++n) {
            for (int k = 0; k < m; ++k) q[k] = b.w[b.idx(n, k, j, i)];
            if (b.cfg.recon == CANOE_RECON_PPM)
              ppm_line(q.data(), b.ks, b.ke + 1, &l[n * (m + 1)], &r[n * (m + 1)]);
            else
              plm_line(q.data(), b.ks, b.ke + 1, &l[n * (m + 1)], &r[n * (m + 1)]);
            for (int f = 0; f < nf; ++f) {
              pl[n * nf + f] = l[n * (m + 1) + b.ks + f];
              pr[n * nf + f] = r[n * (m + 1) + b.ks + f];
            }
          }
          riemann(b, b.ivz, pl.data(), pr.data(), fx.data(), nf);
          for (int n = 0; n < nv; ++n)
            for (int f = 0; f < nf; ++f)
              b.flx3[(((size_t)n * (b.nc3 + 1) + b.ks + f) * b.nc2 + j) * b.nc1 + i] =
                  fx[n * nf + f];
        }
    }
  }
}

// Athena AddFluxDivergence for a Cartesian block (external; restated as the
// finite-volume divergence, face differences times the reciprocal widths),
// accumulated into du with weight wght = beta dt.
void add_flux_divergence(Block &b, double wght, std::vector<double> &du) {
  const int nc1 = b.nc1, nc2 = b.nc2;
#pragma omp parallel for collapse(3) schedule(static)
  for (int n = 0; n < b.nv; ++n)
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i) {
          size_t f1 = (((size_t)n * b.nc3 + k) * nc2 + j) * (nc1 + 1) + i;
          double d = (b.flx1[f1 + 1] - b.flx1[f1]) * (1. / b.dx1f[i]);
          if (b.f2) {
            size_t f2 = (((size_t)n * b.nc3 + k) * (nc2 + 1) + j) * nc1 + i;
            d += (b.flx2[f2 + nc1] - b.flx2[f2]) * (1. / b.dx2);
          }
          if (b.f3) {
            size_t f3 = (((size_t)n * (b.nc3 + 1) + k) * nc2 + j) * nc1 + i;
            d += (b.flx3[f3 + (size_t)nc2 * nc1] - b.flx3[f3]) * (1. / b.dx3);
          }
          du[b.idx(n, k, j, i)] -= wght * d;
        }
}

// Constant x1 gravity source: HydroSourceTerms::ConstantAcceleration of
// Athena++ (chengcli/athenapp @ 8c221aa, external) as patched by canoe
// patches/25.constant_acc.patch:35-52: src = dt rho g with rho the total
// density (prim(IDN); no passive scalars on this path), added to the x1
// momentum, and src v1 added to the energy.
void add_gravity_source(Block &b, double dt, std::vector<double> &du) {
  const double g = b.th.grav;
  if (g == 0.) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double src = dt * b.w[b.idx(0, k, j, i)] * g;
        du[b.idx(b.ivx, k, j, i)] += src;
        du[b.idx(b.ipr, k, j, i)] += src * b.w[b.idx(b.ivx, k, j, i)];
      }
}

// The user explicit source of the dense sinking bubble example:
// examples/2019-Li-snap/straka.cpp:125-190 (Diffusion), 2-D (k = ks), added
// into du with the stage weight as ImplicitHydroTasks::AddSourceTerms does
// (src/tasklist/implicit_hydro_tasks.cpp:192-216).  dx = dx1f(is), dy =
// dx2f(js); theta = T (p0 / p)^chi with T from the equation of state.
void add_diffusion_source(Block &b, double dt, std::vector<double> &du) {
  const double K = b.diff_K;
  if (K <= 0.) return;
  const double chi = (b.th.gammad - 1.) / b.th.gammad;
  const double cp = b.th.gammad / (b.th.gammad - 1.) * b.th.rd;
  const double dx = b.dx1f[b.is], dy = b.dx2;
  const int64_t s = (int64_t)b.cells();
  const int k = b.ks;
  auto theta = [&](int j, int i, double &T) {
    const double *w = &b.w[b.idx(0, k, j, i)];
    T = temperature_of_prim(b.th, w, s);
    return T * std::pow(b.diff_p0 / w[b.ipr * s], chi);
  };
#pragma omp parallel for schedule(static)
  for (int j = b.js; j <= b.je; ++j)
    for (int i = b.is; i <= b.ie; ++i) {
      auto W = [&](int n, int jj, int ii) { return b.w[b.idx(n, k, jj, ii)]; };
      double T, Tn;
      const double th = theta(j, i, T);
      const double th_sum = theta(j + 1, i, Tn) + theta(j - 1, i, Tn) + theta(j, i + 1, Tn) +
                            theta(j, i - 1, Tn);
      const double f = dt * K * W(0, j, i) / (dx * dy);
      du[b.idx(b.ivx, k, j, i)] += f * (W(b.ivx, j, i - 1) + W(b.ivx, j, i + 1) +
                                        W(b.ivx, j - 1, i) + W(b.ivx, j + 1, i) -
                                        4. * W(b.ivx, j, i));
      du[b.idx(b.ivy, k, j, i)] += f * (W(b.ivy, j, i - 1) + W(b.ivy, j, i + 1) +
                                        W(b.ivy, j - 1, i) + W(b.ivy, j + 1, i) -
                                        4. * W(b.ivy, j, i));
      du[b.idx(b.ipr, k, j, i)] += f * cp * T / th * (th_sum - 4. * th);
    }
}

// Hydro::NewBlockTimeStep with canoe patches/21.new_blockdt.patch:20-40
// (an implicit direction uses |v| only: x1 when nx2 > 1, x2 and x3 by their
// bits); returns cfl * min over interior cells.
double new_dt(const Block &b) {
  double cfl = b.cfg.cfl;
  bool imp1 = (b.cfg.implicit_flag & 1) && (b.nx2 > 1);
  double mn = std::numeric_limits<double>::infinity();
  size_t s = b.cells();
#pragma omp parallel for collapse(2) reduction(min : mn) schedule(static)
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double wi[CANOE_MAX_NV];
        for (int n = 0; n < b.nv; ++n) wi[n] = b.w[b.idx(0, k, j, i) + n * s];
        double cs = sound_speed(b.th, wi);
        double dt1 = b.dx1f[i];
        if (imp1) dt1 /= cfl * std::fabs(wi[b.ivx]);
        else dt1 /= (std::fabs(wi[b.ivx]) + cs);
        mn = std::min(mn, dt1);
        const int flag = b.cfg.implicit_flag;
        if (b.f2)
          mn = std::min(mn, (flag & 2) ? b.dx2 / (cfl * std::fabs(wi[b.ivy]))
                                       : b.dx2 / (std::fabs(wi[b.ivy]) + cs));
        if (b.f3)
          mn = std::min(mn, (flag & 4) ? b.dx3 / (cfl * std::fabs(wi[b.ivz]))
                                       : b.dx3 / (std::fabs(wi[b.ivz]) + cs));
      }
  return cfl * mn;
}

// One SSPRK(3,3) step (Shu & Osher 1988) in the register form of
// ImplicitHydroTasks::IntegrateHydro (src/tasklist/implicit_hydro_tasks.cpp:
// 134-190): u = g1 u + g2 u1; du = -beta dt div F + sources; implicit
// correction (:267-288); u += du; saturation adjustment at the last stage
// (:290-313); then boundaries and cons2prim.
void stage_step(Block &b, double dt, int stage) {
  static const double g1[3] = {0., 0.25, 2. / 3.};
  static const double g2[3] = {1., 0.75, 1. / 3.};
  static const double be[3] = {1., 0.25, 2. / 3.};
  {
    calculate_fluxes(b);
#pragma omp parallel for collapse(3) schedule(static)
    for (int n = 0; n < b.nv; ++n)
      for (int k = b.ks; k <= b.ke; ++k)
        for (int j = b.js; j <= b.je; ++j)
          for (int i = b.is; i <= b.ie; ++i) {
            size_t c = b.idx(n, k, j, i);
            if (stage == 0) b.u1[c] = b.u[c];
            b.u[c] = g1[stage] * b.u[c] + g2[stage] * b.u1[c];
            b.du[c] = 0.;
          }
    double wght = be[stage] * dt;
    add_flux_divergence(b, wght, b.du);
    add_gravity_source(b, wght, b.du);
    add_diffusion_source(b, wght, b.du);
    if (b.cfg.implicit_flag & 7) solve_implicit(b, b.du, wght);
#pragma omp parallel for collapse(3) schedule(static)
    for (int n = 0; n < b.nv; ++n)
      for (int k = b.ks; k <= b.ke; ++k)
        for (int j = b.js; j <= b.je; ++j)
          for (int i = b.is; i <= b.ie; ++i) {
            size_t c = b.idx(n, k, j, i);
            b.u[c] += b.du[c];
          }
    if (stage == 2 && b.cfg.satadj && b.ny > 0) {
      canoe_satadj_opts_t o{1e-8, 30, 0};
      satadj_block(b, o);
    }
    cons_to_prim_block(b);
  }
}

void step(Block &b, double dt) {
  for (int stage = 0; stage < 3; ++stage) stage_step(b, dt, stage);
}

}  // namespace oracle

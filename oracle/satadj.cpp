// satadj.cpp -- oracle restatement of the isochoric, isoenergetic ("UV")
// saturation adjustment that canoe runs at the last RK stage:
// ImplicitHydroTasks::UpdateAllConserved (src/tasklist/implicit_hydro_tasks.
// cpp:290-313) -> kintera ThermoY::forward(rho, intEng, yfrac) (external,
// version unpinned; parity unpinned).
//
// Model (restated from the reference's thermo data and Li et al. 2019):
//  * constant-cp species, h = h0 + cp0 (T - T0)  (examples/2019-Li-snap/
//    jup-thermo.yaml:7-10); condensates have zero molar volume
//    (earth-moist.yaml:31-32);
//  * "ideal" saturation vapour pressure
//      p_sat(T) = p3 exp[beta (1 - t3/T) - delta ln(T/t3)]
//    (earth-moist.yaml:37, jup-thermo.yaml:100-116) with liquid above t3
//    and ice below (minT / maxT at jup-thermo.yaml:102-104);
//  * internal energy per kg: gases cv T, condensates cv_c T + u0_c, so
//    ie = rho [cv_d (q_d + sum_n q_n (1 + cv_ratio_m1_n)) T + sum_c q_c u0_c].
// Unknown T solves f(T) = rho e(T, q(T)) - ie = 0 where every vapor is at
// min(total, saturation).  Newton from a guess (cold start: the temperature
// of the unadjusted state; warm start: a supplied guess) stops at |dT| < tol;
// if the residual fails to drop, a bracketed Newton/bisection (the fallback)
// finishes the solve.  One polishing Newton step follows convergence, so the
// answer does not depend on the starting point beyond roundoff.  A root on a liquid/ice jump at t3 is resolved by
// splitting the condensate between the two phases at T = t3.  Total energy
// u[IEN] and dry density u[IDN] are untouched; only u[1..ny] change.
// TEST INFRASTRUCTURE ONLY.
#include <cmath>
#include <limits>

#include "oracle.hpp"

namespace oracle {

namespace {

struct Eval {
  double f, fp;
  double q[CANOE_MAX_NY + 1];
};

struct Cell {
  double rho, ie, qd;
  double qt[CANOE_MAX_VAPOR];       // total of each condensable family
  double qinert[CANOE_MAX_NY + 1];  // slots outside any family
};

// evaluate f(T) and df/dT; `force_phase` (-1 none) pins vapor v to liquid(0)
// / ice(1) to evaluate the two sides of a t3 jump.
Eval evaluate(const canoe_thermo_t &th, const Cell &c, double T, int fv = -1,
              int fphase = 0) {
  Eval e;
  const double cvd = th.rd / (th.gammad - 1.);
  for (int n = 0; n <= th.ny; ++n) e.q[n] = c.qinert[n];
  double cvs = c.qd;  // sum of q (1 + cv_ratio_m1), dry first
  double lat = 0., dlat = 0.;
  for (int n = 1; n <= th.ny; ++n)
    if (c.qinert[n] != 0.) {
      cvs += c.qinert[n] * (1. + th.cv_ratio_m1[n - 1]);
      lat += c.qinert[n] * th.u0[n - 1];
    }
  for (int v = 0; v < th.nvapor; ++v) {
    int vs = 1 + v, ls = th.liq_slot[v], ss = th.ice_slot[v];
    if (ls < 0 && ss < 0) {
      e.q[vs] = c.qt[v];
      cvs += c.qt[v] * (1. + th.cv_ratio_m1[vs - 1]);
      continue;
    }
    bool liquid = (ss < 0) || (ls >= 0 && T >= th.t3[v]);
    if (v == fv) liquid = (fphase == 0);
    int cs = liquid ? ls : ss;
    double beta = liquid ? th.beta_l[v] : th.beta_s[v];
    double delta = liquid ? th.delta_l[v] : th.delta_s[v];
    double rv = th.rd * (1. + th.inv_mu_ratio_m1[vs - 1]);
    double lnps = std::log(th.p3[v]) + beta * (1. - th.t3[v] / T) -
                  delta * std::log(T / th.t3[v]);
    double qs = std::exp(lnps) / (c.rho * rv * T);
    double qv, qc, dqv;
    if (qs < c.qt[v]) {
      qv = qs;
      qc = c.qt[v] - qs;
      dqv = qs * (beta * th.t3[v] / (T * T) - delta / T - 1. / T);
    } else {
      qv = c.qt[v];
      qc = 0.;
      dqv = 0.;
    }
    double cvv = 1. + th.cv_ratio_m1[vs - 1];
    double cvc = 1. + th.cv_ratio_m1[cs - 1];
    e.q[vs] = qv;
    e.q[cs] += qc;
    cvs += qv * cvv + qc * cvc;
    lat += qc * th.u0[cs - 1];
    dlat += dqv * (cvd * cvv * T - cvd * cvc * T - th.u0[cs - 1]);
  }
  e.f = c.rho * (cvd * cvs * T + lat) - c.ie;
  e.fp = c.rho * (cvd * cvs + dlat);
  return e;
}

}  // namespace

SatResult satadj_cell(const canoe_thermo_t &th, const canoe_satadj_opts_t &o,
                      double *u, int64_t s, double t_guess) {
  const int ny = th.ny, ivx = 1 + ny, ien = 4 + ny;
  const double cvd = th.rd / (th.gammad - 1.);
  Cell c;
  // implicit_hydro_tasks.cpp:304-307: rho, ke, ie, yfrac
  c.rho = u[0];
  for (int n = 1; n <= ny; ++n) c.rho += u[n * s];
  double m1 = u[ivx * s], m2 = u[(ivx + 1) * s], m3 = u[(ivx + 2) * s];
  double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / c.rho;
  c.ie = u[ien * s] - ke;
  double q[CANOE_MAX_NY + 1];
  double qsum = 0.;
  for (int n = 1; n <= ny; ++n) {
    q[n] = u[n * s] / c.rho;
    qsum += q[n];
  }
  c.qd = 1. - qsum;
  for (int n = 0; n <= ny; ++n) c.qinert[n] = 0.;
  bool member[CANOE_MAX_NY + 1] = {false};
  for (int v = 0; v < th.nvapor; ++v) {
    c.qt[v] = q[1 + v];
    member[1 + v] = true;
    if (th.liq_slot[v] > 0) {
      c.qt[v] += q[th.liq_slot[v]];
      member[th.liq_slot[v]] = true;
    }
    if (th.ice_slot[v] > 0) {
      c.qt[v] += q[th.ice_slot[v]];
      member[th.ice_slot[v]] = true;
    }
  }
  for (int n = 1; n <= ny; ++n)
    if (!member[n]) c.qinert[n] = q[n];
  // cold start: temperature of the unadjusted state
  double cvs = c.qd, lat = 0.;
  for (int n = 1; n <= ny; ++n) {
    cvs += q[n] * (1. + th.cv_ratio_m1[n - 1]);
    lat += q[n] * th.u0[n - 1];
  }
  double t_cold = (c.ie / c.rho - lat) / (cvd * cvs);

  SatResult r{t_cold, 0, false, false};
  double T = t_cold;
  // start (o.warm): 0 cold, 1 the guess, 2 gated: the guess when it exceeds
  // the cold start by 0.05 K of latent heating, else cold.  iters counts
  // evaluations of f.
  const bool guess_ok = std::isfinite(t_guess) && t_guess > 1. && t_guess < 1.e4;
  if (o.warm == 1 && guess_ok) T = t_guess;
  if (o.warm == 2 && guess_ok && t_guess - t_cold > 0.05) T = t_guess;
  double fprev = std::numeric_limits<double>::infinity();
  Eval e;
  const int it0 = 0;
  for (int it = it0; it < o.max_iter && !r.converged; ++it) {
    e = evaluate(th, c, T);
    if (!(std::fabs(e.f) < fprev) && it > 0) {
      r.fallback = true;
      break;
    }
    double dT = -e.f / e.fp;
    T += dT;
    r.iters++;
    fprev = std::fabs(e.f);
    if (std::fabs(dT) < o.tol) {
      r.converged = true;
      e = evaluate(th, c, T);  // one polishing Newton step
      T -= e.f / e.fp;
      r.iters++;
      break;
    }
  }
  if (!r.converged) {
    // bracketed fallback
    r.fallback = true;
    double lo = 1., hi = 1.e4;
    if (!(T > lo && T < hi)) T = t_cold;
    for (int it = 0; it < 200; ++it) {
      e = evaluate(th, c, T);
      if (e.f < 0.) lo = T;
      else hi = T;
      double tn = T - e.f / e.fp;
      if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
      double dT = tn - T;
      T = tn;
      r.iters++;
      if (std::fabs(dT) < o.tol || hi - lo < o.tol) {
        r.converged = true;
        e = evaluate(th, c, T);
        // polish unless the step leaves the bracket (a root on a jump)
        double tp = T - e.f / e.fp;
        if (tp > lo - 2. * o.tol && tp < hi + 2. * o.tol) T = tp;
        break;
      }
    }
  }
  e = evaluate(th, c, T);
  // a root on the liquid/ice jump of vapor v: split at T = t3
  for (int v = 0; v < th.nvapor; ++v) {
    if (th.liq_slot[v] < 0 || th.ice_slot[v] < 0) continue;
    // f is increasing in T, so the root sits on the jump iff
    // f_ice(t3) < 0 < f_liquid(t3); only iterates ending near t3 can be there
    if (std::fabs(T - th.t3[v]) > 1e-3) continue;
    Eval el = evaluate(th, c, th.t3[v], v, 0), es = evaluate(th, c, th.t3[v], v, 1);
    if ((el.f > 0.) == (es.f > 0.)) continue;
    double x = -es.f / (el.f - es.f);  // liquid share, f linear in x
    T = th.t3[v];
    e = el;
    int ls = th.liq_slot[v], ss = th.ice_slot[v];
    double qc = el.q[ls];
    e.q[ls] = x * qc;
    e.q[ss] = qc - x * qc;
    break;
  }
  // implicit_hydro_tasks.cpp:310: u[1..ny] = yfrac * rho
  for (int n = 1; n <= ny; ++n) u[n * s] = e.q[n] * c.rho;
  r.t = T;
  return r;
}

void satadj_block(Block &b, const canoe_satadj_opts_t &o) {
  size_t s = b.cells();
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i)
        satadj_cell(b.th, o, &b.u[b.idx(0, k, j, i)], s, 0.);
}

// ---------------------------------------------------------------------------
// MLP 4 -> nh -> nh -> 1 with tanh hidden activations: the warm-start
// network of the learned saturation adjustment (a project addition with no
// counterpart in the reference).

void mlp_forward(const Mlp &m, const double *x, int64_t n, double *y) {
  const int ni = m.nin, nh = m.nh;
  std::vector<double> h1(nh), h2(nh);
  for (int64_t s = 0; s < n; ++s) {
    for (int o = 0; o < nh; ++o) {
      double a = m.b1[o];
      for (int i = 0; i < ni; ++i) a += m.w1[o * ni + i] * x[s * ni + i];
      h1[o] = std::tanh(a);
    }
    for (int o = 0; o < nh; ++o) {
      double a = m.b2[o];
      for (int i = 0; i < nh; ++i) a += m.w2[o * nh + i] * h1[i];
      h2[o] = std::tanh(a);
    }
    double a = m.b3[0];
    for (int i = 0; i < nh; ++i) a += m.w3[i] * h2[i];
    y[s] = a;
  }
}

double mlp_loss_grad(const Mlp &m, const double *x, const double *y, int64_t n,
                     Mlp &g) {
  const int ni = m.nin, nh = m.nh;
  g = m;
  for (auto *v : {&g.w1, &g.b1, &g.w2, &g.b2, &g.w3, &g.b3})
    for (auto &e : *v) e = 0.;
  std::vector<double> h1(nh), h2(nh), d2(nh), d1(nh);
  double loss = 0.;
  for (int64_t s = 0; s < n; ++s) {
    const double *xs = x + s * ni;
    for (int o = 0; o < nh; ++o) {
      double a = m.b1[o];
      for (int i = 0; i < ni; ++i) a += m.w1[o * ni + i] * xs[i];
      h1[o] = std::tanh(a);
    }
    for (int o = 0; o < nh; ++o) {
      double a = m.b2[o];
      for (int i = 0; i < nh; ++i) a += m.w2[o * nh + i] * h1[i];
      h2[o] = std::tanh(a);
    }
    double out = m.b3[0];
    for (int i = 0; i < nh; ++i) out += m.w3[i] * h2[i];
    double r = out - y[s];
    loss += r * r;
    double dy = 2. * r / (double)n;  // d(mean r^2)/d out
    g.b3[0] += dy;
    for (int i = 0; i < nh; ++i) {
      g.w3[i] += dy * h2[i];
      d2[i] = dy * m.w3[i] * (1. - h2[i] * h2[i]);
    }
    for (int o = 0; o < nh; ++o) {
      g.b2[o] += d2[o];
      for (int i = 0; i < nh; ++i) g.w2[o * nh + i] += d2[o] * h1[i];
    }
    for (int i = 0; i < nh; ++i) {
      double a = 0.;
      for (int o = 0; o < nh; ++o) a += m.w2[o * nh + i] * d2[o];
      d1[i] = a * (1. - h1[i] * h1[i]);
    }
    for (int o = 0; o < nh; ++o) {
      g.b1[o] += d1[o];
      for (int i = 0; i < ni; ++i) g.w1[o * ni + i] += d1[o] * xs[i];
    }
  }
  return loss / (double)n;
}

}  // namespace oracle

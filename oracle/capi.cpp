// capi.cpp -- C entry points of the oracle for the Python test harness
// (ctypes).  TEST INFRASTRUCTURE ONLY.
#include <cstring>
#include <exception>
#include <string>

#include "oracle.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

using oracle::Block;

static thread_local std::string g_err;

extern "C" {

const char *oracle_last_error() { return g_err.c_str(); }

int oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void *oracle_block_new(const canoe_block_config_t *cfg) {
  try {
    Block *b = new Block();
    oracle::block_init(*b, *cfg);
    return b;
  } catch (std::exception &e) {
    g_err = e.what();
    return nullptr;
  }
}

void oracle_block_free(void *h) { delete static_cast<Block *>(h); }

void oracle_block_set_roundtrip(void *h, int on) {
  static_cast<Block *>(h)->fix_roundtrip = on != 0;
}

void oracle_block_set_diffusion(void *h, double K, double p0) {
  static_cast<Block *>(h)->diff_K = K;
  static_cast<Block *>(h)->diff_p0 = p0;
}

int oracle_block_set_conserved(void *h, const double *u) {
  Block &b = *static_cast<Block *>(h);
  std::memcpy(b.u.data(), u, b.u.size() * sizeof(double));
  oracle::cons_to_prim_block(b);
  return 0;
}

int oracle_block_set_primitive(void *h, const double *w) {
  Block &b = *static_cast<Block *>(h);
  std::memcpy(b.w.data(), w, b.w.size() * sizeof(double));
  return 0;
}

int oracle_block_get_conserved(void *h, double *u) {
  Block &b = *static_cast<Block *>(h);
  std::memcpy(u, b.u.data(), b.u.size() * sizeof(double));
  return 0;
}

int oracle_block_get_primitive(void *h, double *w) {
  Block &b = *static_cast<Block *>(h);
  std::memcpy(w, b.w.data(), b.w.size() * sizeof(double));
  return 0;
}

int oracle_block_calculate_fluxes(void *h, double *f1, double *f2, double *f3) {
  Block &b = *static_cast<Block *>(h);
  try {
    std::fill(b.flx1.begin(), b.flx1.end(), 0.);
    std::fill(b.flx2.begin(), b.flx2.end(), 0.);
    std::fill(b.flx3.begin(), b.flx3.end(), 0.);
    oracle::calculate_fluxes(b);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  if (f1) std::memcpy(f1, b.flx1.data(), b.flx1.size() * sizeof(double));
  if (f2) std::memcpy(f2, b.flx2.data(), b.flx2.size() * sizeof(double));
  if (f3) std::memcpy(f3, b.flx3.data(), b.flx3.size() * sizeof(double));
  return 0;
}

int oracle_block_solve_implicit(void *h, double *du, double dt) {
  Block &b = *static_cast<Block *>(h);
  try {
    std::vector<double> d(du, du + b.u.size());
    oracle::solve_implicit(b, d, dt);
    std::memcpy(du, d.data(), d.size() * sizeof(double));
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

int oracle_periodic_block_solve(int nb, int n, const double *a, const double *b,
                                const double *c, const double *rhs, double *x) {
  return oracle::periodic_block_solve(nb, n, a, b, c, rhs, x);
}

int oracle_block_step(void *h, double dt, int nsteps) {
  Block &b = *static_cast<Block *>(h);
  try {
    for (int s = 0; s < nsteps; ++s) {
      double d = dt > 0. ? dt : oracle::new_dt(b);
      oracle::step(b, d);
    }
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

double oracle_block_new_dt(void *h) { return oracle::new_dt(*static_cast<Block *>(h)); }

int oracle_block_stage(void *h, int stage, double dt) {
  Block &b = *static_cast<Block *>(h);
  try {
    oracle::stage_step(b, dt, stage);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

// The x1 hydrostatic decomposition of column (k, j) of the block's primitive
// state: q (nv x nc1) receives the decomposed pencil (T, p'), psf (nc1 + 1),
// psv and gam (nc1) the column's hydrostatic arrays.
int oracle_x1_change_to_temperature(void *h, int k, int j, double *q, double *psf,
                                    double *psv, double *gam) {
  Block &b = *static_cast<Block *>(h);
  for (int n = 0; n < b.nv; ++n)
    for (int i = 0; i < b.nc1; ++i) q[n * b.nc1 + i] = b.w[b.idx(n, k, j, i)];
  oracle::change_to_temperature_pencil(b, k, j, q);
  std::memcpy(psf, &b.psf[((size_t)k * b.nc2 + j) * (b.nc1 + 1)], (b.nc1 + 1) * sizeof(double));
  std::memcpy(psv, &b.psv[b.idx(0, k, j, 0)], b.nc1 * sizeof(double));
  std::memcpy(gam, &b.gam[b.idx(0, k, j, 0)], b.nc1 * sizeof(double));
  return 0;
}

// Its inverse with the column's arrays of the last call above: q back to rho
// and p, face states wl / wr (nv x (nc1 + 1)) of faces lo..hi restored.
int oracle_x1_restore_from_temperature(void *h, int k, int j, double *q, double *wl,
                                       double *wr, int lo, int hi) {
  Block &b = *static_cast<Block *>(h);
  oracle::restore_from_temperature_pencil(b, k, j, q, wl, wr, lo, hi);
  return 0;
}

int oracle_riemann(int rsolver, const canoe_thermo_t *th, int ivx,
                   const double *wl, const double *wr, double *flx, int64_t n) {
  if (rsolver == CANOE_RSOLVER_LMARS)
    oracle::riemann_lmars(*th, ivx, wl, wr, flx, n);
  else
    oracle::riemann_hllc(*th, ivx, wl, wr, flx, n);
  return 0;
}

int oracle_cons_to_prim(const canoe_thermo_t *th, const double *u, double *w,
                        int64_t n) {
  for (int64_t c = 0; c < n; ++c) oracle::cons_to_prim_cell(*th, u + c, w + c, n);
  return 0;
}

int oracle_prim_to_cons(const canoe_thermo_t *th, const double *w, double *u,
                        int64_t n) {
  for (int64_t c = 0; c < n; ++c) oracle::prim_to_cons_cell(*th, w + c, u + c, n);
  return 0;
}

int oracle_satadj(const canoe_thermo_t *th, const canoe_satadj_opts_t *o,
                  double *u, int64_t n, const double *t_guess, double *t_out,
                  int32_t *iters, int32_t *flags) {
  // o->warm: 0 cold, 1 start at t_guess, 2 hybrid (see satadj_cell)
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    oracle::SatResult r =
        oracle::satadj_cell(*th, *o, u + c, n, t_guess ? t_guess[c] : 0.);
    if (t_out) t_out[c] = r.t;
    if (iters) iters[c] = r.iters;
    if (flags) flags[c] = (r.fallback ? 1 : 0) | (r.converged ? 0 : 2);
  }
  return 0;
}

// params: w1[nh*4], b1[nh], w2[nh*nh], b2[nh], w3[nh], b3[1], contiguous
static oracle::Mlp unpack(const double *p, int nh) {
  oracle::Mlp m;
  m.nh = nh;
  const double *q = p;
  m.w1.assign(q, q + nh * 4); q += nh * 4;
  m.b1.assign(q, q + nh); q += nh;
  m.w2.assign(q, q + nh * nh); q += nh * nh;
  m.b2.assign(q, q + nh); q += nh;
  m.w3.assign(q, q + nh); q += nh;
  m.b3.assign(q, q + 1);
  return m;
}

int oracle_mlp_forward(const double *params, int nh, const double *x, int64_t n,
                       double *y) {
  oracle::mlp_forward(unpack(params, nh), x, n, y);
  return 0;
}

double oracle_mlp_loss_grad(const double *params, int nh, const double *x,
                            const double *y, int64_t n, double *grad) {
  oracle::Mlp m = unpack(params, nh), g;
  double loss = oracle::mlp_loss_grad(m, x, y, n, g);
  double *q = grad;
  for (auto *v : {&g.w1, &g.b1, &g.w2, &g.b2, &g.w3, &g.b3}) {
    std::memcpy(q, v->data(), v->size() * sizeof(double));
    q += v->size();
  }
  return loss;
}

// ---------------------------------------------------------------------------
// cubed-sphere shell: state arrays are (6, nv, nc3, nc2, nc1)

void *oracle_shell_new(const canoe_shell_config_t *cfg) {
  try {
    oracle::Shell *s = new oracle::Shell();
    oracle::shell_init(*s, *cfg);
    return s;
  } catch (std::exception &e) {
    g_err = e.what();
    return nullptr;
  }
}

void oracle_shell_free(void *h) { delete static_cast<oracle::Shell *>(h); }

static size_t panel_size(const oracle::Shell &s) { return s.p[0].u.size(); }

int oracle_shell_set_conserved(void *h, const double *u) {
  auto &s = *static_cast<oracle::Shell *>(h);
  const size_t n = panel_size(s);
  for (int p = 0; p < 6; ++p) std::memcpy(s.p[p].u.data(), u + p * n, n * sizeof(double));
  return 0;
}

int oracle_shell_get(void *h, int which, double *out) {
  auto &s = *static_cast<oracle::Shell *>(h);
  const size_t n = panel_size(s);
  for (int p = 0; p < 6; ++p)
    std::memcpy(out + p * n, (which ? s.p[p].w : s.p[p].u).data(), n * sizeof(double));
  return 0;
}

int oracle_shell_set_primitive(void *h, const double *w) {
  auto &s = *static_cast<oracle::Shell *>(h);
  const size_t n = panel_size(s);
  for (int p = 0; p < 6; ++p) std::memcpy(s.p[p].w.data(), w + p * n, n * sizeof(double));
  return 0;
}

int oracle_shell_fill_ghosts(void *h) {
  try {
    oracle::shell_fill_ghosts(*static_cast<oracle::Shell *>(h));
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

int oracle_shell_cons_to_prim(void *h) {
  oracle::shell_cons_to_prim(*static_cast<oracle::Shell *>(h));
  return 0;
}

int oracle_shell_prim_to_cons(void *h) {
  oracle::shell_prim_to_cons(*static_cast<oracle::Shell *>(h));
  return 0;
}

// fluxes of the shell's current primitive state; f1/f2/f3 are
// (6, nv, nc3, nc2, nc1+1), (6, nv, nc3, nc2+1, nc1), (6, nv, nc3+1, nc2, nc1)
int oracle_shell_calculate_fluxes(void *h, double *f1, double *f2, double *f3) {
  auto &s = *static_cast<oracle::Shell *>(h);
  try {
    for (int p = 0; p < 6; ++p) {
      std::fill(s.p[p].flx1.begin(), s.p[p].flx1.end(), 0.);
      std::fill(s.p[p].flx2.begin(), s.p[p].flx2.end(), 0.);
      std::fill(s.p[p].flx3.begin(), s.p[p].flx3.end(), 0.);
    }
    oracle::shell_calculate_fluxes(s);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  for (int p = 0; p < 6; ++p) {
    const auto &b = s.p[p];
    if (f1) std::memcpy(f1 + p * b.flx1.size(), b.flx1.data(), b.flx1.size() * sizeof(double));
    if (f2) std::memcpy(f2 + p * b.flx2.size(), b.flx2.data(), b.flx2.size() * sizeof(double));
    if (f3) std::memcpy(f3 + p * b.flx3.size(), b.flx3.data(), b.flx3.size() * sizeof(double));
  }
  return 0;
}

int oracle_shell_step(void *h, double dt, int nsteps) {
  auto &s = *static_cast<oracle::Shell *>(h);
  try {
    for (int q = 0; q < nsteps; ++q) oracle::shell_step(s, dt);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

}  // extern "C"

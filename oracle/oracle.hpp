// oracle.hpp -- CPU FP64 restatement of canoe's dynamical-core hot path.
//
// TEST INFRASTRUCTURE ONLY.  This code is the checker for the CUDA path: it
// is imported only by tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg.  Nothing in the product (canoe_b200/) links or calls it.
//
// Parity status.  canoe's own arithmetic (Riemann solvers, hydrostatic
// decomposition, implicit vertical solver) is restated line for line from
// the canoe sources cited at each function.  The parts canoe delegates to
// external code that is absent from the reference snapshot are restated
// from published methods and are "parity unpinned":
//   * Athena++ (chengcli/athenapp @ 8c221aa): PLM (van Leer 1979), PPM
//     (Colella & Woodward 1984), SSPRK(3,3) (Shu & Osher 1988), flux
//     divergence, constant-gravity source, reflecting/periodic ghost cells;
//   * snapy (version unpinned): ideal-moist EOS cons<->prim;
//   * kintera (version unpinned): UV saturation adjustment.
// The reference ships no golden vectors for this path (its unit tests are
// disabled and its regression goldens are Git-LFS pointers), so the
// restatement is not pinned against reference outputs.
#pragma once

#include <cstdint>
#include <vector>

#include "../include/canoe_b200.h"

namespace oracle {

constexpr int NG = CANOE_NGHOST;

struct Block {
  canoe_block_config_t cfg;
  canoe_thermo_t th;
  int ny, nv, ivx, ivy, ivz, ipr;
  int nx1, nx2, nx3, nc1, nc2, nc3;
  int is, ie, js, je, ks, ke;
  bool f2, f3;
  std::vector<double> x1f, x1v, dx1f;  // x1 faces (nc1+1), centres, widths
  double dx2, dx3;
  // state: (nv, nc3, nc2, nc1)
  std::vector<double> u, w, u1, du;
  // fluxes: flx1 (nv,nc3,nc2,nc1+1), flx2 (nv,nc3,nc2+1,nc1),
  //         flx3 (nv,nc3+1,nc2,nc1)
  std::vector<double> flx1, flx2, flx3;
  // decomposition scratch (canoe decomposition.hpp:77-87)
  std::vector<double> psf, psv, gam;  // (nc3,nc2,nc1+1), (nc3,nc2,nc1) x2
  bool fix_roundtrip = true;  // write the T/p' round trip back into w

  size_t cells() const { return (size_t)nc3 * nc2 * nc1; }
  size_t idx(int n, int k, int j, int i) const {
    return (((size_t)n * nc3 + k) * nc2 + j) * nc1 + i;
  }
};

void block_init(Block &b, const canoe_block_config_t &cfg);

// thermodynamics ------------------------------------------------------------
double get_gamma(const canoe_thermo_t &th, const double *w);
double sound_speed(const canoe_thermo_t &th, const double *w);
void cons_to_prim_cell(const canoe_thermo_t &th, const double *u, double *w,
                       int64_t stride);
void prim_to_cons_cell(const canoe_thermo_t &th, const double *w, double *u,
                       int64_t stride);
double temperature_of_prim(const canoe_thermo_t &th, const double *w,
                           int64_t stride);

// Riemann solvers on (nv, n) face arrays ------------------------------------
void riemann_lmars(const canoe_thermo_t &th, int ivx, const double *wl,
                   const double *wr, double *flx, int64_t n);
void riemann_hllc(const canoe_thermo_t &th, int ivx, const double *wl,
                  const double *wr, double *flx, int64_t n);

// block-level -----------------------------------------------------------------
void apply_bc(Block &b, std::vector<double> &w);
void cons_to_prim_block(Block &b);
void calculate_fluxes(Block &b);
void add_flux_divergence(Block &b, double wght, std::vector<double> &du);
void add_gravity_source(Block &b, double dt, std::vector<double> &du);
void solve_implicit(Block &b, std::vector<double> &du, double dt);
double new_dt(const Block &b);
void step(Block &b, double dt);

// saturation adjustment (one cell, conserved, stride between variables) ----
struct SatResult {
  double t;
  int iters;
  bool fallback;
  bool converged;
};
SatResult satadj_cell(const canoe_thermo_t &th, const canoe_satadj_opts_t &o,
                      double *u, int64_t stride, double t_guess);
void satadj_block(Block &b, const canoe_satadj_opts_t &o);

// MLP (4 -> H -> H -> 1, tanh), fp32/fp64 reference -------------------------
struct Mlp {
  int nin = 4, nh = 64;
  std::vector<double> w1, b1, w2, b2, w3, b3;  // row-major [out][in]
};
void mlp_forward(const Mlp &m, const double *x, int64_t n, double *y);
// mean-squared-error loss and its gradient over a batch
double mlp_loss_grad(const Mlp &m, const double *x, const double *y, int64_t n,
                     Mlp &grad);

}  // namespace oracle

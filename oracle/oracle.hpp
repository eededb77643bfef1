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

// Panel geometry of an equiangular gnomonic cubed sphere
// (canoe src/exo3/gnomonic_equiangle.cpp:24-222); the six panels of a shell
// share one.  Angles x2, x3 in [-pi/4, pi/4]; (k, j) tables are row-major
// [k * nc2 + j].
struct ShellGeo {
  int N = 0, nc2 = 0, nc3 = 0;
  std::vector<double> x2f, x2v, x3f, x3v;
  std::vector<double> cosc, sinc, cosf2, sinf2, cosf3, sinf3;
  std::vector<double> dx2a, dx3a, dx2a_f3, dx3a_f2;
  size_t kj(int k, int j) const { return (size_t)k * nc2 + j; }
};

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
  // user source: the sinking bubble's dissipation (diffusivity, p0; 0 = off)
  double diff_K = 0., diff_p0 = 1.e5;
  // cubed-sphere panel: geometry and blockID - 1 (nullptr / -1 otherwise)
  const ShellGeo *geo = nullptr;
  int panel = -1;

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
// ke_cth: cosine of the cell for the covariant kinetic energy of the x1
// Riemann problem on a cubed-sphere panel (hllc_transform.cpp:92-101); null
// elsewhere
void riemann_hllc(const canoe_thermo_t &th, int ivx, const double *wl,
                  const double *wr, double *flx, int64_t n,
                  const double *ke_cth = nullptr);

// reconstruction along one line: cell values q, faces f between cells f-1
// and f; ql[f] / qr[f] left / right of face f for faces lo..hi
void plm_line(const double *q, int lo, int hi, double *ql, double *qr);
void ppm_line(const double *q, int lo, int hi, double *ql, double *qr);

// block-level -----------------------------------------------------------------
void apply_bc(Block &b, std::vector<double> &w);
void cons_to_prim_block(Block &b);
void calculate_fluxes(Block &b);
void calculate_fluxes_x1_only(Block &b);
// the x1 hydrostatic decomposition of one column's pencil q (nv x nc1) and its
// inverse on q and on face states wl / wr (nv x (nc1 + 1)) of faces lo..hi;
// psf / psv / gamma_ of the column live in the block
void change_to_temperature_pencil(Block &b, int k, int j, double *q);
void restore_from_temperature_pencil(Block &b, int k, int j, double *q, double *wl,
                                     double *wr, int lo, int hi);
void add_flux_divergence(Block &b, double wght, std::vector<double> &du);
void add_gravity_source(Block &b, double dt, std::vector<double> &du);
void solve_implicit(Block &b, std::vector<double> &du, double dt);
// the cyclic block-tridiagonal solve alone: rows 1..n of nb x nb blocks a, b,
// c (row-major, n + 1 blocks each; c[0] is the lower corner, the coupling of
// row n to row 1) and rhs; x receives rows 1..n
int periodic_block_solve(int nb, int n, const double *a, const double *b, const double *c,
                         const double *rhs, double *x);
double new_dt(const Block &b);
void step(Block &b, double dt);
// one RK stage (0, 1, 2) of step(): fluxes, divergence, sources, implicit
// correction, register update, saturation adjustment at stage 2, cons2prim
void stage_step(Block &b, double dt, int stage);

// cubed-sphere shell (exo3.cpp) ------------------------------------------------
struct Shell {
  canoe_shell_config_t cfg;
  int N = 0, nv = 0;
  ShellGeo geo;
  Block p[6];
  // x2 / x3 face states of every panel (CubedSphere L3DValues / R3DValues,
  // cubed_sphere.hpp:67): (nv, nc3, nc2 + 1, nc1) and (nv, nc3 + 1, nc2, nc1)
  std::vector<double> L2[6], R2[6], L3[6], R3[6];
};
void shell_init(Shell &s, const canoe_shell_config_t &cfg);
void shell_fill_ghosts(Shell &s);
void shell_cons_to_prim(Shell &s);
void shell_prim_to_cons(Shell &s);
void shell_calculate_fluxes(Shell &s);
void shell_step(Shell &s, double dt);
void shell_swap_lr(Shell &s);
void shell_add_divergence(Block &b, double wght, std::vector<double> &du);
// radial geometry of a panel cell (gnomonic_equiangle.cpp:224-432)
double shell_face1_area(const Block &b, int k, int j, int i);
double shell_cell_volume(const Block &b, int k, int j, int i);

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

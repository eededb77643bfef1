// ref_harness.cpp -- C entry points around a few of the reference's own
// source files, compiled as they lie in the reference tree against the shim
// headers of oracle/ref_shim.  TEST INFRASTRUCTURE ONLY: the checker that
// pins the oracle's restatement to the reference's arithmetic; nothing on the
// product path loads it.
//
// One library per unit and per NHYDRO (recipe: oracle/Makefile, target ref):
//   REF_UNIT_RIEMANN  Hydro::RiemannSolver of src/snap/riemann/lmars.cpp or
//                     src/snap/riemann/hllc_transform.cpp, with
//                     EquationOfState::SoundSpeed and the constructor of
//                     src/snap/eos/ideal_moist_hydro.cpp and get_gamma /
//                     get_rd / get_gammad of src/interface/eos.hpp
//   REF_UNIT_DECOMP   Decomposition::ChangeToTemperature and
//                     RestoreFromTemperature of
//                     src/snap/decomposition/change_to_temperature.cpp
//   REF_UNIT_IMPLICIT ImplicitSolver::PartialCorrection and FullCorrection of
//                     src/snap/implicit/{partial,full}_correction.cpp with
//                     the ForwardSweep / BackwardSubstitution and the flux
//                     decomposition of forward_backward.hpp and
//                     flux_decomposition.hpp, and SoundSpeed of
//                     src/snap/eos/ideal_moist_hydro.cpp
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <athena/athena.hpp>
#include <athena/coordinates/coordinates.hpp>
#include <athena/eos/eos.hpp>
#include <athena/hydro/hydro.hpp>
#include <athena/mesh/mesh.hpp>
#include <athena/parameter_input.hpp>
#include <impl.hpp>

#include "canoe_b200.h"

#ifdef REF_UNIT_DECOMP
#include <checks.hpp>
#include <snap/decomposition/decomposition.hpp>
#endif
#ifdef REF_UNIT_IMPLICIT
#include <snap/implicit/implicit_solver.hpp>
#endif

namespace {

std::string g_err;

// A MeshBlock with the members the compiled files reach, its thermodynamics
// taken from a canoe_thermo_t.  mu_d and cvd_R give kintera's dry molecular
// weight [kg/mol] and dry cv / R, from which src/interface/eos.hpp:14-21
// derives Rd and gamma_d.
struct RefBlock {
  MeshBlock mb;
  Coordinates co;
  Hydro hy;
  BoundaryValues bv;
  ParameterInput pin;
  std::unique_ptr<EquationOfState> eos;

  RefBlock(const canoe_thermo_t &th, double mu_d, double cvd_R) {
    if (th.ny != NHYDRO - 5) throw std::runtime_error("ny does not match this build's NHYDRO");
    kintera::species_weights = {mu_d};
    kintera::species_cref_R = {cvd_R};
    auto im = std::make_shared<snap::IdealMoistImpl>();
    im->pthermo = std::make_shared<kintera::ThermoYImpl>();
    // kintera lists the dry species among the vapours (eos.hpp:54)
    im->pthermo->options.vapor_ids_.assign(1 + th.nvapor, 0);
    im->pthermo->options.cloud_ids_.assign(th.ny - th.nvapor, 0);
    std::vector<double> cv(th.cv_ratio_m1, th.cv_ratio_m1 + CANOE_MAX_NY);
    std::vector<double> mu(th.inv_mu_ratio_m1, th.inv_mu_ratio_m1 + CANOE_MAX_NY);
    im->cv_ratio_m1 = torch::Tensor::from_vector(cv);
    im->inv_mu_ratio_m1 = torch::Tensor::from_vector(mu);
    mb.pimpl = std::make_shared<MeshBlock::Impl>();
    mb.pimpl->peos = im;
    mb.pcoord = &co;
    mb.phydro = &hy;
    mb.pbval = &bv;
    hy.pmy_block = &mb;
    hy.hsrc.g1_ = th.grav;
    pin.vals["hydro/gamma"] = th.gammad;
  }
};

}  // namespace

#if defined(REF_UNIT_RIEMANN) || defined(REF_UNIT_IMPLICIT)
// EquationOfState's general-EOS hooks: declared by Athena++, reached only
// when GENERAL_EOS is set (it is not in canoe's ideal-moist build).
Real EquationOfState::EgasFromRhoP(Real, Real) {
  throw std::runtime_error("general EOS is not part of this build");
}
Real EquationOfState::AsqFromRhoP(Real, Real) {
  throw std::runtime_error("general EOS is not part of this build");
}
#endif

#ifdef REF_UNIT_RIEMANN

extern "C" {

// Hydro::RiemannSolver on n faces: wl, wr (NHYDRO, n) left / right states,
// flx (NHYDRO, n) the face fluxes; ivx the normal velocity slot.
int ref_riemann(const canoe_thermo_t *th, double mu_d, double cvd_R, int ivx, const double *wl,
                const double *wr, double *flx, int64_t n) {
  try {
    RefBlock rb(*th, mu_d, cvd_R);
    rb.eos.reset(new EquationOfState(&rb.mb, &rb.pin));
    rb.mb.peos = rb.eos.get();
    rb.co.m.NewAthenaArray(1, 1, (int)n);
    AthenaArray<Real> L, R, F, dxw;
    L.InitWithShallowSlice(const_cast<double *>(wl), 1, 1, NHYDRO, (int)n);
    R.InitWithShallowSlice(const_cast<double *>(wr), 1, 1, NHYDRO, (int)n);
    F.InitWithShallowSlice(flx, NHYDRO, 1, 1, (int)n);
    rb.hy.RiemannSolver(0, 0, 0, (int)n - 1, ivx, L, R, F, dxw);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

// EquationOfState::SoundSpeed of n primitive states w (NHYDRO, n).
int ref_sound_speed(const canoe_thermo_t *th, double mu_d, double cvd_R, const double *w,
                    double *cs, int64_t n) {
  try {
    RefBlock rb(*th, mu_d, cvd_R);
    rb.eos.reset(new EquationOfState(&rb.mb, &rb.pin));
    Real prim[NHYDRO];
    for (int64_t c = 0; c < n; ++c) {
      for (int v = 0; v < NHYDRO; ++v) prim[v] = w[v * n + c];
      cs[c] = rb.eos->SoundSpeed(prim);
    }
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

const char *ref_last_error() { return g_err.c_str(); }
int ref_nhydro() { return NHYDRO; }

}  // extern "C"
#endif  // REF_UNIT_RIEMANN

#ifdef REF_UNIT_DECOMP
// The members of Decomposition that decomposition.cpp (MPI set-up and the
// other decompositions) would define: a single block with no neighbours.
namespace {
int g_nc1 = 0, g_nc2 = 0, g_nc3 = 0;
AthenaArray<Real> *g_psf = nullptr, *g_psv = nullptr, *g_gamma = nullptr;
}  // namespace

Decomposition::Decomposition(MeshBlock *pmb) : pmy_block_(pmb) {
  has_top_neighbor = has_bot_neighbor = false;
  psf_.NewAthenaArray(g_nc3, g_nc2, g_nc1 + 1);
  psv_.NewAthenaArray(g_nc3, g_nc2, g_nc1);
  gamma_.NewAthenaArray(g_nc3, g_nc2, g_nc1);
  g_psf = &psf_;
  g_psv = &psv_;
  g_gamma = &gamma_;
}
Decomposition::~Decomposition() {}
void Decomposition::FindNeighbors() { has_top_neighbor = has_bot_neighbor = false; }
void Decomposition::RecvFromTop(AthenaArray<Real> &, int, int, int, int) {
  throw std::runtime_error("a single block has no top neighbour");
}
void Decomposition::SendToBottom(AthenaArray<Real> const &, int, int, int, int) {
  throw std::runtime_error("a single block has no bottom neighbour");
}
// src/checks.cpp:113-131: the body is commented out in the reference
void check_decomposition(AthenaArray<Real> const &, AthenaArray<Real> const &, int, int, int,
                         int) {}

namespace {
BoundaryFlag flag_of(int bc) {
  switch (bc) {
    case CANOE_BC_REFLECT: return BoundaryFlag::reflect;
    case CANOE_BC_PERIODIC: return BoundaryFlag::periodic;
    case CANOE_BC_OUTFLOW: return BoundaryFlag::outflow;
    default: return BoundaryFlag::block;
  }
}

struct DecompBlock : RefBlock {
  std::unique_ptr<Decomposition> dec;
  DecompBlock(const canoe_thermo_t &th, double mu_d, int nc3, int nc2, int nc1, int is, int ie,
              const double *dx1f, const int *bc)
      : RefBlock(th, mu_d, 2.5) {
    mb.is = is;
    mb.ie = ie;
    co.dx1f.NewAthenaArray(nc1);
    for (int i = 0; i < nc1; ++i) co.dx1f(i) = dx1f[i];
    for (int q = 0; q < 6; ++q) bv.block_bcs[q] = flag_of(bc[q]);
    g_nc1 = nc1;
    g_nc2 = nc2;
    g_nc3 = nc3;
    dec.reset(new Decomposition(&mb));
  }
};
}  // namespace

extern "C" {

// ChangeToTemperature over columns kl..ku, jl..ju of a block w (NHYDRO, nc3,
// nc2, nc1) in place; psf (nc3, nc2, nc1 + 1), psv and gam (nc3, nc2, nc1)
// receive the decomposition's arrays.  bc[6] are canoe_bc flags (the x1
// inner / outer ones are used).
int ref_change_to_temperature(const canoe_thermo_t *th, double mu_d, int nc3, int nc2, int nc1,
                              int is, int ie, const double *dx1f, const int *bc, int kl, int ku,
                              int jl, int ju, double *w, double *psf, double *psv, double *gam) {
  try {
    DecompBlock db(*th, mu_d, nc3, nc2, nc1, is, ie, dx1f, bc);
    AthenaArray<Real> W;
    W.InitWithShallowSlice(w, NHYDRO, nc3, nc2, nc1);
    db.dec->ChangeToTemperature(W, kl, ku, jl, ju);
    std::memcpy(psf, g_psf->data(), sizeof(double) * nc3 * nc2 * (nc1 + 1));
    std::memcpy(psv, g_psv->data(), sizeof(double) * nc3 * nc2 * nc1);
    std::memcpy(gam, g_gamma->data(), sizeof(double) * nc3 * nc2 * nc1);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

// RestoreFromTemperature of column (k, j) with the given decomposition arrays
// (as ChangeToTemperature returned them): w (NHYDRO, nc3, nc2, nc1) in place,
// face states wl, wr (NHYDRO, nc1 + 1) of faces il..iu in place.
int ref_restore_from_temperature(const canoe_thermo_t *th, double mu_d, int nc3, int nc2,
                                 int nc1, int is, int ie, const double *dx1f, const int *bc,
                                 const double *psf, const double *psv, const double *gam,
                                 double *w, double *wl, double *wr, int k, int j, int il,
                                 int iu) {
  try {
    DecompBlock db(*th, mu_d, nc3, nc2, nc1, is, ie, dx1f, bc);
    std::memcpy(g_psf->data(), psf, sizeof(double) * nc3 * nc2 * (nc1 + 1));
    std::memcpy(g_psv->data(), psv, sizeof(double) * nc3 * nc2 * nc1);
    std::memcpy(g_gamma->data(), gam, sizeof(double) * nc3 * nc2 * nc1);
    AthenaArray<Real> W, L, R;
    W.InitWithShallowSlice(w, NHYDRO, nc3, nc2, nc1);
    L.InitWithShallowSlice(wl, 1, 1, NHYDRO, nc1 + 1);
    R.InitWithShallowSlice(wr, 1, 1, NHYDRO, nc1 + 1);
    db.dec->RestoreFromTemperature(W, L, R, k, j, il, iu);
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

const char *ref_last_error() { return g_err.c_str(); }
int ref_nhydro() { return NHYDRO; }

}  // extern "C"
#endif  // REF_UNIT_DECOMP

#ifdef REF_UNIT_IMPLICIT
// The members of ImplicitSolver that implicit_solver.cpp (input parsing, MPI
// set-up, the direction switch) would define: one block, whole columns,
// the x1 direction, reflecting ends (first and last block, not periodic).
namespace {
int gi_nc1 = 0, gi_nc2 = 0, gi_nc3 = 0;
AthenaArray<Real> *g_du = nullptr;
}  // namespace

ImplicitSolver::ImplicitSolver(MeshBlock *pmb, ParameterInput *) : pmy_block_(pmb) {
  implicit_flag_ = 1;
  mydir_ = X1DIR;
  has_top_neighbor = has_bot_neighbor = false;
  first_block = last_block = true;
  periodic_boundary = false;
  pole_at_bot = pole_at_top = false;
  buffer_ = nullptr;
  du_.NewAthenaArray(NHYDRO, gi_nc3, gi_nc2, gi_nc1);
  coefficients_.NewAthenaArray(gi_nc3, gi_nc2, gi_nc1, 100);
  g_du = &du_;
}
ImplicitSolver::~ImplicitSolver() {}

extern "C" {

// SolveImplicit3D's x1 part (solve_implicit_3d.cpp:92-142) on a Cartesian
// block: du (NHYDRO, nc3, nc2, nc1) is corrected in place column by column
// by PartialCorrection (full = 0) or FullCorrection (full = 1) with the
// primitive state w and the stage's dt; dx1f has nc1 entries.
int ref_implicit_correction(const canoe_thermo_t *th, double mu_d, double cvd_R, int full,
                            int nc3, int nc2, int nc1, int is, int ie, int js, int je, int ks,
                            int ke, const double *dx1f, double dx2, double dx3,
                            const double *w, double *du, double dt) {
  try {
    RefBlock rb(*th, mu_d, cvd_R);
    rb.eos.reset(new EquationOfState(&rb.mb, &rb.pin));
    rb.mb.peos = rb.eos.get();
    rb.mb.is = is;
    rb.mb.ie = ie;
    rb.mb.js = js;
    rb.mb.je = je;
    rb.mb.ks = ks;
    rb.mb.ke = ke;
    rb.co.dx1f.NewAthenaArray(nc1);
    for (int i = 0; i < nc1; ++i) rb.co.dx1f(i) = dx1f[i];
    rb.co.dx2f.NewAthenaArray(nc2);
    for (int j = 0; j < nc2; ++j) rb.co.dx2f(j) = dx2;
    rb.co.dx3f.NewAthenaArray(nc3);
    for (int k = 0; k < nc3; ++k) rb.co.dx3f(k) = dx3;
    rb.hy.w.InitWithShallowSlice(const_cast<double *>(w), NHYDRO, nc3, nc2, nc1);
    gi_nc1 = nc1;
    gi_nc2 = nc2;
    gi_nc3 = nc3;
    ImplicitSolver solver(&rb.mb, nullptr);
    const size_t n = (size_t)NHYDRO * nc3 * nc2 * nc1;
    std::memcpy(g_du->data(), du, n * sizeof(double));
    for (int k = ks; k <= ke; ++k)
      for (int j = js; j <= je; ++j) {
        if (full)
          solver.FullCorrection(*g_du, rb.hy.w, dt, k, j, is, ie);
        else
          solver.PartialCorrection(*g_du, rb.hy.w, dt, k, j, is, ie);
      }
    std::memcpy(du, g_du->data(), n * sizeof(double));
  } catch (std::exception &e) {
    g_err = e.what();
    return 1;
  }
  return 0;
}

const char *ref_last_error() { return g_err.c_str(); }
int ref_nhydro() { return NHYDRO; }

}  // extern "C"
#endif  // REF_UNIT_IMPLICIT

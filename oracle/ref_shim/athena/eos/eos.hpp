// Shim of Athena++ eos/eos.hpp: the EquationOfState members that canoe's
// src/snap/eos/ideal_moist_hydro.cpp defines and the Riemann solvers call.
#pragma once
#include "../athena.hpp"

class MeshBlock;
class ParameterInput;
class Coordinates;
struct FaceField;

class EquationOfState {
 public:
  EquationOfState(MeshBlock *pmb, ParameterInput *pin);
  void ConservedToPrimitive(AthenaArray<Real> &cons, const AthenaArray<Real> &prim_old,
                            const FaceField &b, AthenaArray<Real> &prim,
                            AthenaArray<Real> &bcc, Coordinates *pco, int il, int iu, int jl,
                            int ju, int kl, int ku);
  void PrimitiveToConserved(const AthenaArray<Real> &prim, const AthenaArray<Real> &bc,
                            AthenaArray<Real> &cons, Coordinates *pco, int il, int iu, int jl,
                            int ju, int kl, int ku);
  Real SoundSpeed(const Real prim[NHYDRO]);
  // Athena++'s general-EOS hooks; only reached when GENERAL_EOS is set
  Real EgasFromRhoP(Real rho, Real pres);
  Real AsqFromRhoP(Real rho, Real pres);
  void ApplyPrimitiveFloors(AthenaArray<Real> &prim, int k, int j, int i);
  void ApplyPrimitiveConservedFloors(AthenaArray<Real> &prim, AthenaArray<Real> &cons,
                                     AthenaArray<Real> &bcc, int k, int j, int i);
  Real GetGamma() const { return gamma_; }

 private:
  MeshBlock *pmy_block_;
  Real gamma_;
  Real density_floor_, pressure_floor_, scalar_floor_;
};

// Shim of Athena++ hydro/hydro.hpp: the Hydro members the compiled files use
// (the Riemann solver hook and the constant-acceleration source's g1).
#pragma once
#include "../athena.hpp"

class MeshBlock;

class HydroSourceTerms {
 public:
  Real GetG1() const { return g1_; }
  Real g1_ = 0.;
};

class Hydro {
 public:
  MeshBlock *pmy_block = nullptr;
  HydroSourceTerms hsrc;
  AthenaArray<Real> w;  // primitive state (the species correction reads it)
  void RiemannSolver(const int k, const int j, const int il, const int iu, const int ivx,
                     AthenaArray<Real> &wl, AthenaArray<Real> &wr, AthenaArray<Real> &flx,
                     const AthenaArray<Real> &dxw);
};

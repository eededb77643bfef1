// Shim of canoe src/impl.hpp: MeshBlock::Impl with the members the compiled
// files use (the snapy EOS; the decomposition object lives in the harness).
#pragma once
#include <memory>
#include <athena/athena.hpp>
#include <athena/mesh/mesh.hpp>
#include <snap/eos/ideal_moist.hpp>

class CubedSphere;
class ImplicitSolver;

class MeshBlock::Impl {
 public:
  AthenaArray<Real> du;
  std::shared_ptr<snap::IdealMoistImpl> peos;
  std::shared_ptr<CubedSphere> pexo3;
  std::shared_ptr<ImplicitSolver> phevi;
};

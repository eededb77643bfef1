// Shim of Athena++ mesh/mesh.hpp: the MeshBlock members the compiled files
// reach (index range, coordinates, EOS, hydro, boundary flags, canoe's Impl).
#pragma once
#include <memory>
#include "../athena.hpp"
#include "../bvals/bvals.hpp"
#include "../coordinates/coordinates.hpp"

class Coordinates;
class EquationOfState;
class Hydro;
class MeshBlock;

// the mesh's block lookup, reached only by neighbour exchanges a single
// block never makes
class Mesh {
 public:
  MeshBlock *FindMeshBlock(int) { return nullptr; }
};

class MeshBlock {
 public:
  class Impl;
  std::shared_ptr<Impl> pimpl;
  Mesh *pmy_mesh = nullptr;
  int gid = 0;
  Coordinates *pcoord = nullptr;
  EquationOfState *peos = nullptr;
  Hydro *phydro = nullptr;
  BoundaryValues *pbval = nullptr;
  int is = 0, ie = 0, js = 0, je = 0, ks = 0, ke = 0;
};

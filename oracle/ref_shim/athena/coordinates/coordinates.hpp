// Shim of Athena++ coordinates/coordinates.hpp: the x1 face spacing and the
// metric array the compiled files reference.
#pragma once
#include "../athena.hpp"

class Coordinates {
 public:
  AthenaArray<Real> dx1f, x1f, x1v, x2v, x3v, x2f, x3f;
  AthenaArray<Real> m;  // metric (unused by Cartesian arithmetic)
};

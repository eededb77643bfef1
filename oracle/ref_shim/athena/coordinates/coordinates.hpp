// Shim of Athena++ coordinates/coordinates.hpp: the spacings, the metric
// array the compiled files reference, and the face areas and cell volume of
// Athena++'s Cartesian coordinates (cartesian.cpp: a face is the product of
// the two transverse widths, a cell the product of all three).
#pragma once
#include "../athena.hpp"

class Coordinates {
 public:
  AthenaArray<Real> dx1f, dx2f, dx3f, x1f, x1v, x2v, x3v, x2f, x3f;
  AthenaArray<Real> m;  // metric (unused by Cartesian arithmetic)
  Real GetFace1Area(int k, int j, int i) { return dx2f(j) * dx3f(k); }
  Real GetFace2Area(int k, int j, int i) { return dx1f(i) * dx3f(k); }
  Real GetFace3Area(int k, int j, int i) { return dx1f(i) * dx2f(j); }
  Real GetCellVolume(int k, int j, int i) { return dx1f(i) * dx2f(j) * dx3f(k); }
};

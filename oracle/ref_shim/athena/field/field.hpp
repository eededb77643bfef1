// Shim of Athena++ field/field.hpp.
#pragma once
#include "../athena.hpp"
struct FaceField {
  AthenaArray<Real> x1f, x2f, x3f;
};

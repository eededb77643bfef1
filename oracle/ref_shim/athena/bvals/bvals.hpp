// Shim of Athena++ bvals/bvals.hpp: boundary flags and the neighbour record.
#pragma once
#include "../athena.hpp"

enum BoundaryFace { undef = -1, inner_x1 = 0, outer_x1, inner_x2, outer_x2, inner_x3, outer_x3 };
enum class BoundaryFlag { block = -1, undef, reflect, outflow, user, periodic, polar,
                          polar_wedge, shear_periodic };

struct SimpleNeighborBlock {
  int rank = 0, level = 0, lid = 0, gid = 0;
};
struct NeighborBlock {
  SimpleNeighborBlock snb;
};

class BoundaryValues {
 public:
  BoundaryFlag block_bcs[6];
};

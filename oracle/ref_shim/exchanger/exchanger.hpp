// Shim: the MPI exchanger is not part of a single-block pin.
#pragma once
#include <athena/bvals/bvals.hpp>

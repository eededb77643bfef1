// Shim of the generated canoe configure.h: a Cartesian, non-MPI build.
#pragma once

// Shim of Athena++ athena.hpp (chengcli/athenapp): the types, variable
// slots and constants the compiled reference files use.  Variable slots
// follow canoe's layout: IDN = 0, mass fractions 1..NHYDRO-5, IVX = IM1 =
// NHYDRO-4, IVY, IVZ, IPR = IEN = NHYDRO-1.
#pragma once
#include <cmath>
#include <limits>

#ifndef NHYDRO
#error "compile with -DNHYDRO=<5 + number of mass-fraction slots>"
#endif

using Real = double;

enum { IDN = 0, IVX = NHYDRO - 4, IVY = NHYDRO - 3, IVZ = NHYDRO - 2, IPR = NHYDRO - 1 };
enum { IM1 = IVX, IM2 = IVY, IM3 = IVZ, IEN = IPR };

#define NGHOST 3
#define NWAVE NHYDRO
#define NSCALARS 0
#define GENERAL_EOS 0
#define NON_BAROTROPIC_EOS 1
#define SIMD_WIDTH 4
// Athena++ athena.hpp
#define TINY_NUMBER 1.0e-20
#define HUGE_NUMBER 1.0e+36
#define SQR(x) ((x) * (x))

constexpr Real float_min{std::numeric_limits<float>::min()};

enum class TaskStatus { fail, success, next };
enum CoordinateDirection { X1DIR = 0, X2DIR = 1, X3DIR = 2 };

#include "athena_arrays.hpp"

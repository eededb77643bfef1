// Shim of snapy's snap.h: the variable-slot constant used by
// canoe src/interface/eos.hpp.
#pragma once
namespace snap {
constexpr int ICY = 1;  // first mass-fraction slot
}

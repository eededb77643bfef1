// Shim of Athena++ globals.hpp.
#pragma once
namespace Globals {
inline int my_rank = 0, nranks = 1;
}

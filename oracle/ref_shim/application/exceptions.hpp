// Shim: no application exceptions are thrown on the compiled path.
#pragma once
#include <stdexcept>

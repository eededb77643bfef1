// Shim: the cubed-sphere class is only reached under CUBED_SPHERE, which
// the Cartesian pin does not define.
#pragma once

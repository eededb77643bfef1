"""canoe_b200 -- B200-native dynamical-core hot path of canoe.

The compute is in the CUDA library canoe_b200/lib/libcanoe_b200.so (C ABI in
include/canoe_b200.h); this package holds the ctypes bindings, the host-side
MeshBlock mirror, thermodynamic parameter sets and the seeded problem
generators.
"""
from ._abi import CanoeError, load  # noqa: F401
from . import thermo, problems  # noqa: F401
from .block import MeshBlock  # noqa: F401
from .shell import Shell  # noqa: F401
from .batch import Batch  # noqa: F401
from .mesh import Mesh  # noqa: F401

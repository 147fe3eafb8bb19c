"""B200-native determinant-space FCI engine behind Forte's FCISolver interface.

The compute path is libfcib200.so (hand-written sm_100a CUDA + C++ host code behind the C ABI
in include/fcib.h); this package holds its ctypes binding, the FCISolver mirror of the
reference's ActiveSpaceMethod interface and the integral input helpers.
"""
from .integrals import ActiveSpaceIntegrals, from_chemist, synthetic, read_fcidump, dress_core  # noqa: F401
from .fci_solver import FCISolver, GenCISolver, StateInfo, RDMs, make_active_space_method, DEFAULT_OPTIONS  # noqa: F401

__all__ = ["ActiveSpaceIntegrals", "from_chemist", "synthetic", "read_fcidump", "dress_core", "FCISolver", "GenCISolver",
           "StateInfo", "RDMs", "make_active_space_method", "DEFAULT_OPTIONS"]

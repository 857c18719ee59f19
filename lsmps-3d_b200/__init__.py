"""lsmps3d_b200: B200-native (sm_100a) LSMPS per-step particle hot path.

Host-side mirror of the lsmps3D C++ module API over the C ABI in
include/lsmps_b200.h.  The directory name contains a hyphen, so the package
is loaded under the import name ``lsmps3d_b200`` (see
__graft_entry__.load_package()).

Importing the package needs only numpy; the device API (``api``) loads torch
and the CUDA library on first use and raises if the library is missing --
there is no CPU fallback.
"""

from . import abi, buffers, cases  # noqa: F401

__all__ = ["abi", "buffers", "cases", "api", "build"]


def __getattr__(name):
    if name in ("api", "build"):
        import importlib

        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)

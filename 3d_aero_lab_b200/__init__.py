"""B200-native 3D Euler cut-cell solver: a drop-in for the solver entry points of
WeiJungSong/3d_aero_lab `src/air_cfd.js`, implemented as hand-written sm_100a CUDA behind
the C ABI of include/aero3d.h (libaero3d.so, built in-tree by build.py).

Import with importlib (the directory name starts with a digit):
    aero = importlib.import_module("3d_aero_lab_b200")
"""
from . import abi, aircraft, engine, field  # noqa: F401  (pure host code, no library needed)
from .aircraft import build_aircraft, shape_of, trefftz_x  # noqa: F401
from .field import fix_states  # noqa: F401


def __getattr__(name):
    # the solver surface loads libaero3d.so on first use and raises if it cannot
    if name in ("cfd", "CfdGPU", "Case", "Batch", "cfd_grid", "cfd_geom", "freestream", "AeroError"):
        import importlib
        cfd = importlib.import_module(__name__ + ".cfd")
        _lib = importlib.import_module(__name__ + "._lib")
        if name == "cfd":
            return cfd
        if name == "AeroError":
            return _lib.AeroError
        return getattr(cfd, name)
    raise AttributeError(name)

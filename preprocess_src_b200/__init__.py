"""B200-native coupled fluid-membrane time step (D3Q19 LBM + immersed boundary +
Skalak membrane FEM), a drop-in for the step modules of
enomoto-catallaxy/preProcess_src.

The compute path is the sm_100a library built from ``csrc/`` and called
through the C ABI of ``include/rbc_step.h``; see ``step.Simulation``.
"""
from . import configs, mesh  # noqa: F401

__all__ = ["configs", "mesh", "Simulation", "lib_path"]


def lib_path():
    from ._native import LIB_PATH
    return LIB_PATH


def __getattr__(name):
    if name == "Simulation":
        from .step import Simulation
        return Simulation
    raise AttributeError(name)

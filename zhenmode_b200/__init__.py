"""B200 (sm_100a) implementation of ZhenMode's global ocean step.

``make_solver_global`` is the drop-in for
``zhenmode.model.solver.factory.make_solver_global``; the arithmetic runs in
the CUDA library ``libzm_b200.so`` behind the C ABI of ``include/zm_b200.h``.
"""
from .config import GlobalOceanGrid, PhysicsConfig  # noqa: F401
from .solver import JaxStateG, UnsupportedOption, make_solver_global  # noqa: F401

__all__ = ["GlobalOceanGrid", "PhysicsConfig", "JaxStateG", "UnsupportedOption", "make_solver_global"]

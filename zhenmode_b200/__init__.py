"""B200 (sm_100a) implementation of ZhenMode's global ocean step.

``make_solver_global`` is the drop-in for
``zhenmode.model.solver.factory.make_solver_global``; the arithmetic runs in
the CUDA library ``libzm_b200.so`` behind the C ABI of ``include/zm_b200.h``.
"""
from .config import GlobalOceanGrid, PhysicsConfig  # noqa: F401
from .solver import (BudgetDiagnostics, JaxStateG, UnsupportedOption, compute_budget_diagnostics,  # noqa: F401
                     make_solver_global)

__all__ = ["GlobalOceanGrid", "PhysicsConfig", "JaxStateG", "UnsupportedOption", "make_solver_global",
           "BudgetDiagnostics", "compute_budget_diagnostics"]

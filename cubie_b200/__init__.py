"""cubie_b200: a B200-native batch ODE integration engine.

Drop-in for the integrator hot path of CuBIE: the same Python surface
(``solve_ivp``, ``Solver``, ``create_ODE_system``, ``SolveResult``) over
hand-written CUDA integrator kernels compiled with NVRTC for sm_100a and
launched through a C ABI (``include/cubie_b200.h``).
"""

from .result_codes import CUBIE_RESULT_CODES, decode_status_codes
from .symbolic import SymbolicODE, create_ODE_system
from .solver import Solver, solve_ivp
from .solveresult import SolveResult, SolveSpec
from .tableaus import TABLEAU_REGISTRY, Tableau, resolve_algorithm
from .graph import GraphSolve
from .interpolator import ArrayInterpolator
from .adjoint import AdjointIntegrator, solve_ivp_adjoint
from .autotune import autotune
from .cellml import load_cellml_model
from .structural import (ExtraEquationsSystemError, ExtraVariablesSystemError, InvalidSystemError,
                         structural_simplify)

__version__ = "0.1.0"

__all__ = [
    "load_cellml_model", "structural_simplify", "InvalidSystemError", "ExtraEquationsSystemError",
    "ExtraVariablesSystemError",
    "CUBIE_RESULT_CODES", "decode_status_codes", "SymbolicODE", "create_ODE_system",
    "Solver", "solve_ivp", "SolveResult", "SolveSpec", "TABLEAU_REGISTRY", "Tableau",
    "resolve_algorithm", "GraphSolve", "ArrayInterpolator", "AdjointIntegrator", "solve_ivp_adjoint", "autotune",
]

"""CPU oracle for the batch ODE integrator: TEST INFRASTRUCTURE ONLY.

This package restates, in numpy, the reference CuBIE integrator's
algorithm (loop, steps, controllers, Newton and Krylov solvers, outputs)
so that the CUDA engine's results can be checked against it.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
may import it; the product path (``cubie_b200``) never does.

Parity pins: the oracle is checked against (a) fixtures produced by the
reference's own kernels run on the CPU under Numba's CUDA simulator
(``tests/golden/make_reference_fixtures.py``) and (b) the reference's
DifferentialEquations.jl golden vectors (``tests/golden/make_julia_fixture.py``).
"""

from .ode_oracle import DriverTable, OracleSystem, integrate, TABLEAUS

__all__ = ["DriverTable", "OracleSystem", "integrate", "TABLEAUS"]

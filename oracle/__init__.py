"""CPU oracle for the pycfd projection hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain NumPy/SciPy, the algorithm of the reference
solver (kiliancmd/pycfd) for the per-timestep projection path: the momentum
stencil, the boundary passes, the immersed-boundary mask, the divergence, the
Poisson assembly and its solvers (Jacobi-PCG, damped Jacobi, red/black SOR,
smoothed-aggregation multigrid standalone and as the CG preconditioner) and the
SSP-RK3/RK2/Euler step with its adaptive time-step control.

It is the *checker*: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
legs of ``bench.py`` (``cpu_baseline`` and ``--impl reference``) may import it.
The product package ``pycfd_b200`` never imports, calls or links anything in
here, and has no CPU fallback onto it.

Pinning: every function cites the reference file:line it restates, and
``tests/test_oracle_golden.py`` checks this restatement against golden vectors
that ``tests/golden/make_golden.py`` produced by running the reference itself
(RHS bit-exact, Poisson operator exact, hierarchy and steps to round-off).
"""

from .stencil import momentum_rhs, divergence
from .boundary import Walls
from .poisson import (PoissonSystem, assemble_poisson, make_solver, CG, Jacobi,
                      SOR, Multigrid, MultigridCG)
from .multigrid import Hierarchy
from .projection import OracleSolver, OracleStepper, circle_mask_oracle, DivergenceError

__all__ = [
    "momentum_rhs", "divergence", "Walls", "PoissonSystem", "assemble_poisson",
    "make_solver", "CG", "Jacobi", "SOR", "Multigrid", "MultigridCG", "Hierarchy",
    "OracleSolver", "OracleStepper", "circle_mask_oracle", "DivergenceError",
]

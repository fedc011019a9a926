"""polysolve_b200 — a B200-native (sm_100a) implementation of polysolve's MAS-preconditioned CG.

The product is ``libpolysolve_mas.so``: hand-written CUDA kernels plus C++ host code behind the C ABI
declared in ``include/polysolve_mas.h``. This package holds its sources (``csrc/``), the build
recipe (``_build.py``), the Python mirror of polysolve's ``Solver`` interface (``solver.py``) and the
seeded synthetic elasticity workloads (``synthetic.py``).
"""

from .solver import (CudaOutOfMemoryError, MasError, MASSolver, Solver, WarmStartTrainer, library, solve_batch,
                     solve_batch_device)

__all__ = ["Solver", "MASSolver", "MasError", "CudaOutOfMemoryError", "WarmStartTrainer", "library", "solve_batch",
           "solve_batch_device"]

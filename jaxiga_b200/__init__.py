"""jaxiga_b200 -- the Galerkin linear-solve path of JAXIGA on NVIDIA B200.

Single-patch tensor-product NURBS spaces; Poisson (incl. per-point
coefficients), linear elasticity and Kirchhoff plates; matrix-free,
sum-factorised FP64 operator application with deterministic accumulation and
device Jacobi-PCG, plus FP32 inner solves inside FP64 iterative refinement.
All arithmetic runs in the hand-written sm_100a kernels of ``libjxb.so``.

Quick start (the reference's README example)::

    import numpy as np
    import jaxiga_b200 as jx

    patch = jx.primitives.quadrilateral([[0, 0], [1, 0], [1, 1], [0, 1]]).elevate(3).refine(5)
    V = jx.FunctionSpace(patch)
    f = lambda x, p: 8 * np.pi**2 * np.sin(2 * np.pi * x[0]) * np.sin(2 * np.pi * x[1])
    problem = jx.Poisson(V, dirichlet=[jx.DirichletBC(0.0, where=lambda x: np.full(len(x), True))], source=f)
    sol = jx.solve(problem, params={"a0": 1.0})
"""

from .adjoint import SOLVE_COUNTER, adjoint_solve, parameter_gradients, reset_solve_counter, value_and_grad
from .csr import CSRPattern, DeviceCG
from .forms import (ClampedBC, DirichletBC, Hyperelasticity, KirchhoffPlate, LinearElasticity, Neumann, PointField,
                    Poisson, Problem)
from .geometry import Patch, primitives
from .hierarchical import HierarchicalSpace, Hierarchy, HierarchyError, dorfler_mark, refine_elements
from .estimators import adapt, residual_indicator
from .newton import history_list
from .operator import Operator
from .pointset import PointSet, gauss
from .solve import LinearOptions, Solution, errornorm, integrate, norm, solve
from .space import FunctionSpace, bezier_extraction, element_spans, expand_dofs

__version__ = "0.1.0"

__all__ = [
    "Patch", "primitives", "FunctionSpace", "expand_dofs", "bezier_extraction", "element_spans",
    "Problem", "DirichletBC", "ClampedBC", "Neumann", "PointField", "Poisson", "LinearElasticity",
    "KirchhoffPlate", "solve", "LinearOptions", "Solution", "errornorm", "norm", "integrate", "Operator",
    "PointSet", "gauss", "value_and_grad", "adjoint_solve", "parameter_gradients", "SOLVE_COUNTER",
    "reset_solve_counter", "DeviceCG", "CSRPattern", "Hyperelasticity", "history_list",
    "HierarchicalSpace", "Hierarchy", "HierarchyError", "refine_elements", "dorfler_mark",
    "residual_indicator", "adapt",
]

"""Drop-in for the reference's ``src.bem`` package (solver.py, BiCGSTAB.py)."""
from .adjoint import cmatmul_adjoint, conj_transpose, listener_pressure  # noqa: F401
from .bicgstab import BiCGSTAB  # noqa: F401
from .modal import solve_modes  # noqa: F401
from .solver import (  # noqa: F401
    BEM_Solver,
    Geometry,
    check_tensor,
    cmatmul,
    gmres,
    map_triangle2vertex,
    preprocess,
    solve_linear_equation,
)

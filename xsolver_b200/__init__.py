"""xsolver_b200 — B200 (sm_100a) preconditioned Krylov solve path behind the
xsolver C API.

The product is the CUDA library ``libxsolver_b200.so`` (built in-tree from
``csrc/`` by ``xsolver_b200.build``) with the C ABI declared in
``include/xsolver_c.h``.  This package holds the host-side Python mirror of
that interface (``api``), the synthetic stencil generators (``stencils``) and
a torch.autograd wrapper over the adjoint (``autograd``).
"""
from .stencils import (CSRMatrix, convdiff3d_27pt, poisson2d_5pt, poisson3d_7pt, rhs_uniform,  # noqa: F401
                       varcoef3d_7pt)

__version__ = "1.0"


def __getattr__(name):
    # lazy: importing the package must not require the CUDA library
    if name in ("Solver", "Plan", "XsError"):
        from . import api

        return getattr(api, name)
    raise AttributeError(name)

"""Linear solver API, drop-in for redbirdpy's ``femsolve``
(redbirdpy/solver.py:385-948).

Every ``method`` resolves to the one GPU solver: Jacobi-preconditioned block
CG (real SPD) or block COCG (complex symmetric) over all right-hand sides at
once, in FP32 with FP64 iterative refinement (``precision='mixed'``, the
default) or entirely in FP64 (``precision='fp64'``).  By default the
refinement runs to the FP64 accuracy floor, which is what the reference's
default direct solver (SuperLU) delivers; ``tol`` sets an explicit relative
residual target instead.
"""

import numpy as np
import torch
from scipy import sparse

from . import engine

__all__ = ["femsolve", "solverinfo", "solver_options"]

_KNOWN_METHODS = {"auto", "direct", "superlu", "pardiso", "umfpack", "cholmod", "blqmr", "cg", "cg+amg",
                  "gmres", "bicgstab", "qmr", "minres", "minres+amg", "gpu"}


def solver_options(kw):
    """Map femsolve keyword arguments onto engine.solve options."""
    opts = {}
    if "precision" in kw:
        opts["precision"] = kw["precision"]
    method = kw.get("method", "auto")
    if method not in _KNOWN_METHODS:
        raise ValueError(f"Unknown solver method: {method}")
    # iterative methods honour the reference's tol; direct ones mean "to FP64 accuracy"
    if "tol" in kw and method not in ("auto", "direct", "superlu", "pardiso", "umfpack", "cholmod"):
        opts["tol"] = float(kw["tol"])
    if "refine_tol" in kw:
        opts["tol"] = float(kw["refine_tol"])
    for k in ("inner_tol", "maxiter", "max_outer", "check_every", "profile", "coarse", "groups", "spmm_lanes"):
        if k in kw:
            opts[k] = kw[k]
    return opts


def femsolve(Amat, rhs, method="auto", **kwargs):
    """Solve ``Amat x = rhs`` for all columns; returns ``(x, flag)`` with
    flag 0 on convergence, 1 when the iteration cap was hit, 2 on Krylov
    breakdown.  1-D rhs gives 1-D x; all-zero columns give exact zeros."""
    if method not in _KNOWN_METHODS:
        raise ValueError(f"Unknown solver method: {method}")
    if sparse.issparse(rhs):
        rhs = rhs.toarray()
    rhs = np.asarray(rhs)
    one_d = rhs.ndim == 1
    if one_d:
        rhs = rhs.reshape(-1, 1)
    if np.iscomplexobj(rhs):
        raise NotImplementedError("complex right-hand sides are outside this engine's scope")
    if isinstance(Amat, engine.DeviceMatrix):
        mat = Amat
    else:
        mat = engine.DeviceMatrix.from_scipy(Amat)
    B = torch.as_tensor(np.ascontiguousarray(rhs, dtype=np.float64), device=mat.val64.device)
    X, info = engine.solve(mat, B, **solver_options(dict(kwargs, method=method)))
    x = X.cpu().numpy()
    if kwargs.get("verbose", False):
        print(f"femsolve: gpu block {'COCG' if mat.is_complex else 'PCG'}, n={mat.n}, ncol={rhs.shape[1]}, "
              f"iters={info['iters']}, sweeps={info['outer']}, relres={info['relres']:.2e}")
    return (x[:, 0] if one_d else x), int(info["flag"])


def solverinfo():
    """Which backend answers femsolve here (redbirdpy/solver.py:951-974)."""
    return {"direct_solver": "gpu-refined-pcg", "has_umfpack": False, "has_cholmod": False,
            "has_amg": False, "has_blqmr": False, "gpu": True}

"""Gauss-Newton reconstruction API, drop-in for redbirdpy's ``recon`` module
(redbirdpy/recon.py): ``runrecon``, ``reginv``, ``reginvunder``,
``reginvover``, ``matreform``, ``matflat``, ``syncprop``.

The device loop keeps the mesh, fields and Jacobian on the GPU: forward
solve -> Jacobian rows (``rb_jac``) -> Frobenius scaling (``rb_sumsq``) ->
``J J^T`` on the tensor cores (``rb_gram``) -> FP64 Cholesky -> ``J^T y``.
Only detector values, misfits and the update vector cross to the host.

Scope: single wavelength, one mesh, node-based properties (the recon prop
has one row per forward-mesh node), no structural prior.  Label-based and
dual-mesh reconstruction, multi-spectral ``param`` and priors raise
NotImplementedError.  Additive options (not in the reference):
``param='mua'`` (default, the reference's update) or ``'mua+D'`` (node-wise
mua and diffusion coefficient with exact Jacobians); ``jac_mode``
('reference' | 'exact'); ``gram`` ('tf32' | 'tf32x3'); ``lambda_rule``
('fixed', the reference's, or 'maxdiag': lambda_ * max diag(J J^T)).
"""

import time

import numpy as np
import torch

from . import engine
from .forward import forward_device
from .utility import sdmap

__all__ = ["runrecon", "reginv", "reginvover", "reginvunder", "matreform", "matflat", "syncprop"]


# ------------------------------------------------------------------ algebra
def matreform(Amat, ymeas, ymodel, form="complex"):
    """Reformulate J dmu = y (recon.py:512-567): 'complex' (as is), 'real' /
    'reim' (stack real and imaginary parts), 'logphase' (log-amplitude and
    phase rows).  Returns (newA, newrhs, nblock)."""
    rhs = ymeas - ymodel
    if form == "complex":
        return Amat, rhs, 1
    if form in ("real", "reim"):
        if not np.isreal(rhs).all() and not np.isreal(Amat).all():
            if form == "reim":
                A = np.block([[np.real(Amat), -np.imag(Amat)], [np.imag(Amat), np.real(Amat)]])
            else:
                A = np.vstack([np.real(Amat), np.imag(Amat)])
            return A, np.concatenate([np.real(rhs), np.imag(rhs)]), 2
        return np.real(Amat), np.real(rhs), 1
    if form == "logphase":
        scale = np.conj(ymodel) / np.abs(ymodel * ymodel)
        A = scale[:, None] * Amat if Amat.ndim == 2 else scale * Amat
        if np.isreal(ymodel).all():
            return np.real(A), np.log(np.abs(ymeas)) - np.log(np.abs(ymodel)), 1
        return (np.vstack([np.real(A), np.imag(A)]),
                np.concatenate([np.log(np.abs(ymeas)) - np.log(np.abs(ymodel)), np.angle(ymeas) - np.angle(ymodel)]),
                2)
    raise ValueError(f"Unknown form: {form}")


def matflat(Amat, weight=None):
    """Concatenate a dict of Jacobian blocks (recon.py:570-593)."""
    if isinstance(Amat, np.ndarray):
        return Amat
    if isinstance(Amat, dict):
        keys = list(Amat.keys())
        w = np.ones(len(keys)) if weight is None else weight
        first = Amat[keys[0]]
        if isinstance(first, dict):
            return np.vstack([np.hstack([Amat[k][wv] * w[j] for j, k in enumerate(keys)]) for wv in first])
        return np.hstack([Amat[k] * w[i] for i, k in enumerate(keys)])
    return Amat


def _device_rows(A):
    """Upload a host matrix as FP32 rows with a 4-float-aligned stride."""
    A = np.asarray(A)
    if np.iscomplexobj(A):
        raise ValueError("reginv expects a real matrix (use matreform first)")
    M, K = A.shape
    ld = engine._pad4(K)
    J = torch.zeros((M, ld), dtype=torch.float32, device=engine._dev())
    J[:, :K] = torch.as_tensor(np.ascontiguousarray(A, dtype=np.float32), device=J.device)
    return J, K


def reginvunder(Amat, rhs, lambda_, invR=None, blocks=None, precision="tf32x3", **kwargs):
    """Underdetermined regularised solve (recon.py:429-509):
    dmu = J^T (J J^T + lambda I)^-1 r with unit-diagonal normalisation.
    J J^T runs on the tensor cores (``precision`` 'tf32' or 'tf32x3'), the
    Cholesky and substitutions in FP64.  (Zero rows/columns that the
    reference drops contribute nothing to J J^T or J^T y, so keeping them
    gives the same result.)"""
    if invR is not None:
        raise NotImplementedError("structural priors are outside this engine's scope")
    J, K = _device_rows(Amat)
    out = engine.reginv_under_device(J, K, np.ravel(rhs), lambda_, 1.0, precision)
    return out.cpu().numpy()


def reginvover(Amat, rhs, lambda_, LTL=None, blocks=None, precision="tf32x3", **kwargs):
    """Overdetermined regularised solve (recon.py:363-426):
    dmu = (J^T J + lambda I)^-1 J^T r with unit-diagonal normalisation."""
    if LTL is not None:
        raise NotImplementedError("structural priors are outside this engine's scope")
    A = np.asarray(Amat, dtype=np.float64)
    # J^T r through the same GEMV kernel, then the Gram of J^T
    Jr, Kr = _device_rows(A)
    r = torch.as_tensor(np.ascontiguousarray(np.ravel(rhs), dtype=np.float64), device=Jr.device)
    proj = engine.gemv_t(Jr, Kr, r)
    JT, K = _device_rows(A.T)
    M = JT.shape[0]
    H, lo = engine.gram(JT, K, 1.0, precision)
    dev = JT.device
    di = torch.empty(M, dtype=torch.float64, device=dev)
    engine.call("rb_reginv_prepare", engine.ptr(H), M, M, float(lambda_), engine.ptr(di), engine.stream())
    wb = engine._lib.lib().rb_cholesky_work_bytes()
    work = torch.empty(wb, dtype=torch.uint8, device=dev)
    engine.call("rb_cholesky", engine.ptr(H), M, M, engine.ptr(work), wb, engine.stream())
    t = torch.empty(M, dtype=torch.float64, device=dev)
    engine.call("rb_vec_mul", engine.ptr(di), engine.ptr(proj), engine.ptr(t), M, engine.stream())
    engine.call("rb_chol_solve", engine.ptr(H), M, M, engine.ptr(t), engine.stream())
    x = torch.empty(M, dtype=torch.float64, device=dev)
    engine.call("rb_vec_mul", engine.ptr(di), engine.ptr(t), engine.ptr(x), M, engine.stream())
    return x.cpu().numpy()


def reginv(Amat, rhs, lambda_, Areg=None, blocks=None, **kwargs):
    """Over/under-determined dispatch (recon.py:338-360)."""
    Areg = Areg or {}
    if Amat.shape[0] >= Amat.shape[1]:
        return reginvover(Amat, rhs, lambda_, Areg.get("ltl"), blocks, **kwargs)
    return reginvunder(Amat, rhs, lambda_, Areg.get("lir"), blocks, **kwargs)


def syncprop(cfg, recon):
    """Copy the reconstruction properties to the forward mesh (recon.py:669-781,
    single-mesh case)."""
    if "prop" in recon and not isinstance(recon["prop"], dict):
        cfg["prop"] = recon["prop"].copy()
    return cfg, recon


def _flatten(detphi):
    if isinstance(detphi, dict):
        raise NotImplementedError("multi-wavelength / multi-mode data are outside this engine's scope")
    return np.asarray(detphi).ravel()


# --------------------------------------------------------------- GN driver
def runrecon(cfg, recon, detphi0, sd=None, **kwargs):
    """Gauss-Newton reconstruction (recon.py:39-335) with the forward model,
    Jacobian and normal equations on the GPU.  Returns
    ``(recon, resid, cfg, updates, Jmua, detphi, phi)`` like the reference;
    ``Jmua`` is ``{'mua': J}`` with the final (matreform-stacked) Jacobian,
    as numpy when it is under 2 GB, else as the CUDA tensor."""
    maxiter = kwargs.get("maxiter", 5)
    lambda_ = kwargs.get("lambda_", recon.get("lambda", 0.05))
    report = kwargs.get("report", True)
    tol = kwargs.get("tol", 0)
    reform = kwargs.get("reform", "real")
    solverflag = kwargs.get("solverflag", {}) or {}
    param = kwargs.get("param", "mua")
    jac_mode = kwargs.get("jac_mode", "reference" if param == "mua" else "exact")
    gram_prec = kwargs.get("gram", "tf32")
    lambda_rule = kwargs.get("lambda_rule", "fixed")
    # each forward solve starts from the previous iterate's fields (the
    # refinement then only removes what the property update changed)
    warm_start = kwargs.get("warm_start", True)
    if kwargs.get("prior") or "lmat" in kwargs or "ltl" in kwargs:
        raise NotImplementedError("structural priors are outside this engine's scope")
    if "param" in recon or isinstance(recon.get("prop"), dict) or isinstance(cfg.get("prop"), dict):
        raise NotImplementedError("multi-spectral reconstruction is outside this engine's scope")
    if "node" in recon and "elem" in recon and "mapid" in recon:
        raise NotImplementedError("dual-mesh reconstruction is outside this engine's scope")
    if reform not in ("real", "reim", "complex"):
        raise NotImplementedError(f"reform '{reform}' is not supported by the device GN loop")
    if sd is None:
        sd = sdmap(cfg)
    if recon["prop"].ndim == 1:
        recon["prop"] = recon["prop"].reshape(1, -1)
    nn = cfg["node"].shape[0]
    if recon["prop"].shape[0] != nn:
        raise NotImplementedError("only node-based reconstruction (one prop row per node) is supported")
    params = ("mua",) if param == "mua" else ("mua", "D")
    y0 = _flatten(detphi0)
    resid = np.zeros(maxiter)
    updates = []
    J = det = phi = None
    for it in range(maxiter):
        t0 = time.time()
        cfg, recon = syncprop(cfg, recon)
        det, phi, _, _, _ = forward_device(cfg, x0=phi if (warm_start and phi is not None) else None,
                                           **solverflag)
        mesh = engine.mesh_of(cfg)
        J, K = engine.jacobian_matrix(mesh, phi, sd, params, jac_mode,
                                      dtype=torch.bfloat16 if gram_prec == "bf16" else torch.float32)
        y = det.cpu().numpy().ravel()
        misfit = y0 - y
        if np.iscomplexobj(misfit) or np.iscomplexobj(y0):
            if reform == "complex":
                raise NotImplementedError("complex normal equations: use reform='real'")
            if reform == "reim":
                raise NotImplementedError("reform 'reim' is not supported by the device GN loop")
            misfit = np.concatenate([np.real(misfit), np.imag(misfit)])
        resid[it] = np.sum(np.abs(misfit))
        scale2 = 1.0 / float(engine.sumsq(J, K).item())  # blockscale^2 (recon.py:235-240)
        if lambda_rule == "maxdiag":
            dmu = engine.reginv_under_device(J, K, misfit, 0.0, scale2, gram_prec, lam_rel=lambda_)
        else:
            dmu = engine.reginv_under_device(J, K, misfit, lambda_, scale2, gram_prec)
        dmu = dmu.cpu().numpy()
        upd = {"mua": dmu[:nn]}
        recon["prop"][:, 0] += dmu[:nn]
        if "D" in params:
            # consistent with the forward model's D = 1/(3 (mua + musp))
            p = recon["prop"]
            musp_old = p[:, 1] * (1 - p[:, 2]) if p.shape[1] >= 3 else p[:, 1]
            mua_old = p[:, 0] - dmu[:nn]
            d_new = 1.0 / (3.0 * (mua_old + musp_old)) + dmu[nn:2 * nn]
            musp_new = 1.0 / (3.0 * d_new) - p[:, 0]
            p[:, 1] = musp_new / (1 - p[:, 2]) if p.shape[1] >= 3 else musp_new
            upd["dcoeff"] = dmu[nn:2 * nn]
        updates.append(upd)
        if report:
            rel = resid[it] / resid[0] if it > 0 else 1.0
            print(f"iter [{it + 1:4d}]: residual={resid[it]:.6e}, relres={rel:.6e} lambda={lambda_:.6e} "
                  f"(time={time.time() - t0:.2f} s)")
        if it > 0 and abs(resid[it] - resid[it - 1]) / resid[0] < tol:
            resid = resid[: it + 1]
            break
    recon["lambda"] = lambda_
    Jout = J[:, :K]
    if Jout.numel() * 4 < 2 ** 31:
        Jout = Jout.float().cpu().numpy()
    return recon, resid, cfg, updates, {"mua": Jout}, det.cpu().numpy(), phi.cpu().numpy()

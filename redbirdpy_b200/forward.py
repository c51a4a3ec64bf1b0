"""Forward model API, drop-in for redbirdpy's ``forward`` module
(redbirdpy/forward.py): ``runforward``, ``femlhs``, ``femrhs``, ``femgetdet``
and ``jac`` with the reference signatures and return types, computed on the
GPU by ``librbb200.so``.

Scope: single-wavelength ``cfg['prop']`` arrays (label/seg, per-node or
per-tet rows), point sources and detectors, CW or frequency domain.
Multi-wavelength dicts and wide-field optodes raise NotImplementedError.
"""

import numpy as np
import torch
from scipy import sparse

from . import engine
from .solver import femsolve, solver_options

__all__ = ["runforward", "femlhs", "femrhs", "femgetdet", "jac", "C0", "forward_device"]

C0 = engine.C0


def _wavelengths(cfg):
    """The wavelength keys of per-wavelength properties, or [''] (forward.py:52-54)."""
    prop = cfg.get("prop")
    return list(prop.keys()) if isinstance(prop, dict) else [""]


def forward_device(cfg, mode=1, x0=None, wv="", **kwargs):
    """One forward pass kept on the device: returns (detval, phi, optodes,
    matrix, solve-info) with detval (ndet x nsrc) and phi (nn x (nsrc+ndet))
    as CUDA tensors.  The order matches runforward: femrhs, femlhs, femsolve,
    femgetdet (redbirdpy/forward.py:66-75); ``wv`` selects the wavelength of
    per-wavelength properties."""
    mesh = engine.mesh_of(cfg)
    opt = engine.locate_optodes(mesh, cfg, wv)
    B = opt.rhs(mesh)
    mat = engine.assemble(mesh, engine.Optics.from_cfg(mesh, cfg, mode, wv))
    phi, info = engine.solve(mat, B, x0=x0, **solver_options(kwargs))
    det = engine.getdet(mesh, opt, phi)
    return det, phi, opt, mat, info


def runforward(cfg, **kwargs):
    """Forward simulation for all sources (redbirdpy/forward.py:40-87).

    Returns ``(detval, phi)`` as numpy arrays (Ndet x Nsrc, Nn x Ncol); with
    a list ``rfcw`` of several modes, dicts keyed by mode like the reference."""
    rfcw = kwargs.get("rfcw", [1])
    if isinstance(rfcw, int):
        rfcw = [rfcw]
    if cfg.get("deldotdel") is None:
        cfg["deldotdel"] = engine.mesh_of(cfg).deldotdel_host()
    wavelengths = _wavelengths(cfg)
    det_out = {md: {"detphi": {}} for md in rfcw}
    phi_out = {md: {"phi": {}} for md in rfcw}
    for wv in wavelengths:
        for md in rfcw:
            det, phi, _, _, info = forward_device(cfg, mode=md, wv=wv, **kwargs)
            det_out[md]["detphi"][wv] = det.cpu().numpy()
            phi_out[md]["phi"][wv] = engine.host_pool.to_numpy(phi)
    # the reference's nesting: modes, then wavelengths, each level dropped when single
    if len(wavelengths) == 1:
        for md in rfcw:
            det_out[md]["detphi"] = det_out[md]["detphi"][wavelengths[0]]
            phi_out[md]["phi"] = phi_out[md]["phi"][wavelengths[0]]
    if len(rfcw) == 1:
        return det_out[rfcw[0]]["detphi"], phi_out[rfcw[0]]["phi"]
    return det_out, phi_out


def femlhs(cfg, deldotdel_mat=None, wavelength="", mode=1):
    """FEM system matrix as scipy CSR (redbirdpy/forward.py:90-256).

    Assembled on the GPU from ``deldotdel_mat`` (as the reference does;
    None = the mesh's own, computed on the GPU) and ``cfg['evol']``."""
    mesh = engine.mesh_of(cfg)
    ddd = None
    if deldotdel_mat is not None and deldotdel_mat is not cfg.get("deldotdel"):
        ddd = torch.as_tensor(np.ascontiguousarray(deldotdel_mat, dtype=np.float64), device=mesh.device)
    mat = engine.assemble(mesh, engine.Optics.from_cfg(mesh, cfg, mode, wavelength), ddd=ddd)
    A = mesh.csr_host(mat.val64)
    A.has_sorted_indices = True
    return A


def femrhs(cfg, sd=None, wv="", md=1):
    """Point-optode RHS ``(rhs, loc, bary, optode)`` (redbirdpy/forward.py:259-362):
    rhs is Nn x (Nsrc+Ndet) CSR with 4 barycentric weights per column, loc
    1-based (NaN outside the mesh)."""
    mesh = engine.mesh_of(cfg)
    opt = engine.locate_optodes(mesh, cfg, wv)
    nn = mesh.nn
    if opt.npts == 0:
        return sparse.csr_matrix((nn, 0)), np.array([]), np.array([]).reshape(0, 4), np.array([])
    loc, bary = opt.loc_bary_host()
    B = opt.rhs(mesh)
    rhs = sparse.csr_matrix(B.cpu().numpy())
    return rhs, loc, bary, opt.pts_host


def femgetdet(phi, cfg, rhs, loc=None, bary=None):
    """Detector readout ``rhs_det^T phi_src`` (redbirdpy/forward.py:365-442).

    With ``loc``/``bary`` given (point detectors) the GPU gathers the four
    barycentric weights per detector; otherwise the sparse product of the
    given rhs columns is formed on the GPU by the same kernel after locating
    the detectors again."""
    ns = np.atleast_2d(cfg["srcpos"]).shape[0] if cfg.get("srcpos") is not None and np.size(cfg["srcpos"]) else 0
    nd = np.atleast_2d(cfg["detpos"]).shape[0] if cfg.get("detpos") is not None and np.size(cfg["detpos"]) else 0
    if ns == 0 or nd == 0:
        return np.array([])
    mesh = engine.mesh_of(cfg)
    dev = mesh.device
    if loc is None or bary is None:
        opt = engine.locate_optodes(mesh, cfg)
    else:
        opt = engine.Optodes.__new__(engine.Optodes)
        loc = np.asarray(loc, dtype=np.float64)
        l0 = np.where(np.isnan(loc), -1, loc - 1).astype(np.int32)
        opt.nsrc, opt.ndet, opt.npts = ns, nd, ns + nd
        opt.loc = torch.as_tensor(l0, device=dev)
        opt.bary = torch.as_tensor(np.nan_to_num(np.asarray(bary, dtype=np.float64)), device=dev)
    phi_t = torch.as_tensor(np.ascontiguousarray(phi), device=dev)
    return engine.getdet(mesh, opt, phi_t).cpu().numpy()


def jac(sd, phi, deldotdel_mat, elem, evol, iselem=False):
    """Adjoint mua Jacobian (redbirdpy/forward.py:509-569).

    Returns ``(Jmua_node, Jmua_elem)`` (Nsd x Nn and Nsd x Ne, FP64, complex
    for complex phi).  The node rows come straight from the node-row kernel;
    the element matrix from the element kernel."""
    phi = np.ascontiguousarray(phi)
    mesh = engine.topology_of(elem, phi.shape[0])
    dev = mesh.device
    ev = torch.as_tensor(np.ascontiguousarray(evol, dtype=np.float64), device=dev)
    phi_t = torch.as_tensor(phi, device=dev)
    jn = engine.jacobian(mesh, phi_t, sd, "mua", out_dtype=torch.float64, evol=ev)
    je = engine.jacobian_elem(mesh, phi_t, sd, evol=ev)
    return jn.cpu().numpy(), je.cpu().numpy()

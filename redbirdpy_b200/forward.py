"""Forward model API, drop-in for redbirdpy's ``forward`` module
(redbirdpy/forward.py): ``runforward``, ``femlhs``, ``femrhs``, ``femgetdet``
and ``jac`` with the reference signatures and return types, computed on the
GPU by ``librbb200.so``.

Scope: ``cfg['prop']`` arrays (label/seg, per-node or per-tet rows) or
per-wavelength dicts of them, point and wide-field (``cfg['widesrc']`` /
``cfg['widedet']`` pattern columns) sources and detectors, CW or frequency
domain.
"""

import numpy as np
import torch
from scipy import sparse

from . import engine
from .solver import femsolve, solver_options

__all__ = ["runforward", "femlhs", "femrhs", "femgetdet", "jac", "jacchrome", "C0", "forward_device"]

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
    """RHS ``(rhs, loc, bary, optode)`` (redbirdpy/forward.py:259-362): rhs is
    Nn x Ncol CSR in the column order [point src | wide src | point det |
    wide det] -- 4 barycentric weights per point column, the pattern's
    nonzeros per wide-field column; loc 1-based (NaN outside the mesh and for
    wide-field columns), bary NaN rows for wide-field columns."""
    mesh = engine.mesh_of(cfg)
    opt = engine.locate_optodes(mesh, cfg, wv)
    nn = mesh.nn
    if opt.ncol == 0:
        return sparse.csr_matrix((nn, 0)), np.array([]), np.array([]).reshape(0, 4), np.array([])
    loc, bary = opt.loc_bary_host()
    # point columns straight from (loc, bary): the 4 weights of each located
    # optode at its tet's nodes, zero weights dropped (as the reference's
    # sparse column writes leave them out); wide columns from the patterns
    inside = ~np.isnan(loc)
    cols = np.repeat(np.nonzero(inside)[0], 4)
    tets = loc[inside].astype(np.int64) - 1
    rows = np.asarray(cfg["elem"])[tets, :4].astype(np.int64).ravel() - 1
    vals = bary[inside].ravel()
    keep = vals != 0
    R, C, V = [rows[keep]], [cols[keep]], [vals[keep]]
    for w, c0 in ((cfg.get("widesrc"), opt.npsrc), (cfg.get("widedet"), opt.nsrc + opt.npdet)):
        if w is not None and np.size(w):
            w = np.asarray(w, dtype=np.float64).reshape(nn, -1)
            r, c = np.nonzero(w)
            R.append(r), C.append(c + c0), V.append(w[r, c])
    rhs = sparse.csr_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(C))), shape=(nn, opt.ncol))
    return rhs, loc, bary, opt.pts_host


def femgetdet(phi, cfg, rhs, loc=None, bary=None):
    """Detector readout ``rhs_det^T phi_src`` (redbirdpy/forward.py:365-442),
    (point + wide detectors) x (point + wide sources).

    With ``loc``/``bary`` given (femrhs's outputs) the GPU gathers the four
    barycentric weights per point detector; otherwise the detectors are
    located again.  Wide-field detector rows come from cfg['widedet']."""
    ns = np.atleast_2d(cfg["srcpos"]).shape[0] if cfg.get("srcpos") is not None and np.size(cfg["srcpos"]) else 0
    nd = np.atleast_2d(cfg["detpos"]).shape[0] if cfg.get("detpos") is not None and np.size(cfg["detpos"]) else 0
    wsrc, wdet = cfg.get("widesrc"), cfg.get("widedet")
    ws = np.asarray(wsrc).reshape(np.shape(wsrc)[0], -1).shape[1] if wsrc is not None and np.size(wsrc) else 0
    wd = np.asarray(wdet).reshape(np.shape(wdet)[0], -1).shape[1] if wdet is not None and np.size(wdet) else 0
    if ns + ws == 0 or nd + wd == 0:
        return np.array([])
    mesh = engine.mesh_of(cfg)
    dev = mesh.device
    if loc is None or bary is None:
        opt = engine.locate_optodes(mesh, cfg)
    else:
        loc = np.asarray(loc, dtype=np.float64).ravel()
        bary = np.asarray(bary, dtype=np.float64).reshape(-1, 4)
        if ws or wd:  # entries in femrhs's column order: keep the point ones
            idx = np.r_[np.arange(ns), ns + ws + np.arange(nd)]
            loc, bary = loc[idx], bary[idx]
        opt = engine.Optodes.__new__(engine.Optodes)
        l0 = np.where(np.isnan(loc), -1, loc - 1).astype(np.int32)
        opt.npsrc, opt.npdet, opt.npts = ns, nd, ns + nd
        opt.loc = torch.as_tensor(l0, device=dev)
        opt.bary = torch.as_tensor(np.nan_to_num(bary), device=dev)
        opt.wsrc = engine.Optodes._patterns(mesh, wsrc)
        opt.wdet = engine.Optodes._patterns(mesh, wdet)
        opt.nwsrc, opt.nwdet = ws, wd
        opt.nsrc, opt.ndet, opt.ncol = ns + ws, nd + wd, ns + ws + nd + wd
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


def jacchrome(Jmua, chromophores, extin=None):
    """Chromophore Jacobians from per-wavelength mua Jacobians
    (redbirdpy/forward.py:572-589): for each chromophore, the wavelengths'
    blocks Jmua[wv] * extin(wv, ch) stacked in wavelength order.  ``extin``
    (Nwv x Nchrome, or see property.extinction) is taken from redbirdpy's
    spectra when not given.  Works on numpy arrays or device tensors."""
    from .property import extinction

    if not isinstance(Jmua, dict):
        raise ValueError("Jmua must be a dict with wavelength keys")
    wavelengths = list(Jmua.keys())
    ext, _ = extinction(wavelengths, chromophores, extin)
    out = {}
    for i, ch in enumerate(chromophores):
        blocks = [Jmua[wv] * ext[j, i] for j, wv in enumerate(wavelengths)]
        out[ch] = torch.cat(blocks, 0) if torch.is_tensor(blocks[0]) else np.vstack(blocks)
    return out

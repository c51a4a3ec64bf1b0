"""Gauss-Newton reconstruction API, drop-in for redbirdpy's ``recon`` module
(redbirdpy/recon.py): ``runrecon``, ``reginv``, ``reginvunder``,
``reginvover``, ``matreform``, ``matflat``, ``syncprop``.

The device loop keeps the mesh, fields and Jacobian on the GPU: forward
solve -> Jacobian rows (``rb_jac``) -> Frobenius scaling (``rb_sumsq``) ->
``J J^T`` on the tensor cores (``rb_gram``) -> FP64 Cholesky -> ``J^T y``.
Only detector values, misfits and the update vector cross to the host.

Scope: node-based reconstruction on the forward mesh or on a separate
reconstruction mesh (dual mesh), one wavelength or several with chromophore
parameters, reform 'real' / 'reim' / 'logphase'.  Label-based
reconstruction and structural priors raise NotImplementedError.  Additive
options (not in the reference): ``param='mua'`` (default, the reference's
update) or ``'mua+D'`` (node-wise mua and diffusion coefficient with exact
Jacobians); ``jac_mode`` ('reference' | 'exact'); ``gram`` ('tf32' |
'tf32x3' | 'bf16'); ``refine`` (FP64 refinement sweeps of the normal
equations, default 3); ``lambda_rule`` ('fixed', the reference's, or
'maxdiag': lambda_ * max diag(J J^T)); ``extin`` (extinction coefficients
{wavelength: {chromophore: value}}, needed when redbirdpy's spectra are not
installed).
"""

import time

import numpy as np
import torch

from . import engine
from .forward import forward_device
from .utility import sdmap

__all__ = ["runrecon", "reginv", "reginvover", "reginvunder", "matreform", "matflat", "syncprop", "meshinterp"]


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
    J = torch.empty((M, ld), dtype=torch.float32, device=engine._dev())
    J[:, :K] = torch.as_tensor(np.ascontiguousarray(A, dtype=np.float32), device=J.device)
    if ld > K:
        J[:, K:].zero_()
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
    H, di, lo, lam = engine.normal_factor(JT, K, float(lambda_), 1.0, precision)
    x = engine.normal_solve(JT, K, H, di, proj, lam, 1.0, lo, return_y=True)
    return x.cpu().numpy()


def reginv(Amat, rhs, lambda_, Areg=None, blocks=None, **kwargs):
    """Over/under-determined dispatch (recon.py:338-360)."""
    Areg = Areg or {}
    if Amat.shape[0] >= Amat.shape[1]:
        return reginvover(Amat, rhs, lambda_, Areg.get("ltl"), blocks, **kwargs)
    return reginvunder(Amat, rhs, lambda_, Areg.get("lir"), blocks, **kwargs)


LABEL_ROWS = 50  # fewer property rows than this: label-based (recon.py:103-112, 697)


def meshinterp(fromval, elemid, elembary, fromelem, toval=None):
    """Interpolate nodal values between meshes (utility.py:973-999): the
    value at each target point is the barycentric mix of the four nodes of
    its enclosing source element (elemid 1-based, NaN outside: left as toval
    or 0)."""
    fromval = np.asarray(fromval, dtype=np.float64)
    col = fromval.ndim == 1
    fv = fromval[:, None] if col else fromval
    elemid = np.asarray(elemid, dtype=np.float64).ravel()
    out = np.zeros((elemid.size, fv.shape[1])) if toval is None else \
        (np.array(toval, dtype=np.float64).reshape(elemid.size, -1).copy())
    ok = ~np.isnan(elemid)
    e0 = np.asarray(fromelem)[:, :4].astype(np.int64) - 1
    nodes = e0[elemid[ok].astype(np.int64) - 1]
    w = np.asarray(elembary, dtype=np.float64).reshape(-1, 4)[ok]
    out[ok] = np.einsum("pj,pjc->pc", w, fv[nodes])
    return out[:, 0] if out.shape[1] == 1 else out


def syncprop(cfg, recon):
    """Copy (single mesh) or interpolate (dual mesh: recon['mapid'] /
    recon['mapweight'], the recon element holding each forward node) the
    reconstruction's 'param' or 'prop' onto the forward mesh
    (recon.py:669-781)."""
    dual = "mapid" in recon and "mapweight" in recon and "elem" in recon

    def move(v):
        if dual:
            return meshinterp(v, recon["mapid"], recon["mapweight"], recon["elem"])
        return v.copy() if hasattr(v, "copy") else v

    if "param" in recon:
        keys = list(recon["param"].keys())
        first = recon["param"][keys[0]]
        if (len(first) if hasattr(first, "__len__") else 1) < LABEL_ROWS:
            cfg["param"] = {k: v.copy() if hasattr(v, "copy") else v for k, v in recon["param"].items()}
        else:
            cfg.setdefault("param", {})
            for k in keys:
                cfg["param"][k] = move(recon["param"][k])
    elif "prop" in recon:
        if not isinstance(recon["prop"], dict):
            p = recon["prop"]
            cfg["prop"] = p.copy() if p.shape[0] < LABEL_ROWS else move(p)
        else:
            first = next(iter(recon["prop"].values()))
            cfg["prop"] = {k: (v.copy() if first.shape[0] < LABEL_ROWS else move(v))
                           for k, v in recon["prop"].items()}
    return cfg, recon


def _flatten(detphi, wavelengths):
    """Measurements of all wavelengths as one vector, wavelength by
    wavelength, each detector-major (_flatten_detphi, recon.py:792-815)."""
    if not isinstance(detphi, dict):
        return np.asarray(detphi).ravel()
    out = []
    for wv in wavelengths:
        v = detphi.get(wv, detphi) if isinstance(detphi, dict) else detphi
        if isinstance(v, dict):
            raise NotImplementedError("multi-mode (rfcw) measurements are outside this engine's scope")
        out.append(np.asarray(v).ravel())
    return np.concatenate(out)


class RemapOp:
    """Dual-mesh maps on the device: the forward mesh's nodes inside the
    reconstruction mesh's elements (recon['mapid'], 1-based, NaN outside;
    recon['mapweight'] their barycentric weights), turned into a list per
    reconstruction node of (forward node, weight) in ascending forward-node
    order for rb_jac_remap (_remap_jacobian, recon.py:818-876)."""

    def __init__(self, recon, nn_fwd, device):
        mapid = np.asarray(recon["mapid"], dtype=np.float64).ravel()
        w = np.asarray(recon["mapweight"], dtype=np.float64).reshape(-1, 4)
        relem = np.asarray(recon["elem"])[:, :4].astype(np.int64) - 1
        self.nq = int(recon["node"].shape[0])
        if mapid.size != nn_fwd:
            raise ValueError("recon['mapid'] needs one entry per forward-mesh node")
        ok = ~np.isnan(mapid)
        eid = np.where(ok, np.nan_to_num(mapid), 1).astype(np.int64) - 1
        ok &= (eid >= 0) & (eid < relem.shape[0])
        fi = np.repeat(np.nonzero(ok)[0], 4)
        q = relem[eid[ok]].ravel()
        ww = w[ok].ravel()
        good = (q >= 0) & (q < self.nq)
        fi, q, ww = fi[good], q[good], ww[good]
        order = np.lexsort((fi, q))
        counts = np.bincount(q, minlength=self.nq)
        self.ptr = torch.as_tensor(np.concatenate([[0], np.cumsum(counts)]).astype(np.int32), device=device)
        self.idx = torch.as_tensor(fi[order].astype(np.int32), device=device)
        self.w = torch.as_tensor(ww[order], device=device)

    def apply(self, J):
        kind = {torch.float32: engine._lib.RB_F32, torch.complex64: engine._lib.RB_C64,
                torch.float64: engine._lib.RB_F64, torch.complex128: engine._lib.RB_C128}[J.dtype]
        out = torch.empty((J.shape[0], self.nq), dtype=J.dtype, device=J.device)
        engine.call("rb_jac_remap", engine.ptr(J), kind, J.shape[0], J.shape[1], engine.ptr(self.ptr),
                    engine.ptr(self.idx), engine.ptr(self.w), self.nq, engine.ptr(out), self.nq, engine.stream())
        return out


def _stacked_matrix(mesh, phis, sds, dets, y0s, wavelengths, weights, nq, remap, reform):
    """The real GN matrix and right-hand side of the general path: per
    wavelength the reference-semantics mua Jacobian rows (rb_jac, FP32 /
    complex64), remapped to the reconstruction mesh (dual mesh), written as
    len(weights[wv]) column blocks of nq columns each scaled by its weight
    (the chromophores' extinction, jacchrome), rows wavelength by wavelength
    and then, for complex data, the imaginary parts below the real ones
    (matreform 'real'); 'reim' doubles the columns ([[Re, -Im], [Im, Re]]),
    'logphase' scales each row by conj(y)/|y|^2 and takes log-amplitude and
    phase differences (recon.py:512-567).  Returns (J, K, rhs)."""
    cplx = any(torch.is_complex(p) for p in phis)
    nrows = [int(np.asarray(sd_).shape[0]) for sd_ in sds]
    R = sum(nrows)
    nb = len(weights[wavelengths[0]])
    K = nb * nq * (2 if (reform == "reim" and cplx) else 1)
    rows_total = 2 * R if cplx else R
    # every (row, column < K) is written by the blocks below; the padding
    # columns are cleared
    J = torch.empty((rows_total, engine._pad4(K)), dtype=torch.float32, device=mesh.device)
    if J.shape[1] > K:
        J[:, K:].zero_()
    rhs = []
    r0 = 0
    for j, wv in enumerate(wavelengths):
        Jw = engine.jacobian(mesh, phis[j], sds[j], "mua", out_dtype=torch.complex64 if cplx else torch.float32)
        if remap is not None:
            Jw = remap.apply(Jw)
        kind = engine._lib.RB_C64 if cplx else engine._lib.RB_F32
        ym = dets[j].cpu().numpy().ravel()
        y0 = y0s[j]
        rs = None
        if reform == "logphase":
            g = np.conj(ym) / np.abs(ym * ym)
            rs = torch.as_tensor(np.column_stack([np.real(g), np.imag(g)]).ravel().astype(np.float64),
                                 device=mesh.device)
        row_im = R + r0 if cplx else -1
        for b in range(nb):
            f = float(weights[wv][b])
            engine.call("rb_jac_block", engine.ptr(Jw), kind, Jw.shape[0], nq, Jw.shape[1], f, 0.0, engine.ptr(rs),
                        engine.ptr(J), J.shape[1], r0, row_im, b * nq, engine.stream())
            if reform == "reim" and cplx:  # second column half: i * block
                engine.call("rb_jac_block", engine.ptr(Jw), kind, Jw.shape[0], nq, Jw.shape[1], 0.0, f, None,
                            engine.ptr(J), J.shape[1], r0, row_im, nb * nq + b * nq, engine.stream())
        if reform == "logphase":
            rhs.append((np.log(np.abs(y0)) - np.log(np.abs(ym)), np.angle(y0) - np.angle(ym)))
        else:
            d = y0 - ym
            rhs.append((np.real(d), np.imag(d)))
        r0 += nrows[j]
    r = np.concatenate([a for a, _ in rhs])
    if cplx:
        r = np.concatenate([r, np.concatenate([b for _, b in rhs])])
    return J, K, r


def _apply_prop(recon, key, dx):
    """Add an update block to recon['prop'] (recon.py:262-293): 'mua' to
    column 0; 'dcoeff' through column 1 as 1/(3 (1/(3 mus) + dx)); node-based
    (or label-based when the table has few rows) rows."""
    prop = recon["prop"]
    col = 0 if key == "mua" else 1
    if prop.shape[0] < len(dx) and prop.shape[0] < LABEL_ROWS:
        n = min(prop.shape[0], len(dx))
        if key == "dcoeff":
            prop[:n, col] = 1.0 / (3 * (1.0 / (3 * prop[:n, col]) + dx[:n]))
        else:
            prop[:n, col] += dx[:n]
    elif key == "dcoeff":
        prop[:, col] = 1.0 / (3 * (1.0 / (3 * prop[:, col]) + dx))
    else:
        prop[:, col] += dx


def _apply_param(cfg, recon, key, dx):
    """Add an update block to a chromophore / scattering parameter
    (recon.py:295-327): in recon['param'] when it holds the key, else in
    cfg['param']; a scalar or short (label) parameter takes the first
    entries of the block."""
    if "param" in recon and key in recon["param"]:
        target = recon
    elif "param" in cfg and key in cfg["param"]:
        target = cfg
    else:
        return
    val = target["param"][key]
    n = len(val) if hasattr(val, "__len__") else 1
    if n < len(dx) and n < LABEL_ROWS:
        if n == 1:
            if hasattr(val, "__len__"):
                target["param"][key][0] += dx[0]
            else:
                target["param"][key] = val + dx[0]
        else:
            for li in range(min(n, len(dx))):
                target["param"][key][li] += dx[li]
    else:
        target["param"][key] = val + dx


# --------------------------------------------------------------- GN driver
def _slab_width(jac_slab, mesh, phi, sd, nparams, dtype):
    """Node slab width of a recomputed Jacobian, or 0 to store it whole."""
    if jac_slab is None or jac_slab is False:
        return 0
    if not isinstance(jac_slab, str):
        return int(jac_slab)
    rows = int(np.count_nonzero(np.asarray(sd)[:, 2] == 1)) if np.asarray(sd).shape[1] >= 3 else len(sd)
    rows *= 2 if phi.is_complex() else 1
    esz = 2 if dtype == torch.bfloat16 else 4
    full = rows * (nparams * mesh.nn + 8) * esz
    free = torch.cuda.mem_get_info(phi.device)[0]
    if full <= 0.5 * free:
        return 0
    # slabs of a quarter of the free memory (the gram's staging copy and
    # the split remainder of tf32x3 come on top of the slab itself)
    return max(1024, int(0.25 * free / (rows * nparams * esz)))


def runrecon(cfg, recon, detphi0, sd=None, **kwargs):
    """Gauss-Newton reconstruction (recon.py:39-335) with the forward model,
    Jacobian and normal equations on the GPU.  Returns
    ``(recon, resid, cfg, updates, Jmua, detphi, phi)`` like the reference;
    ``Jmua`` holds the final GN matrix (matreform-stacked) under 'mua' (or
    the block keys), as numpy when it is under 2 GB, else as the CUDA tensor.

    Covered: one or several wavelengths (``cfg['prop']`` keyed by
    wavelength) with chromophore parameters (``cfg['param']`` /
    ``recon['param']``: the Jacobian blocks of jacchrome, extinction
    coefficients from ``extin=`` / ``cfg['extin']`` or redbirdpy's spectra),
    one mesh or a separate reconstruction mesh (``recon['node']``,
    ``recon['elem']``, ``recon['mapid']``, ``recon['mapweight']``),
    reform 'real', 'reim' or 'logphase'.  On one mesh and wavelength with
    reform 'real', a Jacobian larger than half the free HBM is not stored:
    ``jac_slab`` (default 'auto'; an int sets the node slab width) makes
    every pass over J recompute it slab by slab from the stored fields, and
    the returned 'mua' entry is then that operator.  Structural priors raise
    NotImplementedError."""
    from .forward import jacchrome  # noqa: F401  (the same weights, as numpy / tensors)
    from .property import CHROMOPHORES, extinction, updateprop

    maxiter = kwargs.get("maxiter", 5)
    lambda_ = kwargs.get("lambda_", recon.get("lambda", 0.05))
    report = kwargs.get("report", True)
    tol = kwargs.get("tol", 0)
    reform = kwargs.get("reform", "real")
    solverflag = kwargs.get("solverflag", {}) or {}
    param = kwargs.get("param", "mua")
    jac_mode = kwargs.get("jac_mode", "reference" if param == "mua" else "exact")
    # J J^T on the tensor cores from a BF16 copy of the FP32 rows (twice the
    # TF32 rate); the FP64 refinement over the FP32 rows makes the update the
    # FP32 rows' solution whatever the product's precision
    gram_prec = kwargs.get("gram", "bf16")
    lambda_rule = kwargs.get("lambda_rule", "fixed")
    refine = kwargs.get("refine", 3)
    # Jacobian storage: 'auto' stores J when it fits in half the free HBM and
    # otherwise recomputes it in node slabs; an int forces slabs that wide;
    # None/False always stores it
    jac_slab = kwargs.get("jac_slab", "auto")
    # FP32 Jacobian rows whose products are formed in FP64: the update then
    # carries only the rows' storage rounding
    jac_acc64 = kwargs.get("jac_acc64", True)
    extin = kwargs.get("extin", cfg.get("extin"))
    # each forward solve starts from the previous iterate's fields (the
    # refinement then only removes what the property update changed)
    warm_start = kwargs.get("warm_start", True)
    if kwargs.get("prior") or "lmat" in kwargs or "ltl" in kwargs:
        raise NotImplementedError("structural priors are outside this engine's scope")
    if reform not in ("real", "reim", "logphase", "complex"):
        raise ValueError(f"Unknown form: {reform}")
    if reform == "complex":
        raise NotImplementedError("complex normal equations: use reform='real'")
    if sd is None:
        sd = sdmap(cfg)
    if "prop" in recon and isinstance(recon["prop"], np.ndarray) and recon["prop"].ndim == 1:
        recon["prop"] = recon["prop"].reshape(1, -1)
    dual = "node" in recon and "elem" in recon and "mapid" in recon
    chrom_mode = ("param" in cfg or "param" in recon) and (
        isinstance(cfg.get("prop"), dict) or isinstance(recon.get("prop"), dict))
    if not chrom_mode and (isinstance(cfg.get("prop"), dict) or isinstance(recon.get("prop"), dict)):
        raise NotImplementedError("multi-wavelength reconstruction needs chromophore parameters ('param'): "
                                  "per-wavelength mua blocks do not form one system with the stacked data")
    if not chrom_mode and "prop" in recon and recon["prop"].shape[0] < LABEL_ROWS:
        raise NotImplementedError("label-based reconstruction is outside this engine's scope")
    fast = not (dual or chrom_mode or reform != "real")
    if not fast and param != "mua":
        raise NotImplementedError("param='mua+D' is available on one mesh, one wavelength, reform 'real'")
    mesh = engine.mesh_of(cfg)
    remap = RemapOp(recon, mesh.nn, mesh.device) if dual else None
    nq = remap.nq if dual else mesh.nn
    resid = np.zeros(maxiter)
    updates = []
    J = None
    prev_phi = {}
    dets = phis = None
    wavelengths = [""]
    for it in range(maxiter):
        t0 = time.time()
        if "param" in recon or "prop" in recon:
            cfg, recon = syncprop(cfg, recon)
        if chrom_mode and "param" in cfg:
            newprop = updateprop(cfg, extin=extin)
            cfg["prop"] = newprop if isinstance(newprop, dict) else {list(cfg["prop"].keys())[0]: newprop}
        wavelengths = list(cfg["prop"].keys()) if isinstance(cfg.get("prop"), dict) else [""]
        dets, phis = [], []
        for wv in wavelengths:
            x0 = prev_phi.get(wv) if warm_start else None
            det, phi, _, _, _ = forward_device(cfg, x0=x0, wv=wv, **solverflag)
            prev_phi[wv] = phi
            dets.append(det)
            phis.append(phi)
        y0s = [_flatten(detphi0.get(wv, detphi0) if isinstance(detphi0, dict) else detphi0, [wv])
               if len(wavelengths) > 1 else _flatten(detphi0, wavelengths) for wv in wavelengths]
        sds = [sd.get(wv, sd) if isinstance(sd, dict) else sd for wv in wavelengths]
        if fast:
            params = ("mua",) if param == "mua" else ("mua", "D")
            # 'bf16': FP32 rows, a BF16 copy for the product (the refinement
            # runs over the FP32 rows); 'bf16_rows': the rows themselves in
            # BF16 (half the memory; the step solves the rounded rows' system)
            jdt = torch.bfloat16 if gram_prec == "bf16_rows" else torch.float32
            width = _slab_width(jac_slab, mesh, phis[0], sds[0], len(params), jdt)
            acc64 = jdt == torch.float32 and jac_acc64
            if width:  # J recomputed in node slabs on every pass instead of stored
                J = engine.SlabJacobian(mesh, phis[0], sds[0], params, jac_mode, width, jdt, acc64=acc64)
                K = J.K
            else:
                J, K = engine.jacobian_matrix(mesh, phis[0], sds[0], params, jac_mode, dtype=jdt, acc64=acc64)
            misfit = y0s[0] - dets[0].cpu().numpy().ravel()
            if np.iscomplexobj(misfit):
                misfit = np.concatenate([np.real(misfit), np.imag(misfit)])
            keys = ["mua"] if param == "mua" else ["mua", "dcoeff"]
        else:
            if chrom_mode:
                keys = [k for k in cfg["param"].keys() if k in CHROMOPHORES]
                given = None if extin is None else np.array([[extin[wv][k] for k in keys] for wv in wavelengths])
                ext, _ = extinction(wavelengths, keys, given)
                weights = {wv: ext[j] for j, wv in enumerate(wavelengths)}
            else:
                keys = ["mua"]
                weights = {wv: np.ones(1) for wv in wavelengths}
            J, K, misfit = _stacked_matrix(mesh, phis, sds, dets, y0s, wavelengths, weights, nq, remap, reform)
        resid[it] = np.sum(np.abs(misfit))
        slabs = isinstance(J, engine.SlabJacobian)
        # row sums of squares: the Frobenius block scale and the exact
        # diagonal of J J^T in one pass
        Jb = None
        if slabs:
            rowsq, ssq = J.row_sumsq()
        elif gram_prec == "bf16" and J.dtype == torch.float32:
            rowsq, ssq, Jb = engine.row_sumsq(J, K, bf16_copy=True)
        else:
            rowsq, ssq = engine.row_sumsq(J, K)
        gprec = "bf16" if gram_prec == "bf16_rows" else gram_prec
        scale2 = 1.0 / float(ssq.item())  # blockscale^2 (recon.py:235-240)
        if slabs and J.rows >= K:
            raise NotImplementedError("an overdetermined system is solved on the host path: it needs J stored")
        if not slabs and J.shape[0] >= K:  # overdetermined: (J^T J + lambda I)^-1 J^T r on the host-side path
            Js = J[:, :K].float().cpu().numpy().astype(np.float64) * np.sqrt(scale2)
            dmu = reginvover(Js, misfit, lambda_) * np.sqrt(scale2)
        else:
            rinfo = {}
            if lambda_rule == "maxdiag":
                dmu = engine.reginv_under_device(J, K, misfit, 0.0, scale2, gprec, lam_rel=lambda_,
                                                 refine=refine, info=rinfo, rowsq=rowsq, Jb=Jb)
            else:
                dmu = engine.reginv_under_device(J, K, misfit, lambda_, scale2, gprec, refine=refine,
                                                 info=rinfo, rowsq=rowsq, Jb=Jb)
            del Jb
            dmu = dmu.cpu().numpy()
        upd = {}
        for b, key in enumerate(keys):
            dx = dmu[b * nq:(b + 1) * nq]
            upd[key] = dx
            if key in ("mua", "dcoeff") and "prop" in recon and isinstance(recon["prop"], np.ndarray):
                if key == "dcoeff" and fast:
                    # consistent with the forward model's D = 1/(3 (mua + musp))
                    p = recon["prop"]
                    musp_old = p[:, 1] * (1 - p[:, 2]) if p.shape[1] >= 3 else p[:, 1]
                    mua_old = p[:, 0] - upd["mua"]
                    d_new = 1.0 / (3.0 * (mua_old + musp_old)) + dx
                    musp_new = 1.0 / (3.0 * d_new) - p[:, 0]
                    p[:, 1] = musp_new / (1 - p[:, 2]) if p.shape[1] >= 3 else musp_new
                else:
                    _apply_prop(recon, key, dx)
            elif key in CHROMOPHORES or key in ("scatamp", "scatpow"):
                _apply_param(cfg, recon, key, dx)
        updates.append(upd)
        if report:
            rel = resid[it] / resid[0] if it > 0 else 1.0
            print(f"iter [{it + 1:4d}]: residual={resid[it]:.6e}, relres={rel:.6e} lambda={lambda_:.6e} "
                  f"(time={time.time() - t0:.2f} s)")
        if it > 0 and abs(resid[it] - resid[it - 1]) / resid[0] < tol:
            resid = resid[: it + 1]
            break
    recon["lambda"] = lambda_
    if isinstance(J, engine.SlabJacobian):
        Jout = J  # never stored whole: the operator that recomputes its slabs
    else:
        Jout = J[:, :K]
        if Jout.numel() * 4 < 2 ** 31:
            Jout = Jout.float().cpu().numpy()
    if len(wavelengths) == 1:
        det_out, phi_out = dets[0].cpu().numpy(), phis[0].cpu().numpy()
    else:
        det_out = {wv: d.cpu().numpy() for wv, d in zip(wavelengths, dets)}
        phi_out = {wv: p.cpu().numpy() for wv, p in zip(wavelengths, phis)}
    return recon, resid, cfg, updates, {"mua": Jout}, det_out, phi_out

"""ORACLE / TEST INFRASTRUCTURE ONLY - never imported by the product path.

A plain numpy/scipy restatement of redbirdpy 0.2.0's FEM hot path, written
from the reference's algorithm (cited per function as
``redbirdpy/<file>.py:<lines>``).  It covers the single-wavelength,
point-optode case that the workloads use:

* mesh preparation fallbacks (reorientation, boundary faces, volumes, reff),
* ``deldotdel``, ``femlhs``, ``femrhs``, ``femgetdet``, ``runforward``,
* ``femsolve`` through SuperLU (the reference's ``method='auto'`` choice with
  no optional solver installed) and per-column scipy CG (``method='cg'``),
* ``jac`` (the numpy branch, so complex fields keep their dtype),
* ``matreform``, ``reginv``/``reginvunder``/``reginvover`` and the
  Gauss-Newton loop of ``runrecon`` for node-based ``mua`` updates.

Pinned against fixtures made by running the reference itself
(``tests/golden/make_golden.py``; checked in ``tests/test_oracle.py``).
"""

import numpy as np
from scipy import sparse
from scipy.sparse import linalg as spla

from .tsearch import tsearchn

C0 = 299792458000.0  # mm/s, redbirdpy/forward.py:36


# --------------------------------------------------------------- mesh prep
def reorient(node, elem):
    """Swap nodes 0 and 1 of negatively oriented tets (utility.py:1047-1063)."""
    elem = np.array(elem, copy=True)
    e0 = elem[:, :4].astype(np.int64) - 1
    x = node[e0]
    vol = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    neg = vol < 0
    elem[neg, 0], elem[neg, 1] = elem[neg, 1].copy(), elem[neg, 0].copy()
    return elem


def volface(elem):
    """Boundary triangles in np.unique(axis=0) order (utility.py:1066-1087)."""
    e0 = elem[:, :4].astype(np.int64) - 1
    faces = np.vstack([e0[:, [0, 2, 1]], e0[:, [0, 1, 3]], e0[:, [0, 3, 2]], e0[:, [1, 2, 3]]])
    srt = np.sort(faces, axis=1)
    # row-wise unique through one lexicographic int64 key per sorted triple
    nn = int(srt.max()) + 1 if srt.size else 1
    key = (srt[:, 0] * nn + srt[:, 1]) * nn + srt[:, 2]
    _, first, counts = np.unique(key, return_index=True, return_counts=True)
    return faces[first[counts == 1]] + 1


def elemvolume(node, elem):
    """|signed volume| of tets, area of triangles (utility.py:1090-1109)."""
    e0 = elem.astype(np.int64) - 1
    if e0.shape[1] >= 4:
        x0 = node[e0[:, 0]]
        return np.abs(np.sum(np.cross(node[e0[:, 1]] - x0, node[e0[:, 2]] - x0) * (node[e0[:, 3]] - x0), axis=1)) / 6.0
    v = np.cross(node[e0[:, 1]] - node[e0[:, 0]], node[e0[:, 2]] - node[e0[:, 0]])
    return 0.5 * np.sqrt(np.sum(v * v, axis=1))


def getreff(n_in, n_out=1.0):
    """Haskell effective reflection coefficient (utility.py:879-904)."""
    if n_in <= n_out:
        return 0.0
    oc = np.arcsin(n_out / n_in)
    step = np.pi / 2000
    o = np.arange(0, oc, step)
    cosop = np.sqrt(1 - (n_in * np.sin(o)) ** 2)
    coso = np.cos(o)
    r = 0.5 * ((n_in * cosop - n_out * coso) / (n_in * cosop + n_out * coso)) ** 2
    r += 0.5 * ((n_in * coso - n_out * cosop) / (n_in * coso + n_out * cosop)) ** 2
    of = np.arange(0, np.pi / 2, step)
    rf = np.ones(len(of))
    rf[: len(r)] = r
    cf = np.cos(of)
    rphi = 2 * np.sum(np.sin(of) * cf * rf) * step
    rj = 3 * np.sum(np.sin(of) * cf ** 2 * rf) * step
    return (rphi + rj) / (2 - rphi + rj)


def getbulk(cfg):
    """Bulk optical properties (property.py:216-332), array-prop cases."""
    default = np.array([0.0, 0.0, 0.0, 1.37])
    prop = cfg.get("prop")
    if prop is None:
        return default
    nn, ne = cfg["node"].shape[0], cfg["elem"].shape[0]
    if prop.shape[0] < min(nn, ne):
        seg = cfg.get("seg")
        if seg is None:
            return prop[1] if prop.shape[0] > 1 else default
        if "face" in cfg and len(seg) == nn:
            label = seg[cfg["face"][0, 0] - 1]
        elif "face" in cfg and len(seg) == ne:
            e0 = cfg["elem"][:, :4].astype(np.int64) - 1
            eid = np.where(np.any(e0 == cfg["face"][0, 0] - 1, axis=1))[0]
            label = seg[eid[0]] if len(eid) else 0
        else:
            label = seg[0]
        label = int(label)
        return prop[label] if prop.shape[0] > label else (prop[1] if prop.shape[0] > 1 else default)
    if prop.shape[0] == nn:
        return prop[cfg["face"][0, 0] - 1] if "face" in cfg else prop[0]
    if prop.shape[0] == ne:
        if "face" in cfg:
            e0 = cfg["elem"][:, :4].astype(np.int64) - 1
            eid = np.where(np.any(e0 == cfg["face"][0, 0] - 1, axis=1))[0]
            if len(eid):
                return prop[eid[0]]
        return prop[0]
    return default


def _nwide(cfg, key):
    w = cfg.get(key)
    return np.asarray(w).reshape(np.shape(w)[0], -1).shape[1] if w is not None and np.size(w) else 0


def sdmap(cfg):
    """Single-wavelength source/detector pair table (utility.py:675-796):
    columns [point src | wide src | point det | wide det], detector-major."""
    ns = np.atleast_2d(cfg["srcpos"]).shape[0]
    nd = np.atleast_2d(cfg["detpos"]).shape[0]
    ws, wd = _nwide(cfg, "widesrc"), _nwide(cfg, "widedet")
    ss, dd = np.meshgrid(np.arange(ns + ws), ns + ws + np.arange(nd + wd))
    sd = np.column_stack([ss.ravel(), dd.ravel()])
    return np.column_stack([sd, np.ones(len(sd))])


def deldotdel(node, elem, evol):
    """V * grad(phi_i) . grad(phi_j), 10 upper-triangle pairs (utility.py:53-98)."""
    e0 = elem[:, :4].astype(np.int64) - 1
    x = node[e0]  # Ne x 4 x 3
    # gradient of barycentric i: cofactor of the opposite face / (6V)
    cof = np.zeros((e0.shape[0], 4, 3))
    for i in range(4):
        a, b, c = [(i + k) % 4 for k in (1, 2, 3)]
        g = np.cross(x[:, b] - x[:, a], x[:, c] - x[:, a])
        # outward normal of face opposite i points away from i; gradient points to i
        s = np.sign(np.einsum("ij,ij->i", g, x[:, i] - x[:, a]))
        cof[:, i] = g * s[:, None]
    grad = cof / (6.0 * evol)[:, None, None]
    out = np.empty((e0.shape[0], 10))
    k = 0
    for i in range(4):
        for j in range(i, 4):
            out[:, k] = np.einsum("ij,ij->i", grad[:, i], grad[:, j])
            k += 1
    return out * evol[:, None]


def meshprep(cfg):
    """Fallback branch of meshprep without iso2mesh (utility.py:101-246)."""
    cfg = dict(cfg)
    for key in ("node", "elem", "srcpos", "srcdir", "detpos", "detdir", "prop", "seg"):
        if key in cfg and isinstance(cfg[key], list):
            cfg[key] = np.array(cfg[key])
    node = np.asarray(cfg["node"], dtype=np.float64)
    elem = cfg["elem"]
    if elem.shape[1] > 4 and cfg.get("seg") is None:
        cfg["seg"] = elem[:, 4].astype(int)
    if not cfg.get("isreoriented", False):
        r = reorient(node, elem[:, :4])
        cfg["elem"] = np.column_stack([r, elem[:, 4:]]) if elem.shape[1] > 4 else r
        cfg["isreoriented"] = True
    if cfg.get("face") is None:
        cfg["face"] = volface(cfg["elem"][:, :4])
    if cfg.get("area") is None:
        cfg["area"] = elemvolume(node, cfg["face"])
    if cfg.get("evol") is None:
        cfg["evol"] = elemvolume(node, cfg["elem"][:, :4])
    if np.any(cfg["evol"] == 0):
        raise ValueError("Degenerate elements detected")
    if cfg.get("reff") is None:
        bk = getbulk(cfg)
        cfg["reff"] = getreff(bk[3], 1.0)
        cfg["musp0"] = bk[1] * (1 - bk[2])
    if cfg.get("deldotdel") is None:
        cfg["deldotdel"] = deldotdel(node, cfg["elem"], cfg["evol"])
    cfg.setdefault("omega", 0)
    return cfg, sdmap(cfg)


# ----------------------------------------------------------------- forward
def props_per_entity(cfg):
    """(mua, musp, nref) per node/element as femlhs reads them (forward.py:126-144)."""
    props = cfg["prop"]
    nn, ne = cfg["node"].shape[0], cfg["elem"].shape[0]
    if props.shape[0] in (nn, ne):
        mua = props[:, 0]
        musp = props[:, 1] * (1 - props[:, 2]) if props.shape[1] >= 3 else props[:, 1]
        nref = props[:, 3] if props.shape[1] >= 4 else 1.37
    elif cfg.get("seg") is not None:
        idx = np.clip(np.asarray(cfg["seg"]).astype(np.int32), 0, props.shape[0] - 1)
        mua = props[idx, 0]
        musp = props[idx, 1] * (1 - props[idx, 2]) if props.shape[1] >= 3 else props[idx, 1]
        nref = props[idx[0], 3] if props.shape[1] >= 4 else 1.37
    else:
        raise ValueError("Property format not recognized")
    return mua, musp, nref


def femlhs(cfg, ddd, mode=1):
    """Assemble A = K D + M mua (+ i w n/c M) + Robin terms (forward.py:90-256)."""
    nn, ne = cfg["node"].shape[0], cfg["elem"].shape[0]
    evol, area = cfg["evol"], cfg["area"]
    e0 = cfg["elem"][:, :4].astype(np.int64) - 1
    f0 = cfg["face"].astype(np.int64) - 1
    reff = cfg.get("reff", 0.493)
    omega = 0 if mode == 2 else cfg.get("omega", 0)
    mua, musp, nref = props_per_entity(cfg)
    dco = 1.0 / (3.0 * (mua + musp))
    pairs = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    offk = [1, 2, 3, 5, 6, 8]
    diagk = [0, 4, 7, 9]
    wc = omega / C0
    cplx = omega > 0
    rows, cols, vals = [], [], []
    if len(mua) == ne:
        for k, (i, j) in enumerate(pairs):
            v = ddd[:, offk[k]] * dco + 0.05 * mua * evol
            if cplx:
                v = v + 1j * 0.05 * wc * nref * evol
            rows += [e0[:, i], e0[:, j]]
            cols += [e0[:, j], e0[:, i]]
            vals += [v, v]
        for i in range(4):
            v = ddd[:, diagk[i]] * dco + 0.10 * mua * evol
            if cplx:
                v = v + 1j * 0.10 * wc * nref * evol
            rows.append(e0[:, i]); cols.append(e0[:, i]); vals.append(v)
    else:
        mua_e = mua[e0]
        dco_e = dco[e0].mean(axis=1)
        nvec = np.ndim(nref) > 0 and len(nref) == nn
        n_e = nref[e0] if nvec else nref
        for k, (i, j) in enumerate(pairs):
            # lumped-pair mass weights: (sum_m mua_m + mua_i + mua_j) / 120
            w = (mua_e.sum(axis=1) + mua_e[:, i] + mua_e[:, j]) / 120.0
            v = ddd[:, offk[k]] * dco_e + w * evol
            if cplx:
                if nvec:
                    v = v + 1j * wc * (n_e.sum(axis=1) + n_e[:, i] + n_e[:, j]) / 120.0 * evol
                else:
                    v = v + 1j * wc * n_e * 0.05 * evol
            rows += [e0[:, i], e0[:, j]]
            cols += [e0[:, j], e0[:, i]]
            vals += [v, v]
        for i in range(4):
            w = (mua_e.sum(axis=1) + 2.0 * mua_e[:, i]) / 60.0
            v = ddd[:, diagk[i]] * dco_e + w * evol
            if cplx:
                if nvec:
                    v = v + 1j * wc * (n_e.sum(axis=1) + 2.0 * n_e[:, i]) / 60.0 * evol
                else:
                    v = v + 1j * wc * n_e * 0.10 * evol
            rows.append(e0[:, i]); cols.append(e0[:, i]); vals.append(v)
    bc = area * (1 - reff) / (12.0 * (1 + reff))
    for i, j in [(0, 1), (0, 2), (1, 2)]:
        rows += [f0[:, i], f0[:, j]]
        cols += [f0[:, j], f0[:, i]]
        vals += [0.5 * bc, 0.5 * bc]
    for i in range(3):
        rows.append(f0[:, i]); cols.append(f0[:, i]); vals.append(bc)
    dt = complex if cplx else float
    r = np.concatenate(rows); c = np.concatenate(cols)
    v = np.concatenate([np.asarray(x, dtype=dt) for x in vals])
    return sparse.coo_matrix((v, (r, c)), shape=(nn, nn), dtype=dt).tocsr()


def getoptodes(cfg):
    """Optodes moved inward by 1/(mua+musp) of the bulk (utility.py:799-876)."""
    bk = getbulk(cfg)
    ltr = 1.0 / (bk[0] + bk[1] * (1 - bk[2]))
    src = np.atleast_2d(cfg["srcpos"]).astype(np.float64)
    sdir = np.atleast_2d(cfg["srcdir"]).astype(np.float64)
    if sdir.shape[0] == 1:
        sdir = np.tile(sdir, (src.shape[0], 1))
    det = np.atleast_2d(cfg["detpos"]).astype(np.float64)
    ddir = np.atleast_2d(cfg.get("detdir", cfg["srcdir"])).astype(np.float64)
    if ddir.shape[0] == 1:
        ddir = np.tile(ddir, (det.shape[0], 1))
    return src + sdir * ltr, det + ddir * ltr


def femrhs(cfg):
    """Right-hand sides (forward.py:259-362), columns [point src | wide src |
    point det | wide det]: 4 barycentric weights per located point optode,
    the cfg['widesrc'] / cfg['widedet'] pattern columns as given; loc / bary
    NaN for wide-field columns."""
    src, det = getoptodes(cfg)
    nn = cfg["node"].shape[0]
    e0 = cfg["elem"][:, :4].astype(np.int64) - 1
    ns, nd = src.shape[0], det.shape[0]
    ws, wd = _nwide(cfg, "widesrc"), _nwide(cfg, "widedet")
    ncol = ns + ws + nd + wd
    pts = np.vstack([src, det])
    ploc, pbary = tsearchn(cfg["node"], cfg["elem"][:, :4], pts[:, :3])
    pcol = np.r_[np.arange(ns), ns + ws + np.arange(nd)]
    loc = np.full(ncol, np.nan)
    bary = np.full((ncol, 4), np.nan)
    loc[pcol], bary[pcol] = ploc, pbary
    rows, cols, vals = [], [], []
    for k, c in enumerate(pcol):
        if not np.isnan(ploc[k]):
            rows += list(e0[int(ploc[k]) - 1]); cols += [c] * 4; vals += list(pbary[k])
    for key, c0, w in (("widesrc", ns, ws), ("widedet", ns + ws + nd, wd)):
        if w:
            W = np.asarray(cfg[key], dtype=np.float64).reshape(nn, -1)
            r, c = np.nonzero(W)
            rows += list(r); cols += list(c + c0); vals += list(W[r, c])
    rhs = sparse.csr_matrix((vals, (rows, cols)), shape=(nn, ncol))
    return rhs, loc, bary, pts


def femgetdet(phi, cfg, rhs):
    """detval = rhs[:, det]^T phi[:, src] over point and wide-field columns
    (forward.py:365-442)."""
    ns = np.atleast_2d(cfg["srcpos"]).shape[0] + _nwide(cfg, "widesrc")
    nd = np.atleast_2d(cfg["detpos"]).shape[0] + _nwide(cfg, "widedet")
    rdet = rhs[:, ns:ns + nd]
    rdet = rdet.toarray() if sparse.issparse(rdet) else rdet
    return rdet.T @ phi[:, :ns]


def femsolve(A, rhs, method="superlu", tol=1e-10, maxiter=1000):
    """SuperLU multi-RHS solve, zero columns kept zero (solver.py:561-588);
    ``method='cg'``: per-column scipy CG (solver.py:717-754)."""
    if sparse.issparse(rhs):
        rhs = rhs.toarray()
    one_d = rhs.ndim == 1
    if one_d:
        rhs = rhs.reshape(-1, 1)
    cplx = np.iscomplexobj(A) or np.iscomplexobj(rhs)
    x = np.zeros(rhs.shape, dtype=complex if cplx else float)
    nz = [i for i in range(rhs.shape[1]) if np.any(rhs[:, i] != 0)]
    flag = 0
    if method == "superlu":
        if nz:
            lu = spla.splu(A.tocsc())
            sol = lu.solve(rhs[:, nz].astype(x.dtype))
            x[:, nz] = sol.reshape(rhs.shape[0], len(nz))
    elif method == "cg":
        for i in nz:
            x[:, i], info = spla.cg(A, rhs[:, i], rtol=tol, maxiter=maxiter)
            flag = max(flag, info)
    else:
        raise ValueError(f"unknown method {method}")
    return (x[:, 0] if one_d else x), flag


def runforward(cfg, **kw):
    """femrhs -> femlhs -> femsolve -> femgetdet (forward.py:40-87)."""
    if cfg.get("deldotdel") is None:
        cfg["deldotdel"] = deldotdel(cfg["node"], cfg["elem"], cfg["evol"])
    rhs, loc, bary, _ = femrhs(cfg)
    A = femlhs(cfg, cfg["deldotdel"])
    phi, _ = femsolve(A, rhs, **kw)
    return femgetdet(phi, cfg, rhs), phi


def jac(sd, phi, elem, evol):
    """Adjoint mua Jacobian, element then node-lumped (forward.py:509-569).

    Je[k, e] = -0.1 V_e (sum_i ps_i pd_i + 1/2 sum_{i!=j} ps_i pd_j);
    Jn = 0.25 * sum over the elements of each node.
    """
    e0 = elem[:, :4].astype(np.int64) - 1
    ne, nn = e0.shape[0], phi.shape[0]
    if sd.shape[1] >= 3:
        sda = sd[sd[:, 2] == 1, :2].astype(np.int64)
    else:
        sda = sd[:, :2].astype(np.int64)
    je = np.zeros((sda.shape[0], ne), dtype=phi.dtype)
    for k, (s, d) in enumerate(sda):
        ps, pd = phi[e0, s], phi[e0, d]
        diag = np.sum(ps * pd, axis=1)
        tot = ps.sum(axis=1) * pd.sum(axis=1)
        je[k] = -(diag + 0.5 * (tot - diag)) * 0.1 * evol
    P = sparse.csr_matrix((np.full(4 * ne, 0.25), (e0.ravel(), np.repeat(np.arange(ne), 4))), shape=(nn, ne))
    return (P @ je.T).T, je


# ------------------------------------------------------------------ recon
def normalize_diag(H):
    """Unit-diagonal scaling (recon.py:784-789)."""
    di = 1.0 / np.sqrt(np.abs(np.diag(H)) + 1e-16)
    return (di[:, None] * di[None, :]) * H, di


def reginvunder(J, r, lam):
    """(J J^T + lam I) y = r with diagonal normalisation, dmu = J^T y
    (recon.py:429-509, no invR)."""
    n = J.shape[1]
    keep_c = np.nonzero(np.sum(np.abs(J), axis=0) != 0)[0]
    Jc = J[:, keep_c]
    keep_r = np.sum(np.abs(Jc), axis=1) != 0
    Jc, r = Jc[keep_r], np.asarray(r)[keep_r]
    H = Jc @ Jc.T
    H[np.diag_indices_from(H)] += lam
    Hn, g = normalize_diag(H)
    y = g * np.linalg.solve(Hn, g * r.ravel())
    out = np.zeros(n, dtype=np.result_type(J, y))
    out[keep_c] = Jc.T @ y
    return out


def reginvover(J, r, lam):
    """(J^T J + lam I) x = J^T r with diagonal normalisation (recon.py:363-426)."""
    n = J.shape[1]
    keep_c = np.nonzero(np.sum(np.abs(J), axis=0) != 0)[0]
    Jc = J[:, keep_c]
    keep_r = np.sum(np.abs(Jc), axis=1) != 0
    Jc, r = Jc[keep_r], np.asarray(r)[keep_r]
    rp = Jc.T @ r.ravel()
    H = Jc.T @ Jc
    H[np.diag_indices_from(H)] += lam
    Hn, g = normalize_diag(H)
    x = g * np.linalg.solve(Hn, g * rp)
    out = np.zeros(n, dtype=x.dtype)
    out[keep_c] = x
    return out


def reginv(J, r, lam):
    """Over/under-determined dispatch (recon.py:338-360)."""
    return reginvover(J, r, lam) if J.shape[0] >= J.shape[1] else reginvunder(J, r, lam)


def matreform(J, ymeas, ymodel, form="real"):
    """'complex' / 'real' / 'reim' / 'logphase' reformulation (recon.py:512-567)."""
    rhs = ymeas - ymodel
    if form == "complex":
        return J, rhs, 1
    if form in ("real", "reim"):
        if not np.isreal(rhs).all() and not np.isreal(J).all():
            if form == "reim":
                A = np.block([[J.real, -J.imag], [J.imag, J.real]])
            else:
                A = np.vstack([J.real, J.imag])
            return A, np.concatenate([rhs.real, rhs.imag]), 2
        return np.real(J), np.real(rhs), 1
    if form == "logphase":
        t = np.conj(ymodel) / np.abs(ymodel * ymodel)
        t = t[:, None] * J if J.ndim == 2 else t * J
        if np.isreal(ymodel).all():
            return np.real(t), np.log(np.abs(ymeas)) - np.log(np.abs(ymodel)), 1
        return (np.vstack([t.real, t.imag]),
                np.concatenate([np.log(np.abs(ymeas)) - np.log(np.abs(ymodel)),
                                np.angle(ymeas) - np.angle(ymodel)]), 2)
    raise ValueError(f"Unknown form: {form}")


def runrecon(cfg, recon, detphi0, sd=None, maxiter=5, lambda_=0.05, tol=0, reform="real"):
    """Gauss-Newton loop for node-based ``mua`` (recon.py:39-335 restricted to
    one wavelength, single mesh, no prior): forward -> jac -> reform ->
    Frobenius block scaling -> reginv -> prop[:,0] += dmu."""
    if sd is None:
        sd = sdmap(cfg)
    resid = np.zeros(maxiter)
    updates = []
    for it in range(maxiter):
        cfg["prop"] = recon["prop"].copy()
        det, phi = runforward(cfg)
        jn, _ = jac(sd, phi, cfg["elem"], cfg["evol"])
        y0, y = np.asarray(detphi0).ravel(), det.ravel()
        if reform != "complex":
            J, misfit, _ = matreform(jn, y0, y, reform)
        else:
            J, misfit = jn, y0 - y
        resid[it] = np.sum(np.abs(misfit))
        scale = 1.0 / np.sqrt(np.sum(J ** 2))
        dmu = reginv(J * scale, misfit, lambda_) * scale
        recon["prop"][:, 0] += dmu
        updates.append({"mua": dmu})
        if it > 0 and abs(resid[it] - resid[it - 1]) / resid[0] < tol:
            resid = resid[: it + 1]
            break
    recon["lambda"] = lambda_
    return recon, resid, cfg, updates, jn, det, phi

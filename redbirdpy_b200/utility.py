"""Mesh preparation and optode bookkeeping (host side of the drop-in API).

Mirrors redbirdpy's ``utility`` functions that the FEM path consumes
(redbirdpy/utility.py).  Index convention as in redbirdpy: ``elem``/``face``
in ``cfg`` are 1-based; the device layer converts once.  Heavy mesh work
(node incidence, the CSR pattern, element gradients) runs on the GPU through
``redbirdpy_b200.engine``.
"""

import weakref

import numpy as np
import torch

__all__ = [
    "meshprep", "deldotdel", "sdmap", "getoptodes", "getdistance", "getltr", "getreff",
    "getbulk", "forcearray", "elem2node",
]

_ARRAY_KEYS = ["node", "elem", "face", "srcpos", "srcdir", "detpos", "detdir", "prop", "seg",
               "widesrc", "widedet"]


def forcearray(cfg, keys=_ARRAY_KEYS):
    """List-valued cfg entries -> numpy arrays (utility.py:1112-1117)."""
    for key in keys:
        if key in cfg and isinstance(cfg[key], list):
            cfg[key] = np.array(cfg[key])
    return cfg


def _signed_volume6(node, e0):
    x0 = node[e0[:, 0]]
    return np.einsum("ij,ij->i", np.cross(node[e0[:, 1]] - x0, node[e0[:, 2]] - x0), node[e0[:, 3]] - x0)


def _reorient(node, elem):
    """Swap nodes 0 and 1 of negatively oriented tets (utility.py:1047-1063)."""
    elem = np.array(elem, copy=True)
    neg = _signed_volume6(node, elem[:, :4].astype(np.int64) - 1) < 0
    elem[neg, 0], elem[neg, 1] = elem[neg, 1].copy(), elem[neg, 0].copy()
    return elem


def _volface(elem, nn):
    """Boundary triangles, in the order redbirdpy's fallback returns them
    (utility.py:1066-1087): sorted by their sorted node triple, keeping the
    orientation of the owning tet.  One int64 key per face replaces the
    row-wise unique."""
    e0 = elem[:, :4].astype(np.int64) - 1
    faces = np.concatenate([e0[:, [0, 2, 1]], e0[:, [0, 1, 3]], e0[:, [0, 3, 2]], e0[:, [1, 2, 3]]])
    s = np.sort(faces, axis=1)
    key = (s[:, 0] * nn + s[:, 1]) * nn + s[:, 2]
    _, first, counts = np.unique(key, return_index=True, return_counts=True)
    return faces[first[counts == 1]] + 1


def _elemvolume(node, cells):
    """|volume| of tets or area of triangles (utility.py:1090-1109)."""
    c0 = cells.astype(np.int64) - 1
    if c0.shape[1] >= 4:
        return np.abs(_signed_volume6(node, c0)) / 6.0
    v = np.cross(node[c0[:, 1]] - node[c0[:, 0]], node[c0[:, 2]] - node[c0[:, 0]])
    return 0.5 * np.sqrt(np.sum(v ** 2, axis=1))


def _nodevolume(nn, elem, evol):
    """Quarter of the incident tet volumes per node (utility.py:1005-1017)."""
    e0 = elem[:, :4].astype(np.int64) - 1
    return 0.25 * np.bincount(e0.ravel(), weights=np.repeat(evol, 4), minlength=nn)


def getreff(n_in, n_out=1.0):
    """Effective reflection coefficient, 2000-step quadrature (utility.py:879-904)."""
    if n_in <= n_out:
        return 0.0
    oc = np.arcsin(n_out / n_in)
    step = np.pi / 2000
    o = np.arange(0, oc, step)
    cos_t = np.sqrt(1 - (n_in * np.sin(o)) ** 2)
    cos_i = np.cos(o)
    fres = 0.5 * ((n_in * cos_t - n_out * cos_i) / (n_in * cos_t + n_out * cos_i)) ** 2
    fres = fres + 0.5 * ((n_in * cos_i - n_out * cos_t) / (n_in * cos_i + n_out * cos_t)) ** 2
    full = np.arange(0, np.pi / 2, step)
    rf = np.ones(len(full))
    rf[: len(fres)] = fres
    cf = np.cos(full)
    r_phi = 2 * np.sum(np.sin(full) * cf * rf) * step
    r_j = 3 * np.sum(np.sin(full) * cf ** 2 * rf) * step
    return (r_phi + r_j) / (2 - r_phi + r_j)


def _first_elem_with_node(cfg, v):
    """Index of the first tet that has (1-based) node v, or None; cached in
    cfg['_b200'] beside the mesh (a full scan of elem otherwise), and dropped
    with it when cfg's elem array is replaced."""
    elem = cfg["elem"]
    cache = cfg.get("_b200")
    hit_cache = isinstance(cache, dict) and cache.get("first_elem_key") == (int(v), np.shape(elem))
    if hit_cache and cache.get("first_elem_ref") is not None and cache["first_elem_ref"]() is elem:
        return cache["first_elem"]
    hit = np.nonzero(np.any(elem[:, :4] == v, axis=1))[0]
    r = int(hit[0]) if len(hit) else None
    if isinstance(cache, dict):
        try:
            ref = weakref.ref(elem)
        except TypeError:
            ref = None
        cache["first_elem_key"], cache["first_elem"], cache["first_elem_ref"] = (int(v), np.shape(elem)), r, ref
    return r


def getbulk(cfg):
    """Bulk [mua, mus, g, n] at the air interface (property.py:216-332)."""
    default = np.array([0.0, 0.0, 0.0, 1.37])
    if "bulk" in cfg:
        b = cfg["bulk"]
        out = default.copy()
        if "mua" in b:
            out[0] = b["mua"]
        if "dcoeff" in b:
            out[1], out[2] = 1.0 / (3 * b["dcoeff"]), 0
        if "musp" in b:
            out[1], out[2] = b["musp"], 0
        if "g" in b:
            out[2] = b["g"]
        if "n" in b:
            out[3] = b["n"]
        return out
    prop = cfg.get("prop")
    if prop is None:
        return default
    if isinstance(prop, dict):  # one bulk per wavelength (property.py:267-271)
        return {wv: _bulk_from_prop(np.atleast_2d(p), cfg, default) for wv, p in prop.items()}
    return _bulk_from_prop(np.atleast_2d(prop), cfg, default)


def _bulk_from_prop(prop, cfg, default):
    """The bulk row of one property table (property.py:275-332)."""
    nn = cfg["node"].shape[0]
    ne = cfg["elem"].shape[0]
    face = cfg.get("face")
    if prop.shape[0] < min(nn, ne):
        seg = cfg.get("seg")
        if seg is None:
            return prop[1] if prop.shape[0] > 1 else default
        seg = np.asarray(seg)
        if face is not None and len(seg) == nn:
            label = seg[face[0, 0] - 1]
        elif face is not None and len(seg) == ne:
            hit = _first_elem_with_node(cfg, face[0, 0])
            label = seg[hit] if hit is not None else 0
        else:
            label = seg[0]
        label = int(label)
        if prop.shape[0] > label:
            return prop[label]
        return prop[1] if prop.shape[0] > 1 else default
    if prop.shape[0] == nn:
        return prop[face[0, 0] - 1] if face is not None else prop[0]
    if prop.shape[0] == ne:
        if face is not None:
            hit = _first_elem_with_node(cfg, face[0, 0])
            if hit is not None:
                return prop[hit]
        return prop[0]
    return default


def getltr(cfg, wv=""):
    """Transport mean free path 1/(mua + musp) of the bulk (utility.py:862-876);
    with per-wavelength properties, of wavelength ``wv`` (default: the first)."""
    bk = getbulk(cfg)
    if isinstance(bk, dict):
        bk = bk[wv if wv else next(iter(bk))]
    return 1.0 / (bk[0] + bk[1] * (1 - bk[2]))


def getoptodes(cfg, wv=""):
    """Point optodes moved inward by ltr along their direction (utility.py:799-822).
    Returns (pointsrc, pointdet, widesrc, widedet)."""
    ltr = getltr(cfg, wv)
    src = det = None
    if cfg.get("srcpos") is not None and np.size(cfg["srcpos"]) > 0:
        sp = np.atleast_2d(np.asarray(cfg["srcpos"], dtype=np.float64))
        sdir = np.atleast_2d(np.asarray(cfg["srcdir"], dtype=np.float64))
        if sdir.shape[0] == 1:
            sdir = np.tile(sdir, (sp.shape[0], 1))
        src = sp[:, :3] + sdir[:, :3] * ltr
    if cfg.get("detpos") is not None and np.size(cfg["detpos"]) > 0:
        dp = np.atleast_2d(np.asarray(cfg["detpos"], dtype=np.float64))
        ddir = np.atleast_2d(np.asarray(cfg.get("detdir", cfg["srcdir"]), dtype=np.float64))
        if ddir.shape[0] == 1:
            ddir = np.tile(ddir, (dp.shape[0], 1))
        det = dp[:, :3] + ddir[:, :3] * ltr
    return src, det, cfg.get("widesrc"), cfg.get("widedet")


def getdistance(srcpos, detpos, badsrc=None, baddet=None, widesrc=None, widedet=None):
    """Source-detector distances, Ndet x Nsrc, inf for excluded (utility.py:825-859)."""
    badsrc, baddet = badsrc or [], baddet or []
    srcpos, detpos = np.atleast_2d(srcpos), np.atleast_2d(detpos)
    dist = np.full((detpos.shape[0], srcpos.shape[0]), np.inf)
    gs = sorted(set(range(srcpos.shape[0])) - set(badsrc))
    gd = sorted(set(range(detpos.shape[0])) - set(baddet))
    if gs and gd:
        diff = srcpos[gs, None, :3] - detpos[None, gd, :3]
        dist[np.ix_(gd, gs)] = np.sqrt(np.sum(diff.transpose(1, 0, 2) ** 2, axis=2))
    return dist


def _npattern(w):
    return np.asarray(w).reshape(np.shape(w)[0], -1).shape[1] if w is not None and np.size(w) else 0


def sdmap(cfg, maxdist=np.inf, **kwargs):
    """Source/detector pair table [src_col, det_col, active] (utility.py:675-796).
    Rows are detector-major (meshgrid); columns index the RHS / phi columns in
    femrhs's order [point src | wide src | point det | wide det].  Excluded
    point optodes are left out; ``maxdist`` deactivates point pairs only
    (wide-field pairs stay active)."""
    ns = np.atleast_2d(cfg["srcpos"]).shape[0] if cfg.get("srcpos") is not None and np.size(cfg["srcpos"]) else 0
    nd = np.atleast_2d(cfg["detpos"]).shape[0] if cfg.get("detpos") is not None and np.size(cfg["detpos"]) else 0
    ws, wd = _npattern(cfg.get("widesrc")), _npattern(cfg.get("widedet"))
    if ns + ws == 0 or nd + wd == 0:
        raise ValueError("Must define at least one source and detector")
    badsrc = kwargs.get("excludesrc", cfg.get("excludesrc", []))
    baddet = kwargs.get("excludedet", cfg.get("excludedet", []))
    gs = sorted(set(range(ns)) - set(badsrc)) + list(range(ns, ns + ws))
    d0 = ns + ws  # first detector column
    gd = [d0 + d for d in sorted(set(range(nd)) - set(baddet))] + [d0 + nd + j for j in range(wd)]
    ss, dd = np.meshgrid(gs, gd)
    sd = np.column_stack([ss.ravel(), dd.ravel()])
    if maxdist < np.inf and ns > 0 and nd > 0:
        dist = getdistance(cfg["srcpos"], cfg["detpos"], badsrc, baddet)
        active = np.array([1.0 if not (s < ns and d - d0 < nd) or dist[int(d) - d0, int(s)] < maxdist else 0.0
                           for s, d in sd])
        out = np.column_stack([sd, active])
    else:
        out = np.column_stack([sd, np.ones(len(sd))])
    if isinstance(cfg.get("prop"), dict):
        # one table per wavelength, with a fourth column of ones (utility.py:733-768)
        out = np.column_stack([out, np.ones(len(out))])
        return {wv: out.copy() for wv in cfg["prop"]}
    return out


def elem2node(elem, elemval, nodelen=None):
    """Average element values onto nodes (utility.py:910-929)."""
    if isinstance(elem, dict):
        nodelen = elem["node"].shape[0]
        elem = elem["elem"]
    e0 = elem[:, :4].astype(np.int64) - 1
    ev = elemval[:, None] if elemval.ndim == 1 else elemval
    out = np.zeros((nodelen, ev.shape[1]))
    for j in range(4):
        np.add.at(out, e0[:, j], ev)
    return (0.25 * out).squeeze()


def deldotdel(cfg):
    """V grad(phi_i).grad(phi_j) for the 10 pairs i<=j, computed on the GPU
    (utility.py:53-98).  Returns ``(ddd, None)``; the reference's second
    output (the 3x4xNe gradients) is not materialised."""
    from . import engine

    return engine.mesh_of(cfg).deldotdel_host(), None


def _device_geometry(cfg, node, nn):
    """Reorientation, boundary faces, face areas and tet volumes on the GPU
    (rb_reorient / rb_volface / rb_face_area): the reference's fallbacks
    (utility.py:1047-1109), bit for bit, returned into cfg as numpy with the
    reference's 1-based indices."""
    from . import engine

    elem = cfg["elem"]
    need = (not cfg.get("isreoriented", False)) or cfg.get("face") is None or cfg.get("area") is None \
        or cfg.get("evol") is None
    if not need:
        return
    dev = engine._dev()
    node_d = torch.as_tensor(np.ascontiguousarray(node[:, :3]), device=dev)
    e0 = torch.as_tensor(np.ascontiguousarray(np.asarray(elem)[:, :4].astype(np.int64) - 1, dtype=np.int32),
                         device=dev)
    ne = e0.shape[0]
    st = engine.stream()
    evol = torch.empty(max(ne, 1), dtype=torch.float64, device=dev)
    if not cfg.get("isreoriented", False):
        engine.call("rb_reorient", engine.ptr(node_d), engine.ptr(e0), ne, engine.ptr(evol), None, st)
        r = e0.cpu().numpy().astype(np.asarray(elem).dtype) + 1
        cfg["elem"] = np.column_stack([r, elem[:, 4:]]) if elem.shape[1] > 4 else r
        cfg["isreoriented"] = True
    elif cfg.get("evol") is None:  # volumes only: a scratch copy takes the swaps
        tmp = e0.clone()
        engine.call("rb_reorient", engine.ptr(node_d), engine.ptr(tmp), ne, engine.ptr(evol), None, st)
    if cfg.get("face") is None or cfg.get("area") is None:
        if cfg.get("face") is None:
            face = torch.empty((4 * ne, 3), dtype=torch.int32, device=dev)
            wb = engine._lib.lib().rb_volface_work_bytes(ne)
            work = torch.empty(wb, dtype=torch.uint8, device=dev)
            nf = engine.ctypes.c_int64(0)
            engine.call("rb_volface", engine.ptr(e0), ne, nn, engine.ptr(face), engine.ctypes.byref(nf),
                        engine.ptr(work), wb, st)
            face = face[: nf.value]
            cfg["face"] = face.cpu().numpy().astype(np.int64) + 1
        else:
            face = torch.as_tensor(np.ascontiguousarray(np.asarray(cfg["face"])[:, :3].astype(np.int64) - 1,
                                                        dtype=np.int32), device=dev)
        if cfg.get("area") is None:
            area = torch.empty(max(face.shape[0], 1), dtype=torch.float64, device=dev)
            engine.call("rb_face_area", engine.ptr(node_d), engine.ptr(face), face.shape[0], engine.ptr(area), st)
            cfg["area"] = area[: face.shape[0]].cpu().numpy()
    if cfg.get("evol") is None:
        cfg["evol"] = evol[:ne].cpu().numpy()


def meshprep(cfg):
    """Prepare the mesh dict in place (utility.py:101-246): reorientation,
    boundary faces, areas/volumes, nodal volumes, reff/musp0, the sparse
    pattern (rows/cols/idxcount/idxsum), deldotdel, omega and the sd table.
    The reorientation, faces and volumes follow redbirdpy's own fallbacks, so
    ``cfg`` comes out identical to the reference's."""
    cfg = forcearray(cfg)
    if "node" not in cfg or "elem" not in cfg:
        raise ValueError("cfg must contain 'node' and 'elem'")
    node = np.asarray(cfg["node"], dtype=np.float64)
    cfg["node"] = node
    elem = cfg["elem"]
    nn = node.shape[0]
    if elem.shape[1] > 4 and cfg.get("seg") is None:
        cfg["seg"] = elem[:, 4].astype(int)
    # a tet that repeats a node has zero volume: caught on the host before any
    # device work (other zero volumes once the device has computed them)
    se = np.sort(np.asarray(cfg["elem"])[:, :4], axis=1)
    rep = np.nonzero(np.any(se[:, 1:] == se[:, :-1], axis=1))[0]
    if rep.size:
        raise ValueError(f"Degenerate elements detected at indices: {rep}")
    _device_geometry(cfg, node, nn)
    if np.any(cfg["evol"] == 0):
        bad = np.where(cfg["evol"] == 0)[0]
        raise ValueError(f"Degenerate elements detected at indices: {bad}")
    if "srcpos" not in cfg:
        raise ValueError("cfg.srcpos is required")
    if "srcdir" not in cfg:
        raise ValueError("cfg.srcdir is required")
    if isinstance(cfg.get("prop"), dict) and "param" in cfg:
        # multi-spectral: per-wavelength properties from the chromophores
        # (utility.py:193-194); coefficients from cfg['extin'] when given
        from .property import updateprop

        cfg["prop"] = updateprop(cfg, extin=cfg.get("extin"))
    if cfg.get("reff") is None:
        bk = getbulk(cfg)
        if isinstance(bk, dict):  # per wavelength (utility.py:198-205)
            cfg["reff"] = {wv: getreff(b[3], 1.0) for wv, b in bk.items()}
            cfg["musp0"] = {wv: b[1] * (1 - b[2]) for wv, b in bk.items()}
        else:
            cfg["reff"] = getreff(bk[3], 1.0)
            cfg["musp0"] = bk[1] * (1 - bk[2])
    # wide-field patterns: taken as given in cfg['widesrc'] / cfg['widedet']
    # (Nn x Npattern); making them from a source type (src2bc's projection of
    # an illumination pattern onto the boundary, utility.py:252-636) is
    # outside this engine (utility.py:210-224 calls it only when they are
    # missing)
    for kind in ("src", "det"):
        typ = cfg.get(kind + "type", "pencil")
        if (typ not in ("pencil", "isotropic") or ("wide%sid" % kind) in cfg) and ("wide" + kind) not in cfg:
            raise NotImplementedError(f"wide-field {kind} patterns must be given as cfg['wide{kind}'] "
                                      "(src2bc's pattern projection is outside this engine's scope)")
    from . import engine

    dm = engine.mesh_of(cfg)
    if cfg.get("nvol") is None:
        nvol = torch.empty(nn, dtype=torch.float64, device=dm.device)
        engine.call("rb_nodevolume", nn, engine.ptr(dm.eptr), engine.ptr(dm.elist), engine.ptr(dm.evol),
                    engine.ptr(nvol), engine.stream())
        cfg["nvol"] = nvol.cpu().numpy()
    if cfg.get("cols") is None:
        cfg["rows"], cfg["cols"], cfg["idxcount"] = dm.adjacency_host()
    if cfg.get("idxsum") is None:
        cfg["idxsum"] = np.cumsum(cfg["idxcount"])
    if cfg.get("deldotdel") is None:
        cfg["deldotdel"] = dm.deldotdel_host()
    if "omega" not in cfg:
        cfg["omega"] = 0
    return cfg, sdmap(cfg)

"""Generate the golden fixtures by running the reference redbirdpy itself.

Usage (in a container that has the reference sources)::

    python tests/golden/make_golden.py [/path/to/redbirdpy-checkout]
    python tests/golden/make_golden.py --contract [--c2] [--c3] [--c5]
    python tests/golden/make_golden.py --wide
    python tests/golden/make_golden.py --recon

The second form writes the contract-size fixtures (the 3M-tet forward on a
source/detector subset, the 375k-tet Jacobian columns and finite
differences, 8 batched instances); it takes several minutes.

The reference is imported from the given checkout (default
``/root/reference``).  iso2mesh is not installed, so the project-written
``oracle.tsearch.tsearchn`` is injected as ``sys.modules['iso2mesh']`` after
the import; redbirdpy then uses its own fallbacks for reorientation, boundary
faces and volumes.  For complex (frequency-domain) Jacobians
``redbirdpy.forward.HAS_NUMBA`` is switched off because the Numba kernel
writes complex values into a float64 array (redbirdpy/forward.py:461).

Each case is written as a small ``.npz`` next to this script.
"""

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def load_reference(path):
    sys.path.insert(0, path)
    sys.path.insert(0, ROOT)
    import redbirdpy as rb  # noqa: E402
    from oracle import tsearch  # noqa: E402

    shim = types.ModuleType("iso2mesh")
    shim.tsearchn = tsearch.tsearchn
    sys.modules["iso2mesh"] = shim
    return rb


def csr_fields(prefix, A):
    return {prefix + "_data": A.data, prefix + "_indices": A.indices, prefix + "_indptr": A.indptr}


def c1_cfg(omega=0.0):
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([60, 60, 30], 5)
    return dict(
        node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
        srcpos=np.array([[30, 30, 0.0]]), srcdir=np.array([[0, 0, 1.0]]),
        detpos=np.array([[30, 40, 0.0], [40, 30, 0.0]]), detdir=np.array([[0, 0, 1.0]]),
        seg=np.ones(elem.shape[0], dtype=int), omega=omega,
    )


def nodal_cfg(omega=0.0, seed=0):
    """40x40x20 mm box at 4 mm (726 nodes, 3000 tets), per-node properties,
    4 sources x 4 detectors on z=0."""
    from redbirdpy_b200.meshgen import kuhn_box, grid_optodes

    node, elem = kuhn_box([40, 40, 20], 4)
    rng = np.random.default_rng(seed)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn),
                            np.zeros(nn), np.full(nn, 1.37)])
    return dict(
        node=node, elem=elem, prop=prop,
        srcpos=grid_optodes([10, 30], [10, 30], 2), srcdir=np.array([[0, 0, 1.0]]),
        detpos=grid_optodes([10, 30], [10, 30], 2, offset=(4, 4)), detdir=np.array([[0, 0, 1.0]]),
        omega=omega,
    )


def run_case(rb, cfg, with_jac=True):
    cfg, sd = rb.meshprep(cfg)
    A = rb.femlhs(cfg, cfg["deldotdel"])
    rhs, loc, bary, optode = rb.femrhs(cfg, sd)
    det, phi = rb.run(cfg)
    out = dict(node=cfg["node"], elem=cfg["elem"], face=cfg["face"], area=cfg["area"],
               evol=cfg["evol"], nvol=cfg["nvol"], deldotdel=cfg["deldotdel"],
               reff=cfg["reff"], sd=sd, loc=loc, bary=bary, optode=optode,
               rhs=rhs.toarray(), detval=det, phi=phi, prop=cfg["prop"],
               srcpos=cfg["srcpos"], detpos=cfg["detpos"], omega=cfg["omega"])
    if cfg.get("seg") is not None:
        out["seg"] = cfg["seg"]
    out.update(csr_fields("A", A))
    if with_jac:
        jn, je = rb.jac(sd, phi, cfg["deldotdel"], cfg["elem"], cfg["evol"])
        out["jn"], out["je"] = jn, je
    return out


def multi_wavelength(rb):
    """Per-wavelength properties (cfg['prop'] keyed by wavelength): meshprep's
    reff per wavelength, runforward's detval / phi per wavelength."""
    cfg = nodal_cfg()
    p1 = cfg["prop"]
    p2 = p1.copy()
    p2[:, 0] *= 1.5
    p2[:, 1] *= 0.8
    p2[:, 3] = 1.40
    cfg["prop"] = {"690": p1, "830": p2}
    cfg, sd = rb.meshprep(cfg)
    det, phi = rb.run(cfg)
    out = dict(node=cfg["node"], elem=cfg["elem"], face=cfg["face"], area=cfg["area"], evol=cfg["evol"],
               deldotdel=cfg["deldotdel"], srcpos=cfg["srcpos"], detpos=cfg["detpos"], omega=cfg["omega"])
    for wv in ("690", "830"):
        out["prop_" + wv] = cfg["prop"][wv]
        out["reff_" + wv] = cfg["reff"][wv]
        out["detval_" + wv] = det[wv]
        out["phi_" + wv] = phi[wv]
        out["sd_" + wv] = sd[wv]
    np.savez_compressed(os.path.join(HERE, "nodal_multiwl.npz"), **out)


def wide_cfg(omega=0.0):
    """nodal_cfg plus wide-field patterns (cfg['widesrc'] / cfg['widedet'],
    Nn x Npattern, given directly so that meshprep does not call src2bc):
    two Gaussian spots and one linear ramp on the z = 0 boundary nodes as
    sources, one Gaussian spot and one uniform strip as detectors."""
    cfg = nodal_cfg(omega)
    node = cfg["node"]
    top = np.isclose(node[:, 2], 0.0)
    x, y = node[:, 0], node[:, 1]

    def spot(cx, cy, s):
        return np.where(top, np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s)), 0.0)

    cfg["widesrc"] = np.column_stack([spot(12, 20, 4), spot(28, 14, 6), np.where(top, x / 40.0, 0.0)])
    cfg["widedet"] = np.column_stack([spot(20, 28, 5), np.where(top & (y > 30), 1.0, 0.0)])
    return cfg


def wide_case(rb, omega):
    cfg, sd = rb.meshprep(wide_cfg(omega))
    rhs, loc, bary, optode = rb.femrhs(cfg, sd)
    det, phi = rb.run(cfg)
    jn, _ = rb.jac(sd, phi, cfg["deldotdel"], cfg["elem"], cfg["evol"])
    return dict(node=cfg["node"], elem=cfg["elem"], face=cfg["face"], area=cfg["area"], evol=cfg["evol"],
                prop=cfg["prop"], srcpos=cfg["srcpos"], detpos=cfg["detpos"], widesrc=cfg["widesrc"],
                widedet=cfg["widedet"], omega=cfg["omega"], reff=cfg["reff"], sd=sd, rhs=rhs.toarray(), loc=loc,
                bary=bary, detval=det, phi=phi, jn=jn)


def multiwl_gn(rb):
    """Two GN iterations of a two-wavelength chromophore reconstruction
    (cfg['param'] hbo / hbr per node; water and lipids take the reference's
    defaults) on the nodal mesh, data from a +20% hbo patch."""
    cfg = nodal_cfg()
    nn = cfg["node"].shape[0]
    rng = np.random.default_rng(4)
    tmpl = np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]])
    cfg["prop"] = {"690": tmpl.copy(), "830": tmpl.copy()}
    hbo, hbr = rng.uniform(40, 60, nn), rng.uniform(20, 30, nn)
    cfg["param"] = {"hbo": hbo.copy(), "hbr": hbr.copy()}
    cfg, sd = rb.meshprep(cfg)
    tcfg = dict(cfg)
    tcfg["param"] = {"hbo": hbo * np.where(np.linalg.norm(cfg["node"] - [20, 20, 8], axis=1) < 9, 1.2, 1.0),
                     "hbr": hbr.copy()}
    tcfg["prop"] = rb.updateprop(tcfg)
    det0, _ = rb.run(tcfg)
    recon = {"param": {"hbo": hbo.copy(), "hbr": hbr.copy()}}
    chroms = ["hbo", "hbr", "water", "lipids"]
    ext, _ = rb.extinction(["690", "830"], chroms)
    newrecon, resid, cfg2, updates, _, det, _ = rb.run(cfg, recon, det0, sd, maxiter=2, lambda_=0.05, report=False)
    out = dict(hbo=hbo, hbr=hbr, ext=ext, chroms=np.array(chroms), resid=resid,
               hbo_out=newrecon["param"]["hbo"], hbr_out=newrecon["param"]["hbr"],
               water_out=np.atleast_1d(cfg2["param"]["water"]), lipids_out=np.atleast_1d(cfg2["param"]["lipids"]))
    for wv in ("690", "830"):
        out["det0_" + wv] = det0[wv]
        out["det_" + wv] = det[wv]
    for k, u in enumerate(updates):
        for key, v in u.items():
            out[f"upd{k}_{key}"] = v
    np.savez_compressed(os.path.join(HERE, "multiwl_gn.npz"), **out)


def dualmesh_gn(rb):
    """Two GN iterations on a coarse reconstruction mesh (box 40 x 40 x 20 mm
    at 10 mm, 75 nodes) mapped onto the nodal forward mesh (mapid / mapweight
    from locating the forward nodes in the coarse tets)."""
    from oracle.tsearch import tsearchn
    from redbirdpy_b200.meshgen import kuhn_box

    cfg = nodal_cfg()
    cfg, sd = rb.meshprep(cfg)
    rnode, relem = kuhn_box([40, 40, 20], 10)
    mapid, mapweight = tsearchn(rnode, relem, cfg["node"])
    nr = rnode.shape[0]
    rprop = np.column_stack([np.full(nr, 0.01), np.full(nr, 1.0), np.zeros(nr), np.full(nr, 1.37)])
    truth = cfg["prop"].copy()
    truth[np.linalg.norm(cfg["node"] - [25, 15, 8], axis=1) < 8, 0] *= 1.5
    tcfg = dict(cfg)
    tcfg["prop"] = truth
    det0, _ = rb.run(tcfg)
    recon = {"node": rnode, "elem": relem, "prop": rprop.copy(), "mapid": mapid, "mapweight": mapweight}
    newrecon, resid, _, updates, _, det, _ = rb.run(cfg, recon, det0, sd, maxiter=2, lambda_=0.05, report=False)
    np.savez_compressed(os.path.join(HERE, "dualmesh_gn.npz"), rnode=rnode, relem=relem, rprop=rprop, mapid=mapid,
                        mapweight=mapweight, det0=det0, resid=resid, prop_out=newrecon["prop"],
                        dmu0=updates[0]["mua"], dmu1=updates[1]["mua"], det=det)


def reform_gn(rb, form):
    """Two GN iterations of the frequency-domain nodal case with matreform
    'logphase' or 'reim' (recon.py:512-567)."""
    cfg = nodal_cfg(2 * np.pi * 1e8)
    cfg, sd = rb.meshprep(cfg)
    truth = cfg["prop"].copy()
    truth[:, 0] *= 1.1
    tcfg = dict(cfg)
    tcfg["prop"] = truth
    det0, _ = rb.run(tcfg)
    prop0 = cfg["prop"].copy()
    recon = {"prop": prop0.copy()}
    newrecon, resid, _, updates, _, det, _ = rb.run(cfg, recon, det0, sd, maxiter=2, lambda_=0.05, report=False,
                                                    reform=form)
    np.savez_compressed(os.path.join(HERE, f"reform_{form}.npz"), prop0=prop0, det0=det0, resid=resid,
                        prop_out=newrecon["prop"], dmu0=updates[0]["mua"], dmu1=updates[1]["mua"], det=det)


# ----------------------------------------------------- contract-size cases
def c3_cfg():
    """Box 100 x 100 x 50 mm at 2 mm (67,626 nodes, 375,000 tets), per-node
    mua ~ U[0.008, 0.012] and mus ~ U[0.9, 1.1] (default_rng(0)), 32 sources
    on an 8 x 4 grid over x in [15, 85], y in [30, 70] on z = 0 and 32
    detectors offset by 5 mm, CW."""
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([100, 100, 50], 2)
    rng = np.random.default_rng(0)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn), np.zeros(nn),
                            np.full(nn, 1.37)])
    # 8 x 4 source grid, detectors offset by 5 mm in x and y
    src = np.column_stack([np.repeat(np.linspace(15, 85, 8), 4), np.tile(np.linspace(30, 70, 4), 8), np.zeros(32)])
    return dict(node=node, elem=elem, prop=prop, srcpos=src, srcdir=np.array([[0, 0, 1.0]]), detpos=src + [5, 5, 0],
                detdir=np.array([[0, 0, 1.0]]), omega=0.0)


def c3_case(rb):
    """The reference's run (detval) and jac (64 seeded node columns) at the
    375k-tet size, plus central differences (h = 1e-4 relative, at fixed D
    for mua and at fixed mua for D) of L = 0.5 ||log det - log target||^2,
    target from a +10% mua perturbation, on the same 64 nodes.  The perturbed
    forward solves reuse the SuperLU factor of the unperturbed matrix through
    the Woodbury identity: a nodal perturbation changes A only on the node's
    neighbourhood S, so det' = det - phi_d[S]^T (I + dA_SS G)^-1 dA_SS phi_s[S]
    with G = A^-1[S, S] -- the same numbers as refactoring A + dA."""
    from scipy.sparse.linalg import splu

    from oracle import femoracle as fo

    cfg = c3_cfg()
    rcfg, sd = rb.meshprep(dict(cfg))
    det, phi = rb.run(rcfg)
    jn, _ = rb.jac(sd, phi, rcfg["deldotdel"], rcfg["elem"], rcfg["evol"])
    rng = np.random.default_rng(17)
    nodes = np.sort(rng.choice(cfg["node"].shape[0], 64, replace=False))
    out = dict(nodes=nodes, detval=det, jn_cols=jn[:, nodes], sd=sd, phi_rows=phi[nodes])
    del jn
    # oracle model with (mua, D) per node: mus = 1 / (3 D) - mua (g = 0)
    ocfg, _ = fo.meshprep(dict(cfg))
    ddd = fo.deldotdel(ocfg["node"], ocfg["elem"], ocfg["evol"])
    prop0 = ocfg["prop"]
    mua0 = prop0[:, 0].copy()
    D0 = 1.0 / (3.0 * (prop0[:, 0] + prop0[:, 1]))

    def prop_of(mua, D):
        p = prop0.copy()
        p[:, 0] = mua
        p[:, 1] = 1.0 / (3.0 * D) - mua
        return p

    A = fo.femlhs(dict(ocfg, prop=prop_of(mua0, D0)), ddd).tocsr()
    rhs, _, _, _ = fo.femrhs(ocfg)
    R = rhs.toarray()
    ns = cfg["srcpos"].shape[0]
    lu = splu(A.tocsc())
    F = lu.solve(R)
    fs, fd = F[:, :ns], F[:, ns:]
    det0 = R[:, ns:].T @ fs
    pt = prop_of(mua0 * 1.1, D0)
    At = fo.femlhs(dict(ocfg, prop=pt), ddd)
    target = R[:, ns:].T @ splu(At.tocsc()).solve(R[:, :ns])
    del At

    def loss(d):
        return 0.5 * np.sum((np.log(d) - np.log(target)) ** 2)

    def det_pert(mua, D):
        dA = (fo.femlhs(dict(ocfg, prop=prop_of(mua, D)), ddd).tocsr() - A).tocoo()
        S = np.unique(np.concatenate([dA.row, dA.col]))
        pos = {v: i for i, v in enumerate(S)}
        dSS = np.zeros((S.size, S.size))
        np.add.at(dSS, ([pos[v] for v in dA.row], [pos[v] for v in dA.col]), dA.data)
        E = np.zeros((A.shape[0], S.size))
        E[S, np.arange(S.size)] = 1.0
        G = lu.solve(E)[S]
        corr = np.linalg.solve(np.eye(S.size) + dSS @ G, dSS @ fs[S])
        return det0 - fd[S].T @ corr

    fd_mua = np.zeros(nodes.size)
    fd_D = np.zeros(nodes.size)
    for i, n in enumerate(nodes):
        h = 1e-4 * mua0[n]
        mp, mm = mua0.copy(), mua0.copy()
        mp[n] += h
        mm[n] -= h
        fd_mua[i] = (loss(det_pert(mp, D0)) - loss(det_pert(mm, D0))) / (2 * h)
        h = 1e-4 * D0[n]
        dp, dm = D0.copy(), D0.copy()
        dp[n] += h
        dm[n] -= h
        fd_D[i] = (loss(det_pert(mua0, dp)) - loss(det_pert(mua0, dm))) / (2 * h)
    out.update(fd_mua=fd_mua, fd_D=fd_D, oracle_det0=det0, target=target)
    np.savez_compressed(os.path.join(HERE, "c3_contract.npz"), **out)


def c2_case(rb):
    """The 3M-tet forward (box 100 x 100 x 50 mm at 1 mm), 4 of its 64 sources
    and 4 of its 64 detectors, through the reference's femsolve(method='cg',
    tol=1e-10) (solver.py:717-754): detval[4 det, 4 src] = rhs_det^T phi_src."""
    from redbirdpy_b200.meshgen import kuhn_box, grid_optodes

    node, elem = kuhn_box([100, 100, 50], 1)
    src = grid_optodes([15, 85], [15, 85], 8)
    det = grid_optodes([15, 85], [15, 85], 8, offset=(5, 5))
    isrc = np.array([0, 9, 36, 63])
    idet = np.array([0, 9, 36, 63])  # each 7 mm from its source, up to 99 mm from the others
    cfg = dict(node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
               seg=np.ones(elem.shape[0], dtype=np.int32), srcpos=src[isrc], srcdir=np.array([[0, 0, 1.0]]),
               detpos=det[idet], detdir=np.array([[0, 0, 1.0]]), omega=0.0)
    cfg, sd = rb.meshprep(cfg)
    A = rb.femlhs(cfg, cfg["deldotdel"])
    rhs, loc, bary, optode = rb.femrhs(cfg, sd)
    R = rhs.toarray() if hasattr(rhs, "toarray") else np.asarray(rhs)
    x, flag = rb.femsolve(A, R[:, :4], method="cg", tol=1e-10, maxiter=20000)
    dv = R[:, 4:].T @ x
    # the same at tol 1e-14: CG's residual criterion is global, so the small
    # far-field detector values need the tighter tolerance to settle
    x14, flag14 = rb.femsolve(A, R[:, :4], method="cg", tol=1e-14, maxiter=40000)
    dv14 = R[:, 4:].T @ x14
    rr = np.linalg.norm(R[:, :4] - A @ x14, axis=0) / np.linalg.norm(R[:, :4], axis=0)
    np.savez_compressed(os.path.join(HERE, "c2_contract.npz"), isrc=isrc, idet=idet, detval=dv, flag=flag,
                        detval14=dv14, flag14=flag14, relres14=rr, loc=loc, bary=bary)


def c5_case(rb):
    """8 of the 256 batched instances (batch_boxes(256, seed=2)), each through
    the reference's meshprep + run on its own."""
    from redbirdpy_b200.meshgen import batch_boxes

    cfgs = batch_boxes(256, seed=2)
    pick = np.array([0, 37, 74, 111, 148, 185, 222, 255])
    dets, shapes = [], []
    for i in pick:
        c, _ = rb.meshprep(dict(cfgs[i]))
        d, _ = rb.run(c)
        d = np.atleast_2d(d)
        dets.append(d.ravel())
        shapes.append(d.shape)
    np.savez_compressed(os.path.join(HERE, "c5_contract.npz"), pick=pick, shapes=np.array(shapes),
                        detval=np.concatenate(dets))


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref = args[0] if args else "/root/reference"
    rb = load_reference(ref)
    if "--only-multiwl" in sys.argv:
        multi_wavelength(rb)
        print("golden fixture written to", HERE)
        return
    if "--recon" in sys.argv:
        multiwl_gn(rb)
        dualmesh_gn(rb)
        rb.forward.HAS_NUMBA = False  # complex Jacobian needs the numpy branch
        reform_gn(rb, "logphase")
        reform_gn(rb, "reim")
        rb.forward.HAS_NUMBA = True
        print("reconstruction fixtures written to", HERE)
        return
    if "--wide" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "wide_cw.npz"), **wide_case(rb, 0.0))
        rb.forward.HAS_NUMBA = False  # complex Jacobian needs the numpy branch
        np.savez_compressed(os.path.join(HERE, "wide_fd.npz"), **wide_case(rb, 2 * np.pi * 1e8))
        rb.forward.HAS_NUMBA = True
        print("wide-field fixtures written to", HERE)
        return
    if "--contract" in sys.argv:
        for name, fn in (("c5", c5_case), ("c3", c3_case), ("c2", c2_case)):
            if "--" + name in sys.argv or not any(a in sys.argv for a in ("--c2", "--c3", "--c5")):
                fn(rb)
                print(name, "contract fixture written to", HERE, flush=True)
        return
    multi_wavelength(rb)
    np.savez_compressed(os.path.join(HERE, "c1_cw.npz"), **run_case(rb, c1_cfg()))
    np.savez_compressed(os.path.join(HERE, "c1_fd.npz"),
                        **run_case(rb, c1_cfg(2 * np.pi * 1e8), with_jac=False))
    np.savez_compressed(os.path.join(HERE, "nodal_cw.npz"), **run_case(rb, nodal_cfg()))
    rb.forward.HAS_NUMBA = False  # complex Jacobian needs the numpy branch
    np.savez_compressed(os.path.join(HERE, "nodal_fd.npz"),
                        **run_case(rb, nodal_cfg(2 * np.pi * 1e8)))
    rb.forward.HAS_NUMBA = True

    # element-based properties (one row per tet) on the c1 mesh
    cfg = c1_cfg()
    rng = np.random.default_rng(3)
    ne = cfg["elem"].shape[0]
    cfg["prop"] = np.column_stack([rng.uniform(0.005, 0.02, ne), rng.uniform(0.5, 1.5, ne),
                                   rng.uniform(0, 0.2, ne), np.full(ne, 1.37)])
    cfg.pop("seg")
    cfg, sd = rb.meshprep(cfg)
    cfg["omega"] = 2 * np.pi * 5e7
    A = rb.femlhs(cfg, cfg["deldotdel"])
    np.savez_compressed(os.path.join(HERE, "c1_elemprop_fd.npz"), prop=cfg["prop"],
                        omega=cfg["omega"], reff=cfg["reff"], **csr_fields("A", A))

    # Gauss-Newton: data from a +10% mua perturbation, two iterations
    cfg = nodal_cfg()
    cfg, sd = rb.meshprep(cfg)
    truth = cfg["prop"].copy()
    truth[:, 0] *= 1.1
    tcfg = dict(cfg)
    tcfg["prop"] = truth
    det0, _ = rb.run(tcfg)
    recon = {"prop": cfg["prop"].copy()}
    prop0 = cfg["prop"].copy()
    newrecon, resid, _, updates, jm, det, _ = rb.run(cfg, recon, det0, sd, maxiter=2,
                                                     lambda_=0.05, report=False)
    np.savez_compressed(os.path.join(HERE, "nodal_gn.npz"), prop0=prop0, detphi0=det0,
                        prop_out=newrecon["prop"], resid=resid,
                        dmu0=updates[0]["mua"], dmu1=updates[1]["mua"], jn=jm["mua"], det=det)

    # reginv / matreform / normalize_diag on seeded dense inputs
    rng = np.random.default_rng(7)
    Ju = rng.standard_normal((24, 300))
    ru = rng.standard_normal(24)
    Jo = rng.standard_normal((60, 20))
    ro = rng.standard_normal(60)
    Jc = rng.standard_normal((10, 40)) + 1j * rng.standard_normal((10, 40))
    y0 = rng.standard_normal(10) + 1j * rng.standard_normal(10)
    y1 = rng.standard_normal(10) + 1j * rng.standard_normal(10)
    H = rng.standard_normal((8, 8))
    Hn, di = rb.recon._normalize_diag(H @ H.T)
    Ar, rr, nb = rb.matreform(Jc, y0, y1, "real")
    Al, rl, nl = rb.matreform(Jc, y0, y1, "logphase")
    Ae, re_, ne_ = rb.matreform(Jc, y0, y1, "reim")
    np.savez_compressed(
        os.path.join(HERE, "dense_recon.npz"), Ju=Ju, ru=ru, Jo=Jo, ro=ro, Jc=Jc, y0=y0, y1=y1, H=H,
        under=rb.reginvunder(Ju, ru, 0.1), over=rb.reginvover(Jo, ro, 0.1), reginv_u=rb.reginv(Ju, ru, 0.3),
        Hn=Hn, di=di, Ar=Ar, rr=rr, Al=Al, rl=rl, Ae=Ae, re=re_,
    )
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

"""Generate the golden fixtures by running the reference redbirdpy itself.

Usage (in a container that has the reference sources)::

    python tests/golden/make_golden.py [/path/to/redbirdpy-checkout]

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


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref = args[0] if args else "/root/reference"
    rb = load_reference(ref)
    if "--only-multiwl" in sys.argv:
        multi_wavelength(rb)
        print("golden fixture written to", HERE)
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

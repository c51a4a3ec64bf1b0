"""The CPU oracle against golden fixtures produced by the reference itself."""

import numpy as np
import pytest
from scipy import sparse

from oracle import femoracle as fo
from oracle.tsearch import tsearchn


def cfg_from(g, keep_prep=False):
    cfg = dict(node=g["node"], elem=g["elem"], prop=g["prop"], srcpos=g["srcpos"],
               srcdir=np.array([[0, 0, 1.0]]), detpos=g["detpos"], detdir=np.array([[0, 0, 1.0]]),
               omega=float(g["omega"]))
    if "seg" in g:
        cfg["seg"] = g["seg"]
    if keep_prep:
        for k in ("face", "area", "evol", "reff", "deldotdel"):
            cfg[k] = g[k]
        cfg["isreoriented"] = True
    return cfg


@pytest.mark.parametrize("case", ["c1_cw", "c1_fd", "nodal_cw", "nodal_fd"])
def test_meshprep_matches_reference(golden, case):
    g = golden(case)
    cfg, sd = fo.meshprep(cfg_from(g))
    assert np.array_equal(cfg["elem"], g["elem"])
    assert np.array_equal(cfg["face"], g["face"])
    np.testing.assert_allclose(cfg["area"], g["area"], rtol=1e-14)
    np.testing.assert_allclose(cfg["evol"], g["evol"], rtol=1e-14)
    assert abs(cfg["reff"] - float(g["reff"])) < 1e-15
    np.testing.assert_allclose(cfg["deldotdel"], g["deldotdel"], rtol=1e-11, atol=1e-13 * np.abs(g["deldotdel"]).max())
    assert np.array_equal(sd, g["sd"])


@pytest.mark.parametrize("case", ["c1_cw", "c1_fd", "nodal_cw", "nodal_fd"])
def test_femlhs_matches_reference(golden, case):
    g = golden(case)
    cfg = cfg_from(g, keep_prep=True)
    A = fo.femlhs(cfg, g["deldotdel"])
    assert np.array_equal(A.indptr, g["A_indptr"])
    assert np.array_equal(A.indices, g["A_indices"])
    assert A.indices.dtype == np.int32 and A.indptr.dtype == np.int32
    err = np.abs(A.data - g["A_data"]).max() / np.abs(g["A_data"]).max()
    assert err < 1e-13


def test_femlhs_elemprop_fd_matches_reference(golden):
    g, m = golden("c1_elemprop_fd"), golden("c1_cw")
    cfg = cfg_from(m, keep_prep=True)
    cfg.pop("seg")
    cfg["prop"], cfg["omega"] = g["prop"], float(g["omega"])
    ddd = fo.deldotdel(cfg["node"], cfg["elem"], cfg["evol"])
    A = fo.femlhs(cfg, ddd)
    assert np.array_equal(A.indices, g["A_indices"]) and np.array_equal(A.indptr, g["A_indptr"])
    assert np.abs(A.data - g["A_data"]).max() / np.abs(g["A_data"]).max() < 1e-13


@pytest.mark.parametrize("case", ["c1_cw", "nodal_cw", "nodal_fd"])
def test_forward_and_jac_match_reference(golden, case):
    g = golden(case)
    cfg = cfg_from(g, keep_prep=True)
    rhs, loc, bary, pts = fo.femrhs(cfg)
    np.testing.assert_array_equal(loc, g["loc"])
    np.testing.assert_allclose(bary, g["bary"], atol=1e-14)
    np.testing.assert_allclose(rhs.toarray(), g["rhs"], atol=1e-14)
    det, phi = fo.runforward(cfg)
    np.testing.assert_allclose(det, g["detval"], rtol=1e-10)
    np.testing.assert_allclose(phi, g["phi"], rtol=1e-9, atol=1e-12 * np.abs(g["phi"]).max())
    if "jn" in g:
        jn, je = fo.jac(g["sd"], g["phi"], cfg["elem"], cfg["evol"])
        np.testing.assert_allclose(jn, g["jn"], rtol=1e-12, atol=1e-14 * np.abs(g["jn"]).max())
        np.testing.assert_allclose(je, g["je"], rtol=1e-12, atol=1e-14 * np.abs(g["je"]).max())


def test_c1_detval_known_answer(golden):
    # survey-time numbers of the reference on this workload
    np.testing.assert_allclose(golden("c1_cw")["detval"].ravel(), [9.6445e-4] * 2, rtol=1e-4)
    d = golden("c1_fd")["detval"].ravel()
    np.testing.assert_allclose(d, [9.3836e-4 - 1.8850e-4j] * 2, rtol=1e-4)
    assert golden("c1_cw")["A_indices"].size == 15067


def test_dense_recon_matches_reference(golden):
    g = golden("dense_recon")
    np.testing.assert_allclose(fo.reginvunder(g["Ju"], g["ru"], 0.1), g["under"], rtol=1e-10)
    np.testing.assert_allclose(fo.reginvover(g["Jo"], g["ro"], 0.1), g["over"], rtol=1e-10)
    np.testing.assert_allclose(fo.reginv(g["Ju"], g["ru"], 0.3), g["reginv_u"], rtol=1e-10)
    H = g["H"] @ g["H"].T
    Hn, di = fo.normalize_diag(H)
    np.testing.assert_allclose(Hn, g["Hn"], rtol=1e-14)
    np.testing.assert_allclose(di, g["di"], rtol=1e-14)
    for form, a, r in (("real", "Ar", "rr"), ("logphase", "Al", "rl"), ("reim", "Ae", "re")):
        A, rhs, _ = fo.matreform(g["Jc"], g["y0"], g["y1"], form)
        np.testing.assert_allclose(A, g[a], rtol=1e-14)
        np.testing.assert_allclose(rhs, g[r], rtol=1e-14)


def test_gn_matches_reference(golden):
    g, m = golden("nodal_gn"), golden("nodal_cw")
    cfg = cfg_from(m, keep_prep=True)
    cfg["prop"] = g["prop0"].copy()
    recon = {"prop": g["prop0"].copy()}
    recon, resid, _, upd, jn, det, _ = fo.runrecon(cfg, recon, g["detphi0"], maxiter=2, lambda_=0.05)
    np.testing.assert_allclose(resid, g["resid"], rtol=1e-8)
    np.testing.assert_allclose(upd[0]["mua"], g["dmu0"], rtol=1e-7, atol=1e-9 * np.abs(g["dmu0"]).max())
    np.testing.assert_allclose(recon["prop"], g["prop_out"], rtol=1e-9)


def test_tsearch_outside_and_ties():
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([2, 2, 2], 1)
    loc, bary = tsearchn(node, elem, np.array([[0.5, 0.5, 0.5], [5, 5, 5], [1.0, 1.0, 1.0]]))
    assert np.isnan(loc[1]) and np.all(np.isnan(bary[1]))
    assert not np.isnan(loc[0]) and abs(bary[0].sum() - 1) < 1e-14 and bary[0].min() >= -1e-9
    # a shared vertex: the lowest-index element that contains it
    e0 = elem - 1
    contains = [k for k in range(len(elem)) if 13 in e0[k]]
    assert loc[2] == contains[0] + 1


@pytest.mark.parametrize("case", ["wide_cw", "wide_fd"])
def test_wide_field_matches_reference(golden, case):
    """Wide-field pattern columns (cfg['widesrc'] / cfg['widedet']) in the
    RHS, the pair table and the readout, against the reference's run."""
    g = golden(case)
    cfg = cfg_from(g)
    cfg["widesrc"], cfg["widedet"] = g["widesrc"], g["widedet"]
    cfg, sd = fo.meshprep(cfg)
    assert np.array_equal(sd, g["sd"])
    rhs, loc, bary, _ = fo.femrhs(cfg)
    np.testing.assert_allclose(rhs.toarray(), g["rhs"], rtol=1e-13, atol=1e-15)
    np.testing.assert_array_equal(np.isnan(loc), np.isnan(g["loc"]))
    np.testing.assert_allclose(loc[~np.isnan(loc)], g["loc"][~np.isnan(g["loc"])])
    det, phi = fo.runforward(cfg)
    assert det.shape == g["detval"].shape
    np.testing.assert_allclose(det, g["detval"], rtol=1e-9)
    jn, _ = fo.jac(sd, phi, cfg["elem"], cfg["evol"])
    np.testing.assert_allclose(jn, g["jn"], rtol=1e-8, atol=1e-12 * np.abs(g["jn"]).max())

"""GPU parity of the Gauss-Newton pieces: the tcgen05 Gram kernel against
FP64 numpy, the regularised solves against the reference's reginv*, and the
device GN loop against the reference's runrecon (golden fixtures)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import redbirdpy_b200 as rbb  # noqa: E402
from redbirdpy_b200 import engine  # noqa: E402
from redbirdpy_b200._lib import RedbirdError  # noqa: E402

from test_gpu_forward import cfg_from  # noqa: E402


@pytest.mark.parametrize("M,K", [(8, 40), (300, 1000), (513, 2048), (1024, 4100)])
# tf32x3 removes the input rounding; what remains is the tensor cores' own
# FP32 accumulation (~2e-5 relative per 4096-long partial sum, measured).
# The partial sums are drained into FP64 every 4096 K-elements, so the error
# does not grow with K.
@pytest.mark.parametrize("precision,tol", [("tf32", 3e-3), ("tf32x3", 6e-5)])
def test_gram_tensor_cores(M, K, precision, tol):
    rng = np.random.default_rng(M + K)
    A = rng.standard_normal((M, K))
    J, Kc = rbb.recon._device_rows(A)
    H, _ = engine.gram(J, Kc, 0.5, precision)
    H = H.cpu().numpy()
    A32 = A.astype(np.float32).astype(np.float64)
    ref = 0.5 * (A32 @ A32.T)
    err = np.abs(H - ref).max() / np.abs(ref).max()
    assert err < tol, err
    assert np.array_equal(H, H.T)


def test_gram_long_k_accuracy():
    """K ~ 1e5 (Jacobian-like rows of mixed sign and decaying scale)."""
    rng = np.random.default_rng(1)
    M, K = 256, 100003
    A = rng.standard_normal((M, K)) * np.exp(-np.linspace(0, 8, K))[None, :]
    J, Kc = rbb.recon._device_rows(A)
    A32 = A.astype(np.float32).astype(np.float64)
    ref = A32 @ A32.T
    for precision, tol in (("tf32", 3e-3), ("tf32x3", 6e-5)):
        J2 = J.clone()
        H, _ = engine.gram(J2, Kc, 1.0, precision)
        err = np.abs(H.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err < tol, (precision, err)


@pytest.mark.parametrize("precision,tol", [("tf32", 3e-3), ("tf32x3", 6e-5), ("bf16", 1e-3)])
def test_gram_segments_in_order(precision, tol):
    """Several tiles and three K segments of 65536: the persistent launch adds
    segment s of a tile only after segment s - 1 (items running at once wait
    on each other); the result is the same on every run."""
    rng = np.random.default_rng(7)
    M, K = 520, 140001
    A = rng.standard_normal((M, K)) * np.exp(-np.linspace(0, 4, K))[None, :]
    if precision == "bf16":
        J, Kc, Ar = _bf16_rows(A)
        args = ()
    else:
        J, Kc = rbb.recon._device_rows(A)
        Ar = A.astype(np.float32).astype(np.float64)
        args = (precision,)
    H1, _ = engine.gram(J.clone(), Kc, 1.0, *args)
    H2, _ = engine.gram(J.clone(), Kc, 1.0, *args)
    H1, H2 = H1.cpu().numpy(), H2.cpu().numpy()
    ref = Ar @ Ar.T
    assert np.abs(H1 - ref).max() / np.abs(ref).max() < tol
    assert np.array_equal(H1, H2)
    assert np.array_equal(H1, H1.T)


@pytest.mark.parametrize("precision", ["tf32", "tf32x3", "bf16"])
def test_gram_staged_slabs_bit_identical(precision):
    """Rows longer than 1 MB take the staged path (compact copies of each
    65536-column slab): the same bits as the products formed in place, and
    within the tolerance of the FP64 product."""
    from redbirdpy_b200 import _lib
    rng = np.random.default_rng(11)
    M, K = (200, 600001) if precision == "bf16" else (300, 300001)  # rows of 1.2 MB
    A = rng.standard_normal((M, K)) * np.exp(-np.linspace(0, 4, K))[None, :]
    if precision == "bf16":
        J, Kc, Ar = _bf16_rows(A)
        args = ()
    else:
        J, Kc = rbb.recon._device_rows(A)
        Ar = A.astype(np.float32).astype(np.float64)
        args = (precision,)
    ldj = J.shape[1]
    assert _lib.lib().rb_gram_stage_bytes(M, Kc, ldj, 2 if precision == "bf16" else 4,
                                          int(precision == "tf32x3")) > 0
    Hs, lo = engine.gram(J, Kc, 1.0, *args)  # staged (J is left as hi for tf32x3)
    wb = _lib.lib().rb_gram_work_bytes()
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    Hp = torch.empty_like(Hs)
    if precision == "bf16":
        engine.call("rb_gram_bf16", engine.ptr(J), M, Kc, ldj, 1.0, engine.ptr(Hp), M, engine.ptr(work), wb,
                    engine.stream())
    else:
        engine.call("rb_gram", engine.ptr(J), engine.ptr(lo), M, Kc, ldj, 1.0, engine.ptr(Hp), M,
                    engine.ptr(work), wb, engine.stream())
    Hs, Hp = Hs.cpu().numpy(), Hp.cpu().numpy()
    assert np.array_equal(Hs, Hp)
    ref = Ar @ Ar.T
    tol = {"tf32": 3e-3, "tf32x3": 6e-5, "bf16": 1e-3}[precision]
    assert np.abs(Hs - ref).max() / np.abs(ref).max() < tol


def test_reginv_matches_reference(golden):
    g = golden("dense_recon")
    for got, ref in ((rbb.reginvunder(g["Ju"], g["ru"], 0.1), g["under"]),
                     (rbb.reginvover(g["Jo"], g["ro"], 0.1), g["over"]),
                     (rbb.reginv(g["Ju"], g["ru"], 0.3), g["reginv_u"])):
        assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-6
    # TF32 single pass for the normal matrix: the FP64 refinement over the
    # FP32 rows takes it to the same accuracy
    d = rbb.reginvunder(g["Ju"], g["ru"], 0.1, precision="tf32")
    assert np.abs(d - g["under"]).max() / np.abs(g["under"]).max() < 1e-6
    # without refinement the factor's own solution carries TF32 rounding
    J, K = rbb.recon._device_rows(g["Ju"])
    d0 = engine.reginv_under_device(J, K, g["ru"], 0.1, 1.0, "tf32", refine=0).cpu().numpy()
    assert 1e-6 < np.abs(d0 - g["under"]).max() / np.abs(g["under"]).max() < 5e-3


def test_matreform_matches_reference(golden):
    g = golden("dense_recon")
    for form, a, r in (("real", "Ar", "rr"), ("logphase", "Al", "rl"), ("reim", "Ae", "re")):
        A, rhs, _ = rbb.matreform(g["Jc"], g["y0"], g["y1"], form)
        np.testing.assert_allclose(A, g[a], rtol=1e-14)
        np.testing.assert_allclose(rhs, g[r], rtol=1e-14)
    with pytest.raises(ValueError):
        rbb.matreform(g["Jc"], g["y0"], g["y1"], "nope")


@pytest.mark.parametrize("M", [5, 64, 65, 300, 1030, 1152, 1153, 2101, 4096])
def test_cholesky_and_solve(M):
    import ctypes

    rng = np.random.default_rng(M)
    B = rng.standard_normal((M, M + 7))
    A = B @ B.T + M * np.eye(M)
    b = rng.standard_normal(M)
    H = torch.as_tensor(A, device="cuda")
    work = torch.empty(engine._lib.lib().rb_cholesky_work_bytes(), dtype=torch.uint8, device="cuda")
    engine.call("rb_cholesky", engine.ptr(H), M, M, engine.ptr(work), work.numel(), engine.stream())
    L = np.tril(H.cpu().numpy())
    np.testing.assert_allclose(L, np.linalg.cholesky(A), rtol=1e-10, atol=1e-12 * np.abs(L).max())
    x = torch.as_tensor(b.copy(), device="cuda")
    cwb = engine._lib.lib().rb_chol_solve_work_bytes(M)
    cwork = torch.empty(cwb, dtype=torch.uint8, device="cuda")
    engine.call("rb_chol_solve", engine.ptr(H), M, M, engine.ptr(x), engine.ptr(cwork), cwb, engine.stream())
    np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(A, b), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("M,ldh,offset", [(1100, 1103, 0), (1100, 1104, 1), (1280, 1280, 1)])
def test_cholesky_strided_and_unaligned(M, ldh, offset):
    """A matrix inside a wider buffer (ldh > M, odd or even) and starting 8
    bytes past a 16-byte boundary: the trailing updates then copy the panel
    in 8-byte pieces; the factor and the solve match LAPACK's.  M = 1280 ends
    its last outer block exactly at M (the in-block update's 2-D mode)."""
    rng = np.random.default_rng(M + ldh + offset)
    B = rng.standard_normal((M, M + 5))
    A = B @ B.T + M * np.eye(M)
    b = rng.standard_normal(M)
    buf = torch.zeros(offset + M * ldh, dtype=torch.float64, device="cuda")
    H = buf[offset:].view(M, ldh)
    H[:, :M] = torch.as_tensor(A, device="cuda")
    assert (H.data_ptr() % 16 == 0) == (offset == 0)
    work = torch.empty(engine._lib.lib().rb_cholesky_work_bytes(), dtype=torch.uint8, device="cuda")
    engine.call("rb_cholesky", engine.ptr(H), M, ldh, engine.ptr(work), work.numel(), engine.stream())
    L = np.tril(H[:, :M].cpu().numpy())
    np.testing.assert_allclose(L, np.linalg.cholesky(A), rtol=1e-10, atol=1e-12 * np.abs(L).max())
    x = torch.as_tensor(b.copy(), device="cuda")
    cwb = engine._lib.lib().rb_chol_solve_work_bytes(M)
    cwork = torch.empty(cwb, dtype=torch.uint8, device="cuda")
    engine.call("rb_chol_solve", engine.ptr(H), M, ldh, engine.ptr(x), engine.ptr(cwork), cwb, engine.stream())
    np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(A, b), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("M,K", [(5, 3), (70, 1030), (1000, 4097)])
def test_gemv_passes_over_padded_rows(M, K):
    """J x and J^T y over FP32 (and BF16) rows padded to a multiple of 4
    with NaN past K: FP64 accumulation, the padding never read into a sum,
    the beta term applied."""
    rng = np.random.default_rng(M + K)
    ldj = (K + 3) // 4 * 4
    J = np.full((M, ldj), np.nan, dtype=np.float32)
    J[:, :K] = rng.standard_normal((M, K))
    x, y = rng.standard_normal(K), rng.standard_normal(M)
    Jd = torch.as_tensor(J, device="cuda")
    xd, yd = torch.as_tensor(x, device="cuda"), torch.as_tensor(y, device="cuda")
    Jk = J[:, :K].astype(np.float64)
    ref_n = Jk @ x
    np.testing.assert_allclose(engine.gemv_n(Jd, K, xd, 2.0).cpu().numpy(), 2.0 * ref_n, rtol=1e-11,
                               atol=1e-12 * np.abs(ref_n).max())
    out = torch.ones(M, dtype=torch.float64, device="cuda")
    engine.gemv_n(Jd, K, xd, 1.0, 3.0, out=out)
    np.testing.assert_allclose(out.cpu().numpy(), 3.0 + ref_n, rtol=1e-11, atol=1e-12 * np.abs(ref_n).max())
    ref_t = Jk.T @ y
    np.testing.assert_allclose(engine.gemv_t(Jd, K, yd, 0.5).cpu().numpy(), 0.5 * ref_t, rtol=1e-11,
                               atol=1e-12 * np.abs(ref_t).max())
    Jb = Jd.to(torch.bfloat16)
    Jbk = Jb.float().cpu().numpy()[:, :K].astype(np.float64)
    np.testing.assert_allclose(engine.gemv_n(Jb, K, xd).cpu().numpy(), Jbk @ x, rtol=1e-11,
                               atol=1e-12 * np.abs(ref_n).max())


@pytest.mark.parametrize("M,cond", [(300, 1e8), (1030, 1e10)])
def test_cholesky_solve_ill_conditioned(M, cond):
    """The solve multiplies by explicit inverses of the 64 x 64 diagonal
    blocks; on a graded spectrum (condition number 1e8-1e10, like J J^T +
    lambda I with a small relative lambda) its backward error stays at the
    level of LAPACK's: ||A x - b|| / (||A|| ||x||) within a small factor."""
    rng = np.random.default_rng(int(M + np.log10(cond)))
    Q, _ = np.linalg.qr(rng.standard_normal((M, M)))
    A = (Q * np.geomspace(1.0, 1.0 / cond, M)) @ Q.T
    A = 0.5 * (A + A.T)
    b = rng.standard_normal(M)
    H = torch.as_tensor(A, device="cuda")
    work = torch.empty(engine._lib.lib().rb_cholesky_work_bytes(), dtype=torch.uint8, device="cuda")
    engine.call("rb_cholesky", engine.ptr(H), M, M, engine.ptr(work), work.numel(), engine.stream())
    x = torch.as_tensor(b.copy(), device="cuda")
    cwb = engine._lib.lib().rb_chol_solve_work_bytes(M)
    cwork = torch.empty(cwb, dtype=torch.uint8, device="cuda")
    engine.call("rb_chol_solve", engine.ptr(H), M, M, engine.ptr(x), engine.ptr(cwork), cwb, engine.stream())
    x = x.cpu().numpy()
    xr = np.linalg.solve(A, b)

    def backward(v):
        return np.linalg.norm(A @ v - b) / (np.linalg.norm(A, 2) * np.linalg.norm(v))

    assert backward(x) <= 20 * max(backward(xr), 1e-16), (backward(x), backward(xr))


def test_cholesky_rejects_indefinite():
    A = np.eye(70)
    with pytest.raises(RedbirdError) as e:
        rbb.reginvunder(A, np.ones(70), -5.0)
    assert e.value.code == engine._lib.RB_ENOTSPD


@pytest.mark.parametrize("gram,tol", [("tf32x3", 2e-6), ("tf32", 2e-6)])
def test_runrecon_matches_reference(golden, gram, tol):
    """Two GN iterations against the reference's runrecon: the tensor-core
    normal matrix plus FP64 refinement over the FP32 Jacobian rows reach the
    reference's FP64 step to the FP32 rows' accuracy (measured 1.5e-7 and
    6.2e-7 for the two updates)."""
    g, m = golden("nodal_gn"), golden("nodal_cw")
    cfg = cfg_from(m)
    cfg["prop"] = g["prop0"].copy()
    recon = {"prop": g["prop0"].copy()}
    recon, resid, cfg, upd, J, det, phi = rbb.run(cfg, recon, g["detphi0"], m["sd"], maxiter=2, lambda_=0.05,
                                                  report=False, gram=gram)
    # resid[0] is the forward model alone; later entries carry the step's precision
    np.testing.assert_allclose(resid[0], g["resid"][0], rtol=1e-8)
    np.testing.assert_allclose(resid, g["resid"], rtol=tol)
    for k, key in enumerate(("dmu0", "dmu1")):
        ref = g[key]
        err = np.abs(upd[k]["mua"] - ref).max() / np.abs(ref).max()
        assert err < tol, (key, err)
    err = np.abs(recon["prop"][:, 0] - g["prop_out"][:, 0]).max() / np.abs(g["prop_out"][:, 0]).max()
    assert err < tol * 0.1
    # the final Jacobian is taken at the final (slightly different) estimate
    jref = g["jn"]
    assert np.linalg.norm(J["mua"] - jref) / np.linalg.norm(jref) < max(tol, 1e-3)


def test_runrecon_residual_decreases_fd_mua_and_d(golden):
    """Frequency domain, exact node-based Jacobians for mua and D: the
    residual drops over the iterations (test_integration.py:292-311)."""
    m = golden("nodal_fd")
    cfg = cfg_from(m)
    truth = cfg["prop"].copy()
    nn = truth.shape[0]
    bump = np.linalg.norm(cfg["node"] - np.array([20.0, 20.0, 6.0]), axis=1) < 8
    truth[bump, 0] *= 1.5
    cfg_t = dict(cfg)
    cfg_t.pop("_b200", None)
    cfg_t["prop"] = truth
    det0, _ = rbb.run(cfg_t)
    recon = {"prop": cfg["prop"].copy()}
    recon, resid, cfg, upd, J, det, phi = rbb.run(cfg, recon, det0, m["sd"], maxiter=4, lambda_=0.01, report=False,
                                                  param="mua+D", lambda_rule="maxdiag")
    assert resid[-1] < 0.5 * resid[0], resid
    assert "dcoeff" in upd[0] and upd[0]["mua"].shape == (nn,)


def _bf16_rows(A):
    """A (numpy) as BF16 device rows with a 16-byte row stride, and the
    FP64 values of the rounded entries."""
    M, K = A.shape
    ldj = (K + 7) // 8 * 8
    J = torch.zeros((M, ldj), dtype=torch.bfloat16, device="cuda")
    J[:, :K] = torch.as_tensor(A, dtype=torch.float32, device="cuda").to(torch.bfloat16)
    return J, K, J[:, :K].double().cpu().numpy()


@pytest.mark.parametrize("M,K", [(8, 40), (300, 1000), (513, 2048), (1024, 40000)])
def test_gram_bf16_tensor_cores(M, K):
    """BF16 rows through the kind::f16 MMA: against FP64 products of the same
    rounded entries (what remains is the FP32 accumulation)."""
    rng = np.random.default_rng(M + K)
    J, Kc, Ar = _bf16_rows(rng.standard_normal((M, K)))
    H, _ = engine.gram(J, Kc, 0.5)
    H = H.cpu().numpy()
    ref = 0.5 * (Ar @ Ar.T)
    assert np.abs(H - ref).max() / np.abs(ref).max() < 1e-3
    assert np.array_equal(H, H.T)
    # the other BF16 pieces of the GN step
    s = engine.sumsq(J, Kc).item()
    assert abs(s - (Ar ** 2).sum()) <= 1e-12 * (Ar ** 2).sum()
    y = rng.standard_normal(M)
    out = engine.gemv_t(J, Kc, torch.as_tensor(y, device="cuda"), 2.0).cpu().numpy()
    np.testing.assert_allclose(out, 2.0 * (Ar.T @ y), rtol=1e-10, atol=1e-12 * np.abs(Ar.T @ y).max())


@pytest.mark.parametrize("case", ["nodal_cw", "nodal_fd"])
def test_jacobian_bf16_rows(golden, case):
    g = golden(case)
    cfg = cfg_from(g)
    mesh = engine.mesh_of(cfg)
    phi = torch.as_tensor(g["phi"], device="cuda")
    sd = g["sd"]
    J32, K = engine.jacobian_matrix(mesh, phi, sd, ("mua", "D"), "exact")
    J16, K16 = engine.jacobian_matrix(mesh, phi, sd, ("mua", "D"), "exact", dtype=torch.bfloat16)
    assert K16 == K and J16.shape[1] % 8 == 0
    a, b = J32[:, :K].double(), J16[:, :K].double()
    assert (torch.abs(a - b) <= 2.0 ** -8 * torch.abs(a) + 1e-30).all()


@pytest.mark.parametrize("gram,tol", [("bf16", 2e-6), ("bf16_rows", 3e-2)])
def test_runrecon_bf16_matches_reference(golden, gram, tol):
    """'bf16': the product from a BF16 copy of the FP32 rows, refined over the
    FP32 rows (the reference's step to the FP32 rows' accuracy); 'bf16_rows':
    the rows themselves stored in BF16 (the rounded rows' step)."""
    g, m = golden("nodal_gn"), golden("nodal_cw")
    cfg = cfg_from(m)
    cfg["prop"] = g["prop0"].copy()
    recon = {"prop": g["prop0"].copy()}
    recon, resid, cfg, upd, J, det, phi = rbb.run(cfg, recon, g["detphi0"], m["sd"], maxiter=2, lambda_=0.05,
                                                  report=False, gram=gram)
    np.testing.assert_allclose(resid, g["resid"], rtol=max(tol, 1e-8) if gram == "bf16" else 1e-2)
    for k, key in enumerate(("dmu0", "dmu1")):
        ref = g[key]
        assert np.abs(upd[k]["mua"] - ref).max() / np.abs(ref).max() < tol, key


def _nodal_cfg(m, omega=0.0):
    cfg = cfg_from(m)
    cfg["omega"] = omega
    return cfg


def test_multiwavelength_chromophore_recon_matches_reference(golden):
    """Two wavelengths, chromophore parameters (hbo, hbr per node; water and
    lipids at the reference's defaults): two GN iterations against the
    reference's runrecon, with the extinction coefficients it used."""
    g, m = golden("multiwl_gn"), golden("nodal_cw")
    cfg = cfg_from(m, prepared=False)
    tmpl = np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]])
    cfg["prop"] = {"690": tmpl.copy(), "830": tmpl.copy()}
    cfg["param"] = {"hbo": g["hbo"].copy(), "hbr": g["hbr"].copy()}
    chroms = [str(c) for c in g["chroms"]]
    extin = {wv: {c: float(g["ext"][j, i]) for i, c in enumerate(chroms)} for j, wv in enumerate(("690", "830"))}
    cfg["extin"] = extin
    cfg, sd = rbb.meshprep(cfg)
    recon = {"param": {"hbo": g["hbo"].copy(), "hbr": g["hbr"].copy()}}
    det0 = {"690": g["det0_690"], "830": g["det0_830"]}
    recon, resid, cfg2, upd, J, det, phi = rbb.run(cfg, recon, det0, sd, maxiter=2, lambda_=0.05, report=False,
                                                  extin=extin)
    np.testing.assert_allclose(resid, g["resid"], rtol=1e-6)
    for k in range(2):
        for c in chroms:
            ref = g[f"upd{k}_{c}"]
            err = np.abs(upd[k][c] - ref).max() / np.abs(ref).max()
            assert err < 2e-6, (k, c, err)
    for c in ("hbo", "hbr"):
        scale = max(np.abs(g[f"upd0_{c}"]).max(), np.abs(g[f"upd1_{c}"]).max())
        np.testing.assert_allclose(recon["param"][c], g[c + "_out"], rtol=0, atol=4e-6 * scale)
    np.testing.assert_allclose(np.atleast_1d(cfg2["param"]["water"]), g["water_out"], rtol=1e-9)
    for wv in ("690", "830"):
        np.testing.assert_allclose(det[wv], g["det_" + wv], rtol=1e-6)


def test_dual_mesh_recon_matches_reference(golden):
    """Reconstruction on a coarse mesh (75 nodes) mapped onto the forward
    mesh: two GN iterations against the reference's runrecon."""
    g, m = golden("dualmesh_gn"), golden("nodal_cw")
    cfg = _nodal_cfg(m)
    recon = {"node": g["rnode"], "elem": g["relem"], "prop": g["rprop"].copy(), "mapid": g["mapid"],
             "mapweight": g["mapweight"]}
    recon, resid, _, upd, J, det, _ = rbb.run(cfg, recon, g["det0"], m["sd"], maxiter=2, lambda_=0.05,
                                              report=False)
    np.testing.assert_allclose(resid, g["resid"], rtol=1e-6)
    for k, key in enumerate(("dmu0", "dmu1")):
        err = np.abs(upd[k]["mua"] - g[key]).max() / np.abs(g[key]).max()
        assert err < 2e-6, (key, err)
    scale = max(np.abs(g["dmu0"]).max(), np.abs(g["dmu1"]).max())
    np.testing.assert_allclose(recon["prop"], g["prop_out"], rtol=0, atol=4e-6 * scale)


@pytest.mark.parametrize("form", ["logphase", "reim"])
def test_reform_recon_matches_reference(golden, form):
    """Frequency-domain GN with matreform 'logphase' / 'reim' in the device
    loop, against the reference's runrecon (two iterations)."""
    g, m = golden(f"reform_{form}"), golden("nodal_fd")
    cfg = _nodal_cfg(m, float(m["omega"]))
    cfg["prop"] = g["prop0"].copy()
    recon = {"prop": g["prop0"].copy()}
    recon, resid, _, upd, J, det, _ = rbb.run(cfg, recon, g["det0"], m["sd"], maxiter=2, lambda_=0.05,
                                              report=False, reform=form)
    np.testing.assert_allclose(resid, g["resid"], rtol=1e-6)
    for k, key in enumerate(("dmu0", "dmu1")):
        err = np.abs(upd[k]["mua"] - g[key]).max() / np.abs(g[key]).max()
        assert err < 2e-6, (key, err)


@pytest.mark.parametrize("case,param", [("nodal_cw", "mua"), ("nodal_fd", "mua+D")])
def test_runrecon_with_recomputed_jacobian_slabs(golden, case, param):
    """A GN loop whose Jacobian is never stored (node slabs recomputed on
    every pass: the Frobenius sum, the tensor-core product, each refinement
    residual and the update) against the same loop with J stored."""
    m = golden(case)
    out = {}
    for slab in (None, 97):
        cfg = cfg_from(m)
        truth = cfg["prop"].copy()
        bump = np.linalg.norm(cfg["node"] - np.array([20.0, 20.0, 6.0]), axis=1) < 8
        truth[bump, 0] *= 1.5
        cfg_t = dict(cfg)
        cfg_t.pop("_b200", None)
        cfg_t["prop"] = truth
        det0, _ = rbb.run(cfg_t)
        recon = {"prop": cfg["prop"].copy()}
        res = rbb.run(cfg, recon, det0, m["sd"], maxiter=2, lambda_=0.05, report=False, param=param,
                      jac_slab=slab)
        out[slab] = res
    (r0, s0, _, u0, J0, _, _), (r1, s1, _, u1, J1, _, _) = out[None], out[97]
    from redbirdpy_b200.engine import SlabJacobian

    assert isinstance(J1["mua"], SlabJacobian) and J1["mua"].passes >= 3
    np.testing.assert_allclose(s1, s0, rtol=1e-9)
    for a, b in zip(u0, u1):
        for key in a:
            e = np.abs(a[key] - b[key]).max() / np.abs(a[key]).max()
            assert e <= 1e-7, (key, e)
    np.testing.assert_allclose(r1["prop"], r0["prop"], rtol=1e-9)


@pytest.mark.parametrize("precision", ["tf32", "bf16", "bf16_of_fp32"])
def test_relative_lambda_uses_the_exact_diagonal(precision):
    """lam = 0.05 max diag(s J J^T) taken from the FP64 row sums of the stored
    rows, not from the tensor-core product: the refined update then equals
    the FP64 solution of the stored rows' system (TF32 or BF16 rows alike,
    and FP32 rows whose product comes from their BF16 copy)."""
    rng = np.random.default_rng(11)
    M, K = 300, 5000
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-2, 2, K))
    Jb = None
    if precision == "bf16":
        J, K_, Ad = _bf16_rows(A)
        gram_prec = "bf16"
    else:
        J = torch.zeros((M, (K + 3) // 4 * 4), dtype=torch.float32, device="cuda")
        J[:, :K] = torch.as_tensor(A, dtype=torch.float32, device="cuda")
        Ad = J[:, :K].double().cpu().numpy()
        gram_prec = "tf32" if precision == "tf32" else "bf16"
    if precision == "bf16_of_fp32":
        rows, tot, Jb = engine.row_sumsq(J, K, bf16_copy=True)
        np.testing.assert_array_equal(Jb[:, :K].float().cpu().numpy(),
                                      J[:, :K].to(torch.bfloat16).float().cpu().numpy())
        assert not Jb[:, K:].float().abs().sum().item()
    else:
        rows, tot = engine.row_sumsq(J, K)
    np.testing.assert_allclose(rows.cpu().numpy(), np.sum(Ad * Ad, axis=1), rtol=1e-12)
    np.testing.assert_allclose(float(tot.item()), np.sum(Ad * Ad), rtol=1e-12)
    s2 = 1.0 / float(tot.item())
    r = rng.standard_normal(M)
    info = {}
    got = engine.reginv_under_device(J, K, r, 0.0, s2, gram_prec, lam_rel=0.05, rowsq=rows, refine=12,
                                     info=info, Jb=Jb).cpu().numpy()
    H = s2 * Ad @ Ad.T
    lam = 0.05 * H.diagonal().max()
    y = np.linalg.solve(H + lam * np.eye(M), r)
    ref = s2 * Ad.T @ y
    assert abs(info["lam"] - lam) <= 1e-12 * lam
    assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max(), info

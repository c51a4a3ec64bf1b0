"""GPU parity of the forward path against the reference's own outputs
(golden fixtures) and the CPU oracle.  Tolerances: CSR indices bit-exact,
assembled values relative <= 1e-12 (FP64), detector values <= 1e-6 relative
after refinement."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import redbirdpy_b200 as rbb  # noqa: E402
from redbirdpy_b200 import engine  # noqa: E402
from oracle import femoracle as fo  # noqa: E402


def cfg_from(g, prepared=True):
    cfg = dict(node=g["node"].copy(), elem=g["elem"].copy(), prop=g["prop"].copy(), srcpos=g["srcpos"],
               srcdir=np.array([[0, 0, 1.0]]), detpos=g["detpos"], detdir=np.array([[0, 0, 1.0]]),
               omega=float(g["omega"]))
    if "seg" in g:
        cfg["seg"] = g["seg"]
    if prepared:
        for k in ("face", "area", "evol", "reff", "deldotdel"):
            cfg[k] = g[k]
        cfg["isreoriented"] = True
    return cfg


CASES = ["c1_cw", "c1_fd", "nodal_cw", "nodal_fd"]


@pytest.mark.parametrize("case", CASES)
def test_csr_pattern_bit_exact(golden, case):
    g = golden(case)
    m = engine.mesh_of(cfg_from(g))
    assert np.array_equal(m.indptr.cpu().numpy(), g["A_indptr"])
    assert np.array_equal(m.indices[: m.nnz].cpu().numpy(), g["A_indices"])


@pytest.mark.parametrize("case", CASES)
def test_femlhs_values(golden, case):
    g = golden(case)
    A = rbb.femlhs(cfg_from(g), g["deldotdel"])
    assert A.indices.dtype == np.int32 and A.indptr.dtype == np.int32
    assert np.array_equal(A.indptr, g["A_indptr"]) and np.array_equal(A.indices, g["A_indices"])
    rel = np.abs(A.data - g["A_data"]).max() / np.abs(g["A_data"]).max()
    assert rel <= 1e-12, rel
    # entrywise relative check as well (no entry is tiny in these matrices)
    assert np.max(np.abs(A.data - g["A_data"]) / np.abs(g["A_data"])) <= 1e-12


def test_femlhs_elemprop_complex(golden):
    g, m = golden("c1_elemprop_fd"), golden("c1_cw")
    cfg = cfg_from(m)
    cfg.pop("seg")
    cfg["prop"], cfg["omega"] = g["prop"], float(g["omega"])
    A = rbb.femlhs(cfg, None)
    assert np.array_equal(A.indices, g["A_indices"])
    assert np.abs(A.data - g["A_data"]).max() / np.abs(g["A_data"]).max() <= 1e-12


@pytest.mark.parametrize("case", CASES)
def test_femrhs(golden, case):
    g = golden(case)
    rhs, loc, bary, optode = rbb.femrhs(cfg_from(g))
    np.testing.assert_array_equal(loc, g["loc"])
    np.testing.assert_allclose(bary, g["bary"], atol=1e-13)
    np.testing.assert_allclose(rhs.toarray(), g["rhs"], atol=1e-13)
    np.testing.assert_allclose(optode, g["optode"], rtol=1e-15)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_runforward_detval(golden, case, precision):
    g = golden(case)
    det, phi = rbb.runforward(cfg_from(g), precision=precision)
    ref = g["detval"]
    assert det.shape == ref.shape and phi.shape == g["phi"].shape
    err = np.abs(det - ref) / np.abs(ref)
    assert err.max() <= 1e-6, err.max()
    perr = np.abs(phi - g["phi"]).max() / np.abs(g["phi"]).max()
    assert perr <= 1e-9, perr


def test_run_facade_and_meshprep(golden):
    g = golden("c1_cw")
    cfg = cfg_from(g, prepared=False)
    cfg, sd = rbb.meshprep(cfg)
    assert np.array_equal(cfg["elem"], g["elem"]) and np.array_equal(cfg["face"], g["face"])
    np.testing.assert_allclose(cfg["deldotdel"], g["deldotdel"], rtol=1e-10,
                               atol=1e-14 * np.abs(g["deldotdel"]).max())
    assert np.array_equal(sd, g["sd"])
    det, phi = rbb.run(cfg)
    np.testing.assert_allclose(det, g["detval"], rtol=1e-6)
    # known answer from the reference on this workload
    np.testing.assert_allclose(det.ravel(), [9.6445e-4] * 2, rtol=1e-4)


def test_femgetdet_drop_in(golden):
    g = golden("nodal_fd")
    cfg = cfg_from(g)
    rhs, loc, bary, _ = rbb.femrhs(cfg)
    d1 = rbb.femgetdet(g["phi"], cfg, rhs, loc, bary)
    d0 = fo.femgetdet(g["phi"], cfg, rhs)
    np.testing.assert_allclose(d1, d0, rtol=1e-12)
    np.testing.assert_allclose(rbb.femgetdet(g["phi"], cfg, rhs), d0, rtol=1e-12)


def spd(n, seed):
    rng = np.random.default_rng(seed)
    from scipy import sparse

    M = sparse.random(n, n, density=0.05, random_state=rng)
    A = (M @ M.T + 10 * sparse.eye(n)).tocsr()
    return A


def test_femsolve_spd_and_edge_cases():
    from scipy.sparse.linalg import spsolve

    A = spd(300, 1)
    rng = np.random.default_rng(2)
    b = rng.standard_normal((300, 5))
    b[:, 2] = 0.0  # zero column -> exact zeros (solver.py:568-581)
    x, flag = rbb.femsolve(A, b)
    assert flag == 0
    assert np.all(x[:, 2] == 0.0)
    ref = np.column_stack([spsolve(A.tocsc(), b[:, i]) if np.any(b[:, i]) else np.zeros(300) for i in range(5)])
    np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-13)
    # 1-D in -> 1-D out; residual as in test_solver.py:68-83
    x1, flag = rbb.femsolve(A, b[:, 0])
    assert x1.ndim == 1 and flag == 0
    assert np.linalg.norm(A @ x1 - b[:, 0]) / np.linalg.norm(b[:, 0]) < 1e-8
    # identity / diagonal known answers (test_solver.py:1660-1681)
    from scipy import sparse

    I = sparse.eye(50).tocsr()
    xi, _ = rbb.femsolve(I, np.arange(50.0))
    np.testing.assert_allclose(xi, np.arange(50.0), rtol=1e-14)
    D = sparse.diags(np.arange(1.0, 51.0)).tocsr()
    xd, _ = rbb.femsolve(D, np.ones(50))
    np.testing.assert_allclose(xd, 1.0 / np.arange(1.0, 51.0), rtol=1e-13)


def test_femsolve_complex_symmetric(golden):
    from scipy.sparse.linalg import splu

    g = golden("nodal_fd")
    from scipy import sparse

    A = sparse.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]))
    b = g["rhs"]
    for prec in ("mixed", "fp64"):
        x, flag = rbb.femsolve(A, b, precision=prec)
        ref = splu(A.tocsc()).solve(b.astype(complex))
        assert flag == 0
        assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-10


def test_femsolve_many_columns(golden):
    """More than one 128-column block."""
    from scipy import sparse
    from scipy.sparse.linalg import splu

    g = golden("c1_cw")
    A = sparse.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]))
    rng = np.random.default_rng(5)
    b = rng.standard_normal((A.shape[0], 130))
    x, flag = rbb.femsolve(A, b)
    ref = splu(A.tocsc()).solve(b)
    assert flag == 0
    assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-11


def test_femsolve_iteration_cap_flag(golden):
    from scipy import sparse

    g = golden("c1_cw")
    A = sparse.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]))
    b = g["rhs"]
    x, flag = rbb.femsolve(A, b, method="cg", maxiter=3, max_outer=1, tol=1e-14)
    assert flag == 1


def test_large_pattern_vs_scipy():
    """51x51x26 box (375k tets): pattern and values against the oracle's scipy assembly."""
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([100, 100, 50], 2)
    rng = np.random.default_rng(0)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn), np.zeros(nn),
                            np.full(nn, 1.37)])
    cfg = dict(node=node, elem=elem, prop=prop, srcpos=np.array([[50, 50, 0.0]]), srcdir=np.array([[0, 0, 1.0]]),
               detpos=np.array([[60, 50, 0.0]]), omega=2 * np.pi * 1e8)
    cfg, _ = rbb.meshprep(cfg)
    A = rbb.femlhs(cfg, None)
    ocfg = dict(cfg)
    R = fo.femlhs(ocfg, fo.deldotdel(cfg["node"], cfg["elem"], cfg["evol"]))
    assert A.nnz == 972876
    assert np.array_equal(A.indptr, R.indptr) and np.array_equal(A.indices, R.indices)
    assert np.abs(A.data - R.data).max() / np.abs(R.data).max() <= 1e-12


@pytest.mark.parametrize("case", CASES)
def test_assembly_tables(golden, case):
    """The contributor tables against a numpy restatement, and the assembly
    through them against the scan of every incident tet."""
    g = golden(case)
    cfg = cfg_from(g)
    m = engine.mesh_of(cfg)
    eptr, elist = m.eptr.cpu().numpy(), m.elist.cpu().numpy()
    indptr, indices = m.indptr.cpu().numpy(), m.indices[: m.nnz].cpu().numpy()
    elem = m.elem.cpu().numpy().reshape(-1, 4)
    if np.diff(eptr).max() > 32 or np.diff(indptr).max() > 255:
        assert m.inc_slot is None and m.struct.inc_slot is None
        return
    inc = m.inc_slot[: 4 * m.ne].cpu().numpy().view(np.uint32)
    msk = m.slot_mask[: m.nnz].cpu().numpy().view(np.uint32)
    want_msk = np.zeros(m.nnz, dtype=np.uint32)
    for n in range(m.nn):
        cols = indices[indptr[n]:indptr[n + 1]]
        for u, e in enumerate(elist[eptr[n]:eptr[n + 1]]):
            pos = np.searchsorted(cols, elem[e])
            assert np.array_equal(cols[pos], elem[e])
            assert inc[eptr[n] + u] == sum(int(p) << (8 * j) for j, p in enumerate(pos))
            want_msk[indptr[n] + pos] |= np.uint32(1 << u)
    assert np.array_equal(msk, want_msk)
    optics = engine.Optics.from_cfg(m, cfg)
    a = engine.assemble(m, optics)
    b = engine.assemble(m, optics, tables=False)
    va, vb = a.val64[: m.nnz].cpu().numpy(), b.val64[: m.nnz].cpu().numpy()
    assert np.abs(va - vb).max() <= 1e-14 * np.abs(vb).max()


@pytest.mark.parametrize("cplx", [False, True])
def test_femsolve_breakdown_is_a_flag_not_a_hang(cplx):
    """(p, A p) = 0 on the first step (indefinite / complex-symmetric
    D^-1 A): the column stops with the breakdown flag 2, like the reference's
    non-zero iterative-solver flags, and the call returns."""
    from scipy import sparse

    dt = complex if cplx else float
    A = sparse.diags(np.array([1.0, -1.0], dtype=dt)).tocsr()
    x, flag = rbb.femsolve(A, np.array([1.0, 1.0]), maxiter=50)
    assert flag == 2


def test_femsolve_nan_matrix_flags_breakdown():
    from scipy import sparse

    A = sparse.diags(np.array([2.0, np.nan, 3.0])).tocsr()
    x, flag = rbb.femsolve(A, np.ones(3), maxiter=50)
    assert flag == 2


def _spd_dense_row(n, seed):
    """SPD matrix whose row/column 7 is full (a row group of more than 256
    values), n not a multiple of the 8-row groups."""
    from scipy import sparse

    rng = np.random.default_rng(seed)
    M = sparse.random(n, n, density=0.03, random_state=rng).tolil()
    M[7, :] = rng.uniform(0.1, 0.2, n)
    M = M.tocsr()
    return (M @ M.T + 20 * sparse.eye(n)).tocsr()


@pytest.mark.parametrize("k", [32, 64, 128])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_femsolve_row_group_spmm(golden, k, precision):
    """32, 64 and 128 columns: the FP64 solves take the row-group SpMM (bulk
    copies of each neighbour row once per 4-row group), the mixed ones the
    per-row SpMM (padded gather batches at 128 columns).  FEM matrices (real
    and complex symmetric) and a ragged SPD matrix with a dense row (a group of
    more than 256 values), against SuperLU."""
    from scipy import sparse
    from scipy.sparse.linalg import splu

    rng = np.random.default_rng(k)
    mats = []
    for case in ("c1_cw", "nodal_fd"):
        g = golden(case)
        mats.append(sparse.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"])))
    mats.append(_spd_dense_row(301, k))
    for A in mats:
        b = rng.standard_normal((A.shape[0], k))
        b[:, 3] = 0.0
        x, flag = rbb.femsolve(A, b, precision=precision)
        ref = splu(A.tocsc()).solve(b.astype(A.dtype))
        assert flag == 0
        assert np.all(x[:, 3] == 0)
        assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-11


@pytest.mark.parametrize("k", [33, 37, 66, 70, 127])
def test_femsolve_column_counts_outside_the_lane_layout(golden, k):
    """Odd counts above 32 and counts 2 mod 4 above 64 (the vector kernels'
    lane layout covers 32 / 64 / 128 of those): the solve runs on a copy
    padded with zero columns.  Against SuperLU, mixed and FP64, cold and warm;
    rb_spmm at the same counts against scipy."""
    import ctypes

    from scipy import sparse
    from scipy.sparse.linalg import splu

    g = golden("nodal_fd")
    A = sparse.csr_matrix((g["A_data"], g["A_indices"], g["A_indptr"]))
    rng = np.random.default_rng(k)
    b = rng.standard_normal((A.shape[0], k))
    b[:, k - 1] = 0.0
    ref = splu(A.tocsc()).solve(b.astype(complex))
    for precision in ("mixed", "fp64"):
        x, flag = rbb.femsolve(A, b, precision=precision)
        assert flag == 0
        assert np.all(x[:, k - 1] == 0)
        assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-11, precision
    mat = engine.DeviceMatrix.from_scipy(A)
    B = torch.as_tensor(b, device="cuda")
    x_cold, i_cold = engine.solve(mat, B)
    x_warm, i_warm = engine.solve(mat, B, x0=x_cold)
    assert i_warm["iters"] == 0 and torch.equal(x_warm, x_cold)
    # rb_spmm (FP64 complex values) at the same column count
    X = torch.as_tensor(rng.standard_normal((A.shape[0], k)) + 1j * rng.standard_normal((A.shape[0], k)),
                        device="cuda")
    Y = torch.empty_like(X)
    from redbirdpy_b200 import _lib

    _lib.call("rb_spmm", ctypes.byref(mat.struct), _lib.RB_C128, _lib.ptr(X), _lib.ptr(Y), k, _lib.stream())
    yref = A @ X.cpu().numpy()
    assert np.abs(Y.cpu().numpy() - yref).max() / np.abs(yref).max() < 1e-13


def test_pinned_result_pool_never_overwrites_live_arrays():
    """runforward copies phi into reused page-locked buffers: a buffer comes
    back only after the array from it, and every view of it, is gone."""
    pool = engine.PinnedPool(per_shape=2, min_bytes=0)
    t = torch.arange(8, dtype=torch.float64, device="cuda")
    a = pool.to_numpy(t)
    b = pool.to_numpy(t + 100)
    assert a[0] == 0 and b[0] == 100  # two live arrays, two buffers
    c = pool.to_numpy(t + 200)  # both pooled buffers in use: a plain copy
    assert a[0] == 0 and b[0] == 100 and c[0] == 200
    view = b[2:]
    del a, b
    d = pool.to_numpy(t + 300)  # reuses a's buffer, never b's (view alive)
    e = pool.to_numpy(t + 400)
    assert view[0] == 102 and d[0] == 300 and e[0] == 400
    assert not np.shares_memory(d, view) and not np.shares_memory(e, view)


def test_label_properties_expand_on_device(golden):
    """prop[seg] on the device (rb_prop_from_labels) gives the reference's
    matrix for the labelled workload, including labels out of range (clipped)."""
    g = golden("c1_cw")
    cfg = cfg_from(g)
    A = rbb.femlhs(cfg, g["deldotdel"])
    assert np.abs(A.data - g["A_data"]).max() / np.abs(g["A_data"]).max() <= 1e-12
    mesh = engine.mesh_of(cfg)
    seg = np.array([-3, 0, 1, 7] * (mesh.ne // 4) + [1] * (mesh.ne % 4))
    cfg2 = dict(cfg, seg=seg, prop=np.array([[0.02, 2.0, 0.5, 1.37], [0.01, 1.0, 0.0, 1.37]]))
    o = engine.Optics.from_cfg(mesh, cfg2)
    idx = np.clip(seg, 0, 1)
    np.testing.assert_array_equal(o.mua.cpu().numpy(), cfg2["prop"][idx, 0])
    np.testing.assert_array_equal(o.musp.cpu().numpy(), cfg2["prop"][idx, 1] * (1 - cfg2["prop"][idx, 2]))


def test_femsolve_warm_start(golden):
    """An initial guess (the Gauss-Newton warm start) changes the iteration
    count, not the answer: from the solution itself the solve ends at once."""
    from redbirdpy_b200 import engine as eng

    g = golden("nodal_fd")
    cfg = cfg_from(g)
    mesh = eng.mesh_of(cfg)
    opt = eng.locate_optodes(mesh, cfg)
    B = opt.rhs(mesh)
    mat = eng.assemble(mesh, eng.Optics.from_cfg(mesh, cfg))
    x_cold, i_cold = eng.solve(mat, B)
    x_same, i_same = eng.solve(mat, B, x0=x_cold)
    assert i_same["iters"] == 0 and i_same["flag"] == 0
    assert torch.equal(x_same, x_cold)
    x_pert = x_cold * (1 + 0.01 * torch.rand_like(x_cold.real))
    x_warm, i_warm = eng.solve(mat, B, x0=x_pert)
    assert i_warm["flag"] == 0 and i_warm["iters"] < i_cold["iters"]
    assert (torch.abs(x_warm - x_cold).max() / torch.abs(x_cold).max()).item() < 1e-12
    with pytest.raises(ValueError):
        eng.solve(mat, B, x0=x_cold[:, :3])


def test_multi_wavelength_forward_matches_reference(golden):
    """cfg['prop'] keyed by wavelength: meshprep's per-wavelength reff and
    runforward's per-wavelength detval / phi, as the reference returns them."""
    g = golden("nodal_multiwl")
    cfg = dict(node=g["node"].copy(), elem=g["elem"].copy(), srcpos=g["srcpos"], srcdir=np.array([[0, 0, 1.0]]),
               detpos=g["detpos"], detdir=np.array([[0, 0, 1.0]]), omega=float(g["omega"]),
               prop={"690": g["prop_690"].copy(), "830": g["prop_830"].copy()})
    cfg, sd = rbb.meshprep(cfg)
    assert isinstance(cfg["reff"], dict) and isinstance(sd, dict)
    det, phi = rbb.run(cfg)
    assert set(det) == {"690", "830"} and set(phi) == {"690", "830"}
    for wv in ("690", "830"):
        assert cfg["reff"][wv] == pytest.approx(float(g["reff_" + wv]), rel=1e-14)
        ref = g["detval_" + wv]
        assert det[wv].shape == ref.shape
        assert np.max(np.abs(det[wv] - ref) / np.abs(ref)) <= 1e-6
        assert np.abs(phi[wv] - g["phi_" + wv]).max() / np.abs(g["phi_" + wv]).max() <= 1e-9
    # one wavelength's matrix through femlhs(cfg, ddd, wavelength)
    A = rbb.femlhs(cfg, cfg["deldotdel"], "830")
    assert A.shape == (cfg["node"].shape[0],) * 2


@pytest.mark.parametrize("case", ["wide_cw", "wide_fd"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_wide_field_forward_and_jacobian(golden, case, precision):
    """Wide-field sources and detectors (pattern columns given in cfg)
    against the reference's meshprep / femrhs / run / jac."""
    g = golden(case)
    cfg = cfg_from(g, prepared=False)
    cfg["widesrc"], cfg["widedet"] = g["widesrc"], g["widedet"]
    cfg, sd = rbb.meshprep(cfg)
    np.testing.assert_array_equal(sd, g["sd"])
    rhs, loc, bary, _ = rbb.femrhs(cfg)
    np.testing.assert_allclose(rhs.toarray(), g["rhs"], rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(np.isnan(loc), np.isnan(g["loc"]))
    ok = ~np.isnan(g["loc"])
    np.testing.assert_array_equal(loc[ok], g["loc"][ok])
    det, phi = rbb.run(cfg, precision=precision)
    assert det.shape == g["detval"].shape
    err = np.abs(det - g["detval"]) / np.abs(g["detval"])
    assert err.max() <= 1e-6, err.max()
    assert np.abs(phi - g["phi"]).max() / np.abs(g["phi"]).max() <= 1e-9
    # the drop-in readout from femrhs's outputs gives the same detector values
    det2 = rbb.femgetdet(phi, cfg, rhs, loc, bary)
    np.testing.assert_allclose(det2, det, rtol=1e-12)
    jn, _ = rbb.jac(sd, phi, cfg["deldotdel"], cfg["elem"], cfg["evol"])
    scale = np.abs(g["jn"]).max()
    assert np.abs(jn - g["jn"]).max() <= 1e-8 * scale


@pytest.mark.parametrize("case", ["c1_cw", "nodal_cw"])
def test_device_meshprep_bit_exact(golden, case):
    """Reorientation, boundary faces (order and orientation), face areas, tet
    and node volumes from the device kernels, against the reference's own
    meshprep fallbacks (exact equality)."""
    g = golden(case)
    cfg = cfg_from(g, prepared=False)
    cfg, _ = rbb.meshprep(cfg)
    np.testing.assert_array_equal(cfg["elem"], g["elem"])
    np.testing.assert_array_equal(cfg["face"], g["face"])
    np.testing.assert_array_equal(cfg["area"], g["area"])
    np.testing.assert_array_equal(cfg["evol"], g["evol"])
    np.testing.assert_array_equal(cfg["nvol"], g["nvol"])


def test_device_meshprep_matches_host_restatement_on_a_shuffled_mesh():
    """A renumbered, jittered box (tets in random order and orientation):
    the device kernels give the host restatement's arrays exactly."""
    from redbirdpy_b200 import utility as ut
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([20, 16, 12], 2)
    rng = np.random.default_rng(9)
    node = node + rng.uniform(-0.3, 0.3, node.shape)
    perm = rng.permutation(node.shape[0])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    node = node[perm]
    elem = inv[elem - 1] + 1
    elem = elem[rng.permutation(elem.shape[0])]
    flip = rng.random(elem.shape[0]) < 0.5
    elem[flip, 2], elem[flip, 3] = elem[flip, 3].copy(), elem[flip, 2].copy()
    cfg = dict(node=node, elem=elem.copy(), prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
               srcpos=np.array([[10, 8, 0.0]]), srcdir=np.array([[0, 0, 1.0]]), detpos=np.array([[12, 8, 0.0]]))
    cfg, _ = rbb.meshprep(cfg)
    r = ut._reorient(node, elem)
    np.testing.assert_array_equal(cfg["elem"], r)
    np.testing.assert_array_equal(cfg["face"], ut._volface(r, node.shape[0]))
    np.testing.assert_array_equal(cfg["area"], ut._elemvolume(node, cfg["face"]))
    np.testing.assert_allclose(cfg["evol"], ut._elemvolume(node, r), rtol=1e-15)
    np.testing.assert_allclose(cfg["nvol"], ut._nodevolume(node.shape[0], r, cfg["evol"]), rtol=1e-14)


def test_femsolve_non_finite_rhs_column_is_flagged():
    """A NaN right-hand-side column ends with flag 2, not as converged; the
    other columns still solve."""
    from scipy.sparse.linalg import splu

    A = spd(200, 3)
    B = np.random.default_rng(1).standard_normal((200, 4))
    B[5, 2] = np.nan
    x, flag = rbb.femsolve(A, B)
    assert flag == 2
    ref = splu(A.tocsc()).solve(np.nan_to_num(B[:, [0, 1, 3]]))
    np.testing.assert_allclose(x[:, [0, 1, 3]], ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())

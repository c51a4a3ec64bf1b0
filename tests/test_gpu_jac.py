"""GPU parity of the adjoint Jacobians: the reference-semantics mua Jacobian
against the reference's own jac output, and the exact node-based mua / D
Jacobians against central finite differences of the GPU forward model."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import redbirdpy_b200 as rbb  # noqa: E402
from redbirdpy_b200 import engine  # noqa: E402
from redbirdpy_b200.forward import forward_device  # noqa: E402

from test_gpu_forward import cfg_from  # noqa: E402
from oracle import femoracle as fo  # noqa: E402


@pytest.mark.parametrize("case", ["c1_cw", "nodal_cw", "nodal_fd"])
def test_jac_drop_in_matches_reference(golden, case):
    g = golden(case)
    jn, je = rbb.jac(g["sd"], g["phi"], g["deldotdel"], g["elem"], g["evol"])
    assert jn.dtype == g["jn"].dtype and jn.shape == g["jn"].shape and je.shape == g["je"].shape
    np.testing.assert_allclose(jn, g["jn"], rtol=1e-10, atol=1e-13 * np.abs(g["jn"]).max())
    np.testing.assert_allclose(je, g["je"], rtol=1e-10, atol=1e-13 * np.abs(g["je"]).max())
    if not np.iscomplexobj(jn):
        # absorption lowers every reading: the rows are dominated by negative
        # sensitivities (test_integration.py:236-244 checks the sign on its mesh)
        assert np.all(jn.sum(axis=1) < 0)


@pytest.mark.parametrize("case", ["nodal_cw", "nodal_fd"])
def test_jac_fp32_rows(golden, case):
    g = golden(case)
    cfg = cfg_from(g)
    mesh = engine.mesh_of(cfg)
    phi = torch.as_tensor(g["phi"], device="cuda")
    J = engine.jacobian(mesh, phi, g["sd"], "mua", out_dtype=torch.float32).cpu().numpy()
    ref = g["jn"]
    err = np.linalg.norm(J - ref) / np.linalg.norm(ref)
    assert err <= 1e-6, err


def test_jac_inactive_pairs(golden):
    g = golden("nodal_cw")
    sd = g["sd"].copy()
    sd[[1, 5, 6], 2] = 0
    jn, _ = rbb.jac(sd, g["phi"], g["deldotdel"], g["elem"], g["evol"])
    keep = sd[:, 2] == 1
    np.testing.assert_allclose(jn, g["jn"][keep], rtol=1e-10, atol=1e-13 * np.abs(g["jn"]).max())


def _oracle_detvals(cfg):
    """Detector values from the CPU oracle (SuperLU), so that the finite
    differences carry direct-solver accuracy."""
    det, _ = fo.runforward(dict(cfg))
    return det.ravel()  # det-major order, like sd rows


@pytest.mark.parametrize("omega", [0.0, 2 * np.pi * 1e8])
def test_exact_jacobians_vs_central_fd(golden, omega):
    g = golden("nodal_cw")
    cfg = cfg_from(g)
    cfg["omega"] = omega
    mesh = engine.mesh_of(cfg)
    # fields from the oracle's direct solve, so that the check isolates the
    # Jacobian kernels from the iterative solver's far-field accuracy
    _, phi_ref = fo.runforward({k: v for k, v in cfg.items() if k != "_b200"})
    phi = torch.as_tensor(phi_ref, device="cuda")
    sd = g["sd"]
    jm = engine.jacobian(mesh, phi, sd, "mua_nodal", out_dtype=torch.float64).cpu().numpy()
    jd = engine.jacobian(mesh, phi, sd, "D", out_dtype=torch.float64).cpu().numpy()
    prop = cfg["prop"].copy()
    D = 1.0 / (3.0 * (prop[:, 0] + prop[:, 1] * (1 - prop[:, 2])))
    ocfg = {k: v for k, v in cfg.items() if k != "_b200"}
    rng = np.random.default_rng(11)
    nodes = rng.choice(mesh.nn, 12, replace=False)
    for n in nodes:
        # d/dmua at fixed musp = dA/dmua|_D + dD/dmua dA/dD ; d/dmus = dD/dmus dA/dD
        for col, expect in ((0, jm[:, n] - 3 * D[n] ** 2 * jd[:, n]), (1, -3 * D[n] ** 2 * jd[:, n])):
            # h = 1e-3 relative: below that the FD quotient is dominated by the
            # rounding of the direct solves (checked on the CPU against h = 1e-2)
            h = 1e-3 * prop[n, col]
            p1, p2 = prop.copy(), prop.copy()
            p1[n, col] += h
            p2[n, col] -= h
            fd = (_oracle_detvals(dict(ocfg, prop=p1)) - _oracle_detvals(dict(ocfg, prop=p2))) / (2 * h)
            scale = np.abs(fd).max()
            assert np.abs(fd - expect).max() <= 1e-5 * scale, (n, col, np.abs(fd - expect).max() / scale)


def _loss(det, target):
    return 0.5 * torch.sum(torch.abs(torch.log(det) - torch.log(target)) ** 2)


@pytest.mark.parametrize("omega", [0.0, 2 * np.pi * 1e8])
@pytest.mark.parametrize("resolve", [False, True])
def test_adjoint_gradient_vs_fd_and_jacobian(golden, omega, resolve):
    """autograd backward of 0.5 ||log(det) - log(target)||^2 through the
    hand-written adjoint (per-node mua and D), target from a +10% mua
    perturbation: against central differences (h = 1e-4 relative, FP64
    solves) on random nodes, and against J^T g with the explicit Jacobians."""
    from redbirdpy_b200.adjoint import DeviceModel, detector_values

    g = golden("nodal_cw")
    cfg = cfg_from(g)
    cfg["omega"] = omega
    prop = cfg["prop"]
    model = DeviceModel(cfg, precision="fp64")
    mua0 = torch.as_tensor(prop[:, 0].copy(), device="cuda")
    d0 = torch.as_tensor(1.0 / (3.0 * (prop[:, 0] + prop[:, 1] * (1 - prop[:, 2]))), device="cuda")
    with torch.no_grad():
        target = detector_values(model, mua0 * 1.1, d0)
    mua = mua0.clone().requires_grad_(True)
    dco = d0.clone().requires_grad_(True)
    loss = _loss(detector_values(model, mua, dco, resolve=resolve), target)
    loss.backward()
    gm, gd = mua.grad.cpu().numpy(), dco.grad.cpu().numpy()
    # J^T g identity (exact up to rounding)
    det = detector_values(model, mua0, d0).detach().requires_grad_(True)
    _loss(det, target).backward()
    gdet = det.grad
    phi, _ = model.fields(mua0, d0)
    ns, nd = model.opt.nsrc, model.opt.ndet
    sd = np.column_stack([np.tile(np.arange(ns), nd), ns + np.repeat(np.arange(nd), ns), np.ones(ns * nd)])
    for what, got in (("mua_nodal", gm), ("D", gd)):
        J = engine.jacobian(model.mesh, phi, sd, what, out_dtype=torch.float64)  # rows det-major
        gv = gdet.reshape(-1)  # det[d, s] -> row d * ns + s
        ref = (torch.conj(gv)[:, None] * J).sum(0).real.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
    # central differences of the FP64 forward model
    rng = np.random.default_rng(3)
    for n in rng.choice(model.mesh.nn, 6, replace=False):
        for vec, grad in ((mua0, gm), (d0, gd)):
            h = 1e-4 * float(vec[n])
            vp, vm = vec.clone(), vec.clone()
            vp[n] += h
            vm[n] -= h
            with torch.no_grad():
                if vec is mua0:
                    lp = _loss(detector_values(model, vp, d0), target).item()
                    lm = _loss(detector_values(model, vm, d0), target).item()
                else:
                    lp = _loss(detector_values(model, mua0, vp), target).item()
                    lm = _loss(detector_values(model, mua0, vm), target).item()
            fd = (lp - lm) / (2 * h)
            scale = np.abs(grad).max()
            assert abs(fd - grad[n]) <= 1e-5 * scale, (n, fd, grad[n], scale)


def test_batched_instances_match_per_instance_models():
    """Uneven box instances as one block-diagonal system (one assembly, one
    solve, one adjoint contraction) give each instance's detector values and
    gradients as its own model does."""
    from redbirdpy_b200.adjoint import BatchModel, DeviceModel, detector_values
    from redbirdpy_b200.meshgen import batch_boxes

    cfgs = [rbb.meshprep(c)[0] for c in batch_boxes(6, seed=5, dims=(12.0, 24.0), spacings=(3.0, 4.0), nopt=(2, 5))]
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-6)):
        bm = BatchModel(cfgs, precision=prec)
        mua = torch.as_tensor(np.concatenate([c["prop"][:, 0] for c in cfgs]), device="cuda").requires_grad_(True)
        dco = torch.as_tensor(np.concatenate([1.0 / (3.0 * (c["prop"][:, 0] + c["prop"][:, 1])) for c in cfgs]),
                              device="cuda").requires_grad_(True)
        det = detector_values(bm, mua, dco)
        parts = bm.split(det)
        # log-amplitude misfit (coarse instances can give slightly negative
        # far-field values: the P1 mass term makes A a non-M-matrix there)
        loss = sum(0.5 * torch.sum(torch.log(torch.abs(p)) ** 2) for p in parts)
        loss.backward()
        gms, gds = bm.node_slices(mua.grad), bm.node_slices(dco.grad)
        for i, c in enumerate(cfgs):
            m = DeviceModel(c, precision="fp64")
            mu = torch.as_tensor(c["prop"][:, 0].copy(), device="cuda").requires_grad_(True)
            dc = torch.as_tensor(1.0 / (3.0 * (c["prop"][:, 0] + c["prop"][:, 1])), device="cuda").requires_grad_(True)
            d1 = detector_values(m, mu, dc)
            assert d1.shape == parts[i].shape
            err = (torch.abs(parts[i] - d1) / torch.abs(d1)).max().item()
            assert err <= tol, (prec, i, err)
            (0.5 * torch.sum(torch.log(torch.abs(d1)) ** 2)).backward()
            for got, ref in ((gms[i], mu.grad), (gds[i], dc.grad)):
                e = (torch.abs(got - ref).max() / torch.abs(ref).max()).item()
                assert e <= max(tol, 1e-9) * 10, (prec, i, e)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_convergence_is_per_instance(precision):
    """Two instances whose right-hand sides differ by 1e8 in scale: each one
    reaches the tolerance against its own ||b_i|| (a whole-column criterion
    would let the small one stop at 1e8 times the tolerance), and each
    matches its own solve; statuses and per-(instance, column) residuals
    come back."""
    from redbirdpy_b200.meshgen import kuhn_box
    from scipy.sparse.linalg import splu

    from oracle import femoracle as fo

    parts = []
    for dims, h, mua in (([20, 16, 12], 2.0, 0.01), ([16, 16, 10], 2.0, 0.03)):
        node, elem = kuhn_box(dims, h)
        cfg = dict(node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [mua, 1.0, 0, 1.37]]),
                   seg=np.ones(elem.shape[0], dtype=np.int32), srcpos=np.array([[8, 8, 0.0]]),
                   srcdir=np.array([[0, 0, 1.0]]), detpos=np.array([[10, 8, 0.0]]), omega=0.0)
        parts.append(rbb.meshprep(cfg)[0])
    A = [fo.femlhs(dict(c), fo.deldotdel(c["node"], c["elem"], c["evol"])) for c in parts]
    n = [a.shape[0] for a in A]
    from scipy import sparse

    Ab = sparse.block_diag(A, format="csr")
    rng = np.random.default_rng(3)
    B = rng.standard_normal((sum(n), 4))
    B[n[0]:] *= 1e-8
    mat = engine.DeviceMatrix.from_scipy(Ab)
    inst = engine.Instances([0, n[0], n[0] + n[1]], "cuda")
    Bd = torch.as_tensor(B, device="cuda")
    X, info = engine.solve(mat, Bd, precision=precision, tol=1e-10, instances=inst, coarse=False, groups=None)
    assert info["flag"] == 0
    assert list(info["inst_status"]) == [0, 0]
    assert info["inst_relres"].shape == (2, 4) and info["inst_relres"].max() <= 1e-10
    X = X.cpu().numpy()
    for i, (a, lo) in enumerate(zip(A, (0, n[0]))):
        xi = X[lo:lo + n[i]]
        bi = B[lo:lo + n[i]]
        rel = np.linalg.norm(bi - a @ xi, axis=0) / np.linalg.norm(bi, axis=0)
        assert rel.max() <= 1e-10, (i, rel)
        ref = splu(a.tocsc()).solve(bi)
        assert np.abs(xi - ref).max() <= 1e-8 * np.abs(ref).max(), i


def _masked_log_loss(own, tgt):
    def loss(det):
        d = torch.where(own, det, torch.ones_like(det))
        t = torch.where(own, tgt, torch.ones_like(tgt))
        return 0.5 * torch.sum((torch.log(torch.abs(d)) - torch.log(torch.abs(t))) ** 2)
    return loss


def test_captured_batch_step_matches_checked_solves():
    """Forward + adjoint of a batch replayed from one CUDA graph (fixed solve
    budget, no host checks) against the same step with checked solves, at
    the captured properties and at new ones copied in before a replay."""
    from redbirdpy_b200.adjoint import BatchModel, CapturedStep, detector_values
    from redbirdpy_b200.meshgen import batch_boxes

    cfgs = [rbb.meshprep(c)[0] for c in batch_boxes(6, seed=5, dims=(12.0, 24.0), spacings=(3.0, 4.0), nopt=(2, 5))]
    bm = BatchModel(cfgs, precision="mixed")
    mua0 = torch.as_tensor(np.concatenate([c["prop"][:, 0] for c in cfgs]), device="cuda")
    d0 = torch.as_tensor(np.concatenate([1.0 / (3.0 * (c["prop"][:, 0] + c["prop"][:, 1])) for c in cfgs]),
                         device="cuda")
    with torch.no_grad():
        tgt = detector_values(bm, mua0 * 1.1, d0)
    loss_fn = _masked_log_loss(bm.own, tgt)

    def checked(mua, dco):
        m = mua.clone().requires_grad_(True)
        d = dco.clone().requires_grad_(True)
        det = detector_values(bm, m, d)
        loss = loss_fn(det)
        loss.backward()
        return loss.detach(), det.detach(), m.grad, d.grad

    step = CapturedStep(bm, loss_fn, mua0, d0)
    assert step.budget[0] >= 1 and step.budget[1] >= 8
    for scale in (1.0, 1.05):
        got = [t.clone() for t in step(mua0 * scale, d0)]
        assert int(step.status.max().item()) == 0
        step_kw = bm.solve_kw
        bm.solve_kw = step.solve_kw_checked
        ref = checked(mua0 * scale, d0)
        bm.solve_kw = step_kw
        for a, b in zip(got, ref):
            e = (torch.abs(a - b).max() / torch.abs(b).max()).item()
            assert e <= 1e-8, (scale, e)
    step.release()


@pytest.mark.parametrize("omega", [0.0, 2 * np.pi * 1e8])
@pytest.mark.parametrize("params", [("mua",), ("mua", "D")])
def test_jacobian_rows_on_tensor_cores(omega, params):
    """The pair products on tcgen05 (TF32 hi/lo split) against the SIMT
    products and the FP64 rows: full source x detector grid, FP32 rows
    (complex fields split into real and imaginary blocks), the whole mesh and
    node ranges that start off a multiple of 4."""
    from redbirdpy_b200.meshgen import kuhn_box, grid_optodes

    node, elem = kuhn_box([40, 40, 20], 2)
    rng = np.random.default_rng(4)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn), np.zeros(nn),
                            np.full(nn, 1.37)])
    cfg = dict(node=node, elem=elem, prop=prop, srcpos=grid_optodes([8, 32], [8, 32], 4),
               srcdir=np.array([[0, 0, 1.0]]), detpos=grid_optodes([8, 32], [8, 32], 4, offset=(2, 2)),
               detdir=np.array([[0, 0, 1.0]]), omega=omega)
    cfg, sd = rbb.meshprep(cfg)
    _, phi, _, _, _ = forward_device(cfg, precision="fp64")
    mesh = engine.mesh_of(cfg)
    mode = "exact" if len(params) > 1 else "reference"
    try:
        engine.jac_tensor_cores(False)
        Js, K = engine.jacobian_matrix(mesh, phi, sd, params, mode)
        Js = Js[:, :K].double().cpu().numpy()
        engine.jac_tensor_cores(True)
        Jt, _ = engine.jacobian_matrix(mesh, phi, sd, params, mode)
        Jt = Jt[:, :K].double().cpu().numpy()
    finally:
        engine.jac_tensor_cores(False)
    # FP64 rows of the same quantities
    ref = []
    for p in params:
        w = "mua" if (p == "mua" and mode == "reference") else ("mua_nodal" if p == "mua" else "D")
        J64 = engine.jacobian(mesh, phi, sd, w, out_dtype=torch.float64).cpu().numpy()
        ref.append(np.concatenate([J64.real, J64.imag]) if np.iscomplexobj(J64) else J64)
    ref = np.concatenate(ref, axis=1)
    scale = np.linalg.norm(ref)
    assert np.linalg.norm(Jt - ref) <= 1e-6 * scale, np.linalg.norm(Jt - ref) / scale
    assert np.linalg.norm(Js - ref) <= 1e-6 * scale
    assert np.abs(Jt - Js).max() <= 1e-5 * np.abs(ref).max()
    # node ranges (slabs) starting off a multiple of 4, on the tensor cores
    op = engine.SlabJacobian(mesh, phi, sd, params, mode, width=1001)
    for a, b in list(op.ranges())[:3]:
        try:
            engine.jac_tensor_cores(True)
            S, ks = op.slab(a, b)
        finally:
            engine.jac_tensor_cores(False)
        S = S[:, :ks].double().cpu().numpy()
        c = b - a
        want = np.concatenate([Jt[:, p * nn + a:p * nn + b] for p in range(len(params))], axis=1)
        assert S.shape == (Jt.shape[0], len(params) * c)
        np.testing.assert_array_equal(S, want)


def test_solve_autotuner_and_lane_layouts():
    """Every lane layout the autotuner tries solves the batch to the same
    solution; the tuner returns one of its candidates and caches it per size
    bucket."""
    from redbirdpy_b200.adjoint import BatchModel
    from redbirdpy_b200.meshgen import batch_boxes

    cfgs = [rbb.meshprep(c)[0] for c in batch_boxes(6, seed=5, dims=(12.0, 24.0), spacings=(3.0, 4.0), nopt=(2, 5))]
    bm = BatchModel(cfgs, precision="mixed")
    mua = torch.as_tensor(np.concatenate([c["prop"][:, 0] for c in cfgs]), device="cuda")
    dco = torch.as_tensor(np.concatenate([1.0 / (3.0 * (c["prop"][:, 0] + c["prop"][:, 1])) for c in cfgs]),
                          device="cuda")
    mat = engine.assemble(bm.mesh, bm.optics(mua, dco))
    ref, _ = engine.solve(mat, bm.B, **bm.solve_kw)
    for lanes in engine.SolveTuner.LANES:
        X, info = engine.solve(mat, bm.B, **dict(bm.solve_kw, spmm_lanes=lanes))
        assert info["flag"] == 0 and list(np.unique(info["inst_status"])) == [0]
        assert (X - ref).abs().max().item() <= 1e-10 * ref.abs().max().item(), lanes
    kw = bm.tune(mua, dco)
    assert (kw["spmm_lanes"], kw["check_every"]) in [(a, b) for a in engine.SolveTuner.LANES
                                                     for b in engine.SolveTuner.CHECKS]
    key = engine.solve_tuner.bucket(mat, bm.B.shape[1], bm.solve_kw)
    assert key in engine.solve_tuner.cache and len(engine.solve_tuner.timings[key]) >= 1
    assert engine.solve_tuner.options(mat, bm.B, **bm.solve_kw) is engine.solve_tuner.cache[key]


@pytest.mark.parametrize("omega", [0.0, 2 * np.pi * 1e8])
def test_jacobian_rows_formed_in_fp64(omega):
    """FP32 rows whose products are formed in FP64 equal the FP64 rows
    rounded to FP32 (only the storage rounds)."""
    from redbirdpy_b200.meshgen import kuhn_box, grid_optodes

    node, elem = kuhn_box([40, 40, 20], 2)
    rng = np.random.default_rng(6)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn), np.zeros(nn),
                            np.full(nn, 1.37)])
    cfg = dict(node=node, elem=elem, prop=prop, srcpos=grid_optodes([8, 32], [8, 32], 4),
               srcdir=np.array([[0, 0, 1.0]]), detpos=grid_optodes([8, 32], [8, 32], 4, offset=(2, 2)),
               detdir=np.array([[0, 0, 1.0]]), omega=omega)
    cfg, sd = rbb.meshprep(cfg)
    _, phi, _, _, _ = forward_device(cfg, precision="fp64")
    mesh = engine.mesh_of(cfg)
    J, K = engine.jacobian_matrix(mesh, phi, sd, ("mua", "D"), "exact", acc64=True)
    J = J[:, :K].double().cpu().numpy()
    ref = []
    for w in ("mua_nodal", "D"):
        J64 = engine.jacobian(mesh, phi, sd, w, out_dtype=torch.float64).cpu().numpy()
        ref.append(np.concatenate([J64.real, J64.imag]) if np.iscomplexobj(J64) else J64)
    ref = np.concatenate(ref, axis=1)
    np.testing.assert_array_equal(J, ref.astype(np.float32).astype(np.float64))


def test_batch_isolates_an_instance_with_non_finite_properties():
    """One instance's properties turn NaN: it alone reports status 3, and the
    other instances' detector values equal those of the clean batch."""
    from redbirdpy_b200.adjoint import BatchModel, detector_values
    from redbirdpy_b200.meshgen import batch_boxes

    cfgs = [rbb.meshprep(c)[0] for c in batch_boxes(6, seed=5, dims=(12.0, 24.0), spacings=(3.0, 4.0), nopt=(2, 5))]
    bm = BatchModel(cfgs, precision="mixed", strict=False)
    mua = torch.as_tensor(np.concatenate([c["prop"][:, 0] for c in cfgs]), device="cuda")
    dco = torch.as_tensor(np.concatenate([1.0 / (3.0 * (c["prop"][:, 0] + c["prop"][:, 1])) for c in cfgs]),
                          device="cuda")
    with torch.no_grad():
        clean = [p.clone() for p in bm.split(detector_values(bm, mua, dco))]
        assert list(np.unique(bm.status)) == [0]
        bad = mua.clone()
        bad[int(bm.node_off[2]) + 3] = float("nan")
        parts = bm.split(detector_values(bm, bad, dco))
    assert int(bm.status[2]) == 3
    assert all(int(bm.status[i]) == 0 for i in range(len(cfgs)) if i != 2)
    for i in range(len(cfgs)):
        if i != 2:
            e = (torch.abs(parts[i] - clean[i]) / torch.abs(clean[i])).max().item()
            assert e <= 1e-6, (i, e)
    strict = BatchModel(cfgs, precision="mixed")
    with pytest.raises(RuntimeError, match="non-finite"):
        detector_values(strict, bad, dco)


"""Parity at the workloads' own sizes, against fixtures made by running the
reference redbirdpy here (tests/golden/make_golden.py --contract):

* the 3M-tet forward (box 100 x 100 x 50 mm at 1 mm, 64 + 64 optodes, CW):
  4 x 4 detector values against the reference's femsolve(method='cg') on
  that subset, at tol=1e-14 and at its default tol=1e-10;
* the 375k-tet adjoint case (2 mm box, per-node properties, 32 x 32 pairs):
  the reference's run (all 32 x 32 detector values) and jac (64 node columns
  of all 1024 rows), and central differences (h = 1e-4 relative) of
  0.5 ||log det - log target||^2 in nodal mua and D on the same 64 nodes
  (SuperLU forward, perturbed solves through the Woodbury identity);
* 8 of the 256 batched instances (batch_boxes(256, seed=2)), each through
  the reference on its own, against the one block-diagonal batch solve.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import redbirdpy_b200 as rbb  # noqa: E402
from redbirdpy_b200 import engine  # noqa: E402
from redbirdpy_b200.meshgen import kuhn_box, grid_optodes, batch_boxes  # noqa: E402

from conftest import GOLDEN  # noqa: E402


def _need(name):
    if not os.path.exists(os.path.join(GOLDEN, name + ".npz")):
        pytest.skip(f"fixture {name}.npz not generated")


def c3_cfg():
    node, elem = kuhn_box([100, 100, 50], 2)
    rng = np.random.default_rng(0)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn), np.zeros(nn),
                            np.full(nn, 1.37)])
    src = np.column_stack([np.repeat(np.linspace(15, 85, 8), 4), np.tile(np.linspace(30, 70, 4), 8), np.zeros(32)])
    return dict(node=node, elem=elem, prop=prop, srcpos=src, srcdir=np.array([[0, 0, 1.0]]), detpos=src + [5, 5, 0],
                detdir=np.array([[0, 0, 1.0]]), omega=0.0)


@pytest.fixture(scope="module")
def c3(golden):
    _need("c3_contract")
    g = golden("c3_contract")
    cfg, sd = rbb.meshprep(c3_cfg())
    return g, cfg, sd


def test_c3_detectors_match_reference(c3):
    g, cfg, sd = c3
    det, phi = rbb.run(cfg)
    err = np.abs(det - g["detval"]) / np.abs(g["detval"])
    assert err.max() <= 1e-6, err.max()
    np.testing.assert_array_equal(sd, g["sd"])
    ep = np.abs(phi[g["nodes"]] - g["phi_rows"]).max() / np.abs(g["phi_rows"]).max()
    assert ep <= 1e-9, ep


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-9), (torch.float32, 1e-6)])
def test_c3_jacobian_columns_match_reference(c3, dtype, tol):
    """Reference-semantics mua Jacobian rows (element mass, 1/4 lumping) on the
    GPU's own forward fields, against the reference jac on 64 node columns."""
    g, cfg, sd = c3
    from redbirdpy_b200.forward import forward_device

    _, phi, _, _, _ = forward_device(cfg)
    mesh = engine.mesh_of(cfg)
    J = engine.jacobian(mesh, phi, sd, "mua", out_dtype=dtype)
    cols = torch.as_tensor(g["nodes"], device=J.device)
    got = J[:, cols].double().cpu().numpy()
    ref = g["jn_cols"]
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= tol, err
    assert np.abs(got - ref).max() / np.abs(ref).max() <= 10 * tol


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_c3_adjoint_gradient_vs_central_fd(c3, precision):
    """The hand-written adjoint (autograd backward) against central
    differences of the direct-solver forward model, h = 1e-4 relative."""
    from redbirdpy_b200.adjoint import DeviceModel, detector_values

    g, cfg, sd = c3
    prop = cfg["prop"]
    model = DeviceModel(cfg, precision=precision)
    mua0 = torch.as_tensor(prop[:, 0].copy(), device="cuda")
    d0 = torch.as_tensor(1.0 / (3.0 * (prop[:, 0] + prop[:, 1])), device="cuda")
    with torch.no_grad():
        det0 = detector_values(model, mua0, d0)
        target = detector_values(model, mua0 * 1.1, d0)
    e0 = np.abs(det0.cpu().numpy() - g["oracle_det0"]) / np.abs(g["oracle_det0"])
    et = np.abs(target.cpu().numpy() - g["target"]) / np.abs(g["target"])
    assert e0.max() <= 1e-6 and et.max() <= 1e-6, (e0.max(), et.max())
    mua = mua0.clone().requires_grad_(True)
    dco = d0.clone().requires_grad_(True)
    # the loss against the fixture's target, as the differences were taken
    tgt = torch.as_tensor(g["target"], device="cuda")
    loss = 0.5 * torch.sum((torch.log(detector_values(model, mua, dco)) - torch.log(tgt)) ** 2)
    loss.backward()
    nodes = torch.as_tensor(g["nodes"], device="cuda")
    for grad, fd in ((mua.grad, g["fd_mua"]), (dco.grad, g["fd_D"])):
        got = grad[nodes].cpu().numpy()
        scale = np.abs(fd).max()
        assert np.abs(got - fd).max() <= 1e-5 * scale, (np.abs(got - fd).max() / scale)


def test_c2_detector_subset_matches_reference_cg(golden):
    """The full 128-column solve of the 3M-tet box against the reference's
    femsolve(method='cg') on 4 sources and 4 detectors.  The subset's values
    span 1 to 1.2e-10 of the largest; a residual-norm criterion determines
    each value only to about (FP64 floor) x (largest / value), so the bar is
    set per magnitude: 1e-6 relative for values >= 1e-4 of the largest
    (against the reference at tol=1e-14, relative residuals ~1e-14), and
    1e-10 of the largest value for every entry.  The reference's default
    tol=1e-10 run stops with the far pairs tens of percent off; against it
    the bar is 1e-6 of the largest value."""
    _need("c2_contract")
    g = golden("c2_contract")
    node, elem = kuhn_box([100, 100, 50], 1)
    cfg = dict(node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
               seg=np.ones(elem.shape[0], dtype=np.int32), srcpos=grid_optodes([15, 85], [15, 85], 8),
               srcdir=np.array([[0, 0, 1.0]]), detpos=grid_optodes([15, 85], [15, 85], 8, offset=(5, 5)),
               detdir=np.array([[0, 0, 1.0]]), omega=0.0)
    cfg, sd = rbb.meshprep(cfg)
    det, _ = rbb.run(cfg)
    sub = det[np.ix_(g["idet"], g["isrc"])]
    assert int(g["flag"]) == 0 and int(g["flag14"]) == 0
    assert g["relres14"].max() <= 1e-13
    ref = g["detval14"]
    big = np.abs(ref).max()
    err = np.abs(sub - ref) / np.abs(ref)
    near = np.abs(ref) >= 1e-4 * big
    assert err[near].max() <= 1e-6, np.array2string(err, precision=2)
    assert np.abs(sub - ref).max() <= 1e-10 * big, np.array2string(err, precision=2)
    err10 = np.abs(sub - g["detval"]).max() / np.abs(g["detval"]).max()
    assert err10 <= 1e-6, err10


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_c5_batch_instances_match_reference(golden, precision):
    """The 256 uneven instances as one block-diagonal system; 8 of them
    against the reference run on each instance alone."""
    _need("c5_contract")
    from redbirdpy_b200.adjoint import BatchModel, detector_values

    g = golden("c5_contract")
    cfgs = [rbb.meshprep(c)[0] for c in batch_boxes(256, seed=2)]
    bm = BatchModel(cfgs, precision=precision)
    mua = torch.as_tensor(np.concatenate([c["prop"][:, 0] for c in cfgs]), device="cuda")
    dco = torch.as_tensor(np.concatenate([1.0 / (3.0 * (c["prop"][:, 0] + c["prop"][:, 1])) for c in cfgs]),
                          device="cuda")
    with torch.no_grad():
        parts = bm.split(detector_values(bm, mua, dco))
    off = 0
    for i, shp in zip(g["pick"], g["shapes"]):
        n = int(np.prod(shp))
        ref = g["detval"][off:off + n].reshape(shp)
        off += n
        got = parts[int(i)].cpu().numpy()
        assert got.shape == ref.shape
        err = np.abs(got - ref) / np.abs(ref)
        assert err.max() <= 1e-6, (int(i), err.max())

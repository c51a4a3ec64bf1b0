"""GPU tests of the two-level preconditioner (Jacobi plus an aggregation
coarse space): the device aggregation against a numpy restatement of the
same binning (exact), and solves with the coarse space against the
Jacobi-only solves and splu (the same FP64 solution; fewer iterations)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import redbirdpy_b200 as rbb  # noqa: E402
from redbirdpy_b200 import engine  # noqa: E402
from redbirdpy_b200.forward import forward_device  # noqa: E402
from redbirdpy_b200.meshgen import kuhn_box  # noqa: E402


def agg_numpy(node, lo, h, nb):
    b = np.clip(np.floor((node - lo) / h), 0, nb - 1).astype(np.int64)
    key = b[:, 0] + nb[0] * (b[:, 1] + nb[1] * b[:, 2])
    _, agg = np.unique(key, return_inverse=True)
    nc = int(agg.max()) + 1
    rows = np.argsort(agg, kind="stable")
    ptr = np.concatenate([[0], np.cumsum(np.bincount(agg, minlength=nc))])
    return agg, ptr, rows


@pytest.mark.parametrize("target", [1, 300, 4096])
def test_aggregate_matches_numpy(target):
    node, elem = kuhn_box([60, 40, 30], 2)
    # shuffled node numbering: aggregates keep their rows ascending all the same
    rng = np.random.default_rng(3)
    perm = rng.permutation(node.shape[0])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    node = node[perm]
    elem = inv[elem - 1] + 1
    mesh = engine.DeviceMesh(node, elem, None, None)
    cs = engine.CoarseSpace(mesh, target)
    assert 1 <= cs.nc <= engine.COARSE_MAX
    lo = mesh.bbox[0]
    agg, ptr, rows = agg_numpy(node, lo, cs.h, np.asarray(cs.nb))
    assert cs.nc == ptr.size - 1
    np.testing.assert_array_equal(cs.agg.cpu().numpy(), agg)
    np.testing.assert_array_equal(cs.agg_ptr[: cs.nc + 1].cpu().numpy(), ptr)
    np.testing.assert_array_equal(cs.agg_rows.cpu().numpy(), rows)
    if target == 1:
        assert cs.nc <= 8  # one cube of the box's volume, rounded up per axis


def box_cfg(size, spacing, omega, seed=0):
    node, elem = kuhn_box(size, spacing)
    rng = np.random.default_rng(seed)
    nn = node.shape[0]
    prop = np.column_stack([rng.uniform(0.008, 0.012, nn), rng.uniform(0.9, 1.1, nn), np.zeros(nn),
                            np.full(nn, 1.37)])
    xs = np.linspace(0.2, 0.8, 4) * size[0]
    ys = np.linspace(0.2, 0.8, 4) * size[1]
    src = np.array([[x, y, 0.0] for x in xs for y in ys])
    det = np.array([[x + 3, y, size[2]] for x in xs for y in ys])
    cfg = dict(node=node, elem=elem, prop=prop, srcpos=src, srcdir=np.array([[0, 0, 1.0]]), detpos=det,
               detdir=np.array([[0, 0, -1.0]]), omega=omega)
    cfg, _ = rbb.meshprep(cfg)
    return cfg


@pytest.mark.parametrize("omega", [0.0, 2 * np.pi * 1e8])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_coarse_solve_matches_jacobi(omega, precision):
    cfg = box_cfg([80, 80, 40], 2, omega)
    d0, p0, _, _, i0 = forward_device(cfg, precision=precision, coarse=False)
    d1, p1, _, _, i1 = forward_device(cfg, precision=precision, coarse=True)
    assert i0["flag"] == 0 and i1["flag"] == 0
    assert i0["coarse_nc"] == 0 and i1["coarse_nc"] > 100
    assert i1["relres"] <= 1e-12 and i0["relres"] <= 1e-12
    err = (torch.abs(p1 - p0).max() / torch.abs(p0).max()).item()
    assert err <= 1e-9, err
    derr = (torch.abs(d1 - d0) / torch.abs(d0)).max().item()
    assert derr <= 1e-6, derr
    assert i1["iters"] < 0.7 * i0["iters"], (i1["iters"], i0["iters"])


def test_coarse_solve_vs_splu_small():
    """Every node its own aggregate (nc = n): the coarse solve is exact."""
    from scipy.sparse.linalg import splu

    cfg = box_cfg([20, 20, 10], 2, 2 * np.pi * 1e8)
    mesh = engine.mesh_of(cfg)
    assert mesh.nn <= engine.COARSE_MAX
    cs = engine.CoarseSpace(mesh, engine.COARSE_MAX)
    assert cs.nc == mesh.nn
    opt = engine.locate_optodes(mesh, cfg)
    B = opt.rhs(mesh)
    mat = engine.assemble(mesh, engine.Optics.from_cfg(mesh, cfg, 1))
    X, info = engine.solve(mat, B, coarse=cs)
    assert info["flag"] == 0
    A = mesh.csr_host(mat.val64)
    ref = splu(A.tocsc()).solve(B.cpu().numpy().astype(complex))
    x = X.cpu().numpy()
    assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-10


def test_coarse_auto_threshold():
    cfg = box_cfg([20, 20, 10], 2, 0.0)
    _, _, _, _, info = forward_device(cfg)
    assert info["coarse_nc"] == 0  # below the node count where 'auto' turns it on
    _, _, _, _, info = forward_device(cfg, coarse=64)
    assert 0 < info["coarse_nc"] <= 64 * 2


def ellipsoid_cfg(omega, nsrc, ndet):
    """A 60 x 60 x 39 mm ellipsoid carved from a 1.5 mm Kuhn box (about 24k
    nodes: many cubes of the coarse grid are partly or wholly empty), with a
    high-contrast spherical inclusion (label 2: mua 0.08, mus 5) and optodes
    on inner planes near the top and bottom."""
    node, elem = kuhn_box([60, 60, 39], 1.5)
    c = node[elem - 1].mean(axis=1)
    keep = ((c[:, 0] - 30) / 30) ** 2 + ((c[:, 1] - 30) / 30) ** 2 + ((c[:, 2] - 19.5) / 19.5) ** 2 <= 1.0
    elem = elem[keep]
    used = np.unique(elem)
    remap = np.zeros(node.shape[0] + 1, dtype=np.int64)
    remap[used] = np.arange(1, used.size + 1)
    node, elem = node[used - 1], remap[elem]
    cc = node[elem - 1].mean(axis=1)
    seg = np.where(np.sum((cc - [30, 30, 12]) ** 2, axis=1) <= 36.0, 2, 1).astype(np.int32)
    rng = np.random.default_rng(7)
    src = np.column_stack([rng.uniform(25, 35, nsrc), rng.uniform(25, 35, nsrc), np.full(nsrc, 36.0)])
    det = np.column_stack([rng.uniform(25, 35, ndet), rng.uniform(25, 35, ndet), np.full(ndet, 3.0)])
    cfg = dict(node=node, elem=elem, seg=seg, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37], [0.08, 5.0, 0, 1.37]]),
               srcpos=src, srcdir=np.array([[0, 0, -1.0]]), detpos=det, detdir=np.array([[0, 0, 1.0]]), omega=omega)
    cfg, _ = rbb.meshprep(cfg)
    return cfg


@pytest.mark.parametrize("omega", [0.0, 2 * np.pi * 1e8])
@pytest.mark.parametrize("cols", [(3, 2), (20, 17)])
def test_coarse_irregular_mesh_odd_columns(omega, cols):
    """Partly empty aggregates, a 8x mua / 5x mus inclusion, 5 and 37 columns
    (the narrow lane-group shapes of the aggregate-ordered kernels): the
    solution matches the Jacobi-only and the plain FP64 solves."""
    cfg = ellipsoid_cfg(omega, *cols)
    d0, p0, _, _, i0 = forward_device(cfg, coarse=False)
    d1, p1, _, _, i1 = forward_device(cfg, coarse=True)
    d2, p2, _, _, i2 = forward_device(cfg, coarse=True, precision="fp64")
    assert i0["flag"] == 0 and i1["flag"] == 0 and i2["flag"] == 0
    assert 0 < i1["coarse_nc"] and i2["coarse_nc"] == i1["coarse_nc"]
    assert i1["iters"] < i0["iters"], (i1["iters"], i0["iters"])
    for p, d in ((p1, d1), (p2, d2)):
        err = (torch.abs(p - p0).max() / torch.abs(p0).max()).item()
        assert err <= 1e-9, err
        derr = (torch.abs(d - d0) / torch.abs(d0)).max().item()
        assert derr <= 1e-6, derr

"""GPU tests of the blocked SpMM over spatial row groups (rb_rowgroups_* and
the group kernel inside rb_femsolve): the groups against a numpy restatement
of the binning (exact), the column unions and row masks against the CSR
pattern (exact), and solves with the groups against solves with the per-row /
row-pair SpMM and against splu."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from scipy import sparse  # noqa: E402
from scipy.sparse.linalg import splu  # noqa: E402

import redbirdpy_b200 as rbb  # noqa: E402
from redbirdpy_b200 import engine  # noqa: E402
from redbirdpy_b200.meshgen import kuhn_box, grid_optodes  # noqa: E402


def groups_numpy(node, lo, edge, h):
    """Rows of every group: cubes of edge h from lo - edge / 2, numbered in
    blocks of 2 x 2 x 2 cubes, each cube's nodes ascending in groups of 8."""
    x0 = lo - 0.5 * edge
    nb = np.maximum(np.ceil((node.max(0) - x0) / h).astype(np.int64) + 1, 1)
    b = np.clip(np.floor((node - x0) / h), 0, nb - 1).astype(np.int64)
    sb = (nb + 1) // 2
    key = 8 * ((b[:, 0] >> 1) + sb[0] * ((b[:, 1] >> 1) + sb[1] * (b[:, 2] >> 1))) + \
        (b[:, 0] & 1) + 2 * (b[:, 1] & 1) + 4 * (b[:, 2] & 1)
    order = np.lexsort((np.arange(node.shape[0]), key))
    out = []
    ks = key[order]
    starts = np.r_[0, np.nonzero(np.diff(ks))[0] + 1, order.size]
    for a, z in zip(starts[:-1], starts[1:]):
        for g in range(a, z, 8):
            rows = np.full(8, -1, np.int64)
            rows[: min(8, z - g)] = order[g:min(g + 8, z)]
            out.append(rows)
    return np.array(out)


@pytest.mark.parametrize("shuffle", [False, True])
def test_rowgroups_match_numpy(shuffle):
    node, elem = kuhn_box([30, 20, 14], 2)
    if shuffle:  # any node numbering: groups stay spatial, rows ascending per cube
        rng = np.random.default_rng(5)
        perm = rng.permutation(node.shape[0])
        inv = np.empty_like(perm)
        inv[perm] = np.arange(perm.size)
        node = node[perm]
        elem = inv[elem - 1] + 1
    mesh = engine.DeviceMesh(node, elem, None, None)
    rg = mesh.row_groups()
    want = groups_numpy(node, mesh.bbox[0], mesh._edge, rg.h)
    got = rg.rows[: rg.ng * 8].cpu().numpy().reshape(-1, 8)
    np.testing.assert_array_equal(got, want)
    # unions and masks against the CSR pattern
    indptr = mesh.indptr.cpu().numpy()
    indices = mesh.indices[: mesh.nnz].cpu().numpy()
    uptr = rg.uptr.cpu().numpy()
    ucol = rg.ucol[: rg.nu].cpu().numpy()
    umask = rg.umask[: rg.nu].cpu().numpy()
    for g in range(rg.ng):
        rows = got[g]
        cols = [set(indices[indptr[r]:indptr[r + 1]]) if r >= 0 else set() for r in rows]
        uni = np.array(sorted(set().union(*cols)))
        np.testing.assert_array_equal(ucol[uptr[g]:uptr[g + 1]], uni)
        m = np.array([sum(1 << i for i in range(8) if c in cols[i]) for c in uni])
        np.testing.assert_array_equal(umask[uptr[g]:uptr[g + 1]], m)


@pytest.mark.parametrize("ncol", [68, 100, 128])
def test_group_spmm_solve_matches_row_kernels_and_splu(ncol):
    node, elem = kuhn_box([40, 36, 20], 1)
    cfg = dict(node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
               seg=np.ones(elem.shape[0], dtype=np.int32), srcpos=grid_optodes([5, 35], [5, 31], 4),
               srcdir=np.array([[0, 0, 1.0]]), detpos=grid_optodes([6, 34], [6, 30], 4),
               detdir=np.array([[0, 0, 1.0]]), omega=0)
    cfg, _ = rbb.meshprep(cfg)
    mesh = engine.mesh_of(cfg)
    mat = engine.assemble(mesh, engine.Optics.from_cfg(mesh, cfg))
    rng = np.random.default_rng(ncol)
    Bh = rng.standard_normal((mesh.nn, ncol)) * (rng.random((mesh.nn, ncol)) < 0.01)
    Bh[:, 3] = 0.0  # a zero column stays exactly zero
    B = torch.as_tensor(Bh, device=mesh.device)
    X0, i0 = engine.solve(mat, B, groups=None, coarse=False)
    X1, i1 = engine.solve(mat, B, groups="auto", coarse=False)
    assert mesh.row_groups() is not None and mesh.row_groups().ng > 0
    assert i0["flag"] == 0 and i1["flag"] == 0 and i1["relres"] <= 1e-14
    assert torch.all(X1[:, 3] == 0)
    err = (torch.abs(X1 - X0).max() / torch.abs(X0).max()).item()
    assert err <= 1e-12, err
    A = mesh.csr_host(mat.val64)
    Xs = splu(sparse.csc_matrix(A)).solve(Bh)
    err = np.abs(X1.cpu().numpy() - Xs).max() / np.abs(Xs).max()
    assert err <= 1e-10, err
    assert abs(i1["iters"] - i0["iters"]) <= 0.1 * i0["iters"] + 2

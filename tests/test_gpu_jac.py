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

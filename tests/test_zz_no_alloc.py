"""rb_femlhs_noalloc: the assembly entry point for callers that cannot
allocate device memory (it uses a fixed scratch array inside the library
instead of a caller workspace).  Checked through the C ABI against the
workspace entry point rb_femlhs, on two calls in a row.  This file is
collected last so that a run stopping at the first failure has run every
other test before it."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from redbirdpy_b200 import _lib, engine  # noqa: E402
from redbirdpy_b200._lib import call, ptr, stream  # noqa: E402

from test_gpu_forward import cfg_from  # noqa: E402


def _outputs(mesh, cplx):
    t64 = torch.complex128 if cplx else torch.float64
    t32 = torch.complex64 if cplx else torch.float32
    out = [torch.full((mesh.nnz,), float("nan"), dtype=t64, device="cuda"),
           torch.full((mesh.nnz,), float("nan"), dtype=t32, device="cuda"),
           torch.full((mesh.nn,), float("nan"), dtype=t64, device="cuda"),
           torch.full((mesh.nn,), float("nan"), dtype=t32, device="cuda")]
    return out


@pytest.mark.parametrize("case", ["nodal_fd", "c1_cw"])
def test_femlhs_noalloc_matches_workspace_entry_point(golden, case):
    g = golden(case)
    cfg = cfg_from(g)
    mesh = engine.mesh_of(cfg)
    optics = engine.Optics.from_cfg(mesh, cfg)
    ref = engine.assemble(mesh, optics)  # rb_femlhs with a caller workspace
    cplx = ref.is_complex
    for _ in range(2):  # the scratch keeps the previous call's contents
        v64, v32, d64, d32 = _outputs(mesh, cplx)
        call("rb_femlhs_noalloc", ctypes.byref(mesh.struct), ctypes.byref(optics.struct), ptr(mesh.evol),
             ptr(mesh.ddd), ptr(v64), ptr(v32), ptr(d64), ptr(d32), stream())
        torch.cuda.synchronize()
        for got, want, tol in ((v64, ref.val64, 1e-12), (d64, ref.dinv64, 1e-12), (v32, ref.val32, 1e-6),
                               (d32, ref.dinv32, 1e-6)):
            got, want = got.cpu().numpy(), want.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.abs(got - want).max() <= tol * np.abs(want).max()
    # same values as the reference's own assembly
    A = v64.cpu().numpy()
    assert np.abs(A - g["A_data"]).max() <= 1e-12 * np.abs(g["A_data"]).max()


def test_femlhs_noalloc_rejects_oversized_mesh():
    """More nodes than the fixed scratch holds: a clear error, before any
    device memory is touched (the mesh pointers here are never read)."""
    m = _lib.RbMesh()
    m.nn, m.ne = 4 * 1024 * 1024 + 1, 1
    o = _lib.RbOptics()
    o.kind = _lib.RB_PROP_NODE
    dummy = ctypes.c_void_p(16)
    code = _lib.lib().rb_femlhs_noalloc(ctypes.byref(m), ctypes.byref(o), dummy, dummy, dummy, None, None, None,
                                        stream())
    assert code == _lib.RB_ESIZE
    assert b"fixed scratch" in _lib.lib().rb_last_error()

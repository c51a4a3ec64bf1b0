"""redbirdpy_b200 - the FEM forward / adjoint-Jacobian / Gauss-Newton hot
path of redbirdpy (diffuse optical tomography), on NVIDIA B200 (sm_100a).

Drop-in for redbirdpy's own API on that path: ``meshprep``, ``run``,
``runforward``, ``femlhs``, ``femrhs``, ``femgetdet``, ``femsolve``, ``jac``,
``runrecon``, ``reginv`` take the same ``cfg`` / ``recon`` dicts (1-based
``elem``/``face``) and return numpy / scipy objects like the reference.  The
numerical work runs in hand-written CUDA kernels (``librbb200.so``, C ABI in
``include/redbird_b200.h``); there is no CPU fallback.
"""

__version__ = "0.1.0"

from . import adjoint, forward, solver, utility, meshgen  # noqa: F401
from .adjoint import DeviceModel, detector_values  # noqa: F401
from .forward import *  # noqa: F401,F403
from .solver import *  # noqa: F401,F403
from .utility import *  # noqa: F401,F403

try:  # the Gauss-Newton layer
    from . import recon  # noqa: F401
    from .recon import *  # noqa: F401,F403
except ImportError:  # pragma: no cover - recon module not present
    recon = None


def run(cfg, recon_cfg=None, detphi0=None, sd=None, **kwargs):
    """Forward (``recon_cfg is None``) or Gauss-Newton reconstruction, like
    redbirdpy's ``run`` (redbirdpy/__init__.py:83-112)."""
    if recon_cfg is None:
        return forward.runforward(cfg, **kwargs)
    if detphi0 is None:
        raise ValueError("detphi0 is required for reconstruction")
    return recon.runrecon(cfg, recon_cfg, detphi0, sd, **kwargs)

"""ORACLE / TEST INFRASTRUCTURE ONLY - never imported by the product path.

Point location in a tetrahedral mesh: a CPU restatement of the contract of
``iso2mesh.tsearchn`` as redbirdpy calls it in ``femrhs``
(redbirdpy/forward.py:316 and :337): ``tsearchn(node, elem_1based, pts)``
returns ``(loc, bary)`` with ``loc`` the 1-based index of an enclosing
element as float (NaN when outside) and ``bary`` the ``Npts x 4`` barycentric
coordinates of each point in that element (NaN rows when outside).

iso2mesh is not installed here, so this module is also injected as
``sys.modules['iso2mesh']`` when the reference itself is run to make golden
fixtures.  The tie-break rule for points on shared faces or edges is fixed
here and mirrored by the CUDA point-location kernel: the LOWEST element index
whose four barycentric coordinates are all >= -BARY_TOL.  (Any choice gives
the same right-hand side because P1 interpolation is continuous.)
"""

import numpy as np

BARY_TOL = 1e-9


def tet_barycentric(node, elem0, pt):
    """Barycentric coordinates of ``pt`` in every tetrahedron of ``elem0``.

    Cramer's rule with signed sub-volumes: lambda_i = vol(tet with vertex i
    replaced by pt) / vol(tet).  ``elem0`` is 0-based ``M x 4``.
    """
    x = node[elem0]  # M x 4 x 3
    p = np.asarray(pt, dtype=np.float64)

    def det3(a, b, c):
        return (
            a[:, 0] * (b[:, 1] * c[:, 2] - b[:, 2] * c[:, 1])
            - a[:, 1] * (b[:, 0] * c[:, 2] - b[:, 2] * c[:, 0])
            + a[:, 2] * (b[:, 0] * c[:, 1] - b[:, 1] * c[:, 0])
        )

    x0, x1, x2, x3 = x[:, 0], x[:, 1], x[:, 2], x[:, 3]
    vol = det3(x1 - x0, x2 - x0, x3 - x0)
    l1 = det3(p - x0, x2 - x0, x3 - x0) / vol
    l2 = det3(x1 - x0, p - x0, x3 - x0) / vol
    l3 = det3(x1 - x0, x2 - x0, p - x0) / vol
    l0 = 1.0 - l1 - l2 - l3
    return np.stack([l0, l1, l2, l3], axis=1)


def tsearchn(node, elem, pts):
    """``(loc, bary)`` as described in the module docstring (elem 1-based)."""
    node = np.asarray(node, dtype=np.float64)
    elem0 = np.asarray(elem)[:, :4].astype(np.int64) - 1
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))[:, :3]
    x = node[elem0]
    lo = x.min(axis=1) - 1e-9
    hi = x.max(axis=1) + 1e-9
    loc = np.full(pts.shape[0], np.nan)
    bary = np.full((pts.shape[0], 4), np.nan)
    for k, p in enumerate(pts):
        cand = np.nonzero(np.all((lo <= p) & (p <= hi), axis=1))[0]
        if cand.size == 0:
            continue
        b = tet_barycentric(node, elem0[cand], p)
        ok = np.nonzero(np.all(b >= -BARY_TOL, axis=1))[0]
        if ok.size == 0:
            continue
        loc[k] = cand[ok[0]] + 1
        bary[k] = b[ok[0]]
    return loc, bary

"""Structured tetrahedral box meshes (Kuhn / Freudenthal split).

The synthetic workloads of this package are boxes meshed on a regular node
grid, each cube cut into the 6 Kuhn tetrahedra that share its main diagonal.
The result is returned in redbirdpy's conventions: ``node`` is ``Nn x 3``
float64 (mm), ``elem`` is ``Ne x 4`` int with **1-based** node indices (the
convention of ``redbirdpy/__init__.py:13-15``), ``face`` is left to
``meshprep``.  Node numbering is x-fastest, then y, then z.

Element orientation is deliberately *not* normalised here: half of the Kuhn
tetrahedra come out with negative signed volume and ``meshprep`` swaps nodes
0 and 1 of those, exactly as ``_meshreorient_fallback``
(redbirdpy/utility.py:1047-1063) does.
"""

import numpy as np

__all__ = ["kuhn_box", "grid_optodes", "batch_boxes"]


def kuhn_box(size, spacing, origin=(0.0, 0.0, 0.0)):
    """Mesh the box ``origin + [0,size_x] x [0,size_y] x [0,size_z]``.

    ``spacing`` is the node pitch (scalar or 3-vector); every extent must be an
    integer multiple of it.  Returns ``(node, elem)`` with 1-based ``elem``.
    """
    size = np.broadcast_to(np.asarray(size, dtype=np.float64), (3,))
    h = np.broadcast_to(np.asarray(spacing, dtype=np.float64), (3,))
    ncell = np.rint(size / h).astype(np.int64)
    if np.any(ncell < 1) or np.any(np.abs(ncell * h - size) > 1e-9 * np.maximum(size, 1)):
        raise ValueError("box extents must be positive integer multiples of the spacing")
    nx, ny, nz = (ncell + 1).tolist()
    xs = origin[0] + h[0] * np.arange(nx)
    ys = origin[1] + h[1] * np.arange(ny)
    zs = origin[2] + h[2] * np.arange(nz)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    node = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])

    cx, cy, cz = ncell.tolist()
    k, j, i = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")
    v000 = (i + nx * (j + ny * k)).ravel()
    step = {0: 1, 1: nx, 2: nx * ny}
    v111 = v000 + 1 + nx + nx * ny
    tets = []
    # one tetrahedron per permutation (a, b, c) of the axes:
    # v000 -> v000+e_a -> v000+e_a+e_b -> v111
    for a, b in ((0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)):
        va = v000 + step[a]
        vab = va + step[b]
        tets.append(np.stack([v000, va, vab, v111], axis=1))
    # cube-major ordering: the 6 tetrahedra of a cube are consecutive
    elem = np.stack(tets, axis=1).reshape(-1, 4) + 1
    return node, elem.astype(np.int64)


def grid_optodes(x_range, y_range, n_per_side, z=0.0, offset=(0.0, 0.0)):
    """``n_per_side x n_per_side`` optodes on the plane ``z``, row-major in y."""
    xs = np.linspace(x_range[0], x_range[1], n_per_side) + offset[0]
    ys = np.linspace(y_range[0], y_range[1], n_per_side) + offset[1]
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    return np.column_stack([xx.ravel(), yy.ravel(), np.full(xx.size, float(z))])


def batch_boxes(count=256, seed=2, dims=(30.0, 80.0), spacings=(2.0, 3.0, 4.0), nopt=(4, 16),
                mua=(0.005, 0.03), mus=(0.5, 2.0), nref=1.37):
    """Independent box workloads of uneven size (unprepared cfg dicts).

    Per instance: extents ~ U[dims] mm per axis rounded to a multiple of a
    spacing drawn from ``spacings``; per-node mua ~ U[mua], mus ~ U[mus],
    g = 0, n = ``nref``; ``nopt`` ranges the number of sources and, separately,
    of detectors, placed at random on the top face (z = 0, pointing +z) at
    least one cell from its edges.  CW (omega = 0)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        h = float(rng.choice(spacings))
        size = np.maximum(np.rint(rng.uniform(dims[0], dims[1], 3) / h), 2) * h
        node, elem = kuhn_box(size, h)
        nn = node.shape[0]
        prop = np.column_stack([rng.uniform(mua[0], mua[1], nn), rng.uniform(mus[0], mus[1], nn), np.zeros(nn),
                                np.full(nn, nref)])
        ns, nd = rng.integers(nopt[0], nopt[1] + 1, 2)

        def top(k):
            return np.column_stack([rng.uniform(h, size[0] - h, k), rng.uniform(h, size[1] - h, k), np.zeros(k)])

        out.append(dict(node=node, elem=elem, prop=prop, srcpos=top(ns), srcdir=np.array([[0, 0, 1.0]]),
                        detpos=top(nd), detdir=np.array([[0, 0, 1.0]]), omega=0.0))
    return out

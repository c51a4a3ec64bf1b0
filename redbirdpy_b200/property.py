"""Multi-spectral properties: chromophore concentrations to per-wavelength
optical properties, drop-in for redbirdpy's ``property`` module on the
reconstruction path (redbirdpy/property.py:30-213): ``extinction``,
``updateprop``.

The molar extinction spectra themselves (the compiled tables inside
redbirdpy/property.py) are not part of this package: ``extinction`` takes
them from an installed redbirdpy when one can be imported, and every
function here also accepts the coefficients directly (``extin``), so that a
caller without redbirdpy passes its own values.
"""

import numpy as np

__all__ = ["extinction", "updateprop", "CHROMOPHORES"]

# the chromophores redbirdpy recognises, in the order it visits them
# (property.py:135, recon.py:170-174)
CHROMOPHORES = ("hbo", "hbr", "water", "lipids", "aa3")


def _wavelength_floats(wavelengths):
    if isinstance(wavelengths, (list, tuple)):
        wavelengths = [float(w) if isinstance(w, str) else w for w in wavelengths]
    return np.atleast_1d(np.asarray(wavelengths, dtype=float))


def extinction(wavelengths, chromophores, extin=None, **interp_opts):
    """Molar extinction coefficients, (Nwv x Nchrome) (property.py:30-89).

    ``extin`` given: returned as an array of that shape (a dict keyed by
    chromophore, each a per-wavelength sequence, is accepted too).
    Otherwise the spectra come from redbirdpy's own tables
    (``redbirdpy.property.extinction``), which must be importable."""
    if isinstance(chromophores, str):
        chromophores = [chromophores]
    wl = _wavelength_floats(wavelengths)
    if extin is not None:
        if isinstance(extin, dict):
            extin = np.column_stack([np.atleast_1d(np.asarray(extin[c], dtype=float)) for c in chromophores])
        extin = np.atleast_2d(np.asarray(extin, dtype=float))
        if extin.shape != (wl.size, len(chromophores)):
            raise ValueError(f"extin must be {wl.size} x {len(chromophores)} (wavelengths x chromophores)")
        return extin, None
    try:
        from redbirdpy.property import extinction as _ref_extinction
    except ImportError as e:  # pragma: no cover - depends on the environment
        raise ImportError("molar extinction spectra are not bundled: install redbirdpy, or pass the "
                          "coefficients as extin= (wavelengths x chromophores)") from e
    return _ref_extinction(list(wl), list(chromophores), **interp_opts)


def updateprop(cfg, wv=None, extin=None):
    """Per-wavelength [mua, musp, g, n] from cfg['param'] (property.py:92-213):
    mua = sum_t extin(wv, t) C_t over the chromophores present (water 0.23
    and lipids 0.58 are inserted into cfg['param'] when missing, as the
    reference does), musp = scatamp * wv ** -scatpow when both are given.
    Label-based templates (fewer rows than nodes and tets) take the values
    into rows 1..; node/element-based ones are rebuilt.  ``extin``: an
    optional dict {wavelength: {chromophore: coefficient}}."""
    if "param" not in cfg or not isinstance(cfg.get("prop"), dict):
        return cfg.get("prop")
    wavelengths = list(cfg["prop"].keys()) if wv is None else [wv]
    params = cfg["param"]
    out = {}
    for wavelen in wavelengths:
        if "water" not in params:
            params["water"] = 0.23
        if "lipids" not in params:
            params["lipids"] = 0.58
        types = [t for t in CHROMOPHORES if t in params]
        if not types:
            raise ValueError("No recognized chromophores in cfg.param. "
                             "Expected one or more of: hbo, hbr, water, lipids, aa3")
        given = None if extin is None else extin.get(wavelen, extin.get(str(wavelen)))
        if given is not None:
            given = [given[t] for t in types]
        ext, _ = extinction(float(wavelen), types, None if given is None else np.atleast_2d(given))
        first = params[types[0]]
        mua = 0.0 if np.isscalar(first) else np.zeros_like(first, dtype=float)
        for j, t in enumerate(types):
            mua = mua + ext[0, j] * params[t]
        musp = params["scatamp"] * float(wavelen) ** (-params["scatpow"]) \
            if ("scatamp" in params and "scatpow" in params) else None
        seg = cfg["prop"][wavelen]
        nn = cfg["node"].shape[0] if "node" in cfg else np.size(mua)
        ne = cfg["elem"].shape[0] if "elem" in cfg else np.size(mua)
        mlen = np.size(mua) if hasattr(mua, "__len__") else 1
        if mlen < min(nn, ne):  # label-based: rows 1.. are the tissue labels
            new = seg.copy()
            rows = slice(1, mlen + 1) if hasattr(mua, "__len__") else 1
            new[rows, 0] = mua
            if musp is not None:
                new[rows, 1] = musp
                new[rows, 2] = 0
        elif musp is not None:
            nref = seg[1, 3] if seg.shape[0] > 1 else 1.37
            if hasattr(mua, "__len__"):
                new = np.column_stack([mua, musp * np.ones_like(mua), np.zeros_like(mua), np.full_like(mua, nref)])
            else:
                new = np.array([[mua, musp, 0, nref]])
        elif hasattr(mua, "__len__"):
            new = np.column_stack([mua, np.tile(seg[1, 1:], (len(mua), 1))])
        else:
            new = np.array([[mua] + list(seg[1, 1:])])
        out[wavelen] = new
    return out if len(wavelengths) > 1 else out[wavelengths[0]]

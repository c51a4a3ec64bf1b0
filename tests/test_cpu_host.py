"""CPU-only checks: the C-ABI library loads and exports every declared entry
point, and the host-side mesh preparation matches the oracle."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "redbird_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(rb_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_header_symbols():
    from redbirdpy_b200 import _lib

    lib = _lib.lib()  # loads without a GPU
    names = header_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.exported_symbols()), set(names) ^ set(_lib.exported_symbols())
    assert lib.rb_version() >= 1


def test_host_meshprep_helpers_match_oracle(golden):
    from redbirdpy_b200 import utility as ut
    from oracle import femoracle as fo

    g = golden("c1_cw")
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([60, 60, 30], 5)
    r = ut._reorient(node, elem)
    assert np.array_equal(r, g["elem"])
    f = ut._volface(r, node.shape[0])
    assert np.array_equal(f, g["face"]) and np.array_equal(f, fo.volface(r))
    np.testing.assert_allclose(ut._elemvolume(node, f), g["area"], rtol=1e-14)
    np.testing.assert_allclose(ut._elemvolume(node, r), g["evol"], rtol=1e-14)
    np.testing.assert_allclose(ut._nodevolume(node.shape[0], r, g["evol"]), g["nvol"], rtol=1e-13)
    assert ut.getreff(1.37) == pytest.approx(float(g["reff"]), abs=1e-15)
    assert ut.getreff(1.0) == 0.0


def test_sdmap_and_optodes_match_oracle(golden):
    from redbirdpy_b200 import utility as ut
    from oracle import femoracle as fo

    g = golden("nodal_cw")
    cfg = dict(node=g["node"], elem=g["elem"], face=g["face"], prop=g["prop"], srcpos=g["srcpos"],
               srcdir=np.array([[0, 0, 1.0]]), detpos=g["detpos"], detdir=np.array([[0, 0, 1.0]]))
    assert np.array_equal(ut.sdmap(cfg), g["sd"])
    s, d, _, _ = ut.getoptodes(cfg)
    os_, od_ = fo.getoptodes(cfg)
    np.testing.assert_allclose(np.vstack([s, d]), g["optode"], rtol=1e-15)
    np.testing.assert_allclose(np.vstack([os_, od_]), g["optode"], rtol=1e-15)
    sd = ut.sdmap(cfg, maxdist=15.0)
    dist = ut.getdistance(cfg["srcpos"], cfg["detpos"])
    for s_, d_, a in sd:
        assert a == (1.0 if dist[int(d_) - 4, int(s_)] < 15.0 else 0.0)


def test_kuhn_box_counts():
    from redbirdpy_b200.meshgen import kuhn_box

    node, elem = kuhn_box([100, 100, 50], 1)
    assert node.shape == (520251, 3) and elem.shape == (3000000, 4)
    assert elem.min() == 1 and elem.max() == 520251


def test_batch_boxes_workload():
    """The uneven-instance workload generator: seeded, extents multiples of
    the spacing, optode counts and properties in their ranges."""
    from redbirdpy_b200.meshgen import batch_boxes

    a = batch_boxes(12, seed=2)
    b = batch_boxes(12, seed=2)
    for x, y in zip(a, b):
        assert np.array_equal(x["node"], y["node"]) and np.array_equal(x["prop"], y["prop"])
    for c in a:
        node, elem = c["node"], c["elem"]
        ext = node.max(axis=0) - node.min(axis=0)
        h = np.diff(np.unique(node[:, 0]))[0]
        assert h in (2.0, 3.0, 4.0)
        assert np.allclose(ext / h, np.rint(ext / h)) and np.all(ext >= 2 * h)
        assert elem.min() == 1 and elem.max() == node.shape[0]
        assert 4 <= c["srcpos"].shape[0] <= 16 and 4 <= c["detpos"].shape[0] <= 16
        assert np.all((c["prop"][:, 0] >= 0.005) & (c["prop"][:, 0] <= 0.03))
        assert np.all((c["prop"][:, 1] >= 0.5) & (c["prop"][:, 1] <= 2.0))
        assert np.all(c["srcpos"][:, 2] == 0) and np.all(c["srcpos"][:, :2] >= h)


def test_multi_wavelength_host_pieces(golden):
    """Per-wavelength bulk, reff and sd tables (property.py:267-271,
    utility.py:198-205, 733-760) against the reference's meshprep output."""
    from redbirdpy_b200 import utility as u

    g = golden("nodal_multiwl")
    cfg = dict(node=g["node"], elem=g["elem"], face=g["face"], srcpos=g["srcpos"], detpos=g["detpos"],
               prop={"690": g["prop_690"], "830": g["prop_830"]})
    bk = u.getbulk(cfg)
    assert set(bk) == {"690", "830"}
    for wv in ("690", "830"):
        assert u.getreff(bk[wv][3], 1.0) == pytest.approx(float(g["reff_" + wv]), rel=1e-14)
        assert u.getltr(cfg, wv) == pytest.approx(1.0 / (bk[wv][0] + bk[wv][1] * (1 - bk[wv][2])))
    sd = u.sdmap(cfg)
    for wv in ("690", "830"):
        assert np.array_equal(sd[wv], g["sd_" + wv])


def test_coarse_space_host_rules():
    """Aggregate counts and the coarse option's resolution (no GPU needed)."""
    from redbirdpy_b200 import engine

    assert engine.coarse_target(520251) == 2048 and engine.coarse_target(520251, True) == 1024
    assert engine.coarse_target(67626) == 1056 and engine.coarse_target(67626, True) == 528
    assert engine.coarse_target(20000) == 312
    assert engine.coarse_target(1000) == 62  # never above nn / 16
    assert all(1 <= engine.coarse_target(n, c) <= engine.COARSE_MAX for n in (1, 17, 10 ** 7) for c in (0, 1))

    class Mat:  # a matrix without a DeviceMesh (e.g. uploaded from scipy)
        n, is_complex, mesh = 10 ** 6, False, None

    assert engine._resolve_coarse(Mat(), None) is None
    assert engine._resolve_coarse(Mat(), False) is None
    assert engine._resolve_coarse(Mat(), "auto") is None
    with pytest.raises(ValueError):
        engine._resolve_coarse(Mat(), True)

    class Mesh:
        def coarse_space(self, target):
            return ("space", target)

    class MeshMat(Mat):
        mesh = Mesh()

    m = MeshMat()
    assert engine._resolve_coarse(m, "auto") == ("space", 2048)
    assert engine._resolve_coarse(m, 300) == ("space", 300)
    m.n = 1000
    assert engine._resolve_coarse(m, "auto") is None  # below COARSE_MIN_NODES
    assert engine._resolve_coarse(m, True) == ("space", 62)
    with pytest.raises(ValueError):
        engine._resolve_coarse(m, "sometimes")
    # the C ABI sizes: nothing without aggregates, growing with nc and columns
    from redbirdpy_b200 import _lib

    wb = _lib.lib().rb_coarse_work_bytes
    assert wb(0, 128, 0, 0) == 0
    assert 0 < wb(256, 128, 0, 0) < wb(2048, 128, 0, 0) < wb(2048, 128, 1, 0)
    assert wb(2048, 32, 0, 0) < wb(2048, 128, 0, 0)
    ab = _lib.lib().rb_coarse_aggregate_work_bytes
    assert ab(0, 10) == 0 and ab(1000, 512) > 0


def test_gram_staging_rule():
    """rb_gram_stage_bytes (host arithmetic only): rows up to 1 MB are formed
    in place (0 bytes); longer rows get one compact 65536-column slab of J
    (and one of Jlo for the split form), plus 256 bytes of alignment slack."""
    from redbirdpy_b200 import _lib

    sb = _lib.lib().rb_gram_stage_bytes
    M = 8192
    assert sb(M, 135252, 135256, 4, 0) == 0              # 541 KB rows
    assert sb(M, 262144, 262144, 4, 0) == 0              # exactly 1 MB
    slab = M * 65536 * 4 + 256
    assert sb(M, 1040502, 1040504, 4, 0) == slab         # 4 MB rows
    assert sb(M, 1040502, 1040504, 4, 1) == 2 * (M * 65536 * 4) + 256
    assert sb(M, 600001, 600008, 2, 0) == M * 65536 * 2 + 256  # BF16 rows of 1.2 MB
    assert sb(M, 300001, 300008, 2, 0) == 0              # BF16 rows of 600 KB
    assert sb(0, 1040502, 1040504, 4, 0) == 0 and sb(M, 1040502, 1040504, 3, 0) == 0


def test_jacobian_slab_width_rule(monkeypatch):
    """runrecon stores J whole while it fits in half the free HBM, else
    recomputes it in node slabs of a quarter of the free memory (rows x
    parameters x slab x element size); an explicit width is kept."""
    torch = pytest.importorskip("torch")
    from redbirdpy_b200 import recon

    class Mesh:
        nn = 520251

    phi = torch.zeros(1, dtype=torch.complex128)  # frequency domain: [Re; Im] rows
    sd = np.column_stack([np.zeros(4096), np.ones(4096), np.ones(4096)])
    sd[:10, 2] = 0  # inactive pairs add no rows
    rows = 2 * 4086
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (180e9, 183e9))
    assert recon._slab_width("auto", Mesh, phi, sd, 2, torch.float32) == 0  # 34 GB <= 90 GB
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (40e9, 183e9))
    w = recon._slab_width("auto", Mesh, phi, sd, 2, torch.float32)
    assert w == int(0.25 * 40e9 / (rows * 2 * 4))
    assert recon._slab_width("auto", Mesh, phi, sd, 2, torch.bfloat16) == 0  # BF16 rows: 17 GB <= 20 GB
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (30e9, 183e9))
    assert recon._slab_width("auto", Mesh, phi, sd, 2, torch.bfloat16) == int(0.25 * 30e9 / (rows * 2 * 2))
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (1e6, 183e9))
    assert recon._slab_width("auto", Mesh, phi, sd, 2, torch.float32) == 1024  # floor
    assert recon._slab_width(None, Mesh, phi, sd, 2, torch.float32) == 0
    assert recon._slab_width(False, Mesh, phi, sd, 2, torch.float32) == 0
    assert recon._slab_width(5000, Mesh, phi, sd, 2, torch.float32) == 5000


def test_solve_tuner_picks_the_fastest_and_caches_per_bucket(monkeypatch):
    """The autotuner times every (lanes, check interval) candidate, skips
    those that did not converge, keeps the fastest and reuses it for every
    system of the same size bucket; another bucket is tuned afresh."""
    torch = pytest.importorskip("torch")
    from redbirdpy_b200 import engine

    ms = {(0, 10): 9.0, (0, 20): 8.0, (8, 10): 3.0, (8, 20): 1.0, (16, 10): 2.0, (16, 20): 4.0,
          (32, 10): 5.0, (32, 20): 6.0}
    calls = []

    def fake_solve(mat, B, **kw):
        key = (kw["spmm_lanes"], kw["check_every"])
        calls.append(key)
        clock["now"] += ms[key]
        return None, {"flag": 2 if key == (8, 20) else 0}  # the fastest shape fails here

    clock = {"now": 0.0}

    class Event:
        def __init__(self, enable_timing=False):
            self.t = None

        def record(self, stream=None):
            self.t = clock["now"]

        def elapsed_time(self, other):
            return other.t - self.t

    monkeypatch.setattr(engine, "solve", fake_solve)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "Event", Event)

    class Mat:
        n, nnz, is_complex = 1000, 15000, False

    tuner = engine.SolveTuner()
    B = torch.zeros(1000, 32)
    best = tuner.options(Mat, B, precision="mixed")
    assert (best["spmm_lanes"], best["check_every"]) == (16, 10)
    assert len(calls) == 1 + 8  # a warm-up, then every candidate once
    calls.clear()
    assert tuner.options(Mat, torch.zeros(1000, 32), precision="mixed") is best  # same bucket: cached
    assert calls == []

    class Big:
        n, nnz, is_complex = 4000, 60000, False

    tuner.options(Big, torch.zeros(4000, 32), precision="mixed")
    assert len(calls) == 9  # another size bucket is tuned again


def test_captured_step_budget_rule(monkeypatch):
    """The fixed solve budget of a captured step: one checked solve, its
    sweep count and 1.25 x the most iterations a sweep took (at least 8),
    cached per (nodes, nonzeros, columns, precision, lanes) so that models of
    one size share it; a solve that did not converge raises."""
    torch = pytest.importorskip("torch")
    from redbirdpy_b200 import adjoint

    infos = [{"flag": 0, "outer": 3, "sweep_iters_max": 41}, {"flag": 0, "outer": 1, "sweep_iters_max": 2},
             {"flag": 1, "outer": 9, "sweep_iters_max": 500}]
    monkeypatch.setattr(adjoint.engine, "assemble", lambda mesh, optics: None)
    monkeypatch.setattr(adjoint.engine, "solve", lambda mat, B, **kw: (None, infos.pop(0)))
    monkeypatch.setattr(adjoint, "_BUDGETS", {})

    def model(nn, nnz):
        m = object.__new__(adjoint.DeviceModel)
        m.mesh = type("Mesh", (), {"nn": nn, "nnz": nnz})()
        m.B = torch.zeros(nn, 16)
        m.solve_kw = {"precision": "mixed", "budget": (1, 1)}
        m.optics = lambda mua, dco: None
        return m

    x = torch.zeros(3)
    a = model(1000, 15000)
    assert a.calibrate_budget(x, x) == (3, 52)  # ceil(1.25 * 41)
    assert model(1000, 15000).calibrate_budget(x, x) == (3, 52)  # same size: cached, no solve
    assert len(infos) == 2
    assert model(2000, 30000).calibrate_budget(x, x) == (1, 8)  # floor of 8 iterations
    with pytest.raises(RuntimeError):
        model(3000, 45000).calibrate_budget(x, x)


def test_instances_host_layout():
    """Instance row offsets: the row -> instance map (zero-row instances
    allowed), the checks on the offsets, and the status codes the header
    documents for rb_instances."""
    torch = pytest.importorskip("torch")
    from redbirdpy_b200 import engine

    inst = engine.Instances([0, 3, 3, 7], "cpu")
    assert inst.ninst == 3 and inst.n == 7
    assert inst.row_inst.tolist() == [0, 0, 0, 2, 2, 2, 2]
    assert inst.row_ptr.tolist() == [0, 3, 3, 7]
    for bad in ([1, 3], [0, 5, 4], [0], [[0, 1]]):
        with pytest.raises(ValueError):
            engine.Instances(bad, "cpu")
    src = open(os.path.join(ROOT, "include", "redbird_b200.h")).read()
    text = re.search(r"int32_t\* status;\s*/\*(.*?)\*/", src, flags=re.S).group(1)
    text = " ".join(text.split())
    for code, word in ((0, "converged"), (1, "not converged"), (2, "breakdown"), (3, "non-finite"), (4, "gave up")):
        assert f"{code} {word}" in text or f"{code} Krylov {word}" in text or f"{code} a bounded in-kernel wait {word}" \
            in text, (code, text)
    assert sorted(engine.INSTANCE_STATUS) == [0, 1, 2, 3, 4]

"""Benchmark: multi-RHS FEM forward solves on the 3M-tet box (RHS solves/s).

Workload (one "step" = one full forward pass, femrhs -> femlhs -> femsolve
-> femgetdet): box 100 x 100 x 50 mm at 1 mm Kuhn spacing (520,251 nodes,
3,000,000 tets), mua 0.01/mm, mus 1.0/mm, g 0, n 1.37, 64 sources on an 8x8
grid over x,y in [15,85] mm on z=0 and 64 detectors offset by 5 mm, CW.
All 128 columns are solved to the FP64 accuracy floor (mixed precision: FP32
block PCG inside FP64 refinement).  ``value`` = 128 RHS / device time per
step with inputs resident in HBM; ``e2e`` = the same through the public
``runforward`` API from host arrays (uploads and the phi/detval download
inside the timed region).  The working set (5 x 266 MB Krylov vectors) is
larger than L2, so no explicit flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RHS solves/s (3M tets, 64 src + 64 det, CW, <=1e-6 detector error)"
UNIT = "RHS/s"


def workload_cfg(spacing=1.0, omega=0.0):
    from redbirdpy_b200.meshgen import kuhn_box, grid_optodes

    node, elem = kuhn_box([100, 100, 50], spacing)
    return dict(node=node, elem=elem, prop=np.array([[0, 0, 1, 1], [0.01, 1.0, 0, 1.37]]),
                seg=np.ones(elem.shape[0], dtype=np.int32),
                srcpos=grid_optodes([15, 85], [15, 85], 8), srcdir=np.array([[0, 0, 1.0]]),
                detpos=grid_optodes([15, 85], [15, 85], 8, offset=(5, 5)), detdir=np.array([[0, 0, 1.0]]),
                omega=omega)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def max_over_ranks(x, world):
    import torch
    import torch.distributed as dist

    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch.distributed as dist

    if world > 1:
        dist.barrier()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def cpu_sample_port(cfg, ncol=1, maxiter=1000, tol=1e-10):
    """The oracle's port of the reference's femsolve(method='cg') on ncol
    columns of the same system (scipy CG per column, tol 1e-10, maxiter 1000:
    the reference defaults, solver.py:448-449, 717-754), one core.  The
    system comes from the oracle's femlhs / femrhs on the prepared mesh."""
    from oracle import femoracle as fo

    ocfg = {k: cfg[k] for k in ("node", "elem", "face", "area", "evol", "reff", "prop", "seg", "srcpos", "srcdir",
                                "detpos", "detdir", "omega")}
    A = fo.femlhs(ocfg, fo.deldotdel(ocfg["node"], ocfg["elem"], ocfg["evol"]))
    rhs, _, _, _ = fo.femrhs(dict(ocfg, srcpos=ocfg["srcpos"][:ncol], detpos=ocfg["detpos"][:1]))
    b = rhs[:, :ncol].toarray()
    t0 = time.perf_counter()
    fo.femsolve(A, b, method="cg", tol=tol, maxiter=maxiter)
    dt = time.perf_counter() - t0
    return ncol / dt, dt


def run_b200(args):
    import torch

    import redbirdpy_b200 as rbb
    from redbirdpy_b200 import engine

    rank, world, local = dist_setup(args.gpus)
    cfg = workload_cfg()
    cfg, sd = rbb.meshprep(cfg)
    mesh = engine.mesh_of(cfg)
    optics = engine.Optics.from_cfg(mesh, cfg)
    nrhs = cfg["srcpos"].shape[0] + cfg["detpos"].shape[0]

    def step(precision, profile=False):
        opt = engine.locate_optodes(mesh, cfg)
        B = opt.rhs(mesh)
        mat = engine.assemble(mesh, optics)
        X, info = engine.solve(mat, B, precision=precision, profile=profile)
        det = engine.getdet(mesh, opt, X)
        return det, X, info

    def timed(precision, k, w, profile=False):
        for _ in range(w):
            step(precision)
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        infos = []
        for _ in range(k):
            det, X, info = step(precision, profile)
            infos.append(info)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        barrier(world)
        return max_over_ranks(ms, world), det, infos

    clocks = ClockSampler(local)
    # mixed precision (the product form); clocks sampled during its timed region
    clocks.start()
    ms_mixed, det_mixed, infos = timed("mixed", args.steps, args.warmup, profile=True)
    clk = clocks.stop()
    # plain FP64 form, same GPU, same accuracy target
    ms_fp64, det_fp64, infos64 = timed("fp64", max(1, min(args.steps, 3)), 1)
    d64 = det_fp64.cpu().numpy()
    dmx = det_mixed.cpu().numpy()
    rel_err = float(np.max(np.abs(dmx - d64) / np.abs(d64)))

    # roofline of the SpMM kernel (dominant bytes per Krylov iteration)
    n, nnz, k = mesh.nn, mesh.nnz, nrhs
    spmm_bytes = nnz * (4 + 4) + 4 * (n + 1) + 2 * k * n * 4
    upd_bytes = 6 * k * n * 4 + 4 * n
    sp_ms = sum(i["spmm_ms"] for i in infos) / max(1, sum(i["spmm_launches"] for i in infos))
    up_ms = sum(i["update_ms"] for i in infos) / max(1, sum(i["update_launches"] for i in infos))
    peak, peak_kind = peaks()
    sp_gbs = spmm_bytes / (sp_ms * 1e-3) / 1e9 if sp_ms > 0 else None
    up_gbs = upd_bytes / (up_ms * 1e-3) / 1e9 if up_ms > 0 else None

    # assembly alone (femlhs kernel pair), CUDA events around 10 launches
    for _ in range(2):
        engine.assemble(mesh, optics)
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ea.record()
    for _ in range(10):
        engine.assemble(mesh, optics)
    eb.record()
    torch.cuda.synchronize()
    asm_ms = ea.elapsed_time(eb) / 10
    ne, nf = mesh.ne, mesh.nf
    pk = 8 if optics.kind == 0 else 8  # mua/musp per entity
    nprop = mesh.nn if optics.kind == 0 else ne
    asm_bytes = (ne * (16 + 80 + 8 + 16) + nprop * (2 * pk + 8) + nnz * (4 + 8 + 4) + n * (4 * 3 + 12)
                 + nf * (12 + 8 + 12))
    asm_gbs = asm_bytes / (asm_ms * 1e-3) / 1e9

    # end to end through the public API (host arrays in, numpy out)
    host_cfg = cfg
    for _ in range(1):
        rbb.runforward(host_cfg)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    ke = max(1, min(args.steps, 3))
    for _ in range(ke):
        det_h, phi_h = rbb.runforward(host_cfg)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / ke, world)
    h2d = (2 * mesh.ne * 8) + 128 * 3 * 8
    d2h = det_h.nbytes + phi_h.nbytes

    it = infos[-1]
    out = {
        "metric": METRIC, "value": round(world * nrhs / (ms_mixed * 1e-3), 3), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": {"workload": "box 100x100x50 mm, 1 mm Kuhn (520251 nodes, 3000000 tets), 64 src + 64 det, CW",
                   "nnz": nnz, "nrhs": nrhs, "precision": "mixed (FP32 Jacobi-PCG in FP64 refinement)",
                   "l2": "working set > L2 (5 x 266 MB vectors), no flush", "parallelism": f"replicas x{world}"},
        "fp64_value": round(world * nrhs / (ms_fp64 * 1e-3), 3), "fp64_ms_per_step": round(ms_fp64, 3),
        "mixed_speedup_vs_fp64": round(ms_fp64 / ms_mixed, 3),
        "det_max_rel_err_vs_fp64": rel_err,
        "krylov": {"iters": it["iters"], "sweeps": it["outer"], "relres": it["relres"], "flag": it["flag"],
                   "fp64_iters": infos64[-1]["iters"]},
        "gpu_launches": int(sum(i["launches"] for i in infos) / len(infos)) + 6,
        "roofline": {"bound": "hbm", "kernel": "spmm_kernel<float> (CSR SpMM, 128 RHS, fused p.Ap)",
                     "achieved": round(sp_gbs, 1) if sp_gbs else None, "peak": peak, "unit": "GB/s",
                     "frac": round(sp_gbs / peak, 4) if sp_gbs else None, "peak_source": peak_kind,
                     "algorithmic_bytes": spmm_bytes, "launch_ms": round(sp_ms, 4), "traffic": None},
        "roofline_update": {"kernel": "cg_update_kernel<float>", "achieved": round(up_gbs, 1) if up_gbs else None,
                            "unit": "GB/s", "frac": round(up_gbs / peak, 4) if up_gbs else None,
                            "algorithmic_bytes": upd_bytes, "launch_ms": round(up_ms, 4)},
        "roofline_assembly": {"kernel": "femlhs_rows_kernel (+ dcoeff prologue)", "achieved": round(asm_gbs, 1),
                              "unit": "GB/s", "frac": round(asm_gbs / peak, 4), "algorithmic_bytes": asm_bytes,
                              "launch_ms": round(asm_ms, 4)},
        "e2e": {"value": round(world * nrhs / e2e_s, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(d2h)},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        v, dt = cpu_sample_port(cfg, ncol=1)
        out["cpu_baseline"] = {"value": round(v, 5), "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"1 of 128 columns, oracle port of femsolve(method='cg') "
                                         f"tol 1e-10 maxiter 1000 (scipy CG), {dt:.1f} s"}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def _ref_worker(args):
    path, col, tol, maxiter = args
    import numpy as np
    from scipy import sparse
    from scipy.sparse.linalg import cg

    z = np.load(path)
    A = sparse.csr_matrix((z["data"], z["indices"], z["indptr"]))
    b = z["rhs"][:, col]
    t0 = time.perf_counter()
    x, info = cg(A, b, rtol=tol, maxiter=maxiter)
    return time.perf_counter() - t0, info


def run_reference(args):
    """The reference's CPU path for this workload on the host cores (the
    oracle port; the reference itself is Python and is not present on the
    GPU machine): femsolve(method='cg') per column in a process pool, like
    redbirdpy's _iterative_parallel (solver.py:310-377), one column per core
    per step, reference defaults tol 1e-10 / maxiter 1000."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    import tempfile

    from oracle import femoracle as fo

    cfg = workload_cfg()
    ocfg, _ = fo.meshprep(cfg)
    A = fo.femlhs(ocfg, fo.deldotdel(ocfg["node"], ocfg["elem"], ocfg["evol"]))
    rhs, _, _, _ = fo.femrhs(ocfg)
    ncore = os.cpu_count() or 1
    tmp = os.path.join(tempfile.gettempdir(), f"rb_ref_{os.getpid()}.npz")
    np.savez(tmp, data=A.data, indices=A.indices, indptr=A.indptr, rhs=rhs.toarray())
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(ncore) as pool:
        col = 0
        for s in range(args.warmup + args.steps):
            jobs = [(tmp, (col + j) % 128, 1e-10, 1000) for j in range(ncore)]
            col += ncore
            t0 = time.perf_counter()
            pool.map(_ref_worker, jobs)
            dt = time.perf_counter() - t0
            if s >= args.warmup:
                times.append(dt)
    os.remove(tmp)
    ms = 1e3 * float(np.mean(times))
    v = ncore / (ms * 1e-3)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "box 100x100x50 mm, 1 mm Kuhn (520251 nodes, 3000000 tets), 64 src + 64 det, CW",
                   "solver": "scipy CG per column (reference femsolve method='cg'), tol 1e-10, maxiter 1000"},
        "cpu_baseline": {"value": round(v, 5), "unit": UNIT, "cores": ncore, "kind": "port",
                         "sample": f"{ncore} columns per step, one per core"},
        "e2e": {"value": round(v, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()

"""Differentiable forward model: per-node (mua, D) -> detector values, with a
hand-written adjoint backward (a ``torch.autograd.Function``).

The forward pass is runforward's pipeline on the device (femrhs, femlhs with
node-based properties, femsolve, femgetdet; redbirdpy/forward.py:40-87).
Sources and detectors are solved as one block of right-hand sides, so the
detector fields phi_d - the adjoint fields that redbirdpy's jac contracts
with the source fields (redbirdpy/forward.py:509-569) - come out of the same
solve.  For a real loss L of detval[d, s] with upstream gradient g (PyTorch's
convention: g = dL/dRe + i dL/dIm for complex detector values):

    dL/dp_n = Re sum_s phi_s^T (-dA/dp_n) lambda_s,
    lambda_s = sum_d conj(g[d, s]) phi_d = A^-1 sum_d conj(g[d, s]) b_d

(A is symmetric, complex-symmetric in the frequency domain).  lambda is the
transposed solve of the backward, formed from the detector columns already in
hand; ``resolve=True`` solves A lambda_s = sum_d conj(g[d, s]) b_d afresh
instead.  The contraction is rb_jac's per-node bilinear form evaluated on the
(source, lambda) column pairs, with the exact derivatives of the node-based
assembly: 'mua_nodal' (mua at fixed D) and 'D' (the nodal D whose element
mean femlhs uses, redbirdpy/forward.py:177-228).
"""

import numpy as np
import torch

from . import engine
from .solver import solver_options

__all__ = ["DeviceModel", "BatchModel", "CapturedStep", "detector_values"]


class DeviceModel:
    """Mesh, optodes and solver settings of one differentiable forward model.

    Right-hand-side columns are [sources | detectors] (``S`` and ``D`` of
    them); ``getdet`` gives the detector values as (detector rows) x S, and
    ``row0``/``det0`` delimit the instances (one here, many in BatchModel)."""

    def __init__(self, cfg, precision="mixed", **solver_kw):
        props = np.atleast_2d(np.asarray(cfg["prop"], dtype=np.float64))
        self.mesh = engine.mesh_of(cfg)
        if props.shape[0] != self.mesh.nn:
            raise ValueError("detector_values needs node-based properties (one prop row per node)")
        self.nref = _nref_of(props[:, 3] if props.shape[1] >= 4 else np.full(props.shape[0], 1.37), self.mesh.device)
        self.omega = float(cfg.get("omega", 0) or 0)
        self.reff = cfg.get("reff", 0.493)
        self.opt = engine.locate_optodes(self.mesh, cfg)
        if self.opt.nsrc < 1 or self.opt.ndet < 1:
            raise ValueError("Must define at least one source and detector")
        if self.opt.nsrc > 64 or self.opt.ndet > 64:
            raise ValueError("detector_values handles at most 64 sources and 64 detectors")
        self.S, self.D = self.opt.nsrc, self.opt.ndet
        self.B = self.opt.rhs(self.mesh)
        dev = self.mesh.device
        self.row0 = torch.tensor([0, self.mesh.nn], dtype=torch.int64, device=dev)
        self.det0 = torch.tensor([0, self.D], dtype=torch.int64, device=dev)
        self.ninst = 1
        self.solve_kw = dict(solver_options(solver_kw), precision=precision)

    def optics(self, mua, dcoef):
        """Optics with node mua and D (musp = 1/(3D) - mua, so that femlhs's
        D = 1/(3(mua + musp)) returns the given D)."""
        musp = 1.0 / (3.0 * dcoef) - mua
        return engine.Optics(self.mesh, mua.contiguous(), musp.contiguous(), self.nref, self.omega, self.reff)

    def fields(self, mua, dcoef):
        mat = engine.assemble(self.mesh, self.optics(mua, dcoef))
        phi, info = engine.solve(mat, self.B, **self.solve_kw)
        if info["flag"] is None:  # fixed budget: the outcome stays on the device
            self.status = info["inst_status"]
        elif info["flag"] != 0:
            raise RuntimeError(f"forward solve did not converge (flag {info['flag']})")
        return phi, mat

    def getdet(self, phi):
        return engine.getdet(self.mesh, self.opt, phi)

    def calibrate_budget(self, mua, dcoef, margin=1.25):
        """A fixed solve budget (sweeps, iterations per sweep) for this model
        at these properties: one solve with host checks, its sweep count and
        the most iterations a sweep took, times ``margin``.  Cached per
        (nn, nnz, columns) bucket so that models of one size share it."""
        key = (self.mesh.nn, self.mesh.nnz, int(self.B.shape[1]), self.solve_kw.get("precision"),
               self.solve_kw.get("spmm_lanes", 0))
        hit = _BUDGETS.get(key)
        if hit is not None:
            return hit
        kw = {k: v for k, v in self.solve_kw.items() if k != "budget"}
        mat = engine.assemble(self.mesh, self.optics(mua.detach(), dcoef.detach()))
        _, info = engine.solve(mat, self.B, **kw)
        if info["flag"] != 0:
            raise RuntimeError(f"budget calibration: the checked solve did not converge (flag {info['flag']})")
        budget = (max(1, int(info["outer"])), max(8, int(np.ceil(margin * info["sweep_iters_max"]))))
        _BUDGETS[key] = budget
        return budget


_BUDGETS = {}


def _nref_of(nref, dev):
    """A per-node refractive index on the device, or the scalar when uniform
    (uploaded once per model, not per assembly)."""
    nref = np.asarray(nref, dtype=np.float64)
    if nref.size and np.ptp(nref) == 0:
        return float(nref.ravel()[0])
    return torch.as_tensor(nref, device=dev)


class BatchModel(DeviceModel):
    """Many independent meshes as one block-diagonal system: one assembly,
    one multi-RHS solve and one adjoint contraction for all of them.

    Instance i's nodes, tets and faces follow those of instance i-1 (indices
    offset, coordinates untouched, so every element's geometry is its own).
    Right-hand-side column j < S is source j of every instance that has one
    (zero elsewhere), column S + j detector j: the solve needs
    max(sources) + max(detectors) columns however many instances there are,
    and the block-diagonal matrix keeps the instances' fields apart.  All
    instances share omega and the boundary reflection coefficient."""

    def __init__(self, cfgs, precision="mixed", strict=True, **solver_kw):
        """``strict``: a forward solve in which any instance fails raises
        (the reference's error behaviour); with ``strict=False`` the outcome
        of every instance is only recorded in ``status`` (see fields)."""
        from .utility import getoptodes

        self.strict = strict

        if not cfgs:
            raise ValueError("BatchModel needs at least one instance")
        nns = [c["node"].shape[0] for c in cfgs]
        nes = [c["elem"].shape[0] for c in cfgs]
        self.node_off = np.concatenate([[0], np.cumsum(nns)])
        self.elem_off = np.concatenate([[0], np.cumsum(nes)])
        node = np.vstack([np.asarray(c["node"], dtype=np.float64)[:, :3] for c in cfgs])
        elem = np.vstack([np.asarray(c["elem"])[:, :4].astype(np.int64) + o for c, o in zip(cfgs, self.node_off)])
        face = np.vstack([np.asarray(c["face"])[:, :3].astype(np.int64) + o for c, o in zip(cfgs, self.node_off)])
        area = np.concatenate([np.asarray(c["area"], dtype=np.float64) for c in cfgs])
        evol = np.concatenate([np.asarray(c["evol"], dtype=np.float64) for c in cfgs])
        omegas = {float(c.get("omega", 0) or 0) for c in cfgs}
        reffs = {float(c.get("reff", 0.493)) for c in cfgs}
        if len(omegas) != 1 or len(reffs) != 1:
            raise ValueError("batched instances must share omega and reff")
        self.omega, self.reff = omegas.pop(), reffs.pop()
        props = [np.atleast_2d(np.asarray(c["prop"], dtype=np.float64)) for c in cfgs]
        if any(p.shape[0] != n for p, n in zip(props, nns)):
            raise ValueError("detector_values needs node-based properties (one prop row per node)")
        nref = np.concatenate([p[:, 3] if p.shape[1] >= 4 else np.full(p.shape[0], 1.37) for p in props])
        self.mesh = engine.DeviceMesh(node, elem, face, area, evol)
        dev = self.mesh.device
        self.nref = _nref_of(nref, dev)
        # optodes: located among each instance's own tets
        self.ns, self.nd = [], []
        locs, barys = [], []
        for i, c in enumerate(cfgs):
            src, det, _, _ = getoptodes(c)
            pts = np.vstack([src, det])
            self.ns.append(src.shape[0])
            self.nd.append(det.shape[0])
            pt = torch.as_tensor(pts, dtype=torch.float64, device=dev)
            loc = torch.empty(pts.shape[0], dtype=torch.int32, device=dev)
            bary = torch.empty((pts.shape[0], 4), dtype=torch.float64, device=dev)
            e0, e1 = int(self.elem_off[i]), int(self.elem_off[i + 1])
            engine.call("rb_tsearch", engine.ptr(self.mesh.node), engine.ptr(self.mesh.elem[e0:e1]), e1 - e0,
                        engine.ptr(pt), pts.shape[0], engine.ptr(loc), engine.ptr(bary), engine.stream())
            locs.append(torch.where(loc >= 0, loc + e0, loc))
            barys.append(bary)
        self.S, self.D = max(self.ns), max(self.nd)
        if self.S + self.D > 128:
            raise ValueError("batched instances: at most 128 source + detector columns")
        self.B = torch.zeros((self.mesh.nn, self.S + self.D), dtype=torch.float64, device=dev)
        for i in range(len(cfgs)):
            ns, nd = self.ns[i], self.nd[i]
            for lo, cnt, col0 in ((0, ns, 0), (ns, nd, self.S)):
                engine.call("rb_point_rhs", engine.ptr(self.mesh.elem), engine.ptr(locs[i][lo:lo + cnt]),
                            engine.ptr(barys[i][lo:lo + cnt]), cnt, self.mesh.nn, self.S + self.D, col0,
                            engine.ptr(self.B), engine.stream())
        self.loc_det = torch.cat([l[n:] for l, n in zip(locs, self.ns)]).contiguous()
        self.bary_det = torch.cat([b[n:] for b, n in zip(barys, self.ns)]).contiguous()
        self.row0 = torch.as_tensor(self.node_off, dtype=torch.int64, device=dev)
        self.det0_host = np.concatenate([[0], np.cumsum(self.nd)]).astype(np.int64)
        self.det0 = torch.as_tensor(self.det0_host, device=dev)
        self.ninst = len(cfgs)
        # the (detector row, source column) entries that are an instance's own
        # pairs; the rest of the block-diagonal detector matrix pairs one
        # instance's detector with another's source column
        own = np.zeros((int(self.det0_host[-1]), self.S), dtype=bool)
        for i in range(self.ninst):
            own[self.det0_host[i]:self.det0_host[i + 1], :self.ns[i]] = True
        self.own = torch.as_tensor(own, device=dev)
        self.solve_kw = dict(solver_options(solver_kw), precision=precision)
        # Jacobi alone unless asked: the position-binned coarse space would put
        # nodes of overlapping instances into one aggregate, coupling blocks
        # that are independent (and were slower: 337 ms against 259 ms for the
        # 256-instance batch of 2.7M nodes)
        self.solve_kw.setdefault("coarse", False)
        # convergence judged per instance: each instance's residual against
        # its own right-hand side, whatever the others' sizes and scales
        self.instances = engine.Instances(self.node_off, dev)
        self.solve_kw["instances"] = self.instances
        if precision == "fp64":
            # the FP64 form is the accuracy reference of the batch: each
            # instance is refined to its own FP64 floor (a sweep that no
            # longer gains 4x ends it), as far-field detector values 1e-11
            # of an instance's largest need; at 1e-15 relative residual they
            # carried errors up to 5e-6
            self.solve_kw.setdefault("tol", 1e-17)
        self.status = None

    def tune(self, mua, dcoef):
        """Pick the solve's launch shapes for this batch with the autotuner
        (engine.SolveTuner; cached per size bucket) and keep them."""
        mat = engine.assemble(self.mesh, self.optics(mua.detach(), dcoef.detach()))
        self.solve_kw.update(engine.solve_tuner.options(mat, self.B, **self.solve_kw))
        return self.solve_kw

    def fields(self, mua, dcoef):
        """Fields of every instance.  An instance whose properties hold a
        non-finite value or a non-positive D is solved on stand-in properties
        (mua 0.01/mm, D 1/3.03 mm) so that its rows cannot spoil the shared
        Krylov scalars of the others, and its status is set to 3
        (non-finite); its values are not valid."""
        inst = self.instances.row_inst.long()
        bad_row = ~(torch.isfinite(mua) & torch.isfinite(dcoef) & (dcoef > 0))
        bad_inst = torch.zeros(self.ninst, dtype=torch.int32, device=mua.device)
        bad_inst.index_add_(0, inst, bad_row.to(torch.int32))
        bad_inst = bad_inst > 0
        iso = bad_inst[inst]
        mua = torch.where(iso, torch.full_like(mua, 0.01), mua)
        dcoef = torch.where(iso, torch.full_like(dcoef, 1.0 / 3.03), dcoef)
        mat = engine.assemble(self.mesh, self.optics(mua, dcoef))
        phi, info = engine.solve(mat, self.B, **self.solve_kw)
        self.status, self.relres = info["inst_status"], info["inst_relres"]
        if info["flag"] is None:  # fixed budget: read the status words later
            self.status = torch.where(bad_inst, torch.full_like(self.status, 3), self.status)
            return phi, mat
        self.status = np.where(bad_inst.cpu().numpy(), 3, self.status).astype(np.int32)
        bad = np.flatnonzero(self.status)
        if bad.size and not self.strict:
            return phi, mat
        if bad.size:
            desc = ", ".join(f"{i}: {engine.INSTANCE_STATUS[int(self.status[i])]}" for i in bad[:8])
            raise RuntimeError(f"forward solve failed for {bad.size} instance(s) ({desc})")
        return phi, mat

    def getdet(self, phi):
        """All instances' detector values: row det0[i] + d, column s."""
        kind = engine._lib.RB_C128 if phi.is_complex() else engine._lib.RB_F64
        nd = int(self.det0_host[-1])
        out = torch.empty((nd, self.S), dtype=phi.dtype, device=phi.device)
        engine.call("rb_femgetdet", engine.ptr(self.mesh.elem), engine.ptr(self.loc_det), engine.ptr(self.bary_det),
                    nd, engine.ptr(phi), phi.shape[1], self.S, kind, engine.ptr(out), engine.stream())
        return out

    def split(self, det):
        """Per-instance (ndet_i x nsrc_i) views of getdet's output."""
        d0 = self.det0_host
        return [det[d0[i]:d0[i + 1], :self.ns[i]] for i in range(self.ninst)]

    def node_slices(self, v):
        return [v[self.node_off[i]:self.node_off[i + 1]] for i in range(self.ninst)]


class _DetectorValues(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mua, dcoef, model, resolve):
        phi, mat = model.fields(mua.detach(), dcoef.detach())
        det = model.getdet(phi)
        ctx.model, ctx.resolve, ctx.mat = model, resolve, mat
        ctx.save_for_backward(phi)
        return det

    @staticmethod
    def backward(ctx, g):
        (phi,) = ctx.saved_tensors
        model = ctx.model
        S, D = model.S, model.D
        g = g.to(phi.dtype).contiguous()
        if ctx.resolve:
            # transposed solve: A lambda_s = sum_d conj(g[d, s]) b_d; the
            # solver takes real right-hand sides, so complex ones go as Re, Im
            gc = g.conj() if phi.is_complex() else g
            bd = model.B[:, S:S + D]
            if phi.is_complex():
                lr, _ = engine.solve(ctx.mat, (bd @ gc.real).contiguous(), **model.solve_kw)
                li, _ = engine.solve(ctx.mat, (bd @ gc.imag).contiguous(), **model.solve_kw)
                lam = lr + 1j * li
            else:
                lam, _ = engine.solve(ctx.mat, (bd @ gc).contiguous(), **model.solve_kw)
        else:
            # the detector columns are A^-1 b_d already
            lam = torch.empty((phi.shape[0], S), dtype=phi.dtype, device=phi.device)
            kind = engine._lib.RB_C128 if phi.is_complex() else engine._lib.RB_F64
            engine.call("rb_adjoint_fields", engine.ptr(phi), phi.shape[0], phi.shape[1], S, engine.ptr(g), S,
                        engine.ptr(model.row0), engine.ptr(model.det0), model.ninst, kind, engine.ptr(lam),
                        engine.stream())
        fields = torch.cat([phi[:, :S], lam], dim=1).contiguous()
        pairs = np.column_stack([np.arange(S), S + np.arange(S), np.ones(S, dtype=np.int64)])
        grads = []
        for what, need in (("mua_nodal", ctx.needs_input_grad[0]), ("D", ctx.needs_input_grad[1])):
            if not need:
                grads.append(None)
                continue
            J = engine.jacobian(model.mesh, fields, pairs, what, out_dtype=torch.float64)
            grads.append((J.real if J.is_complex() else J).sum(dim=0))
        return grads[0], grads[1], None, None


def detector_values(model, mua, dcoef, resolve=False):
    """Detector values of the node-based forward model at per-node ``mua``
    and ``dcoef`` (D, mm), differentiable in both through the adjoint
    backward: (ndet x nsrc) for a DeviceModel, all instances' detector rows x
    max(nsrc) for a BatchModel (``split`` gives the per-instance blocks).
    Real for CW, complex in the frequency domain."""
    return _DetectorValues.apply(mua, dcoef, model, resolve)


class CapturedStep:
    """Forward plus adjoint gradient of a loss, captured once as a CUDA graph
    and replayed per call.

    The solves run on a fixed budget (sweeps x iterations per sweep, see
    engine.solve), so nothing in the step waits for the host; the budget
    comes from ``model.calibrate_budget`` (one checked solve, with margin)
    unless given.  ``loss_fn(det)`` maps the model's detector values to a
    scalar with torch operations.  A call copies ``mua`` / ``dcoef`` into the
    captured inputs, replays the graph and returns (loss, det, dL/dmua,
    dL/dD), device tensors that the next call overwrites.  ``status`` holds
    the per-instance outcome of the last replay's forward solve (0
    converged; see engine.INSTANCE_STATUS); check it before trusting a
    result, since a fixed budget can end before convergence."""

    def __init__(self, model, loss_fn, mua, dcoef, budget=None, warmup=2):
        if budget is None:
            budget = model.calibrate_budget(mua, dcoef)
        self.budget = tuple(budget)
        self.model = model
        self.solve_kw_checked = model.solve_kw
        model.solve_kw = dict(model.solve_kw, budget=self.budget)
        if "instances" not in model.solve_kw:
            model.solve_kw["instances"] = engine.Instances([0, model.mesh.nn], model.mesh.device)
        self.mua = mua.detach().clone().requires_grad_(True)
        self.dco = dcoef.detach().clone().requires_grad_(True)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self.mua.grad = self.dco.grad = None
                loss_fn(detector_values(model, self.mua, self.dco)).backward()
        torch.cuda.current_stream().wait_stream(side)
        self.mua.grad = self.dco.grad = None
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.det = detector_values(model, self.mua, self.dco)
            self.loss = loss_fn(self.det)
            self.loss.backward()
        self.gmua, self.gdco = self.mua.grad, self.dco.grad
        self.status = model.status

    def __call__(self, mua, dcoef):
        with torch.no_grad():
            self.mua.copy_(mua)
            self.dco.copy_(dcoef)
        self.graph.replay()
        return self.loss, self.det, self.gmua, self.gdco

    def release(self):
        """Drop the graph and give the model back its checked solves."""
        self.graph = None
        self.model.solve_kw = self.solve_kw_checked

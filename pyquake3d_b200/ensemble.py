"""Ensembles of independent faults on one GPU.

The reference simulates one fault per (MPI) job; a batch of independent faults
is run as separate jobs.  Here a batch shares the device: the H-matrices of all
faults form one block-diagonal operator (one set of matvec work items, one
launch), and one cooperative step kernel (pq3d_ens_step) advances every fault
with its own DP5(4) step-size controller, exactly as QDsim.simu_forward
(src/QDsim.py:892-996) advances a single fault.

Layout: fault f owns the contiguous tree-order rows [row0[f], row0[f] + n_f),
ordered by its own cluster tree; the combined element numbering concatenates
the faults in the same order.  Fault f's ACA starting rows/columns are the ones
its own QDsim would draw (seed `ACA seed` of its parameter file), so each
fault's operator entries are those of the fault assembled alone.
"""
import numpy as np

from . import _lib
from ._lib import check, ptr
from .hmatrix import ClusterNode, LeafBlock, DeviceHMatrix, aca_start_indices, pack_x


def _copy_tree(root, off):
    """Copy of a cluster tree with tree positions and element ids shifted by off."""
    mapping = {}
    st = [root]
    order = []
    while st:
        nd = st.pop()
        order.append(nd)
        if nd.left is not None:
            st.append(nd.right)
            st.append(nd.left)
    for nd in order:
        c = ClusterNode(nd.indices + off, nd.level)
        c.start = nd.start + off
        c.bbox_min, c.bbox_max = nd.bbox_min, nd.bbox_max
        c.leaf_id = nd.leaf_id
        mapping[id(nd)] = c
    for nd in order:
        if nd.left is not None:
            mapping[id(nd)].left = mapping[id(nd.left)]
            mapping[id(nd)].right = mapping[id(nd.right)]
    return mapping


class EnsembleStructure:
    """Block-diagonal union of per-fault HStructures (the interface DeviceHMatrix
    and build_plan_arrays read: n, perm, iperm, leaves, blocks, aca_starts)."""

    def __init__(self, structs, seeds):
        self.faults = len(structs)
        self.sizes = np.array([s.n for s in structs], dtype=np.int64)
        self.row0 = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.n = int(self.row0[-1])
        self.mini_leaf = structs[0].mini_leaf
        self.eta = structs[0].eta
        self.min_size = structs[0].min_size
        if any((s.mini_leaf, s.eta, s.min_size) != (self.mini_leaf, self.eta, self.min_size) for s in structs):
            raise _lib.Pq3dError("ensemble faults must share the H-matrix parameters")
        self.perm = np.concatenate([s.perm + o for s, o in zip(structs, self.row0)])
        self.iperm = np.empty_like(self.perm)
        self.iperm[self.perm] = np.arange(self.n)
        self.leaves, self.blocks, self.aca_starts = [], [], []
        for s, o, seed in zip(structs, self.row0, seeds):
            m = _copy_tree(s.row_root, int(o))
            for lf in s.leaves:
                c = m[id(lf)]
                c.leaf_id = len(self.leaves)
                self.leaves.append(c)
            for b in s.blocks:
                self.blocks.append(LeafBlock(m[id(b.row)], m[id(b.col)], b.aca, b.admissible, b.level))
            self.aca_starts += aca_start_indices(s.blocks, seed)

    def fault_of_row(self):
        return np.repeat(np.arange(self.faults), self.sizes)


def ensemble_tasks(row0, task_rows):
    """CTA tasks of the ensemble step kernel: consecutive chunks of at most
    task_rows rows, never spanning two faults.  Returns (task_row: T+1 row
    boundaries, task_fault: fault of each task, fault_task: M+1 task offsets)."""
    row0 = np.asarray(row0, dtype=np.int64)
    M = len(row0) - 1
    starts, fault = [], []
    for f in range(M):
        for r in range(int(row0[f]), int(row0[f + 1]), task_rows):
            starts.append(r)
            fault.append(f)
    task_row = np.array(starts + [int(row0[-1])], dtype=np.int32)
    task_fault = np.array(fault, dtype=np.int32)
    fault_task = np.searchsorted(task_fault, np.arange(M + 1), side="left").astype(np.int32)
    return task_row, task_fault, fault_task


class Ensemble:
    """Independent faults (QDsim objects, host-initialized) stepped together."""

    FIELDS = ["Tno", "Tt1o", "Tt2o", "psi", "slip1", "slip2", "slipv1", "slipv2", "slipv", "rake", "Tt", "fric", "slip"]
    CONST = ["a", "b", "dc", "f0", "shear_loading", "normal_loading", "vplc", "cr0", "sr0"]

    def __init__(self, sims, precision="fp32", want=None, device="cuda", share=None):
        """sims: host-initialized QDsim objects of the faults.  share: another Ensemble
        of the same faults whose assembled operator is reused (its plans must
        include `precision`)."""
        import torch
        self.torch = torch
        self.L = _lib.load()
        self.sims = list(sims)
        self.precision = precision
        s0 = self.sims[0]
        from .qdsim import hs_mode
        for s in self.sims:
            same = (s.mu, s.lambda_, s.V0, s.Cs, s.RelTol, bool(s.fix_Tn), hs_mode(s))
            if same != (s0.mu, s0.lambda_, s0.V0, s0.Cs, s0.RelTol, bool(s0.fix_Tn), hs_mode(s0)):
                raise _lib.Pq3dError("ensemble faults must share elastic constants, V0, RelTol, Fix_Tn and "
                                     "the half-space setting")
        P = s0.Para0
        if share is not None:
            if len(share.sims) != len(self.sims):
                raise _lib.Pq3dError("shared ensemble has another number of faults")
            self.struct, self.op = share.struct, share.op
        else:
            seeds = [int(s.Para0.get("ACA seed", 0)) for s in self.sims]
            self.struct = EnsembleStructure([s.tree_block.struct for s in self.sims], seeds)
            xg = np.concatenate([s.xg for s in self.sims])
            ev = np.concatenate([s.eleVec for s in self.sims])
            noff = np.concatenate([[0], np.cumsum([len(s.nodelst) for s in self.sims])])
            nodes = np.concatenate([s.nodelst for s in self.sims])
            tri = np.concatenate([np.asarray(s.elelst) + o for s, o in zip(self.sims, noff)])
            tol = float(P.get("ACA tolerance", 0.01))
            rel = P.get("ACA relative tolerance", "False") == "True"
            want = tuple(want or (("fp64",) if precision == "fp64" else ("fp64", precision)))
            self.op = DeviceHMatrix(self.struct, xg, ev, nodes, tri, s0.mu, s0.lambda_, device=device, aca_tol=tol,
                                    aca_rel=rel, halfspace=hs_mode(s0)).assemble(want)
        self.n = n = self.struct.n
        self.M = M = self.struct.faults
        self.perm = self.struct.perm
        dev = self.op.dev
        f64 = dict(dtype=torch.float64, device=dev)

        def cat(get):
            return np.concatenate([np.broadcast_to(np.asarray(get(s), dtype=np.float64), (len(s.xg),))
                                   for s in self.sims])[self.perm]
        getters = dict(Tno=lambda s: s.Tno, Tt1o=lambda s: s.Tt1o, Tt2o=lambda s: s.Tt2o, psi=lambda s: s.state,
                       slip1=lambda s: s.slip1, slip2=lambda s: s.slip2, slipv1=lambda s: s.slipv1,
                       slipv2=lambda s: s.slipv2, slipv=lambda s: s.slipv, rake=lambda s: s.rake,
                       Tt=lambda s: np.sqrt(s.Tt1o * s.Tt1o + s.Tt2o * s.Tt2o), fric=lambda s: s.fric,
                       slip=lambda s: s.slip, a=lambda s: s.a, b=lambda s: s.b, dc=lambda s: s.dc, f0=lambda s: s.f0,
                       shear_loading=lambda s: s.shear_loading, normal_loading=lambda s: s.normal_loading,
                       vplc=lambda s: s.slipvC, cr0=lambda s: np.cos(s.rake0), sr0=lambda s: np.sin(s.rake0))
        self.t = {k: torch.tensor(np.ascontiguousarray(cat(g)), **f64) for k, g in getters.items()}
        task_row, task_fault, fault_task = ensemble_tasks(self.struct.row0, self.L.pq3d_ens_task_rows())
        self.n_tasks = T = len(task_fault)
        self.task_row = torch.tensor(task_row, device=dev)
        self.task_fault = torch.tensor(task_fault, device=dev)
        self.fault_task = torch.tensor(fault_task, device=dev)
        self.grid = self.L.pq3d_ens_grid(T)
        if self.grid <= 0:
            raise _lib.Pq3dError("pq3d_ens_grid failed")
        self.y = torch.zeros((n, 3), **f64)
        self.cand = torch.zeros(4 * n, **f64)
        self.tmax = torch.zeros(4 * T, **f64)
        self.ctrl = torch.zeros((M, 16), **f64)
        self.fstate = torch.zeros((M, 8), **f64)
        self.bar = torch.zeros(4, dtype=torch.int32, device=dev)
        self.hist = None
        self.hist_cap = 0
        self.hforce = None
        self.hforce_cap = 0
        self.x = self.op.new_x(precision)
        vp = cat(lambda s: s.slipvC)
        x0 = pack_x(cat(lambda s: s.slipv1) - vp * cat(lambda s: np.cos(s.rake0)),
                    cat(lambda s: s.slipv2) - vp * cat(lambda s: np.sin(s.rake0)), n)
        self.x.copy_(torch.tensor(x0, dtype=self.x.dtype))
        self.steps = 0
        A = np.zeros(1, dtype=_lib.ENS_ARGS)
        for k in self.FIELDS + self.CONST:
            A[k] = self.t[k].data_ptr()
        for k in ("y", "cand", "x", "task_row", "task_fault", "fault_task", "tmax", "ctrl", "fstate", "bar"):
            A[k] = getattr(self, k).data_ptr()
        Pl = self.op.plan(precision)
        A["slots"] = Pl["slots"].data_ptr()
        for k in ("leaf_of_row", "leaf_ptr", "leaf_off"):
            A[k] = Pl[k].data_ptr()
        A["n"], A["n_faults"], A["n_tasks"] = n, M, T
        A["fix_tn"] = 1 if s0.fix_Tn else 0
        A["x_fp32"] = 0 if self.x.dtype == torch.float64 else 1
        A["fuse_rowsum"] = 1
        A["slots_fp32"] = 0 if Pl["acc"] == torch.float64 else 1
        A["V0"], A["eta"], A["reltol"] = s0.V0, s0.mu / (2.0 * s0.Cs), s0.RelTol
        self.args = A

    # ------------------------------------------------------------------ stepping
    def launch(self, step_index=0, stream=None):
        """Enqueue one step of every fault (matvec + ensemble step kernel), no host sync."""
        self.op.matvec(self.x, self.precision, stream=stream, slots_only=True)
        self.args["step_index"] = step_index
        self.args["hist"] = self.hist.data_ptr() if self.hist is not None and step_index < self.hist_cap else 0
        if self.hforce is not None and step_index >= self.hforce_cap:
            raise _lib.Pq3dError("dt replay shorter than the run")
        self.args["hforce"] = self.hforce.data_ptr() if self.hforce is not None else 0
        check(self.L.pq3d_ens_step(self.args.ctypes.data, self.grid, _lib.stream_ptr(stream)), "pq3d_ens_step")

    def set_history(self, nsteps):
        self.hist = self.torch.zeros((max(nsteps, 1), self.M, 6), dtype=self.torch.float64, device=self.op.dev)
        self.hist_cap = max(nsteps, 1)

    def set_replay(self, h):
        """dt replay: h[s, f] is step s of fault f (device tensor, steps x faults)."""
        h = h.to(dtype=self.torch.float64).contiguous()
        if h.dim() != 2 or h.shape[1] != self.M:
            raise _lib.Pq3dError("replay must be (steps, faults)")
        self.hforce = h
        self.hforce_cap = h.shape[0]

    def _status(self):
        c = self.ctrl.cpu().numpy()
        bad = np.nonzero(c[:, 4] != 0)[0]
        if len(bad):
            raise _lib.Pq3dError(f"time step failed for faults {bad.tolist()}: status {int(c[bad[0], 4])}")
        return c

    def step(self, dttry):
        """One step of every fault; dttry scalar or per fault.  Returns (h, dtnext) per fault."""
        self.ctrl[:, 0] = self.torch.as_tensor(np.broadcast_to(np.asarray(dttry, dtype=np.float64), (self.M,)).copy(),
                                               device=self.op.dev)
        self.launch(self.steps)
        c = self._status()
        self.steps += 1
        return c[:, 1].copy(), c[:, 0].copy()

    def run(self, nsteps, dttry):
        """nsteps steps back to back; returns the history (nsteps x faults x 6:
        h, dtnext, time, max|V1|, max|V2|, rejects)."""
        self.set_history(nsteps)
        self.ctrl[:, 0] = self.torch.as_tensor(np.broadcast_to(np.asarray(dttry, dtype=np.float64), (self.M,)).copy(),
                                               device=self.op.dev)
        for i in range(nsteps):
            self.launch(i)
        self._status()
        self.steps += nsteps
        return self.hist.cpu().numpy()[:nsteps]

    def capture(self, nsteps):
        """CUDA graph of nsteps consecutive steps (dt chained on the device)."""
        torch = self.torch
        if self.hist is None or self.hist_cap < nsteps:
            self.set_history(nsteps)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        try:
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    for i in range(nsteps):
                        self.launch(i)
        except (RuntimeError, _lib.Pq3dError):
            torch.cuda.synchronize()
            return None
        torch.cuda.current_stream().wait_stream(s)
        return g

    def time(self):
        return self.ctrl[:, 2].cpu().numpy().copy()

    def get(self, name, f):
        """Field of fault f in its own element order (FP64 host copy)."""
        a, b = int(self.struct.row0[f]), int(self.struct.row0[f + 1])
        v = self.t[name][a:b].cpu().numpy()
        local = self.perm[a:b] - a
        out = np.empty_like(v)
        out[local] = v
        return out

    def to_host(self):
        """Write every fault's state back into its QDsim attributes."""
        t = self.time()
        for f, s in enumerate(self.sims):
            s.Tno, s.Tt1o, s.Tt2o, s.state = (self.get(k, f) for k in ("Tno", "Tt1o", "Tt2o", "psi"))
            s.slip1, s.slip2, s.slip = (self.get(k, f) for k in ("slip1", "slip2", "slip"))
            s.slipv1, s.slipv2, s.slipv = (self.get(k, f) for k in ("slipv1", "slipv2", "slipv"))
            s.rake, s.Tt, s.fric = (self.get(k, f) for k in ("rake", "Tt", "fric"))
            s.time = float(t[f])

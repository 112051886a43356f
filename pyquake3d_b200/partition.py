"""Row partition of one fault's H-matrix over several GPUs, and the distributed step.

The reference spreads the H-matrix blocks over MPI ranks and sums the partial
products of every rank with a reduce (src/QDsim.py:906-922,
src/Hmatrix.py:1445-1538, BlockTree.parallel_block_scatter_send).  Here each
rank owns a contiguous range of tree-order ROWS instead:

  * cuts are placed at cluster-leaf boundaries, preferably ones that split no
    low-rank (ACA) block; a low-rank block crossing a cut is assembled by both
    ranks with the single-GPU operator's starting rows (identical factors), and
    each applies U to its own rows only; dense blocks crossing a cut are split
    by rows;
  * cuts balance the matvec bytes of each rank (dense entries of its rows, U
    rows and V of its low-rank blocks);
  * a rank computes y only for its rows and steps only its rows; the one data
    exchange per step is an all-gather of the slip-rate deficit (each rank
    contributes its rows, 2 (r1 - r0) values in tree order, (x1, x2)
    interleaved; ranks own consecutive row ranges, so the gathered pieces in
    rank order are the whole deficit), and every DP5(4) attempt reduces four
    error maxima (max over ranks, NaN flags carried separately so NaN
    propagates as in the reference).  No reduce of y.

The step orchestration (PartitionedStepper) is written against two small
interfaces: a backend per local rank (matvec, attempt over its rows, accept)
and a communicator (gather / max over all ranks).  DeviceRowBackend runs the
libpq3d.so row-range kernels; TorchComm reduces over torch.distributed ranks
(and over several local backends, which is how two ranks are emulated on one
GPU without kernels that wait on each other).
"""
import numpy as np

from . import _lib
from ._lib import check, ptr
from .hmatrix import ClusterNode, LeafBlock, DTYPES, MIXED_TOL, _CW_LR, _cdiv


# ----------------------------------------------------------------------------- host partition


def row_costs(struct, kS, kD, code):
    """Matvec bytes attributed to each tree-order row for storage code (0 FP64,
    1 FP32, 2 FP32 dense + BF16 low rank): dense entries of the row, its U rows,
    and each low-rank block's V spread evenly over the block's rows."""
    esz_d = 8 if code == 0 else 4
    esz_l = {0: 8, 1: 4, 2: 2}[code]
    d = np.zeros(struct.n + 1)
    ai = 0
    for b in struct.blocks:
        r0, m = b.row.start, len(b.row.indices)
        n = len(b.col.indices)
        if b.aca:
            k = int(kS[ai]) + int(kD[ai])
            ai += 1
            per_row = 3 * k * esz_l * (1 + n / m)
        else:
            per_row = 6 * n * esz_d
        d[r0] += per_row
        d[r0 + m] -= per_row
    return np.cumsum(d)[:-1]


def safe_cuts(struct):
    """Leaf starts (and n) that lie strictly inside no ACA block's row range:
    a cut there splits no low-rank block."""
    n = struct.n
    cand = np.array(sorted({lf.start for lf in struct.leaves} | {0, n}), dtype=np.int64)
    inside = np.zeros(n + 2, dtype=np.int64)
    for b in struct.blocks:
        if b.aca:
            s, e = b.row.start, b.row.start + len(b.row.indices)
            inside[s + 1] += 1
            inside[e] -= 1
    covered = np.cumsum(inside)[:n + 1] > 0     # covered[p]: p strictly inside some ACA row range
    return cand[~covered[cand]]


def row_partition(struct, nranks, kS=None, kD=None, code=1, k_guess=16, slack=0.02):
    """Boundaries b (nranks + 1 tree positions, b[0] = 0, b[-1] = n) at cluster-leaf
    starts, each as close as possible to an equal share of the matvec bytes.  A
    cut that splits no low-rank block is preferred when one lies within `slack`
    of the total bytes from the target; otherwise the nearest leaf start is
    taken and the low-rank blocks it splits are shared (each side computes its
    own rows of U and the whole V x).  Without ACA ranks (before assembly) every
    low-rank block is costed at k_guess per slip direction."""
    if kS is None or kD is None:
        na = sum(1 for b in struct.blocks if b.aca)
        kS = kD = np.full(na, k_guess)
    cost = row_costs(struct, kS, kD, code)
    pref = np.concatenate([[0.0], np.cumsum(cost)])
    leaves = np.array(sorted({lf.start for lf in struct.leaves} | {0, struct.n}), dtype=np.int64)
    safe = safe_cuts(struct)
    total = pref[-1]
    b = [0]
    for r in range(1, nranks):
        target = total * r / nranks
        ok = safe[safe > b[-1]]
        if len(ok):
            j = int(np.argmin(np.abs(pref[ok] - target)))
            if abs(pref[ok[j]] - target) <= slack * total:
                b.append(int(ok[j]))
                continue
        ok = leaves[leaves > b[-1]]
        ok = ok if len(ok) else np.array([struct.n])
        b.append(int(ok[int(np.argmin(np.abs(pref[ok] - target)))]))
    b.append(struct.n)
    return np.array(b, dtype=np.int64)


class _ClippedAca(LeafBlock):
    """A low-rank block shared by two ranks: assembled whole (same ACA factors on
    both), U applied to the block-local rows [rows[0], rows[1]) only."""
    __slots__ = ("rows",)

    def __init__(self, b, lo, hi):
        super().__init__(b.row, b.col, True, b.admissible, b.level)
        self.rows = (int(lo), int(hi))


class _RowNode:
    """Cluster node restricted to a row sub-range (dense blocks crossing a cut)."""
    __slots__ = ("indices", "start")

    def __init__(self, indices, start):
        self.indices = indices
        self.start = start


class RankStructure:
    """The blocks of one rank (rows [r0, r1) of a global HStructure or
    EnsembleStructure): whole ACA blocks, dense blocks clipped to the rows.
    Columns, leaves and the permutation stay global, so x and y keep the global
    layout and rows outside [r0, r1) simply get no contributions."""

    def __init__(self, struct, r0, r1, seed=0):
        self.n = struct.n
        self.perm, self.iperm = struct.perm, struct.iperm
        self.leaves = struct.leaves
        self.mini_leaf, self.eta, self.min_size = struct.mini_leaf, struct.eta, struct.min_size
        self.r0, self.r1 = int(r0), int(r1)
        starts = getattr(struct, "aca_starts", None)
        if starts is None:
            from .hmatrix import aca_start_indices
            starts = aca_start_indices(struct.blocks, seed)
        self.blocks, self.aca_starts, self.aca_global = [], [], []
        ai = 0
        for b in struct.blocks:
            s, m = b.row.start, len(b.row.indices)
            e = s + m
            if b.aca:
                if self.r0 <= s and e <= self.r1:
                    self.blocks.append(b)
                elif s < self.r1 and e > self.r0:
                    self.blocks.append(_ClippedAca(b, max(s, self.r0) - s, min(e, self.r1) - s))
                else:
                    ai += 1
                    continue
                self.aca_starts.append(starts[ai])
                self.aca_global.append(ai)
                ai += 1
                continue
            a, z = max(s, self.r0), min(e, self.r1)
            if a >= z:
                continue
            if a == s and z == e:
                self.blocks.append(b)
            else:
                # element ids of the clipped rows (the dense kernels only use start/len and perm)
                node = _RowNode(self.perm[a:z], a)
                self.blocks.append(LeafBlock(node, b.col, False, b.admissible, b.level))


# ----------------------------------------------------------------------------- communicator


class TorchComm:
    """Gather / sum / max over the local backends' tensors, then over
    torch.distributed ranks (when a process group is given or initialized)."""

    def __init__(self, use_dist=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.use_dist = dist.is_available() and dist.is_initialized() if use_dist is None else use_dist

    def _local(self, parts, fn):
        t = parts[0].clone()
        for p in parts[1:]:
            t = fn(t, p.to(t.device))
        return t

    def sum(self, parts):
        t = self._local(parts, lambda a, b: a + b)
        if self.use_dist:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t

    def gather(self, parts):
        """Concatenation, in rank order, of every rank's 1-D piece (the local
        backends' pieces being consecutive ranks).  Across processes: one
        all-gather of the pieces padded to the longest (the piece lengths are
        exchanged once and kept, as the partition does not change)."""
        torch = self.torch
        t = parts[0] if len(parts) == 1 else torch.cat([p.to(parts[0].device) for p in parts])
        if not self.use_dist:
            return t.clone() if len(parts) == 1 else t
        sizes = getattr(self, "_sizes", None)
        if sizes is None or sizes[self.dist.get_rank()] != t.numel():
            n = torch.tensor([t.numel()], dtype=torch.int64, device=t.device)
            out = [torch.zeros_like(n) for _ in range(self.dist.get_world_size())]
            self.dist.all_gather(out, n)
            sizes = self._sizes = [int(v.item()) for v in out]
            self._gbuf = None
        m = max(sizes)
        g = getattr(self, "_gbuf", None)
        if g is None or g.dtype != t.dtype or g.device != t.device:
            # one all-gather into a persistent buffer (world x longest piece); the pieces
            # are then picked out by one index gather when their lengths differ
            self._gbuf = torch.empty(len(sizes) * m, dtype=t.dtype, device=t.device)
            self._gpad = torch.zeros(m, dtype=t.dtype, device=t.device)
            idx = np.concatenate([np.arange(r * m, r * m + k) for r, k in enumerate(sizes)])
            self._gidx = None if min(sizes) == m else torch.tensor(idx, dtype=torch.int64, device=t.device)
        if t.numel() == m:
            pad = t.contiguous()
        else:
            self._gpad[:t.numel()].copy_(t)
            pad = self._gpad
        self.dist.all_gather_into_tensor(self._gbuf, pad)
        return self._gbuf if self._gidx is None else self._gbuf.index_select(0, self._gidx)

    def max(self, parts):
        t = self._local(parts, self.torch.maximum)
        if self.use_dist:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return t

    def max_inplace(self, parts):
        """max, reduced into the one local part itself when there is one (no copy);
        the caller reads it before that buffer is written again."""
        if len(parts) != 1:
            return self.max(parts)
        if self.use_dist:
            self.dist.all_reduce(parts[0], op=self.dist.ReduceOp.MAX)
        return parts[0]


# control block of the device-controlled step (pq3d_rk_rows_control, include/pq3d.h)
PC_H, PC_DTNEXT, PC_TIME, PC_NRJCT, PC_STATUS, PC_ACC, PC_V1, PC_V2, PC_STEPS, PC_REJ, PC_HALT, PC_FIRST, PC_ATT = range(13)
PC_LASTH = 13          # accepted h of the last step (pq3d_rk_rows_finish, or the host after a halted step)


def _nan_encode(v):
    """(values with NaN -> 0, NaN flags) so that a max over ranks keeps NaN."""
    torch = __import__("torch")
    nan = torch.isnan(v)
    return torch.cat([torch.where(nan, torch.zeros_like(v), v), nan.to(v.dtype)])


def _nan_decode(e):
    k = len(e) // 2
    v = np.array(e[:k], dtype=np.float64)
    v[np.asarray(e[k:]) > 0] = np.nan
    return v


def _py_min(a, b):
    return b if b < a else a


def _py_max(a, b):
    return b if b > a else a


class PartitionedStepper:
    """QDsim.simu_forward (src/QDsim.py:892-996) over row-partitioned ranks.

    backends: the ranks of this process (one per GPU in a multi-process run; two
    or more to emulate ranks in one process), in rank order.  Each backend provides
      x_rows()          its rows of the slip-rate deficit: 2 (r1 - r0) values,
                        tree order, (x1, x2) interleaved
      matvec_gathered(xt) H-matvec of its blocks for the whole deficit xt (2n
                        values, tree order, interleaved: all ranks' pieces)
      attempt(h, first) DP5(4) attempt of size h on its rows -> 8 values:
                        4 error maxima (psi, Tt1, Tt2, Tno) with NaN -> 0, 4 NaN flags
      accept(h)         accepted-step update of its rows -> (max|V1|, max|V2|, 0, 0 flags)
    comm: gather / max over all ranks (TorchComm)."""

    def __init__(self, backends, comm, reltol, attempts=3):
        self.backends = list(backends)
        self.comm = comm
        self.reltol = float(reltol)
        self.attempts = int(attempts)      # attempt slots per step of the device-controlled run
        self.time = 0.0
        self.steps = 0
        self.rejects = 0
        self.vmax = (0.0, 0.0)

    def step(self, dttry, h_forced=None):
        xt = self.comm.gather([b.x_rows() for b in self.backends])
        for b in self.backends:
            b.matvec_gathered(xt)
        return self._attempts(float(dttry), 0, True, h_forced)

    def _attempts(self, h, nrjct, first, h_forced=None):
        """Attempts of one step from trial size h (nrjct rejections so far) until one is
        accepted, then the accepted update; returns (h, dtnext)."""
        while True:
            if h_forced is not None:
                h = float(h_forced)
            E = _nan_decode(self.comm.max([b.attempt(h, first) for b in self.backends]).cpu().numpy())
            first = False
            R1 = E[0] + 1e-10
            R2 = _py_max(_py_max(E[1], E[2]), E[3]) + 1e-10
            c1, c2 = R1 / self.reltol, R2 / self.reltol
            hn1 = h * 0.9 * (self.reltol / R1) ** 0.2
            hn2 = h * 0.9 * (self.reltol / R2) ** 0.2
            if h_forced is not None or (_py_max(c1, c2) < 1.0 and not (np.isnan(c1) or np.isnan(c2))):
                dtnext = _py_min(_py_min(hn1, hn2), 1.5 * h)
                break
            nrjct += 1
            dtnext = _py_min(hn1, hn2)
            h = _py_max(0.5 * h, dtnext)
            if h < 1.e-15 or nrjct > 20:
                raise _lib.Pq3dError("time step failed: h < 1e-15 or more than 20 rejections")
        V = self.comm.max([b.accept(h) for b in self.backends]).cpu().numpy()
        self.vmax = (float(V[0]), float(V[1]))
        self.time += h
        self.steps += 1
        self.rejects += nrjct
        return h, dtnext

    # ------------------------------------------------------------------ controller on the device
    def enqueue_device_step(self):
        """One step as a fixed launch sequence with the controller on the device: the
        deficit gather and the matvec, then `attempts` x (attempt, max over ranks,
        controller), then the accepted update, max over ranks, finish.  No host
        synchronisation: steps can be enqueued back to back (or captured).  Every
        rank issues the same collectives in the same order whatever the decisions."""
        xt = self.comm.gather([b.x_rows() for b in self.backends])
        for b in self.backends:
            b.matvec_gathered(xt)
        for _ in range(self.attempts):
            E = self.comm.max_inplace([b.attempt_dev() for b in self.backends])
            for b in self.backends:
                b.control(E, self.reltol, self.attempts)
        V = self.comm.max_inplace([b.accept_dev() for b in self.backends])
        for b in self.backends:
            b.finish(V)

    def run_device(self, nsteps, dttry, chunk=None):
        """nsteps steps with the controller on the device, enqueued `chunk` at a time
        (default: all); the host reads the control block once per chunk.  A step that
        needs more attempts than the launched slots halts the device sequence and is
        finished here with the host controller (same decisions), after which the
        device run resumes.  Returns the accepted step sizes when chunk == 1, else the
        last one's (h, dtnext)."""
        for b in self.backends:
            b.pc_start(dttry, self)
        chunk = int(chunk or nsteps)
        hs = []
        done = 0
        while done < nsteps:
            k = min(chunk, nsteps - done)
            s0 = self.steps
            for _ in range(k):
                self.enqueue_device_step()
            pc = self.backends[0].pc.cpu().numpy()
            ran = int(pc[PC_STEPS]) - s0
            self.steps, self.time = int(pc[PC_STEPS]), float(pc[PC_TIME])
            self.rejects, self.vmax = int(pc[PC_REJ]), (float(pc[PC_V1]), float(pc[PC_V2]))
            if chunk == 1 and ran == 1:
                hs.append(float(self.last_h()))
            done += ran
            if pc[PC_HALT] != 0.0:
                if pc[PC_STATUS] != 0.0:
                    raise _lib.Pq3dError("time step failed: h < 1e-15 or more than 20 rejections")
                # the halted step: the host's attempts from where the device stopped
                h, dtnext = self._attempts(float(pc[PC_H]), int(pc[PC_NRJCT]), False)
                hs.append(h) if chunk == 1 else None
                done += 1
                for b in self.backends:
                    b.pc_resume(self, dtnext, h)
        return hs if chunk == 1 else (self.last_h(), float(self.backends[0].pc[PC_H]))

    def last_h(self):
        return float(self.backends[0].pc[PC_LASTH])

    def capture(self, nsteps):
        """CUDA graph of nsteps device-controlled steps (enqueue_device_step); replays
        chain on the control blocks.  The communicator's collectives are captured
        with the kernels, so every rank must capture and replay alike.  Returns None
        when capture is not possible here."""
        import torch
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        try:
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    for _ in range(nsteps):
                        self.enqueue_device_step()
        except (RuntimeError, _lib.Pq3dError):
            torch.cuda.synchronize()
            return None
        torch.cuda.current_stream().wait_stream(s)
        return g


# ----------------------------------------------------------------------------- device backend


class DeviceRowBackend:
    """One rank on one GPU: the operator of its RankStructure and the row-range
    step kernels of libpq3d.so (pq3d_rk_rows_attempt / pq3d_rk_rows_accept).
    State vectors are held at full length in tree order; only rows [r0, r1)
    are read or written."""

    FIELDS = ["Tno", "Tt1o", "Tt2o", "psi", "slip1", "slip2", "slipv1", "slipv2", "slipv", "rake", "Tt", "fric", "slip"]
    CONST = ["a", "b", "dc", "f0", "shear_loading", "normal_loading", "vplc", "cr0", "sr0"]

    def __init__(self, sim, struct, r0, r1, precision="fp32", device="cuda", op=None):
        """sim: the host-initialized QDsim of the fault; struct: its global
        structure; rows [r0, r1) of tree order belong to this rank."""
        import torch
        from .hmatrix import DeviceHMatrix, pack_x
        self.torch = torch
        self.L = _lib.load()
        self.rs = RankStructure(struct, r0, r1, seed=int(sim.Para0.get("ACA seed", 0)))
        self.r0, self.r1 = self.rs.r0, self.rs.r1
        self.precision = precision
        P = sim.Para0
        if op is None:
            from .qdsim import hs_mode
            op = DeviceHMatrix(self.rs, sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_,
                               device=device, aca_tol=float(P.get("ACA tolerance", 0.01)),
                               aca_rel=P.get("ACA relative tolerance", "False") == "True", halfspace=hs_mode(sim),
                               mixed_tol=float(P.get("Mixed precision tolerance", MIXED_TOL)))
            op.assemble(("fp64",) if precision == "fp64" else ("fp64", precision))
        self.op = op
        n = self.n = struct.n
        perm = struct.perm
        dev = op.dev
        f64 = dict(dtype=torch.float64, device=dev)
        src = dict(Tno=sim.Tno, Tt1o=sim.Tt1o, Tt2o=sim.Tt2o, psi=sim.state, slip1=sim.slip1, slip2=sim.slip2,
                   slipv1=sim.slipv1, slipv2=sim.slipv2, slipv=sim.slipv, rake=sim.rake,
                   Tt=np.sqrt(sim.Tt1o * sim.Tt1o + sim.Tt2o * sim.Tt2o), fric=sim.fric, slip=sim.slip,
                   a=sim.a, b=sim.b, dc=sim.dc, f0=sim.f0, shear_loading=sim.shear_loading,
                   normal_loading=sim.normal_loading, vplc=sim.slipvC, cr0=np.cos(sim.rake0), sr0=np.sin(sim.rake0))
        self.t = {k: torch.tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (n,))[perm]),
                                  **f64) for k, v in src.items()}
        self.y = torch.zeros((n, 3), **f64)
        self.cand = torch.zeros(4 * n, **f64)
        rows = max(self.r1 - self.r0, 1)
        self.grid = min(_cdiv(rows, 256), 4 * 148)
        self.blk = torch.zeros(8 * self.grid + 16, **f64)
        self.ctrl = torch.zeros(16, **f64)
        self.bar = torch.zeros(4, dtype=torch.int32, device=dev)
        self.out = torch.zeros(8, **f64)
        acc = op.plan(precision)["acc"]
        # this rank's rows of the deficit (zeros elsewhere), written by the accept kernel
        xs = pack_x((sim.slipv1 - sim.slipvC * np.cos(sim.rake0))[perm],
                    (sim.slipv2 - sim.slipvC * np.sin(sim.rake0))[perm], n)
        mask = np.zeros(n, dtype=bool)
        mask[self.r0:self.r1] = True
        from .hmatrix import x_stride
        Ps = x_stride(n)
        keep = np.zeros(4 * Ps, dtype=bool)
        keep[0:2 * n:2] = mask
        keep[1:2 * n:2] = mask
        keep[2 * Ps:2 * Ps + n] = mask
        keep[3 * Ps:3 * Ps + n] = mask
        self.xl = torch.tensor(np.where(keep, xs, 0.0), dtype=acc, device=dev)
        self.xg_buf = torch.zeros_like(self.xl)       # the whole deficit, operator layout
        self.n, self.Ps = n, Ps
        A = np.zeros(1, dtype=_lib.RK_ARGS)
        for k in self.FIELDS + self.CONST:
            A[k] = self.t[k].data_ptr()
        for k in ("y", "cand", "blk", "ctrl", "bar"):
            A[k] = getattr(self, k).data_ptr()
        A["x"] = self.xl.data_ptr()
        Pl = op.plan(precision)
        A["slots"] = Pl["slots"].data_ptr()
        for k in ("leaf_of_row", "leaf_ptr", "leaf_off"):
            A[k] = Pl[k].data_ptr()
        A["n"] = n
        A["fix_tn"] = 1 if sim.fix_Tn else 0
        A["x_fp32"] = 0 if acc == torch.float64 else 1
        A["fuse_rowsum"] = 1
        A["slots_fp32"] = 0 if Pl["acc"] == torch.float64 else 1
        A["V0"], A["eta"], A["reltol"] = sim.V0, sim.mu / (2.0 * sim.Cs), sim.RelTol
        self.args = A

    def x_rows(self):
        """This rank's rows of the deficit: the interleaved part of its x buffer,
        which the accept kernel writes."""
        return self.xl[2 * self.r0:2 * self.r1]

    def matvec_gathered(self, xt):
        """H-matvec for the whole deficit xt (tree order, interleaved): the
        operator's layout takes the interleaved pairs and the two planes."""
        n, P = self.n, self.Ps
        xg = self.xg_buf
        xg[0:2 * n].copy_(xt)
        xg[2 * P:2 * P + n].copy_(xt[0::2])
        xg[3 * P:3 * P + n].copy_(xt[1::2])
        self.op.matvec(xg, self.precision, slots_only=True)

    def attempt(self, h, first):
        check(self.L.pq3d_rk_rows_attempt(self.args.ctypes.data, self.grid, self.r0, self.r1, float(h),
                                          1 if first else 0, ptr(self.out), _lib.stream_ptr()),
              "pq3d_rk_rows_attempt")
        return self.out.clone()

    def accept(self, h):
        check(self.L.pq3d_rk_rows_accept(self.args.ctypes.data, self.grid, self.r0, self.r1, float(h), ptr(self.out),
                                         _lib.stream_ptr()), "pq3d_rk_rows_accept")
        return self.out.clone()

    def get(self, name):
        """This rank's rows of a state vector (tree order slice [r0, r1))."""
        return self.t[name][self.r0:self.r1].cpu().numpy()

    # ------------------------------------------------------------------ controller on the device
    def pc_start(self, dttry, ps):
        """Control block for a device-controlled run from trial size dttry."""
        pc = np.zeros(16)
        pc[PC_H], pc[PC_TIME], pc[PC_STEPS], pc[PC_REJ] = dttry, ps.time, ps.steps, ps.rejects
        pc[PC_V1], pc[PC_V2] = ps.vmax
        pc[PC_FIRST] = 1.0
        if getattr(self, "pc", None) is None:
            self.pc = self.torch.tensor(pc, dtype=self.torch.float64, device=self.op.dev)
            self.E8 = self.torch.zeros(8, dtype=self.torch.float64, device=self.op.dev)
        else:
            self.pc.copy_(self.torch.tensor(pc, dtype=self.torch.float64))   # captured graphs keep the address

    def pc_resume(self, ps, dtnext, h):
        """After the host finished a halted step: the next step from dtnext."""
        pc = np.zeros(16)
        pc[PC_H], pc[PC_TIME], pc[PC_STEPS], pc[PC_REJ] = dtnext, ps.time, ps.steps, ps.rejects
        pc[PC_V1], pc[PC_V2] = ps.vmax
        pc[PC_FIRST], pc[PC_LASTH] = 1.0, h
        self.pc.copy_(self.torch.tensor(pc, dtype=self.torch.float64))

    def attempt_dev(self):
        check(self.L.pq3d_rk_rows_attempt_dev(self.args.ctypes.data, self.grid, self.r0, self.r1, ptr(self.pc),
                                              ptr(self.out), _lib.stream_ptr()), "pq3d_rk_rows_attempt_dev")
        return self.out

    def _reduced(self, E):
        """The reduced maxima where the control kernels read them: this rank's own
        output buffer when the reduction ran in place, else a copy (a buffer of the
        communicator's may be reused by the next reduction)."""
        if E.data_ptr() == self.out.data_ptr():
            return self.out
        self.E8.copy_(E)
        return self.E8

    def control(self, E, reltol, attempts):
        check(self.L.pq3d_rk_rows_control(ptr(self.pc), ptr(self._reduced(E)), float(reltol), int(attempts),
                                          _lib.stream_ptr()), "pq3d_rk_rows_control")

    def accept_dev(self):
        check(self.L.pq3d_rk_rows_accept_dev(self.args.ctypes.data, self.grid, self.r0, self.r1, ptr(self.pc),
                                             ptr(self.out), _lib.stream_ptr()), "pq3d_rk_rows_accept_dev")
        return self.out

    def finish(self, V):
        check(self.L.pq3d_rk_rows_finish(ptr(self.pc), ptr(self._reduced(V)), _lib.stream_ptr()),
              "pq3d_rk_rows_finish")

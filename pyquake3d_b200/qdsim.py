"""QDsim: the quasi-dynamic simulation object, reference call surface.

Mirrors QDsim.QDsim of the reference (src/QDsim.py): the constructor takes
(elelst, nodelst, fnamePara), parses parameter.txt (readPara0, :91-100),
builds element frames (readmsh.get_eleVec), sets initial conditions
(Init_condition :387-654, read_parameter :687-757) and the H-matrix
structure (createHmatrix).  Assembly, the H-matvec and the DP5(4) step run on
the GPU (libpq3d.so); the host keeps FP64 copies only on request.

Parameter keys added by this implementation (all optional, reference
behaviour by default):
  H-matrix leaf size        mini_leaf of create_recursive_blocks (32)
  Admissibility eta         eta of is_admissible (2.0)
  Cluster leaf size         min_size of build_block_tree (16)
  ACA tolerance             stopping tolerance (0.01, absolute as the reference)
  ACA relative tolerance    True: tolerance relative to ||A_k||_F (False)
  ACA seed                  seed of the ACA starting rows/cols (0)
  Precision                 fp64 | fp32 | bf16 operator storage (fp64)
  RK RelTol                 DP5(4) relative tolerance (1e-4)
  Half space vertical sides reference | exact: free-surface term of a triangle
                            side along z (the reference's compiled library
                            repeats the previous side's term; exact adds none)
  Initial time step         htry (1e-3)
"""
import ctypes
import math
import os
import queue
import threading
import weakref

import numpy as np

from . import _lib
from ._lib import ptr, check
from .hmatrix import HStructure, DeviceHMatrix, MIXED_TOL
from .mesh import get_eleVec, find_boundary_edges_and_nodes


def readPara0(fname):
    """key: value lines -> dict of stripped strings (split on ':', field 1)."""
    para = {}
    with open(fname, "r") as f:
        for line in f:
            if ":" in line:
                tem = line.split(":")
                para[tem[0].strip()] = tem[1].strip()
    return para


def hs_mode(sim):
    """Green's-function mode of a simulation: 0 full space; with `Half space: True`,
    2 (the side handling of the reference's compiled library, which its H-matrix
    assembly uses) unless `Half space vertical sides: exact` asks for 1 (a
    triangle side along z adds no free-surface term)."""
    if not sim.halfspace_jud:
        return 0
    return 1 if sim.Para0.get("Half space vertical sides", "reference").strip() == "exact" else 2


def _flag(p, key, default=False):
    return p.get(key, "True" if default else "False") == "True"


# QDsim state vectors (reference attribute name -> device field name)
_STATE = {"Tno": "Tno", "Tt1o": "Tt1o", "Tt2o": "Tt2o", "state": "psi", "slip1": "slip1", "slip2": "slip2",
          "slipv1": "slipv1", "slipv2": "slipv2", "slipv": "slipv", "rake": "rake", "Tt": "Tt", "fric": "fric",
          "slip": "slip"}


class _DeviceState:
    """A QDsim state vector under the reference's attribute name.  Until the device
    steps it is the host array; once any step kernel has run since the host copy
    was taken (simu_forward, or bulk stepping through the DeviceStepper: run,
    launch, graph replays), the first read of the attribute fetches the device's
    current values (element order).  So the reference main loop's per-step reads
    (np.max(np.abs(sim0.slipv1)), SLIPV.append(sim0.slipv), src/main.py:168-184)
    see the step just taken.  Vectors read after one simu_forward are gathered by
    the next one as soon as its step ends (DeviceStepper.step prefetch), so a
    loop that reads the same attributes every step waits only for a copy already
    in flight."""

    def __set_name__(self, owner, name):
        self.name = name
        self.key = "_h_" + name

    def __get__(self, obj, owner=None):
        if obj is None:
            return self
        d = obj.__dict__
        dev = d.get("_dev")
        if dev is not None:
            key = (dev._token, dev.version)
            if d.get("_host_key") != key:          # the device stepped since the host copies
                d["_host_key"] = key
                d["_stale"] = set(_STATE)
            stale = d["_stale"]
            if self.name in stale:
                d[self.key] = dev.read_field(_STATE[self.name])
                stale.discard(self.name)
                d.setdefault("_reads", set()).add(self.name)
        return d[self.key]

    def __set__(self, obj, value):
        obj.__dict__[self.key] = value
        stale = obj.__dict__.get("_stale")
        if stale:
            stale.discard(self.name)


class QDsim:
    Tno = _DeviceState()
    Tt1o = _DeviceState()
    Tt2o = _DeviceState()
    state = _DeviceState()
    slip1 = _DeviceState()
    slip2 = _DeviceState()
    slipv1 = _DeviceState()
    slipv2 = _DeviceState()
    slipv = _DeviceState()
    rake = _DeviceState()
    Tt = _DeviceState()
    fric = _DeviceState()
    slip = _DeviceState()

    def __init__(self, elelst, nodelst, fnamePara, device="cuda", precision=None):
        i = fnamePara.rfind("/")
        self.dirname = fnamePara[:i] if i != -1 else fnamePara
        self.Para0 = readPara0(fnamePara)
        P = self.Para0
        self.Corefunc_directory = P.get("Corefunc directory", "core")
        self.save_corefunc = _flag(P, "save Corefunc")
        jud_ele_order = _flag(P, "Node_order")
        jud_scalekm = _flag(P, "Scale_km")
        self.mu = float(P["Shear modulus"])
        self.lambda_ = float(P["Lame constants"])
        self.density = float(P["Rock density"])
        self.halfspace_jud = _flag(P, "Half space")
        self.InputHetoparamter = _flag(P, "InputHetoparamter")
        self.hmatrix_mpi_plot = _flag(P, "Hmatrix_mpi_plot")
        if not jud_scalekm:
            nodelst = nodelst / 1e3
        eleVec, xg = get_eleVec(nodelst, elelst, jud_ele_order)
        self.eleVec, self.elelst, self.nodelst, self.xg = eleVec, elelst, nodelst, xg
        self.htry = float(P.get("Initial time step", 1e-3))
        self.Cs = math.sqrt(self.mu / self.density)
        self.time = 0
        self.YoungsM = self.mu * (3.0 * self.lambda_ + 2.0 * self.mu) / (self.lambda_ + self.mu)
        self.possonratio = self.lambda_ / 2.0 / (self.lambda_ + self.mu)
        self.RelTol = float(P.get("RK RelTol", 1e-4))
        self.precision = precision or P.get("Precision", "fp64")
        self.device = device
        self.Init_condition()
        self.max_slipv1 = float(np.max(np.abs(self.slipv1)))   # updated by every simu_forward
        self.max_slipv2 = float(np.max(np.abs(self.slipv2)))
        self.tree_block = BlockTree(self, int(P.get("H-matrix leaf size", 32)), float(P.get("Admissibility eta", 2.0)),
                                    int(P.get("Cluster leaf size", 16)))
        self._dev = None

    # ------------------------------------------------------------------ initial conditions
    def Init_condition(self):
        P = self.Para0
        N = len(self.eleVec)
        self.Tt1o = np.zeros(N)
        self.Tt2o = np.zeros(N)
        self.Tno = np.zeros(N)
        self.fix_Tn = _flag(P, "Fix_Tn")
        ssv_scale = float(P["Vertical principal stress"])
        ssh1_scale = float(P["Maximum horizontal principal stress"])
        ssv0_scale = float(P["Minimum horizontal principal stress"])
        trac_nor = float(P["Vertical principal stress value"])
        depth_var = P.get("Vertical principal stress value varies with depth") == "True"
        solve_normal = _flag(P, "Normal traction solved from stress tensor")
        ang = np.pi / 180. * float(P["Angle between ssh1 and X-axis"])
        c, s = math.cos(ang), math.sin(ang)
        R = np.array([[c, -s], [s, c]])
        for i in range(N):
            if depth_var:
                ssv = -self.xg[i, 2] / float(P["Turnning depth"]) + 0.2
                if ssv > 1.0:
                    ssv = 1.0
                ssv = trac_nor * ssv * ssv_scale
            else:
                ssv = trac_nor * ssv_scale
            ssh1 = -ssv * ssh1_scale
            ssh2 = -ssv * ssv0_scale
            ssv = -ssv
            st = np.dot(np.dot(R, np.array([[ssh1, 0], [0, ssh2]])), R.transpose())
            s3 = np.array([[st[0][0], st[0][1], 0], [st[1][0], st[1][1], 0], [0, 0, ssv]])
            tra = np.dot(s3, self.eleVec[i, -3:])
            ev = self.eleVec[i]
            self.Tt1o[i] = tra[0] * ev[0] + tra[1] * ev[1] + tra[2] * ev[2]
            self.Tt2o[i] = tra[0] * ev[3] + tra[1] * ev[4] + tra[2] * ev[5]
            self.Tno[i] = tra[0] * ev[6] + tra[1] * ev[7] + tra[2] * ev[8]
            if not solve_normal:
                self.Tno[i] = ssv
        self.Tno = np.abs(self.Tno)
        self.Tt = np.sqrt(self.Tt1o * self.Tt1o + self.Tt2o * self.Tt2o)
        with np.errstate(invalid="ignore", divide="ignore"):
            x = self.Tt1o / self.Tt
            y = self.Tt2o / self.Tt
        solve_shear = _flag(P, "Shear traction solved from stress tensor")
        if P.get("Rake solved from stress tensor") == "True":
            self.rake = np.arctan2(y, x)
        else:
            self.rake = np.ones(len(self.Tt)) * float(P["Fix_rake"]) / 180.0 * np.pi
        if not solve_normal and not depth_var:
            self.Tno = np.ones(len(self.Tno)) * trac_nor
        self.vec_Tra = np.array([x, y]).transpose()
        N = self.Tt1o.shape[0]
        self.Vpl_con = float(P["Plate loading rate"])
        self.Grad_slpv_con(const=True)
        self.shear_loading = np.zeros(N)
        self.normal_loading = np.zeros(N)
        self.V0 = float(P["Reference slip rate"])
        self.dc = np.ones(N) * 0.02
        self.f0 = np.ones(N) * float(P["Reference friction coefficient"])
        self.a = np.zeros(N)
        self.b = np.ones(N) * 0.03
        self.slipv1 = np.zeros(N)
        self.slipv2 = np.zeros(N)
        self.slipv = self.slipvC          # same array object, as in the reference (:499)
        self.slip1 = np.zeros(N)
        self.slip2 = np.zeros(N)
        self.slip = np.zeros(N)
        if self.InputHetoparamter:
            self.read_parameter(P["Inputparamter file"])
        else:
            self._init_regions(solve_shear)
        self.maxslipv0 = np.max(self.slipv)
        self.rake0 = np.copy(self.rake)
        self.calc_nucleaszie_cohesivezone()

    def _init_regions(self, solve_shear):
        """Velocity-strengthening border / nucleation patch layout (src/QDsim.py:528-654)."""
        from scipy.spatial.distance import cdist
        P = self.Para0
        N = len(self.xg)
        _, bnodes = find_boundary_edges_and_nodes(self.elelst)
        bcoord = self.nodelst[bnodes - 1]
        isurf = np.where(np.abs(bcoord[:, 2] - 0.0) < 1e-5)[0]
        isb = np.setdiff1d(np.arange(len(bcoord)), isurf)
        bsurf, bsb = bcoord[isurf], bcoord[isb]
        nuc = np.array([float(P["Nuclea_posx"]), float(P["Nuclea_posy"]), float(P["Nuclea_posz"])])
        W = float(P["Widths of VS region"])
        Ws = float(P["Widths of surface VS region"])
        tr = float(P["Transition region from VS to VW region"])
        aVs, bVs, dVs = (float(P["Rate-and-state parameters a in VS region"]),
                         float(P["Rate-and-state parameters b in VS region"]),
                         float(P["Characteristic slip distance in VS region"]))
        aVw, bVw, dVw = (float(P["Rate-and-state parameters a in VW region"]),
                         float(P["Rate-and-state parameters b in VW region"]),
                         float(P["Characteristic slip distance in VW region"]))
        aNu, bNu, dNu = (float(P["Rate-and-state parameters a in nucleation region"]),
                         float(P["Rate-and-state parameters b in nucleation region"]),
                         float(P["Characteristic slip distance in nucleation region"]))
        vNu = float(P["Initial slip rate in nucleation region"])
        set_nuc = _flag(P, "Set_nucleation")
        rnuc = float(P["Radius of nucleation"])
        chA = _flag(P, "ChangefriA")
        for i in range(N):
            c1 = np.array([self.xg[i]])
            dist = np.min(cdist(c1, bsb))
            dis = dist / W
            dis_s = np.copy(dis)
            dis1 = (dist - W) / tr
            if len(bsurf) > 10:
                dsurf = np.min(cdist(c1, bsurf))
                dis_s = dsurf / Ws
                dis1 = min(dist - W, dsurf - Ws) / tr
            if dis < 1.0 or dis_s < 1.0:
                self.a[i], self.b[i], self.dc[i] = aVs, bVs, dVs
            elif dis1 < 1.0:
                if chA:
                    self.a[i], self.b[i] = aVs - (aVs - aVw) * dis1, bVs
                else:
                    self.a[i], self.b[i] = aVs, bVs - (bVs - bVw) * dis1
                self.dc[i] = dVs
            else:
                self.a[i], self.b[i], self.dc[i] = aVw, bVw, dVw
            if np.linalg.norm(self.xg[i] - nuc) < rnuc and set_nuc:
                self.slipv[i] = vNu
                self.dc[i], self.a[i], self.b[i] = dNu, aNu, bNu
        self.slipv1 = self.slipv * np.cos(self.rake) + 1e-16
        self.slipv2 = self.slipv * np.sin(self.rake) + 1e-16
        if not solve_shear:
            self.Tt = self.Tno * self.a * np.arcsinh(
                self.slipv / (2.0 * self.V0) * np.exp((self.f0 + self.b * np.log(self.V0 / self.slipvC)) / self.a))
        x, y = np.cos(self.rake), np.sin(self.rake)
        self.vec_Tra = np.array([x, y]).transpose()
        self.fric = self.Tt / self.Tno
        self.state = np.log(np.sinh(self.Tt / self.Tno / self.a) * 2.0 * self.V0 / self.slipv) * self.a
        self.Tt1o = self.Tt * x
        self.Tt2o = self.Tt * y

    def read_parameter(self, fname):
        """Per-element 10-column file: rake a b dc f0 Tt Tno V shear_loading normal_loading."""
        vals = np.array([np.array(l.split()).astype(float) for l in open(self.dirname + "/" + fname)])
        Nc = self.eleVec.shape[0]
        self.rake = vals[:Nc, 0]
        self.a = vals[:Nc, 1]
        self.b = vals[:Nc, 2]
        self.dc = vals[:Nc, 3]
        self.f0 = vals[:Nc, 4]
        self.Tt = vals[:Nc, 5]
        self.Tno = vals[:Nc, 6]
        self.slipv = vals[:Nc, 7]
        self.shear_loading = vals[:Nc, 8]
        self.normal_loading = vals[:Nc, 9]
        x, y = np.cos(self.rake), np.sin(self.rake)
        self.slipv1 = self.slipv * x + 1e-16
        self.slipv2 = self.slipv * y + 1e-16
        self.vec_Tra = np.array([x, y]).transpose()
        self.Tt = self.Tno * self.a * np.arcsinh(
            self.slipv / (2.0 * self.V0) * np.exp((self.f0 + self.b * np.log(self.V0 / self.slipvC)) / self.a))
        self.Tt1o = self.Tt * x
        self.Tt2o = self.Tt * y
        self.fric = self.Tt / self.Tno
        self.state = np.log(np.sinh(self.Tt / self.Tno / self.a) * 2.0 * self.V0 / self.slipv) * self.a

    def Grad_slpv_con(self, const):
        self.slipvC = np.ones(len(self.xg)) * self.Vpl_con
        if not const:
            vmin = 1e-16
            for i in range(len(self.xg)):
                if self.xg[i, 2] < -5000:
                    self.slipvC[i] = self.Vpl_con
                else:
                    self.slipvC[i] = vmin + abs(self.xg[i, 2]) / 5000.0 * (self.Vpl_con - vmin)

    def calc_nucleaszie_cohesivezone(self):
        P1 = self.nodelst[self.elelst[:, 0] - 1]
        P2 = self.nodelst[self.elelst[:, 1] - 1]
        P3 = self.nodelst[self.elelst[:, 2] - 1]
        size = np.max(np.stack([np.linalg.norm(P1 - P2, axis=1), np.linalg.norm(P1 - P3, axis=1),
                                np.linalg.norm(P2 - P3, axis=1)]), axis=0)
        self.maxsize = float(np.max(size))
        self.ave_elesize = float(np.mean(size))
        b, a = np.max(self.b), np.min(self.a)
        sigma = np.mean(self.Tno * 1e6)
        L = np.min(self.dc)
        with np.errstate(divide="ignore", invalid="ignore"):
            self.hRA = 2.0 / np.pi * self.mu * b * L / (b - a) / (b - a) / sigma * np.pi * np.pi / 4.0
            self.A0 = 9.0 * np.pi / 32 * self.mu * L / (b * sigma)
        return self.maxsize

    def get_block_core(self):
        """(loaded, blocks) as QDsim.get_block_core (src/QDsim.py:199-218).  True when the
        Corefunc directory holds an operator checkpoint written for this mesh and these
        parameters (pyquake3d_b200.checkpoint); the operator is then on the device.  A
        checkpoint of another mesh or parameter set is ignored (False)."""
        from . import checkpoint
        os.makedirs(self.Corefunc_directory, exist_ok=True)
        path = os.path.join(self.Corefunc_directory, checkpoint.FILE_NAME)
        if not os.path.exists(path):
            return False, []
        try:
            self.tree_block.load(path)
        except _lib.Pq3dError as e:
            print("operator checkpoint not used:", e, flush=True)
            return False, []
        return True, self.tree_block.blocks_to_process

    # ------------------------------------------------------------------ device state
    def _ensure_device(self):
        if self._dev is None:
            self._dev = DeviceStepper(self, self.tree_block.op(), self.precision)
            self._host_key = (self._dev._token, self._dev.version)    # built from the host arrays
            self._stale = set()
        return self._dev

    def simu_forward(self, dttry):
        """One time step (one operator application, adaptive DP5(4)); returns (h, dtnext).
        The state attributes (slipv, Tt, ...) read after it hold the new step's values."""
        st = self._ensure_device()
        reads = self.__dict__.get("_reads") or set()
        self._reads = set()
        h, dtnext = st.step(dttry, prefetch=tuple(sorted(_STATE[k] for k in reads)))
        self.time = st.time
        # max |V1|, max |V2| of the step (the values the reference main loop computes
        # from slipv1 / slipv2 for state.txt), from the step kernel's control block
        self.max_slipv1, self.max_slipv2 = st.vmax
        return h, dtnext

    def snapshot_async(self, names=("slipv", "Tt")):
        """Asynchronous copy of device state vectors to pinned host memory (element order);
        see DeviceStepper.snapshot_async."""
        return self._ensure_device().snapshot_async(names)

    def sync_to_host(self):
        """Copy the device state back into the reference attribute names (element order)."""
        if self._dev is not None:
            self._dev.to_host(self)

    def ouputVTK(self, fname):
        from .output import write_vtk
        self.sync_to_host()
        write_vtk(self, fname)

    def outputtxt(self, fname):
        from .output import write_txt
        self.sync_to_host()
        write_txt(self, fname)


class BlockTree:
    """Reference-facing H-matrix object (BlockTree of src/Hmatrix.py:268-1538)."""

    def __init__(self, sim, mini_leaf, eta, min_size):
        self.sim = sim
        self.mini_leaf = mini_leaf
        self.struct = HStructure(sim.xg, mini_leaf=mini_leaf, eta=eta, min_size=min_size)
        self.blocks_to_process = self.struct.blocks
        self.halfspace_jud = sim.halfspace_jud
        self._op = None

    def op(self):
        if self._op is None:
            self.master()
        return self._op

    def _want(self):
        sim = self.sim
        return getattr(self, "want", None) or (("fp64",) if sim.precision == "fp64" else ("fp64", sim.precision))

    def _new_op(self):
        sim = self.sim
        P = sim.Para0
        tol = float(P.get("ACA tolerance", 0.01))
        rel = P.get("ACA relative tolerance", "False") == "True"
        seed = int(P.get("ACA seed", 0))
        mtol = float(P.get("Mixed precision tolerance", MIXED_TOL))
        return DeviceHMatrix(self.struct, sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_,
                             device=sim.device, aca_tol=tol, aca_rel=rel, aca_seed=seed, halfspace=hs_mode(sim),
                             mixed_tol=mtol)

    def master(self, dir=None, blocks_to_process=None, num_workers=None, save_corefunc=False):
        """Assemble every block on the GPU (dense near field + batched ACA); with
        save_corefunc, write the operator checkpoint into dir (the reference's
        blocks_to_process.joblib, src/Hmatrix.py:1240-1241)."""
        self._op = self._new_op().assemble(self._want())
        if save_corefunc and dir:
            from . import checkpoint
            os.makedirs(dir, exist_ok=True)
            checkpoint.save_operator(self._op, os.path.join(dir, checkpoint.FILE_NAME), self.sim.xg,
                                     self.sim.eleVec)
        return self._op

    def load(self, path):
        """Operator from a checkpoint (every precision the simulation needs must be in it)."""
        from . import checkpoint
        header = checkpoint.read_header(path)
        missing = [d for d in self._want() if d not in header["precisions"]]
        if missing:
            raise _lib.Pq3dError(f"checkpoint lacks the {missing} operator(s)")
        op = self._new_op()
        checkpoint.load_operator(op, path, self.sim.xg, self.sim.eleVec)
        self._op = op
        return op

    def worker(self):
        return None

    def parallel_block_scatter_send(self, blocks_to_process, plotHmatrix=False):
        self.op()
        return blocks_to_process

    def blocks_process_MVM(self, xvector, blocks_to_process, type):
        """y = K_type x for one of the six operators (element order, FP64 host arrays)."""
        op = self.op()
        z = np.zeros_like(np.asarray(xvector, dtype=np.float64))
        if type.endswith("s"):
            y = op.apply(xvector, z, "fp64")
        else:
            y = op.apply(z, xvector, "fp64")
        return y[{"A1": 0, "A2": 1, "B": 2}[type[:-1]]]


def _release_host_io(L, hosts, events):
    for h in hosts:
        L.pq3d_host_map_free(h)
    for e in events:
        L.pq3d_event_destroy(e)


class HostEvent:
    """Completion of a snapshot (a CUDA event without timing)."""

    def __init__(self, L, ev):
        self._L = L
        self._ev = ev

    def synchronize(self):
        check(self._L.pq3d_event_sync(self._ev), "pq3d_event_sync")

    def query(self):
        rc = self._L.pq3d_event_query(self._ev)
        if rc < 0:
            check(rc, "pq3d_event_query")
        return rc == 1


class _CopyJob:
    """The host copies of one step's prefetched vectors, filled by _PrefetchCopier."""

    def __init__(self, names):
        self.names = names
        self.out = {}
        self.ready = {nm: threading.Event() for nm in names}
        self.taken = set()
        self.error = None

    def has(self, name):
        return name in self.ready and name not in self.taken

    def get(self, name):
        self.taken.add(name)
        self.ready[name].wait()
        if self.error is not None:
            raise self.error
        return self.out.pop(name)

    def wait_all(self):
        for ev in self.ready.values():
            ev.wait()


class _PrefetchCopier:
    """Host threads that turn each step's prefetched state vectors (pinned host
    memory, written by the copy engine after the step) into the fresh arrays the
    reference main loop reads and keeps (np.max(np.abs(sim0.slipv1)),
    SLIPV.append(sim0.slipv), src/main.py:168-184).  The loop keeps every array, so
    none is reused, and first touches of fresh memory cost more than the copy: one
    thread keeps a small pool of arrays whose pages it has touched, the other waits
    for each step's copy to land and copies every vector into one of them, while the
    device already runs the next step's H-matvec.  A read then waits only for its own
    vector.  (With one thread doing both, the page touching sat in the copies' path:
    1,680-1,850 steps/s at 60k against 1,970-1,985 with a separate maker thread, and
    1,280-1,370 with the copies made by the reading thread.)"""

    def __init__(self, n, device_index, spare=16, makers=2):
        self.n = n
        self.q = queue.Queue()
        self.pool = queue.Queue(maxsize=spare)
        self.stopped = False
        self.thread = threading.Thread(target=self._run, args=(device_index,), daemon=True)
        # the loop takes four fresh 8n-byte arrays per step; one maker thread kept up at
        # 60k on B200 hosts (1,956-1,968 steps/s with one or two), the second is headroom
        # for hosts whose page faults are slower
        self.makers = [threading.Thread(target=self._make, daemon=True) for _ in range(makers)]
        for t in self.makers:
            t.start()
        self.thread.start()

    def submit(self, done, views, names):
        job = _CopyJob(names)
        self.q.put((job, done, views))
        return job

    def stop(self):
        self.stopped = True
        self.q.put(None)

    def _touched(self):
        a = np.empty(self.n)
        ctypes.memset(a.ctypes.data, 0, a.nbytes)        # first touch, without the GIL
        return a

    def _make(self):
        while not self.stopped:
            a = self._touched()
            while not self.stopped:
                try:
                    self.pool.put(a, timeout=0.5)
                    break
                except queue.Full:
                    pass

    def _fresh(self):
        try:
            return self.pool.get_nowait()
        except queue.Empty:
            return self._touched()

    def _bind(self, device_index):
        import torch
        torch.cuda.set_device(device_index)

    def _run(self, device_index):
        self._bind(device_index)
        while True:
            item = self.q.get()
            if item is None:
                return
            job, done, views = item
            try:
                done.synchronize()
                for nm in job.names:
                    a = self._fresh()
                    np.copyto(a, views[nm])
                    job.out[nm] = a
                    job.ready[nm].set()
            except Exception as e:          # handed to the reader
                job.error = e
            for ev in job.ready.values():
                ev.set()


class _StepGraph:
    """CUDA graph of consecutive steps.  A replay rewrites the operator's slots
    and advances the state, so it invalidates pre-launched products and the
    stepper's step event."""

    def __init__(self, graph, plan, stepper):
        self.graph = graph
        self.plan = plan
        self.stepper = stepper

    def replay(self):
        self.plan["slots_owner"] = None
        self.stepper._state_event = False
        self.stepper._prefetched = None
        self.stepper.version += 1
        self.graph.replay()


class DeviceStepper:
    """Device-resident state (tree order) and the per-step launch sequence:
    H-matvec of the deficit -> cooperative DP5(4) step kernel."""

    FIELDS = ["Tno", "Tt1o", "Tt2o", "psi", "slip1", "slip2", "slipv1", "slipv2", "slipv", "rake", "Tt", "fric", "slip"]
    CONST = ["a", "b", "dc", "f0", "shear_loading", "normal_loading", "vplc", "cr0", "sr0"]

    def __init__(self, sim, op, precision):
        import torch
        self.torch = torch
        self.L = _lib.load()
        self.op = op
        self.precision = precision
        self.n = n = sim.xg.shape[0]
        self.perm = op.s.perm
        dev = op.dev
        f64 = dict(dtype=torch.float64, device=dev)
        src = dict(Tno=sim.Tno, Tt1o=sim.Tt1o, Tt2o=sim.Tt2o, psi=sim.state, slip1=sim.slip1, slip2=sim.slip2,
                   slipv1=sim.slipv1, slipv2=sim.slipv2, slipv=sim.slipv, rake=sim.rake,
                   Tt=np.sqrt(sim.Tt1o * sim.Tt1o + sim.Tt2o * sim.Tt2o), fric=sim.fric, slip=sim.slip,
                   a=sim.a, b=sim.b, dc=sim.dc, f0=sim.f0, shear_loading=sim.shear_loading,
                   normal_loading=sim.normal_loading, vplc=sim.slipvC, cr0=np.cos(sim.rake0), sr0=np.sin(sim.rake0))
        self.t = {k: torch.tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (n,))[self.perm]),
                                  **f64) for k, v in src.items()}
        self.y = torch.zeros((n, 3), **f64)
        self.cand = torch.zeros(4 * n, **f64)
        self.grid = self.L.pq3d_rk_grid(n)
        if self.grid <= 0:
            raise _lib.Pq3dError("pq3d_rk_grid failed")
        self.blk = torch.zeros(10 * self.grid + 16, **f64)     # per-CTA maxima + grid-max result slots
        self.ctrl = torch.zeros(16, **f64)
        self.bar = torch.zeros(4, dtype=torch.int32, device=dev)
        self.hist = None
        self.hist_cap = 0
        self.hforce = None
        self.hforce_cap = 0
        self._token = object()          # plan["slots_owner"]: whose products the slots hold
        self.version = 0                # step kernels launched (QDsim attributes compare it)
        self._io = None                 # mapped control block and step event (step())
        self._state_event = False       # step_done marks the current state (no launch since)
        self._snaps = {}                # snapshot buffers per tuple of names
        self._prefetched = None         # _CopyJob of the last step's prefetch
        self._copier = None             # _PrefetchCopier, started by the first prefetch
        self.x = op.new_x(precision)
        from .hmatrix import pack_x
        x0 = pack_x((sim.slipv1 - sim.slipvC * np.cos(sim.rake0))[self.perm],
                    (sim.slipv2 - sim.slipvC * np.sin(sim.rake0))[self.perm], n)
        self.x.copy_(torch.tensor(x0, dtype=self.x.dtype))
        self.V0 = sim.V0
        self.eta = sim.mu / (2.0 * sim.Cs)
        self.reltol = sim.RelTol
        self.fix_tn = 1 if sim.fix_Tn else 0
        self.time = 0.0
        self.vmax = (0.0, 0.0)          # max |V1|, max |V2| of the last step()
        self.steps = 0
        self.args = np.zeros(1, dtype=_lib.RK_ARGS)
        for k in self.FIELDS + self.CONST:
            self.args[k] = self.t[k].data_ptr()
        self.args["y"] = self.y.data_ptr()
        self.args["cand"] = self.cand.data_ptr()
        self.args["blk"] = self.blk.data_ptr()
        self.args["x"] = self.x.data_ptr()
        self.args["ctrl"] = self.ctrl.data_ptr()
        self.args["hist"] = 0
        self.args["bar"] = self.bar.data_ptr()
        self.args["n"] = n
        self.args["fix_tn"] = self.fix_tn
        self.args["x_fp32"] = 0 if self.x.dtype == torch.float64 else 1
        P = op.plan(precision)
        self._plan = P                  # the plan whose buffers args points into
        self.args["slots"] = P["slots"].data_ptr()
        self.args["leaf_of_row"] = P["leaf_of_row"].data_ptr()
        self.args["leaf_ptr"] = P["leaf_ptr"].data_ptr()
        self.args["leaf_off"] = P["leaf_off"].data_ptr()
        self.args["fuse_rowsum"] = 1
        self.args["slots_fp32"] = 0 if P["acc"] == torch.float64 else 1
        self.args["V0"] = self.V0
        self.args["eta"] = self.eta
        self.args["reltol"] = self.reltol

    def launch(self, step_index=0, stream=None):
        """Enqueue one step (matvec + DP5(4) kernel) without host synchronization; the
        step kernel reduces the matvec's per-row slots itself.  The trial size is the
        device-carried ctrl[0]."""
        self.op.matvec(self.x, self.precision, stream=stream, slots_only=True)
        self._rk(step_index, 0.0, stream)

    def _rk(self, step_index, h_in, stream=None, ctrl_host=0):
        """Enqueue the step kernel alone (the slots must hold the products of x)."""
        if self.op.plans.get(self.precision) is not self._plan:
            raise _lib.Pq3dError("the operator's work items were rebuilt after this stepper was created; "
                                 "create a new stepper")
        self._state_event = False
        self._prefetched = None
        self.version += 1
        self.args["step_index"] = step_index
        self.args["h_in"] = h_in
        self.args["ctrl_host"] = ctrl_host
        # per-step records only while the buffers have room for this step index
        self.args["hist"] = self.hist.data_ptr() if self.hist is not None and step_index < self.hist_cap else 0
        if self.hforce is not None and step_index >= self.hforce_cap:
            raise _lib.Pq3dError("dt replay shorter than the run")
        self.args["hforce"] = self.hforce.data_ptr() if self.hforce is not None else 0
        check(self.L.pq3d_rk_step(self.args.ctypes.data, self.grid, _lib.stream_ptr(stream)), "pq3d_rk_step")

    def set_history(self, nsteps):
        self.hist = self.torch.zeros(6 * max(nsteps, 1), dtype=self.torch.float64, device=self.op.dev)
        self.hist_cap = max(nsteps, 1)

    def set_replay(self, h):
        """dt replay: step s takes h[s] and is accepted (device tensor, FP64)."""
        self.hforce = h.to(dtype=self.torch.float64).contiguous()
        self.hforce_cap = self.hforce.numel()

    def step(self, dttry, prefetch=()):
        """One step from the host (QDsim.simu_forward): returns (h, dtnext).

        The H-matvec needs only the deficit x, not the step size, so the products of
        the NEXT step are enqueued before the host waits for this step's result: the
        device works on them while the caller runs its own code between steps, and
        the next call enqueues only the step kernel (dttry goes to it as a kernel
        argument).  The step kernel stores its control block in mapped host memory,
        so the host waits on an event and reads it without a copy.  The operator's
        slots are shared by every stepper of this precision: any other matvec into
        them, or a graph replay, clears the plan's slots_owner, and the products are
        then computed again here.  prefetch names state vectors to snapshot as soon
        as the step ends (before the next matvec is enqueued, so the gather does not
        queue behind it); read_field then returns them."""
        io = self._io if self._io is not None else self._host_io()
        L = self.L
        P = self.op.plan(self.precision)
        stream = _lib.stream_ptr()
        if P.get("slots_owner") is not self._token:
            self.op.matvec(self.x, self.precision, slots_only=True)
        self._rk(self.steps, float(dttry), stream, ctrl_host=io["ctrl_dev"])
        check(L.pq3d_event_record(io["step_done"], stream), "pq3d_event_record")
        self._state_event = True                      # step_done marks the state of this step
        pre = self._snapshot(prefetch, compute_waits=False) if prefetch else None
        self.op.matvec(self.x, self.precision, slots_only=True)   # products for the next step
        P["slots_owner"] = self._token
        if pre is not None:
            # only the next step kernel (which writes the state) waits for the gather
            check(L.pq3d_stream_wait_event(stream, pre[2]), "pq3d_stream_wait_event")
            if self._copier is None:
                self._copier = _PrefetchCopier(self.n, self.op.dev.index or 0)
                weakref.finalize(self, self._copier.stop)
            self._prefetched = self._copier.submit(pre[0], pre[1], prefetch)
            S = self._snaps[tuple(prefetch)]
            S["jobs"][S["k"] ^ 1] = self._prefetched      # reads that buffer until done
        check(L.pq3d_event_sync(io["step_done"]), "pq3d_event_sync")
        c = io["ctrl"]
        if c[15] != self.steps + 1:
            c = self.ctrl.cpu().numpy()                # the step ended early: the device copy has the status
            if c[4] == 0:
                raise _lib.Pq3dError("time step ended without storing its result")
        if c[4] != 0:
            raise _lib.Pq3dError(f"time step failed: status {int(c[4])} (h={c[1]:.3e}, rejects={int(c[3])})")
        self.steps += 1
        self.time = float(c[2])
        self.vmax = (float(c[5]), float(c[6]))
        return float(c[1]), float(c[0])

    def _host_io(self):
        """Mapped host memory for the control block (16 doubles) and the step event,
        created on first use and released with the stepper."""
        L = self.L
        h, d, ev = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(L.pq3d_host_map_alloc(16 * 8, ctypes.byref(h), ctypes.byref(d)), "pq3d_host_map_alloc")
        rc = L.pq3d_event_create(ctypes.byref(ev))
        if rc != 0:
            L.pq3d_host_map_free(h)
            check(rc, "pq3d_event_create")
        ctrl = np.ctypeslib.as_array((ctypes.c_double * 16).from_address(h.value))
        ctrl[:] = 0.0
        self._io = {"ctrl": ctrl, "ctrl_dev": d.value, "step_done": ev.value}
        weakref.finalize(self, _release_host_io, L, [h.value], [ev.value])
        return self._io

    def capture(self, nsteps):
        """CUDA graph of nsteps consecutive steps (matvec + step kernel each).  The
        step size is carried on the device (ctrl[0]), so replays chain; step s of a
        replay writes history row s.  Returns None if capture is not possible here."""
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
        return _StepGraph(g, self.op.plan(self.precision), self)

    def run(self, nsteps, dttry):
        """nsteps steps back to back on the device; returns the history (nsteps x 6)."""
        self.set_history(nsteps)
        self.ctrl[0] = float(dttry)
        for i in range(nsteps):
            self.launch(i)
        c = self.ctrl.cpu().numpy()
        if c[4] != 0:
            raise _lib.Pq3dError(f"time step failed: status {int(c[4])}")
        self.steps += nsteps
        self.time = float(c[2])
        return self.hist.view(-1, 6).cpu().numpy()[:nsteps]

    def snapshot_async(self, names):
        """Start copying state vectors (element order) to host memory without holding
        up the next step.  On a high-priority side stream, after the step that
        produced them (the step event when no launch came since): one gather kernel
        into a device staging buffer, which runs between the waves of the
        pre-launched H-matvec, then a copy-engine transfer to pinned host memory.
        The next step kernel waits for the gather only.  Two buffers alternate.
        Returns (event, {name: float64 array}); the arrays are valid once
        event.synchronize() returns and stay valid until the snapshot after next
        (the buffer is then reused)."""
        done, views, _ = self._snapshot(names)
        return done, views

    def _snapshot(self, names, compute_waits=True):
        """snapshot_async; also returns the raw `gathered` event."""
        torch = self.torch
        L = self.L
        names = tuple(names)
        S = self._snaps.get(names)
        if S is None:
            n, nf = self.n, len(names)
            hosts, views, events = [], [], []
            for _ in range(2):
                h, d = ctypes.c_void_p(), ctypes.c_void_p()
                check(L.pq3d_host_map_alloc(nf * n * 8, ctypes.byref(h), ctypes.byref(d)), "pq3d_host_map_alloc")
                hosts.append(h.value)
                a = np.ctypeslib.as_array((ctypes.c_double * (nf * n)).from_address(h.value)).reshape(nf, n)
                views.append({nm: a[j] for j, nm in enumerate(names)})
                for _ in range(2):
                    ev = ctypes.c_void_p()
                    check(L.pq3d_event_create(ctypes.byref(ev)), "pq3d_event_create")
                    events.append(ev.value)
            S = {"names": names, "k": 0, "side": torch.cuda.Stream(device=self.op.dev, priority=-100),
                 "iperm": torch.as_tensor(np.argsort(self.perm), dtype=torch.int64, device=self.op.dev),
                 "fields": np.array([self.t[nm].data_ptr() for nm in names], dtype=np.uint64),
                 "stage": [torch.empty(nf * n, dtype=torch.float64, device=self.op.dev) for _ in range(2)],
                 "host": hosts, "views": views, "gathered": events[0::2],
                 "done": [HostEvent(L, e) for e in events[1::2]], "jobs": [None, None]}
            S["release"] = weakref.finalize(self, _release_host_io, L, hosts, events)
            self._snaps[names] = S
        b = S["k"]
        S["k"] ^= 1
        job = S["jobs"][b]
        if job is not None:
            job.wait_all()                  # the host copier still reads this buffer
            S["jobs"][b] = None
        compute = _lib.stream_ptr()
        io = self._io if self._io is not None else self._host_io()
        if not self._state_event:
            # the state is whatever the compute stream has enqueued so far
            check(L.pq3d_event_record(io["step_done"], compute), "pq3d_event_record")
            self._state_event = True
        done = S["done"][b]
        check(L.pq3d_snapshot(len(names), S["fields"].ctypes.data, S["iperm"].data_ptr(), self.n,
                              S["stage"][b].data_ptr(), S["host"][b], io["step_done"], S["gathered"][b], done._ev,
                              compute, S["side"].cuda_stream, 1 if compute_waits else 0), "pq3d_snapshot")
        return done, S["views"][b], S["gathered"][b]

    def fetch(self, names):
        """Element-order copies of state vectors as the last step left them, waiting
        for the snapshot only (not for work enqueued after the step)."""
        done, v = self.snapshot_async(names)
        done.synchronize()
        return {k: np.array(v[k]) for k in names}

    def read_field(self, name):
        """One state vector (element order, a new array) as the last step left it:
        from that step's prefetch when it holds the vector and nothing was launched
        since, else by a snapshot of its own."""
        pf = self._prefetched
        if pf is not None and pf.has(name):
            return pf.get(name)
        return self.fetch((name,))[name]

    def get(self, name):
        v = self.t[name].cpu().numpy()
        out = np.empty_like(v)
        out[self.perm] = v
        return out

    def to_host(self, sim):
        sim._host_key = (self._token, self.version)       # the host copies below are current
        sim._stale = set()
        sim.Tno, sim.Tt1o, sim.Tt2o, sim.state = self.get("Tno"), self.get("Tt1o"), self.get("Tt2o"), self.get("psi")
        sim.slip1, sim.slip2, sim.slip = self.get("slip1"), self.get("slip2"), self.get("slip")
        sim.slipv1, sim.slipv2, sim.slipv = self.get("slipv1"), self.get("slipv2"), self.get("slipv")
        sim.rake, sim.Tt, sim.fric = self.get("rake"), self.get("Tt"), self.get("fric")
        sim.time = self.time

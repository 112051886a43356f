"""V-mode stepping and the Newton-seeding MLP (device side in csrc/vmode.cu, csrc/mlp.cu).

V-mode integrates (slip, state) with DP5(4) and one H-matvec per stage; the
slip rate solves the radiation-damped friction law per element with Newton.
It has no counterpart in the reference (whose stepper freezes the elastic
load over a step); it uses the reference's friction law, aging law, loading
and operators.  The initial guess of every Newton solve is one of
  seed 0: the element's previous rate        seed 1: the undamped bound z = S
  seed 2: the MLP (trained here on the stepper's own converged solves), consulted
          only where one Newton step from z = S does not already converge
  seed 3: the gated MLP: the undamped start takes the first Newton step; plain
          Newton goes on when its correction is at most MLP_GATE in z, and only
          larger corrections (strong radiation damping) evaluate the MLP
and plain Newton (from z = S) stays the fallback and the judge: an MLP start
whose residual is above 1e-10 after 8 steps is discarded.
"""
import ctypes

import numpy as np

# seed 3: first Newton correction from the undamped start (in z) above which the MLP
# proposes the start; smaller ones converge in a step or two of plain Newton
MLP_GATE = 0.5

from . import _lib
from ._lib import check, ptr, stream_ptr

VARGS_PTRS = ["y0", "k", "y5", "mv", "tq1", "tq2", "sig0", "a", "b", "dc", "f0", "shear_loading", "normal_loading",
              "vplc", "cr0", "sr0", "V", "x", "ctrl", "blk", "bar", "stats", "mlp", "log_x", "log_n"]
VARGS = np.dtype([(p, "u8") for p in VARGS_PTRS] + [("log_cap", "i8"), ("n", "i4"), ("x_fp32", "i4"),
                                                    ("seed_mode", "i4"), ("newton_max", "i4"), ("V0", "f8"),
                                                    ("eta", "f8"), ("reltol", "f8"), ("atol", "f8"),
                                                    ("newton_tol", "f8"), ("mlp_gate", "f8")], align=True)
# control block: [0] h of the next attempt, [1] last accepted h, [2] time, [3] consecutive rejects,
# [4] status, [8] accepted steps, [9] rejects, [10] attempts, [11] last attempt accepted, [12] dtnext, [13] E
MLP_NP = 4609


def _bind(L):
    if getattr(L, "_vmode_bound", False):
        return
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    L.pq3d_vmode_args_bytes.restype = ctypes.c_size_t
    L.pq3d_vmode_stage.argtypes = [vp, i32, vp]
    L.pq3d_vmode_grid.argtypes = [i32]
    L.pq3d_mlp_param_count.restype = i32
    L.pq3d_mlp_scratch_floats.argtypes = [i32]
    L.pq3d_mlp_scratch_floats.restype = i64
    L.pq3d_mlp_forward.argtypes = [vp, vp, i32, i32, vp, vp]
    L.pq3d_mlp_grad.argtypes = [vp, vp, i32, vp, i32, i32, vp, vp, vp, vp]
    f = ctypes.c_float
    L.pq3d_mlp_train_step.argtypes = [vp, vp, vp, vp, i32, vp, i32, i32, vp, vp, f, f, f, f, i32, vp, vp]
    if L.pq3d_vmode_args_bytes() != VARGS.itemsize:
        raise _lib.Pq3dError("VArgs layout mismatch")
    if L.pq3d_mlp_param_count() != MLP_NP:
        raise _lib.Pq3dError("MLP parameter count mismatch")
    L._vmode_bound = True


def mlp_init_params(seed=0):
    """W ~ N(0, 1/fan_in), zero biases (same rule as the oracle's mlp_init), flat FP32 layout."""
    rng = np.random.default_rng(seed)
    P = np.zeros(MLP_NP, dtype=np.float64)
    P[0:320] = rng.normal(0, 1 / np.sqrt(5), (64, 5)).ravel()
    P[384:4480] = rng.normal(0, 1 / np.sqrt(64), (64, 64)).ravel()
    P[4544:4608] = rng.normal(0, 1 / np.sqrt(64), 64)
    return P


def mlp_unflatten(P):
    P = np.asarray(P, dtype=np.float64)
    return dict(W1=P[0:320].reshape(64, 5), b1=P[320:384], W2=P[384:4480].reshape(64, 64), b2=P[4480:4544],
                W3=P[4544:4608].reshape(1, 64), b3=P[4608:4609])


class MLPTrainer:
    """Adam training of the 5-64-64-1 network with the hand-written kernels of mlp.cu."""

    def __init__(self, device="cuda", seed=0):
        import torch
        self.torch = torch
        self.L = _lib.load()
        _bind(self.L)
        self.dev = torch.device(device)
        self.P = torch.tensor(mlp_init_params(seed), dtype=torch.float32, device=self.dev)
        self.M = torch.zeros_like(self.P)
        self.V = torch.zeros_like(self.P)
        self.G = torch.zeros_like(self.P)
        self.step = 0
        self.history = []

    def grad(self, X, T):
        """Gradient of 0.5 mean((MLP(X) - T)^2) for rows of X (first 5 columns) and targets T."""
        torch = self.torch
        B = X.shape[0]
        scratch = torch.empty(self.L.pq3d_mlp_scratch_floats(B), dtype=torch.float32, device=self.dev)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        check(self.L.pq3d_mlp_grad(ptr(self.P), ptr(X), X.stride(0), ptr(T), T.stride(0), B, ptr(scratch),
                                   ptr(self.G), ptr(loss), stream_ptr()), "pq3d_mlp_grad")
        return self.G.clone(), float(loss.item())

    def fit(self, data, epochs=20, batch=4096, lr=2e-3, seed=0):
        """data: N x 6 FP32 device tensor (5 features, target)."""
        torch = self.torch
        N = data.shape[0]
        B = min(batch, N)
        scratch = torch.empty(self.L.pq3d_mlp_scratch_floats(B), dtype=torch.float32, device=self.dev)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        g = torch.Generator(device=self.dev)
        g.manual_seed(seed)
        for ep in range(epochs):
            perm = torch.randperm(N, device=self.dev, generator=g)
            loss.zero_()
            nb = 0
            for s in range(0, N - B + 1, B):
                xb = data.index_select(0, perm[s:s + B]).contiguous()
                self.step += 1
                check(self.L.pq3d_mlp_train_step(ptr(self.P), ptr(self.M), ptr(self.V), ptr(xb), 6, ptr(xb[:, 5:]),
                                                 6, B, ptr(scratch), ptr(self.G), lr, 0.9, 0.999, 1e-8, self.step,
                                                 ptr(loss), stream_ptr()), "pq3d_mlp_train_step")
                nb += 1
            self.history.append(float(loss.item()) / max(nb, 1))
        return self.history

    def predict(self, X):
        torch = self.torch
        Y = torch.empty(X.shape[0], dtype=torch.float32, device=self.dev)
        check(self.L.pq3d_mlp_forward(ptr(self.P), ptr(X), X.stride(0), X.shape[0], ptr(Y), stream_ptr()),
              "pq3d_mlp_forward")
        return Y


class VStepper:
    """Device-resident V-mode state (tree order) and its launch sequence."""

    def __init__(self, sim, op, precision="fp64", seed_mode=1, reltol=1e-4, atol=1e-9, log_cap=0,
                 mlp_params=None, newton_max=200):
        import torch
        self.torch = torch
        self.L = _lib.load()
        _bind(self.L)
        self.sim, self.op, self.precision = sim, op, precision
        self.n = n = sim.xg.shape[0]
        perm = op.s.perm
        self.perm = perm
        dev = op.dev
        f64 = dict(dtype=torch.float64, device=dev)
        eta = sim.mu / (2.0 * sim.Cs)
        t = lambda v: torch.tensor(np.ascontiguousarray(np.asarray(v, dtype=np.float64)[perm]), **f64)
        self.c = {k: t(v) for k, v in dict(
            tq1=sim.Tt1o * 1e6 + eta * sim.slipv1, tq2=sim.Tt2o * 1e6 + eta * sim.slipv2, sig0=sim.Tno * 1e6,
            a=sim.a, b=sim.b, dc=sim.dc, f0=sim.f0, shear_loading=sim.shear_loading,
            normal_loading=sim.normal_loading, vplc=sim.slipvC, cr0=np.cos(sim.rake0),
            sr0=np.sin(sim.rake0)).items()}
        self.y0 = torch.cat([torch.zeros(2 * n, **f64), t(sim.state)])
        self.k = torch.zeros(21 * n, **f64)
        self.y5 = torch.zeros(3 * n, **f64)
        self.V = torch.cat([t(sim.slipv1), t(sim.slipv2)])
        self.mv = torch.zeros((n, 3), **f64)
        self.x = op.new_x(precision)
        grid = self.L.pq3d_vmode_grid(n)
        self.blk = torch.zeros(grid, **f64)
        self.ctrl = torch.zeros(16, **f64)
        self.bar = torch.zeros(4, dtype=torch.int32, device=dev)
        self.stats = torch.zeros(4, dtype=torch.int64, device=dev)
        self.mlp = None if mlp_params is None else mlp_params.to(device=dev, dtype=torch.float32).contiguous()
        self.log_cap = int(log_cap)
        self.log_x = torch.zeros(max(self.log_cap, 1) * 6, dtype=torch.float32, device=dev)
        self.log_n = torch.zeros(1, dtype=torch.int64, device=dev)
        A = np.zeros(1, dtype=VARGS)
        for k in ("y0", "k", "y5", "mv", "V", "x", "ctrl", "blk", "bar", "stats"):
            A[k] = getattr(self, k).data_ptr()
        for k, v in self.c.items():
            A[k] = v.data_ptr()
        A["mlp"] = self.mlp.data_ptr() if self.mlp is not None else 0
        A["log_x"] = self.log_x.data_ptr() if self.log_cap > 0 else 0
        A["log_n"] = self.log_n.data_ptr()
        A["log_cap"] = self.log_cap
        A["n"] = n
        A["x_fp32"] = 0 if self.x.dtype == torch.float64 else 1
        A["seed_mode"] = seed_mode
        A["newton_max"] = newton_max
        A["V0"], A["eta"], A["reltol"], A["atol"], A["newton_tol"] = sim.V0, eta, reltol, atol, 1e-12
        A["mlp_gate"] = MLP_GATE
        self.args = A
        self.started = False

    def set_seed_mode(self, mode, mlp_params=None):
        if mlp_params is not None:
            self.mlp = mlp_params.to(device=self.op.dev, dtype=self.torch.float32).contiguous()
            self.args["mlp"] = self.mlp.data_ptr()
        self.args["seed_mode"] = mode

    def _stage(self, s, stream=None):
        check(self.L.pq3d_vmode_stage(self.args.ctypes.data, s, stream_ptr(stream)), "pq3d_vmode_stage")

    def start(self, h0, stream=None):
        """Stage 1 at the current state: the first matvec and k1."""
        self.ctrl[0] = float(h0)
        self._stage(-1, stream)
        self.op.matvec(self.x, self.precision, y=self.mv, stream=stream)
        self._stage(1, stream)
        self.started = True

    def attempt(self, stream=None):
        """One DP5(4) attempt (stages 2..7, six matvecs) and its accept/reject finalization."""
        for s in range(2, 8):
            self.op.matvec(self.x, self.precision, y=self.mv, stream=stream)
            self._stage(s, stream)
        self._stage(0, stream)

    def run(self, nsteps, h0=1e-3, chunk=8, max_attempts=None):
        """Attempts until nsteps more steps are accepted; returns ctrl."""
        if not self.started:
            self.start(h0)
        target = float(self.ctrl[8].item()) + nsteps
        budget = max_attempts or 4 * nsteps + 40
        done = 0
        while True:
            for _ in range(chunk):
                self.attempt()
            done += chunk
            c = self.ctrl.cpu().numpy()
            if c[4] != 0:
                raise _lib.Pq3dError("V-mode step failed: status %d" % int(c[4]))
            if c[8] >= target or done >= budget:
                return c

    def capture(self, nattempts):
        torch = self.torch
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        try:
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    for _ in range(nattempts):
                        self.attempt()
        except (RuntimeError, _lib.Pq3dError):
            torch.cuda.synchronize()
            return None
        torch.cuda.current_stream().wait_stream(s)
        return g

    def newton_stats(self):
        s = self.stats.cpu().numpy()
        return dict(iterations=int(s[0]), solves=int(s[1]), mean=float(s[0]) / max(int(s[1]), 1),
                    max=int(s[2]), fallbacks=int(s[3]))

    def reset_stats(self):
        self.stats.zero_()

    def samples(self):
        m = min(int(self.log_n.item()), self.log_cap)
        return self.log_x[:6 * m].view(m, 6)

    def get(self, name):
        n = self.n
        src = {"slip1": self.y0[:n], "slip2": self.y0[n:2 * n], "psi": self.y0[2 * n:], "V1": self.V[:n],
               "V2": self.V[n:]}[name].cpu().numpy()
        out = np.empty_like(src)
        out[self.perm] = src
        return out

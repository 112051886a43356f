"""ORACLE -- test infrastructure only (tests/, smoke, bench CPU legs).

FP64 numpy restatement of the V-mode stepper and of the Newton-seeding MLP.
The reference has no V-mode: parity of this file is UNPINNED by the
reference.  It is a statement of the formulation the device kernels
(pyquake3d_b200/csrc/vmode.cu, mlp.cu) implement, checked against the
reference-mode stepper on slow-slip intervals (both integrate the same
rate-and-state ODE; see tests/test_vmode_oracle.py).

Formulation (same friction law, elasticity and loading as the reference,
src/QDsim.py:760-813 and :892-996):
  state y = (slip1, slip2, psi); deficit d(t) = slip - Vpl (cos r0, sin r0) t
  quasi-static tractions  tq_c(t) = tq_c(0) - (A_c d)(t) + shear_loading t   (c = 1, 2)
  normal stress           sig(t) = sig(0) + (B d)(t) + normal_loading t
  with tq_c(0) = Tt_c(0) + eta V_c(0) (the reference's tractions include damping).
  Per component the slip rate solves  tq_c - eta V_c = a sig asinh(V_c e^{psi/a} / (2 V0)),
  written with z = asinh(|V_c| e^{psi/a}/(2V0)):  F(z) = z + kappa sinh z - S = 0,
  S = |tq_c| / (a sig), kappa = 2 V0 eta e^{-psi/a} / (a sig); F is increasing and
  convex on [0, S], Newton with the step clamped to [0, S].
  d slip_c/dt = V_c,  d psi/dt = (b/Dc)(V0 exp((f0 - psi)/b) - |V|)  (aging law).
  DP5(4) with FSAL; error E = max over elements of
  max(|dpsi|/|psi|, |dslip_c| / (|slip_c| + atol)) / RelTol; accept when E < 1,
  h_new = 0.9 h E^(-1/5), growth capped at 1.5 h (the reference's constants).
"""
import numpy as np

C = np.array([0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0])
A = [[],
     [1 / 5],
     [3 / 40, 9 / 40],
     [44 / 45, -56 / 15, 32 / 9],
     [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
     [9017 / 3168, -355 / 33, -46732 / 5247, 49 / 176, -5103 / 18656],
     [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]]
B4 = [5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40]
ATOL_SLIP = 1e-9


def vsolve(tq, sig, psi, a, V0, eta, z0=None, tol=1e-12, maxit=100):
    """Slip rate of one traction component; returns (V, iterations, z, S, kappa)."""
    S = np.abs(tq) / (a * sig)
    lk = np.log(2.0 * V0 * eta / (a * sig)) - psi / a          # log kappa
    z = np.array(S if z0 is None else np.clip(z0, 0.0, S), dtype=np.float64)
    it = np.zeros(np.shape(S), dtype=np.int64)
    active = np.ones(np.shape(S), dtype=bool)
    for k in range(maxit):
        # kappa sinh z and kappa cosh z without overflow
        ks = np.exp(lk + z) * 0.5 * (1.0 - np.exp(-2.0 * z))
        kc = np.exp(lk + z) * 0.5 * (1.0 + np.exp(-2.0 * z))
        F = z + ks - S
        dz = F / (1.0 + kc)
        znew = np.clip(z - dz, 0.0, S)
        conv = np.abs(znew - z) <= tol * np.maximum(1.0, z)
        it = np.where(active, it + 1, it)
        z = np.where(active, znew, z)
        active = active & ~conv
        if not active.any():
            break
    V = np.sign(tq) * 2.0 * V0 * np.exp(-psi / a + z) * 0.5 * (1.0 - np.exp(-2.0 * z))
    return V, it, z, S, np.exp(lk)


class VModeOracle:
    """V-mode stepper on a generic linear operator mvm(d1, d2) -> (B d, A1 d, A2 d)."""

    def __init__(self, st, mvm, V0, mu, Cs, reltol=1e-4):
        self.mvm = mvm
        self.V0, self.eta = V0, mu / (2.0 * Cs)
        self.reltol = reltol
        for k in ("a", "b", "dc", "f0", "shear_loading", "normal_loading", "slipvC", "rake0"):
            setattr(self, k, np.array(st[k], dtype=np.float64))
        self.cr0, self.sr0 = np.cos(self.rake0), np.sin(self.rake0)
        V1, V2 = np.array(st["slipv1"], dtype=np.float64), np.array(st["slipv2"], dtype=np.float64)
        self.tq1 = np.array(st["Tt1o"]) * 1e6 + self.eta * V1
        self.tq2 = np.array(st["Tt2o"]) * 1e6 + self.eta * V2
        self.sig0 = np.array(st["Tno"]) * 1e6
        n = len(self.a)
        self.s1, self.s2 = np.zeros(n), np.zeros(n)
        self.psi = np.array(st["state"], dtype=np.float64)
        self.time = 0.0
        self.V1, self.V2 = V1, V2
        self.newton_iters = []
        self.k1 = None

    def rates(self, s1, s2, psi, t, seed=None):
        d1 = s1 - self.slipvC * self.cr0 * t
        d2 = s2 - self.slipvC * self.sr0 * t
        bd, a1, a2 = self.mvm(d1, d2)
        tq1 = self.tq1 - a1 + self.shear_loading * t
        tq2 = self.tq2 - a2 + self.shear_loading * t
        sig = self.sig0 + bd + self.normal_loading * t
        V1, it1, _, _, _ = vsolve(tq1, sig, psi, self.a, self.V0, self.eta)
        V2, it2, _, _, _ = vsolve(tq2, sig, psi, self.a, self.V0, self.eta)
        self.newton_iters.append((it1.mean() + it2.mean()) / 2)
        V = np.sqrt(V1 * V1 + V2 * V2)
        dpsi = self.b / self.dc * (self.V0 * np.exp(np.clip((self.f0 - psi) / self.b, -700, 700)) - V)
        return np.stack([V1, V2, dpsi]), sig

    def step(self, h):
        """One DP5(4) step attempt loop; returns (h_accepted, dtnext)."""
        y0 = np.stack([self.s1, self.s2, self.psi])
        if self.k1 is None:
            self.k1, _ = self.rates(*y0, self.time)
        nrej = 0
        while True:
            k = [self.k1]
            for s in range(1, 7):
                ys = y0 + h * sum(A[s][j] * k[j] for j in range(s))
                ks, _ = self.rates(*ys, self.time + C[s] * h)
                k.append(ks)
            y5 = y0 + h * sum(A[6][j] * k[j] for j in range(6))
            y4 = y0 + h * sum(B4[j] * k[j] for j in range(7))
            e = np.abs(y5 - y4)
            E = max(np.max(e[2] / np.abs(y5[2])), np.max(e[0] / (np.abs(y5[0]) + ATOL_SLIP)),
                    np.max(e[1] / (np.abs(y5[1]) + ATOL_SLIP))) / self.reltol
            hnew = 0.9 * h * E ** -0.2 if E > 0 else 1.5 * h
            if E < 1.0:
                self.s1, self.s2, self.psi = y5
                self.time += h
                self.k1 = k[6]
                self.V1, self.V2 = k[6][0], k[6][1]
                return h, min(hnew, 1.5 * h)
            nrej += 1
            h = max(0.5 * h, hnew)
            if h < 1e-15 or nrej > 20:
                raise RuntimeError("V-mode step size controller gave up")


# ---------------------------------------------------------------- MLP (5 -> 64 -> 64 -> 1, tanh)

def mlp_features(S, kappa, a, b, sig):
    """Inputs of the Newton-seeding MLP (traction, state, a, b, sigma), scaled to O(1)."""
    return np.stack([np.log1p(S) / 5.0, np.log10(kappa + 1e-300) / 20.0, a * 50.0, b * 50.0,
                     np.log10(sig / 1e6) / 2.0], axis=-1)


def mlp_target(z, S):
    """Regression target: logit of z/S (the seed is z0 = S * sigmoid(output))."""
    r = np.clip(z / np.maximum(S, 1e-300), 1e-6, 1 - 1e-6)
    return np.log(r / (1 - r))


def mlp_init(seed=0):
    rng = np.random.default_rng(seed)
    return dict(W1=rng.normal(0, 1 / np.sqrt(5), (64, 5)), b1=np.zeros(64),
                W2=rng.normal(0, 1 / np.sqrt(64), (64, 64)), b2=np.zeros(64),
                W3=rng.normal(0, 1 / np.sqrt(64), (1, 64)), b3=np.zeros(1))


def mlp_forward(P, X):
    h1 = np.tanh(X @ P["W1"].T + P["b1"])
    h2 = np.tanh(h1 @ P["W2"].T + P["b2"])
    return (h2 @ P["W3"].T + P["b3"])[:, 0], (h1, h2)


def mlp_loss_grad(P, X, t):
    """Mean squared error 0.5 mean((y - t)^2) and its gradients (FP64)."""
    y, (h1, h2) = mlp_forward(P, X)
    B = len(t)
    d3 = (y - t) / B
    g = {"W3": d3[None, :] @ h2, "b3": np.array([d3.sum()])}
    d2 = (d3[:, None] * P["W3"]) * (1 - h2 ** 2)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ P["W2"]) * (1 - h1 ** 2)
    g["W1"] = d1.T @ X
    g["b1"] = d1.sum(0)
    return 0.5 * np.mean((y - t) ** 2), g

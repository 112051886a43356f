"""The V-mode oracle (project formulation; no reference counterpart, parity unpinned
by the reference): Newton solve, MLP gradients, and agreement with the reference-mode
stepper, which integrates the same rate-and-state ODE with a frozen elastic load."""
import numpy as np
import pytest

import qd_oracle
import vmode_oracle as vo
from pyquake3d_b200.hmatrix import aca_start_indices


def test_newton_solves_the_damped_friction_law():
    rng = np.random.default_rng(0)
    n = 20000
    a = rng.uniform(0.005, 0.03, n)
    sig = rng.uniform(10e6, 100e6, n)
    psi = rng.uniform(0.3, 1.0, n)
    tq = rng.uniform(-1.0, 1.0, n) * 0.9 * sig
    V0, eta = 1e-6, 32e9 / (2 * 3464.0)
    V, it, z, S, kap = vo.vsolve(tq, sig, psi, a, V0, eta)
    tau = tq - eta * V
    resid = tau - a * sig * np.arcsinh(V / (2 * V0) * np.exp(psi / a))
    assert np.all(np.abs(resid) <= 1e-9 * np.abs(tq) + 1e-6)
    assert np.all(np.sign(V) == np.sign(tq))
    assert np.all((z >= 0) & (z <= S))
    assert it.max() < 100


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = vo.mlp_init(2)
    X = rng.standard_normal((64, 5))
    t = rng.standard_normal(64)
    L, g = vo.mlp_loss_grad(P, X, t)
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        W = P[name]
        idx = tuple(rng.integers(0, s) for s in W.shape)
        e = 1e-6
        W[idx] += e
        Lp, _ = vo.mlp_loss_grad(P, X, t)
        W[idx] -= 2 * e
        Lm, _ = vo.mlp_loss_grad(P, X, t)
        W[idx] += e
        fd = (Lp - Lm) / (2 * e)
        assert abs(fd - g[name][idx]) <= 1e-6 * max(1e-8, abs(fd)) + 1e-10, name


def test_vmode_agrees_with_reference_mode_on_a_slow_interval(tiny_sim, tiny_golden):
    s = tiny_sim
    st = s.tree_block.struct
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks],
                                  aca_start_indices(st.blocks, int(tiny_golden["aca_seed"])), eps=0.01)
    state = qd_oracle.sim_state(s)
    ref = qd_oracle.OracleStepper(state, qd_oracle.operator_mvm(op), s.V0, s.mu, s.Cs)
    vm = vo.VModeOracle(state, qd_oracle.operator_mvm(op), s.V0, s.mu, s.Cs, reltol=1e-6)
    T = 2.0
    for _ in range(200):
        ref.simu_forward(0.01, h_forced=0.01)
    h = 1e-3
    while vm.time < T - 1e-12:
        h = min(h, T - vm.time)
        _, h = vm.step(h)
    assert abs(vm.time - T) < 1e-9 and abs(ref.time - T) < 1e-9
    # the frozen-load reference mode is first order in the elastic coupling: agreement to O(h)
    for a, b in ((vm.s1, ref.slip1), (vm.psi, ref.state)):
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b)

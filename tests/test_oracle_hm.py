"""The numpy oracle (ACA, MVM, DP5(4) stepper) against the reference's own run of
the tiny case (tests/golden/tiny_case.npz, produced by tests/golden/make_golden.py)."""
import numpy as np
import pytest

import qd_oracle
from pyquake3d_b200.hmatrix import aca_start_indices


@pytest.fixture(scope="module")
def oracle_op(tiny_sim, tiny_golden):
    s = tiny_sim
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    blocks = s.tree_block.struct.blocks
    starts = aca_start_indices(blocks, int(tiny_golden["aca_seed"]))
    return qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in blocks], starts, eps=0.01)


def test_aca_ranks_match_reference(oracle_op, tiny_golden):
    r = np.array(oracle_op.ranks())
    assert np.array_equal(r[:, 0], tiny_golden["aca_kS"])
    assert np.array_equal(r[:, 1], tiny_golden["aca_kD"])


def test_aca_factors_match_reference(oracle_op, tiny_golden):
    g = tiny_golden
    idx = sorted({int(k.split("_")[0][1:]) for k in g if k.startswith("f")})
    assert idx
    for i in idx:
        kind, rc, cc, S, D = oracle_op.blocks[i]
        assert kind == "aca"
        for d, sfx in ((S, "s"), (D, "d")):
            for name, key in (("U1", "U_ACA_A1"), ("V1", "V_ACA_A1"), ("U2", "U_ACA_A2"), ("V2", "V_ACA_A2"),
                              ("UB", "U_ACA_B"), ("VB", "V_ACA_B")):
                ref = g["f%d_%s%s" % (i, key, sfx)]
                got = np.asarray(d[name], dtype=np.float64)
                assert got.shape == ref.shape
                np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_mvm_matches_reference(oracle_op, tiny_golden):
    g = tiny_golden
    X = g["mvm_x"]
    for op in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"):
        x = X[0] if op.endswith("s") else X[1]
        y = oracle_op.mvm(x, op)
        ref = g["mvm_" + op]
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


def test_stepper_matches_reference_30_steps(oracle_op, tiny_sim, tiny_golden):
    g = tiny_golden
    s = tiny_sim
    st = qd_oracle.OracleStepper(qd_oracle.sim_state(s), qd_oracle.operator_mvm(oracle_op), s.V0, s.mu, s.Cs)
    dttry = s.htry
    hs = []
    for i in range(30):
        h, dtnext = st.simu_forward(dttry)
        hs.append(h)
        dttry = dtnext
        if i == 0:
            for k in ("Tno", "Tt1o", "Tt2o", "state", "slipv1", "slipv2", "slip1", "slip2"):
                ref = g["step1_" + k]
                assert np.abs(getattr(st, k) - ref).max() <= 1e-12 * np.abs(ref).max() + 1e-300, k
    np.testing.assert_allclose(hs, g["steps_h"], rtol=1e-9)
    np.testing.assert_allclose(st.time, g["steps_time"][-1], rtol=1e-9)
    for k in ("Tno", "Tt1o", "state", "slip1", "slip"):
        ref = g["step30_" + k]
        assert np.abs(getattr(st, k) - ref).max() <= 1e-8 * np.abs(ref).max(), k


# ---------------------------------------------------------------- half space
@pytest.fixture(scope="module")
def tiny_hs_golden():
    import os
    from conftest import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "tiny_hs_case.npz")))


@pytest.fixture(scope="module")
def oracle_op_hs(tiny_sim, tiny_hs_golden):
    s = tiny_sim
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_, hs_mode=2)
    blocks = s.tree_block.struct.blocks
    starts = aca_start_indices(blocks, int(tiny_hs_golden["aca_seed"]))
    return qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in blocks], starts, eps=0.01)


def test_halfspace_operator_matches_reference(oracle_op_hs, tiny_hs_golden):
    """Tiny fault reaching the free surface, `Half space: True`: ACA ranks and the six
    operator products of the reference (its compiled half-space library).

    The half-space entries are a different formulation of the same function
    (agreeing with the reference to ~4e-11 per entry); ACA+ divides the A2 and B
    residuals by their own pivot entries, which magnifies that difference where
    a pivot is small, so the products agree to ~1e-7 of their maximum (ranks and
    pivots identical): 1e-6 here, far inside the ACA truncation error itself."""
    g = tiny_hs_golden
    r = np.array(oracle_op_hs.ranks())
    assert np.array_equal(r[:, 0], g["aca_kS"]) and np.array_equal(r[:, 1], g["aca_kD"])
    X = g["mvm_x"]
    for op in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"):
        y = oracle_op_hs.mvm(X[0] if op.endswith("s") else X[1], op)
        ref = g["mvm_" + op]
        assert np.abs(y - ref).max() <= 1e-6 * np.abs(ref).max(), op


def test_halfspace_stepper_matches_reference(oracle_op_hs, tiny_sim, tiny_hs_golden):
    g = tiny_hs_golden
    st = qd_oracle.OracleStepper(qd_oracle.sim_state(tiny_sim), qd_oracle.operator_mvm(oracle_op_hs), tiny_sim.V0,
                                 tiny_sim.mu, tiny_sim.Cs)
    dttry = tiny_sim.htry
    hs = []
    for _ in range(30):
        h, dttry = st.simu_forward(dttry)
        hs.append(h)
    np.testing.assert_allclose(hs, g["steps_h"], rtol=1e-8)
    for k in ("Tno", "Tt1o", "state", "slip1", "slip"):
        ref = g["step30_" + k]
        assert np.abs(getattr(st, k) - ref).max() <= 1e-7 * np.abs(ref).max(), k

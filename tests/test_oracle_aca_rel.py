"""The oracle's relative-tolerance ACA+ (`ACA relative tolerance: True`).

The reference stops ACA+ on an absolute step size (src/Hmatrix.py:727,736).
The relative stop is this project's key; its oracle restatement
(qd_oracle.aca_plus(rel=True)) keeps the reference's pivots, reference sets
and residual updates and only changes the stopping test.  Pinned here on the
reference's tiny case:
  * the pivot sequence does not depend on the stop, so the relative-mode
    factors are exactly (bitwise) the first k terms of a run that never stops
    on the step size, and that run's pivots are the reference's own (its
    absolute-mode factors are pinned to the reference by test_oracle_hm.py);
  * k is the first step with ||u_k|| ||v_k/alpha|| <= eps ||S_k||_F, where the
    test recomputes ||S_k||_F from the explicit product U[:, :k] V[:k] (the
    oracle updates it incrementally);
  * the approximant meets the tolerance as ACA's step-size heuristic does:
    the median block error ||A1 - S_k||_F / ||A1||_F is at most eps and no
    block exceeds 20 eps (on this case: median 0.5 eps, 90th percentile
    1.1 eps, maximum 11 eps).
"""
import numpy as np
import pytest

import qd_oracle
from pyquake3d_b200.hmatrix import aca_start_indices


@pytest.fixture(scope="module")
def setup(tiny_sim, tiny_golden):
    s = tiny_sim
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    blocks = [b for b in s.tree_block.struct.blocks]
    starts = aca_start_indices(blocks, int(tiny_golden["aca_seed"]))
    aca = [b for b in blocks if b.aca]
    return geo, aca, starts


def _full_run(geo, b, which, start):
    # eps = 0: the step-size test never stops the loop (|alpha| < 1e-4, max_iter or an
    # exhausted reference set still do)
    return qd_oracle.aca_plus(geo, np.asarray(b.row.indices), np.asarray(b.col.indices), which, 0.0, *start)


@pytest.mark.parametrize("eps", [1e-3, 1e-5])
def test_relative_mode_is_prefix_with_explicit_stop(setup, eps):
    geo, aca, starts = setup
    checked = 0
    for bi, b in enumerate(aca):
        for which in (1, 2):
            start = starts[bi][which - 1]
            full = _full_run(geo, b, which, start)
            rel = qd_oracle.aca_plus(geo, np.asarray(b.row.indices), np.asarray(b.col.indices), which, eps, *start,
                                     rel=True)
            k = rel["U1"].shape[1]
            for name in ("U1", "U2"):
                assert np.array_equal(rel[name], full[name][:, :k]), (bi, which, name)
            for name in ("V1", "V2"):
                assert np.array_equal(rel[name], full[name][:k]), (bi, which, name)
            # the stop from explicit Frobenius norms of the A1 approximant
            U, V = full["U1"], full["V1"]
            kk = U.shape[1]
            stop = kk
            for q in range(kk):
                step = np.linalg.norm(U[:, q]) * np.linalg.norm(V[q])     # V rows hold v_q / alpha
                if step <= eps * np.linalg.norm(U[:, :q + 1] @ V[:q + 1]):
                    stop = q + 1
                    break
            assert k == stop, (bi, which, k, stop)
            checked += 1
    assert checked >= 10


@pytest.mark.parametrize("eps", [1e-3, 1e-5])
def test_relative_mode_meets_its_tolerance(setup, eps):
    geo, aca, starts = setup
    errs = []
    for bi, b in enumerate(aca):
        for which in (1, 2):
            r = qd_oracle.aca_plus(geo, np.asarray(b.row.indices), np.asarray(b.col.indices), which, eps,
                                   *starts[bi][which - 1], rel=True)
            A = geo.gf_block(np.asarray(b.row.indices), np.asarray(b.col.indices), which)[0]
            errs.append(np.linalg.norm(A - r["U1"] @ r["V1"]) / np.linalg.norm(A))
    assert np.median(errs) <= eps, np.median(errs)
    assert max(errs) <= 20 * eps, max(errs)

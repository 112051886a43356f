"""GPU: the mixed storage of the low-rank factors (FP32 / FP16 / INT8 term classes).

On the reference's tiny case (device assembly, the reference's absolute ACA):
  * tolerance 0 puts every term in the FP32 class; the mixed kernels then run
    the FP32 plan's operations in the same order, so the products are bitwise
    equal to the FP32 storage's;
  * at 2^-22 and 2^-16 the products stay within the classification's bound of
    the oracle's FP64 blocks_process_MVM products (the bound and the numpy
    emulation of the same kernels: tests/test_mixed_emulation.py), and INT8 /
    FP16 terms are in use;
  * linearity and bitwise determinism;
  * the bulk-copy (streamed) kernels give the plain kernels' products, and
    their status word stays 0 (no wait timed out).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyquake3d_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="module")
def oracle(tiny_sim, tiny_golden):
    import qd_oracle
    from pyquake3d_b200.hmatrix import aca_start_indices
    s = tiny_sim
    st = s.tree_block.struct
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks],
                                  aca_start_indices(st.blocks, int(tiny_golden["aca_seed"])), eps=0.01)
    return st, op


def _device_op(tiny_sim, tiny_golden, tol, stream=True):
    from pyquake3d_b200.hmatrix import DeviceHMatrix
    s = tiny_sim
    op = DeviceHMatrix(s.tree_block.struct, s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_, aca_tol=0.01,
                       aca_rel=False, aca_seed=int(tiny_golden["aca_seed"]), mixed_tol=tol, keep_factors=True)
    op.mixed_stream = stream
    op.use_plan_cache = False          # the FP32 and mixed plans on the same built-in work-item shapes
    return op.assemble(("fp64", "fp32", "mixed"))


def test_mixed_at_zero_tolerance_equals_fp32_bitwise(lib, tiny_sim, tiny_golden):
    op = _device_op(tiny_sim, tiny_golden, 0.0, stream=False)
    ct = op.plan("mixed")["mixed"]["class_terms"]
    assert sum(ct[1]) == 0 and sum(ct[2]) == 0 and not op.plan("mixed")["stream"]
    rng = np.random.default_rng(5)
    x1, x2 = rng.standard_normal((2, op.n))
    a = np.array(op.apply(x1, x2, "mixed"))
    b = np.array(op.apply(x1, x2, "fp32"))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("stream", [True, False])
@pytest.mark.parametrize("tol", [2.0 ** -22, 2.0 ** -16])
def test_mixed_products_within_bound_of_oracle(lib, tiny_sim, tiny_golden, oracle, tol, stream):
    from test_mixed_emulation import _near_rowabs, _reference
    st, oop = oracle
    op = _device_op(tiny_sim, tiny_golden, tol, stream)
    assert op.plan("mixed")["stream"] == stream
    ct = np.array(op.plan("mixed")["mixed"]["class_terms"])
    assert ct[1:].sum() > 0
    if tol == 2.0 ** -16:
        assert ct[2].sum() > 0
    R = _near_rowabs(st, oop)[st.iperm]            # element order
    rng = np.random.default_rng(7)
    x1, x2 = rng.standard_normal((2, op.n))
    y = np.stack(op.apply(x1, x2, "mixed"), axis=1)
    ref = _reference(oop, x1, x2)
    xmax = max(np.abs(x1).max(), np.abs(x2).max())
    err = np.abs(y - ref).max(axis=1) / (R * xmax)
    assert err.max() <= 40 * tol + 2e-6, err.max()
    # linearity and determinism
    a, b = rng.standard_normal((2, 2, op.n))
    ya = np.array(op.apply(a[0], a[1], "mixed"))
    yb = np.array(op.apply(b[0], b[1], "mixed"))
    yab = np.array(op.apply(a[0] + 2 * b[0], a[1] + 2 * b[1], "mixed"))
    assert np.abs(yab - (ya + 2 * yb)).max() <= 1e-5 * np.abs(yab).max()
    assert np.array_equal(ya, np.array(op.apply(a[0], a[1], "mixed")))
    assert op.kernel_status("mixed") == 0


@pytest.mark.parametrize("tol", [0.0, 2.0 ** -16])
def test_streamed_kernels_equal_plain_mixed_kernels(lib, tiny_sim, tiny_golden, oracle, tol):
    """The bulk-copy (streamed) low-rank kernels against k_v_mixed / k_du_mixed on the
    same packed operator: the same products up to FP32 summation order."""
    from test_mixed_emulation import _near_rowabs
    st, _ = oracle
    op = _device_op(tiny_sim, tiny_golden, tol, stream=True)
    rng = np.random.default_rng(9)
    x1, x2 = rng.standard_normal((2, op.n))
    ys = np.stack(op.apply(x1, x2, "mixed"), axis=1)
    assert op.kernel_status("mixed") == 0
    op.mixed_stream = False
    P = op.plans.pop("mixed")
    op.plan("mixed")                          # the same factors, plain layout
    assert not op.plan("mixed")["stream"] and P["stream"]
    yp = np.stack(op.apply(x1, x2, "mixed"), axis=1)
    R = _near_rowabs(st, oracle[1])[st.iperm]
    err = np.abs(ys - yp).max(axis=1) / (R * max(np.abs(x1).max(), np.abs(x2).max()))
    assert err.max() <= 1e-6, err.max()

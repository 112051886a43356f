"""GPU: the batched ACA+ kernel in relative-tolerance mode against the oracle.

Every benchmark configuration from thrust20k up compresses with `ACA relative
tolerance: True`.  The relative stop has no counterpart in the reference; its
oracle restatement (qd_oracle.aca_plus(rel=True), pinned in
tests/test_oracle_aca_rel.py to the reference's own pivot sequence) keeps the
reference's pivots and residual updates.  On a mid-size thrust fault
(2,420 triangles, leaf 64, the thrust20k geometry at 1.8 km edges) at
tolerances 1e-4 and 1e-5, k_aca must give the oracle's rank for every
(block, slip pass), the same first pivot (the first term's A1 factors within
1e-9 of their own largest entry), and the same approximation to the
tolerance: the products U V of all three operators within 2 tol of the A1
product's largest entry in every block, and within 1e-9 in the median block
(on this planar fault the normal-stress operator B is analytically zero, its
factors rounding noise, so B has no scale of its own).  Late terms can differ
by a term's own size: term k divides its residual row by a pivot that has
fallen to about the tolerance times the first one, and where two pivot
candidates are nearly equal the GPU Green's function's own differences from
the C restatement (fused multiply-adds against separately rounded products,
1e-12 to 1e-10 of an entry) can pick the other one; the rank stays the same
(measured at tolerance 1e-5: worst block 8.9e-6, late factors 3e-7 of their
largest entry).
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


def _align(rows, ref_rows):
    """Permutation taking the device's tree-order rows to the oracle's order."""
    pos = {int(e): i for i, e in enumerate(rows)}
    return np.array([pos[int(e)] for e in ref_rows])


@pytest.mark.parametrize("tol", [1e-4, 1e-5])
def test_relative_aca_matches_oracle(lib, tmp_path_factory, tol):
    import qd_oracle
    from pyquake3d_b200 import QDsim, meshgen, read_mshV2
    from pyquake3d_b200.hmatrix import aca_start_indices, export_blocks
    msh, para = meshgen.make_case("thrust20k", str(tmp_path_factory.mktemp("acarel")), n_target=2500, tol=tol)
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para, precision="fp64")
    assert sim.Para0["ACA relative tolerance"] == "True" and float(sim.Para0["ACA tolerance"]) == tol
    st = sim.tree_block.struct
    op = sim.tree_block.op()
    geo = qd_oracle.Geometry(sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_)
    aca = [b for b in st.blocks if b.aca]
    assert len(aca) >= 100
    oop = qd_oracle.build_operator_parallel(geo, [(b.row.indices, b.col.indices, True) for b in aca],
                                            aca_start_indices(st.blocks, 0), eps=tol, rel=True)
    kS, kD = op.ranks()
    ro = np.array(oop.ranks())
    assert np.array_equal(kS, ro[:, 0]) and np.array_equal(kD, ro[:, 1])
    dev = [b for b in export_blocks(op) if b[0] == "aca"]
    worst_f = 0.0
    per_block = []
    for (kind, rows, cols, S, D), (_, rc, cc, So, Do) in zip(dev, oop.blocks):
        ir, ic = _align(rows, rc), _align(cols, cc)
        for d, o in ((S, So), (D, Do)):
            u1, v1 = np.asarray(o["U1"]), np.asarray(o["V1"])
            assert d["U1"].shape == u1.shape and d["V1"].shape == v1.shape
            worst_f = max(worst_f, np.abs(d["U1"][ir, 0] - u1[:, 0]).max() / np.abs(u1[:, 0]).max(),
                          np.abs(d["V1"][0, ic] - v1[0]).max() / np.abs(v1[0]).max())
            scale = np.abs(u1 @ v1).max()
            worst_p = 0.0
            for un, vn in (("U1", "V1"), ("U2", "V2"), ("UB", "VB")):
                uo, vo = np.asarray(o[un], dtype=np.float64), np.asarray(o[vn], dtype=np.float64)
                po = uo @ vo if uo.size else 0.0     # the oracle drops an all-zero B factor
                pd = d[un][ir] @ d[vn][:, ic] if d[un].size else 0.0
                worst_p = max(worst_p, np.abs(pd - po).max() / scale)
            per_block.append(worst_p)
    assert worst_f <= 1e-9, worst_f
    assert max(per_block) <= 2 * tol, max(per_block)
    assert np.median(per_block) <= 1e-9, np.median(per_block)

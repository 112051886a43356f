"""GPU: libpq3d.so behind the reference's own ctypes binding.

The reference loads its Green's-function library with ctypes.CDLL and declares
the two entry points' argument types itself (src/Hmatrix.py:22-49); the drop-in
promise is that pointing that CDLL at libpq3d.so changes nothing else.  This
test binds libpq3d.so afresh with those declarations (pointer-to-double,
size_t, double and bool arguments, no restype), then assembles the reference's
tiny case the way the reference's BlockTree does:
  * dense blocks column by column, one TDstressFS_C call per source triangle
    over the block's receivers (calc_stressfunc_fromCS/CD, src/Hmatrix.py:425-511);
  * ACA residual rows one receiver at a time through
    TDstressEachSourceAtReceiver_C (calc_stressfunc_fromC_rowS/D, :318-422),
    residual columns through TDstressFS_C, inside ACA+ with the reference's
    seeded starts (the oracle's restatement, pinned to the reference);
  * stress projected on the receiver's frame (GetTtstress, :295-313).
The six MVM products of that operator must equal the reference's own products
in tests/golden/tiny_case.npz (computed with the reference's library) to 1e-9
of the operator scale, and the ACA ranks the reference's block by block.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DP = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def reflib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyquake3d_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)        # what the reference's ctypes.CDLL would load
    # the argument types the reference declares for the two entry points
    lib.TDstressFS_C.argtypes = [DP, DP, DP, ctypes.c_size_t, DP, DP, DP, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_bool, DP, DP]
    lib.TDstressEachSourceAtReceiver_C.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, DP, DP, DP,
                                                   ctypes.c_size_t, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_bool, DP, DP]
    return lib


def _p(a):
    return a.ctypes.data_as(DP)


class BindingGeometry:
    """Green's-function blocks through the reference's calling pattern on libpq3d.so;
    gf_block(rows, cols, which) as qd_oracle.Geometry (planes A1, A2, B; 6 for which=3)."""

    def __init__(self, lib, sim):
        self.lib, self.s = lib, sim
        self.calls = {"columns": 0, "rows": 0}

    def _project(self, stress, receivers):
        """stress: 6 x k (xx, yy, zz, xy, xz, yz) at receivers -> (tau1, tau2, sigma_n) x k."""
        ev = self.s.eleVec[receivers]
        e1, e2, e3 = ev[:, 0:3], ev[:, 3:6], ev[:, 6:9]
        tr1 = stress[0] * e3[:, 0] + stress[3] * e3[:, 1] + stress[4] * e3[:, 2]
        tr2 = stress[3] * e3[:, 0] + stress[1] * e3[:, 1] + stress[5] * e3[:, 2]
        trn = stress[4] * e3[:, 0] + stress[5] * e3[:, 1] + stress[2] * e3[:, 2]
        return np.stack([tr1 * e1[:, 0] + tr2 * e1[:, 1] + trn * e1[:, 2],
                         tr1 * e2[:, 0] + tr2 * e2[:, 1] + trn * e2[:, 2],
                         tr1 * e3[:, 0] + tr2 * e3[:, 1] + trn * e3[:, 2]])

    def gf_block(self, rows, cols, which):
        s = self.s
        rows, cols = np.asarray(rows), np.asarray(cols)
        slips = [(1.0, 0.0), (0.0, 1.0)] if which == 3 else [(1.0, 0.0) if which == 1 else (0.0, 1.0)]
        out = np.zeros((3 * len(slips), len(rows), len(cols)))
        tri = np.asarray(s.elelst)
        nodes = np.asarray(s.nodelst)
        for si, (Ss, Ds) in enumerate(slips):
            if which != 3 and len(rows) < len(cols):
                # an ACA residual row: one receiver, every source of the block
                # (calc_stressfunc_fromC_rowS/D)
                P1 = np.ascontiguousarray(nodes[tri[cols, 0] - 1]).ravel()
                P2 = np.ascontiguousarray(nodes[tri[cols, 1] - 1]).ravel()
                P3 = np.ascontiguousarray(nodes[tri[cols, 2] - 1]).ravel()
                for r, i in enumerate(rows):
                    st = np.zeros(6 * len(cols))
                    sn = np.zeros(6 * len(cols))
                    x, y, z = s.xg[i]
                    self.lib.TDstressEachSourceAtReceiver_C(x, y, z, _p(P1), _p(P2), _p(P3), len(cols), Ss, Ds, 0.0,
                                                            s.mu, s.lambda_, False, _p(st), _p(sn))
                    self.calls["rows"] += 1
                    T = self._project(st.reshape(len(cols), 6).T, np.full(len(cols), i))
                    out[3 * si:3 * si + 3, r, :] = T
            else:
                # a dense block or an ACA residual column: one source, every receiver of the
                # block (calc_stressfunc_fromCS/CD)
                X = np.ascontiguousarray(s.xg[rows, 0])
                Y = np.ascontiguousarray(s.xg[rows, 1])
                Z = np.ascontiguousarray(s.xg[rows, 2])
                for c, j in enumerate(cols):
                    P1, P2, P3 = (np.ascontiguousarray(nodes[tri[j, k] - 1]) for k in range(3))
                    st = np.zeros(6 * len(rows))
                    sn = np.zeros(6 * len(rows))
                    self.lib.TDstressFS_C(_p(X), _p(Y), _p(Z), len(rows), _p(P1), _p(P2), _p(P3), Ss, Ds, 0.0,
                                          s.mu, s.lambda_, False, _p(st), _p(sn))
                    self.calls["columns"] += 1
                    out[3 * si:3 * si + 3, :, c] = self._project(st.reshape(len(rows), 6).T, rows)
        return out


def test_reference_binding_reproduces_reference_products(reflib, tiny_sim, tiny_golden):
    import qd_oracle
    from pyquake3d_b200.hmatrix import aca_start_indices
    s = tiny_sim
    g = tiny_golden
    geo = BindingGeometry(reflib, s)
    blocks = s.tree_block.struct.blocks
    op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in blocks],
                                  aca_start_indices(blocks, int(g["aca_seed"])), eps=0.01)
    assert geo.calls["columns"] > 0 and geo.calls["rows"] > 0
    r = np.array(op.ranks())
    assert np.array_equal(r[:, 0], g["aca_kS"]) and np.array_equal(r[:, 1], g["aca_kD"])
    X = g["mvm_x"]
    scale = max(np.abs(g["mvm_" + k]).max() for k in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"))
    for k in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"):
        y = op.mvm(X[0] if k.endswith("s") else X[1], k)
        assert np.abs(y - g["mvm_" + k]).max() <= 1e-9 * scale, (k, np.abs(y - g["mvm_" + k]).max() / scale)

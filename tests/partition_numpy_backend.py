"""Numpy backend of one rank of the row-partitioned step (test infrastructure).

Implements the backend interface of pyquake3d_b200.partition.PartitionedStepper
with the oracle: the rank's blocks as an OracleOperator, the DP5(4) stages of
OracleStepper on the element arrays, maxima and updates restricted to the
rank's rows.  Used by the gloo tests to check the product's orchestration
(partition, deficit exchange, cross-rank maxima, controller) on the CPU."""
import numpy as np
import torch

import qd_oracle


class NumpyRowBackend:
    def __init__(self, sim, rs):
        geo = qd_oracle.Geometry(sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_)
        self.op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in rs.blocks],
                                           rs.aca_starts, eps=0.01)
        self.n = len(sim.xg)
        self.perm = sim.tree_block.struct.perm
        self.tree_rows = self.perm[rs.r0:rs.r1]          # element ids of the rank's rows, tree order
        self.rows = np.sort(self.tree_rows)
        self.st = qd_oracle.OracleStepper(qd_oracle.sim_state(sim), None, sim.V0, sim.mu, sim.Cs, sim.RelTol,
                                          sim.fix_Tn)
        self.y5 = None

    def x_rows(self):
        """The rank's tree-order rows of the deficit, (x1, x2) interleaved."""
        st, e = self.st, self.tree_rows
        out = np.empty(2 * len(e))
        out[0::2] = (st.slipv1 - st.slipvC * np.cos(st.rake0))[e]
        out[1::2] = (st.slipv2 - st.slipvC * np.sin(st.rake0))[e]
        return torch.tensor(out)

    def matvec_gathered(self, xt):
        xt = xt.numpy()
        n, op, st = self.n, self.op, self.st
        x1, x2 = np.empty(n), np.empty(n)
        x1[self.perm] = xt[0::2]
        x2[self.perm] = xt[1::2]
        sigB = op.mvm(x1, "Bs") + op.mvm(x2, "Bd")
        st.AdotV1 = op.mvm(x1, "A1s") + op.mvm(x2, "A1d")
        st.AdotV2 = op.mvm(x1, "A2s") + op.mvm(x2, "A2d")
        st.dsigmadt = st.normal_loading if st.fix_Tn else sigB + st.normal_loading

    def attempt(self, h, first):
        y5, y8 = self.st.rk_stages(h)
        r = self.rows
        rel = [np.abs(np.abs(y8[q][r] - y5[q][r]) / y8[q][r]) for q in range(4)]
        E = np.array([np.max(rel[3]), np.max(rel[1]), np.max(rel[2]), np.max(rel[0])])
        self.y5 = y5
        nan = np.isnan(E)
        return torch.tensor(np.concatenate([np.where(nan, 0.0, E), nan.astype(np.float64)]))

    def accept(self, h):
        st, r = self.st, self.rows
        Tn, T1, T2, ps = (a[r] for a in self.y5)
        st.Tno[r], st.Tt1o[r], st.Tt2o[r], st.state[r] = Tn, T1, T2, ps
        a = st.a[r]
        v1 = (2.0 * st.V0) * np.exp(-ps / a) * np.sinh(T1 / Tn / a)
        v2 = (2.0 * st.V0) * np.exp(-ps / a) * np.sinh(T2 / Tn / a)
        st.slipv1[r], st.slipv2[r] = v1, v2
        v = np.sqrt(v1 * v1 + v2 * v2)
        v[v < 1e-30] = 1e-30
        st.slipv[r] = v
        st.slip1[r] = st.slip1[r] + v1 * h
        st.slip2[r] = st.slip2[r] + v2 * h
        return torch.tensor([np.max(np.abs(v1)), np.max(np.abs(v2)), 0, 0, 0, 0, 0, 0], dtype=torch.float64)


def run_rank(rank, world, files, steps=30, seed=7):
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.partition import PartitionedStepper, RankStructure, TorchComm, row_partition
    msh, para = files
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para)
    st = sim.tree_block.struct
    b = row_partition(st, world)
    rs = RankStructure(st, b[rank], b[rank + 1], seed=seed)
    ps = PartitionedStepper([NumpyRowBackend(sim, rs)], TorchComm(use_dist=True), sim.RelTol)
    dttry = sim.htry
    hs = []
    for _ in range(steps):
        h, dttry = ps.step(dttry)
        hs.append(h)
    return np.array(hs)

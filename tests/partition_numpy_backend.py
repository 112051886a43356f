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

    # The device-controlled forms: the kernels of pq3d_rk_rows_attempt_dev / control /
    # accept_dev / finish (pyquake3d_b200/csrc/rk.cu) emulated on a CPU control block,
    # so that PartitionedStepper.run_device runs over gloo.
    def _pc(self, ps, h, lasth=0.0):
        from pyquake3d_b200 import partition as P
        pc = np.zeros(16)
        pc[P.PC_H], pc[P.PC_TIME], pc[P.PC_STEPS], pc[P.PC_REJ] = h, ps.time, ps.steps, ps.rejects
        pc[P.PC_V1], pc[P.PC_V2] = ps.vmax
        pc[P.PC_FIRST], pc[P.PC_LASTH] = 1.0, lasth
        return torch.tensor(pc)

    def pc_start(self, dttry, ps):
        self.pc = self._pc(ps, dttry)
        self.out = torch.zeros(8, dtype=torch.float64)

    def pc_resume(self, ps, dtnext, h):
        self.pc = self._pc(ps, dtnext, h)

    def attempt_dev(self):
        from pyquake3d_b200 import partition as P
        pc = self.pc
        if pc[P.PC_HALT] == 0 and pc[P.PC_ACC] == 0:
            self.out = self.attempt(float(pc[P.PC_H]), pc[P.PC_FIRST] != 0)
        return self.out

    def control(self, E8, reltol, attempts):
        from pyquake3d_b200 import partition as P
        pc = self.pc
        if pc[P.PC_HALT] != 0 or pc[P.PC_ACC] != 0:
            return
        E = np.where(E8[4:].numpy() > 0, np.nan, E8[:4].numpy())
        mx, mn = P._py_max, P._py_min             # the comparison forms of the kernels (NaN order)
        h = float(pc[P.PC_H])
        R1, R2 = E[0] + 1e-10, mx(mx(E[1], E[2]), E[3]) + 1e-10
        c1, c2 = R1 / reltol, R2 / reltol
        hn1, hn2 = h * 0.9 * (reltol / R1) ** 0.2, h * 0.9 * (reltol / R2) ** 0.2
        pc[P.PC_ATT] += 1
        pc[P.PC_FIRST] = 0
        if mx(c1, c2) < 1.0 and not (np.isnan(c1) or np.isnan(c2)):
            pc[P.PC_DTNEXT] = mn(mn(hn1, hn2), 1.5 * h)
            pc[P.PC_ACC] = 1
            return
        pc[P.PC_DTNEXT] = mn(hn1, hn2)
        pc[P.PC_NRJCT] += 1
        pc[P.PC_H] = mx(0.5 * h, float(pc[P.PC_DTNEXT]))
        if pc[P.PC_H] < 1e-15 or pc[P.PC_NRJCT] > 20:
            pc[P.PC_STATUS], pc[P.PC_HALT] = 1, 1
        elif pc[P.PC_ATT] >= attempts:
            pc[P.PC_HALT] = 1

    def accept_dev(self):
        from pyquake3d_b200 import partition as P
        pc = self.pc
        if pc[P.PC_HALT] == 0 and pc[P.PC_ACC] != 0:
            self.out = self.accept(float(pc[P.PC_H]))
        return self.out

    def finish(self, V8):
        from pyquake3d_b200 import partition as P
        pc = self.pc
        if pc[P.PC_HALT] != 0 or pc[P.PC_ACC] == 0:
            return
        pc[P.PC_TIME] += pc[P.PC_H]
        pc[P.PC_STEPS] += 1
        pc[P.PC_REJ] += pc[P.PC_NRJCT]
        pc[P.PC_V1], pc[P.PC_V2] = V8[0], V8[1]
        pc[P.PC_LASTH] = pc[P.PC_H]
        pc[P.PC_H] = pc[P.PC_DTNEXT]
        pc[P.PC_NRJCT] = pc[P.PC_ACC] = pc[P.PC_ATT] = 0
        pc[P.PC_FIRST] = 1


def run_rank_device(rank, world, files, steps, dttry_scale, attempts, seed=7):
    """run_device over gloo from a trial size dttry_scale x the initial one;
    returns (accepted sizes, rejections)."""
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.partition import PartitionedStepper, RankStructure, TorchComm, row_partition
    msh, para = files
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para)
    st = sim.tree_block.struct
    b = row_partition(st, world)
    rs = RankStructure(st, b[rank], b[rank + 1], seed=seed)
    ps = PartitionedStepper([NumpyRowBackend(sim, rs)], TorchComm(use_dist=True), sim.RelTol, attempts=attempts)
    hs = ps.run_device(steps, sim.htry * dttry_scale, chunk=1)
    return np.array(hs), ps.rejects


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

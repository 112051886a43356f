"""Ensemble host logic on the CPU: the block-diagonal union of per-fault
H-matrix structures, the CTA task table, the seeded ensemble deck, and the
packed matvec of the union (numpy emulation of the kernels) against each
fault's own oracle operator."""
import numpy as np
import pytest

import qd_oracle
from pyquake3d_b200 import QDsim, read_mshV2
from pyquake3d_b200.ensemble import EnsembleStructure, ensemble_tasks
from pyquake3d_b200.hmatrix import aca_start_indices, pack_x
from pyquake3d_b200.meshgen import ensemble_faults
from test_plan_emulation import emulate, pack


@pytest.fixture(scope="module")
def small_ensemble(tmp_path_factory):
    d = tmp_path_factory.mktemp("ens")
    files = ensemble_faults(str(d), n_faults=3, seed=4, lo=150, hi=320, edge=1.0)
    sims = []
    for msh, para in files:
        nodes, tris = read_mshV2(msh)
        sims.append(QDsim(tris, nodes, para))
    return sims


def test_deck_is_seeded_and_uneven(tmp_path):
    a = ensemble_faults(str(tmp_path / "a"), n_faults=4, seed=4, lo=100, hi=400, edge=1.0)
    b = ensemble_faults(str(tmp_path / "b"), n_faults=4, seed=4, lo=100, hi=400, edge=1.0)
    sizes = []
    for (ma, pa), (mb, pb) in zip(a, b):
        assert open(ma).read() == open(mb).read()
        _, ta = read_mshV2(ma)
        sizes.append(len(ta))
    assert len(set(sizes)) > 1 and min(sizes) >= 64


def test_structure_is_block_diagonal(small_ensemble):
    sims = small_ensemble
    structs = [s.tree_block.struct for s in sims]
    E = EnsembleStructure(structs, [0] * len(sims))
    assert E.n == sum(s.n for s in structs)
    assert np.array_equal(np.sort(E.perm), np.arange(E.n))
    assert len(E.blocks) == sum(len(s.blocks) for s in structs)
    fault = E.fault_of_row()
    covered = 0
    for b in E.blocks:
        r, c = b.row, b.col
        # node indices keep the reference's (ascending) order; as sets they are the tree range
        assert np.array_equal(np.sort(E.perm[r.start:r.start + len(r.indices)]), np.sort(r.indices))
        assert np.array_equal(np.sort(E.perm[c.start:c.start + len(c.indices)]), np.sort(c.indices))
        assert fault[r.start] == fault[r.start + len(r.indices) - 1] == fault[c.start]
        covered += len(r.indices) * len(c.indices)
    assert covered == sum(s.n ** 2 for s in structs)
    assert [lf.leaf_id for lf in E.leaves] == list(range(len(E.leaves)))
    want = sum((aca_start_indices(s.blocks, 0) for s in structs), [])
    assert E.aca_starts == want


@pytest.mark.parametrize("rows,task", [([0, 5, 5 + 256, 1000], 256), ([0, 1], 256), ([0, 300, 301, 900], 128)])
def test_task_table(rows, task):
    task_row, task_fault, fault_task = ensemble_tasks(np.array(rows), task)
    assert task_row[0] == 0 and task_row[-1] == rows[-1]
    d = np.diff(task_row)
    assert (d > 0).all() and (d <= task).all()
    for t in range(len(task_fault)):
        f = task_fault[t]
        assert rows[f] <= task_row[t] and task_row[t + 1] <= rows[f + 1]
        assert fault_task[f] <= t < fault_task[f + 1]
    assert fault_task[-1] == len(task_fault)


@pytest.mark.parametrize("code", [0, 2])
def test_union_matvec_equals_per_fault_operators(small_ensemble, code):
    sims = small_ensemble
    structs = [s.tree_block.struct for s in sims]
    E = EnsembleStructure(structs, [0] * len(sims))
    noff = np.concatenate([[0], np.cumsum([len(s.nodelst) for s in sims])])
    geo = qd_oracle.Geometry(np.concatenate([s.xg for s in sims]), np.concatenate([s.eleVec for s in sims]),
                             np.concatenate([s.nodelst for s in sims]),
                             np.concatenate([np.asarray(s.elelst) + o for s, o in zip(sims, noff)]),
                             sims[0].mu, sims[0].lambda_)
    op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in E.blocks], E.aca_starts,
                                  eps=0.01)
    A, D, U, V = pack(E, op, code)
    rng = np.random.default_rng(5)
    x1, x2 = rng.standard_normal((2, E.n))
    y = emulate(E, A, D, U, V, pack_x(x1[E.perm], x2[E.perm], E.n), code)
    out = np.empty_like(y)
    out[E.perm] = y
    for f, (s, st) in enumerate(zip(sims, structs)):
        g = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
        of = qd_oracle.OracleOperator(g, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks],
                                      aca_start_indices(st.blocks, 0), eps=0.01)
        sl = slice(int(E.row0[f]), int(E.row0[f + 1]))
        a1, a2 = x1[sl], x2[sl]
        ref = (of.mvm(a1, "A1s") + of.mvm(a2, "A1d"), of.mvm(a1, "A2s") + of.mvm(a2, "A2d"),
               of.mvm(a1, "Bs") + of.mvm(a2, "Bd"))
        for c in range(3):
            assert np.abs(out[sl, c] - ref[c]).max() <= 1e-12 * np.abs(ref[c]).max(), (f, c)

"""Row partition for several GPUs, on the CPU.

Host logic: safe cuts (leaf starts outside every ACA block's rows), balanced
boundaries, and rank structures that cover the operator exactly once.  The
distributed step: two gloo processes, each owning the rows of its rank, run
PartitionedStepper (the product's orchestration: deficit exchange, max over
ranks of the error maxima per attempt, the reference controller) with a numpy
backend built on the oracle; both follow the reference's 30-step dt sequence
of the tiny case (tests/golden/tiny_case.npz)."""
import os
import socket

import numpy as np
import pytest

from pyquake3d_b200.hmatrix import HStructure, aca_start_indices
from pyquake3d_b200.partition import RankStructure, row_partition, safe_cuts


@pytest.fixture(scope="module")
def big_struct():
    rng = np.random.default_rng(1)
    u, w = rng.uniform(0, 1, (2, 6000))
    xg = np.stack([80 * u, 0.3 * np.sin(6 * u), -20 * w], axis=1)
    return HStructure(xg, mini_leaf=64, eta=2.0, min_size=16)


def test_safe_cuts(big_struct):
    st = big_struct
    cuts = safe_cuts(st)
    assert cuts[0] == 0 and cuts[-1] == st.n
    starts = {lf.start for lf in st.leaves}
    for c in cuts[1:-1]:
        assert c in starts
        for b in st.blocks:
            if b.aca:
                assert not (b.row.start < c < b.row.start + len(b.row.indices))


@pytest.mark.parametrize("R", [2, 3, 4])
def test_partition_balanced_and_covering(big_struct, R):
    st = big_struct
    b = row_partition(st, R)
    assert b[0] == 0 and b[-1] == st.n and (np.diff(b) > 0).all()
    from pyquake3d_b200.partition import row_costs
    na = sum(1 for x in st.blocks if x.aca)
    cost = row_costs(st, np.full(na, 16), np.full(na, 16), 1)
    share = np.array([cost[b[r]:b[r + 1]].sum() for r in range(R)]) / cost.sum()
    assert share.max() <= 1.25 / R
    seen = np.zeros((st.n, st.n), dtype=np.int8)
    for r in range(R):
        rs = RankStructure(st, b[r], b[r + 1])
        for blk in rs.blocks:
            lo, hi = getattr(blk, "rows", (0, len(blk.row.indices)))   # shared low-rank blocks: own rows only
            r0, r1 = blk.row.start + lo, blk.row.start + hi
            assert b[r] <= r0 and r1 <= b[r + 1]
            c0, n = blk.col.start, len(blk.col.indices)
            seen[r0:r1, c0:c0 + n] += 1
    assert (seen == 1).all()


def test_shared_low_rank_rows_partition_the_block(big_struct):
    st = big_struct
    b = row_partition(st, 3)
    rows = {}
    for r in range(3):
        for blk in RankStructure(st, b[r], b[r + 1]).blocks:
            if blk.aca:
                lo, hi = getattr(blk, "rows", (0, len(blk.row.indices)))
                rows.setdefault(id(blk.row), []).append((blk.row.start + lo, blk.row.start + hi, len(blk.col.indices),
                                                         blk.col.start))
    for parts in rows.values():
        parts.sort()
        assert all(parts[i][1] == parts[i + 1][0] for i in range(len(parts) - 1)) or len(set(p[3] for p in parts)) > 1


def test_rank_structure_keeps_global_aca_starts(big_struct):
    st = big_struct
    b = row_partition(st, 2)
    starts = aca_start_indices(st.blocks, 3)
    got = []
    for r in range(2):
        rs = RankStructure(st, b[r], b[r + 1], seed=3)
        got += list(zip(rs.aca_global, rs.aca_starts))
    for i, s in got:                       # shared blocks appear on both ranks, with the same starts
        assert s == starts[i]
    assert sorted(set(i for i, _ in got)) == list(range(len(starts)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, files, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from partition_numpy_backend import run_rank
        hs = run_rank(rank, world, files)
        out_q.put((rank, hs))
    except Exception as e:       # report to the parent instead of hanging it
        out_q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_follow_reference(tiny_files, tiny_golden):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, tiny_files, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    for r in range(2):
        assert not isinstance(res[r], str), res[r]
        np.testing.assert_allclose(res[r], tiny_golden["steps_h"], rtol=1e-8)
    assert np.array_equal(res[0], res[1])


def _worker_device(rank, world, port, files, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from partition_numpy_backend import run_rank_device
        out_q.put((rank, run_rank_device(rank, world, files, 8, 2.0 ** 36, attempts=1)))
    except Exception as e:
        out_q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_device_controller(tiny_files, tiny_golden):
    """PartitionedStepper.run_device over two gloo ranks, the control kernels
    emulated on the CPU, one attempt slot per step and a first trial size 2^36
    times the initial one: the first step is rejected 5 times, so the device
    sequence halts and the host controller finishes it; every rank issues the
    same collectives whatever the decisions.  Sizes and rejections equal the
    oracle's single-process stepping from the same trial size."""
    import torch.multiprocessing as mp
    import qd_oracle
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1])
    st = sim.tree_block.struct
    geo = qd_oracle.Geometry(sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_)
    op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks],
                                  aca_start_indices(st.blocks, 7), eps=0.01)
    ref = qd_oracle.OracleStepper(qd_oracle.sim_state(sim), qd_oracle.operator_mvm(op), sim.V0, sim.mu, sim.Cs,
                                  sim.RelTol, sim.fix_Tn)
    dt, hs, rej = sim.htry * 2.0 ** 36, [], 0
    for _ in range(8):
        h, dt = ref.simu_forward(dt)
        hs.append(h)
        rej += ref.nrjct
    assert rej >= 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_device, args=(r, 2, port, tiny_files, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    for r in range(2):
        assert not isinstance(res[r], str), res[r]
        np.testing.assert_allclose(res[r][0], hs, rtol=1e-8)
        assert res[r][1] == rej
    assert np.array_equal(res[0][0], res[1][0])


@pytest.mark.parametrize("R", [2, 3, 5])
def test_rank_plans_sum_to_the_operator(tiny_sim, tiny_golden, R):
    """Packed per-rank plans (numpy emulation of the kernels), shared low-rank
    blocks included, add up to the full operator; each rank writes only its rows."""
    import qd_oracle
    from pyquake3d_b200.hmatrix import pack_x
    from test_plan_emulation import emulate, pack
    s = tiny_sim
    st = s.tree_block.struct
    seed = int(tiny_golden["aca_seed"])
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    full = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks],
                                    aca_start_indices(st.blocks, seed), eps=0.01)
    rng = np.random.default_rng(2)
    x1, x2 = rng.standard_normal((2, st.n))
    x = pack_x(x1[st.perm], x2[st.perm], st.n)
    b = row_partition(st, R, slack=0.0)
    total = np.zeros((st.n, 3))
    shared = 0
    for r in range(R):
        rs = RankStructure(st, b[r], b[r + 1], seed=seed)
        shared += sum(1 for blk in rs.blocks if hasattr(blk, "rows"))
        op = qd_oracle.OracleOperator(geo, [(blk.row.indices, blk.col.indices, blk.aca) for blk in rs.blocks],
                                      rs.aca_starts, eps=0.01)
        A, D, U, V = pack(rs, op, 0)
        y = emulate(rs, A, D, U, V, x, 0)
        outside = np.ones(st.n, dtype=bool)
        outside[b[r]:b[r + 1]] = False
        assert (y[outside] == 0).all()
        total += y
    out = np.empty_like(total)
    out[st.perm] = total
    ref = (full.mvm(x1, "A1s") + full.mvm(x2, "A1d"), full.mvm(x1, "A2s") + full.mvm(x2, "A2d"),
           full.mvm(x1, "Bs") + full.mvm(x2, "Bd"))
    for c in range(3):
        assert np.abs(out[:, c] - ref[c]).max() <= 1e-12 * np.abs(ref[c]).max()
    if R >= 3:
        assert shared > 0

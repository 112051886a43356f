"""Host logic against the reference run on the tiny case: mesh reading, element
frames, initial conditions and the H-matrix block structure."""
import numpy as np
import pytest

from pyquake3d_b200 import read_mshV2, get_eleVec
from pyquake3d_b200.hmatrix import HStructure, aca_start_indices


def test_mesh_and_frames(tiny_files, tiny_golden):
    g = tiny_golden
    nodes, tris = read_mshV2(tiny_files[0])
    assert np.array_equal(nodes, g["nodes"])
    assert np.array_equal(tris, g["tris"])
    ev, xg = get_eleVec(nodes, tris, False)
    assert np.array_equal(ev, g["eleVec"])
    assert np.array_equal(xg, g["xg"])


def test_initial_conditions(tiny_sim, tiny_golden):
    g = tiny_golden
    for k in ("Tno", "Tt1o", "Tt2o", "state", "slipv1", "slipv2", "slipv", "a", "b", "dc", "f0", "rake",
              "shear_loading", "normal_loading", "slipvC", "Tt", "fric"):
        assert np.array_equal(getattr(tiny_sim, k), g["init_" + k]), k


def test_block_structure_matches_reference(tiny_sim, tiny_golden):
    g = tiny_golden
    blocks = tiny_sim.tree_block.struct.blocks
    assert len(blocks) == len(g["blk_m"])
    ro = np.concatenate([[0], np.cumsum(g["blk_m"])])
    co = np.concatenate([[0], np.cumsum(g["blk_n"])])
    for i, b in enumerate(blocks):
        assert np.array_equal(b.row.indices, g["blk_rows"][ro[i]:ro[i + 1]])
        assert np.array_equal(b.col.indices, g["blk_cols"][co[i]:co[i + 1]])
        assert b.aca == bool(g["blk_aca"][i])


def test_tree_order_ranges(tiny_sim):
    s = tiny_sim.tree_block.struct
    assert np.array_equal(np.sort(s.perm), np.arange(s.n))
    for b in s.blocks:
        assert np.array_equal(np.sort(s.perm[b.row.start:b.row.start + len(b.row.indices)]), b.row.indices)
        assert np.array_equal(np.sort(s.perm[b.col.start:b.col.start + len(b.col.indices)]), b.col.indices)


def test_blocks_cover_matrix_once(tiny_sim):
    s = tiny_sim.tree_block.struct
    cover = np.zeros((s.n, s.n), dtype=np.int32)
    for b in s.blocks:
        cover[np.ix_(b.row.indices, b.col.indices)] += 1
    assert (cover == 1).all()


def test_seeded_aca_starts_match_reference_draws(tiny_sim, tiny_golden):
    """np.random.seed(s) + the reference's randint calls == aca_start_indices(blocks, s)."""
    blocks = tiny_sim.tree_block.struct.blocks
    st = aca_start_indices(blocks, int(tiny_golden["aca_seed"]))
    np.random.seed(int(tiny_golden["aca_seed"]))
    for b, (s, d) in zip([b for b in blocks if b.aca], st):
        m, n = len(b.row.indices), len(b.col.indices)
        assert s == (np.random.randint(m) - 3, np.random.randint(n) - 3)
        assert d == (np.random.randint(m) - 3, np.random.randint(n) - 3)


def test_plan_cache_picks_entry_of_nearest_size(tmp_path, monkeypatch):
    """Work-item shapes: the autotuner's entry tuned on the workload size closest to
    the operator's (log scale); a single-entry cache (older form) still reads."""
    import json
    from pyquake3d_b200 import hmatrix
    cache = {"GPU X": {"fp32": [dict(dense_chunk=4, v_chunk=8, u_rows=256, workload="plain2k (1936 triangles)"),
                                dict(dense_chunk=16, v_chunk=64, u_rows=512, n=59696)],
                       "mixed": dict(dense_chunk=16, v_chunk=64, u_rows=512, workload="curved60k (59696 triangles)")}}
    p = tmp_path / "plan_cache.json"
    p.write_text(json.dumps(cache))
    monkeypatch.setattr(hmatrix, "PLAN_CACHE", str(p))
    monkeypatch.setattr(hmatrix, "_plan_cache", None)
    assert hmatrix.plan_cache_entry("GPU X", "fp32", 2000)["dense_chunk"] == 4
    assert hmatrix.plan_cache_entry("GPU X", "fp32", 20480)["dense_chunk"] == 16
    assert hmatrix.plan_cache_entry("GPU X", "fp32", 120000)["dense_chunk"] == 16
    assert hmatrix.plan_cache_entry("GPU X", "mixed", 2000)["v_chunk"] == 64
    assert hmatrix.plan_cache_entry("GPU X", "bf16", 2000) is None
    assert hmatrix.plan_cache_entry("GPU Y", "fp32", 2000) is None


def test_prefetch_copier_hands_out_fresh_copies():
    """The reference loop's attribute reads go through the host copier: every read of
    every step gets its own array (the loop keeps them all), equal to the pinned
    buffer at that step even after the buffer is overwritten, and an error in the
    wait reaches the reader."""
    import threading
    from pyquake3d_b200 import qdsim

    class NoDevice(qdsim._PrefetchCopier):
        def _bind(self, device_index):
            pass

    class Done:
        def __init__(self):
            self.ev = threading.Event()

        def synchronize(self):
            self.ev.wait(5.0)

    n = 1000
    c = NoDevice(n, 0, spare=4)
    buf = {"slipv": np.zeros(n), "Tt": np.zeros(n)}
    kept = []
    for step in range(20):
        buf["slipv"][:] = step
        buf["Tt"][:] = -step
        d = Done()
        job = c.submit(d, buf, ("Tt", "slipv"))
        d.ev.set()
        assert job.has("slipv") and job.has("Tt")
        v, t = job.get("slipv"), job.get("Tt")
        assert not job.has("slipv")
        kept.append((step, v, t))
    for step, v, t in kept:
        assert np.all(v == step) and np.all(t == -step)
    assert len({id(v) for _, v, _ in kept}) == len(kept)

    class Bad:
        def synchronize(self):
            raise RuntimeError("wait failed")

    job = c.submit(Bad(), buf, ("slipv",))
    with pytest.raises(RuntimeError):
        job.get("slipv")
    c.stop()

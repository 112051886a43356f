"""Host logic of the packed H-matvec, checked without a GPU.

The oracle's FP64 operator (dense blocks + ACA factors of the tiny case) is
packed into the device layouts with the same index formulas the CUDA kernels
use (hm_layout.cuh: dense_index, u_index, v_index; k_dense_assemble and
k_aca_pack write that way), then the work items, slots and per-leaf slot lists
from build_plan_arrays are executed by numpy emulations of k_dense_v,
k_u and k_rowsum.  The result must equal the oracle's
blocks_process_MVM products."""
import numpy as np
import pytest

import qd_oracle
from pyquake3d_b200.hmatrix import aca_start_indices, build_plan_arrays, dense_layout, pack_x, x_stride

CW_D = {0: 2, 1: 4, 2: 4}
CW_L = {0: 2, 1: 4, 2: 8}


def dense_index(m, i, j, c, s, cw):
    return (((j // cw) * 6 + 2 * c + s) * m + i) * cw + (j % cw)


def u_index(m, i, c, q, cw):
    return (((q // cw) * 3 + c) * m + i) * cw + (q % cw)


def v_index(Q, q, jj, cw):
    return ((jj // cw) * Q + q) * cw + (jj % cw)


@pytest.fixture(scope="module")
def setup(tiny_sim, tiny_golden):
    s = tiny_sim
    st = s.tree_block.struct
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    starts = aca_start_indices(st.blocks, int(tiny_golden["aca_seed"]))
    op = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks], starts, eps=0.01)
    return st, op


def pack(st, op, code):
    """Pack the oracle operator like k_dense_assemble / k_aca_pack (tree order)."""
    cwd, cwl = CW_D[code], CW_L[code]
    dblocks = [b for b in st.blocks if not b.aca]
    recs, off64, off32 = dense_layout(dblocks)
    D = np.zeros(max(off64 if code == 0 else off32, 1))
    offs = recs["off64"] if code == 0 else recs["off32"]
    ob = [b for b in op.blocks if b[0] == "dense"]
    for k, b in enumerate(dblocks):
        M = ob[k][3]                       # 6 x m x n, reference order (ascending element ids)
        m, n = M.shape[1:]
        # tree-local index of each of the block's elements
        ti = st.iperm[b.row.indices] - b.row.start
        tj = st.iperm[b.col.indices] - b.col.start
        I, J = np.meshgrid(ti, tj + b.col.start % cwd, indexing="ij")
        for slip in range(2):
            for c in range(3):
                D[offs[k] + dense_index(m, I, J, c, slip, cwd)] = M[3 * slip + c]
    ranks = np.array(op.ranks()).reshape(-1, 2)
    A = build_plan_arrays(st, recs, ranks[:, 0], ranks[:, 1], code, dense_chunk=2, v_chunk=3, u_rows=40)
    U = np.zeros(max(A["u_size"], 8))
    V = np.zeros(max(A["v_size"], 8))
    ab = [b for b in st.blocks if b.aca]
    oa = [b for b in op.blocks if b[0] == "aca"]
    for (bi, p, u_off, v_off, K, Q, ks, kd) in A["pack"]:
        b = ab[bi]
        d = oa[bi][3 if p == 0 else 4]
        m, n = len(b.row.indices), len(b.col.indices)
        ti = st.iperm[b.row.indices] - b.row.start
        tj = st.iperm[b.col.indices] - b.col.start
        k = ks if p == 0 else kd
        qoff = 0 if p == 0 else ks
        for c, (un, vn) in enumerate((("U1", "V1"), ("U2", "V2"), ("UB", "VB"))):
            Uc = np.asarray(d[un]) if len(d[un]) else np.zeros((m, k))
            Vc = np.asarray(d[vn]) if len(d[vn]) else np.zeros((k, n))
            for q in range(k):
                U[u_off + u_index(m, ti, c, qoff + q, cwl)] = Uc[:, q]
                row = c * ks + q if p == 0 else 3 * ks + c * kd + q
                V[v_off + v_index(Q, row, b.col.start % cwl + tj, cwl)] = Vc[q]
    return A, D, U, V


def emulate(st, A, D, U, V, x, code):
    cwd, cwl = CW_D[code], CW_L[code]
    for it in A["ditems"][:A["n_ditems"]]:
        assert int(it["c0"]) % cwd == 0          # aligned x slices (vector loads)
    for it in A["vitems"][:A["n_vitems"]]:
        assert int(it["c0"]) % cwl == 0
    slots = np.zeros(3 * max(A["n_slots"], 1))
    tpart = np.zeros(max(A["n_tpart"], 1))
    for it in A["ditems"][:A["n_ditems"]]:
        m, r0 = int(it["m"]), int(it["r"])
        rr = np.arange(r0, min(r0 + 32, m))
        acc = np.zeros((len(rr), 3))
        for g in range(int(it["g0"]), int(it["g1"])):
            for c in range(3):
                for s in range(2):
                    for t in range(cwd):
                        j = g * cwd + t
                        acc[:, c] += D[it["off"] + ((g * 6 + 2 * c + s) * m + rr) * cwd + t] * \
                            x[2 * (int(it["c0"]) + j) + s]
        slots[3 * (int(it["slot"]) + rr)[:, None] + np.arange(3)] = acc
    for it in A["vitems"][:A["n_vitems"]]:
        Q, q0, nr, s = int(it["Q"]), int(it["q"]), int(it["nr"]), int(it["s"])
        for q in range(q0, q0 + nr):
            acc = 0.0
            for g in range(int(it["g0"]), int(it["g1"])):
                for t in range(cwl):
                    acc += V[it["off"] + (g * Q + q) * cwl + t] * x[(2 + s) * x_stride(st.n) + int(it["c0"]) + g * cwl + t]
            tpart[int(it["tp"]) + q] = acc
    for T in A["utasks"][:A["n_utasks"]]:
        ks, kd, K, Q, m = int(T["kS"]), int(T["kD"]), int(T["K"]), int(T["Q"]), int(T["m"])
        tv = np.zeros(3 * K)
        for c in range(3):
            for q in range(K):
                row = c * ks + q if q < ks else (3 * ks + c * kd + q - ks if q < ks + kd else -1)
                if row >= 0:
                    tv[c * K + q] = sum(tpart[int(T["tp"]) + ch * Q + row] for ch in range(int(T["nch"])))
        rr = np.arange(int(T["r0"]), int(T["r1"]))
        acc = np.zeros((len(rr), 3))
        for g in range(K // cwl):
            for c in range(3):
                for k in range(cwl):
                    acc[:, c] += U[T["off"] + ((g * 3 + c) * m + rr) * cwl + k] * tv[c * K + g * cwl + k]
        slots[3 * (int(T["slot"]) + rr)[:, None] + np.arange(3)] = acc
    y = np.zeros((st.n, 3))
    for i in range(st.n):
        lf = A["leaf_of_row"][i]
        for k in range(A["leaf_ptr"][lf], A["leaf_ptr"][lf + 1]):
            y[i] += slots[3 * (A["leaf_off"][k] + i):3 * (A["leaf_off"][k] + i) + 3]
    return y


@pytest.mark.parametrize("code", [0, 1, 2])
def test_packed_matvec_emulation_equals_oracle(setup, code):
    st, op = setup
    A, D, U, V = pack(st, op, code)
    rng = np.random.default_rng(11)
    x1, x2 = rng.standard_normal((2, st.n))
    x = pack_x(x1[st.perm], x2[st.perm], st.n)
    y = emulate(st, A, D, U, V, x, code)
    out = np.empty_like(y)
    out[st.perm] = y
    ref = (op.mvm(x1, "A1s") + op.mvm(x2, "A1d"), op.mvm(x1, "A2s") + op.mvm(x2, "A2d"),
           op.mvm(x1, "Bs") + op.mvm(x2, "Bd"))
    for c in range(3):
        assert np.abs(out[:, c] - ref[c]).max() <= 1e-12 * np.abs(ref[c]).max(), c


def test_slot_lists_cover_every_row_owner_once(setup):
    st, op = setup
    ranks = np.array(op.ranks()).reshape(-1, 2)
    recs, _, _ = dense_layout([b for b in st.blocks if not b.aca])
    A = build_plan_arrays(st, recs, ranks[:, 0], ranks[:, 1], 2, dense_chunk=4, v_chunk=2, u_rows=16)
    owner_of_slot = np.full(A["n_slots"], -1)
    for k, (s0, r0, m) in enumerate(A["slot_rows"]):
        owner_of_slot[s0:s0 + m] = k
    assert (owner_of_slot >= 0).all()
    for i in range(st.n):
        lf = A["leaf_of_row"][i]
        slots = A["leaf_off"][A["leaf_ptr"][lf]:A["leaf_ptr"][lf + 1]] + i
        own = owner_of_slot[slots]
        assert len(set(own.tolist())) == len(own)          # each owner once
        for sl, o in zip(slots, own):
            s0, r0, m = A["slot_rows"][o]
            assert r0 <= i < r0 + m and sl - s0 == i - r0  # the slot of row i in that owner
        # all owners covering row i are listed
        cover = [k for k, (s0, r0, m) in enumerate(A["slot_rows"]) if r0 <= i < r0 + m]
        assert sorted(cover) == sorted(own.tolist())

"""Host logic of the mixed storage (FP32 / FP16 / INT8 ACA term classes), checked
without a GPU.

The oracle's FP64 operator of the reference's tiny case is classified and
packed with the index formulas of the CUDA kernels (mixed_pack.cu:
k_nearfield_rowabs, k_term_weights, k_pack_mixed; hm_layout.cuh u_index /
v_index with column groups 4, 8, 16); every packed index is checked against
the array sizes build_plan_arrays_mixed gives, and the work items are executed
by numpy emulations of k_v_mixed, k_du_mixed and k_rowsum (INT8 entries are
stored as the byte b + 128 and the arrays filled with 128, which decodes to
zero in padding).  The products must
stay within the classification's error bound of the oracle's FP64
blocks_process_MVM products: every row within a small multiple of
tol * R_i * max|x| (R_i the near-field absolute row sum the weights use), and
equal to FP32 rounding when the tolerance admits no quantised term."""
import numpy as np
import pytest

import qd_oracle
from pyquake3d_b200.hmatrix import (MIXED_CW, aca_start_indices, build_plan_arrays_mixed, classify_terms,
                                    dense_layout, pack_x, x_stride)


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


def _near_rowabs(st, op):
    """k_nearfield_rowabs: R3[c][tree row] = sum over dense blocks of |K^c| (both slips)."""
    R3 = np.zeros((3, st.n))
    for b, ob in zip([b for b in st.blocks if not b.aca], [b for b in op.blocks if b[0] == "dense"]):
        M = ob[3]
        rows = st.iperm[b.row.indices]
        for c in range(3):
            R3[c, rows] += np.abs(M[c]).sum(axis=1) + np.abs(M[3 + c]).sum(axis=1)
    return R3.max(axis=0)


def _factors(d, name_u, name_v, m, n, k):
    U = np.asarray(d[name_u]) if len(d[name_u]) else np.zeros((m, k))
    V = np.asarray(d[name_v]) if len(d[name_v]) else np.zeros((k, n))
    return U, V


def _weights(st, op, R):
    """k_term_weights: w = max over components of max_i(|u_i| / R_i) * ||v||_1."""
    out = []
    for b, ob in zip([b for b in st.blocks if b.aca], [b for b in op.blocks if b[0] == "aca"]):
        m, n = len(b.row.indices), len(b.col.indices)
        Rr = R[st.iperm[b.row.indices]]
        per = []
        for d in (ob[3], ob[4]):
            k = np.asarray(d["U1"]).shape[1]
            w = np.zeros(k)
            for un, vn in (("U1", "V1"), ("U2", "V2"), ("UB", "VB")):
                U, V = _factors(d, un, vn, m, n, k)
                w = np.maximum(w, (np.abs(U) / Rr[:, None]).max(axis=0) * np.abs(V).sum(axis=1))
            per.append(w)
        out.append(per)
    return out


def pack_mixed(st, op, tol, stream=False):
    recs, _, off32 = dense_layout([b for b in st.blocks if not b.aca])
    D = np.zeros(max(off32, 1), np.float32)
    for k, (b, ob) in enumerate(zip([b for b in st.blocks if not b.aca], [b for b in op.blocks if b[0] == "dense"])):
        M = ob[3]
        m = M.shape[1]
        ti = st.iperm[b.row.indices] - b.row.start
        tj = st.iperm[b.col.indices] - b.col.start
        I, J = np.meshgrid(ti, tj + b.col.start % 4, indexing="ij")
        for s_ in range(2):
            for c in range(3):
                D[recs["off32"][k] + dense_index(m, I, J, c, s_, 4)] = M[3 * s_ + c]
    R = _near_rowabs(st, op)
    W = _weights(st, op, R)
    cls_lists = [classify_terms(wS, wD, tol) for wS, wD in W]
    A = build_plan_arrays_mixed(st, recs, cls_lists, dense_chunk=2, v_chunk=3, u_rows=40, stream=stream, ncta=5,
                                nwarps=16)
    dt, fill = (np.float32, np.float16, np.uint8), (0, 0, 128)      # INT8 entries stored as b + 128
    U = [np.full(max(A["u_sizes"][c], 16), fill[c], dt[c]) for c in range(3)]
    V = [np.full(max(A["v_sizes"][c], 16), fill[c], dt[c]) for c in range(3)]
    scales = np.zeros(max(A["n_scales"], 4), np.float32)
    layout = {(bi, p): (uo, vo, ks, kd, Q, K, sb) for (bi, p, uo, vo, ks, kd, Q, K, sb) in A["pack"]}
    ab, oa = [b for b in st.blocks if b.aca], [b for b in op.blocks if b[0] == "aca"]
    for bi, b in enumerate(ab):
        m, n = len(b.row.indices), len(b.col.indices)
        ti = st.iperm[b.row.indices] - b.row.start
        tj = st.iperm[b.col.indices] - b.col.start
        for p in (0, 1):
            if (bi, p) not in layout:
                continue
            uo, vo, ks, kd, Q, K, sb = layout[(bi, p)]
            d = oa[bi][3 + p]
            cl = cls_lists[bi][p]
            k = len(cl)
            for q in range(k):
                c_ = int(cl[q])
                pos = int((cl[:q] == c_).sum())
                col = pos if p == 0 else ks[c_] + pos
                cw = MIXED_CW[c_]
                for c, (un, vn) in enumerate((("U1", "V1"), ("U2", "V2"), ("UB", "VB"))):
                    Uc, Vc = _factors(d, un, vn, m, n, k)
                    u, v = Uc[:, q], Vc[q]
                    row = c * ks[c_] + pos if p == 0 else 3 * ks[c_] + c * kd[c_] + pos
                    iu = uo[c_] + u_index(m, ti, c, col, cw)
                    iv = vo[c_] + v_index(Q[c_], row, b.col.start % cw + tj, cw)
                    assert iu.max() < A["u_sizes"][c_] and iv.max() < A["v_sizes"][c_]
                    assert (iu >= uo[c_]).all() and (iv >= vo[c_]).all()
                    if c_ == 0:
                        U[0][iu], V[0][iv] = u.astype(np.float32), v.astype(np.float32)
                        continue
                    su, sv = np.abs(u).max(), np.abs(v).max()
                    if su == 0 or sv == 0:
                        continue
                    assert sb[c_] + row < A["n_scales"]
                    if c_ == 1:
                        U[1][iu] = (u / su).astype(np.float32).astype(np.float16)
                        V[1][iv] = (v / sv).astype(np.float32).astype(np.float16)
                        scales[sb[1] + row] = np.float32(su * sv)
                    else:
                        U[2][iu] = (np.clip(np.rint(127 * u / su), -127, 127) + 128).astype(np.uint8)
                        V[2][iv] = (np.clip(np.rint(127 * v / sv), -127, 127) + 128).astype(np.uint8)
                        scales[sb[2] + row] = np.float32(su * sv / 127.0 ** 2)
    return A, D, U, V, scales, R, cls_lists


def _decode(a, cls):
    """Stored class entries as float64 (INT8 bytes hold b + 128)."""
    return a.astype(np.float64) - 128.0 if cls == 2 else a.astype(np.float64)


def emulate_stream(st, A, D, U, V, scales, x):
    """k_stream phase A (dense and V tasks), k_t_gather, k_stream phase B (U tasks), k_rowsum:
    every task read through the byte ranges its pieces copy, checked against the arrays."""
    P = x_stride(st.n)
    STAGE, BUF = 12288, 3072
    slots = np.zeros(3 * max(A["n_slots"], 1))
    tpart = np.zeros(max(A["n_tpart"], 1))
    for name, ncta in (("a", A["ncta_a"]), ("b", A["ncta_b"])):
        cta = A["cta_" + name]
        assert cta[0] == 0 and np.all(np.diff(cta) >= 0)
        if name == "b":
            # k_t_gather: the blocks' t, contiguous per block
            tfull = np.zeros(max(A["n_tfull"], 4))
            for g in A["gather"][:A["n_gather"]]:
                o = int(g["tb"])
                for cls in range(3):
                    K, ks, kd, Q = (int(g[k][cls]) for k in ("K", "kS", "kD", "Q"))
                    for e in range(3 * K):
                        c, q = divmod(e, K)
                        row = c * ks + q if q < ks else (3 * ks + c * kd + q - ks if q < ks + kd else -1)
                        if row >= 0:
                            v = sum(tpart[int(g["tp"][cls]) + ch * Q + row] for ch in range(int(g["nch"][cls])))
                            tfull[o + e] = v * (scales[int(g["sb"][cls]) + row] if cls else 1.0)
                    o += 3 * K
                assert o <= A["n_tfull"]
        for T in A["tasks_" + name][:cta[ncta]]:
            kind, G = int(T["kind"]), int(T["g1"]) - int(T["g0"])
            if kind == 0:
                m, r0, r1, g0 = int(T["m"]), int(T["r0"]), int(T["r1"]), int(T["g0"])
                R = r1 - r0
                assert 1 <= R <= 128 and 8 * G <= BUF and 6 * R * 16 <= STAGE and int(T["c0"]) % 4 == 0
                rr = np.arange(r0, r1)
                acc = np.zeros((R, 3))
                for g in range(g0, g0 + G):
                    for c in range(3):
                        for sl in range(2):
                            idx = int(T["off"]) + ((g * 6 + 2 * c + sl) * m + rr)[:, None] * 4 + np.arange(4)
                            assert idx.max() < len(D)
                            xv = x[2 * (int(T["c0"]) + g * 4 + np.arange(4)) + sl]
                            acc[:, c] += D[idx].astype(np.float64) @ xv
                slots[3 * (int(T["out"]) + rr)[:, None] + np.arange(3)] = acc
            elif kind == 1:
                cls, Q, kS3, g0 = int(T["cls"]), int(T["m"]), int(T["kS3"]), int(T["g0"])
                cw = MIXED_CW[cls]
                assert Q * 16 <= STAGE and 2 * G * cw <= BUF and int(T["c0"]) % cw == 0
                for q in range(Q):
                    plane = 2 if q < kS3 else 3
                    acc = 0.0
                    for g in range(g0, g0 + G):
                        idx = int(T["off"]) + (g * Q + q) * cw + np.arange(cw)
                        assert idx.max() < len(V[cls])
                        acc += float(np.dot(_decode(V[cls][idx], cls), x[plane * P + int(T["c0"]) + g * cw + np.arange(cw)]))
                    tpart[int(T["out"]) + q] = acc
            else:
                m, r0, r1, tb = int(T["m"]), int(T["r0"]), int(T["r1"]), int(T["tb"])
                Ks = (int(T["K0"]), int(T["K1"]), int(T["K2"]))
                assert 1 <= r1 - r0 <= 256 and 3 * sum(Ks) <= BUF
                rr = np.arange(r0, r1)
                acc = np.zeros((len(rr), 3))
                base = tb
                for cls, off in enumerate((int(T["off"]), int(T["off1"]), int(T["off2"]))):
                    cw, K = MIXED_CW[cls], Ks[cls]
                    for g in range(K // cw):
                        for c in range(3):
                            for k in range(cw):
                                idx = off + ((g * 3 + c) * m + rr) * cw + k
                                assert idx.max() < len(U[cls])
                                acc[:, c] += _decode(U[cls][idx], cls) * tfull[base + c * K + g * cw + k]
                    base += 3 * K
                slots[3 * (int(T["out"]) + rr)[:, None] + np.arange(3)] = acc
    y = np.zeros((st.n, 3))
    for i in range(st.n):
        lf = A["leaf_of_row"][i]
        for k in range(A["leaf_ptr"][lf], A["leaf_ptr"][lf + 1]):
            y[i] += slots[3 * (A["leaf_off"][k] + i):3 * (A["leaf_off"][k] + i) + 3]
    return y


def emulate(st, A, D, U, V, scales, x):
    if A.get("stream"):
        return emulate_stream(st, A, D, U, V, scales, x)
    slots = np.zeros(3 * max(A["n_slots"], 1))
    tpart = np.zeros(max(A["n_tpart"], 1))
    for it in A["ditems"][:A["n_ditems"]]:
        m, r0 = int(it["m"]), int(it["r"])
        rr = np.arange(r0, min(r0 + 32, m))
        acc = np.zeros((len(rr), 3))
        for g in range(int(it["g0"]), int(it["g1"])):
            for c in range(3):
                for s in range(2):
                    for t in range(4):
                        acc[:, c] += D[it["off"] + ((g * 6 + 2 * c + s) * m + rr) * 4 + t] * \
                            x[2 * (int(it["c0"]) + g * 4 + t) + s]
        slots[3 * (int(it["slot"]) + rr)[:, None] + np.arange(3)] = acc
    # merged V items: rows (one class, one slip) of the blocks sharing a column cluster,
    # each row with its own class-array base, group stride and t index
    written = np.zeros(len(tpart), dtype=bool)
    vw = A["vwarp"]                       # k_v_mixed's per-warp item lists
    assert vw[0] == 0 and vw[-1] == A["n_vitems"] and np.all(np.diff(vw) >= 0)
    for it in (A["vitems"][i] for w in range(len(vw) - 1) for i in range(vw[w], vw[w + 1])):
        cls, slip = int(it["s"]) >> 8, int(it["s"]) & 255
        cw = MIXED_CW[cls]
        assert int(it["c0"]) % cw == 0 and 0 < int(it["nr"]) <= 32
        for R in A["vrows"][int(it["rows"]):int(it["rows"]) + int(it["nr"])]:
            acc = 0.0
            for g in range(int(it["g0"]), int(it["g1"])):
                idx = int(R["base"]) + g * int(R["stride"]) + np.arange(cw)
                assert idx.max() < len(V[cls])
                acc += float(np.dot(_decode(V[cls][idx], cls),
                                    x[(2 + slip) * x_stride(st.n) + int(it["c0"]) + g * cw + np.arange(cw)]))
            assert not written[int(R["out"])]          # every partial written once
            written[int(R["out"])] = True
            tpart[int(R["out"])] = acc
    for T in A["utasks"][:A["n_utasks"]]:
        m = int(T["m"])
        rr = np.arange(int(T["r0"]), int(T["r1"]))
        acc = np.zeros((len(rr), 3))
        for cls in range(3):
            K, ks, kd, Q = int(T["K"][cls]), int(T["kS"][cls]), int(T["kD"][cls]), int(T["Q"][cls])
            cw = MIXED_CW[cls]
            assert K % cw == 0
            tv = np.zeros(3 * K)
            for c in range(3):
                for q in range(K):
                    row = c * ks + q if q < ks else (3 * ks + c * kd + q - ks if q < ks + kd else -1)
                    if row >= 0:
                        v = sum(tpart[int(T["tp"][cls]) + ch * Q + row] for ch in range(int(T["nch"][cls])))
                        tv[c * K + q] = v * (scales[int(T["sb"][cls]) + row] if cls else 1.0)
            for g in range(K // cw):
                for c in range(3):
                    for k in range(cw):
                        idx = T["off"][cls] + ((g * 3 + c) * m + rr) * cw + k
                        assert idx.max() < len(U[cls])
                        acc[:, c] += _decode(U[cls][idx], cls) * tv[c * K + g * cw + k]
        slots[3 * (int(T["slot"]) + rr)[:, None] + np.arange(3)] = acc
    y = np.zeros((st.n, 3))
    for i in range(st.n):
        lf = A["leaf_of_row"][i]
        for k in range(A["leaf_ptr"][lf], A["leaf_ptr"][lf + 1]):
            y[i] += slots[3 * (A["leaf_off"][k] + i):3 * (A["leaf_off"][k] + i) + 3]
    return y


def _reference(op, x1, x2):
    return np.stack([op.mvm(x1, "A1s") + op.mvm(x2, "A1d"), op.mvm(x1, "A2s") + op.mvm(x2, "A2d"),
                     op.mvm(x1, "Bs") + op.mvm(x2, "Bd")], axis=1)


@pytest.mark.parametrize("stream", [False, True])
@pytest.mark.parametrize("tol", [0.0, 2.0 ** -22, 2.0 ** -16])
def test_mixed_matvec_emulation_within_bound(setup, tol, stream):
    st, op = setup
    A, D, U, V, scales, R, cls = pack_mixed(st, op, tol, stream)
    if stream:
        assert A["ncta_a"] > 1 and A["ncta_b"] > 1
    rng = np.random.default_rng(7)
    x1, x2 = rng.standard_normal((2, st.n))
    x = pack_x(x1[st.perm], x2[st.perm], st.n)
    y = emulate(st, A, D, U, V, scales, x)
    out = np.empty_like(y)
    out[st.perm] = y
    ref = _reference(op, x1, x2)
    xmax = max(np.abs(x1).max(), np.abs(x2).max())
    Rel = R[st.iperm]                       # element order
    err = np.abs(out - ref).max(axis=1) / (Rel * xmax)
    n_q = sum(int((c > 0).sum()) for cs in cls for c in cs)
    if tol == 0.0:
        assert n_q == 0                      # every term FP32
        assert err.max() <= 2e-6, err.max()
    else:
        # each quantised term moves a row by at most ~tol R_i max|x|; a row meets a few
        # dozen such terms, whose errors are mostly independent
        assert n_q > 0
        assert err.max() <= 40 * tol + 2e-6, (err.max(), tol)
    if tol == 2.0 ** -16:
        assert sum(int((c == 2).sum()) for cs in cls for c in cs) > 0      # INT8 terms exercised


@pytest.mark.parametrize("tol", [2.0 ** -22, 2.0 ** -16])
def test_u_task_prefetch_runs_cover_the_task_reads(setup, tol):
    """k_du_mixed's U-task CTAs prefetch their rows into L2 before waiting for the V kernel:
    one bulk prefetch per (class, column group, component), starting at byte
    off_c * size_c + ((3 g + c) m + r0) * 16 with length (r1 - r0) * 16.  Restated here:
    every run lies inside its class array, starts 16-byte aligned, has a nonzero size that
    is a multiple of 16, and the runs cover exactly the 16-byte units the task's rows read."""
    st, op = setup
    A, D, U, V, scales, R, cls = pack_mixed(st, op, tol)
    size = (4, 2, 1)
    for T in A["utasks"][:A["n_utasks"]]:
        m, r0, r1 = int(T["m"]), int(T["r0"]), int(T["r1"])
        nr = r1 - r0
        assert nr > 0
        for c in range(3):
            cw, K, off = MIXED_CW[c], int(T["K"][c]), int(T["off"][c])
            assert K % cw == 0
            runs = set()
            for q in range(3 * (K // cw)):                  # the kernel's run index e - n_prev
                start = off * size[c] + (q * m + r0) * 16
                assert start % 16 == 0 and nr * 16 > 0
                assert start + nr * 16 <= len(U[c]) * size[c]
                runs.update(range(start // 16, start // 16 + nr))
            reads = set()
            for g in range(K // cw):
                for comp in range(3):
                    e = off + ((g * 3 + comp) * m + np.arange(r0, r1)) * cw    # u_row_class's units
                    reads.update((e * size[c] // 16).tolist())
            assert runs == reads


def test_classify_terms_keeps_required_precision():
    rng = np.random.default_rng(3)
    tol = 2.0 ** -22
    eps16, eps8 = 2.0 ** -11, 0.5 / 127
    for _ in range(200):
        kS, kD = rng.integers(0, 40, 2)
        wS = 10 ** rng.uniform(-12, -3, kS)
        wD = 10 ** rng.uniform(-12, -3, kD)
        cS, cD = classify_terms(wS, wD, tol)
        w = np.concatenate([wS, wD])
        c = np.concatenate([cS, cD])
        req = np.where(2 * eps16 * w > tol, 0, np.where(2 * eps8 * w > tol, 1, 2))
        assert (c <= req).all()                                     # never less precise than required
        # classes are ordered by weight: a more important term is never in a lower class
        o = np.argsort(-w, kind="stable")
        assert (np.diff(c[o]) >= 0).all()

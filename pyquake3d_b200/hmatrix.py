"""H-matrix structure (host) and the packed device operator.

Host part (FP64, numpy), a restatement of src/Hmatrix.py:
  * build_cluster_tree  <- build_block_tree   (:143-182)  bisection of the
    longest bounding-box axis at its midpoint, leaves of <= min_size elements;
  * is_admissible       <- is_admissible      (:88-103)   min(diam) <= eta*dist;
  * build_blocks        <- create_recursive_blocks + collect_blocks (:1611-1672,
    :1291-1297) quad-split, a leaf when admissible or when either cluster has
    <= mini_leaf elements; leaves listed depth-first (the reference's order);
  * ACA vs dense        <- BlockTree.ACA_worker (:1014-1066): ACA when both
    dimensions exceed mini_leaf, dense otherwise.
Every cluster is also given its range in tree order (depth-first, left child
first), the layout of all device vectors.

Device part: DeviceHMatrix assembles the operator on the GPU (dense near field
with the FP64 Green's function, admissible blocks with batched ACA), packs it
for one or more storage precisions and applies it with pq3d_hmatvec.
"""
import math
import os

import numpy as np

from . import _lib
from ._lib import ptr, check

# ----------------------------------------------------------------------------- host tree


class ClusterNode:
    __slots__ = ("indices", "left", "right", "start", "level", "bbox_min", "bbox_max", "leaf_id", "_box")

    def __init__(self, indices, level):
        self.indices = indices
        self.left = None
        self.right = None
        self.start = 0
        self.level = level
        self.bbox_min = None
        self.bbox_max = None
        self._box = None
        self.leaf_id = -1


def build_cluster_tree(points, min_size=16):
    """Cluster tree of build_block_tree (src/Hmatrix.py:143-182).

    Returns (root, perm, leaves): perm[p] = element at tree position p."""
    root = ClusterNode(np.arange(len(points)), 0)
    stack = [(root, points)]
    while stack:
        node, pts = stack.pop()
        cl = node.indices
        node.bbox_min = np.min(pts, axis=0)
        node.bbox_max = np.max(pts, axis=0)
        if len(cl) <= min_size:
            continue
        alpha, beta = node.bbox_min, node.bbox_max
        j = int(np.argmax(beta - alpha))
        gamma = (alpha[j] + beta[j]) / 2
        i1 = pts[:, j] <= gamma
        i2 = pts[:, j] > gamma
        t1, t2 = cl[i1], cl[i2]
        if len(t1) == 0 or len(t2) == 0:
            continue
        node.left = ClusterNode(t1, node.level + 1)
        node.right = ClusterNode(t2, node.level + 1)
        stack.append((node.right, pts[i2]))
        stack.append((node.left, pts[i1]))
    # tree-order ranges (left first) and leaves
    perm = np.empty(len(points), dtype=np.int64)
    leaves = []
    pos = 0
    st = [root]
    while st:
        nd = st.pop()
        nd.start = pos if nd.left is None else nd.start
        if nd.left is None:
            nd.start = pos
            nd.leaf_id = len(leaves)
            leaves.append(nd)
            perm[pos:pos + len(nd.indices)] = nd.indices
            pos += len(nd.indices)
        else:
            st.append(nd.right)
            st.append(nd.left)
    _fix_starts(root)
    return root, perm, leaves


def _fix_starts(root):
    st = [root]
    order = []
    while st:
        nd = st.pop()
        order.append(nd)
        if nd.left is not None:
            st.append(nd.right)
            st.append(nd.left)
    for nd in reversed(order):
        if nd.left is not None:
            nd.start = nd.left.start


def _box(nd):
    """(bbox_min, bbox_max as floats, diameter) of a cluster, computed once."""
    if nd._box is None:
        lo, hi = [float(v) for v in nd.bbox_min], [float(v) for v in nd.bbox_max]
        e = [h - l for l, h in zip(lo, hi)]
        nd._box = (lo, hi, math.sqrt((e[0] * e[0] + e[1] * e[1]) + e[2] * e[2]))
    return nd._box


def is_admissible(a, b, eta):
    """min(diam_a, diam_b) <= eta * dist(bbox_a, bbox_b).  The sums run in numpy's
    order for three terms ((t0 + t1) + t2) and every operation is correctly rounded,
    so the decisions are those of the reference's numpy expression."""
    alo, ahi, da = _box(a)
    blo, bhi, db = _box(b)
    t = []
    for k in range(3):
        u = max(0.0, blo[k] - ahi[k])
        v = max(0.0, alo[k] - bhi[k])
        t.append(u * u + v * v)
    dq = math.sqrt((t[0] + t[1]) + t[2])
    return min(da, db) <= eta * dq


class LeafBlock:
    """A leaf of the block tree: rows = row cluster, cols = col cluster."""
    __slots__ = ("row", "col", "aca", "admissible", "level")

    def __init__(self, row, col, aca, admissible, level):
        self.row = row
        self.col = col
        self.aca = aca
        self.admissible = admissible
        self.level = level

    @property
    def row_cluster(self):
        return self.row.indices

    @property
    def col_cluster(self):
        return self.col.indices

    @property
    def judaca(self):
        return self.aca


def build_blocks(row_root, col_root, eta=2.0, mini_leaf=32):
    """Leaves of create_recursive_blocks in collect_blocks (depth-first) order."""
    out = []
    st = [(row_root, col_root, 0)]
    while st:
        r, c, lev = st.pop()
        adm = is_admissible(r, c, eta)
        if adm or len(r.indices) <= mini_leaf or len(c.indices) <= mini_leaf or \
                r.left is None or r.right is None or c.left is None or c.right is None:
            aca = len(r.indices) > mini_leaf and len(c.indices) > mini_leaf
            out.append(LeafBlock(r, c, aca, bool(adm), lev))
            continue
        st.append((r.right, c.right, lev + 1))
        st.append((r.right, c.left, lev + 1))
        st.append((r.left, c.right, lev + 1))
        st.append((r.left, c.left, lev + 1))
    return out


class HStructure:
    """Cluster trees and leaf blocks of the operator (the part QDsim.__init__ builds)."""

    def __init__(self, xg, mini_leaf=32, eta=2.0, min_size=16):
        self.n = len(xg)
        self.mini_leaf = mini_leaf
        self.eta = eta
        self.min_size = min_size
        self.row_root, self.perm, self.leaves = build_cluster_tree(xg, min_size)
        # the reference builds the column tree with the same call: identical tree
        self.col_root = self.row_root
        self.iperm = np.empty_like(self.perm)
        self.iperm[self.perm] = np.arange(self.n)
        self.blocks = build_blocks(self.row_root, self.col_root, eta, mini_leaf)

    def stats(self):
        nd = sum(1 for b in self.blocks if not b.aca)
        na = len(self.blocks) - nd
        dense_entries = sum(len(b.row.indices) * len(b.col.indices) for b in self.blocks if not b.aca)
        aca_mn = sum(len(b.row.indices) + len(b.col.indices) for b in self.blocks if b.aca)
        return dict(n=self.n, blocks=len(self.blocks), dense_blocks=nd, aca_blocks=na,
                    dense_entries=dense_entries, aca_m_plus_n=aca_mn, leaves=len(self.leaves))


def aca_start_indices(blocks, seed):
    """Starting reference row/col of every ACA pass, drawn as the reference does
    (np.random.randint(n_rows) - 3, np.random.randint(n_cols) - 3 for the strike
    pass, then again for the dip pass, src/Hmatrix.py:660-661 and :888-889), with
    a seeded legacy RandomState and blocks taken in list order."""
    rs = np.random.RandomState(seed)
    out = []
    for b in blocks:
        if not b.aca:
            continue
        m, n = len(b.row.indices), len(b.col.indices)
        s = (rs.randint(m) - 3, rs.randint(n) - 3)
        d = (rs.randint(m) - 3, rs.randint(n) - 3)
        out.append((s, d))
    return out


# ----------------------------------------------------------------------------- packed layout (host)


def x_stride(n):
    """Plane stride of the device deficit vector (hm_layout.cuh x_stride)."""
    return ((n + 16 + 7) // 8) * 8


def pack_x(x1, x2, n):
    """Deficit vector in the device layout: interleaved pairs, then strike and dip
    planes (x1, x2 already in tree order)."""
    P = x_stride(n)
    x = np.zeros(4 * P)
    x[0:2 * n:2] = x1
    x[1:2 * n:2] = x2
    x[2 * P:2 * P + n] = x1
    x[3 * P:3 * P + n] = x2
    return x


def dense_layout(dense_blocks):
    """DenseBlock records with FP64 / FP32 offsets, and the two array sizes.  Stored
    columns start at the column-group-aligned c0 - (c0 % CW)."""
    recs = np.zeros(len(dense_blocks), dtype=_lib.DENSE_BLOCK)
    off64 = off32 = 0
    for i, b in enumerate(dense_blocks):
        m, n, c0 = len(b.row.indices), len(b.col.indices), b.col.start
        recs[i] = (off64, off32, m, n, b.row.start, c0)
        off64 += _cdiv(n + c0 % 2, 2) * m * 12
        off32 += _cdiv(n + c0 % 4, 4) * m * 24
    return recs, off64, off32


def build_plan_arrays(struct, dense_recs, kS, kD, code, dense_chunk=64, v_chunk=256, u_rows=512):
    """Matvec work items, slot layout and per-leaf slot lists for storage code
    (0 FP64, 1 FP32, 2 FP32 dense + BF16 low rank).  Pure numpy.

    Slots: every dense (block, column chunk) and every low-rank block owns m
    consecutive slots (one per block row); row i of a block with slot base s
    and first row r0 writes slot s + (i - r0).  leaf_off lists, per leaf
    cluster, the offsets s - r0 of all slot owners covering that leaf."""
    cwd, cwl = _CW_DENSE[code], _CW_LR[code]
    n = struct.n
    dense_off = dense_recs["off64"] if code == 0 else dense_recs["off32"]
    ditems, slot_rows, slot = _dense_items(dense_recs, cwd, dense_off, dense_chunk)
    aca_blocks = [b for b in struct.blocks if b.aca]
    u_off = v_off = tp = 0
    vitems, utasks, pack = [], [], []
    lr_entries = 0
    kmax = 0
    for bi, b in enumerate(aca_blocks):
        m, nn = len(b.row.indices), len(b.col.indices)
        lo, hi = getattr(b, "rows", (0, m))      # block-local rows this plan computes (all, unless clipped)
        ks, kd = int(kS[bi]), int(kD[bi])
        lr_entries += 3 * (ks + kd) * ((hi - lo) + nn)
        if ks + kd == 0:
            continue
        K = _cdiv(ks + kd, cwl) * cwl
        kmax = max(kmax, K)
        Q = 3 * (ks + kd)
        lead = b.col.start % cwl
        ngv = _cdiv(nn + lead, cwl)
        npad = ngv * cwl
        nch = _cdiv(ngv, v_chunk)
        for ch in range(nch):
            g0 = ch * v_chunk
            g1 = min(ngv, g0 + v_chunk)
            for s_, (qa, qb) in enumerate(((0, 3 * ks), (3 * ks, Q))):
                for q in range(qa, qb, 32):
                    vitems.append((v_off, Q, q, min(32, qb - q), g0, g1, b.col.start - lead, s_, tp + ch * Q))
        # row r of the block writes slot (slot - lo) + r, for r in [lo, hi)
        for r0 in range(lo, hi, u_rows):
            utasks.append((u_off, m, r0, min(hi, r0 + u_rows), K, ks, kd, Q, tp, nch, slot - lo))
        slot_rows.append((slot, b.row.start + lo, hi - lo))
        for p in (0, 1):
            pack.append((bi, p, u_off, v_off, K, Q, ks, kd))
        slot += hi - lo
        tp += nch * Q
        u_off += (K // cwl) * m * 3 * cwl
        v_off += Q * npad
    L = _leaf_lists(struct, slot_rows)
    esz_d = 8 if code == 0 else 4
    esz_l = {0: 8, 1: 4, 2: 2}[code]
    dense_entries = int(np.sum(dense_recs["m"].astype(np.int64) * dense_recs["n"])) if len(dense_recs) else 0
    return dict(ditems=_rec(ditems, _lib.DENSE_ITEM), vitems=_rec(vitems, _lib.V_ITEM),
                utasks=_rec(utasks, _lib.U_TASK),
                n_ditems=len(ditems), n_vitems=len(vitems), n_utasks=len(utasks), n_slots=slot, n_tpart=tp, kmax=kmax,
                u_size=u_off, v_size=v_off, pack=pack, alg_bytes=dense_entries * 6 * esz_d + lr_entries * esz_l +
                2 * n * esz_d + 3 * n * 8, **L)


def _dense_items(dense_recs, cwd, dense_off, dense_chunk):
    """Dense work items (one warp: 32 rows x a chunk of column groups) and their slots:
    every (block, column chunk) owns m consecutive slots."""
    ditems, slot_rows = [], []
    slot = 0
    for i in range(len(dense_recs)):
        m, nn, r0, c0 = (int(dense_recs[k][i]) for k in ("m", "n", "r0", "c0"))
        lead = c0 % cwd
        ng = _cdiv(nn + lead, cwd)
        for g0 in range(0, ng, dense_chunk):
            g1 = min(ng, g0 + dense_chunk)
            for r in range(0, m, 32):
                ditems.append((int(dense_off[i]), m, r, g0, g1, c0 - lead, slot))
            slot_rows.append((slot, r0, m))
            slot += m
    return ditems, slot_rows, slot


def _leaf_lists(struct, slot_rows):
    """Per leaf cluster, the offsets (slot - first row) of every slot owner covering it."""
    n = struct.n
    nleaf = len(struct.leaves)
    leaf_of_row = np.empty(n, dtype=np.int32)
    for lf in struct.leaves:
        leaf_of_row[lf.start:lf.start + len(lf.indices)] = lf.leaf_id
    sr = np.array(slot_rows, dtype=np.int64).reshape(-1, 3)
    first = leaf_of_row[sr[:, 1]].astype(np.int64)
    last = leaf_of_row[sr[:, 1] + sr[:, 2] - 1].astype(np.int64)
    cnt = last - first + 1
    rep_leaf = np.repeat(first, cnt) + (np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    rep_off = np.repeat(sr[:, 0] - sr[:, 1], cnt)
    order = np.argsort(rep_leaf, kind="stable")
    leaf_off = rep_off[order].astype(np.int32)
    leaf_ptr = np.zeros(nleaf + 1, dtype=np.int64)
    np.add.at(leaf_ptr, rep_leaf + 1, 1)
    leaf_ptr = np.cumsum(leaf_ptr).astype(np.int32)
    return dict(leaf_of_row=leaf_of_row, leaf_ptr=leaf_ptr,
                leaf_off=leaf_off if len(leaf_off) else np.zeros(1, np.int32), slot_rows=sr)


# ----------------------------------------------------------------------------- mixed storage (host)

MIXED_CW = (4, 8, 16)               # column groups of the FP32 / FP16 / INT8 term classes
MIXED_BYTES = (4, 2, 1)
# relative rounding of a stored entry against its vector's largest magnitude
MIXED_EPS = (2.0 ** -24, 2.0 ** -11, 0.5 / 127.0)


def classify_terms(wS, wD, tol):
    """Classes (0 FP32, 1 FP16, 2 INT8) of one block's ACA terms from their weights
    w = max_i(|u_i| / R_i) ||v||_1 (strike terms wS, dip terms wD, in ACA order).

    A term needs FP32 when 2 eps_FP16 w > tol (quantising u and v to FP16 would move a
    row by more than tol times its near-field absolute row sum), FP16 when 2 eps_INT8 w
    > tol, else INT8 suffices.  Each class's column count is padded to its column
    group (4, 8, 16); the padding is filled by promoting the next most important terms
    instead of storing zeros, and an INT8 remnant of at most 8 terms (or an FP16
    remnant of at most 4 after FP32 and with no INT8 terms) moves up a class at no
    extra storage.  Returns (cls_S, cls_D) arrays of class codes."""
    w = np.concatenate([np.asarray(wS, dtype=np.float64), np.asarray(wD, dtype=np.float64)])
    K = len(w)
    if K == 0:
        return np.zeros(0, np.int32), np.zeros(0, np.int32)
    req = np.where(2 * MIXED_EPS[1] * w > tol, 0, np.where(2 * MIXED_EPS[2] * w > tol, 1, 2))
    n0, n1 = int((req == 0).sum()), int((req == 1).sum())
    n0p = min(K, _cdiv(n0, 4) * 4) if n0 else 0
    rem1 = max(0, n0 + n1 - n0p)
    left = K - n0p
    n1p = min(left, _cdiv(rem1, 8) * 8) if rem1 else 0
    n2p = left - n1p
    if 0 < n2p <= 8:
        n1p, n2p = n1p + n2p, 0
    if n2p == 0 and 0 < n1p <= 4 and n0p % 4 == 0:
        n0p, n1p = n0p + n1p, 0
    order = np.argsort(-w, kind="stable")
    cls = np.empty(K, np.int32)
    cls[order[:n0p]] = 0
    cls[order[n0p:n0p + n1p]] = 1
    cls[order[n0p + n1p:]] = 2
    return cls[:len(wS)], cls[len(wS):]


def build_plan_arrays_mixed(struct, dense_recs, cls_lists, dense_chunk=16, v_chunk=32, u_rows=512, stream=False,
                            ncta=148, nwarps=None):
    """Work items, slot layout and packing records of the mixed storage (code 3):
    FP32 dense items as in the FP32 plan; per low-rank block and term class c
    (FP32, FP16, INT8) the class's own U / V arrays with column groups MIXED_CW[c].
    cls_lists[bi] = (cls_S, cls_D) from classify_terms.  Pure numpy.

    stream=True lays the work out for the persistent bulk-copy kernel k_stream:
    StreamTask lists of phase A (dense tasks of at most STREAM_DENSE_ROWS rows and
    1,024 columns; V tasks over all rows of one class of one block and at most
    1,024 columns) and phase B (U tasks of at most STREAM_ROWS rows), each list
    split over `ncta` persistent CTAs balanced by the bytes they stream, plus
    one TGather record per low-rank block (the t it gathers into tfull)."""
    if stream:
        return _build_stream_mixed(struct, dense_recs, cls_lists, ncta)
    ditems, slot_rows, slot = _dense_items(dense_recs, 4, dense_recs["off32"], dense_chunk)
    aca_blocks = [b for b in struct.blocks if b.aca]
    u_off, v_off = [0, 0, 0], [0, 0, 0]
    tp = sb = 0
    vitems, utasks, pack = [], [], []
    lr_bytes = 0
    kmax = 0
    counts = np.zeros((3, 2), np.int64)      # terms per (class, slip)
    vgroups = {}                             # (column start, columns, class) -> the blocks' V rows
    for bi, b in enumerate(aca_blocks):
        m, nn = len(b.row.indices), len(b.col.indices)
        lo, hi = getattr(b, "rows", (0, m))
        cS, cD = cls_lists[bi]
        ks = np.bincount(cS, minlength=3).tolist()
        kd = np.bincount(cD, minlength=3).tolist()
        if sum(ks) + sum(kd) == 0:
            continue
        Ks = [_cdiv(ks[c] + kd[c], MIXED_CW[c]) * MIXED_CW[c] for c in range(3)]
        Qs = [3 * (ks[c] + kd[c]) for c in range(3)]
        kmax = max(kmax, sum(Ks))
        rec_off, rec_tp, rec_nch, rec_sb, rec_voff = [0] * 3, [0] * 3, [0] * 3, [0] * 3, [0] * 3
        for c in range(3):
            counts[c] += (ks[c], kd[c])
            cw = MIXED_CW[c]
            lr_bytes += Qs[c] * ((hi - lo) + nn) * MIXED_BYTES[c] + (Qs[c] * 4 if c else 0)
            rec_off[c], rec_voff[c] = u_off[c], v_off[c]
            if Ks[c] == 0:
                continue
            lead = b.col.start % cw
            ngv = _cdiv(nn + lead, cw)
            gch = min(v_chunk, _lib.STREAM_XMAX // cw) if stream else v_chunk
            nch = _cdiv(ngv, gch)
            if stream and Qs[c] * 16 > _lib.STREAM_STAGE_BYTES:
                raise _lib.Pq3dError("a block's term class has %d V rows, more than one stream stage holds" % Qs[c])
            if stream:
                for ch in range(nch):
                    g0, g1 = ch * gch, min(ngv, (ch + 1) * gch)
                    vitems.append((v_off[c], Qs[c], 0, Qs[c], g0, g1, b.col.start - lead, (3 * ks[c]) | (c << 16),
                                   tp + ch * Qs[c]))
            else:
                # the block's V rows join those of the other blocks with the same columns
                vgroups.setdefault((b.col.start, nn, c), []).append((v_off[c], Qs[c], 3 * ks[c], tp))
            rec_tp[c], rec_nch[c] = tp, nch
            tp += nch * Qs[c]
            if c:
                rec_sb[c] = sb
                sb += Qs[c]
            u_off[c] += Ks[c] * m * 3
            v_off[c] += Qs[c] * ngv * cw
        for r0 in range(lo, hi, u_rows):
            utasks.append((rec_off, m, r0, min(hi, r0 + u_rows), slot - lo, Ks, ks, kd, Qs, rec_tp, rec_nch, rec_sb, 0))
        slot_rows.append((slot, b.row.start + lo, hi - lo))
        for p in (0, 1):
            pack.append((bi, p, rec_off, rec_voff, ks, kd, Qs, Ks, rec_sb))
        slot += hi - lo
    A = _leaf_lists(struct, slot_rows)
    dense_entries = int(np.sum(dense_recs["m"].astype(np.int64) * dense_recs["n"])) if len(dense_recs) else 0
    n = struct.n
    vrows = vwarp = None
    if not stream:
        if max(v_off) >= 1 << 32:
            raise _lib.Pq3dError("a V class array of the mixed storage holds 2^32 elements or more")
        vitems, vwarp, vrows = _merged_v_items(vgroups, v_chunk, nwarps or VMIX_WARPS)
    A.update(ditems=_rec(ditems, _lib.DENSE_ITEM), vitems=_rec(vitems, _lib.V_ITEM_M if not stream else _lib.V_ITEM),
             vrows=vrows, vwarp=vwarp, utasks=_rec(utasks, _lib.U_TASK_M), n_ditems=len(ditems), n_vitems=len(vitems), n_utasks=len(utasks),
             n_slots=slot, n_tpart=tp, n_scales=sb, kmax=kmax, u_sizes=u_off, v_sizes=v_off, pack=pack, stream=stream,
             class_terms=counts, alg_bytes=dense_entries * 6 * 4 + lr_bytes + 2 * n * 4 + 3 * n * 8)
    return A


VMIX_WARPS = 8 * 148 * 4      # k_v_mixed warps when no device says otherwise (B200, 4 CTAs per SM)
VMIX_ROWS = 32                # rows per merged V item (k_v_mixed handles up to 32)


def _merged_v_items(vgroups, v_chunk, nwarps=VMIX_WARPS):
    """V items of the mixed storage's plain kernels (k_v_mixed): for each column
    cluster, class and slip, the V rows of all low-rank blocks with those columns
    (in block order), per column chunk, 32 rows to an item, so the x slice is loaded
    once for all of them.  vgroups: (column start, columns, class) -> [(V offset of
    the block in its class array, Q, strike rows, t base)].  Returns the items
    ordered by warp, the per-warp offsets (nwarps + 1) and the row records.  Items go
    largest first to the least loaded of the nwarps warps (cost: row slots of 8 x
    column groups, plus a fixed start), so the persistent warps end together."""
    items, recs = [], []
    nrec = 0
    for (col0, nn, c), blocks in vgroups.items():
        cw = MIXED_CW[c]
        lead = col0 % cw
        ngv = _cdiv(nn + lead, cw)
        nch = _cdiv(ngv, v_chunk)
        bl = np.array(blocks, dtype=np.int64).reshape(-1, 4)     # off, Q, strike rows, t base
        for s_ in (0, 1):
            # the slip's rows of every block, in block order: q in [0, ks3) or [ks3, Q)
            lo = np.zeros(len(bl), np.int64) if s_ == 0 else bl[:, 2]
            cnt = (bl[:, 2] if s_ == 0 else bl[:, 1]) - lo
            nrows = int(cnt.sum())
            if nrows == 0:
                continue
            blk = np.repeat(np.arange(len(bl)), cnt)
            q = np.arange(nrows) - np.repeat(np.cumsum(cnt) - cnt, cnt) + lo[blk]
            off, Q, tp = bl[blk, 0], bl[blk, 1], bl[blk, 3]
            for ch in range(nch):
                g0, g1 = ch * v_chunk, min(ngv, (ch + 1) * v_chunk)
                for r in range(0, nrows, VMIX_ROWS):
                    items.append((nrec + r, min(VMIX_ROWS, nrows - r), g0, g1, col0 - lead, s_ | (c << 8), 0))
                # row records of this chunk's items, consecutive in item order
                recs.append(np.stack([off + q * cw, Q * cw, tp + ch * Q + q], axis=1))
                nrec += nrows
    import heapq
    cost = [((nr + 7) // 8) * (g1 - g0) + 16 for _, nr, g0, g1, _, _, _ in items]
    order = sorted(range(len(items)), key=lambda i: -cost[i])
    nwarps = max(8, min(int(nwarps), max(len(items), 1)) // 8 * 8)
    heap = [(0, w) for w in range(nwarps)]
    lists = [[] for _ in range(nwarps)]
    for i in order:
        load, w = heapq.heappop(heap)
        lists[w].append(i)
        heapq.heappush(heap, (load + cost[i], w))
    vwarp = np.zeros(nwarps + 1, dtype=np.int32)
    vwarp[1:] = np.cumsum([len(l) for l in lists])
    items = [items[i] for l in lists for i in l]
    rec = np.zeros(max(nrec, 1), dtype=_lib.V_ROW)
    if recs:
        a = np.concatenate(recs)
        rec["base"], rec["stride"], rec["out"] = a[:, 0], a[:, 1], a[:, 2]
    return items, vwarp, rec


def _balance(tasks, nbytes, ncta):
    """Tasks grouped by CTA (largest first to the least loaded CTA): (records sorted by
    CTA, per-CTA ranges of ncta' + 1 entries, ncta' = CTAs with work)."""
    import heapq
    if not tasks:
        return np.zeros(1, dtype=_lib.STREAM_TASK), np.zeros(1, np.int32), 0
    ncta = max(1, min(int(ncta), len(tasks)))
    heap = [(0, c) for c in range(ncta)]
    owner = np.empty(len(tasks), np.int64)
    for i in np.argsort(-np.asarray(nbytes, np.int64), kind="stable"):
        load, c = heapq.heappop(heap)
        owner[i] = c
        heapq.heappush(heap, (load + int(nbytes[i]), c))
    order = np.argsort(owner, kind="stable")
    rec = np.array([tasks[i] for i in order], dtype=_lib.STREAM_TASK)
    ptr = np.zeros(ncta + 1, np.int32)
    np.add.at(ptr, owner + 1, 1)
    return rec, np.cumsum(ptr).astype(np.int32), ncta


def _task(kind, **kw):
    t = dict(off=0, off1=0, off2=0, kind=kind, cls=0, m=0, r0=0, r1=0, g0=0, g1=0, c0=0, out=0, kS3=0, K0=0, K1=0,
             K2=0, tb=0)
    t.update(kw)
    return tuple(t[k] for k in _lib.STREAM_TASK.names)


def _build_stream_mixed(struct, dense_recs, cls_lists, ncta):
    """Task lists of the streamed mixed storage (build_plan_arrays_mixed, stream=True)."""
    DCOLS, VCOLS = 1024, 1024                  # columns of a dense / V task (x slice in shared memory)
    n = struct.n
    ta, ba, tb_, bb, gather = [], [], [], [], []
    slot_rows, slot = [], 0
    # dense tasks: (block, column chunk) owns m slots; row ranges share them
    for i in range(len(dense_recs)):
        m, nn, r0b, c0 = (int(dense_recs[k][i]) for k in ("m", "n", "r0", "c0"))
        lead = c0 % 4
        ng = _cdiv(nn + lead, 4)
        gch = DCOLS // 4
        for g0 in range(0, ng, gch):
            g1 = min(ng, g0 + gch)
            for r0 in range(0, m, _lib.STREAM_DENSE_ROWS):
                r1 = min(m, r0 + _lib.STREAM_DENSE_ROWS)
                ta.append(_task(0, off=int(dense_recs["off32"][i]), m=m, r0=r0, r1=r1, g0=g0, g1=g1, c0=c0 - lead,
                                out=slot))
                ba.append((g1 - g0) * (6 * (r1 - r0) * 16 + 32))
            slot_rows.append((slot, r0b, m))
            slot += m
    aca_blocks = [b for b in struct.blocks if b.aca]
    u_off, v_off = [0, 0, 0], [0, 0, 0]
    tp = sb = tb = 0
    pack = []
    lr_bytes = 0
    counts = np.zeros((3, 2), np.int64)
    for bi, b in enumerate(aca_blocks):
        m, nn = len(b.row.indices), len(b.col.indices)
        lo, hi = getattr(b, "rows", (0, m))
        cS, cD = cls_lists[bi]
        ks = np.bincount(cS, minlength=3).tolist()
        kd = np.bincount(cD, minlength=3).tolist()
        if sum(ks) + sum(kd) == 0:
            continue
        Ks = [_cdiv(ks[c] + kd[c], MIXED_CW[c]) * MIXED_CW[c] for c in range(3)]
        Qs = [3 * (ks[c] + kd[c]) for c in range(3)]
        if 3 * sum(Ks) > _lib.STREAM_BUF:
            raise _lib.Pq3dError("a block's t (%d values) exceeds the stream buffer" % (3 * sum(Ks)))
        rec_off, rec_voff, rec_tp, rec_nch, rec_sb = [0] * 3, [0] * 3, [0] * 3, [0] * 3, [0] * 3
        for c in range(3):
            counts[c] += (ks[c], kd[c])
            cw = MIXED_CW[c]
            lr_bytes += Qs[c] * ((hi - lo) + nn) * MIXED_BYTES[c] + (Qs[c] * 4 if c else 0)
            rec_off[c], rec_voff[c] = u_off[c], v_off[c]
            if Ks[c] == 0:
                continue
            if Qs[c] * 16 > _lib.STREAM_STAGE_BYTES:
                raise _lib.Pq3dError("a block's term class has %d V rows, more than one stream stage holds" % Qs[c])
            lead = b.col.start % cw
            ngv = _cdiv(nn + lead, cw)
            gch = VCOLS // cw
            nch = _cdiv(ngv, gch)
            for ch in range(nch):
                g0, g1 = ch * gch, min(ngv, (ch + 1) * gch)
                ta.append(_task(1, off=v_off[c], cls=c, m=Qs[c], g0=g0, g1=g1, c0=b.col.start - lead,
                                out=tp + ch * Qs[c], kS3=3 * ks[c]))
                ba.append((g1 - g0) * (Qs[c] * 16 + 8 * cw))
            rec_tp[c], rec_nch[c] = tp, nch
            tp += nch * Qs[c]
            if c:
                rec_sb[c] = sb
                sb += Qs[c]
            u_off[c] += Ks[c] * m * 3
            v_off[c] += Qs[c] * ngv * cw
        gather.append((Ks, ks, kd, Qs, rec_tp, rec_nch, rec_sb, tb, 0))
        for r0 in range(lo, hi, _lib.STREAM_ROWS):
            r1 = min(hi, r0 + _lib.STREAM_ROWS)
            tb_.append(_task(2, off=rec_off[0], off1=rec_off[1], off2=rec_off[2], m=m, r0=r0, r1=r1, out=slot - lo,
                             K0=Ks[0], K1=Ks[1], K2=Ks[2], tb=tb))
            bb.append(3 * (r1 - r0) * 16 * (Ks[0] // 4 + Ks[1] // 8 + Ks[2] // 16) + 12 * sum(Ks))
        tb += 3 * sum(Ks)
        slot_rows.append((slot, b.row.start + lo, hi - lo))
        for p in (0, 1):
            pack.append((bi, p, rec_off, rec_voff, ks, kd, Qs, Ks, rec_sb))
        slot += hi - lo
    A = _leaf_lists(struct, slot_rows)
    tasks_a, cta_a, ncta_a = _balance(ta, ba, ncta)
    tasks_b, cta_b, ncta_b = _balance(tb_, bb, ncta)
    dense_entries = int(np.sum(dense_recs["m"].astype(np.int64) * dense_recs["n"])) if len(dense_recs) else 0
    A.update(ditems=_rec([], _lib.DENSE_ITEM), vitems=_rec([], _lib.V_ITEM), utasks=_rec([], _lib.U_TASK_M),
             n_ditems=0, n_vitems=0, n_utasks=0, n_slots=slot, n_tpart=tp, n_scales=sb, kmax=0, u_sizes=u_off,
             v_sizes=v_off, pack=pack, stream=True, class_terms=counts,
             tasks_a=tasks_a, cta_a=cta_a, ncta_a=ncta_a, tasks_b=tasks_b, cta_b=cta_b, ncta_b=ncta_b,
             gather=_rec(gather, _lib.T_GATHER), n_gather=len(gather), n_tfull=tb,
             alg_bytes=dense_entries * 6 * 4 + lr_bytes + 2 * n * 4 + 3 * n * 8)
    return A


def _rec(rows, dt):
    return np.array(rows, dtype=dt) if rows else np.zeros(1, dtype=dt)


# ----------------------------------------------------------------------------- plan cache

PLAN_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "plan_cache.json")
_plan_cache = None


def _entry_n(e):
    """Element count of the workload a cache entry was tuned on."""
    if "n" in e:
        return int(e["n"])
    import re
    m = re.search(r"\((\d+) triangles\)", e.get("workload", ""))
    return int(m.group(1)) if m else None


def plan_cache_entry(gpu_name, dtype, n=None):
    """Work-item shapes measured by pyquake3d_b200.autotune for this GPU model and
    storage, or None.  The cache may hold entries tuned on workloads of several
    sizes (a list); the one tuned on the size closest to n (log scale) is used."""
    global _plan_cache
    if _plan_cache is None:
        _plan_cache = {}
        if os.path.exists(PLAN_CACHE):
            import json
            with open(PLAN_CACHE) as f:
                _plan_cache = json.load(f)
    ent = _plan_cache.get(gpu_name, {}).get(dtype)
    if ent is None or isinstance(ent, dict):
        return ent
    sized = [e for e in ent if _entry_n(e)]
    if n is None or not sized:
        return ent[0] if ent else None
    return min(sized, key=lambda e: abs(np.log(_entry_n(e) / float(n))))


# ----------------------------------------------------------------------------- device operator

DTYPES = {"fp64": 0, "fp32": 1, "bf16": 2, "mixed": 3}
# default term-class tolerance of the mixed storage: a quantised term may move a row
# by at most 2^-22 of its near-field absolute row sum (4 ulps of FP32 storage)
MIXED_TOL = 2.0 ** -22
_CW_DENSE = {0: 2, 1: 4, 2: 4, 3: 4}
_CW_LR = {0: 2, 1: 4, 2: 8}


def _cdiv(a, b):
    return (a + b - 1) // b


class DeviceHMatrix:
    """The packed operator on one GPU.

    assemble() computes dense blocks and ACA factors in FP64 on the device;
    plan(dtype) packs them into the matvec layout of one storage precision
    ("fp64": FP64 everywhere; "fp32": FP32 everywhere; "bf16": FP32 dense,
    BF16 low rank).  matvec(x_dev, dtype) returns y (n x 3, FP64, tree order)."""

    # work-item shapes per storage code (0 FP64, 1 FP32, 2 BF16 low rank, 3 mixed): these
    # defaults unless the plan cache written by pyquake3d_b200.autotune has an entry for
    # this GPU and storage (shapes()).
    DENSE_CHUNK_GROUPS = {0: 64, 1: 16, 2: 16, 3: 16}   # column groups per dense work item
    V_CHUNK_GROUPS = {0: 128, 1: 32, 2: 32, 3: 32}      # column groups per V work item
    U_ROWS = 512                                        # rows per U task (one CTA)

    def __init__(self, struct, xg, ev, nodes, tri, mu, lam, device="cuda", aca_tol=0.01, aca_rel=False,
                 aca_seed=0, kcap=96, ws_budget_bytes=8 << 30, keep_factors=False, halfspace=0,
                 mixed_tol=MIXED_TOL):
        """halfspace: 0 full space; 1 half space, a triangle side along z adds no
        free-surface term; 2 half space with the side handling of the reference's
        compiled library (the values its H-matrix assembly uses).  mixed_tol: the
        term-class tolerance of the "mixed" storage (classify_terms)."""
        self.mixed_tol = float(mixed_tol)
        self.mixed_stream = False      # mixed storage: True selects the bulk-copy (streamed) kernels
        self.use_plan_cache = True
        import torch
        self.torch = torch
        self.L = _lib.load()
        self.s = struct
        self.n = struct.n
        self.mu, self.lam = float(mu), float(lam)
        self.dev = torch.device(device)
        self.aca_tol, self.aca_rel, self.aca_seed = float(aca_tol), bool(aca_rel), int(aca_seed)
        self.kcap = int(kcap)
        self.keep_factors = bool(keep_factors)
        self.ws_budget = int(ws_budget_bytes)
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.xg = torch.tensor(np.ascontiguousarray(xg), **f64)
        self.ev = torch.tensor(np.ascontiguousarray(ev), **f64)
        self.nodes = torch.tensor(np.ascontiguousarray(nodes), **f64)
        self.tri = torch.tensor(np.ascontiguousarray(tri, dtype=np.int64), dtype=torch.int64, device=self.dev)
        self.perm = torch.tensor(struct.perm.astype(np.int32), dtype=torch.int32, device=self.dev)
        self.iperm = torch.tensor(struct.iperm.astype(np.int32), dtype=torch.int32, device=self.dev)
        rb = self.L.pq3d_src_record_bytes()
        self.rec = torch.empty((self.n * rb + 7) // 8, **f64)
        self._stream = _lib.stream_ptr()
        check(self.L.pq3d_src_records(ptr(self.nodes), ptr(self.tri), self.n, ptr(self.rec), self._stream),
              "pq3d_src_records")
        self.halfspace = int(halfspace)
        self.hs = None
        if self.halfspace:
            hb = self.L.pq3d_hs_record_bytes()
            self.hs = torch.empty((self.n * hb + 7) // 8, **f64)
            check(self.L.pq3d_hs_records(ptr(self.nodes), ptr(self.tri), self.n, ptr(self.hs), self._stream),
                  "pq3d_hs_records")
        self.dense_blocks = [b for b in struct.blocks if not b.aca]
        self.aca_blocks = [b for b in struct.blocks if b.aca]
        self.plans = {}
        self.assembled = False
        self.timings = {}

    # ------------------------------------------------------------------ assembly
    def assemble(self, want=("fp64", "bf16")):
        """Dense near field + ACA factors (FP64 on device), then pack for each dtype."""
        import time
        torch = self.torch
        want = tuple(want)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self._assemble_dense(want)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        self._run_aca()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        self.timings.update(dense_s=t1 - t0, aca_s=t2 - t1)
        for d in want:
            self.plan(d)
        torch.cuda.synchronize()
        self.timings["pack_s"] = time.perf_counter() - t2
        self.assembled = True
        if not self.keep_factors:
            # packed copies are all that the matvec needs: release the FP64 ACA workspaces
            self.aca_ws = [(None, keep) for _, keep in self.aca_ws]
            torch.cuda.empty_cache()
        return self

    def _assemble_dense(self, want):
        torch = self.torch
        need64 = "fp64" in want
        need32 = any(d in want for d in ("fp32", "bf16", "mixed"))
        recs, off64, off32 = dense_layout(self.dense_blocks)
        order = np.argsort(-(recs["m"].astype(np.int64) * recs["n"]), kind="stable")
        self.dense_recs = recs
        self.dense64 = torch.zeros(max(off64, 1), dtype=torch.float64, device=self.dev) if need64 else None
        self.dense32 = torch.zeros(max(off32, 1), dtype=torch.float32, device=self.dev) if need32 else None
        if len(recs):
            d_recs = torch.from_numpy(recs[order].view(np.uint8)).to(self.dev)
            check(self.L.pq3d_dense_assemble(ptr(self.xg), ptr(self.ev), ptr(self.rec), ptr(self.perm), ptr(d_recs),
                                             len(recs), self.mu, self.lam, ptr(self.dense64), ptr(self.dense32),
                                             ptr(self.hs), self.halfspace, self._stream), "pq3d_dense_assemble")
            torch.cuda.synchronize()

    def _run_aca(self):
        """Batched ACA over all admissible blocks; ranks and FP64 factors kept per task."""
        torch = self.torch
        starts = getattr(self.s, "aca_starts", None)
        if starts is None:
            starts = aca_start_indices(self.s.blocks, self.aca_seed)
        rowlist, collist = [], []
        tasks = []
        roff = 0
        for bi, b in enumerate(self.aca_blocks):
            m, n = len(b.row.indices), len(b.col.indices)
            rowlist.append(b.row.indices)
            collist.append(b.col.indices)
            for p in (0, 1):
                tasks.append(dict(block=bi, pass_=p, m=m, n=n, rows_off=roff, cols_off=roff,
                                  iref0=starts[bi][p][0], jref0=starts[bi][p][1]))
            roff += 0  # offsets assigned below
        # row and col lists stored separately
        rl = np.concatenate(rowlist).astype(np.int32) if rowlist else np.zeros(1, np.int32)
        cl = np.concatenate(collist).astype(np.int32) if collist else np.zeros(1, np.int32)
        ro = np.concatenate([[0], np.cumsum([len(r) for r in rowlist])]).astype(np.int64) if rowlist else np.zeros(1, np.int64)
        co = np.concatenate([[0], np.cumsum([len(c) for c in collist])]).astype(np.int64) if collist else np.zeros(1, np.int64)
        for t in tasks:
            t["rows_off"] = int(ro[t["block"]])
            t["cols_off"] = int(co[t["block"]])
        self.rowlist = torch.tensor(rl, dtype=torch.int32, device=self.dev)
        self.collist = torch.tensor(cl, dtype=torch.int32, device=self.dev)
        self.aca_tasks = tasks
        self.aca_ranks = np.zeros(len(tasks), dtype=np.int32)
        self.aca_flags = np.zeros(len(tasks), dtype=np.int32)
        self.aca_ws = []  # (tensor, {task index: ws_off, kmax})
        pending = list(range(len(tasks)))
        kcap = self.kcap
        while pending:
            # batches bounded by the workspace budget, largest tasks first
            pending.sort(key=lambda i: -(tasks[i]["m"] + tasks[i]["n"]))
            retry = []
            i0 = 0
            while i0 < len(pending):
                batch, ws_off = [], 0
                while i0 < len(pending):
                    t = tasks[pending[i0]]
                    kmax = min(t["m"], t["n"], t.get("kcap", kcap))
                    need = self.L.pq3d_aca_ws_doubles(t["m"], t["n"], kmax)
                    if batch and (ws_off + need) * 8 > self.ws_budget:
                        break
                    batch.append((pending[i0], ws_off, kmax))
                    ws_off += need
                    i0 += 1
                rec = np.zeros(len(batch), dtype=_lib.ACA_TASK)
                max_mn = 0
                for j, (ti, wo, kmax) in enumerate(batch):
                    t = tasks[ti]
                    rec[j] = (t["rows_off"], t["cols_off"], wo, t["m"], t["n"], kmax, t["pass_"], t["iref0"], t["jref0"])
                    max_mn = max(max_mn, t["m"], t["n"])
                ws = torch.empty(max(ws_off, 1), dtype=torch.float64, device=self.dev)
                d_rec = torch.from_numpy(rec.view(np.uint8)).to(self.dev)
                d_rank = torch.zeros(len(batch), dtype=torch.int32, device=self.dev)
                d_flag = torch.zeros(len(batch), dtype=torch.int32, device=self.dev)
                check(self.L.pq3d_aca_batched(ptr(self.xg), ptr(self.ev), ptr(self.rec), ptr(self.rowlist),
                                              ptr(self.collist), ptr(d_rec), len(batch), ptr(ws), self.mu, self.lam,
                                              self.aca_tol, 1 if self.aca_rel else 0, max_mn, ptr(d_rank),
                                              ptr(d_flag), ptr(self.hs), self.halfspace, self._stream),
                      "pq3d_aca_batched")
                ranks = d_rank.cpu().numpy()
                flags = d_flag.cpu().numpy()
                if (flags & 8).any():
                    raise _lib.Pq3dError("pq3d_aca_batched: a task has more rows or columns than the batch's "
                                         "max_mn (not run)")
                # flag 4 (every remaining pivot candidate excluded) ends a task normally: the
                # factors found so far are the block's approximation, as in the reference loop
                keep = {}
                for j, (ti, wo, kmax) in enumerate(batch):
                    if flags[j] & 1 and kmax < min(tasks[ti]["m"], tasks[ti]["n"]):
                        tasks[ti]["kcap"] = min(2 * kmax, min(tasks[ti]["m"], tasks[ti]["n"]))
                        retry.append(ti)
                        continue
                    self.aca_ranks[ti] = ranks[j]
                    self.aca_flags[ti] = flags[j]
                    keep[ti] = (wo, kmax)
                self.aca_ws.append((ws, keep))
            pending = retry
        self.task_ws = {}
        for wi, (ws, keep) in enumerate(self.aca_ws):
            for ti, (wo, kmax) in keep.items():
                self.task_ws[ti] = (wi, wo, kmax)

    def ranks(self):
        """(kS, kD) per ACA block."""
        r = self.aca_ranks.reshape(-1, 2)
        return r[:, 0], r[:, 1]

    # ------------------------------------------------------------------ packing / plans
    def plan(self, dtype):
        if dtype in self.plans:
            return self.plans[dtype]
        if self.assembled and not self.keep_factors and self.aca_blocks:
            raise _lib.Pq3dError("ACA factors were released after assembly; request every precision in "
                                 "assemble(want=...) or construct with keep_factors=True")
        torch = self.torch
        code = DTYPES[dtype]
        if code == 3:
            return self._plan_mixed()
        A = self.plan_arrays(dtype)
        lr_dtype = torch.float64 if code == 0 else (torch.float32 if code == 1 else torch.bfloat16)
        Ubuf = torch.zeros(max(A["u_size"], 8), dtype=lr_dtype, device=self.dev)
        Vbuf = torch.zeros(max(A["v_size"], 8), dtype=lr_dtype, device=self.dev)
        # pack every ACA task into the layout, one launch per workspace batch
        ro_np = self._row_offsets()
        by_ws = {}
        for (bi, p, u_off, v_off, K, Q, ks, kd) in A["pack"]:
            ti = 2 * bi + p
            wi, wo, kmax = self.task_ws[ti]
            b = self.aca_blocks[bi]
            by_ws.setdefault(wi, []).append((wo, u_off, v_off, ro_np[bi][0], ro_np[bi][1], len(b.row.indices),
                                             len(b.col.indices), kmax, ks if p == 0 else kd, p, ks, kd, K, Q,
                                             b.row.start, b.col.start, 1 if self.aca_flags[ti] & 2 else 0))
        for wi, rows in by_ws.items():
            rec = np.array(rows, dtype=_lib.PACK_TASK)
            d_rec = torch.from_numpy(rec.view(np.uint8)).to(self.dev)
            check(self.L.pq3d_aca_pack(ptr(d_rec), len(rows), ptr(self.aca_ws[wi][0]), ptr(self.rowlist),
                                       ptr(self.collist), ptr(self.iperm), code, ptr(Ubuf), ptr(Vbuf), self._stream),
                  "pq3d_aca_pack")
        return self._finish_plan(dtype, A, Ubuf, Vbuf)

    def shapes(self, dtype):
        """(dense_chunk, v_chunk, u_rows) of a storage: an explicit override
        (set_shapes), else the plan cache's entry for this GPU, else the defaults."""
        code = DTYPES[dtype]
        ov = getattr(self, "_shape_override", {}).get(dtype)
        if ov is not None:
            return ov
        if self.use_plan_cache:
            ent = plan_cache_entry(self.torch.cuda.get_device_name(self.dev), dtype, self.n)
            if ent is not None:
                return int(ent["dense_chunk"]), int(ent["v_chunk"]), int(ent["u_rows"])
        return self.DENSE_CHUNK_GROUPS[code], self.V_CHUNK_GROUPS[code], self.U_ROWS

    def set_shapes(self, dtype, dense_chunk, v_chunk, u_rows):
        """Rebuild one storage's work items with other shapes; the packed operator data
        does not depend on them and is kept (the autotuner's move)."""
        if not hasattr(self, "_shape_override"):
            self._shape_override = {}
        self._shape_override[dtype] = (int(dense_chunk), int(v_chunk), int(u_rows))
        P = self.plans.get(dtype)
        if P is None:
            return None
        if DTYPES[dtype] == 3:
            offs = np.concatenate([[0], np.cumsum(np.asarray(self.aca_ranks, np.int64))])
            t = self.mixed_tmap
            cls_lists = [(t[offs[2 * bi]:offs[2 * bi + 1]] & 3, t[offs[2 * bi + 1]:offs[2 * bi + 2]] & 3)
                         for bi in range(len(self.aca_blocks))]
            A = self._mixed_arrays(cls_lists)
            A["mixed"] = P["mixed"]
        else:
            A = self.plan_arrays(dtype)
        del self.plans[dtype]
        return self._finish_plan(dtype, A, P["U"], P["V"])

    def plan_arrays(self, dtype):
        """Host work-item arrays of one storage precision (deterministic from the
        structure and the ACA ranks)."""
        code = DTYPES[dtype]
        kS, kD = self.ranks()
        dc, vc, ur = self.shapes(dtype)
        return build_plan_arrays(self.s, self.dense_recs, kS, kD, code, dc, vc, ur)

    def _task_records_mixed(self, keep_ws):
        """PackTaskM records (per workspace batch) for every ACA task, with the weight /
        term-map offset of each task (tasks in block order, strike pass first)."""
        ro_np = self._row_offsets()
        recs, tmap_off = {}, 0
        offs = np.zeros(len(self.aca_tasks) + 1, np.int64)
        for ti in range(len(self.aca_tasks)):
            bi, p = divmod(ti, 2)
            k = int(self.aca_ranks[ti])
            offs[ti] = tmap_off
            wi, wo, kmax = self.task_ws[ti]
            b = self.aca_blocks[bi]
            r = np.zeros(1, dtype=_lib.PACK_TASK_M)
            r["ws_off"], r["rows_off"], r["cols_off"], r["tmap_off"] = wo, ro_np[bi][0], ro_np[bi][1], tmap_off
            r["m"], r["n"], r["kmax"], r["k"], r["pass_"] = len(b.row.indices), len(b.col.indices), kmax, k, p
            r["r0"], r["c0"], r["zeroB"] = b.row.start, b.col.start, 1 if self.aca_flags[ti] & 2 else 0
            recs.setdefault(wi, []).append((ti, r))
            tmap_off += k
        offs[-1] = tmap_off
        return recs, offs

    def _plan_mixed(self):
        """Mixed storage (code 3): FP32 dense near field; ACA terms in FP32 / FP16 / INT8
        classes chosen from their weights against the near-field row sums."""
        torch = self.torch
        if self.dense32 is None:
            raise _lib.Pq3dError("the mixed plan needs the FP32 dense blocks: request it in assemble(want=...)")
        n = self.n
        L = self.L
        st = self._stream
        # near-field absolute row sums (tree order), largest component
        R3 = torch.zeros(3 * n, dtype=torch.float64, device=self.dev)
        recs = self.dense_recs
        if len(recs):
            d_recs = torch.from_numpy(np.ascontiguousarray(recs).view(np.uint8)).to(self.dev)
            check(L.pq3d_nearfield_rowabs(ptr(self.dense32), ptr(d_recs), len(recs), n, ptr(R3), st),
                  "pq3d_nearfield_rowabs")
        R = R3.view(3, n).max(dim=0).values.contiguous()
        by_ws, offs = self._task_records_mixed(None)
        w = torch.zeros(max(int(offs[-1]), 1), dtype=torch.float64, device=self.dev)
        for wi, rows in by_ws.items():
            rec = np.concatenate([r for _, r in rows])
            d_rec = torch.from_numpy(rec.view(np.uint8)).to(self.dev)
            check(L.pq3d_aca_term_weights(ptr(d_rec), len(rec), ptr(self.aca_ws[wi][0]), ptr(self.rowlist),
                                          ptr(self.iperm), ptr(R), ptr(w), st), "pq3d_aca_term_weights")
        w = w.cpu().numpy()
        # classes per block, then each term's position within its class (per pass)
        tmap = np.zeros(max(int(offs[-1]), 1), np.int32)
        cls_lists = []
        for bi in range(len(self.aca_blocks)):
            tS, tD = 2 * bi, 2 * bi + 1
            cS, cD = classify_terms(w[offs[tS]:offs[tS + 1]], w[offs[tD]:offs[tD + 1]], self.mixed_tol)
            cls_lists.append((cS, cD))
            for ti, cc in ((tS, cS), (tD, cD)):
                pos = np.zeros(len(cc), np.int32)
                for c in range(3):
                    sel = np.nonzero(cc == c)[0]
                    pos[sel] = np.arange(len(sel))
                tmap[offs[ti]:offs[ti + 1]] = cc | (pos << 2)
        self.mixed_tmap = tmap[:int(offs[-1])]
        A = self._mixed_arrays(cls_lists)
        # INT8-class entries are stored as b + 128: the fill 128 decodes to zero, so padding
        # columns (a block's lead and tail columns, its K padding) contribute nothing
        tdt, fill = (torch.float32, torch.float16, torch.uint8), (0, 0, 128)
        Ub = [torch.full((max(int(A["u_sizes"][c]), 16),), fill[c], dtype=tdt[c], device=self.dev) for c in range(3)]
        Vb = [torch.full((max(int(A["v_sizes"][c]), 16),), fill[c], dtype=tdt[c], device=self.dev) for c in range(3)]
        scales = torch.zeros(max(A["n_scales"], 4), dtype=torch.float32, device=self.dev)
        d_tmap = torch.from_numpy(tmap).to(self.dev)
        layout = {}
        for (bi, p, uo, vo, ks, kd, Q, K, sb) in A["pack"]:
            layout[2 * bi + p] = (uo, vo, ks, kd, Q, K, sb)
        for wi, rows in by_ws.items():
            recl = []
            for ti, r in rows:
                if ti not in layout:
                    continue                       # a block without terms
                uo, vo, ks, kd, Q, K, sb = layout[ti]
                r = r.copy()
                r["u_off"], r["v_off"], r["kS"], r["kD"], r["Q"], r["K"], r["sb"] = uo, vo, ks, kd, Q, K, sb
                recl.append(r)
            if not recl:
                continue
            rec = np.concatenate(recl)
            d_rec = torch.from_numpy(rec.view(np.uint8)).to(self.dev)
            check(L.pq3d_aca_pack_mixed(ptr(d_rec), len(rec), ptr(self.aca_ws[wi][0]), ptr(self.rowlist),
                                        ptr(self.collist), ptr(self.iperm), ptr(d_tmap), ptr(Ub[0]), ptr(Ub[1]),
                                        ptr(Ub[2]), ptr(Vb[0]), ptr(Vb[1]), ptr(Vb[2]), ptr(scales), st),
                  "pq3d_aca_pack_mixed")
        A["mixed"] = dict(U=Ub, V=Vb, scales=scales, tol=self.mixed_tol, class_terms=A["class_terms"].tolist())
        return self._finish_plan("mixed", A, Ub[0], Vb[0])

    def _mixed_arrays(self, cls_lists):
        dc, vc, ur = self.shapes("mixed")
        if self.mixed_stream:
            ncta = self.L.pq3d_stream_ctas()
            if ncta > 0:
                try:
                    return build_plan_arrays_mixed(self.s, self.dense_recs, cls_lists, dc, vc, ur, stream=True,
                                                   ncta=ncta)
                except _lib.Pq3dError:
                    pass               # a term class too large for a stream stage: the plain kernels
        nw = self.L.pq3d_vmix_ctas()
        return build_plan_arrays_mixed(self.s, self.dense_recs, cls_lists, dc, vc, ur,
                                       nwarps=8 * nw if nw > 0 else VMIX_WARPS)

    def install_mixed(self, tmap, U, V, scales):
        """Register a mixed plan whose class arrays come from elsewhere (an operator
        checkpoint): tmap holds every term's class code (bits 0-1) in task order."""
        offs = np.concatenate([[0], np.cumsum(np.asarray(self.aca_ranks, np.int64))])
        cls_lists = [(tmap[offs[2 * bi]:offs[2 * bi + 1]] & 3, tmap[offs[2 * bi + 1]:offs[2 * bi + 2]] & 3)
                     for bi in range(len(self.aca_blocks))]
        self.mixed_tmap = np.asarray(tmap, np.int32)
        A = self._mixed_arrays(cls_lists)
        A["mixed"] = dict(U=list(U), V=list(V), scales=scales, tol=self.mixed_tol,
                          class_terms=A["class_terms"].tolist())
        return self._finish_plan("mixed", A, U[0], V[0])

    def install_plan(self, dtype, Ubuf, Vbuf):
        """Register a plan whose packed low-rank buffers were produced elsewhere (an
        operator checkpoint); dense blocks must already be in dense64/dense32."""
        return self._finish_plan(dtype, self.plan_arrays(dtype), Ubuf, Vbuf)

    def _finish_plan(self, dtype, A, Ubuf, Vbuf):
        torch = self.torch
        code = DTYPES[dtype]

        def dev_rec(a):
            return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).to(self.dev)

        acc = torch.float64 if code == 0 else torch.float32
        dense = self.dense64 if code == 0 else self.dense32
        if A["n_ditems"] > 0 and dense is None:
            raise _lib.Pq3dError(f"dense blocks of the {dtype} plan were not assembled")
        P = dict(code=code, dtype=dtype, acc=acc,
                 dense=self.dense64 if code == 0 else self.dense32, U=Ubuf, V=Vbuf,
                 ditems=dev_rec(A["ditems"]), vitems=dev_rec(A["vitems"]), utasks=dev_rec(A["utasks"]),
                 leaf_of_row=torch.tensor(A["leaf_of_row"], device=self.dev),
                 leaf_ptr=torch.tensor(A["leaf_ptr"], device=self.dev),
                 leaf_off=torch.tensor(A["leaf_off"], device=self.dev),
                 n_ditems=A["n_ditems"], n_vitems=A["n_vitems"], n_utasks=A["n_utasks"],
                 n_slots=A["n_slots"], n_tpart=A["n_tpart"], kmax=A["kmax"])
        P["slots"] = torch.empty(3 * max(P["n_slots"], 1), dtype=acc, device=self.dev)
        P["tpart"] = torch.empty(max(P["n_tpart"], 1), dtype=acc, device=self.dev)
        hp = np.zeros(1, dtype=_lib.HM_PLAN)
        hp["n"] = self.n
        hp["dtype"] = code
        for k in ("dense", "U", "V", "ditems", "vitems", "utasks", "leaf_of_row", "leaf_ptr", "leaf_off"):
            hp[k] = P[k].data_ptr() if P[k] is not None else 0
        for k in ("n_ditems", "n_vitems", "n_utasks", "n_slots", "n_tpart", "kmax"):
            hp[k] = P[k]
        if code == 3:
            M = A["mixed"]
            P["mixed"] = M
            hp["U16"], hp["U8"] = M["U"][1].data_ptr(), M["U"][2].data_ptr()
            hp["V16"], hp["V8"] = M["V"][1].data_ptr(), M["V"][2].data_ptr()
            hp["scales"] = M["scales"].data_ptr()
            P["status"] = torch.zeros(1, dtype=torch.int32, device=self.dev)
            hp["status"] = P["status"].data_ptr()
            hp["stream"] = 1 if A.get("stream") else 0
            P["stream"] = bool(A.get("stream"))
            if not P["stream"]:
                P["vrows"] = dev_rec(A["vrows"])
                hp["vrows"] = P["vrows"].data_ptr()
                P["vwarp"] = torch.tensor(A["vwarp"], dtype=torch.int32, device=self.dev)
                hp["vwarp"], hp["n_vwarp"] = P["vwarp"].data_ptr(), len(A["vwarp"]) - 1
            if P["stream"]:
                for k in ("tasks_a", "tasks_b", "gather"):
                    P[k] = dev_rec(A[k])
                    hp[k] = P[k].data_ptr()
                for k in ("cta_a", "cta_b"):
                    P[k] = torch.tensor(A[k], dtype=torch.int32, device=self.dev)
                    hp[k] = P[k].data_ptr()
                P["tfull"] = torch.zeros(max(A["n_tfull"], 4), dtype=torch.float32, device=self.dev)
                hp["tfull"] = P["tfull"].data_ptr()
                hp["n_gather"], hp["ncta_a"], hp["ncta_b"] = A["n_gather"], A["ncta_a"], A["ncta_b"]
        P["host_plan"] = hp
        P["alg_bytes"] = A["alg_bytes"]
        P["stored_bytes"] = (P["dense"].numel() * P["dense"].element_size() if P["dense"] is not None else 0) + \
            Ubuf.numel() * Ubuf.element_size() + Vbuf.numel() * Vbuf.element_size()
        if code == 3:
            P["stored_bytes"] += sum(t.numel() * t.element_size() for t in P["mixed"]["U"][1:] + P["mixed"]["V"][1:])
        self.plans[dtype] = P
        return P

    def _row_offsets(self):
        if not hasattr(self, "_ro_cache"):
            ro, co = 0, 0
            res = []
            for b in self.aca_blocks:
                res.append((ro, co))
                ro += len(b.row.indices)
                co += len(b.col.indices)
            self._ro_cache = res
        return self._ro_cache

    def kernel_status(self, dtype):
        """Status word of a plan's streamed kernels: 0, 1 after a timed-out wait, 2 after a
        task of a size they do not take (nothing of the kind is expected)."""
        P = self.plans.get(dtype)
        return int(P["status"].item()) if P is not None and "status" in P else 0

    def new_x(self, dtype):
        """Zero deficit buffer (tree order, device layout of pack_x) for the given plan."""
        P = self.plan(dtype)
        return self.torch.zeros(4 * x_stride(self.n), dtype=P["acc"], device=self.dev)

    def matvec(self, x, dtype, y=None, add=(None, None, None), stream=None, slots_only=False):
        """y[i, c] = sum_j K_c(i, j) x  (tree order, FP64 output).  slots_only: write the
        per-row partial sums only (the step kernel reduces them)."""
        P = self.plan(dtype)
        if y is None and not slots_only:
            y = self.torch.empty((self.n, 3), dtype=self.torch.float64, device=self.dev)
        P["slots_owner"] = None     # the slots now hold this call's products
        st = _lib.stream_ptr(stream)
        check(self.L.pq3d_hmatvec(P["host_plan"].ctypes.data, ptr(x), ptr(P["slots"]), ptr(P["tpart"]),
                                  ptr(add[0]), ptr(add[1]), ptr(add[2]), None if slots_only else ptr(y), st),
              "pq3d_hmatvec")
        return y

    def apply(self, x1, x2, dtype="fp64"):
        """Host convenience: (y1, y2, yB) in element order for deficits x1, x2 (element order)."""
        torch = self.torch
        P = self.plan(dtype)
        xt = pack_x(np.asarray(x1)[self.s.perm], np.asarray(x2)[self.s.perm], self.n)
        x = torch.tensor(xt, dtype=P["acc"], device=self.dev)
        y = self.matvec(x, dtype).cpu().numpy()
        out = np.empty_like(y)
        out[self.s.perm] = y
        return out[:, 0], out[:, 1], out[:, 2]


def export_blocks(op):
    """Host copy of the FP64 operator per block, in the reference's block format:
    list of ("dense", rows, cols, M[6][m][n]) or ("aca", rows, cols, S, D) with
    S/D dicts of U1 V1 U2 V2 UB VB (rows/cols are element ids in tree order).
    Used to run the reference's CPU step on the same operator."""
    P = op.plan("fp64")
    perm = op.s.perm
    dense = op.dense64.cpu().numpy() if op.dense64 is not None else None
    U = P["U"].cpu().numpy()
    V = P["V"].cpu().numpy()
    out = []
    recs = op.dense_recs
    for i in range(len(recs)):
        m, n, r0, c0 = (int(recs[k][i]) for k in ("m", "n", "r0", "c0"))
        lead = c0 % 2
        ng = _cdiv(n + lead, 2)
        a = dense[int(recs["off64"][i]):int(recs["off64"][i]) + ng * m * 12].reshape(ng, 3, 2, m, 2)
        # (group, comp, slip, row, t) -> (slip, comp, row, col)
        M = a.transpose(2, 1, 3, 0, 4).reshape(2, 3, m, ng * 2)[:, :, :, lead:lead + n].reshape(6, m, n)
        out.append(("dense", perm[r0:r0 + m], perm[c0:c0 + n], np.ascontiguousarray(M)))
    kS, kD = op.ranks()
    u_off = v_off = 0
    for bi, b in enumerate(op.aca_blocks):
        m, n = len(b.row.indices), len(b.col.indices)
        ks, kd = int(kS[bi]), int(kD[bi])
        rows = perm[b.row.start:b.row.start + m]
        cols = perm[b.col.start:b.col.start + n]
        if ks + kd == 0:
            z = dict(U1=np.zeros((m, 0)), V1=np.zeros((0, n)), U2=np.zeros((m, 0)), V2=np.zeros((0, n)), UB=[], VB=[])
            out.append(("aca", rows, cols, z, dict(z)))
            continue
        K = _cdiv(ks + kd, 2) * 2
        Q = 3 * (ks + kd)
        lead = b.col.start % 2
        ngv = _cdiv(n + lead, 2)
        Ub = U[u_off:u_off + K // 2 * m * 6].reshape(K // 2, 3, m, 2).transpose(1, 2, 0, 3).reshape(3, m, K)
        Vb = V[v_off:v_off + ngv * Q * 2].reshape(ngv, Q, 2).transpose(1, 0, 2).reshape(Q, ngv * 2)[:, lead:lead + n]
        S, D = {}, {}
        for c, (un, vn) in enumerate((("U1", "V1"), ("U2", "V2"), ("UB", "VB"))):
            S[un] = np.ascontiguousarray(Ub[c, :, :ks])
            S[vn] = np.ascontiguousarray(Vb[c * ks:(c + 1) * ks])
            D[un] = np.ascontiguousarray(Ub[c, :, ks:ks + kd])
            D[vn] = np.ascontiguousarray(Vb[3 * ks + c * kd:3 * ks + (c + 1) * kd])
        out.append(("aca", rows, cols, S, D))
        u_off += K // 2 * m * 6
        v_off += ngv * Q * 2
    return out

"""Mesh input: Gmsh 2.2 ASCII reader/writer and per-element frames.

read_mshV2 follows src/readmsh.py:12-68 (node coordinates in km are scaled
by 1e3; an element line is a triangle when it has at least 8 tokens, its
last three tokens are the 1-based node ids).  get_eleVec follows
src/readmsh.py:75-134 (unit normal from the node order, strike
e1 = (n_y, -n_x, 0)/|.| or (1, 0, 0) for a horizontal element, dip
e2 = n x e1; rows of eleVec are e1, e2, e3=n).
"""
import numpy as np


def read_mshV2(fname):
    nodes, eles = [], []
    in_nodes = in_eles = False
    k = 0
    with open(fname, "r") as f:
        for raw in f:
            line = raw[:-1] if raw.endswith("\n") else raw
            if in_nodes:
                k += 1
                if k > 1:
                    tok = line.split()
                    try:
                        nodes.append([float(tok[1]), float(tok[2]), float(tok[3])])
                    except (ValueError, IndexError):
                        in_nodes = False
                        k = 0
            if in_eles:
                k += 1
                if k > 1:
                    tok = line.split()
                    try:
                        if len(tok) >= 8:
                            eles.append([int(tok[-3]), int(tok[-2]), int(tok[-1])])
                    except ValueError:
                        in_eles = False
            if line == "$Nodes":
                in_nodes = True
            if line == "$Elements":
                in_eles = True
    return np.array(nodes) * 1e3, np.array(eles)


def write_msh(fname, nodes_km, tris):
    """Write a Gmsh 2.2 ASCII mesh: nodes in km, triangles (1-based) with 2 tags."""
    with open(fname, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(nodes_km))
        for i, p in enumerate(nodes_km):
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        f.write("$EndNodes\n$Elements\n%d\n" % len(tris))
        for i, t in enumerate(tris):
            f.write("%d 2 2 0 1 %d %d %d\n" % (i + 1, t[0], t[1], t[2]))
        f.write("$EndElements\n")


def get_eleVec(nodelst, elelst, jud_ele_order):
    """Element frames (N x 9: e1, e2, e3) and centroids (N x 3)."""
    xa = nodelst[elelst[:, 0] - 1]
    xb = nodelst[elelst[:, 1] - 1]
    xc = nodelst[elelst[:, 2] - 1]
    xg = np.empty((len(elelst), 3))
    for d in range(3):
        # np.mean of three scalars: ((a + b) + c) / 3
        xg[:, d] = (xa[:, d] + xb[:, d] + xc[:, d]) / 3.0
    vba = xb - xa
    vca = xc - xa
    if jud_ele_order:
        e3 = np.stack([vca[:, 1] * vba[:, 2] - vca[:, 2] * vba[:, 1],
                       vca[:, 2] * vba[:, 0] - vca[:, 0] * vba[:, 2],
                       vca[:, 0] * vba[:, 1] - vca[:, 1] * vba[:, 0]], axis=1)
    else:
        e3 = np.stack([vba[:, 1] * vca[:, 2] - vba[:, 2] * vca[:, 1],
                       vba[:, 2] * vca[:, 0] - vba[:, 0] * vca[:, 2],
                       vba[:, 0] * vca[:, 1] - vba[:, 1] * vca[:, 0]], axis=1)
    rr = np.sqrt(e3[:, 0] * e3[:, 0] + e3[:, 1] * e3[:, 1] + e3[:, 2] * e3[:, 2])
    e3 = e3 / rr[:, None]
    horiz = ~(np.abs(e3[:, 2]) < 1)
    e1 = np.stack([e3[:, 1], -e3[:, 0], np.zeros(len(e3))], axis=1)
    r1 = np.sqrt(e1[:, 0] * e1[:, 0] + e1[:, 1] * e1[:, 1])
    with np.errstate(invalid="ignore", divide="ignore"):
        e1[:, 0] /= r1
        e1[:, 1] /= r1
    e1[horiz] = [1.0, 0.0, 0.0]
    e2 = np.stack([e3[:, 1] * e1[:, 2] - e3[:, 2] * e1[:, 1],
                   e3[:, 2] * e1[:, 0] - e3[:, 0] * e1[:, 2],
                   e3[:, 0] * e1[:, 1] - e3[:, 1] * e1[:, 0]], axis=1)
    return np.concatenate([e1, e2, e3], axis=1), xg


def find_boundary_edges_and_nodes(triangles):
    """Edges used by exactly one triangle, and their nodes (src/QDsim.py:56-78)."""
    tri = np.asarray(triangles)
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e = np.sort(e, axis=1)
    uniq, cnt = np.unique(e, axis=0, return_counts=True)
    bedges = uniq[cnt == 1]
    # order of first appearance, as the reference's dict iteration
    key = e[:, 0].astype(np.int64) * (int(tri.max()) + 1) + e[:, 1]
    bkey = set((bedges[:, 0].astype(np.int64) * (int(tri.max()) + 1) + bedges[:, 1]).tolist())
    seen, order = set(), []
    for k in key.tolist():
        if k in bkey and k not in seen:
            seen.add(k)
            order.append(k)
    m = int(tri.max()) + 1
    edges = [(k // m, k % m) for k in order]
    nodes = set()
    for a, b in edges:
        nodes.add(a)
        nodes.add(b)
    return edges, np.array(list(nodes))

"""Operator checkpoint: the assembled, packed H-matrix on disk.

Replaces the reference's `blocks_to_process.joblib` (written by BlockTree.master,
src/Hmatrix.py:1240-1241; found and loaded by QDsim.get_block_core,
src/QDsim.py:199-218).  The reference pickles per-block Python objects; this file
holds the device buffers the matvec reads, so a load is a few large host->device
copies and no Green's-function work.

File layout (little endian):
  bytes 0-7     magic b"PQ3DOP\\x00\\x01"
  bytes 8-15    uint64 header length L
  bytes 16-     JSON header (L bytes): version, fingerprint, operator parameters,
                and a section table [{name, dtype, count, offset}]
  sections      raw arrays, each starting on a 4096-byte boundary
Sections: dense_recs (DENSE_BLOCK records), aca_ranks, aca_flags (int32 per ACA
task), dense64 / dense32 (when assembled), U_<prec> / V_<prec> for each packed
storage precision.

The fingerprint is a SHA-256 over the element centroids and frames, the elastic
constants, the cluster/admissibility/ACA parameters, the half-space mode and
the layout constants; a
load with any of them different is refused (Pq3dError) rather than silently
producing another operator.
"""
import hashlib
import json
import os
import struct as _struct

import numpy as np

from . import _lib

MAGIC = b"PQ3DOP\x00\x01"
VERSION = 1
ALIGN = 4096
FILE_NAME = "operator.pq3d"

_NP = {"float64": np.float64, "float32": np.float32, "int32": np.int32, "uint16": np.uint16, "uint8": np.uint8,
       "int16": np.int16, "int8": np.int8}


def fingerprint(xg, ev, mu, lam, mini_leaf, eta, min_size, aca_tol, aca_rel, aca_seed, kcap, layout, halfspace=0):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(xg, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(ev, dtype=np.float64).tobytes())
    h.update(json.dumps(dict(mu=float(mu), lam=float(lam), mini_leaf=int(mini_leaf), eta=float(eta),
                             min_size=int(min_size), aca_tol=float(aca_tol), aca_rel=bool(aca_rel),
                             aca_seed=int(aca_seed), kcap=int(kcap), layout=layout, halfspace=int(halfspace)),
                        sort_keys=True).encode())
    return h.hexdigest()


def _layout(op):
    return dict(dense={str(k): v for k, v in op.DENSE_CHUNK_GROUPS.items()},
                v={str(k): v for k, v in op.V_CHUNK_GROUPS.items()}, u_rows=op.U_ROWS,
                dense_block=_lib.DENSE_BLOCK.itemsize, mixed_tol=float(getattr(op, "mixed_tol", 0.0)))


def op_fingerprint(op, xg, ev):
    s = op.s
    return fingerprint(xg, ev, op.mu, op.lam, s.mini_leaf, s.eta, s.min_size, op.aca_tol, op.aca_rel, op.aca_seed,
                       op.kcap, _layout(op), getattr(op, "halfspace", 0))


def _host(t):
    """Device tensor -> numpy array (bf16 kept as its raw 16-bit pattern)."""
    import torch
    if t.dtype == torch.bfloat16:
        return t.view(torch.int16).cpu().numpy().view(np.uint16)
    return t.cpu().numpy()


def save_operator(op, path, xg, ev):
    """Write every packed precision of an assembled DeviceHMatrix."""
    if not op.assembled:
        raise _lib.Pq3dError("operator is not assembled")
    arrays = [("dense_recs", np.ascontiguousarray(op.dense_recs).view(np.uint8)),
              ("aca_ranks", np.asarray(op.aca_ranks, dtype=np.int32)),
              ("aca_flags", np.asarray(op.aca_flags, dtype=np.int32))]
    if op.dense64 is not None:
        arrays.append(("dense64", _host(op.dense64)))
    if op.dense32 is not None:
        arrays.append(("dense32", _host(op.dense32)))
    precisions = sorted(op.plans)
    for d in precisions:
        arrays.append(("U_" + d, _host(op.plans[d]["U"])))
        arrays.append(("V_" + d, _host(op.plans[d]["V"])))
        if d == "mixed":
            # the FP16 / INT8 class arrays, their scales and every term's class code
            M = op.plans[d]["mixed"]
            arrays += [("U16_mixed", _host(M["U"][1]).view(np.int16)), ("V16_mixed", _host(M["V"][1]).view(np.int16)),
                       ("U8_mixed", _host(M["U"][2])), ("V8_mixed", _host(M["V"][2])),
                       ("scales_mixed", _host(M["scales"])), ("tmap_mixed", np.asarray(op.mixed_tmap, np.int32))]
    table, off = [], 0
    for name, a in arrays:
        table.append(dict(name=name, dtype=str(a.dtype), count=int(a.size), offset=off))
        off += -(-a.nbytes // ALIGN) * ALIGN
    header = dict(version=VERSION, n=int(op.n), fingerprint=op_fingerprint(op, xg, ev), precisions=precisions,
                  n_dense=int(len(op.dense_recs)), n_aca_tasks=int(len(op.aca_ranks)), sections=table)
    hb = json.dumps(header).encode()
    data0 = -(-(16 + len(hb)) // ALIGN) * ALIGN
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(_struct.pack("<Q", len(hb)))
        f.write(hb)
        for (name, a), t in zip(arrays, table):
            f.seek(data0 + t["offset"])
            f.write(np.ascontiguousarray(a).tobytes())
        end = data0 + off
        f.truncate(end)
    os.replace(tmp, path)
    return header


def read_header(path):
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise _lib.Pq3dError(f"{path}: not an operator checkpoint")
        (L,) = _struct.unpack("<Q", f.read(8))
        header = json.loads(f.read(L).decode())
    if header.get("version") != VERSION:
        raise _lib.Pq3dError(f"{path}: checkpoint version {header.get('version')} != {VERSION}")
    header["_data0"] = -(-(16 + L) // ALIGN) * ALIGN
    return header


def _read(path, header, name):
    for t in header["sections"]:
        if t["name"] == name:
            return np.fromfile(path, dtype=_NP[t["dtype"]], count=t["count"], offset=header["_data0"] + t["offset"])
    return None


def load_operator(op, path, xg, ev):
    """Fill a freshly constructed (unassembled) DeviceHMatrix from a checkpoint.
    Raises Pq3dError if the file belongs to another mesh or parameter set."""
    import torch
    header = read_header(path)
    if header["n"] != op.n or header["fingerprint"] != op_fingerprint(op, xg, ev):
        raise _lib.Pq3dError(f"{path}: checkpoint was written for another mesh or operator parameters")
    op.dense_recs = _read(path, header, "dense_recs").view(_lib.DENSE_BLOCK).copy()
    op.aca_ranks = _read(path, header, "aca_ranks").copy()
    op.aca_flags = _read(path, header, "aca_flags").copy()
    if len(op.dense_recs) != header["n_dense"] or len(op.aca_ranks) != 2 * len(op.aca_blocks):
        raise _lib.Pq3dError(f"{path}: block counts do not match the cluster structure")
    d64 = _read(path, header, "dense64")
    d32 = _read(path, header, "dense32")
    op.dense64 = torch.from_numpy(d64).to(op.dev) if d64 is not None else None
    op.dense32 = torch.from_numpy(d32).to(op.dev) if d32 is not None else None
    op.aca_ws = []
    op.task_ws = {}
    for d in header["precisions"]:
        U, V = _read(path, header, "U_" + d), _read(path, header, "V_" + d)
        if d == "mixed":
            t = lambda name, dt=None: torch.from_numpy(_read(path, header, name).copy()).to(op.dev)
            op.install_mixed(_read(path, header, "tmap_mixed").copy(),
                             [t("U_mixed"), t("U16_mixed").view(torch.float16), t("U8_mixed")],
                             [t("V_mixed"), t("V16_mixed").view(torch.float16), t("V8_mixed")], t("scales_mixed"))
            continue
        if d == "bf16":
            Ut = torch.from_numpy(U.view(np.int16)).to(op.dev).view(torch.bfloat16)
            Vt = torch.from_numpy(V.view(np.int16)).to(op.dev).view(torch.bfloat16)
        else:
            Ut, Vt = torch.from_numpy(U).to(op.dev), torch.from_numpy(V).to(op.dev)
        op.install_plan(d, Ut, Vt)
    op.assembled = True
    torch.cuda.synchronize()
    return header

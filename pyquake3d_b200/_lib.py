"""ctypes binding of libpq3d.so (declared in include/pq3d.h).

The library is the only compute path: if it is missing or a call fails, an
exception is raised.  There is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpq3d.so")

c_dp = ctypes.POINTER(ctypes.c_double)
vp = ctypes.c_void_p
i64 = ctypes.c_int64
i32 = ctypes.c_int

# Record layouts (must match pyquake3d_b200/csrc/*.cu; checked at load time).
DENSE_BLOCK = np.dtype([("off64", "i8"), ("off32", "i8"), ("m", "i4"), ("n", "i4"), ("r0", "i4"), ("c0", "i4")], align=True)
DENSE_ITEM = np.dtype([("off", "i8"), ("m", "i4"), ("r", "i4"), ("g0", "i4"), ("g1", "i4"), ("c0", "i4"), ("slot", "i4")], align=True)
V_ITEM = np.dtype([("off", "i8"), ("Q", "i4"), ("q", "i4"), ("nr", "i4"), ("g0", "i4"), ("g1", "i4"), ("c0", "i4"), ("s", "i4"), ("tp", "i4")], align=True)
# mixed storage, plain kernels: merged V items over the rows of blocks sharing a column cluster
V_ITEM_M = np.dtype([("rows", "i8"), ("nr", "i4"), ("g0", "i4"), ("g1", "i4"), ("c0", "i4"), ("s", "i4"), ("pad", "i4")],
                    align=True)
V_ROW = np.dtype([("base", "i8"), ("stride", "i4"), ("out", "i4")], align=True)
U_TASK = np.dtype([("off", "i8"), ("m", "i4"), ("r0", "i4"), ("r1", "i4"), ("K", "i4"), ("kS", "i4"), ("kD", "i4"), ("Q", "i4"), ("tp", "i4"), ("nch", "i4"), ("slot", "i4")], align=True)
ACA_TASK = np.dtype([("rows_off", "i8"), ("cols_off", "i8"), ("ws_off", "i8"), ("m", "i4"), ("n", "i4"), ("kmax", "i4"), ("pass_", "i4"), ("iref0", "i4"), ("jref0", "i4")], align=True)
PACK_TASK = np.dtype([("ws_off", "i8"), ("u_off", "i8"), ("v_off", "i8"), ("rows_off", "i8"), ("cols_off", "i8"),
                      ("m", "i4"), ("n", "i4"), ("kmax", "i4"), ("k", "i4"), ("pass_", "i4"), ("kS", "i4"), ("kD", "i4"),
                      ("K", "i4"), ("Q", "i4"), ("r0", "i4"), ("c0", "i4"), ("zeroB", "i4")], align=True)
_PLAN_PTRS = ["dense", "U", "V", "ditems", "vitems", "utasks", "leaf_of_row", "leaf_ptr", "leaf_off"]
HM_PLAN = np.dtype([("n", "i4"), ("dtype", "i4")] + [(p, "u8") for p in _PLAN_PTRS] +
                   [(k, "i8") for k in ("n_ditems", "n_vitems", "n_utasks", "n_slots", "n_tpart")] +
                   [("kmax", "i4"), ("pad", "i4")] +
                   [(p, "u8") for p in ("U16", "V16", "U8", "V8", "scales", "status")] +
                   [("stream", "i4"), ("pad2", "i4")] +
                   [(p, "u8") for p in ("tasks_a", "tasks_b", "cta_a", "cta_b", "gather", "tfull")] +
                   [("n_gather", "i8"), ("ncta_a", "i4"), ("ncta_b", "i4"), ("vrows", "u8"), ("vwarp", "u8"),
                    ("n_vwarp", "i4"), ("pad3", "i4")], align=True)
# streamed mixed kernels (k_stream in hmatvec.cu): stage bytes, shared x/t buffer (floats),
# the row limits of dense and U tasks
STREAM_STAGE_BYTES, STREAM_BUF, STREAM_DENSE_ROWS, STREAM_ROWS = 12288, 3072, 128, 256
STREAM_TASK = np.dtype([("off", "i8"), ("off1", "i8"), ("off2", "i8")] +
                       [(k, "i4") for k in ("kind", "cls", "m", "r0", "r1", "g0", "g1", "c0", "out", "kS3",
                                            "K0", "K1", "K2", "tb")], align=True)
T_GATHER = np.dtype([(k, "i4", 3) for k in ("K", "kS", "kD", "Q", "tp", "nch", "sb")] + [("tb", "i4"), ("pad", "i4")],
                    align=True)
# mixed storage (FP32 / FP16 / INT8 term classes): U task and packing records
U_TASK_M = np.dtype([("off", "i8", 3), ("m", "i4"), ("r0", "i4"), ("r1", "i4"), ("slot", "i4")] +
                    [(k, "i4", 3) for k in ("K", "kS", "kD", "Q", "tp", "nch", "sb")] + [("pad", "i4")], align=True)
PACK_TASK_M = np.dtype([("ws_off", "i8"), ("rows_off", "i8"), ("cols_off", "i8"), ("tmap_off", "i8"),
                        ("u_off", "i8", 3), ("v_off", "i8", 3)] +
                       [(k, "i4") for k in ("m", "n", "kmax", "k", "pass_", "r0", "c0", "zeroB")] +
                       [(k, "i4", 3) for k in ("kS", "kD", "Q", "K", "sb")] + [("pad", "i4")], align=True)
_RK_PTRS = ["Tno", "Tt1o", "Tt2o", "psi", "slip1", "slip2", "slipv1", "slipv2", "slipv", "rake", "Tt", "fric", "slip",
            "a", "b", "dc", "f0", "shear_loading", "normal_loading", "vplc", "cr0", "sr0",
            "y", "cand", "blk", "x", "ctrl", "hist", "hforce", "bar", "slots", "leaf_of_row", "leaf_ptr", "leaf_off",
            "ctrl_host"]
RK_ARGS = np.dtype([(p, "u8") for p in _RK_PTRS] +
                   [("n", "i4"), ("fix_tn", "i4"), ("x_fp32", "i4"), ("step_index", "i4"), ("fuse_rowsum", "i4"),
                    ("slots_fp32", "i4"), ("V0", "f8"), ("eta", "f8"), ("reltol", "f8"), ("h_in", "f8")],
                   align=True)

_ENS_PTRS = ["Tno", "Tt1o", "Tt2o", "psi", "slip1", "slip2", "slipv1", "slipv2", "slipv", "rake", "Tt", "fric", "slip",
             "a", "b", "dc", "f0", "shear_loading", "normal_loading", "vplc", "cr0", "sr0",
             "y", "cand", "x", "slots", "leaf_of_row", "leaf_ptr", "leaf_off", "task_row", "task_fault", "fault_task",
             "tmax", "ctrl", "fstate", "hist", "hforce", "bar"]
ENS_ARGS = np.dtype([(p, "u8") for p in _ENS_PTRS] +
                    [(k, "i4") for k in ("n", "n_faults", "n_tasks", "fix_tn", "x_fp32", "step_index", "fuse_rowsum",
                                         "slots_fp32")] +
                    [("V0", "f8"), ("eta", "f8"), ("reltol", "f8")], align=True)

_lib = None


class Pq3dError(RuntimeError):
    pass


_ERR = {-1: "bad argument", -2: "CUDA runtime failure", -3: "ACA rank cap", -4: "step-size controller gave up",
        -5: "device wait timed out", -6: "scratch too small"}


def check(rc, what):
    if rc != 0:
        raise Pq3dError(f"{what} failed: {rc} ({_ERR.get(rc, 'unknown')})")


def load():
    """Load libpq3d.so (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise Pq3dError(f"{LIB_PATH} is missing: build it with `python -m pyquake3d_b200.build` "
                        "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.TDstressFS_C.argtypes = [c_dp, c_dp, c_dp, ctypes.c_size_t, c_dp, c_dp, c_dp, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_bool, c_dp, c_dp]
    L.TDstressFS_C.restype = None
    L.TDstressEachSourceAtReceiver_C.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, c_dp, c_dp, c_dp,
                                                 ctypes.c_size_t, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_bool, c_dp, c_dp]
    L.TDstressEachSourceAtReceiver_C.restype = None
    L.pq3d_src_record_bytes.restype = ctypes.c_size_t
    L.pq3d_src_records.argtypes = [vp, vp, i64, vp, vp]
    L.pq3d_traction_pairs.argtypes = [vp, vp, vp, vp, vp, i64, ctypes.c_double, ctypes.c_double, vp, vp, i32, vp]
    L.pq3d_hs_record_bytes.restype = ctypes.c_size_t
    L.pq3d_hs_records.argtypes = [vp, vp, i64, vp, vp]
    L.pq3d_stress_points.argtypes = [vp, vp, vp, i64, vp, i64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, i32, vp, vp, vp]
    L.pq3d_dense_assemble.argtypes = [vp, vp, vp, vp, vp, i64, ctypes.c_double, ctypes.c_double, vp, vp, vp, i32, vp]
    L.pq3d_aca_ws_doubles.argtypes = [i32, i32, i32]
    L.pq3d_aca_ws_doubles.restype = i64
    L.pq3d_aca_task_bytes.restype = ctypes.c_size_t
    L.pq3d_pack_task_bytes.restype = ctypes.c_size_t
    L.pq3d_aca_batched.argtypes = [vp, vp, vp, vp, vp, vp, i64, vp, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, i32, i32, vp, vp, vp, i32, vp]
    L.pq3d_aca_pack.argtypes = [vp, i64, vp, vp, vp, vp, i32, vp, vp, vp]
    L.pq3d_item_bytes.argtypes = [i32]
    L.pq3d_item_bytes.restype = ctypes.c_size_t
    L.pq3d_hmatvec.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.pq3d_pack_mixed_task_bytes.restype = ctypes.c_size_t
    L.pq3d_stream_ctas.restype = ctypes.c_int
    L.pq3d_vmix_ctas.restype = ctypes.c_int
    L.pq3d_nearfield_rowabs.argtypes = [vp, vp, i64, i32, vp, vp]
    L.pq3d_aca_term_weights.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp]
    L.pq3d_aca_pack_mixed.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.pq3d_rk_args_bytes.restype = ctypes.c_size_t
    L.pq3d_rk_grid.argtypes = [i32]
    L.pq3d_rk_step.argtypes = [vp, i32, vp]
    L.pq3d_rk_rows_attempt.argtypes = [vp, i32, i32, i32, ctypes.c_double, i32, vp, vp]
    L.pq3d_rk_rows_accept.argtypes = [vp, i32, i32, i32, ctypes.c_double, vp, vp]
    L.pq3d_rk_rows_attempt_dev.argtypes = [vp, i32, i32, i32, vp, vp, vp]
    L.pq3d_rk_rows_control.argtypes = [vp, vp, ctypes.c_double, i32, vp]
    L.pq3d_rk_rows_accept_dev.argtypes = [vp, i32, i32, i32, vp, vp, vp]
    L.pq3d_rk_rows_finish.argtypes = [vp, vp, vp]
    L.pq3d_host_map_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(vp), ctypes.POINTER(vp)]
    L.pq3d_host_map_free.argtypes = [vp]
    L.pq3d_event_create.argtypes = [ctypes.POINTER(vp)]
    for f in ("pq3d_event_destroy", "pq3d_event_sync", "pq3d_event_query"):
        getattr(L, f).argtypes = [vp]
    L.pq3d_event_record.argtypes = [vp, vp]
    L.pq3d_snapshot.argtypes = [i32, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, i32]
    L.pq3d_stream_wait_event.argtypes = [vp, vp]
    L.pq3d_ens_args_bytes.restype = ctypes.c_size_t
    L.pq3d_ens_grid.argtypes = [i32]
    L.pq3d_ens_step.argtypes = [vp, i32, vp]
    for f in ("pq3d_src_records", "pq3d_hs_records", "pq3d_traction_pairs", "pq3d_stress_points", "pq3d_dense_assemble",
              "pq3d_aca_batched", "pq3d_aca_pack", "pq3d_hmatvec", "pq3d_nearfield_rowabs", "pq3d_aca_term_weights",
              "pq3d_aca_pack_mixed", "pq3d_rk_grid", "pq3d_rk_step", "pq3d_ens_grid",
              "pq3d_ens_step", "pq3d_ens_task_rows", "pq3d_rk_rows_attempt", "pq3d_rk_rows_accept",
              "pq3d_rk_rows_attempt_dev", "pq3d_rk_rows_control", "pq3d_rk_rows_accept_dev", "pq3d_rk_rows_finish",
              "pq3d_host_map_alloc", "pq3d_host_map_free", "pq3d_event_create", "pq3d_event_destroy",
              "pq3d_event_record", "pq3d_event_sync", "pq3d_event_query", "pq3d_snapshot", "pq3d_stream_wait_event"):
        getattr(L, f).restype = ctypes.c_int
    sizes = {"DenseItem": (L.pq3d_item_bytes(0), DENSE_ITEM.itemsize), "VItem": (L.pq3d_item_bytes(1), V_ITEM.itemsize),
             "UTask": (L.pq3d_item_bytes(2), U_TASK.itemsize), "UTaskM": (L.pq3d_item_bytes(6), U_TASK_M.itemsize),
             "PackTaskM": (L.pq3d_pack_mixed_task_bytes(), PACK_TASK_M.itemsize),
             "StreamTask": (L.pq3d_item_bytes(7), STREAM_TASK.itemsize), "TGather": (L.pq3d_item_bytes(8), T_GATHER.itemsize),
             "VItemM": (L.pq3d_item_bytes(9), V_ITEM_M.itemsize), "VRowRec": (L.pq3d_item_bytes(10), V_ROW.itemsize),
             "DenseBlock": (L.pq3d_item_bytes(4), DENSE_BLOCK.itemsize), "HmPlan": (L.pq3d_item_bytes(5), HM_PLAN.itemsize),
             "AcaTask": (L.pq3d_aca_task_bytes(), ACA_TASK.itemsize), "PackTask": (L.pq3d_pack_task_bytes(), PACK_TASK.itemsize),
             "RkArgs": (L.pq3d_rk_args_bytes(), RK_ARGS.itemsize),
             "EnsArgs": (L.pq3d_ens_args_bytes(), ENS_ARGS.itemsize)}
    bad = {k: v for k, v in sizes.items() if v[0] != v[1]}
    if bad:
        raise Pq3dError(f"record layout mismatch between libpq3d.so and Python: {bad}")
    _lib = L
    return L


def exported_symbols():
    """Symbol names declared in include/pq3d.h."""
    hdr = os.path.join(os.path.dirname(_HERE), "include", "pq3d.h")
    import re
    names = []
    for line in open(hdr):
        m = re.match(r"^\s*(?:void|int|int64_t|size_t)\s+(\w+)\s*\(", line)
        if m:
            names.append(m.group(1))
    return names


def ptr(t):
    """Device (or host) address of a torch tensor / numpy array, None for None."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def stream_ptr(stream=None):
    """cudaStream_t of a torch stream, of the current stream (None), or a raw handle (int)."""
    if isinstance(stream, int):
        return stream
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream

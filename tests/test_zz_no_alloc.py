"""The allocation-free step entry point (pq3d_rk_step_noalloc) against pq3d_rk_step.

Callers that cannot allocate device memory (a host framework that owns every
device buffer, an embedded solver that is handed only its state vectors, a
time loop that must not call cudaMalloc) use pq3d_rk_step_noalloc: its
scratch is a static array inside libpq3d.so.  Both entry points run the same
deterministic kernel on the same inputs, so this test requires bitwise equal
results: two identical device states are stepped twice, one through each
entry point; then a third stepper takes an allocating step with its own
scratch, and a third allocation-free step must still equal the allocating
one (each call resets the static array's barrier and result words).  It
builds its own case so it runs alone in a fresh process as well as after
other tests.
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FIELDS = ("Tno", "Tt1o", "Tt2o", "psi", "slip1", "slip2", "slipv1", "slipv2", "slipv")


@pytest.fixture(scope="module")
def steppers(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyquake3d_b200 import QDsim, meshgen, read_mshV2
    from pyquake3d_b200.qdsim import DeviceStepper
    d = str(tmp_path_factory.mktemp("noalloc"))
    msh, para = meshgen.make_case("tiny", d, n_target=400)
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para, precision="fp64")
    op = sim.tree_block.op()
    return sim, op, DeviceStepper(sim, op, "fp64"), DeviceStepper(sim, op, "fp64"), DeviceStepper(sim, op, "fp64")


def _noalloc_fn(L):
    fn = L.pq3d_rk_step_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _assert_bitwise(new, ref, call):
    c_ref, c_new = ref.ctrl.cpu().numpy(), new.ctrl.cpu().numpy()
    assert c_new[4] == 0 and c_ref[4] == 0
    assert np.array_equal(c_new[:12], c_ref[:12]), call          # dtnext, h, time, rejects, maxima, counters
    for k in FIELDS:
        a, b = new.t[k].cpu().numpy(), ref.t[k].cpu().numpy()
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (call, k)


def test_noalloc_step_matches_allocating_step_bitwise(steppers):
    from pyquake3d_b200 import _lib
    L = _lib.load()
    fn = _noalloc_fn(L)
    sim, op, ref, new, other = steppers
    st = _lib.stream_ptr()
    ref.ctrl[0] = sim.htry
    new.ctrl[0] = sim.htry
    other.ctrl[0] = 0.5 * sim.htry
    for call in range(3):
        if call == 2:
            # an allocating step of another stepper (its own cand/blk/bar scratch) in between
            op.matvec(other.x, "fp64", y=other.y)
            other.args["step_index"] = 0
            _lib.check(L.pq3d_rk_step(other.args.ctypes.data, other.grid, st), "pq3d_rk_step")
        op.matvec(ref.x, "fp64", y=ref.y)
        ref.args["step_index"] = call
        _lib.check(L.pq3d_rk_step(ref.args.ctypes.data, ref.grid, st), "pq3d_rk_step")
        op.matvec(new.x, "fp64", y=new.y)
        new.args["step_index"] = call
        _lib.check(fn(new.args.ctypes.data, new.grid, st), "pq3d_rk_step_noalloc")
        torch.cuda.synchronize()
        _assert_bitwise(new, ref, call)


def test_noalloc_rejects_sizes_beyond_its_scratch(steppers):
    from pyquake3d_b200 import _lib
    L = _lib.load()
    fn = _noalloc_fn(L)
    sim, op, ref, new, other = steppers
    big = new.args.copy()
    big["n"] = 131072 + 1
    assert fn(big.ctypes.data, new.grid, _lib.stream_ptr()) == -6     # PQ3D_ERR_NOMEM, nothing launched
    assert fn(new.args.ctypes.data, 4096 + 1, _lib.stream_ptr()) == -6  # grid above the static per-CTA slots

"""GPU: the host-driven step (QDsim.simu_forward) with pre-launched products.

DeviceStepper.step enqueues the NEXT step's H-matvec before it waits for the
current step's control block.  The products live in the operator's slots, which
every stepper of one precision shares, so any other writer of the slots (another
stepper's step, a direct matvec, a graph replay) must make the next step compute
them again.  Each trajectory must stay bitwise equal to an uninterrupted run."""
import numpy as np
import pytest

from pyquake3d_b200 import _lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _lib.load()


@pytest.fixture(scope="module")
def tiny(lib, tiny_files):
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1], precision="fp32")    # operator packed FP64 and FP32
    return sim, sim.tree_block.op()


def _trajectory(st, dttry, nsteps, between=None):
    out = []
    for i in range(nsteps):
        h, dttry = st.step(dttry)
        out.append((h, dttry))
        if between is not None:
            between(i)
    return out, {k: st.get(k) for k in ("slipv", "Tt", "slip", "psi")}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_interleaved_steppers_bitwise(tiny, prec):
    from pyquake3d_b200.qdsim import DeviceStepper
    sim, op = tiny
    n = 12
    ref_h, ref_s = _trajectory(DeviceStepper(sim, op, prec), sim.htry, n)

    a, b, c = (DeviceStepper(sim, op, prec) for _ in range(3))
    g = c.capture(1)
    assert g is not None
    c.ctrl[0] = sim.htry
    hb, dtb = [], [sim.htry]

    def between(i):
        # another stepper of the same precision steps: its products overwrite the slots
        h, d = b.step(dtb[-1])
        hb.append((h, d))
        dtb.append(d)
        if i == 4:
            op.matvec(a.x, prec, slots_only=True)      # a direct matvec of the same plan
        if i == 7:
            g.replay()                                  # a graph replay writes the slots too

    got_h, got_s = _trajectory(a, sim.htry, n, between)
    assert got_h == ref_h
    assert hb == ref_h
    for k in ref_s:
        assert np.array_equal(got_s[k], ref_s[k]), k
        assert np.array_equal(b.get(k), ref_s[k]), k


def test_step_reuses_prelaunched_products(tiny):
    """Back-to-back calls consume the pre-launched products (one matvec per step,
    not two): the plan's owner token survives between calls."""
    from pyquake3d_b200.qdsim import DeviceStepper
    sim, op = tiny
    st = DeviceStepper(sim, op, "fp64")
    P = op.plan("fp64")
    calls = []
    orig = op.matvec

    def counting(*a, **k):
        calls.append(1)
        return orig(*a, **k)

    op.matvec = counting
    try:
        d = sim.htry
        for _ in range(5):
            _, d = st.step(d)
    finally:
        del op.matvec
    assert P["slots_owner"] is st._token
    assert len(calls) == 6          # one for the first step, then one pre-launch per step


def test_snapshot_after_other_launches(tiny):
    """snapshot_async after launches that bypass step() (run, a graph replay) reads
    the state those launches left; after step() it reads that step's state while
    the next H-matvec is already enqueued."""
    from pyquake3d_b200.qdsim import DeviceStepper
    sim, op = tiny
    names = ("slipv", "Tt", "psi")
    st = DeviceStepper(sim, op, "fp64")

    def check_snapshot():
        done, host = st.snapshot_async(names)
        done.synchronize()
        assert done.query()
        for k in names:
            assert np.array_equal(host[k], st.get(k)), k

    st.run(3, sim.htry)
    check_snapshot()
    g = st.capture(2)
    g.replay()
    check_snapshot()
    d = float(st.ctrl[0].item())
    for _ in range(3):
        _, d = st.step(d)
        check_snapshot()


def test_reference_loop_reads_current_state(lib, tiny_files):
    """The reference main loop reads sim0.slipv1, sim0.slipv2, sim0.slipv and sim0.Tt
    after every simu_forward (src/main.py:168-184).  Those attributes hold the step
    just taken: equal to the device state read back synchronously, distinct arrays
    per step, and max |V1|, max |V2| equal to the step kernel's own maxima."""
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1])
    v0 = sim.slipv.copy()
    dttry = sim.htry
    slipv_hist, copies = [], []
    for i in range(6):
        dttry, dtnext = sim.simu_forward(dttry)
        st = sim._dev
        m1, m2 = np.max(np.abs(sim.slipv1)), np.max(np.abs(sim.slipv2))
        c = st.ctrl.cpu().numpy()
        assert m1 == c[5] and m2 == c[6], i
        assert (sim.max_slipv1, sim.max_slipv2) == (m1, m2), i
        for name, dev in (("slipv", "slipv"), ("Tt", "Tt"), ("state", "psi"), ("slip", "slip")):
            assert np.array_equal(getattr(sim, name), st.get(dev)), (i, name)
        slipv_hist.append(sim.slipv)
        copies.append(st.get("slipv"))
        dttry = dtnext
    # the kept arrays are the host copier's fresh arrays: later steps leave them alone
    for i, (a, b) in enumerate(zip(slipv_hist, copies)):
        assert np.array_equal(a, b), i
    assert not np.array_equal(slipv_hist[0], v0)
    assert not np.array_equal(slipv_hist[0], slipv_hist[-1])
    assert len({id(a) for a in slipv_hist}) == len(slipv_hist)


def test_attributes_follow_bulk_device_steps(lib, tiny_files):
    """After bulk stepping through the DeviceStepper (run, a captured graph), the
    QDsim attributes read the device state, without an explicit sync_to_host;
    after sync_to_host they are the synced arrays themselves."""
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1])
    st = sim._ensure_device()
    v0 = sim.slipv.copy()
    assert np.array_equal(sim.slipv, v0)              # no step yet: the host arrays
    st.run(5, sim.htry)
    assert np.array_equal(sim.slipv, st.get("slipv"))
    assert not np.array_equal(sim.slipv, v0)
    g = st.capture(2)
    g.replay()
    for name, dev in (("Tt", "Tt"), ("state", "psi"), ("slip1", "slip1")):
        assert np.array_equal(getattr(sim, name), st.get(dev)), name
    sim.sync_to_host()
    a = sim.slipv
    assert a is sim.slipv and np.array_equal(a, st.get("slipv"))

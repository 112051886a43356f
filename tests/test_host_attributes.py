"""Host logic of QDsim's device-backed state attributes (no GPU: a stand-in for
the DeviceStepper).  An attribute is the host array until the stepper's launch
count moves; then its first read fetches the device values (once), reads are
remembered for the next step's prefetch, assignments replace the value, and a
sync marks every attribute current."""
import numpy as np


class FakeStepper:
    def __init__(self, n):
        self._token = object()
        self.version = 0
        self.n = n
        self.fetches = []

    def read_field(self, name):
        self.fetches.append(name)
        return np.full(self.n, float(self.version) + (0.5 if name == "psi" else 0.0))


def _attach(sim):
    st = FakeStepper(len(sim.xg))
    sim._dev = st
    sim._host_key = (st._token, st.version)
    sim._stale = set()
    return st


def test_attributes_follow_the_stepper_version(tiny_files):
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1])          # its own instance: the attributes get overwritten
    v0 = sim.slipv.copy()
    st = _attach(sim)
    assert np.array_equal(sim.slipv, v0) and st.fetches == []          # nothing launched: host arrays
    st.version += 1                                                     # a step kernel ran
    a = sim.slipv
    assert st.fetches == ["slipv"] and np.all(a == 1.0)
    assert sim.slipv is a and st.fetches == ["slipv"]                   # fetched once per step
    assert np.all(sim.state == 1.5) and st.fetches[-1] == "psi"         # reference name -> device field
    assert {"slipv", "state"} <= sim._reads
    sim.Tt = np.zeros(len(sim.xg))                                      # assignment replaces the value
    assert np.all(sim.Tt == 0.0) and "Tt" not in st.fetches
    st.version += 2
    assert np.all(sim.slipv == 3.0) and np.all(sim.Tt == 3.0)           # stale again after more launches
    # a sync marks everything current for this stepper version
    sim._host_key = (st._token, st.version)
    sim._stale = set()
    n = len(st.fetches)
    sim.slip1, sim.Tno
    assert len(st.fetches) == n
    # another stepper object with the same version number is still another state
    other = FakeStepper(len(sim.xg))
    other.version = st.version
    sim._dev = other
    sim.slipv
    assert other.fetches == ["slipv"]

"""GPU: the ensemble step kernel against single-fault runs.

Three faults of uneven size stepped together (one block-diagonal matvec, one
cooperative step launch per step) follow, fault by fault, the adaptive step
sequences of the same faults run alone with the single-fault stepper (FP64
operators: h to 1e-9 relative, slip to 1e-9 of its maximum).  A CUDA graph of
ensemble steps reproduces eager stepping bitwise, and an FP32 ensemble on the
FP64 ensemble's step sizes (dt replay) stays within 1e-6 in slip per fault."""
import numpy as np
import pytest

from pyquake3d_b200 import _lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

STEPS = 20


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    _lib.load()
    from pyquake3d_b200.meshgen import ensemble_faults
    return ensemble_faults(str(tmp_path_factory.mktemp("ens")), n_faults=3, seed=4, lo=300, hi=900, edge=1.0)


def _sims(files):
    from pyquake3d_b200 import QDsim, read_mshV2
    out = []
    for msh, para in files:
        nodes, tris = read_mshV2(msh)
        out.append(QDsim(tris, nodes, para, precision="fp64"))
    return out


def test_ensemble_follows_single_fault_runs(files):
    from pyquake3d_b200.ensemble import Ensemble
    sims = _sims(files)
    E = Ensemble(sims, precision="fp64")
    hist = E.run(STEPS, [s.htry for s in sims])
    for f, s in enumerate(_sims(files)):
        st = s._ensure_device()
        h1 = st.run(STEPS, s.htry)
        np.testing.assert_allclose(hist[:, f, 0], h1[:, 0], rtol=1e-9)
        np.testing.assert_allclose(hist[:, f, 2], h1[:, 2], rtol=1e-9)
        for name in ("slip1", "slip2", "psi", "Tt1o"):
            a, b = E.get(name, f), st.get(name)
            assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), (f, name)


def test_ensemble_graph_equals_eager(files):
    from pyquake3d_b200.ensemble import Ensemble
    sims = _sims(files)
    E = Ensemble(sims, precision="fp32")
    saved = {k: v.clone() for k, v in E.t.items()}
    x0 = E.x.clone()
    ha = E.run(10, [s.htry for s in sims])
    slip_a = E.t["slip1"].cpu().numpy()
    for k, v in saved.items():
        E.t[k].copy_(v)
    E.x.copy_(x0)
    E.ctrl.zero_()
    E.ctrl[:, 0] = torch.tensor([s.htry for s in sims], dtype=torch.float64, device=E.op.dev)
    E.set_history(10)
    g = E.capture(10)
    assert g is not None
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(ha, E.hist.cpu().numpy()[:10])
    assert np.array_equal(slip_a, E.t["slip1"].cpu().numpy())


def test_ensemble_mixed_precision_on_fp64_steps(files):
    from pyquake3d_b200.ensemble import Ensemble
    ref = Ensemble(_sims(files), precision="fp64")
    h = ref.run(STEPS, [s.htry for s in ref.sims])
    mix = Ensemble(_sims(files), precision="fp32")
    mix.set_replay(torch.tensor(h[:, :, 0], device=mix.op.dev))
    hm = mix.run(STEPS, [s.htry for s in mix.sims])
    assert np.array_equal(hm[:, :, 0], h[:, :, 0])
    for f in range(ref.M):
        a, b = mix.get("slip", f), ref.get("slip", f)
        assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b), f

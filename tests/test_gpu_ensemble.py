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


def test_full_32_fault_deck_fp32_and_mixed_within_target_or_chaos_floor(tmp_path_factory):
    """The benchmark's config-4 deck (32 planar faults of U[2000, 20000] triangles, seed 4,
    dips U[20, 90] degrees, seeded friction), 100 steps: the FP32 and mixed-storage
    ensembles on the FP64 ensemble's step sizes (dt replay).  Each fault's slip error
    must stay within the 1e-5 target, or within twice that fault's FP64 chaos floor --
    the same error between two FP64 runs whose initial shear tractions differ by a
    relative 1e-12 -- where the fault itself amplifies any perturbation beyond the
    target (an accelerating fault: no storage short of the FP64 run reproduces it)."""
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.ensemble import Ensemble
    from pyquake3d_b200.meshgen import ensemble_faults
    files = ensemble_faults(str(tmp_path_factory.mktemp("deck32")), n_faults=32, seed=4, lo=2000, hi=20000, edge=0.5)
    sims = []
    for msh, para in files:
        nodes, tris = read_mshV2(msh)
        sims.append(QDsim(tris, nodes, para, precision="fp32"))
    nrep = 100
    h0 = [s.htry for s in sims]
    E64 = Ensemble(sims, precision="fp64", want=("fp64", "fp32", "mixed"))
    h = E64.run(nrep, h0)
    runs = {}
    for name, prec in (("fp32", "fp32"), ("mixed", "mixed"), ("floor", "fp64")):
        R = Ensemble(sims, precision=prec, share=E64)
        if name == "floor":                    # both shear components (a pure-dip fault has Tt1o = 0)
            R.t["Tt1o"].mul_(1.0 + 1e-12)
            R.t["Tt2o"].mul_(1.0 + 1e-12)
        R.set_replay(torch.tensor(h[:, :, 0], device=R.op.dev))
        R.run(nrep, h0)
        runs[name] = R
    worst = {}
    for f in range(len(sims)):
        b = E64.get("slip", f)
        e = {k: float(np.linalg.norm(R.get("slip", f) - b) / np.linalg.norm(b)) for k, R in runs.items()}
        for k in ("fp32", "mixed"):
            assert e[k] <= max(1e-5, 2.0 * e["floor"]), (f, e)
            worst[k] = max(worst.get(k, 0.0), e[k])
    assert worst["fp32"] <= 1e-4 and worst["mixed"] <= 1e-4, worst

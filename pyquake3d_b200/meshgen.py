"""Synthetic fault inputs in the reference's own formats.

Each case is written as a Gmsh 2.2 ASCII mesh (node coordinates in km,
`Scale_km: True`), a 10-column per-element parameter file
(rake a b dc f0 Tt Tno V shear_loading normal_loading, the layout read by
QDsim.read_parameter, src/QDsim.py:687-712) and a parameter.txt, so they run
through the reference input path unchanged.  All randomness is seeded.

Cases (sizes of the benchmark configurations):
  plain2k     planar vertical strike-slip fault 40 x 20 km, ~1.9k triangles, dense operator
  thrust20k   30-degree thrust 100 x 40 km, ~20k triangles, 10% node jitter, leaf 64, ACA 1e-4
  curved60k   150 km rough strike-slip fault + 40 km branch at 20 degrees, ~60k triangles
  curved120k  curved60k refined to ~120k triangles, heterogeneous a-b and sigma_n
  tiny        small planar fault for tests (size set by the caller)
"""
import os

import numpy as np

from .mesh import write_msh

MU = 32e9
LAM = 32e9            # Poisson ratio 0.25
CS = 3464.0
RHO = MU / CS ** 2
V0 = 1e-6
F0 = 0.6
VPL = 1e-9


def grid_surface(nx, nz, point, jitter=0.0, seed=0):
    """Structured triangulation of a parametric surface point(u, w), u, w in [0, 1].
    Diagonals alternate so the mesh is near-uniform.  Interior nodes may be
    jittered by `jitter` times the cell size."""
    u = np.linspace(0.0, 1.0, nx + 1)
    w = np.linspace(0.0, 1.0, nz + 1)
    U, W = np.meshgrid(u, w, indexing="ij")
    if jitter > 0:
        rng = np.random.default_rng(seed)
        du, dw = 1.0 / nx, 1.0 / nz
        J = rng.uniform(-jitter, jitter, size=(2,) + U.shape)
        inner = np.zeros(U.shape, bool)
        inner[1:-1, 1:-1] = True
        U = U + J[0] * du * inner
        W = W + J[1] * dw * inner
    P = point(U.ravel(), W.ravel())
    idx = np.arange((nx + 1) * (nz + 1)).reshape(nx + 1, nz + 1) + 1
    tris = []
    for i in range(nx):
        for k in range(nz):
            a, b, c, d = idx[i, k], idx[i + 1, k], idx[i + 1, k + 1], idx[i, k + 1]
            if (i + k) % 2 == 0:
                tris += [(a, b, c), (a, c, d)]
            else:
                tris += [(a, b, d), (b, c, d)]
    return P, np.array(tris, dtype=np.int64)


def planar(length, width, dip_deg, nx, nz, top=0.0, jitter=0.0, seed=0):
    dip = np.deg2rad(dip_deg)

    def pt(u, w):
        x = (u - 0.5) * length
        d = w * width
        return np.stack([x, d * np.cos(dip), top - d * np.sin(dip)], axis=1)
    return grid_surface(nx, nz, pt, jitter, seed)


def rough_trace(length, seed, ratio=1e-2, wavelengths=(5.0, 10.0, 20.0, 40.0)):
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, len(wavelengths))

    def y(x):
        return sum(ratio * lam * np.sin(2 * np.pi * x / lam + p) for lam, p in zip(wavelengths, ph))
    return y


def curved_branch(n_target, seed=2, depth=20.0):
    """150 km rough vertical strike-slip fault plus a 40 km vertical branch at 20 degrees."""
    L_main, L_br = 150.0, 40.0
    area = (L_main + L_br) * depth
    s = np.sqrt(2.0 * area / n_target)
    ym = rough_trace(L_main, seed)
    nxm, nz = int(round(L_main / s)), int(round(depth / s))
    nxb = int(round(L_br / s))

    def main(u, w):
        x = (u - 0.5) * L_main
        return np.stack([x, ym(x), -w * depth], axis=1)
    P1, T1 = grid_surface(nxm, nz, main)
    # branch leaves the main trace at x = +10 km with a 1 km gap, heading 20 degrees off strike
    th = np.deg2rad(20.0)
    x0 = 10.0
    yb = rough_trace(L_br, seed + 100)

    def branch(u, w):
        d = 1.0 + u * L_br
        x = x0 + d * np.cos(th) - yb(d) * np.sin(th)
        y = ym(x0) + d * np.sin(th) + yb(d) * np.cos(th)
        return np.stack([x, y, -w * depth], axis=1)
    P2, T2 = grid_surface(nxb, nz, branch)
    P = np.concatenate([P1, P2])
    T = np.concatenate([T1, T2 + len(P1)])
    return P, T


def centroids_km(P, T):
    return (P[T[:, 0] - 1] + P[T[:, 1] - 1] + P[T[:, 2] - 1]) / 3.0


def gaussian_field(xc, corr, seed, lo, hi, nmodes=256):
    """Seeded smooth random field (random Fourier features, correlation length corr),
    rescaled into [lo, hi]."""
    rng = np.random.default_rng(seed)
    k = rng.normal(0, 1.0 / corr, size=(nmodes, 3))
    ph = rng.uniform(0, 2 * np.pi, nmodes)
    f = np.sqrt(2.0 / nmodes) * np.cos(xc @ k.T + ph).sum(axis=1)
    f = (f - f.mean()) / (f.std() + 1e-30)
    return np.clip(lo + (hi - lo) * (0.5 + f / 6.0), lo, hi)


def friction_layout(xc, strike_half, seed, core=(2.0, 15.0), a_vw=0.010, a_vs=0.025, b=0.015, dc=0.02,
                    sigma=50.0, perturb=0.01, vw_patch=None, nuc=None):
    """Columns rake a b dc f0 Tt Tno V shear_loading normal_loading for each element."""
    n = len(xc)
    depth = -xc[:, 2]
    a = np.full(n, a_vs)
    inside = (depth >= core[0]) & (depth <= core[1]) & (np.abs(xc[:, 0]) <= strike_half - 2.0)
    if vw_patch is not None:
        inside = vw_patch(xc)
    a[inside] = a_vw
    rng = np.random.default_rng(seed)
    V = VPL * (1.0 + perturb * rng.standard_normal(n))
    if nuc is not None:
        c, r, vn = nuc
        V[np.linalg.norm(xc - np.asarray(c), axis=1) < r] = vn
    cols = np.zeros((n, 10))
    cols[:, 0] = 0.0
    cols[:, 1] = a
    cols[:, 2] = b
    cols[:, 3] = dc
    cols[:, 4] = F0
    cols[:, 5] = 0.0
    cols[:, 6] = sigma
    cols[:, 7] = V
    return cols


PARAM_TEMPLATE = """#Files
Corefunc directory: core
save Corefunc: False
Hmatrix_mpi_plot:False
Node_order: False
Scale_km: True

#Property
Lame constants: {lam!r}
Shear modulus: {mu!r}
Rock density: {rho!r}
InputHetoparamter: True
Inputparamter file: {datname}

#Stress
Half space: False
Fix_Tn:False
Vertical principal stress: 1.0
Maximum horizontal principal stress: 1.6
Minimum horizontal principal stress: 0.6
Angle between ssh1 and X-axis: 30
Vertical principal stress value: 5e7
Vertical principal stress value varies with depth: False
Turnning depth: 15000
Shear traction solved from stress tensor: False
Normal traction solved from stress tensor: False
Rake solved from stress tensor: False
Fix_rake: 0
Widths of VS region: 2000
Widths of surface VS region: 2000
Transition region from VS to VW region: 2000

#Friction
Reference slip rate: {v0!r}
Reference friction coefficient: {f0!r}
Plate loading rate: {vpl!r}
Initlab: False

#output
outputSLIPV: False
outputTt: False
totaloutputsteps: {steps}
outsteps: 100
outputvtk: False
outputmatrix: False

#H-matrix and stepper
H-matrix leaf size: {leaf}
Admissibility eta: 2.0
ACA tolerance: {tol!r}
ACA relative tolerance: {rel}
ACA seed: 0
Precision: {precision}
RK RelTol: 1e-4
"""


def write_case(outdir, name, P, T, cols, leaf, tol, rel, precision, steps):
    os.makedirs(outdir, exist_ok=True)
    msh = os.path.join(outdir, name + ".msh")
    dat = name + "param.dat"
    write_msh(msh, P, T)
    np.savetxt(os.path.join(outdir, dat), cols, fmt="%.17g")
    para = os.path.join(outdir, "parameter.txt")
    with open(para, "w") as f:
        f.write(PARAM_TEMPLATE.format(lam=LAM, mu=MU, rho=RHO, datname=dat, v0=V0, f0=F0, vpl=VPL, steps=steps,
                                      leaf=leaf, tol=tol, rel="True" if rel else "False", precision=precision))
    return msh, para


def ensemble_faults(outdir, n_faults=32, seed=4, lo=2000, hi=20000, edge=0.5, precision="fp32", steps=2000):
    """Batch of independent planar faults of uneven size: N ~ U[lo, hi] triangles
    (seeded), dip ~ U[20, 90] degrees, length = 2 x width, edge ~`edge` km, 10% node
    jitter; velocity weakening a in the core drawn from a seeded smooth random
    field in [0.008, 0.012] (b = 0.015), a = 0.025 elsewhere.  Each fault gets its
    own directory (mesh, 10-column parameter file, parameter.txt); returns the
    list of (msh, parameter.txt)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, n_faults)
    dips = rng.uniform(20.0, 90.0, n_faults)
    out = []
    for f in range(n_faults):
        nz = max(2, int(round(np.sqrt(sizes[f] / 4.0))))
        nx = 2 * nz
        width, length = nz * edge, nx * edge
        P, T = planar(length, width, float(dips[f]), nx, nz, jitter=0.1, seed=seed * 1000 + f)
        xc = centroids_km(P, T)
        depth = -xc[:, 2]
        core = (depth >= 0.1 * width * np.sin(np.deg2rad(dips[f]))) & \
               (depth <= 0.8 * width * np.sin(np.deg2rad(dips[f]))) & (np.abs(xc[:, 0]) <= 0.4 * length)
        cols = friction_layout(xc, length / 2, seed=seed * 1000 + f, vw_patch=lambda c: core)
        cols[core, 1] = gaussian_field(xc[core], max(2.0, width / 4), seed=seed * 1000 + f + 500, lo=0.008, hi=0.012) \
            if core.sum() > 1 else 0.010
        d = os.path.join(outdir, "fault%02d" % f)
        out.append(write_case(d, "fault%02d" % f, P, T, cols, leaf=64, tol=1e-5, rel=True, precision=precision,
                              steps=steps))
    return out


def make_case(name, outdir, n_target=None, precision=None, tol=None):
    """Write one of the named cases; returns (msh_path, parameter_path).  n_target
    resizes `tiny`, `tinynuc`, `thrust20k` (same 100 x 40 km domain, coarser or
    finer edges) and the curved cases; tol overrides the ACA tolerance."""
    if name == "plain2k":
        P, T = planar(40.0, 20.0, 90.0, 44, 22)
        cols = friction_layout(centroids_km(P, T) * 1e3 / 1e3, 20.0, seed=0)
        return write_case(outdir, name, P, T, cols, leaf=100000, tol=0.01, rel=False,
                          precision=precision or "fp64", steps=2000)
    if name == "tiny":
        nx = int(np.sqrt((n_target or 512) / 4.0) * 2)
        nz = max(2, (n_target or 512) // (2 * nx))
        P, T = planar(16.0, 8.0, 70.0, nx, nz, jitter=0.1, seed=5)
        xc = centroids_km(P, T)
        cols = friction_layout(xc, 8.0, seed=0, core=(1.0, 6.0))
        return write_case(outdir, name, P, T, cols, leaf=32, tol=0.01, rel=False,
                          precision=precision or "fp64", steps=100)
    if name == "tinynuc":
        # tiny fault with a 2 km patch slipping at 1 m/s: radiation damping matters there
        nx = int(np.sqrt((n_target or 512) / 4.0) * 2)
        nz = max(2, (n_target or 512) // (2 * nx))
        P, T = planar(16.0, 8.0, 70.0, nx, nz, jitter=0.1, seed=5)
        xc = centroids_km(P, T)
        cols = friction_layout(xc, 8.0, seed=0, core=(1.0, 6.0), nuc=(xc[len(xc) // 2], 2.0, 1.0))
        return write_case(outdir, name, P, T, cols, leaf=32, tol=0.01, rel=False,
                          precision=precision or "fp64", steps=100)
    if name == "thrust20k":
        nz = 64 if n_target is None else max(4, int(round(np.sqrt(n_target / 5.0))))
        nx = 160 if n_target is None else int(round(2.5 * nz))
        P, T = planar(100.0, 40.0, 30.0, nx, nz, jitter=0.1, seed=1)
        xc = centroids_km(P, T)
        dd = -xc[:, 2] / np.sin(np.deg2rad(30.0))   # down-dip distance
        patch = lambda c: (np.abs(c[:, 0]) <= 30.0) & (np.abs(-c[:, 2] / np.sin(np.deg2rad(30.0)) - 20.0) <= 10.0)
        cols = friction_layout(xc, 50.0, seed=1, vw_patch=patch,
                               nuc=((-20.0e0, 20.0 * np.cos(np.deg2rad(30.0)), -10.0), 3.0, 1e-6))
        cols[:, 0] = np.pi / 2   # thrust: rake 90 degrees
        del dd
        return write_case(outdir, name, P, T, cols, leaf=64, tol=tol or 1e-4, rel=True,
                          precision=precision or "fp32", steps=20000)
    if name in ("curved60k", "curved120k"):
        n = n_target or (60000 if name == "curved60k" else 120000)
        P, T = curved_branch(n, seed=2)
        xc = centroids_km(P, T)
        cols = friction_layout(xc, 75.0, seed=2)
        if name == "curved120k":
            amb = gaussian_field(xc, 5.0, seed=3, lo=-0.006, hi=0.006)
            cols[:, 1] = cols[:, 2] + amb
            cols[:, 6] = gaussian_field(xc, 5.0, seed=4, lo=20.0, hi=80.0)
        return write_case(outdir, name, P, T, cols, leaf=64, tol=tol or 1e-5, rel=True,
                          precision=precision or "bf16", steps=20000 if name == "curved60k" else 50000)
    raise ValueError(name)

"""ORACLE -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module, and only as the checker or as the timed CPU path; the
product (pyquake3d_b200) never does.

A CPU restatement, in numpy, of the reference's FP64 hot path:
  gf_block              calc_stressfunc_fromCS/CD, calc_stressfunc_fromC_rowS/D
                        (src/Hmatrix.py:318-511) through the C restatement
                        oracle/td_oracle.c of TDstressFS (src/TDstressFS_C.cpp:274-521)
  aca_plus              ACA_plus_full_traceS/D (src/Hmatrix.py:581-1011)
  OracleOperator        ACA_worker (src/Hmatrix.py:1014-1066) +
                        blocks_process_MVM (src/Hmatrix.py:1445-1538)
  OracleStepper         derivative (src/QDsim.py:760-813),
                        RungeKutte_solve_Dormand_Prince (src/QDsim.py:1001-1134),
                        simu_forward (src/QDsim.py:892-996)
The numpy expressions keep the reference's operation order, so on the same
inputs the results agree with the reference to rounding (pinned by
tests/golden fixtures produced by the reference itself).
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "_build", "libtd_oracle.so")
_td = None


def td_lib():
    global _td
    if _td is None:
        if not os.path.exists(_LIB):
            import subprocess
            subprocess.run(["make", "-C", HERE, os.path.join(HERE, "_build", "libtd_oracle.so")], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(_LIB)
        D = ctypes.POINTER(ctypes.c_double)
        L.td_stress_fs_batch.argtypes = [D, D, D, ctypes.c_size_t, D, D, D] + [ctypes.c_double] * 5 + [D, D]
        L.td_stress_each_source.argtypes = [ctypes.c_double] * 3 + [D, D, D, ctypes.c_size_t] + [ctypes.c_double] * 5 + [D, D]
        L.td_stress_hs_batch.argtypes = [D, D, D, ctypes.c_size_t, D, D, D] + [ctypes.c_double] * 5 + \
            [ctypes.c_int, D, D]
        L.td_traction_block.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                                                 ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                                 ctypes.c_int, ctypes.c_void_p]
        _td = L
    return _td


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def td_stress_fs(X, Y, Z, P1, P2, P3, Ss, Ds, Ts, mu, lam):
    """stress, strain (n x 6) at receivers for one source (TDstressFS_C layout)."""
    L = td_lib()
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    n = len(X)
    s, e = np.zeros(6 * n), np.zeros(6 * n)
    L.td_stress_fs_batch(_p(X), _p(Y), _p(Z), n, _p(np.ascontiguousarray(P1, dtype=np.float64)),
                         _p(np.ascontiguousarray(P2, dtype=np.float64)), _p(np.ascontiguousarray(P3, dtype=np.float64)),
                         Ss, Ds, Ts, mu, lam, _p(s), _p(e))
    return s.reshape(n, 6), e.reshape(n, 6)


def td_stress_hs(X, Y, Z, P1, P2, P3, Ss, Ds, Ts, mu, lam, mode=2):
    """Half-space stress, strain (n x 6), TDstressHS (src/TDstressFS_C.cpp:1911-2000);
    mode 2 follows the compiled C++ path, mode 1 the numpy twin (they differ only
    for a triangle side along z that is not the first side)."""
    L = td_lib()
    X, Y, Z = (np.ascontiguousarray(v, dtype=np.float64) for v in (X, Y, Z))
    n = len(X)
    s, e = np.zeros(6 * n), np.zeros(6 * n)
    L.td_stress_hs_batch(_p(X), _p(Y), _p(Z), n, _p(np.ascontiguousarray(P1, dtype=np.float64)),
                         _p(np.ascontiguousarray(P2, dtype=np.float64)), _p(np.ascontiguousarray(P3, dtype=np.float64)),
                         Ss, Ds, Ts, mu, lam, int(mode), _p(s), _p(e))
    return s.reshape(n, 6), e.reshape(n, 6)


class Geometry:
    """Elements of a mesh; hs_mode 0 full space, 1 / 2 half space (td_stress_hs)."""

    def __init__(self, xg, ev, nodes, tri, mu, lam, hs_mode=0):
        self.hs_mode = int(hs_mode)
        self.xg = np.ascontiguousarray(xg, dtype=np.float64)
        self.ev = np.ascontiguousarray(ev, dtype=np.float64)
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.tri = np.ascontiguousarray(tri, dtype=np.int64)
        self.mu, self.lam = float(mu), float(lam)

    def gf_block(self, rows, cols, which):
        """(A1, A2, B) m x n for which = 1 (strike) or 2 (dip); 6 planes for 3."""
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        m, n = len(rows), len(cols)
        nm = 2 if which == 3 else 1
        out = np.zeros((3 * nm, m, n))
        td_lib().td_traction_block(self.xg.ctypes.data, self.ev.ctypes.data, self.nodes.ctypes.data,
                                   self.tri.ctypes.data, rows.ctypes.data, m, cols.ctypes.data, n, self.mu, self.lam,
                                   which, self.hs_mode, out.ctypes.data)
        return out


def aca_plus(geo, row_cluster, col_cluster, which, eps, iref0, jref0, max_iter=None, rel=False):
    """ACA+ of one block for one slip mode; returns dict of U (m x k) and V (k x n)
    for A1, A2, B (B empty when all its u vectors are zero), and the pivots.

    rel=False: the reference's stop, ||u_k|| ||v_k / alpha|| < eps with eps
    absolute (src/Hmatrix.py:727,736; eps = 0.01 at :1020-1028).
    rel=True: the relative stop of the `ACA relative tolerance` key, which has
    no counterpart in the reference: ||u_k|| ||v_k / alpha|| <= eps ||S_k||_F,
    where S_k = sum_{p<=k} u_p v_p^T is the A1 approximant after this step and
    its squared Frobenius norm is updated incrementally,
        ||S_k||^2 = ||S_{k-1}||^2 + 2 sum_{p<k} (u_p . u_k)(v_p . v_k/alpha)
                    + ||u_k||^2 ||v_k/alpha||^2,
    with v_p the stored (pivot-scaled) rows.  Pivots, reference sets and the
    other stops are the reference's."""
    n_rows, n_cols = len(row_cluster), len(col_cluster)
    us1, vs1, us2, vs2, usB, vsB = [], [], [], [], [], []
    prevI, prevJ = [], []

    def argmax_not_in_list(arr, disallowed):
        srt = arr.argsort()
        k = srt.shape[0] - 1
        while k >= 0:
            if srt[k] not in disallowed:
                return srt[k]
            k -= 1
        raise RuntimeError("All entries disallowed.")

    def rows_res(I0, I1):
        o = geo.gf_block(row_cluster[I0:I1], col_cluster, which)
        a1, a2, b = o[0], o[1], o[2]
        for i in range(len(us1)):
            a1 -= us1[i][I0:I1][:, None] * vs1[i][None, :]
            a2 -= us2[i][I0:I1][:, None] * vs2[i][None, :]
            b -= usB[i][I0:I1][:, None] * vsB[i][None, :]
        return a1, a2, b

    def cols_res(J0, J1):
        o = geo.gf_block(row_cluster, col_cluster[J0:J1], which)
        a1, a2, b = o[0], o[1], o[2]
        for i in range(len(us1)):
            a1 -= vs1[i][J0:J1][None, :] * us1[i][:, None]
            a2 -= vs2[i][J0:J1][None, :] * us2[i][:, None]
            b -= vsB[i][J0:J1][None, :] * usB[i][:, None]
        return a1, a2, b

    def reset_row(Iref):
        att, mx, scan = 0, n_rows // 3 + 1, False
        while True:
            Iref = (Iref + 3) % n_rows
            Iref -= Iref % 3
            att += 1
            if Iref not in prevI:
                break
            if att > mx:
                scan = True
                break
        o = rows_res(Iref, Iref + 3)
        return o[0], Iref, scan

    def reset_col(Jref):
        att, mx, scan = 0, n_cols // 3 + 1, False
        while True:
            Jref = (Jref + 3) % n_cols
            Jref -= Jref % 3
            att += 1
            if Jref not in prevJ:
                break
            if att > mx:
                scan = True
                break
        o = cols_res(Jref, Jref + 3)
        return o[0], Jref, scan

    if max_iter is None:
        max_iter = min(n_rows, n_cols)
    RIstar, RIstar1, RIstar2 = np.zeros(n_cols), np.zeros(n_cols), np.zeros(n_cols)
    RJstar, RJstar1, RJstar2 = np.zeros(n_rows), np.zeros(n_rows), np.zeros(n_rows)
    RIref, Iref, scan_all = reset_row(iref0)
    RJref, Jref, scan_all = reset_col(jref0)
    frob2 = 0.0
    for k in range(max_iter):
        mR = np.max(np.abs(RIref), axis=0)
        Jstar = argmax_not_in_list(mR, prevJ)
        mC = np.max(np.abs(RJref), axis=1)
        Istar = argmax_not_in_list(mC, prevI)
        if mC[Istar] > mR[Jstar]:
            o = rows_res(Istar, Istar + 1)
            RIstar[:], RIstar1[:], RIstar2[:] = o[0][0], o[1][0], o[2][0]
            Jstar = argmax_not_in_list(np.abs(RIstar), prevJ)
            o = cols_res(Jstar, Jstar + 1)
            RJstar[:], RJstar1[:], RJstar2[:] = o[0][:, 0], o[1][:, 0], o[2][:, 0]
        else:
            o = cols_res(Jstar, Jstar + 1)
            RJstar[:], RJstar1[:], RJstar2[:] = o[0][:, 0], o[1][:, 0], o[2][:, 0]
            Istar = argmax_not_in_list(np.abs(RJstar), prevI)
            o = rows_res(Istar, Istar + 1)
            RIstar[:], RIstar1[:], RIstar2[:] = o[0][0], o[1][0], o[2][0]
        alpha, alpha1, alpha2 = RIstar[Jstar], RIstar1[Jstar], RIstar2[Jstar]
        if np.abs(alpha) < 1e-4:
            break
        prevI.append(Istar)
        prevJ.append(Jstar)
        u_k, v_k = RJstar.copy(), RIstar.copy()
        us1.append(u_k)
        vs1.append(v_k / (alpha + 1e-16))
        us2.append(RJstar1.copy())
        vs2.append(RIstar1.copy() / (alpha1 + 1e-16))
        usB.append(RJstar2.copy())
        vsB.append(np.zeros(len(RIstar2)) if abs(alpha2) < 1e-10 else RIstar2.copy() / (alpha2 + 1e-16))
        su, sv = np.sum(u_k ** 2), np.sum((v_k / alpha) ** 2)
        step = np.sqrt(su * sv)
        if rel:
            w = v_k / alpha
            cross = 0.0
            for p in range(len(us1) - 1):
                cross += np.dot(us1[p], u_k) * np.dot(vs1[p], w)
            frob2 += 2.0 * cross + su * sv
            if step <= eps * np.sqrt(abs(frob2)):
                break
        elif step < eps:
            break
        if k == max_iter - 1:
            break
        if Iref <= Istar < Iref + 3:
            RIref, Iref, scan_all = reset_row(Iref)
        else:
            RIref -= u_k[Iref:Iref + 3][:, None] * (v_k / alpha)[None, :]
        if scan_all:
            break
        if Jref <= Jstar < Jref + 3:
            RJref, Jref, scan_all = reset_col(Jref)
        else:
            RJref -= (v_k / alpha)[Jref:Jref + 3][None, :] * u_k[:, None]
        if scan_all:
            break
    res = dict(U1=np.array(us1).T, V1=np.array(vs1), U2=np.array(us2).T, V2=np.array(vs2), prevI=prevI, prevJ=prevJ)
    uB = np.array(usB)
    if not np.all(uB == 0):
        res["UB"], res["VB"] = uB.T, np.array(vsB)
    else:
        res["UB"], res["VB"] = [], []
    return res


class OracleOperator:
    """Per-block FP64 operator: dense Mf_* or ACA factors, as ACA_worker builds them.

    blocks: list of (row_cluster, col_cluster, is_aca) with the reference's
    cluster index order (ascending element ids); starts: per ACA block
    ((iref0_S, jref0_S), (iref0_D, jref0_D))."""

    OPS = ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd")

    def __init__(self, geo, blocks, starts=None, eps=0.01, rel=False):
        self.geo = geo
        self.blocks = []
        si = 0
        for rc, cc, aca in blocks:
            rc = np.asarray(rc)
            cc = np.asarray(cc)
            if aca:
                (i0, j0), (i1, j1) = starts[si]
                si += 1
                S = aca_plus(geo, rc, cc, 1, eps, i0, j0, rel=rel)
                D = aca_plus(geo, rc, cc, 2, eps, i1, j1, rel=rel)
                self.blocks.append(("aca", rc, cc, S, D))
            else:
                o = geo.gf_block(rc, cc, 3)
                self.blocks.append(("dense", rc, cc, o))

    def mvm(self, x, op):
        """blocks_process_MVM(x, blocks, op) (src/Hmatrix.py:1445-1538)."""
        y = np.zeros(len(x))
        k = self.OPS.index(op)
        for b in self.blocks:
            x_ = x[b[2]]
            if b[0] == "aca":
                d = b[3] if k < 3 else b[4]
                c = k % 3
                U = d[("U1", "U2", "UB")[c]]
                V = d[("V1", "V2", "VB")[c]]
                if len(U) == 0 or (hasattr(U, "size") and U.size == 0):
                    ax = np.zeros(len(b[1]))
                else:
                    ax = U.dot(V.dot(x_))
            else:
                ax = b[3][k] @ x_
            y[b[1]] = y[b[1]] + ax
        return y

    def ranks(self):
        return [(b[3]["U1"].shape[1] if b[3]["U1"].size else 0, b[4]["U1"].shape[1] if b[4]["U1"].size else 0)
                for b in self.blocks if b[0] == "aca"]


class OracleStepper:
    """simu_forward + RungeKutte_solve_Dormand_Prince + derivative in FP64 numpy.

    mvm(x1, x2) -> (dsig_from_B, AdotV1, AdotV2) supplies the elastic load."""

    def __init__(self, state, mvm, V0, mu, Cs, reltol=1e-4, fix_tn=False):
        for k in ("Tno", "Tt1o", "Tt2o", "state", "slipv1", "slipv2", "slipv", "slip1", "slip2", "a", "b", "dc",
                  "f0", "shear_loading", "normal_loading", "slipvC", "rake0"):
            setattr(self, k, np.array(state[k], dtype=np.float64, copy=True))
        self.mvm = mvm
        self.V0, self.mu, self.Cs = V0, mu, Cs
        self.RelTol = reltol
        self.fix_Tn = fix_tn
        self.time = 0.0

    def derivative(self, Tno, Tt1o, Tt2o, state):
        Tno = Tno * 1e6
        Tt1o = Tt1o * 1e6
        Tt2o = Tt2o * 1e6

        def safe_exp(x, max_value=700):
            return np.exp(np.clip(x, -max_value, max_value))
        V0, a, b, dc, f0 = self.V0, self.a, self.b, self.dc, self.f0
        dV1dtau = 2 * V0 / (a * Tno) * 0.5 * (np.exp(-state / a + Tt1o / (a * Tno)) + np.exp(-state / a - Tt1o / (a * Tno)))
        dV2dtau = 2 * V0 / (a * Tno) * 0.5 * (np.exp(-state / a + Tt2o / (a * Tno)) + np.exp(-state / a - Tt2o / (a * Tno)))
        dV1dsigma = -2 * V0 * Tt1o / (a * Tno ** 2) * 0.5 * (np.exp(-state / a + Tt1o / (a * Tno)) + np.exp(-state / a - Tt1o / (a * Tno)))
        dV2dsigma = -2 * V0 * Tt2o / (a * Tno ** 2) * 0.5 * (np.exp(-state / a + Tt2o / (a * Tno)) + np.exp(-state / a - Tt2o / (a * Tno)))
        dV1dstate = -2 * V0 / a * 0.5 * (np.exp(-state / a + Tt1o / (a * Tno)) - np.exp(-state / a - Tt1o / (a * Tno)))
        dV2dstate = -2 * V0 / a * 0.5 * (np.exp(-state / a + Tt2o / (a * Tno)) - np.exp(-state / a - Tt2o / (a * Tno)))
        dstatedt = b / dc * (V0 * safe_exp((f0 - state) / b) - self.slipv)
        eta = self.mu / (2.0 * self.Cs)
        dtau1dt = (-self.AdotV1 + self.shear_loading - eta * (dV1dsigma * self.dsigmadt + dV1dstate * dstatedt)) / (1.0 + eta * dV1dtau)
        dtau2dt = (-self.AdotV2 + self.shear_loading - eta * (dV2dsigma * self.dsigmadt + dV2dstate * dstatedt)) / (1.0 + eta * dV2dtau)
        return dstatedt, self.dsigmadt / 1e6, dtau1dt / 1e6, dtau2dt / 1e6

    def rk_stages(self, h):
        """The seven DP5(4) stages (src/QDsim.py:1001-1134): (y5, y8), each the
        tuple (Tno, Tt1o, Tt2o, psi) of element arrays."""
        B21 = .2
        B31, B32 = 3. / 40, 9. / 40.
        B41, B42, B43 = 44. / 45., -56. / 15, 32. / 9
        B51, B52, B53, B54 = 19372. / 6561., -25360 / 2187., 64448. / 6561., -212. / 729.
        B61, B62, B63, B64, B65 = 9017. / 3168., -355. / 33., -46732. / 5247., 49. / 176., -5103. / 18656.
        B71, B73, B74, B75, B76 = 35. / 384., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.
        B81, B83, B84, B85, B86, B87 = 5179. / 57600., 7571. / 16695., 393. / 640., -92097. / 339200., 187. / 2100., 1. / 40.
        y0 = (self.Tno, self.Tt1o, self.Tt2o, self.state)
        order = (1, 2, 3, 0)  # derivative returns (dpsi, dsig, dt1, dt2); state order is (Tno, Tt1o, Tt2o, psi)

        def der(y):
            d = self.derivative(*y)
            return (d[1], d[2], d[3], d[0])
        k1 = der(y0)
        y = tuple(y0[q] + h * B21 * k1[q] for q in range(4))
        k2 = der(y)
        y = tuple(y0[q] + h * (B31 * k1[q] + B32 * k2[q]) for q in range(4))
        k3 = der(y)
        y = tuple(y0[q] + h * (B41 * k1[q] + B42 * k2[q] + B43 * k3[q]) for q in range(4))
        k4 = der(y)
        y = tuple(y0[q] + h * (B51 * k1[q] + B52 * k2[q] + B53 * k3[q] + B54 * k4[q]) for q in range(4))
        k5 = der(y)
        y = tuple(y0[q] + h * (B61 * k1[q] + B62 * k2[q] + B63 * k3[q] + B64 * k4[q] + B65 * k5[q]) for q in range(4))
        k6 = der(y)
        y5 = tuple(y0[q] + h * (B71 * k1[q] + B73 * k3[q] + B74 * k4[q] + B75 * k5[q] + B76 * k6[q]) for q in range(4))
        k7 = der(y5)
        y8 = tuple(y0[q] + h * (B81 * k1[q] + B83 * k3[q] + B84 * k4[q] + B85 * k5[q] + B86 * k6[q] + B87 * k7[q])
                   for q in range(4))
        del order
        return y5, y8

    def rk(self, h):
        """One attempt: 5th-order candidate, error ratios and proposed steps."""
        y5, y8 = self.rk_stages(h)
        err = tuple(np.abs(y8[q] - y5[q]) for q in range(4))
        R1 = np.max(np.abs(err[3] / y8[3])) + 1e-10
        R2 = max(np.max(np.abs(err[1] / y8[1])), np.max(np.abs(err[2] / y8[2])), np.max(np.abs(err[0] / y8[0]))) + 1e-10
        c1, c2 = R1 / self.RelTol, R2 / self.RelTol
        hn1 = h * 0.9 * (self.RelTol / R1) ** 0.2
        hn2 = h * 0.9 * (self.RelTol / R2) ** 0.2
        return y5, c1, c2, hn1, hn2

    def simu_forward(self, dttry, h_forced=None):
        x1 = self.slipv1 - self.slipvC * np.cos(self.rake0)
        x2 = self.slipv2 - self.slipvC * np.sin(self.rake0)
        sigB, self.AdotV1, self.AdotV2 = self.mvm(x1, x2)
        self.dsigmadt = self.normal_loading if self.fix_Tn else sigB + self.normal_loading
        nrjct = 0
        h = dttry
        while True:
            y5, c1, c2, hn1, hn2 = self.rk(h if h_forced is None else h_forced)
            if h_forced is not None:
                h = h_forced
                dtnext = min(min(hn1, hn2), 1.5 * h)
                break
            if max(c1, c2) < 1.0 and not (np.isnan(c1) or np.isnan(c2)):
                dtnext = min(hn1, hn2)
                dtnext = min(1.5 * h, dtnext)
                break
            nrjct += 1
            dtnext = min(hn1, hn2)
            h = max(0.5 * h, dtnext)
            if h < 1.e-15 or nrjct > 20:
                raise RuntimeError("error: dt is too small")
        self.time = self.time + h
        self.Tno, self.Tt1o, self.Tt2o, self.state = y5
        self.Tt = np.sqrt(self.Tt1o * self.Tt1o + self.Tt2o * self.Tt2o)
        self.slipv1 = (2.0 * self.V0) * np.exp(-self.state / self.a) * np.sinh(self.Tt1o / self.Tno / self.a)
        self.slipv2 = (2.0 * self.V0) * np.exp(-self.state / self.a) * np.sinh(self.Tt2o / self.Tno / self.a)
        self.slipv = np.sqrt(self.slipv1 * self.slipv1 + self.slipv2 * self.slipv2)
        self.rake = np.arctan2(self.Tt2o, self.Tt1o)
        self.slipv[self.slipv < 1e-30] = 1e-30
        self.slip1 = self.slip1 + self.slipv1 * h
        self.slip2 = self.slip2 + self.slipv2 * h
        self.slip = np.sqrt(self.slip1 * self.slip1 + self.slip2 * self.slip2)
        self.nrjct = nrjct
        return h, dtnext


def operator_mvm(op):
    """Elastic load (B x, A1 x, A2 x) from an OracleOperator, six MVMs as simu_forward."""
    def f(x1, x2):
        sig = op.mvm(x1, "Bs") + op.mvm(x2, "Bd")
        a1 = op.mvm(x1, "A1s") + op.mvm(x2, "A1d")
        a2 = op.mvm(x1, "A2s") + op.mvm(x2, "A2d")
        return sig, a1, a2
    return f


def sim_state(sim):
    """Initial state dict from a QDsim-like object (reference attribute names)."""
    return dict(Tno=sim.Tno, Tt1o=sim.Tt1o, Tt2o=sim.Tt2o, state=sim.state, slipv1=sim.slipv1, slipv2=sim.slipv2,
                slipv=sim.slipv, slip1=sim.slip1, slip2=sim.slip2, a=sim.a, b=sim.b, dc=sim.dc, f0=sim.f0,
                shear_loading=sim.shear_loading, normal_loading=sim.normal_loading, slipvC=sim.slipvC,
                rake0=sim.rake0)


# ------------------------------------------------------------------ parallel assembly
# The reference assembles with an MPI master handing blocks to worker ranks
# (BlockTree.master / worker / ACA_worker, src/Hmatrix.py:1014-1066, 1136-1260).
# Here a process pool stands in for the ranks; every block is computed exactly
# as OracleOperator computes it, and the results are collected in block order.
_POOL_GEO = {}


def _pool_init(geo):
    _POOL_GEO["geo"] = geo


def _pool_block(task):
    rc, cc, aca, start, eps, rel = task
    geo = _POOL_GEO["geo"]
    if aca:
        (i0, j0), (i1, j1) = start
        S = aca_plus(geo, rc, cc, 1, eps, i0, j0, rel=rel)
        D = aca_plus(geo, rc, cc, 2, eps, i1, j1, rel=rel)
        for d in (S, D):
            d.pop("prevI", None)
            d.pop("prevJ", None)
        return ("aca", rc, cc, S, D)
    return ("dense", rc, cc, geo.gf_block(rc, cc, 3))


def build_operator_parallel(geo, blocks, starts, eps=0.01, rel=False, procs=None):
    """OracleOperator of `blocks` [(row_cluster, col_cluster, is_aca)] assembled by a
    pool of `procs` spawned processes (default: every host core).  Largest blocks are
    handed out first; the block list keeps the input order."""
    import multiprocessing as mp
    tasks, si = [], 0
    for rc, cc, aca in blocks:
        st = None
        if aca:
            st = starts[si]
            si += 1
        tasks.append((np.asarray(rc), np.asarray(cc), bool(aca), st, float(eps), bool(rel)))
    cost = [len(t[0]) * len(t[1]) if not t[2] else 60 * (len(t[0]) + len(t[1])) for t in tasks]
    order = np.argsort(cost)[::-1]
    procs = procs or os.cpu_count() or 1
    out = [None] * len(tasks)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_pool_init, initargs=(geo,)) as pool:
        for i, res in zip(order, pool.imap(_pool_block, [tasks[i] for i in order], chunksize=4)):
            out[i] = res
    op = object.__new__(OracleOperator)
    op.geo = geo
    op.blocks = out
    return op

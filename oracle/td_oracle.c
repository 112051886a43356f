/*
 * ORACLE -- test infrastructure only.  Nothing in the product links this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it,
 * and only as the checker.
 *
 * Plain-C restatement of the full-space triangular-dislocation (TD) stress of
 * Nikkhoo & Walter (2015), following the reference implementation
 * src/TDstressFS_C.cpp (PyQuake3D):
 *   tens_trans      <- TensTrans          TDstressFS_C.cpp:21-49
 *   ang_dis_strain  <- AngDisStrain       TDstressFS_C.cpp:51-121
 *   trimode         <- trimodefinder      TDstressFS_C.cpp:125-166
 *   td_setup        <- TDSetupS           TDstressFS_C.cpp:185-256
 *   td_stress_fs    <- TDstressFS         TDstressFS_C.cpp:274-521
 *   td_stress_fs_batch / td_stress_each_source
 *                   <- TDstressFS_C / TDstressEachSourceAtReceiver_C
 *                                         TDstressFS_C.cpp:2048-2143 (full space only)
 *   td_traction     <- BlockTree.GetTtstress  src/Hmatrix.py:295-313
 *
 * Differences kept on purpose: none in arithmetic intent.  The horizontal-
 * triangle case (strike vector of zero length) divides by zero exactly as the
 * reference does (TDstressFS_C.cpp:318-325), so it yields NaN there too.
 * Component order of every 6-vector is xx, yy, zz, xy, xz, yz.
 * Parity of this restatement is pinned against the reference library built
 * from source (oracle/_ref) and the reference's numpy twin
 * (src/SH_greenfunction.py:198-318) through tests/golden fixtures.
 */
#include <math.h>
#include <stddef.h>

static const double TD_PI = 3.141592653589793;

/* Rotate a symmetric tensor t (xx,yy,zz,xy,xz,yz) with matrix A: t' = A^T t A. */
static void tens_trans(double t[6], const double A[3][3])
{
    double xx = t[0], yy = t[1], zz = t[2], xy = t[3], xz = t[4], yz = t[5];
    double o[6];
    int p[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int c = 0; c < 6; ++c) {
        int i = p[c][0], j = p[c][1];
        o[c] = A[0][i] * A[0][j] * xx + (A[0][i] * A[1][j] + A[0][j] * A[1][i]) * xy
             + (A[0][i] * A[2][j] + A[0][j] * A[2][i]) * xz
             + (A[2][j] * A[1][i] + A[2][i] * A[1][j]) * yz
             + A[1][j] * A[1][i] * yy + A[2][i] * A[2][j] * zz;
    }
    for (int c = 0; c < 6; ++c) t[c] = o[c];
}

/* Strain of one angular dislocation (Burgers vector bx,by,bz, angle alpha)
 * at point (x,y,z) of its own coordinate system. */
static void ang_dis_strain(double x, double y, double z, double alpha,
                           double bx, double by, double bz, double nu, double e[6])
{
    double cA = cos(alpha), sA = sin(alpha);
    double eta = y * cA - z * sA;
    double zeta = y * sA + z * cA;
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double r2 = x2 + y2 + z2;
    double r = sqrt(r2);
    double r3 = r2 * r;
    double rz = r * (r - z);
    double r2z2 = r2 * (r - z) * (r - z);
    double r3z = r3 * (r - z);
    double W = zeta - r;
    double W2 = W * W;
    double Wr = W * r;
    double W2r = W2 * r;
    double Wr3 = W * r3;
    double W2r2 = W2 * r2;
    double C = (r * cA - z) / Wr;
    double S = (r * sA - y) / Wr;
    /* Same association order as the reference: b / 8 / pi / (1 - nu) * (...). */
#define KF(b) ((b) / 8.0 / TD_PI / (1 - nu))
    double rFi_rx = (eta / r / (r - zeta) - y / r / (r - z)) / 4.0 / TD_PI;
    double rFi_ry = (x / r / (r - z) - cA * x / r / (r - zeta)) / 4.0 / TD_PI;
    double rFi_rz = (sA * x / r / (r - zeta)) / 4.0 / TD_PI;

    e[0] = bx * rFi_rx
         + KF(bx) * (eta / Wr + eta * x2 / W2r2 - eta * x2 / Wr3 + y / rz - x2 * y / r2z2 - x2 * y / r3z)
         - KF(by * x) * (((2 * nu + 1) / Wr + x2 / W2r2 - x2 / Wr3) * cA + (2 * nu + 1) / rz - x2 / r2z2 - x2 / r3z)
         + KF(bz * x * sA) * ((2 * nu + 1) / Wr + x2 / W2r2 - x2 / Wr3);
    e[1] = by * rFi_ry
         + KF(bx) * ((1.0 / Wr + S * S - y2 / Wr3) * eta + (2 * nu + 1) * y / rz - y2 * y / r2z2 - y2 * y / r3z - 2 * nu * cA * S)
         - KF(by * x) * (1.0 / rz - y2 / r2z2 - y2 / r3z + (1.0 / Wr + S * S - y2 / Wr3) * cA)
         + KF(bz * x * sA) * (1.0 / Wr + S * S - y2 / Wr3);
    e[2] = bz * rFi_rz
         + KF(bx) * (eta / W / r + eta * C * C - eta * z2 / Wr3 + y * z / r3 + 2 * nu * sA * C)
         - KF(by * x) * ((1.0 / Wr + C * C - z2 / Wr3) * cA + z / r3)
         + KF(bz * x * sA) * (1.0 / Wr + C * C - z2 / Wr3);
    e[3] = bx * rFi_ry / 2 + by * rFi_rx / 2
         - KF(bx) * (x * y2 / r2z2 - nu * x / rz + x * y2 / r3z - nu * x * cA / Wr + eta * x * S / Wr + eta * x * y / Wr3)
         + KF(by) * (x2 * y / r2z2 - nu * y / rz + x2 * y / r3z + nu * cA * S + x2 * y * cA / Wr3 + x2 * cA * S / Wr)
         - KF(bz * sA) * (nu * S + x2 * S / Wr + x2 * y / Wr3);
    e[4] = bx * rFi_rz / 2 + bz * rFi_rx / 2
         - KF(bx) * (-x * y / r3 + nu * x * sA / Wr + eta * x * C / Wr + eta * x * z / Wr3)
         + KF(by) * (-x2 / r3 + nu / r + nu * cA * C + x2 * z * cA / Wr3 + x2 * cA * C / Wr)
         - KF(bz * sA) * (nu * C + x2 * C / Wr + x2 * z / Wr3);
    e[5] = by * rFi_rz / 2 + bz * rFi_ry / 2
         + KF(bx) * (y2 / r3 - nu / r - nu * cA * C + nu * sA * S + eta * sA * cA / W2 - eta * (y * cA + z * sA) / W2r + eta * y * z / W2r2 - eta * y * z / Wr3)
         - KF(by * x) * (y / r3 + sA * cA * cA / W2 - cA * (y * cA + z * sA) / W2r + y * z * cA / W2r2 - y * z * cA / Wr3)
         - KF(bz * x * sA) * (y * z / Wr3 - sA * cA / W2 + (y * cA + z * sA) / W2r - y * z / W2r2);
#undef KF
}

/* Barycentric configuration test in the TD coordinate system (x normal,
 * y strike, z dip): +1 regular, -1 the "negative" cone, 0 on the TD plane
 * edge lines. */
static int trimode(const double X[3], const double p1[3], const double p2[3], const double p3[3])
{
    double x1 = p1[1], x2 = p2[1], x3 = p3[1];
    double y1 = p1[2], y2 = p2[2], y3 = p3[2];
    double den = (x1 - x3) * (y2 - y3) - (x2 - x3) * (y1 - y3);
    double xp = X[1], yp = X[2], zp = X[0];
    double a = ((xp - x3) * (y2 - y3) - (x2 - x3) * (yp - y3)) / den;
    double b = ((x1 - x3) * (yp - y3) - (xp - x3) * (y1 - y3)) / den;
    double c = 1.0 - a - b;
    int m = 1;
    if (a <= 0 && b > c && c > a) m = -1;
    else if (b <= 0 && c > a && a > b) m = -1;
    else if (c <= 0 && a > b && b > c) m = -1;
    else if (a == 0 && b >= 0 && c >= 0) m = 0;
    else if (a >= 0 && b == 0 && c >= 0) m = 0;
    else if (a >= 0 && b >= 0 && c == 0) m = 0;
    if (m == 0 && zp != 0) m = 1;
    return m;
}

/* One angular-dislocation pair contribution: rotate the point into the
 * angular-dislocation system attached at vertex tv with side vector sv, take
 * the strain there and rotate it back (TDSetupS). */
static void td_setup(const double X[3], double alpha, double bx, double by, double bz,
                     double nu, const double tv[3], const double sv[3], double e[6])
{
    double A00 = sv[2], A01 = -sv[1], A10 = sv[1], A11 = sv[2];
    double ry = X[1] - tv[1], rz = X[2] - tv[2];
    double y1 = A00 * ry + A01 * rz;
    double z1 = A10 * ry + A11 * rz;
    double by1 = A00 * by + A01 * bz;
    double bz1 = A10 * by + A11 * bz;
    ang_dis_strain(X[0], y1, z1, -TD_PI + alpha, bx, by1, bz1, nu, e);
    const double B[3][3] = {{1.0, 0.0, 0.0}, {0.0, A00, A01}, {0.0, A10, A11}};
    tens_trans(e, B);
}

void td_stress_fs(const double obs[3], const double P1[3], const double P2[3], const double P3[3],
                  double Ss, double Ds, double Ts, double mu, double lam,
                  double stress[6], double strain[6])
{
    double bx = Ts, by = Ss, bz = Ds;
    double nu = 1.0 / (1.0 + lam / mu) / 2.0;
    double vn[3], vs[3], vd[3];
    vn[0] = (P2[1] - P1[1]) * (P3[2] - P1[2]) - (P2[2] - P1[2]) * (P3[1] - P1[1]);
    vn[1] = (P2[2] - P1[2]) * (P3[0] - P1[0]) - (P2[0] - P1[0]) * (P3[2] - P1[2]);
    vn[2] = (P2[0] - P1[0]) * (P3[1] - P1[1]) - (P2[1] - P1[1]) * (P3[0] - P1[0]);
    double nn = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
    vn[0] /= nn; vn[1] /= nn; vn[2] /= nn;
    /* strike = eZ x n */
    vs[0] = 0.0 * vn[2] - 1.0 * vn[1];
    vs[1] = 1.0 * vn[0] - 0.0 * vn[2];
    vs[2] = 0.0 * vn[1] - 0.0 * vn[0];
    double ns = sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
    if (ns == 0) { vs[0] = 0.0 * vn[2]; vs[1] = 1.0 * vn[2]; vs[2] = 0.0 * vn[2]; }
    vs[0] /= ns; vs[1] /= ns; vs[2] /= ns;
    vd[0] = vn[1] * vs[2] - vn[2] * vs[1];
    vd[1] = vn[2] * vs[0] - vn[0] * vs[2];
    vd[2] = vn[0] * vs[1] - vn[1] * vs[0];

    /* columns of At are (n, s, d): local = At^T (p - P2) */
    double d[3] = {obs[0] - P2[0], obs[1] - P2[1], obs[2] - P2[2]};
    double X1[3], p1[3], p2[3] = {0, 0, 0}, p3[3];
    double d1[3] = {P1[0] - P2[0], P1[1] - P2[1], P1[2] - P2[2]};
    double d3[3] = {P3[0] - P2[0], P3[1] - P2[1], P3[2] - P2[2]};
    const double *ax[3] = {vn, vs, vd};
    for (int j = 0; j < 3; ++j) {
        X1[j] = ax[j][0] * d[0] + ax[j][1] * d[1] + ax[j][2] * d[2];
        p1[j] = ax[j][0] * d1[0] + ax[j][1] * d1[1] + ax[j][2] * d1[2];
        p3[j] = ax[j][0] * d3[0] + ax[j][1] * d3[1] + ax[j][2] * d3[2];
    }
    double e12[3], e13[3], e23[3];
    for (int j = 0; j < 3; ++j) { e12[j] = p2[j] - p1[j]; e13[j] = p3[j] - p1[j]; e23[j] = p3[j] - p2[j]; }
    double n12 = sqrt(e12[0] * e12[0] + e12[1] * e12[1] + e12[2] * e12[2]);
    double n13 = sqrt(e13[0] * e13[0] + e13[1] * e13[1] + e13[2] * e13[2]);
    double n23 = sqrt(e23[0] * e23[0] + e23[1] * e23[1] + e23[2] * e23[2]);
    for (int j = 0; j < 3; ++j) { e12[j] /= n12; e13[j] /= n13; e23[j] /= n23; }
    double angA = acos(e12[0] * e13[0] + e12[1] * e13[1] + e12[2] * e13[2]);
    double angB = acos((-e12[0]) * e23[0] + (-e12[1]) * e23[1] + (-e12[2]) * e23[2]);
    double angC = acos(e23[0] * e13[0] + e23[1] * e13[1] + e23[2] * e13[2]);

    int m = trimode(X1, p1, p2, p3);
    double e[6] = {0, 0, 0, 0, 0, 0};
    if (m != 0) {
        double s = (m == 1) ? 1.0 : -1.0;
        double me13[3] = {-s * e13[0], -s * e13[1], -s * e13[2]};
        double se12[3] = {s * e12[0], s * e12[1], s * e12[2]};
        double se23[3] = {s * e23[0], s * e23[1], s * e23[2]};
        double ea[6], eb[6], ec[6];
        td_setup(X1, angA, bx, by, bz, nu, p1, me13, ea);
        td_setup(X1, angB, bx, by, bz, nu, p2, se12, eb);
        td_setup(X1, angC, bx, by, bz, nu, p3, se23, ec);
        for (int c = 0; c < 6; ++c) e[c] = ea[c] + eb[c] + ec[c];
    }
    const double R[3][3] = {{vn[0], vn[1], vn[2]}, {vs[0], vs[1], vs[2]}, {vd[0], vd[1], vd[2]}};
    tens_trans(e, R);
    double tr = e[0] + e[1] + e[2];
    stress[0] = 2 * mu * e[0] + lam * tr;
    stress[1] = 2 * mu * e[1] + lam * tr;
    stress[2] = 2 * mu * e[2] + lam * tr;
    stress[3] = 2 * mu * e[3];
    stress[4] = 2 * mu * e[4];
    stress[5] = 2 * mu * e[5];
    if (strain) for (int c = 0; c < 6; ++c) strain[c] = e[c];
}

/* One source triangle, n receivers (layout of TDstressFS_C). */
void td_stress_fs_batch(const double *X, const double *Y, const double *Z, size_t n,
                        const double *P1, const double *P2, const double *P3,
                        double Ss, double Ds, double Ts, double mu, double lam,
                        double *stress, double *strain)
{
    for (size_t i = 0; i < n; ++i) {
        double o[3] = {X[i], Y[i], Z[i]};
        td_stress_fs(o, P1, P2, P3, Ss, Ds, Ts, mu, lam, stress + 6 * i, strain ? strain + 6 * i : 0);
    }
}

/* One receiver, n sources (layout of TDstressEachSourceAtReceiver_C). */
void td_stress_each_source(double x, double y, double z,
                           const double *P1, const double *P2, const double *P3, size_t ns,
                           double Ss, double Ds, double Ts, double mu, double lam,
                           double *stress, double *strain)
{
    double o[3] = {x, y, z};
    for (size_t i = 0; i < ns; ++i)
        td_stress_fs(o, P1 + 3 * i, P2 + 3 * i, P3 + 3 * i, Ss, Ds, Ts, mu, lam,
                     stress + 6 * i, strain ? strain + 6 * i : 0);
}

/* Traction (tau1, tau2, sigma_n) of a stress tensor on the receiver frame
 * ev = (e1 strike, e2 dip, e3 normal) row-major (GetTtstress). */
static void td_traction(const double s[6], const double *ev, double t[3])
{
    double tr1 = s[0] * ev[6] + s[3] * ev[7] + s[4] * ev[8];
    double tr2 = s[3] * ev[6] + s[1] * ev[7] + s[5] * ev[8];
    double trn = s[4] * ev[6] + s[5] * ev[7] + s[2] * ev[8];
    t[0] = tr1 * ev[0] + tr2 * ev[1] + trn * ev[2];
    t[1] = tr1 * ev[3] + tr2 * ev[4] + trn * ev[5];
    t[2] = tr1 * ev[6] + tr2 * ev[7] + trn * ev[8];
}

/* Traction block: rows = receivers (centroids xg[ri], frames ev[ri]),
 * cols = source elements.  which: 1 strike slip (Ss=1), 2 dip slip (Ds=1),
 * 3 both; hs_mode 0 full space, 1 or 2 half space (td_stress_hs).  out holds
 * 3 planes per computed mode of m*n doubles, row-major, in
 * the order A1, A2, B (strike first when both): the values of
 * calc_stressfunc_fromCS/CD and calc_stressfunc_fromC_rowS/D
 * (src/Hmatrix.py:318-511). */
void td_stress_hs(const double obs[3], const double P1[3], const double P2[3], const double P3[3],
                  double Ss, double Ds, double Ts, double mu, double lam, int mode,
                  double stress[6], double strain[6]);

void td_traction_block(const double *xg, const double *ev, const double *nodes, const long *tri,
                       const long *rows, size_t m, const long *cols, size_t n,
                       double mu, double lam, int which, int hs_mode, double *out)
{
    int modes[2], nm = 0;
    if (which & 1) modes[nm++] = 0;
    if (which & 2) modes[nm++] = 1;
    for (size_t j = 0; j < n; ++j) {
        long e = cols[j];
        const double *P1 = nodes + 3 * (tri[3 * e + 0] - 1);
        const double *P2 = nodes + 3 * (tri[3 * e + 1] - 1);
        const double *P3 = nodes + 3 * (tri[3 * e + 2] - 1);
        for (size_t i = 0; i < m; ++i) {
            long r = rows[i];
            double s[6], t[3];
            for (int q = 0; q < nm; ++q) {
                int slip = modes[q];
                if (hs_mode)
                    td_stress_hs(xg + 3 * r, P1, P2, P3, slip == 0 ? 1.0 : 0.0, slip == 0 ? 0.0 : 1.0, 0.0,
                                 mu, lam, hs_mode, s, 0);
                else
                    td_stress_fs(xg + 3 * r, P1, P2, P3, slip == 0 ? 1.0 : 0.0, slip == 0 ? 0.0 : 1.0, 0.0,
                                 mu, lam, s, 0);
                td_traction(s, ev + 9 * r, t);
                for (int c = 0; c < 3; ++c) out[(size_t)(3 * q + c) * m * n + i * n + j] = t[c];
            }
        }
    }
}

/* ================================================================ half space
 * TDstressHS of the reference (src/TDstressFS_C.cpp:1911-2000, numpy twin
 * src/SH_greenfunction.py:861-888): main dislocation (full space) + image
 * dislocation (vertices mirrored to z > 0; xz, yz terms negated when all three
 * vertices lie on z = 0) + free-surface correction of the three angular
 * dislocation pairs along the sides (TDstress_HarFunc :1766-1908, AngSetupFSC_S
 * :1489-1763).
 *
 * Free-surface correction: instead of the expanded strain expressions of
 * AngDisStrainFSC (:613-1486), the strain is obtained by forward-mode
 * differentiation (dual numbers in y1, y2, y3) of the nine displacement terms
 * u_i(b_k) of the angular-dislocation harmonic correction (Comninou & Dundurs
 * 1975; Nikkhoo & Walter 2015), whose y-derivatives are the reference's strain
 * expressions; the Burgers function enters only through its gradient, given in
 * closed form.
 *
 * mode 1: a side along z contributes nothing (numpy twin, :743-746).
 * mode 2: as the compiled C++ path: such a side repeats the contribution of the
 *         side computed before it in the same call (its output vectors are left
 *         untouched, :1517-1522), none if it is the first side. */
typedef struct { double v, d[3]; } dual;

static dual dl(double v, double d0, double d1, double d2) { dual r = {v, {d0, d1, d2}}; return r; }
static dual dc(double v) { return dl(v, 0, 0, 0); }
static dual dadd(dual a, dual b) { return dl(a.v + b.v, a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]); }
static dual dsub(dual a, dual b) { return dl(a.v - b.v, a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]); }
static dual dmul(dual a, dual b)
{
    return dl(a.v * b.v, a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]);
}
static dual dscl(dual a, double s) { return dl(a.v * s, a.d[0] * s, a.d[1] * s, a.d[2] * s); }
static dual dads(dual a, double s) { return dl(a.v + s, a.d[0], a.d[1], a.d[2]); }
static dual ddiv(dual a, dual b)
{
    double ib = 1.0 / b.v, v = a.v * ib;
    return dl(v, (a.d[0] - v * b.d[0]) * ib, (a.d[1] - v * b.d[1]) * ib, (a.d[2] - v * b.d[2]) * ib);
}
static dual dinv(dual b) { return ddiv(dc(1.0), b); }
static dual dsqrtd(dual a)
{
    double v = sqrt(a.v), h = 0.5 / v;
    return dl(v, a.d[0] * h, a.d[1] * h, a.d[2] * h);
}
static dual dlogd(dual a) { return dl(log(a.v), a.d[0] / a.v, a.d[1] / a.v, a.d[2] / a.v); }

/* Strain basis (ADCS, components 11 22 33 12 13 23) of the free-surface
 * correction of one angular dislocation at (y1, y2, y3), for unit b1, b2, b3:
 * out[k][6].  sB, cB, ctB: sin, cos, cot of the angle; a: depth parameter. */
static void fsc_basis(double y1v, double y2v, double y3v, double sB, double cB, double ctB, double nu, double a,
                      double out[3][6])
{
    const double y3bv = y3v + 2 * a;
    const double rr = y1v * y1v + y2v * y2v + y3bv * y3bv;
    if (sqrt(rr) < 1e-12) {
        for (int k = 0; k < 3; ++k) for (int c = 0; c < 6; ++c) out[k][c] = 0.0;
        return;
    }
    const dual y1 = dl(y1v, 1, 0, 0), y2 = dl(y2v, 0, 1, 0), y3 = dl(y3v, 0, 0, 1);
    const double N1 = 1 - 2 * nu, t2 = 2 * (1 - nu);
    const dual y3b = dads(y3, 2 * a);
    const dual z1b = dadd(dscl(y1, cB), dscl(y3b, sB));
    const dual z3b = dadd(dscl(y1, -sB), dscl(y3b, cB));
    const dual rb = dsqrtd(dadd(dadd(dmul(y1, y1), dmul(y2, y2)), dmul(y3b, y3b)));
    const dual irb = dinv(rb), rb2 = dmul(rb, rb), irb2 = dmul(irb, irb), irb3 = dmul(irb2, irb);
    const dual ar = dscl(irb, a);                                  /* a / rb */
    const dual W1 = dadd(dscl(rb, cB), y3b);
    const dual W2 = dads(ar, cB), W4 = dads(ar, nu), W5 = dads(ar, 2 * nu);
    const dual W6 = dadd(rb, y3b), W7 = dadd(rb, z3b), W8 = dads(y3, a);
    const dual W9 = dads(dscl(irb, a / cB), 1.0);
    const dual iW6 = dinv(W6), iW7 = dinv(W7);
    const dual lW6 = dlogd(W6), lW7 = dlogd(W7);
    /* gradient of the Burgers function (value irrelevant: it enters linearly) */
    const double r = rb.v, Y3b = y3b.v, Z3b = z3b.v, Z1b = z1b.v;
    const dual Fib = dl(0.0, y2v / (r * (r + Y3b)) - cB * y2v / (r * (r + Z3b)),
                        Z1b / (r * (r + Z3b)) - y1v / (r * (r + Y3b)), -sB * y2v / (r * (r + Z3b)));
    const dual ay3br2 = dmul(dscl(y3b, a), irb2);                    /* a y3b / rb^2 */
    const dual rsBy1 = dsub(dscl(rb, sB), y1);                       /* rb sin - y1 */
    dual U[3][3];
    /* u1 */
    U[0][0] = dadd(dadd(dadd(dscl(Fib, -t2 * N1 * ctB * ctB),
                             dmul(dscl(dmul(y2, iW6), N1), dsub(dscl(dads(dscl(W5, -1.0), 1.0), ctB), dmul(dmul(y1, W4), iW6)))),
                        dadd(dscl(dmul(dmul(y2, W2), iW7), N1 * cB * ctB), dscl(dmul(dmul(y2, W8), irb3), a * ctB))),
                   dadd(dmul(dmul(dmul(y2, W8), dmul(irb, iW6)),
                             dadd(dadd(dc(-N1 * ctB), dmul(dmul(y1, W5), iW6)), dmul(dscl(y1, a), irb2))),
                        dmul(dmul(dmul(y2, W8), dmul(irb, iW7)),
                             dsub(dscl(dmul(iW7, dadd(dscl(dmul(W1, dads(dscl(ar, -1.0), N1 * cB)), ctB), dscl(rsBy1, t2 * cB))), cB),
                                  dscl(ay3br2, cB * ctB)))));
    U[0][1] = dadd(dadd(dadd(dscl(dsub(dscl(lW6, t2 * ctB * ctB + nu), dscl(lW7, (t2 * ctB * ctB + 1) * cB)), N1),
                             dscl(dmul(iW6, dadd(dadd(dscl(y1, -N1 * ctB), dads(dscl(y3b, nu), -a)),
                                                 dadd(dmul(dscl(y1, a * ctB), irb), dmul(dmul(dmul(y1, y1), W4), iW6)))), N1)),
                        dadd(dscl(dmul(iW7, dsub(dscl(z1b, cB), dscl(dmul(rsBy1, irb), a / cB))), -N1 * ctB),
                             dscl(dmul(dmul(y1, W8), irb3), -a * ctB))),
                   dadd(dmul(dmul(W8, iW6), dsub(dsub(dadd(dc(2 * nu), dmul(dads(dscl(y1, N1 * ctB), a), irb)),
                                                      dmul(dmul(dmul(y1, y1), W5), dmul(irb, iW6))),
                                                 dmul(dscl(dmul(y1, y1), a), irb3))),
                        dscl(dmul(dmul(W8, iW7), dadd(dadd(dc(-cB * sB), dscl(dmul(dmul(y1, y3b), irb3), a / cB)),
                                                      dmul(dmul(rsBy1, irb), dsub(dc(t2 * cB), dmul(dmul(W1, W9), iW7))))),
                             ctB)));
    U[0][2] = dadd(dscl(dsub(dmul(dmul(y2, dads(ar, 1.0)), iW6), dscl(dmul(dmul(y2, W2), iW7), cB)), N1),
                   dadd(dscl(dmul(dmul(dmul(y2, W8), irb), dadd(dscl(irb2, a), iW6)), -1.0),
                        dscl(dmul(dmul(dmul(y2, W8), dmul(irb, iW7)), dadd(dmul(dmul(W1, W2), iW7), ay3br2)), cB)));
    /* u2 */
    U[1][0] = dadd(dadd(dadd(dscl(dsub(dscl(lW6, t2 * ctB * ctB - nu), dscl(lW7, (t2 * ctB * ctB + 1 - 2 * nu) * cB)), N1),
                             dscl(dmul(iW6, dadd(dadd(dscl(dmul(y1, dads(dscl(W5, -1.0), 1.0)), ctB), dads(dscl(y3b, nu), -a)),
                                                 dmul(dmul(dmul(y2, y2), W4), iW6))), -N1)),
                        dadd(dscl(dmul(dmul(z1b, W2), iW7), -N1 * ctB), dscl(dmul(dmul(y1, W8), irb3), -a * ctB))),
                   dadd(dmul(dmul(W8, iW6), dadd(dadd(dc(-2 * nu), dmul(dads(dscl(y1, N1 * ctB), -a), irb)),
                                                 dadd(dmul(dmul(dmul(y2, y2), W5), dmul(irb, iW6)),
                                                      dmul(dscl(dmul(y2, y2), a), irb3)))),
                        dmul(dmul(W8, iW7),
                             dsub(dadd(dsub(dc(cB * cB), dmul(dads(dscl(z1b, N1 * ctB), a * cB), irb)),
                                       dmul(dscl(dmul(y3b, z1b), a * ctB), irb3)),
                                  dmul(dsub(dscl(dmul(y2, y2), cB * cB), dmul(dscl(dmul(z1b, W1), a * ctB), irb)),
                                       dmul(irb, iW7))))));
    U[1][1] = dadd(dadd(dadd(dscl(Fib, t2 * N1 * ctB * ctB),
                             dscl(dmul(dmul(y2, iW6), dadd(dscl(dads(W5, -1.0), ctB), dmul(dmul(y1, W4), iW6))), N1)),
                        dadd(dscl(dmul(dmul(y2, W9), iW7), -N1 * ctB), dscl(dmul(dmul(y2, W8), irb3), -a * ctB))),
                   dadd(dmul(dmul(dmul(y2, W8), dmul(irb, iW6)),
                             dsub(dsub(dc(N1 * ctB), dscl(dmul(y1, iW6), 2 * nu)),
                                  dmul(dmul(dscl(y1, a), irb), dadd(irb, iW6)))),
                        dscl(dmul(dmul(dmul(y2, W8), dmul(irb, iW7)),
                                  dadd(dadd(dc(-t2 * cB), dmul(dmul(W1, W9), iW7)), dscl(dmul(y3b, irb2), a / cB))),
                             ctB)));
    U[1][2] = dadd(dscl(dadd(dsub(dscl(lW7, -sB), dmul(dmul(y1, dads(ar, 1.0)), iW6)), dmul(dmul(z1b, W2), iW7)), N1),
                   dsub(dmul(dmul(dmul(y1, W8), irb), dadd(dscl(irb2, a), iW6)),
                        dmul(dmul(W8, iW7),
                             dsub(dadd(dscl(dads(dscl(ar, -1.0), cB), sB), dmul(dmul(z1b, irb), dads(ay3br2, 1.0))),
                                  dmul(dsub(dscl(dmul(y2, y2), cB * sB), dmul(dscl(dmul(z1b, W1), a), irb)),
                                       dmul(irb, iW7))))));
    /* u3 */
    U[2][0] = dadd(dscl(dadd(dscl(Fib, N1 * ctB), dsub(dmul(dmul(y2, W5), iW6), dscl(dmul(dmul(y2, W2), iW7), cB))), t2),
                   dadd(dmul(dmul(dmul(y2, W8), irb), dadd(dscl(iW6, 2 * nu), dscl(irb2, a))),
                        dscl(dmul(dmul(dmul(y2, W8), dmul(irb, iW7)),
                                  dsub(dsub(dc(1 - 2 * nu), dmul(dmul(W1, W2), iW7)), ay3br2)), cB)));
    U[2][1] = dadd(dadd(dscl(dsub(lW6, dscl(lW7, cB)), -t2 * N1 * ctB),
                        dadd(dscl(dmul(dmul(y1, W5), iW6), -t2), dscl(dmul(dmul(z1b, W2), iW7), t2))),
                   dsub(dmul(dmul(W8, irb), dsub(dsub(dc(N1 * ctB), dscl(dmul(y1, iW6), 2 * nu)), dmul(dscl(y1, a), irb2))),
                        dmul(dmul(W8, iW7),
                             dadd(dadd(dc(cB * sB),
                                       dmul(dscl(dmul(W1, irb), ctB), dsub(dc(t2 * cB), dmul(W1, iW7)))),
                                  dmul(dscl(irb, a),
                                       dsub(dsub(dc(sB), dmul(dmul(y3b, z1b), irb2)),
                                            dmul(dmul(z1b, W1), dmul(irb, iW7))))))));
    U[2][2] = dadd(dscl(dadd(Fib, dscl(dmul(dmul(y2, W2), iW7), sB)), t2),
                   dscl(dmul(dmul(dmul(y2, W8), dmul(irb, iW7)), dadd(dads(dmul(dmul(W1, W2), iW7), 1.0), ay3br2)), sB));
    (void)rb2;
    const double c = 1.0 / (4.0 * TD_PI * (1.0 - nu));
    for (int k = 0; k < 3; ++k) {
        double G[3][3];
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) G[i][j] = c * U[i][k].d[j];
        out[k][0] = G[0][0];
        out[k][1] = G[1][1];
        out[k][2] = G[2][2];
        out[k][3] = 0.5 * (G[0][1] + G[1][0]);
        out[k][4] = 0.5 * (G[0][2] + G[2][0]);
        out[k][5] = 0.5 * (G[1][2] + G[2][1]);
    }
}

/* Free-surface correction strain (global frame) of the angular-dislocation pair
 * on side PA -> PB for Burgers vector B (global).  Returns 0 for a side along z. */
static int fsc_side(const double obs[3], const double PA[3], const double PB[3], const double B[3], double nu,
                    double e[6])
{
    const double sv[3] = {PB[0] - PA[0], PB[1] - PA[1], PB[2] - PA[2]};
    const double ns = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    const double beta = acos(-sv[2] / ns);
    for (int c = 0; c < 6; ++c) e[c] = 0.0;
    if (fabs(beta) < 2.2204e-16 || fabs(TD_PI - beta) < 2.2204e-16) return 0;
    const double nh = sqrt(sv[0] * sv[0] + sv[1] * sv[1]);
    const double ex = sv[0] / nh, ey = sv[1] / nh;
    /* side frame: ey1 = (ex, ey, 0), ey2 = ey3 x ey1 = (ey, -ex, 0), ey3 = (0, 0, -1) */
    const double F[3][3] = {{ex, ey, 0.0}, {ey, -ex, 0.0}, {0.0, 0.0, -1.0}};
    double yA[3], yAB[3], bv[3];
    const double d[3] = {obs[0] - PA[0], obs[1] - PA[1], obs[2] - PA[2]};
    for (int k = 0; k < 3; ++k) {
        yA[k] = F[k][0] * d[0] + F[k][1] * d[1] + F[k][2] * d[2];
        yAB[k] = F[k][0] * sv[0] + F[k][1] * sv[1] + F[k][2] * sv[2];
        bv[k] = F[k][0] * B[0] + F[k][1] * B[1] + F[k][2] * B[2];
    }
    const double yB[3] = {yA[0] - yAB[0], yA[1] - yAB[1], yA[2] - yAB[2]};
    double vA[6], vB[6], bA[3][6], bB[3][6];
    if (beta * yA[0] >= 0) {                 /* configuration I: mirrored pair, angle pi - beta */
        const double g = TD_PI - beta, s = sin(g), co = cos(g), ct = 1.0 / tan(g);
        const double b[3] = {-bv[0], -bv[1], bv[2]};
        fsc_basis(-yA[0], -yA[1], yA[2], s, co, ct, nu, -PA[2], bA);
        fsc_basis(-yB[0], -yB[1], yB[2], s, co, ct, nu, -PB[2], bB);
        for (int c = 0; c < 6; ++c) {
            vA[c] = b[0] * bA[0][c] + b[1] * bA[1][c] + b[2] * bA[2][c];
            vB[c] = b[0] * bB[0][c] + b[1] * bB[1][c] + b[2] * bB[2][c];
        }
        vA[4] = -vA[4]; vA[5] = -vA[5];
        vB[4] = -vB[4]; vB[5] = -vB[5];
    } else {
        const double s = sin(beta), co = cos(beta), ct = 1.0 / tan(beta);
        fsc_basis(yA[0], yA[1], yA[2], s, co, ct, nu, -PA[2], bA);
        fsc_basis(yB[0], yB[1], yB[2], s, co, ct, nu, -PB[2], bB);
        for (int c = 0; c < 6; ++c) {
            vA[c] = bv[0] * bA[0][c] + bv[1] * bA[1][c] + bv[2] * bA[2][c];
            vB[c] = bv[0] * bB[0][c] + bv[1] * bB[1][c] + bv[2] * bB[2][c];
        }
    }
    for (int c = 0; c < 6; ++c) e[c] = vB[c] - vA[c];
    tens_trans(e, F);
    return 1;
}

void td_stress_hs(const double obs[3], const double P1[3], const double P2[3], const double P3[3],
                  double Ss, double Ds, double Ts, double mu, double lam, int mode,
                  double stress[6], double strain[6])
{
    const double nu = 1.0 / (1.0 + lam / mu) / 2.0;
    double sm[6], em[6], si[6], ei[6];
    td_stress_fs(obs, P1, P2, P3, Ss, Ds, Ts, mu, lam, sm, em);
    const double Q1[3] = {P1[0], P1[1], -P1[2]}, Q2[3] = {P2[0], P2[1], -P2[2]}, Q3[3] = {P3[0], P3[1], -P3[2]};
    td_stress_fs(obs, Q1, Q2, Q3, Ss, Ds, Ts, mu, lam, si, ei);
    if (P1[2] == 0 && P2[2] == 0 && P3[2] == 0) { si[4] = -si[4]; si[5] = -si[5]; ei[4] = -ei[4]; ei[5] = -ei[5]; }
    /* Burgers vector in the global frame: (n, strike, dip) frame of TDstress_HarFunc */
    double vn[3], vs[3], vd[3];
    vn[0] = (P2[1] - P1[1]) * (P3[2] - P1[2]) - (P2[2] - P1[2]) * (P3[1] - P1[1]);
    vn[1] = (P2[2] - P1[2]) * (P3[0] - P1[0]) - (P2[0] - P1[0]) * (P3[2] - P1[2]);
    vn[2] = (P2[0] - P1[0]) * (P3[1] - P1[1]) - (P2[1] - P1[1]) * (P3[0] - P1[0]);
    double nn = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
    if (nn != 0) { vn[0] /= nn; vn[1] /= nn; vn[2] /= nn; }
    vs[0] = -vn[1]; vs[1] = vn[0]; vs[2] = 0.0;
    double ns = sqrt(vs[0] * vs[0] + vs[1] * vs[1]);
    if (ns == 0) { vs[0] = 0.0; vs[1] = vn[2]; vs[2] = 0.0; }
    else { vs[0] /= ns; vs[1] /= ns; }
    vd[0] = vn[1] * vs[2] - vn[2] * vs[1];
    vd[1] = vn[2] * vs[0] - vn[0] * vs[2];
    vd[2] = vn[0] * vs[1] - vn[1] * vs[0];
    double B[3];
    for (int k = 0; k < 3; ++k) B[k] = vn[k] * Ts + vs[k] * Ss + vd[k] * Ds;
    const double *V[4] = {P1, P2, P3, P1};
    double ef[6] = {0, 0, 0, 0, 0, 0}, prev[6] = {0, 0, 0, 0, 0, 0};
    int have_prev = 0;
    for (int k = 0; k < 3; ++k) {
        double e[6];
        if (fsc_side(obs, V[k], V[k + 1], B, nu, e)) {
            for (int c = 0; c < 6; ++c) prev[c] = e[c];
            have_prev = 1;
        } else if (mode == 2 && have_prev) {
            for (int c = 0; c < 6; ++c) e[c] = prev[c];
        }
        for (int c = 0; c < 6; ++c) ef[c] += e[c];
    }
    double sf[6];
    double tr = ef[0] + ef[1] + ef[2];
    for (int c = 0; c < 3; ++c) sf[c] = 2 * mu * ef[c] + lam * tr;
    for (int c = 3; c < 6; ++c) sf[c] = 2 * mu * ef[c];
    for (int c = 0; c < 6; ++c) {
        stress[c] = sm[c] + sf[c] + si[c];
        if (strain) strain[c] = em[c] + ef[c] + ei[c];
    }
}

/* One source triangle, n receivers, half space (mode as td_stress_hs). */
void td_stress_hs_batch(const double *X, const double *Y, const double *Z, size_t n,
                        const double *P1, const double *P2, const double *P3,
                        double Ss, double Ds, double Ts, double mu, double lam, int mode,
                        double *stress, double *strain)
{
    for (size_t i = 0; i < n; ++i) {
        double o[3] = {X[i], Y[i], Z[i]};
        td_stress_hs(o, P1, P2, P3, Ss, Ds, Ts, mu, lam, mode, stress + 6 * i, strain ? strain + 6 * i : 0);
    }
}

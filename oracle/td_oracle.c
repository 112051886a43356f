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
 * 3 both.  out holds 3 planes per computed mode of m*n doubles, row-major, in
 * the order A1, A2, B (strike first when both): the values of
 * calc_stressfunc_fromCS/CD and calc_stressfunc_fromC_rowS/D
 * (src/Hmatrix.py:318-511). */
void td_traction_block(const double *xg, const double *ev, const double *nodes, const long *tri,
                       const long *rows, size_t m, const long *cols, size_t n,
                       double mu, double lam, int which, double *out)
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
                td_stress_fs(xg + 3 * r, P1, P2, P3, slip == 0 ? 1.0 : 0.0, slip == 0 ? 0.0 : 1.0, 0.0,
                             mu, lam, s, 0);
                td_traction(s, ev + 9 * r, t);
                for (int c = 0; c < 3; ++c) out[(size_t)(3 * q + c) * m * n + i * n + j] = t[c];
            }
        }
    }
}

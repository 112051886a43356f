// Full-space triangular-dislocation (TD) stress, FP64 device code.
//
// Algorithm: Nikkhoo & Walter (2015) as implemented by the reference in
// src/TDstressFS_C.cpp: TDstressFS (:274-521) sums three angular dislocations
// (TDSetupS :185-256 -> AngDisStrain :51-121), picks the configuration with
// trimodefinder (:125-166), rotates back (TensTrans :21-49) and applies
// Hooke's law.  The traction projection on the receiver frame follows
// BlockTree.GetTtstress (src/Hmatrix.py:295-313).
//
// GPU layout: everything that depends only on the source triangle (TD frame,
// local vertices, unit side vectors, cos/sin of the three angles) is computed
// once per element into a SrcRec; a pair evaluation then only transforms the
// receiver.  Strain is linear in the Burgers vector, so each angular
// dislocation is evaluated once as a basis (unit by, unit bz [, unit bx]) and
// the strike-slip (Ss=1) and dip-slip (Ds=1) responses are combined from the
// same basis.  Quotients share four reciprocals per angular dislocation.
#pragma once
#include <math.h>

namespace pq3d {

constexpr double kPi = 3.141592653589793;

struct SrcRec {
    double vn[3], vs[3], vd[3];  // TD frame: normal, strike, dip (TDstressFS_C.cpp:297-333)
    double P2[3];                // origin of the TD coordinate system
    double p1[3], p3[3];         // vertices 1 and 3 in TD coordinates (vertex 2 is the origin)
    double e12[3], e13[3], e23[3];
    double cA[3], sA[3];         // cos/sin(-pi + angle) for the dislocations at p1, p2, p3
};

__host__ __device__ inline double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Per-source setup (TDstressFS_C.cpp:294-385).
__device__ inline void make_src_rec(const double *P1, const double *P2, const double *P3, SrcRec &s)
{
    double vn[3];
    vn[0] = (P2[1] - P1[1]) * (P3[2] - P1[2]) - (P2[2] - P1[2]) * (P3[1] - P1[1]);
    vn[1] = (P2[2] - P1[2]) * (P3[0] - P1[0]) - (P2[0] - P1[0]) * (P3[2] - P1[2]);
    vn[2] = (P2[0] - P1[0]) * (P3[1] - P1[1]) - (P2[1] - P1[1]) * (P3[0] - P1[0]);
    double nn = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
    vn[0] /= nn; vn[1] /= nn; vn[2] /= nn;
    double vs[3] = {-vn[1], vn[0], 0.0};
    double ns = sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
    // Horizontal TD: the reference replaces the strike by eY*n_z and still divides
    // by the zero norm (TDstressFS_C.cpp:318-325); the NaN it produces is kept.
    if (ns == 0) { vs[0] = 0.0 * vn[2]; vs[1] = vn[2]; vs[2] = 0.0 * vn[2]; }
    vs[0] /= ns; vs[1] /= ns; vs[2] /= ns;
    double vd[3] = {vn[1] * vs[2] - vn[2] * vs[1], vn[2] * vs[0] - vn[0] * vs[2], vn[0] * vs[1] - vn[1] * vs[0]};
    double d1[3] = {P1[0] - P2[0], P1[1] - P2[1], P1[2] - P2[2]};
    double d3[3] = {P3[0] - P2[0], P3[1] - P2[1], P3[2] - P2[2]};
    for (int j = 0; j < 3; ++j) {
        s.vn[j] = vn[j]; s.vs[j] = vs[j]; s.vd[j] = vd[j]; s.P2[j] = P2[j];
    }
    const double *ax[3] = {vn, vs, vd};
    for (int j = 0; j < 3; ++j) {
        s.p1[j] = ax[j][0] * d1[0] + ax[j][1] * d1[1] + ax[j][2] * d1[2];
        s.p3[j] = ax[j][0] * d3[0] + ax[j][1] * d3[1] + ax[j][2] * d3[2];
    }
    double e12[3], e13[3], e23[3];
    for (int j = 0; j < 3; ++j) { e12[j] = -s.p1[j]; e13[j] = s.p3[j] - s.p1[j]; e23[j] = s.p3[j]; }
    double n12 = sqrt(dot3(e12, e12)), n13 = sqrt(dot3(e13, e13)), n23 = sqrt(dot3(e23, e23));
    for (int j = 0; j < 3; ++j) {
        e12[j] /= n12; e13[j] /= n13; e23[j] /= n23;
        s.e12[j] = e12[j]; s.e13[j] = e13[j]; s.e23[j] = e23[j];
    }
    double angA = acos(dot3(e12, e13));
    double angB = acos((-e12[0]) * e23[0] + (-e12[1]) * e23[1] + (-e12[2]) * e23[2]);
    double angC = acos(dot3(e23, e13));
    double ang[3] = {angA, angB, angC};
    for (int k = 0; k < 3; ++k) {
        double a = -kPi + ang[k];
        s.cA[k] = cos(a);
        s.sA[k] = sin(a);
    }
}

// Configuration of a TD-frame point (trimodefinder, TDstressFS_C.cpp:125-166).
__device__ inline int td_trimode(const double *X, const SrcRec &s)
{
    double x1 = s.p1[1], x2 = 0.0, x3 = s.p3[1];
    double y1 = s.p1[2], y2 = 0.0, y3 = s.p3[2];
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

// Rotate a symmetric tensor (xx,yy,zz,xy,xz,yz) by A: t' = A^T t A (TensTrans).
__device__ inline void tens_trans(double *t, const double A[3][3])
{
    double xx = t[0], yy = t[1], zz = t[2], xy = t[3], xz = t[4], yz = t[5];
    double o[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const int i = (c == 0 || c == 3 || c == 4) ? 0 : (c == 1 || c == 5) ? 1 : 2;
        const int j = (c == 0) ? 0 : (c == 1 || c == 3) ? 1 : 2;
        o[c] = A[0][i] * A[0][j] * xx + (A[0][i] * A[1][j] + A[0][j] * A[1][i]) * xy
             + (A[0][i] * A[2][j] + A[0][j] * A[2][i]) * xz
             + (A[2][j] * A[1][i] + A[2][i] * A[1][j]) * yz
             + A[1][j] * A[1][i] * yy + A[2][i] * A[2][j] * zz;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) t[c] = o[c];
}

// Strain basis of one angular dislocation at (x, y, z): Fy for unit by, Fz for
// unit bz and, when WITH_X, Fx for unit bx (AngDisStrain, TDstressFS_C.cpp:51-121).
template <bool WITH_X>
__device__ inline void ang_dis_basis(double x, double y, double z, double cA, double sA, double nu,
                                     double *Fx, double *Fy, double *Fz)
{
    double eta = y * cA - z * sA;
    double zeta = y * sA + z * cA;
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double r2 = x2 + y2 + z2;
    double r = sqrt(r2);
    double W = zeta - r;
    double ir = 1.0 / r;
    double iW = 1.0 / W;
    double irz = 1.0 / (r - z);      // 1/(r-z)
    double irzeta = 1.0 / (r - zeta);
    double ir2 = ir * ir;
    double iWr = iW * ir;            // 1/(W r)
    double iW2 = iW * iW;
    double iW2r = iW2 * ir;
    double iW2r2 = iWr * iWr;
    double iWr3 = iWr * ir2;
    double ir3 = ir2 * ir;
    double iRz = ir * irz;           // 1/(r (r-z))
    double iR2z2 = iRz * iRz;        // 1/(r^2 (r-z)^2)
    double iR3z = iRz * ir2;         // 1/(r^3 (r-z))
    double C = (r * cA - z) * iWr;
    double S = (r * sA - y) * iWr;
    const double k = 1.0 / (8.0 * kPi * (1 - nu));
    const double fq = 1.0 / (4.0 * kPi);
    double rFi_rx = (eta * ir * irzeta - y * iRz) * fq;
    double rFi_ry = (x * iRz - cA * x * ir * irzeta) * fq;
    double rFi_rz = (sA * x * ir * irzeta) * fq;
    double tnu = 2 * nu + 1;

    double Q1 = tnu * iWr + x2 * iW2r2 - x2 * iWr3;
    double P1 = Q1 * cA + tnu * iRz - x2 * iR2z2 - x2 * iR3z;
    double Q2 = iWr + S * S - y2 * iWr3;
    double P2 = iRz - y2 * iR2z2 - y2 * iR3z + Q2 * cA;
    double Q3 = iWr + C * C - z2 * iWr3;
    double P3 = Q3 * cA + z * ir3;
    double P4 = x2 * y * iR2z2 - nu * y * iRz + x2 * y * iR3z + nu * cA * S + x2 * y * cA * iWr3 + x2 * cA * S * iWr;
    double Q4 = nu * S + x2 * S * iWr + x2 * y * iWr3;
    double P5 = -x2 * ir3 + nu * ir + nu * cA * C + x2 * z * cA * iWr3 + x2 * cA * C * iWr;
    double Q5 = nu * C + x2 * C * iWr + x2 * z * iWr3;
    double ycs = y * cA + z * sA;
    double P6 = y * ir3 + sA * cA * cA * iW2 - cA * ycs * iW2r + y * z * cA * iW2r2 - y * z * cA * iWr3;
    double Q6 = y * z * iWr3 - sA * cA * iW2 + ycs * iW2r - y * z * iW2r2;
    double kx = k * x, kxs = k * x * sA, ks = k * sA;

    Fy[0] = -kx * P1;
    Fy[1] = rFi_ry - kx * P2;
    Fy[2] = -kx * P3;
    Fy[3] = rFi_rx * 0.5 + k * P4;
    Fy[4] = k * P5;
    Fy[5] = rFi_rz * 0.5 - kx * P6;

    Fz[0] = kxs * Q1;
    Fz[1] = kxs * Q2;
    Fz[2] = rFi_rz + kxs * Q3;
    Fz[3] = -ks * Q4;
    Fz[4] = rFi_rx * 0.5 - ks * Q5;
    Fz[5] = rFi_ry * 0.5 - kxs * Q6;

    if (WITH_X) {
        Fx[0] = rFi_rx + k * (eta * iWr + eta * x2 * iW2r2 - eta * x2 * iWr3 + y * iRz - x2 * y * iR2z2 - x2 * y * iR3z);
        Fx[1] = k * (Q2 * eta + tnu * y * iRz - y2 * y * iR2z2 - y2 * y * iR3z - 2 * nu * cA * S);
        Fx[2] = k * (eta * iWr + eta * C * C - eta * z2 * iWr3 + y * z * ir3 + 2 * nu * sA * C);
        Fx[3] = rFi_ry * 0.5 - k * (x * y2 * iR2z2 - nu * x * iRz + x * y2 * iR3z - nu * x * cA * iWr + eta * x * S * iWr + eta * x * y * iWr3);
        Fx[4] = rFi_rz * 0.5 - k * (-x * y * ir3 + nu * x * sA * iWr + eta * x * C * iWr + eta * x * z * iWr3);
        Fx[5] = k * (y2 * ir3 - nu * ir - nu * cA * C + nu * sA * S + eta * sA * cA * iW2 - eta * ycs * iW2r + eta * y * z * iW2r2 - eta * y * z * iWr3);
    }
}

// Strain (TD frame) of NB Burgers vectors b[q] = (bx, by, bz) at TD-frame point X1.
// out[q][6] receives the strain rotated back to the global frame.
template <int NB, bool WITH_X>
__device__ inline void td_strain_multi(const double *X1, const SrcRec &s, double nu,
                                       const double (*b)[3], double (*out)[6])
{
#pragma unroll
    for (int q = 0; q < NB; ++q)
#pragma unroll
        for (int c = 0; c < 6; ++c) out[q][c] = 0.0;
    int m = td_trimode(X1, s);
    if (m != 0) {
        const double sg = (m == 1) ? 1.0 : -1.0;
#pragma unroll 1
        for (int ad = 0; ad < 3; ++ad) {
            double sv[3], tv1, tv2;
            if (ad == 0) { sv[1] = -sg * s.e13[1]; sv[2] = -sg * s.e13[2]; tv1 = s.p1[1]; tv2 = s.p1[2]; }
            else if (ad == 1) { sv[1] = sg * s.e12[1]; sv[2] = sg * s.e12[2]; tv1 = 0.0; tv2 = 0.0; }
            else { sv[1] = sg * s.e23[1]; sv[2] = sg * s.e23[2]; tv1 = s.p3[1]; tv2 = s.p3[2]; }
            const double A00 = sv[2], A01 = -sv[1], A10 = sv[1], A11 = sv[2];
            double ry = X1[1] - tv1, rz = X1[2] - tv2;
            double y1 = A00 * ry + A01 * rz;
            double z1 = A10 * ry + A11 * rz;
            double Fx[6], Fy[6], Fz[6];
            ang_dis_basis<WITH_X>(X1[0], y1, z1, s.cA[ad], s.sA[ad], nu, Fx, Fy, Fz);
            const double B[3][3] = {{1.0, 0.0, 0.0}, {0.0, A00, A01}, {0.0, A10, A11}};
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                double by1 = A00 * b[q][1] + A01 * b[q][2];
                double bz1 = A10 * b[q][1] + A11 * b[q][2];
                double e[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    e[c] = by1 * Fy[c] + bz1 * Fz[c];
                    if (WITH_X) e[c] += b[q][0] * Fx[c];
                }
                tens_trans(e, B);
#pragma unroll
                for (int c = 0; c < 6; ++c) out[q][c] += e[c];
            }
        }
    }
    const double R[3][3] = {{s.vn[0], s.vn[1], s.vn[2]}, {s.vs[0], s.vs[1], s.vs[2]}, {s.vd[0], s.vd[1], s.vd[2]}};
#pragma unroll
    for (int q = 0; q < NB; ++q) tens_trans(out[q], R);
}

__device__ inline void to_td_frame(const double *obs, const SrcRec &s, double *X1)
{
    double d[3] = {obs[0] - s.P2[0], obs[1] - s.P2[1], obs[2] - s.P2[2]};
    X1[0] = dot3(s.vn, d);
    X1[1] = dot3(s.vs, d);
    X1[2] = dot3(s.vd, d);
}

__device__ inline void hooke(const double *e, double mu, double lam, double *sig)
{
    double tr = e[0] + e[1] + e[2];
    sig[0] = 2 * mu * e[0] + lam * tr;
    sig[1] = 2 * mu * e[1] + lam * tr;
    sig[2] = 2 * mu * e[2] + lam * tr;
    sig[3] = 2 * mu * e[3];
    sig[4] = 2 * mu * e[4];
    sig[5] = 2 * mu * e[5];
}

// (tau1, tau2, sigma_n) of stress s on the receiver frame ev = (e1, e2, e3) row-major.
__device__ inline void traction(const double *s, const double *ev, double *t)
{
    double tr1 = s[0] * ev[6] + s[3] * ev[7] + s[4] * ev[8];
    double tr2 = s[3] * ev[6] + s[1] * ev[7] + s[5] * ev[8];
    double trn = s[4] * ev[6] + s[5] * ev[7] + s[2] * ev[8];
    t[0] = tr1 * ev[0] + tr2 * ev[1] + trn * ev[2];
    t[1] = tr1 * ev[3] + tr2 * ev[4] + trn * ev[5];
    t[2] = tr1 * ev[6] + tr2 * ev[7] + trn * ev[8];
}

// Tractions on receiver (centroid obs, frame ev) from unit strike slip (out[0..2])
// and unit dip slip (out[3..5]) on source s: one entry of A1s,A2s,Bs,A1d,A2d,Bd.
__device__ inline void gf_traction_sd(const double *obs, const double *ev, const SrcRec &s,
                                      double mu, double lam, double nu, double *out)
{
    double X1[3];
    to_td_frame(obs, s, X1);
    const double b[2][3] = {{0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    double e[2][6];
    td_strain_multi<2, false>(X1, s, nu, b, e);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        double sig[6];
        hooke(e[q], mu, lam, sig);
        traction(sig, ev, out + 3 * q);
    }
}

// Tractions for a single slip mode (0 = strike, 1 = dip): out[0..2] = (A1, A2, B).
__device__ inline void gf_traction_one(const double *obs, const double *ev, const SrcRec &s,
                                       double mu, double lam, double nu, int mode, double *out)
{
    double X1[3];
    to_td_frame(obs, s, X1);
    const double b[1][3] = {{0.0, mode == 0 ? 1.0 : 0.0, mode == 0 ? 0.0 : 1.0}};
    double e[1][6];
    td_strain_multi<1, false>(X1, s, nu, b, e);
    double sig[6];
    hooke(e[0], mu, lam, sig);
    traction(sig, ev, out);
}

}  // namespace pq3d

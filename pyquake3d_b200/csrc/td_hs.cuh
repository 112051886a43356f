// Half-space triangular-dislocation stress, FP64 device code.
//
// TDstressHS of the reference (src/TDstressFS_C.cpp:1911-2000): the full-space
// solution of the triangle, of its image (vertices mirrored to z > 0; the
// image's xz, yz terms change sign when all three vertices lie on z = 0), and
// the free-surface correction of the three angular-dislocation pairs along its
// sides (TDstress_HarFunc :1766-1908, AngSetupFSC_S :1489-1763).
//
// The free-surface correction strain is computed by forward-mode
// differentiation: the nine displacement terms u_i(b_k) of the harmonic
// correction of an angular dislocation (Comninou & Dundurs 1975; Nikkhoo &
// Walter 2015) are evaluated on dual numbers carrying d/dy1, d/dy2, d/dy3, so one
// pass yields the 3 x 3 displacement gradient for each unit Burgers component;
// the strain is its symmetric part.  These derivatives are the strain terms of
// the reference's AngDisStrainFSC (:613-1486).  The Burgers function enters the
// displacement linearly, so only its gradient (closed form) is carried.
//
// Side handling (hs mode): 1 = a side along z adds no correction (numpy twin,
// src/SH_greenfunction.py:743-746); 2 = as the reference's compiled library,
// which leaves its output untouched for such a side, so the side repeats the
// correction of the side computed before it (none when it is the first side).
//
// GPU layout: everything that depends only on the source triangle (image TD
// record, per-side frame, side vector, angle terms of both configurations) is
// precomputed per element in an HsRec; a pair evaluation transforms the
// receiver into each side frame and evaluates two dual-number corrections per
// side (ends A and B).
#pragma once
#include "td_gf.cuh"

namespace pq3d {

struct HsSide {
    double PA[3];               // side start
    double ex, ey;              // side frame: ey1 = (ex, ey, 0), ey2 = (ey, -ex, 0), ey3 = (0, 0, -1)
    double yAB[3];              // side vector in the side frame
    double aA, aB;              // depth parameters -PA_z, -PB_z
    double sI, cI, ctI;         // sin, cos, cot of pi - beta (configuration I)
    double sN, cN, ctN;         // sin, cos, cot of beta      (configuration II)
    int vertical;               // side along z: no correction of its own
    int pad;
};

struct HsRec {
    SrcRec img;                 // image triangle
    HsSide side[3];             // P1P2, P2P3, P3P1
    int surface;                // all vertices on z = 0
    int pad;
};

__device__ inline void make_hs_rec(const double *P1, const double *P2, const double *P3, HsRec &h)
{
    const double Q1[3] = {P1[0], P1[1], -P1[2]}, Q2[3] = {P2[0], P2[1], -P2[2]}, Q3[3] = {P3[0], P3[1], -P3[2]};
    make_src_rec(Q1, Q2, Q3, h.img);
    h.surface = (P1[2] == 0 && P2[2] == 0 && P3[2] == 0) ? 1 : 0;
    h.pad = 0;
    const double *V[4] = {P1, P2, P3, P1};
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
        HsSide &S = h.side[k];
        const double *A = V[k], *B = V[k + 1];
        const double sv[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
        const double ns = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
        const double beta = acos(-sv[2] / ns);
        S.PA[0] = A[0]; S.PA[1] = A[1]; S.PA[2] = A[2];
        S.aA = -A[2];
        S.aB = -B[2];
        S.vertical = (fabs(beta) < 2.2204e-16 || fabs(kPi - beta) < 2.2204e-16) ? 1 : 0;
        S.pad = 0;
        const double nh = sqrt(sv[0] * sv[0] + sv[1] * sv[1]);
        S.ex = S.vertical ? 1.0 : sv[0] / nh;
        S.ey = S.vertical ? 0.0 : sv[1] / nh;
        S.yAB[0] = S.ex * sv[0] + S.ey * sv[1];
        S.yAB[1] = S.ey * sv[0] - S.ex * sv[1];
        S.yAB[2] = -sv[2];
        const double g = kPi - beta;
        S.sI = sin(g); S.cI = cos(g); S.ctI = 1.0 / tan(g);
        S.sN = sin(beta); S.cN = cos(beta); S.ctN = 1.0 / tan(beta);
    }
}

// ---------------------------------------------------------------- dual numbers in (y1, y2, y3)
struct Dual {
    double v, d0, d1, d2;
};
__device__ inline Dual dnum(double v, double a, double b, double c) { return Dual{v, a, b, c}; }
__device__ inline Dual dcst(double v) { return Dual{v, 0.0, 0.0, 0.0}; }
__device__ inline Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d0 + b.d0, a.d1 + b.d1, a.d2 + b.d2}; }
__device__ inline Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d0 - b.d0, a.d1 - b.d1, a.d2 - b.d2}; }
__device__ inline Dual operator+(Dual a, double s) { return Dual{a.v + s, a.d0, a.d1, a.d2}; }
__device__ inline Dual operator+(double s, Dual a) { return a + s; }
__device__ inline Dual operator-(Dual a, double s) { return Dual{a.v - s, a.d0, a.d1, a.d2}; }
__device__ inline Dual operator-(double s, Dual a) { return Dual{s - a.v, -a.d0, -a.d1, -a.d2}; }
__device__ inline Dual operator*(Dual a, double s) { return Dual{a.v * s, a.d0 * s, a.d1 * s, a.d2 * s}; }
__device__ inline Dual operator*(double s, Dual a) { return a * s; }
__device__ inline Dual operator*(Dual a, Dual b)
{
    return Dual{a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1, a.d2 * b.v + a.v * b.d2};
}
__device__ inline Dual inv(Dual b)
{
    const double i = 1.0 / b.v, i2 = -i * i;
    return Dual{i, b.d0 * i2, b.d1 * i2, b.d2 * i2};
}
__device__ inline Dual dsqrt(Dual a)
{
    const double v = sqrt(a.v), h = 0.5 / v;
    return Dual{v, a.d0 * h, a.d1 * h, a.d2 * h};
}
__device__ inline Dual dlog(Dual a)
{
    const double i = 1.0 / a.v;
    return Dual{log(a.v), a.d0 * i, a.d1 * i, a.d2 * i};
}

// Strain basis (side frame; 11 22 33 12 13 23) of the free-surface correction
// of one angular dislocation at (y1, y2, y3) for unit b1, b2, b3: out[k][6].
// s, c, ct: sin, cos, cot of the angle; a: depth parameter.
__device__ inline void fsc_basis(double y1v, double y2v, double y3v, double sB, double cB, double ctB, double nu,
                                 double a, double out[3][6])
{
    const double y3bv = y3v + 2 * a;
    if (sqrt(y1v * y1v + y2v * y2v + y3bv * y3bv) < 1e-12) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int c = 0; c < 6; ++c) out[k][c] = 0.0;
        return;
    }
    const Dual y1 = dnum(y1v, 1, 0, 0), y2 = dnum(y2v, 0, 1, 0), y3 = dnum(y3v, 0, 0, 1);
    const double N1 = 1 - 2 * nu, t2 = 2 * (1 - nu);
    const Dual y3b = y3 + 2 * a;
    const Dual z1b = y1 * cB + y3b * sB;
    const Dual z3b = y3b * cB - y1 * sB;
    const Dual rb = dsqrt(y1 * y1 + y2 * y2 + y3b * y3b);
    const Dual irb = inv(rb), irb2 = irb * irb, irb3 = irb2 * irb;
    const Dual ar = irb * a;                                     // a / rb
    const Dual W1 = rb * cB + y3b, W2 = ar + cB, W4 = ar + nu, W5 = ar + 2 * nu;
    const Dual W6 = rb + y3b, W7 = rb + z3b, W8 = y3 + a, W9 = irb * (a / cB) + 1.0;
    const Dual iW6 = inv(W6), iW7 = inv(W7), lW6 = dlog(W6), lW7 = dlog(W7);
    const double r = rb.v, Y3b = y3b.v, Z3b = z3b.v, Z1b = z1b.v;
    const Dual Fib = dnum(0.0, y2v / (r * (r + Y3b)) - cB * y2v / (r * (r + Z3b)),
                          Z1b / (r * (r + Z3b)) - y1v / (r * (r + Y3b)), -sB * y2v / (r * (r + Z3b)));
    const Dual ay3br2 = y3b * irb2 * a;                          // a y3b / rb^2
    const Dual rsB = rb * sB - y1;                               // rb sin - y1
    const Dual y2W8 = y2 * W8, rW6 = irb * iW6, rW7 = irb * iW7;
    const double ct2 = ctB * ctB;
    Dual U[3][3];
    // u1
    U[0][0] = Fib * (-t2 * N1 * ct2) + y2 * iW6 * N1 * ((1.0 - W5) * ctB - y1 * W4 * iW6)
            + y2 * W2 * iW7 * (N1 * cB * ctB) + y2W8 * irb3 * (a * ctB)
            + y2W8 * rW6 * (y1 * W5 * iW6 + y1 * irb2 * a - N1 * ctB)
            + y2W8 * rW7 * (iW7 * (W1 * (N1 * cB - ar) * ctB + rsB * (t2 * cB)) * cB - ay3br2 * (cB * ctB));
    U[0][1] = (lW6 * (t2 * ct2 + nu) - lW7 * ((t2 * ct2 + 1) * cB)) * N1
            + iW6 * (y1 * (-N1 * ctB) + y3b * nu - a + y1 * irb * (a * ctB) + y1 * y1 * W4 * iW6) * N1
            - iW7 * (z1b * cB - rsB * irb * (a / cB)) * (N1 * ctB) - y1 * W8 * irb3 * (a * ctB)
            + W8 * iW6 * (2 * nu + (y1 * (N1 * ctB) + a) * irb - y1 * y1 * W5 * rW6 - y1 * y1 * irb3 * a)
            + W8 * iW7 * (y1 * y3b * irb3 * (a / cB) - cB * sB + rsB * irb * (t2 * cB - W1 * W9 * iW7)) * ctB;
    U[0][2] = (y2 * (ar + 1.0) * iW6 - y2 * W2 * iW7 * cB) * N1 - y2W8 * irb * (irb2 * a + iW6)
            + y2W8 * rW7 * (W1 * W2 * iW7 + ay3br2) * cB;
    // u2
    U[1][0] = (lW6 * (t2 * ct2 - nu) - lW7 * ((t2 * ct2 + 1 - 2 * nu) * cB)) * N1
            - iW6 * (y1 * (1.0 - W5) * ctB + y3b * nu - a + y2 * y2 * W4 * iW6) * N1
            - z1b * W2 * iW7 * (N1 * ctB) - y1 * W8 * irb3 * (a * ctB)
            + W8 * iW6 * ((y1 * (N1 * ctB) - a) * irb - 2 * nu + y2 * y2 * W5 * rW6 + y2 * y2 * irb3 * a)
            + W8 * iW7 * (cB * cB - (z1b * (N1 * ctB) + a * cB) * irb + y3b * z1b * irb3 * (a * ctB)
                          - (y2 * y2 * (cB * cB) - z1b * W1 * irb * (a * ctB)) * rW7);
    U[1][1] = Fib * (t2 * N1 * ct2) + y2 * iW6 * ((W5 - 1.0) * ctB + y1 * W4 * iW6) * N1
            - y2 * W9 * iW7 * (N1 * ctB) - y2W8 * irb3 * (a * ctB)
            + y2W8 * rW6 * (N1 * ctB - y1 * iW6 * (2 * nu) - y1 * irb * (irb + iW6) * a)
            + y2W8 * rW7 * (W1 * W9 * iW7 + y3b * irb2 * (a / cB) - t2 * cB) * ctB;
    U[1][2] = (z1b * W2 * iW7 - lW7 * sB - y1 * (ar + 1.0) * iW6) * N1 + y1 * W8 * irb * (irb2 * a + iW6)
            - W8 * iW7 * ((cB - ar) * sB + z1b * irb * (ay3br2 + 1.0)
                          - (y2 * y2 * (cB * sB) - z1b * W1 * irb * a) * rW7);
    // u3
    U[2][0] = (Fib * (N1 * ctB) + y2 * W5 * iW6 - y2 * W2 * iW7 * cB) * t2
            + y2W8 * irb * (iW6 * (2 * nu) + irb2 * a) + y2W8 * rW7 * ((1 - 2 * nu) - W1 * W2 * iW7 - ay3br2) * cB;
    U[2][1] = (lW6 - lW7 * cB) * (-t2 * N1 * ctB) - y1 * W5 * iW6 * t2 + z1b * W2 * iW7 * t2
            + W8 * irb * (N1 * ctB - y1 * iW6 * (2 * nu) - y1 * irb2 * a)
            - W8 * iW7 * (cB * sB + W1 * irb * ctB * (t2 * cB - W1 * iW7)
                          + irb * a * (sB - y3b * z1b * irb2 - z1b * W1 * rW7));
    U[2][2] = (Fib + y2 * W2 * iW7 * sB) * t2 + y2W8 * rW7 * (W1 * W2 * iW7 + ay3br2 + 1.0) * sB;
    const double c = 1.0 / (4.0 * kPi * (1.0 - nu));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const Dual &a0 = U[0][k], &a1 = U[1][k], &a2 = U[2][k];
        out[k][0] = c * a0.d0;
        out[k][1] = c * a1.d1;
        out[k][2] = c * a2.d2;
        out[k][3] = 0.5 * c * (a0.d1 + a1.d0);
        out[k][4] = 0.5 * c * (a0.d2 + a2.d0);
        out[k][5] = 0.5 * c * (a1.d2 + a2.d1);
    }
}

// Free-surface correction strain (global frame) of one side for NB Burgers
// vectors B[q] (global frame): out[q][6].
template <int NB>
__device__ inline void fsc_side(const double *obs, const HsSide &S, double nu, const double (*B)[3],
                                double (*out)[6])
{
    const double F[3][3] = {{S.ex, S.ey, 0.0}, {S.ey, -S.ex, 0.0}, {0.0, 0.0, -1.0}};
    const double d[3] = {obs[0] - S.PA[0], obs[1] - S.PA[1], obs[2] - S.PA[2]};
    const double yA[3] = {S.ex * d[0] + S.ey * d[1], S.ey * d[0] - S.ex * d[1], -d[2]};
    const double yB[3] = {yA[0] - S.yAB[0], yA[1] - S.yAB[1], yA[2] - S.yAB[2]};
    const bool confI = yA[0] >= 0;            // beta * yA_x >= 0 with beta in (0, pi)
    double bA[3][6], bB[3][6];
    if (confI) {
        fsc_basis(-yA[0], -yA[1], yA[2], S.sI, S.cI, S.ctI, nu, S.aA, bA);
        fsc_basis(-yB[0], -yB[1], yB[2], S.sI, S.cI, S.ctI, nu, S.aB, bB);
    } else {
        fsc_basis(yA[0], yA[1], yA[2], S.sN, S.cN, S.ctN, nu, S.aA, bA);
        fsc_basis(yB[0], yB[1], yB[2], S.sN, S.cN, S.ctN, nu, S.aB, bB);
    }
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        double bv[3] = {S.ex * B[q][0] + S.ey * B[q][1], S.ey * B[q][0] - S.ex * B[q][1], -B[q][2]};
        if (confI) { bv[0] = -bv[0]; bv[1] = -bv[1]; }
        double e[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double vA = bv[0] * bA[0][c] + bv[1] * bA[1][c] + bv[2] * bA[2][c];
            const double vB = bv[0] * bB[0][c] + bv[1] * bB[1][c] + bv[2] * bB[2][c];
            e[c] = vB - vA;
        }
        if (confI) { e[4] = -e[4]; e[5] = -e[5]; }
        tens_trans(e, F);
#pragma unroll
        for (int c = 0; c < 6; ++c) out[q][c] = e[c];
    }
}

// Adds the image and free-surface terms of the half space to the full-space
// strain e[q] of source s at obs, for NB Burgers vectors b[q] = (bx, by, bz) in the
// source's TD frame.  mode: 1 or 2 (side handling, see above).
template <int NB, bool WITH_X>
__device__ inline void hs_add_strain(const double *obs, const SrcRec &s, const HsRec &h, double nu,
                                     const double (*b)[3], int mode, double (*e)[6])
{
    double X1[3];
    to_td_frame(obs, h.img, X1);
    double ei[NB][6];
    td_strain_multi<NB, WITH_X>(X1, h.img, nu, b, ei);
    const double sg = h.surface ? -1.0 : 1.0;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
#pragma unroll
        for (int c = 0; c < 4; ++c) e[q][c] += ei[q][c];
        e[q][4] += sg * ei[q][4];
        e[q][5] += sg * ei[q][5];
    }
    double B[NB][3];
#pragma unroll
    for (int q = 0; q < NB; ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) B[q][k] = s.vn[k] * b[q][0] + s.vs[k] * b[q][1] + s.vd[k] * b[q][2];
    double prev[NB][6];
    bool have_prev = false;
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
        if (h.side[k].vertical) {
            if (mode == 2 && have_prev)
#pragma unroll
                for (int q = 0; q < NB; ++q)
#pragma unroll
                    for (int c = 0; c < 6; ++c) e[q][c] += prev[q][c];
            continue;
        }
        fsc_side<NB>(obs, h.side[k], nu, B, prev);
        have_prev = true;
#pragma unroll
        for (int q = 0; q < NB; ++q)
#pragma unroll
            for (int c = 0; c < 6; ++c) e[q][c] += prev[q][c];
    }
}

// Half-space tractions on a receiver from unit strike (out[0..2]) and dip (out[3..5]) slip.
__device__ inline void gf_traction_sd_hs(const double *obs, const double *ev, const SrcRec &s, const HsRec &h,
                                         int mode, double mu, double lam, double nu, double *out)
{
    double X1[3];
    to_td_frame(obs, s, X1);
    const double b[2][3] = {{0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    double e[2][6];
    td_strain_multi<2, false>(X1, s, nu, b, e);
    hs_add_strain<2, false>(obs, s, h, nu, b, mode, e);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        double sig[6];
        hooke(e[q], mu, lam, sig);
        traction(sig, ev, out + 3 * q);
    }
}

// Half-space tractions for one slip mode (0 strike, 1 dip).
__device__ inline void gf_traction_one_hs(const double *obs, const double *ev, const SrcRec &s, const HsRec &h,
                                          int mode, double mu, double lam, double nu, int slip, double *out)
{
    double X1[3];
    to_td_frame(obs, s, X1);
    const double b[1][3] = {{0.0, slip == 0 ? 1.0 : 0.0, slip == 0 ? 0.0 : 1.0}};
    double e[1][6];
    td_strain_multi<1, false>(X1, s, nu, b, e);
    hs_add_strain<1, false>(obs, s, h, nu, b, mode, e);
    double sig[6];
    hooke(e[0], mu, lam, sig);
    traction(sig, ev, out);
}

}  // namespace pq3d

// excl.cuh — cylinder-cylinder excluded volume, CylinderExclVolRepulsion
// (Volume/CylinderExclVolRepulsion.cpp:330-882): the analytic integral of
// 1/r^4 over two segments and its gradient. The energy and force functions
// reproduce the reference's expression order for R = double. Pairs whose
// analytic result is non-finite are flagged for the quadrature fallback
// (excl_fallback.cu), as energyN/forceN are in the reference.
#pragma once

#include "device_math.cuh"
#include "dual.cuh"

namespace mb {

template <class R>
struct ExclS {
    R a, b, c, d, e, F, AA, BB, CC, DD, EE, FF, GG, HH, JJ, ATG1, ATG2, ATG3, ATG4;
};

template <class R>
__device__ __forceinline__ R atan_r(R x);
template <>
__device__ __forceinline__ double atan_r<double>(double x) { return atan(x); }
template <>
__device__ __forceinline__ float atan_r<float>(float x) { return atanf(x); }
template <>
__device__ __forceinline__ Dual atan_r<Dual>(Dual x) { return atan(x); }

// Scalars of the analytic integral, :360-410 / :643-690. Inputs are the four
// bead positions; all differences are formed in FP64.
template <class R, class P3 = V3>
__device__ __forceinline__ void excl_scalars(const P3& c1, const P3& c2, const P3& c3, const P3& c4, ExclS<R>& s) {
    T3<R> r12 = diff<R>(c1, c2);  // c2 - c1
    T3<R> r34 = diff<R>(c3, c4);  // c4 - c3
    T3<R> r31 = diff<R>(c3, c1);  // c1 - c3
    T3<R> r14 = diff<R>(c1, c4);  // c4 - c1
    T3<R> r32 = diff<R>(c3, c2);  // c2 - c3
    s.a = dot(r12, r12);
    s.b = dot(r34, r34);
    s.c = dot(r31, r31);
    s.d = dot(r12, r34);
    s.e = dot(r12, r31);
    s.F = dot(r34, r31);
    R g = dot(r12, r14);  // scalarProduct(c1, c2, c1, c4)
    R h = dot(r34, r32);  // scalarProduct(c3, c4, c3, c2)
    R I = dot(r34, r14);  // scalarProduct(c3, c4, c1, c4)
    // sqmagnitude(c1, c4) = |c1 - c4|^2 and sqmagnitude(c3, c2) = |c3 - c2|^2.
    R dx = R(c1.x - c4.x), dy = R(c1.y - c4.y), dz = R(c1.z - c4.z);
    R sqD = (dx * dx + dy * dy + dz * dz);
    dx = R(c3.x - c2.x);
    dy = R(c3.y - c2.y);
    dz = R(c3.z - c2.z);
    R sqE = (dx * dx + dy * dy + dz * dz);
    // vec_A = c1 - c2, vec_B = c3 - c4, vec_C = c3 - c1.
    T3<R> vA{R(c1.x - c2.x), R(c1.y - c2.y), R(c1.z - c2.z)};
    T3<R> vB{R(c3.x - c4.x), R(c3.y - c4.y), R(c3.z - c4.z)};
    T3<R> vC{R(c3.x - c1.x), R(c3.y - c1.y), R(c3.z - c1.z)};
    const R a = s.a, b = s.b, c = s.c, d = s.d, e = s.e, F = s.F;
    R ac = sqrt(a * c);
    R bc = sqrt(b * c);
    R aD = sqrt(a * sqD);
    R bE = sqrt(b * sqE);
    s.AA = sqrt(stdmax<R>(R(0), (ac + e) * (ac - e)));
    s.BB = sqrt(stdmax<R>(R(0), (bc + F) * (bc - F)));
    s.CC = d * e - a * F;
    s.DD = b * e - d * F;
    s.EE = sqrt(stdmax<R>(R(0), (aD + g) * (aD - g)));
    s.FF = sqrt(stdmax<R>(R(0), (bE + h) * (bE - h)));
    s.GG = d * g - a * I;
    s.HH = s.CC + s.GG - s.DD;
    R cpx = vA.y * vB.z - vA.z * vB.y;
    R cpy = vA.z * vB.x - vA.x * vB.z;
    R cpz = vA.x * vB.y - vA.y * vB.x;
    R JJ = cpx * vC.x + cpy * vC.y + cpz * vC.z;
    s.JJ = -JJ * JJ;
    s.ATG1 = atan_r<R>((a + e) / s.AA) - atan_r<R>(e / s.AA);
    s.ATG2 = atan_r<R>((a + e - d) / s.EE) - atan_r<R>((e - d) / s.EE);
    s.ATG3 = atan_r<R>((F) / s.BB) - atan_r<R>((F - b) / s.BB);
    s.ATG4 = atan_r<R>((d + F) / s.FF) - atan_r<R>((d + F - b) / s.FF);
}

// Analytic pair energy (:355 and :393-435). kRS = krep*L1*L2.
template <class R, class P3 = V3>
__device__ __forceinline__ R excl_energy_r(const P3& c1, const P3& c2, const P3& c3, const P3& c4, double kRS) {
    ExclS<R> s;
    excl_scalars<R, P3>(c1, c2, c3, c4, s);
    return R(0.5) * R(kRS) / s.JJ *
           (s.CC / s.AA * s.ATG1 + s.GG / s.EE * s.ATG2 + s.DD / s.BB * s.ATG3 + s.HH / s.FF * s.ATG4);
}
template <class R, class P3 = V3>
__device__ __forceinline__ double excl_energy(const P3& c1, const P3& c2, const P3& c3, const P3& c4, double kRS) {
    return double(excl_energy_r<R, P3>(c1, c2, c3, c4, kRS));
}

// The reference accepts an energy unless it is +-inf, NaN or below -1 (:447-449).
__device__ __forceinline__ bool excl_energy_bad(double U) { return isinf(U) || U != U || U < -1.0; }

// areInPlane (MathFunctions.h:1101-1133) and movePointOutOfPlane for bead 2 by
// d (:1221-1270), used by the force path (:610-626). FP64.
__device__ __forceinline__ bool in_plane(const V3& p1, const V3& p2, const V3& p3, const V3& p4) {
    double v1[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
    double v2[3] = {p3.x - p1.x, p3.y - p1.y, p3.z - p1.z};
    double v3[3] = {p4.x - p1.x, p4.y - p1.y, p4.z - p1.z};
    double cp[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
    double n1 = sqrt(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]);
    cp[0] = cp[0] / n1;
    cp[1] = cp[1] / n1;
    cp[2] = cp[2] / n1;
    double n3 = sqrt(v3[0] * v3[0] + v3[1] * v3[1] + v3[2] * v3[2]);
    v3[0] = v3[0] / n3;
    v3[1] = v3[1] / n3;
    v3[2] = v3[2] / n3;
    return fabs(v3[0] * cp[0] + v3[1] * cp[1] + v3[2] * cp[2]) < 1e-1;
}
__device__ __forceinline__ V3 move_bead2_out_of_plane(const V3& p1, const V3& p2, const V3& p3, double d) {
    double v1[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
    double v2[3] = {p3.x - p1.x, p3.y - p1.y, p3.z - p1.z};
    double n[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
    double m = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] = n[0] / m;
    n[1] = n[1] / m;
    n[2] = n[2] / m;
    return V3{p2.x + n[0] * d, p2.y + n[1] * d, p2.z + n[2] * d};
}
// Dual positions: the in-plane test on the values, the move on the duals.
__device__ __forceinline__ V3 value3(const DV3& p) { return V3{p.x.v, p.y.v, p.z.v}; }
__device__ __forceinline__ bool in_plane(const DV3& p1, const DV3& p2, const DV3& p3, const DV3& p4) {
    return in_plane(value3(p1), value3(p2), value3(p3), value3(p4));
}
__device__ __forceinline__ DV3 move_bead2_out_of_plane(const DV3& p1, const DV3& p2, const DV3& p3, double d) {
    const DV3 v1 = diff<Dual>(p1, p2), v2 = diff<Dual>(p1, p3);
    DV3 n{v1.y * v2.z - v1.z * v2.y, v1.z * v2.x - v1.x * v2.z, v1.x * v2.y - v1.y * v2.x};
    const Dual m = sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    n = DV3{n.x / m, n.y / m, n.z / m};
    return DV3{p2.x + n.x * d, p2.y + n.y * d, p2.z + n.z * d};
}

// checkNaN_INF (MathFunctions.h:1377-1384).
template <class R>
__device__ __forceinline__ bool bad_force(R x) {
    return isinf(x) || isnan(x) || fabs(double(x)) > 1e15;
}

// Analytic pair forces (:578-882), regrouped: the mixed-precision mode's
// form. Returns false when any component is non-finite or above 1e15 (the
// caller then uses the quadrature fallback).
//
// The kernel is bound by FP64 throughput, and division is the costliest FP64
// operation in the formula. The expression is the reference's, regrouped so
// that each of the four arctangent blocks (A: a,c,e; E: a,|c1-c4|^2,g;
// B: b,c,F; F: b,|c3-c2|^2,h) divides once for 1/Q and twice for its two
// weights, instead of about a dozen times (x/Q, x/Q^2, x/Q^3 become
// products with 1/Q). Results agree with the reference's order to a few
// ulps for most pairs, but near-parallel pairs amplify that to ~1e-8
// relative within the pair: well inside the mixed mode's 1e-6 force
// tolerance, outside the FP64 mode's 1e-12, which uses excl_force_exact.
template <class R>
struct ExclBlockF {
    R iQ, cN, cQ, cd, c1, T;  // 1/Q, the four coefficients, N/Q*ATG
};

template <class R>
__device__ __forceinline__ ExclBlockF<R> excl_force_block(R alpha, R beta, R gam, R u1, R u2, R N) {
    ExclBlockF<R> o;
    const R P = sqrt(alpha * beta);
    const R Q = sqrt(stdmax<R>(R(0), (P + gam) * (P - gam)));
    const R iQ = R(1) / Q;
    const R ATG = atan_r<R>(u1 * iQ) - atan_r<R>(u2 * iQ);
    const R Q2 = Q * Q, iQ2 = iQ * iQ;
    const R W1 = Q2 / (Q2 + u1 * u1);
    const R W2 = Q2 / (Q2 + u2 * u2);
    const R NiQ2 = N * iQ2;
    o.iQ = iQ;
    o.cN = ATG * iQ;
    o.cQ = -(ATG * NiQ2) + (-W1 * u1 + W2 * u2) * NiQ2 * iQ;
    o.cd = (W1 - W2) * NiQ2;
    o.c1 = W1 * NiQ2;
    o.T = N * iQ * ATG;
    return o;
}

template <class R>
__device__ __forceinline__ bool excl_force_fast(const V3& c1, V3 c2, const V3& c3, const V3& c4, double kRS,
                                           T3<R> (&fo)[4]) {
    if (in_plane(c1, c2, c3, c4)) c2 = move_bead2_out_of_plane(c1, c2, c3, 0.01);
    T3<R> r12 = diff<R>(c1, c2), r34 = diff<R>(c3, c4), r31 = diff<R>(c3, c1), r14 = diff<R>(c1, c4),
          r32 = diff<R>(c3, c2);
    const R a = dot(r12, r12), b = dot(r34, r34), c = dot(r31, r31);
    const R d = dot(r12, r34), e = dot(r12, r31), F = dot(r34, r31);
    const R g = dot(r12, r14), h = dot(r34, r32), I = dot(r34, r14);
    R dx = R(c1.x - c4.x), dy = R(c1.y - c4.y), dz = R(c1.z - c4.z);
    const R sqD = (dx * dx + dy * dy + dz * dz);
    dx = R(c3.x - c2.x);
    dy = R(c3.y - c2.y);
    dz = R(c3.z - c2.z);
    const R sqE = (dx * dx + dy * dy + dz * dz);
    T3<R> vA{R(c1.x - c2.x), R(c1.y - c2.y), R(c1.z - c2.z)};
    T3<R> vB{R(c3.x - c4.x), R(c3.y - c4.y), R(c3.z - c4.z)};
    T3<R> vC{R(c3.x - c1.x), R(c3.y - c1.y), R(c3.z - c1.z)};
    const R cpx = vA.y * vB.z - vA.z * vB.y;
    const R cpy = vA.z * vB.x - vA.x * vB.z;
    const R cpz = vA.x * vB.y - vA.y * vB.x;
    const R JJ0 = cpx * vC.x + cpy * vC.y + cpz * vC.z;
    const R JJ = -JJ0 * JJ0;
    const R CC = d * e - a * F, GG = d * g - a * I, DD = b * e - d * F, HH = CC + GG - DD;
    const ExclBlockF<R> A = excl_force_block<R>(a, c, e, a + e, e, CC);
    const ExclBlockF<R> E = excl_force_block<R>(a, sqD, g, a + e - d, e - d, GG);
    const ExclBlockF<R> B = excl_force_block<R>(b, c, F, F, F - b, DD);
    const ExclBlockF<R> Fb = excl_force_block<R>(b, sqE, h, d + F, d + F - b, HH);
    const R invJJ = R(1) / JJ;
    const R sumBlock = A.T + E.T + B.T + Fb.T;
    const R enFactor = R(kRS) * invJJ * R(0.5);
    // b_ij of the reference (:747-781) with x/Q written as x*(1/Q)
    const R b11 = A.cN * (-2 * F) + A.cQ * (c * A.iQ) + A.c1 * 2 + E.cN * (2 * (F - b)) +
                  E.cQ * ((b + c - 2 * F) * E.iQ) + E.c1 * 2 + Fb.cN * (-2 * b) + Fb.cQ * (b * Fb.iQ);
    const R b12 = A.cN * e + E.cN * (2 * d - e) + E.cQ * ((e - d) * E.iQ) - E.cd + B.cN * (-F) +
                  Fb.cN * (2 * d + F) + Fb.cQ * (-(d + F) * Fb.iQ) + Fb.cd;
    const R b13 = A.cN * d + A.cQ * (-e * A.iQ) + A.cd + E.cN * (-d) + E.cQ * (-(e - d) * E.iQ) + E.cd + B.cN * b +
                  Fb.cN * (-b) + Fb.cQ * (b * Fb.iQ);
    const R b22 = E.cN * (-2 * a) + E.cQ * (a * E.iQ) + B.cN * (2 * e) + B.cQ * (c * B.iQ) + B.cd * (-2) + B.c1 * 2 +
                  Fb.cN * (-2 * (a + e)) + Fb.cQ * ((a + c + 2 * e) * Fb.iQ) + Fb.cd * (-2) + Fb.c1 * 2;
    const R b23 = A.cN * (-a) + E.cN * a + E.cQ * (-a * E.iQ) + B.cN * (-d) + B.cQ * (-F * B.iQ) + B.cd + Fb.cN * d +
                  Fb.cQ * (-(d + F) * Fb.iQ) + Fb.cd;
    const R b33 = A.cQ * (a * A.iQ) + E.cQ * (a * E.iQ) + B.cQ * (b * B.iQ) + Fb.cQ * (b * Fb.iQ);
    const R b21 = b12, b31 = b13, b32 = b23;
    const R J11 = 2 * (-b * c + F * F), J12 = 2 * (c * d - e * F), J13 = 2 * (b * e - d * F);
    const R J21 = J12, J22 = 2 * (-a * c + e * e), J23 = 2 * (-d * e + a * F);
    const R J31 = J13, J32 = J23, J33 = 2 * (d * d - a * b);
    const R q = -invJJ * sumBlock;
    R dv[4][3];
    dv[0][0] = enFactor * (q * (J31 - J11) + (b31 - b11));
    dv[0][1] = enFactor * (q * (J32 - J12) + (b32 - b12));
    dv[0][2] = enFactor * (q * (J33 - J13) + (b33 - b13));
    dv[1][0] = enFactor * (q * (J11) + (b11));
    dv[1][1] = enFactor * (q * (J12) + (b12));
    dv[1][2] = enFactor * (q * (J13) + (b13));
    dv[2][0] = enFactor * (q * (-J31 - J21) + (-b31 - b21));
    dv[2][1] = enFactor * (q * (-J32 - J22) + (-b32 - b22));
    dv[2][2] = enFactor * (q * (-J33 - J23) + (-b33 - b23));
    dv[3][0] = enFactor * (q * (J21) + (b21));
    dv[3][1] = enFactor * (q * (J22) + (b22));
    dv[3][2] = enFactor * (q * (J23) + (b23));
    const T3<R> u = r12, v = r34, w = diff<R>(c3, c1);
    bool bad = false;
#pragma unroll
    for (int bi = 0; bi < 4; ++bi) {
        fo[bi].x = -(dv[bi][0] * u.x + dv[bi][1] * v.x + dv[bi][2] * w.x);
        fo[bi].y = -(dv[bi][0] * u.y + dv[bi][1] * v.y + dv[bi][2] * w.y);
        fo[bi].z = -(dv[bi][0] * u.z + dv[bi][1] * v.z + dv[bi][2] * w.z);
        bad |= bad_force(fo[bi].x) | bad_force(fo[bi].y) | bad_force(fo[bi].z);
    }
    return !bad;
}

// Analytic pair forces (:578-882) in the reference's expression order: the
// FP64 mode's form. Near-parallel pairs cancel heavily in the b_ij sums, so
// only the reference's own order keeps the forces within 1e-12 of it there
// (on the 400k-cylinder network one pair at cos 0.993 is 3e-8 relative off
// with any other grouping; the reference's own fast-math build is 1e-9 off).
// Returns false when any component is non-finite or above 1e15 (the caller
// then uses the quadrature fallback).
template <class R, class P3 = V3>
__device__ __forceinline__ bool excl_force_exact(const P3& c1, P3 c2, const P3& c3, const P3& c4, double kRS,
                                           T3<R> (&fo)[4]) {
    if (in_plane(c1, c2, c3, c4)) c2 = move_bead2_out_of_plane(c1, c2, c3, 0.01);
    ExclS<R> S;
    excl_scalars<R, P3>(c1, c2, c3, c4, S);
    const R a = S.a, b = S.b, c = S.c, d = S.d, e = S.e, F = S.F;
    const R AA = S.AA, BB = S.BB, CC = S.CC, DD = S.DD, EE = S.EE, FF = S.FF, GG = S.GG, HH = S.HH;
    const R JJ = S.JJ, ATG1 = S.ATG1, ATG2 = S.ATG2, ATG3 = S.ATG3, ATG4 = S.ATG4;
    const R invJJ = R(1) / JJ;
    const R sumBlock = CC / AA * ATG1 + GG / EE * ATG2 + DD / BB * ATG3 + HH / FF * ATG4;
    const R enFactor = R(kRS) * invJJ / R(2);
    const R A1 = AA * AA / (AA * AA + (a + e) * (a + e));
    const R A2 = AA * AA / (AA * AA + e * e);
    const R E1 = EE * EE / (EE * EE + (a + e - d) * (a + e - d));
    const R E2 = EE * EE / (EE * EE + (e - d) * (e - d));
    const R B1 = BB * BB / (BB * BB + F * F);
    const R B2 = BB * BB / (BB * BB + (F - b) * (F - b));
    const R F1 = FF * FF / (FF * FF + (d + F) * (d + F));
    const R F2 = FF * FF / (FF * FF + (d + F - b) * (d + F - b));
    const R bA_C = ATG1 / AA;
    const R bA_A = -(ATG1 * CC) / (AA * AA) + (-A1 * (a + e) + A2 * e) * CC / (AA * AA * AA);
    const R bA_e = ((A1 - A2) * CC) / (AA * AA);
    const R bA_a = (A1 * CC) / (AA * AA);
    const R bE_G = ATG2 / EE;
    const R bE_E = -(ATG2 * GG) / (EE * EE) + (-E1 * (a + e - d) + E2 * (e - d)) * GG / (EE * EE * EE);
    const R bE_emd = ((E1 - E2) * GG) / (EE * EE);
    const R bE_a = (E1 * GG) / (EE * EE);
    const R bB_D = ATG3 / BB;
    const R bB_B = -(ATG3 * DD) / (BB * BB) + (-B1 * F + B2 * (F - b)) * DD / (BB * BB * BB);
    const R bB_fmb = ((B1 - B2) * DD) / (BB * BB);
    const R bB_b = (B1 * DD) / (BB * BB);
    const R bF_H = ATG4 / FF;
    const R bF_F = -(ATG4 * HH) / (FF * FF) + (-F1 * (d + F) + F2 * (d + F - b)) * HH / (FF * FF * FF);
    const R bF_dpfmb = ((F1 - F2) * HH) / (FF * FF);
    const R bF_b = (F1 * HH) / (FF * FF);
    const R b11 = bA_C * (-2 * F) + bA_A * (c / AA) + bA_a * 2 + bE_G * (2 * (F - b)) + bE_E * ((b + c - 2 * F) / EE) +
                  bE_a * 2 + bF_H * (-2 * b) + bF_F * (b / FF);
    const R b12 = bA_C * e + bE_G * (2 * d - e) + bE_E * ((e - d) / EE) + bE_emd * (-1) + bB_D * (-F) +
                  bF_H * (2 * d + F) + bF_F * (-(d + F) / FF) + bF_dpfmb;
    const R b13 = bA_C * d + bA_A * (-e / AA) + bA_e + bE_G * (-d) + bE_E * (-(e - d) / EE) + bE_emd + bB_D * b +
                  bF_H * (-b) + bF_F * (b / FF);
    const R b21 = b12;
    const R b22 = bE_G * (-2 * a) + bE_E * (a / EE) + bB_D * (2 * e) + bB_B * (c / BB) + bB_fmb * (-2) + bB_b * 2 +
                  bF_H * (-2 * (a + e)) + bF_F * ((a + c + 2 * e) / FF) + bF_dpfmb * (-2) + bF_b * 2;
    const R b23 = bA_C * (-a) + bE_G * a + bE_E * (-a / EE) + bB_D * (-d) + bB_B * (-F / BB) + bB_fmb + bF_H * d +
                  bF_F * (-(d + F) / FF) + bF_dpfmb;
    const R b31 = b13;
    const R b32 = b23;
    const R b33 = bA_A * (a / AA) + bE_E * (a / EE) + bB_B * (b / BB) + bF_F * (b / FF);
    const R J11 = 2 * (-b * c + F * F), J12 = 2 * (c * d - e * F), J13 = 2 * (b * e - d * F);
    const R J21 = 2 * (c * d - e * F), J22 = 2 * (-a * c + e * e), J23 = 2 * (-d * e + a * F);
    const R J31 = 2 * (b * e - d * F), J32 = 2 * (-d * e + a * F), J33 = 2 * (d * d - a * b);
    const R q = -invJJ * sumBlock;
    R dv[4][3];
    dv[0][0] = enFactor * (q * (J31 - J11) + (b31 - b11));
    dv[0][1] = enFactor * (q * (J32 - J12) + (b32 - b12));
    dv[0][2] = enFactor * (q * (J33 - J13) + (b33 - b13));
    dv[1][0] = enFactor * (q * (J11) + (b11));
    dv[1][1] = enFactor * (q * (J12) + (b12));
    dv[1][2] = enFactor * (q * (J13) + (b13));
    dv[2][0] = enFactor * (q * (-J31 - J21) + (-b31 - b21));
    dv[2][1] = enFactor * (q * (-J32 - J22) + (-b32 - b22));
    dv[2][2] = enFactor * (q * (-J33 - J23) + (-b33 - b23));
    dv[3][0] = enFactor * (q * (J21) + (b21));
    dv[3][1] = enFactor * (q * (J22) + (b22));
    dv[3][2] = enFactor * (q * (J23) + (b23));
    const T3<R> u = diff<R>(c1, c2), v = diff<R>(c3, c4), w = diff<R>(c3, c1);
    bool bad = false;
#pragma unroll
    for (int bi = 0; bi < 4; ++bi) {
        fo[bi].x = -(dv[bi][0] * u.x + dv[bi][1] * v.x + dv[bi][2] * w.x);
        fo[bi].y = -(dv[bi][0] * u.y + dv[bi][1] * v.y + dv[bi][2] * w.y);
        fo[bi].z = -(dv[bi][0] * u.z + dv[bi][1] * v.z + dv[bi][2] * w.z);
        bad |= bad_force(fo[bi].x) | bad_force(fo[bi].y) | bad_force(fo[bi].z);
    }
    return !bad;
}

// The form each precision mode uses: FP64 the reference's order, mixed the
// regrouped one.
template <bool EXACT>
__device__ __forceinline__ bool excl_force(const V3& c1, const V3& c2, const V3& c3, const V3& c4, double kRS,
                                           T3<double> (&fo)[4]) {
    if constexpr (EXACT) return excl_force_exact<double>(c1, c2, c3, c4, kRS, fo);
    else return excl_force_fast<double>(c1, c2, c3, c4, kRS, fo);
}

}  // namespace mb

/*
 * medyan_oracle.c — CPU restatement (FP64) of MEDYAN's mechanical-equilibration
 * path. TEST INFRASTRUCTURE ONLY: it checks the CUDA library in tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py; the product
 * never links or calls it.
 *
 * Each function restates the reference code at the cited file:line (paths
 * relative to the reference's src/), keeping its operation order. Built with
 * -ffp-contract=off so every expression rounds as written.
 */
#define _DEFAULT_SOURCE /* M_PI */
#include "medyan_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- helpers */
/* mathfunc::scalarProduct(v1, v2, v3, v4), MathFunctions.h:469-478. */
static inline double sp4(const double* v1, const double* v2, const double* v3, const double* v4) {
    return (v2[0] - v1[0]) * (v4[0] - v3[0]) + (v2[1] - v1[1]) * (v4[1] - v3[1]) +
           (v2[2] - v1[2]) * (v4[2] - v3[2]);
}
/* mathfunc::twoPointDistance, MathFunctions.h:294-298. */
static inline double tpd(const double* v1, const double* v2) {
    return sqrt((v2[0] - v1[0]) * (v2[0] - v1[0]) + (v2[1] - v1[1]) * (v2[1] - v1[1]) +
                (v2[2] - v1[2]) * (v2[2] - v1[2]));
}
/* mathfunc::midPointCoordinate (array template), MathFunctions.h:963-969. */
static inline void midpt(double* v, const double* v1, const double* v2, double alpha) {
    double beta = 1 - alpha;
    v[0] = (v1[0] * beta + alpha * v2[0]);
    v[1] = (v1[1] * beta + alpha * v2[1]);
    v[2] = (v1[2] * beta + alpha * v2[2]);
}
/* areEqual / areEqualLT, utility.h:75-83 (ZERO_PREC = 1e-6 for double). */
static inline int are_equal(double a, double b) { return fabs(a - b) < 1e-6; }
static inline int are_equal_lt(double a, double b) { return fabs(a - b) < 1e-1; }
/* std::max(a, b) as the reference calls it: (a < b) ? b : a. */
static inline double stdmax(double a, double b) { return (a < b) ? b : a; }
/* crossProduct, MathFunctions.h:910-916. */
static inline void cross(double* cp, const double* v1, const double* v2) {
    cp[0] = v1[1] * v2[2] - v1[2] * v2[1];
    cp[1] = v1[2] * v2[0] - v1[0] * v2[2];
    cp[2] = v1[0] * v2[1] - v1[1] * v2[0];
}
/* dotProduct, MathFunctions.h:445-449. */
static inline double dot3(const double* v1, const double* v2) { return v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2]; }
/* normalizeVector (array version), MathFunctions.h:178-188. */
static inline void normalize3(double* v) {
    double x2 = v[0] * v[0], y2 = v[1] * v[1], z2 = v[2] * v[2];
    double norm = sqrt(x2 + y2 + z2);
    v[0] = v[0] / norm;
    v[1] = v[1] / norm;
    v[2] = v[2] / norm;
}
/* vectorProduct (array template), MathFunctions.h:695-717. */
static inline void vprod(double* v, const double* v1, const double* v2, const double* v3, const double* v4) {
    double v211 = (v2[1] - v1[1]), v430 = (v4[0] - v3[0]), v212 = (v2[2] - v1[2]);
    double v432 = (v4[2] - v3[2]), v431 = (v4[1] - v3[1]), v210 = (v2[0] - v1[0]);
    v[0] = v211 * v432 - v212 * v431;
    v[1] = v212 * v430 - v210 * v432;
    v[2] = v210 * v431 - v211 * v430;
}
/* areInPlane (array version), MathFunctions.h:1101-1133. */
static int in_plane(const double* p1, const double* p2, const double* p3, const double* p4) {
    double v1[3], v2[3], v3[3], cp[3];
    for (int k = 0; k < 3; ++k) {
        v1[k] = p2[k] - p1[k];
        v2[k] = p3[k] - p1[k];
        v3[k] = p4[k] - p1[k];
    }
    cross(cp, v1, v2);
    normalize3(cp);
    normalize3(v3);
    return are_equal_lt(dot3(v3, cp), 0.0);
}
/* movePointOutOfPlane (in-place array version), MathFunctions.h:1221-1270. */
static void move_out_of_plane(const double* p1, const double* p2, const double* p3, const double* p4, double* newp,
                              int i, double d) {
    double norm[3], v1[3], v2[3];
    for (int k = 0; k < 3; ++k) {
        v1[k] = p2[k] - p1[k];
        v2[k] = p3[k] - p1[k];
    }
    cross(norm, v1, v2);
    normalize3(norm);
    const double* p = i == 1 ? p1 : i == 2 ? p2 : i == 3 ? p3 : p4;
    for (int k = 0; k < 3; ++k) newp[k] = (p[k] + norm[k] * d);
}
/* checkNaN_INF over 3 components, MathFunctions.h:1377-1384. */
static int bad3(const double* x) {
    for (int i = 0; i < 3; ++i)
        if (isinf(x[i]) || isnan(x[i]) || fabs(x[i]) > 1e15) return 1;
    return 0;
}

/* ----------------------------------------------------- filament stretching */
/* FilamentStretchingHarmonic::energy, Filament/FilamentStretchingHarmonic.cpp:185-210. */
double oracle_fil_stretch_energy(const double* x, int32_t n, const int32_t* bs, const double* k, const double* l0) {
    double U = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs[2 * i];
        const double* c2 = x + bs[2 * i + 1];
        double dist = tpd(c1, c2) - l0[i];
        U += 0.5 * k[i] * dist * dist;
    }
    return U;
}
/* FilamentStretchingHarmonic::forces, FilamentStretchingHarmonic.cpp:212-275. */
void oracle_fil_stretch_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k,
                               const double* l0) {
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs[2 * i];
        const double* c2 = x + bs[2 * i + 1];
        double dist = tpd(c1, c2);
        double invL = 1 / dist;
        double f0 = k[i] * (dist - l0[i]) * invL;
        double* f1 = f + bs[2 * i];
        double* f2 = f + bs[2 * i + 1];
        for (int d = 0; d < 3; ++d) {
            double Fr = -f0 * (c2[d] - c1[d]);
            f2[d] += Fr;
            f1[d] += -Fr;
        }
    }
}

/* ------------------------------------------------------- filament bending */
/* FilamentBendingCosine::energy, Filament/FilamentBendingCosine.cpp:199-246. */
double oracle_fil_bend_energy(const double* x, int32_t n, const int32_t* bs, const double* k, const double* t0) {
    double U = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs[3 * i];
        const double* c2 = x + bs[3 * i + 1];
        const double* c3 = x + bs[3 * i + 2];
        double L1 = sqrt(sp4(c1, c2, c1, c2));
        double L2 = sqrt(sp4(c2, c3, c2, c3));
        double L1L2 = L1 * L2;
        double l1l2 = sp4(c1, c2, c2, c3);
        double xx = l1l2 / L1L2;
        if (xx < -1.0) xx = -1.0;
        else if (xx > 1.0) xx = 1.0;
        double Ui;
        if (are_equal(t0[i], 0.0)) {
            Ui = k[i] * (1 - xx);
        } else {
            double cosA = xx;
            double sinA = stdmax(sqrt(1 - cosA * cosA), 0.0);
            double cosAmB = cosA * cos(t0[i]) + sinA * sin(t0[i]);
            Ui = k[i] * (1 - cosAmB);
        }
        U += Ui;
    }
    return U;
}
/* Shared by FilamentBendingCosine::forces (FilamentBendingCosine.cpp:249-345) and
   BranchingBendingCosine::forces (Branching/BranchingBendingCosine.cpp:246-330):
   returns k, A, B, C for bond vectors r1 = p2 - p1, r2 = p4 - p3. */
static double bend_coeffs(const double* p1, const double* p2, const double* p3, const double* p4, double kb,
                          double eqt, double* A, double* B, double* C) {
    double L1sq = sp4(p1, p2, p1, p2);
    double L2sq = sp4(p3, p4, p3, p4);
    double l1l2 = sp4(p1, p2, p3, p4);
    *A = 1 / sqrt(L1sq * L2sq);
    double xx = l1l2 * *A;
    *B = xx / L1sq;
    *C = xx / L2sq;
    if (are_equal(eqt, 0.0)) return kb;
    if (fabs(fabs(xx) - 1.0) < 0.001) xx = 0.999 * xx;
    if (xx < -1.0) xx = -1.0;
    else if (xx > 1.0) xx = 1.0;
    double cosp = xx;
    double sinp = sqrt(stdmax((1 - cosp * cosp), 0.0));
    double sinpmq = sinp * cos(eqt) - cosp * sin(eqt);
    return kb * sinpmq / sinp;
}
void oracle_fil_bend_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k,
                            const double* t0) {
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs[3 * i];
        const double* c2 = x + bs[3 * i + 1];
        const double* c3 = x + bs[3 * i + 2];
        double A, B, C;
        double kk = bend_coeffs(c1, c2, c2, c3, k[i], t0[i], &A, &B, &C);
        double* f1 = f + bs[3 * i];
        double* f2 = f + bs[3 * i + 1];
        double* f3 = f + bs[3 * i + 2];
        for (int d = 0; d < 3; ++d) {
            double r1 = c2[d] - c1[d], r2 = c3[d] - c2[d];
            double Fr1 = kk * (r2 * A - r1 * B);
            double Fr2 = kk * (r1 * A - r2 * C);
            f1[d] += -Fr1;
            f2[d] += Fr1 - Fr2;
            f3[d] += Fr2;
        }
    }
}

/* ------------------------------------------------------ linker / motor */
/* LinkerStretchingHarmonic::energy (Linker/LinkerStretchingHarmonic.cpp:191-220)
   and MotorGhostStretchingHarmonic::energy (MotorGhost/...Harmonic.cpp:234-262):
   identical math. */
double oracle_two_point_spring_energy(const double* x, int32_t n, const int32_t* bs, const double* k,
                                      const double* l0, const double* p1, const double* p2) {
    double U = 0.0, v1[3], v2[3];
    for (int32_t i = 0; i < n; ++i) {
        midpt(v1, x + bs[4 * i], x + bs[4 * i + 1], p1[i]);
        midpt(v2, x + bs[4 * i + 2], x + bs[4 * i + 3], p2[i]);
        double dist = tpd(v1, v2) - l0[i];
        U += 0.5 * k[i] * dist * dist;
    }
    return U;
}
/* LinkerStretchingHarmonic::forces, LinkerStretchingHarmonic.cpp:223-292. */
void oracle_two_point_spring_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k,
                                    const double* l0, const double* p1, const double* p2) {
    double v1[3], v2[3];
    for (int32_t i = 0; i < n; ++i) {
        midpt(v1, x + bs[4 * i], x + bs[4 * i + 1], p1[i]);
        midpt(v2, x + bs[4 * i + 2], x + bs[4 * i + 3], p2[i]);
        double dist = tpd(v1, v2);
        double invL = 1 / dist;
        double f0 = k[i] * (dist - l0[i]) * invL;
        double* f1 = f + bs[4 * i];
        double* f2 = f + bs[4 * i + 1];
        double* f3 = f + bs[4 * i + 2];
        double* f4 = f + bs[4 * i + 3];
        for (int d = 0; d < 3; ++d) {
            double Fl = -f0 * (v2[d] - v1[d]);
            f1[d] += -Fl * (1 - p1[i]);
            f2[d] += -Fl * (p1[i]);
            f3[d] += Fl * (1 - p2[i]);
            f4[d] += Fl * (p2[i]);
        }
    }
}

/* --------------------------------------------------------------- branching */
/* BranchingStretchingHarmonic::energy, Branching/BranchingStretchingHarmonic.cpp:195-219.
   bs4 holds 4 offsets per branch point; stretching uses the first 3. */
double oracle_branch_stretch_energy(const double* x, int32_t n, const int32_t* bs4, const double* k,
                                    const double* l0, const double* pos) {
    double U = 0.0, v1[3];
    for (int32_t i = 0; i < n; ++i) {
        midpt(v1, x + bs4[4 * i], x + bs4[4 * i + 1], pos[i]);
        double dist = tpd(v1, x + bs4[4 * i + 2]) - l0[i];
        U += 0.5 * k[i] * dist * dist;
    }
    return U;
}
/* BranchingStretchingHarmonic::forces, BranchingStretchingHarmonic.cpp:222-266. */
void oracle_branch_stretch_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                                  const double* l0, const double* pos) {
    double v1[3];
    for (int32_t i = 0; i < n; ++i) {
        const double* c3 = x + bs4[4 * i + 2];
        midpt(v1, x + bs4[4 * i], x + bs4[4 * i + 1], pos[i]);
        double dist = tpd(v1, c3);
        double invL = 1 / dist;
        double f0 = k[i] * (dist - l0[i]) * invL;
        double* f1 = f + bs4[4 * i];
        double* f2 = f + bs4[4 * i + 1];
        double* f3 = f + bs4[4 * i + 2];
        for (int d = 0; d < 3; ++d) {
            double r1 = c3[d] - v1[d];
            f1[d] += -f0 * (r1) * (pos[i] - 1);
            f2[d] += f0 * (r1) * pos[i];
            f3[d] += -f0 * (r1);
        }
    }
}
/* BranchingBendingCosine::energy, Branching/BranchingBendingCosine.cpp:196-242. */
double oracle_branch_bend_energy(const double* x, int32_t n, const int32_t* bs4, const double* k, const double* t0) {
    double U = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs4[4 * i];
        const double* c2 = x + bs4[4 * i + 1];
        const double* c3 = x + bs4[4 * i + 2];
        const double* c4 = x + bs4[4 * i + 3];
        double L1 = sqrt(sp4(c1, c2, c1, c2));
        double L2 = sqrt(sp4(c3, c4, c3, c4));
        double L1L2 = L1 * L2;
        double l1l2 = sp4(c1, c2, c3, c4);
        double xx = l1l2 / L1L2;
        if (xx < -1.0) xx = -1.0;
        else if (xx > 1.0) xx = 1.0;
        double Ui;
        if (are_equal(t0[i], 0.0)) {
            Ui = k[i] * (1 - xx);
        } else {
            double cosA = xx;
            double sinA = stdmax(sqrt(1 - cosA * cosA), 0.0);
            double cosAmB = cosA * cos(t0[i]) + sinA * sin(t0[i]);
            Ui = k[i] * (1 - cosAmB);
        }
        U += Ui;
    }
    return U;
}
/* BranchingBendingCosine::forces, BranchingBendingCosine.cpp:245-330. */
void oracle_branch_bend_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                               const double* t0) {
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs4[4 * i];
        const double* c2 = x + bs4[4 * i + 1];
        const double* c3 = x + bs4[4 * i + 2];
        const double* c4 = x + bs4[4 * i + 3];
        double A, B, C;
        double kk = bend_coeffs(c1, c2, c3, c4, k[i], t0[i], &A, &B, &C);
        double* f1 = f + bs4[4 * i];
        double* f2 = f + bs4[4 * i + 1];
        double* f3 = f + bs4[4 * i + 2];
        double* f4 = f + bs4[4 * i + 3];
        for (int d = 0; d < 3; ++d) {
            double r1 = c2[d] - c1[d], r2 = c4[d] - c3[d];
            double Fr1 = kk * (r2 * A - r1 * B);
            double Fr2 = kk * (r1 * A - r2 * C);
            f1[d] += -Fr1;
            f2[d] += Fr1;
            f3[d] += -Fr2;
            f4[d] += Fr2;
        }
    }
}

/* Plus-end branch handling shared by the dihedral and position potentials
   (Branching/BranchingDihedralCosine.cpp:236-243): at pos == 1 the parent's
   plus end is replaced by a virtual plus end and the position becomes 0.5. */
static double virtual_plus_end(const double* c1, const double* c2, double pos, double* c2prime) {
    double position = pos;
    if (are_equal(position, 1.0)) {
        position = 0.5;
        for (int d = 0; d < 3; ++d) c2prime[d] = (1 / position) * (c2[d] - (1 - position) * c1[d]);
    } else {
        for (int d = 0; d < 3; ++d) c2prime[d] = c2[d];
    }
    return position;
}

/* BranchingDihedralCosine::energy, Branching/BranchingDihedralCosine.cpp:211-263. */
double oracle_branch_dihedral_energy(const double* x, int32_t n, const int32_t* bs4, const double* k,
                                     const double* pos) {
    double U = 0.0, c2p[3], mp[3], n1[3], n2[3];
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs4[4 * i];
        const double* c3 = x + bs4[4 * i + 2];
        const double* c4 = x + bs4[4 * i + 3];
        double position = virtual_plus_end(c1, x + bs4[4 * i + 1], pos[i], c2p);
        midpt(mp, c1, c2p, position);
        vprod(n1, mp, c2p, mp, c3);
        vprod(n2, c3, c4, mp, c3);
        normalize3(n1);
        normalize3(n2);
        U += k[i] * (1 - dot3(n1, n2));
    }
    return U;
}
/* BranchingDihedralCosine::forces (LAMMPS-style), BranchingDihedralCosine.cpp:268-490. */
void oracle_branch_dihedral_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                                   const double* pos) {
    for (int32_t i = 0; i < n; ++i) {
        double c1[3], c2[3], c3[3], c4[3], mp[3];
        for (int d = 0; d < 3; ++d) {
            c1[d] = x[bs4[4 * i] + d];
            c2[d] = x[bs4[4 * i + 1] + d];
            c3[d] = x[bs4[4 * i + 2] + d];
            c4[d] = x[bs4[4 * i + 3] + d];
        }
        double position = pos[i];
        if (are_equal(position, 1.0)) {
            position = 0.5;
            c2[0] = (1 / position) * (c2[0] - (1 - position) * c1[0]);
            c2[1] = (1 / position) * (c2[1] - (1 - position) * c1[1]);
            c2[2] = (1 / position) * (c2[2] - (1 - position) * c1[2]);
        }
        midpt(mp, c1, c2, position);
        double vb1x = c2[0] - mp[0], vb1y = c2[1] - mp[1], vb1z = c2[2] - mp[2];
        double vb2x = c3[0] - mp[0], vb2y = c3[1] - mp[1], vb2z = c3[2] - mp[2];
        double vb2xm = -vb2x, vb2ym = -vb2y, vb2zm = -vb2z;
        double vb3x = c4[0] - c3[0], vb3y = c4[1] - c3[1], vb3z = c4[2] - c3[2];
        double ax = vb1y * vb2zm - vb1z * vb2ym;
        double ay = vb1z * vb2xm - vb1x * vb2zm;
        double az = vb1x * vb2ym - vb1y * vb2xm;
        double bx = vb3y * vb2zm - vb3z * vb2ym;
        double by = vb3z * vb2xm - vb3x * vb2zm;
        double bz = vb3x * vb2ym - vb3y * vb2xm;
        double rasq = ax * ax + ay * ay + az * az;
        double rbsq = bx * bx + by * by + bz * bz;
        double rgsq = vb2xm * vb2xm + vb2ym * vb2ym + vb2zm * vb2zm;
        double rg = sqrt(rgsq);
        double rginv = 0.0, ra2inv = 0.0, rb2inv = 0.0;
        if (rg > 0) rginv = 1.0 / rg;
        if (rasq > 0) ra2inv = 1.0 / rasq;
        if (rbsq > 0) rb2inv = 1.0 / rbsq;
        double rabinv = sqrt(ra2inv * rb2inv);
        double c = (ax * bx + ay * by + az * bz) * rabinv;
        double s = rg * rabinv * (ax * vb3x + ay * vb3y + az * vb3z);
        if (c > 1.0) c = 1.0;
        if (c < -1.0) c = -1.0;
        (void)c;
        double df1 = s;
        double fg = vb1x * vb2xm + vb1y * vb2ym + vb1z * vb2zm;
        double hg = vb3x * vb2xm + vb3y * vb2ym + vb3z * vb2zm;
        double fga = fg * ra2inv * rginv;
        double hgb = hg * rb2inv * rginv;
        double gaa = -ra2inv * rg;
        double gbb = rb2inv * rg;
        double dtfx = gaa * ax, dtfy = gaa * ay, dtfz = gaa * az;
        double dtgx = fga * ax - hgb * bx, dtgy = fga * ay - hgb * by, dtgz = fga * az - hgb * bz;
        double dthx = gbb * bx, dthy = gbb * by, dthz = gbb * bz;
        double df = -k[i] * df1;
        double sx2 = df * dtgx, sy2 = df * dtgy, sz2 = df * dtgz;
        double L4[3] = {df * dthx, df * dthy, df * dthz};
        double L3[3] = {-sx2 - L4[0], -sy2 - L4[1], -sz2 - L4[2]};
        double L1[3], L2[3];
        if (are_equal(pos[i], 1.0)) {
            double L2p[3] = {df * dtfx, df * dtfy, df * dtfz};
            L2[0] = sx2 - L2p[0];
            L2[1] = sy2 - L2p[1];
            L2[2] = sz2 - L2p[2];
            double factor = (position - 1) / position;
            L1[0] = L2p[0] * factor;
            L1[1] = L2p[1] * factor;
            L1[2] = L2p[2] * factor;
            factor = (1 / position);
            L2[0] += L2p[0] * factor;
            L2[1] += L2p[1] * factor;
            L2[2] += L2p[2] * factor;
        } else {
            L2[0] = df * dtfx;
            L2[1] = df * dtfy;
            L2[2] = df * dtfz;
            double Lmp[3] = {sx2 - L2[0], sy2 - L2[1], sz2 - L2[2]};
            L1[0] = (1 - position) * Lmp[0];
            L1[1] = (1 - position) * Lmp[1];
            L1[2] = (1 - position) * Lmp[2];
            L2[0] += (position)*Lmp[0];
            L2[1] += (position)*Lmp[1];
            L2[2] += (position)*Lmp[2];
        }
        double* f1 = f + bs4[4 * i];
        double* f2 = f + bs4[4 * i + 1];
        double* f3 = f + bs4[4 * i + 2];
        double* f4 = f + bs4[4 * i + 3];
        for (int d = 0; d < 3; ++d) {
            f1[d] += L1[d];
            f2[d] += L2[d];
            f3[d] += L3[d];
            f4[d] += L4[d];
        }
    }
}
/* BranchingPositionCosine::energy, Branching/BranchingPositionCosine.cpp:190-240. */
double oracle_branch_position_energy(const double* x, int32_t n, const int32_t* bs4, const double* k,
                                     const double* pos) {
    double U = 0.0, c2p[3], mp[3];
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs4[4 * i];
        const double* c3 = x + bs4[4 * i + 2];
        double position = virtual_plus_end(c1, x + bs4[4 * i + 1], pos[i], c2p);
        midpt(mp, c1, c2p, position);
        double X = sqrt(sp4(mp, c2p, mp, c2p));
        double D = sqrt(sp4(mp, c3, mp, c3));
        double XD = X * D;
        double xd = sp4(mp, c2p, mp, c3);
        double xx = xd / XD;
        if (fabs(fabs(xx) - 1.0) < 0.001) {
            xd = 0.999 * XD;
            xx = xd / XD;
        }
        if (xx < -1.0) xx = -1.0;
        else if (xx > 1.0) xx = 1.0;
        double cosp = xx;
        double posheta = 0.5 * M_PI;
        double sinp = sqrt(stdmax((1 - cosp * cosp), 0.0));
        double cospmq = cosp * cos(posheta) + sinp * sin(posheta);
        U += k[i] * (1 - cospmq);
    }
    return U;
}
/* BranchingPositionCosine::forces, BranchingPositionCosine.cpp:310-440. */
void oracle_branch_position_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                                   const double* pos) {
    double c2p[3], mp[3];
    for (int32_t i = 0; i < n; ++i) {
        const double* c1 = x + bs4[4 * i];
        const double* c3 = x + bs4[4 * i + 2];
        double position = virtual_plus_end(c1, x + bs4[4 * i + 1], pos[i], c2p);
        midpt(mp, c1, c2p, position);
        double Xsq = sp4(mp, c2p, mp, c2p);
        double Dsq = sp4(mp, c3, mp, c3);
        double xd = sp4(mp, c2p, mp, c3);
        double A = 1 / sqrt(Xsq * Dsq);
        double xx = xd * A;
        double B = xx / Xsq;
        double C = xx / Dsq;
        if (fabs(fabs(xx) - 1.0) < 0.001) xx = 0.999 * xx;
        if (xx < -1.0) xx = -1.0;
        else if (xx > 1.0) xx = 1.0;
        double cosp = xx;
        double posheta = 0.5 * M_PI;
        double sinp = sqrt(stdmax((1 - cosp * cosp), 0.0));
        double sinpmq = sinp * cos(posheta) - cosp * sin(posheta);
        double kk = k[i] * sinpmq / sinp;
        double f1t[3], f2t[3], f3t[3];
        for (int d = 0; d < 3; ++d) {
            double r1 = c2p[d] - mp[d], r2 = c3[d] - mp[d];
            double Fr1 = kk * (r2 * A - r1 * B);
            double Fr2 = kk * (r1 * A - r2 * C);
            double fmp = -Fr1 - Fr2;
            f1t[d] = (1 - position) * fmp;
            f2t[d] = Fr1 + position * fmp;
            f3t[d] = Fr2;
        }
        double* f1 = f + bs4[4 * i];
        double* f2 = f + bs4[4 * i + 1];
        double* f3 = f + bs4[4 * i + 2];
        for (int d = 0; d < 3; ++d) f3[d] += f3t[d];
        if (are_equal(pos[i], 1.0)) {
            double factor = (position - 1) / position;
            for (int d = 0; d < 3; ++d) {
                f1[d] += f1t[d] + f2t[d] * factor;
                f2[d] += f2t[d] * (1 / position);
            }
        } else {
            for (int d = 0; d < 3; ++d) {
                f1[d] += f1t[d];
                f2[d] += f2t[d];
            }
        }
    }
}

/* ------------------------------------------------ cylinder excluded volume */
/* Intermediate scalars of the analytic integral,
   Volume/CylinderExclVolRepulsion.cpp:360-410 (energy) and :643-690 (forces). */
typedef struct ExclScalars {
    double a, b, c, d, e, F, g, h, I, AA, BB, CC, DD, EE, FF, GG, HH, JJ, ATG1, ATG2, ATG3, ATG4;
} ExclScalars;

static void excl_scalars(const double* c1, const double* c2, const double* c3, const double* c4, ExclScalars* s) {
    double vA[3], vB[3], vC[3], cp[3];
    s->a = sp4(c1, c2, c1, c2);
    s->b = sp4(c3, c4, c3, c4);
    s->c = sp4(c3, c1, c3, c1);
    s->d = sp4(c1, c2, c3, c4);
    s->e = sp4(c1, c2, c3, c1);
    s->F = sp4(c3, c4, c3, c1);
    s->g = sp4(c1, c2, c1, c4);
    s->h = sp4(c3, c4, c3, c2);
    s->I = sp4(c3, c4, c1, c4);
    /* sqmagnitude(c1, c2) with doubleprecision temporaries, MathFunctions.h:210-217. */
    double dx = c1[0] - c4[0], dy = c1[1] - c4[1], dz = c1[2] - c4[2];
    double sqD = (dx * dx + dy * dy + dz * dz);
    dx = c3[0] - c2[0];
    dy = c3[1] - c2[1];
    dz = c3[2] - c2[2];
    double sqE = (dx * dx + dy * dy + dz * dz);
    for (int k = 0; k < 3; ++k) {
        vA[k] = c1[k] - c2[k];
        vB[k] = c3[k] - c4[k];
        vC[k] = c3[k] - c1[k];
    }
    double ac = sqrt(s->a * s->c);
    double bc = sqrt(s->b * s->c);
    double aD = sqrt(s->a * sqD);
    double bE = sqrt(s->b * sqE);
    s->AA = sqrt(stdmax(0.0, (ac + s->e) * (ac - s->e)));
    s->BB = sqrt(stdmax(0.0, (bc + s->F) * (bc - s->F)));
    s->CC = s->d * s->e - s->a * s->F;
    s->DD = s->b * s->e - s->d * s->F;
    s->EE = sqrt(stdmax(0.0, (aD + s->g) * (aD - s->g)));
    s->FF = sqrt(stdmax(0.0, (bE + s->h) * (bE - s->h)));
    s->GG = s->d * s->g - s->a * s->I;
    s->HH = s->CC + s->GG - s->DD;
    cross(cp, vA, vB);
    double JJ = cp[0] * vC[0] + cp[1] * vC[1] + cp[2] * vC[2];
    s->JJ = -JJ * JJ;
    const double a = s->a, b = s->b, d = s->d, e = s->e, F = s->F;
    s->ATG1 = atan((a + e) / s->AA) - atan(e / s->AA);
    s->ATG2 = atan((a + e - d) / s->EE) - atan((e - d) / s->EE);
    s->ATG3 = atan((F) / s->BB) - atan((F - b) / s->BB);
    s->ATG4 = atan((d + F) / s->FF) - atan((d + F - b) / s->FF);
}

double oracle_excl_pair_energy(const double* c1, const double* c2, const double* c3, const double* c4,
                               double krep_scaled) {
    ExclScalars s;
    excl_scalars(c1, c2, c3, c4, &s);
    return 0.5 * krep_scaled / s.JJ *
           (s.CC / s.AA * s.ATG1 + s.GG / s.EE * s.ATG2 + s.DD / s.BB * s.ATG3 + s.HH / s.FF * s.ATG4);
}

/* getenergyintegrand / getforceintegrand, Volume/CylinderExclVolRepulsion.h:50-71. */
static inline double r2_of(double a, double b, double c, double d, double e, double F, double s, double t) {
    return c + 2 * s * e + s * s * a - 2 * t * F - 2 * s * t * d + t * t * b;
}
static inline double energy_integrand(double a, double b, double c, double d, double e, double F, double s,
                                      double t) {
    double r_2 = r2_of(a, b, c, d, e, F, s, t);
    return (1.0 / (r_2 * r_2));
}

/* CylinderExclVolRepulsion::energyN, CylinderExclVolRepulsion.cpp:884-999:
   2-D composite Simpson sum with the reference's index bookkeeping (s and t
   advance before use). The moved-beads retry's result is discarded in the
   reference, so it is not restated. */
static double excl_energyN(const double* c1, const double* c2, const double* c3, const double* c4, double kRS) {
    double a = sp4(c1, c2, c1, c2), b = sp4(c3, c4, c3, c4), c = sp4(c3, c1, c3, c1);
    double d = sp4(c1, c2, c3, c4), e = sp4(c1, c2, c3, c1), F = sp4(c3, c4, c3, c1);
    const int N1 = 400, N2 = 400;
    double ds = 1.0 / ((double)N1), dt = 1.0 / ((double)N2);
    double T1 = energy_integrand(a, b, c, d, e, F, 0.0, 0.0) + energy_integrand(a, b, c, d, e, F, 0.0, 1.0) +
                energy_integrand(a, b, c, d, e, F, 1.0, 0.0) + energy_integrand(a, b, c, d, e, F, 1.0, 1.0);
    double T2 = 0.0, T3 = 0.0, T4 = 0.0, s = 0.0, t = 0.0;
    for (int i = 0; i <= N1; i++) {
        t = 0.0;
        s += ds;
        double fs = (i % 2 == 0) ? 2.0 : 4.0;
        if (i > 0 && i < N1)
            T2 += fs * (energy_integrand(a, b, c, d, e, F, s, 0.0) + energy_integrand(a, b, c, d, e, F, s, 1.0));
        for (int j = 0; j <= N2; j++) {
            t += dt;
            double ft = (j % 2 == 0) ? 2.0 : 4.0;
            if (j > 0 && j < N2) {
                if (i == 0)
                    T3 += ft * (energy_integrand(a, b, c, d, e, F, 0.0, t) + energy_integrand(a, b, c, d, e, F, 1.0, t));
                else if (i < N1)
                    T4 += fs * ft * energy_integrand(a, b, c, d, e, F, s, t);
            }
        }
    }
    return kRS * (ds * dt / 9.0) * (T1 + T2 + T3 + T4);
}

static int energy_bad(double U) { return isinf(U) || U != U || U < -1.0; }

/* CylinderExclVolRepulsion::energy, CylinderExclVolRepulsion.cpp:330-575. */
double oracle_excl_energy(const double* x, int32_t n, const int32_t* bs, const double* k, const double* eqlen) {
    double U = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double kRS = k[i] * eqlen[2 * i] * eqlen[2 * i + 1];
        const double* c1 = x + bs[4 * i];
        const double* c2 = x + bs[4 * i + 1];
        const double* c3 = x + bs[4 * i + 2];
        const double* c4 = x + bs[4 * i + 3];
        double Ui = oracle_excl_pair_energy(c1, c2, c3, c4, kRS);
        if (energy_bad(Ui)) {
            Ui = excl_energyN(c1, c2, c3, c4, kRS);
            if (energy_bad(Ui)) return -1;
        }
        U += Ui;
    }
    return U;
}

/* CylinderExclVolRepulsion::forceN, CylinderExclVolRepulsion.cpp:1001-1256.
   Returns 0 when it accumulated forces, 1 when they stayed non-finite. */
static int excl_forceN(const double* x, double* f, const int32_t* bs, double kRS, int movebeads) {
    const double* c1 = x + bs[0];
    const double* c2 = x + bs[1];
    const double* c3 = x + bs[2];
    const double* c4 = x + bs[3];
    double newc1[3], newc2[3];
    if (movebeads && in_plane(c1, c2, c3, c4)) {
        move_out_of_plane(c1, c2, c3, c4, newc2, 2, 0.01);
        move_out_of_plane(c1, c2, c3, c4, newc1, 1, 0.01);
        c2 = newc2;
        c1 = newc1;
    }
    double a = sp4(c1, c2, c1, c2), b = sp4(c3, c4, c3, c4), c = sp4(c3, c1, c3, c1);
    double d = sp4(c1, c2, c3, c4), e = sp4(c1, c2, c3, c1), F = sp4(c3, c4, c3, c1);
    double vA[3], vB[3], vC[3];
    for (int k = 0; k < 3; ++k) {
        vA[k] = c1[k] - c2[k];
        vB[k] = c3[k] - c4[k];
        vC[k] = c3[k] - c1[k];
    }
    const int N1 = 10000, N2 = 10000;
    double ds = 1.0 / ((double)N1), dt = 1.0 / ((double)N2);
    double T1[6] = {0}, T2[6] = {0}, T3[6] = {0}, T4[6] = {0}, in[6];
    const double lim[2] = {0.0, 1.0};
#define FORCE_INTEGRAND(S, T)                                        \
    do {                                                             \
        double r_2 = r2_of(a, b, c, d, e, F, (S), (T));              \
        double xi = (1.0 / (r_2 * r_2 * r_2));                       \
        in[0] = xi;                                                  \
        in[1] = (S) * xi;                                            \
        in[2] = (S) * (S) * xi;                                      \
        in[3] = (S) * (T) * xi;                                      \
        in[4] = (T) * xi;                                            \
        in[5] = (T) * (T) * xi;                                      \
    } while (0)
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            FORCE_INTEGRAND(lim[i], lim[j]);
            for (int q = 0; q < 6; q++) T1[q] += in[q];
        }
    double s = 0.0, t = 0.0;
    for (int i = 0; i <= N1; i++) {
        t = 0.0;
        s += ds;
        double fs = (i % 2 == 0) ? 2.0 : 4.0;
        if (i > 0 && i < N1)
            for (int l = 0; l < 2; l++) {
                FORCE_INTEGRAND(s, lim[l]);
                for (int q = 0; q < 6; q++) T2[q] += fs * in[q];
            }
        for (int j = 0; j <= N2; j++) {
            t += dt;
            double ft = (j % 2 == 0) ? 2.0 : 4.0;
            if (j > 0 && j < N2) {
                if (i == 0) {
                    for (int l = 0; l < 2; l++) {
                        FORCE_INTEGRAND(lim[l], t);
                        for (int q = 0; q < 6; q++) T3[q] += ft * in[q];
                    }
                } else if (i < N1) {
                    FORCE_INTEGRAND(s, t);
                    for (int q = 0; q < 6; q++) T4[q] += fs * ft * in[q];
                }
            }
        }
    }
#undef FORCE_INTEGRAND
    double I[6];
    for (int q = 0; q < 6; q++) I[q] = (ds * dt / 9.0) * (T1[q] + T2[q] + T3[q] + T4[q]);
    double f1l[3], f2l[3], f3l[3], f4l[3];
    for (int k = 0; k < 3; k++) {
        f1l[k] = 4.0 * kRS * (-I[0] * vC[k] + I[1] * (vC[k] - vA[k]) + I[2] * vA[k] + I[4] * vB[k] - I[3] * vB[k]);
        f2l[k] = 4.0 * kRS * (-I[1] * vC[k] - I[2] * vA[k] + I[3] * vB[k]);
        f3l[k] = 4.0 * kRS * (I[0] * vC[k] + I[1] * vA[k] - I[4] * (vB[k] + vC[k]) - I[3] * vA[k] + I[5] * vB[k]);
        f4l[k] = 4.0 * kRS * (I[4] * vC[k] + I[3] * vA[k] - I[5] * vB[k]);
    }
    if (bad3(f1l) || bad3(f2l) || bad3(f3l) || bad3(f4l)) {
        if (!movebeads) return excl_forceN(x, f, bs, kRS, 1);
        return 1; /* the reference prints diagnostics and exits here */
    }
    for (int k = 0; k < 3; k++) {
        f[bs[0] + k] += f1l[k];
        f[bs[1] + k] += f2l[k];
        f[bs[2] + k] += f3l[k];
        f[bs[3] + k] += f4l[k];
    }
    return 0;
}

/* CylinderExclVolRepulsion::forces, CylinderExclVolRepulsion.cpp:578-882. */
void oracle_excl_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k,
                        const double* eqlen) {
    for (int32_t i = 0; i < n; ++i) {
        const double kRS = k[i] * eqlen[2 * i] * eqlen[2 * i + 1];
        const double* c1 = x + bs[4 * i];
        const double* c2 = x + bs[4 * i + 1];
        const double* c3 = x + bs[4 * i + 2];
        const double* c4 = x + bs[4 * i + 3];
        double newc2[3];
        if (in_plane(c1, c2, c3, c4)) {
            move_out_of_plane(c1, c2, c3, c4, newc2, 2, 0.01);
            c2 = newc2;
        }
        ExclScalars S;
        excl_scalars(c1, c2, c3, c4, &S);
        const double a = S.a, b = S.b, c = S.c, d = S.d, e = S.e, F = S.F;
        const double AA = S.AA, BB = S.BB, CC = S.CC, DD = S.DD, EE = S.EE, FF = S.FF, GG = S.GG, HH = S.HH;
        const double JJ = S.JJ, ATG1 = S.ATG1, ATG2 = S.ATG2, ATG3 = S.ATG3, ATG4 = S.ATG4;
        const double invJJ = 1 / JJ;
        const double sumBlock = CC / AA * ATG1 + GG / EE * ATG2 + DD / BB * ATG3 + HH / FF * ATG4;
        const double enFactor = kRS * invJJ / 2;
        const double A1 = AA * AA / (AA * AA + (a + e) * (a + e));
        const double A2 = AA * AA / (AA * AA + e * e);
        const double E1 = EE * EE / (EE * EE + (a + e - d) * (a + e - d));
        const double E2 = EE * EE / (EE * EE + (e - d) * (e - d));
        const double B1 = BB * BB / (BB * BB + F * F);
        const double B2 = BB * BB / (BB * BB + (F - b) * (F - b));
        const double F1 = FF * FF / (FF * FF + (d + F) * (d + F));
        const double F2 = FF * FF / (FF * FF + (d + F - b) * (d + F - b));
        const double bA_C = ATG1 / AA;
        const double bA_A = -(ATG1 * CC) / (AA * AA) + (-A1 * (a + e) + A2 * e) * CC / (AA * AA * AA);
        const double bA_e = ((A1 - A2) * CC) / (AA * AA);
        const double bA_a = (A1 * CC) / (AA * AA);
        const double bE_G = ATG2 / EE;
        const double bE_E = -(ATG2 * GG) / (EE * EE) + (-E1 * (a + e - d) + E2 * (e - d)) * GG / (EE * EE * EE);
        const double bE_emd = ((E1 - E2) * GG) / (EE * EE);
        const double bE_a = (E1 * GG) / (EE * EE);
        const double bB_D = ATG3 / BB;
        const double bB_B = -(ATG3 * DD) / (BB * BB) + (-B1 * F + B2 * (F - b)) * DD / (BB * BB * BB);
        const double bB_fmb = ((B1 - B2) * DD) / (BB * BB);
        const double bB_b = (B1 * DD) / (BB * BB);
        const double bF_H = ATG4 / FF;
        const double bF_F = -(ATG4 * HH) / (FF * FF) + (-F1 * (d + F) + F2 * (d + F - b)) * HH / (FF * FF * FF);
        const double bF_dpfmb = ((F1 - F2) * HH) / (FF * FF);
        const double bF_b = (F1 * HH) / (FF * FF);
        const double b11 = bA_C * (-2 * F) + bA_A * (c / AA) + bA_a * 2 + bE_G * (2 * (F - b)) +
                           bE_E * ((b + c - 2 * F) / EE) + bE_a * 2 + bF_H * (-2 * b) + bF_F * (b / FF);
        const double b12 = bA_C * e + bE_G * (2 * d - e) + bE_E * ((e - d) / EE) + bE_emd * (-1) + bB_D * (-F) +
                           bF_H * (2 * d + F) + bF_F * (-(d + F) / FF) + bF_dpfmb;
        const double b13 = bA_C * d + bA_A * (-e / AA) + bA_e + bE_G * (-d) + bE_E * (-(e - d) / EE) + bE_emd +
                           bB_D * b + bF_H * (-b) + bF_F * (b / FF);
        const double b21 = bA_C * e + bE_G * (2 * d - e) + bE_E * ((e - d) / EE) + bE_emd * (-1) + bB_D * (-F) +
                           bF_H * (2 * d + F) + bF_F * (-(d + F) / FF) + bF_dpfmb;
        const double b22 = bE_G * (-2 * a) + bE_E * (a / EE) + bB_D * (2 * e) + bB_B * (c / BB) + bB_fmb * (-2) +
                           bB_b * 2 + bF_H * (-2 * (a + e)) + bF_F * ((a + c + 2 * e) / FF) + bF_dpfmb * (-2) +
                           bF_b * 2;
        const double b23 = bA_C * (-a) + bE_G * a + bE_E * (-a / EE) + bB_D * (-d) + bB_B * (-F / BB) + bB_fmb +
                           bF_H * d + bF_F * (-(d + F) / FF) + bF_dpfmb;
        const double b31 = bA_C * d + bA_A * (-e / AA) + bA_e + bE_G * (-d) + bE_E * (-(e - d) / EE) + bE_emd +
                           bB_D * b + bF_H * (-b) + bF_F * (b / FF);
        const double b32 = bA_C * (-a) + bE_G * a + bE_E * (-a / EE) + bB_D * (-d) + bB_B * (-F / BB) + bB_fmb +
                           bF_H * d + bF_F * (-(d + F) / FF) + bF_dpfmb;
        const double b33 = bA_A * (a / AA) + bE_E * (a / EE) + bB_B * (b / BB) + bF_F * (b / FF);
        const double J11 = 2 * (-b * c + F * F), J12 = 2 * (c * d - e * F), J13 = 2 * (b * e - d * F);
        const double J21 = 2 * (c * d - e * F), J22 = 2 * (-a * c + e * e), J23 = 2 * (-d * e + a * F);
        const double J31 = 2 * (b * e - d * F), J32 = 2 * (-d * e + a * F), J33 = 2 * (d * d - a * b);
        double dv[4][3];
        dv[0][0] = enFactor * (-invJJ * sumBlock * (J31 - J11) + (b31 - b11));
        dv[0][1] = enFactor * (-invJJ * sumBlock * (J32 - J12) + (b32 - b12));
        dv[0][2] = enFactor * (-invJJ * sumBlock * (J33 - J13) + (b33 - b13));
        dv[1][0] = enFactor * (-invJJ * sumBlock * (J11) + (b11));
        dv[1][1] = enFactor * (-invJJ * sumBlock * (J12) + (b12));
        dv[1][2] = enFactor * (-invJJ * sumBlock * (J13) + (b13));
        dv[2][0] = enFactor * (-invJJ * sumBlock * (-J31 - J21) + (-b31 - b21));
        dv[2][1] = enFactor * (-invJJ * sumBlock * (-J32 - J22) + (-b32 - b22));
        dv[2][2] = enFactor * (-invJJ * sumBlock * (-J33 - J23) + (-b33 - b23));
        dv[3][0] = enFactor * (-invJJ * sumBlock * (J21) + (b21));
        dv[3][1] = enFactor * (-invJJ * sumBlock * (J22) + (b22));
        dv[3][2] = enFactor * (-invJJ * sumBlock * (J23) + (b23));
        double fo[4][3];
        for (int bi = 0; bi < 4; ++bi)
            for (int k2 = 0; k2 < 3; ++k2)
                fo[bi][k2] = -(dv[bi][0] * (c2[k2] - c1[k2]) + dv[bi][1] * (c4[k2] - c3[k2]) +
                               dv[bi][2] * (c1[k2] - c3[k2]));
        if (bad3(fo[0]) || bad3(fo[1]) || bad3(fo[2]) || bad3(fo[3])) {
            excl_forceN(x, f, bs + 4 * i, kRS, 0);
        } else {
            for (int k2 = 0; k2 < 3; k2++) {
                f[bs[4 * i] + k2] += fo[0][k2];
                f[bs[4 * i + 1] + k2] += fo[1][k2];
                f[bs[4 * i + 2] + k2] += fo[2][k2];
                f[bs[4 * i + 3] + k2] += fo[3][k2];
            }
        }
    }
}

/* ---------------------------------------------------------------- boundary */
/* PlaneBoundaryElement::distance, Structure/BoundaryElementImpl.h:71-74. */
static inline double plane_distance(const double* pl, const double* p) {
    return (pl[0] * p[0] + pl[1] * p[1] + pl[2] * p[2] + pl[3]) /
           sqrt(pow(pl[0], 2) + pow(pl[1], 2) + pow(pl[2], 2));
}
/* BoundaryCylinderRepulsionExp::energy, Boundary/BoundaryCylinderRepulsionExp.cpp:27-63. */
double oracle_boundary_energy(const double* x, const medyan_system* s) {
    double U = 0.0;
    int32_t cum = 0;
    for (int32_t ib = 0; ib < s->n_planes; ++ib) {
        const double* pl = s->plane_eq + 4 * ib;
        int32_t nc = s->plane_nneighbors[ib];
        for (int32_t ic = 0; ic < nc; ++ic) {
            double r = plane_distance(pl, x + s->boundary_beads[cum + ic]);
            double R = -r / s->boundary_slen[cum + ic];
            U += s->boundary_k[cum + ic] * exp(R);
        }
        cum += nc;
    }
    return U;
}
/* BoundaryCylinderRepulsionExp::forces, BoundaryCylinderRepulsionExp.cpp:66-110. */
void oracle_boundary_forces(const double* x, double* f, const medyan_system* s) {
    int32_t cum = 0;
    for (int32_t ib = 0; ib < s->n_planes; ++ib) {
        const double* pl = s->plane_eq + 4 * ib;
        int32_t nc = s->plane_nneighbors[ib];
        for (int32_t ic = 0; ic < nc; ++ic) {
            const int32_t o = s->boundary_beads[cum + ic];
            double r = plane_distance(pl, x + o);
            double R = -r / s->boundary_slen[cum + ic];
            double f0 = s->boundary_k[cum + ic] * exp(R) / s->boundary_slen[cum + ic];
            f[o] += f0 * pl[0];
            f[o + 1] += f0 * pl[1];
            f[o + 2] += f0 * pl[2];
        }
        cum += nc;
    }
}

/* ------------------------------------------------------------------ manager */
static int has_br(const medyan_system* s, int bit) { return s->n_branch > 0 && ((s->branch_ff_mask >> bit) & 1); }

/* ForceFieldManager::computeEnergy, ForceFieldManager.cpp:96-207. */
double oracle_energy(const medyan_system* s, const double* x, double* e) {
    double tmp[MEDYAN_FF_COUNT];
    if (!e) e = tmp;
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) e[i] = 0.0;
    if (s->n_stretch) e[0] = oracle_fil_stretch_energy(x, s->n_stretch, s->stretch_beads, s->stretch_k, s->stretch_l0);
    if (s->n_bend) e[1] = oracle_fil_bend_energy(x, s->n_bend, s->bend_beads, s->bend_k, s->bend_theta0);
    if (s->n_linker)
        e[2] = oracle_two_point_spring_energy(x, s->n_linker, s->linker_beads, s->linker_k, s->linker_l0,
                                              s->linker_pos1, s->linker_pos2);
    if (s->n_motor)
        e[3] = oracle_two_point_spring_energy(x, s->n_motor, s->motor_beads, s->motor_k, s->motor_l0, s->motor_pos1,
                                              s->motor_pos2);
    if (has_br(s, 0))
        e[4] = oracle_branch_stretch_energy(x, s->n_branch, s->branch_beads, s->branch_stretch_k,
                                            s->branch_stretch_l0, s->branch_pos);
    if (has_br(s, 1))
        e[5] = oracle_branch_bend_energy(x, s->n_branch, s->branch_beads, s->branch_bend_k, s->branch_bend_theta0);
    if (has_br(s, 2))
        e[6] = oracle_branch_dihedral_energy(x, s->n_branch, s->branch_beads, s->branch_dihedral_k, s->branch_pos);
    if (has_br(s, 3))
        e[7] = oracle_branch_position_energy(x, s->n_branch, s->branch_beads, s->branch_position_k, s->branch_pos);
    if (s->n_excl) e[8] = oracle_excl_energy(x, s->n_excl, s->excl_beads, s->excl_k, s->excl_eqlen);
    if (s->n_boundary) e[9] = oracle_boundary_energy(x, s);
    double total = 0.0;
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
        if (e[i] <= -1) return INFINITY;
        total += e[i];
    }
    return total;
}

/* ForceFieldManager::computeForces, ForceFieldManager.cpp:242-290. */
void oracle_forces(const medyan_system* s, const double* x, double* f) {
    memset(f, 0, sizeof(double) * 3 * (size_t)s->n_beads);
    if (s->n_stretch) oracle_fil_stretch_forces(x, f, s->n_stretch, s->stretch_beads, s->stretch_k, s->stretch_l0);
    if (s->n_bend) oracle_fil_bend_forces(x, f, s->n_bend, s->bend_beads, s->bend_k, s->bend_theta0);
    if (s->n_linker)
        oracle_two_point_spring_forces(x, f, s->n_linker, s->linker_beads, s->linker_k, s->linker_l0, s->linker_pos1,
                                       s->linker_pos2);
    if (s->n_motor)
        oracle_two_point_spring_forces(x, f, s->n_motor, s->motor_beads, s->motor_k, s->motor_l0, s->motor_pos1,
                                       s->motor_pos2);
    if (has_br(s, 0))
        oracle_branch_stretch_forces(x, f, s->n_branch, s->branch_beads, s->branch_stretch_k, s->branch_stretch_l0,
                                     s->branch_pos);
    if (has_br(s, 1))
        oracle_branch_bend_forces(x, f, s->n_branch, s->branch_beads, s->branch_bend_k, s->branch_bend_theta0);
    if (has_br(s, 2))
        oracle_branch_dihedral_forces(x, f, s->n_branch, s->branch_beads, s->branch_dihedral_k, s->branch_pos);
    if (has_br(s, 3))
        oracle_branch_position_forces(x, f, s->n_branch, s->branch_beads, s->branch_position_k, s->branch_pos);
    if (s->n_excl) oracle_excl_forces(x, f, s->n_excl, s->excl_beads, s->excl_k, s->excl_eqlen);
    if (s->n_boundary) oracle_boundary_forces(x, f, s);
}

/* -------------------------------------------------------------------- CG */
typedef struct CGState {
    oracle_energy_fn efn;
    oracle_force_fn ffn;
    void* ctx;
    int ndof;
    double *force, *forcePrev, *searchDir, *coordLS, *coordMinE;
    int haveMinE;
    double minimumE, maxForcebackup, TotalEnergy;
} CGState;

/* CGMethod::maxF, CGMethod.hpp:202-212 (non-finite -> error). */
static double cg_maxf(const CGState* st, int* err) {
    double m = 0;
    for (int i = 0; i < st->ndof; ++i) m = stdmax(m, fabs(st->force[i]));
    if (!isfinite(m)) *err = 1;
    return m;
}
/* CGMethod.cpp:317-347: double accumulators. */
static double cg_dot(const double* a, const double* b, int n) {
    double r = 0.0;
    for (int i = 0; i < n; ++i) r += a[i] * b[i];
    return r;
}
/* resetCGParams lambda, CGMethod.hpp:963-972. */
static void cg_reset(CGState* st, int method, double* lastFDotF) {
    for (int i = 0; i < st->ndof; ++i) st->searchDir[i] = st->force[i] + 0.0 * st->searchDir[i];
    if (method != MEDYAN_CG_STEEPEST) *lastFDotF = cg_dot(st->force, st->force, st->ndof);
    if (method == MEDYAN_CG_POLAK_RIBIERE) memcpy(st->forcePrev, st->force, sizeof(double) * st->ndof);
}

/* CGMethod::backtrackingLineSearch, CGMethod.hpp:238-373 (running-average
   lambda is inactive: the manager is recreated every iteration, :1316-1317). */
static double cg_backtrack(CGState* st, const double* x, double maxDist, double maxForce, double lambdaMax,
                           double armijo, int* nEnergy, double* newEnergy) {
    *newEnergy = 0;
    if (maxForce == 0.0) return 0.0;
    double lambda = lambdaMax < maxDist / maxForce ? lambdaMax : maxDist / maxForce;
    const double currentEnergy = st->efn(st->ctx, x);
    ++*nEnergy;
    const double expectedSlope = cg_dot(st->searchDir, st->force, st->ndof);
    const double reducedSlope = armijo * expectedSlope;
    int done = 0;
    double energyLambda = 0.0;
    while (!done) {
        for (int i = 0; i < st->ndof; ++i) st->coordLS[i] = x[i] + lambda * st->searchDir[i];
        energyLambda = st->efn(st->ctx, st->coordLS);
        ++*nEnergy;
        const double ideal = -reducedSlope * lambda;
        if (lambda < 0 || ideal > 0) {
            done = 1;
            lambda = 0.0;
        }
        double energyChange = energyLambda - currentEnergy;
        if (energyChange <= ideal) done = 1;
        else lambda *= 0.5;
        if (lambda <= 0.0 || lambda <= 1e-8) {
            done = 1;
            lambda = 0.0;
            energyLambda = currentEnergy;
        }
    }
    st->TotalEnergy = energyLambda;
    *newEnergy = energyLambda;
    return lambda;
}

/* CGMethod::quadraticoptimization, CGMethod.hpp:644-765: iterated quadratic
   model through (x0,y0), (x1,y1), (x2,y2). The reference loops until one of
   its exits; the loop here stops after 100 models and returns x1. */
static double cg_quad_opt(CGState* st, const double* x, int* nEnergy, double x0, double x1, double x2, double y0,
                          double y1, double y2) {
    const double btlambda = x1;
    for (int it = 0; it < 100; ++it) {
        const double d = (x0 - x1) * (x0 - x2) * (x1 - x2);
        const double a = y0 * (x1 - x2) - y1 * (x0 - x2) + y2 * (x0 - x1);
        const double b = -(y0 * (x1 + x2) * (x1 - x2) - y1 * (x0 + x2) * (x0 - x2) + y2 * (x0 + x1) * (x0 - x1));
        const double lq = -b / (2 * a);
        if (fabs(lq - x1) / x1 < 1e-3) return lq;  /* LAMBDAQUADTOL */
        if (a / d < 0) return btlambda;           /* no minimum: the backtracking lambda */
        for (int i = 0; i < st->ndof; ++i) st->coordLS[i] = x[i] + lq * st->searchDir[i];
        const double eq = st->efn(st->ctx, st->coordLS);
        ++*nEnergy;
        if (fabs(eq - y1) / y1 < 1e-3) return lq;
        if (lq < x1) {
            if (eq < y0 && eq < y1) { x1 = lq; y1 = eq; }
            else { x0 = lq; y0 = eq; }
        } else if (x1 < lq) {
            if (eq < y1 && eq < y2) { x1 = lq; y1 = eq; }
            else { x2 = lq; y2 = eq; }
        } else {
            return x1;
        }
    }
    return x1;
}

/* CGMethod::quadraticLineSearchV2, CGMethod.hpp:521-640: backtracking with
   the Armijo slope 0.4, then, when at least one halving happened and a later
   trial's energy was above the accepted one, quadratic optimization through
   (0, E0), (lambda, E(lambda)) and (first lambda, its energy). The reference
   exits the program when the ideal energy change is positive; that ends the
   search with lambda = 0 here. */
static double cg_quadratic(CGState* st, const double* x, double maxDist, double maxForce, double lambdaMax,
                           int* nEnergy, double* newEnergy) {
    *newEnergy = 0;
    if (maxForce == 0.0) return 0.0;
    double lambda = lambdaMax < maxDist / maxForce ? lambdaMax : maxDist / maxForce;
    const double currentEnergy = st->efn(st->ctx, x);
    ++*nEnergy;
    const double slope = cg_dot(st->searchDir, st->force, st->ndof);
    double energyLambda = 0.0, prevEnergy = 0.0, prevLambda = 0.0;
    double lv[64], ev[64];
    int nv = 0, iter = 0, done = 0;
    while (!done) {
        iter++;
        for (int i = 0; i < st->ndof; ++i) st->coordLS[i] = x[i] + lambda * st->searchDir[i];
        energyLambda = st->efn(st->ctx, st->coordLS);
        ++*nEnergy;
        const double ideal = -0.4 * lambda * slope;
        if (ideal > 0) {
            lambda = 0.0;
            done = 1;
            break;
        }
        if (energyLambda - currentEnergy <= ideal) done = 1;
        else {
            prevLambda = lambda;
            prevEnergy = energyLambda;
            lambda *= 0.5;
        }
        if (nv < 64) {
            if (lambda <= 0.0 || lambda <= 1e-8) {
                lv[nv] = 0.0;
                ev[nv++] = currentEnergy;
            } else if (done) {
                lv[nv] = lambda;
                ev[nv++] = energyLambda;
            } else {
                lv[nv] = prevLambda;
                ev[nv++] = prevEnergy;
            }
        }
        if (lambda <= 0.0 || lambda <= 1e-8) {
            done = 1;
            lambda = 0.0;
        }
    }
    if (lambda > 0.0 && iter > 1 && energyLambda < currentEnergy) {
        int quad = 0, i;
        for (i = nv - 1; i >= 1; i--)
            if (energyLambda < ev[i]) quad = 1;
        if (quad) {
            const double lq = cg_quad_opt(st, x, nEnergy, 0.0, lambda, lv[i], currentEnergy, energyLambda, ev[i]);
            lambda = (lq <= 0.0 || lq <= 1e-8) ? 0.0 : lq;
        }
    }
    st->TotalEnergy = lambda > 0 ? energyLambda : currentEnergy;
    *newEnergy = energyLambda;
    return lambda;
}

static double sys_energy(void* ctx, const double* x) { return oracle_energy((const medyan_system*)ctx, x, NULL); }
static void sys_forces(void* ctx, const double* x, double* f) { oracle_forces((const medyan_system*)ctx, x, f); }
static void sys_individual(void* ctx, const double* x, double* per) { oracle_energy((const medyan_system*)ctx, x, per); }

/* computeIndividualEnergies + total (ForceFieldManager.cpp:209-240). */
static void fill_energies(oracle_individual_fn ifn, void* ctx, const double* x, double* per, double* total) {
    double e[MEDYAN_FF_COUNT];
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) e[i] = 0.0;
    ifn(ctx, x, e);
    double t = 0.0;
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
        per[i] = e[i];
        t += e[i];
    }
    *total = t;
}

int32_t oracle_cg_minimize(const medyan_system* s, const medyan_cg_params* p, double* x, double* f_out,
                           medyan_min_result* out) {
    return oracle_cg_minimize_cb(3 * s->n_beads, s->n_beads, p, x, f_out, out, sys_energy, sys_forces,
                                 sys_individual, (void*)s);
}

/* CGMethod::minimize, CGMethod.hpp:826-1743, with MController's recovery step
   (src/Controller/MController.h:273-339). */
int32_t oracle_cg_minimize_cb(int32_t ndof, int32_t n_beads, const medyan_cg_params* p, double* x, double* f_out,
                              medyan_min_result* out, oracle_energy_fn efn, oracle_force_fn ffn,
                              oracle_individual_fn ifn, void* ctx) {
    CGState st;
    memset(&st, 0, sizeof st);
    st.efn = efn;
    st.ffn = ffn;
    st.ctx = ctx;
    st.ndof = ndof;
    const int n = st.ndof;
    st.force = calloc((size_t)n + 1, sizeof(double));
    st.forcePrev = calloc((size_t)n + 1, sizeof(double));
    st.searchDir = calloc((size_t)n + 1, sizeof(double));
    st.coordLS = calloc((size_t)n + 1, sizeof(double));
    st.coordMinE = calloc((size_t)n + 1, sizeof(double));
    st.minimumE = INFINITY;
    medyan_min_result r;
    memset(&r, 0, sizeof r);
    r.energy_call_limit = p->energy_call_limit;
    r.grad_tol = p->grad_tol;
    r.energy_rel_tol = p->energy_rel_tol;
    r.force_call_limit = p->force_call_limit > 3 * n_beads ? p->force_call_limit : 3 * n_beads;
    r.grad_inf_norm = INFINITY;
    r.energy_rel_change = INFINITY;
    int32_t status = MEDYAN_OK;
    int err = 0;
    const int method = p->method;

    fill_energies(ifn, ctx, x, r.energy_before, &r.energy_before_total);
    ++r.num_energy_call;
    ffn(ctx, x, st.force);
    ++r.num_force_call;
    r.grad_inf_norm = cg_maxf(&st, &err);
    if (err) { status = MEDYAN_ERR_NONFINITE; goto done; }
    double prevEnergy = r.energy_before_total;
    int safeMode = 0, numIter = 0;
    double lastFDotF = 0;
    cg_reset(&st, method, &lastFDotF);

#define CALL_LIMIT() ((r.energy_call_limit != 0 && r.num_energy_call > r.energy_call_limit) || \
                      (r.force_call_limit != 0 && r.num_force_call > r.force_call_limit))
#define CONVERGED() (r.grad_inf_norm < r.grad_tol || r.energy_rel_change < r.energy_rel_tol)
    while (!CALL_LIMIT() && !CONVERGED()) {
        double beta = 0, newGrad = 0, prevGrad = 0, newEnergy = 0;
        numIter++;
        int nE = 0;
        /* QUADRATIC uses quadraticLineSearchV2 except in safe mode (CGMethod.hpp:1319-1332) */
        double lambda = (p->line_search && !safeMode)
                            ? cg_quadratic(&st, x, p->max_dist, r.grad_inf_norm, p->lambda_max, &nE, &newEnergy)
                            : cg_backtrack(&st, x, p->max_dist, r.grad_inf_norm, p->lambda_max, safeMode ? 0 : 0.4,
                                           &nE, &newEnergy);
        r.num_energy_call += nE;
        if (lambda == 0) {
            if (p->try_to_recover) {
                if (safeMode) {
                    double step = INFINITY;
                    for (int i = 0; i < n; ++i) {
                        double c = p->max_dist / fabs(st.searchDir[i]);
                        step = step < c ? step : c;
                    }
                    if (step == INFINITY) { status = MEDYAN_ERR_NONFINITE; goto done; }
                    for (int i = 0; i < n; ++i) x[i] += step * st.searchDir[i];
                    ffn(ctx, x, st.force);
                    ++r.num_force_call;
                    r.grad_inf_norm = cg_maxf(&st, &err);
                    if (err) { status = MEDYAN_ERR_NONFINITE; goto done; }
                    cg_reset(&st, method, &lastFDotF);
                    safeMode = 0;
                } else {
                    cg_reset(&st, method, &lastFDotF);
                    safeMode = 1;
                }
            } else {
                r.error_flags |= 1u;
                status = MEDYAN_ERR_LINE_SEARCH;
                r.num_iter = numIter;
                if (f_out) memcpy(f_out, st.force, sizeof(double) * n);
                if (out) *out = r;
                goto cleanup;
            }
        } else {
            for (int i = 0; i < n; ++i) x[i] += lambda * st.searchDir[i];
            ffn(ctx, x, st.force);
            ++r.num_force_call;
            r.grad_inf_norm = cg_maxf(&st, &err);
            if (err) { status = MEDYAN_ERR_NONFINITE; goto done; }
            r.energy_rel_change = fabs(newEnergy - prevEnergy) / fabs(prevEnergy);
            prevEnergy = newEnergy;
            if (method != MEDYAN_CG_STEEPEST) newGrad = cg_dot(st.force, st.force, n);
            if (method == MEDYAN_CG_POLAK_RIBIERE) prevGrad = cg_dot(st.force, st.forcePrev, n);
            if (method == MEDYAN_CG_FLETCHER_RIEVES) beta = newGrad / lastFDotF;
            else if (method == MEDYAN_CG_POLAK_RIBIERE) beta = stdmax(0.0, (newGrad - prevGrad) / lastFDotF);
            for (int i = 0; i < n; ++i) st.searchDir[i] = st.force[i] + beta * st.searchDir[i];
            if (cg_dot(st.searchDir, st.force, n) <= 0) cg_reset(&st, method, &lastFDotF);
            if (method == MEDYAN_CG_POLAK_RIBIERE) memcpy(st.forcePrev, st.force, sizeof(double) * n);
            /* copycoordsifminimumE when every |f| <= 10*gradTol late in the run (:1564-1566) */
            int relaxed = 1;
            for (int i = 0; i < n; ++i)
                if (fabs(st.force[i]) > 10 * p->grad_tol) { relaxed = 0; break; }
            if (relaxed && numIter > r.force_call_limit / 2 && st.TotalEnergy <= st.minimumE) {
                st.minimumE = st.TotalEnergy;
                st.maxForcebackup = r.grad_inf_norm;
                memcpy(st.coordMinE, x, sizeof(double) * n);
                st.haveMinE = 1;
            }
            if (method != MEDYAN_CG_STEEPEST) lastFDotF = newGrad;
        }
    }
    if (CALL_LIMIT() && st.haveMinE) memcpy(x, st.coordMinE, sizeof(double) * n);
#undef CALL_LIMIT
#undef CONVERGED
    fill_energies(ifn, ctx, x, r.energy_after, &r.energy_after_total);
    ++r.num_energy_call;
    r.num_iter = numIter;
done:
    if (f_out) memcpy(f_out, st.force, sizeof(double) * n);
    if (out) *out = r;
cleanup:
    free(st.force);
    free(st.forcePrev);
    free(st.searchDir);
    free(st.coordLS);
    free(st.coordMinE);
    return status;
}

/* ------------------------------------------------------------ neighbor list */
typedef struct Pair { int32_t key, nb; } Pair;
static int pair_cmp(const void* a, const void* b) {
    const Pair* p = a;
    const Pair* q = b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    if (p->nb != q->nb) return p->nb < q->nb ? -1 : 1;
    return 0;
}

/* HybridCylinderCylinderNL::initializeBinGrid (HybridNeighborListImpl.cpp:176-240)
   bin geometry and getBin (:243-286); pair rule from updateNeighborsbin
   (:332-471): key id > neighbor id, same filament needs |Δposition| > 2,
   rmin² <= d² <= rmax² with d² = Σ(Δ)² of the midpoints 0.5*(b1+b2)
   (Cylinder.cpp:48, Util/Math/Vec.hpp:378-384) against float rmax², rmin². */
int32_t oracle_nl_build(const medyan_cylinders* cy, const double* x, int32_t n_beads, const medyan_nl_params* p,
                        int32_t* pairs, int64_t capacity, int64_t* n_pairs) {
    (void)n_beads;
    const int32_t n = cy->n_cyl;
    const float rmaxsq = p->rmax * p->rmax, rminsq = p->rmin * p->rmin;
    const double bin = 1.125 * (double)sqrtf(rmaxsq);
    int grid[3];
    for (int d = 0; d < 3; ++d) {
        int size = (int)(p->grid_size[d]);
        grid[d] = (size % (int)bin == 0) ? (int)(size / bin) : (int)(size / bin + 1);
    }
    double* mid = malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
    int64_t* cell = malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) {
        const double* b1 = x + 3 * (int64_t)cy->bead1[i];
        const double* b2 = x + 3 * (int64_t)cy->bead2[i];
        int64_t idx = 0, stride = 1;
        for (int d = 0; d < 3; ++d) {
            mid[3 * i + d] = 0.5 * (b1[d] + b2[d]);
            double v = mid[3 * i + d];
            if (!(v >= 0) || v >= bin * grid[d]) {
                free(mid);
                free(cell);
                *n_pairs = 0;
                return MEDYAN_ERR_OUT_OF_GRID;
            }
            idx += (int64_t)(int)(v / bin) * stride;
            stride *= grid[d];
        }
        cell[i] = idx;
    }
    const int64_t ncell = (int64_t)grid[0] * grid[1] * grid[2];
    int64_t* start = calloc((size_t)ncell + 1, sizeof(int64_t));
    int32_t* order = malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) start[cell[i] + 1]++;
    for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
    int64_t* fillp = malloc(sizeof(int64_t) * (size_t)ncell);
    memcpy(fillp, start, sizeof(int64_t) * (size_t)ncell);
    for (int32_t i = 0; i < n; ++i) order[fillp[cell[i]]++] = i;
    free(fillp);

    int64_t cap = 1024, np = 0;
    Pair* out = malloc(sizeof(Pair) * (size_t)cap);
    for (int32_t i = 0; i < n; ++i) {
        int64_t ci = cell[i];
        int ix = (int)(ci % grid[0]), iy = (int)((ci / grid[0]) % grid[1]), iz = (int)(ci / ((int64_t)grid[0] * grid[1]));
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                    if (jx < 0 || jx >= grid[0] || jy < 0 || jy >= grid[1] || jz < 0 || jz >= grid[2]) continue;
                    int64_t cj = jx + (int64_t)grid[0] * (jy + (int64_t)grid[1] * jz);
                    for (int64_t q = start[cj]; q < start[cj + 1]; ++q) {
                        int32_t j = order[q];
                        if (cy->id[i] <= cy->id[j]) continue;
                        if (cy->filament_id[i] == cy->filament_id[j]) {
                            int ds = cy->position_on_filament[i] - cy->position_on_filament[j];
                            if (abs(ds) <= 2) continue;
                        }
                        double ex = mid[3 * j] - mid[3 * i], ey = mid[3 * j + 1] - mid[3 * i + 1];
                        double ez = mid[3 * j + 2] - mid[3 * i + 2];
                        double d2 = ex * ex + ey * ey + ez * ez;
                        if (d2 > (double)rmaxsq || d2 < (double)rminsq) continue;
                        if (np == cap) {
                            cap *= 2;
                            out = realloc(out, sizeof(Pair) * (size_t)cap);
                        }
                        out[np].key = i;
                        out[np].nb = j;
                        ++np;
                    }
                }
    }
    qsort(out, (size_t)np, sizeof(Pair), pair_cmp);
    *n_pairs = np;
    int32_t status = MEDYAN_OK;
    if (pairs) {
        if (np > capacity) status = MEDYAN_ERR_CAPACITY;
        else
            for (int64_t k = 0; k < np; ++k) {
                pairs[2 * k] = out[k].key;
                pairs[2 * k + 1] = out[k].nb;
            }
    }
    free(out);
    free(order);
    free(start);
    free(cell);
    free(mid);
    return status;
}

/* CylinderExclVolume::vectorize, Volume/CylinderExclVolume.cpp:66-107:
   skip a pair when the neighbor's branching cylinder is the key cylinder;
   krep is the max of the two cylinders' constants when their types differ. */
int64_t oracle_excl_vectorize(const medyan_cylinders* c, const int32_t* pairs, int64_t n_pairs, int32_t* beads,
                              double* k, double* eqlen) {
    int64_t m = 0;
    for (int64_t q = 0; q < n_pairs; ++q) {
        int32_t ci = pairs[2 * q], cn = pairs[2 * q + 1];
        if (c->branching_cylinder && c->branching_cylinder[cn] == ci) continue;
        if (beads) {
            beads[4 * m] = 3 * c->bead1[ci];
            beads[4 * m + 1] = 3 * c->bead2[ci];
            beads[4 * m + 2] = 3 * c->bead1[cn];
            beads[4 * m + 3] = 3 * c->bead2[cn];
            eqlen[2 * m] = c->eq_length[ci];
            eqlen[2 * m + 1] = c->eq_length[cn];
            if (c->type[ci] != c->type[cn]) {
                double ki = c->excl_k[ci], kn = c->excl_k[cn];
                k[m] = ki < kn ? kn : ki;
            } else {
                k[m] = c->excl_k[ci];
            }
        }
        ++m;
    }
    return m;
}

/* BoundaryCylinderNL::updateNeighbors (Structure/NeighborListImpl.cpp:738-753)
   and BoundaryCylinderRepulsion::vectorize (Boundary/BoundaryCylinderRepulsion.cpp:33-88):
   per plane, every cylinder whose midpoint b1*(1-0.5) + 0.5*b2 is closer than
   the float cutoff contributes its first bead (minus-end cylinders only) and
   its second bead. */
int64_t oracle_boundary_vectorize(const medyan_cylinders* c, const double* x, const medyan_boundary_params* b,
                                  int32_t* beads, double* k, double* slen, int32_t* nneighbors) {
    int64_t m = 0;
    for (int32_t p = 0; p < b->n_planes; ++p) {
        const double* pl = b->plane_eq + 4 * p;
        int32_t cnt = 0;
        for (int32_t i = 0; i < c->n_cyl; ++i) {
            double mid[3];
            midpt(mid, x + 3 * (int64_t)c->bead1[i], x + 3 * (int64_t)c->bead2[i], 0.5);
            if (!(plane_distance(pl, mid) < (double)b->cutoff)) continue;
            if (c->is_minus_end && c->is_minus_end[i]) {
                if (beads) {
                    beads[m] = 3 * c->bead1[i];
                    k[m] = b->k;
                    slen[m] = b->screen_length;
                }
                ++m;
                ++cnt;
            }
            if (beads) {
                beads[m] = 3 * c->bead2[i];
                k[m] = b->k;
                slen[m] = b->screen_length;
            }
            ++m;
            ++cnt;
        }
        if (nneighbors) nneighbors[p] = cnt;
    }
    return m;
}

/* ForceFieldManager::computeHessian, ForceFieldManager.cpp:354-398: for each
   degree of freedom i, forces at copies of the coordinates with x_i + delta
   and x_i - delta (delta a float, as the reference's hessDelta), and
   H[i][j] = (float)(-(Fp[j] - Fm[j]) / (2 * delta)) stored in a double. */
void oracle_hessian(const medyan_system* s, const double* x, float delta, double* H) {
    const int n = 3 * s->n_beads;
    double* cp = (double*)malloc(sizeof(double) * (size_t)n);
    double* cm = (double*)malloc(sizeof(double) * (size_t)n);
    double* fp = (double*)malloc(sizeof(double) * (size_t)n);
    double* fm = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        memcpy(cp, x, sizeof(double) * (size_t)n);
        memcpy(cm, x, sizeof(double) * (size_t)n);
        cp[i] += delta;
        cm[i] -= delta;
        oracle_forces(s, cp, fp);
        oracle_forces(s, cm, fm);
        for (int j = 0; j < n; ++j) {
            float h = -(fp[j] - fm[j]) / (2 * delta);
            H[(size_t)i * n + j] = h;
        }
    }
    free(cp);
    free(cm);
    free(fp);
    free(fm);
}

/* The force magnitudes of ForceFieldManager::assignallforcemags
   (ForceFieldManager.cpp:346-351): linker and motor stretchforce = f0/invL
   (LinkerStretchingHarmonic.cpp:227-293, MotorGhostStretchingHarmonic.cpp:274-339),
   and per branch point the force each enabled branching force field puts on
   the third bead of its bead set, added in force-field order (stretching,
   bending, dihedral, position; their forces() store f3 as stretchforce).
   The branch value is read off each force field's forces on an otherwise
   empty force array, which is the third bead's contribution whenever the
   bead set's beads are distinct, as in every branch point. */
void oracle_force_magnitudes(const medyan_system* s, const double* x, double* lin, double* mot, double* br) {
    double v1[3], v2[3];
    for (int pass = 0; pass < 2; ++pass) {
        const int32_t n = pass ? s->n_motor : s->n_linker;
        const int32_t* bs = pass ? s->motor_beads : s->linker_beads;
        const double *k = pass ? s->motor_k : s->linker_k, *l0 = pass ? s->motor_l0 : s->linker_l0;
        const double *p1 = pass ? s->motor_pos1 : s->linker_pos1, *p2 = pass ? s->motor_pos2 : s->linker_pos2;
        double* out = pass ? mot : lin;
        if (!out) continue;
        for (int32_t i = 0; i < n; ++i) {
            midpt(v1, x + bs[4 * i], x + bs[4 * i + 1], p1[i]);
            midpt(v2, x + bs[4 * i + 2], x + bs[4 * i + 3], p2[i]);
            double dist = tpd(v1, v2);
            double invL = 1 / dist;
            double f0 = k[i] * (dist - l0[i]) * invL;
            out[i] = f0 / invL;
        }
    }
    if (!br || s->n_branch == 0) return;
    double* tmp = (double*)calloc(3 * (size_t)s->n_beads, sizeof(double));
    for (int32_t i = 0; i < s->n_branch; ++i) {
        const int32_t* b = s->branch_beads + 4 * i;
        double acc[3] = {0.0, 0.0, 0.0};
        for (int ffi = 0; ffi < 4; ++ffi) {
            if (!has_br(s, ffi)) continue;
            if (ffi == 0)
                oracle_branch_stretch_forces(x, tmp, 1, b, s->branch_stretch_k + i, s->branch_stretch_l0 + i,
                                             s->branch_pos + i);
            else if (ffi == 1)
                oracle_branch_bend_forces(x, tmp, 1, b, s->branch_bend_k + i, s->branch_bend_theta0 + i);
            else if (ffi == 2)
                oracle_branch_dihedral_forces(x, tmp, 1, b, s->branch_dihedral_k + i, s->branch_pos + i);
            else
                oracle_branch_position_forces(x, tmp, 1, b, s->branch_position_k + i, s->branch_pos + i);
            for (int d = 0; d < 3; ++d) acc[d] += tmp[b[2] + d];
            for (int j = 0; j < 4; ++j)
                for (int d = 0; d < 3; ++d) tmp[b[j] + d] = 0.0;
        }
        for (int d = 0; d < 3; ++d) br[3 * i + d] = acc[d];
    }
    free(tmp);
}

/* BoundaryCylinderRepulsion::computeLoadForces with BoundaryCylinderRepulsionExp
   (BoundaryCylinderRepulsion.cpp:125-196, BoundaryCylinderRepulsionExp.cpp:113-118):
   the tip's cylinder is a neighbor of a plane when its midpoint lies within
   the boundary cutoff (the boundary neighbor list, as oracle_boundary_vectorize);
   loads of tip t at out[offset_t + i], i < n_mon[t]. */
void oracle_boundary_load_forces(const medyan_cylinders* c, const double* x, const medyan_boundary_params* b,
                                 int32_t n_tips, const int32_t* cyl, const int32_t* plus_end, const int32_t* n_mon,
                                 const double* mon_size, double* out) {
    int64_t o = 0;
    for (int32_t t = 0; t < n_tips; ++t) {
        const int32_t ci = cyl[t];
        const double* bo = x + 3 * (int64_t)(plus_end[t] ? c->bead1[ci] : c->bead2[ci]);
        const double* bd = x + 3 * (int64_t)(plus_end[t] ? c->bead2[ci] : c->bead1[ci]);
        double v[3] = {bd[0] - bo[0], bd[1] - bo[1], bd[2] - bo[2]};
        double m = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double dir[3] = {v[0] / m, v[1] / m, v[2] / m};
        for (int32_t i = 0; i < n_mon[t]; ++i) out[o + i] = 0.0;
        double mid[3];
        midpt(mid, x + 3 * (int64_t)c->bead1[ci], x + 3 * (int64_t)c->bead2[ci], 0.5);
        for (int32_t p = 0; p < b->n_planes; ++p) {
            const double* pl = b->plane_eq + 4 * p;
            if (!(plane_distance(pl, mid) < (double)b->cutoff)) continue;
            for (int32_t i = 0; i < n_mon[t]; ++i) {
                double sft = i * mon_size[t];
                double nc[3] = {bd[0] + sft * dir[0], bd[1] + sft * dir[1], bd[2] + sft * dir[2]};
                double proj = -(pl[0] * dir[0] + pl[1] * dir[1] + pl[2] * dir[2]);
                if (proj < 0.0) proj = 0.0;
                double R = -plane_distance(pl, nc) / b->screen_length;
                out[o + i] += proj * (b->k * exp(R) / b->screen_length);
            }
        }
        o += n_mon[t];
    }
}

// potentials.cuh — per-interaction energy and force of every force field on
// the path. Template parameter R is the arithmetic type after the FP64
// geometry step (double: FP64 path, float: mixed path). With R = double each
// function evaluates the reference's expressions in the reference's order.
//
// Forces are returned per bead (caller accumulates); energies as double.
//
// The position type P3 is V3 (FP64 coordinates) everywhere but in the
// directional derivatives (diff.cu), which pass DV3 positions with R = Dual
// (dual.cuh): the same formulas then also return their derivative along the
// direction the positions carry.
#pragma once

#include "device_math.cuh"
#include "dual.cuh"

namespace mb {

// ----------------------------------------------------------------------------
// Bond length and its deviation from a rest length.
// FP64: dist = sqrt(d.d), dev = dist - l0 (twoPointDistance - eql).
// Mixed: dev = (d.d - l0^2)/(dist + l0) with d.d and d.d - l0^2 in FP64, so
// the deviation keeps float relative accuracy when dist ~ l0.
// ----------------------------------------------------------------------------
template <class R>
struct LenDev {
    R dist, dev;
};
template <class R>
__device__ __forceinline__ LenDev<R> length_dev(double dx, double dy, double dz, double l0);
template <>
__device__ __forceinline__ LenDev<double> length_dev<double>(double dx, double dy, double dz, double l0) {
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    return LenDev<double>{dist, dist - l0};
}
template <>
__device__ __forceinline__ LenDev<float> length_dev<float>(double dx, double dy, double dz, double l0) {
    double d2 = dx * dx + dy * dy + dz * dz;
    float dist = sqrtf(float(d2));
    float dev = float(d2 - l0 * l0) / (dist + float(l0));
    return LenDev<float>{dist, dev};
}
// Dual differences (directional derivatives): the FP64 form.
template <class R>
__device__ __forceinline__ LenDev<R> length_dev(const Dual& dx, const Dual& dy, const Dual& dz, double l0) {
    const Dual dist = sqrt(dx * dx + dy * dy + dz * dz);
    return LenDev<R>{dist, dist - l0};
}

// ---------------------------------------------------------------------------
// FilamentStretchingHarmonic, Filament/FilamentStretchingHarmonic.cpp:185-275.
// ---------------------------------------------------------------------------
template <class R, class P3 = V3>
__device__ __forceinline__ double stretch_energy(const P3& c1, const P3& c2, double k, double l0) {
    LenDev<R> L = length_dev<R>(c2.x - c1.x, c2.y - c1.y, c2.z - c1.z, l0);
    return double(R(0.5) * R(k) * L.dev * L.dev);
}
// Force on c2 (c1 receives the negative).
template <class R, class P3 = V3>
__device__ __forceinline__ T3<R> stretch_force(const P3& c1, const P3& c2, double k, double l0) {
    LenDev<R> L = length_dev<R>(c2.x - c1.x, c2.y - c1.y, c2.z - c1.z, l0);
    R invL = R(1) / L.dist;
    R f0 = R(k) * L.dev * invL;
    T3<R> r = diff<R>(c1, c2);
    return T3<R>{-f0 * r.x, -f0 * r.y, -f0 * r.z};
}

// ---------------------------------------------------------------------------
// FilamentBendingCosine, Filament/FilamentBendingCosine.cpp:199-345, and
// BranchingBendingCosine, Branching/BranchingBendingCosine.cpp:196-330.
// r1 = p2 - p1 and r2 = p4 - p3 (filament: p3 = p2).
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ double bend_energy(const T3<R>& r1, const T3<R>& r2, double k, double eqt) {
    R L1 = sqrt(dot(r1, r1));
    R L2 = sqrt(dot(r2, r2));
    R L1L2 = L1 * L2;
    R l1l2 = dot(r1, r2);
    if (are_equal(eqt, 0.0)) {
        if constexpr (sizeof(R) == 4) {
            // 1 - cos = |r1 x r2|^2 / (L1L2 (L1L2 + r1.r2)): no cancellation near straight.
            R cx = r1.y * r2.z - r1.z * r2.y, cy = r1.z * r2.x - r1.x * r2.z, cz = r1.x * r2.y - r1.y * r2.x;
            R s2 = cx * cx + cy * cy + cz * cz;
            R den = L1L2 * (L1L2 + l1l2);
            R one_minus = den > R(0) ? s2 / den : R(1) - l1l2 / L1L2;
            if (one_minus > R(2)) one_minus = R(2);
            return double(R(k) * one_minus);
        } else {
            R x = l1l2 / L1L2;
            if (x < R(-1)) x = R(-1);
            else if (x > R(1)) x = R(1);
            return double(R(k) * (R(1) - x));
        }
    }
    R x = l1l2 / L1L2;
    if (x < R(-1)) x = R(-1);
    else if (x > R(1)) x = R(1);
    R cosA = x;
    R sinA = stdmax<R>(sqrt(R(1) - cosA * cosA), R(0));
    R cosAmB = cosA * R(cos(eqt)) + sinA * R(sin(eqt));
    return double(R(k) * (R(1) - cosAmB));
}

// Returns (Fr1, Fr2): the filament bead forces are -Fr1, Fr1 - Fr2, Fr2; the
// branch bead forces are -Fr1, Fr1, -Fr2, Fr2.
template <class R>
__device__ __forceinline__ void bend_force(const T3<R>& r1, const T3<R>& r2, double kb, double eqt, T3<R>& Fr1,
                                           T3<R>& Fr2) {
    R L1sq = dot(r1, r1);
    R L2sq = dot(r2, r2);
    R l1l2 = dot(r1, r2);
    R A = R(1) / sqrt(L1sq * L2sq);
    R x = l1l2 * A;
    R B = x / L1sq;
    R C = x / L2sq;
    R k;
    if (are_equal(eqt, 0.0)) {
        k = R(kb);
    } else {
        if (fabs(fabs(x) - R(1)) < R(0.001)) x = R(0.999) * x;
        if (x < R(-1)) x = R(-1);
        else if (x > R(1)) x = R(1);
        R cosp = x;
        R sinp = sqrt(stdmax<R>((R(1) - cosp * cosp), R(0)));
        R sinpmq = sinp * R(cos(eqt)) - cosp * R(sin(eqt));
        k = R(kb) * sinpmq / sinp;
    }
    Fr1 = T3<R>{k * (r2.x * A - r1.x * B), k * (r2.y * A - r1.y * B), k * (r2.z * A - r1.z * B)};
    Fr2 = T3<R>{k * (r1.x * A - r2.x * C), k * (r1.y * A - r2.y * C), k * (r1.z * A - r2.z * C)};
}

// ---------------------------------------------------------------------------
// LinkerStretchingHarmonic (Linker/LinkerStretchingHarmonic.cpp:191-292) and
// MotorGhostStretchingHarmonic (MotorGhost/...Harmonic.cpp:234-345): a spring
// between points at fractions p1, p2 along two cylinders. Midpoints in FP64.
// ---------------------------------------------------------------------------
template <class R, class P3 = V3>
__device__ __forceinline__ double spring_energy(const P3& c1, const P3& c2, const P3& c3, const P3& c4, double k,
                                                double l0, double p1, double p2) {
    P3 v1 = midpoint(c1, c2, p1);
    P3 v2 = midpoint(c3, c4, p2);
    LenDev<R> L = length_dev<R>(v2.x - v1.x, v2.y - v1.y, v2.z - v1.z, l0);
    return double(R(0.5) * R(k) * L.dev * L.dev);
}
// Returns Fl; bead forces are -Fl(1-p1), -Fl p1, Fl(1-p2), Fl p2.
template <class R, class P3 = V3>
__device__ __forceinline__ T3<R> spring_force(const P3& c1, const P3& c2, const P3& c3, const P3& c4, double k,
                                              double l0, double p1, double p2) {
    P3 v1 = midpoint(c1, c2, p1);
    P3 v2 = midpoint(c3, c4, p2);
    LenDev<R> L = length_dev<R>(v2.x - v1.x, v2.y - v1.y, v2.z - v1.z, l0);
    R invL = R(1) / L.dist;
    R f0 = R(k) * L.dev * invL;
    T3<R> l = diff<R>(v1, v2);
    return T3<R>{-f0 * l.x, -f0 * l.y, -f0 * l.z};
}

// ---------------------------------------------------------------------------
// BranchingStretchingHarmonic, Branching/BranchingStretchingHarmonic.cpp:195-266.
// ---------------------------------------------------------------------------
template <class R, class P3 = V3>
__device__ __forceinline__ double branch_stretch_energy(const P3& c1, const P3& c2, const P3& c3, double k, double l0,
                                                        double pos) {
    P3 v1 = midpoint(c1, c2, pos);
    LenDev<R> L = length_dev<R>(c3.x - v1.x, c3.y - v1.y, c3.z - v1.z, l0);
    return double(R(0.5) * R(k) * L.dev * L.dev);
}
// Returns g = f0*r1; bead forces are -g(pos-1), g pos, -g.
template <class R, class P3 = V3>
__device__ __forceinline__ T3<R> branch_stretch_force(const P3& c1, const P3& c2, const P3& c3, double k, double l0,
                                                      double pos) {
    P3 v1 = midpoint(c1, c2, pos);
    LenDev<R> L = length_dev<R>(c3.x - v1.x, c3.y - v1.y, c3.z - v1.z, l0);
    R invL = R(1) / L.dist;
    R f0 = R(k) * L.dev * invL;
    T3<R> r1 = diff<R>(v1, c3);
    return T3<R>{f0 * r1.x, f0 * r1.y, f0 * r1.z};
}

// Virtual plus end for a branch at pos == 1 (Branching/BranchingDihedralCosine.cpp:236-243).
template <class P3>
__device__ __forceinline__ double virtual_plus_end(const P3& c1, P3& c2, double pos) {
    if (are_equal(pos, 1.0)) {
        const double position = 0.5;
        c2 = P3{(1 / position) * (c2.x - (1 - position) * c1.x), (1 / position) * (c2.y - (1 - position) * c1.y),
                (1 / position) * (c2.z - (1 - position) * c1.z)};
        return position;
    }
    return pos;
}

// ---------------------------------------------------------------------------
// BranchingDihedralCosine::energy, BranchingDihedralCosine.cpp:211-263.
// ---------------------------------------------------------------------------
template <class R, class P3 = V3>
__device__ __forceinline__ R branch_dihedral_energy_r(const P3& c1, P3 c2, const P3& c3, const P3& c4, double k,
                                                      double pos) {
    double position = virtual_plus_end(c1, c2, pos);
    P3 mp = midpoint(c1, c2, position);
    // vectorProduct(n1, mp, c2, mp, c3) and vectorProduct(n2, c3, c4, mp, c3).
    T3<R> a = diff<R>(mp, c2), b = diff<R>(mp, c3), c = diff<R>(c3, c4);
    T3<R> n1{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    T3<R> n2{c.y * b.z - c.z * b.y, c.z * b.x - c.x * b.z, c.x * b.y - c.y * b.x};
    R m1 = sqrt(n1.x * n1.x + n1.y * n1.y + n1.z * n1.z);
    R m2 = sqrt(n2.x * n2.x + n2.y * n2.y + n2.z * n2.z);
    n1 = T3<R>{n1.x / m1, n1.y / m1, n1.z / m1};
    n2 = T3<R>{n2.x / m2, n2.y / m2, n2.z / m2};
    return R(k) * (R(1) - dot(n1, n2));
}
template <class R, class P3 = V3>
__device__ __forceinline__ double branch_dihedral_energy(const P3& c1, const P3& c2, const P3& c3, const P3& c4,
                                                         double k, double pos) {
    return double(branch_dihedral_energy_r<R, P3>(c1, c2, c3, c4, k, pos));
}

// BranchingDihedralCosine::forces (LAMMPS form), BranchingDihedralCosine.cpp:268-490.
template <class R, class P3 = V3>
__device__ __forceinline__ void branch_dihedral_force(const P3& c1, P3 c2, const P3& c3, const P3& c4, double k,
                                                      double pos, T3<R>& L1, T3<R>& L2, T3<R>& L3, T3<R>& L4) {
    double position = virtual_plus_end(c1, c2, pos);
    P3 mp = midpoint(c1, c2, position);
    T3<R> vb1 = diff<R>(mp, c2), vb2 = diff<R>(mp, c3), vb3 = diff<R>(c3, c4);
    R vb2xm = -vb2.x, vb2ym = -vb2.y, vb2zm = -vb2.z;
    R ax = vb1.y * vb2zm - vb1.z * vb2ym;
    R ay = vb1.z * vb2xm - vb1.x * vb2zm;
    R az = vb1.x * vb2ym - vb1.y * vb2xm;
    R bx = vb3.y * vb2zm - vb3.z * vb2ym;
    R by = vb3.z * vb2xm - vb3.x * vb2zm;
    R bz = vb3.x * vb2ym - vb3.y * vb2xm;
    R rasq = ax * ax + ay * ay + az * az;
    R rbsq = bx * bx + by * by + bz * bz;
    R rgsq = vb2xm * vb2xm + vb2ym * vb2ym + vb2zm * vb2zm;
    R rg = sqrt(rgsq);
    R rginv = 0, ra2inv = 0, rb2inv = 0;
    if (rg > 0) rginv = R(1) / rg;
    if (rasq > 0) ra2inv = R(1) / rasq;
    if (rbsq > 0) rb2inv = R(1) / rbsq;
    R rabinv = sqrt(ra2inv * rb2inv);
    R s = rg * rabinv * (ax * vb3.x + ay * vb3.y + az * vb3.z);
    R fg = vb1.x * vb2xm + vb1.y * vb2ym + vb1.z * vb2zm;
    R hg = vb3.x * vb2xm + vb3.y * vb2ym + vb3.z * vb2zm;
    R fga = fg * ra2inv * rginv;
    R hgb = hg * rb2inv * rginv;
    R gaa = -ra2inv * rg;
    R gbb = rb2inv * rg;
    R dtfx = gaa * ax, dtfy = gaa * ay, dtfz = gaa * az;
    R dtgx = fga * ax - hgb * bx, dtgy = fga * ay - hgb * by, dtgz = fga * az - hgb * bz;
    R dthx = gbb * bx, dthy = gbb * by, dthz = gbb * bz;
    R df = -R(k) * s;
    R sx2 = df * dtgx, sy2 = df * dtgy, sz2 = df * dtgz;
    L4 = T3<R>{df * dthx, df * dthy, df * dthz};
    L3 = T3<R>{-sx2 - L4.x, -sy2 - L4.y, -sz2 - L4.z};
    const R P = R(position);
    if (are_equal(pos, 1.0)) {
        T3<R> L2p{df * dtfx, df * dtfy, df * dtfz};
        L2 = T3<R>{sx2 - L2p.x, sy2 - L2p.y, sz2 - L2p.z};
        R factor = (P - R(1)) / P;
        L1 = T3<R>{L2p.x * factor, L2p.y * factor, L2p.z * factor};
        factor = (R(1) / P);
        L2.x += L2p.x * factor;
        L2.y += L2p.y * factor;
        L2.z += L2p.z * factor;
    } else {
        L2 = T3<R>{df * dtfx, df * dtfy, df * dtfz};
        T3<R> Lmp{sx2 - L2.x, sy2 - L2.y, sz2 - L2.z};
        L1 = T3<R>{(R(1) - P) * Lmp.x, (R(1) - P) * Lmp.y, (R(1) - P) * Lmp.z};
        L2.x += (P)*Lmp.x;
        L2.y += (P)*Lmp.y;
        L2.z += (P)*Lmp.z;
    }
}

// ---------------------------------------------------------------------------
// BranchingPositionCosine, Branching/BranchingPositionCosine.cpp:190-440.
// ---------------------------------------------------------------------------
template <class R, class P3 = V3>
__device__ __forceinline__ R branch_position_energy_r(const P3& c1, P3 c2, const P3& c3, double k, double pos) {
    double position = virtual_plus_end(c1, c2, pos);
    P3 mp = midpoint(c1, c2, position);
    T3<R> a = diff<R>(mp, c2), b = diff<R>(mp, c3);
    R X = sqrt(dot(a, a));
    R D = sqrt(dot(b, b));
    R XD = X * D;
    R xd = dot(a, b);
    R x = xd / XD;
    if (fabs(fabs(x) - R(1)) < R(0.001)) {
        xd = R(0.999) * XD;
        x = xd / XD;
    }
    if (x < R(-1)) x = R(-1);
    else if (x > R(1)) x = R(1);
    R cosp = x;
    const double posheta = 0.5 * M_PI;
    R sinp = sqrt(stdmax<R>((R(1) - cosp * cosp), R(0)));
    R cospmq = cosp * R(cos(posheta)) + sinp * R(sin(posheta));
    return R(k) * (R(1) - cospmq);
}
template <class R, class P3 = V3>
__device__ __forceinline__ double branch_position_energy(const P3& c1, const P3& c2, const P3& c3, double k,
                                                         double pos) {
    return double(branch_position_energy_r<R, P3>(c1, c2, c3, k, pos));
}
template <class R, class P3 = V3>
__device__ __forceinline__ void branch_position_force(const P3& c1, P3 c2, const P3& c3, double k, double pos,
                                                      T3<R>& F1, T3<R>& F2, T3<R>& F3) {
    double position = virtual_plus_end(c1, c2, pos);
    P3 mp = midpoint(c1, c2, position);
    T3<R> r1 = diff<R>(mp, c2), r2 = diff<R>(mp, c3);
    R Xsq = dot(r1, r1);
    R Dsq = dot(r2, r2);
    R xd = dot(r1, r2);
    R A = R(1) / sqrt(Xsq * Dsq);
    R x = xd * A;
    R B = x / Xsq;
    R C = x / Dsq;
    if (fabs(fabs(x) - R(1)) < R(0.001)) x = R(0.999) * x;
    if (x < R(-1)) x = R(-1);
    else if (x > R(1)) x = R(1);
    R cosp = x;
    const double posheta = 0.5 * M_PI;
    R sinp = sqrt(stdmax<R>((R(1) - cosp * cosp), R(0)));
    R sinpmq = sinp * R(cos(posheta)) - cosp * R(sin(posheta));
    R kk = R(k) * sinpmq / sinp;
    T3<R> Fr1{kk * (r2.x * A - r1.x * B), kk * (r2.y * A - r1.y * B), kk * (r2.z * A - r1.z * B)};
    T3<R> Fr2{kk * (r1.x * A - r2.x * C), kk * (r1.y * A - r2.y * C), kk * (r1.z * A - r2.z * C)};
    const R P = R(position);
    T3<R> fmp{-Fr1.x - Fr2.x, -Fr1.y - Fr2.y, -Fr1.z - Fr2.z};
    T3<R> f1t{(R(1) - P) * fmp.x, (R(1) - P) * fmp.y, (R(1) - P) * fmp.z};
    T3<R> f2t{Fr1.x + P * fmp.x, Fr1.y + P * fmp.y, Fr1.z + P * fmp.z};
    F3 = Fr2;
    if (are_equal(pos, 1.0)) {
        R factor = (P - R(1)) / P;
        F1 = T3<R>{f1t.x + f2t.x * factor, f1t.y + f2t.y * factor, f1t.z + f2t.z * factor};
        F2 = T3<R>{f2t.x * (R(1) / P), f2t.y * (R(1) / P), f2t.z * (R(1) / P)};
    } else {
        F1 = f1t;
        F2 = f2t;
    }
}

// ---------------------------------------------------------------------------
// BoundaryCylinderRepulsionExp, Boundary/BoundaryCylinderRepulsionExp.cpp:27-110,
// plane distance from PlaneBoundaryElement::distance (BoundaryElementImpl.h:71-74),
// always in FP64 because it is formed from absolute coordinates.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double plane_distance(const double4& pl, const V3& p) {
    return (pl.x * p.x + pl.y * p.y + pl.z * p.z + pl.w) / sqrt(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z);
}
__device__ __forceinline__ Dual plane_distance(const double4& pl, const DV3& p) {
    return (pl.x * p.x + pl.y * p.y + pl.z * p.z + pl.w) / sqrt(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z);
}
template <class R, class P3 = V3>
__device__ __forceinline__ double boundary_energy(const double4& pl, const P3& p, double k, double slen) {
    const auto r = plane_distance(pl, p);
    R Rr = R(-r / slen);
    return double(R(k) * exp(Rr));
}
template <class R, class P3 = V3>
__device__ __forceinline__ R boundary_force_mag(const double4& pl, const P3& p, double k, double slen) {
    const auto r = plane_distance(pl, p);
    R Rr = R(-r / slen);
    return R(k) * exp(Rr) / R(slen);
}

}  // namespace mb

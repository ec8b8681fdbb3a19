// quadrature.cuh — the composite Simpson fallbacks of the excluded-volume
// potential for pairs whose analytic integral is not finite:
// CylinderExclVolRepulsion::energyN (400 x 400 grid) and ::forceN
// (10^4 x 10^4 grid), Volume/CylinderExclVolRepulsion.cpp:884-1256. Each is
// evaluated by one whole block, all threads splitting the grid.
//
// Every translation unit that includes this header gets its own copy of the
// abscissa grids (device variables are per module) and must fill them once
// per device with k_fill_quadrature_grids before the fallbacks run. Include
// only from files built with --fmad=false, so that the sums round as the
// reference's loops do.
#pragma once

#include "excl.cuh"

namespace mb {
namespace {

// r^2(s, t) of CylinderExclVolRepulsion.h:50-71.
__device__ __forceinline__ double r2_of(double a, double b, double c, double d, double e, double F, double s,
                                        double t) {
    return c + 2 * s * e + s * s * a - 2 * t * F - 2 * s * t * d + t * t * b;
}

struct Six {
    double a, b, c, d, e, F;
};
__device__ __forceinline__ Six six_of(const V3& c1, const V3& c2, const V3& c3, const V3& c4) {
    T3<double> r12 = diff<double>(c1, c2), r34 = diff<double>(c3, c4), r31 = diff<double>(c3, c1);
    return Six{dot(r12, r12), dot(r34, r34), dot(r31, r31), dot(r12, r34), dot(r12, r31), dot(r34, r31)};
}

// Grid abscissae advance by repeated addition, as the reference's loops do
// (s += deltas): grid[i] = value of s in iteration i. Both grids are filled
// once per device (k_fill_quadrature_grids) and read from global memory.
__device__ double g_grid_energyN[400 + 1];
__device__ double g_grid_forceN[10000 + 1];

__global__ void k_fill_quadrature_grids() {
    double s = 0.0;
    for (int i = 0; i <= 400; ++i) {
        s += 1.0 / 400.0;
        g_grid_energyN[i] = s;
    }
    s = 0.0;
    for (int i = 0; i <= 10000; ++i) {
        s += 1.0 / 10000.0;
        g_grid_forceN[i] = s;
    }
}

// energyN: 400 x 400 composite Simpson sum (:884-999). Block-parallel over
// the interior grid; T1..T4 are reduced separately and combined as written.
__device__ double energyN_block(const Six& q, double kRS, double* red) {
    const int N = 400;
    const double ds = 1.0 / double(N), dt = 1.0 / double(N);
    const double* __restrict__ grid = g_grid_energyN;
    auto g = [&](double s, double t) {
        double r_2 = r2_of(q.a, q.b, q.c, q.d, q.e, q.F, s, t);
        return (1.0 / (r_2 * r_2));
    };
    double T[4] = {0, 0, 0, 0};
    if (threadIdx.x == 0) T[0] = g(0.0, 0.0) + g(0.0, 1.0) + g(1.0, 0.0) + g(1.0, 1.0);
    for (int i = 1 + threadIdx.x; i < N; i += blockDim.x) {
        const double s = grid[i], fs = (i % 2 == 0) ? 2.0 : 4.0;
        T[1] += fs * (g(s, 0.0) + g(s, 1.0));
        const double t = grid[i], ft = fs;  // the t grid equals the s grid (N1 == N2)
        T[2] += ft * (g(0.0, t) + g(1.0, t));
    }
    for (int idx = threadIdx.x; idx < (N - 1) * (N - 1); idx += blockDim.x) {
        const int i = 1 + idx / (N - 1), j = 1 + idx % (N - 1);
        const double fs = (i % 2 == 0) ? 2.0 : 4.0, ft = (j % 2 == 0) ? 2.0 : 4.0;
        T[3] += fs * ft * g(grid[i], grid[j]);
    }
    block_sum<4>(T, red);
    __shared__ double result;
    if (threadIdx.x == 0) result = kRS * (ds * dt / 9.0) * (T[0] + T[1] + T[2] + T[3]);
    __syncthreads();
    return result;
}

// forceN: 10^4 x 10^4 composite Simpson sums of the six force integrands,
// then the bead forces of :1133-1148. Returns true when finite.
__device__ bool forceN_block(V3 c1, V3 c2, const V3& c3, const V3& c4, double kRS, bool movebeads,
                             double* red, double (&out)[4][3]) {
    if (movebeads && in_plane(c1, c2, c3, c4)) {
        // movePointOutOfPlane for beads 2 and 1, both along the normal of the
        // original (c1, c2, c3) plane.
        double v1[3] = {c2.x - c1.x, c2.y - c1.y, c2.z - c1.z};
        double v2[3] = {c3.x - c1.x, c3.y - c1.y, c3.z - c1.z};
        double n[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
        double m = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        n[0] = n[0] / m;
        n[1] = n[1] / m;
        n[2] = n[2] / m;
        c2 = V3{c2.x + n[0] * 0.01, c2.y + n[1] * 0.01, c2.z + n[2] * 0.01};
        c1 = V3{c1.x + n[0] * 0.01, c1.y + n[1] * 0.01, c1.z + n[2] * 0.01};
    }
    const Six q = six_of(c1, c2, c3, c4);
    const int N = 10000;
    const double ds = 1.0 / double(N), dt = 1.0 / double(N);
    const double* __restrict__ grid = g_grid_forceN;
    double T[6] = {0, 0, 0, 0, 0, 0};
    auto acc = [&](double s, double t, double w) {
        double r_2 = r2_of(q.a, q.b, q.c, q.d, q.e, q.F, s, t);
        double xi = (1.0 / (r_2 * r_2 * r_2));
        T[0] += w * xi;
        T[1] += w * (s * xi);
        T[2] += w * (s * s * xi);
        T[3] += w * (s * t * xi);
        T[4] += w * (t * xi);
        T[5] += w * (t * t * xi);
    };
    if (threadIdx.x == 0) {
        acc(0.0, 0.0, 1.0); acc(0.0, 1.0, 1.0); acc(1.0, 0.0, 1.0); acc(1.0, 1.0, 1.0);
    }
    for (int i = 1 + threadIdx.x; i < N; i += blockDim.x) {
        const double s = grid[i], w = (i % 2 == 0) ? 2.0 : 4.0;
        acc(s, 0.0, w);
        acc(s, 1.0, w);
        acc(0.0, s, w);
        acc(1.0, s, w);
    }
    for (long long idx = threadIdx.x; idx < (long long)(N - 1) * (N - 1); idx += blockDim.x) {
        const int i = 1 + int(idx / (N - 1)), j = 1 + int(idx % (N - 1));
        const double w = ((i % 2 == 0) ? 2.0 : 4.0) * ((j % 2 == 0) ? 2.0 : 4.0);
        acc(grid[i], grid[j], w);
    }
    block_sum<6>(T, red);
    __shared__ double I[6];
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) I[k] = (ds * dt / 9.0) * T[k];
    __syncthreads();
    double vA[3] = {c1.x - c2.x, c1.y - c2.y, c1.z - c2.z};
    double vB[3] = {c3.x - c4.x, c3.y - c4.y, c3.z - c4.z};
    double vC[3] = {c3.x - c1.x, c3.y - c1.y, c3.z - c1.z};
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
        out[0][k] = 4.0 * kRS * (-I[0] * vC[k] + I[1] * (vC[k] - vA[k]) + I[2] * vA[k] + I[4] * vB[k] - I[3] * vB[k]);
        out[1][k] = 4.0 * kRS * (-I[1] * vC[k] - I[2] * vA[k] + I[3] * vB[k]);
        out[2][k] = 4.0 * kRS * (I[0] * vC[k] + I[1] * vA[k] - I[4] * (vB[k] + vC[k]) - I[3] * vA[k] + I[5] * vB[k]);
        out[3][k] = 4.0 * kRS * (I[4] * vC[k] + I[3] * vA[k] - I[5] * vB[k]);
        for (int b = 0; b < 4; ++b) ok &= !bad_force(out[b][k]);
    }
    return ok;
}

}  // namespace
}  // namespace mb

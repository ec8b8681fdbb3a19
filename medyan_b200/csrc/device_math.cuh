// device_math.cuh — small vector helpers shared by the potential kernels.
//
// Coordinates stay FP64 everywhere. A potential first forms the difference
// vectors it needs in FP64 (that is where cancellation would hurt), then does
// the rest of its arithmetic in R: double for the FP64 path, float for the
// mixed path. With R = double the operation order follows the reference's
// source so results round like the CPU code.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace mb {

struct V3 {
    double x, y, z;
};

template <class R>
struct T3 {
    R x, y, z;
};

__device__ __forceinline__ V3 load3(const double* __restrict__ p) { return V3{__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }

// x + lam*d rounded as the reference's calcCoordLineSearch (CGMethod.cpp:43-46):
// a product then a sum, no fused multiply-add.
__device__ __forceinline__ double move1(double x, double lam, double d) { return __dadd_rn(x, __dmul_rn(lam, d)); }
__device__ __forceinline__ V3 move3(V3 x, double lam, V3 d) {
    return V3{move1(x.x, lam, d.x), move1(x.y, lam, d.y), move1(x.z, lam, d.z)};
}

// b - a, formed in FP64 then converted to R.
template <class R>
__device__ __forceinline__ T3<R> diff(const V3& a, const V3& b) {
    return T3<R>{R(b.x - a.x), R(b.y - a.y), R(b.z - a.z)};
}

template <class R>
__device__ __forceinline__ R dot(const T3<R>& a, const T3<R>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

// Reference midPointCoordinate (MathFunctions.h:963-969): v1*(1-alpha) + alpha*v2, in FP64.
__device__ __forceinline__ V3 midpoint(const V3& v1, const V3& v2, double alpha) {
    double beta = 1 - alpha;
    return V3{v1.x * beta + alpha * v2.x, v1.y * beta + alpha * v2.y, v1.z * beta + alpha * v2.z};
}

template <class R>
__device__ __forceinline__ R rsqrt_r(R x);
template <>
__device__ __forceinline__ double rsqrt_r<double>(double x) { return 1.0 / sqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_r<float>(float x) { return 1.0f / sqrtf(x); }

// areEqual (utility.h:75-77) with ZERO_PREC = 1e-6.
__device__ __forceinline__ bool are_equal(double a, double b) { return fabs(a - b) < 1e-6; }

// std::max(a, b) as the reference uses it.
template <class R>
__device__ __forceinline__ R stdmax(R a, R b) { return (a < b) ? b : a; }

// f[0] += v at device scope without reading the old value back: a reduction
// (red) rather than an atomic that returns (atomicAdd whose result is unused
// still waits for the L2's answer), so the thread does not stall on it.
__device__ __forceinline__ void red_add(double* p, double v) {
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// Arrival tickets of the last-block-done reductions. A block publishes what
// its thread 0 wrote (a row of partial sums) and learns whether it is the
// last to arrive with one acquire-release atomic: the release orders the
// thread's earlier stores before the increment, and the acquire makes every
// earlier arriver's stores visible to the last one (and, after a block
// barrier, to its other threads). A sequentially consistent __threadfence()
// per block costs several microseconds when the memory system is busy, and
// the finishing block of a pass used to wait on four of them in a row.
__device__ __forceinline__ unsigned ticket_add(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
// Release fence for stores of threads other than the one taking the ticket
// (made before the block barrier that precedes the ticket).
__device__ __forceinline__ void fence_release() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Accumulate an R-valued force into the FP64 force array.
template <class R>
__device__ __forceinline__ void add_force(double* __restrict__ f, int off, R fx, R fy, R fz) {
    red_add(f + off, double(fx));
    red_add(f + off + 1, double(fy));
    red_add(f + off + 2, double(fz));
}

// Block-wide sum of NV values per thread into smem-reduced totals held by
// thread 0 (deterministic: fixed shuffle tree, fixed warp order).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* [NV][32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarp = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) smem[k * 32 + warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nwarp ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            v[k] = s;
        }
    }
    __syncthreads();
}

}  // namespace mb

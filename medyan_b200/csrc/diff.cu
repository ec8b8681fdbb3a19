// diff.cu — derivatives for sensitivity analysis (no counterpart in the
// reference): energy gradients with respect to each interaction's
// parameters, their derivative along a direction of the coordinates (the
// mixed second derivative an implicit adjoint needs), and Hessian-vector
// products of the total energy.
//
// Parameter gradients are analytic, per interaction, in FP64, at the
// handle's coordinates (optionally moved to x + e v on the fly):
//   harmonic stretch / linker / motor  U = k/2 (L - l0)^2:
//       dU/dk = (L - l0)^2 / 2,  dU/dl0 = -k (L - l0)
//   cosine bending  U = k (1 - cos(theta - theta0)):
//       dU/dk = 1 - cos(theta - theta0),  dU/dtheta0 = -k sin(theta - theta0)
//   excluded volume  U = kRS * I(geometry), kRS = krep L1 L2:  dU/dkRS = U / kRS
//   boundary  U = k exp(-r/s):  dU/dk = exp(-r/s),  dU/ds = k exp(-r/s) r / s^2
// The directional form is a centred difference of the analytic gradient
// along v, both sides in one kernel. The Hessian-vector product is a centred
// difference of the analytic forces along v, both sides evaluated by the
// force kernels (on-the-fly move x +- e v), then combined.
#include <algorithm>
#include <cmath>

#include "handle.h"
#include "excl.cuh"
#include "potentials.cuh"

namespace mb {

namespace {

constexpr int kThreads = 256;

struct Moved {
    const double* __restrict__ x;
    const double* __restrict__ v;
    double e;  // step along v (0: no move)
    __device__ __forceinline__ V3 operator()(int o) const {
        V3 p = load3(x + o);
        return v ? move3(p, e, load3(v + o)) : p;
    }
};

__device__ __forceinline__ double dist3(const V3& a, const V3& b) {
    const double dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// (dU/dk, dU/dl0) of a harmonic spring of length L.
__device__ __forceinline__ void harmonic_grad(double L, double k, double l0, double& gk, double& gl) {
    const double dev = L - l0;
    gk = 0.5 * dev * dev;
    gl = -k * dev;
}

// (dU/dk, dU/dtheta0) of the cosine bending energy, with the reference's
// clamping of cos(theta).
__device__ __forceinline__ void bend_grad(const V3& c1, const V3& c2, const V3& c3, double k, double eqt, double& gk,
                                          double& gt) {
    const T3<double> r1 = diff<double>(c1, c2), r2 = diff<double>(c2, c3);
    const double L1L2 = sqrt(dot(r1, r1)) * sqrt(dot(r2, r2));
    double x = dot(r1, r2) / L1L2;
    if (x < -1.0) x = -1.0;
    else if (x > 1.0) x = 1.0;
    const double sinA = sqrt(stdmax<double>(1.0 - x * x, 0.0));
    const double cosAmB = x * cos(eqt) + sinA * sin(eqt);
    const double sinAmB = sinA * cos(eqt) - x * sin(eqt);
    gk = 1.0 - cosAmB;
    gt = -k * sinAmB;
}

// One interaction's (dU/dk, dU/dp) at the positions P gives.
template <int FF, class Pos>
__device__ __forceinline__ void grad_of(const ChainDev& ch, const DeviceFF& ff, const int* __restrict__ map, int i,
                                        const Pos& P, double& gk, double& gp) {
    gk = 0.0;
    gp = 0.0;
    if constexpr (FF == MEDYAN_FF_FILAMENT_STRETCHING) {
        const int m = map[i];
        double2 kp;
        int o1, o2;
        if (m >= 0) {
            kp = ch.link_p[m];
            o1 = 3 * m;
            o2 = 3 * (m + 1);
        } else {
            const int2 q = ff.stretch_bs[-1 - m];
            kp = ff.stretch_p[-1 - m];
            o1 = q.x;
            o2 = q.y;
        }
        harmonic_grad(dist3(P(o1), P(o2)), kp.x, kp.y, gk, gp);
    } else if constexpr (FF == MEDYAN_FF_FILAMENT_BENDING) {
        const int m = map[i];
        double2 kp;
        int o1, o2, o3;
        if (m >= 0) {
            kp = ch.bend_p[m];
            o1 = 3 * (m - 1);
            o2 = 3 * m;
            o3 = 3 * (m + 1);
        } else {
            const int4 q = ff.bend_bs[-1 - m];
            kp = ff.bend_p[-1 - m];
            o1 = q.x;
            o2 = q.y;
            o3 = q.z;
        }
        bend_grad(P(o1), P(o2), P(o3), kp.x, kp.y, gk, gp);
    } else if constexpr (FF == MEDYAN_FF_LINKER_STRETCHING || FF == MEDYAN_FF_MOTOR_STRETCHING) {
        const int4 q = FF == MEDYAN_FF_LINKER_STRETCHING ? ff.linker_bs[i] : ff.motor_bs[i];
        const double4 p = FF == MEDYAN_FF_LINKER_STRETCHING ? ff.linker_p[i] : ff.motor_p[i];
        const V3 v1 = midpoint(P(q.x), P(q.y), p.z), v2 = midpoint(P(q.z), P(q.w), p.w);
        harmonic_grad(dist3(v1, v2), p.x, p.y, gk, gp);
    } else if constexpr (FF == MEDYAN_FF_EXCLUDED_VOLUME) {
        const int4 q = ff.excl_bs[i];
        const double krs = ff.excl_krs[i];
        const double U = excl_energy<double>(P(q.x), P(q.y), P(q.z), P(q.w), krs);
        gk = excl_energy_bad(U) ? __longlong_as_double(0x7ff8000000000000ULL) : U / krs;
    } else if constexpr (FF == MEDYAN_FF_BOUNDARY) {
        const int o = ff.boundary_bs[i];
        const double2 p = ff.boundary_p[i];
        const double r = plane_distance(ff.planes[ff.boundary_plane[i]], P(o));
        const double ex = exp(-r / p.y);
        gk = ex;
        gp = p.x * ex * r / (p.y * p.y);
    }
}

template <int FF>
__global__ void __launch_bounds__(kThreads) k_param_grad(const ChainDev ch, const DeviceFF ff,
                                                         const int* __restrict__ map, int n,
                                                         const double* __restrict__ x, const double* __restrict__ v,
                                                         double e, double* __restrict__ gk_out,
                                                         double* __restrict__ gp_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double gk, gp;
    if (!v) {
        grad_of<FF>(ch, ff, map, i, Moved{x, nullptr, 0.0}, gk, gp);
    } else {
        double ak, ap, bk, bp;
        grad_of<FF>(ch, ff, map, i, Moved{x, v, e}, ak, ap);
        grad_of<FF>(ch, ff, map, i, Moved{x, v, -e}, bk, bp);
        gk = (ak - bk) / (2.0 * e);
        gp = (ap - bp) / (2.0 * e);
    }
    if (gk_out) gk_out[i] = gk;
    if (gp_out) gp_out[i] = gp;
}

// hv = -(fa - fb) / (2 e)
__global__ void k_hvp_combine(int n3, const double* __restrict__ fa, const double* __restrict__ fb, double e,
                              double* __restrict__ hv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
        hv[i] = -(fa[i] - fb[i]) / (2.0 * e);
}

int blocks_for(int n) {
    const int b = (n + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
}

// Step of the centred differences: 1e-5 nm in the max-norm of v.
double step_for(const double* v, int n3) {
    double m = 0.0;
    for (int i = 0; i < n3; ++i) m = std::fmax(m, std::fabs(v[i]));
    return m > 0.0 ? 1e-5 / m : 0.0;
}

// Uploads v (caller's order) into h->hv_v (internal order).
cudaError_t upload_direction(medyan_mech* h, const double* v) {
    const int n3 = 3 * h->n_beads;
    cudaError_t e = h->hv_v.reserve(n3 ? n3 : 1);
    if (e == cudaSuccess) e = coords_to_device(h, v, h->hv_v.raw(), h->stream);
    return e;
}

}  // namespace

}  // namespace mb

using namespace mb;

extern "C" medyan_status medyan_mech_param_grad(medyan_mech* h, int32_t ff, const double* v, double* d_k, double* d_p,
                                                int64_t n) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    int count = 0;
    const int* map = nullptr;
    switch (ff) {
        case MEDYAN_FF_FILAMENT_STRETCHING: count = h->n_stretch_in; map = h->stretch_map.raw(); break;
        case MEDYAN_FF_FILAMENT_BENDING: count = h->n_bend_in; map = h->bend_map.raw(); break;
        case MEDYAN_FF_LINKER_STRETCHING: count = h->ff.n_linker; break;
        case MEDYAN_FF_MOTOR_STRETCHING: count = h->ff.n_motor; break;
        case MEDYAN_FF_EXCLUDED_VOLUME: count = h->ff.n_excl; break;
        case MEDYAN_FF_BOUNDARY: count = h->ff.n_boundary; break;
        default: return ff >= 0 && ff < MEDYAN_FF_COUNT ? MEDYAN_ERR_UNSUPPORTED : MEDYAN_ERR_INVALID_ARG;
    }
    if (n != count) return MEDYAN_ERR_CAPACITY;
    if (count == 0) return MEDYAN_OK;
    double e = 0.0;
    cudaError_t ce = cudaSuccess;
    if (v) {
        e = step_for(v, 3 * h->n_beads);
        if (e == 0.0) {
            if (d_k) std::fill(d_k, d_k + n, 0.0);
            if (d_p) std::fill(d_p, d_p + n, 0.0);
            return MEDYAN_OK;
        }
        ce = upload_direction(h, v);
    }
    DevBuf<double>& gk = h->pg_k;
    DevBuf<double>& gp = h->pg_p;
    if (ce == cudaSuccess) ce = gk.reserve(count);
    if (ce == cudaSuccess) ce = gp.reserve(count);
    if (ce != cudaSuccess) return cuda_status(ce);
    const double* dv = v ? h->hv_v.raw() : nullptr;
    const int g = (count + kThreads - 1) / kThreads;
    cudaStream_t s = h->stream;
#define LAUNCH(F) k_param_grad<F><<<g, kThreads, 0, s>>>(h->chain, h->ff, map, count, h->x.raw(), dv, e, gk.raw(), gp.raw())
    switch (ff) {
        case MEDYAN_FF_FILAMENT_STRETCHING: LAUNCH(MEDYAN_FF_FILAMENT_STRETCHING); break;
        case MEDYAN_FF_FILAMENT_BENDING: LAUNCH(MEDYAN_FF_FILAMENT_BENDING); break;
        case MEDYAN_FF_LINKER_STRETCHING: LAUNCH(MEDYAN_FF_LINKER_STRETCHING); break;
        case MEDYAN_FF_MOTOR_STRETCHING: LAUNCH(MEDYAN_FF_MOTOR_STRETCHING); break;
        case MEDYAN_FF_EXCLUDED_VOLUME: LAUNCH(MEDYAN_FF_EXCLUDED_VOLUME); break;
        default: LAUNCH(MEDYAN_FF_BOUNDARY); break;
    }
#undef LAUNCH
    ce = cudaGetLastError();
    if (ce == cudaSuccess && d_k) ce = cudaMemcpyAsync(d_k, gk.raw(), sizeof(double) * count, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && d_p) ce = cudaMemcpyAsync(d_p, gp.raw(), sizeof(double) * count, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    return cuda_status(ce);
}

extern "C" medyan_status medyan_mech_hvp(medyan_mech* h, const double* v, double* hv) {
    if (!h || (h->n_beads && (!v || !hv))) return MEDYAN_ERR_INVALID_ARG;
    const int n3 = 3 * h->n_beads;
    if (n3 == 0) return MEDYAN_OK;
    const double e = step_for(v, n3);
    if (e == 0.0) {
        std::fill(hv, hv + n3, 0.0);
        return MEDYAN_OK;
    }
    cudaStream_t s = h->stream;
    cudaError_t ce = upload_direction(h, v);
    if (ce == cudaSuccess) ce = h->hv_a.reserve(n3);
    if (ce == cudaSuccess) ce = h->hv_b.reserve(n3);
    if (ce == cudaSuccess) ce = h->hv_lam.reserve(2);
    const double lam[2] = {e, -e};
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(h->hv_lam.raw(), lam, sizeof lam, cudaMemcpyHostToDevice, s);
    if (ce != cudaSuccess) return cuda_status(ce);
    const ForceTarget ta{h->hv_a.raw(), nullptr, nullptr, nullptr, h->hv_v.raw(), h->hv_lam.raw()};
    const ForceTarget tb{h->hv_b.raw(), nullptr, nullptr, nullptr, h->hv_v.raw(), h->hv_lam.raw() + 1};
    launch_forces(h->chain, h->ff, h->prec, h->x.raw(), ta, h->fs, s, &h->fork);
    launch_forces(h->chain, h->ff, h->prec, h->x.raw(), tb, h->fs, s, &h->fork);
    k_hvp_combine<<<blocks_for(n3), kThreads, 0, s>>>(n3, h->hv_a.raw(), h->hv_b.raw(), e, h->hv_a.raw());
    ce = cudaGetLastError();
    int status = 0;
    if (ce == cudaSuccess) ce = coords_to_host(h, h->hv_a.raw(), hv, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(&status, h->force_status.raw(), sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->force_status.raw(), 0, sizeof(int), s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return cuda_status(ce);
    return status ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
}

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
//   cosine bending  U = k (1 - cos(theta - theta0)), filament and branch:
//       dU/dk = 1 - cos(theta - theta0),  dU/dtheta0 = -k sin(theta - theta0)
//   branch dihedral and position  U = k (1 - ...):  dU/dk = U / k
//   excluded volume  U = kRS * I(geometry), kRS = krep L1 L2:  dU/dkRS = U / kRS
//   boundary  U = k exp(-r/s):  dU/dk = exp(-r/s),  dU/ds = k exp(-r/s) r / s^2
// The directional form v . d2E/dx dtheta and the Hessian-vector product are
// forward mode: the same formulas evaluated on dual positions x + eps v
// (dual.cuh) return their exact derivative along v. The Hessian-vector
// product runs every force formula of the force pass that way (filament
// links and bends, leftovers, linkers, motors, the four branching
// potentials, boundary repulsion, the analytic excluded-volume forces) and
// adds -dF/deps per bead, in FP64 whatever the handle's precision.
#include <algorithm>
#include <cmath>

#include "handle.h"
#include "dual.cuh"
#include "excl.cuh"
#include "potentials.cuh"

namespace mb {

namespace {

constexpr int kThreads = 256;

// Positions x, or dual positions x + eps v (the directional derivative).
struct Plain {
    const double* __restrict__ x;
    using P = V3;
    using S = double;
    __device__ __forceinline__ V3 operator()(int o) const { return load3(x + o); }
};
struct Along {
    const double* __restrict__ x;
    const double* __restrict__ v;
    using P = DV3;
    using S = Dual;
    __device__ __forceinline__ DV3 operator()(int o) const { return dual3(load3(x + o), load3(v + o)); }
};

template <class P3>
__device__ __forceinline__ auto dist3(const P3& a, const P3& b) {
    const auto dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// (dU/dk, dU/dl0) of a harmonic spring of length L.
template <class S>
__device__ __forceinline__ void harmonic_grad(S L, double k, double l0, S& gk, S& gl) {
    const S dev = L - l0;
    gk = 0.5 * dev * dev;
    gl = -k * dev;
}

// (dU/dk, dU/dtheta0) of the cosine bending energy between the bond vectors
// r1, r2 (filament: p2 - p1, p3 - p2; branch: parent and child cylinders),
// with the reference's clamping of cos(theta).
template <class S>
__device__ __forceinline__ void bend_grad_vec(const T3<S>& r1, const T3<S>& r2, double k, double eqt, S& gk, S& gt) {
    const S L1L2 = sqrt(dot(r1, r1)) * sqrt(dot(r2, r2));
    S x = dot(r1, r2) / L1L2;
    if (x < -1.0) x = S(-1.0);
    else if (x > 1.0) x = S(1.0);
    const S sinA = sqrt(stdmax<S>(1.0 - x * x, S(0.0)));
    const S cosAmB = x * cos(eqt) + sinA * sin(eqt);
    const S sinAmB = sinA * cos(eqt) - x * sin(eqt);
    gk = 1.0 - cosAmB;
    gt = -k * sinAmB;
}
template <class S, class P3>
__device__ __forceinline__ void bend_grad(const P3& c1, const P3& c2, const P3& c3, double k, double eqt, S& gk,
                                          S& gt) {
    bend_grad_vec<S>(diff<S>(c1, c2), diff<S>(c2, c3), k, eqt, gk, gt);
}

// One interaction's (dU/dk, dU/dp) at the positions P gives (with Along:
// their derivatives along v in the dual parts).
template <int FF, class Pos, class S = typename Pos::S>
__device__ __forceinline__ void grad_of(const ChainDev& ch, const DeviceFF& ff, const int* __restrict__ map, int i,
                                        const Pos& P, S& gk, S& gp) {
    gk = S(0.0);
    gp = S(0.0);
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
        harmonic_grad<S>(dist3(P(o1), P(o2)), kp.x, kp.y, gk, gp);
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
        bend_grad<S>(P(o1), P(o2), P(o3), kp.x, kp.y, gk, gp);
    } else if constexpr (FF == MEDYAN_FF_LINKER_STRETCHING || FF == MEDYAN_FF_MOTOR_STRETCHING) {
        const int4 q = FF == MEDYAN_FF_LINKER_STRETCHING ? ff.linker_bs[i] : ff.motor_bs[i];
        const double4 p = FF == MEDYAN_FF_LINKER_STRETCHING ? ff.linker_p[i] : ff.motor_p[i];
        const auto v1 = midpoint(P(q.x), P(q.y), p.z), v2 = midpoint(P(q.z), P(q.w), p.w);
        harmonic_grad<S>(dist3(v1, v2), p.x, p.y, gk, gp);
    } else if constexpr (FF == MEDYAN_FF_EXCLUDED_VOLUME) {
        const int4 q = ff.excl_bs[i];
        const double krs = ff.excl_krs[i];
        const S U = excl_energy_r<S>(P(q.x), P(q.y), P(q.z), P(q.w), krs);
        gk = excl_energy_bad(double(U)) ? S(__longlong_as_double(0x7ff8000000000000ULL)) : U / krs;
    } else if constexpr (FF >= MEDYAN_FF_BRANCHING_STRETCHING && FF <= MEDYAN_FF_BRANCHING_POSITION) {
        // branch point i: pa = (position, stretch k, stretch l0, bend k),
        // pb = (bend theta0, dihedral k, position k, -); a potential that is
        // off (branch_ff_mask) has zero sensitivity
        const int4 q = ff.branch_bs[i];
        const double4 pa = ff.branch_pa[i], pb = ff.branch_pb[i];
        if (!(ff.branch_mask & (1 << (FF - MEDYAN_FF_BRANCHING_STRETCHING)))) return;
        if constexpr (FF == MEDYAN_FF_BRANCHING_STRETCHING) {
            // U = k/2 (|c3 - mp| - l0)^2, mp the branch position on the parent
            harmonic_grad<S>(dist3(midpoint(P(q.x), P(q.y), pa.x), P(q.z)), pa.y, pa.z, gk, gp);
        } else if constexpr (FF == MEDYAN_FF_BRANCHING_BENDING) {
            // U = k (1 - cos(theta - theta0)) between parent and child
            bend_grad_vec<S>(diff<S>(P(q.x), P(q.y)), diff<S>(P(q.z), P(q.w)), pa.w, pb.x, gk, gp);
        } else if constexpr (FF == MEDYAN_FF_BRANCHING_DIHEDRAL) {
            // U = k (1 - n1 . n2): dU/dk = U/k
            gk = branch_dihedral_energy_r<S>(P(q.x), P(q.y), P(q.z), P(q.w), 1.0, pa.x);
        } else {
            // U = k (1 - cos(phi - pi/2)): dU/dk = U/k
            gk = branch_position_energy_r<S>(P(q.x), P(q.y), P(q.z), 1.0, pa.x);
        }
    } else if constexpr (FF == MEDYAN_FF_BOUNDARY) {
        const int o = ff.boundary_bs[i];
        const double2 p = ff.boundary_p[i];
        const S r = plane_distance(ff.planes[ff.boundary_plane[i]], P(o));
        const S ex = exp(-r / p.y);
        gk = ex;
        gp = p.x * ex * r / (p.y * p.y);
    }
}

template <int FF>
__global__ void __launch_bounds__(kThreads) k_param_grad(const ChainDev ch, const DeviceFF ff,
                                                         const int* __restrict__ map, int n,
                                                         const double* __restrict__ x, const double* __restrict__ v,
                                                         double* __restrict__ gk_out, double* __restrict__ gp_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double gk, gp;
    if (!v) {
        grad_of<FF>(ch, ff, map, i, Plain{x}, gk, gp);
    } else {
        // v . d2U/dx dtheta: the dual parts of the gradient at x + eps v
        Dual dk, dp;
        grad_of<FF>(ch, ff, map, i, Along{x, v}, dk, dp);
        gk = dk.d;
        gp = dp.d;
    }
    if (gk_out) gk_out[i] = gk;
    if (gp_out) gp_out[i] = gp;
}

// ---------------------------------------------------------- Hessian-vector
// hv -= dF/deps per bead, F the force formulas at dual positions x + eps v.
__device__ __forceinline__ void hv_sub(double* __restrict__ hv, int o, const T3<Dual>& F) {
    red_add(hv + o, -F.x.d);
    red_add(hv + o + 1, -F.y.d);
    red_add(hv + o + 2, -F.z.d);
}
__device__ __forceinline__ void hv_add(double* __restrict__ hv, int o, const T3<Dual>& F) {
    red_add(hv + o, F.x.d);
    red_add(hv + o + 1, F.y.d);
    red_add(hv + o + 2, F.z.d);
}
__device__ __forceinline__ T3<Dual> tsub(const T3<Dual>& a, const T3<Dual>& b) {
    return T3<Dual>{a.x - b.x, a.y - b.y, a.z - b.z};
}

// Filament chains: the link (q, q+1) and the bend centred at q, per position.
__global__ void __launch_bounds__(kThreads) k_hvp_chain(const ChainDev ch, const double* __restrict__ x,
                                                        const double* __restrict__ v, double* __restrict__ hv) {
    const Along P{x, v};
    const int n = ch.n_pos;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const unsigned char fl = ch.flags[q];
        if (fl & 1) {
            const double2 lp = ch.link_p[q];
            const T3<Dual> F = stretch_force<Dual>(P(3 * q), P(3 * q + 3), lp.x, lp.y);  // on q + 1
            hv_sub(hv, 3 * q + 3, F);
            hv_add(hv, 3 * q, F);
        }
        if (fl & 2) {
            const double2 bp = ch.bend_p[q];
            const DV3 a = P(3 * q - 3), b = P(3 * q), c = P(3 * q + 3);
            T3<Dual> A, B;
            bend_force<Dual>(diff<Dual>(a, b), diff<Dual>(b, c), bp.x, bp.y, A, B);
            hv_add(hv, 3 * q - 3, A);         // force -A on the first bead
            hv_sub(hv, 3 * q, tsub(A, B));    // A - B on the middle
            hv_sub(hv, 3 * q + 3, B);         // B on the last
        }
    }
}

// Generic records: leftover stretches (segment 0) and bends (1), linkers
// (2), motors (3), branch points (4), boundary terms (5), one record per
// thread over the segments' concatenated index space.
__global__ void __launch_bounds__(kThreads) k_hvp_records(const DeviceFF ff, const double* __restrict__ x,
                                                          const double* __restrict__ v, double* __restrict__ hv) {
    const Along P{x, v};
    const int n[6] = {ff.n_stretch, ff.n_bend, ff.n_linker, ff.n_motor, ff.n_branch, ff.n_boundary};
    const int total = n[0] + n[1] + n[2] + n[3] + n[4] + n[5];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int s = 0, i = t;
        while (i >= n[s]) i -= n[s++];
        if (s == 0) {
            const int2 q = ff.stretch_bs[i];
            const double2 p = ff.stretch_p[i];
            const T3<Dual> F = stretch_force<Dual>(P(q.x), P(q.y), p.x, p.y);
            hv_sub(hv, q.y, F);
            hv_add(hv, q.x, F);
        } else if (s == 1) {
            const int4 q = ff.bend_bs[i];
            const double2 p = ff.bend_p[i];
            const DV3 a = P(q.x), b = P(q.y), c = P(q.z);
            T3<Dual> A, B;
            bend_force<Dual>(diff<Dual>(a, b), diff<Dual>(b, c), p.x, p.y, A, B);
            hv_add(hv, q.x, A);
            hv_sub(hv, q.y, tsub(A, B));
            hv_sub(hv, q.z, B);
        } else if (s == 2 || s == 3) {
            const int4 q = s == 2 ? ff.linker_bs[i] : ff.motor_bs[i];
            const double4 p = s == 2 ? ff.linker_p[i] : ff.motor_p[i];
            const T3<Dual> Fl = spring_force<Dual>(P(q.x), P(q.y), P(q.z), P(q.w), p.x, p.y, p.z, p.w);
            const double a1 = 1.0 - p.z, a2 = p.z, b1 = 1.0 - p.w, b2 = p.w;
            hv_add(hv, q.x, T3<Dual>{Fl.x * a1, Fl.y * a1, Fl.z * a1});
            hv_add(hv, q.y, T3<Dual>{Fl.x * a2, Fl.y * a2, Fl.z * a2});
            hv_sub(hv, q.z, T3<Dual>{Fl.x * b1, Fl.y * b1, Fl.z * b1});
            hv_sub(hv, q.w, T3<Dual>{Fl.x * b2, Fl.y * b2, Fl.z * b2});
        } else if (s == 4) {
            const int4 q = ff.branch_bs[i];
            const double4 pa = ff.branch_pa[i], pb = ff.branch_pb[i];
            const DV3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z), c4 = P(q.w);
            const Dual z(0.0);
            T3<Dual> F1{z, z, z}, F2{z, z, z}, F3{z, z, z}, F4{z, z, z};
            auto acc = [](T3<Dual>& a, const T3<Dual>& b, double w) {
                a.x += b.x * w;
                a.y += b.y * w;
                a.z += b.z * w;
            };
            if (ff.branch_mask & 1) {
                const T3<Dual> g = branch_stretch_force<Dual>(c1, c2, c3, pa.y, pa.z, pa.x);
                acc(F1, g, -(pa.x - 1.0));
                acc(F2, g, pa.x);
                acc(F3, g, -1.0);
            }
            if (ff.branch_mask & 2) {
                T3<Dual> Fr1, Fr2;
                bend_force<Dual>(diff<Dual>(c1, c2), diff<Dual>(c3, c4), pa.w, pb.x, Fr1, Fr2);
                acc(F1, Fr1, -1.0);
                acc(F2, Fr1, 1.0);
                acc(F3, Fr2, -1.0);
                acc(F4, Fr2, 1.0);
            }
            if (ff.branch_mask & 4) {
                T3<Dual> L1, L2, L3, L4;
                branch_dihedral_force<Dual>(c1, c2, c3, c4, pb.y, pa.x, L1, L2, L3, L4);
                acc(F1, L1, 1.0);
                acc(F2, L2, 1.0);
                acc(F3, L3, 1.0);
                acc(F4, L4, 1.0);
            }
            if (ff.branch_mask & 8) {
                T3<Dual> Q1, Q2, Q3;
                branch_position_force<Dual>(c1, c2, c3, pb.z, pa.x, Q1, Q2, Q3);
                acc(F1, Q1, 1.0);
                acc(F2, Q2, 1.0);
                acc(F3, Q3, 1.0);
            }
            hv_sub(hv, q.x, F1);
            hv_sub(hv, q.y, F2);
            hv_sub(hv, q.z, F3);
            hv_sub(hv, q.w, F4);
        } else {
            const int o = ff.boundary_bs[i];
            const double2 p = ff.boundary_p[i];
            const double4 pl = ff.planes[ff.boundary_plane[i]];
            const Dual f0 = boundary_force_mag<Dual>(pl, P(o), p.x, p.y);
            hv_sub(hv, o, T3<Dual>{f0 * pl.x, f0 * pl.y, f0 * pl.z});
        }
    }
}

// Cylinder pairs: the analytic forces in the reference's expression order.
// A pair the analytic formula rejects (the quadrature fallback's pairs) has
// no forward-mode derivative here: it sets *status.
__global__ void __launch_bounds__(kThreads) k_hvp_excl(const DeviceFF ff, const double* __restrict__ x,
                                                       const double* __restrict__ v, double* __restrict__ hv,
                                                       int* __restrict__ status) {
    const Along P{x, v};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ff.n_excl; i += gridDim.x * blockDim.x) {
        const int4 q = ff.excl_bs[i];
        T3<Dual> fo[4];
        if (excl_force_exact<Dual>(P(q.x), P(q.y), P(q.z), P(q.w), ff.excl_krs[i], fo)) {
            hv_sub(hv, q.x, fo[0]);
            hv_sub(hv, q.y, fo[1]);
            hv_sub(hv, q.z, fo[2]);
            hv_sub(hv, q.w, fo[3]);
        } else {
            atomicOr(status, 1);
        }
    }
}

int blocks_for(int n) {
    const int b = (n + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
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
        case MEDYAN_FF_BRANCHING_STRETCHING:
        case MEDYAN_FF_BRANCHING_BENDING:
        case MEDYAN_FF_BRANCHING_DIHEDRAL:
        case MEDYAN_FF_BRANCHING_POSITION: count = h->ff.n_branch; break;
        case MEDYAN_FF_EXCLUDED_VOLUME: count = h->ff.n_excl; break;
        case MEDYAN_FF_BOUNDARY: count = h->ff.n_boundary; break;
        default: return ff >= 0 && ff < MEDYAN_FF_COUNT ? MEDYAN_ERR_UNSUPPORTED : MEDYAN_ERR_INVALID_ARG;
    }
    if (n != count) return MEDYAN_ERR_CAPACITY;
    if (count == 0) return MEDYAN_OK;
    cudaError_t ce = cudaSuccess;
    if (v) ce = upload_direction(h, v);
    DevBuf<double>& gk = h->pg_k;
    DevBuf<double>& gp = h->pg_p;
    if (ce == cudaSuccess) ce = gk.reserve(count);
    if (ce == cudaSuccess) ce = gp.reserve(count);
    if (ce != cudaSuccess) return cuda_status(ce);
    const double* dv = v ? h->hv_v.raw() : nullptr;
    const int g = (count + kThreads - 1) / kThreads;
    cudaStream_t s = h->stream;
#define LAUNCH(F) k_param_grad<F><<<g, kThreads, 0, s>>>(h->chain, h->ff, map, count, h->x.raw(), dv, gk.raw(), gp.raw())
    switch (ff) {
        case MEDYAN_FF_FILAMENT_STRETCHING: LAUNCH(MEDYAN_FF_FILAMENT_STRETCHING); break;
        case MEDYAN_FF_FILAMENT_BENDING: LAUNCH(MEDYAN_FF_FILAMENT_BENDING); break;
        case MEDYAN_FF_LINKER_STRETCHING: LAUNCH(MEDYAN_FF_LINKER_STRETCHING); break;
        case MEDYAN_FF_MOTOR_STRETCHING: LAUNCH(MEDYAN_FF_MOTOR_STRETCHING); break;
        case MEDYAN_FF_BRANCHING_STRETCHING: LAUNCH(MEDYAN_FF_BRANCHING_STRETCHING); break;
        case MEDYAN_FF_BRANCHING_BENDING: LAUNCH(MEDYAN_FF_BRANCHING_BENDING); break;
        case MEDYAN_FF_BRANCHING_DIHEDRAL: LAUNCH(MEDYAN_FF_BRANCHING_DIHEDRAL); break;
        case MEDYAN_FF_BRANCHING_POSITION: LAUNCH(MEDYAN_FF_BRANCHING_POSITION); break;
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
    cudaStream_t s = h->stream;
    cudaError_t ce = upload_direction(h, v);
    if (ce == cudaSuccess) ce = h->hv_a.reserve(n3);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->hv_a.raw(), 0, sizeof(double) * n3, s);
    if (ce != cudaSuccess) return cuda_status(ce);
    const double* x = h->x.raw();
    const double* dv = h->hv_v.raw();
    double* out = h->hv_a.raw();
    const DeviceFF& ff = h->ff;
    const int nrec = ff.n_stretch + ff.n_bend + ff.n_linker + ff.n_motor + ff.n_branch + ff.n_boundary;
    k_hvp_chain<<<blocks_for(h->chain.n_pos), kThreads, 0, s>>>(h->chain, x, dv, out);
    if (nrec > 0) k_hvp_records<<<blocks_for(nrec), kThreads, 0, s>>>(ff, x, dv, out);
    if (ff.n_excl > 0) k_hvp_excl<<<blocks_for(ff.n_excl), kThreads, 0, s>>>(ff, x, dv, out, h->force_status.raw());
    ce = cudaGetLastError();
    int status = 0;
    if (ce == cudaSuccess) ce = coords_to_host(h, out, hv, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(&status, h->force_status.raw(), sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->force_status.raw(), 0, sizeof(int), s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return cuda_status(ce);
    return status ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
}

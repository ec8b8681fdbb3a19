// ff_kernels.cu — fused energy and force kernels for the bonded force fields
// (filament stretching and bending, linker, motor, the four branching
// potentials, boundary repulsion). The excluded-volume kernels live in
// excl_kernels.cu, built without FMA contraction.
//
// One launch covers every bonded force field: blocks are assigned to
// contiguous segments (one force field per segment), so a warp never mixes
// potentials. Energy passes evaluate up to kMaxLambda positions x + lam*d per
// interaction from one read of the interaction record and of x and d; the
// per-block sums are reduced deterministically by the finish kernel. Forces
// are accumulated into the FP64 force array with atomic adds. A record whose
// first bead offset is -1 is padding (batched layouts align each replica's
// records to whole blocks) and contributes nothing.
#include "internal.h"
#include "potentials.cuh"

namespace mb {

namespace {

// Segment of global bonded block b, among segments [S0, S1).
template <int S0, int S1>
__device__ __forceinline__ int segment_of(const DeviceFF& ff, int b) {
    int s = S0;
#pragma unroll
    for (int q = S0 + 1; q < S1; ++q) s += (b >= ff.seg[q]) ? 1 : 0;
    return s;
}

// Segment c is compiled into the instantiation for [S0, S1).
template <int S0, int S1>
__device__ constexpr bool has_seg(int c) { return S0 <= c && c < S1; }

__device__ __forceinline__ V3 at(const V3& x, const V3& d, double lam, bool move) { return move ? move3(x, lam, d) : x; }

template <class R, int S0, int S1>
__global__ void __launch_bounds__(kMaxShapeThreads) k_bonded_energy(const DeviceFF ff, const double* __restrict__ x,
                                                          const double* __restrict__ d,
                                                          const LambdaSet* __restrict__ lset,
                                                          double* __restrict__ partial, int nblk_total, int blk_off,
                                                          int n_logical) {
    __shared__ double smem[4 * 32];
    // logical block lb of this group; a capped grid walks them (batched
    // layouts: blocks of replicas outside the pass cost a skipped trip)
    for (int lb = blockIdx.x; lb < n_logical; lb += gridDim.x) {
        const int b = lb + ff.seg[S0];
        if (ff.act && !ff.act[ff.rep_bonded[b]]) continue;  // batched: replica not in this pass
        const int s = segment_of<S0, S1>(ff, b);
        const int i = (b - ff.seg[s]) * blockDim.x + threadIdx.x;
        const bool move = d != nullptr;
        V3 X[4] = {}, D[4] = {};
        double4 pa = {}, pb = {};
        int nb = 0;
        bool valid = false;
        int plane = 0;
        switch (s) {
            case 0:
                if (has_seg<S0, S1>(0) && i < ff.n_stretch) {
                    int2 q = ff.stretch_bs[i];
                    if (q.x < 0) break;  // padding record
                    double2 p = ff.stretch_p[i];
                    pa = double4{p.x, p.y, 0, 0};
                    X[0] = load3(x + q.x);
                    X[1] = load3(x + q.y);
                    if (move) { D[0] = load3(d + q.x); D[1] = load3(d + q.y); }
                    valid = true;
                }
                break;
            case 1:
                if (has_seg<S0, S1>(1) && i < ff.n_bend) {
                    int4 q = ff.bend_bs[i];
                    if (q.x < 0) break;
                    double2 p = ff.bend_p[i];
                    pa = double4{p.x, p.y, 0, 0};
                    X[0] = load3(x + q.x);
                    X[1] = load3(x + q.y);
                    X[2] = load3(x + q.z);
                    if (move) { D[0] = load3(d + q.x); D[1] = load3(d + q.y); D[2] = load3(d + q.z); }
                    valid = true;
                }
                break;
            case 2:
            case 3: {
                const int n = s == 2 ? ff.n_linker : ff.n_motor;
                if ((has_seg<S0, S1>(2) || has_seg<S0, S1>(3)) && i < n) {
                    int4 q = s == 2 ? ff.linker_bs[i] : ff.motor_bs[i];
                    if (q.x < 0) break;
                    pa = s == 2 ? ff.linker_p[i] : ff.motor_p[i];
                    X[0] = load3(x + q.x);
                    X[1] = load3(x + q.y);
                    X[2] = load3(x + q.z);
                    X[3] = load3(x + q.w);
                    if (move) {
                        D[0] = load3(d + q.x); D[1] = load3(d + q.y); D[2] = load3(d + q.z); D[3] = load3(d + q.w);
                    }
                    valid = true;
                }
                break;
            }
            case 4:
                if (has_seg<S0, S1>(4) && i < ff.n_branch) {
                    int4 q = ff.branch_bs[i];
                    if (q.x < 0) break;
                    pa = ff.branch_pa[i];
                    pb = ff.branch_pb[i];
                    X[0] = load3(x + q.x);
                    X[1] = load3(x + q.y);
                    X[2] = load3(x + q.z);
                    X[3] = load3(x + q.w);
                    if (move) {
                        D[0] = load3(d + q.x); D[1] = load3(d + q.y); D[2] = load3(d + q.z); D[3] = load3(d + q.w);
                    }
                    valid = true;
                }
                break;
            default:
                if (has_seg<S0, S1>(5) && i < ff.n_boundary) {
                    int o = ff.boundary_bs[i];
                    if (o < 0) break;
                    double2 p = ff.boundary_p[i];
                    plane = ff.boundary_plane[i];
                    pa = double4{p.x, p.y, 0, 0};
                    X[0] = load3(x + o);
                    if (move) D[0] = load3(d + o);
                    valid = true;
                }
                break;
        }
        (void)nb;
        const int K = lset ? lset->K : 1;
    #pragma unroll
        for (int k = 0; k < kMaxLambda; ++k) {
            if (k >= K) break;
            const double lam = lset ? lset->lam[k] : 0.0;
            double e[4] = {0.0, 0.0, 0.0, 0.0};
            if (valid) {
                V3 P0 = at(X[0], D[0], lam, move), P1 = at(X[1], D[1], lam, move);
                V3 P2 = at(X[2], D[2], lam, move), P3 = at(X[3], D[3], lam, move);
                switch (s) {
                    case 0:
                        if constexpr (has_seg<S0, S1>(0)) e[0] = stretch_energy<R>(P0, P1, pa.x, pa.y);
                        break;
                    case 1:
                        if constexpr (has_seg<S0, S1>(1))
                            e[0] = bend_energy<R>(diff<R>(P0, P1), diff<R>(P1, P2), pa.x, pa.y);
                        break;
                    case 2:
                    case 3:
                        if constexpr (has_seg<S0, S1>(2) || has_seg<S0, S1>(3))
                            e[0] = spring_energy<R>(P0, P1, P2, P3, pa.x, pa.y, pa.z, pa.w);
                        break;
                    case 4:
                        if constexpr (has_seg<S0, S1>(4)) {
                            if (ff.branch_mask & 1) e[0] = branch_stretch_energy<R>(P0, P1, P2, pa.y, pa.z, pa.x);
                            if (ff.branch_mask & 2) e[1] = bend_energy<R>(diff<R>(P0, P1), diff<R>(P2, P3), pa.w, pb.x);
                            if (ff.branch_mask & 4) e[2] = branch_dihedral_energy<R>(P0, P1, P2, P3, pb.y, pa.x);
                            if (ff.branch_mask & 8) e[3] = branch_position_energy<R>(P0, P1, P2, pb.z, pa.x);
                        }
                        break;
                    default:
                        if constexpr (has_seg<S0, S1>(5)) e[0] = boundary_energy<R>(ff.planes[plane], P0, pa.x, pa.y);
                        break;
                }
            }
            block_sum<4>(e, smem);
            if (threadIdx.x == 0) {
                double* o = partial + ((size_t)k * nblk_total + blk_off + b) * 4;
                o[0] = e[0];
                o[1] = e[1];
                o[2] = e[2];
                o[3] = e[3];
            }
        }
        __syncthreads();  // smem of block_sum is reused by the next trip
    }
}

// Position of the bead at coordinate offset o for a force pass.
struct PosLoader {
    const double* __restrict__ x;
    const double* __restrict__ d;
    double lam;
    __device__ __forceinline__ V3 operator()(int o) const {
        V3 p = load3(x + o);
        return d ? move3(p, lam, load3(d + o)) : p;
    }
};

template <class R, int S0, int S1>
__global__ void __launch_bounds__(kMaxShapeThreads) k_bonded_forces(const DeviceFF ff, const double* __restrict__ x,
                                                          const ForceTarget tgt, int n_logical) {
    if (tgt.skip && *tgt.skip) return;
    double* __restrict__ f = target_force(tgt);
    const PosLoader P{x, tgt.d, tgt.lam ? *tgt.lam : 0.0};
    for (int lb = blockIdx.x; lb < n_logical; lb += gridDim.x) {
        const int b = lb + ff.seg[S0];
        if (ff.act && !ff.act[ff.rep_bonded[b]]) continue;  // batched: replica not in this pass
        const int s = segment_of<S0, S1>(ff, b);
        const int i = (b - ff.seg[s]) * blockDim.x + threadIdx.x;
        switch (s) {
            case 0:
                if (has_seg<S0, S1>(0) && i < ff.n_stretch) {
                    int2 q = ff.stretch_bs[i];
                    if (q.x < 0) break;  // padding record
                    double2 p = ff.stretch_p[i];
                    T3<R> F = stretch_force<R>(P(q.x), P(q.y), p.x, p.y);
                    target_add(tgt, f, q.y, F.x, F.y, F.z);
                    target_add(tgt, f, q.x, -F.x, -F.y, -F.z);
                }
                break;
            case 1:
                if (has_seg<S0, S1>(1) && i < ff.n_bend) {
                    int4 q = ff.bend_bs[i];
                    if (q.x < 0) break;
                    double2 p = ff.bend_p[i];
                    V3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z);
                    T3<R> Fr1, Fr2;
                    bend_force<R>(diff<R>(c1, c2), diff<R>(c2, c3), p.x, p.y, Fr1, Fr2);
                    target_add(tgt, f, q.x, -Fr1.x, -Fr1.y, -Fr1.z);
                    target_add(tgt, f, q.y, Fr1.x - Fr2.x, Fr1.y - Fr2.y, Fr1.z - Fr2.z);
                    target_add(tgt, f, q.z, Fr2.x, Fr2.y, Fr2.z);
                }
                break;
            case 2:
            case 3: {
                const int n = s == 2 ? ff.n_linker : ff.n_motor;
                if ((has_seg<S0, S1>(2) || has_seg<S0, S1>(3)) && i < n) {
                    int4 q = s == 2 ? ff.linker_bs[i] : ff.motor_bs[i];
                    if (q.x < 0) break;
                    double4 p = s == 2 ? ff.linker_p[i] : ff.motor_p[i];
                    T3<R> Fl = spring_force<R>(P(q.x), P(q.y), P(q.z), P(q.w), p.x, p.y, p.z, p.w);
                    const R a1 = R(1) - R(p.z), a2 = R(p.z), b1 = R(1) - R(p.w), b2 = R(p.w);
                    target_add(tgt, f, q.x, -Fl.x * a1, -Fl.y * a1, -Fl.z * a1);
                    target_add(tgt, f, q.y, -Fl.x * a2, -Fl.y * a2, -Fl.z * a2);
                    target_add(tgt, f, q.z, Fl.x * b1, Fl.y * b1, Fl.z * b1);
                    target_add(tgt, f, q.w, Fl.x * b2, Fl.y * b2, Fl.z * b2);
                }
                break;
            }
            case 4:
                if (has_seg<S0, S1>(4) && i < ff.n_branch) {
                    int4 q = ff.branch_bs[i];
                    if (q.x < 0) break;
                    double4 pa = ff.branch_pa[i], pb = ff.branch_pb[i];
                    V3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z), c4 = P(q.w);
                    T3<R> F1{0, 0, 0}, F2{0, 0, 0}, F3{0, 0, 0}, F4{0, 0, 0};
                    if (ff.branch_mask & 1) {
                        T3<R> g = branch_stretch_force<R>(c1, c2, c3, pa.y, pa.z, pa.x);
                        const R pm1 = R(pa.x) - R(1), pp = R(pa.x);
                        F1.x += -g.x * pm1; F1.y += -g.y * pm1; F1.z += -g.z * pm1;
                        F2.x += g.x * pp; F2.y += g.y * pp; F2.z += g.z * pp;
                        F3.x += -g.x; F3.y += -g.y; F3.z += -g.z;
                    }
                    if (ff.branch_mask & 2) {
                        T3<R> Fr1, Fr2;
                        bend_force<R>(diff<R>(c1, c2), diff<R>(c3, c4), pa.w, pb.x, Fr1, Fr2);
                        F1.x += -Fr1.x; F1.y += -Fr1.y; F1.z += -Fr1.z;
                        F2.x += Fr1.x; F2.y += Fr1.y; F2.z += Fr1.z;
                        F3.x += -Fr2.x; F3.y += -Fr2.y; F3.z += -Fr2.z;
                        F4.x += Fr2.x; F4.y += Fr2.y; F4.z += Fr2.z;
                    }
                    if (ff.branch_mask & 4) {
                        T3<R> L1, L2, L3, L4;
                        branch_dihedral_force<R>(c1, c2, c3, c4, pb.y, pa.x, L1, L2, L3, L4);
                        F1.x += L1.x; F1.y += L1.y; F1.z += L1.z;
                        F2.x += L2.x; F2.y += L2.y; F2.z += L2.z;
                        F3.x += L3.x; F3.y += L3.y; F3.z += L3.z;
                        F4.x += L4.x; F4.y += L4.y; F4.z += L4.z;
                    }
                    if (ff.branch_mask & 8) {
                        T3<R> P1, P2, P3;
                        branch_position_force<R>(c1, c2, c3, pb.z, pa.x, P1, P2, P3);
                        F1.x += P1.x; F1.y += P1.y; F1.z += P1.z;
                        F2.x += P2.x; F2.y += P2.y; F2.z += P2.z;
                        F3.x += P3.x; F3.y += P3.y; F3.z += P3.z;
                    }
                    target_add(tgt, f, q.x, F1.x, F1.y, F1.z);
                    target_add(tgt, f, q.y, F2.x, F2.y, F2.z);
                    target_add(tgt, f, q.z, F3.x, F3.y, F3.z);
                    target_add(tgt, f, q.w, F4.x, F4.y, F4.z);
                }
                break;
            default:
                if (has_seg<S0, S1>(5) && i < ff.n_boundary) {
                    int o = ff.boundary_bs[i];
                    if (o < 0) break;
                    double2 p = ff.boundary_p[i];
                    double4 pl = ff.planes[ff.boundary_plane[i]];
                    R f0 = boundary_force_mag<R>(pl, P(o), p.x, p.y);
                    target_add(tgt, f, o, f0 * R(pl.x), f0 * R(pl.y), f0 * R(pl.z));
                }
                break;
        }
    }
}

}  // namespace

int bonded_blocks(const DeviceFF& ff) { return ff.seg[6]; }

namespace {

// Deterministic mode: the fixed-point sums back to double, in place.
// rep/act (packed batches): the positions of replicas not in the pass were
// not written by it and still hold doubles; they are left alone.
__global__ void __launch_bounds__(256) k_fixed_to_double(const ForceTarget t, int n3, const int* __restrict__ rep,
                                                         const int* __restrict__ act) {
    if (t.skip && *t.skip) return;
    double* __restrict__ f = target_force(t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
        if (!act || act[rep[i / 3]]) f[i] = double(__double_as_longlong(f[i])) / kFixedScale;
}

}  // namespace

void launch_fixed_to_double(const ForceTarget& t, int n3, cudaStream_t s, const int* rep, const int* act) {
    if (!t.fixed || n3 <= 0) return;
    int g = (n3 + 255) / 256;
    g = g > 148 * 8 ? 148 * 8 : g;
    k_fixed_to_double<<<g, 256, 0, s>>>(t, n3, rep, act);
}

namespace {

// Bonded kernels are launched per group of segments, so each group gets the
// registers its own potentials need: filament leftovers [0, 2), linker and
// motor [2, 4), branching [4, 5), boundary [5, 6).
template <int S0, int S1>
void bonded_energy_group(const DeviceFF& ff, const double* x, const double* d, const LambdaSet* lam,
                         const EnergyScratch& es, cudaStream_t s) {
    const int nb = ff.seg[S1] - ff.seg[S0];
    if (nb > 0)
        k_bonded_energy<double, S0, S1><<<logical_grid(ff, nb), bonded_block_of(ff), 0, s>>>(
            ff, x, d, lam, es.partial, es.total(), es.n_blocks_chain, nb);
}

template <int S0, int S1>
void bonded_forces_group(const DeviceFF& ff, int prec, const double* x, const ForceTarget& t, cudaStream_t s) {
    const int nb = ff.seg[S1] - ff.seg[S0];
    if (nb <= 0) return;
    if (prec == MEDYAN_PREC_MIXED)
        k_bonded_forces<float, S0, S1><<<logical_grid(ff, nb), bonded_block_of(ff), 0, s>>>(ff, x, t, nb);
    else
        k_bonded_forces<double, S0, S1><<<logical_grid(ff, nb), bonded_block_of(ff), 0, s>>>(ff, x, t, nb);
}

void fork_to(const Fork* fk, cudaStream_t s, int n) {
    cudaEventRecord(fk->fork, s);
    for (int k = 0; k < n; ++k) cudaStreamWaitEvent(fk->side[k], fk->fork, 0);
}

void join_from(const Fork* fk, cudaStream_t s, int n) {
    for (int k = 0; k < n; ++k) {
        cudaEventRecord(fk->join[k], fk->side[k]);
        cudaStreamWaitEvent(s, fk->join[k], 0);
    }
}

}  // namespace

void launch_energy_producers(const ChainDev& ch, const DeviceFF& ff, const double* x, const double* d,
                             const LambdaSet* lam, const EnergyScratch& es, cudaStream_t s, const Fork* fk,
                             const int4* chain_table, int chain_table_blocks) {
    // five branches: chain | excluded volume | linker, motor | branching |
    // boundary, filament leftovers
    cudaStream_t b[4] = {s, s, s, s};
    if (fk) {
        fork_to(fk, s, 4);
        for (int k = 0; k < 4; ++k) b[k] = fk->side[k];
    }
    launch_excl_energy(ff, MEDYAN_PREC_FP64, x, d, lam, es, b[0]);
    bonded_energy_group<2, 4>(ff, x, d, lam, es, b[1]);
    bonded_energy_group<4, 5>(ff, x, d, lam, es, b[2]);
    bonded_energy_group<5, 6>(ff, x, d, lam, es, b[3]);
    bonded_energy_group<0, 2>(ff, x, d, lam, es, b[3]);
    launch_chain_energy(ch, MEDYAN_PREC_FP64, x, d, lam, es.partial, es.total(), 0, s, chain_table,
                        chain_table_blocks);
    if (fk) join_from(fk, s, 4);
}

void launch_energy(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const double* d,
                   const LambdaSet* lam, const EnergyScratch& es, cudaStream_t s, const Fork* fk) {
    // Energies are evaluated in double in both precision modes: the backtracking
    // line search compares totals whose differences are ~1e-9 of the total,
    // below float resolution per term. Only the force pass runs in float.
    (void)prec;
    launch_energy_producers(ch, ff, x, d, lam, es, s, fk, nullptr, 0);
    launch_excl_energy_fallback_and_finish(ff, x, d, lam, es, s);
}

void launch_forces(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const ForceTarget& t,
                   const ForceScratch& fs, cudaStream_t s, const Fork* fk) {
    // the chain pass stores every bead's force; everything after adds, in four
    // branches: excluded volume | linker, motor | branching | boundary,
    // filament leftovers
    launch_chain_forces(ch, prec, x, t, s);
    cudaStream_t b[4] = {s, s, s, s};
    if (fk) {
        fork_to(fk, s, 3);
        for (int k = 0; k < 3; ++k) b[k + 1] = fk->side[k];
    }
    bonded_forces_group<2, 4>(ff, prec, x, t, b[1]);
    bonded_forces_group<4, 5>(ff, prec, x, t, b[2]);
    bonded_forces_group<5, 6>(ff, prec, x, t, b[3]);
    bonded_forces_group<0, 2>(ff, prec, x, t, b[3]);
    launch_excl_forces(ff, prec, x, t, fs, s);
    if (fk) join_from(fk, s, 3);
    launch_fixed_to_double(t, 3 * ch.n_pos, s, ch.rep, ch.act);
}

void launch_evaluate(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const double* d,
                     const LambdaSet* lam,
                     const ForceTarget& t, const EnergyScratch& es, const ForceScratch& fs, cudaStream_t s,
                     const Fork* fk) {
    if (!fk) {
        launch_energy(ch, ff, prec, x, d, lam, es, s, nullptr);
        launch_forces(ch, ff, prec, x, t, fs, s, nullptr);
        return;
    }
    // side 0: excluded-volume energy, then the finish once sides 1-4 are done;
    // sides 1-4: bonded groups and chain energy; main: chain forces, then
    // the excluded-volume forces; sides 5-7: bonded forces after the chain
    // forces (which initialize the force array)
    fork_to(fk, s, kForkWays);
    launch_excl_energy(ff, MEDYAN_PREC_FP64, x, d, lam, es, fk->side[0]);
    bonded_energy_group<2, 4>(ff, x, d, lam, es, fk->side[1]);
    bonded_energy_group<4, 5>(ff, x, d, lam, es, fk->side[2]);
    bonded_energy_group<5, 6>(ff, x, d, lam, es, fk->side[3]);
    bonded_energy_group<0, 2>(ff, x, d, lam, es, fk->side[3]);
    launch_chain_energy(ch, MEDYAN_PREC_FP64, x, d, lam, es.partial, es.total(), 0, fk->side[4], nullptr, 0);
    launch_chain_forces(ch, prec, x, t, s);
    cudaEventRecord(fk->mid, s);
    for (int k = 5; k < 8; ++k) cudaStreamWaitEvent(fk->side[k], fk->mid, 0);
    bonded_forces_group<2, 4>(ff, prec, x, t, fk->side[5]);
    bonded_forces_group<4, 5>(ff, prec, x, t, fk->side[6]);
    bonded_forces_group<5, 6>(ff, prec, x, t, fk->side[7]);
    bonded_forces_group<0, 2>(ff, prec, x, t, fk->side[7]);
    launch_excl_forces(ff, prec, x, t, fs, s);
    for (int k = 1; k < 5; ++k) {
        cudaEventRecord(fk->join[k], fk->side[k]);
        cudaStreamWaitEvent(fk->side[0], fk->join[k], 0);
    }
    launch_excl_energy_fallback_and_finish(ff, x, d, lam, es, fk->side[0]);
    for (int k : {0, 5, 6, 7}) {
        cudaEventRecord(fk->join[k], fk->side[k]);
        cudaStreamWaitEvent(s, fk->join[k], 0);
    }
    launch_fixed_to_double(t, 3 * ch.n_pos, s, ch.rep, ch.act);
}

}  // namespace mb

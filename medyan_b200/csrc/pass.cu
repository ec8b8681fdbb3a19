// pass.cu — fused single-network passes: the energy and/or the forces of
// every force field at one set of positions, in one zero fill and three
// kernels that run side by side.
//
//   k_pass_zero    zeroes the force target (force passes only);
//   k_pass_main    filament chains (warp tiles of 30 consecutive beads, as in
//                  chain.cu) and the generic records of filament leftovers,
//                  linkers, motors and boundary terms;
//   k_pass_branch  branch points (their four potentials need more registers
//                  than the rest, so they get their own kernel);
//   k_pass_excl    cylinder excluded volume (FP64 in both precision modes).
//
// Every contribution to a bead's force is added atomically into the zeroed
// target, so the three kernels have no order among themselves and the graph
// runs them concurrently: the FP64-heavy excluded-volume pairs overlap the
// bandwidth-bound chain tiles and the gather-bound linker records instead of
// following them. Energy and force of an interaction come from one read of
// its record and its beads' positions.
//
// Energies: each block writes one row of per-force-field sums (fixed
// reduction tree), and takes a ticket shared by all three kernels. The block
// that takes the last ticket, whichever kernel it belongs to, sums the rows
// in row order (deterministic for a given grid), runs the quadrature
// fallbacks (energyN / forceN) for the pairs the analytic formulas rejected,
// applies ForceFieldManager::computeEnergy's rule (a force field at or below
// -1 makes the total +inf, ForceFieldManager.cpp:137-176) and resets the
// ticket and the queues. No block waits for another: the last one to finish
// does the finishing work.
//
// Built with --fmad=false (the excluded-volume formula and the quadrature
// fallbacks round as the reference's code does).
#include "handle.h"
#include "potentials.cuh"
#include "excl.cuh"
#include "quadrature.cuh"
#include "pass.h"

#include <mutex>

// Pass timeline (profiling build only: compiled with -DMEDYAN_PASS_TRACE into
// libmedyan_b200_trace.so by `python -m medyan_b200.build --trace`). Thread 0
// of every block of the pass kernels records the block's kernel kind, SM,
// index and its start and end on the global timer; the blocks that complete
// a group of energy rows and the block that finishes the pass record those
// stages too. medyan_pass_trace_reset / medyan_pass_trace_dump read the
// records back (medyan_b200/pass_timeline.py prints them per kernel).
#ifdef MEDYAN_PASS_TRACE
namespace mb {
namespace trace {
struct Rec {
    unsigned kind, smid, block, pad;
    unsigned long long t0, t1;
};
constexpr unsigned kCap = 1u << 16;
__device__ Rec g_rec[kCap];
__device__ unsigned g_n;
__device__ __forceinline__ unsigned long long now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void record(unsigned kind, unsigned long long t0) {
    if (threadIdx.x != 0) return;
    unsigned sm;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
    const unsigned i = atomicAdd(&g_n, 1u);
    if (i < kCap) g_rec[i] = Rec{kind, sm, blockIdx.x, 0u, t0, now()};
}
}  // namespace trace
}  // namespace mb
extern "C" int medyan_pass_trace_reset() {
    const unsigned z = 0;
    return (int)cudaMemcpyToSymbol(mb::trace::g_n, &z, sizeof(z));
}
// Copies up to max records to host (32 bytes each); returns how many.
extern "C" int medyan_pass_trace_dump(void* host, int max) {
    unsigned n = 0;
    if (cudaMemcpyFromSymbol(&n, mb::trace::g_n, sizeof(n)) != cudaSuccess) return -1;
    if (n > mb::trace::kCap) n = mb::trace::kCap;
    if ((int)n > max) n = (unsigned)max;
    if (n && cudaMemcpyFromSymbol(host, mb::trace::g_rec, n * sizeof(mb::trace::Rec)) != cudaSuccess) return -1;
    return (int)n;
}
#define PASS_TRACE_BEGIN const unsigned long long trace_t0 = mb::trace::now();
#define PASS_TRACE_END(kind) mb::trace::record((kind), trace_t0);
#else
#define PASS_TRACE_BEGIN
#define PASS_TRACE_END(kind)
#endif

namespace mb {

namespace {

constexpr int kSlots = MEDYAN_FF_COUNT;
constexpr int kWarpOut = 30;  // forces written per warp tile: lanes 1..30 of 32 centres
constexpr unsigned char kLink = 1, kBend = 2;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kZeroThreads = 256;
// Resident blocks of the main kernel per SM: 80 registers a thread, room
// for a chain tile's loads in flight beside the one being computed
constexpr int kMainBlocksPerSM = 3;
constexpr int kTilesPerWarp = 4;  // chain tiles per warp in a force-only pass's chain unit
template <class R, bool E, bool F, bool LS>
constexpr int main_blocks_per_sm() {
    return kMainBlocksPerSM;
}
constexpr int kExclThreadsMax = 128;

__device__ __forceinline__ V3 shfl_up3(const V3& v) {
    return V3{__shfl_up_sync(kFull, v.x, 1), __shfl_up_sync(kFull, v.y, 1), __shfl_up_sync(kFull, v.z, 1)};
}
__device__ __forceinline__ V3 shfl_down3(const V3& v) {
    return V3{__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1), __shfl_down_sync(kFull, v.z, 1)};
}
template <class R>
__device__ __forceinline__ T3<R> shfl_up3(const T3<R>& v) {
    return T3<R>{__shfl_up_sync(kFull, v.x, 1), __shfl_up_sync(kFull, v.y, 1), __shfl_up_sync(kFull, v.z, 1)};
}
template <class R>
__device__ __forceinline__ T3<R> shfl_down3(const T3<R>& v) {
    return T3<R>{__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1), __shfl_down_sync(kFull, v.z, 1)};
}

// Positions of a pass: x, or x + lam*d rounded as calcCoordLineSearch.
struct Pos {
    const double* __restrict__ x;
    const double* __restrict__ d;
    double lam;
    __device__ __forceinline__ V3 operator()(int o) const {
        const V3 p = load3(x + o);
        return d ? move3(p, lam, load3(d + o)) : p;
    }
};

__device__ __forceinline__ Pos pos_of(const PassArgs& a) { return Pos{a.x, a.t.d, a.t.lam ? *a.t.lam : 0.0}; }

// ------------------------------------------------------------ finish
// Energy rows: each kernel's blocks hold a few per-thread sums, mapped to
// force-field slots by the kernel kind (0 main: filament stretching and
// bending, linker, motor, boundary; 1 branch: the four branching slots;
// 2 excluded volume).
constexpr int kMainVals = 5, kBranchVals = 4, kExclVals = 1;
template <int KIND>
__device__ constexpr int slot_of(int j) {
    return KIND == 0 ? (j == 4 ? MEDYAN_FF_BOUNDARY : j)
                     : (KIND == 1 ? MEDYAN_FF_BRANCHING_STRETCHING + j : MEDYAN_FF_EXCLUDED_VOLUME);
}

// Energy rows are summed by a fixed tree over arrival tickets. Row r belongs
// to group r / kGroup; the block that completes a group (its group ticket)
// sums the group's rows with one warp (lane j holds row kGroup*g + j, then a
// fixed shuffle tree) into a group row, and takes the pass ticket; the block
// that completes the last group sums the group rows the same way and
// finishes. Which blocks do this varies from pass to pass; the order of every
// addition does not.
constexpr int kGroup = kPassGroup;

// Sum over lanes of v (lane j's value), fixed tree; valid in lane 0.
__device__ __forceinline__ double warp_tree(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return v;
}

// Runs the queued fallbacks and writes the results from the group rows;
// called by the block that completes the last group (all its threads).
template <bool E, bool F>
__device__ __noinline__ void pass_finish(const PassArgs& a) {
    __shared__ double red[6 * 32];
    __shared__ double sums[kSlots];
    __shared__ double fbE;
    __shared__ int nfb;
    const Pos P = pos_of(a);
    if constexpr (E) {
        __shared__ int n_queued, bad0;
        // the queue length and status are fetched while the group rows load
        if (threadIdx.x == 0) {
            n_queued = __ldcg(a.e_fb_count);
            bad0 = __ldcg(a.e_bad);
        }
        // warp w sums slots w, w + nwarp, ...: every warp's loads are in
        // flight at once (ten slots one after another were ten L2 round
        // trips in a row). Per slot the lanes add their groups in group
        // order and the warp tree is fixed, whichever warp does it.
        {
            const int ng = (a.n_rows + kGroup - 1) / kGroup;
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
            for (int s = warp; s < kSlots; s += nwarp) {
                double v = 0.0;
                for (int g = lane; g < ng; g += 32) v += __ldcg(a.group_rows + (size_t)s * a.n_groups + g);
                v = warp_tree(v);
                if (lane == 0) sums[s] = v;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // queued pairs in pair order (the queue fills in arrival order)
            const int n = min(n_queued, a.e_fb_cap);
            for (int i = 1; i < n; ++i) {
                const int2 q = __ldcg(a.e_fb_list + i);
                int j = i - 1;
                while (j >= 0 && __ldcg(a.e_fb_list + j).x > q.x) {
                    a.e_fb_list[j + 1] = __ldcg(a.e_fb_list + j);
                    --j;
                }
                a.e_fb_list[j + 1] = q;
            }
            nfb = n;
            fbE = 0.0;
        }
        __syncthreads();
        for (int q = 0; q < nfb; ++q) {
            const int i = __ldcg(a.e_fb_list + q).x;
            const int4 bs = a.ff.excl_bs[i];
            const double U = energyN_block(six_of(P(bs.x), P(bs.y), P(bs.z), P(bs.w)), a.ff.excl_krs[i], red);
            if (threadIdx.x == 0) {
                if (excl_energy_bad(U)) atomicOr(a.e_bad, 1);
                else fbE += U;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double v[kSlots];
#pragma unroll
            for (int s = 0; s < kSlots; ++s) v[s] = sums[s];
            double tot = 0.0;
            bool inf = false;
            v[MEDYAN_FF_EXCLUDED_VOLUME] += fbE;
            // the fallbacks may have flagged a pair: read the status again then
            if (nfb > 0 ? __ldcg(a.e_bad) : bad0) v[MEDYAN_FF_EXCLUDED_VOLUME] = -1.0;
#pragma unroll
            for (int s = 0; s < kSlots; ++s) {
                if (v[s] <= -1) inf = true;
                else tot += v[s];
            }
            const double total = inf ? __longlong_as_double(0x7ff0000000000000ULL) : tot;
            // a plain pass writes its one evaluation to every requested slot
            const int K = a.lam_set ? a.lam_set->K : 1;
            for (int k = 0; k < K; ++k) {
                double* o = a.out + k * (kSlots + 1);
#pragma unroll
                for (int s = 0; s < kSlots; ++s) o[s] = v[s];
                o[kSlots] = total;
            }
            *a.e_fb_count = 0;
            for (int k = 0; k < kMaxLambda; ++k) a.e_bad[k] = 0;
        }
    }
    if constexpr (F) {
        double* __restrict__ f = target_force(a.t);
        const int n = min(__ldcg(a.f_fb_count), a.f_fb_cap);
        for (int q = 0; q < n; ++q) {
            const int i = __ldcg(a.f_fb_list + q);
            const int4 bs = a.ff.excl_bs[i];
            const V3 c1 = P(bs.x), c2 = P(bs.y), c3 = P(bs.z), c4 = P(bs.w);
            double out[4][3];
            bool ok = forceN_block(c1, c2, c3, c4, a.ff.excl_krs[i], false, red, out);
            if (!ok) ok = forceN_block(c1, c2, c3, c4, a.ff.excl_krs[i], true, red, out);
            if (threadIdx.x == 0) {
                if (ok) {
                    target_add(a.t, f, bs.x, out[0][0], out[0][1], out[0][2]);
                    target_add(a.t, f, bs.y, out[1][0], out[1][1], out[1][2]);
                    target_add(a.t, f, bs.z, out[2][0], out[2][1], out[2][2]);
                    target_add(a.t, f, bs.w, out[3][0], out[3][1], out[3][2]);
                } else {
                    atomicOr(a.f_status, 1);
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) *a.f_fb_count = 0;
    }
    if (threadIdx.x == 0) *a.ticket = 0u;
}

// Writes the block's energy row, takes its group's ticket and, for the block
// that completes a group, sums the group and takes the pass ticket; the
// block that completes the last group finishes the pass.
template <int KIND, bool E, bool F, int NV>
__device__ __forceinline__ void block_done(const PassArgs& a, double (&acc)[NV], int row, bool queued) {
    __shared__ double smem[NV * 32];
    __shared__ int state;  // 0 not last in its group, 1 completed its group, 2 completed the pass
    if constexpr (E) {
        block_sum<NV>(acc, smem);
        if (threadIdx.x == 0) {
            // slot-major rows: rows[slot * n_rows + row]
#pragma unroll
            for (int s = 0; s < kSlots; ++s) {
                double v = 0.0;
#pragma unroll
                for (int j = 0; j < NV; ++j)
                    if (slot_of<KIND>(j) == s) v = acc[j];
                a.rows[(size_t)s * a.n_rows + row] = v;
            }
        }
    }
    // the row (thread 0's stores) is published by thread 0's ticket; a
    // fallback-queue entry (stored by the thread that queued it) by that
    // thread's release fence before the barrier. The force additions need no
    // ordering: the finishing block only adds to them
    if (queued) fence_release();
    __syncthreads();
    const int g = row / kGroup;
    if (threadIdx.x == 0) {
        const int gsize = min(kGroup, a.n_rows - kGroup * g);
        state = ticket_add(a.group_ticket + g, 1u) == (unsigned)gsize - 1 ? 1 : 0;
    }
    __syncthreads();
    if (state == 0) return;
    PASS_TRACE_BEGIN
    if constexpr (E) {
        if (threadIdx.x < 32) {
            const int r = kGroup * g + threadIdx.x;
            const bool in = r < a.n_rows;
            double v[kSlots];
#pragma unroll
            for (int s = 0; s < kSlots; ++s) v[s] = in ? __ldcg(a.rows + (size_t)s * a.n_rows + r) : 0.0;
#pragma unroll
            for (int s = 0; s < kSlots; ++s) {
                const double t = warp_tree(v[s]);
                if (threadIdx.x == 0) a.group_rows[(size_t)s * a.n_groups + g] = t;
            }
        }
    }
    if (threadIdx.x == 0) {
        // the group row (thread 0's store) is published by the pass ticket
        a.group_ticket[g] = 0u;
        const int ng = (a.n_rows + kGroup - 1) / kGroup;
        state = ticket_add(a.ticket, 1u) == (unsigned)ng - 1 ? 2 : 1;
    }
    __syncthreads();
    PASS_TRACE_END(100 + KIND)
    if (state != 2) return;
#ifdef MEDYAN_PASS_TRACE
    const unsigned long long trace_f0 = mb::trace::now();
#endif
    pass_finish<E, F>(a);
#ifdef MEDYAN_PASS_TRACE
    __syncthreads();
    mb::trace::record(200 + KIND, trace_f0);
#endif
}

// ------------------------------------------------------------ main kernel
// One warp tile of the chains: lanes hold centres q = 30w-1 .. 30w+30; the
// link (q, q+1) and the bend centred at q are evaluated once, and lanes
// 1..30 add the five terms acting on their bead and own their link's and
// bend's energy. A tile is fetched (loads only) one tile ahead of its
// computation, so a warp's loads for its next tile are in flight while it
// computes the current one.
template <bool LS>
struct ChainRaw;
template <>
struct ChainRaw<false> {
    V3 c, e;  // the centre's position; lanes 0 and 31: the halo position (q-1, q+1)
    double2 lp, bp;
    unsigned fl;
};
template <>
struct ChainRaw<true> {  // positions x + lam*d: x and d of the centre and the halo
    V3 c, e, cd, ed;
    double2 lp, bp;
    unsigned fl;
};

template <bool LS>
__device__ __forceinline__ void chain_fetch(const PassArgs& a, const Pos& P, int w, ChainRaw<LS>& r) {
    const ChainDev& ch = a.ch;
    const int n = ch.n_pos;
    const int lane = threadIdx.x & 31;
    const int q = w * kWarpOut - 1 + lane;
    const bool in = q >= 0 && q < n;
    const int qe = lane == 0 ? q - 1 : q + 1;  // the halo position of lanes 0 and 31
    const bool halo = (lane == 0 || lane == 31) && qe >= 0 && qe < n;
    r.c = r.e = V3{0.0, 0.0, 0.0};
    if (in) r.c = load3(P.x + 3 * q);
    if (halo) r.e = load3(P.x + 3 * qe);
    if constexpr (LS) {
        r.cd = r.ed = V3{0.0, 0.0, 0.0};
        if (in) r.cd = load3(P.d + 3 * q);
        if (halo) r.ed = load3(P.d + 3 * qe);
    }
    r.fl = in ? ch.flags[q] : 0u;
    r.lp = in ? ch.link_p[q] : double2{0.0, 0.0};
    r.bp = in ? ch.bend_p[q] : double2{0.0, 0.0};
}

template <class R, bool E, bool F, bool LS>
__device__ __forceinline__ void chain_compute(const PassArgs& a, const Pos& P, double* __restrict__ f, int w,
                                              const ChainRaw<LS>& r, double (&acc)[kMainVals]) {
    const int n = a.ch.n_pos;
    const int lane = threadIdx.x & 31;
    const int q = w * kWarpOut - 1 + lane;
    const bool in = q >= 0 && q < n;
    V3 c = r.c, ce = r.e;
    if constexpr (LS) {
        c = move3(r.c, P.lam, r.cd);
        ce = move3(r.e, P.lam, r.ed);
    }
    const unsigned fl = r.fl;
    V3 cprev = shfl_up3(c), cnext = shfl_down3(c);
    if (lane == 0) cprev = ce;
    if (lane == 31) cnext = ce;
    const bool own = lane >= 1 && lane <= kWarpOut && in;
    if constexpr (F) {
        T3<R> Fl{0, 0, 0}, A{0, 0, 0}, B{0, 0, 0};
        if (fl & kLink) Fl = stretch_force<R>(c, cnext, r.lp.x, r.lp.y);
        if (fl & kBend) bend_force<R>(diff<R>(cprev, c), diff<R>(c, cnext), r.bp.x, r.bp.y, A, B);
        const T3<R> Fp = shfl_up3(Fl), Bp = shfl_up3(B), An = shfl_down3(A);
        if (own) {
            // link (q-1, q) acts on q; link (q, q+1) reacts on q; bends centred
            // at q-1 (third bead), q (middle), q+1 (first bead); summed in double
            const double fx = double(Fp.x) - double(Fl.x) + double(Bp.x) + (double(A.x) - double(B.x)) - double(An.x);
            const double fy = double(Fp.y) - double(Fl.y) + double(Bp.y) + (double(A.y) - double(B.y)) - double(An.y);
            const double fz = double(Fp.z) - double(Fl.z) + double(Bp.z) + (double(A.z) - double(B.z)) - double(An.z);
            target_add(a.t, f, 3 * q, fx, fy, fz);
        }
    }
    if constexpr (E) {
        if (own) {
            if (fl & kLink) acc[0] += stretch_energy<double>(c, cnext, r.lp.x, r.lp.y);
            if (fl & kBend) acc[1] += bend_energy<double>(diff<double>(cprev, c), diff<double>(c, cnext), r.bp.x, r.bp.y);
        }
    }
}

// Record i of bonded segment s (0 leftover stretch, 1 leftover bend, 2
// linker, 3 motor, 5 boundary): energy into acc[0], forces added to f.
template <class R, bool E, bool F>
__device__ __forceinline__ void bonded_record(const DeviceFF& ff, const ForceTarget& t, const Pos& P,
                                              double* __restrict__ f, int s, int i, double (&acc)[4]) {
    switch (s) {
        case 0:
            if (i < ff.n_stretch) {
                const int2 q = ff.stretch_bs[i];
                const double2 p = ff.stretch_p[i];
                const V3 c1 = P(q.x), c2 = P(q.y);
                if constexpr (E) acc[0] += stretch_energy<double>(c1, c2, p.x, p.y);
                if constexpr (F) {
                    const T3<R> Fs = stretch_force<R>(c1, c2, p.x, p.y);
                    target_add(t, f, q.y, Fs.x, Fs.y, Fs.z);
                    target_add(t, f, q.x, -Fs.x, -Fs.y, -Fs.z);
                }
            }
            break;
        case 1:
            if (i < ff.n_bend) {
                const int4 q = ff.bend_bs[i];
                const double2 p = ff.bend_p[i];
                const V3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z);
                if constexpr (E) acc[0] += bend_energy<double>(diff<double>(c1, c2), diff<double>(c2, c3), p.x, p.y);
                if constexpr (F) {
                    T3<R> Fr1, Fr2;
                    bend_force<R>(diff<R>(c1, c2), diff<R>(c2, c3), p.x, p.y, Fr1, Fr2);
                    target_add(t, f, q.x, -Fr1.x, -Fr1.y, -Fr1.z);
                    target_add(t, f, q.y, Fr1.x - Fr2.x, Fr1.y - Fr2.y, Fr1.z - Fr2.z);
                    target_add(t, f, q.z, Fr2.x, Fr2.y, Fr2.z);
                }
            }
            break;
        case 2:
        case 3: {
            const int n = s == 2 ? ff.n_linker : ff.n_motor;
            if (i < n) {
                const int4 q = s == 2 ? ff.linker_bs[i] : ff.motor_bs[i];
                const double4 p = s == 2 ? ff.linker_p[i] : ff.motor_p[i];
                const V3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z), c4 = P(q.w);
                if constexpr (E) acc[0] += spring_energy<double>(c1, c2, c3, c4, p.x, p.y, p.z, p.w);
                if constexpr (F) {
                    const T3<R> Fl = spring_force<R>(c1, c2, c3, c4, p.x, p.y, p.z, p.w);
                    const R a1 = R(1) - R(p.z), a2 = R(p.z), b1 = R(1) - R(p.w), b2 = R(p.w);
                    target_add(t, f, q.x, -Fl.x * a1, -Fl.y * a1, -Fl.z * a1);
                    target_add(t, f, q.y, -Fl.x * a2, -Fl.y * a2, -Fl.z * a2);
                    target_add(t, f, q.z, Fl.x * b1, Fl.y * b1, Fl.z * b1);
                    target_add(t, f, q.w, Fl.x * b2, Fl.y * b2, Fl.z * b2);
                }
            }
            break;
        }
        default:
            if (i < ff.n_boundary) {
                const int o = ff.boundary_bs[i];
                const double2 p = ff.boundary_p[i];
                const double4 pl = ff.planes[ff.boundary_plane[i]];
                const V3 c = P(o);
                if constexpr (E) acc[0] += boundary_energy<double>(pl, c, p.x, p.y);
                if constexpr (F) {
                    const R f0 = boundary_force_mag<R>(pl, c, p.x, p.y);
                    target_add(t, f, o, f0 * R(pl.x), f0 * R(pl.y), f0 * R(pl.z));
                }
            }
            break;
    }
}

// Bonded chunk b of the main kernel: blockDim records of one segment.
template <class R, bool E, bool F>
__device__ __forceinline__ void main_chunk(const PassArgs& a, const Pos& P, double* __restrict__ f, int b,
                                           double (&acc)[kMainVals]) {
    int k = 0;
#pragma unroll
    for (int j = 1; j < 5; ++j) k += b >= a.seg[j] ? 1 : 0;
    const int i = (b - a.seg[k]) * blockDim.x + threadIdx.x;
    double e[4] = {0.0, 0.0, 0.0, 0.0};
    bonded_record<R, E, F>(a.ff, a.t, P, f, k == 4 ? 5 : k, i, e);
    // acc: 0 stretching, 1 bending, 2 linker, 3 motor, 4 boundary
#pragma unroll
    for (int j = 0; j < kMainVals; ++j)
        if (j == k) acc[j] += e[0];
}

// The main kernel's grid is resident (a few blocks per SM) and walks its
// work in two phases: the chain tiles, one warp per tile with the next tile
// fetched while the current one is computed, then the bonded chunks of
// blockDim records (a.seg[k] is the first chunk of leftover stretch,
// leftover bend, linker, motor, boundary). In an energy pass both walks are
// fixed by the grid, so each block's energy row covers a fixed set of tiles
// and chunks and the sums are reproducible; a force-only pass takes its
// tiles and chunks from work counters instead.
template <class R, bool E, bool F, bool LS>
__global__ void __launch_bounds__(kPassThreads, main_blocks_per_sm<R, E, F, LS>())
    k_pass_main(const __grid_constant__ PassArgs a) {
    PASS_TRACE_BEGIN
    if (F && a.t.skip && *a.t.skip) return;
    double* __restrict__ f = F ? target_force(a.t) : nullptr;
    const Pos P = pos_of(a);
    double acc[kMainVals] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // no chain units: the chain runs in the streamed chain kernel
    const int tiles = a.nch > 0 ? (a.ch.n_pos + kWarpOut - 1) / kWarpOut : 0;
    if constexpr (F && !E) {
        // force-only passes: one unit per block, so the hardware hands units
        // to SMs as they free up (the pass's other kernels hold some SMs at
        // first). Units [0, a.nch) are chain units, kTilesPerWarp consecutive
        // tiles per warp, each fetched while the one before is computed;
        // then one bonded chunk per unit.
        const int u = blockIdx.x;
        if (u < a.nch) {
            const int w0 = (u * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kTilesPerWarp;
            ChainRaw<LS> cur, nxt;
            if (w0 < tiles) chain_fetch<LS>(a, P, w0, cur);
#pragma unroll 1
            for (int j = 0; j < kTilesPerWarp && w0 + j < tiles; ++j) {
                const int w = w0 + j;
                if (j + 1 < kTilesPerWarp && w + 1 < tiles) chain_fetch<LS>(a, P, w + 1, nxt);
                chain_compute<R, E, F, LS>(a, P, f, w, cur, acc);
                cur = nxt;
            }
        } else {
            main_chunk<R, E, F>(a, P, f, u - a.nch, acc);
        }
    } else {
        const int warps = gridDim.x * (blockDim.x >> 5);
        int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        ChainRaw<LS> cur, nxt;
        if (w < tiles) chain_fetch<LS>(a, P, w, cur);
        for (; w < tiles; w += warps) {
            if (w + warps < tiles) chain_fetch<LS>(a, P, w + warps, nxt);
            chain_compute<R, E, F, LS>(a, P, f, w, cur, acc);
            cur = nxt;
        }
        for (int b = blockIdx.x; b < a.nb_main; b += gridDim.x) main_chunk<R, E, F>(a, P, f, b, acc);
    }
    // a force-only pass has no rows here: the main kernel's blocks take no ticket
    if constexpr (E) block_done<0, E, F>(a, acc, a.row_main + blockIdx.x, false);
    PASS_TRACE_END(0 + (E ? 10 : 0))
}

// ------------------------------------------------------------ streamed chain
// Chain segments staged through shared memory (pass layout 2). Segment s
// covers output positions [s0, s0 + kChainSeg), s0 = s * kChainSeg, as
// kChainWarps warp tiles of kWarpOut positions (the warp-tile kernel's
// tiles, lanes holding centres s0 + 30w - 1 + lane). A tile needs the
// centres s0-1 .. s0+S and the positions s0-2 .. s0+S+1.
//
// Warp-specialized pipeline: a producer warp issues bulk copies
// (cp.async.bulk, completion counted in bytes on the stage's "full"
// mbarrier) of the next kChainStages segments' coordinates, link and bend
// parameters and flags, so a block keeps ~55 KB of loads in flight with no
// registers held for them. Each consumer warp computes its tile from shared
// memory on its own (neighbours by warp shuffles, no block barrier) and
// arrives on the stage's "empty" mbarrier; the producer refills a stage once
// all consumer warps have arrived. Segments whose windows would start before
// the arrays or run past their ends are filled by the producer warp with
// plain loads instead.
constexpr int kChainWarps = kChainThreads / 32;  // consumer warps (one tile each per segment)
constexpr int kSegPos = kChainSeg + 4;           // positions s0-2 .. s0+S+1
constexpr int kSegCen = kChainSeg + 2;           // centres s0-1 .. s0+S
static_assert(kChainSeg == kChainWarps * kWarpOut, "a segment is one tile per consumer warp");
static_assert(kChainSeg % 2 == 0, "segment starts must keep the coordinate window 16-byte aligned");

template <bool LS>
struct ChainStage {
    double x[3 * kSegPos];             // positions s0-2 .. s0+S+1
    double d[LS ? 3 * kSegPos : 2];    // their search directions (x + lam d passes)
    double2 lp[kSegCen];               // (k, l0) of centres s0-1 .. s0+S
    double2 bp[kSegCen];               // (k, theta0) of the same centres
    unsigned char fl[kChainSeg + 32];  // flags from (s0-1) rounded down to 16 bytes
};

// Dynamic shared memory of a chain block with `stages` stages.
template <bool LS>
constexpr size_t chain_smem_bytes(int stages = kChainStages) {
    return stages * sizeof(ChainStage<LS>) + 2 * stages * sizeof(unsigned long long);
}

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(smem_addr(bar)) : "memory");
}
// Waits for the phase of the given parity to complete; gives up after a
// bounded number of polls (false).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const unsigned a = smem_addr(bar);
    for (int i = 0; i < (1 << 20); ++i) {
        unsigned done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from global to shared memory, counted on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// The flag window of the segment at s0: first byte and length, and whether
// all of the segment's windows lie inside the arrays (bulk copies).
__device__ __forceinline__ int flag_first(int s0) { return (s0 - 1) & ~15; }
__device__ __forceinline__ int flag_bytes(int s0) { return ((s0 + kChainSeg + 1 - flag_first(s0)) + 15) & ~15; }
__device__ __forceinline__ bool seg_inside(int s0, int n) {
    return s0 >= 2 && s0 + kChainSeg + 2 <= n && flag_first(s0) + flag_bytes(s0) <= n;
}

// Producer warp: loads segment seg into stage st and completes the stage's
// full barrier, by bulk copies (lane 0) or by plain loads (all lanes; zeros
// outside the arrays).
template <bool LS>
__device__ __forceinline__ void chain_produce(const PassArgs& a, const double* d, bool bulk, int seg,
                                              ChainStage<LS>& st, unsigned long long* full) {
    const int n = a.ch.n_pos;
    const int s0 = seg * kChainSeg;
    const int lane = threadIdx.x & 31;
    if (bulk && seg_inside(s0, n)) {
        if (lane == 0) {
            // the stage may last have been written through the generic proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const unsigned bx = 24u * kSegPos, bp = 16u * kSegCen;
            const int ff = flag_first(s0);
            const unsigned bf = (unsigned)flag_bytes(s0);
            mbar_expect_tx(full, bx * (LS ? 2u : 1u) + 2u * bp + bf);
            bulk_load(st.x, a.x + 3 * (s0 - 2), bx, full);
            if constexpr (LS) bulk_load(st.d, d + 3 * (s0 - 2), bx, full);
            bulk_load(st.lp, a.ch.link_p + (s0 - 1), bp, full);
            bulk_load(st.bp, a.ch.bend_p + (s0 - 1), bp, full);
            bulk_load(st.fl, a.ch.flags + ff, bf, full);
        }
        return;
    }
    for (int i = lane; i < 3 * kSegPos; i += 32) {
        const int q = s0 - 2 + i / 3;
        const bool in = q >= 0 && q < n;
        st.x[i] = in ? __ldg(a.x + 3 * (s0 - 2) + i) : 0.0;
        if constexpr (LS) st.d[i] = in ? __ldg(d + 3 * (s0 - 2) + i) : 0.0;
    }
    const int fo = (s0 - 1) - flag_first(s0);
    for (int j = lane; j < kSegCen; j += 32) {
        const int c = s0 - 1 + j;
        const bool in = c >= 0 && c < n;
        st.lp[j] = in ? a.ch.link_p[c] : double2{0.0, 0.0};
        st.bp[j] = in ? a.ch.bend_p[c] : double2{0.0, 0.0};
        st.fl[fo + j] = in ? a.ch.flags[c] : (unsigned char)0;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(full);  // release: the consumers see the stores
}

template <bool LS>
__device__ __forceinline__ V3 stage_pos(const ChainStage<LS>& st, int p, double lam) {
    const V3 v{st.x[3 * p], st.x[3 * p + 1], st.x[3 * p + 2]};
    if constexpr (LS) return move3(v, lam, V3{st.d[3 * p], st.d[3 * p + 1], st.d[3 * p + 2]});
    return v;
}

// The grid is resident and walks the segments in a fixed order (blockIdx.x,
// + gridDim.x, ...), so each block's energy row covers a fixed set of
// centres. Force-only passes take no tickets here.
template <class R, bool E, bool F, bool LS>
__global__ void __launch_bounds__(kChainThreads + 32) k_pass_chain(const __grid_constant__ PassArgs a) {
    PASS_TRACE_BEGIN
    if (F && a.t.skip && *a.t.skip) return;
    extern __shared__ __align__(128) unsigned char chain_smem[];
    const int K = a.chain_stages;  // stages of the ring (1 when each block takes one segment)
    ChainStage<LS>* stages = reinterpret_cast<ChainStage<LS>*>(chain_smem);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(chain_smem + K * sizeof(ChainStage<LS>));
    unsigned long long* empty = full + K;
    double* __restrict__ f = F ? target_force(a.t) : nullptr;
    const double* d = LS ? a.t.d : nullptr;
    const double lam = LS ? *a.t.lam : 0.0;
    const int n = a.ch.n_pos;
    const int nseg = (n + kChainSeg - 1) / kChainSeg;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool bulk = aligned16(a.x) && (!LS || aligned16(d)) && aligned16(a.ch.link_p) && aligned16(a.ch.bend_p) &&
                      aligned16(a.ch.flags);
    double acc[kMainVals] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k) {
            mbar_init(full + k, 1);
            mbar_init(empty + k, kChainWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == kChainWarps) {
        // producer: segment m of this block goes to stage m % K once its
        // previous occupant (segment m - K) has been consumed
        int m = 0;
        bool ok = true;
        for (int seg = blockIdx.x; seg < nseg; seg += gridDim.x, ++m) {
            const int k = m % K;
            if (m >= K) {
                bool ready = lane == 0 ? mbar_wait(empty + k, ((m / K) - 1) & 1) : true;
                ready = __shfl_sync(kFull, ready, 0);
                if (!ready) {
                    ok = false;
                    break;
                }
            }
            chain_produce<LS>(a, d, bulk, seg, stages[k], full + k);
        }
        if (!ok && lane == 0) {
            // the consumers stopped: report it and wait (bounded) for the
            // copies still in flight before the block's shared memory goes
            if (F) atomicOr(a.f_status, 8);
            if (E) atomicOr(a.e_bad, 4);
            for (int q = m - K; q < m; ++q)
                if (q >= 0) mbar_wait(full + q % K, (q / K) & 1);
        }
    } else {
        int it = 0;
        for (int seg = blockIdx.x; seg < nseg; seg += gridDim.x, ++it) {
            const int k = it % K;
            const ChainStage<LS>& st = stages[k];
            bool ready = lane == 0 ? mbar_wait(full + k, (it / K) & 1) : true;
            ready = __shfl_sync(kFull, ready, 0);
            if (!ready) {
                if (lane == 0) {
                    if (F) atomicOr(a.f_status, 8);
                    if (E) atomicOr(a.e_bad, 4);
                }
                break;
            }
            const int s0 = seg * kChainSeg;
            const int j = warp * kWarpOut + lane;  // centre s0 - 1 + j
            const int q = s0 - 1 + j;
            const unsigned fl = st.fl[(s0 - 1) - flag_first(s0) + j];
            const V3 cp = stage_pos<LS>(st, j, lam), c = stage_pos<LS>(st, j + 1, lam),
                     cn = stage_pos<LS>(st, j + 2, lam);
            const double2 lp = st.lp[j], bp = st.bp[j];
            const bool own = lane >= 1 && lane <= kWarpOut && q < n;
            if constexpr (F) {
                T3<R> Fl{0, 0, 0}, A{0, 0, 0}, B{0, 0, 0};
                if (fl & kLink) Fl = stretch_force<R>(c, cn, lp.x, lp.y);
                if (fl & kBend) bend_force<R>(diff<R>(cp, c), diff<R>(c, cn), bp.x, bp.y, A, B);
                const T3<R> Fp = shfl_up3(Fl), Bp = shfl_up3(B), An = shfl_down3(A);
                if (own) {
                    // link (q-1, q) acts on q; link (q, q+1) reacts on q; bends
                    // centred at q-1 (third bead), q (middle), q+1 (first bead)
                    const double fx =
                        double(Fp.x) - double(Fl.x) + double(Bp.x) + (double(A.x) - double(B.x)) - double(An.x);
                    const double fy =
                        double(Fp.y) - double(Fl.y) + double(Bp.y) + (double(A.y) - double(B.y)) - double(An.y);
                    const double fz =
                        double(Fp.z) - double(Fl.z) + double(Bp.z) + (double(A.z) - double(B.z)) - double(An.z);
                    target_add(a.t, f, 3 * q, fx, fy, fz);
                }
            }
            if constexpr (E) {
                if (own) {
                    if (fl & kLink) acc[0] += stretch_energy<double>(c, cn, lp.x, lp.y);
                    if (fl & kBend) acc[1] += bend_energy<double>(diff<double>(cp, c), diff<double>(c, cn), bp.x, bp.y);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + k);
        }
    }
    if constexpr (E) block_done<0, E, F>(a, acc, a.row_chain + blockIdx.x, false);
    PASS_TRACE_END(4 + (E ? 10 : 0))
}

// ------------------------------------------------------------ branch points
template <class R, bool E, bool F>
__global__ void __launch_bounds__(kPassThreads) k_pass_branch(const __grid_constant__ PassArgs a) {
    PASS_TRACE_BEGIN
    if (F && a.t.skip && *a.t.skip) return;
    double* __restrict__ f = F ? target_force(a.t) : nullptr;
    const Pos P = pos_of(a);
    const DeviceFF& ff = a.ff;
    double acc[kBranchVals] = {0.0, 0.0, 0.0, 0.0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ff.n_branch) {
        const int4 q = ff.branch_bs[i];
        const double4 pa = ff.branch_pa[i], pb = ff.branch_pb[i];
        const V3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z), c4 = P(q.w);
        const int m = ff.branch_mask;
        if constexpr (E) {
            if (m & 1) acc[0] += branch_stretch_energy<double>(c1, c2, c3, pa.y, pa.z, pa.x);
            if (m & 2) acc[1] += bend_energy<double>(diff<double>(c1, c2), diff<double>(c3, c4), pa.w, pb.x);
            if (m & 4) acc[2] += branch_dihedral_energy<double>(c1, c2, c3, c4, pb.y, pa.x);
            if (m & 8) acc[3] += branch_position_energy<double>(c1, c2, c3, pb.z, pa.x);
        }
        if constexpr (F) {
            T3<R> F1{0, 0, 0}, F2{0, 0, 0}, F3{0, 0, 0}, F4{0, 0, 0};
            if (m & 1) {
                const T3<R> g = branch_stretch_force<R>(c1, c2, c3, pa.y, pa.z, pa.x);
                const R pm1 = R(pa.x) - R(1), pp = R(pa.x);
                F1.x += -g.x * pm1; F1.y += -g.y * pm1; F1.z += -g.z * pm1;
                F2.x += g.x * pp; F2.y += g.y * pp; F2.z += g.z * pp;
                F3.x += -g.x; F3.y += -g.y; F3.z += -g.z;
            }
            if (m & 2) {
                T3<R> Fr1, Fr2;
                bend_force<R>(diff<R>(c1, c2), diff<R>(c3, c4), pa.w, pb.x, Fr1, Fr2);
                F1.x += -Fr1.x; F1.y += -Fr1.y; F1.z += -Fr1.z;
                F2.x += Fr1.x; F2.y += Fr1.y; F2.z += Fr1.z;
                F3.x += -Fr2.x; F3.y += -Fr2.y; F3.z += -Fr2.z;
                F4.x += Fr2.x; F4.y += Fr2.y; F4.z += Fr2.z;
            }
            if (m & 4) {
                T3<R> L1, L2, L3, L4;
                branch_dihedral_force<R>(c1, c2, c3, c4, pb.y, pa.x, L1, L2, L3, L4);
                F1.x += L1.x; F1.y += L1.y; F1.z += L1.z;
                F2.x += L2.x; F2.y += L2.y; F2.z += L2.z;
                F3.x += L3.x; F3.y += L3.y; F3.z += L3.z;
                F4.x += L4.x; F4.y += L4.y; F4.z += L4.z;
            }
            if (m & 8) {
                T3<R> P1, P2, P3;
                branch_position_force<R>(c1, c2, c3, pb.z, pa.x, P1, P2, P3);
                F1.x += P1.x; F1.y += P1.y; F1.z += P1.z;
                F2.x += P2.x; F2.y += P2.y; F2.z += P2.z;
                F3.x += P3.x; F3.y += P3.y; F3.z += P3.z;
            }
            target_add(a.t, f, q.x, F1.x, F1.y, F1.z);
            target_add(a.t, f, q.y, F2.x, F2.y, F2.z);
            target_add(a.t, f, q.z, F3.x, F3.y, F3.z);
            target_add(a.t, f, q.w, F4.x, F4.y, F4.z);
        }
    }
    if constexpr (E) block_done<1, E, F>(a, acc, a.row_branch + blockIdx.x, false);
    PASS_TRACE_END(1 + (E ? 10 : 0))
}

// ------------------------------------------------------------ excluded volume
// One pair per thread, FP64. A pair whose analytic energy or forces the
// reference would reject goes to the fallback queue instead.
template <bool E, bool F, bool EXACT>
__global__ void __launch_bounds__(kExclThreadsMax) k_pass_excl(const __grid_constant__ PassArgs a) {
    PASS_TRACE_BEGIN
    if (F && a.t.skip && *a.t.skip) return;
    double* __restrict__ f = F ? target_force(a.t) : nullptr;
    const Pos P = pos_of(a);
    const DeviceFF& ff = a.ff;
    double acc[kExclVals] = {0.0};
    bool queued = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ff.n_excl; i += gridDim.x * blockDim.x) {
        const int4 q = ff.excl_bs[i];
        const double krs = ff.excl_krs[i];
        const V3 c1 = P(q.x), c2 = P(q.y), c3 = P(q.z), c4 = P(q.w);
        if constexpr (E) {
            const double U = excl_energy<double>(c1, c2, c3, c4, krs);
            if (excl_energy_bad(U)) {
                const int slot = atomicAdd(a.e_fb_count, 1);
                if (slot < a.e_fb_cap) a.e_fb_list[slot] = make_int2(i, 0);
                else atomicOr(a.e_bad, 2);
                queued = true;
            } else {
                acc[0] += U;
            }
        }
        if constexpr (F) {
            T3<double> fo[4];
            if (excl_force<EXACT>(c1, c2, c3, c4, krs, fo)) {
                target_add(a.t, f, q.x, fo[0].x, fo[0].y, fo[0].z);
                target_add(a.t, f, q.y, fo[1].x, fo[1].y, fo[1].z);
                target_add(a.t, f, q.z, fo[2].x, fo[2].y, fo[2].z);
                target_add(a.t, f, q.w, fo[3].x, fo[3].y, fo[3].z);
            } else {
                const int slot = atomicAdd(a.f_fb_count, 1);
                if (slot < a.f_fb_cap) a.f_fb_list[slot] = i;
                else atomicOr(a.f_status, 2);
                queued = true;
            }
        }
    }
    block_done<2, E, F>(a, acc, a.row_excl + blockIdx.x, queued);
    PASS_TRACE_END(2 + (E ? 10 : 0))
}

// ------------------------------------------------------------ zero fill
__global__ void __launch_bounds__(kZeroThreads) k_pass_zero(const ForceTarget t, int n3) {
    PASS_TRACE_BEGIN
    if (t.skip && *t.skip) return;
    double* __restrict__ f = target_force(t);
    // cudaMalloc'd buffers are 256-byte aligned: pairs of doubles, then the odd tail
    double2* __restrict__ f2 = reinterpret_cast<double2*>(f);
    const int n2 = n3 >> 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) f2[i] = double2{0.0, 0.0};
    if ((n3 & 1) && blockIdx.x == 0 && threadIdx.x == 0) f[n3 - 1] = 0.0;
    PASS_TRACE_END(3)
}

template <class R, bool E, bool F>
void launch_kernels(const PassArgs& a, const PassGeometry& g, int prec, cudaStream_t s_main, cudaStream_t s_branch,
                    cudaStream_t s_excl, cudaStream_t s_chain) {
    // the excluded-volume pairs first: their FP64 chains are the longest, and
    // their blocks should be resident before the main kernel's fill the SMs
    if (g.excl_blocks > 0) {
        if (prec == MEDYAN_PREC_FP64)
            k_pass_excl<E, F, true><<<g.excl_blocks, g.excl_threads, 0, s_excl>>>(a);
        else
            k_pass_excl<E, F, false><<<g.excl_blocks, g.excl_threads, 0, s_excl>>>(a);
    }
    if (g.chain_blocks > 0) {
        if (a.t.d)
            k_pass_chain<R, E, F, true>
                <<<g.chain_blocks, kChainThreads + 32, chain_smem_bytes<true>(g.chain_stages), s_chain>>>(a);
        else
            k_pass_chain<R, E, F, false>
                <<<g.chain_blocks, kChainThreads + 32, chain_smem_bytes<false>(g.chain_stages), s_chain>>>(a);
    }
    if (g.branch_blocks > 0) k_pass_branch<R, E, F><<<g.branch_blocks, g.threads, 0, s_branch>>>(a);
    const int mb = E ? g.main_blocks : g.main_blocks_forces;
    if (a.t.d)
        k_pass_main<R, E, F, true><<<mb, g.threads, 0, s_main>>>(a);
    else
        k_pass_main<R, E, F, false><<<mb, g.threads, 0, s_main>>>(a);
}

// Opts every chain kernel in to its dynamic shared memory (above the 48 KB
// default).
template <class R, bool E, bool F>
cudaError_t chain_attrs() {
    cudaError_t e = cudaFuncSetAttribute(k_pass_chain<R, E, F, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)chain_smem_bytes<false>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_pass_chain<R, E, F, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)chain_smem_bytes<true>());
    return e;
}

}  // namespace

namespace {
int g_num_sms = 148;  // SMs of the device (set at init; B200: 148)
}  // namespace

PassGeometry pass_geometry(const ChainDev& ch, const DeviceFF& ff, bool stream) {
    PassGeometry g{};
    g.threads = kPassThreads;
    g.excl_threads = excl_block_of(ff) > 128 ? 128 : excl_block_of(ff);
    const int tiles = (ch.n_pos + kWarpOut - 1) / kWarpOut;
    const int warps = g.threads / 32;
    g.nch = (tiles + warps - 1) / warps;
    const int counts[5] = {ff.n_stretch, ff.n_bend, ff.n_linker, ff.n_motor, ff.n_boundary};
    g.seg[0] = 0;
    for (int k = 0; k < 5; ++k) g.seg[k + 1] = g.seg[k] + (counts[k] + g.threads - 1) / g.threads;
    g.nb_main = g.seg[5];
    // fixed grids that walk the units (one block at least: it can finish the pass)
    const int units = g.nch + g.nb_main;
    // a resident grid that walks the units: one block per unit measured
    // slower (each block's end, a fence and two tickets, holds its SM slot)
    const int cap = g_num_sms * kMainBlocksPerSM;
    g.main_blocks = units < 1 ? 1 : (units < cap ? units : cap);
    g.branch_blocks = (ff.n_branch + g.threads - 1) / g.threads;
    const int eb = (ff.n_excl + g.excl_threads - 1) / g.excl_threads;
    const int ecap = g_num_sms * 32;
    g.excl_blocks = eb < ecap ? eb : ecap;
    // a force-only pass: one unit per block, chain units of kTilesPerWarp
    // tiles per warp
    g.nch_forces = (tiles + warps * kTilesPerWarp - 1) / (warps * kTilesPerWarp);
    const int funits = g.nch_forces + g.nb_main;
    g.main_blocks_forces = funits < 1 ? 1 : funits;
    g.stream = stream;
    g.nseg = (ch.n_pos + kChainSeg - 1) / kChainSeg;
    g.chain_blocks = 0;
    g.chain_stages = kChainStages;
    if (stream) {
        // the chain kernel takes the chain; the main kernel keeps the
        // records. One unit (chain segment, record chunk) per block and one
        // energy row per unit: the hardware balances the blocks over the SMs
        // (resident grids walking fixed unit sets left some SMs busy twice
        // as long as the average), and the sums still add each unit's row
        // in a fixed order
        g.nch = g.nch_forces = 0;
        g.main_blocks = g.nb_main < 1 ? 1 : g.nb_main;
        g.main_blocks_forces = g.nb_main < 1 ? 1 : g.nb_main;
        g.chain_blocks = g.nseg;
        g.chain_stages = 1;
    }
    g.rows = g.main_blocks + g.branch_blocks + g.excl_blocks + g.chain_blocks;
    g.groups = (g.rows + kGroup - 1) / kGroup;
    return g;
}

namespace {

// The argument block of one energy-only or force-only pass.
PassArgs pass_args(const ChainDev& ch, const DeviceFF& ff, const PassGeometry& g, const double* x,
                   const ForceTarget* t, bool energy, const LambdaSet* lam_set, const EnergyScratch& es,
                   const ForceScratch& fs, const PassScratch& ps) {
    PassArgs a{};
    a.ch = ch;
    a.ff = ff;
    a.x = x;
    if (t) a.t = *t;
    a.rows = ps.rows;
    a.group_rows = ps.group_rows;
    a.group_ticket = ps.group_ticket;
    a.ticket = ps.ticket;
    // the blocks that take tickets: every block of an energy pass; of a
    // force-only pass the excluded-volume blocks, which own the fallback queue
    a.n_rows = energy ? g.rows : g.excl_blocks;
    a.n_groups = (a.n_rows + kGroup - 1) / kGroup;
    a.row_main = 0;
    a.row_branch = g.main_blocks;
    a.row_excl = energy ? g.main_blocks + g.branch_blocks : 0;
    a.row_chain = g.main_blocks + g.branch_blocks + g.excl_blocks;  // energy passes only
    a.chain_stages = g.chain_stages;
    a.nch = energy ? g.nch : g.nch_forces;
    a.nb_main = g.nb_main;
    for (int k = 0; k < 6; ++k) a.seg[k] = g.seg[k];
    a.out = es.out;
    a.lam_set = lam_set;
    a.e_fb_count = es.fb_count;
    a.e_fb_list = es.fb_list;
    a.e_fb_cap = fb_capacity(es.fb_cap);
    a.f_fb_cap = fb_capacity(fs.fb_cap);
    a.e_bad = es.bad;
    a.f_fb_count = fs.fb_count;
    a.f_fb_list = fs.fb_list;
    a.f_status = fs.status;
    return a;
}

}  // namespace

void launch_pass_fused(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const ForceTarget* t,
                       bool energy, const LambdaSet* lam_set, const EnergyScratch& es, const ForceScratch& fs,
                       const PassScratch& ps, const PassScratch& ps_forces, cudaStream_t s, const Fork* fk,
                       bool stream) {
    const PassGeometry g = pass_geometry(ch, ff, stream);
    const bool force = t != nullptr;
    const bool mixed = prec == MEDYAN_PREC_MIXED;
    // streams: the force side on s, sides 0-1 (and 5 for a streamed chain);
    // the energy side on sides 2-4 (and 6) (everything on s without a fork)
    constexpr int kSides = 7;
    cudaStream_t sf[4] = {s, s, s, s}, se[4] = {s, s, s, s};
    if (fk) {
        cudaEventRecord(fk->fork, s);
        for (int k = 0; k < kSides; ++k) cudaStreamWaitEvent(fk->side[k], fk->fork, 0);
        sf[1] = fk->side[0];
        sf[2] = fk->side[1];
        sf[3] = fk->side[5];
        se[0] = fk->side[2];
        se[1] = fk->side[3];
        se[2] = fk->side[4];
        se[3] = fk->side[6];
    }
    if (energy) {
        // energy-only kernels (FP64 in both modes), their own tickets
        const PassArgs a = pass_args(ch, ff, g, x, t, true, lam_set, es, fs, ps);
        launch_kernels<double, true, false>(a, g, prec, se[0], se[1], se[2], se[3]);
    }
    if (force) {
        // the zero fill, then the force-only kernels side by side
        const PassArgs a = pass_args(ch, ff, g, x, t, false, lam_set, es, fs, ps_forces);
        const int n3 = 3 * ch.n_pos;
        int zb = (n3 / 2 + kZeroThreads - 1) / kZeroThreads;
        zb = zb < 1 ? 1 : (zb > 148 * 8 ? 148 * 8 : zb);
        if (n3 > 0) k_pass_zero<<<zb, kZeroThreads, 0, s>>>(*t, n3);
        if (fk) {
            cudaEventRecord(fk->mid, s);
            cudaStreamWaitEvent(sf[1], fk->mid, 0);
            cudaStreamWaitEvent(sf[2], fk->mid, 0);
            cudaStreamWaitEvent(sf[3], fk->mid, 0);
        }
        if (mixed) launch_kernels<float, false, true>(a, g, prec, sf[0], sf[1], sf[2], sf[3]);
        else launch_kernels<double, false, true>(a, g, prec, sf[0], sf[1], sf[2], sf[3]);
    }
    if (fk) {
        for (int k = 0; k < kSides; ++k) {
            cudaEventRecord(fk->join[k], fk->side[k]);
            cudaStreamWaitEvent(s, fk->join[k], 0);
        }
    }
    if (force) launch_fixed_to_double(*t, 3 * ch.n_pos, s);
}

cudaError_t init_pass_kernels() {
    static std::mutex mu;
    static bool filled[64];
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (filled[dev]) return cudaSuccess;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (sms > 0) g_num_sms = sms;
    e = chain_attrs<double, true, false>();
    if (e == cudaSuccess) e = chain_attrs<double, false, true>();
    if (e == cudaSuccess) e = chain_attrs<float, false, true>();
    if (e != cudaSuccess) return e;
    cudaStream_t s = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    k_fill_quadrature_grids<<<1, 1, 0, s>>>();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e == cudaSuccess) filled[dev] = true;
    return e;
}

}  // namespace mb

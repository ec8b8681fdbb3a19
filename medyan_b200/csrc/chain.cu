// chain.cu — filament stretching and bending as one bead-centric pass, and
// the library's internal bead order.
//
// Internal order. At create the beads are put in filament-chain order:
// walking the stretching links (b1 -> b2) from every bead without a
// predecessor, in bead-index order, gives each bead a position p, beads of a
// filament consecutive (FilamentStretching::vectorize,
// Filament/FilamentStretching.cpp:24-44, and FilamentBending::vectorize,
// Filament/FilamentBending.cpp:28-66, produce exactly this structure). The
// handle stores coordinates, forces and every bead offset in that order and
// converts at the host boundary, so the chain kernels read and write the
// coordinate array as contiguous tiles.
//
// Chains. A link (b1 -> b2) with pos[b2] == pos[b1] + 1 and a bend
// (b1, b2, b3) with pos[b1] + 1 == pos[b2] == pos[b3] - 1 are evaluated
// here; anything else (a second link out of a bead, links closing a cycle,
// bends across chain ends, interactions of a later update that no longer fit
// the order) stays on the generic per-interaction path.
//
// Both kernels work on warp tiles of consecutive positions: each lane loads
// one position (coalesced, no index loads) and gets its neighbours by warp
// shuffles, so there is no shared memory and no block barrier. The force
// kernel evaluates each link and bend once and writes each bead's force with
// a plain store; every bead is written, so the pass also initializes the
// force array for the potentials that add atomically afterwards. The energy
// kernel evaluates the link and bend owned by each position at up to
// kMaxLambda step sizes from one read of x and d.
#include <algorithm>
#include <vector>

#include "handle.h"
#include "potentials.cuh"

namespace mb {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpOut = 30;  // forces written per warp: lanes 1..30 of 32 centres
constexpr unsigned char kLink = 1, kBend = 2;
constexpr unsigned kFull = 0xffffffffu;

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

// Coordinates of internal position q (zero outside [0, n)).
__device__ __forceinline__ V3 pos_of(const double* __restrict__ x, int n, int q) {
    return (q >= 0 && q < n) ? load3(x + 3 * q) : V3{0.0, 0.0, 0.0};
}

// Forces. Each warp owns 32 consecutive centres q = p0-1 .. p0+30 (one per
// lane): the lane loads its position, flags and parameters (coalesced, all
// independent), gets its neighbours' coordinates by shuffles (lanes 0 and 31
// load the one outside the warp), evaluates the link (q, q+1) and the bend
// centred at q once, and lanes 1..30 sum the five terms acting on their
// position from their neighbours by shuffles. No shared memory, no block
// barriers; every position is written exactly once.
template <class R>
__global__ void __launch_bounds__(kMaxShapeThreads) k_chain_forces(const ChainDev ch, const double* __restrict__ x,
                                                           const ForceTarget tgt) {
    if (tgt.skip && *tgt.skip) return;
    double* __restrict__ f = target_force(tgt);
    const double* __restrict__ d = tgt.d;
    const double lam = tgt.lam ? *tgt.lam : 0.0;
    const int n = ch.n_pos;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; (long long)w * kWarpOut < n; w += nw) {
        const int q = w * kWarpOut - 1 + lane;
        const bool in = q >= 0 && q < n;
        const int qe = lane == 0 ? q - 1 : q + 1;  // the halo position of lanes 0 and 31
        V3 c = pos_of(x, n, q), ce{0.0, 0.0, 0.0};
        if (lane == 0 || lane == 31) ce = pos_of(x, n, qe);
        if (d) {
            c = move3(c, lam, pos_of(d, n, q));
            if (lane == 0 || lane == 31) ce = move3(ce, lam, pos_of(d, n, qe));
        }
        const unsigned char fl = in ? ch.flags[q] : 0;
        const double2 lp = in ? ch.link_p[q] : double2{0.0, 0.0};
        const double2 bp = in ? ch.bend_p[q] : double2{0.0, 0.0};
        V3 cprev = shfl_up3(c), cnext = shfl_down3(c);
        if (lane == 0) cprev = ce;
        if (lane == 31) cnext = ce;
        T3<R> F{0, 0, 0}, A{0, 0, 0}, B{0, 0, 0};
        if (fl & kLink) F = stretch_force<R>(c, cnext, lp.x, lp.y);
        if (fl & kBend) bend_force<R>(diff<R>(cprev, c), diff<R>(c, cnext), bp.x, bp.y, A, B);
        const T3<R> Fp = shfl_up3(F), Bp = shfl_up3(B), An = shfl_down3(A);
        if (lane >= 1 && lane <= kWarpOut && in && (!ch.act || ch.act[ch.rep[q]])) {
            // link (q-1, q) acts on q; link (q, q+1) reacts on q; bends centred
            // at q-1 (third bead), q (middle), q+1 (first bead); summed in double
            target_store(tgt, f, 3 * q,
                         double(Fp.x) - double(F.x) + double(Bp.x) + (double(A.x) - double(B.x)) - double(An.x),
                         double(Fp.y) - double(F.y) + double(Bp.y) + (double(A.y) - double(B.y)) - double(An.y),
                         double(Fp.z) - double(F.z) + double(Bp.z) + (double(A.z) - double(B.z)) - double(An.z));
        }
    }
}

// Energies. Each warp owns 32 consecutive positions and each lane the link
// and bend of its own position, at up to KMAX step sizes from one read of x
// and d (MOVE), or at x itself (a plain pass: one evaluation, copied to every
// requested slot). A fixed grid (grid-stride over warp tiles) keeps the
// per-block partial sums deterministic. The plain variant holds no trial
// state, which keeps it at four blocks per SM.
template <class R, int KMAX, bool MOVE>
__global__ void __launch_bounds__(kThreads, KMAX == 1 ? 4 : 2)
    k_chain_energy(const ChainDev ch, const double* __restrict__ x, const double* __restrict__ d,
                   const LambdaSet* __restrict__ lset, double* __restrict__ partial, int nblk_total, int blk_off,
                   const int4* __restrict__ table, int n_table) {
    __shared__ double sm[4 * 32];
    const int n = ch.n_pos;
    const int K = lset ? lset->K : 1;
    const int lane = threadIdx.x & 31;
    // grid-stride over all positions (one partial row per block), or (table)
    // the chunks [table.y, table.z) of one replica's positions, one row per
    // chunk, walked by a capped grid
    const int trips = table ? n_table : gridDim.x;
    for (int row = blockIdx.x; row < trips; row += (table ? gridDim.x : trips)) {
        int lo = 0, hi = n, w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, ws = (gridDim.x * blockDim.x) >> 5;
        if (table) {
            const int4 t = table[row];
            if (ch.act && !ch.act[t.x]) continue;  // replica not in this pass
            lo = t.y;
            hi = t.z;
            w0 = threadIdx.x >> 5;
            ws = blockDim.x >> 5;
        }
        double acc[KMAX][2];
    #pragma unroll
        for (int k = 0; k < KMAX; ++k) acc[k][0] = acc[k][1] = 0.0;
        for (int w = w0; lo + (long long)w * 32 < hi; w += ws) {
            const int q = lo + w * 32 + lane;
            const bool in = q < hi;
            const int qe = lane == 0 ? q - 1 : q + 1;
            const V3 c = pos_of(x, n, q), dc = MOVE ? pos_of(d, n, q) : V3{0.0, 0.0, 0.0};
            V3 ce{0.0, 0.0, 0.0}, de{0.0, 0.0, 0.0};
            if (lane == 0 || lane == 31) {
                ce = pos_of(x, n, qe);
                if (MOVE) de = pos_of(d, n, qe);
            }
            const unsigned char fl = in ? ch.flags[q] : 0;
            const double2 lp = in ? ch.link_p[q] : double2{0.0, 0.0};
            const double2 bp = in ? ch.bend_p[q] : double2{0.0, 0.0};
            V3 cp = shfl_up3(c), cn = shfl_down3(c);
            if (lane == 0) cp = ce;
            if (lane == 31) cn = ce;
            if (!MOVE) {
                if (fl & kLink) acc[0][0] += stretch_energy<R>(c, cn, lp.x, lp.y);
                if (fl & kBend) acc[0][1] += bend_energy<R>(diff<R>(cp, c), diff<R>(c, cn), bp.x, bp.y);
                continue;
            }
            V3 dp = shfl_up3(dc), dn = shfl_down3(dc);
            if (lane == 0) dp = de;
            if (lane == 31) dn = de;
            if (fl) {
    #pragma unroll
                for (int k = 0; k < KMAX; ++k) {
                    if (k >= K) break;
                    const double lam = lset ? lset->lam[k] : 0.0;
                    const V3 Pc = move3(c, lam, dc), Pn = move3(cn, lam, dn);
                    if (fl & kLink) acc[k][0] += stretch_energy<R>(Pc, Pn, lp.x, lp.y);
                    if (fl & kBend) {
                        const V3 Pp = move3(cp, lam, dp);
                        acc[k][1] += bend_energy<R>(diff<R>(Pp, Pc), diff<R>(Pc, Pn), bp.x, bp.y);
                    }
                }
            }
        }
    #pragma unroll
        for (int k = 0; k < KMAX; ++k) {
            if (k >= K) break;
            double e[2] = {acc[k][0], acc[k][1]};
            block_sum<2>(e, sm);
            if (threadIdx.x == 0) {
                // a plain pass writes its one evaluation to every requested slot
                for (int kk = k; kk < (MOVE ? k + 1 : K); ++kk) {
                    double* o = partial + ((size_t)kk * nblk_total + blk_off + row) * 4;
                    o[0] = e[0];
                    o[1] = e[1];
                    o[2] = 0.0;
                    o[3] = 0.0;
                }
            }
        }
        __syncthreads();  // smem of block_sum is reused by the next trip
    }
}

// Reordering between the caller's bead order and the internal one:
// internal position p holds external bead order[p].
__global__ void k_to_internal(int n3, const int* __restrict__ order, const double* __restrict__ ext,
                              double* __restrict__ in) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        const int p = i / 3, k = i - 3 * p;
        in[i] = ext[3 * order[p] + k];
    }
}

__global__ void k_to_external(int n3, const int* __restrict__ order, const double* __restrict__ in,
                              double* __restrict__ ext) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        const int p = i / 3, k = i - 3 * p;
        ext[3 * order[p] + k] = in[i];
    }
}

int reorder_blocks(int n3) {
    const int b = (n3 + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
}

}  // namespace

int chain_blocks(const ChainDev& ch) {
    // energy: one 32-position tile per warp, at most energy_blocks_per_sm
    // blocks per SM (4 by default)
    const int per_block = 32 * (kThreads / 32);
    const int b = (ch.n_pos + per_block - 1) / per_block;
    const int cap = 148 * (ch.energy_blocks_per_sm > 0 ? ch.energy_blocks_per_sm : 4);
    return b < 1 ? 1 : (b < cap ? b : cap);
}

void launch_chain_forces(const ChainDev& ch, int prec, const double* x, const ForceTarget& t, cudaStream_t s) {
    if (ch.n_pos <= 0) return;
    const int threads = ch.force_threads > 0 ? ch.force_threads : kThreads;
    const int per_block = kWarpOut * (threads / 32);
    int g = (ch.n_pos + per_block - 1) / per_block;
    if (ch.act && g > 2 * kBatchGridCap) g = 2 * kBatchGridCap;  // batched: the warp loop covers the rest
    if (prec == MEDYAN_PREC_MIXED)
        k_chain_forces<float><<<g, threads, 0, s>>>(ch, x, t);
    else
        k_chain_forces<double><<<g, threads, 0, s>>>(ch, x, t);
}

void launch_chain_energy(const ChainDev& ch, int prec, const double* x, const double* d, const LambdaSet* lam,
                         double* partial, int nblk_total, int blk_off, cudaStream_t s, const int4* table,
                         int table_blocks) {
    if (ch.n_pos <= 0) return;
    const int nrows = table ? table_blocks : chain_blocks(ch);
    if (nrows <= 0) return;
    const int g = table && nrows > kBatchGridCap ? kBatchGridCap : nrows;
    if (prec == MEDYAN_PREC_MIXED) {
        if (d) k_chain_energy<float, kMaxLambda, true><<<g, kThreads, 0, s>>>(ch, x, d, lam, partial, nblk_total, blk_off, table, nrows);
        else k_chain_energy<float, 1, false><<<g, kThreads, 0, s>>>(ch, x, d, lam, partial, nblk_total, blk_off, table, nrows);
    } else {
        if (d) k_chain_energy<double, kMaxLambda, true><<<g, kThreads, 0, s>>>(ch, x, d, lam, partial, nblk_total, blk_off, table, nrows);
        else k_chain_energy<double, 1, false><<<g, kThreads, 0, s>>>(ch, x, d, lam, partial, nblk_total, blk_off, table, nrows);
    }
}

void launch_to_internal(int n3, const int* order, const double* ext, double* in, cudaStream_t s) {
    if (n3 > 0) k_to_internal<<<reorder_blocks(n3), kThreads, 0, s>>>(n3, order, ext, in);
}

void launch_to_external(int n3, const int* order, const double* in, double* ext, cudaStream_t s) {
    if (n3 > 0) k_to_external<<<reorder_blocks(n3), kThreads, 0, s>>>(n3, order, in, ext);
}

// Internal order: walk the stretching links from every bead without a
// predecessor, in bead-index order; beads left unvisited lie on link cycles,
// which are entered at their smallest bead. order[p] = external bead.
void chain_order(const medyan_system* s, std::vector<int>& order) {
    const int nb = s->n_beads;
    std::vector<int> next(nb, -1), prev(nb, -1);
    for (int i = 0; i < s->n_stretch; ++i) {
        const int a = s->stretch_beads[2 * i] / 3, c = s->stretch_beads[2 * i + 1] / 3;
        if (a != c && next[a] < 0 && prev[c] < 0) {
            next[a] = c;
            prev[c] = a;
        }
    }
    std::vector<char> seen(nb, 0);
    order.clear();
    order.reserve(nb);
    auto walk = [&](int h) {
        for (int b = h; b >= 0 && !seen[b]; b = next[b]) {
            seen[b] = 1;
            order.push_back(b);
        }
    };
    for (int b = 0; b < nb; ++b)
        if (prev[b] < 0) walk(b);
    for (int b = 0; b < nb; ++b)
        if (!seen[b]) walk(b);
}

// Chains over a fixed internal order (pos = inverse of order). Bead offsets in
// s are external; the leftover lists index s's interactions.
void build_chains(const medyan_system* s, const std::vector<int>& pos, ChainHost& out) {
    const int n = s->n_beads;
    out.left_stretch.clear();
    out.left_bend.clear();
    out.flags.assign(n, 0);
    out.link_p.assign(n, make_double2(0, 0));
    out.bend_p.assign(n, make_double2(0, 0));
    for (int i = 0; i < s->n_stretch; ++i) {
        const int p = pos[s->stretch_beads[2 * i] / 3], q = pos[s->stretch_beads[2 * i + 1] / 3];
        if (q == p + 1 && !(out.flags[p] & kLink)) {
            out.flags[p] |= kLink;
            out.link_p[p] = make_double2(s->stretch_k[i], s->stretch_l0[i]);
        } else {
            out.left_stretch.push_back(i);
        }
    }
    for (int i = 0; i < s->n_bend; ++i) {
        const int p1 = pos[s->bend_beads[3 * i] / 3], p = pos[s->bend_beads[3 * i + 1] / 3],
                  p3 = pos[s->bend_beads[3 * i + 2] / 3];
        if (p1 == p - 1 && p3 == p + 1 && !(out.flags[p] & kBend)) {
            out.flags[p] |= kBend;
            out.bend_p[p] = make_double2(s->bend_k[i], s->bend_theta0[i]);
        } else {
            out.left_bend.push_back(i);
        }
    }
}

}  // namespace mb

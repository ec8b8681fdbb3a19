// excl_kernels.cu — cylinder excluded-volume energy/force kernels, the
// quadrature fallbacks, and the energy-pass finish kernel.
//
// Built with --fmad=false: the analytic excluded-volume formula cancels
// heavily for close or near-parallel cylinders, and rounding each operation
// as written keeps the FP64 path within a few ulps of the CPU reference.
//
// Pairs whose analytic energy is +-inf, NaN or < -1 (or whose forces are
// non-finite or > 1e15) go to a queue; a one-block kernel then evaluates the
// reference's composite Simpson quadrature for them
// (CylinderExclVolRepulsion::energyN/forceN, CylinderExclVolRepulsion.cpp:884-1256)
// with all threads of the block splitting the grid.
#include <mutex>

#include "internal.h"
#include "excl.cuh"
#include "quadrature.cuh"

namespace mb {

namespace {

constexpr int kMaxExclThreads = 128;  // largest tunable excluded-volume block

__device__ __forceinline__ V3 at(const V3& x, const V3& d, double lam, bool move) { return move ? move3(x, lam, d) : x; }

template <class R, bool MOVE>
__global__ void __launch_bounds__(kMaxExclThreads) k_excl_energy(const DeviceFF ff, const double* __restrict__ x,
                                                            const double* __restrict__ d,
                                                            const LambdaSet* __restrict__ lset,
                                                            double* __restrict__ partial, int nblk_total,
                                                            int blk_off, int* __restrict__ fb_count,
                                                            int2* __restrict__ fb_list, int fb_cap, int* __restrict__ bad,
                                                            int n_logical) {
    __shared__ double smem[4 * 32];
    for (int lb = blockIdx.x; lb < n_logical; lb += gridDim.x) {  // capped grid in batches
        if (ff.act && !ff.act[ff.rep_excl[lb]]) continue;  // batched: replica not in this pass
        const int i = lb * blockDim.x + threadIdx.x;
        const bool move = MOVE;
        bool valid = i < ff.n_excl;
        V3 X[4] = {}, D[4] = {};
        double krs = 0;
        int4 q = valid ? ff.excl_bs[i] : int4{-1, 0, 0, 0};
        valid = valid && q.x >= 0;  // -1: padding record
        if (valid) {
            krs = ff.excl_krs[i];
            X[0] = load3(x + q.x); X[1] = load3(x + q.y); X[2] = load3(x + q.z); X[3] = load3(x + q.w);
            if (move) { D[0] = load3(d + q.x); D[1] = load3(d + q.y); D[2] = load3(d + q.z); D[3] = load3(d + q.w); }
        }
        const int K = lset ? lset->K : 1;
    #pragma unroll
        for (int k = 0; k < kMaxLambda; ++k) {
            if (k >= K) break;
            const double lam = lset ? lset->lam[k] : 0.0;
            double e[1] = {0.0};
            if (valid) {
                double U = excl_energy<R>(at(X[0], D[0], lam, move), at(X[1], D[1], lam, move),
                                          at(X[2], D[2], lam, move), at(X[3], D[3], lam, move), krs);
                if (excl_energy_bad(U)) {
                    int slot = atomicAdd(fb_count, 1);
                    if (slot < fb_cap) fb_list[slot] = make_int2(i, k);
                    else atomicOr(bad + k, 2);
                    U = 0.0;
                }
                e[0] = U;
            }
            block_sum<1>(e, smem);
            if (threadIdx.x == 0) {
                double* o = partial + ((size_t)k * nblk_total + blk_off + lb) * 4;
                o[0] = e[0];
                o[1] = 0.0;
                o[2] = 0.0;
                o[3] = 0.0;
            }
        }
        __syncthreads();  // smem of block_sum is reused by the next trip
    }
}

__device__ __forceinline__ V3 pos_at(const double* __restrict__ x, const ForceTarget& t, double lam, int o) {
    V3 p = load3(x + o);
    return t.d ? move3(p, lam, load3(t.d + o)) : p;
}

template <bool EXACT>
__global__ void __launch_bounds__(kMaxExclThreads) k_excl_forces(const DeviceFF ff, const double* __restrict__ x,
                                                            const ForceTarget tgt, int* __restrict__ fb_count,
                                                            int* __restrict__ fb_list, int fb_cap, int* __restrict__ status,
                                                            int n_logical) {
    if (tgt.skip && *tgt.skip) return;
    for (int lb = blockIdx.x; lb < n_logical; lb += gridDim.x) {  // capped grid in batches
        if (ff.act && !ff.act[ff.rep_excl[lb]]) continue;  // batched: replica not in this pass
        const int i = lb * blockDim.x + threadIdx.x;
        if (i >= ff.n_excl) continue;
        double* __restrict__ f = target_force(tgt);
        const double lam = tgt.lam ? *tgt.lam : 0.0;
        int4 q = ff.excl_bs[i];
        if (q.x < 0) continue;  // padding record
        T3<double> fo[4];
        if (excl_force<EXACT>(pos_at(x, tgt, lam, q.x), pos_at(x, tgt, lam, q.y), pos_at(x, tgt, lam, q.z),
                          pos_at(x, tgt, lam, q.w), ff.excl_krs[i], fo)) {
            target_add(tgt, f, q.x, fo[0].x, fo[0].y, fo[0].z);
            target_add(tgt, f, q.y, fo[1].x, fo[1].y, fo[1].z);
            target_add(tgt, f, q.z, fo[2].x, fo[2].y, fo[2].z);
            target_add(tgt, f, q.w, fo[3].x, fo[3].y, fo[3].z);
        } else {
            int slot = atomicAdd(fb_count, 1);
            if (slot < fb_cap) fb_list[slot] = i;
            else atomicOr(status, 2);
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_excl_force_fallback(const DeviceFF ff, const double* __restrict__ x,
                                                                const ForceTarget tgt, int* __restrict__ fb_count,
                                                                const int* __restrict__ fb_list, int fb_cap,
                                                                int* __restrict__ status) {
    __shared__ double red[6 * 32];
    const int n = min(*fb_count, fb_cap);
    if (n == 0) return;
    double* __restrict__ f = target_force(tgt);
    const double lam = tgt.lam ? *tgt.lam : 0.0;
    for (int e = 0; e < n; ++e) {
        const int i = fb_list[e];
        const int4 q = ff.excl_bs[i];
        const V3 c1 = pos_at(x, tgt, lam, q.x), c2 = pos_at(x, tgt, lam, q.y), c3 = pos_at(x, tgt, lam, q.z),
                 c4 = pos_at(x, tgt, lam, q.w);
        double out[4][3];
        bool ok = forceN_block(c1, c2, c3, c4, ff.excl_krs[i], false, red, out);
        if (!ok) ok = forceN_block(c1, c2, c3, c4, ff.excl_krs[i], true, red, out);
        if (threadIdx.x == 0) {
            if (ok) {
                target_add(tgt, f, q.x, out[0][0], out[0][1], out[0][2]);
                target_add(tgt, f, q.y, out[1][0], out[1][1], out[1][2]);
                target_add(tgt, f, q.z, out[2][0], out[2][1], out[2][2]);
                target_add(tgt, f, q.w, out[3][0], out[3][1], out[3][2]);
            } else {
                atomicOr(status, 1);
            }
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) *fb_count = 0;
}

constexpr int kFinishThreads = 1024;
constexpr int kSplitFinishThreads = 256;

// Slot sums of one block's share [r_lo, r_hi) of the partial rows of the K
// step sizes (the rows of step size k start at base + k * stride): each
// thread adds its rows' columns into the slot their range belongs to (chain
// rows: slots 0 and 1; bonded segment s: slot s, or slots 4-7 for branching,
// slot 9 for the boundary; excluded-volume rows: slot 8), then the block
// reduces in a fixed tree. The rows of all K step sizes are loaded in one
// round (one round of loads and barriers per step size made a line-search
// pass's finish several L2 round trips longer); per step size the additions
// are those of a single one. Valid in thread 0 (out + k * out_stride).
__device__ void finish_rows(const DeviceFF& ff, const double* __restrict__ base, size_t stride, int K, int r_lo,
                            int r_hi, int nch, int nbb,
                            double* wsum /* [32][kMaxLambda][MEDYAN_FF_COUNT] */, double* out, size_t out_stride) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    int seg[7];
#pragma unroll
    for (int i = 0; i < 7; ++i) seg[i] = ff.seg[i];
    double acc[kMaxLambda][MEDYAN_FF_COUNT];
#pragma unroll
    for (int k = 0; k < kMaxLambda; ++k)
#pragma unroll
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) acc[k][i] = 0.0;
    for (int r = r_lo + threadIdx.x; r < r_hi; r += blockDim.x) {
        double2 lo[kMaxLambda], hi[kMaxLambda];
#pragma unroll
        for (int k = 0; k < kMaxLambda; ++k) {
            if (k < K) {
                const double2* row = reinterpret_cast<const double2*>(base + k * stride + (size_t)r * 4);
                lo[k] = __ldcg(row);
                hi[k] = __ldcg(row + 1);
            } else {
                lo[k] = hi[k] = double2{0.0, 0.0};
            }
        }
        int cls;  // 0 chain, 1-4 bonded segment 0-3, 5 branching, 6 boundary, 7 excluded volume
        if (r < nch) {
            cls = 0;
        } else {
            const int rb = r - nch;
            if (rb >= nbb) cls = 7;
            else if (rb < seg[4]) cls = 1 + (rb < seg[1] ? 0 : rb < seg[2] ? 1 : rb < seg[3] ? 2 : 3);
            else if (rb < seg[5]) cls = 5;
            else cls = 6;
        }
#pragma unroll
        for (int k = 0; k < kMaxLambda; ++k) {
            if (cls == 0) {
                acc[k][0] += lo[k].x;
                acc[k][1] += lo[k].y;
            } else if (cls <= 4) {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (i == cls - 1) acc[k][i] += lo[k].x;
            } else if (cls == 5) {
                acc[k][4] += lo[k].x;
                acc[k][5] += lo[k].y;
                acc[k][6] += hi[k].x;
                acc[k][7] += hi[k].y;
            } else if (cls == 6) {
                acc[k][9] += lo[k].x;
            } else {
                acc[k][MEDYAN_FF_EXCLUDED_VOLUME] += lo[k].x;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kMaxLambda; ++k) {
        if (k >= K) break;
#pragma unroll
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
            double v = acc[k][i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) wsum[(warp * kMaxLambda + k) * MEDYAN_FF_COUNT + i] = v;
        }
    }
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < K; ++k) {
#pragma unroll
            for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
                double v = lane < nwarp ? wsum[(lane * kMaxLambda + k) * MEDYAN_FF_COUNT + i] : 0.0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) out[k * out_stride + i] = v;
            }
        }
    }
    __syncthreads();
}

// Sums the per-block energy partials of each force field, evaluates the
// energyN fallback for queued pairs in (slot, pair) order, and applies
// ForceFieldManager::computeEnergy's rule (ForceFieldManager.cpp:137-176): a
// force field at or below -1 makes the total +inf.
//
// With stage/ticket the rows are split over gridDim.x blocks: block b sums
// its share into stage[k][b][slot], and the last block to arrive (ticket)
// adds the shares in block order and finishes. With one block and no stage
// the block does everything. Either way every sum is taken in a fixed order,
// so the result does not depend on scheduling.
__global__ void __launch_bounds__(kSplitFinishThreads) k_energy_finish(
    const DeviceFF ff, const double* __restrict__ x, const double* __restrict__ d, const LambdaSet* __restrict__ lset,
    const double* __restrict__ partial, int nch, int nbb, int nbe, int* __restrict__ fb_count,
    int2* __restrict__ fb_list, int fb_cap, int* __restrict__ bad, double* __restrict__ out,
    double* __restrict__ stage, unsigned int* __restrict__ ticket) {
    __shared__ double red[4 * 32];
    __shared__ double wsum[(kSplitFinishThreads / 32) * kMaxLambda * MEDYAN_FF_COUNT];
    __shared__ double sums[kMaxLambda][MEDYAN_FF_COUNT];
    __shared__ double fbE[kMaxLambda];
    __shared__ int nfb, n_queued, bad0[kMaxLambda];
    __shared__ bool last;
    const int K = lset ? lset->K : 1;
    const int total_blocks = nch + nbb + nbe;
    const int G = gridDim.x;
    const int chunk = (total_blocks + G - 1) / G;
    const int r_lo = min(total_blocks, (int)blockIdx.x * chunk), r_hi = min(total_blocks, r_lo + chunk);
    if (G > 1)
        finish_rows(ff, partial, (size_t)total_blocks * 4, K, r_lo, r_hi, nch, nbb, wsum,
                    stage + (size_t)blockIdx.x * MEDYAN_FF_COUNT, (size_t)G * MEDYAN_FF_COUNT);
    else
        finish_rows(ff, partial, (size_t)total_blocks * 4, K, r_lo, r_hi, nch, nbb, wsum, &sums[0][0],
                    MEDYAN_FF_COUNT);
    if (G > 1) {
        // last-block-done: this block's shares (thread 0's stores) are
        // published by thread 0's acquire-release ticket
        __syncthreads();
        if (threadIdx.x == 0) last = ticket_add(ticket, 1u) == (unsigned)G - 1;
        __syncthreads();
        if (!last) return;
        if (threadIdx.x < K * MEDYAN_FF_COUNT) {
            // the G shares loaded at once, added in block order
            const int k = threadIdx.x / MEDYAN_FF_COUNT, slot = threadIdx.x % MEDYAN_FF_COUNT;
            double sh[kFinishBlocks];
#pragma unroll
            for (int b = 0; b < kFinishBlocks; ++b)
                sh[b] = b < G ? __ldcg(stage + ((size_t)k * G + b) * MEDYAN_FF_COUNT + slot) : 0.0;
            double v = 0.0;
#pragma unroll
            for (int b = 0; b < kFinishBlocks; ++b)
                if (b < G) v += sh[b];
            sums[k][slot] = v;
        }
        if (threadIdx.x == 0) *ticket = 0u;
    }
    // the queue length and the status flags, fetched before they are needed
    if (threadIdx.x == 0) n_queued = *fb_count;
    if (threadIdx.x < kMaxLambda) bad0[threadIdx.x] = bad[threadIdx.x];
    __syncthreads();
    // queued fallback pairs: energyN in (slot, pair) order
    if (threadIdx.x == 0) {
        int n = min(n_queued, fb_cap);
        for (int a = 1; a < n; ++a) {
            int2 v = fb_list[a];
            int b = a - 1;
            while (b >= 0 && (fb_list[b].y > v.y || (fb_list[b].y == v.y && fb_list[b].x > v.x))) {
                fb_list[b + 1] = fb_list[b];
                --b;
            }
            fb_list[b + 1] = v;
        }
        nfb = n;
        for (int k = 0; k < kMaxLambda; ++k) fbE[k] = 0.0;
    }
    __syncthreads();
    for (int e = 0; e < nfb; ++e) {
        const int2 q = fb_list[e];
        const int4 bs = ff.excl_bs[q.x];
        const double lam = lset ? lset->lam[q.y] : 0.0;
        V3 P[4];
        const int offs[4] = {bs.x, bs.y, bs.z, bs.w};
        for (int j = 0; j < 4; ++j) {
            V3 X = load3(x + offs[j]);
            P[j] = d ? move3(X, lam, load3(d + offs[j])) : X;
        }
        double U = energyN_block(six_of(P[0], P[1], P[2], P[3]), ff.excl_krs[q.x], red);
        if (threadIdx.x == 0) {
            if (excl_energy_bad(U)) atomicOr(bad + q.y, 1);
            else fbE[q.y] += U;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k) {
            double* o = out + k * (MEDYAN_FF_COUNT + 1);
            double tot = 0.0;
            bool inf = false;
            for (int slot = 0; slot < MEDYAN_FF_COUNT; ++slot) {
                double v = sums[k][slot];
                if (slot == MEDYAN_FF_EXCLUDED_VOLUME) {
                    v += fbE[k];
                    // the fallbacks may have flagged a pair: read the flag again then
                    if (nfb > 0 ? bad[k] : bad0[k]) v = -1.0;
                }
                o[slot] = v;
                if (v <= -1) inf = true;
                else tot += v;
            }
            o[MEDYAN_FF_COUNT] = inf ? __longlong_as_double(0x7ff0000000000000ULL) : tot;
            bad[k] = 0;
        }
        *fb_count = 0;
    }
}

// Batched form: one block per replica. Replica r's partial rows are
// rows.chain[r..r+1) (chain), nch + rows.seg[s][r..r+1) (bonded segment s)
// and nch + nbb + rows.excl[r..r+1) (excluded volume); queued fallback pairs
// belong to r when their index is in excl_pairs[r..r+1). Writes
// out[(r * kMaxLambda + k) * (MEDYAN_FF_COUNT + 1) + slot]. The queue count
// and overflow flags are cleared by the caller after every block has read them.
__global__ void __launch_bounds__(kFinishThreads) k_energy_finish_batched(
    const DeviceFF ff, const double* __restrict__ x, const double* __restrict__ d, const LambdaSet* __restrict__ lset,
    const double* __restrict__ partial, int nch, int nbb, int nbe, const int* __restrict__ rows_chain,
    const int* __restrict__ rows_seg /* [6][R+1] */, const int* __restrict__ rows_excl,
    const int* __restrict__ excl_pairs, int R, const int* __restrict__ fb_count, const int2* __restrict__ fb_list,
    const int* __restrict__ bad, double* __restrict__ out) {
    __shared__ double red[4 * 32];
    __shared__ double sums[kMaxLambda][MEDYAN_FF_COUNT];
    __shared__ double fbE[kMaxLambda];
    __shared__ int fbBad[kMaxLambda];
    __shared__ int2 mine[kFallbackCap];
    __shared__ int nfb;
    for (int r = blockIdx.x; r < R; r += gridDim.x) {  // capped grid over the replicas
        if (ff.act && !ff.act[r]) continue;  // replica not in this pass
        const int K = lset ? lset->K : 1;
        const int total_blocks = nch + nbb + nbe;
        if (threadIdx.x == 0) {
            const int n = min(*fb_count, kFallbackCap);
            const int p0 = excl_pairs[r], p1 = excl_pairs[r + 1];
            int m = 0;
            for (int a = 0; a < n; ++a) {
                const int2 v = fb_list[a];
                if (v.x >= p0 && v.x < p1) mine[m++] = v;
            }
            // deterministic order: by slot, then pair
            for (int a = 1; a < m; ++a) {
                int2 v = mine[a];
                int b = a - 1;
                while (b >= 0 && (mine[b].y > v.y || (mine[b].y == v.y && mine[b].x > v.x))) {
                    mine[b + 1] = mine[b];
                    --b;
                }
                mine[b + 1] = v;
            }
            nfb = m;
            for (int k = 0; k < kMaxLambda; ++k) {
                fbE[k] = 0.0;
                fbBad[k] = bad[k];  // queue overflow marks every replica
            }
        }
        __syncthreads();
        for (int e = 0; e < nfb; ++e) {
            const int2 q = mine[e];
            const int4 bs = ff.excl_bs[q.x];
            const double lam = lset ? lset->lam[q.y] : 0.0;
            V3 P[4];
            const int offs[4] = {bs.x, bs.y, bs.z, bs.w};
            for (int j = 0; j < 4; ++j) {
                V3 X = load3(x + offs[j]);
                P[j] = d ? move3(X, lam, load3(d + offs[j])) : X;
            }
            double U = energyN_block(six_of(P[0], P[1], P[2], P[3]), ff.excl_krs[q.x], red);
            if (threadIdx.x == 0) {
                if (excl_energy_bad(U)) fbBad[q.y] |= 1;
                else fbE[q.y] += U;
            }
            __syncthreads();
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
        auto range_sum = [&](const double* base, int b0, int b1, int j) {
            double acc = 0.0;
            int b = b0 + lane;
            for (; b + 32 * 7 < b1; b += 32 * 8) {
                double v[8];
    #pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = __ldcg(base + (size_t)(b + 32 * u) * 4 + j);
    #pragma unroll
                for (int u = 0; u < 8; ++u) acc += v[u];
            }
            for (; b < b1; b += 32) acc += __ldcg(base + (size_t)b * 4 + j);
            return acc;
        };
        const int R1 = R + 1;
        for (int combo = warp; combo < K * MEDYAN_FF_COUNT; combo += nwarp) {
            const int k = combo / MEDYAN_FF_COUNT, slot = combo % MEDYAN_FF_COUNT;
            int seg = -1, j = 0, cj = -1;
            switch (slot) {
                case 0: seg = 0; cj = 0; break;
                case 1: seg = 1; cj = 1; break;
                case 2: seg = 2; break;
                case 3: seg = 3; break;
                case 4: case 5: case 6: case 7: seg = 4; j = slot - 4; break;
                case 8: break;
                default: seg = 5; break;
            }
            const double* base = partial + (size_t)k * total_blocks * 4;
            double sv;
            if (slot == 8) {
                sv = range_sum(base, nch + nbb + rows_excl[r], nch + nbb + rows_excl[r + 1], 0);
            } else {
                sv = range_sum(base, nch + rows_seg[seg * R1 + r], nch + rows_seg[seg * R1 + r + 1], j);
                if (cj >= 0) sv += range_sum(base, rows_chain[r], rows_chain[r + 1], cj);
            }
    #pragma unroll
            for (int o = 16; o > 0; o >>= 1) sv += __shfl_down_sync(0xffffffffu, sv, o);
            if (lane == 0) sums[k][slot] = sv;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < K; ++k) {
                double* o = out + ((size_t)r * kMaxLambda + k) * (MEDYAN_FF_COUNT + 1);
                double tot = 0.0;
                bool inf = false;
                for (int slot = 0; slot < MEDYAN_FF_COUNT; ++slot) {
                    double v = sums[k][slot];
                    if (slot == MEDYAN_FF_EXCLUDED_VOLUME) {
                        v += fbE[k];
                        if (fbBad[k]) v = -1.0;
                    }
                    o[slot] = v;
                    if (v <= -1) inf = true;
                    else tot += v;
                }
                o[MEDYAN_FF_COUNT] = inf ? __longlong_as_double(0x7ff0000000000000ULL) : tot;
            }
        }
        __syncthreads();  // shared state is reused by the next replica
    }
}

}  // namespace

void launch_excl_energy(const DeviceFF& ff, int prec, const double* x, const double* d, const LambdaSet* lam,
                        const EnergyScratch& es, cudaStream_t s) {
    const int nbe = es.n_blocks_excl;
    if (nbe <= 0) return;
    const int total = es.total();
    // FP64 in both precision modes: the analytic integral (differences of
    // arctangents, JJ = -(triple product)^2) loses ~1e-6 relative in float.
    (void)prec;
    const int g = logical_grid(ff, nbe), off = es.n_blocks_chain + es.n_blocks_bonded;
    if (d)
        k_excl_energy<double, true><<<g, excl_block_of(ff), 0, s>>>(ff, x, d, lam, es.partial, total, off, es.fb_count,
                                                                   es.fb_list, fb_capacity(es.fb_cap), es.bad, nbe);
    else
        k_excl_energy<double, false><<<g, excl_block_of(ff), 0, s>>>(ff, x, d, lam, es.partial, total, off,
                                                                    es.fb_count, es.fb_list, fb_capacity(es.fb_cap),
                                                                    es.bad, nbe);
}

void launch_excl_energy_fallback_and_finish(const DeviceFF& ff, const double* x, const double* d,
                                            const LambdaSet* lam, const EnergyScratch& es, cudaStream_t s) {
    const int g = es.stage && es.ticket ? kFinishBlocks : 1;
    k_energy_finish<<<g, kSplitFinishThreads, 0, s>>>(ff, x, d, lam, es.partial, es.n_blocks_chain,
                                                      es.n_blocks_bonded, es.n_blocks_excl, es.fb_count, es.fb_list,
                                                      fb_capacity(es.fb_cap), es.bad, es.out, es.stage, es.ticket);
}

void launch_excl_forces(const DeviceFF& ff, int prec, const double* x, const ForceTarget& t, const ForceScratch& fs,
                        cudaStream_t s) {
    const int nbe = excl_blocks(ff);
    if (nbe <= 0) return;
    // FP64 arithmetic in both modes, as for the energy; the FP64 mode keeps
    // the reference's expression order
    if (prec == MEDYAN_PREC_FP64)
        k_excl_forces<true><<<logical_grid(ff, nbe), excl_block_of(ff), 0, s>>>(ff, x, t, fs.fb_count, fs.fb_list,
                                                                             fb_capacity(fs.fb_cap), fs.status, nbe);
    else
        k_excl_forces<false><<<logical_grid(ff, nbe), excl_block_of(ff), 0, s>>>(ff, x, t, fs.fb_count, fs.fb_list,
                                                                              fb_capacity(fs.fb_cap), fs.status, nbe);
    k_excl_force_fallback<<<1, kBlock, 0, s>>>(ff, x, t, fs.fb_count, fs.fb_list, fb_capacity(fs.fb_cap), fs.status);
}

void launch_energy_finish_batched(const DeviceFF& ff, const double* x, const double* d, const LambdaSet* lam,
                                  const EnergyScratch& es, const int* rows_chain, const int* rows_seg,
                                  const int* rows_excl, const int* excl_pairs, int R, double* out, cudaStream_t s) {
    if (R <= 0) return;
    k_energy_finish_batched<<<R < 148 ? R : 148, kFinishThreads, 0, s>>>(ff, x, d, lam, es.partial, es.n_blocks_chain,
                                                         es.n_blocks_bonded, es.n_blocks_excl, rows_chain, rows_seg,
                                                         rows_excl, excl_pairs, R, es.fb_count, es.fb_list, es.bad,
                                                         out);
}

cudaError_t init_excl_kernels() {
    static std::mutex mu;
    static bool filled[64];
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (filled[dev]) return cudaSuccess;
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

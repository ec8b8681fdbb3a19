// internal.h — device-side data layout and launch entry points shared by the
// library's translation units. Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "medyan_b200.h"
#include "device_math.cuh"

namespace mb {

constexpr int kMaxLambda = 4;   // step sizes evaluated per line-search energy pass
constexpr int kBlock = 256;     // threads per block for interaction kernels
constexpr int kFallbackCap = 256;

// Vectorized force fields in device memory. Interaction records are packed so
// each thread issues 16- or 32-byte loads: bead sets as int2/int4 coordinate
// offsets (3*bead), parameters as double2/double4.
struct DeviceFF {
    int n_beads;
    int n_stretch, n_bend, n_linker, n_motor, n_branch, n_excl, n_boundary, n_planes;
    int branch_mask;
    const int2* stretch_bs;    const double2* stretch_p;   // (k, l0)
    const int4* bend_bs;       const double2* bend_p;      // beads x,y,z (w unused); (k, theta0)
    const int4* linker_bs;     const double4* linker_p;    // (k, l0, pos1, pos2)
    const int4* motor_bs;      const double4* motor_p;
    const int4* branch_bs;     const double4* branch_pa;   // (pos, stretch k, stretch l0, bend k)
    const double4* branch_pb;                              // (bend theta0, dihedral k, position k, 0)
    const int4* excl_bs;       const double* excl_krs;     // krep*L1*L2 per pair
    const int* boundary_bs;    const double2* boundary_p;  // (k, screening length)
    const int* boundary_plane; const double4* planes;      // plane index per term; a, b, c, d
    // Block ranges of the bonded kernel: [seg[s], seg[s+1]) for
    // stretch, bend, linker, motor, branch, boundary.
    int seg[7];
    // batched layouts only (null otherwise): act[r] != 0 when replica r takes
    // part in the current pass; the replica of each bonded / excluded-volume
    // block. Blocks of inactive replicas do nothing.
    const int* act;
    const int* rep_bonded;
    const int* rep_excl;
    // launch shapes (0: the defaults kBlock / kExclBlock): interaction
    // records (= threads) per block of the bonded and excluded-volume kernels
    int bonded_block;
    int excl_block;
};

// Filament chains (chain.cu) over the internal bead order: chain position p
// is internal bead p (coordinate offset 3p).
struct ChainDev {
    int n_pos;                   // = n_beads
    const unsigned char* flags;  // bit 0: link (p, p+1); bit 1: bend centred at p
    const double2* link_p;       // (k, l0) of link (p, p+1)
    const double2* bend_p;       // (k, theta0) of the bend centred at p
    // batched layouts only (null otherwise): replica of each position and the
    // pass's active mask; positions of inactive replicas are not written
    const int* rep;
    const int* act;
    // launch shapes (0: defaults): threads per block of the force kernel,
    // blocks per SM of the energy kernel's fixed grid
    int force_threads;
    int energy_blocks_per_sm;
};

struct ChainHost {
    std::vector<unsigned char> flags;
    std::vector<double2> link_p, bend_p;
    std::vector<int> left_stretch, left_bend;  // interactions kept on the generic path
};

// Step sizes for one energy pass: positions are x + lam[k]*d.
struct LambdaSet {
    int K;
    int pad;
    double lam[kMaxLambda];
};

// Energy pass scratch: per-block partial sums and the quadrature fallback queue.
struct EnergyScratch {
    double* partial;      // [kMaxLambda][n_blocks_total][4]: chain rows, bonded rows, excluded-volume rows
    int* fb_count;        // excluded-volume pairs needing energyN
    int2* fb_list;        // (pair, lambda slot)
    int fb_cap;           // entries of fb_list (0: kFallbackCap)
    int* bad;             // per lambda slot: fallback failed / queue overflow
    double* out;          // [kMaxLambda][MEDYAN_FF_COUNT + 1]: per FF, then total
    // split finish (null: one block does it all): per-block slot sums
    // [kMaxLambda][kFinishBlocks][MEDYAN_FF_COUNT] and the arrival ticket
    // (zero between passes; the last block resets it)
    double* stage;
    unsigned int* ticket;
    int n_blocks_chain;
    int n_blocks_bonded;
    int n_blocks_excl;
    int total() const { return n_blocks_chain + n_blocks_bonded + n_blocks_excl; }
};

// Where a force pass writes and at which positions it evaluates. The
// standalone path uses f0 at x. The minimizer passes both force buffers and
// a device-side parity (the new force goes to the buffer not holding the
// current one), a skip flag, and a move x + (*lam)*d evaluated on the fly.
//
// fixed = 1 (deterministic mode): every contribution is rounded to a 64-bit
// integer count of kFixedUnit pN and summed with integer additions, which
// give the same bits in any order; the pass ends with a conversion of the
// sums back to double in place (launch_fixed_to_double). A contribution of
// kFixedRange pN or more is out of the format's range: it sets bit 2 of
// *status and is dropped.
struct ForceTarget {
    double* f0;
    double* f1;
    const int* parity;   // nullable: write f0
    const int* skip;     // nullable: nonzero -> the pass does nothing
    const double* d;     // nullable: positions are x
    const double* lam;   // step along d
    int fixed;           // 1: deterministic fixed-point accumulation
    int* status;         // fixed mode: range flag (bit 2)
};

constexpr double kFixedScale = 4294967296.0;  // counts per pN (2^32: 2.3e-10 pN resolution)
constexpr double kFixedRange = 16777216.0;    // |contribution| < 2^24 pN: sums of up to 2^7 such fit in 63 bits

__device__ __forceinline__ double* target_force(const ForceTarget& t) {
    return t.parity ? (*t.parity ? t.f0 : t.f1) : t.f0;
}

// v as a fixed-point count (0 and the range flag when out of range).
__device__ __forceinline__ long long fixed_of(double v, int* status) {
    if (!(fabs(v) < kFixedRange)) {
        if (status) atomicOr(status, 4);
        return 0;
    }
    return __double2ll_rn(v * kFixedScale);
}

__device__ __forceinline__ void red_add_fixed(double* p, long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Adds a bead's force contribution to the target's buffer f.
template <class R>
__device__ __forceinline__ void target_add(const ForceTarget& t, double* __restrict__ f, int off, R fx, R fy, R fz) {
    if (t.fixed) {
        red_add_fixed(f + off, fixed_of(double(fx), t.status));
        red_add_fixed(f + off + 1, fixed_of(double(fy), t.status));
        red_add_fixed(f + off + 2, fixed_of(double(fz), t.status));
    } else {
        add_force(f, off, fx, fy, fz);
    }
}

// Stores a bead's whole force (the chain pass, which writes before any
// addition).
__device__ __forceinline__ void target_store(const ForceTarget& t, double* __restrict__ f, int off, double fx, double fy,
                                             double fz) {
    if (t.fixed) {
        f[off] = __longlong_as_double(fixed_of(fx, t.status));
        f[off + 1] = __longlong_as_double(fixed_of(fy, t.status));
        f[off + 2] = __longlong_as_double(fixed_of(fz, t.status));
    } else {
        f[off] = fx;
        f[off + 1] = fy;
        f[off + 2] = fz;
    }
}

struct ForceScratch {
    int* fb_count;        // excluded-volume pairs needing forceN
    int* fb_list;
    int* status;          // bit 0: fallback failed, bit 1: queue overflow
    int fb_cap;           // entries of fb_list (0: kFallbackCap)
};

// The capacity of a fallback queue (fb_cap, or kFallbackCap when unset).
__host__ __device__ __forceinline__ int fb_capacity(int fb_cap) { return fb_cap > 0 ? fb_cap : kFallbackCap; }

// Two side streams and their events. A pass launched with a Fork runs its
// independent kernels on separate streams joined back into the caller's
// stream; under stream capture the fork and join become graph edges, so the
// kernels are parallel branches of the graph.
constexpr int kForkWays = 8;
struct Fork {
    cudaStream_t side[kForkWays];
    cudaEvent_t fork, join[kForkWays];
    cudaEvent_t mid;  // a point inside a pass that later branches wait for
};

// Launchers (ff_kernels.cu / excl_kernels.cu / chain.cu). prec: MEDYAN_PREC_*.
// The chain pass writes every bead's force first; the other passes add.
// fk may be null (everything on s, in order).
void launch_energy(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const double* d,
                   const LambdaSet* lam, const EnergyScratch& es, cudaStream_t s, const Fork* fk = nullptr);
void launch_forces(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const ForceTarget& t,
                   const ForceScratch& fs, cudaStream_t s, const Fork* fk = nullptr);
// Energy (at x, or x + lam_k d for the step sizes of lam when d is set) and
// forces (where t says) in one pass: the energy producers and the force
// kernels run side by side (with fk), the energy finish after its producers.
void launch_evaluate(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const double* d,
                     const LambdaSet* lam,
                     const ForceTarget& t, const EnergyScratch& es, const ForceScratch& fs, cudaStream_t s,
                     const Fork* fk);
void launch_chain_forces(const ChainDev& ch, int prec, const double* x, const ForceTarget& t, cudaStream_t s);
// Deterministic mode: the target's fixed-point sums back to double, in place
// (nothing when t.fixed is 0).
void launch_fixed_to_double(const ForceTarget& t, int n3, cudaStream_t s, const int* rep = nullptr,
                            const int* act = nullptr);
// table (optional): block b evaluates positions [table[b].y, table[b].z) of one
// replica (batched layouts), table_blocks blocks; else a grid-stride pass.
void launch_chain_energy(const ChainDev& ch, int prec, const double* x, const double* d, const LambdaSet* lam,
                         double* partial, int nblk_total, int blk_off, cudaStream_t s,
                         const int4* table = nullptr, int table_blocks = 0);
int chain_blocks(const ChainDev& ch);
void chain_order(const medyan_system* s, std::vector<int>& order);
void build_chains(const medyan_system* s, const std::vector<int>& pos, ChainHost& out);
// coordinate-layout conversion: internal position p <-> external bead order[p]
void launch_to_internal(int n3, const int* order, const double* ext, double* in, cudaStream_t s);
void launch_to_external(int n3, const int* order, const double* in, double* ext, cudaStream_t s);

void launch_excl_energy(const DeviceFF& ff, int prec, const double* x, const double* d, const LambdaSet* lam,
                        const EnergyScratch& es, cudaStream_t s);
void launch_excl_forces(const DeviceFF& ff, int prec, const double* x, const ForceTarget& t, const ForceScratch& fs,
                        cudaStream_t s);
void launch_excl_energy_fallback_and_finish(const DeviceFF& ff, const double* x, const double* d,
                                            const LambdaSet* lam, const EnergyScratch& es, cudaStream_t s);

// One-time per-device kernel attributes (forceN's 80 KB abscissa table).
// Batched energy finish (one block per replica); see excl_kernels.cu.
void launch_energy_finish_batched(const DeviceFF& ff, const double* x, const double* d, const LambdaSet* lam,
                                  const EnergyScratch& es, const int* rows_chain, const int* rows_seg,
                                  const int* rows_excl, const int* excl_pairs, int R, double* out, cudaStream_t s);
// Energy producers only (chain, bonded groups, excluded volume), no finish.
void launch_energy_producers(const ChainDev& ch, const DeviceFF& ff, const double* x, const double* d,
                             const LambdaSet* lam, const EnergyScratch& es, cudaStream_t s, const Fork* fk,
                             const int4* chain_table, int chain_table_blocks);

// Fills the quadrature grids of the excluded-volume fallbacks, once per
// device (the current one); call before any stream capture.
cudaError_t init_excl_kernels();

int bonded_blocks(const DeviceFF& ff);
constexpr int kFinishBlocks = 8;  // blocks of the split energy finish
constexpr int kExclBlock = 64;  // small blocks: the pair count is low and each pair is heavy
inline int excl_block_of(const DeviceFF& ff) { return ff.excl_block > 0 ? ff.excl_block : kExclBlock; }
inline int bonded_block_of(const DeviceFF& ff) { return ff.bonded_block > 0 ? ff.bonded_block : kBlock; }
inline int excl_blocks(const DeviceFF& ff) { return (ff.n_excl + excl_block_of(ff) - 1) / excl_block_of(ff); }
constexpr int kMaxShapeThreads = 512;  // largest block any tunable kernel is launched with
// Grid of a kernel over n logical blocks: one block each for a single
// network; for a batched layout (ff.act set) a capped grid that loops over
// them, so blocks of replicas outside the pass are skipped in a loop trip
// instead of being scheduled (the tail of a batch, where few replicas are
// still minimizing, is launch-bound).
constexpr int kBatchGridCap = 148 * 4;
inline int logical_grid(const DeviceFF& ff, int n) { return ff.act && n > kBatchGridCap ? kBatchGridCap : n; }

}  // namespace mb

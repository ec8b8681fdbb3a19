// pass.h — fused single-network passes (pass.cu): launch geometry, scratch
// and the argument block the pass kernels share.
#pragma once

#include "internal.h"

namespace mb {

// Device scratch of the fused passes, owned by the handle: one energy row per
// block of the pass's kernels and one per group of kPassGroup rows, a ticket
// per group and the pass ticket (all tickets zero between passes; the blocks
// that complete them reset them).
constexpr int kPassGroup = 32;
struct PassScratch {
    double* rows;             // [MEDYAN_FF_COUNT][rows], slot-major
    double* group_rows;       // [MEDYAN_FF_COUNT][groups]
    unsigned* group_ticket;   // [groups]
    unsigned* ticket;
};

constexpr int kPassThreads = 256;  // threads per block of the main and branch kernels

// Blocks and threads of one fused pass over a network.
struct PassGeometry {
    int threads;        // threads per block of the main and branch kernels (= records per bonded block)
    int seg[6];         // first bonded block of leftover stretch, leftover bend, linker, motor, boundary; end
    int excl_threads;   // pairs per excluded-volume block
    int nch;            // chain blocks of the main kernel (threads/32 warp tiles of 30 beads each)
    int nb_main;        // bonded blocks of the main kernel (segments 0-3 and 5)
    int main_blocks, branch_blocks, excl_blocks;
    int nch_forces;     // chain units of a force-only pass (kTilesPerWarp tiles per warp)
    int main_blocks_forces;  // main kernel grid of a force-only pass: one unit per block
    int rows;           // energy rows = blocks of all the pass's kernels
    int groups;         // rows / kPassGroup, rounded up
    // streamed chain (pass layout 2): the chain segments run in their own
    // kernel (k_pass_chain) and the main kernel keeps the generic records
    bool stream;
    int nseg;           // chain segments of kChainSeg positions
    int chain_blocks;   // grid of the chain kernel (0 without streaming)
    int chain_stages;   // segments in flight per chain block
};

// Streamed chain segments: kChainSeg positions per segment (one 30-position
// warp tile per consumer warp; even, so every segment's coordinate window
// starts on a 16-byte boundary), kChainStages segments in flight per block;
// blocks of kChainThreads consumer threads and one producer warp.
constexpr int kChainThreads = 256;
constexpr int kChainSeg = (kChainThreads / 32) * 30;
constexpr int kChainStages = 4;

struct PassArgs {
    ChainDev ch;
    DeviceFF ff;
    const double* x;
    ForceTarget t;            // force target and the positions (x, or x + (*lam) d) of both outputs
    double* rows;
    double* group_rows;
    unsigned* group_ticket;
    unsigned* ticket;
    int n_rows, n_groups, row_main, row_branch, row_excl, row_chain;
    int nch, nb_main;         // chain units (of this pass's kind), bonded chunks
    int chain_stages;         // PassGeometry::chain_stages
    int seg[6];               // PassGeometry::seg
    double* out;              // [kMaxLambda][MEDYAN_FF_COUNT + 1] energies
    const LambdaSet* lam_set; // result copied to slots [0, K) (null: slot 0)
    int* e_fb_count;
    int2* e_fb_list;
    int e_fb_cap, f_fb_cap;   // entries of the fallback queues
    int* e_bad;
    int* f_fb_count;
    int* f_fb_list;
    int* f_status;
};

// stream: the chain segments in their own kernel (pass layout 2)
PassGeometry pass_geometry(const ChainDev& ch, const DeviceFF& ff, bool stream);

// Energy (energy = true) and/or forces (t set) of a single network's force
// fields at t's positions (x when t is null or t->d is null). The energy lands
// in es.out; the forces in target_force(*t), overwritten. Single networks
// only (ff.act == null). Energies and forces are separate sets of kernels
// with their own tickets (ps, ps_forces); with fk all of them run on parallel
// branches. stream: the chain segments are staged through shared memory by
// bulk copies in their own kernel (pass layout 2).
void launch_pass_fused(const ChainDev& ch, const DeviceFF& ff, int prec, const double* x, const ForceTarget* t,
                       bool energy, const LambdaSet* lam_set, const EnergyScratch& es, const ForceScratch& fs,
                       const PassScratch& ps, const PassScratch& ps_forces, cudaStream_t s, const Fork* fk,
                       bool stream);

// Fills pass.cu's quadrature grids, once per device (the current one); call
// before any stream capture.
cudaError_t init_pass_kernels();

}  // namespace mb

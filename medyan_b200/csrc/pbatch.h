// pbatch.h — the packed layout of a batch of independent networks.
//
// All replicas' beads, chains and interaction records are concatenated into
// one set of device arrays, so every force and energy kernel runs once per
// pass for the whole batch. Each replica's records of a force field are
// padded to whole blocks (padding records carry bead offset -1 and are
// skipped), so every block of the energy kernels belongs to one replica and
// its partial sums are that replica's. The conjugate-gradient state, the
// line-search step sizes and the reductions of the vector passes are per
// replica (cg.cu, batched kernels).
#pragma once

#include <vector>

#include "handle.h"

namespace mb {

struct PackedBatch {
    int R = 0;                        // replicas
    int nb = 0;                       // packed beads
    std::vector<int> base;            // bead base of each replica (R + 1)
    DevBuf<int> base_dev;             // the same on the device
    long long gen = -1;               // sum of the replicas' ff_gen at packing

    // records (internal bead order of each replica, offsets shifted by 3 * base)
    DevBuf<unsigned char> flags;
    DevBuf<double2> link_p, bend_p;
    DevBuf<int2> stretch_bs;
    DevBuf<double2> stretch_p;
    DevBuf<int4> bend_bs;
    DevBuf<double2> bend_pp;
    DevBuf<int4> linker_bs, motor_bs, branch_bs, excl_bs;
    DevBuf<double4> linker_p, motor_p, branch_pa, branch_pb, planes;
    DevBuf<double> excl_krs;
    DevBuf<int> boundary_bs, boundary_plane;
    DevBuf<double2> boundary_p;
    DeviceFF ff{};
    ChainDev ch{};
    // launch shapes of the packed layout (medyan_batch_set_shapes): records
    // per bonded block and pairs per excluded-volume block (each replica's
    // records are padded to whole blocks), chain force threads per block,
    // positions per chain energy block
    int bonded_block = kBlock, excl_block = kExclBlock, chain_threads = 256, chain_chunk = 256;
    bool repack = false;  // shapes changed since the last packing

    // per-replica block and row tables
    DevBuf<int4> chain_table;         // chain energy block -> (replica, first, end position)
    int n_chain_blocks = 0;
    DevBuf<int> rows;                 // chain[R+1] | seg[6][R+1] | excl[R+1] | excl pairs[R+1]
    DevBuf<int> rep_bead, rep_bonded, rep_excl;  // replica of each position / bonded block / excl block
    DevBuf<int> act;                  // replicas taking part in the current pass

    // energy / force scratch
    EnergyScratch es{};
    ForceScratch fs{};
    DevBuf<double> partial;
    DevBuf<int> e_fb_count, e_bad, f_fb_count, f_fb_list, force_status;
    DevBuf<int2> e_fb_list;

    // conjugate gradient
    DevBuf<double> x, d, dS, fcur, fnew, minE, out, eout, one;
    DevBuf<CGState> st;
    DevBuf<LambdaSet> Lr, Lg, Lzero;
    DevBuf<double> lam0;
    DevBuf<int> off;
    cudaGraphExec_t graph = nullptr;
    int graph_prec = -1;
    long long graph_gen = -1;
    // fixed-point force sums (medyan_batch_set_deterministic); the graph
    // is rebuilt when it changes
    bool deterministic = false;
    bool graph_det = false;

    cudaStream_t stream = nullptr;
    Fork fork{};

    const int* rows_chain() const { return rows.raw(); }
    const int* rows_seg() const { return rows.raw() + (R + 1); }
    const int* rows_excl() const { return rows.raw() + 7 * (R + 1); }
    const int* excl_pairs() const { return rows.raw() + 8 * (R + 1); }

    ~PackedBatch();
};

// Builds (or rebuilds) the packed arrays from the replicas' handles.
medyan_status pack_batch(PackedBatch& pb, const std::vector<medyan_mech*>& h);
// Runs one batched minimization on the packed arrays (coordinates already in
// pb.x); results stay on the device (pb.x, pb.fcur, pb.st, pb.eout).
medyan_status cg_batch_run(PackedBatch& pb, int prec, const medyan_cg_params* p);
// Mean time (ms) of one packed evaluate (energy and forces of every replica
// at pb.x) after two warm-up passes; for the autotuner.
medyan_status cg_batch_time_evaluate(PackedBatch& pb, int prec, int reps, float* ms);

}  // namespace mb

// tune.cu — launch shapes per potential and the autotuner.
//
// The tunable shapes are the records (threads) per block of the bonded and
// excluded-volume kernels, the threads per block of the chain force kernel,
// the fixed grid of the chain energy kernel, and the pass layout (fused
// kernels or one kernel per potential group). The autotuner times the
// handle's evaluate pass (energy and forces, one CUDA graph) for each
// candidate of one field at a time, keeps the fastest, and moves to the next
// field (coordinate descent from the current shapes).
#include <cstring>

#include "handle.h"

using namespace mb;

namespace {

constexpr int kNone = -1;
bool allowed(int v, const int (&set)[3]) { return v != kNone && (v == set[0] || v == set[1] || v == set[2]); }
constexpr int kBonded[3] = {128, 256, 512};
constexpr int kExcl[3] = {32, 64, 128};
constexpr int kChain[3] = {128, 256, 512};
constexpr int kEnergyBps[3] = {2, 4, 8};
constexpr int kLayout[3] = {0, 1, 2};

medyan_launch_shapes current(const medyan_mech* h) {
    medyan_launch_shapes s{};
    s.bonded_threads = bonded_block_of(h->ff);
    s.excl_threads = excl_block_of(h->ff);
    s.chain_threads = h->chain.force_threads > 0 ? h->chain.force_threads : 256;
    s.chain_energy_blocks_per_sm = h->chain.energy_blocks_per_sm > 0 ? h->chain.energy_blocks_per_sm : 4;
    s.pass_layout = h->pass_layout;
    return s;
}

// Mean time of one evaluate pass (ms) after two warm-up passes.
medyan_status time_evaluate(medyan_mech* h, int reps, float* ms) {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = launch_pass(h, kPassBoth);
    if (e == cudaSuccess) e = cudaEventRecord(a, h->stream);
    for (int i = 0; i < reps && e == cudaSuccess; ++i) e = launch_pass(h, kPassBoth);
    if (e == cudaSuccess) e = cudaEventRecord(b, h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float t = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    // a failed force fallback during tuning is not the caller's concern
    if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.raw(), 0, sizeof(int), h->stream);
    if (e != cudaSuccess) return cuda_status(e);
    *ms = t / (float)reps;
    return MEDYAN_OK;
}

}  // namespace

extern "C" {

medyan_status medyan_mech_set_shapes(medyan_mech* h, const medyan_launch_shapes* s) {
    if (!h || !s) return MEDYAN_ERR_INVALID_ARG;
    if (!allowed(s->bonded_threads, kBonded) || !allowed(s->excl_threads, kExcl) ||
        !allowed(s->chain_threads, kChain) || !allowed(s->chain_energy_blocks_per_sm, kEnergyBps) ||
        !allowed(s->pass_layout, kLayout))
        return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);  // no pass may still read the old tables
    if (e != cudaSuccess) return cuda_status(e);
    h->ff.bonded_block = s->bonded_threads;
    h->ff.excl_block = s->excl_threads;
    h->chain.force_threads = s->chain_threads;
    h->chain.energy_blocks_per_sm = s->chain_energy_blocks_per_sm;
    h->pass_layout = s->pass_layout;
    return refresh_device_ff(h);
}

medyan_status medyan_mech_get_shapes(medyan_mech* h, medyan_launch_shapes* s) {
    if (!h || !s) return MEDYAN_ERR_INVALID_ARG;
    *s = current(h);
    return MEDYAN_OK;
}

medyan_status medyan_mech_autotune(medyan_mech* h, int32_t reps, medyan_launch_shapes* chosen) {
    if (!h || reps <= 0) return MEDYAN_ERR_INVALID_ARG;
    medyan_launch_shapes best = current(h);
    medyan_status st = medyan_mech_set_shapes(h, &best);
    float best_ms = 0.0f;
    if (st == MEDYAN_OK) st = time_evaluate(h, reps, &best_ms);
    // the layout first: the other fields' best values depend on it
    int32_t* fields[5] = {&best.pass_layout, &best.bonded_threads, &best.excl_threads, &best.chain_threads,
                          &best.chain_energy_blocks_per_sm};
    const int* sets[5] = {kLayout, kBonded, kExcl, kChain, kEnergyBps};
    for (int f = 0; f < 5 && st == MEDYAN_OK; ++f) {
        const int keep = *fields[f];
        for (int c = 0; c < 3 && st == MEDYAN_OK; ++c) {
            if (sets[f][c] == keep || sets[f][c] == kNone) continue;
            medyan_launch_shapes trial = best;
            int32_t* tf[5] = {&trial.pass_layout, &trial.bonded_threads, &trial.excl_threads, &trial.chain_threads,
                              &trial.chain_energy_blocks_per_sm};
            *tf[f] = sets[f][c];
            st = medyan_mech_set_shapes(h, &trial);
            float ms = 0.0f;
            if (st == MEDYAN_OK) st = time_evaluate(h, reps, &ms);
            if (st == MEDYAN_OK && ms < best_ms) {
                best_ms = ms;
                best = trial;
            }
        }
    }
    if (st == MEDYAN_OK) st = medyan_mech_set_shapes(h, &best);
    if (st == MEDYAN_OK && chosen) *chosen = best;
    return st;
}

}  // extern "C"

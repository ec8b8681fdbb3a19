// batch.cu — many independent networks minimized together.
//
// Each replica keeps its own handle (vectorization, internal bead order,
// device neighbor list, single-network passes). A batched minimization packs
// the replicas' device arrays into one set (pbatch.h) and runs one
// conjugate-gradient loop for all of them: every force and energy kernel
// launches once per pass for the whole batch, while the CG state, the
// line-search step sizes and the reductions stay per replica, so each replica
// follows CGMethod::minimize exactly and stops at its own convergence test
// (a done replica is masked out of the remaining iterations).
#include <cstring>
#include <vector>

#include "handle.h"
#include "pbatch.h"

struct medyan_batch {
    std::vector<medyan_mech*> h;
    mb::PackedBatch pb;
    ~medyan_batch() {
        for (auto* p : h) medyan_mech_destroy(p);
    }
};

using namespace mb;

extern "C" {

medyan_status medyan_batch_create(const medyan_system* systems, int32_t n_replicas, int32_t precision,
                                  medyan_batch** out) {
    if (!out || n_replicas < 0 || (n_replicas > 0 && !systems)) return MEDYAN_ERR_INVALID_ARG;
    *out = nullptr;
    auto* b = new medyan_batch();
    b->h.reserve(n_replicas);
    for (int r = 0; r < n_replicas; ++r) {
        medyan_mech* h = nullptr;
        medyan_status st = medyan_mech_create(&systems[r], precision, &h);
        if (st != MEDYAN_OK) {
            delete b;
            return st;
        }
        b->h.push_back(h);
    }
    *out = b;
    return MEDYAN_OK;
}

medyan_status medyan_batch_destroy(medyan_batch* b) {
    if (!b) return MEDYAN_ERR_INVALID_ARG;
    delete b;
    return MEDYAN_OK;
}

int32_t medyan_batch_size(const medyan_batch* b) { return b ? (int32_t)b->h.size() : 0; }

medyan_status medyan_batch_set_deterministic(medyan_batch* b, int32_t on) {
    if (!b || (on != 0 && on != 1)) return MEDYAN_ERR_INVALID_ARG;
    if (b->pb.stream) {
        cudaError_t e = cudaStreamSynchronize(b->pb.stream);  // no packed pass may still write the old way
        if (e != cudaSuccess) return cuda_status(e);
    }
    // the replicas' own passes (medyan_batch_evaluate) follow the same setting
    for (medyan_mech* h : b->h) {
        const medyan_status st = medyan_mech_set_deterministic(h, on);
        if (st != MEDYAN_OK) return st;
    }
    b->pb.deterministic = on != 0;
    return MEDYAN_OK;
}

medyan_mech* medyan_batch_replica(medyan_batch* b, int32_t r) {
    return (b && r >= 0 && r < (int32_t)b->h.size()) ? b->h[r] : nullptr;
}

medyan_status medyan_batch_minimize(medyan_batch* b, const medyan_cg_params* p, double* const* coords_inout,
                                    double* const* forces_out, medyan_min_result* results, int32_t* statuses) {
    if (!b || !p || (!b->h.empty() && (!coords_inout || !statuses))) return MEDYAN_ERR_INVALID_ARG;
    const int n = (int)b->h.size();
    if (n == 0) return MEDYAN_OK;
    for (int r = 0; r < n; ++r)
        if (!coords_inout[r] && b->h[r]->n_beads) return MEDYAN_ERR_INVALID_ARG;
    PackedBatch& pb = b->pb;
    medyan_status st = pack_batch(pb, b->h);
    if (st != MEDYAN_OK) return st;
    cudaStream_t s = pb.stream;
    for (int r = 0; r < n; ++r) {
        cudaError_t e = coords_to_device(b->h[r], coords_inout[r], pb.x.raw() + 3 * (size_t)pb.base[r], s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    st = cg_batch_run(pb, b->h[0]->prec, p);
    if (st != MEDYAN_OK) return st;
    std::vector<CGState> sf(n);
    std::vector<double> eo((size_t)n * 2 * (MEDYAN_FF_COUNT + 1));
    cudaError_t e = cudaMemcpyAsync(sf.data(), pb.st.raw(), sizeof(CGState) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(eo.data(), pb.eout.raw(), sizeof(double) * eo.size(), cudaMemcpyDeviceToHost, s);
    for (int r = 0; r < n && e == cudaSuccess; ++r) {
        const size_t o = 3 * (size_t)pb.base[r];
        e = coords_to_host(b->h[r], pb.x.raw() + o, coords_inout[r], s);
        if (e == cudaSuccess && forces_out && forces_out[r]) e = coords_to_host(b->h[r], pb.fcur.raw() + o, forces_out[r], s);
    }
    int force_status = 0;
    if (e == cudaSuccess && pb.deterministic)
        e = cudaMemcpyAsync(&force_status, pb.fs.status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    const int kOut = MEDYAN_FF_COUNT + 1;
    // a force contribution out of the fixed-point range (bit 2) leaves the
    // sums wrong for the whole batch
    medyan_status worst = (force_status & 4) ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
    for (int r = 0; r < n; ++r) {
        const CGState& c = sf[r];
        statuses[r] = c.status;
        if (c.status != MEDYAN_OK && c.status != MEDYAN_ERR_LINE_SEARCH && worst == MEDYAN_OK)
            worst = (medyan_status)c.status;
        if (!results) continue;
        medyan_min_result& out = results[r];
        std::memset(&out, 0, sizeof out);
        const double* before = eo.data() + (size_t)r * 2 * kOut;
        const double* after = before + kOut;
        const bool ls = c.status == MEDYAN_ERR_LINE_SEARCH;
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
            out.energy_before[i] = before[i];
            out.energy_after[i] = ls ? 0.0 : after[i];
        }
        out.energy_before_total = before[MEDYAN_FF_COUNT];
        out.energy_after_total = ls ? 0.0 : after[MEDYAN_FF_COUNT];
        out.error_flags = (uint32_t)c.error_flags;
        out.num_energy_call = c.num_energy_call;
        out.energy_call_limit = c.energy_call_limit;
        out.num_force_call = c.num_force_call;
        out.force_call_limit = c.force_call_limit;
        out.num_iter = c.num_iter;
        out.grad_inf_norm = c.grad_inf_norm;
        out.grad_tol = c.grad_tol;
        out.energy_rel_change = c.energy_rel_change;
        out.energy_rel_tol = c.energy_rel_tol;
    }
    return worst;
}

static bool in3(int v, int a, int b, int c) { return v == a || v == b || v == c; }

medyan_status medyan_batch_set_shapes(medyan_batch* b, const medyan_batch_shapes* sh) {
    if (!b || !sh) return MEDYAN_ERR_INVALID_ARG;
    if (!in3(sh->bonded_threads, 128, 256, 512) || !in3(sh->excl_threads, 32, 64, 128) ||
        !in3(sh->chain_threads, 128, 256, 512) || !in3(sh->chain_chunk, 256, 512, 1024))
        return MEDYAN_ERR_INVALID_ARG;
    PackedBatch& pb = b->pb;
    if (pb.stream) {
        cudaError_t e = cudaStreamSynchronize(pb.stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    pb.bonded_block = sh->bonded_threads;
    pb.excl_block = sh->excl_threads;
    pb.chain_threads = sh->chain_threads;
    pb.chain_chunk = sh->chain_chunk;
    pb.repack = true;
    if (pb.graph) {  // captured with the old layout
        cudaGraphExecDestroy(pb.graph);
        pb.graph = nullptr;
    }
    return MEDYAN_OK;
}

medyan_status medyan_batch_get_shapes(medyan_batch* b, medyan_batch_shapes* sh) {
    if (!b || !sh) return MEDYAN_ERR_INVALID_ARG;
    const PackedBatch& pb = b->pb;
    *sh = medyan_batch_shapes{pb.bonded_block, pb.excl_block, pb.chain_threads, pb.chain_chunk};
    return MEDYAN_OK;
}

medyan_status medyan_batch_autotune(medyan_batch* b, int32_t reps, medyan_batch_shapes* chosen) {
    if (!b || reps <= 0) return MEDYAN_ERR_INVALID_ARG;
    if (b->h.empty()) return MEDYAN_OK;
    PackedBatch& pb = b->pb;
    const int prec = b->h[0]->prec;
    // pack with the given shapes, take each replica's current coordinates, time
    auto trial = [&](const medyan_batch_shapes& sh, float* ms) -> medyan_status {
        medyan_status st = medyan_batch_set_shapes(b, &sh);
        if (st == MEDYAN_OK) st = pack_batch(pb, b->h);
        if (st != MEDYAN_OK) return st;
        for (size_t r = 0; r < b->h.size(); ++r) {
            const medyan_mech* h = b->h[r];
            if (!h->n_beads) continue;
            cudaError_t e = cudaMemcpyAsync(pb.x.raw() + 3 * (size_t)pb.base[r], h->x.raw(),
                                            sizeof(double) * 3 * (size_t)h->n_beads, cudaMemcpyDeviceToDevice,
                                            pb.stream);
            if (e != cudaSuccess) return cuda_status(e);
        }
        return cg_batch_time_evaluate(pb, prec, reps, ms);
    };
    medyan_batch_shapes best{};
    medyan_status st = medyan_batch_get_shapes(b, &best);
    float best_ms = 0.0f;
    if (st == MEDYAN_OK) st = trial(best, &best_ms);
    const int sets[4][3] = {{128, 256, 512}, {32, 64, 128}, {128, 256, 512}, {256, 512, 1024}};
    for (int f = 0; f < 4 && st == MEDYAN_OK; ++f) {
        for (int c = 0; c < 3 && st == MEDYAN_OK; ++c) {
            medyan_batch_shapes t = best;
            int32_t* field[4] = {&t.bonded_threads, &t.excl_threads, &t.chain_threads, &t.chain_chunk};
            if (*field[f] == sets[f][c]) continue;
            *field[f] = sets[f][c];
            float ms = 0.0f;
            st = trial(t, &ms);
            if (st == MEDYAN_OK && ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        }
    }
    if (st == MEDYAN_OK) st = medyan_batch_set_shapes(b, &best);
    if (st == MEDYAN_OK && chosen) *chosen = best;
    return st;
}

medyan_status medyan_batch_evaluate(medyan_batch* b, const double* const* coords, double* e_totals,
                                    double* const* forces_out) {
    if (!b || (!b->h.empty() && (!coords || !e_totals || !forces_out))) return MEDYAN_ERR_INVALID_ARG;
    const int n = (int)b->h.size();
    // enqueue all replicas' passes, then read back in order
    for (int r = 0; r < n; ++r) {
        medyan_mech* h = b->h[r];
        cudaError_t e = coords_to_device(h, coords[r], h->x.raw(), h->stream);
        if (e == cudaSuccess) e = launch_pass(h, kPassBoth);
        if (e != cudaSuccess) return cuda_status(e);
    }
    medyan_status worst = MEDYAN_OK;
    for (int r = 0; r < n; ++r) {
        medyan_mech* h = b->h[r];
        double out[MEDYAN_FF_COUNT + 1];
        int status = 0;
        cudaError_t e = cudaMemcpyAsync(out, h->energy_out.raw(), sizeof out, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = coords_to_host(h, h->f.raw(), forces_out[r], h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&status, h->force_status.raw(), sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.raw(), 0, sizeof(int), h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_status(e);
        e_totals[r] = out[MEDYAN_FF_COUNT];
        if ((status || std::isinf(out[MEDYAN_FF_COUNT])) && worst == MEDYAN_OK) worst = MEDYAN_ERR_NONFINITE;
    }
    return worst;
}

}  // extern "C"

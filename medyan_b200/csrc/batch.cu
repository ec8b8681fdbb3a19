// batch.cu — many independent networks minimized together.
//
// Each replica gets its own handle (device buffers, internal bead order,
// stream, pass graphs and minimization graph). A batch minimization enqueues
// every replica's whole minimization (one graph launch each, with its
// conditional loops running on the device) on its own stream before waiting
// for any, so the replicas run concurrently and each finishes as soon as its
// own convergence test passes: the per-replica convergence mask is the
// replica's own loop condition. Results are identical to minimizing each
// replica alone (CGMethod::minimize semantics per replica).
#include <vector>

#include "handle.h"

struct medyan_batch {
    std::vector<medyan_mech*> h;
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

medyan_mech* medyan_batch_replica(medyan_batch* b, int32_t r) {
    return (b && r >= 0 && r < (int32_t)b->h.size()) ? b->h[r] : nullptr;
}

medyan_status medyan_batch_minimize(medyan_batch* b, const medyan_cg_params* p, double* const* coords_inout,
                                    double* const* forces_out, medyan_min_result* results, int32_t* statuses) {
    if (!b || !p || (!b->h.empty() && (!coords_inout || !statuses))) return MEDYAN_ERR_INVALID_ARG;
    const int n = (int)b->h.size();
    for (int r = 0; r < n; ++r)
        if (!coords_inout[r]) return MEDYAN_ERR_INVALID_ARG;
    // enqueue every replica first, then collect in order; a replica that
    // could not be enqueued reports its own status and is not collected
    std::vector<medyan_status> enq(n);
    for (int r = 0; r < n; ++r) enq[r] = cg_enqueue(b->h[r], p, coords_inout[r]);
    medyan_status worst = MEDYAN_OK;
    for (int r = 0; r < n; ++r) {
        medyan_status st = enq[r];
        if (st == MEDYAN_OK)
            st = cg_collect(b->h[r], coords_inout[r], forces_out ? forces_out[r] : nullptr,
                            results ? &results[r] : nullptr);
        statuses[r] = st;
        // a failed line search is a per-replica result; anything else is an error
        if (st != MEDYAN_OK && st != MEDYAN_ERR_LINE_SEARCH && worst == MEDYAN_OK) worst = st;
    }
    return worst;
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

// async.cu — asynchronous, double-buffered energy + force evaluation.
//
// medyan_mech_evaluate moves the coordinates in, runs the evaluate pass and
// moves the forces out on one stream and waits: the two host copies (24 bytes
// per bead each way) run one after the other and dominate the call. Here each
// call is three stages on three streams:
//
//   in stream:      host coordinates -> input slot k             (H2D)
//   handle stream:  slot k -> internal coordinates, evaluate pass,
//                   forces -> output slot k, energies -> slot k
//   out stream:     output slot k -> host forces and energies    (D2H)
//
// with two slots (k alternates), so the inbound copy of call n+1 runs while
// call n's pass and its outbound copy run: the host link carries traffic in
// both directions at once, and a stream of calls is bound by the slower
// direction instead of the sum. Events order each slot's reuse: an input slot
// is refilled only after the pass that read it, an output slot only after the
// copy that drained it.
#include <cstring>

#include "handle.h"

namespace mb {

struct medyan_async {
    cudaStream_t in = nullptr, out = nullptr;
    DevBuf<double> x_slot[2], f_slot[2], e_slot[2];
    cudaEvent_t in_ready[2] = {}, in_free[2] = {}, computed[2] = {}, out_free[2] = {};
    bool in_used[2] = {false, false}, out_used[2] = {false, false};
    int next = 0;

    cudaError_t init(int n3) {
        cudaError_t e = cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking);
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
            e = x_slot[k].reserve(n3 ? n3 : 1);
            if (e == cudaSuccess) e = f_slot[k].reserve(n3 ? n3 : 1);
            if (e == cudaSuccess) e = e_slot[k].reserve(MEDYAN_FF_COUNT + 1);
            cudaEvent_t* evs[4] = {&in_ready[k], &in_free[k], &computed[k], &out_free[k]};
            for (int j = 0; j < 4 && e == cudaSuccess; ++j) e = cudaEventCreateWithFlags(evs[j], cudaEventDisableTiming);
        }
        return e;
    }
    ~medyan_async() {
        if (in) cudaStreamSynchronize(in);
        if (out) cudaStreamSynchronize(out);
        for (int k = 0; k < 2; ++k)
            for (cudaEvent_t ev : {in_ready[k], in_free[k], computed[k], out_free[k]})
                if (ev) cudaEventDestroy(ev);
        if (in) cudaStreamDestroy(in);
        if (out) cudaStreamDestroy(out);
    }
};

void destroy_async(medyan_mech* h) {
    delete h->async;
    h->async = nullptr;
}

// Waits for the copy streams (the handle's own stream is the caller's to sync).
static cudaError_t drain_async(medyan_mech* h) {
    if (!h->async) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(h->async->in);
    cudaError_t e2 = cudaStreamSynchronize(h->async->out);
    return e != cudaSuccess ? e : e2;
}

}  // namespace mb

using namespace mb;

extern "C" {

medyan_status medyan_mech_evaluate_async(medyan_mech* h, const double* coord, double* force_out, double* e_out) {
    if (!h || !coord || !force_out || !e_out) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_status(e);
    const int n3 = 3 * h->n_beads;
    if (!h->async) {
        h->async = new medyan_async();
        e = h->async->init(n3);
        if (e != cudaSuccess) {
            destroy_async(h);
            return cuda_status(e);
        }
    }
    medyan_async& A = *h->async;
    const int k = A.next;
    A.next ^= 1;
    const size_t bytes = sizeof(double) * (size_t)n3;
    cudaStream_t s = h->stream;
    // in: refill slot k once the pass that read it last has
    if (A.in_used[k]) e = cudaStreamWaitEvent(A.in, A.in_free[k], 0);
    if (e == cudaSuccess && n3) e = cudaMemcpyAsync(A.x_slot[k].raw(), coord, bytes, cudaMemcpyHostToDevice, A.in);
    if (e == cudaSuccess) e = cudaEventRecord(A.in_ready[k], A.in);
    // the pass: slot k's coordinates into the internal layout, then evaluate
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, A.in_ready[k], 0);
    if (e == cudaSuccess && n3) {
        if (h->identity_order) e = cudaMemcpyAsync(h->x.raw(), A.x_slot[k].raw(), bytes, cudaMemcpyDeviceToDevice, s);
        else launch_to_internal(n3, h->order.raw(), A.x_slot[k].raw(), h->x.raw(), s);
    }
    if (e == cudaSuccess) e = cudaEventRecord(A.in_free[k], s);
    A.in_used[k] = true;
    if (e == cudaSuccess) e = launch_pass(h, kPassBoth);
    // results into output slot k once its previous contents have left
    if (e == cudaSuccess && A.out_used[k]) e = cudaStreamWaitEvent(s, A.out_free[k], 0);
    if (e == cudaSuccess && n3) {
        if (h->identity_order) e = cudaMemcpyAsync(A.f_slot[k].raw(), h->f.raw(), bytes, cudaMemcpyDeviceToDevice, s);
        else launch_to_external(n3, h->order.raw(), h->f.raw(), A.f_slot[k].raw(), s);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(A.e_slot[k].raw(), h->energy_out.raw(), sizeof(double) * (MEDYAN_FF_COUNT + 1),
                            cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(A.computed[k], s);
    // out: drain slot k to the caller's buffers
    if (e == cudaSuccess) e = cudaStreamWaitEvent(A.out, A.computed[k], 0);
    if (e == cudaSuccess && n3) e = cudaMemcpyAsync(force_out, A.f_slot[k].raw(), bytes, cudaMemcpyDeviceToHost, A.out);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(e_out, A.e_slot[k].raw(), sizeof(double) * (MEDYAN_FF_COUNT + 1), cudaMemcpyDeviceToHost,
                            A.out);
    if (e == cudaSuccess) e = cudaEventRecord(A.out_free[k], A.out);
    A.out_used[k] = true;
    if (e == cudaSuccess) e = cudaGetLastError();
    return cuda_status(e);
}

medyan_status medyan_mech_wait(medyan_mech* h) {
    if (!h) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_status(e);
    // the force-fallback status of every pass since the last wait (the
    // passes OR their bits into it)
    int status = 0;
    e = cudaMemcpyAsync(&status, h->force_status.ptr(), sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.ptr(), 0, sizeof(int), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = drain_async(h);
    if (e != cudaSuccess) return cuda_status(e);
    return status ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
}

}  // extern "C"

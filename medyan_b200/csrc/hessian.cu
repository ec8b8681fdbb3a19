// hessian.cu — ForceFieldManager::computeHessian on the device.
//
// ForceFieldManager::computeHessian (src/Mechanics/ForceField/ForceFieldManager.cpp:354-398)
// builds the dense Hessian column by column by central differences of the
// forces: for every degree of freedom i it evaluates the forces with
// coordinate i moved by +delta and by -delta and stores
//   H[i][j] = (float)( -(F_j(x + delta e_i) - F_j(x - delta e_i)) / (2*delta) )
// (the reference keeps each entry in a float, then in its double matrix).
//
// Here one CUDA graph does one column: perturb x_i (device-side index and
// saved value), a force pass into one buffer, perturb to x_i - delta, a
// force pass into a second buffer, the row kernel, restore x_i and advance
// the index. The host launches that graph once per degree of freedom and
// copies finished rows out in chunks; the coordinates are restored exactly.
#include <algorithm>
#include <vector>

#include "handle.h"

namespace mb {

namespace {

constexpr int kThreads = 256;
constexpr int kRowsPerChunk = 128;  // rows staged on the device between host copies

struct HessState {
    int k;        // internal degree of freedom being perturbed
    int pad;
    double orig;  // its unperturbed coordinate
};

// mode 0: save x_k and set x_k + delta; mode 1: set x_k - delta (the
// reference adds and subtracts the float delta to copies of the coordinates)
__global__ void k_hess_perturb(double* __restrict__ x, HessState* __restrict__ st, float delta, int mode) {
    const int k = st->k;
    if (mode == 0) {
        const double o = x[k];
        st->orig = o;
        x[k] = o + (double)delta;
    } else {
        x[k] = st->orig - (double)delta;
    }
}

// Row of internal degree of freedom k into the staging rows, in the caller's
// column order: col(j) = 3*order[j/3] + j%3 (identity when order is null).
__global__ void __launch_bounds__(kThreads) k_hess_row(int n3, const double* __restrict__ fp,
                                                       const double* __restrict__ fm, float delta,
                                                       const int* __restrict__ order,
                                                       const HessState* __restrict__ st,
                                                       double* __restrict__ rows) {
    const int k = st->k;
    double* __restrict__ row = rows + (size_t)(k % kRowsPerChunk) * n3;
    const double two_delta = (double)(2.0f * delta);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n3; j += gridDim.x * blockDim.x) {
        const int col = order ? 3 * order[j / 3] + j % 3 : j;
        const float h = (float)(-(fp[j] - fm[j]) / two_delta);
        row[col] = (double)h;
    }
}

__global__ void k_hess_restore(double* __restrict__ x, HessState* __restrict__ st) {
    x[st->k] = st->orig;
    st->k += 1;
}

int row_blocks(int n3) {
    const int b = (n3 + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
}

}  // namespace

}  // namespace mb

using namespace mb;

extern "C" medyan_status medyan_mech_hessian(medyan_mech* h, float delta, double* H) {
    if (!h || !(delta > 0.0f) || (h->n_beads && !H)) return MEDYAN_ERR_INVALID_ARG;
    const int n3 = 3 * h->n_beads;
    if (n3 == 0) return MEDYAN_OK;
    if (n3 > MEDYAN_HESSIAN_MAX_DOF) return MEDYAN_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_status(e);
    cudaStream_t s = h->stream;
    DevBuf<HessState> st;
    DevBuf<double> rows;
    if (e == cudaSuccess) e = h->hv_a.reserve(n3);
    if (e == cudaSuccess) e = h->hv_b.reserve(n3);
    if (e == cudaSuccess) e = st.reserve(1);
    if (e == cudaSuccess) e = rows.reserve((size_t)kRowsPerChunk * n3);
    if (e != cudaSuccess) return cuda_status(e);
    const HessState s0{0, 0, 0.0};
    e = st.assign(&s0, 1, s);
    if (e != cudaSuccess) return cuda_status(e);

    // one column as a graph
    const ForceTarget tp{h->hv_a.raw(), nullptr, nullptr, nullptr, nullptr, nullptr};
    const ForceTarget tm{h->hv_b.raw(), nullptr, nullptr, nullptr, nullptr, nullptr};
    const int* order = h->identity_order ? nullptr : h->order.raw();
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e);
    k_hess_perturb<<<1, 1, 0, s>>>(h->x.raw(), st.raw(), delta, 0);
    launch_forces(h->chain, h->ff, h->prec, h->x.raw(), tp, h->fs, s, &h->fork);
    k_hess_perturb<<<1, 1, 0, s>>>(h->x.raw(), st.raw(), delta, 1);
    launch_forces(h->chain, h->ff, h->prec, h->x.raw(), tm, h->fs, s, &h->fork);
    k_hess_row<<<row_blocks(n3), kThreads, 0, s>>>(n3, h->hv_a.raw(), h->hv_b.raw(), delta, order, st.raw(),
                                                   rows.raw());
    k_hess_restore<<<1, 1, 0, s>>>(h->x.raw(), st.raw());
    e = cudaStreamEndCapture(s, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_status(e);

    // rows of a chunk land in staging row k % kRowsPerChunk; the caller's
    // row of internal degree of freedom k is 3*order[k/3] + k%3
    for (int k0 = 0; k0 < n3 && e == cudaSuccess; k0 += kRowsPerChunk) {
        const int k1 = std::min(n3, k0 + kRowsPerChunk);
        for (int k = k0; k < k1 && e == cudaSuccess; ++k) e = cudaGraphLaunch(exec, s);
        for (int k = k0; k < k1 && e == cudaSuccess; ++k) {
            const int rowi = h->identity_order ? k : 3 * h->order_host[k / 3] + k % 3;
            e = cudaMemcpyAsync(H + (size_t)rowi * n3, rows.raw() + (size_t)(k % kRowsPerChunk) * n3,
                                sizeof(double) * n3, cudaMemcpyDeviceToHost, s);
        }
    }
    int status = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&status, h->force_status.raw(), sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->force_status.raw(), 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaGraphExecDestroy(exec);
    if (e != cudaSuccess) return cuda_status(e);
    return status ? MEDYAN_ERR_NONFINITE : MEDYAN_OK;
}

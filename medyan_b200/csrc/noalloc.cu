// noalloc.cu — excluded-volume energy of caller-owned device arrays with no
// device allocation.
//
// The handle-based entry points keep their scratch in buffers the handle
// allocates with cudaMalloc. Some callers cannot let a library allocate
// device memory at the point where they need an energy: an application that
// hands the whole device to its own pool allocator (cudaMalloc there would
// fail or fragment the pool), or one that evaluates energies from a step
// loop whose device memory footprint has to stay fixed. For those callers,
// medyan_excl_energy_noalloc runs the same excluded-volume kernels as the
// handle path (the analytic CylinderExclVolRepulsion energy, the energyN
// fallback for degenerate pairs and the deterministic finish) with all
// scratch in one fixed-size static device array of this library.
//
// Set-up: every call looks up the array's device address on the current
// device with cudaGetSymbolAddress (a cheap host query; the address is not
// cached, so it stays right if the device's context is ever recreated). The
// first call on each device also fills the quadrature grids of the fallback
// for degenerate pairs, once; make that first call before any stream capture
// begins on the device. A cudaDeviceReset discards that one-time set-up along
// with every handle: do not use the library across a device reset.
//
// The call is synchronous: it waits for `stream` before it returns.
//
// The scratch array is shared by every call on a device: calls that overlap
// in time on one device (two host threads, or two streams) race on it and
// give wrong results. Serialize them.
#include <cstring>

#include "handle.h"

namespace mb {

namespace {

// Scratch layout, in doubles:
//   [0, 64)          out: per-force-field energies and total (one step size)
//   [64, 72)         int bad[kMaxLambda], int fb_count, int index_error
//   [128, 640)       int2 fb_list[kFallbackCap]
//   [1024, ...)      block partials: (excl blocks) x 4
constexpr int kOutOff = 0;
constexpr int kFlagOff = 64;
constexpr int kFbListOff = 128;
constexpr int kPartialOff = 1024;
constexpr int kMaxBlocks = (MEDYAN_NOALLOC_MAX_EXCL_PAIRS + kExclBlock - 1) / kExclBlock;
constexpr int kScratchDoubles = kPartialOff + 4 * (kMaxBlocks + 1);
static_assert(kMaxLambda * (MEDYAN_FF_COUNT + 1) <= kFlagOff - kOutOff, "out region");
static_assert(kMaxLambda + 2 <= 2 * (kFbListOff - kFlagOff), "flag region");
static_assert(kFallbackCap <= kPartialOff - kFbListOff, "fallback-queue region");

// About 129 KiB for the maximum of 262144 pairs.
static __device__ __align__(256) double g_scratch[kScratchDoubles];

// Device address of g_scratch on the current device, looked up on every
// call; the excluded-volume kernels' one-time set-up runs on first use.
cudaError_t scratch_on_current_device(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    e = init_excl_kernels();
    if (e != cudaSuccess) return e;
    *out = static_cast<double*>(p);
    return cudaSuccess;
}

// Bead-set entries must be coordinate offsets 3*b with 0 <= b < n_beads.
__global__ void k_check_offsets(const int* __restrict__ bs, long long n, long long n3, int* __restrict__ err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int o = bs[i];
        if (o < 0 || o >= n3 || o % 3 != 0) atomicOr(err, 1);
    }
}

}  // namespace

}  // namespace mb

using namespace mb;

extern "C" medyan_status medyan_excl_energy_noalloc(const double* d_coords, int32_t n_beads,
                                                    const int32_t* d_excl_beads, const double* d_excl_krs,
                                                    int32_t n_pairs, double* e_out, void* stream) {
    if (!e_out || n_beads < 0 || n_pairs < 0) return MEDYAN_ERR_INVALID_ARG;
    if (n_pairs > MEDYAN_NOALLOC_MAX_EXCL_PAIRS) return MEDYAN_ERR_CAPACITY;
    if (n_pairs == 0) {
        *e_out = 0.0;
        return MEDYAN_OK;
    }
    if (!d_coords || !d_excl_beads || !d_excl_krs) return MEDYAN_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(d_excl_beads) % alignof(int4) != 0) return MEDYAN_ERR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) return cuda_status(e);

    int* flags = reinterpret_cast<int*>(scratch + kFlagOff);
    int* bad = flags;                      // [kMaxLambda]
    int* fb_count = flags + kMaxLambda;    // must start at zero
    int* index_error = fb_count + 1;       // must start at zero

    // zero the flags (bad, queue count, index error) before any kernel reads them
    e = cudaMemsetAsync(flags, 0, sizeof(int) * (kMaxLambda + 2), s);
    if (e != cudaSuccess) return cuda_status(e);
    const long long n_offs = 4LL * n_pairs;
    const int check_blocks = (int)((n_offs + kBlock - 1) / kBlock < 148 * 4 ? (n_offs + kBlock - 1) / kBlock : 148 * 4);
    k_check_offsets<<<check_blocks, kBlock, 0, s>>>(d_excl_beads, n_offs, 3LL * n_beads, index_error);
    int host_err = 0;
    e = cudaMemcpyAsync(&host_err, index_error, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    if (host_err) return MEDYAN_ERR_INDEX_RANGE;

    DeviceFF ff;
    std::memset(&ff, 0, sizeof ff);
    ff.n_beads = n_beads;
    ff.n_excl = n_pairs;
    ff.excl_bs = reinterpret_cast<const int4*>(d_excl_beads);
    ff.excl_krs = d_excl_krs;

    EnergyScratch es;
    es.partial = scratch + kPartialOff;
    es.fb_count = fb_count;
    es.fb_list = reinterpret_cast<int2*>(scratch + kFbListOff);
    es.fb_cap = kFallbackCap;  // the static array's queue holds kFallbackCap entries
    es.bad = bad;
    es.out = scratch + kOutOff;
    es.stage = nullptr;  // one-block finish: no arrival ticket to keep
    es.ticket = nullptr;
    es.n_blocks_chain = 0;
    es.n_blocks_bonded = 0;
    es.n_blocks_excl = excl_blocks(ff);

    // one step size (lambda = 0, no direction): the finish kernel treats a
    // null step-size set as K = 1
    launch_excl_energy(ff, MEDYAN_PREC_FP64, d_coords, nullptr, nullptr, es, s);
    launch_excl_energy_fallback_and_finish(ff, d_coords, nullptr, nullptr, es, s);
    double out[MEDYAN_FF_COUNT + 1];
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, es.out, sizeof out, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    *e_out = out[MEDYAN_FF_EXCLUDED_VOLUME];
    if (std::isinf(out[MEDYAN_FF_COUNT])) return MEDYAN_ERR_NONFINITE;
    return MEDYAN_OK;
}

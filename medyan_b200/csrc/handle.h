// handle.h — the medyan_mech handle: owned device buffers, the stream and the
// scratch of every pass. All device allocation happens at create, update,
// set_cylinders and neighbor rebuilds (grow-only); the energy, force and CG
// passes allocate nothing.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>

#include "internal.h"

namespace mb {

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    size_t n = 0;

    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    // Grow-only: keeps the old contents only when no reallocation is needed.
    cudaError_t reserve(size_t count) {
        if (count <= cap && p) {
            n = count;
            return cudaSuccess;
        }
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = count ? count : 1;
        cudaError_t e = cudaMalloc(&p, want * sizeof(T));
        if (e != cudaSuccess) return e;
        cap = want;
        n = count;
        return cudaSuccess;
    }
    // Copies count host elements in; returns once the host data is consumed.
    cudaError_t assign(const T* host, size_t count, cudaStream_t s) {
        cudaError_t e = reserve(count);
        if (e != cudaSuccess || count == 0) return e;
        e = cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(s);
    }
    T* ptr() const { return n ? p : nullptr; }
    T* raw() const { return p; }
};

// Device-resident state of one conjugate-gradient minimization
// (the scalars of CGMethod::minimize, CGMethod.hpp:826-1743).
struct CGState {
    // parameters
    int method;
    int try_to_recover;
    int energy_call_limit;
    int force_call_limit;
    double max_dist, lambda_max, grad_tol, energy_rel_tol;
    // counters and flags
    int num_energy_call, num_force_call, num_iter;
    int safe_mode;
    int done;            // loop finished (converged, call limit, error)
    int status;          // medyan_status of the run
    int error_flags;     // MinimizationResult::errorLineSearch
    int parity;          // force[parity] holds the current force
    int ls_active;       // a line search is in progress
    int ls_need_e0;      // E(x) must be evaluated in the next pass
    int ls_result;       // 0 pending, 1 accepted, 2 failed
    int have_min_e;
    int ls_passes;       // passes used by the current line search
    int last_backtracks; // halvings needed by the previous line search
    // reals
    double E_cur;        // energy at x
    double grad_inf_norm;
    double energy_rel_change;
    double prev_energy;
    double last_fdotf;
    double slope;        // searchDir . force at the start of the line search
    double lambda;       // next lambda to try / accepted lambda
    double lambda_next;  // first lambda of the next pass
    double E_new;        // energy at the accepted lambda
    double beta;
    double new_grad, prev_grad;
    double min_e;
    double total_energy; // CGMethod::TotalEnergy (energy of the last line search)
    double recovery_step;
    double dot_sf;       // searchDir . force after the direction update
};

// Per-block partials of the CG vector passes.
struct CGScratch {
    double* part;        // [blocks][4]
    int nblocks;
};

}  // namespace mb

struct medyan_mech {
    int device = 0;
    int prec = 0;
    int n_beads = 0;
    cudaStream_t stream = nullptr;

    mb::DeviceFF ff{};
    mb::EnergyScratch es{};
    mb::ForceScratch fs{};

    // force-field records
    mb::DevBuf<int2> stretch_bs;
    mb::DevBuf<double2> stretch_p;
    mb::DevBuf<int4> bend_bs;
    mb::DevBuf<double2> bend_p;
    mb::DevBuf<int4> linker_bs, motor_bs, branch_bs, excl_bs;
    mb::DevBuf<double4> linker_p, motor_p, branch_pa, branch_pb, planes;
    mb::DevBuf<double> excl_krs;
    mb::DevBuf<int> boundary_bs, boundary_plane;
    mb::DevBuf<double2> boundary_p;

    // coordinates, forces, scratch
    mb::DevBuf<double> x, f, partial, energy_out;
    mb::DevBuf<int> e_fb_count, e_bad, f_fb_count, f_fb_list, force_status;
    mb::DevBuf<int2> e_fb_list;
    mb::DevBuf<mb::LambdaSet> lam_zero;

    // conjugate gradient
    mb::DevBuf<double> cg_dir, cg_force2, cg_min_coords, cg_part;
    mb::DevBuf<mb::CGState> cg_state;
    mb::DevBuf<mb::LambdaSet> cg_lam;
    mb::DevBuf<double> cg_eout;   // energy outputs of the first/last individual energy calls

    // neighbor list (nl.cu)
    struct NL;
    NL* nl = nullptr;

    medyan_status init();
    ~medyan_mech();
};

namespace mb {
medyan_status cuda_status(cudaError_t e);
medyan_status validate_system(const medyan_system* s);
medyan_status upload_system(medyan_mech* h, const medyan_system* s);
medyan_status refresh_device_ff(medyan_mech* h);
medyan_status sync_status(medyan_mech* h);
void enqueue_energy(medyan_mech* h, const double* x, const double* d, const LambdaSet* lam);
void enqueue_forces(medyan_mech* h, const double* x, double* f);
void destroy_nl(medyan_mech* h);
}  // namespace mb

// handle.h — the medyan_mech handle: owned device buffers, the stream and the
// scratch of every pass. All device allocation happens at create, update,
// set_cylinders and neighbor rebuilds (grow-only); the energy, force and CG
// passes allocate nothing.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "internal.h"
#include "pass.h"

namespace mb {

struct medyan_async;  // async.cu

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

// Device-resident state of one conjugate-gradient minimization: the scalars
// of CGMethod::minimize (src/Mechanics/Minimizer/CGMethod.hpp:826-1743) plus
// the flags that steer the per-iteration kernels without the host.
struct CGState {
    // parameters (ConjugateGradientParams)
    int method, try_to_recover, energy_call_limit, force_call_limit;
    double max_dist, lambda_max, grad_tol, energy_rel_tol;
    // MinimizationResult counters
    int num_energy_call, num_force_call, num_iter;
    int error_flags;
    int status;            // medyan_status of the run
    int done;              // loop finished
    int safe_mode;
    int parity;            // force[parity] holds the current force
    // line search
    int ls_active;         // a line search is in progress
    int ls_first_pass;     // the next pass is the first of its line search
    int need_e0;           // E(x) is not known and must be evaluated
    int ls_immediate_fail; // maxF == 0: the line search returns lambda = 0 at once
    int backtracks;        // halvings in the current line search
    int last_backtracks;   // halvings of the previous line search
    int k_trials;          // trial slots in the current pass
    // step bookkeeping
    int skip_force;        // 1: no move this iteration (no force pass, no dots pass)
    int move_kind;         // 1: line-search step, 2: recovery step
    int dir_mode;          // 0: d = F + beta*d, 1: d = F
    int reset_after_dir;   // d.F <= 0 after the update: reset to d = F
    int copy_min_e;        // copy x to the lowest-energy backup
    int have_min_e;
    int call_limit;        // loop left because a call limit was exceeded
    // reduction tickets (last-block-done)
    unsigned int ticket_dots, ticket_dir;
    // reals
    double E_cur, E_new, prev_energy, total_energy;
    double grad_inf_norm, energy_rel_change;
    double last_fdotf, new_grad, prev_grad, beta;
    double slope, reduced_slope;
    double lam_next;       // first trial lambda of the next pass
    double lam_move;       // step taken by the pending force pass
    double dmax;           // max |d_i| of the current search direction
    double min_e;
    // quadratic line search (lineSearchAlgorithm QUADRATIC)
    int ls_quad;           // parameter: 1 = quadraticLineSearchV2 outside safe mode
    int q_mode;            // the current line search is quadraticLineSearchV2
    int q_phase;           // quadratic-optimization passes in progress
    int q_iter;            // quadratic models built in this line search
    int q_used;            // the pending step came from a quadratic optimization
    int q_pad;
    double q_x0, q_x1, q_x2, q_y0, q_y1, q_y2;  // model points (lambda, energy)
    double q_bt;           // backtracking lambda (returned when the model has no minimum)
    double q_ebt;          // its energy (TotalEnergy and newEnergy of the search)
    double q_maxe;         // largest energy of a failed trial after the first
    double q_lq;           // lambda of the pending quadratic pass
    // batched minimization: every line-search pass offers the full set of
    // trial step sizes (the batch evaluates the largest set any replica asks
    // for, so fewer trials save nothing there and cost extra rounds)
    int full_passes;
    // speculative force (single network): the first line-search pass also
    // computes the forces at the first trial step; when that step is the one
    // accepted, the iteration's force pass is skipped
    int spec_skip;         // 1: the speculative force kernels do nothing this pass
    int spec_valid;        // the speculative force of this line search was computed
    int force_skip;        // 1: the iteration's force pass does nothing
    int spec_status;       // force-pass status bits of the speculative force
    double spec_lam;       // its step (the line search's first trial)
};

}  // namespace mb

struct medyan_mech {
    int device = 0;
    int prec = 0;
    int n_beads = 0;
    cudaStream_t stream = nullptr;
    mb::Fork fork{};                      // side streams of the passes

    // standalone passes at the handle's coordinates as instantiated graphs:
    // [0] energy, [1] forces, [2] energy then forces
    cudaGraphExec_t pass_graph[3] = {nullptr, nullptr, nullptr};
    long long pass_graph_gen[3] = {-1, -1, -1};
    int pass_kernels[3] = {0, 0, 0};      // kernel nodes of each pass graph

    mb::DeviceFF ff{};
    mb::EnergyScratch es{};
    mb::ForceScratch fs{};
    // fused passes (pass.cu): layout choice, energy rows and arrival ticket
    int pass_layout = 0;                  // 0 fused, 1 one kernel per potential group, 2 fused with streamed chain
    int deterministic = 0;                // 1: fixed-point force sums (ForceTarget::fixed)
    // energy side; the force side has its own tickets (its rows are unused)
    mb::DevBuf<double> pass_rows, pass_group_rows;
    mb::DevBuf<unsigned int> pass_group_ticket, pass_ticket, pass_fgroup_ticket;
    mb::PassScratch pass_scratch() const {
        return mb::PassScratch{pass_rows.raw(), pass_group_rows.raw(), pass_group_ticket.raw(), pass_ticket.raw()};
    }
    mb::PassScratch pass_scratch_forces() const {
        return mb::PassScratch{nullptr, nullptr, pass_fgroup_ticket.raw(), pass_ticket.raw() + 1};
    }

    // internal bead order (chain.cu), fixed at create: internal position p
    // holds the caller's bead order_host[p]; pos_host is the inverse.
    // Coordinates, forces and all bead offsets on the device are internal.
    std::vector<int> order_host, pos_host;
    bool identity_order = true;
    mb::DevBuf<int> order;       // device copy of order_host (empty when identity)
    mb::DevBuf<int> pos_dev;     // device copy of pos_host (device packing)
    mb::DevBuf<unsigned char> vec_stage;  // the caller's arrays during device packing
    int host_packing = 0;        // 1: the next update packs records with the host loops
    mb::DevBuf<double> stage;    // 3*n_beads staging for reordered transfers

    // filament chains (chain.cu)
    mb::ChainDev chain{};
    mb::DevBuf<unsigned char> chain_flags;
    mb::DevBuf<double2> chain_link_p, chain_bend_p;

    // interaction i of the caller's stretching / bending arrays -> chain
    // position p (>= 0) or leftover record q (encoded -1 - q); used by the
    // parameter gradients (diff.cu), which report in the caller's order
    int n_stretch_in = 0, n_bend_in = 0;
    mb::DevBuf<int> stretch_map, bend_map;
    // Hessian-vector product scratch (diff.cu)
    mb::DevBuf<double> hv_v, hv_a, hv_b, hv_lam, pg_k, pg_p;

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
    mb::DevBuf<double> e_stage;
    mb::DevBuf<unsigned int> e_ticket;
    mb::DevBuf<mb::LambdaSet> lam_zero;

    // conjugate gradient (cg.cu)
    mb::DevBuf<double> cg_dir, cg_force2, cg_min_coords, cg_part, cg_eout;
    mb::DevBuf<mb::CGState> cg_state;
    mb::DevBuf<mb::LambdaSet> cg_lam;
    cudaGraphExec_t cg_graph = nullptr;   // instantiated minimization graph
    // pinned host staging of a minimization's inputs and results, so that
    // enqueueing it never waits on the device (batched minimization)
    unsigned char* cg_pinned = nullptr;
    size_t cg_pinned_bytes = 0;
    // pinned landing area for the per-call results the host reads back
    // (energies, force status), so their copies are asynchronous
    struct SmallPinned {
        double energy[MEDYAN_FF_COUNT + 1];
        int force_status;
    }* small = nullptr;
    int cg_graph_prec = -1;
    long long cg_graph_gen = -1;          // ff_gen the graph was captured with
    long long ff_gen = 0;                 // bumped whenever DeviceFF changes

    // neighbor list (nl.cu)
    struct NL;
    NL* nl = nullptr;

    // asynchronous evaluations (async.cu): copy streams, staging slots and
    // their events, created by the first medyan_mech_evaluate_async
    mb::medyan_async* async = nullptr;

    medyan_status init();
    ~medyan_mech();
};

namespace mb {
medyan_status cuda_status(cudaError_t e);
medyan_status validate_system(const medyan_system* s);
medyan_status upload_system(medyan_mech* h, const medyan_system* s);
medyan_status upload_system_device(medyan_mech* h, const medyan_system* s);
medyan_status refresh_device_ff(medyan_mech* h);
medyan_status sync_status(medyan_mech* h);
void enqueue_energy(medyan_mech* h, const double* x, const double* d, const LambdaSet* lam, cudaStream_t s);
void enqueue_forces(medyan_mech* h, const double* x, double* f, cudaStream_t s);
// The handle's force pass into target t (the minimizer's force pass), in
// the handle's pass layout.
void enqueue_force_target(medyan_mech* h, const double* x, const ForceTarget& t, const ForceScratch& fs,
                          cudaStream_t s);
// Energy (kPassEnergy), forces (kPassForces) or both at h->x into h->es.out /
// h->f, launched as the handle's graph for that pass (rebuilt when the force
// fields change).
constexpr int kPassEnergy = 0, kPassForces = 1, kPassBoth = 2;
cudaError_t launch_pass(medyan_mech* h, int which);
// Host coordinates/forces (caller's bead order) to and from internal device
// arrays; stream-ordered on s (the host buffer must stay valid until s syncs).
cudaError_t coords_to_device(medyan_mech* h, const double* host, double* dev, cudaStream_t s);
// A minimization in two halves (cg.cu): enqueue everything on the handle's
// stream without waiting, then wait and copy the results out.
medyan_status cg_enqueue(medyan_mech* h, const medyan_cg_params* p, const double* coord_in);
medyan_status cg_collect(medyan_mech* h, double* coord_out, double* force_out, medyan_min_result* out);
cudaError_t coords_to_host(medyan_mech* h, const double* dev, double* host, cudaStream_t s);
void destroy_nl(medyan_mech* h);
void destroy_async(medyan_mech* h);
}  // namespace mb

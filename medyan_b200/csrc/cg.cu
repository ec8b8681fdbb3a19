// cg.cu — the conjugate-gradient minimizer on the device.
//
// CGMethod::minimize (src/Mechanics/Minimizer/CGMethod.hpp:826-1743) with its
// backtracking line search (:238-373), safe mode and MController's recovery
// step (src/Controller/MController.h:273-339). Every scalar of the method
// (lambda, beta, the dot products, counters and flags) lives in a device
// CGState; single-thread logic runs in the last block of each vector pass or in
// a one-thread kernel, so an iteration never waits on the host.
//
// One iteration:
//   line-search passes: energy at up to kMaxLambda step sizes lam_k = lam*2^-k
//     from one read of x and d, then `decide` replays the reference's
//     sequential Armijo loop over them (so the accepted lambda and the energy
//     call count are the reference's);
//   force pass at x + lam*d into the force buffer that does not hold the
//     current force, unless the first line-search pass already computed
//     those forces (speculatively, at its first trial step, when the
//     previous line search took its first trial) and lam is that step;
//   dots pass: commit x += lam*d, F.F, F.Fprev, max|F|;
//     its last block computes beta (PR: max(0, (F.F - F.Fprev)/lastF.F));
//   direction pass: d = F + beta*d (or F), d.F, max|d|; its last block checks
//     d.F <= 0 (reset), convergence and call limits, and prepares the next
//     line search;
//   reset pass (only when flagged): d = F.
// Energy at the start of a line search is the accepted energy of the
// previous one (same coordinates, same deterministic reduction); it is
// counted as an energy call as in the reference.
//
// The iteration runs as a CUDA graph whose loops are conditional WHILE nodes
// (line-search passes inside, iterations outside) and whose force pass sits
// under a conditional IF node, so a whole minimization is one graph launch.
// The host only reads the result.
#include <cstring>
#include <vector>

#include "device_math.cuh"
#include "handle.h"
#include "pbatch.h"

namespace mb {

namespace {

constexpr int kVecThreads = 256;
constexpr double kLambdaTol = 1e-8;      // CGMethod::LAMBDATOL (double build)
constexpr double kBacktrackSlope = 0.4;  // CGMethod::BACKTRACKSLOPE
constexpr double kLambdaQuadTol = 1e-3;   // CGMethod::LAMBDAQUADTOL
constexpr int kQuadMaxModels = 100;       // bound on quadraticoptimization's loop
constexpr int kOut = MEDYAN_FF_COUNT + 1;

int vec_blocks(int n3) {
    int b = (n3 + kVecThreads - 1) / kVecThreads;
    if (b > 148 * 8) b = 148 * 8;
    return b < 1 ? 1 : b;
}

// ---------------------------------------------------------------- scalars
__device__ __forceinline__ double dmin_ref(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }  // std::max

__device__ void fill_pass(CGState& s, LambdaSet& L) {
    int k = 0;
    if (s.need_e0) L.lam[k++] = 0.0;
    const int want = (s.ls_first_pass && !s.full_passes) ? max(1, s.last_backtracks + 1) : kMaxLambda;
    double lam = s.lam_next;
    int trials = 0;
    while (k < kMaxLambda && trials < want) {
        L.lam[k++] = lam;
        ++trials;
        lam *= 0.5;
        if (lam <= 0.0 || lam <= kLambdaTol) break;  // a further trial would already be a failure
    }
    L.K = k;
    s.k_trials = trials;
}

// Start of a line search (CGMethod.hpp:1316-1324 and :238-262).
__device__ void begin_line_search(CGState& s, LambdaSet& L) {
    s.num_iter++;
    s.ls_active = 1;
    s.ls_first_pass = 1;
    s.backtracks = 0;
    s.skip_force = 1;
    s.move_kind = 0;
    s.reduced_slope = (s.safe_mode ? 0.0 : kBacktrackSlope) * s.slope;
    // QUADRATIC: quadraticLineSearchV2, except in safe mode (CGMethod.hpp:1322-1324)
    s.q_mode = s.ls_quad && !s.safe_mode;
    s.q_phase = 0;
    s.q_maxe = -__builtin_inf();
    s.spec_skip = 1;
    s.spec_valid = 0;
    if (s.grad_inf_norm == 0.0) {  // "return zero if no forces": lambda 0, no energy call
        s.ls_immediate_fail = 1;
        L.K = 0;
        return;
    }
    s.lam_next = dmin_ref(s.lambda_max, s.max_dist / s.grad_inf_norm);
    // speculative force at the first trial, when the previous line search
    // took its first trial (read only by the single-network minimizer)
    if (s.last_backtracks == 0) {
        s.spec_lam = s.lam_next;
        s.spec_skip = 0;
        s.spec_valid = 1;
        s.spec_status = 0;
    }
    fill_pass(s, L);
}

// Line search returned lambda = 0 (CGMethod.hpp:1337-1367).
__device__ void line_search_failed(CGState& s) {
    if (!s.try_to_recover) {
        s.error_flags |= 1;
        s.status = MEDYAN_ERR_LINE_SEARCH;
        s.done = 1;
        s.skip_force = 1;
        return;
    }
    if (s.safe_mode) {
        // funcRecoveryOnError: step = min over coordinates of maxDist/|d_i|
        // = maxDist / max|d_i| (division is monotone), then reset, safe mode off.
        if (!(s.dmax > 0.0)) {
            s.status = MEDYAN_ERR_NONFINITE;  // the reference throws "Invalid step size"
            s.done = 1;
            s.skip_force = 1;
            return;
        }
        s.lam_move = s.max_dist / s.dmax;
        s.move_kind = 2;
        s.skip_force = 0;
    } else {
        s.skip_force = 1;  // resetCGParams, safe mode on; no new force needed
        s.move_kind = 0;
        s.dir_mode = 1;
        s.safe_mode = 1;
    }
}

// End of a quadratic line search with step lq (CGMethod.hpp:637-649):
// lambda = 0 below LAMBDATOL; TotalEnergy and newEnergy stay the
// backtracking energy. The energy at the new point is evaluated at the start
// of the next line search (need_e0), since lq was not the accepted trial.
__device__ void quad_finish(CGState& s, LambdaSet& L, double lq) {
    const double lam = (lq <= 0.0 || lq <= kLambdaTol) ? 0.0 : lq;
    s.q_phase = 0;
    s.ls_active = 0;
    s.last_backtracks = s.backtracks;
    L.K = 0;
    s.total_energy = lam > 0 ? s.q_ebt : s.E_cur;
    if (lam == 0.0) {
        line_search_failed(s);
        return;
    }
    s.lam_move = lam;
    s.E_new = s.q_ebt;
    s.move_kind = 1;
    s.skip_force = 0;
    s.q_used = 1;
}

// One model of quadraticoptimization (CGMethod.hpp:662-714): the parabola
// through (x0,y0), (x1,y1), (x2,y2) and its vertex lq; either the search ends
// or the next pass evaluates E(x + lq*d). The reference's loop has no bound;
// after kQuadMaxModels models it returns x1 here.
__device__ void quad_model(CGState& s, LambdaSet& L) {
    if (s.q_iter >= kQuadMaxModels) {
        quad_finish(s, L, s.q_x1);
        return;
    }
    s.q_iter++;
    const double x0 = s.q_x0, x1 = s.q_x1, x2 = s.q_x2, y0 = s.q_y0, y1 = s.q_y1, y2 = s.q_y2;
    const double d = __dmul_rn(__dmul_rn(__dsub_rn(x0, x1), __dsub_rn(x0, x2)), __dsub_rn(x1, x2));
    const double a = __dadd_rn(__dsub_rn(__dmul_rn(y0, __dsub_rn(x1, x2)), __dmul_rn(y1, __dsub_rn(x0, x2))),
                               __dmul_rn(y2, __dsub_rn(x0, x1)));
    const double t0 = __dmul_rn(__dmul_rn(y0, __dadd_rn(x1, x2)), __dsub_rn(x1, x2));
    const double t1 = __dmul_rn(__dmul_rn(y1, __dadd_rn(x0, x2)), __dsub_rn(x0, x2));
    const double t2 = __dmul_rn(__dmul_rn(y2, __dadd_rn(x0, x1)), __dsub_rn(x0, x1));
    const double b = -__dadd_rn(__dsub_rn(t0, t1), t2);
    const double lq = -b / __dmul_rn(2.0, a);
    if (fabs(__dsub_rn(lq, x1)) / x1 < kLambdaQuadTol) {  // lambda converged
        quad_finish(s, L, lq);
        return;
    }
    if (a / d < 0) {  // no minimum: the backtracking lambda
        quad_finish(s, L, s.q_bt);
        return;
    }
    s.q_lq = lq;
    L.K = 1;
    L.lam[0] = lq;
    s.k_trials = 1;
}

// Energy at the pending quadratic point (CGMethod.hpp:716-763): accept, or
// replace one of the three points and build the next model.
__device__ void quad_eval(CGState& s, LambdaSet& L, double eq) {
    s.num_energy_call++;
    const double lq = s.q_lq, x1 = s.q_x1, y1 = s.q_y1;
    if (fabs(__dsub_rn(eq, y1)) / y1 < kLambdaQuadTol) {
        quad_finish(s, L, lq);
        return;
    }
    if (lq < x1) {
        if (eq < s.q_y0 && eq < y1) {
            s.q_x1 = lq;
            s.q_y1 = eq;
        } else {
            s.q_x0 = lq;
            s.q_y0 = eq;
        }
    } else if (x1 < lq) {
        if (eq < y1 && eq < s.q_y2) {
            s.q_x1 = lq;
            s.q_y1 = eq;
        } else {
            s.q_x2 = lq;
            s.q_y2 = eq;
        }
    } else {  // "Lambda out of range": the previous model's x1
        quad_finish(s, L, x1);
        return;
    }
    quad_model(s, L);
}

// After an energy pass: the reference's backtracking loop over the evaluated
// trial lambdas (CGMethod.hpp:264-362), or the backtracking phase of
// quadraticLineSearchV2 (:564-629) with its trial history, or one
// quadratic-optimization point.
__device__ void ls_decide(CGState& s, LambdaSet& Lr, const double* __restrict__ out) {
    LambdaSet* L = &Lr;
    s.reset_after_dir = 0;
    if (s.done || !s.ls_active) {
        L->K = 0;
        return;
    }
    if (s.ls_immediate_fail) {
        s.ls_immediate_fail = 0;
        s.ls_active = 0;
        s.last_backtracks = 0;
        line_search_failed(s);
        L->K = 0;
        return;
    }
    int slot = 0;
    if (s.need_e0) {
        s.E_cur = out[kOut - 1];
        s.need_e0 = 0;
        slot = 1;
    }
    if (s.q_phase) {
        quad_eval(s, *L, out[kOut - 1]);
        return;
    }
    if (s.ls_first_pass) {
        s.num_energy_call++;  // currentEnergy = energyFunc(coord)
        s.ls_first_pass = 0;
    }
    for (; slot < L->K; ++slot) {
        double lam = L->lam[slot];
        double E_lam = out[slot * kOut + kOut - 1];
        s.num_energy_call++;
        // idealEnergyChange: -(slope*d.F)*lambda (backtracking), -slope*lambda*d.F (V2)
        const double ideal = s.q_mode ? (-kBacktrackSlope * lam) * s.slope : -s.reduced_slope * lam;
        bool decided = false;
        if (lam < 0 || ideal > 0) {  // V2 exits the program here; both end with lambda = 0
            decided = true;
            lam = 0.0;
        }
        const double dE = E_lam - s.E_cur;
        if (dE <= ideal) decided = true;
        else {
            if (s.q_mode) {  // lambdavec/energyvec: the first trial, and the failed ones after it
                if (s.backtracks == 0) {
                    s.q_x2 = lam;
                    s.q_y2 = E_lam;
                } else if (E_lam > s.q_maxe) {
                    s.q_maxe = E_lam;
                }
            }
            lam *= 0.5;
        }
        if (lam <= 0.0 || lam <= kLambdaTol) {
            decided = true;
            lam = 0.0;
            E_lam = s.E_cur;
        }
        if (decided) {
            s.total_energy = E_lam;
            s.ls_active = 0;
            s.last_backtracks = s.backtracks;
            L->K = 0;
            if (lam == 0.0) {
                line_search_failed(s);
            } else if (s.q_mode && s.backtracks > 0 && E_lam < s.E_cur && s.q_maxe > E_lam) {
                // quadratic optimization through (0, E0), (lambda, E), (first lambda, its E)
                s.ls_active = 1;
                s.q_phase = 1;
                s.q_iter = 0;
                s.q_x0 = 0.0;
                s.q_y0 = s.E_cur;
                s.q_x1 = lam;
                s.q_y1 = E_lam;
                s.q_bt = lam;
                s.q_ebt = E_lam;
                quad_model(s, *L);
            } else {
                s.lam_move = lam;
                s.E_new = E_lam;
                s.move_kind = 1;
                s.skip_force = 0;
            }
            return;
        }
        s.backtracks++;
        s.lam_next = lam;
    }
    fill_pass(s, *L);  // undecided: evaluate the next halvings
}

// Single network: the decision, then the speculative force. The first pass
// of a line search also computed the forces at its first trial step; when
// the line search ends on a move by exactly that step, those forces (already
// in the new-force buffer) are the ones the force pass would compute, so it
// is skipped and their status bits count as its own.
// It also sets the line-search loop's condition (another round?) and, when
// the line search ends, the condition of the force pass (its kernels also
// check force_skip themselves).
__global__ void k_ls_decide(CGState* __restrict__ st, LambdaSet* __restrict__ L, const double* __restrict__ out,
                            int* __restrict__ force_status, cudaGraphConditionalHandle h_ls,
                            cudaGraphConditionalHandle h_force) {
    CGState& s = *st;
    ls_decide(s, *L, out);
    s.spec_skip = 1;  // later passes of this line search compute no forces
    cudaGraphSetConditional(h_ls, (!s.done && s.ls_active) ? 1u : 0u);
    if (s.ls_active) return;
    s.force_skip = s.skip_force;
    if (s.spec_valid && !s.skip_force && s.lam_move == s.spec_lam) {
        s.force_skip = 1;
        *force_status |= s.spec_status;
    }
    s.spec_valid = 0;
    cudaGraphSetConditional(h_force, (s.force_skip || s.done) ? 0u : 1u);
}

// ----------------------------------------------------------- vector passes
__device__ __forceinline__ void block_reduce3(double& a, double& b, double& m, double* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        m = dmax_ref(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    if (lane == 0) {
        sm[warp] = a;
        sm[32 + warp] = b;
        sm[64 + warp] = m;
    }
    __syncthreads();
    if (warp == 0) {
        a = lane < nw ? sm[lane] : 0.0;
        b = lane < nw ? sm[32 + lane] : 0.0;
        m = lane < nw ? sm[64 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
            m = dmax_ref(m, __shfl_down_sync(0xffffffffu, m, o));
        }
    }
    __syncthreads();
}

// Returns true in exactly one block: the last to finish. Each block's
// partials are stored by its thread 0, whose acquire-release ticket publishes
// them; the last block's threads see every block's partials after the
// barrier that follows its ticket.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) last = ticket_add(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    return last;
}

// Sums the per-block partials in block order (deterministic).
__device__ void reduce_partials(const double* __restrict__ part, int nblk, double& a, double& b, double& m,
                                double* sm) {
    a = 0.0;
    b = 0.0;
    m = 0.0;
    for (int q = threadIdx.x; q < nblk; q += blockDim.x) {
        a += __ldcg(part + 4 * q);
        b += __ldcg(part + 4 * q + 1);
        m = dmax_ref(m, __ldcg(part + 4 * q + 2));
    }
    block_reduce3(a, b, m, sm);
}

// Scalar part of the dots pass (one thread): F.F = a, F.Fprev = b, max|F| = m.
__device__ void dots_tail(CGState& s, double a, double b, double m) {
    s.num_force_call++;
    s.grad_inf_norm = m;  // maxF (CGMethod.hpp:202-212)
    if (isinf(m)) {
        s.status = MEDYAN_ERR_NONFINITE;  // "maxF is infinity"
        s.done = 1;
    }
    s.new_grad = a;
    s.prev_grad = b;
    if (s.move_kind == 1) {
        s.energy_rel_change = fabs(s.E_new - s.prev_energy) / fabs(s.prev_energy);
        s.prev_energy = s.E_new;
        s.E_cur = s.E_new;
        s.need_e0 = s.q_used;  // a quadratic step moved to a point whose energy is not known
        s.q_used = 0;
        if (s.method == MEDYAN_CG_POLAK_RIBIERE) s.beta = dmax_ref(0.0, (s.new_grad - s.prev_grad) / s.last_fdotf);
        else if (s.method == MEDYAN_CG_FLETCHER_RIEVES) s.beta = s.new_grad / s.last_fdotf;
        else s.beta = 0.0;
        s.dir_mode = 0;
        // copycoordsifminimumE (CGMethod.hpp:1564-1566)
        s.copy_min_e = 0;
        if (m <= 10 * s.grad_tol && s.num_iter > s.force_call_limit / 2 && s.total_energy <= s.min_e) {
            s.min_e = s.total_energy;
            s.copy_min_e = 1;
            s.have_min_e = 1;
        }
    } else {
        // setup (move_kind 0) or recovery step (2): resetCGParams follows
        if (s.move_kind == 2) {
            s.need_e0 = 1;
            s.safe_mode = 0;
        }
        s.dir_mode = 1;
        s.copy_min_e = 0;
    }
    s.parity ^= 1;
    s.skip_force = 1;
}

// dots pass: commit the move, F.F, F.Fprev, max|F|.
__global__ void __launch_bounds__(kVecThreads) k_cg_dots(int n3, double* __restrict__ x, const double* __restrict__ d,
                                                         double* __restrict__ f0, double* __restrict__ f1,
                                                         CGState* __restrict__ st, double* __restrict__ part) {
    __shared__ double sm[96];
    if (st->done || st->skip_force) return;
    const int parity = st->parity;
    const double* __restrict__ Fn = parity ? f0 : f1;  // new force (written by the force pass)
    const double* __restrict__ Fo = parity ? f1 : f0;  // force at the previous point
    const double lam = st->lam_move;
    double a = 0.0, b = 0.0, m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        x[i] = move1(x[i], lam, d[i]);
        const double fn = Fn[i], fo = Fo[i];
        a += fn * fn;
        b += fn * fo;
        m = dmax_ref(m, fabs(fn));
    }
    block_reduce3(a, b, m, sm);
    if (threadIdx.x == 0) {
        part[4 * blockIdx.x] = a;
        part[4 * blockIdx.x + 1] = b;
        part[4 * blockIdx.x + 2] = m;
    }
    if (!last_block(&st->ticket_dots)) return;
    reduce_partials(part, gridDim.x, a, b, m, sm);
    if (threadIdx.x != 0) return;
    st->ticket_dots = 0;
    dots_tail(*st, a, b, m);
}

// Scalar part of the direction pass (one thread): d.F = a, max|d| = m.
__device__ void dir_tail(CGState& s, LambdaSet& L, double a, double m) {
    s.copy_min_e = 0;
    s.dmax = m;
    if (s.dir_mode == 0 && a <= 0) {
        // conjugacy lost: resetCGParams (d = F; its d.F is F.F)
        s.reset_after_dir = 1;
        s.slope = s.new_grad;
        s.dmax = s.grad_inf_norm;
    } else {
        s.slope = a;
    }
    if (s.method != MEDYAN_CG_STEEPEST) s.last_fdotf = s.new_grad;
    s.dir_mode = 0;
    // loop condition (CGMethod.hpp:1279-1282)
    const bool limit = (s.energy_call_limit != 0 && s.num_energy_call > s.energy_call_limit) ||
                       (s.force_call_limit != 0 && s.num_force_call > s.force_call_limit);
    const bool conv = s.grad_inf_norm < s.grad_tol || s.energy_rel_change < s.energy_rel_tol;
    if (limit || conv) {
        s.done = 1;
        s.call_limit = limit;
        L.K = 0;
    } else {
        begin_line_search(s, L);
    }
}

// direction pass: d = F + beta*d (dir_mode 0) or d = F + 0*d (1), d.F, max|d|.
__global__ void __launch_bounds__(kVecThreads) k_cg_dir(int n3, const double* __restrict__ x, double* __restrict__ d,
                                                        const double* __restrict__ f0, const double* __restrict__ f1,
                                                        CGState* __restrict__ st, double* __restrict__ part,
                                                        double* __restrict__ min_e, LambdaSet* __restrict__ L) {
    __shared__ double sm[96];
    if (st->done || st->ls_active) return;
    const double* __restrict__ F = st->parity ? f1 : f0;
    const double beta = st->dir_mode ? 0.0 : st->beta;
    const bool copy = st->copy_min_e;
    double a = 0.0, b = 0.0, m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        const double fi = F[i];
        const double dn = fi + beta * d[i];  // shiftSearchDir (CGMethod.cpp:356-360)
        d[i] = dn;
        a += dn * fi;
        m = dmax_ref(m, fabs(dn));
        if (copy) min_e[i] = x[i];
    }
    block_reduce3(a, b, m, sm);
    if (threadIdx.x == 0) {
        part[4 * blockIdx.x] = a;
        part[4 * blockIdx.x + 1] = 0.0;
        part[4 * blockIdx.x + 2] = m;
    }
    if (!last_block(&st->ticket_dir)) return;
    reduce_partials(part, gridDim.x, a, b, m, sm);
    if (threadIdx.x != 0) return;
    st->ticket_dir = 0;
    dir_tail(*st, *L, a, m);
}

// In the loop graph (cond_iter set) the kernel also sets the iteration
// loop's condition.
__global__ void __launch_bounds__(kVecThreads) k_cg_reset_dir(int n3, double* __restrict__ d,
                                                              const double* __restrict__ f0,
                                                              const double* __restrict__ f1,
                                                              const CGState* __restrict__ st, int cond_iter,
                                                              cudaGraphConditionalHandle h_iter) {
    if (cond_iter && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_iter, st->done ? 0u : 1u);
    if (!st->reset_after_dir) return;
    const double* __restrict__ F = st->parity ? f1 : f0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
        d[i] = F[i] + 0.0 * d[i];
}

// energiesBefore / energiesAfter from a standalone energy pass.
__global__ void k_cg_record_energy(CGState* __restrict__ st, const double* __restrict__ out,
                                   double* __restrict__ dst, int before) {
    CGState& s = *st;
    double tot = 0.0;
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
        dst[i] = out[i];
        tot += out[i];  // computeIndividualEnergies sums without the -1 rule
    }
    dst[MEDYAN_FF_COUNT] = tot;
    s.num_energy_call++;
    if (before) {
        s.prev_energy = tot;
        s.need_e0 = 1;
    }
}

// After the loop (MController / CGMethod epilogue): unless the line search
// failed, restore the lowest-energy coordinates when a call limit ended the
// run (copycoordsifminimumE); copy the current force into f0.
__global__ void __launch_bounds__(kVecThreads) k_cg_finalize(int n3, double* __restrict__ x,
                                                             const double* __restrict__ minE,
                                                             double* __restrict__ f0, const double* __restrict__ f1,
                                                             const CGState* __restrict__ st) {
    const bool restore = st->status != MEDYAN_ERR_LINE_SEARCH && st->call_limit && st->have_min_e;
    const bool copy_f = st->parity != 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        if (restore) x[i] = minE[i];
        if (copy_f) f0[i] = f1[i];
    }
}

// energiesAfter, recorded unless the line search failed (the reference
// returns at once then).
__global__ void k_cg_record_final(CGState* __restrict__ st, const double* __restrict__ out, double* __restrict__ dst) {
    if (st->status == MEDYAN_ERR_LINE_SEARCH) return;
    CGState& s = *st;
    double tot = 0.0;
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
        dst[i] = out[i];
        tot += out[i];
    }
    dst[MEDYAN_FF_COUNT] = tot;
    s.num_energy_call++;
}

// Arms the line-search WHILE node at the start of an iteration; later rounds
// are armed by k_ls_decide and the next iteration by k_cg_reset_dir.
__global__ void k_cond_arm_ls(const CGState* __restrict__ st, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, (!st->done && st->ls_active) ? 1u : 0u);
}

// ------------------------------------------------------------ batched form
// One block per replica for the vector passes (bead range [base[r],
// base[r+1])); one thread per replica for the scalar steps. The per-replica
// scalar logic is the single-network code above (dots_tail, dir_tail,
// ls_decide, fill_pass).
//
// Step sizes: every replica's trials in a line-search pass are lam0_r * 2^-j
// (fill_pass halves), so the energy kernels evaluate x + Lg.lam[k] * dS with
// dS = lam0_r * d per replica and Lg.lam = {1, 1/2, 1/4, 1/8} (preceded by 0
// when some replica needs E(x)): scaling by a power of two is exact, so each
// position is bitwise the reference's x + lam * d. The force pass uses
// dS = lam_move_r * d with step 1.

// Global pass plan from the replicas' lambda sets (one block).
__global__ void k_b_plan(int R, CGState* __restrict__ st, LambdaSet* __restrict__ Lr, LambdaSet* __restrict__ Lg,
                         double* __restrict__ lam0, int* __restrict__ off, int* __restrict__ act) {
    __shared__ int e0s, maxt;
    if (threadIdx.x == 0) {
        e0s = 0;
        maxt = 0;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const CGState& s = st[r];
        if (!s.done && s.ls_active && Lr[r].K > 0 && s.need_e0) atomicOr(&e0s, 1);
    }
    __syncthreads();
    const int e0 = e0s;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const CGState& s = st[r];
        LambdaSet& L = Lr[r];
        if (s.done || !s.ls_active || L.K <= 0) {
            lam0[r] = 0.0;
            off[r] = 0;
            act[r] = 0;
            continue;
        }
        act[r] = 1;
        const int ne = s.need_e0 ? 1 : 0;
        int t = L.K - ne;
        const int cap = kMaxLambda - e0;  // trial slots this pass can hold
        if (t > cap) t = cap;             // the rest follow in the next pass
        L.K = ne + t;
        lam0[r] = t > 0 ? L.lam[ne] : 0.0;
        off[r] = (e0 && !ne) ? 1 : 0;
        atomicMax(&maxt, t);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        LambdaSet g{};
        int k = 0;
        if (e0) g.lam[k++] = 0.0;
        double l = 1.0;
        for (int j = 0; j < maxt && k < kMaxLambda; ++j, l *= 0.5) g.lam[k++] = l;
        g.K = (e0 || maxt) ? k : 0;
        *Lg = g;
    }
}

// dS = lam0_r * d (line search) or lam_move_r * d (force pass), per replica.
__global__ void __launch_bounds__(kVecThreads) k_b_scale(const int* __restrict__ base, const double* __restrict__ d,
                                                         double* __restrict__ dS, const CGState* __restrict__ st,
                                                         const double* __restrict__ lam0, int force_pass,
                                                         int* __restrict__ act) {
    const int r = blockIdx.x;
    const CGState& s = st[r];
    double lam;
    if (force_pass) {
        const bool on = !(s.done || s.skip_force);
        lam = on ? s.lam_move : 0.0;
        if (threadIdx.x == 0) act[r] = on ? 1 : 0;
        if (!on) return;
    } else {
        lam = lam0[r];
        if (!act[r]) return;
    }
    const int i0 = 3 * base[r], i1 = 3 * base[r + 1];
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) dS[i] = __dmul_rn(lam, d[i]);
}

__global__ void k_b_decide(int R, CGState* __restrict__ st, LambdaSet* __restrict__ Lr,
                           const double* __restrict__ out, const int* __restrict__ off, int* __restrict__ fb_count,
                           int* __restrict__ bad) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) {
        *fb_count = 0;  // every replica's finish block has read the queue
        for (int k = 0; k < kMaxLambda; ++k) bad[k] = 0;
    }
    if (r >= R) return;
    ls_decide(st[r], Lr[r], out + ((size_t)r * kMaxLambda + off[r]) * kOut);
}

// dots pass per replica: commit the move, F.F, F.Fprev, max|F|; the new
// force becomes the current one.
__global__ void __launch_bounds__(kVecThreads) k_b_dots(const int* __restrict__ base, double* __restrict__ x,
                                                        const double* __restrict__ d, double* __restrict__ fcur,
                                                        const double* __restrict__ fnew, CGState* __restrict__ st) {
    __shared__ double sm[96];
    const int r = blockIdx.x;
    CGState& s = st[r];
    if (s.done || s.skip_force) return;
    const double lam = s.lam_move;
    double a = 0.0, b = 0.0, m = 0.0;
    const int i0 = 3 * base[r], i1 = 3 * base[r + 1];
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        x[i] = move1(x[i], lam, d[i]);
        const double fn = fnew[i], fo = fcur[i];
        a += fn * fn;
        b += fn * fo;
        m = dmax_ref(m, fabs(fn));
        fcur[i] = fn;
    }
    block_reduce3(a, b, m, sm);
    if (threadIdx.x == 0) dots_tail(s, a, b, m);
}

__global__ void __launch_bounds__(kVecThreads) k_b_dir(const int* __restrict__ base, const double* __restrict__ x,
                                                       double* __restrict__ d, const double* __restrict__ fcur,
                                                       CGState* __restrict__ st, double* __restrict__ min_e,
                                                       LambdaSet* __restrict__ Lr) {
    __shared__ double sm[96];
    const int r = blockIdx.x;
    CGState& s = st[r];
    if (s.done || s.ls_active) return;
    const double beta = s.dir_mode ? 0.0 : s.beta;
    const bool copy = s.copy_min_e;
    double a = 0.0, b = 0.0, m = 0.0;
    const int i0 = 3 * base[r], i1 = 3 * base[r + 1];
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const double fi = fcur[i];
        const double dn = fi + beta * d[i];
        d[i] = dn;
        a += dn * fi;
        m = dmax_ref(m, fabs(dn));
        if (copy) min_e[i] = x[i];
    }
    block_reduce3(a, b, m, sm);
    if (threadIdx.x == 0) dir_tail(s, Lr[r], a, m);
}

__global__ void __launch_bounds__(kVecThreads) k_b_reset(const int* __restrict__ base, double* __restrict__ d,
                                                         const double* __restrict__ fcur,
                                                         const CGState* __restrict__ st) {
    const int r = blockIdx.x;
    if (!st[r].reset_after_dir) return;
    const int i0 = 3 * base[r], i1 = 3 * base[r + 1];
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) d[i] = fcur[i] + 0.0 * d[i];
}

__global__ void k_b_act_all(int R, int* __restrict__ act) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) act[r] = 1;
}

// energiesBefore (before = 1) or energiesAfter, per replica, from slot 0.
__global__ void k_b_record(int R, CGState* __restrict__ st, const double* __restrict__ out,
                           double* __restrict__ eout, int before) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    CGState& s = st[r];
    if (!before && s.status == MEDYAN_ERR_LINE_SEARCH) return;
    const double* o = out + (size_t)r * kMaxLambda * kOut;
    double* dst = eout + ((size_t)r * 2 + (before ? 0 : 1)) * kOut;
    double tot = 0.0;
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
        dst[i] = o[i];
        tot += o[i];
    }
    dst[MEDYAN_FF_COUNT] = tot;
    s.num_energy_call++;
    if (before) {
        s.prev_energy = tot;
        s.need_e0 = 1;
    }
}

__global__ void __launch_bounds__(kVecThreads) k_b_finalize(const int* __restrict__ base, double* __restrict__ x,
                                                            const double* __restrict__ minE,
                                                            const CGState* __restrict__ st) {
    const int r = blockIdx.x;
    const CGState& s = st[r];
    if (!(s.status != MEDYAN_ERR_LINE_SEARCH && s.call_limit && s.have_min_e)) return;
    const int i0 = 3 * base[r], i1 = 3 * base[r + 1];
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) x[i] = minE[i];
}

// Loop conditions: any replica still iterating / still in a line search.
__global__ void k_b_cond(int R, const CGState* __restrict__ st, cudaGraphConditionalHandle h, int ls) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const CGState& s = st[r];
        if (!s.done && (!ls || s.ls_active)) any = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

}  // namespace

// ----------------------------------------------------------------- host side
namespace {

struct CGLaunch {
    medyan_mech* h;
    int n3, vb;
    double *x, *d, *f0, *f1, *part, *minE;
    CGState* st;
    LambdaSet* L;
    ForceTarget tgt;   // the iteration's force pass
    ForceTarget spec;  // the speculative force of a line search's first pass
    ForceScratch spec_fs;
};

CGLaunch make_launch(medyan_mech* h) {
    CGLaunch c{};
    c.h = h;
    c.n3 = 3 * h->n_beads;
    c.vb = vec_blocks(c.n3);
    c.x = h->x.raw();
    c.d = h->cg_dir.raw();
    c.f0 = h->f.raw();
    c.f1 = h->cg_force2.raw();
    c.part = h->cg_part.raw();
    c.minE = h->cg_min_coords.raw();
    c.st = h->cg_state.raw();
    c.L = h->cg_lam.raw();
    c.tgt = ForceTarget{c.f0,           c.f1, &c.st->parity, &c.st->force_skip, c.d, &c.st->lam_move,
                        h->deterministic, h->fs.status};
    c.spec = ForceTarget{c.f0,           c.f1, &c.st->parity, &c.st->spec_skip, c.d, &c.st->spec_lam,
                         h->deterministic, &c.st->spec_status};
    c.spec_fs = ForceScratch{h->fs.fb_count, h->fs.fb_list, &c.st->spec_status, h->fs.fb_cap};
    return c;
}

// Energies at the pass's trial steps; with them, in the first pass of a line
// search, the forces at its first trial step.
void enqueue_ls_pass(const CGLaunch& c, cudaStream_t s, cudaGraphConditionalHandle h_ls,
                     cudaGraphConditionalHandle h_force) {
    launch_evaluate(c.h->chain, c.h->ff, c.h->prec, c.x, c.d, c.L, c.spec, c.h->es, c.spec_fs, s, &c.h->fork);
    k_ls_decide<<<1, 1, 0, s>>>(c.st, c.L, c.h->energy_out.raw(), c.h->fs.status, h_ls, h_force);
}

void enqueue_force_pass(const CGLaunch& c, cudaStream_t s) {
    enqueue_force_target(c.h, c.x, c.tgt, c.h->fs, s);
}

// The move and its dots, the new direction. cond_iter: in the loop graph,
// where the last kernel sets the iteration condition h_iter.
void enqueue_move_and_direction(const CGLaunch& c, cudaStream_t s, int cond_iter = 0,
                                cudaGraphConditionalHandle h_iter = 0) {
    k_cg_dots<<<c.vb, kVecThreads, 0, s>>>(c.n3, c.x, c.d, c.f0, c.f1, c.st, c.part);
    k_cg_dir<<<c.vb, kVecThreads, 0, s>>>(c.n3, c.x, c.d, c.f0, c.f1, c.st, c.part, c.minE, c.L);
    k_cg_reset_dir<<<c.vb, kVecThreads, 0, s>>>(c.n3, c.d, c.f0, c.f1, c.st, cond_iter, h_iter);
}

// The force pass, then the move and the new direction.
void enqueue_step(const CGLaunch& c, cudaStream_t s) {
    enqueue_force_pass(c, s);
    enqueue_move_and_direction(c, s);
}

// Whole minimization loop as one graph:
// WHILE(iter) { arm; WHILE(ls) { pass; decide }; IF(force) { force pass }; move, direction }.
// The IF skips the force pass's launches when the line search ended without
// a move or on the step whose forces the first pass already computed.
cudaError_t build_graph(const CGLaunch& c, cudaGraphExec_t* exec) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle h_iter, h_ls, h_force;
    e = cudaGraphConditionalHandleCreate(&h_iter, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t n_iter;
    cudaGraphNodeParams p_iter = {};
    if (e == cudaSuccess) {
        p_iter.type = cudaGraphNodeTypeConditional;
        p_iter.conditional.handle = h_iter;
        p_iter.conditional.type = cudaGraphCondTypeWhile;
        p_iter.conditional.size = 1;
        e = cudaGraphAddNode(&n_iter, g, nullptr, 0, &p_iter);
    }
    cudaGraph_t body = e == cudaSuccess ? p_iter.conditional.phGraph_out[0] : nullptr;
    cudaStream_t s = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    // iteration body: arm the line-search condition, the line-search loop,
    // then the step kernels and the iteration condition
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h_ls, body, 0, 0);
    // force pass: runs unless the line search's end says otherwise
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h_force, body, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t n_arm = nullptr;
    if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            k_cond_arm_ls<<<1, 1, 0, s>>>(c.st, h_ls);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
        size_t nn = 0;
        if (e == cudaSuccess) e = cudaGraphGetNodes(body, nullptr, &nn);
        if (e == cudaSuccess && nn == 1) e = cudaGraphGetNodes(body, &n_arm, &nn);
        if (e == cudaSuccess && !n_arm) e = cudaErrorUnknown;
    }
    cudaGraphNode_t n_ls;
    cudaGraphNodeParams p_ls = {};
    if (e == cudaSuccess) {
        p_ls.type = cudaGraphNodeTypeConditional;
        p_ls.conditional.handle = h_ls;
        p_ls.conditional.type = cudaGraphCondTypeWhile;
        p_ls.conditional.size = 1;
        e = cudaGraphAddNode(&n_ls, body, &n_arm, 1, &p_ls);
    }
    if (e == cudaSuccess) {
        cudaGraph_t ls_body = p_ls.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(s, ls_body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            enqueue_ls_pass(c, s, h_ls, h_force);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
    }
    cudaGraphNode_t n_force;
    cudaGraphNodeParams p_force = {};
    if (e == cudaSuccess) {
        p_force.type = cudaGraphNodeTypeConditional;
        p_force.conditional.handle = h_force;
        p_force.conditional.type = cudaGraphCondTypeIf;
        p_force.conditional.size = 1;
        e = cudaGraphAddNode(&n_force, body, &n_ls, 1, &p_force);
    }
    if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(s, p_force.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            enqueue_force_pass(c, s);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
    }
    if (e == cudaSuccess) {
        const cudaGraphNode_t deps[1] = {n_force};
        e = cudaStreamBeginCaptureToGraph(s, body, deps, nullptr, 1, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            enqueue_move_and_direction(c, s, 1, h_iter);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (s) cudaStreamDestroy(s);
    cudaGraphDestroy(g);
    return e;
}

}  // namespace

}  // namespace mb

using namespace mb;

namespace mb {

// Enqueues a whole minimization on the handle's stream: setup, the first
// energy and force, the loop graph, the epilogue and the final energy. No
// host synchronization; cg_collect reads the results.
medyan_status cg_enqueue(medyan_mech* h, const medyan_cg_params* p, const double* coord_in) {
    if (!h || !p || !coord_in) return MEDYAN_ERR_INVALID_ARG;
    if (p->method < 0 || p->method > 2 || !(p->max_dist > 0) || !(p->lambda_max > 0) || p->line_search < 0 ||
        p->line_search > 1)
        return MEDYAN_ERR_INVALID_ARG;
    const int n3 = 3 * h->n_beads;
    cudaStream_t s = h->stream;
    cudaError_t e = h->cg_dir.reserve(n3 ? n3 : 1);
    if (e == cudaSuccess) e = h->cg_force2.reserve(n3 ? n3 : 1);
    if (e == cudaSuccess) e = h->cg_min_coords.reserve(n3 ? n3 : 1);
    if (e == cudaSuccess) e = h->cg_part.reserve(4 * (size_t)vec_blocks(n3) + 4);
    if (e == cudaSuccess) e = h->cg_eout.reserve(2 * kOut);
    if (e == cudaSuccess) e = h->cg_state.reserve(1);
    if (e == cudaSuccess) e = h->cg_lam.reserve(1);
    if (e != cudaSuccess) return cuda_status(e);
    const size_t bytes = sizeof(double) * (size_t)n3;
    // pinned staging: coordinates in, coordinates and forces out, state, lambda set
    const size_t need = 2 * bytes + sizeof(CGState) + sizeof(LambdaSet) + 64;
    if (h->cg_pinned_bytes < need) {
        if (h->cg_pinned) cudaFreeHost(h->cg_pinned);
        h->cg_pinned = nullptr;
        h->cg_pinned_bytes = 0;
        e = cudaMallocHost(reinterpret_cast<void**>(&h->cg_pinned), need);
        if (e != cudaSuccess) return cuda_status(e);
        h->cg_pinned_bytes = need;
    }
    double* px = reinterpret_cast<double*>(h->cg_pinned);
    CGState* ps = reinterpret_cast<CGState*>(h->cg_pinned + 2 * bytes);
    LambdaSet* pl = reinterpret_cast<LambdaSet*>(h->cg_pinned + 2 * bytes + sizeof(CGState));
    CGLaunch c = make_launch(h);

    CGState s0{};
    s0.method = p->method;
    s0.try_to_recover = p->try_to_recover;
    s0.energy_call_limit = p->energy_call_limit;
    s0.force_call_limit = p->force_call_limit > 3 * h->n_beads ? p->force_call_limit : 3 * h->n_beads;
    s0.max_dist = p->max_dist;
    s0.lambda_max = p->lambda_max;
    s0.grad_tol = p->grad_tol;
    s0.energy_rel_tol = p->energy_rel_tol;
    s0.ls_quad = p->line_search;
    s0.status = MEDYAN_OK;
    s0.parity = 1;  // the first force lands in f0
    s0.grad_inf_norm = __builtin_inf();
    s0.energy_rel_change = __builtin_inf();
    s0.min_e = __builtin_inf();
    s0.lam_move = 0.0;
    s0.skip_force = 0;
    s0.force_skip = 0;
    s0.spec_skip = 1;
    s0.move_kind = 0;
    LambdaSet l0{};
    if (n3) std::memcpy(px, coord_in, bytes);
    *ps = s0;
    *pl = l0;
    e = coords_to_device(h, px, c.x, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c.st, ps, sizeof s0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c.L, pl, sizeof l0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d, 0, bytes ? bytes : 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.f0, 0, bytes ? bytes : 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.f1, 0, bytes ? bytes : 8, s);
    if (e != cudaSuccess) return cuda_status(e);

    // energiesBefore, then the first force (parity 1 -> f0), F.F, d = F.
    enqueue_energy(h, c.x, nullptr, h->lam_zero.raw(), s);
    k_cg_record_energy<<<1, 1, 0, s>>>(c.st, h->energy_out.raw(), h->cg_eout.raw(), 1);
    enqueue_step(c, s);

    // main loop: one graph launch
    // the graph captures the force-field records by value: rebuild it after
    // any re-vectorization (generation counter) or precision change
    if (h->cg_graph && (h->cg_graph_gen != h->ff_gen || h->cg_graph_prec != h->prec)) {
        cudaGraphExecDestroy(h->cg_graph);
        h->cg_graph = nullptr;
    }
    if (!h->cg_graph) {
        e = build_graph(c, &h->cg_graph);
        if (e != cudaSuccess) return cuda_status(e);
        h->cg_graph_gen = h->ff_gen;
        h->cg_graph_prec = h->prec;
    }
    e = cudaGraphLaunch(h->cg_graph, s);
    if (e != cudaSuccess) return cuda_status(e);

    // epilogue and energiesAfter, on the device
    k_cg_finalize<<<c.vb, kVecThreads, 0, s>>>(n3, c.x, c.minE, c.f0, c.f1, c.st);
    enqueue_energy(h, c.x, nullptr, h->lam_zero.raw(), s);
    k_cg_record_final<<<1, 1, 0, s>>>(c.st, h->energy_out.raw(), h->cg_eout.raw() + kOut);
    return cuda_status(cudaGetLastError());
}

// Waits for the handle's minimization and copies its results out.
medyan_status cg_collect(medyan_mech* h, double* coord_out, double* force_out, medyan_min_result* out) {
    cudaStream_t s = h->stream;
    const size_t bytes = sizeof(double) * 3 * (size_t)h->n_beads;
    double* px = reinterpret_cast<double*>(h->cg_pinned);
    double* pf = reinterpret_cast<double*>(h->cg_pinned + bytes);
    CGState* ps = reinterpret_cast<CGState*>(h->cg_pinned + 2 * bytes);
    cudaError_t e = coords_to_host(h, h->x.raw(), px, s);
    if (e == cudaSuccess && force_out) e = coords_to_host(h, h->f.raw(), pf, s);
    if (e != cudaSuccess) return cuda_status(e);
    double eo[2 * kOut];
    e = cudaMemcpyAsync(ps, h->cg_state.raw(), sizeof(CGState), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    const CGState sf = *ps;
    e = cudaMemcpy(eo, h->cg_eout.raw(), sizeof eo, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e);
    if (bytes) std::memcpy(coord_out, px, bytes);
    if (force_out && bytes) std::memcpy(force_out, pf, bytes);
    if (out) {
        std::memset(out, 0, sizeof *out);
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
            out->energy_before[i] = eo[i];
            out->energy_after[i] = sf.status == MEDYAN_ERR_LINE_SEARCH ? 0.0 : eo[kOut + i];
        }
        out->energy_before_total = eo[MEDYAN_FF_COUNT];
        out->energy_after_total = sf.status == MEDYAN_ERR_LINE_SEARCH ? 0.0 : eo[kOut + MEDYAN_FF_COUNT];
        out->error_flags = (uint32_t)sf.error_flags;
        out->num_energy_call = sf.num_energy_call;
        out->energy_call_limit = sf.energy_call_limit;
        out->num_force_call = sf.num_force_call;
        out->force_call_limit = sf.force_call_limit;
        out->num_iter = sf.num_iter;
        out->grad_inf_norm = sf.grad_inf_norm;
        out->grad_tol = sf.grad_tol;
        out->energy_rel_change = sf.energy_rel_change;
        out->energy_rel_tol = sf.energy_rel_tol;
    }
    return (medyan_status)sf.status;
}

namespace {

void b_energy_pass(PackedBatch& pb, const double* dS, const LambdaSet* L, cudaStream_t s) {
    launch_energy_producers(pb.ch, pb.ff, pb.x.raw(), dS, L, pb.es, s, &pb.fork, pb.chain_table.raw(),
                            pb.n_chain_blocks);
    launch_energy_finish_batched(pb.ff, pb.x.raw(), dS, L, pb.es, pb.rows_chain(), pb.rows_seg(), pb.rows_excl(),
                                 pb.excl_pairs(), pb.R, pb.out.raw(), s);
}

void b_step(PackedBatch& pb, int prec, cudaStream_t s) {
    const int R = pb.R;
    k_b_scale<<<R, kVecThreads, 0, s>>>(pb.base_dev.raw(), pb.d.raw(), pb.dS.raw(), pb.st.raw(), pb.lam0.raw(), 1,
                                        pb.act.raw());
    const ForceTarget t{pb.fnew.raw(), nullptr, nullptr, nullptr, pb.dS.raw(), pb.one.raw(), pb.deterministic ? 1 : 0,
                        pb.fs.status};
    launch_forces(pb.ch, pb.ff, prec, pb.x.raw(), t, pb.fs, s, &pb.fork);
    k_b_dots<<<R, kVecThreads, 0, s>>>(pb.base_dev.raw(), pb.x.raw(), pb.d.raw(), pb.fcur.raw(), pb.fnew.raw(),
                                       pb.st.raw());
    k_b_dir<<<R, kVecThreads, 0, s>>>(pb.base_dev.raw(), pb.x.raw(), pb.d.raw(), pb.fcur.raw(), pb.st.raw(),
                                      pb.minE.raw(), pb.Lr.raw());
    k_b_reset<<<R, kVecThreads, 0, s>>>(pb.base_dev.raw(), pb.d.raw(), pb.fcur.raw(), pb.st.raw());
}

void b_ls_pass(PackedBatch& pb, cudaStream_t s) {
    const int R = pb.R;
    k_b_plan<<<1, 256, 0, s>>>(R, pb.st.raw(), pb.Lr.raw(), pb.Lg.raw(), pb.lam0.raw(), pb.off.raw(), pb.act.raw());
    k_b_scale<<<R, kVecThreads, 0, s>>>(pb.base_dev.raw(), pb.d.raw(), pb.dS.raw(), pb.st.raw(), pb.lam0.raw(), 0,
                                        pb.act.raw());
    b_energy_pass(pb, pb.dS.raw(), pb.Lg.raw(), s);
    k_b_decide<<<(R + 127) / 128, 128, 0, s>>>(R, pb.st.raw(), pb.Lr.raw(), pb.out.raw(), pb.off.raw(),
                                               pb.es.fb_count, pb.es.bad);
}

// WHILE(any replica iterating) { WHILE(any replica in a line search) { pass }; step }
cudaError_t b_build_graph(PackedBatch& pb, int prec, cudaGraphExec_t* exec) {
    const int R = pb.R;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle h_iter, h_ls;
    e = cudaGraphConditionalHandleCreate(&h_iter, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t n_iter;
    cudaGraphNodeParams p_iter = {};
    if (e == cudaSuccess) {
        p_iter.type = cudaGraphNodeTypeConditional;
        p_iter.conditional.handle = h_iter;
        p_iter.conditional.type = cudaGraphCondTypeWhile;
        p_iter.conditional.size = 1;
        e = cudaGraphAddNode(&n_iter, g, nullptr, 0, &p_iter);
    }
    cudaGraph_t body = e == cudaSuccess ? p_iter.conditional.phGraph_out[0] : nullptr;
    cudaStream_t s = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h_ls, body, 0, 0);
    cudaGraphNode_t n_arm = nullptr;
    if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            k_b_cond<<<1, 256, 0, s>>>(R, pb.st.raw(), h_ls, 1);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
        size_t nn = 0;
        if (e == cudaSuccess) e = cudaGraphGetNodes(body, nullptr, &nn);
        if (e == cudaSuccess && nn == 1) e = cudaGraphGetNodes(body, &n_arm, &nn);
        if (e == cudaSuccess && !n_arm) e = cudaErrorUnknown;
    }
    cudaGraphNode_t n_ls;
    cudaGraphNodeParams p_ls = {};
    if (e == cudaSuccess) {
        p_ls.type = cudaGraphNodeTypeConditional;
        p_ls.conditional.handle = h_ls;
        p_ls.conditional.type = cudaGraphCondTypeWhile;
        p_ls.conditional.size = 1;
        e = cudaGraphAddNode(&n_ls, body, &n_arm, 1, &p_ls);
    }
    if (e == cudaSuccess) {
        cudaGraph_t ls_body = p_ls.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(s, ls_body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            b_ls_pass(pb, s);
            k_b_cond<<<1, 256, 0, s>>>(R, pb.st.raw(), h_ls, 1);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
    }
    if (e == cudaSuccess) {
        const cudaGraphNode_t deps[1] = {n_ls};
        e = cudaStreamBeginCaptureToGraph(s, body, deps, nullptr, 1, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            b_step(pb, prec, s);
            k_b_cond<<<1, 256, 0, s>>>(R, pb.st.raw(), h_iter, 0);
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(s, &tmp);
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (s) cudaStreamDestroy(s);
    cudaGraphDestroy(g);
    return e;
}

}  // namespace

medyan_status cg_batch_time_evaluate(PackedBatch& pb, int prec, int reps, float* ms) {
    const int R = pb.R;
    if (R == 0 || reps <= 0) return MEDYAN_ERR_INVALID_ARG;
    const size_t n3 = 3 * (size_t)pb.nb;
    cudaStream_t s = pb.stream;
    cudaError_t e = pb.fnew.reserve(n3 ? n3 : 1);
    if (e == cudaSuccess) e = pb.out.reserve((size_t)R * kMaxLambda * kOut);
    LambdaSet z{};
    z.K = 1;
    if (e == cudaSuccess) e = pb.Lzero.assign(&z, 1, s);
    if (e != cudaSuccess) return cuda_status(e);
    const ForceTarget t{pb.fnew.raw(), nullptr, nullptr, nullptr, nullptr, nullptr, pb.deterministic ? 1 : 0,
                        pb.fs.status};
    auto pass = [&] {
        b_energy_pass(pb, nullptr, pb.Lzero.raw(), s);
        // the CG's decide step clears the fallback queue; do it here
        cudaMemsetAsync(pb.es.fb_count, 0, sizeof(int), s);
        cudaMemsetAsync(pb.es.bad, 0, sizeof(int) * kMaxLambda, s);
        launch_forces(pb.ch, pb.ff, prec, pb.x.raw(), t, pb.fs, s, &pb.fork);
    };
    k_b_act_all<<<(R + 255) / 256, 256, 0, s>>>(R, pb.act.raw());
    pass();
    pass();
    cudaEvent_t a = nullptr, b = nullptr;
    e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaEventRecord(a, s);
    for (int i = 0; i < reps && e == cudaSuccess; ++i) {
        pass();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(b, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float t_ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t_ms, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.fs.status, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    *ms = t_ms / (float)reps;
    return MEDYAN_OK;
}

// Batched CGMethod::minimize over the packed replicas; see the kernels above.
medyan_status cg_batch_run(PackedBatch& pb, int prec, const medyan_cg_params* p) {
    const int R = pb.R;
    if (!p || p->method < 0 || p->method > 2 || !(p->max_dist > 0) || !(p->lambda_max > 0) || p->line_search < 0 ||
        p->line_search > 1)
        return MEDYAN_ERR_INVALID_ARG;
    if (R == 0) return MEDYAN_OK;
    const size_t n3 = 3 * (size_t)pb.nb;
    cudaStream_t s = pb.stream;
    cudaError_t e = cudaSuccess;
    for (DevBuf<double>* b : {&pb.d, &pb.dS, &pb.fcur, &pb.fnew, &pb.minE})
        if (e == cudaSuccess) e = b->reserve(n3 ? n3 : 1);
    if (e == cudaSuccess) e = pb.out.reserve((size_t)R * kMaxLambda * kOut);
    if (e == cudaSuccess) e = pb.eout.reserve((size_t)R * 2 * kOut);
    if (e == cudaSuccess) e = pb.st.reserve(R);
    if (e == cudaSuccess) e = pb.Lr.reserve(R);
    if (e == cudaSuccess) e = pb.Lg.reserve(1);
    if (e == cudaSuccess) e = pb.Lzero.reserve(1);
    if (e == cudaSuccess) e = pb.lam0.reserve(R);
    if (e == cudaSuccess) e = pb.off.reserve(R);
    if (e == cudaSuccess) e = pb.one.reserve(1);
    if (e != cudaSuccess) return cuda_status(e);

    std::vector<CGState> s0(R);
    for (int r = 0; r < R; ++r) {
        CGState& c = s0[r];
        c = CGState{};
        const int nbr = pb.base[r + 1] - pb.base[r];
        c.method = p->method;
        c.try_to_recover = p->try_to_recover;
        c.energy_call_limit = p->energy_call_limit;
        c.force_call_limit = p->force_call_limit > 3 * nbr ? p->force_call_limit : 3 * nbr;
        c.max_dist = p->max_dist;
        c.lambda_max = p->lambda_max;
        c.grad_tol = p->grad_tol;
        c.energy_rel_tol = p->energy_rel_tol;
        c.ls_quad = p->line_search;
        c.full_passes = 1;
        c.status = MEDYAN_OK;
        c.parity = 1;
        c.grad_inf_norm = __builtin_inf();
        c.energy_rel_change = __builtin_inf();
        c.min_e = __builtin_inf();
    }
    LambdaSet z{};
    z.K = 1;
    const double one = 1.0;
    const size_t bytes = sizeof(double) * n3;
    e = pb.st.assign(s0.data(), R, s);
    if (e == cudaSuccess) e = pb.Lzero.assign(&z, 1, s);
    if (e == cudaSuccess) e = pb.one.assign(&one, 1, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.Lr.raw(), 0, sizeof(LambdaSet) * R, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.d.raw(), 0, bytes ? bytes : 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.fcur.raw(), 0, bytes ? bytes : 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.fnew.raw(), 0, bytes ? bytes : 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(pb.fs.status, 0, sizeof(int), s);
    if (e != cudaSuccess) return cuda_status(e);

    // energiesBefore, then the first force, F.F, d = F
    k_b_act_all<<<(R + 255) / 256, 256, 0, s>>>(R, pb.act.raw());
    b_energy_pass(pb, nullptr, pb.Lzero.raw(), s);
    k_b_decide<<<1, 1, 0, s>>>(0, pb.st.raw(), pb.Lr.raw(), pb.out.raw(), pb.off.raw(), pb.es.fb_count, pb.es.bad);
    k_b_record<<<(R + 127) / 128, 128, 0, s>>>(R, pb.st.raw(), pb.out.raw(), pb.eout.raw(), 1);
    b_step(pb, prec, s);

    if (pb.graph && (pb.graph_gen != pb.gen || pb.graph_prec != prec || pb.graph_det != pb.deterministic)) {
        cudaGraphExecDestroy(pb.graph);
        pb.graph = nullptr;
    }
    if (!pb.graph) {
        e = b_build_graph(pb, prec, &pb.graph);
        if (e != cudaSuccess) return cuda_status(e);
        pb.graph_gen = pb.gen;
        pb.graph_prec = prec;
        pb.graph_det = pb.deterministic;
    }
    e = cudaGraphLaunch(pb.graph, s);
    if (e != cudaSuccess) return cuda_status(e);

    // epilogue and energiesAfter
    k_b_finalize<<<R, kVecThreads, 0, s>>>(pb.base_dev.raw(), pb.x.raw(), pb.minE.raw(), pb.st.raw());
    k_b_act_all<<<(R + 255) / 256, 256, 0, s>>>(R, pb.act.raw());
    b_energy_pass(pb, nullptr, pb.Lzero.raw(), s);
    k_b_decide<<<1, 1, 0, s>>>(0, pb.st.raw(), pb.Lr.raw(), pb.out.raw(), pb.off.raw(), pb.es.fb_count, pb.es.bad);
    k_b_record<<<(R + 127) / 128, 128, 0, s>>>(R, pb.st.raw(), pb.out.raw(), pb.eout.raw(), 0);
    return cuda_status(cudaGetLastError());
}

}  // namespace mb

extern "C" medyan_status medyan_cg_minimize(medyan_mech* h, const medyan_cg_params* p, double* coord_inout,
                                            double* force_out, medyan_min_result* out) {
    medyan_status st = cg_enqueue(h, p, coord_inout);
    if (st != MEDYAN_OK) return st;
    return cg_collect(h, coord_inout, force_out, out);
}

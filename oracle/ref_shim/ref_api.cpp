// ref_api.cpp — C entry points over the reference's own potential and
// conjugate-gradient sources, compiled from the reference tree with stand-in
// headers (see oracle/Makefile, target `ref`). This is test infrastructure: it
// lets the oracle restatement and the CUDA kernels be checked against the
// reference's compiled code on identical inputs, and it is the CPU baseline
// for the reference benchmark arm. Nothing in the product links it.
//
// The per-force-field loop restates ForceFieldManager::computeEnergy /
// computeForces (src/Mechanics/ForceField/ForceFieldManager.cpp:96-290):
// energies are summed in force-field order and any force-field energy <= -1
// makes the total +inf; forces are zero-filled and then accumulated.
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

#include "ref_stub_counts.h"
#include "BoundaryElement.h"
#include "Bead.h"

#include "Mechanics/ForceField/Filament/FilamentStretchingHarmonic.h"
#include "Mechanics/ForceField/Filament/FilamentBendingCosine.h"
#include "Mechanics/ForceField/Linker/LinkerStretchingHarmonic.h"
#include "Mechanics/ForceField/MotorGhost/MotorGhostStretchingHarmonic.h"
#include "Mechanics/ForceField/Branching/BranchingStretchingHarmonic.h"
#include "Mechanics/ForceField/Branching/BranchingBendingCosine.h"
#include "Mechanics/ForceField/Branching/BranchingDihedralCosine.h"
#include "Mechanics/ForceField/Branching/BranchingPositionCosine.h"
#include "Mechanics/ForceField/Volume/CylinderExclVolRepulsion.h"
#include "Mechanics/ForceField/Boundary/BoundaryCylinderRepulsionExp.h"
#include "Mechanics/Minimizer/CGMethod.hpp"

#include "medyan_b200.h"

using namespace medyan;

namespace {

// Mutable copies of the caller's arrays: the reference kernels take
// non-const pointers (and the dihedral/position kernels unsigned bead sets).
struct RefSystem {
    medyan_system s{};
    std::vector<int> st_b, be_b, li_b, mo_b, br3_b, br4_b, ex_b, bd_b, bd_nn;
    std::vector<unsigned> br4_u, br3_u;
    std::vector<double> st_k, st_l, be_k, be_t, li_k, li_l, li_p1, li_p2, mo_k, mo_l, mo_p1, mo_p2;
    std::vector<double> br_p, bs_k, bs_l, bb_k, bb_t, bdh_k, bp_k, ex_k, ex_l, bd_k, bd_s;
    std::vector<BoundaryElement> planes;
    std::vector<double> stretchforce;
    CylinderExclVolRepulsion excl;

    template <class T> static std::vector<T> cp(const T* p, long n) {
        return p && n > 0 ? std::vector<T>(p, p + n) : std::vector<T>();
    }

    explicit RefSystem(const medyan_system* in) : s(*in) {
        st_b = cp(in->stretch_beads, 2L * in->n_stretch);
        st_k = cp(in->stretch_k, in->n_stretch); st_l = cp(in->stretch_l0, in->n_stretch);
        be_b = cp(in->bend_beads, 3L * in->n_bend);
        be_k = cp(in->bend_k, in->n_bend); be_t = cp(in->bend_theta0, in->n_bend);
        li_b = cp(in->linker_beads, 4L * in->n_linker);
        li_k = cp(in->linker_k, in->n_linker); li_l = cp(in->linker_l0, in->n_linker);
        li_p1 = cp(in->linker_pos1, in->n_linker); li_p2 = cp(in->linker_pos2, in->n_linker);
        mo_b = cp(in->motor_beads, 4L * in->n_motor);
        mo_k = cp(in->motor_k, in->n_motor); mo_l = cp(in->motor_l0, in->n_motor);
        mo_p1 = cp(in->motor_pos1, in->n_motor); mo_p2 = cp(in->motor_pos2, in->n_motor);
        const long nb = in->n_branch;
        br4_b = cp(in->branch_beads, 4L * nb);
        br3_b.resize(3 * nb);
        for (long i = 0; i < nb; ++i)
            for (int k = 0; k < 3; ++k) br3_b[3 * i + k] = br4_b[4 * i + k];
        br4_u.assign(br4_b.begin(), br4_b.end());
        br3_u.assign(br3_b.begin(), br3_b.end());
        br_p = cp(in->branch_pos, nb);
        bs_k = cp(in->branch_stretch_k, nb); bs_l = cp(in->branch_stretch_l0, nb);
        bb_k = cp(in->branch_bend_k, nb); bb_t = cp(in->branch_bend_theta0, nb);
        bdh_k = cp(in->branch_dihedral_k, nb); bp_k = cp(in->branch_position_k, nb);
        ex_b = cp(in->excl_beads, 4L * in->n_excl);
        ex_k = cp(in->excl_k, in->n_excl); ex_l = cp(in->excl_eqlen, 2L * in->n_excl);
        bd_b = cp(in->boundary_beads, in->n_boundary);
        bd_k = cp(in->boundary_k, in->n_boundary); bd_s = cp(in->boundary_slen, in->n_boundary);
        bd_nn = cp(in->plane_nneighbors, in->n_planes);
        planes.resize(in->n_planes);
        for (int p = 0; p < in->n_planes; ++p) {
            planes[p].a = in->plane_eq[4 * p + 0];
            planes[p].b = in->plane_eq[4 * p + 1];
            planes[p].c = in->plane_eq[4 * p + 2];
            planes[p].d = in->plane_eq[4 * p + 3];
        }
        long nsf = std::max<long>({(long)in->n_linker, (long)in->n_motor, 3 * nb, 1L});
        stretchforce.assign(nsf, 0.0);
    }

    void bind_globals() {
        RefCounts::cylinders = s.n_stretch;
        RefCounts::linkers = s.n_linker;
        RefCounts::motors = s.n_motor;
        RefCounts::branches = s.n_branch;
        Bead::count = s.n_beads;
        auto& el = BoundaryElement::getBoundaryElements();
        el.clear();
        for (auto& p : planes) el.push_back(&p);
    }

    bool has_branch(int bit) const { return s.n_branch > 0 && (s.branch_ff_mask >> bit & 1); }

    // Per-force-field energies in MEDYAN_FF_* order; returns the manager total.
    double energy(const double* coord_in, double* e) {
        bind_globals();
        double* coord = const_cast<double*>(coord_in);
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) e[i] = 0.0;
        if (s.n_stretch) e[0] = FilamentStretchingHarmonic{}.energy(coord, st_b.data(), st_k.data(), st_l.data());
        if (s.n_bend) e[1] = FilamentBendingCosine{}.energy(coord, s.n_bend, be_b.data(), be_k.data(), be_t.data());
        if (s.n_linker) e[2] = LinkerStretchingHarmonic{}.energy(coord, li_b.data(), li_k.data(), li_l.data(), li_p1.data(), li_p2.data());
        if (s.n_motor) e[3] = MotorGhostStretchingHarmonic{}.energy(coord, mo_b.data(), mo_k.data(), mo_l.data(), mo_p1.data(), mo_p2.data());
        if (has_branch(0)) e[4] = BranchingStretchingHarmonic{}.energy(coord, br3_b.data(), bs_k.data(), bs_l.data(), br_p.data());
        if (has_branch(1)) e[5] = BranchingBendingCosine{}.energy(coord, br4_b.data(), bb_k.data(), bb_t.data());
        if (has_branch(2)) e[6] = BranchingDihedralCosine{}.energy(coord, s.n_branch, br4_u.data(), bdh_k.data(), br_p.data());
        if (has_branch(3)) e[7] = BranchingPositionCosine{}.energy(coord, br3_u.data(), bp_k.data(), br_p.data());
        if (s.n_excl) e[8] = excl.energy(coord, ex_b.data(), ex_k.data(), ex_l.data(), s.n_excl);
        if (s.n_boundary) e[9] = BoundaryCylinderRepulsionExp{}.energy(coord, bd_b.data(), bd_k.data(), bd_s.data(), bd_nn.data());
        double total = 0.0;
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
            if (e[i] <= -1) return std::numeric_limits<double>::infinity();
            total += e[i];
        }
        return total;
    }

    void forces(const double* coord_in, double* f) {
        bind_globals();
        double* coord = const_cast<double*>(coord_in);
        std::memset(f, 0, sizeof(double) * 3 * (size_t)s.n_beads);
        double* sf = stretchforce.data();
        if (s.n_stretch) FilamentStretchingHarmonic{}.forces(coord, f, st_b.data(), st_k.data(), st_l.data());
        if (s.n_bend) FilamentBendingCosine{}.forces(coord, f, s.n_bend, be_b.data(), be_k.data(), be_t.data());
        if (s.n_linker) LinkerStretchingHarmonic{}.forces(coord, f, li_b.data(), li_k.data(), li_l.data(), li_p1.data(), li_p2.data(), sf);
        if (s.n_motor) MotorGhostStretchingHarmonic{}.forces(coord, f, mo_b.data(), mo_k.data(), mo_l.data(), mo_p1.data(), mo_p2.data(), sf);
        if (has_branch(0)) BranchingStretchingHarmonic{}.forces(coord, f, br3_b.data(), bs_k.data(), bs_l.data(), br_p.data(), sf);
        if (has_branch(1)) BranchingBendingCosine{}.forces(coord, f, br4_b.data(), bb_k.data(), bb_t.data(), sf);
        if (has_branch(2)) BranchingDihedralCosine{}.forces(coord, f, s.n_branch, br4_u.data(), bdh_k.data(), br_p.data(), sf);
        if (has_branch(3)) BranchingPositionCosine{}.forces(coord, f, br3_u.data(), bp_k.data(), br_p.data(), sf);
        if (s.n_excl) excl.forces(coord, f, ex_b.data(), ex_k.data(), ex_l.data(), s.n_excl);
        if (s.n_boundary) BoundaryCylinderRepulsionExp{}.forces(coord, f, bd_b.data(), bd_k.data(), bd_s.data(), bd_nn.data());
    }
};

void fill_report(const EnergyReport& r, double* per, double* total) {
    for (int i = 0; i < MEDYAN_FF_COUNT; ++i) per[i] = 0.0;
    for (size_t i = 0; i < r.individual.size() && i < MEDYAN_FF_COUNT; ++i) per[i] = r.individual[i].energy;
    *total = r.total;
}

}  // namespace

extern "C" {

double medyan_ref_energy(const medyan_system* sys, const double* coord, double* e_per_ff) {
    RefSystem r(sys);
    double tmp[MEDYAN_FF_COUNT];
    return r.energy(coord, e_per_ff ? e_per_ff : tmp);
}

void medyan_ref_forces(const medyan_system* sys, const double* coord, double* force) {
    RefSystem r(sys);
    r.forces(coord, force);
}

// Repeated evaluation on one prepared system (CPU baseline timing).
void* medyan_ref_prepare(const medyan_system* sys) { return new RefSystem(sys); }
void medyan_ref_release(void* h) { delete static_cast<RefSystem*>(h); }
double medyan_ref_prepared_energy(void* h, const double* coord, double* e_per_ff) {
    double tmp[MEDYAN_FF_COUNT];
    return static_cast<RefSystem*>(h)->energy(coord, e_per_ff ? e_per_ff : tmp);
}
void medyan_ref_prepared_forces(void* h, const double* coord, double* force) {
    static_cast<RefSystem*>(h)->forces(coord, force);
}

// CGMethod::minimize from the reference sources, driven by the reference
// potentials. The recovery callback restates MController::
// moveAlongDirectionLimitingBeadMove_ (src/Controller/MController.h:273-339)
// for a bead-only system: step = min over all coordinates of
// maxDist/|dir_i|, then coord += step*dir over the DOF.
// ConjugateGradientParams::lambdaRunningAverageProbability of the next
// medyan_ref_cg_minimize calls (0 unless set), to exercise the reference's
// LambdaRunningAverageManager (Mechanics/Minimizer/LineSearch.hpp:21-48).
static double g_lambda_avg_probability = 0.0;
extern "C" void medyan_ref_set_lambda_running_average(double probability) {
    g_lambda_avg_probability = probability;
}

int medyan_ref_cg_minimize(const medyan_system* sys, const medyan_cg_params* p, double* coord_io,
                           double* force_out, medyan_min_result* out) {
    RefSystem r(sys);
    const int ndof = 3 * sys->n_beads;
    std::vector<floatingpoint> coord(coord_io, coord_io + ndof);
    std::vector<floatingpoint> force;

    ConjugateGradientParams cg;
    cg.descentSearchMethod = p->method == 0 ? ConjugateGradientDescentSearch::steepest
                             : p->method == 1 ? ConjugateGradientDescentSearch::fletcherRieves
                                              : ConjugateGradientDescentSearch::polakRibiere;
    cg.maxDist = p->max_dist;
    cg.lambdaMax = p->lambda_max;
    cg.gradTol = p->grad_tol;
    cg.energyRelTol = p->energy_rel_tol;
    cg.energyCallLimit = p->energy_call_limit;
    cg.forceCallLimit = p->force_call_limit;
    cg.tryToRecoverInLineSearchError = p->try_to_recover != 0;
    cg.lineSearchAlgorithm = p->line_search ? "QUADRATIC" : "BACKTRACKING";
    cg.reportOnCallLimit = true;
    cg.lambdaRunningAverageProbability = g_lambda_avg_probability;

    const auto energyFunc = [&](floatingpoint* c) {
        double e[MEDYAN_FF_COUNT];
        return r.energy(c, e);
    };
    const auto forceFunc = [&](floatingpoint* c, floatingpoint* f, int) { r.forces(c, f); };
    const auto energyFuncIndividual = [&](floatingpoint* c) {
        double e[MEDYAN_FF_COUNT];
        EnergyReport rep;
        rep.total = 0.0;
        r.energy(c, e);
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
            rep.individual.push_back({"", e[i]});
            rep.total += e[i];
        }
        return rep;
    };
    const double maxDist = p->max_dist;
    const auto recovery = [&](std::vector<floatingpoint>& c, const std::vector<floatingpoint>& dir) {
        double step = std::numeric_limits<double>::infinity();
        for (int i = 0; i < ndof; ++i) step = std::min(step, maxDist / std::abs(dir[i]));
        if (step == std::numeric_limits<double>::infinity()) throw std::runtime_error("Invalid step size.");
        for (int i = 0; i < ndof; ++i) c[i] += step * dir[i];
    };

    CGMethod method;
    MinimizationResult res;
    try {
        res = method.minimize(cg, coord, ndof, energyFunc, forceFunc, energyFuncIndividual, recovery, &force);
    } catch (const std::exception&) {
        return MEDYAN_ERR_NONFINITE;
    }
    std::copy(coord.begin(), coord.begin() + ndof, coord_io);
    // a failed line search returns before minimize fills outForce
    if (force_out && (int)force.size() >= ndof) std::copy(force.begin(), force.begin() + ndof, force_out);
    if (out) {
        fill_report(res.energiesBefore, out->energy_before, &out->energy_before_total);
        fill_report(res.energiesAfter, out->energy_after, &out->energy_after_total);
        out->error_flags = (uint32_t)res.errorFlags;
        out->num_energy_call = res.numEnergyCall;
        out->energy_call_limit = res.energyCallLimit;
        out->num_force_call = res.numForceCall;
        out->force_call_limit = res.forceCallLimit;
        out->num_iter = -1;
        out->grad_inf_norm = res.gradInfNorm;
        out->grad_tol = res.gradTol;
        out->energy_rel_change = res.energyRelChange;
        out->energy_rel_tol = res.energyRelTol;
    }
    return res.errorFlags ? MEDYAN_ERR_LINE_SEARCH : MEDYAN_OK;
}

// CGMethod::minimize from the reference sources driven by C callbacks
// (energy, forces, per-force-field energies), as the reference's own
// TestCGMethod drives it with plain lambdas.
typedef double (*ref_energy_fn)(void* ctx, const double* x);
typedef void (*ref_force_fn)(void* ctx, const double* x, double* f);
typedef void (*ref_individual_fn)(void* ctx, const double* x, double* per);

int medyan_ref_cg_minimize_cb(int ndof, int n_beads, const medyan_cg_params* p, double* coord_io, double* force_out,
                              medyan_min_result* out, ref_energy_fn efn, ref_force_fn ffn, ref_individual_fn ifn,
                              void* ctx) {
    Bead::count = n_beads;
    std::vector<floatingpoint> coord(coord_io, coord_io + ndof);
    std::vector<floatingpoint> force;
    ConjugateGradientParams cg;
    cg.descentSearchMethod = p->method == 0 ? ConjugateGradientDescentSearch::steepest
                             : p->method == 1 ? ConjugateGradientDescentSearch::fletcherRieves
                                              : ConjugateGradientDescentSearch::polakRibiere;
    cg.maxDist = p->max_dist;
    cg.lambdaMax = p->lambda_max;
    cg.gradTol = p->grad_tol;
    cg.energyRelTol = p->energy_rel_tol;
    cg.energyCallLimit = p->energy_call_limit;
    cg.forceCallLimit = p->force_call_limit;
    cg.tryToRecoverInLineSearchError = p->try_to_recover != 0;
    cg.lineSearchAlgorithm = p->line_search ? "QUADRATIC" : "BACKTRACKING";
    const auto energyFunc = [&](floatingpoint* c) { return efn(ctx, c); };
    const auto forceFunc = [&](floatingpoint* c, floatingpoint* f, int) { ffn(ctx, c, f); };
    const auto energyFuncIndividual = [&](floatingpoint* c) {
        double e[MEDYAN_FF_COUNT] = {0};
        ifn(ctx, c, e);
        EnergyReport rep;
        rep.total = 0.0;
        for (int i = 0; i < MEDYAN_FF_COUNT; ++i) {
            rep.individual.push_back({"", e[i]});
            rep.total += e[i];
        }
        return rep;
    };
    const double maxDist = p->max_dist;
    const auto recovery = [&](std::vector<floatingpoint>& c, const std::vector<floatingpoint>& dir) {
        double step = std::numeric_limits<double>::infinity();
        for (int i = 0; i < ndof; ++i) step = std::min(step, maxDist / std::abs(dir[i]));
        if (step == std::numeric_limits<double>::infinity()) throw std::runtime_error("Invalid step size.");
        for (int i = 0; i < ndof; ++i) c[i] += step * dir[i];
    };
    CGMethod method;
    MinimizationResult res;
    try {
        res = method.minimize(cg, coord, ndof, energyFunc, forceFunc, energyFuncIndividual, recovery, &force);
    } catch (const std::exception&) {
        return MEDYAN_ERR_NONFINITE;
    }
    std::copy(coord.begin(), coord.begin() + ndof, coord_io);
    // a failed line search returns before minimize fills outForce
    if (force_out && (int)force.size() >= ndof) std::copy(force.begin(), force.begin() + ndof, force_out);
    if (out) {
        fill_report(res.energiesBefore, out->energy_before, &out->energy_before_total);
        fill_report(res.energiesAfter, out->energy_after, &out->energy_after_total);
        out->error_flags = (uint32_t)res.errorFlags;
        out->num_energy_call = res.numEnergyCall;
        out->energy_call_limit = res.energyCallLimit;
        out->num_force_call = res.numForceCall;
        out->force_call_limit = res.forceCallLimit;
        out->num_iter = -1;
        out->grad_inf_norm = res.gradInfNorm;
        out->grad_tol = res.gradTol;
        out->energy_rel_change = res.energyRelChange;
        out->energy_rel_tol = res.energyRelTol;
    }
    return res.errorFlags ? MEDYAN_ERR_LINE_SEARCH : MEDYAN_OK;
}

}  // extern "C"

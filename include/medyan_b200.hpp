// medyan_b200.hpp — C++ drop-in layer over the C ABI (medyan_b200.h).
//
// It mirrors the reference's C++ interfaces for the mechanical-equilibration
// path, so that MEDYAN's MController can hold this manager where it holds
// its ForceFieldManager and call this CGMethod where it calls its own:
//   - EnergyReport            src/Mechanics/ForceField/Types.hpp:24-33
//   - ConjugateGradientParams src/Mechanics/Minimizer/CGMethod.hpp:44-63
//   - MinimizationResult      src/Mechanics/Minimizer/MinimizationTypes.hpp:10-64
//   - ForceFieldManager       src/Mechanics/ForceField/ForceFieldManager.h/.cpp
//                             (vectorizeAllForceFields :35-93, computeEnergy
//                             :96-207, computeIndividualEnergies :209-240,
//                             computeForces :242-290)
//   - CGMethod::minimize      src/Mechanics/Minimizer/CGMethod.hpp:826-836
//   - neighbor-list reset     src/Structure/HybridNeighborListImpl.cpp:332-471
//                             via SubSystem::resetNeighborLists
//
// Error behaviour follows the reference: computeEnergy returns +inf when a
// force field reports its error value (ForceFieldManager.cpp:150-161) and
// lets a NaN term through as the reference does; a failed
// line search is reported in MinimizationResult::errorFlags, not thrown.
// Everything else the library reports (bad arguments, index range, CUDA
// errors, no device) throws medyan_b200::Error. No arithmetic happens on the
// host: without a GPU the constructor throws.
#pragma once

#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "medyan_b200.h"

namespace medyan_b200 {

class Error : public std::runtime_error {
public:
    Error(medyan_status s, const std::string& what)
        : std::runtime_error(what + ": " + medyan_status_string(s) + cuda_detail(s)), status(s) {}
    medyan_status status;

private:
    static std::string cuda_detail(medyan_status s) {
        if (s != MEDYAN_ERR_CUDA && s != MEDYAN_ERR_NO_DEVICE) return "";
        return std::string(" [") + medyan_last_cuda_error() + "]";
    }
};

inline void check(medyan_status s, const char* what) {
    if (s != MEDYAN_OK) throw Error(s, what);
}

inline const char* force_field_name(int slot) {
    static const char* names[MEDYAN_FF_COUNT] = {
        "FilamentStretching", "FilamentBending",   "LinkerStretching",  "MotorGhostStretching",
        "BranchingStretching", "BranchingBending", "BranchingDihedral", "BranchingPosition",
        "CylinderExcludedVolume", "BoundaryRepulsion"};
    return names[slot];
}

struct EnergyReport {
    struct EachEnergy {
        std::string name;
        double energy;
    };
    double total = 0.0;
    std::vector<EachEnergy> individual;
};

enum class ConjugateGradientDescentSearch { steepest, fletcherRieves, polakRibiere };

struct ConjugateGradientParams {
    ConjugateGradientDescentSearch descentSearchMethod = ConjugateGradientDescentSearch::polakRibiere;
    double maxDist = 1.0;
    double lambdaMax = 0.01;
    double lambdaRunningAverageProbability = 0.0;  // accepted in [0, 1]; no effect, as in the reference
    std::string lineSearchAlgorithm = "BACKTRACKING";  // BACKTRACKING, or QUADRATIC (any other value, as in the reference)
    double gradTol = 1e-1;
    double energyRelTol = 1e-9;
    int energyCallLimit = 0;
    int forceCallLimit = 10000;
    bool reportOnCallLimit = true;
    bool tryToRecoverInLineSearchError = true;
};

struct MinimizationResult {
    static constexpr std::uint_fast32_t errorLineSearch = 1 << 0;

    EnergyReport energiesBefore;
    EnergyReport energiesAfter;
    std::uint_fast32_t errorFlags = 0;
    int numEnergyCall = 0;
    int energyCallLimit = 0;
    int numForceCall = 0;
    int forceCallLimit = 0;
    int numCGMethodCall = 0;
    int numIter = 0;  // CG iterations (not in the reference struct)
    double gradInfNorm = std::numeric_limits<double>::infinity();
    double gradTol = 0;
    double energyRelChange = std::numeric_limits<double>::infinity();
    double energyRelTol = 0;

    void updateWithMinimizationResult(const MinimizationResult& res) {
        if (numCGMethodCall == 0) energiesBefore = res.energiesBefore;
        energiesAfter = res.energiesAfter;
        errorFlags |= res.errorFlags;
        numEnergyCall += res.numEnergyCall;
        energyCallLimit += res.energyCallLimit;
        numForceCall += res.numForceCall;
        forceCallLimit += res.forceCallLimit;
        numIter += res.numIter;
        ++numCGMethodCall;
        gradInfNorm = res.gradInfNorm;
        gradTol = res.gradTol;
        energyRelChange = res.energyRelChange;
        energyRelTol = res.energyRelTol;
    }
    bool success() const { return errorFlags == 0; }
    bool callLimitExceeded() const {
        return (energyCallLimit != 0 && numEnergyCall > energyCallLimit) ||
               (forceCallLimit != 0 && numForceCall > forceCallLimit);
    }
    bool gradInfNormConverged() const { return gradInfNorm < gradTol; }
    bool energyRelChangeConverged() const { return energyRelChange < energyRelTol; }
    bool converged() const { return gradInfNormConverged() || energyRelChangeConverged(); }
};

inline EnergyReport make_report(const double* per, double total) {
    EnergyReport r;
    r.total = total;
    for (int s = 0; s < MEDYAN_FF_COUNT; ++s) r.individual.push_back({force_field_name(s), per[s]});
    return r;
}

// The force fields of one network on one GPU (one handle, one CUDA stream;
// not thread-safe, like the reference's manager).
class ForceFieldManager {
public:
    explicit ForceFieldManager(medyan_precision precision = MEDYAN_PREC_FP64) : precision_(precision) {}
    ~ForceFieldManager() {
        if (h_) medyan_mech_destroy(h_);
    }
    ForceFieldManager(const ForceFieldManager&) = delete;
    ForceFieldManager& operator=(const ForceFieldManager&) = delete;

    // The arrays every ForceField::vectorize produces, gathered in one
    // medyan_system (reference layout: bead sets hold offsets 3*bead).
    void vectorizeAllForceFields(const medyan_system& sys) {
        if (h_ && n_beads_ == sys.n_beads) {
            check(medyan_mech_update(h_, &sys), "vectorizeAllForceFields");
        } else {
            if (h_) medyan_mech_destroy(h_);
            h_ = nullptr;
            check(medyan_mech_create(&sys, precision_, &h_), "vectorizeAllForceFields");
            n_beads_ = sys.n_beads;
        }
        n_linker_ = sys.n_linker;
        n_motor_ = sys.n_motor;
        n_branch_ = sys.n_branch;
    }

    // Total energy at coord (double[3*n_beads]); +inf when a force field's
    // energy is invalid.
    double computeEnergy(const double* coord) {
        check(medyan_mech_set_coords(handle(), coord), "computeEnergy");
        double total = 0;
        medyan_status s = medyan_mech_energy(h_, &total, nullptr);
        if (s == MEDYAN_ERR_NONFINITE) return std::numeric_limits<double>::infinity();
        check(s, "computeEnergy");
        return total;
    }

    EnergyReport computeIndividualEnergies(const double* coord) {
        check(medyan_mech_set_coords(handle(), coord), "computeIndividualEnergies");
        double total = 0, per[MEDYAN_FF_COUNT];
        medyan_status s = medyan_mech_energy(h_, &total, per);
        if (s != MEDYAN_ERR_NONFINITE) check(s, "computeIndividualEnergies");
        // the reference sums the individual energies without the +inf rule
        double sum = 0;
        for (double e : per) sum += e;
        return make_report(per, sum);
    }

    // force = -dE/dx at coord; numVar = 3*n_beads.
    void computeForces(const double* coord, double* force, int numVar) {
        if (numVar != 3 * n_beads_) throw Error(MEDYAN_ERR_INVALID_ARG, "computeForces: numVar");
        check(medyan_mech_set_coords(handle(), coord), "computeForces");
        medyan_status s = medyan_mech_forces(h_, force);
        if (s != MEDYAN_ERR_NONFINITE) check(s, "computeForces");
    }

    // Cylinder topology and neighbor-list / boundary parameters for
    // resetNeighborLists.
    void setNeighborListInputs(const medyan_cylinders& cyl, const medyan_nl_params& nl,
                               const medyan_boundary_params& boundary) {
        check(medyan_mech_set_cylinders(handle(), &cyl, &nl, &boundary), "setNeighborListInputs");
    }

    // SubSystem::resetNeighborLists followed by the excluded-volume and
    // boundary vectorize steps, at the current device coordinates. Returns
    // (excluded-volume pairs, boundary terms).
    std::pair<int64_t, int64_t> resetNeighborLists() {
        int64_t ne = 0, nb = 0;
        check(medyan_mech_rebuild_neighbors(handle(), &ne, &nb), "resetNeighborLists");
        return {ne, nb};
    }

    void setCoordinates(const double* coord) { check(medyan_mech_set_coords(handle(), coord), "setCoordinates"); }

    // ForceFieldManager::computeHessian (ForceFieldManager.cpp:354-398): the
    // dense finite-difference Hessian at coord, row-major ndof x ndof, entries
    // rounded to float as the reference stores them.
    std::vector<double> computeHessian(const double* coord, float delta) {
        setCoordinates(coord);
        const size_t n = 3 * (size_t)n_beads_;
        std::vector<double> H(n * n);
        check(medyan_mech_hessian(handle(), delta, H.data()), "computeHessian");
        return H;
    }

    // The values ForceFieldManager::assignallforcemags (ForceFieldManager.cpp:346-351)
    // hands to the linkers, motors and branch points, at coord.
    struct ForceMagnitudes {
        std::vector<double> linkerStretch, motorStretch, branchForce;  // branchForce: 3 per branch point
    };
    ForceMagnitudes forceMagnitudes(const double* coord) {
        setCoordinates(coord);
        ForceMagnitudes m;
        m.linkerStretch.resize(n_linker_);
        m.motorStretch.resize(n_motor_);
        m.branchForce.resize(3 * (size_t)n_branch_);
        check(medyan_mech_force_magnitudes(handle(), m.linkerStretch.data(), m.motorStretch.data(),
                                           m.branchForce.data()),
              "forceMagnitudes");
        return m;
    }

    // BoundaryCylinderRepulsion::computeLoadForces for the given filament tips
    // (after resetNeighborLists): tip t's loadForcesP / loadForcesM vector is
    // out[o_t .. o_t + n_mon[t]), o_t the sum of the earlier tips' n_mon.
    std::vector<double> computeLoadForces(const medyan_load_tips& tips) {
        int64_t total = 0;
        for (int t = 0; t < tips.n_tips; ++t) total += tips.n_mon[t];
        std::vector<double> out((size_t)total);
        check(medyan_mech_boundary_load_forces(handle(), &tips, out.data(), total), "computeLoadForces");
        return out;
    }

    // Block and tile shapes per potential for this network (no reference
    // counterpart: the reference's kernels run on the CPU).
    medyan_launch_shapes autotune(int reps = 10) {
        medyan_launch_shapes s{};
        check(medyan_mech_autotune(handle(), reps, &s), "autotune");
        return s;
    }

    // Bitwise reproducible force sums (fixed point; medyan_mech_set_deterministic).
    void setDeterministic(bool on) { check(medyan_mech_set_deterministic(handle(), on ? 1 : 0), "setDeterministic"); }

    // Many evaluations back to back with the copies overlapped
    // (medyan_mech_evaluate_async): results land in force[i] and energy[i]
    // (MEDYAN_FF_COUNT + 1 each) by the time the call returns; page-locked
    // buffers overlap, pageable ones work.
    void evaluateMany(const std::vector<const double*>& coord, const std::vector<double*>& force,
                      const std::vector<double*>& energy) {
        if (coord.size() != force.size() || coord.size() != energy.size())
            throw Error(MEDYAN_ERR_INVALID_ARG, "evaluateMany: sizes");
        for (size_t i = 0; i < coord.size(); ++i)
            check(medyan_mech_evaluate_async(handle(), coord[i], force[i], energy[i]), "evaluateMany");
        const medyan_status st = medyan_mech_wait(handle());
        if (st != MEDYAN_OK && st != MEDYAN_ERR_NONFINITE) check(st, "evaluateMany");
    }

    int numBeads() const { return n_beads_; }
    medyan_mech* handle() const {
        if (!h_) throw Error(MEDYAN_ERR_INVALID_ARG, "vectorizeAllForceFields was not called");
        return h_;
    }

private:
    medyan_precision precision_;
    medyan_mech* h_ = nullptr;
    int n_beads_ = 0;
    int n_linker_ = 0, n_motor_ = 0, n_branch_ = 0;
};

// CGMethod::minimize over a ForceFieldManager's force fields. The reference
// takes energy/force callables; here the energy and forces are the
// manager's, evaluated on the device, and the whole loop runs there.
class CGMethod {
public:
    static MinimizationResult minimize(const ConjugateGradientParams& p, std::vector<double>& coord,
                                       ForceFieldManager& ffm, std::vector<double>* outForce = nullptr) {
        // lambdaRunningAverageProbability changes nothing in the reference:
        // CGMethod::minimize builds a new LambdaRunningAverageManager in every
        // iteration (CGMethod.hpp:1316-1317) and records one lambda into it,
        // and the manager acts only after ten records (LineSearch.hpp:33-42).
        // Any probability therefore gives the trajectory of 0 (checked on the
        // reference's compiled CGMethod in tests/test_oracle_pins.py).
        if (!(p.lambdaRunningAverageProbability >= 0.0 && p.lambdaRunningAverageProbability <= 1.0))
            throw Error(MEDYAN_ERR_INVALID_ARG, "CGMethod::minimize: lambdaRunningAverageProbability");
        if ((int)coord.size() != 3 * ffm.numBeads()) throw Error(MEDYAN_ERR_INVALID_ARG, "CGMethod::minimize: coord");
        medyan_cg_params cp{};
        cp.method = p.descentSearchMethod == ConjugateGradientDescentSearch::steepest         ? MEDYAN_CG_STEEPEST
                    : p.descentSearchMethod == ConjugateGradientDescentSearch::fletcherRieves ? MEDYAN_CG_FLETCHER_RIEVES
                                                                                             : MEDYAN_CG_POLAK_RIBIERE;
        cp.max_dist = p.maxDist;
        cp.lambda_max = p.lambdaMax;
        cp.grad_tol = p.gradTol;
        cp.energy_rel_tol = p.energyRelTol;
        cp.energy_call_limit = p.energyCallLimit;
        cp.force_call_limit = p.forceCallLimit;
        cp.try_to_recover = p.tryToRecoverInLineSearchError ? 1 : 0;
        // CGMethod.hpp:1319-1332: anything but BACKTRACKING is quadraticLineSearchV2
        cp.line_search = p.lineSearchAlgorithm == "BACKTRACKING" ? 0 : 1;
        if (outForce) outForce->resize(coord.size());
        medyan_min_result r{};
        medyan_status s = medyan_cg_minimize(ffm.handle(), &cp, coord.data(), outForce ? outForce->data() : nullptr, &r);
        if (s != MEDYAN_OK && s != MEDYAN_ERR_LINE_SEARCH) check(s, "CGMethod::minimize");
        MinimizationResult res;
        res.energiesBefore = make_report(r.energy_before, r.energy_before_total);
        res.energiesAfter = make_report(r.energy_after, r.energy_after_total);
        res.errorFlags = r.error_flags;
        res.numEnergyCall = r.num_energy_call;
        res.energyCallLimit = r.energy_call_limit;
        res.numForceCall = r.num_force_call;
        res.forceCallLimit = r.force_call_limit;
        res.numCGMethodCall = 1;
        res.numIter = r.num_iter;
        res.gradInfNorm = r.grad_inf_norm;
        res.gradTol = r.grad_tol;
        res.energyRelChange = r.energy_rel_change;
        res.energyRelTol = r.energy_rel_tol;
        return res;
    }
};

}  // namespace medyan_b200

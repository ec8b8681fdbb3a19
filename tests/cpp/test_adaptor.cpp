// Drives the C++ drop-in layer (include/medyan_b200.hpp) the way MController
// drives the reference's ForceFieldManager and CGMethod, and checks it
// against the oracle (linked here only as the checker).
//
//   test_adaptor nodevice : on a machine without a GPU, vectorizeAllForceFields
//                           must throw medyan_b200::Error (no host fallback)
//   test_adaptor gpu      : energies, individual energies, forces, the
//                           neighbor-list reset and a short minimization
//                           against the oracle
//
// Exit status 0 = pass; a failed check prints its line and exits 1.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "medyan_b200.hpp"
#include "medyan_oracle.h"

using namespace medyan_b200;

#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c); \
            return 1;                                              \
        }                                                          \
    } while (0)

namespace {

// 8 straight filaments of 6 beads (5 cylinders, 20 nm) in a 400 nm box,
// stretching + bending on every filament, linkers between filament pairs.
// Directions are tilted at random: parallel cylinders make the analytic
// excluded-volume integral ill-conditioned, and the comparison here is a
// generic one.
struct Net {
    int nb = 0;
    std::vector<double> x;
    std::vector<int32_t> sb, bb, lb;
    std::vector<double> sk, sl0, bk, bt0, lk, ll0, lp1, lp2;
    // cylinders for the neighbor list
    std::vector<int32_t> c1, c2, cid, cfil, cpos, ctype, cbranch, cminus;
    std::vector<double> ceq, cexk;

    Net() {
        std::mt19937_64 rng(7);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        const int nf = 8, nbf = 6;
        for (int f = 0; f < nf; ++f) {
            double o[3] = {100 + 40.0 * f, 120 + 5.0 * u(rng), 100 + 20.0 * (f % 3)};
            double dir[3] = {0.15 * u(rng), 1.0, 0.15 * u(rng)};
            const double m = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
            for (double& v : dir) v /= m;
            for (int b = 0; b < nbf; ++b)
                for (int k = 0; k < 3; ++k) x.push_back(o[k] + 20.0 * b * dir[k] + 0.8 * u(rng));
            const int b0 = f * nbf;
            for (int b = 0; b + 1 < nbf; ++b) {
                sb.push_back(3 * (b0 + b));
                sb.push_back(3 * (b0 + b + 1));
                sk.push_back(100.0);
                sl0.push_back(20.0);
                const int c = (int)cid.size();
                c1.push_back(b0 + b);  // bead indices
                c2.push_back(b0 + b + 1);
                cid.push_back(c);
                cfil.push_back(f);
                cpos.push_back(b);
                ctype.push_back(0);
                cbranch.push_back(-1);
                cminus.push_back(b == 0);
                ceq.push_back(20.0);
                cexk.push_back(1e5);
            }
            for (int b = 0; b + 2 < nbf; ++b) {
                bb.push_back(3 * (b0 + b));
                bb.push_back(3 * (b0 + b + 1));
                bb.push_back(3 * (b0 + b + 2));
                bk.push_back(672.0);
                bt0.push_back(0.0);
            }
        }
        nb = nf * nbf;
        for (int f = 0; f + 1 < nf; ++f) {
            const int a = f * nbf + 1, c = (f + 1) * nbf + 2;
            const int32_t q[4] = {3 * a, 3 * (a + 1), 3 * c, 3 * (c + 1)};
            for (int32_t v : q) lb.push_back(v);
            lk.push_back(8.0);
            ll0.push_back(30.0);
            lp1.push_back(0.25);
            lp2.push_back(0.75);
        }
    }

    medyan_system system() const {
        medyan_system s;
        std::memset(&s, 0, sizeof s);
        s.n_beads = nb;
        s.n_stretch = (int32_t)sk.size();
        s.stretch_beads = sb.data();
        s.stretch_k = sk.data();
        s.stretch_l0 = sl0.data();
        s.n_bend = (int32_t)bk.size();
        s.bend_beads = bb.data();
        s.bend_k = bk.data();
        s.bend_theta0 = bt0.data();
        s.n_linker = (int32_t)lk.size();
        s.linker_beads = lb.data();
        s.linker_k = lk.data();
        s.linker_l0 = ll0.data();
        s.linker_pos1 = lp1.data();
        s.linker_pos2 = lp2.data();
        return s;
    }

    medyan_cylinders cylinders() const {
        medyan_cylinders c;
        std::memset(&c, 0, sizeof c);
        c.n_cyl = (int32_t)cid.size();
        c.bead1 = c1.data();
        c.bead2 = c2.data();
        c.id = cid.data();
        c.filament_id = cfil.data();
        c.position_on_filament = cpos.data();
        c.type = ctype.data();
        c.branching_cylinder = cbranch.data();
        c.is_minus_end = cminus.data();
        c.eq_length = ceq.data();
        c.excl_k = cexk.data();
        return c;
    }
};

double rel(double a, double b) { return std::fabs(a - b) / std::fmax(std::fabs(b), 1e-300); }

double max_rel_vec(const std::vector<double>& a, const std::vector<double>& b) {
    double m = 0, s = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        m = std::fmax(m, std::fabs(a[i] - b[i]));
        s = std::fmax(s, std::fabs(b[i]));
    }
    return m / std::fmax(s, 1e-300);
}

int run_nodevice() {
    Net net;
    medyan_system s = net.system();
    ForceFieldManager ffm;
    try {
        ffm.vectorizeAllForceFields(s);
    } catch (const Error& e) {
        std::printf("threw as expected: %s\n", e.what());
        CHECK(e.status == MEDYAN_ERR_NO_DEVICE || e.status == MEDYAN_ERR_CUDA);
        return 0;
    }
    std::fprintf(stderr, "vectorizeAllForceFields succeeded without a device\n");
    return 1;
}

int run_gpu() {
    Net net;
    medyan_system s = net.system();
    const int nd = 3 * net.nb;

    ForceFieldManager ffm(MEDYAN_PREC_FP64);
    ffm.vectorizeAllForceFields(s);

    // energy and individual energies
    double per_o[MEDYAN_FF_COUNT];
    const double eo = oracle_energy(&s, net.x.data(), per_o);
    const double eg = ffm.computeEnergy(net.x.data());
    CHECK(rel(eg, eo) <= 1e-12);
    EnergyReport rep = ffm.computeIndividualEnergies(net.x.data());
    CHECK(rep.individual.size() == (size_t)MEDYAN_FF_COUNT);
    CHECK(rep.individual[0].name == "FilamentStretching");
    for (int k = 0; k < MEDYAN_FF_COUNT; ++k)
        CHECK(std::fabs(rep.individual[k].energy - per_o[k]) <= 1e-12 * std::fmax(std::fabs(per_o[k]), 1.0));

    // forces (the caller's buffer is overwritten, not accumulated into)
    std::vector<double> fo(nd, 0.0), fg(nd, 123.0);
    oracle_forces(&s, net.x.data(), fo.data());
    ffm.computeForces(net.x.data(), fg.data(), nd);
    CHECK(max_rel_vec(fg, fo) <= 1e-12);
    bool threw = false;
    try {
        ffm.computeForces(net.x.data(), fg.data(), nd - 3);
    } catch (const Error& e) {
        threw = e.status == MEDYAN_ERR_INVALID_ARG;
    }
    CHECK(threw);

    // a zero-length cylinder makes a bend energy NaN; the reference's bending
    // energy has no check (FilamentBendingCosine.cpp:199-243), so the NaN
    // reaches the total as it does in the oracle
    std::vector<double> xbad = net.x;
    for (int k = 0; k < 3; ++k) xbad[3 + k] = xbad[k];
    CHECK(std::isnan(oracle_energy(&s, xbad.data(), nullptr)));
    CHECK(std::isnan(ffm.computeEnergy(xbad.data())));

    // neighbor-list reset against the oracle's pair set size
    medyan_cylinders cyl = net.cylinders();
    medyan_nl_params nlp;
    std::memset(&nlp, 0, sizeof nlp);
    nlp.rmax = 54.0f;
    nlp.rmin = 0.0f;
    for (int d = 0; d < 3; ++d) nlp.grid_size[d] = 1000.0;
    medyan_boundary_params bp;
    std::memset(&bp, 0, sizeof bp);
    ffm.setCoordinates(net.x.data());
    ffm.setNeighborListInputs(cyl, nlp, bp);
    auto counts = ffm.resetNeighborLists();
    std::vector<int32_t> pairs(2 * 4096);
    int64_t np = 0;
    CHECK(oracle_nl_build(&cyl, net.x.data(), net.nb, &nlp, pairs.data(), 4096, &np) == MEDYAN_OK);
    CHECK(np > 0);
    std::vector<int32_t> eb(4 * np);
    std::vector<double> ek(np), el(2 * np);
    const int64_t ne = oracle_excl_vectorize(&cyl, pairs.data(), np, eb.data(), ek.data(), el.data());
    CHECK(counts.first == ne);
    CHECK(counts.second == 0);

    // the oracle with the same excluded-volume interactions
    medyan_system s2 = s;
    s2.n_excl = (int32_t)ne;
    s2.excl_beads = eb.data();
    s2.excl_k = ek.data();
    s2.excl_eqlen = el.data();
    const double eo2 = oracle_energy(&s2, net.x.data(), nullptr);
    CHECK(rel(ffm.computeEnergy(net.x.data()), eo2) <= 1e-12);

    // a short minimization: same call counts as the oracle's CGMethod. The
    // bonded force fields only: the reference's excluded-volume force moves a
    // bead out of plane when a pair is nearly coplanar (a discontinuity), so
    // trajectories with excluded volume separate once rounding flips it.
    ForceFieldManager ffm2(MEDYAN_PREC_FP64);
    ffm2.vectorizeAllForceFields(s);
    ConjugateGradientParams p;
    p.gradTol = 1e-4;
    p.energyRelTol = 1e-14;
    p.energyCallLimit = 40;
    std::vector<double> xg = net.x, xo = net.x, fout;
    MinimizationResult r = CGMethod::minimize(p, xg, ffm2, &fout);
    medyan_cg_params cp;
    std::memset(&cp, 0, sizeof cp);
    cp.method = MEDYAN_CG_POLAK_RIBIERE;
    cp.max_dist = p.maxDist;
    cp.lambda_max = p.lambdaMax;
    cp.grad_tol = p.gradTol;
    cp.energy_rel_tol = p.energyRelTol;
    cp.energy_call_limit = p.energyCallLimit;
    cp.force_call_limit = p.forceCallLimit;
    cp.try_to_recover = 1;
    medyan_min_result ro;
    std::vector<double> fo2(nd);
    CHECK(oracle_cg_minimize(&s, &cp, xo.data(), fo2.data(), &ro) == MEDYAN_OK);
    CHECK(r.success());
    CHECK(r.numEnergyCall == ro.num_energy_call && r.numForceCall == ro.num_force_call && r.numIter == ro.num_iter);
    CHECK(rel(r.energiesBefore.total, ro.energy_before_total) <= 1e-12);
    double dx = 0;
    for (int i = 0; i < nd; ++i) dx = std::fmax(dx, std::fabs(xg[i] - xo[i]));
    std::printf("minimize: E after %.17g (oracle %.17g), max |dx| %.3g nm\n", r.energiesAfter.total,
                ro.energy_after_total, dx);
    CHECK(dx <= 1e-7);
    // coordinates agree to rounding carried through the run; the reported
    // energy is the energy of the returned coordinates
    CHECK(rel(r.energiesAfter.total, oracle_energy(&s, xg.data(), nullptr)) <= 1e-12);
    CHECK(rel(r.energiesAfter.total, ro.energy_after_total) <= 1e-10);
    CHECK((int)fout.size() == nd);

    // after a minimization: the force magnitudes the chemistry reads
    {
        const ForceFieldManager::ForceMagnitudes m = ffm2.forceMagnitudes(xg.data());
        std::vector<double> lo(s.n_linker), mo(s.n_motor), bo(3 * (size_t)s.n_branch);
        oracle_force_magnitudes(&s, xg.data(), lo.data(), mo.data(), bo.data());
        double scale = 0, err = 0;
        for (int i = 0; i < s.n_linker; ++i) {
            scale = std::fmax(scale, std::fabs(lo[i]));
            err = std::fmax(err, std::fabs(m.linkerStretch[i] - lo[i]));
        }
        CHECK((int)m.linkerStretch.size() == s.n_linker && err <= 1e-12 * scale + 1e-9);
    }
    // the autotuner leaves a handle that still computes the same energy
    {
        const medyan_launch_shapes sh = ffm2.autotune(3);
        CHECK(sh.bonded_threads == 128 || sh.bonded_threads == 256 || sh.bonded_threads == 512);
        CHECK(rel(ffm2.computeEnergy(xg.data()), oracle_energy(&s, xg.data(), nullptr)) <= 1e-12);
    }

    // lambdaRunningAverageProbability: no effect in the reference (the manager
    // is rebuilt every iteration), so a run with 0.5 is the run with 0; a value
    // outside [0, 1] is refused
    {
        ffm2.setDeterministic(true);
        ConjugateGradientParams q = p;
        std::vector<double> xa = xg, xb = xg;
        const MinimizationResult ra = CGMethod::minimize(q, xa, ffm2);
        q.lambdaRunningAverageProbability = 0.5;
        const MinimizationResult rb = CGMethod::minimize(q, xb, ffm2);
        CHECK(ra.numIter == rb.numIter && ra.numEnergyCall == rb.numEnergyCall && xa == xb);
        q.lambdaRunningAverageProbability = 2.0;
        threw = false;
        try {
            CGMethod::minimize(q, xg, ffm2);
        } catch (const Error& e) {
            threw = e.status == MEDYAN_ERR_INVALID_ARG;
        }
        CHECK(threw);
        ffm2.setDeterministic(false);
    }
    std::printf("adaptor ok: E=%.10g, %lld pairs, %d CG iterations\n", eg, (long long)ne, r.numIter);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    const char* mode = argc > 1 ? argv[1] : "gpu";
    try {
        if (!std::strcmp(mode, "nodevice")) return run_nodevice();
        return run_gpu();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "unexpected exception: %s\n", e.what());
        return 1;
    }
}

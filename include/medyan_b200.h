/*
 * medyan_b200.h — C ABI of the B200 mechanical-equilibration library.
 *
 * The library evaluates MEDYAN's mechanical energy and forces, rebuilds the
 * cylinder neighbor list and runs the Polak–Ribière conjugate-gradient
 * minimizer on one GPU. Every entry point takes plain host pointers and sizes;
 * the library owns all device memory. A handle is not thread-safe and uses
 * one CUDA stream.
 *
 * Array layouts are the ones the reference's ForceField::vectorize produces:
 *   - coordinates and forces: AoS double[3*n_beads] (x0 y0 z0 x1 ...),
 *     src/Structure/DofSerializer.hpp:64-190;
 *   - bead sets: int32 coordinate offsets 3*beadIndex, n beads per
 *     interaction, e.g. src/Mechanics/ForceField/Filament/FilamentStretching.cpp:35-36.
 *
 * Energy slots follow the reference's ForceFieldManager::forceFields order
 * (src/Controller/MController.cpp:65-188): filament → linker → motor →
 * branching → cylinder excluded volume → boundary.
 */
#ifndef MEDYAN_B200_H
#define MEDYAN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum medyan_status {
    MEDYAN_OK = 0,
    MEDYAN_ERR_INVALID_ARG = 1,   /* null pointer, negative size, bad enum      */
    MEDYAN_ERR_INDEX_RANGE = 2,   /* bead-set entry outside [0, 3*n_beads) or not a multiple of 3 */
    MEDYAN_ERR_NONFINITE = 3,     /* NaN/Inf energy: ForceFieldManager::computeEnergy returns +inf
                                     (src/Mechanics/ForceField/ForceFieldManager.cpp:150-161) */
    MEDYAN_ERR_ITER_CAP = 4,      /* a device loop hit its iteration cap      */
    MEDYAN_ERR_CUDA = 5,          /* CUDA runtime error                        */
    MEDYAN_ERR_OUT_OF_GRID = 6,   /* NL: midpoint outside the bin grid
                                     (src/Structure/HybridNeighborListImpl.cpp:243-262 throws) */
    MEDYAN_ERR_LINE_SEARCH = 7,   /* CG: line search failed, recovery disabled
                                     (MinimizationResult::errorLineSearch) */
    MEDYAN_ERR_NO_DEVICE = 8,     /* no CUDA device visible                    */
    MEDYAN_ERR_CAPACITY = 9,      /* caller's output buffer too small          */
    MEDYAN_ERR_UNSUPPORTED = 10   /* option the library does not implement     */
} medyan_status;

/* Energy slots (reference force-field order). */
enum {
    MEDYAN_FF_FILAMENT_STRETCHING = 0, /* FilamentStretching<FilamentStretchingHarmonic> */
    MEDYAN_FF_FILAMENT_BENDING = 1,    /* FilamentBending<FilamentBendingCosine>         */
    MEDYAN_FF_LINKER_STRETCHING = 2,   /* LinkerStretching<LinkerStretchingHarmonic>     */
    MEDYAN_FF_MOTOR_STRETCHING = 3,    /* MotorGhostStretching<MotorGhostStretchingHarmonic> */
    MEDYAN_FF_BRANCHING_STRETCHING = 4,/* BranchingStretching<BranchingStretchingHarmonic> */
    MEDYAN_FF_BRANCHING_BENDING = 5,   /* BranchingBending<BranchingBendingCosine>       */
    MEDYAN_FF_BRANCHING_DIHEDRAL = 6,  /* BranchingDihedral<BranchingDihedralCosine>     */
    MEDYAN_FF_BRANCHING_POSITION = 7,  /* BranchingPosition<BranchingPositionCosine>     */
    MEDYAN_FF_EXCLUDED_VOLUME = 8,     /* CylinderExclVolume<CylinderExclVolRepulsion>   */
    MEDYAN_FF_BOUNDARY = 9,            /* BoundaryCylinderRepulsion<BoundaryCylinderRepulsionExp> */
    MEDYAN_FF_COUNT = 10
};

typedef enum medyan_precision {
    MEDYAN_PREC_FP64 = 0,   /* all arithmetic in double                                  */
    MEDYAN_PREC_MIXED = 1   /* per-interaction force math in float after FP64 coordinate
                               differences (excluded volume stays double); energies, force
                               sums, dots, beta and the Armijo test in double, so the line
                               search compares the same energies as the FP64 mode */
} medyan_precision;

/* ------------------------------------------------------------------------ */
/* Vectorized force-field description                                        */
/* ------------------------------------------------------------------------ */
/*
 * One struct holds every force field's vectorized arrays. A count of 0 turns
 * a force field off (its pointers may then be NULL). Each group cites the
 * reference vectorize() that produces it.
 */
typedef struct medyan_system {
    int32_t n_beads;                 /* DOF = 3*n_beads */

    /* FilamentStretching::vectorize, Filament/FilamentStretching.cpp:24-44:
       beads[2i..2i+1], k = kstr, l0 = eql (per cylinder). */
    int32_t n_stretch;
    const int32_t* stretch_beads;
    const double* stretch_k;
    const double* stretch_l0;

    /* FilamentBending::vectorize, Filament/FilamentBending.cpp:28-66:
       beads[3i..3i+2], k = kbend, theta0 = eqt. */
    int32_t n_bend;
    const int32_t* bend_beads;
    const double* bend_k;
    const double* bend_theta0;

    /* LinkerStretching::vectorize, Linker/LinkerStretching.cpp:29-59:
       beads[4i..4i+3], k, l0, pos1, pos2. */
    int32_t n_linker;
    const int32_t* linker_beads;
    const double* linker_k;
    const double* linker_l0;
    const double* linker_pos1;
    const double* linker_pos2;

    /* MotorGhostStretching::vectorize, MotorGhost/MotorGhostStretching.cpp:29-59. */
    int32_t n_motor;
    const int32_t* motor_beads;
    const double* motor_k;
    const double* motor_l0;
    const double* motor_pos1;
    const double* motor_pos2;

    /* Branching point b: beads are parent cylinder (first, second bead) and
       child cylinder (first, second bead). BranchingStretching uses the
       first 3 (Branching/BranchingStretching.cpp:29-52), BranchingBending and
       BranchingDihedral all 4, BranchingPosition the first 3. One position
       per branch point is shared by stretching, dihedral and position. */
    int32_t n_branch;
    const int32_t* branch_beads;     /* 4 per branch point */
    const double* branch_pos;        /* adjusted relative position on the parent */
    const double* branch_stretch_k;
    const double* branch_stretch_l0;
    const double* branch_bend_k;
    const double* branch_bend_theta0;
    const double* branch_dihedral_k;
    const double* branch_position_k; /* NULL or all-zero disables BranchingPosition */
    int32_t branch_ff_mask;          /* bit 0 stretch, 1 bend, 2 dihedral, 3 position */

    /* CylinderExclVolume::vectorize, Volume/CylinderExclVolume.cpp:33-179:
       beads[4i..4i+3] = (c1, c2) of the key cylinder and (c3, c4) of its
       neighbor, krep, eqlen[2i], eqlen[2i+1]. */
    int32_t n_excl;
    const int32_t* excl_beads;
    const double* excl_k;
    const double* excl_eqlen;

    /* BoundaryCylinderRepulsion::vectorize,
       Boundary/BoundaryCylinderRepulsion.cpp:33-88: terms are grouped by
       boundary element; element e owns nneighbors[e] consecutive terms.
       Elements are planes a*x + b*y + c*z + d = 0
       (src/Structure/BoundaryElementImpl.h:30-106). */
    int32_t n_boundary;
    const int32_t* boundary_beads;   /* 1 per term */
    const double* boundary_k;
    const double* boundary_slen;
    int32_t n_planes;
    const double* plane_eq;          /* 4 per plane: a, b, c, d */
    const int32_t* plane_nneighbors; /* terms per plane */
} medyan_system;

/* ------------------------------------------------------------------------ */
/* Force-field handle                                                        */
/* ------------------------------------------------------------------------ */
typedef struct medyan_mech medyan_mech;

/* Create a handle on the current CUDA device and upload the vectorized
   force fields (the device copy of ForceFieldManager::vectorizeAllForceFields,
   src/Mechanics/ForceField/ForceFieldManager.cpp:35-93). Bead-set entries are
   range-checked on the host before upload. */
medyan_status medyan_mech_create(const medyan_system* sys, int32_t precision, medyan_mech** out);

/* Replace every force field's arrays after a new vectorization (same handle,
   same bead count). Device buffers grow when needed; none are freed. */
medyan_status medyan_mech_update(medyan_mech* h, const medyan_system* sys);
/* Create and update pack the force-field records on the device: the
   caller's arrays are copied as they are and kernels remap the bead offsets
   to the library's internal bead order, assign links and bends to filament
   chains and pack the parameters (the per-record work of the reference's
   ForceField::vectorize calls, ForceFieldManager.cpp:35-93). With on = 1 the
   next updates pack with host loops instead: the same records bit for bit,
   kept to check the device packing against. */
medyan_status medyan_mech_set_host_packing(medyan_mech* h, int32_t on);

medyan_status medyan_mech_destroy(medyan_mech* h);

/* Upload coordinates (double[3*n_beads], reference AoS order). */
medyan_status medyan_mech_set_coords(medyan_mech* h, const double* coord);
medyan_status medyan_mech_get_coords(medyan_mech* h, double* coord);

/* ForceFieldManager::computeEnergy / computeIndividualEnergies
   (ForceFieldManager.cpp:96-240): total and per-force-field energies at the
   uploaded coordinates. e_per_ff may be NULL, else double[MEDYAN_FF_COUNT].
   A force field whose energy is the reference's error value (at or below -1:
   the excluded-volume energy when its quadrature fallback also fails) sets
   *e_total = +inf and returns MEDYAN_ERR_NONFINITE. A NaN term (e.g. a bend
   over a zero-length cylinder) propagates into the total, as in the
   reference, whose bonded energies carry no check. */
medyan_status medyan_mech_energy(medyan_mech* h, double* e_total, double* e_per_ff);

/* ForceFieldManager::computeForces (ForceFieldManager.cpp:242-290):
   force_out = -dE/dx at the uploaded coordinates (zero-filled, then every
   force field accumulates). */
medyan_status medyan_mech_forces(medyan_mech* h, double* force_out);

/* One call of both: upload coord, compute energy and forces, download forces.
   This is MController::updateMechanics without the (de)serialization
   (src/Controller/MController.h:214-230). */
medyan_status medyan_mech_evaluate(medyan_mech* h, const double* coord, double* e_total,
                                   double* e_per_ff, double* force_out);

/* Device-resident variants for callers that keep data on the GPU: each
   enqueues its work on the handle's stream and returns without synchronizing
   or copying to the host. Results stay in the handle's device buffers
   (medyan_mech_device_buffers); medyan_mech_synchronize waits and reports the
   status of the enqueued passes. */
medyan_status medyan_mech_enqueue_energy(medyan_mech* h);
medyan_status medyan_mech_enqueue_forces(medyan_mech* h);
/* Energy and forces at the handle's coordinates in one pass (what
   medyan_mech_evaluate runs), the two sets of kernels side by side. */
medyan_status medyan_mech_enqueue_evaluate(medyan_mech* h);
medyan_status medyan_mech_synchronize(medyan_mech* h);

/* Deterministic force sums (no counterpart in the reference, whose CPU loops
   add in a fixed order). Forces are normally summed with floating-point
   atomic additions, whose order varies from run to run, so a force's last
   bits, and with them a long minimization's trajectory, are not
   reproducible. With on = 1 every force contribution is rounded to a 64-bit
   integer count of 2^-32 pN and summed with integer additions, which give
   the same bits in any order; the sums are converted back to double at the
   end of each force pass. Forces then differ from the floating-point sums by
   at most about 1e-9 pN per bead, and a contribution of 2^24 pN (1.7e7 pN)
   or more is out of range: the call reports MEDYAN_ERR_NONFINITE. Energies
   are deterministic in both modes. Applies to the standalone passes, the
   evaluate entry points and the minimizer (packed batches have
   medyan_batch_set_deterministic; not to the Hessian or the
   Hessian-vector product). on = 0 restores the default. */
medyan_status medyan_mech_set_deterministic(medyan_mech* h, int32_t on);

/* Asynchronous medyan_mech_evaluate, for a caller that evaluates many
   coordinate sets back to back (no counterpart in the reference, whose
   evaluation is a synchronous CPU call). Enqueues the host-to-device copy of
   coord on its own stream, the evaluate pass on the handle's stream and the
   device-to-host copies of the forces and energies on a third stream, and
   returns without waiting. Consecutive calls alternate between two staging
   slots, so the inbound copy of one call overlaps the pass and the outbound
   copy of the previous one.
     coord      double[3*n_beads] host, caller's bead order
     force_out  double[3*n_beads] host
     e_out      double[MEDYAN_FF_COUNT + 1] host: per force field, then the
                total (+inf when a force field is at or below -1, as
                medyan_mech_evaluate reports with MEDYAN_ERR_NONFINITE)
   All three must stay valid and untouched until medyan_mech_wait returns;
   the copies overlap only when they are page-locked (cudaHostAlloc,
   cudaHostRegister). Call medyan_mech_wait before any other entry point on
   the handle reads the results. */
medyan_status medyan_mech_evaluate_async(medyan_mech* h, const double* coord, double* force_out, double* e_out);
/* Waits for every asynchronous evaluation enqueued on the handle. Returns
   MEDYAN_ERR_NONFINITE when the quadrature fallback failed in any of them. */
medyan_status medyan_mech_wait(medyan_mech* h);
/* The handle's cudaStream_t, for event timing or stream ordering. */
void* medyan_mech_stream(medyan_mech* h);
/* Kernel launches in one standalone pass (which: 0 energy, 1 forces, 2 both)
   as the handle builds it for its current force fields (the kernel nodes of
   the pass graph; empty force-field groups launch nothing). Builds the pass
   graph if needed; -1 on error. A diagnostic with no counterpart in the
   reference. */
int32_t medyan_mech_pass_kernel_count(medyan_mech* h, int32_t which);
/* Device pointers of the coordinate and force arrays (double[3*n_beads]) and
   of the energy output (double[MEDYAN_FF_COUNT + 1]: per force field, then total).
   The device arrays hold the beads in the library's internal order (filament
   chains contiguous, fixed when the handle is created), which differs from
   the caller's order unless each filament's beads are already consecutive;
   medyan_mech_set_coords / get_coords / forces convert. */
medyan_status medyan_mech_device_buffers(medyan_mech* h, double** coord, double** force, double** energy);

/* ------------------------------------------------------------------------ */
/* Conjugate-gradient minimizer                                              */
/* ------------------------------------------------------------------------ */
typedef enum medyan_cg_method {
    MEDYAN_CG_STEEPEST = 0,
    MEDYAN_CG_FLETCHER_RIEVES = 1,
    MEDYAN_CG_POLAK_RIBIERE = 2
} medyan_cg_method;

/* ConjugateGradientParams, src/Mechanics/Minimizer/CGMethod.hpp:44-63. */
typedef struct medyan_cg_params {
    int32_t method;                 /* medyan_cg_method                        */
    double max_dist;                /* maxDist                                  */
    double lambda_max;              /* lambdaMax                                */
    double grad_tol;                /* gradTol (component infinity norm)        */
    double energy_rel_tol;          /* energyRelTol                             */
    int32_t energy_call_limit;      /* 0 = no limit                             */
    int32_t force_call_limit;       /* raised to max(limit, 3*n_beads)          */
    int32_t try_to_recover;         /* tryToRecoverInLineSearchError            */
    int32_t line_search;            /* lineSearchAlgorithm: 0 BACKTRACKING,
                                       1 QUADRATIC (quadraticLineSearchV2,
                                       CGMethod.hpp:521-765; backtracking in safe mode) */
} medyan_cg_params;

/* MinimizationResult, src/Mechanics/Minimizer/MinimizationTypes.hpp:10-64. */
typedef struct medyan_min_result {
    double energy_before[MEDYAN_FF_COUNT];
    double energy_before_total;
    double energy_after[MEDYAN_FF_COUNT];
    double energy_after_total;
    uint32_t error_flags;           /* bit 0: errorLineSearch                   */
    int32_t num_energy_call;
    int32_t energy_call_limit;
    int32_t num_force_call;
    int32_t force_call_limit;
    int32_t num_iter;
    double grad_inf_norm;
    double grad_tol;
    double energy_rel_change;
    double energy_rel_tol;
} medyan_min_result;

/* CGMethod::minimize (CGMethod.hpp:826-1743) with backtracking line search
   (:238-373) and MController's recovery step (src/Controller/MController.h:273-339).
   The whole loop runs on the device. coord_inout is double[3*n_beads];
   force_out may be NULL. */
medyan_status medyan_cg_minimize(medyan_mech* h, const medyan_cg_params* p, double* coord_inout,
                                 double* force_out, medyan_min_result* out);

/* ------------------------------------------------------------------------ */
/* Cylinder neighbor list                                                    */
/* ------------------------------------------------------------------------ */
/* Per-cylinder data the hybrid neighbor list reads (Cylinder::DbData,
   src/Structure/Cylinder.cpp:31-42) plus the per-cylinder parameters that
   CylinderExclVolume::vectorize and BoundaryCylinderRepulsion::vectorize
   read. Cylinder order is Cylinder::getCylinders() order. */
typedef struct medyan_cylinders {
    int32_t n_cyl;
    const int32_t* bead1;           /* bead index (not coordinate offset)      */
    const int32_t* bead2;
    const int32_t* id;              /* Cylinder::getId(), unique               */
    const int32_t* filament_id;
    const int32_t* position_on_filament;
    const int32_t* type;            /* filament type                            */
    const int32_t* branching_cylinder; /* index of the cylinder branching off this one, or -1
                                          (Cylinder::getBranchingCylinder)   */
    const int32_t* is_minus_end;    /* Cylinder::isMinusEnd()                  */
    const double* eq_length;        /* MCylinder::getEqLength()                 */
    const double* excl_k;           /* MCylinder::getExVolConst()               */
} medyan_cylinders;

/* Neighbor-list parameters: HybridCylinderCylinderNL with one
   (rmin, rmax) bound, bins of 1.125*rmax over a grid of size grid_size
   (NX*compartmentSizeX, ...), HybridNeighborListImpl.cpp:176-240. */
typedef struct medyan_nl_params {
    float rmax;                     /* stored as float, as in the reference    */
    float rmin;
    double grid_size[3];
} medyan_nl_params;

/* Cubic boundary (src/Structure/BoundaryImpl.cpp:24-52) and the boundary
   cylinder NL (src/Structure/NeighborListImpl.cpp:738-809). */
typedef struct medyan_boundary_params {
    int32_t n_planes;
    const double* plane_eq;         /* 4 per plane */
    double k;                       /* BOUNDARYINTERACTIONK */
    double screen_length;           /* BOUNDARYSCREENLENGTH */
    float cutoff;                   /* BOUNDARYCUTOFF (NeighborList::_rMax is float) */
} medyan_boundary_params;

/* Standalone neighbor-list build from host arrays (parity entry point).
   coord is double[3*n_beads]. Writes canonical pairs (key, neighbor) as
   cylinder indices into pairs_out[2*k], ordered by key index then neighbor
   index; key is the cylinder with the larger id. */
medyan_status medyan_nl_build(const medyan_cylinders* cyl, const double* coord, int32_t n_beads,
                              const medyan_nl_params* p, int32_t* pairs_out, int64_t capacity,
                              int64_t* n_pairs);

/* Attach cylinder topology and NL/boundary parameters to a handle. After this,
   medyan_mech_rebuild_neighbors rebuilds the cylinder NL and the boundary NL
   from the device coordinates and re-vectorizes the excluded-volume and
   boundary force fields on the device. */
medyan_status medyan_mech_set_cylinders(medyan_mech* h, const medyan_cylinders* cyl,
                                        const medyan_nl_params* nl,
                                        const medyan_boundary_params* boundary);
medyan_status medyan_mech_rebuild_neighbors(medyan_mech* h, int64_t* n_excl_out,
                                            int64_t* n_boundary_out);

/* Copy the excluded-volume interactions currently on the device to the host
   (beads: 4 per interaction). */
medyan_status medyan_mech_get_excl_volume(medyan_mech* h, int32_t* beads_out, double* k_out,
                                          double* eqlen_out, int64_t capacity, int64_t* n_out);

/* ------------------------------------------------------------------------ */
/* Derivatives (sensitivity analysis)                                        */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference. Gradient of the total energy with respect
   to every interaction's parameters, at the handle's coordinates, analytic
   and in FP64. With v != NULL (double[3*n_beads], caller's bead order) the
   outputs are instead the derivatives of those gradients along v,
   d/de [dE/dtheta](x + e v) = v . d2E/(dx dtheta), in forward mode (the
   gradient formulas on dual numbers carrying v: exact to rounding) — the
   mixed term an implicit adjoint needs. Outputs are double[n] in the force field's interaction order (the
   order given at vectorization; for excluded volume and boundary rebuilt on
   the device, the order of medyan_mech_get_excl_volume); either may be NULL.
     MEDYAN_FF_FILAMENT_STRETCHING, _LINKER_STRETCHING, _MOTOR_STRETCHING:
         d_k = dE/dk,      d_p = dE/dl0
     MEDYAN_FF_FILAMENT_BENDING:     d_k = dE/dk,   d_p = dE/dtheta0
     MEDYAN_FF_BRANCHING_STRETCHING: d_k = dE/dk,   d_p = dE/dl0
     MEDYAN_FF_BRANCHING_BENDING:    d_k = dE/dk,   d_p = dE/dtheta0
     MEDYAN_FF_BRANCHING_DIHEDRAL, _BRANCHING_POSITION: d_k = dE/dk; d_p = 0
                                     (the four branching slots: one entry per
                                     branch point; zero when that potential is
                                     off in branch_ff_mask)
     MEDYAN_FF_EXCLUDED_VOLUME:      d_k = dE/dkRS with kRS = krep*L1*L2
                                     (multiply by L1*L2 for dE/dkrep); d_p = 0
     MEDYAN_FF_BOUNDARY:             d_k = dE/dk,   d_p = dE/dscreen_length
   n must equal the force field's interaction count (else
   MEDYAN_ERR_CAPACITY). */
medyan_status medyan_mech_param_grad(medyan_mech* h, int32_t ff, const double* v, double* d_k, double* d_p,
                                     int64_t n);

/* Hessian-vector product hv = (d2E/dx2) v at the handle's coordinates
   (double[3*n_beads], caller's bead order), in forward mode: every force
   formula of the force pass evaluated on dual numbers carrying v (positions
   x + e v), hv = -dF/de, exact to rounding and in FP64 whatever the handle's
   precision. It replaces the reference's finite-difference Hessian columns
   (ForceFieldManager::computeHessian, ForceFieldManager.cpp:354-489) for
   products. An excluded-volume pair that the analytic formula rejects (the
   quadrature fallback's pairs) has no forward-mode derivative: the call
   returns MEDYAN_ERR_NONFINITE. */
medyan_status medyan_mech_hvp(medyan_mech* h, const double* v, double* hv);

/* ---- launch shapes and the autotuner (no counterpart in the reference,
   whose kernels run on the CPU) ----
   Block and tile shapes per potential. Every shape gives the same physics;
   the energy reduction tree, and so the last bits of the energies, depend on
   the shape (deterministic for a given shape). */
typedef struct medyan_launch_shapes {
    int32_t bonded_threads;         /* records (= threads) per block of the bonded
                                       potentials (linker, motor, branching,
                                       boundary, leftover filament terms): 128, 256, 512 */
    int32_t excl_threads;           /* pairs (= threads) per block of the
                                       excluded-volume kernels: 32, 64, 128 */
    int32_t chain_threads;          /* threads per block of the filament-chain
                                       force kernel (30 beads per warp): 128, 256, 512 */
    int32_t chain_energy_blocks_per_sm; /* fixed grid of the filament-chain energy
                                       kernel, in blocks of 256 per SM: 2, 4, 8 */
    int32_t pass_layout;            /* kernels of the standalone passes and of the
                                       minimizer's force pass: 0 = fused (forces: a
                                       zero fill, then three kernels side by side:
                                       chains with linker, motor, boundary and
                                       leftover records; branch points; excluded
                                       volume; energies: the same three kernels
                                       with the row reduction built in), 1 = one
                                       kernel per potential group (chain forces
                                       first, the rest after), 2 = fused with
                                       the filament chains in a kernel of their
                                       own that stages chain segments through
                                       shared memory by bulk copies */
} medyan_launch_shapes;

/* The defaults are 256, 64, 256, 4, 0. Setting shapes re-derives the block
   tables and invalidates the handle's captured passes (rebuilt on next use). */
medyan_status medyan_mech_set_shapes(medyan_mech* h, const medyan_launch_shapes* shapes);
medyan_status medyan_mech_get_shapes(medyan_mech* h, medyan_launch_shapes* shapes);
/* Picks the shapes for this handle's network: coordinate descent over the
   five fields above (each candidate timed as the mean of `reps` evaluate
   passes after two warm-up passes, CUDA events on the handle's stream, at
   the handle's current coordinates), keeps the fastest and reports it in
   *chosen (may be null). */
medyan_status medyan_mech_autotune(medyan_mech* h, int32_t reps, medyan_launch_shapes* chosen);

/* ---- after a minimization: inputs of the chemical rate changers ----
   MController::afterMinimization_ (src/Controller/MController.h:238-268)
   runs ffm.assignallforcemags() and ffm.computeAuxParams(), whose
   computeLoadForces fills the filament tips' load forces. */

/* The force magnitudes each force field stores during its force pass and
   assignforcemags adds to the chemistry's objects
   (ForceFieldManager::assignallforcemags, ForceFieldManager.cpp:346-351), at
   the handle's coordinates, FP64, caller's interaction order; each array may
   be null:
     linker_stretch[i] = f0/invL = k (L - l0) of linker i, the value
       LinkerStretching::assignforcemags adds to MLinker::stretchForce
       (LinkerStretchingHarmonic.cpp:227-293, LinkerStretching.cpp:118-123);
     motor_stretch[i]: the same for motor i (MotorGhostStretching.cpp:125-130);
     branch_force[3*i .. 3*i+2]: the force each enabled branching force
       field puts on the third bead of branch point i, summed in force-field
       order (stretching, bending, dihedral, position), the value their
       assignforcemags add to MBranchingPoint::branchForce. */
medyan_status medyan_mech_force_magnitudes(medyan_mech* h, double* linker_stretch, double* motor_stretch,
                                           double* branch_force);

/* Filament tips whose boundary load forces are wanted. Cylinder indices
   refer to the list given to medyan_mech_set_cylinders. */
typedef struct medyan_load_tips {
    int32_t n_tips;
    const int32_t* cylinder;        /* the tip's cylinder                       */
    const int32_t* plus_end;        /* 1: plus end (load on bead2, growing from
                                       bead1 to bead2); 0: minus end (bead1)   */
    const int32_t* n_mon;           /* cylinderNumMon of the tip bead's type   */
    const double* mon_size;         /* monomerSize of that type                */
} medyan_load_tips;

/* BoundaryCylinderRepulsion::computeLoadForces with the exponential
   repulsion (BoundaryCylinderRepulsion.cpp:125-196, BoundaryCylinderRepulsionExp.cpp:113-118):
   for each boundary plane whose neighbor list (the last
   medyan_mech_rebuild_neighbors) holds the tip's cylinder, and each monomer
   position i < n_mon of the tip, newCoord = tip bead + i*mon_size*dir (dir
   the unit vector from the other bead to the tip bead),
     load[i] += max(-normal . dir, 0) * k exp(-distance(newCoord)/screen_length)/screen_length,
   with normal = (a, b, c) of the plane and distance its signed distance. The
   loads of tip t are load_out[o_t .. o_t + n_mon[t]), o_t = sum of the earlier
   tips' n_mon; capacity is the length of load_out. Loads start at zero (the
   reference resets them in ForceFieldManager::computeLoadForces). No
   boundary: all zero. */
medyan_status medyan_mech_boundary_load_forces(medyan_mech* h, const medyan_load_tips* tips, double* load_out,
                                               int64_t capacity);

/* ForceFieldManager::computeHessian (src/Mechanics/ForceField/ForceFieldManager.cpp:354-398):
   the dense finite-difference Hessian at the handle's coordinates, row i
   the perturbed degree of freedom, column j the force component (caller's
   bead order, ndof = 3*n_beads, row-major host array of ndof*ndof doubles):
     H[i*ndof + j] = (float)(-(F_j(x + delta e_i) - F_j(x - delta e_i)) / (2*delta)),
   each entry rounded to float as the reference stores it, delta the
   reference's float hessDelta. 2*ndof force passes; the coordinates are
   restored exactly. The reference's eigenmode analysis (symmetrization,
   eigensolve, participation ratios, :400-480) works on this matrix and is
   left to the caller (medyan_b200.forcefield.hessian_modes). Use an FP64
   handle. ndof above MEDYAN_HESSIAN_MAX_DOF: MEDYAN_ERR_INVALID_ARG. */
#define MEDYAN_HESSIAN_MAX_DOF 24576
medyan_status medyan_mech_hessian(medyan_mech* h, float delta, double* H);

/* ------------------------------------------------------------------------ */
/* Batched minimization of independent networks                              */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference (which minimizes one system at a time).
   A batch holds one handle per replica network. medyan_batch_minimize
   enqueues every replica's whole minimization (one graph launch each, loops
   on the device) before waiting for any, so the replicas run concurrently and
   each stops at its own convergence test; every replica gets exactly the
   CGMethod::minimize semantics of medyan_cg_minimize. */
typedef struct medyan_batch medyan_batch;

medyan_status medyan_batch_create(const medyan_system* systems, int32_t n_replicas, int32_t precision,
                                  medyan_batch** out);
medyan_status medyan_batch_destroy(medyan_batch* b);
int32_t medyan_batch_size(const medyan_batch* b);
/* The handle of replica r (owned by the batch), e.g. for
   medyan_mech_set_cylinders / medyan_mech_rebuild_neighbors; NULL if out of range. */
medyan_mech* medyan_batch_replica(medyan_batch* b, int32_t r);
/* coords_inout[r]: double[3*n_beads(r)]; forces_out may be NULL, else
   forces_out[r] likewise; results may be NULL, else medyan_min_result[n];
   statuses[n] receives each replica's status (MEDYAN_ERR_LINE_SEARCH is a
   per-replica outcome). Returns the first status that is neither OK nor
   MEDYAN_ERR_LINE_SEARCH, else MEDYAN_OK. */
medyan_status medyan_batch_minimize(medyan_batch* b, const medyan_cg_params* p, double* const* coords_inout,
                                    double* const* forces_out, medyan_min_result* results, int32_t* statuses);
/* Bitwise reproducible force sums for the whole batch (no counterpart in
   the reference, whose CPU sums are sequential): the packed minimizer's
   force passes and every replica's own passes sum force contributions as
   64-bit fixed-point integers, as medyan_mech_set_deterministic does for one
   network, so a batched minimization gives the same bits on every run. A
   contribution of 2^24 pN or more makes medyan_batch_minimize return
   MEDYAN_ERR_NONFINITE. on = 0 restores floating-point atomic sums. */
medyan_status medyan_batch_set_deterministic(medyan_batch* b, int32_t on);
/* Energy and forces of every replica (e_totals: double[n]). */
medyan_status medyan_batch_evaluate(medyan_batch* b, const double* const* coords, double* e_totals,
                                    double* const* forces_out);

/* Shapes of a batch's packed layout (each replica's records are padded to
   whole blocks, so small replicas favour small blocks). Defaults 256, 64,
   256, 256. Setting them repacks on the next batched call. */
typedef struct medyan_batch_shapes {
    int32_t bonded_threads;         /* 128, 256, 512 */
    int32_t excl_threads;           /* 32, 64, 128 */
    int32_t chain_threads;          /* 128, 256, 512 */
    int32_t chain_chunk;            /* positions per chain-energy block: 256, 512, 1024 */
} medyan_batch_shapes;
medyan_status medyan_batch_set_shapes(medyan_batch* b, const medyan_batch_shapes* shapes);
medyan_status medyan_batch_get_shapes(medyan_batch* b, medyan_batch_shapes* shapes);
/* Coordinate descent over the four fields, each candidate timed as the mean
   of `reps` packed evaluate passes (energy and forces of every replica at
   its handle's current coordinates); keeps the fastest. */
medyan_status medyan_batch_autotune(medyan_batch* b, int32_t reps, medyan_batch_shapes* chosen);

/* ------------------------------------------------------------------------ */
/* Excluded-volume energy without device allocation                          */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference: it has no entry point of this kind.
   Handles allocate their device scratch with cudaMalloc. This entry point
   allocates nothing, for callers that cannot let a library allocate device
   memory when they need an energy. Examples: an application whose own pool
   allocator owns the device, or a step loop whose device footprint must stay
   fixed.

   Computes the excluded-volume energy of n_pairs cylinder pairs. All array
   pointers are DEVICE pointers on the current device, owned by the caller:
     d_coords      double[3*n_beads]   AoS coordinates
     d_excl_beads  int32[4*n_pairs]    coordinate offsets 3*bead, 16-byte aligned
     d_excl_krs    double[n_pairs]     krep * eqLength1 * eqLength2 per pair
   The kernels and the fallback for degenerate pairs are those of
   medyan_mech_energy's excluded-volume slot, in FP64. The call is
   synchronous: it enqueues on `stream` (a cudaStream_t; NULL = legacy
   default stream), waits for that stream and stores the energy in *e_out
   (host).

   Scratch lives in a fixed static device array of the library, sized for
   MEDYAN_NOALLOC_MAX_EXCL_PAIRS pairs. Larger n_pairs returns
   MEDYAN_ERR_CAPACITY. Bead offsets outside [0, 3*n_beads) or not multiples
   of 3 return MEDYAN_ERR_INDEX_RANGE before any energy kernel runs. When a
   pair's energy is non-finite (or below -1) even after the quadrature
   fallback, the call returns MEDYAN_ERR_NONFINITE and *e_out holds -1, the
   value the reference's force field reports for a bad energy.

   Every call looks up the scratch array's device address on the current
   device (cudaGetSymbolAddress). The first call on each device also fills
   the fallback's quadrature grids once: make that first call before any
   stream capture begins. A cudaDeviceReset discards that set-up: do not use
   the library across a device reset. All calls on one device share the
   scratch: calls that overlap in time (other host threads, other streams)
   race and give wrong results, so serialize them. */
#define MEDYAN_NOALLOC_MAX_EXCL_PAIRS 262144
medyan_status medyan_excl_energy_noalloc(const double* d_coords, int32_t n_beads,
                                         const int32_t* d_excl_beads, const double* d_excl_krs,
                                         int32_t n_pairs, double* e_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Library info                                                              */
/* ------------------------------------------------------------------------ */
const char* medyan_status_string(int32_t status);
/* Name of the CUDA runtime error behind the most recent MEDYAN_ERR_CUDA (or
   MEDYAN_ERR_NO_DEVICE) any entry point returned on the calling thread, e.g.
   "cudaErrorInvalidValue"; "" when there was none. */
const char* medyan_last_cuda_error(void);
int32_t medyan_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MEDYAN_B200_H */

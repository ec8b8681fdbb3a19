/*
 * medyan_oracle.h — CPU restatement of MEDYAN's mechanical-equilibration
 * path, used ONLY as a checker (tests, smoke test, CPU-baseline timing).
 * The product path (the CUDA library) never calls it.
 *
 * Parity of this restatement is pinned against the reference's own compiled
 * sources (oracle/_ref/libmedyan_ref.so built by `make -C oracle ref`) and
 * against the inputs of the reference's unit tests (tests/golden/).
 */
#ifndef MEDYAN_ORACLE_H
#define MEDYAN_ORACLE_H

#include <stdint.h>
#include "medyan_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-force-field kernels. Bead sets hold coordinate offsets 3*bead. */
double oracle_fil_stretch_energy(const double* x, int32_t n, const int32_t* bs, const double* k, const double* l0);
void oracle_fil_stretch_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k, const double* l0);
double oracle_fil_bend_energy(const double* x, int32_t n, const int32_t* bs, const double* k, const double* t0);
void oracle_fil_bend_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k, const double* t0);
double oracle_two_point_spring_energy(const double* x, int32_t n, const int32_t* bs, const double* k,
                                      const double* l0, const double* p1, const double* p2);
void oracle_two_point_spring_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k,
                                    const double* l0, const double* p1, const double* p2);
double oracle_branch_stretch_energy(const double* x, int32_t n, const int32_t* bs4, const double* k,
                                    const double* l0, const double* pos);
void oracle_branch_stretch_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                                  const double* l0, const double* pos);
double oracle_branch_bend_energy(const double* x, int32_t n, const int32_t* bs4, const double* k, const double* t0);
void oracle_branch_bend_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                               const double* t0);
double oracle_branch_dihedral_energy(const double* x, int32_t n, const int32_t* bs4, const double* k, const double* pos);
void oracle_branch_dihedral_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                                   const double* pos);
double oracle_branch_position_energy(const double* x, int32_t n, const int32_t* bs4, const double* k, const double* pos);
void oracle_branch_position_forces(const double* x, double* f, int32_t n, const int32_t* bs4, const double* k,
                                   const double* pos);
/* Returns -1 when an interaction stays non-finite after the numeric fallback. */
double oracle_excl_energy(const double* x, int32_t n, const int32_t* bs, const double* k, const double* eqlen);
void oracle_excl_forces(const double* x, double* f, int32_t n, const int32_t* bs, const double* k, const double* eqlen);
/* Per-pair analytic energy (no fallback), for diagnostics. */
double oracle_excl_pair_energy(const double* c1, const double* c2, const double* c3, const double* c4,
                               double krep_scaled);
double oracle_boundary_energy(const double* x, const medyan_system* s);
void oracle_boundary_forces(const double* x, double* f, const medyan_system* s);

/* ForceFieldManager semantics. */
double oracle_energy(const medyan_system* s, const double* x, double* e_per_ff);
void oracle_forces(const medyan_system* s, const double* x, double* f);
/* ForceFieldManager::assignallforcemags inputs: linker/motor tensions, branch-point forces (3 per branch). */
void oracle_force_magnitudes(const medyan_system* s, const double* x, double* lin, double* mot, double* br);
/* BoundaryCylinderRepulsion::computeLoadForces on filament tips. */
void oracle_boundary_load_forces(const medyan_cylinders* c, const double* x, const medyan_boundary_params* b,
                                 int32_t n_tips, const int32_t* cyl, const int32_t* plus_end, const int32_t* n_mon,
                                 const double* mon_size, double* out);
/* ForceFieldManager::computeHessian: dense FD Hessian, row-major 3N x 3N. */
void oracle_hessian(const medyan_system* s, const double* x, float delta, double* H);

/* CGMethod::minimize driven by callbacks: energy(x), forces(x, f) and the
   per-force-field energies (x, per[MEDYAN_FF_COUNT]). n_beads only sets the
   force-call limit max(limit, 3*n_beads). */
typedef double (*oracle_energy_fn)(void* ctx, const double* x);
typedef void (*oracle_force_fn)(void* ctx, const double* x, double* f);
typedef void (*oracle_individual_fn)(void* ctx, const double* x, double* per);
int32_t oracle_cg_minimize_cb(int32_t ndof, int32_t n_beads, const medyan_cg_params* p, double* x, double* f_out,
                              medyan_min_result* out, oracle_energy_fn efn, oracle_force_fn ffn,
                              oracle_individual_fn ifn, void* ctx);

/* CGMethod::minimize over the force fields of s. Returns MEDYAN_OK,
   MEDYAN_ERR_LINE_SEARCH or MEDYAN_ERR_NONFINITE. */
int32_t oracle_cg_minimize(const medyan_system* s, const medyan_cg_params* p, double* x, double* f_out,
                           medyan_min_result* out);

/* HybridCylinderCylinderNL::reset restated as a pair set; pairs written as
   (key index, neighbor index), sorted. */
int32_t oracle_nl_build(const medyan_cylinders* c, const double* x, int32_t n_beads, const medyan_nl_params* p,
                        int32_t* pairs, int64_t capacity, int64_t* n_pairs);
/* CylinderExclVolume::vectorize over a sorted pair list. */
int64_t oracle_excl_vectorize(const medyan_cylinders* c, const int32_t* pairs, int64_t n_pairs,
                              int32_t* beads, double* k, double* eqlen);
/* BoundaryCylinderNL::reset + BoundaryCylinderRepulsion::vectorize. With
   beads == NULL only counts. Fills per-plane nneighbors. */
int64_t oracle_boundary_vectorize(const medyan_cylinders* c, const double* x, const medyan_boundary_params* b,
                                  int32_t* beads, double* k, double* slen, int32_t* nneighbors);

#ifdef __cplusplus
}
#endif

#endif

/*
 * CPU FP64 oracle for the DUGKS step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of dugksFoam's fvDVM::evolution()
 * (src/fvDVM/fvDVM/fvDVM.C:2128-2174) and of the OpenFOAM mesh/gradient
 * arithmetic it relies on.  Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark load it, as the checker; the product path
 * never calls it.
 *
 * Parity status: the quadrature is pinned bit-exactly against the
 * reference's own setDV.py; the step itself is unpinned (the reference
 * needs OpenFOAM, MPI and legacy TBB, none of which exist here, and ships
 * no outputs of this code path).  It is checked by known-answer tests.
 */
#ifndef DUGKS_ORACLE_H
#define DUGKS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* patch types by the rho patch type (discreteVelocity::setBCtype,
 * discreteVelocity.C:188-195): calculatedMaxwell -> maxwellWall, farField,
 * zeroGradient, fixedValue -> mixed, symmetryPlane, symmetryMod ->
 * DVMsymmetry, pressureIn / pressureOut -> farField plus the macro update of
 * fvDVM::updatePressureInOutBC */
enum {
    ORACLE_PATCH_MAXWELL_WALL = 1,
    ORACLE_PATCH_FAR_FIELD = 2,
    ORACLE_PATCH_ZERO_GRADIENT = 3,
    ORACLE_PATCH_MIXED = 4,
    ORACLE_PATCH_SYMMETRY = 5,
    ORACLE_PATCH_DVM_SYMMETRY = 6,
    ORACLE_PATCH_PRESSURE_IN = 7,
    ORACLE_PATCH_PRESSURE_OUT = 8
};
enum { ORACLE_LS_MAGSF = 0, ORACLE_LS_INVDIST = 1, ORACLE_LS_UNWEIGHTED = 2 };

typedef struct oracle_state oracle_state;

/* OpenFOAM primitiveMesh geometry over ALL faces (empty patches included,
 * they close the cells): face centres/area vectors, cell centres/volumes. */
void oracle_geometry(int n_points, const double* points, int n_faces, const int64_t* face_offsets,
                     const int64_t* face_points, const int64_t* owner, int n_internal,
                     const int64_t* neighbour, int n_cells, double* Cf, double* Sf, double* C,
                     double* V);

/* Build the solver.  Faces: n_internal internal faces then n_boundary
 * boundary faces of non-empty patches; patch_start has n_patches+1 entries
 * (offsets into the boundary faces). */
oracle_state* oracle_create(int D, int K_inner, double R, double omega, double Tref, double muRef,
                            double Pr, int n_cells, int n_internal, int n_boundary,
                            const int64_t* owner, const int64_t* neighbour, const double* C,
                            const double* V, const double* Cf, const double* Sf, int n_patches,
                            const int* patch_type, const int* patch_start, const double* rho_b,
                            const double* U_b, const double* T_b, int n_dv, const double* xi,
                            const double* w, double xi_max, int ls_weighting, int n_threads);
void oracle_destroy(oracle_state* s);

/* Per-face pressure of pressureIn/pressureOut faces (the patch dictionary's
 * pressureIn / pressureOut entry; others ignored) and the DV count per
 * dimension (symmetry targets, fvDVM.C:300-372).  Call before
 * oracle_set_macros when the mesh has such patches. */
void oracle_set_patch_extra(oracle_state* s, int n_dv_1d, const double* p_b);

/* fvDVMparas macroFlux (fvDVM.C:1940): 0 "no"; 1 "yes", the cell rho, rho U
 * and rho E advance by the face macro fluxes (fvDVM.C:1613-1679); 2 "yes" in
 * the unstructured-velocity-mesh build, by the fluxes of the relaxed face
 * DFs (fvDVM.C:1562-1611). */
void oracle_set_macro_flux(oracle_state* s, int mode);

/* fvDVM ctor tail: initialiseDV (Maxwellian g/h), setCalculatedMaxwellRhoBC,
 * updateTau, linear Usurf (fvDVM.C:2110-2116). */
void oracle_set_macros(oracle_state* s, const double* rho, const double* U, const double* T);
/* One fvDVM::evolution() with time step dt. */
void oracle_evolve(oracle_state* s, double dt);
/* fvDVM::getCoNum (fvDVM.C:2177-2185) */
void oracle_co_num(oracle_state* s, double dt, double* co_max, double* co_mean);

void oracle_get_macros(oracle_state* s, double* rho, double* U, double* T, double* q, double* tau);
/* face macros: internal faces then boundary faces */
void oracle_get_face_macros(oracle_state* s, double* rho, double* U, double* T, double* q,
                            double* tau);
void oracle_get_wall(oracle_state* s, double* rho_w, double* in_coming_by_rho);
/* g~ and h~ for all DVs, DV-major [dv][cell] */
void oracle_get_state(oracle_state* s, double* g, double* h);
void oracle_set_state(oracle_state* s, const double* g, const double* h);
/* intermediate arrays of the last step (for per-sub-step checks) */
void oracle_get_ghbar(oracle_state* s, double* g, double* h);
void oracle_get_face_values(oracle_state* s, double* g_int, double* h_int, double* g_b,
                            double* h_b);
/* least-squares vectors (p, n per internal face; boundary vectors) */
void oracle_get_ls(oracle_state* s, double* p, double* n, double* b);
void oracle_get_weights(oracle_state* s, double* w, double* delta_coeffs);

/* Tangent-linear run (dugks_tangent.cpp): n_steps steps of dt from the
 * current state, which is left unchanged, on dual numbers.  J = 1/N sum
 * over steps and boundary faces b and DVs i of w_i (xi_i . S_b)
 * [heat_w_b (|xi_i|^2 g + h)/2 + (force_w_b . xi_i) g] over the relaxed
 * boundary-face DFs; dJ = its derivative along the direction (dT_b per
 * boundary face, dU_b per boundary face, d_muRef).  NULL weights or
 * directions are zero.  g_out / h_out (or NULL) get the final g~, h~.
 * Returns -1 for patches other than maxwellWall and farField or macroFlux. */
int oracle_tangent(const oracle_state* s, int n_steps, double dt, const double* heat_w, const double* force_w,
                   const double* dT_b, const double* dU_b, double d_muRef, double* J, double* dJ, double* g_out,
                   double* h_out);

#ifdef __cplusplus
}
#endif
#endif

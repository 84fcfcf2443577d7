/*
 * dugks_b200 -- C ABI of the B200-native DUGKS step.
 *
 * This ABI replaces the step of dugksFoam's Foam::fvDVM class
 * (src/fvDVM/fvDVM/fvDVM.H:80-409).  A thin fvDVM shim keeps that class's
 * public interface and calls into this library:
 *
 *   fvDVM::fvDVM(rho, U, T, argc, argv, args)   fvDVM.C:1901-2117
 *       -> dugks_create + dugks_set_macros
 *   fvDVM::evolution()                          fvDVM.C:2128-2174
 *       -> dugks_step, then dugks_get_macros into the app's rho/U/T fields
 *   fvDVM::getCoNum(maxCo, meanCo)              fvDVM.C:2177-2185
 *       -> dugks_co_num
 *   fvDVM::writeDFonCells()                     fvDVM.C:1835-1897
 *       -> dugks_get_df
 *   qVol()/qSurf() accessors (fvDVM.H:330-396)  -> dugks_get_macros,
 *                                                  dugks_get_face_macros
 *
 * Conventions.  Plain pointers and sizes only.  Host buffers are owned by
 * the caller and copied; the distribution functions live in device memory
 * owned by the handle.  Every function returns a dugks_status; no function
 * aborts the process.  dugks_last_error() returns the text of the last
 * error on a handle.  One handle is used by one host thread at a time.
 *
 * Mesh convention: OpenFOAM fvMesh addressing.  Faces are the internal
 * faces (owner < neighbour, any order) followed by the boundary faces of the
 * non-empty patches, grouped by patch (empty patches have no fv faces).
 * Vectors are stored xyz-interleaved.  Cell and face geometry is what
 * fvMesh provides (C, V, Cf, Sf); dugks_mesh_geometry computes it from a
 * polyMesh when OpenFOAM is not present.
 */
#ifndef DUGKS_B200_H
#define DUGKS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DUGKS_ABI_VERSION 2

typedef enum dugks_status {
    DUGKS_OK = 0,
    DUGKS_ERR_ARG = 1,       /* invalid argument (null pointer, bad size, bad mesh) */
    DUGKS_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    DUGKS_ERR_OOM = 3,       /* device or host allocation failed */
    DUGKS_ERR_TIMEOUT = 4,   /* a bounded device wait ran out */
    DUGKS_ERR_NAN = 5,       /* non-finite or non-positive rho/T given or computed */
    DUGKS_ERR_STATE = 6,     /* call out of order (e.g. step before set_macros) */
    DUGKS_ERR_UNSUPPORTED = 7
} dugks_status;

/* Boundary patch types.  The reference selects the g/h surface patch type
 * from the rho patch type (discreteVelocity::setBCtype,
 * src/fvDVM/discreteVelocity/discreteVelocity.C:188-195); the g/h
 * surface values per type are those of fvDVM::updateGHbarSurf
 * (fvDVM.C:866-1027), their relaxation fvDVM.C:1429-1453:
 *   rho calculatedMaxwell -> maxwellWall  diffuse Maxwell wall
 *   rho farField          -> farField     incoming rho_b M(U_owner, T_b), outgoing upwind
 *   rho zeroGradient      -> zeroGradient every DV takes the owner cell's gbar+
 *   rho fixedValue        -> mixed        incoming keep the Maxwellian of the patch rho,
 *                                         U, T set at start (discreteVelocity.C:226-258)
 *   symmetryPlane         -> symmetryPlane incoming DV = the face value of its mirror DV
 *                                         (discreteVelocity.C:745-771)
 *   rho symmetryMod       -> DVMsymmetry  the same, and every DV relaxed once more
 *   rho pressureIn        -> farField     and after each step rho_b = p/(R T_b)
 *   rho pressureOut       -> farField     and after each step rho_b, T_b from the owner
 *                                         cell and p (fvDVM::updatePressureInOutBC,
 *                                         fvDVM.C:1745-1821)
 * Symmetry patches must be planar and normal to a coordinate axis (the
 * reference mirrors by the patch's first face normal); they are not
 * supported on a DV-sharded handle (the mirror DV can live on another
 * shard). */
typedef enum dugks_patch_type {
    DUGKS_PATCH_MAXWELL_WALL = 1,
    DUGKS_PATCH_FAR_FIELD = 2,
    DUGKS_PATCH_ZERO_GRADIENT = 3,
    DUGKS_PATCH_MIXED = 4,
    DUGKS_PATCH_SYMMETRY = 5,
    DUGKS_PATCH_DVM_SYMMETRY = 6,
    DUGKS_PATCH_PRESSURE_IN = 7,
    DUGKS_PATCH_PRESSURE_OUT = 8
} dugks_patch_type;

typedef enum dugks_precision {
    DUGKS_FP64 = 0,   /* FP64 storage and arithmetic, the plain path */
    DUGKS_FP32C = 1   /* FP32 g/h storage and flux arithmetic; FP64 moment accumulation,
                         conserved update, heat-flux term and quadrature weights.  With a
                         tensor DV set the FP32 arrays hold deviations from the Maxwellian of
                         the mean state that dugks_set_macros was given (one value per DV),
                         so rounding acts on the deviation only; dugks_get_state,
                         dugks_get_df and dugks_set_state convert to and from full values */
} dugks_precision;

/* Least-squares weighting (the stock leastSquares scheme as written in
 * src/fvDVM/zeroBoundaryGrad/zeroBoundaryVectors.C:110-123 is the default;
 * the two variants are invDistLeastSquaresVectors.C:109-167 and
 * unweightedLeastSquaresVectors.C:108-162 of the same directory). */
typedef enum dugks_ls_weighting {
    DUGKS_LS_MAGSF = 0,
    DUGKS_LS_INVDIST = 1,
    DUGKS_LS_UNWEIGHTED = 2
} dugks_ls_weighting;

typedef struct dugks_mesh {
    int32_t n_cells;
    int32_t n_internal_faces;
    int32_t n_boundary_faces;       /* faces of non-empty patches */
    int32_t n_solution_dims;        /* fvMesh::nSolutionD(): 2 (z empty) or 3 */
    const int64_t* owner;           /* [n_internal_faces + n_boundary_faces] */
    const int64_t* neighbour;       /* [n_internal_faces] */
    const double* cell_centres;     /* [n_cells*3]  fvMesh::C() */
    const double* cell_volumes;     /* [n_cells]    fvMesh::V() */
    const double* face_centres;     /* [n_faces*3]  fvMesh::Cf() */
    const double* face_areas;       /* [n_faces*3]  fvMesh::Sf() */
    int32_t n_patches;              /* non-empty patches */
    const int32_t* patch_start;     /* [n_patches+1] offsets into the boundary faces */
} dugks_mesh;

/* constant/Xis, constant/weights and DVMProperties fvDVMparas
 * (fvDVM.C:62-123, :1928-1933); the D-dimensional tensor product is built
 * as fvDVM::initialiseDV does (fvDVM.C:293-374). */
typedef struct dugks_dv_set {
    int32_t n_per_dim;              /* nDV */
    const double* xis;              /* [n_per_dim] */
    const double* weights;          /* [n_per_dim] */
    double xi_max;                  /* xiMax, used by the Courant number only */
} dugks_dv_set;

/* A DV set that is no tensor product: the reference's unstructured velocity
 * mesh (the VMESH build, fvDVM.C:129-277), whose DVs are the cell centres of
 * constant/vMesh and whose weights are their cell volumes (xiMax = the
 * largest |xi|).  In 2-D the z components are ignored. */
typedef struct dugks_dv_list {
    int32_t n_dv;
    const double* xi;               /* [n_dv*3] */
    const double* weights;          /* [n_dv] */
    double xi_max;
} dugks_dv_list;

/* DVMProperties gasProperties (fvDVM.C:1943-1948) */
typedef struct dugks_gas {
    double R;
    double omega;
    double Tref;
    double mu_ref;
    double Pr;
    int32_t K_inner;
} dugks_gas;

/* Boundary conditions of the non-empty patches.  Per boundary face values
 * are the patch values of the app's rho, U and T fields.  For maxwellWall
 * faces rho is ignored (computed each step from the outgoing flux,
 * calculatedMaxwellFvPatchField.C:140-164); for farField faces rho and T
 * stay at these values (farFieldFvPatchField.H assignment operators are
 * no-ops) and U is not used (the owner-cell velocity is, fvDVM.C:929-934).
 * pressureIn / pressureOut faces start from these rho and T (the reference's
 * patch constructors set rho to 1, pressureInFvPatchField.C:72-75) and p is
 * their pressureIn / pressureOut value.  p may be NULL without pressure
 * patches; zeroGradient and symmetry faces use no values. */
typedef struct dugks_bc {
    const int32_t* patch_type;      /* [n_patches] dugks_patch_type */
    const double* rho;              /* [n_boundary_faces] */
    const double* U;                /* [n_boundary_faces*3] */
    const double* T;                /* [n_boundary_faces] */
    const double* p;                /* [n_boundary_faces] or NULL */
} dugks_bc;

typedef struct dugks_options {
    int32_t precision;              /* dugks_precision */
    int32_t ls_weighting;           /* dugks_ls_weighting */
    int32_t device;                 /* CUDA device ordinal */
    int32_t tile_cells;             /* cells per tile; 0 = automatic */
    int32_t dv_chunks;              /* DV chunks per tile; 0 = automatic */
    int32_t macro_flux;             /* fvDVMparas macroFlux: 0 "no" (cell macros from the
                                       DF moments), 1 "yes" (cell rho, rho U, rho E advance by
                                       the face macro fluxes, fvDVM.C:1613-1679; the
                                       unstructured-velocity-mesh variant of that branch is
                                       not built) */
    int32_t reserved[10];
} dugks_options;

typedef struct dugks_handle dugks_handle;

int dugks_abi_version(void);

/* Default options (FP64, magSf-weighted least squares, device 0, automatic tiling). */
void dugks_default_options(dugks_options* opt);

/* Host-only: OpenFOAM primitiveMesh geometry from a polyMesh (all faces,
 * empty patches included).  Face centres/area vectors by the triangle fan
 * about the point average; cell centres/volumes by face pyramids about the
 * average of the face centres. */
int dugks_mesh_geometry(int32_t n_points, const double* points, int32_t n_faces,
                        const int64_t* face_offsets, const int64_t* face_points,
                        const int64_t* owner, int32_t n_internal, const int64_t* neighbour,
                        int32_t n_cells, double* face_centres, double* face_areas,
                        double* cell_centres, double* cell_volumes);

/* fvDVM::fvDVM, first half: mesh, DV set, gas, boundary conditions; builds
 * the least-squares vectors and the device layout.  fvDVM.C:1901-2110 */
int dugks_create(const dugks_mesh* mesh, const dugks_dv_set* dv, const dugks_gas* gas,
                 const dugks_bc* bc, const dugks_options* opt, dugks_handle** out);

/* Velocity-space sharding (the reference's -dvParallel with fieldMPIreducer,
 * fvDVM.C:381-383 and the reduceField calls of fvDVM.C:1241-1245,
 * :1547-1552, :1738-1740).  Rank r of world W owns a contiguous block of DV
 * rows (n_dv_1d DVs along x at fixed y, z): rows*r/W .. rows*(r+1)/W.  Its
 * g~, h~ and face values cover those DVs only; the raw face moments (after
 * the face reconstruction) and the raw cell moments (after the update) are
 * summed over all ranks, so every rank holds the same macros, which equal
 * the unsharded step's up to the summation order.  (The reference's own DV
 * decomposition leaves the face heat flux unreduced, fvDVM.C:1353-1356; it
 * is not followed there.)
 *   use_nccl != 0: the library all-reduces with NCCL on its own stream inside
 *       dugks_step, dugks_step_adaptive and dugks_set_state.  nccl_id is the
 *       NCCL unique id rank 0 made with dugks_nccl_unique_id and the host
 *       sent to every rank; dugks_create_sharded is collective (every rank
 *       calls it) and each rank drives its own GPU.  NCCL is loaded at this
 *       call (libnccl.so.2); without it the call fails with DUGKS_ERR_UNSUPPORTED.
 *   use_nccl == 0: the host reduces, through dugks_shard_phase. */
typedef struct dugks_dv_shard {
    int32_t rank;
    int32_t world;
    int32_t use_nccl;
    unsigned char nccl_id[128];
} dugks_dv_shard;

int dugks_nccl_unique_id(unsigned char id[128]);

/* dugks_create (shard NULL) or dugks_create_sharded with a DV list.  The
 * passes then evaluate each DV's Maxwellian with its own exponential (the
 * tensor-product factoring does not apply).  macroFlux yes takes the VMESH
 * branch (fvDVM.C:1562-1611): the cell rho, rho U, rho E advance by the
 * fluxes of the relaxed face DFs.  Not built for DV lists: symmetry patches
 * (the reference's VMESH build leaves their mirror ids unset), and
 * macroFlux yes on more than one shard. */
int dugks_create_dv_list(const dugks_mesh* mesh, const dugks_dv_list* dv, const dugks_gas* gas,
                         const dugks_bc* bc, const dugks_options* opt, const dugks_dv_shard* shard,
                         dugks_handle** out);
int dugks_create_sharded(const dugks_mesh* mesh, const dugks_dv_set* dv, const dugks_gas* gas,
                         const dugks_bc* bc, const dugks_options* opt, const dugks_dv_shard* shard,
                         dugks_handle** out);

/* First global DV index and number of DVs this handle holds (all of them
 * unless sharded).  dugks_get_state, dugks_set_state and dugks_get_df work
 * on these DVs only; macros and face values are global on every rank. */
int dugks_dv_range(const dugks_handle* h, int32_t* first_dv, int32_t* n_dv_local);

/* One step of a sharded handle with host-side reduction, in three calls:
 *   phase 0 (dt): face reconstruction and raw face moments of this shard;
 *   phase 1: face macros, face relaxation, update, raw cell moments (with a
 *            DV list and macro_flux, followed by the cell moments of the
 *            update's flux term);
 *   phase 2: cell macros; the step is complete.
 * After phases 0 and 1, *part / *n_part are a DEVICE buffer of doubles that
 * the host replaces, in place, by its sum over all shards before the next
 * phase (the stream is synchronised at the end of each phase).  Every shard
 * runs the same phases with the same dt. */
int dugks_shard_phase(dugks_handle* h, int32_t phase, double dt, double** part, int64_t* n_part);

/* fvDVM::fvDVM, second half: g~ = Maxwellian(rho,U,T), h~ = (K+3-D)RT g~,
 * wall inComingByRho, tau, q = 0, linear face velocity.
 * fvDVM.C:414-426, :578-624, :2115-2116.  U is [n_cells*3].  A non-finite
 * or non-positive rho or T, or a non-finite U, returns DUGKS_ERR_NAN and
 * leaves the handle as it was (the reference runs on into NaNs). */
int dugks_set_macros(dugks_handle* h, const double* rho, const double* U, const double* T);

/* n_steps calls of fvDVM::evolution() (fvDVM.C:2128-2174) with time steps
 * dt[0..n_steps-1]. */
int dugks_step(dugks_handle* h, int32_t n_steps, const double* dt);

/* Adjustable time step (controlDict adjustTimeStep yes): maxCo and
 * maxDeltaT as src/readTimeControlsExplicit.H:39-46 reads them. */
typedef struct dugks_adapt {
    double max_co;
    double max_delta_t;
} dugks_adapt;

/* n_steps iterations of the solver loop with an adjustable time step
 * (src/dugksFoam.C:71-80: CourantNo, setDeltaTvar, evolution).  Before each
 * step dt <- min(f dt, maxDeltaT), f = min(min(F, 1 + 0.1 F), 1.2),
 * F = maxCo / (CoNum + 1e-15), CoNum the Courant number of the current face
 * velocities at dt (src/setDeltaTvar.H:34-48, fvDVM.C:2177-2185).  The time
 * step is kept and updated on the device, so the call does not wait for
 * the host between steps.  *dt: in, the time step of the last step taken
 * (runTime.deltaTValue(), e.g. controlDict deltaT); out, the time step of
 * the last of these steps.  dt_history (may be NULL) receives the n_steps
 * time steps used. */
int dugks_step_adaptive(dugks_handle* h, int32_t n_steps, const dugks_adapt* adapt, double* dt, double* dt_history);

/* fvDVM::getCoNum (fvDVM.C:2177-2185) for time step dt, from the current
 * face velocities. */
int dugks_co_num(dugks_handle* h, double dt, double* co_max, double* co_mean);

/* Cell macros rho [n], U [n*3], T [n], q [n*3]; any pointer may be NULL. */
int dugks_get_macros(dugks_handle* h, double* rho, double* U, double* T, double* q);

/* Face macros of the last step (internal faces then boundary faces):
 * rhoSurf, Usurf, Tsurf, qSurf (fvDVM.C:1181-1300); any pointer may be NULL. */
int dugks_get_face_macros(dugks_handle* h, double* rho, double* U, double* T, double* q);

/* Boundary rho patch values: wall density of the last step on maxwellWall
 * faces, the fixed value on farField faces. [n_boundary_faces] */
int dugks_get_boundary_rho(dugks_handle* h, double* rho_b);

/* g~ (and h~) at the given cells for all DVs, [n][n_dv] row per cell
 * (fvDVM::writeDFonCell, fvDVM.C:1835-1890). h_out may be NULL. */
int dugks_get_df(dugks_handle* h, const int32_t* cells, int32_t n, double* g_out, double* h_out);

/* Whole state g~, h~ as DV-major [n_dv][n_cells] doubles, for exact
 * restart (the reference writes only macros and re-initialises the DFs to
 * the Maxwellian on restart, fvDVM.C:414-426).  dugks_set_state (after
 * dugks_set_macros) recomputes the cell macros from the given DFs as
 * fvDVM::updateMacroVol does (fvDVM.C:1528-1554, :1682-1742); dt_prev is
 * the time step that produced them (it enters the heat-flux correction).
 * DFs whose moments give a non-finite or non-positive rho or T return
 * DUGKS_ERR_NAN. */
int dugks_get_state(dugks_handle* h, double* g, double* hh);
int dugks_set_state(dugks_handle* h, const double* g, const double* hh, double dt_prev);

/* The record the next step starts from besides g~, h~: per cell (in the
 * mesh's cell order) rho, U[3], T, q[3], tau as the last step's moment sums
 * gave them, then the largest and the summed |U_f| + sqrt(D) xi_max over
 * delta_f of the internal faces (Courant number per unit time step), then
 * rho_b, T_b per boundary face (the pressure patches carry them from step
 * to step; T_b is restored on those faces only).  dugks_set_state recomputes the
 * cell part from the DFs in another summation order, which differs in the
 * last bits; setting the saved record after it makes a restart continue bit
 * for bit.  Length: dugks_step_record_size doubles (9 n_cells + 2 +
 * 2 n_boundary_faces).  dugks_set_step_record requires rho, T, tau > 0. */
int64_t dugks_step_record_size(const dugks_handle* h);
int dugks_get_step_record(dugks_handle* h, double* rec);
int dugks_set_step_record(dugks_handle* h, const double* rec);

/* Many independent cases stepped together (no counterpart in the
 * reference, which runs one case per dugksFoam process).  One CUDA graph
 * holds two steps of every handle, each handle a parallel branch on its own
 * stream, so that the tiles of small cases share the GPU; dugks_batch_step
 * replays it (an odd step count ends with one ordinary step per handle).
 * The handles must be initialised (dugks_set_macros), on one device and
 * unsharded; dt[i] is handle i's fixed time step.  Every handle's result is
 * bitwise the one dugks_step gives it alone.  A handle stays usable on its
 * own between batch steps; the batch holds no copy of its state. */
typedef struct dugks_batch dugks_batch;
int dugks_batch_create(dugks_handle* const* handles, int32_t n, const double* dt, dugks_batch** out);
int dugks_batch_step(dugks_batch* b, int32_t n_steps);
/* CUDA-event milliseconds of the last dugks_batch_step call (graph replays
 * only), and the kernels one replay of the two-step graph launches */
int dugks_batch_last_ms(const dugks_batch* b, double* ms);
int64_t dugks_batch_graph_kernels(const dugks_batch* b);
const char* dugks_batch_last_error(const dugks_batch* b);
void dugks_batch_destroy(dugks_batch* b);

/* Discrete adjoint of the FP64 step (no counterpart in the reference: it
 * differentiates fvDVM::evolution, fvDVM.C:2128-2174, in reverse mode).
 * The objective of a run of n_steps fixed-dt steps from the handle's
 * current state is the time average, over steps window_start .. n_steps-1,
 * of the energy and momentum flux through the boundary faces carried by the
 * relaxed boundary DFs of each step (the fluxes of fvDVM::updateGHtildeVol,
 * fvDVM.C:1500-1517):
 *   J_n = sum_b sum_i w_i (xi_i . Sf_b) [a_b (|xi_i|^2 g + h) / 2 + (c_b . xi_i) g]
 * a_b = energy_weight[b] (wall heat flux: 1 on the wall faces), c_b =
 * momentum_weight[3b..] (lid shear: (1,0,0) on the lid faces); NULL means 0.
 * The gradient is taken with respect to the T and U patch values of every
 * boundary face (boundary face b is mesh face n_internal_faces + b) and
 * muRef; Kn is proportional to muRef, so dJ/dKn = dJ/dmuRef muRef / Kn.
 * The start state counts as independent of the parameters.
 * States are checkpointed binomially (Griewank's revolve schedule) in
 * max_snapshots device copies of the state, so a run of N steps costs at
 * most r N forward steps with C(max_snapshots + r, r) >= N.
 * Supported: FP64, unsharded handles, maxwellWall and farField patches,
 * macroFlux no (DUGKS_ERR_UNSUPPORTED otherwise).  On return the handle
 * holds the state it started from. */
typedef struct dugks_objective {
    const double* energy_weight;    /* [n_boundary_faces] or NULL */
    const double* momentum_weight;  /* [n_boundary_faces * 3] or NULL */
    int32_t n_steps;                /* >= 1 */
    int32_t window_start;           /* 0 <= window_start < n_steps */
    double dt;                      /* fixed time step, > 0 */
    int32_t max_snapshots;          /* device state copies for the checkpoints, >= 1 */
    int32_t reserved[3];
} dugks_objective;

typedef struct dugks_adjoint_stats {
    int64_t forward_steps;   /* forward steps run, recomputations included */
    int64_t reverse_steps;   /* = n_steps */
    int32_t snapshots;       /* state copies allocated */
    int32_t reserved;
    double ms_total;         /* CUDA-event milliseconds of the whole run */
    double ms_forward;       /* of which the forward steps */
    double device_bytes;     /* device memory the run allocated */
} dugks_adjoint_stats;

/* J, dJ_dT_b [n_boundary_faces], dJ_dU_b [n_boundary_faces * 3] and
 * dJ_dmu_ref are host outputs (any may be NULL); stats may be NULL. */
int dugks_adjoint_run(dugks_handle* h, const dugks_objective* obj, double* J, double* dJ_dT_b, double* dJ_dU_b,
                      double* dJ_dmu_ref, dugks_adjoint_stats* stats);

/* The objective alone: a forward run of obj->n_steps steps (the handle
 * advances by n_steps) that evaluates J as dugks_adjoint_run defines it;
 * max_snapshots is not used.  For finite-difference checks and line
 * searches. */
int dugks_objective_run(dugks_handle* h, const dugks_objective* obj, double* J, dugks_adjoint_stats* stats);

/* The forward steps a dugks_adjoint_run of n_steps with n_snapshots state
 * copies runs (recomputation included), from its checkpoint schedule alone;
 * no device work.  -1 on bad arguments or an inconsistent schedule. */
int64_t dugks_checkpoint_forward_steps(int32_t n_steps, int32_t n_snapshots);

/* Fluxes through every boundary face of the step a dugks_step(dt) from the
 * current state would take, from the relaxed boundary DFs that its update
 * uses (fvDVM::updateGHtildeVol, fvDVM.C:1500-1517); along Sf, i.e. out of
 * the gas: flux[5b..5b+4] = sum_i w_i (xi_i.Sf) {g, xi_x g, xi_y g, xi_z g,
 * (|xi|^2 g + h)/2} -- mass, momentum and energy per second.  A wall's drag
 * is the sum of its faces' momentum fluxes, its heat load the sum of their
 * energy fluxes.  The state does not advance.  FP64, unsharded handles with
 * maxwellWall and farField patches (the dugks_adjoint_run restrictions). */
int dugks_boundary_fluxes(dugks_handle* h, double dt, double* flux);

/* The launch layout dugks_create chose: cells per tile (after shrinking
 * to fit), number of tiles and DV chunks per tile.  An autotuner reads it
 * to scale dugks_options.tile_cells / dv_chunks from the automatic choice. */
int dugks_layout(const dugks_handle* h, int32_t* tile_cells, int32_t* n_tiles, int32_t* dv_chunks);

/* Number of discrete velocities (nDV^D). */
int32_t dugks_n_dv(const dugks_handle* h);

/* Wall-clock of the kernels of the last dugks_step call, in milliseconds,
 * measured with CUDA events on the handle's stream. */
int dugks_last_step_ms(dugks_handle* h, double* ms);

/* dugks_step with CUDA events around every kernel stage on the handle's
 * stream; stage_ms[0..4] receive the summed milliseconds of pass A (face
 * reconstruction and moments), the face combine, pass B (relaxation, flux,
 * update, cell moments), the cell combine, and the whole call. */
int dugks_step_timed(dugks_handle* h, int32_t n_steps, const double* dt, double* stage_ms);

/* Number of kernels this handle has launched so far. */
int64_t dugks_kernel_launches(const dugks_handle* h);

const char* dugks_last_error(const dugks_handle* h);
void dugks_destroy(dugks_handle* h);

/* Cell macros of caller-owned device DFs without any device allocation.
 * No counterpart in the reference: it is the reduction of dugks_set_state
 * (fvDVM::updateMacroVol, fvDVM.C:1528-1554, :1682-1742) for callers that
 * cannot allocate -- a monitor or post-processing step between time steps,
 * on its own stream, next to a solver that has taken the device memory up
 * front: cudaMalloc would fail there, and cudaFree synchronises the whole
 * device and stalls the solver's queued work.  Its scratch is a fixed
 * 16 MiB device array inside this library.
 *   n_dims, n_dv, xi [n_dv*3], w [n_dv]: the DV set, as dugks_get_state's
 *       DV order uses it (x fastest); g, hh: DV-major [n_dv][n_cells] FP64;
 *   gas, dt: as dugks_create's gas and the time step that produced g, hh
 *       (it enters the heat-flux factor 2 tau/(2 tau + dt Pr));
 *   rho [n], U [n*3], T [n], q [n*3]: outputs, any may be NULL.
 * xi, w, g, hh and the outputs are DEVICE pointers of the current device
 * (others are rejected); gas is a host pointer; stream is a cudaStream_t
 * (NULL: the default stream); the call only enqueues work on it.  msg
 * (msg_len bytes, may be NULL) receives the error text.
 * Each pointer's allocation must have room for what is read or written
 * there (DUGKS_ERR_ARG otherwise, before any launch).
 * Limits: n_cells <= 131072 per call (DUGKS_ERR_ARG beyond).  The first call
 * on a device looks up the scratch address and caches it per CUDA context
 * (a reset device is looked up again): make the first call in a context
 * before any stream capture on that device.  Nothing has to start at zero.
 * Calls that overlap in time on one device share the scratch and race:
 * serialise them. */
int dugks_cell_macros_noalloc(int32_t n_dims, int32_t n_dv, const double* xi, const double* w, int32_t n_cells,
                              const double* g, const double* hh, const dugks_gas* gas, double dt, double* rho,
                              double* U, double* T, double* q, void* stream, char* msg, int32_t msg_len);

#ifdef __cplusplus
}
#endif
#endif

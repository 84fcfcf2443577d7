// Internal declarations of the B200 DUGKS step library: device layout,
// per-tile stencil tables and the handle.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "dugks.h"

namespace dugks {

constexpr int kThreads = 512;      // threads per CTA of the two tile passes
constexpr int kMaxTile = 128;      // cells per tile (L0) at most
constexpr int kMaxLocal = 256;     // L0 + L1 cells per tile at most
constexpr int kMaxItems = kThreads - 1;  // items per tile at most (one per thread; one flux slot kept zero)
constexpr int kMaxN1d = 64;        // DV nodes per dimension at most
constexpr int kNM = 16;            // stride of a partial-moment record (doubles)
constexpr int kFX = 8;             // stride of a flux-moment record: M0, M1[3], W/2
constexpr double kVSmall = 1.0e-300;  // OpenFOAM VSMALL (upwind switch, fvDVM.C:829-847)

// Moment record layout (raw velocity moments of one face or cell, summed
// over DVs; a = w g, b = w h, u = a|xi|^2 + b):
//   0 M0 = sum a            1..3  M1 = sum a xi
//   4 W  = sum u            5..7  V3 = sum u xi
//   8..13 M2 = sum a xi xi (xx xy xz yy yz zz)
//   14 outgoing wall flux  sum_{xi.S>0} w (xi.S) gbar   (faces only)
enum {
    MOM_M0 = 0, MOM_M1 = 1, MOM_W = 4, MOM_V3 = 5, MOM_M2 = 8, MOM_OUT = 14
};

// item kinds of a tile (faces touching the tile's own cells); a tile lists
// its items sorted by kind so that warps see one kind at a time
enum : int32_t {
    ITEM_TILE_INTERNAL = 0,   // owner and neighbour both in the tile
    ITEM_TB_OWN = 1,          // tile-boundary face, owner side in the tile
    ITEM_TB_NEI = 2,          // tile-boundary face, neighbour side in the tile
    ITEM_MESH_BOUNDARY = 3    // boundary face of a non-empty patch
};

// Record fields of the structure-of-arrays coefficient tables.  Cell
// records (gbar+ half step, fvDVM.C:668-679) and face records (face
// relaxation, fvDVM.C:1374-1444) share the layout: field k of entity e is
// rec[k * n + e].
enum {
    REC_UX = 0, REC_UY = 1, REC_UZ = 2,
    REC_INVRT = 3,   // 1/(R T)
    REC_A = 4,       // rho (2 pi R T)^(-D/2)
    REC_R = 5,       // relax factor: cells 1.5 dt/(2 tau + dt), faces 0.5 dt/(2 tau + 0.5 dt)
    REC_QX = 6, REC_QY = 7, REC_QZ = 8,   // (1-Pr) q / (5 rho (R T)^2)
    REC_RTH = 9,     // R T used by h^S (boundary faces: the internal-face T at the patch-local index)
    REC_N = 10
};

// Incoming-DF parameters of a mesh-boundary face: g_in = rho_in K_in exp(-|U_in - xi|^2 invRT_in / 2),
// h_in = g_in * hfac (fvDVM.C:926-938, :1079-1092).
struct __align__(16) BRec {
    double U[3];       // wall and mixed: patch velocity (farField: the owner-cell U is taken)
    double K_in;       // (2 pi R T_in)^(-D/2)
    double invRT_in;
    double hfac;       // R T_in (K+3-D)
    double rho_in;     // farField, mixed: fixed patch rho; wall: rho_w of the current step;
                       // pressureIn/Out: updated after each step
    double inByRho;    // wall: inComingByRho
    double T;          // T_in
    double p;          // pressureIn / pressureOut value
};

// Device-side view of everything the kernels read.
struct DevMesh {
    int D, K;
    double R, Pr, omega, Tref, muRef;
    int nC, nIF, nBF, nv, n_tiles;
    // DVs this device holds: global DVs dv_base .. dv_base + nv_loc - 1, the
    // DV rows row_base ..; the state and face-value arrays are [nv_loc][..]
    int nv_loc, dv_base, row_base;
    int prec;              // dugks_precision of the state and tables
    // DV set
    const double* xi;      // [nv*3]
    const double* w;       // [nv]
    int n1d;               // nodes per dimension; DV d = (iz n + iy) n + ix
    int general_dv;        // 1: a DV list that is no tensor product (n1d is 1, a "row" is one DV)
    const double* X1;      // [n1d] one-dimensional nodes
    const double* W1;      // [n1d] one-dimensional weights
    // tiles
    const int32_t* tile_begin;     // [n_tiles+1] L0 = [begin, begin+n0) (renumbered cells)
    const int32_t* tile_loc_off;   // [n_tiles+1] into loc_cells
    const int32_t* loc_cells;      // local cells (L0 then L1), renumbered ids
    const int32_t* tile_item_off;  // [n_tiles+1] into the item arrays
    // items (structure of arrays over all tiles' items)
    const int32_t* it_meta;        // kind | ptype << 4
    const int32_t* it_loc;         // lo | ln << 16 (0xffff: none); local indices
    const int32_t* it_face;        // internal face id, or boundary face id
    const int32_t* it_other;       // tile-boundary items: the item of the face's other side
    const double* it_geo;          // [9][n_items]: S, Cf - C_own, Cf - C_nei
    // gradient stencils and flux lists, slot-major [slot][cell]
    int nb_max, nf_max;
    const int32_t* grad_nb;        // [nb_max][nC] local index of the neighbour, -1: none
    const double* grad_ls;         // [nb_max][3][nC] least-squares vector
    const int32_t* cf_item;        // [nf_max][nC] (local item + 1) * (+1 nei / -1 own), 0: none
    const double* dtV;             // 1/V per renumbered cell
    // combine maps
    const int32_t* face_items;     // [nF*2] global item ids of each face (-1 none)
    const int32_t* bface_patch_local;  // [nBF] index within its patch
    const int32_t* bface_ptype;    // [nBF]
    const int32_t* bface_owner;    // [nBF] renumbered owner cell
    const int32_t* bface_mirror;   // [nBF] symmetry faces: mirrored DV axis 0..2; -1 otherwise
    int n_sym_faces, n_pressure_faces;
    // macroFlux yes: faces of each (renumbered) cell in face order, entry
    // f * 2 + (1 if the cell is the neighbour); face area vectors and volumes
    int macro_flux;
    const int32_t* mf_off;         // [nC+1]
    const int32_t* mf_ent;         // [2 nIF + nBF]
    const double* mf_Sf;           // [nF*3]
    const double* mf_V;            // [nC] renumbered
    const double* dc;              // [nIF] deltaCoeffs
    const double* bS;              // [nBF*3] boundary face area vectors
    int n_items;
    double xi_max_co;              // sqrt(D) * xiMax
    // FP32 storage of a tensor DV set: g~, gbar+, the face values and the
    // fluxes are stored as deviations from a per-DV reference Maxwellian,
    // g = stored + gref[d] (h likewise), so that FP32 rounding acts on the
    // deviation only; null for FP64 and for DV lists (absolute storage)
    const double* gref;            // [nv_loc] local DVs
    const double* href;
};

// Mutable device state
struct DevState {
    void* g[2];        // state g~ [nv][nC] (Real); g[1] aliases g[0]: pass B updates in place
    void* h[2];
    int cur;
    // face values [nv][n_items] (Real): pass A's upwind reconstruction at the
    // half step of every item, weighted by the side's share on tile-boundary
    // faces; pass B relaxes them instead of reconstructing again
    void* fvg;
    void* fvh;
    double* partF;     // [chunks][n_items][kNM]
    double* partC;     // [chunks][nC][kNM]
    double* partX;     // [chunks][nC][kFX] DV-list macroFlux: moments of the flux term (else null)
    double* redC;      // sharded DV-list macroFlux: [nC][kNM] cell moments then [nC][kFX] flux moments, reduced together
    double* cellrec;   // [REC_N][nC]
    // face records in item order (each face's record is written to its one
    // or two items, so that a tile reads its faces' records contiguously)
    double* facerec;   // [REC_N][n_items]
    // one-dimensional Maxwellian factors, FP64 for both precisions (the
    // equilibrium and the relaxation are evaluated in FP64, so that the FP32
    // path injects no rounding bias into the conserved moments): table k of
    // entity e at node i is tab[(k * n1d + i) * n + e] = exp(-(X_i - U_k)^2 /
    // (2 R T)), the x table multiplied by A = rho (2 pi R T)^(-D/2)
    double* ctab;      // [D][n1d][nC]
    double* ftab;      // [D][n1d][n_items]  (item order, as facerec)
    BRec* brec;        // [nBF]
    double* bmom_in;   // [nBF][kNM] incoming wall moments per unit rho_w
    double* cm;        // cell macros [nC][9]: rho U(3) T q(3) tau (renumbered)
    // FP32 storage of a tensor DV set: the raw moments of the reference
    // Maxwellian over each DV chunk, [chunks][kNM] (null otherwise); a face
    // or cell whose DVs all count in full adds them once instead of per DV
    double* refmom;
    double* fm;        // face macros [nF][9]
    double* co;        // [2] Courant max (as ordered bits) and sum
    int* err;          // [4] device error flags
};

struct Tiling {
    int n_tiles = 0;
    int tile_cells = 0;
    int max_local = 0, max_l0 = 0, max_items = 0;
    int nb_max = 0, nf_max = 0;
    std::vector<int32_t> perm;      // new -> old cell
    std::vector<int32_t> iperm;     // old -> new
    std::vector<int32_t> tile_begin, tile_loc_off, loc_cells, tile_item_off;
    std::vector<int32_t> it_meta, it_loc, it_face, it_other;
    std::vector<double> it_geo;     // [9][n_items]
    std::vector<int32_t> grad_nb;   // [nb_max][nC]
    std::vector<double> grad_ls;    // [nb_max][3][nC]
    std::vector<int32_t> cf_item;   // [nf_max][nC]
    std::vector<int32_t> face_items;
    int n_items() const { return static_cast<int>(it_meta.size()); }
};

}  // namespace dugks

struct dugks_handle {
    int device = 0;
    int precision = DUGKS_FP64;
    int D = 3;
    int nC = 0, nIF = 0, nBF = 0, nP = 0, nv = 0, n1d = 0;
    dugks_gas gas{};
    double xi_max = 0;
    std::vector<int32_t> patch_type, patch_start;
    std::vector<int32_t> bface_ptype, bface_patch_local;
    std::vector<double> bc_rho, bc_U, bc_T, bc_p;
    std::vector<int32_t> bface_mirror;   // symmetry faces: mirrored DV axis; -1 otherwise
    std::vector<double> xi, w;      // tensor-product DV set
    std::vector<double> X1, W1;     // one-dimensional nodes and weights
    std::vector<double> gref, href; // host copy of the FP32-storage reference (empty: none)
    // geometry (original numbering)
    std::vector<int64_t> owner, neighbour;
    std::vector<double> C, V, Cf, Sf, weights, dc, lsP, lsN, lsB;
    dugks::Tiling tiling;
    int chunks = 1;
    std::vector<int32_t> chunk_begin;   // DV chunk boundaries in global DV rows [chunks+1]
    // velocity-space shard (world 1: the whole DV set)
    int shard_rank = 0, shard_world = 1;
    bool shard_nccl = false;
    void* nccl_comm = nullptr;          // ncclComm_t
    int shard_phase_next = 0;           // dugks_shard_phase: the phase expected next
    double shard_dt = 0;                // dugks_shard_phase: dt of the step in progress
    // device
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    dugks::DevMesh dm{};
    dugks::DevState ds{};
    std::vector<void*> allocations;
    int32_t* d_chunk_begin = nullptr;
    double* d_dt = nullptr;         // [2] device time steps of adaptive stepping (ping-pong)
    double* d_hist = nullptr;       // time steps of the last adaptive call
    int32_t hist_cap = 0;
    bool initialised = false;
    // h~ is identically zero: D = 3 and KInner = 0 make K + 3 - D = 0 in
    // every formula that feeds h (initial state, equilibria, boundary
    // DFs), so h stays zero unless dugks_set_state loads a nonzero h~
    bool h_zero = false;
    double cellrec_dt = 0;          // time step the cell records' relax factors were built for
    long steps_done = 0;
    int64_t launches = 0;           // kernels launched by this handle
    double last_step_ms = 0;
    double* host_cm = nullptr;      // pinned staging of the cell macros (dugks_get_macros)
    std::string last_error;
};

namespace dugks {
// host preparation (dugks_host.cpp)
void compute_weights_and_ls(dugks_handle* h, int weighting);
void build_tiling(dugks_handle* h, int tile_cells);
int set_error(dugks_handle* h, int code, const std::string& msg);
// ABI helper (dugks_abi.cpp): cell records and tables from ds.cm
int rebuild_cell_records(dugks_handle* h);
// pass A of a step of size dt from the current state: the face-value buffer
// then holds the step's upwind face values at the half step
int record_face_values(dugks_handle* h, double dt);
}  // namespace dugks

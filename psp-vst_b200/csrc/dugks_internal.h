// Internal declarations of the B200 DUGKS step library: device layout,
// per-tile stencil tables and the handle.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "dugks.h"

namespace dugks {

constexpr int kThreads = 256;      // threads per CTA of the two tile passes
constexpr int kNM = 16;            // stride of a partial-moment record (doubles)
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

// item kinds of a tile (faces touching the tile's own cells)
enum : int32_t {
    ITEM_TILE_INTERNAL = 0,   // owner and neighbour both in the tile
    ITEM_TB_OWN = 1,          // tile-boundary face, owner side in the tile
    ITEM_TB_NEI = 2,          // tile-boundary face, neighbour side in the tile
    ITEM_MESH_BOUNDARY = 3    // boundary face of a non-empty patch
};

// One face as seen from a tile.  Geometry is stored per item so that a tile
// reads a contiguous block.
struct __align__(16) Item {
    int32_t kind;
    int32_t lo;        // local index of the owner (-1 if outside the tile's L0+L1)
    int32_t ln;        // local index of the neighbour (-1 for boundary faces)
    int32_t face;      // internal face id, or boundary face id for mesh-boundary items
    int32_t xb_w;      // XB slot this tile writes (tile-boundary items)
    int32_t xb_r;      // XB slot of the other side this tile reads
    int32_t ptype;     // patch type (mesh-boundary items)
    int32_t pad;
    double S[3];       // face area vector
    double dO[3];      // Cf - C_owner
    double dN[3];      // Cf - C_neighbour (internal faces)
};

// Per-cell coefficients of the Shakhov equilibrium used by the gbar+
// half-step (fvDVM.C:668-679).  Rewritten after each cell-moment pass.
struct __align__(16) CellRec {
    double U[3];
    double invRT;      // 1/(R T)
    double A;          // rho (2 pi R T)^(-D/2)
    double r;          // 1.5 dt / (2 tau + dt)
    double qv[3];      // (1-Pr) q / (5 rho (R T)^2)
    double RT;
};

// Face coefficients for the face relaxation (fvDVM.C:1374-1444).
struct __align__(16) FaceRec {
    double U[3];
    double invRT;
    double A;
    double r;          // 0.5 dt / (2 tau + 0.5 dt)
    double qv[3];
    double RTh;        // R T used by h^S; boundary faces: internal face T at the patch-local index
};

// Incoming-DF parameters of a mesh-boundary face: g_in = rho_in K_in exp(-|U_in - xi|^2 invRT_in / 2),
// h_in = g_in * hfac (fvDVM.C:926-938, :1079-1092).
struct __align__(16) BRec {
    double U[3];       // wall velocity (farField: unused, the owner-cell U is taken)
    double K_in;       // (2 pi R T_in)^(-D/2)
    double invRT_in;
    double hfac;       // R T_in (K+3-D)
    double rho_in;     // farField: fixed patch rho; wall: rho_w of the current step
    double inByRho;    // wall: inComingByRho
};

// Device-side view of everything the kernels read.
struct DevMesh {
    int D, K;
    double R, Pr, omega, Tref, muRef;
    int nC, nIF, nBF, nv, n_tiles;
    // DV set
    const double* xi;      // [nv*3]
    const double* w;       // [nv]
    // tiles
    const int32_t* tile_begin;     // [n_tiles+1] L0 = [begin, begin+n0) (renumbered cells)
    const int32_t* tile_loc_off;   // [n_tiles+1] into loc_cells
    const int32_t* loc_cells;      // local cells (L0 then L1), renumbered ids
    const int32_t* tile_item_off;  // [n_tiles+1] into items
    const Item* items;
    // gradient stencil per renumbered cell
    const int32_t* grad_off;       // [nC+1]
    const int32_t* grad_nb;        // local index (within the cell's tile)
    const double* grad_ls;         // [*3]
    // flux gather per renumbered cell: local item indices with sign (+1 nei, -1 own)
    const int32_t* cf_off;         // [nC+1]
    const int32_t* cf_item;        // signed: (item+1) * sign
    const double* dtV;             // 1/V per renumbered cell
    // combine maps
    const int32_t* face_items;     // [nF*2] global item ids of each face (-1 none)
    const int32_t* bface_patch_local;  // [nBF] index within its patch
    const int32_t* bface_ptype;    // [nBF]
    const int32_t* bface_owner;    // [nBF] renumbered owner cell
    const double* dc;              // [nIF] deltaCoeffs
    const double* bS;              // [nBF*3] boundary face area vectors
    int n_items;
    int n_tbf;
    double xi_max_co;              // sqrt(D) * xiMax
};

// Mutable device state
struct DevState {
    void* g[2];        // state g~ double buffer [nv][nC] (Real)
    void* h[2];
    int cur;
    void* xbg[2];      // XB buffers [side][nv][n_tbf]
    void* xbh[2];
    double* partF;     // [chunks][n_items][kNM]
    double* partC;     // [chunks][nC][kNM]
    CellRec* cellrec;  // [nC]
    FaceRec* facerec;  // [nIF+nBF]
    BRec* brec;        // [nBF]
    double* bmom_in;   // [nBF][kNM] incoming wall moments per unit rho_w
    double* cm;        // cell macros [nC][9]: rho U(3) T q(3) tau (renumbered)
    double* fm;        // face macros [nF][9]
    double* co;        // [2] Courant max (as ordered bits) and sum
    int* err;          // [4] device error flags
};

struct Tiling {
    int n_tiles = 0;
    int tile_cells = 0;
    int max_local = 0, max_l0 = 0, max_items = 0;
    std::vector<int32_t> perm;      // new -> old cell
    std::vector<int32_t> iperm;     // old -> new
    std::vector<int32_t> tile_begin, tile_loc_off, loc_cells, tile_item_off;
    std::vector<Item> items;
    std::vector<int32_t> grad_off, grad_nb;
    std::vector<double> grad_ls;
    std::vector<int32_t> cf_off, cf_item;
    std::vector<int32_t> face_items;
    int n_tbf = 0;
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
    std::vector<double> bc_rho, bc_U, bc_T;
    std::vector<double> xi, w;      // tensor-product DV set
    // geometry (original numbering)
    std::vector<int64_t> owner, neighbour;
    std::vector<double> C, V, Cf, Sf, weights, dc, lsP, lsN, lsB;
    dugks::Tiling tiling;
    int chunks = 1;
    std::vector<int32_t> chunk_begin;   // DV chunk boundaries [chunks+1]
    // device
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    dugks::DevMesh dm{};
    dugks::DevState ds{};
    std::vector<void*> allocations;
    int32_t* d_chunk_begin = nullptr;
    bool initialised = false;
    double cellrec_dt = 0;          // time step the cell records' relax factors were built for
    long steps_done = 0;
    int64_t launches = 0;           // kernels launched by this handle
    double last_step_ms = 0;
    std::string last_error;
};

namespace dugks {
// host preparation (dugks_host.cpp)
void compute_weights_and_ls(dugks_handle* h, int weighting);
void build_tiling(dugks_handle* h, int tile_cells);
int set_error(dugks_handle* h, int code, const std::string& msg);
}  // namespace dugks

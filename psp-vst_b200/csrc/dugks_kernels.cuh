// Launch interface of the DUGKS step kernels (dugks_kernels.cu).
#pragma once

#include "dugks_internal.h"

namespace dugks {

struct StepArgs {
    DevMesh dm;
    DevState ds;
    double dt;
    int chunks;
    const int32_t* chunk_begin;  // [chunks+1] DV rows
    double dt_next;              // time step of the following step (0 = unknown)
    // device-resident time steps (adaptive stepping): when set, the kernels
    // read this step's dt from *dtp and the next step's from *dtnp instead of
    // dt and dt_next
    const double* dtp;
    const double* dtnp;
    int wideA, wideB;            // batch width of each pass: 1 wide, 0 narrow
    // 1: h is identically zero (3-D, KInner = 0, h~ = 0 in the state): the
    // tensor-DV passes carry g alone
    int hzero;
    int wideA16;                 // g-only pass A in batches of 16 DVs (16 nodes per dimension)
    int wideB16;                 // g-only pass B likewise (FP32 storage)
    int row10;                   // g-only passes in batches of 10 DVs (20 nodes per dimension)
    int row20;                   // FP32 storage: g-only passes in batches of a whole 20-node row
    int fullA, fullB;            // 1: every DV row splits into whole batches
    size_t smemA, smemB;         // dynamic shared memory of the passes
};

enum { STAGE_PASS_A = 0, STAGE_FACE_COMBINE = 1, STAGE_PASS_B = 2, STAGE_CELL_COMBINE = 3 };

// Bounds-checked build (-DDUGKS_CHECK, libdugks_b200_check.so): every index
// the kernels read from a device table is tested against its range before
// use.  One outside [lo, hi) sets bit 2 (value 4) of the handle's error
// flags and is replaced by lo, so the access stays in bounds; the host then
// returns DUGKS_ERR_ARG.  In the normal build the check is the index itself.
#ifdef DUGKS_CHECK
__device__ __forceinline__ int chk(int i, int lo, int hi, int* err) {
    if (i < lo || i >= hi) {
        atomicOr(err, 4);
        return lo;
    }
    return i;
}
#else
__device__ __forceinline__ int chk(int i, int, int, int*) { return i; }
#endif

// one DUGKS step (fvDVM::evolution) on the handle's stream, or one stage
// of it; `launches` (may be null) is incremented by the kernels launched
cudaError_t launch_step(const StepArgs& a, int precision, cudaStream_t s, int* launches);
cudaError_t launch_stage(const StepArgs& a, int precision, int stage, cudaStream_t s, int* launches);
// r = 1.5 dt / (2 tau + dt) for every cell record
cudaError_t launch_cell_prep(const StepArgs& a, cudaStream_t s);
// g~, h~ = Maxwellian; wall inComingByRho and incoming-moment vectors
cudaError_t launch_init(const StepArgs& a, int precision, cudaStream_t s);
// cell macros from the current state (raw moments over all DVs, then the
// cell combine with time step dt for the heat-flux correction)
cudaError_t launch_state_macros(const StepArgs& a, int precision, cudaStream_t s);
// dt of the next step from the Courant number of this step's faces (in
// ds.co) and dt_in, as src/setDeltaTvar.H:34-48 adjusts it; also stored to
// *hist when hist is not null
// raw cell moments of the state (this device's DVs) into partC chunk 0, and
// the cell macros and records from partC chunk 0
cudaError_t launch_state_moments(const StepArgs& a, int precision, cudaStream_t s);
cudaError_t launch_cell_combine_one(const StepArgs& a, double dt_next, cudaStream_t s);
// partial moments of all chunks summed into chunk 0 (n doubles per chunk)
cudaError_t launch_sum_chunks(double* part, int chunks, size_t n, cudaStream_t s);
// cell records and Maxwellian tables rebuilt from the cell macros
cudaError_t launch_cell_records(const StepArgs& a, cudaStream_t s);
cudaError_t launch_adapt(const StepArgs& a, const double* dt_in, double* dt_out, double* hist, double max_co,
                         double max_dt, cudaStream_t s);
// one of the two tile passes (dugks_passes.cu)
cudaError_t launch_pass(const StepArgs& a, int precision, bool pass_b, cudaStream_t s);
// batch widths and dynamic shared memory of the passes for a DV set of n1d
// nodes per dimension
void pass_config(int D, int precision, int n1d, StepArgs* a);
cudaError_t configure_kernels(int precision, const StepArgs& a);

}  // namespace dugks

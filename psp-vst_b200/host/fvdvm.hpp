// dugks_host::FvDVM: the public interface of dugksFoam's Foam::fvDVM
// (src/fvDVM/fvDVM/fvDVM.H:80-409) over the B200 C ABI (include/dugks.h),
// for hosts without OpenFOAM.  The macro fields live on the host, the
// distribution functions on the GPU.
//
//   fvDVM(rho, U, T, ...)        FvDVM(const Case&, options)     fvDVM.C:1901-2117
//   evolution()                  evolution(dt)                    fvDVM.C:2128-2174
//   getCoNum(maxCo, meanCo)      getCoNum(dt, maxCo, meanCo)      fvDVM.C:2177-2185
//   rhoVol() Uvol() Tvol() qVol()  same names (host arrays)       fvDVM.H:338-352
//   writeDFonCell(s)             dfOnCells(cells, g, h)           fvDVM.C:1835-1897
//   nXi() nXiPerDim()            same names                       fvDVM.H:373-376
//
// The reference stops the program on errors (FatalError); FvDVM throws
// FvDVMError with the library's message instead.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "dugks.h"
#include "foam_case.hpp"

namespace dugks_host {

struct FvDVMError : std::runtime_error {
    int status;
    FvDVMError(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

class FvDVM {
public:
    // precision: DUGKS_FP64 or DUGKS_FP32C; device: CUDA ordinal
    explicit FvDVM(const Case& c, int precision = DUGKS_FP64, int device = 0);
    ~FvDVM();
    FvDVM(const FvDVM&) = delete;
    FvDVM& operator=(const FvDVM&) = delete;

    // one DUGKS step of size dt; refreshes the host macro fields
    void evolution(double dt);
    // CourantNo.H + setDeltaTvar.H + evolution() (src/dugksFoam.C:65-75):
    // dt (the previous step's) is adjusted on the device to hold maxCo and
    // returned as the step taken
    void evolutionAdjustable(double& dt, double maxCo, double maxDeltaT);
    void getCoNum(double dt, double& maxCo, double& meanCo) const;

    const std::vector<double>& rhoVol() const { return rho_; }
    const std::vector<double>& Uvol() const { return U_; }
    const std::vector<double>& Tvol() const { return T_; }
    const std::vector<double>& qVol() const { return q_; }
    // face macros of the last step (internal faces, then boundary faces)
    void surfMacros(std::vector<double>& rho, std::vector<double>& U, std::vector<double>& T,
                    std::vector<double>& q) const;
    // wall density of the last step on wall faces, the fixed value on far-field faces
    std::vector<double> boundaryRho() const;
    // g~ and h~ of the given cells, [cells][nXi] (fvDVM::writeDFonCell)
    void dfOnCells(const std::vector<int32_t>& cells, std::vector<double>& g, std::vector<double>& h) const;

    // Exact restart file (no reference counterpart: dugksFoam re-initialises
    // the DFs to the Maxwellian of the written macros, fvDVM.C:414-426).
    // Binary, native byte order: the 8 bytes "DUGKSST2", int32 D, int32 n1d,
    // int64 n_cells, int64 n_dv, double dt_prev, double time, then g~ and h~
    // as DV-major [n_dv][n_cells] doubles in the case's cell numbering, then
    // the step record (dugks_get_step_record: 9 n_cells + 2 doubles).
    // dt_prev is the step that produced the state (it enters the cell heat
    // flux); readState restores the state, the cell macros and the Courant
    // sums exactly, so that the run continues bit for bit, and returns
    // dt_prev and time.
    void writeState(const std::string& path, double dt_prev, double time) const;
    void readState(const std::string& path, double& dt_prev, double& time);

    int nXi() const { return n_xi_; }
    int nXiPerDim() const { return static_cast<int>(case_.xis.size()); }
    const FlatMesh& mesh() const { return flat_; }
    const Case& caseData() const { return case_; }

private:
    void check(int st, const char* what) const;
    void refresh();

    Case case_;
    FlatMesh flat_;
    dugks_handle* h_ = nullptr;
    int n_xi_ = 0;
    std::vector<double> rho_, U_, T_, q_;
};

}  // namespace dugks_host

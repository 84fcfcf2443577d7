// dugks_host::FvDVM (see fvdvm.hpp).
#include "fvdvm.hpp"

#include <cstdio>
#include <cstring>

namespace dugks_host {

FvDVM::FvDVM(const Case& c, int precision, int device) : case_(c), flat_(flatten(c)) {
    const FlatMesh& f = flat_;
    dugks_mesh mesh{f.n_cells,     f.n_internal,  f.n_boundary,
                    f.D,           f.owner.data(), f.neighbour.data(),
                    f.C.data(),    f.V.data(),    f.Cf.data(),
                    f.Sf.data(),   static_cast<int32_t>(f.patch_type.size()), f.patch_start.data()};
    dugks_dv_set dv{static_cast<int32_t>(case_.xis.size()), case_.xis.data(), case_.weights.data(), case_.xi_max};
    dugks_gas gas{case_.R, case_.omega, case_.Tref, case_.mu_ref, case_.Pr, case_.K_inner};
    dugks_bc bc{f.patch_type.data(), f.rho_b.data(), f.U_b.data(), f.T_b.data(), f.p_b.data()};
    dugks_options opt;
    dugks_default_options(&opt);
    opt.precision = precision;
    opt.device = device;
    opt.macro_flux = case_.macro_flux ? 1 : 0;
    int st;
    if (!case_.dv_w.empty()) {
        const dugks_dv_list dl{static_cast<int32_t>(case_.dv_w.size()), case_.dv_xi.data(), case_.dv_w.data(),
                               case_.xi_max};
        st = dugks_create_dv_list(&mesh, &dl, &gas, &bc, &opt, nullptr, &h_);
    } else {
        st = dugks_create(&mesh, &dv, &gas, &bc, &opt, &h_);
    }
    if (st != DUGKS_OK) {
        const std::string msg = h_ ? dugks_last_error(h_) : "dugks_create failed";
        if (h_) dugks_destroy(h_);
        h_ = nullptr;
        throw FvDVMError(st, msg);
    }
    n_xi_ = dugks_n_dv(h_);
    check(dugks_set_macros(h_, case_.rho0.data(), case_.U0.data(), case_.T0.data()), "dugks_set_macros");
    rho_ = case_.rho0;
    U_ = case_.U0;
    T_ = case_.T0;
    q_.assign(3 * static_cast<size_t>(f.n_cells), 0.0);
}

FvDVM::~FvDVM() {
    if (h_) dugks_destroy(h_);
}

void FvDVM::check(int st, const char* what) const {
    if (st != DUGKS_OK) throw FvDVMError(st, std::string(what) + ": " + dugks_last_error(h_));
}

void FvDVM::refresh() {
    check(dugks_get_macros(h_, rho_.data(), U_.data(), T_.data(), q_.data()), "dugks_get_macros");
}

void FvDVM::evolution(double dt) {
    check(dugks_step(h_, 1, &dt), "dugks_step");
    refresh();
}

void FvDVM::evolutionAdjustable(double& dt, double maxCo, double maxDeltaT) {
    const dugks_adapt ad{maxCo, maxDeltaT};
    check(dugks_step_adaptive(h_, 1, &ad, &dt, nullptr), "dugks_step_adaptive");
    refresh();
}

void FvDVM::getCoNum(double dt, double& maxCo, double& meanCo) const {
    check(dugks_co_num(h_, dt, &maxCo, &meanCo), "dugks_co_num");
}

void FvDVM::surfMacros(std::vector<double>& rho, std::vector<double>& U, std::vector<double>& T,
                       std::vector<double>& q) const {
    const size_t nF = static_cast<size_t>(flat_.n_internal) + flat_.n_boundary;
    rho.assign(nF, 0.0);
    T.assign(nF, 0.0);
    U.assign(3 * nF, 0.0);
    q.assign(3 * nF, 0.0);
    check(dugks_get_face_macros(h_, rho.data(), U.data(), T.data(), q.data()), "dugks_get_face_macros");
}

std::vector<double> FvDVM::boundaryRho() const {
    std::vector<double> r(static_cast<size_t>(flat_.n_boundary), 0.0);
    check(dugks_get_boundary_rho(h_, r.data()), "dugks_get_boundary_rho");
    return r;
}

void FvDVM::dfOnCells(const std::vector<int32_t>& cells, std::vector<double>& g, std::vector<double>& h) const {
    g.assign(cells.size() * static_cast<size_t>(n_xi_), 0.0);
    h.assign(cells.size() * static_cast<size_t>(n_xi_), 0.0);
    check(dugks_get_df(h_, cells.data(), static_cast<int32_t>(cells.size()), g.data(), h.data()), "dugks_get_df");
}

namespace {
constexpr char kStateMagic[8] = {'D', 'U', 'G', 'K', 'S', 'S', 'T', '2'};
}

void FvDVM::writeState(const std::string& path, double dt_prev, double time) const {
    const size_t n = static_cast<size_t>(n_xi_) * flat_.n_cells;
    std::vector<double> g(n), h(n);
    check(dugks_get_state(h_, g.data(), h.data()), "dugks_get_state");
    std::vector<double> rec(static_cast<size_t>(dugks_step_record_size(h_)));
    check(dugks_get_step_record(h_, rec.data()), "dugks_get_step_record");
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw FvDVMError(DUGKS_ERR_ARG, "cannot write " + path);
    const int32_t D = flat_.D, n1d = nXiPerDim();
    const int64_t nc = flat_.n_cells, nv = n_xi_;
    bool ok = std::fwrite(kStateMagic, 1, 8, f) == 8 && std::fwrite(&D, sizeof D, 1, f) == 1 &&
              std::fwrite(&n1d, sizeof n1d, 1, f) == 1 && std::fwrite(&nc, sizeof nc, 1, f) == 1 &&
              std::fwrite(&nv, sizeof nv, 1, f) == 1 && std::fwrite(&dt_prev, sizeof dt_prev, 1, f) == 1 &&
              std::fwrite(&time, sizeof time, 1, f) == 1 && std::fwrite(g.data(), sizeof(double), n, f) == n &&
              std::fwrite(h.data(), sizeof(double), n, f) == n &&
              std::fwrite(rec.data(), sizeof(double), rec.size(), f) == rec.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw FvDVMError(DUGKS_ERR_ARG, "error writing " + path);
}

void FvDVM::readState(const std::string& path, double& dt_prev, double& time) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw FvDVMError(DUGKS_ERR_ARG, "cannot open " + path);
    char magic[8];
    int32_t D = 0, n1d = 0;
    int64_t nc = 0, nv = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::fread(&D, sizeof D, 1, f) == 1 &&
              std::fread(&n1d, sizeof n1d, 1, f) == 1 && std::fread(&nc, sizeof nc, 1, f) == 1 &&
              std::fread(&nv, sizeof nv, 1, f) == 1 && std::fread(&dt_prev, sizeof dt_prev, 1, f) == 1 &&
              std::fread(&time, sizeof time, 1, f) == 1;
    if (!ok || std::memcmp(magic, kStateMagic, 8) != 0) {
        std::fclose(f);
        throw FvDVMError(DUGKS_ERR_ARG, path + ": not a DUGKS state file");
    }
    if (D != flat_.D || n1d != nXiPerDim() || nc != flat_.n_cells || nv != n_xi_) {
        std::fclose(f);
        throw FvDVMError(DUGKS_ERR_ARG, path + ": state of another mesh or DV set");
    }
    const size_t n = static_cast<size_t>(nv) * static_cast<size_t>(nc);
    std::vector<double> g(n), h(n), rec(static_cast<size_t>(dugks_step_record_size(h_)));
    ok = std::fread(g.data(), sizeof(double), n, f) == n && std::fread(h.data(), sizeof(double), n, f) == n &&
         std::fread(rec.data(), sizeof(double), rec.size(), f) == rec.size();
    std::fclose(f);
    if (!ok) throw FvDVMError(DUGKS_ERR_ARG, path + ": truncated state file");
    check(dugks_set_state(h_, g.data(), h.data(), dt_prev), "dugks_set_state");
    check(dugks_set_step_record(h_, rec.data()), "dugks_set_step_record");
    refresh();
}

}  // namespace dugks_host

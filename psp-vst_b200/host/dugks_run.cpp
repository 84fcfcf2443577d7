// dugks_run: a standalone dugksFoam-style driver over the B200 C ABI.
//
// Reads a dugksFoam case directory (constant/polyMesh, constant/Xis,
// constant/weights, constant/DVMProperties, 0/rho, 0/U, 0/T and, when
// present, system/controlDict), advances it with FvDVM::evolution as the
// reference's time loop does (src/dugksFoam.C:63-110), and writes rho, U, T
// and q into time directories.
//
//   dugks_run CASE [--steps N] [--dt DT] [--precision fp64|fp32c] [--device D]
//                  [--write-interval N] [--no-write] [--write-state] [--restart TIME] [--check]
//                  [--max-co C] [--max-delta-t DT] [--fixed-dt] [--vmesh]
//
// The time step is --dt, else controlDict deltaT, else the Courant number
// 0.5 of the initial state (fvDVM::getCoNum).  With controlDict
// adjustTimeStep on, or --max-co given, every step first adjusts it to hold
// the Courant number at maxCo (CourantNo.H + setDeltaTvar.H, on the device);
// --fixed-dt turns that off.  The step count is --steps, else the steps that
// reach endTime (Time::run: time < endTime - dt/2).  Fixed steps write every
// --write-interval steps, else every writeInterval / deltaT steps; adjusted
// steps write when the time passes a multiple of writeInterval (the time step
// is not shortened to land on it).  --vmesh takes the DVs from the velocity
// mesh constant/vMesh (cell centres, cell volumes), as the reference's VMESH
// build does.  --write-state adds an exact restart file
// (dugksState, see fvdvm.hpp) to every written time directory; --restart TIME
// continues from CASE/TIME/dugksState.  --check reads the case and computes the
// mesh geometry on the host only (no GPU) and prints a summary.  The last
// line printed is a JSON summary.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fvdvm.hpp"

using namespace dugks_host;

namespace {

struct Args {
    std::string dir;
    long steps = -1;
    double dt = 0;
    int precision = DUGKS_FP64;
    int device = 0;
    long write_interval = 0;
    bool write = true;
    bool write_state = false;
    bool check = false;
    bool fixed_dt = false;
    bool vmesh = false;
    double max_co = 0, max_delta_t = 0;
    std::string restart;
};

[[noreturn]] void usage(const char* msg) {
    std::fprintf(stderr, "dugks_run: %s\nusage: dugks_run CASE [--steps N] [--dt DT] [--precision fp64|fp32c] "
                         "[--device D] [--write-interval N] [--no-write] [--write-state] [--restart TIME] "
                         "[--check] [--max-co C] [--max-delta-t DT] [--fixed-dt] [--vmesh]\n", msg);
    std::exit(2);
}

Args parse(int argc, char** argv) {
    Args a;
    for (int i = 1; i < argc; ++i) {
        const std::string s = argv[i];
        auto val = [&]() -> const char* {
            if (i + 1 >= argc) usage(("missing value after " + s).c_str());
            return argv[++i];
        };
        if (s == "--steps") a.steps = std::atol(val());
        else if (s == "--dt") a.dt = std::atof(val());
        else if (s == "--device") a.device = std::atoi(val());
        else if (s == "--write-interval") a.write_interval = std::atol(val());
        else if (s == "--no-write") a.write = false;
        else if (s == "--check") a.check = true;
        else if (s == "--write-state") a.write_state = true;
        else if (s == "--restart") a.restart = val();
        else if (s == "--max-co") a.max_co = std::atof(val());
        else if (s == "--max-delta-t") a.max_delta_t = std::atof(val());
        else if (s == "--fixed-dt") a.fixed_dt = true;
        else if (s == "--vmesh") a.vmesh = true;
        else if (s == "--precision") {
            const std::string p = val();
            if (p == "fp64") a.precision = DUGKS_FP64;
            else if (p == "fp32c") a.precision = DUGKS_FP32C;
            else usage("unknown precision");
        } else if (!s.empty() && s[0] == '-') {
            usage(("unknown option " + s).c_str());
        } else if (a.dir.empty()) {
            a.dir = s;
        } else {
            usage("more than one case directory");
        }
    }
    if (a.dir.empty()) usage("no case directory");
    return a;
}

using PatchValues = std::vector<std::pair<std::string, std::pair<std::string, std::vector<double>>>>;

// rho, U, T, q of the current state into CASE/<time>/ (the AUTO_WRITE
// macro fields of src/createFields.H and fvDVM.C:2016-2105)
void write_time(const FvDVM& s, double time, bool state, double dt) {
    const std::string tname = time_name(time);
    const Case& c = s.caseData();
    const FlatMesh& f = s.mesh();
    std::vector<double> frho, fU, fT, fq;
    s.surfMacros(frho, fU, fT, fq);
    const std::vector<double> brho = s.boundaryRho();
    PatchValues prho, pU, pT, pq;
    size_t fp = 0;   // index into the non-empty patches
    for (size_t p = 0; p < c.mesh.patches.size(); ++p) {
        const std::string& name = c.mesh.patches[p].name;
        if (c.kinds[p] == PatchKind::Empty) {
            for (PatchValues* v : {&prho, &pU, &pT, &pq}) v->push_back({name, {"empty", {}}});
            continue;
        }
        const size_t b0 = f.patch_start[fp], b1 = f.patch_start[fp + 1];
        ++fp;
        std::vector<double> r(brho.begin() + b0, brho.begin() + b1), u, t, q;
        for (size_t b = b0; b < b1; ++b) {
            u.insert(u.end(), f.U_b.begin() + 3 * b, f.U_b.begin() + 3 * b + 3);
            t.push_back(f.T_b[b]);
            const size_t face = static_cast<size_t>(f.n_internal) + b;
            q.insert(q.end(), fq.begin() + 3 * face, fq.begin() + 3 * face + 3);
        }
        prho.push_back({name, {c.rho_types[p], r}});
        pU.push_back({name, {c.U_types[p], u}});
        pT.push_back({name, {c.T_types[p], t}});
        pq.push_back({name, {"calculated", q}});
    }
    const std::string dir = c.dir + "/" + tname;
    write_vol_field(dir + "/rho", "rho", 1, s.rhoVol(), prho, "[1 -3 0 0 0 0 0]", tname);
    write_vol_field(dir + "/U", "U", 3, s.Uvol(), pU, "[0 1 -1 0 0 0 0]", tname);
    write_vol_field(dir + "/T", "T", 1, s.Tvol(), pT, "[0 0 0 1 0 0 0]", tname);
    write_vol_field(dir + "/q", "q", 3, s.qVol(), pq, "[1 0 -3 0 0 0 0]", tname);
    if (state) s.writeState(dir + "/dugksState", dt, time);
}

double total(const std::vector<double>& v, const std::vector<double>& w) {
    double s = 0;
    for (size_t i = 0; i < v.size(); ++i) s += v[i] * w[i];
    return s;
}

}  // namespace

int main(int argc, char** argv) {
    const Args a = parse(argc, argv);
    try {
        const Case c = read_case(a.dir, a.vmesh);
        if (a.check) {
            const FlatMesh f = flatten(c);
            double vol = 0;
            for (double v : f.V) vol += v;
            std::printf("{\"cells\": %d, \"internal_faces\": %d, \"boundary_faces\": %d, \"D\": %d, "
                        "\"n_dv\": %.0f, \"volume\": %.17g, \"mass\": %.17g, \"xi_max\": %.17g, "
                        "\"adjust_time_step\": %s, \"max_co\": %.17g, \"max_delta_t\": %.17g, "
                        "\"macro_flux\": %s, \"patches\": [",
                        f.n_cells, f.n_internal, f.n_boundary, f.D,
                        c.dv_w.empty() ? std::pow(double(c.xis.size()), f.D) : double(c.dv_w.size()), vol,
                        total(c.rho0, f.V), c.xi_max, c.adjust_time_step ? "true" : "false", c.max_co,
                        c.max_delta_t, c.macro_flux ? "true" : "false");
            for (size_t p = 0; p < c.mesh.patches.size(); ++p)
                std::printf("%s{\"name\": \"%s\", \"kind\": \"%s\", \"faces\": %lld}", p ? ", " : "",
                            c.mesh.patches[p].name.c_str(), kind_name(c.kinds[p]),
                            static_cast<long long>(c.mesh.patches[p].size));
            std::printf("]}\n");
            return 0;
        }
        FvDVM s(c, a.precision, a.device);
        double dt = a.dt > 0 ? a.dt : c.delta_t;
        if (!(dt > 0)) {
            double co_max, co_mean;
            s.getCoNum(1.0, co_max, co_mean);   // Courant number per unit time step
            dt = 0.5 / co_max;
        }
        const bool adjust = !a.fixed_dt && (c.adjust_time_step || a.max_co > 0);
        const double max_co = a.max_co > 0 ? a.max_co : c.max_co;
        const double max_dt = a.max_delta_t > 0 ? a.max_delta_t : c.max_delta_t;
        double t0 = c.start_time;
        if (!a.restart.empty()) {
            double dt_prev = 0;
            s.readState(c.dir + "/" + a.restart + "/dugksState", dt_prev, t0);
        }
        long steps = a.steps;
        if (steps < 0 && !adjust) steps = c.end_time > t0 ? std::lround((c.end_time - t0) / dt) : 1;
        if (steps < 0 && !(c.end_time > t0)) steps = 1;
        long every = a.write_interval;
        if (every <= 0 && !adjust && c.write_interval > 0 && c.delta_t > 0)
            every = std::lround(c.write_interval / c.delta_t);
        const bool by_time = adjust && a.write_interval <= 0 && c.write_interval > 0;
        long write_index = 0;
        double t = t0;
        long n = 0;
        bool written = false;
        while (steps >= 0 ? n < steps : t < c.end_time - 0.5 * dt) {
            if (adjust) s.evolutionAdjustable(dt, max_co, max_dt);
            else s.evolution(dt);
            ++n;
            t = adjust ? t + dt : t0 + n * dt;
            std::printf("Time = %s\n", time_name(t).c_str());
            bool due = every > 0 && n % every == 0;
            if (by_time) {   // Time::writeTime for adjustableRunTime
                const long idx = static_cast<long>(std::floor((t - t0 + 0.5 * dt) / c.write_interval));
                due = idx > write_index;
                if (due) write_index = idx;
            }
            written = a.write && due;
            if (written) write_time(s, t, a.write_state, dt);
        }
        const long done = n;
        if (a.write && done > 0 && !written) write_time(s, t, a.write_state, dt);
        double co_max = 0, co_mean = 0;
        s.getCoNum(dt, co_max, co_mean);
        std::printf("{\"steps\": %ld, \"dt\": %.17g, \"time\": %.17g, \"time_name\": \"%s\", \"mass\": %.17g, "
                    "\"co_max\": %.17g, \"co_mean\": %.17g, \"n_dv\": %d}\n",
                    done, dt, t, time_name(t).c_str(), total(s.rhoVol(), s.mesh().V), co_max, co_mean, s.nXi());
        return 0;
    } catch (const FvDVMError& e) {
        std::fprintf(stderr, "dugks_run: %s (status %d)\n", e.what(), e.status);
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "dugks_run: %s\n", e.what());
        return 1;
    }
}

// dugks_adjoint_run: the discrete adjoint of the FP64 DUGKS step on the
// GPU.  The forward steps between checkpoints are the library's tiled
// passes (dugks_step); the step being reversed is recorded again by the
// plain per-(DV, entity) kernels of dugks_adjoint.cuh from its start state,
// then reversed by the kernels there.  All arrays are FP64 in HBM.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cstring>
#include <string>
#include <vector>

#include "dugks_adjoint.cuh"
#include "dugks_internal.h"

namespace {

using dugks::set_error;
namespace adj = dugks::adj;

#define ADJ_TRY(h, call)                                                                                \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return set_error((h), e_ == cudaErrorMemoryAllocation ? DUGKS_ERR_OOM : DUGKS_ERR_CUDA,     \
                             std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

constexpr int kBlock = 256;

// CTAs of 256 threads a functor asks to keep resident per SM (a register cap)
template <class F, class = void>
struct MinCtas {
    static constexpr int value = 1;
};
template <class F>
struct MinCtas<F, std::void_t<decltype(F::kMinCtas)>> {
    static constexpr int value = F::kMinCtas;
};

template <class F>
__global__ void __launch_bounds__(kBlock, MinCtas<F>::value) k_adjoint(F f, int64_t n) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) f(i);
}

// runs a functor over 0..n-1 on the handle's stream: a grid-stride launch
// of at most 16 CTAs of 256 threads per SM
struct GpuEx {
    dugks_handle* h;
    int sms;
    template <class F>
    int run(int64_t n, const F& f) {
        if (n <= 0) return DUGKS_OK;
        const int64_t want = (n + kBlock - 1) / kBlock;
        const int grid = static_cast<int>(std::min<int64_t>(want, static_cast<int64_t>(sms) * 16));
        k_adjoint<F><<<grid, kBlock, 0, h->stream>>>(f, n);
        h->launches += 1;
        ADJ_TRY(h, cudaGetLastError());
        return DUGKS_OK;
    }
    // the tiled pass A of the recorded step, into the handle's face-value buffer
    int pass_a(const adj::View& v) { return dugks::record_face_values(h, v.dt); }
};

// device allocations of one run, freed together
struct Arena {
    std::vector<void*> p;
    double bytes = 0;
    ~Arena() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    int get(dugks_handle* h, T** out, size_t n) {
        void* q = nullptr;
        const size_t b = std::max<size_t>(n, 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&q, b);
        if (e != cudaSuccess)
            return set_error(h, e == cudaErrorMemoryAllocation ? DUGKS_ERR_OOM : DUGKS_ERR_CUDA,
                             "dugks_adjoint_run: cudaMalloc of " + std::to_string(b) + " bytes: " +
                                 cudaGetErrorString(e));
        p.push_back(q);
        bytes += static_cast<double>(b);
        *out = static_cast<T*>(q);
        return DUGKS_OK;
    }
    template <class T>
    int put(dugks_handle* h, T** out, const std::vector<T>& v) {
        if (int st = get(h, out, v.size())) return st;
        if (!v.empty()) ADJ_TRY(h, cudaMemcpyAsync(*out, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                                                   h->stream));
        return DUGKS_OK;
    }
    template <class T>
    int zeros(dugks_handle* h, T** out, size_t n) {
        if (int st = get(h, out, n)) return st;
        ADJ_TRY(h, cudaMemsetAsync(*out, 0, std::max<size_t>(n, 1) * sizeof(T), h->stream));
        return DUGKS_OK;
    }
};

// checkpoint operations on the handle (revolve's Ops)
struct HandleOps {
    dugks_handle* h;
    GpuEx ex;
    adj::View v;
    int n_steps, window_start;
    double dt;
    size_t nvc;
    std::vector<double*> slot;    // [slots]: g, h, cm of a saved state
    double* lam[4];               // adjoint of the state: in g, in h, out g, out h
    int64_t forward_steps = 0;
    float ms_forward = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;

    int save(int s) {
        double* d = slot[s];
        const int c = h->ds.cur;
        ADJ_TRY(h, cudaMemcpyAsync(d, h->ds.g[c], nvc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        ADJ_TRY(h, cudaMemcpyAsync(d + nvc, h->ds.h[c], nvc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        ADJ_TRY(h, cudaMemcpyAsync(d + 2 * nvc, h->ds.cm, 9 * static_cast<size_t>(h->nC) * sizeof(double),
                                   cudaMemcpyDeviceToDevice, h->stream));
        return DUGKS_OK;
    }
    int restore(int s) {
        const double* d = slot[s];
        const int c = h->ds.cur;
        ADJ_TRY(h, cudaMemcpyAsync(h->ds.g[c], d, nvc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        ADJ_TRY(h, cudaMemcpyAsync(h->ds.h[c], d + nvc, nvc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        ADJ_TRY(h, cudaMemcpyAsync(h->ds.cm, d + 2 * nvc, 9 * static_cast<size_t>(h->nC) * sizeof(double),
                                   cudaMemcpyDeviceToDevice, h->stream));
        return dugks::rebuild_cell_records(h);
    }
    int advance(int k) {
        if (k <= 0) return DUGKS_OK;
        std::vector<double> dts(k, dt);
        ADJ_TRY(h, cudaEventRecord(e0, h->stream));
        if (int st = dugks_step(h, k, dts.data())) return st;
        ADJ_TRY(h, cudaEventRecord(e1, h->stream));
        ADJ_TRY(h, cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ms_forward += ms;
        forward_steps += k;
        return DUGKS_OK;
    }
    int reverse(int n) {
        adj::View w = v;
        const int c = h->ds.cur;
        w.g = static_cast<const double*>(h->ds.g[c]);
        w.h = static_cast<const double*>(h->ds.h[c]);
        w.cm = h->ds.cm;
        w.wn = n >= window_start ? 1.0 / (n_steps - window_start) : 0.0;
        w.fold = n >= 1 ? 1 : 0;
        w.lg = lam[0];
        w.lh = lam[1];
        w.og = lam[2];
        w.oh = lam[3];
        int st = adj::record_step(ex, w);
        if (!st) st = adj::reverse_step(ex, w);
        if (st) return st;
        std::swap(lam[0], lam[2]);
        std::swap(lam[1], lam[3]);
        return DUGKS_OK;
    }
};

}  // namespace

namespace {

// checks, mesh tables and the record buffers shared by both entry points;
// with_adjoint also allocates the adjoint arrays
int prepare(dugks_handle* h, const dugks_objective* obj, const char* who, Arena& ar, adj::View& v, int& sms,
            bool with_adjoint, double** lam) {
    if (!obj) return set_error(h, DUGKS_ERR_ARG, std::string(who) + ": null objective");
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, std::string(who) + " before dugks_set_macros");
    if (obj->n_steps < 1 || obj->window_start < 0 || obj->window_start >= obj->n_steps || !(obj->dt > 0) ||
        obj->max_snapshots < 1)
        return set_error(h, DUGKS_ERR_ARG, std::string(who) + ": need n_steps >= 1, 0 <= window_start < n_steps, "
                                                              "dt > 0, max_snapshots >= 1");
    if (h->precision != DUGKS_FP64 || h->shard_world > 1 || h->shard_nccl || h->dm.macro_flux)
        return set_error(h, DUGKS_ERR_UNSUPPORTED, std::string(who) + ": FP64, unsharded handles with macroFlux no only");
    for (int b = 0; b < h->nBF; ++b)
        if (h->bface_ptype[b] != DUGKS_PATCH_MAXWELL_WALL && h->bface_ptype[b] != DUGKS_PATCH_FAR_FIELD)
            return set_error(h, DUGKS_ERR_UNSUPPORTED, std::string(who) + ": maxwellWall and farField patches only");
    ADJ_TRY(h, cudaSetDevice(h->device));
    ADJ_TRY(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));

    const int nC = h->nC, nIF = h->nIF, nBF = h->nBF, nF = nIF + nBF, nv = h->nv;
    const size_t nvc = static_cast<size_t>(nv) * nC, nvf = static_cast<size_t>(nv) * nF;
    // mesh tables in the handle's cell numbering
    const std::vector<int32_t>& perm = h->tiling.perm;
    const std::vector<int32_t>& iperm = h->tiling.iperm;
    std::vector<int32_t> own(nF), nei(nIF);
    for (int f = 0; f < nF; ++f) own[f] = iperm[h->owner[f]];
    for (int f = 0; f < nIF; ++f) nei[f] = iperm[h->neighbour[f]];
    std::vector<double> Cn(3 * static_cast<size_t>(nC)), Vn(nC);
    for (int c = 0; c < nC; ++c) {
        for (int k = 0; k < 3; ++k) Cn[3 * c + k] = h->C[3 * static_cast<size_t>(perm[c]) + k];
        Vn[c] = h->V[perm[c]];
    }
    adj::HostTables t;
    adj::build_tables(nC, nIF, nBF, own.data(), nei.data(), Vn.data(), h->bface_patch_local.data(), t);
    std::vector<double> ha(nBF, 0.0), fw(3 * static_cast<size_t>(nBF), 0.0);
    if (obj->energy_weight) std::copy(obj->energy_weight, obj->energy_weight + nBF, ha.begin());
    if (obj->momentum_weight) std::copy(obj->momentum_weight, obj->momentum_weight + 3 * nBF, fw.begin());
    for (int b = 0; b < nBF; ++b) {
        bool ok = std::isfinite(ha[b]);
        for (int k = 0; k < 3; ++k) ok = ok && std::isfinite(fw[3 * b + k]);
        if (!ok) return set_error(h, DUGKS_ERR_ARG, std::string(who) + ": non-finite objective weight");
    }
    std::vector<double> Sf(h->Sf.begin(), h->Sf.begin() + 3 * static_cast<size_t>(nF));
    std::vector<double> Cf(h->Cf.begin(), h->Cf.begin() + 3 * static_cast<size_t>(nF));

    v = adj::View{};
    v.nC = nC;
    v.nIF = nIF;
    v.nBF = nBF;
    v.nF = nF;
    v.nv = nv;
    v.D = h->D;
    v.K = h->gas.K_inner;
    const int64_t target = static_cast<int64_t>(sms) * 2048;
    v.nchF = adj::chunks_for(nF, nv, target);
    v.nchC = adj::chunks_for(nC, nv, target);
    v.R = h->gas.R;
    v.Pr = h->gas.Pr;
    v.omega = h->gas.omega;
    v.Tref = h->gas.Tref;
    v.mu = h->gas.mu_ref;
    v.dt = obj->dt;
    v.xi = h->dm.xi;
    v.w = h->dm.w;

    int32_t *d_own, *d_nei, *d_cfo, *d_cfe, *d_tho, *d_the, *d_bt, *d_bl;
    double *d_S, *d_Cf, *d_C, *d_iV, *d_lsP, *d_lsN, *d_bU, *d_bT, *d_brho, *d_ha, *d_fw;
    int st;
    if ((st = ar.put(h, &d_own, own)) || (st = ar.put(h, &d_nei, nei)) || (st = ar.put(h, &d_cfo, t.cf_off)) ||
        (st = ar.put(h, &d_cfe, t.cf_ent)) || (st = ar.put(h, &d_tho, t.th_off)) || (st = ar.put(h, &d_the, t.th_ent)) ||
        (st = ar.put(h, &d_bt, h->bface_ptype)) || (st = ar.put(h, &d_bl, h->bface_patch_local)) ||
        (st = ar.put(h, &d_S, Sf)) || (st = ar.put(h, &d_Cf, Cf)) || (st = ar.put(h, &d_C, Cn)) ||
        (st = ar.put(h, &d_iV, t.invV)) || (st = ar.put(h, &d_lsP, h->lsP)) || (st = ar.put(h, &d_lsN, h->lsN)) ||
        (st = ar.put(h, &d_bU, h->bc_U)) || (st = ar.put(h, &d_bT, h->bc_T)) || (st = ar.put(h, &d_brho, h->bc_rho)) ||
        (st = ar.put(h, &d_ha, ha)) || (st = ar.put(h, &d_fw, fw)))
        return st;
    v.own = d_own;
    v.nei = d_nei;
    v.cf_off = d_cfo;
    v.cf_ent = d_cfe;
    v.th_off = d_tho;
    v.th_ent = d_the;
    v.btype = d_bt;
    v.blocal = d_bl;
    v.S = d_S;
    v.Cf = d_Cf;
    v.C = d_C;
    v.invV = d_iV;
    v.lsP = d_lsP;
    v.lsN = d_lsN;
    v.bU = d_bU;
    v.bT = d_bT;
    v.brho = d_brho;
    v.ha = d_ha;
    v.fw = d_fw;
    v.fvg = static_cast<const double*>(h->ds.fvg);
    v.fvh = static_cast<const double*>(h->ds.fvh);
    v.fitems = h->dm.face_items;
    v.nI = h->dm.n_items;
    if ((st = ar.get(h, &v.fg, nvf)) || (st = ar.get(h, &v.fh, nvf)) ||
        (st = ar.get(h, &v.pf, static_cast<size_t>(v.nchF) * nF * adj::kP)) || (st = ar.get(h, &v.rhow, nBF)) ||
        (st = ar.get(h, &v.inby, nBF)) || (st = ar.get(h, &v.fmac, static_cast<size_t>(nF) * adj::kMac)) ||
        (st = ar.zeros(h, &v.Jb, nBF)))
        return st;
    if (!with_adjoint) return DUGKS_OK;
    if ((st = ar.get(h, &v.pc, static_cast<size_t>(v.nchC) * nC * adj::kP)) ||
        (st = ar.get(h, &v.cmac, static_cast<size_t>(nC) * adj::kMac)) || (st = ar.get(h, &v.ag, nvf)) ||
        (st = ar.get(h, &v.ah, nvf)) || (st = ar.get(h, &v.aGg, 3 * nvc)) || (st = ar.get(h, &v.aGh, 3 * nvc)) ||
        (st = ar.get(h, &v.fco, static_cast<size_t>(nF) * adj::kCo)) ||
        (st = ar.get(h, &v.cco, static_cast<size_t>(nC) * adj::kCo)) || (st = ar.get(h, &v.aout, nBF)) ||
        (st = ar.get(h, &v.aUown, 3 * static_cast<size_t>(nBF))) || (st = ar.zeros(h, &v.gTb, nBF)) ||
        (st = ar.zeros(h, &v.gUb, 3 * static_cast<size_t>(nBF))) || (st = ar.zeros(h, &v.aI, nBF)) ||
        (st = ar.zeros(h, &v.amuF, nF)) || (st = ar.zeros(h, &v.amuC, nC)) || (st = ar.zeros(h, &lam[0], nvc)) ||
        (st = ar.zeros(h, &lam[1], nvc)) || (st = ar.get(h, &lam[2], nvc)) || (st = ar.get(h, &lam[3], nvc)))
        return st;
    return DUGKS_OK;
}

double host_sum(const std::vector<double>& a) {
    double s = 0;
    for (double x : a) s += x;
    return s;
}

}  // namespace

extern "C" int dugks_adjoint_run(dugks_handle* h, const dugks_objective* obj, double* J, double* dJ_dT_b,
                                 double* dJ_dU_b, double* dJ_dmu_ref, dugks_adjoint_stats* stats) {
    if (!h) return DUGKS_ERR_ARG;
    Arena ar;
    adj::View v;
    double* lam[4] = {};
    int sms = 0, st;
    if ((st = prepare(h, obj, "dugks_adjoint_run", ar, v, sms, true, lam))) return st;
    const int nC = h->nC, nBF = h->nBF, nF = v.nF;
    const size_t nvc = static_cast<size_t>(h->nv) * nC;

    HandleOps ops;
    ops.h = h;
    ops.ex = GpuEx{h, sms};
    ops.v = v;
    ops.n_steps = obj->n_steps;
    ops.window_start = obj->window_start;
    ops.dt = obj->dt;
    ops.nvc = nvc;
    const int n_slots = std::min(obj->max_snapshots, obj->n_steps);
    ops.slot.resize(n_slots);
    for (int s = 0; s < n_slots; ++s)
        if ((st = ar.get(h, &ops.slot[s], 2 * nvc + 9 * static_cast<size_t>(nC)))) return st;
    for (int k = 0; k < 4; ++k) ops.lam[k] = lam[k];
    ADJ_TRY(h, cudaEventCreate(&ops.e0));
    ADJ_TRY(h, cudaEventCreate(&ops.e1));
    struct EvGuard {
        HandleOps& o;
        ~EvGuard() {
            cudaEventDestroy(o.e0);
            cudaEventDestroy(o.e1);
        }
    } guard{ops};

    const long steps_before = h->steps_done;
    cudaEvent_t t0, t1;
    ADJ_TRY(h, cudaEventCreate(&t0));
    ADJ_TRY(h, cudaEventCreate(&t1));
    ADJ_TRY(h, cudaEventRecord(t0, h->stream));
    if ((st = ops.ex.run(nBF, adj::FInBy{v}))) return st;
    if ((st = adj::revolve_run(ops, obj->n_steps, n_slots))) return st;
    if ((st = ops.ex.run(nBF, adj::RInBy{v}))) return st;
    ADJ_TRY(h, cudaEventRecord(t1, h->stream));
    std::vector<double> Jb(nBF), gT(nBF), gU(3 * static_cast<size_t>(nBF)), mF(nF), mC(nC);
    ADJ_TRY(h, cudaMemcpyAsync(Jb.data(), v.Jb, nBF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ADJ_TRY(h, cudaMemcpyAsync(gT.data(), v.gTb, nBF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ADJ_TRY(h, cudaMemcpyAsync(gU.data(), v.gUb, gU.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ADJ_TRY(h, cudaMemcpyAsync(mF.data(), v.amuF, nF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ADJ_TRY(h, cudaMemcpyAsync(mC.data(), v.amuC, nC * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ADJ_TRY(h, cudaStreamSynchronize(h->stream));
    float ms_total = 0;
    cudaEventElapsedTime(&ms_total, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    h->steps_done = steps_before;

    const double Jsum = host_sum(Jb), mu = host_sum(mF) + host_sum(mC);
    if (J) *J = Jsum;
    if (dJ_dT_b) std::copy(gT.begin(), gT.end(), dJ_dT_b);
    if (dJ_dU_b) std::copy(gU.begin(), gU.end(), dJ_dU_b);
    if (dJ_dmu_ref) *dJ_dmu_ref = mu;
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->forward_steps = ops.forward_steps;
        stats->reverse_steps = obj->n_steps;
        stats->snapshots = n_slots;
        stats->ms_total = ms_total;
        stats->ms_forward = ops.ms_forward;
        stats->device_bytes = ar.bytes;
    }
    if (!std::isfinite(Jsum) || !std::isfinite(mu))
        return set_error(h, DUGKS_ERR_NAN, "dugks_adjoint_run: non-finite objective or gradient");
    return DUGKS_OK;
}

namespace {
// revolve's operations that only count what a run would do
struct CountOps {
    int64_t forward = 0, reverses = 0, saves = 0, restores = 0;
    int next = 0;  // the step whose reverse comes next: must run n-1, ..., 0 in order
    bool order_ok = true;
    int save(int) { ++saves; return 0; }
    int restore(int) { ++restores; return 0; }
    int advance(int k) { forward += k; return 0; }
    int reverse(int n) {
        if (n != next) order_ok = false;
        --next;
        ++reverses;
        return 0;
    }
};
}  // namespace

extern "C" int64_t dugks_checkpoint_forward_steps(int32_t n_steps, int32_t n_snapshots) {
    if (n_steps < 1 || n_snapshots < 1) return -1;
    CountOps ops;
    ops.next = n_steps - 1;
    const int slots = n_snapshots < n_steps ? n_snapshots : n_steps;
    if (adj::revolve_run(ops, n_steps, slots) != 0 || !ops.order_ok || ops.reverses != n_steps) return -1;
    return ops.forward;
}

extern "C" int dugks_boundary_fluxes(dugks_handle* h, double dt, double* flux) {
    if (!h) return DUGKS_ERR_ARG;
    if (!flux) return set_error(h, DUGKS_ERR_ARG, "dugks_boundary_fluxes: null output");
    dugks_objective obj{};
    obj.n_steps = 1;
    obj.dt = dt;
    obj.max_snapshots = 1;
    Arena ar;
    adj::View v;
    int sms = 0, st;
    if ((st = prepare(h, &obj, "dugks_boundary_fluxes", ar, v, sms, false, nullptr))) return st;
    const int nBF = h->nBF;
    if (nBF == 0) return DUGKS_OK;
    double* d_out;
    if ((st = ar.get(h, &d_out, 5 * static_cast<size_t>(nBF)))) return st;
    GpuEx ex{h, sms};
    const int c = h->ds.cur;
    v.g = static_cast<const double*>(h->ds.g[c]);
    v.h = static_cast<const double*>(h->ds.h[c]);
    v.cm = h->ds.cm;
    if ((st = ex.run(nBF, adj::FInBy{v}))) return st;
    if ((st = adj::record_step(ex, v))) return st;
    if ((st = ex.run(nBF, adj::FBoundaryFlux{v, d_out}))) return st;
    ADJ_TRY(h, cudaMemcpyAsync(flux, d_out, 5 * static_cast<size_t>(nBF) * sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
    ADJ_TRY(h, cudaStreamSynchronize(h->stream));
    return DUGKS_OK;
}

extern "C" int dugks_objective_run(dugks_handle* h, const dugks_objective* obj, double* J,
                                   dugks_adjoint_stats* stats) {
    if (!h) return DUGKS_ERR_ARG;
    Arena ar;
    adj::View v;
    int sms = 0, st;
    if ((st = prepare(h, obj, "dugks_objective_run", ar, v, sms, false, nullptr))) return st;
    GpuEx ex{h, sms};
    const int nBF = h->nBF;
    const double dt = obj->dt;
    cudaEvent_t t0, t1;
    ADJ_TRY(h, cudaEventCreate(&t0));
    ADJ_TRY(h, cudaEventCreate(&t1));
    ADJ_TRY(h, cudaEventRecord(t0, h->stream));
    if ((st = ex.run(nBF, adj::FInBy{v}))) return st;
    if (obj->window_start > 0) {
        std::vector<double> dts(obj->window_start, dt);
        if ((st = dugks_step(h, obj->window_start, dts.data()))) return st;
    }
    for (int n = obj->window_start; n < obj->n_steps; ++n) {
        adj::View w = v;
        const int c = h->ds.cur;
        w.g = static_cast<const double*>(h->ds.g[c]);
        w.h = static_cast<const double*>(h->ds.h[c]);
        w.cm = h->ds.cm;
        w.wn = 1.0 / (obj->n_steps - obj->window_start);
        if ((st = adj::record_step(ex, w))) return st;
        if ((st = ex.run(nBF, adj::FObjective{w}))) return st;
        if ((st = dugks_step(h, 1, &dt))) return st;
    }
    ADJ_TRY(h, cudaEventRecord(t1, h->stream));
    std::vector<double> Jb(nBF);
    ADJ_TRY(h, cudaMemcpyAsync(Jb.data(), v.Jb, nBF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ADJ_TRY(h, cudaStreamSynchronize(h->stream));
    float ms_total = 0;
    cudaEventElapsedTime(&ms_total, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    const double Jsum = host_sum(Jb);
    if (J) *J = Jsum;
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->forward_steps = obj->n_steps;
        stats->ms_total = ms_total;
        stats->device_bytes = ar.bytes;
    }
    if (!std::isfinite(Jsum)) return set_error(h, DUGKS_ERR_NAN, "dugks_objective_run: non-finite objective");
    return DUGKS_OK;
}

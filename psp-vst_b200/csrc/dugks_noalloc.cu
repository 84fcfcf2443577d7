// dugks_cell_macros_noalloc: cell macros rho, U, T, q of caller-owned
// device distribution functions, computed without allocating device memory.
//
// It is the raw-moment reduction of the restart path (dugks_set_state:
// per-cell raw moments over DV chunks, then a combine into macros as
// fvDVM::updateMacroVol does, src/fvDVM/fvDVM/fvDVM.C:1528-1554,
// :1682-1742) with its scratch -- the per-chunk partial moments -- held in a
// fixed file-scope device array instead of a handle's allocation.  The
// reference has no counterpart of this entry point.
//
// Who needs it: code that reduces a distribution-function state held in its
// own device buffers while a solver owns the rest of the GPU -- a monitor or
// post-processing step between time steps, on its own stream, next to a
// solver that sized HBM for its DF state up front.  Such a caller cannot
// allocate: cudaMalloc fails once the solver holds the memory, and cudaFree
// synchronises the whole device, stalling the solver's queued work.
//
// Limits and rules (repeated in include/dugks.h):
//   * at most kNoAllocMaxCells cells per call (the scratch holds 15 partial
//     moments per cell and DV chunk; 16 MiB in all); larger calls are
//     rejected with DUGKS_ERR_ARG before anything is launched;
//   * the first call on a device looks up the scratch address
//     (cudaGetSymbolAddress) and caches it, keyed by the device's current
//     CUDA context: after cudaDeviceReset (or a released and re-created
//     primary context) the module may load at another address, and the
//     next call looks it up again; make the first call in each context
//     before any stream capture on that device;
//   * every buffer must have room for what the kernels touch: the call
//     checks each pointer's allocation range and rejects short buffers with
//     DUGKS_ERR_ARG before anything is launched;
//   * nothing has to start at zero: every call writes each scratch element
//     it reads before reading it;
//   * calls that overlap in time on one device (different streams, or
//     different host threads) share the scratch and race; serialise them.
#include <algorithm>
#include <mutex>
#include <cstdarg>
#include <cstdio>

#include <cuda.h>   // driver types for the entry points below; libcuda is not linked

#include "dugks_device.cuh"

namespace dugks {
namespace {

constexpr int kNoAllocMaxCells = 131072;
constexpr int kNoAllocMom = 15;                        // raw moments per cell (layout in dugks_internal.h)
constexpr size_t kNoAllocScratch = static_cast<size_t>(kNoAllocMaxCells) * 16;  // doubles (16 MiB)
constexpr int kNoAllocThreads = 128;
constexpr int kNoAllocTargetBlocks = 1184;             // 8 CTAs per SM on 148 SMs
constexpr int kNoAllocMaxDevices = 64;

// partial moments, SoA [chunk][moment][cell]
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

std::mutex g_noalloc_mutex;
// scratch address per device, and the id of the context it was looked up in
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
unsigned long long g_noalloc_ctx[kNoAllocMaxDevices] = {};

// driver entry points reached through the runtime (no link-time dependency
// on libcuda): the current context's unique id and allocation ranges
struct DriverFns {
    CUresult (*ctx_current)(CUcontext*) = nullptr;
    CUresult (*ctx_id)(CUcontext, unsigned long long*) = nullptr;
    CUresult (*addr_range)(CUdeviceptr*, size_t*, CUdeviceptr) = nullptr;
};

const DriverFns& driver_fns() {
    static const DriverFns f = [] {
        DriverFns d;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault) == cudaSuccess && p)
            d.ctx_current = reinterpret_cast<CUresult (*)(CUcontext*)>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault) == cudaSuccess && p)
            d.ctx_id = reinterpret_cast<CUresult (*)(CUcontext, unsigned long long*)>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault) == cudaSuccess && p)
            d.addr_range = reinterpret_cast<CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr)>(p);
        cudaGetLastError();
        return d;
    }();
    return f;
}

// unique id of the current context (0: unknown)
unsigned long long current_ctx_id() {
    const DriverFns& d = driver_fns();
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!d.ctx_current || !d.ctx_id || d.ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (d.ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// true when the allocation holding p extends at least `bytes` past p
bool has_room(const void* p, size_t bytes) {
    const DriverFns& d = driver_fns();
    if (!d.addr_range) return true;   // no range query on this driver: the type check alone
    CUdeviceptr base = 0;
    size_t size = 0;
    const CUdeviceptr dp = reinterpret_cast<CUdeviceptr>(p);
    if (d.addr_range(&base, &size, dp) != CUDA_SUCCESS) return false;
    return dp >= base && dp - base <= size && bytes <= size - (dp - base);
}

// raw moments of the DVs [d0, d1) of chunk blockIdx.y, one thread per cell;
// rows of g, h are contiguous in cells, so a warp reads coalesced
template <int D>
__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_partials(const double* __restrict__ xi,
                                                                      const double* __restrict__ w,
                                                                      const double* __restrict__ g,
                                                                      const double* __restrict__ hh, int nC, int nv,
                                                                      int chunks, double* __restrict__ scratch) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    const int ch = blockIdx.y;
    const int d0 = static_cast<int>(static_cast<long long>(nv) * ch / chunks);
    const int d1 = static_cast<int>(static_cast<long long>(nv) * (ch + 1) / chunks);
    double acc[kNoAllocMom];
    for (int j = 0; j < kNoAllocMom; ++j) acc[j] = 0.0;
    for (int d = d0; d < d1; ++d) {
        const double x[3] = {__ldg(xi + 3 * d), __ldg(xi + 3 * d + 1), D == 3 ? __ldg(xi + 3 * d + 2) : 0.0};
        const double x2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const size_t idx = static_cast<size_t>(d) * nC + c;
        accum<D>(acc, __ldg(w + d), x, x2, __ldg(g + idx), __ldg(hh + idx));
    }
    for (int j = 0; j < kNoAllocMom; ++j)
        scratch[(static_cast<size_t>(ch) * kNoAllocMom + j) * nC + c] = acc[j];
}

// sum of the chunk partials in chunk order, then the cell macros
__global__ void k_noalloc_macros(const double* __restrict__ scratch, int nC, int chunks, const Consts k,
                                 double* rho, double* U, double* T, double* q) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double s[kNoAllocMom];
    for (int j = 0; j < kNoAllocMom; ++j) s[j] = 0.0;
    for (int ch = 0; ch < chunks; ++ch)
        for (int j = 0; j < kNoAllocMom; ++j) s[j] += scratch[(static_cast<size_t>(ch) * kNoAllocMom + j) * nC + c];
    double r, u[3], t, qq[3], tau;
    macros_from_moments(s, k, r, u, t, qq, tau);
    const double fac = 2.0 * tau / (2.0 * tau + k.dt * k.Pr);  // fvDVM.C:1742
    if (rho) rho[c] = r;
    if (T) T[c] = t;
    for (int i = 0; i < 3; ++i) {
        if (U) U[3 * static_cast<size_t>(c) + i] = u[i];
        if (q) q[3 * static_cast<size_t>(c) + i] = qq[i] * fac;
    }
}

int report(char* msg, int32_t msg_len, int code, const char* fmt, ...) {
    if (msg && msg_len > 0) {
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(msg, static_cast<size_t>(msg_len), fmt, ap);
        va_end(ap);
    }
    return code;
}

// true when p is device (or managed) memory usable from the current device
bool on_device(const void* p, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace
}  // namespace dugks

extern "C" int dugks_cell_macros_noalloc(int32_t n_dims, int32_t n_dv, const double* xi, const double* w,
                                         int32_t n_cells, const double* g, const double* hh, const dugks_gas* gas,
                                         double dt, double* rho, double* U, double* T, double* q, void* stream,
                                         char* msg, int32_t msg_len) {
    using namespace dugks;
    if (msg && msg_len > 0) msg[0] = '\0';
    if (n_dims != 2 && n_dims != 3)
        return report(msg, msg_len, DUGKS_ERR_ARG, "dugks_cell_macros_noalloc: n_dims must be 2 or 3, got %d", n_dims);
    if (n_dv < 1 || n_cells < 0)
        return report(msg, msg_len, DUGKS_ERR_ARG, "dugks_cell_macros_noalloc: bad sizes n_dv=%d n_cells=%d", n_dv,
                      n_cells);
    if (n_cells > kNoAllocMaxCells)
        return report(msg, msg_len, DUGKS_ERR_ARG,
                      "dugks_cell_macros_noalloc: n_cells=%d exceeds the fixed scratch of this entry point "
                      "(at most %d cells per call)",
                      n_cells, kNoAllocMaxCells);
    if (!xi || !w || !g || !hh || !gas)
        return report(msg, msg_len, DUGKS_ERR_ARG, "dugks_cell_macros_noalloc: null input pointer");
    if (!(dt > 0.0) || !(gas->R > 0.0) || !(gas->mu_ref > 0.0) || !(gas->Tref > 0.0) || gas->K_inner < 0)
        return report(msg, msg_len, DUGKS_ERR_ARG, "dugks_cell_macros_noalloc: bad dt or gas parameters");
    if (n_cells == 0) return DUGKS_OK;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return report(msg, msg_len, DUGKS_ERR_CUDA, "dugks_cell_macros_noalloc: cudaGetDevice: %s",
                      cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return report(msg, msg_len, DUGKS_ERR_UNSUPPORTED, "dugks_cell_macros_noalloc: device %d out of range", dev);
    // every pointer the kernels touch must be device memory of this device,
    // so that a host buffer is turned into an error instead of a fault
    const void* ptrs[8] = {xi, w, g, hh, rho, U, T, q};
    for (int i = 0; i < 8; ++i)
        if (ptrs[i] && !on_device(ptrs[i], dev))
            return report(msg, msg_len, DUGKS_ERR_ARG,
                          "dugks_cell_macros_noalloc: argument %d is not device memory of the current device %d", i,
                          dev);
    // ... and long enough for what the kernels read and write
    const size_t nvc = static_cast<size_t>(n_dv) * n_cells, n1 = static_cast<size_t>(n_cells);
    const size_t need[8] = {3 * static_cast<size_t>(n_dv), static_cast<size_t>(n_dv), nvc, nvc, n1, 3 * n1, n1, 3 * n1};
    for (int i = 0; i < 8; ++i)
        if (ptrs[i] && !has_room(ptrs[i], need[i] * sizeof(double)))
            return report(msg, msg_len, DUGKS_ERR_ARG,
                          "dugks_cell_macros_noalloc: argument %d is too small (needs %zu doubles)", i, need[i]);

    double* scratch = nullptr;
    {
        // looked up once per device and context (a reset context may hold
        // the module at another address)
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        const unsigned long long ctx = current_ctx_id();
        if (!g_noalloc_ptr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                g_noalloc_ptr[dev] = nullptr;
                return report(msg, msg_len, DUGKS_ERR_CUDA, "dugks_cell_macros_noalloc: cudaGetSymbolAddress: %s",
                              cudaGetErrorString(e));
            }
            g_noalloc_ptr[dev] = static_cast<double*>(p);
            g_noalloc_ctx[dev] = ctx;
        }
        scratch = g_noalloc_ptr[dev];
    }

    // DV chunks: enough CTAs to fill the GPU, within the scratch; a function
    // of the sizes only, so the summation order is the same on every call
    const int nb = (n_cells + kNoAllocThreads - 1) / kNoAllocThreads;
    const int fit = static_cast<int>(kNoAllocScratch / (static_cast<size_t>(kNoAllocMom) * n_cells));
    int chunks = (kNoAllocTargetBlocks + nb - 1) / nb;
    chunks = std::max(1, std::min(chunks, std::min(fit, static_cast<int>(n_dv))));

    Consts k{};
    k.dt = dt;
    k.Pr1 = 1.0 - gas->Pr;
    k.K3D = gas->K_inner + 3.0 - n_dims;
    k.Kin = gas->K_inner;
    k.R = gas->R;
    k.omega = gas->omega;
    k.Tref = gas->Tref;
    k.muRef = gas->mu_ref;
    k.Pr = gas->Pr;
    k.D = n_dims;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 grid(nb, chunks);
    if (n_dims == 3)
        k_noalloc_partials<3><<<grid, kNoAllocThreads, 0, s>>>(xi, w, g, hh, n_cells, n_dv, chunks, scratch);
    else
        k_noalloc_partials<2><<<grid, kNoAllocThreads, 0, s>>>(xi, w, g, hh, n_cells, n_dv, chunks, scratch);
    k_noalloc_macros<<<(n_cells + 255) / 256, 256, 0, s>>>(scratch, n_cells, chunks, k, rho, U, T, q);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return report(msg, msg_len, DUGKS_ERR_CUDA, "dugks_cell_macros_noalloc: launch: %s", cudaGetErrorString(e));
    return DUGKS_OK;
}

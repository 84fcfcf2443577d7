// C ABI of the B200 DUGKS step (declarations and reference mapping in
// include/dugks.h).  Owns the device layout and drives the kernels.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "dugks_internal.h"
#include "dugks_kernels.cuh"

using dugks::set_error;

namespace {

constexpr double kPi = 3.14159265358979323846;

#define CUDA_TRY(h, call)                                                                               \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return set_error((h), e_ == cudaErrorMemoryAllocation ? DUGKS_ERR_OOM : DUGKS_ERR_CUDA,     \
                             std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

template <typename T>
int dev_alloc(dugks_handle* h, T** p, size_t count) {
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
        return set_error(h, e == cudaErrorMemoryAllocation ? DUGKS_ERR_OOM : DUGKS_ERR_CUDA,
                         "cudaMalloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
    h->allocations.push_back(q);
    *p = static_cast<T*>(q);
    return DUGKS_OK;
}

template <typename T>
int upload(dugks_handle* h, T** p, const std::vector<T>& v) {
    int st = dev_alloc(h, p, v.size());
    if (st) return st;
    if (!v.empty()) CUDA_TRY(h, cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return DUGKS_OK;
}

double inv_norm_host(double RT, int D) {
    const double t = 2.0 * kPi * RT;
    return D == 3 ? 1.0 / (t * std::sqrt(t)) : (D == 2 ? 1.0 / t : 1.0 / std::sqrt(t));
}

size_t real_size(const dugks_handle* h) { return h->precision == DUGKS_FP64 ? sizeof(double) : sizeof(float); }

dugks::StepArgs make_args(const dugks_handle* h, double dt, double dt_next) {
    dugks::StepArgs a{};
    a.dm = h->dm;
    a.ds = h->ds;
    a.dt = dt;
    a.dt_next = dt_next;
    a.chunks = h->chunks;
    a.chunk_begin = h->d_chunk_begin;
    a.hzero = h->h_zero ? 1 : 0;
    dugks::pass_config(h->D, h->precision, h->n1d, &a);
    return a;
}

// NCCL, opened on first use so that the library does not depend on it (and
// does not clash with another NCCL a host process has loaded: dlopen of the
// same soname returns that one)
struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
    std::string error;
};

const NcclApi& nccl_api() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) {
            const char* e = dlerror();
            api.error = std::string("cannot load NCCL: ") + (e ? e : "libnccl.so.2 not found");
            return;
        }
        api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(dlsym(lib, "ncclGetUniqueId"));
        api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(dlsym(lib, "ncclCommInitRank"));
        api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(dlsym(lib, "ncclAllReduce"));
        api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(dlsym(lib, "ncclCommDestroy"));
        api.error_string = reinterpret_cast<decltype(api.error_string)>(dlsym(lib, "ncclGetErrorString"));
        if (!api.get_unique_id || !api.comm_init_rank || !api.all_reduce || !api.comm_destroy || !api.error_string) {
            api.error = "NCCL library lacks a needed symbol";
            api.get_unique_id = nullptr;
        }
    });
    return api;
}

// the sum over all shards of n doubles at buf (device), on the handle's stream
int shard_allreduce(dugks_handle* h, double* buf, size_t n) {
    if (!h->shard_nccl || n == 0) return DUGKS_OK;
    const NcclApi& api = nccl_api();
    const ncclResult_t r = api.all_reduce(buf, buf, n, ncclDouble, ncclSum, static_cast<ncclComm_t>(h->nccl_comm),
                                          h->stream);
    if (r != ncclSuccess) return set_error(h, DUGKS_ERR_CUDA, std::string("ncclAllReduce: ") + api.error_string(r));
    return DUGKS_OK;
}

bool sharded(const dugks_handle* h) { return h->shard_world > 1 || h->shard_nccl; }

int check_device_errors(dugks_handle* h) {
    int err[4] = {0, 0, 0, 0};
    CUDA_TRY(h, cudaMemcpyAsync(err, h->ds.err, sizeof err, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (err[0] & 1) return set_error(h, DUGKS_ERR_NAN, "non-finite or non-positive rho/T in the cell macros");
    if (err[0] & 2) return set_error(h, DUGKS_ERR_TIMEOUT, "a bounded device wait ran out");
    if (err[0] & 4)
        return set_error(h, DUGKS_ERR_ARG, "an index in the device tables was out of range (bounds-checked build)");
    return DUGKS_OK;
}

}  // namespace

extern "C" {

int dugks_abi_version(void) { return DUGKS_ABI_VERSION; }

void dugks_default_options(dugks_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof *opt);
    opt->precision = DUGKS_FP64;
    opt->ls_weighting = DUGKS_LS_MAGSF;
}

// dv: a tensor-product set; dvl: a DV list (exactly one of them)
static int create_impl(const dugks_mesh* mesh, const dugks_dv_set* dv, const dugks_dv_list* dvl,
                       const dugks_gas* gas, const dugks_bc* bc, const dugks_options* opt_in,
                       const dugks_dv_shard* shard, dugks_handle** out) {
    if (!out) return DUGKS_ERR_ARG;
    *out = nullptr;
    if (!mesh || (!dv && !dvl) || !gas || !bc) return DUGKS_ERR_ARG;
    dugks_options opt;
    dugks_default_options(&opt);
    if (opt_in) opt = *opt_in;
    dugks_handle* h = new (std::nothrow) dugks_handle();
    if (!h) return DUGKS_ERR_OOM;
    auto fail = [&](int code, const std::string& msg) {
        // keep the handle so that the caller can read the message
        set_error(h, code, msg);
        *out = h;
        return code;
    };
    if (mesh->n_cells <= 0 || mesh->n_internal_faces < 0 || mesh->n_boundary_faces < 0 || !mesh->owner ||
        (mesh->n_internal_faces > 0 && !mesh->neighbour) || !mesh->cell_centres || !mesh->cell_volumes ||
        !mesh->face_centres || !mesh->face_areas || mesh->n_patches < 0 ||
        (mesh->n_patches > 0 && !mesh->patch_start))
        return fail(DUGKS_ERR_ARG, "dugks_create: incomplete mesh");
    if (mesh->n_solution_dims != 2 && mesh->n_solution_dims != 3)
        return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create: n_solution_dims must be 2 or 3");
    if (dvl) {
        if (dvl->n_dv < 1 || !dvl->xi || !dvl->weights) return fail(DUGKS_ERR_ARG, "dugks_create_dv_list: empty DV list");
    } else if (dv->n_per_dim < 1 || !dv->xis || !dv->weights) {
        return fail(DUGKS_ERR_ARG, "dugks_create: empty DV set");
    }
    if (!dvl && dv->n_per_dim > dugks::kMaxN1d)
        return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create: more than 64 DV nodes per dimension");
    if (opt.precision != DUGKS_FP64 && opt.precision != DUGKS_FP32C)
        return fail(DUGKS_ERR_ARG, "dugks_create: unknown precision");
    if (!(gas->R > 0) || !(gas->Tref > 0) || !(gas->mu_ref > 0)) return fail(DUGKS_ERR_ARG, "dugks_create: bad gas");
    h->precision = opt.precision;
    h->device = opt.device;
    h->D = mesh->n_solution_dims;
    h->nC = mesh->n_cells;
    h->nIF = mesh->n_internal_faces;
    h->nBF = mesh->n_boundary_faces;
    h->nP = mesh->n_patches;
    h->gas = *gas;
    h->xi_max = dvl ? dvl->xi_max : dv->xi_max;
    const int nC = h->nC, nIF = h->nIF, nBF = h->nBF, nF = nIF + nBF;
    h->owner.assign(mesh->owner, mesh->owner + nF);
    h->neighbour.assign(mesh->neighbour, mesh->neighbour + nIF);
    for (int f = 0; f < nF; ++f)
        if (h->owner[f] < 0 || h->owner[f] >= nC) return fail(DUGKS_ERR_ARG, "dugks_create: owner out of range");
    for (int f = 0; f < nIF; ++f)
        if (h->neighbour[f] < 0 || h->neighbour[f] >= nC || h->neighbour[f] == h->owner[f])
            return fail(DUGKS_ERR_ARG, "dugks_create: neighbour out of range");
    h->C.assign(mesh->cell_centres, mesh->cell_centres + 3 * static_cast<size_t>(nC));
    h->V.assign(mesh->cell_volumes, mesh->cell_volumes + nC);
    for (int c = 0; c < nC; ++c)
        if (!(h->V[c] > 0) || !std::isfinite(h->V[c])) return fail(DUGKS_ERR_ARG, "dugks_create: non-positive cell volume");
    h->Cf.assign(mesh->face_centres, mesh->face_centres + 3 * static_cast<size_t>(nF));
    h->Sf.assign(mesh->face_areas, mesh->face_areas + 3 * static_cast<size_t>(nF));
    for (size_t i = 0; i < 3 * static_cast<size_t>(nC); ++i)
        if (!std::isfinite(h->C[i])) return fail(DUGKS_ERR_ARG, "dugks_create: non-finite cell centre");
    for (size_t i = 0; i < 3 * static_cast<size_t>(nF); ++i)
        if (!std::isfinite(h->Cf[i]) || !std::isfinite(h->Sf[i]))
            return fail(DUGKS_ERR_ARG, "dugks_create: non-finite face centre or area");
    {
        // every cell is the owner or neighbour of some face (a cell without
        // faces has no flux list and no gradient stencil)
        std::vector<unsigned char> seen(nC, 0);
        for (int f = 0; f < nF; ++f) seen[h->owner[f]] = 1;
        for (int f = 0; f < nIF; ++f) seen[h->neighbour[f]] = 1;
        for (int c = 0; c < nC; ++c)
            if (!seen[c]) return fail(DUGKS_ERR_ARG, "dugks_create: cell " + std::to_string(c) + " has no faces");
    }
    h->patch_start.assign(mesh->patch_start, mesh->patch_start + h->nP + 1);
    if (h->nP == 0) h->patch_start.assign(1, 0);
    if (h->patch_start[0] != 0 || h->patch_start[h->nP] != nBF)
        return fail(DUGKS_ERR_ARG, "dugks_create: patch_start must span the boundary faces");
    h->patch_type.assign(bc->patch_type, bc->patch_type + h->nP);
    h->bface_ptype.assign(nBF, 0);
    h->bface_patch_local.assign(nBF, 0);
    bool any_pressure = false, any_symmetry = false;
    for (int p = 0; p < h->nP; ++p) {
        const int pt = h->patch_type[p];
        if (pt < DUGKS_PATCH_MAXWELL_WALL || pt > DUGKS_PATCH_PRESSURE_OUT)
            return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create: unsupported patch type " + std::to_string(pt));
        any_pressure = any_pressure || pt == DUGKS_PATCH_PRESSURE_IN || pt == DUGKS_PATCH_PRESSURE_OUT;
        any_symmetry = any_symmetry || pt == DUGKS_PATCH_SYMMETRY || pt == DUGKS_PATCH_DVM_SYMMETRY;
        if (h->patch_start[p + 1] < h->patch_start[p]) return fail(DUGKS_ERR_ARG, "dugks_create: bad patch_start");
        for (int b = h->patch_start[p]; b < h->patch_start[p + 1]; ++b) {
            h->bface_ptype[b] = h->patch_type[p];
            h->bface_patch_local[b] = b - h->patch_start[p];
        }
    }
    // the boundary relaxation of h takes the internal-face temperature at the
    // face's patch-local index (fvDVM.C:1367, :1413; macroFlux the internal
    // Sf there, :1668-1669); a patch with more faces than the mesh has
    // internal faces would read past them, which the reference leaves undefined
    for (int p = 0; p < h->nP; ++p)
        if (h->patch_start[p + 1] - h->patch_start[p] > nIF)
            return fail(DUGKS_ERR_UNSUPPORTED,
                        "dugks_create: patch " + std::to_string(p) + " has " +
                            std::to_string(h->patch_start[p + 1] - h->patch_start[p]) + " faces, more than the " +
                            std::to_string(nIF) + " internal faces its patch-local indices address");
    if (nBF > 0 && (!bc->rho || !bc->U || !bc->T)) return fail(DUGKS_ERR_ARG, "dugks_create: missing BC values");
    h->bc_rho.assign(bc->rho, bc->rho + nBF);
    h->bc_U.assign(bc->U, bc->U + 3 * static_cast<size_t>(nBF));
    h->bc_T.assign(bc->T, bc->T + nBF);
    h->bc_p.assign(nBF, 0.0);
    if (any_pressure) {
        if (!bc->p) return fail(DUGKS_ERR_ARG, "dugks_create: pressure patches need bc->p");
        h->bc_p.assign(bc->p, bc->p + nBF);
        for (int b = 0; b < nBF; ++b) {
            const int pt = h->bface_ptype[b];
            if ((pt == DUGKS_PATCH_PRESSURE_IN || pt == DUGKS_PATCH_PRESSURE_OUT) &&
                (!(h->bc_p[b] > 0) || !std::isfinite(h->bc_p[b])))
                return fail(DUGKS_ERR_ARG, "dugks_create: pressure must be > 0");
        }
    }
    if (any_symmetry && dvl)
        return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create_dv_list: symmetry patches need a tensor-product DV set");
    if (any_symmetry && shard && shard->world > 1)
        return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create_sharded: symmetry patches need the whole DV set on one handle");
    // tensor-product DV set, x fastest (fvDVM.C:293-374); a DV list as given
    // (the unstructured velocity mesh, fvDVM.C:166-196), one DV per "row"
    const int n = dvl ? 1 : dv->n_per_dim;
    h->n1d = n;
    if (dvl) {
        for (int d = 0; d < dvl->n_dv; ++d) {
            h->w.push_back(dvl->weights[d]);
            h->xi.insert(h->xi.end(), {dvl->xi[3 * d], dvl->xi[3 * d + 1], h->D == 3 ? dvl->xi[3 * d + 2] : 0.0});
        }
    } else if (h->D == 3) {
        for (int iz = 0; iz < n; ++iz)
            for (int iy = 0; iy < n; ++iy)
                for (int ix = 0; ix < n; ++ix) {
                    h->w.push_back(dv->weights[iz] * dv->weights[iy] * dv->weights[ix]);
                    h->xi.insert(h->xi.end(), {dv->xis[ix], dv->xis[iy], dv->xis[iz]});
                }
    } else {
        for (int iy = 0; iy < n; ++iy)
            for (int ix = 0; ix < n; ++ix) {
                h->w.push_back(dv->weights[iy] * dv->weights[ix] * 1);
                h->xi.insert(h->xi.end(), {dv->xis[ix], dv->xis[iy], 0.0});
            }
    }
    h->nv = static_cast<int>(h->w.size());
    // symmetry patches: the reference mirrors incoming DV d into DV
    // round(|n . (symmX, symmY, symmZ)(d)|), n the unit normal of the patch's
    // first face (discreteVelocity.C:735-738, :762-764; ids fvDVM.C:300-372).
    // That is the mirror along one axis when n is (nearly) a coordinate axis;
    // other planes are rejected.
    h->bface_mirror.assign(nBF, -1);
    for (int p = 0; p < h->nP; ++p) {
        const int pt = h->patch_type[p];
        if (pt != DUGKS_PATCH_SYMMETRY && pt != DUGKS_PATCH_DVM_SYMMETRY) continue;
        if (h->patch_start[p + 1] == h->patch_start[p]) continue;
        const double* S = &h->Sf[3 * static_cast<size_t>(nIF + h->patch_start[p])];
        const double mS = std::sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
        int axis = -1;
        for (int k = 0; k < h->D && axis < 0; ++k) {
            bool all = true;
            for (int d = 0; d < h->nv && all; ++d) {
                const int ix = d % n, iy = (d / n) % n, iz = h->D == 3 ? d / (n * n) : 0;
                double t[3];
                if (h->D == 3) {
                    t[0] = iz * n * n + iy * n + (n - ix - 1);
                    t[1] = iz * n * n + (n - iy - 1) * n + ix;
                    t[2] = (n - iz - 1) * n * n + iy * n + ix;
                } else {
                    t[0] = iy * n + (n - ix - 1);
                    t[1] = (n - iy - 1) * n + ix;
                    t[2] = 0;
                }
                const double target = std::round(std::fabs(S[0] / mS * t[0] + S[1] / mS * t[1] + S[2] / mS * t[2]));
                all = target == t[k];
            }
            if (all) axis = k;
        }
        if (axis < 0) return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create: symmetry patch not normal to a coordinate axis");
        for (int b = h->patch_start[p]; b < h->patch_start[p + 1]; ++b) h->bface_mirror[b] = axis;
    }
    if (opt.ls_weighting < 0 || opt.ls_weighting > 2) return fail(DUGKS_ERR_ARG, "dugks_create: bad ls_weighting");
    dugks::compute_weights_and_ls(h, opt.ls_weighting);
    for (double x : h->lsP)
        if (!std::isfinite(x)) return fail(DUGKS_ERR_ARG, "dugks_create: singular least-squares system");

    // tiles: at most kMaxTile cells, kMaxLocal cells with the ring, and one
    // item per thread.  By default greedy tiles as large as those limits
    // allow; a given tile_cells cuts uniform tiles, shrunk until the largest
    // fits
    if (opt.tile_cells > 0) {
        int tile = std::min(opt.tile_cells, dugks::kMaxTile);
        for (;;) {
            dugks::build_tiling(h, tile);
            const bool fits = h->tiling.max_items <= dugks::kMaxItems && h->tiling.max_local <= dugks::kMaxLocal;
            if (fits || tile <= 4) break;
            tile = std::max(4, tile * 7 / 8);
        }
    } else {
        dugks::build_tiling(h, 0);
    }
    if (h->tiling.max_items > dugks::kMaxItems || h->tiling.max_local > dugks::kMaxLocal)
        return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create: cells with too many faces for the tile layout");
    // DV chunks: enough CTAs to fill the GPU several times over
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= 0)
        return fail(DUGKS_ERR_CUDA, "dugks_create: no CUDA device");
    if (h->device < 0 || h->device >= dev_count) return fail(DUGKS_ERR_ARG, "dugks_create: bad device ordinal");
    cudaError_t ce = cudaSetDevice(h->device);
    if (ce != cudaSuccess) return fail(DUGKS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    // one CTA per SM runs at a time; aim at about two waves.  Chunks are
    // whole DV rows (n1d DVs along x at fixed y, z): the passes walk a row in
    // batches and factor the x direction out of their sums
    const int rows = h->nv / h->n1d;
    // velocity-space shard: this device's block of DV rows
    int row0 = 0, row1 = rows;
    if (shard) {
        if (shard->world < 1 || shard->rank < 0 || shard->rank >= shard->world)
            return fail(DUGKS_ERR_ARG, "dugks_create_sharded: bad rank or world");
        if (shard->world > rows)
            return fail(DUGKS_ERR_ARG, "dugks_create_sharded: more shards than DV rows (" + std::to_string(rows) + ")");
        h->shard_rank = shard->rank;
        h->shard_world = shard->world;
        row0 = static_cast<int>(static_cast<int64_t>(rows) * shard->rank / shard->world);
        row1 = static_cast<int>(static_cast<int64_t>(rows) * (shard->rank + 1) / shard->world);
    }
    const int rows_loc = row1 - row0;
    int chunks = opt.dv_chunks > 0 ? opt.dv_chunks : (2 * sms + h->tiling.n_tiles - 1) / h->tiling.n_tiles;
    chunks = std::max(1, std::min(chunks, rows_loc));
    h->chunks = chunks;
    h->chunk_begin.resize(chunks + 1);
    for (int c = 0; c <= chunks; ++c)
        h->chunk_begin[c] = row0 + static_cast<int32_t>((static_cast<int64_t>(rows_loc) * c) / chunks);

    // ---- device layout ----
    const dugks::Tiling& t = h->tiling;
    dugks::DevMesh& dm = h->dm;
    dm.D = h->D;
    dm.K = gas->K_inner;
    dm.R = gas->R;
    dm.Pr = gas->Pr;
    dm.omega = gas->omega;
    dm.Tref = gas->Tref;
    dm.muRef = gas->mu_ref;
    dm.nC = nC;
    dm.nIF = nIF;
    dm.nBF = nBF;
    dm.nv = h->nv;
    dm.row_base = row0;
    dm.dv_base = row0 * h->n1d;
    dm.nv_loc = rows_loc * h->n1d;
    dm.prec = h->precision;
    dm.n1d = h->n1d;
    dm.general_dv = dvl ? 1 : 0;
    dm.n_tiles = t.n_tiles;
    dm.n_items = t.n_items();
    dm.nb_max = t.nb_max;
    dm.nf_max = t.nf_max;
    dm.xi_max_co = std::sqrt(static_cast<double>(h->D)) * h->xi_max;
    int st;
    ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(DUGKS_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(ce));
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    double *d_xi, *d_w, *d_grad_ls, *d_dtV, *d_dc, *d_bS, *d_geo;
    int32_t *d_tb, *d_tlo, *d_lc, *d_tio, *d_gnb, *d_cfi, *d_fi, *d_bpl, *d_bpt, *d_bown;
    int32_t *d_meta, *d_loc, *d_face, *d_other, *d_bmir;
    std::vector<double> dtV(nC);
    for (int c = 0; c < nC; ++c) dtV[c] = 1.0 / h->V[t.perm[c]];
    std::vector<double> bS(3 * static_cast<size_t>(nBF));
    std::vector<int32_t> bown(nBF);
    for (int b = 0; b < nBF; ++b) {
        for (int k = 0; k < 3; ++k) bS[3 * b + k] = h->Sf[3 * (nIF + b) + k];
        bown[b] = t.iperm[h->owner[nIF + b]];
    }
    if (dvl) {
        h->X1.assign(1, 0.0);
        h->W1.assign(1, 1.0);
    } else {
        h->X1.assign(dv->xis, dv->xis + h->n1d);
        h->W1.assign(dv->weights, dv->weights + h->n1d);
    }
    double *d_X1, *d_W1;
    if ((st = upload(h, &d_X1, h->X1)) || (st = upload(h, &d_W1, h->W1)) ||
        (st = upload(h, &d_xi, h->xi)) || (st = upload(h, &d_w, h->w)) || (st = upload(h, &d_tb, t.tile_begin)) ||
        (st = upload(h, &d_tlo, t.tile_loc_off)) || (st = upload(h, &d_lc, t.loc_cells)) ||
        (st = upload(h, &d_tio, t.tile_item_off)) || (st = upload(h, &d_meta, t.it_meta)) ||
        (st = upload(h, &d_loc, t.it_loc)) || (st = upload(h, &d_face, t.it_face)) ||
        (st = upload(h, &d_other, t.it_other)) || (st = upload(h, &d_geo, t.it_geo)) ||
        (st = upload(h, &d_gnb, t.grad_nb)) || (st = upload(h, &d_grad_ls, t.grad_ls)) ||
        (st = upload(h, &d_cfi, t.cf_item)) || (st = upload(h, &d_dtV, dtV)) || (st = upload(h, &d_fi, t.face_items)) ||
        (st = upload(h, &d_bpl, h->bface_patch_local)) || (st = upload(h, &d_bpt, h->bface_ptype)) ||
        (st = upload(h, &d_bown, bown)) || (st = upload(h, &d_dc, h->dc)) || (st = upload(h, &d_bS, bS)) ||
        (st = upload(h, &d_bmir, h->bface_mirror)) ||
        (st = upload(h, &h->d_chunk_begin, h->chunk_begin))) {
        *out = h;
        return st;
    }
    dm.X1 = d_X1;
    dm.W1 = d_W1;
    dm.xi = d_xi;
    dm.w = d_w;
    dm.tile_begin = d_tb;
    dm.tile_loc_off = d_tlo;
    dm.loc_cells = d_lc;
    dm.tile_item_off = d_tio;
    dm.it_meta = d_meta;
    dm.it_loc = d_loc;
    dm.it_face = d_face;
    dm.it_other = d_other;
    dm.it_geo = d_geo;
    dm.grad_nb = d_gnb;
    dm.grad_ls = d_grad_ls;
    dm.cf_item = d_cfi;
    dm.dtV = d_dtV;
    dm.face_items = d_fi;
    dm.bface_patch_local = d_bpl;
    dm.bface_ptype = d_bpt;
    dm.bface_owner = d_bown;
    dm.bface_mirror = d_bmir;
    // macroFlux yes: the faces of every cell in face order (internal, then
    // boundary), as the reference's face loops visit them
    dm.macro_flux = opt.macro_flux ? 1 : 0;
    dm.mf_off = nullptr;
    dm.mf_ent = nullptr;
    dm.mf_Sf = nullptr;
    dm.mf_V = nullptr;
    if (dm.macro_flux) {
        std::vector<int32_t> cnt(nC + 1, 0), off(nC + 1, 0), ent(2 * static_cast<size_t>(nIF) + nBF);
        for (int f = 0; f < nF; ++f) {
            ++cnt[t.iperm[h->owner[f]]];
            if (f < nIF) ++cnt[t.iperm[h->neighbour[f]]];
        }
        for (int c = 0; c < nC; ++c) off[c + 1] = off[c] + cnt[c];
        std::vector<int32_t> pos(off.begin(), off.end() - 1);
        for (int f = 0; f < nF; ++f) {
            ent[pos[t.iperm[h->owner[f]]]++] = 2 * f;
            if (f < nIF) ent[pos[t.iperm[h->neighbour[f]]]++] = 2 * f + 1;
        }
        std::vector<double> Vr(nC);
        for (int c = 0; c < nC; ++c) Vr[c] = h->V[t.perm[c]];
        int32_t *d_mo, *d_me;
        double *d_ms, *d_mv;
        if ((st = upload(h, &d_mo, off)) || (st = upload(h, &d_me, ent)) || (st = upload(h, &d_ms, h->Sf)) ||
            (st = upload(h, &d_mv, Vr))) {
            *out = h;
            return st;
        }
        dm.mf_off = d_mo;
        dm.mf_ent = d_me;
        dm.mf_Sf = d_ms;
        dm.mf_V = d_mv;
    }
    dm.n_sym_faces = dm.n_pressure_faces = 0;
    for (int b = 0; b < nBF; ++b) {
        const int pt = h->bface_ptype[b];
        if (pt == DUGKS_PATCH_SYMMETRY || pt == DUGKS_PATCH_DVM_SYMMETRY) ++dm.n_sym_faces;
        if (pt == DUGKS_PATCH_PRESSURE_IN || pt == DUGKS_PATCH_PRESSURE_OUT) ++dm.n_pressure_faces;
    }
    dm.dc = d_dc;
    dm.bS = d_bS;
    dugks::DevState& ds = h->ds;
    const size_t rs = real_size(h);
    const size_t nvc = static_cast<size_t>(dm.nv_loc) * nC;
    const size_t nfv = static_cast<size_t>(dm.nv_loc) * std::max(dm.n_items, 1);
    unsigned char* p;
    // One state buffer.  Pass B reads each (DV, cell) entry of its own L0
    // cells once and then writes it, and no kernel of a step reads the old
    // state after pass B, so the update runs in place: g[1], h[1] alias
    // g[0], h[0] and the step's buffer flip changes nothing.  This halves
    // the state's HBM (the FP64 64^3 x 20^3 cube fits one B200 with it).
    if ((st = dev_alloc(h, &p, nvc * rs))) return *out = h, st;
    ds.g[0] = ds.g[1] = p;
    if ((st = dev_alloc(h, &p, nvc * rs))) return *out = h, st;
    ds.h[0] = ds.h[1] = p;
    if ((st = dev_alloc(h, &p, nfv * rs))) return *out = h, st;
    ds.fvg = p;
    if ((st = dev_alloc(h, &p, nfv * rs))) return *out = h, st;
    ds.fvh = p;
    // face values start at zero: with h identically zero no pass writes fvh,
    // and the symmetry pass reads its boundary slots
    if (cudaMemset(ds.fvg, 0, nfv * rs) != cudaSuccess || cudaMemset(ds.fvh, 0, nfv * rs) != cudaSuccess)
        return fail(DUGKS_ERR_CUDA, "cudaMemset of the face values");
    ds.cur = 0;
    if ((st = dev_alloc(h, &ds.partF, static_cast<size_t>(chunks) * dm.n_items * dugks::kNM)) ||
        (st = dev_alloc(h, &ds.partC, static_cast<size_t>(chunks) * nC * dugks::kNM)) ||
        (dvl && opt.macro_flux && (st = dev_alloc(h, &ds.partX, static_cast<size_t>(chunks) * nC * dugks::kFX))) ||
        (dvl && opt.macro_flux && shard &&
         (st = dev_alloc(h, &ds.redC, static_cast<size_t>(nC) * (dugks::kNM + dugks::kFX)))) ||
        (st = dev_alloc(h, &ds.cellrec, static_cast<size_t>(dugks::REC_N) * nC)) ||
        (st = dev_alloc(h, &ds.facerec, static_cast<size_t>(dugks::REC_N) * dm.n_items)) ||
        (st = dev_alloc(h, &ds.ctab, static_cast<size_t>(h->D) * h->n1d * nC)) ||
        (st = dev_alloc(h, &ds.ftab, static_cast<size_t>(h->D) * h->n1d * dm.n_items)) ||
        (st = dev_alloc(h, &ds.brec, nBF)) || (st = dev_alloc(h, &ds.bmom_in, static_cast<size_t>(nBF) * dugks::kNM)) ||
        (st = dev_alloc(h, &ds.cm, static_cast<size_t>(nC) * 9)) ||
        (st = dev_alloc(h, &ds.fm, static_cast<size_t>(nF) * 9)) || (st = dev_alloc(h, &ds.co, 2)) ||
        (st = dev_alloc(h, &ds.err, 4)) || (st = dev_alloc(h, &h->d_dt, 2))) {
        *out = h;
        return st;
    }
    if (h->precision == DUGKS_FP32C && !dvl) {
        double *d_gref, *d_href;
        if ((st = dev_alloc(h, &d_gref, dm.nv_loc)) || (st = dev_alloc(h, &d_href, dm.nv_loc)) ||
            (st = dev_alloc(h, &ds.refmom, static_cast<size_t>(chunks) * dugks::kNM))) {
            *out = h;
            return st;
        }
        dm.gref = d_gref;
        dm.href = d_href;
    } else {
        dm.gref = dm.href = nullptr;
        ds.refmom = nullptr;
    }
    ce = cudaMemset(ds.err, 0, 4 * sizeof(int));
    if (ce != cudaSuccess) return fail(DUGKS_ERR_CUDA, cudaGetErrorString(ce));
    ce = cudaMemset(ds.partF, 0, static_cast<size_t>(chunks) * dm.n_items * dugks::kNM * sizeof(double));
    if (ce != cudaSuccess) return fail(DUGKS_ERR_CUDA, cudaGetErrorString(ce));
    dugks::StepArgs a = make_args(h, 0.0, 0.0);
    ce = dugks::configure_kernels(h->precision, a);
    if (ce != cudaSuccess) return fail(DUGKS_ERR_CUDA, std::string("configure kernels: ") + cudaGetErrorString(ce));
    if (shard && shard->use_nccl) {
        // collective: every rank of the shard set makes this call
        const NcclApi& api = nccl_api();
        if (!api.get_unique_id) return fail(DUGKS_ERR_UNSUPPORTED, "dugks_create_sharded: " + api.error);
        ncclUniqueId id;
        static_assert(sizeof id == sizeof shard->nccl_id, "NCCL unique id size");
        std::memcpy(&id, shard->nccl_id, sizeof id);
        ncclComm_t comm = nullptr;
        const ncclResult_t r = api.comm_init_rank(&comm, shard->world, id, shard->rank);
        if (r != ncclSuccess) return fail(DUGKS_ERR_CUDA, std::string("ncclCommInitRank: ") + api.error_string(r));
        h->nccl_comm = comm;
        h->shard_nccl = true;
    }
    *out = h;
    return DUGKS_OK;
}

int dugks_create(const dugks_mesh* mesh, const dugks_dv_set* dv, const dugks_gas* gas, const dugks_bc* bc,
                 const dugks_options* opt, dugks_handle** out) {
    return create_impl(mesh, dv, nullptr, gas, bc, opt, nullptr, out);
}

int dugks_create_sharded(const dugks_mesh* mesh, const dugks_dv_set* dv, const dugks_gas* gas, const dugks_bc* bc,
                         const dugks_options* opt, const dugks_dv_shard* shard, dugks_handle** out) {
    if (!shard) {
        if (out) *out = nullptr;
        return DUGKS_ERR_ARG;
    }
    return create_impl(mesh, dv, nullptr, gas, bc, opt, shard, out);
}

int dugks_create_dv_list(const dugks_mesh* mesh, const dugks_dv_list* dv, const dugks_gas* gas, const dugks_bc* bc,
                         const dugks_options* opt, const dugks_dv_shard* shard, dugks_handle** out) {
    if (!dv) {
        if (out) *out = nullptr;
        return DUGKS_ERR_ARG;
    }
    return create_impl(mesh, nullptr, dv, gas, bc, opt, shard, out);
}

int dugks_nccl_unique_id(unsigned char id[128]) {
    if (!id) return DUGKS_ERR_ARG;
    const NcclApi& api = nccl_api();
    if (!api.get_unique_id) return DUGKS_ERR_UNSUPPORTED;
    ncclUniqueId u;
    if (api.get_unique_id(&u) != ncclSuccess) return DUGKS_ERR_CUDA;
    std::memcpy(id, &u, sizeof u);
    return DUGKS_OK;
}

int dugks_dv_range(const dugks_handle* h, int32_t* first_dv, int32_t* n_dv_local) {
    if (!h || !first_dv || !n_dv_local) return DUGKS_ERR_ARG;
    *first_dv = h->dm.dv_base;
    *n_dv_local = h->dm.nv_loc;
    return DUGKS_OK;
}

int dugks_set_macros(dugks_handle* h, const double* rho, const double* U, const double* T) {
    if (!h) return DUGKS_ERR_ARG;
    if (!rho || !U || !T) return set_error(h, DUGKS_ERR_ARG, "dugks_set_macros: null field");
    CUDA_TRY(h, cudaSetDevice(h->device));
    const int nC = h->nC, nIF = h->nIF, nBF = h->nBF, D = h->D;
    const double R = h->gas.R;
    const dugks::Tiling& t = h->tiling;
    std::vector<double> cm(static_cast<size_t>(nC) * 9);
    std::vector<double> cr(static_cast<size_t>(dugks::REC_N) * nC, 0.0);
    for (int c = 0; c < nC; ++c) {
        const int o = t.perm[c];
        // a non-finite or non-positive macroscopic state is refused as the
        // step refuses one it computes (DUGKS_ERR_NAN), before any launch
        if (!(rho[o] > 0) || !(T[o] > 0) || !std::isfinite(rho[o]) || !std::isfinite(T[o]) ||
            !std::isfinite(U[3 * o]) || !std::isfinite(U[3 * o + 1]) || !std::isfinite(U[3 * o + 2]))
            return set_error(h, DUGKS_ERR_NAN,
                             "dugks_set_macros: non-finite or non-positive rho/T (or non-finite U) in cell " +
                                 std::to_string(o));
        const double tau = h->gas.mu_ref * std::exp(h->gas.omega * std::log(T[o] / h->gas.Tref)) / rho[o] / T[o] / R;
        double* m = &cm[9 * static_cast<size_t>(c)];
        m[0] = rho[o];
        m[1] = U[3 * o];
        m[2] = U[3 * o + 1];
        m[3] = U[3 * o + 2];
        m[4] = T[o];
        m[5] = m[6] = m[7] = 0.0;
        m[8] = tau;
        const double RT = R * T[o];
        const size_t n = static_cast<size_t>(nC);
        cr[dugks::REC_UX * n + c] = m[1];
        cr[dugks::REC_UY * n + c] = m[2];
        cr[dugks::REC_UZ * n + c] = m[3];
        cr[dugks::REC_INVRT * n + c] = 1.0 / RT;
        cr[dugks::REC_A * n + c] = rho[o] * inv_norm_host(RT, D);
        cr[dugks::REC_RTH * n + c] = RT;  // relax factor and heat-flux terms stay 0 (q = 0)
    }
    // boundary records
    const double K3D = h->gas.K_inner + 3.0 - D;
    std::vector<dugks::BRec> br(nBF);
    for (int b = 0; b < nBF; ++b) {
        const int pt = h->bface_ptype[b];
        // zeroGradient and symmetry faces take no patch values
        const bool uses_values = pt != DUGKS_PATCH_ZERO_GRADIENT && pt != DUGKS_PATCH_SYMMETRY &&
                                 pt != DUGKS_PATCH_DVM_SYMMETRY;
        const double RT = uses_values ? R * h->bc_T[b] : R * h->gas.Tref;
        if (!(RT > 0)) return set_error(h, DUGKS_ERR_ARG, "dugks_set_macros: boundary T must be > 0");
        br[b].U[0] = h->bc_U[3 * b];
        br[b].U[1] = h->bc_U[3 * b + 1];
        br[b].U[2] = h->bc_U[3 * b + 2];
        br[b].K_in = inv_norm_host(RT, D);
        br[b].invRT_in = 1.0 / RT;
        br[b].hfac = RT * K3D;
        br[b].rho_in = h->bface_ptype[b] == DUGKS_PATCH_MAXWELL_WALL ? 1.0 : h->bc_rho[b];
        br[b].inByRho = 0.0;
        br[b].T = h->bc_T[b];
        br[b].p = h->bc_p[b];
    }
    // face velocity for the first Courant number: linear interpolation
    // (fvDVM.C:2116), U_f = w (U_own - U_nei) + U_nei
    std::vector<double> fm(static_cast<size_t>(nIF + nBF) * 9, 0.0);
    double co_max = 0, co_sum = 0;
    for (int f = 0; f < nIF; ++f) {
        const int64_t o = h->owner[f], n = h->neighbour[f];
        double u2 = 0;
        for (int k = 0; k < 3; ++k) {
            const double uf = h->weights[f] * (U[3 * o + k] - U[3 * n + k]) + U[3 * n + k];
            fm[9 * static_cast<size_t>(f) + 1 + k] = uf;
            u2 += uf * uf;
        }
        const double co = h->dc[f] * (std::sqrt(u2) + h->dm.xi_max_co);
        co_max = std::max(co_max, co);
        co_sum += co;
    }
    double co_host[2];
    std::memcpy(&co_host[0], &co_max, sizeof(double));
    co_host[1] = co_sum;
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.cm, cm.data(), cm.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.cellrec, cr.data(), cr.size() * sizeof(double), cudaMemcpyHostToDevice,
                                h->stream));
    if (nBF > 0)
        CUDA_TRY(h, cudaMemcpyAsync(h->ds.brec, br.data(), br.size() * sizeof(dugks::BRec), cudaMemcpyHostToDevice,
                                    h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.fm, fm.data(), fm.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.co, co_host, sizeof co_host, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemsetAsync(h->ds.err, 0, 4 * sizeof(int), h->stream));
    if (h->dm.gref) {
        // FP32 storage reference: the Maxwellian of the volume-mean density
        // and the mass-weighted mean velocity and temperature of these macros
        double vs = 0, ms = 0, mu[3] = {0, 0, 0}, mt = 0;
        for (int o = 0; o < nC; ++o) {
            const double Vm = h->V[o], mm = Vm * rho[o];
            vs += Vm;
            ms += mm;
            for (int k = 0; k < 3; ++k) mu[k] += mm * U[3 * o + k];
            mt += mm * T[o];
        }
        const double rb = ms / vs, Tb = mt / ms, RT = R * Tb;
        const double Ub[3] = {mu[0] / ms, mu[1] / ms, mu[2] / ms};
        const int nl = h->dm.nv_loc;
        h->gref.assign(nl, 0.0);
        h->href.assign(nl, 0.0);
        for (int d = 0; d < nl; ++d) {
            const double* xi = &h->xi[3 * static_cast<size_t>(h->dm.dv_base + d)];
            const double c2 = (xi[0] - Ub[0]) * (xi[0] - Ub[0]) + (xi[1] - Ub[1]) * (xi[1] - Ub[1]) +
                              (xi[2] - Ub[2]) * (xi[2] - Ub[2]);
            h->gref[d] = rb * inv_norm_host(RT, D) * std::exp(-0.5 * c2 / RT);
            h->href[d] = K3D * RT * h->gref[d];
        }
        CUDA_TRY(h, cudaMemcpyAsync(const_cast<double*>(h->dm.gref), h->gref.data(), nl * sizeof(double),
                                    cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(const_cast<double*>(h->dm.href), h->href.data(), nl * sizeof(double),
                                    cudaMemcpyHostToDevice, h->stream));
        // raw moments of the reference over each DV chunk (moment record layout)
        std::vector<double> rm(static_cast<size_t>(h->chunks) * dugks::kNM, 0.0);
        for (int ch = 0; ch < h->chunks; ++ch) {
            double* m = &rm[static_cast<size_t>(ch) * dugks::kNM];
            for (int r = h->chunk_begin[ch]; r < h->chunk_begin[ch + 1]; ++r)
                for (int ix = 0; ix < h->n1d; ++ix) {
                    const int d = (r - h->dm.row_base) * h->n1d + ix;
                    const double* xi = &h->xi[3 * static_cast<size_t>(h->dm.dv_base + d)];
                    const double wd = h->w[h->dm.dv_base + d];
                    const double a = wd * h->gref[d], u = a * (xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]) +
                                                          wd * h->href[d];
                    m[dugks::MOM_M0] += a;
                    m[dugks::MOM_W] += u;
                    for (int k = 0; k < 3; ++k) {
                        m[dugks::MOM_M1 + k] += a * xi[k];
                        m[dugks::MOM_V3 + k] += u * xi[k];
                    }
                    m[dugks::MOM_M2] += a * xi[0] * xi[0];
                    m[dugks::MOM_M2 + 1] += a * xi[0] * xi[1];
                    m[dugks::MOM_M2 + 2] += a * xi[0] * xi[2];
                    m[dugks::MOM_M2 + 3] += a * xi[1] * xi[1];
                    m[dugks::MOM_M2 + 4] += a * xi[1] * xi[2];
                    m[dugks::MOM_M2 + 5] += a * xi[2] * xi[2];
                }
        }
        CUDA_TRY(h, cudaMemcpyAsync(h->ds.refmom, rm.data(), rm.size() * sizeof(double), cudaMemcpyHostToDevice,
                                    h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    h->ds.cur = 0;
    dugks::StepArgs a = make_args(h, 0.0, 0.0);
    CUDA_TRY(h, dugks::launch_init(a, h->precision, h->stream));
    h->launches += h->nBF > 0 ? 3 : 2;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->initialised = true;
    h->h_zero = h->D == 3 && h->gas.K_inner == 0;
    h->last_step_ms = 0;
    return DUGKS_OK;
}

// the adaptive time step between the face combine and pass B
struct AdaptCall {
    const double* dt_in;
    double* dt_out;
    double* hist;
    double max_co, max_dt;
};

// The cell partials of a sharded handle summed over its DV chunks, ready for
// the reduction over the shards: partC's first chunk, or (DV-list macroFlux)
// redC, which gathers the cell moments and the flux-term moments so that one
// reduction covers both.  *one is pointed at what the cell combine reads.
static int gather_cell_partials(dugks_handle* h, dugks::StepArgs* one, double** buf, size_t* n, int* launches) {
    const size_t nm = static_cast<size_t>(h->nC) * dugks::kNM;
    CUDA_TRY(h, dugks::launch_sum_chunks(h->ds.partC, h->chunks, nm, h->stream));
    if (h->chunks > 1) ++*launches;
    if (!h->ds.redC) {
        *buf = h->ds.partC;
        *n = nm;
        return DUGKS_OK;
    }
    const size_t nx = static_cast<size_t>(h->nC) * dugks::kFX;
    CUDA_TRY(h, dugks::launch_sum_chunks(h->ds.partX, h->chunks, nx, h->stream));
    if (h->chunks > 1) ++*launches;
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.redC, h->ds.partC, nm * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.redC + nm, h->ds.partX, nx * sizeof(double), cudaMemcpyDeviceToDevice,
                                h->stream));
    one->ds.partC = h->ds.redC;
    one->ds.partX = h->ds.redC + nm;
    *buf = h->ds.redC;
    *n = nm + nx;
    return DUGKS_OK;
}

// One step's stages on the handle's stream.  A sharded handle sums its DV
// chunks and all-reduces the raw moments before each combine, which then
// read one chunk.  sev (5 events, or null) are recorded before pass A and
// after each stage; adapt (or null) runs after the face combine.
static int enqueue_step(dugks_handle* h, const dugks::StepArgs& a, cudaEvent_t* sev, int* launches,
                        const AdaptCall* adapt) {
    const bool sh = sharded(h);
    dugks::StepArgs one = a;
    if (sh) one.chunks = 1;
    if (sev) CUDA_TRY(h, cudaEventRecord(sev[0], h->stream));
    CUDA_TRY(h, dugks::launch_stage(a, h->precision, dugks::STAGE_PASS_A, h->stream, launches));
    if (sev) CUDA_TRY(h, cudaEventRecord(sev[1], h->stream));
    if (sh) {
        const size_t n = static_cast<size_t>(h->dm.n_items) * dugks::kNM;
        CUDA_TRY(h, dugks::launch_sum_chunks(h->ds.partF, h->chunks, n, h->stream));
        if (h->chunks > 1) ++*launches;
        const int st = shard_allreduce(h, h->ds.partF, n);
        if (st) return st;
    }
    CUDA_TRY(h, dugks::launch_stage(one, h->precision, dugks::STAGE_FACE_COMBINE, h->stream, launches));
    if (adapt) {
        CUDA_TRY(h, dugks::launch_adapt(a, adapt->dt_in, adapt->dt_out, adapt->hist, adapt->max_co, adapt->max_dt,
                                        h->stream));
        ++*launches;
    }
    if (sev) CUDA_TRY(h, cudaEventRecord(sev[2], h->stream));
    CUDA_TRY(h, dugks::launch_stage(a, h->precision, dugks::STAGE_PASS_B, h->stream, launches));
    if (sev) CUDA_TRY(h, cudaEventRecord(sev[3], h->stream));
    if (sh) {
        double* buf = nullptr;
        size_t n = 0;
        int st = gather_cell_partials(h, &one, &buf, &n, launches);
        if (st || (st = shard_allreduce(h, buf, n))) return st;
    }
    CUDA_TRY(h, dugks::launch_stage(one, h->precision, dugks::STAGE_CELL_COMBINE, h->stream, launches));
    if (sev) CUDA_TRY(h, cudaEventRecord(sev[4], h->stream));
    return DUGKS_OK;
}

static int require_internal_reduction(dugks_handle* h, const char* what) {
    if (sharded(h) && !h->shard_nccl)
        return set_error(h, DUGKS_ERR_STATE,
                         std::string(what) + ": a handle sharded without NCCL steps through dugks_shard_phase");
    return DUGKS_OK;
}

static int run_steps(dugks_handle* h, int32_t n_steps, const double* dt, double* stage_ms) {
    if (!h) return DUGKS_ERR_ARG;
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_step before dugks_set_macros");
    if (int st = require_internal_reduction(h, "dugks_step")) return st;
    if (n_steps < 0 || (n_steps > 0 && !dt)) return set_error(h, DUGKS_ERR_ARG, "dugks_step: bad arguments");
    for (int i = 0; i < n_steps; ++i)
        if (!(dt[i] > 0) || !std::isfinite(dt[i])) return set_error(h, DUGKS_ERR_ARG, "dugks_step: dt must be > 0");
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaEvent_t sev[5] = {};
    if (stage_ms) {
        for (int k = 0; k < 5; ++k) {
            CUDA_TRY(h, cudaEventCreate(&sev[k]));
            stage_ms[k] = 0.0;
        }
    }
    CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
    int launches = 0;
    for (int i = 0; i < n_steps; ++i) {
        dugks::StepArgs a = make_args(h, dt[i], i + 1 < n_steps ? dt[i + 1] : 0.0);
        if (h->cellrec_dt != dt[i]) {
            CUDA_TRY(h, dugks::launch_cell_prep(a, h->stream));
            ++launches;
        }
        CUDA_TRY(h, cudaMemsetAsync(h->ds.co, 0, 2 * sizeof(double), h->stream));
        if (const int st = enqueue_step(h, a, stage_ms ? sev : nullptr, &launches, nullptr)) return st;
        if (stage_ms) {
            CUDA_TRY(h, cudaEventSynchronize(sev[4]));
            for (int stg = 0; stg < 4; ++stg) {
                float ms = 0;
                cudaEventElapsedTime(&ms, sev[stg], sev[stg + 1]);
                stage_ms[stg] += ms;
            }
        }
        h->cellrec_dt = a.dt_next;
        h->ds.cur = 1 - h->ds.cur;
        h->steps_done++;
    }
    CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
    h->launches += launches;
    int st = check_device_errors(h);
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_step_ms = ms;
    if (stage_ms) {
        stage_ms[4] = ms;
        for (int k = 0; k < 5; ++k) cudaEventDestroy(sev[k]);
    }
    return st;
}

int dugks_step(dugks_handle* h, int32_t n_steps, const double* dt) { return run_steps(h, n_steps, dt, nullptr); }

int dugks_step_timed(dugks_handle* h, int32_t n_steps, const double* dt, double* stage_ms) {
    if (!stage_ms) return set_error(h, DUGKS_ERR_ARG, "dugks_step_timed: null stage_ms");
    return run_steps(h, n_steps, dt, stage_ms);
}

int dugks_step_adaptive(dugks_handle* h, int32_t n_steps, const dugks_adapt* adapt, double* dt, double* dt_history) {
    if (!h) return DUGKS_ERR_ARG;
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_step_adaptive before dugks_set_macros");
    if (int st = require_internal_reduction(h, "dugks_step_adaptive")) return st;
    if (n_steps < 0 || !adapt || !dt || !(*dt > 0) || !std::isfinite(*dt) || !(adapt->max_co > 0) ||
        !(adapt->max_delta_t > 0))
        return set_error(h, DUGKS_ERR_ARG, "dugks_step_adaptive: bad arguments");
    if (n_steps == 0) return DUGKS_OK;
    CUDA_TRY(h, cudaSetDevice(h->device));
    if (n_steps > h->hist_cap) {
        int st = dev_alloc(h, &h->d_hist, static_cast<size_t>(n_steps));
        if (st) return st;
        h->hist_cap = n_steps;
    }
    CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->d_dt, dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    // step k (1-based) runs with slot k & 1 and writes the next dt to the other
    // slot after its face combine; step 1's dt comes from the current faces
    auto slot = [&](int k) { return h->d_dt + (k & 1); };
    int launches = 0;
    dugks::StepArgs a = make_args(h, 0.0, 0.0);
    CUDA_TRY(h, dugks::launch_adapt(a, h->d_dt, slot(1), h->d_hist, adapt->max_co, adapt->max_delta_t, h->stream));
    a.dtp = slot(1);
    CUDA_TRY(h, dugks::launch_cell_prep(a, h->stream));
    launches += 2;
    for (int k = 1; k <= n_steps; ++k) {
        a = make_args(h, 0.0, 0.0);
        a.dtp = slot(k);
        a.dtnp = slot(k + 1);
        CUDA_TRY(h, cudaMemsetAsync(h->ds.co, 0, 2 * sizeof(double), h->stream));
        const AdaptCall ac{slot(k), slot(k + 1), k < n_steps ? h->d_hist + k : nullptr, adapt->max_co,
                           adapt->max_delta_t};
        if (const int st = enqueue_step(h, a, nullptr, &launches, &ac)) return st;
        h->ds.cur = 1 - h->ds.cur;
        h->steps_done++;
    }
    CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(dt, slot(n_steps), sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (dt_history)
        CUDA_TRY(h, cudaMemcpyAsync(dt_history, h->d_hist, static_cast<size_t>(n_steps) * sizeof(double),
                                    cudaMemcpyDeviceToHost, h->stream));
    h->launches += launches;
    h->cellrec_dt = 0.0;   // the records hold the next adaptive dt; a fixed step rebuilds them
    int st = check_device_errors(h);
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_step_ms = ms;
    return st;
}

int dugks_shard_phase(dugks_handle* h, int32_t phase, double dt, double** part, int64_t* n_part) {
    if (!h) return DUGKS_ERR_ARG;
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_shard_phase before dugks_set_macros");
    if (h->shard_nccl) return set_error(h, DUGKS_ERR_STATE, "dugks_shard_phase: the handle reduces with NCCL");
    if (phase != h->shard_phase_next)
        return set_error(h, DUGKS_ERR_STATE, "dugks_shard_phase: expected phase " + std::to_string(h->shard_phase_next));
    if (phase < 2 && (!part || !n_part)) return set_error(h, DUGKS_ERR_ARG, "dugks_shard_phase: null output");
    CUDA_TRY(h, cudaSetDevice(h->device));
    int launches = 0;
    if (phase == 0) {
        if (!(dt > 0) || !std::isfinite(dt)) return set_error(h, DUGKS_ERR_ARG, "dugks_shard_phase: dt must be > 0");
        h->shard_dt = dt;
        const dugks::StepArgs a = make_args(h, dt, 0.0);
        if (h->cellrec_dt != dt) {
            CUDA_TRY(h, dugks::launch_cell_prep(a, h->stream));
            ++launches;
        }
        CUDA_TRY(h, cudaMemsetAsync(h->ds.co, 0, 2 * sizeof(double), h->stream));
        CUDA_TRY(h, dugks::launch_stage(a, h->precision, dugks::STAGE_PASS_A, h->stream, &launches));
        const size_t n = static_cast<size_t>(h->dm.n_items) * dugks::kNM;
        CUDA_TRY(h, dugks::launch_sum_chunks(h->ds.partF, h->chunks, n, h->stream));
        if (h->chunks > 1) ++launches;
        *part = h->ds.partF;
        *n_part = static_cast<int64_t>(n);
    } else if (phase == 1) {
        const dugks::StepArgs a = make_args(h, h->shard_dt, 0.0);
        dugks::StepArgs one = a;
        one.chunks = 1;
        CUDA_TRY(h, dugks::launch_stage(one, h->precision, dugks::STAGE_FACE_COMBINE, h->stream, &launches));
        CUDA_TRY(h, dugks::launch_stage(a, h->precision, dugks::STAGE_PASS_B, h->stream, &launches));
        double* buf = nullptr;
        size_t n = 0;
        if (int st = gather_cell_partials(h, &one, &buf, &n, &launches)) return st;
        *part = buf;
        *n_part = static_cast<int64_t>(n);
    } else {
        dugks::StepArgs one = make_args(h, h->shard_dt, 0.0);
        one.chunks = 1;
        if (h->ds.redC) {
            one.ds.partC = h->ds.redC;
            one.ds.partX = h->ds.redC + static_cast<size_t>(h->nC) * dugks::kNM;
        }
        CUDA_TRY(h, dugks::launch_stage(one, h->precision, dugks::STAGE_CELL_COMBINE, h->stream, &launches));
        h->cellrec_dt = 0.0;   // the next phase 0 sets the relax factors for its dt
        h->ds.cur = 1 - h->ds.cur;
        h->steps_done++;
    }
    h->launches += launches;
    h->shard_phase_next = (phase + 1) % 3;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return phase == 2 ? check_device_errors(h) : DUGKS_OK;
}

}  // extern "C"

struct dugks_batch {
    std::vector<dugks_handle*> hs;
    std::vector<double> dt;
    std::vector<cudaEvent_t> joins;
    int device = 0;
    cudaStream_t s0 = nullptr;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int> launches_per_pair;   // per handle
    std::vector<char> hzero;              // per handle, as captured
    int64_t graph_kernels = 0;
    double last_ms = 0;
    std::string last_error;
};

namespace {

int batch_fail(dugks_batch* b, int code, const std::string& msg) {
    b->last_error = msg;
    return code;
}

void batch_free(dugks_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->s0) cudaStreamSynchronize(b->s0);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->joins) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->s0) cudaStreamDestroy(b->s0);
    delete b;
}

}  // namespace

extern "C" {

int dugks_batch_create(dugks_handle* const* handles, int32_t n, const double* dt, dugks_batch** out) {
    if (!out) return DUGKS_ERR_ARG;
    *out = nullptr;
    if (!handles || !dt || n < 1) return DUGKS_ERR_ARG;
    for (int i = 0; i < n; ++i) {
        dugks_handle* h = handles[i];
        if (!h || !h->initialised || sharded(h) || h->device != handles[0]->device || !(dt[i] > 0) ||
            !std::isfinite(dt[i]))
            return DUGKS_ERR_ARG;
        for (int j = 0; j < i; ++j)
            if (handles[j] == h) return DUGKS_ERR_ARG;
    }
    dugks_batch* b = new (std::nothrow) dugks_batch();
    if (!b) return DUGKS_ERR_OOM;
    b->hs.assign(handles, handles + n);
    b->dt.assign(dt, dt + n);
    b->device = handles[0]->device;
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        b->last_error = std::string(what) + ": " + cudaGetErrorString(e);
        *out = b;
        return DUGKS_ERR_CUDA;
    };
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&b->s0, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess)
        return cuda_fail(e, "stream or event creation");
    b->joins.assign(n, nullptr);
    for (int i = 0; i < n; ++i)
        if ((e = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "cudaEventCreate");
    // every handle's cell records carry the relax factors of its dt, as the
    // graph's cell combines write them for the next step
    for (int i = 0; i < n; ++i) {
        dugks_handle* h = b->hs[i];
        if (h->cellrec_dt != b->dt[i]) {
            if ((e = dugks::launch_cell_prep(make_args(h, b->dt[i], 0.0), h->stream)) != cudaSuccess)
                return cuda_fail(e, "cell prep");
            h->cellrec_dt = b->dt[i];
        }
        if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    }
    // capture: fork from s0 into every handle's stream, two steps each, join
    if ((e = cudaStreamBeginCapture(b->s0, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamBeginCapture");
    int st = DUGKS_OK;
    cudaEventRecord(b->fork, b->s0);
    b->launches_per_pair.assign(n, 0);
    for (int i = 0; i < n && st == DUGKS_OK; ++i) {
        dugks_handle* h = b->hs[i];
        cudaStreamWaitEvent(h->stream, b->fork, 0);
        const int cur0 = h->ds.cur;
        b->hzero.push_back(h->h_zero ? 1 : 0);
        for (int k = 0; k < 2 && st == DUGKS_OK; ++k) {
            const dugks::StepArgs a = make_args(h, b->dt[i], b->dt[i]);
            if (cudaMemsetAsync(h->ds.co, 0, 2 * sizeof(double), h->stream) != cudaSuccess) st = DUGKS_ERR_CUDA;
            else st = enqueue_step(h, a, nullptr, &b->launches_per_pair[i], nullptr);
            h->ds.cur = 1 - h->ds.cur;
        }
        h->ds.cur = cur0;
        cudaEventRecord(b->joins[i], h->stream);
        cudaStreamWaitEvent(b->s0, b->joins[i], 0);
    }
    e = cudaStreamEndCapture(b->s0, &b->graph);
    if (st != DUGKS_OK) {
        *out = b;
        return batch_fail(b, st, "capturing a step failed");
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    for (int c : b->launches_per_pair) b->graph_kernels += c;
    *out = b;
    return DUGKS_OK;
}

int dugks_batch_step(dugks_batch* b, int32_t n_steps) {
    if (!b) return DUGKS_ERR_ARG;
    if (n_steps < 0 || !b->exec) return batch_fail(b, DUGKS_ERR_ARG, "dugks_batch_step: bad arguments");
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) return batch_fail(b, DUGKS_ERR_CUDA, cudaGetErrorString(e));
    const int pairs = n_steps / 2;
    for (size_t i = 0; i < b->hs.size(); ++i)
        if ((b->hs[i]->h_zero ? 1 : 0) != b->hzero[i])
            return batch_fail(b, DUGKS_ERR_STATE, "dugks_batch_step: a handle's state was replaced since the batch was built");
    // handles' own queued work comes first
    for (dugks_handle* h : b->hs) {
        if ((e = cudaEventRecord(h->ev0, h->stream)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(b->s0, h->ev0, 0)) != cudaSuccess)
            return batch_fail(b, DUGKS_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaEventRecord(b->ev0, b->s0);
    for (int p = 0; p < pairs; ++p)
        if ((e = cudaGraphLaunch(b->exec, b->s0)) != cudaSuccess)
            return batch_fail(b, DUGKS_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    cudaEventRecord(b->ev1, b->s0);
    if ((e = cudaStreamSynchronize(b->s0)) != cudaSuccess)
        return batch_fail(b, DUGKS_ERR_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    for (size_t i = 0; i < b->hs.size(); ++i) {
        dugks_handle* h = b->hs[i];
        h->steps_done += 2 * pairs;
        h->launches += static_cast<int64_t>(b->launches_per_pair[i]) * pairs;
        if (n_steps % 2) {
            // the odd step on the handle's own stream, then the relax factors
            // of its dt again for the next replay
            int st = run_steps(h, 1, &b->dt[i], nullptr);
            if (st == DUGKS_OK && (e = dugks::launch_cell_prep(make_args(h, b->dt[i], 0.0), h->stream)) != cudaSuccess)
                st = set_error(h, DUGKS_ERR_CUDA, cudaGetErrorString(e));
            if (st != DUGKS_OK) return batch_fail(b, st, "handle " + std::to_string(i) + ": " + h->last_error);
            h->cellrec_dt = b->dt[i];
        }
        const int st = check_device_errors(h);
        if (st != DUGKS_OK) return batch_fail(b, st, "handle " + std::to_string(i) + ": " + h->last_error);
    }
    return DUGKS_OK;
}

int dugks_batch_last_ms(const dugks_batch* b, double* ms) {
    if (!b || !ms) return DUGKS_ERR_ARG;
    *ms = b->last_ms;
    return DUGKS_OK;
}

int64_t dugks_batch_graph_kernels(const dugks_batch* b) { return b ? b->graph_kernels : 0; }

const char* dugks_batch_last_error(const dugks_batch* b) { return b ? b->last_error.c_str() : "null batch"; }

void dugks_batch_destroy(dugks_batch* b) { batch_free(b); }

int64_t dugks_kernel_launches(const dugks_handle* h) { return h ? h->launches : 0; }

int dugks_co_num(dugks_handle* h, double dt, double* co_max, double* co_mean) {
    if (!h || !co_max || !co_mean) return set_error(h, DUGKS_ERR_ARG, "dugks_co_num: null output");
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_co_num before dugks_set_macros");
    double co[2];
    CUDA_TRY(h, cudaMemcpyAsync(co, h->ds.co, sizeof co, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    double mx;
    std::memcpy(&mx, &co[0], sizeof mx);
    *co_max = mx * dt;
    *co_mean = h->nIF > 0 ? co[1] / h->nIF * dt : 0.0;
    return DUGKS_OK;
}

int64_t dugks_step_record_size(const dugks_handle* h) {
    return h ? 9 * static_cast<int64_t>(h->nC) + 2 + 2 * static_cast<int64_t>(h->nBF) : 0;
}

int dugks_get_step_record(dugks_handle* h, double* rec) {
    if (!h || !rec) return set_error(h, DUGKS_ERR_ARG, "dugks_get_step_record: null argument");
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_get_step_record before dugks_set_macros");
    const int nC = h->nC;
    std::vector<double> cm(static_cast<size_t>(nC) * 9);
    CUDA_TRY(h, cudaMemcpyAsync(cm.data(), h->ds.cm, cm.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(rec + cm.size(), h->ds.co, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    std::vector<dugks::BRec> br(h->nBF);
    if (h->nBF > 0)
        CUDA_TRY(h, cudaMemcpyAsync(br.data(), h->ds.brec, br.size() * sizeof(dugks::BRec), cudaMemcpyDeviceToHost,
                                    h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const std::vector<int32_t>& perm = h->tiling.perm;
    for (int c = 0; c < nC; ++c) std::memcpy(rec + 9 * static_cast<size_t>(perm[c]), &cm[9 * static_cast<size_t>(c)],
                                             9 * sizeof(double));
    double* rb = rec + cm.size() + 2;
    for (int b = 0; b < h->nBF; ++b) {
        rb[2 * b] = br[b].rho_in;
        rb[2 * b + 1] = br[b].T;
    }
    return DUGKS_OK;
}

int dugks_set_step_record(dugks_handle* h, const double* rec) {
    if (!h || !rec) return set_error(h, DUGKS_ERR_ARG, "dugks_set_step_record: null argument");
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_set_step_record before dugks_set_macros");
    const int nC = h->nC;
    std::vector<double> cm(static_cast<size_t>(nC) * 9);
    const std::vector<int32_t>& perm = h->tiling.perm;
    for (int c = 0; c < nC; ++c) {
        const double* r = rec + 9 * static_cast<size_t>(perm[c]);
        bool ok = r[0] > 0 && r[4] > 0 && r[8] > 0;
        for (int j = 0; j < 9; ++j) ok = ok && std::isfinite(r[j]);
        if (!ok) return set_error(h, DUGKS_ERR_ARG, "dugks_set_step_record: bad record of cell " + std::to_string(perm[c]));
        std::memcpy(&cm[9 * static_cast<size_t>(c)], r, 9 * sizeof(double));
    }
    const double* co = rec + cm.size();
    double co_max;
    std::memcpy(&co_max, &co[0], sizeof co_max);
    if (!(co_max >= 0) || !std::isfinite(co_max) || !(co[1] >= 0) || !std::isfinite(co[1]))
        return set_error(h, DUGKS_ERR_ARG, "dugks_set_step_record: bad Courant sums");
    // boundary rho and T: the pressure patches carry them from step to step
    std::vector<dugks::BRec> br(h->nBF);
    if (h->nBF > 0)
        CUDA_TRY(h, cudaMemcpy(br.data(), h->ds.brec, br.size() * sizeof(dugks::BRec), cudaMemcpyDeviceToHost));
    const double* rb = co + 2;
    const double K3D = h->gas.K_inner + 3.0 - h->D;
    for (int b = 0; b < h->nBF; ++b) {
        // rho_b of every face (walls: the last step's rho_w, an output);
        // T_b and its factors on the pressure faces, the only ones it changes on
        br[b].rho_in = rb[2 * b];
        const int pt = h->bface_ptype[b];
        if (pt != DUGKS_PATCH_PRESSURE_IN && pt != DUGKS_PATCH_PRESSURE_OUT) continue;
        const double rho_b = rb[2 * b], T_b = rb[2 * b + 1];
        if (!(rho_b > 0) || !(T_b > 0) || !std::isfinite(rho_b + T_b))
            return set_error(h, DUGKS_ERR_ARG, "dugks_set_step_record: bad boundary record");
        const double RT = h->gas.R * T_b;
        br[b].T = T_b;
        br[b].K_in = inv_norm_host(RT, h->D);
        br[b].invRT_in = 1.0 / RT;
        br[b].hfac = RT * K3D;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (h->nBF > 0)
        CUDA_TRY(h, cudaMemcpyAsync(h->ds.brec, br.data(), br.size() * sizeof(dugks::BRec), cudaMemcpyHostToDevice,
                                    h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.cm, cm.data(), cm.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->ds.co, co, 2 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, dugks::launch_cell_records(make_args(h, 0.0, 0.0), h->stream));
    h->launches += 1;
    h->cellrec_dt = 0;   // the next step sets the relax factors for its dt
    return check_device_errors(h);
}

int dugks_get_macros(dugks_handle* h, double* rho, double* U, double* T, double* q) {
    if (!h) return DUGKS_ERR_ARG;
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_get_macros before dugks_set_macros");
    const int nC = h->nC;
    const size_t bytes = static_cast<size_t>(nC) * 9 * sizeof(double);
    // a pinned staging buffer, kept by the handle: the copy runs at the
    // link's speed instead of through a pageable bounce buffer every step
    if (!h->host_cm) CUDA_TRY(h, cudaMallocHost(reinterpret_cast<void**>(&h->host_cm), bytes));
    CUDA_TRY(h, cudaMemcpyAsync(h->host_cm, h->ds.cm, bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const double* cm = h->host_cm;
    const std::vector<int32_t>& perm = h->tiling.perm;
    for (int c = 0; c < nC; ++c) {
        const int o = perm[c];
        const double* m = &cm[9 * static_cast<size_t>(c)];
        if (rho) rho[o] = m[0];
        if (U)
            for (int k = 0; k < 3; ++k) U[3 * o + k] = m[1 + k];
        if (T) T[o] = m[4];
        if (q)
            for (int k = 0; k < 3; ++k) q[3 * o + k] = m[5 + k];
    }
    return DUGKS_OK;
}

int dugks_get_face_macros(dugks_handle* h, double* rho, double* U, double* T, double* q) {
    if (!h) return DUGKS_ERR_ARG;
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_get_face_macros before dugks_set_macros");
    const int nF = h->nIF + h->nBF;
    std::vector<double> fm(static_cast<size_t>(nF) * 9);
    CUDA_TRY(h, cudaMemcpyAsync(fm.data(), h->ds.fm, fm.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int f = 0; f < nF; ++f) {
        const double* m = &fm[9 * static_cast<size_t>(f)];
        if (rho) rho[f] = m[0];
        if (U)
            for (int k = 0; k < 3; ++k) U[3 * f + k] = m[1 + k];
        if (T) T[f] = m[4];
        if (q)
            for (int k = 0; k < 3; ++k) q[3 * f + k] = m[5 + k];
    }
    return DUGKS_OK;
}

int dugks_get_boundary_rho(dugks_handle* h, double* rho_b) {
    if (!h || !rho_b) return set_error(h, DUGKS_ERR_ARG, "dugks_get_boundary_rho: null output");
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_get_boundary_rho before dugks_set_macros");
    std::vector<dugks::BRec> br(h->nBF);
    if (h->nBF > 0) {
        CUDA_TRY(h, cudaMemcpyAsync(br.data(), h->ds.brec, br.size() * sizeof(dugks::BRec), cudaMemcpyDeviceToHost,
                                    h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    for (int b = 0; b < h->nBF; ++b) rho_b[b] = br[b].rho_in;
    return DUGKS_OK;
}

int dugks_get_df(dugks_handle* h, const int32_t* cells, int32_t n, double* g_out, double* h_out) {
    if (!h || (n > 0 && (!cells || !g_out))) return set_error(h, DUGKS_ERR_ARG, "dugks_get_df: bad arguments");
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "dugks_get_df before dugks_set_macros");
    const size_t rs = real_size(h);
    std::vector<unsigned char> col(static_cast<size_t>(h->dm.nv_loc) * rs);
    for (int i = 0; i < n; ++i) {
        if (cells[i] < 0 || cells[i] >= h->nC) return set_error(h, DUGKS_ERR_ARG, "dugks_get_df: cell out of range");
        const int c = h->tiling.iperm[cells[i]];
        for (int which = 0; which < 2; ++which) {
            double* dst = which == 0 ? g_out : h_out;
            if (!dst) continue;
            const unsigned char* src =
                static_cast<const unsigned char*>(which == 0 ? h->ds.g[h->ds.cur] : h->ds.h[h->ds.cur]) + c * rs;
            CUDA_TRY(h, cudaMemcpy2DAsync(col.data(), rs, src, static_cast<size_t>(h->nC) * rs, rs, h->dm.nv_loc,
                                          cudaMemcpyDeviceToHost, h->stream));
            CUDA_TRY(h, cudaStreamSynchronize(h->stream));
            for (int d = 0; d < h->dm.nv_loc; ++d) {
                double v;
                if (rs == sizeof(double)) std::memcpy(&v, &col[d * rs], sizeof v);
                else {
                    float fv;
                    std::memcpy(&fv, &col[d * rs], sizeof fv);
                    const std::vector<double>& ref = which == 0 ? h->gref : h->href;
                    v = ref.empty() ? fv : fv + ref[d];
                }
                dst[static_cast<size_t>(i) * h->dm.nv_loc + d] = v;
            }
        }
    }
    return DUGKS_OK;
}

static int state_io(dugks_handle* h, double* g, double* hh, const double* gi, const double* hi, bool get) {
    if (!h) return DUGKS_ERR_ARG;
    if (!h->initialised) return set_error(h, DUGKS_ERR_STATE, "state access before dugks_set_macros");
    const size_t rs = real_size(h);
    const size_t nvc = static_cast<size_t>(h->dm.nv_loc) * h->nC;
    std::vector<unsigned char> buf(nvc * rs);
    const std::vector<int32_t>& perm = h->tiling.perm;
    for (int which = 0; which < 2; ++which) {
        void* dev = which == 0 ? h->ds.g[h->ds.cur] : h->ds.h[h->ds.cur];
        const std::vector<double>& ref = which == 0 ? h->gref : h->href;
        if (get) {
            double* dst = which == 0 ? g : hh;
            if (!dst) continue;
            CUDA_TRY(h, cudaMemcpy(buf.data(), dev, nvc * rs, cudaMemcpyDeviceToHost));
            for (int d = 0; d < h->dm.nv_loc; ++d)
                for (int c = 0; c < h->nC; ++c) {
                    const size_t s = static_cast<size_t>(d) * h->nC + c;
                    const size_t o = static_cast<size_t>(d) * h->nC + perm[c];
                    if (rs == sizeof(double)) std::memcpy(&dst[o], &buf[s * rs], sizeof(double));
                    else {
                        float fv;
                        std::memcpy(&fv, &buf[s * rs], sizeof fv);
                        dst[o] = ref.empty() ? fv : fv + ref[d];
                    }
                }
        } else {
            const double* src = which == 0 ? gi : hi;
            if (!src) return set_error(h, DUGKS_ERR_ARG, "dugks_set_state: null array");
            for (int d = 0; d < h->dm.nv_loc; ++d)
                for (int c = 0; c < h->nC; ++c) {
                    const size_t s = static_cast<size_t>(d) * h->nC + c;
                    const size_t o = static_cast<size_t>(d) * h->nC + perm[c];
                    if (rs == sizeof(double)) std::memcpy(&buf[s * rs], &src[o], sizeof(double));
                    else {
                        const float fv = static_cast<float>(ref.empty() ? src[o] : src[o] - ref[d]);
                        std::memcpy(&buf[s * rs], &fv, sizeof fv);
                    }
                }
            CUDA_TRY(h, cudaMemcpy(dev, buf.data(), nvc * rs, cudaMemcpyHostToDevice));
        }
    }
    return DUGKS_OK;
}

int dugks_get_state(dugks_handle* h, double* g, double* hh) { return state_io(h, g, hh, nullptr, nullptr, true); }

int dugks_set_state(dugks_handle* h, const double* g, const double* hh, double dt_prev) {
    if (!h) return DUGKS_ERR_ARG;
    if (int st = require_internal_reduction(h, "dugks_set_state")) return st;
    int st = state_io(h, nullptr, nullptr, g, hh, false);
    if (st) return st;
    if (!(dt_prev > 0)) return set_error(h, DUGKS_ERR_ARG, "dugks_set_state: dt_prev must be > 0");
    // a nonzero h~ ends the g-only passes for this handle
    if (h->h_zero) {
        const size_t nvc = static_cast<size_t>(h->dm.nv_loc) * h->nC;
        for (size_t i = 0; i < nvc && h->h_zero; ++i) h->h_zero = hh[i] == 0.0;
    }
    dugks::StepArgs a = make_args(h, dt_prev, 0.0);
    a.dm.macro_flux = 0;   // the macros of given DFs are their moments (macroFlux yes: restore the step record)
    // a new state replaces a poisoned one: its own check starts clear
    CUDA_TRY(h, cudaMemsetAsync(h->ds.err, 0, 4 * sizeof(int), h->stream));
    CUDA_TRY(h, dugks::launch_state_moments(a, h->precision, h->stream));
    if ((st = shard_allreduce(h, h->ds.partC, static_cast<size_t>(h->nC) * dugks::kNM))) return st;
    CUDA_TRY(h, dugks::launch_cell_combine_one(a, 0.0, h->stream));
    h->launches += 2;
    h->cellrec_dt = 0;
    return check_device_errors(h);
}

int32_t dugks_n_dv(const dugks_handle* h) { return h ? h->nv : 0; }

int dugks_layout(const dugks_handle* h, int32_t* tile_cells, int32_t* n_tiles, int32_t* dv_chunks) {
    if (!h) return DUGKS_ERR_ARG;
    if (tile_cells) *tile_cells = h->tiling.tile_cells;
    if (n_tiles) *n_tiles = h->tiling.n_tiles;
    if (dv_chunks) *dv_chunks = h->chunks;
    return DUGKS_OK;
}

int dugks_last_step_ms(dugks_handle* h, double* ms) {
    if (!h || !ms) return DUGKS_ERR_ARG;
    *ms = h->last_step_ms;
    return DUGKS_OK;
}

const char* dugks_last_error(const dugks_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

void dugks_destroy(dugks_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->nccl_comm) nccl_api().comm_destroy(static_cast<ncclComm_t>(h->nccl_comm));
    for (void* p : h->allocations) cudaFree(p);
    if (h->host_cm) cudaFreeHost(h->host_cm);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"

namespace dugks {

// Rebuilds the cell records and Maxwellian tables from the cell macros in
// ds.cm, as dugks_set_step_record does after restoring them; the next step
// sets the relax factors for its dt.
int rebuild_cell_records(dugks_handle* h) {
    CUDA_TRY(h, launch_cell_records(make_args(h, 0.0, 0.0), h->stream));
    h->launches += 1;
    h->cellrec_dt = 0;
    return DUGKS_OK;
}

int record_face_values(dugks_handle* h, double dt) {
    const StepArgs a = make_args(h, dt, 0.0);
    int launches = 0;
    if (h->cellrec_dt != dt) {
        CUDA_TRY(h, launch_cell_prep(a, h->stream));
        ++launches;
        h->cellrec_dt = dt;   // the relax factors are now dt's
    }
    CUDA_TRY(h, launch_stage(a, h->precision, STAGE_PASS_A, h->stream, &launches));
    h->launches += launches;
    return DUGKS_OK;
}

}  // namespace dugks

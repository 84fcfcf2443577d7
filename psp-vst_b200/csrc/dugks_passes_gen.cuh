// The two tile passes for a DV set that is not a tensor product (the
// reference's unstructured velocity mesh: xi = vMesh cell centres, weights =
// vMesh cell volumes, fvDVM.C:129-277).  Included inside the anonymous
// namespace of dugks_passes.cu; tiles, items, stencils, staging and the
// stage sequence are those of the row-factored passes.  What differs: a batch
// is NB consecutive DVs of the list; each DV's velocity and weight come from
// a per-batch table; the Shakhov equilibrium is evaluated with its own
// exponential per (entity, DV); the raw moments are summed DV by DV.
// Chunks are DV ranges (the handle keeps one DV per "row").

// DV velocities and weights of a batch into shared memory (the first NB
// threads; visible after the next barrier)
template <int NB>
__device__ __forceinline__ void load_dv_batch(const DevMesh& m, double* xw, int dglob0, int nb) {
    const int j = threadIdx.x;
    if (j < NB) {
        const int d = dglob0 + (j < nb ? j : 0);
        xw[4 * j] = __ldg(m.xi + 3 * d);
        xw[4 * j + 1] = __ldg(m.xi + 3 * d + 1);
        xw[4 * j + 2] = __ldg(m.xi + 3 * d + 2);
        xw[4 * j + 3] = j < nb ? __ldg(m.w + d) : 0.0;
    }
}

// a record (structure of arrays over n entities) as a Rec
__device__ __forceinline__ Rec<double> rec_at(const double* __restrict__ rec, size_t n, int e) {
    Rec<double> r;
    r.U[0] = __ldg(rec + REC_UX * n + e);
    r.U[1] = __ldg(rec + REC_UY * n + e);
    r.U[2] = __ldg(rec + REC_UZ * n + e);
    r.invRT = __ldg(rec + REC_INVRT * n + e);
    r.A = __ldg(rec + REC_A * n + e);
    r.r = __ldg(rec + REC_R * n + e);
    r.qv[0] = __ldg(rec + REC_QX * n + e);
    r.qv[1] = __ldg(rec + REC_QY * n + e);
    r.qv[2] = __ldg(rec + REC_QZ * n + e);
    r.RTh = __ldg(rec + REC_RTH * n + e);
    return r;
}

// (1 - r) g + r gS with the record's equilibrium at xi (fvDVM.C:668-679,
// :1374-1391)
template <int D>
__device__ __forceinline__ void relax_gen(const Rec<double>& r, const double xi[3], double g, double h, double K3D,
                                          double Kin, double& go, double& ho) {
    double gS, hS;
    shakhov<D, double>(xi, r, K3D, Kin, gS, hS);
    go = (1.0 - r.r) * g + r.r * gS;
    ho = (1.0 - r.r) * h + r.r * hS;
}

template <int D, typename Real, int NB>
struct SmemAG {
    double* xw;     // [2][NB][4] DV velocity and weight, per batch parity
    Real* stg;      // [2][2][NB][kSL] staged g~, h~ of the local cells
    Real* gB;       // [NB][kSL] gbar+
    Real* hB;
    Real* Gg;       // [NB][D][kS0]
    Real* Gh;
    int* snb;       // [kMaxRegStencil][kS0]
    Real* sls;      // [kMaxRegStencil][D][kS0]
    static constexpr size_t bytes() {
        return 2 * NB * 4 * sizeof(double) + static_cast<size_t>(kMaxRegStencil) * kS0 * sizeof(int) +
               (2 * 2 * static_cast<size_t>(NB) * kSL + 2 * NB * kSL + 2 * NB * D * kS0 +
                static_cast<size_t>(kMaxRegStencil) * D * kS0) *
                   sizeof(Real);
    }
};

template <int D, typename Real, int NB>
__device__ __forceinline__ SmemAG<D, Real, NB> carve_ag(unsigned char* base) {
    SmemAG<D, Real, NB> s;
    s.xw = reinterpret_cast<double*>(base);
    Real* p = reinterpret_cast<Real*>(s.xw + 2 * NB * 4);
    s.stg = p;
    p += 2 * 2 * NB * kSL;
    s.gB = p;
    p += NB * kSL;
    s.hB = p;
    p += NB * kSL;
    s.Gg = p;
    p += NB * D * kS0;
    s.Gh = p;
    p += NB * D * kS0;
    s.sls = p;
    p += kMaxRegStencil * D * kS0;
    s.snb = reinterpret_cast<int*>(p);
    return s;
}

// recon from local L0 cell l of DV j: gbar+_l + grad_l . (Cf - C_l - xi dt/2)
template <int D, typename Real, int NB>
__device__ __forceinline__ void recon_g(const SmemAG<D, Real, NB>& sm, int j, int l, Real vx, Real vy, Real vz,
                                        Real& g, Real& h) {
    const Real* Gg = sm.Gg + j * D * kS0 + l;
    const Real* Gh = sm.Gh + j * D * kS0 + l;
    Real gg = fma(Gg[0], vx, sm.gB[j * kSL + l]);
    Real hh = fma(Gh[0], vx, sm.hB[j * kSL + l]);
    gg = fma(Gg[kS0], vy, gg);
    hh = fma(Gh[kS0], vy, hh);
    if (D == 3) {
        gg = fma(Gg[2 * kS0], vz, gg);
        hh = fma(Gh[2 * kS0], vz, hh);
    }
    g = gg;
    h = hh;
}

// the per-item moment accumulation of one DV: raw moments (accum) plus the
// wall out-flux w (xi.S) g of outgoing wall DVs
template <int D>
__device__ __forceinline__ void add_dv(double* acc, double w, const double xi[3], double g, double h) {
    const double xi2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
    accum<D>(acc, w, xi, xi2, g, h);
}

// least-squares gradients of the L0 cells for a batch of nb DVs (the
// row-factored pass's stage 2)
template <int D, typename Real, int NB>
__device__ __forceinline__ void stage2_gen(const DevMesh& m, const SmemAG<D, Real, NB>& sm, int nb,
                                           const TileRange& t, int* err) {
    const int l = threadIdx.x % kS0, part = threadIdx.x / kS0;
    if (l >= t.n0) return;
    const int c = t.b + l;
    for (int j = part; j < nb; j += kParts0) {
        const Real* gB = sm.gB + j * kSL;
        const Real* hB = sm.hB + j * kSL;
        const Real g0 = gB[l], h0 = hB[l];
        Real gx[D], hx[D];
#pragma unroll
        for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
        if (m.nb_max <= kMaxRegStencil) {
#pragma unroll
            for (int k = 0; k < kMaxRegStencil; ++k) {
                const int n = sm.snb[k * kS0 + l];
                const Real dg = gB[n] - g0, dh = hB[n] - h0;
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    const Real ls = sm.sls[(k * D + q) * kS0 + l];
                    gx[q] = fma(ls, dg, gx[q]);
                    hx[q] = fma(ls, dh, hx[q]);
                }
            }
        } else {
            for (int k = 0; k < m.nb_max; ++k) {
                const int n0 = __ldg(m.grad_nb + static_cast<size_t>(k) * m.nC + c);
                if (n0 < 0) continue;
                const int n = chk(n0, 0, t.nloc, err);
                const Real dg = gB[n] - g0, dh = hB[n] - h0;
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    const Real ls = Real(__ldg(m.grad_ls + (static_cast<size_t>(k) * 3 + q) * m.nC + c));
                    gx[q] = fma(ls, dg, gx[q]);
                    hx[q] = fma(ls, dh, hx[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < D; ++q) {
            sm.Gg[(j * D + q) * kS0 + l] = gx[q];
            sm.Gh[(j * D + q) * kS0 + l] = hx[q];
        }
    }
}

template <int D, typename Real, int NB>
__global__ void __launch_bounds__(kThreads, 1) k_pass_a_gen(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemAG<D, Real, NB> sm = carve_ag<D, Real, NB>(smem_raw);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    Real* const fvg = reinterpret_cast<Real*>(a.ds.fvg);
    Real* const fvh = reinterpret_cast<Real*>(a.ds.fvh);
    const double K3D = m.K + 3.0 - m.D, Kin = m.K;
    const double hdt = 0.5 * step_dt(a);
    const size_t nI = static_cast<size_t>(m.n_items), nC = static_cast<size_t>(m.nC);

    const int l1 = threadIdx.x % kSL, p1 = threadIdx.x / kSL;
    const bool act1 = l1 < t.nloc;
    const int c1 = act1 ? chk(__ldg(m.loc_cells + t.loff + l1), 0, m.nC, a.ds.err) : 0;
    const Rec<double> cr1 = act1 ? rec_at(a.ds.cellrec, nC, c1) : Rec<double>{};
    if (threadIdx.x < kS0 && m.nb_max <= kMaxRegStencil) {
        const int l = threadIdx.x;
        const int c = t.b + l;
#pragma unroll
        for (int k = 0; k < kMaxRegStencil; ++k) {
            const int n = (l < t.n0 && k < m.nb_max) ? __ldg(m.grad_nb + static_cast<size_t>(k) * m.nC + c) : -1;
            sm.snb[k * kS0 + l] = n >= 0 ? chk(n, 0, t.nloc, a.ds.err) : l;
#pragma unroll
            for (int q = 0; q < D; ++q)
                sm.sls[(k * D + q) * kS0 + l] =
                    n >= 0 ? Real(__ldg(m.grad_ls + (static_cast<size_t>(k) * 3 + q) * m.nC + c)) : Real(0);
        }
    }
    const int it = threadIdx.x;
    const bool has_item = it < t.nit;
    Item v{};
    if (has_item) {
        v = load_item(m, t.ioff + it);
        v.la = chk(v.la, 0, t.nloc, a.ds.err);
        if (v.kind != ITEM_MESH_BOUNDARY) v.lb = chk(v.lb, 0, t.nloc, a.ds.err);
        else v.face = chk(v.face, 0, m.nBF, a.ds.err);
        if (v.kind == ITEM_TB_OWN || v.kind == ITEM_TB_NEI) v.other = chk(v.other, 0, m.n_items, a.ds.err);
    }
    double acc[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;

    // this chunk's DVs: [r0, r1) of the list (one DV per row)
    const int d_first = t.r0 - m.row_base, d_end = t.r1 - m.row_base;
    const int nbt = (d_end - d_first + NB - 1) / NB;
    auto stage_batch = [&](int k, int buf) {
        const int d0 = d_first + k * NB, nb = min(NB, d_end - d0);
        load_dv_batch<NB>(m, sm.xw + buf * NB * 4, m.dv_base + d0, nb);
        if (act1) {
            constexpr int H = NB / kPartsL;
            Real* sg = sm.stg + static_cast<size_t>(buf) * 2 * NB * kSL;
#pragma unroll
            for (int jj = 0; jj < H; ++jj) {
                const int j = p1 * H + jj;
                if (j < nb) {
                    cp_async(sg + j * kSL + l1, g + static_cast<size_t>(d0 + j) * nC + c1);
                    cp_async(sg + (NB + j) * kSL + l1, h + static_cast<size_t>(d0 + j) * nC + c1);
                }
            }
        }
        cp_commit();
    };
    if (nbt > 0) stage_batch(0, 0);
    for (int k = 0; k < nbt; ++k) {
        const int buf = k & 1;
        const int nb = min(NB, d_end - (d_first + k * NB));
        const int d0 = d_first + k * NB;
        cp_wait_all();
        __syncthreads();  // batch k staged; the previous batch's stage 3 is done
        if (k + 1 < nbt) stage_batch(k + 1, buf ^ 1);
        const double* xw = sm.xw + buf * NB * 4;
        // stage 1: gbar+ of the local cells
        if (act1) {
            constexpr int H = NB / kPartsL;
            const Real* sg = sm.stg + static_cast<size_t>(buf) * 2 * NB * kSL;
#pragma unroll
            for (int jj = 0; jj < H; ++jj) {
                const int j = p1 * H + jj;
                if (j < nb) {
                    const double xi[3] = {xw[4 * j], xw[4 * j + 1], xw[4 * j + 2]};
                    double go, ho;
                    relax_gen<D>(cr1, xi, double(sg[j * kSL + l1]), double(sg[(NB + j) * kSL + l1]), K3D, Kin, go,
                                 ho);
                    sm.gB[j * kSL + l1] = Real(go);
                    sm.hB[j * kSL + l1] = Real(ho);
                }
            }
        }
        __syncthreads();
        stage2_gen<D, Real, NB>(m, sm, nb, t, a.ds.err);
        __syncthreads();
        if (!has_item) continue;
        // stage 3: reconstruction, face values, raw face moments
        Real* fg = fvg + static_cast<size_t>(d0) * nI + v.gi;
        Real* fh = fvh + static_cast<size_t>(d0) * nI + v.gi;
        for (int j = 0; j < nb; ++j) {
            const double xi[3] = {xw[4 * j], xw[4 * j + 1], xw[4 * j + 2]};
            const double w = xw[4 * j + 3];
            const double xs = xi_dot_s(xi, v.S);
            const bool own_up = xs >= kVSmall, nei_up = xs < -kVSmall;
            const Real hx = Real(hdt * xi[0]), hy = Real(hdt * xi[1]), hz = Real(hdt * xi[2]);
            Real gg = 0, hh = 0;
            bool store = true, count = true;
            if (v.kind == ITEM_TILE_INTERNAL) {
                recon_g<D, Real, NB>(sm, j, own_up ? v.la : v.lb, Real(own_up ? v.da[0] : v.db[0]) - hx,
                                     Real(own_up ? v.da[1] : v.db[1]) - hy, Real(own_up ? v.da[2] : v.db[2]) - hz, gg,
                                     hh);
                if (!own_up && !nei_up) {   // exactly tangential: both sides (fvDVM.C:847-863)
                    Real g1, h1;
                    recon_g<D, Real, NB>(sm, j, v.la, Real(v.da[0]) - hx, Real(v.da[1]) - hy, Real(v.da[2]) - hz,
                                         g1, h1);
                    gg = Real(0.5) * (gg + g1);
                    hh = Real(0.5) * (hh + h1);
                }
            } else if (v.kind != ITEM_MESH_BOUNDARY) {
                // tile-boundary face: this side weighted 1 upwind, 1/2
                // tangential, 0 downwind; the upwind tile writes both slots
                const bool own_side = v.kind == ITEM_TB_OWN;
                const bool up = own_side ? own_up : nei_up;
                const bool tang = !own_up && !nei_up;
                if (up || tang) {
                    recon_g<D, Real, NB>(sm, j, v.la, Real(v.da[0]) - hx, Real(v.da[1]) - hy, Real(v.da[2]) - hz,
                                         gg, hh);
                    if (!up) {
                        gg *= Real(0.5);
                        hh *= Real(0.5);
                    } else {
                        fvg[static_cast<size_t>(d0 + j) * nI + v.other] = gg;
                        fvh[static_cast<size_t>(d0 + j) * nI + v.other] = hh;
                    }
                } else {
                    store = count = false;
                }
            } else {
                const int pt = v.ptype;
                if (pt == DUGKS_PATCH_ZERO_GRADIENT) {
                    gg = sm.gB[j * kSL + v.la];
                    hh = sm.hB[j * kSL + v.la];
                } else if (xs > 0) {
                    recon_g<D, Real, NB>(sm, j, v.la, Real(v.da[0]) - hx, Real(v.da[1]) - hy, Real(v.da[2]) - hz,
                                         gg, hh);
                    if (pt == DUGKS_PATCH_MAXWELL_WALL) acc[MOM_OUT] = fma(w * double(gg), xs, acc[MOM_OUT]);
                } else if (pt == DUGKS_PATCH_MAXWELL_WALL) {
                    store = count = false;   // through rho_w in the face combine
                } else {
                    // far field, pressure: rho_b M(U_owner, T_b); mixed: rho_b M(U_b, T_b)
                    const BRec* br = a.ds.brec + v.face;
                    double bU[3];
                    if (pt == DUGKS_PATCH_MIXED) {
                        for (int i = 0; i < 3; ++i) bU[i] = __ldg(&br->U[i]);
                    } else {
                        const int own = chk(__ldg(m.bface_owner + v.face), 0, m.nC, a.ds.err);
                        for (int i = 0; i < 3; ++i) bU[i] = __ldg(a.ds.cellrec + (REC_UX + i) * nC + own);
                    }
                    const double cx = xi[0] - bU[0], cy = xi[1] - bU[1], cz = xi[2] - bU[2];
                    const double ge = __ldg(&br->rho_in) * __ldg(&br->K_in) *
                                      exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                    gg = Real(ge);
                    hh = Real(ge * __ldg(&br->hfac));
                    store = false;
                }
            }
            if (count) add_dv<D>(acc, w, xi, double(gg), double(hh));
            if (store) {
                fg[j * nI] = gg;
                fh[j * nI] = hh;
            }
        }
    }
    if (has_item) {
        double* p = a.ds.partF + (static_cast<size_t>(blockIdx.y) * m.n_items + v.gi) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) p[j] = acc[j];
    }
}

template <typename Real, int NB>
struct SmemBG {
    double* xw;    // [2][NB][4]
    Real* st;      // [2][NB][kSI] staged face values g, h of the items
    Real* Fg;      // [NB][kSI] fluxes xi.S g_f
    Real* Fh;
    double* red;   // end-of-CTA reduction of the split cell moments (aliases st, Fg, Fh)
    static constexpr size_t bytes() {
        return 2 * NB * 4 * sizeof(double) + 4 * static_cast<size_t>(NB) * kSI * sizeof(Real);
    }
};

static_assert(static_cast<size_t>(kParts0 - 1) * kS0 * 20 * sizeof(double) <= 4 * 8 * kSI * sizeof(float),
              "the cell-moment reduction must fit in the staging arrays");

template <typename Real, int NB>
__device__ __forceinline__ SmemBG<Real, NB> carve_bg(unsigned char* base) {
    SmemBG<Real, NB> s;
    s.xw = reinterpret_cast<double*>(base);
    s.st = reinterpret_cast<Real*>(s.xw + 2 * NB * 4);
    s.Fg = s.st + 2 * NB * kSI;
    s.Fh = s.Fg + NB * kSI;
    s.red = reinterpret_cast<double*>(s.st);
    return s;
}

template <int D, typename Real, int NB>
__global__ void __launch_bounds__(kThreads, 1) k_pass_b_gen(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemBG<Real, NB> sm = carve_bg<Real, NB>(smem_raw);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    Real* gn = reinterpret_cast<Real*>(a.ds.g[1 - a.ds.cur]);
    Real* hn = reinterpret_cast<Real*>(a.ds.h[1 - a.ds.cur]);
    const Real* fvg = reinterpret_cast<const Real*>(a.ds.fvg);
    const Real* fvh = reinterpret_cast<const Real*>(a.ds.fvh);
    const double K3D = m.K + 3.0 - m.D, Kin = m.K;
    const size_t nI = static_cast<size_t>(m.n_items), nC = static_cast<size_t>(m.nC);

    const int it = threadIdx.x;
    const bool has_item = it < t.nit;
    const int gi = t.ioff + (has_item ? it : 0);
    int kind = 0, other = 0, pt = 0, face = 0;
    double S[3] = {0, 0, 0};
    Rec<double> fr{};
    if (has_item) {
        kind = __ldg(m.it_meta + gi) & 15;
        pt = __ldg(m.it_meta + gi) >> 4;
        other = __ldg(m.it_other + gi);
        face = __ldg(m.it_face + gi);
        if (kind == ITEM_TB_OWN || kind == ITEM_TB_NEI) other = chk(other, 0, m.n_items, a.ds.err);
        if (kind == ITEM_MESH_BOUNDARY) face = chk(face, 0, m.nBF, a.ds.err);
#pragma unroll
        for (int q = 0; q < 3; ++q) S[q] = __ldg(m.it_geo + q * nI + gi);
    }
    const int lc = threadIdx.x % kS0, part = threadIdx.x / kS0;
    const bool has_cell = lc < t.n0;
    const int c = t.b + (has_cell ? lc : 0);
    const double dtV = has_cell ? step_dt(a) * __ldg(m.dtV + c) : 0.0;
    Rec<double> cr{};
    if (has_cell) cr = rec_at(a.ds.cellrec, nC, c);
    int ent_off[kRegFaces];
    unsigned ent_neg[kRegFaces];
#pragma unroll
    for (int s = 0; s < kRegFaces; ++s) {
        const int e = (has_cell && s < m.nf_max) ? __ldg(m.cf_item + static_cast<size_t>(s) * nC + c) : 0;
        ent_off[s] = e == 0 ? kSI - 1 : chk((e > 0 ? e : -e) - 1, 0, t.nit, a.ds.err);
        ent_neg[s] = e < 0 ? 1u : 0u;
    }
    if (threadIdx.x == kThreads - 1)
        for (int j = 0; j < NB; ++j) {
            sm.Fg[j * kSI + kSI - 1] = Real(0);
            sm.Fh[j * kSI + kSI - 1] = Real(0);
        }
    double acc[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;
    // macroFlux yes (the velocity-mesh branch, fvDVM.C:1562-1611): the cell's
    // rho, rho U, rho E gain sum_DV w (1, xi, |xi|^2/2 & h/2) times the flux
    // term dt/V sum_f (+-)(xi.S) g_f of the update
    double accx[5] = {0, 0, 0, 0, 0};
    const bool fx = m.macro_flux != 0;

    const int d_first = t.r0 - m.row_base, d_end = t.r1 - m.row_base;
    const int nbt = (d_end - d_first + NB - 1) / NB;
    auto stage_batch = [&](int k, int buf) {
        const int d0 = d_first + k * NB, nb = min(NB, d_end - d0);
        load_dv_batch<NB>(m, sm.xw + buf * NB * 4, m.dv_base + d0, nb);
        if (has_item) {
            for (int j = 0; j < nb; ++j) {
                cp_async(sm.st + j * kSI + it, fvg + static_cast<size_t>(d0 + j) * nI + gi);
                cp_async(sm.st + (NB + j) * kSI + it, fvh + static_cast<size_t>(d0 + j) * nI + gi);
            }
        }
        cp_commit();
    };
    if (nbt > 0) stage_batch(0, 0);
    for (int k = 0; k < nbt; ++k) {
        const int buf = k & 1;
        const int d0 = d_first + k * NB, nb = min(NB, d_end - d0);
        cp_wait_all();
        __syncthreads();  // batch k staged; the previous batch's stage 4 is done with the fluxes
        if (has_item && k == 0) fr = rec_at(a.ds.facerec, nI, gi);
        const double* xw = sm.xw + buf * NB * 4;
        // stage 3: relaxed face DFs and fluxes of the items
        if (has_item) {
            for (int j = 0; j < nb; ++j) {
                const double xi[3] = {xw[4 * j], xw[4 * j + 1], xw[4 * j + 2]};
                const double xs = xi_dot_s(xi, S);
                double gf = double(sm.st[j * kSI + it]), hf = double(sm.st[(NB + j) * kSI + it]);
                if (kind != ITEM_MESH_BOUNDARY) {
                    if (kind != ITEM_TILE_INTERNAL && !(xs >= kVSmall) && !(xs < -kVSmall)) {
                        const size_t o = static_cast<size_t>(d0 + j) * nI + other;
                        gf += double(__ldg(fvg + o));
                        hf += double(__ldg(fvh + o));
                    }
                    relax_gen<D>(fr, xi, gf, hf, K3D, Kin, gf, hf);
                } else if (xs > 0) {
                    relax_gen<D>(fr, xi, gf, hf, K3D, Kin, gf, hf);
                } else if (pt != DUGKS_PATCH_ZERO_GRADIENT) {
                    const BRec* br = a.ds.brec + face;
                    double bU[3];
                    if (pt == DUGKS_PATCH_MAXWELL_WALL || pt == DUGKS_PATCH_MIXED) {
                        for (int i = 0; i < 3; ++i) bU[i] = __ldg(&br->U[i]);
                    } else {
                        const int own = chk(__ldg(m.bface_owner + face), 0, m.nC, a.ds.err);
                        for (int i = 0; i < 3; ++i) bU[i] = __ldg(a.ds.cellrec + (REC_UX + i) * nC + own);
                    }
                    const double cx = xi[0] - bU[0], cy = xi[1] - bU[1], cz = xi[2] - bU[2];
                    const double ge = br->rho_in * __ldg(&br->K_in) *
                                      exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                    gf = double(Real(ge));
                    hf = double(Real(ge * __ldg(&br->hfac)));
                }
                sm.Fg[j * kSI + it] = Real(xs * gf);
                sm.Fh[j * kSI + it] = Real(xs * hf);
            }
        }
        __syncthreads();
        if (k + 1 < nbt) stage_batch(k + 1, buf ^ 1);
        // stage 4: g~ <- -g~/3 + 4/3 gbar+ - dt/V sum_f (+-)(xi.S) g_f, cell moments
        if (has_cell) {
            for (int j = part; j < nb; j += kParts0) {
                const double xi[3] = {xw[4 * j], xw[4 * j + 1], xw[4 * j + 2]};
                const size_t idx = static_cast<size_t>(d0 + j) * nC + c;
                const Real gt = g[idx], ht = h[idx];
                double gb, hb;
                relax_gen<D>(cr, xi, double(gt), double(ht), K3D, Kin, gb, hb);
                const Real* Fg = sm.Fg + j * kSI;
                const Real* Fh = sm.Fh + j * kSI;
                Real sg = 0, sh = 0;
#pragma unroll
                for (int s = 0; s < kRegFaces; ++s) {
                    sg += flip_sign(Fg[ent_off[s]], ent_neg[s]);
                    sh += flip_sign(Fh[ent_off[s]], ent_neg[s]);
                }
                for (int s = kRegFaces; s < m.nf_max; ++s) {
                    const int e = __ldg(m.cf_item + static_cast<size_t>(s) * nC + c);
                    if (e != 0) {
                        const int i = chk((e > 0 ? e : -e) - 1, 0, t.nit, a.ds.err);
                        sg += e > 0 ? Fg[i] : -Fg[i];
                        sh += e > 0 ? Fh[i] : -Fh[i];
                    }
                }
                const Real g_new = Real(fma(-1.0 / 3, double(gt), fma(4.0 / 3, gb, double(sg) * dtV)));
                const Real h_new = Real(fma(-1.0 / 3, double(ht), fma(4.0 / 3, hb, double(sh) * dtV)));
                gn[idx] = g_new;
                hn[idx] = h_new;
                add_dv<D>(acc, xw[4 * j + 3], xi, double(g_new), double(h_new));
                if (fx) {
                    const double w = xw[4 * j + 3], fg = double(sg) * dtV, fhh = double(sh) * dtV;
                    const double a = w * fg;
                    accx[0] += a;
                    accx[1] += a * xi[0];
                    accx[2] += a * xi[1];
                    accx[3] += a * xi[2];
                    accx[4] += 0.5 * w * (fg * (xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]) + fhh);
                }
            }
        }
    }
    // the cell moments of a cell are split over kParts0 threads: reduce them
    // through shared memory in a fixed order
    __syncthreads();
    if (part > 0 && has_cell) {
        for (int j = 0; j < 15; ++j) sm.red[((part - 1) * kS0 + lc) * 20 + j] = acc[j];
        for (int j = 0; j < 5; ++j) sm.red[((part - 1) * kS0 + lc) * 20 + 15 + j] = accx[j];
    }
    __syncthreads();
    if (part == 0 && has_cell) {
        for (int p = 1; p < kParts0; ++p) {
            for (int j = 0; j < 15; ++j) acc[j] += sm.red[((p - 1) * kS0 + lc) * 20 + j];
            for (int j = 0; j < 5; ++j) accx[j] += sm.red[((p - 1) * kS0 + lc) * 20 + 15 + j];
        }
        double* dst = a.ds.partC + (static_cast<size_t>(blockIdx.y) * m.nC + c) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) dst[j] = acc[j];
        if (fx) {
            double* dx = a.ds.partX + (static_cast<size_t>(blockIdx.y) * m.nC + c) * kFX;
            for (int j = 0; j < 5; ++j) dx[j] = accx[j];
        }
    }
}

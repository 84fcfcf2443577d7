// The two tile passes of the DUGKS step (sm_100a).
//
// A CTA of 512 threads owns one tile (up to 256 L0 cells, their L1 ring, and
// the items = faces touching L0, sorted by kind) and one chunk of discrete
// velocities, which it walks in batches of NB DVs.  Per batch:
//   stage 1  gbar+/hbar+ of the L0+L1 cells into shared memory
//            (updateGHbarPvol, fvDVM.C:648-683); one thread per cell
//   stage 2  least-squares gradients of the L0 cells (leastSquaresGrad;
//            boundary faces add lsB * (patch value - cell value) = 0, the
//            gBarPvol patches being zero-gradient fixedGradient,
//            fvDVM.C:456-485, :775-809); two threads per cell, DVs split
//   stage 3  per item: upwind reconstruction at the half step
//            (updateGHbarSurf, fvDVM.C:755-1029), branch-free: the upwind
//            side is selected, not branched on
//            pass A: raw face moments in registers (updateMacroSurf,
//                    :1181-1297), wall out-flux, XB hand-over
//            pass B: face relaxation (updateGHsurf, :1362-1457), flux
//   stage 4  (pass B) flux gather, g~/h~ update (updateGHtildeVol,
//            :1462-1519) and raw cell moments (updateMacroVol, :1528-1554)
// Every table the CTA reads (cell and face records, item geometry, stencils)
// is a structure of arrays indexed by consecutive threads; the DV rows of
// g~, h~ are read with consecutive threads on consecutive cells.
#include "dugks_device.cuh"

namespace dugks {

namespace {

constexpr int kCellSplit = kThreads / kMaxTile;  // threads per L0 cell in stages 2 and 4

template <typename Real>
struct Batch;
template <>
struct Batch<double> {
    static constexpr int A = 8, B = 4;
};
template <>
struct Batch<float> {
    static constexpr int A = 16, B = 8;
};

template <int D, typename Real, int NB>
struct Smem {
    double* dv;      // [NB][5]: xi (3), w, |xi|^2
    int* dvi;        // [NB][4]: ix, iy, iz of the DV
    Real *gB, *hB;   // [NB][sl]
    Real *Gg, *Gh;   // [NB][sg]
    Real *Fg, *Fh;   // [NB][si]   pass B
    Real *gT, *hT;   // [NB][s0]   pass B
    int sl, sg, si, s0;
};

template <int D, typename Real, int NB>
__device__ __forceinline__ Smem<D, Real, NB> carve(unsigned char* base, const StepArgs& a) {
    Smem<D, Real, NB> s;
    s.dv = reinterpret_cast<double*>(base);
    s.dvi = reinterpret_cast<int*>(base + NB * 5 * sizeof(double));
    Real* p = reinterpret_cast<Real*>(base + NB * 5 * sizeof(double) + NB * 4 * sizeof(int));
    s.sl = a.dims_local;
    s.sg = a.dims_l0 * D;
    s.si = a.dims_items;
    s.s0 = a.dims_l0;
    s.gB = p;
    p += NB * s.sl;
    s.hB = p;
    p += NB * s.sl;
    s.Gg = p;
    p += NB * s.sg;
    s.Gh = p;
    p += NB * s.sg;
    s.Fg = p;
    p += NB * s.si;
    s.Fh = p;
    p += NB * s.si;
    s.gT = p;
    p += NB * s.s0;
    s.hT = p;
    return s;
}

template <int D, typename Real, int NB>
size_t smem_bytes(int max_local, int max_l0, int max_items, bool pass_b) {
    size_t n = 2 * static_cast<size_t>(max_local) + 2 * static_cast<size_t>(max_l0) * D;
    if (pass_b) n += 2 * static_cast<size_t>(max_items) + 2 * static_cast<size_t>(max_l0);
    size_t bytes = NB * 5 * sizeof(double) + NB * 4 * sizeof(int) + NB * n * sizeof(Real);
    // the end-of-CTA reduction of the split cell moments reuses the arrays
    const size_t red = static_cast<size_t>(kMaxTile) * 15 * sizeof(double) + NB * 5 * sizeof(double);
    return bytes > red ? bytes : red;
}

struct TileRange {
    int b, n0, loff, nloc, ioff, nit, d0, d1;
};

__device__ __forceinline__ TileRange tile_range(const DevMesh& m, const int32_t* chunk_begin) {
    TileRange t;
    const int tile = blockIdx.x, chunk = blockIdx.y;
    t.b = __ldg(m.tile_begin + tile);
    t.n0 = __ldg(m.tile_begin + tile + 1) - t.b;
    t.loff = __ldg(m.tile_loc_off + tile);
    t.nloc = __ldg(m.tile_loc_off + tile + 1) - t.loff;
    t.ioff = __ldg(m.tile_item_off + tile);
    t.nit = __ldg(m.tile_item_off + tile + 1) - t.ioff;
    t.d0 = __ldg(chunk_begin + chunk);
    t.d1 = __ldg(chunk_begin + chunk + 1);
    return t;
}

// load a coefficient record (structure of arrays, n entities)
template <typename Real>
__device__ __forceinline__ Rec<Real> load_rec_soa(const double* __restrict__ rec, int n, int e) {
    Rec<Real> r;
    r.U[0] = Real(__ldg(rec + REC_UX * static_cast<size_t>(n) + e));
    r.U[1] = Real(__ldg(rec + REC_UY * static_cast<size_t>(n) + e));
    r.U[2] = Real(__ldg(rec + REC_UZ * static_cast<size_t>(n) + e));
    r.invRT = Real(__ldg(rec + REC_INVRT * static_cast<size_t>(n) + e));
    r.A = Real(__ldg(rec + REC_A * static_cast<size_t>(n) + e));
    r.r = Real(__ldg(rec + REC_R * static_cast<size_t>(n) + e));
    r.qv[0] = Real(__ldg(rec + REC_QX * static_cast<size_t>(n) + e));
    r.qv[1] = Real(__ldg(rec + REC_QY * static_cast<size_t>(n) + e));
    r.qv[2] = Real(__ldg(rec + REC_QZ * static_cast<size_t>(n) + e));
    r.RTh = Real(__ldg(rec + REC_RTH * static_cast<size_t>(n) + e));
    return r;
}

struct ItemSoa {
    int kind, ptype, lo, ln, face, xbw, xbr;
    double S[3], dO[3], dN[3];
};

__device__ __forceinline__ ItemSoa load_item_soa(const DevMesh& m, int i) {
    ItemSoa v;
    const int meta = __ldg(m.it_meta + i), loc = __ldg(m.it_loc + i);
    v.kind = meta & 15;
    v.ptype = meta >> 4;
    v.lo = loc & 0xffff;
    v.ln = (loc >> 16) & 0xffff;
    v.face = __ldg(m.it_face + i);
    v.xbw = __ldg(m.it_xbw + i);
    v.xbr = __ldg(m.it_xbr + i);
    const size_t n = static_cast<size_t>(m.n_items);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        v.S[q] = __ldg(m.it_geo + q * n + i);
        v.dO[q] = __ldg(m.it_geo + (3 + q) * n + i);
        v.dN[q] = __ldg(m.it_geo + (6 + q) * n + i);
    }
    return v;
}

// DV table of a batch (also the barrier that releases the previous batch's
// shared arrays)
template <int D, typename Real, int NB>
__device__ __forceinline__ int load_batch(const DevMesh& m, int d0, int d1, const Smem<D, Real, NB>& sm) {
    const int nb = min(NB, d1 - d0);
    __syncthreads();
    if (threadIdx.x < nb) {
        const int d = d0 + threadIdx.x;
        const double x = __ldg(m.xi + 3 * d), y = __ldg(m.xi + 3 * d + 1), z = __ldg(m.xi + 3 * d + 2);
        double* p = sm.dv + 5 * threadIdx.x;
        p[0] = x;
        p[1] = y;
        p[2] = z;
        p[3] = __ldg(m.w + d);
        p[4] = x * x + y * y + z * z;
        const int n = m.n1d;
        int* q = sm.dvi + 4 * threadIdx.x;
        q[0] = d % n;
        q[1] = (d / n) % n;
        q[2] = d / (n * n);
    }
    __syncthreads();
    return nb;
}

// Maxwellian A e_x e_y e_z of entity e (cell or face) at the DV with 1-D
// indices q[0..2], from the tables the combine kernels write
template <int D, typename Real>
__device__ __forceinline__ Real maxwell_tab(const Real* __restrict__ tab, size_t n, int n1d, int e, const int* q) {
    Real E = __ldg(tab + static_cast<size_t>(q[0]) * n + e) * __ldg(tab + (static_cast<size_t>(n1d) + q[1]) * n + e);
    if (D == 3) E *= __ldg(tab + (2 * static_cast<size_t>(n1d) + q[2]) * n + e);
    return E;
}

template <int D, typename Real, int NB, bool KEEP>
__device__ __forceinline__ void stage_ghbar(const DevMesh& m, const double* __restrict__ crec,
                                            const Real* __restrict__ ctab, const Real* __restrict__ g,
                                            const Real* __restrict__ h, int d0, int nb, const TileRange& t,
                                            const Smem<D, Real, NB>& sm, Real K3D, Real Kin) {
    // state rows are loaded LG DVs at a time (LG loads in flight per thread)
    constexpr int LG = NB < 4 ? NB : 4;
    for (int l = threadIdx.x; l < t.nloc; l += kThreads) {
        const int c = __ldg(m.loc_cells + t.loff + l);
        const Rec<Real> r = load_rec_soa<Real>(crec, m.nC, c);
        const Real* gr = g + static_cast<size_t>(d0) * m.nC + c;
        const Real* hr = h + static_cast<size_t>(d0) * m.nC + c;
#pragma unroll 1
        for (int b0 = 0; b0 < nb; b0 += LG) {
            Real gt[LG], ht[LG];
#pragma unroll
            for (int j = 0; j < LG; ++j) {
                if (b0 + j < nb) {
                    gt[j] = gr[static_cast<size_t>(b0 + j) * m.nC];
                    ht[j] = hr[static_cast<size_t>(b0 + j) * m.nC];
                }
            }
#pragma unroll
            for (int j = 0; j < LG; ++j) {
                const int b = b0 + j;
                if (b >= nb) continue;
                const Real xi[3] = {Real(sm.dv[5 * b]), Real(sm.dv[5 * b + 1]), Real(sm.dv[5 * b + 2])};
                const Real E = maxwell_tab<D, Real>(ctab, m.nC, m.n1d, c, sm.dvi + 4 * b);
                Real gS, hS;
                shakhov_m<D, Real>(xi, r, E, K3D, Kin, gS, hS);
                sm.gB[b * sm.sl + l] = gt[j] + r.r * (gS - gt[j]);
                sm.hB[b * sm.sl + l] = ht[j] + r.r * (hS - ht[j]);
                if (KEEP && l < t.n0) {
                    sm.gT[b * sm.s0 + l] = gt[j];
                    sm.hT[b * sm.s0 + l] = ht[j];
                }
            }
        }
    }
    __syncthreads();
}

// Hex cells have at most 6 face neighbours: their stencil stays in
// registers while the thread walks its DVs of the batch
constexpr int kMaxRegStencil = 6;

template <int D, typename Real, int NB>
__device__ __forceinline__ void grad_one(const Smem<D, Real, NB>& sm, int b, int l, const int* nbi,
                                         const Real (*ls)[D], int nk) {
    const Real* gB = sm.gB + b * sm.sl;
    const Real* hB = sm.hB + b * sm.sl;
    const Real g0 = gB[l], h0 = hB[l];
    Real gx[D], hx[D];
#pragma unroll
    for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
#pragma unroll
    for (int k = 0; k < kMaxRegStencil; ++k) {
        if (k < nk) {
            const Real dg = gB[nbi[k]] - g0, dh = hB[nbi[k]] - h0;
#pragma unroll
            for (int q = 0; q < D; ++q) {
                gx[q] += ls[k][q] * dg;
                hx[q] += ls[k][q] * dh;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < D; ++q) {
        sm.Gg[b * sm.sg + q * sm.s0 + l] = gx[q];
        sm.Gh[b * sm.sg + q * sm.s0 + l] = hx[q];
    }
}

template <int D, typename Real, int NB>
__device__ __forceinline__ void stage_grad(const DevMesh& m, int nb, const TileRange& t,
                                           const Smem<D, Real, NB>& sm) {
    const int l = threadIdx.x % kMaxTile, part = threadIdx.x / kMaxTile;
    if (l < t.n0) {
        const int c = t.b + l;
        if (m.nb_max <= kMaxRegStencil) {
            int nbi[kMaxRegStencil];
            Real ls[kMaxRegStencil][D];
            int nk = 0;
#pragma unroll
            for (int k = 0; k < kMaxRegStencil; ++k) {
                nbi[k] = l;
#pragma unroll
                for (int q = 0; q < D; ++q) ls[k][q] = Real(0);
                if (k < m.nb_max) {
                    const int n = __ldg(m.grad_nb + static_cast<size_t>(k) * m.nC + c);
                    if (n >= 0) {
                        nbi[k] = n;
                        nk = k + 1;
#pragma unroll
                        for (int q = 0; q < D; ++q)
                            ls[k][q] = Real(__ldg(m.grad_ls + (static_cast<size_t>(k) * 3 + q) * m.nC + c));
                    }
                }
            }
#pragma unroll 1
            for (int b = part; b < nb; b += kCellSplit) grad_one<D, Real, NB>(sm, b, l, nbi, ls, nk);
        } else {
#pragma unroll 1
            for (int b = part; b < nb; b += kCellSplit) {
                const Real* gB = sm.gB + b * sm.sl;
                const Real* hB = sm.hB + b * sm.sl;
                const Real g0 = gB[l], h0 = hB[l];
                Real gx[D], hx[D];
#pragma unroll
                for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
                for (int k = 0; k < m.nb_max; ++k) {
                    const int n = __ldg(m.grad_nb + static_cast<size_t>(k) * m.nC + c);
                    if (n < 0) continue;
                    const Real dg = gB[n] - g0, dh = hB[n] - h0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        const Real lsq = Real(__ldg(m.grad_ls + (static_cast<size_t>(k) * 3 + q) * m.nC + c));
                        gx[q] += lsq * dg;
                        hx[q] += lsq * dh;
                    }
                }
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    sm.Gg[b * sm.sg + q * sm.s0 + l] = gx[q];
                    sm.Gh[b * sm.sg + q * sm.s0 + l] = hx[q];
                }
            }
        }
    }
    __syncthreads();
}

// reconstruction at the half step from local cell l (fvDVM.C:832-836):
// gbar+_l + grad_l . (Cf - C_l - xi dt/2)
// (the offset d is passed by value: selecting between two arrays by pointer
// would put the item in local memory)
template <int D, typename Real, int NB>
__device__ __forceinline__ void recon(const Smem<D, Real, NB>& sm, int b, int l, double dx, double dy, double dz,
                                      const Real xi[3], Real hdt, Real& g, Real& h) {
    const Real v[3] = {Real(dx) - hdt * xi[0], Real(dy) - hdt * xi[1], Real(dz) - hdt * xi[2]};
    const Real* Gg = sm.Gg + b * sm.sg + l;
    const Real* Gh = sm.Gh + b * sm.sg + l;
    Real gg = sm.gB[b * sm.sl + l], hh = sm.hB[b * sm.sl + l];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        gg += Gg[q * sm.s0] * v[q];
        hh += Gh[q * sm.s0] * v[q];
    }
    g = gg;
    h = hh;
}

// reconstruction from the side `own` (owner) or not (neighbour) of an item
template <int D, typename Real, int NB>
__device__ __forceinline__ void recon_side(const Smem<D, Real, NB>& sm, int b, const ItemSoa& v, bool own,
                                           const Real xi[3], Real hdt, Real& g, Real& h) {
    recon<D, Real, NB>(sm, b, own ? v.lo : v.ln, own ? v.dO[0] : v.dN[0], own ? v.dO[1] : v.dN[1],
                       own ? v.dO[2] : v.dN[2], xi, hdt, g, h);
}

// reconstruction from the upwind side of an item whose both sides are in
// L0: the side is selected per DV, the code path is the same for all lanes
// (the exactly tangential case, both sides averaged, is the only branch)
template <int D, typename Real, int NB>
__device__ __forceinline__ void recon_upwind(const Smem<D, Real, NB>& sm, int b, const ItemSoa& v, double xs,
                                             const Real xi[3], Real hdt, Real& g, Real& h) {
    const bool own_up = xs >= kVSmall, nei_up = xs < -kVSmall;
    if (own_up || nei_up) {
        recon_side<D, Real, NB>(sm, b, v, own_up, xi, hdt, g, h);
    } else {
        Real g1, h1, g2, h2;
        recon_side<D, Real, NB>(sm, b, v, true, xi, hdt, g1, h1);
        recon_side<D, Real, NB>(sm, b, v, false, xi, hdt, g2, h2);
        g = Real(0.5) * (g2 + g1);
        h = Real(0.5) * (h2 + h1);
    }
}

// ---------------------------------------------------------------------
// Pass A: face reconstruction and raw face moments
// ---------------------------------------------------------------------
template <int D, typename Real, int IPT, int NB>
__global__ void __launch_bounds__(kThreads, 1) k_pass_a(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem<D, Real, NB> sm = carve<D, Real, NB>(smem_raw, a);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    const Real* ctab = reinterpret_cast<const Real*>(a.ds.ctab);
    Real* const xbg0 = reinterpret_cast<Real*>(a.ds.xbg[0]);
    Real* const xbg1 = reinterpret_cast<Real*>(a.ds.xbg[1]);
    Real* const xbh0 = reinterpret_cast<Real*>(a.ds.xbh[0]);
    Real* const xbh1 = reinterpret_cast<Real*>(a.ds.xbh[1]);
    const Real K3D = Real(m.K + 3 - m.D), Kin = Real(m.K);
    const Real hdt = Real(0.5 * a.dt);
    double acc[IPT][15];
#pragma unroll
    for (int i = 0; i < IPT; ++i)
#pragma unroll
        for (int j = 0; j < 15; ++j) acc[i][j] = 0.0;

    for (int d0 = t.d0; d0 < t.d1; d0 += NB) {
        const int nb = load_batch<D, Real, NB>(m, d0, t.d1, sm);
        stage_ghbar<D, Real, NB, false>(m, a.ds.cellrec, ctab, g, h, d0, nb, t, sm, K3D, Kin);
        stage_grad<D, Real, NB>(m, nb, t, sm);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int it = threadIdx.x + k * kThreads;
            if (it >= t.nit) continue;
            const ItemSoa v = load_item_soa(m, t.ioff + it);
#pragma unroll 1
            for (int b = 0; b < nb; ++b) {
                const double xid[3] = {sm.dv[5 * b], sm.dv[5 * b + 1], sm.dv[5 * b + 2]};
                const double wd = sm.dv[5 * b + 3], xi2 = sm.dv[5 * b + 4];
                const Real xi[3] = {Real(xid[0]), Real(xid[1]), Real(xid[2])};
                const double xs = xi_dot_s(xid, v.S);
                if (v.kind == ITEM_TILE_INTERNAL) {
                    Real gg, hh;
                    recon_upwind<D, Real, NB>(sm, b, v, xs, xi, hdt, gg, hh);
                    accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                } else if (v.kind != ITEM_MESH_BOUNDARY) {
                    // tile-boundary face: this tile contributes its side only
                    // (weight 1 upwind, 1/2 tangential, 0 downwind) and hands
                    // it to the other tile through XB
                    const bool own_side = v.kind == ITEM_TB_OWN;
                    const bool up = own_side ? xs >= kVSmall : xs < -kVSmall;
                    const bool tang = !(xs >= kVSmall) && !(xs < -kVSmall);
                    const Real cs = up ? Real(1) : (tang ? Real(0.5) : Real(0));
                    Real g1, h1;
                    recon_side<D, Real, NB>(sm, b, v, own_side, xi, hdt, g1, h1);
                    g1 *= cs;
                    h1 *= cs;
                    if (up || tang) {
                        const size_t xi_ = static_cast<size_t>(d0 + b) * m.n_tbf + v.xbw;
                        (own_side ? xbg0 : xbg1)[xi_] = g1;
                        (own_side ? xbh0 : xbh1)[xi_] = h1;
                    }
                    accum<D>(acc[k], wd, xid, xi2, double(g1), double(h1));
                } else if (xs > 0) {
                    // outgoing boundary DF: upwind from the owner (fvDVM.C:916-923, :950-961)
                    Real gg, hh;
                    recon_side<D, Real, NB>(sm, b, v, true, xi, hdt, gg, hh);
                    accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                    if (v.ptype == DUGKS_PATCH_MAXWELL_WALL) acc[k][MOM_OUT] += wd * xs * double(gg);
                } else if (v.ptype == DUGKS_PATCH_FAR_FIELD) {
                    // incoming far field: rho_b M(xi; U_owner, T_b) (fvDVM.C:926-938);
                    // incoming maxwellWall DFs enter through rho_w in the face combine
                    const BRec* br = a.ds.brec + v.face;
                    const int own = __ldg(m.bface_owner + v.face);
                    const double ux = __ldg(a.ds.cellrec + REC_UX * static_cast<size_t>(m.nC) + own);
                    const double uy = __ldg(a.ds.cellrec + REC_UY * static_cast<size_t>(m.nC) + own);
                    const double uz = __ldg(a.ds.cellrec + REC_UZ * static_cast<size_t>(m.nC) + own);
                    const double cx = xid[0] - ux, cy = xid[1] - uy, cz = xid[2] - uz;
                    const double ge = __ldg(&br->rho_in) * __ldg(&br->K_in) *
                                      exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                    const Real gg = Real(ge), hh = Real(ge * __ldg(&br->hfac));
                    accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                }
            }
        }
    }
    const size_t base = static_cast<size_t>(blockIdx.y) * m.n_items + t.ioff;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const int it = threadIdx.x + k * kThreads;
        if (it >= t.nit) continue;
        double* p = a.ds.partF + (base + it) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) p[j] = acc[k][j];
    }
}

// ---------------------------------------------------------------------
// Pass B: face relaxation, volume update, raw cell moments
// ---------------------------------------------------------------------
template <int D, typename Real, int IPT, int NB>
__global__ void __launch_bounds__(kThreads, 1) k_pass_b(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem<D, Real, NB> sm = carve<D, Real, NB>(smem_raw, a);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    Real* gn = reinterpret_cast<Real*>(a.ds.g[1 - a.ds.cur]);
    Real* hn = reinterpret_cast<Real*>(a.ds.h[1 - a.ds.cur]);
    const Real* const xbg0 = reinterpret_cast<const Real*>(a.ds.xbg[0]);
    const Real* const xbg1 = reinterpret_cast<const Real*>(a.ds.xbg[1]);
    const Real* const xbh0 = reinterpret_cast<const Real*>(a.ds.xbh[0]);
    const Real* const xbh1 = reinterpret_cast<const Real*>(a.ds.xbh[1]);
    const Real* ctab = reinterpret_cast<const Real*>(a.ds.ctab);
    const Real* ftab = reinterpret_cast<const Real*>(a.ds.ftab);
    const Real K3D = Real(m.K + 3 - m.D), Kin = Real(m.K);
    const Real hdt = Real(0.5 * a.dt);
    const int lc = threadIdx.x % kMaxTile, part = threadIdx.x / kMaxTile;
    double acc[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;

    for (int d0 = t.d0; d0 < t.d1; d0 += NB) {
        const int nb = load_batch<D, Real, NB>(m, d0, t.d1, sm);
        stage_ghbar<D, Real, NB, true>(m, a.ds.cellrec, ctab, g, h, d0, nb, t, sm, K3D, Kin);
        stage_grad<D, Real, NB>(m, nb, t, sm);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int it = threadIdx.x + k * kThreads;
            if (it >= t.nit) continue;
            const ItemSoa v = load_item_soa(m, t.ioff + it);
            const bool boundary = v.kind == ITEM_MESH_BOUNDARY;
            const int fe = t.ioff + it;  // face records and tables are in item order
            const Rec<Real> fr = load_rec_soa<Real>(a.ds.facerec, m.n_items, fe);
#pragma unroll 1
            for (int b = 0; b < nb; ++b) {
                const double xid[3] = {sm.dv[5 * b], sm.dv[5 * b + 1], sm.dv[5 * b + 2]};
                const Real xi[3] = {Real(xid[0]), Real(xid[1]), Real(xid[2])};
                const double xs = xi_dot_s(xid, v.S);
                Real gf, hf;
                if (v.kind == ITEM_TILE_INTERNAL) {
                    Real gg, hh, gS, hS;
                    recon_upwind<D, Real, NB>(sm, b, v, xs, xi, hdt, gg, hh);
                    const Real E = maxwell_tab<D, Real>(ftab, m.n_items, m.n1d, fe, sm.dvi + 4 * b);
                    shakhov_m<D, Real>(xi, fr, E, K3D, Kin, gS, hS);
                    gf = gg + fr.r * (gS - gg);
                    hf = hh + fr.r * (hS - hh);
                } else if (!boundary) {
                    // tile-boundary face: this side reconstructed here, the
                    // other side's contribution from XB (written in pass A)
                    const bool own_side = v.kind == ITEM_TB_OWN;
                    const bool own_up = xs >= kVSmall, nei_up = xs < -kVSmall;
                    const bool here_up = own_side ? own_up : nei_up;
                    const bool there_up = own_side ? nei_up : own_up;
                    const bool tang = !own_up && !nei_up;
                    Real g1, h1;
                    recon_side<D, Real, NB>(sm, b, v, own_side, xi, hdt, g1, h1);
                    Real xg = 0, xh = 0;
                    if (there_up || tang) {
                        const size_t xr = static_cast<size_t>(d0 + b) * m.n_tbf + v.xbr;
                        xg = (own_side ? xbg1 : xbg0)[xr];
                        xh = (own_side ? xbh1 : xbh0)[xr];
                    }
                    const Real gg = here_up ? g1 : (there_up ? xg : Real(0.5) * g1 + xg);
                    const Real hh = here_up ? h1 : (there_up ? xh : Real(0.5) * h1 + xh);
                    Real gS, hS;
                    const Real E = maxwell_tab<D, Real>(ftab, m.n_items, m.n1d, fe, sm.dvi + 4 * b);
                    shakhov_m<D, Real>(xi, fr, E, K3D, Kin, gS, hS);
                    gf = gg + fr.r * (gS - gg);
                    hf = hh + fr.r * (hS - hh);
                } else if (xs > 0) {
                    // outgoing boundary DF: reconstruct and relax with the
                    // boundary face coefficients; h uses the internal-face T at
                    // the patch-local index (fvDVM.C:1367, :1413, :1429-1444)
                    Real gg, hh, gS, hS;
                    recon_side<D, Real, NB>(sm, b, v, true, xi, hdt, gg, hh);
                    const Real E = maxwell_tab<D, Real>(ftab, m.n_items, m.n1d, fe, sm.dvi + 4 * b);
                    shakhov_m<D, Real>(xi, fr, E, K3D, Kin, gS, hS);
                    gf = gg + fr.r * (gS - gg);
                    hf = hh + fr.r * (hS - hh);
                } else {
                    // incoming, never relaxed: wall rho_w M(U_w,T_w)
                    // (fvDVM.C:1079-1092), far field rho_b M(U_owner,T_b)
                    const BRec* br = a.ds.brec + v.face;
                    double ux, uy, uz;
                    if (v.ptype == DUGKS_PATCH_FAR_FIELD) {
                        const int own = __ldg(m.bface_owner + v.face);
                        ux = __ldg(a.ds.cellrec + REC_UX * static_cast<size_t>(m.nC) + own);
                        uy = __ldg(a.ds.cellrec + REC_UY * static_cast<size_t>(m.nC) + own);
                        uz = __ldg(a.ds.cellrec + REC_UZ * static_cast<size_t>(m.nC) + own);
                    } else {
                        ux = __ldg(&br->U[0]);
                        uy = __ldg(&br->U[1]);
                        uz = __ldg(&br->U[2]);
                    }
                    const double cx = xid[0] - ux, cy = xid[1] - uy, cz = xid[2] - uz;
                    const double ge = br->rho_in * __ldg(&br->K_in) *
                                      exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                    gf = Real(ge);
                    hf = Real(ge * __ldg(&br->hfac));
                }
                const Real xsr = Real(xs);
                sm.Fg[b * sm.si + it] = xsr * gf;
                sm.Fh[b * sm.si + it] = xsr * hf;
            }
        }
        __syncthreads();
        // volume update of the L0 cells, two threads per cell with the DVs
        // split: g~ <- -g~/3 + 4/3 gbar+ - dt/V sum_f (+-)(xi.S) g_f
        if (lc < t.n0) {
            const int c = t.b + lc;
            const Real dtV = Real(a.dt * __ldg(m.dtV + c));
            int ent[8];
            const int nf = m.nf_max < 8 ? m.nf_max : 8;
#pragma unroll
            for (int s = 0; s < 8; ++s) ent[s] = s < nf ? __ldg(m.cf_item + static_cast<size_t>(s) * m.nC + c) : 0;
#pragma unroll 1
            for (int b = part; b < nb; b += kCellSplit) {
                const Real* Fg = sm.Fg + b * sm.si;
                const Real* Fh = sm.Fh + b * sm.si;
                Real sg = 0, sh = 0;
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    const int e = ent[s];
                    if (e != 0) {
                        const int it = (e > 0 ? e : -e) - 1;
                        sg += e > 0 ? Fg[it] : -Fg[it];
                        sh += e > 0 ? Fh[it] : -Fh[it];
                    }
                }
                for (int s = 8; s < m.nf_max; ++s) {
                    const int e = __ldg(m.cf_item + static_cast<size_t>(s) * m.nC + c);
                    if (e != 0) {
                        const int it = (e > 0 ? e : -e) - 1;
                        sg += e > 0 ? Fg[it] : -Fg[it];
                        sh += e > 0 ? Fh[it] : -Fh[it];
                    }
                }
                const Real g_new =
                    Real(-1.0 / 3) * sm.gT[b * sm.s0 + lc] + Real(4.0 / 3) * sm.gB[b * sm.sl + lc] + sg * dtV;
                const Real h_new =
                    Real(-1.0 / 3) * sm.hT[b * sm.s0 + lc] + Real(4.0 / 3) * sm.hB[b * sm.sl + lc] + sh * dtV;
                const size_t idx = static_cast<size_t>(d0 + b) * m.nC + c;
                gn[idx] = g_new;
                hn[idx] = h_new;
                const double xid[3] = {sm.dv[5 * b], sm.dv[5 * b + 1], sm.dv[5 * b + 2]};
                accum<D>(acc, sm.dv[5 * b + 3], xid, sm.dv[5 * b + 4], double(g_new), double(h_new));
            }
        }
    }
    // the cell moments of a cell are split over kCellSplit threads: reduce
    // them through shared memory in a fixed order
    __syncthreads();
    double* red = reinterpret_cast<double*>(smem_raw);
    if (part > 0 && lc < t.n0)
        for (int j = 0; j < 15; ++j) red[((part - 1) * kMaxTile + lc) * 15 + j] = acc[j];
    __syncthreads();
    if (part == 0 && lc < t.n0) {
        for (int p = 1; p < kCellSplit; ++p)
            for (int j = 0; j < 15; ++j) acc[j] += red[((p - 1) * kMaxTile + lc) * 15 + j];
        double* dst = a.ds.partC + (static_cast<size_t>(blockIdx.y) * m.nC + t.b + lc) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) dst[j] = acc[j];
    }
}

template <int D, typename Real, int IPT>
void launch_pass_t(const StepArgs& a, bool pass_b, cudaStream_t s) {
    dim3 grid(a.dm.n_tiles, a.chunks);
    if (!pass_b) k_pass_a<D, Real, IPT, Batch<Real>::A><<<grid, kThreads, a.smemA, s>>>(a);
    else k_pass_b<D, Real, IPT, Batch<Real>::B><<<grid, kThreads, a.smemB, s>>>(a);
}

template <int D, typename Real>
cudaError_t launch_pass_d(const StepArgs& a, bool pass_b, cudaStream_t s) {
    switch (a.ipt) {
        case 1: launch_pass_t<D, Real, 1>(a, pass_b, s); break;
        case 2: launch_pass_t<D, Real, 2>(a, pass_b, s); break;
        case 3: launch_pass_t<D, Real, 3>(a, pass_b, s); break;
        default: return cudaErrorInvalidConfiguration;
    }
    return cudaGetLastError();
}

template <int D, typename Real, int IPT>
cudaError_t configure_t(size_t smemA, size_t smemB) {
    cudaError_t e = cudaFuncSetAttribute(k_pass_a<D, Real, IPT, Batch<Real>::A>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemA));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_pass_b<D, Real, IPT, Batch<Real>::B>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smemB));
}

template <int D, typename Real>
cudaError_t configure_d(int ipt, size_t smemA, size_t smemB) {
    switch (ipt) {
        case 1: return configure_t<D, Real, 1>(smemA, smemB);
        case 2: return configure_t<D, Real, 2>(smemA, smemB);
        case 3: return configure_t<D, Real, 3>(smemA, smemB);
        default: return cudaErrorInvalidConfiguration;
    }
}

}  // namespace

cudaError_t launch_pass(const StepArgs& a, int precision, bool pass_b, cudaStream_t s) {
    if (precision == DUGKS_FP64)
        return a.dm.D == 3 ? launch_pass_d<3, double>(a, pass_b, s) : launch_pass_d<2, double>(a, pass_b, s);
    return a.dm.D == 3 ? launch_pass_d<3, float>(a, pass_b, s) : launch_pass_d<2, float>(a, pass_b, s);
}

void pass_smem(const DevMesh& dm, int max_local, int max_l0, int max_items, int precision, size_t* smemA,
               size_t* smemB) {
    if (precision == DUGKS_FP64) {
        if (dm.D == 3) {
            *smemA = smem_bytes<3, double, Batch<double>::A>(max_local, max_l0, max_items, false);
            *smemB = smem_bytes<3, double, Batch<double>::B>(max_local, max_l0, max_items, true);
        } else {
            *smemA = smem_bytes<2, double, Batch<double>::A>(max_local, max_l0, max_items, false);
            *smemB = smem_bytes<2, double, Batch<double>::B>(max_local, max_l0, max_items, true);
        }
    } else {
        if (dm.D == 3) {
            *smemA = smem_bytes<3, float, Batch<float>::A>(max_local, max_l0, max_items, false);
            *smemB = smem_bytes<3, float, Batch<float>::B>(max_local, max_l0, max_items, true);
        } else {
            *smemA = smem_bytes<2, float, Batch<float>::A>(max_local, max_l0, max_items, false);
            *smemB = smem_bytes<2, float, Batch<float>::B>(max_local, max_l0, max_items, true);
        }
    }
}

cudaError_t configure_kernels(int precision, int D, int ipt, size_t smemA, size_t smemB) {
    if (precision == DUGKS_FP64)
        return D == 3 ? configure_d<3, double>(ipt, smemA, smemB) : configure_d<2, double>(ipt, smemA, smemB);
    return D == 3 ? configure_d<3, float>(ipt, smemA, smemB) : configure_d<2, float>(ipt, smemA, smemB);
}

}  // namespace dugks

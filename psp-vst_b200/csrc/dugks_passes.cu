// The two tile passes of the DUGKS step (sm_100a).
//
// A CTA owns one tile (L0 cells, L1 ring, the items = faces touching L0)
// and one chunk of discrete velocities, which it walks in batches of B
// DVs.  Per batch:
//   stage 1  gbar+/hbar+ of the L0+L1 cells, B DVs, into shared memory
//            (updateGHbarPvol, fvDVM.C:648-683)
//   stage 2  least-squares gradients of the L0 cells (leastSquaresGrad;
//            boundary faces add lsB * (patch value - cell value) = 0, the
//            gBarPvol patches being zero-gradient fixedGradient,
//            fvDVM.C:456-485, :775-809)
//   stage 3  per item: upwind reconstruction at the half step
//            (updateGHbarSurf, fvDVM.C:755-1029)
//            pass A: raw face moments in registers (updateMacroSurf,
//                    :1181-1297), wall out-flux, XB hand-over
//            pass B: face relaxation (updateGHsurf, :1362-1457), flux
//   stage 4  (pass B) flux gather, g~/h~ update (updateGHtildeVol,
//            :1462-1519) and raw cell moments (updateMacroVol, :1528-1554)
// Tile-invariant data (cell records, stencils, item geometry) is read once
// per batch; the DV rows of g~, h~ are read with consecutive threads on
// consecutive cells.
#include "dugks_device.cuh"

namespace dugks {

namespace {

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
    Real* p = reinterpret_cast<Real*>(base + NB * 5 * sizeof(double));
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
    return NB * 5 * sizeof(double) + NB * n * sizeof(Real);
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
    }
    __syncthreads();
    return nb;
}

template <int D, typename Real, int NB, bool KEEP>
__device__ __forceinline__ void stage_ghbar(const DevMesh& m, const CellRec* __restrict__ crec,
                                            const Real* __restrict__ g, const Real* __restrict__ h, int d0, int nb,
                                            const TileRange& t, const Smem<D, Real, NB>& sm, Real K3D, Real Kin) {
    for (int l = threadIdx.x; l < t.nloc; l += kThreads) {
        const int c = __ldg(m.loc_cells + t.loff + l);
        const Rec<Real> r = load_rec<Real>(crec + c);
        Real gt[NB], ht[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (b < nb) {
                const size_t idx = static_cast<size_t>(d0 + b) * m.nC + c;
                gt[b] = g[idx];
                ht[b] = h[idx];
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (b < nb) {
                const Real xi[3] = {Real(sm.dv[5 * b]), Real(sm.dv[5 * b + 1]), Real(sm.dv[5 * b + 2])};
                Real gS, hS;
                shakhov<D, Real>(xi, r, K3D, Kin, gS, hS);
                sm.gB[b * sm.sl + l] = gt[b] + r.r * (gS - gt[b]);
                sm.hB[b * sm.sl + l] = ht[b] + r.r * (hS - ht[b]);
                if (KEEP && l < t.n0) {
                    sm.gT[b * sm.s0 + l] = gt[b];
                    sm.hT[b * sm.s0 + l] = ht[b];
                }
            }
        }
    }
    __syncthreads();
}

// Hex cells have at most 6 face neighbours: their stencil stays in
// registers while the thread walks the DV batch; larger polyhedra read it
// from memory per DV.
constexpr int kMaxRegStencil = 6;

template <int D, typename Real, int NB>
__device__ __forceinline__ void stage_grad(const DevMesh& m, int nb, const TileRange& t,
                                           const Smem<D, Real, NB>& sm) {
    for (int l = threadIdx.x; l < t.n0; l += kThreads) {
        const int c = t.b + l;
        const int k0 = __ldg(m.grad_off + c), k1 = __ldg(m.grad_off + c + 1);
        const int nk = k1 - k0;
        if (nk <= kMaxRegStencil) {
            int nbi[kMaxRegStencil];
            Real ls[kMaxRegStencil][D];
#pragma unroll
            for (int k = 0; k < kMaxRegStencil; ++k) {
                nbi[k] = k < nk ? __ldg(m.grad_nb + k0 + k) : l;
#pragma unroll
                for (int q = 0; q < D; ++q) ls[k][q] = k < nk ? Real(__ldg(m.grad_ls + 3 * (k0 + k) + q)) : Real(0);
            }
#pragma unroll 1
            for (int b = 0; b < nb; ++b) {
                const Real* gB = sm.gB + b * sm.sl;
                const Real* hB = sm.hB + b * sm.sl;
                const Real g0 = gB[l], h0 = hB[l];
                Real gx[D], hx[D];
#pragma unroll
                for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
#pragma unroll
                for (int k = 0; k < kMaxRegStencil; ++k) {
                    const Real dg = gB[nbi[k]] - g0, dh = hB[nbi[k]] - h0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        gx[q] += ls[k][q] * dg;
                        hx[q] += ls[k][q] * dh;
                    }
                }
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    sm.Gg[b * sm.sg + l * D + q] = gx[q];
                    sm.Gh[b * sm.sg + l * D + q] = hx[q];
                }
            }
        } else {
#pragma unroll 1
            for (int b = 0; b < nb; ++b) {
                const Real* gB = sm.gB + b * sm.sl;
                const Real* hB = sm.hB + b * sm.sl;
                const Real g0 = gB[l], h0 = hB[l];
                Real gx[D], hx[D];
#pragma unroll
                for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
                for (int k = k0; k < k1; ++k) {
                    const int n = __ldg(m.grad_nb + k);
                    const Real dg = gB[n] - g0, dh = hB[n] - h0;
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        const Real lsq = Real(__ldg(m.grad_ls + 3 * k + q));
                        gx[q] += lsq * dg;
                        hx[q] += lsq * dh;
                    }
                }
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    sm.Gg[b * sm.sg + l * D + q] = gx[q];
                    sm.Gh[b * sm.sg + l * D + q] = hx[q];
                }
            }
        }
    }
    __syncthreads();
}

// reconstruction at the half step from local cell l (fvDVM.C:832-836):
// gbar+_l + grad_l . (Cf - C_l - xi dt/2)
template <int D, typename Real, int NB>
__device__ __forceinline__ void recon(const Smem<D, Real, NB>& sm, int b, int l, const double d[3], const Real xi[3],
                                      Real hdt, Real& g, Real& h) {
    Real v[3];
#pragma unroll
    for (int q = 0; q < D; ++q) v[q] = Real(d[q]) - hdt * xi[q];
    Real gg = sm.gB[b * sm.sl + l], hh = sm.hB[b * sm.sl + l];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        gg += sm.Gg[b * sm.sg + l * D + q] * v[q];
        hh += sm.Gh[b * sm.sg + l * D + q] * v[q];
    }
    g = gg;
    h = hh;
}

// ---------------------------------------------------------------------
// Pass A: face reconstruction and raw face moments
// ---------------------------------------------------------------------
template <int D, typename Real, int IPT, int NB>
__global__ void __launch_bounds__(kThreads) k_pass_a(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem<D, Real, NB> sm = carve<D, Real, NB>(smem_raw, a);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    Real* xbg[2] = {reinterpret_cast<Real*>(a.ds.xbg[0]), reinterpret_cast<Real*>(a.ds.xbg[1])};
    Real* xbh[2] = {reinterpret_cast<Real*>(a.ds.xbh[0]), reinterpret_cast<Real*>(a.ds.xbh[1])};
    const Real K3D = Real(m.K + 3 - m.D), Kin = Real(m.K);
    const Real hdt = Real(0.5 * a.dt);
    double acc[IPT][15];
#pragma unroll
    for (int i = 0; i < IPT; ++i)
#pragma unroll
        for (int j = 0; j < 15; ++j) acc[i][j] = 0.0;

    for (int d0 = t.d0; d0 < t.d1; d0 += NB) {
        const int nb = load_batch<D, Real, NB>(m, d0, t.d1, sm);
        stage_ghbar<D, Real, NB, false>(m, a.ds.cellrec, g, h, d0, nb, t, sm, K3D, Kin);
        stage_grad<D, Real, NB>(m, nb, t, sm);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int it = threadIdx.x + k * kThreads;
            if (it >= t.nit) continue;
            const ItemView v = load_item(m.items + t.ioff + it);
#pragma unroll 1
            for (int b = 0; b < nb; ++b) {
                const double xid[3] = {sm.dv[5 * b], sm.dv[5 * b + 1], sm.dv[5 * b + 2]};
                const double wd = sm.dv[5 * b + 3], xi2 = sm.dv[5 * b + 4];
                const Real xi[3] = {Real(xid[0]), Real(xid[1]), Real(xid[2])};
                const double xs = xi_dot_s(xid, v.S);
                if (v.kind == ITEM_MESH_BOUNDARY) {
                    if (xs > 0) {  // outgoing: upwind from the owner (fvDVM.C:916-923, :950-961)
                        Real gg, hh;
                        recon<D, Real, NB>(sm, b, v.lo, v.dO, xi, hdt, gg, hh);
                        accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                        if (v.ptype == DUGKS_PATCH_MAXWELL_WALL) acc[k][MOM_OUT] += wd * xs * double(gg);
                    } else if (v.ptype == DUGKS_PATCH_FAR_FIELD) {
                        // incoming far field: rho_b M(xi; U_owner, T_b) (fvDVM.C:926-938)
                        const BRec* br = a.ds.brec + v.face;
                        const Rec<double> cr = load_rec<double>(a.ds.cellrec + __ldg(m.bface_owner + v.face));
                        const double cx = xid[0] - cr.U[0], cy = xid[1] - cr.U[1], cz = xid[2] - cr.U[2];
                        const double ge = __ldg(&br->rho_in) * __ldg(&br->K_in) *
                                          exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                        const Real gg = Real(ge), hh = Real(ge * __ldg(&br->hfac));
                        accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                    }
                    // incoming maxwellWall DFs enter through rho_w in the face combine
                    continue;
                }
                double co, cn;
                upwind_coeffs(xs, co, cn);
                if (v.kind == ITEM_TILE_INTERNAL) {
                    Real gg = 0, hh = 0, g1, h1;
                    if (co != 0.0) {
                        recon<D, Real, NB>(sm, b, v.lo, v.dO, xi, hdt, g1, h1);
                        gg += Real(co) * g1;
                        hh += Real(co) * h1;
                    }
                    if (cn != 0.0) {
                        recon<D, Real, NB>(sm, b, v.ln, v.dN, xi, hdt, g1, h1);
                        gg += Real(cn) * g1;
                        hh += Real(cn) * h1;
                    }
                    accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                } else {
                    // tile-boundary face: this tile contributes its side only
                    // and hands it to the other tile through XB
                    const bool own_side = v.kind == ITEM_TB_OWN;
                    const double cs = own_side ? co : cn;
                    if (cs != 0.0) {
                        Real g1, h1;
                        if (own_side) recon<D, Real, NB>(sm, b, v.lo, v.dO, xi, hdt, g1, h1);
                        else recon<D, Real, NB>(sm, b, v.ln, v.dN, xi, hdt, g1, h1);
                        g1 *= Real(cs);
                        h1 *= Real(cs);
                        const size_t xi_ = static_cast<size_t>(d0 + b) * m.n_tbf + v.xb_w;
                        xbg[own_side ? 0 : 1][xi_] = g1;
                        xbh[own_side ? 0 : 1][xi_] = h1;
                        accum<D>(acc[k], wd, xid, xi2, double(g1), double(h1));
                    }
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
__global__ void __launch_bounds__(kThreads) k_pass_b(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem<D, Real, NB> sm = carve<D, Real, NB>(smem_raw, a);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    Real* gn = reinterpret_cast<Real*>(a.ds.g[1 - a.ds.cur]);
    Real* hn = reinterpret_cast<Real*>(a.ds.h[1 - a.ds.cur]);
    const Real* xbg[2] = {reinterpret_cast<const Real*>(a.ds.xbg[0]), reinterpret_cast<const Real*>(a.ds.xbg[1])};
    const Real* xbh[2] = {reinterpret_cast<const Real*>(a.ds.xbh[0]), reinterpret_cast<const Real*>(a.ds.xbh[1])};
    const Real K3D = Real(m.K + 3 - m.D), Kin = Real(m.K);
    const Real hdt = Real(0.5 * a.dt);
    const double dt = a.dt;
    double acc[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;

    for (int d0 = t.d0; d0 < t.d1; d0 += NB) {
        const int nb = load_batch<D, Real, NB>(m, d0, t.d1, sm);
        stage_ghbar<D, Real, NB, true>(m, a.ds.cellrec, g, h, d0, nb, t, sm, K3D, Kin);
        stage_grad<D, Real, NB>(m, nb, t, sm);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int it = threadIdx.x + k * kThreads;
            if (it >= t.nit) continue;
            const ItemView v = load_item(m.items + t.ioff + it);
            const bool boundary = v.kind == ITEM_MESH_BOUNDARY;
            const Rec<Real> fr = load_rec<Real>(a.ds.facerec + (boundary ? m.nIF + v.face : v.face));
#pragma unroll 1
            for (int b = 0; b < nb; ++b) {
                const double xid[3] = {sm.dv[5 * b], sm.dv[5 * b + 1], sm.dv[5 * b + 2]};
                const Real xi[3] = {Real(xid[0]), Real(xid[1]), Real(xid[2])};
                const double xs = xi_dot_s(xid, v.S);
                Real gf, hf;
                if (boundary) {
                    if (xs > 0) {
                        // outgoing: reconstruct and relax with the boundary face
                        // coefficients; h uses the internal-face T at the
                        // patch-local index (fvDVM.C:1367, :1413, :1429-1444)
                        Real gg, hh, gS, hS;
                        recon<D, Real, NB>(sm, b, v.lo, v.dO, xi, hdt, gg, hh);
                        shakhov<D, Real>(xi, fr, K3D, Kin, gS, hS);
                        gf = gg + fr.r * (gS - gg);
                        hf = hh + fr.r * (hS - hh);
                    } else {
                        // incoming, never relaxed: wall rho_w M(U_w,T_w)
                        // (fvDVM.C:1079-1092), far field rho_b M(U_owner,T_b)
                        const BRec* br = a.ds.brec + v.face;
                        double Ui[3];
                        if (v.ptype == DUGKS_PATCH_FAR_FIELD) {
                            const Rec<double> cr = load_rec<double>(a.ds.cellrec + __ldg(m.bface_owner + v.face));
                            Ui[0] = cr.U[0];
                            Ui[1] = cr.U[1];
                            Ui[2] = cr.U[2];
                        } else {
                            Ui[0] = __ldg(&br->U[0]);
                            Ui[1] = __ldg(&br->U[1]);
                            Ui[2] = __ldg(&br->U[2]);
                        }
                        const double cx = xid[0] - Ui[0], cy = xid[1] - Ui[1], cz = xid[2] - Ui[2];
                        const double ge = br->rho_in * __ldg(&br->K_in) *
                                          exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                        gf = Real(ge);
                        hf = Real(ge * __ldg(&br->hfac));
                    }
                } else {
                    double co, cn;
                    upwind_coeffs(xs, co, cn);
                    Real gg = 0, hh = 0, g1, h1;
                    const size_t xr = static_cast<size_t>(d0 + b) * m.n_tbf + v.xb_r;
                    if (co != 0.0) {
                        if (v.kind != ITEM_TB_NEI) {
                            recon<D, Real, NB>(sm, b, v.lo, v.dO, xi, hdt, g1, h1);
                            gg += Real(co) * g1;
                            hh += Real(co) * h1;
                        } else {
                            gg += xbg[0][xr];
                            hh += xbh[0][xr];
                        }
                    }
                    if (cn != 0.0) {
                        if (v.kind != ITEM_TB_OWN) {
                            recon<D, Real, NB>(sm, b, v.ln, v.dN, xi, hdt, g1, h1);
                            gg += Real(cn) * g1;
                            hh += Real(cn) * h1;
                        } else {
                            gg += xbg[1][xr];
                            hh += xbh[1][xr];
                        }
                    }
                    Real gS, hS;
                    shakhov<D, Real>(xi, fr, K3D, Kin, gS, hS);
                    gf = gg + fr.r * (gS - gg);
                    hf = hh + fr.r * (hS - hh);
                }
                const Real xsr = Real(xs);
                sm.Fg[b * sm.si + it] = xsr * gf;
                sm.Fh[b * sm.si + it] = xsr * hf;
            }
        }
        __syncthreads();
        // volume update of the L0 cells:
        // g~ <- -g~/3 + 4/3 gbar+ - dt/V sum_f (+-)(xi.S) g_f
        for (int l = threadIdx.x; l < t.n0; l += kThreads) {
            const int c = t.b + l;
            const int k0 = __ldg(m.cf_off + c), k1 = __ldg(m.cf_off + c + 1);
            Real sg[NB], sh[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) sg[b] = sh[b] = Real(0);
            for (int k = k0; k < k1; ++k) {
                const int e = __ldg(m.cf_item + k);
                const int it = (e > 0 ? e : -e) - 1;
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    if (b < nb) {
                        const Real fg = sm.Fg[b * sm.si + it], fh = sm.Fh[b * sm.si + it];
                        sg[b] += e > 0 ? fg : -fg;
                        sh[b] += e > 0 ? fh : -fh;
                    }
                }
            }
            const Real dtV = Real(dt * __ldg(m.dtV + c));
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                if (b < nb) {
                    const Real g_new = Real(-1.0 / 3) * sm.gT[b * sm.s0 + l] + Real(4.0 / 3) * sm.gB[b * sm.sl + l] +
                                       sg[b] * dtV;
                    const Real h_new = Real(-1.0 / 3) * sm.hT[b * sm.s0 + l] + Real(4.0 / 3) * sm.hB[b * sm.sl + l] +
                                       sh[b] * dtV;
                    const size_t idx = static_cast<size_t>(d0 + b) * m.nC + c;
                    gn[idx] = g_new;
                    hn[idx] = h_new;
                    const double xid[3] = {sm.dv[5 * b], sm.dv[5 * b + 1], sm.dv[5 * b + 2]};
                    accum<D>(acc, sm.dv[5 * b + 3], xid, sm.dv[5 * b + 4], double(g_new), double(h_new));
                }
            }
        }
    }
    // tiles have at most kThreads cells: one cell per thread
    if (static_cast<int>(threadIdx.x) < t.n0) {
        double* p = a.ds.partC + (static_cast<size_t>(blockIdx.y) * m.nC + t.b + threadIdx.x) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) p[j] = acc[j];
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
        case 4: launch_pass_t<D, Real, 4>(a, pass_b, s); break;
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
        case 4: return configure_t<D, Real, 4>(smemA, smemB);
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

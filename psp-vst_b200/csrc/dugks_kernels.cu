// DUGKS step kernels for sm_100a.
//
// One fvDVM::evolution() (src/fvDVM/fvDVM/fvDVM.C:2128-2174) is four
// kernel stages:
//   pass A  (tile x DV-chunk)  gbar+ half step, least-squares gradient,
//           upwind face reconstruction, raw face moments, wall out-flux;
//           writes the reconstruction at tile-boundary faces (XB buffer)
//   face combine (internal, then boundary faces)  face macros rho,U,T,q,tau,
//           wall density, face relaxation coefficients
//   pass B  (tile x DV-chunk)  gbar+ and gradient again, face relaxation,
//           flux gather, g~/h~ update, raw cell moments
//   cell combine  cell macros and the next step's cell coefficients
// The state g~, h~ is DV-major [dv][cell] (each DV a contiguous row of
// cells, cells renumbered along a Morton curve), double-buffered between
// steps because pass B reads neighbour tiles' cells while they are written.
#include <cstdio>

#include "dugks_kernels.cuh"

namespace dugks {

namespace {

struct Consts {
    double dt, Pr1, K3D, Kin, R, omega, Tref, muRef, Pr;
    int D;
};

inline Consts make_consts(const DevMesh& m, double dt) {
    Consts k;
    k.dt = dt;
    k.Pr1 = 1.0 - m.Pr;
    k.K3D = m.K + 3.0 - m.D;
    k.Kin = m.K;
    k.R = m.R;
    k.omega = m.omega;
    k.Tref = m.Tref;
    k.muRef = m.muRef;
    k.Pr = m.Pr;
    k.D = m.D;
    return k;
}

template <typename Real>
struct RealOps;
template <>
struct RealOps<double> {
    __device__ static __forceinline__ double ex(double x) { return exp(x); }
};
template <>
struct RealOps<float> {
    __device__ static __forceinline__ float ex(float x) { return expf(x); }
};

// Coefficient record of a Shakhov equilibrium, in the working precision.
template <typename Real>
struct Rec {
    Real U[3], invRT, A, r, qv[3], RTh;
};

template <typename Real>
__device__ __forceinline__ Rec<Real> load_rec(const CellRec* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4);
    Rec<Real> r;
    r.U[0] = Real(a.x);
    r.U[1] = Real(a.y);
    r.U[2] = Real(b.x);
    r.invRT = Real(b.y);
    r.A = Real(c.x);
    r.r = Real(c.y);
    r.qv[0] = Real(d.x);
    r.qv[1] = Real(d.y);
    r.qv[2] = Real(e.x);
    r.RTh = Real(e.y);
    return r;
}

// Shakhov equilibrium pair at velocity xi (fvDVM.C:673-679,
// discreteVelocity.C:997-1007):
//   gS = A e^{-cs/2} (1 + s (cs - D - 2)),
//   hS = A e^{-cs/2} RT ((K+3-D) + s ((cs - D)(K+3-D) - 2K)),
// cs = |xi-U|^2/RT, s = (xi-U).q (1-Pr)/(5 rho RT^2).
template <int D, typename Real>
__device__ __forceinline__ void shakhov(const Real xi[3], const Rec<Real>& r, Real K3D, Real Kin, Real& gS,
                                        Real& hS) {
    const Real cx = xi[0] - r.U[0], cy = xi[1] - r.U[1];
    const Real cz = D == 3 ? xi[2] - r.U[2] : Real(0);
    const Real cs = (cx * cx + cy * cy + cz * cz) * r.invRT;
    const Real s = cx * r.qv[0] + cy * r.qv[1] + (D == 3 ? cz * r.qv[2] : Real(0));
    const Real E = r.A * RealOps<Real>::ex(Real(-0.5) * cs);
    gS = E * (Real(1) + s * (cs - Real(D + 2)));
    hS = E * r.RTh * (K3D + s * ((cs - Real(D)) * K3D - Real(2) * Kin));
}

// raw moments of one (g, h) pair with weight w (layout in dugks_internal.h)
template <int D>
__device__ __forceinline__ void accum(double* acc, double w, const double xi[3], double xi2, double g, double h) {
    const double a = w * g, b = w * h;
    const double u = fma(a, xi2, b);
    acc[MOM_M0] += a;
    acc[MOM_M1 + 0] = fma(a, xi[0], acc[MOM_M1 + 0]);
    acc[MOM_M1 + 1] = fma(a, xi[1], acc[MOM_M1 + 1]);
    acc[MOM_W] += u;
    acc[MOM_V3 + 0] = fma(u, xi[0], acc[MOM_V3 + 0]);
    acc[MOM_V3 + 1] = fma(u, xi[1], acc[MOM_V3 + 1]);
    const double ax = a * xi[0], ay = a * xi[1];
    acc[MOM_M2 + 0] = fma(ax, xi[0], acc[MOM_M2 + 0]);
    acc[MOM_M2 + 1] = fma(ax, xi[1], acc[MOM_M2 + 1]);
    acc[MOM_M2 + 3] = fma(ay, xi[1], acc[MOM_M2 + 3]);
    if (D == 3) {
        acc[MOM_M1 + 2] = fma(a, xi[2], acc[MOM_M1 + 2]);
        acc[MOM_V3 + 2] = fma(u, xi[2], acc[MOM_V3 + 2]);
        const double az = a * xi[2];
        acc[MOM_M2 + 2] = fma(ax, xi[2], acc[MOM_M2 + 2]);
        acc[MOM_M2 + 4] = fma(ay, xi[2], acc[MOM_M2 + 4]);
        acc[MOM_M2 + 5] = fma(az, xi[2], acc[MOM_M2 + 5]);
    }
}

// Macros of a raw moment record, FP64 for every storage precision:
// rho = M0, U = M1/rho, T = (W/2 - rho|U|^2/2)/((K+3)/2 R rho)
// (fvDVM.C:1249-1251, :1683-1684), tau (fvDVM.C:1831), and the heat flux
// 1/2 sum w c (|c|^2 g + h), c = xi - U (fvDVM.C:1273-1297, :1702-1715),
// expanded in raw moments: 1/2 [V3 - 2 M2.U - U W + 2 rho |U|^2 U].
__device__ __forceinline__ void macros_from_moments(const double* s, const Consts& k, double& rho, double U[3],
                                                    double& T, double q[3], double& tau) {
    rho = s[MOM_M0];
    for (int i = 0; i < 3; ++i) U[i] = s[MOM_M1 + i] / rho;
    const double u2 = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
    const double rE = 0.5 * s[MOM_W];
    T = (rE - 0.5 * rho * u2) / ((k.Kin + 3.0) / 2.0 * k.R * rho);
    tau = k.muRef * exp(k.omega * log(T / k.Tref)) / rho / T / k.R;
    const double* M2 = s + MOM_M2;
    const double M2U[3] = {M2[0] * U[0] + M2[1] * U[1] + M2[2] * U[2], M2[1] * U[0] + M2[3] * U[1] + M2[4] * U[2],
                           M2[2] * U[0] + M2[4] * U[1] + M2[5] * U[2]};
    for (int i = 0; i < 3; ++i)
        q[i] = 0.5 * (s[MOM_V3 + i] - 2.0 * M2U[i] - U[i] * s[MOM_W] + 2.0 * rho * u2 * U[i]);
}

__device__ __forceinline__ double inv_norm(double RT, int D) {  // (2 pi R T)^(-D/2)
    const double t = 2.0 * 3.14159265358979323846 * RT;
    return D == 3 ? 1.0 / (t * sqrt(t)) : (D == 2 ? 1.0 / t : 1.0 / sqrt(t));
}

struct ItemView {
    int kind, lo, ln, face, xb_w, xb_r, ptype;
    double S[3], dO[3], dN[3];
};

__device__ __forceinline__ ItemView load_item(const Item* p) {
    ItemView v;
    const int4* ip = reinterpret_cast<const int4*>(p);
    const int4 i0 = __ldg(ip), i1 = __ldg(ip + 1);
    v.kind = i0.x;
    v.lo = i0.y;
    v.ln = i0.z;
    v.face = i0.w;
    v.xb_w = i1.x;
    v.xb_r = i1.y;
    v.ptype = i1.z;
    const double2* dp = reinterpret_cast<const double2*>(p) + 2;
    const double2 a = __ldg(dp), b = __ldg(dp + 1), c = __ldg(dp + 2), d = __ldg(dp + 3), e = __ldg(dp + 4);
    v.S[0] = a.x;
    v.S[1] = a.y;
    v.S[2] = b.x;
    v.dO[0] = b.y;
    v.dO[1] = c.x;
    v.dO[2] = c.y;
    v.dN[0] = d.x;
    v.dN[1] = d.y;
    v.dN[2] = e.x;
    return v;
}

// upwind weights of the owner and neighbour reconstructions at an internal
// face (fvDVM.C:829-863): owner if xi.S >= VSMALL, neighbour if < -VSMALL,
// the average otherwise
__device__ __forceinline__ void upwind_coeffs(double xs, double& co, double& cn) {
    if (xs >= kVSmall) {
        co = 1.0;
        cn = 0.0;
    } else if (xs < -kVSmall) {
        co = 0.0;
        cn = 1.0;
    } else {
        co = 0.5;
        cn = 0.5;
    }
}

template <typename Real, int D>
struct Smem {
    Real *gB, *hB, *Gg, *Gh, *Fg, *Fh, *gT, *hT;
};

template <typename Real, int D>
__device__ __forceinline__ Smem<Real, D> carve(void* base, int max_local, int max_l0, int max_items) {
    Smem<Real, D> s;
    Real* p = reinterpret_cast<Real*>(base);
    s.gB = p;
    p += max_local;
    s.hB = p;
    p += max_local;
    s.Gg = p;
    p += max_l0 * D;
    s.Gh = p;
    p += max_l0 * D;
    s.Fg = p;
    p += max_items;
    s.Fh = p;
    p += max_items;
    s.gT = p;
    p += max_l0;
    s.hT = p;
    return s;
}

// reconstruction at the half step from local cell l along d - xi dt/2
// (fvDVM.C:832-836): gbar+_l + grad_l . (Cf - C_l - xi dt/2)
template <int D, typename Real>
__device__ __forceinline__ void recon(const Smem<Real, D>& sm, int l, const double d[3], const Real xi[3], Real hdt,
                                      Real& g, Real& h) {
    Real v[3];
    for (int q = 0; q < D; ++q) v[q] = Real(d[q]) - hdt * xi[q];
    Real gg = sm.gB[l], hh = sm.hB[l];
#pragma unroll
    for (int q = 0; q < D; ++q) {
        gg += sm.Gg[l * D + q] * v[q];
        hh += sm.Gh[l * D + q] * v[q];
    }
    g = gg;
    h = hh;
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

// Stages 1-2 of both passes: gbar+/hbar+ at the tile's L0+L1 cells
// (updateGHbarPvol, fvDVM.C:648-683) into shared memory, then the
// least-squares gradients at the L0 cells (leastSquaresGrad; the boundary
// faces add lsB * (patch value - cell value) = 0 because the fixedGradient
// patches of gBarPvol keep a zero gradient, fvDVM.C:456-485, :775-809).
template <int D, typename Real, bool KEEP>
__device__ __forceinline__ void stage_ghbar_grad(const DevMesh& m, const CellRec* __restrict__ crec,
                                                 const Real* __restrict__ g, const Real* __restrict__ h, int d,
                                                 const Real xi[3], Real K3D, Real Kin, const TileRange& t,
                                                 const Smem<Real, D>& sm) {
    const size_t row = static_cast<size_t>(d) * m.nC;
    for (int l = threadIdx.x; l < t.nloc; l += kThreads) {
        const int c = __ldg(m.loc_cells + t.loff + l);
        const Rec<Real> r = load_rec<Real>(crec + c);
        const Real gt = g[row + c], ht = h[row + c];
        Real gS, hS;
        shakhov<D, Real>(xi, r, K3D, Kin, gS, hS);
        sm.gB[l] = gt + r.r * (gS - gt);
        sm.hB[l] = ht + r.r * (hS - ht);
        if (KEEP && l < t.n0) {
            sm.gT[l] = gt;
            sm.hT[l] = ht;
        }
    }
    __syncthreads();
    for (int l = threadIdx.x; l < t.n0; l += kThreads) {
        const int c = t.b + l;
        const int k0 = __ldg(m.grad_off + c), k1 = __ldg(m.grad_off + c + 1);
        const Real g0 = sm.gB[l], h0 = sm.hB[l];
        Real gx[3] = {0, 0, 0}, hx[3] = {0, 0, 0};
        for (int k = k0; k < k1; ++k) {
            const int nb = __ldg(m.grad_nb + k);
            const Real dg = sm.gB[nb] - g0, dh = sm.hB[nb] - h0;
#pragma unroll
            for (int q = 0; q < D; ++q) {
                const Real ls = Real(__ldg(m.grad_ls + 3 * k + q));
                gx[q] += ls * dg;
                hx[q] += ls * dh;
            }
        }
#pragma unroll
        for (int q = 0; q < D; ++q) {
            sm.Gg[l * D + q] = gx[q];
            sm.Gh[l * D + q] = hx[q];
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------
// Pass A: face reconstruction and raw face moments
// (updateGHbarSurf fvDVM.C:755-1029 and updateMacroSurf :1181-1297)
// ---------------------------------------------------------------------
template <int D, typename Real, int IPT>
__global__ void __launch_bounds__(kThreads) k_pass_a(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem<Real, D> sm = carve<Real, D>(smem_raw, a.dims_local, a.dims_l0, a.dims_items);
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

    for (int d = t.d0; d < t.d1; ++d) {
        const double xid[3] = {__ldg(m.xi + 3 * d), __ldg(m.xi + 3 * d + 1), __ldg(m.xi + 3 * d + 2)};
        const double wd = __ldg(m.w + d);
        const double xi2 = xid[0] * xid[0] + xid[1] * xid[1] + xid[2] * xid[2];
        const Real xi[3] = {Real(xid[0]), Real(xid[1]), Real(xid[2])};
        stage_ghbar_grad<D, Real, false>(m, a.ds.cellrec, g, h, d, xi, K3D, Kin, t, sm);
        const size_t xrow = static_cast<size_t>(d) * m.n_tbf;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int it = threadIdx.x + k * kThreads;
            if (it >= t.nit) continue;
            const ItemView v = load_item(m.items + t.ioff + it);
            const double xs = xid[0] * v.S[0] + xid[1] * v.S[1] + xid[2] * v.S[2];
            if (v.kind == ITEM_MESH_BOUNDARY) {
                if (xs > 0) {  // outgoing: upwind from the owner (fvDVM.C:916-923, :950-961)
                    Real gg, hh;
                    recon<D, Real>(sm, v.lo, v.dO, xi, hdt, gg, hh);
                    accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
                    if (v.ptype == DUGKS_PATCH_MAXWELL_WALL) acc[k][MOM_OUT] += wd * xs * double(gg);
                } else if (v.ptype == DUGKS_PATCH_FAR_FIELD) {
                    // incoming far field: rho_b M(xi; U_owner, T_b) (fvDVM.C:926-938)
                    const BRec* br = a.ds.brec + v.face;
                    const int own = __ldg(m.bface_owner + v.face);
                    const Rec<double> cr = load_rec<double>(a.ds.cellrec + own);
                    const double cx = xid[0] - cr.U[0], cy = xid[1] - cr.U[1], cz = xid[2] - cr.U[2];
                    const double ge = __ldg(&br->rho_in) * __ldg(&br->K_in) *
                                      exp(-0.5 * (cx * cx + cy * cy + cz * cz) * __ldg(&br->invRT_in));
                    const Real gg = Real(ge);
                    const Real hh = Real(ge * __ldg(&br->hfac));
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
                    recon<D, Real>(sm, v.lo, v.dO, xi, hdt, g1, h1);
                    gg += Real(co) * g1;
                    hh += Real(co) * h1;
                }
                if (cn != 0.0) {
                    recon<D, Real>(sm, v.ln, v.dN, xi, hdt, g1, h1);
                    gg += Real(cn) * g1;
                    hh += Real(cn) * h1;
                }
                accum<D>(acc[k], wd, xid, xi2, double(gg), double(hh));
            } else {
                // tile-boundary face: this tile contributes its side only and
                // hands the value to the other tile through XB
                const bool own_side = v.kind == ITEM_TB_OWN;
                const double cs = own_side ? co : cn;
                if (cs != 0.0) {
                    Real g1, h1;
                    if (own_side) recon<D, Real>(sm, v.lo, v.dO, xi, hdt, g1, h1);
                    else recon<D, Real>(sm, v.ln, v.dN, xi, hdt, g1, h1);
                    g1 *= Real(cs);
                    h1 *= Real(cs);
                    const int side = own_side ? 0 : 1;
                    xbg[side][xrow + v.xb_w] = g1;
                    xbh[side][xrow + v.xb_w] = h1;
                    accum<D>(acc[k], wd, xid, xi2, double(g1), double(h1));
                }
            }
        }
        __syncthreads();
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
// Pass B: face relaxation (updateGHsurf fvDVM.C:1362-1457), volume update
// (updateGHtildeVol :1462-1519) and raw cell moments (updateMacroVol
// :1528-1554, :1702-1715)
// ---------------------------------------------------------------------
template <int D, typename Real, int IPT>
__global__ void __launch_bounds__(kThreads) k_pass_b(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem<Real, D> sm = carve<Real, D>(smem_raw, a.dims_local, a.dims_l0, a.dims_items);
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
    constexpr int CPT = 1;  // L0 cells per thread (tiles have at most kThreads cells)
    double acc[CPT][15];
#pragma unroll
    for (int i = 0; i < CPT; ++i)
#pragma unroll
        for (int j = 0; j < 15; ++j) acc[i][j] = 0.0;

    for (int d = t.d0; d < t.d1; ++d) {
        const double xid[3] = {__ldg(m.xi + 3 * d), __ldg(m.xi + 3 * d + 1), __ldg(m.xi + 3 * d + 2)};
        const double wd = __ldg(m.w + d);
        const double xi2 = xid[0] * xid[0] + xid[1] * xid[1] + xid[2] * xid[2];
        const Real xi[3] = {Real(xid[0]), Real(xid[1]), Real(xid[2])};
        stage_ghbar_grad<D, Real, true>(m, a.ds.cellrec, g, h, d, xi, K3D, Kin, t, sm);
        const size_t xrow = static_cast<size_t>(d) * m.n_tbf;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int it = threadIdx.x + k * kThreads;
            if (it >= t.nit) continue;
            const ItemView v = load_item(m.items + t.ioff + it);
            const double xs = xid[0] * v.S[0] + xid[1] * v.S[1] + xid[2] * v.S[2];
            Real gf, hf;
            if (v.kind == ITEM_MESH_BOUNDARY) {
                const BRec* br = a.ds.brec + v.face;
                if (xs > 0) {
                    // outgoing: reconstruct and relax with the boundary face
                    // coefficients; h uses the internal-face T at the
                    // patch-local index (fvDVM.C:1367, :1413, :1429-1444)
                    Real gg, hh;
                    recon<D, Real>(sm, v.lo, v.dO, xi, hdt, gg, hh);
                    const Rec<Real> fr = load_rec<Real>(reinterpret_cast<const CellRec*>(a.ds.facerec + m.nIF + v.face));
                    Real gS, hS;
                    shakhov<D, Real>(xi, fr, K3D, Kin, gS, hS);
                    gf = gg + fr.r * (gS - gg);
                    hf = hh + fr.r * (hS - hh);
                } else {
                    // incoming, never relaxed: wall rho_w M(U_w,T_w)
                    // (fvDVM.C:1079-1092) or far field rho_b M(U_owner,T_b)
                    const double* Ui;
                    Rec<double> cr;
                    if (v.ptype == DUGKS_PATCH_FAR_FIELD) {
                        cr = load_rec<double>(a.ds.cellrec + __ldg(m.bface_owner + v.face));
                        Ui = cr.U;
                    } else {
                        Ui = br->U;
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
                const bool own_in = v.kind != ITEM_TB_NEI;
                const bool nei_in = v.kind != ITEM_TB_OWN;
                if (co != 0.0) {
                    if (own_in) {
                        recon<D, Real>(sm, v.lo, v.dO, xi, hdt, g1, h1);
                        gg += Real(co) * g1;
                        hh += Real(co) * h1;
                    } else {
                        gg += xbg[0][xrow + v.xb_r];
                        hh += xbh[0][xrow + v.xb_r];
                    }
                }
                if (cn != 0.0) {
                    if (nei_in) {
                        recon<D, Real>(sm, v.ln, v.dN, xi, hdt, g1, h1);
                        gg += Real(cn) * g1;
                        hh += Real(cn) * h1;
                    } else {
                        gg += xbg[1][xrow + v.xb_r];
                        hh += xbh[1][xrow + v.xb_r];
                    }
                }
                const Rec<Real> fr = load_rec<Real>(reinterpret_cast<const CellRec*>(a.ds.facerec + v.face));
                Real gS, hS;
                shakhov<D, Real>(xi, fr, K3D, Kin, gS, hS);
                gf = gg + fr.r * (gS - gg);
                hf = hh + fr.r * (hS - hh);
            }
            const Real xsr = Real(xs);
            sm.Fg[it] = xsr * gf;
            sm.Fh[it] = xsr * hf;
        }
        __syncthreads();
        // volume update of the L0 cells: g~ <- -g~/3 + 4/3 gbar+ - dt/V sum_f (+-)(xi.S) g_f
        for (int l = threadIdx.x; l < t.n0; l += kThreads) {
            const int c = t.b + l;
            const int k0 = __ldg(m.cf_off + c), k1 = __ldg(m.cf_off + c + 1);
            Real sg = 0, sh = 0;
            for (int k = k0; k < k1; ++k) {
                const int e = __ldg(m.cf_item + k);
                const int it = (e > 0 ? e : -e) - 1;
                if (e > 0) {
                    sg += sm.Fg[it];
                    sh += sm.Fh[it];
                } else {
                    sg -= sm.Fg[it];
                    sh -= sm.Fh[it];
                }
            }
            const Real dtV = Real(dt * __ldg(m.dtV + c));
            const Real g_new = Real(-1.0 / 3) * sm.gT[l] + Real(4.0 / 3) * sm.gB[l] + sg * dtV;
            const Real h_new = Real(-1.0 / 3) * sm.hT[l] + Real(4.0 / 3) * sm.hB[l] + sh * dtV;
            const size_t idx = static_cast<size_t>(d) * m.nC + c;
            gn[idx] = g_new;
            hn[idx] = h_new;
            accum<D>(acc[0], wd, xid, xi2, double(g_new), double(h_new));
        }
        __syncthreads();
    }
    for (int l = threadIdx.x; l < t.n0; l += kThreads) {
        double* p = a.ds.partC + (static_cast<size_t>(blockIdx.y) * m.nC + t.b + l) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) p[j] = acc[0][j];
    }
}

// ---------------------------------------------------------------------
// Face combine: sums the DV-chunk partials of a face, adds the incoming
// wall DFs through rho_w, and forms the face macros and the face
// relaxation coefficients (updateMaxwellWallRho fvDVM.C:1032-1052,
// calculatedMaxwellFvPatchField.C:140-164, updateMacroSurf :1248-1300).
// ---------------------------------------------------------------------
__device__ __forceinline__ void sum_face_partials(const StepArgs& a, int f, double* s) {
    const DevMesh& m = a.dm;
    for (int j = 0; j < 15; ++j) s[j] = 0.0;
    const int i0 = __ldg(m.face_items + 2 * f), i1 = __ldg(m.face_items + 2 * f + 1);
    for (int ch = 0; ch < a.chunks; ++ch) {
        const double* p0 = a.ds.partF + (static_cast<size_t>(ch) * m.n_items + i0) * kNM;
        for (int j = 0; j < 15; ++j) s[j] += p0[j];
        if (i1 >= 0) {
            const double* p1 = a.ds.partF + (static_cast<size_t>(ch) * m.n_items + i1) * kNM;
            for (int j = 0; j < 15; ++j) s[j] += p1[j];
        }
    }
}

__device__ __forceinline__ void write_face(const StepArgs& a, const Consts& k, int f, const double* s, double RTh_T,
                                           bool use_RTh_T) {
    double rho, U[3], T, q[3], tau;
    macros_from_moments(s, k, rho, U, T, q, tau);
    const double fac = 2.0 * tau / (2.0 * tau + 0.5 * k.dt * k.Pr);  // fvDVM.C:1300
    for (int i = 0; i < 3; ++i) q[i] *= fac;
    double* fm = a.ds.fm + static_cast<size_t>(f) * 9;
    fm[0] = rho;
    fm[1] = U[0];
    fm[2] = U[1];
    fm[3] = U[2];
    fm[4] = T;
    fm[5] = q[0];
    fm[6] = q[1];
    fm[7] = q[2];
    fm[8] = tau;
    const double RT = k.R * T;
    FaceRec fr;
    fr.U[0] = U[0];
    fr.U[1] = U[1];
    fr.U[2] = U[2];
    fr.invRT = 1.0 / RT;
    fr.A = rho * inv_norm(RT, k.D);
    fr.r = 0.5 * k.dt / (2.0 * tau + 0.5 * k.dt);
    const double qs = k.Pr1 / (5.0 * rho * RT * RT);
    fr.qv[0] = q[0] * qs;
    fr.qv[1] = q[1] * qs;
    fr.qv[2] = q[2] * qs;
    fr.RTh = use_RTh_T ? k.R * RTh_T : RT;
    a.ds.facerec[f] = fr;
}

__global__ void k_face_combine_internal(const StepArgs a, const Consts k) {
    const DevMesh& m = a.dm;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    double co = 0.0;
    bool valid = false;
    if (f < m.nIF) {
        double s[15];
        sum_face_partials(a, f, s);
        write_face(a, k, f, s, 0.0, false);
        const double* fm = a.ds.fm + static_cast<size_t>(f) * 9;
        const double umag = sqrt(fm[1] * fm[1] + fm[2] * fm[2] + fm[3] * fm[3]);
        co = __ldg(m.dc + f) * (umag + m.xi_max_co);  // getCoNum, fvDVM.C:2180-2182
        valid = true;
    }
    // block max and sum of the Courant numbers (per dt)
    __shared__ double smax[32], ssum[32];
    double vmax = valid ? co : 0.0, vsum = valid ? co : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
        vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        vsum += __shfl_xor_sync(0xffffffffu, vsum, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        smax[wid] = vmax;
        ssum[wid] = vsum;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        vmax = lane < nw ? smax[lane] : 0.0;
        vsum = lane < nw ? ssum[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
            vsum += __shfl_xor_sync(0xffffffffu, vsum, o);
        }
        if (lane == 0) {
            // positive doubles order like their bit patterns
            atomicMax(reinterpret_cast<unsigned long long*>(a.ds.co), __double_as_longlong(vmax));
            atomicAdd(a.ds.co + 1, vsum);
        }
    }
}

__global__ void k_face_combine_boundary(const StepArgs a, const Consts k) {
    const DevMesh& m = a.dm;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.nBF) return;
    const int f = m.nIF + b;
    double s[15];
    sum_face_partials(a, f, s);
    const int ptype = __ldg(m.bface_ptype + b);
    BRec* br = a.ds.brec + b;
    if (ptype == DUGKS_PATCH_MAXWELL_WALL) {
        // rho_w = outGoing / |inComingByRho|; outGoing restarts from zero
        const double rho_w = s[MOM_OUT] / fabs(br->inByRho);
        br->rho_in = rho_w;
        const double* mi = a.ds.bmom_in + static_cast<size_t>(b) * kNM;
        for (int j = 0; j < 14; ++j) s[j] += rho_w * mi[j];
    }
    const int li = __ldg(m.bface_patch_local + b);
    const double Tint = li < m.nIF ? a.ds.fm[static_cast<size_t>(li) * 9 + 4] : 0.0;
    write_face(a, k, f, s, Tint, li < m.nIF);
}

// ---------------------------------------------------------------------
// Cell combine: cell macros (updateMacroVol, fvDVM.C:1682-1742) and the
// cell coefficient records of the next half step.
// ---------------------------------------------------------------------
__device__ __forceinline__ void write_cellrec(const StepArgs& a, const Consts& k, int c, double rho, const double U[3],
                                              double T, const double q[3], double tau, double dt_next) {
    const double RT = k.R * T;
    CellRec cr;
    cr.U[0] = U[0];
    cr.U[1] = U[1];
    cr.U[2] = U[2];
    cr.invRT = 1.0 / RT;
    cr.A = rho * inv_norm(RT, k.D);
    cr.r = dt_next > 0 ? 1.5 * dt_next / (2.0 * tau + dt_next) : 0.0;  // relax factor, fvDVM.C:668
    const double qs = k.Pr1 / (5.0 * rho * RT * RT);
    cr.qv[0] = q[0] * qs;
    cr.qv[1] = q[1] * qs;
    cr.qv[2] = q[2] * qs;
    cr.RT = RT;
    a.ds.cellrec[c] = cr;
}

__global__ void k_cell_combine(const StepArgs a, const Consts k, double dt_next) {
    const DevMesh& m = a.dm;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nC) return;
    double s[15];
    for (int j = 0; j < 15; ++j) s[j] = 0.0;
    for (int ch = 0; ch < a.chunks; ++ch) {
        const double* p = a.ds.partC + (static_cast<size_t>(ch) * m.nC + c) * kNM;
        for (int j = 0; j < 14; ++j) s[j] += p[j];
    }
    double rho, U[3], T, q[3], tau;
    macros_from_moments(s, k, rho, U, T, q, tau);
    const double fac = 2.0 * tau / (2.0 * tau + k.dt * k.Pr);  // fvDVM.C:1742
    for (int i = 0; i < 3; ++i) q[i] *= fac;
    if (!(rho > 0.0) || !(T > 0.0) || !isfinite(rho + T + U[0] + U[1] + U[2])) atomicOr(a.ds.err, 1);
    double* cm = a.ds.cm + static_cast<size_t>(c) * 9;
    cm[0] = rho;
    cm[1] = U[0];
    cm[2] = U[1];
    cm[3] = U[2];
    cm[4] = T;
    cm[5] = q[0];
    cm[6] = q[1];
    cm[7] = q[2];
    cm[8] = tau;
    write_cellrec(a, k, c, rho, U, T, q, tau, dt_next);
}

// relax factor of the cell records for a time step (when the records were
// written without knowing it)
__global__ void k_cell_prep(const StepArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.dm.nC) return;
    const double tau = a.ds.cm[static_cast<size_t>(c) * 9 + 8];
    a.ds.cellrec[c].r = 1.5 * a.dt / (2.0 * tau + a.dt);
}

// initial Maxwellian state (fvDVM.C:414-426), DV-major
template <typename Real>
__global__ void k_init_state(const StepArgs a) {
    const DevMesh& m = a.dm;
    const size_t n = static_cast<size_t>(m.nv) * m.nC;
    const double K3D = m.K + 3.0 - m.D;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int d = static_cast<int>(i / m.nC), c = static_cast<int>(i % m.nC);
        const double* cm = a.ds.cm + static_cast<size_t>(c) * 9;
        const double RT = m.R * cm[4];
        const double cx = cm[1] - m.xi[3 * d], cy = cm[2] - m.xi[3 * d + 1], cz = cm[3] - m.xi[3 * d + 2];
        const double ge = cm[0] * inv_norm(RT, m.D) * exp(-0.5 * (cx * cx + cy * cy + cz * cz) / RT);
        reinterpret_cast<Real*>(a.ds.g[a.ds.cur])[i] = Real(ge);
        reinterpret_cast<Real*>(a.ds.h[a.ds.cur])[i] = Real(K3D * ge * RT);
    }
}

// wall: inComingByRho_f = sum_{xi.S<0} -w (xi.S) M/rho (fvDVM.C:598-617) and
// the raw moments of the incoming wall DFs per unit rho_w
// (xi.S <= 0, fvDVM.C:1079-1092)
__global__ void k_init_wall(const StepArgs a) {
    const DevMesh& m = a.dm;
    const int b = blockIdx.x;
    if (b >= m.nBF || m.bface_ptype[b] != DUGKS_PATCH_MAXWELL_WALL) return;
    BRec* br = a.ds.brec + b;
    const double Sx = m.bS[3 * b], Sy = m.bS[3 * b + 1], Sz = m.bS[3 * b + 2];
    double acc[15];
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;
    double inby = 0.0;
    const double K3D = m.K + 3.0 - m.D;
    const double RTw = 1.0 / br->invRT_in;
    for (int d = threadIdx.x; d < m.nv; d += blockDim.x) {
        const double xi[3] = {m.xi[3 * d], m.xi[3 * d + 1], m.xi[3 * d + 2]};
        const double xs = xi[0] * Sx + xi[1] * Sy + xi[2] * Sz;
        if (xs > 0) continue;
        const double cx = br->U[0] - xi[0], cy = br->U[1] - xi[1], cz = br->U[2] - xi[2];
        const double mm = br->K_in * exp(-(cx * cx + cy * cy + cz * cz) / (2.0 * RTw));
        const double w = m.w[d];
        if (xs < 0) inby += -w * xs * mm;
        const double xi2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        if (m.D == 3) accum<3>(acc, w, xi, xi2, mm, mm * RTw * K3D);
        else accum<2>(acc, w, xi, xi2, mm, mm * RTw * K3D);
    }
    // block reduction in a fixed order
    __shared__ double red[256][15];
    __shared__ double redi[256];
    for (int j = 0; j < 15; ++j) red[threadIdx.x][j] = acc[j];
    redi[threadIdx.x] = inby;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[15] = {0};
        double si = 0;
        for (int t = 0; t < blockDim.x; ++t) {
            for (int j = 0; j < 15; ++j) s[j] += red[t][j];
            si += redi[t];
        }
        double* mi = a.ds.bmom_in + static_cast<size_t>(b) * kNM;
        for (int j = 0; j < 15; ++j) mi[j] = s[j];
        br->inByRho = si;
    }
}

// raw cell moments of the current state, one thread per cell looping over
// all DVs (rows are contiguous in cells, so a warp reads coalesced)
template <int D, typename Real>
__global__ void k_state_moments(const StepArgs a) {
    const DevMesh& m = a.dm;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nC) return;
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    double acc[15];
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;
    for (int d = 0; d < m.nv; ++d) {
        const double xi[3] = {__ldg(m.xi + 3 * d), __ldg(m.xi + 3 * d + 1), __ldg(m.xi + 3 * d + 2)};
        const double xi2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        const size_t idx = static_cast<size_t>(d) * m.nC + c;
        accum<D>(acc, __ldg(m.w + d), xi, xi2, double(g[idx]), double(h[idx]));
    }
    double* p = a.ds.partC + static_cast<size_t>(c) * kNM;
    for (int j = 0; j < 15; ++j) p[j] = acc[j];
}

template <int D, typename Real, int IPT>
void launch_pass_t(const StepArgs& a, bool pass_b, cudaStream_t s) {
    dim3 grid(a.dm.n_tiles, a.chunks);
    if (!pass_b) k_pass_a<D, Real, IPT><<<grid, kThreads, a.smemA, s>>>(a);
    else k_pass_b<D, Real, IPT><<<grid, kThreads, a.smemB, s>>>(a);
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

cudaError_t launch_pass(const StepArgs& a, int precision, bool pass_b, cudaStream_t s) {
    if (precision == DUGKS_FP64)
        return a.dm.D == 3 ? launch_pass_d<3, double>(a, pass_b, s) : launch_pass_d<2, double>(a, pass_b, s);
    return a.dm.D == 3 ? launch_pass_d<3, float>(a, pass_b, s) : launch_pass_d<2, float>(a, pass_b, s);
}

template <int D, typename Real, int IPT>
cudaError_t configure_t(size_t smemA, size_t smemB) {
    cudaError_t e = cudaFuncSetAttribute(k_pass_a<D, Real, IPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smemA));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_pass_b<D, Real, IPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
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

cudaError_t launch_stage(const StepArgs& a, int precision, int stage, cudaStream_t s, int* launches) {
    const Consts k = make_consts(a.dm, a.dt);
    const int tb = 256;
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (stage) {
        case STAGE_PASS_A:
            e = launch_pass(a, precision, false, s);
            n = 1;
            break;
        case STAGE_FACE_COMBINE:
            if (a.dm.nIF > 0) {
                k_face_combine_internal<<<(a.dm.nIF + tb - 1) / tb, tb, 0, s>>>(a, k);
                ++n;
            }
            if (a.dm.nBF > 0) {
                k_face_combine_boundary<<<(a.dm.nBF + tb - 1) / tb, tb, 0, s>>>(a, k);
                ++n;
            }
            e = cudaGetLastError();
            break;
        case STAGE_PASS_B:
            e = launch_pass(a, precision, true, s);
            n = 1;
            break;
        case STAGE_CELL_COMBINE:
            k_cell_combine<<<(a.dm.nC + tb - 1) / tb, tb, 0, s>>>(a, k, a.dt_next);
            n = 1;
            e = cudaGetLastError();
            break;
        default:
            return cudaErrorInvalidValue;
    }
    if (launches) *launches += n;
    return e;
}

cudaError_t launch_step(const StepArgs& a, int precision, cudaStream_t s, int* launches) {
    for (int st = 0; st < 4; ++st) {
        cudaError_t e = launch_stage(a, precision, st, s, launches);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_state_macros(const StepArgs& a, int precision, cudaStream_t s) {
    const int tb = 128, nb = (a.dm.nC + tb - 1) / tb;
    if (precision == DUGKS_FP64) {
        if (a.dm.D == 3) k_state_moments<3, double><<<nb, tb, 0, s>>>(a);
        else k_state_moments<2, double><<<nb, tb, 0, s>>>(a);
    } else {
        if (a.dm.D == 3) k_state_moments<3, float><<<nb, tb, 0, s>>>(a);
        else k_state_moments<2, float><<<nb, tb, 0, s>>>(a);
    }
    StepArgs one = a;
    one.chunks = 1;
    const Consts k = make_consts(a.dm, a.dt);
    k_cell_combine<<<(a.dm.nC + 255) / 256, 256, 0, s>>>(one, k, 0.0);
    return cudaGetLastError();
}

cudaError_t launch_cell_prep(const StepArgs& a, cudaStream_t s) {
    k_cell_prep<<<(a.dm.nC + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_init(const StepArgs& a, int precision, cudaStream_t s) {
    if (precision == DUGKS_FP64) k_init_state<double><<<1184, 256, 0, s>>>(a);
    else k_init_state<float><<<1184, 256, 0, s>>>(a);
    if (a.dm.nBF > 0) k_init_wall<<<a.dm.nBF, 256, 0, s>>>(a);
    return cudaGetLastError();
}

void pass_smem(const DevMesh& dm, int max_local, int max_l0, int max_items, int precision, size_t* smemA,
               size_t* smemB) {
    const size_t rs = precision == DUGKS_FP64 ? sizeof(double) : sizeof(float);
    const size_t n = static_cast<size_t>(2 * max_local + 2 * max_l0 * dm.D + 2 * max_items + 2 * max_l0);
    *smemA = n * rs;
    *smemB = n * rs;
}

cudaError_t configure_kernels(int precision, int D, int ipt, size_t smemA, size_t smemB) {
    if (precision == DUGKS_FP64) return D == 3 ? configure_d<3, double>(ipt, smemA, smemB)
                                               : configure_d<2, double>(ipt, smemA, smemB);
    return D == 3 ? configure_d<3, float>(ipt, smemA, smemB) : configure_d<2, float>(ipt, smemA, smemB);
}

}  // namespace dugks

// The two tile passes of the DUGKS step (sm_100a).
//
// Discrete velocities are walked in batches of NB consecutive DVs of one DV
// row (the n1d DVs along x at fixed y and z).  Within a batch xi = (x_j, Y, Z)
// varies in x only, so xi.S, the Shakhov exponent and the raw moments split
// into a part computed once per batch (Y, Z) and a short per-DV part in x.
//
// Pass A: one CTA of 512 threads per (tile, DV chunk).  A tile is up to 128
// L0 cells, their L1 ring (up to 256 local cells in all) and its items = the
// faces touching L0 (up to 512, one per thread), sorted by kind.  Per batch:
//   stage 0  cp.async of the NEXT batch's g~, h~ (and, for DV sets of more
//            than 2 NB nodes per dimension, x Maxwellian factors) of the
//            local cells into shared memory, overlapping this batch's stages
//   stage 1  gbar+/hbar+ of the local cells (updateGHbarPvol,
//            fvDVM.C:648-683); the y and z Maxwellian factors of the row are
//            computed here from the cell record: two exponentials per cell
//            cost less than gathering them for the ring cells
//   stage 2  least-squares gradients of the L0 cells (leastSquaresGrad;
//            the zero-gradient boundary terms vanish, fvDVM.C:456-485,
//            :775-809)
//   stage 3  per item: upwind reconstruction at the half step
//            (updateGHbarSurf, fvDVM.C:755-1029); raw face moments in
//            registers (updateMacroSurf, :1181-1297) and the wall out-flux;
//            the reconstructed value goes to the face-value buffer
// Pass B: one CTA per (tile, DV chunk), L0 cells and items only.  Per batch:
//   stage 3  per item: relaxation of the stored face value (updateGHsurf,
//            :1362-1457), incoming boundary DFs, flux xi.S g_f to shared memory
//   stage 4  per L0 cell: gbar+ of the cell, flux gather and g~/h~ update
//            (updateGHtildeVol, :1462-1519), raw cell moments (updateMacroVol,
//            :1528-1554)
#include "dugks_device.cuh"

namespace dugks {

namespace {

constexpr int kSL = kMaxLocal;           // row stride of local-cell arrays in shared memory
constexpr int kS0 = kMaxTile;            // row stride of L0-cell arrays
constexpr int kSI = kMaxItems + 1;       // row stride of item arrays (slot kSI - 1: zero flux)
constexpr int kPartsL = kThreads / kSL;  // threads per local cell in stages 0-1
constexpr int kParts0 = kThreads / kS0;  // threads per L0 cell in stages 2 and 4
// Hex cells have at most 6 face neighbours: such stencils are kept in
// shared memory for the whole CTA (larger ones are read from global memory)
constexpr int kMaxRegStencil = 6;

// batch widths: pass A (narrow, wide), pass B (narrow, wide)
template <typename Real>
struct Width;
template <>
struct Width<double> {
    static constexpr int A0 = 8, A1 = 8, B0 = 8, B1 = 8;
};
template <>
struct Width<float> {
    static constexpr int A0 = 8, A1 = 8, B0 = 8, B1 = 8;
};

// FP32 storage holds deviations from the per-DV reference Maxwellian
// (DevMesh::gref, href): g = stored + ref.  These add and remove the
// reference; for FP64 storage they are the identity and read nothing.
template <typename Real>
__device__ __forceinline__ double dv_ref(const double* ref, int d) {
    if constexpr (sizeof(Real) == 4) return __ldg(ref + d);
    else return 0.0;
}
template <typename Real>
__device__ __forceinline__ double plus_ref(double x, double r) {
    if constexpr (sizeof(Real) == 4) return x + r;
    else return x;
}
template <typename Real>
__device__ __forceinline__ double minus_ref(double x, double r) {
    if constexpr (sizeof(Real) == 4) return x - r;
    else return x;
}

// ---------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async, L1-allocating)
// ---------------------------------------------------------------------
template <typename Real>
__device__ __forceinline__ void cp_async(Real* sdst, const Real* gsrc) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    if (sizeof(Real) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------
struct TileRange {
    int b, n0, loff, nloc, ioff, nit, r0, r1;
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
    t.r0 = __ldg(chunk_begin + chunk);
    t.r1 = __ldg(chunk_begin + chunk + 1);
    return t;
}

// position of batch k of a chunk: first x index, width, first DV of this
// device's DV block (the state and face-value row), row indices
struct BatchPos {
    int ix0, nb, d0, iy, iz;
};

// walks the batches of a chunk of DV rows in order (x batches of a row,
// then the next row) without integer divisions per batch
template <int D, int NB>
struct BatchWalk {
    int row, iy, iz, kb, nbr, n1d, rb;
    // r0: first global row of the chunk; base: first global row this device holds
    __device__ __forceinline__ BatchWalk(int r0, int n, int base)
        : row(r0), kb(0), nbr((n + NB - 1) / NB), n1d(n), rb(base) {
        iy = D == 3 ? r0 % n : r0;
        iz = D == 3 ? r0 / n : 0;
    }
    __device__ __forceinline__ BatchPos pos() const {
        BatchPos p;
        p.ix0 = kb * NB;
        p.nb = min(NB, n1d - p.ix0);
        p.d0 = (row - rb) * n1d + p.ix0;
        p.iy = iy;
        p.iz = iz;
        return p;
    }
    __device__ __forceinline__ void next() {
        if (++kb == nbr) {
            kb = 0;
            ++row;
            if (++iy == n1d && D == 3) {
                iy = 0;
                ++iz;
            }
        }
    }
};

// per-batch DV constants: the y, z velocity and weight of the row and the
// products the moment fold needs.  The DV weight is w1[iz] w1[iy] w1[ix]
// (3-D) or w1[iy] w1[ix] (2-D), as the tensor product is formed.
struct RowConst {
    double Y, Z, wyz, R2, cY, cZ, cYY, cYZ, cZZ;
};

template <int D>
__device__ __forceinline__ RowConst row_const(const double* x1, const double* w1, const BatchPos& p) {
    RowConst q;
    q.Y = x1[p.iy];
    q.Z = D == 3 ? x1[p.iz] : 0.0;
    q.wyz = D == 3 ? w1[p.iz] * w1[p.iy] : w1[p.iy];
    q.R2 = q.Y * q.Y + q.Z * q.Z;
    q.cY = q.wyz * q.Y;
    q.cZ = q.wyz * q.Z;
    q.cYY = q.cY * q.Y;
    q.cYZ = q.cY * q.Z;
    q.cZZ = q.cZ * q.Z;
    return q;
}

// Raw moments of one batch, summed along x (a = w_x g, b = w_x h):
// S_k = sum a x^k (k = 0..3), B_k = sum b x^k (k = 0, 1), O = sum a xi.S
// over outgoing wall DVs.  row_fold turns them into the moment record
// (layout in dugks_internal.h) with |xi|^2 = x^2 + Y^2 + Z^2.
struct RowSums {
    double S0, S1, S2, S3, B0, B1, O;
};

__device__ __forceinline__ void row_zero(RowSums& r) { r.S0 = r.S1 = r.S2 = r.S3 = r.B0 = r.B1 = r.O = 0.0; }

// HZ: h is identically zero (D = 3, KInner = 0); its sums stay zero
template <bool HZ = false>
__device__ __forceinline__ double row_add(RowSums& r, double wx, double x, double g, double h) {
    const double a = wx * g;
    r.S0 += a;
    const double ax = a * x;
    r.S1 += ax;
    const double ax2 = ax * x;
    r.S2 += ax2;
    r.S3 = fma(ax2, x, r.S3);
    if constexpr (!HZ) {
        const double b = wx * h;
        r.B0 += b;
        r.B1 = fma(b, x, r.B1);
    }
    return a;
}

template <int D>
__device__ __forceinline__ void row_fold(double* acc, const RowSums& r, const RowConst& q) {
    const double c = q.wyz;
    const double Wb = r.S2 + fma(q.R2, r.S0, r.B0);   // sum a |xi|^2 + b
    const double Vx = r.S3 + fma(q.R2, r.S1, r.B1);   // sum (a |xi|^2 + b) x
    acc[MOM_M0] = fma(c, r.S0, acc[MOM_M0]);
    acc[MOM_M1] = fma(c, r.S1, acc[MOM_M1]);
    acc[MOM_M1 + 1] = fma(q.cY, r.S0, acc[MOM_M1 + 1]);
    acc[MOM_W] = fma(c, Wb, acc[MOM_W]);
    acc[MOM_V3] = fma(c, Vx, acc[MOM_V3]);
    acc[MOM_V3 + 1] = fma(q.cY, Wb, acc[MOM_V3 + 1]);
    acc[MOM_M2] = fma(c, r.S2, acc[MOM_M2]);
    acc[MOM_M2 + 1] = fma(q.cY, r.S1, acc[MOM_M2 + 1]);
    acc[MOM_M2 + 3] = fma(q.cYY, r.S0, acc[MOM_M2 + 3]);
    if (D == 3) {
        acc[MOM_M1 + 2] = fma(q.cZ, r.S0, acc[MOM_M1 + 2]);
        acc[MOM_V3 + 2] = fma(q.cZ, Wb, acc[MOM_V3 + 2]);
        acc[MOM_M2 + 2] = fma(q.cZ, r.S1, acc[MOM_M2 + 2]);
        acc[MOM_M2 + 4] = fma(q.cYZ, r.S0, acc[MOM_M2 + 4]);
        acc[MOM_M2 + 5] = fma(q.cZZ, r.S0, acc[MOM_M2 + 5]);
    }
    acc[MOM_OUT] = fma(c, r.O, acc[MOM_OUT]);
}

// xi.S rounded as the reference evaluates it, ((x Sx + y Sy) + z Sz) without
// fused multiply-adds, with the y and z products of the row precomputed
__device__ __forceinline__ double xs_row(double x, double Sx, double p2, double p3) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, Sx), p2), p3);
}

// ---------------------------------------------------------------------
// Shakhov relaxation pair of one DV from the per-batch parts of a record
//   gbar = (1-r) g + r gS,  hbar = (1-r) h + r hS   (fvDVM.C:668-679, :1374-1391)
//   gS = E (1 + s (cs - D - 2)),  hS = E RTh (K3D + s ((cs - D) K3D - 2 K))
//   cs = |xi-U|^2 / RT = (x-Ux)^2 / RT + Cyz,  s = (xi-U).qv = (x-Ux) qx + Syz
//   r E = (A e_x(x)) (r e_y(Y) e_z(Z))
// ---------------------------------------------------------------------
template <typename Real>
struct Shk {
    Real Ux, invRT, qx, RTh, omr;   // per entity
    Real Cyz, Syz, eyzr;            // per entity and batch
};

template <int D, typename Real>
__device__ __forceinline__ void shk_batch(Shk<Real>& s, Real Uy, Real Uz, Real qy, Real qz, Real r, double Y, double Z,
                                          Real ey, Real ez) {
    const Real cy = Real(Y) - Uy;
    const Real cz = D == 3 ? Real(Z) - Uz : Real(0);
    s.Cyz = (cy * cy + cz * cz) * s.invRT;
    s.Syz = D == 3 ? cy * qy + cz * qz : cy * qy;
    s.eyzr = D == 3 ? r * ey * ez : r * ey;
}

template <int D, typename Real>
__device__ __forceinline__ void shk_relax(const Shk<Real>& s, Real x, Real ex, Real g, Real h, Real K3D, Real c0h,
                                          Real& go, Real& ho) {
    const Real cx = x - s.Ux;
    const Real cs = fma(cx * cx, s.invRT, s.Cyz);
    const Real sq = fma(cx, s.qx, s.Syz);
    const Real Er = ex * s.eyzr;
    const Real pg = fma(sq, cs - Real(D + 2), Real(1));
    const Real ph = fma(sq, fma(cs, K3D, c0h), K3D);
    go = fma(s.omr, g, Er * pg);
    ho = fma(s.omr, h, (Er * s.RTh) * ph);
}

// ---------------------------------------------------------------------
// Shared memory
// ---------------------------------------------------------------------
enum { CR_UX, CR_UY, CR_UZ, CR_INVRT, CR_QX, CR_QY, CR_QZ, CR_RTH, CR_OMR, CR_R, CR_N };

template <int D, typename Real, int NB, bool HZ = false>
struct SmemA {
    // DF arrays per local cell: g~ and h~, or g~ alone when h is identically zero
    static constexpr int NH = HZ ? 1 : 2;
    // rows of stgx: [2][NB] staged per batch, or the resident table [n1d];
    // the g-only 16-wide pass runs on DV sets of at most NB nodes per
    // dimension and keeps the resident table only
    static constexpr int XR = (HZ && NB >= 16) ? NB : 2 * NB;
    double* x1;     // [kMaxN1d] 1-D nodes
    double* w1;     // [kMaxN1d] 1-D weights
    double* crec;   // [CR_N][kSL] records of the local cells
    // e_x of the local cells: when the DV set has at most 2 NB nodes per
    // dimension, the whole table [n1d][kSL] is loaded once per CTA (e_x does
    // not depend on the row); otherwise [2][NB][kSL] staged per batch
    double* stgx;
    Real* stg;      // [2][NH][NB][kSL] staged g~ (and h~)
    // FP32 storage: gbar+ is double-buffered by batch parity ([2][NB][kSL])
    static constexpr int GB = sizeof(Real) == 4 ? 2 : 1;
    Real* gB;       // [GB][NB][kSL] gbar+
    Real* hB;       // (null when h is identically zero)
    Real* Gg;       // [NB][D][kS0] gradients of the L0 cells
    Real* Gh;       // (null when h is identically zero)
    int* snb;       // [kMaxRegStencil][kS0] gradient stencils of the L0 cells: local neighbour
    Real* sls;      // [kMaxRegStencil][D][kS0] and least-squares vector
    static constexpr size_t bytes() {
        return 2 * kMaxN1d * sizeof(double) + static_cast<size_t>(kMaxRegStencil) * kS0 * sizeof(int) +
               (static_cast<size_t>(CR_N) * kSL + static_cast<size_t>(XR) * kSL) * sizeof(double) +
               (2 * NH * static_cast<size_t>(NB) * kSL + GB * NH * NB * kSL + NH * NB * D * kS0 +
                static_cast<size_t>(kMaxRegStencil) * D * kS0) *
                   sizeof(Real);
    }
};

template <int D, typename Real, int NB, bool HZ = false>
__device__ __forceinline__ SmemA<D, Real, NB, HZ> carve_a(unsigned char* base) {
    using S = SmemA<D, Real, NB, HZ>;
    S s;
    s.x1 = reinterpret_cast<double*>(base);
    s.w1 = s.x1 + kMaxN1d;
    s.crec = s.w1 + kMaxN1d;
    s.stgx = s.crec + CR_N * kSL;
    Real* p = reinterpret_cast<Real*>(s.stgx + S::XR * kSL);
    s.stg = p;
    p += 2 * S::NH * NB * kSL;
    s.gB = p;
    p += S::GB * NB * kSL;
    s.hB = HZ ? nullptr : p;
    if (!HZ) p += S::GB * NB * kSL;
    s.Gg = p;
    p += NB * D * kS0;
    s.Gh = HZ ? nullptr : p;
    if (!HZ) p += NB * D * kS0;
    s.sls = p;
    p += kMaxRegStencil * D * kS0;
    s.snb = reinterpret_cast<int*>(p);
    return s;
}

template <typename Real, int NB, bool HZ = false>
struct SmemB {
    // DF arrays per item: g and h, or g alone when h is identically zero
    static constexpr int NH = HZ ? 1 : 2;
    // rows of stx: e_x of the items does not depend on the row, so a DV set
    // of at most XR nodes per dimension keeps the whole table [n1d][kSI],
    // loaded once per CTA; larger sets stage [NB][kSI] per batch.  Where h is
    // identically zero, 8-DV batches keep 16 rows in the shared memory h
    // would take (16- and 20-wide batches hold a whole row already; for
    // 10-DV batches on 20-node sets the resident table measured slower than
    // staging)
    static constexpr int XR = (HZ && 2 * NB <= 16) ? 2 * NB : NB;
    double* x1;
    double* w1;
    double* frec;  // [CR_N][kSI] face records of the items
    double* crec;  // [CR_N][kS0] records of the L0 cells
    double* stx;   // [XR][kSI] e_x of the items: the resident table, or staged per batch
    Real* st;      // [NH][NB][kSI] staged face values g (and h) of the items
    Real* Fg;      // [NB][kSI] fluxes xi.S g_f of the items
    Real* Fh;      // (null when h is identically zero)
    double* red;   // end-of-CTA reduction of the split cell moments (aliases stx and st)
    static constexpr size_t bytes() {
        return 2 * kMaxN1d * sizeof(double) +
               (static_cast<size_t>(CR_N) * (kSI + kS0) + static_cast<size_t>(XR) * kSI) * sizeof(double) +
               2 * NH * static_cast<size_t>(NB) * kSI * sizeof(Real);
    }
};

template <typename Real, int NB, bool HZ = false>
__device__ __forceinline__ SmemB<Real, NB, HZ> carve_b(unsigned char* base) {
    using S = SmemB<Real, NB, HZ>;
    S s;
    s.x1 = reinterpret_cast<double*>(base);
    s.w1 = s.x1 + kMaxN1d;
    s.frec = s.w1 + kMaxN1d;
    s.crec = s.frec + CR_N * kSI;
    s.stx = s.crec + CR_N * kS0;
    s.st = reinterpret_cast<Real*>(s.stx + S::XR * kSI);
    s.Fg = s.st + S::NH * NB * kSI;
    s.Fh = HZ ? nullptr : s.Fg + NB * kSI;
    s.red = s.stx;
    return s;
}

// a coefficient record (structure of arrays over n entities) into shared
// memory: U, 1/RT, qv, RTh, 1 - r, r
template <typename Real>
__device__ __forceinline__ void stash_rec(Real* dst, int stride, int l, const double* __restrict__ rec, size_t n, int e) {
    dst[CR_UX * stride + l] = Real(__ldg(rec + REC_UX * n + e));
    dst[CR_UY * stride + l] = Real(__ldg(rec + REC_UY * n + e));
    dst[CR_UZ * stride + l] = Real(__ldg(rec + REC_UZ * n + e));
    dst[CR_INVRT * stride + l] = Real(__ldg(rec + REC_INVRT * n + e));
    dst[CR_QX * stride + l] = Real(__ldg(rec + REC_QX * n + e));
    dst[CR_QY * stride + l] = Real(__ldg(rec + REC_QY * n + e));
    dst[CR_QZ * stride + l] = Real(__ldg(rec + REC_QZ * n + e));
    dst[CR_RTH * stride + l] = Real(__ldg(rec + REC_RTH * n + e));
    const double r = __ldg(rec + REC_R * n + e);
    dst[CR_OMR * stride + l] = Real(1.0 - r);
    dst[CR_R * stride + l] = Real(r);
}

// the Shakhov parts of a stashed record for one batch
template <int D, typename Real>
__device__ __forceinline__ Shk<Real> shk_from(const Real* src, int stride, int l, const RowConst& q, Real ey, Real ez) {
    Shk<Real> s;
    s.Ux = src[CR_UX * stride + l];
    s.invRT = src[CR_INVRT * stride + l];
    s.qx = src[CR_QX * stride + l];
    s.RTh = src[CR_RTH * stride + l];
    s.omr = src[CR_OMR * stride + l];
    shk_batch<D, Real>(s, src[CR_UY * stride + l], src[CR_UZ * stride + l], src[CR_QY * stride + l],
                       src[CR_QZ * stride + l], src[CR_R * stride + l], q.Y, q.Z, ey, ez);
    return s;
}
static_assert(static_cast<size_t>(kParts0 - 1) * kS0 * 15 * sizeof(double) <=
                  static_cast<size_t>(Width<double>::B0) * kSI * (sizeof(double) + 2 * sizeof(double)),
              "the cell-moment reduction must fit in the staging arrays");
static_assert(static_cast<size_t>(kParts0 - 1) * kS0 * 15 * sizeof(double) <=
                  static_cast<size_t>(Width<float>::B0) * kSI * (sizeof(double) + 2 * sizeof(float)),
              "the cell-moment reduction must fit in the staging arrays");

__device__ __forceinline__ void load_dv_tables(const DevMesh& m, double* x1, double* w1) {
    if (threadIdx.x < m.n1d) {
        x1[threadIdx.x] = __ldg(m.X1 + threadIdx.x);
        w1[threadIdx.x] = __ldg(m.W1 + threadIdx.x);
    }
}

// ---------------------------------------------------------------------
// Items
// ---------------------------------------------------------------------
// Per-item registers.  la/da: the side reconstructed here (internal items:
// the owner; tile-boundary items: the side in the tile; boundary items: the
// owner), lb/db: the neighbour of internal items.
struct Item {
    int kind, ptype, la, lb, gi, face, other;
    double S[3], da[3], db[3];
};

__device__ __forceinline__ Item load_item(const DevMesh& m, int gi) {
    Item v;
    const int meta = __ldg(m.it_meta + gi), loc = __ldg(m.it_loc + gi);
    v.kind = meta & 15;
    v.ptype = meta >> 4;
    v.gi = gi;
    v.face = __ldg(m.it_face + gi);
    v.other = __ldg(m.it_other + gi);
    const int lo = loc & 0xffff, ln = (loc >> 16) & 0xffff;
    const size_t n = static_cast<size_t>(m.n_items);
    double dO[3], dN[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        v.S[q] = __ldg(m.it_geo + q * n + gi);
        dO[q] = __ldg(m.it_geo + (3 + q) * n + gi);
        dN[q] = __ldg(m.it_geo + (6 + q) * n + gi);
    }
    const bool nei_here = v.kind == ITEM_TB_NEI;
    v.la = nei_here ? ln : lo;
    v.lb = ln;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        v.da[q] = nei_here ? dN[q] : dO[q];
        v.db[q] = dN[q];
    }
    return v;
}

// reconstruction at the half step from local L0 cell l (fvDVM.C:832-836):
// gbar+_l + grad_l . v,  v = Cf - C_l - xi dt/2
template <int D, typename Real, int NB, bool HZ = false>
__device__ __forceinline__ void recon(const SmemA<D, Real, NB, HZ>& sm, int j, int l, Real vx, Real vy, Real vz, Real& g,
                                      Real& h) {
    const Real* Gg = sm.Gg + j * D * kS0 + l;
    Real gg = fma(Gg[0], vx, sm.gB[j * kSL + l]);
    gg = fma(Gg[kS0], vy, gg);
    if (D == 3) gg = fma(Gg[2 * kS0], vz, gg);
    g = gg;
    if constexpr (HZ) {
        h = Real(0);
    } else {
        const Real* Gh = sm.Gh + j * D * kS0 + l;
        Real hh = fma(Gh[0], vx, sm.hB[j * kSL + l]);
        hh = fma(Gh[kS0], vy, hh);
        if (D == 3) hh = fma(Gh[2 * kS0], vz, hh);
        h = hh;
    }
}

// ---------------------------------------------------------------------
// Pass A stages
// ---------------------------------------------------------------------
// cp.async of batch bp's inputs of local cell l (thread part `part` of it)
template <int D, typename Real, int NB, bool FULL, bool HZ>
__device__ __forceinline__ void stage0(const DevMesh& m, const SmemA<D, Real, NB, HZ>& sm, int buf, const BatchPos& bp,
                                       const Real* __restrict__ g, const Real* __restrict__ h,
                                       const double* __restrict__ ctab, int l, int part, int c, bool active,
                                       bool ex_res) {
    if (active) {
        constexpr int H = NB / kPartsL;
        Real* sg = sm.stg + static_cast<size_t>(buf) * SmemA<D, Real, NB, HZ>::NH * NB * kSL;
        double* sx = sm.stgx + static_cast<size_t>(buf) * NB * kSL;
        const size_t nC = static_cast<size_t>(m.nC);
#pragma unroll
        for (int jj = 0; jj < H; ++jj) {
            const int j = part * H + jj;
            if (FULL || j < bp.nb) {
                cp_async(sg + j * kSL + l, g + static_cast<size_t>(bp.d0 + j) * nC + c);
                if (!HZ) cp_async(sg + (NB + j) * kSL + l, h + static_cast<size_t>(bp.d0 + j) * nC + c);
                if (!ex_res) cp_async(sx + j * kSL + l, ctab + static_cast<size_t>(bp.ix0 + j) * nC + c);
            }
        }

    }
    cp_commit();
}

template <int D, typename Real, int NB, bool FULL, bool HZ>
__device__ __forceinline__ void stage1(const SmemA<D, Real, NB, HZ>& sm, int buf, const BatchPos& bp, const RowConst& q,
                                       int l, int part, bool active, double K3D, double c0h, bool ex_res,
                                       const double* gref, const double* href, double& ey, double& ez) {
    if (!active) return;
    Shk<double> s;
    s.Ux = sm.crec[CR_UX * kSL + l];
    s.invRT = sm.crec[CR_INVRT * kSL + l];
    s.qx = sm.crec[CR_QX * kSL + l];
    s.RTh = sm.crec[CR_RTH * kSL + l];
    s.omr = sm.crec[CR_OMR * kSL + l];
    // the y and z Maxwellian factors of the batch's row, as the combine
    // kernels tabulate them (write_maxwell_tables): exp(-x^2/2 invRT); the
    // thread's cell is the same in every batch, so the g-only pass, which
    // has the registers to spare, computes them on the row's first batch
    // and keeps them for the others
    const double uy = sm.crec[CR_UY * kSL + l], uz = sm.crec[CR_UZ * kSL + l];
    if (!HZ || bp.ix0 == 0) {
        const double yy = q.Y - uy, zz = q.Z - uz;
        ey = exp(-0.5 * yy * yy * s.invRT);
        ez = D == 3 ? exp(-0.5 * zz * zz * s.invRT) : 1.0;
    }
    shk_batch<D, double>(s, uy, uz, sm.crec[CR_QY * kSL + l], sm.crec[CR_QZ * kSL + l], sm.crec[CR_R * kSL + l], q.Y,
                         q.Z, ey, ez);
    const Real* sg = sm.stg + static_cast<size_t>(buf) * SmemA<D, Real, NB, HZ>::NH * NB * kSL;
    const double* sx = sm.stgx + (ex_res ? bp.ix0 : buf * NB) * kSL;
    constexpr int H = NB / kPartsL;
#pragma unroll
    for (int jj = 0; jj < H; ++jj) {
        const int j = part * H + jj;
        if (FULL || j < bp.nb) {
            double go, ho;
            const double gr = dv_ref<Real>(gref, bp.d0 + j), hr = dv_ref<Real>(href, bp.d0 + j);
            const double hin = HZ ? 0.0 : plus_ref<Real>(double(sg[(NB + j) * kSL + l]), hr);
            shk_relax<D, double>(s, sm.x1[bp.ix0 + j], sx[j * kSL + l], plus_ref<Real>(double(sg[j * kSL + l]), gr),
                                 hin, K3D, c0h, go, ho);
            sm.gB[j * kSL + l] = Real(minus_ref<Real>(go, gr));
            if (!HZ) sm.hB[j * kSL + l] = Real(minus_ref<Real>(ho, hr));
        }
    }
}


template <int D, typename Real, int NB, bool HZ>
__device__ __forceinline__ void grad_one(const SmemA<D, Real, NB, HZ>& sm, int j, int l, const int* nbi,
                                         const Real (*ls)[D], int nk) {
    const Real* gB = sm.gB + j * kSL;
    const Real* hB = HZ ? nullptr : sm.hB + j * kSL;
    const Real g0 = gB[l], h0 = HZ ? Real(0) : hB[l];
    Real gx[D], hx[D];
#pragma unroll
    for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
#pragma unroll
    for (int k = 0; k < kMaxRegStencil; ++k) {
        if (k < nk) {
            const Real dg = gB[nbi[k]] - g0;
#pragma unroll
            for (int q = 0; q < D; ++q) gx[q] = fma(ls[k][q], dg, gx[q]);
            if constexpr (!HZ) {
                const Real dh = hB[nbi[k]] - h0;
#pragma unroll
                for (int q = 0; q < D; ++q) hx[q] = fma(ls[k][q], dh, hx[q]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < D; ++q) {
        sm.Gg[(j * D + q) * kS0 + l] = gx[q];
        if (!HZ) sm.Gh[(j * D + q) * kS0 + l] = hx[q];
    }
}

template <int D, typename Real, int NB, bool FULL, bool HZ>
__device__ __forceinline__ void stage2(const DevMesh& m, const SmemA<D, Real, NB, HZ>& sm, const BatchPos& bp,
                                       const TileRange& t, int* err) {
    const int l = threadIdx.x % kS0, part = threadIdx.x / kS0;
    if (l >= t.n0) return;
    const int c = t.b + l;
    constexpr int H = (NB + kParts0 - 1) / kParts0;
    if (m.nb_max <= kMaxRegStencil) {
        // stencil from shared memory (absent neighbours: the cell itself
        // with a zero vector)
        int nbi[kMaxRegStencil];
        Real ls[kMaxRegStencil][D];
#pragma unroll
        for (int k = 0; k < kMaxRegStencil; ++k) {
            nbi[k] = sm.snb[k * kS0 + l];
#pragma unroll
            for (int q = 0; q < D; ++q) ls[k][q] = sm.sls[(k * D + q) * kS0 + l];
        }
#pragma unroll
        for (int jj = 0; jj < H; ++jj) {
            const int j = part + kParts0 * jj;
            if (FULL || j < bp.nb) grad_one<D, Real, NB, HZ>(sm, j, l, nbi, ls, kMaxRegStencil);
        }
    } else {
#pragma unroll 1
        for (int jj = 0; jj < H; ++jj) {
            const int j = part + kParts0 * jj;
            if (!FULL && j >= bp.nb) break;
            const Real* gB = sm.gB + j * kSL;
            const Real* hB = HZ ? nullptr : sm.hB + j * kSL;
            const Real g0 = gB[l], h0 = HZ ? Real(0) : hB[l];
            Real gx[D], hx[D];
#pragma unroll
            for (int q = 0; q < D; ++q) gx[q] = hx[q] = Real(0);
            for (int k = 0; k < m.nb_max; ++k) {
                const int n0 = __ldg(m.grad_nb + static_cast<size_t>(k) * m.nC + c);
                if (n0 < 0) continue;
                const int n = chk(n0, 0, t.nloc, err);
                const Real dg = gB[n] - g0, dh = HZ ? Real(0) : hB[n] - h0;
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    const Real lsq = Real(__ldg(m.grad_ls + (static_cast<size_t>(k) * 3 + q) * m.nC + c));
                    gx[q] = fma(lsq, dg, gx[q]);
                    hx[q] = fma(lsq, dh, hx[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < D; ++q) {
                sm.Gg[(j * D + q) * kS0 + l] = gx[q];
                if (!HZ) sm.Gh[(j * D + q) * kS0 + l] = hx[q];
            }
        }
    }
}

// ---------------------------------------------------------------------
// Pass A: face reconstruction, raw face moments, face values
// ---------------------------------------------------------------------
// HZ: h is identically zero (D = 3 and KInner = 0 make K + 3 - D = 0 in
// every h formula, fvDVM.C:414-426, :673-679, :1079-1092): the pass reads,
// reconstructs and writes g alone; its results are those of the full pass
template <int D, typename Real, int NB, bool FULL, bool HZ>
__global__ void __launch_bounds__(kThreads, 1) k_pass_a(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemA<D, Real, NB, HZ> sm = carve_a<D, Real, NB, HZ>(smem_raw);
    // FP32 storage: gbar+ double-buffered by batch parity, so stage 1 of a
    // batch overwrites no buffer the previous batch's stage 3 still reads,
    // and the loop needs no barrier before stage 1.  Used where it costs no
    // register spills (2-D, and 3-D rows that do not split into whole
    // batches); measured 1.96 -> 1.68 ms on a 256^2 x 28^2 cavity, while the
    // spilling 3-D 16-wide variant lost 4 %
    constexpr bool kDbl = SmemA<D, Real, NB, HZ>::GB == 2 && (D == 2 || !FULL);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    const double* ctab = a.ds.ctab;
    Real* const fvg = reinterpret_cast<Real*>(a.ds.fvg);
    Real* const fvh = reinterpret_cast<Real*>(a.ds.fvh);
    const double K3D = m.K + 3.0 - m.D, c0h = -(m.D * (m.K + 3.0 - m.D) + 2.0 * m.K);
    const Real hdt = Real(0.5 * step_dt(a));
    const size_t nI = static_cast<size_t>(m.n_items);

    // CTA set-up: DV tables, records of the local cells, this thread's cell
    // of stages 0-1 and its item
    load_dv_tables(m, sm.x1, sm.w1);
    const int l1 = threadIdx.x % kSL, p1 = threadIdx.x / kSL;
    const bool act1 = l1 < t.nloc;
    const int c1 = act1 ? chk(__ldg(m.loc_cells + t.loff + l1), 0, m.nC, a.ds.err) : 0;
    if (act1 && p1 == 0) {
        const double* cr = a.ds.cellrec;
        const size_t n = static_cast<size_t>(m.nC);
        sm.crec[CR_UX * kSL + l1] = __ldg(cr + REC_UX * n + c1);
        sm.crec[CR_UY * kSL + l1] = __ldg(cr + REC_UY * n + c1);
        sm.crec[CR_UZ * kSL + l1] = __ldg(cr + REC_UZ * n + c1);
        sm.crec[CR_INVRT * kSL + l1] = __ldg(cr + REC_INVRT * n + c1);
        sm.crec[CR_QX * kSL + l1] = __ldg(cr + REC_QX * n + c1);
        sm.crec[CR_QY * kSL + l1] = __ldg(cr + REC_QY * n + c1);
        sm.crec[CR_QZ * kSL + l1] = __ldg(cr + REC_QZ * n + c1);
        sm.crec[CR_RTH * kSL + l1] = __ldg(cr + REC_RTH * n + c1);
        const double r = __ldg(cr + REC_R * n + c1);
        sm.crec[CR_OMR * kSL + l1] = 1.0 - r;
        sm.crec[CR_R * kSL + l1] = r;
    }
    const bool ex_res = m.n1d <= 2 * NB;
    if (ex_res && act1)
        for (int ix = p1; ix < m.n1d; ix += kPartsL)
            sm.stgx[ix * kSL + l1] = __ldg(ctab + static_cast<size_t>(ix) * m.nC + c1);
    // gradient stencils of the L0 cells (slot-major tables, -1: none)
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

    BatchWalk<D, NB> walk(t.r0, m.n1d, m.row_base), ahead(t.r0, m.n1d, m.row_base);
    const int nbt = (t.r1 - t.r0) * walk.nbr;
    double ey1 = 1.0, ez1 = 1.0;   // y, z Maxwellian factors of this thread's local cell and row
    if (nbt > 0) stage0<D, Real, NB, FULL, HZ>(m, sm, 0, ahead.pos(), g, h, ctab, l1, p1, c1, act1, ex_res);
    if constexpr (kDbl) __syncthreads();  // the CTA set-up above is visible to every thread
    for (int k = 0; k < nbt; ++k, walk.next()) {
        const int buf = k & 1;
        const BatchPos bp = walk.pos();
        // this thread's staged entries of batch k (stage 1 reads only what the
        // same thread staged)
        cp_wait_all();
        if constexpr (kDbl) {
            const SmemA<D, Real, NB, HZ> s0 = carve_a<D, Real, NB, HZ>(smem_raw);
            sm.gB = s0.gB + buf * NB * kSL;
            if (!HZ) sm.hB = s0.hB + buf * NB * kSL;
        } else {
            __syncthreads();  // the previous batch's stage 3 is done with gbar+ (and the set-up is visible)
        }
        if (k + 1 < nbt) {
            ahead.next();
            stage0<D, Real, NB, FULL, HZ>(m, sm, buf ^ 1, ahead.pos(), g, h, ctab, l1, p1, c1, act1, ex_res);
        }
        const RowConst q = row_const<D>(sm.x1, sm.w1, bp);
        stage1<D, Real, NB, FULL, HZ>(sm, buf, bp, q, l1, p1, act1, K3D, c0h, ex_res, m.gref, m.href, ey1, ez1);
        __syncthreads();
        stage2<D, Real, NB, FULL, HZ>(m, sm, bp, t, a.ds.err);
        __syncthreads();
        if (!has_item) continue;
        // stage 3
        const double p2 = __dmul_rn(q.Y, v.S[1]);
        const double p3 = D == 3 ? __dmul_rn(q.Z, v.S[2]) : 0.0;
        const Real ay = Real(v.da[1]) - hdt * Real(q.Y), az = Real(v.da[2]) - hdt * Real(q.Z);
        RowSums rs;
        row_zero(rs);
        Real* fg = fvg + static_cast<size_t>(bp.d0) * nI + v.gi;
        Real* fh = fvh + static_cast<size_t>(bp.d0) * nI + v.gi;
        if (v.kind == ITEM_TILE_INTERNAL) {
            const Real by = Real(v.db[1]) - hdt * Real(q.Y), bz = Real(v.db[2]) - hdt * Real(q.Z);
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (FULL || j < bp.nb) {
                    const double x = sm.x1[bp.ix0 + j];
                    const double xs = xs_row(x, v.S[0], p2, p3);
                    const bool own_up = xs >= kVSmall, nei_up = xs < -kVSmall;
                    const Real hx = hdt * Real(x);
                    Real gg, hh;
                    if (own_up || nei_up) {
                        recon<D, Real, NB, HZ>(sm, j, own_up ? v.la : v.lb, Real(own_up ? v.da[0] : v.db[0]) - hx,
                                               own_up ? ay : by, own_up ? az : bz, gg, hh);
                    } else {
                        // exactly tangential: both sides averaged (fvDVM.C:847-863)
                        Real g1, h1, g2, h2;
                        recon<D, Real, NB, HZ>(sm, j, v.la, Real(v.da[0]) - hx, ay, az, g1, h1);
                        recon<D, Real, NB, HZ>(sm, j, v.lb, Real(v.db[0]) - hx, by, bz, g2, h2);
                        gg = Real(0.5) * (g2 + g1);
                        hh = Real(0.5) * (h2 + h1);
                    }
                    // FP32 storage: the deviations only; the reference part is added once below
                    row_add<HZ>(rs, sm.w1[bp.ix0 + j], x, double(gg), double(hh));
                    fg[j * nI] = gg;
                    if (!HZ) fh[j * nI] = hh;
                }
            }
        } else if (v.kind != ITEM_MESH_BOUNDARY) {
            // tile-boundary face: this tile's side only, weighted 1 upwind,
            // 1/2 tangential, 0 downwind; the other tile adds its side.  The
            // upwind tile writes the face value into both items' slots, so
            // that each tile's pass B reads its own slot, coalesced (reading
            // the other tile's slot instead cost pass B more than the
            // second store costs here); tangential halves stay in their own
            // slots
            const bool own_side = v.kind == ITEM_TB_OWN;
            Real* og = fvg + static_cast<size_t>(bp.d0) * nI + v.other;
            Real* oh = fvh + static_cast<size_t>(bp.d0) * nI + v.other;
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (FULL || j < bp.nb) {
                    const double x = sm.x1[bp.ix0 + j];
                    const double xs = xs_row(x, v.S[0], p2, p3);
                    const bool own_up = xs >= kVSmall, nei_up = xs < -kVSmall;
                    const bool up = own_side ? own_up : nei_up;
                    const bool tang = !own_up && !nei_up;
                    // the downwind side contributes nothing; neighbouring
                    // tile-boundary faces share their orientation, so whole
                    // warps skip together
                    if (up || tang) {
                        const Real cs = up ? Real(1) : Real(0.5);
                        Real gg, hh;
                        recon<D, Real, NB, HZ>(sm, j, v.la, Real(v.da[0]) - hdt * Real(x), ay, az, gg, hh);
                        gg *= cs;
                        hh *= cs;
                        // this side's share of the face value and of its reference part
                        const double gr = double(cs) * dv_ref<Real>(m.gref, bp.d0 + j);
                        const double hr = double(cs) * dv_ref<Real>(m.href, bp.d0 + j);
                        row_add<HZ>(rs, sm.w1[bp.ix0 + j], x, plus_ref<Real>(double(gg), gr), plus_ref<Real>(double(hh), hr));
                        fg[j * nI] = gg;
                        if (!HZ) fh[j * nI] = hh;
                        if (up) {
                            og[j * nI] = gg;
                            if (!HZ) oh[j * nI] = hh;
                        }
                    }
                }
            }
        } else {
            // mesh boundary, by patch type (fvDVM.C:866-1027)
            const int pt = v.ptype;
            const bool wall = pt == DUGKS_PATCH_MAXWELL_WALL;
            const bool zero_grad = pt == DUGKS_PATCH_ZERO_GRADIENT;
            const bool sym = pt == DUGKS_PATCH_SYMMETRY || pt == DUGKS_PATCH_DVM_SYMMETRY;
            // incoming DFs computed here: far field and pressure patches
            // rho_b M(xi; U_owner, T_b) (fvDVM.C:926-938); mixed patches the
            // Maxwellian of the patch rho, U, T kept from the start
            // (discreteVelocity.C:226-258)
            const bool eq_in = !wall && !zero_grad && !sym;
            double bK = 0, bInv = 0, bHf = 0, bU[3] = {0, 0, 0};
            if (eq_in) {
                const BRec* br = a.ds.brec + v.face;
                bK = __ldg(&br->rho_in) * __ldg(&br->K_in);
                bInv = __ldg(&br->invRT_in);
                bHf = __ldg(&br->hfac);
                if (pt == DUGKS_PATCH_MIXED) {
                    for (int i = 0; i < 3; ++i) bU[i] = __ldg(&br->U[i]);
                } else {
                    const int own = chk(__ldg(m.bface_owner + v.face), 0, m.nC, a.ds.err);
                    const size_t n = static_cast<size_t>(m.nC);
                    for (int i = 0; i < 3; ++i) bU[i] = __ldg(a.ds.cellrec + (REC_UX + i) * n + own);
                }
            }
            const double cyz = (q.Y - bU[1]) * (q.Y - bU[1]) + (q.Z - bU[2]) * (q.Z - bU[2]);
            if (zero_grad || sym) {
                // (a loop of its own: the rare types stay off the common path)
#pragma unroll 1
                for (int j = 0; j < NB; ++j) {
                    if (FULL || j < bp.nb) {
                        const double x = sm.x1[bp.ix0 + j];
                        const double xs = xs_row(x, v.S[0], p2, p3);
                        const double wx = sm.w1[bp.ix0 + j];
                        Real gg, hh;
                        if (zero_grad) {
                            // every DV: the owner cell's gbar+ (fvDVM.C:887-891)
                            gg = sm.gB[j * kSL + v.la];
                            hh = HZ ? Real(0) : sm.hB[j * kSL + v.la];
                        } else if (xs > -kVSmall) {
                            // outgoing and tangential: upwind from the owner
                            // (fvDVM.C:1013-1023); incoming ones are the mirror
                            // DVs' values, added by the symmetry pass after this one
                            recon<D, Real, NB, HZ>(sm, j, v.la, Real(v.da[0]) - hdt * Real(x), ay, az, gg, hh);
                        } else {
                            continue;
                        }
                        const double gr = dv_ref<Real>(m.gref, bp.d0 + j), hr = dv_ref<Real>(m.href, bp.d0 + j);
                        row_add<HZ>(rs, wx, x, plus_ref<Real>(double(gg), gr), plus_ref<Real>(double(hh), hr));
                        fg[j * nI] = gg;
                        if (!HZ) fh[j * nI] = hh;
                    }
                }
            } else
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (FULL || j < bp.nb) {
                    const double x = sm.x1[bp.ix0 + j];
                    const double xs = xs_row(x, v.S[0], p2, p3);
                    const double wx = sm.w1[bp.ix0 + j];
                    const double gr = dv_ref<Real>(m.gref, bp.d0 + j), hr = dv_ref<Real>(m.href, bp.d0 + j);
                    if (xs > 0) {
                        // outgoing: upwind from the owner (fvDVM.C:916-923, :950-961)
                        Real gg, hh;
                        recon<D, Real, NB, HZ>(sm, j, v.la, Real(v.da[0]) - hdt * Real(x), ay, az, gg, hh);
                        const double aw =
                            row_add<HZ>(rs, wx, x, plus_ref<Real>(double(gg), gr), plus_ref<Real>(double(hh), hr));
                        if (wall) rs.O = fma(aw, xs, rs.O);
                        fg[j * nI] = gg;
                        if (!HZ) fh[j * nI] = hh;
                    } else if (eq_in) {
                        const double cx = x - bU[0];
                        const double ge = bK * exp(-0.5 * (cx * cx + cyz) * bInv);
                        // rounded as pass B rounds the same incoming DF
                        row_add<HZ>(rs, wx, x, plus_ref<Real>(double(Real(minus_ref<Real>(ge, gr))), gr),
                                plus_ref<Real>(double(Real(minus_ref<Real>(ge * bHf, hr))), hr));
                    }
                    // incoming wall DFs enter through rho_w in the face combine
                }
            }
        }
        row_fold<D>(acc, rs, q);
    }
    if (has_item) {
        if constexpr (sizeof(Real) == 4) {
            // a tile-internal face counts every DV of the chunk in full: its
            // moments gain the reference's chunk moments once
            if (v.kind == ITEM_TILE_INTERNAL) {
                const double* rm = a.ds.refmom + static_cast<size_t>(blockIdx.y) * kNM;
#pragma unroll
                for (int j = 0; j < 14; ++j) acc[j] += __ldg(rm + j);
            }
        }
        double* p = a.ds.partF + (static_cast<size_t>(blockIdx.y) * m.n_items + v.gi) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) p[j] = acc[j];
    }
}

// ---------------------------------------------------------------------
// Pass B: face relaxation, volume update, raw cell moments
// ---------------------------------------------------------------------
// faces of a cell whose flux list stays in registers (hex cells have 6)
constexpr int kRegFaces = 6;

// v with its sign flipped when neg is 1
__device__ __forceinline__ double flip_sign(double v, unsigned neg) {
    return __hiloint2double(__double2hiint(v) ^ static_cast<int>(neg << 31), __double2loint(v));
}
__device__ __forceinline__ float flip_sign(float v, unsigned neg) {
    return __int_as_float(__float_as_int(v) ^ static_cast<int>(neg << 31));
}

// cp.async of an item's own face-value slot and Maxwellian x factors for a
// batch (each thread stages and later reads only its own item's entries)
template <typename Real, int NB, bool FULL, bool HZ>
__device__ __forceinline__ void stage_items(const SmemB<Real, NB, HZ>& sm, const BatchPos& bp, const Real* __restrict__ fvg,
                                            const Real* __restrict__ fvh, const double* __restrict__ ftab, size_t nI,
                                            int it, int gi, bool x_res) {
    const size_t base = static_cast<size_t>(bp.d0) * nI + gi;
    const size_t tb = static_cast<size_t>(bp.ix0) * nI + gi;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        if (FULL || j < bp.nb) {
            cp_async(sm.st + j * kSI + it, fvg + base + j * nI);
            if (!HZ) cp_async(sm.st + (NB + j) * kSI + it, fvh + base + j * nI);
            if (!x_res) cp_async(sm.stx + j * kSI + it, ftab + tb + j * nI);
        }
    }
    cp_commit();
}

// the L0 cell's g~, h~ and Maxwellian x factors of its DVs of a batch, into
// registers one batch ahead
template <typename Real, int NB, bool FULL, bool HZ>
__device__ __forceinline__ void fetch_cells(const BatchPos& bp, const Real* __restrict__ g, const Real* __restrict__ h,
                                            const double* __restrict__ ctab, size_t nC, int c, int part, Real* pg,
                                            Real* ph, double* pe) {
    constexpr int H = (NB + kParts0 - 1) / kParts0;
#pragma unroll
    for (int jj = 0; jj < H; ++jj) {
        const int j = part + kParts0 * jj;
        if (FULL || j < bp.nb) {
            const size_t idx = static_cast<size_t>(bp.d0 + j) * nC + c;
            pg[jj] = __ldg(g + idx);
            ph[jj] = HZ ? Real(0) : __ldg(h + idx);
            pe[jj] = __ldg(ctab + static_cast<size_t>(bp.ix0 + j) * nC + c);
        }
    }
}

// HZ: as for pass A, g alone (h stays identically zero)
template <int D, typename Real, int NB, bool FULL, bool HZ>
__global__ void __launch_bounds__(kThreads, 1) k_pass_b(const StepArgs a) {
    const DevMesh& m = a.dm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SmemB<Real, NB, HZ> sm = carve_b<Real, NB, HZ>(smem_raw);
    const TileRange t = tile_range(m, a.chunk_begin);
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    Real* gn = reinterpret_cast<Real*>(a.ds.g[1 - a.ds.cur]);
    Real* hn = reinterpret_cast<Real*>(a.ds.h[1 - a.ds.cur]);
    const Real* fvg = reinterpret_cast<const Real*>(a.ds.fvg);
    const Real* fvh = reinterpret_cast<const Real*>(a.ds.fvh);
    const double* ctab = a.ds.ctab;
    const double* ftab = a.ds.ftab;
    const double K3D = m.K + 3.0 - m.D, c0h = -(m.D * (m.K + 3.0 - m.D) + 2.0 * m.K);
    const size_t nI = static_cast<size_t>(m.n_items), nC = static_cast<size_t>(m.nC);
    load_dv_tables(m, sm.x1, sm.w1);

    // item of stage 3; its face record (item order) goes to shared memory
    const int it = threadIdx.x;
    const bool has_item = it < t.nit;
    const int gi = t.ioff + (has_item ? it : 0);
    int kind = 0, other = 0;
    double S[3] = {0, 0, 0};
    if (has_item) {
        kind = __ldg(m.it_meta + gi) & 15;
        other = __ldg(m.it_other + gi);
        if (kind == ITEM_TB_OWN || kind == ITEM_TB_NEI) other = chk(other, 0, m.n_items, a.ds.err);
#pragma unroll
        for (int q = 0; q < 3; ++q) S[q] = __ldg(m.it_geo + q * nI + gi);
        stash_rec(sm.frec, kSI, it, a.ds.facerec, nI, gi);
    }
    // e_x of this thread's item for every node, when the table fits (each
    // thread reads back only its own item's column)
    // (a variant whose table is only a batch wide stages: decided at compile time)
    constexpr int kXR = SmemB<Real, NB, HZ>::XR;
    const bool x_res = (kXR > NB || NB >= 16) && m.n1d <= kXR;
    if (x_res && has_item)
        for (int ix = 0; ix < m.n1d; ++ix) sm.stx[ix * kSI + it] = __ldg(ftab + static_cast<size_t>(ix) * nI + gi);
    // L0 cell of stage 4 (kParts0 threads per cell, DVs interleaved)
    const int lc = threadIdx.x % kS0, part = threadIdx.x / kS0;
    const bool has_cell = lc < t.n0;
    const int c = t.b + (has_cell ? lc : 0);
    if (has_cell && part == 0) stash_rec(sm.crec, kS0, lc, a.ds.cellrec, nC, c);
    const double dtV = has_cell ? step_dt(a) * __ldg(m.dtV + c) : 0.0;
    // flux list of the cell: item slot and sign (owner side: outflow, negated
    // by flipping the sign bit); absent entries read the zero slot kSI - 1,
    // which no item uses
    int ent_off[kRegFaces];
    unsigned ent_neg[kRegFaces];
#pragma unroll
    for (int s = 0; s < kRegFaces; ++s) {
        const int e = (has_cell && s < m.nf_max) ? __ldg(m.cf_item + static_cast<size_t>(s) * nC + c) : 0;
        ent_off[s] = e == 0 ? kSI - 1 : chk((e > 0 ? e : -e) - 1, 0, t.nit, a.ds.err);
        ent_neg[s] = e < 0 ? 1u : 0u;
    }
    if (threadIdx.x == kThreads - 1) {
        for (int j = 0; j < NB; ++j) {
            sm.Fg[j * kSI + kSI - 1] = Real(0);
            if (!HZ) sm.Fh[j * kSI + kSI - 1] = Real(0);
        }
    }
    double acc[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;

    constexpr int H = (NB + kParts0 - 1) / kParts0;
    Real pg[H], ph[H];
    double pe[H];
    BatchWalk<D, NB> walk(t.r0, m.n1d, m.row_base), ahead(t.r0, m.n1d, m.row_base);
    const int nbt = (t.r1 - t.r0) * walk.nbr;
    if (nbt > 0) {
        if (has_item) stage_items<Real, NB, FULL, HZ>(sm, walk.pos(), fvg, fvh, ftab, nI, it, gi, x_res);
        if (has_cell) fetch_cells<Real, NB, FULL, HZ>(walk.pos(), g, h, ctab, nC, c, part, pg, ph, pe);
    }
    for (int k = 0; k < nbt; ++k, walk.next()) {
        const BatchPos bp = walk.pos();
        if (k + 1 < nbt) ahead.next();
        __syncthreads();  // records stashed; the previous batch's stage 4 is done with the fluxes
        const RowConst q = row_const<D>(sm.x1, sm.w1, bp);
        // stage 3: relaxed face DFs and fluxes of the items
        if (has_item) {
            const double p2 = __dmul_rn(q.Y, S[1]);
            const double p3 = D == 3 ? __dmul_rn(q.Z, S[2]) : 0.0;
            const double ey = __ldg(ftab + static_cast<size_t>(m.n1d + bp.iy) * nI + gi);
            const double ez = D == 3 ? __ldg(ftab + static_cast<size_t>(2 * m.n1d + bp.iz) * nI + gi) : 1.0;
            const Shk<double> fs = shk_from<D, double>(sm.frec, kSI, it, q, ey, ez);
            const double* sx = sm.stx + (x_res ? bp.ix0 * kSI : 0) + it;
            cp_wait_all();  // this item's staged entries of batch k
            const Real* sg = sm.st + it;
            if (kind != ITEM_MESH_BOUNDARY) {
                // internal and tile-boundary faces: the staged slot holds the
                // upwind face value; on an exactly tangential tile-boundary
                // face it holds this side's half and the other slot the rest
                const bool tb = kind != ITEM_TILE_INTERNAL;
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    if (FULL || j < bp.nb) {
                        const double x = sm.x1[bp.ix0 + j];
                        const double xs = xs_row(x, S[0], p2, p3);
                        Real rg = sg[j * kSI], rh = HZ ? Real(0) : sg[(NB + j) * kSI];
                        if (tb && !(xs >= kVSmall) && !(xs < -kVSmall)) {
                            const size_t o = static_cast<size_t>(bp.d0 + j) * nI + other;
                            rg += __ldg(fvg + o);
                            if (!HZ) rh += __ldg(fvh + o);
                        }
                        const double gr = dv_ref<Real>(m.gref, bp.d0 + j), hr = dv_ref<Real>(m.href, bp.d0 + j);
                        double gf, hf;
                        shk_relax<D, double>(fs, x, sx[j * kSI], plus_ref<Real>(double(rg), gr),
                                             plus_ref<Real>(double(rh), hr), K3D, c0h, gf, hf);
                        // the reference part of the fluxes cancels over a closed cell (sum of +-Sf = 0)
                        sm.Fg[j * kSI + it] = Real(xs * minus_ref<Real>(gf, gr));
                        if (!HZ) sm.Fh[j * kSI + it] = Real(xs * minus_ref<Real>(hf, hr));
                    }
                }
            } else {
                // mesh boundary, by patch type.  Outgoing DFs are relaxed with
                // the boundary face's record, whose h uses the internal-face T
                // at the patch-local index (fvDVM.C:1367, :1413, :1429-1444).
                // Incoming ones are not relaxed: wall rho_w M(U_w, T_w)
                // (fvDVM.C:1079-1092), far field and pressure rho_b M(U_owner,
                // T_b) (fvDVM.C:926-938) and mixed rho_b M(U_b, T_b) computed
                // here; zero-gradient and symmetry ones come from the face-value
                // buffer.  DVMsymmetry relaxes every DV once more
                // (fvDVM.C:1445-1453).  Read per batch: boundary items are few.
                const int face = chk(__ldg(m.it_face + gi), 0, m.nBF, a.ds.err);
                const int pt = __ldg(m.it_meta + gi) >> 4;
                const bool stored_in = pt == DUGKS_PATCH_ZERO_GRADIENT || pt == DUGKS_PATCH_SYMMETRY ||
                                       pt == DUGKS_PATCH_DVM_SYMMETRY;
                const bool again = pt == DUGKS_PATCH_DVM_SYMMETRY;
                const BRec* br = a.ds.brec + face;
                const double bK = br->rho_in * __ldg(&br->K_in);
                const double bInv = __ldg(&br->invRT_in), bHf = __ldg(&br->hfac);
                double bU[3];
                if (pt == DUGKS_PATCH_MAXWELL_WALL || pt == DUGKS_PATCH_MIXED) {
                    for (int i = 0; i < 3; ++i) bU[i] = __ldg(&br->U[i]);
                } else {
                    const int own = chk(__ldg(m.bface_owner + face), 0, m.nC, a.ds.err);
                    for (int i = 0; i < 3; ++i) bU[i] = __ldg(a.ds.cellrec + (REC_UX + i) * nC + own);
                }
                const double cyz = (q.Y - bU[1]) * (q.Y - bU[1]) + (q.Z - bU[2]) * (q.Z - bU[2]);
                if (again) {
                    // DVMsymmetry: every DV relaxed once more after the outgoing
                    // ones (a loop of its own: the rare type stays off the common path)
#pragma unroll 1
                    for (int j = 0; j < NB; ++j) {
                        if (FULL || j < bp.nb) {
                            const double x = sm.x1[bp.ix0 + j];
                            const double xs = xs_row(x, S[0], p2, p3);
                            const double gr = dv_ref<Real>(m.gref, bp.d0 + j), hr = dv_ref<Real>(m.href, bp.d0 + j);
                            double gf = plus_ref<Real>(double(sg[j * kSI]), gr);
                            double hf = plus_ref<Real>(double(HZ ? Real(0) : sg[(NB + j) * kSI]), hr);
                            if (xs > 0) shk_relax<D, double>(fs, x, sx[j * kSI], gf, hf, K3D, c0h, gf, hf);
                            shk_relax<D, double>(fs, x, sx[j * kSI], gf, hf, K3D, c0h, gf, hf);
                            sm.Fg[j * kSI + it] = Real(xs * minus_ref<Real>(gf, gr));
                            if (!HZ) sm.Fh[j * kSI + it] = Real(xs * minus_ref<Real>(hf, hr));
                        }
                    }
                } else
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    if (FULL || j < bp.nb) {
                        const double x = sm.x1[bp.ix0 + j];
                        const double xs = xs_row(x, S[0], p2, p3);
                        const double gr = dv_ref<Real>(m.gref, bp.d0 + j), hr = dv_ref<Real>(m.href, bp.d0 + j);
                        double gf, hf;
                        if (xs > 0) {
                            shk_relax<D, double>(fs, x, sx[j * kSI], plus_ref<Real>(double(sg[j * kSI]), gr),
                                                 plus_ref<Real>(double(HZ ? Real(0) : sg[(NB + j) * kSI]), hr), K3D, c0h, gf, hf);
                        } else if (stored_in) {
                            gf = plus_ref<Real>(double(sg[j * kSI]), gr);
                            hf = plus_ref<Real>(double(HZ ? Real(0) : sg[(NB + j) * kSI]), hr);
                        } else {
                            const double cx = x - bU[0];
                            const double ge = bK * exp(-0.5 * (cx * cx + cyz) * bInv);
                            gf = plus_ref<Real>(double(Real(minus_ref<Real>(ge, gr))), gr);
                            hf = plus_ref<Real>(double(Real(minus_ref<Real>(ge * bHf, hr))), hr);
                        }
                        sm.Fg[j * kSI + it] = Real(xs * minus_ref<Real>(gf, gr));
                        if (!HZ) sm.Fh[j * kSI + it] = Real(xs * minus_ref<Real>(hf, hr));
                    }
                }
            }
            // this thread has read its staged entries: stage the next batch
            if (k + 1 < nbt) stage_items<Real, NB, FULL, HZ>(sm, ahead.pos(), fvg, fvh, ftab, nI, it, gi, x_res);
        }
        __syncthreads();
        // stage 4: g~ <- -g~/3 + 4/3 gbar+ - dt/V sum_f (+-)(xi.S) g_f, cell moments
        if (has_cell) {
            const double ey = __ldg(ctab + static_cast<size_t>(m.n1d + bp.iy) * nC + c);
            const double ez = D == 3 ? __ldg(ctab + static_cast<size_t>(2 * m.n1d + bp.iz) * nC + c) : 1.0;
            const Shk<double> cs = shk_from<D, double>(sm.crec, kS0, lc, q, ey, ez);
            RowSums rs;
            row_zero(rs);
#pragma unroll
            for (int jj = 0; jj < H; ++jj) {
                const int j = part + kParts0 * jj;
                if (FULL || j < bp.nb) {
                    const Real gt = pg[jj], ht = ph[jj];
                    const double x = sm.x1[bp.ix0 + j];
                    const double gr = dv_ref<Real>(m.gref, bp.d0 + j), hr = dv_ref<Real>(m.href, bp.d0 + j);
                    double gb, hb;
                    shk_relax<D, double>(cs, x, pe[jj], plus_ref<Real>(double(gt), gr), plus_ref<Real>(double(ht), hr),
                                         K3D, c0h, gb, hb);
                    const Real* Fg = sm.Fg + j * kSI;
                    const Real* Fh = HZ ? nullptr : sm.Fh + j * kSI;
                    Real sg = 0, sh = 0;
#pragma unroll
                    for (int s = 0; s < kRegFaces; ++s) {
                        sg += flip_sign(Fg[ent_off[s]], ent_neg[s]);
                        if (!HZ) sh += flip_sign(Fh[ent_off[s]], ent_neg[s]);
                    }
                    for (int s = kRegFaces; s < m.nf_max; ++s) {
                        const int e = __ldg(m.cf_item + static_cast<size_t>(s) * nC + c);
                        if (e != 0) {
                            const int i = chk((e > 0 ? e : -e) - 1, 0, t.nit, a.ds.err);
                            sg += e > 0 ? Fg[i] : -Fg[i];
                            if (!HZ) sh += e > 0 ? Fh[i] : -Fh[i];
                        }
                    }
                    // the update in FP64, one rounding to the storage type; with a
                    // reference, -g/3 + 4/3 gbar+ - ref = -(g - ref)/3 + 4/3 (gbar+ - ref)
                    const Real g_new =
                        Real(fma(-1.0 / 3, double(gt), fma(4.0 / 3, minus_ref<Real>(gb, gr), double(sg) * dtV)));
                    const Real h_new =
                        Real(fma(-1.0 / 3, double(ht), fma(4.0 / 3, minus_ref<Real>(hb, hr), double(sh) * dtV)));
                    const size_t idx = static_cast<size_t>(bp.d0 + j) * nC + c;
                    gn[idx] = g_new;
                    if (!HZ) hn[idx] = h_new;
                    row_add<HZ>(rs, sm.w1[bp.ix0 + j], x, double(g_new), double(h_new));  // reference part below
                }
            }
            row_fold<D>(acc, rs, q);
            // the next batch's cell inputs fly during the barrier and stage 3
            if (k + 1 < nbt) fetch_cells<Real, NB, FULL, HZ>(ahead.pos(), g, h, ctab, nC, c, part, pg, ph, pe);
        }
    }
    // the cell moments of a cell are split over kParts0 threads: reduce them
    // through shared memory in a fixed order
    __syncthreads();
    if (part > 0 && has_cell)
        for (int j = 0; j < 15; ++j) sm.red[((part - 1) * kS0 + lc) * 15 + j] = acc[j];
    __syncthreads();
    if (part == 0 && has_cell) {
        for (int p = 1; p < kParts0; ++p)
            for (int j = 0; j < 15; ++j) acc[j] += sm.red[((p - 1) * kS0 + lc) * 15 + j];
        if constexpr (sizeof(Real) == 4) {
            // FP32 storage: the reference's moments over this chunk's DVs
            const double* rm = a.ds.refmom + static_cast<size_t>(blockIdx.y) * kNM;
            for (int j = 0; j < 14; ++j) acc[j] += __ldg(rm + j);
        }
        double* dst = a.ds.partC + (static_cast<size_t>(blockIdx.y) * m.nC + c) * kNM;
#pragma unroll
        for (int j = 0; j < 15; ++j) dst[j] = acc[j];
    }
}

#include "dugks_passes_gen.cuh"

template <typename K>
cudaError_t set_smem(K* kernel, size_t bytes);

// ---------------------------------------------------------------------
// launch plumbing
// ---------------------------------------------------------------------
constexpr int kNbGen = 8;   // DVs per batch of the general-DV passes

template <int D, typename Real>
cudaError_t launch_gen(const StepArgs& a, bool pass_b, cudaStream_t s) {
    const dim3 grid(a.dm.n_tiles, a.chunks);
    if (!pass_b) k_pass_a_gen<D, Real, kNbGen><<<grid, kThreads, a.smemA, s>>>(a);
    else k_pass_b_gen<D, Real, kNbGen><<<grid, kThreads, a.smemB, s>>>(a);
    return cudaGetLastError();
}

template <int D, typename Real>
cudaError_t configure_gen(const StepArgs& a) {
    cudaError_t e = set_smem(k_pass_a_gen<D, Real, kNbGen>, a.smemA);
    return e != cudaSuccess ? e : set_smem(k_pass_b_gen<D, Real, kNbGen>, a.smemB);
}
template <int D, typename Real, int NA, int NBB, bool HZ>
cudaError_t launch_nb_h(const StepArgs& a, bool pass_b, cudaStream_t s) {
    const dim3 grid(a.dm.n_tiles, a.chunks);
    if constexpr (HZ) {
        if (!pass_b && a.wideA16) {
            k_pass_a<D, Real, 16, true, true><<<grid, kThreads, a.smemA, s>>>(a);
            return cudaGetLastError();
        }
        if constexpr (sizeof(Real) == 4) {
            if (pass_b && a.wideB16) {
                k_pass_b<D, Real, 16, true, true><<<grid, kThreads, a.smemB, s>>>(a);
                return cudaGetLastError();
            }
        }
        if constexpr (sizeof(Real) == 4) {
            // FP32 storage, 20 nodes per dimension: a whole row per batch
            if (a.row20) {
                if (!pass_b) k_pass_a<D, Real, 20, true, true><<<grid, kThreads, a.smemA, s>>>(a);
                else k_pass_b<D, Real, 20, true, true><<<grid, kThreads, a.smemB, s>>>(a);
                return cudaGetLastError();
            }
        }
        // 20 nodes per dimension: two batches of 10 per row (guarded: 10 DVs
        // do not split evenly over the threads of a cell)
        if (a.row10) {
            if (!pass_b) k_pass_a<D, Real, 10, false, true><<<grid, kThreads, a.smemA, s>>>(a);
            else k_pass_b<D, Real, 10, false, true><<<grid, kThreads, a.smemB, s>>>(a);
            return cudaGetLastError();
        }
    }
    if (!pass_b) {
        if (a.fullA) k_pass_a<D, Real, NA, true, HZ><<<grid, kThreads, a.smemA, s>>>(a);
        else k_pass_a<D, Real, NA, false, HZ><<<grid, kThreads, a.smemA, s>>>(a);
    } else {
        if (a.fullB) k_pass_b<D, Real, NBB, true, HZ><<<grid, kThreads, a.smemB, s>>>(a);
        else k_pass_b<D, Real, NBB, false, HZ><<<grid, kThreads, a.smemB, s>>>(a);
    }
    return cudaGetLastError();
}

// h identically zero (StepArgs::hzero) exists in 3-D only
template <int D, typename Real, int NA, int NBB>
cudaError_t launch_nb(const StepArgs& a, bool pass_b, cudaStream_t s) {
    if constexpr (D == 3) {
        if (a.hzero) return launch_nb_h<D, Real, NA, NBB, true>(a, pass_b, s);
    }
    return launch_nb_h<D, Real, NA, NBB, false>(a, pass_b, s);
}

template <int D, typename Real>
cudaError_t launch_pass_d(const StepArgs& a, bool pass_b, cudaStream_t s) {
    using W = Width<Real>;
    if (!pass_b) return a.wideA ? launch_nb<D, Real, W::A1, W::B0>(a, false, s) : launch_nb<D, Real, W::A0, W::B0>(a, false, s);
    return a.wideB ? launch_nb<D, Real, W::A0, W::B1>(a, true, s) : launch_nb<D, Real, W::A0, W::B0>(a, true, s);
}

template <int D, typename Real>
void smem_d(bool wideA, bool wideB, size_t* smemA, size_t* smemB) {
    *smemA = wideA ? SmemA<D, Real, Width<Real>::A1>::bytes() : SmemA<D, Real, Width<Real>::A0>::bytes();
    *smemB = wideB ? SmemB<Real, Width<Real>::B1>::bytes() : SmemB<Real, Width<Real>::B0>::bytes();
}

template <typename K>
cudaError_t set_smem(K* kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

template <int D, typename Real, int NA, int NBB, bool HZ>
cudaError_t configure_nb_h(const StepArgs& a, bool pass_b) {
    if (!pass_b)
        return a.fullA ? set_smem(k_pass_a<D, Real, NA, true, HZ>, a.smemA)
                       : set_smem(k_pass_a<D, Real, NA, false, HZ>, a.smemA);
    return a.fullB ? set_smem(k_pass_b<D, Real, NBB, true, HZ>, a.smemB)
                   : set_smem(k_pass_b<D, Real, NBB, false, HZ>, a.smemB);
}

template <int D, typename Real, int NA, int NBB>
cudaError_t configure_nb(const StepArgs& a, bool pass_b) {
    cudaError_t e = configure_nb_h<D, Real, NA, NBB, false>(a, pass_b);
    if constexpr (D == 3) {
        if (e == cudaSuccess) e = configure_nb_h<D, Real, NA, NBB, true>(a, pass_b);
        if (e == cudaSuccess && !pass_b)
            e = set_smem(k_pass_a<D, Real, 16, true, true>, SmemA<D, Real, 16, true>::bytes());
        if (e == cudaSuccess)
            e = pass_b ? set_smem(k_pass_b<D, Real, 10, false, true>, SmemB<Real, 10, true>::bytes())
                       : set_smem(k_pass_a<D, Real, 10, false, true>, SmemA<D, Real, 10, true>::bytes());
        if constexpr (sizeof(Real) == 4) {
            if (e == cudaSuccess && pass_b)
                e = set_smem(k_pass_b<D, Real, 16, true, true>, SmemB<Real, 16, true>::bytes());
            if (e == cudaSuccess)
                e = pass_b ? set_smem(k_pass_b<D, Real, 20, true, true>, SmemB<Real, 20, true>::bytes())
                           : set_smem(k_pass_a<D, Real, 20, true, true>, SmemA<D, Real, 20, true>::bytes());
        }
    }
    return e;
}

template <int D, typename Real>
cudaError_t configure_d(const StepArgs& a) {
    using W = Width<Real>;
    cudaError_t e = a.wideA ? configure_nb<D, Real, W::A1, W::B0>(a, false) : configure_nb<D, Real, W::A0, W::B0>(a, false);
    if (e != cudaSuccess) return e;
    return a.wideB ? configure_nb<D, Real, W::A0, W::B1>(a, true) : configure_nb<D, Real, W::A0, W::B0>(a, true);
}

// padding of the last batch of a row of n1d DVs at width nb
int row_waste(int n1d, int nb) { return (n1d + nb - 1) / nb * nb - n1d; }

}  // namespace

// every launched layout fits the 227 KB of shared memory a B200 CTA may
// opt into (cudaFuncAttributeMaxDynamicSharedMemorySize)
constexpr size_t kSmemMax = 232448;
template <int D, typename Real>
constexpr bool fits_d() {
    return SmemA<D, Real, 8>::bytes() <= kSmemMax && SmemA<D, Real, 8, true>::bytes() <= kSmemMax &&
           SmemB<Real, 8>::bytes() <= kSmemMax && SmemB<Real, 8, true>::bytes() <= kSmemMax &&
           SmemA<3, Real, 16, true>::bytes() <= kSmemMax && SmemA<3, Real, 10, true>::bytes() <= kSmemMax &&
           SmemB<Real, 10, true>::bytes() <= kSmemMax && SmemAG<D, Real, kNbGen>::bytes() <= kSmemMax &&
           SmemBG<Real, kNbGen>::bytes() <= kSmemMax;
}
static_assert(fits_d<2, double>() && fits_d<3, double>() && fits_d<2, float>() && fits_d<3, float>(),
              "a pass layout exceeds the shared memory of a CTA");
static_assert(SmemB<float, 16, true>::bytes() <= kSmemMax && SmemA<3, float, 20, true>::bytes() <= kSmemMax &&
                  SmemB<float, 20, true>::bytes() <= kSmemMax,
              "a wide FP32 pass layout exceeds the shared memory of a CTA");

cudaError_t launch_pass(const StepArgs& a, int precision, bool pass_b, cudaStream_t s) {
    if (a.dm.general_dv) {
        if (precision == DUGKS_FP64)
            return a.dm.D == 3 ? launch_gen<3, double>(a, pass_b, s) : launch_gen<2, double>(a, pass_b, s);
        return a.dm.D == 3 ? launch_gen<3, float>(a, pass_b, s) : launch_gen<2, float>(a, pass_b, s);
    }
    if (precision == DUGKS_FP64)
        return a.dm.D == 3 ? launch_pass_d<3, double>(a, pass_b, s) : launch_pass_d<2, double>(a, pass_b, s);
    return a.dm.D == 3 ? launch_pass_d<3, float>(a, pass_b, s) : launch_pass_d<2, float>(a, pass_b, s);
}

void pass_config(int D, int precision, int n1d, StepArgs* a) {
    const bool f64 = precision == DUGKS_FP64;
    if (a->dm.general_dv) {
        a->wideA = a->wideB = a->fullA = a->fullB = 0;
        if (f64) {
            a->smemA = D == 3 ? SmemAG<3, double, kNbGen>::bytes() : SmemAG<2, double, kNbGen>::bytes();
            a->smemB = SmemBG<double, kNbGen>::bytes();
        } else {
            a->smemA = D == 3 ? SmemAG<3, float, kNbGen>::bytes() : SmemAG<2, float, kNbGen>::bytes();
            a->smemB = SmemBG<float, kNbGen>::bytes();
        }
        return;
    }
    const int a0 = f64 ? Width<double>::A0 : Width<float>::A0, a1 = f64 ? Width<double>::A1 : Width<float>::A1;
    const int b0 = f64 ? Width<double>::B0 : Width<float>::B0, b1 = f64 ? Width<double>::B1 : Width<float>::B1;
    // the wide batch unless it pads the rows more than the narrow one;
    // rows that split into whole batches take the unguarded kernels
    a->wideA = row_waste(n1d, a1) <= row_waste(n1d, a0) ? 1 : 0;
    a->wideB = row_waste(n1d, b1) <= row_waste(n1d, b0) ? 1 : 0;
    a->fullA = row_waste(n1d, a->wideA ? a1 : a0) == 0 ? 1 : 0;
    a->fullB = row_waste(n1d, a->wideB ? b1 : b0) == 0 ? 1 : 0;
    if (f64) {
        if (D == 3) smem_d<3, double>(a->wideA, a->wideB, &a->smemA, &a->smemB);
        else smem_d<2, double>(a->wideA, a->wideB, &a->smemA, &a->smemB);
    } else {
        if (D == 3) smem_d<3, float>(a->wideA, a->wideB, &a->smemA, &a->smemB);
        else smem_d<2, float>(a->wideA, a->wideB, &a->smemA, &a->smemB);
    }
    // the g-only instantiations' own sizes (no h arrays; pass B keeps its
    // items' e_x table resident in part of that room)
    if (D == 3 && a->hzero) {
        using WD = Width<double>;
        using WF = Width<float>;
        if (f64) {
            a->smemA = a->wideA ? SmemA<3, double, WD::A1, true>::bytes() : SmemA<3, double, WD::A0, true>::bytes();
            a->smemB = a->wideB ? SmemB<double, WD::B1, true>::bytes() : SmemB<double, WD::B0, true>::bytes();
        } else {
            a->smemA = a->wideA ? SmemA<3, float, WF::A1, true>::bytes() : SmemA<3, float, WF::A0, true>::bytes();
            a->smemB = a->wideB ? SmemB<float, WF::B1, true>::bytes() : SmemB<float, WF::B0, true>::bytes();
        }
    }
    // g-only pass A in batches of 16 DVs (a whole row) for 16 nodes per
    // dimension: half the per-batch work and barriers per DV, and the
    // shared memory the h arrays would take holds the wider batch
    a->wideA16 = a->wideB16 = a->row10 = a->row20 = 0;
    if (D == 3 && a->hzero && n1d == 20) {
        if (f64) {
            // both passes in batches of 10 DVs: two per row instead of 8 + 8 + 4
            a->row10 = 1;
            a->smemA = SmemA<3, double, 10, true>::bytes();
            a->smemB = SmemB<double, 10, true>::bytes();
        } else {
            // FP32 storage: a whole row per batch (the 20-wide FP64 staging
            // does not fit in shared memory)
            a->row20 = 1;
            a->smemA = SmemA<3, float, 20, true>::bytes();
            a->smemB = SmemB<float, 20, true>::bytes();
        }
    }
    if (D == 3 && a->hzero && n1d == 16) {
        a->wideA16 = 1;
        a->smemA = f64 ? SmemA<3, double, 16, true>::bytes() : SmemA<3, float, 16, true>::bytes();
        // pass B likewise with FP32 storage (in FP64 the 16-wide staging does
        // not fit in shared memory)
        if (!f64) {
            a->wideB16 = 1;
            a->smemB = SmemB<float, 16, true>::bytes();
        }
    }
}

cudaError_t configure_kernels(int precision, const StepArgs& a) {
    if (a.dm.general_dv) {
        if (precision == DUGKS_FP64) return a.dm.D == 3 ? configure_gen<3, double>(a) : configure_gen<2, double>(a);
        return a.dm.D == 3 ? configure_gen<3, float>(a) : configure_gen<2, float>(a);
    }
    if (precision == DUGKS_FP64) return a.dm.D == 3 ? configure_d<3, double>(a) : configure_d<2, double>(a);
    return a.dm.D == 3 ? configure_d<3, float>(a) : configure_d<2, float>(a);
}

}  // namespace dugks

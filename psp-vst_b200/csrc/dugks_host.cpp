// Host-side preparation of the DUGKS step: OpenFOAM mesh geometry,
// surface-interpolation weights, least-squares gradient vectors, and the
// tile layout the device passes work on.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>

#include "dugks_internal.h"

namespace {

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double magsqr3(const double* a) { return dot3(a, a); }

// symmetric tensor (xx xy xz yy yz zz) inverse by the adjugate
void sym_inverse(const double* a, double* r) {
    const double xx = a[0], xy = a[1], xz = a[2], yy = a[3], yz = a[4], zz = a[5];
    const double det = xx * yy * zz + xy * yz * xz + xz * xy * yz - xx * yz * yz - xy * xy * zz - xz * yy * xz;
    r[0] = (yy * zz - yz * yz) / det;
    r[1] = (xz * yz - xy * zz) / det;
    r[2] = (xy * yz - xz * yy) / det;
    r[3] = (xx * zz - xz * xz) / det;
    r[4] = (xy * xz - xx * yz) / det;
    r[5] = (xx * yy - xy * xy) / det;
}

void sym_apply(const double* t, const double* d, double* o) {
    o[0] = t[0] * d[0] + t[1] * d[1] + t[2] * d[2];
    o[1] = t[1] * d[0] + t[3] * d[1] + t[4] * d[2];
    o[2] = t[2] * d[0] + t[4] * d[1] + t[5] * d[2];
}

uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

}  // namespace

extern "C" int dugks_mesh_geometry(int32_t n_points, const double* p, int32_t n_faces, const int64_t* fo,
                                   const int64_t* fp, const int64_t* owner, int32_t n_internal,
                                   const int64_t* neighbour, int32_t n_cells, double* Cf, double* Sf, double* C,
                                   double* V) {
    if (!p || !fo || !fp || !owner || (n_internal && !neighbour) || !Cf || !Sf || !C || !V || n_cells <= 0 ||
        n_faces < n_internal || n_points <= 0)
        return DUGKS_ERR_ARG;
    // face centres and area vectors: triangle fan about the point average
    for (int32_t f = 0; f < n_faces; ++f) {
        const int64_t b = fo[f], e = fo[f + 1];
        const int np = static_cast<int>(e - b);
        if (np < 3) return DUGKS_ERR_ARG;
        for (int64_t k = b; k < e; ++k)
            if (fp[k] < 0 || fp[k] >= n_points) return DUGKS_ERR_ARG;
        if (np == 3) {
            const double *a = p + 3 * fp[b], *bb = p + 3 * fp[b + 1], *c = p + 3 * fp[b + 2];
            const double u[3] = {bb[0] - a[0], bb[1] - a[1], bb[2] - a[2]};
            const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            for (int k = 0; k < 3; ++k) Cf[3 * f + k] = (1.0 / 3.0) * (a[k] + bb[k] + c[k]);
            Sf[3 * f + 0] = 0.5 * (u[1] * v[2] - u[2] * v[1]);
            Sf[3 * f + 1] = 0.5 * (u[2] * v[0] - u[0] * v[2]);
            Sf[3 * f + 2] = 0.5 * (u[0] * v[1] - u[1] * v[0]);
            continue;
        }
        double fc[3] = {0, 0, 0};
        for (int i = 0; i < np; ++i)
            for (int k = 0; k < 3; ++k) fc[k] += p[3 * fp[b + i] + k];
        for (int k = 0; k < 3; ++k) fc[k] /= np;
        double sn[3] = {0, 0, 0}, sa = 0, sac[3] = {0, 0, 0};
        for (int i = 0; i < np; ++i) {
            const double* pi = p + 3 * fp[b + i];
            const double* pn = p + 3 * fp[b + (i + 1) % np];
            double c[3], u[3], v[3];
            for (int k = 0; k < 3; ++k) {
                c[k] = pi[k] + pn[k] + fc[k];
                u[k] = pn[k] - pi[k];
                v[k] = fc[k] - pi[k];
            }
            const double n[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
            const double a = std::sqrt(magsqr3(n));
            for (int k = 0; k < 3; ++k) {
                sn[k] += n[k];
                sac[k] += a * c[k];
            }
            sa += a;
        }
        for (int k = 0; k < 3; ++k) {
            Cf[3 * f + k] = sa < 1e-150 ? fc[k] : (1.0 / 3.0) * sac[k] / sa;
            Sf[3 * f + k] = sa < 1e-150 ? 0.0 : 0.5 * sn[k];
        }
    }
    // cell centres and volumes: face pyramids about the face-centre average
    std::vector<double> est(3 * static_cast<size_t>(n_cells), 0.0);
    std::vector<int> nf(n_cells, 0);
    for (int32_t f = 0; f < n_faces; ++f) {
        if (owner[f] < 0 || owner[f] >= n_cells) return DUGKS_ERR_ARG;
        for (int k = 0; k < 3; ++k) est[3 * owner[f] + k] += Cf[3 * f + k];
        nf[owner[f]]++;
    }
    for (int32_t f = 0; f < n_internal; ++f) {
        if (neighbour[f] < 0 || neighbour[f] >= n_cells) return DUGKS_ERR_ARG;
        for (int k = 0; k < 3; ++k) est[3 * neighbour[f] + k] += Cf[3 * f + k];
        nf[neighbour[f]]++;
    }
    for (int32_t c = 0; c < n_cells; ++c) {
        if (nf[c] == 0) return DUGKS_ERR_ARG;
        for (int k = 0; k < 3; ++k) est[3 * c + k] /= nf[c];
    }
    std::fill(C, C + 3 * static_cast<size_t>(n_cells), 0.0);
    std::fill(V, V + n_cells, 0.0);
    auto pyramid = [&](int32_t f, int64_t c, double sgn) {
        const double d[3] = {sgn * (Cf[3 * f] - est[3 * c]), sgn * (Cf[3 * f + 1] - est[3 * c + 1]),
                             sgn * (Cf[3 * f + 2] - est[3 * c + 2])};
        const double pyr3 = dot3(Sf + 3 * f, d);
        for (int k = 0; k < 3; ++k) C[3 * c + k] += pyr3 * ((3.0 / 4.0) * Cf[3 * f + k] + (1.0 / 4.0) * est[3 * c + k]);
        V[c] += pyr3;
    };
    for (int32_t f = 0; f < n_faces; ++f) pyramid(f, owner[f], 1.0);
    for (int32_t f = 0; f < n_internal; ++f) pyramid(f, neighbour[f], -1.0);
    for (int32_t c = 0; c < n_cells; ++c) {
        if (std::fabs(V[c]) > 1e-300) {
            for (int k = 0; k < 3; ++k) C[3 * c + k] /= V[c];
        } else {
            for (int k = 0; k < 3; ++k) C[3 * c + k] = est[3 * c + k];
        }
        V[c] *= (1.0 / 3.0);
    }
    return DUGKS_OK;
}

namespace dugks {

int set_error(dugks_handle* h, int code, const std::string& msg) {
    if (h) h->last_error = msg;
    return code;
}

// surfaceInterpolation::makeWeights / makeDeltaCoeffs and the weighted
// least-squares vectors of zeroBoundaryVectors.C:90-221 with the
// non-coupled boundary terms restored (stock leastSquares).  The boundary
// d-vector is fvPatch::delta() for non-coupled patches, n (n . (Cf - C)).
void compute_weights_and_ls(dugks_handle* h, int weighting) {
    const int nC = h->nC, nIF = h->nIF, nBF = h->nBF;
    const int nF = nIF + nBF;
    std::vector<double> magSf(nF);
    for (int f = 0; f < nF; ++f) magSf[f] = std::sqrt(magsqr3(&h->Sf[3 * f]));
    h->weights.assign(nIF, 0.0);
    h->dc.assign(nIF, 0.0);
    for (int f = 0; f < nIF; ++f) {
        const double* S = &h->Sf[3 * f];
        const double* co = &h->C[3 * h->owner[f]];
        const double* cn = &h->C[3 * h->neighbour[f]];
        const double* cf = &h->Cf[3 * f];
        const double a[3] = {cf[0] - co[0], cf[1] - co[1], cf[2] - co[2]};
        const double b[3] = {cn[0] - cf[0], cn[1] - cf[1], cn[2] - cf[2]};
        const double so = std::fabs(dot3(S, a)), sn = std::fabs(dot3(S, b));
        h->weights[f] = sn / (so + sn);
        const double d[3] = {cn[0] - co[0], cn[1] - co[1], cn[2] - co[2]};
        h->dc[f] = 1.0 / std::sqrt(magsqr3(d));
    }
    auto face_factor = [&](int f, double wgt, const double* d, bool own_side, bool boundary) {
        if (weighting == DUGKS_LS_MAGSF) {
            const double c = magSf[f] / magsqr3(d);
            if (boundary) return c;
            return own_side ? (1 - wgt) * c : wgt * c;
        }
        if (weighting == DUGKS_LS_INVDIST) return 1.0 / magsqr3(d);
        return 1.0;
    };
    std::vector<double> dd(6 * static_cast<size_t>(nC), 0.0);
    for (int f = 0; f < nIF; ++f) {
        const int64_t o = h->owner[f], n = h->neighbour[f];
        const double d[3] = {h->C[3 * n] - h->C[3 * o], h->C[3 * n + 1] - h->C[3 * o + 1],
                             h->C[3 * n + 2] - h->C[3 * o + 2]};
        const double sq[6] = {d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]};
        const double fo = face_factor(f, h->weights[f], d, true, false);
        const double fn = face_factor(f, h->weights[f], d, false, false);
        for (int k = 0; k < 6; ++k) {
            dd[6 * o + k] += fo * sq[k];
            dd[6 * n + k] += fn * sq[k];
        }
    }
    std::vector<double> bdelta(3 * static_cast<size_t>(nBF));
    for (int b = 0; b < nBF; ++b) {
        const int f = nIF + b;
        const int64_t o = h->owner[f];
        const double* S = &h->Sf[3 * f];
        const double nrm[3] = {S[0] / magSf[f], S[1] / magSf[f], S[2] / magSf[f]};
        const double cfc[3] = {h->Cf[3 * f] - h->C[3 * o], h->Cf[3 * f + 1] - h->C[3 * o + 1],
                               h->Cf[3 * f + 2] - h->C[3 * o + 2]};
        const double dn = dot3(nrm, cfc);
        double* d = &bdelta[3 * b];
        for (int k = 0; k < 3; ++k) d[k] = nrm[k] * dn;
        const double sq[6] = {d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]};
        const double fb = face_factor(f, 1.0, d, true, true);
        for (int k = 0; k < 6; ++k) dd[6 * o + k] += fb * sq[k];
    }
    // OpenFOAM's inverse of a symmTensorField drops the directions whose
    // diagonal is negligible in the first tensor (2-D and 1-D meshes)
    bool rm[3] = {false, false, false};
    if (nC > 0) {
        const double* t = dd.data();
        const double scale = t[0] * t[0] + 2 * t[1] * t[1] + 2 * t[2] * t[2] + t[3] * t[3] + 2 * t[4] * t[4] + t[5] * t[5];
        rm[0] = t[0] * t[0] / scale < 1e-15;
        rm[1] = t[3] * t[3] / scale < 1e-15;
        rm[2] = t[5] * t[5] / scale < 1e-15;
    }
    std::vector<double> inv(6 * static_cast<size_t>(nC));
    for (int c = 0; c < nC; ++c) {
        double a[6];
        std::memcpy(a, &dd[6 * c], sizeof a);
        if (rm[0]) a[0] += 1.0;
        if (rm[1]) a[3] += 1.0;
        if (rm[2]) a[5] += 1.0;
        sym_inverse(a, &inv[6 * c]);
        if (rm[0]) inv[6 * c] -= 1.0;
        if (rm[1]) inv[6 * c + 3] -= 1.0;
        if (rm[2]) inv[6 * c + 5] -= 1.0;
    }
    h->lsP.assign(3 * static_cast<size_t>(nIF), 0.0);
    h->lsN.assign(3 * static_cast<size_t>(nIF), 0.0);
    h->lsB.assign(3 * static_cast<size_t>(nBF), 0.0);
    for (int f = 0; f < nIF; ++f) {
        const int64_t o = h->owner[f], n = h->neighbour[f];
        const double d[3] = {h->C[3 * n] - h->C[3 * o], h->C[3 * n + 1] - h->C[3 * o + 1],
                             h->C[3 * n + 2] - h->C[3 * o + 2]};
        const double fo = face_factor(f, h->weights[f], d, true, false);
        const double fn = -face_factor(f, h->weights[f], d, false, false);
        double a[3], b[3];
        sym_apply(&inv[6 * o], d, a);
        sym_apply(&inv[6 * n], d, b);
        for (int k = 0; k < 3; ++k) {
            h->lsP[3 * f + k] = fo * a[k];
            h->lsN[3 * f + k] = fn * b[k];
        }
    }
    for (int b = 0; b < nBF; ++b) {
        const int f = nIF + b;
        const double* d = &bdelta[3 * b];
        const double fb = face_factor(f, 1.0, d, true, true);
        double a[3];
        sym_apply(&inv[6 * h->owner[f]], d, a);
        for (int k = 0; k < 3; ++k) h->lsB[3 * b + k] = fb * a[k];
    }
}

// Tile layout.  Cells are renumbered along a Morton curve of their centres
// and cut into tiles of `tile_cells` consecutive cells (L0).  Each tile also
// holds its ring L1 (face neighbours of L0 outside it), the gradient
// stencils of its L0 cells and one item per face touching L0.
void build_tiling(dugks_handle* h, int tile_cells) {
    Tiling& t = h->tiling;
    const int nC = h->nC, nIF = h->nIF, nBF = h->nBF;
    // Morton renumbering
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < nC; ++c)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], h->C[3 * c + k]);
            hi[k] = std::max(hi[k], h->C[3 * c + k]);
        }
    double span = 0;
    for (int k = 0; k < 3; ++k) span = std::max(span, hi[k] - lo[k]);
    if (span <= 0) span = 1;
    std::vector<uint64_t> code(nC);
    for (int c = 0; c < nC; ++c) {
        uint64_t q[3];
        for (int k = 0; k < 3; ++k) {
            double x = (h->C[3 * c + k] - lo[k]) / span;
            x = std::min(std::max(x, 0.0), 1.0);
            q[k] = static_cast<uint64_t>(x * 2097151.0);
        }
        code[c] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
    }
    t.perm.resize(nC);
    std::iota(t.perm.begin(), t.perm.end(), 0);
    std::stable_sort(t.perm.begin(), t.perm.end(), [&](int a, int b) { return code[a] < code[b]; });
    t.iperm.assign(nC, 0);
    for (int c = 0; c < nC; ++c) t.iperm[t.perm[c]] = c;

    // cell -> faces (original numbering)
    std::vector<int32_t> cfo(nC + 1, 0);
    for (int f = 0; f < nIF + nBF; ++f) cfo[h->owner[f] + 1]++;
    for (int f = 0; f < nIF; ++f) cfo[h->neighbour[f] + 1]++;
    for (int c = 0; c < nC; ++c) cfo[c + 1] += cfo[c];
    std::vector<int32_t> cfl(cfo[nC]), fill(cfo.begin(), cfo.end() - 1);
    for (int f = 0; f < nIF + nBF; ++f) cfl[fill[h->owner[f]]++] = f;
    for (int f = 0; f < nIF; ++f) cfl[fill[h->neighbour[f]]++] = f;

    t.tile_cells = tile_cells;
    t.n_tiles = (nC + tile_cells - 1) / tile_cells;
    t.tile_begin.assign(t.n_tiles + 1, 0);
    t.tile_loc_off.assign(t.n_tiles + 1, 0);
    t.tile_item_off.assign(t.n_tiles + 1, 0);
    t.loc_cells.clear();
    t.items.clear();
    t.grad_off.assign(nC + 1, 0);
    t.grad_nb.clear();
    t.grad_ls.clear();
    t.cf_off.assign(nC + 1, 0);
    t.cf_item.clear();
    t.max_local = t.max_l0 = t.max_items = 0;
    std::vector<int32_t> tile_of(nC);
    for (int c = 0; c < nC; ++c) tile_of[c] = c / tile_cells;
    // first pass per tile; XB slots assigned afterwards
    std::vector<int32_t> face_item0(nIF + nBF, -1), face_item1(nIF + nBF, -1);
    std::vector<int32_t> local_of(nC, -1);
    for (int ti = 0; ti < t.n_tiles; ++ti) {
        const int b = ti * tile_cells, e = std::min(nC, b + tile_cells), n0 = e - b;
        t.tile_begin[ti] = b;
        t.tile_loc_off[ti] = static_cast<int32_t>(t.loc_cells.size());
        std::vector<int32_t> l1;
        for (int c = b; c < e; ++c) {
            const int o = t.perm[c];
            for (int k = cfo[o]; k < cfo[o + 1]; ++k) {
                const int f = cfl[k];
                if (f >= nIF) continue;
                const int other = h->owner[f] == o ? static_cast<int>(h->neighbour[f]) : static_cast<int>(h->owner[f]);
                const int on = t.iperm[other];
                if (on < b || on >= e) l1.push_back(on);
            }
        }
        std::sort(l1.begin(), l1.end());
        l1.erase(std::unique(l1.begin(), l1.end()), l1.end());
        for (int c = b; c < e; ++c) {
            local_of[c] = c - b;
            t.loc_cells.push_back(c);
        }
        for (size_t i = 0; i < l1.size(); ++i) {
            local_of[l1[i]] = n0 + static_cast<int>(i);
            t.loc_cells.push_back(l1[i]);
        }
        const int item0 = static_cast<int>(t.items.size());
        t.tile_item_off[ti] = item0;
        // items and gradient/flux stencils of the L0 cells
        std::unordered_map<int, int> face_to_local_item;
        for (int c = b; c < e; ++c) {
            const int o = t.perm[c];
            for (int k = cfo[o]; k < cfo[o + 1]; ++k) {
                const int f = cfl[k];
                const bool is_own = h->owner[f] == o;
                if (f < nIF) {
                    const int other = is_own ? static_cast<int>(h->neighbour[f]) : static_cast<int>(h->owner[f]);
                    const int on = t.iperm[other];
                    // gradient stencil
                    t.grad_nb.push_back(local_of[on]);
                    const double* ls = is_own ? &h->lsP[3 * f] : &h->lsN[3 * f];
                    t.grad_ls.insert(t.grad_ls.end(), ls, ls + 3);
                }
                int li;
                auto it = face_to_local_item.find(f);
                if (it != face_to_local_item.end()) {
                    li = it->second;
                } else {
                    Item item{};
                    item.face = f < nIF ? f : f - nIF;
                    item.xb_w = item.xb_r = -1;
                    item.ptype = 0;
                    const int64_t fo_ = h->owner[f];
                    const int own_new = t.iperm[fo_];
                    item.lo = local_of[own_new];
                    for (int q = 0; q < 3; ++q) {
                        item.S[q] = h->Sf[3 * f + q];
                        item.dO[q] = h->Cf[3 * f + q] - h->C[3 * fo_ + q];
                        item.dN[q] = 0.0;
                    }
                    if (f < nIF) {
                        const int64_t fn_ = h->neighbour[f];
                        const int nei_new = t.iperm[fn_];
                        item.ln = local_of[nei_new];
                        for (int q = 0; q < 3; ++q) item.dN[q] = h->Cf[3 * f + q] - h->C[3 * fn_ + q];
                        const bool own_in = own_new >= b && own_new < e;
                        const bool nei_in = nei_new >= b && nei_new < e;
                        item.kind = (own_in && nei_in) ? ITEM_TILE_INTERNAL : (own_in ? ITEM_TB_OWN : ITEM_TB_NEI);
                    } else {
                        item.ln = -1;
                        item.kind = ITEM_MESH_BOUNDARY;
                        item.ptype = h->bface_ptype[f - nIF];
                    }
                    li = static_cast<int>(t.items.size()) - item0;
                    t.items.push_back(item);
                    face_to_local_item[f] = li;
                    const int gi = item0 + li;
                    if (face_item0[f] < 0) face_item0[f] = gi;
                    else face_item1[f] = gi;
                }
                // flux gather: owner subtracts, neighbour adds
                t.cf_item.push_back(is_own ? -(li + 1) : (li + 1));
            }
            t.grad_off[c + 1] = static_cast<int32_t>(t.grad_nb.size());
            t.cf_off[c + 1] = static_cast<int32_t>(t.cf_item.size());
        }
        for (int c = b; c < e; ++c) local_of[c] = -1;
        for (int c : l1) local_of[c] = -1;
        t.max_local = std::max(t.max_local, n0 + static_cast<int>(l1.size()));
        t.max_l0 = std::max(t.max_l0, n0);
        t.max_items = std::max(t.max_items, static_cast<int>(t.items.size()) - item0);
    }
    t.tile_begin[t.n_tiles] = nC;
    t.tile_loc_off[t.n_tiles] = static_cast<int32_t>(t.loc_cells.size());
    t.tile_item_off[t.n_tiles] = static_cast<int32_t>(t.items.size());
    // the per-cell offsets were filled only at c+1; make them cumulative
    // (cells are visited in increasing order, so entries are already set)
    // XB slots of tile-boundary faces: side 0 (owner side) numbered in the
    // order the owner tiles list them, side 1 in the order of the neighbour tiles
    std::vector<int32_t> slot0(nIF, -1), slot1(nIF, -1);
    int n0s = 0, n1s = 0;
    for (size_t i = 0; i < t.items.size(); ++i) {
        Item& it = t.items[i];
        if (it.kind == ITEM_TB_OWN) slot0[it.face] = n0s++;
        else if (it.kind == ITEM_TB_NEI) slot1[it.face] = n1s++;
    }
    t.n_tbf = n0s;
    for (size_t i = 0; i < t.items.size(); ++i) {
        Item& it = t.items[i];
        if (it.kind == ITEM_TB_OWN) {
            it.xb_w = slot0[it.face];
            it.xb_r = slot1[it.face];
        } else if (it.kind == ITEM_TB_NEI) {
            it.xb_w = slot1[it.face];
            it.xb_r = slot0[it.face];
        }
    }
    t.face_items.assign(2 * static_cast<size_t>(nIF + nBF), -1);
    for (int f = 0; f < nIF + nBF; ++f) {
        t.face_items[2 * f] = face_item0[f];
        t.face_items[2 * f + 1] = face_item1[f];
    }
}

}  // namespace dugks

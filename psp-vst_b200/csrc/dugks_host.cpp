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

}  // namespace dugks

namespace {

// Recursive coordinate bisection: cut the cell set along the longest axis
// of its bounding box so that the first part holds a whole number of tiles,
// until every part is one tile.  Consecutive tiles are neighbours in space.
void rcb_order(const std::vector<double>& C, std::vector<int32_t>& idx, size_t b, size_t e, int tile) {
    const size_t n = e - b;
    if (n <= static_cast<size_t>(tile)) return;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (size_t i = b; i < e; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], C[3 * idx[i] + k]);
            hi[k] = std::max(hi[k], C[3 * idx[i] + k]);
        }
    int ax = 0;
    for (int k = 1; k < 3; ++k)
        if (hi[k] - lo[k] > hi[ax] - lo[ax]) ax = k;
    const size_t nt = (n + tile - 1) / tile;
    const size_t nl = (nt / 2) * static_cast<size_t>(tile);
    std::stable_sort(idx.begin() + b, idx.begin() + e, [&](int32_t p, int32_t q) { return C[3 * p + ax] < C[3 * q + ax]; });
    rcb_order(C, idx, b, b + nl, tile);
    rcb_order(C, idx, b + nl, e, tile);
}

// Greedy tile boundaries over the RCB cell order: each tile takes the next
// cells in order while it keeps at most kMaxTile L0 cells, kMaxLocal cells
// with its ring and kMaxItems faces.  A pass CTA costs about the same
// whatever its tile's size, so the fewest tiles that fit is the aim; tiles
// end where the ring, not a fixed size, runs out.
std::vector<int32_t> greedy_bounds(int nC, int nIF, const std::vector<int64_t>& owner,
                                   const std::vector<int64_t>& neighbour, const std::vector<int32_t>& cfo,
                                   const std::vector<int32_t>& cfl, const std::vector<int32_t>& perm,
                                   const std::vector<int32_t>& iperm) {
    std::vector<int32_t> bounds(1, 0);
    std::vector<unsigned char> in_l0(nC, 0);
    std::vector<int32_t> ring_cnt(nC, 0);  // L0 neighbours of a cell outside L0
    std::vector<int32_t> fresh;
    int b = 0, ring = 0, items = 0;
    // fn(n) for every face of renumbered cell c: n the renumbered cell on
    // the other side, -1 for a boundary face
    auto others = [&](int c, auto&& fn) {
        const int o = perm[c];
        for (int k = cfo[o]; k < cfo[o + 1]; ++k) {
            const int f = cfl[k];
            if (f < nIF) fn(iperm[owner[f] == o ? neighbour[f] : owner[f]]);
            else fn(-1);
        }
    };
    for (int c = 0; c < nC; ++c) {
        int d_items = 0, d_ring = ring_cnt[c] > 0 ? -1 : 0;
        fresh.clear();
        others(c, [&](int n) {
            if (n < 0) {
                ++d_items;
            } else if (!in_l0[n]) {
                ++d_items;
                if (ring_cnt[n] == 0 && std::find(fresh.begin(), fresh.end(), n) == fresh.end()) {
                    fresh.push_back(n);
                    ++d_ring;
                }
            }
        });
        const int n0 = c - b;
        const bool fits = n0 + 1 <= dugks::kMaxTile && n0 + 1 + ring + d_ring <= dugks::kMaxLocal &&
                          items + d_items <= dugks::kMaxItems;
        if (n0 > 0 && !fits) {
            // close the tile [b, c); cell c starts the next one
            for (int x = b; x < c; ++x) {
                in_l0[x] = 0;
                others(x, [&](int n) {
                    if (n >= 0) ring_cnt[n] = 0;
                });
            }
            bounds.push_back(c);
            b = c;
            ring = items = 0;
            --c;
            continue;
        }
        in_l0[c] = 1;
        items += d_items;
        ring += d_ring;
        others(c, [&](int n) {
            if (n >= 0 && !in_l0[n]) ++ring_cnt[n];
        });
    }
    bounds.push_back(nC);
    return bounds;
}

}  // namespace

namespace dugks {

// Tile layout.  Cells are renumbered by recursive coordinate bisection and
// cut into tiles of `tile_cells` consecutive cells (L0), or, with
// tile_cells = 0, into the greedy tiles of greedy_bounds.  Each tile also
// holds its ring L1 (face neighbours of L0 outside it), and one item per
// face touching L0, sorted by item kind.  Gradient stencils and flux lists
// are stored slot-major ([slot][cell]) so that consecutive threads read
// consecutive words.
void build_tiling(dugks_handle* h, int tile_cells) {
    Tiling& t = h->tiling;
    const int nC = h->nC, nIF = h->nIF, nBF = h->nBF;
    t.perm.resize(nC);
    std::iota(t.perm.begin(), t.perm.end(), 0);
    const bool greedy = tile_cells <= 0;
    rcb_order(h->C, t.perm, 0, nC, greedy ? 4 : tile_cells);
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
    t.nb_max = t.nf_max = 0;
    for (int c = 0; c < nC; ++c) {
        int nb = 0;
        for (int k = cfo[c]; k < cfo[c + 1]; ++k) nb += cfl[k] < nIF;
        t.nb_max = std::max(t.nb_max, nb);
        t.nf_max = std::max(t.nf_max, cfo[c + 1] - cfo[c]);
    }

    std::vector<int32_t> bounds;
    if (greedy) {
        bounds = greedy_bounds(nC, nIF, h->owner, h->neighbour, cfo, cfl, t.perm, t.iperm);
    } else {
        for (int b = 0; b < nC; b += tile_cells) bounds.push_back(b);
        bounds.push_back(nC);
    }
    t.n_tiles = static_cast<int>(bounds.size()) - 1;
    t.tile_cells = 0;
    for (int ti = 0; ti < t.n_tiles; ++ti) t.tile_cells = std::max(t.tile_cells, bounds[ti + 1] - bounds[ti]);
    t.tile_begin.assign(t.n_tiles + 1, 0);
    t.tile_loc_off.assign(t.n_tiles + 1, 0);
    t.tile_item_off.assign(t.n_tiles + 1, 0);
    t.loc_cells.clear();
    t.it_meta.clear();
    t.it_loc.clear();
    t.it_face.clear();
    t.it_other.clear();
    std::vector<double> geo;  // item-major scratch [n_items][9]
    t.grad_nb.assign(static_cast<size_t>(t.nb_max) * nC, -1);
    t.grad_ls.assign(static_cast<size_t>(t.nb_max) * 3 * nC, 0.0);
    t.cf_item.assign(static_cast<size_t>(t.nf_max) * nC, 0);
    t.max_local = t.max_l0 = t.max_items = 0;
    std::vector<int32_t> face_item0(nIF + nBF, -1), face_item1(nIF + nBF, -1);
    std::vector<int32_t> local_of(nC, -1);
    struct Pending {
        int kind, f;
    };
    for (int ti = 0; ti < t.n_tiles; ++ti) {
        const int b = bounds[ti], e = bounds[ti + 1], n0 = e - b;
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
        // the tile's faces, sorted by kind
        std::vector<Pending> pend;
        for (int c = b; c < e; ++c) {
            const int o = t.perm[c];
            for (int k = cfo[o]; k < cfo[o + 1]; ++k) {
                const int f = cfl[k];
                int kind;
                if (f < nIF) {
                    const int own_new = t.iperm[h->owner[f]], nei_new = t.iperm[h->neighbour[f]];
                    const bool own_in = own_new >= b && own_new < e, nei_in = nei_new >= b && nei_new < e;
                    if (own_in && nei_in && own_new != c) continue;  // listed once, from the owner
                    kind = (own_in && nei_in) ? ITEM_TILE_INTERNAL : (own_in ? ITEM_TB_OWN : ITEM_TB_NEI);
                } else {
                    kind = ITEM_MESH_BOUNDARY;
                }
                pend.push_back({kind, f});
            }
        }
        std::stable_sort(pend.begin(), pend.end(), [](const Pending& p, const Pending& q) { return p.kind < q.kind; });
        const int item0 = t.n_items();
        t.tile_item_off[ti] = item0;
        std::unordered_map<int, int> face_to_local_item;
        for (const Pending& p : pend) {
            const int f = p.f;
            const int64_t fo = h->owner[f];
            const int lo = local_of[t.iperm[fo]];
            int ln = 0xffff, ptype = 0;
            double g9[9];
            for (int q = 0; q < 3; ++q) {
                g9[q] = h->Sf[3 * f + q];
                g9[3 + q] = h->Cf[3 * f + q] - h->C[3 * fo + q];
                g9[6 + q] = 0.0;
            }
            if (f < nIF) {
                const int64_t fn = h->neighbour[f];
                ln = local_of[t.iperm[fn]];
                for (int q = 0; q < 3; ++q) g9[6 + q] = h->Cf[3 * f + q] - h->C[3 * fn + q];
            } else {
                ptype = h->bface_ptype[f - nIF];
            }
            t.it_meta.push_back(p.kind | (ptype << 4));
            t.it_loc.push_back(lo | (ln << 16));
            t.it_face.push_back(f < nIF ? f : f - nIF);
            t.it_other.push_back(-1);
            geo.insert(geo.end(), g9, g9 + 9);
            const int li = t.n_items() - 1 - item0;
            face_to_local_item[f] = li;
            if (face_item0[f] < 0) face_item0[f] = item0 + li;
            else face_item1[f] = item0 + li;
        }
        // gradient stencils and flux lists of the L0 cells
        for (int c = b; c < e; ++c) {
            const int o = t.perm[c];
            int sb = 0, sf = 0;
            for (int k = cfo[o]; k < cfo[o + 1]; ++k) {
                const int f = cfl[k];
                const bool is_own = h->owner[f] == o;
                if (f < nIF) {
                    const int other = is_own ? static_cast<int>(h->neighbour[f]) : static_cast<int>(h->owner[f]);
                    t.grad_nb[static_cast<size_t>(sb) * nC + c] = local_of[t.iperm[other]];
                    const double* ls = is_own ? &h->lsP[3 * f] : &h->lsN[3 * f];
                    for (int q = 0; q < 3; ++q) t.grad_ls[(static_cast<size_t>(sb) * 3 + q) * nC + c] = ls[q];
                    ++sb;
                }
                const int li = face_to_local_item.at(f);
                t.cf_item[static_cast<size_t>(sf) * nC + c] = is_own ? -(li + 1) : (li + 1);
                ++sf;
            }
        }
        for (int c = b; c < e; ++c) local_of[c] = -1;
        for (int c : l1) local_of[c] = -1;
        t.max_local = std::max(t.max_local, n0 + static_cast<int>(l1.size()));
        t.max_l0 = std::max(t.max_l0, n0);
        t.max_items = std::max(t.max_items, t.n_items() - item0);
    }
    t.tile_begin[t.n_tiles] = nC;
    t.tile_loc_off[t.n_tiles] = static_cast<int32_t>(t.loc_cells.size());
    t.tile_item_off[t.n_tiles] = t.n_items();
    // the item of the other side of every tile-boundary face: pass B reads
    // that side's share of the face value from the item's face-value slot
    const int ni = t.n_items();
    for (int i = 0; i < ni; ++i) {
        const int kind = t.it_meta[i] & 15;
        if (kind != ITEM_TB_OWN && kind != ITEM_TB_NEI) continue;
        const int f = t.it_face[i];
        t.it_other[i] = face_item0[f] == i ? face_item1[f] : face_item0[f];
    }
    t.it_geo.assign(static_cast<size_t>(9) * ni, 0.0);
    for (int i = 0; i < ni; ++i)
        for (int q = 0; q < 9; ++q) t.it_geo[static_cast<size_t>(q) * ni + i] = geo[static_cast<size_t>(i) * 9 + q];
    t.face_items.assign(2 * static_cast<size_t>(nIF + nBF), -1);
    for (int f = 0; f < nIF + nBF; ++f) {
        t.face_items[2 * f] = face_item0[f];
        t.face_items[2 * f + 1] = face_item1[f];
    }
}

}  // namespace dugks

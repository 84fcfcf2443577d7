/*
 * Tangent-linear restatement of the DUGKS step -- TEST INFRASTRUCTURE ONLY,
 * like the oracle it extends (dugks_oracle.c).  It reruns oracle_evolve's
 * arithmetic (fvDVM::evolution, src/fvDVM/fvDVM/fvDVM.C:2128-2174) on
 * dual numbers, value and one directional derivative, for cases whose
 * patches are maxwellWall and farField and whose macros come from the DF
 * moments (macroFlux no).  The value part keeps the oracle's operand order,
 * so it reproduces the oracle's trajectory; the derivative part is the
 * exact forward-mode derivative of that arithmetic.
 *
 * Parameters: the wall temperature and velocity of every boundary face
 * (the T and U patch values: calculatedMaxwellFvPatchField.C:140-164 and
 * fvDVM.C:578-624, :1054-1098 read them; farField faces read T only,
 * fvDVM.C:926-938) and muRef (fvDVM::updateTau, fvDVM.C:1823-1832).  The
 * objective is the time average over the steps of a weighted sum of the
 * energy and momentum fluxes through the boundary faces, taken from the
 * relaxed face DFs that enter the update (fvDVM.C:1462-1519):
 *
 *   J = 1/N sum_n sum_b sum_i w_i (xi_i . S_b) [a_b (|xi_i|^2 g + h)/2 + (c_b . xi_i) g]
 *
 * The start state (the oracle's current g~, h~ and cell macros) is taken as
 * independent of the parameters, which holds for a state made by
 * oracle_set_macros.
 */
#include <cmath>
#include <cstring>
#include <vector>

#include "dugks_oracle.h"
#include "dugks_oracle_state.h"

namespace {

const double kVSmall = 1.0e-300;

struct Dual {
    double v = 0, d = 0;
    Dual() = default;
    Dual(double x) : v(x) {}  // NOLINT: constants promote
    Dual(double x, double y) : v(x), d(y) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual exp(Dual a) {
    const double e = std::exp(a.v);
    return {e, e * a.d};
}
inline Dual log(Dual a) { return {std::log(a.v), a.d / a.v}; }
inline Dual sqrt(Dual a) {
    const double r = std::sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}
inline Dual pow(Dual a, double p) { return {std::pow(a.v, p), p * std::pow(a.v, p - 1.0) * a.d}; }
inline Dual fabs(Dual a) { return a.v < 0 ? -a : a; }

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Dual magsqr3(const Dual* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

struct Tangent {
    const oracle_state* s;
    double dt;
    Dual muRef;
    std::vector<Dual> Tb, Ub, rho_b, inByRho;
    std::vector<Dual> gT, hT, gBP, hBP, gS, hS, gSb, hSb;
    std::vector<Dual> rho, U, T, q;
    std::vector<Dual> rhoF, UF, TF, qF, tauF;
    std::vector<Dual> Gg, Gh;

    Dual tau_of(Dual Tc, Dual r) const { return muRef * exp(s->omega * log(Tc / s->Tref)) / r / Tc / s->R; }

    // discreteVelocity::equilibriumMaxwellByRho (discreteVelocity.C:1027-1039)
    Dual eq_by_rho(const double* xi, const Dual* Uv, Dual Tv) const {
        Dual c[3] = {Uv[0] - xi[0], Uv[1] - xi[1], Uv[2] - xi[2]};
        return 1.0 / pow(sqrt(2.0 * M_PI * s->R * Tv), (double)s->D) * exp(-magsqr3(c) / (2.0 * s->R * Tv));
    }

    // the Shakhov equilibrium of fvDVM.C:648-683 and :1362-1457; Th is the
    // temperature the h part is scaled by
    void shakhov(const double* xi, const Dual* Uv, Dual Tv, Dual r, const Dual* qv, Dual Th, Dual& gEq,
                 Dual& hEq) const {
        const int D = s->D, K = s->K;
        const double R = s->R, Pr = s->Pr;
        Dual um[3] = {Uv[0] - xi[0], Uv[1] - xi[1], Uv[2] - xi[2]};
        Dual cSqrByRT = magsqr3(um) / (R * Tv);
        Dual xu[3] = {xi[0] - Uv[0], xi[1] - Uv[1], xi[2] - Uv[2]};
        Dual cqBy5pRT = (xu[0] * qv[0] + xu[1] * qv[1] + xu[2] * qv[2]) / (5.0 * r * R * Tv * R * Tv);
        Dual gEqBGK = r / pow(sqrt(2.0 * M_PI * R * Tv), (double)D) * exp(-cSqrByRT / 2.0);
        gEq = (1.0 + (1.0 - Pr) * cqBy5pRT * (cSqrByRT - D - 2.0)) * gEqBGK;
        hEq = ((K + 3.0 - D) + (1.0 - Pr) * cqBy5pRT * ((cSqrByRT - D) * (K + 3.0 - D) - 2 * K)) * gEqBGK * R * Th;
    }

    Dual recon(Dual phi, const Dual* G, const double* Cf, const double* Cc, const double* xi) const {
        double v[3];
        for (int k = 0; k < 3; ++k) v[k] = Cf[k] - Cc[k] - 0.5 * xi[k] * dt;
        return phi + (G[0] * v[0] + G[1] * v[1] + G[2] * v[2]);
    }

    // face or cell macros from DV-major values with the given stride/column
    // (fvDVM.C:1181-1300 and :1683-1742); a is dt Pr/2 on faces, dt Pr in cells
    void macros(const Dual* g, const Dual* h, size_t stride, size_t col, double a, Dual& r, Dual* Uv, Dual& Tv,
                Dual* qv, Dual& tv) const {
        const int K = s->K, nv = s->nv;
        const double R = s->R;
        Dual rho_ = 0, rU[3] = {0, 0, 0}, rE = 0;
        for (int i = 0; i < nv; ++i) {
            const double* xi = s->xi + 3 * i;
            const Dual gg = g[i * stride + col], hh = h[i * stride + col];
            const double w = s->wv[i];
            rho_ += w * gg;
            for (int k = 0; k < 3; ++k) rU[k] += w * gg * xi[k];
            rE += 0.5 * w * (gg * dot3(xi, xi) + hh);
        }
        for (int k = 0; k < 3; ++k) Uv[k] = rU[k] / rho_;
        Tv = (rE - 0.5 * rho_ * magsqr3(Uv)) / ((K + 3) / 2.0 * R * rho_);
        tv = tau_of(Tv, rho_);
        Dual Q[3] = {0, 0, 0};
        for (int i = 0; i < nv; ++i) {
            const double* xi = s->xi + 3 * i;
            const Dual gg = g[i * stride + col], hh = h[i * stride + col];
            const double w = s->wv[i];
            Dual c[3] = {xi[0] - Uv[0], xi[1] - Uv[1], xi[2] - Uv[2]};
            Dual m = magsqr3(c) * gg + hh;
            for (int k = 0; k < 3; ++k) Q[k] += 0.5 * w * c[k] * m;
        }
        const Dual fac = 2.0 * tv / (2.0 * tv + a);
        r = rho_;
        for (int k = 0; k < 3; ++k) qv[k] = fac * Q[k];
    }

    Dual step(const double* heat_w, const double* force_w) {
        const oracle_state& o = *s;
        const int D = o.D, K = o.K, nC = o.nC, nIF = o.nIF, nBF = o.nBF, nv = o.nv;
        const double R = o.R, Pr = o.Pr;
        /* 1. updateGHbarPvol (fvDVM.C:648-683) */
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = o.xi + 3 * dvi;
            for (int c = 0; c < nC; ++c) {
                const Dual tau = tau_of(T[c], rho[c]);
                const Dual relaxFactor = 1.5 * dt / (2.0 * tau + dt);
                Dual gEq, hEq;
                shakhov(xi, &U[3 * c], T[c], rho[c], &q[3 * c], T[c], gEq, hEq);
                const size_t id = (size_t)dvi * nC + c;
                gBP[id] = (1.0 - relaxFactor) * gT[id] + relaxFactor * gEq;
                hBP[id] = (1.0 - relaxFactor) * hT[id] + relaxFactor * hEq;
            }
        }
        /* 2-4. least-squares gradient and the face reconstruction
         *      (fvDVM.C:749-1029) */
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = o.xi + 3 * dvi;
            const Dual* g = &gBP[(size_t)dvi * nC];
            const Dual* h = &hBP[(size_t)dvi * nC];
            for (auto& x : Gg) x = 0;
            for (auto& x : Gh) x = 0;
            for (int f = 0; f < nIF; ++f) {
                const int64_t ow = o.own[f], ne = o.nei[f];
                const Dual dg = g[ne] - g[ow], dh = h[ne] - h[ow];
                for (int k = 0; k < 3; ++k) {
                    Gg[3 * ow + k] += o.lsP[3 * f + k] * dg;
                    Gg[3 * ne + k] -= o.lsN[3 * f + k] * dg;
                    Gh[3 * ow + k] += o.lsP[3 * f + k] * dh;
                    Gh[3 * ne + k] -= o.lsN[3 * f + k] * dh;
                }
            }
            Dual* gs = &gS[(size_t)dvi * nIF];
            Dual* hs = &hS[(size_t)dvi * nIF];
            for (int f = 0; f < nIF; ++f) {
                const int64_t ow = o.own[f], ne = o.nei[f];
                const double* Cf = o.Cf + 3 * f;
                const double xs = dot3(xi, o.Sf + 3 * f);
                if (xs >= kVSmall) {
                    gs[f] = recon(g[ow], &Gg[3 * ow], Cf, o.C + 3 * ow, xi);
                    hs[f] = recon(h[ow], &Gh[3 * ow], Cf, o.C + 3 * ow, xi);
                } else if (xs < -kVSmall) {
                    gs[f] = recon(g[ne], &Gg[3 * ne], Cf, o.C + 3 * ne, xi);
                    hs[f] = recon(h[ne], &Gh[3 * ne], Cf, o.C + 3 * ne, xi);
                } else {
                    Dual dn = recon(0.0, &Gg[3 * ne], Cf, o.C + 3 * ne, xi);
                    Dual d_o = recon(0.0, &Gg[3 * ow], Cf, o.C + 3 * ow, xi);
                    gs[f] = 0.5 * (((g[ne] + dn) + g[ow]) + d_o);
                    dn = recon(0.0, &Gh[3 * ne], Cf, o.C + 3 * ne, xi);
                    d_o = recon(0.0, &Gh[3 * ow], Cf, o.C + 3 * ow, xi);
                    hs[f] = 0.5 * (((h[ne] + dn) + h[ow]) + d_o);
                }
            }
            Dual* gsb = &gSb[(size_t)dvi * nBF];
            Dual* hsb = &hSb[(size_t)dvi * nBF];
            for (int b = 0; b < nBF; ++b) {
                const int f = nIF + b;
                const int64_t ow = o.own[f];
                const double xs = dot3(xi, o.Sf + 3 * f);
                const int type = o.ptype[o.bf_patch[b]];
                if (xs > 0) {
                    gsb[b] = recon(g[ow], &Gg[3 * ow], o.Cf + 3 * f, o.C + 3 * ow, xi);
                    hsb[b] = recon(h[ow], &Gh[3 * ow], o.Cf + 3 * f, o.C + 3 * ow, xi);
                } else if (type == ORACLE_PATCH_FAR_FIELD) {
                    /* incoming: rho_b M(U_owner, T_b) (fvDVM.C:926-938) */
                    gsb[b] = rho_b[b] * eq_by_rho(xi, &U[3 * ow], Tb[b]);
                    hsb[b] = gsb[b] * (R * Tb[b]) * (double)(K + 3 - D);
                }
            }
        }
        /* 5. the wall density from the outgoing flux (fvDVM.C:959-960,
         *    calculatedMaxwellFvPatchField.C:140-164) */
        for (int b = 0; b < nBF; ++b) {
            if (o.ptype[o.bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
            const double* S = o.Sf + 3 * (nIF + b);
            Dual out = 0.0;
            for (int dvi = 0; dvi < nv; ++dvi) {
                const double xs = dot3(o.xi + 3 * dvi, S);
                if (xs > 0) out += o.wv[dvi] * xs * gSb[(size_t)dvi * nBF + b];
            }
            rho_b[b] = out / fabs(inByRho[b]);
        }
        /* 6. updateGHbarSurfMaxwellWallIn (fvDVM.C:1054-1098) */
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = o.xi + 3 * dvi;
            for (int b = 0; b < nBF; ++b) {
                if (o.ptype[o.bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
                if (dot3(xi, o.Sf + 3 * (nIF + b)) <= 0) {
                    const size_t id = (size_t)dvi * nBF + b;
                    gSb[id] = rho_b[b] * eq_by_rho(xi, &Ub[3 * b], Tb[b]);
                    hSb[id] = gSb[id] * (R * Tb[b]) * (double)(K + 3 - D);
                }
            }
        }
        /* 8. updateMacroSurf (fvDVM.C:1181-1300) */
        for (int f = 0; f < nIF + nBF; ++f) {
            const bool internal = f < nIF;
            macros(internal ? gS.data() : gSb.data(), internal ? hS.data() : hSb.data(),
                   internal ? (size_t)nIF : (size_t)nBF, internal ? (size_t)f : (size_t)(f - nIF), 0.5 * dt * Pr,
                   rhoF[f], &UF[3 * f], TF[f], &qF[3 * f], tauF[f]);
        }
        /* 9. updateGHsurf (fvDVM.C:1362-1457); the boundary h equilibrium is
         *    scaled by the internal-face temperature at the patch-local index */
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = o.xi + 3 * dvi;
            for (int f = 0; f < nIF; ++f) {
                const Dual r = 0.5 * dt / (2.0 * tauF[f] + 0.5 * dt);
                Dual gEq, hEq;
                shakhov(xi, &UF[3 * f], TF[f], rhoF[f], &qF[3 * f], TF[f], gEq, hEq);
                const size_t id = (size_t)dvi * nIF + f;
                gS[id] = (1.0 - r) * gS[id] + r * gEq;
                hS[id] = (1.0 - r) * hS[id] + r * hEq;
            }
            for (int b = 0; b < nBF; ++b) {
                const int f = nIF + b;
                if (!(dot3(xi, o.Sf + 3 * f) > 0)) continue;
                const Dual r = 0.5 * dt / (2.0 * tauF[f] + 0.5 * dt);
                Dual gEq, hEq;
                shakhov(xi, &UF[3 * f], TF[f], rhoF[f], &qF[3 * f], TF[o.bf_local[b]], gEq, hEq);
                const size_t id = (size_t)dvi * nBF + b;
                gSb[id] = (1.0 - r) * gSb[id] + r * gEq;
                hSb[id] = (1.0 - r) * hSb[id] + r * hEq;
            }
        }
        /* the objective: boundary energy and momentum fluxes of this step */
        Dual Jn = 0.0;
        for (int b = 0; b < nBF; ++b) {
            const double a = heat_w ? heat_w[b] : 0.0;
            const double* cw = force_w ? force_w + 3 * b : nullptr;
            const double* S = o.Sf + 3 * (nIF + b);
            for (int dvi = 0; dvi < nv; ++dvi) {
                const double* xi = o.xi + 3 * dvi;
                const double wx = o.wv[dvi] * dot3(xi, S);
                const double cg = cw ? dot3(cw, xi) : 0.0;
                const size_t id = (size_t)dvi * nBF + b;
                Jn += wx * (a * 0.5 * (dot3(xi, xi) * gSb[id] + hSb[id]) + cg * gSb[id]);
            }
        }
        /* 10. updateGHtildeVol (fvDVM.C:1462-1519) */
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = o.xi + 3 * dvi;
            Dual* g = &gT[(size_t)dvi * nC];
            Dual* h = &hT[(size_t)dvi * nC];
            const Dual* gb = &gBP[(size_t)dvi * nC];
            const Dual* hb = &hBP[(size_t)dvi * nC];
            for (int c = 0; c < nC; ++c) {
                g[c] = -1.0 / 3 * g[c] + 4.0 / 3 * gb[c];
                h[c] = -1.0 / 3 * h[c] + 4.0 / 3 * hb[c];
            }
            for (int f = 0; f < nIF; ++f) {
                const int64_t ow = o.own[f], ne = o.nei[f];
                const double xs = dot3(xi, o.Sf + 3 * f);
                const Dual gs = gS[(size_t)dvi * nIF + f], hs = hS[(size_t)dvi * nIF + f];
                g[ow] -= (xs * gs * dt / o.V[ow]);
                g[ne] += (xs * gs * dt / o.V[ne]);
                h[ow] -= (xs * hs * dt / o.V[ow]);
                h[ne] += (xs * hs * dt / o.V[ne]);
            }
            for (int b = 0; b < nBF; ++b) {
                const int64_t ow = o.own[nIF + b];
                const double xs = dot3(xi, o.Sf + 3 * (nIF + b));
                g[ow] -= xs * gSb[(size_t)dvi * nBF + b] * dt / o.V[ow];
                h[ow] -= xs * hSb[(size_t)dvi * nBF + b] * dt / o.V[ow];
            }
        }
        /* 11. updateMacroVol (fvDVM.C:1521-1554, 1683-1742) */
        for (int c = 0; c < nC; ++c) {
            Dual tv;
            macros(gT.data(), hT.data(), (size_t)nC, (size_t)c, dt * Pr, rho[c], &U[3 * c], T[c], &q[3 * c], tv);
        }
        return Jn;
    }
};

std::vector<Dual> seeded(const double* v, const double* d, size_t n) {
    std::vector<Dual> r(n);
    for (size_t i = 0; i < n; ++i) r[i] = Dual(v[i], d ? d[i] : 0.0);
    return r;
}

std::vector<Dual> plain(const double* v, size_t n) { return seeded(v, nullptr, n); }

}  // namespace

extern "C" int oracle_tangent(const oracle_state* s, int n_steps, double dt, const double* heat_w,
                              const double* force_w, const double* dT_b, const double* dU_b, double d_muRef,
                              double* J, double* dJ, double* g_out, double* h_out) {
    if (s->macro_flux) return -1;
    for (int p = 0; p < s->nP; ++p)
        if (s->ptype[p] != ORACLE_PATCH_MAXWELL_WALL && s->ptype[p] != ORACLE_PATCH_FAR_FIELD) return -1;
    if (n_steps < 1) return -1;
    const int nC = s->nC, nIF = s->nIF, nBF = s->nBF, nv = s->nv, nF = nIF + nBF;
    Tangent t;
    t.s = s;
    t.dt = dt;
    t.muRef = Dual(s->muRef, d_muRef);
    t.Tb = seeded(s->T_b, dT_b, nBF);
    t.Ub = seeded(s->U_b, dU_b, 3 * (size_t)nBF);
    t.rho_b = plain(s->rho_b, nBF);
    t.gT = plain(s->gT, (size_t)nv * nC);
    t.hT = plain(s->hT, (size_t)nv * nC);
    t.rho = plain(s->rho, nC);
    t.U = plain(s->U, 3 * (size_t)nC);
    t.T = plain(s->T, nC);
    t.q = plain(s->q, 3 * (size_t)nC);
    t.gBP.resize((size_t)nv * nC);
    t.hBP.resize((size_t)nv * nC);
    t.gS.resize((size_t)nv * nIF);
    t.hS.resize((size_t)nv * nIF);
    t.gSb.resize((size_t)nv * nBF);
    t.hSb.resize((size_t)nv * nBF);
    t.rhoF.resize(nF);
    t.UF.resize(3 * (size_t)nF);
    t.TF.resize(nF);
    t.qF.resize(3 * (size_t)nF);
    t.tauF.resize(nF);
    t.Gg.resize(3 * (size_t)nC);
    t.Gh.resize(3 * (size_t)nC);
    /* setCalculatedMaxwellRhoBC (fvDVM.C:578-624) from the seeded patch values */
    t.inByRho.assign(nBF, Dual(0.0));
    for (int b = 0; b < nBF; ++b) {
        if (s->ptype[s->bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
        const double* S = s->Sf + 3 * (nIF + b);
        Dual acc = 0.0;
        for (int i = 0; i < nv; ++i) {
            const double* xi = s->xi + 3 * i;
            const double xs = dot3(xi, S);
            if (xs < 0) acc += -s->wv[i] * xs * t.eq_by_rho(xi, &t.Ub[3 * b], t.Tb[b]);
        }
        t.inByRho[b] = acc;
    }
    Dual sum = 0.0;
    for (int n = 0; n < n_steps; ++n) sum += t.step(heat_w, force_w);
    const Dual avg = sum / (double)n_steps;
    if (J) *J = avg.v;
    if (dJ) *dJ = avg.d;
    for (size_t i = 0; i < (size_t)nv * nC; ++i) {
        if (g_out) g_out[i] = t.gT[i].v;
        if (h_out) h_out[i] = t.hT[i].v;
    }
    return 0;
}

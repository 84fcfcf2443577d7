// Discrete adjoint of the FP64 DUGKS step (fvDVM::evolution,
// src/fvDVM/fvDVM/fvDVM.C:2128-2174) for cases whose patches are maxwellWall
// and farField and whose cell macros are the moments of the DFs (macroFlux
// no).  Reverse mode of exactly the arithmetic of one step:
//
//   1 gbar+ = (1-r) g~ + r g^S(cell macros)           fvDVM.C:648-683
//   2 least-squares gradient of gbar+                 discreteVelocity.C:366-369
//   3 upwind face values at the half step, far-field  fvDVM.C:755-1029
//     incoming rho_b M(U_owner, T_b)
//   4 rho_w = outgoing / |inComingByRho|              fvDVM.C:1032-1052
//   5 incoming wall DFs rho_w M(U_w, T_w)             fvDVM.C:1054-1098
//   6 face macros                                     fvDVM.C:1181-1300
//   7 face relaxation (boundary: outgoing DVs, h^S    fvDVM.C:1362-1457
//     scaled by the internal-face T at the patch-local index)
//   8 g~ <- -g~/3 + 4/3 gbar+ - dt/V sum (xi.S) g_f   fvDVM.C:1462-1519
//   9 cell macros of the new DFs                      fvDVM.C:1521-1554, 1683-1742
//
// The objective of a step is the energy and momentum flux through the
// boundary faces, taken from the relaxed boundary DFs that enter step 8:
//   J_n = sum_b sum_i w_i (xi_i.S_b) [a_b (|xi_i|^2 g + h)/2 + (c_b.xi_i) g]
// and the run's objective is a weighted sum of the J_n (a time average over a
// window of steps).  Parameters: the T and U patch values of every boundary
// face (wall faces: incoming DFs and inComingByRho, fvDVM.C:578-624; far-field
// faces: T of the incoming DFs, fvDVM.C:926-938) and muRef (the relaxation
// times, fvDVM::updateTau, fvDVM.C:1823-1832).
//
// Every stage is a functor over a flat index with a __host__ __device__ body,
// run by an executor (a grid-stride CUDA launch in the library).  Sums over
// DVs are split into DV chunks written to per-chunk partials and added in
// chunk order by a combine functor, so results are reproducible run to run.
// Layouts: DV-major [dv][entity] for per-(entity, DV) arrays, entity-major
// [entity][k] for per-entity records, [chunk][entity][kP] for partials.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#ifdef __CUDACC__
#define ADJ_HD __host__ __device__ __forceinline__
#else
#define ADJ_HD inline
#endif

namespace dugks {
namespace adj {

constexpr double kPi = 3.14159265358979323846;
constexpr double kVSmall = 1.0e-300;  // OpenFOAM VSMALL, the upwind switch of fvDVM.C:829-847
constexpr int kP = 16;                // stride of a partial record (doubles)
constexpr int kMac = 20;              // stride of a macro record
constexpr int kCo = 11;               // stride of a moment-adjoint coefficient record

// macro record of a face or cell: the macros and the raw moments the
// reverse of the macro formulas reads
enum {
    MAC_RHO = 0, MAC_U = 1, MAC_T = 4, MAC_Q = 5, MAC_TAU = 8, MAC_RE = 9, MAC_M2 = 10, MAC_QRAW = 16, MAC_FAC = 19
};
// coefficient record: the adjoint of a DF of DV i from the adjoint of its
// entity's macros is w_i [al + be.xi + ga |xi|^2 + (aq.c) |c|^2 / 2] for g and
// w_i [ga + (aq.c) / 2] for h, with c = xi - U
enum { CO_AL = 0, CO_BE = 1, CO_GA = 4, CO_AQ = 5, CO_U = 8 };

struct View {
    int nC, nIF, nBF, nF, nv, D, K, nchF, nchC;
    double R, Pr, omega, Tref, mu, dt;
    // mesh (cells in the handle's numbering; faces internal then boundary)
    const int32_t* own;     // [nF]
    const int32_t* nei;     // [nIF]
    const double* S;        // [nF][3]
    const double* Cf;       // [nF][3]
    const double* C;        // [nC][3]
    const double* invV;     // [nC]
    const double* lsP;      // [nIF][3]
    const double* lsN;      // [nIF][3]
    const int32_t* cf_off;  // [nC+1] faces of each cell in face order
    const int32_t* cf_ent;  // face * 2 + (1 if the cell is the neighbour)
    const int32_t* th_off;  // [nF+1] boundary faces whose h^S is scaled by this face's T
    const int32_t* th_ent;
    const int32_t* btype;   // [nBF] 1 maxwellWall, 2 farField
    const int32_t* blocal;  // [nBF] index within the patch
    const double* bU;       // [nBF][3]
    const double* bT;       // [nBF]
    const double* brho;     // [nBF] far-field rho_b (fixed)
    const double* xi;       // [nv][3]
    const double* w;        // [nv]
    const double* ha;       // [nBF] objective: energy-flux weights
    const double* fw;       // [nBF][3] objective: momentum-flux weights
    // state of the step (input)
    const double* g;        // [nv][nC]
    const double* h;
    const double* cm;       // [nC][9] rho U T q tau the step starts from
    // the tiled pass A's face-value buffer [nv][n_items] and the items of
    // every face ([nF][2], -1: none), from which the record takes its face values
    const double* fvg;
    const double* fvh;
    const int32_t* fitems;
    int64_t nI;
    // forward record of the step
    double* fg;             // [nv][nF] face values before the relaxation
    double* fh;
    double* pf;             // [nchF][nF][kP]
    double* pc;             // [nchC][nC][kP]
    double* rhow;           // [nBF]
    double* inby;           // [nBF] inComingByRho of the patch values
    double* fmac;           // [nF][kMac]
    double* cmac;           // [nC][kMac] macros of the state, from its moments
    // adjoint of the step
    const double* lg;       // [nv][nC] adjoint of the state after the step
    const double* lh;
    double* og;             // [nv][nC] adjoint of the state before the step (output)
    double* oh;
    double* ag;             // [nv][nF] adjoint of the face values before the relaxation
    double* ah;
    double* aGg;            // [3][nv][nC] adjoint of the gradients
    double* aGh;
    double* fco;            // [nF][kCo]
    double* cco;            // [nC][kCo]
    double* aout;           // [nBF] adjoint of a wall face's outgoing flux
    double* aUown;          // [nBF][3] adjoint of the owner-cell U through far-field incoming DFs
    // accumulated over the run
    double* gTb;            // [nBF] dJ/dT_b
    double* gUb;            // [nBF][3] dJ/dU_b
    double* aI;             // [nBF] adjoint of inComingByRho
    double* amuF;           // [nF] dJ/dmuRef through the face relaxation times
    double* amuC;           // [nC] dJ/dmuRef through the cell relaxation times
    double* Jb;             // [nBF] objective per boundary face
    double wn;              // objective weight of this step
    int fold;               // 1: the step's cell macros are moments of its DFs (every step but the first)
};

ADJ_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// loads of arrays a kernel only reads: on the device through the read-only
// data path, which also lets the compiler issue the next DV's loads before
// this DV's stores (the per-chunk DV loops are otherwise serialised by them)
ADJ_HD double ro(const double* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
ADJ_HD int32_t ro(const int32_t* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
ADJ_HD double magsqr3(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

// xi . Sf as the reference evaluates it: each product rounded, the sums
// unfused, left to right.  Its sign picks the upwind side of a face and
// whether a boundary DV is outgoing; on curved faces some DVs are
// tangential up to rounding, so a contraction into FMAs would flip
// decisions the forward made.
ADJ_HD double xs_of(const double* xi, const double* S) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(__dadd_rn(__dmul_rn(xi[0], S[0]), __dmul_rn(xi[1], S[1])), __dmul_rn(xi[2], S[2]));
#else
    return (xi[0] * S[0] + xi[1] * S[1]) + xi[2] * S[2];
#endif
}
ADJ_HD size_t at(int i, int n, int e) { return static_cast<size_t>(i) * n + e; }
ADJ_HD int chunk_lo(int nv, int nch, int ch) { return static_cast<int>(static_cast<int64_t>(nv) * ch / nch); }

// fvDVM::updateTau (fvDVM.C:1823-1832)
ADJ_HD double tau_of(const View& v, double T, double rho) {
    return v.mu * exp(v.omega * log(T / v.Tref)) / rho / T / v.R;
}

// discreteVelocity::equilibriumMaxwellByRho (discreteVelocity.C:1027-1039)
ADJ_HD double eq_by_rho(const View& v, const double* xi, const double* U, double T) {
    double c[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
    return 1.0 / pow(sqrt(2.0 * kPi * v.R * T), v.D) * exp(-magsqr3(c) / (2.0 * v.R * T));
}

// its derivatives: dE/dT and dE/dU
ADJ_HD void eq_by_rho_d(const View& v, const double* xi, const double* U, double T, double E, double& dT,
                        double* dU) {
    double c[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
    const double RT = v.R * T;
    dT = E * (-0.5 * v.D / T + magsqr3(c) / (2.0 * RT * T));
    for (int k = 0; k < 3; ++k) dU[k] = -E * c[k] / RT;
}

// the Shakhov equilibrium of fvDVM.C:648-683 and :1362-1457 (operand order of
// the reference); Th is the temperature h^S is scaled by
ADJ_HD void shakhov(const View& v, const double* xi, const double* U, double T, double rho, const double* q,
                    double Th, double& gEq, double& hEq) {
    const int D = v.D, K = v.K;
    const double R = v.R, Pr = v.Pr;
    double um[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
    const double cSqrByRT = magsqr3(um) / (R * T);
    double xu[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
    const double cqBy5pRT = dot3(xu, q) / (5.0 * rho * R * T * R * T);
    const double gEqBGK = rho / pow(sqrt(2.0 * kPi * R * T), D) * exp(-cSqrByRT / 2.0);
    gEq = (1.0 + (1.0 - Pr) * cqBy5pRT * (cSqrByRT - D - 2.0)) * gEqBGK;
    hEq = ((K + 3.0 - D) + (1.0 - Pr) * cqBy5pRT * ((cSqrByRT - D) * (K + 3.0 - D) - 2 * K)) * gEqBGK * R * Th;
}

// Reverse of shakhov(): given the adjoints ag, ah of gEq, hEq, add the
// adjoints of rho, U, T, q and Th into s[0], s[1..3], s[4], s[5..7], s[8].
ADJ_HD void shakhov_rev(const View& v, const double* xi, const double* U, double T, double rho, const double* q,
                        double Th, double ag, double ah, double* s) {
    const int D = v.D, K = v.K;
    const double R = v.R, omp = 1.0 - v.Pr, k3 = K + 3.0 - D;
    double c[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
    const double RT = R * T;
    const double cS = magsqr3(c) / RT;
    const double den = 5.0 * rho * RT * RT;
    const double P = dot3(c, q) / den;
    const double G0 = rho / pow(sqrt(2.0 * kPi * RT), D) * exp(-cS / 2.0);
    const double A = 1.0 + omp * P * (cS - D - 2.0);
    const double Bh = k3 + omp * P * ((cS - D) * k3 - 2 * K);
    const double aG0 = ag * A + ah * Bh * R * Th;
    const double aA = ag * G0, aB = ah * G0 * R * Th;
    const double aP = omp * (aA * (cS - D - 2.0) + aB * ((cS - D) * k3 - 2 * K));
    const double acS = omp * P * (aA + aB * k3) - 0.5 * aG0 * G0;
    s[0] += aG0 * G0 / rho - aP * P / rho;
    s[4] += -0.5 * D * aG0 * G0 / T - acS * cS / T - 2.0 * aP * P / T;
    for (int k = 0; k < 3; ++k) {
        const double ac = acS * 2.0 * c[k] / RT + aP * q[k] / den;
        s[1 + k] -= ac;
        s[5 + k] += aP * c[k] / den;
    }
    s[8] += ah * Bh * G0 * R;
}

// the face reconstruction at the half step from cell c (fvDVM.C:832-836):
// phi_c + grad_c . (Cf - C_c - xi dt / 2)
ADJ_HD void recon_vec(const View& v, int f, int c, const double* xi, double* d) {
    for (int k = 0; k < 3; ++k) d[k] = v.Cf[3 * f + k] - v.C[3 * c + k] - 0.5 * xi[k] * v.dt;
}
ADJ_HD double recon(const View& v, double phi, const double* G, size_t stride, size_t id, int f, int c,
                    const double* xi) {
    double d[3];
    recon_vec(v, f, c, xi, d);
    return phi + (G[id] * d[0] + G[stride + id] * d[1] + G[2 * stride + id] * d[2]);
}

// macro record from the raw moments m (M0, M1[3], W, V3[3], M2[6]);
// a = dt Pr / 2 on faces, dt Pr in cells (fvDVM.C:1249-1300, :1683-1742)
ADJ_HD void macros_from_moments(const View& v, const double* m, double a, double* r) {
    const double rho = m[0];
    double U[3] = {m[1] / rho, m[2] / rho, m[3] / rho};
    const double rE = 0.5 * m[4];
    const double T = (rE - 0.5 * rho * magsqr3(U)) / ((v.K + 3) / 2.0 * v.R * rho);
    const double tau = tau_of(v, T, rho);
    const double* M2 = m + 8;  // xx xy xz yy yz zz
    const double M2U[3] = {M2[0] * U[0] + M2[1] * U[1] + M2[2] * U[2], M2[1] * U[0] + M2[3] * U[1] + M2[4] * U[2],
                           M2[2] * U[0] + M2[4] * U[1] + M2[5] * U[2]};
    const double u2 = magsqr3(U);
    const double fac = 2.0 * tau / (2.0 * tau + a);
    r[MAC_RHO] = rho;
    r[MAC_T] = T;
    r[MAC_TAU] = tau;
    r[MAC_RE] = rE;
    r[MAC_FAC] = fac;
    for (int k = 0; k < 3; ++k) {
        const double Q = 0.5 * (m[5 + k] - 2.0 * M2U[k] - U[k] * m[4] + 2.0 * rho * u2 * U[k]);
        r[MAC_U + k] = U[k];
        r[MAC_QRAW + k] = Q;
        r[MAC_Q + k] = fac * Q;
    }
    for (int k = 0; k < 6; ++k) r[MAC_M2 + k] = M2[k];
}

// Reverse of macros_from_moments: from the adjoints of rho, U, T, q and tau
// (aM[0], aM[1..3], aM[4], aM[5..7], aM[8]) the coefficient record of the
// per-DV adjoint, and the adjoint of muRef (returned).
ADJ_HD double macros_rev(const View& v, const double* r, double a, const double* aM, double* co) {
    const double rho = r[MAC_RHO], T = r[MAC_T], tau = r[MAC_TAU], rE = r[MAC_RE], fac = r[MAC_FAC];
    const double* U = r + MAC_U;
    const double* M2 = r + MAC_M2;
    const double cv = (v.K + 3) / 2.0 * v.R;
    const double u2 = magsqr3(U);
    double aQ[3], afac = 0;
    for (int k = 0; k < 3; ++k) {
        aQ[k] = fac * aM[5 + k];
        afac += aM[5 + k] * r[MAC_QRAW + k];
    }
    const double atau = aM[8] + afac * 2.0 * a / ((2.0 * tau + a) * (2.0 * tau + a));
    const double aT = aM[4] + atau * tau * (v.omega - 1.0) / T;
    double arho = aM[0] - atau * tau / rho;
    const double amu = atau * tau / v.mu;
    // dQ/dU = -E2/2 I - P with E2 = sum w (|c|^2 g + h) = 2 rE - rho |U|^2
    // and P = sum w g c c^T = M2 - rho U U^T
    const double E2 = 2.0 * rE - rho * u2;
    const double Pm[3][3] = {{M2[0] - rho * U[0] * U[0], M2[1] - rho * U[0] * U[1], M2[2] - rho * U[0] * U[2]},
                             {M2[1] - rho * U[1] * U[0], M2[3] - rho * U[1] * U[1], M2[4] - rho * U[1] * U[2]},
                             {M2[2] - rho * U[2] * U[0], M2[4] - rho * U[2] * U[1], M2[5] - rho * U[2] * U[2]}};
    double aU[3];
    for (int j = 0; j < 3; ++j)
        aU[j] = aM[1 + j] - 0.5 * E2 * aQ[j] - (Pm[j][0] * aQ[0] + Pm[j][1] * aQ[1] + Pm[j][2] * aQ[2]) -
                aT * U[j] / cv;
    const double arE = aT / (cv * rho);
    arho += aT * (-0.5 * u2 / (cv * rho) - T / rho);
    double aUU = 0;
    for (int j = 0; j < 3; ++j) aUU += aU[j] * U[j];
    arho -= aUU / rho;
    co[CO_AL] = arho;
    for (int j = 0; j < 3; ++j) {
        co[CO_BE + j] = aU[j] / rho;
        co[CO_AQ + j] = aQ[j];
        co[CO_U + j] = U[j];
    }
    co[CO_GA] = 0.5 * arE;
    return amu;
}

ADJ_HD void moment_adjoint(const double* co, const double* xi, double wi, double& a_g, double& a_h) {
    double c[3] = {xi[0] - co[CO_U], xi[1] - co[CO_U + 1], xi[2] - co[CO_U + 2]};
    const double aqc = co[CO_AQ] * c[0] + co[CO_AQ + 1] * c[1] + co[CO_AQ + 2] * c[2];
    a_g = wi * (co[CO_AL] + co[CO_BE] * xi[0] + co[CO_BE + 1] * xi[1] + co[CO_BE + 2] * xi[2] +
                co[CO_GA] * magsqr3(xi) + 0.5 * aqc * magsqr3(c));
    a_h = wi * (co[CO_GA] + 0.5 * aqc);
}

// raw moments of one DV's pair (g, h) added to m
ADJ_HD void add_moments(const double* xi, double wi, double g, double h, double* m) {
    const double a = wi * g, u = a * magsqr3(xi) + wi * h;
    m[0] += a;
    for (int k = 0; k < 3; ++k) {
        m[1 + k] += a * xi[k];
        m[5 + k] += u * xi[k];
    }
    m[4] += u;
    m[8] += a * xi[0] * xi[0];
    m[9] += a * xi[0] * xi[1];
    m[10] += a * xi[0] * xi[2];
    m[11] += a * xi[1] * xi[1];
    m[12] += a * xi[1] * xi[2];
    m[13] += a * xi[2] * xi[2];
}

// The Shakhov equilibrium of one entity (cell or face) over many DVs, with
// the entity's constants computed once: the same formula as shakhov(),
// with (2 pi R T)^(D/2) by multiplication and one exp per DV, and its
// reverse from the same intermediates.
struct ShkEntity {
    double U[3], q[3], rho, T, R, invRT, pref, iden, RTh, omp, k3;
    int D, K;
    ADJ_HD ShkEntity(const View& v, const double* Uv, double Tv, double rhov, const double* qv, double Th) {
        D = v.D;
        K = v.K;
        for (int k = 0; k < 3; ++k) {
            U[k] = Uv[k];
            q[k] = qv[k];
        }
        rho = rhov;
        T = Tv;
        R = v.R;
        const double RT = v.R * Tv;
        invRT = 1.0 / RT;
        const double s = sqrt(2.0 * kPi * RT);
        pref = rhov / (D == 3 ? s * s * s : D == 2 ? s * s : s);
        iden = 1.0 / (5.0 * rhov * RT * RT);
        RTh = v.R * Th;
        omp = 1.0 - v.Pr;
        k3 = K + 3.0 - D;
    }
    // per-DV intermediates
    struct DV {
        double c[3], cS, P, G0, A, Bh;
    };
    ADJ_HD DV at(const double* xi) const {
        DV d;
        for (int k = 0; k < 3; ++k) d.c[k] = xi[k] - U[k];
        d.cS = magsqr3(d.c) * invRT;
        d.P = dot3(d.c, q) * iden;
        d.G0 = pref * exp(-0.5 * d.cS);
        d.A = 1.0 + omp * d.P * (d.cS - D - 2.0);
        d.Bh = k3 + omp * d.P * ((d.cS - D) * k3 - 2 * K);
        return d;
    }
    ADJ_HD double g(const DV& d) const { return d.A * d.G0; }
    ADJ_HD double h(const DV& d) const { return d.Bh * d.G0 * RTh; }
    // adds the adjoints of rho, U, T, q and Th into s[0], s[1..3], s[4],
    // s[5..7], s[8], given the adjoints ag, ah of g^S and h^S
    ADJ_HD void rev(const DV& d, double ag, double ah, double* s) const {
        const double aG0 = ag * d.A + ah * d.Bh * RTh;
        const double aA = ag * d.G0, aB = ah * d.G0 * RTh;
        const double aP = omp * (aA * (d.cS - D - 2.0) + aB * ((d.cS - D) * k3 - 2 * K));
        const double acS = omp * d.P * (aA + aB * k3) - 0.5 * aG0 * d.G0;
        const double invT = 1.0 / T;
        s[0] += (aG0 * d.G0 - aP * d.P) / rho;
        s[4] += (-0.5 * D * aG0 * d.G0 - acS * d.cS - 2.0 * aP * d.P) * invT;
        const double f1 = 2.0 * acS * invRT, f2 = aP * iden;
        for (int k = 0; k < 3; ++k) {
            s[1 + k] -= f1 * d.c[k] + f2 * q[k];
            s[5 + k] += f2 * d.c[k];
        }
        s[8] += ah * d.Bh * d.G0 * R;
    }
};

// ---------------------------------------------------------------- forward

// inComingByRho of the wall faces (fvDVM.C:578-624)
struct FInBy {
    View v;
    ADJ_HD void operator()(int64_t b) const {
        double acc = 0;
        if (v.btype[b] == 1) {
            const double* S = v.S + 3 * (v.nIF + b);
            for (int i = 0; i < v.nv; ++i) {
                const double* xi = v.xi + 3 * i;
                const double xs = xs_of(xi, S);
                if (xs < 0) acc += -v.w[i] * xs * eq_by_rho(v, xi, v.bU + 3 * b, v.bT[b]);
            }
        }
        v.inby[b] = acc;
    }
};

// 1-3: the face values at the half step (wall incoming DVs come in stage 5)
// from the tiled pass A of the step (gbar+, the least-squares gradients and
// the upwind reconstruction, fvDVM.C:648-683, discreteVelocity.C:366-369,
// fvDVM.C:755-1029), gathered from item to face order.  A tile-boundary face
// has an item in each tile: the upwind tile writes the value into both, and
// on an exactly tangential face each holds its own side's half.  Far-field
// incoming DVs are not stored by pass A: rho_b M(U_owner, T_b) here.
struct FFace {
    View v;
    static constexpr int kMinCtas = 4;  // 32 warps per SM: at most 64 registers
    ADJ_HD void operator()(int64_t idx) const {
        const int i = static_cast<int>(idx / v.nF), f = static_cast<int>(idx % v.nF);
        const double* xi = v.xi + 3 * i;
        const double xs = xs_of(xi, v.S + 3 * f);
        const size_t r = static_cast<size_t>(i) * static_cast<size_t>(v.nI);
        const int it0 = v.fitems[2 * f], it1 = v.fitems[2 * f + 1];
        if (f < v.nIF) {
            double g = v.fvg[r + it0], h = v.fvh[r + it0];
            if (it1 >= 0 && !(xs >= kVSmall) && !(xs < -kVSmall)) {
                g += v.fvg[r + it1];
                h += v.fvh[r + it1];
            }
            v.fg[idx] = g;
            v.fh[idx] = h;
            return;
        }
        const int b = f - v.nIF, ow = v.own[f];
        if (xs > 0) {
            v.fg[idx] = v.fvg[r + it0];
            v.fh[idx] = v.fvh[r + it0];
        } else if (v.btype[b] == 2) {
            const double Tb = v.bT[b];
            const double gi = v.brho[b] * eq_by_rho(v, xi, v.cm + 9 * static_cast<size_t>(ow) + 1, Tb);
            v.fg[idx] = gi;
            v.fh[idx] = gi * (v.R * Tb) * static_cast<double>(v.K + 3 - v.D);
        }
    }
};

// 4: outgoing flux of the wall faces, per DV chunk (slot 14)
struct FWallOut {
    View v;
    ADJ_HD void operator()(int64_t idx) const {
        const int ch = static_cast<int>(idx / v.nBF), b = static_cast<int>(idx % v.nBF);
        const int f = v.nIF + b;
        double out = 0;
        if (v.btype[b] == 1) {
            const double* S = v.S + 3 * f;
            for (int i = chunk_lo(v.nv, v.nchF, ch); i < chunk_lo(v.nv, v.nchF, ch + 1); ++i) {
                const double xs = xs_of(v.xi + 3 * i, S);
                if (xs > 0) out += v.w[i] * xs * v.fg[at(i, v.nF, f)];
            }
        }
        v.pf[(static_cast<size_t>(ch) * v.nF + f) * kP + 14] = out;
    }
};

// 4b: rho_w = outgoing / |inComingByRho|
struct FWallRho {
    View v;
    ADJ_HD void operator()(int64_t b) const {
        const int f = v.nIF + static_cast<int>(b);
        double out = 0;
        for (int ch = 0; ch < v.nchF; ++ch) out += v.pf[(static_cast<size_t>(ch) * v.nF + f) * kP + 14];
        v.rhow[b] = v.btype[b] == 1 ? out / fabs(v.inby[b]) : 0.0;
    }
};

// 5: incoming wall DFs
struct FWallIn {
    View v;
    ADJ_HD void operator()(int64_t idx) const {
        const int i = static_cast<int>(idx / v.nBF), b = static_cast<int>(idx % v.nBF);
        if (v.btype[b] != 1) return;
        const int f = v.nIF + b;
        const double* xi = v.xi + 3 * i;
        if (xs_of(xi, v.S + 3 * f) <= 0) {
            const double Tb = v.bT[b];
            const double gi = v.rhow[b] * eq_by_rho(v, xi, v.bU + 3 * b, Tb);
            v.fg[at(i, v.nF, f)] = gi;
            v.fh[at(i, v.nF, f)] = gi * (v.R * Tb) * static_cast<double>(v.K + 3 - v.D);
        }
    }
};

// 6: raw moments of the face values, per DV chunk (slots 0..13)
struct FFaceMom {
    View v;
    static constexpr int kMinCtas = 4;  // 32 warps per SM: at most 64 registers
    ADJ_HD void operator()(int64_t idx) const {
        const int ch = static_cast<int>(idx / v.nF), f = static_cast<int>(idx % v.nF);
        double m[14] = {0};
        for (int i = chunk_lo(v.nv, v.nchF, ch); i < chunk_lo(v.nv, v.nchF, ch + 1); ++i)
            add_moments(v.xi + 3 * i, v.w[i], v.fg[at(i, v.nF, f)], v.fh[at(i, v.nF, f)], m);
        double* p = v.pf + (static_cast<size_t>(ch) * v.nF + f) * kP;
        for (int k = 0; k < 14; ++k) p[k] = m[k];
    }
};

// 6b: face macro records
struct FFaceMac {
    View v;
    ADJ_HD void operator()(int64_t f) const {
        double m[14] = {0};
        for (int ch = 0; ch < v.nchF; ++ch) {
            const double* p = v.pf + (static_cast<size_t>(ch) * v.nF + f) * kP;
            for (int k = 0; k < 14; ++k) m[k] += p[k];
        }
        macros_from_moments(v, m, 0.5 * v.dt * v.Pr, v.fmac + kMac * static_cast<size_t>(f));
    }
};

// raw moments of the state, per DV chunk, and the cell macro records
struct FCellMom {
    View v;
    static constexpr int kMinCtas = 3;  // 24 warps per SM: at most 80 registers
    ADJ_HD void operator()(int64_t idx) const {
        const int ch = static_cast<int>(idx / v.nC), c = static_cast<int>(idx % v.nC);
        double m[14] = {0};
        for (int i = chunk_lo(v.nv, v.nchC, ch); i < chunk_lo(v.nv, v.nchC, ch + 1); ++i)
            add_moments(v.xi + 3 * i, v.w[i], v.g[at(i, v.nC, c)], v.h[at(i, v.nC, c)], m);
        double* p = v.pc + (static_cast<size_t>(ch) * v.nC + c) * kP;
        for (int k = 0; k < 14; ++k) p[k] = m[k];
    }
};
struct FCellMac {
    View v;
    ADJ_HD void operator()(int64_t c) const {
        double m[14] = {0};
        for (int ch = 0; ch < v.nchC; ++ch) {
            const double* p = v.pc + (static_cast<size_t>(ch) * v.nC + c) * kP;
            for (int k = 0; k < 14; ++k) m[k] += p[k];
        }
        macros_from_moments(v, m, v.dt * v.Pr, v.cmac + kMac * static_cast<size_t>(c));
    }
};

// the relaxed value of face f's DV i, and whether it is relaxed
ADJ_HD bool relaxed_value(const View& v, int i, int f, double& gr, double& hr, double& gEq, double& hEq,
                          double& r) {
    const double* xi = v.xi + 3 * i;
    const size_t id = at(i, v.nF, f);
    gr = v.fg[id];
    hr = v.fh[id];
    if (f >= v.nIF && !(xs_of(xi, v.S + 3 * f) > 0)) return false;
    const double* m = v.fmac + kMac * static_cast<size_t>(f);
    const double Th = f < v.nIF ? m[MAC_T] : v.fmac[kMac * static_cast<size_t>(v.blocal[f - v.nIF]) + MAC_T];
    r = 0.5 * v.dt / (2.0 * m[MAC_TAU] + 0.5 * v.dt);
    shakhov(v, xi, m + MAC_U, m[MAC_T], m[MAC_RHO], m + MAC_Q, Th, gEq, hEq);
    gr = (1.0 - r) * gr + r * gEq;
    hr = (1.0 - r) * hr + r * hEq;
    return true;
}

// the objective of one step: every boundary face's energy and momentum flux
// of its relaxed DFs, weighted by wn, added to Jb
struct FObjective {
    View v;
    ADJ_HD void operator()(int64_t bi) const {
        const int b = static_cast<int>(bi), f = v.nIF + b;
        const double* S = v.S + 3 * f;
        const double ea = v.wn * v.ha[b];
        double s = 0;
        for (int i = 0; i < v.nv; ++i) {
            const double* xi = v.xi + 3 * i;
            double gr, hr, gEq, hEq, r;
            relaxed_value(v, i, f, gr, hr, gEq, hEq, r);
            const double wx = v.w[i] * xs_of(xi, S);
            s += wx * (ea * 0.5 * (magsqr3(xi) * gr + hr) + v.wn * dot3(v.fw + 3 * b, xi) * gr);
        }
        v.Jb[b] += s;
    }
};

// mass, momentum and energy flux of every boundary face's relaxed DFs
// (the fluxes of fvDVM::updateGHtildeVol, fvDVM.C:1500-1517), along Sf:
// out[5b..5b+4] = sum_i w_i (xi_i.Sf) {g, xi g, (|xi|^2 g + h)/2}
struct FBoundaryFlux {
    View v;
    double* out;
    ADJ_HD void operator()(int64_t bi) const {
        const int b = static_cast<int>(bi), f = v.nIF + b;
        const double* S = v.S + 3 * f;
        double m = 0, p[3] = {0, 0, 0}, e = 0;
        for (int i = 0; i < v.nv; ++i) {
            const double* xi = v.xi + 3 * i;
            double gr, hr, gEq, hEq, r;
            relaxed_value(v, i, f, gr, hr, gEq, hEq, r);
            const double a = v.w[i] * xs_of(xi, S) * gr;
            m += a;
            for (int k = 0; k < 3; ++k) p[k] += a * xi[k];
            e += v.w[i] * xs_of(xi, S) * 0.5 * (magsqr3(xi) * gr + hr);
        }
        double* o = out + 5 * static_cast<size_t>(b);
        o[0] = m;
        for (int k = 0; k < 3; ++k) o[1 + k] = p[k];
        o[4] = e;
    }
};

// ---------------------------------------------------------------- reverse

// R1: adjoint of the relaxed face values (from the update and the
// objective), its part through the relaxation, the Shakhov and relax-factor
// sums per DV chunk, and the objective
struct RRelax {
    View v;
    static constexpr int kMinCtas = 2;  // 16 warps per SM: at most 128 registers
    ADJ_HD void operator()(int64_t idx) const {
        const int ch = static_cast<int>(idx / v.nF), f = static_cast<int>(idx % v.nF);
        const bool bnd = f >= v.nIF;
        const int b = f - v.nIF;
        const int ow = v.own[f], ne = bnd ? ow : v.nei[f];
        const double* m = v.fmac + kMac * static_cast<size_t>(f);
        const double dtVo = v.dt * v.invV[ow], dtVn = bnd ? 0.0 : v.dt * v.invV[ne];
        const double ea = bnd ? v.wn * v.ha[b] : 0.0;
        double cw[3] = {0, 0, 0};
        if (bnd)
            for (int k = 0; k < 3; ++k) cw[k] = v.wn * v.fw[3 * b + k];
        const double S[3] = {v.S[3 * f], v.S[3 * f + 1], v.S[3 * f + 2]};
        // h^S of a boundary face is scaled by the internal-face T at its patch-local index
        const double Th = !bnd ? m[MAC_T] : v.fmac[kMac * static_cast<size_t>(v.blocal[b]) + MAC_T];
        const ShkEntity e(v, m + MAC_U, m[MAC_T], m[MAC_RHO], m + MAC_Q, Th);
        const double r = 0.5 * v.dt / (2.0 * m[MAC_TAU] + 0.5 * v.dt);
        double s[12] = {0};
        for (int i = chunk_lo(v.nv, v.nchF, ch); i < chunk_lo(v.nv, v.nchF, ch + 1); ++i) {
            const double* xi = v.xi + 3 * i;
            const double xs = xs_of(xi, S);
            const size_t id = at(i, v.nF, f);
            const double lgo = ro(v.lg + at(i, v.nC, ow)), lho = ro(v.lh + at(i, v.nC, ow));
            const double lgn = ro(v.lg + at(i, v.nC, ne)), lhn = ro(v.lh + at(i, v.nC, ne));
            const double pg = ro(v.fg + id), ph = ro(v.fh + id);
            double a_g = xs * (dtVn * lgn - dtVo * lgo);
            double a_h = xs * (dtVn * lhn - dtVo * lho);
            const bool rel = !bnd || xs > 0;
            ShkEntity::DV d{};
            double gEq = 0, hEq = 0;
            if (rel) {
                d = e.at(xi);
                gEq = e.g(d);
                hEq = e.h(d);
            }
            if (bnd) {
                const double gr = rel ? (1.0 - r) * pg + r * gEq : pg;
                const double hr = rel ? (1.0 - r) * ph + r * hEq : ph;
                const double wx = v.w[i] * xs, x2 = magsqr3(xi), cg = dot3(cw, xi);
                s[10] += wx * (ea * 0.5 * (x2 * gr + hr) + cg * gr);
                a_g += wx * (ea * 0.5 * x2 + cg);
                a_h += wx * ea * 0.5;
            }
            if (rel) {
                s[0] += (gEq - pg) * a_g + (hEq - ph) * a_h;
                e.rev(d, r * a_g, r * a_h, s + 1);
                v.ag[id] = (1.0 - r) * a_g;
                v.ah[id] = (1.0 - r) * a_h;
            } else {
                v.ag[id] = a_g;
                v.ah[id] = a_h;
            }
        }
        double* p = v.pf + (static_cast<size_t>(ch) * v.nF + f) * kP;
        for (int k = 0; k < 11; ++k) p[k] = s[k];
    }
};

// R2: the face macro adjoint (with the h^S temperatures of boundary faces
// that take this face's T) and its per-DV coefficient record; muRef and the
// objective are accumulated
struct RFaceMac {
    View v;
    ADJ_HD double psum(int f, int k) const {
        double a = 0;
        for (int ch = 0; ch < v.nchF; ++ch) a += v.pf[(static_cast<size_t>(ch) * v.nF + f) * kP + k];
        return a;
    }
    ADJ_HD void operator()(int64_t fi) const {
        const int f = static_cast<int>(fi);
        const double* m = v.fmac + kMac * static_cast<size_t>(f);
        double aM[9];
        for (int k = 0; k < 8; ++k) aM[k] = psum(f, 1 + k);
        // h^S scaled by this face's own T (internal faces), and by it on the
        // boundary faces whose patch-local index is f
        if (f < v.nIF) aM[4] += psum(f, 9);
        for (int e = v.th_off[f]; e < v.th_off[f + 1]; ++e) aM[4] += psum(v.nIF + v.th_ent[e], 9);
        const double ar = psum(f, 0);
        const double tau = m[MAC_TAU], den = 2.0 * tau + 0.5 * v.dt;
        aM[8] = -ar * v.dt / (den * den);
        v.amuF[f] += macros_rev(v, m, 0.5 * v.dt * v.Pr, aM, v.fco + kCo * static_cast<size_t>(f));
        if (f >= v.nIF) v.Jb[f - v.nIF] += psum(f, 10);
    }
};

// R3: the face-moment part of the face-value adjoint; on boundary faces the
// incoming DFs' parameters, per DV chunk: wall rho_w (slot 0), T_b (1),
// U_b or the owner U (2..4)
struct RFaceMom {
    View v;
    static constexpr int kMinCtas = 4;  // 32 warps per SM: at most 64 registers
    ADJ_HD void operator()(int64_t idx) const {
        const int ch = static_cast<int>(idx / v.nF), f = static_cast<int>(idx % v.nF);
        const double* co = v.fco + kCo * static_cast<size_t>(f);
        const bool bnd = f >= v.nIF;
        const int b = f - v.nIF;
        const int type = bnd ? v.btype[b] : 0;
        double s[5] = {0, 0, 0, 0, 0};
        for (int i = chunk_lo(v.nv, v.nchF, ch); i < chunk_lo(v.nv, v.nchF, ch + 1); ++i) {
            const double* xi = v.xi + 3 * i;
            const size_t id = at(i, v.nF, f);
            double a_g, a_h;
            moment_adjoint(co, xi, v.w[i], a_g, a_h);
            a_g += v.ag[id];
            a_h += v.ah[id];
            v.ag[id] = a_g;
            v.ah[id] = a_h;
            if (!bnd || xs_of(xi, v.S + 3 * f) > 0) continue;
            // incoming: g = rho_in E(U_in, T_b), h = g R T_b (K+3-D)
            const double Tb = v.bT[b], k3 = static_cast<double>(v.K + 3 - v.D);
            const double* Uin = type == 1 ? v.bU + 3 * b : v.cm + 9 * static_cast<size_t>(v.own[f]) + 1;
            const double rin = type == 1 ? v.rhow[b] : v.brho[b];
            const double E = eq_by_rho(v, xi, Uin, Tb);
            double dET, dEU[3];
            eq_by_rho_d(v, xi, Uin, Tb, E, dET, dEU);
            const double agt = a_g + a_h * v.R * Tb * k3;
            s[0] += agt * E;
            s[1] += agt * rin * dET + a_h * rin * E * v.R * k3;
            for (int k = 0; k < 3; ++k) s[2 + k] += agt * rin * dEU[k];
        }
        if (bnd) {
            double* p = v.pf + (static_cast<size_t>(ch) * v.nF + f) * kP;
            for (int k = 0; k < 5; ++k) p[k] = s[k];
        }
    }
};

// R3b: per boundary face: the wall density's adjoint into the outgoing
// flux and inComingByRho, the parameters' adjoints
struct RBoundary {
    View v;
    ADJ_HD void operator()(int64_t bi) const {
        const int b = static_cast<int>(bi), f = v.nIF + b;
        double s[5] = {0, 0, 0, 0, 0};
        for (int ch = 0; ch < v.nchF; ++ch)
            for (int k = 0; k < 5; ++k) s[k] += v.pf[(static_cast<size_t>(ch) * v.nF + f) * kP + k];
        v.gTb[b] += s[1];
        if (v.btype[b] == 1) {
            const double I = v.inby[b];
            v.aout[b] = s[0] / fabs(I);
            v.aI[b] += -s[0] * v.rhow[b] / I;
            for (int k = 0; k < 3; ++k) {
                v.gUb[3 * b + k] += s[2 + k];
                v.aUown[3 * b + k] = 0.0;
            }
        } else {
            v.aout[b] = 0.0;
            for (int k = 0; k < 3; ++k) v.aUown[3 * b + k] = s[2 + k];
        }
    }
};

// R3c: the outgoing flux's adjoint into the outgoing wall DFs
struct RWallOut {
    View v;
    ADJ_HD void operator()(int64_t idx) const {
        const int i = static_cast<int>(idx / v.nBF), b = static_cast<int>(idx % v.nBF);
        if (v.btype[b] != 1) return;
        const int f = v.nIF + b;
        const double xs = xs_of(v.xi + 3 * i, v.S + 3 * f);
        if (xs > 0) v.ag[at(i, v.nF, f)] += v.aout[b] * v.w[i] * xs;
    }
};

// R4: per (DV, cell): the adjoints of the cell's gradients and the direct
// part of the gbar+ adjoint (faces where the cell is the upwind side), with
// 4/3 of the state adjoint; written to og/oh
struct RGradAdj {
    View v;
    ADJ_HD void operator()(int64_t idx) const {
        const int i = static_cast<int>(idx / v.nC), c = static_cast<int>(idx % v.nC);
        const double* xi = v.xi + 3 * i;
        double Gg[3] = {0, 0, 0}, Gh[3] = {0, 0, 0};
        double dg = 4.0 / 3 * v.lg[idx], dh = 4.0 / 3 * v.lh[idx];
        for (int e = v.cf_off[c]; e < v.cf_off[c + 1]; ++e) {
            const int f = v.cf_ent[e] >> 1;
            const bool is_nei = v.cf_ent[e] & 1;
            const double xs = xs_of(xi, v.S + 3 * f);
            double share;
            if (f >= v.nIF) share = xs > 0 ? 1.0 : 0.0;
            else if (xs >= kVSmall) share = is_nei ? 0.0 : 1.0;
            else if (xs < -kVSmall) share = is_nei ? 1.0 : 0.0;
            else share = 0.5;
            if (share == 0.0) continue;
            const size_t id = at(i, v.nF, f);
            const double a_g = share * v.ag[id], a_h = share * v.ah[id];
            double d[3];
            recon_vec(v, f, c, xi, d);
            dg += a_g;
            dh += a_h;
            for (int k = 0; k < 3; ++k) {
                Gg[k] += a_g * d[k];
                Gh[k] += a_h * d[k];
            }
        }
        const size_t n = static_cast<size_t>(v.nv) * v.nC;
        for (int k = 0; k < 3; ++k) {
            v.aGg[k * n + idx] = Gg[k];
            v.aGh[k * n + idx] = Gh[k];
        }
        v.og[idx] = dg;
        v.oh[idx] = dh;
    }
};

// R5: per (cell, DV chunk): the gradient's adjoint into gbar+, the half
// step's reverse into the state adjoint, and the cell's Shakhov and
// relax-factor sums.  A cell with at most kRegF internal faces keeps its
// face list (face, other cell, side) in registers for the chunk's DVs and
// walks it unrolled, so the neighbours' gradient-adjoint loads of all its
// faces are independent of one another; cells with more faces walk the
// list from memory.  Either way the faces are added in list order.
struct RHalf {
    View v;
    static constexpr int kRegF = 6;
    static constexpr int kMinCtas = 2;  // 16 warps per SM: at most 128 registers
    ADJ_HD void face_add(size_t cb, size_t n, int f, int o, bool is_nei, const double* gc, const double* hc,
                         double& abg, double& abh) const {
        const size_t io = cb + o;
        const double go[3] = {ro(v.aGg + io), ro(v.aGg + n + io), ro(v.aGg + 2 * n + io)};
        const double ho[3] = {ro(v.aGh + io), ro(v.aGh + n + io), ro(v.aGh + 2 * n + io)};
        const double P[3] = {ro(v.lsP + 3 * f), ro(v.lsP + 3 * f + 1), ro(v.lsP + 3 * f + 2)};
        const double N[3] = {ro(v.lsN + 3 * f), ro(v.lsN + 3 * f + 1), ro(v.lsN + 3 * f + 2)};
        // s_f = lsP . aG_own - lsN . aG_nei; the neighbour adds it, the owner subtracts it
        if (is_nei) {
            abg += dot3(P, go) - dot3(N, gc);
            abh += dot3(P, ho) - dot3(N, hc);
        } else {
            abg -= dot3(P, gc) - dot3(N, go);
            abh -= dot3(P, hc) - dot3(N, ho);
        }
    }
    ADJ_HD void operator()(int64_t idx) const {
        const int ch = static_cast<int>(idx / v.nC), c = static_cast<int>(idx % v.nC);
        const double* m = v.cm + 9 * static_cast<size_t>(c);
        const double tau = tau_of(v, m[4], m[0]);
        const double r = 1.5 * v.dt / (2.0 * tau + v.dt);
        const ShkEntity e(v, m + 1, m[4], m[0], m + 5, m[4]);
        const size_t n = static_cast<size_t>(v.nv) * v.nC;
        const int e0 = v.cf_off[c], e1 = v.cf_off[c + 1];
        // the internal faces lead the cell's list
        int nf = 0;
        while (e0 + nf < e1 && (ro(v.cf_ent + e0 + nf) >> 1) < v.nIF) ++nf;
        const bool reg = nf <= kRegF;
        int rf[kRegF], oc[kRegF];
        unsigned rn = 0;
#pragma unroll
        for (int q = 0; q < kRegF; ++q) {
            rf[q] = 0;
            oc[q] = 0;
            if (reg && q < nf) {
                const int ent = ro(v.cf_ent + e0 + q);
                rf[q] = ent >> 1;
                if (ent & 1) rn |= 1u << q;
                oc[q] = (ent & 1) ? ro(v.own + rf[q]) : ro(v.nei + rf[q]);  // the other cell of the face
            }
        }
        double s[9] = {0};
        for (int i = chunk_lo(v.nv, v.nchC, ch); i < chunk_lo(v.nv, v.nchC, ch + 1); ++i) {
            const size_t cb = at(i, v.nC, 0), id = cb + c;
            double abg = v.og[id], abh = v.oh[id];
            const double gc[3] = {ro(v.aGg + id), ro(v.aGg + n + id), ro(v.aGg + 2 * n + id)};
            const double hc[3] = {ro(v.aGh + id), ro(v.aGh + n + id), ro(v.aGh + 2 * n + id)};
            if (reg) {
#pragma unroll
                for (int q = 0; q < kRegF; ++q)
                    if (q < nf) face_add(cb, n, rf[q], oc[q], (rn >> q) & 1u, gc, hc, abg, abh);
            } else {
                for (int en = e0; en < e0 + nf; ++en) {
                    const int ent = ro(v.cf_ent + en);
                    const int f = ent >> 1;
                    face_add(cb, n, f, (ent & 1) ? ro(v.own + f) : ro(v.nei + f), ent & 1, gc, hc, abg, abh);
                }
            }
            const ShkEntity::DV d = e.at(v.xi + 3 * i);
            const double gEq = e.g(d), hEq = e.h(d);
            s[0] += (gEq - ro(v.g + id)) * abg + (hEq - ro(v.h + id)) * abh;
            double t[9] = {0};
            e.rev(d, r * abg, r * abh, t);
            for (int k = 0; k < 8; ++k) s[1 + k] += t[k];
            s[5] += t[8];  // h^S of a cell is scaled by the cell's own T
            v.og[id] = -1.0 / 3 * ro(v.lg + id) + (1.0 - r) * abg;
            v.oh[id] = -1.0 / 3 * ro(v.lh + id) + (1.0 - r) * abh;
        }
        double* p = v.pc + (static_cast<size_t>(ch) * v.nC + c) * kP;
        for (int k = 0; k < 9; ++k) p[k] = s[k];
    }
};

// R6: per cell: the macro adjoint (with the far-field incoming DFs that take
// the cell's U) and, when the macros are moments of the state, its per-DV
// coefficient record
struct RCellMac {
    View v;
    ADJ_HD void operator()(int64_t ci) const {
        const int c = static_cast<int>(ci);
        const double* m = v.cm + 9 * static_cast<size_t>(c);
        double s[9] = {0};
        for (int ch = 0; ch < v.nchC; ++ch)
            for (int k = 0; k < 9; ++k) s[k] += v.pc[(static_cast<size_t>(ch) * v.nC + c) * kP + k];
        double aM[9];
        for (int k = 0; k < 8; ++k) aM[k] = s[1 + k];
        for (int e = v.cf_off[c]; e < v.cf_off[c + 1]; ++e) {
            const int f = v.cf_ent[e] >> 1;
            if (f < v.nIF || v.btype[f - v.nIF] != 2) continue;
            for (int k = 0; k < 3; ++k) aM[1 + k] += v.aUown[3 * (f - v.nIF) + k];
        }
        // r = 1.5 dt / (2 tau + dt), tau = tau_of(T, rho)
        const double tau = tau_of(v, m[4], m[0]);
        const double den = 2.0 * tau + v.dt;
        const double atau = -s[0] * 3.0 * v.dt / (den * den);
        aM[4] += atau * tau * (v.omega - 1.0) / m[4];
        aM[0] -= atau * tau / m[0];
        v.amuC[c] += atau * tau / v.mu;
        if (!v.fold) return;
        aM[8] = 0.0;  // the step recomputes tau from T and rho
        v.amuC[c] += macros_rev(v, v.cmac + kMac * static_cast<size_t>(c), v.dt * v.Pr, aM,
                                v.cco + kCo * static_cast<size_t>(c));
    }
};

// R7: the cell macros' adjoint into the state adjoint
struct RCellMom {
    View v;
    ADJ_HD void operator()(int64_t idx) const {
        const int i = static_cast<int>(idx / v.nC), c = static_cast<int>(idx % v.nC);
        double a_g, a_h;
        moment_adjoint(v.cco + kCo * static_cast<size_t>(c), v.xi + 3 * i, v.w[i], a_g, a_h);
        v.og[idx] += a_g;
        v.oh[idx] += a_h;
    }
};

// the parameters' adjoint through inComingByRho (wall faces), at the end
struct RInBy {
    View v;
    ADJ_HD void operator()(int64_t bi) const {
        const int b = static_cast<int>(bi);
        if (v.btype[b] != 1) return;
        const double* S = v.S + 3 * (v.nIF + b);
        double sT = 0, sU[3] = {0, 0, 0};
        for (int i = 0; i < v.nv; ++i) {
            const double* xi = v.xi + 3 * i;
            const double xs = xs_of(xi, S);
            if (!(xs < 0)) continue;
            const double E = eq_by_rho(v, xi, v.bU + 3 * b, v.bT[b]);
            double dET, dEU[3];
            eq_by_rho_d(v, xi, v.bU + 3 * b, v.bT[b], E, dET, dEU);
            sT += -v.w[i] * xs * dET;
            for (int k = 0; k < 3; ++k) sU[k] += -v.w[i] * xs * dEU[k];
        }
        v.gTb[b] += v.aI[b] * sT;
        for (int k = 0; k < 3; ++k) v.gUb[3 * b + k] += v.aI[b] * sU[k];
    }
};

// ---------------------------------------------------------------- sequences

// Ex: run(n, functor) applies the functor to 0..n-1 (in any order).
template <class Ex>
int record_step(Ex& ex, const View& v) {
    int st;
    if ((st = ex.pass_a(v))) return st;
    if ((st = ex.run(static_cast<int64_t>(v.nv) * v.nF, FFace{v}))) return st;
    if (v.nBF > 0) {
        if ((st = ex.run(static_cast<int64_t>(v.nchF) * v.nBF, FWallOut{v}))) return st;
        if ((st = ex.run(v.nBF, FWallRho{v}))) return st;
        if ((st = ex.run(static_cast<int64_t>(v.nv) * v.nBF, FWallIn{v}))) return st;
    }
    if ((st = ex.run(static_cast<int64_t>(v.nchF) * v.nF, FFaceMom{v}))) return st;
    return ex.run(v.nF, FFaceMac{v});
}

// reverse of one step from its record: og/oh = adjoint of the state before
// the step, given lg/lh, the adjoint of the state after it
template <class Ex>
int reverse_step(Ex& ex, const View& v) {
    int st;
    if (v.fold) {
        if ((st = ex.run(static_cast<int64_t>(v.nchC) * v.nC, FCellMom{v}))) return st;
        if ((st = ex.run(v.nC, FCellMac{v}))) return st;
    }
    if ((st = ex.run(static_cast<int64_t>(v.nchF) * v.nF, RRelax{v}))) return st;
    if ((st = ex.run(v.nF, RFaceMac{v}))) return st;
    if ((st = ex.run(static_cast<int64_t>(v.nchF) * v.nF, RFaceMom{v}))) return st;
    if (v.nBF > 0) {
        if ((st = ex.run(v.nBF, RBoundary{v}))) return st;
        if ((st = ex.run(static_cast<int64_t>(v.nv) * v.nBF, RWallOut{v}))) return st;
    }
    if ((st = ex.run(static_cast<int64_t>(v.nv) * v.nC, RGradAdj{v}))) return st;
    if ((st = ex.run(static_cast<int64_t>(v.nchC) * v.nC, RHalf{v}))) return st;
    if ((st = ex.run(v.nC, RCellMac{v}))) return st;
    if (v.fold) return ex.run(static_cast<int64_t>(v.nv) * v.nC, RCellMom{v});
    return 0;
}

// DV chunk count of a per-entity reduction: enough (entity, chunk) threads
// to fill the GPU, at most 64 chunks and one DV per chunk
inline int chunks_for(int n_entities, int nv, int64_t target_threads) {
    int64_t c = (target_threads + n_entities - 1) / (n_entities > 0 ? n_entities : 1);
    if (c < 1) c = 1;
    if (c > 64) c = 64;
    if (c > nv) c = nv;
    return static_cast<int>(c);
}

// ---------------------------------------------------------------- checkpoints

// Binomial checkpointing (Griewank's revolve schedule).  A segment of n
// steps whose start state is held in one slot, with c slots in all (that one
// included), can be reversed with r recomputations of each step as long as
// n <= beta(c, r) = C(c + r, c); the fewest forward steps are
//   T(n, c) = r n - beta(c + 1, r - 1),  r the least with beta(c, r) >= n.
// The next checkpoint goes m steps in, where the rest (n - m steps, c - 1
// slots) needs exactly r recomputations and the first m steps (c slots)
// r - 1: then m + T(n - m, c - 1) + T(m, c) = T(n, c) by Pascal's rule.
// Ops provides save(slot), restore(slot), advance(k) (k forward steps from
// the current state) and reverse(n) (record and reverse step n, whose start
// state is current).
inline double beta(int c, int r) {
    if (r < 0) return 0;
    double b = 1;
    for (int j = 1; j <= c; ++j) b = b * (r + j) / j;
    return b;
}

inline int reps_for(double n, int c) {
    int r = 0;
    while (beta(c, r) < n) ++r;
    return r;
}

// fewest forward steps to reverse n steps with c slots (the start's included)
inline double optimal_forward(int n, int c) {
    if (n <= 1) return 0;
    const int r = reps_for(n, c);
    return r * static_cast<double>(n) - beta(c + 1, r - 1);
}

// offset of the next checkpoint in a segment of n >= 2 steps with c >= 2 slots
inline int checkpoint_split(int n, int c) {
    const int r = reps_for(n, c);
    const double lo = std::max({static_cast<double>(n) - beta(c - 1, r), beta(c, r - 2) + 1, 1.0});
    const double hi = std::min({static_cast<double>(n) - beta(c - 1, r - 1) - 1, beta(c, r - 1), n - 1.0});
    if (lo <= hi) return static_cast<int>(hi);
    // just past a boundary beta(c, r - 1) the optimal split mixes other
    // recomputation counts: search for it
    const double best = optimal_forward(n, c);
    for (int m = n - 1; m >= 1; --m)
        if (m + optimal_forward(n - m, c - 1) + optimal_forward(m, c) == best) return m;
    return 1;
}

template <class Ops>
int revolve(Ops& ops, int a, int b, int slot_a, int free_lo, int free_n) {
    int st;
    const int n = b - a;
    if (n == 1) return ops.reverse(a);
    if (free_n == 0) {
        for (int j = b - 1; j >= a; --j) {
            if ((st = ops.restore(slot_a))) return st;
            if ((st = ops.advance(j - a))) return st;
            if ((st = ops.reverse(j))) return st;
        }
        return 0;
    }
    const int m = a + checkpoint_split(n, free_n + 1);
    if ((st = ops.advance(m - a))) return st;
    if ((st = ops.save(free_lo))) return st;
    if ((st = revolve(ops, m, b, free_lo, free_lo + 1, free_n - 1))) return st;
    if ((st = ops.restore(slot_a))) return st;
    return revolve(ops, a, m, slot_a, free_lo, free_n);
}

// whole run: slot 0 holds the start state; n_slots >= 1
template <class Ops>
int revolve_run(Ops& ops, int n_steps, int n_slots) {
    int st;
    if ((st = ops.save(0))) return st;
    return revolve(ops, 0, n_steps, 0, 1, n_slots - 1);
}

// host-side mesh tables of the adjoint, from the flattened mesh in the
// numbering the state uses
struct HostTables {
    std::vector<int32_t> own, nei, cf_off, cf_ent, th_off, th_ent;
    std::vector<double> invV;
};

inline void build_tables(int nC, int nIF, int nBF, const int32_t* own, const int32_t* nei, const double* V,
                         const int32_t* blocal, HostTables& t) {
    const int nF = nIF + nBF;
    t.own.assign(own, own + nF);
    t.nei.assign(nei, nei + nIF);
    t.invV.resize(nC);
    for (int c = 0; c < nC; ++c) t.invV[c] = 1.0 / V[c];
    std::vector<int32_t> cnt(nC + 1, 0);
    for (int f = 0; f < nF; ++f) {
        cnt[own[f] + 1]++;
        if (f < nIF) cnt[nei[f] + 1]++;
    }
    t.cf_off.assign(nC + 1, 0);
    for (int c = 0; c < nC; ++c) t.cf_off[c + 1] = t.cf_off[c] + cnt[c + 1];
    t.cf_ent.assign(t.cf_off[nC], 0);
    std::vector<int32_t> pos(t.cf_off.begin(), t.cf_off.end() - 1);
    for (int f = 0; f < nF; ++f) {  // face order within each cell
        t.cf_ent[pos[own[f]]++] = 2 * f;
        if (f < nIF) t.cf_ent[pos[nei[f]]++] = 2 * f + 1;
    }
    std::vector<int32_t> tc(nF + 1, 0);
    for (int b = 0; b < nBF; ++b)
        if (blocal[b] >= 0 && blocal[b] < nF) tc[blocal[b] + 1]++;
    t.th_off.assign(nF + 1, 0);
    for (int f = 0; f < nF; ++f) t.th_off[f + 1] = t.th_off[f] + tc[f + 1];
    t.th_ent.assign(t.th_off[nF], 0);
    std::vector<int32_t> tp(t.th_off.begin(), t.th_off.end() - 1);
    for (int b = 0; b < nBF; ++b)
        if (blocal[b] >= 0 && blocal[b] < nF) t.th_ent[tp[blocal[b]]++] = b;
}

}  // namespace adj
}  // namespace dugks

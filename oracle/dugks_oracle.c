/*
 * CPU FP64 oracle for the DUGKS step -- TEST INFRASTRUCTURE ONLY (see
 * dugks_oracle.h).  Each function names the reference lines it restates;
 * expressions keep the reference's operand order so that the rounding
 * matches as far as a restatement can.
 *
 * Reference files (paths inside the dugksFoam project):
 *   src/fvDVM/fvDVM/fvDVM.C                       the step and its sub-steps
 *   src/fvDVM/discreteVelocity/discreteVelocity.C equilibria, BC-type map
 *   src/fvDVM/BCs/calculatedMaxwellFvPatchField/calculatedMaxwellFvPatchField.C
 *   src/fvDVM/BCs/farFieldFvPatchField/farFieldFvPatchField.H (no-op assignment)
 *   src/fvDVM/BCs/pressureInFvPatchField, pressureOutFvPatchField,
 *   symmetryModFvPatchField (their value starts at one: the dictionary
 *       constructors assign pTraits<Type>::one)
 *   src/fvDVM/zeroBoundaryGrad/zeroBoundaryVectors.C, zeroBoundaryGrad.C
 *       (least squares; the commented boundary terms restored = stock
 *        leastSquares, which the cases select in system/fvSchemes)
 */
#include "dugks_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VSMALL 1.0e-300

#include "dugks_oracle_state.h"

static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline double magsqr3(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

/* ------------------------------------------------------------------------
 * Mesh geometry: OpenFOAM primitiveMesh face centres/areas (triangle fan
 * about the point average) and cell centres/volumes (face pyramids about
 * the face-centre average).
 * ---------------------------------------------------------------------- */
void oracle_geometry(int n_points, const double* p, int n_faces, const int64_t* fo, const int64_t* fp,
                     const int64_t* owner, int n_internal, const int64_t* neighbour, int n_cells,
                     double* Cf, double* Sf, double* C, double* V) {
    (void)n_points;
    for (int f = 0; f < n_faces; ++f) {
        int64_t b = fo[f], e = fo[f + 1];
        int np = (int)(e - b);
        if (np == 3) {
            const double *a = p + 3 * fp[b], *bb = p + 3 * fp[b + 1], *c = p + 3 * fp[b + 2];
            double u[3] = {bb[0] - a[0], bb[1] - a[1], bb[2] - a[2]};
            double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
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
        double sumN[3] = {0, 0, 0}, sumA = 0.0, sumAc[3] = {0, 0, 0};
        for (int i = 0; i < np; ++i) {
            const double* pi = p + 3 * fp[b + i];
            const double* pn = p + 3 * fp[b + (i + 1) % np];
            double c[3], u[3], v[3], n[3];
            for (int k = 0; k < 3; ++k) {
                c[k] = pi[k] + pn[k] + fc[k];
                u[k] = pn[k] - pi[k];
                v[k] = fc[k] - pi[k];
            }
            n[0] = u[1] * v[2] - u[2] * v[1];
            n[1] = u[2] * v[0] - u[0] * v[2];
            n[2] = u[0] * v[1] - u[1] * v[0];
            double a = sqrt(magsqr3(n));
            for (int k = 0; k < 3; ++k) {
                sumN[k] += n[k];
                sumAc[k] += a * c[k];
            }
            sumA += a;
        }
        if (sumA < 1.0e-150) {
            for (int k = 0; k < 3; ++k) {
                Cf[3 * f + k] = fc[k];
                Sf[3 * f + k] = 0.0;
            }
        } else {
            for (int k = 0; k < 3; ++k) {
                Cf[3 * f + k] = (1.0 / 3.0) * sumAc[k] / sumA;
                Sf[3 * f + k] = 0.5 * sumN[k];
            }
        }
    }
    double* cEst = (double*)calloc((size_t)3 * n_cells, sizeof(double));
    int* nf = (int*)calloc((size_t)n_cells, sizeof(int));
    for (int f = 0; f < n_faces; ++f) {
        for (int k = 0; k < 3; ++k) cEst[3 * owner[f] + k] += Cf[3 * f + k];
        nf[owner[f]]++;
    }
    for (int f = 0; f < n_internal; ++f) {
        for (int k = 0; k < 3; ++k) cEst[3 * neighbour[f] + k] += Cf[3 * f + k];
        nf[neighbour[f]]++;
    }
    for (int c = 0; c < n_cells; ++c)
        for (int k = 0; k < 3; ++k) cEst[3 * c + k] /= nf[c];
    memset(C, 0, sizeof(double) * 3 * n_cells);
    memset(V, 0, sizeof(double) * n_cells);
    for (int f = 0; f < n_faces; ++f) {
        int64_t c = owner[f];
        double d[3] = {Cf[3 * f] - cEst[3 * c], Cf[3 * f + 1] - cEst[3 * c + 1], Cf[3 * f + 2] - cEst[3 * c + 2]};
        double pyr3 = dot3(Sf + 3 * f, d);
        for (int k = 0; k < 3; ++k) C[3 * c + k] += pyr3 * ((3.0 / 4.0) * Cf[3 * f + k] + (1.0 / 4.0) * cEst[3 * c + k]);
        V[c] += pyr3;
    }
    for (int f = 0; f < n_internal; ++f) {
        int64_t c = neighbour[f];
        double d[3] = {cEst[3 * c] - Cf[3 * f], cEst[3 * c + 1] - Cf[3 * f + 1], cEst[3 * c + 2] - Cf[3 * f + 2]};
        double pyr3 = dot3(Sf + 3 * f, d);
        for (int k = 0; k < 3; ++k) C[3 * c + k] += pyr3 * ((3.0 / 4.0) * Cf[3 * f + k] + (1.0 / 4.0) * cEst[3 * c + k]);
        V[c] += pyr3;
    }
    for (int c = 0; c < n_cells; ++c) {
        if (fabs(V[c]) > 1.0e-300) {
            for (int k = 0; k < 3; ++k) C[3 * c + k] /= V[c];
        } else {
            for (int k = 0; k < 3; ++k) C[3 * c + k] = cEst[3 * c + k];
        }
        V[c] *= (1.0 / 3.0);
    }
    free(cEst);
    free(nf);
}

/* symmetric 3x3 (xx xy xz yy yz zz) inverse via the adjugate */
static void sym_inv(const double* a, double* r) {
    double xx = a[0], xy = a[1], xz = a[2], yy = a[3], yz = a[4], zz = a[5];
    double det = xx * yy * zz + xy * yz * xz + xz * xy * yz - xx * yz * yz - xy * xy * zz - xz * yy * xz;
    r[0] = (yy * zz - yz * yz) / det;
    r[1] = (xz * yz - xy * zz) / det;
    r[2] = (xy * yz - xz * yy) / det;
    r[3] = (xx * zz - xz * xz) / det;
    r[4] = (xy * xz - xx * yz) / det;
    r[5] = (xx * yy - xy * xy) / det;
}

static void sym_apply(const double* t, const double* d, double* out) {
    out[0] = t[0] * d[0] + t[1] * d[1] + t[2] * d[2];
    out[1] = t[1] * d[0] + t[3] * d[1] + t[4] * d[2];
    out[2] = t[2] * d[0] + t[4] * d[1] + t[5] * d[2];
}

/* Weighted least-squares vectors: zeroBoundaryVectors.C:90-221 with the
 * non-coupled boundary contributions (commented out at :159-165) restored,
 * i.e. the stock leastSquares scheme the cases use.  2-D/1-D meshes: the
 * field inverse drops directions whose diagonal is negligible, decided from
 * the first cell (OpenFOAM's inv(symmTensorField)). */
static void build_ls(oracle_state* s, int weighting) {
    int nC = s->nC;
    double* dd = (double*)calloc((size_t)6 * nC, sizeof(double));
    for (int f = 0; f < s->nIF; ++f) {
        int64_t o = s->own[f], n = s->nei[f];
        double d[3] = {s->C[3 * n] - s->C[3 * o], s->C[3 * n + 1] - s->C[3 * o + 1], s->C[3 * n + 2] - s->C[3 * o + 2]};
        double sq[6] = {d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]};
        double fo, fn;
        if (weighting == ORACLE_LS_MAGSF) {
            double c = s->magSf[f] / magsqr3(d);
            fo = (1 - s->w[f]) * c;
            fn = s->w[f] * c;
        } else if (weighting == ORACLE_LS_INVDIST) {
            fo = fn = 1.0 / magsqr3(d);
        } else {
            fo = fn = 1.0;
        }
        for (int k = 0; k < 6; ++k) {
            dd[6 * o + k] += fo * sq[k];
            dd[6 * n + k] += fn * sq[k];
        }
    }
    for (int b = 0; b < s->nBF; ++b) {
        int f = s->nIF + b;
        int64_t o = s->own[f];
        const double* S = s->Sf + 3 * f;
        double nrm[3] = {S[0] / s->magSf[f], S[1] / s->magSf[f], S[2] / s->magSf[f]};
        double cfc[3] = {s->Cf[3 * f] - s->C[3 * o], s->Cf[3 * f + 1] - s->C[3 * o + 1], s->Cf[3 * f + 2] - s->C[3 * o + 2]};
        double dn = dot3(nrm, cfc);
        double d[3] = {nrm[0] * dn, nrm[1] * dn, nrm[2] * dn}; /* fvPatch::delta() */
        double sq[6] = {d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]};
        double fb;
        if (weighting == ORACLE_LS_MAGSF) fb = s->magSf[f] / magsqr3(d);
        else if (weighting == ORACLE_LS_INVDIST) fb = 1.0 / magsqr3(d);
        else fb = 1.0;
        for (int k = 0; k < 6; ++k) dd[6 * o + k] += fb * sq[k];
        memcpy(s->lsB + 3 * b, d, sizeof d); /* temporarily keep delta */
    }
    /* inverse with component removal decided on cell 0 */
    int rm[3] = {0, 0, 0};
    if (nC > 0) {
        const double* t = dd;
        double scale = t[0] * t[0] + 2 * t[1] * t[1] + 2 * t[2] * t[2] + t[3] * t[3] + 2 * t[4] * t[4] + t[5] * t[5];
        rm[0] = (t[0] * t[0]) / scale < 1.0e-15;
        rm[1] = (t[3] * t[3]) / scale < 1.0e-15;
        rm[2] = (t[5] * t[5]) / scale < 1.0e-15;
    }
    double* inv = (double*)malloc(sizeof(double) * 6 * nC);
    for (int c = 0; c < nC; ++c) {
        double a[6];
        memcpy(a, dd + 6 * c, sizeof a);
        if (rm[0]) a[0] += 1.0;
        if (rm[1]) a[3] += 1.0;
        if (rm[2]) a[5] += 1.0;
        sym_inv(a, inv + 6 * c);
        if (rm[0]) inv[6 * c + 0] -= 1.0;
        if (rm[1]) inv[6 * c + 3] -= 1.0;
        if (rm[2]) inv[6 * c + 5] -= 1.0;
    }
    for (int f = 0; f < s->nIF; ++f) {
        int64_t o = s->own[f], n = s->nei[f];
        double d[3] = {s->C[3 * n] - s->C[3 * o], s->C[3 * n + 1] - s->C[3 * o + 1], s->C[3 * n + 2] - s->C[3 * o + 2]};
        double fo, fn;
        if (weighting == ORACLE_LS_MAGSF) {
            double c = s->magSf[f] / magsqr3(d);
            fo = (1 - s->w[f]) * c;
            fn = -s->w[f] * c;
        } else if (weighting == ORACLE_LS_INVDIST) {
            fo = 1.0 / magsqr3(d);
            fn = -1.0 / magsqr3(d);
        } else {
            fo = 1.0;
            fn = -1.0;
        }
        double a[3], b[3];
        sym_apply(inv + 6 * o, d, a);
        sym_apply(inv + 6 * n, d, b);
        for (int k = 0; k < 3; ++k) {
            s->lsP[3 * f + k] = fo * a[k];
            s->lsN[3 * f + k] = fn * b[k];
        }
    }
    for (int b = 0; b < s->nBF; ++b) {
        int f = s->nIF + b;
        int64_t o = s->own[f];
        double d[3];
        memcpy(d, s->lsB + 3 * b, sizeof d);
        double fb;
        if (weighting == ORACLE_LS_MAGSF) fb = s->magSf[f] * (1.0 / magsqr3(d));
        else if (weighting == ORACLE_LS_INVDIST) fb = 1.0 / magsqr3(d);
        else fb = 1.0;
        double a[3];
        sym_apply(inv + 6 * o, d, a);
        for (int k = 0; k < 3; ++k) s->lsB[3 * b + k] = fb * a[k];
    }
    free(dd);
    free(inv);
}

static double* dup(const double* src, size_t n) {
    double* d = (double*)malloc(sizeof(double) * (n ? n : 1));
    if (src) memcpy(d, src, sizeof(double) * n);
    else memset(d, 0, sizeof(double) * n);
    return d;
}

oracle_state* oracle_create(int D, int K_inner, double R, double omega, double Tref, double muRef, double Pr,
                            int n_cells, int n_internal, int n_boundary, const int64_t* owner,
                            const int64_t* neighbour, const double* C, const double* V, const double* Cf,
                            const double* Sf, int n_patches, const int* patch_type, const int* patch_start,
                            const double* rho_b, const double* U_b, const double* T_b, int n_dv,
                            const double* xi, const double* w, double xi_max, int ls_weighting, int n_threads) {
    oracle_state* s = (oracle_state*)calloc(1, sizeof(oracle_state));
    s->D = D;
    s->K = K_inner;
    s->R = R;
    s->omega = omega;
    s->Tref = Tref;
    s->muRef = muRef;
    s->Pr = Pr;
    s->nC = n_cells;
    s->nIF = n_internal;
    s->nBF = n_boundary;
    s->nP = n_patches;
    s->nthreads = n_threads > 0 ? n_threads : 1;
    int nF = n_internal + n_boundary;
    s->own = (int64_t*)malloc(sizeof(int64_t) * (nF ? nF : 1));
    memcpy(s->own, owner, sizeof(int64_t) * nF);
    s->nei = (int64_t*)malloc(sizeof(int64_t) * (n_internal ? n_internal : 1));
    memcpy(s->nei, neighbour, sizeof(int64_t) * n_internal);
    s->C = dup(C, 3 * (size_t)n_cells);
    s->V = dup(V, n_cells);
    s->Cf = dup(Cf, 3 * (size_t)nF);
    s->Sf = dup(Sf, 3 * (size_t)nF);
    s->magSf = dup(NULL, nF);
    for (int f = 0; f < nF; ++f) s->magSf[f] = sqrt(magsqr3(s->Sf + 3 * f));
    /* surfaceInterpolation weights and deltaCoeffs */
    s->w = dup(NULL, n_internal);
    s->dc = dup(NULL, n_internal);
    for (int f = 0; f < n_internal; ++f) {
        const double* S = s->Sf + 3 * f;
        const double *co = s->C + 3 * s->own[f], *cn = s->C + 3 * s->nei[f], *cf = s->Cf + 3 * f;
        double a[3] = {cf[0] - co[0], cf[1] - co[1], cf[2] - co[2]};
        double b[3] = {cn[0] - cf[0], cn[1] - cf[1], cn[2] - cf[2]};
        double SfdOwn = fabs(dot3(S, a)), SfdNei = fabs(dot3(S, b));
        s->w[f] = SfdNei / (SfdOwn + SfdNei);
        double d[3] = {cn[0] - co[0], cn[1] - co[1], cn[2] - co[2]};
        s->dc[f] = 1.0 / sqrt(magsqr3(d));
    }
    s->ptype = (int*)malloc(sizeof(int) * (n_patches ? n_patches : 1));
    memcpy(s->ptype, patch_type, sizeof(int) * n_patches);
    s->pstart = (int*)malloc(sizeof(int) * (n_patches + 1));
    memcpy(s->pstart, patch_start, sizeof(int) * (n_patches + 1));
    s->bf_patch = (int*)malloc(sizeof(int) * (n_boundary ? n_boundary : 1));
    s->bf_local = (int*)malloc(sizeof(int) * (n_boundary ? n_boundary : 1));
    for (int p = 0; p < n_patches; ++p)
        for (int b = patch_start[p]; b < patch_start[p + 1]; ++b) {
            s->bf_patch[b] = p;
            s->bf_local[b] = b - patch_start[p];
        }
    s->rho_b = dup(rho_b, n_boundary);
    s->U_b = dup(U_b, 3 * (size_t)n_boundary);
    s->T_b = dup(T_b, n_boundary);
    s->p_b = dup(NULL, n_boundary);
    s->inByRho = dup(NULL, n_boundary);
    s->outGoing = dup(NULL, n_boundary);
    s->nv = n_dv;
    s->xi = dup(xi, 3 * (size_t)n_dv);
    s->wv = dup(w, n_dv);
    s->xi_max = xi_max;
    s->lsP = dup(NULL, 3 * (size_t)n_internal);
    s->lsN = dup(NULL, 3 * (size_t)n_internal);
    s->lsB = dup(NULL, 3 * (size_t)n_boundary);
    build_ls(s, ls_weighting);
    size_t nvc = (size_t)n_dv * n_cells;
    s->gT = dup(NULL, nvc);
    s->hT = dup(NULL, nvc);
    s->gBP = dup(NULL, nvc);
    s->hBP = dup(NULL, nvc);
    s->gS = dup(NULL, (size_t)n_dv * n_internal);
    s->hS = dup(NULL, (size_t)n_dv * n_internal);
    s->gSb = dup(NULL, (size_t)n_dv * n_boundary);
    s->hSb = dup(NULL, (size_t)n_dv * n_boundary);
    s->rho = dup(NULL, n_cells);
    s->U = dup(NULL, 3 * (size_t)n_cells);
    s->T = dup(NULL, n_cells);
    s->q = dup(NULL, 3 * (size_t)n_cells);
    s->tau = dup(NULL, n_cells);
    s->rhoF = dup(NULL, nF);
    s->UF = dup(NULL, 3 * (size_t)nF);
    s->TF = dup(NULL, nF);
    s->qF = dup(NULL, 3 * (size_t)nF);
    s->tauF = dup(NULL, nF);
    return s;
}

void oracle_destroy(oracle_state* s) {
    if (!s) return;
    void* ptrs[] = {s->own, s->nei, s->C, s->V, s->Cf, s->Sf, s->magSf, s->w, s->dc, s->lsP, s->lsN, s->lsB,
                    s->ptype, s->pstart, s->bf_patch, s->bf_local, s->rho_b, s->U_b, s->T_b, s->inByRho,
                    s->outGoing, s->xi, s->wv, s->gT, s->hT, s->gBP, s->hBP, s->gS, s->hS, s->gSb, s->hSb,
                    s->rho, s->U, s->T, s->q, s->tau, s->rhoF, s->UF, s->TF, s->qF, s->tauF, s->p_b};
    for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; ++i) free(ptrs[i]);
    free(s);
}

/* discreteVelocity::equilibriumMaxwellByRho (discreteVelocity.C:1027-1039) */
static inline double eq_by_rho(const oracle_state* s, const double* xi, const double* U, double T) {
    double c[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
    return 1.0 / pow(sqrt(2.0 * M_PI * s->R * T), s->D) * exp(-magsqr3(c) / (2.0 * s->R * T));
}

/* fvDVM::updateTau (fvDVM.C:1823-1832) */
static inline double tau_of(const oracle_state* s, double T, double rho) {
    return s->muRef * exp(s->omega * log(T / s->Tref)) / rho / T / s->R;
}

void oracle_set_macro_flux(oracle_state* s, int mode) { s->macro_flux = mode == 2 ? 2 : (mode != 0); }

void oracle_set_patch_extra(oracle_state* s, int n_dv_1d, const double* p_b) {
    s->n1d = n_dv_1d;
    if (p_b) memcpy(s->p_b, p_b, sizeof(double) * s->nBF);
}

/* the DV a symmetry patch mirrors DV d into: round(|n . (symmX, symmY,
 * symmZ)(d)|) with n the unit normal of the patch's first face
 * (discreteVelocity.C:735-738, :762-764; target ids fvDVM.C:300-372) */
static int sym_target(const oracle_state* s, int patch, int d) {
    const int n = s->n1d, D = s->D;
    const int ix = d % n, iy = D >= 2 ? (d / n) % n : 0, iz = D == 3 ? d / (n * n) : 0;
    double tx, ty, tz;
    if (D == 3) {
        tx = iz * n * n + iy * n + (n - ix - 1);
        ty = iz * n * n + (n - iy - 1) * n + ix;
        tz = (n - iz - 1) * n * n + iy * n + ix;
    } else {
        tx = iy * n + (n - ix - 1);
        ty = (n - iy - 1) * n + ix;
        tz = 0;
    }
    const double* S = s->Sf + 3 * (s->nIF + s->pstart[patch]);
    const double m = sqrt(magsqr3(S));
    return (int)round(fabs(S[0] / m * tx + S[1] / m * ty + S[2] / m * tz));
}

void oracle_set_macros(oracle_state* s, const double* rho, const double* U, const double* T) {
    int D = s->D;
    double R = s->R;
    memcpy(s->rho, rho, sizeof(double) * s->nC);
    memcpy(s->U, U, sizeof(double) * 3 * s->nC);
    memcpy(s->T, T, sizeof(double) * s->nC);
    memset(s->q, 0, sizeof(double) * 3 * s->nC);
    /* initialiseDV (fvDVM.C:414-426) */
#pragma omp parallel for num_threads(s->nthreads)
    for (int i = 0; i < s->nv; ++i) {
        const double* xi = s->xi + 3 * i;
        for (int c = 0; c < s->nC; ++c) {
            double d[3] = {s->U[3 * c] - xi[0], s->U[3 * c + 1] - xi[1], s->U[3 * c + 2] - xi[2]};
            double cSqrByRT = magsqr3(d) / (R * s->T[c]);
            double gEq = s->rho[c] / pow(sqrt(2.0 * M_PI * R * s->T[c]), D) * exp(-cSqrByRT / 2.0);
            s->gT[(size_t)i * s->nC + c] = gEq;
            s->hT[(size_t)i * s->nC + c] = (s->K + 3.0 - D) * gEq * R * s->T[c];
        }
    }
    /* setCalculatedMaxwellRhoBC (fvDVM.C:578-624) */
    for (int b = 0; b < s->nBF; ++b) {
        if (s->ptype[s->bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
        const double* S = s->Sf + 3 * (s->nIF + b);
        double acc = 0;
        for (int i = 0; i < s->nv; ++i) {
            const double* xi = s->xi + 3 * i;
            double xs = dot3(xi, S);
            if (xs < 0) acc += -s->wv[i] * xs * eq_by_rho(s, xi, s->U_b + 3 * b, s->T_b[b]);
        }
        s->inByRho[b] = acc;
        s->outGoing[b] = 0.0;
    }
    /* mixed (rho fixedValue) patches: g/h = equilibriumMaxwell of the patch
     * rho, U, T for every DV (discreteVelocity::initBoundaryField,
     * discreteVelocity.C:226-258, :1010-1024); the incoming DVs keep it */
    for (int b = 0; b < s->nBF; ++b) {
        if (s->ptype[s->bf_patch[b]] != ORACLE_PATCH_MIXED) continue;
        const double Tb = s->T_b[b];
        for (int i = 0; i < s->nv; ++i) {
            const double* xi = s->xi + 3 * i;
            double d[3] = {s->U_b[3 * b] - xi[0], s->U_b[3 * b + 1] - xi[1], s->U_b[3 * b + 2] - xi[2]};
            size_t id = (size_t)i * s->nBF + b;
            s->gSb[id] = s->rho_b[b] / pow(sqrt(2.0 * M_PI * R * Tb), D) * exp(-magsqr3(d) / (2.0 * R * Tb));
            s->hSb[id] = (s->K + 3 - D) * R * Tb * s->gSb[id];
        }
    }
    for (int c = 0; c < s->nC; ++c) s->tau[c] = tau_of(s, s->T[c], s->rho[c]);
    /* Usurf = linear interpolate(Uvol) (fvDVM.C:2116), for the first CFL */
    for (int f = 0; f < s->nIF; ++f)
        for (int k = 0; k < 3; ++k) {
            double uo = s->U[3 * s->own[f] + k], un = s->U[3 * s->nei[f] + k];
            s->UF[3 * f + k] = s->w[f] * (uo - un) + un;
        }
    for (int b = 0; b < s->nBF; ++b)
        for (int k = 0; k < 3; ++k) s->UF[3 * (s->nIF + b) + k] = s->U_b[3 * b + k];
}

/* reconstruction at the half step from cell c: phi_c + grad_c . (Cf - C_c - xi dt/2)
 * (fvDVM.C:832-836) */
static inline double recon(double phi, const double* G, const double* Cf, const double* Cc, const double* xi,
                           double dt) {
    double v[3];
    for (int k = 0; k < 3; ++k) v[k] = Cf[k] - Cc[k] - 0.5 * xi[k] * dt;
    return phi + (G[0] * v[0] + G[1] * v[1] + G[2] * v[2]);
}

void oracle_evolve(oracle_state* s, double dt) {
    const int D = s->D, K = s->K, nC = s->nC, nIF = s->nIF, nBF = s->nBF, nv = s->nv;
    const double R = s->R, Pr = s->Pr;

    /* 1. updateGHbarPvol (fvDVM.C:648-683) */
#pragma omp parallel for schedule(dynamic) num_threads(s->nthreads)
    for (int dvi = 0; dvi < nv; ++dvi) {
        const double* xi = s->xi + 3 * dvi;
        for (int c = 0; c < nC; ++c) {
            const double *U = s->U + 3 * c, *q = s->q + 3 * c;
            double T = s->T[c], rho = s->rho[c];
            double relaxFactor = 1.5 * dt / (2.0 * s->tau[c] + dt);
            double um[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
            double cSqrByRT = magsqr3(um) / (R * T);
            double xu[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
            double cqBy5pRT = dot3(xu, q) / (5.0 * rho * R * T * R * T);
            double gEqBGK = rho / pow(sqrt(2.0 * M_PI * R * T), D) * exp(-cSqrByRT / 2.0);
            size_t id = (size_t)dvi * nC + c;
            s->gBP[id] = (1.0 - relaxFactor) * s->gT[id] +
                         relaxFactor * (1.0 + (1.0 - Pr) * cqBy5pRT * (cSqrByRT - D - 2.0)) * gEqBGK;
            s->hBP[id] = (1.0 - relaxFactor) * s->hT[id] +
                         relaxFactor *
                             ((K + 3.0 - D) + (1.0 - Pr) * cqBy5pRT * ((cSqrByRT - D) * (K + 3.0 - D) - 2 * K)) *
                             gEqBGK * R * T;
        }
    }

    /* 2-4. GHbarPvolComm (boundary value = owner value, the fixedGradient
     * patches keep a zero gradient: fvDVM.C:456-485, 775-809), updateGrad
     * (leastSquares, fvDVM.C:749-753) and updateGHbarSurf (fvDVM.C:755-1029).
     * The gradient of one DV is built and used before the next DV. */
#pragma omp parallel num_threads(s->nthreads)
    {
        double* Gg = (double*)malloc(sizeof(double) * 3 * (nC ? nC : 1));
        double* Gh = (double*)malloc(sizeof(double) * 3 * (nC ? nC : 1));
#pragma omp for schedule(dynamic)
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = s->xi + 3 * dvi;
            const double* g = s->gBP + (size_t)dvi * nC;
            const double* h = s->hBP + (size_t)dvi * nC;
            memset(Gg, 0, sizeof(double) * 3 * nC);
            memset(Gh, 0, sizeof(double) * 3 * nC);
            for (int f = 0; f < nIF; ++f) {
                int64_t o = s->own[f], n = s->nei[f];
                double dg = g[n] - g[o], dh = h[n] - h[o];
                for (int k = 0; k < 3; ++k) {
                    Gg[3 * o + k] += s->lsP[3 * f + k] * dg;
                    Gg[3 * n + k] -= s->lsN[3 * f + k] * dg;
                    Gh[3 * o + k] += s->lsP[3 * f + k] * dh;
                    Gh[3 * n + k] -= s->lsN[3 * f + k] * dh;
                }
            }
            for (int b = 0; b < nBF; ++b) {
                int64_t o = s->own[nIF + b];
                double dg = g[o] - g[o], dh = h[o] - h[o]; /* patch value equals cell value */
                for (int k = 0; k < 3; ++k) {
                    Gg[3 * o + k] += s->lsB[3 * b + k] * dg;
                    Gh[3 * o + k] += s->lsB[3 * b + k] * dh;
                }
            }
            double* gS = s->gS + (size_t)dvi * nIF;
            double* hS = s->hS + (size_t)dvi * nIF;
            for (int f = 0; f < nIF; ++f) {
                int64_t o = s->own[f], n = s->nei[f];
                const double* Cf = s->Cf + 3 * f;
                double xs = dot3(xi, s->Sf + 3 * f);
                if (xs >= VSMALL) {
                    gS[f] = recon(g[o], Gg + 3 * o, Cf, s->C + 3 * o, xi, dt);
                    hS[f] = recon(h[o], Gh + 3 * o, Cf, s->C + 3 * o, xi, dt);
                } else if (xs < -VSMALL) {
                    gS[f] = recon(g[n], Gg + 3 * n, Cf, s->C + 3 * n, xi, dt);
                    hS[f] = recon(h[n], Gh + 3 * n, Cf, s->C + 3 * n, xi, dt);
                } else {
                    /* 0.5*(phi_n + G_n.v_n + phi_o + G_o.v_o), left to right (fvDVM.C:849-862) */
                    double dn = recon(0.0, Gg + 3 * n, Cf, s->C + 3 * n, xi, dt);
                    double d_o = recon(0.0, Gg + 3 * o, Cf, s->C + 3 * o, xi, dt);
                    gS[f] = 0.5 * (((g[n] + dn) + g[o]) + d_o);
                    dn = recon(0.0, Gh + 3 * n, Cf, s->C + 3 * n, xi, dt);
                    d_o = recon(0.0, Gh + 3 * o, Cf, s->C + 3 * o, xi, dt);
                    hS[f] = 0.5 * (((h[n] + dn) + h[o]) + d_o);
                }
            }
            double* gSb = s->gSb + (size_t)dvi * nBF;
            double* hSb = s->hSb + (size_t)dvi * nBF;
            for (int b = 0; b < nBF; ++b) {
                int f = nIF + b;
                int64_t o = s->own[f];
                const double* S = s->Sf + 3 * f;
                double xs = dot3(xi, S);
                int type = s->ptype[s->bf_patch[b]];
                if (type == ORACLE_PATCH_ZERO_GRADIENT) {
                    /* gSurf == gBarPvol patchInternalField, every DV (fvDVM.C:887-891) */
                    gSb[b] = g[o];
                    hSb[b] = h[o];
                } else if (type == ORACLE_PATCH_MIXED) {
                    /* outgoing upwind; incoming keep the initial Maxwellian (fvDVM.C:892-909) */
                    if (xs > 0) {
                        gSb[b] = recon(g[o], Gg + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                        hSb[b] = recon(h[o], Gh + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                    }
                } else if (type == ORACLE_PATCH_SYMMETRY || type == ORACLE_PATCH_DVM_SYMMETRY) {
                    /* outgoing and tangential upwind; incoming from the mirror DV below
                     * (fvDVM.C:1009-1025) */
                    if (xs > -VSMALL) {
                        gSb[b] = recon(g[o], Gg + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                        hSb[b] = recon(h[o], Gh + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                    }
                } else if (type == ORACLE_PATCH_FAR_FIELD || type == ORACLE_PATCH_PRESSURE_IN ||
                           type == ORACLE_PATCH_PRESSURE_OUT) {
                    if (xs > 0) {
                        gSb[b] = recon(g[o], Gg + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                        hSb[b] = recon(h[o], Gh + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                    } else {
                        /* incoming: rho_b M(U_owner, T_b) (fvDVM.C:926-938) */
                        gSb[b] = s->rho_b[b] * eq_by_rho(s, xi, s->U + 3 * o, s->T_b[b]);
                        hSb[b] = gSb[b] * (R * s->T_b[b]) * (double)(K + 3 - D);
                    }
                } else if (type == ORACLE_PATCH_MAXWELL_WALL) {
                    if (xs > 0) {
                        gSb[b] = recon(g[o], Gg + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                        hSb[b] = recon(h[o], Gh + 3 * o, s->Cf + 3 * f, s->C + 3 * o, xi, dt);
                    }
                }
            }
        }
        free(Gg);
        free(Gh);
    }
    /* outGoing += w (xi.S) gbar_f for outgoing DVs, DV-ascending (fvDVM.C:959-960) */
    for (int b = 0; b < nBF; ++b) {
        if (s->ptype[s->bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
        const double* S = s->Sf + 3 * (nIF + b);
        for (int dvi = 0; dvi < nv; ++dvi) {
            double xs = dot3(s->xi + 3 * dvi, S);
            if (xs > 0) s->outGoing[b] += s->wv[dvi] * xs * s->gSb[(size_t)dvi * nBF + b];
        }
    }

    /* 5. updateMaxwellWallRho -> calculatedMaxwell::evaluate
     *    (calculatedMaxwellFvPatchField.C:140-164) */
    for (int b = 0; b < nBF; ++b) {
        if (s->ptype[s->bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
        s->rho_b[b] = s->outGoing[b] / fabs(s->inByRho[b]);
        s->outGoing[b] = 0.0;
    }

    /* 6. updateGHbarSurfMaxwellWallIn (fvDVM.C:1054-1098) */
#pragma omp parallel for schedule(dynamic) num_threads(s->nthreads)
    for (int dvi = 0; dvi < nv; ++dvi) {
        const double* xi = s->xi + 3 * dvi;
        for (int b = 0; b < nBF; ++b) {
            if (s->ptype[s->bf_patch[b]] != ORACLE_PATCH_MAXWELL_WALL) continue;
            if (dot3(xi, s->Sf + 3 * (nIF + b)) <= 0) {
                size_t id = (size_t)dvi * nBF + b;
                s->gSb[id] = s->rho_b[b] * eq_by_rho(s, xi, s->U_b + 3 * b, s->T_b[b]);
                s->hSb[id] = s->gSb[id] * (R * s->T_b[b]) * (double)(K + 3 - D);
            }
        }
    }

    /* 7. updateGHbarSurfSymmetryIn (fvDVM.C:1100-1179, discreteVelocity.C:691-773):
     *    incoming DVs (xi . S_first <= 0) take the mirror DV's face value, DVs
     *    in ascending order */
    for (int b = 0; b < nBF; ++b) {
        const int p = s->bf_patch[b], type = s->ptype[p];
        if (type != ORACLE_PATCH_SYMMETRY && type != ORACLE_PATCH_DVM_SYMMETRY) continue;
        const double* S0 = s->Sf + 3 * (nIF + s->pstart[p]);
        for (int dvi = 0; dvi < nv; ++dvi) {
            if (dot3(s->xi + 3 * dvi, S0) > 0) continue;
            const int t = sym_target(s, p, dvi);
            s->gSb[(size_t)dvi * nBF + b] = s->gSb[(size_t)t * nBF + b];
            s->hSb[(size_t)dvi * nBF + b] = s->hSb[(size_t)t * nBF + b];
        }
    }

    /* 8. updateMacroSurf (fvDVM.C:1181-1300): DV-ascending sums */
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
    for (int f = 0; f < nIF + nBF; ++f) {
        int internal = f < nIF;
        size_t stride = internal ? (size_t)nIF : (size_t)nBF;
        size_t col = internal ? (size_t)f : (size_t)(f - nIF);
        const double* gs = internal ? s->gS : s->gSb;
        const double* hs = internal ? s->hS : s->hSb;
        double rho = 0, rU[3] = {0, 0, 0}, rE = 0;
        for (int i = 0; i < nv; ++i) {
            const double* xi = s->xi + 3 * i;
            double g = gs[i * stride + col], h = hs[i * stride + col], w = s->wv[i];
            rho += w * g;
            for (int k = 0; k < 3; ++k) rU[k] += w * g * xi[k];
            rE += 0.5 * w * (g * magsqr3(xi) + h);
        }
        double U[3] = {rU[0] / rho, rU[1] / rho, rU[2] / rho};
        double T = (rE - 0.5 * rho * magsqr3(U)) / ((K + 3) / 2.0 * R * rho);
        double tau = tau_of(s, T, rho);
        double q[3] = {0, 0, 0};
        for (int i = 0; i < nv; ++i) {
            const double* xi = s->xi + 3 * i;
            double g = gs[i * stride + col], h = hs[i * stride + col], w = s->wv[i];
            double c[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
            double m = magsqr3(c) * g + h;
            for (int k = 0; k < 3; ++k) q[k] += 0.5 * w * c[k] * m;
        }
        double fac = 2.0 * tau / (2.0 * tau + 0.5 * dt * Pr);
        s->rhoF[f] = rho;
        s->TF[f] = T;
        s->tauF[f] = tau;
        for (int k = 0; k < 3; ++k) {
            s->UF[3 * f + k] = U[k];
            s->qF[3 * f + k] = fac * q[k];
        }
    }

    /* 9. updateGHsurf (fvDVM.C:1362-1457) */
#pragma omp parallel for schedule(dynamic) num_threads(s->nthreads)
    for (int dvi = 0; dvi < nv; ++dvi) {
        const double* xi = s->xi + 3 * dvi;
        double* gS = s->gS + (size_t)dvi * nIF;
        double* hS = s->hS + (size_t)dvi * nIF;
        for (int f = 0; f < nIF; ++f) {
            const double *U = s->UF + 3 * f, *q = s->qF + 3 * f;
            double T = s->TF[f], rho = s->rhoF[f];
            double relaxFactor = 0.5 * dt / (2.0 * s->tauF[f] + 0.5 * dt);
            double um[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
            double cSqrByRT = magsqr3(um) / (R * T);
            double xu[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
            double cqBy5pRT = dot3(xu, q) / (5.0 * rho * R * T * R * T);
            double gEqBGK = rho / pow(sqrt(2.0 * M_PI * R * T), D) * exp(-cSqrByRT / 2.0);
            gS[f] = (1.0 - relaxFactor) * gS[f] +
                    relaxFactor * (1.0 + (1.0 - Pr) * cqBy5pRT * (cSqrByRT - D - 2.0)) * gEqBGK;
            hS[f] = (1.0 - relaxFactor) * hS[f] +
                    relaxFactor *
                        ((K + 3.0 - D) + (1.0 - Pr) * cqBy5pRT * ((cSqrByRT - D) * (K + 3.0 - D) - 2 * K)) *
                        gEqBGK * R * T;
        }
        double* gSb = s->gSb + (size_t)dvi * nBF;
        double* hSb = s->hSb + (size_t)dvi * nBF;
        for (int b = 0; b < nBF; ++b) {
            int f = nIF + b;
            const int dvm_sym = s->ptype[s->bf_patch[b]] == ORACLE_PATCH_DVM_SYMMETRY;
            const int out = dot3(xi, s->Sf + 3 * f) > 0;
            if (!out && !dvm_sym) continue;
            const double *U = s->UF + 3 * f, *q = s->qF + 3 * f;
            double T = s->TF[f], rho = s->rhoF[f];
            double um[3] = {U[0] - xi[0], U[1] - xi[1], U[2] - xi[2]};
            double cSqrByRT = magsqr3(um) / (R * T);
            double xu[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
            double cqBy5pRT = dot3(xu, q) / (5.0 * rho * R * T * R * T);
            double gEqBGK = rho / pow(sqrt(2.0 * M_PI * R * T), D) * exp(-cSqrByRT / 2.0);
            double gEq = (1.0 + (1.0 - Pr) * cqBy5pRT * (cSqrByRT - D - 2.0)) * gEqBGK;
            /* hEq multiplies by the INTERNAL-face temperature at the patch-local
             * index (fvDVM.C:1367, :1413) */
            double Tint = s->TF[s->bf_local[b]];
            double hEq = ((K + 3.0 - D) + (1.0 - Pr) * cqBy5pRT * ((cSqrByRT - D) * (K + 3.0 - D) - 2 * K)) *
                         gEqBGK * R * Tint;
            double r = 0.5 * dt / (2.0 * s->tauF[f] + 0.5 * dt);
            if (out) {
                gSb[b] = (1.0 - r) * gSb[b] + r * gEq;
                hSb[b] = (1.0 - r) * hSb[b] + r * hEq;
            }
            if (dvm_sym) {
                /* DVMsymmetry: every DV relaxed (again), fvDVM.C:1445-1453 */
                gSb[b] = (1.0 - r) * gSb[b] + r * gEq;
                hSb[b] = (1.0 - r) * hSb[b] + r * hEq;
            }
        }
    }

    /* 10. updateGHtildeVol (fvDVM.C:1462-1519) */
#pragma omp parallel for schedule(dynamic) num_threads(s->nthreads)
    for (int dvi = 0; dvi < nv; ++dvi) {
        const double* xi = s->xi + 3 * dvi;
        double* g = s->gT + (size_t)dvi * nC;
        double* h = s->hT + (size_t)dvi * nC;
        const double* gb = s->gBP + (size_t)dvi * nC;
        const double* hb = s->hBP + (size_t)dvi * nC;
        for (int c = 0; c < nC; ++c) {
            g[c] = -1.0 / 3 * g[c] + 4.0 / 3 * gb[c];
            h[c] = -1.0 / 3 * h[c] + 4.0 / 3 * hb[c];
        }
        const double* gS = s->gS + (size_t)dvi * nIF;
        const double* hS = s->hS + (size_t)dvi * nIF;
        for (int f = 0; f < nIF; ++f) {
            int64_t o = s->own[f], n = s->nei[f];
            double xs = dot3(xi, s->Sf + 3 * f);
            g[o] -= (xs * gS[f] * dt / s->V[o]);
            g[n] += (xs * gS[f] * dt / s->V[n]);
            h[o] -= (xs * hS[f] * dt / s->V[o]);
            h[n] += (xs * hS[f] * dt / s->V[n]);
        }
        const double* gSb = s->gSb + (size_t)dvi * nBF;
        const double* hSb = s->hSb + (size_t)dvi * nBF;
        for (int b = 0; b < nBF; ++b) {
            int64_t o = s->own[nIF + b];
            double xs = dot3(xi, s->Sf + 3 * (nIF + b));
            g[o] -= xs * gSb[b] * dt / s->V[o];
            h[o] -= xs * hSb[b] * dt / s->V[o];
        }
    }

    /* 11a. updateMacroVol, macroFlux yes (fvDVM.C:1523-1526, :1613-1679): the
     *      old rho, rho U, rho E advance by the face fluxes of this step's face
     *      macros, internal faces in order, then the boundary faces.  The face
     *      stress stays zero (its sum is commented out, fvDVM.C:1270, :1305).
     *      The boundary momentum flux takes Sf of the INTERNAL face at the
     *      patch-local index (fvDVM.C:1668-1669, Sf is the internal field).
     *      "X & Sf*dt/V" is X & ((Sf dt)/V) by C++ precedence. */
    double *mrho = NULL, *mrU = NULL, *mrE = NULL;
    if (s->macro_flux == 2) {
        /* 11b. the unstructured-velocity-mesh branch (fvDVM.C:1562-1611):
         *      fluxes from the relaxed face DFs of every DV, DVs in order,
         *      internal faces then boundary faces; dXiCellSize = 1 (:1934-1939) */
        double* fr = dup(NULL, nC);
        double* fU = dup(NULL, 3 * (size_t)nC);
        double* fE = dup(NULL, nC);
        for (int dvi = 0; dvi < nv; ++dvi) {
            const double* xi = s->xi + 3 * dvi;
            const double w = 1.0 * s->wv[dvi], xi2 = magsqr3(xi);
            for (int f = 0; f < nIF + nBF; ++f) {
                const int internal = f < nIF;
                const double g = internal ? s->gS[(size_t)dvi * nIF + f] : s->gSb[(size_t)dvi * nBF + f - nIF];
                const double h = internal ? s->hS[(size_t)dvi * nIF + f] : s->hSb[(size_t)dvi * nBF + f - nIF];
                const double rf = w * g, ef = 0.5 * 1.0 * s->wv[dvi] * (g * xi2 + h);
                const double xs = dot3(xi, s->Sf + 3 * f);
                for (int side = 0; side < (internal ? 2 : 1); ++side) {
                    const int64_t c = side == 0 ? s->own[f] : s->nei[f];
                    const double V = s->V[c];
                    const double dr = xs * rf * dt / V, dE = xs * ef * dt / V;
                    double dU[3];
                    for (int k = 0; k < 3; ++k) dU[k] = xs * (rf * xi[k]) * dt / V;
                    if (side == 0) {
                        fr[c] -= dr;
                        for (int k = 0; k < 3; ++k) fU[3 * c + k] -= dU[k];
                        fE[c] -= dE;
                    } else {
                        fr[c] += dr;
                        for (int k = 0; k < 3; ++k) fU[3 * c + k] += dU[k];
                        fE[c] += dE;
                    }
                }
            }
        }
        mrho = dup(NULL, nC);
        mrU = dup(NULL, 3 * (size_t)nC);
        mrE = dup(NULL, nC);
        for (int c = 0; c < nC; ++c) {
            const double* U = s->U + 3 * c;
            mrho[c] = s->rho[c] + fr[c];
            for (int k = 0; k < 3; ++k) mrU[3 * c + k] = s->rho[c] * U[k] + fU[3 * c + k];
            mrE[c] = s->rho[c] * (0.5 * magsqr3(U) + (K + 3) / 2.0 * R * s->T[c]) + fE[c];
        }
        free(fr);
        free(fU);
        free(fE);
    } else if (s->macro_flux) {
        mrho = dup(NULL, nC);
        mrU = dup(NULL, 3 * (size_t)nC);
        mrE = dup(NULL, nC);
        for (int c = 0; c < nC; ++c) {
            const double* U = s->U + 3 * c;
            mrho[c] = s->rho[c];
            for (int k = 0; k < 3; ++k) mrU[3 * c + k] = s->rho[c] * U[k];
            mrE[c] = s->rho[c] * (0.5 * magsqr3(U) + (K + 3) / 2.0 * R * s->T[c]);
        }
        for (int f = 0; f < nIF + nBF; ++f) {
            const int internal = f < nIF;
            const int64_t o = s->own[f];
            const double *Uf = s->UF + 3 * f, *qf = s->qF + 3 * f, *S = s->Sf + 3 * f;
            const double rf = s->rhoF[f];
            const double rUf[3] = {rf * Uf[0], rf * Uf[1], rf * Uf[2]};
            const double rEf = rf * (magsqr3(Uf) + (K + 3) / 2.0 * R * s->TF[f]);
            const double ev[3] = {rEf * Uf[0] + qf[0], rEf * Uf[1] + qf[1], rEf * Uf[2] + qf[2]};
            /* momentum: (rho_f U_f U_f + 0) & Sm */
            const double* Sm = internal ? S : s->Sf + 3 * s->bf_local[f - nIF];
            for (int side = 0; side < (internal ? 2 : 1); ++side) {
                const int64_t c = side == 0 ? o : s->nei[f];
                const double V = s->V[c], sgn = side == 0 ? -1.0 : 1.0;
                const double Sd[3] = {S[0] * dt / V, S[1] * dt / V, S[2] * dt / V};
                const double Smd[3] = {Sm[0] * dt / V, Sm[1] * dt / V, Sm[2] * dt / V};
                double mU[3];
                for (int i = 0; i < 3; ++i)
                    mU[i] = (rUf[i] * Uf[0] + 0.0) * Smd[0] + (rUf[i] * Uf[1] + 0.0) * Smd[1] +
                            (rUf[i] * Uf[2] + 0.0) * Smd[2];
                const double mr = dot3(rUf, S) * dt / V;
                const double mE = dot3(ev, Sd);
                if (sgn < 0) {
                    mrho[c] -= mr;
                    for (int i = 0; i < 3; ++i) mrU[3 * c + i] -= mU[i];
                    mrE[c] -= mE;
                } else {
                    mrho[c] += mr;
                    for (int i = 0; i < 3; ++i) mrU[3 * c + i] += mU[i];
                    mrE[c] += mE;
                }
            }
        }
    }

    /* 11. updateMacroVol (fvDVM.C:1521-1554 macroFlux no, 1683-1742) */
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
    for (int c = 0; c < nC; ++c) {
        double rho = 0, rU[3] = {0, 0, 0}, rE = 0;
        if (s->macro_flux) {
            rho = mrho[c];
            for (int k = 0; k < 3; ++k) rU[k] = mrU[3 * c + k];
            rE = mrE[c];
        } else {
            for (int i = 0; i < nv; ++i) {
                const double* xi = s->xi + 3 * i;
                double g = s->gT[(size_t)i * nC + c], h = s->hT[(size_t)i * nC + c];
                double w = 1.0 * s->wv[i];
                rho += w * g;
                for (int k = 0; k < 3; ++k) rU[k] += w * g * xi[k];
                rE += 0.5 * 1.0 * s->wv[i] * (magsqr3(xi) * g + h);
            }
        }
        double U[3] = {rU[0] / rho, rU[1] / rho, rU[2] / rho};
        double T = (rE - 0.5 * rho * magsqr3(U)) / ((K + 3) / 2.0 * R * rho);
        double tau = tau_of(s, T, rho);
        double q[3] = {0, 0, 0};
        for (int i = 0; i < nv; ++i) {
            const double* xi = s->xi + 3 * i;
            double g = s->gT[(size_t)i * nC + c], h = s->hT[(size_t)i * nC + c];
            double cc[3] = {xi[0] - U[0], xi[1] - U[1], xi[2] - U[2]};
            double m = magsqr3(cc) * g + h;
            for (int k = 0; k < 3; ++k) q[k] += 0.5 * s->wv[i] * cc[k] * m;
        }
        double fac = 2.0 * tau / (2.0 * tau + dt * Pr);
        s->rho[c] = rho;
        s->T[c] = T;
        s->tau[c] = tau;
        for (int k = 0; k < 3; ++k) {
            s->U[3 * c + k] = U[k];
            s->q[3 * c + k] = fac * q[k];
        }
    }

    free(mrho);
    free(mrU);
    free(mrE);

    /* 12. updatePressureInOutBC (fvDVM.C:1745-1821): the pressureIn rho and
     *     the pressureOut rho and T patch values from the owner cell (the
     *     next step's far-field incoming DFs read them); U patch values by
     *     the characteristics, kept for output */
    for (int b = 0; b < nBF; ++b) {
        const int type = s->ptype[s->bf_patch[b]];
        if (type != ORACLE_PATCH_PRESSURE_IN && type != ORACLE_PATCH_PRESSURE_OUT) continue;
        const int64_t o = s->own[nIF + b];
        const double* Sf = s->Sf + 3 * (nIF + b);
        const double magSf = s->magSf[nIF + b];
        const double* Ui = s->U + 3 * o;
        const double Ti = s->T[o], rhoi = s->rho[o], p = s->p_b[b];
        const double ai = sqrt(R * Ti * (K + 5) / (K + 3));
        double n[3] = {Sf[0] / magSf, Sf[1] / magSf, Sf[2] / magSf};
        const double Un = dot3(Ui, n);
        double UnIn;
        if (type == ORACLE_PATCH_PRESSURE_IN) {
            s->rho_b[b] = p / R / s->T_b[b];
            UnIn = Un + (p - rhoi * R * Ti) / rhoi / ai;
        } else {
            s->rho_b[b] = rhoi + (p - rhoi * R * Ti) / ai / ai;
            s->T_b[b] = p / (R * rhoi);
            UnIn = Un + (rhoi * R * Ti - p) / rhoi / ai;
        }
        for (int k = 0; k < 3; ++k) s->U_b[3 * b + k] = UnIn * n[k] + (Ui[k] - Un * n[k]);
    }
}

void oracle_co_num(oracle_state* s, double dt, double* co_max, double* co_mean) {
    double mx = -1e300, sum = 0;
    double sq = sqrt((double)s->D);
    for (int f = 0; f < s->nIF; ++f) {
        double u = s->dc[f] * (sqrt(magsqr3(s->UF + 3 * f)) + sq * s->xi_max);
        if (u > mx) mx = u;
        sum += u;
    }
    *co_max = mx * dt;
    *co_mean = s->nIF ? sum / s->nIF * dt : 0.0;
}

void oracle_get_macros(oracle_state* s, double* rho, double* U, double* T, double* q, double* tau) {
    if (rho) memcpy(rho, s->rho, sizeof(double) * s->nC);
    if (U) memcpy(U, s->U, sizeof(double) * 3 * s->nC);
    if (T) memcpy(T, s->T, sizeof(double) * s->nC);
    if (q) memcpy(q, s->q, sizeof(double) * 3 * s->nC);
    if (tau) memcpy(tau, s->tau, sizeof(double) * s->nC);
}

void oracle_get_face_macros(oracle_state* s, double* rho, double* U, double* T, double* q, double* tau) {
    int nF = s->nIF + s->nBF;
    if (rho) memcpy(rho, s->rhoF, sizeof(double) * nF);
    if (U) memcpy(U, s->UF, sizeof(double) * 3 * nF);
    if (T) memcpy(T, s->TF, sizeof(double) * nF);
    if (q) memcpy(q, s->qF, sizeof(double) * 3 * nF);
    if (tau) memcpy(tau, s->tauF, sizeof(double) * nF);
}

void oracle_get_wall(oracle_state* s, double* rho_w, double* in_by_rho) {
    if (rho_w) memcpy(rho_w, s->rho_b, sizeof(double) * s->nBF);
    if (in_by_rho) memcpy(in_by_rho, s->inByRho, sizeof(double) * s->nBF);
}

void oracle_get_state(oracle_state* s, double* g, double* h) {
    size_t n = (size_t)s->nv * s->nC;
    if (g) memcpy(g, s->gT, sizeof(double) * n);
    if (h) memcpy(h, s->hT, sizeof(double) * n);
}

void oracle_set_state(oracle_state* s, const double* g, const double* h) {
    size_t n = (size_t)s->nv * s->nC;
    memcpy(s->gT, g, sizeof(double) * n);
    memcpy(s->hT, h, sizeof(double) * n);
}

void oracle_get_ghbar(oracle_state* s, double* g, double* h) {
    size_t n = (size_t)s->nv * s->nC;
    if (g) memcpy(g, s->gBP, sizeof(double) * n);
    if (h) memcpy(h, s->hBP, sizeof(double) * n);
}

void oracle_get_face_values(oracle_state* s, double* g_int, double* h_int, double* g_b, double* h_b) {
    if (g_int) memcpy(g_int, s->gS, sizeof(double) * (size_t)s->nv * s->nIF);
    if (h_int) memcpy(h_int, s->hS, sizeof(double) * (size_t)s->nv * s->nIF);
    if (g_b) memcpy(g_b, s->gSb, sizeof(double) * (size_t)s->nv * s->nBF);
    if (h_b) memcpy(h_b, s->hSb, sizeof(double) * (size_t)s->nv * s->nBF);
}

void oracle_get_ls(oracle_state* s, double* p, double* n, double* b) {
    if (p) memcpy(p, s->lsP, sizeof(double) * 3 * s->nIF);
    if (n) memcpy(n, s->lsN, sizeof(double) * 3 * s->nIF);
    if (b) memcpy(b, s->lsB, sizeof(double) * 3 * s->nBF);
}

void oracle_get_weights(oracle_state* s, double* w, double* dc) {
    if (w) memcpy(w, s->w, sizeof(double) * s->nIF);
    if (dc) memcpy(dc, s->dc, sizeof(double) * s->nIF);
}

/*
 * Layout of the CPU oracle's state, shared by the oracle (dugks_oracle.c)
 * and its tangent-linear restatement (dugks_tangent.cpp).  TEST
 * INFRASTRUCTURE ONLY, like the oracle itself.
 */
#ifndef DUGKS_ORACLE_STATE_H
#define DUGKS_ORACLE_STATE_H

#include <stdint.h>

struct oracle_state {
    int D, K;
    double R, omega, Tref, muRef, Pr;
    int nC, nIF, nBF, nP, nthreads;
    int64_t *own, *nei;
    double *C, *V, *Cf, *Sf, *magSf, *w, *dc;
    double *lsP, *lsN, *lsB;
    int *ptype, *pstart, *bf_patch, *bf_local;
    double *rho_b, *U_b, *T_b;      /* rho patch values (farField keeps them), U/T patch values */
    double *p_b;                    /* pressureIn / pressureOut values */
    int n1d;                        /* DV nodes per dimension (symmetry targets) */
    int macro_flux;                 /* fvDVMparas macroFlux yes */
    double *inByRho, *outGoing;     /* calculatedMaxwell patch members */
    int nv;
    double *xi, *wv, xi_max;
    /* state (DV-major, as fvDVM.C:403-408) */
    double *gT, *hT, *gBP, *hBP, *gS, *hS, *gSb, *hSb;
    /* cell macros */
    double *rho, *U, *T, *q, *tau;
    /* face macros, internal then boundary */
    double *rhoF, *UF, *TF, *qF, *tauF;
};

#endif

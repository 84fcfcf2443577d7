// Device helpers shared by the DUGKS kernels: equilibria, raw moments,
// record loads.
#pragma once

#include "dugks_kernels.cuh"

namespace dugks {

struct Consts {
    double dt, Pr1, K3D, Kin, R, omega, Tref, muRef, Pr;
    int D;
};

// this step's time step (device-resident when adaptive)
__device__ __forceinline__ double step_dt(const StepArgs& a) { return a.dtp ? *a.dtp : a.dt; }

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

// xi . S exactly as the reference evaluates it ((x*Sx + y*Sy) + z*Sz, no
// fused multiply-add): the upwind switch and the in/out tests branch on its
// sign, and on faces where xi is (numerically) tangential the sign is set by
// rounding, so it must round like the reference's x86 build.
__device__ __forceinline__ double xi_dot_s(const double* xi, const double* S) {
    return __dadd_rn(__dadd_rn(__dmul_rn(xi[0], S[0]), __dmul_rn(xi[1], S[1])), __dmul_rn(xi[2], S[2]));
}

// Coefficient record of a Shakhov equilibrium in the working precision.
template <typename Real>
struct Rec {
    Real U[3], invRT, A, r, qv[3], RTh;
};

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

// The same pair from a precomputed Maxwellian value E = A e^{-cs/2}: the
// D-dimensional Maxwellian of a tensor-product DV set is the product of
// D one-dimensional factors A e_x(xi_x) e_y(xi_y) e_z(xi_z), tabulated per
// cell and per face by the combine kernels.
template <int D, typename Real>
__device__ __forceinline__ void shakhov_m(const Real xi[3], const Rec<Real>& r, Real E, Real K3D, Real Kin, Real& gS,
                                          Real& hS) {
    const Real cx = xi[0] - r.U[0], cy = xi[1] - r.U[1];
    const Real cz = D == 3 ? xi[2] - r.U[2] : Real(0);
    const Real cs = (cx * cx + cy * cy + cz * cz) * r.invRT;
    const Real s = cx * r.qv[0] + cy * r.qv[1] + (D == 3 ? cz * r.qv[2] : Real(0));
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

}  // namespace dugks

// DUGKS step kernels for sm_100a: combine, initialisation and bookkeeping
// kernels, and the stage sequence of one step.
//
// One fvDVM::evolution() (src/fvDVM/fvDVM/fvDVM.C:2128-2174) is
//   pass A  (dugks_passes.cu)  reconstruction and raw face moments
//   face combine (internal, then boundary faces)  face macros rho,U,T,q,tau,
//           wall density, face relaxation coefficients, Courant number
//   pass B  (dugks_passes.cu)  relaxation, flux, g~/h~ update, cell moments
//   cell combine  cell macros and the next step's cell coefficients
// The state g~, h~ is DV-major [dv][cell] (cells renumbered along a Morton
// curve), double-buffered between steps.
#include <algorithm>

#include "dugks_device.cuh"

namespace dugks {

namespace {

// ---------------------------------------------------------------------
// Face combine: sums the DV-chunk partials of a face, adds the incoming
// wall DFs through rho_w, and forms the face macros and the face
// relaxation coefficients (updateMaxwellWallRho fvDVM.C:1032-1052,
// calculatedMaxwellFvPatchField.C:140-164, updateMacroSurf :1248-1300).
// ---------------------------------------------------------------------
__device__ __forceinline__ void sum_face_partials(const StepArgs& a, int f, double* s) {
    const DevMesh& m = a.dm;
    for (int j = 0; j < 15; ++j) s[j] = 0.0;
    const int i0 = chk(__ldg(m.face_items + 2 * f), 0, m.n_items, a.ds.err);
    const int i1 = chk(__ldg(m.face_items + 2 * f + 1), -1, m.n_items, a.ds.err);
    for (int ch = 0; ch < a.chunks; ++ch) {
        const double* p0 = a.ds.partF + (static_cast<size_t>(ch) * m.n_items + i0) * kNM;
        for (int j = 0; j < 15; ++j) s[j] += p0[j];
        if (i1 >= 0) {
            const double* p1 = a.ds.partF + (static_cast<size_t>(ch) * m.n_items + i1) * kNM;
            for (int j = 0; j < 15; ++j) s[j] += p1[j];
        }
    }
}

// one-dimensional Maxwellian factors of one cell or face (layout in
// dugks_internal.h): D * n1d exponentials instead of one per DV
__device__ __forceinline__ void write_maxwell_tables(const DevMesh& m, double* tab, size_t n, int e, const double U[3],
                                                     double invRT, double A) {
    for (int k = 0; k < m.D; ++k)
        for (int i = 0; i < m.n1d; ++i) {
            const double x = __ldg(m.X1 + i) - U[k];
            double v = exp(-0.5 * x * x * invRT);
            if (k == 0) v *= A;
            const size_t idx = (static_cast<size_t>(k) * m.n1d + i) * n + e;
            tab[idx] = v;
        }
}

__device__ __forceinline__ void write_face(const StepArgs& a, const Consts& k, int f, const double* s, double T_h,
                                           bool use_T_h) {
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
    const double qs = k.Pr1 / (5.0 * rho * RT * RT);
    const size_t n = static_cast<size_t>(a.dm.n_items);
    double* fr = a.ds.facerec;
    for (int side = 0; side < 2; ++side) {
        const int it = chk(__ldg(a.dm.face_items + 2 * f + side), -1, a.dm.n_items, a.ds.err);
        if (it < 0) continue;
        fr[REC_UX * n + it] = U[0];
        fr[REC_UY * n + it] = U[1];
        fr[REC_UZ * n + it] = U[2];
        fr[REC_INVRT * n + it] = 1.0 / RT;
        fr[REC_A * n + it] = rho * inv_norm(RT, k.D);
        fr[REC_R * n + it] = 0.5 * k.dt / (2.0 * tau + 0.5 * k.dt);
        fr[REC_QX * n + it] = q[0] * qs;
        fr[REC_QY * n + it] = q[1] * qs;
        fr[REC_QZ * n + it] = q[2] * qs;
        fr[REC_RTH * n + it] = use_T_h ? k.R * T_h : RT;
        write_maxwell_tables(a.dm, a.ds.ftab, n, it, U, 1.0 / RT, rho * inv_norm(RT, k.D));
    }
}

__global__ void k_face_combine_internal(const StepArgs a, Consts k) {
    k.dt = step_dt(a);
    const DevMesh& m = a.dm;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    double co = 0.0;
    if (f < m.nIF) {
        double s[15];
        sum_face_partials(a, f, s);
        write_face(a, k, f, s, 0.0, false);
        const double* fm = a.ds.fm + static_cast<size_t>(f) * 9;
        const double umag = sqrt(fm[1] * fm[1] + fm[2] * fm[2] + fm[3] * fm[3]);
        co = __ldg(m.dc + f) * (umag + m.xi_max_co);  // getCoNum, fvDVM.C:2180-2182
    }
    // block max and sum of the Courant numbers (per unit dt)
    __shared__ double smax[32], ssum[32];
    double vmax = co, vsum = co;
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
            // non-negative doubles order like their bit patterns
            atomicMax(reinterpret_cast<unsigned long long*>(a.ds.co),
                      static_cast<unsigned long long>(__double_as_longlong(vmax)));
            atomicAdd(a.ds.co + 1, vsum);
        }
    }
}

__global__ void k_face_combine_boundary(const StepArgs a, Consts k) {
    k.dt = step_dt(a);
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
    const double qs = k.Pr1 / (5.0 * rho * RT * RT);
    const size_t n = static_cast<size_t>(a.dm.nC);
    double* cr = a.ds.cellrec;
    cr[REC_UX * n + c] = U[0];
    cr[REC_UY * n + c] = U[1];
    cr[REC_UZ * n + c] = U[2];
    cr[REC_INVRT * n + c] = 1.0 / RT;
    cr[REC_A * n + c] = rho * inv_norm(RT, k.D);
    cr[REC_R * n + c] = dt_next > 0 ? 1.5 * dt_next / (2.0 * tau + dt_next) : 0.0;  // relax factor, fvDVM.C:668
    cr[REC_QX * n + c] = q[0] * qs;
    cr[REC_QY * n + c] = q[1] * qs;
    cr[REC_QZ * n + c] = q[2] * qs;
    cr[REC_RTH * n + c] = RT;
    write_maxwell_tables(a.dm, a.ds.ctab, n, c, U, 1.0 / RT, rho * inv_norm(RT, k.D));
}

// macroFlux yes (fvDVM.C:1523-1526, :1613-1679): the cell's old rho, rho U,
// rho E advanced by this step's face macro fluxes, faces in face order.  The
// face stress is zero (its sum is commented out, fvDVM.C:1270, :1305); the
// boundary momentum flux takes Sf of the internal face at the patch-local
// index (fvDVM.C:1668-1669); "X & Sf*dt/V" is X & ((Sf dt)/V).
__device__ __forceinline__ void macro_flux_update(const StepArgs& a, const Consts& k, int c, double& rho, double rU[3],
                                                  double& rE) {
    const DevMesh& m = a.dm;
    const double* cm = a.ds.cm + static_cast<size_t>(c) * 9;
    const double U0[3] = {cm[1], cm[2], cm[3]};
    rho = cm[0];
    for (int i = 0; i < 3; ++i) rU[i] = rho * U0[i];
    rE = rho * (0.5 * (U0[0] * U0[0] + U0[1] * U0[1] + U0[2] * U0[2]) + (k.Kin + 3) / 2.0 * k.R * cm[4]);
    const double V = __ldg(m.mf_V + c), dt = k.dt;
    for (int e = __ldg(m.mf_off + c); e < __ldg(m.mf_off + c + 1); ++e) {
        const int code = __ldg(m.mf_ent + e), f = chk(code >> 1, 0, m.nIF + m.nBF, a.ds.err);
        const bool add = code & 1;
        const double* fm = a.ds.fm + static_cast<size_t>(f) * 9;
        const double rf = fm[0], Uf[3] = {fm[1], fm[2], fm[3]}, qf[3] = {fm[5], fm[6], fm[7]};
        const double* S = m.mf_Sf + 3 * static_cast<size_t>(f);
        const double* Sm = f < m.nIF ? S
                                     : m.mf_Sf + 3 * static_cast<size_t>(chk(__ldg(m.bface_patch_local + f - m.nIF), 0,
                                                                             m.nIF + m.nBF, a.ds.err));
        const double rUf[3] = {__dmul_rn(rf, Uf[0]), __dmul_rn(rf, Uf[1]), __dmul_rn(rf, Uf[2])};
        const double rEf = __dmul_rn(rf, __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(Uf[0], Uf[0]), __dmul_rn(Uf[1], Uf[1])),
                                                             __dmul_rn(Uf[2], Uf[2])),
                                                   __dmul_rn(__dmul_rn((k.Kin + 3) / 2.0, k.R), fm[4])));
        double ev[3], Sd[3], Smd[3];
        for (int i = 0; i < 3; ++i) {
            ev[i] = __dadd_rn(__dmul_rn(rEf, Uf[i]), qf[i]);
            Sd[i] = __ddiv_rn(__dmul_rn(__ldg(S + i), dt), V);
            Smd[i] = __ddiv_rn(__dmul_rn(__ldg(Sm + i), dt), V);
        }
        const double mr = __ddiv_rn(__dmul_rn(xi_dot_s(rUf, S), dt), V);
        const double mE = xi_dot_s(ev, Sd);
        double mU[3];
        for (int i = 0; i < 3; ++i) {
            const double t[3] = {__dmul_rn(rUf[i], Uf[0]), __dmul_rn(rUf[i], Uf[1]), __dmul_rn(rUf[i], Uf[2])};
            mU[i] = xi_dot_s(t, Smd);
        }
        if (add) {
            rho += mr;
            for (int i = 0; i < 3; ++i) rU[i] += mU[i];
            rE += mE;
        } else {
            rho -= mr;
            for (int i = 0; i < 3; ++i) rU[i] -= mU[i];
            rE -= mE;
        }
    }
}

__global__ void k_cell_combine(const StepArgs a, Consts k, double dt_next) {
    k.dt = step_dt(a);
    if (a.dtnp) dt_next = *a.dtnp;
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
    if (!m.macro_flux) {
        macros_from_moments(s, k, rho, U, T, q, tau);
    } else {
        // rho, U, T from the fluxes; q from the DF moments about that U:
        // q = 1/2 [V3 - 2 M2.U + |U|^2 M1 - U W + 2 U (M1.U) - U |U|^2 M0]
        double rU[3], rE;
        if (!m.general_dv) {
            macro_flux_update(a, k, c, rho, rU, rE);
        } else {
            // the velocity-mesh branch (fvDVM.C:1562-1611): the old rho, rho U,
            // rho E plus the moments of the update's flux term (pass B)
            const double* cm = a.ds.cm + static_cast<size_t>(c) * 9;
            double f[5] = {0, 0, 0, 0, 0};
            for (int ch = 0; ch < a.chunks; ++ch) {
                const double* p = a.ds.partX + (static_cast<size_t>(ch) * m.nC + c) * kFX;
                for (int j = 0; j < 5; ++j) f[j] += p[j];
            }
            const double U0[3] = {cm[1], cm[2], cm[3]};
            rho = cm[0] + f[0];
            for (int i = 0; i < 3; ++i) rU[i] = cm[0] * U0[i] + f[1 + i];
            rE = cm[0] * (0.5 * (U0[0] * U0[0] + U0[1] * U0[1] + U0[2] * U0[2]) + (k.Kin + 3) / 2.0 * k.R * cm[4]) +
                 f[4];
        }
        for (int i = 0; i < 3; ++i) U[i] = rU[i] / rho;
        const double u2 = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
        T = (rE - 0.5 * rho * u2) / ((k.Kin + 3.0) / 2.0 * k.R * rho);
        tau = k.muRef * exp(k.omega * log(T / k.Tref)) / rho / T / k.R;
        const double* M2 = s + MOM_M2;
        const double M2U[3] = {M2[0] * U[0] + M2[1] * U[1] + M2[2] * U[2], M2[1] * U[0] + M2[3] * U[1] + M2[4] * U[2],
                               M2[2] * U[0] + M2[4] * U[1] + M2[5] * U[2]};
        const double M1U = s[MOM_M1] * U[0] + s[MOM_M1 + 1] * U[1] + s[MOM_M1 + 2] * U[2];
        for (int i = 0; i < 3; ++i)
            q[i] = 0.5 * (s[MOM_V3 + i] - 2.0 * M2U[i] + u2 * s[MOM_M1 + i] - U[i] * s[MOM_W] + 2.0 * U[i] * M1U -
                          U[i] * u2 * s[MOM_M0]);
    }
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

// cell records and Maxwellian tables from the cell macros in cm (a restored
// step record); the relax factor is left to k_cell_prep
__global__ void k_cell_records(const StepArgs a, Consts k) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.dm.nC) return;
    const double* cm = a.ds.cm + static_cast<size_t>(c) * 9;
    const double U[3] = {cm[1], cm[2], cm[3]}, q[3] = {cm[5], cm[6], cm[7]};
    write_cellrec(a, k, c, cm[0], U, cm[4], q, cm[8], 0.0);
}

// Maxwellian tables of every cell from its record (after the host wrote
// the records at initialisation)
__global__ void k_cell_tables(const StepArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.dm.nC) return;
    const size_t n = static_cast<size_t>(a.dm.nC);
    const double* cr = a.ds.cellrec;
    const double U[3] = {cr[REC_UX * n + c], cr[REC_UY * n + c], cr[REC_UZ * n + c]};
    write_maxwell_tables(a.dm, a.ds.ctab, n, c, U, cr[REC_INVRT * n + c], cr[REC_A * n + c]);
}

// relax factor of the cell records for a time step (when the records were
// written without knowing it)
__global__ void k_cell_prep(const StepArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.dm.nC) return;
    const double tau = a.ds.cm[static_cast<size_t>(c) * 9 + 8];
    const double dt = step_dt(a);
    a.ds.cellrec[REC_R * static_cast<size_t>(a.dm.nC) + c] = 1.5 * dt / (2.0 * tau + dt);
}

// initial Maxwellian state (fvDVM.C:414-426), DV-major
template <typename Real>
__global__ void k_init_state(const StepArgs a) {
    const DevMesh& m = a.dm;
    const size_t n = static_cast<size_t>(m.nv_loc) * m.nC;
    const double K3D = m.K + 3.0 - m.D;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int d = m.dv_base + static_cast<int>(i / m.nC), c = static_cast<int>(i % m.nC);
        const double* cm = a.ds.cm + static_cast<size_t>(c) * 9;
        const double RT = m.R * cm[4];
        const double cx = cm[1] - m.xi[3 * d], cy = cm[2] - m.xi[3 * d + 1], cz = cm[3] - m.xi[3 * d + 2];
        const double ge = cm[0] * inv_norm(RT, m.D) * exp(-0.5 * (cx * cx + cy * cy + cz * cz) / RT);
        const double he = K3D * ge * RT;
        if (sizeof(Real) == 4 && m.gref) {
            // FP32 storage of a tensor DV set: the deviation from the reference
            const int dl = static_cast<int>(i / m.nC);
            reinterpret_cast<Real*>(a.ds.g[a.ds.cur])[i] = Real(ge - m.gref[dl]);
            reinterpret_cast<Real*>(a.ds.h[a.ds.cur])[i] = Real(he - m.href[dl]);
        } else {
            reinterpret_cast<Real*>(a.ds.g[a.ds.cur])[i] = Real(ge);
            reinterpret_cast<Real*>(a.ds.h[a.ds.cur])[i] = Real(he);
        }
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
    const double S[3] = {m.bS[3 * b], m.bS[3 * b + 1], m.bS[3 * b + 2]};
    double acc[15];
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;
    double inby = 0.0;
    const double K3D = m.K + 3.0 - m.D;
    const double RTw = 1.0 / br->invRT_in;
    for (int d = threadIdx.x; d < m.nv; d += blockDim.x) {
        const double xi[3] = {m.xi[3 * d], m.xi[3 * d + 1], m.xi[3 * d + 2]};
        const double xs = xi_dot_s(xi, S);
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
        for (int t = 0; t < static_cast<int>(blockDim.x); ++t) {
            for (int j = 0; j < 15; ++j) s[j] += red[t][j];
            si += redi[t];
        }
        double* mi = a.ds.bmom_in + static_cast<size_t>(b) * kNM;
        for (int j = 0; j < 15; ++j) mi[j] = s[j];
        br->inByRho = si;
    }
}

// adjustable time step of src/setDeltaTvar.H:34-48 from the Courant number
// CoNum = max_f dc_f (|U_f| + sqrt(D) xiMax) dt (fvDVM::getCoNum) of the
// faces in co[0] (the maximum per unit dt, as double bits): F = maxCo /
// (CoNum + SMALL), f = min(min(F, 1 + 0.1 F), 1.2), dt_out = min(f dt, maxDeltaT);
// SMALL = 1e-15 (OpenFOAM's double SMALL).  Unfused operations, so that
// the host evaluation of the same formula gives the same bits.
__global__ void k_adapt(const double* co, const double* dt_in, double* dt_out, double* hist, double max_co,
                        double max_dt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double per_dt = __longlong_as_double(*reinterpret_cast<const long long*>(co));
    const double dt = *dt_in;
    const double co_num = __dmul_rn(per_dt, dt);
    const double F = max_co / __dadd_rn(co_num, 1.0e-15);
    const double f = fmin(fmin(F, __dadd_rn(1.0, __dmul_rn(0.1, F))), 1.2);
    const double dtn = fmin(__dmul_rn(f, dt), max_dt);
    *dt_out = dtn;
    if (hist) *hist = dtn;
}

// raw cell moments of the current state, one thread per cell looping over
// this device's DVs (rows are contiguous in cells, so a warp reads coalesced)
template <int D, typename Real>
__global__ void k_state_moments(const StepArgs a) {
    const DevMesh& m = a.dm;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nC) return;
    const Real* g = reinterpret_cast<const Real*>(a.ds.g[a.ds.cur]);
    const Real* h = reinterpret_cast<const Real*>(a.ds.h[a.ds.cur]);
    double acc[15];
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;
    for (int dl = 0; dl < m.nv_loc; ++dl) {
        const int d = m.dv_base + dl;
        const double xi[3] = {__ldg(m.xi + 3 * d), __ldg(m.xi + 3 * d + 1), __ldg(m.xi + 3 * d + 2)};
        const double xi2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        const size_t idx = static_cast<size_t>(dl) * m.nC + c;
        const double gr = (sizeof(Real) == 4 && m.gref) ? __ldg(m.gref + dl) : 0.0;
        const double hr = (sizeof(Real) == 4 && m.href) ? __ldg(m.href + dl) : 0.0;
        accum<D>(acc, __ldg(m.w + d), xi, xi2, double(g[idx]) + gr, double(h[idx]) + hr);
    }
    double* p = a.ds.partC + static_cast<size_t>(c) * kNM;
    for (int j = 0; j < 15; ++j) p[j] = acc[j];
}

// Symmetry patches, after pass A (updateGHbarSurfSymmetryIn, fvDVM.C:1100-1179,
// discreteVelocity.C:691-773): every DV d incoming through the patch's first
// face (xi.S <= 0) takes the face value of its mirror DV along the patch's
// axis, and the face's raw moments gain it.  Pass A reconstructed the DVs
// with xi.S > -VSMALL through the face's own area vector and summed them; a
// mirror DV that is the DV itself changes nothing.  One thread per boundary
// face, DVs in ascending order.
template <int D, typename Real>
__global__ void k_symmetry_in(const StepArgs a) {
    const DevMesh& m = a.dm;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.nBF) return;
    const int axis = __ldg(m.bface_mirror + b);
    if (axis < 0) return;
    const int it = chk(__ldg(m.face_items + 2 * (m.nIF + b)), 0, m.n_items, a.ds.err);
    const int b0 = chk(b - __ldg(m.bface_patch_local + b), 0, m.nBF, a.ds.err);
    const double S0[3] = {__ldg(m.bS + 3 * b0), __ldg(m.bS + 3 * b0 + 1), __ldg(m.bS + 3 * b0 + 2)};
    const double S[3] = {__ldg(m.bS + 3 * b), __ldg(m.bS + 3 * b + 1), __ldg(m.bS + 3 * b + 2)};
    Real* fg = reinterpret_cast<Real*>(a.ds.fvg);
    Real* fh = reinterpret_cast<Real*>(a.ds.fvh);
    const size_t nI = static_cast<size_t>(m.n_items);
    const int n = m.n1d;
    double acc[15];
    for (int j = 0; j < 15; ++j) acc[j] = 0.0;
    for (int d = 0; d < m.nv; ++d) {
        const double xi[3] = {__ldg(m.xi + 3 * d), __ldg(m.xi + 3 * d + 1), __ldg(m.xi + 3 * d + 2)};
        if (xi_dot_s(xi, S0) > 0) continue;
        const int ix = d % n, iy = (d / n) % n, iz = D == 3 ? d / (n * n) : 0;
        const int t = axis == 0 ? d + (n - 1 - 2 * ix) : (axis == 1 ? d + (n - 1 - 2 * iy) * n
                                                                     : d + (n - 1 - 2 * iz) * n * n);
        if (t == d) continue;
        const double w = __ldg(m.w + d), xi2 = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
        const size_t sd = static_cast<size_t>(d) * nI + it, st = static_cast<size_t>(t) * nI + it;
        // FP32 storage of a tensor DV set holds deviations from the per-DV
        // reference: the mirror's value moves with its own reference
        const bool dev = sizeof(Real) == 4 && m.gref;
        const double grd = dev ? m.gref[d] : 0.0, hrd = dev ? m.href[d] : 0.0;
        const double grt = dev ? m.gref[t] : 0.0, hrt = dev ? m.href[t] : 0.0;
        if (xi_dot_s(xi, S) > -kVSmall) accum<D>(acc, -w, xi, xi2, double(fg[sd]) + grd, double(fh[sd]) + hrd);
        if (dev) {
            fg[sd] = Real(double(fg[st]) + grt - grd);
            fh[sd] = Real(double(fh[st]) + hrt - hrd);
        } else {
            fg[sd] = fg[st];
            fh[sd] = fh[st];
        }
        accum<D>(acc, w, xi, xi2, double(fg[sd]) + grd, double(fh[sd]) + hrd);
    }
    double* p = a.ds.partF + static_cast<size_t>(it) * kNM;
    for (int j = 0; j < 14; ++j) p[j] += acc[j];
}

// pressureIn / pressureOut faces after the cell macros (updatePressureInOutBC,
// fvDVM.C:1745-1821): the next step's incoming far-field DFs take
//   pressureIn:  rho_b = p / R / T_b
//   pressureOut: rho_b = rho_i + (p - rho_i R T_i) / a_i / a_i, T_b = p / (R rho_i)
// from the owner cell i, a_i = sqrt(R T_i (K+5)/(K+3)); the patch velocity
// follows the characteristics (kept for output).
__global__ void k_pressure_bc(const StepArgs a) {
    const DevMesh& m = a.dm;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.nBF) return;
    const int pt = __ldg(m.bface_ptype + b);
    if (pt != DUGKS_PATCH_PRESSURE_IN && pt != DUGKS_PATCH_PRESSURE_OUT) return;
    BRec* br = a.ds.brec + b;
    const double* cm = a.ds.cm + static_cast<size_t>(chk(__ldg(m.bface_owner + b), 0, m.nC, a.ds.err)) * 9;
    const double rhoi = cm[0], Ui[3] = {cm[1], cm[2], cm[3]}, Ti = cm[4];
    const double R = m.R, p = br->p;
    const double ai = sqrt(R * Ti * (m.K + 5) / (m.K + 3));
    const double S[3] = {__ldg(m.bS + 3 * b), __ldg(m.bS + 3 * b + 1), __ldg(m.bS + 3 * b + 2)};
    const double magS = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
    const double nv[3] = {S[0] / magS, S[1] / magS, S[2] / magS};
    const double Un = Ui[0] * nv[0] + Ui[1] * nv[1] + Ui[2] * nv[2];
    double UnIn;
    if (pt == DUGKS_PATCH_PRESSURE_IN) {
        br->rho_in = p / R / br->T;
        UnIn = Un + (p - rhoi * R * Ti) / rhoi / ai;
    } else {
        br->rho_in = rhoi + (p - rhoi * R * Ti) / ai / ai;
        br->T = p / (R * rhoi);
        const double RT = R * br->T;
        br->K_in = inv_norm(RT, m.D);
        br->invRT_in = 1.0 / RT;
        br->hfac = RT * (m.K + 3.0 - m.D);
        UnIn = Un + (rhoi * R * Ti - p) / rhoi / ai;
    }
    for (int k = 0; k < 3; ++k) br->U[k] = UnIn * nv[k] + (Ui[k] - Un * nv[k]);
}

// part[0][i] = sum over chunks of part[ch][i], in chunk order (the order the
// combine kernels sum them in), for the cross-shard reduction
__global__ void k_sum_chunks(double* part, int chunks, size_t n) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        double v = part[i];
        for (int ch = 1; ch < chunks; ++ch) v += part[static_cast<size_t>(ch) * n + i];
        part[i] = v;
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
            if (e == cudaSuccess && a.dm.n_sym_faces > 0) {
                const int nb = (a.dm.nBF + 127) / 128;
                if (precision == DUGKS_FP64) {
                    if (a.dm.D == 3) k_symmetry_in<3, double><<<nb, 128, 0, s>>>(a);
                    else k_symmetry_in<2, double><<<nb, 128, 0, s>>>(a);
                } else {
                    if (a.dm.D == 3) k_symmetry_in<3, float><<<nb, 128, 0, s>>>(a);
                    else k_symmetry_in<2, float><<<nb, 128, 0, s>>>(a);
                }
                ++n;
                e = cudaGetLastError();
            }
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
            if (a.dm.n_pressure_faces > 0) {
                k_pressure_bc<<<(a.dm.nBF + tb - 1) / tb, tb, 0, s>>>(a);
                ++n;
            }
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

cudaError_t launch_state_moments(const StepArgs& a, int precision, cudaStream_t s) {
    const int tb = 128, nb = (a.dm.nC + tb - 1) / tb;
    if (precision == DUGKS_FP64) {
        if (a.dm.D == 3) k_state_moments<3, double><<<nb, tb, 0, s>>>(a);
        else k_state_moments<2, double><<<nb, tb, 0, s>>>(a);
    } else {
        if (a.dm.D == 3) k_state_moments<3, float><<<nb, tb, 0, s>>>(a);
        else k_state_moments<2, float><<<nb, tb, 0, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_cell_combine_one(const StepArgs& a, double dt_next, cudaStream_t s) {
    StepArgs one = a;
    one.chunks = 1;
    const Consts k = make_consts(a.dm, a.dt);
    k_cell_combine<<<(a.dm.nC + 255) / 256, 256, 0, s>>>(one, k, dt_next);
    return cudaGetLastError();
}

cudaError_t launch_state_macros(const StepArgs& a, int precision, cudaStream_t s) {
    cudaError_t e = launch_state_moments(a, precision, s);
    return e != cudaSuccess ? e : launch_cell_combine_one(a, 0.0, s);
}

cudaError_t launch_sum_chunks(double* part, int chunks, size_t n, cudaStream_t s) {
    if (chunks <= 1 || n == 0) return cudaSuccess;
    const int tb = 256;
    const int nb = static_cast<int>(std::min<size_t>((n + tb - 1) / tb, 148 * 16));
    k_sum_chunks<<<nb, tb, 0, s>>>(part, chunks, n);
    return cudaGetLastError();
}

cudaError_t launch_cell_records(const StepArgs& a, cudaStream_t s) {
    k_cell_records<<<(a.dm.nC + 255) / 256, 256, 0, s>>>(a, make_consts(a.dm, a.dt));
    return cudaGetLastError();
}

cudaError_t launch_adapt(const StepArgs& a, const double* dt_in, double* dt_out, double* hist, double max_co,
                         double max_dt, cudaStream_t s) {
    k_adapt<<<1, 32, 0, s>>>(a.ds.co, dt_in, dt_out, hist, max_co, max_dt);
    return cudaGetLastError();
}

cudaError_t launch_cell_prep(const StepArgs& a, cudaStream_t s) {
    k_cell_prep<<<(a.dm.nC + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_init(const StepArgs& a, int precision, cudaStream_t s) {
    if (precision == DUGKS_FP64) k_init_state<double><<<1184, 256, 0, s>>>(a);
    else k_init_state<float><<<1184, 256, 0, s>>>(a);
    k_cell_tables<<<(a.dm.nC + 255) / 256, 256, 0, s>>>(a);
    if (a.dm.nBF > 0) k_init_wall<<<a.dm.nBF, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace dugks

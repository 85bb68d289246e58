// kernels3d.cuh -- CUDA kernels of the 3D (x, y, z) semi-implicit time step.
//
// Same execution model as the 2D kernels: one thread per cell, explicit
// passes written face-owner style (each face value has exactly one writing
// thread, chosen as the last writer of the reference's lexicographic loop),
// and the implicit corrector as three colour phases per outer sweep with
// colour = (i + j + k) mod 3.  A cell's in-cell solve writes velocities and
// mass fluxes only at the cell and its three lower face neighbours and reads
// within the axis cross of radius 2, so two cells of one colour never touch
// each other's data.
#pragma once
#include "kernels2d.cuh"
#include "phys3d.cuh"

namespace pdac {

__device__ __forceinline__ void ijk_of(const Prm &P, int c, int &i, int &j, int &k) {
    const unsigned long long u = (unsigned)c;
    const unsigned q1 = P.mnx ? (unsigned)__umul64hi(u, P.mnx) : (unsigned)c / (unsigned)P.nx;  // c / nx
    const unsigned q2 = P.mny ? (unsigned)__umul64hi(q1, P.mny) : q1 / (unsigned)P.ny;           // c / (nx ny)
    i = (int)((unsigned)c - q1 * (unsigned)P.nx) + 1;
    j = (int)(q1 - q2 * (unsigned)P.ny) + 1;
    k = (int)q2 + 1;
}
#define MFX(ph, comp, face) (F.mf + ((size_t)((ph) * 3 + (comp)) * 3 + (face)) * P.ncell)

// ---------------------------------------------------------------------------
// boundary, bdry.f:22-726 + inoutflow.f:1-126 (3D)
// ---------------------------------------------------------------------------
__device__ void boundary_cell3d(const Prm &P, const Fld &F, int c) {
    int f0 = P.flag[c];
    if (!(f0 == FLUID || f0 == DOME || f0 == BL_CELL)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    raw3(P, i, j, k, R);
    const int *fl = P.flag;
    auto acts = [](int f) { return f == SLIP || f == NOSLIP || f == FREE_IO || f == ZERO_GRAD; };
    if (!acts(fl[R.e]) && !acts(fl[R.w]) && !acts(fl[R.n]) && !acts(fl[R.s]) && !acts(fl[R.t]) && !acts(fl[R.b])) return;
    double usv[PDAC_MAXP];
    int ns = P.ns;
    auto set_s = [&](double *a, int dst, double v) { for (int is = 1; is <= ns; ++is) SOL(a, dst, is) = v; };
    auto copy_s = [&](double *a, int dst, int src, double f) { for (int is = 1; is <= ns; ++is) SOL(a, dst, is) = f * SOL(a, src, is); };
    // East, bdry.f:216-283
    {
        int n2 = R.e, n1 = c, n0 = R.w, f2 = fl[n2];
        if (f2 == SLIP) {
            F.ug[n1] = 0; set_s(F.us, n1, 0.0); F.ug[n2] = 0; set_s(F.us, n2, 0.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
        } else if (f2 == NOSLIP) {
            F.ug[n1] = 0; set_s(F.us, n1, 0.0); F.ug[n2] = 0; set_s(F.us, n2, 0.0);
            if (!(fl[R.et] & 1)) { F.wg[n2] = -F.wg[n1]; copy_s(F.ws, n2, n1, -1.0); }
            if (!(fl[R.en] & 1)) { F.vg[n2] = -F.vg[n1]; copy_s(F.vs, n2, n1, -1.0); }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.ug[n1] = F.ug[n0]; copy_s(F.us, n1, n0, 1.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
            double gnorm = P.gravx * 0.5 * (P.dx[i + 1] + P.dx[i]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.us, n1, is);
            inoutflow_d(P, F, F.ug[n1], usv, n2, n1, k, gnorm);
        }
    }
    // West, bdry.f:285-344
    {
        int n2 = R.w, n1 = c, f2 = fl[n2];
        if (f2 == SLIP) {
            F.ug[n2] = 0; set_s(F.us, n2, 0.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
        } else if (f2 == NOSLIP) {
            F.ug[n2] = 0; set_s(F.us, n2, 0.0);
            if (!(fl[R.wt] & 1)) { F.wg[n2] = -F.wg[n1]; copy_s(F.ws, n2, n1, -1.0); }
            // bdry.f:318 tests the west-top cell for the y velocity as well
            if (!(fl[R.wt] & 1)) { F.vg[n2] = -F.vg[n1]; copy_s(F.vs, n2, n1, -1.0); }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
            double gnorm = P.gravx * 0.5 * (P.dx[i - 1] + P.dx[i]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.us, n2, is);
            inoutflow_d(P, F, F.ug[n2], usv, n2, n1, k, gnorm);
        }
    }
    // North, bdry.f:350-408
    {
        int n2 = R.n, n1 = c, n0 = R.s, f2 = fl[n2];
        if (f2 == SLIP) {
            F.vg[n1] = 0; set_s(F.vs, n1, 0.0); F.vg[n2] = 0; set_s(F.vs, n2, 0.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
        } else if (f2 == NOSLIP) {
            F.vg[n1] = 0; set_s(F.vs, n1, 0.0); F.vg[n2] = 0; set_s(F.vs, n2, 0.0);
            if (!(fl[R.en] & 1)) { F.ug[n2] = -F.ug[n1]; copy_s(F.us, n2, n1, -1.0); }
            if (!(fl[R.nt] & 1)) { F.wg[n2] = -F.wg[n1]; copy_s(F.ws, n2, n1, -1.0); }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.vg[n1] = F.vg[n0]; copy_s(F.vs, n1, n0, 1.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
            double gnorm = P.gravy * 0.5 * (P.dy[j] + P.dy[j + 1]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.vs, n1, is);
            inoutflow_d(P, F, F.vg[n1], usv, n2, n1, k, gnorm);
        }
    }
    // South, bdry.f:410-470
    {
        int n2 = R.s, n1 = c, f2 = fl[n2];
        if (f2 == SLIP) {
            F.vg[n2] = 0; set_s(F.vs, n2, 0.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
        } else if (f2 == NOSLIP) {
            F.vg[n2] = 0; set_s(F.vs, n2, 0.0);
            if (!(fl[R.es] & 1)) { F.ug[n2] = -F.ug[n1]; copy_s(F.us, n2, n1, -1.0); }
            if (!(fl[R.st] & 1)) { F.wg[n2] = -F.wg[n1]; copy_s(F.ws, n2, n1, -1.0); }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
            double gnorm = P.gravy * 0.5 * (P.dy[j - 1] + P.dy[j]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.vs, n2, is);
            inoutflow_d(P, F, F.vg[n2], usv, n2, n1, k, gnorm);
        }
    }
    // Top, bdry.f:476-583
    {
        int n2 = R.t, n1 = c, f2 = fl[n2];
        if (f2 == SLIP) {
            F.wg[n1] = 0; set_s(F.ws, n1, 0.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
        } else if (f2 == NOSLIP) {
            F.wg[n1] = 0; set_s(F.ws, n1, 0.0);
            if (!(fl[R.et] & 1)) { F.ug[n2] = -F.ug[n1]; copy_s(F.us, n2, n1, -1.0); }
            if (!(fl[R.nt] & 1)) { F.vg[n2] = -F.vg[n1]; copy_s(F.vs, n2, n1, -1.0); }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            double d0 = P.dz[k - 1], d1 = P.dz[k], d2 = P.dz[k + 1];
            const int ord = 0;
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            auto extrap = [&](double f2v, double f1v, double d12, double dxv) {
                double gradient = (f2v - f1v) / d12 * ord;
                return f2v + gradient * dxv;
            };
            F.wg[c] = extrap(F.wg[R.b], F.wg[R.bb], d0, d1);
            for (int is = 1; is <= ns; ++is) SOL(F.ws, c, is) = extrap(SOL(F.ws, R.b, is), SOL(F.ws, R.bb, is), d0, d1);
            F.wg[R.t] = extrap(F.wg[c], F.wg[R.b], d1, d2);
            for (int is = 1; is <= ns; ++is) SOL(F.ws, R.t, is) = extrap(SOL(F.ws, c, is), SOL(F.ws, R.b, is), d1, d2);
            if (f2 == ZERO_GRAD) {
                zerograd_d(P, F, n2, n1);
            } else {
                double gnorm = P.gravz * 0.5 * (P.dz[k] + P.dz[k + 1]);
                for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.ws, n1, is);
                inoutflow_d(P, F, F.wg[n1], usv, n2, n1, k + 1, gnorm);
            }
        }
    }
    // Bottom, bdry.f:587-683
    {
        int n1 = c, n2 = R.b, f2 = fl[n2];
        if (f2 == SLIP) {
            F.wg[n2] = 0; set_s(F.ws, n2, 0.0);
            if (fl[R.eb] == SLIP) { F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0); }
            if (fl[R.nb] == SLIP) { F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0); }
        } else if (f2 == NOSLIP) {
            F.wg[n2] = 0; set_s(F.ws, n2, 0.0);
            if (fl[R.eb] == NOSLIP) { F.ug[n2] = -F.ug[n1]; copy_s(F.us, n2, n1, -1.0); }
            if (fl[R.nb] == NOSLIP) { F.vg[n2] = -F.vg[n1]; copy_s(F.vs, n2, n1, -1.0); }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.wg[n2] = F.wg[n1]; copy_s(F.ws, n2, n1, 1.0);
            F.ug[n2] = F.ug[n1]; copy_s(F.us, n2, n1, 1.0);
            F.vg[n2] = F.vg[n1]; copy_s(F.vs, n2, n1, 1.0);
            double gnorm = P.gravz * 0.5 * (P.dz[k - 1] + P.dz[k]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.ws, n2, is);
            inoutflow_d(P, F, F.wg[n2], usv, n2, n1, k - 1, gnorm);
        }
    }
}

// the 3D boundary pass with one thread per cell (see k_boundary2d)
__global__ void k_boundary3d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < P.ncell) boundary_cell3d(P, F, c);
}

// ---------------------------------------------------------------------------
// fieldn, tilde.f:125-274 (3D)
// ---------------------------------------------------------------------------
__global__ void k_fieldn3d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    bool interior = i >= 2 && i <= P.nx - 1 && j >= 2 && j <= P.ny - 1 && k >= 2 && k <= P.nz - 1;
    int ns = P.ns;
    if (interior) {
        Raw3 R;
        raw3(P, i, j, k, R);
        int ijke = is_wallf(P.flag[R.e]) ? c : R.e;
        int ijkn = is_wallf(P.flag[R.n]) ? c : R.n;
        int ijkt = is_wallf(P.flag[R.t]) ? c : R.t;
        const double *dx = P.dx, *dy = P.dy, *dz = P.dz;
        double indxp = P.hx[i], indyp = P.hy[j], indzp = P.hz[k];
        double rgp_e = (dx[i + 1] * F.rgp[c] + dx[i] * F.rgp[ijke]) * indxp;
        double rgp_n = (dy[j + 1] * F.rgp[c] + dy[j] * F.rgp[ijkn]) * indyp;
        double rgp_t = (dz[k + 1] * F.rgp[c] + dz[k] * F.rgp[ijkt]) * indzp;
        F.rugn[c] = rgp_e * F.ug[c];
        F.rvgn[c] = rgp_n * F.vg[c];
        F.rwgn[c] = rgp_t * F.wg[c];
        for (int is = 1; is <= ns; ++is) {
            double rlk_e = (SOL(F.rlk, c, is) * dx[i + 1] + SOL(F.rlk, ijke, is) * dx[i]) * indxp;
            double rlk_n = (SOL(F.rlk, c, is) * dy[j + 1] + SOL(F.rlk, ijkn, is) * dy[j]) * indyp;
            double rlk_t = (SOL(F.rlk, c, is) * dz[k + 1] + SOL(F.rlk, ijkt, is) * dz[k]) * indzp;
            SOL(F.rusn, c, is) = rlk_e * SOL(F.us, c, is);
            SOL(F.rvsn, c, is) = rlk_n * SOL(F.vs, c, is);
            SOL(F.rwsn, c, is) = rlk_t * SOL(F.ws, c, is);
        }
    } else {
        F.rugn[c] = 0; F.rvgn[c] = 0; F.rwgn[c] = 0;
        for (int is = 1; is <= ns; ++is) { SOL(F.rusn, c, is) = 0; SOL(F.rvsn, c, is) = 0; SOL(F.rwsn, c, is) = 0; }
    }
    F.pn[c] = F.p[c];
    F.epn[c] = F.ep[c];
    F.rgpn[c] = F.rgp[c];
    F.siegn[c] = F.sieg[c];
    for (int ig = 0; ig < P.ng; ++ig) GAS(F.rgpgcn, c, ig) = F.rgpn[c] * GAS(F.ygc, c, ig);
    for (int is = 1; is <= ns; ++is) {
        SOL(F.rlkn, c, is) = SOL(F.rlk, c, is);
        SOL(F.siesn, c, is) = SOL(F.sies, c, is);
    }
    double xg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) xg[ig] = GAS(F.xgc, c, ig);
    double mu, ka;
    viscon(P, mu, ka, xg, F.tg[c]);
    F.mug[c] = mu;
    F.kapg[c] = ka;
}

// ---------------------------------------------------------------------------
// tilde momentum fluxes, compute_all_fluxes_tilde tilde.f:850-1326 (3D)
// ---------------------------------------------------------------------------
// one thread per (cell, phase) for one momentum component COMP (0 = x,
// 1 = y, 2 = z): consecutive threads take consecutive cells of one phase.
// Real is the arithmetic type: double, or float in the mixed-precision mode
// (the FP64 state is converted as it is read; fluxes are stored in FP64).
template <int COMP, typename Real = double>
__global__ void __launch_bounds__(128, PDAC_FLUX_MINB) k_tilde_flux3d(Prm P, Fld F) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)P.ncell * (unsigned)(P.ns + 1)) return;
    int ph = (int)(t / (unsigned)P.ncell), c = (int)(t % (unsigned)P.ncell);
    if (!fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    bool dw = !fluid(P, R.w), ds = !fluid(P, R.s), db = !fluid(P, R.b);
    bool mus = P.muscl > 0 && P.flag[c] == FLUID;
    size_t n = P.ncell;
    size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
    const double *U = ph == 0 ? F.ug : F.us + off;
    const double *V = ph == 0 ? F.vg : F.vs + off;
    const double *W = ph == 0 ? F.wg : F.ws + off;
    const double *D = ph == 0 ? F.rgp : F.rlk + off;
    S3T<Real> u, v, w, d, ds3;
    rnb3(u, U, R);
    rnb3(v, V, R);
    rnb3(w, W, R);
    if (ib_masked(P, c)) { ib_mask3(P, u, R, 1); ib_mask3(P, v, R, 16); ib_mask3(P, w, R, 4); }
    nb3(d, D, R, M);
    F6T<Real> f = {0, 0, 0, 0, 0, 0};
    if (COMP == 0) {  // x momentum
        interp_x3(P, d, i, ds3);
        flu_3d(P, f, dw, ds, db, ds3, u, v, w, i);
        if (mus && i != P.nx - 1) muscl_flu_3d(P, f, ds3, u, v, w, i, j, k);
    } else if (COMP == 1) {  // y momentum
        interp_y3(P, d, j, ds3);
        flv_3d(P, f, dw, ds, db, ds3, u, v, w, j);
        if (mus && j != P.ny - 1) muscl_flv_3d(P, f, ds3, u, v, w, i, j, k);
    } else {  // z momentum
        interp_z3(P, d, k, ds3);
        flw_3d(P, f, dw, ds, db, ds3, u, v, w, k);
        if (mus && k != P.nz - 1) muscl_flw_3d(P, f, ds3, u, v, w, i, j, k);
    }
    MFX(ph, COMP, 0)[c] = f.e; MFX(ph, COMP, 1)[c] = f.n; MFX(ph, COMP, 2)[c] = f.t;
    if (dw) MFX(ph, COMP, 0)[R.w] = f.w;
    if (ds) MFX(ph, COMP, 1)[R.s] = f.s;
    if (db) MFX(ph, COMP, 2)[R.b] = f.b;
}

// tilde mesh loop, tilde.f:276-848 (3D), with stress3D, kdrags/sdrag and
// inter (drag.f:11-298).  app0 holds the interphase matrix of the previous
// visit of each cell in this step; it is read only when alpha < 1.
// viscous stress divergence of one phase of one cell (viscg / viscs,
// visc.f:150-291, stress3D visc.f:293-559) with the particle repulsion term
// (tilde.f:362-416); one thread per (cell, phase), consecutive threads take
// consecutive cells of one phase
__global__ void __launch_bounds__(128, PDAC_FLUX_MINB) k_visc3d(Prm P, Fld F) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)P.ncell * (unsigned)(P.ns + 1)) return;
    int ph = (int)(t / (unsigned)P.ncell), c = (int)(t % (unsigned)P.ncell);
    if (!fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    const double *dx = P.dx, *dy = P.dy, *dz = P.dz;
    size_t n = P.ncell;
    size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
    int ijke = M.e, ijkn = M.n, ijkt = M.t;
    double indxp = P.hx[i], indyp = P.hy[j], indzp = P.hz[k];
    const double a_rep = -8.76, b_rep = -0.27;
    double vx = 0, vy = 0, vz = 0;
    if (ph == 0) {
        if (P.gas_viscosity) {
            const double *mug = F.mug, *mut = P.iturb ? F.mugt : F.mug, *ep = F.ep;
            stress3d_cell(P, R, M, i, j, k, [&](int q) { return mut[q]; }, [&](int q) { return mug[q]; },
                          [&](int q) { return ep[q]; }, F.ug, F.vg,
                          F.wg, vx, vy, vz);
        }
    } else if (P.part_viscosity) {
        const double cm = P.cmus[ph], ir = P.inrl[ph];
        const double *rl = F.rlk + off;
        const double *mst = P.iss ? F.must + off : nullptr;
        stress3d_cell(P, R, M, i, j, k, [&](int q) { return mst ? mst[q] : cm; }, [&](int) { return cm; },
                      [&](int q) { return rl[q] * ir; }, F.us + off,
                      F.vs + off, F.ws + off, vx, vy, vz);
        if (P.repulsive_model == 1) {
            double rc = rl[c], re = rl[ijke], rn = rl[ijkn], rt = rl[ijkt];
            double epsx = (dx[i + 1] * rc + dx[i] * re) * indxp * ir;
            double gepx = pdac_fp::pow(10.0, -a_rep * epsx + b_rep);
            vx = vx - gepx * indxp * 2.0 * (re - rc) * ir;
            double epsz = (dz[k + 1] * rc + dz[k] * rt) * indzp * ir;
            double gepz = pdac_fp::pow(10.0, -a_rep * epsz + b_rep);
            vz = vz - gepz * indzp * 2.0 * (rt - rc) * ir;
            double epsy = (dy[j + 1] * rc + dy[j] * rn) * indyp * ir;
            double gepy = pdac_fp::pow(10.0, -a_rep * epsy + b_rep);
            vy = vy - gepy * indyp * 2.0 * (rn - rc) * ir;
        }
    }
    F.vis[(size_t)(ph * 3 + 0) * n + c] = vx;
    F.vis[(size_t)(ph * 3 + 1) * n + c] = vy;
    F.vis[(size_t)(ph * 3 + 2) * n + c] = vz;
}

template <int NP>
__global__ void __launch_bounds__(128, PDAC_FLUX_MINB) k_tilde3d(Prm P, Fld F, double dt, const double *app0u, const double *app0v, const double *app0w) {
    constexpr int MP = Sys<NP>::M;  // phase capacity + 1
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    const double *dx = P.dx, *dy = P.dy, *dz = P.dz, *indx = P.indx, *indy = P.indy, *indz = P.indz;
    size_t n = P.ncell;
    const int ns = nphases<NP>(P) - 1, nph = ns + 1;
    int imjk = R.w, ijmk = R.s, ijkm = R.b, ijke = M.e, ijkn = M.n, ijkt = M.t;
    double alpha = P.alpha, ag = P.alphagrav;
    double dxi = dx[i], dxip1 = dx[i + 1], dyj = dy[j], dyjp1 = dy[j + 1], dzk = dz[k], dzkp1 = dz[k + 1];
    double indxp = P.hx[i], indyp = P.hy[j], indzp = P.hz[k];
    double rr[MP][3];
    double kpgv[MP];
#pragma unroll
    for (int ph = 0; ph <= ns; ++ph) {
        size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
        // viscous terms from k_visc3d
        double vx = F.vis[(size_t)(ph * 3 + 0) * n + c], vy = F.vis[(size_t)(ph * 3 + 1) * n + c];
        double vz = F.vis[(size_t)(ph * 3 + 2) * n + c];
        double ufx = MFX(ph, 0, 0)[c] - MFX(ph, 0, 0)[imjk], ufy = MFX(ph, 0, 1)[c] - MFX(ph, 0, 1)[ijmk];
        double ufz = MFX(ph, 0, 2)[c] - MFX(ph, 0, 2)[ijkm];
        double vfx = MFX(ph, 1, 0)[c] - MFX(ph, 1, 0)[imjk], vfy = MFX(ph, 1, 1)[c] - MFX(ph, 1, 1)[ijmk];
        double vfz = MFX(ph, 1, 2)[c] - MFX(ph, 1, 2)[ijkm];
        double wfx = MFX(ph, 2, 0)[c] - MFX(ph, 2, 0)[imjk], wfy = MFX(ph, 2, 1)[c] - MFX(ph, 2, 1)[ijmk];
        double wfz = MFX(ph, 2, 2)[c] - MFX(ph, 2, 2)[ijkm];
        double ep_e, ep_n, ep_t, d_c, d_e, d_n, d_t;
        if (ph == 0) {
            if (P.pmodel == 1) {
                ep_e = (dxi * F.epn[ijke] + dxip1 * F.epn[c]) * indxp;
                ep_n = (dyj * F.epn[ijkn] + dyjp1 * F.epn[c]) * indyp;
                ep_t = (dzk * F.epn[ijkt] + dzkp1 * F.epn[c]) * indzp;
            } else { ep_e = ep_n = ep_t = 1.0; }
            d_c = F.rgpn[c]; d_e = F.rgpn[ijke]; d_n = F.rgpn[ijkn]; d_t = F.rgpn[ijkt];
        } else {
            const double *rln = F.rlkn + off;
            if (P.pmodel == 1) {
                ep_e = (dxi * rln[ijke] + dxip1 * rln[c]) * indxp * P.inrl[ph];
                ep_n = (dyj * rln[ijkn] + dyjp1 * rln[c]) * indyp * P.inrl[ph];
                ep_t = (dzk * rln[ijkt] + dzkp1 * rln[c]) * indzp * P.inrl[ph];
            } else { ep_e = ep_n = ep_t = 0.0; }
            d_c = rln[c]; d_e = rln[ijke]; d_n = rln[ijkn]; d_t = rln[ijkt];
        }
        double t_;
        // x momentum, tilde.f:482-489 (gas) / 537-546 (particles)
        t_ = vx;
        t_ = t_ - indxp * 2.0 * ufx;
        if (ph == 0) t_ = t_ + (1.0 - ag) * (dx[i + 1] * d_c + dx[i] * d_e) * indxp * P.gravx;
        else t_ = t_ + (1.0 - ag) * indxp * P.gravx * (dx[i + 1] * d_c + dx[i] * d_e);
        t_ = t_ - indy[j] * ufy;
        t_ = t_ - indz[k] * ufz;
        t_ = t_ + (1.0 - alpha) * indxp * 2.0 * ep_e * (F.pn[c] - F.pn[ijke]);
        rr[ph][0] = (ph == 0 ? F.rugn[c] : SOL(F.rusn, c, ph)) + dt * t_;
        if (ph > 0) rr[ph][0] = rr[ph][0] + dt * SOL(F.sink, c, ph) * SOL(F.us, c, ph);
        // y momentum
        t_ = vy;
        if (ph == 0) t_ = t_ + (1.0 - ag) * (dy[j + 1] * d_c + dy[j] * d_n) * indyp * P.gravy;
        else t_ = t_ + (1.0 - ag) * indyp * P.gravy * (dy[j + 1] * d_c + dy[j] * d_n);
        t_ = t_ - indx[i] * vfx;
        t_ = t_ - indyp * 2.0 * vfy;
        t_ = t_ - indz[k] * vfz;
        t_ = t_ + (1.0 - alpha) * indyp * 2.0 * ep_n * (F.pn[c] - F.pn[ijkn]);
        rr[ph][1] = (ph == 0 ? F.rvgn[c] : SOL(F.rvsn, c, ph)) + dt * t_;
        if (ph > 0) rr[ph][1] = rr[ph][1] + dt * SOL(F.sink, c, ph) * SOL(F.vs, c, ph);
        // z momentum
        t_ = vz;
        if (ph == 0) t_ = t_ + (1.0 - ag) * (dz[k + 1] * d_c + dz[k] * d_t) * indzp * P.gravz;
        else t_ = t_ + (1.0 - ag) * indzp * P.gravz * (d_c * dz[k + 1] + d_t * dz[k]);
        t_ = t_ - indx[i] * wfx;
        t_ = t_ - indy[j] * wfy;
        t_ = t_ - indzp * 2.0 * wfz;
        t_ = t_ + (1.0 - alpha) * indzp * 2.0 * ep_t * (F.pn[c] - F.pn[ijkt]);
        rr[ph][2] = (ph == 0 ? F.rwgn[c] : SOL(F.rwsn, c, ph)) + dt * t_;
        if (ph > 0) rr[ph][2] = rr[ph][2] + dt * SOL(F.sink, c, ph) * SOL(F.ws, c, ph);
        if (ph > 0) {
            int is = ph;
            double dugs = ((F.ug[c] - SOL(F.us, c, is)) + (F.ug[imjk] - SOL(F.us, imjk, is))) * 0.5;
            double dwgs = ((F.wg[c] - SOL(F.ws, c, is)) + (F.wg[ijkm] - SOL(F.ws, ijkm, is))) * 0.5;
            double dvgs = ((F.vg[c] - SOL(F.vs, c, is)) + (F.vg[ijmk] - SOL(F.vs, ijmk, is))) * 0.5;
            kpgv[is] = drag_coeff(P, dugs, dvgs, dwgs, F.ep[c], F.rgp[c], SOL(F.rlk, c, is), F.mug[c], is);
        }
    }
    // inter, drag.f:173-246
    constexpr int NA = MP * (MP - 1) / 2 + 1;
    double au[NA], av[NA], aw[NA];
    double rlkc[MP];
#pragma unroll
    for (int is = 1; is <= ns; ++is) rlkc[is] = SOL(F.rlk, c, is);
    int ks = 0;
#pragma unroll
    for (int kk1 = 1; kk1 <= nph; ++kk1) {
        if (kk1 == 1) { ks++; au[ks] = av[ks] = aw[ks] = 0; }
        else {
#pragma unroll
            for (int kk = 1; kk <= kk1; ++kk) {
                ks++;
                if (kk == 1) { au[ks] = -kpgv[kk1 - 1] * dt; av[ks] = -kpgv[kk1 - 1] * dt; aw[ks] = -kpgv[kk1 - 1] * dt; }
                else if (kk == kk1) { au[ks] = av[ks] = aw[ks] = 0; }
                else {
                    double con = ppdrag(P, rlkc, kk1, kk);
                    double du = fabs(SOL(F.us, c, kk1 - 1) - SOL(F.us, c, kk - 1) + SOL(F.us, imjk, kk1 - 1) - SOL(F.us, imjk, kk - 1)) * 0.5;
                    double dv = fabs(SOL(F.vs, c, kk1 - 1) - SOL(F.vs, c, kk - 1) + SOL(F.vs, ijmk, kk1 - 1) - SOL(F.vs, ijmk, kk - 1)) * 0.5;
                    double dw = fabs(SOL(F.ws, c, kk1 - 1) - SOL(F.ws, c, kk - 1) + SOL(F.ws, ijkm, kk1 - 1) - SOL(F.ws, ijkm, kk - 1)) * 0.5;
                    au[ks] = -(con * du) * dt;
                    av[ks] = -(con * dv) * dt;
                    aw[ks] = -(con * dw) * dt;
                }
            }
        }
    }
#pragma unroll
    for (int kk1 = 1; kk1 <= nph; ++kk1) {
        double sx = 0, sy = 0, sz = 0;
#pragma unroll
        for (int kk = 1; kk <= kk1; ++kk) { int q = kk + kk1 * (kk1 - 1) / 2; sx = sx + au[q]; sy = sy + av[q]; sz = sz + aw[q]; }
#pragma unroll
        for (int kk = kk1; kk <= nph; ++kk) { int q = kk1 + kk * (kk - 1) / 2; sx = sx + au[q]; sy = sy + av[q]; sz = sz + aw[q]; }
        int q = kk1 * (kk1 + 1) / 2;
        au[q] = -sx; av[q] = -sy; aw[q] = -sz;
    }
    const int nap = nph * (nph + 1) / 2;
#pragma unroll
    for (int q = 1; q <= nap; ++q) { APP(F.appu, c, q) = au[q]; APP(F.appv, c, q) = av[q]; APP(F.appw, c, q) = aw[q]; }
    // (1 - alpha) explicit interphase part, tilde.f:597-680
    if (alpha != 1.0) {
        double coef0[3] = {dxi, dyj, dzk}, coef1[3] = {dxip1, dyjp1, dzkp1}, inv[3] = {indxp, indyp, indzp};
        int nbr[3] = {ijke, ijkn, ijkt};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double *a0 = q == 0 ? app0u : (q == 1 ? app0v : app0w);
            const double *gvq = q == 0 ? F.ug : (q == 1 ? F.vg : F.wg);
            const double *svq = q == 0 ? F.us : (q == 1 ? F.vs : F.ws);
            auto A = [&](int cell, int ls) {
                double own = q == 0 ? au[ls] : (q == 1 ? av[ls] : aw[ls]);
                return cell == c ? own : APP(a0, cell, ls);
            };
            auto AP = [&](int ls) { return (1.0 - alpha) * (coef0[q] * A(nbr[q], ls) + coef1[q] * A(c, ls)) * inv[q]; };
            auto vel = [&](int ph) { return ph == 0 ? gvq[c] : SOL(svq, c, ph); };
            rr[0][q] = rr[0][q] - AP(1) * vel(0);
#pragma unroll
            for (int l = 2; l <= nph; ++l) {
                int ls1 = l * (l - 1) / 2;
#pragma unroll
                for (int ll = 1; ll <= l; ++ll) {
                    int ls = ls1 + ll;
                    double f = AP(ls);
                    if (ll == 1) {
                        rr[0][q] = rr[0][q] - f * vel(l - 1);
                        rr[l - 1][q] = rr[l - 1][q] - f * vel(0);
                    } else if (ll == l) {
                        rr[l - 1][q] = rr[l - 1][q] - f * vel(l - 1);
                    } else {
                        rr[l - 1][q] = rr[l - 1][q] - f * vel(ll - 1);
                        rr[ll - 1][q] = rr[ll - 1][q] - f * vel(l - 1);
                    }
                }
            }
        }
    }
    if (P.immb) {
        double rs[MP];
        const int nb3[3] = {M.e, M.n, M.t}, nm3[3] = {R.w, R.s, R.b};
        const double *d3[3] = {P.dx, P.dy, P.dz};
        const int q3[3] = {i, j, k};
        for (int ax = 0; ax < 3; ++ax) {
            for (int is = 1; is <= ns; ++is) rs[is] = rr[is][ax];
            const double dm = d3[ax][q3[ax]], dp = d3[ax][q3[ax] + 1];
            ib_force(P, F, c, ax, nb3[ax], nm3[ax], dm, dp, 1.0 / (dm + dp), dt, kpgv, rr[0][ax], rs);
            for (int is = 1; is <= ns; ++is) rr[is][ax] = rs[is];
        }
    }
    F.rug[c] = rr[0][0]; F.rvg[c] = rr[0][1]; F.rwg[c] = rr[0][2];
#pragma unroll
    for (int is = 1; is <= ns; ++is) { SOL(F.rus, c, is) = rr[is][0]; SOL(F.rvs, c, is) = rr[is][1]; SOL(F.rws, c, is) = rr[is][2]; }
}

// predictor, iter.f:135-145
template <int NP>
__global__ void k_predictor3d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    face_solve<NP>(P, F, c, M.e, R.e, i, 0, +1, dt);
    face_solve<NP>(P, F, c, M.n, R.n, j, 1, +1, dt);
    face_solve<NP>(P, F, c, M.t, R.t, k, 2, +1, dt);
}

// mass flux of one cell over its six faces (calc_gas_mass_flux and
// calc_part_mass_flux, iter.f:597-925): densities remapped, velocities raw
__device__ __forceinline__ void cell_massflux3d(const Prm &P, const double *D, const double *U, const double *V,
                                                const double *W, const Raw3 &R, const Rem3 &M, int i, int j, int k,
                                                F6d &f) {
    S3 d;
    first_nb3(d, D, R, M);
    bool mus = P.muscl > 0 && P.flag[R.c] == FLUID;
    if (mus) third_nb3(d, D, M);
    const int *fl = P.flag;
    massflux_3d(P, d, U[R.w], U[R.c], V[R.s], V[R.c], W[R.b], W[R.c], i, j, k, mus, fl[R.w], fl[R.e], fl[R.s],
                fl[R.n], fl[R.b], fl[R.t], f);
}

// betas, iter.f:1112-1248 (3D)
__device__ __forceinline__ void betas_3d(const Prm &P, const Fld &F, const Raw3 &R, const Rem3 &M, int i, int j, int k,
                                         double dt, double &cnv, double &abt) {
    const double *dx = P.dx, *dy = P.dy, *dz = P.dz;
    int c = R.c;
    double indxp = P.hx[i], indxm = P.hx[i - 1];
    double indzp = P.hz[k], indzm = P.hz[k - 1];
    double indyp = P.hy[j], indym = P.hy[j - 1];
    auto open = [](int f) { return f == BL_CELL || f == FLUID || f == DOME || f == IMMB || f == FREE_IO || f == ZERO_GRAD; };
    const int *fl = P.flag;
    double iep_e = open(fl[R.e]) ? (dx[i + 1] * F.ep[c] + dx[i] * F.ep[M.e]) * indxp * indxp * 2.0 : 0.0;
    double iep_w = open(fl[R.w]) ? (dx[i - 1] * F.ep[c] + dx[i] * F.ep[M.w]) * indxm * indxm * 2.0 : 0.0;
    double iep_t = open(fl[R.t]) ? (dz[k + 1] * F.ep[c] + dz[k] * F.ep[M.t]) * indzp * indzp * 2.0 : 0.0;
    double iep_b = open(fl[R.b]) ? (dz[k - 1] * F.ep[c] + dz[k] * F.ep[M.b]) * indzm * indzm * 2.0 : 0.0;
    double iep_n = open(fl[R.n]) ? (dy[j + 1] * F.ep[c] + dy[j] * F.ep[M.n]) * indyp * indyp * 2.0 : 0.0;
    double iep_s = open(fl[R.s]) ? (dy[j - 1] * F.ep[c] + dy[j] * F.ep[M.s]) * indym * indym * 2.0 : 0.0;
    double iepx = (1.0 * iep_e + 1.0 * iep_w) * P.indx[i] * 1.0;
    double iepz = (iep_t + iep_b) * P.indz[k];
    double iepy = (iep_n + iep_s) * P.indy[j];
    double sqc = P.gammaair * F.p[c] / F.rog[c];
    double rbeta = F.ep[c] / sqc;
    rbeta = rbeta + dt * dt * (iepx + iepy + iepz);
    abt = 1.0 / rbeta;
    cnv = P.delg * F.rgp[c];
}

// initial gas mass fluxes + betas (iter.f:170-191): a face shared by two
// fluid cells ends with the value of the later cell in the reference loop
__global__ void k_mflux_init3d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    F6d f;
    cell_massflux3d(P, F.rgp, F.ug, F.vg, F.wg, R, M, i, j, k, f);
    F.rgfe[R.w] = f.w;
    F.rgfn[R.s] = f.s;
    F.rgft[R.b] = f.b;
    if (!fluid(P, R.e)) F.rgfe[c] = f.e;
    if (!fluid(P, R.n)) F.rgfn[c] = f.n;
    if (!fluid(P, R.t)) F.rgft[c] = f.t;
    betas_3d(P, F, R, M, i, j, k, dt, F.conv[c], F.abeta[c]);
}

// calc_res, iter.f:743-771 (3D)
__device__ __forceinline__ double calc_res_3d(const Prm &P, const Fld &F, const Raw3 &R, int i, int j, int k, double dt) {
    int c = R.c;
    const CellFaces b = cell_faces(P, c);
    double resx = (b.e * F.rgfe[c] - b.w * F.rgfe[R.w]) * P.indx[i] * 1.0;
    double resz = (b.t * F.rgft[c] - b.b * F.rgft[R.b]) * P.indz[k];
    double resy = (b.n * F.rgfn[c] - b.s * F.rgfn[R.s]) * P.indy[j];
    return F.rgp[c] - F.rgpn[c] + dt * b.ivf * (resx + resy + resz);
}

// calc_eps, iter.f:927-994 (3D)
template <int NP>
__device__ __forceinline__ void calc_eps_3d(const Prm &P, const Fld &F, const Raw3 &R, int i, int j, int k, double dt) {
    int c = R.c;
    const CellFaces b = cell_faces(P, c);
    double rls = 0;
#pragma unroll
    for (int is = 1; is <= nphases<NP>(P) - 1; ++is) {
        double rlkx = (b.e * SOL(F.rsfe, c, is) - b.w * SOL(F.rsfe, R.w, is)) * P.indx[i] * 1.0;
        double rlkz = (b.t * SOL(F.rsft, c, is) - b.b * SOL(F.rsft, R.b, is)) * P.indz[k];
        double rlky = (b.n * SOL(F.rsfn, c, is) - b.s * SOL(F.rsfn, R.s, is)) * P.indy[j];
        double t = SOL(F.rlkn, c, is) - dt * b.ivf * (rlkx + rlky + rlkz);
        t = t + dt * b.ivf * SOL(F.sink, c, is);
        double v = fmax(0.0, t);
        SOL(F.rlk, c, is) = v;
        rls = rls + v * P.inrl[is];
    }
    F.ep[c] = 1.0 - rls;
    if (rls > 1.0) atomicAdd(&F.counters[2], 1);
}


// ---------------------------------------------------------------------------
// ygas, ygas.f:27-325 (3D)
// ---------------------------------------------------------------------------
template <typename Real = double>
__global__ void __launch_bounds__(128, PDAC_SCALAR_FLUX_MINB) k_ygas_flux3d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    bool dw = !fluid(P, R.w), ds = !fluid(P, R.s), db = !fluid(P, R.b);
    bool mus = P.muscl > 0 && P.flag[c] == FLUID;
    S3T<Real> d;
    first_nb3(d, F.rgp, R, M);
    if (mus) third_nb3(d, F.rgp, M);
    Real uw = F.ug[R.w], uc = F.ug[c], vs = F.vg[R.s], vc = F.vg[c], wb = F.wg[R.b], wc = F.wg[c];
    for (int ig = 0; ig < P.ng; ++ig) {
        const double *Y = F.ygc + (size_t)ig * P.ncell;
        S3T<Real> y;
        first_nb3(y, Y, R, M);
        F6T<Real> f = {0, 0, 0, 0, 0, 0};
        fsc_3d(P, f, dw, ds, db, d, y, uw, uc, vs, vc, wb, wc);
        if (mus) {
            third_nb3(y, Y, M);
            muscl_fsc_3d(P, f, d, y, uc, vc, wc, i, j, k);
        }
        GAS(F.yfe, c, ig) = f.e;
        GAS(F.yfn, c, ig) = f.n;
        GAS(F.yft, c, ig) = f.t;
        if (dw) GAS(F.yfe, R.w, ig) = f.w;
        if (ds) GAS(F.yfn, R.s, ig) = f.s;
        if (db) GAS(F.yft, R.b, ig) = f.b;
    }
}

__global__ void k_ygas3d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    int imjk = at3(P, max(i - 1, 1), j, k), ijmk = at3(P, i, max(j - 1, 1), k), ijkm = at3(P, i, j, max(k - 1, 1));
    const CellFaces b = cell_faces(P, c);
    double rgpgc[PDAC_MAXG], rgpt = 0;
    for (int ig = 0; ig < P.ng; ++ig) {
        double yfx = b.e * GAS(F.yfe, c, ig) - b.w * GAS(F.yfe, imjk, ig);
        double yfz = b.t * GAS(F.yft, c, ig) - b.b * GAS(F.yft, ijkm, ig);
        double yfy = b.n * GAS(F.yfn, c, ig) - b.s * GAS(F.yfn, ijmk, ig);
        double v = GAS(F.rgpgcn, c, ig);
        v = v - b.ivf * dt * P.indx[i] * yfx * 1.0;
        v = v - b.ivf * dt * P.indy[j] * yfy;
        v = v - b.ivf * dt * P.indz[k] * yfz;
        if (v < 0.0) v = 0.0;
        rgpgc[ig] = v;
        rgpt = rgpt + v;
    }
    double rgpinv = 1.0 / rgpt, ygcdfg = 1.0, yg[PDAC_MAXG], xg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng - 1; ++ig) {
        yg[ig] = rgpgc[ig] * rgpinv;
        ygcdfg = ygcdfg - yg[ig];
    }
    yg[P.ng - 1] = ygcdfg;
    mole(P, xg, yg);
    for (int ig = 0; ig < P.ng; ++ig) { GAS(F.ygc, c, ig) = yg[ig]; GAS(F.xgc, c, ig) = xg[ig]; }
}

// ---------------------------------------------------------------------------
// htilde, htilde.f:25-575 (3D)
// ---------------------------------------------------------------------------
// GRAV as in k_htilde_flux2d
template <bool GRAV, typename Real = double>
__global__ void __launch_bounds__(128, PDAC_SCALAR_FLUX_MINB) k_htilde_flux3d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    bool dw = !fluid(P, R.w), ds = !fluid(P, R.s), db = !fluid(P, R.b);
    bool mus = P.muscl > 0 && P.flag[c] == FLUID;
    bool hw = P.flag[R.w] != 1, hs = P.flag[R.s] != 1, hb = P.flag[R.b] != 1;  // hotc.f tests the flag value
    size_t n = P.ncell;
    for (int ph = 0; ph <= P.ns; ++ph) {
        size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
        const double *EN = ph == 0 ? F.sieg : F.sies + off;
        const double *DE = ph == 0 ? F.rgp : F.rlk + off;
        const double *U = ph == 0 ? F.ug : F.us + off;
        const double *V = ph == 0 ? F.vg : F.vs + off;
        const double *W = ph == 0 ? F.wg : F.ws + off;
        double *fE = ph == 0 ? F.egfe : F.esfe + off;
        double *fN = ph == 0 ? F.egfn : F.esfn + off;
        double *fT = ph == 0 ? F.egft : F.esft + off;
        S3T<Real> en, de;
        first_nb3(en, EN, R, M);
        first_nb3(de, DE, R, M);
        Real uw = U[R.w], uc = U[c], vs = V[R.s], vc = V[c], wb = W[R.b], wc = W[c];
        F6T<Real> f = {0, 0, 0, 0, 0, 0};
        fsc_3d(P, f, dw, ds, db, en, de, uw, uc, vs, vc, wb, wc);
        if (mus) {
            third_nb3(en, EN, M);
            third_nb3(de, DE, M);
            muscl_fsc_3d(P, f, en, de, uc, vc, wc, i, j, k);
        }
        F6T<Real> h = {0, 0, 0, 0, 0, 0};
        bool visc = ph == 0 ? P.gas_viscosity : P.part_viscosity;
        if (visc) {
            S3T<Real> ka, ep, te;
            if (ph == 0) {
                first_nb3(ka, P.iturb ? F.kapgt : F.kapg, R, M);
                first_nb3(ep, F.ep, R, M);
                first_nb3(te, F.tg, R, M);
            } else {
                Real kk = P.kap[ph], ir = P.inrl[ph];
                ka.c = ka.e = ka.w = ka.n = ka.s = ka.t = ka.b = kk;
                ep.c = ir * de.c; ep.e = ir * de.e; ep.w = ir * de.w; ep.n = ir * de.n; ep.s = ir * de.s;
                ep.t = ir * de.t; ep.b = ir * de.b;
                first_nb3(te, F.ts + off, R, M);
            }
            hotc_3d(P, h, hw, hs, hb, ep, te, ka, i, j, k);
        }
        if (GRAV) {
            fE[c] = f.e - h.e + DE[c] * P.gravx * uc;
            fT[c] = f.t - h.t + DE[c] * P.gravz * wc;
            fN[c] = f.n - h.n + DE[c] * P.gravy * vc;
        } else {
            fE[c] = f.e - h.e;
            fT[c] = f.t - h.t;
            fN[c] = f.n - h.n;
        }
        // W/S/B faces towards non-fluid cells (a non-fluid flag is never 1,
        // so hotc has produced the conductive part there)
        if (dw) fE[R.w] = f.w - h.w;
        if (ds) fN[R.s] = f.s - h.s;
        if (db) fT[R.b] = f.b - h.b;
    }
}

__global__ void k_htilde3d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    int imjk = at3(P, max(i - 1, 1), j, k), ijmk = at3(P, i, max(j - 1, 1), k), ijkm = at3(P, i, j, max(k - 1, 1));
    const CellFaces b = cell_faces(P, c);
    double egfx = b.e * F.egfe[c] - b.w * F.egfe[imjk];
    double egfz = b.t * F.egft[c] - b.b * F.egft[ijkm];
    double egfy = b.n * F.egfn[c] - b.s * F.egfn[ijmk];
    double flx = dt * P.indx[i] * egfx * 1.0 + dt * P.indy[j] * egfy + dt * P.indz[k] * egfz;
    flx = flx * b.ivf;
    F.rhg[c] = -flx;
    for (int is = 1; is <= P.ns; ++is) {
        double ex, ez, ey;
        if (SOL(F.rlk, imjk, is) * P.inrl[is] <= 1.0e-9) ex = b.e * SOL(F.esfe, c, is);
        else ex = b.e * SOL(F.esfe, c, is) - b.w * SOL(F.esfe, imjk, is);
        if (SOL(F.rlk, ijkm, is) * P.inrl[is] <= 1.0e-9) ez = b.t * SOL(F.esft, c, is);
        else ez = b.t * SOL(F.esft, c, is) - b.b * SOL(F.esft, ijkm, is);
        if (SOL(F.rlk, ijmk, is) * P.inrl[is] <= 1.0e-9) ey = b.n * SOL(F.esfn, c, is);
        else ey = b.n * SOL(F.esfn, c, is) - b.s * SOL(F.esfn, ijmk, is);
        flx = dt * P.indx[i] * ex * 1.0 + dt * P.indy[j] * ey + dt * P.indz[k] * ez;
        flx = flx * b.ivf;
        SOL(F.rhs, c, is) = -flx + SOL(F.sink, c, is) * dt * b.ivf * SOL(F.sies, c, is);
    }
}

// ---------------------------------------------------------------------------
// ftem, ftem.f:19-248 (3D)
// ---------------------------------------------------------------------------
__global__ void k_ftem3d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    Rem3 M;
    raw3(P, i, j, k, R);
    rem3(P, i, j, k, R, M);
    const double *dx = P.dx, *dy = P.dy, *dz = P.dz;
    int ns = P.ns, nph = P.nph;
    double alpha = P.alpha;
    int imjk = R.w, ijmk = R.s, ijkm = R.b;
    double indxc = 1.0 / (dx[i] + (dx[i + 1] + dx[i - 1]) * 0.5);
    double indzc = 1.0 / (dz[k] + (dz[k + 1] + dz[k - 1]) * 0.5);
    const CellFaces bf = cell_faces(P, c);
    double ugc = 0.5 * (bf.e * F.ug[c] + bf.w * F.ug[imjk]);
    double wgc = 0.5 * (bf.t * F.wg[c] + bf.b * F.wg[ijkm]);
    double indyc = 1.0 / (dy[j] + (dy[j + 1] + dy[j - 1]) * 0.5);
    double vgc = 0.5 * (bf.n * F.vg[c] + bf.s * F.vg[ijmk]);
    double dpxyz = 0.0;
    dpxyz = dpxyz + dt * indxc * ugc * (F.p[M.e] - F.p[M.w]);
    dpxyz = dpxyz + dt * indyc * vgc * (F.p[M.n] - F.p[M.s]);
    dpxyz = dpxyz + dt * indzc * wgc * (F.p[M.t] - F.p[M.b]);
    double deltap = F.ep[c] * (F.p[c] - F.pn[c] + dpxyz);
    double workg = F.rgp[c] * (F.ug[c] * P.gravx + F.wg[c] * P.gravz);
    workg = workg + F.vg[c] * P.gravy;  // ftem.f:120 adds the y term without the density factor
    double at[PDAC_MAXP + 1][PDAC_MAXP + 1], bt[PDAC_MAXP + 1];
    at[1][1] = F.rgp[c];
    bt[1] = F.siegn[c] * F.rgpn[c] + F.rhg[c] + deltap + workg - 0.0;
    double cgc = F.cg[c];
    for (int is = 1; is <= ns; ++is) {
        int is1 = is + 1;
        double dugs = ((F.ug[c] - SOL(F.us, c, is)) + (F.ug[imjk] - SOL(F.us, imjk, is))) * 0.5;
        double dwgs = ((F.wg[c] - SOL(F.ws, c, is)) + (F.wg[ijkm] - SOL(F.ws, ijkm, is))) * 0.5;
        double dvgs = ((F.vg[c] - SOL(F.vs, c, is)) + (F.vg[ijmk] - SOL(F.vs, ijmk, is))) * 0.5;
        double hv = hvs(P, SOL(F.rlk, c, is), F.rog[c], dugs, dvgs, dwgs, F.mug[c], F.kapg[c], cgc, is);
        double works = SOL(F.rlk, c, is) * (SOL(F.us, c, is) * P.gravx + SOL(F.ws, c, is) * P.gravz);
        works = works + SOL(F.vs, c, is) * P.gravy;
        double ck = P.cps[is];
        at[1][1] = at[1][1] + alpha * dt * hv / cgc;
        at[1][is1] = -alpha * dt * hv / ck;
        at[is1][1] = -alpha * dt * hv / cgc;
        at[is1][is1] = SOL(F.rlk, c, is) + alpha * dt * hv / ck;
        bt[1] = bt[1] + (1.0 - alpha) * dt * hv * SOL(F.ts, c, is) - (1.0 - alpha) * dt * hv * F.tg[c];
        bt[is1] = SOL(F.rlkn, c, is) * SOL(F.siesn, c, is) + SOL(F.rhs, c, is) + works +
                  (1.0 - alpha) * dt * hv * F.tg[c] - (1.0 - alpha) * dt * hv * SOL(F.ts, c, is);
    }
    for (int is = nph; is >= 2; --is) {
        if (fabs(at[is][is]) < P.flim) {
            at[1][is] = 0.0; at[is][1] = 0.0; bt[is] = 0.0;
        } else {
            double div = 1.0 / at[is][is];
            at[is][1] = at[is][1] * div;
            bt[is] = bt[is] * div;
            bt[1] = bt[1] - at[1][is] * bt[is];
            at[1][1] = at[1][1] - at[1][is] * at[is][1];
        }
    }
    bt[1] = bt[1] / at[1][1];
    for (int is = 2; is <= nph; ++is) bt[is] = bt[is] - at[is][1] * bt[1];
    F.sieg[c] = bt[1];
    for (int is = 1; is <= ns; ++is) SOL(F.sies, c, is) = bt[is + 1];
    double yg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) yg[ig] = GAS(F.ygc, c, ig);
    double tg = F.tg[c], cg;
    int info = caloric_eosg(P, cg, tg, yg, bt[1]);
    F.tg[c] = tg;
    F.cg[c] = cg;
    for (int is = 1; is <= ns; ++is) {
        double t = 0.0 + (bt[is + 1] - 0.0) / P.cps[is];
        SOL(F.ts, c, is) = t;
        if (t < 0.0) info++;
    }
    if (info) atomicAdd(&F.counters[1], info);
}

}  // namespace pdac

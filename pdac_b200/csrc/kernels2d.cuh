// kernels2d.cuh -- CUDA kernels of the 2D semi-implicit time step.
//
// One thread per cell.  The explicit passes (boundary, fieldn, tilde,
// ygas, htilde, ftem) are order independent: each face value is produced by
// exactly one owner thread with the rule the reference's lexicographic loop
// implies.  The implicit corrector (iter.f:204-410) runs as three colour
// phases per outer sweep, colour = (i + j + k) mod 3 (1-based indices, j = 1
// in 2D): every read and write of a cell's in-cell solve lies in the axis
// cross of radius 2 around it, and two cells of one colour are never within
// that cross of each other, so a phase is race free and equals a
// Gauss-Seidel sweep in colour-major order.
#pragma once
#include "solve.cuh"

namespace pdac {

__device__ __forceinline__ bool fluid(const Prm &P, int c) { return (P.flag[c] & 1) != 0; }
#define SOL(a, c, is) (a)[(size_t)((is) - 1) * P.ncell + (c)]
#define GAS(a, c, ig) (a)[(size_t)(ig) * P.ncell + (c)]
#define APP(a, c, ls) (a)[(size_t)((ls) - 1) * P.ncell + (c)]

// ---------------------------------------------------------------------------
// vent velocity fluctuations, vent.f:902-936
// ---------------------------------------------------------------------------
__global__ void k_vent(Prm P, Fld F, const int *vent, int nvent, double *fact, double *fact0) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nvent) return;
    int c = vent[q];
    double intensity = 0.01;
    double rann = fact[q] * intensity, ranold = fact0[q] * intensity;
    fact0[q] = fact[q];
    F.ug[c] = F.ug[c] * (1.0 + rann) / (1.0 + ranold);
    if (P.d3) F.vg[c] = F.vg[c] * (1.0 + rann) / (1.0 + ranold);
    F.wg[c] = F.wg[c] * (1.0 + rann) / (1.0 + ranold);
    for (int is = 1; is <= P.ns; ++is) {
        SOL(F.us, c, is) = SOL(F.us, c, is) * (1.0 + rann) / (1.0 + ranold);
        if (P.d3) SOL(F.vs, c, is) = SOL(F.vs, c, is) * (1.0 + rann) / (1.0 + ranold);
        SOL(F.ws, c, is) = SOL(F.ws, c, is) * (1.0 + rann) / (1.0 + ranold);
    }
}

// ---------------------------------------------------------------------------
// boundary, bdry.f:22-726 + inoutflow.f:1-126 (2D)
// ---------------------------------------------------------------------------
__device__ void inoutflow_d(const Prm &P, const Fld &F, double ugv, const double *usv, int n2, int n1, int k, double gnorm) {
    int sgn = (n2 - n1) >= 0 ? 1 : -1;
    if (ugv * sgn > 0.0) {
        F.tg[n2] = F.tg[n1];
        F.sieg[n2] = F.sieg[n1];
        for (int ig = 0; ig < P.ng; ++ig) { GAS(F.ygc, n2, ig) = GAS(F.ygc, n1, ig); GAS(F.xgc, n2, ig) = GAS(F.xgc, n1, ig); }
        F.rog[n2] = F.rog[n1];
    } else if (ugv * sgn <= 0.0) {
        F.tg[n2] = P.t_atm[k];
        double yg[PDAC_MAXG], xg[PDAC_MAXG];
        for (int ig = 0; ig < P.ng; ++ig) { yg[ig] = P.atm_ygc[P.gas_type[ig] - 1]; GAS(F.ygc, n2, ig) = yg[ig]; }
        mole(P, xg, yg);
        for (int ig = 0; ig < P.ng; ++ig) GAS(F.xgc, n2, ig) = xg[ig];
        F.rog[n2] = thermal_eosg(P, P.t_atm[k], P.p_atm[k], xg);
    }
    double rls = 0.0;
    for (int is = 1; is <= P.ns; ++is) {
        if (usv[is] * sgn > 0.0) {
            SOL(F.rlk, n2, is) = SOL(F.rlk, n1, is);
            SOL(F.ts, n2, is) = SOL(F.ts, n1, is);
            SOL(F.sies, n2, is) = SOL(F.sies, n1, is);
        } else if (usv[is] * sgn <= 0.0) {
            SOL(F.rlk, n2, is) = P.rl[is] * (1.0 - P.void_fraction) / P.ns;
            SOL(F.ts, n2, is) = P.t_atm[k];
        }
        rls = rls + SOL(F.rlk, n2, is) * P.inrl[is];
    }
    F.ep[n2] = 1.0 - rls;
    F.rgp[n2] = F.rog[n2] * F.ep[n2];
    double rhomix = F.rgp[n2];
    if (P.pmodel == 1)
        for (int is = 1; is <= P.ns; ++is) rhomix = rhomix + SOL(F.rlk, n2, is);
    if (rls >= 1.0) atomicAdd(&F.counters[3], 1);
    F.p[n2] = F.p[n1] + rhomix * gnorm;
}

__device__ void zerograd_d(const Prm &P, const Fld &F, int n2, int n1) {
    F.tg[n2] = F.tg[n1];
    F.sieg[n2] = F.sieg[n1];
    for (int ig = 0; ig < P.ng; ++ig) { GAS(F.ygc, n2, ig) = GAS(F.ygc, n1, ig); GAS(F.xgc, n2, ig) = GAS(F.xgc, n1, ig); }
    F.rog[n2] = F.rog[n1];
    double rls = 0.0;
    for (int is = 1; is <= P.ns; ++is) {
        SOL(F.rlk, n2, is) = SOL(F.rlk, n1, is);
        SOL(F.ts, n2, is) = SOL(F.ts, n1, is);
        SOL(F.sies, n2, is) = SOL(F.sies, n1, is);
        rls = rls + SOL(F.rlk, n2, is) * P.inrl[is];
    }
    F.ep[n2] = 1.0 - rls;
    F.rgp[n2] = F.rog[n2] * F.ep[n2];
    if (rls >= 1.0) atomicAdd(&F.counters[3], 1);
    F.p[n2] = F.p[n1];
}

__device__ void boundary_cell2d(const Prm &P, const Fld &F, int c) {
    int f0 = P.flag[c];
    if (!(f0 == FLUID || f0 == DOME || f0 == BL_CELL)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    raw2(P, i, k, R);
    const int *fl = P.flag;
    // bdry.f acts only through neighbours that are walls or open boundaries
    auto acts = [](int f) { return f == SLIP || f == NOSLIP || f == FREE_IO || f == ZERO_GRAD; };
    if (!acts(fl[R.e]) && !acts(fl[R.w]) && !acts(fl[R.t]) && !acts(fl[R.b])) return;
    double usv[PDAC_MAXP];
    int ns = P.ns;
    // East
    {
        int n2 = R.e, n1 = c, n0 = R.w, f2 = fl[n2];
        if (f2 == SLIP || f2 == NOSLIP) {
            F.ug[n1] = 0; F.ug[n2] = 0;
            for (int is = 1; is <= ns; ++is) { SOL(F.us, n1, is) = 0; SOL(F.us, n2, is) = 0; }
            if (f2 == SLIP) {
                F.wg[n2] = F.wg[n1];
                for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = SOL(F.ws, n1, is);
            } else if (!(fl[R.et] & 1)) {
                F.wg[n2] = -F.wg[n1];
                for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = -SOL(F.ws, n1, is);
            }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.ug[n1] = F.ug[n0];
            for (int is = 1; is <= ns; ++is) SOL(F.us, n1, is) = SOL(F.us, n0, is);
            F.ug[n2] = F.ug[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = SOL(F.us, n1, is);
            F.wg[n2] = F.wg[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = SOL(F.ws, n1, is);
            double gnorm = P.gravx * 0.5 * (P.dx[i + 1] + P.dx[i]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.us, n1, is);
            inoutflow_d(P, F, F.ug[n1], usv, n2, n1, k, gnorm);
        }
    }
    // West
    {
        int n2 = R.w, n1 = c, f2 = fl[n2];
        if (f2 == SLIP) {
            F.ug[n2] = 0;
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = 0;
            F.wg[n2] = F.wg[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = SOL(F.ws, n1, is);
        } else if (f2 == NOSLIP) {
            F.ug[n2] = 0;
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = 0;
            if (!(fl[R.wt] & 1)) {
                F.wg[n2] = -F.wg[n1];
                for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = -SOL(F.ws, n1, is);
            }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.ug[n2] = F.ug[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = SOL(F.us, n1, is);
            F.wg[n2] = F.wg[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = SOL(F.ws, n1, is);
            double gnorm = P.gravx * 0.5 * (P.dx[i - 1] + P.dx[i]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.us, n2, is);
            inoutflow_d(P, F, F.ug[n2], usv, n2, n1, k, gnorm);
        }
    }
    // Top
    {
        int n2 = R.t, n1 = c, f2 = fl[n2];
        if (f2 == SLIP) {
            F.wg[n1] = 0;
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n1, is) = 0;
            F.ug[n2] = F.ug[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = SOL(F.us, n1, is);
        } else if (f2 == NOSLIP) {
            F.wg[n1] = 0;
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n1, is) = 0;
            if (!(fl[R.et] & 1)) {
                F.ug[n2] = -F.ug[n1];
                for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = -SOL(F.us, n1, is);
            }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            double d0 = P.dz[k - 1], d1 = P.dz[k], d2 = P.dz[k + 1];
            const int ord = 0;
            F.ug[n2] = F.ug[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = SOL(F.us, n1, is);
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
    // Bottom
    {
        int n1 = c, n2 = R.b, f2 = fl[n2];
        if (f2 == SLIP) {
            F.wg[n2] = 0;
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = 0;
            if (fl[R.eb] == SLIP) {
                F.ug[n2] = F.ug[n1];
                for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = SOL(F.us, n1, is);
            }
        } else if (f2 == NOSLIP) {
            F.wg[n2] = 0;
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = 0;
            if (fl[R.eb] == NOSLIP) {
                F.ug[n2] = -F.ug[n1];
                for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = -SOL(F.us, n1, is);
            }
        } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
            F.wg[n2] = F.wg[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.ws, n2, is) = SOL(F.ws, n1, is);
            F.ug[n2] = F.ug[n1];
            for (int is = 1; is <= ns; ++is) SOL(F.us, n2, is) = SOL(F.us, n1, is);
            double gnorm = P.gravz * 0.5 * (P.dz[k - 1] + P.dz[k]);
            if (f2 == ZERO_GRAD) gnorm = 0.0;
            for (int is = 1; is <= ns; ++is) usv[is] = SOL(F.ws, n2, is);
            inoutflow_d(P, F, F.wg[n2], usv, n2, n1, k - 1, gnorm);
        }
    }
}

// the boundary pass (bdry.f:22-726) with one thread per cell, for meshes on
// which no two cells' boundary updates touch the same cell
__global__ void k_boundary2d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < P.ncell) boundary_cell2d(P, F, c);
}

// ---------------------------------------------------------------------------
// fieldn, tilde.f:125-274 (2D), with viscon (visc.f:37-148)
// ---------------------------------------------------------------------------
__global__ void k_fieldn2d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    bool interior = i >= 2 && i <= P.nx - 1 && k >= 2 && k <= P.nz - 1;
    if (interior) {
        Raw2 R;
        raw2(P, i, k, R);
        int ijke = is_wallf(P.flag[R.e]) ? c : R.e;
        int ijkt = is_wallf(P.flag[R.t]) ? c : R.t;
        const double *dx = P.dx, *dz = P.dz;
        double indxp = P.hx[i], indzp = P.hz[k];
        double rgp_e = (dx[i + 1] * F.rgp[c] + dx[i] * F.rgp[ijke]) * indxp;
        double rgp_t = (dz[k + 1] * F.rgp[c] + dz[k] * F.rgp[ijkt]) * indzp;
        F.rugn[c] = rgp_e * F.ug[c];
        F.rwgn[c] = rgp_t * F.wg[c];
        for (int is = 1; is <= P.ns; ++is) {
            double rlk_e = (SOL(F.rlk, c, is) * dx[i + 1] + SOL(F.rlk, ijke, is) * dx[i]) * indxp;
            double rlk_t = (SOL(F.rlk, c, is) * dz[k + 1] + SOL(F.rlk, ijkt, is) * dz[k]) * indzp;
            SOL(F.rusn, c, is) = rlk_e * SOL(F.us, c, is);
            SOL(F.rwsn, c, is) = rlk_t * SOL(F.ws, c, is);
        }
    } else {
        F.rugn[c] = 0; F.rwgn[c] = 0;
        for (int is = 1; is <= P.ns; ++is) { SOL(F.rusn, c, is) = 0; SOL(F.rwsn, c, is) = 0; }
    }
    F.pn[c] = F.p[c];
    F.epn[c] = F.ep[c];
    F.rgpn[c] = F.rgp[c];
    F.siegn[c] = F.sieg[c];
    for (int ig = 0; ig < P.ng; ++ig) GAS(F.rgpgcn, c, ig) = F.rgpn[c] * GAS(F.ygc, c, ig);
    for (int is = 1; is <= P.ns; ++is) {
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
// tilde fluxes, compute_all_fluxes_tilde tilde.f:850-1326 (2D)
// ---------------------------------------------------------------------------
// Real: the arithmetic of the face fluxes (float in PDAC_PREC_MIXED; the
// stencil values are the FP64 state rounded once, the fluxes stored in FP64)
template <typename Real = double>
__global__ void k_tilde_flux2d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    bool dow = !fluid(P, R.w), dob = !fluid(P, R.b);
    bool mus = P.muscl > 0 && P.flag[c] == FLUID;
    for (int ph = 0; ph <= P.ns; ++ph) {
        const double *U = ph == 0 ? F.ug : F.us + (size_t)(ph - 1) * P.ncell;
        const double *W = ph == 0 ? F.wg : F.ws + (size_t)(ph - 1) * P.ncell;
        const double *D = ph == 0 ? F.rgp : F.rlk + (size_t)(ph - 1) * P.ncell;
        double *fue = ph == 0 ? F.ugfe : F.usfe + (size_t)(ph - 1) * P.ncell;
        double *fut = ph == 0 ? F.ugft : F.usft + (size_t)(ph - 1) * P.ncell;
        double *fwe = ph == 0 ? F.wgfe : F.wsfe + (size_t)(ph - 1) * P.ncell;
        double *fwt = ph == 0 ? F.wgft : F.wsft + (size_t)(ph - 1) * P.ncell;
        St2T<Real> u, w, d, dsx, dsz;
        rnb2(u, U, R);
        rnb2(w, W, R);
        if (ib_masked(P, c)) { ib_mask2(P, u, R, 1); ib_mask2(P, w, R, 4); }
        nb2(d, D, R, M);
        interp_x2(P, d, i, dsx);
        interp_z2(P, d, k, dsz);
        Real ue = 0, ut = 0, uw = 0, ub = 0, we = 0, wt = 0, ww = 0, wb = 0;
        flu_2d(P, ue, ut, uw, ub, dow, dob, dsx, u, w, i);
        flw_2d(P, we, wt, ww, wb, dow, dob, dsz, u, w, i, k);
        if (mus) {
            muscl_flu_2d(P, ue, ut, dsx, u, w, i, k, i != P.nx - 1, i != P.nx - 1);
            muscl_flw_2d(P, we, wt, dsz, u, w, i, k, k != P.nz - 1, k != P.nz - 1);
        }
        fue[c] = ue; fut[c] = ut; fwe[c] = we; fwt[c] = wt;
        if (dow) { fue[R.w] = uw; fwe[R.w] = ww; }
        if (dob) { fut[R.b] = ub; fwt[R.b] = wb; }
    }
}

// stress2D, visc.f:561-696, for one cell; mu/lambda/eps accessors
template <typename MU, typename LAM, typename EPS>
__device__ __forceinline__ void stress2d_cell(const Prm &P, const Raw2 &R, const Rem2 &M, int i, int k, MU mu, LAM lam, EPS eps,
                                              const double *u, const double *w, double &visx, double &visz) {
    const double *dx = P.dx, *dz = P.dz, *indx = P.indx, *indz = P.indz, *r = P.r, *rb = P.rb, *inr = P.inr, *inrb = P.inrb;
    const double cm = 2.0 / 3.0;
    int c = R.c;
    double indxp = P.hx[i], indxm = P.hx[i - 1];
    double indzp = P.hz[k], indzm = P.hz[k - 1];
    double divr = ((rb[i + 1] * u[R.e] - rb[i] * u[c]) * inr[i + 1] * indx[i + 1] + (w[R.e] - w[R.eb]) * indz[k]);
    double divc = ((rb[i] * u[c] - rb[i - 1] * u[R.w]) * inr[i] * indx[i] + (w[c] - w[R.b]) * indz[k]);
    double divt = ((rb[i] * u[R.t] - rb[i - 1] * u[R.wt]) * inr[i] * indx[i] + (w[R.t] - w[c]) * indz[k + 1]);
    double txx2 = 2.0 * (u[R.e] - u[c]) * indx[i + 1];
    double txx1 = 2.0 * (u[c] - u[R.w]) * indx[i];
    double tyy2 = 2.0 * (w[R.t] - w[c]) * indz[k + 1];
    double tyy1 = 2.0 * (w[c] - w[R.b]) * indz[k];
    txx2 = mu(M.e) * txx2 - cm * lam(M.e) * divr;
    txx1 = mu(c) * txx1 - cm * lam(c) * divc;
    tyy2 = mu(M.t) * tyy2 - cm * lam(M.t) * divt;
    tyy1 = mu(c) * tyy1 - cm * lam(c) * divc;
    double tyx2 = (u[R.t] - u[c]) * indzp * 2.0 + (w[R.e] - w[c]) * indxp * 2.0;
    double tyx1 = (u[c] - u[R.b]) * indzm * 2.0 + (w[R.eb] - w[R.b]) * indxp * 2.0;
    double txy2 = tyx2;
    double txy1 = (u[R.wt] - u[R.w]) * indzp * 2.0 + (w[c] - w[R.w]) * indxm * 2.0;
    double t0 = 0.0, eps0 = 0.0;
    if (P.itc == 1) {
        eps0 = (eps(c) * dx[i + 1] + eps(M.e) * dx[i]) * indxp;
        double mu0 = (mu(c) * dx[i + 1] + mu(M.e) * dx[i]) * indxp;
        double lambda0 = (lam(c) * dx[i + 1] + lam(M.e) * dx[i]) * indxp;
        t0 = 2.0 * u[c] * inrb[i];
        double du = (rb[i + 1] * u[R.e] - rb[i - 1] * u[R.w]);
        double wm2 = (dx[i] * w[R.e] + dx[i + 1] * w[c]) * indxp;
        double wm1 = (dx[i] * w[R.eb] + dx[i + 1] * w[R.b]) * indxp;
        double dw = wm2 - wm1;
        double dive = (inrb[i] * du * indxp + dw * indz[k]);
        t0 = mu0 * t0 - cm * lambda0 * dive;
    }
    double epsmu21 = (dz[k] * eps(M.t) * mu(M.t) + dz[k + 1] * eps(c) * mu(c)) * indzp;
    double epsmu22 = (dz[k] * eps(M.et) * mu(M.et) + dz[k + 1] * eps(M.e) * mu(M.e)) * indzp;
    double epsmu2 = (dx[i + 1] * epsmu21 + dx[i] * epsmu22) * indxp;
    double epsmu11 = (dz[k - 1] * eps(c) * mu(c) + dz[k] * eps(M.b) * mu(M.b)) * indzm;
    double epsmu12 = (dz[k - 1] * eps(M.e) * mu(M.e) + dz[k] * eps(M.eb) * mu(M.eb)) * indzm;
    double epsmu1 = (dx[i + 1] * epsmu11 + dx[i] * epsmu12) * indxp;
    double gradxx = (eps(M.e) * txx2 * r[i + 1] - eps(c) * txx1 * r[i]);
    gradxx = gradxx * indxp * 2.0 * inrb[i];
    double gradyx = (epsmu2 * tyx2 - epsmu1 * tyx1);
    gradyx = gradyx * indz[k];
    visx = gradxx + gradyx - eps0 * t0 * inrb[i];
    epsmu11 = (dz[k] * eps(M.wt) * mu(M.wt) + dz[k + 1] * eps(M.w) * mu(M.w)) * indzp;
    epsmu1 = (dx[i] * epsmu11 + dx[i - 1] * epsmu21) * indxm;
    double gradyy = (eps(M.t) * tyy2 - eps(c) * tyy1);
    gradyy = gradyy * indzp * 2.0;
    double gradxy = (rb[i] * epsmu2 * txy2 - rb[i - 1] * epsmu1 * txy1);
    gradxy = gradxy * inr[i] * indx[i];
    visz = gradyy + gradxy;
}

// The forcing terms of tilde's mesh loop at a forcing point of cell c along
// `axis` (0 x, 1 y, 2 z), tilde.f:708-801: the momentum that brings the face
// velocity to the forcing point's value (the interpolated no-slip velocity
// of the last boundary pass) in one step, less the pressure and drag terms
// the corrector adds back.  nb is the remapped plus-side neighbour, nm the
// raw minus-side one (the cell-centre relative velocities dugs, dvgs, dwgs
// of tilde.f:597-612 are recomputed from it), dm and dp the cell sizes d(i)
// and d(i+1) of the axis, inv = 1 / (dm + dp).
__device__ __forceinline__ void ib_force(const Prm &P, const Fld &F, int c, int axis, int nb, int nm, double dm,
                                         double dp, double inv, double dt, const double *kpgv, double &rg,
                                         double *rs) {
    const int f = __ldg(P.ib_num[axis] + c);
    if (f == 0) return;
    const double *vel = P.ib_vel[axis] + (size_t)(f - 1) * P.nph;
    const double *G = axis == 0 ? F.ug : (axis == 1 ? F.vg : F.wg);
    const double *S = axis == 0 ? F.us : (axis == 1 ? F.vs : F.ws);
    const int ns = P.ns;
    auto dgs = [&](int is) { return ((G[c] - SOL(S, c, is)) + (G[nm] - SOL(S, nm, is))) * 0.5; };
    double pseudo = vel[0];
    double force = (inv * (dp * F.rgp[c] + dm * F.rgp[nb]) * pseudo - rg) / dt;
    double ep_e = (dm * F.ep[nb] + dp * F.ep[c]) * inv;
    double presn = -inv * 2.0 * ep_e * (F.p[nb] - F.p[c]);
    double dragn = 0.0;
    for (int is = 1; is <= ns; ++is) dragn = dragn - kpgv[is] * dgs(is);
    force = force - presn - dragn;
    rg = rg + dt * force;
    for (int is = 1; is <= ns; ++is) {
        pseudo = vel[is];
        force = (inv * (dp * SOL(F.rlk, c, is) + dm * SOL(F.rlk, nb, is)) * pseudo - rs[is]) / dt;
        ep_e = (dm * SOL(F.rlk, nb, is) + dp * SOL(F.rlk, c, is)) * inv * P.inrl[is];
        presn = -inv * 2.0 * ep_e * (F.p[nb] - F.p[c]);
        dragn = kpgv[is] * dgs(is);
        force = force - presn - dragn;
        rs[is] = rs[is] + dt * force;
    }
}

// tilde mesh loop, tilde.f:418-806 (2D), with viscg/viscs (visc.f:150-291),
// kdrags/sdrag and inter (drag.f:11-298).  app0 holds the interphase matrix
// of the previous visit of each cell in this step (zero at step start); it is
// read only when alpha < 1.
__global__ void k_tilde2d(Prm P, Fld F, double dt, const double *app0u, const double *app0w) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    const double *dx = P.dx, *dz = P.dz, *indx = P.indx, *indz = P.indz, *inr = P.inr, *inrb = P.inrb;
    int n = P.ncell, ns = P.ns;
    int imjk = R.w, ijkm = R.b, ijke = M.e, ijkt = M.t;
    // viscous stresses
    double gvx = 0, gvz = 0;
    if (P.gas_viscosity) {
        // viscg: mu = mugt (the sub-grid model's, molecular part added) or mug, lambda = mug
        const double *mug = F.mug, *mut = P.iturb ? F.mugt : F.mug, *ep = F.ep;
        stress2d_cell(P, R, M, i, k, [&](int q) { return mut[q]; }, [&](int q) { return mug[q]; },
                      [&](int q) { return ep[q]; }, F.ug, F.wg, gvx, gvz);
    }
    double alpha = P.alpha, ag = P.alphagrav;
    double dxi = dx[i], dxip1 = dx[i + 1], dzk = dz[k], dzkp1 = dz[k + 1];
    double indxp = P.hx[i], indzp = P.hz[k];
    double ugfx = F.ugfe[c] - F.ugfe[imjk], ugfz = F.ugft[c] - F.ugft[ijkm];
    double wgfx = F.wgfe[c] - F.wgfe[imjk], wgfz = F.wgft[c] - F.wgft[ijkm];
    double epn_e = 1.0, epn_t = 1.0;
    if (P.pmodel == 1) {
        epn_e = (dxi * F.epn[ijke] + dxip1 * F.epn[c]) * indxp;
        epn_t = (dzk * F.epn[ijkt] + dzkp1 * F.epn[c]) * indzp;
    }
    double t_ = gvx;
    t_ = t_ - indxp * 2.0 * ugfx * inrb[i];
    t_ = t_ + (1.0 - ag) * (dx[i + 1] * F.rgpn[c] + dx[i] * F.rgpn[ijke]) * indxp * P.gravx;
    t_ = t_ - indz[k] * ugfz;
    t_ = t_ + (1.0 - alpha) * indxp * 2.0 * epn_e * (F.pn[c] - F.pn[ijke]);
    double rug = F.rugn[c] + dt * t_;
    t_ = gvz;
    t_ = t_ + (1.0 - ag) * (dz[k + 1] * F.rgpn[c] + dz[k] * F.rgpn[ijkt]) * indzp * P.gravz;
    t_ = t_ - indx[i] * wgfx * inr[i];
    t_ = t_ - indzp * 2.0 * wgfz;
    t_ = t_ + (1.0 - alpha) * indzp * 2.0 * epn_t * (F.pn[c] - F.pn[ijkt]);
    double rwg = F.rwgn[c] + dt * t_;
    double rus[PDAC_MAXP], rws[PDAC_MAXP], kpgv[PDAC_MAXP];
    const double a_rep = -8.76, b_rep = -0.27;
    for (int is = 1; is <= ns; ++is) {
        double pvx = 0, pvz = 0;
        if (P.part_viscosity) {
            const double cm = P.cmus[is], ir = P.inrl[is];
            const double *rl = F.rlk + (size_t)(is - 1) * n;
            const double *mst = P.iss ? F.must + (size_t)(is - 1) * n : nullptr;
            stress2d_cell(P, R, M, i, k, [&](int q) { return mst ? mst[q] : cm; }, [&](int) { return cm; },
                          [&](int q) { return rl[q] * ir; },
                          F.us + (size_t)(is - 1) * n, F.ws + (size_t)(is - 1) * n, pvx, pvz);
            if (P.repulsive_model == 1) {
                double rc = rl[c], re = rl[ijke], rt = rl[ijkt];
                double epsx = (dx[i + 1] * rc + dx[i] * re) * indxp * ir;
                double gepx = pdac_fp::pow(10.0, -a_rep * epsx + b_rep);
                pvx = pvx - gepx * indxp * 2.0 * (re - rc) * ir;
                double epsz = (dz[k + 1] * rc + dz[k] * rt) * indzp * ir;
                double gepz = pdac_fp::pow(10.0, -a_rep * epsz + b_rep);
                pvz = pvz - gepz * indzp * 2.0 * (rt - rc) * ir;
            }
        }
        double usfx = SOL(F.usfe, c, is) - SOL(F.usfe, imjk, is), usfz = SOL(F.usft, c, is) - SOL(F.usft, ijkm, is);
        double wsfx = SOL(F.wsfe, c, is) - SOL(F.wsfe, imjk, is), wsfz = SOL(F.wsft, c, is) - SOL(F.wsft, ijkm, is);
        double epsn_e = 0, epsn_t = 0;
        if (P.pmodel == 1) {
            epsn_e = (dxi * SOL(F.rlkn, ijke, is) + dxip1 * SOL(F.rlkn, c, is)) * indxp * P.inrl[is];
            epsn_t = (dzk * SOL(F.rlkn, ijkt, is) + dzkp1 * SOL(F.rlkn, c, is)) * indzp * P.inrl[is];
        }
        double r_ = pvx;
        r_ = r_ - indxp * 2.0 * usfx * inrb[i];
        r_ = r_ + (1.0 - ag) * indxp * P.gravx * (dx[i + 1] * SOL(F.rlkn, c, is) + dx[i] * SOL(F.rlkn, ijke, is));
        r_ = r_ - indz[k] * usfz;
        r_ = r_ + (1.0 - alpha) * indxp * 2.0 * epsn_e * (F.pn[c] - F.pn[ijke]);
        rus[is] = SOL(F.rusn, c, is) + dt * r_;
        rus[is] = rus[is] + dt * SOL(F.sink, c, is) * SOL(F.us, c, is);
        r_ = pvz;
        r_ = r_ + (1.0 - ag) * indzp * P.gravz * (SOL(F.rlkn, c, is) * dz[k + 1] + SOL(F.rlkn, ijkt, is) * dz[k]);
        r_ = r_ - indx[i] * wsfx * inr[i];
        r_ = r_ - indzp * 2.0 * wsfz;
        r_ = r_ + (1.0 - alpha) * indzp * 2.0 * epsn_t * (F.pn[c] - F.pn[ijkt]);
        rws[is] = SOL(F.rwsn, c, is) + dt * r_;
        rws[is] = rws[is] + dt * SOL(F.sink, c, is) * SOL(F.ws, c, is);
        double dugs = ((F.ug[c] - SOL(F.us, c, is)) + (F.ug[imjk] - SOL(F.us, imjk, is))) * 0.5;
        double dwgs = ((F.wg[c] - SOL(F.ws, c, is)) + (F.wg[ijkm] - SOL(F.ws, ijkm, is))) * 0.5;
        kpgv[is] = drag_coeff(P, dugs, 0.0, dwgs, F.ep[c], F.rgp[c], SOL(F.rlk, c, is), F.mug[c], is);
    }
    // inter, drag.f:173-246
    double au[PDAC_MAXP * (PDAC_MAXP + 1) / 2 + 1], aw[PDAC_MAXP * (PDAC_MAXP + 1) / 2 + 1];
    double rlkc[PDAC_MAXP];
    for (int is = 1; is <= ns; ++is) rlkc[is] = SOL(F.rlk, c, is);
    int ks = 0;
    for (int kk1 = 1; kk1 <= P.nph; ++kk1) {
        if (kk1 == 1) { ks++; au[ks] = 0; aw[ks] = 0; }
        else {
            for (int kk = 1; kk <= kk1; ++kk) {
                ks++;
                if (kk == 1) { au[ks] = -kpgv[kk1 - 1] * dt; aw[ks] = -kpgv[kk1 - 1] * dt; }
                else if (kk == kk1) { au[ks] = 0; aw[ks] = 0; }
                else {
                    double con = ppdrag(P, rlkc, kk1, kk);
                    double du = fabs(SOL(F.us, c, kk1 - 1) - SOL(F.us, c, kk - 1) + SOL(F.us, imjk, kk1 - 1) - SOL(F.us, imjk, kk - 1)) * 0.5;
                    double dw = fabs(SOL(F.ws, c, kk1 - 1) - SOL(F.ws, c, kk - 1) + SOL(F.ws, ijkm, kk1 - 1) - SOL(F.ws, ijkm, kk - 1)) * 0.5;
                    au[ks] = -(con * du) * dt;
                    aw[ks] = -(con * dw) * dt;
                }
            }
        }
    }
    for (int kk1 = 1; kk1 <= P.nph; ++kk1) {
        double sx = 0, sz = 0;
        for (int kk = 1; kk <= kk1; ++kk) { int q = kk + kk1 * (kk1 - 1) / 2; sx = sx + au[q]; sz = sz + aw[q]; }
        for (int kk = kk1; kk <= P.nph; ++kk) { int q = kk1 + kk * (kk - 1) / 2; sx = sx + au[q]; sz = sz + aw[q]; }
        int q = kk1 * (kk1 + 1) / 2;
        au[q] = -sx;
        aw[q] = -sz;
    }
    for (int q = 1; q <= P.nap; ++q) { APP(F.appu, c, q) = au[q]; APP(F.appw, c, q) = aw[q]; }
    // (1 - alpha) explicit interphase part, tilde.f:597-680
    if (alpha != 1.0) {
        auto AU = [&](int cell, int ls) { return cell == c ? au[ls] : APP(app0u, cell, ls); };
        auto AW = [&](int cell, int ls) { return cell == c ? aw[ls] : APP(app0w, cell, ls); };
        rug = rug - (1.0 - alpha) * (dxi * AU(ijke, 1) + dxip1 * AU(c, 1)) * indxp * F.ug[c];
        rwg = rwg - (1.0 - alpha) * (dzk * AW(ijkt, 1) + dzkp1 * AW(c, 1)) * indzp * F.wg[c];
        for (int l = 2; l <= P.nph; ++l) {
            int ls1 = l * (l - 1) / 2;
            for (int ll = 1; ll <= l; ++ll) {
                int ls = ls1 + ll;
                double fu = (1.0 - alpha) * (dxi * AU(ijke, ls) + dxip1 * AU(c, ls)) * indxp;
                double fw = (1.0 - alpha) * (dzk * AW(ijkt, ls) + dzkp1 * AW(c, ls)) * indzp;
                if (ll == 1) {
                    rug = rug - fu * SOL(F.us, c, l - 1);
                    rwg = rwg - fw * SOL(F.ws, c, l - 1);
                    rus[l - 1] = rus[l - 1] - fu * F.ug[c];
                    rws[l - 1] = rws[l - 1] - fw * F.wg[c];
                } else if (ll == l) {
                    rus[l - 1] = rus[l - 1] - fu * SOL(F.us, c, l - 1);
                    rws[l - 1] = rws[l - 1] - fw * SOL(F.ws, c, l - 1);
                } else {
                    rus[l - 1] = rus[l - 1] - fu * SOL(F.us, c, ll - 1);
                    rus[ll - 1] = rus[ll - 1] - fu * SOL(F.us, c, l - 1);
                    rws[l - 1] = rws[l - 1] - fw * SOL(F.ws, c, ll - 1);
                    rws[ll - 1] = rws[ll - 1] - fw * SOL(F.ws, c, l - 1);
                }
            }
        }
    }
    if (P.immb) {
        ib_force(P, F, c, 0, ijke, imjk, dx[i], dx[i + 1], 1.0 / (dx[i] + dx[i + 1]), dt, kpgv, rug, rus);
        ib_force(P, F, c, 2, ijkt, ijkm, dz[k], dz[k + 1], 1.0 / (dz[k] + dz[k + 1]), dt, kpgv, rwg, rws);
    }
    F.rug[c] = rug;
    F.rwg[c] = rwg;
    for (int is = 1; is <= ns; ++is) { SOL(F.rus, c, is) = rus[is]; SOL(F.rws, c, is) = rws[is]; }
}

// predictor, iter.f:135-145
template <int NP>
__global__ void k_predictor2d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    face_solve<NP>(P, F, c, M.e, R.e, i, 0, +1, dt);
    face_solve<NP>(P, F, c, M.t, R.t, k, 2, +1, dt);
}

// gas mass flux of one cell over its four faces (calc_gas_mass_flux,
// iter.f:597-740): densities remapped, velocities raw
__device__ __forceinline__ void cell_massflux(const Prm &P, const double *D, const double *U, const double *W,
                                              const Raw2 &R, const Rem2 &M, int i, int k, MF2 &f) {
    St d;
    first_nb2(d, D, R, M);
    bool mus = P.muscl > 0 && P.flag[R.c] == FLUID;
    if (mus) third_nb2(d, D, M);
    massflux_2d(P, d, U[R.w], U[R.c], W[R.b], W[R.c], i, k, mus, P.flag[R.w], P.flag[R.e], P.flag[R.b], P.flag[R.t], f);
}

// betas, iter.f:1112-1248
__device__ __forceinline__ void betas_2d(const Prm &P, const Fld &F, const Raw2 &R, const Rem2 &M, int i, int k, double dt,
                                         double &cnv, double &abt) {
    const double *dx = P.dx, *dz = P.dz;
    int c = R.c;
    double indxp = P.hx[i], indxm = P.hx[i - 1];
    double indzp = P.hz[k], indzm = P.hz[k - 1];
    auto open = [](int f) { return f == BL_CELL || f == FLUID || f == DOME || f == IMMB || f == FREE_IO || f == ZERO_GRAD; };
    double iep_e = open(P.flag[R.e]) ? (dx[i + 1] * F.ep[c] + dx[i] * F.ep[M.e]) * indxp * indxp * 2.0 : 0.0;
    double iep_w = open(P.flag[R.w]) ? (dx[i - 1] * F.ep[c] + dx[i] * F.ep[M.w]) * indxm * indxm * 2.0 : 0.0;
    double iep_t = open(P.flag[R.t]) ? (dz[k + 1] * F.ep[c] + dz[k] * F.ep[M.t]) * indzp * indzp * 2.0 : 0.0;
    double iep_b = open(P.flag[R.b]) ? (dz[k - 1] * F.ep[c] + dz[k] * F.ep[M.b]) * indzm * indzm * 2.0 : 0.0;
    double iepx = (P.rb[i] * iep_e + P.rb[i - 1] * iep_w) * P.indx[i] * P.inr[i];
    double iepz = (iep_t + iep_b) * P.indz[k];
    double iepy = 0.0;
    double sqc = P.gammaair * F.p[c] / F.rog[c];
    double rbeta = F.ep[c] / sqc;
    rbeta = rbeta + dt * dt * (iepx + iepy + iepz);
    abt = 1.0 / rbeta;
    cnv = P.delg * F.rgp[c];
}

// initial gas mass fluxes + betas (iter.f:170-191).  In the reference loop a
// face shared by two fluid cells ends with the value of the later (upper)
// cell; this thread writes exactly the faces it is the last writer of.
__global__ void k_mflux_init2d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    MF2 f;
    cell_massflux(P, F.rgp, F.ug, F.wg, R, M, i, k, f);
    F.rgfe[R.w] = f.w;
    F.rgft[R.b] = f.b;
    if (!fluid(P, R.e)) F.rgfe[c] = f.e;
    if (!fluid(P, R.t)) F.rgft[c] = f.t;
    betas_2d(P, F, R, M, i, k, dt, F.conv[c], F.abeta[c]);
}

// calc_res, iter.f:743-771
__device__ __forceinline__ double calc_res_2d(const Prm &P, const Fld &F, const Raw2 &R, int i, int k, double dt) {
    int c = R.c;
    const CellFaces b = cell_faces(P, c);
    double resx = (b.e * F.rgfe[c] - b.w * F.rgfe[R.w]) * P.indx[i] * P.inr[i];
    double resz = (b.t * F.rgft[c] - b.b * F.rgft[R.b]) * P.indz[k];
    double resy = 0.0;
    return F.rgp[c] - F.rgpn[c] + dt * b.ivf * (resx + resy + resz);
}

// calc_eps, iter.f:927-994
__device__ __forceinline__ void calc_eps_2d(const Prm &P, const Fld &F, const Raw2 &R, int i, int k, double dt) {
    int c = R.c;
    const CellFaces b = cell_faces(P, c);
    double rls = 0;
    for (int is = 1; is <= P.ns; ++is) {
        double rlkx = (b.e * SOL(F.rsfe, c, is) - b.w * SOL(F.rsfe, R.w, is)) * P.indx[i] * P.inr[i];
        double rlkz = (b.t * SOL(F.rsft, c, is) - b.b * SOL(F.rsft, R.b, is)) * P.indz[k];
        double rlky = 0.0;
        double t = SOL(F.rlkn, c, is) - dt * b.ivf * (rlkx + rlky + rlkz);
        t = t + dt * b.ivf * SOL(F.sink, c, is);
        double v = fmax(0.0, t);
        SOL(F.rlk, c, is) = v;
        rls = rls + v * P.inrl[is];
    }
    F.ep[c] = 1.0 - rls;
    if (rls > 1.0) atomicAdd(&F.counters[2], 1);
}

// padjust + newp, iter.f:997-1109 (bracketing state in registers)
struct PAdj { double dp, d1, d2, p1, p2, d12; };

__device__ __forceinline__ void padjust(PAdj &s, double &p, int &kros, double d3, double &p3, double omega, double &abeta) {
    if (kros != 3) {
        if (d3 > 0.0) {
            s.d1 = d3; s.p1 = p3;
            if (kros == -1) kros = 0;
            else if (kros == 1) kros = 2;
        } else if (d3 <= 0.0) {
            s.d2 = d3; s.p2 = p3;
            if (kros == -1) kros = 1;
            else if (kros == 0) kros = 2;
        }
        if (kros == 2) {
            s.d12 = 1.0 / (s.d1 - s.d2);
            p = (s.d1 * s.p2 - s.d2 * s.p1) * s.d12;
            abeta = (s.p1 - s.p2) * s.d12;
            kros = 3;
        } else if (kros < 2) {
            s.dp = -d3 * abeta;
            s.dp = s.dp * omega;
            double sg = copysign(1.0, d3);
            if (-s.dp * sg > 2.5e-1 * p3) s.dp = -2.5e-1 * sg * p3;
            p = p + s.dp;
        }
    } else {
        double d1 = s.d1, d2 = s.d2, p1 = s.p1, p2 = s.p2, pa = 0, pb = 0;
        if (d1 != d3) pa = (d1 * p3 - d3 * p1) / (d1 - d3);
        if (d1 * d3 <= 0.0) {
            if (d2 != d3) pb = (d2 * p3 - d3 * p2) / (d2 - d3);
            else pb = 0.5 * (p1 + p3);
            if (pb < p3 || pb > p1) pb = 0.5 * (p1 + p3);
        } else {
            if (d1 == d3) pa = 0.5 * (p2 + p3);
            if (pa < p2 || pa > p3) pa = 0.5 * (p2 + p3);
            pb = (d2 * p3 - d3 * p2) / (d2 - d3);
        }
        p = 0.5 * (pa + pb);
        if (d3 > 0.0) { s.d1 = d3; s.p1 = p3; }
        else { s.d2 = d3; s.p2 = p3; }
    }
    p3 = p;
}


// ---------------------------------------------------------------------------
// ygas, ygas.f:27-325 (2D)
// ---------------------------------------------------------------------------
template <typename Real = double>
__global__ void k_ygas_flux2d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    bool dow = !fluid(P, R.w), dob = !fluid(P, R.b), mus = P.muscl > 0 && P.flag[c] == FLUID;
    St2T<Real> d;
    first_nb2(d, F.rgp, R, M);
    if (mus) third_nb2(d, F.rgp, M);
    Real uw = F.ug[R.w], uc = F.ug[c], wb = F.wg[R.b], wc = F.wg[c];
    for (int ig = 0; ig < P.ng; ++ig) {
        const double *Y = F.ygc + (size_t)ig * P.ncell;
        St2T<Real> y;
        first_nb2(y, Y, R, M);
        Real fe = 0, ft = 0, fw = 0, fb = 0;
        fsc_2d(P, fe, ft, fw, fb, dow, dob, d, y, uw, uc, wb, wc, i);
        if (mus) {
            third_nb2(y, Y, M);
            muscl_fsc_2d(P, fe, ft, d, y, uc, wc, i, k);
        }
        GAS(F.yfe, c, ig) = fe;
        GAS(F.yft, c, ig) = ft;
        if (dow) GAS(F.yfe, R.w, ig) = fw;
        if (dob) GAS(F.yft, R.b, ig) = fb;
    }
}

__global__ void k_ygas2d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    int imjk = at2(P, max(i - 1, 1), k), ijkm = at2(P, i, max(k - 1, 1));  // raw W/B neighbours
    const CellFaces b = cell_faces(P, c);
    double rgpgc[PDAC_MAXG], rgpt = 0, yfy = 0;
    for (int ig = 0; ig < P.ng; ++ig) {
        double yfw = GAS(F.yfe, imjk, ig), yfb = GAS(F.yft, ijkm, ig);
        double yfx = b.e * GAS(F.yfe, c, ig) - b.w * yfw;
        double yfz = b.t * GAS(F.yft, c, ig) - b.b * yfb;
        double v = GAS(F.rgpgcn, c, ig);
        v = v - b.ivf * dt * P.indx[i] * yfx * P.inr[i];
        v = v - b.ivf * dt * 0.0 * yfy;
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
// htilde, htilde.f:25-575 (2D)
// ---------------------------------------------------------------------------
// GRAV adds the work of gravity to the convective flux (htilde); the
// explicit solver's calc_all_fluxes (explicit_solver.f:2165-2885) has none
template <bool GRAV, typename Real = double>
__global__ void k_htilde_flux2d(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    bool dow = !fluid(P, R.w), dob = !fluid(P, R.b), mus = P.muscl > 0 && P.flag[c] == FLUID;
    bool hw = P.flag[R.w] != 1, hb = P.flag[R.b] != 1;  // hotc.f:34,52 test the flag value
    int n = P.ncell;
    for (int ph = 0; ph <= P.ns; ++ph) {
        size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
        const double *EN = ph == 0 ? F.sieg : F.sies + off;
        const double *DE = ph == 0 ? F.rgp : F.rlk + off;
        const double *U = ph == 0 ? F.ug : F.us + off;
        const double *W = ph == 0 ? F.wg : F.ws + off;
        double *fE = ph == 0 ? F.egfe : F.esfe + off;
        double *fT = ph == 0 ? F.egft : F.esft + off;
        St2T<Real> en, de;
        first_nb2(en, EN, R, M);
        first_nb2(de, DE, R, M);
        Real uw = U[R.w], uc = U[c], wb = W[R.b], wc = W[c];
        Real fe = 0, ft = 0, fw = 0, fb = 0;
        fsc_2d(P, fe, ft, fw, fb, dow, dob, en, de, uw, uc, wb, wc, i);
        if (mus) {
            third_nb2(en, EN, M);
            third_nb2(de, DE, M);
            muscl_fsc_2d(P, fe, ft, en, de, uc, wc, i, k);
        }
        Real he = 0, ht = 0, hwv = 0, hbv = 0;
        bool visc = ph == 0 ? P.gas_viscosity : P.part_viscosity;
        if (visc) {
            St2T<Real> ka, ep, te;
            if (ph == 0) {
                first_nb2(ka, P.iturb ? F.kapgt : F.kapg, R, M);
                first_nb2(ep, F.ep, R, M);
                first_nb2(te, F.tg, R, M);
            } else {
                Real kk = P.kap[ph], ir = P.inrl[ph];
                ka.c = ka.e = ka.w = ka.t = ka.b = kk;
                ep.c = ir * de.c; ep.e = ir * de.e; ep.w = ir * de.w; ep.t = ir * de.t; ep.b = ir * de.b;
                first_nb2(te, F.ts + off, R, M);
            }
            hotc_2d(P, he, ht, hwv, hbv, hw, hb, ep, te, ka, i, k);
        }
        double gx = P.gravx, gz = P.gravz;
        if (GRAV) {
            fE[c] = fe - he + DE[c] * gx * uc;
            fT[c] = ft - ht + DE[c] * gz * wc;
        } else {
            fE[c] = fe - he;
            fT[c] = ft - ht;
        }
        // W/B faces towards non-fluid cells; when the neighbour's flag is not
        // exactly 1 but still fluid (dome/immb), hotc writes hgfw yet htilde
        // does not subtract it (htilde.f:338-339) -- only non-fluid matter here.
        if (dow) fE[R.w] = fw - (hw ? hwv : Real(0));
        if (dob) fT[R.b] = fb - (hb ? hbv : Real(0));
    }
}

__global__ void k_htilde2d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    int imjk = at2(P, max(i - 1, 1), k), ijkm = at2(P, i, max(k - 1, 1));  // raw W/B neighbours
    const CellFaces b = cell_faces(P, c);
    double egfx = b.e * F.egfe[c] - b.w * F.egfe[imjk];
    double egfz = b.t * F.egft[c] - b.b * F.egft[ijkm];
    double egfy = 0.0;
    double flx = dt * P.indx[i] * egfx * P.inr[i] + dt * 0.0 * egfy + dt * P.indz[k] * egfz;
    flx = flx * b.ivf;
    F.rhg[c] = -flx;
    for (int is = 1; is <= P.ns; ++is) {
        double esfx, esfz;
        if (SOL(F.rlk, imjk, is) * P.inrl[is] <= 1.0e-9) esfx = b.e * SOL(F.esfe, c, is);
        else esfx = b.e * SOL(F.esfe, c, is) - b.w * SOL(F.esfe, imjk, is);
        if (SOL(F.rlk, ijkm, is) * P.inrl[is] <= 1.0e-9) esfz = b.t * SOL(F.esft, c, is);
        else esfz = b.t * SOL(F.esft, c, is) - b.b * SOL(F.esft, ijkm, is);
        double esfy = 0.0;
        flx = dt * P.indx[i] * esfx * P.inr[i] + dt * 0.0 * esfy + dt * P.indz[k] * esfz;
        flx = flx * b.ivf;
        SOL(F.rhs, c, is) = -flx + SOL(F.sink, c, is) * dt * b.ivf * SOL(F.sies, c, is);
    }
}

// ---------------------------------------------------------------------------
// ftem, ftem.f:19-248 (2D)
// ---------------------------------------------------------------------------
__global__ void k_ftem2d(Prm P, Fld F, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    const double *dx = P.dx, *dz = P.dz;
    int ns = P.ns, nph = P.nph;
    double alpha = P.alpha;
    int imjk = R.w, ijkm = R.b;
    double indxc = 1.0 / (dx[i] + (dx[i + 1] + dx[i - 1]) * 0.5);
    double indzc = 1.0 / (dz[k] + (dz[k + 1] + dz[k - 1]) * 0.5);
    const CellFaces bf = cell_faces(P, c);
    double ugc = 0.5 * (bf.e * F.ug[c] + bf.w * F.ug[imjk]);
    double wgc = 0.5 * (bf.t * F.wg[c] + bf.b * F.wg[ijkm]);
    double dpxyz = 0.0;
    dpxyz = dpxyz + dt * indxc * ugc * (F.p[M.e] - F.p[M.w]);
    dpxyz = dpxyz + dt * 0.0 * 0.0 * 0.0;
    dpxyz = dpxyz + dt * indzc * wgc * (F.p[M.t] - F.p[M.b]);
    double deltap = F.ep[c] * (F.p[c] - F.pn[c] + dpxyz);
    double workg = F.rgp[c] * (F.ug[c] * P.gravx + F.wg[c] * P.gravz);
    double at[PDAC_MAXP + 1][PDAC_MAXP + 1], bt[PDAC_MAXP + 1];
    at[1][1] = F.rgp[c];
    bt[1] = F.siegn[c] * F.rgpn[c] + F.rhg[c] + deltap + workg - 0.0;
    double cgc = F.cg[c];
    for (int is = 1; is <= ns; ++is) {
        int is1 = is + 1;
        double dugs = ((F.ug[c] - SOL(F.us, c, is)) + (F.ug[imjk] - SOL(F.us, imjk, is))) * 0.5;
        double dwgs = ((F.wg[c] - SOL(F.ws, c, is)) + (F.wg[ijkm] - SOL(F.ws, ijkm, is))) * 0.5;
        double hv = hvs(P, SOL(F.rlk, c, is), F.rog[c], dugs, 0.0, dwgs, F.mug[c], F.kapg[c], cgc, is);
        double works = SOL(F.rlk, c, is) * (SOL(F.us, c, is) * P.gravx + SOL(F.ws, c, is) * P.gravz);
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

// deterministic two-pass reduction of the mass totals (residuals.f:14-130)
__global__ void k_mass_partial(Prm P, Fld F, double *partial, int nq) {
    extern __shared__ double sh[];
    int tid = threadIdx.x;
    for (int q = 0; q < nq; ++q) sh[q * blockDim.x + tid] = 0.0;
    for (int c = blockIdx.x * blockDim.x + tid; c < P.ncell; c += gridDim.x * blockDim.x) {
        if (!fluid(P, c)) continue;
        int i = c % P.nx + 1, j = (c / P.nx) % P.ny + 1, k = c / (P.nx * P.ny) + 1;
        double vol = P.dx[i] * P.dz[k] * (P.itc == 1 ? P.r[i] : 1.0) * (P.d3 ? P.dy[j] : 1.0);
        sh[tid] += F.rgp[c] * vol;
        for (int is = 1; is <= P.ns; ++is) sh[is * blockDim.x + tid] += SOL(F.rlk, c, is) * vol;
        for (int ig = 0; ig < P.ng; ++ig) sh[(1 + P.ns + ig) * blockDim.x + tid] += F.rgp[c] * GAS(F.ygc, c, ig) * vol;
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s)
            for (int q = 0; q < nq; ++q) sh[q * blockDim.x + tid] += sh[q * blockDim.x + tid + s];
        __syncthreads();
    }
    if (tid == 0)
        for (int q = 0; q < nq; ++q) partial[(size_t)q * gridDim.x + blockIdx.x] = sh[q * blockDim.x];
}

}  // namespace pdac

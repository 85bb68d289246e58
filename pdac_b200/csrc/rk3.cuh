// rk3.cuh -- the explicit SSP-RK3 solver (time_integration = 1,
// explicit_solver.f) on the device, 2D (D = 2) and 3D (D = 3).
//
// The star variables of the reference (rgpstar, ugstar ...) are the state
// arrays themselves: compute_fluxes (explicit_solver.f:1225-1345) copies star
// into state before every flux pass and nothing on the path reads a state
// value that differs from its star value, so one copy suffices.
//
// Execution of explicit_iter (explicit_solver.f:996-1223):
//  * each of the first two stages is a flux pass, one parallel kernel for
//    every equation except gas enthalpy, and a wavefront for gas enthalpy.
//    In the reference one loop in cell order computes a cell's right-hand
//    side and then its new star values (update_star :1752-1969), so a cell
//    sees the new values of its west/south/bottom neighbours.  Of all the
//    right-hand sides only the gas-enthalpy one reads such values (pressure
//    and gas velocity in its p-div(u) term, compute_rhs :779-798), and the
//    new pressure depends on the new gas enthalpy: that chain is sequential
//    along every path of increasing i + j + k.  k_rk3_stage computes all
//    other rows and updates from stage-start values and parks the new
//    densities, volume fraction and gas velocities in K.x* (their neighbours
//    still need the old ones); k_rk3_wave then runs hyperplane by
//    hyperplane, i + j + k = d, completing the gas enthalpy, temperature and
//    pressure of the cells on the plane and committing their parked values.
//    Cells on one hyperplane are independent: their only cross reads are
//    first neighbours, which lie on d - 1 (already done) or d + 1 (not yet).
//  * stage 3, the final combination and the implicit drag / heat-exchange
//    solve (compute_physical_coeff :2105-2163, compute_linear_systems
//    :822-994, solve_linear_systems :1347-1607) are parallel.
#pragma once
#include <cooperative_groups.h>
#include "kernels3d.cuh"

namespace pdac {

// fields of the explicit solver next to the state
struct RkF {
    double *ugn, *vgn, *wgn;        // n-level gas velocities (ncell)
    double *usn, *vsn, *wsn;        // n-level particle velocities (ncell, ns)
    double *hv;                     // gas-particle heat exchange coefficient (ncell, ns)
    double *k1, *k2;                // stage right-hand sides, row eq at [eq * ncell + c]; k1 holds rhs3 after stage 3
    double *xrgp, *xrlk, *xep;      // new densities / volume fraction of stages 1-2, pending commit
    double *xug, *xvg, *xwg;        // new gas velocities of stages 1-2, pending commit
};

constexpr double RK3_LIMIT = 1.0e-12;  // explicit_solver.f:134

// first neighbours of a cell: raw (myijk, clamped) and remapped (myinds:
// wall and filled cells -> the cell itself, ghost.f:963-989)
template <int D>
struct Cell {
    int c, i, j, k;
    int rw, rs, rb, re, rn, rt;
    int mw, ms, mb, me, mn, mt;
};

template <int D>
__device__ __forceinline__ void cell_of(const Prm &P, int c, Cell<D> &q) {
    q.c = c;
    if (D == 3) {
        ijk_of(P, c, q.i, q.j, q.k);
    } else {
        q.i = c % P.nx + 1;
        q.j = 1;
        q.k = c / P.nx + 1;
    }
    const int plane = P.nx * P.ny;
    q.rw = q.i > 1 ? c - 1 : c;
    q.re = q.i < P.nx ? c + 1 : c;
    q.rb = q.k > 1 ? c - plane : c;
    q.rt = q.k < P.nz ? c + plane : c;
    if (D == 3) {
        q.rs = q.j > 1 ? c - P.nx : c;
        q.rn = q.j < P.ny ? c + P.nx : c;
    } else {
        q.rs = q.rn = c;
    }
    const int *fl = P.flag;
    q.mw = is_wallf(fl[q.rw]) ? c : q.rw;
    q.me = is_wallf(fl[q.re]) ? c : q.re;
    q.mb = is_wallf(fl[q.rb]) ? c : q.rb;
    q.mt = is_wallf(fl[q.rt]) ? c : q.rt;
    if (D == 3) {
        q.ms = is_wallf(fl[q.rs]) ? c : q.rs;
        q.mn = is_wallf(fl[q.rn]) ? c : q.rn;
    } else {
        q.ms = q.mn = c;
    }
}

// ---- face fluxes of the flux pass ---------------------------------------------
// mass flux of phase ph across the x (f = 0), y (1) or z (2) face at cell c
__device__ __forceinline__ double rk_mass(const Prm &P, const Fld &F, int ph, int f, int c) {
    size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * P.ncell;
    const double *a = f == 0 ? (ph == 0 ? F.rgfe : F.rsfe + off)
                    : f == 1 ? (ph == 0 ? F.rgfn : F.rsfn + off)
                             : (ph == 0 ? F.rgft : F.rsft + off);
    return a[c];
}
// momentum component comp (0 = x, 1 = y, 2 = z) of phase ph across face f
template <int D>
__device__ __forceinline__ double rk_mom(const Prm &P, const Fld &F, int ph, int comp, int f, int c) {
    if (D == 3) return F.mf[((size_t)(ph * 3 + comp) * 3 + f) * P.ncell + c];
    size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * P.ncell;
    const double *a;
    if (comp == 0) a = f == 0 ? (ph == 0 ? F.ugfe : F.usfe + off) : (ph == 0 ? F.ugft : F.usft + off);
    else a = f == 0 ? (ph == 0 ? F.wgfe : F.wsfe + off) : (ph == 0 ? F.wgft : F.wsft + off);
    return a[c];
}
// enthalpy flux of phase ph across face f
__device__ __forceinline__ double rk_enth(const Prm &P, const Fld &F, int ph, int f, int c) {
    size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * P.ncell;
    const double *a = f == 0 ? (ph == 0 ? F.egfe : F.esfe + off)
                    : f == 1 ? (ph == 0 ? F.egfn : F.esfn + off)
                             : (ph == 0 ? F.egft : F.esft + off);
    return a[c];
}

// ---- compute_rhs, explicit_solver.f:566-820, one row at a time ------------------
// mass of phase ph (:617-642)
template <int D>
__device__ __forceinline__ double rhs_mass(const Prm &P, const Fld &F, const Cell<D> &q, int ph) {
    int c = q.c;
    double fx = (rk_mass(P, F, ph, 0, c) - rk_mass(P, F, ph, 0, q.rw)) * P.indx[q.i] * P.inr[q.i];
    double fy = 0.0;
    if (D == 3) fy = (rk_mass(P, F, ph, 1, c) - rk_mass(P, F, ph, 1, q.rs)) * P.indy[q.j];
    double fz = (rk_mass(P, F, ph, 2, c) - rk_mass(P, F, ph, 2, q.rb)) * P.indz[q.k];
    double tmp = fx + fy + fz;
    return 0.0 - tmp;
}

// momentum along axis ax (0 = x, 1 = y, 2 = z) of phase ph (:644-777): flux
// divergence, pressure gradient, gravity and the viscous term of the
// n-level stress (vis, block (ph * 3 + ax))
template <int D>
__device__ __forceinline__ double rhs_mom(const Prm &P, const Fld &F, const Cell<D> &q, int ph, int ax) {
    const int c = q.c, i = q.i, j = q.j, k = q.k;
    const int comp = D == 3 ? ax : (ax == 0 ? 0 : 1);
    const int fzf = 2;
    double fx, fy = 0.0, fz;
    if (ax == 0) {
        double indxp = 1.0 / (P.dx[i] + P.dx[i + 1]);
        fx = (rk_mom<D>(P, F, ph, comp, 0, c) - rk_mom<D>(P, F, ph, comp, 0, q.rw)) * 2.0 * indxp * P.inrb[i];
        if (D == 3) fy = (rk_mom<D>(P, F, ph, comp, 1, c) - rk_mom<D>(P, F, ph, comp, 1, q.rs)) * P.indy[j];
        fz = (rk_mom<D>(P, F, ph, comp, fzf, c) - rk_mom<D>(P, F, ph, comp, fzf, q.rb)) * P.indz[k];
    } else if (ax == 1) {
        double indyp = 1.0 / (P.dy[j] + P.dy[j + 1]);
        fx = (rk_mom<D>(P, F, ph, comp, 0, c) - rk_mom<D>(P, F, ph, comp, 0, q.rw)) * P.indx[i];
        fy = (rk_mom<D>(P, F, ph, comp, 1, c) - rk_mom<D>(P, F, ph, comp, 1, q.rs)) * 2.0 * indyp;
        fz = (rk_mom<D>(P, F, ph, comp, fzf, c) - rk_mom<D>(P, F, ph, comp, fzf, q.rb)) * P.indz[k];
    } else {
        double indzp = 1.0 / (P.dz[k] + P.dz[k + 1]);
        fx = (rk_mom<D>(P, F, ph, comp, 0, c) - rk_mom<D>(P, F, ph, comp, 0, q.rw)) * P.indx[i] * P.inr[i];
        if (D == 3) fy = (rk_mom<D>(P, F, ph, comp, 1, c) - rk_mom<D>(P, F, ph, comp, 1, q.rs)) * P.indy[j];
        fz = (rk_mom<D>(P, F, ph, comp, fzf, c) - rk_mom<D>(P, F, ph, comp, fzf, q.rb)) * 2.0 * indzp;
    }
    double tmp = fx + fy + fz;
    // metric pair and remapped neighbour along the axis
    double d0, d1, g;
    int nb;
    if (ax == 0) { d0 = P.dx[i]; d1 = P.dx[i + 1]; nb = q.me; g = P.gravx; }
    else if (ax == 1) { d0 = P.dy[j]; d1 = P.dy[j + 1]; nb = q.mn; g = P.gravy; }
    else { d0 = P.dz[k]; d1 = P.dz[k + 1]; nb = q.mt; g = P.gravz; }
    double inp = 1.0 / (d0 + d1);
    double dn, gterm, vis = F.vis[(size_t)(ph * 3 + ax) * P.ncell + c];
    if (ph == 0) {
        dn = 1.0;
        if (P.pmodel == 1) dn = (d0 * F.ep[nb] + d1 * F.ep[c]) * inp;
        gterm = (d0 * F.rgp[nb] + d1 * F.rgp[c]) * inp * g;
    } else {
        const double *rl = F.rlk + (size_t)(ph - 1) * P.ncell;
        double eps = (d0 * rl[nb] + d1 * rl[c]) * inp * P.inrl[ph];
        dn = eps * (double)(2 - P.pmodel);
        gterm = (d0 * rl[nb] + d1 * rl[c]) * inp * g;
    }
    double r = 0.0;
    r = r - tmp;
    r = r - dn * (F.p[nb] - F.p[c]) * 2.0 * inp;
    r = r + gterm;
    r = r + vis;
    return r;
}

// enthalpy flux divergence of phase ph (:800-817), the whole particle row
template <int D>
__device__ __forceinline__ double enth_div(const Prm &P, const Fld &F, const Cell<D> &q, int ph) {
    int c = q.c;
    double fx = (rk_enth(P, F, ph, 0, c) - rk_enth(P, F, ph, 0, q.rw)) * P.indx[q.i] * P.inr[q.i];
    double fy = 0.0;
    if (D == 3) fy = (rk_enth(P, F, ph, 1, c) - rk_enth(P, F, ph, 1, q.rs)) * P.indy[q.j];
    double fz = (rk_enth(P, F, ph, 2, c) - rk_enth(P, F, ph, 2, q.rb)) * P.indz[q.k];
    return fx + fy + fz;
}

// gas enthalpy (:779-798): flux divergence plus ep (dp/dt + u.grad p), with
// the gas velocities and pressures the arrays hold when it is called
template <int D>
__device__ __forceinline__ double rhs_gas_enth(const Prm &P, const Fld &F, const Cell<D> &q, double dt) {
    const int c = q.c, i = q.i, j = q.j, k = q.k;
    const double *dx = P.dx, *dz = P.dz;
    double indxc = 1.0 / (dx[i] + (dx[i + 1] + dx[i - 1]) * 0.5);
    double indyc = 0.0;
    double indzc = 1.0 / (dz[k] + (dz[k + 1] + dz[k - 1]) * 0.5);
    double ugc = 0.5 * (F.ug[c] + F.ug[q.rw]);
    double vgc = 0.0;
    double wgc = 0.5 * (F.wg[c] + F.wg[q.rb]);
    if (D == 3) {
        indyc = 1.0 / (P.dy[j] + (P.dy[j + 1] + P.dy[j - 1]) * 0.5);
        vgc = 0.5 * (F.vg[c] + F.vg[q.rs]);
    }
    double tmp = enth_div<D>(P, F, q, 0);
    double dpxyz = 0.0;
    dpxyz = dpxyz + indxc * ugc * (F.p[q.me] - F.p[q.mw]);
    // in 2D the y term is 0 * 0 * (...), which leaves the (non -0) sum as it is
    if (D == 3) dpxyz = dpxyz + indyc * vgc * (F.p[q.mn] - F.p[q.ms]);
    else dpxyz = dpxyz + 0.0;
    dpxyz = dpxyz + indzc * wgc * (F.p[q.mt] - F.p[q.mb]);
    double r = 0.0;
    r = r - tmp;
    tmp = 1.0 / dt;
    r = r + F.ep[c] * (F.p[c] - F.pn[c]) * tmp;
    r = r + F.ep[c] * dpxyz;
    return r;
}

// init_rhs (explicit_solver.f:1645-1750): the n-level conserved variable of
// row (kind, ph, ax): kind 0 mass, 1 momentum along ax, 2 enthalpy
template <int D>
__device__ __forceinline__ double init_row(const Prm &P, const Fld &F, const RkF &K, const Cell<D> &q, int kind, int ph,
                                           int ax) {
    const int c = q.c;
    const size_t n = P.ncell, off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
    if (kind == 0) return ph == 0 ? F.rgpn[c] : F.rlkn[off + c];
    if (kind == 2) return ph == 0 ? F.rgpn[c] * F.siegn[c] : F.rlkn[off + c] * F.siesn[off + c];
    double d0, d1;
    int nb;
    const double *vg, *vs;
    if (ax == 0) { d0 = P.dx[q.i]; d1 = P.dx[q.i + 1]; nb = q.me; vg = K.ugn; vs = K.usn; }
    else if (ax == 1) { d0 = P.dy[q.j]; d1 = P.dy[q.j + 1]; nb = q.mn; vg = K.vgn; vs = K.vsn; }
    else { d0 = P.dz[q.k]; d1 = P.dz[q.k + 1]; nb = q.mt; vg = K.wgn; vs = K.wsn; }
    double inp = 1.0 / (d0 + d1);
    if (ph == 0) {
        double rold = (d0 * F.rgpn[nb] + d1 * F.rgpn[c]) * inp;
        return rold * vg[c];
    }
    double rold = (d0 * F.rlkn[off + nb] + d1 * F.rlkn[off + c]) * inp;
    return rold * vs[off + c];
}

// ---- compute_physical_coeff, explicit_solver.f:2105-2163 ------------------------
// viscosity / conductivity, heat exchange, kdrags (always, whatever the drag
// model) and the interphase matrix inter (drag.f:173-246) from the state;
// the dt of inter is the module time step at the call
template <int NP, int D>
__device__ __forceinline__ void phys_coeff(const Prm &P, const Fld &F, const RkF &K, const Cell<D> &q, double dt) {
    constexpr int MP = Sys<NP>::M;
    constexpr int MA = MP * (MP + 1) / 2 + 1;
    const int c = q.c, ns = nphases<NP>(P) - 1, nph = ns + 1;
    const size_t n = P.ncell;
    double xg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) xg[ig] = GAS(F.xgc, c, ig);
    double mu, ka;
    viscon(P, mu, ka, xg, F.tg[c]);
    F.mug[c] = mu;
    F.kapg[c] = ka;
    double kp[MP], rlkc[MP];
    for (int is = 1; is <= ns; ++is) {
        size_t off = (size_t)(is - 1) * n;
        double dugs = ((F.ug[c] - F.us[off + c]) + (F.ug[q.rw] - F.us[off + q.rw])) * 0.5;
        double dwgs = ((F.wg[c] - F.ws[off + c]) + (F.wg[q.rb] - F.ws[off + q.rb])) * 0.5;
        double dvgs = 0.0;
        if (D == 3) dvgs = ((F.vg[c] - F.vs[off + c]) + (F.vg[q.rs] - F.vs[off + q.rs])) * 0.5;
        rlkc[is] = F.rlk[off + c];
        K.hv[off + c] = hvs(P, rlkc[is], F.rog[c], dugs, dvgs, dwgs, mu, ka, F.cg[c], is);
        kp[is] = kdrags(P, dugs, dvgs, dwgs, F.ep[c], F.rgp[c], rlkc[is], mu, is);
    }
    double au[MA], av[MA], aw[MA];
    int ks = 0;
    for (int k1 = 1; k1 <= nph; ++k1) {
        if (k1 == 1) {
            ks++;
            au[ks] = 0; av[ks] = 0; aw[ks] = 0;
        } else {
            for (int kk = 1; kk <= k1; ++kk) {
                ks++;
                if (kk == 1) {
                    au[ks] = -kp[k1 - 1] * dt; av[ks] = -kp[k1 - 1] * dt; aw[ks] = -kp[k1 - 1] * dt;
                } else if (kk == k1) {
                    au[ks] = 0; av[ks] = 0; aw[ks] = 0;
                } else {
                    double con = ppdrag(P, rlkc, k1, kk);
                    const double *U = F.us, *Wv = F.ws;
                    size_t o1 = (size_t)(k1 - 2) * n, o2 = (size_t)(kk - 2) * n;
                    double du = fabs(U[o1 + c] - U[o2 + c] + U[o1 + q.rw] - U[o2 + q.rw]) * 0.5;
                    double dv = 0.0;
                    if (D == 3) dv = fabs(F.vs[o1 + c] - F.vs[o2 + c] + F.vs[o1 + q.rs] - F.vs[o2 + q.rs]) * 0.5;
                    double dw = fabs(Wv[o1 + c] - Wv[o2 + c] + Wv[o1 + q.rb] - Wv[o2 + q.rb]) * 0.5;
                    au[ks] = -(con * du) * dt;
                    av[ks] = -(con * dv) * dt;
                    aw[ks] = -(con * dw) * dt;
                }
            }
        }
    }
    for (int k1 = 1; k1 <= nph; ++k1) {
        double sx = 0, sy = 0, sz = 0;
        for (int kk = 1; kk <= k1; ++kk) {
            int t = kk + k1 * (k1 - 1) / 2;
            sx = sx + au[t]; sy = sy + av[t]; sz = sz + aw[t];
        }
        for (int kk = k1; kk <= nph; ++kk) {
            int t = k1 + kk * (kk - 1) / 2;
            sx = sx + au[t]; sy = sy + av[t]; sz = sz + aw[t];
        }
        int t = k1 * (k1 + 1) / 2;
        au[t] = -sx; av[t] = -sy; aw[t] = -sz;
    }
    const int nap = nph * (nph + 1) / 2;
    for (int t = 1; t <= nap; ++t) {
        APP(F.appu, c, t) = au[t];
        APP(F.appw, c, t) = aw[t];
        if (D == 3) APP(F.appv, c, t) = av[t];
    }
}

// ---- kernels ------------------------------------------------------------------

// initialize_fieldn (explicit_solver.f:419-564) for every cell: n-level
// copies and the physical coefficients of the state at full dt
template <int NP, int D>
__global__ void k_rk3_fieldn(Prm P, Fld F, RkF K, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    const size_t n = P.ncell;
    F.pn[c] = F.p[c];
    F.epn[c] = F.ep[c];
    F.rgpn[c] = F.rgp[c];
    F.siegn[c] = F.sieg[c];
    K.ugn[c] = F.ug[c];
    if (D == 3) K.vgn[c] = F.vg[c];
    K.wgn[c] = F.wg[c];
    for (int is = 1; is <= P.ns; ++is) {
        size_t off = (size_t)(is - 1) * n;
        F.rlkn[off + c] = F.rlk[off + c];
        F.siesn[off + c] = F.sies[off + c];
        K.usn[off + c] = F.us[off + c];
        if (D == 3) K.vsn[off + c] = F.vs[off + c];
        K.wsn[off + c] = F.ws[off + c];
    }
    for (int ig = 0; ig < P.ng; ++ig) GAS(F.rgpgcn, c, ig) = F.rgpn[c] * GAS(F.ygc, c, ig);
    Cell<D> q;
    cell_of<D>(P, c, q);
    phys_coeff<NP, D>(P, F, K, q, dt);
}

// 2D viscous stress divergence of one phase of one fluid cell (viscg /
// viscs, visc.f:150-291, stress2D visc.f:561-696) with the particle
// repulsion term, into vis blocks (ph * 3 + 0) and (ph * 3 + 2)
__global__ void k_visc2d(Prm P, Fld F) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)P.ncell * (unsigned)(P.ns + 1)) return;
    int ph = (int)(t / (unsigned)P.ncell), c = (int)(t % (unsigned)P.ncell);
    if (!fluid(P, c)) return;
    int i = c % P.nx + 1, k = c / P.nx + 1;
    Raw2 R;
    Rem2 M;
    raw2(P, i, k, R);
    rem2(P, i, k, R, M);
    const double *dx = P.dx, *dz = P.dz;
    size_t n = P.ncell, off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
    double vx = 0, vz = 0;
    if (ph == 0) {
        if (P.gas_viscosity) {
            const double *mug = F.mug, *mut = P.iturb ? F.mugt : F.mug, *ep = F.ep;
            stress2d_cell(P, R, M, i, k, [&](int q) { return mut[q]; }, [&](int q) { return mug[q]; },
                          [&](int q) { return ep[q]; }, F.ug, F.wg, vx, vz);
        }
    } else if (P.part_viscosity) {
        const double cm = P.cmus[ph], ir = P.inrl[ph];
        const double *rl = F.rlk + off;
        const double *mst = P.iss ? F.must + off : nullptr;
        stress2d_cell(P, R, M, i, k, [&](int q) { return mst ? mst[q] : cm; }, [&](int) { return cm; },
                      [&](int q) { return rl[q] * ir; }, F.us + off, F.ws + off,
                      vx, vz);
        if (P.repulsive_model == 1) {
            const double a_rep = -8.76, b_rep = -0.27;
            double indxp = P.hx[i], indzp = P.hz[k];
            double rc = rl[c], re = rl[M.e], rt = rl[M.t];
            double epsx = (dx[i + 1] * rc + dx[i] * re) * indxp * ir;
            double gepx = pdac_fp::pow(10.0, -a_rep * epsx + b_rep);
            vx = vx - gepx * indxp * 2.0 * (re - rc) * ir;
            double epsz = (dz[k + 1] * rc + dz[k] * rt) * indzp * ir;
            double gepz = pdac_fp::pow(10.0, -a_rep * epsz + b_rep);
            vz = vz - gepz * indzp * 2.0 * (rt - rc) * ir;
        }
    }
    F.vis[(size_t)(ph * 3 + 0) * n + c] = vx;
    F.vis[(size_t)(ph * 3 + 2) * n + c] = vz;
}

// mass fluxes of every phase for the flux pass (masf + fmas inside
// calc_all_fluxes :2240-2320): the density stencil is nb, whose second
// minus-side members (ww, ss, bb) the reference never sets and reads as
// zero.  A face shared by two fluid cells ends with the value of the later
// cell of the reference loop, so this thread writes its W/S/B faces always
// and its E/N/T faces only towards non-fluid cells.
// Real as in k_tilde_flux3d (float only in 3D).
template <int D, typename Real = double>
__global__ void __launch_bounds__(128, PDAC_FLUX_MINB) k_rk3_mflux(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    const size_t n = P.ncell;
    const bool mus = P.muscl > 0 && P.flag[c] == FLUID;
    const int *fl = P.flag;
    if (D == 3) {
        int i, j, k;
        ijk_of(P, c, i, j, k);
        Raw3 R;
        Rem3 M;
        raw3(P, i, j, k, R);
        rem3(P, i, j, k, R, M);
        for (int ph = 0; ph <= P.ns; ++ph) {
            size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
            const double *Dn = ph == 0 ? F.rgp : F.rlk + off;
            const double *U = ph == 0 ? F.ug : F.us + off;
            const double *V = ph == 0 ? F.vg : F.vs + off;
            const double *W = ph == 0 ? F.wg : F.ws + off;
            double *fe = ph == 0 ? F.rgfe : F.rsfe + off;
            double *fn = ph == 0 ? F.rgfn : F.rsfn + off;
            double *ft = ph == 0 ? F.rgft : F.rsft + off;
            S3T<Real> d;
            first_nb3(d, Dn, R, M);
            if (mus) {
                third_nb3(d, Dn, M);
                d.ww = 0.0; d.ss = 0.0; d.bb = 0.0;
            }
            F6T<Real> f;
            massflux_3d(P, d, Real(U[R.w]), Real(U[c]), Real(V[R.s]), Real(V[c]), Real(W[R.b]), Real(W[c]), i, j, k, mus, fl[R.w], fl[R.e], fl[R.s], fl[R.n],
                        fl[R.b], fl[R.t], f);
            fe[R.w] = f.w;
            fn[R.s] = f.s;
            ft[R.b] = f.b;
            if (!fluid(P, R.e)) fe[c] = f.e;
            if (!fluid(P, R.n)) fn[c] = f.n;
            if (!fluid(P, R.t)) ft[c] = f.t;
        }
    } else {
        int i = c % P.nx + 1, k = c / P.nx + 1;
        Raw2 R;
        Rem2 M;
        raw2(P, i, k, R);
        rem2(P, i, k, R, M);
        for (int ph = 0; ph <= P.ns; ++ph) {
            size_t off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
            const double *Dn = ph == 0 ? F.rgp : F.rlk + off;
            const double *U = ph == 0 ? F.ug : F.us + off;
            const double *W = ph == 0 ? F.wg : F.ws + off;
            double *fe = ph == 0 ? F.rgfe : F.rsfe + off;
            double *ft = ph == 0 ? F.rgft : F.rsft + off;
            St2T<Real> d;
            first_nb2(d, Dn, R, M);
            if (mus) {
                third_nb2(d, Dn, M);
                d.ww = 0.0; d.bb = 0.0;
            }
            MF2T<Real> f;
            massflux_2d(P, d, Real(U[R.w]), Real(U[c]), Real(W[R.b]), Real(W[c]), i, k, mus, fl[R.w], fl[R.e], fl[R.b],
                        fl[R.t], f);
            fe[R.w] = f.w;
            ft[R.b] = f.b;
            if (!fluid(P, R.e)) fe[c] = f.e;
            if (!fluid(P, R.t)) ft[c] = f.t;
        }
    }
}

// stages 1 and 2, everything but gas enthalpy: right-hand sides from the
// stage-start state (into k1 / k2) and update_star's new values
// (explicit_solver.f:1752-1969) with rk_a = (1, 0) or (0.25, 0.25)
template <int NP, int D>
__global__ void k_rk3_stage(Prm P, Fld F, RkF K, double dt, int stage) {
    constexpr int MP = Sys<NP>::M;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    Cell<D> q;
    cell_of<D>(P, c, q);
    const size_t n = P.ncell;
    const int ns = nphases<NP>(P) - 1, nph = ns + 1;
    const double a1 = stage == 1 ? 1.0 : 0.25, a2 = stage == 1 ? 0.0 : 0.25;
    double *ks = stage == 1 ? K.k1 : K.k2;
    // store this stage's row and return the (k1, k2) pair of update_star;
    // in stage 1 k2 is the zero init_rhs left
    auto row = [&](int eq, double r, double &v1, double &v2) {
        ks[(size_t)eq * n + c] = r;
        if (stage == 1) { v1 = r; v2 = 0.0; }
        else { v1 = K.k1[(size_t)eq * n + c]; v2 = r; }
    };
    double v1, v2;
    // mass
    row(0, rhs_mass<D>(P, F, q, 0), v1, v2);
    const double rgpnew = F.rgpn[c] + a1 * dt * v1 + a2 * dt * v2;
    double rlknew[MP];
    for (int is = 1; is <= ns; ++is) {
        row(is, rhs_mass<D>(P, F, q, is), v1, v2);
        double t = F.rlkn[(size_t)(is - 1) * n + c] + a1 * dt * v1 + a2 * dt * v2;
        rlknew[is] = (0.0 < t) ? t : 0.0;
    }
    // momenta; the east (north, top) neighbour still holds its old density
    // unless it is the cell itself
    for (int ax = 0; ax < 3; ++ax) {
        if (D == 2 && ax == 1) continue;
        const int blk = D == 3 ? ax + 1 : (ax == 0 ? 1 : 2);
        double d0, d1;
        int nb;
        const double *gN, *sN;
        double *gX, *sS;
        if (ax == 0) { d0 = P.dx[q.i]; d1 = P.dx[q.i + 1]; nb = q.me; gN = K.ugn; sN = K.usn; gX = K.xug; sS = F.us; }
        else if (ax == 1) { d0 = P.dy[q.j]; d1 = P.dy[q.j + 1]; nb = q.mn; gN = K.vgn; sN = K.vsn; gX = K.xvg; sS = F.vs; }
        else { d0 = P.dz[q.k]; d1 = P.dz[q.k + 1]; nb = q.mt; gN = K.wgn; sN = K.wsn; gX = K.xwg; sS = F.ws; }
        const double inp = 1.0 / (d0 + d1);
        row(blk * nph, rhs_mom<D>(P, F, q, 0, ax), v1, v2);
        double rold = (d0 * F.rgpn[nb] + d1 * F.rgpn[c]) * inp;
        double temp = rold * gN[c] + a1 * dt * v1 + a2 * dt * v2;
        double rnb = nb == c ? rgpnew : F.rgp[nb];
        double rnow = (d0 * rnb + d1 * rgpnew) * inp;
        double tmp = 1.0 / rnow;
        gX[c] = temp * tmp;
        for (int is = 1; is <= ns; ++is) {
            size_t off = (size_t)(is - 1) * n;
            row(blk * nph + is, rhs_mom<D>(P, F, q, is, ax), v1, v2);
            rold = (d0 * F.rlkn[off + nb] + d1 * F.rlkn[off + c]) * inp;
            temp = rold * sN[off + c] + a1 * dt * v1 + a2 * dt * v2;
            double lnb = nb == c ? rlknew[is] : F.rlk[off + nb];
            rnow = (d0 * lnb + d1 * rlknew[is]) * inp;
            sS[off + c] = (rnow > RK3_LIMIT) ? temp * (1.0 / rnow) : 0.0;
        }
    }
    // particle enthalpies and temperatures (caloric_eosl, eosl.f:10-40)
    const int e0 = (D == 3 ? 4 : 3) * nph;
    for (int is = 1; is <= ns; ++is) {
        size_t off = (size_t)(is - 1) * n;
        double r = 0.0;
        r = r - enth_div<D>(P, F, q, is);
        row(e0 + is, r, v1, v2);
        double siestmp = F.rlkn[off + c] * F.siesn[off + c] + a1 * dt * v1 + a2 * dt * v2;
        double sies = 0.0;
        if (rlknew[is] > RK3_LIMIT) sies = siestmp * (1.0 / rlknew[is]);
        F.sies[off + c] = sies;
        F.ts[off + c] = 0.0 + (sies - 0.0) / P.cps[is];
    }
    // volume fraction and gas density
    double epstot = 0.0;
    for (int is = 1; is <= ns; ++is) {
        double epsstar = rlknew[is] * P.inrl[is];
        epstot = epstot + epsstar;
    }
    double ep = 1.0 - epstot;
    F.rog[c] = rgpnew / ep;
    K.xep[c] = ep;
    K.xrgp[c] = rgpnew;
    for (int is = 1; is <= ns; ++is) K.xrlk[(size_t)(is - 1) * n + c] = rlknew[is];
}

// stages 1 and 2, gas enthalpy on hyperplane i + j + k = d (j = 1 in 2D):
// right-hand side, new enthalpy, temperature (caloric_eosg) and pressure,
// then commit of the values k_rk3_stage parked.  One thread per (j, k) of
// the plane's k range kmin.. (k only in 2D).
template <int D>
__global__ void k_rk3_wave(Prm P, Fld F, RkF K, double dt, int stage, int d, int kmin, int nthreads) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nthreads) return;
    int i, j, k;
    if (D == 3) {
        int nj = P.ny - 2;
        j = 2 + t % nj;
        k = kmin + t / nj;
        i = d - j - k;
    } else {
        j = 1;
        k = kmin + t;
        i = d - k;
    }
    if (i < 2 || i > P.nx - 1 || k > P.nz - 1) return;
    const int c = (i - 1) + P.nx * ((j - 1) + P.ny * (k - 1));
    if (!fluid(P, c)) return;
    Cell<D> q;
    cell_of<D>(P, c, q);
    const size_t n = P.ncell;
    const int nph = P.nph, e0 = (D == 3 ? 4 : 3) * nph;
    const double a1 = stage == 1 ? 1.0 : 0.25, a2 = stage == 1 ? 0.0 : 0.25;
    double r = rhs_gas_enth<D>(P, F, q, dt);
    double v1, v2;
    if (stage == 1) { K.k1[(size_t)e0 * n + c] = r; v1 = r; v2 = 0.0; }
    else { K.k2[(size_t)e0 * n + c] = r; v1 = K.k1[(size_t)e0 * n + c]; v2 = r; }
    double siegtmp = F.rgpn[c] * F.siegn[c] + a1 * dt * v1 + a2 * dt * v2;
    double rgpnew = K.xrgp[c];
    double tmp = 1.0 / rgpnew;
    double sieg = siegtmp * tmp;
    double yg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) yg[ig] = GAS(F.ygc, c, ig);
    double tg = F.tg[c], cg;
    caloric_eosg(P, cg, tg, yg, sieg);
    double mg = 0.0;
    for (int ig = 0; ig < P.ng; ++ig) mg = mg + GAS(F.xgc, c, ig) * P.gmw[P.gas_type[ig]];
    F.sieg[c] = sieg;
    F.tg[c] = tg;
    F.cg[c] = cg;
    F.p[c] = F.rog[c] * tg * P.rgas / mg;
    // commit
    F.rgp[c] = rgpnew;
    F.ep[c] = K.xep[c];
    F.ug[c] = K.xug[c];
    if (D == 3) F.vg[c] = K.xvg[c];
    F.wg[c] = K.xwg[c];
    for (int is = 1; is <= P.ns; ++is) F.rlk[(size_t)(is - 1) * n + c] = K.xrlk[(size_t)(is - 1) * n + c];
}

// ---- the wavefront on hyperplane-ordered records -----------------------------
// Of a cell's gas-enthalpy update only the pressures of its west, south and
// bottom neighbours come from the wavefront itself; everything else is known
// once the stage kernel has run.  k_rk3_wave_pre computes those parts once
// per stage in parallel and stores them as records ordered hyperplane by
// hyperplane (interior fluid cells only), so that the wavefront reads them
// coalesced and takes the three neighbour pressures from the previous
// hyperplane's slice of pnew, which stays in L2.  The arithmetic and its
// order are those of rhs_gas_enth and k_rk3_wave.
struct Wave {
    const int *order;   // record position -> cell
    const int *pos_of;  // cell -> record position, -1 for cells without a record
    const int *src;     // [3][npos]: record of the W / S / B neighbour when it is a fluid cell, else -1
    const int *start;   // hyperplane dmin + q holds records start[q] .. start[q + 1] - 1
    double *rec;        // [WR_YG + ng][npos]
    double *pnew;       // new pressure per record
    int npos, nplanes, dmin;
};
// record fields; the wavefront's results (WR_O*) are stored in record order
// too and scattered to the cell arrays by k_rk3_wave_post
enum { WR_OR, WR_OSIEG, WR_OTG, WR_OCG, WR_AX, WR_AY, WR_AZ, WR_PE, WR_PN, WR_PT, WR_PW, WR_PS, WR_PB, WR_R0, WR_EP,
       WR_SP, WR_INV, WR_TG, WR_ROG, WR_MG, WR_YG };

// the non-recurrent part of every record, then the commit of the values
// k_rk3_stage parked (nothing of this stage reads the old ones afterwards).
// One thread per cell in cell order, so that the reads coalesce; the record
// stores scatter, but the records of one hyperplane's neighbouring cells
// (i - 1, j + 1, k) are written a few rows apart in time and meet in L2.
template <int D>
__global__ void k_rk3_wave_pre(Prm P, Fld F, RkF K, Wave W, double dt, int stage) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    const int pos = W.pos_of[c];
    if (pos < 0) return;
    Cell<D> q;
    cell_of<D>(P, c, q);
    const size_t n = P.ncell, np = W.npos;
    const int i = q.i, j = q.j, k = q.k, e0 = (D == 3 ? 4 : 3) * P.nph;
    auto R = [&](int f) -> double & { return W.rec[(size_t)f * np + pos]; };
    const double *dx = P.dx, *dz = P.dz;
    // lower-face gas velocities as the wavefront sees them: new (parked)
    // where that neighbour is a record, committed one hyperplane earlier
    const double ugw = W.src[pos] >= 0 ? K.xug[q.rw] : F.ug[q.rw];
    const double wgb = W.src[2 * np + pos] >= 0 ? K.xwg[q.rb] : F.wg[q.rb];
    double indxc = 1.0 / (dx[i] + (dx[i + 1] + dx[i - 1]) * 0.5);
    double indyc = 0.0;
    double indzc = 1.0 / (dz[k] + (dz[k + 1] + dz[k - 1]) * 0.5);
    double ugc = 0.5 * (F.ug[c] + ugw);
    double vgc = 0.0;
    double wgc = 0.5 * (F.wg[c] + wgb);
    if (D == 3) {
        const double vgs = W.src[np + pos] >= 0 ? K.xvg[q.rs] : F.vg[q.rs];
        indyc = 1.0 / (P.dy[j] + (P.dy[j + 1] + P.dy[j - 1]) * 0.5);
        vgc = 0.5 * (F.vg[c] + vgs);
    }
    R(WR_AX) = indxc * ugc;
    R(WR_AY) = indyc * vgc;
    R(WR_AZ) = indzc * wgc;
    // the old pressures: E / N / T are still old when the cell is reached,
    // W / S / B are replaced by the wavefront where they are records
    R(WR_PE) = F.p[q.me];
    R(WR_PN) = D == 3 ? F.p[q.mn] : 0.0;
    R(WR_PT) = F.p[q.mt];
    R(WR_PW) = F.p[q.mw];
    R(WR_PS) = D == 3 ? F.p[q.ms] : 0.0;
    R(WR_PB) = F.p[q.mb];
    double tmp = enth_div<D>(P, F, q, 0);
    double r = 0.0;
    r = r - tmp;
    tmp = 1.0 / dt;
    r = r + F.ep[c] * (F.p[c] - F.pn[c]) * tmp;
    R(WR_R0) = r;
    R(WR_EP) = F.ep[c];
    double sp = F.rgpn[c] * F.siegn[c];
    if (stage == 2) sp = sp + 0.25 * dt * K.k1[(size_t)e0 * n + c];
    R(WR_SP) = sp;
    R(WR_INV) = 1.0 / K.xrgp[c];
    R(WR_TG) = F.tg[c];
    R(WR_ROG) = F.rog[c];
    double mg = 0.0;
    for (int ig = 0; ig < P.ng; ++ig) mg = mg + GAS(F.xgc, c, ig) * P.gmw[P.gas_type[ig]];
    R(WR_MG) = mg;
    for (int ig = 0; ig < P.ng; ++ig) R(WR_YG + ig) = GAS(F.ygc, c, ig);
    F.rgp[c] = K.xrgp[c];
    F.ep[c] = K.xep[c];
    F.ug[c] = K.xug[c];
    if (D == 3) F.vg[c] = K.xvg[c];
    F.wg[c] = K.xwg[c];
    for (int is = 1; is <= P.ns; ++is) F.rlk[(size_t)(is - 1) * n + c] = K.xrlk[(size_t)(is - 1) * n + c];
}

// the inputs of one record
struct WaveIn {
    double ax, ay, az, pe, pn, pt, pw, ps, pb, r0, ep, sp, inv, tg, rog, mg, yg[PDAC_MAXG];
    int sw, ss, sb;
};

template <int D>
__device__ __forceinline__ void wave_load(const Prm &P, const Wave &W, int pos, WaveIn &v) {
    const size_t np = W.npos;
    auto R = [&](int f) { return W.rec[(size_t)f * np + pos]; };
    v.ax = R(WR_AX); v.ay = D == 3 ? R(WR_AY) : 0.0; v.az = R(WR_AZ);
    v.pe = R(WR_PE); v.pn = D == 3 ? R(WR_PN) : 0.0; v.pt = R(WR_PT);
    v.pw = R(WR_PW); v.ps = D == 3 ? R(WR_PS) : 0.0; v.pb = R(WR_PB);
    v.r0 = R(WR_R0); v.ep = R(WR_EP); v.sp = R(WR_SP); v.inv = R(WR_INV); v.tg = R(WR_TG); v.rog = R(WR_ROG);
    v.mg = R(WR_MG);
    for (int ig = 0; ig < P.ng; ++ig) v.yg[ig] = R(WR_YG + ig);
    v.sw = W.src[pos]; v.ss = D == 3 ? W.src[np + pos] : -1; v.sb = W.src[2 * np + pos];
}

// the recurrent part: neighbour pressures, right-hand side, enthalpy,
// temperature and pressure of one record; stores in record order only
template <int D>
__device__ __forceinline__ void wave_solve(const Prm &P, const Wave &W, const WaveIn &v, int pos, double a1dt,
                                           double a2dt, int stage) {
    const double pw = v.sw >= 0 ? __ldcg(W.pnew + v.sw) : v.pw;
    const double pb = v.sb >= 0 ? __ldcg(W.pnew + v.sb) : v.pb;
    double dpxyz = 0.0;
    dpxyz = dpxyz + v.ax * (v.pe - pw);
    if (D == 3) {
        const double ps = v.ss >= 0 ? __ldcg(W.pnew + v.ss) : v.ps;
        dpxyz = dpxyz + v.ay * (v.pn - ps);
    } else {
        dpxyz = dpxyz + 0.0;
    }
    dpxyz = dpxyz + v.az * (v.pt - pb);
    const double r = v.r0 + v.ep * dpxyz;
    const double siegtmp = stage == 1 ? v.sp + a1dt * r + a2dt * 0.0 : v.sp + a2dt * r;
    const double sieg = siegtmp * v.inv;
    double tg = v.tg, cg;
    caloric_eosg(P, cg, tg, v.yg, sieg);
    const double p = v.rog * tg * P.rgas / v.mg;
    const size_t np = W.npos;
    __stcg(W.pnew + pos, p);
    W.rec[(size_t)WR_OR * np + pos] = r;
    W.rec[(size_t)WR_OSIEG * np + pos] = sieg;
    W.rec[(size_t)WR_OTG * np + pos] = tg;
    W.rec[(size_t)WR_OCG * np + pos] = cg;
}

// every hyperplane of a stage in one cooperative launch over the records: a
// grid-wide barrier separates the hyperplanes (all blocks are co-resident,
// so it always completes) and the neighbour pressures of the previous
// hyperplane are read past L1.  When the grid covers the widest hyperplane
// (ONE) a thread holds at most one record per hyperplane and loads the next
// one before the barrier, which leaves only the three neighbour pressures on
// the critical path after it.
template <int D, bool ONE>
__global__ void __launch_bounds__(128) k_rk3_wave_rec(Prm P, Wave W, double dt, int stage) {
    namespace cg = cooperative_groups;
    cg::grid_group g = cg::this_grid();
    const int nthr = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const double a1dt = (stage == 1 ? 1.0 : 0.25) * dt, a2dt = (stage == 1 ? 0.0 : 0.25) * dt;
    if (ONE) {
        WaveIn v;
        int pos = W.start[0] + tid;
        bool have = pos < W.start[1];
        if (have) wave_load<D>(P, W, pos, v);
        for (int q = 0; q < W.nplanes; ++q) {
            if (have) wave_solve<D>(P, W, v, pos, a1dt, a2dt, stage);
            if (q + 1 < W.nplanes) {
                pos = W.start[q + 1] + tid;
                have = pos < W.start[q + 2];
                if (have) wave_load<D>(P, W, pos, v);
            }
            g.sync();
        }
    } else {
        for (int q = 0; q < W.nplanes; ++q) {
            const int end = W.start[q + 1];
            for (int pos = W.start[q] + tid; pos < end; pos += nthr) {
                WaveIn v;
                wave_load<D>(P, W, pos, v);
                wave_solve<D>(P, W, v, pos, a1dt, a2dt, stage);
            }
            g.sync();
        }
    }
}

// the wavefront's results to the cell arrays
template <int D>
__global__ void k_rk3_wave_post(Prm P, Fld F, RkF K, Wave W, int stage) {
    int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= W.npos) return;
    const size_t np = W.npos, n = P.ncell;
    const int c = W.order[pos], e0 = (D == 3 ? 4 : 3) * P.nph;
    (stage == 1 ? K.k1 : K.k2)[(size_t)e0 * n + c] = W.rec[(size_t)WR_OR * np + pos];
    F.sieg[c] = W.rec[(size_t)WR_OSIEG * np + pos];
    F.tg[c] = W.rec[(size_t)WR_OTG * np + pos];
    F.cg[c] = W.rec[(size_t)WR_OCG * np + pos];
    F.p[c] = W.pnew[pos];
}

// stage 3 and the final combination rhs3 = init + dt (k1 + k2 + 4 k3) / 6
// (explicit_solver.f:1092-1114), written over k1
template <int NP, int D>
__global__ void k_rk3_final_rhs(Prm P, Fld F, RkF K, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    Cell<D> q;
    cell_of<D>(P, c, q);
    const size_t n = P.ncell;
    const int ns = nphases<NP>(P) - 1, nph = ns + 1;
    const double b1 = 1.0 / 6.0, b2 = 1.0 / 6.0, b3 = 4.0 / 6.0;
    auto fin = [&](int eq, double init, double k3) {
        double *p1 = K.k1 + (size_t)eq * n + c;
        double v2 = K.k2[(size_t)eq * n + c];
        *p1 = init + b1 * dt * *p1 + b2 * dt * v2 + b3 * dt * k3;
    };
    for (int ph = 0; ph <= ns; ++ph) fin(ph, init_row<D>(P, F, K, q, 0, ph, 0), rhs_mass<D>(P, F, q, ph));
    for (int ax = 0; ax < 3; ++ax) {
        if (D == 2 && ax == 1) continue;
        const int blk = D == 3 ? ax + 1 : (ax == 0 ? 1 : 2);
        for (int ph = 0; ph <= ns; ++ph)
            fin(blk * nph + ph, init_row<D>(P, F, K, q, 1, ph, ax), rhs_mom<D>(P, F, q, ph, ax));
    }
    const int e0 = (D == 3 ? 4 : 3) * nph;
    fin(e0, init_row<D>(P, F, K, q, 2, 0, 0), rhs_gas_enth<D>(P, F, q, dt));
    for (int is = 1; is <= ns; ++is) {
        double r = 0.0;
        r = r - enth_div<D>(P, F, q, is);
        fin(e0 + is, init_row<D>(P, F, K, q, 2, is, 0), r);
    }
}

// the densities of the final ODE solve (explicit_solver.f:1116-1143) and
// compute_physical_coeff for every fluid cell
template <int NP, int D>
__global__ void k_rk3_final_phys(Prm P, Fld F, RkF K, double dt) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    const size_t n = P.ncell;
    F.rgp[c] = K.k1[c];
    for (int is = 1; is <= P.ns; ++is) {
        double t = K.k1[(size_t)is * n + c];
        F.rlk[(size_t)(is - 1) * n + c] = (0.0 < t) ? t : 0.0;
    }
    Cell<D> q;
    cell_of<D>(P, c, q);
    phys_coeff<NP, D>(P, F, K, q, dt);
}

// compute_linear_systems + solve_linear_systems + the closure relations of
// explicit_iter for one fluid cell; caloric failures add to counters[1]
template <int NP, int D>
__global__ void k_rk3_solve(Prm P, Fld F, RkF K, double dt) {
    constexpr int MP = Sys<NP>::M;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell || !fluid(P, c)) return;
    Cell<D> q;
    cell_of<D>(P, c, q);
    const size_t n = P.ncell;
    const int ns = nphases<NP>(P) - 1, nph = ns + 1;
    const double alpha = P.alpha;
    auto R3 = [&](int eq) { return K.k1[(size_t)eq * n + c]; };
    // momentum, one axis at a time: matrix, Crank-Nicolson part of the
    // interphase terms on the right-hand side, Gauss-Jordan solve when the
    // raw neighbour along the axis is fluid
    for (int ax = 0; ax < 3; ++ax) {
        if (D == 2 && ax == 1) continue;
        const int blk = D == 3 ? ax + 1 : (ax == 0 ? 1 : 2);
        double d0, d1;
        int nb, raw;
        const double *app;
        double *gS, *sS;
        if (ax == 0) { d0 = P.dx[q.i]; d1 = P.dx[q.i + 1]; nb = q.me; raw = q.re; app = F.appu; gS = F.ug; sS = F.us; }
        else if (ax == 1) { d0 = P.dy[q.j]; d1 = P.dy[q.j + 1]; nb = q.mn; raw = q.rn; app = F.appv; gS = F.vg; sS = F.vs; }
        else { d0 = P.dz[q.k]; d1 = P.dz[q.k + 1]; nb = q.mt; raw = q.rt; app = F.appw; gS = F.wg; sS = F.ws; }
        const double inp = 1.0 / (d0 + d1);
        auto AP = [&](int cell, int ls) { return APP(app, cell, ls); };
        auto SV = [&](int is) { return sS[(size_t)(is - 1) * n + c]; };
        double a[MP][MP], b[MP];
        a[1][1] = (d0 * F.rgp[nb] + d1 * F.rgp[c]) * inp;
        a[1][1] = a[1][1] + alpha * (d0 * AP(nb, 1) + d1 * AP(c, 1)) * inp;
        for (int l = 2; l <= nph; ++l) {
            int ls1 = l * (l - 1) / 2;
            for (int ll = 1; ll <= l; ++ll) {
                int ls = ls1 + ll;
                a[l][ll] = alpha * (d0 * AP(nb, ls) + d1 * AP(c, ls)) * inp;
                a[ll][l] = a[l][ll];
            }
            const double *rl = F.rlk + (size_t)(l - 2) * n;
            a[l][l] = a[l][l] + (d0 * rl[nb] + d1 * rl[c]) * inp;
        }
        for (int l = 1; l <= nph; ++l) b[l] = R3(blk * nph + l - 1);
        if (alpha < 1.0) {
            const double ca = 1.0 - alpha;
            b[1] = b[1] - ca * (d0 * AP(nb, 1) + d1 * AP(c, 1)) * inp * gS[c];
            for (int l = 2; l <= nph; ++l) {
                int ls1 = l * (l - 1) / 2;
                for (int ll = 1; ll <= l; ++ll) {
                    int ls = ls1 + ll;
                    if (ll == 1) {
                        b[1] = b[1] - ca * (d0 * AP(nb, ls) + d1 * AP(c, ls)) * inp * SV(l - 1);
                        b[l] = b[l] - ca * (d0 * AP(nb, ls) + d1 * AP(c, ls)) * inp * gS[c];
                    } else if (ll == l) {
                        b[l] = b[l] - ca * (d0 * AP(nb, ls) + d1 * AP(c, ls)) * inp * SV(l - 1);
                    } else {
                        b[l] = b[l] - ca * (d0 * AP(nb, ls) + d1 * AP(c, ls)) * inp * SV(ll - 1);
                        // the reference uses the cell's own interphase term twice here
                        b[ll] = b[ll] - ca * (d0 * AP(c, ls) + d1 * AP(c, ls)) * inp * SV(l - 1);
                    }
                }
            }
        }
        if (fluid(P, raw)) {
            gauss_jordan_t<NP, MP>(P, a, b);
            gS[c] = b[1];
            for (int l = 2; l <= nph; ++l) sS[(size_t)(l - 2) * n + c] = b[l];
        }
    }
    // enthalpies
    const int e0 = (D == 3 ? 4 : 3) * nph;
    double bt[MP], hvv[MP];
    for (int is = 1; is <= nph; ++is) bt[is] = R3(e0 + is - 1);
    for (int is = 1; is <= ns; ++is) hvv[is] = K.hv[(size_t)(is - 1) * n + c];
    const double cgc = F.cg[c];
    if (alpha < 1.0) {
        for (int is = 1; is <= ns; ++is) {
            double tsv = F.ts[(size_t)(is - 1) * n + c];
            bt[1] = bt[1] + (1.0 - alpha) * dt * hvv[is] * (tsv - F.tg[c]);
            bt[is + 1] = bt[is + 1] + (1.0 - alpha) * dt * hvv[is] * (F.tg[c] - tsv);
        }
    }
    double rmin = F.rlk[c];
    for (int is = 2; is <= ns; ++is) rmin = fmin(rmin, F.rlk[(size_t)(is - 1) * n + c]);
    double sieg;
    double sies[MP];
    if (rmin > RK3_LIMIT) {
        double cgammag = F.rgp[c], rhsg = bt[1];
        double num = rhsg, den = cgammag;
        for (int is = 1; is <= ns; ++is) {
            double cgam = F.rlk[(size_t)(is - 1) * n + c];
            double alfak = hvv[is] * dt / P.cps[is], alfag = hvv[is] * dt / cgc;
            double t = cgam + alfak;
            t = 1.0 / t;
            double coeff = cgam * t;
            num = num + bt[is + 1];
            num = num - coeff * bt[is + 1];
            den = den + coeff * alfag;
        }
        den = 1.0 / den;
        sieg = num * den;
        for (int is = 1; is <= ns; ++is) {
            double cgam = F.rlk[(size_t)(is - 1) * n + c];
            double alfak = hvv[is] * dt / P.cps[is], alfag = hvv[is] * dt / cgc;
            double nm = bt[is + 1] + alfag * sieg;
            double t = cgam + alfak;
            double dn = 1.0 / t;
            sies[is] = nm * dn;
        }
    } else {
        double at[MP][MP];
        at[1][1] = F.rgp[c];
        for (int is = 1; is <= ns; ++is) {
            int is1 = is + 1;
            double ck = P.cps[is];
            at[1][1] = at[1][1] + alpha * dt * hvv[is] / cgc;
            at[is1][1] = -alpha * dt * hvv[is] / cgc;
            at[1][is1] = -alpha * dt * hvv[is] / ck;
            at[is1][is1] = F.rlk[(size_t)(is - 1) * n + c] + alpha * dt * hvv[is] / ck;
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
        sieg = bt[1];
        for (int is = 1; is <= ns; ++is) sies[is] = bt[is + 1];
    }
    // closure: caloric_eosg, caloric_eosl, volume fraction, density, pressure
    double yg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) yg[ig] = GAS(F.ygc, c, ig);
    double tg = F.tg[c], cg;
    int info = caloric_eosg(P, cg, tg, yg, sieg);
    F.sieg[c] = sieg;
    F.tg[c] = tg;
    F.cg[c] = cg;
    double epstot = 0.0;
    for (int is = 1; is <= ns; ++is) {
        size_t off = (size_t)(is - 1) * n;
        F.sies[off + c] = sies[is];
        double t = 0.0 + (sies[is] - 0.0) / P.cps[is];
        F.ts[off + c] = t;
        if (t < 0.0) info++;
        double epsstar = F.rlk[off + c] * P.inrl[is];
        epstot = epstot + epsstar;
    }
    double ep = 1.0 - epstot;
    F.ep[c] = ep;
    double rog = F.rgp[c] / ep;
    F.rog[c] = rog;
    double mg = 0.0;
    for (int ig = 0; ig < P.ng; ++ig) mg = mg + GAS(F.xgc, c, ig) * P.gmw[P.gas_type[ig]];
    F.p[c] = rog * tg * P.rgas / mg;
    if (info) atomicAdd(&F.counters[1], info);
}

}  // namespace pdac

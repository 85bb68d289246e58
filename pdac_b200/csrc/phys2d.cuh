// phys2d.cuh -- per-cell device physics of the 2D (x|r, z) hot path.
//
// Every function restates the reference routine it names (file:line in its
// comment) with the same floating-point operation order; Fortran REAL(4)
// literals appear as (double)x.f.  Indices i, k are the reference's 1-based
// cell indices; flat cell numbers are 0-based.
#pragma once
#include "common.cuh"

namespace pdac {

// ---- neighbour indices -----------------------------------------------------
// Raw neighbours (myijk): offsets clamped into the domain, which is what
// ghost.f:527-560 stores for cells of the interior.
struct Raw2 {
    int c, e, w, t, b, et, wt, eb, wb, ee, ww, tt, bb, eet, ett, eee, ttt;
};
// Boundary-remapped neighbours (myinds), ghost.f:963-1277.
struct Rem2 {
    int e, w, t, b, et, wt, eb, wb, ee, ww, tt, bb, eet, ett, eee, ttt;
};

__device__ __forceinline__ int at2(const Prm &P, int i, int k) { return (i - 1) + P.nx * (k - 1); }

__device__ __forceinline__ void raw2(const Prm &P, int i, int k, Raw2 &R) {
    auto f = [&](int di, int dk) { return at2(P, clampi(i + di, 1, P.nx), clampi(k + dk, 1, P.nz)); };
    R.c = at2(P, i, k);
    R.e = f(1, 0); R.w = f(-1, 0); R.t = f(0, 1); R.b = f(0, -1);
    R.et = f(1, 1); R.wt = f(-1, 1); R.eb = f(1, -1); R.wb = f(-1, -1);
    R.ee = f(2, 0); R.ww = f(-2, 0); R.tt = f(0, 2); R.bb = f(0, -2);
    R.eet = f(2, 1); R.ett = f(1, 2); R.eee = f(3, 0); R.ttt = f(0, 3);
}

// symmetric diagonal rule (ghost.f:990-1056): D a wall -> fall back on the
// axis cells A, B next to it, or the base cell
__device__ __forceinline__ int diag_rule(const int *fl, int d, int a, int b, int base, bool trig) {
    if (!trig) return d;
    bool wa = is_wall(fl[a]), wb = is_wall(fl[b]);
    if (wa && wb) return base;
    if (wa) return b;
    if (wb) return a;
    return base;
}

__device__ __forceinline__ void rem2(const Prm &P, int i, int k, const Raw2 &R, Rem2 &M) {
    const int *fl = P.flag;
    int c = R.c;
    M.e = is_wallf(fl[R.e]) ? c : R.e;
    M.w = is_wallf(fl[R.w]) ? c : R.w;
    M.t = is_wallf(fl[R.t]) ? c : R.t;
    M.b = is_wallf(fl[R.b]) ? c : R.b;
    M.wt = diag_rule(fl, R.wt, R.w, R.t, c, is_wall(fl[R.wt]));
    M.eb = diag_rule(fl, R.eb, R.e, R.b, c, is_wall(fl[R.eb]));
    M.et = diag_rule(fl, R.et, R.e, R.t, c, is_wall(fl[R.et]));
    M.wb = diag_rule(fl, R.wb, R.w, R.b, c, is_wall(fl[R.wb]));
    M.ee = is_wallf(fl[R.ee]) ? R.e : R.ee;
    if (i == P.nx - 1) M.ee = M.e;
    M.tt = is_wallf(fl[R.tt]) ? R.t : R.tt;
    if (k == P.nz - 1) M.tt = M.t;
    M.ww = is_wallf(fl[R.ww]) ? R.w : R.ww;
    if (i == 2) M.ww = M.w;
    M.bb = is_wallf(fl[R.bb]) ? R.b : R.bb;
    if (k == 2) M.bb = M.b;
    M.eet = diag_rule(fl, R.eet, R.et, R.ee, R.e, is_wallf(fl[R.eet]));
    if (i == P.nx - 1) M.eet = M.et;
    M.ett = diag_rule(fl, R.ett, R.et, R.tt, R.t, is_wallf(fl[R.ett]));
    if (k == P.nz - 1) M.ett = M.et;
    M.ttt = is_wallf(fl[R.ttt]) ? R.tt : R.ttt;
    if (k == P.nz - 1) M.ttt = M.t;
    if (k == P.nz - 2) M.ttt = M.tt;
    M.eee = is_wallf(fl[R.eee]) ? R.ee : R.eee;
    if (i == P.nx - 1) M.eee = M.e;
    if (i == P.nx - 2) M.eee = M.ee;
}

// ---- stencils (subscr.f TYPE(stencil)) -------------------------------------
template <typename Real>
struct St2T {
    Real c, e, w, t, b, ee, ww, tt, bb, et, wt, eb, eet, ett, eee, ttt;
};
using St = St2T<double>;
template <typename T, typename Real>
__device__ __forceinline__ void nb2(St2T<Real> &s, const T *a, const Raw2 &R, const Rem2 &M) {  // subscr.f nb
    s.c = a[R.c]; s.e = a[M.e]; s.t = a[M.t]; s.w = a[M.w]; s.b = a[M.b];
    s.et = a[M.et]; s.wt = a[M.wt]; s.eb = a[M.eb]; s.ee = a[M.ee]; s.tt = a[M.tt];
    s.eet = a[M.eet]; s.ett = a[M.ett]; s.eee = a[M.eee]; s.ttt = a[M.ttt];
    s.ww = 0; s.bb = 0;
}
template <typename T, typename Real>
__device__ __forceinline__ void rnb2(St2T<Real> &s, const T *a, const Raw2 &R) {  // subscr.f rnb_r
    s.c = a[R.c]; s.e = a[R.e]; s.t = a[R.t]; s.w = a[R.w]; s.b = a[R.b];
    s.wt = a[R.wt]; s.et = a[R.et]; s.eb = a[R.eb]; s.ee = a[R.ee]; s.tt = a[R.tt];
    s.eet = a[R.eet]; s.ett = a[R.ett]; s.eee = a[R.eee]; s.ttt = a[R.ttt];
    s.ww = 0; s.bb = 0;
}

// Velocity masks of tilde's flux stencils in boundary-layer and immersed
// cells with immersed boundaries (tilde.f:896-945, subscr.f:1548-1582): each
// raw stencil velocity times the open-face factor of its own cell (bit 1 =
// b_e_ for u, 4 = b_t_ for w).  The members the reference leaves undefined
// are not read by the first-order fluxes such cells take.
__device__ __forceinline__ double ib_open(const Prm &P, int cell, int bit) {
    return (__ldg(P.ib_faces + cell) & bit) ? 1.0 : 0.0;
}
__device__ __forceinline__ bool ib_masked(const Prm &P, int c) {
    return P.immb && (P.flag[c] == BL_CELL || P.flag[c] == IMMB);
}
template <typename Real>
__device__ __forceinline__ void ib_mask2(const Prm &P, St2T<Real> &s, const Raw2 &R, int bit) {
    s.c = s.c * Real(ib_open(P, R.c, bit)); s.e = s.e * Real(ib_open(P, R.e, bit)); s.w = s.w * Real(ib_open(P, R.w, bit));
    s.t = s.t * Real(ib_open(P, R.t, bit)); s.b = s.b * Real(ib_open(P, R.b, bit));
    s.ee = s.ee * Real(ib_open(P, R.ee, bit)); s.tt = s.tt * Real(ib_open(P, R.tt, bit));
    s.et = s.et * Real(ib_open(P, R.et, bit)); s.eb = s.eb * Real(ib_open(P, R.eb, bit)); s.wt = s.wt * Real(ib_open(P, R.wt, bit));
}
template <typename T, typename Real>
__device__ __forceinline__ void first_nb2(St2T<Real> &s, const T *a, const Raw2 &R, const Rem2 &M) {
    s.c = a[R.c]; s.e = a[M.e]; s.t = a[M.t]; s.w = a[M.w]; s.b = a[M.b];
}
template <typename T, typename Real>
__device__ __forceinline__ void first_rnb2(St2T<Real> &s, const T *a, const Raw2 &R) {
    s.c = a[R.c]; s.e = a[R.e]; s.t = a[R.t]; s.w = a[R.w]; s.b = a[R.b];
}
template <typename T, typename Real>
__device__ __forceinline__ void third_nb2(St2T<Real> &s, const T *a, const Rem2 &M) {
    s.ee = a[M.ee]; s.tt = a[M.tt]; s.ww = a[M.ww]; s.bb = a[M.bb];
}

// ---- limiters.f:14-56 --------------------------------------------------------
// Real is the arithmetic type of the flux pass (double, or float in the
// mixed-precision mode of the 3D flux kernels)
template <typename Real>
__device__ __forceinline__ Real limiter(int t, Real erre, double beta_) {
    const Real beta = Real(beta_);
    switch (t) {
    case 1: return fmax(Real(0.0), Real(2.0) * erre / (Real(1.0) + erre));
    case 2: return fmax(Real(0.0), fmin(erre, Real(1.0)));
    case 3: return fmax(fmax(Real(0.0), fmin(Real(2.0) * erre, Real(1.0))), fmin(erre, Real(2.0)));
    case 4: { Real bu = (Real(1.0) - beta) + beta * erre; return fmax(Real(0.0), fmin(fmin(Real(2.0) * erre, bu), Real(2.0))); }
    case 0: return (Real(1.0) - beta) + beta * erre;
    default: return Real(0.0);
    }
}

// ---- interp.f:14-320, members used in 2D -------------------------------------
template <typename Real>
__device__ __forceinline__ void interp_x2(const Prm &P, const St2T<Real> &f, int i, St2T<Real> &s) {
    const Real *dx = Met<Real>::dx(P);
    int ip2 = min(P.nx, i + 2), ip3 = min(P.nx, i + 3);
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i];
    Real indxpp = Met<Real>::hx(P)[i + 1], indxppp = Met<Real>::hx(P)[ip2];
    s.c = (dx[i + 1] * f.c + dx[i] * f.e) * indxp;
    s.e = (dx[ip2] * f.e + dx[i + 1] * f.ee) * indxpp;
    s.t = (dx[i + 1] * f.t + dx[i] * f.et) * indxp;
    s.w = (dx[i] * f.w + dx[i - 1] * f.c) * indxm;
    s.b = (dx[i + 1] * f.b + dx[i] * f.eb) * indxp;
    s.ee = (dx[ip2] * f.eee + dx[ip3] * f.ee) * indxppp;
    s.tt = (dx[i] * f.ett + dx[i + 1] * f.tt) * indxp;
}
template <typename Real>
__device__ __forceinline__ void interp_z2(const Prm &P, const St2T<Real> &f, int k, St2T<Real> &s) {
    const Real *dz = Met<Real>::dz(P);
    int kp2 = min(P.nz, k + 2), kp3 = min(P.nz, k + 3);
    Real indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k];
    Real indzpp = Met<Real>::hz(P)[k + 1], indzppp = Met<Real>::hz(P)[kp2];
    s.c = (dz[k + 1] * f.c + dz[k] * f.t) * indzp;
    s.e = (dz[k + 1] * f.e + dz[k] * f.et) * indzp;
    s.t = (dz[kp2] * f.t + dz[k + 1] * f.tt) * indzpp;
    s.w = (dz[k + 1] * f.w + dz[k] * f.wt) * indzp;
    s.b = (dz[k] * f.b + dz[k - 1] * f.c) * indzm;
    s.ee = (dz[k] * f.eet + dz[k + 1] * f.ee) * indzp;
    s.tt = (dz[kp2] * f.ttt + dz[kp3] * f.tt) * indzppp;
}

// ---- momentum fluxes, flux_u.f:230-340 and flux_w.f:220-356 -------------------
// W/B fluxes are produced only when that neighbour is not a fluid cell.
template <typename Real>
__device__ __forceinline__ void flu_2d(const Prm &P, Real &fe, Real &ft, Real &fw, Real &fb, bool dow, bool dob,
                                       const St2T<Real> &d, const St2T<Real> &u, const St2T<Real> &w, int i) {
    const Real *dx = Met<Real>::dx(P);
    Real indxp = Met<Real>::hx(P)[i], cs;
    if (dow) {
        cs = Real(0.5) * (u.c + u.w);
        fw = Real(0.5) * (cs - fabs(cs)) * d.c * u.c * Met<Real>::r(P)[i] + Real(0.5) * (cs + fabs(cs)) * d.w * u.w * Met<Real>::r(P)[i];
    }
    if (dob) {
        cs = (dx[i + 1] * w.b + dx[i] * w.eb) * indxp;
        fb = Real(0.5) * (cs - fabs(cs)) * d.c * u.c + Real(0.5) * (cs + fabs(cs)) * d.b * u.b;
    }
    cs = Real(0.5) * (u.c + u.e);
    fe = Real(0.5) * (cs - fabs(cs)) * d.e * u.e * Met<Real>::r(P)[i + 1] + Real(0.5) * (cs + fabs(cs)) * d.c * u.c * Met<Real>::r(P)[i + 1];
    cs = (dx[i + 1] * w.c + dx[i] * w.e) * indxp;
    ft = Real(0.5) * (cs - fabs(cs)) * d.t * u.t + Real(0.5) * (cs + fabs(cs)) * d.c * u.c;
}

template <typename Real>
__device__ __forceinline__ void muscl_flu_2d(const Prm &P, Real &fe, Real &ft, const St2T<Real> &d, const St2T<Real> &u, const St2T<Real> &w,
                                             int i, int k, bool doe, bool dot) {
    const Real *dx = Met<Real>::dx(P), *dz = Met<Real>::dz(P), *indx = Met<Real>::indx(P);
    int ip2 = min(P.nx, i + 2), kp2 = min(P.nz, k + 2);
    Real indxp = Met<Real>::hx(P)[i], indzm = Met<Real>::hz(P)[k - 1];
    Real indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real erre, incr = 0, cs, lim, upwnd, gradc;
    if (doe) {
        gradc = indx[i + 1] * (d.e * u.e - d.c * u.c);
        Real gradw = indx[i] * (d.c * u.c - d.w * u.w);
        Real grade = indx[ip2] * (d.ee * u.ee - d.e * u.e);
        erre = 0; cs = Real(0.5) * (u.c + u.e);
        if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = Real(0.5) * dx[i + 1]; }
        else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -Real(0.5) * dx[i + 1]; }
        lim = limiter(P.lv, erre, P.beta);
        upwnd = lim * gradc * incr;
        fe = fe + upwnd * cs * Met<Real>::r(P)[i + 1];
    }
    if (dot) {
        gradc = (d.t * u.t - d.c * u.c) * Real(2.0) * indzp;
        Real gradb = (d.c * u.c - d.b * u.b) * Real(2.0) * indzm;
        Real gradt = (d.tt * u.tt - d.t * u.t) * Real(2.0) * indzpp;
        erre = 0; cs = (dx[i + 1] * w.c + dx[i] * w.e) * indxp;
        if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = Real(0.5) * dz[k]; }
        else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -Real(0.5) * dz[k + 1]; }
        lim = limiter(P.lv, erre, P.beta);
        upwnd = lim * gradc * incr;
        ft = ft + upwnd * cs;
    }
}

template <typename Real>
__device__ __forceinline__ void flw_2d(const Prm &P, Real &fe, Real &ft, Real &fw, Real &fb, bool dow, bool dob,
                                       const St2T<Real> &d, const St2T<Real> &u, const St2T<Real> &w, int i, int k) {
    const Real *dz = Met<Real>::dz(P);
    Real indzp = Met<Real>::hz(P)[k], cs;
    if (dow) {
        cs = (u.wt * dz[k] + u.w * dz[k + 1]) * indzp;
        fw = Real(0.5) * d.w * w.w * (cs + fabs(cs)) * Met<Real>::rb(P)[i - 1] + Real(0.5) * d.c * w.c * (cs - fabs(cs)) * Met<Real>::rb(P)[i - 1];
    }
    if (dob) {
        cs = Real(0.5) * (w.c + w.b);
        fb = Real(0.5) * d.b * w.b * (cs + fabs(cs)) + Real(0.5) * d.c * w.c * (cs - fabs(cs));
    }
    cs = indzp * (u.c * dz[k + 1] + u.t * dz[k]);
    fe = Real(0.5) * d.c * w.c * (cs + fabs(cs)) * Met<Real>::rb(P)[i] + Real(0.5) * d.e * w.e * (cs - fabs(cs)) * Met<Real>::rb(P)[i];
    cs = Real(0.5) * (w.t + w.c);
    ft = Real(0.5) * d.c * w.c * (cs + fabs(cs)) + Real(0.5) * d.t * w.t * (cs - fabs(cs));
}

template <typename Real>
__device__ __forceinline__ void muscl_flw_2d(const Prm &P, Real &fe, Real &ft, const St2T<Real> &d, const St2T<Real> &u, const St2T<Real> &w,
                                             int i, int k, bool doe, bool dot) {
    const Real *dx = Met<Real>::dx(P), *dz = Met<Real>::dz(P), *indz = Met<Real>::indz(P);
    int ip2 = min(P.nx, i + 2), kp2 = min(P.nz, k + 2);
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i];
    Real indxpp = Met<Real>::hx(P)[i + 1], indzp = Met<Real>::hz(P)[k];
    Real erre, incr = 0, cs, lim, upwnd, gradc;
    if (doe) {
        gradc = Real(2.0) * indxp * (d.e * w.e - d.c * w.c);
        Real gradw = Real(2.0) * indxm * (d.c * w.c - d.w * w.w);
        Real grade = Real(2.0) * indxpp * (d.ee * w.ee - d.e * w.e);
        erre = 0; cs = indzp * (u.c * dz[k + 1] + u.t * dz[k]);
        if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = Real(0.5) * dx[i]; }
        else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -Real(0.5) * dx[i + 1]; }
        lim = limiter(P.lv, erre, P.beta);
        upwnd = lim * gradc * incr;
        fe = fe + upwnd * cs * Met<Real>::rb(P)[i];
    }
    if (dot) {
        gradc = (d.t * w.t - d.c * w.c) * indz[k + 1];
        Real gradb = (d.c * w.c - d.b * w.b) * indz[k];
        Real gradt = (d.tt * w.tt - d.t * w.t) * indz[kp2];
        erre = 0; cs = Real(0.5) * (w.t + w.c);
        if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = Real(0.5) * dz[k + 1]; }
        else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -Real(0.5) * dz[k + 1]; }
        lim = limiter(P.lv, erre, P.beta);
        upwnd = lim * gradc * incr;
        ft = ft + upwnd * cs;
    }
}

// ---- mass fluxes, flux_m.f:326-531 (masf_2d + fmas_2d), face by face ----------
// Each helper returns one face of the cell (i, k) as the reference computes it
// in that cell's call: first-order donor cell plus the MUSCL correction when
// `muscl_on` (cell flag == fluid) and the neighbour test of fmas holds.
template <typename Real>
struct MF2T { Real w, e, b, t; };
using MF2 = MF2T<double>;

template <typename Real>
__device__ __forceinline__ void massflux_2d(const Prm &P, const St2T<Real> &d, Real uw, Real uc, Real wb, Real wc,
                                            int i, int k, bool muscl_on, int flw, int fle, int flb, int flt, MF2T<Real> &f) {
    const Real *dx = Met<Real>::dx(P), *dz = Met<Real>::dz(P), *rb = Met<Real>::rb(P);
    Real cs;
    cs = uw; f.w = Real(0.5) * (cs - fabs(cs)) * d.c * rb[i - 1] + Real(0.5) * (cs + fabs(cs)) * d.w * rb[i - 1];
    cs = wb; f.b = Real(0.5) * (cs - fabs(cs)) * d.c + Real(0.5) * (cs + fabs(cs)) * d.b;
    cs = uc; f.e = Real(0.5) * (cs - fabs(cs)) * d.e * rb[i] + Real(0.5) * (cs + fabs(cs)) * d.c * rb[i];
    cs = wc; f.t = Real(0.5) * (cs - fabs(cs)) * d.t + Real(0.5) * (cs + fabs(cs)) * d.c;
    if (!muscl_on) return;
    int im2 = max(1, i - 2), ip2 = min(P.nx, i + 2), km2 = max(1, k - 2), kp2 = min(P.nz, k + 2);
    Real indxmm = Met<Real>::hx(P)[max(i - 2, 0)], indxm = Met<Real>::hx(P)[i - 1];
    Real indxp = Met<Real>::hx(P)[i], indxpp = Met<Real>::hx(P)[i + 1];
    Real indzmm = Met<Real>::hz(P)[max(k - 2, 0)], indzm = Met<Real>::hz(P)[k - 1];
    Real indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real gradc, gradw, grade, gradb, gradt, erre, incr = 0, lim, upwnd;
    // West
    gradc = Real(2.0) * indxm * (d.c - d.w);
    gradw = Real(2.0) * indxmm * (d.w - d.ww);
    grade = Real(2.0) * indxp * (d.e - d.c);
    lim = 0; erre = 0; cs = uw;
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = Real(0.5) * dx[i - 1]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -Real(0.5) * dx[i]; }
    if (i != 2 && flw == FLUID) lim = limiter(P.lm, erre, P.beta);
    upwnd = lim * gradc * incr;
    f.w = f.w + upwnd * cs * rb[i - 1];
    // East
    gradw = gradc; gradc = grade;
    grade = Real(2.0) * indxpp * (d.ee - d.e);
    lim = 0; erre = 0; cs = uc;
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = Real(0.5) * dx[i]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -Real(0.5) * dx[i + 1]; }
    if (i != P.nx - 1 && fle == FLUID) lim = limiter(P.lm, erre, P.beta);
    upwnd = lim * gradc * incr;
    f.e = f.e + upwnd * cs * rb[i];
    // Bottom
    gradc = Real(2.0) * indzm * (d.c - d.b);
    gradb = Real(2.0) * indzmm * (d.b - d.bb);
    gradt = Real(2.0) * indzp * (d.t - d.c);
    lim = 0; erre = 0; cs = wb;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = Real(0.5) * dz[k - 1]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -Real(0.5) * dz[k]; }
    if (k != 2 && flb == FLUID) lim = limiter(P.lm, erre, P.beta);
    upwnd = lim * gradc * incr;
    f.b = f.b + upwnd * cs;
    // Top
    gradb = gradc; gradc = gradt;
    gradt = Real(2.0) * indzpp * (d.tt - d.t);
    lim = 0; erre = 0; cs = wc;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = Real(0.5) * dz[k]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -Real(0.5) * dz[k + 1]; }
    if (k != P.nz - 1 && flt == FLUID) lim = limiter(P.lm, erre, P.beta);
    upwnd = lim * gradc * incr;
    f.t = f.t + upwnd * cs;
}

// ---- scalar fluxes, flux_sc.f:236-390 -------------------------------------------
template <typename Real>
__device__ __forceinline__ void fsc_2d(const Prm &P, Real &fe, Real &ft, Real &fw, Real &fb, bool dow, bool dob,
                                       const St2T<Real> &d, const St2T<Real> &f, Real uw, Real uc, Real wb, Real wc, int i) {
    const Real *rb = Met<Real>::rb(P);
    Real cs;
    if (dow) { cs = uw; fw = Real(0.5) * (cs - fabs(cs)) * d.c * f.c * rb[i - 1] + Real(0.5) * (cs + fabs(cs)) * d.w * f.w * rb[i - 1]; }
    if (dob) { cs = wb; fb = Real(0.5) * (cs - fabs(cs)) * d.c * f.c + Real(0.5) * (cs + fabs(cs)) * d.b * f.b; }
    cs = uc; fe = Real(0.5) * (cs - fabs(cs)) * d.e * f.e * rb[i] + Real(0.5) * (cs + fabs(cs)) * d.c * f.c * rb[i];
    cs = wc; ft = Real(0.5) * (cs - fabs(cs)) * d.t * f.t + Real(0.5) * (cs + fabs(cs)) * d.c * f.c;
}
template <typename Real>
__device__ __forceinline__ void muscl_fsc_2d(const Prm &P, Real &fe, Real &ft, const St2T<Real> &d, const St2T<Real> &f, Real uc,
                                             Real wc, int i, int k) {
    const Real *dx = Met<Real>::dx(P), *dz = Met<Real>::dz(P);
    int ip2 = min(P.nx, i + 2), kp2 = min(P.nz, k + 2);
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i], indxpp = Met<Real>::hx(P)[i + 1];
    Real indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real gradc = Real(2.0) * indxp * (d.e * f.e - d.c * f.c);
    Real gradw = Real(2.0) * indxm * (d.c * f.c - d.w * f.w);
    Real grade = Real(2.0) * indxpp * (d.ee * f.ee - d.e * f.e);
    Real lim = 0, erre = 0, incr = 0, cs = uc, upwnd;
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = Real(0.5) * dx[i]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -Real(0.5) * dx[i + 1]; }
    if (i != P.nx - 1) lim = limiter(P.lm, erre, P.beta);
    upwnd = lim * gradc * incr;
    fe = fe + upwnd * cs * Met<Real>::rb(P)[i];
    gradc = Real(2.0) * indzp * (d.t * f.t - d.c * f.c);
    Real gradb = Real(2.0) * indzm * (d.c * f.c - d.b * f.b);
    Real gradt = Real(2.0) * indzpp * (d.tt * f.tt - d.t * f.t);
    lim = 0; erre = 0; cs = wc;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = Real(0.5) * dz[k]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -Real(0.5) * dz[k + 1]; }
    if (k != P.nz - 1) lim = limiter(P.lm, erre, P.beta);
    upwnd = lim * gradc * incr;
    ft = ft + upwnd * cs;
}

// ---- hotc.f:12-82 (2D members) ---------------------------------------------------
template <typename Real>
__device__ __forceinline__ void hotc_2d(const Prm &P, Real &hfe, Real &hft, Real &hfw, Real &hfb, bool dow, bool dob,
                                        const St2T<Real> &ep, const St2T<Real> &tg, const St2T<Real> &ka, int i, int k) {
    const Real *dx = Met<Real>::dx(P), *dz = Met<Real>::dz(P);
    if (dow) {
        Real indxm = Met<Real>::hx(P)[i - 1];
        Real kmw = (dx[i - 1] * ka.c + dx[i] * ka.w) * indxm;
        Real epmw = (dx[i - 1] * ep.c + dx[i] * ep.w) * indxm;
        hfw = kmw * epmw * (tg.c - tg.w) * indxm * Real(2.0) * Met<Real>::rb(P)[i - 1];
    }
    if (dob) {
        Real indzm = Met<Real>::hz(P)[k - 1];
        Real kmb = (dz[k - 1] * ka.c + dz[k] * ka.b) * indzm;
        Real epmb = (dz[k - 1] * ep.c + dz[k] * ep.b) * indzm;
        hfb = kmb * epmb * (tg.c - tg.b) * indzm * Real(2.0);
    }
    Real indxp = Met<Real>::hx(P)[i];
    Real kme = (dx[i + 1] * ka.c + dx[i] * ka.e) * indxp;
    Real epme = (dx[i + 1] * ep.c + dx[i] * ep.e) * indxp;
    hfe = kme * epme * (tg.e - tg.c) * indxp * Real(2.0) * Met<Real>::rb(P)[i];
    Real indzp = Met<Real>::hz(P)[k];
    Real kmt = (dz[k + 1] * ka.c + dz[k] * ka.t) * indzp;
    Real epmt = (dz[k + 1] * ep.c + dz[k] * ep.t) * indzp;
    hft = kmt * epmt * (tg.t - tg.c) * indzp * Real(2.0);
}

// ---- closures ----------------------------------------------------------------
// visc.f:37-148
__device__ __forceinline__ void viscon(const Prm &P, double &mu, double &kap, const double *xg, double tg) {
    double mmug[PDAC_MAXG], ckg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) {
        int g = P.gas_type[ig];
        double tst = tg / P.mmugek[g];
        double om = 1.16145 * pdac_fp::pow(tst, -0.14874) + 0.52487 * pdac_fp::exp(-0.77320 * tst) + 2.16178 * pdac_fp::exp(-2.43787 * tst);
        double m = 1.0e3 * P.gmw[g];
        double v = 26.69 * sqrt(m * tg) / (P.mmugs[g] * P.mmugs[g] * om);
        mmug[ig] = v * 1.0e-7;
    }
    double t1 = tg, t2 = t1 * tg, t3 = t2 * tg;
    double tr = tg / 132.5;
    double trm1 = 1.0 / tr, trm2 = trm1 * trm1, trm3 = trm2 * trm1, trm4 = trm3 * trm1, trsrt = sqrt(tr);
    for (int ig = 0; ig < P.ng; ++ig) {
        switch (P.gas_type[ig]) {
        case 1: ckg[ig] = -3.273e-4 + 9.966e-5 * t1 - 3.743e-8 * t2 + 9.732e-12 * t3; break;
        case 2: ckg[ig] = 3.919e-4 + 9.816e-5 * t1 - 5.067e-8 * t2 + 1.504e-11 * t3; break;
        case 3: ckg[ig] = -7.215e-3 + 8.015e-5 * t1 + 5.477e-9 * t2 - 1.053e-11 * t3; break;
        case 4: ckg[ig] = 8.099e-3 + 6.689e-4 * t1 - 4.158e-7 * t2 + 1.562e-10 * t3; break;
        case 5: ckg[ig] = 7.341e-3 - 1.013e-5 * t1 + 1.801e-7 * t2 - 9.100e-11 * t3; break;
        case 6: ckg[ig] = 25.9778e-3 * (0.2395 * tr + 6.4977e-3 * trsrt + 1.0 - 1.92615 * trm1 + 2.00383 * trm2 -
                                        1.07553 * trm3 + 0.229414 * trm4); break;
        default: ckg[ig] = -8.086e-3 + 6.344e-5 * t1 - 1.382e-8 * t2 + 2.303e-12 * t3; break;
        }
    }
    mu = 0; kap = 0;
    for (int ig = 0; ig < P.ng; ++ig) {
        int g = P.gas_type[ig];
        double sum = 0;
        for (int jg = 0; jg < P.ng; ++jg) {
            int h = P.gas_type[jg];
            double aa = P.gmw[g] / P.gmw[h];
            double bb = mmug[ig] / mmug[jg];
            double cc = 1.0 + sqrt(bb) * pdac_fp::pow(aa, -0.25);
            double phij = cc * cc / sqrt(8.0 * (1.0 + aa));
            sum = sum + xg[jg] * phij;
        }
        double suminv = 1.0 / sum;
        mu = mu + xg[ig] * mmug[ig] * suminv;
        kap = kap + xg[ig] * ckg[ig] * suminv;
    }
}

// hcapgs.f:33-85, for one reference gas type g (1..7)
__device__ __forceinline__ double hcapg1(const Prm &P, int g, double tg) {
    double t1 = (P.icpc <= 1) ? P.tref : tg, t2 = t1 * t1, t3 = t1 * t2, c;
    switch (g) {
    case 1: c = (2.811e1 - 3.68e-6 * t1 + 1.746e-5 * t2 - 1.065e-8 * t3); break;
    case 2: c = (3.115e1 - 1.357e-2 * t1 + 2.680e-5 * t2 - 1.168e-8 * t3); break;
    case 3: c = (1.980e1 + 7.344e-2 * t1 - 5.602e-5 * t2 + 1.715e-8 * t3); break;
    case 4: c = (2.714e1 + 9.274e-3 * t1 - 1.381e-5 * t2 + 7.645e-9 * t3); break;
    case 5: c = (3.224e1 + 1.924e-3 * t1 + 1.055e-5 * t2 - 3.596e-9 * t3); break;
    case 6: c = (3.0413e1 - 1.059e-2 * t1 + 2.458e-5 * t2 - 1.135e-8 * t3); break;
    default: c = (2.385e1 + 6.699e-2 * t1 - 4.961e-5 * t2 + 1.328e-8 * t3); break;
    }
    c = c / P.gmw[g];
    if (P.icpc == 0) { if (g == 5) c = 1810.0; if (g == 6) c = 1004.0; }
    return c;
}

// eosg.f:114-137
__device__ __forceinline__ double thermal_eosg(const Prm &P, double tg, double p, const double *xg) {
    double mg = 0;
    for (int ig = 0; ig < P.ng; ++ig) mg = mg + xg[ig] * P.gmw[P.gas_type[ig]];
    return p / (P.rgas * tg) * mg;
}

// eosg.f:38-68
__device__ __forceinline__ void mole(const Prm &P, double *xg, const double *yg) {
    double mol = 0;
    for (int ig = 0; ig < P.ng; ++ig) mol = mol + yg[ig] / P.gmw[P.gas_type[ig]];
    double molinv = (fabs(mol) <= 1e-10) ? 0.0 : 1.0 / mol;
    for (int ig = 0; ig < P.ng; ++ig) xg[ig] = yg[ig] / P.gmw[P.gas_type[ig]] * molinv;
}

// eosg.f:139-223 (fixed-point caloric inversion, <= 2000 iterations)
__device__ __forceinline__ int caloric_eosg(const Prm &P, double &cgas, double &tg, const double *yg, double sieg) {
    int info = 1;
    for (int ii = 1; ii <= 2000; ++ii) {
        double tgnn = tg;
        cgas = 0;
        for (int ig = 0; ig < P.ng; ++ig) cgas = hcapg1(P, P.gas_type[ig], tg) * yg[ig] + cgas;
        tg = 0.0 + (sieg - 0.0) / cgas;
        if (fabs((tgnn - tg) / tgnn) <= 1.0e-8) { info = 0; break; }
    }
    if (tg <= 0.0) info = 1;
    return info;
}

// drag.f:60-157 (kdrags)
__device__ __forceinline__ double kdrags(const Prm &P, double du, double dv, double dw, double ep, double rgp, double rlk,
                                         double mug, int is) {
    double vrel = sqrt(du * du + dv * dv + dw * dw);
    double drag;
    {
        if (ep < 0.8) {
            double denom = 1.0 / (P.dk[is] * P.phis[is] * ep);
            drag = 150.0 * ep * rlk * P.inrl[is] * mug * denom + 1.75 * rgp * vrel;
            drag = drag * rlk * P.inrl[is] * denom;
        } else {
            double eps = rlk * P.inrl[is];
            double reynum = rgp * P.dk[is] * P.phis[is] * vrel / mug;
            double dc;
            if (reynum <= 1000.0) dc = (24.0 / reynum) * (1.0 + (double)0.15f * pdac_fp::pow(reynum, (double)0.687f));
            else dc = (double)0.43828814f;
            dc = fmin(dc, 1.0e4);
            drag = 0.75 * dc * eps / (P.dk[is] * P.phis[is]) * rgp * vrel;
            drag = drag * pdac_fp::pow(ep, (double)(-2.65f));
        }
    }
    return drag;
}

// drag.f:11-58 (sdrag)
__device__ __forceinline__ double sdrag(const Prm &P, double du, double dv, double dw, double ep, double rgp, double rlk,
                                        double mug, int is) {
    double vrel = sqrt(du * du + dv * dv + dw * dw);
    double drag;
    {
        double eps = rlk * P.inrl[is];
        double reynum = rgp * P.dk[is] * P.phis[is] * vrel / mug;
        double a = pdac_fp::pow(ep, (double)4.14f), b;
        if (ep <= (double)0.85f) b = (double)0.8f * pdac_fp::pow(ep, (double)1.28f);
        else b = pdac_fp::pow(ep, (double)2.65f);
        double vr = 0.5 * (a - (double)0.06f * reynum +
                           sqrt((double)0.0036f * reynum * reynum + (double)0.12f * reynum * (2.0 * b - a) + a * a));
        double dc = (0.63 + 4.8 / sqrt(reynum));
        dc = dc * dc;
        dc = fmin(dc, 1.0e4);
        drag = 0.75 * dc * eps / (P.dk[is] * P.phis[is]) * rgp * vrel;
        drag = drag / vr;
    }
    return drag;
}

// the drag law the run selects (tilde.f:617-623)
__device__ __forceinline__ double drag_coeff(const Prm &P, double du, double dv, double dw, double ep, double rgp, double rlk,
                                             double mug, int is) {
    return P.drag_model == 1 ? kdrags(P, du, dv, dw, ep, rgp, rlk, mug, is) : sdrag(P, du, dv, dw, ep, rgp, rlk, mug, is);
}

// drag.f:248-298
__device__ __forceinline__ double ppdrag(const Prm &P, const double *rlkc, int k, int kk) {
    int k1, k2;
    if (P.dk[k - 1] >= P.dk[kk - 1]) { k1 = k - 1; k2 = kk - 1; }
    else { k1 = kk - 1; k2 = k - 1; }
    double ep1 = rlkc[k1] * P.inrl[k1], ep2 = rlkc[k2] * P.inrl[k2], epsum = ep1 + ep2;
    if (ep1 > 0 && ep2 > 0) {
        double xbar = ep1 / epsum, epkl;
        if (xbar <= P.philim[k - 1][kk - 1]) epkl = P.epsl[k - 1][kk - 1] * xbar + P.phi[k2];
        else epkl = P.epsu[k - 1][kk - 1] * (1.0 - xbar) + P.phi[k1];
        double espo = 1.0 / 3.0;
        double m1 = pdac_fp::pow(epkl, espo), m2 = pdac_fp::pow(epsum, espo);
        double effe = (3.0 * m1 + m2) / (2.0 * (m1 - m2));
        return 1.0 * (1.0 + 1.0) * rlkc[k - 1] * rlkc[kk - 1] * P.dkf[k - 1][kk - 1] * effe;
    }
    return 0.0;
}

// hvs.f:9-83
__device__ __forceinline__ double hvs(const Prm &P, double rlk, double rog, double du, double dv, double dw, double mug,
                                      double kapg, double cg, int k) {
    if (rlk <= 0.0) return 0.0;
    double eps = rlk * P.inrl[k];
    double eps2 = eps * eps;
    double asurf = 6.0 * kapg * eps / (P.dk[k] * P.dk[k]);
    double vrel = sqrt(du * du + dv * dv + dw * dw);
    double reynum = P.dk[k] * vrel * rog / mug;
    double pranum = cg * mug / kapg;
    double pranumexp = pdac_fp::pow(pranum, 1.0 / 3.0);
    double nusselt = (2.0 + 5.0 * eps2) * (1.0 + 0.7 * pdac_fp::pow(reynum, 0.2) * pranumexp);
    nusselt = nusselt + (0.13 + 1.2 * eps2) * pdac_fp::pow(reynum, 0.7) * pranumexp;
    return nusselt * asurf;
}

// Gauss-Jordan with plim decoupling, matrix.f:351-391; a, b 1-based, n = nph
__device__ __forceinline__ void gauss_jordan(const Prm &P, double (*a)[PDAC_MAXP + 1], double *b) {
    int nph = P.nph;
    for (int l = 2; l <= nph; ++l) {
        if (fabs(a[l][l]) < P.plim[l - 1]) {
            for (int ll = 1; ll <= nph; ++ll) {
                a[ll][ll] = a[ll][ll] + a[l][ll];
                a[l][ll] = 0.0;
                a[ll][l] = 0.0;
            }
            b[l] = 0.0;
        }
    }
    for (int l = 1; l <= nph; ++l) {
        if (a[l][l] != 0.0) {
            int lp1 = l + 1;
            double div = 1.0 / a[l][l];
            for (int lj = lp1; lj <= nph; ++lj) a[l][lj] = a[l][lj] * div;
            b[l] = b[l] * div;
            a[l][l] = 0.0;
            for (int li = 1; li <= nph; ++li) {
                double amul = a[li][l];
                for (int lj = lp1; lj <= nph; ++lj) a[li][lj] = a[li][lj] - amul * a[l][lj];
                b[li] = b[li] - amul * b[l];
            }
        }
    }
}

}  // namespace pdac

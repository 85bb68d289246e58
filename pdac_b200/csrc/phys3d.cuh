// phys3d.cuh -- per-cell device physics of the 3D (x, y, z) hot path.
//
// Neighbour rules of ghost.f:1417-2100 (3D myinds), stencils of subscr.f,
// interpolation of interp.f, momentum fluxes flu_3d/flv_3d/flw_3d with their
// MUSCL corrections (flux_u.f:41-224, flux_v.f:41-222, flux_w.f:40-218), mass
// fluxes masf_3d/fmas_3d (flux_m.f:47-324), scalar fluxes fsc_3d/muscl_fsc_3d
// (flux_sc.f:44-234), hotc (hotc.f:12-82) and stress3D (visc.f:293-559), each
// with the reference's floating-point operation order.
#pragma once
#include "phys2d.cuh"

namespace pdac {

struct Raw3 {
    int c, e, w, n, s, t, b, ee, ww, nn, ss, tt, bb;
    int en, wn, es, ws, et, wt, nt, st, eb, wb, nb, sb;
    int eet, een, enn, nnt, ett, ntt, eee, nnn, ttt;
};
struct Rem3 {
    int e, w, n, s, t, b, ee, ww, nn, ss, tt, bb;
    int eb, wb, nb, sb;  // en, wn, es, ws, et, wt, nt, st are raw in 3D
    int eet, een, enn, nnt, ett, ntt, eee, nnn, ttt;
};

__device__ __forceinline__ int at3(const Prm &P, int i, int j, int k) { return (i - 1) + P.nx * ((j - 1) + P.ny * (k - 1)); }

__device__ __forceinline__ void raw3(const Prm &P, int i, int j, int k, Raw3 &R) {
    auto f = [&](int di, int dj, int dk) {
        return at3(P, clampi(i + di, 1, P.nx), clampi(j + dj, 1, P.ny), clampi(k + dk, 1, P.nz));
    };
    R.c = at3(P, i, j, k);
    R.e = f(1, 0, 0); R.w = f(-1, 0, 0); R.n = f(0, 1, 0); R.s = f(0, -1, 0); R.t = f(0, 0, 1); R.b = f(0, 0, -1);
    R.ee = f(2, 0, 0); R.ww = f(-2, 0, 0); R.nn = f(0, 2, 0); R.ss = f(0, -2, 0); R.tt = f(0, 0, 2); R.bb = f(0, 0, -2);
    R.en = f(1, 1, 0); R.wn = f(-1, 1, 0); R.es = f(1, -1, 0); R.ws = f(-1, -1, 0);
    R.et = f(1, 0, 1); R.wt = f(-1, 0, 1); R.nt = f(0, 1, 1); R.st = f(0, -1, 1);
    R.eb = f(1, 0, -1); R.wb = f(-1, 0, -1); R.nb = f(0, 1, -1); R.sb = f(0, -1, -1);
    R.eet = f(2, 0, 1); R.een = f(2, 1, 0); R.enn = f(1, 2, 0); R.nnt = f(0, 2, 1); R.ett = f(1, 0, 2); R.ntt = f(0, 1, 2);
    R.eee = f(3, 0, 0); R.nnn = f(0, 3, 0); R.ttt = f(0, 0, 3);
}

// the remapped neighbours (ghost.f:963-989 and the fall-backs of
// ghost.f:1417-2476) from the flags fl at the raw indices R: global indices
// with the flag array, or the indices of a shared-memory tile with the
// tile's copy of the flags
__device__ __forceinline__ void rem3_fl(const Prm &P, const int *fl, int i, int j, int k, const Raw3 &R, Rem3 &M) {
    int c = R.c;
    M.e = is_wallf(fl[R.e]) ? c : R.e;
    M.w = is_wallf(fl[R.w]) ? c : R.w;
    M.n = is_wallf(fl[R.n]) ? c : R.n;
    M.s = is_wallf(fl[R.s]) ? c : R.s;
    M.t = is_wallf(fl[R.t]) ? c : R.t;
    M.b = is_wallf(fl[R.b]) ? c : R.b;
    M.ee = is_wallf(fl[R.ee]) ? R.e : R.ee;
    if (i == P.nx - 1) M.ee = M.e;
    M.tt = is_wallf(fl[R.tt]) ? R.t : R.tt;
    if (k == P.nz - 1) M.tt = M.t;
    M.nn = is_wallf(fl[R.nn]) ? M.n : R.nn;  // ghost.f:1616-1621 falls back on the remapped ijkn
    if (j == P.ny - 1) M.nn = M.n;
    M.ss = is_wallf(fl[R.ss]) ? M.s : R.ss;
    if (j == 2) M.ss = M.s;
    M.ww = is_wallf(fl[R.ww]) ? R.w : R.ww;
    if (i == 2) M.ww = M.w;
    M.bb = is_wallf(fl[R.bb]) ? R.b : R.bb;
    if (k == 2) M.bb = M.b;
    M.eb = is_wallf(fl[R.eb]) ? R.e : R.eb;
    M.wb = is_wallf(fl[R.wb]) ? R.w : R.wb;
    M.nb = is_wallf(fl[R.nb]) ? R.n : R.nb;
    M.sb = is_wallf(fl[R.sb]) ? R.s : R.sb;
    M.eet = (i == P.nx - 1) ? R.et : R.eet;
    M.een = (i == P.nx - 1) ? R.en : R.een;
    M.enn = (j == P.ny - 1) ? R.en : R.enn;
    M.nnt = (j == P.ny - 1) ? R.nt : R.nnt;
    M.ett = (k == P.nz - 1) ? R.et : R.ett;
    M.ntt = (k == P.nz - 1) ? R.nt : R.ntt;
    M.ttt = is_wallf(fl[R.ttt]) ? R.tt : R.ttt;
    if (k == P.nz - 1) M.ttt = M.t;
    if (k == P.nz - 2) M.ttt = M.tt;
    M.eee = is_wallf(fl[R.eee]) ? R.ee : R.eee;
    if (i == P.nx - 1) M.eee = M.e;
    if (i == P.nx - 2) M.eee = M.ee;
    M.nnn = is_wallf(fl[R.nnn]) ? R.nn : R.nnn;
    if (j == P.ny - 1) M.nnn = M.n;
    if (j == P.ny - 2) M.nnn = M.nn;
}

__device__ __forceinline__ void rem3(const Prm &P, int i, int j, int k, const Raw3 &R, Rem3 &M) {
    rem3_fl(P, P.flag, i, j, k, R, M);
}

template <typename Real>
struct S3T {
    Real c, e, w, n, s, t, b, ee, ww, nn, ss, tt, bb;
    Real en, et, es, eb, nt, wn, nb, wt, st, eee, nnn, ttt, een, eet, enn, nnt, ett, ntt;
};
using S3 = S3T<double>;
template <typename T, typename Real>
__device__ __forceinline__ void nb3(S3T<Real> &s, const T *a, const Raw3 &R, const Rem3 &M) {
    s.c = a[R.c]; s.e = a[M.e]; s.w = a[M.w]; s.n = a[M.n]; s.s = a[M.s]; s.t = a[M.t]; s.b = a[M.b];
    s.ee = a[M.ee]; s.nn = a[M.nn]; s.tt = a[M.tt];
    s.en = a[R.en]; s.et = a[R.et]; s.es = a[R.es]; s.eb = a[M.eb]; s.nt = a[R.nt]; s.wn = a[R.wn];
    s.nb = a[M.nb]; s.wt = a[R.wt]; s.st = a[R.st];
    s.eee = a[M.eee]; s.nnn = a[M.nnn]; s.ttt = a[M.ttt];
    s.een = a[M.een]; s.eet = a[M.eet]; s.enn = a[M.enn]; s.nnt = a[M.nnt]; s.ett = a[M.ett]; s.ntt = a[M.ntt];
    s.ww = s.ss = s.bb = 0;
}
template <typename T, typename Real>
__device__ __forceinline__ void rnb3(S3T<Real> &s, const T *a, const Raw3 &R) {
    s.c = a[R.c]; s.e = a[R.e]; s.n = a[R.n]; s.t = a[R.t]; s.w = a[R.w]; s.s = a[R.s]; s.b = a[R.b];
    s.ee = a[R.ee]; s.nn = a[R.nn]; s.tt = a[R.tt];
    s.en = a[R.en]; s.et = a[R.et]; s.es = a[R.es]; s.eb = a[R.eb]; s.nt = a[R.nt]; s.wn = a[R.wn];
    s.nb = a[R.nb]; s.wt = a[R.wt]; s.st = a[R.st];
    s.eee = a[R.eee]; s.nnn = a[R.nnn]; s.ttt = a[R.ttt];
    s.een = a[R.een]; s.eet = a[R.eet]; s.enn = a[R.enn]; s.nnt = a[R.nnt]; s.ett = a[R.ett]; s.ntt = a[R.ntt];
    s.ww = s.ss = s.bb = 0;
}

// the 3D velocity masks of tilde.f:1072-1124 (bit 1 = b_e_ for u, 16 = b_n_
// for v, 4 = b_t_ for w); see ib_mask2
template <typename Real>
__device__ __forceinline__ void ib_mask3(const Prm &P, S3T<Real> &s, const Raw3 &R, int bit) {
    auto m = [&](int cell) { return Real(ib_open(P, cell, bit)); };
    s.c = s.c * m(R.c); s.e = s.e * m(R.e); s.w = s.w * m(R.w); s.n = s.n * m(R.n); s.s = s.s * m(R.s);
    s.t = s.t * m(R.t); s.b = s.b * m(R.b); s.ee = s.ee * m(R.ee); s.nn = s.nn * m(R.nn); s.tt = s.tt * m(R.tt);
    s.en = s.en * m(R.en); s.es = s.es * m(R.es); s.wn = s.wn * m(R.wn); s.et = s.et * m(R.et);
    s.wt = s.wt * m(R.wt); s.nt = s.nt * m(R.nt); s.st = s.st * m(R.st); s.eb = s.eb * m(R.eb);
    s.nb = s.nb * m(R.nb);
}
template <typename T, typename Real>
__device__ __forceinline__ void first_nb3(S3T<Real> &s, const T *a, const Raw3 &R, const Rem3 &M) {
    s.c = a[R.c]; s.e = a[M.e]; s.w = a[M.w]; s.n = a[M.n]; s.s = a[M.s]; s.t = a[M.t]; s.b = a[M.b];
}
template <typename T, typename Real>
__device__ __forceinline__ void third_nb3(S3T<Real> &s, const T *a, const Rem3 &M) {
    s.ee = a[M.ee]; s.ww = a[M.ww]; s.nn = a[M.nn]; s.ss = a[M.ss]; s.tt = a[M.tt]; s.bb = a[M.bb];
}

// interp.f (3D members)
template <typename Real>
__device__ __forceinline__ void interp_x3(const Prm &P, const S3T<Real> &f, int i, S3T<Real> &s) {
    const Real *dx = Met<Real>::dx(P);
    int ip2 = min(P.nx, i + 2), ip3 = min(P.nx, i + 3);
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i];
    Real indxpp = Met<Real>::hx(P)[i + 1], indxppp = Met<Real>::hx(P)[ip2];
    s.c = (dx[i + 1] * f.c + dx[i] * f.e) * indxp;
    s.e = (dx[ip2] * f.e + dx[i + 1] * f.ee) * indxpp;
    s.n = (dx[i + 1] * f.n + dx[i] * f.en) * indxp;
    s.t = (dx[i + 1] * f.t + dx[i] * f.et) * indxp;
    s.w = (dx[i] * f.w + dx[i - 1] * f.c) * indxm;
    s.s = (dx[i + 1] * f.s + dx[i] * f.es) * indxp;
    s.b = (dx[i + 1] * f.b + dx[i] * f.eb) * indxp;
    s.ee = (dx[ip2] * f.eee + dx[ip3] * f.ee) * indxppp;
    s.nn = (dx[i] * f.enn + dx[i + 1] * f.nn) * indxp;
    s.tt = (dx[i] * f.ett + dx[i + 1] * f.tt) * indxp;
}
template <typename Real>
__device__ __forceinline__ void interp_y3(const Prm &P, const S3T<Real> &f, int j, S3T<Real> &s) {
    const Real *dy = Met<Real>::dy(P);
    int jp2 = min(P.ny, j + 2), jp3 = min(P.ny, j + 3);
    Real indym = Met<Real>::hy(P)[j - 1], indyp = Met<Real>::hy(P)[j];
    Real indypp = Met<Real>::hy(P)[j + 1], indyppp = Met<Real>::hy(P)[jp2];
    s.c = (dy[j + 1] * f.c + dy[j] * f.n) * indyp;
    s.e = (dy[j + 1] * f.e + dy[j] * f.en) * indyp;
    s.n = (dy[jp2] * f.n + dy[j + 1] * f.nn) * indypp;
    s.t = (dy[j + 1] * f.t + dy[j] * f.nt) * indyp;
    s.w = (dy[j + 1] * f.w + dy[j] * f.wn) * indyp;
    s.s = (dy[j] * f.s + dy[j - 1] * f.c) * indym;
    s.b = (dy[j + 1] * f.b + dy[j] * f.nb) * indyp;
    s.ee = (dy[j] * f.een + dy[j + 1] * f.ee) * indyp;
    s.nn = (dy[jp2] * f.nnn + dy[jp3] * f.nn) * indyppp;
    s.tt = (dy[j] * f.ntt + dy[j + 1] * f.tt) * indyp;
}
template <typename Real>
__device__ __forceinline__ void interp_z3(const Prm &P, const S3T<Real> &f, int k, S3T<Real> &s) {
    const Real *dz = Met<Real>::dz(P);
    int kp2 = min(P.nz, k + 2), kp3 = min(P.nz, k + 3);
    Real indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k];
    Real indzpp = Met<Real>::hz(P)[k + 1], indzppp = Met<Real>::hz(P)[kp2];
    s.c = (dz[k + 1] * f.c + dz[k] * f.t) * indzp;
    s.e = (dz[k + 1] * f.e + dz[k] * f.et) * indzp;
    s.n = (dz[k + 1] * f.n + dz[k] * f.nt) * indzp;
    s.t = (dz[kp2] * f.t + dz[k + 1] * f.tt) * indzpp;
    s.w = (dz[k + 1] * f.w + dz[k] * f.wt) * indzp;
    s.s = (dz[k + 1] * f.s + dz[k] * f.st) * indzp;
    s.b = (dz[k] * f.b + dz[k - 1] * f.c) * indzm;
    s.ee = (dz[k] * f.eet + dz[k + 1] * f.ee) * indzp;
    s.nn = (dz[k] * f.nnt + dz[k + 1] * f.nn) * indzp;
    s.tt = (dz[kp2] * f.ttt + dz[kp3] * f.tt) * indzppp;
}

template <typename Real>
struct F6T { Real e, n, t, w, s, b; };
using F6d = F6T<double>;

// one limited face correction: shared by the momentum, mass and scalar MUSCL
// routines, which differ only in the gradients and increments they pass
template <typename Real>
__device__ __forceinline__ void muscl_face(int lt, double beta, Real &fx, Real cs, Real gradc, Real gradm,
                                           Real gradp, Real incr_p, Real incr_m, bool lim_on) {
    Real erre = 0, incr = 0, lim = 0;
    if (cs >= 0) { if (gradc != 0) erre = gradm / gradc; incr = incr_p; }
    else if (cs < 0) { if (gradc != 0) erre = gradp / gradc; incr = incr_m; }
    if (lim_on) lim = limiter(lt, erre, beta);
    Real upwnd = lim * gradc * incr;
    fx = fx + upwnd * cs;
}

template <typename Real>
__device__ __forceinline__ void flu_3d(const Prm &P, F6T<Real> &f, bool dw, bool ds, bool db, const S3T<Real> &d, const S3T<Real> &u,
                                       const S3T<Real> &v, const S3T<Real> &w, int i) {
    const Real *dx = Met<Real>::dx(P);
    Real indxp = Met<Real>::hx(P)[i], cs;
    if (dw) { cs = Real(0.5) * (u.c + u.w); f.w = Real(0.5) * (cs - fabs(cs)) * d.c * u.c + Real(0.5) * (cs + fabs(cs)) * d.w * u.w; }
    if (ds) { cs = (dx[i + 1] * v.s + dx[i] * v.es) * indxp; f.s = Real(0.5) * (cs - fabs(cs)) * d.c * u.c + Real(0.5) * (cs + fabs(cs)) * d.s * u.s; }
    if (db) { cs = (dx[i + 1] * w.b + dx[i] * w.eb) * indxp; f.b = Real(0.5) * (cs - fabs(cs)) * d.c * u.c + Real(0.5) * (cs + fabs(cs)) * d.b * u.b; }
    cs = Real(0.5) * (u.c + u.e);
    f.e = Real(0.5) * (cs - fabs(cs)) * d.e * u.e + Real(0.5) * (cs + fabs(cs)) * d.c * u.c;
    cs = (dx[i + 1] * v.c + dx[i] * v.e) * indxp;
    f.n = Real(0.5) * (cs - fabs(cs)) * d.n * u.n + Real(0.5) * (cs + fabs(cs)) * d.c * u.c;
    cs = (dx[i + 1] * w.c + dx[i] * w.e) * indxp;
    f.t = Real(0.5) * (cs - fabs(cs)) * d.t * u.t + Real(0.5) * (cs + fabs(cs)) * d.c * u.c;
}
template <typename Real>
__device__ __forceinline__ void muscl_flu_3d(const Prm &P, F6T<Real> &f, const S3T<Real> &d, const S3T<Real> &u, const S3T<Real> &v, const S3T<Real> &w,
                                             int i, int j, int k) {
    const Real *dx = Met<Real>::dx(P), *dy = Met<Real>::dy(P), *dz = Met<Real>::dz(P), *indx = Met<Real>::indx(P);
    int ip2 = min(P.nx, i + 2), jp2 = min(P.ny, j + 2), kp2 = min(P.nz, k + 2);
    Real indxp = Met<Real>::hx(P)[i];
    Real indym = Met<Real>::hy(P)[j - 1], indyp = Met<Real>::hy(P)[j], indypp = Met<Real>::hy(P)[j + 1];
    Real indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real gradw = indx[i] * (u.c * d.c - u.w * d.w);
    Real gradc = indx[i + 1] * (u.e * d.e - u.c * d.c);
    Real grade = indx[ip2] * (u.ee * d.ee - u.e * d.e);
    muscl_face(P.lv, P.beta, f.e, Real(0.5) * (u.c + u.e), gradc, gradw, grade, Real(0.5) * dx[i + 1], -Real(0.5) * dx[i + 1], true);
    Real grads = (u.c * d.c - u.s * d.s) * Real(2.0) * indym;
    gradc = (u.n * d.n - u.c * d.c) * Real(2.0) * indyp;
    Real gradn = (u.nn * d.nn - u.n * d.n) * Real(2.0) * indypp;
    muscl_face(P.lv, P.beta, f.n, (dx[i + 1] * v.c + dx[i] * v.e) * indxp, gradc, grads, gradn, Real(0.5) * dy[j], -Real(0.5) * dy[j + 1], true);
    Real gradb = (u.c * d.c - u.b * d.b) * Real(2.0) * indzm;
    gradc = (u.t * d.t - u.c * d.c) * Real(2.0) * indzp;
    Real gradt = (u.tt * d.tt - u.t * d.t) * Real(2.0) * indzpp;
    muscl_face(P.lv, P.beta, f.t, (dx[i + 1] * w.c + dx[i] * w.e) * indxp, gradc, gradb, gradt, Real(0.5) * dz[k], -Real(0.5) * dz[k + 1], true);
}
template <typename Real>
__device__ __forceinline__ void flv_3d(const Prm &P, F6T<Real> &f, bool dw, bool ds, bool db, const S3T<Real> &d, const S3T<Real> &u,
                                       const S3T<Real> &v, const S3T<Real> &w, int j) {
    const Real *dy = Met<Real>::dy(P);
    Real indyp = Met<Real>::hy(P)[j], cs;
    if (dw) { cs = (u.wn * dy[j] + u.w * dy[j + 1]) * indyp; f.w = Real(0.5) * (cs - fabs(cs)) * d.c * v.c + Real(0.5) * (cs + fabs(cs)) * d.w * v.w; }
    if (ds) { cs = Real(0.5) * (v.c + v.s); f.s = Real(0.5) * (cs - fabs(cs)) * d.c * v.c + Real(0.5) * (cs + fabs(cs)) * d.s * v.s; }
    if (db) { cs = (w.nb * dy[j] + w.b * dy[j + 1]) * indyp; f.b = Real(0.5) * (cs - fabs(cs)) * d.c * v.c + Real(0.5) * (cs + fabs(cs)) * d.b * v.b; }
    cs = indyp * (u.c * dy[j + 1] + u.n * dy[j]);
    f.e = Real(0.5) * (cs - fabs(cs)) * d.e * v.e + Real(0.5) * (cs + fabs(cs)) * d.c * v.c;
    cs = Real(0.5) * (v.n + v.c);
    f.n = Real(0.5) * (cs - fabs(cs)) * d.n * v.n + Real(0.5) * (cs + fabs(cs)) * d.c * v.c;
    cs = indyp * (w.c * dy[j + 1] + w.n * dy[j]);
    f.t = Real(0.5) * (cs - fabs(cs)) * d.t * v.t + Real(0.5) * (cs + fabs(cs)) * d.c * v.c;
}
template <typename Real>
__device__ __forceinline__ void muscl_flv_3d(const Prm &P, F6T<Real> &f, const S3T<Real> &d, const S3T<Real> &u, const S3T<Real> &v, const S3T<Real> &w,
                                             int i, int j, int k) {
    const Real *dx = Met<Real>::dx(P), *dy = Met<Real>::dy(P), *dz = Met<Real>::dz(P), *indy = Met<Real>::indy(P);
    int ip2 = min(P.nx, i + 2), jp2 = min(P.ny, j + 2), kp2 = min(P.nz, k + 2);
    Real indyp = Met<Real>::hy(P)[j];
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i], indxpp = Met<Real>::hx(P)[i + 1];
    Real indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real gradw = Real(2.0) * indxm * (v.c * d.c - v.w * d.w);
    Real gradc = Real(2.0) * indxp * (v.e * d.e - v.c * d.c);
    Real grade = Real(2.0) * indxpp * (v.ee * d.ee - v.e * d.e);
    muscl_face(P.lv, P.beta, f.e, indyp * (u.c * dy[j + 1] + u.n * dy[j]), gradc, gradw, grade, Real(0.5) * dx[i], -Real(0.5) * dx[i + 1], true);
    Real grads = (v.c * d.c - v.s * d.s) * indy[j];
    gradc = (v.n * d.n - v.c * d.c) * indy[j + 1];
    Real gradn = (v.nn * d.nn - v.n * d.n) * indy[jp2];
    muscl_face(P.lv, P.beta, f.n, Real(0.5) * (v.n + v.c), gradc, grads, gradn, Real(0.5) * dy[j + 1], -Real(0.5) * dy[j + 1], true);
    Real gradb = (v.c * d.c - v.b * d.b) * Real(2.0) * indzm;
    gradc = (v.t * d.t - v.c * d.c) * Real(2.0) * indzp;
    Real gradt = (v.tt * d.tt - v.t * d.t) * Real(2.0) * indzpp;
    muscl_face(P.lv, P.beta, f.t, (dy[j + 1] * w.c + dy[j] * w.n) * indyp, gradc, gradb, gradt, Real(0.5) * dz[k], -Real(0.5) * dz[k + 1], true);
}
template <typename Real>
__device__ __forceinline__ void flw_3d(const Prm &P, F6T<Real> &f, bool dw, bool ds, bool db, const S3T<Real> &d, const S3T<Real> &u,
                                       const S3T<Real> &v, const S3T<Real> &w, int k) {
    const Real *dz = Met<Real>::dz(P);
    Real indzp = Met<Real>::hz(P)[k], cs;
    if (dw) { cs = (dz[k + 1] * u.w + dz[k] * u.wt) * indzp; f.w = Real(0.5) * d.w * w.w * (cs + fabs(cs)) + Real(0.5) * d.c * w.c * (cs - fabs(cs)); }
    if (ds) { cs = (dz[k + 1] * v.s + dz[k] * v.st) * indzp; f.s = Real(0.5) * d.s * w.s * (cs + fabs(cs)) + Real(0.5) * d.c * w.c * (cs - fabs(cs)); }
    if (db) { cs = Real(0.5) * (w.b + w.c); f.b = Real(0.5) * d.b * w.b * (cs + fabs(cs)) + Real(0.5) * d.c * w.c * (cs - fabs(cs)); }
    cs = (dz[k + 1] * u.c + dz[k] * u.t) * indzp;
    f.e = Real(0.5) * d.c * w.c * (cs + fabs(cs)) + Real(0.5) * d.e * w.e * (cs - fabs(cs));
    cs = (dz[k + 1] * v.c + dz[k] * v.t) * indzp;
    f.n = Real(0.5) * d.c * w.c * (cs + fabs(cs)) + Real(0.5) * d.n * w.n * (cs - fabs(cs));
    cs = Real(0.5) * (w.c + w.t);
    f.t = Real(0.5) * d.c * w.c * (cs + fabs(cs)) + Real(0.5) * d.t * w.t * (cs - fabs(cs));
}
template <typename Real>
__device__ __forceinline__ void muscl_flw_3d(const Prm &P, F6T<Real> &f, const S3T<Real> &d, const S3T<Real> &u, const S3T<Real> &v, const S3T<Real> &w,
                                             int i, int j, int k) {
    const Real *dx = Met<Real>::dx(P), *dy = Met<Real>::dy(P), *dz = Met<Real>::dz(P), *indz = Met<Real>::indz(P);
    int ip2 = min(P.nx, i + 2), jp2 = min(P.ny, j + 2), kp2 = min(P.nz, k + 2);
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i], indxpp = Met<Real>::hx(P)[i + 1];
    Real indym = Met<Real>::hy(P)[j - 1], indyp = Met<Real>::hy(P)[j], indypp = Met<Real>::hy(P)[j + 1];
    Real indzp = Met<Real>::hz(P)[k];
    Real gradw = Real(2.0) * indxm * (w.c * d.c - w.w * d.w);
    Real gradc = Real(2.0) * indxp * (w.e * d.e - w.c * d.c);
    Real grade = Real(2.0) * indxpp * (w.ee * d.ee - w.e * d.e);
    muscl_face(P.lv, P.beta, f.e, (dz[k + 1] * u.c + dz[k] * u.t) * indzp, gradc, gradw, grade, Real(0.5) * dx[i], -Real(0.5) * dx[i + 1], true);
    Real grads = Real(2.0) * indym * (w.c * d.c - w.s * d.s);
    gradc = Real(2.0) * indyp * (w.n * d.n - w.c * d.c);
    Real gradn = Real(2.0) * indypp * (w.nn * d.nn - w.n * d.n);
    muscl_face(P.lv, P.beta, f.n, (dz[k + 1] * v.c + dz[k] * v.t) * indzp, gradc, grads, gradn, Real(0.5) * dy[j], -Real(0.5) * dy[j + 1], true);
    Real gradb = indz[k] * (w.c * d.c - w.b * d.b);
    gradc = indz[k + 1] * (w.t * d.t - w.c * d.c);
    Real gradt = indz[kp2] * (w.tt * d.tt - w.t * d.t);
    muscl_face(P.lv, P.beta, f.t, Real(0.5) * (w.c + w.t), gradc, gradb, gradt, Real(0.5) * dz[k + 1], -Real(0.5) * dz[k + 1], true);
}

// masf_3d + fmas_3d for one cell; face velocities given directly
template <typename Real>
__device__ __forceinline__ void massflux_3d(const Prm &P, const S3T<Real> &d, Real uw, Real uc, Real vs, Real vc,
                                            Real wb, Real wc, int i, int j, int k, bool muscl_on, int flw, int fle,
                                            int fls, int fln, int flb, int flt, F6T<Real> &f) {
    Real cs;
    cs = uw; f.w = Real(0.5) * (cs - fabs(cs)) * d.c + Real(0.5) * (cs + fabs(cs)) * d.w;
    cs = vs; f.s = Real(0.5) * (cs - fabs(cs)) * d.c + Real(0.5) * (cs + fabs(cs)) * d.s;
    cs = wb; f.b = Real(0.5) * (cs - fabs(cs)) * d.c + Real(0.5) * (cs + fabs(cs)) * d.b;
    cs = uc; f.e = Real(0.5) * (cs - fabs(cs)) * d.e + Real(0.5) * (cs + fabs(cs)) * d.c;
    cs = vc; f.n = Real(0.5) * (cs - fabs(cs)) * d.n + Real(0.5) * (cs + fabs(cs)) * d.c;
    cs = wc; f.t = Real(0.5) * (cs - fabs(cs)) * d.t + Real(0.5) * (cs + fabs(cs)) * d.c;
    if (!muscl_on) return;
    const Real *dx = Met<Real>::dx(P), *dy = Met<Real>::dy(P), *dz = Met<Real>::dz(P);
    int im2 = max(1, i - 2), ip2 = min(P.nx, i + 2), jm2 = max(1, j - 2), jp2 = min(P.ny, j + 2);
    int km2 = max(1, k - 2), kp2 = min(P.nz, k + 2);
    Real indxmm = Met<Real>::hx(P)[max(i - 2, 0)], indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i], indxpp = Met<Real>::hx(P)[i + 1];
    Real indymm = Met<Real>::hy(P)[max(j - 2, 0)], indym = Met<Real>::hy(P)[j - 1], indyp = Met<Real>::hy(P)[j], indypp = Met<Real>::hy(P)[j + 1];
    Real indzmm = Met<Real>::hz(P)[max(k - 2, 0)], indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real gradc, gradw, grade, grads, gradn, gradb, gradt;
    gradc = Real(2.0) * indxm * (d.c - d.w); gradw = Real(2.0) * indxmm * (d.w - d.ww); grade = Real(2.0) * indxp * (d.e - d.c);
    muscl_face(P.lm, P.beta, f.w, uw, gradc, gradw, grade, Real(0.5) * dx[i - 1], -Real(0.5) * dx[i], i != 2 && flw == FLUID);
    gradw = gradc; gradc = grade; grade = Real(2.0) * indxpp * (d.ee - d.e);
    muscl_face(P.lm, P.beta, f.e, uc, gradc, gradw, grade, Real(0.5) * dx[i], -Real(0.5) * dx[i + 1], i != P.nx - 1 && fle == FLUID);
    gradc = Real(2.0) * indym * (d.c - d.s); grads = Real(2.0) * indymm * (d.s - d.ss); gradn = Real(2.0) * indyp * (d.n - d.c);
    muscl_face(P.lm, P.beta, f.s, vs, gradc, grads, gradn, Real(0.5) * dy[j - 1], -Real(0.5) * dy[j], j != 2 && fls == FLUID);
    grads = gradc; gradc = gradn; gradn = Real(2.0) * indypp * (d.nn - d.n);
    muscl_face(P.lm, P.beta, f.n, vc, gradc, grads, gradn, Real(0.5) * dy[j], -Real(0.5) * dy[j + 1], j != P.ny - 1 && fln == FLUID);
    gradc = Real(2.0) * indzm * (d.c - d.b); gradb = Real(2.0) * indzmm * (d.b - d.bb); gradt = Real(2.0) * indzp * (d.t - d.c);
    muscl_face(P.lm, P.beta, f.b, wb, gradc, gradb, gradt, Real(0.5) * dz[k - 1], -Real(0.5) * dz[k], k != 2 && flb == FLUID);
    gradb = gradc; gradc = gradt; gradt = Real(2.0) * indzpp * (d.tt - d.t);
    muscl_face(P.lm, P.beta, f.t, wc, gradc, gradb, gradt, Real(0.5) * dz[k], -Real(0.5) * dz[k + 1], k != P.nz - 1 && flt == FLUID);
}

// fsc_3d + muscl_fsc_3d; W/S/B only where that neighbour is not fluid
template <typename Real>
__device__ __forceinline__ void fsc_3d(const Prm &P, F6T<Real> &f, bool dw, bool ds, bool db, const S3T<Real> &d, const S3T<Real> &fl,
                                       Real uw, Real uc, Real vs, Real vc, Real wb, Real wc) {
    Real cs;
    if (dw) { cs = uw; f.w = Real(0.5) * (cs - fabs(cs)) * d.c * fl.c + Real(0.5) * (cs + fabs(cs)) * d.w * fl.w; }
    if (ds) { cs = vs; f.s = Real(0.5) * (cs - fabs(cs)) * d.c * fl.c + Real(0.5) * (cs + fabs(cs)) * d.s * fl.s; }
    if (db) { cs = wb; f.b = Real(0.5) * (cs - fabs(cs)) * d.c * fl.c + Real(0.5) * (cs + fabs(cs)) * d.b * fl.b; }
    cs = uc; f.e = Real(0.5) * (cs - fabs(cs)) * d.e * fl.e + Real(0.5) * (cs + fabs(cs)) * d.c * fl.c;
    cs = vc; f.n = Real(0.5) * (cs - fabs(cs)) * d.n * fl.n + Real(0.5) * (cs + fabs(cs)) * d.c * fl.c;
    cs = wc; f.t = Real(0.5) * (cs - fabs(cs)) * d.t * fl.t + Real(0.5) * (cs + fabs(cs)) * d.c * fl.c;
}
template <typename Real>
__device__ __forceinline__ void muscl_fsc_3d(const Prm &P, F6T<Real> &f, const S3T<Real> &d, const S3T<Real> &fl, Real uc, Real vc,
                                             Real wc, int i, int j, int k) {
    const Real *dx = Met<Real>::dx(P), *dy = Met<Real>::dy(P), *dz = Met<Real>::dz(P);
    int ip2 = min(P.nx, i + 2), jp2 = min(P.ny, j + 2), kp2 = min(P.nz, k + 2);
    Real indxm = Met<Real>::hx(P)[i - 1], indxp = Met<Real>::hx(P)[i], indxpp = Met<Real>::hx(P)[i + 1];
    Real indym = Met<Real>::hy(P)[j - 1], indyp = Met<Real>::hy(P)[j], indypp = Met<Real>::hy(P)[j + 1];
    Real indzm = Met<Real>::hz(P)[k - 1], indzp = Met<Real>::hz(P)[k], indzpp = Met<Real>::hz(P)[k + 1];
    Real gradc = Real(2.0) * indxp * (d.e * fl.e - d.c * fl.c);
    Real gradw = Real(2.0) * indxm * (d.c * fl.c - d.w * fl.w);
    Real grade = Real(2.0) * indxpp * (d.ee * fl.ee - d.e * fl.e);
    muscl_face(P.lm, P.beta, f.e, uc, gradc, gradw, grade, Real(0.5) * dx[i], -Real(0.5) * dx[i + 1], i != P.nx - 1);
    gradc = Real(2.0) * indyp * (d.n * fl.n - d.c * fl.c);
    Real grads = Real(2.0) * indym * (d.c * fl.c - d.s * fl.s);
    Real gradn = Real(2.0) * indypp * (d.nn * fl.nn - d.n * fl.n);
    muscl_face(P.lm, P.beta, f.n, vc, gradc, grads, gradn, Real(0.5) * dy[j], -Real(0.5) * dy[j + 1], j != P.ny - 1);
    gradc = Real(2.0) * indzp * (d.t * fl.t - d.c * fl.c);
    Real gradb = Real(2.0) * indzm * (d.c * fl.c - d.b * fl.b);
    Real gradt = Real(2.0) * indzpp * (d.tt * fl.tt - d.t * fl.t);
    muscl_face(P.lm, P.beta, f.t, wc, gradc, gradb, gradt, Real(0.5) * dz[k], -Real(0.5) * dz[k + 1], k != P.nz - 1);
}

// hotc.f:12-82 (3D)
template <typename Real>
__device__ __forceinline__ void hotc_3d(const Prm &P, F6T<Real> &h, bool hw, bool hs, bool hb, const S3T<Real> &ep, const S3T<Real> &tg,
                                        const S3T<Real> &ka, int i, int j, int k) {
    const Real *dx = Met<Real>::dx(P), *dy = Met<Real>::dy(P), *dz = Met<Real>::dz(P);
    if (hw) {
        Real indxm = Met<Real>::hx(P)[i - 1];
        Real km = (dx[i - 1] * ka.c + dx[i] * ka.w) * indxm, em = (dx[i - 1] * ep.c + dx[i] * ep.w) * indxm;
        h.w = km * em * (tg.c - tg.w) * indxm * Real(2.0);
    }
    if (hs) {
        Real indym = Met<Real>::hy(P)[j - 1];
        Real km = (dy[j - 1] * ka.c + dy[j] * ka.s) * indym, em = (dy[j - 1] * ep.c + dy[j] * ep.s) * indym;
        h.s = km * em * (tg.c - tg.s) * indym * Real(2.0);
    }
    if (hb) {
        Real indzm = Met<Real>::hz(P)[k - 1];
        Real km = (dz[k - 1] * ka.c + dz[k] * ka.b) * indzm, em = (dz[k - 1] * ep.c + dz[k] * ep.b) * indzm;
        h.b = km * em * (tg.c - tg.b) * indzm * Real(2.0);
    }
    Real indxp = Met<Real>::hx(P)[i];
    Real kme = (dx[i + 1] * ka.c + dx[i] * ka.e) * indxp, epme = (dx[i + 1] * ep.c + dx[i] * ep.e) * indxp;
    h.e = kme * epme * (tg.e - tg.c) * indxp * Real(2.0);
    Real indyp = Met<Real>::hy(P)[j];
    Real kmn = (dy[j + 1] * ka.c + dy[j] * ka.n) * indyp, epmn = (dy[j + 1] * ep.c + dy[j] * ep.n) * indyp;
    h.n = kmn * epmn * (tg.n - tg.c) * indyp * Real(2.0);
    Real indzp = Met<Real>::hz(P)[k];
    Real kmt = (dz[k + 1] * ka.c + dz[k] * ka.t) * indzp, epmt = (dz[k + 1] * ep.c + dz[k] * ep.t) * indzp;
    h.t = kmt * epmt * (tg.t - tg.c) * indzp * Real(2.0);
}

// stress3D (visc.f:293-559) for one cell; mu == lambda on this path
template <typename MU, typename LAM, typename EPS>
__device__ __forceinline__ void stress3d_cell(const Prm &P, const Raw3 &R, const Rem3 &M, int i, int j, int k, MU mu, LAM lam,
                                              EPS eps, const double *u, const double *v, const double *w,
                                              double &visx, double &visy, double &visz) {
    const double *dx = P.dx, *dy = P.dy, *dz = P.dz, *indx = P.indx, *indy = P.indy, *indz = P.indz;
    const double cm = 2.0 / 3.0;
    int c = R.c;
    double indxp = P.hx[i], indxm = P.hx[i - 1];
    double indyp = P.hy[j], indym = P.hy[j - 1];
    double indzp = P.hz[k], indzm = P.hz[k - 1];
    double indxp2 = indxp * 2.0, indxm2 = indxm * 2.0, indyp2 = indyp * 2.0, indym2 = indym * 2.0;
    double indzp2 = indzp * 2.0, indzm2 = indzm * 2.0;
    double dum = u[c] - u[R.w], dup = u[R.e] - u[c], dvm = v[c] - v[R.s], dvp = v[R.n] - v[c];
    double dwm = w[c] - w[R.b], dwp = w[R.t] - w[c];
    double dupm1 = u[R.n] - u[R.wn], dupm2 = u[R.t] - u[R.wt], dvpm1 = v[R.e] - v[R.es];
    double dvpm2 = v[R.t] - v[R.st], dwpm1 = w[R.e] - w[R.eb], dwpm2 = w[R.n] - w[R.nb];
    double divc = dum * indx[i] + dvm * indy[j] + dwm * indz[k];
    double dive = dup * indx[i + 1] + dvpm1 * indy[j] + dwpm1 * indz[k];
    double divn = dupm1 * indx[i] + dvp * indy[j + 1] + dwpm2 * indz[k];
    double divt = dupm2 * indx[i] + dvpm2 * indy[j] + dwp * indz[k + 1];
    double txx2 = 2.0 * dup * indx[i + 1], txx1 = 2.0 * dum * indx[i];
    double tyy2 = 2.0 * dvp * indy[j + 1], tyy1 = 2.0 * dvm * indy[j];
    double tzz2 = 2.0 * dwp * indz[k + 1], tzz1 = 2.0 * dwm * indz[k];
    txx2 = mu(M.e) * txx2 - cm * lam(M.e) * dive;
    txx1 = mu(c) * txx1 - cm * lam(c) * divc;
    tyy2 = mu(M.n) * tyy2 - cm * lam(M.n) * divn;
    tyy1 = mu(c) * tyy1 - cm * lam(c) * divc;
    tzz2 = mu(M.t) * tzz2 - cm * lam(M.t) * divt;
    tzz1 = mu(c) * tzz1 - cm * lam(c) * divc;
    dum = u[c] - u[R.s]; dup = u[R.n] - u[c]; dvm = v[c] - v[R.w]; dvp = v[R.e] - v[c];
    dwm = w[c] - w[R.s]; dwp = w[R.n] - w[c];
    dupm1 = u[R.wn] - u[R.w]; dupm2 = u[R.wt] - u[R.w]; dvpm1 = v[R.es] - v[R.s];
    dvpm2 = v[R.st] - v[R.s]; dwpm1 = w[R.nb] - w[R.b]; dwpm2 = w[R.eb] - w[R.b];
    double tyx2 = dup * indyp2 + dvp * indxp2, tyx1 = dum * indym2 + dvpm1 * indxp2;
    double txy2 = tyx2, txy1 = dupm1 * indyp2 + dvm * indxm2;
    dvp = v[R.t] - v[c]; dvm = v[c] - v[R.b];
    double tzy2 = dvp * indzp2 + dwp * indyp2, tzy1 = dvm * indzm2 + dwpm1 * indyp2;
    double tyz2 = tzy2, tyz1 = dvpm2 * indzp2 + dwm * indym2;
    dwp = w[R.e] - w[c]; dwm = w[c] - w[R.w]; dup = u[R.t] - u[c]; dum = u[c] - u[R.b];
    double txz2 = dwp * indxp2 + dup * indzp2, txz1 = dwm * indxm2 + dupm2 * indzp2;
    double tzx2 = txz2, tzx1 = dwpm2 * indxp2 + dum * indzm2;
    double epsc = eps(c), epse = eps(M.e), epsw = eps(M.w), epsn = eps(M.n), epss = eps(M.s), epst = eps(M.t), epsb = eps(M.b);
    double epsen = eps(R.en), epset = eps(R.et), epses = eps(R.es), epseb = eps(M.eb), epswn = eps(R.wn);
    double epswt = eps(R.wt), epsnt = eps(R.nt), epsnb = eps(M.nb), epsst = eps(R.st);
    double muc = mu(c), mue = mu(M.e), muw = mu(M.w), mun = mu(M.n), mus = mu(M.s), mut = mu(M.t), mub = mu(M.b);
    double muen = mu(R.en), muet = mu(R.et), mues = mu(R.es), mueb = mu(M.eb), muwn = mu(R.wn);
    double muwt = mu(R.wt), munt = mu(R.nt), munb = mu(M.nb), must = mu(R.st);
    double epm1 = (dy[j] * epsn * mun + dy[j + 1] * epsc * muc) * indyp;
    double epm2 = (dy[j] * epsen * muen + dy[j + 1] * epse * mue) * indyp;
    double epmyx2 = (dx[i + 1] * epm1 + dx[i] * epm2) * indxp;
    epm1 = (dy[j - 1] * epsc * muc + dy[j] * epss * mus) * indym;
    epm2 = (dy[j - 1] * epse * mue + dy[j] * epses * mues) * indym;
    double epmyx1 = (dx[i + 1] * epm1 + dx[i] * epm2) * indxp;
    epm1 = (dz[k] * epst * mut + dz[k + 1] * epsc * muc) * indzp;
    epm2 = (dz[k] * epset * muet + dz[k + 1] * epse * mue) * indzp;
    double epmzx2 = (dx[i + 1] * epm1 + dx[i] * epm2) * indxp;
    epm1 = (dz[k - 1] * epsc * muc + dz[k] * epsb * mub) * indzm;
    epm2 = (dz[k - 1] * epse * mue + dz[k] * epseb * mueb) * indzm;
    double epmzx1 = (dx[i + 1] * epm1 + dx[i] * epm2) * indxp;
    visx = (epse * txx2 - epsc * txx1) * indxp2;
    visx = visx + (epmyx2 * tyx2 - epmyx1 * tyx1) * indy[j];
    visx = visx + (epmzx2 * tzx2 - epmzx1 * tzx1) * indz[k];
    epm1 = (dy[j] * epswn * muwn + dy[j + 1] * epsw * muw) * indyp;
    epm2 = (dy[j] * epsn * mun + dy[j + 1] * epsc * muc) * indyp;
    double epmxy1 = (dx[i] * epm1 + dx[i - 1] * epm2) * indxm;
    double epmxy2 = epmyx2;
    epm1 = (dz[k] * epst * mut + dz[k + 1] * epsc * muc) * indzp;
    epm2 = (dz[k] * epsnt * munt + dz[k + 1] * epsn * mun) * indzp;
    double epmzy2 = (dy[j + 1] * epm1 + dy[j] * epm2) * indyp;
    epm1 = (dz[k - 1] * epsc * muc + dz[k] * epsb * mub) * indzm;
    epm2 = (dz[k - 1] * epsn * mun + dz[k] * epsnb * munb) * indzm;
    double epmzy1 = (dy[j + 1] * epm1 + dy[j] * epm2) * indyp;
    visy = (epsn * tyy2 - epsc * tyy1) * indyp2;
    visy = visy + (epmxy2 * txy2 - epmxy1 * txy1) * indx[i];
    visy = visy + (epmzy2 * tzy2 - epmzy1 * tzy1) * indz[k];
    double epmxz2 = epmzx2;
    epm1 = (dz[k] * epswt * muwt + dz[k + 1] * epsw * muw) * indzp;
    epm2 = (dz[k] * epst * mut + dz[k + 1] * epsc * muc) * indzp;
    double epmxz1 = (dx[i] * epm1 + dx[i - 1] * epm2) * indxm;
    double epmyz2 = epmzy2;
    epm1 = (dz[k] * epsst * must + dz[k + 1] * epss * mus) * indzp;
    epm2 = (dz[k] * epst * mut + dz[k + 1] * epsc * muc) * indzp;
    double epmyz1 = (dy[j] * epm1 + dy[j - 1] * epm2) * indym;
    visz = (epst * tzz2 - epsc * tzz1) * indzp2;
    visz = visz + (epmxz2 * txz2 - epmxz1 * txz1) * indx[i];
    visz = visz + (epmyz2 * tyz2 - epmyz1 * tyz1) * indy[j];
}

}  // namespace pdac

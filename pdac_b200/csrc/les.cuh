// les.cuh -- the sub-grid turbulence model of turbo.f on the device
// (iturb = 1: static Smagorinsky, modturbo = 1, or the dynamic model in 3D,
// modturbo = 2; iturb = 2 the same with the ground-roughness mixing length;
// iss = 1 particle sub-grid stress).
//
// smag = lm^2 (x anis in 3D), lm = cmut delta or, with iturb = 2, matched
// with the roughness length, is fixed per cell at set-up on the host
// (turbulence_setup, turbo.f:42-108).  Each step k_sgsg sets the
// turbulent viscosity and conductivity of the fluid cells from the strain
// rate (sgsg, turbo.f:145-349) and k_sgss the particle sub-grid viscosity
// (sgss, turbo.f:437-475).  The consumers add the molecular values in place
// before they read them, as the reference's module arrays do (k_accum):
// mugt = mug + mugt before each gas stress (viscg, visc.f:150-180), must =
// must + mus before each particle stress (viscs, visc.f:193-205), kapgt =
// kapgt + kapg before each enthalpy flux pass (htilde.f:218-224,
// explicit_solver.f:1285-1290).
#pragma once
#include "kernels3d.cuh"

namespace pdac {

// strain2d, turbo.f:623-668: modulus of the strain rate of (u, w) at (i, k)
__device__ __forceinline__ double strain2d(const Prm &P, const double *u, const double *w, int c, int i, int k) {
    const double *dx = P.dx, *dz = P.dz;
    const int nx = P.nx;
    int imjk = i > 1 ? c - 1 : c, ipjk = i < nx ? c + 1 : c;
    int ijkm = k > 1 ? c - nx : c, ijkp = k < P.nz ? c + nx : c;
    int imjkp = at2(P, max(i - 1, 1), min(k + 1, P.nz)), imjkm = at2(P, max(i - 1, 1), max(k - 1, 1));
    int ipjkm = at2(P, min(i + 1, nx), max(k - 1, 1));
    double dxp = dx[i] + dx[i + 1], dxm = dx[i] + dx[i - 1], dzp = dz[k] + dz[k + 1], dzm = dz[k] + dz[k - 1];
    double indxp = 1.0 / dxp, indxm = 1.0 / dxm, indzp = 1.0 / dzp, indzm = 1.0 / dzm;
    double sr1 = (u[c] - u[imjk]) * P.indx[i];
    double sr2 = (w[c] - w[ijkm]) * P.indz[k];
    double d33 = P.itc == 1 ? 0.5 * (u[c] + u[imjk]) * P.inr[i] : 0.0;
    double u3 = 0.5 * (u[ijkp] + u[imjkp]), u2 = 0.5 * (u[c] + u[imjk]), u1 = 0.5 * (u[ijkm] + u[imjkm]);
    double w3 = 0.5 * (w[ipjk] + w[ipjkm]), w2 = 0.5 * (w[c] + w[ijkm]), w1 = 0.5 * (w[imjk] + w[imjkm]);
    double um2 = u2 + (u3 - u2) * dz[k] * indzp;
    double um1 = u1 + (u2 - u1) * dz[k - 1] * indzm;
    double wm2 = w2 + (w3 - w2) * dx[i] * indxp;
    double wm1 = w1 + (w2 - w1) * dx[i - 1] * indxm;
    double sr12 = ((um2 - um1) * P.indz[k] + (wm2 - wm1) * P.indx[i]) * 0.5;
    return sqrt(2.0 * (sr1 * sr1 + sr2 * sr2 + 2.0 * (sr12 * sr12) + d33 * d33));
}

// strain3d, turbo.f:519-621: the modulus and the six components
struct Strain {
    double mod, s11, s12, s22, s13, s23, s33;
};
__device__ __forceinline__ Strain strain3d_c(const Prm &P, const double *u, const double *v, const double *w,
                                             const Raw3 &R, int i, int j, int k) {
    const double *dx = P.dx, *dy = P.dy, *dz = P.dz;
    const int c = R.c;
    double dxp = dx[i] + dx[i + 1], dxm = dx[i] + dx[i - 1];
    double dyp = dy[j] + dy[j + 1], dym = dy[j] + dy[j - 1];
    double dzp = dz[k] + dz[k + 1], dzm = dz[k] + dz[k - 1];
    double sr11 = (u[c] - u[R.w]) * P.indx[i];
    double sr22 = (v[c] - v[R.s]) * P.indy[j];
    double sr33 = (w[c] - w[R.b]) * P.indz[k];
    double uzp = 0.5 * (u[R.t] + u[R.wt]), uzm = 0.5 * (u[R.b] + u[R.wb]);
    double uyp = 0.5 * (u[R.n] + u[R.wn]), uym = 0.5 * (u[R.s] + u[R.ws]);
    double vxp = 0.5 * (v[R.e] + v[R.es]), vxm = 0.5 * (v[R.w] + v[R.ws]);
    double vzp = 0.5 * (v[R.t] + v[R.st]), vzm = 0.5 * (v[R.b] + v[R.sb]);
    double wxp = 0.5 * (w[R.e] + w[R.eb]), wxm = 0.5 * (w[R.w] + w[R.wb]);
    double wyp = 0.5 * (w[R.n] + w[R.nb]), wym = 0.5 * (w[R.s] + w[R.sb]);
    double sr12 = (uyp - uym) / (dyp + dym) + (vxp - vxm) / (dxp + dxm);
    double sr13 = (uzp - uzm) / (dzp + dzm) + (wxp - wxm) / (dxp + dxm);
    double sr23 = (vzp - vzm) / (dzp + dzm) + (wyp - wym) / (dyp + dym);
    double mod = sqrt(2.0 * (sr11 * sr11 + sr22 * sr22 + sr33 * sr33 + 2.0 * (sr12 * sr12) + 2.0 * (sr13 * sr13) +
                             2.0 * (sr23 * sr23)));
    return {mod, sr11, sr12, sr22, sr13, sr23, sr33};
}
__device__ __forceinline__ double strain3d(const Prm &P, const double *u, const double *v, const double *w,
                                           const Raw3 &R, int i, int j, int k) {
    return strain3d_c(P, u, v, w, R, i, j, k).mod;
}

// ---- dynamic model (modturbo = 2, 3D), turbo.f:180-349 ---------------------
// Seven-point values of first_rnb (subscr.f:2259-2289): the centre from the
// index given, the six neighbours from the current cell's raw indices.
struct St7 {
    double c, e, w, n, s, t, b;
};
__device__ __forceinline__ St7 first_rnb7(const double *a, int c0, const Raw3 &R) {
    return {a[c0], a[R.e], a[R.w], a[R.n], a[R.s], a[R.t], a[R.b]};
}
__device__ __forceinline__ St7 st_half_sum(const St7 &p, const St7 &q) {
    return {0.5 * (p.c + q.c), 0.5 * (p.e + q.e), 0.5 * (p.w + q.w), 0.5 * (p.n + q.n), 0.5 * (p.s + q.s),
            0.5 * (p.t + q.t), 0.5 * (p.b + q.b)};
}
__device__ __forceinline__ St7 st_prod(const St7 &p, const St7 &q) {
    return {p.c * q.c, p.e * q.e, p.w * q.w, p.n * q.n, p.s * q.s, p.t * q.t, p.b * q.b};
}
// filter_3d (turbo.f:436-474): the mean of the 1-2-1 filters along x, y, z
__device__ __forceinline__ double filter_3d(const St7 &q) {
    double fx = 0.25 * (q.w + 2.0 * q.c + q.e);
    double fy = 0.25 * (q.s + 2.0 * q.c + q.n);
    double fz = 0.25 * (q.b + 2.0 * q.c + q.t);
    return 1.0 / 3.0 * (fx + fy + fz);
}
// the 16 per-cell blocks of F.dyn: |S|, |S| S_ij (6), the test-filtered
// velocities (3) and their filtered products (uu, vv, ww, uv, uw, vw)
enum { DY_MOD, DY_P11, DY_P12, DY_P22, DY_P13, DY_P23, DY_P33, DY_FU, DY_FV, DY_FW, DY_FUU, DY_FVV, DY_FWW,
       DY_FUV, DY_FUW, DY_FVW, DY_N };

// pass 1 (turbo.f:199-233, vel_hat turbo.f:385-433), every cell: fluid
// cells get their strain products and filtered velocities, others zeros
__global__ void k_sgsg_dyn1(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    const size_t n = P.ncell;
    double *d = F.dyn;
    if (!fluid(P, c)) {
        for (int q = 0; q < DY_N; ++q) d[q * n + c] = 0.0;
        return;
    }
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    raw3(P, i, j, k, R);
    Strain sr = strain3d_c(P, F.ug, F.vg, F.wg, R, i, j, k);
    d[DY_MOD * n + c] = sr.mod;
    d[DY_P11 * n + c] = sr.mod * sr.s11;
    d[DY_P12 * n + c] = sr.mod * sr.s12;
    d[DY_P22 * n + c] = sr.mod * sr.s22;
    d[DY_P13 * n + c] = sr.mod * sr.s13;
    d[DY_P23 * n + c] = sr.mod * sr.s23;
    d[DY_P33 * n + c] = sr.mod * sr.s33;
    const St7 u = st_half_sum(first_rnb7(F.ug, c, R), first_rnb7(F.ug, R.w, R));
    const St7 v = st_half_sum(first_rnb7(F.vg, c, R), first_rnb7(F.vg, R.s, R));
    const St7 w = st_half_sum(first_rnb7(F.wg, c, R), first_rnb7(F.wg, R.b, R));
    d[DY_FU * n + c] = filter_3d(u);
    d[DY_FV * n + c] = filter_3d(v);
    d[DY_FW * n + c] = filter_3d(w);
    d[DY_FUU * n + c] = filter_3d(st_prod(u, u));
    d[DY_FVV * n + c] = filter_3d(st_prod(v, v));
    d[DY_FWW * n + c] = filter_3d(st_prod(w, w));
    d[DY_FUV * n + c] = filter_3d(st_prod(u, v));
    d[DY_FUW * n + c] = filter_3d(st_prod(u, w));
    d[DY_FVW * n + c] = filter_3d(st_prod(v, w));
}

// pass 2 (turbo.f:255-349), every cell: the Germano coefficient cdyn from
// the Leonard stress L of the filtered velocities and M = 4 |S^| S^ - (|S| S)^,
// smag = cdyn delta^2, then the viscosity and conductivity as the static
// model; delta = (dx dy dz)^(1/3) per cell is set up on the host
__global__ void k_sgsg_dyn2(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    if (!fluid(P, c)) {
        F.mugt[c] = 0.0;
        F.kapgt[c] = 0.0;
        return;
    }
    const size_t n = P.ncell;
    const double *d = F.dyn;
    int i, j, k;
    ijk_of(P, c, i, j, k);
    Raw3 R;
    raw3(P, i, j, k, R);
    const double fu = d[DY_FU * n + c], fv = d[DY_FV * n + c], fw = d[DY_FW * n + c];
    Strain fs = strain3d_c(P, d + DY_FU * n, d + DY_FV * n, d + DY_FW * n, R, i, j, k);
    double fp11 = filter_3d(first_rnb7(d + DY_P11 * n, c, R));
    double fp12 = filter_3d(first_rnb7(d + DY_P12 * n, c, R));
    double fp22 = filter_3d(first_rnb7(d + DY_P22 * n, c, R));
    double fp13 = filter_3d(first_rnb7(d + DY_P13 * n, c, R));
    double fp23 = filter_3d(first_rnb7(d + DY_P23 * n, c, R));
    double fp33 = filter_3d(first_rnb7(d + DY_P33 * n, c, R));
    double l11 = fu * fu - d[DY_FUU * n + c];
    double l12 = fu * fv - d[DY_FUV * n + c];
    double l22 = fv * fv - d[DY_FVV * n + c];
    double l13 = fu * fw - d[DY_FUW * n + c];
    double l23 = fv * fw - d[DY_FVW * n + c];
    double l33 = fw * fw - d[DY_FWW * n + c];
    double m11 = (4.0 * fs.mod * fs.s11 - fp11);
    double m12 = (4.0 * fs.mod * fs.s12 - fp12);
    double m22 = (4.0 * fs.mod * fs.s22 - fp22);
    double m13 = (4.0 * fs.mod * fs.s13 - fp13);
    double m23 = (4.0 * fs.mod * fs.s23 - fp23);
    double m33 = (4.0 * fs.mod * fs.s33 - fp33);
    const double delt = F.delt[c];
    double num = l11 * m11 + l22 * m22 + l33 * m33 + 2.0 * l12 * m12 + 2.0 * l13 * m13 + 2.0 * l23 * m23;
    double den = (delt * delt) * (m11 * m11 + m22 * m22 + m33 * m33 + 2.0 * (m12 * m12) + 2.0 * (m13 * m13) +
                                  2.0 * (m23 * m23));
    double cdyn = den == 0.0 ? 0.0 : 0.5 * num / den;
    const double smag = cdyn * (delt * delt);
    F.smag[c] = smag;
    F.scoeff[c] = cdyn;
    const double pranumt = 0.5;
    double mugt = F.rog[c] * smag * d[DY_MOD * n + c];
    if (mugt < 0.0) mugt = 0.0;
    F.mugt[c] = mugt;
    F.kapgt[c] = mugt * F.cg[c] / pranumt;
}

// sgsg (modturbo = 1, and the 2D fall-back of modturbo = 2), every cell
template <int D>
__global__ void k_sgsg(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    if (!fluid(P, c)) {
        F.mugt[c] = 0.0;
        F.kapgt[c] = 0.0;
        return;
    }
    double modsr;
    if (D == 3) {
        int i, j, k;
        ijk_of(P, c, i, j, k);
        Raw3 R;
        raw3(P, i, j, k, R);
        modsr = strain3d(P, F.ug, F.vg, F.wg, R, i, j, k);
    } else {
        modsr = strain2d(P, F.ug, F.wg, c, c % P.nx + 1, c / P.nx + 1);
    }
    const double pranumt = 0.5;
    double mugt = F.rog[c] * F.smag[c] * modsr;
    if (mugt < 0.0) mugt = 0.0;
    F.mugt[c] = mugt;
    F.kapgt[c] = mugt * F.cg[c] / pranumt;
}

// sgss, fluid cells; one thread per (cell, class)
template <int D>
__global__ void k_sgss(Prm P, Fld F) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)P.ncell * (unsigned)P.ns) return;
    int is = (int)(t / (unsigned)P.ncell) + 1, c = (int)(t % (unsigned)P.ncell);
    if (!fluid(P, c)) return;
    size_t off = (size_t)(is - 1) * P.ncell;
    double modsr;
    if (D == 3) {
        int i, j, k;
        ijk_of(P, c, i, j, k);
        Raw3 R;
        raw3(P, i, j, k, R);
        modsr = strain3d(P, F.us + off, F.vs + off, F.ws + off, R, i, j, k);
    } else {
        modsr = strain2d(P, F.us + off, F.ws + off, c, c % P.nx + 1, c / P.nx + 1);
    }
    const double cst = 0.5 * sqrt(2.0);
    double ex = (3.98 * F.rlk[off + c] * P.inrl[is] - 1.69);
    double fact = pdac_fp::pow(10.0, ex);
    F.must[off + c] = cst * P.cmus[is] * P.rl[is] * (P.dk[is] * P.dk[is]) * fact * modsr;
}

// a = a + b over n values (the in-place additions of viscg and htilde)
__global__ void k_accum(double *a, const double *b, size_t n) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] = a[q] + b[q];
}

// a = a + v over n values (viscs: must = must + mus, mus constant per class)
__global__ void k_accum_const(double *a, double v, size_t n) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] = a[q] + v;
}

}  // namespace pdac

// les.cuh -- the sub-grid turbulence model of turbo.f on the device
// (iturb = 1, static Smagorinsky; iss = 1 particle sub-grid stress).
//
// smag = (cmut delta)^2 (x anis in 3D) is fixed per cell at set-up on the
// host (turbulence_setup, turbo.f:42-108).  Each step k_sgsg sets the
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

// strain3d, turbo.f:519-621
__device__ __forceinline__ double strain3d(const Prm &P, const double *u, const double *v, const double *w,
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
    return sqrt(2.0 * (sr11 * sr11 + sr22 * sr22 + sr33 * sr33 + 2.0 * (sr12 * sr12) + 2.0 * (sr13 * sr13) +
                       2.0 * (sr23 * sr23)));
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
    double fact = pow(10.0, ex);
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

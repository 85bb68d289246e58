// solve.cuh -- the per-face phase-coupled momentum system of the corrector,
// sized at compile time.
//
// NP is the number of phases (gas + solid classes).  With NP > 0 every loop
// over phases has a constant trip count and is unrolled, so the matrix and
// right-hand side of a face live in registers; NP = 0 keeps the run-time
// phase count (any nsolid up to PDAC_MAXS) with the arrays in local memory.
// The arithmetic, and its order, is the same for every NP.
#pragma once
#include "phys2d.cuh"

namespace pdac {

template <int NP>
struct Sys {
    static constexpr int M = (NP > 0 ? NP : PDAC_MAXP) + 1;  // 1-based rows and columns
};

template <int NP>
__device__ __forceinline__ int nphases(const Prm &P) { return NP > 0 ? NP : P.nph; }

// Gauss-Jordan with plim decoupling, matrix.f:351-391; a, b 1-based
template <int NP, int M>
__device__ __forceinline__ void gauss_jordan_t(const Prm &P, double (&a)[M][M], double (&b)[M]) {
    const int nph = nphases<NP>(P);
#pragma unroll
    for (int l = 2; l <= nph; ++l) {
        if (fabs(a[l][l]) < P.plim[l - 1]) {
#pragma unroll
            for (int ll = 1; ll <= nph; ++ll) {
                a[ll][ll] = a[ll][ll] + a[l][ll];
                a[l][ll] = 0.0;
                a[ll][l] = 0.0;
            }
            b[l] = 0.0;
        }
    }
#pragma unroll
    for (int l = 1; l <= nph; ++l) {
        if (a[l][l] != 0.0) {
            double div = 1.0 / a[l][l];
#pragma unroll
            for (int lj = l + 1; lj <= nph; ++lj) a[l][lj] = a[l][lj] * div;
            b[l] = b[l] * div;
            a[l][l] = 0.0;
#pragma unroll
            for (int li = 1; li <= nph; ++li) {
                double amul = a[li][l];
#pragma unroll
                for (int lj = l + 1; lj <= nph; ++lj) a[li][lj] = a[li][lj] - amul * a[l][lj];
                b[li] = b[li] - amul * b[l];
            }
        }
    }
}

// Phase matrix of one face, matrix.f:38-328, then its solution stored as the
// face velocities (matrix.f:351-630).  dir 0/1/2 = x/y/z; side +1 = the
// E/N/T face of cell c (assemble_matrix), side -1 = its W/S/B face
// (assemble_all_matrix).  nb = remapped face neighbour, raw = raw face
// neighbour (the cell whose face velocity is stored for side -1), ii = the
// cell's index along dir.  The system is solved only when the raw
// neighbour is fluid.
template <int NP>
__device__ __forceinline__ void face_solve(const Prm &P, const Fld &F, int c, int nb, int raw, int ii, int dir,
                                           int side, double dt) {
    if (!(P.flag[raw] & 1)) return;
    constexpr int M = Sys<NP>::M;
    const int nph = nphases<NP>(P);
    const size_t n = P.ncell;
    const double *dd = dir == 0 ? P.dx : (dir == 1 ? P.dy : P.dz);
    double grav = dir == 0 ? P.gravx : (dir == 1 ? P.gravy : P.gravz);
    const double *app = dir == 0 ? F.appu : (dir == 1 ? F.appv : F.appw);
    const double *rg = dir == 0 ? F.rug : (dir == 1 ? F.rvg : F.rwg);
    const double *rs = dir == 0 ? F.rus : (dir == 1 ? F.rvs : F.rws);
    double alpha = P.alpha, ag = P.alphagrav, pijk = F.p[c];
    double a[M][M], b[M];
    // side +1: d0 = d(ii), d1 = d(ii+1), the face value of c's own row;
    // side -1: d0 = d(ii), d1 = d(ii-1), the row of the lower neighbour
    double d0 = dd[ii], d1 = side > 0 ? dd[ii + 1] : dd[ii - 1];
    double inv = 1.0 / (d0 + d1);
    int rowc = side > 0 ? c : raw;  // cell holding the tilde momentum of this face
    double dp = side > 0 ? pijk - F.p[nb] : F.p[nb] - pijk;
    double ep_f = 1.0;
    if (P.pmodel == 1) ep_f = (d0 * F.ep[nb] + d1 * F.ep[c]) * inv;
    b[1] = rg[rowc] + alpha * dt * inv * 2.0 * ep_f * dp;
    b[1] = b[1] + dt * ag * inv * grav * (d0 * F.rgp[nb] + d1 * F.rgp[c]);
    a[1][1] = alpha * (d0 * app[nb] + d1 * app[c]) * inv;
    a[1][1] = a[1][1] + (d0 * F.rgp[nb] + d1 * F.rgp[c]) * inv;
#pragma unroll
    for (int l = 2; l <= nph; ++l) {
        double rn = F.rlk[(l - 2) * n + nb], rc = F.rlk[(l - 2) * n + c];
        double eps_f = 0.0;
        if (P.pmodel == 1) eps_f = (d0 * rn + d1 * rc) * inv * P.inrl[l - 1];
        b[l] = rs[(l - 2) * n + rowc] + alpha * dt * inv * 2.0 * eps_f * dp;
        b[l] = b[l] + dt * ag * inv * grav * (d0 * rn + d1 * rc);
        int ls1 = l * (l - 1) / 2;
#pragma unroll
        for (int ll = 1; ll <= l; ++ll) {
            int ls = ls1 + ll;
            double v = alpha * (d0 * app[(ls - 1) * n + nb] + d1 * app[(ls - 1) * n + c]) * inv;
            a[l][ll] = v;
            a[ll][l] = v;
        }
        a[l][l] = a[l][l] + (d0 * rn + d1 * rc) * inv;
    }
    gauss_jordan_t<NP>(P, a, b);
    int store = side > 0 ? c : raw;
    double *g = dir == 0 ? F.ug : (dir == 1 ? F.vg : F.wg);
    double *s = dir == 0 ? F.us : (dir == 1 ? F.vs : F.ws);
    g[store] = b[1];
#pragma unroll
    for (int l = 2; l <= nph; ++l) s[(l - 2) * n + store] = b[l];
}

// Warp-aggregated append of cell c to a worklist when want is set: one
// atomic per warp.  Every lane of the warp must reach this call.
__device__ __forceinline__ void work_append(int *list, int *count, int c, bool want) {
    unsigned m = __ballot_sync(0xffffffffu, want);
    if (m == 0) return;
    int lane = threadIdx.x & 31, leader = __ffs(m) - 1, base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) list[base + __popc(m & ((1u << lane) - 1u))] = c;
}

// Warp-aggregated count of the lanes with flag set.  Every lane of the warp
// must reach this call.
__device__ __forceinline__ void warp_count(int *count, bool flag) {
    unsigned m = __ballot_sync(0xffffffffu, flag);
    if (m != 0 && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(count, __popc(m));
}

}  // namespace pdac

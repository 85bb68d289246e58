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

// Phase matrix of one face, matrix.f:38-328, solved (matrix.f:351-630) into
// the face velocities v[0..nph-1] (gas first).  dir 0/1/2 = x/y/z; side +1 =
// the E/N/T face of cell c (assemble_matrix), side -1 = its W/S/B face
// (assemble_all_matrix).  nb = remapped face neighbour, raw = raw face
// neighbour (whose row holds the tilde momentum of a W/S/B face), ii = the
// cell's index along dir.  The cell's own p, ep, rgp and rlk come in
// registers; neighbour values and the tilde terms are read-only here.
template <int NP>
__device__ __forceinline__ void face_system(const Prm &P, const Fld &F, int c, int nb, int raw, int ii, int dir,
                                            int side, double dt, double pc, double epc, double rgpc,
                                            const double *rlkc, double *v) {
    constexpr int M = Sys<NP>::M;
    const int nph = nphases<NP>(P);
    const size_t n = P.ncell;
    const double *dd = dir == 0 ? P.dx : (dir == 1 ? P.dy : P.dz);
    double grav = dir == 0 ? P.gravx : (dir == 1 ? P.gravy : P.gravz);
    const double *app = dir == 0 ? F.appu : (dir == 1 ? F.appv : F.appw);
    const double *rg = dir == 0 ? F.rug : (dir == 1 ? F.rvg : F.rwg);
    const double *rs = dir == 0 ? F.rus : (dir == 1 ? F.rvs : F.rws);
    double alpha = P.alpha, ag = P.alphagrav;
    double a[M][M], b[M];
    // side +1: d0 = d(ii), d1 = d(ii+1); side -1: d0 = d(ii), d1 = d(ii-1)
    double d0 = dd[ii], d1 = side > 0 ? dd[ii + 1] : dd[ii - 1];
    double inv = 1.0 / (d0 + d1);
    int rowc = side > 0 ? c : raw;
    double pnb = __ldg(F.p + nb), rgpnb = __ldg(F.rgp + nb);
    double dp = side > 0 ? pc - pnb : pnb - pc;
    double ep_f = 1.0;
    if (P.pmodel == 1) ep_f = (d0 * __ldg(F.ep + nb) + d1 * epc) * inv;
    b[1] = __ldg(rg + rowc) + alpha * dt * inv * 2.0 * ep_f * dp;
    b[1] = b[1] + dt * ag * inv * grav * (d0 * rgpnb + d1 * rgpc);
    a[1][1] = alpha * (d0 * __ldg(app + nb) + d1 * __ldg(app + c)) * inv;
    a[1][1] = a[1][1] + (d0 * rgpnb + d1 * rgpc) * inv;
#pragma unroll
    for (int l = 2; l <= nph; ++l) {
        double rn = __ldg(F.rlk + (l - 2) * n + nb), rc = rlkc[l - 2];
        double eps_f = 0.0;
        if (P.pmodel == 1) eps_f = (d0 * rn + d1 * rc) * inv * P.inrl[l - 1];
        b[l] = __ldg(rs + (l - 2) * n + rowc) + alpha * dt * inv * 2.0 * eps_f * dp;
        b[l] = b[l] + dt * ag * inv * grav * (d0 * rn + d1 * rc);
        int ls1 = l * (l - 1) / 2;
#pragma unroll
        for (int ll = 1; ll <= l; ++ll) {
            int ls = ls1 + ll;
            double val = alpha * (d0 * __ldg(app + (ls - 1) * n + nb) + d1 * __ldg(app + (ls - 1) * n + c)) * inv;
            a[l][ll] = val;
            a[ll][l] = val;
        }
        a[l][l] = a[l][l] + (d0 * rn + d1 * rc) * inv;
    }
    gauss_jordan_t<NP>(P, a, b);
#pragma unroll
    for (int l = 1; l <= nph; ++l) v[l - 1] = b[l];
}

// face_system with the cell's state read from and the velocities stored to
// memory, when the raw face neighbour is fluid (the predictor, iter.f:135-145)
template <int NP>
__device__ __forceinline__ void face_solve(const Prm &P, const Fld &F, int c, int nb, int raw, int ii, int dir,
                                           int side, double dt) {
    if (!(P.flag[raw] & 1)) return;
    constexpr int M = Sys<NP>::M;
    const int nph = nphases<NP>(P);
    const size_t n = P.ncell;
    double rlkc[M - 1], v[M - 1];
#pragma unroll
    for (int l = 2; l <= nph; ++l) rlkc[l - 2] = F.rlk[(l - 2) * n + c];
    face_system<NP>(P, F, c, nb, raw, ii, dir, side, dt, F.p[c], F.ep[c], F.rgp[c], rlkc, v);
    int store = side > 0 ? c : raw;
    double *g = dir == 0 ? F.ug : (dir == 1 ? F.vg : F.wg);
    double *s = dir == 0 ? F.us : (dir == 1 ? F.vs : F.ws);
    g[store] = v[0];
#pragma unroll
    for (int l = 2; l <= nph; ++l) s[(l - 2) * n + store] = v[l - 1];
}

// value of a stencil slot: the cell's own current value where the (remapped)
// slot index is the cell itself, else the read-only neighbour value
__device__ __forceinline__ double slot(const double *a, int idx, int c, double own) {
    return idx == c ? own : __ldg(a + idx);
}

// Block-aggregated append of up to CAP cells per thread (cells[0..ncand))
// and count of tested cells (tested_count may be NULL): one atomic per block
// and counter.  Every thread of the block (TPBK threads) must reach this call.
template <int TPBK, int CAP>
__device__ __forceinline__ void block_append_n(int *list, int *count, const int *cells, int ncand, int *tested_count,
                                               int ntested) {
    constexpr int NW = TPBK / 32;
    __shared__ int s_off[NW], s_tst[NW], s_base;
    const unsigned full = 0xffffffffu;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = ncand;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += v;
    }
    int tst = ntested;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tst += __shfl_xor_sync(full, tst, o);
    if (lane == 31) s_off[wid] = incl;
    if (lane == 0) s_tst[wid] = tst;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0, tt = 0;
        for (int w = 0; w < NW; ++w) { int v = s_off[w]; s_off[w] = tot; tot += v; tt += s_tst[w]; }
        s_base = tot ? atomicAdd(count, tot) : 0;
        if (tt && tested_count) atomicAdd(tested_count, tt);
    }
    __syncthreads();
    int off = s_base + s_off[wid] + incl - ncand;
#pragma unroll 1
    for (int q = 0; q < ncand && q < CAP; ++q) list[off + q] = cells[q];
    __syncthreads();
}

// set the active-set bit of cell x (one bit per cell, 32 per word)
__device__ __forceinline__ void mark_dirty(unsigned *dirty, int x) { atomicOr(dirty + (x >> 5), 1u << (x & 31)); }

}  // namespace pdac

// tiles3d.cuh -- shared-memory tiled stencil passes of the 3D path.
//
// A block owns a TX x TY column of cells (i fastest, then j) and marches up
// k through a chunk of planes.  The fields a pass reads for planes k-2 ..
// k+3 sit in a ring of six shared-memory planes of (TX + 5) x (TY + 5)
// cells: the block's cells plus the halo the reference's stencils reach
// (subscr.f: two cells on the minus side, three on the plus side).  Every
// halo position holds the value of the clamped global cell that raw3 (the
// myijk table, ghost.f:486-680) names for it, so the stencil of a cell is
// read from the tile at fixed offsets: the same values, hence the same
// results, as the one-thread-per-cell gathers from global memory.  Each
// plane is loaded once per block, in rows of consecutive i (coalesced), and
// the vertical halo is shared by the k steps of the march.
#pragma once
#include "kernels3d.cuh"

namespace pdac {

constexpr int TILE_RING = 6;  // planes k-2 .. k+3

// raw neighbour indices inside a tile: in-plane position lc of the cell,
// plane stride SX, and the offsets of the ring slots of planes k-2 .. k+3
__device__ __forceinline__ void raw3_tile(Raw3 &R, int lc, int SX, const int *poff) {
    auto f = [&](int di, int dj, int dk) { return lc + di + SX * dj + poff[dk + 2]; };
    R.c = f(0, 0, 0);
    R.e = f(1, 0, 0); R.w = f(-1, 0, 0); R.n = f(0, 1, 0); R.s = f(0, -1, 0); R.t = f(0, 0, 1); R.b = f(0, 0, -1);
    R.ee = f(2, 0, 0); R.ww = f(-2, 0, 0); R.nn = f(0, 2, 0); R.ss = f(0, -2, 0); R.tt = f(0, 0, 2); R.bb = f(0, 0, -2);
    R.en = f(1, 1, 0); R.wn = f(-1, 1, 0); R.es = f(1, -1, 0); R.ws = f(-1, -1, 0);
    R.et = f(1, 0, 1); R.wt = f(-1, 0, 1); R.nt = f(0, 1, 1); R.st = f(0, -1, 1);
    R.eb = f(1, 0, -1); R.wb = f(-1, 0, -1); R.nb = f(0, 1, -1); R.sb = f(0, -1, -1);
    R.eet = f(2, 0, 1); R.een = f(2, 1, 0); R.enn = f(1, 2, 0); R.nnt = f(0, 2, 1); R.ett = f(1, 0, 2); R.ntt = f(0, 1, 2);
    R.eee = f(3, 0, 0); R.nnn = f(0, 3, 0); R.ttt = f(0, 0, 3);
}

// bytes of shared memory of a tile pass over nf fields of type Real
template <int TX, int TY, typename Real>
constexpr int tile_smem_bytes(int nf) {
    return TILE_RING * (TX + 5) * (TY + 5) * (nf * (int)sizeof(Real) + (int)sizeof(int));
}

// Momentum face fluxes of all three components of one phase, tilde.f:850-1326
// with flu/flv/flw and their MUSCL corrections (flux_u.f, flux_v.f,
// flux_w.f): what k_tilde_flux3d<0|1|2> compute, from one staged copy of the
// phase's velocities and density.  Grid: (ceil(nx / TX), ceil(ny / TY),
// nphase * nchunk), chunks of kchunk planes; dynamic shared memory
// tile_smem_bytes<TX, TY, Real>(4).
template <int TX, int TY, typename Real = double>
__global__ void __launch_bounds__(TX * TY, 384 / (TX * TY)) k_mom_flux3d_tile(Prm P, Fld F, int kchunk) {
    constexpr int SX = TX + 5, SY = TY + 5, PL = SX * SY, NR = TILE_RING, NT = TX * TY;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    Real *sv = reinterpret_cast<Real *>(tile_smem);          // [4][NR][PL]: u, v, w, density
    int *sf = reinterpret_cast<int *>(sv + 4 * NR * PL);      // [NR][PL]: flags
    const int nph = P.ns + 1;
    const int ph = blockIdx.z % nph, chunk = blockIdx.z / nph;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
    const int kb = 1 + chunk * kchunk, ke = min(P.nz, kb + kchunk - 1);
    const size_t n = P.ncell, off = (size_t)(ph > 0 ? ph - 1 : 0) * n;
    const double *U = ph == 0 ? F.ug : F.us + off;
    const double *V = ph == 0 ? F.vg : F.vs + off;
    const double *W = ph == 0 ? F.wg : F.ws + off;
    const double *D = ph == 0 ? F.rgp : F.rlk + off;
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    // plane kg (clamped to [1, nz], as raw3 clamps) into its ring slot
    auto load_plane = [&](int kg) {
        const int kc = clampi(kg, 1, P.nz), slot = ((kg % NR) + NR) % NR;
        const size_t base = (size_t)P.nx * P.ny * (kc - 1);
        for (int q = tid; q < PL; q += NT) {
            const int li = q % SX, lj = q / SX;
            const int gi = clampi(i0 - 2 + li, 1, P.nx), gj = clampi(j0 - 2 + lj, 1, P.ny);
            const size_t g = base + (size_t)(gi - 1) + (size_t)P.nx * (gj - 1);
            sv[(0 * NR + slot) * PL + q] = (Real)__ldg(U + g);
            sv[(1 * NR + slot) * PL + q] = (Real)__ldg(V + g);
            sv[(2 * NR + slot) * PL + q] = (Real)__ldg(W + g);
            sv[(3 * NR + slot) * PL + q] = (Real)__ldg(D + g);
            sf[slot * PL + q] = __ldg(P.flag + g);
        }
    };
    for (int kg = kb - 2; kg <= kb + 2; ++kg) load_plane(kg);
    const Real *su = sv, *svv = sv + NR * PL, *sw = sv + 2 * NR * PL, *sd = sv + 3 * NR * PL;
    for (int k = kb; k <= ke; ++k) {
        load_plane(k + 3);
        __syncthreads();
        const int i = i0 + tx, j = j0 + ty;
        int poff[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) poff[q] = (((k - 2 + q) % NR + NR) % NR) * PL;
        const int lc = (tx + 2) + SX * (ty + 2);
        if (i <= P.nx && j <= P.ny && (sf[lc + poff[2]] & 1)) {
            const int fc = sf[lc + poff[2]];
            const bool dw = !(sf[lc - 1 + poff[2]] & 1), ds = !(sf[lc - SX + poff[2]] & 1), db = !(sf[lc + poff[1]] & 1);
            const bool mus = P.muscl > 0 && fc == FLUID;
            const int c = at3(P, i, j, k), cw = c - 1, cs = c - P.nx, cb = c - P.nx * P.ny;
#pragma unroll 1
            for (int comp = 0; comp < 3; ++comp) {
                // the tile indices, rebuilt per component (integer work is
                // cheaper than holding ~60 indices across the loop)
                Raw3 R;
                Rem3 M;
                raw3_tile(R, lc, SX, poff);
                rem3_fl(P, sf, i, j, k, R, M);
                S3T<Real> u, v, w, d, ds3;
                rnb3(u, su, R);
                rnb3(v, svv, R);
                rnb3(w, sw, R);
                nb3(d, sd, R, M);
                F6T<Real> f = {0, 0, 0, 0, 0, 0};
                if (comp == 0) {
                    interp_x3(P, d, i, ds3);
                    flu_3d(P, f, dw, ds, db, ds3, u, v, w, i);
                    if (mus && i != P.nx - 1) muscl_flu_3d(P, f, ds3, u, v, w, i, j, k);
                } else if (comp == 1) {
                    interp_y3(P, d, j, ds3);
                    flv_3d(P, f, dw, ds, db, ds3, u, v, w, j);
                    if (mus && j != P.ny - 1) muscl_flv_3d(P, f, ds3, u, v, w, i, j, k);
                } else {
                    interp_z3(P, d, k, ds3);
                    flw_3d(P, f, dw, ds, db, ds3, u, v, w, k);
                    if (mus && k != P.nz - 1) muscl_flw_3d(P, f, ds3, u, v, w, i, j, k);
                }
                MFX(ph, comp, 0)[c] = f.e; MFX(ph, comp, 1)[c] = f.n; MFX(ph, comp, 2)[c] = f.t;
                if (dw) MFX(ph, comp, 0)[cw] = f.w;
                if (ds) MFX(ph, comp, 1)[cs] = f.s;
                if (db) MFX(ph, comp, 2)[cb] = f.b;
            }
        }
        __syncthreads();  // every thread is done with plane k-2 before its slot takes plane k+4
    }
}

}  // namespace pdac

// common.cuh -- shared definitions of the B200 PDAC engine (sm_100a).
//
// Data layout in HBM: one flat index c = i0 + nx*(j0 + ny*k0) over all
// cells including the one-cell boundary frame (the reference's ijk order,
// i fastest), structure-of-arrays, one contiguous array per field; per-solid
// and per-gas fields are (ncell, n) column-major, i.e. class-major blocks of
// ncell values.  Mesh metric arrays are 1-based with padding so that device
// formulas use the reference's indices (dx(i-1), dx(i+2) ...) unchanged.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fpmath.h"  // exp and pow with the same bits as the host's (the oracle's)

#define PDAC_MAXS 8          // max solid classes
#define PDAC_MAXP (PDAC_MAXS + 1)
#define PDAC_MAXG 7
#define TPB_RESID 256        // threads per block of the corrector's residual test

// Register caps of the 128-thread stencil kernels, as the minimum number of
// resident blocks per SM passed to __launch_bounds__.  Uncapped, the 3D
// momentum and stress kernels take 150-200 registers a thread and run at
// 2-3 blocks per SM, too few warps to cover their gathers' latency.  4 blocks
// (128 registers) suits the momentum flux and stress kernels, 6 blocks (80
// registers) the scalar flux kernels; a tighter cap makes the momentum
// kernels spill.
#ifndef PDAC_FLUX_MINB
#define PDAC_FLUX_MINB 4
#endif
#ifndef PDAC_SCALAR_FLUX_MINB
#define PDAC_SCALAR_FLUX_MINB 6
#endif

namespace pdac {

// cell flags, grid.f:45-58
enum : int { FLUID = 1, SLIP = 2, NOSLIP = 4, BL_CELL = 5, FREE_IO = 8, INLET = 16, ZERO_GRAD = 32,
             VENT = 64, DOME = 129, IMMB = 257, FILLED1 = 512, FILLED2 = 1024 };

// Scalar run parameters, passed by value to every kernel.
struct Prm {
    int nx, ny, nz, ncell, ns, ng, nph, nap;
    int d3;  // 1 for the 3D Cartesian path, 0 for 2D (x, z)
    int itc, muscl, lv, lm, pmodel, drag_model, icpc;
    int gas_viscosity, part_viscosity, repulsive_model, inmax;
    int iturb, iss, modturbo;  // sub-grid models (turbo.f)
    int opt;                   // 2: opt_inner_loop's loop-entry density in self-remapped stencil slots
    int gas_type[PDAC_MAXG];
    double alpha, alphagrav, omega, delg, beta, flim, tref;
    double gravx, gravy, gravz, void_fraction;
    double atm_ygc[PDAC_MAXG];
    double gmw[8], mmugs[8], mmugek[8];
    double rgas, gammaair;
    double dk[PDAC_MAXP], rl[PDAC_MAXP], inrl[PDAC_MAXP], phis[PDAC_MAXP], cmus[PDAC_MAXP];
    double cps[PDAC_MAXP], kap[PDAC_MAXP], plim[PDAC_MAXP], phi[PDAC_MAXP];
    double philim[PDAC_MAXP][PDAC_MAXP], epsl[PDAC_MAXP][PDAC_MAXP], epsu[PDAC_MAXP][PDAC_MAXP];
    double dkf[PDAC_MAXP][PDAC_MAXP];
    // device metric, 1-based padded
    const double *dx, *dy, *dz, *indx, *indy, *indz, *r, *rb, *inr, *inrb;
    // hx[m] = 1 / (dx[m] + dx[m+1]) over the padded range (hy, hz alike): the
    // reciprocal face spacings of interp.f and flux_*.f, divided once on the host
    // (an IEEE division, so the same bits as dividing in the kernel)
    const double *hx, *hy, *hz;
    const float *dxf, *dyf, *dzf, *indxf, *indyf, *indzf, *hxf, *hyf, *hzf, *rf, *rbf;  // FP32 copies (mixed precision), else null
    int mixed;  // 1: the face-flux passes compute in FP32 (PDAC_PREC_MIXED)
    // c / nx and c / (nx ny) as a 64-bit multiply-high: mnx = ceil(2^64 / nx)
    // (mny likewise for ny), exact for every c < 2^32; 0 = divide instead
    unsigned long long mnx, mny;
    const double *p_atm, *t_atm;
    const int *flag;
    // immersed boundaries (immb.f, ghost.f:2888-3345); immb = 0: none, and
    // every face factor below reads as 1
    int immb;
    const int *ib_faces;     // per cell: the open faces b_e_ .. b_s_ as bits (1 E, 2 W, 4 T, 8 B, 16 N, 32 S)
    const double *ib_ivf;    // per cell: ivf_, 1 / fluid volume fraction
    const int *ib_num[3];    // per cell: numx, numy, numz (1-based forcing point, 0 none)
    const double *ib_vel[3]; // per forcing point: the nph velocities of the last boundary pass
};

// The face factors of one cell (faces, immb.f:1263-1278); all 1 without
// immersed boundaries, as face_init sets them (ghost.f:3323-3344).
struct CellFaces {
    double e, w, n, s, t, b, ivf;
};
__device__ __forceinline__ CellFaces cell_faces(const Prm &P, int c) {
    CellFaces f = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
    if (P.immb) {
        const int m = __ldg(P.ib_faces + c);
        f.e = (m & 1) ? 1.0 : 0.0;
        f.w = (m & 2) ? 1.0 : 0.0;
        f.t = (m & 4) ? 1.0 : 0.0;
        f.b = (m & 8) ? 1.0 : 0.0;
        f.n = (m & 16) ? 1.0 : 0.0;
        f.s = (m & 32) ? 1.0 : 0.0;
        f.ivf = __ldg(P.ib_ivf + c);
    }
    return f;
}

// The metric arrays in the arithmetic type of a flux pass.
template <typename Real> struct Met;
template <> struct Met<double> {
    static __device__ __forceinline__ const double *dx(const Prm &P) { return P.dx; }
    static __device__ __forceinline__ const double *dy(const Prm &P) { return P.dy; }
    static __device__ __forceinline__ const double *dz(const Prm &P) { return P.dz; }
    static __device__ __forceinline__ const double *indx(const Prm &P) { return P.indx; }
    static __device__ __forceinline__ const double *indy(const Prm &P) { return P.indy; }
    static __device__ __forceinline__ const double *indz(const Prm &P) { return P.indz; }
    static __device__ __forceinline__ const double *hx(const Prm &P) { return P.hx; }
    static __device__ __forceinline__ const double *hy(const Prm &P) { return P.hy; }
    static __device__ __forceinline__ const double *hz(const Prm &P) { return P.hz; }
    static __device__ __forceinline__ const double *r(const Prm &P) { return P.r; }
    static __device__ __forceinline__ const double *rb(const Prm &P) { return P.rb; }
};
template <> struct Met<float> {
    static __device__ __forceinline__ const float *dx(const Prm &P) { return P.dxf; }
    static __device__ __forceinline__ const float *dy(const Prm &P) { return P.dyf; }
    static __device__ __forceinline__ const float *dz(const Prm &P) { return P.dzf; }
    static __device__ __forceinline__ const float *indx(const Prm &P) { return P.indxf; }
    static __device__ __forceinline__ const float *indy(const Prm &P) { return P.indyf; }
    static __device__ __forceinline__ const float *indz(const Prm &P) { return P.indzf; }
    static __device__ __forceinline__ const float *hx(const Prm &P) { return P.hxf; }
    static __device__ __forceinline__ const float *hy(const Prm &P) { return P.hyf; }
    static __device__ __forceinline__ const float *hz(const Prm &P) { return P.hzf; }
    static __device__ __forceinline__ const float *r(const Prm &P) { return P.rf; }
    static __device__ __forceinline__ const float *rb(const Prm &P) { return P.rbf; }
};

// Device pointers of every field (state, n-level, tilde, fluxes, solver).
struct Fld {
    double *p, *ep, *rog, *rgp, *tg, *sieg, *cg, *ug, *vg, *wg;
    double *rlk, *ts, *sies, *us, *vs, *ws, *ygc, *xgc;
    double *pn, *epn, *rgpn, *siegn, *rlkn, *siesn, *rgpgcn, *mug, *kapg;
    double *rugn, *rvgn, *rwgn, *rusn, *rvsn, *rwsn;
    double *rug, *rvg, *rwg, *rus, *rvs, *rws, *appu, *appv, *appw;
    double *ugfe, *ugft, *wgfe, *wgft, *usfe, *usft, *wsfe, *wsft;  // 2D momentum fluxes
    double *mf;  // 3D momentum fluxes, block ((phase*3 + component)*3 + face) of ncell values
    double *vis; // 3D viscous stress divergence, block (phase*3 + component) of ncell values
    double *rgfe, *rgfn, *rgft, *rsfe, *rsfn, *rsft, *conv, *abeta;
    double *egfe, *egfn, *egft, *esfe, *esfn, *esft, *rhg, *rhs;
    double *yfe, *yfn, *yft;
    double *sink;
    double *smag, *mugt, *kapgt, *must;  // sub-grid model (turbo.f:10-14); must (ncell, ns)
    double *dyn, *delt, *scoeff;         // dynamic model: per-cell work blocks, filter width, cdyn
    double *rhom, *um, *vm, *wm, *tm, *yd;  // mixture fields (mixture.f); yd (ncell, ng + ns)
    int *counters;  // [0] non-converged cells this sweep, [1] eos failures, [2] rls>1 cells, [3] boundary errors
};

__host__ __device__ inline bool is_wall(int f) { return f == SLIP || f == NOSLIP; }
__host__ __device__ inline bool is_wallf(int f) { return f == SLIP || f == NOSLIP || f == FILLED1; }
__host__ __device__ inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace pdac

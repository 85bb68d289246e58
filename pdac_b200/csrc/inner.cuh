// inner.cuh -- inner_loop of the corrector (iter.f:480-580) on a team of
// lanes per cell.
//
// A team of T lanes (6 in 3D, 4 in 2D) owns one unconverged cell of the
// worklist.  Lane q < NF owns face q of the cell (3D: W, S, B, E, N, T; 2D:
// W, B, E, T): it assembles and solves that face's phase system and computes
// that face's mass fluxes.  The per-cell quantities (pressure adjustment,
// equation of state, volume fractions, continuity residual) are evaluated by
// every lane of the team from the same inputs, so all lanes hold identical
// values and take the same branches; face values reach the other lanes by
// warp shuffles.  Each value is computed with the same operations in the same
// order as the one-thread form, and the cell's state, face velocities and
// fluxes stay in registers until the final store (nothing else touches the
// cell's neighbourhood within a colour phase).
#pragma once
#include <cooperative_groups.h>
#include "kernels3d.cuh"

namespace pdac {

// a load of a value that no thread of the current launch writes: through
// the read-only cache in the one-launch-per-colour-phase form (RO); a plain
// load in the persistent form, where other blocks write it between the
// phases (separated by grid-wide barriers)
template <bool RO>
__device__ __forceinline__ double ldro(const double *p) {
    if (RO) return __ldg(p);
    return *p;
}

// mass flux through one face (masf + fmas, flux_m.f:47-324), written for a
// face on the minus side (W/S/B) or the plus side (E/N/T) of the cell.
// dc = cell value, dm/dmm = first/second neighbour on the minus side, dp/dpp
// on the plus side; r = radial factor of x faces in cylindrical 2D, else 1.
struct FaceGeo {
    double inmm, inm, inp, inpp, incr_p, incr_m, r;
    bool lim_on;
};

__device__ __forceinline__ double face_mflux(const Prm &P, const FaceGeo &g, bool minus, double cs, double dc,
                                             double dm, double dmm, double dp, double dpp, bool mus) {
    double f;
    if (minus) f = 0.5 * (cs - fabs(cs)) * dc * g.r + 0.5 * (cs + fabs(cs)) * dm * g.r;
    else f = 0.5 * (cs - fabs(cs)) * dp * g.r + 0.5 * (cs + fabs(cs)) * dc * g.r;
    if (!mus) return f;
    double gradc, gradm, gradp;
    if (minus) {
        gradc = 2.0 * g.inm * (dc - dm);
        gradm = 2.0 * g.inmm * (dm - dmm);
        gradp = 2.0 * g.inp * (dp - dc);
    } else {
        gradm = 2.0 * g.inm * (dc - dm);
        gradc = 2.0 * g.inp * (dp - dc);
        gradp = 2.0 * g.inpp * (dpp - dp);
    }
    double erre = 0, incr = 0, lim = 0;
    if (cs >= 0) { if (gradc != 0) erre = gradm / gradc; incr = g.incr_p; }
    else if (cs < 0) { if (gradc != 0) erre = gradp / gradc; incr = g.incr_m; }
    if (g.lim_on) lim = limiter(P.lm, erre, P.beta);
    double upwnd = lim * gradc * incr;
    return f + upwnd * cs * g.r;
}

// Loop-invariant part of one face's phase system (matrix.f:38-328) for the
// cell's inner loop: everything that does not depend on the cell's own p,
// ep, rgp and rlk, evaluated once with the operations of face_system so that
// the in-loop assembly (face_assemble) reproduces face_system bit for bit:
// A(ls) = alpha (d0 app(nb) + d1 app(c)) / (d0 + d1) by interphase index,
// brow(l) the tilde momenta of the face (gas first), d0rn(l) = d0 x the
// neighbour bulk densities (l = 0: d0 rgp(nb)), and six scalars.  Two
// storage forms with one interface: SH = true keeps them in this lane's
// column of a shared [N][KS] array (blocks of KS threads), which frees ~50
// registers of the inner loop for a third resident block per SM; SH = false
// (the generic phase count, whose array would not fit) keeps them in
// registers.
constexpr int KS = 128;  // threads per block of every kernel running the inner loop

template <int NP, bool SH>
struct FaceK;

template <int NP>
struct FaceK<NP, false> {
    static constexpr int M = Sys<NP>::M, NA = M * (M - 1) / 2;
    double A_[NA], brow_[M - 1], d0rn_[M - 1], sc_[6];
    __device__ __forceinline__ explicit FaceK(double *) {}
    __device__ __forceinline__ double &A(int i) { return A_[i]; }
    __device__ __forceinline__ double &brow(int l) { return brow_[l]; }
    __device__ __forceinline__ double &d0rn(int l) { return d0rn_[l]; }
    __device__ __forceinline__ double &sc(int q) { return sc_[q]; }
};

template <int NP>
struct FaceK<NP, true> {
    static constexpr int M = Sys<NP>::M, NA = M * (M - 1) / 2, N = NA + 2 * (M - 1) + 6;
    double *s;  // this lane's column: element q at s[q * KS]
    __device__ __forceinline__ explicit FaceK(double *col) : s(col) {}
    __device__ __forceinline__ double &A(int i) { return s[i * KS]; }
    __device__ __forceinline__ double &brow(int l) { return s[(NA + l) * KS]; }
    __device__ __forceinline__ double &d0rn(int l) { return s[(NA + M - 1 + l) * KS]; }
    __device__ __forceinline__ double &sc(int q) { return s[(NA + 2 * (M - 1) + q) * KS]; }
};

// the six scalars of FaceK
enum { FK_PNB = 0, FK_D0EPNB, FK_K1, FK_K2, FK_D1, FK_INV };

// The loop-invariant density stencil of one face's mass fluxes by phase:
// the near (cm, cp) and far (cf) neighbour values and the cell's own values
// at loop entry (o, read by opt_inner_loop's stale slots).  SH = true keeps
// them in this lane's column of a shared [4 NC][KS] array, as FaceK does.
template <int NC, bool SH>
struct DensK;

template <int NC>
struct DensK<NC, false> {
    double cm_[NC], cp_[NC], cf_[NC], o_[NC];
    __device__ __forceinline__ explicit DensK(double *) {}
    __device__ __forceinline__ double &cm(int l) { return cm_[l]; }
    __device__ __forceinline__ double &cp(int l) { return cp_[l]; }
    __device__ __forceinline__ double &cf(int l) { return cf_[l]; }
    __device__ __forceinline__ double &o(int l) { return o_[l]; }
};

template <int NC>
struct DensK<NC, true> {
    double *s;  // this lane's column: element q at s[q * KS]
    __device__ __forceinline__ explicit DensK(double *col) : s(col) {}
    __device__ __forceinline__ double &cm(int l) { return s[l * KS]; }
    __device__ __forceinline__ double &cp(int l) { return s[(NC + l) * KS]; }
    __device__ __forceinline__ double &cf(int l) { return s[(2 * NC + l) * KS]; }
    __device__ __forceinline__ double &o(int l) { return s[(3 * NC + l) * KS]; }
};

template <int NP, bool RO, class KT>
__device__ __forceinline__ void face_prepare(const Prm &P, const Fld &F, int c, int nb, int raw, int ii, int dir,
                                             int side, double dt, KT &K) {
    const int nph = nphases<NP>(P);
    const size_t n = P.ncell;
    const double *dd = dir == 0 ? P.dx : (dir == 1 ? P.dy : P.dz);
    double grav = dir == 0 ? P.gravx : (dir == 1 ? P.gravy : P.gravz);
    const double *app = dir == 0 ? F.appu : (dir == 1 ? F.appv : F.appw);
    const double *rg = dir == 0 ? F.rug : (dir == 1 ? F.rvg : F.rwg);
    const double *rs = dir == 0 ? F.rus : (dir == 1 ? F.rvs : F.rws);
    double alpha = P.alpha, ag = P.alphagrav;
    double d0 = dd[ii], d1 = side > 0 ? dd[ii + 1] : dd[ii - 1];
    double inv = 1.0 / (d0 + d1);
    int rowc = side > 0 ? c : raw;
    K.sc(FK_D1) = d1;
    K.sc(FK_INV) = inv;
    K.sc(FK_PNB) = ldro<RO>(F.p + nb);
    K.sc(FK_D0EPNB) = P.pmodel == 1 ? d0 * ldro<RO>(F.ep + nb) : 0.0;
    K.sc(FK_K1) = alpha * dt * inv * 2.0;
    K.sc(FK_K2) = dt * ag * inv * grav;
    K.brow(0) = ldro<RO>(rg + rowc);
    K.d0rn(0) = d0 * ldro<RO>(F.rgp + nb);
#pragma unroll
    for (int l = 2; l <= nph; ++l) {
        K.brow(l - 1) = ldro<RO>(rs + (l - 2) * n + rowc);
        K.d0rn(l - 1) = d0 * ldro<RO>(F.rlk + (l - 2) * n + nb);
    }
    const int nap = nph * (nph + 1) / 2;
#pragma unroll
    for (int ls = 1; ls <= nap; ++ls)
        K.A(ls - 1) = alpha * (d0 * ldro<RO>(app + (ls - 1) * n + nb) + d1 * ldro<RO>(app + (ls - 1) * n + c)) * inv;
}

// the in-loop assembly and solution; side as in face_system
template <int NP, class KT>
__device__ __forceinline__ void face_assemble(const Prm &P, KT &K, int side, double pc, double epc,
                                              double rgpc, const double *rlkc, double *v) {
    constexpr int M = Sys<NP>::M;
    const int nph = nphases<NP>(P);
    double a[M][M], b[M];
    double d1 = K.sc(FK_D1), inv = K.sc(FK_INV), pnb = K.sc(FK_PNB), K1 = K.sc(FK_K1), K2 = K.sc(FK_K2);
    double dp = side > 0 ? pc - pnb : pnb - pc;
    double ep_f = 1.0;
    if (P.pmodel == 1) ep_f = (K.sc(FK_D0EPNB) + d1 * epc) * inv;
    b[1] = K.brow(0) + K1 * ep_f * dp;
    b[1] = b[1] + K2 * (K.d0rn(0) + d1 * rgpc);
    a[1][1] = K.A(0) + (K.d0rn(0) + d1 * rgpc) * inv;
#pragma unroll
    for (int l = 2; l <= nph; ++l) {
        double rc = rlkc[l - 2];
        double eps_f = 0.0;
        if (P.pmodel == 1) eps_f = (K.d0rn(l - 1) + d1 * rc) * inv * P.inrl[l - 1];
        b[l] = K.brow(l - 1) + K1 * eps_f * dp;
        b[l] = b[l] + K2 * (K.d0rn(l - 1) + d1 * rc);
        int ls1 = l * (l - 1) / 2;
#pragma unroll
        for (int ll = 1; ll <= l; ++ll) {
            double val = K.A(ls1 + ll - 1);
            a[l][ll] = val;
            a[ll][l] = val;
        }
        a[l][l] = a[l][l] + (K.d0rn(l - 1) + d1 * rc) * inv;
    }
    gauss_jordan_t<NP>(P, a, b);
#pragma unroll
    for (int l = 1; l <= nph; ++l) v[l - 1] = b[l];
}

// minimum resident blocks per SM the register allocation must allow: with
// the face terms in shared memory, up to four phases fit 168 registers and
// three blocks per SM without spilling; more phases take two blocks
#ifndef PDAC_INNER_MINB_SMALL
#define PDAC_INNER_MINB_SMALL 3
#endif
#ifndef PDAC_INNER_MINB_LARGE
#define PDAC_INNER_MINB_LARGE 2
#endif
#define PDAC_INNER_MINB(NP) ((NP) > 0 && (NP) <= 4 ? PDAC_INNER_MINB_SMALL : PDAC_INNER_MINB_LARGE)
#ifndef PDAC_INNER_SHD_MAXP
#define PDAC_INNER_SHD_MAXP 6
#endif

// the inner loop's shared memory, allocated at launch (dynamic): FaceK
// columns for up to six phases, then DensK columns up to
// PDAC_INNER_SHD_MAXP phases (64.5 KB per block at six phases)
template <int NP>
__host__ __device__ constexpr int inner_face_rows() { return (NP > 0 && NP <= 6) ? FaceK<NP, true>::N : 0; }
template <int NP>
__host__ __device__ constexpr int inner_dens_rows() {
    return (NP > 0 && NP <= PDAC_INNER_SHD_MAXP) ? 4 * (Sys<NP>::M - 1) : 0;
}
template <int NP>
__host__ __device__ constexpr size_t inner_smem_bytes() {
    return (size_t)(inner_face_rows<NP>() + inner_dens_rows<NP>()) * KS * sizeof(double);
}

// The inner loop of cell c (outer sweep nit, 1-based) by the team of lanes
// tb .. tb + T - 1 of this warp (lane q of the team owns face q); kcols and
// dcols are the shared FaceK and DensK arrays.  RO as in ldro.
template <int NP, int D, bool RO>
__device__ __forceinline__ void inner_team_cell(const Prm &P, const Fld &F, double dt, int nit, int c, unsigned *dirty,
                                                int q, int tb, unsigned tmask, double *kcols, double *dcols) {
    constexpr int NC = Sys<NP>::M - 1;   // phase capacity
    constexpr bool SH = inner_face_rows<NP>() > 0;   // FaceK in shared memory (40 KB per block at NP = 6)
    constexpr bool SHD = inner_dens_rows<NP>() > 0;  // DensK too (16 KB at NP = 4, 24 KB at NP = 6)
    const int nph = nphases<NP>(P), ns = nph - 1;
    const size_t n = P.ncell;
    int i, j, k;
    if (D == 3) ijk_of(P, c, i, j, k);
    else { i = c % P.nx + 1; j = 1; k = c / P.nx + 1; }
    const int *fl = P.flag;
    // ---- this lane's face: axis, side, raw and remapped neighbours -------
    const int a = D == 3 ? q % 3 : q % 2;
    const bool minus = D == 3 ? q < 3 : q < 2;
    const int dir = D == 3 ? a : (a == 0 ? 0 : 2);
    const int ii = dir == 0 ? i : (dir == 1 ? j : k);
    const int nax = dir == 0 ? P.nx : (dir == 1 ? P.ny : P.nz);
    int raw_m, raw_p, rm, rmm, rp, rpp;
    if (D == 3) {
        Raw3 R;
        Rem3 M;
        raw3(P, i, j, k, R);
        rem3(P, i, j, k, R, M);
        if (dir == 0) { raw_m = R.w; raw_p = R.e; rm = M.w; rmm = M.ww; rp = M.e; rpp = M.ee; }
        else if (dir == 1) { raw_m = R.s; raw_p = R.n; rm = M.s; rmm = M.ss; rp = M.n; rpp = M.nn; }
        else { raw_m = R.b; raw_p = R.t; rm = M.b; rmm = M.bb; rp = M.t; rpp = M.tt; }
    } else {
        Raw2 R;
        Rem2 M;
        raw2(P, i, k, R);
        rem2(P, i, k, R, M);
        if (dir == 0) { raw_m = R.w; raw_p = R.e; rm = M.w; rmm = M.ww; rp = M.e; rpp = M.ee; }
        else { raw_m = R.b; raw_p = R.t; rm = M.b; rmm = M.bb; rp = M.t; rpp = M.tt; }
    }
    const int rawnb = minus ? raw_m : raw_p;
    const bool solved = (fl[rawnb] & 1) != 0;
    const int fcell = minus ? rawnb : c;  // where this face's velocity and fluxes live
    const bool mus = P.muscl > 0 && fl[c] == FLUID;
    FaceGeo g;
    {
        const double *dd = dir == 0 ? P.dx : (dir == 1 ? P.dy : P.dz);
        int im2 = max(1, ii - 2), ip2 = min(nax, ii + 2);
        g.inmm = 1.0 / (dd[ii - 1] + dd[im2]);
        g.inm = 1.0 / (dd[ii] + dd[ii - 1]);
        g.inp = 1.0 / (dd[ii] + dd[ii + 1]);
        g.inpp = 1.0 / (dd[ii + 1] + dd[ip2]);
        g.incr_p = minus ? 0.5 * dd[ii - 1] : 0.5 * dd[ii];
        g.incr_m = minus ? -0.5 * dd[ii] : -0.5 * dd[ii + 1];
        g.r = (D == 2 && dir == 0) ? (minus ? P.rb[i - 1] : P.rb[i]) : 1.0;
        g.lim_on = minus ? (ii != 2 && fl[raw_m] == FLUID) : (ii != nax - 1 && fl[raw_p] == FLUID);
    }
    double *const gvel = dir == 0 ? F.ug : (dir == 1 ? F.vg : F.wg);
    double *const svel = dir == 0 ? F.us : (dir == 1 ? F.vs : F.ws);
    double vel[NC];
    vel[0] = gvel[fcell];
#pragma unroll
    for (int l = 2; l <= nph; ++l) vel[l - 1] = svel[(l - 2) * n + fcell];
    FaceK<NP, SH> K(kcols + threadIdx.x);
    if (solved) face_prepare<NP, RO>(P, F, c, minus ? rm : rp, rawnb, ii, dir, minus ? -1 : +1, dt, K);
    // mass-flux stencil of this face by phase (gas first): neighbour
    // values, or the cell's own current value where the slot is the cell
    const int rfar = minus ? rmm : rpp;
    const bool sm = rm == c, sp = rp == c, sfar = rfar == c;
    DensK<NC, SHD> Dk(dcols + threadIdx.x);
    Dk.cm(0) = ldro<RO>(F.rgp + rm); Dk.cp(0) = ldro<RO>(F.rgp + rp); Dk.cf(0) = mus ? ldro<RO>(F.rgp + rfar) : 0.0;
#pragma unroll
    for (int l = 2; l <= nph; ++l) {
        const double *D_ = F.rlk + (size_t)(l - 2) * n;
        Dk.cm(l - 1) = ldro<RO>(D_ + rm); Dk.cp(l - 1) = ldro<RO>(D_ + rp);
        Dk.cf(l - 1) = mus ? ldro<RO>(D_ + rfar) : 0.0;
    }
    // opt_inner_loop (iter.f:1255-1547) builds the density stencils once
    // and updates only their centre: a neighbour slot remapped to the
    // cell keeps the loop-entry value there
    Dk.o(0) = F.rgp[c];
#pragma unroll
    for (int l = 2; l <= nph; ++l) Dk.o(l - 1) = F.rlk[(size_t)(l - 2) * n + c];
    const bool stale = P.opt == 2;
    auto mflux = [&](int ph, double own) {
        const double slot = stale ? Dk.o(ph) : own;
        double dm = sm ? slot : Dk.cm(ph), dp = sp ? slot : Dk.cp(ph), df = sfar ? slot : Dk.cf(ph);
        return minus ? face_mflux(P, g, true, vel[ph], own, dm, df, dp, 0.0, mus)
                     : face_mflux(P, g, false, vel[ph], own, dm, 0.0, dp, df, mus);
    };
    // ---- cell state (identical in every lane) ------------------------------
    const double rx = D == 2 ? P.inr[i] : 1.0;
    const double idx_i = P.indx[i], idz_k = P.indz[k], idy_j = D == 3 ? P.indy[j] : 0.0;
    const double rgpn_c = F.rgpn[c];
    const CellFaces bf = cell_faces(P, c);  // faces, iter.f:259
    auto resid = [&](double fe, double fw, double fn, double fs, double ft, double fb, double rgpc) {
        double resx = (bf.e * fe - bf.w * fw) * idx_i * rx;
        double resz = (bf.t * ft - bf.b * fb) * idz_k;
        double resy = D == 3 ? (bf.n * fn - bf.s * fs) * idy_j : 0.0;
        return rgpc - rgpn_c + dt * bf.ivf * (resx + resy + resz);
    };
    double dg;  // calc_res of the stored state (raw W/S/B neighbours)
    if (D == 3) {
        int cw = at3(P, max(i - 1, 1), j, k), cs = at3(P, i, max(j - 1, 1), k), cb = at3(P, i, j, max(k - 1, 1));
        dg = resid(F.rgfe[c], F.rgfe[cw], F.rgfn[c], F.rgfn[cs], F.rgft[c], F.rgft[cb], F.rgp[c]);
    } else {
        int cw = at2(P, max(i - 1, 1), k), cb = at2(P, i, max(k - 1, 1));
        dg = resid(F.rgfe[c], F.rgfe[cw], 0.0, 0.0, F.rgft[c], F.rgft[cb], F.rgp[c]);
    }
    double dgorig = dg;
    const double conv = F.conv[c];
    double d3 = dg, p3 = F.p[c], abeta = F.abeta[c];
    // the mixture molecular weight of thermal_eosg (eosg.f:114-137), which
    // does not change within the loop: summed once, in thermal_eosg's order
    double mg = 0;
    for (int ig = 0; ig < P.ng; ++ig) mg = mg + GAS(F.xgc, c, ig) * P.gmw[P.gas_type[ig]];
    const double tgc = F.tg[c];
    const double rgas_tg = P.rgas * tgc;
    int kros = -1;
    PAdj s = {0, 0, 0, 0, 0, 0};
    double p = F.p[c], ep = F.ep[c], rog = F.rog[c], rgp = F.rgp[c];
    double rlk[NC], rlkn[NC], sink[NC];
#pragma unroll
    for (int is = 1; is <= ns; ++is) {
        rlk[is - 1] = F.rlk[(is - 1) * n + c];
        rlkn[is - 1] = F.rlkn[(is - 1) * n + c];
        sink[is - 1] = F.sink[(is - 1) * n + c];
    }
    double flux[NC];  // this lane's face mass flux by phase (gas first)
#pragma unroll
    for (int l = 0; l < NC; ++l) flux[l] = 0.0;
    // source lanes of the faces (3D: W S B E N T = 0..5; 2D: W B E T = 0..3)
    const int lW = tb + 0, lE = tb + (D == 3 ? 3 : 2), lB = tb + (D == 3 ? 2 : 1), lT = tb + (D == 3 ? 5 : 3);
    const int lS = tb + 1, lN = tb + 4;
    for (int loop = 1; loop <= P.inmax; ++loop) {
        if (loop > 1 || nit > 1) padjust(s, p, kros, d3, p3, P.omega, abeta);
        rog = p / rgas_tg * mg;  // thermal_eosg
        rgp = ep * rog;
        // this lane's face system (matrix.f:351-630)
        if (solved) face_assemble<NP>(P, K, minus ? -1 : +1, p, ep, rgp, rlk, vel);
        // particle mass fluxes and volume fractions (iter.f:778-994)
#pragma unroll
        for (int is = 1; is <= ns; ++is) flux[is] = mflux(is, rlk[is - 1]);
        double rls = 0;
#pragma unroll
        for (int is = 1; is <= ns; ++is) {
            double fW = __shfl_sync(tmask, flux[is], lW), fE = __shfl_sync(tmask, flux[is], lE);
            double fB = __shfl_sync(tmask, flux[is], lB), fT = __shfl_sync(tmask, flux[is], lT);
            double fS = 0, fN = 0;
            if (D == 3) { fS = __shfl_sync(tmask, flux[is], lS); fN = __shfl_sync(tmask, flux[is], lN); }
            double rlkx = (bf.e * fE - bf.w * fW) * idx_i * rx;
            double rlkz = (bf.t * fT - bf.b * fB) * idz_k;
            double rlky = D == 3 ? (bf.n * fN - bf.s * fS) * idy_j : 0.0;
            double t = rlkn[is - 1] - dt * bf.ivf * (rlkx + rlky + rlkz);
            t = t + dt * bf.ivf * sink[is - 1];
            double v = fmax(0.0, t);
            rlk[is - 1] = v;
            rls = rls + v * P.inrl[is];
        }
        ep = 1.0 - rls;
        if (rls > 1.0 && q == 0) atomicAdd(&F.counters[2], 1);
        rgp = ep * rog;
        // gas mass flux and continuity residual (iter.f:597-771)
        flux[0] = mflux(0, rgp);
        {
            double fW = __shfl_sync(tmask, flux[0], lW), fE = __shfl_sync(tmask, flux[0], lE);
            double fB = __shfl_sync(tmask, flux[0], lB), fT = __shfl_sync(tmask, flux[0], lT);
            double fS = 0, fN = 0;
            if (D == 3) { fS = __shfl_sync(tmask, flux[0], lS); fN = __shfl_sync(tmask, flux[0], lN); }
            dg = resid(fE, fW, fN, fS, fT, fB, rgp);
        }
        if (fabs(dg) > conv || fabs(dg) >= fabs(dgorig)) {
            if (nit == 1 && loop == 1) dgorig = dg;
            d3 = dg;
        } else if (fabs(dg) <= conv) {
            break;
        }
    }
    // ---- final values -----------------------------------------------------
    {
        // face mass fluxes (every face, as calc_*_mass_flux writes them)
        double *gfa = dir == 0 ? F.rgfe : (dir == 1 ? F.rgfn : F.rgft);
        double *sfa = dir == 0 ? F.rsfe : (dir == 1 ? F.rsfn : F.rsft);
        gfa[fcell] = flux[0];
#pragma unroll
        for (int is = 1; is <= ns; ++is) sfa[(size_t)(is - 1) * n + fcell] = flux[is];
        if (solved) {
            gvel[fcell] = vel[0];
#pragma unroll
            for (int l = 2; l <= nph; ++l) svel[(l - 2) * n + fcell] = vel[l - 1];
        }
        mark_dirty(dirty, rawnb);
    }
    if (q == 0) {
        F.p[c] = p; F.rog[c] = rog; F.rgp[c] = rgp; F.ep[c] = ep;
#pragma unroll
        for (int is = 1; is <= ns; ++is) F.rlk[(is - 1) * n + c] = rlk[is - 1];
        F.abeta[c] = abeta;
        mark_dirty(dirty, c);
    }
}

// the inner loop of the worklist's nwork cells (outer sweep nit, 1-based)
// by the warps warp, warp + nwarps, ... of the launch; RO as in ldro
template <int NP, int D, bool RO>
__device__ __forceinline__ void inner_team_run(const Prm &P, const Fld &F, double dt, int nit, const int *list,
                                               int nwork, unsigned *dirty, int warp, int nwarps) {
    constexpr int T = D == 3 ? 6 : 4;    // lanes per cell
    constexpr int TPW = 32 / T;          // teams per warp (3D: 5, lanes 30 and 31 idle)
    const int lane = threadIdx.x & 31, tw = lane / T;
    if (tw >= TPW) return;  // idle lanes take no part in any team
    const int q = lane - tw * T, tb = tw * T;
    const unsigned tmask = ((1u << T) - 1u) << tb;
    extern __shared__ __align__(16) double inner_smem[];
    double *const kcols = inner_smem;                              // [FaceK rows][KS]
    double *const dcols = inner_smem + inner_face_rows<NP>() * KS;  // [4 NC][KS]
    for (int w = warp * TPW + tw; w < nwork; w += nwarps * TPW)
        inner_team_cell<NP, D, RO>(P, F, dt, nit, list[w], dirty, q, tb, tmask, kcols, dcols);
}

template <int NP, int D>
__global__ void __launch_bounds__(128, PDAC_INNER_MINB(NP)) k_inner_team(Prm P, Fld F, double dt, const int *nitp, const int *list,
                                                                     const int *count, unsigned *dirty) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    inner_team_run<NP, D, true>(P, F, dt, *nitp, list, *count, dirty, warp, nwarps);
}

// Residual test of one colour phase (iter.f:241-319) in two launches.
// The active set is one bit per cell: the test of a cell reads only its own
// p/rog/rgp and the mass fluxes of its faces, which change only when the
// cell or a face neighbour runs the inner loop; such a run sets the bits of
// those cells (mark_dirty).  A converged test rewrites the cell's volume
// fractions (calc_eps, from the same fluxes) and rgp = ep rog: if that
// changes rgp, the next test computes a different residual, so the cell
// keeps its bit; otherwise a clean cell would recompute exactly the values
// it holds, and it is not tested.  k_resid_collect turns the set bits of
// one colour's fluid cells into a candidate list (clearing them, and the
// bits of non-fluid cells, which are never tested); k_resid_test tests each
// candidate: a converged cell updates its volume fractions and rgp, an
// unconverged one goes to the worklist of k_inner_team.
// candidates of one colour: the block's threads take consecutive words of
// the bitmask, block-uniform rounds over the grid (one round when the grid
// covers the words)
template <int TPBK>
__device__ __forceinline__ void collect_phase(const Prm &P, int colour, unsigned *dirty, int *cand, int *ncand) {
    const unsigned nwords = ((unsigned)P.ncell + 31u) / 32u;
    for (unsigned base = blockIdx.x * (unsigned)TPBK; base < nwords; base += gridDim.x * (unsigned)TPBK) {
    unsigned t = base + threadIdx.x;
    int mine[32], nmine = 0;
    if (t < nwords) {
        unsigned w = dirty[t], keep = w;
        while (w) {
            int b = __ffs(w) - 1;
            w &= w - 1u;
            int c = (int)(32u * t) + b;
            if (c >= P.ncell) break;
            if (!(P.flag[c] & 1)) { keep &= ~(1u << b); continue; }
            int i = c % P.nx + 1, r = c / P.nx, j = r % P.ny + 1, k = r / P.ny + 1;
            if ((i + j + k) % 3 != colour) continue;
            keep &= ~(1u << b);
            mine[nmine++] = c;
        }
        if (keep != dirty[t]) dirty[t] = keep;
    }
    block_append_n<TPBK, 32>(cand, ncand, mine, nmine, nullptr, 0);
    }
}

__global__ void __launch_bounds__(TPB_RESID) k_resid_collect(Prm P, int colour, unsigned *dirty, int *cand,
                                                             int *ncand) {
    collect_phase<TPB_RESID>(P, colour, dirty, cand, ncand);
}

// the residual test of cell c (iter.f:241-319): a converged cell updates its
// volume fractions and rgp (keeping its active-set bit if rgp changed);
// returns true for an unconverged cell, which goes to the inner loop
template <int NP, int D>
__device__ __forceinline__ bool test_cell(const Prm &P, const Fld &F, double dt, int c, unsigned *dirty) {
    double dg;
    if (D == 3) {
        int i, j, k;
        ijk_of(P, c, i, j, k);
        Raw3 R;
        raw3(P, i, j, k, R);
        dg = calc_res_3d(P, F, R, i, j, k, dt);
        if (fabs(dg) <= F.conv[c]) calc_eps_3d<NP>(P, F, R, i, j, k, dt);
    } else {
        int i = c % P.nx + 1, k = c / P.nx + 1;
        Raw2 R;
        raw2(P, i, k, R);
        dg = calc_res_2d(P, F, R, i, k, dt);
        if (fabs(dg) <= F.conv[c]) calc_eps_2d(P, F, R, i, k, dt);
    }
    if (fabs(dg) <= F.conv[c]) {
        const double old = F.rgp[c];
        F.rgp[c] = F.ep[c] * F.rog[c];
        if (__double_as_longlong(F.rgp[c]) != __double_as_longlong(old)) mark_dirty(dirty, c);
        return false;
    }
    return true;
}

// the residual test of the len candidates, block-uniform rounds
template <int TPBK, int NP, int D>
__device__ __forceinline__ void test_phase(const Prm &P, const Fld &F, double dt, const int *cand, int len, int *work,
                                           int *count, unsigned *dirty) {
    for (int base = blockIdx.x * TPBK; base < len; base += gridDim.x * TPBK) {
        int idx = base + threadIdx.x, c = -1, nmine = 0;
        if (idx < len) {
            c = cand[idx];
            nmine = test_cell<NP, D>(P, F, dt, c, dirty) ? 1 : 0;
        }
        block_append_n<TPBK, 1>(work, count, &c, nmine, count + 3, idx < len ? 1 : 0);
    }
}

template <int NP, int D>
__global__ void __launch_bounds__(TPB_RESID) k_resid_test(Prm P, Fld F, double dt, const int *cand, const int *ncand,
                                                          int *work, int *count, unsigned *dirty) {
    test_phase<TPB_RESID, NP, D>(P, F, dt, cand, *ncand, work, count, dirty);
}

// One colour phase of the cooperative sweep loop in one pass: collect, test
// and inner loop fused, with one grid barrier after it instead of three.
// Each warp takes one word of the active set (32 consecutive cells) at a time:
// lane b tests the cell of bit b when that bit is set and the cell is a
// fluid cell of the colour, the unconverged cells (at most 11 of the 32 are
// of one colour) go to a warp-local list in shared memory, and the warp's
// teams run their inner loops.  Cells of one colour share no stencil data,
// so testing and iterating them in this order gives the bits of the
// three-launch form.  The colour's set bits of a word are cleared
// atomically before its cells are tested: other warps set bits of the
// neighbouring cells meanwhile.  Appends the unconverged cells to the
// colour's worklist (work, wcount[col] long; the cells the last sweep left
// unconverged, as pdac_gpu_unconverged_cells reports them) and adds the
// tested ones to wcount[3 + col].  RO as in ldro.
template <int NP, int D, bool RO>
__device__ __forceinline__ void fused_phase(const Prm &P, const Fld &F, double dt, int nit, int colour,
                                            unsigned *dirty, int *wcount, int *work, unsigned warp, unsigned nwarps) {
    const int lane = threadIdx.x & 31;
    __shared__ int wlist[KS / 32][32];
    int *const mylist = wlist[threadIdx.x >> 5];
    const unsigned nwords = ((unsigned)P.ncell + 31u) / 32u;
    int ntest_sum = 0;
    for (unsigned t = warp; t < nwords; t += nwarps) {  // uniform across the warp
        const unsigned w = __ldcg(dirty + t);
        const int c = (int)(32u * t) + lane;
        bool cand = false, clear = false;
        if (((w >> lane) & 1u) && c < P.ncell) {
            if (!(P.flag[c] & 1)) {
                clear = true;  // a non-fluid cell is never tested
            } else {
                int i = c % P.nx + 1, r = c / P.nx, j = r % P.ny + 1, k = r / P.ny + 1;
                cand = (i + j + k) % 3 == colour;
                clear = cand;
            }
        }
        const unsigned cm = __ballot_sync(0xffffffffu, clear);
        if (lane == 0 && cm) atomicAnd(dirty + t, ~cm);
        __syncwarp();
        const bool unconv = cand && test_cell<NP, D>(P, F, dt, c, dirty);
        const unsigned um = __ballot_sync(0xffffffffu, unconv);
        if (unconv) mylist[__popc(um & ((1u << lane) - 1u))] = c;
        ntest_sum += __popc(__ballot_sync(0xffffffffu, cand));
        __syncwarp();
        const int nwork = __popc(um);
        if (nwork) {
            int base = 0;
            if (lane == 0) base = atomicAdd(wcount + colour, nwork);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (unconv) work[base + __popc(um & ((1u << lane) - 1u))] = c;
            inner_team_run<NP, D, RO>(P, F, dt, nit, mylist, nwork, dirty, 0, 1);
        }
        __syncwarp();  // the list is read before the next word overwrites it
    }
    if (lane == 0 && ntest_sum) atomicAdd(wcount + 3 + colour, ntest_sum);
}

// The whole outer sweep loop of iter (iter.f:204-410) in one cooperative
// launch, for small domains: the colour phases (fused_phase: collect, test
// and inner loop in one pass) follow each other across grid-wide barriers
// instead of launches.
// Every thread of the grid takes every barrier the same number of times:
// the loop ends on counters that all threads read after the same barrier.
struct SweepWork {
    int *wcount;      // [col] worklist length, [3 + col] cells tested, [6 + col] candidates
    int *cand, *work; // candidate list of one colour phase; worklists, colour col at work + col * wstride
    unsigned *dirty;  // active set, one bit per cell
    int *nit;         // the sweep count on return, as the graph's k_sweep_check leaves it
    long wstride;     // ints per colour's worklist
};

template <int NP, int D>
__global__ void __launch_bounds__(128, PDAC_INNER_MINB(NP)) k_iter_coop(Prm P, Fld F, double dt, SweepWork W, int maxout) {
    namespace cg = cooperative_groups;
    cg::grid_group g = cg::this_grid();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    int nit = 1;
    for (;;) {
        if (blockIdx.x == 0 && threadIdx.x < 9) W.wcount[threadIdx.x] = 0;
        g.sync();
        for (int col = 0; col < 3; ++col) {
            fused_phase<NP, D, false>(P, F, dt, nit, col, W.dirty, W.wcount, W.work + col * W.wstride, warp, nwarps);
            g.sync();
        }
        const long unconverged = (long)__ldcg(W.wcount) + __ldcg(W.wcount + 1) + __ldcg(W.wcount + 2);
        if (unconverged == 0) break;
        if (nit >= maxout) {
            nit = maxout + 1;
            break;
        }
        ++nit;
        g.sync();  // every thread has read the counters before they are cleared
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *W.nit = nit;
}

// End of one outer sweep on the device (iter.f:388-410): with no unconverged
// cell left, or after maxout sweeps, the sweep loop stops; otherwise the
// sweep number advances.  *nit ends as the host loop's nit (maxout + 1 when
// the sweeps did not converge).
__global__ void k_sweep_check(const int *wcount, int *nit, int maxout, cudaGraphConditionalHandle loop) {
    long unconverged = (long)wcount[0] + wcount[1] + wcount[2];
    if (unconverged == 0) { cudaGraphSetConditional(loop, 0); return; }
    if (*nit >= maxout) { *nit = maxout + 1; cudaGraphSetConditional(loop, 0); return; }
    *nit += 1;
    cudaGraphSetConditional(loop, 1);
}

}  // namespace pdac

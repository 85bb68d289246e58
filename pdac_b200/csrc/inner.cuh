// inner.cuh -- inner_loop of the corrector (iter.f:480-580) on a team of
// lanes per cell.
//
// A team of T lanes (8 in 3D, 4 in 2D) owns one unconverged cell of the
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
#include "kernels3d.cuh"

namespace pdac {

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

template <int NP, int D>
__global__ void __launch_bounds__(128) k_inner_team(Prm P, Fld F, double dt, int nit, const int *list, const int *count,
                                                    unsigned char *dirty) {
    constexpr int T = D == 3 ? 8 : 4;    // lanes per cell
    constexpr int NF = D == 3 ? 6 : 4;   // faces per cell
    constexpr int NC = Sys<NP>::M - 1;   // phase capacity
    const int nph = nphases<NP>(P), ns = nph - 1;
    const size_t n = P.ncell;
    const int lane = threadIdx.x & 31, q = lane & (T - 1), tb = lane & ~(T - 1);
    const unsigned tmask = (T == 32 ? 0xffffffffu : ((1u << T) - 1u)) << tb;
    const int nwork = *count;
    const int team0 = (blockIdx.x * blockDim.x + threadIdx.x) / T, nteams = gridDim.x * blockDim.x / T;
    for (int w = team0; w < nwork; w += nteams) {
        const int c = list[w];
        int i, j, k;
        if (D == 3) ijk_of(P, c, i, j, k);
        else { i = c % P.nx + 1; j = 1; k = c / P.nx + 1; }
        const int *fl = P.flag;
        // ---- this lane's face ------------------------------------------------
        // axis and side; raw / remapped neighbours on both sides along the
        // axis (first and second); cell holding the face velocity
        int dir = 0, ii = i, nax = P.nx;
        bool minus = true, own_face = q < NF;
        int raw_m = c, raw_p = c, rm = c, rmm = c, rp = c, rpp = c, rawnb = c;
        if (own_face) {
            int a = D == 3 ? q % 3 : q % 2;  // axis slot
            minus = D == 3 ? q < 3 : q < 2;
            dir = D == 3 ? a : (a == 0 ? 0 : 2);
            ii = dir == 0 ? i : (dir == 1 ? j : k);
            nax = dir == 0 ? P.nx : (dir == 1 ? P.ny : P.nz);
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
            rawnb = minus ? raw_m : raw_p;
        }
        const bool solved = own_face && (fl[rawnb] & 1);
        const int fcell = minus ? rawnb : c;  // where this face's velocity and fluxes live
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
            g.lim_on = own_face && (minus ? (ii != 2 && fl[raw_m] == FLUID) : (ii != nax - 1 && fl[raw_p] == FLUID));
        }
        double *const gvel = dir == 0 ? F.ug : (dir == 1 ? F.vg : F.wg);
        double *const svel = dir == 0 ? F.us : (dir == 1 ? F.vs : F.ws);
        double vel[NC];
        if (own_face) {
            vel[0] = gvel[fcell];
#pragma unroll
            for (int l = 2; l <= nph; ++l) vel[l - 1] = svel[(l - 2) * n + fcell];
        }
        // ---- cell state (identical in every lane) ------------------------------
        const double rx = D == 2 ? P.inr[i] : 1.0;
        auto resid = [&](double fe, double fw, double fn, double fs, double ft, double fb, double rgpc) {
            double resx = (1.0 * fe - 1.0 * fw) * P.indx[i] * rx;
            double resz = (1.0 * ft - 1.0 * fb) * P.indz[k];
            double resy = D == 3 ? (1.0 * fn - 1.0 * fs) * P.indy[j] : 0.0;
            return rgpc - F.rgpn[c] + dt * 1.0 * (resx + resy + resz);
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
        double xg[PDAC_MAXG];
        for (int ig = 0; ig < P.ng; ++ig) xg[ig] = GAS(F.xgc, c, ig);
        const double tgc = F.tg[c];
        int kros = -1;
        PAdj s = {0, 0, 0, 0, 0, 0};
        double p = F.p[c], ep = F.ep[c], rog = F.rog[c], rgp = F.rgp[c];
        double rlk[NC];
#pragma unroll
        for (int is = 1; is <= ns; ++is) rlk[is - 1] = F.rlk[(is - 1) * n + c];
        double flux[NC];  // this lane's face mass flux by phase (gas first)
#pragma unroll
        for (int l = 0; l < NC; ++l) flux[l] = 0.0;
        const bool mus = P.muscl > 0 && fl[c] == FLUID;
        // source lanes of the faces (3D: W S B E N T = 0..5; 2D: W B E T = 0..3)
        const int lW = tb + 0, lE = tb + (D == 3 ? 3 : 2), lB = tb + (D == 3 ? 2 : 1), lT = tb + (D == 3 ? 5 : 3);
        const int lS = tb + 1, lN = tb + 4;
        auto stencil = [&](const double *a, double own, double &dm, double &dmm, double &dp, double &dpp) {
            dm = slot(a, rm, c, own);
            dp = slot(a, rp, c, own);
            if (mus) {
                if (minus) dmm = slot(a, rmm, c, own);
                else dpp = slot(a, rpp, c, own);
            }
        };
        for (int loop = 1; loop <= P.inmax; ++loop) {
            if (loop > 1 || nit > 1) padjust(s, p, kros, d3, p3, P.omega, abeta);
            rog = thermal_eosg(P, tgc, p, xg);
            rgp = ep * rog;
            // this lane's face system (matrix.f:351-630)
            if (solved) face_system<NP>(P, F, c, minus ? rm : rp, rawnb, ii, dir, minus ? -1 : +1, dt, p, ep, rgp, rlk, vel);
            // particle mass fluxes and volume fractions (iter.f:778-994)
            double rls = 0;
#pragma unroll
            for (int is = 1; is <= ns; ++is) {
                double own = rlk[is - 1];
                if (own_face) {
                    double dm = 0, dmm = 0, dp = 0, dpp = 0;
                    stencil(F.rlk + (size_t)(is - 1) * n, own, dm, dmm, dp, dpp);
                    flux[is] = face_mflux(P, g, minus, vel[is], own, dm, dmm, dp, dpp, mus);
                }
                double fW = __shfl_sync(tmask, flux[is], lW), fE = __shfl_sync(tmask, flux[is], lE);
                double fB = __shfl_sync(tmask, flux[is], lB), fT = __shfl_sync(tmask, flux[is], lT);
                double fS = 0, fN = 0;
                if (D == 3) { fS = __shfl_sync(tmask, flux[is], lS); fN = __shfl_sync(tmask, flux[is], lN); }
                size_t off = (size_t)(is - 1) * n;
                double rlkx = (1.0 * fE - 1.0 * fW) * P.indx[i] * rx;
                double rlkz = (1.0 * fT - 1.0 * fB) * P.indz[k];
                double rlky = D == 3 ? (1.0 * fN - 1.0 * fS) * P.indy[j] : 0.0;
                double t = F.rlkn[off + c] - dt * 1.0 * (rlkx + rlky + rlkz);
                t = t + dt * 1.0 * F.sink[off + c];
                double v = fmax(0.0, t);
                rlk[is - 1] = v;
                rls = rls + v * P.inrl[is];
            }
            ep = 1.0 - rls;
            if (rls > 1.0 && q == 0) atomicAdd(&F.counters[2], 1);
            rgp = ep * rog;
            // gas mass flux and continuity residual (iter.f:597-771)
            if (own_face) {
                double dm = 0, dmm = 0, dp = 0, dpp = 0;
                stencil(F.rgp, rgp, dm, dmm, dp, dpp);
                flux[0] = face_mflux(P, g, minus, vel[0], rgp, dm, dmm, dp, dpp, mus);
            }
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
        if (own_face) {
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
            dirty[rawnb] = 1;
        }
        if (q == 0) {
            F.p[c] = p; F.rog[c] = rog; F.rgp[c] = rgp; F.ep[c] = ep;
#pragma unroll
            for (int is = 1; is <= ns; ++is) F.rlk[(is - 1) * n + c] = rlk[is - 1];
            F.abeta[c] = abeta;
            dirty[c] = 1;
        }
    }
}

}  // namespace pdac

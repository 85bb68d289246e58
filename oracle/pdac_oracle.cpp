// pdac_oracle.cpp -- CPU FP64 restatement of PDAC's per-time-step hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the
// timed CPU baseline for the B200 engine; it is never linked into, loaded by
// or called from the product path (pdac_b200/).  Only tests/, the smoke()
// check of __graft_entry__.py and bench.py's cpu_baseline / reference arm use
// it, as the checker.
//
// It follows the reference Fortran (tomaso-espostiongaro/pdac) routine by
// routine, serially, with the reference's data structures: flat 1-D cell
// arrays (i fastest), explicit raw-neighbour (myijk) and boundary-remapped
// neighbour (myinds) tables built with the rules of ghost.f, and the same
// lexicographic cell loops.  Each routine cites the reference lines it
// restates.  Fortran REAL(4) literals are written as (double)x.f, which is
// what the Fortran compiler feeds to the REAL(8) arithmetic.
//
// Two sweep orders exist for iter's corrector (iter.f:241-319):
//   order 0 = "colored": cells of colour (i+j+k) mod 3 == c for c = 0,1,2,
//             which is the order the GPU engine executes;
//   order 1 = "lexicographic": the reference's own in-place order.
// Everything else is order independent and identical in both.
//
// Parity status: the reference ships no tests and no golden outputs and no
// Fortran compiler exists on this image, so this restatement is pinned by
// known-answer checks derived from the reference source (limiters, padjust,
// Gauss-Jordan, invdm, heat capacities, hydrostatic profile) and by
// conservation properties; see the tests.  "Parity unpinned" by reference
// runs.
//
// Build: g++ -O2 -fno-fast-math -ffp-contract=off -shared -fPIC (oracle/Makefile)

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "../include/pdac_gpu.h"
// exp and pow of the per-cell physics: the engine's own routines (the same
// bits on the host and the device; the C library's may differ from CUDA's in
// the last bit)
#include "../pdac_b200/csrc/fpmath.h"

// The 3D passes run their cell loops on several host threads: every such
// loop writes each value from exactly one cell -- the cell that writes it
// last in the reference's serial cell order -- and reads only values that no
// iteration of the loop writes, so the results are the same bits on any
// number of threads.  The corrector runs the cells of one colour in parallel
// (they share no stencil); the lexicographic order stays serial.  Threads:
// PDAC_ORACLE_THREADS, else every hardware thread; pdac_oracle_set_threads.
#include <atomic>
#include <thread>

static int g_oracle_threads = 0;  // 0: not yet chosen

static int oracle_threads() {
    if (g_oracle_threads <= 0) {
        const char *e = std::getenv("PDAC_ORACLE_THREADS");
        int n = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
        g_oracle_threads = n > 0 ? n : 1;
    }
    return g_oracle_threads;
}

// f(lo, hi) over [0, n) in one contiguous range per thread
template <class Fn>
static void par_range(int n, Fn f) {
    const int T = oracle_threads();
    if (T <= 1 || n < 4096) { f(0, n); return; }
    const int chunk = (n + T - 1) / T;
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) {
        const int lo = t * chunk, hi = std::min(n, lo + chunk);
        if (lo < hi) th.emplace_back(f, lo, hi);
    }
    f(0, std::min(n, chunk));
    for (auto &x : th) x.join();
}

// f(lo, hi) over [lo0, hi0) in chunks of 256 taken from a shared counter
// (for loops whose iterations differ in cost)
template <class Fn>
static void par_dynamic(int lo0, int hi0, Fn f) {
    const int T = oracle_threads();
    if (T <= 1 || hi0 - lo0 < 512) { f(lo0, hi0); return; }
    std::atomic<int> next(lo0);
    auto work = [&]() {
        for (;;) {
            const int lo = next.fetch_add(256);
            if (lo >= hi0) return;
            f(lo, std::min(hi0, lo + 256));
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
}

namespace {

using std::vector;

// flag constants, grid.f:45-58
constexpr int FLUID = 1, SLIP = 2, NOSLIP = 4, BL_CELL = 5, FREE_IO = 8, INLET = 16,
              ZERO_GRAD = 32, VENT = 64, DOME = 129, IMMB = 257, FILLED1 = 512, FILLED2 = 1024;

// neighbour slots (di, dj, dk)
enum Nb {
    C = 0, E, W, N, S, T, B,          // first neighbours
    EE, WW, NN, SS, TT, BB,           // second along axes
    ET, WT, EB, WB, EN, ES, WN, WS, NT, ST, NB_, SB,  // edge diagonals
    EET, ETT, EEE, NNN, TTT, EEN, ENN, NNT, NTT,      // used by nb() stencils
    NSLOT
};
const int OFF[NSLOT][3] = {
    {0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1},
    {2,0,0},{-2,0,0},{0,2,0},{0,-2,0},{0,0,2},{0,0,-2},
    {1,0,1},{-1,0,1},{1,0,-1},{-1,0,-1},{1,1,0},{1,-1,0},{-1,1,0},{-1,-1,0},{0,1,1},{0,-1,1},{0,1,-1},{0,-1,-1},
    {2,0,1},{1,0,2},{3,0,0},{0,3,0},{0,0,3},{2,1,0},{1,2,0},{0,2,1},{0,1,2}};

// TYPE(stencil) of subscr.f:63-357 (members used on this path)
struct Sten {
    double c = 0, e = 0, w = 0, n = 0, s = 0, t = 0, b = 0;
    double ee = 0, ww = 0, nn = 0, ss = 0, tt = 0, bb = 0;
    double et = 0, wt = 0, eb = 0, en = 0, es = 0, wn = 0, nt = 0, st = 0, nb = 0;
    double eet = 0, ett = 0, eee = 0, nnn = 0, ttt = 0, een = 0, enn = 0, nnt = 0, ntt = 0;
};

// fields of the SSP-RK3 explicit path (explicit_solver.f:15-83)
struct RK3State {
    int neq = 0;
    std::vector<double> rgpS, rlkS, ugS, usS, vgS, vsS, wgS, wsS, tgS, tsS, siegS, siesS, pS, epS, rhogS;
    std::vector<double> ugN, usN, vgN, vsN, wgN, wsN;
    std::vector<double> hv, kpgv;            // (ncell, ns) column-major
    std::vector<double> rhs3, k1, k2, k3;    // row per cell: [c * neq + eq]
    std::vector<double> hf3;                 // 3D diffusive heat fluxes, [phase][face e,n,t]
};

struct Oracle {
    pdac_cfg cfg{};
    RK3State rk;
    bool d3 = false;
    int nx = 0, ny = 1, nz = 0, ncell = 0, ns = 0, ng = 0, nph = 0, nap = 0;
    int order = 0;                 // 0 colored, 1 lexicographic
    std::string err;

    // metric, 1-based with padding on both ends (index 0 .. n+3)
    vector<double> dx, dy, dz, indx, indy, indz, r, rb, inr, inrb;
    vector<int> flag;
    vector<double> p_atm, t_atm;   // 1-based
    vector<int> raw, rem;          // [slot * ncell + ijk]

    // gas constants (setup.f:551-616), reference gas index 1..7
    double gmw[8]{}, mmugs[8]{}, mmugek[8]{};
    double rgas = 8.31432, gammaair = 1.4, tzero = 0.0, hzerog = 0.0, hzeros = 0.0;
    int gas_type[PDAC_MAX_NGAS]{};
    // particle constants (particles.f:35-79, input.f:1097-1105), 1-based
    double dk[PDAC_MAX_NSOLID + 1]{}, rl[PDAC_MAX_NSOLID + 1]{}, inrl[PDAC_MAX_NSOLID + 1]{},
        phis[PDAC_MAX_NSOLID + 1]{}, cmus[PDAC_MAX_NSOLID + 1]{}, cps[PDAC_MAX_NSOLID + 1]{},
        kap[PDAC_MAX_NSOLID + 1]{}, plim[PDAC_MAX_NSOLID + 1]{}, phi[PDAC_MAX_NSOLID + 1]{};
    double philim[PDAC_MAX_NSOLID + 1][PDAC_MAX_NSOLID + 1]{}, epsl[PDAC_MAX_NSOLID + 1][PDAC_MAX_NSOLID + 1]{},
        epsu[PDAC_MAX_NSOLID + 1][PDAC_MAX_NSOLID + 1]{}, dkf[PDAC_MAX_NSOLID + 1][PDAC_MAX_NSOLID + 1]{};

    // prognostic state
    vector<double> p, ep, rog, rgp, tg, sieg, cg, ug, vg, wg;
    vector<double> rlk, ts, sies, us, vs, ws;   // (ncell, ns) column-major
    vector<double> ygc, xgc;                    // (ncell, ng)
    // n-level and derived
    vector<double> pn, epn, rgpn, siegn, rlkn, siesn, rgpgcn, mug, kapg;
    vector<double> rugn, rvgn, rwgn, rusn, rvsn, rwsn;
    vector<double> rug, rvg, rwg, rus, rvs, rws, appu, appv, appw, rhg, rhs;
    vector<double> gvisx, gvisy, gvisz, pvisx, pvisy, pvisz;
    vector<double> ugfe, ugft, wgfe, wgft, usfe, usft, wsfe, wsft;
    vector<double> rgfe, rgfn, rgft, rsfe, rsfn, rsft, conv, abeta;
    vector<double> egfe, egft, esfe, esft, hgfe, hgft, hsfe, hsft, yfe, yft;
    vector<double> sink;
    // the ground sink (sink.f): cell-centre coordinates x(i), y(j) of
    // grid.f:286-298 (1-based), the mass taken out per ground column and
    // solid (massl, ntr x ns with ntr = nx in 2D, nx ny in 3D) and the
    // values a restart adds back at each column's first update (mass_loss)
    vector<double> xc, yc, massl, mass_loss;
    vector<double> rhom, um, vm, wm, tm, yd;  // mixture fields (mixture.f), yd (ncell, ng + ns)
    vector<double> mf3, ef3, yfn;   // 3D momentum / enthalpy face fluxes, species y-fluxes
    vector<double> smag, mugt, kapgt, must;  // sub-grid model (turbo.f:10-14)
    vector<double> scoeff;                   // dynamic coefficient cdyn of the last sgsg (modturbo = 2)
    vector<double> dgres;   // |dg|/conv at the last corrector visit (diagnostic)
    vector<int> unconv;     // cells of the last outer sweep that ran the inner loop (iter.f:428-447)
    vector<double> app0;    // 3D tilde on several threads: the interphase terms of the previous call
    vector<double> vent_fact, vent_fact0;
    int last_nit = 0, eos_fail = 0, ierr = 0;

    // immersed boundaries (immb.f, interp.f:321-919, ghost.f:2888-3345):
    // the cut-cell face factors and forcing-point tables of pdac_cfg, the
    // forcing-point velocities of the last boundary pass (nfp x nph per
    // axis, fptx/y/z(:)%vel) and the filled_cell_2 toggles (fc2)
    int immb = 0;
    vector<int> ib_faces;
    vector<double> ib_ivf;
    vector<int> ib_num[3], ib_fp[3];
    vector<double> ib_nsl[3], ib_vel[3];
    vector<char> fc2;
    vector<double> xm, xbm, ym, ybm, zm, zbm;  // mesh coordinates, 1-based

    // ---- indexing ------------------------------------------------------
    int idx(int i, int j, int k) const {  // 1-based -> flat 0-based
        return (i - 1) + nx * ((j - 1) + ny * (k - 1));
    }
    void ijk_of(int c, int &i, int &j, int &k) const {
        i = c % nx + 1;
        j = (c / nx) % ny + 1;
        k = c / (nx * ny) + 1;
    }
    int nbraw(int slot, int c) const { return raw[(size_t)slot * ncell + c]; }
    int nbrem(int slot, int c) const { return rem[(size_t)slot * ncell + c]; }
    bool fluidbit(int c) const { return (flag[c] & 1) != 0; }
    double &S(vector<double> &a, int c, int is) { return a[(size_t)(is - 1) * ncell + c]; }  // (c, is) 1-based is
    double S(const vector<double> &a, int c, int is) const { return a[(size_t)(is - 1) * ncell + c]; }
};

// ---------------------------------------------------------------------------
// neighbour tables: ghost.f:486-680 (myijk, clamped offsets) and
// ghost.f:866-1415 / 1417-2476 (myinds remap for walls)
// ---------------------------------------------------------------------------
bool is_wall(int f) { return f == SLIP || f == NOSLIP; }
bool is_wallf(int f) { return f == SLIP || f == NOSLIP || f == FILLED1; }

#include "pdac_oracle_les.inc"

void build_tables(Oracle &o) {
    o.raw.assign((size_t)NSLOT * o.ncell, 0);
    o.rem.assign((size_t)NSLOT * o.ncell, 0);
    auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
    for (int c = 0; c < o.ncell; ++c) {
        int i, j, k;
        o.ijk_of(c, i, j, k);
        for (int s = 0; s < NSLOT; ++s) {
            int ii = clampi(i + OFF[s][0], 1, o.nx);
            int jj = o.d3 ? clampi(j + OFF[s][1], 1, o.ny) : 1;
            int kk = clampi(k + OFF[s][2], 1, o.nz);
            if (!o.d3 && OFF[s][1] != 0) { ii = i; kk = k; }
            o.raw[(size_t)s * o.ncell + c] = o.idx(ii, jj, kk);
            o.rem[(size_t)s * o.ncell + c] = -1;  // undefined outside the interior
        }
        bool interior = i >= 2 && i <= o.nx - 1 && k >= 2 && k <= o.nz - 1 && (!o.d3 || (j >= 2 && j <= o.ny - 1));
        if (!interior || o.d3) continue;
        auto R = [&](int s) { return o.raw[(size_t)s * o.ncell + c]; };
        auto F = [&](int s) { return o.flag[R(s)]; };
        auto setr = [&](int s, int v) { o.rem[(size_t)s * o.ncell + c] = v; };
        setr(C, c);
        // first neighbours (ghost.f:963-989): walls and filled cells -> self
        for (int s : {E, W, N, S, T, B}) {
            if (!o.d3 && (s == N || s == S)) continue;
            setr(s, is_wallf(F(s)) ? c : R(s));
        }
        // edge diagonals (ghost.f:990-1056): symmetric rule on the two
        // axis cells A, B adjacent to the diagonal D
        auto diag = [&](int sd, int sa, int sb) {
            int v = R(sd);
            if (is_wall(F(sd))) {
                bool wa = is_wall(F(sa)), wb = is_wall(F(sb));
                if (wa && wb) v = c;
                else if (wa) v = R(sb);
                else if (wb) v = R(sa);
                else v = c;
            }
            setr(sd, v);
        };
        diag(WT, W, T);
        diag(EB, E, B);
        diag(ET, E, T);
        diag(WB, W, B);
        // second neighbours (ghost.f:1058-1092)
        int ijke = o.nbrem(E, c), ijkw = o.nbrem(W, c), ijkt = o.nbrem(T, c), ijkb = o.nbrem(B, c);
        setr(EE, is_wallf(F(EE)) ? R(E) : R(EE));
        if (i == o.nx - 1) setr(EE, ijke);
        setr(TT, is_wallf(F(TT)) ? R(T) : R(TT));
        if (k == o.nz - 1) setr(TT, ijkt);
        setr(WW, is_wallf(F(WW)) ? R(W) : R(WW));
        if (i == 2) setr(WW, ijkw);
        setr(BB, is_wallf(F(BB)) ? R(B) : R(BB));
        if (k == 2) setr(BB, ijkb);
        // (2,1) and (1,2) diagonals (ghost.f:1094-1152): same rule relative
        // to the base cell one step inward, triggered by wall-or-filled
        auto diag2 = [&](int sd, int sa, int sb, int sbase) {
            int v = R(sd);
            if (is_wallf(F(sd))) {
                bool wa = is_wall(F(sa)), wb = is_wall(F(sb));
                if (wa && wb) v = R(sbase);
                else if (wa) v = R(sb);
                else if (wb) v = R(sa);
                else v = R(sbase);
            }
            setr(sd, v);
        };
        // ijkeet: D=(2,0,1), checks ipjkp (1,0,1) then ippjk (2,0,0), base ipjk
        diag2(EET, ET, EE, E);
        if (i == o.nx - 1) setr(EET, o.nbrem(ET, c));
        // ijkett: D=(1,0,2), checks ipjkp then ijkpp, base ijkp
        diag2(ETT, ET, TT, T);
        if (k == o.nz - 1) setr(ETT, o.nbrem(ET, c));
        // third neighbours (ghost.f:1258-1278)
        setr(TTT, is_wallf(F(TTT)) ? R(TT) : R(TTT));
        if (k == o.nz - 1) setr(TTT, ijkt);
        if (k == o.nz - 2) setr(TTT, o.nbrem(TT, c));
        setr(EEE, is_wallf(F(EEE)) ? R(EE) : R(EEE));
        if (i == o.nx - 1) setr(EEE, ijke);
        if (i == o.nx - 2) setr(EEE, o.nbrem(EE, c));
        (void)ijkb;
    }
}

// ---------------------------------------------------------------------------
// limiters.f:14-56
// ---------------------------------------------------------------------------
double limiter(int lim_type, double erre, double beta) {
    switch (lim_type) {
    case 1: return std::max(0.0, 2.0 * erre / (1.0 + erre));
    case 2: return std::max(0.0, std::min(erre, 1.0));
    case 3: return std::max(std::max(0.0, std::min(2.0 * erre, 1.0)), std::min(erre, 2.0));
    case 4: {
        double bu = (1.0 - beta) + beta * erre;
        return std::max(0.0, std::min(std::min(2.0 * erre, bu), 2.0));
    }
    case 0: return (1.0 - beta) + beta * erre;
    default: return 0.0;
    }
}

// ---------------------------------------------------------------------------
// stencil gathers, subscr.f:2196-2450
// ---------------------------------------------------------------------------
// nb (remapped, 2D members)
void nb2(const Oracle &o, Sten &s, const double *a, int c) {
    s.c = a[c]; s.e = a[o.nbrem(E, c)]; s.t = a[o.nbrem(T, c)]; s.w = a[o.nbrem(W, c)]; s.b = a[o.nbrem(B, c)];
    s.et = a[o.nbrem(ET, c)]; s.wt = a[o.nbrem(WT, c)]; s.eb = a[o.nbrem(EB, c)];
    s.ee = a[o.nbrem(EE, c)]; s.tt = a[o.nbrem(TT, c)]; s.eet = a[o.nbrem(EET, c)];
    s.ett = a[o.nbrem(ETT, c)]; s.eee = a[o.nbrem(EEE, c)]; s.ttt = a[o.nbrem(TTT, c)];
}
// rnb (raw, 2D members)
void rnb2(const Oracle &o, Sten &s, const double *a, int c) {
    s.c = a[c]; s.e = a[o.nbraw(E, c)]; s.t = a[o.nbraw(T, c)]; s.w = a[o.nbraw(W, c)]; s.b = a[o.nbraw(B, c)];
    s.wt = a[o.nbraw(WT, c)]; s.et = a[o.nbraw(ET, c)]; s.eb = a[o.nbraw(EB, c)];
    s.ee = a[o.nbraw(EE, c)]; s.tt = a[o.nbraw(TT, c)]; s.eet = a[o.nbraw(EET, c)];
    s.ett = a[o.nbraw(ETT, c)]; s.eee = a[o.nbraw(EEE, c)]; s.ttt = a[o.nbraw(TTT, c)];
}
#include "pdac_oracle_ib.inc"

void first_nb2(const Oracle &o, Sten &s, const double *a, int c) {
    s.c = a[c]; s.e = a[o.nbrem(E, c)]; s.t = a[o.nbrem(T, c)]; s.w = a[o.nbrem(W, c)]; s.b = a[o.nbrem(B, c)];
}
void first_rnb2(const Oracle &o, Sten &s, const double *a, int c) {
    s.c = a[c]; s.e = a[o.nbraw(E, c)]; s.t = a[o.nbraw(T, c)]; s.w = a[o.nbraw(W, c)]; s.b = a[o.nbraw(B, c)];
}
void third_nb2(const Oracle &o, Sten &s, const double *a, int c) {
    s.ee = a[o.nbrem(EE, c)]; s.tt = a[o.nbrem(TT, c)]; s.ww = a[o.nbrem(WW, c)]; s.bb = a[o.nbrem(BB, c)];
}
Sten scale(const Sten &a, double f) {  // OPERATOR(*) of subscr.f
    Sten s;
    s.c = f * a.c; s.e = f * a.e; s.w = f * a.w; s.n = f * a.n; s.s = f * a.s; s.t = f * a.t; s.b = f * a.b;
    s.ee = f * a.ee; s.ww = f * a.ww; s.nn = f * a.nn; s.ss = f * a.ss; s.tt = f * a.tt; s.bb = f * a.bb;
    s.et = f * a.et; s.wt = f * a.wt; s.eb = f * a.eb; s.en = f * a.en; s.es = f * a.es; s.wn = f * a.wn;
    s.nt = f * a.nt; s.st = f * a.st; s.nb = f * a.nb; s.eet = f * a.eet; s.ett = f * a.ett; s.eee = f * a.eee;
    s.nnn = f * a.nnn; s.ttt = f * a.ttt; s.een = f * a.een; s.enn = f * a.enn; s.nnt = f * a.nnt; s.ntt = f * a.ntt;
    return s;
}
Sten cte(double v) {
    Sten s;
    s.c = s.e = s.w = s.n = s.s = s.t = s.b = v;
    s.ee = s.ww = s.nn = s.ss = s.tt = s.bb = v;
    s.et = s.wt = s.eb = s.en = s.es = s.wn = s.nt = s.st = s.nb = v;
    s.eet = s.ett = s.eee = s.nnn = s.ttt = s.een = s.enn = s.nnt = s.ntt = v;
    return s;
}

// ---------------------------------------------------------------------------
// interp.f:14-114 (x) and 215-320 (z), 2D members
// ---------------------------------------------------------------------------
Sten interp_x2(const Oracle &o, const Sten &f, int i) {
    const auto &dx = o.dx;
    int ip2 = std::min(o.nx, i + 2), ip3 = std::min(o.nx, i + 3);
    double dxm = dx[i] + dx[i - 1], dxp = dx[i] + dx[i + 1], dxpp = dx[i + 1] + dx[ip2], dxppp = dx[ip2] + dx[ip3];
    double indxm = 1.0 / dxm, indxp = 1.0 / dxp, indxpp = 1.0 / dxpp, indxppp = 1.0 / dxppp;
    Sten s;
    s.c = (dx[i + 1] * f.c + dx[i] * f.e) * indxp;
    s.e = (dx[ip2] * f.e + dx[i + 1] * f.ee) * indxpp;
    s.t = (dx[i + 1] * f.t + dx[i] * f.et) * indxp;
    s.w = (dx[i] * f.w + dx[i - 1] * f.c) * indxm;
    s.b = (dx[i + 1] * f.b + dx[i] * f.eb) * indxp;
    s.ee = (dx[ip2] * f.eee + dx[ip3] * f.ee) * indxppp;
    s.tt = (dx[i] * f.ett + dx[i + 1] * f.tt) * indxp;
    return s;
}
Sten interp_z2(const Oracle &o, const Sten &f, int k) {
    const auto &dz = o.dz;
    int kp2 = std::min(o.nz, k + 2), kp3 = std::min(o.nz, k + 3);
    double dzm = dz[k] + dz[k - 1], dzp = dz[k] + dz[k + 1], dzpp = dz[k + 1] + dz[kp2], dzppp = dz[kp2] + dz[kp3];
    double indzm = 1.0 / dzm, indzp = 1.0 / dzp, indzpp = 1.0 / dzpp, indzppp = 1.0 / dzppp;
    Sten s;
    s.c = (dz[k + 1] * f.c + dz[k] * f.t) * indzp;
    s.e = (dz[k + 1] * f.e + dz[k] * f.et) * indzp;
    s.t = (dz[kp2] * f.t + dz[k + 1] * f.tt) * indzpp;
    s.w = (dz[k + 1] * f.w + dz[k] * f.wt) * indzp;
    s.b = (dz[k] * f.b + dz[k - 1] * f.c) * indzm;
    s.ee = (dz[k] * f.eet + dz[k + 1] * f.ee) * indzp;
    s.tt = (dz[kp2] * f.ttt + dz[kp3] * f.tt) * indzppp;
    return s;
}

// ---------------------------------------------------------------------------
// momentum fluxes: flu_2d / muscl_flu_2d (flux_u.f:230-340),
// flw_2d / muscl_flw_2d (flux_w.f:220-356)
// ---------------------------------------------------------------------------
void flu_2d(const Oracle &o, double &fe, double &ft, double &fw, double &fb, const Sten &dens, const Sten &u,
            const Sten &w, int i, int c) {
    const auto &dx = o.dx;
    double dxp = dx[i] + dx[i + 1], indxp = 1.0 / dxp, cs;
    if (!o.fluidbit(o.nbraw(W, c))) {
        cs = 0.5 * (u.c + u.w);
        fw = 0.5 * (cs - std::fabs(cs)) * dens.c * u.c * o.r[i] + 0.5 * (cs + std::fabs(cs)) * dens.w * u.w * o.r[i];
    }
    if (!o.fluidbit(o.nbraw(B, c))) {
        cs = (dx[i + 1] * w.b + dx[i] * w.eb) * indxp;
        fb = 0.5 * (cs - std::fabs(cs)) * dens.c * u.c + 0.5 * (cs + std::fabs(cs)) * dens.b * u.b;
    }
    cs = 0.5 * (u.c + u.e);
    fe = 0.5 * (cs - std::fabs(cs)) * dens.e * u.e * o.r[i + 1] + 0.5 * (cs + std::fabs(cs)) * dens.c * u.c * o.r[i + 1];
    cs = (dx[i + 1] * w.c + dx[i] * w.e) * indxp;
    ft = 0.5 * (cs - std::fabs(cs)) * dens.t * u.t + 0.5 * (cs + std::fabs(cs)) * dens.c * u.c;
}

void muscl_flu_2d(const Oracle &o, double &fe, double &ft, const Sten &dens, const Sten &u, const Sten &w, int i, int k) {
    const auto &dx = o.dx, &dz = o.dz, &indx = o.indx;
    int lv = o.cfg.lv;
    int ip2 = std::min(o.nx, i + 2), kp2 = std::min(o.nz, k + 2);
    double dxp = dx[i] + dx[i + 1], dzm = dz[k] + dz[k - 1], dzp = dz[k] + dz[k + 1], dzpp = dz[k + 1] + dz[kp2];
    double indxp = 1.0 / dxp, indzm = 1.0 / dzm, indzp = 1.0 / dzp, indzpp = 1.0 / dzpp;
    double gradc = indx[i + 1] * (dens.e * u.e - dens.c * u.c);
    double gradw = indx[i] * (dens.c * u.c - dens.w * u.w);
    double grade = indx[ip2] * (dens.ee * u.ee - dens.e * u.e);
    double erre = 0, incr = 0, cs = 0.5 * (u.c + u.e);
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = 0.5 * dx[i + 1]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -0.5 * dx[i + 1]; }
    double lim = limiter(lv, erre, o.cfg.beta);
    double upwnd = lim * gradc * incr;
    fe = fe + upwnd * cs * o.r[i + 1];
    gradc = (dens.t * u.t - dens.c * u.c) * 2.0 * indzp;
    double gradb = (dens.c * u.c - dens.b * u.b) * 2.0 * indzm;
    double gradt = (dens.tt * u.tt - dens.t * u.t) * 2.0 * indzpp;
    erre = 0;
    cs = (dx[i + 1] * w.c + dx[i] * w.e) * indxp;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = 0.5 * dz[k]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -0.5 * dz[k + 1]; }
    lim = limiter(lv, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    ft = ft + upwnd * cs;
}

void flw_2d(const Oracle &o, double &fe, double &ft, double &fw, double &fb, const Sten &dens, const Sten &u,
            const Sten &w, int i, int k, int c) {
    const auto &dz = o.dz;
    double dzp = dz[k] + dz[k + 1], indzp = 1.0 / dzp, cs;
    if (!o.fluidbit(o.nbraw(W, c))) {
        cs = (u.wt * dz[k] + u.w * dz[k + 1]) * indzp;
        fw = 0.5 * dens.w * w.w * (cs + std::fabs(cs)) * o.rb[i - 1] + 0.5 * dens.c * w.c * (cs - std::fabs(cs)) * o.rb[i - 1];
    }
    if (!o.fluidbit(o.nbraw(B, c))) {
        cs = 0.5 * (w.c + w.b);
        fb = 0.5 * dens.b * w.b * (cs + std::fabs(cs)) + 0.5 * dens.c * w.c * (cs - std::fabs(cs));
    }
    cs = indzp * (u.c * dz[k + 1] + u.t * dz[k]);
    fe = 0.5 * dens.c * w.c * (cs + std::fabs(cs)) * o.rb[i] + 0.5 * dens.e * w.e * (cs - std::fabs(cs)) * o.rb[i];
    cs = 0.5 * (w.t + w.c);
    ft = 0.5 * dens.c * w.c * (cs + std::fabs(cs)) + 0.5 * dens.t * w.t * (cs - std::fabs(cs));
}

void muscl_flw_2d(const Oracle &o, double &fe, double &ft, const Sten &dens, const Sten &u, const Sten &w, int i, int k) {
    const auto &dx = o.dx, &dz = o.dz, &indz = o.indz;
    int lv = o.cfg.lv;
    int ip2 = std::min(o.nx, i + 2), kp2 = std::min(o.nz, k + 2);
    double dxm = dx[i] + dx[i - 1], dxp = dx[i] + dx[i + 1], dxpp = dx[i + 1] + dx[ip2], dzp = dz[k] + dz[k + 1];
    double indxm = 1.0 / dxm, indxp = 1.0 / dxp, indxpp = 1.0 / dxpp, indzp = 1.0 / dzp;
    double gradc = 2.0 * indxp * (dens.e * w.e - dens.c * w.c);
    double gradw = 2.0 * indxm * (dens.c * w.c - dens.w * w.w);
    double grade = 2.0 * indxpp * (dens.ee * w.ee - dens.e * w.e);
    double erre = 0, incr = 0;
    double cs = indzp * (u.c * dz[k + 1] + u.t * dz[k]);
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = 0.5 * dx[i]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -0.5 * dx[i + 1]; }
    double lim = limiter(lv, erre, o.cfg.beta);
    double upwnd = lim * gradc * incr;
    fe = fe + upwnd * cs * o.rb[i];
    gradc = (dens.t * w.t - dens.c * w.c) * indz[k + 1];
    double gradb = (dens.c * w.c - dens.b * w.b) * indz[k];
    double gradt = (dens.tt * w.tt - dens.t * w.t) * indz[kp2];
    erre = 0;
    cs = 0.5 * (w.t + w.c);
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = 0.5 * dz[k + 1]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -0.5 * dz[k + 1]; }
    lim = limiter(lv, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    ft = ft + upwnd * cs;
}

// ---------------------------------------------------------------------------
// mass fluxes: masf_2d / fmas_2d (flux_m.f:326-531)
// ---------------------------------------------------------------------------
void masf_2d(const Oracle &o, double &fe, double &ft, double &fw, double &fb, const Sten &dens, const Sten &u,
             const Sten &w, int i) {
    double cs = u.w;
    fw = 0.5 * (cs - std::fabs(cs)) * dens.c * o.rb[i - 1] + 0.5 * (cs + std::fabs(cs)) * dens.w * o.rb[i - 1];
    cs = w.b;
    fb = 0.5 * (cs - std::fabs(cs)) * dens.c + 0.5 * (cs + std::fabs(cs)) * dens.b;
    cs = u.c;
    fe = 0.5 * (cs - std::fabs(cs)) * dens.e * o.rb[i] + 0.5 * (cs + std::fabs(cs)) * dens.c * o.rb[i];
    cs = w.c;
    ft = 0.5 * (cs - std::fabs(cs)) * dens.t + 0.5 * (cs + std::fabs(cs)) * dens.c;
}

void fmas_2d(const Oracle &o, double &fe, double &ft, double &fw, double &fb, const Sten &dens, const Sten &u,
             const Sten &w, int c) {
    const auto &dx = o.dx, &dz = o.dz;
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int lm = o.cfg.lm;
    int im2 = std::max(1, i - 2), ip2 = std::min(o.nx, i + 2), km2 = std::max(1, k - 2), kp2 = std::min(o.nz, k + 2);
    double dxmm = dx[i - 1] + dx[im2], dxm = dx[i] + dx[i - 1], dxp = dx[i] + dx[i + 1], dxpp = dx[i + 1] + dx[ip2];
    double dzmm = dz[k - 1] + dz[km2], dzm = dz[k] + dz[k - 1], dzp = dz[k] + dz[k + 1], dzpp = dz[k + 1] + dz[kp2];
    double indxmm = 1.0 / dxmm, indxm = 1.0 / dxm, indxp = 1.0 / dxp, indxpp = 1.0 / dxpp;
    double indzmm = 1.0 / dzmm, indzm = 1.0 / dzm, indzp = 1.0 / dzp, indzpp = 1.0 / dzpp;
    double gradc, gradw, grade, gradb, gradt, erre, incr = 0, lim, upwnd, cs;
    // West
    gradc = 2.0 * indxm * (dens.c - dens.w);
    gradw = 2.0 * indxmm * (dens.w - dens.ww);
    grade = 2.0 * indxp * (dens.e - dens.c);
    lim = 0; erre = 0;
    cs = u.w;
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = 0.5 * dx[i - 1]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -0.5 * dx[i]; }
    if (i != 2 && o.flag[o.nbraw(W, c)] == FLUID) lim = limiter(lm, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    fw = fw + upwnd * cs * o.rb[i - 1];
    // East
    gradw = gradc; gradc = grade;
    grade = 2.0 * indxpp * (dens.ee - dens.e);
    lim = 0; erre = 0;
    cs = u.c;
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = 0.5 * dx[i]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -0.5 * dx[i + 1]; }
    if (i != o.nx - 1 && o.flag[o.nbraw(E, c)] == FLUID) lim = limiter(lm, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    fe = fe + upwnd * cs * o.rb[i];
    // Bottom
    gradc = 2.0 * indzm * (dens.c - dens.b);
    gradb = 2.0 * indzmm * (dens.b - dens.bb);
    gradt = 2.0 * indzp * (dens.t - dens.c);
    lim = 0; erre = 0;
    cs = w.b;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = 0.5 * dz[k - 1]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -0.5 * dz[k]; }
    if (k != 2 && o.flag[o.nbraw(B, c)] == FLUID) lim = limiter(lm, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    fb = fb + upwnd * cs;
    // Top
    gradb = gradc; gradc = gradt;
    gradt = 2.0 * indzpp * (dens.tt - dens.t);
    lim = 0; erre = 0;
    cs = w.c;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = 0.5 * dz[k]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -0.5 * dz[k + 1]; }
    if (k != o.nz - 1 && o.flag[o.nbraw(T, c)] == FLUID) lim = limiter(lm, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    ft = ft + upwnd * cs;
}

// ---------------------------------------------------------------------------
// scalar fluxes: fsc_2d / muscl_fsc_2d (flux_sc.f:236-390)
// ---------------------------------------------------------------------------
void fsc_2d(const Oracle &o, double &fe, double &ft, double &fw, double &fb, const Sten &dens, const Sten &field,
            const Sten &u, const Sten &w, int c) {
    int i, j, k;
    o.ijk_of(c, i, j, k);
    double cs;
    if (!o.fluidbit(o.nbraw(W, c))) {
        cs = u.w;
        fw = 0.5 * (cs - std::fabs(cs)) * dens.c * field.c * o.rb[i - 1] + 0.5 * (cs + std::fabs(cs)) * dens.w * field.w * o.rb[i - 1];
    }
    if (!o.fluidbit(o.nbraw(B, c))) {
        cs = w.b;
        fb = 0.5 * (cs - std::fabs(cs)) * dens.c * field.c + 0.5 * (cs + std::fabs(cs)) * dens.b * field.b;
    }
    cs = u.c;
    fe = 0.5 * (cs - std::fabs(cs)) * dens.e * field.e * o.rb[i] + 0.5 * (cs + std::fabs(cs)) * dens.c * field.c * o.rb[i];
    cs = w.c;
    ft = 0.5 * (cs - std::fabs(cs)) * dens.t * field.t + 0.5 * (cs + std::fabs(cs)) * dens.c * field.c;
}

void muscl_fsc_2d(const Oracle &o, double &fe, double &ft, const Sten &dens, const Sten &field, const Sten &u,
                  const Sten &w, int c) {
    const auto &dx = o.dx, &dz = o.dz;
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int lm = o.cfg.lm;
    int ip2 = std::min(o.nx, i + 2), kp2 = std::min(o.nz, k + 2);
    double dxm = dx[i] + dx[i - 1], dxp = dx[i] + dx[i + 1], dxpp = dx[i + 1] + dx[ip2];
    double dzm = dz[k] + dz[k - 1], dzp = dz[k] + dz[k + 1], dzpp = dz[k + 1] + dz[kp2];
    double indxm = 1.0 / dxm, indxp = 1.0 / dxp, indxpp = 1.0 / dxpp;
    double indzm = 1.0 / dzm, indzp = 1.0 / dzp, indzpp = 1.0 / dzpp;
    double gradc = 2.0 * indxp * (dens.e * field.e - dens.c * field.c);
    double gradw = 2.0 * indxm * (dens.c * field.c - dens.w * field.w);
    double grade = 2.0 * indxpp * (dens.ee * field.ee - dens.e * field.e);
    double lim = 0, erre = 0, incr = 0, cs = u.c;
    if (cs >= 0) { if (gradc != 0) erre = gradw / gradc; incr = 0.5 * dx[i]; }
    else if (cs < 0) { if (gradc != 0) erre = grade / gradc; incr = -0.5 * dx[i + 1]; }
    if (i != o.nx - 1) lim = limiter(lm, erre, o.cfg.beta);
    double upwnd = lim * gradc * incr;
    fe = fe + upwnd * cs * o.rb[i];
    gradc = 2.0 * indzp * (dens.t * field.t - dens.c * field.c);
    double gradb = 2.0 * indzm * (dens.c * field.c - dens.b * field.b);
    double gradt = 2.0 * indzpp * (dens.tt * field.tt - dens.t * field.t);
    lim = 0; erre = 0;
    cs = w.c;
    if (cs >= 0) { if (gradc != 0) erre = gradb / gradc; incr = 0.5 * dz[k]; }
    else if (cs < 0) { if (gradc != 0) erre = gradt / gradc; incr = -0.5 * dz[k + 1]; }
    if (k != o.nz - 1) lim = limiter(lm, erre, o.cfg.beta);
    upwnd = lim * gradc * incr;
    ft = ft + upwnd * cs;
}

// diffusive enthalpy flux, hotc.f:12-82 (2D: y members unused)
void hotc_2d(const Oracle &o, double &hfe, double &hft, double &hfw, double &hfb, const Sten &ep, const Sten &tg,
             const Sten &kapgt, int c) {
    const auto &dx = o.dx, &dz = o.dz;
    int i, j, k;
    o.ijk_of(c, i, j, k);
    if (o.flag[o.nbraw(W, c)] != 1) {
        double dxm = dx[i] + dx[i - 1], indxm = 1.0 / dxm;
        double kmw = (dx[i - 1] * kapgt.c + dx[i] * kapgt.w) * indxm;
        double epmw = (dx[i - 1] * ep.c + dx[i] * ep.w) * indxm;
        hfw = kmw * epmw * (tg.c - tg.w) * indxm * 2.0 * o.rb[i - 1];
    }
    if (o.flag[o.nbraw(B, c)] != 1) {
        double dzm = dz[k] + dz[k - 1], indzm = 1.0 / dzm;
        double kmb = (dz[k - 1] * kapgt.c + dz[k] * kapgt.b) * indzm;
        double epmb = (dz[k - 1] * ep.c + dz[k] * ep.b) * indzm;
        hfb = kmb * epmb * (tg.c - tg.b) * indzm * 2.0;
    }
    double dxp = dx[i] + dx[i + 1], indxp = 1.0 / dxp;
    double kme = (dx[i + 1] * kapgt.c + dx[i] * kapgt.e) * indxp;
    double epme = (dx[i + 1] * ep.c + dx[i] * ep.e) * indxp;
    hfe = kme * epme * (tg.e - tg.c) * indxp * 2.0 * o.rb[i];
    double dzp = dz[k] + dz[k + 1], indzp = 1.0 / dzp;
    double kmt = (dz[k + 1] * kapgt.c + dz[k] * kapgt.t) * indzp;
    double epmt = (dz[k + 1] * ep.c + dz[k] * ep.t) * indzp;
    hft = kmt * epmt * (tg.t - tg.c) * indzp * 2.0;
}

// ---------------------------------------------------------------------------
// closures
// ---------------------------------------------------------------------------
// gas viscosity / conductivity, visc.f:37-148
void viscon(const Oracle &o, double &mu, double &kap, const double *xgc, double tg) {
    double mmug[8] = {0}, ckg[8] = {0}, phij[8][8] = {{0}};
    for (int ig = 0; ig < o.ng; ++ig) {
        int igg = o.gas_type[ig];
        double tst = tg / o.mmugek[igg];
        double om = 1.16145 * pdac_fp::pow(tst, -0.14874) + 0.52487 * pdac_fp::exp(-0.77320 * tst) + 2.16178 * pdac_fp::exp(-2.43787 * tst);
        double m = 1.0e3 * o.gmw[igg];
        mmug[igg] = 26.69 * std::sqrt(m * tg) / (o.mmugs[igg] * o.mmugs[igg] * om);
        mmug[igg] = mmug[igg] * 1.0e-7;
    }
    double t1 = tg, t2 = t1 * tg, t3 = t2 * tg;
    double tr = tg / 132.5;
    double trm1 = 1.0 / tr, trm2 = trm1 * trm1, trm3 = trm2 * trm1, trm4 = trm3 * trm1;
    double trsrt = std::sqrt(tr);
    ckg[1] = -3.273e-4 + 9.966e-5 * t1 - 3.743e-8 * t2 + 9.732e-12 * t3;
    ckg[2] = 3.919e-4 + 9.816e-5 * t1 - 5.067e-8 * t2 + 1.504e-11 * t3;
    ckg[3] = -7.215e-3 + 8.015e-5 * t1 + 5.477e-9 * t2 - 1.053e-11 * t3;
    ckg[4] = 8.099e-3 + 6.689e-4 * t1 - 4.158e-7 * t2 + 1.562e-10 * t3;
    ckg[5] = 7.341e-3 - 1.013e-5 * t1 + 1.801e-7 * t2 - 9.100e-11 * t3;
    ckg[6] = 25.9778e-3 * (0.2395 * tr + 6.4977e-3 * trsrt + 1.0 - 1.92615 * trm1 + 2.00383 * trm2 - 1.07553 * trm3 + 0.229414 * trm4);
    ckg[7] = -8.086e-3 + 6.344e-5 * t1 - 1.382e-8 * t2 + 2.303e-12 * t3;
    for (int ig = 0; ig < o.ng; ++ig) {
        int igg = o.gas_type[ig];
        for (int jg = 0; jg < o.ng; ++jg) {
            int jgg = o.gas_type[jg];
            double aa = o.gmw[igg] / o.gmw[jgg];
            double bb = mmug[igg] / mmug[jgg];
            double cc = 1.0 + std::sqrt(bb) * pdac_fp::pow(aa, -0.25);
            phij[igg][jgg] = cc * cc / std::sqrt(8.0 * (1.0 + aa));
        }
    }
    mu = 0; kap = 0;
    for (int ig = 0; ig < o.ng; ++ig) {
        int igg = o.gas_type[ig];
        double sum = 0;
        for (int jg = 0; jg < o.ng; ++jg) sum = sum + xgc[jg] * phij[igg][o.gas_type[jg]];
        double suminv = 1.0 / sum;
        mu = mu + xgc[ig] * mmug[igg] * suminv;
        kap = kap + xgc[ig] * ckg[igg] * suminv;
    }
}

// heat capacities, hcapgs.f:33-85 (cpc 1-based, 7 entries)
void hcapg(const Oracle &o, double *cpc, double tg) {
    double t1 = (o.cfg.icpc <= 1) ? o.cfg.tref : tg;
    double t2 = t1 * t1, t3 = t1 * t2;
    cpc[1] = (2.811e1 - 3.68e-6 * t1 + 1.746e-5 * t2 - 1.065e-8 * t3);
    cpc[2] = (3.115e1 - 1.357e-2 * t1 + 2.680e-5 * t2 - 1.168e-8 * t3);
    cpc[3] = (1.980e1 + 7.344e-2 * t1 - 5.602e-5 * t2 + 1.715e-8 * t3);
    cpc[4] = (2.714e1 + 9.274e-3 * t1 - 1.381e-5 * t2 + 7.645e-9 * t3);
    cpc[5] = (3.224e1 + 1.924e-3 * t1 + 1.055e-5 * t2 - 3.596e-9 * t3);
    cpc[6] = (3.0413e1 - 1.059e-2 * t1 + 2.458e-5 * t2 - 1.135e-8 * t3);
    cpc[7] = (2.385e1 + 6.699e-2 * t1 - 4.961e-5 * t2 + 1.328e-8 * t3);
    for (int g = 1; g <= 7; ++g) cpc[g] = cpc[g] / o.gmw[g];
    if (o.cfg.icpc == 0) { cpc[5] = 1810.0; cpc[6] = 1004.0; }
}

// eosg.f:114-137
double thermal_eosg(const Oracle &o, double tg, double p, const double *xg) {
    double mg = 0;
    for (int ig = 0; ig < o.ng; ++ig) mg = mg + xg[ig] * o.gmw[o.gas_type[ig]];
    return p / (o.rgas * tg) * mg;
}

// eosg.f:38-68
void mole(const Oracle &o, double *xg, const double *yg) {
    double mol = 0;
    for (int ig = 0; ig < o.ng; ++ig) mol = mol + yg[ig] / o.gmw[o.gas_type[ig]];
    double molinv = (std::fabs(mol) <= 1e-10) ? 0.0 : 1.0 / mol;
    for (int ig = 0; ig < o.ng; ++ig) xg[ig] = yg[ig] / o.gmw[o.gas_type[ig]] * molinv;
}

// eosg.f:139-223; returns info (0 ok)
int caloric_eosg(const Oracle &o, double &cgas, double &tg, const double *yg, double sieg) {
    double cpc[8];
    int info = 1;
    for (int ii = 1; ii <= 2000; ++ii) {
        double tgnn = tg;
        hcapg(o, cpc, tg);
        cgas = 0;
        for (int ig = 0; ig < o.ng; ++ig) cgas = cpc[o.gas_type[ig]] * yg[ig] + cgas;
        tg = o.tzero + (sieg - o.hzerog) / cgas;
        if (std::fabs((tgnn - tg) / tgnn) <= 1.0e-8) { info = 0; break; }
    }
    if (tg <= 0.0) info = 1;
    return info;
}

// drag.f:60-157
double kdrags(const Oracle &o, double du, double dv, double dw, double ep, double rgp, double rlk, double mug, int is) {
    double vrel = std::sqrt(du * du + dv * dv + dw * dw);
    double drag;
    if (ep < 0.8) {  // kdragl, drag.f:120-143
        double denom = 1.0 / (o.dk[is] * o.phis[is] * ep);
        drag = 150.0 * ep * rlk * o.inrl[is] * mug * denom + 1.75 * rgp * vrel;
        drag = drag * rlk * o.inrl[is] * denom;
    } else {         // kdragg, drag.f:83-118
        double eps = rlk * o.inrl[is];
        double reynum = rgp * o.dk[is] * o.phis[is] * vrel / mug;
        double dc;
        if (reynum <= 1000.0) dc = (24.0 / reynum) * (1.0 + (double)0.15f * pdac_fp::pow(reynum, (double)0.687f));
        else dc = (double)0.43828814f;
        dc = std::min(dc, 1.0e4);
        drag = 0.75 * dc * eps / (o.dk[is] * o.phis[is]) * rgp * vrel;
        drag = drag * pdac_fp::pow(ep, (double)(-2.65f));
    }
    return drag;
}

// drag.f:11-58
double sdrag(const Oracle &o, double du, double dv, double dw, double ep, double rgp, double rlk, double mug, int is) {
    double vrel = std::sqrt(du * du + dv * dv + dw * dw);
    double eps = rlk * o.inrl[is];
    double reynum = rgp * o.dk[is] * o.phis[is] * vrel / mug;
    double a = pdac_fp::pow(ep, (double)4.14f), b;
    if (ep <= (double)0.85f) b = (double)0.8f * pdac_fp::pow(ep, (double)1.28f);
    else b = pdac_fp::pow(ep, (double)2.65f);
    double vr = 0.5 * (a - (double)0.06f * reynum +
                       std::sqrt((double)0.0036f * reynum * reynum + (double)0.12f * reynum * (2.0 * b - a) + a * a));
    double dc = (0.63 + 4.8 / std::sqrt(reynum));
    dc = dc * dc;
    dc = std::min(dc, 1.0e4);
    double drag = 0.75 * dc * eps / (o.dk[is] * o.phis[is]) * rgp * vrel;
    return drag / vr;
}

// drag.f:248-298
double ppdrag(const Oracle &o, const double *rlkc, int k, int kk) {  // rlkc 1-based per class
    int k1, k2;
    if (o.dk[k - 1] >= o.dk[kk - 1]) { k1 = k - 1; k2 = kk - 1; }
    else { k1 = kk - 1; k2 = k - 1; }
    double ep1 = rlkc[k1] * o.inrl[k1], ep2 = rlkc[k2] * o.inrl[k2], epsum = ep1 + ep2;
    if (ep1 > 0 && ep2 > 0) {
        double xbar = ep1 / epsum, epkl;
        if (xbar <= o.philim[k - 1][kk - 1]) epkl = o.epsl[k - 1][kk - 1] * xbar + o.phi[k2];
        else epkl = o.epsu[k - 1][kk - 1] * (1.0 - xbar) + o.phi[k1];
        double espo = 1.0 / 3.0;
        double m1 = pdac_fp::pow(epkl, espo), m2 = pdac_fp::pow(epsum, espo);
        double effe = (3.0 * m1 + m2) / (2.0 * (m1 - m2));
        return 1.0 * (1.0 + 1.0) * rlkc[k - 1] * rlkc[kk - 1] * o.dkf[k - 1][kk - 1] * effe;
    }
    return 0.0;
}

// hvs.f:9-83
double hvs(const Oracle &o, double rlk, double rog, double ep, double du, double dv, double dw, double mug,
           double kapg, double cg, int k) {
    (void)ep;
    if (rlk <= 0.0) return 0.0;
    double eps = rlk * o.inrl[k];
    double eps2 = eps * eps;
    double asurf = 6.0 * kapg * eps / (o.dk[k] * o.dk[k]);
    double vrel = std::sqrt(du * du + dv * dv + dw * dw);
    double reynum = o.dk[k] * vrel * rog / mug;
    double pranum = cg * mug / kapg;
    double pranumexp = pdac_fp::pow(pranum, 1.0 / 3.0);
    double nusselt = (2.0 + 5.0 * eps2) * (1.0 + 0.7 * pdac_fp::pow(reynum, 0.2) * pranumexp);
    nusselt = nusselt + (0.13 + 1.2 * eps2) * pdac_fp::pow(reynum, 0.7) * pranumexp;
    return nusselt * asurf;
}

// Gauss-Jordan of matrix.f:351-391 on an nph x nph system (1-based a[l][ll])
void gauss_jordan(const Oracle &o, double a[PDAC_MAX_NSOLID + 2][PDAC_MAX_NSOLID + 2], double *b) {
    int nph = o.nph;
    for (int l = 2; l <= nph; ++l) {
        if (std::fabs(a[l][l]) < o.plim[l - 1]) {
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

using Mat = double[PDAC_MAX_NSOLID + 2][PDAC_MAX_NSOLID + 2];

// ---------------------------------------------------------------------------
// matrix.f:186-328 assemble_matrix (E/T faces), 2D
// ---------------------------------------------------------------------------
void assemble_et_2d(Oracle &o, int c, double dt, Mat &au, double *bu, Mat &aw, double *bw) {
    const auto &dx = o.dx, &dz = o.dz;
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int ijke = o.nbrem(E, c), ijkt = o.nbrem(T, c);
    double alpha = o.cfg.alpha, ag = o.cfg.alphagrav;
    double dxi = dx[i], dxip1 = dx[i + 1], dzk = dz[k], dzkp1 = dz[k + 1];
    double pijk = o.p[c];
    double dxp = dxi + dxip1, dzp = dzk + dzkp1;
    double indxp = 1.0 / dxp, indzp = 1.0 / dzp;
    double ep_e, ep_t;
    if (o.cfg.pmodel == 1) {
        ep_e = (dxi * o.ep[ijke] + dxip1 * o.ep[c]) * indxp;
        ep_t = (dzk * o.ep[ijkt] + dzkp1 * o.ep[c]) * indzp;
    } else { ep_e = 1.0; ep_t = 1.0; }
    auto A = [&](vector<double> &app, int cell, int ls) { return app[(size_t)(ls - 1) * o.ncell + cell]; };
    bu[1] = o.rug[c] + alpha * dt * indxp * 2.0 * ep_e * (pijk - o.p[ijke]);
    bw[1] = o.rwg[c] + alpha * dt * indzp * 2.0 * ep_t * (pijk - o.p[ijkt]);
    bu[1] = bu[1] + dt * ag * indxp * o.cfg.gravx * (dxi * o.rgp[ijke] + dxip1 * o.rgp[c]);
    bw[1] = bw[1] + dt * ag * indzp * o.cfg.gravz * (dzk * o.rgp[ijkt] + dzkp1 * o.rgp[c]);
    au[1][1] = alpha * (dxi * A(o.appu, ijke, 1) + dxip1 * A(o.appu, c, 1)) * indxp;
    au[1][1] = au[1][1] + (dxi * o.rgp[ijke] + dxip1 * o.rgp[c]) * indxp;
    aw[1][1] = alpha * (dzk * A(o.appw, ijkt, 1) + dzkp1 * A(o.appw, c, 1)) * indzp;
    aw[1][1] = aw[1][1] + (dzk * o.rgp[ijkt] + dzkp1 * o.rgp[c]) * indzp;
    for (int l = 2; l <= o.nph; ++l) {
        double eps_e, eps_t;
        if (o.cfg.pmodel == 1) {
            eps_e = (dxi * o.S(o.rlk, ijke, l - 1) + dxip1 * o.S(o.rlk, c, l - 1)) * indxp * o.inrl[l - 1];
            eps_t = (dzk * o.S(o.rlk, ijkt, l - 1) + dzkp1 * o.S(o.rlk, c, l - 1)) * indzp * o.inrl[l - 1];
        } else { eps_e = 0.0; eps_t = 0.0; }
        bu[l] = o.S(o.rus, c, l - 1) + alpha * dt * indxp * 2.0 * eps_e * (pijk - o.p[ijke]);
        bw[l] = o.S(o.rws, c, l - 1) + alpha * dt * indzp * 2.0 * eps_t * (pijk - o.p[ijkt]);
        bu[l] = bu[l] + dt * ag * indxp * o.cfg.gravx * (dxi * o.S(o.rlk, ijke, l - 1) + dxip1 * o.S(o.rlk, c, l - 1));
        bw[l] = bw[l] + dt * ag * indzp * o.cfg.gravz * (dzk * o.S(o.rlk, ijkt, l - 1) + dzkp1 * o.S(o.rlk, c, l - 1));
        int ls1 = l * (l - 1) / 2;
        for (int ll = 1; ll <= l; ++ll) {
            int ls = ls1 + ll;
            au[l][ll] = alpha * (dxi * A(o.appu, ijke, ls) + dxip1 * A(o.appu, c, ls)) * indxp;
            au[ll][l] = au[l][ll];
            aw[l][ll] = alpha * (dzk * A(o.appw, ijkt, ls) + dzkp1 * A(o.appw, c, ls)) * indzp;
            aw[ll][l] = aw[l][ll];
        }
        au[l][l] = au[l][l] + (dxi * o.S(o.rlk, ijke, l - 1) + dxip1 * o.S(o.rlk, c, l - 1)) * indxp;
        aw[l][l] = aw[l][l] + (dzk * o.S(o.rlk, ijkt, l - 1) + dzkp1 * o.S(o.rlk, c, l - 1)) * indzp;
    }
}

// matrix.f:38-184 assemble_all_matrix (W/B faces), 2D
void assemble_wb_2d(Oracle &o, int c, double dt, Mat &au1, double *bu1, Mat &aw1, double *bw1) {
    const auto &dx = o.dx, &dz = o.dz;
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    int ijkw = o.nbrem(W, c), ijkb = o.nbrem(B, c);
    double alpha = o.cfg.alpha, ag = o.cfg.alphagrav;
    double dxi = dx[i], dxm = dx[i] + dx[i - 1], dxim1 = dx[i - 1];
    double dzk = dz[k], dzm = dz[k] + dz[k - 1], dzkm1 = dz[k - 1];
    double pijk = o.p[c], epijk = o.ep[c], rgpijk = o.rgp[c];
    double indxm = 1.0 / dxm, indzm = 1.0 / dzm;
    double ep_w, ep_b;
    if (o.cfg.pmodel == 1) {
        ep_w = (dxi * o.ep[ijkw] + dxim1 * epijk) * indxm;
        ep_b = (dzk * o.ep[ijkb] + dzkm1 * epijk) * indzm;
    } else { ep_w = 1.0; ep_b = 1.0; }
    auto A = [&](vector<double> &app, int cell, int ls) { return app[(size_t)(ls - 1) * o.ncell + cell]; };
    bu1[1] = o.rug[imjk] + alpha * dt * indxm * 2.0 * ep_w * (o.p[ijkw] - pijk);
    bw1[1] = o.rwg[ijkm] + alpha * dt * indzm * 2.0 * ep_b * (o.p[ijkb] - pijk);
    bu1[1] = bu1[1] + dt * ag * indxm * o.cfg.gravx * (dxi * o.rgp[ijkw] + dxim1 * o.rgp[c]);
    bw1[1] = bw1[1] + dt * ag * indzm * o.cfg.gravz * (dzk * o.rgp[ijkb] + dzkm1 * o.rgp[c]);
    au1[1][1] = alpha * (dxi * A(o.appu, ijkw, 1) + dxim1 * A(o.appu, c, 1)) * indxm;
    au1[1][1] = au1[1][1] + (dxi * o.rgp[ijkw] + dxim1 * rgpijk) * indxm;
    aw1[1][1] = alpha * (dzk * A(o.appw, ijkb, 1) + dzkm1 * A(o.appw, c, 1)) * indzm;
    aw1[1][1] = aw1[1][1] + (dzk * o.rgp[ijkb] + dzkm1 * rgpijk) * indzm;
    for (int l = 2; l <= o.nph; ++l) {
        double rlklm1 = o.S(o.rlk, c, l - 1);
        double eps_w, eps_b;
        if (o.cfg.pmodel == 1) {
            eps_w = (dxi * o.S(o.rlk, ijkw, l - 1) + dxim1 * rlklm1) * indxm * o.inrl[l - 1];
            eps_b = (dzk * o.S(o.rlk, ijkb, l - 1) + dzkm1 * rlklm1) * indzm * o.inrl[l - 1];
        } else { eps_w = 0.0; eps_b = 0.0; }
        bu1[l] = o.S(o.rus, imjk, l - 1) + alpha * dt * indxm * 2.0 * eps_w * (o.p[ijkw] - pijk);
        bw1[l] = o.S(o.rws, ijkm, l - 1) + alpha * dt * indzm * 2.0 * eps_b * (o.p[ijkb] - pijk);
        bu1[l] = bu1[l] + dt * ag * indxm * o.cfg.gravx * (dxi * o.S(o.rlk, ijkw, l - 1) + dxim1 * o.S(o.rlk, c, l - 1));
        bw1[l] = bw1[l] + dt * ag * indzm * o.cfg.gravz * (dzk * o.S(o.rlk, ijkb, l - 1) + dzkm1 * o.S(o.rlk, c, l - 1));
        int ls1 = l * (l - 1) / 2;
        for (int ll = 1; ll <= l; ++ll) {
            int ls = ls1 + ll;
            au1[ll][l] = alpha * (dxi * A(o.appu, ijkw, ls) + dxim1 * A(o.appu, c, ls)) * indxm;
            au1[l][ll] = au1[ll][l];
            aw1[ll][l] = alpha * (dzk * A(o.appw, ijkb, ls) + dzkm1 * A(o.appw, c, ls)) * indzm;
            aw1[l][ll] = aw1[ll][l];
        }
        au1[l][l] = au1[l][l] + (dxi * o.S(o.rlk, ijkw, l - 1) + dxim1 * rlklm1) * indxm;
        aw1[l][l] = aw1[l][l] + (dzk * o.S(o.rlk, ijkb, l - 1) + dzkm1 * rlklm1) * indzm;
    }
}

// matrix.f:481-631 solve_velocities (E, T faces)
void solve_et_2d(Oracle &o, int c, Mat &au, double *bu, Mat &aw, double *bw) {
    if (o.fluidbit(o.nbraw(E, c))) {
        gauss_jordan(o, au, bu);
        o.ug[c] = bu[1];
        for (int l = 2; l <= o.nph; ++l) o.S(o.us, c, l - 1) = bu[l];
    }
    if (o.fluidbit(o.nbraw(T, c))) {
        gauss_jordan(o, aw, bw);
        o.wg[c] = bw[1];
        for (int l = 2; l <= o.nph; ++l) o.S(o.ws, c, l - 1) = bw[l];
    }
}

// matrix.f:330-479 solve_all_velocities (W, B faces then E, T)
void solve_all_2d(Oracle &o, int c, Mat &au1, double *bu1, Mat &aw1, double *bw1, Mat &au, double *bu, Mat &aw, double *bw) {
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    if (o.fluidbit(imjk)) {
        gauss_jordan(o, au1, bu1);
        o.ug[imjk] = bu1[1];
        for (int l = 2; l <= o.nph; ++l) o.S(o.us, imjk, l - 1) = bu1[l];
    }
    if (o.fluidbit(ijkm)) {
        gauss_jordan(o, aw1, bw1);
        o.wg[ijkm] = bw1[1];
        for (int l = 2; l <= o.nph; ++l) o.S(o.ws, ijkm, l - 1) = bw1[l];
    }
    solve_et_2d(o, c, au, bu, aw, bw);
}

// ---------------------------------------------------------------------------
// stress2D, visc.f:561-696
// ---------------------------------------------------------------------------
void stress2d(Oracle &o, double *visx, double *visz, const double *mu, const double *lambda, const double *eps,
              const double *u, const double *w) {
    const auto &dx = o.dx, &dz = o.dz, &indx = o.indx, &indz = o.indz, &r = o.r, &rb = o.rb, &inr = o.inr, &inrb = o.inrb;
    double cm = 2.0 / 3.0;
    for (int c = 0; c < o.ncell; ++c) { visx[c] = 0; visz[c] = 0; }
    for (int c = 0; c < o.ncell; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int ipjk = o.nbraw(E, c), imjk = o.nbraw(W, c), ijkp = o.nbraw(T, c), ijkm = o.nbraw(B, c);
        int ipjkm = o.nbraw(EB, c), imjkp = o.nbraw(WT, c);
        int ijke = o.nbrem(E, c), ijkt = o.nbrem(T, c), ijket = o.nbrem(ET, c), ijkeb = o.nbrem(EB, c);
        int ijkb = o.nbrem(B, c), ijkw = o.nbrem(W, c), ijkwt = o.nbrem(WT, c);
        double dxp = (dx[i] + dx[i + 1]), dxm = (dx[i] + dx[i - 1]), dzp = (dz[k] + dz[k + 1]), dzm = (dz[k] + dz[k - 1]);
        double indxp = 1.0 / dxp, indxm = 1.0 / dxm, indzp = 1.0 / dzp, indzm = 1.0 / dzm;
        double divr = ((rb[i + 1] * u[ipjk] - rb[i] * u[c]) * inr[i + 1] * indx[i + 1] + (w[ipjk] - w[ipjkm]) * indz[k]);
        double divc = ((rb[i] * u[c] - rb[i - 1] * u[imjk]) * inr[i] * indx[i] + (w[c] - w[ijkm]) * indz[k]);
        double divt = ((rb[i] * u[ijkp] - rb[i - 1] * u[imjkp]) * inr[i] * indx[i] + (w[ijkp] - w[c]) * indz[k + 1]);
        double txx2 = 2.0 * (u[ipjk] - u[c]) * indx[i + 1];
        double txx1 = 2.0 * (u[c] - u[imjk]) * indx[i];
        double tyy2 = 2.0 * (w[ijkp] - w[c]) * indz[k + 1];
        double tyy1 = 2.0 * (w[c] - w[ijkm]) * indz[k];
        txx2 = mu[ijke] * txx2 - cm * lambda[ijke] * divr;
        txx1 = mu[c] * txx1 - cm * lambda[c] * divc;
        tyy2 = mu[ijkt] * tyy2 - cm * lambda[ijkt] * divt;
        tyy1 = mu[c] * tyy1 - cm * lambda[c] * divc;
        double tyx2 = (u[ijkp] - u[c]) * indzp * 2.0 + (w[ipjk] - w[c]) * indxp * 2.0;
        double tyx1 = (u[c] - u[ijkm]) * indzm * 2.0 + (w[ipjkm] - w[ijkm]) * indxp * 2.0;
        double txy2 = tyx2;
        double txy1 = (u[imjkp] - u[imjk]) * indzp * 2.0 + (w[c] - w[imjk]) * indxm * 2.0;
        double t0;
        double eps0 = 0;
        if (o.cfg.itc == 1) {
            eps0 = (eps[c] * dx[i + 1] + eps[ijke] * dx[i]) * indxp;
            double mu0 = (mu[c] * dx[i + 1] + mu[ijke] * dx[i]) * indxp;
            double lambda0 = (lambda[c] * dx[i + 1] + lambda[ijke] * dx[i]) * indxp;
            t0 = 2.0 * u[c] * inrb[i];
            double du = (rb[i + 1] * u[ipjk] - rb[i - 1] * u[imjk]);
            double wm2 = (dx[i] * w[ipjk] + dx[i + 1] * w[c]) * indxp;
            double wm1 = (dx[i] * w[ipjkm] + dx[i + 1] * w[ijkm]) * indxp;
            double dw = wm2 - wm1;
            double dive = (inrb[i] * du * indxp + dw * indz[k]);
            t0 = mu0 * t0 - cm * lambda0 * dive;
        } else {
            t0 = 0.0;
        }
        double epsmu21 = (dz[k] * eps[ijkt] * mu[ijkt] + dz[k + 1] * eps[c] * mu[c]) * indzp;
        double epsmu22 = (dz[k] * eps[ijket] * mu[ijket] + dz[k + 1] * eps[ijke] * mu[ijke]) * indzp;
        double epsmu2 = (dx[i + 1] * epsmu21 + dx[i] * epsmu22) * indxp;
        double epsmu11 = (dz[k - 1] * eps[c] * mu[c] + dz[k] * eps[ijkb] * mu[ijkb]) * indzm;
        double epsmu12 = (dz[k - 1] * eps[ijke] * mu[ijke] + dz[k] * eps[ijkeb] * mu[ijkeb]) * indzm;
        double epsmu1 = (dx[i + 1] * epsmu11 + dx[i] * epsmu12) * indxp;
        double gradxx = (eps[ijke] * txx2 * r[i + 1] - eps[c] * txx1 * r[i]);
        gradxx = gradxx * indxp * 2.0 * inrb[i];
        double gradyx = (epsmu2 * tyx2 - epsmu1 * tyx1);
        gradyx = gradyx * indz[k];
        visx[c] = gradxx + gradyx - eps0 * t0 * inrb[i];
        epsmu11 = (dz[k] * eps[ijkwt] * mu[ijkwt] + dz[k + 1] * eps[ijkw] * mu[ijkw]) * indzp;
        epsmu1 = (dx[i] * epsmu11 + dx[i - 1] * epsmu21) * indxm;
        double gradyy = (eps[ijkt] * tyy2 - eps[c] * tyy1);
        gradyy = gradyy * indzp * 2.0;
        double gradxy = (rb[i] * epsmu2 * txy2 - rb[i - 1] * epsmu1 * txy1);
        gradxy = gradxy * inr[i] * indx[i];
        visz[c] = gradyy + gradxy;
    }
}

// ---------------------------------------------------------------------------
// fieldn, tilde.f:125-274 (2D)
// ---------------------------------------------------------------------------
void fieldn(Oracle &o) {
    const auto &dx = o.dx, &dz = o.dz;
    for (int c = 0; c < o.ncell; ++c) {
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int ijke = o.nbrem(E, c), ijkt = o.nbrem(T, c);
        if (ijke >= 0 && ijkt >= 0) {
            double dxp = dx[i] + dx[i + 1], dzp = dz[k] + dz[k + 1];
            double indxp = 1.0 / dxp, indzp = 1.0 / dzp;
            double rgp_e = (dx[i + 1] * o.rgp[c] + dx[i] * o.rgp[ijke]) * indxp;
            double rgp_t = (dz[k + 1] * o.rgp[c] + dz[k] * o.rgp[ijkt]) * indzp;
            o.rugn[c] = rgp_e * o.ug[c];
            o.rwgn[c] = rgp_t * o.wg[c];
            for (int is = 1; is <= o.ns; ++is) {
                double rlk_e = (o.S(o.rlk, c, is) * dx[i + 1] + o.S(o.rlk, ijke, is) * dx[i]) * indxp;
                double rlk_t = (o.S(o.rlk, c, is) * dz[k + 1] + o.S(o.rlk, ijkt, is) * dz[k]) * indzp;
                o.S(o.rusn, c, is) = rlk_e * o.S(o.us, c, is);
                o.S(o.rwsn, c, is) = rlk_t * o.S(o.ws, c, is);
            }
        } else {
            // frame cells: the reference reads myinds = 0 here (out of
            // range); the values are never used, they are set to zero.
            o.rugn[c] = 0; o.rwgn[c] = 0;
            for (int is = 1; is <= o.ns; ++is) { o.S(o.rusn, c, is) = 0; o.S(o.rwsn, c, is) = 0; }
        }
        o.pn[c] = o.p[c];
        o.epn[c] = o.ep[c];
        o.rgpn[c] = o.rgp[c];
        o.siegn[c] = o.sieg[c];
        for (int ig = 1; ig <= o.ng; ++ig) o.S(o.rgpgcn, c, ig) = o.rgpn[c] * o.S(o.ygc, c, ig);
        for (int is = 1; is <= o.ns; ++is) {
            o.S(o.rlkn, c, is) = o.S(o.rlk, c, is);
            o.S(o.siesn, c, is) = o.S(o.sies, c, is);
        }
        double xg[PDAC_MAX_NGAS];
        for (int ig = 0; ig < o.ng; ++ig) xg[ig] = o.xgc[(size_t)ig * o.ncell + c];
        viscon(o, o.mug[c], o.kapg[c], xg, o.tg[c]);
    }
}

// inter, drag.f:173-246 (2D: appv slot unused); app arrays (ncell, nap)
void inter_2d(Oracle &o, int c, const double *kpgv, double dt) {
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    double au[64], aw[64];
    int ks = 0;
    double rlkc[PDAC_MAX_NSOLID + 1];
    for (int is = 1; is <= o.ns; ++is) rlkc[is] = o.S(o.rlk, c, is);
    for (int k = 1; k <= o.nph; ++k) {
        if (k == 1) { ks++; au[ks] = 0; aw[ks] = 0; }
        else {
            for (int kk = 1; kk <= k; ++kk) {
                ks++;
                if (kk == 1) { au[ks] = -kpgv[k - 1] * dt; aw[ks] = -kpgv[k - 1] * dt; }
                else if (kk == k) { au[ks] = 0; aw[ks] = 0; }
                else {
                    double con = ppdrag(o, rlkc, k, kk);
                    double du = std::fabs(o.S(o.us, c, k - 1) - o.S(o.us, c, kk - 1) + o.S(o.us, imjk, k - 1) - o.S(o.us, imjk, kk - 1)) * 0.5;
                    double dw = std::fabs(o.S(o.ws, c, k - 1) - o.S(o.ws, c, kk - 1) + o.S(o.ws, ijkm, k - 1) - o.S(o.ws, ijkm, kk - 1)) * 0.5;
                    au[ks] = -(con * du) * dt;
                    aw[ks] = -(con * dw) * dt;
                }
            }
        }
    }
    for (int k = 1; k <= o.nph; ++k) {
        double sx = 0, sz = 0;
        for (int kk = 1; kk <= k; ++kk) { int q = kk + k * (k - 1) / 2; sx = sx + au[q]; sz = sz + aw[q]; }
        for (int kk = k; kk <= o.nph; ++kk) { int q = k + kk * (kk - 1) / 2; sx = sx + au[q]; sz = sz + aw[q]; }
        int q = k * (k + 1) / 2;
        au[q] = -sx;
        aw[q] = -sz;
    }
    for (int q = 1; q <= o.nap; ++q) {
        o.appu[(size_t)(q - 1) * o.ncell + c] = au[q];
        o.appw[(size_t)(q - 1) * o.ncell + c] = aw[q];
    }
}

// viscs repulsive term, visc.f:247-287 (2D)
void repulsive_2d(Oracle &o) {
    const auto &dx = o.dx, &dz = o.dz;
    double a = -8.76, b = -0.27;
    for (int c = 0; c < o.ncell; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int ijke = o.nbrem(E, c), ijkt = o.nbrem(T, c);
        double dxp = (dx[i] + dx[i + 1]), dzp = (dz[k] + dz[k + 1]);
        double indxp = 1.0 / dxp, indzp = 1.0 / dzp;
        for (int is = 1; is <= o.ns; ++is) {
            double rc = o.S(o.rlk, c, is), re = o.S(o.rlk, ijke, is), rt = o.S(o.rlk, ijkt, is);
            double epsx = (dx[i + 1] * rc + dx[i] * re) * indxp * o.inrl[is];
            double gepx = pdac_fp::pow(10.0, -a * epsx + b);
            o.S(o.pvisx, c, is) = o.S(o.pvisx, c, is) - gepx * indxp * 2.0 * (re - rc) * o.inrl[is];
            double epsz = (dz[k + 1] * rc + dz[k] * rt) * indzp * o.inrl[is];
            double gepz = pdac_fp::pow(10.0, -a * epsz + b);
            o.S(o.pvisz, c, is) = o.S(o.pvisz, c, is) - gepz * indzp * 2.0 * (rt - rc) * o.inrl[is];
        }
    }
}

// tilde.f:276-848 with compute_all_fluxes_tilde tilde.f:850-1326 (2D)
void tilde_2d(Oracle &o, double dt) {
    const auto &dx = o.dx, &dz = o.dz, &indx = o.indx, &indz = o.indz, &inr = o.inr, &inrb = o.inrb;
    int n = o.ncell, ns = o.ns;
    std::fill(o.gvisx.begin(), o.gvisx.end(), 0.0);
    std::fill(o.gvisz.begin(), o.gvisz.end(), 0.0);
    std::fill(o.pvisx.begin(), o.pvisx.end(), 0.0);
    std::fill(o.pvisz.begin(), o.pvisz.end(), 0.0);
    if (o.cfg.gas_viscosity)  // viscg
        stress2d(o, o.gvisx.data(), o.gvisz.data(), viscg_mu(o), o.mug.data(), o.ep.data(), o.ug.data(), o.wg.data());
    if (o.cfg.part_viscosity) {
        vector<double> mus(n), must(n), rlkinrl(n);
        for (int is = 1; is <= ns; ++is) {
            viscs_mu(o, is, must);
            for (int c = 0; c < n; ++c) { mus[c] = o.cmus[is]; rlkinrl[c] = o.S(o.rlk, c, is) * o.inrl[is]; }
            stress2d(o, &o.pvisx[(size_t)(is - 1) * n], &o.pvisz[(size_t)(is - 1) * n], must.data(), mus.data(),
                     rlkinrl.data(), &o.us[(size_t)(is - 1) * n], &o.ws[(size_t)(is - 1) * n]);
        }
        if (o.cfg.repulsive_model == 1) repulsive_2d(o);
    }
    // convective fluxes (zeroed per call)
    std::fill(o.ugfe.begin(), o.ugfe.end(), 0.0); std::fill(o.ugft.begin(), o.ugft.end(), 0.0);
    std::fill(o.wgfe.begin(), o.wgfe.end(), 0.0); std::fill(o.wgft.begin(), o.wgft.end(), 0.0);
    std::fill(o.usfe.begin(), o.usfe.end(), 0.0); std::fill(o.usft.begin(), o.usft.end(), 0.0);
    std::fill(o.wsfe.begin(), o.wsfe.end(), 0.0); std::fill(o.wsft.begin(), o.wsft.end(), 0.0);
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        Sten u, w, dens;
        for (int ph = 0; ph <= ns; ++ph) {
            const double *U = ph == 0 ? o.ug.data() : &o.us[(size_t)(ph - 1) * n];
            const double *Wv = ph == 0 ? o.wg.data() : &o.ws[(size_t)(ph - 1) * n];
            const double *D = ph == 0 ? o.rgp.data() : &o.rlk[(size_t)(ph - 1) * n];
            double *fue = ph == 0 ? o.ugfe.data() : &o.usfe[(size_t)(ph - 1) * n];
            double *fut = ph == 0 ? o.ugft.data() : &o.usft[(size_t)(ph - 1) * n];
            double *fwe = ph == 0 ? o.wgfe.data() : &o.wsfe[(size_t)(ph - 1) * n];
            double *fwt = ph == 0 ? o.wgft.data() : &o.wsft[(size_t)(ph - 1) * n];
            rnb2(o, u, U, c);
            rnb2(o, w, Wv, c);
            ib_mask(o, u, c, 1);  // b_e_ (tilde.f:896-945)
            ib_mask(o, w, c, 4);  // b_t_
            nb2(o, dens, D, c);
            Sten dsx = interp_x2(o, dens, i);
            Sten dsz = interp_z2(o, dens, k);
            flu_2d(o, fue[c], fut[c], fue[imjk], fut[ijkm], dsx, u, w, i, c);
            flw_2d(o, fwe[c], fwt[c], fwe[imjk], fwt[ijkm], dsz, u, w, i, k, c);
            if (o.cfg.muscl > 0 && o.flag[c] == FLUID) {
                if (i != o.nx - 1) muscl_flu_2d(o, fue[c], fut[c], dsx, u, w, i, k);
                if (k != o.nz - 1) muscl_flw_2d(o, fwe[c], fwt[c], dsz, u, w, i, k);
            }
        }
    }
    // app: zeroed with the fluxes at the start of each step (allocate_fluxes)
    double alpha = o.cfg.alpha, ag = o.cfg.alphagrav;
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        int ijke = o.nbrem(E, c), ijkt = o.nbrem(T, c);
        double ugfx = o.ugfe[c] - o.ugfe[imjk], ugfz = o.ugft[c] - o.ugft[ijkm];
        double wgfx = o.wgfe[c] - o.wgfe[imjk], wgfz = o.wgft[c] - o.wgft[ijkm];
        double dxi = dx[i], dxip1 = dx[i + 1], dzk = dz[k], dzkp1 = dz[k + 1];
        double dxp = dx[i] + dx[i + 1], dzp = dz[k] + dz[k + 1];
        double indxp = 1.0 / dxp, indzp = 1.0 / dzp;
        double epn_e, epn_t;
        if (o.cfg.pmodel == 1) {
            epn_e = (dxi * o.epn[ijke] + dxip1 * o.epn[c]) * indxp;
            epn_t = (dzk * o.epn[ijkt] + dzkp1 * o.epn[c]) * indzp;
        } else { epn_e = 1.0; epn_t = 1.0; }
        double t_ = o.gvisx[c];
        t_ = t_ - indxp * 2.0 * ugfx * inrb[i];
        t_ = t_ + (1.0 - ag) * (dx[i + 1] * o.rgpn[c] + dx[i] * o.rgpn[ijke]) * indxp * o.cfg.gravx;
        t_ = t_ - indz[k] * ugfz;
        t_ = t_ + (1.0 - alpha) * indxp * 2.0 * epn_e * (o.pn[c] - o.pn[ijke]);
        o.rug[c] = o.rugn[c] + dt * t_;
        t_ = o.gvisz[c];
        t_ = t_ + (1.0 - ag) * (dz[k + 1] * o.rgpn[c] + dz[k] * o.rgpn[ijkt]) * indzp * o.cfg.gravz;
        t_ = t_ - indx[i] * wgfx * inr[i];
        t_ = t_ - indzp * 2.0 * wgfz;
        t_ = t_ + (1.0 - alpha) * indzp * 2.0 * epn_t * (o.pn[c] - o.pn[ijkt]);
        o.rwg[c] = o.rwgn[c] + dt * t_;
        double kpgv[PDAC_MAX_NSOLID + 1] = {0};
        double dugs_c[PDAC_MAX_NSOLID + 1] = {0}, dvgs_c[PDAC_MAX_NSOLID + 1] = {0}, dwgs_c[PDAC_MAX_NSOLID + 1] = {0};
        for (int is = 1; is <= ns; ++is) {
            double usfx = o.S(o.usfe, c, is) - o.S(o.usfe, imjk, is), usfz = o.S(o.usft, c, is) - o.S(o.usft, ijkm, is);
            double wsfx = o.S(o.wsfe, c, is) - o.S(o.wsfe, imjk, is), wsfz = o.S(o.wsft, c, is) - o.S(o.wsft, ijkm, is);
            double epsn_e, epsn_t;
            if (o.cfg.pmodel == 1) {
                epsn_e = (dxi * o.S(o.rlkn, ijke, is) + dxip1 * o.S(o.rlkn, c, is)) * indxp * o.inrl[is];
                epsn_t = (dzk * o.S(o.rlkn, ijkt, is) + dzkp1 * o.S(o.rlkn, c, is)) * indzp * o.inrl[is];
            } else { epsn_e = 0; epsn_t = 0; }
            double r_ = o.S(o.pvisx, c, is);
            r_ = r_ - indxp * 2.0 * usfx * inrb[i];
            r_ = r_ + (1.0 - ag) * indxp * o.cfg.gravx * (dx[i + 1] * o.S(o.rlkn, c, is) + dx[i] * o.S(o.rlkn, ijke, is));
            r_ = r_ - indz[k] * usfz;
            r_ = r_ + (1.0 - alpha) * indxp * 2.0 * epsn_e * (o.pn[c] - o.pn[ijke]);
            o.S(o.rus, c, is) = o.S(o.rusn, c, is) + dt * r_;
            o.S(o.rus, c, is) = o.S(o.rus, c, is) + dt * o.S(o.sink, c, is) * o.S(o.us, c, is);
            r_ = o.S(o.pvisz, c, is);
            r_ = r_ + (1.0 - ag) * indzp * o.cfg.gravz * (o.S(o.rlkn, c, is) * dz[k + 1] + o.S(o.rlkn, ijkt, is) * dz[k]);
            r_ = r_ - indx[i] * wsfx * inr[i];
            r_ = r_ - indzp * 2.0 * wsfz;
            r_ = r_ + (1.0 - alpha) * indzp * 2.0 * epsn_t * (o.pn[c] - o.pn[ijkt]);
            o.S(o.rws, c, is) = o.S(o.rwsn, c, is) + dt * r_;
            o.S(o.rws, c, is) = o.S(o.rws, c, is) + dt * o.S(o.sink, c, is) * o.S(o.ws, c, is);
            double dugs = ((o.ug[c] - o.S(o.us, c, is)) + (o.ug[imjk] - o.S(o.us, imjk, is))) * 0.5;
            double dwgs = ((o.wg[c] - o.S(o.ws, c, is)) + (o.wg[ijkm] - o.S(o.ws, ijkm, is))) * 0.5;
            if (o.cfg.drag_model == 1)
                kpgv[is] = kdrags(o, dugs, 0.0, dwgs, o.ep[c], o.rgp[c], o.S(o.rlk, c, is), o.mug[c], is);
            else
                kpgv[is] = sdrag(o, dugs, 0.0, dwgs, o.ep[c], o.rgp[c], o.S(o.rlk, c, is), o.mug[c], is);
            dugs_c[is] = dugs;
            dwgs_c[is] = dwgs;
        }
        inter_2d(o, c, kpgv, dt);
        // (1 - alpha) explicit interphase part, tilde.f:597-680; app of the
        // E/T neighbour is read before that cell has been visited in this
        // step, i.e. as left by the previous visit (zero at step start).
        auto APPU = [&](int cell, int ls) { return o.appu[(size_t)(ls - 1) * n + cell]; };
        auto APPW = [&](int cell, int ls) { return o.appw[(size_t)(ls - 1) * n + cell]; };
        o.rug[c] = o.rug[c] - (1.0 - alpha) * (dxi * APPU(ijke, 1) + dxip1 * APPU(c, 1)) * indxp * o.ug[c];
        o.rwg[c] = o.rwg[c] - (1.0 - alpha) * (dzk * APPW(ijkt, 1) + dzkp1 * APPW(c, 1)) * indzp * o.wg[c];
        for (int l = 2; l <= o.nph; ++l) {
            int ls1 = l * (l - 1) / 2;
            for (int ll = 1; ll <= l; ++ll) {
                int ls = ls1 + ll;
                double fu = (1.0 - alpha) * (dxi * APPU(ijke, ls) + dxip1 * APPU(c, ls)) * indxp;
                double fw = (1.0 - alpha) * (dzk * APPW(ijkt, ls) + dzkp1 * APPW(c, ls)) * indzp;
                if (ll == 1) {
                    o.rug[c] = o.rug[c] - fu * o.S(o.us, c, l - 1);
                    o.rwg[c] = o.rwg[c] - fw * o.S(o.ws, c, l - 1);
                    o.S(o.rus, c, l - 1) = o.S(o.rus, c, l - 1) - fu * o.ug[c];
                    o.S(o.rws, c, l - 1) = o.S(o.rws, c, l - 1) - fw * o.wg[c];
                } else if (ll == l) {
                    o.S(o.rus, c, l - 1) = o.S(o.rus, c, l - 1) - fu * o.S(o.us, c, l - 1);
                    o.S(o.rws, c, l - 1) = o.S(o.rws, c, l - 1) - fw * o.S(o.ws, c, l - 1);
                } else {
                    o.S(o.rus, c, l - 1) = o.S(o.rus, c, l - 1) - fu * o.S(o.us, c, ll - 1);
                    o.S(o.rus, c, ll - 1) = o.S(o.rus, c, ll - 1) - fu * o.S(o.us, c, l - 1);
                    o.S(o.rws, c, l - 1) = o.S(o.rws, c, l - 1) - fw * o.S(o.ws, c, ll - 1);
                    o.S(o.rws, c, ll - 1) = o.S(o.rws, c, ll - 1) - fw * o.S(o.ws, c, l - 1);
                }
            }
        }
        ib_tilde_forcing(o, c, dt, kpgv, dugs_c, dvgs_c, dwgs_c);  // tilde.f:708-801
    }
}

// ---------------------------------------------------------------------------
// iter.f:38-1248 (2D)
// ---------------------------------------------------------------------------
// opt_inner_loop's density stencils (iter.f:1330-1360): built at loop entry,
// only the centre updated, so slots remapped to the cell hold its
// loop-entry value v
void stale_first2(const Oracle &o, Sten &s, int c, double v) {
    if (o.nbrem(E, c) == c) s.e = v;
    if (o.nbrem(T, c) == c) s.t = v;
    if (o.nbrem(W, c) == c) s.w = v;
    if (o.nbrem(B, c) == c) s.b = v;
}
void stale_third2(const Oracle &o, Sten &s, int c, double v) {
    if (o.nbrem(EE, c) == c) s.ee = v;
    if (o.nbrem(TT, c) == c) s.tt = v;
    if (o.nbrem(WW, c) == c) s.ww = v;
    if (o.nbrem(BB, c) == c) s.bb = v;
}

void calc_gas_mass_flux_2d(Oracle &o, int c, const double *own0 = nullptr) {
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    Sten dens, u, w;
    first_nb2(o, dens, o.rgp.data(), c);
    if (own0) stale_first2(o, dens, c, *own0);
    first_rnb2(o, u, o.ug.data(), c);
    first_rnb2(o, w, o.wg.data(), c);
    masf_2d(o, o.rgfe[c], o.rgft[c], o.rgfe[imjk], o.rgft[ijkm], dens, u, w, i);
    if (o.cfg.muscl > 0 && o.flag[c] == FLUID) {
        third_nb2(o, dens, o.rgp.data(), c);
        if (own0) stale_third2(o, dens, c, *own0);
        fmas_2d(o, o.rgfe[c], o.rgft[c], o.rgfe[imjk], o.rgft[ijkm], dens, u, w, c);
    }
}

void calc_part_mass_flux_2d(Oracle &o, int c, const double *own0 = nullptr) {
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int n = o.ncell;
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    for (int is = 1; is <= o.ns; ++is) {
        Sten dens, u, w;
        const double *R = &o.rlk[(size_t)(is - 1) * n];
        first_nb2(o, dens, R, c);
        if (own0) stale_first2(o, dens, c, own0[is]);
        first_rnb2(o, u, &o.us[(size_t)(is - 1) * n], c);
        first_rnb2(o, w, &o.ws[(size_t)(is - 1) * n], c);
        double *fe = &o.rsfe[(size_t)(is - 1) * n], *ft = &o.rsft[(size_t)(is - 1) * n];
        masf_2d(o, fe[c], ft[c], fe[imjk], ft[ijkm], dens, u, w, i);
        if (o.cfg.muscl > 0 && o.flag[c] == FLUID) {
            third_nb2(o, dens, R, c);
            if (own0) stale_third2(o, dens, c, own0[is]);
            fmas_2d(o, fe[c], ft[c], fe[imjk], ft[ijkm], dens, u, w, c);
        }
    }
}

double calc_res_2d(Oracle &o, int c, double dt) {
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    const CellFaces b = cell_faces(o, c);
    double resx = (b.e * o.rgfe[c] - b.w * o.rgfe[imjk]) * o.indx[i] * o.inr[i];
    double resz = (b.t * o.rgft[c] - b.b * o.rgft[ijkm]) * o.indz[k];
    double resy = 0.0;
    return o.rgp[c] - o.rgpn[c] + dt * b.ivf * (resx + resy + resz);
}

void calc_eps_2d(Oracle &o, int c, double dt) {
    int i, j, k;
    o.ijk_of(c, i, j, k);
    int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
    const CellFaces b = cell_faces(o, c);
    double rls = 0;
    for (int is = 1; is <= o.ns; ++is) {
        double rlkx = (b.e * o.S(o.rsfe, c, is) - b.w * o.S(o.rsfe, imjk, is)) * o.indx[i] * o.inr[i];
        double rlkz = (b.t * o.S(o.rsft, c, is) - b.b * o.S(o.rsft, ijkm, is)) * o.indz[k];
        double rlky = 0.0;
        double t = o.S(o.rlkn, c, is) - dt * b.ivf * (rlkx + rlky + rlkz);
        t = t + dt * b.ivf * o.S(o.sink, c, is);
        o.S(o.rlk, c, is) = std::max(0.0, t);
        rls = rls + o.S(o.rlk, c, is) * o.inrl[is];
    }
    o.ep[c] = 1.0 - rls;
    if (rls > 1.0) o.ierr++;
}

// padjust's SAVE variables (iter.f:1005).  The reference keeps one copy per
// process; here each thread keeps its own, so that cells of one colour can
// run on several threads.  The values a cell reads are always the ones that
// cell wrote: kros starts at -1 in every cell, the secant (kros = 2) needs
// both sides set in that cell, and newp (kros = 3) follows it.
struct PadjustSave {
    double pa_dp = 0, pa_d1 = 0, pa_d2 = 0, pa_p1 = 0, pa_p2 = 0, pa_d12 = 0;
};
thread_local PadjustSave g_padjust_save;

// iter.f:997-1072
void padjust(Oracle &, double &p, int &kros, double d3, double &p3, double omega, double &abeta) {
    PadjustSave &o = g_padjust_save;
    if (kros != 3) {
        if (d3 > 0.0) {
            o.pa_d1 = d3; o.pa_p1 = p3;
            if (kros == -1) kros = 0;
            else if (kros == 1) kros = 2;
        } else if (d3 <= 0.0) {
            o.pa_d2 = d3; o.pa_p2 = p3;
            if (kros == -1) kros = 1;
            else if (kros == 0) kros = 2;
        }
        if (kros == 2) {
            o.pa_d12 = 1.0 / (o.pa_d1 - o.pa_d2);
            p = (o.pa_d1 * o.pa_p2 - o.pa_d2 * o.pa_p1) * o.pa_d12;
            abeta = (o.pa_p1 - o.pa_p2) * o.pa_d12;
            kros = 3;
        } else if (kros < 2) {
            o.pa_dp = -d3 * abeta;
            o.pa_dp = o.pa_dp * omega;
            double sg = std::copysign(1.0, d3);
            if (-o.pa_dp * sg > 2.5e-1 * p3) o.pa_dp = -2.5e-1 * sg * p3;
            p = p + o.pa_dp;
        }
    } else if (kros == 3) {
        // newp, iter.f:1075-1109
        double d1 = o.pa_d1, d2 = o.pa_d2, p1 = o.pa_p1, p2 = o.pa_p2, pa = 0, pb = 0;
        if (d1 != d3) pa = (d1 * p3 - d3 * p1) / (d1 - d3);
        if (d1 * d3 <= 0.0) {
            if (d2 != d3) pb = (d2 * p3 - d3 * p2) / (d2 - d3);
            else pb = 0.5 * (p1 + p3);
            if (pb < p3 || pb > p1) pb = 0.5 * (p1 + p3);
        } else {
            if (d1 == d3) pa = 0.5 * (p2 + p3);
            if (pa < p2 || pa > p3) pa = 0.5 * (p2 + p3);
            pb = (d2 * p3 - d3 * p2) / (d2 - d3);
        }
        p = 0.5 * (pa + pb);
        if (d3 > 0.0) { o.pa_d1 = d3; o.pa_p1 = p3; }
        else { o.pa_d2 = d3; o.pa_p2 = p3; }
    }
    p3 = p;
}

void betas_2d(Oracle &o, int c, double dt, double &cnv, double &abt) {
    const auto &dx = o.dx, &dz = o.dz;
    int i, j, k;
    o.ijk_of(c, i, j, k);
    double dxp = dx[i] + dx[i + 1], dxm = dx[i] + dx[i - 1], dzp = dz[k] + dz[k + 1], dzm = dz[k] + dz[k - 1];
    double indxp = 1.0 / dxp, indxm = 1.0 / dxm, indzp = 1.0 / dzp, indzm = 1.0 / dzm;
    auto open = [](int f) { return f == BL_CELL || f == FLUID || f == DOME || f == IMMB || f == FREE_IO || f == ZERO_GRAD; };
    int ijke = o.nbrem(E, c), ijkw = o.nbrem(W, c), ijkt = o.nbrem(T, c), ijkb = o.nbrem(B, c);
    double iep_e = open(o.flag[o.nbraw(E, c)]) ? (dx[i + 1] * o.ep[c] + dx[i] * o.ep[ijke]) * indxp * indxp * 2.0 : 0.0;
    double iep_w = open(o.flag[o.nbraw(W, c)]) ? (dx[i - 1] * o.ep[c] + dx[i] * o.ep[ijkw]) * indxm * indxm * 2.0 : 0.0;
    double iep_t = open(o.flag[o.nbraw(T, c)]) ? (dz[k + 1] * o.ep[c] + dz[k] * o.ep[ijkt]) * indzp * indzp * 2.0 : 0.0;
    double iep_b = open(o.flag[o.nbraw(B, c)]) ? (dz[k - 1] * o.ep[c] + dz[k] * o.ep[ijkb]) * indzm * indzm * 2.0 : 0.0;
    double iepx = (o.rb[i] * iep_e + o.rb[i - 1] * iep_w) * o.indx[i] * o.inr[i];
    double iepz = (iep_t + iep_b) * o.indz[k];
    double iepy = 0.0;
    double sqc = o.gammaair * o.p[c] / o.rog[c];
    double rbeta = o.ep[c] / sqc;
    rbeta = rbeta + dt * dt * (iepx + iepy + iepz);
    abt = 1.0 / rbeta;
    cnv = o.cfg.delg * o.rgp[c];
}

void inner_loop_2d(Oracle &o, int c, int nit, double &d3, double &p3, double &abeta_, double conv_, double &dgorig, double dt) {
    int kros = -1;
    double xg[PDAC_MAX_NGAS];
    for (int ig = 0; ig < o.ng; ++ig) xg[ig] = o.xgc[(size_t)ig * o.ncell + c];
    // optimization >= 2: opt_inner_loop (iter.f:1255-1547)
    const bool opt = o.cfg.optimization >= 2;
    double own0[PDAC_MAX_NSOLID + 1];
    own0[0] = o.rgp[c];
    for (int is = 1; is <= o.ns; ++is) own0[is] = o.S(o.rlk, c, is);
    for (int loop = 1; loop <= o.cfg.inmax; ++loop) {
        if (loop > 1 || nit > 1) padjust(o, o.p[c], kros, d3, p3, o.cfg.omega, abeta_);
        o.rog[c] = thermal_eosg(o, o.tg[c], o.p[c], xg);
        o.rgp[c] = o.ep[c] * o.rog[c];
        Mat au1{}, aw1{}, au{}, aw{};
        double bu1[PDAC_MAX_NSOLID + 2]{}, bw1[PDAC_MAX_NSOLID + 2]{}, bu[PDAC_MAX_NSOLID + 2]{}, bw[PDAC_MAX_NSOLID + 2]{};
        assemble_wb_2d(o, c, dt, au1, bu1, aw1, bw1);
        assemble_et_2d(o, c, dt, au, bu, aw, bw);
        solve_all_2d(o, c, au1, bu1, aw1, bw1, au, bu, aw, bw);
        calc_part_mass_flux_2d(o, c, opt ? own0 : nullptr);
        calc_eps_2d(o, c, dt);
        o.rgp[c] = o.ep[c] * o.rog[c];
        calc_gas_mass_flux_2d(o, c, opt ? own0 : nullptr);
        double dg = calc_res_2d(o, c, dt);
        if (std::fabs(dg) > conv_ || std::fabs(dg) >= std::fabs(dgorig)) {
            if (nit == 1 && loop == 1) dgorig = dg;
            d3 = dg;
        } else if (std::fabs(dg) <= conv_) {
            break;
        }
    }
}

void htilde_2d(Oracle &o, double dt);
int ftem_2d(Oracle &o, double dt);

// allocate_fluxes (tilde.f:56-102, prog.f:229): the tilde momenta,
// interphase terms and enthalpy right-hand sides start every RK stage at
// zero; with implicit_fluxes iter's predictor reads those zeros
void zero_tilde_terms(Oracle &o) {
    for (auto *v : {&o.rug, &o.rvg, &o.rwg, &o.rus, &o.rvs, &o.rws, &o.appu, &o.appv, &o.appw, &o.rhg, &o.rhs})
        std::fill(v->begin(), v->end(), 0.0);
}

int iter_2d(Oracle &o, double dt, int *nit_out) {
    int n = o.ncell;
    if (o.cfg.implicit_fluxes) zero_tilde_terms(o);
    bool eos = false;
    std::fill(o.rgfe.begin(), o.rgfe.end(), 0.0); std::fill(o.rgft.begin(), o.rgft.end(), 0.0);
    std::fill(o.rsfe.begin(), o.rsfe.end(), 0.0); std::fill(o.rsft.begin(), o.rsft.end(), 0.0);
    std::fill(o.conv.begin(), o.conv.end(), 0.0); std::fill(o.abeta.begin(), o.abeta.end(), 0.0);
    // predictor, iter.f:135-145
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        Mat au{}, aw{};
        double bu[PDAC_MAX_NSOLID + 2]{}, bw[PDAC_MAX_NSOLID + 2]{};
        assemble_et_2d(o, c, dt, au, bu, aw, bw);
        solve_et_2d(o, c, au, bu, aw, bw);
    }
    // initial gas mass fluxes and betas, iter.f:170-191
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        calc_gas_mass_flux_2d(o, c);
        betas_2d(o, c, dt, o.conv[c], o.abeta[c]);
    }
    // cell visit order of the corrector
    vector<int> order;
    if (o.order == 1) {
        for (int c = 0; c < n; ++c) order.push_back(c);
    } else {
        for (int col = 0; col < 3; ++col)
            for (int c = 0; c < n; ++c) {
                int i, j, k;
                o.ijk_of(c, i, j, k);
                if ((i + j + k) % 3 == col) order.push_back(c);
            }
    }
    int nit;
    for (nit = 1; nit <= o.cfg.maxout; ++nit) {
        o.ierr = 0;
        o.unconv.clear();
        if (o.cfg.implicit_fluxes) tilde_2d(o, dt);  // iter.f:211-226
        bool all = true;
        for (int c : order) {
            if (!o.fluidbit(c)) continue;
            double dg = calc_res_2d(o, c, dt);
            double dgorig = dg;
            o.dgres[c] = std::fabs(dg) / o.conv[c];
            if (std::fabs(dg) <= o.conv[c]) {
                calc_eps_2d(o, c, dt);
                o.rgp[c] = o.ep[c] * o.rog[c];
            } else {
                all = false;
                o.unconv.push_back(c);
                double d3 = dg, p3 = o.p[c];
                inner_loop_2d(o, c, nit, d3, p3, o.abeta[c], o.conv[c], dgorig, dt);
            }
        }
        if (o.cfg.implicit_enthalpy) {  // iter.f:362-379
            if (o.cfg.implicit_fluxes) htilde_2d(o, dt);
            if (ftem_2d(o, dt) != PDAC_OK) eos = true;
        }
        if (all) break;
    }
    o.last_nit = nit;
    if (nit_out) *nit_out = nit;
    if (eos) return PDAC_ERR_EOS;
    return nit > o.cfg.maxout && o.cfg.cstop ? PDAC_ERR_MAXOUT : PDAC_OK;  // iter.f:449
}

// ---------------------------------------------------------------------------
// ygas.f:27-325 (2D)
// ---------------------------------------------------------------------------
void ygas_2d(Oracle &o, double dt) {
    int n = o.ncell, ng = o.ng;
    if (ng == 1) {
        for (int c = 0; c < n; ++c) { o.ygc[c] = 1.0; o.xgc[c] = 1.0; }
        return;
    }
    o.yfe.assign((size_t)n * ng, 0.0);
    o.yft.assign((size_t)n * ng, 0.0);
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        for (int ig = 1; ig <= ng; ++ig) {
            Sten dens, conc, u, w;
            const double *Y = &o.ygc[(size_t)(ig - 1) * n];
            first_nb2(o, dens, o.rgp.data(), c);
            first_nb2(o, conc, Y, c);
            first_rnb2(o, u, o.ug.data(), c);
            first_rnb2(o, w, o.wg.data(), c);
            double *fe = &o.yfe[(size_t)(ig - 1) * n], *ft = &o.yft[(size_t)(ig - 1) * n];
            fsc_2d(o, fe[c], ft[c], fe[imjk], ft[ijkm], dens, conc, u, w, c);
            if (o.cfg.muscl > 0 && o.flag[c] == FLUID) {
                third_nb2(o, dens, o.rgp.data(), c);
                third_nb2(o, conc, Y, c);
                muscl_fsc_2d(o, fe[c], ft[c], dens, conc, u, w, c);
            }
        }
    }
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        const CellFaces b = cell_faces(o, c);
        double rgpgc[PDAC_MAX_NGAS + 1], rgpt = 0, yfy = 0;
        for (int ig = 1; ig <= ng; ++ig) {
            double yfw = o.S(o.yfe, imjk, ig), yfb = o.S(o.yft, ijkm, ig);
            double yfx = b.e * o.S(o.yfe, c, ig) - b.w * yfw;
            double yfz = b.t * o.S(o.yft, c, ig) - b.b * yfb;
            rgpgc[ig] = o.S(o.rgpgcn, c, ig);
            rgpgc[ig] = rgpgc[ig] - b.ivf * dt * o.indx[i] * yfx * o.inr[i];
            rgpgc[ig] = rgpgc[ig] - b.ivf * dt * 0.0 * yfy;
            rgpgc[ig] = rgpgc[ig] - b.ivf * dt * o.indz[k] * yfz;
            if (rgpgc[ig] < 0.0) rgpgc[ig] = 0.0;
            rgpt = rgpt + rgpgc[ig];
        }
        double rgpinv = 1.0 / rgpt, ygcdfg = 1.0;
        for (int ig = 1; ig <= ng - 1; ++ig) {
            o.S(o.ygc, c, ig) = rgpgc[ig] * rgpinv;
            ygcdfg = ygcdfg - o.S(o.ygc, c, ig);
        }
        o.S(o.ygc, c, ng) = ygcdfg;
        double yg[PDAC_MAX_NGAS], xg[PDAC_MAX_NGAS];
        for (int ig = 0; ig < ng; ++ig) yg[ig] = o.ygc[(size_t)ig * n + c];
        mole(o, xg, yg);
        for (int ig = 0; ig < ng; ++ig) o.xgc[(size_t)ig * n + c] = xg[ig];
    }
}

// ---------------------------------------------------------------------------
// htilde.f:25-575 (2D)
// ---------------------------------------------------------------------------
void htilde_2d(Oracle &o, double dt) {
    int n = o.ncell, ns = o.ns;
    const double *kapgt = flux_kapgt(o);
    o.egfe.assign(n, 0.0); o.egft.assign(n, 0.0); o.hgfe.assign(n, 0.0); o.hgft.assign(n, 0.0);
    o.esfe.assign((size_t)n * ns, 0.0); o.esft.assign((size_t)n * ns, 0.0);
    o.hsfe.assign((size_t)n * ns, 0.0); o.hsft.assign((size_t)n * ns, 0.0);
    const double gx = o.cfg.gravx, gz = o.cfg.gravz;
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        Sten enth, dens, u, w;
        first_nb2(o, enth, o.sieg.data(), c);
        first_nb2(o, dens, o.rgp.data(), c);
        first_rnb2(o, u, o.ug.data(), c);
        first_rnb2(o, w, o.wg.data(), c);
        fsc_2d(o, o.egfe[c], o.egft[c], o.egfe[imjk], o.egft[ijkm], enth, dens, u, w, c);
        if (o.cfg.muscl > 0 && o.flag[c] == FLUID) {
            third_nb2(o, enth, o.sieg.data(), c);
            third_nb2(o, dens, o.rgp.data(), c);
            muscl_fsc_2d(o, o.egfe[c], o.egft[c], enth, dens, u, w, c);
        }
        if (o.cfg.gas_viscosity) {
            Sten kappa, eps, temp;
            first_nb2(o, kappa, kapgt, c);
            first_nb2(o, eps, o.ep.data(), c);
            first_nb2(o, temp, o.tg.data(), c);
            hotc_2d(o, o.hgfe[c], o.hgft[c], o.hgfe[imjk], o.hgft[ijkm], eps, temp, kappa, c);
        }
        o.egfe[c] = o.egfe[c] - o.hgfe[c] + o.rgp[c] * gx * o.ug[c];
        o.egft[c] = o.egft[c] - o.hgft[c] + o.rgp[c] * gz * o.wg[c];
        if (!o.fluidbit(imjk)) o.egfe[imjk] = o.egfe[imjk] - o.hgfe[imjk];
        if (!o.fluidbit(ijkm)) o.egft[ijkm] = o.egft[ijkm] - o.hgft[ijkm];
        for (int is = 1; is <= ns; ++is) {
            const double *SI = &o.sies[(size_t)(is - 1) * n], *RL = &o.rlk[(size_t)(is - 1) * n];
            double *fe = &o.esfe[(size_t)(is - 1) * n], *ft = &o.esft[(size_t)(is - 1) * n];
            double *he = &o.hsfe[(size_t)(is - 1) * n], *ht = &o.hsft[(size_t)(is - 1) * n];
            Sten en2, de2, u2, w2;
            first_nb2(o, en2, SI, c);
            first_nb2(o, de2, RL, c);
            first_rnb2(o, u2, &o.us[(size_t)(is - 1) * n], c);
            first_rnb2(o, w2, &o.ws[(size_t)(is - 1) * n], c);
            fsc_2d(o, fe[c], ft[c], fe[imjk], ft[ijkm], en2, de2, u2, w2, c);
            if (o.cfg.muscl > 0 && o.flag[c] == FLUID) {
                third_nb2(o, en2, SI, c);
                third_nb2(o, de2, RL, c);
                muscl_fsc_2d(o, fe[c], ft[c], en2, de2, u2, w2, c);
            }
            if (o.cfg.part_viscosity) {
                Sten eps = scale(de2, o.inrl[is]);
                Sten kappa = cte(o.kap[is]);
                Sten temp;
                first_nb2(o, temp, &o.ts[(size_t)(is - 1) * n], c);
                hotc_2d(o, he[c], ht[c], he[imjk], ht[ijkm], eps, temp, kappa, c);
            }
            fe[c] = fe[c] - he[c] + RL[c] * gx * o.S(o.us, c, is);
            ft[c] = ft[c] - ht[c] + RL[c] * gz * o.S(o.ws, c, is);
            if (!o.fluidbit(imjk)) fe[imjk] = fe[imjk] - he[imjk];
            if (!o.fluidbit(ijkm)) ft[ijkm] = ft[ijkm] - ht[ijkm];
        }
    }
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        const CellFaces b = cell_faces(o, c);
        double egfx = b.e * o.egfe[c] - b.w * o.egfe[imjk];
        double egfz = b.t * o.egft[c] - b.b * o.egft[ijkm];
        double egfy = 0.0;
        double flx = dt * o.indx[i] * egfx * o.inr[i] + dt * 0.0 * egfy + dt * o.indz[k] * egfz;
        flx = flx * b.ivf;
        o.rhg[c] = -flx;
        for (int is = 1; is <= ns; ++is) {
            double esfx, esfz;
            if (o.S(o.rlk, imjk, is) * o.inrl[is] <= 1.0e-9) esfx = b.e * o.S(o.esfe, c, is);
            else esfx = b.e * o.S(o.esfe, c, is) - b.w * o.S(o.esfe, imjk, is);
            if (o.S(o.rlk, ijkm, is) * o.inrl[is] <= 1.0e-9) esfz = b.t * o.S(o.esft, c, is);
            else esfz = b.t * o.S(o.esft, c, is) - b.b * o.S(o.esft, ijkm, is);
            double esfy = 0.0;
            flx = dt * o.indx[i] * esfx * o.inr[i] + dt * 0.0 * esfy + dt * o.indz[k] * esfz;
            flx = flx * b.ivf;
            o.S(o.rhs, c, is) = -flx + o.S(o.sink, c, is) * dt * b.ivf * o.S(o.sies, c, is);
        }
    }
}

// ---------------------------------------------------------------------------
// ftem.f:19-248 (2D)
// ---------------------------------------------------------------------------
int ftem_2d(Oracle &o, double dt) {
    const auto &dx = o.dx, &dz = o.dz;
    int n = o.ncell, ns = o.ns, nph = o.nph, num = 0;
    double alpha = o.cfg.alpha;
    for (int c = 0; c < n; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        int imjk = o.nbraw(W, c), ijkm = o.nbraw(B, c);
        int ijke = o.nbrem(E, c), ijkw = o.nbrem(W, c), ijkt = o.nbrem(T, c), ijkb = o.nbrem(B, c);
        double indxc = 1.0 / (dx[i] + (dx[i + 1] + dx[i - 1]) * 0.5);
        double indzc = 1.0 / (dz[k] + (dz[k + 1] + dz[k - 1]) * 0.5);
        const CellFaces bf = cell_faces(o, c);
        double ugc = 0.5 * (bf.e * o.ug[c] + bf.w * o.ug[imjk]);
        double wgc = 0.5 * (bf.t * o.wg[c] + bf.b * o.wg[ijkm]);
        double dpxyz = 0.0;
        dpxyz = dpxyz + dt * indxc * ugc * (o.p[ijke] - o.p[ijkw]);
        dpxyz = dpxyz + dt * 0.0 * 0.0 * 0.0;
        dpxyz = dpxyz + dt * indzc * wgc * (o.p[ijkt] - o.p[ijkb]);
        double deltap = o.ep[c] * (o.p[c] - o.pn[c] + dpxyz);
        double workg = o.rgp[c] * (o.ug[c] * o.cfg.gravx + o.wg[c] * o.cfg.gravz);
        double at[PDAC_MAX_NSOLID + 2][PDAC_MAX_NSOLID + 2] = {{0}}, bt[PDAC_MAX_NSOLID + 2] = {0};
        at[1][1] = o.rgp[c];
        bt[1] = o.siegn[c] * o.rgpn[c] + o.rhg[c] + deltap + workg - 0.0;
        for (int is = 1; is <= ns; ++is) {
            int is1 = is + 1;
            double dugs = ((o.ug[c] - o.S(o.us, c, is)) + (o.ug[imjk] - o.S(o.us, imjk, is))) * 0.5;
            double dwgs = ((o.wg[c] - o.S(o.ws, c, is)) + (o.wg[ijkm] - o.S(o.ws, ijkm, is))) * 0.5;
            double hv = hvs(o, o.S(o.rlk, c, is), o.rog[c], o.ep[c], dugs, 0.0, dwgs, o.mug[c], o.kapg[c], o.cg[c], is);
            double works = o.S(o.rlk, c, is) * (o.S(o.us, c, is) * o.cfg.gravx + o.S(o.ws, c, is) * o.cfg.gravz);
            double ck = o.cps[is];
            at[1][1] = at[1][1] + alpha * dt * hv / o.cg[c];
            at[1][is1] = -alpha * dt * hv / ck;
            at[is1][1] = -alpha * dt * hv / o.cg[c];
            at[is1][is1] = o.S(o.rlk, c, is) + alpha * dt * hv / ck;
            bt[1] = bt[1] + (1.0 - alpha) * dt * hv * o.S(o.ts, c, is) - (1.0 - alpha) * dt * hv * o.tg[c];
            bt[is1] = o.S(o.rlkn, c, is) * o.S(o.siesn, c, is) + o.S(o.rhs, c, is) + works +
                      (1.0 - alpha) * dt * hv * o.tg[c] - (1.0 - alpha) * dt * hv * o.S(o.ts, c, is);
        }
        // invdm, ftem.f:201-248
        for (int is = nph; is >= 2; --is) {
            if (std::fabs(at[is][is]) < o.cfg.flim) {
                at[1][is] = 0.0; at[is][1] = 0.0; bt[is] = 0.0;
            } else {
                double div = 1.0 / at[is][is];
                at[is][1] = at[is][1] * div;
                bt[is] = bt[is] * div;
                bt[1] = bt[1] - at[1][is] * bt[is];
                at[1][1] = at[1][1] - at[1][is] * at[is][1];
            }
        }
        bt[1] = bt[1] / at[1][1];
        for (int is = 2; is <= nph; ++is) bt[is] = bt[is] - at[is][1] * bt[1];
        o.sieg[c] = bt[1];
        for (int is = 1; is <= ns; ++is) o.S(o.sies, c, is) = bt[is + 1];
        double yg[PDAC_MAX_NGAS];
        for (int ig = 0; ig < o.ng; ++ig) yg[ig] = o.ygc[(size_t)ig * n + c];
        int info = caloric_eosg(o, o.cg[c], o.tg[c], yg, o.sieg[c]);
        for (int is = 1; is <= ns; ++is) {
            double ck = o.cps[is];
            o.S(o.ts, c, is) = o.tzero + (o.S(o.sies, c, is) - o.hzeros) / ck;
            if (o.S(o.ts, c, is) < 0.0) info++;
        }
        num += info;
    }
    o.eos_fail = num;
    return num > 1 ? PDAC_ERR_EOS : PDAC_OK;
}

// ---------------------------------------------------------------------------
// boundary, bdry.f:22-726 with inoutflow.f:1-126 (2D)
// ---------------------------------------------------------------------------
void inoutflow(Oracle &o, double ugv, const double *usv, int n2, int n1, int k, double gnorm) {
    int n = o.ncell;
    int sgn = (n2 - n1) >= 0 ? 1 : -1;
    if (ugv * sgn > 0.0) {
        o.tg[n2] = o.tg[n1];
        o.sieg[n2] = o.sieg[n1];
        for (int ig = 0; ig < o.ng; ++ig) {
            o.ygc[(size_t)ig * n + n2] = o.ygc[(size_t)ig * n + n1];
            o.xgc[(size_t)ig * n + n2] = o.xgc[(size_t)ig * n + n1];
        }
        o.rog[n2] = o.rog[n1];
    } else if (ugv * sgn <= 0.0) {
        o.tg[n2] = o.t_atm[k];
        double yg[PDAC_MAX_NGAS], xg[PDAC_MAX_NGAS];
        for (int ig = 0; ig < o.ng; ++ig) { yg[ig] = o.cfg.atm_ygc[o.gas_type[ig] - 1]; o.ygc[(size_t)ig * n + n2] = yg[ig]; }
        mole(o, xg, yg);
        for (int ig = 0; ig < o.ng; ++ig) o.xgc[(size_t)ig * n + n2] = xg[ig];
        o.rog[n2] = thermal_eosg(o, o.t_atm[k], o.p_atm[k], xg);
    }
    double rls = 0.0;
    for (int is = 1; is <= o.ns; ++is) {
        if (usv[is] * sgn > 0.0) {
            o.S(o.rlk, n2, is) = o.S(o.rlk, n1, is);
            o.S(o.ts, n2, is) = o.S(o.ts, n1, is);
            o.S(o.sies, n2, is) = o.S(o.sies, n1, is);
        } else if (usv[is] * sgn <= 0.0) {
            o.S(o.rlk, n2, is) = o.rl[is] * (1.0 - o.cfg.void_fraction) / o.ns;
            o.S(o.ts, n2, is) = o.t_atm[k];
        }
        rls = rls + o.S(o.rlk, n2, is) * o.inrl[is];
    }
    o.ep[n2] = 1.0 - rls;
    o.rgp[n2] = o.rog[n2] * o.ep[n2];
    double rhomix;
    if (o.cfg.pmodel == 1) {
        rhomix = o.rgp[n2];
        for (int is = 1; is <= o.ns; ++is) rhomix = rhomix + o.S(o.rlk, n2, is);
    } else {
        rhomix = o.rgp[n2];
    }
    if (rls >= 1.0) o.err = "bdry: control transport on boundary";
    o.p[n2] = o.p[n1] + rhomix * gnorm;
}

void zerograd(Oracle &o, int n2, int n1) {
    int n = o.ncell;
    o.tg[n2] = o.tg[n1];
    o.sieg[n2] = o.sieg[n1];
    for (int ig = 0; ig < o.ng; ++ig) {
        o.ygc[(size_t)ig * n + n2] = o.ygc[(size_t)ig * n + n1];
        o.xgc[(size_t)ig * n + n2] = o.xgc[(size_t)ig * n + n1];
    }
    o.rog[n2] = o.rog[n1];
    double rls = 0.0;
    for (int is = 1; is <= o.ns; ++is) {
        o.S(o.rlk, n2, is) = o.S(o.rlk, n1, is);
        o.S(o.ts, n2, is) = o.S(o.ts, n1, is);
        o.S(o.sies, n2, is) = o.S(o.sies, n1, is);
        rls = rls + o.S(o.rlk, n2, is) * o.inrl[is];
    }
    o.ep[n2] = 1.0 - rls;
    o.rgp[n2] = o.rog[n2] * o.ep[n2];
    if (rls >= 1.0) o.err = "bdry: control transport on boundary";
    o.p[n2] = o.p[n1];
}

// ---------------------------------------------------------------------------
// ground sink, sink.f:22-121
// ---------------------------------------------------------------------------
// allocate_sink (sink.f:22-43) and the cell-centre coordinates (grid.f:286-298)
void sink_setup(Oracle &o) {
    int ntr = o.d3 ? o.nx * o.ny : o.nx;
    o.massl.assign((size_t)ntr * o.ns, 0.0);
    o.mass_loss.assign((size_t)ntr * o.ns, 0.0);
    o.xc.assign(o.nx + 1, 0.0);
    o.yc.assign(o.ny + 1, 0.0);
    double xb = 0.0;
    o.xc[1] = -0.5 * o.dx[1] + xb;
    for (int i = 2; i <= o.nx; ++i) {
        xb = (xb + o.dx[i]);
        o.xc[i] = (xb - 0.5 * o.dx[i]);
    }
    double yb = 0.0;
    o.yc[1] = -0.5 * o.dy[1] + yb;  // dy = 0 in 2D: y(1) = 0
    for (int j = 2; j <= o.ny; ++j) {
        yb = yb + o.dy[j];
        o.yc[j] = (yb - 0.5 * o.dy[j]);
    }
}

// sink_update (sink.f:46-121) of fluid cell c above a wall or filled cell:
// the downward flux rlk min(0, ws) / dz of the cell centre inside the ring
// rprox < r < rdist, and its mass over the step into the column's massl
void sink_update(Oracle &o, int c, int is) {
    int i, j, k;
    o.ijk_of(c, i, j, k);
    double rsft_up = o.S(o.rlk, c, is);
    double wst = std::min(0.0, o.S(o.ws, c, is));  // wsink, interp.f:811
    double cx = o.xc[i] - o.cfg.center_x, cy = o.yc[j] - o.cfg.center_y;
    double dist2 = cx * cx + cy * cy;
    double rprox2 = o.cfg.rprox * o.cfg.rprox, rdist2 = o.cfg.rdist * o.cfg.rdist;
    if (dist2 > rprox2 && dist2 < rdist2) o.S(o.sink, c, is) = rsft_up * wst * o.indz[k];
    int ntr = o.d3 ? o.nx * o.ny : o.nx;
    size_t b = (size_t)(is - 1) * ntr + (o.d3 ? (i - 1) + o.nx * (j - 1) : (i - 1));
    double dt = o.cfg.dt;
    if (!o.d3) o.massl[b] = o.massl[b] + o.S(o.sink, c, is) * o.dx[i] * o.dz[k] * dt;
    else o.massl[b] = o.massl[b] + o.S(o.sink, c, is) * o.dx[i] * o.dy[j] * o.dz[k] * dt;
    o.massl[b] = o.mass_loss[b] + o.massl[b];
    o.mass_loss[b] = 0.0;
}

void boundary_2d(Oracle &o, int sweep) {
    (void)sweep;
    int n = o.ncell, ns = o.ns;
    if (o.cfg.isink > 0) std::fill(o.sink.begin(), o.sink.end(), 0.0);  // bdry.f:73
    auto US = [&](vector<double> &a, int c, int is) -> double & { return a[(size_t)(is - 1) * n + c]; };
    auto copy_s = [&](vector<double> &a, int dst, int src, double f) { for (int is = 1; is <= ns; ++is) US(a, dst, is) = f * US(a, src, is); };
    auto set_s = [&](vector<double> &a, int dst, double v) { for (int is = 1; is <= ns; ++is) US(a, dst, is) = v; };
    double usv[PDAC_MAX_NSOLID + 1];
    for (int c = 0; c < n; ++c) {
        int i, j, k;
        o.ijk_of(c, i, j, k);
        if (o.flag[c] == VENT) {
            // inlet_velocity_fluctuations, vent.f:902-936
            if (o.cfg.irand >= 1) {
                int nv = -1;
                for (int q = 0; q < o.cfg.nvent; ++q) if (o.cfg.vent_ijk[q] == c) nv = q;
                if (nv >= 0) {
                    double intensity = 0.01;
                    double rann = o.vent_fact[nv] * intensity, ranold = o.vent_fact0[nv] * intensity;
                    o.vent_fact0[nv] = o.vent_fact[nv];
                    o.ug[c] = o.ug[c] * (1.0 + rann) / (1.0 + ranold);
                    o.wg[c] = o.wg[c] * (1.0 + rann) / (1.0 + ranold);
                    for (int is = 1; is <= ns; ++is) {
                        US(o.us, c, is) = US(o.us, c, is) * (1.0 + rann) / (1.0 + ranold);
                        US(o.ws, c, is) = US(o.ws, c, is) * (1.0 + rann) / (1.0 + ranold);
                    }
                }
            }
            continue;
        }
        if (ib_cell(o.flag[c])) {  // forcing points, bdry.f:103-204
            ib_boundary_cell(o, c);
            continue;
        }
        if (!(o.flag[c] == FLUID || o.flag[c] == DOME || o.flag[c] == BL_CELL)) continue;
        int ipjk = o.nbraw(E, c), imjk = o.nbraw(W, c), ijkp = o.nbraw(T, c), ijkm = o.nbraw(B, c);
        int ipjkp = o.nbraw(ET, c), imjkp = o.nbraw(WT, c), ipjkm = o.nbraw(EB, c);
        int ijkmm = o.nbraw(BB, c);
        // East
        {
            int n2 = ipjk, n1 = c, n0 = imjk;
            int f2 = o.flag[n2];
            if (f2 == SLIP) {
                o.ug[n1] = 0; set_s(o.us, n1, 0.0); o.ug[n2] = 0; set_s(o.us, n2, 0.0);
                o.wg[n2] = o.wg[n1]; copy_s(o.ws, n2, n1, 1.0);
            } else if (f2 == NOSLIP) {
                o.ug[n1] = 0; set_s(o.us, n1, 0.0); o.ug[n2] = 0; set_s(o.us, n2, 0.0);
                if (!o.fluidbit(ipjkp)) { o.wg[n2] = -o.wg[n1]; copy_s(o.ws, n2, n1, -1.0); }
            } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
                o.ug[n1] = o.ug[n0]; copy_s(o.us, n1, n0, 1.0);
                o.ug[n2] = o.ug[n1]; copy_s(o.us, n2, n1, 1.0);
                o.wg[n2] = o.wg[n1]; copy_s(o.ws, n2, n1, 1.0);
                double gnorm = o.cfg.gravx * 0.5 * (o.dx[i + 1] + o.dx[i]);
                if (f2 == ZERO_GRAD) gnorm = 0.0;
                for (int is = 1; is <= ns; ++is) usv[is] = US(o.us, n1, is);
                inoutflow(o, o.ug[n1], usv, n2, n1, k, gnorm);
            }
        }
        // West
        {
            int n2 = imjk, n1 = c;
            int f2 = o.flag[n2];
            if (f2 == SLIP) {
                o.ug[n2] = 0; set_s(o.us, n2, 0.0);
                o.wg[n2] = o.wg[n1]; copy_s(o.ws, n2, n1, 1.0);
            } else if (f2 == NOSLIP) {
                o.ug[n2] = 0; set_s(o.us, n2, 0.0);
                if (!o.fluidbit(imjkp)) { o.wg[n2] = -o.wg[n1]; copy_s(o.ws, n2, n1, -1.0); }
            } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
                o.ug[n2] = o.ug[n1]; copy_s(o.us, n2, n1, 1.0);
                o.wg[n2] = o.wg[n1]; copy_s(o.ws, n2, n1, 1.0);
                double gnorm = o.cfg.gravx * 0.5 * (o.dx[i - 1] + o.dx[i]);
                if (f2 == ZERO_GRAD) gnorm = 0.0;
                for (int is = 1; is <= ns; ++is) usv[is] = US(o.us, n2, is);
                inoutflow(o, o.ug[n2], usv, n2, n1, k, gnorm);
            }
        }
        // Top
        {
            int n2 = ijkp, n1 = c;
            int f2 = o.flag[n2];
            if (f2 == SLIP) {
                o.wg[n1] = 0; set_s(o.ws, n1, 0.0);
                o.ug[n2] = o.ug[n1]; copy_s(o.us, n2, n1, 1.0);
            } else if (f2 == NOSLIP) {
                o.wg[n1] = 0; set_s(o.ws, n1, 0.0);
                // bdry.f:540-543 indexes us with an undefined class; all
                // classes are reflected here (the evident intent)
                if (!o.fluidbit(ipjkp)) { o.ug[n2] = -o.ug[n1]; copy_s(o.us, n2, n1, -1.0); }
            } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
                double d0 = o.dz[k - 1], d1 = o.dz[k], d2 = o.dz[k + 1];
                int ord = 0;
                o.ug[n2] = o.ug[n1]; copy_s(o.us, n2, n1, 1.0);
                auto extrap = [&](double f2v, double f1v, double d12, double dxv) {
                    double gradient = (f2v - f1v) / d12 * ord;
                    return f2v + gradient * dxv;
                };
                o.wg[c] = extrap(o.wg[ijkm], o.wg[ijkmm], d0, d1);
                for (int is = 1; is <= ns; ++is) US(o.ws, c, is) = extrap(US(o.ws, ijkm, is), US(o.ws, ijkmm, is), d0, d1);
                o.wg[ijkp] = extrap(o.wg[c], o.wg[ijkm], d1, d2);
                // bdry.f:576 uses the loop index past its end (an
                // out-of-range class); each class is extrapolated here
                for (int is = 1; is <= ns; ++is) US(o.ws, ijkp, is) = extrap(US(o.ws, c, is), US(o.ws, ijkm, is), d1, d2);
                if (f2 == ZERO_GRAD) zerograd(o, n2, n1);
                else {
                    double gnorm = o.cfg.gravz * 0.5 * (o.dz[k] + o.dz[k + 1]);
                    for (int is = 1; is <= ns; ++is) usv[is] = US(o.ws, n1, is);
                    inoutflow(o, o.wg[n1], usv, n2, n1, k + 1, gnorm);
                }
            }
        }
        // Bottom
        {
            int n1 = c, n2 = ijkm;
            int f2 = o.flag[n2];
            if (f2 == SLIP) {
                o.wg[n2] = 0; set_s(o.ws, n2, 0.0);
                if (o.flag[ipjkm] == SLIP) { o.ug[n2] = o.ug[n1]; copy_s(o.us, n2, n1, 1.0); }
                if (o.cfg.isink > 0) for (int is = 1; is <= ns; ++is) sink_update(o, n1, is);
            } else if (f2 == NOSLIP) {
                o.wg[n2] = 0; set_s(o.ws, n2, 0.0);
                if (o.flag[ipjkm] == NOSLIP) { o.ug[n2] = -o.ug[n1]; copy_s(o.us, n2, n1, -1.0); }
                if (o.cfg.isink > 0) for (int is = 1; is <= ns; ++is) sink_update(o, n1, is);
            } else if (f2 == FILLED1 || f2 == FILLED2) {
                if (o.cfg.isink > 0) for (int is = 1; is <= ns; ++is) sink_update(o, n1, is);
            } else if (f2 == FREE_IO || f2 == ZERO_GRAD) {
                o.wg[n2] = o.wg[n1]; copy_s(o.ws, n2, n1, 1.0);
                o.ug[n2] = o.ug[n1]; copy_s(o.us, n2, n1, 1.0);
                double gnorm = o.cfg.gravz * 0.5 * (o.dz[k - 1] + o.dz[k]);
                if (f2 == ZERO_GRAD) gnorm = 0.0;
                for (int is = 1; is <= ns; ++is) usv[is] = US(o.ws, n2, is);
                inoutflow(o, o.wg[n2], usv, n2, n1, k - 1, gnorm);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// setup of constants (setup.f:551-616, particles.f:35-79)
// ---------------------------------------------------------------------------
void setc(Oracle &o) {
    double g[8] = {0, 32.0, 28.0, 44.0, 2.0, 18.0, 28.96442, 64.0};
    for (int q = 1; q <= 7; ++q) o.gmw[q] = g[q] * 1.0e-3;
    double s[8] = {0, 3.467, 3.798, 3.941, 2.827, 2.641, 3.711, 4.112};
    double e[8] = {0, 106.7, 71.4, 195.2, 59.7, 809.1, 78.6, 335.4};
    for (int q = 1; q <= 7; ++q) { o.mmugs[q] = s[q]; o.mmugek[q] = e[q]; }
    for (int is = 1; is <= o.ns; ++is) {
        o.dk[is] = o.cfg.dk[is - 1];
        o.rl[is] = o.cfg.rl[is - 1];
        o.inrl[is] = 1.0 / o.rl[is];
        o.phis[is] = o.cfg.phis[is - 1];
        o.cmus[is] = o.cfg.cmus[is - 1];
        o.cps[is] = o.cfg.cps[is - 1];
        o.kap[is] = o.cfg.kap[is - 1];
        o.plim[is] = o.cfg.plim[is - 1];
        o.phi[is] = (double)0.63f;
    }
    for (int k = 1; k <= o.ns; ++k)
        for (int kk = 1; kk <= o.ns; ++kk) {
            int k1, k2;
            if (o.dk[k] >= o.dk[kk]) { k1 = k; k2 = kk; }
            else { k1 = kk; k2 = k; }
            double a = std::sqrt(o.dk[k2] / o.dk[k1]);
            o.philim[k][kk] = o.phi[k1] / (o.phi[k1] + (1.0 - o.phi[k1]) * o.phi[k2]);
            o.epsl[k][kk] = (o.phi[k1] - o.phi[k2]) + ((1.0 - a) * (1.0 - o.phi[k1]) * o.phi[k2]);
            double fact = (o.phi[k1] + (1.0 - o.phi[k2]) * o.phi[k1]) / o.phi[k1];
            o.epsl[k][kk] = o.epsl[k][kk] * fact;
            o.epsu[k][kk] = (1.0 - a) * (o.phi[k1] + (1.0 - o.phi[k1]) * o.phi[k2]);
            double s2 = o.dk[k] + o.dk[kk];
            o.dkf[k][kk] = s2 * s2 / (o.rl[k] * o.dk[k] * o.dk[k] * o.dk[k] + o.rl[kk] * o.dk[kk] * o.dk[kk] * o.dk[kk]);
            o.dkf[kk][k] = o.dkf[k][kk];
        }
}

void alloc(Oracle &o) {
    size_t n = o.ncell, ns = o.ns, ng = o.ng;
    for (auto *v : {&o.p, &o.ep, &o.rog, &o.rgp, &o.tg, &o.sieg, &o.cg, &o.ug, &o.vg, &o.wg, &o.pn, &o.epn, &o.rgpn,
                    &o.siegn, &o.mug, &o.kapg, &o.rugn, &o.rvgn, &o.rwgn, &o.rug, &o.rvg, &o.rwg, &o.rhg, &o.gvisx,
                    &o.gvisy, &o.gvisz, &o.ugfe, &o.ugft, &o.wgfe, &o.wgft, &o.rgfe, &o.rgfn, &o.rgft, &o.conv, &o.abeta, &o.dgres})
        v->assign(n, 0.0);
    for (auto *v : {&o.rlk, &o.ts, &o.sies, &o.us, &o.vs, &o.ws, &o.rlkn, &o.siesn, &o.rusn, &o.rvsn, &o.rwsn, &o.rus,
                    &o.rvs, &o.rws, &o.rhs, &o.pvisx, &o.pvisy, &o.pvisz, &o.usfe, &o.usft, &o.wsfe, &o.wsft, &o.rsfe,
                    &o.rsfn, &o.rsft, &o.sink})
        v->assign(n * ns, 0.0);
    for (auto *v : {&o.ygc, &o.xgc, &o.rgpgcn}) v->assign(n * ng, 0.0);
    for (auto *v : {&o.appu, &o.appv, &o.appw}) v->assign(n * o.nap, 0.0);
    if (o.d3) o.mf3.assign((size_t)(ns + 1) * 9 * n, 0.0);
}

#include "pdac_oracle3d.inc"
#include "pdac_oracle_rk3.inc"

}  // namespace

// ===========================================================================
// extern "C" interface used by the tests (ctypes) and bench.py's CPU arm
// ===========================================================================
extern "C" {

int pdac_oracle_create(const pdac_cfg *cfg, void **out) {
    if (!cfg || !out) return PDAC_ERR_ARG;
    Oracle *o = new Oracle();
    o->cfg = *cfg;
    o->d3 = cfg->job_type == 3;
    o->nx = cfg->nx; o->ny = o->d3 ? cfg->ny : 1; o->nz = cfg->nz;
    o->ncell = o->nx * o->ny * o->nz;
    o->ns = cfg->nsolid; o->ng = cfg->ngas; o->nph = o->ns + 1; o->nap = o->nph * (o->nph + 1) / 2;
    for (int ig = 0; ig < o->ng; ++ig) o->gas_type[ig] = cfg->gas_type[ig];
    auto fill1 = [](vector<double> &v, const double *src, int nn) {
        v.assign(nn + 4, 0.0);
        for (int q = 1; q <= nn; ++q) v[q] = src[q - 1];
        v[0] = v[1];
        v[nn + 1] = v[nn]; v[nn + 2] = v[nn]; v[nn + 3] = v[nn];
    };
    fill1(o->dx, cfg->dx, o->nx);
    fill1(o->dz, cfg->dz, o->nz);
    if (o->d3) fill1(o->dy, cfg->dy, o->ny); else o->dy.assign(4, 0.0);
    if (o->d3) { o->indy.resize(o->dy.size()); for (size_t q = 0; q < o->dy.size(); ++q) o->indy[q] = 1.0 / o->dy[q]; }
    auto inv = [](vector<double> &out, const vector<double> &in) { out.resize(in.size()); for (size_t q = 0; q < in.size(); ++q) out[q] = 1.0 / in[q]; };
    inv(o->indx, o->dx); inv(o->indz, o->dz);
    if (!o->d3) o->indy.assign(o->dy.size(), 0.0);
    // grid.f:306-345
    int nx = o->nx;
    o->r.assign(nx + 4, 1.0); o->rb.assign(nx + 4, 1.0); o->inr.assign(nx + 4, 1.0); o->inrb.assign(nx + 4, 1.0);
    if (cfg->itc == 1 && !o->d3) {
        vector<double> xb(nx + 4, 0.0), x(nx + 4, 0.0);
        xb[1] = 0.0; x[1] = -0.5 * o->dx[1] + xb[1];
        for (int i = 2; i <= nx; ++i) { xb[i] = (xb[i - 1] + o->dx[i]); x[i] = (xb[i] - 0.5 * o->dx[i]); }
        for (int i = 1; i <= nx; ++i) { o->r[i] = x[i]; o->rb[i] = xb[i]; }
        o->rb[0] = o->rb[1] - o->dx[1];  // padding only
        o->inrb[1] = (o->rb[1] == 0.0) ? 1.0e10 : 1.0 / o->rb[1];
        for (int i = 2; i <= nx; ++i) o->inrb[i] = 1.0 / o->rb[i];
        for (int i = 1; i <= nx; ++i) o->inr[i] = 1.0 / o->r[i];
    }
    o->flag.assign(cfg->flag, cfg->flag + o->ncell);
    o->p_atm.assign(o->nz + 2, 0.0); o->t_atm.assign(o->nz + 2, 0.0);
    for (int k = 1; k <= o->nz; ++k) { o->p_atm[k] = cfg->p_atm[k - 1]; o->t_atm[k] = cfg->t_atm[k - 1]; }
    o->vent_fact.assign(cfg->nvent, 1.0);
    o->vent_fact0.assign(cfg->nvent, 0.0);
    static vector<int> dummy;
    o->cfg.dx = o->cfg.dy = o->cfg.dz = nullptr; o->cfg.flag = nullptr; o->cfg.p_atm = o->cfg.t_atm = nullptr;
    // keep our own copy of the vent list
    int *vl = new int[cfg->nvent > 0 ? cfg->nvent : 1];
    for (int q = 0; q < cfg->nvent; ++q) vl[q] = cfg->vent_ijk[q];
    o->cfg.vent_ijk = vl;
    o->cfg.ib_faces = nullptr; o->cfg.ib_ivf = nullptr;
    for (int a = 0; a < 3; ++a) { o->cfg.ib_num[a] = nullptr; o->cfg.ib_fp[a] = nullptr; o->cfg.ib_nsl[a] = nullptr; }
    o->cfg.x = o->cfg.xb = o->cfg.y = o->cfg.yb = o->cfg.z = o->cfg.zb = nullptr;
    o->cfg.topo_c = nullptr;
    ib_setup(*o, cfg);
    if (ib_check(*o) != PDAC_OK) {
        delete[] vl;
        delete o;
        return PDAC_ERR_CONFIG;
    }
    setc(*o);
    build_tables(*o);
    if (o->d3) build_tables3(*o);
    alloc(*o);
    les_setup(*o, cfg);
    sink_setup(*o);
    *out = o;
    return PDAC_OK;
}

int pdac_oracle_destroy(void *h) {
    Oracle *o = (Oracle *)h;
    if (!o) return PDAC_ERR_ARG;
    delete[] o->cfg.vent_ijk;
    delete o;
    return PDAC_OK;
}

int pdac_oracle_set_order(void *h, int order) {
    ((Oracle *)h)->order = order;
    return PDAC_OK;
}

static void copy_in(vector<double> &dst, const double *src, size_t n) {
    if (src) std::memcpy(dst.data(), src, n * sizeof(double));
}
static void copy_out(double *dst, const vector<double> &src, size_t n) {
    if (dst) std::memcpy(dst, src.data(), n * sizeof(double));
}

int pdac_oracle_set_state(void *h, const pdac_state_view *s) {
    Oracle &o = *(Oracle *)h;
    size_t n = o.ncell, ns = o.ns, ng = o.ng;
    copy_in(o.p, s->p, n); copy_in(o.ep, s->ep, n); copy_in(o.rog, s->rog, n); copy_in(o.rgp, s->rgp, n);
    copy_in(o.tg, s->tg, n); copy_in(o.sieg, s->sieg, n); copy_in(o.cg, s->cg, n);
    copy_in(o.ug, s->ug, n); copy_in(o.vg, s->vg, n); copy_in(o.wg, s->wg, n);
    copy_in(o.rlk, s->rlk, n * ns); copy_in(o.ts, s->ts, n * ns); copy_in(o.sies, s->sies, n * ns);
    copy_in(o.us, s->us, n * ns); copy_in(o.vs, s->vs, n * ns); copy_in(o.ws, s->ws, n * ns);
    copy_in(o.ygc, s->ygc, n * ng); copy_in(o.xgc, s->xgc, n * ng);
    return PDAC_OK;
}

int pdac_oracle_get_state(void *h, pdac_state_view *s) {
    Oracle &o = *(Oracle *)h;
    size_t n = o.ncell, ns = o.ns, ng = o.ng;
    copy_out(s->p, o.p, n); copy_out(s->ep, o.ep, n); copy_out(s->rog, o.rog, n); copy_out(s->rgp, o.rgp, n);
    copy_out(s->tg, o.tg, n); copy_out(s->sieg, o.sieg, n); copy_out(s->cg, o.cg, n);
    copy_out(s->ug, o.ug, n); copy_out(s->vg, o.vg, n); copy_out(s->wg, o.wg, n);
    copy_out(s->rlk, o.rlk, n * ns); copy_out(s->ts, o.ts, n * ns); copy_out(s->sies, o.sies, n * ns);
    copy_out(s->us, o.us, n * ns); copy_out(s->vs, o.vs, n * ns); copy_out(s->ws, o.ws, n * ns);
    copy_out(s->ygc, o.ygc, n * ng); copy_out(s->xgc, o.xgc, n * ng);
    return PDAC_OK;
}

int pdac_oracle_boundary(void *h, int sweep) {
    Oracle &o = *(Oracle *)h;
    if (o.d3) boundary_3d(o, sweep); else boundary_2d(o, sweep);
    return PDAC_OK;
}
int pdac_oracle_fieldn(void *h) {
    Oracle &o = *(Oracle *)h;
    if (o.d3) fieldn3(o); else fieldn(o);
    // allocate_fluxes (tilde.f:56-102): tilde/app terms zeroed once per step
    for (auto *v : {&o.rug, &o.rwg, &o.rhg}) std::fill(v->begin(), v->end(), 0.0);
    for (auto *v : {&o.rus, &o.rws, &o.rhs, &o.appu, &o.appw}) std::fill(v->begin(), v->end(), 0.0);
    if (o.d3) for (auto *v : {&o.rvg, &o.rvs, &o.appv}) std::fill(v->begin(), v->end(), 0.0);
    return PDAC_OK;
}
int pdac_oracle_tilde(void *h, double dt) {
    Oracle &o = *(Oracle *)h;
    if (o.d3) tilde_3d(o, dt); else tilde_2d(o, dt);
    return PDAC_OK;
}
int pdac_oracle_iter(void *h, double dt, int *nit) {
    Oracle &o = *(Oracle *)h;
    return o.d3 ? iter_3d(o, dt, nit) : iter_2d(o, dt, nit);
}
int pdac_oracle_ygas(void *h, double dt) {
    Oracle &o = *(Oracle *)h;
    if (o.d3) ygas_3d(o, dt); else ygas_2d(o, dt);
    return PDAC_OK;
}
int pdac_oracle_htilde(void *h, double dt) {
    Oracle &o = *(Oracle *)h;
    if (o.d3) htilde_3d(o, dt); else htilde_2d(o, dt);
    return PDAC_OK;
}
int pdac_oracle_ftem(void *h, double dt) {
    Oracle &o = *(Oracle *)h;
    return o.d3 ? ftem_3d(o, dt) : ftem_2d(o, dt);
}

// compute_mixture_fields (mixture.f:32-52): derived.f:220-331 over every cell
int pdac_oracle_compute_mixture_fields(void *h) {
    Oracle &o = *(Oracle *)h;
    const int n = o.ncell, ns = o.ns, ng = o.ng;
    for (auto *v : {&o.rhom, &o.um, &o.vm, &o.wm, &o.tm}) v->assign(n, 0.0);
    o.yd.assign((size_t)n * (ng + ns), 0.0);
    for (int c = 0; c < n; ++c) {
        double srl = 0.0;
        for (int is = 1; is <= ns; ++is) srl = srl + o.S(o.rlk, c, is);
        o.rhom[c] = o.rgp[c] + srl;
        double cpgc[8];
        hcapg(o, cpgc, o.tg[c]);
        double cgas = 0.0;
        for (int ig = 0; ig < ng; ++ig) cgas = cpgc[o.gas_type[ig]] * o.ygc[(size_t)ig * n + c] + cgas;
        double sts = 0.0, scp = 0.0;
        for (int is = 1; is <= ns; ++is) {
            sts = sts + o.S(o.rlk, c, is) * o.cps[is] * o.S(o.ts, c, is);
            scp = scp + o.S(o.rlk, c, is) * o.cps[is];
        }
        double tm = o.rgp[c] * cgas * o.tg[c] + sts;
        double den = o.rgp[c] * cgas + scp;
        o.tm[c] = tm / den;
        auto velm = [&](const vector<double> &ug, const vector<double> &us) {
            double sv = 0.0;
            for (int is = 1; is <= ns; ++is) sv = sv + o.S(o.rlk, c, is) * us[(size_t)(is - 1) * n + c];
            double v = o.rgp[c] * ug[c] + sv;
            return v / o.rhom[c];
        };
        o.um[c] = velm(o.ug, o.us);
        if (o.d3) o.vm[c] = velm(o.vg, o.vs);
        o.wm[c] = velm(o.wg, o.ws);
        double inrhom = 1.0 / o.rhom[c];
        for (int ig = 0; ig < ng; ++ig) o.yd[(size_t)ig * n + c] = o.ygc[(size_t)ig * n + c] * o.rgp[c] * inrhom;
        for (int is = 1; is <= ns; ++is) o.yd[(size_t)(ng + is - 1) * n + c] = o.S(o.rlk, c, is) * inrhom;
    }
    return PDAC_OK;
}

// sgsg / sgss as prog.f:207-208 calls them after fieldn
int pdac_oracle_sgs(void *h) {
    Oracle &o = *(Oracle *)h;
    if (o.cfg.iturb >= 1) sgsg(o);
    if (o.cfg.iss == 1) sgss(o);
    return PDAC_OK;
}

// initialize_fieldn (explicit_solver.f:419-564), the time_integration = 1
// counterpart of fieldn; coefficients use the full time step
int pdac_oracle_initialize_fieldn(void *h) {
    Oracle &o = *(Oracle *)h;
    rk3_fieldn(o, o.cfg.dt);
    return PDAC_OK;
}
// explicit_iter (explicit_solver.f:996-1223); PDAC_ERR_EOS when more than
// one caloric failure, as explicit_solver.f:1214-1215 aborts
int pdac_oracle_explicit_iter(void *h, double dt) {
    Oracle &o = *(Oracle *)h;
    if (o.rk.neq == 0) return PDAC_ERR_ARG;
    int num = rk3_iter(o, dt);
    return num > 1 ? PDAC_ERR_EOS : PDAC_OK;
}

// prog.f:143-417 for one step
int pdac_oracle_step(void *h, int sweep, int *nit) {
    Oracle &o = *(Oracle *)h;
    pdac_oracle_boundary(h, sweep);
    if (o.cfg.update_eosg) {
        for (int c = 0; c < o.ncell; ++c) {
            double xg[PDAC_MAX_NGAS];
            for (int ig = 0; ig < o.ng; ++ig) xg[ig] = o.xgc[(size_t)ig * o.ncell + c];
            o.rog[c] = thermal_eosg(o, o.tg[c], o.p[c], xg);
            o.rgp[c] = o.rog[c] * o.ep[c];
        }
    }
    double dt0 = o.cfg.dt;
    int st = PDAC_OK;
    if (o.cfg.time_integration == 1) {
        pdac_oracle_initialize_fieldn(h);
        pdac_oracle_sgs(h);
        if (nit) *nit = 0;
        for (int rk = 1; rk <= o.cfg.rungekut; ++rk) {
            double dt = dt0 / (o.cfg.rungekut + 1 - rk);
            int s2 = pdac_oracle_explicit_iter(h, dt);
            if (s2 != PDAC_OK) st = s2;
            pdac_oracle_ygas(h, dt);
        }
        if (o.cfg.compute_mixture) pdac_oracle_compute_mixture_fields(h);  // prog.f:331
        return st;
    }
    pdac_oracle_fieldn(h);
    pdac_oracle_sgs(h);
    const bool ifx = o.cfg.implicit_fluxes != 0, ien = o.cfg.implicit_enthalpy != 0;
    for (int rk = 1; rk <= o.cfg.rungekut; ++rk) {
        double dt = dt0 / (o.cfg.rungekut + 1 - rk);
        // prog.f:246-292
        if (!ifx) {
            pdac_oracle_tilde(h, dt);
            if (ien) pdac_oracle_htilde(h, dt);
        }
        int s1 = pdac_oracle_iter(h, dt, nit);
        if (s1 == PDAC_ERR_MAXOUT) return s1;  // error() stops the run (iter.f:449)
        if (s1 != PDAC_OK) st = s1;
        pdac_oracle_ygas(h, dt);
        if (!ien) {
            pdac_oracle_htilde(h, dt);
            int s2 = pdac_oracle_ftem(h, dt);
            if (s2 != PDAC_OK) st = s2;
        }
    }
    if (o.cfg.compute_mixture) pdac_oracle_compute_mixture_fields(h);  // prog.f:331
    return st;
}

int pdac_oracle_get_array(void *h, const char *name, double *out, long *n_inout) {
    Oracle &o = *(Oracle *)h;
    struct E { const char *n; vector<double> *v; };
    E tab[] = {{"p", &o.p}, {"ep", &o.ep}, {"rog", &o.rog}, {"rgp", &o.rgp}, {"tg", &o.tg}, {"sieg", &o.sieg},
               {"cg", &o.cg}, {"ug", &o.ug}, {"vg", &o.vg}, {"wg", &o.wg}, {"rlk", &o.rlk}, {"ts", &o.ts},
               {"sies", &o.sies}, {"us", &o.us}, {"vs", &o.vs}, {"ws", &o.ws}, {"ygc", &o.ygc}, {"xgc", &o.xgc},
               {"pn", &o.pn}, {"epn", &o.epn}, {"rgpn", &o.rgpn}, {"siegn", &o.siegn}, {"rlkn", &o.rlkn},
               {"siesn", &o.siesn}, {"rgpgcn", &o.rgpgcn}, {"mug", &o.mug}, {"kapg", &o.kapg},
               {"rugn", &o.rugn}, {"rwgn", &o.rwgn}, {"rusn", &o.rusn}, {"rwsn", &o.rwsn},
               {"rug", &o.rug}, {"rwg", &o.rwg}, {"rus", &o.rus}, {"rws", &o.rws},
               {"appu", &o.appu}, {"appw", &o.appw}, {"gvisx", &o.gvisx}, {"gvisz", &o.gvisz},
               {"pvisx", &o.pvisx}, {"pvisz", &o.pvisz}, {"ugfe", &o.ugfe}, {"ugft", &o.ugft},
               {"wgfe", &o.wgfe}, {"wgft", &o.wgft}, {"usfe", &o.usfe}, {"usft", &o.usft},
               {"wsfe", &o.wsfe}, {"wsft", &o.wsft}, {"rgfe", &o.rgfe}, {"rgft", &o.rgft},
               {"rsfe", &o.rsfe}, {"rsft", &o.rsft}, {"conv", &o.conv}, {"abeta", &o.abeta},
               {"rhg", &o.rhg}, {"rhs", &o.rhs}, {"sink", &o.sink}, {"egfe", &o.egfe}, {"egft", &o.egft},
               {"esfe", &o.esfe}, {"esft", &o.esft}, {"dgres", &o.dgres},
               {"rvgn", &o.rvgn}, {"rvsn", &o.rvsn}, {"rvg", &o.rvg}, {"rvs", &o.rvs}, {"appv", &o.appv},
               {"rgfn", &o.rgfn}, {"rsfn", &o.rsfn}, {"mf3", &o.mf3}, {"ef3", &o.ef3},
               {"gvisy", &o.gvisy}, {"pvisy", &o.pvisy}, {"hgfe", &o.hgfe}, {"hgft", &o.hgft},
               {"hsfe", &o.hsfe}, {"hsft", &o.hsft}, {"smag", &o.smag}, {"scoeff", &o.scoeff}, {"massl", &o.massl}, {"rhom", &o.rhom}, {"um", &o.um},
               {"vm", &o.vm}, {"wm", &o.wm}, {"tm", &o.tm}, {"yd", &o.yd}, {"mugt", &o.mugt}, {"kapgt", &o.kapgt},
               {"must", &o.must},
               // explicit-solver fields (explicit_solver.f:15-83)
               {"rgpstar", &o.rk.rgpS}, {"rlkstar", &o.rk.rlkS}, {"ugstar", &o.rk.ugS}, {"usstar", &o.rk.usS},
               {"vgstar", &o.rk.vgS}, {"vsstar", &o.rk.vsS}, {"wgstar", &o.rk.wgS}, {"wsstar", &o.rk.wsS},
               {"tgstar", &o.rk.tgS}, {"tsstar", &o.rk.tsS}, {"siegstar", &o.rk.siegS}, {"siesstar", &o.rk.siesS},
               {"pstar", &o.rk.pS}, {"epstar", &o.rk.epS}, {"rhogstar", &o.rk.rhogS}, {"ugn", &o.rk.ugN},
               {"usn", &o.rk.usN}, {"vgn", &o.rk.vgN}, {"vsn", &o.rk.vsN}, {"wgn", &o.rk.wgN}, {"wsn", &o.rk.wsN},
               {"hv", &o.rk.hv}, {"kpgv", &o.rk.kpgv}, {"rhs3", &o.rk.rhs3}, {"k1", &o.rk.k1}, {"k2", &o.rk.k2},
               {"k3", &o.rk.k3}, {"hf3", &o.rk.hf3}};
    for (auto &e : tab) {
        if (std::strcmp(e.n, name) == 0) {
            long need = (long)e.v->size();
            if (*n_inout < need) { *n_inout = need; return PDAC_ERR_ARG; }
            std::memcpy(out, e.v->data(), need * sizeof(double));
            *n_inout = need;
            return PDAC_OK;
        }
    }
    return PDAC_ERR_ARG;
}

int pdac_oracle_set_vent_factors(void *h, const double *fact, int nvent) {
    Oracle &o = *(Oracle *)h;
    if (nvent != (int)o.vent_fact.size()) return PDAC_ERR_ARG;
    for (int q = 0; q < nvent; ++q) o.vent_fact[q] = fact[q];
    return PDAC_OK;
}

int pdac_oracle_mass_totals(void *h, double *out, int nout) {
    Oracle &o = *(Oracle *)h;
    int need = 1 + o.ns + o.ng;
    if (nout < need) return PDAC_ERR_ARG;
    for (int q = 0; q < need; ++q) out[q] = 0.0;
    // residuals.f:14-130: volume-weighted sums over fluid cells
    for (int c = 0; c < o.ncell; ++c) {
        if (!o.fluidbit(c)) continue;
        int i, j, k;
        o.ijk_of(c, i, j, k);
        double vol = o.dx[i] * o.dz[k] * (o.cfg.itc == 1 ? o.r[i] : 1.0) * (o.d3 ? o.dy[j] : 1.0);
        out[0] += o.rgp[c] * vol;
        for (int is = 1; is <= o.ns; ++is) out[is] += o.S(o.rlk, c, is) * vol;
        for (int ig = 1; ig <= o.ng; ++ig) out[o.ns + ig] += o.rgp[c] * o.S(o.ygc, c, ig) * vol;
    }
    return PDAC_OK;
}

int pdac_oracle_last_nit(void *h) { return ((Oracle *)h)->last_nit; }
// the shared exp and pow (for their accuracy tests)
double pdac_oracle_fp_pow(double x, double y) { return pdac_fp::pow(x, y); }
double pdac_oracle_fp_exp(double x) { return pdac_fp::exp(x); }
// threads of the 3D cell loops (n <= 0 keeps the current count); returns
// the number in use afterwards
int pdac_oracle_set_threads(int n) {
    if (n > 0) g_oracle_threads = n;
    return oracle_threads();
}
// the cells of the last outer sweep that ran the inner loop, increasing
int pdac_oracle_unconverged_cells(void *h, int *ijk, long *n_inout) {
    Oracle &o = *(Oracle *)h;
    vector<int> v = o.unconv;
    std::sort(v.begin(), v.end());
    if (!ijk || *n_inout < (long)v.size()) { *n_inout = (long)v.size(); return v.empty() ? PDAC_OK : PDAC_ERR_ARG; }
    std::copy(v.begin(), v.end(), ijk);
    *n_inout = (long)v.size();
    return PDAC_OK;
}
int pdac_oracle_eos_fail(void *h) { return ((Oracle *)h)->eos_fail; }

// known-answer helpers (pure functions of the reference formulas)
double pdac_oracle_limiter(int lim_type, double erre, double beta) { return limiter(lim_type, erre, beta); }


// Gauss-Jordan of matrix.f:351-391 on a caller-given system (row-major a,
// nph <= 9); plim has nph-1 entries.  Known-answer helper for the tests.
int pdac_oracle_gauss_jordan(int nph, double *a, double *b, const double *plim) {
    if (nph < 1 || nph > PDAC_MAX_NSOLID + 1) return PDAC_ERR_ARG;
    Oracle o;
    o.nph = nph;
    for (int l = 1; l < nph; ++l) o.plim[l] = plim[l - 1];
    Mat m{};
    double bb[PDAC_MAX_NSOLID + 2]{};
    for (int r = 1; r <= nph; ++r) {
        bb[r] = b[r - 1];
        for (int q = 1; q <= nph; ++q) m[r][q] = a[(r - 1) * nph + (q - 1)];
    }
    gauss_jordan(o, m, bb);
    for (int r = 1; r <= nph; ++r) b[r - 1] = bb[r];
    return PDAC_OK;
}

// hcapgs.f:33-85 for all 7 species
void pdac_oracle_hcapg(int icpc, double tref, double tg, double *out7) {
    Oracle o;
    o.cfg.icpc = icpc;
    o.cfg.tref = tref;
    double g[8] = {0, 32.0, 28.0, 44.0, 2.0, 18.0, 28.96442, 64.0};
    for (int q = 1; q <= 7; ++q) o.gmw[q] = g[q] * 1.0e-3;
    double cpc[8];
    hcapg(o, cpc, tg);
    for (int q = 0; q < 7; ++q) out7[q] = cpc[q + 1];
}

// caloric_eosg (eosg.f:139-223) for one gas mixture; returns info
int pdac_oracle_caloric(int ngas, const int *gas_type, const double *yg, double sieg, double *tg, double *cg) {
    Oracle o;
    o.ng = ngas;
    o.cfg.icpc = 2;
    double g[8] = {0, 32.0, 28.0, 44.0, 2.0, 18.0, 28.96442, 64.0};
    for (int q = 1; q <= 7; ++q) o.gmw[q] = g[q] * 1.0e-3;
    for (int q = 0; q < ngas; ++q) o.gas_type[q] = gas_type[q];
    return caloric_eosg(o, *cg, *tg, yg, sieg);
}

// padjust (iter.f:997-1072) driven on a scalar residual d(p) = a*(p - p0)
// for nsteps; writes the pressure after each step.  Known-answer helper.
int pdac_oracle_padjust_trace(double a, double p0, double pstart, double abeta, double omega, int nsteps, double *ptrace) {
    Oracle o;
    int kros = -1;
    double p = pstart, p3 = pstart, d3 = a * (pstart - p0);
    for (int q = 0; q < nsteps; ++q) {
        padjust(o, p, kros, d3, p3, omega, abeta);
        ptrace[q] = p;
        d3 = a * (p - p0);
    }
    return kros;
}

}  // extern "C"

// engine.cu -- host side of the B200 PDAC engine: context, device memory,
// kernel orchestration and the C ABI of include/pdac_gpu.h.
//
// One context owns one device-resident domain on the current CUDA device and
// one stream; every entry point enqueues work on that stream and returns a
// status.  The outer corrector sweeps of iter run as three colour-phase
// launches; the host reads the non-converged count after each sweep (the
// reference's parallel_sum_integer(mustit), iter.f:388).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>

#include "../../include/pdac_gpu.h"
#include "inner.cuh"
#include "tiles3d.cuh"
#include "rk3.cuh"
#include "io.cuh"
#include "les.cuh"
#include "sink.cuh"
#include "mixture.cuh"
#include "ib.cuh"

using namespace pdac;

struct pdac_ctx {
    pdac_cfg cfg;
    Prm P;
    Fld F;
    int nx = 0, ny = 1, nz = 0, ncell = 0, ns = 0, ng = 0, nph = 0, nap = 0;
    bool d3 = false;
    cudaStream_t stream = nullptr;
    double *arena = nullptr;
    size_t arena_doubles = 0;
    double *metric = nullptr;
    float *metric_f = nullptr;  // FP32 dx, dy, dz, indx, indy, indz of the mixed-precision flux passes
    int *d_flag = nullptr, *d_vent = nullptr, *d_counters = nullptr, *h_counters = nullptr;
    double *d_vfact = nullptr, *d_vfact0 = nullptr;
    double *d_app0u = nullptr, *d_app0v = nullptr, *d_app0w = nullptr;
    double *d_partial = nullptr;
    int nvent = 0;
    std::string err;
    cudaEvent_t ev[16];
    float phase_ms[7] = {0};
    // statistics: kernel launches, corrector launch timing (when profiling)
    long long launches = 0, sweeps = 0, corr_launches = 0, work_cells = 0, tested_cells = 0;
    double corr_ms = 0.0, resid_ms = 0.0, inner_ms = 0.0;
    // corrector worklists, one per colour (colour col at d_work + col *
    // work_stride, so the last sweep's lists remain for
    // pdac_gpu_unconverged_cells), and their per-colour lengths
    int *d_work = nullptr, *d_wcount = nullptr;
    long work_stride = 0;
    int last_nit = 0;                             // sweep count of the last pdac_gpu_iter
    int *d_nonfinite = nullptr, *h_nonfinite = nullptr;  // non-finite flag of the state checks
    // the whole semi-implicit time step as one graph (members of a batch):
    // its kernels outside the sweep loop, and the step's outcome [nit, caloric
    // failures of ftem, non-finite flag] read back once per step
    cudaGraph_t step_graph = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    long graph_gen = 0;  // bumped whenever captured launch shapes go stale (put_tuning)
    long long step_launches = 0;
    int *d_status = nullptr, *h_status = nullptr;
    unsigned *d_dirty = nullptr;                 // corrector active set, one bit per cell
    int *d_cand = nullptr;                       // candidate cells of one colour phase
    int inner_grid = 0;
    int *d_nit = nullptr, *h_nit = nullptr;  // outer sweep number (device, pinned host)
    // the outer sweep loop as a graph: a conditional WHILE node whose body is
    // one sweep, instantiated for one dt
    cudaGraph_t it_graph = nullptr;
    cudaGraphExec_t it_exec = nullptr;
    double it_dt = 0.0;
    long long it_per_sweep = 10;  // kernels of one sweep of that graph
    // small domains: the whole sweep loop as one cooperative launch of
    // coop_blocks blocks (0: the graph), coop_cpb cells per block, at most
    // coop_max_blocks blocks resident at once
    int coop_blocks = 0, coop_cpb = 1024, coop_max_blocks = 0;
    // grid of the residual-test kernels (0: half the inner-loop grid)
    int test_grid = 0;
    // cooperative launches (the small-domain sweep loop, the explicit
    // solver's wavefront) only when the context is not stepped alongside
    // others: a batch turns them off in its members, so that no two
    // cooperative grids are in flight on the device at once
    bool allow_coop = true;
    std::vector<double> sweep_log;  // per colour phase when profiling: sweep, colour, worklist, tested, ms x2
    bool prof = false;
    cudaEvent_t cev[9];
    cudaEvent_t user_ev[32];
    std::vector<std::pair<std::string, std::pair<double *, size_t>>> names;
    // explicit SSP-RK3 solver (time_integration = 1): its fields and the
    // graph of one explicit_iter, instantiated for one dt
    int ti = 0;
    RkF K{};
    cudaGraph_t ex_graph = nullptr;
    cudaGraphExec_t ex_exec = nullptr;
    double ex_dt = 0.0;
    long long ex_launches = 0;  // kernel launches of one explicit_iter
    // profiling of explicit_iter: marks between its kernel groups and the
    // accumulated device ms of the groups [flux passes, stage kernels,
    // gas-enthalpy wavefronts, final rhs + coefficients + solve]
    cudaEvent_t xev[9];
    // pdac_gpu_exchange_state: its upload stream and one event per field,
    // created at its first call
    cudaStream_t up_stream = nullptr;
    cudaEvent_t fev[20] = {};
    cudaEvent_t up_done = nullptr;
    double ex_ms[4] = {0, 0, 0, 0};
    long long ex_calls = 0;
    // gas-enthalpy wavefront on hyperplane-ordered records: the cooperative
    // grid (0 when the device cannot co-schedule one; the wavefront then
    // runs as one launch per hyperplane) and whether it covers the widest
    // hyperplane
    // ground sink (isink > 0): per-column mass taken out, restart values,
    // ring mask
    pdac::Sink S{};
    double *d_sinkbuf = nullptr;
    // immersed boundaries: the forcing-point tables and mesh coordinates
    // (d_ibint, d_ibdbl) and the state they carry from one boundary pass to
    // the next (d_ibstate: forcing-point velocities, then the filled_cell_2
    // toggles, ibstate_doubles in all)
    pdac::IbDev IB{};
    int *d_ibint = nullptr;
    double *d_ibdbl = nullptr, *d_ibstate = nullptr;
    size_t ibstate_doubles = 0;
    // the ordered boundary pass (ib.cuh): the boundary cells sorted by level
    // and the start of every level (empty when one thread per cell gives the
    // reference's result)
    int *d_bitems = nullptr;
    std::vector<int> blevel;
    int *d_ring = nullptr;
    pdac::Wave W{};
    // shared-memory tiled 3D stencil passes: tile shape (index into
    // TILE_SHAPES) and planes per block of the march up k
    int tile_shape = 0, tile_kchunk = 32;
    int *d_wave_idx = nullptr;    // order, src[3], start
    double *d_wave_rec = nullptr; // records and pnew
    int wave_grid_blocks = 0;
    bool wave_one = false;
};

namespace {

// forms of the 3D momentum-flux pass (launch_mom_tile): 0 = one thread per
// (cell, phase) and component, three launches (k_tilde_flux3d<0|1|2>, the
// stencils gathered through L1); 1..4 = the shared-memory tiled pass
// k_mom_flux3d_tile with 32 x 4, 32 x 8, 16 x 8 or 64 x 2 cells (i x j) per
// block.  Measured on the 256 x 256 x 192 plume (the autotuner picks per
// run): form 0 took 8.2 ms per tilde, the 32 x 4 tile ~9 ms -- its threads
// run all three components between two barriers at 12 warps per SM
const int N_TILE_SHAPES = 5;

// set_attr: raise the kernel's dynamic shared-memory limit (done once per
// context at create, outside any stream capture); else launch it
template <int TX, int TY, typename Real>
cudaError_t launch_mom_tile_t(const pdac::Prm &P, const pdac::Fld &F, int nph, int kchunk, cudaStream_t st,
                              bool set_attr) {
    const int sm = pdac::tile_smem_bytes<TX, TY, Real>(4);
    if (set_attr)
        return cudaFuncSetAttribute(pdac::k_mom_flux3d_tile<TX, TY, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    dim3 grid((P.nx + TX - 1) / TX, (P.ny + TY - 1) / TY, nph * ((P.nz + kchunk - 1) / kchunk));
    pdac::k_mom_flux3d_tile<TX, TY, Real><<<grid, TX * TY, sm, st>>>(P, F, kchunk);
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_mom_tile(const pdac::Prm &P, const pdac::Fld &F, int nph, int shape, int kchunk, cudaStream_t st,
                            bool set_attr = false) {
    // the tiled pass reads its stencils from shared memory and does not
    // apply the immersed-boundary velocity masks: immersed boundaries use form 0
    if (P.immb && !set_attr) shape = 0;
    switch (shape) {
        case 1: return launch_mom_tile_t<32, 4, Real>(P, F, nph, kchunk, st, set_attr);
        case 2: return launch_mom_tile_t<32, 8, Real>(P, F, nph, kchunk, st, set_attr);
        case 3: return launch_mom_tile_t<16, 8, Real>(P, F, nph, kchunk, st, set_attr);
        case 4: return launch_mom_tile_t<64, 2, Real>(P, F, nph, kchunk, st, set_attr);
        default: {
            if (set_attr) return cudaSuccess;
            const long nt = (long)P.ncell * nph;
            const int g = (int)((nt + 127) / 128);
            pdac::k_tilde_flux3d<0, Real><<<g, 128, 0, st>>>(P, F);
            pdac::k_tilde_flux3d<1, Real><<<g, 128, 0, st>>>(P, F);
            pdac::k_tilde_flux3d<2, Real><<<g, 128, 0, st>>>(P, F);
            return cudaGetLastError();
        }
    }
}

// kernel launches of one momentum-flux pass of form shape
inline int mom_launches(int shape) { return shape == 0 ? 3 : 1; }

cudaError_t set_tile_attrs(const pdac::Prm &P, const pdac::Fld &F) {
    for (int s = 0; s < N_TILE_SHAPES; ++s) {
        cudaError_t e = launch_mom_tile<double>(P, F, 1, s, 1, nullptr, true);
        if (e == cudaSuccess) e = launch_mom_tile<float>(P, F, 1, s, 1, nullptr, true);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

const int TPB = 128;
const int TPB_TEAM = 128;

int fail(pdac_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) return fail(ctx, PDAC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline int blocks(long n, int tpb = TPB) { return (int)((n + tpb - 1) / tpb); }

// launch a kernel template instantiated for the run's phase count (gas +
// solid classes): 2, 3, 4 and 6 phases have register-resident phase systems,
// any other count runs the generic instantiation
#define PHASE_LAUNCH(nph, KERNEL, grid, tpb, st, ...)                              \
    do {                                                                           \
        switch (nph) {                                                             \
            case 2: KERNEL<2><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;           \
            case 3: KERNEL<3><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;           \
            case 4: KERNEL<4><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;           \
            case 6: KERNEL<6><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;           \
            default: KERNEL<0><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;          \
        }                                                                          \
    } while (0)

// the same for a kernel template over (phases, dimensions)
#define PHASE_LAUNCH_D(nph, KERNEL, D, grid, tpb, st, ...)                         \
    do {                                                                           \
        switch (nph) {                                                             \
            case 2: KERNEL<2, D><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;        \
            case 3: KERNEL<3, D><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;        \
            case 4: KERNEL<4, D><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;        \
            case 6: KERNEL<6, D><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;        \
            default: KERNEL<0, D><<<grid, tpb, 0, st>>>(__VA_ARGS__); break;       \
        }                                                                          \
    } while (0)

// the inner-loop kernels (k_inner_team) with their dynamic shared memory
#define INNER_LAUNCH_D(nph, KERNEL, D, grid, tpb, st, ...)                                                   \
    do {                                                                                                     \
        switch (nph) {                                                                                       \
            case 2: KERNEL<2, D><<<grid, tpb, pdac::inner_smem_bytes<2>(), st>>>(__VA_ARGS__); break;      \
            case 3: KERNEL<3, D><<<grid, tpb, pdac::inner_smem_bytes<3>(), st>>>(__VA_ARGS__); break;      \
            case 4: KERNEL<4, D><<<grid, tpb, pdac::inner_smem_bytes<4>(), st>>>(__VA_ARGS__); break;      \
            case 6: KERNEL<6, D><<<grid, tpb, pdac::inner_smem_bytes<6>(), st>>>(__VA_ARGS__); break;      \
            default: KERNEL<0, D><<<grid, tpb, pdac::inner_smem_bytes<0>(), st>>>(__VA_ARGS__); break;     \
        }                                                                                                    \
    } while (0)

// raise the dynamic shared-memory limit of the inner-loop kernels (once per
// context at create, outside any stream capture)
template <int NP>
static cudaError_t set_inner_attrs_np() {
    const int sm = (int)pdac::inner_smem_bytes<NP>();
    cudaError_t e = cudaFuncSetAttribute(pdac::k_inner_team<NP, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pdac::k_inner_team<NP, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pdac::k_iter_coop<NP, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pdac::k_iter_coop<NP, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    return e;
}
static cudaError_t set_inner_attrs() {
    cudaError_t e = set_inner_attrs_np<2>();
    if (e == cudaSuccess) e = set_inner_attrs_np<3>();
    if (e == cudaSuccess) e = set_inner_attrs_np<4>();
    if (e == cudaSuccess) e = set_inner_attrs_np<6>();
    if (e == cudaSuccess) e = set_inner_attrs_np<0>();
    return e;
}

// setup.f:551-616 and particles.f:35-79: gas and particle constants
void set_constants(pdac_ctx *ctx) {
    Prm &P = ctx->P;
    const pdac_cfg &c = ctx->cfg;
    double g[8] = {0, 32.0, 28.0, 44.0, 2.0, 18.0, 28.96442, 64.0};
    double s[8] = {0, 3.467, 3.798, 3.941, 2.827, 2.641, 3.711, 4.112};
    double e[8] = {0, 106.7, 71.4, 195.2, 59.7, 809.1, 78.6, 335.4};
    for (int q = 0; q < 8; ++q) { P.gmw[q] = g[q] * 1.0e-3; P.mmugs[q] = s[q]; P.mmugek[q] = e[q]; }
    P.rgas = 8.31432;
    P.gammaair = 1.4;
    for (int is = 1; is <= ctx->ns; ++is) {
        P.dk[is] = c.dk[is - 1];
        P.rl[is] = c.rl[is - 1];
        P.inrl[is] = 1.0 / P.rl[is];
        P.phis[is] = c.phis[is - 1];
        P.cmus[is] = c.cmus[is - 1];
        P.cps[is] = c.cps[is - 1];
        P.kap[is] = c.kap[is - 1];
        P.plim[is] = c.plim[is - 1];
        P.phi[is] = (double)0.63f;
    }
    for (int k = 1; k <= ctx->ns; ++k)
        for (int kk = 1; kk <= ctx->ns; ++kk) {
            int k1, k2;
            if (P.dk[k] >= P.dk[kk]) { k1 = k; k2 = kk; }
            else { k1 = kk; k2 = k; }
            double a = std::sqrt(P.dk[k2] / P.dk[k1]);
            P.philim[k][kk] = P.phi[k1] / (P.phi[k1] + (1.0 - P.phi[k1]) * P.phi[k2]);
            P.epsl[k][kk] = (P.phi[k1] - P.phi[k2]) + ((1.0 - a) * (1.0 - P.phi[k1]) * P.phi[k2]);
            double fact = (P.phi[k1] + (1.0 - P.phi[k2]) * P.phi[k1]) / P.phi[k1];
            P.epsl[k][kk] = P.epsl[k][kk] * fact;
            P.epsu[k][kk] = (1.0 - a) * (P.phi[k1] + (1.0 - P.phi[k1]) * P.phi[k2]);
            double s2 = P.dk[k] + P.dk[kk];
            P.dkf[k][kk] = s2 * s2 / (P.rl[k] * P.dk[k] * P.dk[k] * P.dk[k] + P.rl[kk] * P.dk[kk] * P.dk[kk] * P.dk[kk]);
            P.dkf[kk][k] = P.dkf[k][kk];
        }
}

// immersed boundaries (pdac_cfg immb = 1): the checks the kernels rely on
// (every index the interpolations and fills reach lies in the mesh) and
// those the reference makes as it runs (bdry.f:111-113: every immersed or
// filled cell is a forcing point; interp.f:520-560: the external points of
// types 21 and 22 lie on the side their interpolation assumes)
int validate_ib(const pdac_cfg *c, std::string &why) {
    if (!c->immb) return 0;
    const bool d3 = c->job_type == 3;
    const int nx = c->nx, ny = d3 ? c->ny : 1, nz = c->nz;
    const long n = (long)nx * ny * nz;
    if (c->time_integration != 0) { why = "immersed boundaries with the explicit solver are not supported"; return 1; }
    if (!c->ib_faces || !c->ib_ivf || !c->x || !c->xb || !c->z || !c->zb || (d3 && (!c->y || !c->yb))) {
        why = "immb: the face factors, ivf and the mesh coordinates are required"; return 1;
    }
    for (int a = 0; a < 3; ++a) {
        if (a == 1 && !d3) continue;
        const int nfp = c->ib_nfp[a];
        if (nfp < 0 || !c->ib_num[a] || (nfp > 0 && (!c->ib_fp[a] || !c->ib_nsl[a]))) {
            why = "immb: forcing-point tables missing"; return 1;
        }
        for (long m = 0; m < n; ++m)
            if (c->ib_num[a][m] < 0 || c->ib_num[a][m] > nfp) { why = "immb: forcing-point number out of range"; return 1; }
        for (int f = 0; f < nfp; ++f) {
            const int *fp = c->ib_fp[a] + (size_t)6 * f;
            const int i = fp[0], j = fp[1], k = fp[2], kind = fp[3];
            if (i < 1 || i > nx || k < 1 || k > nz || (d3 && (j < 1 || j > ny))) {
                why = "immb: forcing point outside the mesh"; return 1;
            }
            if (!d3) {
                const double nsx = c->ib_nsl[a][(size_t)3 * f];
                const double cxi = (a == 0 ? c->xb : c->x)[i - 1];
                if ((kind == 22 && !(nsx < cxi)) || (kind == 21 && !(nsx > cxi))) {
                    why = "immb: control fpoint (interp.f:520-560)"; return 1;
                }
            } else {
                int di = 0, dj = 0, dk = 0;
                const int DI[9] = {0, -1, -1, 0, 1, 1, 1, 0, -1}, DJ[9] = {0, 0, -1, -1, -1, 0, 1, 1, 1};
                if (kind == 0 || kind == 20) dk = 1;
                else if (kind >= 1 && kind <= 8) { di = DI[kind]; dj = DJ[kind]; }
                else if (kind >= 21 && kind <= 28) { di = DI[kind - 20]; dj = DJ[kind - 20]; }
                else { why = "immb: 3D forcing-point type out of range"; return 1; }
                auto flat = [&](int ii, int jj, int kk) -> long {
                    if (ii < 1 || ii > nx || jj < 1 || jj > ny || kk < 1 || kk > nz) return -1;
                    return (ii - 1) + (long)nx * ((jj - 1) + (long)ny * (kk - 1));
                };
                const long q = flat(i + di, j + dj, k + dk), qq = flat(i + 2 * di, j + 2 * dj, k + 2 * dk);
                if (q < 0 || fp[4] != q) { why = "immb: index_q of a forcing point"; return 1; }
                if ((kind % 2 != 0 || kind == 0) && (qq < 0 || fp[5] != qq)) { why = "immb: index_qq of a forcing point"; return 1; }
            }
        }
    }
    for (long m = 0; m < n; ++m) {
        const int f = c->flag[m];
        if ((f == IMMB || f == FILLED1 || f == FILLED2) && !c->ib_num[0][m] && !(d3 && c->ib_num[1][m]) &&
            !c->ib_num[2][m]) {
            why = "immb: an immersed or filled cell is not a forcing point (bdry.f:111-113)"; return 1;
        }
    }
    return 0;
}

int validate(const pdac_cfg *c, std::string &why) {
    if (c->job_type != 2 && c->job_type != 3) { why = "job_type must be 2 (2D) or 3 (3D)"; return 1; }
    if (c->nx < 5 || c->nz < 5) { why = "nx and nz must be >= 5"; return 1; }
    if (c->job_type == 3 && c->ny < 5) { why = "ny must be >= 5 in 3D"; return 1; }
    if (c->job_type == 3 && c->itc != 0) { why = "3D runs are Cartesian (itc = 0)"; return 1; }
    if (c->job_type == 3 && !c->dy) { why = "dy pointer is NULL"; return 1; }
    if ((long)c->nx * (c->job_type == 3 ? c->ny : 1) * c->nz > 2000000000L) { why = "mesh too large"; return 1; }
    if (c->nsolid < 1 || c->nsolid > PDAC_MAX_NSOLID) { why = "nsolid out of range"; return 1; }
    if (c->ngas < 1 || c->ngas > PDAC_MAX_NGAS) { why = "ngas out of range"; return 1; }
    for (int ig = 0; ig < c->ngas; ++ig)
        if (c->gas_type[ig] < 1 || c->gas_type[ig] > 7) { why = "gas_type out of range"; return 1; }
    if (c->inmax < 1 || c->maxout < 1) { why = "inmax and maxout must be >= 1"; return 1; }
    if (c->rungekut < 1) { why = "rungekut must be >= 1"; return 1; }
    if (!c->dx || !c->dz || !c->flag || !c->p_atm || !c->t_atm) { why = "metric, flag or atmosphere pointer is NULL"; return 1; }
    if (c->nvent > 0 && !c->vent_ijk) { why = "vent_ijk is NULL"; return 1; }
    if (c->precision != PDAC_PREC_FP64 && c->precision != PDAC_PREC_MIXED) {
        why = "precision must be PDAC_PREC_FP64 or PDAC_PREC_MIXED";
        return 1;
    }
    if (c->time_integration != 0 && c->time_integration != 1) { why = "time_integration must be 0 or 1"; return 1; }
    if (c->iturb < 0 || c->iturb > 2) { why = "iturb must be 0, 1 or 2"; return 1; }
    if (c->iturb == 2 && !c->topo_c) { why = "iturb = 2 needs topo_c, the ground level of every column"; return 1; }
    if (c->iturb >= 1 && c->modturbo != 1 && c->modturbo != 2) {
        why = "modturbo must be 1 (static Smagorinsky) or 2 (dynamic; static in 2D, as turbo.f:180-185)";
        return 1;
    }
    if (c->iss != 0 && c->iss != 1) { why = "iss must be 0 or 1"; return 1; }
    if (c->implicit_fluxes && c->alpha != 1.0) { why = "implicit_fluxes needs alpha = 1"; return 1; }
    if (c->optimization < 1 || c->optimization > 3) { why = "optimization must be 1, 2 or 3"; return 1; }
    if (c->optimization == 3 && c->job_type == 3 && c->nsolid == 2) {
        why = "optimization = 3 in 3D with two classes (opt3_inner_loop) is not built";
        return 1;
    }
    if (c->time_integration == 1 && c->pmodel != 1 && c->pmodel != 2) {
        why = "time_integration = 1 needs pmodel 1 or 2 (explicit_solver.f:632-642)";
        return 1;
    }
    return validate_ib(c, why);
}

// The boundary cells of the ordered boundary pass (ib.cuh) in levels.  A
// fluid cell next to a wall or an open boundary reads itself and, along
// every such direction, the neighbour there and the first and second
// neighbours on the opposite side, and writes itself and that neighbour
// (bdry.f:208-726); a forcing point reads the cells its interpolation uses
// and writes itself and the neighbour hn may fill (bdry.f:103-204).  Cells
// are taken in index order; each goes one level after the last earlier cell
// that writes what it reads or touches what it writes.  Returns the cells
// sorted by level (index order within a level) and the level starts; no
// levels at all when every cell falls in the first level and there are no
// forcing points (one thread per cell then gives the same result).
void boundary_levels(const pdac_cfg *c, std::vector<int> &items, std::vector<int> &starts) {
    items.clear();
    starts.clear();
    const bool d3 = c->job_type == 3;
    const int nx = c->nx, ny = d3 ? c->ny : 1, nz = c->nz;
    const long n = (long)nx * ny * nz;
    const int *fl = c->flag;
    auto acts = [](int f) { return f == SLIP || f == NOSLIP || f == FREE_IO || f == ZERO_GRAD; };
    auto at = [&](int i, int j, int k) -> int {
        i = std::min(std::max(i, 1), nx); j = std::min(std::max(j, 1), ny); k = std::min(std::max(k, 1), nz);
        return (i - 1) + nx * ((j - 1) + ny * (k - 1));
    };
    std::vector<int> lw(n, 0), lt(n, 0);  // last level writing / touching each cell
    std::vector<std::pair<int, int>> lev;  // (level, cell)
    bool any_ib = false;
    int maxl = 0;
    std::vector<int> T, W;
    for (long m = 0; m < n; ++m) {
        const int f = fl[m];
        const int i = (int)(m % nx) + 1, j = (int)((m / nx) % ny) + 1, k = (int)(m / ((long)nx * ny)) + 1;
        T.assign(1, (int)m);
        W.assign(1, (int)m);
        if (c->immb && (f == IMMB || f == FILLED1 || f == FILLED2)) {
            any_ib = true;
            for (int a = 0; a < 3; ++a) {
                if (a == 1 && !d3) continue;
                const int num = c->ib_num[a][m];
                if (!num) continue;
                const int *fp = c->ib_fp[a] + (size_t)6 * (num - 1);
                if (d3) {
                    T.push_back(fp[4]);
                    if (fp[5] >= 0) T.push_back(fp[5]);
                } else {
                    for (int di : {-2, -1, 1, 2}) T.push_back(at(i + di, 1, k));
                    for (int dk : {1, 2}) T.push_back(at(i, 1, k + dk));
                    T.push_back(at(i + 1, 1, k + 1));
                    T.push_back(at(i - 1, 1, k + 1));
                }
                if (fp[3] >= 20) {  // hn on the neighbour along the axis
                    const int nb = a == 0 ? at(i + 1, j, k) : (a == 1 ? at(i, j + 1, k) : at(i, j, k + 1));
                    T.push_back(nb);
                    W.push_back(nb);
                }
            }
        } else if (f == FLUID || f == DOME || f == BL_CELL) {
            const int dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}, {0, 1, 0}, {0, -1, 0}};
            bool any = false;
            for (int d = 0; d < (d3 ? 6 : 4); ++d) {
                const int di = dirs[d][0], dj = dirs[d][1], dk = dirs[d][2];
                const int nb = at(i + di, j + dj, k + dk);
                if (!acts(fl[nb])) continue;
                any = true;
                T.push_back(nb);
                T.push_back(at(i - di, j - dj, k - dk));
                T.push_back(at(i - 2 * di, j - 2 * dj, k - 2 * dk));
                W.push_back(nb);
            }
            if (!any) continue;
        } else {
            continue;
        }
        int L = 0;
        for (int t : T) L = std::max(L, lw[t]);
        for (int w : W) L = std::max(L, lt[w]);
        ++L;
        for (int t : T) lt[t] = std::max(lt[t], L);
        for (int w : W) { lw[w] = std::max(lw[w], L); lt[w] = std::max(lt[w], L); }
        lev.push_back({L, (int)m});
        maxl = std::max(maxl, L);
    }
    if (maxl <= 1 && !any_ib) return;
    std::stable_sort(lev.begin(), lev.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
        return a.first < b.first;
    });
    int cur = 0;
    for (size_t q = 0; q < lev.size(); ++q) {
        while (cur < lev[q].first) { starts.push_back((int)q); ++cur; }
        items.push_back(lev[q].second);
    }
    starts.push_back((int)lev.size());
}

// The records of the explicit solver's gas-enthalpy wavefront (fixed by the
// cell flags): interior fluid cells in hyperplane order d = i + j + k (i + k
// in 2D), cell order within a hyperplane; empty hyperplanes are dropped, as
// no cell depends on one.  Also picks the cooperative grid.
int setup_wave(pdac_ctx *ctx, const int *flag) {
    const int nx = ctx->nx, ny = ctx->d3 ? ctx->ny : 1, nz = ctx->nz, n = ctx->ncell;
    const int jlo = ctx->d3 ? 2 : 1, jhi = ctx->d3 ? ny - 1 : 1;
    const int dmin = 2 + jlo + 2, dmax = (nx - 1) + jhi + (nz - 1);
    const int nd = dmax - dmin + 1;
    std::vector<int> count(nd + 1, 0), pos_of(n, -1);
    auto each = [&](auto fn) {
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = jlo; j <= jhi; ++j)
                for (int i = 2; i <= nx - 1; ++i) {
                    int c = (i - 1) + nx * ((j - 1) + ny * (k - 1));
                    if (flag[c] & 1) fn(c, i + j + k - dmin);
                }
    };
    each([&](int, int q) { count[q + 1]++; });
    std::vector<int> first(nd + 1, 0);
    for (int q = 0; q < nd; ++q) first[q + 1] = first[q] + count[q + 1];
    const int np = first[nd];
    std::vector<int> order(std::max(np, 1), 0), fill(first.begin(), first.end() - 1);
    each([&](int c, int q) {
        pos_of[c] = fill[q];
        order[fill[q]++] = c;
    });
    std::vector<int> start;
    int widest = 0;
    for (int q = 0; q < nd; ++q)
        if (first[q + 1] > first[q]) {
            start.push_back(first[q]);
            widest = std::max(widest, first[q + 1] - first[q]);
        }
    const int nplanes = (int)start.size();
    start.push_back(np);
    start.push_back(np);  // read one past the last hyperplane by the prefetch guard
    std::vector<int> src(3 * (size_t)std::max(np, 1), -1);
    for (int p = 0; p < np; ++p) {
        const int c = order[p];
        src[p] = pos_of[c - 1];
        if (ctx->d3) src[(size_t)np + p] = pos_of[c - nx];
        src[2 * (size_t)np + p] = pos_of[c - nx * ny];
    }
    const size_t ni = order.size() + src.size() + start.size() + pos_of.size();
    CK(cudaMalloc(&ctx->d_wave_idx, ni * sizeof(int)));
    int *o = ctx->d_wave_idx, *s = o + order.size(), *st = s + src.size(), *po = st + start.size();
    CK(cudaMemcpy(o, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(st, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(po, pos_of.data(), pos_of.size() * sizeof(int), cudaMemcpyHostToDevice));
    const size_t nrec = (size_t)(pdac::WR_YG + ctx->ng) + 1;  // the fields and pnew
    CK(cudaMalloc(&ctx->d_wave_rec, nrec * std::max(np, 1) * sizeof(double)));
    pdac::Wave &W = ctx->W;
    W.order = o;
    W.pos_of = po;
    W.src = s;
    W.start = st;
    W.rec = ctx->d_wave_rec;
    W.pnew = ctx->d_wave_rec + (nrec - 1) * std::max(np, 1);
    W.npos = np;
    W.nplanes = nplanes;
    W.dmin = dmin;
    // a cooperative grid of co-resident blocks: one record per thread and
    // hyperplane when the device holds enough blocks for the widest one
    int dev = 0, coop = 0, nsm = 0, occ1 = 0, occn = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ctx->wave_grid_blocks = 0;
    ctx->wave_one = false;
    if (!coop || np == 0) return PDAC_OK;
    if (ctx->d3) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, pdac::k_rk3_wave_rec<3, true>, TPB, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occn, pdac::k_rk3_wave_rec<3, false>, TPB, 0));
    } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, pdac::k_rk3_wave_rec<2, true>, TPB, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occn, pdac::k_rk3_wave_rec<2, false>, TPB, 0));
    }
    const int need = blocks(widest);
    if (need <= occ1 * nsm) {
        ctx->wave_grid_blocks = need;
        ctx->wave_one = true;
    } else {
        ctx->wave_grid_blocks = occn * nsm;
    }
    return PDAC_OK;
}

}  // namespace

// Domains of at most this many cells run iter's sweep loop as one
// cooperative launch (k_iter_coop): their colour phases are a few
// microseconds of work each, less than the launch of a graph node.
#ifndef PDAC_COOP_MAX_CELLS
#define PDAC_COOP_MAX_CELLS (1 << 18)
#endif
#ifndef PDAC_COOP_CELLS_PER_BLOCK
#define PDAC_COOP_CELLS_PER_BLOCK 1024
#endif

template <int NP>
static cudaError_t launch_iter_coop_np(pdac_ctx *ctx, double dt, cudaStream_t st, const pdac::SweepWork &W) {
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.gridDim = dim3(ctx->coop_blocks);
    lc.blockDim = dim3(TPB_TEAM);
    lc.dynamicSmemBytes = pdac::inner_smem_bytes<NP>();
    lc.stream = st;
    lc.attrs = at;
    lc.numAttrs = 1;
    if (ctx->d3) return cudaLaunchKernelEx(&lc, pdac::k_iter_coop<NP, 3>, ctx->P, ctx->F, dt, W, ctx->cfg.maxout);
    return cudaLaunchKernelEx(&lc, pdac::k_iter_coop<NP, 2>, ctx->P, ctx->F, dt, W, ctx->cfg.maxout);
}

static cudaError_t launch_iter_coop(pdac_ctx *ctx, double dt, cudaStream_t st, const pdac::SweepWork &W) {
    switch (ctx->nph) {
        case 2: return launch_iter_coop_np<2>(ctx, dt, st, W);
        case 3: return launch_iter_coop_np<3>(ctx, dt, st, W);
        case 4: return launch_iter_coop_np<4>(ctx, dt, st, W);
        case 6: return launch_iter_coop_np<6>(ctx, dt, st, W);
        default: return launch_iter_coop_np<0>(ctx, dt, st, W);
    }
}

// the cooperative grid of a small domain: one block of 128 threads per
// PDAC_COOP_CELLS_PER_BLOCK cells, within what the device holds at once
// (measured on the 128 x 192 2D plume: 1024 and 256 cells per block run
// the step in 6.43 ms, 4096 in 7.46 ms, 64 in 6.76 ms)
static int setup_iter_coop(pdac_ctx *ctx) {
    ctx->coop_blocks = 0;
    if ((long)ctx->ncell > PDAC_COOP_MAX_CELLS) return PDAC_OK;
    int dev = 0, coop = 0, nsm = 0, occ = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (!coop) return PDAC_OK;
    auto occ_of = [&](auto kernel, size_t smem) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, TPB_TEAM, smem);
    };
    cudaError_t e;
    switch (ctx->nph) {
        case 2: e = ctx->d3 ? occ_of(pdac::k_iter_coop<2, 3>, pdac::inner_smem_bytes<2>())
                            : occ_of(pdac::k_iter_coop<2, 2>, pdac::inner_smem_bytes<2>()); break;
        case 3: e = ctx->d3 ? occ_of(pdac::k_iter_coop<3, 3>, pdac::inner_smem_bytes<3>())
                            : occ_of(pdac::k_iter_coop<3, 2>, pdac::inner_smem_bytes<3>()); break;
        case 4: e = ctx->d3 ? occ_of(pdac::k_iter_coop<4, 3>, pdac::inner_smem_bytes<4>())
                            : occ_of(pdac::k_iter_coop<4, 2>, pdac::inner_smem_bytes<4>()); break;
        case 6: e = ctx->d3 ? occ_of(pdac::k_iter_coop<6, 3>, pdac::inner_smem_bytes<6>())
                            : occ_of(pdac::k_iter_coop<6, 2>, pdac::inner_smem_bytes<6>()); break;
        default: e = ctx->d3 ? occ_of(pdac::k_iter_coop<0, 3>, pdac::inner_smem_bytes<0>())
                             : occ_of(pdac::k_iter_coop<0, 2>, pdac::inner_smem_bytes<0>()); break;
    }
    CK(e);
    ctx->coop_cpb = PDAC_COOP_CELLS_PER_BLOCK;
    ctx->coop_max_blocks = occ * nsm;
    const int want = std::max(1, (int)((ctx->ncell + ctx->coop_cpb - 1) / ctx->coop_cpb));
    ctx->coop_blocks = std::min(want, ctx->coop_max_blocks);
    return PDAC_OK;
}

extern "C" {

const char *pdac_gpu_last_error(const pdac_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int pdac_gpu_create(const pdac_cfg *cfg, pdac_ctx **out) {
    if (!cfg || !out) return PDAC_ERR_ARG;
    *out = nullptr;
    std::string why;
    if (validate(cfg, why)) {
        fprintf(stderr, "pdac_gpu_create: %s\n", why.c_str());
        return PDAC_ERR_CONFIG;
    }
    pdac_ctx *ctx = new pdac_ctx();
    ctx->cfg = *cfg;
    ctx->d3 = cfg->job_type == 3;
    ctx->nx = cfg->nx; ctx->ny = ctx->d3 ? cfg->ny : 1; ctx->nz = cfg->nz;
    ctx->ncell = ctx->nx * ctx->ny * ctx->nz;
    ctx->ns = cfg->nsolid; ctx->ng = cfg->ngas; ctx->nph = ctx->ns + 1; ctx->nap = ctx->nph * (ctx->nph + 1) / 2;
    int n = ctx->ncell, ns = ctx->ns, ng = ctx->ng, nap = ctx->nap;
    Prm &P = ctx->P;
    std::memset(&P, 0, sizeof(P));
    P.nx = ctx->nx; P.ny = ctx->ny; P.nz = ctx->nz; P.ncell = n; P.d3 = ctx->d3 ? 1 : 0; P.ns = ns; P.ng = ng; P.nph = ctx->nph; P.nap = nap;
    P.itc = cfg->itc; P.muscl = cfg->muscl; P.lv = cfg->lv; P.lm = cfg->lm; P.pmodel = cfg->pmodel;
    P.drag_model = cfg->drag_model; P.icpc = cfg->icpc; P.gas_viscosity = cfg->gas_viscosity;
    P.part_viscosity = cfg->part_viscosity; P.repulsive_model = cfg->repulsive_model; P.inmax = cfg->inmax;
    P.iturb = cfg->iturb; P.iss = cfg->iss; P.modturbo = cfg->modturbo;
    P.opt = cfg->optimization >= 2 ? 2 : 1;  // 3 runs as 2 outside 3D with two classes (iter.f:160-161)
    {  // the multipliers of ijk_of, checked on every cell index of this mesh
        auto magic = [&](unsigned d) -> unsigned long long {
            if (d < 2) return 0ull;
            unsigned long long m = ~0ull / d + 1ull;
            const unsigned nmax = (unsigned)n;
            for (unsigned c = 0; c < nmax; ++c)
                if ((unsigned)(((unsigned __int128)c * m) >> 64) != c / d) return 0ull;
            return m;
        };
        P.mnx = ctx->d3 ? magic((unsigned)ctx->nx) : 0ull;
        P.mny = ctx->d3 ? magic((unsigned)ctx->ny) : 0ull;
    }
    for (int ig = 0; ig < ng; ++ig) P.gas_type[ig] = cfg->gas_type[ig];
    P.alpha = cfg->alpha; P.alphagrav = cfg->alphagrav; P.omega = cfg->omega; P.delg = cfg->delg;
    P.beta = cfg->beta; P.flim = cfg->flim; P.tref = cfg->tref;
    P.gravx = cfg->gravx; P.gravy = cfg->gravy; P.gravz = cfg->gravz; P.void_fraction = cfg->void_fraction;
    for (int g = 0; g < PDAC_MAX_NGAS; ++g) P.atm_ygc[g] = cfg->atm_ygc[g];
    set_constants(ctx);

    // host metric, 1-based padded, grid.f:306-345
    int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    std::vector<double> dx(nx + 4), dz(nz + 4), indx(nx + 4), indz(nz + 4), r(nx + 4, 1.0), rb(nx + 4, 1.0),
        inr(nx + 4, 1.0), inrb(nx + 4, 1.0), patm(nz + 2, 0.0), tatm(nz + 2, 0.0), dy(ny + 4, 0.0), indy(ny + 4, 0.0);
    for (int i = 1; i <= nx; ++i) dx[i] = cfg->dx[i - 1];
    dx[0] = dx[1]; dx[nx + 1] = dx[nx + 2] = dx[nx + 3] = dx[nx];
    for (int k = 1; k <= nz; ++k) dz[k] = cfg->dz[k - 1];
    dz[0] = dz[1]; dz[nz + 1] = dz[nz + 2] = dz[nz + 3] = dz[nz];
    for (int i = 0; i < nx + 4; ++i) indx[i] = 1.0 / dx[i];
    for (int k = 0; k < nz + 4; ++k) indz[k] = 1.0 / dz[k];
    if (ctx->d3) {
        for (int j = 1; j <= ny; ++j) dy[j] = cfg->dy[j - 1];
        dy[0] = dy[1]; dy[ny + 1] = dy[ny + 2] = dy[ny + 3] = dy[ny];
        for (int j = 0; j < ny + 4; ++j) indy[j] = 1.0 / dy[j];
    }
    if (cfg->itc == 1) {
        std::vector<double> xb(nx + 4, 0.0), x(nx + 4, 0.0);
        xb[1] = 0.0; x[1] = -0.5 * dx[1] + xb[1];
        for (int i = 2; i <= nx; ++i) { xb[i] = (xb[i - 1] + dx[i]); x[i] = (xb[i] - 0.5 * dx[i]); }
        for (int i = 1; i <= nx; ++i) { r[i] = x[i]; rb[i] = xb[i]; }
        rb[0] = rb[1] - dx[1];
        inrb[1] = (rb[1] == 0.0) ? 1.0e10 : 1.0 / rb[1];
        for (int i = 2; i <= nx; ++i) inrb[i] = 1.0 / rb[i];
        for (int i = 1; i <= nx; ++i) inr[i] = 1.0 / r[i];
    }
    for (int k = 1; k <= nz; ++k) { patm[k] = cfg->p_atm[k - 1]; tatm[k] = cfg->t_atm[k - 1]; }
    // reciprocal face spacings; the last entry pairs the padding with itself
    auto recip = [](const std::vector<double> &d, bool on) {
        std::vector<double> h(d.size(), 0.0);
        if (on)
            for (size_t m = 0; m < d.size(); ++m) h[m] = 1.0 / (d[m] + d[std::min(m + 1, d.size() - 1)]);
        return h;
    };
    std::vector<double> hx = recip(dx, true), hy = recip(dy, ctx->d3), hz = recip(dz, true);

    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    for (auto &e : ctx->ev) CK(cudaEventCreate(&e));
    for (auto &e : ctx->cev) CK(cudaEventCreate(&e));
    for (auto &e : ctx->user_ev) CK(cudaEventCreate(&e));
    for (auto &e : ctx->xev) CK(cudaEventCreate(&e));
    std::vector<std::vector<double> *> mets = {&dx, &dy, &dz, &indx, &indy, &indz, &r, &rb, &inr, &inrb, &patm, &tatm,
                                               &hx, &hy, &hz};
    size_t mtot = 0;
    for (auto *v : mets) mtot += v->size();
    CK(cudaMalloc(&ctx->metric, mtot * sizeof(double)));
    size_t off = 0;
    std::vector<const double *> mp;
    for (auto *v : mets) {
        CK(cudaMemcpy(ctx->metric + off, v->data(), v->size() * sizeof(double), cudaMemcpyHostToDevice));
        mp.push_back(ctx->metric + off);
        off += v->size();
    }
    P.dx = mp[0]; P.dy = mp[1]; P.dz = mp[2]; P.indx = mp[3]; P.indy = mp[4]; P.indz = mp[5];
    P.r = mp[6]; P.rb = mp[7]; P.inr = mp[8]; P.inrb = mp[9]; P.p_atm = mp[10]; P.t_atm = mp[11];
    P.hx = mp[12]; P.hy = mp[13]; P.hz = mp[14];
    P.mixed = cfg->precision == PDAC_PREC_MIXED;
    if (P.mixed) {  // the metric of the FP32 flux passes: each FP64 value rounded to nearest
        const int qs[11] = {0, 1, 2, 3, 4, 5, 12, 13, 14, 6, 7};
        size_t ftot = 0;
        for (int q : qs) ftot += mets[q]->size();
        std::vector<float> hf;
        hf.reserve(ftot);
        for (int q : qs)
            for (double v : *mets[q]) hf.push_back((float)v);
        CK(cudaMalloc(&ctx->metric_f, ftot * sizeof(float)));
        CK(cudaMemcpy(ctx->metric_f, hf.data(), ftot * sizeof(float), cudaMemcpyHostToDevice));
        const float *fp[11];
        size_t fo = 0;
        for (int q = 0; q < 11; ++q) { fp[q] = ctx->metric_f + fo; fo += mets[qs[q]]->size(); }
        P.dxf = fp[0]; P.dyf = fp[1]; P.dzf = fp[2]; P.indxf = fp[3]; P.indyf = fp[4]; P.indzf = fp[5];
        P.hxf = fp[6]; P.hyf = fp[7]; P.hzf = fp[8]; P.rf = fp[9]; P.rbf = fp[10];
    }
    CK(cudaMalloc(&ctx->d_flag, n * sizeof(int)));
    CK(cudaMemcpy(ctx->d_flag, cfg->flag, n * sizeof(int), cudaMemcpyHostToDevice));
    P.flag = ctx->d_flag;
    // immersed boundaries: the tables and coordinates (read-only) and the
    // state the boundary pass hands to tilde and to the next pass
    P.immb = cfg->immb ? 1 : 0;
    if (P.immb) {
        const int nfp[3] = {cfg->ib_nfp[0], ctx->d3 ? cfg->ib_nfp[1] : 0, cfg->ib_nfp[2]};
        std::vector<int> hint((size_t)4 * n + (size_t)6 * (nfp[0] + nfp[1] + nfp[2]), 0);
        std::copy(cfg->ib_faces, cfg->ib_faces + n, hint.begin());
        size_t io = (size_t)n;
        size_t inum[3], ifp[3];
        for (int a = 0; a < 3; ++a) {
            inum[a] = io;
            if (nfp[a] > 0 || cfg->ib_num[a]) {
                if (a != 1 || ctx->d3) std::copy(cfg->ib_num[a], cfg->ib_num[a] + n, hint.begin() + io);
            }
            io += n;
        }
        for (int a = 0; a < 3; ++a) {
            ifp[a] = io;
            if (nfp[a] > 0) std::copy(cfg->ib_fp[a], cfg->ib_fp[a] + (size_t)6 * nfp[a], hint.begin() + io);
            io += (size_t)6 * nfp[a];
        }
        const int lens[6] = {ctx->nx, ctx->nx, ctx->ny, ctx->ny, ctx->nz, ctx->nz};
        const double *srcs[6] = {cfg->x, cfg->xb, ctx->d3 ? cfg->y : nullptr, ctx->d3 ? cfg->yb : nullptr, cfg->z, cfg->zb};
        size_t nd = (size_t)n + 3 * ((size_t)nfp[0] + nfp[1] + nfp[2]);
        for (int q = 0; q < 6; ++q) nd += lens[q] + 5;
        std::vector<double> hdbl(nd, 0.0);
        std::copy(cfg->ib_ivf, cfg->ib_ivf + n, hdbl.begin());
        size_t dofs = (size_t)n, dnsl[3], dcrd[6];
        for (int a = 0; a < 3; ++a) {
            dnsl[a] = dofs;
            if (nfp[a] > 0) std::copy(cfg->ib_nsl[a], cfg->ib_nsl[a] + (size_t)3 * nfp[a], hdbl.begin() + dofs);
            dofs += (size_t)3 * nfp[a];
        }
        for (int q = 0; q < 6; ++q) {  // 1-based, two cells of padding: a[q + 1]
            dcrd[q] = dofs;
            const int m = lens[q];
            double *d = hdbl.data() + dofs;
            if (srcs[q]) {
                for (int t = 1; t <= m; ++t) d[t + 1] = srcs[q][t - 1];
                d[0] = d[1] = d[2];
                d[m + 3] = d[m + 4] = d[m + 2];
            }
            dofs += m + 5;
        }
        CK(cudaMalloc(&ctx->d_ibint, hint.size() * sizeof(int)));
        CK(cudaMemcpy(ctx->d_ibint, hint.data(), hint.size() * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&ctx->d_ibdbl, hdbl.size() * sizeof(double)));
        CK(cudaMemcpy(ctx->d_ibdbl, hdbl.data(), hdbl.size() * sizeof(double), cudaMemcpyHostToDevice));
        ctx->ibstate_doubles = (size_t)ctx->nph * (nfp[0] + nfp[1] + nfp[2]) + (size_t)n;
        CK(cudaMalloc(&ctx->d_ibstate, ctx->ibstate_doubles * sizeof(double)));
        CK(cudaMemset(ctx->d_ibstate, 0, ctx->ibstate_doubles * sizeof(double)));
        P.ib_faces = ctx->d_ibint;
        P.ib_ivf = ctx->d_ibdbl;
        size_t vo = 0;
        for (int a = 0; a < 3; ++a) {
            P.ib_num[a] = ctx->d_ibint + inum[a];
            ctx->IB.fp[a] = ctx->d_ibint + ifp[a];
            ctx->IB.nsl[a] = ctx->d_ibdbl + dnsl[a];
            ctx->IB.vel[a] = ctx->d_ibstate + vo;
            P.ib_vel[a] = ctx->IB.vel[a];
            vo += (size_t)ctx->nph * nfp[a];
        }
        ctx->IB.fc2 = ctx->d_ibstate + vo;
        ctx->IB.x = ctx->d_ibdbl + dcrd[0]; ctx->IB.xb = ctx->d_ibdbl + dcrd[1];
        ctx->IB.y = ctx->d_ibdbl + dcrd[2]; ctx->IB.yb = ctx->d_ibdbl + dcrd[3];
        ctx->IB.z = ctx->d_ibdbl + dcrd[4]; ctx->IB.zb = ctx->d_ibdbl + dcrd[5];
    }
    {  // the ordered boundary pass, where cells' boundary updates meet
        std::vector<int> items;
        boundary_levels(cfg, items, ctx->blevel);
        if (!items.empty()) {
            CK(cudaMalloc(&ctx->d_bitems, items.size() * sizeof(int)));
            CK(cudaMemcpy(ctx->d_bitems, items.data(), items.size() * sizeof(int), cudaMemcpyHostToDevice));
        }
    }
    ctx->nvent = cfg->nvent;
    int nv = std::max(1, cfg->nvent);
    CK(cudaMalloc(&ctx->d_vent, nv * sizeof(int)));
    CK(cudaMalloc(&ctx->d_vfact, nv * sizeof(double)));
    CK(cudaMalloc(&ctx->d_vfact0, nv * sizeof(double)));
    if (cfg->nvent > 0) {
        CK(cudaMemcpy(ctx->d_vent, cfg->vent_ijk, cfg->nvent * sizeof(int), cudaMemcpyHostToDevice));
        // vent.f:176-178 initialises fact = 1 and fact0 = 0; random_switch
        // (vent.f:824-873) redraws fact only in 3D
        std::vector<double> one(cfg->nvent, 1.0), zero(cfg->nvent, 0.0);
        CK(cudaMemcpy(ctx->d_vfact, one.data(), cfg->nvent * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->d_vfact0, zero.data(), cfg->nvent * sizeof(double), cudaMemcpyHostToDevice));
    }
    // a colour phase holds at most ceil(nx / 3) * ny * nz cells: for fixed
    // (j, k), (i + j + k) mod 3 takes one value on every third i
    ctx->work_stride = ((long)((ctx->nx + 2) / 3) * ctx->ny * ctx->nz + 63) / 64 * 64;
    CK(cudaMalloc(&ctx->d_work, (size_t)3 * ctx->work_stride * sizeof(int)));
    CK(cudaMalloc(&ctx->d_nonfinite, sizeof(int)));
    CK(cudaMallocHost(&ctx->h_nonfinite, sizeof(int)));
    CK(cudaMalloc(&ctx->d_status, 4 * sizeof(int)));
    CK(cudaMallocHost(&ctx->h_status, 4 * sizeof(int)));
    CK(cudaMalloc(&ctx->d_wcount, 16 * sizeof(int)));
    CK(cudaMalloc(&ctx->d_dirty, ((size_t)n + 31) / 32 * sizeof(unsigned)));
    CK(cudaMalloc(&ctx->d_cand, (size_t)n * sizeof(int)));
    {
        int dev = 0, nsm = 148;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        ctx->inner_grid = nsm * 16;
    }
    CK(cudaMalloc(&ctx->d_nit, sizeof(int)));
    CK(cudaMallocHost(&ctx->h_nit, sizeof(int)));
    CK(cudaMalloc(&ctx->d_counters, 8 * sizeof(int)));
    CK(cudaMemset(ctx->d_counters, 0, 8 * sizeof(int)));
    CK(cudaMallocHost(&ctx->h_counters, 8 * sizeof(int)));

    // field arena: (name, number of ncell blocks)
    Fld &F = ctx->F;
    struct Slot { const char *name; double **ptr; int blocks; };
    // 2D-only and 3D-only slots get zero blocks on the other path, the
    // previous-visit interphase copies exist only when alpha < 1
    int d3 = ctx->d3 ? 1 : 0, d2 = 1 - d3, a0 = cfg->alpha != 1.0 ? 1 : 0;
    ctx->ti = cfg->time_integration;
    // the explicit solver's own fields exist only when it is selected; its
    // right-hand-side rows: mass, momentum per axis and enthalpy of each phase
    int t1 = ctx->ti == 1 ? 1 : 0, neq = (ctx->d3 ? 5 : 4) * ctx->nph;
    int lt = cfg->iturb >= 1 ? 1 : 0, ls = cfg->iss >= 1 ? 1 : 0;  // sub-grid model fields
    int ld = lt && ctx->d3 && cfg->modturbo == 2 ? 1 : 0;              // the dynamic model's
    int lmix = cfg->compute_mixture ? 1 : 0;                           // mixture fields
    RkF &K = ctx->K;
    std::vector<Slot> slots = {
        {"p", &F.p, 1}, {"ep", &F.ep, 1}, {"rog", &F.rog, 1}, {"rgp", &F.rgp, 1}, {"tg", &F.tg, 1},
        {"sieg", &F.sieg, 1}, {"cg", &F.cg, 1}, {"ug", &F.ug, 1}, {"vg", &F.vg, 1}, {"wg", &F.wg, 1},
        {"rlk", &F.rlk, ns}, {"ts", &F.ts, ns}, {"sies", &F.sies, ns}, {"us", &F.us, ns}, {"vs", &F.vs, ns},
        {"ws", &F.ws, ns}, {"ygc", &F.ygc, ng}, {"xgc", &F.xgc, ng},
        {"pn", &F.pn, 1}, {"epn", &F.epn, 1}, {"rgpn", &F.rgpn, 1}, {"siegn", &F.siegn, 1},
        {"rlkn", &F.rlkn, ns}, {"siesn", &F.siesn, ns}, {"rgpgcn", &F.rgpgcn, ng}, {"mug", &F.mug, 1},
        {"kapg", &F.kapg, 1}, {"rugn", &F.rugn, 1}, {"rvgn", &F.rvgn, d3}, {"rwgn", &F.rwgn, 1},
        {"rusn", &F.rusn, ns}, {"rvsn", &F.rvsn, ns * d3}, {"rwsn", &F.rwsn, ns},
        {"rug", &F.rug, 1}, {"rvg", &F.rvg, d3}, {"rwg", &F.rwg, 1}, {"rus", &F.rus, ns},
        {"rvs", &F.rvs, ns * d3}, {"rws", &F.rws, ns}, {"appu", &F.appu, nap}, {"appv", &F.appv, nap * d3},
        {"appw", &F.appw, nap},
        {"ugfe", &F.ugfe, d2}, {"ugft", &F.ugft, d2}, {"wgfe", &F.wgfe, d2}, {"wgft", &F.wgft, d2},
        {"usfe", &F.usfe, ns * d2}, {"usft", &F.usft, ns * d2}, {"wsfe", &F.wsfe, ns * d2},
        {"wsft", &F.wsft, ns * d2}, {"mf", &F.mf, 9 * (ns + 1) * d3},
        {"vis", &F.vis, 3 * (ns + 1) * std::max(d3, t1)},
        {"rgfe", &F.rgfe, 1}, {"rgfn", &F.rgfn, d3}, {"rgft", &F.rgft, 1}, {"rsfe", &F.rsfe, ns},
        {"rsfn", &F.rsfn, ns * d3}, {"rsft", &F.rsft, ns},
        {"conv", &F.conv, 1}, {"abeta", &F.abeta, 1}, {"egfe", &F.egfe, 1}, {"egfn", &F.egfn, d3},
        {"egft", &F.egft, 1}, {"esfe", &F.esfe, ns}, {"esfn", &F.esfn, ns * d3}, {"esft", &F.esft, ns},
        {"rhg", &F.rhg, 1}, {"rhs", &F.rhs, ns},
        {"yfe", &F.yfe, ng}, {"yfn", &F.yfn, ng * d3}, {"yft", &F.yft, ng}, {"sink", &F.sink, ns},
        {"app0u", &ctx->d_app0u, nap * a0}, {"app0v", &ctx->d_app0v, nap * a0 * d3},
        {"app0w", &ctx->d_app0w, nap * a0},
        {"ugn", &K.ugn, t1}, {"vgn", &K.vgn, t1 * d3}, {"wgn", &K.wgn, t1}, {"usn", &K.usn, ns * t1},
        {"vsn", &K.vsn, ns * t1 * d3}, {"wsn", &K.wsn, ns * t1}, {"hv", &K.hv, ns * t1},
        {"k1", &K.k1, neq * t1}, {"k2", &K.k2, neq * t1}, {"xrgp", &K.xrgp, t1}, {"xrlk", &K.xrlk, ns * t1},
        {"xep", &K.xep, t1}, {"xug", &K.xug, t1}, {"xvg", &K.xvg, t1 * d3}, {"xwg", &K.xwg, t1},
        {"smag", &F.smag, lt}, {"mugt", &F.mugt, lt}, {"kapgt", &F.kapgt, lt}, {"must", &F.must, ns * ls},
        {"sgsdyn", &F.dyn, pdac::DY_N * ld}, {"delt", &F.delt, ld}, {"scoeff", &F.scoeff, ld},
        {"rhom", &F.rhom, lmix}, {"um", &F.um, lmix}, {"vm", &F.vm, lmix * d3}, {"wm", &F.wm, lmix},
        {"tm", &F.tm, lmix}, {"yd", &F.yd, (ng + ns) * lmix}};
    // each field starts on a 256-byte boundary
    size_t stride = ((size_t)n + 31) / 32 * 32;
    size_t total = 0;
    for (auto &s : slots) total += stride * s.blocks;
    ctx->arena_doubles = total;
    CK(cudaMalloc(&ctx->arena, total * sizeof(double)));
    CK(cudaMemset(ctx->arena, 0, total * sizeof(double)));
    size_t o2 = 0;
    for (auto &s : slots) {
        if (s.blocks == 0) { *s.ptr = nullptr; continue; }
        *s.ptr = ctx->arena + o2;
        ctx->names.push_back({s.name, {*s.ptr, (size_t)n * s.blocks}});
        o2 += stride * s.blocks;
    }
    // per-class blocks inside a slot are exactly ncell apart, as the
    // reference's (ncell, n) column-major arrays; the stride pads slot ends
    F.counters = ctx->d_counters;
    if (lt) {
        // turbulence_setup (turbo.f:42-108): smag = lm^2 with the
        // Smagorinsky length lm = cmut delta, delta = sqrt(dz dx) in 2D and
        // (dz dy dx)^(1/3) in 3D (times anis in 3D).  With iturb = 2 a cell
        // whose centre is zsgs = z(k) - topo_c above the ground matches it
        // with the roughness length lb = 0.4 (zsgs + zrough):
        // lm = sqrt(1 / (1 / ls^2 + 1 / lb^2)); a cell at or below the ground
        // keeps the lm of the cell before it in the loop, as the reference's
        // loop variable does (0 before the first assigned cell, which the
        // reference leaves undefined; only fluid cells, all above the
        // ground, use smag)
        std::vector<double> smag(n);
        double lm = 0.0;
        auto rough = [&](double ls, double zsgs) {
            if (cfg->iturb == 1) { lm = ls; return; }
            if (zsgs > 0.0) {
                double lb = 0.4 * (zsgs + cfg->zrough);
                lm = std::sqrt(1.0 / (1.0 / (ls * ls) + 1.0 / (lb * lb)));
            }
        };
        for (int c = 0; c < n; ++c) {
            int i = c % nx + 1, j = (c / nx) % ny + 1, k = c / (nx * ny) + 1;
            if (!ctx->d3) {
                double delt = std::sqrt(dz[k] * dx[i]);
                double ls = cfg->cmut * delt;
                rough(ls, cfg->iturb == 2 ? cfg->z[k - 1] - cfg->topo_c[i - 1] : 0.0);
                smag[c] = lm * lm;
            } else {
                double delt = std::pow(dz[k] * dy[j] * dx[i], 1.0 / 3.0);
                double ls = cfg->cmut * delt;
                rough(ls, cfg->iturb == 2 ? cfg->z[k - 1] - cfg->topo_c[(size_t)(j - 1) * nx + (i - 1)] : 0.0);
                smag[c] = lm * lm;
                // anis, turbo.f:670-700
                double deltamax = std::max(dx[i], std::max(dy[j], dz[k]));
                double a1 = dx[i] / deltamax, a2 = dy[j] / deltamax, a3 = dz[k] / deltamax;
                double la1 = std::log(a1), la2 = std::log(a2), la3 = std::log(a3);
                double fla = la1 * la1 + la2 * la2 + la3 * la3 - la1 * la2 + la1 * la3 - la2 * la3;
                fla = 4.0 / 27.0 * fla;
                fla = std::sqrt(fla);
                smag[c] = smag[c] * std::cosh(fla);
            }
        }
        CK(cudaMemcpy(F.smag, smag.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (ld) {
        // the dynamic model's filter width, (dz dy dx)^(1/3) (turbo.f:318)
        std::vector<double> delt(n);
        for (int c = 0; c < n; ++c) {
            int i = c % nx + 1, j = (c / nx) % ny + 1, k = c / (nx * ny) + 1;
            delt[c] = std::pow(dz[k] * dy[j] * dx[i], 1.0 / 3.0);
        }
        CK(cudaMemcpy(F.delt, delt.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    }
    int nq = 1 + ns + ng;
    CK(cudaMalloc(&ctx->d_partial, (size_t)nq * 1024 * sizeof(double)));
    if (ctx->d3) CK(set_tile_attrs(ctx->P, ctx->F));
    CK(set_inner_attrs());
    if (t1) {
        int st = setup_wave(ctx, cfg->flag);
        if (st) return st;
    } else {
        int st = setup_iter_coop(ctx);
        if (st) return st;
    }
    if (cfg->isink > 0) {
        // allocate_sink (sink.f:22-43); the ring test of sink_update
        // (sink.f:95-96) per ground column from the cell-centre coordinates
        // of grid.f:286-298 (dy = 0 in 2D, so y(1) = 0)
        const int ntr = ctx->d3 ? nx * ny : nx;
        std::vector<double> xc(nx + 1, 0.0), yc(ny + 1, 0.0);
        double xb = 0.0;
        xc[1] = -0.5 * dx[1] + xb;
        for (int i = 2; i <= nx; ++i) { xb = (xb + dx[i]); xc[i] = (xb - 0.5 * dx[i]); }
        if (ctx->d3) {
            double yb = 0.0;
            yc[1] = -0.5 * dy[1] + yb;
            for (int j = 2; j <= ny; ++j) { yb = yb + dy[j]; yc[j] = (yb - 0.5 * dy[j]); }
        }
        std::vector<int> ring(ntr);
        const double rprox2 = cfg->rprox * cfg->rprox, rdist2 = cfg->rdist * cfg->rdist;
        for (int b = 0; b < ntr; ++b) {
            int i = b % nx + 1, j = ctx->d3 ? b / nx + 1 : 1;
            double cx = xc[i] - cfg->center_x, cy = yc[j] - cfg->center_y;
            double dist2 = cx * cx + cy * cy;
            ring[b] = (dist2 > rprox2 && dist2 < rdist2) ? 1 : 0;
        }
        const size_t nm = (size_t)ntr * ns;
        CK(cudaMalloc(&ctx->d_sinkbuf, 2 * nm * sizeof(double)));
        CK(cudaMemset(ctx->d_sinkbuf, 0, 2 * nm * sizeof(double)));
        CK(cudaMalloc(&ctx->d_ring, ntr * sizeof(int)));
        CK(cudaMemcpy(ctx->d_ring, ring.data(), ntr * sizeof(int), cudaMemcpyHostToDevice));
        ctx->S.massl = ctx->d_sinkbuf;
        ctx->S.mass_loss = ctx->d_sinkbuf + nm;
        ctx->S.ring = ctx->d_ring;
        ctx->S.ntr = ntr;
        ctx->names.push_back({"massl", {ctx->S.massl, nm}});
        ctx->names.push_back({"mass_loss", {ctx->S.mass_loss, nm}});
    }
    *out = ctx;
    return PDAC_OK;
}

int pdac_gpu_destroy(pdac_ctx *ctx) {
    if (!ctx) return PDAC_ERR_ARG;
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->arena);
    cudaFree(ctx->metric);
    cudaFree(ctx->metric_f);
    cudaFree(ctx->d_flag);
    cudaFree(ctx->d_vent);
    cudaFree(ctx->d_vfact);
    cudaFree(ctx->d_vfact0);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->d_work);
    cudaFree(ctx->d_nonfinite);
    cudaFreeHost(ctx->h_nonfinite);
    if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
    if (ctx->step_graph) cudaGraphDestroy(ctx->step_graph);
    cudaFree(ctx->d_status);
    cudaFreeHost(ctx->h_status);
    cudaFree(ctx->d_wcount);
    cudaFree(ctx->d_dirty);
    if (ctx->it_exec) cudaGraphExecDestroy(ctx->it_exec);
    if (ctx->it_graph) cudaGraphDestroy(ctx->it_graph);
    if (ctx->ex_exec) cudaGraphExecDestroy(ctx->ex_exec);
    if (ctx->ex_graph) cudaGraphDestroy(ctx->ex_graph);
    cudaFree(ctx->d_nit);
    cudaFreeHost(ctx->h_nit);
    cudaFree(ctx->d_cand);
    cudaFree(ctx->d_partial);
    cudaFree(ctx->d_sinkbuf);
    cudaFree(ctx->d_ring);
    cudaFree(ctx->d_wave_idx);
    cudaFree(ctx->d_wave_rec);
    cudaFree(ctx->d_ibint);
    cudaFree(ctx->d_ibdbl);
    cudaFree(ctx->d_ibstate);
    cudaFree(ctx->d_bitems);
    cudaFreeHost(ctx->h_counters);
    for (auto &e : ctx->ev) cudaEventDestroy(e);
    for (auto &e : ctx->cev) cudaEventDestroy(e);
    for (auto &e : ctx->user_ev) cudaEventDestroy(e);
    for (auto &e : ctx->xev) cudaEventDestroy(e);
    for (auto &e : ctx->fev) if (e) cudaEventDestroy(e);
    if (ctx->up_done) cudaEventDestroy(ctx->up_done);
    if (ctx->up_stream) cudaStreamDestroy(ctx->up_stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PDAC_OK;
}

namespace pdac {
// up to 24 device arrays of doubles to scan for NaN / Inf
struct FinList {
    const double *a[24];
    long long n[24];
    int m;
};

// sets *flag when any value of the listed arrays is not finite; 16-byte
// loads over each array's even-length body (every arena slot starts on a
// 256-byte boundary), one scalar load for an odd tail
__global__ void __launch_bounds__(256) k_nonfinite(FinList L, int *flag) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nthr = (long long)gridDim.x * blockDim.x;
    bool bad = false;
    for (int q = 0; q < L.m; ++q) {
        const double2 *v = reinterpret_cast<const double2 *>(L.a[q]);
        const long long half = L.n[q] / 2;
        for (long long t = tid; t < half; t += nthr) {
            double2 x = __ldg(v + t);
            bad |= !isfinite(x.x) || !isfinite(x.y);
        }
        if ((L.n[q] & 1) && tid == 0) bad |= !isfinite(__ldg(L.a[q] + L.n[q] - 1));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}
}  // namespace pdac

// scan arrays on the context's stream; PDAC_ERR_NONFINITE names the first
// listed array that holds a NaN or Inf
static int check_finite(pdac_ctx *ctx, const std::vector<std::pair<const double *, size_t>> &arrs,
                        const std::vector<std::string> &names, const char *where) {
    cudaStream_t st = ctx->stream;
    CK(cudaMemsetAsync(ctx->d_nonfinite, 0, sizeof(int), st));
    int dev = 0, nsm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (size_t b = 0; b < arrs.size(); b += 24) {
        pdac::FinList L{};
        L.m = (int)std::min<size_t>(24, arrs.size() - b);
        for (int q = 0; q < L.m; ++q) { L.a[q] = arrs[b + q].first; L.n[q] = (long long)arrs[b + q].second; }
        pdac::k_nonfinite<<<nsm * 8, 256, 0, st>>>(L, ctx->d_nonfinite);
        ctx->launches++;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_nonfinite, ctx->d_nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (!*ctx->h_nonfinite) return PDAC_OK;
    // name the field: one array at a time (only on this error path)
    std::string which = "?";
    for (size_t q = 0; q < arrs.size(); ++q) {
        pdac::FinList L{};
        L.m = 1;
        L.a[0] = arrs[q].first;
        L.n[0] = (long long)arrs[q].second;
        CK(cudaMemsetAsync(ctx->d_nonfinite, 0, sizeof(int), st));
        pdac::k_nonfinite<<<nsm * 8, 256, 0, st>>>(L, ctx->d_nonfinite);
        CK(cudaMemcpyAsync(ctx->h_nonfinite, ctx->d_nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (*ctx->h_nonfinite) { which = names[q]; break; }
    }
    return fail(ctx, PDAC_ERR_NONFINITE, std::string(where) + ": non-finite value in " + which);
}

// the state fields of a view with their device arrays, element counts and
// whether an upload needs them
struct XField { double *h; double *d; size_t cnt; bool need; const char *name; };
static constexpr int kStateFields = 18;
static void state_fields(pdac_ctx *ctx, const pdac_state_view *s, XField (&xs)[kStateFields]) {
    size_t n = ctx->ncell, ns = ctx->ns, ng = ctx->ng;
    Fld &F = ctx->F;
    XField v[kStateFields] = {
        {s->p, F.p, n, true, "p"}, {s->ep, F.ep, n, true, "ep"}, {s->rog, F.rog, n, true, "rog"},
        {s->rgp, F.rgp, n, true, "rgp"}, {s->tg, F.tg, n, true, "tg"}, {s->sieg, F.sieg, n, true, "sieg"},
        {s->cg, F.cg, n, true, "cg"}, {s->ug, F.ug, n, true, "ug"}, {s->vg, F.vg, n, ctx->d3, "vg"},
        {s->wg, F.wg, n, true, "wg"}, {s->rlk, F.rlk, n * ns, true, "rlk"}, {s->ts, F.ts, n * ns, true, "ts"},
        {s->sies, F.sies, n * ns, true, "sies"}, {s->us, F.us, n * ns, true, "us"},
        {s->vs, F.vs, n * ns, ctx->d3, "vs"}, {s->ws, F.ws, n * ns, true, "ws"},
        {s->ygc, F.ygc, n * ng, true, "ygc"}, {s->xgc, F.xgc, n * ng, true, "xgc"}};
    for (int q = 0; q < kStateFields; ++q) xs[q] = v[q];
}

static int xfer_state(pdac_ctx *ctx, pdac_state_view *s, bool up) {
    if (!ctx || !s) return PDAC_ERR_ARG;
    XField xs[kStateFields];
    state_fields(ctx, s, xs);
    std::vector<std::pair<const double *, size_t>> sent;
    std::vector<std::string> names;
    for (auto &x : xs) {
        if (!x.h) {
            if (up && x.need) return fail(ctx, PDAC_ERR_ARG, "upload: a required state field is NULL");
            continue;
        }
        if (up) {
            CK(cudaMemcpyAsync(x.d, x.h, x.cnt * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            if (x.cnt) { sent.push_back({x.d, x.cnt}); names.push_back(x.name); }
        } else {
            CK(cudaMemcpyAsync(x.h, x.d, x.cnt * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    // an uploaded NaN or Inf would spread through the corrector's
    // neighbourhoods within a sweep: refuse it at the boundary
    if (up) return check_finite(ctx, sent, names, "upload");
    CK(cudaStreamSynchronize(ctx->stream));
    return PDAC_OK;
}

// the state after a step: pressure, void fraction, gas bulk density,
// temperature, enthalpy and the particle bulk densities, through which every
// cell's update passes (a non-finite value anywhere in the stencil of a
// fluid cell reaches them within the step)
static int check_step_state(pdac_ctx *ctx) {
    const Fld &F = ctx->F;
    const size_t n = ctx->ncell;
    return check_finite(ctx, {{F.p, n}, {F.ep, n}, {F.rgp, n}, {F.tg, n}, {F.sieg, n}, {F.rlk, n * ctx->ns}},
                        {"p", "ep", "rgp", "tg", "sieg", "rlk"}, "step");
}

int pdac_gpu_upload_state(pdac_ctx *ctx, const pdac_state_view *s) { return xfer_state(ctx, const_cast<pdac_state_view *>(s), true); }
int pdac_gpu_download_state(pdac_ctx *ctx, pdac_state_view *s) { return xfer_state(ctx, s, false); }

// pdac_gpu_exchange_state: pdac_gpu_download_state into `out`, then
// pdac_gpu_upload_state from `in`, with the two directions overlapped.
// Field f is copied device -> host on the context's stream (after every
// earlier call's kernels) and host -> device on a second stream that first
// waits for that download, so the upload of field f may read the buffer its
// download has just filled (out == in) and overwrites nothing the device or
// the download still needs, while the download of field f + 1 runs beside
// it on the other copy engine.  The context's stream waits for the last
// upload; the uploaded fields are checked as pdac_gpu_upload_state checks
// them, and the call returns with both directions complete.
int pdac_gpu_exchange_state(pdac_ctx *ctx, pdac_state_view *out, const pdac_state_view *in) {
    if (!ctx || !out || !in) return PDAC_ERR_ARG;
    XField xo[kStateFields], xi[kStateFields];
    state_fields(ctx, out, xo);
    state_fields(ctx, in, xi);
    for (int q = 0; q < kStateFields; ++q)
        if (!xi[q].h && xi[q].need) return fail(ctx, PDAC_ERR_ARG, "exchange: a required state field of in is NULL");
    if (!ctx->up_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->up_stream, cudaStreamNonBlocking));
        for (auto &e : ctx->fev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->up_done, cudaEventDisableTiming));
    }
    cudaStream_t a = ctx->stream, b = ctx->up_stream;
    std::vector<std::pair<const double *, size_t>> sent;
    std::vector<std::string> names;
    for (int q = 0; q < kStateFields; ++q) {
        const size_t bytes = xi[q].cnt * sizeof(double);
        if (xo[q].h) CK(cudaMemcpyAsync(xo[q].h, xo[q].d, bytes, cudaMemcpyDeviceToHost, a));
        CK(cudaEventRecord(ctx->fev[q], a));
        if (!xi[q].h) continue;
        CK(cudaStreamWaitEvent(b, ctx->fev[q], 0));
        CK(cudaMemcpyAsync(xi[q].d, xi[q].h, bytes, cudaMemcpyHostToDevice, b));
        if (xi[q].cnt) { sent.push_back({xi[q].d, xi[q].cnt}); names.push_back(xi[q].name); }
    }
    CK(cudaEventRecord(ctx->up_done, b));
    CK(cudaStreamWaitEvent(a, ctx->up_done, 0));
    return check_finite(ctx, sent, names, "exchange");
}

// the kernels of boundary on stream st (also inside a whole-step graph)
static int enqueue_boundary(pdac_ctx *ctx, cudaStream_t st) {
    if (ctx->nvent > 0 && ctx->cfg.irand >= 1)
        pdac::k_vent<<<blocks(ctx->nvent), TPB, 0, st>>>(ctx->P, ctx->F, ctx->d_vent, ctx->nvent, ctx->d_vfact, ctx->d_vfact0), ctx->launches++;
    if (!ctx->blevel.empty()) {  // in levels (ib.cuh)
        for (size_t L = 0; L + 1 < ctx->blevel.size(); ++L) {
            const int lo = ctx->blevel[L], hi = ctx->blevel[L + 1];
            if (hi <= lo) continue;
            if (ctx->d3) pdac::k_boundary_items<3><<<blocks(hi - lo), TPB, 0, st>>>(ctx->P, ctx->F, ctx->IB, ctx->d_bitems, lo, hi);
            else pdac::k_boundary_items<2><<<blocks(hi - lo), TPB, 0, st>>>(ctx->P, ctx->F, ctx->IB, ctx->d_bitems, lo, hi);
            ctx->launches++;
        }
    } else {
        if (ctx->d3) pdac::k_boundary3d<<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F);
        else pdac::k_boundary2d<<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F);
        ctx->launches++;
    }
    if (ctx->S.ntr > 0) {
        const long nt = (long)ctx->S.ntr * ctx->ns;
        if (ctx->d3) pdac::k_sink<3><<<blocks(nt), TPB, 0, st>>>(ctx->P, ctx->F, ctx->S, ctx->cfg.dt);
        else pdac::k_sink<2><<<blocks(nt), TPB, 0, st>>>(ctx->P, ctx->F, ctx->S, ctx->cfg.dt);
        ctx->launches++;
    }
    CK(cudaGetLastError());
    return PDAC_OK;
}

int pdac_gpu_boundary(pdac_ctx *ctx, int sweep) {
    if (!ctx) return PDAC_ERR_ARG;
    (void)sweep;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    int s = enqueue_boundary(ctx, ctx->stream);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    return PDAC_OK;
}

// the kernels of fieldn on stream st
static int enqueue_fieldn(pdac_ctx *ctx, cudaStream_t st) {
    if (ctx->d3) pdac::k_fieldn3d<<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F);
    else pdac::k_fieldn2d<<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F);
    ctx->launches++;
    // allocate_fluxes (tilde.f:56-102): tilde and interphase terms start from
    // zero in every step
    size_t n = ctx->ncell;
    Fld &F = ctx->F;
    for (double *a : {F.rug, F.rvg, F.rwg})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.rus, F.rvs, F.rws})
        if (a) CK(cudaMemsetAsync(a, 0, n * ctx->ns * sizeof(double), st));
    for (double *a : {F.appu, F.appv, F.appw, ctx->d_app0u, ctx->d_app0v, ctx->d_app0w})
        if (a) CK(cudaMemsetAsync(a, 0, n * ctx->nap * sizeof(double), st));
    CK(cudaGetLastError());
    return PDAC_OK;
}

int pdac_gpu_fieldn(pdac_ctx *ctx) {
    if (!ctx) return PDAC_ERR_ARG;
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    int s = enqueue_fieldn(ctx, ctx->stream);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    return PDAC_OK;
}

// viscg / viscs before a stress evaluation (visc.f:150-205): mugt = mug +
// mugt with the sub-grid model, must = must + mus with the particle one
static int accumulate_viscosities(pdac_ctx *ctx, cudaStream_t st) {
    const size_t n = ctx->ncell;
    if (ctx->P.iturb && ctx->P.gas_viscosity) {
        pdac::k_accum<<<blocks((long)n), TPB, 0, st>>>(ctx->F.mugt, ctx->F.mug, n);
        ctx->launches++;
    }
    if (ctx->P.iss && ctx->P.part_viscosity)
        for (int is = 1; is <= ctx->ns; ++is) {
            pdac::k_accum_const<<<blocks((long)n), TPB, 0, st>>>(ctx->F.must + (size_t)(is - 1) * n, ctx->P.cmus[is], n);
            ctx->launches++;
        }
    CK(cudaGetLastError());
    return PDAC_OK;
}

// the conductivity of an enthalpy flux pass: kapgt = kapgt + kapg with the
// sub-grid model (htilde.f:218-224); the flux kernels then read kapgt
static void accumulate_conductivity(pdac_ctx *ctx, cudaStream_t st) {
    if (!ctx->P.iturb) return;
    pdac::k_accum<<<blocks((long)ctx->ncell), TPB, 0, st>>>(ctx->F.kapgt, ctx->F.kapg, (size_t)ctx->ncell);
    ctx->launches++;
}

// the kernels of tilde on stream st (also inside the sweep graph of iter
// with implicit_fluxes)
static int enqueue_tilde(pdac_ctx *ctx, double dt, cudaStream_t st) {
    size_t n = ctx->ncell, ns = ctx->ns;
    Fld &F = ctx->F;
    int s = accumulate_viscosities(ctx, st);
    if (s) return s;
    if (ctx->d3) {
        CK(cudaMemsetAsync(F.mf, 0, n * 9 * (ns + 1) * sizeof(double), st));
        pdac::k_visc3d<<<blocks((long)n * (ns + 1)), TPB, 0, st>>>(ctx->P, F);
        ctx->launches++;
        if (ctx->P.mixed) CK(launch_mom_tile<float>(ctx->P, F, ctx->nph, ctx->tile_shape, ctx->tile_kchunk, st));
        else CK(launch_mom_tile<double>(ctx->P, F, ctx->nph, ctx->tile_shape, ctx->tile_kchunk, st));
        ctx->launches += mom_launches(ctx->tile_shape);
        PHASE_LAUNCH(ctx->nph, pdac::k_tilde3d, blocks(n), TPB, st, ctx->P, F, dt, ctx->d_app0u, ctx->d_app0v, ctx->d_app0w);
        ctx->launches++;
    } else {
        for (double *a : {F.ugfe, F.ugft, F.wgfe, F.wgft}) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
        for (double *a : {F.usfe, F.usft, F.wsfe, F.wsft}) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
        (ctx->P.mixed ? pdac::k_tilde_flux2d<float> : pdac::k_tilde_flux2d<double>)<<<blocks(n), TPB, 0, st>>>(ctx->P, F),
            ctx->launches++;
        pdac::k_tilde2d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt, ctx->d_app0u, ctx->d_app0w), ctx->launches++;
    }
    if (ctx->P.alpha != 1.0 && ctx->cfg.rungekut > 1) {
        CK(cudaMemcpyAsync(ctx->d_app0u, F.appu, n * ctx->nap * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ctx->d_app0w, F.appw, n * ctx->nap * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (ctx->d3) CK(cudaMemcpyAsync(ctx->d_app0v, F.appv, n * ctx->nap * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaGetLastError());
    return PDAC_OK;
}

int pdac_gpu_tilde(pdac_ctx *ctx, double dt) {
    if (!ctx) return PDAC_ERR_ARG;
    cudaStream_t st = ctx->stream;
    CK(cudaEventRecord(ctx->ev[4], st));
    int s = enqueue_tilde(ctx, dt, st);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[5], st));
    return PDAC_OK;
}

static int enqueue_htilde(pdac_ctx *ctx, double dt, cudaStream_t st);
static int enqueue_ftem(pdac_ctx *ctx, double dt, cudaStream_t st, bool in_sweep);

// one outer sweep of the corrector (iter.f:241-410): three colour phases of
// candidate collection, residual test and inner loop; the sweep number is
// read on the device from d_nit
// kernels of the corrector in one graph sweep, k_sweep_check included
static long long sweep_kernels(const pdac_ctx *) { return 10; }

static int enqueue_sweep(pdac_ctx *ctx, double dt, cudaStream_t st, bool prof) {
    Fld &F = ctx->F;
    // implicit_fluxes: momentum fluxes, stresses and drag of the current
    // velocities before the cells are visited (iter.f:211-226)
    if (ctx->cfg.implicit_fluxes) {
        int s = enqueue_tilde(ctx, dt, st);
        if (s) return s;
    }
    const int nph = ctx->nph;
    const size_t n = ctx->ncell, nwords = (n + 31) / 32;
    const long nthr = (long)((ctx->nx + 2) / 3) * ctx->ny * ctx->nz;
    const int test_grid = ctx->test_grid > 0 ? ctx->test_grid : std::max(1, ctx->inner_grid / 2);
    // one team of lanes per worklist cell (5 teams of 6 lanes per warp in
    // 3D, 8 of 4 in 2D)
    const long team_threads = (nthr + (ctx->d3 ? 4 : 7)) / (ctx->d3 ? 5 : 8) * 32;
    const int g = std::min(ctx->inner_grid, blocks(team_threads, TPB_TEAM));
    unsigned *dirty = ctx->d_dirty;
    // [col] worklist length, [3 + col] cells tested, [6 + col] candidates, of colour col
    CK(cudaMemsetAsync(ctx->d_wcount, 0, 9 * sizeof(int), st));
    for (int col = 0; col < 3; ++col) {
        int *cnt = ctx->d_wcount + col, *ncand = ctx->d_wcount + 6 + col;
        if (prof) CK(cudaEventRecord(ctx->cev[3 * col], st));
        pdac::k_resid_collect<<<blocks((long)nwords, TPB_RESID), TPB_RESID, 0, st>>>(ctx->P, col, dirty, ctx->d_cand, ncand);
        int *wl = ctx->d_work + col * ctx->work_stride;
        if (ctx->d3) PHASE_LAUNCH_D(nph, pdac::k_resid_test, 3, test_grid, TPB_RESID, st, ctx->P, F, dt, ctx->d_cand, ncand, wl, cnt, dirty);
        else PHASE_LAUNCH_D(nph, pdac::k_resid_test, 2, test_grid, TPB_RESID, st, ctx->P, F, dt, ctx->d_cand, ncand, wl, cnt, dirty);
        if (prof) CK(cudaEventRecord(ctx->cev[3 * col + 1], st));
        if (ctx->d3) INNER_LAUNCH_D(nph, pdac::k_inner_team, 3, g, TPB_TEAM, st, ctx->P, F, dt, ctx->d_nit, wl, cnt, dirty);
        else INNER_LAUNCH_D(nph, pdac::k_inner_team, 2, g, TPB_TEAM, st, ctx->P, F, dt, ctx->d_nit, wl, cnt, dirty);
        if (prof) CK(cudaEventRecord(ctx->cev[3 * col + 2], st));
    }
    // implicit_enthalpy: the enthalpy fluxes (with implicit_fluxes) and the
    // enthalpy / interphase solve after the cells (iter.f:362-379), before
    // the convergence test, so also in the last sweep
    if (ctx->cfg.implicit_enthalpy) {
        int s = PDAC_OK;
        if (ctx->cfg.implicit_fluxes) s = enqueue_htilde(ctx, dt, st);
        if (!s) s = enqueue_ftem(ctx, dt, st, true);
        if (s) return s;
    }
    CK(cudaGetLastError());
    return PDAC_OK;
}

// (re)build the graph of the outer sweep loop for time step dt: a WHILE
// conditional node around one sweep plus k_sweep_check, which clears the
// condition when the sweep left no unconverged cell or maxout is reached
static int build_iter_graph(pdac_ctx *ctx, double dt) {
    if (ctx->it_exec) { cudaGraphExecDestroy(ctx->it_exec); ctx->it_exec = nullptr; }
    if (ctx->it_graph) { cudaGraphDestroy(ctx->it_graph); ctx->it_graph = nullptr; }
    cudaStream_t st = ctx->stream;
    CK(cudaGraphCreate(&ctx->it_graph, 0));
    cudaGraphConditionalHandle loop;
    CK(cudaGraphConditionalHandleCreate(&loop, ctx->it_graph, 1, cudaGraphCondAssignDefault));
    // the union inside cudaGraphNodeParams has no default constructor:
    // build the parameters in zeroed storage
    alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams &cp = *reinterpret_cast<cudaGraphNodeParams *>(cp_storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, ctx->it_graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    // kernels of one sweep: the nine of the colour phases, the check, and
    // those the implicit modes add (counted by their enqueue functions,
    // which run here only to record them)
    const long long before = ctx->launches;
    int s = enqueue_sweep(ctx, dt, st, false);
    ctx->it_per_sweep = sweep_kernels(ctx) + (ctx->launches - before);
    ctx->launches = before;
    if (!s) pdac::k_sweep_check<<<1, 1, 0, st>>>(ctx->d_wcount, ctx->d_nit, ctx->cfg.maxout, loop);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &captured);
    if (s) return s;
    if (e != cudaSuccess) return fail(ctx, PDAC_ERR_CUDA, std::string("iter graph capture: ") + cudaGetErrorString(e));
    CK(cudaGetLastError());
    CK(cudaGraphInstantiate(&ctx->it_exec, ctx->it_graph, 0));
    ctx->it_dt = dt;
    return PDAC_OK;
}

// allocate_fluxes (tilde.f:56-102), run by prog.f:229 before every RK
// stage, leaves the tilde momenta, interphase terms and enthalpy
// right-hand sides at zero; with implicit_fluxes no tilde precedes iter, so
// its predictor reads those zeros
static int zero_tilde_terms(pdac_ctx *ctx, cudaStream_t st) {
    Fld &F = ctx->F;
    const size_t n = ctx->ncell, ns = ctx->ns, nap = ctx->nap;
    for (double *a : {F.rug, F.rvg, F.rwg, F.rhg})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.rus, F.rvs, F.rws, F.rhs})
        if (a) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
    for (double *a : {F.appu, F.appv, F.appw})
        if (a) CK(cudaMemsetAsync(a, 0, n * nap * sizeof(double), st));
    return PDAC_OK;
}

static int maxout_status(pdac_ctx *ctx, int nit);

int pdac_gpu_iter(pdac_ctx *ctx, double dt, int *nit_out) {
    if (!ctx) return PDAC_ERR_ARG;
    cudaStream_t st = ctx->stream;
    size_t n = ctx->ncell, ns = ctx->ns;
    Fld &F = ctx->F;
    CK(cudaEventRecord(ctx->ev[6], st));
    if (ctx->cfg.implicit_fluxes) {
        int s = zero_tilde_terms(ctx, st);
        if (s) return s;
    }
    CK(cudaMemsetAsync(ctx->d_counters + 5, 0, sizeof(int), st));  // caloric failures of in-sweep ftem calls
    for (double *a : {F.rgfe, F.rgfn, F.rgft, F.conv, F.abeta})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.rsfe, F.rsfn, F.rsft})
        if (a) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
    int nph = ctx->nph;
    if (ctx->d3) {
        PHASE_LAUNCH(nph, pdac::k_predictor3d, blocks(n), TPB, st, ctx->P, F, dt);
        pdac::k_mflux_init3d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt);
    } else {
        PHASE_LAUNCH(nph, pdac::k_predictor2d, blocks(n), TPB, st, ctx->P, F, dt);
        pdac::k_mflux_init2d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt);
    }
    ctx->launches += 2;
    CK(cudaGetLastError());
    // every cell is tested in the first sweep
    CK(cudaMemsetAsync(ctx->d_dirty, 0xff, (n + 31) / 32 * sizeof(unsigned), st));
    int nit;
    const bool coop = ctx->coop_blocks > 0 && ctx->allow_coop && !ctx->cfg.implicit_fluxes && !ctx->cfg.implicit_enthalpy;
    if (!ctx->prof && coop) {
        // small domain: the sweep loop in one cooperative launch
        pdac::SweepWork W{ctx->d_wcount, ctx->d_cand, ctx->d_work, ctx->d_dirty, ctx->d_nit, ctx->work_stride};
        CK(launch_iter_coop(ctx, dt, st, W));
        CK(cudaMemcpyAsync(ctx->h_nit, ctx->d_nit, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        nit = *ctx->h_nit;
        ctx->sweeps += std::min(nit, ctx->cfg.maxout);
        ctx->launches++;
    } else if (!ctx->prof) {
        // the sweep loop runs on the device; one read-back of its count
        if (!ctx->it_exec || ctx->it_dt != dt) {
            int s = build_iter_graph(ctx, dt);
            if (s) return s;
        }
        *ctx->h_nit = 1;
        CK(cudaMemcpyAsync(ctx->d_nit, ctx->h_nit, sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(ctx->it_exec, st));
        CK(cudaMemcpyAsync(ctx->h_nit, ctx->d_nit, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ctx->h_counters + 5, ctx->d_counters + 5, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        nit = *ctx->h_nit;
        int done = std::min(nit, ctx->cfg.maxout);
        ctx->sweeps += done;
        ctx->launches += ctx->it_per_sweep * done;
    } else {
        // host loop with per-colour-phase timing
        for (nit = 1; nit <= ctx->cfg.maxout; ++nit) {
            *ctx->h_nit = nit;
            CK(cudaMemcpyAsync(ctx->d_nit, ctx->h_nit, sizeof(int), cudaMemcpyHostToDevice, st));
            int s = enqueue_sweep(ctx, dt, st, true);
            if (s) return s;
            ctx->launches += 9;
            CK(cudaMemcpyAsync(ctx->h_counters, ctx->d_wcount, 6 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            ctx->sweeps++;
            ctx->launches += (long long)ctx->cfg.implicit_enthalpy;  // k_eos_sticky
            long unconverged = (long)ctx->h_counters[0] + ctx->h_counters[1] + ctx->h_counters[2];
            ctx->work_cells += unconverged;
            ctx->tested_cells += (long)ctx->h_counters[3] + ctx->h_counters[4] + ctx->h_counters[5];
            for (int col = 0; col < 3; ++col) {
                float t0 = 0, t1 = 0;
                CK(cudaEventElapsedTime(&t0, ctx->cev[3 * col], ctx->cev[3 * col + 1]));
                CK(cudaEventElapsedTime(&t1, ctx->cev[3 * col + 1], ctx->cev[3 * col + 2]));
                ctx->resid_ms += t0;
                ctx->inner_ms += t1;
                ctx->corr_ms += t0 + t1;
                ctx->corr_launches++;
                double rec[6] = {(double)nit, (double)col, (double)ctx->h_counters[col],
                                 (double)ctx->h_counters[3 + col], t0, t1};
                ctx->sweep_log.insert(ctx->sweep_log.end(), rec, rec + 6);
            }
            if (unconverged == 0) break;
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[7], st));
    if (nit_out) *nit_out = nit;
    ctx->last_nit = nit;
    if (ctx->cfg.implicit_enthalpy) {
        if (ctx->prof) {
            CK(cudaMemcpyAsync(ctx->h_counters + 5, ctx->d_counters + 5, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        if (ctx->h_counters[5]) return fail(ctx, PDAC_ERR_EOS, "iter: caloric equation of state failed in a sweep's ftem");
    }
    return maxout_status(ctx, nit);
}

// the end of iter without convergence (iter.f:428-450): the reference
// reports the unconverged cells and stops the run only with cstop
static int maxout_status(pdac_ctx *ctx, int nit) {
    if (nit <= ctx->cfg.maxout || !ctx->cfg.cstop) return PDAC_OK;
    return fail(ctx, PDAC_ERR_MAXOUT, "iter: max number of iters exceeded (" + std::to_string(ctx->cfg.maxout) +
                                          " outer sweeps without convergence)");
}

int pdac_gpu_unconverged_cells(pdac_ctx *ctx, int *ijk, long *n_inout) {
    if (!ctx || !n_inout) return PDAC_ERR_ARG;
    cudaStream_t st = ctx->stream;
    int cnt[3] = {0, 0, 0};
    if (ctx->last_nit > 0) {
        CK(cudaMemcpyAsync(ctx->h_counters, ctx->d_wcount, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int c = 0; c < 3; ++c) cnt[c] = ctx->h_counters[c];
    }
    const long total = (long)cnt[0] + cnt[1] + cnt[2];
    if (!ijk || *n_inout < total) {
        *n_inout = total;
        return total ? fail(ctx, PDAC_ERR_ARG, "unconverged_cells: the list holds " + std::to_string(total) + " cells")
                     : PDAC_OK;
    }
    long at = 0;
    for (int c = 0; c < 3; ++c) {
        if (cnt[c]) CK(cudaMemcpy(ijk + at, ctx->d_work + c * ctx->work_stride, cnt[c] * sizeof(int), cudaMemcpyDeviceToHost));
        at += cnt[c];
    }
    std::sort(ijk, ijk + total);
    *n_inout = total;
    return PDAC_OK;
}

// ---------------------------------------------------------------------------
// pdac_gpu_iter_static: pdac_gpu_iter with its corrector scratch (per-colour
// counters, worklist, active-set flags) in one fixed static device array
// instead of the context's buffers; the call allocates nothing.
//
// Layout of the static array: bytes [0, 256) hold the nine int counters
// (worklist length, tested cells and candidates per colour) and the sweep
// number (int 12), then the
// worklist and the candidate list (one int per cell of the largest colour
// phase each, 256-aligned lengths), then the active set (one bit per cell).
// The counters must be zero when a colour phase starts: the call clears them
// itself on its stream before every sweep, and sets every active-set bit
// before the first sweep, so no part of the array has to start at zero.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_iter_scratch[PDAC_ITER_STATIC_SCRATCH_BYTES];

namespace {
std::mutex g_scratch_mutex;
unsigned char *g_scratch_ptr[64] = {nullptr};  // device address of g_iter_scratch, by device ordinal

// one-time set-up per device, with that device current
int static_scratch(pdac_ctx *ctx, unsigned char **out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(ctx, PDAC_ERR_ARG, "iter_static: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_iter_scratch);
        if (e != cudaSuccess)
            return fail(ctx, PDAC_ERR_CUDA, std::string("iter_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<unsigned char *>(ptr);
    }
    *out = g_scratch_ptr[dev];
    return PDAC_OK;
}
}  // namespace

int pdac_gpu_iter_static(pdac_ctx *ctx, double dt, int *nit_out) {
    if (!ctx) return PDAC_ERR_ARG;
    if (ctx->cfg.implicit_fluxes || ctx->cfg.implicit_enthalpy)
        return fail(ctx, PDAC_ERR_CONFIG, "iter_static: the implicit-flux modes run through pdac_gpu_iter only");
    int m = (ctx->nx + 2) / 3;
    long nthr = (long)m * ctx->ny * ctx->nz;
    size_t n = ctx->ncell, ns = ctx->ns;
    size_t work_bytes = ((size_t)nthr * sizeof(int) + 255) / 256 * 256;
    size_t nwords = (n + 31) / 32;
    size_t need = 256 + 2 * work_bytes + nwords * sizeof(unsigned);
    if (need > (size_t)PDAC_ITER_STATIC_SCRATCH_BYTES)
        return fail(ctx, PDAC_ERR_ARG, "iter_static: this mesh needs " + std::to_string(need) +
                                           " bytes of static scratch, the limit is " +
                                           std::to_string((size_t)PDAC_ITER_STATIC_SCRATCH_BYTES));
    unsigned char *base = nullptr;
    int st_ = static_scratch(ctx, &base);
    if (st_) return st_;
    int *wcount = reinterpret_cast<int *>(base);
    int *dnit = wcount + 12;  // sweep number, read by the inner loop
    int *work = reinterpret_cast<int *>(base + 256);
    int *cand = reinterpret_cast<int *>(base + 256 + work_bytes);
    unsigned *dirty = reinterpret_cast<unsigned *>(base + 256 + 2 * work_bytes);
    cudaStream_t st = ctx->stream;
    Fld &F = ctx->F;
    CK(cudaEventRecord(ctx->ev[6], st));
    for (double *a : {F.rgfe, F.rgfn, F.rgft, F.conv, F.abeta})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.rsfe, F.rsfn, F.rsft})
        if (a) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
    int nph = ctx->nph;
    if (ctx->d3) {
        PHASE_LAUNCH(nph, pdac::k_predictor3d, blocks(n), TPB, st, ctx->P, F, dt);
        pdac::k_mflux_init3d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt);
    } else {
        PHASE_LAUNCH(nph, pdac::k_predictor2d, blocks(n), TPB, st, ctx->P, F, dt);
        pdac::k_mflux_init2d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt);
    }
    ctx->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(dirty, 0xff, nwords * sizeof(unsigned), st));
    // the context's own worklist lengths describe an earlier pdac_gpu_iter
    ctx->last_nit = 0;
    const int test_grid = std::max(1, ctx->inner_grid / 2);
    int nit;
    for (nit = 1; nit <= ctx->cfg.maxout; ++nit) {
        *ctx->h_nit = nit;
        CK(cudaMemcpyAsync(dnit, ctx->h_nit, sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(wcount, 0, 9 * sizeof(int), st));
        for (int col = 0; col < 3; ++col) {
            int *cnt = wcount + col, *ncand = wcount + 6 + col;
            pdac::k_resid_collect<<<blocks((long)nwords, TPB_RESID), TPB_RESID, 0, st>>>(ctx->P, col, dirty, cand, ncand);
            if (ctx->d3) PHASE_LAUNCH_D(nph, pdac::k_resid_test, 3, test_grid, TPB_RESID, st, ctx->P, F, dt, cand, ncand, work, cnt, dirty);
            else PHASE_LAUNCH_D(nph, pdac::k_resid_test, 2, test_grid, TPB_RESID, st, ctx->P, F, dt, cand, ncand, work, cnt, dirty);
            ctx->launches++;
            long team_threads = (nthr + (ctx->d3 ? 4 : 7)) / (ctx->d3 ? 5 : 8) * 32;
            int g = std::min(ctx->inner_grid, blocks(team_threads, TPB_TEAM));
            if (ctx->d3) INNER_LAUNCH_D(nph, pdac::k_inner_team, 3, g, TPB_TEAM, st, ctx->P, F, dt, dnit, work, cnt, dirty);
            else INNER_LAUNCH_D(nph, pdac::k_inner_team, 2, g, TPB_TEAM, st, ctx->P, F, dt, dnit, work, cnt, dirty);
            ctx->launches += 2;
        }
        CK(cudaMemcpyAsync(ctx->h_counters, wcount, 6 * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ctx->sweeps++;
        long unconverged = (long)ctx->h_counters[0] + ctx->h_counters[1] + ctx->h_counters[2];
        if (ctx->prof) {
            ctx->work_cells += unconverged;
            ctx->tested_cells += (long)ctx->h_counters[3] + ctx->h_counters[4] + ctx->h_counters[5];
        }
        if (unconverged == 0) break;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[7], st));
    if (nit_out) *nit_out = nit;
    return maxout_status(ctx, nit);
}

// the kernels of ygas with more than one gas, on stream st
static int enqueue_ygas(pdac_ctx *ctx, double dt, cudaStream_t st) {
    const size_t n = ctx->ncell;
    for (double *a : {ctx->F.yfe, ctx->F.yfn, ctx->F.yft})
        if (a) CK(cudaMemsetAsync(a, 0, n * ctx->ng * sizeof(double), st));
    if (ctx->d3) {
        (ctx->P.mixed ? pdac::k_ygas_flux3d<float> : pdac::k_ygas_flux3d<double>)<<<blocks(n), TPB, 0, st>>>(ctx->P, ctx->F),
            ctx->launches++;
        pdac::k_ygas3d<<<blocks(n), TPB, 0, st>>>(ctx->P, ctx->F, dt), ctx->launches++;
    } else {
        (ctx->P.mixed ? pdac::k_ygas_flux2d<float> : pdac::k_ygas_flux2d<double>)<<<blocks(n), TPB, 0, st>>>(ctx->P, ctx->F),
            ctx->launches++;
        pdac::k_ygas2d<<<blocks(n), TPB, 0, st>>>(ctx->P, ctx->F, dt), ctx->launches++;
    }
    CK(cudaGetLastError());
    return PDAC_OK;
}

int pdac_gpu_ygas(pdac_ctx *ctx, double dt) {
    if (!ctx) return PDAC_ERR_ARG;
    cudaStream_t st = ctx->stream;
    size_t n = ctx->ncell;
    CK(cudaEventRecord(ctx->ev[8], st));
    if (ctx->ng == 1) {
        std::vector<double> one(n, 1.0);
        CK(cudaMemcpyAsync(ctx->F.ygc, one.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->F.xgc, one.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    } else {
        int s = enqueue_ygas(ctx, dt, st);
        if (s) return s;
    }
    CK(cudaEventRecord(ctx->ev[9], st));
    return PDAC_OK;
}

// the kernels of htilde on stream st
static int enqueue_htilde(pdac_ctx *ctx, double dt, cudaStream_t st) {
    size_t n = ctx->ncell, ns = ctx->ns;
    Fld &F = ctx->F;
    for (double *a : {F.egfe, F.egfn, F.egft})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.esfe, F.esfn, F.esft})
        if (a) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
    accumulate_conductivity(ctx, st);
    if (ctx->d3) {
        (ctx->P.mixed ? pdac::k_htilde_flux3d<true, float> : pdac::k_htilde_flux3d<true, double>)<<<blocks(n), TPB, 0, st>>>(
            ctx->P, F),
            ctx->launches++;
        pdac::k_htilde3d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt), ctx->launches++;
    } else {
        (ctx->P.mixed ? pdac::k_htilde_flux2d<true, float> : pdac::k_htilde_flux2d<true, double>)<<<blocks(n), TPB, 0, st>>>(
            ctx->P, F),
            ctx->launches++;
        pdac::k_htilde2d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt), ctx->launches++;
    }
    CK(cudaGetLastError());
    return PDAC_OK;
}

int pdac_gpu_htilde(pdac_ctx *ctx, double dt) {
    if (!ctx) return PDAC_ERR_ARG;
    cudaStream_t st = ctx->stream;
    CK(cudaEventRecord(ctx->ev[10], st));
    int s = enqueue_htilde(ctx, dt, st);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[11], st));
    return PDAC_OK;
}

namespace pdac {
// an ftem inside the sweeps of iter: more than one caloric failure
// (ftem.f:191-193) is remembered in counters[5] until iter returns
__global__ void k_eos_sticky(int *counters) {
    if (counters[1] > 1) counters[5] = 1;
}
}  // namespace pdac

static int enqueue_ftem(pdac_ctx *ctx, double dt, cudaStream_t st, bool in_sweep) {
    CK(cudaMemsetAsync(ctx->d_counters + 1, 0, sizeof(int), st));
    if (ctx->d3) pdac::k_ftem3d<<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F, dt);
    else pdac::k_ftem2d<<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F, dt);
    ctx->launches++;
    if (in_sweep) pdac::k_eos_sticky<<<1, 1, 0, st>>>(ctx->d_counters);
    CK(cudaGetLastError());
    return PDAC_OK;
}

int pdac_gpu_ftem(pdac_ctx *ctx, double dt) {
    if (!ctx) return PDAC_ERR_ARG;
    cudaStream_t st = ctx->stream;
    CK(cudaEventRecord(ctx->ev[12], st));
    int s = enqueue_ftem(ctx, dt, st, false);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[13], st));
    CK(cudaMemcpyAsync(ctx->h_counters + 1, ctx->d_counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ctx->h_counters[1] > 1) return fail(ctx, PDAC_ERR_EOS, "ftem: caloric equation of state failed");
    return PDAC_OK;
}

// ---------------------------------------------------------------------------
// explicit SSP-RK3 solver (time_integration = 1), explicit_solver.f
// ---------------------------------------------------------------------------
int pdac_gpu_initialize_fieldn(pdac_ctx *ctx) {
    if (!ctx) return PDAC_ERR_ARG;
    if (ctx->ti != 1) return fail(ctx, PDAC_ERR_CONFIG, "initialize_fieldn: the context runs time_integration = 0");
    cudaStream_t st = ctx->stream;
    size_t n = ctx->ncell, ns = ctx->ns;
    Fld &F = ctx->F;
    CK(cudaEventRecord(ctx->ev[2], st));
    // fluxes and stresses start from zero (explicit_solver.f:446-509)
    for (double *a : {F.rgfe, F.rgfn, F.rgft, F.egfe, F.egfn, F.egft, F.ugfe, F.ugft, F.wgfe, F.wgft})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.rsfe, F.rsfn, F.rsft, F.esfe, F.esfn, F.esft, F.usfe, F.usft, F.wsfe, F.wsft})
        if (a) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
    if (F.mf) CK(cudaMemsetAsync(F.mf, 0, n * 9 * (ns + 1) * sizeof(double), st));
    CK(cudaMemsetAsync(F.vis, 0, n * 3 * (ns + 1) * sizeof(double), st));
    if (ctx->d3) {
        PHASE_LAUNCH_D(ctx->nph, pdac::k_rk3_fieldn, 3, blocks(n), TPB, st, ctx->P, F, ctx->K, ctx->cfg.dt);
        if (int s = accumulate_viscosities(ctx, st)) return s;
        pdac::k_visc3d<<<blocks((long)n * (ns + 1)), TPB, 0, st>>>(ctx->P, F);
    } else {
        PHASE_LAUNCH_D(ctx->nph, pdac::k_rk3_fieldn, 2, blocks(n), TPB, st, ctx->P, F, ctx->K, ctx->cfg.dt);
        if (int s = accumulate_viscosities(ctx, st)) return s;
        pdac::k_visc2d<<<blocks((long)n * (ns + 1)), TPB, 0, st>>>(ctx->P, F);
    }
    ctx->launches += 2;
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[3], st));
    return PDAC_OK;
}

// ---------------------------------------------------------------------------
// sub-grid turbulence model, turbo.f
// ---------------------------------------------------------------------------
// sgsg (turbo.f:145-349), called after fieldn / initialize_fieldn
// (prog.f:207); nothing to do without the sub-grid model
int pdac_gpu_sgsg(pdac_ctx *ctx) {
    if (!ctx) return PDAC_ERR_ARG;
    if (!ctx->P.iturb) return PDAC_OK;
    if (ctx->F.dyn) {
        pdac::k_sgsg_dyn1<<<blocks(ctx->ncell), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
        pdac::k_sgsg_dyn2<<<blocks(ctx->ncell), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
        ctx->launches += 2;
    } else {
        if (ctx->d3) pdac::k_sgsg<3><<<blocks(ctx->ncell), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
        else pdac::k_sgsg<2><<<blocks(ctx->ncell), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
        ctx->launches++;
    }
    CK(cudaGetLastError());
    return PDAC_OK;
}

// sgss (turbo.f:437-475), prog.f:208, with iss = 1
int pdac_gpu_sgss(pdac_ctx *ctx) {
    if (!ctx) return PDAC_ERR_ARG;
    if (ctx->P.iss != 1) return PDAC_OK;
    long nt = (long)ctx->ncell * ctx->ns;
    if (ctx->d3) pdac::k_sgss<3><<<blocks(nt), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
    else pdac::k_sgss<2><<<blocks(nt), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
    ctx->launches++;
    CK(cudaGetLastError());
    return PDAC_OK;
}

// the kernels of one explicit_iter on stream st; returns their count.  With
// prof, events xev[0..8] mark the group boundaries: flux pass, stage 1,
// wavefront 1, flux pass, stage 2, wavefront 2, flux pass, final kernels
static long long enqueue_explicit(pdac_ctx *ctx, double dt, cudaStream_t st, bool prof) {
    int q = 0;
    auto mark = [&]() { if (prof) cudaEventRecord(ctx->xev[q++], st); };
    const Prm &P = ctx->P;
    const Fld &F = ctx->F;
    const RkF &K = ctx->K;
    const long n = ctx->ncell;
    const int nph = ctx->nph, nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    long long L = 0;
    // compute_fluxes: mass, momentum and enthalpy face fluxes of the state
    auto fluxes = [&]() {
        if (P.iturb) {
            pdac::k_accum<<<blocks(n), TPB, 0, st>>>(F.kapgt, F.kapg, (size_t)n);
            L++;
        }
        if (ctx->d3) {
            if (P.mixed) {
                pdac::k_rk3_mflux<3, float><<<blocks(n), TPB, 0, st>>>(P, F);
                (void)launch_mom_tile<float>(P, F, nph, ctx->tile_shape, ctx->tile_kchunk, st);
                pdac::k_htilde_flux3d<false, float><<<blocks(n), TPB, 0, st>>>(P, F);
            } else {
                pdac::k_rk3_mflux<3><<<blocks(n), TPB, 0, st>>>(P, F);
                (void)launch_mom_tile<double>(P, F, nph, ctx->tile_shape, ctx->tile_kchunk, st);
                pdac::k_htilde_flux3d<false><<<blocks(n), TPB, 0, st>>>(P, F);
            }
            L += 2 + mom_launches(ctx->tile_shape);
        } else {
            if (P.mixed) {
                pdac::k_rk3_mflux<2, float><<<blocks(n), TPB, 0, st>>>(P, F);
                pdac::k_tilde_flux2d<float><<<blocks(n), TPB, 0, st>>>(P, F);
                pdac::k_htilde_flux2d<false, float><<<blocks(n), TPB, 0, st>>>(P, F);
            } else {
                pdac::k_rk3_mflux<2><<<blocks(n), TPB, 0, st>>>(P, F);
                pdac::k_tilde_flux2d<<<blocks(n), TPB, 0, st>>>(P, F);
                pdac::k_htilde_flux2d<false><<<blocks(n), TPB, 0, st>>>(P, F);
            }
            L += 3;
        }
    };
    for (int stage = 1; stage <= 2; ++stage) {
        mark();
        fluxes();
        mark();
        if (ctx->d3) PHASE_LAUNCH_D(nph, pdac::k_rk3_stage, 3, blocks(n), TPB, st, P, F, K, dt, stage);
        else PHASE_LAUNCH_D(nph, pdac::k_rk3_stage, 2, blocks(n), TPB, st, P, F, K, dt, stage);
        L++;
        mark();
        // gas-enthalpy wavefront over the hyperplanes i + j + k = d of the
        // interior (2 <= i <= nx - 1 ...), in increasing d: records, one
        // cooperative launch over all hyperplanes, scatter of the results
        if (ctx->wave_grid_blocks > 0 && ctx->allow_coop) {
            const pdac::Wave &W = ctx->W;
            const int rb = blocks(W.npos);
            cudaLaunchConfig_t lc = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeCooperative;
            at[0].val.cooperative = 1;
            lc.gridDim = dim3(ctx->wave_grid_blocks);
            lc.blockDim = dim3(TPB);
            lc.stream = st;
            lc.attrs = at;
            lc.numAttrs = 1;
            if (ctx->d3) {
                pdac::k_rk3_wave_pre<3><<<blocks(n), TPB, 0, st>>>(P, F, K, W, dt, stage);
                if (ctx->wave_one) cudaLaunchKernelEx(&lc, pdac::k_rk3_wave_rec<3, true>, P, W, dt, stage);
                else cudaLaunchKernelEx(&lc, pdac::k_rk3_wave_rec<3, false>, P, W, dt, stage);
                pdac::k_rk3_wave_post<3><<<rb, TPB, 0, st>>>(P, F, K, W, stage);
            } else {
                pdac::k_rk3_wave_pre<2><<<blocks(n), TPB, 0, st>>>(P, F, K, W, dt, stage);
                if (ctx->wave_one) cudaLaunchKernelEx(&lc, pdac::k_rk3_wave_rec<2, true>, P, W, dt, stage);
                else cudaLaunchKernelEx(&lc, pdac::k_rk3_wave_rec<2, false>, P, W, dt, stage);
                pdac::k_rk3_wave_post<2><<<rb, TPB, 0, st>>>(P, F, K, W, stage);
            }
            L += 3;
        } else if (ctx->d3) {
            const int nj = ny - 2, dmax = (nx - 1) + (ny - 1) + (nz - 1);
            for (int d = 6; d <= dmax; ++d) {
                int kmin = std::max(2, d - (nx - 1) - (ny - 1)), kmax = std::min(nz - 1, d - 4);
                int nt = nj * (kmax - kmin + 1);
                pdac::k_rk3_wave<3><<<blocks(nt), TPB, 0, st>>>(P, F, K, dt, stage, d, kmin, nt);
                L++;
            }
        } else {
            const int dmax = (nx - 1) + (nz - 1);
            for (int d = 4; d <= dmax; ++d) {
                int kmin = std::max(2, d - (nx - 1)), kmax = std::min(nz - 1, d - 2);
                int nt = kmax - kmin + 1;
                pdac::k_rk3_wave<2><<<blocks(nt), TPB, 0, st>>>(P, F, K, dt, stage, d, kmin, nt);
                L++;
            }
        }
    }
    mark();
    fluxes();
    mark();
    cudaMemsetAsync(ctx->d_counters + 1, 0, sizeof(int), st);
    if (ctx->d3) {
        PHASE_LAUNCH_D(nph, pdac::k_rk3_final_rhs, 3, blocks(n), TPB, st, P, F, K, dt);
        PHASE_LAUNCH_D(nph, pdac::k_rk3_final_phys, 3, blocks(n), TPB, st, P, F, K, dt);
        PHASE_LAUNCH_D(nph, pdac::k_rk3_solve, 3, blocks(n), TPB, st, P, F, K, dt);
    } else {
        PHASE_LAUNCH_D(nph, pdac::k_rk3_final_rhs, 2, blocks(n), TPB, st, P, F, K, dt);
        PHASE_LAUNCH_D(nph, pdac::k_rk3_final_phys, 2, blocks(n), TPB, st, P, F, K, dt);
        PHASE_LAUNCH_D(nph, pdac::k_rk3_solve, 2, blocks(n), TPB, st, P, F, K, dt);
    }
    L += 3;
    mark();
    return L;
}

// explicit_iter as one graph for time step dt
static int build_explicit_graph(pdac_ctx *ctx, double dt) {
    if (ctx->ex_exec) { cudaGraphExecDestroy(ctx->ex_exec); ctx->ex_exec = nullptr; }
    if (ctx->ex_graph) { cudaGraphDestroy(ctx->ex_graph); ctx->ex_graph = nullptr; }
    cudaStream_t st = ctx->stream;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    long long L = enqueue_explicit(ctx, dt, st, false);
    cudaError_t e = cudaStreamEndCapture(st, &ctx->ex_graph);
    if (e != cudaSuccess) return fail(ctx, PDAC_ERR_CUDA, std::string("explicit_iter graph capture: ") + cudaGetErrorString(e));
    CK(cudaGetLastError());
    CK(cudaGraphInstantiate(&ctx->ex_exec, ctx->ex_graph, 0));
    ctx->ex_dt = dt;
    ctx->ex_launches = L;
    return PDAC_OK;
}

int pdac_gpu_explicit_iter(pdac_ctx *ctx, double dt) {
    if (!ctx) return PDAC_ERR_ARG;
    if (ctx->ti != 1) return fail(ctx, PDAC_ERR_CONFIG, "explicit_iter: the context runs time_integration = 0");
    cudaStream_t st = ctx->stream;
    CK(cudaEventRecord(ctx->ev[6], st));
    if (ctx->prof) {
        ctx->launches += enqueue_explicit(ctx, dt, st, true);
        CK(cudaGetLastError());
    } else {
        if (!ctx->ex_exec || ctx->ex_dt != dt) {
            int s = build_explicit_graph(ctx, dt);
            if (s) return s;
        }
        CK(cudaGraphLaunch(ctx->ex_exec, st));
        ctx->launches += ctx->ex_launches;
    }
    CK(cudaEventRecord(ctx->ev[7], st));
    CK(cudaMemcpyAsync(ctx->h_counters + 1, ctx->d_counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ctx->prof) {
        float t[8];
        for (int q = 0; q < 8; ++q) CK(cudaEventElapsedTime(&t[q], ctx->xev[q], ctx->xev[q + 1]));
        ctx->ex_ms[0] += t[0] + t[3] + t[6];
        ctx->ex_ms[1] += t[1] + t[4];
        ctx->ex_ms[2] += t[2] + t[5];
        ctx->ex_ms[3] += t[7];
        ctx->ex_calls++;
    }
    // explicit_solver.f:1214-1215 stops the run on more than one failure
    if (ctx->h_counters[1] > 1) return fail(ctx, PDAC_ERR_EOS, "explicit_iter: caloric equation of state failed");
    return PDAC_OK;
}

int pdac_gpu_step(pdac_ctx *ctx, int sweep, int *nit) {
    if (!ctx) return PDAC_ERR_ARG;
    int s;
    if ((s = pdac_gpu_boundary(ctx, sweep))) return s;
    if (ctx->cfg.update_eosg) return fail(ctx, PDAC_ERR_CONFIG, "update_eosg is not built");
    double dt0 = ctx->cfg.dt;
    int status = PDAC_OK;
    if (ctx->ti == 1) {
        // prog.f:191-274 with time_integration = 1
        if ((s = pdac_gpu_initialize_fieldn(ctx))) return s;
        if ((s = pdac_gpu_sgsg(ctx)) || (s = pdac_gpu_sgss(ctx))) return s;
        if (nit) *nit = 0;
        for (int rk = 1; rk <= ctx->cfg.rungekut; ++rk) {
            double dt = dt0 / (ctx->cfg.rungekut + 1 - rk);
            s = pdac_gpu_explicit_iter(ctx, dt);
            if (s == PDAC_ERR_EOS) status = s;
            else if (s) return s;
            if ((s = pdac_gpu_ygas(ctx, dt))) return s;
        }
        if (ctx->cfg.compute_mixture && (s = pdac_gpu_compute_mixture_fields(ctx))) return s;  // prog.f:331
        if ((s = check_step_state(ctx))) return s;
        return status;
    }
    if ((s = pdac_gpu_fieldn(ctx))) return s;
    if ((s = pdac_gpu_sgsg(ctx)) || (s = pdac_gpu_sgss(ctx))) return s;
    const bool ifx = ctx->cfg.implicit_fluxes != 0, ien = ctx->cfg.implicit_enthalpy != 0;
    for (int rk = 1; rk <= ctx->cfg.rungekut; ++rk) {
        double dt = dt0 / (ctx->cfg.rungekut + 1 - rk);
        // prog.f:246-292: tilde (and htilde with implicit_enthalpy) before
        // iter unless implicit_fluxes moves them into the sweeps; htilde and
        // ftem after ygas unless implicit_enthalpy moved them
        if (!ifx) {
            if ((s = pdac_gpu_tilde(ctx, dt))) return s;
            if (ien && (s = pdac_gpu_htilde(ctx, dt))) return s;
        }
        s = pdac_gpu_iter(ctx, dt, nit);
        if (s == PDAC_ERR_EOS) status = s;
        else if (s) return s;  // PDAC_ERR_MAXOUT under cstop stops here, as error() does (iter.f:449)
        if ((s = pdac_gpu_ygas(ctx, dt))) return s;
        if (!ien) {
            if ((s = pdac_gpu_htilde(ctx, dt))) return s;
            s = pdac_gpu_ftem(ctx, dt);
            if (s == PDAC_ERR_EOS) status = s;
            else if (s) return s;
        }
    }
    if (ctx->cfg.compute_mixture && (s = pdac_gpu_compute_mixture_fields(ctx))) return s;  // prog.f:331
    if ((s = check_step_state(ctx))) return s;
    return status;
}

int pdac_gpu_get_array(pdac_ctx *ctx, const char *name, double *out, long *n_inout) {
    if (!ctx || !name || !n_inout) return PDAC_ERR_ARG;
    for (auto &e : ctx->names) {
        if (e.first == name) {
            long need = (long)e.second.second;
            if (!out || *n_inout < need) { *n_inout = need; return PDAC_ERR_ARG; }
            CK(cudaMemcpyAsync(out, e.second.first, need * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            *n_inout = need;
            return PDAC_OK;
        }
    }
    return fail(ctx, PDAC_ERR_ARG, std::string("unknown array ") + name);
}

int pdac_gpu_mass_totals(pdac_ctx *ctx, double *out, int nout) {
    if (!ctx || !out) return PDAC_ERR_ARG;
    int nq = 1 + ctx->ns + ctx->ng;
    if (nout < nq) return PDAC_ERR_ARG;
    int nb = 148;
    pdac::k_mass_partial<<<nb, 256, nq * 256 * sizeof(double), ctx->stream>>>(ctx->P, ctx->F, ctx->d_partial, nq);
    ctx->launches++;
    CK(cudaGetLastError());
    std::vector<double> h((size_t)nq * nb);
    CK(cudaMemcpyAsync(h.data(), ctx->d_partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < nq; ++q) {
        double s = 0;
        for (int b = 0; b < nb; ++b) s += h[(size_t)q * nb + b];
        out[q] = s;
    }
    return PDAC_OK;
}

int pdac_gpu_phase_times(pdac_ctx *ctx, double *ms7) {
    if (!ctx || !ms7) return PDAC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < 7; ++q) {
        float t = 0;
        if (cudaEventElapsedTime(&t, ctx->ev[2 * q], ctx->ev[2 * q + 1]) != cudaSuccess) t = 0;
        ms7[q] = t;
    }
    cudaGetLastError();
    return PDAC_OK;
}

// ---------------------------------------------------------------------------
// autotuner of the launch shapes (no counterpart in the reference)
// ---------------------------------------------------------------------------
namespace {
struct Tuning {
    int tile_shape, tile_kchunk, inner_grid, test_grid, coop_cpb;
};
constexpr int N_TUNE = 5;

Tuning get_tuning(const pdac_ctx *ctx) {
    return {ctx->tile_shape, ctx->tile_kchunk, ctx->inner_grid,
            ctx->test_grid > 0 ? ctx->test_grid : std::max(1, ctx->inner_grid / 2), ctx->coop_cpb};
}

// install t; the captured graphs hold the old launch shapes, so they are
// rebuilt at their next use
void put_tuning(pdac_ctx *ctx, const Tuning &t) {
    ctx->tile_shape = t.tile_shape;
    ctx->tile_kchunk = t.tile_kchunk;
    ctx->inner_grid = t.inner_grid;
    ctx->test_grid = t.test_grid;
    ctx->coop_cpb = t.coop_cpb;
    if (ctx->coop_max_blocks > 0)
        ctx->coop_blocks = std::min(std::max(1, (int)((ctx->ncell + t.coop_cpb - 1) / t.coop_cpb)), ctx->coop_max_blocks);
    if (ctx->it_exec) { cudaGraphExecDestroy(ctx->it_exec); ctx->it_exec = nullptr; }
    if (ctx->it_graph) { cudaGraphDestroy(ctx->it_graph); ctx->it_graph = nullptr; }
    if (ctx->ex_exec) { cudaGraphExecDestroy(ctx->ex_exec); ctx->ex_exec = nullptr; }
    if (ctx->ex_graph) { cudaGraphDestroy(ctx->ex_graph); ctx->ex_graph = nullptr; }
    if (ctx->step_exec) { cudaGraphExecDestroy(ctx->step_exec); ctx->step_exec = nullptr; }
    if (ctx->step_graph) { cudaGraphDestroy(ctx->step_graph); ctx->step_graph = nullptr; }
    ctx->graph_gen++;
}

bool tuning_valid(const pdac_ctx *ctx, const Tuning &t) {
    return t.tile_shape >= 0 && t.tile_shape < N_TILE_SHAPES && t.tile_kchunk >= 1 && t.inner_grid >= 1 &&
           t.test_grid >= 1 && t.coop_cpb >= 32 && t.tile_kchunk <= std::max(ctx->nz, 1);
}

// the cache key: what the best shapes depend on
std::string tuning_key(const pdac_ctx *ctx) {
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        std::snprintf(prop.name, sizeof prop.name, "unknown");
    }
    std::string name(prop.name);
    for (char &ch : name)
        if (ch == ' ' || ch == '\t') ch = '_';
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s grid=%dx%dx%d nsolid=%d ngas=%d precision=%d time_integration=%d implicit=%d%d",
                  name.c_str(), ctx->nx, ctx->ny, ctx->nz, ctx->ns, ctx->ng, ctx->cfg.precision, ctx->ti,
                  ctx->cfg.implicit_fluxes, ctx->cfg.implicit_enthalpy);
    return buf;
}

// cache file: one line per key, "<key> | t0 t1 t2 t3 t4"; the last line of a
// key wins
bool cache_find(const char *path, const std::string &key, Tuning &t) {
    FILE *f = path ? std::fopen(path, "r") : nullptr;
    if (!f) return false;
    bool found = false;
    char line[512];
    while (std::fgets(line, sizeof line, f)) {
        std::string l(line);
        size_t bar = l.find(" | ");
        if (bar == std::string::npos || l.compare(0, bar, key) != 0 || bar != key.size()) continue;
        Tuning u{};
        if (std::sscanf(l.c_str() + bar + 3, "%d %d %d %d %d", &u.tile_shape, &u.tile_kchunk, &u.inner_grid,
                        &u.test_grid, &u.coop_cpb) == N_TUNE) {
            t = u;
            found = true;
        }
    }
    std::fclose(f);
    return found;
}

bool cache_add(const char *path, const std::string &key, const Tuning &t) {
    FILE *f = path ? std::fopen(path, "a") : nullptr;
    if (!f) return false;
    bool ok = std::fprintf(f, "%s | %d %d %d %d %d\n", key.c_str(), t.tile_shape, t.tile_kchunk, t.inner_grid,
                           t.test_grid, t.coop_cpb) > 0;
    return std::fclose(f) == 0 && ok;
}

void tuning_out(const Tuning &t, int *out, int nout) {
    const int v[N_TUNE] = {t.tile_shape, t.tile_kchunk, t.inner_grid, t.test_grid, t.coop_cpb};
    for (int q = 0; q < nout && q < N_TUNE; ++q) out[q] = v[q];
}
}  // namespace

int pdac_gpu_set_tuning(pdac_ctx *ctx, const int *in, int nin) {
    if (!ctx || !in || nin < N_TUNE) return PDAC_ERR_ARG;
    Tuning t{in[0], in[1], in[2], in[3], in[4]};
    if (!tuning_valid(ctx, t)) return fail(ctx, PDAC_ERR_ARG, "set_tuning: a value is out of range");
    put_tuning(ctx, t);
    return PDAC_OK;
}

int pdac_gpu_autotune(pdac_ctx *ctx, const char *cache_path, int *out, int nout) {
    if (!ctx || (out && nout < 0)) return PDAC_ERR_ARG;
    const std::string key = tuning_key(ctx);
    Tuning best = get_tuning(ctx);
    if (cache_find(cache_path, key, best) && tuning_valid(ctx, best)) {
        put_tuning(ctx, best);
        if (out) tuning_out(best, out, nout);
        return PDAC_OK;
    }
    cudaStream_t st = ctx->stream;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    auto elapsed = [&](float &ms) -> int {
        CK(cudaEventSynchronize(b));
        CK(cudaEventElapsedTime(&ms, a, b));
        return PDAC_OK;
    };
    int status = PDAC_OK;
    // 1. tile shape and chunk of the 3D momentum-flux pass: a pure function
    // of the state (it rewrites the same face fluxes), timed on it directly
    if (ctx->d3 && status == PDAC_OK) {
        float best_ms = 1e30f;
        const int chunks[] = {16, 32, 64, ctx->nz};
        for (int shape = 0; shape < N_TILE_SHAPES && status == PDAC_OK; ++shape)
            for (int kc : chunks) {
                if (kc < 1 || kc > ctx->nz || (shape == 0 && kc != chunks[1])) continue;  // form 0 has no chunks
                auto launch = [&]() {
                    return ctx->P.mixed ? launch_mom_tile<float>(ctx->P, ctx->F, ctx->nph, shape, kc, st)
                                        : launch_mom_tile<double>(ctx->P, ctx->F, ctx->nph, shape, kc, st);
                };
                cudaError_t e = launch();
                if (e == cudaSuccess) e = cudaEventRecord(a, st);
                for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch();
                if (e == cudaSuccess) e = cudaEventRecord(b, st);
                float ms = 0;
                if (e != cudaSuccess) { status = fail(ctx, PDAC_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e)); break; }
                if ((status = elapsed(ms))) break;
                if (ms < best_ms) { best_ms = ms; best.tile_shape = shape; best.tile_kchunk = kc; }
            }
    }
    // 2. the corrector's grids (and the cells per block of the one-launch
    // sweep loop of small domains): whole time steps on the current state,
    // restored after each candidate from a device copy; skipped when the
    // copy does not fit in device memory
    const bool semi = ctx->ti == 0;
    double *snap = nullptr;
    size_t nv = std::max(ctx->nvent, 1), nm = ctx->S.ntr > 0 ? (size_t)2 * ctx->S.ntr * ctx->ns : 0;
    const size_t nib = ctx->ibstate_doubles;
    const size_t snap_doubles = ctx->arena_doubles + 2 * nv + nm + nib;
    if (status == PDAC_OK && semi && cudaMalloc(&snap, snap_doubles * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        snap = nullptr;
    }
    if (snap) {
        auto copy_state = [&](bool save) -> int {
            double *s0 = snap, *s1 = snap + ctx->arena_doubles, *s2 = s1 + nv, *s3 = s2 + nv;
            auto cp = [&](double *dev, double *keep, size_t cnt) {
                return cudaMemcpyAsync(save ? keep : dev, save ? dev : keep, cnt * sizeof(double),
                                       cudaMemcpyDeviceToDevice, st);
            };
            CK(cp(ctx->arena, s0, ctx->arena_doubles));
            CK(cp(ctx->d_vfact, s1, nv));
            CK(cp(ctx->d_vfact0, s2, nv));
            if (nm) CK(cp(ctx->d_sinkbuf, s3, nm));
            if (nib) CK(cp(ctx->d_ibstate, s3 + nm, nib));
            return PDAC_OK;
        };
        // statistics and the last iter's count are the caller's, not the tuner's
        const long long launches = ctx->launches, sweeps = ctx->sweeps, corr_launches = ctx->corr_launches,
                        work_cells = ctx->work_cells, tested_cells = ctx->tested_cells, ex_calls = ctx->ex_calls;
        const double corr_ms = ctx->corr_ms, resid_ms = ctx->resid_ms, inner_ms = ctx->inner_ms;
        const int last_nit = ctx->last_nit;
        const bool prof = ctx->prof;
        const std::vector<double> sweep_log = ctx->sweep_log;
        ctx->prof = false;
        status = copy_state(true);
        auto time_step = [&](const Tuning &t, float &ms) -> int {
            put_tuning(ctx, t);
            int nit = 0, s2;
            // the first step builds the graphs for the shapes; the second is timed
            for (int rep = 0; rep < 2; ++rep) {
                if ((s2 = copy_state(false))) return s2;
                CK(cudaEventRecord(a, st));
                s2 = pdac_gpu_step(ctx, 1, &nit);
                if (s2 == PDAC_ERR_CUDA) return s2;
                CK(cudaEventRecord(b, st));
                if ((s2 = elapsed(ms))) return s2;
            }
            return PDAC_OK;
        };
        int dev = 0, nsm = 148;
        if (!status) status = cudaGetDevice(&dev) == cudaSuccess &&
                                      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess
                                  ? PDAC_OK
                                  : fail(ctx, PDAC_ERR_CUDA, "autotune: device query");
        const bool coop = ctx->coop_max_blocks > 0 && ctx->allow_coop && !ctx->cfg.implicit_fluxes &&
                          !ctx->cfg.implicit_enthalpy;
        float best_ms = 1e30f;
        if (!status && coop) {
            for (int cpb : {256, 512, 1024, 2048}) {
                Tuning t = best;
                t.coop_cpb = cpb;
                float ms = 0;
                if ((status = time_step(t, ms))) break;
                if (ms < best_ms) { best_ms = ms; best = t; }
            }
        } else if (!status) {
            for (int mult : {4, 8, 16, 32}) {
                Tuning t = best;
                t.inner_grid = nsm * mult;
                t.test_grid = std::max(1, t.inner_grid / 2);
                float ms = 0;
                if ((status = time_step(t, ms))) break;
                if (ms < best_ms) { best_ms = ms; best = t; }
            }
            for (int mult : {2, 4, 16}) {
                if (status) break;
                Tuning t = best;
                t.test_grid = nsm * mult;
                float ms = 0;
                if ((status = time_step(t, ms))) break;
                if (ms < best_ms) { best_ms = ms; best = t; }
            }
        }
        int s3 = copy_state(false);
        if (!status) status = s3;
        if (!status) status = cudaStreamSynchronize(st) == cudaSuccess ? PDAC_OK : fail(ctx, PDAC_ERR_CUDA, "autotune: restore");
        cudaFree(snap);
        ctx->launches = launches; ctx->sweeps = sweeps; ctx->corr_launches = corr_launches;
        ctx->work_cells = work_cells; ctx->tested_cells = tested_cells; ctx->ex_calls = ex_calls;
        ctx->corr_ms = corr_ms; ctx->resid_ms = resid_ms; ctx->inner_ms = inner_ms;
        ctx->last_nit = last_nit; ctx->prof = prof; ctx->sweep_log = sweep_log;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (status) return status;
    put_tuning(ctx, best);
    if (cache_path && !cache_add(cache_path, key, best))
        return fail(ctx, PDAC_ERR_ARG, std::string("autotune: cannot append to ") + cache_path);
    if (out) tuning_out(best, out, nout);
    return PDAC_OK;
}

// ---------------------------------------------------------------------------
// files of the time loop: pdac.res, output.NNNN, pdac.chm
// ---------------------------------------------------------------------------
// the state arrays of tapewr / taperd in file order (io_restart.f:52-118)
static std::vector<std::pair<double *, const char *>> restart_arrays(pdac_ctx *ctx) {
    Fld &F = ctx->F;
    const size_t n = ctx->ncell;
    std::vector<std::pair<double *, const char *>> a;
    a.push_back({F.p, "p"});
    a.push_back({F.ug, "ug"});
    if (ctx->d3) a.push_back({F.vg, "vg"});
    a.push_back({F.wg, "wg"});
    a.push_back({F.sieg, "sieg"});
    for (int is = 0; is < ctx->ns; ++is) a.push_back({F.rlk + is * n, "rlk"});
    for (int is = 0; is < ctx->ns; ++is) {
        a.push_back({F.us + is * n, "us"});
        if (ctx->d3) a.push_back({F.vs + is * n, "vs"});
        a.push_back({F.ws + is * n, "ws"});
    }
    for (int is = 0; is < ctx->ns; ++is) a.push_back({F.sies + is * n, "sies"});
    for (int ig = 0; ig < ctx->ng; ++ig) a.push_back({F.ygc + ig * n, "ygc"});
    a.push_back({F.rgp, "rgp"});
    a.push_back({F.rog, "rog"});
    a.push_back({F.tg, "tg"});
    for (int is = 0; is < ctx->ns; ++is) a.push_back({F.ts + is * n, "ts"});
    return a;
}

// tapewr (io_restart.f:31-124): header (time, nx, ny, nz, nsolid, ngas,
// nfil), gas_type, then one REAL*8 record per array
int pdac_gpu_write_restart(pdac_ctx *ctx, const char *path, double time, int nfil) {
    if (!ctx || !path) return PDAC_ERR_ARG;
    const size_t n = ctx->ncell;
    pdac::io::Writer w(path);
    if (!w.ok) return fail(ctx, PDAC_ERR_ARG, std::string("write_restart: cannot open ") + path);
    unsigned char head[32];
    int32_t dims[6] = {ctx->nx, ctx->ny, ctx->nz, ctx->ns, ctx->ng, nfil};
    std::memcpy(head, &time, 8);
    std::memcpy(head + 8, dims, 24);
    w.record(head, 32);
    std::vector<int32_t> gt(ctx->cfg.gas_type, ctx->cfg.gas_type + ctx->ng);
    w.record(gt.data(), gt.size() * 4);
    std::vector<double> buf(n);
    for (auto &a : restart_arrays(ctx)) {
        CK(cudaMemcpyAsync(buf.data(), a.first, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        w.record(buf.data(), n * sizeof(double));
    }
    if (!w.close()) return fail(ctx, PDAC_ERR_ARG, std::string("write_restart: write error on ") + path);
    return PDAC_OK;
}

// taperd (io_restart.f:126-339) followed by cnvert's restart branch
// (setup.f:359-391): the file's gas types replace the run's; xgc, ep and cg
// are derived from the arrays read
int pdac_gpu_read_restart(pdac_ctx *ctx, const char *path, double *time, int *nfil) {
    if (!ctx || !path) return PDAC_ERR_ARG;
    const size_t n = ctx->ncell;
    pdac::io::Reader r(path);
    if (!r.f) return fail(ctx, PDAC_ERR_ARG, "read_restart: " + r.err);
    unsigned char head[32];
    if (!r.record(head, 32, "the header")) return fail(ctx, PDAC_ERR_ARG, "read_restart: " + r.err);
    double t;
    int32_t dims[6];
    std::memcpy(&t, head, 8);
    std::memcpy(dims, head + 8, 24);
    const char *dn[5] = {"nx", "ny", "nz", "nsolid", "ngas"};
    int want[5] = {ctx->nx, ctx->ny, ctx->nz, ctx->ns, ctx->ng};
    for (int q = 0; q < 5; ++q)
        if (dims[q] != want[q])
            return fail(ctx, PDAC_ERR_ARG, std::string("read_restart: inconsistent dimension ") + dn[q] + " (file " +
                                               std::to_string(dims[q]) + ", run " + std::to_string(want[q]) + ")");
    std::vector<int32_t> gt(ctx->ng);
    if (!r.record(gt.data(), gt.size() * 4, "gas_type")) return fail(ctx, PDAC_ERR_ARG, "read_restart: " + r.err);
    for (int ig = 0; ig < ctx->ng; ++ig)
        if (gt[ig] < 1 || gt[ig] > 7) return fail(ctx, PDAC_ERR_ARG, "read_restart: gas_type out of range");
    bool regas = false;
    for (int ig = 0; ig < ctx->ng; ++ig) regas |= gt[ig] != ctx->cfg.gas_type[ig];
    if (regas) {
        // kernels and captured graphs carry the gas table by value
        for (int ig = 0; ig < ctx->ng; ++ig) ctx->cfg.gas_type[ig] = ctx->P.gas_type[ig] = gt[ig];
        if (ctx->it_exec) { cudaGraphExecDestroy(ctx->it_exec); ctx->it_exec = nullptr; }
        if (ctx->it_graph) { cudaGraphDestroy(ctx->it_graph); ctx->it_graph = nullptr; }
        if (ctx->ex_exec) { cudaGraphExecDestroy(ctx->ex_exec); ctx->ex_exec = nullptr; }
        if (ctx->ex_graph) { cudaGraphDestroy(ctx->ex_graph); ctx->ex_graph = nullptr; }
    }
    std::vector<double> buf(n);
    for (auto &a : restart_arrays(ctx)) {
        if (!r.record(buf.data(), n * sizeof(double), a.second)) return fail(ctx, PDAC_ERR_ARG, "read_restart: " + r.err);
        bool neg = false;
        for (size_t c = 0; c < n && !neg; ++c) neg = buf[c] < 0.0;
        const char *ch = a.second;
        if (neg && std::strcmp(ch, "ug") && std::strcmp(ch, "vg") && std::strcmp(ch, "wg") && std::strcmp(ch, "us") &&
            std::strcmp(ch, "vs") && std::strcmp(ch, "ws"))
            fprintf(stderr, "WARNING reading restart, %s < 0\n", ch);
        CK(cudaMemcpyAsync(a.first, buf.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    pdac::k_restart_derive<<<blocks(n), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    if (time) *time = t;
    if (nfil) *nfil = dims[5];
    return PDAC_OK;
}

// outp (outp.f:194-384), unformatted: REAL(time, 4), then single-precision
// records of p, gas velocity, tg, xgc per gas, and per class eps = rlk/rl,
// particle velocity and ts
// outp (outp.f:194-384): the output fields in the reference's order; the
// mixture fields follow with compute_mixture.  Unformatted: REAL(time, 4)
// and one REAL*4 record per field.  Formatted (formatted_output):
// '(1x,///,1x,"@@@ TIME = ",g11.4)', then per field a header
// '(1x,//,1x,<name>,/)' and the values of each k plane (nx, or nx ny in 3D,
// cells) with FORMAT(1x,10(1x,G14.6E3)), ten to a line
// (write_array, io_parallel.f:38-50).
int pdac_gpu_write_output(pdac_ctx *ctx, const char *path, double time) {
    if (!ctx || !path) return PDAC_ERR_ARG;
    const size_t n = ctx->ncell;
    const bool lform = ctx->cfg.formatted_output != 0;
    Fld &F = ctx->F;
    pdac::io::Writer w(lform ? nullptr : path);
    std::string text;
    if (lform) {
        text = "\n\n\n @@@ TIME = " + pdac::io::fortran_g(time, 11, 4, 2) + "\n";
    } else {
        if (!w.ok) return fail(ctx, PDAC_ERR_ARG, std::string("write_output: cannot open ") + path);
        float t4 = (float)time;
        w.record(&t4, 4);
    }
    std::vector<double> buf(n);
    std::vector<float> sgl(n);
    const size_t ntr = (size_t)ctx->nx * (ctx->d3 ? ctx->ny : 1);
    auto put = [&](const char *head, const double *d, double scale, bool scaled) -> int {
        CK(cudaMemcpyAsync(buf.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (scaled)
            for (size_t c = 0; c < n; ++c) buf[c] = buf[c] * scale;
        if (!lform) {
            for (size_t c = 0; c < n; ++c) sgl[c] = (float)buf[c];
            w.record(sgl.data(), n * sizeof(float));
            return PDAC_OK;
        }
        text += std::string("\n\n ") + head + "\n\n";
        for (size_t first = 0; first < n; first += ntr) {
            text += " ";
            for (size_t q = 0; q < ntr; ++q) {
                if (q > 0 && q % 10 == 0) text += "\n";
                text += " " + pdac::io::fortran_g(buf[first + q], 14, 6, 3);
            }
            text += "\n";
        }
        return PDAC_OK;
    };
    auto name1 = [](const char *pre, int q) { return std::string(pre) + std::to_string(q); };
    int s;
    if ((s = put("P   ", F.p, 1.0, false))) return s;
    if ((s = put("UG  ", F.ug, 1.0, false))) return s;
    if (ctx->d3 && (s = put("VG  ", F.vg, 1.0, false))) return s;
    if ((s = put("WG  ", F.wg, 1.0, false))) return s;
    if ((s = put("TG  ", F.tg, 1.0, false))) return s;
    for (int ig = 0; ig < ctx->ng; ++ig)
        if ((s = put(name1("XGC", ig + 1).c_str(), F.xgc + ig * n, 1.0, false))) return s;
    for (int is = 1; is <= ctx->ns; ++is) {
        size_t off = (size_t)(is - 1) * n;
        if ((s = put(name1("EPS", is).c_str(), F.rlk + off, ctx->P.inrl[is], true))) return s;
        if ((s = put(name1(" US", is).c_str(), F.us + off, 1.0, false))) return s;
        if (ctx->d3 && (s = put(name1(" VS", is).c_str(), F.vs + off, 1.0, false))) return s;
        if ((s = put(name1(" WS", is).c_str(), F.ws + off, 1.0, false))) return s;
        if ((s = put(name1(" TS", is).c_str(), F.ts + off, 1.0, false))) return s;
    }
    if (ctx->cfg.compute_mixture) {
        if ((s = put("RHOM", F.rhom, 1.0, false))) return s;
        if ((s = put("UM  ", F.um, 1.0, false))) return s;
        if (ctx->d3 && (s = put("VM  ", F.vm, 1.0, false))) return s;
        if ((s = put("WM  ", F.wm, 1.0, false))) return s;
        if ((s = put("TM  ", F.tm, 1.0, false))) return s;
        for (int q = 1; q <= ctx->ng + ctx->ns; ++q)
            if ((s = put(name1("YD", q).c_str(), F.yd + (size_t)(q - 1) * n, 1.0, false))) return s;
    }
    if (lform) {
        FILE *f = std::fopen(path, "w");
        if (!f) return fail(ctx, PDAC_ERR_ARG, std::string("write_output: cannot open ") + path);
        bool ok = std::fputs(text.c_str(), f) >= 0;
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) return fail(ctx, PDAC_ERR_ARG, std::string("write_output: write error on ") + path);
        return PDAC_OK;
    }
    if (!w.close()) return fail(ctx, PDAC_ERR_ARG, std::string("write_output: write error on ") + path);
    return PDAC_OK;
}

int pdac_gpu_compute_mixture_fields(pdac_ctx *ctx) {
    if (!ctx) return PDAC_ERR_ARG;
    if (!ctx->F.rhom) return fail(ctx, PDAC_ERR_CONFIG, "compute_mixture_fields: the run has compute_mixture = 0");
    if (ctx->d3) pdac::k_mixture<3><<<blocks(ctx->ncell), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
    else pdac::k_mixture<2><<<blocks(ctx->ncell), TPB, 0, ctx->stream>>>(ctx->P, ctx->F);
    ctx->launches++;
    CK(cudaGetLastError());
    return PDAC_OK;
}

// print_mass_residuals (residuals.f:15-136) and the mass flow rate of
// compute_mass_flow_rate (residuals.f:171-251): out = [res_g, res_s(ns),
// res_gc(ng), mfr]
int pdac_gpu_mass_residuals(pdac_ctx *ctx, int nswp, double dt, double *out, int nout) {
    if (!ctx || !out) return PDAC_ERR_ARG;
    const int ns = ctx->ns, ng = ctx->ng, nres = 2 + ns + ng, nq = 4 + 2 * ns + ng;
    if (nout < nres) return PDAC_ERR_ARG;
    // the partial sums fit the reduction buffer of mass_totals, which holds
    // (1 + ns + ng) x 1024 doubles
    const int nb = 148, tpb = 128;
    double *part = ctx->d_partial;
    pdac::k_mass_resid<<<nb, tpb, (size_t)nq * tpb * sizeof(double), ctx->stream>>>(ctx->P, ctx->F, nswp, dt, part, nq);
    ctx->launches++;
    CK(cudaGetLastError());
    std::vector<double> h((size_t)nq * nb);
    CK(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<double> tot(nq, 0.0);
    for (int q = 0; q < nq; ++q)
        for (int b = 0; b < nb; ++b) tot[q] += h[(size_t)q * nb + b];
    for (int q = 0; q < 1 + ns + ng; ++q) out[q] = tot[q];
    out[1 + ns + ng] = tot[1 + ns + ng];  // mfr
    return PDAC_OK;
}

// one line of pdac.chm, FORMAT(I8,15(G30.20E3)) (residuals.f:123-127),
// appended to path
int pdac_gpu_append_mass_check(pdac_ctx *ctx, const char *path, int nswp, double dt) {
    if (!ctx || !path) return PDAC_ERR_ARG;
    const int nres = 2 + ctx->ns + ctx->ng;
    std::vector<double> v(nres);
    int s = pdac_gpu_mass_residuals(ctx, nswp, dt, v.data(), nres);
    if (s) return s;
    char head[32];
    std::snprintf(head, sizeof head, "%8d", nswp);
    std::string line = head;
    for (int q = 0; q < nres; ++q) {
        // format reversion: after 15 items the line ends and the group repeats
        if (q > 0 && q % 15 == 0) line += "\n";
        line += pdac::io::fortran_g(v[q], 30, 20, 3);
    }
    line += "\n";
    FILE *f = std::fopen(path, "a");
    if (!f) return fail(ctx, PDAC_ERR_ARG, std::string("append_mass_check: cannot open ") + path);
    bool ok = std::fputs(line.c_str(), f) >= 0;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(ctx, PDAC_ERR_ARG, std::string("append_mass_check: write error on ") + path);
    return PDAC_OK;
}

// print_mass_loss (sink.f:123-167): the columns' accumulated mass in the
// reference's formatted layout, FORMAT(10(1x,G14.6E3)): in 2D one line per
// column i with the ns values and the running total over the columns, in
// 3D per solid a header '(1x,//,1x,"ML",I1,"=",G14.6,/)' with that solid's
// total and then the ntr column values, ten to a line
int pdac_gpu_write_mass_loss(pdac_ctx *ctx, const char *path) {
    if (!ctx || !path) return PDAC_ERR_ARG;
    if (ctx->S.ntr == 0) return fail(ctx, PDAC_ERR_CONFIG, "write_mass_loss: the run has no sink (isink = 0)");
    const int ntr = ctx->S.ntr, ns = ctx->ns;
    std::vector<double> ml((size_t)ntr * ns);
    CK(cudaMemcpyAsync(ml.data(), ctx->S.massl, ml.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    auto at = [&](int b, int is) { return ml[(size_t)(is - 1) * ntr + b]; };
    std::string out;
    auto group = [&](const std::vector<double> &v) {
        for (size_t q = 0; q < v.size(); ++q) {
            if (q > 0 && q % 10 == 0) out += "\n";
            out += " " + pdac::io::fortran_g(v[q], 14, 6, 3);
        }
        out += "\n";
    };
    if (!ctx->d3) {
        double masstotal = 0.0;
        for (int b = 0; b < ntr; ++b) {
            double sum = 0.0;
            std::vector<double> v;
            for (int is = 1; is <= ns; ++is) { sum = sum + at(b, is); v.push_back(at(b, is)); }
            masstotal = masstotal + sum;
            v.push_back(masstotal);
            group(v);
        }
    } else {
        for (int is = 1; is <= ns; ++is) {
            double masstotal = 0.0;
            std::vector<double> v(ntr);
            for (int b = 0; b < ntr; ++b) { masstotal = masstotal + at(b, is); v[b] = at(b, is); }
            char head[64];
            std::snprintf(head, sizeof head, "\n\n ML%1d=", is);
            out += head + pdac::io::fortran_g(masstotal, 14, 6, 2) + "\n\n";
            group(v);
        }
    }
    FILE *f = std::fopen(path, "w");
    if (!f) return fail(ctx, PDAC_ERR_ARG, std::string("write_mass_loss: cannot open ") + path);
    bool ok = std::fputs(out.c_str(), f) >= 0;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(ctx, PDAC_ERR_ARG, std::string("write_mass_loss: write error on ") + path);
    return PDAC_OK;
}

// read_mass_loss (sink.f:168-207): a file written by print_mass_loss into
// the values that the next sink update of each column adds back
int pdac_gpu_read_mass_loss(pdac_ctx *ctx, const char *path) {
    if (!ctx || !path) return PDAC_ERR_ARG;
    if (ctx->S.ntr == 0) return fail(ctx, PDAC_ERR_CONFIG, "read_mass_loss: the run has no sink (isink = 0)");
    const int ntr = ctx->S.ntr, ns = ctx->ns;
    FILE *f = std::fopen(path, "r");
    if (!f) return fail(ctx, PDAC_ERR_ARG, std::string("read_mass_loss: cannot open ") + path);
    std::vector<std::string> tok;
    char word[256];
    while (std::fscanf(f, "%255s", word) == 1) tok.push_back(word);
    std::fclose(f);
    std::vector<double> ml((size_t)ntr * ns);
    size_t q = 0;
    auto num = [&](double &x) {
        if (q >= tok.size()) return false;
        char *end = nullptr;
        x = std::strtod(tok[q].c_str(), &end);
        return end && *end == '\0' && tok[q++].size() > 0;
    };
    bool ok = true;
    if (!ctx->d3) {
        for (int b = 0; b < ntr && ok; ++b) {
            double total;
            for (int is = 1; is <= ns && ok; ++is) ok = num(ml[(size_t)(is - 1) * ntr + b]);
            ok = ok && num(total);
        }
    } else {
        for (int is = 1; is <= ns && ok; ++is) {
            double total;
            ok = q < tok.size() && tok[q].rfind("ML", 0) == 0;
            if (ok) ++q;
            ok = ok && num(total);
            for (int b = 0; b < ntr && ok; ++b) ok = num(ml[(size_t)(is - 1) * ntr + b]);
        }
    }
    if (!ok || q != tok.size()) return fail(ctx, PDAC_ERR_ARG, std::string("read_mass_loss: unexpected layout in ") + path);
    CK(cudaMemcpyAsync(ctx->S.mass_loss, ml.data(), ml.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PDAC_OK;
}

// vent fluctuation factors for the next boundary call (random_switch, vent.f:824-873)
int pdac_gpu_set_vent_factors(pdac_ctx *ctx, const double *fact, int nvent) {
    if (!ctx || !fact || nvent != ctx->nvent) return PDAC_ERR_ARG;
    CK(cudaMemcpyAsync(ctx->d_vfact, fact, nvent * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PDAC_OK;
}


// statistics: out[0] kernel launches, out[1] outer sweeps, out[2] timed
// corrector launches, out[3] their total device time in ms
int pdac_gpu_stats(pdac_ctx *ctx, double *out, int nout) {
    if (!ctx || !out || nout < 4) return PDAC_ERR_ARG;
    out[0] = (double)ctx->launches;
    out[1] = (double)ctx->sweeps;
    out[2] = (double)ctx->corr_launches;
    out[3] = ctx->corr_ms;
    if (nout >= 7) {
        out[4] = ctx->resid_ms;
        out[5] = ctx->inner_ms;
        out[6] = (double)ctx->work_cells;
    }
    if (nout >= 8) out[7] = (double)ctx->tested_cells;
    if (nout >= 13) {
        for (int q = 0; q < 4; ++q) out[8 + q] = ctx->ex_ms[q];
        out[12] = (double)ctx->ex_calls;
    }
    return PDAC_OK;
}

int pdac_gpu_reset_stats(pdac_ctx *ctx, int profile_corrector) {
    if (!ctx) return PDAC_ERR_ARG;
    ctx->launches = ctx->sweeps = ctx->corr_launches = ctx->work_cells = ctx->tested_cells = 0;
    ctx->corr_ms = ctx->resid_ms = ctx->inner_ms = 0.0;
    for (double &x : ctx->ex_ms) x = 0.0;
    ctx->ex_calls = 0;
    ctx->sweep_log.clear();
    ctx->prof = profile_corrector != 0;
    return PDAC_OK;
}

// per colour phase since the last profiling reset: sweep, colour, worklist
// length, cells tested, residual-test ms, inner-loop ms (6 doubles each)
int pdac_gpu_sweep_log(pdac_ctx *ctx, double *out, long *n_inout) {
    if (!ctx || !n_inout) return PDAC_ERR_ARG;
    long need = (long)ctx->sweep_log.size();
    if (!out || *n_inout < need) { *n_inout = need; return need ? PDAC_ERR_ARG : PDAC_OK; }
    std::copy(ctx->sweep_log.begin(), ctx->sweep_log.end(), out);
    *n_inout = need;
    return PDAC_OK;
}

// record a timing mark (0..31) on the context's stream
int pdac_gpu_mark(pdac_ctx *ctx, int slot) {
    if (!ctx || slot < 0 || slot >= 32) return PDAC_ERR_ARG;
    CK(cudaEventRecord(ctx->user_ev[slot], ctx->stream));
    return PDAC_OK;
}

// device time between two marks, after synchronising the stream
int pdac_gpu_elapsed(pdac_ctx *ctx, int a, int b, double *ms) {
    if (!ctx || !ms || a < 0 || b < 0 || a >= 32 || b >= 32) return PDAC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    float t = 0;
    CK(cudaEventElapsedTime(&t, ctx->user_ev[a], ctx->user_ev[b]));
    *ms = t;
    return PDAC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// ensembles: many independent contexts advanced together
// ---------------------------------------------------------------------------
// Each member keeps its own stream, graphs and host synchronisation points
// (the sweep count of iter, the caloric-failure count of ftem); a pool of
// host threads runs pdac_gpu_step on the members, so the members' kernels
// run concurrently on the device while one member's host waits for its own
// stream.  Small 2D members fill a few percent of the SMs each; run side by
// side they fill the device.  Members are spread over the threads by the
// longest-processing-time rule on their cell counts.
// ---------------------------------------------------------------------------
// the whole semi-implicit time step as one CUDA graph (prog.f:162-331 with
// rungekut = 1): boundary, fieldn, the sub-grid models, tilde and iter's
// set-up as one child graph, the outer sweep loop as a conditional WHILE node
// (the body of pdac_gpu_iter's graph), then ygas, htilde, ftem, the mixture
// fields, the non-finite check and the copy of the step's outcome to pinned
// host memory as a second child graph.  The same kernels in the same order
// as pdac_gpu_step, so the same results; a batch launches it for each of its
// members from one host thread.
// ---------------------------------------------------------------------------
namespace pdac {
__global__ void k_set_int(int *p, int v) { *p = v; }
__global__ void k_step_status(const int *nit, const int *counters, const int *nonfinite, int *out) {
    out[0] = *nit;
    out[1] = counters[1];
    out[2] = *nonfinite;
}
}  // namespace pdac

static bool step_graph_eligible(const pdac_ctx *ctx) {
    const pdac_cfg &c = ctx->cfg;
    return ctx->ti == 0 && c.rungekut == 1 && !c.implicit_fluxes && !c.implicit_enthalpy && !c.cstop &&
           !c.update_eosg && ctx->ng > 1;
}

static int enqueue_step_pre(pdac_ctx *ctx, double dt, cudaStream_t st) {
    int s;
    if ((s = enqueue_boundary(ctx, st)) || (s = enqueue_fieldn(ctx, st))) return s;
    if ((s = pdac_gpu_sgsg(ctx)) || (s = pdac_gpu_sgss(ctx))) return s;
    if ((s = enqueue_tilde(ctx, dt, st))) return s;
    // iter's set-up, as in pdac_gpu_iter
    Fld &F = ctx->F;
    const size_t n = ctx->ncell, ns = ctx->ns;
    CK(cudaMemsetAsync(ctx->d_counters + 5, 0, sizeof(int), st));
    for (double *a : {F.rgfe, F.rgfn, F.rgft, F.conv, F.abeta})
        if (a) CK(cudaMemsetAsync(a, 0, n * sizeof(double), st));
    for (double *a : {F.rsfe, F.rsfn, F.rsft})
        if (a) CK(cudaMemsetAsync(a, 0, n * ns * sizeof(double), st));
    const int nph = ctx->nph;
    if (ctx->d3) {
        PHASE_LAUNCH(nph, pdac::k_predictor3d, blocks(n), TPB, st, ctx->P, F, dt);
        pdac::k_mflux_init3d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt);
    } else {
        PHASE_LAUNCH(nph, pdac::k_predictor2d, blocks(n), TPB, st, ctx->P, F, dt);
        pdac::k_mflux_init2d<<<blocks(n), TPB, 0, st>>>(ctx->P, F, dt);
    }
    CK(cudaMemsetAsync(ctx->d_dirty, 0xff, (n + 31) / 32 * sizeof(unsigned), st));
    pdac::k_set_int<<<1, 1, 0, st>>>(ctx->d_nit, 1);
    ctx->launches += 3;
    CK(cudaGetLastError());
    return PDAC_OK;
}

static int enqueue_step_post(pdac_ctx *ctx, double dt, cudaStream_t st) {
    int s;
    if ((s = enqueue_ygas(ctx, dt, st)) || (s = enqueue_htilde(ctx, dt, st)) || (s = enqueue_ftem(ctx, dt, st, false)))
        return s;
    if (ctx->cfg.compute_mixture) {
        if (ctx->d3) pdac::k_mixture<3><<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F);
        else pdac::k_mixture<2><<<blocks(ctx->ncell), TPB, 0, st>>>(ctx->P, ctx->F);
        ctx->launches++;
    }
    // check_step_state's fields, without its host read
    const Fld &F = ctx->F;
    const size_t n = ctx->ncell;
    pdac::FinList L{};
    const double *arr[6] = {F.p, F.ep, F.rgp, F.tg, F.sieg, F.rlk};
    for (int q = 0; q < 6; ++q) { L.a[q] = arr[q]; L.n[q] = (long long)(q == 5 ? n * ctx->ns : n); }
    L.m = 6;
    int dev = 0, nsm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaMemsetAsync(ctx->d_nonfinite, 0, sizeof(int), st));
    pdac::k_nonfinite<<<nsm * 8, 256, 0, st>>>(L, ctx->d_nonfinite);
    pdac::k_step_status<<<1, 1, 0, st>>>(ctx->d_nit, ctx->d_counters, ctx->d_nonfinite, ctx->d_status);
    CK(cudaMemcpyAsync(ctx->h_status, ctx->d_status, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    ctx->launches += 2;
    CK(cudaGetLastError());
    return PDAC_OK;
}

// the nodes of one whole semi-implicit step of ctx in graph g: the kernels
// before the sweep loop (a child graph), the loop as a conditional WHILE
// node, the kernels after it (a child graph, ending with the step's status
// copied to pinned host memory); the kernels are captured on ctx's stream
static int add_step_nodes(pdac_ctx *ctx, cudaGraph_t g) {
    const double dt = ctx->cfg.dt;
    cudaStream_t st = ctx->stream;
    const long long before = ctx->launches;
    cudaGraph_t part = nullptr;
    // the kernels before the sweep loop
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    int s = enqueue_step_pre(ctx, dt, st);
    cudaError_t e = cudaStreamEndCapture(st, &part);
    if (s) { ctx->launches = before; return s; }
    CK(e);
    cudaGraphNode_t pre, loop_node, post;
    e = cudaGraphAddChildGraphNode(&pre, g, nullptr, 0, part);
    cudaGraphDestroy(part);
    CK(e);
    // the sweep loop
    cudaGraphConditionalHandle loop;
    CK(cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault));
    alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams &cp = *reinterpret_cast<cudaGraphNodeParams *>(cp_storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    CK(cudaGraphAddNode(&loop_node, g, &pre, 1, &cp));
    CK(cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const long long mid = ctx->launches;
    s = enqueue_sweep(ctx, dt, st, false);
    ctx->it_per_sweep = sweep_kernels(ctx) + (ctx->launches - mid);
    ctx->launches = mid;
    if (!s) pdac::k_sweep_check<<<1, 1, 0, st>>>(ctx->d_wcount, ctx->d_nit, ctx->cfg.maxout, loop);
    cudaGraph_t body = nullptr;
    e = cudaStreamEndCapture(st, &body);
    if (s) { ctx->launches = before; return s; }
    CK(e);
    // the kernels after it
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    s = enqueue_step_post(ctx, dt, st);
    e = cudaStreamEndCapture(st, &part);
    ctx->step_launches = ctx->launches - before;
    ctx->launches = before;
    if (s) return s;
    CK(e);
    e = cudaGraphAddChildGraphNode(&post, g, &loop_node, 1, part);
    cudaGraphDestroy(part);
    CK(e);
    return PDAC_OK;
}

static int build_step_graph(pdac_ctx *ctx) {
    if (ctx->step_exec) { cudaGraphExecDestroy(ctx->step_exec); ctx->step_exec = nullptr; }
    if (ctx->step_graph) { cudaGraphDestroy(ctx->step_graph); ctx->step_graph = nullptr; }
    CK(cudaGraphCreate(&ctx->step_graph, 0));
    int s = add_step_nodes(ctx, ctx->step_graph);
    if (s) return s;
    CK(cudaGraphInstantiate(&ctx->step_exec, ctx->step_graph, 0));
    return PDAC_OK;
}

// after a graph step has completed: its sweep count and status
static int step_graph_outcome(pdac_ctx *ctx, int *nit) {
    const int *h = ctx->h_status;
    const int done = std::min(h[0], ctx->cfg.maxout);
    ctx->sweeps += done;
    ctx->launches += ctx->step_launches + ctx->it_per_sweep * done;
    ctx->last_nit = h[0];
    if (nit) *nit = h[0];
    if (h[2]) return fail(ctx, PDAC_ERR_NONFINITE, "step: non-finite value in p, ep, rgp, tg, sieg or rlk");
    if (h[1] > 1) return fail(ctx, PDAC_ERR_EOS, "ftem: caloric equation of state failed");
    return PDAC_OK;
}

struct pdac_batch {
    std::vector<pdac_ctx *> m;
    std::vector<char> graph;             // member i steps as one CUDA graph launched by the caller's thread
    std::vector<std::vector<int>> work;  // the other members, by thread
    std::vector<std::thread> th;
    std::mutex mu;
    std::condition_variable go, done;
    long gen = 0;
    int pending = 0, sweep = 0, dev = 0;
    bool quit = false;
    std::vector<int> nit, status;
    cudaStream_t lead = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> fin;
    double last_ms = 0.0;
    std::string err;
    // every graph member's whole step in one graph, launched once per batch
    // step on the lead stream (the members' branches are independent); the
    // members' graph generations it was built at
    cudaGraph_t bgraph = nullptr;
    cudaGraphExec_t bexec = nullptr;
    std::vector<long> bgen;
    bool one_graph = true;
};

static void batch_worker(pdac_batch *b, int w) {
    cudaSetDevice(b->dev);
    long seen = 0;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(b->mu);
            b->go.wait(lk, [&] { return b->quit || b->gen != seen; });
            if (b->quit) return;
            seen = b->gen;
        }
        for (int i : b->work[w]) {
            pdac_ctx *c = b->m[i];
            int nit = 0, s = PDAC_OK;
            if (cudaStreamWaitEvent(c->stream, b->t0, 0) != cudaSuccess) s = PDAC_ERR_CUDA;
            if (!s) s = pdac_gpu_step(c, b->sweep, &nit);
            // the completion mark is recorded whatever the status, so that
            // the lead stream's wait below always refers to this step
            cudaEventRecord(b->fin[i], c->stream);
            b->nit[i] = nit;
            b->status[i] = s;
        }
        std::lock_guard<std::mutex> lk(b->mu);
        if (--b->pending == 0) b->done.notify_all();
    }
}

static void batch_free(pdac_batch *b) {
    {
        std::lock_guard<std::mutex> lk(b->mu);
        b->quit = true;
    }
    b->go.notify_all();
    for (auto &t : b->th) t.join();
    for (pdac_ctx *c : b->m) {
        c->allow_coop = true;
        c->ex_dt = -1.0;
    }
    for (auto e : b->fin) if (e) cudaEventDestroy(e);
    if (b->bexec) cudaGraphExecDestroy(b->bexec);
    if (b->bgraph) cudaGraphDestroy(b->bgraph);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    if (b->lead) cudaStreamDestroy(b->lead);
    delete b;
}

extern "C" {

int pdac_gpu_batch_create(pdac_ctx *const *members, int nmember, int nthreads, pdac_batch **out) {
    if (!members || !out || nmember < 1) return PDAC_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < nmember; ++i) {
        if (!members[i]) return PDAC_ERR_ARG;
        for (int j = 0; j < i; ++j)
            if (members[j] == members[i]) return PDAC_ERR_ARG;  // one context stepped twice at once would race
    }
    pdac_batch *b = new pdac_batch();
    b->m.assign(members, members + nmember);
    // semi-implicit members step as whole-step graphs; the others (explicit
    // solver, implicit-flux modes, cstop, one gas ...) through pdac_gpu_step
    // on the thread pool
    b->graph.assign(nmember, 0);
    int nthread_members = 0;
    for (int i = 0; i < nmember; ++i) {
        b->graph[i] = step_graph_eligible(members[i]) ? 1 : 0;
        nthread_members += b->graph[i] ? 0 : 1;
    }
    int nt = nthreads > 0 ? std::min(nthreads, nthread_members) : nthread_members;
    // members take the non-cooperative paths while in the batch (the
    // explicit_iter graph, built with the cooperative wavefront, is rebuilt)
    for (pdac_ctx *c : b->m) {
        c->allow_coop = false;
        c->ex_dt = -1.0;
    }
    b->nit.assign(nmember, 0);
    b->status.assign(nmember, 0);
    b->fin.assign(nmember, nullptr);
    if (cudaGetDevice(&b->dev) != cudaSuccess || cudaStreamCreateWithFlags(&b->lead, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess) {
        batch_free(b);
        return PDAC_ERR_CUDA;
    }
    for (auto &e : b->fin)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            batch_free(b);
            return PDAC_ERR_CUDA;
        }
    // longest processing time first: each member, largest first, to the
    // thread with the fewest cells so far
    std::vector<int> order(nmember);
    for (int i = 0; i < nmember; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->m[a]->ncell > b->m[c]->ncell; });
    std::vector<long> load(nt, 0);
    b->work.assign(nt, {});
    for (int i : order) {
        if (b->graph[i]) continue;
        int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->work[w].push_back(i);
        load[w] += b->m[i]->ncell;
    }
    for (int w = 0; w < nt; ++w) b->th.emplace_back(batch_worker, b, w);
    *out = b;
    return PDAC_OK;
}

// (re)build the batch graph: every graph member's step nodes in one graph
static int build_batch_graph(pdac_batch *b) {
    if (b->bexec) { cudaGraphExecDestroy(b->bexec); b->bexec = nullptr; }
    if (b->bgraph) { cudaGraphDestroy(b->bgraph); b->bgraph = nullptr; }
    if (cudaGraphCreate(&b->bgraph, 0) != cudaSuccess) return PDAC_ERR_CUDA;
    b->bgen.assign(b->m.size(), -1);
    for (size_t i = 0; i < b->m.size(); ++i) {
        if (!b->graph[i]) continue;
        int s = add_step_nodes(b->m[i], b->bgraph);
        if (s) return s;
        b->bgen[i] = b->m[i]->graph_gen;
    }
    if (cudaGraphInstantiate(&b->bexec, b->bgraph, 0) != cudaSuccess) {
        cudaGetLastError();
        return PDAC_ERR_CUDA;
    }
    return PDAC_OK;
}

int pdac_gpu_batch_step(pdac_batch *b, int sweep, int *nit, int *status) {
    if (!b) return PDAC_ERR_ARG;
    std::vector<char> launched(b->m.size(), 0);
    bool any_graph = false;
    for (size_t i = 0; i < b->m.size(); ++i) any_graph = any_graph || b->graph[i];
    // the batch graph runs on the lead stream: it first waits for what the
    // graph members' own streams hold (uploads, set-up)
    if (any_graph && b->one_graph)
        for (size_t i = 0; i < b->m.size(); ++i) {
            if (!b->graph[i]) continue;
            if (cudaEventRecord(b->fin[i], b->m[i]->stream) != cudaSuccess ||
                cudaStreamWaitEvent(b->lead, b->fin[i], 0) != cudaSuccess)
                return PDAC_ERR_CUDA;
        }
    if (cudaEventRecord(b->t0, b->lead) != cudaSuccess) return PDAC_ERR_CUDA;
    // the graph members: all in one graph launched on the lead stream, built
    // at the first batch step with the members' streams idle (and again when
    // a member's launch shapes change); if that graph cannot be built, one
    // graph launch per member from this thread
    bool stale = !b->bexec;
    for (size_t i = 0; i < b->m.size() && !stale; ++i) stale = b->graph[i] && b->bgen[i] != b->m[i]->graph_gen;
    if (any_graph && b->one_graph && stale && build_batch_graph(b) != PDAC_OK) {
        b->one_graph = false;
        if (b->bexec) { cudaGraphExecDestroy(b->bexec); b->bexec = nullptr; }
        if (b->bgraph) { cudaGraphDestroy(b->bgraph); b->bgraph = nullptr; }
        for (pdac_ctx *c : b->m) c->err.clear();
    }
    if (any_graph && b->one_graph) {
        const bool ok = cudaGraphLaunch(b->bexec, b->lead) == cudaSuccess;
        for (size_t i = 0; i < b->m.size(); ++i) {
            if (!b->graph[i]) continue;
            b->status[i] = ok ? PDAC_OK : fail(b->m[i], PDAC_ERR_CUDA, "batch: batch graph launch failed");
            b->nit[i] = 0;
            launched[i] = ok;
        }
    } else {
        for (size_t i = 0; i < b->m.size(); ++i) {
            if (!b->graph[i]) continue;
            pdac_ctx *c = b->m[i];
            int s = c->step_exec ? PDAC_OK : build_step_graph(c);
            if (!s && (cudaStreamWaitEvent(c->stream, b->t0, 0) != cudaSuccess ||
                       cudaGraphLaunch(c->step_exec, c->stream) != cudaSuccess))
                s = fail(c, PDAC_ERR_CUDA, "batch: step graph launch failed");
            cudaEventRecord(b->fin[i], c->stream);
            b->status[i] = s;
            b->nit[i] = 0;
            launched[i] = s == PDAC_OK;
        }
    }
    {
        std::lock_guard<std::mutex> lk(b->mu);
        b->sweep = sweep;
        b->pending = (int)b->th.size();
        b->gen++;
    }
    b->go.notify_all();
    {
        std::unique_lock<std::mutex> lk(b->mu);
        b->done.wait(lk, [&] { return b->pending == 0; });
    }
    for (size_t i = 0; i < b->m.size(); ++i) {
        if (b->graph[i] && b->one_graph) continue;  // ran on the lead stream
        if (cudaStreamWaitEvent(b->lead, b->fin[i], 0) != cudaSuccess) return PDAC_ERR_CUDA;
    }
    if (cudaEventRecord(b->t1, b->lead) != cudaSuccess || cudaEventSynchronize(b->t1) != cudaSuccess) return PDAC_ERR_CUDA;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, b->t0, b->t1) != cudaSuccess) return PDAC_ERR_CUDA;
    b->last_ms = ms;
    for (size_t i = 0; i < b->m.size(); ++i)
        if (launched[i]) b->status[i] = step_graph_outcome(b->m[i], &b->nit[i]);
    int first = PDAC_OK;
    for (size_t i = 0; i < b->m.size(); ++i) {
        if (nit) nit[i] = b->nit[i];
        if (status) status[i] = b->status[i];
        if (b->status[i] && !first) {
            first = b->status[i];
            b->err = "member " + std::to_string(i) + ": " + b->m[i]->err;
        }
    }
    return first;
}

int pdac_gpu_batch_elapsed(pdac_batch *b, double *ms) {
    if (!b || !ms) return PDAC_ERR_ARG;
    *ms = b->last_ms;
    return PDAC_OK;
}

const char *pdac_gpu_batch_last_error(const pdac_batch *b) { return b ? b->err.c_str() : "null batch"; }

int pdac_gpu_batch_destroy(pdac_batch *b) {
    if (!b) return PDAC_ERR_ARG;
    batch_free(b);
    return PDAC_OK;
}

}  // extern "C"

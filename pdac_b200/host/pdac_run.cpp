// pdac_run.cpp -- the time loop of PDAC's main program (prog.f:143-417) as a
// compiled host over the C ABI of include/pdac_gpu.h.
//
//     pdac_run CASEFILE WORKDIR [MAX_STEPS]
//
// CASEFILE is a set-up run (pdac_b200/casefile.py: the cfg struct, the
// &control values of the loop, mesh, flags, atmosphere, vent cells and the
// initial state).  The loop writes the reference's files into WORKDIR:
// output.NNNN at the first step and every nprint steps (outp, prog.f:165,
// 357), massl.NNNN before each of those and massl.res after each restart
// file with the ground sink (prog.f:355, 386), pdac.chm every step with
// imr >= 1 (prog.f:363) and pdac.res every ndump steps or when max_seconds
// is exceeded (tapewr, prog.f:385), with nprint = NINT(tpr/dt) and ndump =
// NINT(tdump/dt) (prog.f:84-85).  A restart case starts from WORKDIR's
// pdac.res (and massl.NNNN of the namelist's nfil), setup.f:146-150.  Any
// non-zero status of the engine ends the run with its message, as the
// reference's error() does (comm/error.F).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pdac_gpu.h"

namespace {

struct Control {
    double tstop, tpr, tdump, max_seconds;
    int imr, nfil, restart, isink, compute_mixture;
};

struct Reader {
    FILE *f = nullptr;
    bool ok = true;
    template <class T>
    void get(std::vector<T> &v, size_t n) {
        v.resize(n);
        if (ok && n && std::fread(v.data(), sizeof(T), n, f) != n) ok = false;
    }
    void raw(void *p, size_t n) {
        if (ok && std::fread(p, 1, n, f) != n) ok = false;
    }
};

// letter.f:1-21
std::string lettera(int k) {
    int ithou = k / 1000, ihund = (k - ithou * 1000) / 100, iten = (k - ithou * 1000 - ihund * 100) / 10;
    int ione = k - ithou * 1000 - ihund * 100 - iten * 10;
    std::string s;
    for (int v : {ithou, ihund, iten, ione}) s += (char)(v + 48);
    return s;
}

// Fortran NINT: nearest integer, halves away from zero
int nint(double x) { return (int)std::floor(std::fabs(x) + 0.5) * (x >= 0 ? 1 : -1); }

int check(pdac_ctx *ctx, int st, const char *what) {
    if (st != PDAC_OK) std::fprintf(stderr, "pdac_run: %s: status %d: %s\n", what, st, pdac_gpu_last_error(ctx));
    return st;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: pdac_run CASEFILE WORKDIR [MAX_STEPS]\n");
        return 2;
    }
    const std::string dir = argv[2];
    const long max_steps = argc > 3 ? std::atol(argv[3]) : -1;
    auto path = [&](const std::string &name) { return dir + "/" + name; };

    // ---- the case -----------------------------------------------------------
    Reader r;
    r.f = std::fopen(argv[1], "rb");
    if (!r.f) {
        std::fprintf(stderr, "pdac_run: cannot open %s\n", argv[1]);
        return 2;
    }
    char magic[8];
    r.raw(magic, 8);
    if (!r.ok || std::memcmp(magic, "PDACCAS1", 8) != 0) {
        std::fprintf(stderr, "pdac_run: %s is not a case file\n", argv[1]);
        return 2;
    }
    pdac_cfg cfg;
    std::memset(&cfg, 0, sizeof cfg);
    r.raw(&cfg, sizeof cfg);
    Control ctl = {};
    r.raw(&ctl.tstop, 8); r.raw(&ctl.tpr, 8); r.raw(&ctl.tdump, 8); r.raw(&ctl.max_seconds, 8);
    r.raw(&ctl.imr, 4); r.raw(&ctl.nfil, 4); r.raw(&ctl.restart, 4); r.raw(&ctl.isink, 4);
    r.raw(&ctl.compute_mixture, 4);
    const bool dims_ok = cfg.nx > 0 && cfg.nz > 0 && (cfg.job_type != 3 || cfg.ny > 0) && cfg.nsolid >= 0 &&
                         cfg.nsolid <= PDAC_MAX_NSOLID && cfg.ngas >= 0 && cfg.ngas <= PDAC_MAX_NGAS &&
                         cfg.nvent >= 0 && (double)cfg.nx * (cfg.job_type == 3 ? cfg.ny : 1) * cfg.nz < 2.0e9;
    if (!r.ok || !dims_ok) {
        std::fclose(r.f);
        std::fprintf(stderr, "pdac_run: %s is truncated or its dimensions are invalid\n", argv[1]);
        return 2;
    }
    const bool d3 = cfg.job_type == 3;
    const size_t nx = cfg.nx, ny = d3 ? cfg.ny : 1, nz = cfg.nz, n = nx * ny * nz;
    const size_t ns = cfg.nsolid, ng = cfg.ngas;
    std::vector<double> dx, dy, dz, p_atm, t_atm;
    std::vector<int32_t> flag, vent;
    r.get(dx, nx);
    if (d3) r.get(dy, ny);
    r.get(dz, nz);
    r.get(flag, n);
    r.get(p_atm, nz);
    r.get(t_atm, nz);
    r.get(vent, (size_t)cfg.nvent);
    const char *names[] = {"p", "ep", "rog", "rgp", "tg", "sieg", "cg", "ug", "vg", "wg",
                           "rlk", "ts", "sies", "us", "vs", "ws", "ygc", "xgc"};
    std::vector<std::vector<double>> fields(18);
    for (int q = 0; q < 18; ++q) {
        std::string nm = names[q];
        if (!d3 && (nm == "vg" || nm == "vs")) continue;
        size_t len = n * (q >= 10 && q <= 15 ? ns : (q >= 16 ? ng : 1));
        r.get(fields[q], len);
    }
    bool ok = r.ok;
    std::fclose(r.f);
    if (!ok) {
        std::fprintf(stderr, "pdac_run: %s is truncated\n", argv[1]);
        return 2;
    }
    cfg.dx = dx.data();
    cfg.dy = d3 ? dy.data() : nullptr;
    cfg.dz = dz.data();
    cfg.flag = flag.data();
    cfg.p_atm = p_atm.data();
    cfg.t_atm = t_atm.data();
    cfg.vent_ijk = cfg.nvent > 0 ? vent.data() : nullptr;
    pdac_state_view view;
    double **slot[] = {&view.p, &view.ep, &view.rog, &view.rgp, &view.tg, &view.sieg, &view.cg, &view.ug, &view.vg,
                       &view.wg, &view.rlk, &view.ts, &view.sies, &view.us, &view.vs, &view.ws, &view.ygc, &view.xgc};
    for (int q = 0; q < 18; ++q) *slot[q] = fields[q].empty() ? nullptr : fields[q].data();

    // ---- set-up (pdac.f, setup.f) -----------------------------------------
    pdac_ctx *ctx = nullptr;
    int st = pdac_gpu_create(&cfg, &ctx);
    if (st != PDAC_OK) {
        std::fprintf(stderr, "pdac_run: create: status %d: %s\n", st, pdac_gpu_last_error(ctx));
        return 1;
    }
    int rc = 0;
    auto run = [&]() -> int {
        if (check(ctx, pdac_gpu_upload_state(ctx, &view), "upload_state")) return 1;
        double t = 0.0;
        int nfil = 0;
        if (ctl.restart) {
            if (ctl.isink > 0 &&
                check(ctx, pdac_gpu_read_mass_loss(ctx, path("massl." + lettera(ctl.nfil)).c_str()), "read_mass_loss"))
                return 1;
            if (check(ctx, pdac_gpu_read_restart(ctx, path("pdac.res").c_str(), &t, &nfil), "read_restart")) return 1;
        }
        const double dt = cfg.dt;
        const int nprint = std::max(1, nint(ctl.tpr / dt)), ndump = std::max(1, nint(ctl.tdump / dt));
        int sweep = nint(t / dt);
        const bool expl = cfg.time_integration == 1;
        const bool ifx = cfg.implicit_fluxes != 0, ien = cfg.implicit_enthalpy != 0;
        const auto w0 = std::chrono::steady_clock::now();
        long steps = 0;
        for (;;) {
            ++sweep;
            if (check(ctx, pdac_gpu_boundary(ctx, sweep), "boundary")) return 1;
            if (sweep == 1) {
                if (check(ctx, pdac_gpu_write_output(ctx, path("output." + lettera(nfil)).c_str(), t), "outp")) return 1;
                ++nfil;
            }
            if (check(ctx, expl ? pdac_gpu_initialize_fieldn(ctx) : pdac_gpu_fieldn(ctx), "fieldn")) return 1;
            if (check(ctx, pdac_gpu_sgsg(ctx), "sgsg") || check(ctx, pdac_gpu_sgss(ctx), "sgss")) return 1;
            int nit = 0;
            for (int rk = 1; rk <= cfg.rungekut; ++rk) {
                const double dtr = dt / (cfg.rungekut + 1 - rk);
                if (expl) {
                    if (check(ctx, pdac_gpu_explicit_iter(ctx, dtr), "explicit_iter")) return 1;
                    if (check(ctx, pdac_gpu_ygas(ctx, dtr), "ygas")) return 1;
                    continue;
                }
                // prog.f:246-292
                if (!ifx) {
                    if (check(ctx, pdac_gpu_tilde(ctx, dtr), "tilde")) return 1;
                    if (ien && check(ctx, pdac_gpu_htilde(ctx, dtr), "htilde")) return 1;
                }
                if (check(ctx, pdac_gpu_iter(ctx, dtr, &nit), "iter")) return 1;
                if (check(ctx, pdac_gpu_ygas(ctx, dtr), "ygas")) return 1;
                if (!ien) {
                    if (check(ctx, pdac_gpu_htilde(ctx, dtr), "htilde")) return 1;
                    if (check(ctx, pdac_gpu_ftem(ctx, dtr), "ftem")) return 1;
                }
            }
            if (ctl.compute_mixture &&
                check(ctx, pdac_gpu_compute_mixture_fields(ctx), "compute_mixture_fields"))  // prog.f:331
                return 1;
            t = t + dt;
            std::printf("Iteration: %6d nit: %5d\n", sweep, nit);
            if (sweep % nprint == 0) {
                if (ctl.isink > 0 &&
                    check(ctx, pdac_gpu_write_mass_loss(ctx, path("massl." + lettera(nfil)).c_str()), "print_mass_loss"))
                    return 1;
                if (check(ctx, pdac_gpu_write_output(ctx, path("output." + lettera(nfil)).c_str(), t), "outp")) return 1;
                ++nfil;
            }
            if (ctl.imr >= 1 &&
                check(ctx, pdac_gpu_append_mass_check(ctx, path("pdac.chm").c_str(), sweep, dt), "print_mass_residuals"))
                return 1;
            ++steps;
            const double elapsed =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
            const bool stop_now = elapsed > ctl.max_seconds;
            if (sweep % ndump == 0 || stop_now) {
                if (check(ctx, pdac_gpu_write_restart(ctx, path("pdac.res").c_str(), t, nfil), "tapewr")) return 1;
                if (ctl.isink > 0 &&
                    check(ctx, pdac_gpu_write_mass_loss(ctx, path("massl.res").c_str()), "print_mass_loss"))
                    return 1;
            }
            if (t + 0.1 * dt >= ctl.tstop || stop_now || (max_steps > 0 && steps >= max_steps)) break;
        }
        std::printf("time %.17g nfil %d sweep %d\n", t, nfil, sweep);
        return 0;
    };
    rc = run();
    pdac_gpu_destroy(ctx);
    return rc;
}

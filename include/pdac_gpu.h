/*
 * pdac_gpu.h -- C ABI of the B200 (sm_100a) PDAC time-step engine.
 *
 * The engine replaces the argument-less Fortran module procedures that
 * PDAC's time loop calls (prog.f:162-331 of the reference) with calls on an
 * opaque context that owns one device-resident domain.  Every entry point
 * returns an int status (PDAC_OK = 0, see the codes below); nothing in these
 * signatures is a torch or CUDA type, so a Fortran (ISO_C_BINDING), C, C++
 * or Python ctypes caller binds them directly.
 *
 * Layout of every host array exchanged through this header is the
 * reference's: one flat index ijk = i + nx*(j + ny*k) (0-based, i fastest;
 * j absent in 2D), per-solid arrays (ncell, nsolid) column-major -- i.e.
 * solid class slowest -- and per-gas arrays (ncell, ngas) likewise
 * (press.f:2-28, velocity.f:2-38, dens.f:2-29, temp.f:2-30, eosg.f:11-17).
 * All cells, including the one-cell boundary frame, are stored.
 */
#ifndef PDAC_GPU_H
#define PDAC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (comm/error.F:1-59 aborts; here they are returned) --- */
#define PDAC_OK                 0
#define PDAC_ERR_CONFIG         1   /* unsupported or inconsistent cfg        */
#define PDAC_ERR_CUDA           2   /* CUDA runtime error                     */
#define PDAC_ERR_MAXOUT         3   /* iter.f:428-450: maxout sweeps reached
                                       with cfg cstop set                    */
#define PDAC_ERR_EOS            4   /* ftem.f:191-193: caloric EOS failures   */
#define PDAC_ERR_NONFINITE      5   /* NaN or Inf in an uploaded field or in
                                       the state after a step                */
#define PDAC_ERR_ARG            6   /* bad argument (NULL, size, name)        */
#define PDAC_ERR_BOUNDARY       7   /* inoutflow.f:99,143: rls >= 1 on a BC   */
#define PDAC_ERR_TIMEOUT        8   /* reserved: no kernel of this build waits
                                       on a flag, so none can time out       */

/* ---- cell flags, grid.f:45-58 ----------------------------------------- */
#define PDAC_FLUID        1
#define PDAC_SLIP_WALL    2
#define PDAC_NOSLIP_WALL  4
#define PDAC_FREE_IO      8
#define PDAC_INLET_CELL   16
#define PDAC_ZERO_GRAD    32
#define PDAC_VENT_CELL    64

#define PDAC_MAX_NSOLID   8
#define PDAC_MAX_NGAS     7

/* precision modes.  PDAC_PREC_MIXED (2D and 3D runs, both time
 * integrations): the face-flux passes -- momentum (flux_u/v/w.f), mass (flux_m.f),
 * species and enthalpy (flux_sc.f, hotc.f) -- compute in FP32 from the FP64
 * state and store their fluxes in FP64; the state, every conservative update,
 * the pressure correction and the equations of state stay in FP64.  A face
 * flux is shared by its two cells in both modes, so the phase masses are
 * conserved to FP64 round-off. */
#define PDAC_PREC_FP64    0   /* every kernel in FP64                         */
#define PDAC_PREC_MIXED   1   /* FP32 face-flux passes, FP64 everything else  */

/*
 * Run configuration: the subset of the reference namelists (input.f:159-209,
 * defaults input.f:219-468, derived values check_input input.f:912-1013)
 * that the per-step path reads, plus the mesh metric and cell flags.  The
 * pointer members are read during pdac_gpu_create only.
 */
typedef struct pdac_cfg {
    int    job_type;            /* 2 = 2D (x|r, z), 3 = 3D (x, y, z)         */
    int    nx, ny, nz;          /* cells including the boundary frame        */
    int    itc;                 /* 1 = cylindrical (2D only)                 */
    int    nsolid, ngas;
    int    gas_type[PDAC_MAX_NGAS]; /* 1..7: O2 N2 CO2 H2 H2O Air SO2 (setup.f:563-571) */

    /* &numeric */
    double dt;
    int    rungekut;
    int    time_integration;    /* 0 = semi-implicit (tilde/iter/htilde/ftem),
                                   1 = explicit SSP-RK3 (explicit_solver.f)  */
    double alpha, alphagrav;
    double omega, delg;
    int    inmax, maxout;
    int    cstop;               /* &control cstop (input.f:239): 1 = a call of
                                   iter that ends without convergence after
                                   maxout sweeps returns PDAC_ERR_MAXOUT, as
                                   the reference stops the run there
                                   (iter.f:449); 0 (the default) = it returns
                                   PDAC_OK with *nit = maxout + 1, and
                                   pdac_gpu_unconverged_cells lists the cells
                                   the reference reports (iter.f:428-447)    */
    int    muscl, lv, lm;       /* limiter types (limiters.f:14-56)          */
    double beta;                /* beta-limiter parameter                    */
    double flim;                /* invdm decoupling threshold (ftem.f:221)   */
    int    update_eosg;
    int    implicit_fluxes;     /* 1: tilde at the start of every outer sweep
                                   of iter (iter.f:211-226), none before it */
    int    implicit_enthalpy;   /* 1: ftem (after htilde when implicit_fluxes)
                                   at the end of every outer sweep
                                   (iter.f:362-379), htilde before iter
                                   otherwise (prog.f:246-292)               */
    int    optimization;        /* inner loop of the corrector: 1 inner_loop
                                   (iter.f:480-580), 2 opt_inner_loop
                                   (iter.f:1255-1547), whose density
                                   stencils keep the loop-entry value of the
                                   cell where a neighbour slot is the cell
                                   itself; 3 is 2 outside 3D with two
                                   classes (iter.f:160-161)                 */

    /* &model */
    int    pmodel, drag_model, icpc;
    double tref;
    int    gas_viscosity, part_viscosity, repulsive_model;
    int    iturb;               /* 0 none, 1 Smagorinsky sub-grid model, 2
                                   the same with ground roughness (zrough,
                                   topo_c below)                             */
    int    modturbo;            /* 1 static Smagorinsky, 2 dynamic (Germano,
                                   turbo.f:180-349; 2D falls back to 1)      */
    int    iss;                 /* 1 particle sub-grid stress (turbo.f:437)  */
    double cmut;                /* Smagorinsky constant                      */
    double gravx, gravy, gravz;

    /* &particles */
    double dk[PDAC_MAX_NSOLID];     /* diameter [m]                          */
    double rl[PDAC_MAX_NSOLID];     /* density [kg/m3]                       */
    double phis[PDAC_MAX_NSOLID];   /* sphericity                            */
    double cmus[PDAC_MAX_NSOLID];   /* particle viscosity [Pa s]             */
    double cps[PDAC_MAX_NSOLID];    /* specific heat                         */
    double kap[PDAC_MAX_NSOLID];    /* thermal conductivity                  */
    double plim[PDAC_MAX_NSOLID];   /* twophase_limit (matrix.f:355)         */

    /* &atmosphere: inflow state for free in/out boundaries */
    double void_fraction;
    double atm_ygc[PDAC_MAX_NGAS];  /* indexed by reference gas type - 1     */

    /* &inlet: vent velocity fluctuations (vent.f:902-936) */
    int    irand;

    /* &model isink, rprox, rdist and &mesh center_x, center_y: the particle
     * sink at the ground (sink.f:46-121): with isink > 0 every fluid cell
     * above a wall takes out the downward particle flux of its cell centre
     * when rprox < distance from (center_x, center_y) < rdist, and the mass
     * taken out accumulates per ground column (massl)                      */
    int    isink;
    double rprox, rdist;
    double center_x, center_y;

    /* &model compute_mixture: the gas-particle mixture fields (mixture.f,
     * derived.f:220-331) at the end of every step (prog.f:331) and in the
     * output files; &control formatted_output: output files as text
     * (outp.f:226-231, io_parallel.f:38-50) instead of unformatted records */
    int    compute_mixture;
    int    formatted_output;

    int    precision;               /* PDAC_PREC_FP64 / PDAC_PREC_MIXED      */

    /* mesh metric and flags (read at create) */
    const double *dx, *dy, *dz;     /* nx, ny, nz cell sizes                 */
    const int    *flag;             /* ncell flags                           */
    const double *p_atm, *t_atm;    /* nz hydrostatic profile (atmosphere.f:160-230) */
    int           nvent;            /* number of vent cells                  */
    const int    *vent_ijk;         /* nvent flat indices of vent cells      */

    /* immersed boundaries over topography (&boundaries immb = 1 with
     * &topography itp = 1; immb.f, interp.f:321-919, ghost.f:2888-3345).
     * Built on the host from the topography (the reference's set_forcing,
     * local_forcing, fill_cells and face_fractions); the arrays are read at
     * create.  immb = 0 leaves every pointer unused (NULL allowed).         */
    int           immb;
    const int    *ib_faces;         /* ncell: the cell's face factors b_e_ ..
                                       b_s_ as bits (1 E, 2 W, 4 T, 8 B,
                                       16 N, 32 S; set = 1)                   */
    const double *ib_ivf;           /* ncell: ivf_, 1 / fluid volume fraction */
    const int    *ib_num[3];        /* ncell each (x, y, z): numx/numy/numz,
                                       the cell's 1-based forcing point, 0 none */
    int           ib_nfp[3];        /* forcing points per axis                */
    const int    *ib_fp[3];         /* nfp x 6 per axis: i, j, k (1-based),
                                       interpolation type, and the flat 0-based
                                       indices of the first and second 3D
                                       interpolation neighbours (index_q,
                                       index_qq; -1 where not used)          */
    const double *ib_nsl[3];        /* nfp x 3 per axis: the no-slip point    */
    const double *x, *xb, *y, *yb, *z, *zb; /* cell-centre and face coordinates
                                       (nx, nx, ny, ny, nz, nz), as the
                                       topography translated them            */

    /* ground roughness of the sub-grid model (iturb = 2; turbo.f:72-101,
     * roughness.f:12-36): the &topography namelist's zrough (m) and the
     * level of the ground under each column, topo_c(i) / topo2d_c(i, j) as
     * set-up leaves them (export_topography, topo.f:1114-1160, overwritten by
     * the immersed boundaries' interpolation, immb.f:117-119, 227-230): nx
     * values in 2D, nx * ny in 3D (i fastest).  Read at create; topo_c may
     * be NULL unless iturb = 2.                                              */
    double        zrough;
    const double *topo_c;
} pdac_cfg;

/*
 * Prognostic state, host pointers in the reference layout.  Members may be
 * NULL in a download call to skip that field; upload requires all fields
 * except the 3D-only ones in 2D (vg, vs).
 */
typedef struct pdac_state_view {
    double *p, *ep, *rog, *rgp, *tg, *sieg, *cg;   /* ncell                  */
    double *ug, *vg, *wg;                          /* ncell (face E, N, T)   */
    double *rlk, *ts, *sies;                       /* ncell * nsolid         */
    double *us, *vs, *ws;                          /* ncell * nsolid         */
    double *ygc, *xgc;                             /* ncell * ngas           */
} pdac_state_view;

typedef struct pdac_ctx pdac_ctx;

/* ---- lifecycle -------------------------------------------------------- */
/* replaces the allocate_* calls of pdac.f:126-131,249-261 */
int pdac_gpu_create(const pdac_cfg *cfg, pdac_ctx **out);
int pdac_gpu_destroy(pdac_ctx *ctx);
/* human-readable text of the last error on this context */
const char *pdac_gpu_last_error(const pdac_ctx *ctx);

/* ---- state transfer ---------------------------------------------------- */
int pdac_gpu_upload_state(pdac_ctx *ctx, const pdac_state_view *s);
int pdac_gpu_download_state(pdac_ctx *ctx, pdac_state_view *s);
/* pdac_gpu_download_state into out followed by pdac_gpu_upload_state from
 * in, as one call whose two copy directions overlap: field by field, each
 * field's upload starts once that field's download is done, so out and in
 * may be the same view (a host that keeps the module arrays of
 * press.f/velocity.f/dens.f/temp.f in step with the device hands back what
 * it read, or what it changed field by field), and the download of the next
 * field runs beside it.  Fields of out may be NULL (not read back); in
 * needs the fields pdac_gpu_upload_state needs.  Returns with both
 * directions complete and the uploaded fields checked (PDAC_ERR_NONFINITE
 * as for an upload).  No counterpart in the reference, whose host arrays
 * are the state; it is the hand-off of those arrays between two time
 * steps (prog.f:162-331) when the host keeps its own copy.                */
int pdac_gpu_exchange_state(pdac_ctx *ctx, pdac_state_view *out, const pdac_state_view *in);

/* ---- per-call mirrors of the time loop (prog.f:143-417) --------------- */
/* boundary (bdry.f:22-726) at time-step number 'sweep' (1-based)          */
int pdac_gpu_boundary(pdac_ctx *ctx, int sweep);
/* fieldn (tilde.f:125-274) incl. viscon (visc.f:37-148)                   */
int pdac_gpu_fieldn(pdac_ctx *ctx);
/* tilde (tilde.f:276-848): fluxes, stresses, drag, interphase matrix      */
int pdac_gpu_tilde(pdac_ctx *ctx, double dt);
/* iter (iter.f:38-477); *nit receives the number of outer sweeps, which is
 * maxout + 1 when the sweeps did not converge (the reference's DO-loop
 * count); then the call returns PDAC_ERR_MAXOUT if cfg cstop is set, else
 * PDAC_OK                                                                 */
int pdac_gpu_iter(pdac_ctx *ctx, double dt, int *nit);
/* the cells of the last outer sweep of the last pdac_gpu_iter that were not
 * converged (|dg| > conv at their residual test, so they ran the inner
 * loop): the report the reference writes to pdac.tst when iter ends at
 * maxout (iter.f:428-447).  Flat 0-based indices in increasing order;
 * *n_inout holds the capacity of ijk on entry and the count on return
 * (PDAC_ERR_ARG with the count when ijk is NULL or too small).  Empty after
 * a converged iter, whose last sweep had no such cell.                    */
int pdac_gpu_unconverged_cells(pdac_ctx *ctx, int *ijk, long *n_inout);
/* Variant of pdac_gpu_iter with no counterpart in the reference: the same
 * computation and results, but the corrector's scratch (per-colour
 * counters, worklist, active-set flags) lives in one fixed static device
 * array of PDAC_ITER_STATIC_SCRATCH_BYTES instead of the context's buffers,
 * and the call makes no device allocation.  It serves hosts that fix
 * their device footprint themselves -- e.g. a driver that reserves all
 * device memory for its own pool at start-up and must not see later
 * allocations, or whose memory accounting admits only the buffers it
 * created.  Limits and rules:
 *  - the mesh must fit: 256 + 2 * (4 * ceil(nx / 3) * ny * nz rounded
 *    up to 256) + 4 * ceil(nx * ny * nz / 32) bytes
 *    <= PDAC_ITER_STATIC_SCRATCH_BYTES, else the
 *    call returns PDAC_ERR_ARG with the sizes in pdac_gpu_last_error;
 *  - the context's device must be current; the first call on a device looks
 *    up the array's address once (cudaGetSymbolAddress), so make that first
 *    call before any stream capture on the device;
 *  - nothing in the array needs to start at zero: the call clears the
 *    counters on the context's stream before every sweep and sets the
 *    active-set bits before the first one;
 *  - one array per device is shared by every context on it, so calls that
 *    overlap in time on one device (other threads or streams) race and are
 *    not allowed;
 *  - the array is part of the library's device image: every device that
 *    loads the library holds its 8 MiB until the process exits, whether or
 *    not the entry point is called;
 *  - it reports the same sweep count and status as pdac_gpu_iter (also
 *    PDAC_ERR_MAXOUT under cfg cstop) and times itself for
 *    pdac_gpu_phase_times, but it keeps no list for
 *    pdac_gpu_unconverged_cells.                                           */
#define PDAC_ITER_STATIC_SCRATCH_BYTES (8 * 1024 * 1024)
int pdac_gpu_iter_static(pdac_ctx *ctx, double dt, int *nit);
/* sub-grid turbulence model (cfg iturb = 1, iss = 1), called after fieldn
 * or initialize_fieldn as prog.f:207-208 does: sgsg (turbo.f:145-349) sets
 * the turbulent viscosity and conductivity from the strain rate, sgss
 * (turbo.f:437-475) the particle sub-grid viscosity; no-ops without them  */
int pdac_gpu_sgsg(pdac_ctx *ctx);
int pdac_gpu_sgss(pdac_ctx *ctx);
/* ygas (ygas.f:27-156)                                                    */
int pdac_gpu_ygas(pdac_ctx *ctx, double dt);
/* htilde (htilde.f:25-178)                                                */
int pdac_gpu_htilde(pdac_ctx *ctx, double dt);
/* ftem (ftem.f:19-199)                                                    */
int pdac_gpu_ftem(pdac_ctx *ctx, double dt);
/* explicit SSP-RK3 solver, contexts created with time_integration = 1:
 * initialize_fieldn (explicit_solver.f:419-564) in place of fieldn, and
 * explicit_iter (explicit_solver.f:996-1223) in place of tilde / iter /
 * htilde / ftem; explicit_iter returns PDAC_ERR_EOS where the reference
 * stops on more than one caloric failure (explicit_solver.f:1214-1215).
 * Both return PDAC_ERR_CONFIG on a time_integration = 0 context.           */
int pdac_gpu_initialize_fieldn(pdac_ctx *ctx);
int pdac_gpu_explicit_iter(pdac_ctx *ctx, double dt);
/* one whole time step: boundary, fieldn, RK loop of tilde/iter/ygas/htilde/ftem
 * (time_integration = 0), or boundary, initialize_fieldn, RK loop of
 * explicit_iter/ygas (time_integration = 1, *nit = 0)                      */
int pdac_gpu_step(pdac_ctx *ctx, int sweep, int *nit);

/* ---- files of the time loop, in the reference's formats -------------- */
/* tapewr (io_restart.f:31-124): the restart file (pdac.res) as Fortran
 * unformatted sequential records, 4-byte little-endian length markers:
 * (time, nx, ny, nz, nsolid, ngas, nfil), gas_type(ngas), then one REAL*8
 * record of ncell values each for p, ug, [vg], wg, sieg, rlk per class, per
 * class us, [vs], ws, sies per class, ygc per gas, rgp, rog, tg, ts per
 * class ([] = 3D only).                                                    */
int pdac_gpu_write_restart(pdac_ctx *ctx, const char *path, double time, int nfil);
/* taperd (io_restart.f:126-339) + the restart branch of cnvert
 * (setup.f:359-391): reads such a file into the context (the file's gas
 * types replace the run's, as in the reference), derives xgc, ep and cg,
 * and returns its time and output counter; PDAC_ERR_ARG with the reason in
 * pdac_gpu_last_error on a missing file, bad framing or a dimension that
 * differs from the context's.                                              */
int pdac_gpu_read_restart(pdac_ctx *ctx, const char *path, double *time, int *nfil);
/* outp (outp.f:194-384): p, ug, [vg], wg, tg, xgc per gas, and per class
 * rlk / rl, us, [vs], ws, ts, then with compute_mixture rhom, um, [vm], wm,
 * tm and yd per gas and class.  Unformatted (the default): REAL(time, 4)
 * and one REAL*4 record per field.  With cfg formatted_output: text, a
 * time header and per field its name and the values of each k plane,
 * FORMAT(1x,10(1x,G14.6E3)) (io_parallel.f:38-50).  The caller names the
 * file output.NNNN (lettera, letter.f).                                    */
int pdac_gpu_write_output(pdac_ctx *ctx, const char *path, double time);
/* compute_mixture_fields (mixture.f:32-52, prog.f:331): mixture density,
 * velocity, temperature and mass fractions of every cell (cfg
 * compute_mixture = 1; readable as rhom, um, vm, wm, tm, yd through
 * pdac_gpu_get_array)                                                     */
int pdac_gpu_compute_mixture_fields(pdac_ctx *ctx);
/* print_mass_residuals (residuals.f:15-136): out = [res_g, res_s(nsolid),
 * res_gc(ngas), mfr], masses in the fluid cells minus the mass that entered
 * through inlet and vent cells in nswp steps of dt, and the vent mass flow
 * rate (compute_mass_flow_rate, residuals.f:171-251); nout >= 2 + nsolid +
 * ngas                                                                     */
int pdac_gpu_mass_residuals(pdac_ctx *ctx, int nswp, double dt, double *out, int nout);
/* the same values appended to path as one pdac.chm line,
 * FORMAT(I8,15(G30.20E3)) (residuals.f:123-127)                           */
int pdac_gpu_append_mass_check(pdac_ctx *ctx, const char *path, int nswp, double dt);
/* print_mass_loss (sink.f:123-167, called at prog.f:355 before outp as
 * massl.NNNN and at prog.f:386 after tapewr as massl.res): the mass each
 * ground column has lost to the sink, formatted as the reference writes it;
 * read_mass_loss (sink.f:168-207, setup.f:147): such a file's values, added
 * back at each column's next sink update.  Both need isink > 0.           */
int pdac_gpu_write_mass_loss(pdac_ctx *ctx, const char *path);
int pdac_gpu_read_mass_loss(pdac_ctx *ctx, const char *path);

/* vent fluctuation factors for the next boundary call, one per vent cell in
 * cfg->vent_ijk order (vent.f:824-873 random_switch draws them in 3D).     */
int pdac_gpu_set_vent_factors(pdac_ctx *ctx, const double *fact, int nvent);

/* ---- diagnostics ------------------------------------------------------- */
/* Copy one named device array (state or intermediate, e.g. "rug", "appu",
 * "rgfe") into host memory; *n_inout holds the capacity in doubles on entry
 * and the element count on return.  Test and debugging aid.               */
int pdac_gpu_get_array(pdac_ctx *ctx, const char *name, double *out, long *n_inout);
/* Mass totals over fluid cells (residuals.f:14-130): out[0] = gas mass,
 * out[1..nsolid] = per-class solid mass, out[1+nsolid ..] = per-gas mass.  */
int pdac_gpu_mass_totals(pdac_ctx *ctx, double *out, int nout);
/* device time (ms) of the kernels of the last call, by phase:
 * [boundary, fieldn, tilde, iter, ygas, htilde, ftem]                    */
int pdac_gpu_phase_times(pdac_ctx *ctx, double *ms7);
/* statistics since the last reset: out[0] kernel launches, out[1] outer
 * sweeps of iter, out[2] timed colour phases of the corrector, out[3] their
 * device time in ms; with nout >= 7 also out[4] / out[5] the device time of
 * the residual-test and inner-loop kernels of those phases and out[6] the
 * number of unconverged cells they processed, with nout >= 8 also out[7]
 * the number of cells the residual tests evaluated (all counted only when
 * the reset enabled profiling); with nout >= 13 also the device ms of the
 * explicit solver's kernel groups over the profiled explicit_iter calls,
 * out[8] flux passes, out[9] stage kernels, out[10] gas-enthalpy
 * wavefronts, out[11] final solve, and out[12] the number of those calls;
 * nout >= 4                                                               */
int pdac_gpu_stats(pdac_ctx *ctx, double *out, int nout);
int pdac_gpu_reset_stats(pdac_ctx *ctx, int profile_corrector);
/* per colour phase of the corrector since the last profiling reset, six
 * doubles each: sweep, colour, worklist length, cells tested, device ms of
 * the residual test and of the inner loop; *n_inout holds the capacity in
 * doubles on entry and the count on return                                */
int pdac_gpu_sweep_log(pdac_ctx *ctx, double *out, long *n_inout);
/* stream-ordered timing marks (slots 0..31) and the device time between two */
int pdac_gpu_mark(pdac_ctx *ctx, int slot);
int pdac_gpu_elapsed(pdac_ctx *ctx, int a, int b, double *ms);

/* ---- launch-shape autotuner (no counterpart in the reference) ---------- */
/* The launch shapes of the engine's tunable kernels, as five ints:
 *   [0] form of the 3D momentum-flux pass: 0 = one thread per (cell,
 *       phase) and component (three launches), 1..4 = the shared-memory
 *       tiled pass with 32 x 4, 32 x 8, 16 x 8 or 64 x 2 cells (i x j) per
 *       block;
 *   [1] planes of a tiled block's march up k;
 *   [2] blocks of the corrector's inner-loop kernel;
 *   [3] blocks of its residual-test kernel;
 *   [4] cells per block of the one-launch sweep loop of small domains.
 * None of them changes a result: only the speed.
 * pdac_gpu_autotune times candidates on the context's current state and
 * installs the fastest: the momentum-flux pass directly (it rewrites the
 * same face fluxes), the corrector's shapes as whole time steps on a device
 * copy of the state that is restored afterwards (skipped if the copy does
 * not fit in device memory; contexts with time_integration = 1 tune the
 * flux pass only).  The state, statistics and sweep count the caller sees
 * are unchanged.  Call it after a step or two, when the state is typical of
 * the run.  With cache_path (may be NULL) the result is looked up first and
 * appended after tuning, one text line per key (device name, grid, nsolid,
 * ngas, precision, time integration, implicit modes); a cached entry is
 * installed without timing.  out (may be NULL) receives the five values.
 * pdac_gpu_set_tuning installs five given values (PDAC_ERR_ARG if out of
 * range).                                                                  */
int pdac_gpu_autotune(pdac_ctx *ctx, const char *cache_path, int *out, int nout);
int pdac_gpu_set_tuning(pdac_ctx *ctx, const int *in, int nin);

/* ---- ensembles of independent runs ------------------------------------ */
/* No counterpart in the reference, which runs one domain per job (an
 * ensemble there is many jobs).  A batch advances many contexts (members:
 * any mix of grids, decks and time integrations, all on the current device)
 * by one time step each, pdac_gpu_step(member, sweep, ...) on every member,
 * with the members' kernels running concurrently on the device.  A member on
 * the semi-implicit path (time_integration = 0, rungekut = 1, no implicit-
 * flux modes, cstop unset, more than one gas) takes its whole step as
 * graph nodes -- boundary to ftem, the outer sweep loop as a conditional
 * node, its outcome copied back once -- and all such members' nodes form
 * ONE CUDA graph (independent branches), launched once per batch step by
 * the calling thread (rebuilt after a member's launch shapes change; one
 * graph per member if that graph cannot be instantiated); the other
 * members are driven by a pool of nthreads host
 * threads (<= 0: one per such member).  Both give the member's results of
 * pdac_gpu_step, bit for bit; pdac_gpu_phase_times is not updated by a
 * graph step.  While in a batch, members run without cooperative launches
 * (the small-domain sweep loop and the explicit solver's wavefront take
 * their multi-launch forms, with the same results), so that no two
 * cooperative grids share the device.  The batch does not own the members: create, upload and download
 * them with the per-context calls, never while a batch step runs, and
 * destroy the batch before them.  A member appears once.
 * pdac_gpu_batch_step fills nit[m] and status[m] (either may be NULL) for
 * every member, steps every member whatever the others return, and returns
 * the first non-zero member status (its message in
 * pdac_gpu_batch_last_error).  pdac_gpu_batch_elapsed gives the device time
 * of the last batch step in ms, from its start on every member's stream to
 * the end of the last member.                                            */
typedef struct pdac_batch pdac_batch;
int pdac_gpu_batch_create(pdac_ctx *const *members, int nmember, int nthreads, pdac_batch **out);
int pdac_gpu_batch_step(pdac_batch *b, int sweep, int *nit, int *status);
int pdac_gpu_batch_elapsed(pdac_batch *b, double *ms);
const char *pdac_gpu_batch_last_error(const pdac_batch *b);
int pdac_gpu_batch_destroy(pdac_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* PDAC_GPU_H */

/*
 * chanrhs.h -- C ABI of the B200 time-step library for the compressible
 * channel solver theparvezahmad/compChan3Dmpi.
 *
 * The library replaces the reference's per-stage and per-step subroutines.
 * The reference calls them from its main program, v1.10/codes/main_v1.10.f90:20-53
 * (module bodies in v1.10/codes/module_comp.f90).  The monolithic form is
 * v1.9/codes/main_v1.9.f90:304-1049.
 * All entry points use plain pointers, sizes and C scalars, so a Fortran host
 * can bind them with iso_c_binding through a bind(c) interface module.
 *
 * Axes and arrays follow the reference exactly.
 *   index 1 (i, nP[0]) : streamwise x, periodic.
 *   index 2 (j, nP[1]) : spanwise, periodic.
 *   index 3 (k, nP[2]) : wall-normal, stretched, isothermal no-slip walls at k=1 and k=nP3.
 * Periodic directions store both duplicate end points, as in
 * v1.9/codes/comdata.f90:85-86, so there are nP-2 unique points.
 * `var` is the reference array var(1:nP1,1:nP2,1:nP3,1:7) (v1.9/codes/main_v1.9.f90:38).
 * It is column-major (i fastest) and holds rho,u,v,w,E,T,p.
 *
 * Ownership: the caller owns every host array.  The library owns all device
 * memory, copies host data only inside chan_upload / chan_download /
 * chan_stats, and never keeps a host pointer.
 * Threading: one context per CUDA stream; a context is not thread-safe.
 * Return codes: 0 OK; negative = usage/IO/CUDA error; positive = numerical status.
 */
#ifndef CHANRHS_H
#define CHANRHS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHAN_OK 0
#define CHAN_BLOWUP 1      /* rho<0 or T<0 after a step (v1.9/codes/main_v1.9.f90:709-743) */
#define CHAN_NONFINITE 2   /* NaN or Inf met in the updated state */
#define CHAN_EINVAL (-1)   /* bad argument */
#define CHAN_ENOMEM (-2)   /* device allocation failed */
#define CHAN_ECUDA (-3)    /* CUDA runtime error (see chan_last_error) */
#define CHAN_ESTATE (-4)   /* call out of order (e.g. step before upload) */
#define CHAN_EIO (-5)      /* file error (see chan_last_error / chan_io_last_error) */

#define CHAN_RK2 2         /* the reference's midpoint RK2: maxiter=2, v1.9/codes/comdata.f90:8 */
#define CHAN_RK3 3         /* SSP-RK3 (Shu-Osher); no reference counterpart */

#define CHAN_FORCE_WALLSHEAR 0  /* reference forcing 0.5*(tauL-tauU)*rhobar(k), lagged (main_v1.9.f90:547-553) */
#define CHAN_FORCE_NONE 1       /* no source term */

/* chan_params.flags: mixed precision.  The intermediate RK stage states are
 * stored in float and the inviscid and viscous fluxes are evaluated in float;
 * the step state, the RK accumulation against it, the temperature/pressure
 * recovery from the total energy, the forcing, the wall BC and every
 * reduction stay in double.  Such a context runs whole steps only
 * (chan_stage returns CHAN_ESTATE).  The reference has no counterpart; its
 * error against the FP64 path is measured, not bounded to 1e-12. */
#define CHAN_MIXED 1

/* Run-time parameters.  Field-for-field equivalent of the reference's
 * compile-time constants and param.dat deck (v1.9/codes/comdata.f90:4-68). */
typedef struct chan_params {
    int32_t nP[3];      /* nP(1..3) grid points including walls and periodic duplicates */
    int32_t istat;      /* cadence of wall-shear/plane statistics (param.dat field) */
    int32_t rk_scheme;  /* CHAN_RK2 (reference) or CHAN_RK3 */
    int32_t forcing;    /* CHAN_FORCE_WALLSHEAR (reference) or CHAN_FORCE_NONE */
    int32_t device;     /* CUDA device ordinal */
    int32_t flags;      /* 0 (plain FP64) or CHAN_MIXED */
    double Re;          /* Reynolds number (param.dat) */
    double Mac;         /* Mach number (param.dat) */
    double dt;          /* time step (param.dat) */
    double Pr;          /* Prandtl number; the reference hardcodes 0.71 (comdata.f90:12) */
    double gama;        /* ratio of specific heats, 1.4 (comdata.f90:11) */
    double Pe[3];       /* PexVal, PeyVal, PezVal: QUICK/central switch thresholds */
    double Lx, Ly;      /* periodic lengths x1(nP1), x2(nP2): 4*pi and 4*pi/3 (comdata.f90:81-82) */
    double Tw[2];       /* wall temperature at k=1 and k=nP3; 1.0 in the reference (main_v1.9.f90:628) */
} chan_params;

typedef struct chan_ctx chan_ctx;

/* Replaces readParam + setupMesh + the wall-coefficient block
 * (v1.9/codes/comdata.f90:31-110, v1.9/codes/main_v1.9.f90:52-76;
 *  v1.10: readParam, calcMeshParam, calcCoeffs, main_v1.10.f90:20-22).
 * x3, jac and invJac are the wall-normal mesh arrays x3(1:nP3), jac(1:nP3)
 * and invJac(1:nP3).  The wall-normal computational coordinate is uniform on [0,2]. */
int chan_init(const chan_params *p, const double *x3, const double *jac,
              const double *invJac, chan_ctx **out);

/* Replaces readInputFile + initSolV + share2P(solV) + share2P(var)
 * (v1.9/codes/main_v1.9.f90:210-301; main_v1.10.f90:25-29).
 * var = var(1:nP1,1:nP2,1:nP3,1:7) read from the restart deck.
 * The lagged forcing restarts at zero, as in the reference. */
int chan_upload(chan_ctx *c, const double *var, int64_t nstep, double time);

/* One Runge-Kutta stage.  Replaces calcFlux, calcSolV, share2P(solV),
 * calcPrim, share2P(var) and calcBC (v1.9/codes/main_v1.9.f90:313-704;
 * main_v1.10.f90:38-46).  iter is 1..2 for RK2 and 1..3 for RK3.  It does not
 * advance nstep or time. */
int chan_stage(chan_ctx *c, int iter);

/* nsteps full time steps.  Each step increments nstep, adds dt to time, runs
 * every stage, then the per-step tail in the reference's order: checkSoln,
 * then calcTauWall and avgSpatial when mod(nstep,istat)==0
 * (main_v1.9.f90:304-311, 709-1049; main_v1.10.f90:31-61).
 * It stops after the step that blew up and returns CHAN_BLOWUP. */
int chan_step(chan_ctx *c, int nsteps);

/* Queue nsteps steps on the context's stream and return without waiting.
 * Poll the result with chan_status.  The reference has no counterpart. */
int chan_step_async(chan_ctx *c, int nsteps);

/* checkSoln: rho<0 or T<0 anywhere (main_v1.9.f90:709-743; module_comp.f90:396). */
int chan_check(chan_ctx *c);

/* calcTauWall without its cadence test (main_v1.9.f90:910-967). */
int chan_tau_wall(chan_ctx *c);

/* avgSpatial without its cadence test (main_v1.9.f90:972-1002). */
int chan_avg_spatial(chan_ctx *c);

/* Copy out the forcing and statistics state.  Any pointer may be NULL.
 * tau2[2]   = tauxzL, tauxzU.
 * stat1[7*nP3], stat2[7*nP3] = stat1Spc(k,p), stat2Spc(k,p) stored as [p][k].
 * corr[9*nP3] = corrSpc(k,c) stored as [c][k].
 * Source: main_v1.9.f90:39-41, 1027-1037. */
int chan_stats(chan_ctx *c, double *tau2, double *stat1, double *stat2, double *corr);

/* Overwrite the lagged forcing state tauxzL, tauxzU and stat1Spc(:,1)
 * (main_v1.9.f90:551-553).  rhobar has nP3 entries.  It is needed to
 * restart with a non-zero forcing.  The reference has no counterpart. */
int chan_set_forcing(chan_ctx *c, double tauL, double tauU, const double *rhobar);

/* State back to var(1:nP1,1:nP2,1:nP3,1:7).  Used like writeSoln
 * (main_v1.9.f90:749-794).  Corner duplicates and wall edge pressures hold
 * the same stale values the reference's var holds. */
int chan_download(chan_ctx *c, double *var);

/* Blow-up / non-finite status.  Any pointer may be NULL.  ijk receives the
 * 1-based (i,j,k) of one offending point.  nstep/time are the step counter
 * and time of the last completed step. */
int chan_status(chan_ctx *c, int32_t *ijk, int64_t *nstep, double *time);

/* Block until queued work is done; return the status code as chan_status does. */
int chan_sync(chan_ctx *c);

/* Per-kernel device timing from CUDA events on the context's stream, for
 * measurement tools.  enable=1 starts accumulating.
 * chan_profile_read returns, per kernel class, the summed milliseconds and
 * the launch count.  Classes: 0 stage, 1 wall BC, 2 statistics.  The
 * reference has no counterpart. */
int chan_profile(chan_ctx *c, int enable);
int chan_profile_read(chan_ctx *c, double *ms3, int64_t *count3);

/* Diagnostics: evaluate the library's T^0.7 (the transport law mu = k = T^0.7
 * of main_v1.9.f90:643,720) and the CUDA math library's pow(T,0.7) on device
 * `device` for n host values; results go to host arrays mine and libm.
 * The reference has no counterpart. */
int chan_selftest_pow07(const double *T, double *mine, double *libm, int64_t n, int32_t device);

/* The context's cudaStream_t (as void*), for callers that record events. */
void *chan_stream(chan_ctx *c);

/* Device bytes held by the context. */
int64_t chan_device_bytes(chan_ctx *c);

/* Last error message of this context, or of chan_init when c is NULL. */
const char *chan_last_error(chan_ctx *c);

/* Library version string. */
const char *chan_version(void);

/* Time averaging of the plane statistics, done on the device.  The reference
 * appends every statistics step to moment1st/2nd/Joint.dat and tauWall.dat
 * and time-averages those files offline (v1.9/codes/avg_v1.7.f90:113-274,
 * avgTauWall.f90).  Here every statistics step (mod(nstep,istat)==0 inside
 * chan_step) adds its stat1Spc, stat2Spc, corrSpc and tauL, tauU into device
 * sums once chan_time_avg_start has been called.
 * chan_time_avg_start: zero the sums and start accumulating.
 * chan_time_avg: copy out the sums (layouts as chan_stats), the number of
 * samples and the times of the first and last sample; any pointer may be
 * NULL.  mean = sum/n; rms = sqrt(sum2/n - mean^2); covariances follow
 * avg_v1.7.f90:264-274. */
int chan_time_avg_start(chan_ctx *c);
int chan_time_avg(chan_ctx *c, double *sum1, double *sum2, double *sumc, double *sumtau, int64_t *nsamples,
                  double *t0, double *t1);

/* Wall boundary-condition plug-in.  It covers the reference's wall-BC
 * variants, which differ only in the wall block of the stage
 * (v1.9/codes/main_v1.9.f90:623-641):
 *   isothermal T_w        v1.9_strat/v1.9_st1,st2 (T_w = 0.2, 1.8)
 *   fixed dT/dz           v1.9_strat/v1.9_st3,st4: c0*T1 + c1*T2 + c2*T3 = dTdz
 *   slip mask             v1.9_groov, v1.9_groov_strat variants: where mask != 0,
 *                         c0*u1 + c1*u2 + c2*u3 = slip_grad (same for v), else u = v = 0
 *   prescribed (u,v)      v1.9_RD variants, rotating discs (field built by the caller)
 *   travelling wave       v1.9_STWNV variants: v_w = A*sin(k*x1(i) + omega*time + phase*(j odd))
 * c0..c2 are the one-sided coefficients of that wall (f1d2 bottom, b1d2 top),
 * w_w = 0 always, and the pressure BC includes the wall velocity terms.
 * The default of both walls is no-slip and isothermal at chan_params.Tw.
 * mask, uv and x1 are copied; x1 (nP1 values) may be NULL to use
 * x1(i) = (i-1)*Lx/(nP1-1) accumulated as comdata.f90:93-95.  A travelling
 * wave uses the time of the step being computed. */
#define CHAN_WALL_NOSLIP 0
#define CHAN_WALL_SLIP_MASK 1
#define CHAN_WALL_UV_FIELD 2
#define CHAN_WALL_WAVE 3
#define CHAN_WALL_ISOTHERMAL 0
#define CHAN_WALL_FIXED_GRADIENT 1
typedef struct chan_wall_bc {
    int32_t velocity;         /* CHAN_WALL_NOSLIP .. CHAN_WALL_WAVE */
    int32_t thermal;          /* CHAN_WALL_ISOTHERMAL or CHAN_WALL_FIXED_GRADIENT */
    double Tw;                /* isothermal wall temperature */
    double dTdz;              /* fixed one-sided wall-normal temperature gradient */
    double slip_grad;         /* one-sided du/dz = dv/dz on slip points */
    double wave[4];           /* A, k, omega, phase added on odd j (1-based) */
    const uint8_t *mask;      /* nP1*nP2, i fastest: nonzero = slip */
    const double *uv;         /* u_w then v_w, each nP1*nP2, i fastest */
    const double *x1;         /* nP1 streamwise coordinates for the wave, or NULL */
} chan_wall_bc;
int chan_set_wall_bc(chan_ctx *c, int32_t wall, const chan_wall_bc *bc);

/* Stage-kernel launch shape (no reference counterpart; it changes no result
 * bits).  tile: CHAN_TILE_32x8 (256 threads, the default), CHAN_TILE_32x4
 * (128 threads), CHAN_TILE_16x16 (256 threads) or CHAN_TILE_32x16 (512
 * threads, one CTA per SM) columns x rows per CTA;
 * nchunks: how many CTAs split the
 * wall-normal march of one tile column (1..nP3-2; 0 picks the count that fills
 * whole waves of resident CTAs, as chan_init does).  chan_get_launch reports
 * the shape in use and the planes per chunk. */
#define CHAN_TILE_32x8 0
#define CHAN_TILE_32x4 1
#define CHAN_TILE_16x16 2
#define CHAN_TILE_32x16 3
#define CHAN_NTILES 4
int chan_set_launch(chan_ctx *c, int32_t tile, int32_t nchunks);
int chan_get_launch(chan_ctx *c, int32_t *tile, int32_t *nchunks, int32_t *kchunk);

/* Buoyancy body force for stratified runs (no reference counterpart: the
 * reference's stratified variants v1.9_strat change only the wall
 * temperature).  Adds, at every interior point,
 *     S(rho*w) = Ri * rho * (T - Tref),   S(rho*E) = ggM * w * S(rho*w)
 * to the right-hand side, w the wall-normal velocity (gravity along -x3) and
 * ggM = gama*(gama-1)*Mac^2 the energy scaling of the forcing term
 * (main_v1.9.f90:565-571).  Ri = 0 (the default) switches it off. */
int chan_set_buoyancy(chan_ctx *c, double Ri, double Tref);

/* Exact binary checkpoint of a context's device state between time steps:
 * the conservative state with its periodic ghosts, both wall planes, the
 * corner columns, the forcing/statistics state and the step counter, time and
 * time-averaging sums.  Restarting from it continues bit for bit.  The
 * reference restarts from its Tecplot deck with the forcing reset to zero
 * (v1.9/codes/main_v1.9.f90:211-282, 749-794); this sidecar has no
 * counterpart there.  chan_checkpoint_read needs a context of the same grid,
 * x3 mesh, physics (Re, Mac, Pr, gama, Pe, Lx, Ly, Tw), dt, RK scheme, forcing
 * and precision; it returns CHAN_EINVAL, naming the first field that
 * differs in chan_last_error, and leaves the context as it was otherwise. */
int chan_checkpoint_write(chan_ctx *c, const char *path);
int chan_checkpoint_read(chan_ctx *c, const char *path);

/* The reference's Tecplot-ASCII deck (3D.dat), read and written on host
 * threads (nthreads <= 0: all hardware threads).  Writer:
 * v1.9/codes/main_v1.9.f90:759-773 (records 3(1X,F10.6),7(1X,E22.15)).
 * Reader: main_v1.9.f90:222-251.  var = var(1:nP1,1:nP2,1:nP3,1:7), and
 * x1(nP1), x2(nP2), x3(nP3) are the coordinate columns (any may be NULL on
 * read).  A short or malformed record returns CHAN_EIO.  chan_io_last_error
 * then names the record as the reference does:
 * "Error in reading combined input file at i j k". */
int chan_deck_read(const char *path, const int32_t *nP, double *var, double *x1, double *x2, double *x3,
                   double *time, int64_t *nstep, int32_t nthreads);
int chan_deck_write(const char *path, const int32_t *nP, const double *var, const double *x1, const double *x2,
                    const double *x3, double time, int64_t nstep, int32_t nthreads);
const char *chan_io_last_error(void);

/* Plane moments stat1Spc, stat2Spc, corrSpc of a host field, computed on GPU
 * `device` without allocating any memory.  This entry point has no
 * counterpart in the reference.
 *
 * Who needs it: Fortran post-processing programs like the reference's
 * avg_v1.7.f90 and fluc.f90 call through iso_c_binding and have no way to
 * call cudaMalloc or to keep a solver context (chan_init allocates the whole
 * solver state).  This call needs neither.  It stages the field through one
 * static device array of CHAN_NOALLOC_MAX_DOUBLES doubles (32 MiB), which
 * every GPU that loads the library holds until the process exits.
 * The results equal chan_avg_spatial + chan_stats on the same field
 * (v1.9/codes/main_v1.9.f90:972-1002 semantics: sums over i=1..nP1,
 * j=1..nP2 divided by nP1*nP2).
 *
 * var    : var(1:nP1,1:nP2,1:nP3,1:7) in host memory.
 * nP     : nP1, nP2, nP3.
 * stat1, stat2 : 7*nP3 doubles each, stored [p][k];  corr : 9*nP3, [c][k].
 * Limit  : 23*nP3 (rounded up to 32) + 7*nP1*nP2 <= CHAN_NOALLOC_MAX_DOUBLES,
 *          i.e. one full wall-normal plane of all seven variables must fit;
 *          larger grids return CHAN_EINVAL with a message (chan_last_error(NULL)).
 * Every call looks up the array's device address in the device's current
 * context (cudaGetSymbolAddress, no allocation); the first call on a device
 * may also load the library's device code there, so make it before any
 * stream capture.  It works on the legacy default stream and synchronizes
 * it.  It restores the calling thread's current device on return.
 * All calls share the one array: calls that overlap on the GPU (concurrent
 * host threads on the same device) race and must be serialized by the caller. */
#define CHAN_NOALLOC_MAX_DOUBLES (4 * 1024 * 1024)
int chan_avg_spatial_noalloc(const double *var, const int32_t *nP, double *stat1, double *stat2, double *corr,
                             int32_t device);

/* Diagnostics series (v1.9/codes/main_v1.9.f90:799-906), computed on the
 * device inside chan_step every `every` steps (the reference: every 10) and
 * kept in a device ring of `capacity` records until chan_diag_read:
 *   KE      = sum over all points of u^2+v^2+w^2 / (nP1*nP2*nP3)    (KE.dat)
 *   rho_b   = bulk density through each x-plane i = planes[m]    (rhobulk.dat)
 *   U_b     = bulk velocity                                         (Ubulk.dat)
 *   rhoU_b  = mass flow                                          (massflow.dat)
 * Bulk values sum, over the cells j=1..nP2-1, k=1..nP3-1 of the plane, the
 * mean of the four corner values times dy*(x3q(k+1)-x3q(k)), then divide by
 * x3q(nP3)*x2end.  A plane outside 3..nP1-2 reports 0, as the reference's
 * single-rank test does.  x3q (nP3 values) and x2end are the coordinates the
 * reference holds when it writes these series: after a restart, the deck's
 * F10.6 columns (x3q NULL: the x3 given to chan_init).  The reference uses
 * planes = {5, 10, 70, 100, 125}.
 * Record layout (3 + 3*nplanes doubles):
 *   [nstep, time, KE, rho_b[nplanes], U_b[nplanes], rhoU_b[nplanes]]
 * chan_diag_enable with every = 0 turns the series off.  chan_diag_read waits
 * for queued work, copies the records in step order (none after a blow-up)
 * and empties the ring; records is NULL to query the count only.  *lost counts
 * the records the ring overwrote. */
#define CHAN_DIAG_MAX_PLANES 8
int chan_diag_enable(chan_ctx *c, const int32_t *planes, int32_t nplanes, int32_t every, const double *x3q,
                     double x2end, int32_t capacity);
int chan_diag_read(chan_ctx *c, double *records, int32_t max_records, int32_t *nrecords, int64_t *lost);

/* Fluctuation field and Q-criterion of the context's current state, on the
 * device.  fluc = var(i,j,k,:) - mean(k,:) as v1.9/codes/fluc.f90:63-69
 * forms it (mean: 7*nP3 doubles stored [p][k], e.g. the time-averaged
 * stat1Spc); qcrit = Q of the fluctuating velocity (u',v',w') as
 * v1.9_strat/v1.9_st1/codes/qInvariant.f90:26-81 computes it:
 * non-uniform central differences on x1, x2, x3, S and R the symmetric and
 * antisymmetric parts of the velocity gradient, Q = (P^2 - sum S^2 + sum R^2)/2
 * with P = -trace; 0 on the box faces.  x1, x2, x3 may be NULL (the
 * context's coordinates: x1, x2 accumulated from Lx, Ly; x3 given to
 * chan_init).  fluc (7*N, var layout) and qcrit (N) may be NULL. */
int chan_fluctuation_q(chan_ctx *c, const double *mean, const double *x1, const double *x2, const double *x3,
                       double *fluc, double *qcrit);

/* The same Q-criterion for host velocity arrays u, v, w (nP1*nP2*nP3 each,
 * i fastest) on GPU `device`, without a context.  It allocates and frees
 * its device buffers.  Errors: chan_last_error(NULL). */
int chan_q_criterion(const int32_t *nP, const double *u, const double *v, const double *w, const double *x1,
                     const double *x2, const double *x3, double *qcrit, int32_t device);

/* Out-of-bounds write detector.  Every state buffer of a context sits
 * between two 512-byte guard zones filled with a NaN bit pattern that no
 * kernel writes; this waits for queued work and counts the guard words that
 * changed (0 when every write stayed inside its buffer).  A substitute for a
 * memory checker in tests; the reference has no counterpart. */
int chan_debug_canaries(chan_ctx *c, int64_t *corrupted);

/* ------------------------------------------------------------------------
 * Learned subgrid closure (no reference counterpart: the reference resolves
 * every scale).  A 13 -> 64 -> 64 -> 9 MLP with GELU activations, BF16
 * weights and activations and F32 accumulation on the tensor cores (tcgen05),
 * F32 master weights trained with Adam on the device.
 *   inputs : du_a/dx_b (a = u, v, w; b = x, spanwise, wall-normal; 9), dT/dx_b
 *            (3) and y+ = rho_w u_tau d Re / mu_w, d the distance to the
 *            nearer wall;
 *   outputs: the Favre subgrid fluxes tau_ab = bar(rho u_a u_b) - bar(rho)
 *            u~_a u~_b (uu, vv, ww, uv, uw, vw) and q_b = bar(rho u_b T) -
 *            bar(rho) u~_b T~ (u, v, w).
 * Both are normalised by a per-column mean and standard deviation
 * (norm[44] = input means[13], input sds[13], output means[9], output sds[9]).
 * Parameters: W1[64][13] b1[64] W2[64][64] b2[64] W3[9][64] b3[9]
 * (chan_closure_nparams() floats). */
typedef struct chan_closure chan_closure;
/* capacity: samples the device dataset holds (13 + 9 floats each) */
int chan_closure_create(int32_t device, int64_t capacity, chan_closure **out);
/* Append samples of a DNS context's current state: the Favre box filter of
 * width fw (even) in x and spanwise, sample points every (sx, sy, sz) grid
 * points away from the walls, gradients by central differences at those
 * strides (the coarse grid the closure runs on). */
int chan_closure_sample(chan_closure *m, chan_ctx *dns, int32_t sx, int32_t sy, int32_t sz, int32_t fw,
                        int64_t *added);
/* append host samples X[n][13], T[n][9] (a saved dataset, or synthetic data) */
int chan_closure_add_data(chan_closure *m, const float *X, const float *T, int64_t n);
int chan_closure_count(chan_closure *m, int64_t *count);
int chan_closure_get_data(chan_closure *m, int64_t first, int64_t n, float *X, float *T);
/* mean / standard deviation of the dataset's columns -> normalisation */
int chan_closure_fit_normalization(chan_closure *m, float *norm_out);
int chan_closure_set_normalization(chan_closure *m, const float *norm);
int chan_closure_get_normalization(chan_closure *m, float *norm);
int chan_closure_nparams(void);
/* Glorot-uniform weights from a seeded generator, zero biases */
int chan_closure_init(chan_closure *m, uint64_t seed);
int chan_closure_set_params(chan_closure *m, const float *params);
int chan_closure_get_params(chan_closure *m, float *params);
/* Adam (beta 0.9 / 0.999, eps 1e-8) on the mean squared error of the
 * normalised outputs, batches of `batch` samples (a multiple of 128) in a
 * seeded order per epoch; losses[epochs] receives each epoch's mean loss. */
int chan_closure_train(chan_closure *m, int32_t epochs, int32_t batch, double lr, uint64_t seed, double *losses);
/* loss sum and parameter gradients (chan_closure_nparams floats) of the mean
 * squared error over one host batch, as one training step computes them */
int chan_closure_grad(chan_closure *m, const float *X, const float *T, int64_t n, float *grads, double *loss_sum);
/* outputs in physical units for host inputs */
int chan_closure_infer(chan_closure *m, const float *X, int64_t n, float *Y);
const char *chan_closure_last_error(chan_closure *m);
/* Frees the closure; contexts running with it must switch it off first
 * (chan_set_closure(c, NULL, 0)).  NULL is allowed. */
void chan_closure_free(chan_closure *m);

/* Run a context with the closure (on = 1 or 2) or without it (on = 0).
 * The closure evaluates the features of a stage's input state at the
 * interior points (central differences on the context's own grid), the MLP,
 * and the source S(rho u_a) = -d tau_ab / dx_b, S(rho E) = -gama d q_b / dx_b
 * (zero fluxes on the walls); every stage adds cdt * S to its output.  With
 * on = 1 the source of a step's first stage is held for its other stages
 * (the subgrid term advanced by forward Euler, one evaluation per step); with
 * on = 2 every stage evaluates it.  Plain FP64 contexts only.  chan_closure_flag reports (and optionally resets) whether
 * a normalised output exceeded 50 in magnitude since the last reset. */
int chan_set_closure(chan_ctx *c, chan_closure *m, int32_t on);
int chan_closure_flag(chan_ctx *c, int32_t *flag, int32_t reset);

/* Tensor-core self-test: D[128][N] = A[128][K] * B[N][K]^T with BF16 A and B
 * (raw bit patterns, row-major) and F32 D, through the same tcgen05 path the
 * closure MLP uses (K and N multiples of 16 up to 256).  For tests. */
int chan_selftest_umma(const uint16_t *A, const uint16_t *B, float *D, int32_t K, int32_t N, int32_t device);

/* Free device memory and the context.  NULL is allowed.  A context that is a
 * member of an ensemble is freed after its ensemble. */
void chan_free(chan_ctx *c);

/* ------------------------------------------------------------------------
 * Ensembles (no reference counterpart: the reference runs one case per MPI
 * job).  Several contexts on one device -- a parameter sweep of cases with
 * their own grids, physics, wall BCs and precision -- stepped together.
 * Every member keeps its own buffers and stream.  A block of L steps of all
 * members (L = least common multiple of their istat) is captured once into
 * one CUDA graph and replayed: by default one branch of kernels per member,
 * run concurrently, or one persistent kernel that runs all members' work
 * (chan_ensemble_set_mode below).  Each member's results are bit for bit those of
 * chan_step on that member alone.  A context belongs to one ensemble at most;
 * members may still be used on their own between ensemble calls. */
typedef struct chan_ensemble chan_ensemble;

/* members: n distinct contexts on one device.  CHAN_EINVAL if a member is
 * NULL, repeated, already in an ensemble, on another device, or if L would
 * exceed 10000 steps. */
int chan_ensemble_create(chan_ctx *const *members, int32_t n, chan_ensemble **out);
int chan_ensemble_size(chan_ensemble *e);
/* L, the steps per graph replay */
int chan_ensemble_block(chan_ensemble *e);

/* nsteps whole steps of every member: graph replays for the whole blocks of
 * L steps, then the remaining steps queued on the members' own streams; each
 * member's per-step tail (statistics every istat, time averaging) as in
 * chan_step.  Waits, then reads every member's status into status[n] (may be
 * NULL) and returns the first nonzero one.  Members must be uploaded and
 * must not have the diagnostics series enabled. */
int chan_ensemble_step(chan_ensemble *e, int32_t nsteps, int32_t *status);

/* Autotuner of the members' stage-kernel launch shapes (chan_set_launch).
 * It times, with CUDA events, all but the last RK stage of every member run
 * concurrently, reps times per trial: first one shape for every member (each
 * tile shape at k-chunk depths of 4 to 128 planes and the whole height),
 * then one pass that tries every candidate for each member in turn, largest
 * grids first, keeping a change that saves more than 0.5%.  The members'
 * states, wall rings, statuses and counters are left as they were.  Writes
 * the best trial time (ms per trial step) to best_ms. */
int chan_ensemble_tune(chan_ensemble *e, int32_t reps, double *best_ms);

/* How a block of L steps runs (no reference counterpart).
 * CHAN_ENSEMBLE_PERSISTENT: one persistent kernel per block.
 *   It walks one work list of every member's units -- the CTAs of each RK
 *   stage, of each wall-BC pass and of the statistics passes, and the step's
 *   clock advance -- members interleaved; a unit starts once its member has
 *   completed its earlier work, which per-member device counters track, and
 *   each such wait is bounded (about a second).  The block is one graph of
 *   three nodes (the members' parameter records into constant memory, counter
 *   reset, the launch).  It needs members of one precision, without the
 *   closure, on the 32x8 or 16x16 tile, at most 64 parameter records (one per
 *   RK stage per member); otherwise the graph mode is used and
 *   chan_ensemble_get_mode says why.  The records' constant memory is one per
 *   device: two ensembles must not step concurrently in persistent mode.
 * CHAN_ENSEMBLE_GRAPH (the default, faster on the stratified sweep): one graph
 *   of every member's kernels, one branch per member on its own stream.
 * Either way each member's results are bit for bit those of chan_step.
 * CHAN_ENSEMBLE_PERSISTENT_STALL_TEST: persistent, with member 0's first stage
 *   made to wait for work that never completes (host-side fault injection
 *   for tests): chan_ensemble_step then returns CHAN_ECUDA after about a
 *   second and every member's state is undefined until uploaded again.
 * chan_ensemble_get_mode reports the mode of the captured block (-1 before
 * the first capture) and, if persistent mode was asked for but not used, the
 * reason (an empty string otherwise; valid until the next call). */
#define CHAN_ENSEMBLE_GRAPH 0
#define CHAN_ENSEMBLE_PERSISTENT 1
#define CHAN_ENSEMBLE_PERSISTENT_STALL_TEST 2
int chan_ensemble_set_mode(chan_ensemble *e, int32_t mode);
int chan_ensemble_get_mode(chan_ensemble *e, int32_t *in_use, const char **fallback_reason);

/* graph replays and graph captures so far, and the device time (CUDA events
 * on the launching stream) of the graph replays of the last
 * chan_ensemble_step call (0 if it replayed none) */
int chan_ensemble_counters(chan_ensemble *e, int64_t *replays, int64_t *captures, double *last_ms);
const char *chan_ensemble_last_error(chan_ensemble *e);
/* Frees the ensemble (not its members).  NULL is allowed. */
void chan_ensemble_free(chan_ensemble *e);

#ifdef __cplusplus
}
#endif

#endif /* CHANRHS_H */

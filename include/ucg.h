/*
 * ucg.h -- C ABI of libucg.so, the B200 (sm_100a) replacement for the 3-D
 * quasi-dynamic boundary-integral hot path of Unicycle (fortran/3d).
 *
 * Plain C types only: pointers, sizes and doubles.  All arrays passed in are
 * host memory owned by the caller and are copied during the call; the library
 * owns every device allocation (matrix, state, Runge-Kutta scratch), one CUDA
 * stream per context.  Every entry point returns an int status (UCG_OK = 0);
 * none aborts the process.  One host thread per context.
 *
 * Coordinates are (north, east, down) in the length unit of the mesh, angles
 * in radians, element orders rectangles -> triangles -> volumes, exactly as the
 * reference's input deck and layout (fortran/3d/src/types.f90:125-223).
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef UCG_H
#define UCG_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ucg_ctx ucg_ctx;

/* status codes */
#define UCG_OK                0
#define UCG_E_BADARG          1   /* invalid argument or size                  */
#define UCG_E_CUDA            2   /* CUDA runtime error (message: ucg_last_error) */
#define UCG_E_OOM             3   /* device allocation failed                  */
#define UCG_E_STEP_UNDERFLOW  4   /* "stepsize underflow in RKQS" (ode45.f90:87-90) */
#define UCG_E_NONFINITE       5   /* non-finite state or rate detected         */
#define UCG_E_TIMEOUT         6   /* a bounded device wait gave up             */
#define UCG_E_STATE           7   /* call out of order (e.g. odefun before assemble) */
#define UCG_E_UNSUPPORTED     8   /* feature not available in this build       */
#define UCG_E_NODEVICE        9   /* no CUDA device / extension unusable       */

/* Okada (1992) interface precision (ucg_assemble) */
#define UCG_OKADA_FP64     0   /* DC3D math and interface in binary64           */
#define UCG_OKADA_REF32IO  1   /* the reference's REAL*4 DC3D interface (okada92.f90:121-160) */

/* matrix storage for the traction product (ucg_set_precision) */
#define UCG_PREC_FP64        0  /* K in binary64, FP64 matvec (the plain method) */
#define UCG_PREC_SPLIT_BF16  1  /* K = diag(s) k, s a per-row scale: stage 1 (the anchor) reads the
                                   split pair of k (bf16 hi + a 16-bit lo extension, together the
                                   FP32 value, FP64 sums), stages 2-6 the velocity increments in
                                   FP32 against an fp16 plane of k (a quarter of the FP64 bytes):
                                   FP32 products over 8 entries, their sums added in FP64 */
#define UCG_PREC_SPLIT_PAIR  4  /* the same split pair for every stage (half of the FP64 bytes),
                                   anchored, FP64 sums: the accurate split form */
#define UCG_PREC_HMATRIX     2  /* hierarchical approximation of K (ucg_build_hmatrix), FP64 */
#define UCG_PREC_HMATRIX_SPLIT 3  /* the same stored as the FP32 value of every entry in two 16-bit
                                     planes (bf16 hi, lo extension): half the FP64 bytes for every
                                     stage, anchored stages, FP64 sums */

/* driver conventions (ucg_create flags) */
#define UCG_DRIVER_RATESTATE      0  /* fortran/3d/src/ratestate.f90     */
#define UCG_DRIVER_VISCOUSCYCLES  1  /* fortran/3d/src/viscouscycles.f90 */

/* ---- context ------------------------------------------------------------ */

/* Create a context on CUDA device `device` for an elastic half-space with shear
   modulus mu and Lame parameter lambda.  flags: UCG_DRIVER_*.
   Replaces the module state set up by init()/initParallelism
   (fortran/3d/src/ratestate.f90:788-899, 958-1739). */
int ucg_create(ucg_ctx **ctx, int device, double mu, double lambda, int flags);
void ucg_destroy(ucg_ctx *ctx);
const char *ucg_strerror(int status);
/* Last detailed error message of this context (CUDA error text etc.). */
const char *ucg_last_error(ucg_ctx *ctx);

/* ---- geometry (copied at the call) --------------------------------------- */

/* n rectangles: x[3*i..3*i+2] upper-left corner (north, east, down), length L,
   width W, strike and dip in radians.  Replaces in%rectangularPatch and
   computeReferenceSystemOkada92 (fortran/3d/src/okada92.f90:59-87). */
int ucg_set_rectangles(ucg_ctx *ctx, int n, const double *x, const double *L,
                       const double *W, const double *strike, const double *dip);

/* n triangles over nve vertices v[3*k..3*k+2]; i1,i2,i3 are 1-based vertex ids.
   Replaces in%triangularPatch and computeReferenceSystemStuart97
   (fortran/3d/src/stuart97.f90:44-101). */
int ucg_set_triangles(ucg_ctx *ctx, int n, const int *i1, const int *i2, const int *i3,
                      int nve, const double *v);

/* n vertical cuboid strain volumes: corner x, length L, thickness T, width W,
   strike.  Replaces in%strainVolume and computeReferenceSystemVerticalStrainVolume
   (fortran/3d/src/strainvolume.f90:135-163). */
int ucg_set_volumes(ucg_ctx *ctx, int n, const double *x, const double *L,
                    const double *T, const double *W, const double *strike);

/* ---- constitutive parameters -------------------------------------------- */

/* Per patch (rectangles then triangles), the PATCH_ELEMENT_STRUCT fields
   (fortran/3d/src/types.f90:35-40): Vpl, rake, mu0, sig, a, b, L, Vo, damping. */
int ucg_set_friction(ucg_ctx *ctx, const double *Vpl, const double *rake,
                     const double *mu0, const double *sig, const double *a,
                     const double *b, const double *L, const double *Vo,
                     const double *damping);

/* Per volume: background strain rate e_bg[6*i..] (e11,e12,e13,e22,e23,e33) and
   the steady-state nonlinear Maxwell fields ngammadot0m, npowerm used by
   odefun (fortran/3d/src/viscouscycles.f90:938-995).  nonlinear_maxwell != 0
   mirrors in%strainVolume%nNonlinearMaxwell > 0. */
int ucg_set_rheology(ucg_ctx *ctx, const double *e_bg, const double *gammadot0m,
                     const double *npowerm, int nonlinear_maxwell);

/* ---- Green's functions ---------------------------------------------------- */

/* Assemble the stress-interaction matrix on the device, FP64, one thread per
   (receiver, source) pair.  Replaces buildG (fortran/3d/src/greens.f90:73-275).
   okada_mode: UCG_OKADA_*. */
int ucg_assemble(ucg_ctx *ctx, int okada_mode);

/* Device time (ms) of the last ucg_assemble per source family: the columns of
   rectangles, triangles and volumes (all receivers each).  No reference
   counterpart (a measurement aid). */
int ucg_assembly_times(ucg_ctx *ctx, double *rect_ms, double *tri_ms, double *vol_ms);

/* Sizes of the reference layout G(n,m): n source DOFs, m receiver DOFs. */
int ucg_dims(ucg_ctx *ctx, long *n, long *m);

/* Copy G in the reference layout: G(c,k) at G[k*ld + c], ld >= n (Fortran
   column-major, greens.f90:214-216,266-271).  Columns [k0,k1). */
int ucg_copy_G(ucg_ctx *ctx, double *G, long ld, long k0, long k1);

/* Select the storage of K used by the traction product (UCG_PREC_*).
   Switching to split-BF16 builds the hi/lo pair from the assembled FP64 K. */
int ucg_set_precision(ucg_ctx *ctx, int precision);

/* Keep (keep != 0, default) or release the FP64 K after a split-BF16 copy
   exists, freeing its HBM. */
int ucg_keep_fp64(ucg_ctx *ctx, int keep);

/* Hierarchical approximation of K for a fault model of one patch family
   (rectangles or triangles; no volumes): patches ordered by a cluster tree
   of `leaf` patches, pairs of clusters with max(diam) <= eta dist stored as
   low-rank factors found by adaptive cross approximation to relative accuracy
   eps (each checked against its dense block), the rest dense.  Every block is
   assembled on the device and compressed at once, so the dense K is never
   held (models beyond what a dense K fits in HBM).  The reference's MATLAB
   toolbox does this with the hmmvp library
   (matlab/+unicycle/+ode/+hmmvp/rateandstate.m:71-143).  Selected for the
   traction product with ucg_set_precision(ctx, UCG_PREC_HMATRIX). */
int ucg_build_hmatrix(ucg_ctx *ctx, int okada_mode, double eta, double eps, int leaf);
/* blocks stored dense (including low-rank candidates that failed their check)
   and low-rank, bytes stored, the largest rank, device time of the build */
int ucg_hmatrix_info(ucg_ctx *ctx, long *n_dense, long *n_lowrank, long *bytes, int *max_rank,
                     double *build_ms);
/* y (m) = H x (n), host arrays */
int ucg_hmatrix_matvec(ucg_ctx *ctx, const double *x, double *y);
/* mean device time (ms) of one product H v over reps launches */
int ucg_hmatrix_profile(ucg_ctx *ctx, int reps, double *ms);

/* ---- state and right-hand side ------------------------------------------- */

/* Length of the state vector: 7 per patch + 12 per volume
   (fortran/3d/src/macros.f90:56-79). */
long ucg_state_len(ucg_ctx *ctx);

/* Reference initial state.  Replaces initStateVector
   (fortran/3d/src/ratestate.f90:548-610, viscouscycles.f90:710-820).
   Volume initial stress needs nGm, nQm, nRm, To (per volume); pass NULL when
   there are no volumes. */
int ucg_init_state(ucg_ctx *ctx, double *y, const double *nGm, const double *nQm,
                   const double *nRm, const double *To);

/* dydt = f(y) with host arrays.  Replaces odefun
   (fortran/3d/src/ratestate.f90:624-778; viscouscycles.f90:834-1093).
   vmax (may be NULL) receives max patch slip velocity. */
int ucg_odefun(ucg_ctx *ctx, double t, const double *y, double *dydt, double *vmax);

/* Integrator settings: the module globals `epsilon` and `maximumTimeStep` of
   fortran/3d/src/ode45.f90:40-43. */
int ucg_set_tolerance(ucg_ctx *ctx, double epsilon, double max_step);

/* One RKQSm call with host arrays (fortran/3d/src/ode45.f90:51-108): attempts
   Cash-Karp steps from (t, y) with derivative dydt and error scale yscal until
   one is accepted.  On return y holds the accepted state, *t += *hdid.
   Returns UCG_E_STEP_UNDERFLOW where the reference prints "stepsize underflow"
   and stops.  *nrej (may be NULL) receives the number of rejected attempts. */
int ucg_rkqs(ucg_ctx *ctx, double *t, double *y, const double *dydt, const double *yscal,
             double htry, double *hdid, double *hnext, long *nrej);

/* One iteration of the reference main loop (fortran/3d/src/ratestate.f90:307-326)
   with host arrays: dydt = f(y), yscal = |y| + |dt_next*dydt| + 1e-30, RKQSm,
   time += dt_done.  dydt receives f(y) at the start of the step (what export()
   writes).  y is updated in place. */
int ucg_step(ucg_ctx *ctx, double *time, double *y, double *dydt, double *dt_next,
             double *dt_done, long *nrej);

/* ---- device-resident integration ---------------------------------------- */

/* Upload y as the device state with time and dt_next (ucg_set_state) or read
   it back (ucg_get_state).  Counters: accepted steps and rejected attempts. */
int ucg_set_state(ucg_ctx *ctx, const double *y, double time, double dt_next);
int ucg_get_state(ucg_ctx *ctx, double *y, double *time, double *dt_next,
                  long *accepted, long *rejected);

/* March the device state with the reference main loop until time >= t_end or
   max_steps accepted steps, without host round trips per step (attempts are
   queued in batches; accept/reject, step size and the time update live on the
   device).  *steps receives the accepted steps taken.  Returns
   UCG_E_STEP_UNDERFLOW / UCG_E_NONFINITE as the device detects them. */
int ucg_run(ucg_ctx *ctx, double t_end, long max_steps, long *steps);

/* ---- observation points (buildO / exportPoints) ---------------------------- */

/* Observation points (north, east, down), 3 per point: the
   reference's observationPoint list (input.f90, "observation points").
   Replaces any previous set and its O; stops a recording in progress. */
int ucg_set_observation_points(ucg_ctx *ctx, int nobs, const double *x);
/* Assemble O on the device: the displacement (north, east, down) at every
   point for unit slip (strike, dip) of every patch and unit eigenstrain
   (11, 12, 13, 22, 23, 33) of every volume, laid out 3 nobs rows x n columns
   (row-major; the columns of K).  Replaces buildO (fortran/3d/src/greens.f90:
   302-462) with computeDisplacementOkada92 / Nikkhoo15 / VerticalStrainVolume;
   okada_mode as for ucg_assemble.  Stops a recording in progress. */
int ucg_build_O(ucg_ctx *ctx, int okada_mode);
/* number of points, values recorded per point (3, or 9 with volumes: total,
   faulting, flow as viscouscycles' exportPoints writes them) and the device
   time of the last ucg_build_O */
int ucg_observation_info(ucg_ctx *ctx, int *nobs, int *per_point, double *build_ms);
/* copy O (3 nobs x n doubles, row-major) to the host */
int ucg_copy_O(ucg_ctx *ctx, double *O);
/* Displacement at every point for the state y (3 nobs values each): the total
   O u, and optionally (NULL to skip) the faulting and flow sets of
   viscouscycles.f90:521-633.  As buildO does, a volume's down column counts
   toward the faulting set, so the flow set's down component is zero. */
int ucg_displacements(ucg_ctx *ctx, const double *y, double *d, double *d_fault, double *d_flow);

/* ---- coseismic perturbations (in%event) --------------------------------------- */

/* A perturbation at `time`: u holds a slip increment (strike, dip) per patch and
   an eigenstrain increment (11, 12, 13, 22, 23, 33) per volume, the source-DOF
   layout of K's columns.  ucg_run ends the step that reaches `time` exactly on
   it, adds u to the slip / strain components of the state and K u to the
   tractions / stresses (the stress change the increment causes), and restarts
   from the reference's initial tentative step (1e-3 s).  The reference reads
   perturbation times into in%event (viscouscycles.f90:2022-2049) without using
   them; this gives them content.  Perturbations at or after a time passed to
   ucg_set_state are pending again.  Needs the FP64 K (ucg_keep_fp64). */
int ucg_add_event(ucg_ctx *ctx, double time, const double *u);
int ucg_clear_events(ucg_ctx *ctx);
/* the same increment applied to the device state now */
int ucg_apply_perturbation(ucg_ctx *ctx, const double *u);

/* ---- output recording (export / exportPoints) ------------------------------ */

/* Record on the device, without host round trips, at the start of every
   `every`-th accepted step of ucg_run / ucg_step: time, dt_done (the step just
   taken; 0 at the first), max slip rate, the accepted-step count, then for each
   listed element (0-based, patches then volumes) its state (7 or 12 values)
   and its rate dydt in a slot of 24 (state at 0.., rate at 12..), then the
   displacements at every observation point built with ucg_build_O (3 per
   point, or 9 with volumes: total, faulting, flow; see ucg_displacements).
   The observation set is the one built when recording starts.  Replaces the per-step formatted writes of export() and
   exportPoints() (fortran/3d/src/ratestate.f90:405-537: time.txt, the
   observation states, opts-*.dat).  Records go to a ring of `capacity`
   records (0 stops recording); ucg_records drains them in order. */
int ucg_record(ucg_ctx *ctx, int every, const int *elements, int nelem, long capacity);
/* doubles per record with the current settings */
long ucg_record_len(ucg_ctx *ctx);
/* Copy up to max_records of the records not yet drained, oldest first;
   *lost receives the records overwritten before they were drained. */
int ucg_records(ucg_ctx *ctx, double *out, long max_records, long *n_records, long *lost);

/* ---- input decks (init) ---------------------------------------------------- */

/* A parsed input deck of the reference's 3-D drivers: the text read by init()
   of fortran/3d/src/ratestate.f90:958-1739 (driver UCG_DRIVER_RATESTATE) or
   fortran/3d/src/viscouscycles.f90:1291-2069 (UCG_DRIVER_VISCOUSCYCLES),
   with the same sections, order and validation; angles are returned in
   radians.  Host-only: needs no device. */
typedef struct ucg_deck ucg_deck;

typedef struct {
    int driver;
    double lambda, mu, interval;
    int n_rect, n_tri, n_vertex, n_vol;
    int nonlinear_maxwell;  /* nonlinear Maxwell properties given for every volume */
    int thermal;            /* thermal properties given for every volume */
    int n_obs_state;        /* observation patches, then observation volumes */
    int n_obs_point;
    int n_events;           /* perturbations; the first is at t = 0 */
} ucg_deck_info;

/* Parse the whole deck text; on UCG_E_BADARG err receives the line number and
   the reason (the reference's STOP message). */
int ucg_deck_parse(const char *text, int driver, ucg_deck **deck, char *err, long err_len);
/* the same for a file */
int ucg_deck_read(const char *path, int driver, ucg_deck **deck, char *err, long err_len);
void ucg_deck_free(ucg_deck *deck);
int ucg_deck_summary(const ucg_deck *deck, ucg_deck_info *info);
/* output directory (the deck's first line) */
const char *ucg_deck_wdir(const ucg_deck *deck);
/* name of observation point k (0-based; at most 10 characters) */
const char *ucg_deck_point_name(const ucg_deck *deck, int k);
/* Copy up to max values of a field into out (out may be NULL); returns the
   field's length, or a negative status for an unknown field.  Doubles:
   rect.x (3 per patch), rect.length, rect.width, rect.strike, rect.dip,
   tri.vertices (3 per vertex), patch.Vpl, patch.rake, patch.mu0, patch.sig,
   patch.a, patch.b, patch.L, patch.Vo, patch.damping (rectangles then
   triangles), vol.x, vol.length, vol.width, vol.thickness, vol.strike,
   vol.e_bg (6 per volume), vol.Gm, vol.gammadot0m, vol.npowerm, vol.Q, vol.R,
   vol.rhoc, vol.To, obs.x (3 per point), events.time.  Integers: tri.i1,
   tri.i2, tri.i3 (1-based vertices), obs.state (1-based elements, volumes
   numbered after all patches). */
long ucg_deck_get(const ucg_deck *deck, const char *field, double *out, long max);
long ucg_deck_get_int(const ucg_deck *deck, const char *field, int *out, long max);
/* Load the deck's elements, friction, rheology and observation points into a
   context (ucg_set_*); ucg_deck_create also creates the context with the
   deck's moduli and driver. */
int ucg_deck_apply(const ucg_deck *deck, ucg_ctx *ctx);
int ucg_deck_create(const ucg_deck *deck, int device, ucg_ctx **ctx);
/* initStateVector with the deck's volume properties (ucg_init_state) */
int ucg_deck_init_state(const ucg_deck *deck, ucg_ctx *ctx, double *y);

/* Options of the reference's command line (ratestate.f90:975-1030) and of
   the device loop. */
typedef struct {
    double epsilon;           /* --epsilon (reference default 1e-6) */
    double maximum_step;      /* --maximum-step (default: no limit) */
    long maximum_iterations;  /* --maximum-iterations (default 1000000) */
    int okada_mode;           /* UCG_OKADA_* for buildG and buildO */
    int precision;            /* UCG_PREC_* of the traction product */
    int device;
    long chunk;               /* iterations per device run between recorder drains */
    const char *wdir;         /* output directory; NULL: the deck's */
    int verbose;              /* progress lines on standard output */
    double hm_eta, hm_eps;    /* UCG_PREC_HMATRIX: ucg_build_hmatrix parameters (0: 2, 1e-6) */
    int hm_leaf;              /*   and leaf size (0: 32); the dense K is then never assembled */
} ucg_run_options;

/* The whole run of a deck, as the reference's main program does it
   (ratestate.f90:170-372): buildG, buildO, initStateVector, dt = 1e-3, then
   iterations until the deck's time interval or maximum_iterations, writing
   time.txt, patch-%08d.dat / volume-%08d.dat for the observation states and
   opts-<name>.dat for the observation points into the output directory, in
   the reference's formats.  *iterations and *time receive the iterations run
   and the final time; the return is the integrator's status. */
int ucg_deck_run(const ucg_deck *deck, const ucg_run_options *opt, long *iterations, double *time);

/* Number of kernel launches this context has issued (for launch accounting). */
long ucg_launch_count(ucg_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), so that callers can order their
   own work or timing events with the library's.  No reference counterpart. */
void *ucg_stream(ucg_ctx *ctx);

/* Launch the traction-product kernel of one Runge-Kutta stage `reps` times on
   the context stream between CUDA events and return the mean device time per
   launch in *ms (a measurement aid for the roofline; the state must have been
   stepped at least once).  No reference counterpart. */
int ucg_profile_traction(ucg_ctx *ctx, int reps, double *ms);

/* Fault injection for testing the bounded device waits (the reference has no
   counterpart: its failures end in STOP).  wait_ns > 0 replaces the 4 s limit
   of the traction product's data waits; hold != 0 makes the product's first
   CTA issue no copies, so that its consumers wait on data that never comes,
   give up after wait_ns and the call (ucg_odefun, ucg_step, ucg_run) returns
   UCG_E_TIMEOUT with the context still usable.  ucg_test_wait_timeout(ctx, 0,
   0) restores normal operation. */
int ucg_test_wait_timeout(ucg_ctx *ctx, long wait_ns, int hold);

/* ---- allocation-free right-hand side ------------------------------------- */

/* dydt = f(y) for a fault model held entirely in caller-owned DEVICE memory,
   without any device allocation: for callers that cannot call cudaMalloc at
   this point (an external memory manager owns the device, or an
   allocation-free real-time loop).  No counterpart in the reference; the
   context-based equivalent is ucg_odefun above.
   K: m x n row-major traction matrix (m = 3 np, n = 2 np; patches only), its
   base address 16-byte aligned (its rows are moved by bulk copies);
   y, dydt: 7 np state and rate; per patch Vpl*cos(rake), Vpl*sin(rake), a, b,
   sig, L, damping; every double array 8-byte aligned.  UCG_E_BADARG, before
   anything is queued, for a null or misaligned pointer or inconsistent sizes.
   Work is queued on `stream` (a cudaStream_t, NULL for the default stream) on
   the current device; the return value reports only the checks and the
   launches.  status (optional, caller-owned DEVICE int, may be NULL) receives,
   in stream order after the result, UCG_OK, UCG_E_NONFINITE (a NaN/Inf state
   or rate) or UCG_E_TIMEOUT (a bounded device wait gave up: dydt incomplete).
   The only working storage is a fixed 8 MB array in the library's device
   image, which bounds n at 2^20 source DOFs (UCG_E_BADARG beyond); every GPU
   that loads the library holds it until the process exits.  The first call on
   a device may load the library's device code and should come before any
   stream capture.  Calls share the array: calls that overlap on the GPU race
   and must be ordered by the caller. */
int ucg_odefun_noalloc(const double *K, long n, long m, int np, const double *y,
                       const double *Vpl_cos_rake, const double *Vpl_sin_rake,
                       const double *a, const double *b, const double *sig,
                       const double *L, const double *damping, double *dydt,
                       void *stream, int *status);

/* ---- batched ensembles (tensor-core traction product) --------------------- */

/* An ensemble marches many instances (frictional-parameter sets) of one or
   more fault geometries together.  Each Runge-Kutta stage evaluates T = K V for
   all instances of a geometry as one contraction on the tcgen05 tensor cores,
   with K and V held as bf16 hi/lo pairs (K with a power-of-two scale per row)
   and FP32 accumulation; state, stage combinations, error norm and step
   control stay FP64, and every instance keeps its own step size, time and
   RKQSm decision (fortran/3d/src/ode45.f90:51-108, per instance).  A run is
   one CUDA-graph launch whose while loop repeats the attempt of all instances
   until every instance reaches t_end or the attempt budget is spent.  No
   reference counterpart: the reference runs one parameter set per job. */
typedef struct ucg_ensemble ucg_ensemble;

#define UCG_ENS_STREAM_K   0   /* (tile, k-block) sequence cut into equal ranges per SM */
#define UCG_ENS_SPLIT_LPT  1   /* k-split tiles, longest-first onto the least loaded SM */

int ucg_ens_create(ucg_ensemble **ens, int device);
void ucg_ens_destroy(ucg_ensemble *ens);
const char *ucg_ens_last_error(ucg_ensemble *ens);

/* Add a geometry from a context that holds an assembled FP64 matrix (patches
   only), with n_instances instances (1..4096).  The matrix is converted to the
   tensor-core image at the call; the context may be destroyed afterwards.
   A context that steps on its hierarchical matrix (ucg_build_hmatrix with
   leaf <= 42, then UCG_PREC_HMATRIX or UCG_PREC_HMATRIX_SPLIT) or holds no
   dense matrix gives a hierarchical geometry: H is laid out as tensor-core
   operand images and every stage runs the two-pass hierarchical contraction
   (UCG_E_UNSUPPORTED for wider leaves).  No reference counterpart (the
   reference runs one parameter set per job).
   *geometry receives the geometry index. */
int ucg_ens_add_geometry(ucg_ensemble *ens, ucg_ctx *ctx, int n_instances, int *geometry);

/* Friction of one instance, the arrays of ucg_set_friction (per patch). */
int ucg_ens_set_friction(ucg_ensemble *ens, int geometry, int instance, const double *Vpl,
                         const double *rake, const double *mu0, const double *sig,
                         const double *a, const double *b, const double *L,
                         const double *Vo, const double *damping);

/* epsilon and maximumTimeStep of fortran/3d/src/ode45.f90:40-43, all instances. */
int ucg_ens_set_tolerance(ucg_ensemble *ens, double epsilon, double max_step);

/* State of one instance (7 per patch, the layout of ucg_set_state).  An
   instance takes part in runs once its state has been set. */
int ucg_ens_set_state(ucg_ensemble *ens, int geometry, int instance, double time,
                      const double *y, double dt_next);
int ucg_ens_get_state(ucg_ensemble *ens, int geometry, int instance, double *y, double *time,
                      double *dt_next, long *accepted, long *rejected, int *status);

/* All instances of one geometry at once: y is instance-major
   (n_instances x 7 n_patches), time, dt_next, accepted, rejected, status one
   per instance (outputs may be NULL).  Setting resets the counters. */
int ucg_ens_set_states(ucg_ensemble *ens, int geometry, const double *y, const double *time,
                       const double *dt_next);
int ucg_ens_get_states(ucg_ensemble *ens, int geometry, double *y, double *time, double *dt_next,
                       long *accepted, long *rejected, int *status);
/* Replace every instance's state vector of a geometry from a host array
   (n_instances x 7 n_patches) and keep each instance's time, step size,
   counters and step-size history: a driver that takes the states to the host
   between runs (ucg_ens_get_states) and hands them back continues exactly as
   the device-resident loop would.  An instance whose state changed in any bit
   re-evaluates f(y) and yscal at its next attempt (a new main-loop iteration,
   fortran/3d/src/ratestate.f90:307-326).  No reference counterpart. */
int ucg_ens_put_states(ucg_ensemble *ens, int geometry, const double *y);

/* Precision of the stage increments (stages 2-6 contract v_s - v1): terms = 3,
   the default, the anchor's form Khi Vhi + 2^-11 (Khi Vlo + Klo Vhi), which
   keeps slip-rate histories within 1e-6 of the FP64 integrator's; terms = 2,
   Khi (Vhi + Vlo) over pairs of M-tiles, half the matrix bytes and fp16
   precision of K (about 2e-5 on the same histories).  No reference
   counterpart. */
int ucg_ens_set_increment_terms(ucg_ensemble *ens, int terms);

/* Operand precision of the hierarchical geometries' tensor-core contraction,
   fixed before the first hierarchical geometry is added (UCG_E_STATE after):
   planes = 3, the default, keeps every image (the low-rank factors, the dense
   leaf blocks, the slip rates and the intermediate Z) as three bf16 planes
   (hi, mid, lo: 24 significant bits) and forms the six products of weight
   2^-16 and above; planes = 2 keeps hi and lo (16 bits: about 2e-5 on slip-rate
   histories), two thirds of the bytes, and allows 128-instance tiles.  No
   reference counterpart. */
int ucg_ens_set_hier_planes(ucg_ensemble *ens, int planes);

/* Fault injection for testing the bounded device waits (no reference
   counterpart).  wait_ns > 0 replaces the 4 s limit of the dense contraction's
   data waits; hold != 0 makes the CTA that owns the first work segment issue
   no copies, so that its MMA issuer waits on data that never comes and gives up: ucg_ens_run (and
   ucg_ens_matvec) then return UCG_E_TIMEOUT, the instances' stage kernels skip
   the attempt, and the ensemble stays usable after ucg_ens_test_wait_timeout(ens,
   0, 0) and fresh states. */
int ucg_ens_test_wait_timeout(ucg_ensemble *ens, long wait_ns, int hold);

/* Contraction plan: instance tile width ni (32, 64 or 128 instances per MMA)
   and schedule (UCG_ENS_*; chunk = k-blocks per split for UCG_ENS_SPLIT_LPT,
   0 = whole tiles).  Without a call the first run picks ni from the largest
   instance count and stream-K. */
int ucg_ens_plan(ucg_ensemble *ens, int ni, int schedule, int chunk);

/* Autotuner: times every candidate plan (`reps` launches each) on the device,
   installs the fastest and writes a one-line-per-candidate report. */
int ucg_ens_tune(ucg_ensemble *ens, int reps, char *report, long report_len);

/* Run attempts as one CUDA-graph launch (use_graph != 0, the default) or
   launch the same kernels one by one from the host (for profilers that do not
   follow conditional graph nodes). */
int ucg_ens_use_graph(ucg_ensemble *ens, int use_graph);

/* March every instance to t_end (attempts of all instances in lockstep, at
   most max_attempts in this call).  *attempts receives the attempts made. */
int ucg_ens_run(ucg_ensemble *ens, double t_end, long max_attempts, long *attempts);

/* T = K V through the tensor-core contraction for one geometry: V is
   instance-major (n_instances x n source DOFs), T instance-major
   (n_instances x m receiver DOFs), host arrays.  terms = 3: Khi Vhi + Khi Vlo +
   Klo Vhi (the stage-1 anchor's product); terms = 2: Khi Vhi + Khi Vlo (the
   stage increments' product, half the matrix bytes). */
int ucg_ens_matvec(ucg_ensemble *ens, int geometry, const double *V, double *T, int terms);

/* Event catalogue per instance: an event starts at the first accepted step
   whose starting max slip rate is >= vmax_on and ends once it is < vmax_off
   (defaults 1e-3 and 1e-4 m/s).  *n_events receives the number of events,
   *t_first the start time of the first one (-1 when there was none). */
int ucg_ens_set_event_threshold(ucg_ensemble *ens, double vmax_on, double vmax_off);
int ucg_ens_get_events(ucg_ensemble *ens, int geometry, int instance, long *n_events,
                       double *t_first);

/* Attempts so far, instances still active after the last attempt, kernel
   launches issued (a run's graph counts once, when it is built), accepted steps
   and rejected attempts summed over the instances, the sum of their simulated
   times, and the installed plan's name.  Any pointer may be NULL. */
int ucg_ens_info(ucg_ensemble *ens, long *total_attempts, int *active, long *launches,
                 long *accepted, long *rejected, double *time_sum, char *plan, long plan_len);

/* The ensemble's CUDA stream (a cudaStream_t), for callers' events. */
void *ucg_ens_stream(ucg_ensemble *ens);

/* Mean device time of one contraction launch over `reps` launches, for the
   anchor's (three-term) and the increments' (two-term) form; either pointer
   may be NULL. */
int ucg_ens_profile_contract(ucg_ensemble *ens, int reps, double *ms_anchor, double *ms_increment);

/* ---- learned step-size proposal ------------------------------------------- */

/* A perceptron 11 -> 64 -> 64 -> 64 (GELU) -> 1 with FP16 weights and
   activations (FP32 sums, FP32 master weights for training) that proposes
   log10 of the next step size from: log10 max V and min log10 theta at the
   start of the step, log10 of the last 8 accepted steps (most recent first)
   and log10 max(errmax, 1e-12) of the step just accepted.  Trained on the
   device by the library's own forward/backward kernels on traces that the
   ensemble integrator records.  In use, the proposal (limited to 0.2..10 times
   the accepted step) replaces RKQSm's hnext; the embedded error estimate still
   accepts or rejects the attempt, and a rejected proposal is shrunk by the plain RKQSm
   rule (fortran/3d/src/ode45.f90:79-84).  No reference counterpart. */
typedef struct ucg_mlp ucg_mlp;

#define UCG_MLP_NIN     11
#define UCG_MLP_NPARAM  9153   /* W1[64][11] b1 W2[64][64] b2 W3[64][64] b3 W4[64] b4 */
#define UCG_MLP_NNORM   24     /* input means[11], deviations[11], output mean, deviation */
#define UCG_TRACE_LEN   14     /* 11 inputs, log10 h of the next first attempt, log10 errmax, accepted */

int ucg_mlp_create(ucg_mlp **mlp, int device, unsigned long long seed);
void ucg_mlp_destroy(ucg_mlp *mlp);
const char *ucg_mlp_last_error(ucg_mlp *mlp);
/* FP32 master weights (UCG_MLP_NPARAM) and standardisation (UCG_MLP_NNORM);
   either may be NULL. */
int ucg_mlp_set_params(ucg_mlp *mlp, const float *params, const float *norm);
int ucg_mlp_get_params(ucg_mlp *mlp, float *params, float *norm);
/* Training set: x (n x 11 raw inputs), y (n labels, log10 dt); standardise != 0
   sets the standardisation from this set. */
int ucg_mlp_set_data(ucg_mlp *mlp, const float *x, const float *y, long n, int standardise);
/* Gradient of the mean loss over samples [offset, offset+count) at the current
   FP16 weights (UCG_MLP_NPARAM floats) and the mean loss. */
int ucg_mlp_gradient(ucg_mlp *mlp, long offset, long count, float *grad, double *loss);
/* Adam over shuffled mini-batches; epoch_loss (may be NULL) gets the mean
   loss of each epoch. */
int ucg_mlp_train(ucg_mlp *mlp, int epochs, int batch, float lr, unsigned long long seed,
                  float *epoch_loss);
/* log10 dt for raw inputs x (n x 11), with the controllers' own evaluation. */
int ucg_mlp_predict(ucg_mlp *mlp, const float *x, long n, float *y);

/* Use a model (NULL: the plain RKQSm controller) for every instance of an
   ensemble.  The model must outlive its use. */
int ucg_ens_set_step_model(ucg_ensemble *ens, const ucg_mlp *model);
/* Record traces (capacity records of UCG_TRACE_LEN floats; 0 stops and frees)
   and read them back. */
int ucg_ens_record_traces(ucg_ensemble *ens, long capacity);
int ucg_ens_get_traces(ucg_ensemble *ens, float *buf, long max_records, long *n_records);

#ifdef __cplusplus
}
#endif
#endif

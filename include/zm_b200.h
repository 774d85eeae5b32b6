/* C ABI of the B200 (sm_100a) global ocean step.
 *
 * Drop-in boundary for ZhenMode's production solver step.  The reference's
 * boundary is the Python factory
 *   make_solver_global(grid, physics, dt, **options) -> (step, init_state, diagnostics[, ...])
 * (src/zhenmode/model/solver/factory.py:30-68, 721-799), whose `step` is a
 * jax.jit closure over `_step_impl` (src/zhenmode/model/solver/timestepping/step.py:341-458).
 * The reference has no C or FFI layer; these entry points are what a jax.ffi
 * custom call or a ctypes/cffi binding of that factory binds.
 *
 * Conventions
 *  - Every array crossing this ABI uses the reference layout: 2-D fields are
 *    (nx, ny) and 3-D fields (nx, ny, nz), C order, longitude periodic on the
 *    first axis (src/zhenmode/model/solver/state.py:10-12).
 *  - State arrays are float32 (the reference's dtype='float32' mode); grid and
 *    parameter arrays are float64 host arrays, copied to the device once.
 *  - Functions return 0 on success or one of the ZM_ERR_* codes; the message of
 *    the last failure is available from zm_last_error().
 *  - A handle is used by one host thread at a time; handles share nothing.
 */
#ifndef ZM_B200_H
#define ZM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZM_OK 0
#define ZM_ERR_INVALID 1      /* invalid argument or configuration (the reference's ValueError) */
#define ZM_ERR_UNSUPPORTED 2  /* an option the B200 path does not implement */
#define ZM_ERR_CUDA 3         /* a CUDA runtime failure */
#define ZM_ERR_TIMEOUT 4      /* a bounded device wait gave up */
#define ZM_ERR_MONITOR 5      /* the device state monitor tripped */

#define ZM_VDIFF_EXPLICIT 0
#define ZM_VDIFF_IMPLICIT 1

#define ZM_LIMITER_CENTERED 0
#define ZM_LIMITER_DONOR 1    /* monotone_adv */
#define ZM_LIMITER_MINMOD 2   /* fct_adv */

typedef struct zm_solver zm_solver;

/* GlobalOceanGrid fields (src/zhenmode/model/solver/geometry/grid.py:13-61). */
typedef struct {
  int32_t nx, ny, nz;
  double dy;                  /* meridional spacing [m] */
  const double* dx_2d;        /* (nx, ny) zonal spacing [m] */
  const double* cos_lat;      /* (ny) */
  const double* f;            /* (nx, ny) Coriolis parameter [1/s] */
  const double* z;            /* (nz) level depths, negative downward */
  const double* dz;           /* (nz-1) layer thicknesses */
  const double* wet_mask;     /* (nx, ny) 1 ocean, 0 land */
  const double* wet_mask_3d;  /* (nx, ny, nz) or NULL: column-uniform from wet_mask */
} zm_grid;

/* Barotropic subcycle kernels: AUTO takes the resident kernel (every tile in
 * shared memory, one cooperative launch) when all tiles fit on the GPU at
 * once and the streaming kernels (three launches per subcycle) otherwise;
 * RESIDENT fails zm_create with ZM_ERR_UNSUPPORTED when they do not fit. */
#define ZM_BT_AUTO 0
#define ZM_BT_RESIDENT 1
#define ZM_BT_STREAMING 2

/* Preconditioner of the column projection's CG (projection_preconditioner). */
#define ZM_PROJ_NONE 0
#define ZM_PROJ_JACOBI 1

/* PhysicsConfig coefficients (src/zhenmode/model/config.py:86-140) and the
 * make_solver_global options of the mode-split production path
 * (src/zhenmode/model/solver/factory.py:30-68, 397-695). */
typedef struct {
  double dt, dt_bt;
  double nu_h, nu_v, kappa_h, kappa_v, kappa_conv, nu_bi, kappa_bi;
  double T_ref, S_ref, r_bot;
  double lambda_bulk, restore_coef_S, ice_salt_flux, ice_freeze_temp_c;
  int32_t nu_nsub;            /* 0: legacy count (= n_subcyc) */
  int32_t polar_cap_rows, polar_cap_taper;
  int32_t limiter;            /* ZM_LIMITER_* */
  int32_t localize_conv, conservative_kv, freeze_adv_vel;
  int32_t vertical_diffusion; /* ZM_VDIFF_* */
  int32_t bt_kernel;          /* ZM_BT_* barotropic kernel choice */
  int32_t autotune;           /* 1: time the result-neutral launch shapes at the first zm_advance */
  /* (nx, ny) float64 fields; NULL means zeros */
  const double* tau_x;
  const double* tau_y;
  const double* q_heat;
  const double* t_atm;               /* bulk target; used only with lambda_bulk > 0 */
  const double* s_ref;               /* SSS restore target */
  const double* coastal_restore_coef;/* 1/s */
  const double* coastal_restore_t;
  const double* coastal_bulk_lambda;
  const double* coastal_kappa_h;
  const double* coastal_kappa_v;
  /* column-divergence projection of the stage-2 advective velocity
   * (project_adv_vel; factory.py:366-386, dynamics/projection.py:64-127) */
  int32_t project_adv_vel;            /* 1: on */
  int32_t projection_niter;           /* CG iterations per solve, >= 1 */
  int32_t projection_preconditioner;  /* ZM_PROJ_NONE / ZM_PROJ_JACOBI */
  int32_t projection_max_refinements; /* 0..2 */
  double projection_rtol;             /* > 0, or 0 for the default 1e-12; floored at 32 float32 eps */
  /* lateral sponge (factory.py:456-491; step.py:142-156; barotropic.py:22-41):
   * NULL sponge_rate or all zeros is off; when on, T_clim and S_clim are required */
  const double* sponge_rate;          /* (nx, ny) Rayleigh rate [1/s] */
  const double* T_clim;               /* (nx, ny, nz) relaxation targets */
  const double* S_clim;
  /* semi-enclosed-sea eta relaxation (factory.py:493-521): off when the rate is 0 or the mask NULL */
  const double* eta_relax_mask;       /* (nx, ny) in [0, 1] */
  double eta_relax_rate;              /* [1/s] */
} zm_params;

/* JaxStateG fields u, v, T, S, eta (float32, reference layout); device
 * pointers unless a function says host pointers. */
typedef struct {
  float* u;
  float* v;
  float* T;
  float* S;
  float* eta;
} zm_state;

/* Build a solver for one grid and parameter set: validates, derives the
 * metric, subcycle counts and filter plans, copies everything to the current
 * CUDA device and allocates the work buffers (replaces the parameter
 * assembly of factory.py:397-718). */
int zm_create(const zm_grid* grid, const zm_params* params, zm_solver** out);

/* Derived counts: out[0] n_subcyc, out[1] nu subcycles, out[2] adv_nsub,
 * out[3] conv_nsub, out[4] row pitch, out[5] device MiB held, out[6] kernel
 * launches in one captured step (0 before the first zm_advance), out[7]
 * barotropic blocks of the resident kernel (0: streaming kernels), out[8] 1
 * when the polar cap of the barotropic mode is active (a band row is wet),
 * out[9] nu_h subcycles per temporally blocked pass (the halo width), out[10]
 * FFT lines per block, out[11] levels per block of the tracer-advection
 * march, out[12] of the linear-finish march, out[13] tile rows of the
 * vertical-transport march, out[14] of the pressure-gradient march, out[15]
 * warps per nu_h tile (8 or 16).  Writes min(n, 16) values. */
int zm_info(const zm_solver* s, int32_t* out, int32_t n);

/* Copy a device state (reference layout) into the solver's resident state. */
int zm_load_state(zm_solver* s, void* stream, const zm_state* in);

/* Advance the resident state nsteps baroclinic steps (step.py:341-458), each
 * one replay of a captured CUDA graph; stream ordered, no host sync. */
int zm_advance(zm_solver* s, void* stream, int32_t nsteps);

/* Copy the resident state out (reference layout, device pointers). */
int zm_store_state(zm_solver* s, void* stream, zm_state* out);

/* The jit `step` of factory.py:724-726 applied nsteps times: load, advance,
 * store.  in and out may alias. */
int zm_step(zm_solver* s, void* stream, const zm_state* in, zm_state* out, int32_t nsteps);

/* As zm_step with HOST pointers (pinned memory gives full copy bandwidth);
 * returns after the result is in `out`.  The copies run on a stream of the
 * solver's own, ordered after the work already queued on `stream`, so that
 * each field's layout change overlaps the next field's transfer. */
int zm_step_host(zm_solver* s, void* stream, const zm_state* in, zm_state* out, int32_t nsteps);

/* Replace the 2-D forcing fields (device float32 arrays, (nx, ny)); the
 * `step_dyn` path of factory.py:735-750.  NULL keeps a field. */
int zm_set_forcing(zm_solver* s, void* stream, const float* tau_x, const float* tau_y, const float* q_heat);

/* Seasonal forcing on the device (inputs/forcing/seasonal.py:86-103): each
 * given (12, nx, ny) float32 stack of monthly fields (device, reference
 * layout; NULL keeps the field) is blended for `day` (30-day months: the
 * current month, with the previous / next month over the first / last
 * blend_days / 2 days) into the forcing of the following steps.  Stream
 * ordered; the captured steps read the blended fields, no recapture. */
int zm_set_forcing_seasonal(zm_solver* s, void* stream, const float* tau_x, const float* tau_y, const float* q_heat,
                            double day, double blend_days);

/* Run one stage of the step on a device state, for stage-level checks:
 * 1 = linear half step L(dt/2) (step.py:76-187), 2 = nonlinear step N(dt)
 * (step.py:249-320), 3 = one full step, 4 = the velocity-only part of the
 * momentum residual into out->u/v (dealiased advection + surface wind -
 * barotropic wind, wet-masked; tendencies.py:39-72, 247-319), 5 = its
 * density part (baroclinic pressure-gradient force minus its barotropic
 * layer average, wet-masked; pressure.py:86-97, 144-180) into out->u/v,
 * 6 = the advection of stage 4 before its longitude filter (latitude
 * filter applied, no wind, no mask) into out->u/v, 7 = the longitude FFT
 * filter alone applied to in->u/v, 8 = the column-divergence projection of
 * in->u/v with the solver's dt (dynamics/projection.py:64-127; needs
 * project_adv_vel) into out->u/v.
 * out->T/S/eta receive the input fields for stages 4 to 8. */
int zm_run_stage(zm_solver* s, void* stream, int32_t stage, const zm_state* in, zm_state* out);

/* Kernel classes reported by zm_profile. */
#define ZM_K_NU_SUB 0        /* nu_h Laplacian subcycles */
#define ZM_K_INNER_LAP 1     /* inner Laplacians of the biharmonic operators */
#define ZM_K_LIN_FINISH 2    /* rest of the linear half step */
#define ZM_K_IMPLICIT 3      /* implicit vertical diffusion */
#define ZM_K_FZ 4            /* interface transport Fz */
#define ZM_K_MADV 5          /* momentum advection + latitude filter */
#define ZM_K_DEALIAS 6       /* longitude FFT filter */
#define ZM_K_TRACER_ADV 7    /* tracer advection substeps */
#define ZM_K_TRACER_REST 8   /* convection, surface sources, tracer RK combine */
#define ZM_K_PGF 9           /* pressure gradient, momentum RK combine, BT forcing */
#define ZM_K_BAROTROPIC 10   /* barotropic subcycle */
#define ZM_K_FINAL 11        /* projection, polar cap, land hold */
#define ZM_K_CLOSURE 12      /* learned closure: features + tensor-core MLP */
#define ZM_K_PROJECTION 13   /* column-divergence projection (right-hand side, CG, correction) */
#define ZM_K_COUNT 14

/* Advance the resident state by one step without the CUDA graph, timing
 * every kernel launch with CUDA events on `stream`; ms[c] and launches[c]
 * receive the summed time and launch count of class c (n >= ZM_K_COUNT).
 * Synchronizes the stream. */
int zm_profile(zm_solver* s, void* stream, float* ms, int32_t* launches, int32_t n);

/* Exercise the bounded grid barrier of the barotropic kernel: `blocks` blocks
 * each wait for `expected` arrivals, polling at most max_polls times.  With
 * expected == blocks the barrier completes (ZM_OK); with expected > blocks
 * the polls run out and ZM_ERR_TIMEOUT is returned with the context intact.
 * 1 <= blocks <= the SM count, expected >= blocks.  Synchronizes. */
int zm_barrier_probe(zm_solver* s, void* stream, int32_t blocks, int32_t expected, int32_t max_polls);

/* Monitor of the resident state after the last zm_advance (runtime/monitor.py:20-30):
 * 0 accepted, 1 non-finite, 3 velocity above 10 m/s, 4 |eta| above 15 m.
 * Returns ZM_ERR_TIMEOUT if a grid barrier of the barotropic or the column
 * projection kernel gave up (the state is then not a valid step result).  Synchronizes the device. */
int zm_status(zm_solver* s, int32_t* monitor_code);

/* One step with the FP64 stage/source ledger of the reference's budget audit
 * (make_budget_step, diagnostics/budgets.py:62-288): device state in -> out,
 * like zm_step with nsteps = 1 but without the CUDA graph, and the raw sums
 * into raw[0..ZM_LED_COUNT) (host memory; synchronizes):
 *   [0, 18)  stage changes [6][3]: linear_diffusion, sponge, nonlinear,
 *            free_surface, polar_cap_and_masks, dynamic_ice x (heat J, salt kg,
 *            volume m^3)
 *   [18, 21) summed magnitudes of the stage changes
 *   [21, 48) source inputs [9][3]: prescribed_heat, bulk_heat,
 *            coastal_bulk_heat, temperature_restore, salinity_restore,
 *            prescribed_brine, sponge, ice_atmosphere_heat, ice_brine
 *   [48, 60) nonlinear process changes [4][3]: advection, convection, gm, redi
 *   [60, 63) their summed magnitudes      [63, 66) advective surface flux
 *   [66, 69) squared surface-transport norms before / after the column
 *            projection and the worst ratio sqrt(after / before)
 *   [69, 72) observed change over the step  [72, 75) eta times the surface
 *            tracers, after minus before
 * The residual identities of the reference's ledger follow from these. */
#define ZM_LED_COUNT 75
int zm_ledger_step(zm_solver* s, void* stream, const zm_state* in, zm_state* out, double* raw, int32_t n);

/* CG iterations of the last column projection (needs project_adv_vel):
 * out[0] the first solve, out[1] and out[2] the refinement solves (0 when not
 * run), out[3] the refinement solves run.  Writes min(n, 4) values;
 * synchronizes the device. */
int zm_projection_stats(zm_solver* s, int32_t* out, int32_t n);

/* The diagnostics closure of make_solver_global (factory.py:752-760) on a
 * state in the caller's device arrays, reference layout (nx, ny, nz) float32:
 * rho = rho0 + rho'(T, S), the hydrostatic pressure rho0 g eta (+ the optional
 * (nx, ny) surface_pressure_pa, NULL for none) + the trapezoid integral of the
 * wet-masked density anomaly (dynamics/pressure.py:32-42, 62-74), and the
 * vertical velocity -Fz wet (dynamics/transport.py:149-166).  Outputs are
 * (nx, ny, nz) float32 device arrays.  Stream ordered, no host sync; uses the
 * handle's work buffers, so it must not overlap a step of the same handle. */
int zm_diagnostics(zm_solver* s, void* stream, const zm_state* in, const float* surface_pressure_pa, float* rho,
                   float* pressure, float* w);

/* ---- learned vertical-mixing closure: the per-column MLP ---------------
 * New in this library (the reference's closure is the plain kappa_v + coastal
 * band + convective gate of physics/vertical.py:40-82, which these calls are
 * trained to stand in for).  256 -> 256 -> 256 -> 64 with GELU after the
 * hidden layers; parameters are one float32 array of ZM_MLP_NPARAMS values:
 * W1 [256][256], b1 [256], W2 [256][256], b2 [256], W3 [64][256], b3 [64],
 * each W[out][in] with the input index contiguous. */
#define ZM_MLP_IN 256
#define ZM_MLP_OUT 64
#define ZM_MLP_NPARAMS 148032

/* Inference on the tensor cores: X [ncol][256] BF16 rows, W1/W2/W3 BF16 as
 * above, float32 biases; Y [ncol][64] float32 (raw outputs).  *err gets bit 0
 * set if a wait on the tensor cores ran out of polls.  Stream ordered. */
int zm_mlp_forward_bf16(void* stream, int32_t ncol, const void* X, const void* W1, const float* b1, const void* W2,
                        const float* b2, const void* W3, const float* b3, float* Y, uint32_t* err);

/* float32 parameters -> BF16 W1, W2, W3 (device arrays). Stream ordered. */
int zm_mlp_pack_bf16(void* stream, const float* params, void* W1, void* W2, void* W3);

/* float32 training: a trainer owns the workspaces for batches of up to
 * batch_max rows.  X [B][256], targets T [B][64], mask M [B][64] (1 where an
 * output is trained), mask_count = sum of M.  The loss is the masked mean
 * square error.  zm_mlp_grad writes the gradient of every parameter;
 * zm_mlp_train_step applies one Adam step (step counts from 1) in place.
 * *loss, when given, receives the batch loss (synchronizes the stream). */
typedef struct zm_mlp_trainer zm_mlp_trainer;
int zm_mlp_trainer_create(int32_t batch_max, zm_mlp_trainer** out);
void zm_mlp_trainer_destroy(zm_mlp_trainer* tr);
int zm_mlp_grad(zm_mlp_trainer* tr, void* stream, int32_t batch, const float* X, const float* T, const float* M,
                double mask_count, const float* params, float* grad_out, double* loss);
int zm_mlp_train_step(zm_mlp_trainer* tr, void* stream, int32_t batch, const float* X, const float* T, const float* M,
                      double mask_count, float* params, float* adam_m, float* adam_v, int32_t step, float lr,
                      float beta1, float beta2, float eps, double* loss);

/* Autotuner: time, on the resident state and through stages that write only
 * work buffers, the launch shapes that change no result (the nu_h halo
 * width 3..6, i.e. subcycles per temporally blocked pass, with 8 or 16 warps
 * per nu_h tile, the FFT lines per
 * block 1..8, the levels per block of the tracer-advection and linear-finish
 * column marches 5..25, and the tile rows of the vertical-transport and
 * pressure-gradient marches 4 or 8) and keep the fastest; the next zm_advance recaptures its
 * graphs.  zm_params.autotune = 1 runs it at the first zm_advance.  Writes
 * the choices when the pointers are given.  Synchronizes. */
int zm_autotune(zm_solver* s, void* stream, int32_t* nu_halo, int32_t* fft_lines);

/* Turn the learned vertical-mixing closure on for every following step of
 * the handle (params: ZM_MLP_NPARAMS float32 device values, see zm_mlp_*), or
 * off (params NULL).  While on, each step first infers a diffusivity per wet
 * interface from the step's input columns on the tensor cores; T and S then
 * diffuse vertically with it in the implicit interface-flux solve of the
 * linear half steps (u and v implicitly with nu_v), and the explicit
 * convective mixing of the tracer residual is dropped, the network standing
 * in for kappa_v + coastal + kappa_conv (physics/vertical.py:40-82).  A column
 * with a feature beyond +-bound (or not finite) takes the plain closure. */
int zm_set_closure(zm_solver* s, void* stream, const float* params, float bound);

/* Columns of the last step that took the plain closure, and tensor-core
 * waits that ran out of polls (ZM_ERR_TIMEOUT if any).  Synchronizes. */
int zm_closure_stats(zm_solver* s, uint32_t* fallback_columns, uint32_t* wait_errors);

/* The closure's diffusivity for a state (reference layout device arrays):
 * kappa [nx*ny][64] float32 in the row order of zm_closure_features, interface
 * m in column m (0 at dry interfaces and beyond nz-2).  Requires a closure set
 * by zm_set_closure.  Stream ordered; uses the handle's work buffers. */
int zm_closure_kappa(zm_solver* s, void* stream, const zm_state* in, float* kappa);

/* Training rows of a state (reference layout device arrays): per column
 * (j-major, i fastest; nx*ny rows) the 256 features X, log10 of the plain
 * closure's diffusivity at interfaces 0..nz-2 in T [.][64] and the wet
 * interface mask M [.][64].  Stream ordered; uses the handle's work buffers. */
int zm_closure_features(zm_solver* s, void* stream, const zm_state* in, float* X, float* T, float* M);

/* ---- ensembles -----------------------------------------------------------
 * Advance several handles (perturbed members, grids of any sizes) together:
 * each zm_ensemble_advance step is one launch of one CUDA graph holding one
 * step of every member, the members on parallel branches so that small grids
 * share the GPU.  The members' cooperative barotropic kernels are chained in
 * member order inside the graph (they never run at the same time).  States
 * are loaded and read per member (zm_load_state / zm_store_state); the
 * ensemble recaptures itself if a member stepped on its own or changed its
 * closure.  *kernels_per_step (optional) receives the graph's launch count.
 * New in this library (the reference runs ensemble members one by one). */
typedef struct zm_ensemble zm_ensemble;
int zm_ensemble_create(zm_solver* const* members, int32_t n, zm_ensemble** out);
int zm_ensemble_advance(zm_ensemble* e, void* stream, int32_t nsteps, int32_t* kernels_per_step);
void zm_ensemble_destroy(zm_ensemble* e);

/* Temperature-term decomposition of a state, the terms_fn of
 * make_solver_global (factory.py:762-764, dynamics/tendencies.py:74-92): terms
 * is a (6, nx, ny, nz) float32 device array receiving the land-masked
 * [advection, horizontal diffusion, vertical diffusion, convection, GM, Redi]
 * tendencies of T at the state (one advection evaluation with the step's face
 * limiter, kappa_h / kappa_v with their coastal parts, kappa_conv with the
 * step's convective gates; GM and Redi are zero on this path).  Stream
 * ordered, no host sync; uses the handle's work buffers, so it must not
 * overlap a step of the same handle. */
int zm_tracer_terms(zm_solver* s, void* stream, const zm_state* in, float* terms);

/* Global heat/salt/volume snapshot of a state (compute_budget_diagnostics,
 * diagnostics/snapshot.py:67-128, legacy node thickness, linear
 * thermodynamics): T and S are (nx, ny, nz) float32 device arrays.  Writes
 * out[8] = mean_T, mean_S, mean_T_top, mean_S_top, heat_content_J,
 * salt_content_kg, total_volume_m3, mean_depth_m.  The sums are float64 with
 * compensation (Neumaier per thread, double-double across threads) in a fixed
 * order, so repeated calls agree bit for bit.  Synchronizes the stream. */
int zm_budgets(zm_solver* s, void* stream, const float* T, const float* S, double rho0, double cp, double* out);

/* Classify a float32 state held in the caller's device arrays (reference
 * layout) without allocating any device memory.  No counterpart in the
 * reference: its classify_state (runtime/monitor.py:20-30) runs inside JAX,
 * which owns all device memory.  This is for callers that cannot call
 * cudaMalloc: a runtime whose memory pool already holds the GPU (XLA
 * preallocates most of it), a check made after a blow-up exhausted that pool,
 * or a coupler working within a fixed memory budget.
 *
 * ice is the (nx, ny) ice field or NULL (the reference's scalar default).
 * metrics (host, 4 floats): max |u|, max(|u|, |v|), max |eta|, like jnp.max:
 * NaN when the field holds a NaN, +-inf counted as inf; then 1 if every value
 * of u, v, T, S, eta and ice is finite, else 0.  *code: 0 accepted,
 * 1 non-finite, 3 velocity above velocity_limit, 4 |eta| above eta_limit
 * (>= with inclusive != 0).  The call waits for its result on the host, so a
 * stream that is capturing is refused with ZM_ERR_INVALID.
 *
 * Its only scratch is a fixed ZM_NOALLOC_SCRATCH_BYTES array inside the
 * library, held by every GPU that loads it until exit; each call looks up the
 * array's device address for the current device.  Fields of more than
 * ZM_NOALLOC_MAX_POINTS points are rejected with ZM_ERR_INVALID.  All calls on
 * a device share the array: calls whose work overlaps on the GPU race, so
 * order them. */
#define ZM_NOALLOC_SCRATCH_BYTES 33024
#define ZM_NOALLOC_MAX_POINTS 134217728LL
int zm_classify_state_noalloc(void* stream, int32_t nx, int32_t ny, int32_t nz, const float* u, const float* v,
                              const float* T, const float* S, const float* eta, const float* ice,
                              float velocity_limit, float eta_limit, int32_t inclusive, float* metrics,
                              int32_t* code);

/* Message of the last failure on this handle ("" if none). */
const char* zm_last_error(const zm_solver* s);

void zm_destroy(zm_solver* s);

#ifdef __cplusplus
}
#endif

#endif /* ZM_B200_H */

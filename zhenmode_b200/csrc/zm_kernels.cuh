// Declarations shared by the kernel translation units and the solver.
#pragma once

#include <cuda_bf16.h>

#include "zm_internal.cuh"

namespace zm {

// Programmatic dependent launch.  A kernel launched by launch_pdl may begin
// while the kernel before it on the stream (or in the captured graph)
// finishes its last blocks: its blocks run the set-up that reads only static
// arrays (grid metrics, masks, face gates), then pdl_wait(), which returns
// once the preceding grid has completed and its memory is visible.  Every
// kernel launched this way calls pdl_wait() before it reads or writes any
// array that a preceding kernel writes or reads.  pdl_trigger() lets the
// next kernel's launch begin once every block of this one has started.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... K, class... A>
inline cudaError_t launch_pdl(void (*kern)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<K>(args)...);
}

struct FftPlan {
  int n, nstages, keep;
  int radix[24];
  int tab_off[24];              // stage s: output bases at base_tab + tab_off[s] (n / R entries)
  int tw_off[24];               // stage s: twiddles at stage_tw + tw_off[s], [r - 1][butterfly]
  const int* base_tab;          // Stockham output base of each butterfly
  const float2* stage_tw;       // exp(-2 pi i (k r n / (ns R) mod n) / n) per butterfly and r >= 1
  const unsigned char* keepbin; // 1 where bin m survives the 2/3 rule, m < n
  // register-resident form for n = r1 r2 r3 (0 when n has no supported split)
  int r1, r2, r3;
  const float2* tw_full;        // exp(-2 pi i j / n), j < n (float64-derived)
};

struct PgfArgs {
  const float *T, *S, *u1, *v1, *Au, *Av, *Ppu, *Ppv;
  float *Pu, *Pv, *uo, *vo, *frx, *fry;
  float *gsx, *gsy;  // per-level gradient scratch (modes 1 and 2)
  float *Fxs, *Fys;  // depth-mean gradient per column (modes 1 and 2, 2-D)
  double *ubt0, *vbt0;
  float dt, bottom_decay;
  int mode;
};

struct RestArgs {
  const float *Tev, *Sev, *accT, *accS, *Tbase, *Sbase;
  float *dT1, *dS1, *To, *So;
  float dt, inv_na;
  int nc, stage;
  int no_conv;  // convective mixing carried by the learned closure instead
  float *convT, *convS;  // ledger mode: the convective tendency per point (null otherwise)
};

// momentum-advection tile rows (k_madv)
constexpr int MADV_TY = 60;
// tracer advection column tile (k_tracer_adv_t marches it down the levels)
constexpr int TA_X = 32, TA_Y = 8;
// temporally blocked nu_h subcycles: tile width, rows per thread, subcycles per pass
constexpr int NB_W = 64;
constexpr int NB_R = 8;
constexpr int NB_T = 6;

// persistent barotropic subcycle
#define ZM_BT_MAX_NB 64
#define ZM_BT_BARRIER_POLLS (1u << 24)
#define ZM_BT_ERR_BARRIER 1u
// barotropic tile of the resident kernel: owned cells, halo width, threads
constexpr int BT_TX = 32, BT_TY = 16, BT_H = 2, BT_THREADS = 128;
struct BtArgs {
  const double *eta0, *ubt0, *vbt0, *Fx, *Fy, *count;
  double *pub_e[2], *pub_u[2], *pub_v[2];  // published fields by subcycle parity
  double *ubt_out, *vbt_out;
  double *part_e[2], *part_u[2], *part_v[2];
  float* eta_out;
  const float* wts;
  unsigned *bar, *err;
  int ntx, nb, nsub, cap_active;
  double dtH, dtb, drag;
  // lateral sponge and eta relaxation (barotropic.py:22-41); off when the flags are 0
  int sponge, relax;
  const double *es, *er;     // exp(-sponge_rate dt_bt), exp(-eta_relax_rate dt_bt mask)
  const double* area;        // dx dy
  double ocean;              // max(sum area wet, 1)
  double *part_s[2], *part_r[2];  // per-block refill partials by subcycle parity
};
size_t bt_tile_smem();
__global__ void k_bt_loop(Dev d, BtArgs a);
__global__ void k_bt_eta(Dev d, const double* eta, const double* ubt, const double* vbt, double* eta_o, double dtH);
__global__ void k_bt_vel(Dev d, const double* eta, const double* ubt, const double* vbt, const double* Fx,
                         const double* Fy, double* ubt_o, double* vbt_o, double dtb, double drag, const double* sv);
__global__ void k_refill_part(Dev d, const double* eta, const double* fac, const double* area, double* part);
__global__ void k_refill_apply(Dev d, double* eta, const double* fac, const double* part, int nparts, double ocean);
__global__ void k_sponge(Dev d, float* u, float* v, float* T, float* S, const float* dec, const float* Tc,
                         const float* Sc);
__global__ void k_cap2d(Dev d, double* f0, double* f1, const float* wts, const double* count, int nb_rows);
__global__ void k_eta_to_float(Dev d, const double* e64, float* e32);
// per-column MLP of the learned closure (zm_mlp.cu); BF16 weights [out][in]
struct MlpBf16 {
  const __nv_bfloat16 *W1, *W2, *W3;
  const float *b1, *b2, *b3;
};
size_t mlp_tc_smem();
// learned closure in the step: features of a column, the plain closure per
// interface, and the fused tensor-core inference writing kappa per interface
struct ClosureArgs {
  const float *T, *S, *u, *v;   // internal layout; T, S as anomalies
  float* kappa3;                // [nz-1][ny][P] diffusivity per interface (fused kernel)
  float *X, *Tt, *Mt;           // features [ncol][256], targets and mask [ncol][64] (features kernel)
  unsigned* fallback;           // columns that took the plain closure
  float bound;                  // largest |feature| the network is trusted with
};
__global__ void k_closure_features(Dev d, ClosureArgs a);
__global__ void k_mlp_closure(MlpBf16 w, Dev d, ClosureArgs a, unsigned* err);
__global__ void k_kappa_rows(Dev d, const float* kap3, float* out);
// diagnostics outside the step (zm_diagnostics.cu)
#define ZM_BUDGET_SUMS 7
__global__ void k_diagnostics(Dev d, const float* T, const float* S, const float* eta, const float* Fz,
                              const float* sp, float* rho, float* pres, float* w);
__global__ void k_budget_partials(Dev d, const float* T, const float* S, const double* area, const double* width,
                                  double* partial);
__global__ void k_budget_final(const double* partial, int nblocks, double* out);
__global__ void k_forcing_blend(Dev d, const float* stack, int prev, int cur, int next, float w_prev, float w_cur,
                                float w_next, float* out);
__global__ void k_barrier_probe(unsigned* bar, unsigned* err, unsigned expected, unsigned max_polls);
// the temporally blocked nu_h subcycles with 8 or 16 warps per tile (NB_W x 8 warps * NB_R)
cudaError_t launch_nu_tb(cudaStream_t s, const Dev& d, int warps, const float* u, const float* v, float* uo,
                         float* vo, float c, int nsub, int halo);
__global__ void k_nu_gates(Dev d, unsigned char* gate);
void launch_lin_t(cudaStream_t s, const Dev& d, const float* usub, const float* vsub, const float* u0,
                  const float* v0, const float* T0, const float* S0, float* uo, float* vo, float* To, float* So,
                  float dth, int implicit_v);
// threads per block of k_implicit_vdiff (two per column) and its launch
constexpr int IV_T = 64;
void launch_implicit_vdiff(cudaStream_t s, const Dev& d, float* u, float* v, float* T, float* S, const float* u0,
                           const float* v0, const float* T0, const float* S0, float dth, const float* kap3);
void launch_fz(cudaStream_t s, const Dev& d, const float* u, const float* v, float* Fz);
void launch_tracer_terms(cudaStream_t s, const Dev& d, const float* T, const float* S, const float* u,
                         const float* v, const float* Fz, float* adv, float* dh, float* dv, float* conv);
__global__ void k_madv(Dev d, const float* u, const float* v, const float* Fz, float* Ayu, float* Ayv);
__global__ void k_dealias_lon(Dev d, FftPlan plan, const float* Ayu, const float* Ayv, float* Au, float* Av,
                              int lines_per_block);
// the longitude dealias filter: the register-resident kernel when the plan
// has a split of nx, else the shared-memory Stockham kernel; `lines` lines per
// block (the register form takes at most 4), stockham_smem its shared memory
cudaError_t launch_dealias(cudaStream_t s, const Dev& d, const FftPlan& plan, const float* Ayu, const float* Ayv,
                           float* Au, float* Av, int lines, size_t stockham_smem, bool pdl);
// the (r1, r2, r3) split of n the register-resident filter supports, or false
bool fft_reg_split(int n, int& r1, int& r2, int& r3);
void launch_tracer_adv(cudaStream_t s, const Dev& d, const float* T, const float* S, const float* u, const float* v,
                       const float* Fz, float* accT, float* accS, float* Tn, float* Sn, float dts, int first, int last,
                       float* topT, float* topS);
void launch_tracer_rest(dim3 g, dim3 b, cudaStream_t s, const Dev& d, const RestArgs& a);
void launch_pgf(cudaStream_t s, const Dev& d, const PgfArgs& a);
__global__ void k_bt_forcing(Dev d, const float* frx, const float* fry, double* Fx, double* Fy, const float* eta32,
                             double* eta64);
__global__ void k_cap3_means(Dev d, const float* u, const float* v, const float* T, const float* S, const double* ubt,
                             const double* ubt0, const double* vbt, const double* vbt0, float* means, int nb_rows);
__global__ void k_final(Dev d, const float* u3, const float* v3, const float* T3, const float* S3, const double* ubt,
                        const double* ubt0, const double* vbt, const double* vbt0, const float* u0, const float* v0,
                        const float* T0, const float* S0, const float* means, const float* wts, int nb_rows,
                        float* uo, float* vo, float* To, float* So);
// column-divergence projection of the stage-2 advective velocity (zm_projection.cu)
constexpr int PJ_THREADS = 1024;
#define ZM_PJ_SUMS 4
struct ProjArgs {
  const double* cx;     // [3][ny][P] weights of D_{i-1}, D_i, D_{i+1} in the east-face column flux
  const double* cy;     // [3][ny][P] weights of E_{j-1}, E_j, E_{j+1} in the north-face column flux
  const double* sxy;    // [2][ny][P] area / dx, area / (dy cos)
  const double* minv;   // Jacobi inverse diagonal [ny][P], or null (no preconditioner)
  const double* rarea;  // 1 / area on wet columns, 0 elsewhere
  const double* b;      // right-hand side -(coldiv / (dt g)) area
  double *psi, *x, *r, *z, *p0, *p1, *Ap;
  double* part;         // [blocks][ZM_PJ_SUMS] block partial sums
  unsigned *bar, *err;
  int* stats;           // iterations of each solve (3), refinement solves run
  double* norms;        // ledger mode: squared surface-transport norms before / after (null otherwise)
  double tol2, trtol2;  // tol^2, transport rtol^2
  double dtg;           // dt g
  int niter, refinements;
};
__global__ void k_proj_coef(Dev d, const double* dzn, const double* cosd, const double* area, double* cx, double* cy,
                            double* sxy, double* minv, double* rarea);
__global__ void k_proj_rhs(Dev d, const float* u, const float* v, const double* dzn, const double* cosd,
                           const double* area, double dtg, double* b);
__global__ void k_proj_cg(Dev d, ProjArgs a);
__global__ void k_proj_correct(Dev d, float* u, float* v, const double* psi, const double* cosd, double dtg);
// FP64 stage/source ledger of one step (diagnostics/budgets.py:62-288), zm_ledger.cu.
// Accumulator layout (doubles) of zm_ledger_step, documented in zm_b200.h.
#define ZM_LED_STAGE 0      // [6][3] stage changes (heat J, salt kg, volume m^3)
#define ZM_LED_SCALE 18     // [3] summed magnitudes of the stage changes
#define ZM_LED_SOURCE 21    // [9][3] source inputs
#define ZM_LED_PROC 48      // [4][3] nonlinear process changes
#define ZM_LED_PSCALE 60    // [3] their summed magnitudes
#define ZM_LED_ADVB 63      // [3] advective flux through the surface
#define ZM_LED_PROJ 66      // squared transport norms before/after the projection, worst ratio
#define ZM_LED_OBS 69       // [3] observed change over the step
#define ZM_LED_DISP 72      // [3] eta * surface tracer change
#ifndef ZM_LED_COUNT
#define ZM_LED_COUNT 75
#endif
constexpr int LED_Q = 16;   // sums per reduction at most
struct LedFold {
  int dst[LED_Q];           // accumulator index of each sum, -1 to drop it
  double scale[LED_Q];      // factor applied to the sum before it is added
};
__global__ void k_led_diff(Dev d, const float* Tb, const float* Sb, const float* eb, const float* Ta, const float* Sa,
                           const float* ea, const double* area, const double* dzn, double* part);
__global__ void k_led_rk(Dev d, const float* Tev, const float* Sev, const float* accT, const float* accS,
                         const float* topT, const float* topS, const float* convT, const float* convS, const float* Fz,
                         float inv_na, const double* area, const double* dzn, double* part);
__global__ void k_led_sponge(Dev d, const float* Tb, const float* Sb, const float* dec, const float* Tc,
                             const float* Sc, const double* area, const double* dzn, double* part);
__global__ void k_led_disp(Dev d, const float* eb, const float* Tb, const float* Sb, const float* ea, const float* Ta,
                           const float* Sa, const double* area, double* part);
__global__ void k_led_fold(const double* part, int nblocks, int nq, LedFold f, double* acc);
__global__ void k_led_proj(const double* norms, double* acc);
__global__ void k_ref_to_int3(Dev d, const float* src, float* dst, float offset);
__global__ void k_int_to_ref3(Dev d, const float* src, float* dst, float offset);
__global__ void k_ref_to_int2(Dev d, const float* src, float* dst);
__global__ void k_int_to_ref2(Dev d, const float* src, float* dst);
__global__ void k_monitor(Dev d, const float* u, const float* v, const float* T, const float* S, const float* eta,
                          float umax, float etamax, unsigned int* flags);

}  // namespace zm

// Internal device structures of the B200 global ocean step.
//
// Layout: every 3-D field is float32 [nz][ny][P] (longitude fastest, row pitch
// P >= nx, P % 4 == 0); 2-D fields are [ny][P].  The reference's (nx, ny, nz)
// C-order arrays are converted only at the C-ABI boundary.
//
// Temperature and salinity are stored as anomalies T - T_ref and S - S_ref
// (converted at the boundary).  Every operator of the step is linear and
// shift-invariant in the tracers (diffusion, flux-form advection with the
// exact discrete continuity inverse, convection, the linear EOS, restoring
// toward shifted targets), so this is the same arithmetic as the reference
// with ~100x finer float32 resolution on salinity (|S - 35| < 1 instead of 35).
//
// The 3-D wet mask is one 64-bit word per column (bit k = level k is wet), so
// nz <= 64.  The ghost-fill level of a column (the deepest wet level,
// numerics/vertical.py:122-135) is the index of its highest set bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define ZM_MAXZ 64

namespace zm {

constexpr float kG = 9.81f;
constexpr float kRho0 = 1025.0f;
constexpr float kAlpha = 2.0e-4f;
constexpr float kBeta = 7.6e-4f;
constexpr float kCp = 3992.0f;

// Per-level coefficients of the non-uniform vertical grid, passed by value.
struct Vert {
  float dz_node[ZM_MAXZ];      // node-cell thickness (nz)
  float inv_dz_node[ZM_MAXZ];
  float inv_dz_iface[ZM_MAXZ]; // 1/|z[k]-z[k+1]| (nz-1)
  float dz3d[ZM_MAXZ];         // layer thickness grid.dz (nz-1)
  float dznorm[ZM_MAXZ];       // dz / H_sw (nz-1)
  float d2_lo[ZM_MAXZ];        // d2/dz2 weight of node k-1 (interior k)
  float d2_hi[ZM_MAXZ];        // d2/dz2 weight of node k+1 (interior k)
  float ddz_inv[ZM_MAXZ];      // 1/(z[k+1]-z[k-1]); ends one-sided
  float d2_top, d2_bot;        // 2/h^2 of the zero-flux end rows
};

// Everything a kernel reads about the grid and physics.
struct Dev {
  int nx, ny, nz, P;
  long long plane;             // ny * P
  // per latitude row (ny)
  const float* cosl;
  const float* inv_cos;
  const float* cfp;            // 0.5 (cos[j] + cos[j+1 mod ny])
  const float* cfm;            // 0.5 (cos[j] + cos[j-1 mod ny])
  const float* tanR;           // tan(lat)/R from f[0,:]
  // 2-D [ny][P]
  const float* inv_dx;
  const float* inv_dx2;
  const float* fcor;
  const float* rot_c;          // cos(f dt/2)
  const float* rot_s;          // sin(f dt/2)
  const float* wet2;           // 2-D wet mask (barotropic mode)
  const uint64_t* wbits;       // 3-D wet mask, one word per column
  const unsigned char* nu_gate; // 3-D [nz][ny][P] face gates of the nu_h Laplacian (k_nu_gates)
  const float* kh2;            // kappa_h + coastal kappa_h
  const float* kv2;            // kappa_v + coastal kappa_v
  const float* tau_x;
  const float* tau_y;
  const float* qheat;
  const float* tatm;           // bulk target T_atm (zero unless bulk is on)
  const float* cbulk;          // coastal bulk lambda
  const float* rest_c;         // coastal restore coefficient (1/s)
  const float* rest_T;         // coastal restore target
  const float* sref;           // SSS restore target
  const double* inv_dx_d;      // double copies for the barotropic mode
  const double* fcor_d;
  // scalars
  float inv_dy, inv_dy2;
  double inv_dy_d;
  float nu_h, nu_v, nu_bi, kappa_bi, kappa_conv;
  float r_bot, T_ref, S_ref, H_sw, dz_surface;
  float lambda_bulk, restore_S, ice_salt, ice_freeze;
  int localize_conv, limiter;  // limiter: 0 centered, 1 donor cell, 2 minmod (fct)
  int conservative_kv;
  // launch shapes that change no result (chosen by the autotuner): levels per
  // block of the tracer-advection and linear-step column marches, tile rows
  // of the pressure-gradient and vertical-transport marches
  int ta_kc, lt_kc, pg_rows, fz_rows;
  Vert vc;
};

__device__ __forceinline__ long long idx3(const Dev& d, int k, int j, int i) {
  return (long long)k * d.plane + (long long)j * d.P + i;
}
__device__ __forceinline__ int idx2(const Dev& d, int j, int i) { return j * d.P + i; }
__device__ __forceinline__ int east(const Dev& d, int i) { return i + 1 == d.nx ? 0 : i + 1; }
__device__ __forceinline__ int west(const Dev& d, int i) { return i == 0 ? d.nx - 1 : i - 1; }
__device__ __forceinline__ int north(const Dev& d, int j) { return j + 1 < d.ny ? j + 1 : d.ny - 1; }
__device__ __forceinline__ int south(int j) { return j > 0 ? j - 1 : 0; }
__device__ __forceinline__ float wetf(uint64_t bits, int k) { return (float)((bits >> k) & 1ull); }
__device__ __forceinline__ bool wetb(uint64_t bits, int k) { return (bits >> k) & 1ull; }
__device__ __forceinline__ int kbot_of(uint64_t bits) { return bits ? 63 - __clzll((long long)bits) : 0; }
__device__ __forceinline__ uint64_t wb(const Dev& d, int j, int i) { return __ldg(d.wbits + idx2(d, j, i)); }
__device__ __forceinline__ float ld(const float* p, long long i) { return __ldg(p + i); }

// Linear equation of state (physics/eos.py:13-18).  Tracers are held on the
// device as anomalies from (T_ref, S_ref), so rho' needs no subtraction.
__device__ __forceinline__ float rho_anom(float Ta, float Sa) {
  return kRho0 * (-kAlpha * Ta + kBeta * Sa);
}

}  // namespace zm

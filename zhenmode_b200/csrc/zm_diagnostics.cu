// Diagnostics of a state, outside the time step.
//
// k_diagnostics: the diagnostics closure of the reference factory
// (factory.py:752-760) on one column per thread: full density rho0 + rho'
// (physics/eos.py:13-18), hydrostatic pressure rho0 g eta (+ a surface load)
// plus the trapezoid integral of the wet-masked density anomaly
// (dynamics/pressure.py:32-42, 62-74), and the dual-face vertical velocity
// w = -Fz[k] wet (dynamics/transport.py:149-166), with Fz from k_fz.
//
// k_budget_partials / k_budget_final: the global heat, salt and volume
// snapshot of diagnostics/snapshot.py:67-128 (legacy node thickness), summed
// in float64 with compensation.  Each lane keeps a Neumaier sum over its
// elements; lanes, warps and blocks are combined as double-double values
// (TwoSum), and the per-block partials are folded by one block in block
// order, so the result is the same on every run.
#include "zm_dd.cuh"
#include "zm_kernels.cuh"

namespace zm {

__global__ void __launch_bounds__(128) k_diagnostics(Dev d, const float* __restrict__ T, const float* __restrict__ S,
                                                     const float* __restrict__ eta, const float* __restrict__ Fz,
                                                     const float* __restrict__ sp, float* __restrict__ rho,
                                                     float* __restrict__ pres, float* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const long long base = idx2(d, j, i);
  const uint64_t bits = __ldg(d.wbits + base);
  float p_bt = kRho0 * kG * ld(eta, base);
  if (sp) p_bt = p_bt + ld(sp, base);
  float p_bc = 0.f, r_prev = 0.f;
  for (int k = 0; k < d.nz; ++k) {
    const long long id = (long long)k * d.plane + base;
    const float r = rho_anom(ld(T, id), ld(S, id));
    const float wk = wetf(bits, k);
    const float rw = r * wk;
    if (k > 0) p_bc += kG * (0.5f * (r_prev + rw)) * d.vc.dz3d[k - 1];
    rho[id] = kRho0 + r;
    pres[id] = p_bt + p_bc;
    w[id] = -ld(Fz, id) * wk;
    r_prev = rw;
  }
}


// sums: 0 wet volume, 1 T volume, 2 S volume, 3 wet surface area,
// 4 T_top surface area, 5 S_top surface area, 6 total cell area.
__global__ void __launch_bounds__(256) k_budget_partials(Dev d, const float* __restrict__ T,
                                                         const float* __restrict__ S,
                                                         const double* __restrict__ area,
                                                         const double* __restrict__ width,
                                                         double* __restrict__ partial) {
  __shared__ DD red[ZM_BUDGET_SUMS][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long ncol = (long long)d.nx * d.ny;
  DD acc[ZM_BUDGET_SUMS];
#pragma unroll
  for (int q = 0; q < ZM_BUDGET_SUMS; ++q) acc[q] = DD{0.0, 0.0};
  // one warp per column of the reference layout (nx, ny, nz): contiguous in z
  for (long long col = (long long)blockIdx.x * 8 + warp; col < ncol; col += (long long)gridDim.x * 8) {
    const int i = (int)(col / d.ny), j = (int)(col - (long long)i * d.ny);
    const double a = area[col];
    const uint64_t bits = __ldg(d.wbits + idx2(d, j, i));
    const float* Tc = T + col * d.nz;
    const float* Sc = S + col * d.nz;
    for (int k = lane; k < d.nz; k += 32) {
      const double vol = (a * width[k]) * (double)((bits >> k) & 1ull);
      neumaier(acc[0], vol);
      neumaier(acc[1], (double)Tc[k] * vol);
      neumaier(acc[2], (double)Sc[k] * vol);
    }
    if (lane == 0) {
      const double sa = a * (double)__ldg(d.wet2 + idx2(d, j, i));
      neumaier(acc[3], sa);
      neumaier(acc[4], (double)Tc[0] * sa);
      neumaier(acc[5], (double)Sc[0] * sa);
      neumaier(acc[6], a);
    }
  }
#pragma unroll
  for (int q = 0; q < ZM_BUDGET_SUMS; ++q) {
    DD x = two_sum(acc[q].hi, acc[q].lo);
    for (int o = 16; o > 0; o >>= 1) x = dd_add(x, shfl_dd(x, o));
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < ZM_BUDGET_SUMS) {
    DD x = red[threadIdx.x][0];
    for (int w = 1; w < 8; ++w) x = dd_add(x, red[threadIdx.x][w]);
    partial[(blockIdx.x * ZM_BUDGET_SUMS + threadIdx.x) * 2] = x.hi;
    partial[(blockIdx.x * ZM_BUDGET_SUMS + threadIdx.x) * 2 + 1] = x.lo;
  }
}

__global__ void k_budget_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
  const int q = threadIdx.x;
  if (q >= ZM_BUDGET_SUMS) return;
  DD x{0.0, 0.0};
  for (int b = 0; b < nblocks; ++b)
    x = dd_add(x, DD{partial[(b * ZM_BUDGET_SUMS + q) * 2], partial[(b * ZM_BUDGET_SUMS + q) * 2 + 1]});
  out[2 * q] = x.hi;
  out[2 * q + 1] = x.lo;
}

}  // namespace zm

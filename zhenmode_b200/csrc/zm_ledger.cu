// FP64 stage/source ledger of one step (the budget audit of
// diagnostics/budgets.py:62-288, legacy mode-split path).
//
// Each kernel walks the columns (one per thread, 32 x 8 blocks), keeps a
// Neumaier sum per quantity, and writes its block's double-double partial;
// k_led_fold adds the partials in block order, times a per-quantity factor,
// into the accumulator of zm_ledger_step (layout ZM_LED_* in zm_kernels.cuh).
// The factors rho0 cp, rho0 / 1000 and the interval dt / 2 are applied to the
// sums, not per point.  Tracers are anomalies from (T_ref, S_ref); every
// quantity here is a difference of tracers except the surface advective flux
// Fz[0] c[0] and eta c[0], which use the absolute values.
#include "zm_dd.cuh"
#include "zm_kernels.cuh"

namespace zm {

namespace {

constexpr int LED_THREADS = 256;

template <int NQ>
__device__ void led_block(DD (&acc)[NQ], double* part) {
  __shared__ DD red[NQ][LED_THREADS / 32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    DD x = two_sum(acc[q].hi, acc[q].lo);
    for (int o = 16; o > 0; o >>= 1) x = dd_add(x, shfl_dd(x, o));
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (tid < NQ) {
    DD x = red[tid][0];
    for (int w = 1; w < LED_THREADS / 32; ++w) x = dd_add(x, red[tid][w]);
    const long long b = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    part[(b * NQ + tid) * 2] = x.hi;
    part[(b * NQ + tid) * 2 + 1] = x.lo;
  }
}

template <int NQ>
__device__ __forceinline__ void led_zero(DD (&acc)[NQ]) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = DD{0.0, 0.0};
}

}  // namespace

// Stage change between two states (budgets.py:122-141): sums of dT vol,
// dS vol, d(eta) area (eta pointers may be null) and of their magnitudes.
__global__ void __launch_bounds__(LED_THREADS) k_led_diff(Dev d, const float* __restrict__ Tb,
                                                          const float* __restrict__ Sb, const float* __restrict__ eb,
                                                          const float* __restrict__ Ta, const float* __restrict__ Sa,
                                                          const float* __restrict__ ea,
                                                          const double* __restrict__ area,
                                                          const double* __restrict__ dzn, double* __restrict__ part) {
  DD acc[6];
  led_zero(acc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) {
    const int g = idx2(d, j, i);
    const uint64_t bits = wb(d, j, i);
    const double ar = area[g];
    for (int k = 0; k < d.nz; ++k) {
      if (!wetb(bits, k)) continue;
      const long long id = (long long)k * d.plane + g;
      const double vol = ar * dzn[k];
      const double h = ((double)Ta[id] - (double)Tb[id]) * vol;
      const double sl = ((double)Sa[id] - (double)Sb[id]) * vol;
      neumaier(acc[0], h);
      neumaier(acc[1], sl);
      neumaier(acc[3], fabs(h));
      neumaier(acc[4], fabs(sl));
    }
    if (ea) {
      const double v = ((double)ea[g] - (double)eb[g]) * (ar * (double)__ldg(d.wet2 + g));
      neumaier(acc[2], v);
      neumaier(acc[5], fabs(v));
    }
  }
  led_block(acc, part);
}

// One RK2 tracer residual (tendencies.py:211-214): advection (mean rate over
// the substeps) and convection per point, the six surface sources at the top
// level, and the surface advective flux Fz[0] c[0] (mean over the substeps).
//  0..3 adv T, |adv T|, adv S, |adv S|     4..7 conv likewise
//  8..11 heat sources: prescribed, bulk, coastal bulk, coastal restore
//  12, 13 salt sources: SSS restore, brine     14, 15 surface flux T, S
__global__ void __launch_bounds__(LED_THREADS) k_led_rk(Dev d, const float* __restrict__ Tev,
                                                        const float* __restrict__ Sev,
                                                        const float* __restrict__ accT, const float* __restrict__ accS,
                                                        const float* __restrict__ topT, const float* __restrict__ topS,
                                                        const float* __restrict__ convT,
                                                        const float* __restrict__ convS, const float* __restrict__ Fz,
                                                        float inv_na, const double* __restrict__ area,
                                                        const double* __restrict__ dzn, double* __restrict__ part) {
  DD acc[16];
  led_zero(acc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) {
    const int g = idx2(d, j, i);
    const uint64_t bits = wb(d, j, i);
    const double ar = area[g];
    for (int k = 0; k < d.nz; ++k) {
      if (!wetb(bits, k)) continue;
      const long long id = (long long)k * d.plane + g;
      const double vol = ar * dzn[k];
      const double aT = (double)(accT[id] * inv_na) * vol, aS = (double)(accS[id] * inv_na) * vol;
      const double cT = (double)convT[id] * vol, cS = (double)convS[id] * vol;
      neumaier(acc[0], aT);
      neumaier(acc[1], fabs(aT));
      neumaier(acc[2], aS);
      neumaier(acc[3], fabs(aS));
      neumaier(acc[4], cT);
      neumaier(acc[5], fabs(cT));
      neumaier(acc[6], cS);
      neumaier(acc[7], fabs(cS));
    }
    if (wetb(bits, 0)) {
      const double vol0 = ar * dzn[0];
      const double sst = Tev[g], sss = Sev[g];
      const double hf = 1.0 / ((double)d.dz_surface * 1025.0 * 3992.0);
      const double ta = (double)__ldg(d.tatm + g);
      neumaier(acc[8], (double)__ldg(d.qheat + g) * hf * vol0);
      neumaier(acc[9], (double)d.lambda_bulk * (ta - sst) * hf * vol0);
      neumaier(acc[10], (double)__ldg(d.cbulk + g) * (ta - sst) * hf * vol0);
      neumaier(acc[11], (double)__ldg(d.rest_c + g) * ((double)__ldg(d.rest_T + g) - sst) * vol0);
      neumaier(acc[12], (double)d.restore_S * ((double)__ldg(d.sref + g) - sss) * vol0);
      neumaier(acc[13], (Tev[g] <= d.ice_freeze ? (double)d.ice_salt : 0.0) * vol0);
    }
    const double sa = ar * (double)__ldg(d.wet2 + g);
    const double fz0 = Fz[g];
    neumaier(acc[14], ((double)(topT[g] * inv_na) + (double)d.T_ref * fz0) * sa);
    neumaier(acc[15], ((double)(topS[g] * inv_na) + (double)d.S_ref * fz0) * sa);
  }
  led_block(acc, part);
}

// Sponge of one linear half step from the state before it (budgets.py:196-204
// and the "sponge" stage): 0, 1 the sources sum (C_clim - C)(1 - decay) vol;
// 2, 3 the stage change of the update that k_sponge applies, 4, 5 its magnitudes.
__global__ void __launch_bounds__(LED_THREADS) k_led_sponge(Dev d, const float* __restrict__ Tb,
                                                            const float* __restrict__ Sb,
                                                            const float* __restrict__ dec,
                                                            const float* __restrict__ Tc,
                                                            const float* __restrict__ Sc,
                                                            const double* __restrict__ area,
                                                            const double* __restrict__ dzn, double* __restrict__ part) {
  DD acc[6];
  led_zero(acc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) {
    const int g = idx2(d, j, i);
    const uint64_t bits = wb(d, j, i);
    const double ar = area[g];
    const float q = ld(dec, g);
    const double frac = 1.0 - (double)q;
    for (int k = 0; k < d.nz; ++k) {
      if (!wetb(bits, k)) continue;
      const long long id = (long long)k * d.plane + g;
      const double vol = ar * dzn[k];
      const float tb = Tb[id], sb = Sb[id], tc = ld(Tc, id), sc = ld(Sc, id);
      const float ta = tc + (tb - tc) * q, sa = sc + (sb - sc) * q;  // as k_sponge
      neumaier(acc[0], ((double)tc - (double)tb) * frac * vol);
      neumaier(acc[1], ((double)sc - (double)sb) * frac * vol);
      const double h = ((double)ta - (double)tb) * vol, sl = ((double)sa - (double)sb) * vol;
      neumaier(acc[2], h);
      neumaier(acc[3], sl);
      neumaier(acc[4], fabs(h));
      neumaier(acc[5], fabs(sl));
    }
  }
  led_block(acc, part);
}

// eta times the surface tracers, after minus before (budgets.py:185-194).
__global__ void __launch_bounds__(LED_THREADS) k_led_disp(Dev d, const float* __restrict__ eb,
                                                          const float* __restrict__ Tb, const float* __restrict__ Sb,
                                                          const float* __restrict__ ea,
                                                          const float* __restrict__ Ta, const float* __restrict__ Sa,
                                                          const double* __restrict__ area, double* __restrict__ part) {
  DD acc[2];
  led_zero(acc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) {
    const int g = idx2(d, j, i);
    const double sa = area[g] * (double)__ldg(d.wet2 + g);
    const double tr = d.T_ref, sr = d.S_ref;
    const double e1 = ea[g], e0 = eb[g];
    neumaier(acc[0], (e1 * ((double)Ta[g] + tr) - e0 * ((double)Tb[g] + tr)) * sa);
    neumaier(acc[1], (e1 * ((double)Sa[g] + sr) - e0 * ((double)Sb[g] + sr)) * sa);
  }
  led_block(acc, part);
}

// Partials of one reduction in block order, scaled, added to the accumulator.
// Several sums may go to one slot: one thread adds them in their order.
__global__ void k_led_fold(const double* __restrict__ part, int nblocks, int nq, LedFold f, double* __restrict__ acc) {
  __shared__ double sum[LED_Q];
  const int q = threadIdx.x;
  if (q < nq) {
    DD x{0.0, 0.0};
    for (int b = 0; b < nblocks; ++b)
      x = dd_add(x, DD{part[((long long)b * nq + q) * 2], part[((long long)b * nq + q) * 2 + 1]});
    sum[q] = x.hi + x.lo;
  }
  __syncthreads();
  if (q == 0)
    for (int r = 0; r < nq; ++r)
      if (f.dst[r] >= 0) acc[f.dst[r]] += f.scale[r] * sum[r];
}

// Column-projection norms of one step into the accumulator (budgets.py:175-183).
__global__ void k_led_proj(const double* __restrict__ norms, double* __restrict__ acc) {
  if (threadIdx.x != 0) return;
  const double n0 = norms[0], n1 = norms[1];
  acc[ZM_LED_PROJ] += n0;
  acc[ZM_LED_PROJ + 1] += n1;
  const double rel = n0 > 0.0 ? sqrt(n1 / n0) : (n1 == 0.0 ? 0.0 : INFINITY);
  acc[ZM_LED_PROJ + 2] = fmax(acc[ZM_LED_PROJ + 2], rel);
}

}  // namespace zm

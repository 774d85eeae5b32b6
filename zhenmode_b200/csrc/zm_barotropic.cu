// Barotropic subcycle of the mode-split step (dynamics/barotropic.py:86-265,
// legacy branch; _subcycle of timestepping/subcycles.py:6-26).
//
// Resident path (k_bt_loop): one cooperative kernel runs all subcycles.  Each
// block owns one BT_TX x BT_TY tile and keeps its float64 state (eta, ubt,
// vbt) plus the static fields it stencils over (wet mask, 1/dx) in shared
// memory, with a two-cell halo, and the forcing and Coriolis parameter of its
// owned cells, for the whole loop.  Per subcycle:
//   1  refresh the halo from the neighbours' published values of the previous
//      subcycle (and apply the polar cap to the velocities);
//   2  continuity eta* = (eta - dt H div(ubt wm, vbt wm)) wm on the tile and,
//      redundantly, on its one-cell ring, so the gradient needs no exchange;
//   3  (cap active only) publish band-row partial sums, grid barrier, cap eta*;
//   4  momentum: adjoint gradient of eta*, u* = ubt + dt (-g grad eta* + F),
//      backward-Euler Coriolis, implicit drag, wet mask; publish eta*, u, v;
//   5  grid barrier.
// The polar cap (numerics/horizontal.py:387-451) needs the wet-point zonal mean
// of each band row; blocks write per-tile partial row sums and every reader
// folds them in tile order, so the result does not depend on timing.  When no
// band row has a wet point the cap is the identity and step 3 is skipped.
// Published fields and partial sums are double-buffered by subcycle parity.
//
// Streaming path (k_bt_eta / k_bt_vel / k_cap2d): for grids whose tiles cannot
// all be resident, three plain kernels per subcycle in the same arithmetic.
//
// Every grid barrier polls with a bounded count; if it runs out the kernel
// records ZM_BT_ERR_BARRIER in *err and every block returns.
#include "zm_kernels.cuh"
#include "zm_sync.cuh"

namespace zm {

namespace {

// band-row index of row j (0..2nb-1), or -1 outside the cap bands
__device__ __forceinline__ int band_of(int ny, int nb, int j) {
  if (nb <= 0) return -1;
  if (j < nb) return j;
  if (j >= ny - nb) return j - (ny - 2 * nb);
  return -1;
}

constexpr int BT_PX = BT_TX + 2 * BT_H, BT_PY = BT_TY + 2 * BT_H;

// Backward-Euler Coriolis with the implicit linear drag
// (barotropic.py:86-265): u = (u* + fd v*) drag / (1 + fd^2), fd = f dt_bt.
// The factor drag / (1 + fd^2) is static per cell; both paths form it here.
__device__ __forceinline__ double bt_drag_factor(double fd, double drag) { return drag / (1.0 + fd * fd); }

struct BtTile {
  double U[BT_PY][BT_PX], V[BT_PY][BT_PX];  // velocities (capped at the subcycle start)
  double E[BT_PY][BT_PX];                   // eta; overwritten in place by eta* on the tile + ring
  double ix[BT_PY][BT_PX];                  // 1/dx
  float w[BT_PY][BT_PX];                    // 2-D wet mask
  double cosl[BT_PY], cfp[BT_PY], cfm[BT_PY];
  double iyc[BT_PY];                        // 1/(dy cos(lat)) of the row
  double mean[3][2 * ZM_BT_MAX_NB];         // band-row means: eta*, u, v
  double red[BT_THREADS];
  double fx[BT_TY][BT_TX], fy[BT_TY][BT_TX];  // forcing of the owned cells
  double fd[BT_TY][BT_TX], rd[BT_TY][BT_TX];  // f dt and drag / (1 + (f dt)^2) of the owned cells
  int gj[BT_PY];                            // global row, -1 beyond the walls
  int gx[BT_PX];                            // global column (periodic wrap)
  unsigned char own_c[BT_PX];               // column owned by this block
};

// Continuity at padded cell (r, c); numerics/horizontal.py:69-97 flux form.
__device__ __forceinline__ double eta_new(const Dev& d, const BtArgs& a, const BtTile& t, int r, int c) {
  const int j = t.gj[r];
  const double w0 = t.w[r][c], we = t.w[r][c + 1], ww = t.w[r][c - 1];
  const double u0 = t.U[r][c] * w0, ue = t.U[r][c + 1] * we, uw = t.U[r][c - 1] * ww;
  const double fe = 0.5 * (u0 + ue) * (w0 * we);
  const double fw = 0.5 * (uw + u0) * (ww * w0);
  const double div_x = (fe - fw) * t.ix[r][c];
  const double v0 = t.V[r][c] * w0;
  double fn = 0.0, fs = 0.0;
  if (j < d.ny - 1) {
    const double wn = t.w[r + 1][c];
    fn = 0.5 * (v0 + t.V[r + 1][c] * wn) * (w0 * wn) * t.cfp[r];
  }
  if (j > 0) {
    const double ws = t.w[r - 1][c];
    fs = 0.5 * (t.V[r - 1][c] * ws + v0) * (ws * w0) * t.cfp[r - 1];
  }
  const double div = div_x + (fn - fs) * t.iyc[r];
  return (t.E[r][c] - a.dtH * div) * w0;
}

// wet-point partial sums of a padded tile field over the owned cells of each band row
__device__ void band_partials(const Dev& d, const BtArgs& a, BtTile& t, const double (*f)[BT_PX], double* part,
                              int xt) {
  for (int r = BT_H; r < BT_H + BT_TY; ++r) {
    const int j = t.gj[r];
    if (j < 0) continue;  // uniform over the block
    const int b = band_of(d.ny, a.nb, j);
    if (b < 0) continue;
    double s = 0.0;
    for (int c = BT_H + threadIdx.x; c < BT_H + BT_TX; c += blockDim.x)
      if (t.own_c[c]) s += f[r][c] * (double)t.w[r][c];
    t.red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) t.red[threadIdx.x] += t.red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[b * a.ntx + xt] = t.red[0];
    __syncthreads();
  }
}

__device__ void band_means(const BtArgs& a, BtTile& t, int q, const double* part) {
  for (int b = threadIdx.x; b < 2 * a.nb; b += blockDim.x) {
    double s = 0.0;
    for (int xt = 0; xt < a.ntx; ++xt) s += part[b * a.ntx + xt];
    t.mean[q][b] = s / a.count[b];
  }
}

// polar-cap blend of value f at row j with wet weight w
__device__ __forceinline__ double cap_val(const BtArgs& a, const BtTile& t, int ny, int q, int j, double w, double f) {
  const int b = band_of(ny, a.nb, j);
  if (b < 0) return f;
  const double wt = (double)a.wts[b < a.nb ? b : 2 * a.nb - 1 - b];
  return wt * (t.mean[q][b] * w) + (1.0 - wt) * (f * w);
}

// Decay of eta* by fac on the tile and its ring with the uniform refill of the
// removed volume (barotropic.py:22-31): the owned cells' sum of
// area (eta fac - eta) is published per block, and after a grid barrier every
// block folds the partials in block order.
__device__ bool refill(const Dev& d, const BtArgs& a, BtTile& t, const double* fac, double* part, unsigned nblocks) {
  const int tid = threadIdx.x, nt = blockDim.x;
  constexpr int NT = BT_TX * BT_TY;
  constexpr int NR = (BT_TX + 2) * (BT_TY + 2);
  double s = 0.0;
  for (int e = tid; e < NT; e += nt) {
    const int r = BT_H + e / BT_TX, c = BT_H + e % BT_TX;
    const int j = t.gj[r];
    if (j < 0 || !t.own_c[c]) continue;
    const int g = idx2(d, j, t.gx[c]);
    const double e0 = t.E[r][c];
    s += a.area[g] * (e0 * fac[g] - e0);
  }
  t.red[tid] = s;
  __syncthreads();
  for (int o = nt / 2; o > 0; o >>= 1) {
    if (tid < o) t.red[tid] += t.red[tid + o];
    __syncthreads();
  }
  if (tid == 0) part[blockIdx.x] = t.red[0];
  if (!grid_barrier(a.bar, a.err, nblocks, ZM_BT_BARRIER_POLLS)) return false;
  if (tid < 32) {
    double x = 0.0;
    for (unsigned b = tid; b < nblocks; b += 32) x += __ldcg(part + b);
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (tid == 0) t.red[0] = x;
  }
  __syncthreads();
  const double shift = -t.red[0] / a.ocean;
  for (int e = tid; e < NR; e += nt) {
    const int r = 1 + e / (BT_TX + 2), c = 1 + e % (BT_TX + 2);
    const int j = t.gj[r];
    if (j < 0) continue;
    const int g = idx2(d, j, t.gx[c]);
    t.E[r][c] = t.E[r][c] * fac[g] + shift * (double)t.w[r][c];
  }
  __syncthreads();
  return true;
}

}  // namespace

size_t bt_tile_smem() { return sizeof(BtTile); }

__global__ void __launch_bounds__(BT_THREADS, 4) k_bt_loop(Dev d, BtArgs a) {
  grid_barrier_begin(a.bar);
  extern __shared__ double bt_smem[];
  BtTile& t = *reinterpret_cast<BtTile*>(bt_smem);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int xt = blockIdx.x % a.ntx, yt = blockIdx.x / a.ntx;
  const int i0 = xt * BT_TX, j0 = yt * BT_TY;
  const unsigned nblocks = gridDim.x;
  const bool cap = a.cap_active != 0;
  constexpr int NC = BT_PX * BT_PY;
  constexpr int NR = (BT_TX + 2) * (BT_TY + 2);  // tile + one-cell ring
  constexpr int NT = BT_TX * BT_TY;
  // ---- geometry, static fields and the initial state on the padded tile
  for (int c = tid; c < BT_PX; c += nt) {
    const int gi = i0 - BT_H + c;
    t.gx[c] = ((gi % d.nx) + d.nx) % d.nx;
    t.own_c[c] = (c >= BT_H && c < BT_H + BT_TX && gi < d.nx) ? 1 : 0;
  }
  for (int r = tid; r < BT_PY; r += nt) {
    const int gj = j0 - BT_H + r;
    t.gj[r] = (gj < 0 || gj >= d.ny) ? -1 : gj;
    const int jc = gj < 0 ? 0 : (gj >= d.ny ? d.ny - 1 : gj);
    t.cosl[r] = (double)__ldg(d.cosl + jc);
    t.cfp[r] = (double)__ldg(d.cfp + jc);
    t.cfm[r] = (double)__ldg(d.cfm + jc);
    t.iyc[r] = d.inv_dy_d / t.cosl[r];
  }
  __syncthreads();
  for (int e = tid; e < NC; e += nt) {
    const int r = e / BT_PX, c = e - r * BT_PX;
    const int gj = t.gj[r];
    if (gj < 0) {  // beyond a closed wall: only ever multiplied by a zero mask
      t.U[r][c] = t.V[r][c] = t.E[r][c] = t.ix[r][c] = 0.0;
      t.w[r][c] = 0.f;
      continue;
    }
    const int g = idx2(d, gj, t.gx[c]);
    t.U[r][c] = a.ubt0[g];
    t.V[r][c] = a.vbt0[g];
    t.E[r][c] = a.eta0[g];
    t.w[r][c] = __ldg(d.wet2 + g);
    t.ix[r][c] = __ldg(d.inv_dx_d + g);
  }
  for (int e = tid; e < NT; e += nt) {
    const int r = e / BT_TX, c = e - r * BT_TX;
    const int gj = t.gj[r + BT_H];
    if (gj < 0 || !t.own_c[c + BT_H]) {
      t.fx[r][c] = t.fy[r][c] = t.fd[r][c] = t.rd[r][c] = 0.0;
      continue;
    }
    const int g = idx2(d, gj, t.gx[c + BT_H]);
    t.fx[r][c] = a.Fx[g];
    t.fy[r][c] = a.Fy[g];
    const double fd = __ldg(d.fcor_d + g) * a.dtb;
    t.fd[r][c] = fd;
    t.rd[r][c] = bt_drag_factor(fd, a.drag);
  }
  __syncthreads();
  const double g9 = 9.81;
  for (int n = 0; n < a.nsub; ++n) {
    const int pin = n & 1, pout = pin ^ 1;
    if (n > 0) {
      // 1: halo from the neighbours' published fields; caps on every cell
      if (cap) {
        band_means(a, t, 1, a.part_u[pin]);
        band_means(a, t, 2, a.part_v[pin]);
        __syncthreads();
      }
      for (int e = tid; e < NC; e += nt) {
        const int r = e / BT_PX, c = e - r * BT_PX;
        const int gj = t.gj[r];
        if (gj < 0) continue;
        const bool own = r >= BT_H && r < BT_H + BT_TY && t.own_c[c];
        if (own && !cap) continue;
        double u, v;
        if (own) {
          u = t.U[r][c];
          v = t.V[r][c];
        } else {
          const int g = idx2(d, gj, t.gx[c]);
          u = a.pub_u[pin][g];
          v = a.pub_v[pin][g];
          t.E[r][c] = a.pub_e[pin][g];
        }
        if (cap) {
          const double w = t.w[r][c];
          u = cap_val(a, t, d.ny, 1, gj, w, u);
          v = cap_val(a, t, d.ny, 2, gj, w, v);
        }
        t.U[r][c] = u;
        t.V[r][c] = v;
      }
      __syncthreads();
    }
    // 2: continuity on the tile and its ring; each cell reads its own eta only,
    // so eta* overwrites eta in place (after all threads computed)
    double en[(NR + BT_THREADS - 1) / BT_THREADS];
#pragma unroll
    for (int q = 0; q < (NR + BT_THREADS - 1) / BT_THREADS; ++q) {
      const int e = tid + q * BT_THREADS;
      en[q] = 0.0;
      if (e < NR) {
        const int r = 1 + e / (BT_TX + 2), c = 1 + e % (BT_TX + 2);
        if (t.gj[r] >= 0) en[q] = eta_new(d, a, t, r, c);
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < (NR + BT_THREADS - 1) / BT_THREADS; ++q) {
      const int e = tid + q * BT_THREADS;
      if (e < NR) {
        const int r = 1 + e / (BT_TX + 2), c = 1 + e % (BT_TX + 2);
        t.E[r][c] = en[q];
      }
    }
    __syncthreads();
    // 2b: lateral sponge, then eta relaxation, each with its volume refill
    if (a.sponge && !refill(d, a, t, a.es, a.part_s[pout], nblocks)) return;
    if (a.relax && !refill(d, a, t, a.er, a.part_r[pout], nblocks)) return;
    // 3: polar cap of eta*
    if (cap) {
      band_partials(d, a, t, t.E, a.part_e[pout], xt);
      if (!grid_barrier(a.bar, a.err, nblocks, ZM_BT_BARRIER_POLLS)) return;
      band_means(a, t, 0, a.part_e[pout]);
      __syncthreads();
      for (int e = tid; e < NR; e += nt) {
        const int r = 1 + e / (BT_TX + 2), c = 1 + e % (BT_TX + 2);
        if (t.gj[r] >= 0) t.E[r][c] = cap_val(a, t, d.ny, 0, t.gj[r], t.w[r][c], t.E[r][c]);
      }
      __syncthreads();
    }
    // 4: momentum on the owned cells; publish eta*, u, v
    for (int e = tid; e < NT; e += nt) {
      const int r = BT_H + e / BT_TX, c = BT_H + e % BT_TX;
      const int j = t.gj[r];
      if (j < 0 || !t.own_c[c]) continue;
      const int g = idx2(d, j, t.gx[c]);
      const double w0 = t.w[r][c];
      const double e0 = t.E[r][c];
      const double gx = t.ix[r][c] * 0.5 *
                        ((t.E[r][c + 1] - e0) * (w0 * t.w[r][c + 1]) + (e0 - t.E[r][c - 1]) * (w0 * t.w[r][c - 1]));
      double dyp = 0.0, dym = 0.0;
      if (j < d.ny - 1) dyp = (t.E[r + 1][c] - e0) * (w0 * t.w[r + 1][c]) * t.cfp[r];
      if (j > 0) dym = (e0 - t.E[r - 1][c]) * (w0 * t.w[r - 1][c]) * t.cfm[r];
      const double gy = t.iyc[r] * 0.5 * (dyp + dym);
      const double us = t.U[r][c] + a.dtb * (-g9 * gx + t.fx[r - BT_H][c - BT_H]);
      const double vs = t.V[r][c] + a.dtb * (-g9 * gy + t.fy[r - BT_H][c - BT_H]);
      const double fd = t.fd[r - BT_H][c - BT_H], rd = t.rd[r - BT_H][c - BT_H];
      double un = (us + fd * vs) * rd * w0;
      double vn = (vs - fd * us) * rd * w0;
      if (a.sponge) {
        un *= a.es[g];
        vn *= a.es[g];
      }
      t.U[r][c] = un;
      t.V[r][c] = vn;
      a.pub_u[pout][g] = un;
      a.pub_v[pout][g] = vn;
      a.pub_e[pout][g] = e0;
    }
    __syncthreads();
    if (cap) {
      band_partials(d, a, t, t.U, a.part_u[pout], xt);
      band_partials(d, a, t, t.V, a.part_v[pout], xt);
    }
    // 5: the published fields are complete
    if (!grid_barrier(a.bar, a.err, nblocks, ZM_BT_BARRIER_POLLS)) return;
  }
  // ---- outputs: capped velocities and the float32 free surface
  const int plast = a.nsub & 1;
  if (cap) {
    band_means(a, t, 1, a.part_u[plast]);
    band_means(a, t, 2, a.part_v[plast]);
  }
  __syncthreads();
  for (int e = tid; e < NT; e += nt) {
    const int r = BT_H + e / BT_TX, c = BT_H + e % BT_TX;
    const int j = t.gj[r];
    if (j < 0 || !t.own_c[c]) continue;
    const int g = idx2(d, j, t.gx[c]);
    double u = t.U[r][c], v = t.V[r][c];
    if (cap) {
      u = cap_val(a, t, d.ny, 1, j, t.w[r][c], u);
      v = cap_val(a, t, d.ny, 2, j, t.w[r][c], v);
    }
    a.ubt_out[g] = u;
    a.vbt_out[g] = v;
    a.eta_out[g] = (float)t.E[r][c];
  }
}

// ---- streaming path: one subcycle as three plain kernels

__global__ void __launch_bounds__(256) k_bt_eta(Dev d, const double* __restrict__ eta, const double* __restrict__ ubt,
                                                const double* __restrict__ vbt, double* __restrict__ eta_o,
                                                double dtH) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const int c = idx2(d, j, i), ce = idx2(d, j, east(d, i)), cw = idx2(d, j, west(d, i));
  const double w0 = __ldg(d.wet2 + c), we = __ldg(d.wet2 + ce), ww = __ldg(d.wet2 + cw);
  const double u0 = ubt[c] * w0, ue = ubt[ce] * we, uw = ubt[cw] * ww;
  const double fe = 0.5 * (u0 + ue) * (w0 * we);
  const double fw = 0.5 * (uw + u0) * (ww * w0);
  const double div_x = (fe - fw) * __ldg(d.inv_dx_d + c);
  double fn = 0.0, fs = 0.0;
  const double v0 = vbt[c] * w0;
  if (j < d.ny - 1) {
    const int cn = idx2(d, j + 1, i);
    const double wn = __ldg(d.wet2 + cn);
    fn = 0.5 * (v0 + vbt[cn] * wn) * (w0 * wn) * (double)__ldg(d.cfp + j);
  }
  if (j > 0) {
    const int cs = idx2(d, j - 1, i);
    const double ws = __ldg(d.wet2 + cs);
    fs = 0.5 * (vbt[cs] * ws + v0) * (ws * w0) * (double)__ldg(d.cfp + j - 1);
  }
  const double div = div_x + (fn - fs) * (d.inv_dy_d / (double)__ldg(d.cosl + j));
  eta_o[c] = (eta[c] - dtH * div) * w0;
}

__global__ void __launch_bounds__(256) k_bt_vel(Dev d, const double* __restrict__ eta, const double* __restrict__ ubt,
                                                const double* __restrict__ vbt, const double* __restrict__ Fx,
                                                const double* __restrict__ Fy, double* __restrict__ ubt_o,
                                                double* __restrict__ vbt_o, double dtb, double drag,
                                                const double* __restrict__ sv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const int c = idx2(d, j, i), ce = idx2(d, j, east(d, i)), cw = idx2(d, j, west(d, i));
  const double w0 = __ldg(d.wet2 + c), we = __ldg(d.wet2 + ce), ww = __ldg(d.wet2 + cw);
  const double e0 = eta[c];
  const double gx = __ldg(d.inv_dx_d + c) * 0.5 * ((eta[ce] - e0) * (w0 * we) + (e0 - eta[cw]) * (w0 * ww));
  double dyp = 0.0, dym = 0.0;
  if (j < d.ny - 1) {
    const int cn = idx2(d, j + 1, i);
    dyp = (eta[cn] - e0) * (w0 * __ldg(d.wet2 + cn)) * (double)__ldg(d.cfp + j);
  }
  if (j > 0) {
    const int cs = idx2(d, j - 1, i);
    dym = (e0 - eta[cs]) * (w0 * __ldg(d.wet2 + cs)) * (double)__ldg(d.cfm + j);
  }
  const double gy = (d.inv_dy_d / (double)__ldg(d.cosl + j)) * 0.5 * (dyp + dym);
  const double us = ubt[c] + dtb * (-9.81 * gx + Fx[c]);
  const double vs = vbt[c] + dtb * (-9.81 * gy + Fy[c]);
  const double fd = __ldg(d.fcor_d + c) * dtb, rd = bt_drag_factor(fd, drag);
  double un = (us + fd * vs) * rd * w0;
  double vn = (vs - fd * us) * rd * w0;
  if (sv) {
    un *= sv[c];
    vn *= sv[c];
  }
  ubt_o[c] = un;
  vbt_o[c] = vn;
}

// Uniform refill of the volume a decay removes (barotropic.py:22-31), streaming
// path: per-block partial sums of area (eta f - eta) ...
__global__ void __launch_bounds__(256) k_refill_part(Dev d, const double* __restrict__ eta,
                                                     const double* __restrict__ fac,
                                                     const double* __restrict__ area, double* __restrict__ part) {
  __shared__ double red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < d.nx && j < d.ny) {
    const int c = idx2(d, j, i);
    const double e0 = eta[c];
    s = area[c] * (e0 * fac[c] - e0);
  }
  red[t] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) red[t] += red[t + o];
    __syncthreads();
  }
  if (t == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = red[0];
}

// ... then every block folds the partials in the same order and applies
// eta f + (-dV / ocean_area) wet.
__global__ void __launch_bounds__(256) k_refill_apply(Dev d, double* __restrict__ eta, const double* __restrict__ fac,
                                                      const double* __restrict__ part, int nparts, double ocean) {
  __shared__ double red[256];
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  double s = 0.0;
  for (int b = t; b < nparts; b += 256) s += part[b];
  red[t] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) red[t] += red[t + o];
    __syncthreads();
  }
  const double shift = -red[0] / ocean;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const int c = idx2(d, j, i);
  eta[c] = eta[c] * fac[c] + shift * (double)__ldg(d.wet2 + c);
}

// Polar cap of up to two 2-D float64 fields in place: one block per band row,
// blockIdx.y selects the field.
__global__ void __launch_bounds__(256) k_cap2d(Dev d, double* f0, double* f1, const float* __restrict__ wts,
                                               const double* __restrict__ count, int nb_rows) {
  __shared__ double red[256];
  const int r = blockIdx.x;  // 0..2*nb_rows-1
  double* f = blockIdx.y == 0 ? f0 : f1;
  if (!f) return;
  const int j = r < nb_rows ? r : d.ny - 2 * nb_rows + r;
  const double wt = (double)(r < nb_rows ? wts[r] : wts[2 * nb_rows - 1 - r]);
  double s = 0.0;
  for (int i = threadIdx.x; i < d.nx; i += blockDim.x) s += f[idx2(d, j, i)] * (double)__ldg(d.wet2 + idx2(d, j, i));
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double mean = red[0] / count[r];
  for (int i = threadIdx.x; i < d.nx; i += blockDim.x) {
    const double w = __ldg(d.wet2 + idx2(d, j, i));
    const double val = f[idx2(d, j, i)] * w;
    f[idx2(d, j, i)] = wt * (mean * w) + (1.0 - wt) * val;
  }
}

__global__ void __launch_bounds__(256) k_eta_to_float(Dev d, const double* __restrict__ e64, float* __restrict__ e32) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) e32[idx2(d, j, i)] = (float)e64[idx2(d, j, i)];
}

// Barrier probe for the timeout path: `expected` arrivals are awaited but only
// gridDim.x blocks arrive, so with expected > gridDim.x every block gives up
// after max_polls polls and records ZM_BT_ERR_BARRIER.
__global__ void k_barrier_probe(unsigned* bar, unsigned* err, unsigned expected, unsigned max_polls) {
  grid_barrier_begin(bar);
  grid_barrier(bar, err, expected, max_polls);
}

}  // namespace zm

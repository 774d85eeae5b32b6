// Column-divergence projection of the stage-2 advective velocity
// (dynamics/projection.py:10-127, applied at timestepping/step.py:292-303).
//
// The reference solves A psi = b with jax.scipy.sparse.linalg.cg, where
//   A psi = -coldiv(grad3(psi)) area,   b = -(coldiv(u, v) / (dt g)) area,
// coldiv the level sum of the face-flux divergence times the node thickness
// on wet columns (transport.py:45-57) and grad3 the conservative gradient of
// the column-uniform psi (horizontal.py:126-151).  It corrects
// (u, v) -= dt g grad3(psi) and then, at most `refinements` times while the
// surface transport of the corrected velocity stays above rtol_t^2 times that
// of the input, solves again for the remaining divergence with an absolute
// floor tol ||b|| and corrects again.
//
// On the device:
//  * A is exactly a two-dimensional operator.  psi does not depend on the
//    level, so the level sum of the masked face fluxes needs only the
//    common-wet depths of two or three neighbouring columns.  With e_i(k) the
//    wet flag of the east face of column i at level k, H2_i = sum_k dz_k e_i
//    and H3_i = sum_k dz_k e_i e_{i+1}, the column flux through the east face is
//      Phi_i = 1/4 [ rdx_i (H3_{i-1} D_{i-1} + H2_i D_i)
//                  + rdx_{i+1} (H2_i D_i + H3_i D_{i+1}) ],   D_i = psi_{i+1} - psi_i,
//    and through the north face, with the face cosines cf_j = (c_j + c_{j+1})/2,
//      Psi_j = rdy cf_j / 4 [ (H2_j cf_j E_j + H3_{j-1} cf_{j-1} E_{j-1}) / c_j
//                           + (H3_j cf_{j+1} E_{j+1} + H2_j cf_j E_j) / c_{j+1} ].
//    k_proj_coef tabulates the three weights of each face once.
//  * The column divergence of the corrected velocity is that of the input plus
//    dt g (A psi) / area, so the right-hand side of a refinement is the
//    residual b - A psi_total of the first system and its transport norm is
//    (dt g)^2 sum res^2 / area.  The refinements therefore need no pass over
//    the 3-D fields: k_proj_rhs reads (u, v) once and k_proj_correct applies
//    the summed potential once.
//  * k_proj_cg runs every solve in one cooperative launch in float64, with the
//    loop of jax's cg: x = 0, r = b, z = M r, p = z, gamma = <r, z>; while the
//    squared residual (gamma without a preconditioner, <r, r> with one) is
//    above max(tol^2 <b, b>, atol^2) and k < maxiter: alpha = gamma / <p, Ap>,
//    x += alpha p, r -= alpha Ap, z = M r, beta = <r, z> / gamma, p = z + beta p.
//    The direction update is folded into the next product (each thread forms
//    z + beta p at its stencil points and stores its own), so an iteration
//    takes two grid barriers.  Dot products are summed per thread, per block in
//    a fixed tree and over blocks in block order by every block, so all blocks
//    take the same branches and the result does not depend on timing.  The
//    whole working set (a dozen 2-D float64 fields) stays in L2.
#include "zm_kernels.cuh"
#include "zm_sync.cuh"

namespace zm {

namespace {

__device__ __forceinline__ double bitd(uint64_t bits, int k) { return (double)((bits >> k) & 1ull); }

__device__ double dz_sum(uint64_t bits, const double* __restrict__ dzn, int nz) {
  double s = 0.0;
  for (int k = 0; k < nz; ++k)
    if ((bits >> k) & 1ull) s += dzn[k];
  return s;
}

// Block partial sums of NQ values, tree order fixed, written to part[block].
template <int NQ>
__device__ __forceinline__ void block_partials(const double (&v)[NQ], double* part) {
  __shared__ double red[NQ][PJ_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = lane < nw ? red[q][lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) part[blockIdx.x * ZM_PJ_SUMS + q] = x;
    }
  }
}

// Totals over all blocks, folded in block order; every block gets the same bits.
template <int NQ>
__device__ __forceinline__ void grid_totals(const double* part, double (&out)[NQ]) {
  __shared__ double tot[NQ];
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = 0.0;
      for (int b = lane; b < (int)gridDim.x; b += 32) x += __ldcg(part + b * ZM_PJ_SUMS + q);
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) tot[q] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) out[q] = tot[q];
  __syncthreads();
}

// Global sums through a grid barrier.  The partials alternate between two
// buffers: a block can only overwrite a buffer after every block has passed
// the next barrier, i.e. has finished reading it.
template <int NQ>
__device__ __forceinline__ bool reduce(const ProjArgs& a, int& red, const double (&v)[NQ], double (&out)[NQ]) {
  double* part = a.part + (size_t)(red & 1) * gridDim.x * ZM_PJ_SUMS;
  ++red;
  block_partials(v, part);
  if (!grid_barrier(a.bar, a.err, gridDim.x, ZM_BT_BARRIER_POLLS)) return false;
  grid_totals(part, out);
  return true;
}

// (A q) at (j, i); val(g) gives q at the 2-D index g.  `center` receives q(j, i).
template <class V>
__device__ __forceinline__ double apply_a(const Dev& d, const ProjArgs& a, int j, int i, V val, double& center) {
  const long long n2 = d.plane;
  const int iw = west(d, i), ie = east(d, i);
  const int iww = west(d, iw), iee = east(d, ie);
  const int js = max(j - 1, 0), jss = max(j - 2, 0);
  const int jn = min(j + 1, d.ny - 1), jnn = min(j + 2, d.ny - 1);
  const int g = idx2(d, j, i), gw = idx2(d, j, iw), gs = idx2(d, js, i);
  const double pc = val(g);
  const double pw = val(gw), pww = val(idx2(d, j, iww));
  const double pe = val(idx2(d, j, ie)), pee = val(idx2(d, j, iee));
  const double ps = val(gs), pss = val(idx2(d, jss, i));
  const double pn = val(idx2(d, jn, i)), pnn = val(idx2(d, jnn, i));
  center = pc;
  const double fe = __ldg(a.cx + g) * (pc - pw) + __ldg(a.cx + n2 + g) * (pe - pc) +
                    __ldg(a.cx + 2 * n2 + g) * (pee - pe);
  const double fw = __ldg(a.cx + gw) * (pw - pww) + __ldg(a.cx + n2 + gw) * (pc - pw) +
                    __ldg(a.cx + 2 * n2 + gw) * (pe - pc);
  const double fn = __ldg(a.cy + g) * (pc - ps) + __ldg(a.cy + n2 + g) * (pn - pc) +
                    __ldg(a.cy + 2 * n2 + g) * (pnn - pn);
  const double fs = j > 0 ? __ldg(a.cy + gs) * (ps - pss) + __ldg(a.cy + n2 + gs) * (pc - ps) +
                                __ldg(a.cy + 2 * n2 + gs) * (pn - pc)
                          : 0.0;
  return -(__ldg(a.sxy + g) * (fe - fw) + __ldg(a.sxy + n2 + g) * (fn - fs));
}

// One CG solve (jax loop) into x, which the caller has zeroed together with
// a.p0, r = rhs and z = M rhs, followed by a barrier.  Returns the iteration
// count, or -1 if a grid barrier gave up.
__device__ int cg_solve(const Dev& d, const ProjArgs& a, double* x, double gamma, double rr, double atol2, int& red) {
  const bool ident = a.minv == nullptr;
  const int ncell = d.nx * d.ny;
  const int stride = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const double* pold = a.p0;
  double* pnew = a.p1;
  double beta = 0.0;
  int k = 0;
  while ((ident ? gamma : rr) > atol2 && k < a.niter) {
    double s[1] = {0.0};
    for (int c = t0; c < ncell; c += stride) {
      const int j = c / d.nx, i = c - j * d.nx;
      double pc;
      const double ap = apply_a(
          d, a, j, i, [&](int g) { return fma(beta, __ldcg(pold + g), __ldcg(a.z + g)); }, pc);
      const int g = idx2(d, j, i);
      pnew[g] = pc;
      a.Ap[g] = ap;
      s[0] += pc * ap;
    }
    double t[1];
    if (!reduce(a, red, s, t)) return -1;
    const double alpha = gamma / t[0];
    double s2[2] = {0.0, 0.0};
    for (int c = t0; c < ncell; c += stride) {
      const int j = c / d.nx, i = c - j * d.nx;
      const int g = idx2(d, j, i);
      x[g] = __ldcg(x + g) + alpha * __ldcg(pnew + g);
      const double rv = __ldcg(a.r + g) - alpha * __ldcg(a.Ap + g);
      const double zv = ident ? rv : rv * __ldg(a.minv + g);
      a.r[g] = rv;
      a.z[g] = zv;
      s2[0] += rv * zv;
      s2[1] += rv * rv;
    }
    double t2[2];
    if (!reduce(a, red, s2, t2)) return -1;
    beta = t2[0] / gamma;
    gamma = t2[0];
    rr = t2[1];
    double* tmp = const_cast<double*>(pold);
    pold = pnew;
    pnew = tmp;
    ++k;
  }
  return k;
}

}  // namespace

// Face weights of the column operator, the row factors, 1/area and the
// Jacobi inverse diagonal (projection.py:10-51: the per-level diagonal of the
// 3-D operator summed with the node thicknesses; 1 where it is not positive).
__global__ void __launch_bounds__(256) k_proj_coef(Dev d, const double* __restrict__ dzn,
                                                   const double* __restrict__ cosd, const double* __restrict__ area,
                                                   double* __restrict__ cx, double* __restrict__ cy,
                                                   double* __restrict__ sxy, double* __restrict__ minv,
                                                   double* __restrict__ rarea) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const long long n2 = d.plane;
  const int g = idx2(d, j, i);
  const int iw = west(d, i), ie = east(d, i), iee = east(d, ie);
  const uint64_t wc = wb(d, j, i), we = wb(d, j, ie), ww = wb(d, j, iw), wee = wb(d, j, iee);
  const uint64_t e_w = ww & wc, e_c = wc & we, e_e = we & wee;
  const double rdx = d.inv_dx_d[g], rdx_e = d.inv_dx_d[idx2(d, j, ie)];
  cx[g] = 0.25 * rdx * dz_sum(e_w & e_c, dzn, d.nz);
  cx[n2 + g] = 0.25 * (rdx + rdx_e) * dz_sum(e_c, dzn, d.nz);
  cx[2 * n2 + g] = 0.25 * rdx_e * dz_sum(e_c & e_e, dzn, d.nz);
  const double rdy = d.inv_dy_d;
  const double c = cosd[j];
  double y0 = 0.0, y1 = 0.0, y2 = 0.0;
  if (j + 1 < d.ny) {
    const double cn = cosd[j + 1];
    const double cf = 0.5 * (c + cn);
    const uint64_t n_c = wc & wb(d, j + 1, i);
    const uint64_t n_s = j > 0 ? (wb(d, j - 1, i) & wc) : 0ull;
    const uint64_t n_n = j + 2 < d.ny ? (wb(d, j + 1, i) & wb(d, j + 2, i)) : 0ull;
    const double q = 0.25 * rdy * cf;
    if (j > 0) y0 = q * dz_sum(n_s & n_c, dzn, d.nz) * (0.5 * (cosd[j - 1] + c)) / c;
    y1 = q * dz_sum(n_c, dzn, d.nz) * cf * (1.0 / c + 1.0 / cn);
    if (j + 2 < d.ny) y2 = q * dz_sum(n_c & n_n, dzn, d.nz) * (0.5 * (cn + cosd[j + 2])) / cn;
  }
  cy[g] = y0;
  cy[n2 + g] = y1;
  cy[2 * n2 + g] = y2;
  const double ar = area[g];
  sxy[g] = ar * rdx;
  sxy[n2 + g] = ar * rdy / c;
  rarea[g] = ar > 0.0 ? 1.0 / ar : 0.0;
  if (minv) {
    const double cnr = cosd[(j + 1) % d.ny], csr = cosd[(j - 1 + d.ny) % d.ny];
    const bool has_n = j + 1 < d.ny, has_s = j > 0;
    const uint64_t wn = has_n ? wb(d, j + 1, i) : 0ull, ws = has_s ? wb(d, j - 1, i) : 0ull;
    double sum = 0.0;
    for (int k = 0; k < d.nz; ++k) {
      double dxg = 0.0;
      if (d.nx > 2) {
        const double pos = bitd(e_c, k), neg = bitd(e_w, k);
        dxg = 0.25 * rdx * rdx * ((pos - neg) * (pos - neg) + pos * pos + neg * neg);
      }
      const double py = bitd(wc & wn, k) * (0.5 * (c + cnr));
      const double ny_ = bitd(wc & ws, k) * (0.5 * (c + csr));
      const double dyg = 0.25 * rdy * rdy *
                         ((py - ny_) * (py - ny_) / (c * c) + py * py / (c * cnr) + ny_ * ny_ / (c * csr));
      sum += (dxg + dyg) * dzn[k];
    }
    const double diag = ar * sum;
    minv[g] = diag > 0.0 ? 1.0 / diag : 1.0;
  }
}

// b = -(coldiv(u, v) / (dt g)) area (projection.py:64-80 with transport.py:45-57
// and horizontal.py:255-281), float64 from the float32 velocity.
__global__ void __launch_bounds__(256) k_proj_rhs(Dev d, const float* __restrict__ u, const float* __restrict__ v,
                                                  const double* __restrict__ dzn, const double* __restrict__ cosd,
                                                  const double* __restrict__ area, double dtg,
                                                  double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const int g = idx2(d, j, i);
  const int iw = west(d, i), ie = east(d, i);
  const uint64_t wc = wb(d, j, i);
  const uint64_t e_c = wc & wb(d, j, ie), e_w = wb(d, j, iw) & wc;
  const bool has_n = j + 1 < d.ny, has_s = j > 0;
  const uint64_t n_c = has_n ? (wc & wb(d, j + 1, i)) : 0ull;
  const uint64_t n_s = has_s ? (wb(d, j - 1, i) & wc) : 0ull;
  const int jn = has_n ? j + 1 : j, js = has_s ? j - 1 : j;
  const double rdx = d.inv_dx_d[g], rdy = d.inv_dy_d;
  const double c = cosd[j];
  const double cfn = has_n ? 0.5 * (c + cosd[j + 1]) : 0.0;
  const double cfs = has_s ? 0.5 * (cosd[j - 1] + c) : 0.0;
  double sum = 0.0;
  for (int k = 0; k < d.nz; ++k) {
    const long long o = (long long)k * d.plane;
    const double uc = ld(u, o + g), ue = ld(u, o + idx2(d, j, ie)), uw = ld(u, o + idx2(d, j, iw));
    const double vc = ld(v, o + g), vn = ld(v, o + idx2(d, jn, i)), vs = ld(v, o + idx2(d, js, i));
    const double fxe = 0.5 * (uc + ue) * bitd(e_c, k);
    const double fxw = 0.5 * (uw + uc) * bitd(e_w, k);
    const double fyn = 0.5 * (vc + vn) * bitd(n_c, k) * cfn;
    const double fys = 0.5 * (vs + vc) * bitd(n_s, k) * cfs;
    sum += ((fxe - fxw) * rdx + (fyn - fys) * rdy / c) * dzn[k];
  }
  const double cdiv = sum * (double)__ldg(d.wet2 + g);
  b[g] = -(cdiv / dtg) * area[g];
}

__global__ void __launch_bounds__(PJ_THREADS, 1) k_proj_cg(Dev d, ProjArgs a) {
  grid_barrier_begin(a.bar);
  const bool ident = a.minv == nullptr;
  const int ncell = d.nx * d.ny;
  const int stride = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  int red = 0;
  // r = b, z = M b, psi = 0, p = 0; <b, b>, <b, z>, sum b^2 / area
  double s[3] = {0.0, 0.0, 0.0};
  for (int c = t0; c < ncell; c += stride) {
    const int j = c / d.nx, i = c - j * d.nx;
    const int g = idx2(d, j, i);
    const double bv = __ldcg(a.b + g);
    const double zv = ident ? bv : bv * __ldg(a.minv + g);
    a.r[g] = bv;
    a.z[g] = zv;
    a.psi[g] = 0.0;
    a.p0[g] = 0.0;
    s[0] += bv * bv;
    s[1] += bv * zv;
    s[2] += bv * bv * __ldg(a.rarea + g);
  }
  double t[3];
  if (!reduce(a, red, s, t)) return;
  const double bb = t[0];
  const double floor2 = a.tol2 * bb;  // (tol ||b||)^2
  const double thresh = a.trtol2 * t[2];
  int it[3] = {0, 0, 0};
  int nref = 0;
  it[0] = cg_solve(d, a, a.psi, t[1], bb, a.tol2 * bb, red);
  if (it[0] < 0) return;
  for (int q = 0; q < a.refinements; ++q) {
    // residual of the corrected velocity: res = b - A psi
    double s3[3] = {0.0, 0.0, 0.0};
    for (int c = t0; c < ncell; c += stride) {
      const int j = c / d.nx, i = c - j * d.nx;
      const int g = idx2(d, j, i);
      double pc;
      const double ap = apply_a(d, a, j, i, [&](int h) { return __ldcg(a.psi + h); }, pc);
      const double res = __ldcg(a.b + g) - ap;
      const double zv = ident ? res : res * __ldg(a.minv + g);
      a.r[g] = res;
      a.z[g] = zv;
      a.x[g] = 0.0;
      a.p0[g] = 0.0;
      s3[0] += res * res;
      s3[1] += res * zv;
      s3[2] += res * res * __ldg(a.rarea + g);
    }
    double t3[3];
    if (!reduce(a, red, s3, t3)) return;
    if (!(t3[2] > thresh)) break;
    ++nref;
    it[1 + q] = cg_solve(d, a, a.x, t3[1], t3[0], fmax(a.tol2 * t3[0], floor2), red);
    if (it[1 + q] < 0) return;
    for (int c = t0; c < ncell; c += stride) {
      const int j = c / d.nx, i = c - j * d.nx;
      const int g = idx2(d, j, i);
      a.psi[g] = __ldcg(a.psi + g) + __ldcg(a.x + g);
    }
    // the next residual reads the neighbours' psi
    if (q + 1 < a.refinements || a.norms)
      if (!grid_barrier(a.bar, a.err, gridDim.x, ZM_BT_BARRIER_POLLS)) return;
  }
  if (a.norms) {
    // ledger mode: squared surface-transport norms of the input and of the
    // corrected velocity, (dt g)^2 sum b^2 / area and (dt g)^2 sum res^2 / area
    // (diagnostics/budgets.py:175-183)
    double s4[1] = {0.0};
    for (int c = t0; c < ncell; c += stride) {
      const int j = c / d.nx, i = c - j * d.nx;
      const int g = idx2(d, j, i);
      double pc;
      const double res = __ldcg(a.b + g) - apply_a(d, a, j, i, [&](int h) { return __ldcg(a.psi + h); }, pc);
      s4[0] += res * res * __ldg(a.rarea + g);
    }
    double t4[1];
    if (!reduce(a, red, s4, t4)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.norms[0] = a.dtg * a.dtg * t[2];
      a.norms[1] = a.dtg * a.dtg * t4[0];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.stats[0] = it[0];
    a.stats[1] = it[1];
    a.stats[2] = it[2];
    a.stats[3] = nref;
  }
}

// (u, v) -= dt g grad3(psi) (projection.py:84-90 with horizontal.py:126-151).
__global__ void __launch_bounds__(256) k_proj_correct(Dev d, float* __restrict__ u, float* __restrict__ v,
                                                      const double* __restrict__ psi,
                                                      const double* __restrict__ cosd, double dtg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const int g = idx2(d, j, i);
  const int iw = west(d, i), ie = east(d, i);
  const uint64_t wc = wb(d, j, i);
  const uint64_t e_c = wc & wb(d, j, ie), e_w = wb(d, j, iw) & wc;
  const bool has_n = j + 1 < d.ny, has_s = j > 0;
  const uint64_t pos = has_n ? (wc & wb(d, j + 1, i)) : 0ull;
  const uint64_t neg = has_s ? (wb(d, j - 1, i) & wc) : 0ull;
  const double pc = psi[g], pe = psi[idx2(d, j, ie)], pw = psi[idx2(d, j, iw)];
  const double pn = has_n ? psi[idx2(d, j + 1, i)] : pc, ps = has_s ? psi[idx2(d, j - 1, i)] : pc;
  const double c = cosd[j];
  const double cp = 0.5 * (c + cosd[(j + 1) % d.ny]), cm = 0.5 * (c + cosd[(j - 1 + d.ny) % d.ny]);
  const double hx = d.inv_dx_d[g] * 0.5, hy = (d.inv_dy_d / c) * 0.5;
  const double dxe = pe - pc, dxw = pc - pw, dyn = (pn - pc) * cp, dys = (pc - ps) * cm;
  for (int k = 0; k < d.nz; ++k) {
    const long long o = (long long)k * d.plane + g;
    const double gx = hx * (dxe * bitd(e_c, k) + dxw * bitd(e_w, k));
    const double gy = hy * (dyn * bitd(pos, k) + dys * bitd(neg, k));
    u[o] = (float)((double)u[o] - dtg * gx);
    v[o] = (float)((double)v[o] - dtg * gy);
  }
}

}  // namespace zm

// Stencil, column and barotropic kernels of the global ocean step.
//
// Each kernel names the reference operator it computes (paths relative to the
// ZhenMode source tree).  Layout and masks: see zm_internal.cuh.
#include "zm_kernels.cuh"

namespace zm {

// ------------------------------------------------------------------ helpers
struct Nb {  // horizontal neighbour indices of (j, i)
  int i, j, ie, iw, jn, js;
};
__device__ __forceinline__ Nb nb(const Dev& d, int j, int i) {
  return Nb{i, j, east(d, i), west(d, i), north(d, j), south(j)};
}

// 4-byte global -> shared copy that completes asynchronously, and the commit
// and wait of such copies in groups (cp.async)
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Plane offset of cell e of a padded column tile PX cells wide whose interior
// starts at (i0, j0), with an H-cell halo: rows clamped at the closed walls
// like north()/south(), longitude wrapped like east()/west().
template <int PX, int H = 1>
__device__ __forceinline__ int tile_cell(const Dev& d, int e, int i0, int j0) {
  const int rr = e / PX, cc = e - rr * PX;
  const int gj = min(max(j0 - H + rr, 0), d.ny - 1);
  int gi = (i0 - H + cc) % d.nx;
  if (gi < 0) gi += d.nx;
  return idx2(d, gj, gi);
}

// Horizontal Laplacian on the sphere, legacy branch
// (numerics/horizontal.py:181-215): face-gated d2/dx2, mirror-ghost face-gated
// d2/dy2, metric term -(tan(lat)/R) d/dy on the unmasked centred difference.
__device__ __forceinline__ float lap_h(const Dev& d, const float* __restrict__ a, int k, const Nb& n) {
  const long long b = (long long)k * d.plane;
  const float a0 = ld(a, b + idx2(d, n.j, n.i));
  const float ae = ld(a, b + idx2(d, n.j, n.ie));
  const float aw = ld(a, b + idx2(d, n.j, n.iw));
  const float an = ld(a, b + idx2(d, n.jn, n.i));
  const float as = ld(a, b + idx2(d, n.js, n.i));
  const float w0 = wetf(wb(d, n.j, n.i), k), we = wetf(wb(d, n.j, n.ie), k);
  const float ww = wetf(wb(d, n.j, n.iw), k), wn = wetf(wb(d, n.jn, n.i), k);
  const float ws = wetf(wb(d, n.js, n.i), k);
  const float d2x = ((ae - a0) * w0 * we - (a0 - aw) * w0 * ww) * __ldg(d.inv_dx2 + idx2(d, n.j, n.i));
  const float d2y = ((an - a0) * wn * w0 - (a0 - as) * w0 * ws) * d.inv_dy2;
  const float ddy = (an - as) * (0.5f * d.inv_dy);
  return d2x + d2y + (-ddy * __ldg(d.tanR + n.j));
}

// Wet-face flux-form diffusion (numerics/horizontal.py:217-243); kap == nullptr
// means unit diffusivity (the biharmonic tracer operator, :245-249).
__device__ __forceinline__ float hdiff(const Dev& d, const float* __restrict__ c, const float* __restrict__ kap,
                                       int k, const Nb& n) {
  const long long b = (long long)k * d.plane;
  const float c0 = ld(c, b + idx2(d, n.j, n.i));
  const float ce = ld(c, b + idx2(d, n.j, n.ie));
  const float cw = ld(c, b + idx2(d, n.j, n.iw));
  const float w0 = wetf(wb(d, n.j, n.i), k), we = wetf(wb(d, n.j, n.ie), k), ww = wetf(wb(d, n.j, n.iw), k);
  float kc = 1.f, ke = 1.f, kw = 1.f, kn = 1.f, ks = 1.f;
  if (kap) {
    kc = __ldg(kap + idx2(d, n.j, n.i));
    ke = __ldg(kap + idx2(d, n.j, n.ie));
    kw = __ldg(kap + idx2(d, n.j, n.iw));
    kn = __ldg(kap + idx2(d, n.jn, n.i));
    ks = __ldg(kap + idx2(d, n.js, n.i));
  }
  const float fe = 0.5f * (kc + ke) * (ce - c0) * __ldg(d.inv_dx + idx2(d, n.j, n.i)) * w0 * we;
  const float fw = 0.5f * (kw + kc) * (c0 - cw) * __ldg(d.inv_dx + idx2(d, n.j, n.iw)) * ww * w0;
  float fn = 0.f, fs = 0.f;
  if (n.j < d.ny - 1) {
    const float cn = ld(c, b + idx2(d, n.jn, n.i));
    const float wn = wetf(wb(d, n.jn, n.i), k);
    fn = 0.5f * (kc + kn) * (cn - c0) * d.inv_dy * w0 * wn * __ldg(d.cfp + n.j);
  }
  if (n.j > 0) {
    const float cs = ld(c, b + idx2(d, n.js, n.i));
    const float ws = wetf(wb(d, n.js, n.i), k);
    fs = 0.5f * (ks + kc) * (c0 - cs) * d.inv_dy * ws * w0 * __ldg(d.cfp + n.js);
  }
  return (fe - fw) * __ldg(d.inv_dx + idx2(d, n.j, n.i)) + (fn - fs) * d.inv_dy * __ldg(d.inv_cos + n.j);
}

// Ghost-filled value of a column at level k (numerics/vertical.py:122-135).
__device__ __forceinline__ float colv(const float* __restrict__ a, long long base, long long plane, int k, int kb) {
  return ld(a, base + (long long)(k < kb ? k : kb) * plane);
}

#define ZM_POINT_IDX                                   \
  const int i = blockIdx.x * blockDim.x + threadIdx.x; \
  const int j = blockIdx.y * blockDim.y + threadIdx.y; \
  const int k = blockIdx.z;                            \
  if (i >= d.nx || j >= d.ny) return;                  \
  const long long id = idx3(d, k, j, i);

// ------------------------------------------------------------------ L half step
// nu_h Laplacian subcycles on (u, v) (timestepping/step.py:94-107), several
// subcycles per pass on one level.  A block covers an NB_W wide, NW * NB_R
// high tile with 32 x NW threads (NW = 8 or 16 warps, chosen by the
// autotuner): lane l of warp w holds columns 2l, 2l+1 of rows
// NB_R w .. NB_R w + NB_R - 1 in registers, as (u, v) pairs, with their face
// coefficients.  East/west neighbours move between lanes by shuffles; the
// rows above and below a warp's strip pass through shared memory, double
// buffered, so one barrier per subcycle suffices.  Values at the tile edge
// are wrong, and the error enters one cell per subcycle: after nsub <= halo
// subcycles the inner (NB_W - 2 halo) x (NW NB_R - 2 halo) points are exact (halo <= NB_T is a
// launch parameter chosen by the autotuner).
//
// The Laplacian of numerics/horizontal.py:181-215 is rewritten per point as
//   lap = aE (uE - u0) + aW (uW - u0) + aN (uN - u0) + aS (uS - u0)
// with aE/aW the gated x faces times 1/dx^2, aN = cN - t, aS = cS + t
// (cN/cS the gated y faces times 1/dy^2, t = tan(lat)/(2 R dy) from the
// metric term -(tan(lat)/R) du/dy), and the mirror ghost of the closed
// walls folded in: at j = ny-1 the north neighbour equals u0, so aN = 0; at
// j = 0, aS = 0.  The coefficients, scaled by nu_h dt_sub, are formed once
// per pass from the face gates of the cell (k_nu_gates, built once per
// solver: one byte per point) and per-row constants, so the set-up needs
// no neighbour wet flags.  Longitude wraps.  The lane's two columns are held
// as packed pairs, so the update runs on the paired FP32 instructions
// (__ffma2_rn, __fadd2_rn; the same roundings as the scalar form).  Points
// of the tile edge see their own values as the missing neighbours (their
// results are discarded with the halo).
template <int NW>
__global__ void __launch_bounds__(32 * NW, 16 / NW)
k_nu_tb(Dev d, const float* __restrict__ u, const float* __restrict__ v, float* __restrict__ uo,
        float* __restrict__ vo, float c, int nsub, int halo) {
  constexpr int NH = NW * NB_R;                   // tile rows
  const int TI = NB_W - 2 * halo, TJ = NH - 2 * halo;
  __shared__ float4 edge[2][NW][2][32];           // [parity][warp][0 bottom row, 1 top row][lane]
  pdl_trigger();
  const int lane = threadIdx.x, wp = threadIdx.y;
  const int k = blockIdx.z;
  const int gx0 = blockIdx.x * TI - halo, gy0 = blockIdx.y * TJ - halo;
  const int c0 = 2 * lane, r0 = wp * NB_R;
  int gi[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int g = (gx0 + c0 + h) % d.nx;
    gi[h] = g < 0 ? g + d.nx : g;
  }
  const long long kb = (long long)k * d.plane;
  const float cn = d.nu_h * c;
  // face coefficients, paired like the state: (column 2l, column 2l+1).  The
  // west and south ones are held negated (nW = -aW, nS = -aS) and negated back
  // in the update, an exact round trip: ptxas 12.9 allocates this form's
  // registers differently, and it ran 4 % faster than holding aW, aS.
  float2 kE[NB_R], nW[NB_R], kN[NB_R], nS[NB_R];
#pragma unroll
  for (int q = 0; q < NB_R; ++q) {
    const int gj = gy0 + r0 + q;
    const int gjc = gj < 0 ? 0 : (gj >= d.ny ? d.ny - 1 : gj);
    const bool n_in = gj < d.ny - 1;  // north neighbour inside the domain
    const bool s_in = gj > 0;
    const float t = 0.5f * d.inv_dy * __ldg(d.tanR + gjc);
    // aN with the north face open / closed, aS likewise (0 beyond the walls)
    const float n1 = n_in ? (d.inv_dy2 - t) * cn : 0.f, n0 = n_in ? (0.f - t) * cn : 0.f;
    const float s1 = s_in ? (d.inv_dy2 + t) * cn : 0.f, s0 = s_in ? (0.f + t) * cn : 0.f;
    float ce[2], cw[2], cnn[2], cs[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int id2 = idx2(d, gjc, gi[h]);
      const unsigned g = __ldg(d.nu_gate + kb + id2);
      const float ax = __ldg(d.inv_dx2 + id2) * cn;
      ce[h] = (g & 1u) ? ax : 0.f;
      cw[h] = (g & 2u) ? ax : 0.f;
      cnn[h] = (g & 4u) ? n1 : n0;
      cs[h] = (g & 8u) ? s1 : s0;
    }
    kE[q] = make_float2(ce[0], ce[1]);
    nW[q] = make_float2(-cw[0], -cw[1]);
    kN[q] = make_float2(cnn[0], cnn[1]);
    nS[q] = make_float2(-cs[0], -cs[1]);
  }
  const unsigned full = 0xffffffffu;
  pdl_wait();  // u, v come from the preceding kernel
  // the lane's two columns as pairs: au[q] = (u[2l], u[2l+1]) of row q, av likewise
  float2 au[NB_R], av[NB_R];
#pragma unroll
  for (int q = 0; q < NB_R; ++q) {
    int gj = gy0 + r0 + q;
    gj = gj < 0 ? 0 : (gj >= d.ny ? d.ny - 1 : gj);
    const long long id0 = kb + (long long)gj * d.P + gi[0], id1 = kb + (long long)gj * d.P + gi[1];
    au[q] = make_float2(ld(u, id0), ld(u, id1));
    av[q] = make_float2(ld(v, id0), ld(v, id1));
  }
  const float2 m1 = make_float2(-1.f, -1.f);
  for (int s = 0; s < nsub; ++s) {
    const int p = s & 1;
    edge[p][wp][0][lane] = make_float4(au[0].x, au[0].y, av[0].x, av[0].y);
    edge[p][wp][1][lane] = make_float4(au[NB_R - 1].x, au[NB_R - 1].y, av[NB_R - 1].x, av[NB_R - 1].y);
    __syncthreads();
    // rows just outside the strip (the tile edge reuses the strip's own row)
    const float4 nt = edge[p][wp + 1 < NW ? wp + 1 : wp][wp + 1 < NW ? 0 : 1][lane];
    const float4 sb = edge[p][wp > 0 ? wp - 1 : wp][wp > 0 ? 1 : 0][lane];
    float2 su = make_float2(sb.x, sb.y), sv = make_float2(sb.z, sb.w);
#pragma unroll
    for (int q = 0; q < NB_R; ++q) {
      const float2 nu = q + 1 < NB_R ? au[q + 1] : make_float2(nt.x, nt.y);
      const float2 nv = q + 1 < NB_R ? av[q + 1] : make_float2(nt.z, nt.w);
      // east of (2l, 2l+1) is (2l+1, 2l+2), west is (2l-1, 2l); the outside
      // columns come from the neighbouring lanes (lanes 0 and 31 get their
      // own values: tile-edge error)
      const float2 eu = make_float2(au[q].y, __shfl_down_sync(full, au[q].x, 1));
      const float2 wu = make_float2(__shfl_up_sync(full, au[q].y, 1), au[q].x);
      const float2 ev = make_float2(av[q].y, __shfl_down_sync(full, av[q].x, 1));
      const float2 wv = make_float2(__shfl_up_sync(full, av[q].y, 1), av[q].x);
      // u0 + aE (uE - u0) + aW (uW - u0) + aN (uN - u0) + aS (uS - u0) on packed pairs
      const float2 ncu = __fmul2_rn(au[q], m1), ncv = __fmul2_rn(av[q], m1);
      float2 ou = __ffma2_rn(kE[q], __fadd2_rn(eu, ncu), au[q]);
      float2 ov = __ffma2_rn(kE[q], __fadd2_rn(ev, ncv), av[q]);
      ou = __ffma2_rn(make_float2(-nW[q].x, -nW[q].y), __fadd2_rn(wu, ncu), ou);
      ov = __ffma2_rn(make_float2(-nW[q].x, -nW[q].y), __fadd2_rn(wv, ncv), ov);
      ou = __ffma2_rn(kN[q], __fadd2_rn(nu, ncu), ou);
      ov = __ffma2_rn(kN[q], __fadd2_rn(nv, ncv), ov);
      ou = __ffma2_rn(make_float2(-nS[q].x, -nS[q].y), __fadd2_rn(su, ncu), ou);
      ov = __ffma2_rn(make_float2(-nS[q].x, -nS[q].y), __fadd2_rn(sv, ncv), ov);
      su = au[q];
      sv = av[q];
      au[q] = ou;
      av[q] = ov;
    }
  }
  // write the exact interior
#pragma unroll
  for (int q = 0; q < NB_R; ++q) {
    const int r = r0 + q;
    const int gj = gy0 + r;
    if (r < halo || r >= NH - halo || gj >= d.ny) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = c0 + h;
      const int ix = gx0 + col;
      if (col < halo || col >= NB_W - halo || ix >= d.nx) continue;
      const long long id = kb + (long long)gj * d.P + ix;
      uo[id] = h == 0 ? au[q].x : au[q].y;
      vo[id] = h == 0 ? av[q].x : av[q].y;
    }
  }
}

// Face gates of the nu_h Laplacian, one byte per point (built once per
// solver): bit 0 east face (this cell and its east neighbour wet), bit 1
// west, bit 2 north (inside the domain), bit 3 south.  Longitude wraps; the
// closed walls have no face.
__global__ void k_nu_gates(Dev d, unsigned char* __restrict__ gate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (j >= d.ny || i >= d.P) return;
  unsigned g = 0u;
  if (i < d.nx && wetb(wb(d, j, i), k)) {
    if (wetb(wb(d, j, east(d, i)), k)) g |= 1u;
    if (wetb(wb(d, j, west(d, i)), k)) g |= 2u;
    if (j < d.ny - 1 && wetb(wb(d, j + 1, i), k)) g |= 4u;
    if (j > 0 && wetb(wb(d, j - 1, i), k)) g |= 8u;
  }
  gate[idx3(d, k, j, i)] = (unsigned char)g;
}

// Whole linear half step except the nu_h subcycles (timestepping/step.py:108-173,
// legacy, mode split).  A block owns an LT_X x LT_Y tile of columns and marches
// down d.lt_kc levels of them (the chunks of a column are separate blocks): u0,
// v0, T0, S0 of each level on the tile with a two-cell halo arrive in shared
// memory by cp.async one level ahead, in LT_NB rotating buffers; the wet flags
// are formed one level ahead from the cells' bitmasks, held in registers; the
// 2-D metric and diffusivity fields are loaded once.  The inner Laplacians of
// the biharmonic operators (numerics/horizontal.py:245-253) are formed on the
// one-cell ring, the outer ones at the tile interior.  Rows beyond the closed
// walls load the clamped row (the edge padding of horizontal.py:14-25); the
// outer biharmonic applies the mirror to the inner Laplacian field, whose edge
// row is padded by itself in the reference.  Vertical diffusion takes the level
// above from registers and the level below from the next buffer; then
// land/ghost hold and the exact Coriolis rotation by f dt/2.
constexpr int LT_X = 32, LT_Y = 8, LT_H = 2, LT_NB = 3;
constexpr int LT_PX = LT_X + 2 * LT_H, LT_PY = LT_Y + 2 * LT_H;
constexpr int LT_CELLS = LT_PX * LT_PY;
static_assert(LT_CELLS <= 2 * LT_X * LT_Y, "two tile cells per thread at most");

struct LtTile {
  float u[LT_NB][LT_PY][LT_PX], v[LT_NB][LT_PY][LT_PX], T[LT_NB][LT_PY][LT_PX], S[LT_NB][LT_PY][LT_PX];
  float Lu[LT_PY][LT_PX], Lv[LT_PY][LT_PX], LT[LT_PY][LT_PX], LS[LT_PY][LT_PX];
  float w[2][LT_PY][LT_PX], kh[LT_PY][LT_PX], ix[LT_PY][LT_PX], ix2[LT_PY][LT_PX];
  float tanR[LT_PY], cfp[LT_PY], icos[LT_PY];
  int gj[LT_PY];
};

// Laplacian of a tile field at (r, c) (horizontal.py:181-215) with the wet
// flags w of its level; `mirror` replaces the outer neighbour at a wall row by
// the row itself.
__device__ __forceinline__ float lap_s(const Dev& d, const LtTile& t, const float (*w)[LT_PX],
                                      const float (*a)[LT_PX], int r, int c, bool mirror) {
  const float a0 = a[r][c], ae = a[r][c + 1], aw = a[r][c - 1];
  float an = a[r + 1][c], as = a[r - 1][c];
  if (mirror) {
    if (t.gj[r] == d.ny - 1) an = a0;
    if (t.gj[r] == 0) as = a0;
  }
  const float w0 = w[r][c];
  const float d2x = ((ae - a0) * w0 * w[r][c + 1] - (a0 - aw) * w0 * w[r][c - 1]) * t.ix2[r][c];
  const float d2y = ((an - a0) * w[r + 1][c] * w0 - (a0 - as) * w0 * w[r - 1][c]) * d.inv_dy2;
  const float ddy = (an - as) * (0.5f * d.inv_dy);
  return d2x + d2y + (-ddy * t.tanR[r]);
}

// Wet-face flux diffusion of a tile field at (r, c) (horizontal.py:217-243)
// with the wet flags w of its level; unit diffusivity when `unit`.  The wall
// faces are closed explicitly.
__device__ __forceinline__ float hdiff_s(const Dev& d, const LtTile& t, const float (*w)[LT_PX],
                                        const float (*a)[LT_PX], int r, int c, bool unit) {
  const float a0 = a[r][c];
  const float k0 = unit ? 1.f : t.kh[r][c];
  const float ke = unit ? 1.f : t.kh[r][c + 1], kw = unit ? 1.f : t.kh[r][c - 1];
  const float kn = unit ? 1.f : t.kh[r + 1][c], ks = unit ? 1.f : t.kh[r - 1][c];
  const float w0 = w[r][c];
  const float fe = 0.5f * (k0 + ke) * (a[r][c + 1] - a0) * t.ix[r][c] * w0 * w[r][c + 1];
  const float fw = 0.5f * (kw + k0) * (a0 - a[r][c - 1]) * t.ix[r][c - 1] * w[r][c - 1] * w0;
  const int gj = t.gj[r];
  float fn = 0.f, fs = 0.f;
  if (gj < d.ny - 1) fn = 0.5f * (k0 + kn) * (a[r + 1][c] - a0) * d.inv_dy * w0 * w[r + 1][c] * t.cfp[r];
  if (gj > 0) fs = 0.5f * (ks + k0) * (a0 - a[r - 1][c]) * d.inv_dy * w[r - 1][c] * w0 * t.cfp[r - 1];
  return (fe - fw) * t.ix[r][c] + (fn - fs) * d.inv_dy * t.icos[r];
}

// The two operators above on a pair of tile fields (u and v, or T and S) that
// share every coefficient, on the paired FP32 instructions (__fadd2_rn,
// __fmul2_rn, __ffma2_rn: each half rounds like the scalar operation).  The
// wet gates are products of 0/1 flags, formed once per point, and a
// difference a0 - ax enters as the exact negation of ax - a0.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 pair(const float (*A)[LT_PX], const float (*B)[LT_PX], int r, int c) {
  return make_float2(A[r][c], B[r][c]);
}

__device__ __forceinline__ float2 lap2(const Dev& d, const LtTile& t, const float (*w)[LT_PX],
                                      const float (*A)[LT_PX], const float (*B)[LT_PX], int r, int c, bool mirror) {
  const float2 m1 = f2(-1.f);
  const float2 a0 = pair(A, B, r, c), ae = pair(A, B, r, c + 1), aw = pair(A, B, r, c - 1);
  float2 an = pair(A, B, r + 1, c), as = pair(A, B, r - 1, c);
  if (mirror) {
    if (t.gj[r] == d.ny - 1) an = a0;
    if (t.gj[r] == 0) as = a0;
  }
  const float w0 = w[r][c];
  const float ge = w0 * w[r][c + 1], gw = w0 * w[r][c - 1], gn = w[r + 1][c] * w0, gs = w0 * w[r - 1][c];
  const float2 na0 = __fmul2_rn(a0, m1);
  // d2x = ((ae - a0) ge - (a0 - aw) gw) / dx^2, d2y likewise / dy^2
  const float2 d2x = __fmul2_rn(__ffma2_rn(__fadd2_rn(aw, na0), f2(gw), __fmul2_rn(__fadd2_rn(ae, na0), f2(ge))),
                                f2(t.ix2[r][c]));
  const float2 d2y = __fmul2_rn(__ffma2_rn(__fadd2_rn(as, na0), f2(gs), __fmul2_rn(__fadd2_rn(an, na0), f2(gn))),
                                f2(d.inv_dy2));
  const float2 ddy = __fmul2_rn(__fadd2_rn(an, __fmul2_rn(as, m1)), f2(0.5f * d.inv_dy));
  return __ffma2_rn(ddy, f2(-t.tanR[r]), __fadd2_rn(d2x, d2y));
}

__device__ __forceinline__ float2 hdiff2(const Dev& d, const LtTile& t, const float (*w)[LT_PX],
                                        const float (*A)[LT_PX], const float (*B)[LT_PX], int r, int c, bool unit) {
  const float2 m1 = f2(-1.f);
  const float2 a0 = pair(A, B, r, c);
  const float k0 = unit ? 1.f : t.kh[r][c];
  const float ke = unit ? 1.f : t.kh[r][c + 1], kw = unit ? 1.f : t.kh[r][c - 1];
  const float kn = unit ? 1.f : t.kh[r + 1][c], ks = unit ? 1.f : t.kh[r - 1][c];
  const float w0 = w[r][c];
  const int gj = t.gj[r];
  // face coefficients: 0.5 (k + k') / dx (or cos_face / dy) times the face gate
  const float ce = 0.5f * (k0 + ke) * t.ix[r][c] * (w0 * w[r][c + 1]);
  const float cw = 0.5f * (kw + k0) * t.ix[r][c - 1] * (w[r][c - 1] * w0);
  const float cn = gj < d.ny - 1 ? 0.5f * (k0 + kn) * d.inv_dy * (w0 * w[r + 1][c]) * t.cfp[r] : 0.f;
  const float cs = gj > 0 ? 0.5f * (ks + k0) * d.inv_dy * (w[r - 1][c] * w0) * t.cfp[r - 1] : 0.f;
  const float2 na0 = __fmul2_rn(a0, m1);
  // (fe - fw) / dx + (fn - fs) / (dy cos), with fw = (a0 - aw) cw = -(aw - a0) cw
  const float2 x = __ffma2_rn(__fadd2_rn(pair(A, B, r, c - 1), na0), f2(cw),
                              __fmul2_rn(__fadd2_rn(pair(A, B, r, c + 1), na0), f2(ce)));
  const float2 y = __ffma2_rn(__fadd2_rn(pair(A, B, r - 1, c), na0), f2(cs),
                              __fmul2_rn(__fadd2_rn(pair(A, B, r + 1, c), na0), f2(cn)));
  return __ffma2_rn(x, f2(t.ix[r][c]), __fmul2_rn(y, f2(d.inv_dy * t.icos[r])));
}

// Node-form d2/dz2 with zero-flux ends (numerics/vertical.py:275-293) and the
// tracer vertical diffusion at a wet level k of a column, from its values at
// k - 1 (am), k (a0) and k + 1 (ap): the column is ghost-filled below kbot
// with its value at kbot (numerics/vertical.py:122-135), so the level below
// reads a0 at k = kbot.
__device__ __forceinline__ float d2z_c(const Dev& d, int k, int kb, float am, float a0, float ap) {
  const float dn = k < kb ? ap : a0;
  if (k == 0) {
    if (d.nz < 2) return 0.f;
    return d.vc.d2_top * (dn - a0);
  }
  if (k == d.nz - 1) return d.vc.d2_bot * (am - a0);
  return d.vc.d2_hi[k] * (dn - a0) + d.vc.d2_lo[k] * (am - a0);
}

__device__ __forceinline__ float vdiff_c(const Dev& d, int k, uint64_t bits, float kappa, float am, float a0,
                                         float ap) {
  if (d.conservative_kv) {  // interface-flux form (numerics/vertical.py:317-332)
    float up = 0.f, dn = 0.f;
    if (k > 0 && wetb(bits, k - 1) && wetb(bits, k)) up = -kappa * (a0 - am) * d.vc.inv_dz_iface[k - 1];
    if (k < d.nz - 1 && wetb(bits, k) && wetb(bits, k + 1)) dn = -kappa * (ap - a0) * d.vc.inv_dz_iface[k];
    return (up - dn) * d.vc.inv_dz_node[k] * wetf(bits, k);
  }
  return kappa * d2z_c(d, k, kbot_of(bits), am, a0, ap);
}

template <bool UV, bool TS, bool IMPL>
__global__ void __launch_bounds__(LT_X * LT_Y, 4) k_lin_t(Dev d, const float* __restrict__ usub,
                                                         const float* __restrict__ vsub, const float* __restrict__ u0,
                                                         const float* __restrict__ v0, const float* __restrict__ T0,
                                                         const float* __restrict__ S0, float* __restrict__ uo,
                                                         float* __restrict__ vo, float* __restrict__ To,
                                                         float* __restrict__ So, float dth) {
  pdl_trigger();
  extern __shared__ float lt_smem[];
  LtTile& t = *reinterpret_cast<LtTile*>(lt_smem);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * LT_X + tx, nt = LT_X * LT_Y;
  const int i0 = blockIdx.x * LT_X, j0 = blockIdx.y * LT_Y;
  const int k0 = blockIdx.z * d.lt_kc, k1 = min(d.nz, k0 + d.lt_kc);  // this block's levels
  const int i = i0 + tx, j = j0 + ty;
  // threads outside the grid copy their tile cells, form their wet flags and
  // meet the barriers, nothing else
  const bool in = i < d.nx && j < d.ny;
  const int e0 = tid, e1 = tid + nt;
  const bool has1 = e1 < LT_CELLS;
  const int s0 = tile_cell<LT_PX, LT_H>(d, e0, i0, j0), s1 = has1 ? tile_cell<LT_PX, LT_H>(d, e1, i0, j0) : 0;
  const uint64_t b0 = __ldg(d.wbits + s0), b1 = has1 ? __ldg(d.wbits + s1) : 0ull;
  (&t.kh[0][0])[e0] = __ldg(d.kh2 + s0);
  (&t.ix[0][0])[e0] = __ldg(d.inv_dx + s0);
  (&t.ix2[0][0])[e0] = __ldg(d.inv_dx2 + s0);
  if (has1) {
    (&t.kh[0][0])[e1] = __ldg(d.kh2 + s1);
    (&t.ix[0][0])[e1] = __ldg(d.inv_dx + s1);
    (&t.ix2[0][0])[e1] = __ldg(d.inv_dx2 + s1);
  }
  if (tid < LT_PY) {
    const int gj = min(max(j0 - LT_H + tid, 0), d.ny - 1);
    t.gj[tid] = gj;
    t.tanR[tid] = __ldg(d.tanR + gj);
    t.cfp[tid] = __ldg(d.cfp + gj);
    t.icos[tid] = __ldg(d.inv_cos + gj);
  }
  auto issue = [&](int k) {  // level k into buffer k % LT_NB; one commit group per call
    if (k < d.nz && k <= k1) {  // level k1 only for the column neighbour below the chunk
      const long long off = (long long)k * d.plane;
      const int q = k % LT_NB;
      cp_async4(&t.u[q][0][0] + e0, u0 + off + s0);
      cp_async4(&t.v[q][0][0] + e0, v0 + off + s0);
      cp_async4(&t.T[q][0][0] + e0, T0 + off + s0);
      cp_async4(&t.S[q][0][0] + e0, S0 + off + s0);
      if (has1) {
        cp_async4(&t.u[q][0][0] + e1, u0 + off + s1);
        cp_async4(&t.v[q][0][0] + e1, v0 + off + s1);
        cp_async4(&t.T[q][0][0] + e1, T0 + off + s1);
        cp_async4(&t.S[q][0][0] + e1, S0 + off + s1);
      }
    }
    cp_async_commit();
  };
  // wet flags of the two tile cells, bit 0 = the next level wet_level forms
  uint64_t rb0 = b0 >> k0, rb1 = b1 >> k0;
  auto wet_level = [&](int k) {  // wet flags of level k into w[k % 2]; called for k0, k0 + 1, ... in turn
    if (k < d.nz) {
      float* pw = &t.w[k & 1][0][0];
      pw[e0] = (float)(unsigned)(rb0 & 1ull);
      if (has1) pw[e1] = (float)(unsigned)(rb1 & 1ull);
      rb0 >>= 1;
      rb1 >>= 1;
    }
  };
  pdl_wait();  // the state comes from the preceding kernels
  issue(k0);
  issue(k0 + 1);
  wet_level(k0);
  const int ic = in ? i : 0, jc = in ? j : 0;
  const long long base = idx2(d, jc, ic);
  const uint64_t bits = __ldg(d.wbits + base);
  const int kbt = kbot_of(bits);
  const float kv = __ldg(d.kv2 + base);
  const float rc = IMPL ? 0.f : __ldg(d.rot_c + base), rs = IMPL ? 0.f : __ldg(d.rot_s + base);
  // u0, v0, T0, S0 of the level above
  float um = 0.f, vm = 0.f, Tm = 0.f, Sm = 0.f;
  if (k0 > 0) {
    const long long pid = base + (long long)(k0 - 1) * d.plane;
    um = ld(u0, pid);
    vm = ld(v0, pid);
    Tm = ld(T0, pid);
    Sm = ld(S0, pid);
  }
  const int r = ty + LT_H, cc = tx + LT_H;
  constexpr bool do_uv = UV, do_ts = TS;
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<0>();  // this thread's copies of levels k and k + 1 are done
    __syncthreads();     // everyone's are, w[k % 2] is formed, the ring fields and level k - 1's buffers are free
    issue(k + 2);
    wet_level(k + 1);
    const int q = k % LT_NB, qn = (k + 1) % LT_NB;
    const float(*w)[LT_PX] = t.w[k & 1];
    if (do_uv || do_ts) {
      // the one-cell ring around the interior, walked over whole padded rows so
      // that a warp's shared-memory addresses are consecutive (no bank conflicts)
      constexpr int RY = LT_Y + 2;
      for (int e = tid; e < LT_PX * RY; e += nt) {
        const int rr = 1 + e / LT_PX, c2 = e % LT_PX;
        if (c2 == 0 || c2 == LT_PX - 1) continue;
        if (do_uv) {
          const float2 L = lap2(d, t, w, t.u[q], t.v[q], rr, c2, false);
          t.Lu[rr][c2] = L.x;
          t.Lv[rr][c2] = L.y;
        }
        if (do_ts) {
          const float2 L = hdiff2(d, t, w, t.T[q], t.S[q], rr, c2, true);
          t.LT[rr][c2] = L.x;
          t.LS[rr][c2] = L.y;
        }
      }
      __syncthreads();
    }
    if (!in) continue;
    const long long id = (long long)k * d.plane + base;
    const bool wet = wetb(bits, k);
    const float uc = t.u[q][r][cc], vc = t.v[q][r][cc], Tc = t.T[q][r][cc], Sc = t.S[q][r][cc];
    float u, v, T, S;
    if (!wet) {
      u = uc;
      v = vc;
      T = Tc;
      S = Sc;
    } else {
      float2 ts = __ffma2_rn(hdiff2(d, t, w, t.T[q], t.S[q], r, cc, false), f2(dth), make_float2(Tc, Sc));
      if (do_ts) ts = __ffma2_rn(hdiff2(d, t, w, t.LT, t.LS, r, cc, true), f2(-d.kappa_bi * dth), ts);
      float2 uv = make_float2(ld(usub, id), ld(vsub, id));
      if (do_uv) uv = __ffma2_rn(lap2(d, t, w, t.Lu, t.Lv, r, cc, true), f2(-d.nu_bi * dth), uv);
      T = ts.x;
      S = ts.y;
      u = uv.x;
      v = uv.y;
      if (!IMPL) {
        const bool below = k + 1 < d.nz;  // level k + 1 sits in buffer qn
        const float up = below ? t.u[qn][r][cc] : uc, vp = below ? t.v[qn][r][cc] : vc;
        const float Tp = below ? t.T[qn][r][cc] : Tc, Sp = below ? t.S[qn][r][cc] : Sc;
        u = u + d.nu_v * d2z_c(d, k, kbt, um, uc, up) * dth;
        v = v + d.nu_v * d2z_c(d, k, kbt, vm, vc, vp) * dth;
        T = T + vdiff_c(d, k, bits, kv, Tm, Tc, Tp) * dth;
        S = S + vdiff_c(d, k, bits, kv, Sm, Sc, Sp) * dth;
      }
    }
    To[id] = T;
    So[id] = S;
    if (IMPL) {  // the column solve and the rotation follow
      uo[id] = u;
      vo[id] = v;
    } else {
      uo[id] = rc * u + rs * v;
      vo[id] = -rs * u + rc * v;
    }
    um = uc;
    vm = vc;
    Tm = Tc;
    Sm = Sc;
  }
}

// The biharmonic and implicit-diffusion options are template arguments: a
// launch carries only the operators its option set uses.
static_assert(sizeof(LtTile) <= 48 * 1024, "k_lin_t tile within the default dynamic shared memory");
void launch_lin_t(cudaStream_t s, const Dev& d, const float* usub, const float* vsub, const float* u0,
                  const float* v0, const float* T0, const float* S0, float* uo, float* vo, float* To, float* So,
                  float dth, int implicit_v) {
  const dim3 g((d.nx + LT_X - 1) / LT_X, (d.ny + LT_Y - 1) / LT_Y, (d.nz + d.lt_kc - 1) / d.lt_kc), b(LT_X, LT_Y);
  const int key = (d.nu_bi > 0.f ? 4 : 0) | (d.kappa_bi > 0.f ? 2 : 0) | (implicit_v ? 1 : 0);
  const size_t sm = sizeof(LtTile);
#define ZM_LIN(K, UV, TS, IM)                                                                       \
  case K:                                                                                           \
    (void)launch_pdl(k_lin_t<UV, TS, IM>, g, b, sm, s, d, usub, vsub, u0, v0, T0, S0, uo, vo, To, So, dth); \
    break;
  switch (key) {
    ZM_LIN(0, false, false, false)
    ZM_LIN(1, false, false, true)
    ZM_LIN(2, false, true, false)
    ZM_LIN(3, false, true, true)
    ZM_LIN(4, true, false, false)
    ZM_LIN(5, true, false, true)
    ZM_LIN(6, true, true, false)
    ZM_LIN(7, true, true, true)
  }
#undef ZM_LIN
}

// Backward-Euler vertical diffusion (extension: the implicit replacement of
// the explicit L-step vertical diffusion).  The matrix is (I - s D2) with D2
// the node-form operator of d2z on the wet levels 0..kbot (ghost fill below);
// Thomas algorithm in FP32 plus one step of iterative refinement, residual
// formed in FP32 against the original right-hand side.  Rows below the
// deepest wet level are untouched.
__device__ __forceinline__ void vcoef(const Dev& d, int k, int kb, float s, float& a, float& b, float& c) {
  a = 0.f; c = 0.f; b = 1.f;
  if (k == 0) { b += s * d.vc.d2_top; c = -s * d.vc.d2_top; return; }
  if (k == d.nz - 1) { a = -s * d.vc.d2_bot; b += s * d.vc.d2_bot; return; }
  a = -s * d.vc.d2_lo[k];
  b += s * (d.vc.d2_lo[k] + d.vc.d2_hi[k]);
  if (k < kb) c = -s * d.vc.d2_hi[k]; else b -= s * d.vc.d2_hi[k];
}

// One thread per (column, field); lanes 2c and 2c+1 hold u and v (blockIdx.z
// = 0: nu_v, node form of d2z with the ghost fill, then the land hold and the
// exact Coriolis rotation, which swaps values within the lane pair) or T and S
// (blockIdx.z = 1: kappa_v + coastal in the node form, or the learned
// closure's diffusivity per interface kap3 in the interface-flux form, then
// the land hold).  Each thread runs its own sequential Thomas sweeps (the two
// fields of a pair repeat the same pivots).  The sweeps are latency-bound, so
// the kernel is held to 32 registers for full occupancy: more independent
// column chains in flight per SM outweigh a few spilled scalars and the
// per-thread level arrays in local memory.  Passes over the n = kbot + 1 wet
// levels:
//   1. forward elimination, keeping 1 / pivot;
//   2. back substitution: the FP32 solution x;
//   3. the residual r - A x (r read again) and its forward elimination;
//   4. back substitution of the correction e; x + e, hold, rotation, store.
// The factor up / pivot is formed again where it is needed.
template <bool KAP>
__global__ void __launch_bounds__(IV_T, 32) k_implicit_vdiff(Dev d, float* __restrict__ u, float* __restrict__ v,
                                                        float* __restrict__ T, float* __restrict__ S,
                                                        const float* __restrict__ u0, const float* __restrict__ v0,
                                                        const float* __restrict__ T0, const float* __restrict__ S0,
                                                        float dth, const float* __restrict__ kap3) {
  const int f = threadIdx.x & 1;
  const int i = blockIdx.x * (IV_T / 2) + (threadIdx.x >> 1);
  const int j = blockIdx.y;
  const bool tracers = blockIdx.z == 1;
  const bool in = i < d.nx;  // lanes past the last column run along (the pair exchange needs every lane) unstored
  const long long base = idx2(d, j, in ? i : d.nx - 1);
  float* __restrict__ fld = tracers ? (f ? S : T) : (f ? v : u);
  const float* __restrict__ hold = tracers ? (f ? S0 : T0) : (f ? v0 : u0);
  const bool kap = KAP && tracers;  // the u, v blocks of a closure launch keep nu_v
  const uint64_t bits = wb(d, j, in ? i : d.nx - 1);
  const int kb = kbot_of(bits);
  const int n = kb > 0 && wetb(bits, 0) ? kb + 1 : 0;
  const float sc = tracers ? __ldg(d.kv2 + base) * dth : d.nu_v * dth;
  const long long pl = d.plane;
  float x[ZM_MAXZ], inv[ZM_MAXZ], e[ZM_MAXZ], kq[KAP ? ZM_MAXZ : 1];
  for (int k = 0; k < n; ++k) {
    x[k] = fld[base + k * pl];
    if (KAP && kap && k + 1 < n) kq[k] = __ldg(kap3 + base + k * pl);
  }
  // tridiagonal row k: lower lo, diagonal dg, upper up
  auto row = [&](int k, float& lo, float& dg, float& up) {
    if (KAP && kap) {
      lo = k > 0 ? -dth * kq[k - 1] * d.vc.inv_dz_iface[k - 1] * d.vc.inv_dz_node[k] : 0.f;
      up = k + 1 < n ? -dth * kq[k] * d.vc.inv_dz_iface[k] * d.vc.inv_dz_node[k] : 0.f;
      dg = 1.f - lo - up;
    } else {
      vcoef(d, k, kb, sc, lo, dg, up);
    }
  };
  // 1. forward elimination (lo = 0 in row 0, so its pivot is dg)
  {
    float cpp = 0.f, y = 0.f;
    for (int k = 0; k < n; ++k) {
      float lo, dg, up;
      row(k, lo, dg, up);
      const float iv = 1.f / (dg - lo * cpp);
      cpp = up * iv;
      y = (x[k] - lo * y) * iv;
      x[k] = y;
      inv[k] = iv;
    }
  }
  // 2. back substitution
  for (int k = n - 2; k >= 0; --k) {
    float lo, dg, up;
    row(k, lo, dg, up);
    x[k] -= (up * inv[k]) * x[k + 1];
  }
  // 3. residual of the FP32 solution, eliminated with the same factorization
  {
    float ep = 0.f, xm = 0.f, x0 = n > 0 ? x[0] : 0.f;
    for (int k = 0; k < n; ++k) {
      float lo, dg, up;
      row(k, lo, dg, up);
      const float xp = k + 1 < n ? x[k + 1] : 0.f;
      float a = dg * x0;
      if (k > 0) a += lo * xm;
      if (k + 1 < n) a += up * xp;
      ep = ((fld[base + k * pl] - a) - lo * ep) * inv[k];
      e[k] = ep;
      xm = x0;
      x0 = xp;
    }
  }
  // 4. back substitution of the correction; x + e, land hold, rotation
  const float rc = tracers ? 0.f : __ldg(d.rot_c + base), rs = tracers ? 0.f : __ldg(d.rot_s + base);
  float en = 0.f;
  for (int k = d.nz - 1; k >= 0; --k) {
    const long long id = base + k * pl;
    const bool wet = wetb(bits, k);
    float val = 0.f;
    if (k < n) {
      float ek = e[k];
      if (k + 1 < n) {
        float lo, dg, up;
        row(k, lo, dg, up);
        ek -= (up * inv[k]) * en;
      }
      en = ek;
      val = x[k] + ek;
    } else if (!tracers && wet) {
      val = fld[id];
    }
    if (!wet) val = ld(hold, id);
    if (tracers) {
      if (in && (k < n || !wet)) fld[id] = val;
    } else {
      const float other = __shfl_xor_sync(0xffffffffu, val, 1);
      const float uu = f ? other : val, vv = f ? val : other;
      if (in) fld[id] = f ? -rs * uu + rc * vv : rc * uu + rs * vv;
    }
  }
}

void launch_implicit_vdiff(cudaStream_t s, const Dev& d, float* u, float* v, float* T, float* S, const float* u0,
                           const float* v0, const float* T0, const float* S0, float dth, const float* kap3) {
  const dim3 g((d.nx + IV_T / 2 - 1) / (IV_T / 2), d.ny, 2);
  if (kap3) k_implicit_vdiff<true><<<g, IV_T, 0, s>>>(d, u, v, T, S, u0, v0, T0, S0, dth, kap3);
  else k_implicit_vdiff<false><<<g, IV_T, 0, s>>>(d, u, v, T, S, u0, v0, T0, S0, dth, kap3);
}

// ------------------------------------------------------------------ transport
// Interface volume transport Fz[k] = sum_{m>=k} div_h[m] dz_node[m]
// (dynamics/transport.py:110-133 with the face-flux divergence of
// numerics/horizontal.py:255-281); Fz[nz] = 0 is implicit.  A block owns a
// FZ_X x RY tile of columns (RY = d.fz_rows) and marches up from the bottom level: each
// level's u and v on the tile and a one-cell halo arrive in shared memory by
// cp.async, FZ_NB - 1 levels ahead, so each value is fetched once; one column
// per thread accumulates the sum.
constexpr int FZ_X = 32, FZ_NB = 4;  // tile columns, level buffers
constexpr int FZ_PX = FZ_X + 2;

template <int RY>
__global__ void __launch_bounds__(FZ_X * RY) k_fz(Dev d, const float* __restrict__ u, const float* __restrict__ v,
                                                    float* __restrict__ Fz) {
  constexpr int FZ_PY = RY + 2, FZ_CELLS = FZ_PX * FZ_PY;
  static_assert(FZ_CELLS <= 2 * FZ_X * RY, "two tile cells per thread at most");
  pdl_trigger();
  __shared__ float su[FZ_NB][FZ_PY][FZ_PX], sv[FZ_NB][FZ_PY][FZ_PX];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * FZ_X + tx;
  const int i0 = blockIdx.x * FZ_X, j0 = blockIdx.y * RY;
  const int i = i0 + tx, j = j0 + ty;
  // threads outside the grid copy their tile cells and meet the barriers, nothing else
  const bool in = i < d.nx && j < d.ny;
  const int e0 = tid, e1 = tid + FZ_X * RY;
  const bool has1 = e1 < FZ_CELLS;
  const int s0 = tile_cell<FZ_PX>(d, e0, i0, j0), s1 = has1 ? tile_cell<FZ_PX>(d, e1, i0, j0) : 0;
  auto issue = [&](int q) {  // the q-th level from the bottom into buffer q % FZ_NB; one commit group per call
    if (q < d.nz) {
      const long long off = (long long)(d.nz - 1 - q) * d.plane;
      float* bu = &su[q % FZ_NB][0][0];
      float* bv = &sv[q % FZ_NB][0][0];
      cp_async4(bu + e0, u + off + s0);
      cp_async4(bv + e0, v + off + s0);
      if (has1) {
        cp_async4(bu + e1, u + off + s1);
        cp_async4(bv + e1, v + off + s1);
      }
    }
    cp_async_commit();
  };
  const int ic = in ? i : 0, jc = in ? j : 0;
  const Nb n = nb(d, jc, ic);
  const uint64_t m0 = wb(d, jc, ic), me = wb(d, jc, n.ie), mw = wb(d, jc, n.iw);
  const uint64_t mn = wb(d, n.jn, ic), ms = wb(d, n.js, ic);
  const long long cc = idx2(d, jc, ic);
  const float idx_c = __ldg(d.inv_dx + cc);
  const float cf_n = __ldg(d.cfp + jc), cf_s = jc > 0 ? __ldg(d.cfp + jc - 1) : 0.f;
  const float yscale = d.inv_dy * __ldg(d.inv_cos + jc);
  float acc = 0.f;
  // wet flags with level nz - 1 in bit 63, shifted up one level per iteration (the march runs upwards)
  const int up = 64 - d.nz;
  uint64_t f0 = m0 << up, fe = me << up, fw = mw << up, fn = mn << up, fs = ms << up;
  pdl_wait();  // u, v come from the preceding kernel
#pragma unroll
  for (int q = 0; q < FZ_NB - 1; ++q) issue(q);
  const int r = ty + 1, c = tx + 1;
  for (int q = 0; q < d.nz; ++q) {
    cp_async_wait<FZ_NB - 2>();  // this thread's copies of level q are done
    __syncthreads();             // everyone's are, and level q - 1's buffer is free
    issue(q + FZ_NB - 1);
    if (!in) continue;
    const int k = d.nz - 1 - q, bq = q % FZ_NB;
    const float uc = su[bq][r][c], ue = su[bq][r][c + 1], uw = su[bq][r][c - 1];
    const float w0 = (float)(unsigned)(f0 >> 63), we = (float)(unsigned)(fe >> 63),
                ww = (float)(unsigned)(fw >> 63), wn = (float)(unsigned)(fn >> 63),
                ws = (float)(unsigned)(fs >> 63);
    f0 <<= 1; fe <<= 1; fw <<= 1; fn <<= 1; fs <<= 1;
    const float fxe = 0.5f * (uc + ue) * w0 * we;
    const float fxw = 0.5f * (uw + uc) * ww * w0;
    float fyn = 0.f, fys = 0.f;
    const float vc = sv[bq][r][c];
    if (jc < d.ny - 1) fyn = 0.5f * (vc + sv[bq][r + 1][c]) * w0 * wn * cf_n;
    if (jc > 0) fys = 0.5f * (sv[bq][r - 1][c] + vc) * ws * w0 * cf_s;
    const float div = (fxe - fxw) * idx_c + (fyn - fys) * yscale;
    acc += div * d.vc.dz_node[k];
    Fz[(long long)k * d.plane + cc] = acc;
  }
}

cudaError_t launch_nu_tb(cudaStream_t s, const Dev& d, int warps, const float* u, const float* v, float* uo,
                         float* vo, float c, int nsub, int halo) {
  const int TI = NB_W - 2 * halo, TJ = warps * NB_R - 2 * halo;
  const dim3 grd((d.nx + TI - 1) / TI, (d.ny + TJ - 1) / TJ, d.nz);
  if (warps == 16) return launch_pdl(k_nu_tb<16>, grd, dim3(32, 16), 0, s, d, u, v, uo, vo, c, nsub, halo);
  return launch_pdl(k_nu_tb<8>, grd, dim3(32, 8), 0, s, d, u, v, uo, vo, c, nsub, halo);
}

void launch_fz(cudaStream_t s, const Dev& d, const float* u, const float* v, float* Fz) {
  if (d.fz_rows == 8)
    (void)launch_pdl(k_fz<8>, dim3((d.nx + FZ_X - 1) / FZ_X, (d.ny + 7) / 8), dim3(FZ_X, 8), 0, s, d, u, v, Fz);
  else
    (void)launch_pdl(k_fz<4>, dim3((d.nx + FZ_X - 1) / FZ_X, (d.ny + 3) / 4), dim3(FZ_X, 4), 0, s, d, u, v, Fz);
}

// Raw advective-form momentum advection -(u d/dx + v d/dy + w d/dz) of u and
// v (dynamics/transport.py:169-197 before its filter) with the latitude half
// of the dealias filter, [1,4,6,4,1]/16 on edge-held rows
// (numerics/horizontal.py:283-305).  The longitude 2/3-rule half runs in the
// FFT kernel; the two filters act on different axes and commute.
__device__ __forceinline__ void adv_point(const Dev& d, const float* __restrict__ u, const float* __restrict__ v,
                                          const float* __restrict__ Fz, int k, int j, int i, float& au, float& av) {
  const Nb n = nb(d, j, i);
  const long long b = (long long)k * d.plane;
  const uint64_t m0 = wb(d, j, i);
  const float w0 = wetf(m0, k);
  if (w0 == 0.f) { au = 0.f; av = 0.f; return; }
  const float we = wetf(wb(d, j, n.ie), k), ww = wetf(wb(d, j, n.iw), k);
  const float wn = wetf(wb(d, n.jn, i), k), ws = wetf(wb(d, n.js, i), k);
  const long long c = b + idx2(d, j, i);
  const float uc = ld(u, c), vc = ld(v, c);
  const float ue = ld(u, b + idx2(d, j, n.ie)), uw = ld(u, b + idx2(d, j, n.iw));
  const float un = ld(u, b + idx2(d, n.jn, i)), us = ld(u, b + idx2(d, n.js, i));
  const float ve = ld(v, b + idx2(d, j, n.ie)), vw = ld(v, b + idx2(d, j, n.iw));
  const float vn = ld(v, b + idx2(d, n.jn, i)), vs = ld(v, b + idx2(d, n.js, i));
  const float hx = __ldg(d.inv_dx + idx2(d, j, i)) * 0.5f, hy = d.inv_dy * 0.5f;
  const float dudx = hx * ((ue - uc) * w0 * we + (uc - uw) * w0 * ww);
  const float dvdx = hx * ((ve - vc) * w0 * we + (vc - vw) * w0 * ww);
  const float dudy = hy * ((un - uc) * wn * w0 + (uc - us) * w0 * ws);
  const float dvdy = hy * ((vn - vc) * wn * w0 + (vc - vs) * w0 * ws);
  // d/dz of the ghost-filled column (numerics/vertical.py:267-272)
  const int kb = kbot_of(m0);
  const long long base = idx2(d, j, i);
  float dudz, dvdz;
  if (k == 0) {
    const float inv = d.vc.ddz_inv[0];
    dudz = (colv(u, base, d.plane, 1, kb) - colv(u, base, d.plane, 0, kb)) * inv;
    dvdz = (colv(v, base, d.plane, 1, kb) - colv(v, base, d.plane, 0, kb)) * inv;
  } else if (k == d.nz - 1) {
    const float inv = d.vc.ddz_inv[k];
    dudz = (colv(u, base, d.plane, k, kb) - colv(u, base, d.plane, k - 1, kb)) * inv;
    dvdz = (colv(v, base, d.plane, k, kb) - colv(v, base, d.plane, k - 1, kb)) * inv;
  } else {
    const float inv = d.vc.ddz_inv[k];
    dudz = (colv(u, base, d.plane, k + 1, kb) - colv(u, base, d.plane, k - 1, kb)) * inv;
    dvdz = (colv(v, base, d.plane, k + 1, kb) - colv(v, base, d.plane, k - 1, kb)) * inv;
  }
  const float w = -ld(Fz, c) * w0;  // dynamics/transport.py:149-166
  au = -(uc * dudx + vc * dudy + w * dudz);
  av = -(uc * dvdx + vc * dvdy + w * dvdz);
}

// One block: 32 columns x MADV_TY (60) rows of one level.  The 8 warps take 8
// of the 64 rows (tile and a 2-row halo on each side) per pass, so the halo
// adds 7 % of the point work (50 % with 8-row tiles).
__global__ void __launch_bounds__(256) k_madv(Dev d, const float* __restrict__ u, const float* __restrict__ v,
                                              const float* __restrict__ Fz, float* __restrict__ Ayu,
                                              float* __restrict__ Ayv) {
  pdl_trigger();
  __shared__ float su[MADV_TY + 4][32];
  __shared__ float sv[MADV_TY + 4][32];
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j0 = blockIdx.y * MADV_TY;
  const int k = blockIdx.z;
  pdl_wait();  // u, v, Fz come from the preceding kernels
  for (int r = threadIdx.y; r < MADV_TY + 4; r += blockDim.y) {
    int jj = j0 - 2 + r;
    jj = jj < 0 ? 0 : (jj >= d.ny ? d.ny - 1 : jj);
    float au = 0.f, av = 0.f;
    if (i < d.nx) adv_point(d, u, v, Fz, k, jj, i, au, av);
    su[r][threadIdx.x] = au;
    sv[r][threadIdx.x] = av;
  }
  __syncthreads();
  // rows j-2..j+2 clamped to the domain: with the tile loaded on clamped rows
  // the clamp is already applied at the tile edges except inside the tile.
  auto row = [&](int jj) { jj = jj < 0 ? 0 : (jj >= d.ny ? d.ny - 1 : jj); return jj - (j0 - 2); };
  const int t = threadIdx.x;
  for (int jr = threadIdx.y; jr < MADV_TY; jr += blockDim.y) {
    const int j = j0 + jr;
    if (i >= d.nx || j >= d.ny) continue;
    const float fu = (su[row(j - 2)][t] + 4.f * su[row(j - 1)][t] + 6.f * su[row(j)][t] + 4.f * su[row(j + 1)][t] +
                      su[row(j + 2)][t]) / 16.f;
    const float fv = (sv[row(j - 2)][t] + 4.f * sv[row(j - 1)][t] + 6.f * sv[row(j)][t] + 4.f * sv[row(j + 1)][t] +
                      sv[row(j + 2)][t]) / 16.f;
    const long long id = idx3(d, k, j, i);
    Ayu[id] = fu;
    Ayv[id] = fv;
  }
}

// Minmod slope over wet neighbours (dynamics/transport.py:199-213).
__device__ __forceinline__ float minmod_slope(float cm, float c0, float cp, float wm, float w0, float wp) {
  // 0.5 (sign l + sign r) min(|l|, |r|): +-min when l and r share a sign, else 0
  const float l = c0 - cm, r = cp - c0;
  const float m = fminf(fabsf(l), fabsf(r));
  const float s = (l > 0.f && r > 0.f) ? m : ((l < 0.f && r < 0.f) ? -m : 0.f);
  return s * w0 * wm * wp;
}

// Tracer advection substep (dynamics/tendencies.py:111-140 with
// _advection_scalar, dynamics/transport.py:365-475).  A block owns a
// TA_X x TA_Y tile of columns and marches down d.ta_kc levels of them (the
// chunks of a column are separate blocks, so the grid fills the GPU in even
// waves): T, S, u, v of each
// level on the tile with a two-cell halo (for the minmod slopes of the face
// states) arrive in shared memory by cp.async one level ahead, in TA_NB
// rotating buffers; the level's wet flags are formed one level ahead from the
// cells' bitmasks, held in registers.  Each thread forms the four faces of its
// point, T and S together; the vertical donor-cell flux takes the level above
// from registers and the level below from the next buffer.  Rows beyond the
// closed walls are loaded from the clamped row, which is the edge padding of
// transport.py:199-290; longitude wraps.
constexpr int TA_H = 2, TA_NB = 3;
constexpr int TA_PX = TA_X + 2 * TA_H, TA_PY = TA_Y + 2 * TA_H;
constexpr int TA_CELLS = TA_PX * TA_PY;
static_assert(TA_CELLS <= 2 * TA_X * TA_Y, "two tile cells per thread at most");

struct TaTile {
  float2 ts[TA_NB][TA_PY][TA_PX];  // (T, S) of a cell, side by side for the paired FP32 face arithmetic
  float u[TA_NB][TA_PY][TA_PX];
  float v[TA_NB][TA_PY][TA_PX];
  float w[2][TA_PY][TA_PX];
};

// Limited face value of one tracer (transport.py:199-290).  With the upwind
// triple (a, b, c) = (c-, c0, c1) for a flow towards +, (c+, c1, c0) towards -,
// the minmod face state is b + 0.5 minmod(a, b, c): for the negative
// direction minmod(c+, c1, c0) = -minmod(c0, c1, c+) exactly, so this is
// c1 - 0.5 minmod(c0, c1, c+) without a divergent branch.  LIM: 2 minmod
// (fct_adv), 1 donor cell (monotone_adv), 0 centred.
template <int LIM>
__device__ __forceinline__ float ta_face_value(bool pos, float cm, float c0, float c1, float cp, float wm,
                                               float w0, float w1, float wp) {
  if (LIM == 2) {
    const float a = pos ? cm : cp, b = pos ? c0 : c1, c = pos ? c1 : c0;
    const float wa = pos ? wm : wp, wb = pos ? w0 : w1, wc = pos ? w1 : w0;
    return b + 0.5f * minmod_slope(a, b, c, wa, wb, wc);
  }
  if (LIM == 1) return pos ? c0 : c1;
  return 0.5f * (c0 + c1);
}

// Minmod slopes of T and S at once (dynamics/transport.py:199-213): the
// differences on the paired FP32 instructions, the sign test per tracer.
__device__ __forceinline__ float2 minmod_slope2(float2 cm, float2 c0, float2 cp) {
  const float2 m1 = f2(-1.f);
  const float2 l = __ffma2_rn(cm, m1, c0), r = __ffma2_rn(c0, m1, cp);
  // l and r of one sign <=> l r > 0 (both differences of float32 tracer
  // anomalies, so the product underflows only where both are below 1e-19, and
  // the slope dropped there is below that too); NaN compares false, as in the
  // sign form
  const float2 lr = __fmul2_rn(l, r);
  const float mx = fminf(fabsf(l.x), fabsf(r.x)), my = fminf(fabsf(l.y), fabsf(r.y));
  return make_float2(lr.x > 0.f ? copysignf(mx, l.x) : 0.f, lr.y > 0.f ? copysignf(my, l.y) : 0.f);
}

// Limited (T, S) face state, the paired form of ta_face_value.  The wet
// weights are 0 or 1, so applying their product once to both slopes rounds
// like the per-tracer product s w0 wm wp.
template <int LIM>
__device__ __forceinline__ float2 ta_face_value2(bool pos, float2 cm, float2 c0, float2 c1, float2 cp, float wm,
                                                 float w0, float w1, float wp) {
  if (LIM == 2) {
    const float2 a = pos ? cm : cp, b = pos ? c0 : c1, c = pos ? c1 : c0;
    const float wgt = pos ? w0 * wm * w1 : w1 * wp * w0;
    return __ffma2_rn(f2(0.5f * wgt), minmod_slope2(a, b, c), b);
  }
  if (LIM == 1) return pos ? c0 : c1;
  return __fmul2_rn(f2(0.5f), __fadd2_rn(c0, c1));
}

// (T, S) fluxes through the x face between tile columns cc and cc+1 of row r
// of level buffer q (wet flags in buffer wq)
template <int LIM>
__device__ __forceinline__ float2 ta_faces_x(const TaTile& t, int q, int wq, int r, int cc) {
  const float w0 = t.w[wq][r][cc], we = t.w[wq][r][cc + 1];
  const float ux = 0.5f * (t.u[q][r][cc] + t.u[q][r][cc + 1]);
  const bool pos = ux >= 0.f;
  const float wm = t.w[wq][r][cc - 1], wp = t.w[wq][r][cc + 2];
  const float2 c = ta_face_value2<LIM>(pos, t.ts[q][r][cc - 1], t.ts[q][r][cc], t.ts[q][r][cc + 1],
                                       t.ts[q][r][cc + 2], wm, w0, we, wp);
  return __fmul2_rn(f2(ux * (w0 * we)), c);
}

// (T, S) fluxes through the y face between tile rows r and r+1 (global rows
// gj, gj+1); zero through the closed walls
template <int LIM>
__device__ __forceinline__ float2 ta_faces_y(const Dev& d, const TaTile& t, int q, int wq, int r, int cc, int gj) {
  if (gj < 0 || gj >= d.ny - 1) return f2(0.f);
  const float w0 = t.w[wq][r][cc], wn = t.w[wq][r + 1][cc];
  const float vy = 0.5f * (t.v[q][r][cc] + t.v[q][r + 1][cc]);
  const bool pos = vy >= 0.f;
  const float wm = t.w[wq][r - 1][cc], wp = t.w[wq][r + 2][cc];
  const float2 c = ta_face_value2<LIM>(pos, t.ts[q][r - 1][cc], t.ts[q][r][cc], t.ts[q][r + 1][cc],
                                       t.ts[q][r + 2][cc], wm, w0, wn, wp);
  return __fmul2_rn(__fmul2_rn(f2(vy * (w0 * wn)), c), f2(__ldg(d.cfp + gj)));
}

template <int LIM>
__global__ void __launch_bounds__(TA_X * TA_Y, 5) k_tracer_adv_t(Dev d, const float* __restrict__ T,
                                                                 const float* __restrict__ S,
                                                                 const float* __restrict__ u,
                                                                 const float* __restrict__ v,
                                                                 const float* __restrict__ Fz,
                                                                 float* __restrict__ accT, float* __restrict__ accS,
                                                                 float* __restrict__ Tn, float* __restrict__ Sn,
                                                                 float dts, int first, int last,
                                                                 float* __restrict__ topT,
                                                                 float* __restrict__ topS) {
  pdl_trigger();
  __shared__ TaTile t;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TA_X + tx;
  const int i0 = blockIdx.x * TA_X, j0 = blockIdx.y * TA_Y;
  const int i = i0 + tx, j = j0 + ty;
  // threads outside the grid copy their tile cells, form their wet flags and
  // meet the barriers, nothing else
  const bool in = i < d.nx && j < d.ny;
  const int e0 = tid, e1 = tid + TA_X * TA_Y;
  const bool has1 = e1 < TA_CELLS;
  const int s0 = tile_cell<TA_PX, TA_H>(d, e0, i0, j0), s1 = has1 ? tile_cell<TA_PX, TA_H>(d, e1, i0, j0) : 0;
  const uint64_t b0 = __ldg(d.wbits + s0), b1 = has1 ? __ldg(d.wbits + s1) : 0ull;
  const int k0 = blockIdx.z * d.ta_kc, k1 = min(d.nz, k0 + d.ta_kc);  // this block's levels
  auto issue = [&](int k) {  // level k into buffer k % TA_NB; one commit group per call
    if (k < d.nz && k <= k1) {  // level k1 only for the column neighbour below the chunk
      const long long off = (long long)k * d.plane;
      const int q = k % TA_NB;
      float* ts = &t.ts[q][0][0].x;
      cp_async4(ts + 2 * e0, T + off + s0);
      cp_async4(ts + 2 * e0 + 1, S + off + s0);
      cp_async4(&t.u[q][0][0] + e0, u + off + s0);
      cp_async4(&t.v[q][0][0] + e0, v + off + s0);
      if (has1) {
        cp_async4(ts + 2 * e1, T + off + s1);
        cp_async4(ts + 2 * e1 + 1, S + off + s1);
        cp_async4(&t.u[q][0][0] + e1, u + off + s1);
        cp_async4(&t.v[q][0][0] + e1, v + off + s1);
      }
    }
    cp_async_commit();
  };
  // wet flags of the two tile cells, bit 0 = the next level wet_level forms
  uint64_t rb0 = b0 >> k0, rb1 = b1 >> k0;
  auto wet_level = [&](int k) {  // wet flags of level k into w[k % 2]; called for k0, k0 + 1, ... in turn
    if (k < d.nz) {
      float* pw = &t.w[k & 1][0][0];
      pw[e0] = (float)(unsigned)(rb0 & 1ull);
      if (has1) pw[e1] = (float)(unsigned)(rb1 & 1ull);
      rb0 >>= 1;
      rb1 >>= 1;
    }
  };
  pdl_wait();  // the tracers, velocities and Fz come from the preceding kernels
  issue(k0);
  issue(k0 + 1);
  wet_level(k0);
  const int ic = in ? i : 0, jc = in ? j : 0;
  const long long base = idx2(d, jc, ic);
  const uint64_t bits = __ldg(d.wbits + base);
  const int kbt = kbot_of(bits);
  const float ix = __ldg(d.inv_dx + base), ysc = d.inv_dy * __ldg(d.inv_cos + jc);
  const int r = ty + TA_H, cc = tx + TA_H;
  // (T, S) of the level above and Fz of the current level
  float2 cm = k0 > 0 ? make_float2(ld(T, base + (long long)(k0 - 1) * d.plane),
                                   ld(S, base + (long long)(k0 - 1) * d.plane))
                     : f2(0.f);
  float fzk = ld(Fz, base + (long long)k0 * d.plane);
  // the column's own wet flags: level k - 1 in wup, level k + 1 in bit 1 of cb
  float wup = k0 > 0 ? wetf(bits, k0 - 1) : 0.f;
  uint64_t cb = bits >> k0;
  for (int k = k0; k < k1; ++k) {
    cp_async_wait<0>();  // this thread's copies of levels k and k + 1 are done
    __syncthreads();     // everyone's are, w[k % 2] is formed, level k - 1's buffers are free
    issue(k + 2);
    wet_level(k + 1);
    const long long id = (long long)k * d.plane + base;
    const float fzn = k + 1 < d.nz ? ld(Fz, id + d.plane) : 0.f;
    if (!in) continue;
    const int q = k % TA_NB, qn = (k + 1) % TA_NB, wq = k & 1;
    const float w0 = t.w[wq][r][cc];
    const float2 ck = t.ts[q][r][cc];
    if (topT && k == 0) {  // ledger mode: the rigid-lid surface flux Fz[0] c[0] of the substep, summed
      topT[base] = (first ? 0.f : topT[base]) + fzk * ck.x;
      topS[base] = (first ? 0.f : topS[base]) + fzk * ck.y;
    }
    float2 a = f2(0.f);
    if (w0 != 0.f) {
      const float2 m1 = f2(-1.f);
      const float2 fxe = ta_faces_x<LIM>(t, q, wq, r, cc), fxw = ta_faces_x<LIM>(t, q, wq, r, cc - 1);
      const float2 fyn = ta_faces_y<LIM>(d, t, q, wq, r, cc, jc), fys = ta_faces_y<LIM>(d, t, q, wq, r - 1, cc, jc - 1);
      const float2 h = __ffma2_rn(__ffma2_rn(fxw, m1, fxe), f2(ix), __fmul2_rn(__ffma2_rn(fys, m1, fyn), f2(ysc)));
      // vertical donor-cell fluxes through the top (up) and bottom (dn) faces;
      // the wet weights are 0 or 1, so folding them into Fz rounds like the
      // product Fz c g
      float2 up, dn = f2(0.f);
      if (k == 0) {
        up = __fmul2_rn(f2(fzk), ck);
      } else {
        up = __fmul2_rn(f2(fzk * (wup * w0)), fzk > 0.f ? cm : ck);
      }
      if (k + 1 < d.nz) {
        // ghost fill below the deepest wet level: node k+1 carries node k's value
        const float2 cn = k + 1 <= kbt ? t.ts[qn][r][cc] : ck;
        dn = __fmul2_rn(f2(fzn * (w0 * (float)(unsigned)((cb >> 1) & 1ull))), fzn > 0.f ? ck : cn);
      }
      a = __fmul2_rn(__ffma2_rn(__ffma2_rn(up, m1, dn), f2(d.vc.inv_dz_node[k]), h), f2(-w0));
    }
    accT[id] = first ? a.x : accT[id] + a.x;
    accS[id] = first ? a.y : accS[id] + a.y;
    if (!last) {
      const float2 cnew = __ffma2_rn(a, f2(dts), ck);
      Tn[id] = cnew.x;
      Sn[id] = cnew.y;
    }
    cm = ck;
    fzk = fzn;
    wup = (float)(unsigned)(cb & 1ull);
    cb >>= 1;
  }
}

// The face limiter is a template argument: the face arithmetic is specialised
// instead of branching on it at every face.
void launch_tracer_adv(cudaStream_t s, const Dev& d, const float* T, const float* S, const float* u, const float* v,
                       const float* Fz, float* accT, float* accS, float* Tn, float* Sn, float dts, int first, int last,
                       float* topT, float* topS) {
  const dim3 g((d.nx + TA_X - 1) / TA_X, (d.ny + TA_Y - 1) / TA_Y, (d.nz + d.ta_kc - 1) / d.ta_kc), b(TA_X, TA_Y);
  auto kern = d.limiter == 2 ? k_tracer_adv_t<2> : (d.limiter == 1 ? k_tracer_adv_t<1> : k_tracer_adv_t<0>);
  (void)launch_pdl(kern, g, b, 0, s, d, T, S, u, v, Fz, accT, accS, Tn, Sn, dts, first, last, topT, topS);
}

// Temperature-term decomposition of a state (dynamics/tendencies.py:74-92,
// the terms_fn of factory.py:762-764), a read-only diagnosis outside the
// step: advection (one evaluation of transport.py:365-475, limiter faces as
// in k_tracer_adv_t), wet-face horizontal diffusion with kappa_h + coastal
// (horizontal.py:217-243), vertical diffusion with kappa_v + coastal
// (physics/vertical.py:45-53) and the interface-flux convective tendency
// (physics/vertical.py:13-37, 63-82) with kappa_conv, each times the wet
// mask.  One column per thread marching down; neighbours by global loads
// (rows clamped at the walls, longitude wrapped).  T and S are anomalies:
// every term is a difference operator of T, or (advection) a flux divergence
// whose constant part cancels through the continuity inverse Fz.
template <int LIM>
__global__ void __launch_bounds__(128) k_tracer_terms(Dev d, const float* __restrict__ T,
                                                      const float* __restrict__ S, const float* __restrict__ u,
                                                      const float* __restrict__ v, const float* __restrict__ Fz,
                                                      float* __restrict__ adv, float* __restrict__ dh,
                                                      float* __restrict__ dv, float* __restrict__ conv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  int ci[5], rj[5];  // columns i-2..i+2 (wrapped), rows j-2..j+2 (clamped)
#pragma unroll
  for (int o = 0; o < 5; ++o) {
    int g = (i + o - 2) % d.nx;
    ci[o] = g < 0 ? g + d.nx : g;
    rj[o] = min(max(j + o - 2, 0), d.ny - 1);
  }
  uint64_t wx[5], wy[5];
#pragma unroll
  for (int o = 0; o < 5; ++o) {
    wx[o] = wb(d, j, ci[o]);
    wy[o] = wb(d, rj[o], i);
  }
  const long long base = idx2(d, j, i);
  const uint64_t bits = wx[2];
  const int kbt = kbot_of(bits);
  const float ix = __ldg(d.inv_dx + base), ysc = d.inv_dy * __ldg(d.inv_cos + j);
  const float kv = __ldg(d.kv2 + base);
  const float cfn = j < d.ny - 1 ? __ldg(d.cfp + j) : 0.f, cfs = j > 0 ? __ldg(d.cfp + j - 1) : 0.f;
  // convective interfaces of the column (k_tracer_rest's gates)
  uint64_t unstable = 0ull, wetpair = 0ull;
  for (int m = 0; m + 1 < d.nz; ++m) {
    const long long a = (long long)m * d.plane + base, b = a + d.plane;
    if (wetb(bits, m) && wetb(bits, m + 1)) {
      wetpair |= 1ull << m;
      if (kBeta * (ld(S, a) - ld(S, b)) > kAlpha * (ld(T, a) - ld(T, b))) unstable |= 1ull << m;
    }
  }
  uint64_t allow = 0ull;
  if (unstable && d.kappa_conv > 0.f) allow = d.localize_conv ? unstable : wetpair;
  float fconv = 0.f;
  for (int k = 0; k < d.nz; ++k) {
    const long long pl = (long long)k * d.plane;
    const float w0 = wetf(bits, k);
    const float ck = ld(T, pl + base);
    const float ckm = k > 0 ? ld(T, pl - d.plane + base) : ck;
    const float ckp = k + 1 < d.nz ? ld(T, pl + d.plane + base) : ck;
    float tx[5], ty[5], mx[5], my[5];
#pragma unroll
    for (int o = 0; o < 5; ++o) {
      tx[o] = ld(T, pl + idx2(d, j, ci[o]));
      ty[o] = ld(T, pl + idx2(d, rj[o], i));
      mx[o] = wetf(wx[o], k);
      my[o] = wetf(wy[o], k);
    }
    float a_ = 0.f;
    if (w0 != 0.f) {
      // x faces east (i, i+1) and west (i-1, i)
      const float uc = ld(u, pl + base), ue = ld(u, pl + idx2(d, j, ci[3])), uw = ld(u, pl + idx2(d, j, ci[1]));
      const float uxe = 0.5f * (uc + ue), uxw = 0.5f * (uw + uc);
      const float fxe = uxe * ta_face_value<LIM>(uxe >= 0.f, tx[1], tx[2], tx[3], tx[4], mx[1], mx[2], mx[3], mx[4]) *
                        (mx[2] * mx[3]);
      const float fxw = uxw * ta_face_value<LIM>(uxw >= 0.f, tx[0], tx[1], tx[2], tx[3], mx[0], mx[1], mx[2], mx[3]) *
                        (mx[1] * mx[2]);
      // y faces north (j, j+1) and south (j-1, j); closed at the walls
      float fyn = 0.f, fys = 0.f;
      const float vc = ld(v, pl + base);
      if (j < d.ny - 1) {
        const float vy = 0.5f * (vc + ld(v, pl + idx2(d, rj[3], i)));
        fyn = vy * ta_face_value<LIM>(vy >= 0.f, ty[1], ty[2], ty[3], ty[4], my[1], my[2], my[3], my[4]) *
              (my[2] * my[3]) * cfn;
      }
      if (j > 0) {
        const float vy = 0.5f * (ld(v, pl + idx2(d, rj[1], i)) + vc);
        fys = vy * ta_face_value<LIM>(vy >= 0.f, ty[0], ty[1], ty[2], ty[3], my[0], my[1], my[2], my[3]) *
              (my[1] * my[2]) * cfs;
      }
      const float h = (fxe - fxw) * ix + (fyn - fys) * ysc;
      const float fz_k = ld(Fz, pl + base);
      float up, dn = 0.f;
      if (k == 0) {
        up = fz_k * ck;
      } else {
        up = fz_k * (fz_k > 0.f ? ckm : ck) * (wetf(bits, k - 1) * w0);
      }
      if (k + 1 < d.nz) {
        const float fz_n = ld(Fz, pl + d.plane + base);
        const float tn = k + 1 <= kbt ? ckp : ck;
        dn = fz_n * (fz_n > 0.f ? ck : tn) * (w0 * wetf(bits, k + 1));
      }
      a_ = -(h + (dn - up) * d.vc.inv_dz_node[k]) * w0;
    }
    adv[pl + base] = a_;
    dh[pl + base] = hdiff(d, T, d.kh2, k, nb(d, j, i)) * w0;
    dv[pl + base] = vdiff_c(d, k, bits, kv, ckm, ck, ckp) * w0;
    float g = 0.f;
    if (k + 1 < d.nz && ((allow >> k) & 1ull)) g = -d.kappa_conv * (ckp - ck) * d.vc.inv_dz_iface[k];
    conv[pl + base] = (fconv - g) * d.vc.inv_dz_node[k] * w0;
    fconv = g;
  }
}

void launch_tracer_terms(cudaStream_t s, const Dev& d, const float* T, const float* S, const float* u,
                         const float* v, const float* Fz, float* adv, float* dh, float* dv, float* conv) {
  const dim3 b(32, 4), g((d.nx + 31) / 32, (d.ny + 3) / 4);
  if (d.limiter == 2) k_tracer_terms<2><<<g, b, 0, s>>>(d, T, S, u, v, Fz, adv, dh, dv, conv);
  else if (d.limiter == 1) k_tracer_terms<1><<<g, b, 0, s>>>(d, T, S, u, v, Fz, adv, dh, dv, conv);
  else k_tracer_terms<0><<<g, b, 0, s>>>(d, T, S, u, v, Fz, adv, dh, dv, conv);
}

// Tracer residual of the N step (dynamics/tendencies.py:94-245) without the
// diffusion pair that the residual adds and removes again: mean advection
// rate + interface-flux convective mixing (physics/vertical.py:13-37, 63-82)
// + surface sources at k = 0.  One column per thread.
//   stage 1: dT1 = r(T1), Tp = T1 + dt dT1
//   stage 2: T2 = T1 + dt (dT1 + r(Tp)) / 2


__device__ __forceinline__ void rest_store(const Dev& d, const RestArgs& a, long long id, long long base, int k,
                                           float w, float rT, float rS) {
  if (k == 0) {  // surface sources (dynamics/tendencies.py:167-207, physics/surface.py:8-20)
    const float sst = ld(a.Tev, id), sss = ld(a.Sev, id);
    const float hf = w / (d.dz_surface * kRho0 * kCp);
    const float tatm = __ldg(d.tatm + base);
    rT += __ldg(d.qheat + base) * hf + d.lambda_bulk * (tatm - sst) * hf + __ldg(d.cbulk + base) * (tatm - sst) * hf +
          __ldg(d.rest_c + base) * (__ldg(d.rest_T + base) - sst);
    rS += d.restore_S * (__ldg(d.sref + base) - sss) + (sst <= d.ice_freeze ? d.ice_salt : 0.f);
  }
  rT *= w;
  rS *= w;
  if (a.stage == 1) {
    a.dT1[id] = rT;
    a.dS1[id] = rS;
    a.To[id] = ld(a.Tbase, id) + rT * a.dt;
    a.So[id] = ld(a.Sbase, id) + rS * a.dt;
  } else {
    a.To[id] = ld(a.Tbase, id) + 0.5f * (ld(a.dT1, id) + rT) * a.dt;
    a.So[id] = ld(a.Sbase, id) + 0.5f * (ld(a.dS1, id) + rS) * a.dt;
  }
}

template <bool ST2>
__global__ void __launch_bounds__(128) k_tracer_rest(Dev d, RestArgs a) {
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const long long base = idx2(d, j, i);
  const uint64_t bits = wb(d, j, i);
  pdl_wait();  // the evaluation state and the advection rates come from the preceding kernels
  const int nz = d.nz;
  // static-instability gates of the evaluation state, in difference form:
  // rho[m] > rho[m+1]  <=>  beta (S[m]-S[m+1]) > alpha (T[m]-T[m+1]).
  uint64_t unstable = 0ull, wetpair = 0ull;
  float Tu = ld(a.Tev, base), Su = ld(a.Sev, base);
#pragma unroll 8
  for (int m = 0; m + 1 < nz; ++m) {
    const long long idn = base + (long long)(m + 1) * d.plane;
    const float Tl = ld(a.Tev, idn), Sl = ld(a.Sev, idn);
    if (wetb(bits, m) && wetb(bits, m + 1)) {
      wetpair |= 1ull << m;
      if (kBeta * (Su - Sl) > kAlpha * (Tu - Tl)) unstable |= 1ull << m;
    }
    Tu = Tl;
    Su = Sl;
  }
  uint64_t allow = 0ull;
  if (unstable && d.kappa_conv > 0.f && !a.no_conv) allow = d.localize_conv ? unstable : wetpair;
  if (a.nc == 1 || allow == 0ull) {
    const float kc = d.kappa_conv;
    float fT = 0.f, fS = 0.f;
    float cT = ld(a.Tev, base), cS = ld(a.Sev, base);
    // the next level's inputs are loaded before this level's stores: the
    // argument pointers may alias, so loads issued after a store would wait
    constexpr bool st2 = ST2;  // stage 2 reads the stage-1 tendency
    float qaT = ld(a.accT, base), qaS = ld(a.accS, base), qbT = ld(a.Tbase, base), qbS = ld(a.Sbase, base);
    float qdT = st2 ? ld(a.dT1, base) : 0.f, qdS = st2 ? ld(a.dS1, base) : 0.f;
#pragma unroll 2
    for (int k = 0; k < nz; ++k) {
      const long long id = base + (long long)k * d.plane;
      float nT = 0.f, nS = 0.f, gT = 0.f, gS = 0.f;
      float naT = 0.f, naS = 0.f, nbT = 0.f, nbS = 0.f, ndT = 0.f, ndS = 0.f;
      if (k + 1 < nz) {
        const long long nid = id + d.plane;
        nT = ld(a.Tev, nid);
        nS = ld(a.Sev, nid);
        naT = ld(a.accT, nid);
        naS = ld(a.accS, nid);
        nbT = ld(a.Tbase, nid);
        nbS = ld(a.Sbase, nid);
        if (st2) {
          ndT = ld(a.dT1, nid);
          ndS = ld(a.dS1, nid);
        }
        if ((allow >> k) & 1ull) {
          gT = -kc * (nT - cT) * d.vc.inv_dz_iface[k];
          gS = -kc * (nS - cS) * d.vc.inv_dz_iface[k];
        }
      }
      const float w = wetf(bits, k);
      const float convT = (fT - gT) * d.vc.inv_dz_node[k] * w;
      const float convS = (fS - gS) * d.vc.inv_dz_node[k] * w;
      if (a.convT) {
        a.convT[id] = convT;
        a.convS[id] = convS;
      }
      // rest_store's arithmetic, on the prefetched values
      float rT = qaT * a.inv_na + convT, rS = qaS * a.inv_na + convS;
      if (k == 0) {
        const float sst = cT, sss = cS;
        const float hf = w / (d.dz_surface * kRho0 * kCp);
        const float tatm = __ldg(d.tatm + base);
        rT += __ldg(d.qheat + base) * hf + d.lambda_bulk * (tatm - sst) * hf + __ldg(d.cbulk + base) * (tatm - sst) * hf +
              __ldg(d.rest_c + base) * (__ldg(d.rest_T + base) - sst);
        rS += d.restore_S * (__ldg(d.sref + base) - sss) + (sst <= d.ice_freeze ? d.ice_salt : 0.f);
      }
      rT *= w;
      rS *= w;
      if (!st2) {
        a.dT1[id] = rT;
        a.dS1[id] = rS;
        a.To[id] = qbT + rT * a.dt;
        a.So[id] = qbS + rS * a.dt;
      } else {
        a.To[id] = qbT + 0.5f * (qdT + rT) * a.dt;
        a.So[id] = qbS + 0.5f * (qdS + rS) * a.dt;
      }
      fT = gT; fS = gS; cT = nT; cS = nS;
      qaT = naT; qaS = naS; qbT = nbT; qbS = nbS; qdT = ndT; qdS = ndS;
    }
    return;
  }
  // several convective substeps (legacy: kappa and time both divided by nc)
  float cT[ZM_MAXZ], cS[ZM_MAXZ], sT[ZM_MAXZ], sS[ZM_MAXZ];
  for (int k = 0; k < nz; ++k) {
    cT[k] = ld(a.Tev, base + (long long)k * d.plane);
    cS[k] = ld(a.Sev, base + (long long)k * d.plane);
    sT[k] = 0.f;
    sS[k] = 0.f;
  }
  const float kc = d.kappa_conv / a.nc;
  const float hc = a.dt / a.nc;
  for (int s = 0; s < a.nc; ++s) {
    float fT = 0.f, fS = 0.f;
    for (int k = 0; k < nz; ++k) {
      float gT = 0.f, gS = 0.f;
      if (k + 1 < nz && ((allow >> k) & 1ull)) {
        gT = -kc * (cT[k + 1] - cT[k]) * d.vc.inv_dz_iface[k];
        gS = -kc * (cS[k + 1] - cS[k]) * d.vc.inv_dz_iface[k];
      }
      const float w = wetf(bits, k);
      const float tT = (fT - gT) * d.vc.inv_dz_node[k] * w;
      const float tS = (fS - gS) * d.vc.inv_dz_node[k] * w;
      sT[k] += tT;
      sS[k] += tS;
      fT = gT;
      fS = gS;
      // node k is not read again in this substep: the flux below it used the
      // pre-update values of k and k+1.
      cT[k] += tT * hc;
      cS[k] += tS * hc;
    }
  }
  const float inv_nc = 1.f / (float)a.nc;
  for (int k = 0; k < nz; ++k) {
    const long long id = base + (long long)k * d.plane;
    if (a.convT) {
      a.convT[id] = sT[k] * inv_nc;
      a.convS[id] = sS[k] * inv_nc;
    }
    rest_store(d, a, id, base, k, wetf(bits, k), ld(a.accT, id) * a.inv_na + sT[k] * inv_nc,
               ld(a.accS, id) * a.inv_na + sS[k] * inv_nc);
  }
}

// The RK stage is a template argument (stage 2 also reads dT1, dS1).
void launch_tracer_rest(dim3 g, dim3 b, cudaStream_t s, const Dev& d, const RestArgs& a) {
  (void)launch_pdl(a.stage == 1 ? k_tracer_rest<false> : k_tracer_rest<true>, g, b, 0, s, d, a);
}

// ------------------------------------------------------------------ pressure
// Baroclinic pressure-gradient force and its barotropic (layer-averaged)
// part, one column per thread (dynamics/pressure.py:32-42, 86-97, 144-180).
// The horizontal pressure differences p[e]-p[c] are accumulated down the
// column from the density differences (the same trapezoid sums as
// differencing the integrated pressure, with less cancellation in FP32).
//   mode 0: F_rho and the barotropic velocity (ubt0, vbt0; transport.py:135-143)
//   mode 1: P = wm (pgf - F_rho); up = u1 + dt (A + P)
//   mode 2: u2 = (u1 + dt/2 ((A + Pp) + (A + P))) * exp(-r_bot dt) at k = nz-1


__device__ __forceinline__ float drho(float2 a, float wa, float2 b, float wb_) {
  // rho'(a) wa - rho'(b) wb in difference form, a = (Ta, Sa): with wet flags
  // of 0 or 1 the products are exact, so this is rho0 (-alpha (Ta - Tb) +
  // beta (Sa - Sb)) when both are wet and rho'(a) wa - rho'(b) wb otherwise;
  // the T and S differences on one paired instruction
  const float2 dd = __ffma2_rn(f2(wa), a, __fmul2_rn(f2(-wb_), b));
  return kRho0 * (-kAlpha * dd.x + kBeta * dd.y);
}

// Pressure-gradient kernel (physics/pressure.py:32-97, legacy trapezoid form,
// in differences), one column per thread.  Modes: 0 the barotropic forcing
// F_rho and the depth-mean velocity; 1 and 2 the P part of the momentum
// residual with the RK combination of the first and second stage.  A block
// owns a PG_X x RY tile of columns (RY = d.pg_rows) and marches down the levels together:
// each level's T and S on the tile and a one-cell halo (rows clamped at the
// closed walls like north()/south(), longitude wrapped like east()/west())
// arrive in shared memory by cp.async, PG_NB - 1 levels ahead of the one being
// used, so every value is fetched once and the loads of later levels overlap
// the arithmetic.  Each thread keeps its column's density differences to the
// four neighbours and their downward accumulation in registers.  Modes 1 and
// 2 need the depth integral before the first output level, so the per-level
// gradient goes to a scratch field and the depth mean to a 2-D one; the
// output pass over all points is k_pgf_out.
constexpr int PG_X = 32, PG_NB = 4;  // tile columns, level buffers
constexpr int PG_PX = PG_X + 2;

template <int MODE, int RY>
__global__ void __launch_bounds__(PG_X * RY) k_pgf(Dev d, PgfArgs a) {
  constexpr int PG_PY = RY + 2, PG_CELLS = PG_PX * PG_PY;
  static_assert(PG_CELLS <= 2 * PG_X * RY, "two tile cells per thread at most");
  pdl_trigger();
  __shared__ float2 sTS[PG_NB][PG_PY][PG_PX];  // (T, S) of a cell side by side
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * PG_X + tx;
  const int i0 = blockIdx.x * PG_X, j0 = blockIdx.y * RY;
  const int i = i0 + tx, j = j0 + ty;
  // threads outside the grid copy their tile cells and meet the barriers, nothing else
  const bool in = i < d.nx && j < d.ny;
  const int e0 = tid, e1 = tid + PG_X * RY;
  const bool has1 = e1 < PG_CELLS;
  const int s0 = tile_cell<PG_PX>(d, e0, i0, j0), s1 = has1 ? tile_cell<PG_PX>(d, e1, i0, j0) : 0;
  auto issue = [&](int k) {  // level k into buffer k % PG_NB; one commit group per call
    if (k < d.nz) {
      const long long off = (long long)k * d.plane;
      float* ts = &sTS[k % PG_NB][0][0].x;
      cp_async4(ts + 2 * e0, a.T + off + s0);
      cp_async4(ts + 2 * e0 + 1, a.S + off + s0);
      if (has1) {
        cp_async4(ts + 2 * e1, a.T + off + s1);
        cp_async4(ts + 2 * e1 + 1, a.S + off + s1);
      }
    }
    cp_async_commit();
  };
  const int ic = in ? i : 0, jc = in ? j : 0;
  const Nb n = nb(d, jc, ic);
  const uint64_t m0 = wb(d, jc, ic), me = wb(d, jc, n.ie), mw = wb(d, jc, n.iw), mn = wb(d, n.jn, ic),
                 ms = wb(d, n.js, ic);
  const long long cc = idx2(d, jc, ic);
  const float hx = __ldg(d.inv_dx + cc) * 0.5f;
  const float hy = d.inv_dy * __ldg(d.inv_cos + jc) * 0.5f;
  const float cfp = __ldg(d.cfp + jc), cfm = __ldg(d.cfm + jc);
  const bool has_n = jc < d.ny - 1, has_s = jc > 0;
  float pe = 0.f, pw = 0.f, pn = 0.f, ps = 0.f;       // p[e]-p[c], p[c]-p[w], p[n]-p[c], p[c]-p[s]
  float de0 = 0.f, dw0 = 0.f, dn0 = 0.f, ds0 = 0.f;   // density differences at the level above
  float gx_prev = 0.f, gy_prev = 0.f, fx = 0.f, fy = 0.f;
  // wet flags of the column and its neighbours, bit 0 = the current level
  uint64_t f0 = m0, fe = me, fw = mw, fn = mn, fs = ms;
  float w0_prev = 0.f;
  // mode 0: the depth mean velocity (transport.py:135-143) along the same march,
  // each level's u, v loaded one level ahead
  double su = 0.0, sv = 0.0;
  float u_prev = 0.f, v_prev = 0.f;
  float u_next = 0.f, v_next = 0.f;
  if (MODE == 0 && in) {
    u_next = ld(a.u1, cc);
    v_next = ld(a.v1, cc);
  }
  constexpr float kInvRho0 = 1.f / kRho0;
  pdl_wait();  // T, S and the momentum parts come from the preceding kernels
#pragma unroll
  for (int q = 0; q < PG_NB - 1; ++q) issue(q);
  const int r = ty + 1, c = tx + 1;
  float* gsx = MODE != 0 ? a.gsx + cc : nullptr;  // this column's gradient scratch, one plane per level
  float* gsy = MODE != 0 ? a.gsy + cc : nullptr;
  for (int k = 0; k < d.nz; ++k) {
    cp_async_wait<PG_NB - 2>();  // this thread's copies of level k are done
    __syncthreads();             // everyone's are, and level k - 1's buffer is free
    issue(k + PG_NB - 1);
    if (!in) continue;
    float uk = 0.f, vk = 0.f;
    if (MODE == 0) {  // this level's u, v arrived during the previous level; the next ones are in flight
      uk = u_next;
      vk = v_next;
      if (k + 1 < d.nz) {
        u_next = ld(a.u1, (long long)(k + 1) * d.plane + cc);
        v_next = ld(a.v1, (long long)(k + 1) * d.plane + cc);
      }
    }
    const int b = k % PG_NB;
    const float2 tc = sTS[b][r][c];
    const float w0 = (float)(unsigned)(f0 & 1ull), we = (float)(unsigned)(fe & 1ull),
                ww = (float)(unsigned)(fw & 1ull), wn = (float)(unsigned)(fn & 1ull),
                ws = (float)(unsigned)(fs & 1ull);
    f0 >>= 1; fe >>= 1; fw >>= 1; fn >>= 1; fs >>= 1;
    const float de = drho(sTS[b][r][c + 1], we, tc, w0);
    const float dw = drho(tc, w0, sTS[b][r][c - 1], ww);
    const float dn = drho(sTS[b][r + 1][c], wn, tc, w0);
    const float ds = drho(tc, w0, sTS[b][r - 1][c], ws);
    if (k > 0) {
      const float h = kG * 0.5f * d.vc.dz3d[k - 1];
      pe += (de0 + de) * h;
      pw += (dw0 + dw) * h;
      pn += (dn0 + dn) * h;
      ps += (ds0 + ds) * h;
    }
    de0 = de; dw0 = dw; dn0 = dn; ds0 = ds;
    const float gx = hx * (pe * w0 * we + pw * w0 * ww);
    const float gy = hy * ((has_n ? pn * w0 * wn : 0.f) * cfp + (has_s ? ps * w0 * ws : 0.f) * cfm);
    if (k > 0) {
      const float wif = w0_prev * w0 * d.vc.dz3d[k - 1];
      fx += 0.5f * (gx_prev + gx) * wif;
      fy += 0.5f * (gy_prev + gy) * wif;
      if (MODE == 0) {
        su += (double)(0.5f * (u_prev + uk) * d.vc.dznorm[k - 1]);
        sv += (double)(0.5f * (v_prev + vk) * d.vc.dznorm[k - 1]);
      }
    }
    w0_prev = w0;
    gx_prev = gx;
    gy_prev = gy;
    u_prev = uk;
    v_prev = vk;
    if (MODE != 0) {
      // -g / rho0 by the float reciprocal of rho0 (within one rounding of the quotient)
      *gsx = -gx * kInvRho0;
      *gsy = -gy * kInvRho0;
      gsx += d.plane;
      gsy += d.plane;
    }
  }
  if (!in) return;
  const float Fx = -fx / (kRho0 * d.H_sw);
  const float Fy = -fy / (kRho0 * d.H_sw);
  if (MODE == 0) {
    a.frx[cc] = Fx;
    a.fry[cc] = Fy;
    a.ubt0[cc] = su;
    a.vbt0[cc] = sv;
    return;
  }
  // modes 1 and 2: the output pass needs the depth mean before the first
  // level, so it is its own fully parallel kernel (k_pgf_out)
  a.Fxs[cc] = Fx;
  a.Fys[cc] = Fy;
}

// Output pass of k_pgf modes 1 and 2, four consecutive points of a row per
// thread with float4 loads and stores (P % 4 == 0):
//   P = wm (pgf - F_rho) from the per-level gradient and the depth mean;
//   mode 1: stores P and up = u1 + dt (A + P);
//   mode 2: u2 = (u1 + dt/2 ((A + Pp) + (A + P))) * exp(-r_bot dt) at the
//   deepest level (the implicit drag), wet points.
template <int MODE>
__global__ void __launch_bounds__(256) k_pgf_out(Dev d, PgfArgs a) {
  pdl_trigger();
  const int p4 = d.P >> 2;
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // float4 index in [nz][ny][P/4]
  if (f >= (long long)d.nz * d.ny * p4) return;
  const int q = (int)(f % p4);
  const long long kj = f / p4;
  const int j = (int)(kj % d.ny), k = (int)(kj / d.ny);
  const int i0 = 4 * q;
  if (i0 >= d.nx) return;
  const int c = idx2(d, j, i0);
  const long long id = (long long)k * d.plane + c;
  const ulonglong2 b01 = __ldg(reinterpret_cast<const ulonglong2*>(d.wbits + c));
  const ulonglong2 b23 = __ldg(reinterpret_cast<const ulonglong2*>(d.wbits + c + 2));
  const float4 w = make_float4(wetf(b01.x, k), wetf(b01.y, k), wetf(b23.x, k), wetf(b23.y, k));
  pdl_wait();  // the gradient scratch and the momentum parts come from the preceding kernels
  const float4 gx = *reinterpret_cast<const float4*>(a.gsx + id), gy = *reinterpret_cast<const float4*>(a.gsy + id);
  const float4 Fx = *reinterpret_cast<const float4*>(a.Fxs + c), Fy = *reinterpret_cast<const float4*>(a.Fys + c);
  const float4 Au = __ldg(reinterpret_cast<const float4*>(a.Au + id));
  const float4 Av = __ldg(reinterpret_cast<const float4*>(a.Av + id));
  const float4 u1 = __ldg(reinterpret_cast<const float4*>(a.u1 + id));
  const float4 v1 = __ldg(reinterpret_cast<const float4*>(a.v1 + id));
  const float4 Pu = make_float4((gx.x - Fx.x) * w.x, (gx.y - Fx.y) * w.y, (gx.z - Fx.z) * w.z, (gx.w - Fx.w) * w.w);
  const float4 Pv = make_float4((gy.x - Fy.x) * w.x, (gy.y - Fy.y) * w.y, (gy.z - Fy.z) * w.z, (gy.w - Fy.w) * w.w);
  const float dt = a.dt;
  if (MODE == 1) {
    *reinterpret_cast<float4*>(a.Pu + id) = Pu;
    *reinterpret_cast<float4*>(a.Pv + id) = Pv;
    *reinterpret_cast<float4*>(a.uo + id) =
        make_float4(u1.x + (Au.x + Pu.x) * dt, u1.y + (Au.y + Pu.y) * dt, u1.z + (Au.z + Pu.z) * dt,
                    u1.w + (Au.w + Pu.w) * dt);
    *reinterpret_cast<float4*>(a.vo + id) =
        make_float4(v1.x + (Av.x + Pv.x) * dt, v1.y + (Av.y + Pv.y) * dt, v1.z + (Av.z + Pv.z) * dt,
                    v1.w + (Av.w + Pv.w) * dt);
  } else {
    const float4 pu = __ldg(reinterpret_cast<const float4*>(a.Ppu + id));
    const float4 pv = __ldg(reinterpret_cast<const float4*>(a.Ppv + id));
    const bool bot = k == d.nz - 1;
    const float4 dec = make_float4(bot && w.x != 0.f ? a.bottom_decay : 1.f, bot && w.y != 0.f ? a.bottom_decay : 1.f,
                                   bot && w.z != 0.f ? a.bottom_decay : 1.f, bot && w.w != 0.f ? a.bottom_decay : 1.f);
    *reinterpret_cast<float4*>(a.uo + id) = make_float4((u1.x + 0.5f * ((Au.x + pu.x) + (Au.x + Pu.x)) * dt) * dec.x,
                                                         (u1.y + 0.5f * ((Au.y + pu.y) + (Au.y + Pu.y)) * dt) * dec.y,
                                                         (u1.z + 0.5f * ((Au.z + pu.z) + (Au.z + Pu.z)) * dt) * dec.z,
                                                         (u1.w + 0.5f * ((Au.w + pu.w) + (Au.w + Pu.w)) * dt) * dec.w);
    *reinterpret_cast<float4*>(a.vo + id) = make_float4((v1.x + 0.5f * ((Av.x + pv.x) + (Av.x + Pv.x)) * dt) * dec.x,
                                                         (v1.y + 0.5f * ((Av.y + pv.y) + (Av.y + Pv.y)) * dt) * dec.y,
                                                         (v1.z + 0.5f * ((Av.z + pv.z) + (Av.z + Pv.z)) * dt) * dec.z,
                                                         (v1.w + 0.5f * ((Av.w + pv.w) + (Av.w + Pv.w)) * dt) * dec.w);
  }
}

// The mode is a template argument: each launch runs only its own passes.
void launch_pgf(cudaStream_t s, const Dev& d, const PgfArgs& a) {
  const int ry = d.pg_rows == 8 ? 8 : 4;
  const dim3 g((d.nx + PG_X - 1) / PG_X, (d.ny + ry - 1) / ry), b(PG_X, ry);
  if (ry == 8)
    (void)launch_pdl(a.mode == 0 ? k_pgf<0, 8> : (a.mode == 1 ? k_pgf<1, 8> : k_pgf<2, 8>), g, b, 0, s, d, a);
  else
    (void)launch_pdl(a.mode == 0 ? k_pgf<0, 4> : (a.mode == 1 ? k_pgf<1, 4> : k_pgf<2, 4>), g, b, 0, s, d, a);
  if (a.mode != 0) {
    const long long n4 = (long long)d.nz * d.ny * (d.P / 4);
    (void)launch_pdl(a.mode == 1 ? k_pgf_out<1> : k_pgf_out<2>, dim3((unsigned)((n4 + 255) / 256)), dim3(256), 0, s,
                     d, a);
  }
}

// Seasonal forcing blend (inputs/forcing/seasonal.py:86-103): the current
// month's field blended with the previous and next month's near the month
// boundaries, weights w_prev, w_cur, w_next from the host; a (12, nx, ny)
// reference-layout stack into the internal 2-D forcing field.
__global__ void k_forcing_blend(Dev d, const float* __restrict__ stack, int prev, int cur, int next, float w_prev,
                                float w_cur, float w_next, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const long long plane = (long long)d.nx * d.ny, r = (long long)i * d.ny + j;
  out[idx2(d, j, i)] = w_cur * stack[cur * plane + r] + w_next * stack[next * plane + r] +
                       w_prev * stack[prev * plane + r];
}

// ------------------------------------------------------------------ barotropic mode (float64)
// Total barotropic forcing F_rho + tau / (rho0 H) in float64.
__global__ void k_bt_forcing(Dev d, const float* __restrict__ frx, const float* __restrict__ fry,
                             double* __restrict__ Fx, double* __restrict__ Fy, const float* __restrict__ eta32,
                             double* __restrict__ eta64) {
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= d.nx || j >= d.ny) return;
  const int c = idx2(d, j, i);
  const double scale = 1.0 / (1025.0 * (double)d.H_sw);
  pdl_wait();  // F_rho comes from the preceding kernel
  Fx[c] = (double)frx[c] + (double)__ldg(d.tau_x + c) * scale;
  Fy[c] = (double)fry[c] + (double)__ldg(d.tau_y + c) * scale;
  eta64[c] = (double)eta32[c];
}

// Wet-point zonal means of the band rows of the projected 3-D fields
// (u + dubt, v + dvbt, T, S) for the final polar cap.
__global__ void __launch_bounds__(256) k_cap3_means(Dev d, const float* __restrict__ u, const float* __restrict__ v,
                                                    const float* __restrict__ T, const float* __restrict__ S,
                                                    const double* __restrict__ ubt, const double* __restrict__ ubt0,
                                                    const double* __restrict__ vbt, const double* __restrict__ vbt0,
                                                    float* __restrict__ means, int nb_rows) {
  pdl_trigger();
  pdl_wait();  // the projected fields come from the preceding kernels
  __shared__ float red[5][256];
  const int r = blockIdx.x;  // band row index
  const int k = blockIdx.y;
  const int j = r < nb_rows ? r : d.ny - 2 * nb_rows + r;
  float s[4] = {0.f, 0.f, 0.f, 0.f}, cnt = 0.f;
  for (int i = threadIdx.x; i < d.nx; i += blockDim.x) {
    const int c = idx2(d, j, i);
    const float w = wetf(wb(d, j, i), k);
    const long long id = idx3(d, k, j, i);
    s[0] += (ld(u, id) + (float)(ubt[c] - ubt0[c])) * w;
    s[1] += (ld(v, id) + (float)(vbt[c] - vbt0[c])) * w;
    s[2] += ld(T, id) * w;
    s[3] += ld(S, id) * w;
    cnt += w;
  }
  for (int q = 0; q < 4; ++q) red[q][threadIdx.x] = s[q];
  red[4][threadIdx.x] = cnt;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 5; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) {
    const float c = fmaxf(red[4][0], 1.f);
    means[((size_t)threadIdx.x * 2 * nb_rows + r) * d.nz + k] = red[threadIdx.x][0] / c;
  }
}

// Lateral sponge of the linear half step (timestepping/step.py:142-156):
// u, v *= decay and C = C_clim + (C - C_clim) decay, decay = exp(-rate dt/2)
// per column; tracers and their targets as anomalies.
__global__ void __launch_bounds__(256) k_sponge(Dev d, float* __restrict__ u, float* __restrict__ v,
                                                float* __restrict__ T, float* __restrict__ S,
                                                const float* __restrict__ dec, const float* __restrict__ Tc,
                                                const float* __restrict__ Sc) {
  ZM_POINT_IDX
  const float q = ld(dec, idx2(d, j, i));
  u[id] = u[id] * q;
  v[id] = v[id] * q;
  const float tc = ld(Tc, id), sc = ld(Sc, id);
  T[id] = tc + (T[id] - tc) * q;
  S[id] = sc + (S[id] - sc) * q;
}

// Uniform barotropic projection, polar cap, land/ghost hold and the no-flux
// wall on v (timestepping/step.py:419-450).
__global__ void __launch_bounds__(256) k_final(Dev d, const float* __restrict__ u3, const float* __restrict__ v3,
                                               const float* __restrict__ T3, const float* __restrict__ S3,
                                               const double* __restrict__ ubt, const double* __restrict__ ubt0,
                                               const double* __restrict__ vbt, const double* __restrict__ vbt0,
                                               const float* __restrict__ u0, const float* __restrict__ v0,
                                               const float* __restrict__ T0, const float* __restrict__ S0,
                                               const float* __restrict__ means, const float* __restrict__ wts,
                                               int nb_rows, float* __restrict__ uo, float* __restrict__ vo,
                                               float* __restrict__ To, float* __restrict__ So) {
  pdl_trigger();
  ZM_POINT_IDX
  const int c = idx2(d, j, i);
  const bool wet = wetb(wb(d, j, i), k);
  pdl_wait();  // every input comes from the preceding kernels
  if (!wet) {
    uo[id] = ld(u0, id);
    vo[id] = (j == 0 || j == d.ny - 1) ? 0.f : ld(v0, id);
    To[id] = ld(T0, id);
    So[id] = ld(S0, id);
    return;
  }
  float u = ld(u3, id) + (float)(ubt[c] - ubt0[c]);
  float v = ld(v3, id) + (float)(vbt[c] - vbt0[c]);
  float T = ld(T3, id), S = ld(S3, id);
  int r = -1;
  if (nb_rows > 0) {
    if (j < nb_rows) r = j;
    else if (j >= d.ny - nb_rows) r = j - (d.ny - 2 * nb_rows);
  }
  if (r >= 0) {
    const float wt = r < nb_rows ? wts[r] : wts[2 * nb_rows - 1 - r];
    const size_t stride = (size_t)2 * nb_rows * d.nz;
    const size_t o = (size_t)r * d.nz + k;
    u = wt * means[o] + (1.f - wt) * u;
    v = wt * means[stride + o] + (1.f - wt) * v;
    T = wt * means[2 * stride + o] + (1.f - wt) * T;
    S = wt * means[3 * stride + o] + (1.f - wt) * S;
  }
  uo[id] = u;
  vo[id] = (j == 0 || j == d.ny - 1) ? 0.f : v;
  // The step hands back absolute float32 tracers, T = anomaly + T_ref, and
  // reads them back as T - T_ref.  Keeping the anomaly that this round trip
  // gives (a fixed point of it for every float32 anomaly) makes the resident
  // state after each step exactly the one reloaded from the step's output, so
  // several steps on the device equal the same steps through the host state
  // and a restart from a saved state continues bit for bit.
  To[id] = __fsub_rn(__fadd_rn(T, d.T_ref), d.T_ref);
  So[id] = __fsub_rn(__fadd_rn(S, d.S_ref), d.S_ref);
}

// ------------------------------------------------------------------ layout conversion
// Reference layout (nx, ny, nz) C order  <->  internal [nz][ny][P].
__global__ void k_ref_to_int3(Dev d, const float* __restrict__ src, float* __restrict__ dst, float offset) {
  __shared__ float tile[32][33];
  const int j = blockIdx.z;
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (i < d.nx && k < d.nz) tile[r][threadIdx.x] = src[((long long)i * d.ny + j) * d.nz + k] - offset;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, i = i0 + threadIdx.x;
    if (i < d.nx && k < d.nz) dst[idx3(d, k, j, i)] = tile[threadIdx.x][r];
  }
}

__global__ void k_int_to_ref3(Dev d, const float* __restrict__ src, float* __restrict__ dst, float offset) {
  __shared__ float tile[32][33];
  const int j = blockIdx.z;
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, i = i0 + threadIdx.x;
    if (i < d.nx && k < d.nz) tile[r][threadIdx.x] = src[idx3(d, k, j, i)];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (i < d.nx && k < d.nz) dst[((long long)i * d.ny + j) * d.nz + k] = tile[threadIdx.x][r] + offset;
  }
}

__global__ void k_ref_to_int2(Dev d, const float* __restrict__ src, float* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) dst[idx2(d, j, i)] = src[(long long)i * d.ny + j];
}

__global__ void k_int_to_ref2(Dev d, const float* __restrict__ src, float* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i < d.nx && j < d.ny) dst[(long long)i * d.ny + j] = src[idx2(d, j, i)];
}

// ------------------------------------------------------------------ monitor
// Device-side state classification (runtime/monitor.py:20-30): bit 0 non-finite,
// bit 1 |u| or |v| above the velocity limit, bit 2 |eta| above its limit.
__global__ void __launch_bounds__(256) k_monitor(Dev d, const float* __restrict__ u, const float* __restrict__ v,
                                                 const float* __restrict__ T, const float* __restrict__ S,
                                                 const float* __restrict__ eta, float umax, float etamax,
                                                 unsigned int* __restrict__ flags) {
  const long long n3 = (long long)d.nz * d.plane;
  unsigned int f = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n3; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % d.P);
    if (i >= d.nx) continue;
    const float a = u[t], b = v[t], c = T[t], e = S[t];
    if (!isfinite(a) || !isfinite(b) || !isfinite(c) || !isfinite(e)) f |= 1u;
    if (fabsf(a) > umax || fabsf(b) > umax) f |= 2u;
    if (t < d.plane) {
      const float h = eta[t];
      if (!isfinite(h)) f |= 1u;
      if (fabsf(h) > etamax) f |= 4u;
    }
  }
  f = __reduce_or_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

}  // namespace zm

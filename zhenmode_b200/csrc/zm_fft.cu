// Longitude half of the momentum-advection dealias filter
// (numerics/horizontal.py:283-305): FFT along each periodic x-line, zero the
// bins outside the 2/3-rule mask (factory.py:529-533), inverse FFT, real part.
// The mask is the reference's own floating-point expression evaluated on the
// host, bin by bin: |fftfreq(nx) * nx| <= floor(nx/2 * 2/3) drops the
// boundary bins +-nx/3 for nx = 90, 180, 360, 720 because the product rounds
// just above the integer.
//
// The two advection fields of a line are packed as one complex signal
// (adv_u + i adv_v); the filter mask is real and even, so the filtered real
// and imaginary parts are the filtered fields.  Each block keeps several lines
// in shared memory and runs a mixed-radix (2, 3, 4, 5) Stockham FFT whose
// per-stage output indices and twiddles (float64-derived) are tabulated on
// the host.  The epilogue adds the surface wind stress
// and removes its barotropic part (dynamics/tendencies.py:59-62, 307-310) and
// applies the wet mask, producing the T/S-independent part of the momentum
// residual.
#include "zm_kernels.cuh"

namespace zm {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i / +i
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
__device__ __forceinline__ float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }

// Forward DFT codelets, y_k = sum_n x_n exp(-2 pi i n k / R).
__device__ __forceinline__ void dft2(float2* v) {
  const float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
__device__ __forceinline__ void dft3(float2* v) {
  const float s3 = 0.86602540378443864676f;  // sin(2 pi / 3)
  const float2 t1 = cadd(v[1], v[2]);
  const float2 t2 = csub(v[0], cscale(t1, 0.5f));
  const float2 t3 = cscale(csub(v[1], v[2]), s3);
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, mul_mi(t3));
  v[2] = cadd(t2, mul_pi(t3));
}
__device__ __forceinline__ void dft4(float2* v) {
  const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  const float2 c = cadd(v[1], v[3]), e = csub(v[1], v[3]);
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, mul_mi(e));
  v[3] = cadd(b, mul_pi(e));
}
__device__ __forceinline__ void dft5(float2* v) {
  const float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
  const float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
  const float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
  const float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
  const float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  const float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  const float2 x0 = v[0];
  const float2 r1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
  const float2 r2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
  const float2 q1 = cadd(cscale(b1, s1), cscale(b2, s2));
  const float2 q2 = csub(cscale(b1, s2), cscale(b2, s1));
  v[0] = cadd(x0, cadd(a1, a2));
  v[1] = cadd(r1, mul_mi(q1));
  v[4] = cadd(r1, mul_pi(q1));
  v[2] = cadd(r2, mul_mi(q2));
  v[3] = cadd(r2, mul_pi(q2));
}

// One Stockham pass of radix R over `lines` lines of length n (ns = product of
// the earlier radices).  Butterfly jj reads x[jj + r m] (m = n / R), applies
// the twiddles of its k = jj mod ns, and writes y[base + r ns] with
// base = (jj / ns) ns R + k; the bases and twiddles come from the plan's
// tables, and one thread runs the same butterfly on every line of the block.
template <int R>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ in, float2* __restrict__ out,
                                              const int* __restrict__ base_tab, const float2* __restrict__ twt,
                                              int n, int ns, int lines) {
  const int m = n / R;
  for (int jj = threadIdx.x; jj < m; jj += blockDim.x) {
    const int base = __ldg(base_tab + jj);
    float2 w[R - 1];
    if (ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) w[r - 1] = __ldg(twt + (r - 1) * m + jj);
    }
#pragma unroll 4
    for (int l = 0; l < lines; ++l) {
      const float2* src = in + l * n;
      float2* dst = out + l * n;
      float2 v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src[jj + r * m];
      if (ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r - 1]);
      }
      if (R == 2) dft2(v);
      if (R == 3) dft3(v);
      if (R == 4) dft4(v);
      if (R == 5) dft5(v);
#pragma unroll
      for (int r = 0; r < R; ++r) dst[base + r * ns] = v[r];
    }
  }
}

// Forward FFT of all lines; returns the buffer holding the result.
__device__ float2* fft_lines(float2* a, float2* b, const FftPlan& plan, int lines) {
  int ns = 1;
  for (int s = 0; s < plan.nstages; ++s) {
    const int R = plan.radix[s];
    const int* bt = plan.base_tab + plan.tab_off[s];
    const float2* tw = plan.stage_tw + plan.tw_off[s];
    if (R == 4) stockham_pass<4>(a, b, bt, tw, plan.n, ns, lines);
    else if (R == 2) stockham_pass<2>(a, b, bt, tw, plan.n, ns, lines);
    else if (R == 3) stockham_pass<3>(a, b, bt, tw, plan.n, ns, lines);
    else stockham_pass<5>(a, b, bt, tw, plan.n, ns, lines);
    __syncthreads();
    float2* t = a; a = b; b = t;
    ns *= R;
  }
  return a;
}

__global__ void __launch_bounds__(256) k_dealias_lon(Dev d, FftPlan plan, const float* __restrict__ Ayu,
                                                     const float* __restrict__ Ayv, float* __restrict__ Au,
                                                     float* __restrict__ Av, int lines_per_block) {
  pdl_trigger();
  pdl_wait();  // the advection fields come from the preceding kernel
  extern __shared__ float2 fsm[];
  const int n = plan.n;
  float2* bufa = fsm;
  float2* bufb = bufa + (size_t)lines_per_block * n;
  const int total = d.ny * d.nz;
  const int first = blockIdx.x * lines_per_block;
  const int lines = min(lines_per_block, total - first);
  if (lines <= 0) return;
  for (int l = 0; l < lines; ++l) {
    const int line = first + l;
    const int k = line / d.ny, j = line - k * d.ny;
    const long long row = idx3(d, k, j, 0);
    for (int i = threadIdx.x; i < n; i += blockDim.x) bufa[l * n + i] = make_float2(ld(Ayu, row + i), ld(Ayv, row + i));
  }
  __syncthreads();
  float2* spec = fft_lines(bufa, bufb, plan, lines);
  float2* other = spec == bufa ? bufb : bufa;
  // 2/3 rule with the reference's bin mask; conjugate for the inverse transform
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    const bool keep = __ldg(plan.keepbin + m) != 0;
    for (int l = 0; l < lines; ++l) {
      const float2 z = spec[l * n + m];
      spec[l * n + m] = keep ? make_float2(z.x, -z.y) : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  float2* res = fft_lines(spec, other, plan, lines);
  const float inv_n = 1.f / (float)n;
  const float wind_s = 1.f / (kRho0 * d.dz_surface);
  const float wind_bt = 1.f / (kRho0 * d.H_sw);
  for (int l = 0; l < lines; ++l) {
    const int line = first + l;
    const int k = line / d.ny, j = line - k * d.ny;
    const long long row = idx3(d, k, j, 0);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int c = idx2(d, j, i);
      const float w = wetf(wb(d, j, i), k);
      const float2 z = res[l * n + i];
      const float fu = z.x * inv_n, fv = -z.y * inv_n;   // conj of the forward transform of conj(X)
      const float tx = __ldg(d.tau_x + c), ty = __ldg(d.tau_y + c);
      const float su = (k == 0 ? tx * wind_s : 0.f) - tx * wind_bt;
      const float sv = (k == 0 ? ty * wind_s : 0.f) - ty * wind_bt;
      Au[row + i] = (fu + su) * w;
      Av[row + i] = (fv + sv) * w;
    }
  }
}

// ---------------------------------------------------------------- register form
// For n = N1 N2 N3 (720 = 8 9 10, 800 = 8 10 10, 360 = 4 9 10, 180 = 4 9 5)
// each line is transformed with its values in registers and only four
// exchanges through shared memory, instead of one round trip per radix stage:
//   forward, decimation in frequency over n = n1 N2 N3 + n2 N3 + n3:
//     A  DFT_N1 over n1 (loaded straight from global memory, coalesced),
//        twiddle W_n^(k1 (n2 N3 + n3));                        exchange
//     B  DFT_N2 over n2, twiddle W_n^(N1 k2 n3);                exchange
//     C  DFT_N3 over n3: X[k1 + N1 k2 + N1 N2 k3] in registers;
//   2/3 mask and conjugation in registers, then the second forward transform
//   over k = k3 N1 N2 + k2 N1 + k1 in the same order of splits:
//     C' DFT_N3 over k3 (the values the thread already holds),
//        twiddle W_n^((k1 + N1 k2) p3);                          exchange
//     B' DFT_N2 over k2, twiddle W_n^(N3 k1 p2);                 exchange
//     A' DFT_N1 over k1: the filtered value at m = p3 + N3 p2 + N3 N2 p1,
//        stored straight to global memory (coalesced) by the epilogue.
// The mask is the same keepbin table as the Stockham kernel's.

// exp(-2 pi i k / N) of the small codelets (float64 values rounded to float)
constexpr float kW8r = 0.70710678118654752f;
constexpr float kW9c1 = 0.76604444311897804f, kW9s1 = 0.64278760968653933f;
constexpr float kW9c2 = 0.17364817766693035f, kW9s2 = 0.98480775301220806f;
constexpr float kW9c4 = 0.93969262078590838f, kW9s4 = 0.34202014332566873f;
constexpr float kW10c1 = 0.80901699437494742f, kW10s1 = 0.58778525229247313f;
constexpr float kW10c2 = 0.30901699437494742f, kW10s2 = 0.95105651629515357f;

// 8 = 2 x 4: dft2 over (n, n + 4), twiddle W8^(b p), dft4 over b; X[p + 2 q]
__device__ __forceinline__ void dft8(float2* v) {
  float2 y0[4], y1[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    float2 t[2] = {v[b], v[b + 4]};
    dft2(t);
    y0[b] = t[0];
    y1[b] = t[1];
  }
  y1[1] = cmul(y1[1], make_float2(kW8r, -kW8r));
  y1[2] = mul_mi(y1[2]);
  y1[3] = cmul(y1[3], make_float2(-kW8r, -kW8r));
  dft4(y0);
  dft4(y1);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    v[2 * q] = y0[q];
    v[2 * q + 1] = y1[q];
  }
}

// 9 = 3 x 3: dft3 over (n, n + 3, n + 6), twiddle W9^(b p), dft3 over b; X[p + 3 q]
__device__ __forceinline__ void dft9(float2* v) {
  float2 y[3][3];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    float2 t[3] = {v[b], v[b + 3], v[b + 6]};
    dft3(t);
    y[0][b] = t[0];
    y[1][b] = t[1];
    y[2][b] = t[2];
  }
  y[1][1] = cmul(y[1][1], make_float2(kW9c1, -kW9s1));
  y[1][2] = cmul(y[1][2], make_float2(kW9c2, -kW9s2));
  y[2][1] = cmul(y[2][1], make_float2(kW9c2, -kW9s2));
  y[2][2] = cmul(y[2][2], make_float2(-kW9c4, -kW9s4));
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    dft3(y[p]);
#pragma unroll
    for (int q = 0; q < 3; ++q) v[p + 3 * q] = y[p][q];
  }
}

// 10 = 2 x 5: dft2 over (n, n + 5), twiddle W10^(b p), dft5 over b; X[p + 2 q]
__device__ __forceinline__ void dft10(float2* v) {
  float2 y0[5], y1[5];
#pragma unroll
  for (int b = 0; b < 5; ++b) {
    float2 t[2] = {v[b], v[b + 5]};
    dft2(t);
    y0[b] = t[0];
    y1[b] = t[1];
  }
  y1[1] = cmul(y1[1], make_float2(kW10c1, -kW10s1));
  y1[2] = cmul(y1[2], make_float2(kW10c2, -kW10s2));
  y1[3] = cmul(y1[3], make_float2(-kW10c2, -kW10s2));
  y1[4] = cmul(y1[4], make_float2(-kW10c1, -kW10s1));
  dft5(y0);
  dft5(y1);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    v[2 * q] = y0[q];
    v[2 * q + 1] = y1[q];
  }
}

template <int R>
__device__ __forceinline__ void dft(float2* v) {
  static_assert(R == 2 || R == 3 || R == 4 || R == 5 || R == 8 || R == 9 || R == 10, "codelet size");
  if (R == 2) dft2(v);
  if (R == 3) dft3(v);
  if (R == 4) dft4(v);
  if (R == 5) dft5(v);
  if (R == 8) dft8(v);
  if (R == 9) dft9(v);
  if (R == 10) dft10(v);
}

// v[r] *= W_n^(r step) for r >= 1, the exponent reduced mod n incrementally
template <int R>
__device__ __forceinline__ void twiddle(float2* v, const float2* __restrict__ tw, int step, int n) {
  int e = 0;
#pragma unroll
  for (int r = 1; r < R; ++r) {
    e += step;
    if (e >= n) e -= n;
    v[r] = cmul(v[r], __ldg(tw + e));
  }
}

template <int N1, int N2, int N3>
constexpr int reg_threads() {
  constexpr int a = N2 * N3, b = N1 * N3, c = N1 * N2;
  constexpr int m = a > b ? (a > c ? a : c) : (b > c ? b : c);
  return (m + 31) / 32 * 32;
}

template <int N1, int N2, int N3>
__global__ void __launch_bounds__(reg_threads<N1, N2, N3>() * 4) k_dealias_reg(Dev d, FftPlan plan,
                                                                                 const float* __restrict__ Ayu,
                                                                                 const float* __restrict__ Ayv,
                                                                                 float* __restrict__ Au,
                                                                                 float* __restrict__ Av) {
  constexpr int N = N1 * N2 * N3, N12 = N1 * N2, N23 = N2 * N3, N13 = N1 * N3;
  pdl_trigger();
  extern __shared__ float2 xsm[];
  float2* ex = xsm + threadIdx.y * N;  // this line's exchange buffer
  const int t = threadIdx.x;
  const int line = blockIdx.x * blockDim.y + threadIdx.y;
  const bool live = line < d.ny * d.nz;
  const int k = live ? line / d.ny : 0, j = live ? line - k * d.ny : 0;
  const long long row = idx3(d, k, j, 0);
  const float2* tw = plan.tw_full;
  pdl_wait();  // the advection fields come from the preceding kernel
  // A: DFT_N1 over n1 for column jj = n2 N3 + n3
  if (live && t < N23) {
    float2 v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = make_float2(ld(Ayu, row + t + n1 * N23), ld(Ayv, row + t + n1 * N23));
    dft<N1>(v);
    twiddle<N1>(v, tw, t, N);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) ex[k1 * N23 + t] = v[k1];
  }
  __syncthreads();
  // B: DFT_N2 over n2 for (k1, n3)
  {
    const int k1 = t / N3, n3 = t - (t / N3) * N3;
    const bool on = live && t < N13;
    float2 v[N2];
    if (on) {
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) v[n2] = ex[k1 * N23 + n2 * N3 + n3];
    }
    __syncthreads();
    if (on) {
      dft<N2>(v);
      twiddle<N2>(v, tw, N1 * n3, N);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) ex[k1 * N23 + k2 * N3 + n3] = v[k2];
    }
  }
  __syncthreads();
  // C, mask, C': for (k1, k2), kp = k1 + N1 k2
  {
    const int k1 = t % N1, k2 = t / N1, kp = t;
    const bool on = live && t < N12;
    float2 v[N3];
    if (on) {
#pragma unroll
      for (int n3 = 0; n3 < N3; ++n3) v[n3] = ex[k1 * N23 + k2 * N3 + n3];
      dft<N3>(v);
#pragma unroll
      for (int k3 = 0; k3 < N3; ++k3) {
        const bool keep = __ldg(plan.keepbin + kp + N12 * k3) != 0;
        v[k3] = keep ? make_float2(v[k3].x, -v[k3].y) : make_float2(0.f, 0.f);
      }
      dft<N3>(v);
      twiddle<N3>(v, tw, kp, N);
    }
    __syncthreads();
    if (on) {
#pragma unroll
      for (int p3 = 0; p3 < N3; ++p3) ex[p3 * N12 + kp] = v[p3];
    }
  }
  __syncthreads();
  // B': DFT_N2 over k2 for (k1, p3)
  {
    const int k1 = t % N1, p3 = t / N1;
    const bool on = live && t < N13;
    float2 v[N2];
    if (on) {
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) v[k2] = ex[p3 * N12 + k2 * N1 + k1];
    }
    __syncthreads();
    if (on) {
      dft<N2>(v);
      twiddle<N2>(v, tw, N3 * k1, N);
#pragma unroll
      for (int p2 = 0; p2 < N2; ++p2) ex[p3 * N12 + p2 * N1 + k1] = v[p2];
    }
  }
  __syncthreads();
  // A': DFT_N1 over k1 for (p3, p2); m = t + N2 N3 p1; epilogue as k_dealias_lon
  if (live && t < N23) {
    const int p3 = t % N3, p2 = t / N3;
    float2 v[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) v[k1] = ex[p3 * N12 + p2 * N1 + k1];
    dft<N1>(v);
    const float inv_n = 1.f / (float)N;
    const float wind_s = 1.f / (kRho0 * d.dz_surface);
    const float wind_bt = 1.f / (kRho0 * d.H_sw);
#pragma unroll
    for (int p1 = 0; p1 < N1; ++p1) {
      const int i = t + N23 * p1;
      const int c = idx2(d, j, i);
      const float w = wetf(wb(d, j, i), k);
      const float fu = v[p1].x * inv_n, fv = -v[p1].y * inv_n;  // conj of the forward transform of conj(X)
      const float tx = __ldg(d.tau_x + c), ty = __ldg(d.tau_y + c);
      const float su = (k == 0 ? tx * wind_s : 0.f) - tx * wind_bt;
      const float sv = (k == 0 ? ty * wind_s : 0.f) - ty * wind_bt;
      Au[row + i] = (fu + su) * w;
      Av[row + i] = (fv + sv) * w;
    }
  }
}

bool fft_reg_split(int n, int& r1, int& r2, int& r3) {
  static const int splits[][4] = {{720, 8, 9, 10}, {800, 8, 10, 10}, {360, 4, 9, 10}, {180, 4, 9, 5}};
  for (const auto& s : splits)
    if (s[0] == n) {
      r1 = s[1];
      r2 = s[2];
      r3 = s[3];
      return true;
    }
  r1 = r2 = r3 = 0;
  return false;
}

template <int N1, int N2, int N3>
static cudaError_t launch_reg(cudaStream_t s, const Dev& d, const FftPlan& plan, const float* Ayu, const float* Ayv,
                              float* Au, float* Av, int lines, bool pdl) {
  constexpr int T = reg_threads<N1, N2, N3>();
  const int nlines = d.ny * d.nz;
  const dim3 g((nlines + lines - 1) / lines), b(T, lines);
  const size_t smem = (size_t)lines * N1 * N2 * N3 * sizeof(float2);
  if (pdl) return launch_pdl(k_dealias_reg<N1, N2, N3>, g, b, smem, s, d, plan, Ayu, Ayv, Au, Av);
  k_dealias_reg<N1, N2, N3><<<g, b, smem, s>>>(d, plan, Ayu, Ayv, Au, Av);
  return cudaGetLastError();
}

cudaError_t launch_dealias(cudaStream_t s, const Dev& d, const FftPlan& plan, const float* Ayu, const float* Ayv,
                           float* Au, float* Av, int lines, size_t stockham_smem, bool pdl) {
  if (plan.r1 > 0) {
    const int l = lines >= 4 ? 4 : (lines >= 2 ? 2 : 1);
    if (plan.n == 720) return launch_reg<8, 9, 10>(s, d, plan, Ayu, Ayv, Au, Av, l, pdl);
    if (plan.n == 800) return launch_reg<8, 10, 10>(s, d, plan, Ayu, Ayv, Au, Av, l, pdl);
    if (plan.n == 360) return launch_reg<4, 9, 10>(s, d, plan, Ayu, Ayv, Au, Av, l, pdl);
    if (plan.n == 180) return launch_reg<4, 9, 5>(s, d, plan, Ayu, Ayv, Au, Av, l, pdl);
  }
  const int nlines = d.ny * d.nz;
  const dim3 g((nlines + lines - 1) / lines), b(256);
  if (pdl) return launch_pdl(k_dealias_lon, g, b, stockham_smem, s, d, plan, Ayu, Ayv, Au, Av, lines);
  k_dealias_lon<<<g, b, stockham_smem, s>>>(d, plan, Ayu, Ayv, Au, Av, lines);
  return cudaGetLastError();
}

}  // namespace zm

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

}  // namespace zm

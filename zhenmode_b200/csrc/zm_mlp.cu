// Per-column MLP of the learned vertical-mixing closure: 256 -> 256 -> 256 -> 64
// (GELU after the two hidden layers; 252 features and 50 outputs used, the
// rest zero padding).  Parameters are one float32 array:
//   W1 [256][256], b1 [256], W2 [256][256], b2 [256], W3 [64][256], b3 [64]
// with W[out][in] (the input index contiguous).
//
// Inference (k_mlp_tc): BF16 operands on the 5th-generation tensor cores with
// float32 accumulation in tensor memory.  A CTA of 128 threads owns 128
// columns: thread t owns column t, which is row t of the A operand and lane t
// of the accumulator.  The activations stay in shared memory as BF16 in the
// canonical K-major layout without swizzle (8-row x 16-byte core matrices;
// the two core matrices of one K=16 step are LBO = 128 B apart, 8-row groups
// SBO = 16 * K bytes apart).  Weights stream through shared memory in K
// chunks of 64; one thread issues the four tcgen05.mma of a chunk and commits
// them to an mbarrier that every thread waits on with a poll limit.  The
// epilogue of a layer reads the accumulator row with tcgen05.ld, adds the
// bias, applies GELU and writes BF16 back into the activation tile, which is
// the next layer's A operand.
//
// Training: float32 SIMT kernels (tiled GEMM with optional transposes, GELU
// and its derivative, masked mean-square loss, bias gradients, Adam), driven
// by zm_mlp_train_step / zm_mlp_grad on a trainer handle that owns the
// workspaces.
#include <cuda_bf16.h>

#include <cstdio>
#include <string>

#include "../../include/zm_b200.h"
#include "zm_kernels.cuh"

namespace zm {

namespace {

constexpr int MT = 128;                          // columns per CTA
constexpr int MK = ZM_MLP_IN;                    // 256: input and hidden width
constexpr int MO = ZM_MLP_OUT;                   // 64: padded output width
constexpr int KC = 64;                           // K chunk of a weight stage
constexpr uint32_t ACT_BYTES = MT * MK * 2;      // 64 KiB
constexpr uint32_t WB_BYTES = MK * KC * 2;       // 32 KiB
constexpr uint32_t TC_SMEM = ACT_BYTES + WB_BYTES + 64;
constexpr unsigned WAIT_POLLS = 1u << 22;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row, k) in a K-major tile of width kw
__device__ __forceinline__ uint32_t core_off(int row, int k, int kw) {
  return (uint32_t)((row >> 3) * (kw * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, leading and stride byte offsets
// (16-byte units), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: F32 accumulator, BF16 A and B, both
// K-major, N >> 3 and M >> 4
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned max_polls) {
  for (unsigned it = 0; it < max_polls; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    __nanosleep(20);
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

}  // namespace

size_t mlp_tc_smem() { return TC_SMEM; }

// One MLP pass over BF16 rows that `stage(t, act)` writes as row t of the
// activation tile (core_off layout), writing the 64 raw outputs of each row
// through `emit`.  Shared by the standalone and the fused kernels.
template <class Stage, class Emit>
__device__ __forceinline__ void mlp_tc_body(const MlpBf16& w, uint8_t* msm, unsigned* err, Stage stage, Emit emit) {
  uint8_t* act = msm;
  uint8_t* wb = msm + ACT_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(msm + ACT_BYTES + WB_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(msm + ACT_BYTES + WB_BYTES + 8);
  int* abort_flag = reinterpret_cast<int*>(msm + ACT_BYTES + WB_BYTES + 16);
  const int t = threadIdx.x, warp = t >> 5;
  if (t == 0) {
    *abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)), "r"(256u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // the inputs of this thread's column as row t of the A tile
  stage(t, act);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  bool failed = false;
  for (int layer = 0; layer < 3 && !failed; ++layer) {
    const __nv_bfloat16* W = layer == 0 ? w.W1 : (layer == 1 ? w.W2 : w.W3);
    const float* bias = layer == 0 ? w.b1 : (layer == 1 ? w.b2 : w.b3);
    const int N = layer < 2 ? MK : MO;
    const uint32_t id = layer < 2 ? idesc_bf16(MT, MK) : idesc_bf16(MT, MO);
    for (int kc = 0; kc < MK / KC; ++kc) {
      for (int p = t; p < N * (KC / 8); p += MT) {
        const int n = p / (KC / 8), kp = p - n * (KC / 8);
        const uint4 v = *reinterpret_cast<const uint4*>(W + (size_t)n * MK + kc * KC + kp * 8);
        *reinterpret_cast<uint4*>(wb + core_off(n, kp * 8, KC)) = v;
      }
      fence_async_smem();
      __syncthreads();
      if (t == 0) {
        fence_after();
#pragma unroll
        for (int s = 0; s < KC / 16; ++s) {
          const uint64_t da = sdesc(su32(act) + (uint32_t)((kc * KC + s * 16) / 8) * 128u, 128u, (uint32_t)MK * 16u);
          const uint64_t db = sdesc(su32(wb) + (uint32_t)s * 256u, 128u, (uint32_t)KC * 16u);
          umma_bf16(tmem, da, db, id, (kc | s) != 0 ? 1u : 0u);
        }
        umma_commit(su32(bar));
      }
      // the chunk's products are done before the weight buffer is refilled
      if (!mbar_wait(su32(bar), phase, WAIT_POLLS)) atomicOr(abort_flag, 1);
      __syncthreads();
      if (*abort_flag) {  // phase still names the outstanding commit
        failed = true;
        break;
      }
      phase ^= 1u;
    }
    if (failed) break;
    fence_after();
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_base + (uint32_t)c0, v);
      if (layer < 2) {
        __align__(16) __nv_bfloat16 h[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) h[j] = __float2bfloat16(gelu(v[j] + __ldg(bias + c0 + j)));
        *reinterpret_cast<uint4*>(act + core_off(t, c0, MK)) = *reinterpret_cast<const uint4*>(h);
        *reinterpret_cast<uint4*>(act + core_off(t, c0 + 8, MK)) = *reinterpret_cast<const uint4*>(h + 8);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += __ldg(bias + c0 + j);
        emit(t, c0, v);
      }
    }
    fence_before();
    fence_async_smem();
    __syncthreads();
  }
  if (failed) {
    // let the outstanding products finish (bounded) before the memory goes
    mbar_wait(su32(bar), phase, WAIT_POLLS);
    if (t == 0) atomicOr(err, 1u);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u) : "memory");
  }
}

// Standalone inference on BF16 feature rows X [ncol][256] -> Y [ncol][64].
__global__ void __launch_bounds__(MT, 1) k_mlp_tc(MlpBf16 w, const __nv_bfloat16* __restrict__ X,
                                                  float* __restrict__ Y, int ncol, unsigned* err) {
  extern __shared__ __align__(1024) uint8_t msm[];
  const long long col = (long long)blockIdx.x * MT + threadIdx.x;
  mlp_tc_body(
      w, msm, err,
      [&](int t, uint8_t* act) {
        for (int kp = 0; kp < MK / 8; ++kp) {
          uint4 v = make_uint4(0u, 0u, 0u, 0u);
          if (col < ncol) v = *reinterpret_cast<const uint4*>(X + col * MK + kp * 8);
          *reinterpret_cast<uint4*>(act + core_off(t, kp * 8, MK)) = v;
        }
      },
      [&](int, int c0, const float* v) {
        if (col < ncol)
          for (int j = 0; j < 16; ++j) Y[col * MO + c0 + j] = v[j];
      });
}

// ---------------------------------------------------------------- the closure in the step

// Feature q of the column at 2-D index base (wet bits `bits`): 0..49 T anomaly
// / 10, 50..99 S anomaly, 100..149 u / 0.5, 150..199 v / 0.5 (wet levels),
// 200..248 asinh(N^2 / 1e-8) / 4 at the wet interfaces, 250 |tau| / 0.1,
// 251 Q / 100, the rest zero.
__device__ __forceinline__ float closure_feature(const Dev& d, const ClosureArgs& a, long long base, uint64_t bits,
                                                 int q) {
  if (q < 200) {
    const int g = q / 50, k = q - g * 50;
    if (k >= d.nz || !wetb(bits, k)) return 0.f;
    const long long id = base + (long long)k * d.plane;
    if (g == 0) return ld(a.T, id) * 0.1f;
    if (g == 1) return ld(a.S, id);
    if (g == 2) return ld(a.u, id) * 2.f;
    return ld(a.v, id) * 2.f;
  }
  if (q < 250) {
    const int m = q - 200;
    if (m + 1 >= d.nz || !wetb(bits, m) || !wetb(bits, m + 1)) return 0.f;
    const long long id = base + (long long)m * d.plane;
    const float dT = ld(a.T, id + d.plane) - ld(a.T, id), dS = ld(a.S, id + d.plane) - ld(a.S, id);
    // N^2 = -(g / rho0) d rho / dz with z up: g (-alpha dT + beta dS) / dz, deeper
    // minus upper, on a signed log scale so that weak stratification keeps its sign
    return asinhf(kG * (-kAlpha * dT + kBeta * dS) * d.vc.inv_dz_iface[m] * 1e8f) * 0.25f;
  }
  if (q == 250) {
    const float tx = __ldg(d.tau_x + base), ty = __ldg(d.tau_y + base);
    return sqrtf(tx * tx + ty * ty) * 10.f;
  }
  if (q == 251) return __ldg(d.qheat + base) * 0.01f;
  return 0.f;
}

// The plain closure at interface m of a wet column (physics/vertical.py:40-82):
// kappa_v + coastal band, plus kappa_conv where the interface is statically
// unstable (localized) or the column has an unstable interface.
__device__ __forceinline__ float plain_kappa(const Dev& d, const ClosureArgs& a, long long base, uint64_t bits, int m,
                                            bool col_unstable) {
  float k = __ldg(d.kv2 + base);
  if (d.kappa_conv > 0.f) {
    bool gate = col_unstable;
    if (d.localize_conv) {
      const long long id = base + (long long)m * d.plane;
      gate = kBeta * (ld(a.S, id) - ld(a.S, id + d.plane)) > kAlpha * (ld(a.T, id) - ld(a.T, id + d.plane));
    }
    if (gate) k += d.kappa_conv;
  }
  return k;
}

__device__ __forceinline__ bool column_unstable(const Dev& d, const ClosureArgs& a, long long base, uint64_t bits) {
  for (int m = 0; m + 1 < d.nz; ++m) {
    if (!wetb(bits, m) || !wetb(bits, m + 1)) continue;
    const long long id = base + (long long)m * d.plane;
    if (kBeta * (ld(a.S, id) - ld(a.S, id + d.plane)) > kAlpha * (ld(a.T, id) - ld(a.T, id + d.plane))) return true;
  }
  return false;
}

// Training rows: features (float32), log10 of the plain closure at the wet
// interfaces and the mask of those interfaces, one column per thread.
__global__ void __launch_bounds__(128) k_closure_features(Dev d, ClosureArgs a) {
  const long long ncol = (long long)d.nx * d.ny;
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int j = (int)(col / d.nx), i = (int)(col - (long long)j * d.nx);
  const long long base = idx2(d, j, i);
  const uint64_t bits = __ldg(d.wbits + base);
  for (int q = 0; q < MK; ++q) a.X[col * MK + q] = closure_feature(d, a, base, bits, q);
  const bool cu = column_unstable(d, a, base, bits);
  for (int m = 0; m < MO; ++m) {
    const bool wet_if = m + 1 < d.nz && wetb(bits, m) && wetb(bits, m + 1);
    a.Tt[col * MO + m] = wet_if ? log10f(plain_kappa(d, a, base, bits, m, cu)) : 0.f;
    a.Mt[col * MO + m] = wet_if ? 1.f : 0.f;
  }
}

// The closure inside the step: features staged straight into the A tile of
// the tensor-core MLP; kappa = 10^y at the wet interfaces, clipped to
// [1e-7, 1] m^2/s, or the plain closure for a column whose features exceed
// the trusted bound (or are not finite).
__global__ void __launch_bounds__(MT, 1) k_mlp_closure(MlpBf16 w, Dev d, ClosureArgs a, unsigned* err) {
  extern __shared__ __align__(1024) uint8_t msm[];
  const long long ncol = (long long)d.nx * d.ny;
  const long long col = (long long)blockIdx.x * MT + threadIdx.x;
  const bool act = col < ncol;
  const int j = act ? (int)(col / d.nx) : 0, i = act ? (int)(col - (long long)j * d.nx) : 0;
  const long long base = idx2(d, j, i);
  const uint64_t bits = act ? __ldg(d.wbits + base) : 0ull;
  bool trusted = true;
  int unstable = -1;  // column gate of the plain closure, formed on first use
  mlp_tc_body(
      w, msm, err,
      [&](int t, uint8_t* tile) {
        // the row is zero, then the features level by level: four loads per
        // level, coalesced over the CTA's consecutive columns; N^2 from the
        // level above kept in registers
        for (int kp = 0; kp < MK / 8; ++kp)
          *reinterpret_cast<uint4*>(tile + core_off(t, kp * 8, MK)) = make_uint4(0u, 0u, 0u, 0u);
        float amax = 0.f;
        auto put = [&](int q, float f) {
          amax = fmaxf(amax, fabsf(f));
          if (!(f == f) || isinf(f)) amax = INFINITY;
          *reinterpret_cast<__nv_bfloat16*>(tile + core_off(t, q, MK)) = __float2bfloat16(f);
        };
        if (act) {
          float Tu = 0.f, Su = 0.f;
          bool wu = false;
#pragma unroll 4
          for (int k = 0; k < d.nz; ++k) {
            const long long id = base + (long long)k * d.plane;
            const float Tk = ld(a.T, id), Sk = ld(a.S, id), uk = ld(a.u, id), vk = ld(a.v, id);
            const bool wk = wetb(bits, k);
            if (wk) {
              put(k, Tk * 0.1f);
              put(50 + k, Sk);
              put(100 + k, uk * 2.f);
              put(150 + k, vk * 2.f);
              if (k > 0 && wu)
                put(199 + k, asinhf(kG * (-kAlpha * (Tk - Tu) + kBeta * (Sk - Su)) * d.vc.inv_dz_iface[k - 1] * 1e8f) *
                                 0.25f);
            }
            Tu = Tk;
            Su = Sk;
            wu = wk;
          }
          const float tx = __ldg(d.tau_x + base), ty = __ldg(d.tau_y + base);
          put(250, sqrtf(tx * tx + ty * ty) * 10.f);
          put(251, __ldg(d.qheat + base) * 0.01f);
        }
        trusted = amax <= a.bound;
      },
      [&](int, int c0, const float* y) {
        if (!act) return;
        if (!trusted && unstable < 0) {
          unstable = column_unstable(d, a, base, bits) ? 1 : 0;
          atomicAdd(a.fallback, 1u);
        }
        for (int e = 0; e < 16; ++e) {
          const int m = c0 + e;
          if (m + 1 >= d.nz) break;
          float k = 0.f;
          if (wetb(bits, m) && wetb(bits, m + 1)) {
            if (trusted) k = fminf(fmaxf(exp10f(y[e]), 1e-7f), 1.f);
            else k = plain_kappa(d, a, base, bits, m, unstable == 1);
          }
          a.kappa3[(long long)m * d.plane + base] = k;
        }
      });
}

// kappa3 [nz-1][ny][P] -> dense rows [col][64] (zero beyond nz-2)
__global__ void k_kappa_rows(Dev d, const float* __restrict__ kap3, float* __restrict__ out) {
  const long long ncol = (long long)d.nx * d.ny;
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int j = (int)(col / d.nx), i = (int)(col - (long long)j * d.nx);
  const long long base = idx2(d, j, i);
  for (int m = 0; m < MO; ++m) out[col * MO + m] = m + 1 < d.nz ? kap3[(long long)m * d.plane + base] : 0.f;
}

// float32 parameters -> BF16 weights (biases stay float32)
__global__ void k_mlp_pack(const float* __restrict__ params, __nv_bfloat16* __restrict__ W1,
                           __nv_bfloat16* __restrict__ W2, __nv_bfloat16* __restrict__ W3) {
  const int n1 = MK * MK, n3 = MO * MK;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += gridDim.x * blockDim.x) {
    W1[i] = __float2bfloat16(params[i]);
    W2[i] = __float2bfloat16(params[n1 + MK + i]);
    if (i < n3) W3[i] = __float2bfloat16(params[2 * (n1 + MK) + i]);
  }
}

// ---------------------------------------------------------------- training (float32)

// C[M][N] = op(A) op(B) (+ bias[n]) with op(A) [M][K], op(B) [K][N]; A is
// [M][K] (ta = 0) or [K][M] (ta = 1), B is [K][N] (tb = 0) or [N][K] (tb = 1).
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float* __restrict__ A, int ta,
                                               const float* __restrict__ B, int tb, const float* __restrict__ bias,
                                               float* __restrict__ C) {
  __shared__ float As[16][64 + 1], Bs[16][64 + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int kk = e / 64, mm = e - kk * 64;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? (ta ? A[(size_t)k * M + m] : A[(size_t)m * K + k]) : 0.f;
      const int n = n0 + mm;
      Bs[kk][mm] = (n < N && k < K) ? (tb ? B[(size_t)n * K + k] : B[(size_t)k * N + n]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty * 4 + q];
        b[q] = Bs[kk][tx * 4 + q];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] += a[q] * b[r];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int m = m0 + ty * 4 + q, n = n0 + tx * 4 + r;
      if (m < M && n < N) C[(size_t)m * N + n] = acc[q][r] + (bias ? bias[n] : 0.f);
    }
}

__global__ void k_gelu_fwd(const float* __restrict__ Z, float* __restrict__ H, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    H[i] = gelu(Z[i]);
}

__global__ void k_gelu_bwd(const float* __restrict__ Z, float* __restrict__ G, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    G[i] *= gelu_grad(Z[i]);
}

// masked mean-square error over the valid outputs: dY = 2 m (Y - T) / sum(m),
// per-block partial losses and mask counts
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ Mk,
                      float* __restrict__ dY, long long n, float inv_count, double* __restrict__ part) {
  __shared__ double red[256];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float e = (Y[i] - T[i]) * Mk[i];
    dY[i] = 2.f * e * inv_count;
    s += (double)e * (double)e;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// column sums of G [rows][cols] -> out[cols]
__global__ void k_colsum(const float* __restrict__ G, int rows, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += G[(size_t)r * cols + c];
  out[c] = s;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

}  // namespace zm

// ---------------------------------------------------------------- C ABI

using namespace zm;

namespace {

struct Off {  // offsets of the parameter blocks in the flat float32 array
  static constexpr long long W1 = 0, b1 = (long long)MK * MK, W2 = b1 + MK, b2 = W2 + (long long)MK * MK,
                             W3 = b2 + MK, b3 = W3 + (long long)MO * MK, total = b3 + MO;
};
static_assert(Off::total == ZM_MLP_NPARAMS, "parameter count");

bool launch_ok(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    return false;
  }
  return true;
}

void sgemm(cudaStream_t s, int M, int N, int K, const float* A, int ta, const float* B, int tb, const float* bias,
           float* C) {
  k_sgemm<<<dim3((N + 63) / 64, (M + 63) / 64), 256, 0, s>>>(M, N, K, A, ta, B, tb, bias, C);
}

}  // namespace

struct zm_mlp_trainer {
  int batch_max = 0;
  float *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *Y = nullptr, *dY = nullptr;
  float *G1 = nullptr, *G2 = nullptr, *grad = nullptr;
  double* part = nullptr;
  int nparts = 0;
};

extern "C" int zm_mlp_forward_bf16(void* stream, int32_t ncol, const void* X, const void* W1, const float* b1,
                                   const void* W2, const float* b2, const void* W3, const float* b3, float* Y,
                                   uint32_t* err) {
  if (ncol < 0 || !X || !W1 || !b1 || !W2 || !b2 || !W3 || !b3 || !Y || !err) return ZM_ERR_INVALID;
  if (ncol == 0) return ZM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM) != cudaSuccess)
    return ZM_ERR_CUDA;
  MlpBf16 w{(const __nv_bfloat16*)W1, (const __nv_bfloat16*)W2, (const __nv_bfloat16*)W3, b1, b2, b3};
  k_mlp_tc<<<(ncol + MT - 1) / MT, MT, TC_SMEM, st>>>(w, (const __nv_bfloat16*)X, Y, ncol, err);
  return launch_ok("zm_mlp_forward_bf16") ? ZM_OK : ZM_ERR_CUDA;
}

extern "C" int zm_mlp_pack_bf16(void* stream, const float* params, void* W1, void* W2, void* W3) {
  if (!params || !W1 || !W2 || !W3) return ZM_ERR_INVALID;
  k_mlp_pack<<<256, 256, 0, (cudaStream_t)stream>>>(params, (__nv_bfloat16*)W1, (__nv_bfloat16*)W2,
                                                     (__nv_bfloat16*)W3);
  return launch_ok("zm_mlp_pack_bf16") ? ZM_OK : ZM_ERR_CUDA;
}

extern "C" int zm_mlp_trainer_create(int32_t batch_max, zm_mlp_trainer** out) {
  if (!out || batch_max < 1) return ZM_ERR_INVALID;
  zm_mlp_trainer* tr = new zm_mlp_trainer();
  tr->batch_max = batch_max;
  tr->nparts = 256;
  const size_t h = (size_t)batch_max * MK, o = (size_t)batch_max * MO;
  float** bufs[] = {&tr->Z1, &tr->H1, &tr->Z2, &tr->H2, &tr->G1, &tr->G2};
  bool ok = true;
  for (float** b : bufs) ok = ok && cudaMalloc(b, h * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&tr->Y, o * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&tr->dY, o * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&tr->grad, (size_t)ZM_MLP_NPARAMS * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&tr->part, (size_t)tr->nparts * sizeof(double)) == cudaSuccess;
  if (!ok) {
    zm_mlp_trainer_destroy(tr);
    return ZM_ERR_CUDA;
  }
  *out = tr;
  return ZM_OK;
}

extern "C" void zm_mlp_trainer_destroy(zm_mlp_trainer* tr) {
  if (!tr) return;
  float* bufs[] = {tr->Z1, tr->H1, tr->Z2, tr->H2, tr->G1, tr->G2, tr->Y, tr->dY, tr->grad};
  for (float* b : bufs) cudaFree(b);
  cudaFree(tr->part);
  delete tr;
}

// forward pass of one batch (float32), keeping the pre-activations for the
// backward pass
static int mlp_forward_train(zm_mlp_trainer* tr, cudaStream_t st, int B, const float* X, const float* P) {
  const long long nh = (long long)B * MK;
  sgemm(st, B, MK, MK, X, 0, P + Off::W1, 1, P + Off::b1, tr->Z1);
  k_gelu_fwd<<<512, 256, 0, st>>>(tr->Z1, tr->H1, nh);
  sgemm(st, B, MK, MK, tr->H1, 0, P + Off::W2, 1, P + Off::b2, tr->Z2);
  k_gelu_fwd<<<512, 256, 0, st>>>(tr->Z2, tr->H2, nh);
  sgemm(st, B, MO, MK, tr->H2, 0, P + Off::W3, 1, P + Off::b3, tr->Y);
  return launch_ok("mlp forward") ? ZM_OK : ZM_ERR_CUDA;
}

// masked mean-square loss and the gradient of every parameter into tr->grad
static int mlp_backward(zm_mlp_trainer* tr, cudaStream_t st, int B, const float* X, const float* T, const float* Mk,
                        const float* P, double count, double* loss) {
  const float *W2 = P + Off::W2, *W3 = P + Off::W3;
  float* g = tr->grad;
  const long long nh = (long long)B * MK, no = (long long)B * MO;
  k_mse<<<tr->nparts, 256, 0, st>>>(tr->Y, T, Mk, tr->dY, no, (float)(1.0 / count), tr->part);
  // layer 3
  sgemm(st, MO, MK, B, tr->dY, 1, tr->H2, 0, nullptr, g + Off::W3);
  k_colsum<<<1, MO, 0, st>>>(tr->dY, B, MO, g + Off::b3);
  sgemm(st, B, MK, MO, tr->dY, 0, W3, 0, nullptr, tr->G2);
  k_gelu_bwd<<<512, 256, 0, st>>>(tr->Z2, tr->G2, nh);
  // layer 2
  sgemm(st, MK, MK, B, tr->G2, 1, tr->H1, 0, nullptr, g + Off::W2);
  k_colsum<<<1, MK, 0, st>>>(tr->G2, B, MK, g + Off::b2);
  sgemm(st, B, MK, MK, tr->G2, 0, W2, 0, nullptr, tr->G1);
  k_gelu_bwd<<<512, 256, 0, st>>>(tr->Z1, tr->G1, nh);
  // layer 1
  sgemm(st, MK, MK, B, tr->G1, 1, X, 0, nullptr, g + Off::W1);
  k_colsum<<<1, MK, 0, st>>>(tr->G1, B, MK, g + Off::b1);
  if (!launch_ok("mlp backward")) return ZM_ERR_CUDA;
  if (loss) {
    double parts[256];
    if (cudaMemcpyAsync(parts, tr->part, (size_t)tr->nparts * sizeof(double), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return ZM_ERR_CUDA;
    double s = 0.0;
    for (int q = 0; q < tr->nparts; ++q) s += parts[q];
    *loss = s / count;
  }
  return ZM_OK;
}

extern "C" int zm_mlp_grad(zm_mlp_trainer* tr, void* stream, int32_t batch, const float* X, const float* T,
                           const float* M, double mask_count, const float* params, float* grad_out, double* loss) {
  if (!tr || batch < 1 || batch > tr->batch_max || !X || !T || !M || !params || !grad_out || !(mask_count > 0))
    return ZM_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = mlp_forward_train(tr, st, batch, X, params);
  if (rc == ZM_OK) rc = mlp_backward(tr, st, batch, X, T, M, params, mask_count, loss);
  if (rc == ZM_OK &&
      cudaMemcpyAsync(grad_out, tr->grad, (size_t)ZM_MLP_NPARAMS * sizeof(float), cudaMemcpyDeviceToDevice, st) !=
          cudaSuccess)
    rc = ZM_ERR_CUDA;
  return rc;
}

extern "C" int zm_mlp_train_step(zm_mlp_trainer* tr, void* stream, int32_t batch, const float* X, const float* T,
                                 const float* M, double mask_count, float* params, float* adam_m, float* adam_v,
                                 int32_t step, float lr, float beta1, float beta2, float eps, double* loss) {
  if (!tr || batch < 1 || batch > tr->batch_max || !X || !T || !M || !params || !adam_m || !adam_v || step < 1 ||
      !(mask_count > 0))
    return ZM_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = mlp_forward_train(tr, st, batch, X, params);
  if (rc == ZM_OK) rc = mlp_backward(tr, st, batch, X, T, M, params, mask_count, loss);
  if (rc != ZM_OK) return rc;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_adam<<<512, 256, 0, st>>>(params, tr->grad, adam_m, adam_v, ZM_MLP_NPARAMS, lr, beta1, beta2, eps, c1, c2);
  return launch_ok("zm_mlp_train_step") ? ZM_OK : ZM_ERR_CUDA;
}

// State classification that allocates no device memory.
//
// Who needs this: a host runtime that gives the whole GPU to its own memory
// pool (JAX/XLA preallocates most of the device by default, so a custom call
// must not cudaMalloc), a model loop checking a state right after a blow-up,
// when that pool may be exhausted, and couplers that share the GPU under a
// fixed memory budget.  They already hold the state in their own device
// arrays; this entry point reads those arrays and keeps its only scratch -
// one partial result per block and a completion counter - in the file-scope
// array below.
//
// The array is part of the loaded library: every GPU that loads it holds
// ZM_NOALLOC_SCRATCH_BYTES until the process exits, and every call on that
// GPU shares it.  Calls whose kernels overlap on the GPU (two streams, or two
// host threads without ordering) race on it; order them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/zm_b200.h"

namespace {

constexpr int kBlocksMax = 2048;         // partial-result slots
constexpr long long kChunk = 65536;      // 3-D points per block
constexpr int kThreads = 256;
constexpr int kSlot = 4;                 // max|u|, max|v|, max|eta|, non-finite flag

// [kBlocksMax * kSlot] partials, then [kSlot] final values, then the counter word
struct Scratch {
  float partial[kBlocksMax * kSlot];
  float result[kSlot];
  unsigned int counter;
};
static_assert(sizeof(Scratch) <= ZM_NOALLOC_SCRATCH_BYTES, "scratch larger than its stated size");

static __device__ __align__(256) unsigned char zm_noalloc_scratch[ZM_NOALLOC_SCRATCH_BYTES];

// Maximum that keeps a NaN once one is seen, like jnp.max: the reference's
// metrics are NaN when a field holds a NaN, and +-inf enters as inf.
__device__ __forceinline__ float nan_max(float m, float a) { return (a != a || a > m) ? a : m; }

__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One pass over the caller's state: each block reduces its chunk into its
// slot; the last block to finish folds all slots into `result` and rezeroes
// the counter.  No block waits on another.  `ice` (2-D) may be null.
__global__ void __launch_bounds__(kThreads) k_classify_noalloc(const float* __restrict__ u, const float* __restrict__ v,
                                                                const float* __restrict__ T, const float* __restrict__ S,
                                                                const float* __restrict__ eta,
                                                                const float* __restrict__ ice, long long n3,
                                                                long long n2, int nblocks, Scratch* sc) {
  __shared__ float red[kSlot][kThreads / 32];
  __shared__ bool last;
  const long long lo3 = (long long)blockIdx.x * kChunk;
  const long long hi3 = lo3 + kChunk < n3 ? lo3 + kChunk : n3;
  const long long chunk2 = (n2 + nblocks - 1) / nblocks;
  const long long lo2 = (long long)blockIdx.x * chunk2;
  const long long hi2 = lo2 + chunk2 < n2 ? lo2 + chunk2 : n2;
  float mu = 0.f, mv = 0.f, me = 0.f, bad = 0.f;
  for (long long t = lo3 + threadIdx.x; t < hi3; t += blockDim.x) {
    const float a = u[t], b = v[t], c = T[t], e = S[t];
    if (!(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(e))) bad = 1.f;
    mu = nan_max(mu, fabsf(a));
    mv = nan_max(mv, fabsf(b));
  }
  for (long long t = lo2 + threadIdx.x; t < hi2; t += blockDim.x) {
    const float h = eta[t];
    if (!isfinite(h) || (ice && !isfinite(ice[t]))) bad = 1.f;
    me = nan_max(me, fabsf(h));
  }
  mu = warp_max(mu);
  mv = warp_max(mv);
  me = warp_max(me);
  bad = warp_max(bad);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][w] = mu;
    red[1][w] = mv;
    red[2][w] = me;
    red[3][w] = bad;
  }
  __syncthreads();
  if (threadIdx.x < kSlot) {
    float m = 0.f;
    for (int q = 0; q < kThreads / 32; ++q) m = nan_max(m, red[threadIdx.x][q]);
    sc->partial[blockIdx.x * kSlot + threadIdx.x] = m;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&sc->counter, 1u) == (unsigned)(nblocks - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < kSlot) {
    float m = 0.f;
    for (int b = 0; b < nblocks; ++b) m = nan_max(m, ((volatile float*)sc->partial)[b * kSlot + threadIdx.x]);
    sc->result[threadIdx.x] = m;
  }
  if (threadIdx.x == 0) sc->counter = 0u;
}

}  // namespace

extern "C" int zm_classify_state_noalloc(void* stream, int32_t nx, int32_t ny, int32_t nz, const float* u,
                                         const float* v, const float* T, const float* S, const float* eta,
                                         const float* ice, float velocity_limit, float eta_limit, int32_t inclusive,
                                         float* metrics, int32_t* code) {
  if (nx < 1 || ny < 1 || nz < 1 || !u || !v || !T || !S || !eta || !metrics || !code) {
    std::fprintf(stderr, "zm_classify_state_noalloc: invalid argument\n");
    return ZM_ERR_INVALID;
  }
  const long long n3 = (long long)nx * ny * nz, n2 = (long long)nx * ny;
  if (n3 > ZM_NOALLOC_MAX_POINTS) {
    std::fprintf(stderr,
                 "zm_classify_state_noalloc: %lld points per 3-D field exceed the maximum of %lld "
                 "(scratch is a fixed %d-byte array)\n",
                 n3, (long long)ZM_NOALLOC_MAX_POINTS, (int)ZM_NOALLOC_SCRATCH_BYTES);
    return ZM_ERR_INVALID;
  }
  cudaStream_t st = (cudaStream_t)stream;
  // the call waits for its result on the host, which a capturing stream
  // cannot do: refuse before touching the stream
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return ZM_ERR_CUDA;
  if (cap != cudaStreamCaptureStatusNone) {
    std::fprintf(stderr, "zm_classify_state_noalloc: the stream is capturing; call it outside a capture\n");
    return ZM_ERR_INVALID;
  }
  // `zm_noalloc_scratch` named in host code is a host-side stand-in, not a
  // device address: look the address up for the current device on every call
  // (cheap, and never stale after the context is recreated)
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, zm_noalloc_scratch);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "zm_classify_state_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
    return ZM_ERR_CUDA;
  }
  Scratch* sc = static_cast<Scratch*>(ptr);
  const int nblocks = (int)((n3 + kChunk - 1) / kChunk);
  // the completion counter must start at zero (the previous call left it zero
  // unless it was interrupted)
  if (cudaMemsetAsync(&sc->counter, 0, sizeof(unsigned int), st) != cudaSuccess) return ZM_ERR_CUDA;
  k_classify_noalloc<<<nblocks, kThreads, 0, st>>>(u, v, T, S, eta, ice, n3, n2, nblocks, sc);
  if (cudaGetLastError() != cudaSuccess) return ZM_ERR_CUDA;
  float res[kSlot];
  if (cudaMemcpyAsync(res, sc->result, sizeof(res), cudaMemcpyDeviceToHost, st) != cudaSuccess) return ZM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return ZM_ERR_CUDA;
  const float mu = res[0], mv = res[1], max_eta = res[2];
  // jnp.maximum: NaN if either is NaN
  const float max_vel = (mu != mu || mv != mv) ? NAN : std::fmax(mu, mv);
  const bool finite = res[3] == 0.f;
  metrics[0] = mu;
  metrics[1] = max_vel;
  metrics[2] = max_eta;
  metrics[3] = finite ? 1.f : 0.f;
  const bool bad_vel = inclusive ? max_vel >= velocity_limit : max_vel > velocity_limit;
  const bool bad_eta = inclusive ? max_eta >= eta_limit : max_eta > eta_limit;
  *code = !finite ? 1 : (bad_vel ? 3 : (bad_eta ? 4 : 0));
  return ZM_OK;
}

// Allocation-free Gram matrix of node4 blocks: tof_gram_noalloc.
//
// tof_gram needs a context, whose creation allocates device memory (its
// partial-sum buffer among it).  Some callers cannot allocate device memory
// at the point where they need a Gram matrix: a host application whose
// memory pool owns every byte of the GPU and forbids other allocations, or a
// latency-critical loop that must not hit cudaMalloc's implicit device
// synchronisation.  This entry point computes the same G = A^T B with every
// temporary in one fixed, file-scope device array.
//
// Limits: na, nb <= 24 (the array holds kNaSlots partial 24 x 24 matrices)
// and n_nodes <= INT_MAX.  The array (about 1.1 MiB) belongs to this
// library's device code: CUDA loads that code on a device lazily, so the
// array takes its device memory at the first call on each device and keeps it
// until the process exits (one copy per GPU).  That first call also looks up
// the array's device address; make it before any stream capture and before a
// memory pool takes over the GPU.  All calls on a GPU share that copy, which
// keeps the last call's partial sums; two calls on the same GPU whose
// executions overlap (for instance on two streams with no ordering between
// them) race on it, so order them.
#include <limits.h>

#include <mutex>
#include <string>

#include "../../include/tof.h"
#include "tof_internal.h"

namespace tof {
namespace {

constexpr int kNaSlots = 256;                 // CTAs, one partial matrix each
constexpr int kNaPairs = 24 * 24;
constexpr int kNaThreads = 256;
constexpr int kNaPerThread = 3;               // 576 pairs over 256 threads
constexpr int kMaxDevices = 64;

// partial matrices, then one 32-bit completion counter in the tail
static __device__ __align__(256) double g_gram_scratch[kNaSlots * kNaPairs + 32];

std::mutex g_mu;
double* g_scratch_dev[kMaxDevices] = {};      // device address of the array, per device

template <typename T, int CH>
__global__ void __launch_bounds__(kNaThreads) k_gram_noalloc(int NN, const T* __restrict__ A, int na,
                                                             const T* __restrict__ B, int nb, double* scratch,
                                                             double* G) {
  using V4 = typename Vec4<T>::type;
  __shared__ V4 sA[24 * CH];
  __shared__ V4 sB[24 * CH];
  __shared__ int s_last;
  const long long vs = (long long)NN * 4;
  const int npair = na * nb;
  double acc[kNaPerThread] = {0.0, 0.0, 0.0};
  const int nchunks = (int)(((long long)NN + CH - 1) / CH);
  const int per = (nchunks + gridDim.x - 1) / gridDim.x;
  const int c0 = blockIdx.x * per, c1 = min(nchunks, c0 + per);
  for (int ch = c0; ch < c1; ++ch) {
    const int n0 = ch * CH;
    const int cnt = min(CH, NN - n0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < na * CH; idx += blockDim.x) {
      const int v = idx / CH, q = idx % CH;
      V4 z{};
      sA[idx] = q < cnt ? reinterpret_cast<const V4*>(A + v * vs)[n0 + q] : z;
    }
    for (int idx = threadIdx.x; idx < nb * CH; idx += blockDim.x) {
      const int v = idx / CH, q = idx % CH;
      V4 z{};
      sB[idx] = q < cnt ? reinterpret_cast<const V4*>(B + v * vs)[n0 + q] : z;
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kNaPerThread; ++t) {
      const int p = threadIdx.x + t * kNaThreads;
      if (p < npair) {
        const V4* a = sA + (p / nb) * CH;
        const V4* b = sB + (p % nb) * CH;
        double s = 0.0;
        for (int q = 0; q < cnt; ++q) {
          s = fma(double(a[q].x), double(b[q].x), s);
          s = fma(double(a[q].y), double(b[q].y), s);
          s = fma(double(a[q].z), double(b[q].z), s);
        }
        acc[t] += s;
      }
    }
  }
  // publish this CTA's partial matrix; the last CTA to finish sums them all
  // in CTA order (deterministic) into G
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNaSlots * kNaPairs);
#pragma unroll
  for (int t = 0; t < kNaPerThread; ++t) {
    const int p = threadIdx.x + t * kNaThreads;
    if (p < npair) scratch[(size_t)blockIdx.x * kNaPairs + p] = acc[t];
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int p = threadIdx.x; p < npair; p += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(scratch + (size_t)b * kNaPairs + p);
    G[p] = s;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

}  // namespace
}  // namespace tof

using namespace tof;

extern "C" int tof_gram_noalloc(long long n_nodes, int dtype, const void* A, int na, const void* B, int nb,
                                double* G, void* stream) {
  if (!A || !B || !G || na < 1 || nb < 1 || (dtype != TOF_F32 && dtype != TOF_F64)) {
    set_global_error("tof_gram_noalloc: invalid argument");
    return TOF_ERR_ARG;
  }
  if (na > 24 || nb > 24) {
    set_global_error("tof_gram_noalloc: na and nb must be <= 24 (the fixed scratch holds 24 x 24 partial matrices)");
    return TOF_ERR_ARG;
  }
  if (n_nodes < 1 || n_nodes > INT_MAX) {
    set_global_error("tof_gram_noalloc: n_nodes must be in [1, INT_MAX]");
    return TOF_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_global_error("tof_gram_noalloc: no usable current CUDA device");
    return TOF_ERR_CUDA;
  }
  double* scratch = nullptr;
  {
    // set-up, once per device, with that device current: the device address
    // of the file-scope array (its host-side name is not a device pointer)
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_gram_scratch);
      if (e != cudaSuccess || !p) {
        set_global_error(std::string("tof_gram_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return TOF_ERR_CUDA;
      }
      g_scratch_dev[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_dev[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int NN = (int)n_nodes;
  // the completion counter must start at zero
  if (cudaMemsetAsync(scratch + kNaSlots * kNaPairs, 0, sizeof(unsigned), s) != cudaSuccess) {
    set_global_error("tof_gram_noalloc: cudaMemsetAsync failed");
    return TOF_ERR_CUDA;
  }
  const int CH = dtype == TOF_F64 ? 16 : 32;
  const int nchunks = (int)(((long long)NN + CH - 1) / CH);
  const int grid = nchunks < kNaSlots ? nchunks : kNaSlots;
  if (dtype == TOF_F64)
    k_gram_noalloc<double, 16><<<grid, kNaThreads, 0, s>>>(NN, (const double*)A, na, (const double*)B, nb,
                                                            scratch, G);
  else
    k_gram_noalloc<float, 32><<<grid, kNaThreads, 0, s>>>(NN, (const float*)A, na, (const float*)B, nb, scratch,
                                                           G);
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_global_error(std::string("tof_gram_noalloc: ") + cudaGetErrorString(e));
    return TOF_ERR_CUDA;
  }
  return TOF_OK;
}

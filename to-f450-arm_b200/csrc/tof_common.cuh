// Common device/host definitions for the voxel SIMP kernels (sm_100a).
//
// Data layout in HBM ("node4"): a nodal vector over the structured grid of
// (nx+1)*(ny+1)*(nz+1) nodes stores the three displacement components of
// node n = k*NX*NY + j*NX + i (the reference's node numbering,
// src/mesh3d.py:134-135) at [n*4 + c], c = 0..2, with [n*4 + 3] == 0.  A block of
// R vectors is R such arrays back to back.  The 16 B (FP32) / 32 B (FP64) node
// record gives vectorised loads and a TMA-able innermost dimension.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef TOF_MAX_RHS
#define TOF_MAX_RHS 8
#endif

namespace tof {

// ----------------------------------------------------------------------------
// Grid / tile description
// ----------------------------------------------------------------------------
struct Grid {
  int nx, ny, nz;      // elements per axis
  int NX, NY, NZ;      // nodes per axis (n + 1)
  int NN;              // nodes
  int NE;              // elements
  int TX, TY, TZ;      // node tile shape
  int ntx, nty, ntz;   // tiles per axis
  int ntiles;
};

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

inline Grid make_grid(int nx, int ny, int nz, int TX, int TY, int TZ) {
  Grid g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.NX = nx + 1; g.NY = ny + 1; g.NZ = nz + 1;
  g.NN = g.NX * g.NY * g.NZ;
  g.NE = nx * ny * nz;
  g.TX = TX; g.TY = TY; g.TZ = TZ;
  g.ntx = ceil_div(g.NX, TX); g.nty = ceil_div(g.NY, TY); g.ntz = ceil_div(g.NZ, TZ);
  g.ntiles = g.ntx * g.nty * g.ntz;
  return g;
}

// Local node index of the corner at offset (ox, oy, oz) in {0,1}^3 of an
// element: bottom face counter-clockwise from (0,0), then the top face
// (src/fem.py:35-46, src/mesh3d.py:140-146).
__host__ __device__ constexpr int local_node(int ox, int oy, int oz) {
  return 4 * oz + (oy ? (ox ? 2 : 3) : (ox ? 1 : 0));
}

// Status codes shared with the C ABI.
enum : int {
  ST_OK = 0,
  ST_NOT_CONVERGED = 1,
  ST_BREAKDOWN = -3,
  ST_NONFINITE = -4,
  ST_TIMEOUT = -5,
};

// ----------------------------------------------------------------------------
// Small PTX helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Wait budget of every spin in this library: a wait that has not completed
// after this long gives up, raises an error flag and returns (a legitimate
// wait here lasts microseconds).  Persistent solver kernels take the budget
// of their context (BarrierState::wait_ns, tof_ctx_set_wait_limit); 0 means
// this default.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;   // 2 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// ----------------------------------------------------------------------------
// Grid-wide barrier for persistent cooperative launches (all CTAs resident).
// Sense-reversing counter: the last CTA to arrive resets the counter and bumps
// the generation word with a release store; the others poll it with acquire
// loads.  Every poll loop is bounded; on timeout (or when another CTA has
// raised the error flag) the barrier returns false and the caller unwinds.
// ----------------------------------------------------------------------------
struct BarrierState {
  unsigned count;
  unsigned gen;
  int error;   // nonzero: some CTA gave up; everybody leaves
  int pad;
  unsigned long long wait_ns;   // wait budget (0: kWaitLimitNs); kept across resets
};
// bytes of BarrierState cleared before each persistent launch (wait_ns stays)
constexpr size_t kBarrierResetBytes = 16;

__device__ __forceinline__ unsigned long long wait_budget(const BarrierState* bs) {
  const unsigned long long w = bs->wait_ns;
  return w ? w : kWaitLimitNs;
}

__device__ __forceinline__ bool grid_barrier(BarrierState* bs, unsigned nblocks) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    fence_proxy_async_global();
    unsigned g = ld_acquire_u32(&bs->gen);
    __threadfence();
    unsigned prev = atomicAdd(&bs->count, 1u);
    if (prev == nblocks - 1) {
      atomicExch(&bs->count, 0u);
      __threadfence();
      st_release_u32(&bs->gen, g + 1);
    } else {
      unsigned long long spins = 0;
      const unsigned long long t0 = global_ns();
      const unsigned long long limit = wait_budget(bs);
      while (ld_acquire_u32(&bs->gen) == g) {
        if (ld_relaxed_i32(&bs->error)) { ok = 0; break; }
        if ((++spins & 255) == 0 && global_ns() - t0 > limit) {
          atomicExch(&bs->error, ST_TIMEOUT);
          ok = 0;
          break;
        }
        if (spins > 64) __nanosleep(32);
      }
    }
    fence_proxy_async_global();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ----------------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk.tensor) helpers.  No multicast anywhere.
// ----------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Bounded wait on phase `parity`; returns false after `limit` ns.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned long long limit = kWaitLimitNs) {
  uint32_t addr = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  for (unsigned long long i = 0;; ++i) {
    if ((i & 1023) == 1023 && global_ns() - t0 > limit) return false;
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 5-D tiled TMA load of a node4 halo box: coordinates (c, i, j, k, r).
__device__ __forceinline__ void tma_load_5d(void* smem_dst, const CUtensorMap* tmap, int c0, int c1, int c2,
                                            int c3, int c4, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmap_prefetch(const CUtensorMap* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// ----------------------------------------------------------------------------
// Reductions
// ----------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of K values per thread; result valid in every thread.
// `scratch` needs K * 32 doubles of shared memory.  Fixed reduction order,
// so every CTA reducing the same data gets bit-identical results.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) scratch[k * 32 + wid] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = (lane < nw) ? scratch[k * 32 + lane] : 0.0;
    v[k] = warp_sum(s);
  }
  __syncthreads();
}

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };

// Last-block-finishes reduction: every block adds its K partial sums; the last
// block to arrive sums all partials in block order (deterministic) into
// `total` and returns true.
template <int K>
__device__ bool last_block(double (&v)[K], double* part, unsigned* counter, double* scratch, double (&total)[K]) {
  __shared__ int s_last;
  block_sum<K>(v, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) part[(size_t)blockIdx.x * K + k] = v[k];
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; ++k) total[k] = 0.0;
  for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; ++k) total[k] += __ldcg(part + (size_t)b * K + k);
  }
  block_sum<K>(total, scratch);
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

}  // namespace tof

// Persistent block PCG on the matrix-free operator (sm_100a).
//
// The reference solves K_ff u_f = F_f with SciPy's Jacobi-preconditioned CG
// (src/fem.py:529-561; CuPy's cg on the GPU, src/fem_gpu.py:46-98), one load
// case per call, with the whole CSR matrix re-uploaded each time.  Here one
// cooperative launch runs the whole Krylov loop for R right-hand sides at once:
// each CTA owns fixed node tiles, the halo of the vector that enters the
// matvec is staged by TMA, dot products are reduced per CTA and combined by
// every CTA in the same order after a bounded grid barrier, so all CTAs take
// identical control decisions.
//
// * pcg_plain64: FP64 Jacobi PCG with exactly SciPy's recurrence
//   (rho = r.z; p = z + beta p; q = A p; alpha = rho / p.q; x += alpha p;
//   r -= alpha q), two grid barriers per iteration.  This is the drop-in form.
// * pcg_pipe32: FP32 pipelined PCG (Ghysels & Vanroose 2014, preconditioned
//   form): the matvec of the next search direction overlaps the dot-product
//   reduction, one grid barrier per iteration.  Used as the inner solver of
//   FP64 iterative refinement (tof_api.cu), which restores the 1e-8 residual.
#include <math.h>

#include "tof_internal.h"
#include "tof_stencil.cuh"

namespace tof {

struct SolveShared {
  // per-rhs control state, identical in every CTA
  double bnorm[TOF_MAX_RHS];
  double alpha[TOF_MAX_RHS], beta[TOF_MAX_RHS], gamma_prev[TOF_MAX_RHS], alpha_prev[TOF_MAX_RHS];
  double relres[TOF_MAX_RHS];
  int frozen[TOF_MAX_RHS];
  int status[TOF_MAX_RHS];
  int iters[TOF_MAX_RHS];
};

// Sum partials[b][k] over all CTAs b, same order in every CTA.
template <int K>
__device__ __forceinline__ void reduce_partials(const double* partials, int nblk, double (&v)[K], double* scratch) {
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __ldcg(partials + (size_t)b * K + k);
  }
  block_sum<K>(v, scratch);
}

template <int K>
__device__ __forceinline__ void write_partials(double* partials, double (&v)[K], double* scratch) {
  block_sum<K>(v, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)blockIdx.x * K + k] = v[k];
  }
}

__device__ __forceinline__ void proxy_fence_all() { fence_proxy_async_global(); }

// ===========================================================================
// FP32 pipelined PCG
// ===========================================================================
template <int R>
struct PipeArgs {
  CUtensorMap tmh[2];          // halo sources hb[0], hb[1]
  Grid g;
  const float* fK;
  const float* keb;
  const uint8_t* fix;
  const float* dinv;           // node4
  const double* b;             // node4 FP64 rhs [R]
  float* hb[2];
  float *x, *r, *u, *w, *z, *q, *s, *p;
  double* partials;
  BarrierState* bar;
  int* status;                 // [R] status, [R..2R) iterations
  double* relres;              // [R]
  double rtol;
  int maxiter;
  long long vs;
};

template <int R>
__global__ void __launch_bounds__(256) k_pcg_pipe(const __grid_constant__ PipeArgs<R> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  using V4 = float4;
  const Grid& g = a.g;
  const unsigned hbytes = halo_bytes<float>(g, R);
  float* sx = reinterpret_cast<float*>(smem);
  float* sKe = reinterpret_cast<float*>(smem + hbytes);
  float* sf = sKe + kKeBlocksLen;
  const int nfe = (g.TX + 1) * (g.TY + 1) * (g.TZ + 1);
  double* red = reinterpret_cast<double*>(smem + ((hbytes + 4 * (kKeBlocksLen + nfe) + 15) & ~15u));
  uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 3 * R * 32);
  __shared__ SolveShared st;

  load_ke_blocks(a.keb, sKe);
  if (threadIdx.x == 0) {
    mbar_init(mbar, 1);
    tmap_prefetch(&a.tmh[0]);
    tmap_prefetch(&a.tmh[1]);
  }
  const int G = gridDim.x;
  const bool single = g.ntiles <= G;
  unsigned phase = 0;
  bool ok = true;
  if (single && blockIdx.x < g.ntiles) load_factor_tile(g, tile_geom(g, blockIdx.x), a.fK, sf);
  __syncthreads();

  // ---- init 0: r = b, x = 0, u = D^-1 r (-> hb[1]), z = q = s = p = 0; ||b||^2
  {
    double v[R];
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = 0.0;
    for (int t = blockIdx.x; t < g.ntiles; t += G) {
      const TileGeom tg = tile_geom(g, t);
      int tx, ty, tz, n;
      if (!thread_node(g, tg, tx, ty, tz, n)) continue;
      const V4 di = reinterpret_cast<const V4*>(a.dinv)[n];
      const V4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const size_t o = k * a.vs / 4 + n;
        const double4 bb = reinterpret_cast<const double4*>(a.b)[o];
        v[k] += bb.x * bb.x + bb.y * bb.y + bb.z * bb.z;
        const V4 rr = make_float4(float(bb.x), float(bb.y), float(bb.z), 0.f);
        const V4 uu = make_float4(di.x * rr.x, di.y * rr.y, di.z * rr.z, 0.f);
        reinterpret_cast<V4*>(a.r)[o] = rr;
        reinterpret_cast<V4*>(a.u)[o] = uu;
        reinterpret_cast<V4*>(a.hb[1])[o] = uu;
        reinterpret_cast<V4*>(a.x)[o] = zero;
        reinterpret_cast<V4*>(a.z)[o] = zero;
        reinterpret_cast<V4*>(a.q)[o] = zero;
        reinterpret_cast<V4*>(a.s)[o] = zero;
        reinterpret_cast<V4*>(a.p)[o] = zero;
      }
    }
    write_partials<R>(a.partials, v, red);
    proxy_fence_all();
    ok = grid_barrier(a.bar, G);
    if (ok) {
      reduce_partials<R>(a.partials, G, v, red);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
          st.bnorm[k] = sqrt(v[k]);
          st.frozen[k] = 0;
          st.status[k] = ST_NOT_CONVERGED;
          st.iters[k] = 0;
          st.relres[k] = 1.0;
          st.alpha_prev[k] = 1.0;
          st.gamma_prev[k] = 1.0;
          if (!(v[k] > 0.0)) {  // zero (or non-finite) rhs
            st.frozen[k] = 1;
            st.status[k] = isfinite(v[k]) ? ST_OK : ST_NONFINITE;
            st.relres[k] = 0.0;
          }
        }
      }
      __syncthreads();
    }
  }
  // ---- init 1 and loop.  `cur` = index of the hb buffer holding m_i (or u_0
  // for the init matvec).
  int cur = 1;
  for (int it = -1; ok; ++it) {
    // matvec on hb[cur] for every owned tile, then local updates
    double v[3 * R];
#pragma unroll
    for (int k = 0; k < 3 * R; ++k) v[k] = 0.0;
    float al[R], be[R];
    bool fz[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      al[k] = float(st.alpha[k]);
      be[k] = float(st.beta[k]);
      fz[k] = st.frozen[k] != 0;
    }
    const int nxt = cur ^ 1;
    for (int t = blockIdx.x; t < g.ntiles; t += G) {
      const TileGeom tg = tile_geom(g, t);
      if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(mbar, hbytes);
        tma_load_5d(sx, &a.tmh[cur], 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, mbar);
      }
      if (!single) {
        load_factor_tile(g, tg, a.fK, sf);
        __syncthreads();
      }
      ok = __syncthreads_and(ok && mbar_wait(mbar, phase, wait_budget(a.bar)));
      phase ^= 1;
      int tx, ty, tz, n;
      if (ok && thread_node(g, tg, tx, ty, tz, n)) {
        float acc[R][3];
        stencil_node<float, R>(sx, tg, sf, sKe, tx, ty, tz, acc);
        const uint8_t fx = __ldg(a.fix + n);
        const V4 di = reinterpret_cast<const V4*>(a.dinv)[n];
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const size_t o = k * a.vs / 4 + n;
          V4 av = make_float4((fx & 1) ? 0.f : acc[k][0], (fx & 2) ? 0.f : acc[k][1], (fx & 4) ? 0.f : acc[k][2], 0.f);
          if (it < 0) {
            // w0 = A u0, m0 = D^-1 w0
            const V4 rr = reinterpret_cast<const V4*>(a.r)[o];
            const V4 uu = reinterpret_cast<const V4*>(a.u)[o];
            reinterpret_cast<V4*>(a.w)[o] = av;
            reinterpret_cast<V4*>(a.hb[nxt])[o] = make_float4(di.x * av.x, di.y * av.y, di.z * av.z, 0.f);
            v[3 * k + 0] += double(rr.x) * uu.x + double(rr.y) * uu.y + double(rr.z) * uu.z;
            v[3 * k + 1] += double(av.x) * uu.x + double(av.y) * uu.y + double(av.z) * uu.z;
            v[3 * k + 2] += double(rr.x) * rr.x + double(rr.y) * rr.y + double(rr.z) * rr.z;
          } else if (!fz[k]) {
            // n_i = A m_i (av), m_i from the staged tile
            const V4 m = halo_center<float>(sx, tg, k, tx, ty, tz);
            V4 zz = reinterpret_cast<const V4*>(a.z)[o];
            V4 qq = reinterpret_cast<const V4*>(a.q)[o];
            V4 ss = reinterpret_cast<const V4*>(a.s)[o];
            V4 pp = reinterpret_cast<const V4*>(a.p)[o];
            V4 xx = reinterpret_cast<const V4*>(a.x)[o];
            V4 rr = reinterpret_cast<const V4*>(a.r)[o];
            V4 uu = reinterpret_cast<const V4*>(a.u)[o];
            V4 ww = reinterpret_cast<const V4*>(a.w)[o];
            const float b_ = be[k], a_ = al[k];
            zz.x = fmaf(b_, zz.x, av.x); zz.y = fmaf(b_, zz.y, av.y); zz.z = fmaf(b_, zz.z, av.z);
            qq.x = fmaf(b_, qq.x, m.x); qq.y = fmaf(b_, qq.y, m.y); qq.z = fmaf(b_, qq.z, m.z);
            ss.x = fmaf(b_, ss.x, ww.x); ss.y = fmaf(b_, ss.y, ww.y); ss.z = fmaf(b_, ss.z, ww.z);
            pp.x = fmaf(b_, pp.x, uu.x); pp.y = fmaf(b_, pp.y, uu.y); pp.z = fmaf(b_, pp.z, uu.z);
            xx.x = fmaf(a_, pp.x, xx.x); xx.y = fmaf(a_, pp.y, xx.y); xx.z = fmaf(a_, pp.z, xx.z);
            rr.x = fmaf(-a_, ss.x, rr.x); rr.y = fmaf(-a_, ss.y, rr.y); rr.z = fmaf(-a_, ss.z, rr.z);
            uu.x = fmaf(-a_, qq.x, uu.x); uu.y = fmaf(-a_, qq.y, uu.y); uu.z = fmaf(-a_, qq.z, uu.z);
            ww.x = fmaf(-a_, zz.x, ww.x); ww.y = fmaf(-a_, zz.y, ww.y); ww.z = fmaf(-a_, zz.z, ww.z);
            reinterpret_cast<V4*>(a.z)[o] = zz;
            reinterpret_cast<V4*>(a.q)[o] = qq;
            reinterpret_cast<V4*>(a.s)[o] = ss;
            reinterpret_cast<V4*>(a.p)[o] = pp;
            reinterpret_cast<V4*>(a.x)[o] = xx;
            reinterpret_cast<V4*>(a.r)[o] = rr;
            reinterpret_cast<V4*>(a.u)[o] = uu;
            reinterpret_cast<V4*>(a.w)[o] = ww;
            reinterpret_cast<V4*>(a.hb[nxt])[o] = make_float4(di.x * ww.x, di.y * ww.y, di.z * ww.z, 0.f);
            v[3 * k + 0] += double(rr.x) * uu.x + double(rr.y) * uu.y + double(rr.z) * uu.z;
            v[3 * k + 1] += double(ww.x) * uu.x + double(ww.y) * uu.y + double(ww.z) * uu.z;
            v[3 * k + 2] += double(rr.x) * rr.x + double(rr.y) * rr.y + double(rr.z) * rr.z;
          }
        }
      }
      __syncthreads();   // smem tile reused by the next TMA
    }
    write_partials<3 * R>(a.partials, v, red);
    proxy_fence_all();
    if (!ok) { atomicExch(&a.bar->error, ST_TIMEOUT); break; }
    ok = grid_barrier(a.bar, G);
    if (!ok) break;
    cur = nxt;
    // reduce gamma_{i+1}, delta_{i+1}, ||r_{i+1}||^2 and decide
    reduce_partials<3 * R>(a.partials, G, v, red);
    if (threadIdx.x == 0) {
      const int itn = it + 1;   // index of the iteration about to run
#pragma unroll
      for (int k = 0; k < R; ++k) {
        if (st.frozen[k]) continue;
        const double gam = v[3 * k], del = v[3 * k + 1], rr = v[3 * k + 2];
        const double rel = sqrt(rr) / st.bnorm[k];
        st.relres[k] = rel;
        st.iters[k] = itn;
        if (!isfinite(gam) || !isfinite(del) || !isfinite(rr)) {
          st.frozen[k] = 1; st.status[k] = ST_NONFINITE; continue;
        }
        if (rel <= a.rtol) { st.frozen[k] = 1; st.status[k] = ST_OK; continue; }
        if (itn >= a.maxiter) { st.frozen[k] = 1; st.status[k] = ST_NOT_CONVERGED; continue; }
        double be = 0.0, den = del;
        if (itn > 0) {
          be = gam / st.gamma_prev[k];
          den = del - be * gam / st.alpha_prev[k];
        }
        if (!(den > 0.0) || !(gam > 0.0)) { st.frozen[k] = 1; st.status[k] = ST_BREAKDOWN; continue; }
        st.beta[k] = be;
        st.alpha[k] = gam / den;
        st.gamma_prev[k] = gam;
        st.alpha_prev[k] = st.alpha[k];
      }
    }
    __syncthreads();
    bool all = true;
#pragma unroll
    for (int k = 0; k < R; ++k) all = all && st.frozen[k];
    if (all) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int err = ld_relaxed_i32(&a.bar->error);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      a.status[k] = err ? err : st.status[k];
      a.status[R + k] = st.iters[k];
      a.relres[k] = st.relres[k];
    }
  }
}

// ===========================================================================
// Standard (SciPy-recurrence) Jacobi PCG, vectors in T = double (the plain
// FP64 drop-in) or T = float (the inner solver of FP64 refinement); scalars,
// dot products and the rhs are FP64 either way.
// ===========================================================================
template <typename T, int R>
struct PlainArgs {
  CUtensorMap tmx, tmz, tmp[2];
  Grid g;
  const T* fK;
  const T* keb;
  const uint8_t* fix;
  const T* dinv;
  const double* b;
  T *x, *r, *z, *q, *p[2];
  double* partials;
  BarrierState* bar;
  int* status;
  double* relres;
  double rtol;
  int maxiter;
  long long vs;
};

template <typename V4, typename S>
__device__ __forceinline__ V4 v4(S x, S y, S z) {
  V4 o;
  o.x = x; o.y = y; o.z = z; o.w = 0;
  return o;
}

template <typename T, int R>
__global__ void __launch_bounds__(256) k_pcg_plain(const __grid_constant__ PlainArgs<T, R> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  using V4 = typename Vec4<T>::type;
  const Grid& g = a.g;
  const unsigned hbytes = halo_bytes<T>(g, R);
  T* sz = reinterpret_cast<T*>(smem);
  T* sp = reinterpret_cast<T*>(smem + hbytes);
  T* sKe = reinterpret_cast<T*>(smem + 2 * hbytes);
  T* sf = sKe + kKeBlocksLen;
  const int nfe = (g.TX + 1) * (g.TY + 1) * (g.TZ + 1);
  double* red = reinterpret_cast<double*>(smem + ((2 * hbytes + sizeof(T) * (kKeBlocksLen + nfe) + 15) & ~15u));
  uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 3 * R * 32);
  __shared__ SolveShared st;

  load_ke_blocks(a.keb, sKe);
  if (threadIdx.x == 0) mbar_init(mbar, 1);
  const int G = gridDim.x;
  const bool single = g.ntiles <= G;
  unsigned phase = 0;
  bool ok = true;
  if (single && blockIdx.x < g.ntiles) load_factor_tile(g, tile_geom(g, blockIdx.x), a.fK, sf);
  __syncthreads();
  const int hsr = (g.TX + 2) * (g.TY + 2) * (g.TZ + 2);

  // ---- init: r = b - A x0, z = D^-1 r, p[0] = 0; rz, rr, bb
  {
    double v[3 * R];
#pragma unroll
    for (int k = 0; k < 3 * R; ++k) v[k] = 0.0;
    for (int t = blockIdx.x; t < g.ntiles; t += G) {
      const TileGeom tg = tile_geom(g, t);
      if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(mbar, hbytes);
        tma_load_5d(sp, &a.tmx, 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, mbar);
      }
      if (!single) { load_factor_tile(g, tg, a.fK, sf); __syncthreads(); }
      ok = __syncthreads_and(ok && mbar_wait(mbar, phase, wait_budget(a.bar)));
      phase ^= 1;
      int tx, ty, tz, n;
      if (ok && thread_node(g, tg, tx, ty, tz, n)) {
        T acc[R][3];
        stencil_node<T, R>(sp, tg, sf, sKe, tx, ty, tz, acc);
        const uint8_t fx = __ldg(a.fix + n);
        const V4 di = reinterpret_cast<const V4*>(a.dinv)[n];
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const size_t o = k * a.vs / 4 + n;
          const double4 bb = reinterpret_cast<const double4*>(a.b)[o];
          const V4 rr = v4<V4, T>((fx & 1) ? T(0) : T(bb.x - double(acc[k][0])),
                                  (fx & 2) ? T(0) : T(bb.y - double(acc[k][1])),
                                  (fx & 4) ? T(0) : T(bb.z - double(acc[k][2])));
          const V4 zz = v4<V4, T>(di.x * rr.x, di.y * rr.y, di.z * rr.z);
          reinterpret_cast<V4*>(a.r)[o] = rr;
          reinterpret_cast<V4*>(a.z)[o] = zz;
          reinterpret_cast<V4*>(a.p[0])[o] = v4<V4, T>(T(0), T(0), T(0));
          v[3 * k + 0] += double(rr.x) * zz.x + double(rr.y) * zz.y + double(rr.z) * zz.z;
          v[3 * k + 1] += double(rr.x) * rr.x + double(rr.y) * rr.y + double(rr.z) * rr.z;
          const double bx = (fx & 1) ? 0.0 : bb.x, by = (fx & 2) ? 0.0 : bb.y, bz = (fx & 4) ? 0.0 : bb.z;
          v[3 * k + 2] += bx * bx + by * by + bz * bz;
        }
      }
      __syncthreads();
    }
    write_partials<3 * R>(a.partials, v, red);
    proxy_fence_all();
    if (!ok) atomicExch(&a.bar->error, ST_TIMEOUT);
    ok = ok && grid_barrier(a.bar, G);
    if (ok) {
      reduce_partials<3 * R>(a.partials, G, v, red);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
          st.bnorm[k] = sqrt(v[3 * k + 2]);
          st.frozen[k] = 0;
          st.status[k] = ST_NOT_CONVERGED;
          st.iters[k] = 0;
          st.gamma_prev[k] = v[3 * k];     // rho = r.z
          st.relres[k] = st.bnorm[k] > 0.0 ? sqrt(v[3 * k + 1]) / st.bnorm[k] : 0.0;
          st.alpha[k] = 0.0;
          st.beta[k] = 0.0;
          if (!(st.bnorm[k] > 0.0)) {
            st.frozen[k] = 1;
            st.status[k] = isfinite(v[3 * k + 2]) ? ST_OK : ST_NONFINITE;
          } else if (!isfinite(v[3 * k]) || !isfinite(v[3 * k + 1])) {
            st.frozen[k] = 1; st.status[k] = ST_NONFINITE;
          } else if (st.relres[k] <= a.rtol) {
            st.frozen[k] = 1; st.status[k] = ST_OK;
          }
        }
      }
      __syncthreads();
    }
  }

  int pc = 0;   // p[pc] holds the previous search direction
  for (int it = 0; ok; ++it) {
    bool all = true;
#pragma unroll
    for (int k = 0; k < R; ++k) all = all && st.frozen[k];
    if (all || it >= a.maxiter) break;
    // ---- phase 1: p = z + beta p; q = A p; p.q
    double v[R];
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = 0.0;
    const int pn = pc ^ 1;
    for (int t = blockIdx.x; t < g.ntiles; t += G) {
      const TileGeom tg = tile_geom(g, t);
      if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(mbar, 2 * hbytes);
        tma_load_5d(sz, &a.tmz, 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, mbar);
        tma_load_5d(sp, &a.tmp[pc], 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, mbar);
      }
      if (!single) load_factor_tile(g, tg, a.fK, sf);
      ok = __syncthreads_and(ok && mbar_wait(mbar, phase, wait_budget(a.bar)));
      phase ^= 1;
      // p_new over the whole halo box (frozen rhs: untouched)
      for (int idx = threadIdx.x; idx < R * hsr; idx += blockDim.x) {
        const int k = idx / hsr;
        if (st.frozen[k]) continue;
        const T be = T(st.beta[k]);
        V4 pz = reinterpret_cast<V4*>(sz)[idx];
        V4 pp = reinterpret_cast<V4*>(sp)[idx];
        pp.x = fma(be, pp.x, pz.x); pp.y = fma(be, pp.y, pz.y); pp.z = fma(be, pp.z, pz.z); pp.w = T(0);
        reinterpret_cast<V4*>(sp)[idx] = pp;
      }
      __syncthreads();
      int tx, ty, tz, n;
      if (ok && thread_node(g, tg, tx, ty, tz, n)) {
        T acc[R][3];
        stencil_node<T, R>(sp, tg, sf, sKe, tx, ty, tz, acc);
        const uint8_t fx = __ldg(a.fix + n);
#pragma unroll
        for (int k = 0; k < R; ++k) {
          if (st.frozen[k]) continue;
          const size_t o = k * a.vs / 4 + n;
          const V4 pp = halo_center<T>(sp, tg, k, tx, ty, tz);
          const V4 qq = v4<V4, T>((fx & 1) ? T(0) : acc[k][0], (fx & 2) ? T(0) : acc[k][1],
                                  (fx & 4) ? T(0) : acc[k][2]);
          reinterpret_cast<V4*>(a.q)[o] = qq;
          reinterpret_cast<V4*>(a.p[pn])[o] = pp;
          v[k] += double(pp.x) * qq.x + double(pp.y) * qq.y + double(pp.z) * qq.z;
        }
      }
      __syncthreads();
    }
    write_partials<R>(a.partials, v, red);
    proxy_fence_all();
    if (!ok) { atomicExch(&a.bar->error, ST_TIMEOUT); break; }
    ok = grid_barrier(a.bar, G);
    if (!ok) break;
    reduce_partials<R>(a.partials, G, v, red);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < R; ++k) {
        if (st.frozen[k]) continue;
        if (!isfinite(v[k])) { st.frozen[k] = 1; st.status[k] = ST_NONFINITE; continue; }
        if (!(v[k] > 0.0)) { st.frozen[k] = 1; st.status[k] = ST_BREAKDOWN; continue; }
        st.alpha[k] = st.gamma_prev[k] / v[k];
      }
    }
    __syncthreads();
    // ---- phase 2: x += alpha p; r -= alpha q; z = D^-1 r; rho, ||r||^2
    double w[2 * R];
#pragma unroll
    for (int k = 0; k < 2 * R; ++k) w[k] = 0.0;
    for (int t = blockIdx.x; t < g.ntiles; t += G) {
      const TileGeom tg = tile_geom(g, t);
      int tx, ty, tz, n;
      if (!thread_node(g, tg, tx, ty, tz, n)) continue;
      const V4 di = reinterpret_cast<const V4*>(a.dinv)[n];
#pragma unroll
      for (int k = 0; k < R; ++k) {
        if (st.frozen[k]) continue;
        const size_t o = k * a.vs / 4 + n;
        const T al = T(st.alpha[k]);
        const V4 pp = reinterpret_cast<const V4*>(a.p[pn])[o];
        const V4 qq = reinterpret_cast<const V4*>(a.q)[o];
        V4 xx = reinterpret_cast<const V4*>(a.x)[o];
        V4 rr = reinterpret_cast<const V4*>(a.r)[o];
        xx.x = fma(al, pp.x, xx.x); xx.y = fma(al, pp.y, xx.y); xx.z = fma(al, pp.z, xx.z);
        rr.x = fma(-al, qq.x, rr.x); rr.y = fma(-al, qq.y, rr.y); rr.z = fma(-al, qq.z, rr.z);
        const V4 zz = v4<V4, T>(di.x * rr.x, di.y * rr.y, di.z * rr.z);
        reinterpret_cast<V4*>(a.x)[o] = xx;
        reinterpret_cast<V4*>(a.r)[o] = rr;
        reinterpret_cast<V4*>(a.z)[o] = zz;
        w[2 * k] += double(rr.x) * zz.x + double(rr.y) * zz.y + double(rr.z) * zz.z;
        w[2 * k + 1] += double(rr.x) * rr.x + double(rr.y) * rr.y + double(rr.z) * rr.z;
      }
    }
    write_partials<2 * R>(a.partials, w, red);
    proxy_fence_all();
    ok = grid_barrier(a.bar, G);
    if (!ok) break;
    pc = pn;
    reduce_partials<2 * R>(a.partials, G, w, red);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < R; ++k) {
        if (st.frozen[k]) continue;
        const double rz = w[2 * k], rr = w[2 * k + 1];
        st.iters[k] = it + 1;
        st.relres[k] = sqrt(rr) / st.bnorm[k];
        if (!isfinite(rz) || !isfinite(rr)) { st.frozen[k] = 1; st.status[k] = ST_NONFINITE; continue; }
        if (st.relres[k] <= a.rtol) { st.frozen[k] = 1; st.status[k] = ST_OK; continue; }
        st.beta[k] = rz / st.gamma_prev[k];
        st.gamma_prev[k] = rz;
      }
    }
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int err = ld_relaxed_i32(&a.bar->error);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      a.status[k] = err ? err : st.status[k];
      a.status[R + k] = st.iters[k];
      a.relres[k] = st.relres[k];
    }
  }
}

// ===========================================================================
// host launchers
// ===========================================================================
static size_t pipe_smem(const Grid& g, int R) {
  const int nfe = (g.TX + 1) * (g.TY + 1) * (g.TZ + 1);
  size_t s = halo_bytes<float>(g, R) + 4 * (kKeBlocksLen + nfe);
  s = (s + 15) & ~size_t(15);
  s += sizeof(double) * 3 * R * 32 + 16;
  return s;
}
template <typename T>
static size_t plain_smem(const Grid& g, int R) {
  const int nfe = (g.TX + 1) * (g.TY + 1) * (g.TZ + 1);
  size_t s = 2 * size_t(halo_bytes<T>(g, R)) + sizeof(T) * (kKeBlocksLen + nfe);
  s = (s + 15) & ~size_t(15);
  return s + sizeof(double) * 3 * R * 32 + 16;
}

template <int R>
static int pipe_launch(Ctx& c, const double* b, float* d, double rtol, int maxiter, cudaStream_t s) {
  PipeArgs<R> a;
  a.g = c.g;
  a.fK = c.fK32; a.keb = c.keb32; a.fix = c.fix; a.dinv = c.dinvK32; a.b = b;
  const size_t blk = (size_t)c.max_rhs * c.g.NN * 4;
  float* w = c.pw32;
  a.hb[0] = w; a.hb[1] = w + blk;
  a.x = d; a.r = w + 2 * blk; a.u = w + 3 * blk; a.w = w + 4 * blk; a.z = w + 5 * blk;
  a.q = w + 6 * blk; a.s = w + 7 * blk; a.p = w + 8 * blk;
  a.partials = c.partials; a.bar = c.bar; a.status = c.status; a.relres = c.scal;
  a.rtol = rtol; a.maxiter = maxiter; a.vs = (long long)c.g.NN * 4;
  std::string err;
  if (!encode_node4_map(&a.tmh[0], a.hb[0], c.g, R, false, &err) ||
      !encode_node4_map(&a.tmh[1], a.hb[1], c.g, R, false, &err)) { c.last_error = err; return -2; }
  const size_t smem = pipe_smem(c.g, R);
  auto kern = k_pcg_pipe<R>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, c.g.TX * c.g.TY * c.g.TZ, smem);
  if (per_sm < 1) { c.last_error = "pipelined PCG: tile does not fit on an SM"; return -2; }
  int grid = per_sm * c.num_sms;
  if (grid > c.g.ntiles) grid = c.g.ntiles;
  if (grid > c.partial_slots) grid = c.partial_slots;
  cudaMemsetAsync(c.bar, 0, kBarrierResetBytes, s);
  void* args[] = {(void*)&a};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(c.g.TX * c.g.TY * c.g.TZ), args,
                                              smem, s);
  count_launch();
  if (e != cudaSuccess) { c.last_error = cudaGetErrorString(e); return -2; }
  return 0;
}

template <typename T, int R>
static int plain_launch(Ctx& c, const double* b, T* x, double rtol, int maxiter, cudaStream_t s) {
  constexpr bool f64 = sizeof(T) == 8;
  PlainArgs<T, R> a;
  a.g = c.g;
  if constexpr (f64) {
    a.fK = c.fK64; a.keb = c.keb64; a.dinv = c.dinvK64;
  } else {
    a.fK = c.fK32; a.keb = c.keb32; a.dinv = c.dinvK32;
  }
  a.fix = c.fix; a.b = b;
  const size_t blk = (size_t)c.max_rhs * c.g.NN * 4;
  T* w;
  if constexpr (f64) w = c.pw64; else w = c.pw32 + blk;   // FP32: slots 2..6
  a.x = x; a.r = w + blk; a.z = w + 2 * blk; a.q = w + 3 * blk; a.p[0] = w + 4 * blk; a.p[1] = w + 5 * blk;
  a.partials = c.partials; a.bar = c.bar; a.status = c.status; a.relres = c.scal;
  a.rtol = rtol; a.maxiter = maxiter; a.vs = (long long)c.g.NN * 4;
  std::string err;
  if (!encode_node4_map(&a.tmx, a.x, c.g, R, f64, &err) || !encode_node4_map(&a.tmz, a.z, c.g, R, f64, &err) ||
      !encode_node4_map(&a.tmp[0], a.p[0], c.g, R, f64, &err) ||
      !encode_node4_map(&a.tmp[1], a.p[1], c.g, R, f64, &err)) { c.last_error = err; return -2; }
  const size_t smem = plain_smem<T>(c.g, R);
  auto kern = k_pcg_plain<T, R>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, c.g.TX * c.g.TY * c.g.TZ, smem);
  if (per_sm < 1) { c.last_error = "plain PCG: tile does not fit on an SM"; return -2; }
  int grid = per_sm * c.num_sms;
  if (grid > c.g.ntiles) grid = c.g.ntiles;
  if (grid > c.partial_slots) grid = c.partial_slots;
  cudaMemsetAsync(c.bar, 0, kBarrierResetBytes, s);
  void* args[] = {(void*)&a};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(c.g.TX * c.g.TY * c.g.TZ), args,
                                              smem, s);
  count_launch();
  if (e != cudaSuccess) { c.last_error = cudaGetErrorString(e); return -2; }
  return 0;
}

__global__ void __launch_bounds__(32) k_barrier_selftest(BarrierState* bar, unsigned expected) {
  grid_barrier(bar, expected);
}

int launch_barrier_selftest(Ctx& c, int G, int expected, cudaStream_t s) {
  unsigned exp = (unsigned)expected;
  void* args[] = {(void*)&c.bar, (void*)&exp};
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_barrier_selftest, dim3(G), dim3(32), args, 0, s);
  count_launch();
  if (e != cudaSuccess) { c.last_error = cudaGetErrorString(e); return -2; }
  return 0;
}

int pcg_plain64(Ctx& c, const double* b, double* x, int R, double rtol, int maxiter, int*, double*, int*,
                cudaStream_t s) {
  switch (R) {
    case 1: return plain_launch<double, 1>(c, b, x, rtol, maxiter, s);
    case 2: return plain_launch<double, 2>(c, b, x, rtol, maxiter, s);
    case 4: return plain_launch<double, 4>(c, b, x, rtol, maxiter, s);
    case 8: return plain_launch<double, 8>(c, b, x, rtol, maxiter, s);
  }
  c.last_error = "plain PCG: nrhs must be 1, 2, 4 or 8";
  return -1;
}

int pcg_std32(Ctx& c, const double* b, float* x, int R, double rtol, int maxiter, cudaStream_t s) {
  switch (R) {
    case 1: return plain_launch<float, 1>(c, b, x, rtol, maxiter, s);
    case 2: return plain_launch<float, 2>(c, b, x, rtol, maxiter, s);
    case 4: return plain_launch<float, 4>(c, b, x, rtol, maxiter, s);
    case 8: return plain_launch<float, 8>(c, b, x, rtol, maxiter, s);
  }
  c.last_error = "FP32 PCG: nrhs must be 1, 2, 4 or 8";
  return -1;
}

int pcg_pipe32(Ctx& c, const double* b, float* d, int R, double rtol, int maxiter, int*, double*, int*,
               cudaStream_t s) {
  switch (R) {
    case 1: return pipe_launch<1>(c, b, d, rtol, maxiter, s);
    case 2: return pipe_launch<2>(c, b, d, rtol, maxiter, s);
    case 4: return pipe_launch<4>(c, b, d, rtol, maxiter, s);
    case 8: return pipe_launch<8>(c, b, d, rtol, maxiter, s);
  }
  c.last_error = "pipelined PCG: nrhs must be 1, 2, 4 or 8";
  return -1;
}

// Load every kernel of this file now (CUDA loads device functions lazily,
// at first use, and a first use in the middle of a solve stalls it).
void preload_kernels_pcg() {
  auto touch = [](auto f) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(f));
  };
  touch(k_pcg_pipe<1>); touch(k_pcg_pipe<2>); touch(k_pcg_pipe<4>); touch(k_pcg_pipe<8>);
  touch(k_pcg_plain<double, 1>); touch(k_pcg_plain<double, 2>); touch(k_pcg_plain<double, 4>);
  touch(k_pcg_plain<double, 8>); touch(k_pcg_plain<float, 1>); touch(k_pcg_plain<float, 2>);
  touch(k_pcg_plain<float, 4>); touch(k_pcg_plain<float, 8>); touch(k_barrier_selftest);
}

}  // namespace tof

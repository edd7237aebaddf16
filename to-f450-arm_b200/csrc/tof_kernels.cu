// Standalone (one-launch) kernels of the voxel SIMP path.
#include <math.h>

#include "tof_internal.h"
#include "tof_stencil.cuh"

namespace tof {

// ---------------------------------------------------------------------------
// SIMP factors.  Stiffness: emin + (1 - emin) rho^p (src/fem.py:316-320).
// Mass (Pedersen): rho for rho >= t, t (max(rho,0)/t)^q below
// (src/fem.py:334-349).  Elements outside the active set get 0 (they are not
// part of the reference's assembly at all).
// ---------------------------------------------------------------------------
__global__ void k_factors(int NE, const double* __restrict__ rho, const uint8_t* __restrict__ active,
                          SimpParams sp, double* fK64, double* fM64, float* fK32, float* fM32) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NE) return;
  double fk = 0.0, fm = 0.0;
  if (active[e]) {
    const double r = rho[e];
    fk = sp.emin + (1.0 - sp.emin) * pow(r, sp.penal);
    fm = (r >= sp.mass_threshold) ? r : sp.mass_threshold * pow(fmax(r, 0.0) / sp.mass_threshold, sp.mass_q);
  }
  fK64[e] = fk; fM64[e] = fm;
  fK32[e] = float(fk); fM32[e] = float(fm);
}

void launch_factors(Ctx& c, const double* rho, cudaStream_t s) {
  const int NE = c.g.NE;
  k_factors<<<ceil_div(NE, 256), 256, 0, s>>>(NE, rho, c.active, c.sp, c.fK64, c.fM64, c.fK32, c.fM32);
  count_launch();
}

// ---------------------------------------------------------------------------
// Diagonals of K and M (node4) and the Jacobi inverse of diag K.  Fixed DOFs
// get diag 0 and inverse 0, so preconditioned vectors stay zero there.  The
// reference's Jacobi preconditioner is 1 / diag(K_ff) (src/fem.py:543-544).
// ---------------------------------------------------------------------------
__global__ void k_diag(Grid g, const double* __restrict__ fK, const double* __restrict__ fM,
                       const double* __restrict__ Ke, const double* __restrict__ Me,
                       const uint8_t* __restrict__ fix, const double* __restrict__ tip, double* dK, double* dM,
                       double* dinv64, float* dinv32) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.NN) return;
  const int i = n % g.NX, j = (n / g.NX) % g.NY, k = n / (g.NX * g.NY);
  double sk[3] = {0, 0, 0}, sm[3] = {0, 0, 0};
  for (int c = -1; c <= 0; ++c)
    for (int b = -1; b <= 0; ++b)
      for (int a = -1; a <= 0; ++a) {
        const int ex = i + a, ey = j + b, ez = k + c;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= g.nx || ey >= g.ny || ez >= g.nz) continue;
        const int e = (ez * g.ny + ey) * g.nx + ex;
        const int ln = local_node(-a, -b, -c);
        for (int q = 0; q < 3; ++q) {
          const int d = (3 * ln + q) * 24 + 3 * ln + q;
          sk[q] += fK[e] * Ke[d];
          sm[q] += fM[e] * Me[d];
        }
      }
  const uint8_t fx = fix[n];
  for (int q = 0; q < 3; ++q) {
    const bool fixed = (fx >> q) & 1;
    const double kq = fixed ? 0.0 : sk[q];
    const double mq = fixed ? 0.0 : sm[q] + tip[4 * n + q];
    dK[4 * n + q] = kq;
    dM[4 * n + q] = mq;
    const double inv = (fixed || kq == 0.0) ? 0.0 : 1.0 / kq;
    dinv64[4 * n + q] = inv;
    dinv32[4 * n + q] = float(inv);
  }
  dK[4 * n + 3] = dM[4 * n + 3] = dinv64[4 * n + 3] = 0.0;
  dinv32[4 * n + 3] = 0.f;
}

void launch_diag(Ctx& c, cudaStream_t s) {
  k_diag<<<ceil_div(c.g.NN, 256), 256, 0, s>>>(c.g, c.fK64, c.fM64, c.Ke64, c.Me64, c.fix, c.tip64, c.dK64,
                                                 c.dM64, c.dinvK64, c.dinvK32);
  count_launch();
}

// ---------------------------------------------------------------------------
// Standalone block matvec: y = A x (or y = b - A x) for R node4 vectors, one
// node tile per CTA.  Input vectors must be zero at fixed DOFs (pack()
// guarantees that).
// ---------------------------------------------------------------------------
template <typename T>
struct MatvecArgs {
  Grid g;
  const T* fe;         // element factors
  const T* keb;        // 64-block matrix
  const uint8_t* fix;
  const T* tip;        // node4 lumped mass (M only) or null
  const T* b;          // residual mode: rhs, else null
  T* y;
  long long vstride;   // elements between consecutive vectors (NN*4)
  // smoother mode (with b): y = sx x + sp y_prev + sr D^-1 (b - A x), the
  // coefficients (sx, sp, sr) a device triple; y_prev (the output buffer's
  // previous content, own node only) is read only with prev
  const T* dinv;
  const float* coef;
  bool prev;
};

template <typename T, int R>
__global__ void __launch_bounds__(512) k_matvec(const __grid_constant__ CUtensorMap tmx, MatvecArgs<T> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  using V4 = typename Vec4<T>::type;
  const Grid& g = a.g;
  const TileGeom tg = tile_geom(g, blockIdx.x);
  T* sx = reinterpret_cast<T*>(smem_raw);
  const unsigned hb = halo_bytes<T>(g, R);
  T* sKe = reinterpret_cast<T*>(smem_raw + hb);
  T* sf = sKe + kKeBlocksLen;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ((hb + sizeof(T) * (kKeBlocksLen + tg.EX * tg.EY * tg.EZ) + 15) & ~15u));
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, hb);
    tma_load_5d(sx, &tmx, 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, bar);
  }
  load_ke_blocks(a.keb, sKe);
  load_factor_tile(g, tg, a.fe, sf);
  __syncthreads();
  if (!mbar_wait(bar, 0)) return;
  int tx, ty, tz, n;
  if (!thread_node(g, tg, tx, ty, tz, n)) return;
  T acc[R][3];
  stencil_node<T, R>(sx, tg, sf, sKe, tx, ty, tz, acc);
  const uint8_t fx = __ldg(a.fix + n);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (a.tip) {
      const V4 xc = halo_center<T>(sx, tg, r, tx, ty, tz);
      const V4 tp = reinterpret_cast<const V4*>(a.tip)[n];
      acc[r][0] = fma(tp.x, xc.x, acc[r][0]);
      acc[r][1] = fma(tp.y, xc.y, acc[r][1]);
      acc[r][2] = fma(tp.z, xc.z, acc[r][2]);
    }
    V4 out;
    if (a.b) {
      const V4 bb = reinterpret_cast<const V4*>(a.b + r * a.vstride)[n];
      out.x = bb.x - acc[r][0]; out.y = bb.y - acc[r][1]; out.z = bb.z - acc[r][2];
      if (a.dinv) {
        const V4 xc = halo_center<T>(sx, tg, r, tx, ty, tz);
        const V4 di = reinterpret_cast<const V4*>(a.dinv)[n];
        const T cx = T(__ldg(a.coef)), cr = T(__ldg(a.coef + 2));
        out.x = fma(cr * di.x, out.x, cx * xc.x);
        out.y = fma(cr * di.y, out.y, cx * xc.y);
        out.z = fma(cr * di.z, out.z, cx * xc.z);
        if (a.prev) {
          const T cp = T(__ldg(a.coef + 1));
          const V4 yp = reinterpret_cast<const V4*>(a.y + r * a.vstride)[n];
          out.x = fma(cp, yp.x, out.x);
          out.y = fma(cp, yp.y, out.y);
          out.z = fma(cp, yp.z, out.z);
        }
      }
    } else {
      out.x = acc[r][0]; out.y = acc[r][1]; out.z = acc[r][2];
    }
    out.x = (fx & 1) ? T(0) : out.x;
    out.y = (fx & 2) ? T(0) : out.y;
    out.z = (fx & 4) ? T(0) : out.z;
    out.w = T(0);
    reinterpret_cast<V4*>(a.y + r * a.vstride)[n] = out;
  }
}

template <typename T, int R>
static int matvec_launch_t(Ctx& c, int op, const void* x, void* y, const void* b, cudaStream_t s,
                           const void* dinv = nullptr, const float* coef = nullptr, bool prev = false) {
  CUtensorMap tm;
  std::string err;
  if (!encode_node4_map(&tm, x, c.g, R, sizeof(T) == 8, &err)) {
    c.last_error = err;
    return -2;
  }
  MatvecArgs<T> a;
  a.g = c.g;
  const bool f64 = sizeof(T) == 8;
  if (op == 2 && !f64) {
    c.last_error = "|K| products are FP64 only";
    return -2;
  }
  a.fe = reinterpret_cast<const T*>(op != 1 ? (f64 ? (const void*)c.fK64 : (const void*)c.fK32)
                                            : (f64 ? (const void*)c.fM64 : (const void*)c.fM32));
  a.keb = reinterpret_cast<const T*>(op == 0   ? (f64 ? (const void*)c.keb64 : (const void*)c.keb32)
                                     : op == 1 ? (f64 ? (const void*)c.meb64 : (const void*)c.meb32)
                                               : (const void*)c.kebabs64);
  a.fix = c.fix;
  a.tip = op == 1 ? reinterpret_cast<const T*>(f64 ? (const void*)c.tip64 : (const void*)c.tip32) : nullptr;
  a.b = reinterpret_cast<const T*>(b);
  a.y = reinterpret_cast<T*>(y);
  a.vstride = (long long)c.g.NN * 4;
  a.dinv = reinterpret_cast<const T*>(dinv);
  a.coef = coef;
  a.prev = prev;
  const TileGeom tg{0, 0, 0, c.g.TX + 2, c.g.TY + 2, c.g.TZ + 2, c.g.TX + 1, c.g.TY + 1, c.g.TZ + 1};
  size_t smem = halo_bytes<T>(c.g, R) + sizeof(T) * (kKeBlocksLen + tg.EX * tg.EY * tg.EZ);
  smem = ((smem + 15) & ~size_t(15)) + 16;
  auto kern = k_matvec<T, R>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<c.g.ntiles, c.g.TX * c.g.TY * c.g.TZ, smem, s>>>(tm, a);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_matvec(Ctx& c, int op, bool f64, const void* x, void* y, int nrhs, const void* b, cudaStream_t s) {
  // split into chunks of at most 8 vectors
  const size_t esz = f64 ? 8 : 4;
  const long long vbytes = (long long)c.g.NN * 4 * esz;
  int done = 0;
  while (done < nrhs) {
    int R = nrhs - done;
    R = R >= 8 ? 8 : R >= 4 ? 4 : R >= 2 ? 2 : 1;
    const char* xp = (const char*)x + done * vbytes;
    char* yp = (char*)y + done * vbytes;
    const char* bp = b ? (const char*)b + done * vbytes : nullptr;
    int rc;
    if (f64) {
      switch (R) {
        case 8: rc = matvec_launch_t<double, 8>(c, op, xp, yp, bp, s); break;
        case 4: rc = matvec_launch_t<double, 4>(c, op, xp, yp, bp, s); break;
        case 2: rc = matvec_launch_t<double, 2>(c, op, xp, yp, bp, s); break;
        default: rc = matvec_launch_t<double, 1>(c, op, xp, yp, bp, s); break;
      }
    } else {
      switch (R) {
        case 8: rc = matvec_launch_t<float, 8>(c, op, xp, yp, bp, s); break;
        case 4: rc = matvec_launch_t<float, 4>(c, op, xp, yp, bp, s); break;
        case 2: rc = matvec_launch_t<float, 2>(c, op, xp, yp, bp, s); break;
        default: rc = matvec_launch_t<float, 1>(c, op, xp, yp, bp, s); break;
      }
    }
    if (rc) return rc;
    done += R;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// K x and M x of the same R vectors in one launch (LOBPCG's block products):
// one TMA halo load of x and both element-matrix block sets staged per CTA;
// each thread forms its node's K row, stores it, then its M row (plus the
// lumped tip mass).  The same per-operator arithmetic as k_matvec, so the
// results are bit-identical to two k_matvec launches.
// ---------------------------------------------------------------------------
template <typename T>
struct MatvecKMArgs {
  Grid g;
  const T* fK;
  const T* fM;
  const T* kebK;
  const T* kebM;
  const uint8_t* fix;
  const T* tip;
  T* yK;
  T* yM;
  long long vstride;
};

template <typename T, int R>
__global__ void __launch_bounds__(512) k_matvec_km(const __grid_constant__ CUtensorMap tmx, MatvecKMArgs<T> a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  using V4 = typename Vec4<T>::type;
  const Grid& g = a.g;
  const TileGeom tg = tile_geom(g, blockIdx.x);
  const int nfe = tg.EX * tg.EY * tg.EZ;
  T* sx = reinterpret_cast<T*>(smem_raw);
  const unsigned hb = halo_bytes<T>(g, R);
  T* sKeK = reinterpret_cast<T*>(smem_raw + hb);
  T* sKeM = sKeK + kKeBlocksLen;
  T* sfK = sKeM + kKeBlocksLen;
  T* sfM = sfK + nfe;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ((hb + sizeof(T) * (2 * kKeBlocksLen + 2 * nfe) + 15) & ~15u));
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, hb);
    tma_load_5d(sx, &tmx, 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, bar);
  }
  load_ke_blocks(a.kebK, sKeK);
  load_ke_blocks(a.kebM, sKeM);
  load_factor_tile(g, tg, a.fK, sfK);
  load_factor_tile(g, tg, a.fM, sfM);
  __syncthreads();   // mbarrier initialised before anyone waits on it
  if (!__syncthreads_and(mbar_wait(bar, 0))) return;
  int tx, ty, tz, n;
  const bool live = thread_node(g, tg, tx, ty, tz, n);
  const uint8_t fx = live ? __ldg(a.fix + n) : uint8_t(0);
  if (live) {
    T acc[R][3];
    stencil_node<T, R>(sx, tg, sfK, sKeK, tx, ty, tz, acc);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      V4 out;
      out.x = (fx & 1) ? T(0) : acc[r][0];
      out.y = (fx & 2) ? T(0) : acc[r][1];
      out.z = (fx & 4) ? T(0) : acc[r][2];
      out.w = T(0);
      reinterpret_cast<V4*>(a.yK + r * a.vstride)[n] = out;
    }
  }
  // the CTA barrier keeps the two products from being interleaved (which
  // would double the live registers)
  __syncthreads();
  if (live) {
    T acc[R][3];
    stencil_node<T, R>(sx, tg, sfM, sKeM, tx, ty, tz, acc);
    const V4 tp = reinterpret_cast<const V4*>(a.tip)[n];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const V4 xc = halo_center<T>(sx, tg, r, tx, ty, tz);
      acc[r][0] = fma(tp.x, xc.x, acc[r][0]);
      acc[r][1] = fma(tp.y, xc.y, acc[r][1]);
      acc[r][2] = fma(tp.z, xc.z, acc[r][2]);
      V4 out;
      out.x = (fx & 1) ? T(0) : acc[r][0];
      out.y = (fx & 2) ? T(0) : acc[r][1];
      out.z = (fx & 4) ? T(0) : acc[r][2];
      out.w = T(0);
      reinterpret_cast<V4*>(a.yM + r * a.vstride)[n] = out;
    }
  }
}

template <typename T, int R>
static int matvec_km_launch_t(Ctx& c, const void* x, void* yK, void* yM, cudaStream_t s) {
  CUtensorMap tm;
  std::string err;
  constexpr bool f64 = sizeof(T) == 8;
  if (!encode_node4_map(&tm, x, c.g, R, f64, &err)) {
    c.last_error = err;
    return -2;
  }
  MatvecKMArgs<T> a;
  a.g = c.g;
  a.fK = reinterpret_cast<const T*>(f64 ? (const void*)c.fK64 : (const void*)c.fK32);
  a.fM = reinterpret_cast<const T*>(f64 ? (const void*)c.fM64 : (const void*)c.fM32);
  a.kebK = reinterpret_cast<const T*>(f64 ? (const void*)c.keb64 : (const void*)c.keb32);
  a.kebM = reinterpret_cast<const T*>(f64 ? (const void*)c.meb64 : (const void*)c.meb32);
  a.fix = c.fix;
  a.tip = reinterpret_cast<const T*>(f64 ? (const void*)c.tip64 : (const void*)c.tip32);
  a.yK = reinterpret_cast<T*>(yK);
  a.yM = reinterpret_cast<T*>(yM);
  a.vstride = (long long)c.g.NN * 4;
  const int nfe = (c.g.TX + 1) * (c.g.TY + 1) * (c.g.TZ + 1);
  size_t smem = halo_bytes<T>(c.g, R) + sizeof(T) * (2 * kKeBlocksLen + 2 * nfe);
  smem = ((smem + 15) & ~size_t(15)) + 16;
  auto kern = k_matvec_km<T, R>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<c.g.ntiles, c.g.TX * c.g.TY * c.g.TZ, smem, s>>>(tm, a);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// yK = K x, yM = M x for nrhs vectors (chunks of at most 8, as launch_matvec)
int launch_matvec_km(Ctx& c, bool f64, const void* x, void* yK, void* yM, int nrhs, cudaStream_t s) {
  const size_t esz = f64 ? 8 : 4;
  const long long vbytes = (long long)c.g.NN * 4 * esz;
  int done = 0;
  while (done < nrhs) {
    int R = nrhs - done;
    R = R >= 8 ? 8 : R >= 4 ? 4 : R >= 2 ? 2 : 1;
    const char* xp = (const char*)x + done * vbytes;
    char* kp = (char*)yK + done * vbytes;
    char* mp = (char*)yM + done * vbytes;
    int rc;
    if (f64) {
      switch (R) {
        case 8: rc = matvec_km_launch_t<double, 8>(c, xp, kp, mp, s); break;
        case 4: rc = matvec_km_launch_t<double, 4>(c, xp, kp, mp, s); break;
        case 2: rc = matvec_km_launch_t<double, 2>(c, xp, kp, mp, s); break;
        default: rc = matvec_km_launch_t<double, 1>(c, xp, kp, mp, s); break;
      }
    } else {
      switch (R) {
        case 8: rc = matvec_km_launch_t<float, 8>(c, xp, kp, mp, s); break;
        case 4: rc = matvec_km_launch_t<float, 4>(c, xp, kp, mp, s); break;
        case 2: rc = matvec_km_launch_t<float, 2>(c, xp, kp, mp, s); break;
        default: rc = matvec_km_launch_t<float, 1>(c, xp, kp, mp, s); break;
      }
    }
    if (rc) return rc;
    done += R;
  }
  return 0;
}

// y = sx x + sp y_prev + sr D^-1 (b - K x) on the fine level, FP32, R in
// {1,2,4,8}; coef = device (sx, sp, sr), y_prev read only with prev
int launch_smooth0(Ctx& c, const float* x, float* y, const float* b, const float* dinv, const float* coef, bool prev,
                   int R, cudaStream_t s) {
  switch (R) {
    case 8: return matvec_launch_t<float, 8>(c, 0, x, y, b, s, dinv, coef, prev);
    case 4: return matvec_launch_t<float, 4>(c, 0, x, y, b, s, dinv, coef, prev);
    case 2: return matvec_launch_t<float, 2>(c, 0, x, y, b, s, dinv, coef, prev);
    default: return matvec_launch_t<float, 1>(c, 0, x, y, b, s, dinv, coef, prev);
  }
}

// ---------------------------------------------------------------------------
// DOF-major (the reference's 3*n + c layout) <-> node4, with the fixed-DOF
// restriction applied on the way in.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_pack(int NN, int nvec, const double* __restrict__ src, long long ld, const uint8_t* fix, T* dst) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)NN * nvec) return;
  const int v = int(idx / NN), n = int(idx % NN);
  const double* s = src + v * ld + 3 * (long long)n;
  const uint8_t fx = fix[n];
  typename Vec4<T>::type o;
  o.x = (fx & 1) ? T(0) : T(s[0]);
  o.y = (fx & 2) ? T(0) : T(s[1]);
  o.z = (fx & 4) ? T(0) : T(s[2]);
  o.w = T(0);
  reinterpret_cast<typename Vec4<T>::type*>(dst)[idx] = o;
}

template <typename T>
__global__ void k_unpack(int NN, int nvec, const T* __restrict__ src, double* dst, long long ld) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)NN * nvec) return;
  const int v = int(idx / NN), n = int(idx % NN);
  const typename Vec4<T>::type i = reinterpret_cast<const typename Vec4<T>::type*>(src)[idx];
  double* d = dst + v * ld + 3 * (long long)n;
  d[0] = double(i.x); d[1] = double(i.y); d[2] = double(i.z);
}

void launch_pack(const Ctx& c, const double* src, long long ld, void* dst, bool f64, int nvec, cudaStream_t s) {
  const long long n = (long long)c.g.NN * nvec;
  const int blocks = int((n + 255) / 256);
  if (f64) k_pack<double><<<blocks, 256, 0, s>>>(c.g.NN, nvec, src, ld, c.fix, (double*)dst);
  else k_pack<float><<<blocks, 256, 0, s>>>(c.g.NN, nvec, src, ld, c.fix, (float*)dst);
  count_launch();
}

void launch_unpack(const Ctx& c, const void* src, bool f64, double* dst, long long ld, int nvec, cudaStream_t s) {
  const long long n = (long long)c.g.NN * nvec;
  const int blocks = int((n + 255) / 256);
  if (f64) k_unpack<double><<<blocks, 256, 0, s>>>(c.g.NN, nvec, (const double*)src, dst, ld);
  else k_unpack<float><<<blocks, 256, 0, s>>>(c.g.NN, nvec, (const float*)src, dst, ld);
  count_launch();
}

// ---------------------------------------------------------------------------
// Gram matrix G = A^T B of two blocks of node4 vectors (na, nb <= 24) with
// FP64 accumulation.
//
// Stage 1 (k_gram_partial): each CTA stages a chunk of kGramChunk nodes of all
// na + nb vectors in shared memory (converted to FP64, one padded row per
// vector) and every warp accumulates the full 24 x 24 product over its own
// nodes of the chunk: lane (rg, cg) = (lane & 7, lane >> 3) owns rows
// 3rg..3rg+2 and columns 6cg..6cg+5, i.e. 9 shared loads per 18 FMAs.  The
// row pitch kGramLd (98 doubles: consecutive rows start 4 banks apart) makes
// both the 8 distinct row reads and the 4 distinct column reads of a warp
// conflict-free.  The 8 warps' tiles are summed in a fixed order into one
// partial per CTA.
// Stage 2 (k_gram_reduce): one warp per output sums the CTA partials in a
// fixed lane-strided order (deterministic).
// ---------------------------------------------------------------------------
constexpr int kGramThreads = 256;
constexpr int kGramChunk = 24;                       // nodes per staged chunk
constexpr int kGramLd = 4 * kGramChunk + 2;          // doubles per staged vector row

template <typename T>
__global__ void __launch_bounds__(kGramThreads) k_gram_partial(int NN, const T* __restrict__ A, ColMap ma, int na,
                                                              const T* __restrict__ B, ColMap mb, int nb,
                                                              long long vstride, double* part) {
  using V4 = typename Vec4<T>::type;
  __shared__ __align__(16) double sm[48 * kGramLd];   // rows 0..23: A, 24..47: B
  static_assert(48 * kGramLd >= 8 * 576, "reduction scratch");
  double* sA = sm;
  double* sB = sm + 24 * kGramLd;
  for (int i = threadIdx.x; i < 48 * kGramLd; i += blockDim.x) sm[i] = 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rg = lane & 7, cg = lane >> 3;
  double acc[3][6];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) acc[i][j] = 0.0;
  const int nchunks = (NN + kGramChunk - 1) / kGramChunk;
  const int nstage = (na + nb) * kGramChunk;
  for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int n0 = ch * kGramChunk;
    const int cnt = min(kGramChunk, NN - n0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nstage; idx += blockDim.x) {
      const int v = idx / kGramChunk, q = idx % kGramChunk;
      if (q >= cnt) continue;
      const bool isA = v < na;
      const T* src = isA ? A + ma.col[v] * vstride : B + mb.col[v - na] * vstride;
      const V4 x = reinterpret_cast<const V4*>(src)[n0 + q];
      double* d = (isA ? sA + v * kGramLd : sB + (v - na) * kGramLd) + 4 * q;
      reinterpret_cast<double2*>(d)[0] = make_double2(double(x.x), double(x.y));
      reinterpret_cast<double2*>(d)[1] = make_double2(double(x.z), 0.0);
    }
    __syncthreads();
    const double* pa = sA + 3 * rg * kGramLd;
    const double* pb = sB + 6 * cg * kGramLd;
    for (int q = w; q < cnt; q += kGramThreads / 32) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int o = 4 * q + c;
        double a[3], b[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) a[i] = pa[i * kGramLd + o];
#pragma unroll
        for (int j = 0; j < 6; ++j) b[j] = pb[j * kGramLd + o];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 6; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
    }
  }
  // CTA reduction of the 8 warp tiles (fixed order)
  __syncthreads();
  double* red = sm;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) red[w * 576 + (3 * rg + i) * 24 + 6 * cg + j] = acc[i][j];
  __syncthreads();
  for (int p = threadIdx.x; p < na * nb; p += blockDim.x) {
    const int r = p / nb, col = p % nb;
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kGramThreads / 32; ++k) sum += red[k * 576 + r * 24 + col];
    part[(size_t)blockIdx.x * 576 + p] = sum;
  }
}

__global__ void __launch_bounds__(256) k_gram_reduce(int nblocks, int npair, const double* __restrict__ part,
                                                     double* G) {
  const int p = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= npair) return;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += part[(size_t)b * 576 + p];
  s = warp_sum(s);
  if (lane == 0) G[p] = s;
}

// Two Gram matrices with a shared left block, G1 = S^T B1 and G2 = S^T B2
// (the K and M Grams of LOBPCG's Rayleigh-Ritz), from one staging of S: the
// same warp tiling as k_gram_partial with 16-node chunks (three staged
// blocks), partials [block][2][576].
constexpr int kGram2Chunk = 16;
constexpr int kGram2Ld = 4 * kGram2Chunk + 2;      // 66 doubles: rows 4 banks apart

template <typename T>
__global__ void __launch_bounds__(kGramThreads) k_gram2_partial(int NN, const T* __restrict__ A,
                                                               const T* __restrict__ B1, const T* __restrict__ B2,
                                                               ColMap cols, int n, long long vstride, double* part) {
  using V4 = typename Vec4<T>::type;
  __shared__ __align__(16) double sm[72 * kGram2Ld];   // rows 0..23: S, 24..47: B1, 48..71: B2
  static_assert(72 * kGram2Ld >= 8 * 576, "reduction scratch");
  for (int i = threadIdx.x; i < 72 * kGram2Ld; i += blockDim.x) sm[i] = 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rg = lane & 7, cg = lane >> 3;
  double acc1[3][6], acc2[3][6];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) acc1[i][j] = acc2[i][j] = 0.0;
  const int nchunks = (NN + kGram2Chunk - 1) / kGram2Chunk;
  const int nstage = 3 * n * kGram2Chunk;
  for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int n0 = ch * kGram2Chunk;
    const int cnt = min(kGram2Chunk, NN - n0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nstage; idx += blockDim.x) {
      const int v = idx / kGram2Chunk, q = idx % kGram2Chunk;
      if (q >= cnt) continue;
      const int blk = v / n, col = v % n;
      const T* base = blk == 0 ? A : blk == 1 ? B1 : B2;
      const V4 x = reinterpret_cast<const V4*>(base + cols.col[col] * vstride)[n0 + q];
      double* d = sm + (blk * 24 + col) * kGram2Ld + 4 * q;
      reinterpret_cast<double2*>(d)[0] = make_double2(double(x.x), double(x.y));
      reinterpret_cast<double2*>(d)[1] = make_double2(double(x.z), 0.0);
    }
    __syncthreads();
    const double* pa = sm + 3 * rg * kGram2Ld;
    const double* pb1 = sm + (24 + 6 * cg) * kGram2Ld;
    const double* pb2 = sm + (48 + 6 * cg) * kGram2Ld;
    for (int q = w; q < cnt; q += kGramThreads / 32) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int o = 4 * q + c;
        double a[3], b1[6], b2[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) a[i] = pa[i * kGram2Ld + o];
#pragma unroll
        for (int j = 0; j < 6; ++j) { b1[j] = pb1[j * kGram2Ld + o]; b2[j] = pb2[j * kGram2Ld + o]; }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 6; ++j) {
            acc1[i][j] = fma(a[i], b1[j], acc1[i][j]);
            acc2[i][j] = fma(a[i], b2[j], acc2[i][j]);
          }
      }
    }
  }
  double* red = sm;                                    // [warp][576], one Gram at a time
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) red[w * 576 + (3 * rg + i) * 24 + 6 * cg + j] = g == 0 ? acc1[i][j] : acc2[i][j];
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int r = e / n, col = e % n;
      double sum = 0.0;
#pragma unroll
      for (int k = 0; k < kGramThreads / 32; ++k) sum += red[k * 576 + r * 24 + col];
      part[(size_t)blockIdx.x * 1152 + g * 576 + e] = sum;
    }
  }
}

// FP64 inputs (LOBPCG's block vectors): the same tiling, with the staging of
// chunk i + 1 overlapped with the products of chunk i.  A node4 FP64 record
// (32 B, padding component 0) is copied unchanged into its row of the staging
// buffer by two 16-byte cp.async operations, double-buffered in dynamic
// shared memory; two CTAs per SM.
constexpr size_t kGram2Smem = 2 * 72 * kGram2Ld * sizeof(double);

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(kGramThreads, 2) k_gram2_partial_f64(int NN, const double* __restrict__ A,
                                                                       const double* __restrict__ B1,
                                                                       const double* __restrict__ B2, ColMap cols,
                                                                       int n, long long vstride, double* part) {
  extern __shared__ __align__(16) double dsm[];     // [2][72 * kGram2Ld]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rg = lane & 7, cg = lane >> 3;
  double acc1[3][6], acc2[3][6];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) acc1[i][j] = acc2[i][j] = 0.0;
  const int nchunks = (NN + kGram2Chunk - 1) / kGram2Chunk;
  const int nstage = 3 * n * kGram2Chunk;
  auto stage = [&](int ch, double* buf) {
    const int n0 = ch * kGram2Chunk;
    const int cnt = min(kGram2Chunk, NN - n0);
    for (int idx = threadIdx.x; idx < nstage; idx += blockDim.x) {
      const int v = idx / kGram2Chunk, q = idx % kGram2Chunk;
      if (q >= cnt) continue;
      const int blk = v / n, col = v % n;
      const double* base = blk == 0 ? A : blk == 1 ? B1 : B2;
      const double* src = base + cols.col[col] * vstride + 4 * (size_t)(n0 + q);
      double* d = buf + (blk * 24 + col) * kGram2Ld + 4 * q;
      cp_async16(d, src);
      cp_async16(d + 2, src + 2);
    }
  };
  int cur = 0;
  if (blockIdx.x < nchunks) stage(blockIdx.x, dsm);
  cp_async_commit();
  for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int nx = ch + gridDim.x;
    if (nx < nchunks) stage(nx, dsm + (cur ^ 1) * 72 * kGram2Ld);
    cp_async_commit();
    cp_async_wait<1>();                              // this chunk's copies are done
    __syncthreads();
    const double* sm = dsm + cur * 72 * kGram2Ld;
    const int cnt = min(kGram2Chunk, NN - ch * kGram2Chunk);
    const double* pa = sm + 3 * rg * kGram2Ld;
    const double* pb1 = sm + (24 + 6 * cg) * kGram2Ld;
    const double* pb2 = sm + (48 + 6 * cg) * kGram2Ld;
    for (int q = w; q < cnt; q += kGramThreads / 32) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int o = 4 * q + c;
        double a[3], b1[6], b2[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) a[i] = pa[i * kGram2Ld + o];
#pragma unroll
        for (int j = 0; j < 6; ++j) { b1[j] = pb1[j * kGram2Ld + o]; b2[j] = pb2[j * kGram2Ld + o]; }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 6; ++j) {
            acc1[i][j] = fma(a[i], b1[j], acc1[i][j]);
            acc2[i][j] = fma(a[i], b2[j], acc2[i][j]);
          }
      }
    }
    __syncthreads();                                 // the buffer is refilled two chunks later
    cur ^= 1;
  }
  cp_async_wait<0>();
  __syncthreads();
  double* red = dsm;                                   // [warp][576], one Gram at a time
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) red[w * 576 + (3 * rg + i) * 24 + 6 * cg + j] = g == 0 ? acc1[i][j] : acc2[i][j];
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int r = e / n, col = e % n;
      double sum = 0.0;
#pragma unroll
      for (int k = 0; k < kGramThreads / 32; ++k) sum += red[k * 576 + r * 24 + col];
      part[(size_t)blockIdx.x * 1152 + g * 576 + e] = sum;
    }
  }
}

__global__ void __launch_bounds__(256) k_gram2_reduce(int nblocks, int npair, const double* __restrict__ part,
                                                      double* G1, double* G2) {
  const int p = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= 2 * npair) return;
  const int g = p / npair, e = p % npair;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += part[(size_t)b * 1152 + g * 576 + e];
  s = warp_sum(s);
  if (lane == 0) (g == 0 ? G1 : G2)[e] = s;
}

void launch_gram2_cols(Ctx& c, bool f64, const void* A, const void* B1, const void* B2, const ColMap& cols, int n,
                       double* G1, double* G2, cudaStream_t s, double* part) {
  if (!part) part = c.gram_part;
  const int nchunks = ceil_div(c.g.NN, kGram2Chunk);
  int blocks = c.gram_blocks < nchunks ? c.gram_blocks : nchunks;
  if (blocks < 1) blocks = 1;
  const long long vs = (long long)c.g.NN * 4;
  if (f64) {
    static_assert(2 * 72 * kGram2Ld >= 8 * 576, "reduction scratch");
    cudaFuncSetAttribute(k_gram2_partial_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGram2Smem);
    k_gram2_partial_f64<<<blocks, kGramThreads, kGram2Smem, s>>>(c.g.NN, (const double*)A, (const double*)B1,
                                                                (const double*)B2, cols, n, vs, part);
  }
  else {
    k_gram2_partial<float><<<blocks, kGramThreads, 0, s>>>(c.g.NN, (const float*)A, (const float*)B1,
                                                          (const float*)B2, cols, n, vs, part);
  }
  count_launch();
  k_gram2_reduce<<<ceil_div(2 * n * n, 8), 256, 0, s>>>(blocks, n * n, part, G1, G2);
  count_launch();
}

void launch_gram_cols(Ctx& c, bool f64, const void* A, const ColMap& ma, int na, const void* B, const ColMap& mb,
                      int nb, double* G, cudaStream_t s, double* part) {
  if (!part) part = c.gram_part;
  const int nchunks = ceil_div(c.g.NN, kGramChunk);
  int blocks = c.gram_blocks < nchunks ? c.gram_blocks : nchunks;
  if (blocks < 1) blocks = 1;
  const long long vs = (long long)c.g.NN * 4;
  if (f64)
    k_gram_partial<double><<<blocks, kGramThreads, 0, s>>>(c.g.NN, (const double*)A, ma, na, (const double*)B, mb,
                                                          nb, vs, part);
  else
    k_gram_partial<float><<<blocks, kGramThreads, 0, s>>>(c.g.NN, (const float*)A, ma, na, (const float*)B, mb, nb,
                                                         vs, part);
  count_launch();
  k_gram_reduce<<<ceil_div(na * nb, 8), 256, 0, s>>>(blocks, na * nb, part, G);
  count_launch();
}

void launch_gram(Ctx& c, bool f64, const void* A, int na, const void* B, int nb, double* G, cudaStream_t s,
                 double* part) {
  ColMap id;
  for (int k = 0; k < 24; ++k) id.col[k] = k;
  launch_gram_cols(c, f64, A, id, na, B, id, nb, G, s, part);
}

// ---------------------------------------------------------------------------
// Element quadratic forms q_e = v_e^T A v_e (A = Ke or Me) for nvec vectors,
// FP64 accumulation.  ce = u_e^T Ke u_e is src/fem.py:605-615; the eigenvalue
// sensitivity's phi_e^T Ke phi_e and phi_e^T Me phi_e are src/fem.py:499-501.
// Output [nvec][NE] over the full element grid (x fastest); 0 for inactive
// elements.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_quadform(Grid g, const T* __restrict__ v, int nvec, long long vstride,
                                                  const double* __restrict__ Ae, const uint8_t* __restrict__ active,
                                                  double* out) {
  __shared__ double sA[576];
  for (int i = threadIdx.x; i < 576; i += blockDim.x) sA[i] = Ae[i];
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.NE) return;
  const int ex = e % g.nx, ey = (e / g.nx) % g.ny, ez = e / (g.nx * g.ny);
  const bool act = active[e] != 0;
  for (int r = 0; r < nvec; ++r) {
    double ue[24];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const int ox = (l == 1 || l == 2 || l == 5 || l == 6) ? 1 : 0;
      const int oy = (l == 2 || l == 3 || l == 6 || l == 7) ? 1 : 0;
      const int oz = l >= 4 ? 1 : 0;
      const int n = ((ez + oz) * g.NY + (ey + oy)) * g.NX + (ex + ox);
      const typename Vec4<T>::type x = reinterpret_cast<const typename Vec4<T>::type*>(v + r * vstride)[n];
      ue[3 * l] = double(x.x); ue[3 * l + 1] = double(x.y); ue[3 * l + 2] = double(x.z);
    }
    double q = 0.0;
#pragma unroll 4
    for (int i = 0; i < 24; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 24; ++j) t = fma(sA[i * 24 + j], ue[j], t);
      q = fma(ue[i], t, q);
    }
    out[(size_t)r * g.NE + e] = act ? q : 0.0;
  }
}

void launch_quadform(const Ctx& c, int op, bool f64, const void* v, int nvec, double* out, cudaStream_t s) {
  const double* A = op == 0 ? c.Ke64 : c.Me64;
  const long long vs = (long long)c.g.NN * 4;
  const int blocks = ceil_div(c.g.NE, 256);
  if (f64) k_quadform<double><<<blocks, 256, 0, s>>>(c.g, (const double*)v, nvec, vs, A, c.active, out);
  else k_quadform<float><<<blocks, 256, 0, s>>>(c.g, (const float*)v, nvec, vs, A, c.active, out);
  count_launch();
}

// ---------------------------------------------------------------------------
// small vector helpers
// ---------------------------------------------------------------------------
template <typename S, typename D>
__global__ void k_convert(const S* __restrict__ src, D* dst, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = D(src[i]);
}

void launch_convert(const void* src, bool src64, void* dst, bool dst64, long long n, cudaStream_t s) {
  const int blocks = int((n + 255) / 256);
  if (src64 && !dst64) k_convert<double, float><<<blocks, 256, 0, s>>>((const double*)src, (float*)dst, n);
  else if (!src64 && dst64) k_convert<float, double><<<blocks, 256, 0, s>>>((const float*)src, (double*)dst, n);
  else if (src64) k_convert<double, double><<<blocks, 256, 0, s>>>((const double*)src, (double*)dst, n);
  else k_convert<float, float><<<blocks, 256, 0, s>>>((const float*)src, (float*)dst, n);
  count_launch();
}

__global__ void k_axpy64(long long n, const double* __restrict__ x, double* y, double a) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = fma(a, x[i], y[i]);
}
__global__ void k_add_f32(long long n, const float* __restrict__ x, float* y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

void launch_add_f32(long long n, const float* x, float* y, cudaStream_t s) {
  k_add_f32<<<int((n + 255) / 256), 256, 0, s>>>(n, x, y);
  count_launch();
}

__global__ void k_abs64(long long n, const double* __restrict__ x, double* y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = fabs(x[i]);
}

void launch_abs64(long long n, const double* x, double* y, cudaStream_t s) {
  k_abs64<<<int((n + 255) / 256), 256, 0, s>>>(n, x, y);
  count_launch();
}

void launch_axpy64(long long n, const double* x, double* y, double a, cudaStream_t s) {
  k_axpy64<<<int((n + 255) / 256), 256, 0, s>>>(n, x, y, a);
  count_launch();
}

__global__ void k_add_f32_to_f64(long long n, const float* __restrict__ d, double* x) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) x[i] += double(d[i]);
}
void launch_add_f32_to_f64(long long n, const float* d, double* x, cudaStream_t s) {
  k_add_f32_to_f64<<<int((n + 255) / 256), 256, 0, s>>>(n, d, x);
  count_launch();
}

// Load every kernel of this file now (CUDA loads device functions lazily,
// at first use, and a first use in the middle of a solve stalls it).
void preload_kernels_core() {
  auto touch = [](auto f) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(f));
  };
  touch(k_factors); touch(k_diag);
  touch(k_matvec<float, 1>); touch(k_matvec<float, 2>); touch(k_matvec<float, 4>); touch(k_matvec<float, 8>);
  touch(k_matvec<double, 1>); touch(k_matvec<double, 2>); touch(k_matvec<double, 4>); touch(k_matvec<double, 8>);
  touch(k_matvec_km<double, 1>); touch(k_matvec_km<double, 2>); touch(k_matvec_km<double, 4>);
  touch(k_matvec_km<double, 8>); touch(k_matvec_km<float, 1>); touch(k_matvec_km<float, 2>);
  touch(k_matvec_km<float, 4>); touch(k_matvec_km<float, 8>);
  touch(k_pack<float>); touch(k_pack<double>); touch(k_unpack<float>); touch(k_unpack<double>);
  touch(k_gram_partial<float>); touch(k_gram_partial<double>); touch(k_gram_reduce);
  touch(k_gram2_partial<float>); touch(k_gram2_partial_f64); touch(k_gram2_reduce);
  touch(k_quadform<float>); touch(k_quadform<double>);
  touch(k_convert<double, float>); touch(k_convert<float, double>); touch(k_convert<double, double>);
  touch(k_convert<float, float>);
  touch(k_axpy64); touch(k_add_f32); touch(k_abs64); touch(k_add_f32_to_f64);
}

}  // namespace tof

// Geometric multigrid on the structured voxel grid (sm_100a), FP32.
//
// The reference preconditions its Krylov solvers with diag(K) only
// (src/fem.py:543-546, 441-443); on the SIMP-penalised arm that needs
// ~1900 PCG iterations and ~2800 LOBPCG iterations.  This module provides a
// V-cycle used as the preconditioner of an FP64 PCG (this file) and of the
// FP64 LOBPCG (tof_lobpcg.cu):
//
// * hierarchy: each axis with >= 2 elements is coarsened 2:1 (ceil), axes of
//   one element are kept (semi-coarsening), until the coarsest level has at
//   most kCoarseNodes nodes;
// * prolongation P: trilinear interpolation from coarse node I to fine node
//   2I (+-1 with weight 1/2), with fixed fine DOFs masked out;
// * coarse operators: Galerkin A_c = P^T A P, formed per coarse element as
//   K_E = sum_children P_c^T (D_c f_c Ke D_c) P_c using the Kronecker
//   structure P_c = W_c (x) I3 (8 x 8 scalar weights), so no matrix is
//   assembled; levels >= 1 store one dense 24x24 FP32 matrix per element;
// * smoother: Chebyshev polynomial in D^-1 A of degree nu on the interval
//   [lambda / 30, 1.3 lambda] (lambda a power-iteration estimate of
//   lambda_max(D^-1 A) per level), as the same three-term recurrence before
//   and after the coarse correction (a symmetric V-cycle, hence an SPD
//   preconditioner for CG); damped Jacobi with the same number of sweeps
//   when TOF_MG_SMOOTHER=jacobi.  The fine-level sweeps use the TMA-tiled
//   matrix-free stencil;
// * coarsest level: dense FP64 inverse, built by one CTA (Cholesky, then
//   L^-T L^-1), applied as a dense matvec.
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include <stdlib.h>

#include "tof_internal.h"
#include "tof_stencil.cuh"

namespace tof {

constexpr int kCoarseNodes = 160;
constexpr int kMaxLevels = 10;
// Jacobi smoothing weight omega = kOmegaScale / lambda_max(D^-1 A).  4/3 is
// the classical high-frequency-optimal choice; a 10-step power iteration
// underestimates lambda_max by ~15 % on these operators, which keeps
// omega * lambda_max near 1.6, inside the stable range (0, 2).
constexpr float kOmegaScale = 1.3333f;
constexpr int kPowerIters = 10;
// Chebyshev smoothing interval [lambda / kChebRatio, kChebUpper lambda]: the
// upper end must cover the power iteration's underestimate of lambda_max
// (2-9 % on the SIMP arm levels), since above the interval the polynomial
// amplifies the error and the V-cycle stops being positive definite; the
// ratio and margin were chosen on the SIMP arm designs (a CPU model of this
// V-cycle: 14 % fewer MG-PCG iterations than damped Jacobi at equal sweeps).
constexpr float kChebUpper = 1.3f;
constexpr float kChebRatio = 30.f;
constexpr int kMaxNu = 4;
constexpr int kCoefStride = 3 * kMaxNu;   // (sx, sp, sr) per sweep

struct MGLevel {
  int nx, ny, nz, NX, NY, NZ, NN, NE;
  int fx, fy, fz;          // coarsening factor from the finer level (1 or 2)
  float* Ae = nullptr;     // [NE][576] Galerkin element matrices (levels >= 1)
  float* St = nullptr;     // [243][NN] assembled node stencils (levels 1 .. nlev-2)
  float* dinv = nullptr;   // node4
  uint8_t* fix = nullptr;  // node bits
};

// V-cycle vectors of one level (node4 x maxR): right-hand side, correction
// and its ping-pong partner, residual
struct MGBuf {
  float *r = nullptr, *e = nullptr, *e2 = nullptr, *t = nullptr;
};
constexpr int kLanes = 2;      // lane 0: static solves, lane 1: modal solves

struct MG {
  int nlev = 0;
  MGLevel L[kMaxLevels];
  MGBuf buf[kLanes][kMaxLevels];
  int nc = 0;                 // coarsest DOFs
  double *A = nullptr, *Y = nullptr, *Ainv = nullptr;
  int maxR = 0;
  // per level: lambda_l, a power-iteration estimate of lambda_max(D^-1 A_l),
  // the first sweep's weight omega_l, and for sweep k = 0 .. nu-1 the
  // coefficients (sx, sp, sr) of x_{k+1} = sx x_k + sp x_{k-1} + sr D^-1 r_k
  // at coef[l * kCoefStride + 3 k] (device)
  float* omega = nullptr;
  float* lam = nullptr;
  float* coef = nullptr;
  int nu = 2;
  int smoother = 0;           // 0 Chebyshev, 1 damped Jacobi
  bool dirty = true;
  // outer FP64 PCG
  double *x = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *p[2] = {nullptr, nullptr};
  double* S = nullptr;        // per-rhs scalars [8][8]
  int* flags = nullptr;       // per-rhs frozen / status
  unsigned* cnt = nullptr;    // last-block counters [8]
  double* part = nullptr;     // partial sums
  int part_blocks = 0;
  int* info = nullptr;
  // a single V-cycle per lane and R, replayed by every caller
  cudaGraphExec_t vexec[kLanes][4] = {};
  size_t vnodes[kLanes][4] = {};
  bool vgraph_failed = false;
};
// MG-PCG iterations between host checks of the convergence flags (even:
// the p double-buffer parity returns to 0), launched kernel by kernel (the
// V-cycle inside each is a graph replay).  This paces the static solve: in
// the SIMP step it runs beside the modal solve, whose chain of short kernels
// is the critical path, and a static stream that never pauses slows that
// chain down.  Measured on the 2 mm arm, per design iteration in the timed
// window: groups of 8 / 4 / 2 iterations replayed as graphs 78 / 73 / 63 ms,
// launched kernel by kernel 61 ms (4) and 59 ms (2); a device-side loop
// without host checks was slower still.  A standalone 4-vector solve costs
// ~5 % more than with graph groups (30.4 vs 28.8 ms).
constexpr int kCheckIters = 2;

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void node_ijk(int n, int NX, int NY, int& i, int& j, int& k) {
  i = n % NX; j = (n / NX) % NY; k = n / (NX * NY);
}


// Transfer weights along one axis.  Restriction: fine offsets -1, 0, +1
// around 2I (weights 1/2, 1, 1/2) when the axis is coarsened, else only the
// offset 0; a fine index outside the grid gets weight 0 and a clamped index.
__device__ __forceinline__ void restrict_axis(int f, int I, int Nf, int* idx, float* w) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int o = d - 1;
    const int i = f * I + o;
    const bool ok = (f == 2 || o == 0) && i >= 0 && i < Nf;
    idx[d] = min(max(i, 0), Nf - 1);
    w[d] = ok ? (o == 0 ? 1.f : 0.5f) : 0.f;
  }
}
// Prolongation: a fine node on a coarse node takes it with weight 1, a node
// between two coarse nodes takes both with weight 1/2.
__device__ __forceinline__ void prolong_axis(int f, int i, int* idx, float* w) {
  if (f == 1) { idx[0] = idx[1] = i; w[0] = 1.f; w[1] = 0.f; }
  else if ((i & 1) == 0) { idx[0] = idx[1] = i / 2; w[0] = 1.f; w[1] = 0.f; }
  else { idx[0] = (i - 1) / 2; idx[1] = (i + 1) / 2; w[0] = w[1] = 0.5f; }
}

// (P ec)_n for fine node n, vector r; src = ec of vector r.  8 unconditional loads.
__device__ __forceinline__ float4 prolong_node(int fx, int fy, int fz, int NXf, int NYf, int NXc, int NYc, int n,
                                               const float* __restrict__ src) {
  int i, j, k;
  node_ijk(n, NXf, NYf, i, j, k);
  int ix[2], iy[2], iz[2];
  float wx[2], wy[2], wz[2];
  prolong_axis(fx, i, ix, wx);
  prolong_axis(fy, j, iy, wy);
  prolong_axis(fz, k, iz, wz);
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int a = t & 1, b = (t >> 1) & 1, c = t >> 2;
    const float w = wx[a] * wy[b] * wz[c];
    const int m = (iz[c] * NYc + iy[b]) * NXc + ix[a];
    const float4 v = __ldg(reinterpret_cast<const float4*>(src) + m);
    a0 = fmaf(w, v.x, a0); a1 = fmaf(w, v.y, a1); a2 = fmaf(w, v.z, a2);
  }
  return make_float4(a0, a1, a2, 0.f);
}


// ---------------------------------------------------------------------------
// Galerkin coarse element matrices
// ---------------------------------------------------------------------------
struct GalerkinArgs {
  // fine level
  int nx, ny, nz, NX, NY;
  const float* Ae_f;       // fine element matrices (levels >= 1) or null
  const double* fK;        // level-0 factors (when Ae_f is null)
  const double* Ke;        // level-0 dense Ke
  const uint8_t* fix0;     // level-0 node fixed bits
  // coarse level
  int cx, cy, cz;
  int fx, fy, fz;
  float* Ae_c;
};

__global__ void __launch_bounds__(128) k_mg_galerkin(GalerkinArgs a) {
  __shared__ double Kc[576], T[576], W[64];
  __shared__ double Dm[24];
  __shared__ double fscale;
  const int E = blockIdx.x;
  const int ex = E % a.cx, ey = (E / a.cx) % a.cy, ez = E / (a.cx * a.cy);
  double acc[5] = {0, 0, 0, 0, 0};
  for (int cd = 0; cd < a.fz; ++cd)
    for (int cb = 0; cb < a.fy; ++cb)
      for (int ca = 0; ca < a.fx; ++ca) {
        const int fxe = a.fx * ex + ca, fye = a.fy * ey + cb, fze = a.fz * ez + cd;
        if (fxe >= a.nx || fye >= a.ny || fze >= a.nz) continue;   // phantom child
        const int ce = (fze * a.ny + fye) * a.nx + fxe;
        if (threadIdx.x == 0) fscale = a.Ae_f ? 1.0 : a.fK[ce];
        if (threadIdx.x < 24) {
          double d = 1.0;
          if (!a.Ae_f) {
            const int l = threadIdx.x / 3, q = threadIdx.x % 3;
            const int ox = (l == 1 || l == 2 || l == 5 || l == 6), oy = (l == 2 || l == 3 || l == 6 || l == 7),
                      oz = l >= 4;
            const int n = ((fze + oz) * a.NY + (fye + oy)) * a.NX + (fxe + ox);
            d = ((a.fix0[n] >> q) & 1) ? 0.0 : 1.0;
          }
          Dm[threadIdx.x] = d;
        }
        if (threadIdx.x < 64) {
          // weight of coarse corner m for child local node l
          const int l = threadIdx.x / 8, m = threadIdx.x % 8;
          const int ox = (l == 1 || l == 2 || l == 5 || l == 6), oy = (l == 2 || l == 3 || l == 6 || l == 7),
                    oz = l >= 4;
          const int mx = (m == 1 || m == 2 || m == 5 || m == 6), my = (m == 2 || m == 3 || m == 6 || m == 7),
                    mz = m >= 4;
          const double px = double(ca + ox) / a.fx, py = double(cb + oy) / a.fy, pz = double(cd + oz) / a.fz;
          W[threadIdx.x] = (mx ? px : 1.0 - px) * (my ? py : 1.0 - py) * (mz ? pz : 1.0 - pz);
        }
        __syncthreads();
        if (fscale == 0.0) { __syncthreads(); continue; }
        for (int i = threadIdx.x; i < 576; i += blockDim.x) {
          const int r = i / 24, c = i % 24;
          Kc[i] = a.Ae_f ? double(a.Ae_f[(size_t)ce * 576 + i]) : fscale * a.Ke[i] * Dm[r] * Dm[c];
        }
        __syncthreads();
        // T[i][3m+q] = sum_l Kc[i][3l+q] W[l][m]
        for (int i = threadIdx.x; i < 576; i += blockDim.x) {
          const int r = i / 24, col = i % 24, m = col / 3, q = col % 3;
          double s = 0.0;
#pragma unroll
          for (int l = 0; l < 8; ++l) s = fma(Kc[r * 24 + 3 * l + q], W[l * 8 + m], s);
          T[i] = s;
        }
        __syncthreads();
        // acc[3m+q][col] += sum_l W[l][m] T[3l+q][col]
        int slot = 0;
        for (int i = threadIdx.x; i < 576; i += blockDim.x, ++slot) {
          const int row = i / 24, col = i % 24, m = row / 3, q = row % 3;
          double s = 0.0;
#pragma unroll
          for (int l = 0; l < 8; ++l) s = fma(W[l * 8 + m], T[(3 * l + q) * 24 + col], s);
          acc[slot] += s;
        }
        __syncthreads();
      }
  int slot = 0;
  for (int i = threadIdx.x; i < 576; i += blockDim.x, ++slot) a.Ae_c[(size_t)E * 576 + i] = float(acc[slot]);
}

// diag / inverse diag / fixed bits of a level >= 1 from its element matrices
__global__ void k_mg_diag(int nx, int ny, int nz, const float* __restrict__ Ae, float* dinv, uint8_t* fix) {
  const int NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= NX * NY * NZ) return;
  int i, j, k;
  node_ijk(n, NX, NY, i, j, k);
  double d[3] = {0, 0, 0};
  for (int c = -1; c <= 0; ++c)
    for (int b = -1; b <= 0; ++b)
      for (int a = -1; a <= 0; ++a) {
        const int ex = i + a, ey = j + b, ez = k + c;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
        const int E = (ez * ny + ey) * nx + ex, ln = local_node(-a, -b, -c);
        for (int q = 0; q < 3; ++q) d[q] += Ae[(size_t)E * 576 + (3 * ln + q) * 24 + 3 * ln + q];
      }
  uint8_t f = 0;
  float4 o;
  float* op = &o.x;
  for (int q = 0; q < 3; ++q) {
    const bool fz = !(d[q] > 0.0);
    if (fz) f |= uint8_t(1u << q);
    op[q] = fz ? 0.f : float(1.0 / d[q]);
  }
  o.w = 0.f;
  reinterpret_cast<float4*>(dinv)[n] = o;
  fix[n] = f;
}

// Assembled node stencil of a coarse level: for node n and neighbour
// nb = (dz+1)*9 + (dy+1)*3 + (dx+1), the 3x3 block coupling n to
// n + (dx, dy, dz) is the sum over the (up to 4) elements holding both nodes
// of Ae[E][3 ln + q][3 lm + p].  Stored structure-of-arrays,
// St[(nb * 9 + q * 3 + p) * NN + n], so that a warp of consecutive nodes reads
// each entry coalesced.  One thread per (node, neighbour).
__global__ void k_mg_stencil(int nx, int ny, int nz, const float* __restrict__ Ae, float* St) {
  const int NX = nx + 1, NY = ny + 1, NN = NX * NY * (nz + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 27LL * NN) return;
  const int n = int(t % NN), nb = int(t / NN);
  const int dx = nb % 3 - 1, dy = (nb / 3) % 3 - 1, dz = nb / 9 - 1;
  int i, j, k;
  node_ijk(n, NX, NY, i, j, k);
  double s[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) s[e] = 0.0;
  for (int c = -1; c <= 0; ++c)
    for (int b = -1; b <= 0; ++b)
      for (int a = -1; a <= 0; ++a) {
        const int ex = i + a, ey = j + b, ez = k + c;
        if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
        const int mx = dx - a, my = dy - b, mz = dz - c;   // neighbour's offset inside the element
        if (mx < 0 || mx > 1 || my < 0 || my > 1 || mz < 0 || mz > 1) continue;
        const int E = (ez * ny + ey) * nx + ex, ln = local_node(-a, -b, -c), lm = local_node(mx, my, mz);
        const float* Kr = Ae + (size_t)E * 576 + (3 * ln) * 24 + 3 * lm;
#pragma unroll
        for (int q = 0; q < 3; ++q)
#pragma unroll
          for (int p = 0; p < 3; ++p) s[q * 3 + p] += double(Kr[q * 24 + p]);
      }
#pragma unroll
  for (int e = 0; e < 9; ++e) St[(size_t)(nb * 9 + e) * NN + n] = float(s[e]);
}

constexpr int kCholB = 16;   // Cholesky panel width
static size_t coarse_setup_smem(int n) { return sizeof(double) * (kCholB + 1) * (kCholB + n); }

// Coarsest level: dense assembly (row per thread) and blocked Cholesky in one
// CTA; the inverse is formed by k_mg_coarse_inverse.  Level 0 (Ae == null)
// assembles from factors and Ke with the fixed mask.
__global__ void __launch_bounds__(1024) k_mg_coarse_setup(int nx, int ny, int nz, const float* __restrict__ Ae,
                                                         const double* __restrict__ fK, const double* __restrict__ Ke,
                                                         const uint8_t* __restrict__ fix, double* A, double* Y,
                                                         int* info) {
  const int NX = nx + 1, NY = ny + 1, NZ = nz + 1, NN = NX * NY * NZ, n = 3 * NN;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) A[i] = 0.0;
  __syncthreads();
  for (int row = threadIdx.x; row < n; row += blockDim.x) {
    const int N = row / 3, q = row % 3;
    int i, j, k;
    node_ijk(N, NX, NY, i, j, k);
    const bool fixed_row = (fix[N] >> q) & 1;
    for (int c = -1; c <= 0; ++c)
      for (int b = -1; b <= 0; ++b)
        for (int a = -1; a <= 0; ++a) {
          const int ex = i + a, ey = j + b, ez = k + c;
          if (ex < 0 || ey < 0 || ez < 0 || ex >= nx || ey >= ny || ez >= nz) continue;
          const int E = (ez * ny + ey) * nx + ex, ln = local_node(-a, -b, -c);
          for (int lm = 0; lm < 8; ++lm) {
            const int mx = (lm == 1 || lm == 2 || lm == 5 || lm == 6), my = (lm == 2 || lm == 3 || lm == 6 || lm == 7),
                      mz = lm >= 4;
            const int M = ((ez + mz) * NY + (ey + my)) * NX + (ex + mx);
            for (int q2 = 0; q2 < 3; ++q2) {
              const int col = 3 * M + q2;
              const bool fixed_col = (fix[M] >> q2) & 1;
              double v;
              if (Ae) v = Ae[(size_t)E * 576 + (3 * ln + q) * 24 + 3 * lm + q2];
              else v = fK[E] * Ke[(3 * ln + q) * 24 + 3 * lm + q2];
              if (!fixed_row && !fixed_col) A[(size_t)row * n + col] += v;
            }
          }
        }
    if (fixed_row) A[(size_t)row * n + row] = 1.0;
  }
  __syncthreads();
  // Blocked right-looking Cholesky A = L L^T (lower triangle, in place),
  // panels of kCholB columns: (1) one warp factors the diagonal block in
  // shared memory, (2) each row below solves against it (thread per row) and
  // the panel is kept in shared memory, (3) the trailing lower triangle is
  // updated once per panel (warp per row, lanes over columns), so A makes
  // n / kCholB passes through L2 instead of n.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  extern __shared__ double sh[];
  constexpr int LD = kCholB + 1;
  double* Dg = sh;                     // [kCholB][LD] diagonal block
  double* Pn = sh + kCholB * LD;       // [rows below][LD] panel
  __shared__ int s_bad;
  __shared__ double Rd[kCholB];
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  for (int kb = 0; kb < n; kb += kCholB) {
    const int w = min(kCholB, n - kb);
    for (int e = threadIdx.x; e < w * w; e += blockDim.x)
      Dg[(e / w) * LD + e % w] = A[(size_t)(kb + e / w) * n + kb + e % w];
    __syncthreads();
    if (warp == 0) {
      for (int t = 0; t < w; ++t) {
        if (lane == 0) {
          double d = Dg[t * LD + t];
          if (!(d > 0.0)) { s_bad = kb + t + 1; d = 1.0; }
          Dg[t * LD + t] = sqrt(d);
        }
        __syncwarp();
        const double ip = 1.0 / Dg[t * LD + t];
        if (lane > t && lane < w) Dg[lane * LD + t] *= ip;
        __syncwarp();
        if (lane > t && lane < w)
          for (int c2 = t + 1; c2 <= lane; ++c2) Dg[lane * LD + c2] -= Dg[lane * LD + t] * Dg[c2 * LD + t];
        __syncwarp();
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
      const int r0 = e / w, c0 = e % w;
      if (c0 <= r0) {
        A[(size_t)(kb + r0) * n + kb + c0] = Dg[r0 * LD + c0];
        A[(size_t)(kb + c0) * n + kb + r0] = Dg[r0 * LD + c0];
      }
      if (c0 == r0) {
        const double rd = 1.0 / Dg[r0 * LD + r0];
        Y[kb + r0] = rd;
        Rd[r0] = rd;
      }
    }
    __syncthreads();
    const int base = kb + w;
    for (int i = base + threadIdx.x; i < n; i += blockDim.x) {
      double x[kCholB];
#pragma unroll
      for (int t = 0; t < kCholB; ++t) x[t] = t < w ? A[(size_t)i * n + kb + t] : 0.0;
#pragma unroll
      for (int t = 0; t < kCholB; ++t) {
        if (t < w) {
#pragma unroll
          for (int u = 0; u < t; ++u) x[t] = fma(-x[u], Dg[t * LD + u], x[t]);
          x[t] *= Rd[t];                          // (the pivots' reciprocals, formed once per panel)
          A[(size_t)i * n + kb + t] = x[t];
          A[(size_t)(kb + t) * n + i] = x[t];      // L^T in the upper triangle
          Pn[(i - base) * LD + t] = x[t];
        }
      }
    }
    __syncthreads();
    for (int i = base + warp; i < n; i += nwarps) {
      double pi[kCholB];
#pragma unroll
      for (int t = 0; t < kCholB; ++t) pi[t] = t < w ? Pn[(i - base) * LD + t] : 0.0;
      for (int j = base + lane; j <= i; j += 32) {
        const double* pj = Pn + (j - base) * LD;
        double sum = 0.0;
#pragma unroll
        for (int t = 0; t < kCholB; ++t) sum = fma(pi[t], t < w ? pj[t] : 0.0, sum);
        A[(size_t)i * n + j] -= sum;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) info[0] = s_bad;
}

// Coarsest inverse from the Cholesky factor: one warp per column j of
// A^-1 = L^-T L^-1.  The column lives in registers (lane l holds entries
// l + 32 m); the forward solve L y = e_j and the back solve L^T x = y run in
// axpy form, so each step is one shuffle broadcast plus coalesced loads of a
// row of L^T (forward) or of L (backward) -- no long dependent dot products.
// LLt: L in the lower and L^T in the upper triangle; idg[k] = 1 / L[k][k].
// The result is written as row j (A^-1 is symmetric); rows and columns of
// fixed DOFs are zero.
constexpr int kInvSlots = (3 * kCoarseNodes + 31) / 32;
__global__ void __launch_bounds__(256) k_mg_coarse_inverse(int n, const double* __restrict__ LLt,
                                                           const double* __restrict__ idg,
                                                           const uint8_t* __restrict__ fix, double* Ainv) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= n) return;
  double y[kInvSlots];
#pragma unroll
  for (int m = 0; m < kInvSlots; ++m) y[m] = (lane + 32 * m == j) ? 1.0 : 0.0;
  // Each step's row of L^T (forward) or L (backward) does not depend on y:
  // it is loaded one step ahead (into cur / nxt), so the L2 latency overlaps
  // the previous step's shuffle and updates instead of adding to every step.
  // The updates are selects, not branches, which keeps y in registers (with
  // branches the compiler placed it in local memory).
  double cur[kInvSlots], nxt[kInvSlots];
#pragma unroll
  for (int m = 0; m < kInvSlots; ++m) {
    const int i = lane + 32 * m;
    cur[m] = i < n ? LLt[(size_t)j * n + i] : 0.0;
    nxt[m] = 0.0;
  }
  // forward: for k = j .. n-1: y_k /= L_kk; y_i -= L_ik y_k (i > k)
  for (int k = j; k < n; ++k) {
    const int kn = k + 1 < n ? k + 1 : k;
#pragma unroll
    for (int m = 0; m < kInvSlots; ++m) {
      const int i = lane + 32 * m;
      nxt[m] = i < n ? LLt[(size_t)kn * n + i] : 0.0;
    }
    const int km = k >> 5;
    double own = 0.0;
#pragma unroll
    for (int m = 0; m < kInvSlots; ++m) own = m == km ? y[m] : own;
    const double yk = __shfl_sync(0xffffffffu, own, k & 31) * idg[k];
#pragma unroll
    for (int m = 0; m < kInvSlots; ++m) {
      const int i = lane + 32 * m;
      const double upd = fma(-((i > k && i < n) ? cur[m] : 0.0), yk, y[m]);
      y[m] = i == k ? yk : upd;
      cur[m] = nxt[m];
    }
  }
  // backward: for k = n-1 .. 0: x_k = y_k / L_kk; y_i -= L_ki x_k (i < k)
#pragma unroll
  for (int m = 0; m < kInvSlots; ++m) {
    const int i = lane + 32 * m;
    cur[m] = i < n ? LLt[(size_t)(n - 1) * n + i] : 0.0;
  }
  for (int k = n - 1; k >= 0; --k) {
    const int kn = k > 0 ? k - 1 : k;
#pragma unroll
    for (int m = 0; m < kInvSlots; ++m) {
      const int i = lane + 32 * m;
      nxt[m] = i < n ? LLt[(size_t)kn * n + i] : 0.0;
    }
    const int km = k >> 5;
    double own = 0.0;
#pragma unroll
    for (int m = 0; m < kInvSlots; ++m) own = m == km ? y[m] : own;
    const double xk = __shfl_sync(0xffffffffu, own, k & 31) * idg[k];
#pragma unroll
    for (int m = 0; m < kInvSlots; ++m) {
      const int i = lane + 32 * m;
      const double upd = fma(-(i < k ? cur[m] : 0.0), xk, y[m]);
      y[m] = i == k ? xk : upd;
      cur[m] = nxt[m];
    }
  }
  const bool fj = (fix[j / 3] >> (j % 3)) & 1;
#pragma unroll
  for (int m = 0; m < kInvSlots; ++m) {
    const int i = lane + 32 * m;
    if (i < n) {
      const bool fi = (fix[i / 3] >> (i % 3)) & 1;
      Ainv[(size_t)j * n + i] = (fi || fj) ? 0.0 : y[m];
    }
  }
}

// ---------------------------------------------------------------------------
// V-cycle kernels
// ---------------------------------------------------------------------------
struct LevelView {
  int nx, ny, nz, NX, NY, NZ, NN;
  const float* St;
  const float* dinv;
  const uint8_t* fix;
};

// Coarse-level operator from the assembled stencil, one thread per
// (node, output component q, right-hand side r): a CTA is 32 consecutive
// nodes x (3 R) warps, so each warp reads the stencil rows of its q
// coalesced and the R warps sharing them hit L1.
// mode 0: y = b - A x;  mode 1: y = sx x + sr D^-1 (b - A x);  mode 3: as 1
// plus sp y_prev (y's previous content);  mode 2: y = D^-1 A x; (sx, sp, sr)
// a device triple (fixed DOFs of modes 0, 1, 3 are set to 0; the padding
// component to 0).
__global__ void __launch_bounds__(768) k_mgs_op(LevelView L, int R, const float* __restrict__ x,
                                                const float* __restrict__ b, float* y,
                                                const float* __restrict__ coef, int mode) {
  const int n = blockIdx.x * 32 + threadIdx.x;
  const int q = threadIdx.y % 3, r = threadIdx.y / 3;
  if (n >= L.NN || r >= R) return;
  const long long vs = (long long)L.NN * 4;
  int i, j, k;
  node_ijk(n, L.NX, L.NY, i, j, k);
  const float* xr = x + r * vs;
  const float* S = L.St + (size_t)q * 3 * L.NN + n;
  int xo[3], yo[3], zo[3];     // clamped neighbour coordinates (their stencil blocks are zero)
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    xo[d] = min(max(i + d - 1, 0), L.NX - 1);
    yo[d] = min(max(j + d - 1, 0), L.NY - 1) * L.NX;
    zo[d] = min(max(k + d - 1, 0), L.NZ - 1) * L.NX * L.NY;
  }
  float acc = 0.f;
#pragma unroll
  for (int nb = 0; nb < 27; ++nb) {
    const int m = zo[nb / 9] + yo[(nb / 3) % 3] + xo[nb % 3];
    const float4 xv = __ldg(reinterpret_cast<const float4*>(xr) + m);
    const float* Sq = S + (size_t)nb * 9 * L.NN;
    acc = fmaf(__ldg(Sq), xv.x, acc);
    acc = fmaf(__ldg(Sq + L.NN), xv.y, acc);
    acc = fmaf(__ldg(Sq + 2 * (size_t)L.NN), xv.z, acc);
  }
  const size_t o = r * vs + 4 * (size_t)n;
  const float di = L.dinv[4 * (size_t)n + q];
  float out;
  if (mode == 2) {
    out = di * acc;
  } else {
    out = b[o + q] - acc;
    if (mode != 0) {
      out = fmaf(__ldg(coef + 2) * di, out, __ldg(coef) * x[o + q]);
      if (mode == 3) out = fmaf(__ldg(coef + 1), y[o + q], out);
    }
    if ((L.fix[n] >> q) & 1) out = 0.f;
  }
  y[o + q] = out;
  if (q == 0) y[o + 3] = 0.f;
}

// The same operator with each (node, q, r) sum split over the three
// z-planes of the 27-neighbour stencil: three threads of 9 neighbours each
// (36 loads instead of 108), combined through shared memory in a fixed
// order.  Three times the threads with a third of the dependent-load chain
// each: these levels are small (a few thousand nodes) and latency-bound.
// CTA: 32 consecutive nodes x kMgsRb right-hand sides x 3 components x 3
// planes; grid.y covers the right-hand sides.
constexpr int kMgsRb = 1;
__global__ void __launch_bounds__(32 * 9 * kMgsRb) k_mgs_op_split(LevelView L, int R, const float* __restrict__ x,
                                                                  const float* __restrict__ b, float* y,
                                                                  const float* __restrict__ coef, int mode) {
  __shared__ float part[3 * kMgsRb][3][32];
  const int tx = threadIdx.x;
  const int pz = threadIdx.y % 3, qr = threadIdx.y / 3;
  const int q = qr % 3, r = blockIdx.y * kMgsRb + qr / 3;
  const int n = blockIdx.x * 32 + tx;
  const bool live = n < L.NN && r < R;
  const long long vs = (long long)L.NN * 4;
  float acc = 0.f;
  if (live) {
    int i, j, k;
    node_ijk(n, L.NX, L.NY, i, j, k);
    const float* xr = x + r * vs;
    const float* S = L.St + (size_t)q * 3 * L.NN + n;
    int xo[3], yo[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      xo[d] = min(max(i + d - 1, 0), L.NX - 1);
      yo[d] = min(max(j + d - 1, 0), L.NY - 1) * L.NX;
    }
    const int zo = min(max(k + pz - 1, 0), L.NZ - 1) * L.NX * L.NY;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int m = zo + yo[t / 3] + xo[t % 3];
      const float4 xv = __ldg(reinterpret_cast<const float4*>(xr) + m);
      const float* Sq = S + (size_t)(pz * 9 + t) * 9 * L.NN;
      acc = fmaf(__ldg(Sq), xv.x, acc);
      acc = fmaf(__ldg(Sq + L.NN), xv.y, acc);
      acc = fmaf(__ldg(Sq + 2 * (size_t)L.NN), xv.z, acc);
    }
  }
  part[qr][pz][tx] = acc;
  __syncthreads();
  if (!live || pz != 0) return;
  acc = (part[qr][0][tx] + part[qr][1][tx]) + part[qr][2][tx];
  const size_t o = r * vs + 4 * (size_t)n;
  const float di = L.dinv[4 * (size_t)n + q];
  float out;
  if (mode == 2) {
    out = di * acc;
  } else {
    out = b[o + q] - acc;
    if (mode != 0) {
      out = fmaf(__ldg(coef + 2) * di, out, __ldg(coef) * x[o + q]);
      if (mode == 3) out = fmaf(__ldg(coef + 1), y[o + q], out);
    }
    if ((L.fix[n] >> q) & 1) out = 0.f;
  }
  y[o + q] = out;
  if (q == 0) y[o + 3] = 0.f;
}

// The split form wins on these small levels (measured on the 2 mm arm, one
// right-hand side per CTA: 3 136 nodes x 4 vectors 7.1 -> 4.4 us, 3 136 x 8
// 7.7 -> 7.1 us, 580 x 4 6.8 -> 3.8 us; with two right-hand sides per CTA
// the 3 136 x 8 case was slower split, 8.1 us).
constexpr long long kMgsSplitBelow = 32768;   // nodes x right-hand sides
static void launch_mgs_op(const LevelView& L, int R, const float* x, const float* b, float* y, const float* coef,
                          int mode, cudaStream_t s) {
  if ((long long)L.NN * R <= kMgsSplitBelow)
    k_mgs_op_split<<<dim3(ceil_div(L.NN, 32), ceil_div(R, kMgsRb)), dim3(32, 9 * kMgsRb), 0, s>>>(L, R, x, b, y, coef,
                                                                                                 mode);
  else
    k_mgs_op<<<ceil_div(L.NN, 32), dim3(32, 3 * R), 0, s>>>(L, R, x, b, y, coef, mode);
  count_launch();
}

// e = omega D^-1 r  (first pre-smoothing sweep from e = 0), any level
__global__ void k_mg_jacobi0(int NN, int R, const float* __restrict__ dinv, const float* __restrict__ r, float* e,
                             const float* __restrict__ omega_p) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)NN * R) return;
  const int n = int(idx % NN);
  const float omega = __ldg(omega_p);
  const float4 d = reinterpret_cast<const float4*>(dinv)[n];
  const float4 v = reinterpret_cast<const float4*>(r)[idx];
  reinterpret_cast<float4*>(e)[idx] = make_float4(omega * d.x * v.x, omega * d.y * v.y, omega * d.z * v.z, 0.f);
}

// power iteration for lambda_max(D^-1 A): start vector, D^-1 scaling, estimate
__global__ void k_mg_power_init(int NN, const uint8_t* __restrict__ fix, float* x) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= NN) return;
  float v[3];
  for (int q = 0; q < 3; ++q) {
    unsigned h = (unsigned)(n * 3 + q) * 2654435761u;   // multiplicative hash
    h ^= h >> 15; h *= 2246822519u; h ^= h >> 13;
    v[q] = ((fix[n] >> q) & 1) ? 0.f : float(h & 0xffff) / 32768.f - 1.f;
  }
  reinterpret_cast<float4*>(x)[n] = make_float4(v[0], v[1], v[2], 0.f);
}

__global__ void k_mg_scale_dinv(int NN, const float* __restrict__ dinv, float* y) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= NN) return;
  const float4 d = reinterpret_cast<const float4*>(dinv)[n];
  float4 v = reinterpret_cast<float4*>(y)[n];
  v.x *= d.x; v.y *= d.y; v.z *= d.z;
  reinterpret_cast<float4*>(y)[n] = v;
}

// lambda = ||x_k|| / ||x_{k-1}|| and the smoothing coefficients of the
// level (one CTA).  Chebyshev on [a, b] = [b / kChebRatio, kChebUpper
// lambda] (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed.,
// Alg. 12.1, with D^-1 as the preconditioner): theta = (a + b) / 2,
// delta = (b - a) / 2, sigma = theta / delta, rho_0 = 1 / sigma;
// x_1 = x_0 + D^-1 r_0 / theta; for k >= 1, rho_k = 1 / (2 sigma - rho_{k-1})
// and x_{k+1} = x_k + rho_k rho_{k-1} (x_k - x_{k-1}) + (2 rho_k / delta) D^-1 r_k.
// Damped Jacobi: every sweep x_{k+1} = x_k + omega D^-1 r_k, omega = 1.3333 / lambda.
__global__ void __launch_bounds__(1024) k_mg_lambda(int NN, const float* __restrict__ xp, const float* __restrict__ xl,
                                                    float* lam, float* omega, float* coef, int nu, int jacobi) {
  __shared__ double red[2 * 32];
  double v[2] = {0.0, 0.0};
  for (int n = threadIdx.x; n < NN; n += blockDim.x) {
    const float4 a = reinterpret_cast<const float4*>(xp)[n];
    const float4 b = reinterpret_cast<const float4*>(xl)[n];
    v[0] += double(a.x) * a.x + double(a.y) * a.y + double(a.z) * a.z;
    v[1] += double(b.x) * b.x + double(b.y) * b.y + double(b.z) * b.z;
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    const double l = fmax((v[0] > 0.0 && v[1] > 0.0) ? sqrt(v[1] / v[0]) : 4.0, 1e-3);
    *lam = float(l);
    if (jacobi) {
      const double w = kOmegaScale / l;
      *omega = float(w);
      for (int k = 0; k < nu; ++k) { coef[3 * k] = 1.f; coef[3 * k + 1] = 0.f; coef[3 * k + 2] = float(w); }
    } else {
      const double bu = kChebUpper * l, al = bu / kChebRatio;
      const double th = 0.5 * (bu + al), de = 0.5 * (bu - al), sg = th / de;
      double rho = 1.0 / sg;
      *omega = float(1.0 / th);
      coef[0] = 1.f; coef[1] = 0.f; coef[2] = float(1.0 / th);
      for (int k = 1; k < nu; ++k) {
        const double rn = 1.0 / (2.0 * sg - rho);
        coef[3 * k] = float(1.0 + rn * rho);
        coef[3 * k + 1] = float(-rn * rho);
        coef[3 * k + 2] = float(2.0 * rn / de);
        rho = rn;
      }
    }
  }
}

struct Transfer {
  int NXf, NYf, NZf;   // fine nodes
  int NXc, NYc, NZc;   // coarse nodes
  int fx, fy, fz;
};

// r_c = P^T t_f (masked by the coarse fixed bits).  The 27 fine-node loads
// of each (coarse node, right-hand side) are split over the three fine
// z-offsets: three threads of 9 loads, combined through shared memory in a
// fixed order (the levels are small and the loads latency-bound; measured
// on the 2 mm arm: V-cycle 100.7 -> 96.5 us with 4 vectors against one
// thread of 27 loads).  CTA: 32 coarse nodes x 3 offsets of one
// right-hand side (grid.y), so a small coarse level still spreads over many
// SMs.
__global__ void __launch_bounds__(32 * 3) k_mg_restrict_split(Transfer T, int R, const float* __restrict__ tf,
                                                             const uint8_t* __restrict__ fixc, float* rc) {
  __shared__ float part[3][3][32];
  const int NNc = T.NXc * T.NYc * T.NZc;
  const int tx = threadIdx.x, c = threadIdx.y, r = blockIdx.y;
  const int N = blockIdx.x * 32 + tx;
  const bool live = N < NNc;
  const long long vsf = (long long)T.NXf * T.NYf * T.NZf * 4, vsc = (long long)NNc * 4;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  if (live) {
    int I, J, K;
    node_ijk(N, T.NXc, T.NYc, I, J, K);
    int ix[3], iy[3], iz[3];
    float wx[3], wy[3], wz[3];
    restrict_axis(T.fx, I, T.NXf, ix, wx);
    restrict_axis(T.fy, J, T.NYf, iy, wy);
    restrict_axis(T.fz, K, T.NZf, iz, wz);
    const float* src = tf + r * vsf;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int a = t % 3, b = t / 3;
      const float w = wx[a] * wy[b] * wz[c];
      const int m = (iz[c] * T.NYf + iy[b]) * T.NXf + ix[a];
      const float4 v = __ldg(reinterpret_cast<const float4*>(src) + m);
      a0 = fmaf(w, v.x, a0); a1 = fmaf(w, v.y, a1); a2 = fmaf(w, v.z, a2);
    }
  }
  part[c][0][tx] = a0;
  part[c][1][tx] = a1;
  part[c][2][tx] = a2;
  __syncthreads();
  if (!live || c != 0) return;
  float o[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) o[q] = (part[0][q][tx] + part[1][q][tx]) + part[2][q][tx];
  const uint8_t fx = fixc[N];
  reinterpret_cast<float4*>(rc + r * vsc)[N] =
      make_float4((fx & 1) ? 0.f : o[0], (fx & 2) ? 0.f : o[1], (fx & 4) ? 0.f : o[2], 0.f);
}

// e_f += P e_c (masked by the fine fixed bits); one thread per (fine node,
// right-hand side)
__global__ void k_mg_prolong(Transfer T, int R, const float* __restrict__ ec, const uint8_t* __restrict__ fixf,
                             float* ef) {
  const int NNf = T.NXf * T.NYf * T.NZf;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)NNf * R) return;
  const int n = int(t % NNf), r = int(t / NNf);
  const long long vsf = (long long)NNf * 4, vsc = (long long)T.NXc * T.NYc * T.NZc * 4;
  const float4 a = prolong_node(T.fx, T.fy, T.fz, T.NXf, T.NYf, T.NXc, T.NYc, n, ec + r * vsc);
  const uint8_t fx = fixf[n];
  float4 o = reinterpret_cast<float4*>(ef + r * vsf)[n];
  if (!(fx & 1)) o.x += a.x;
  if (!(fx & 2)) o.y += a.y;
  if (!(fx & 4)) o.z += a.z;
  reinterpret_cast<float4*>(ef + r * vsf)[n] = o;
}

// coarsest: e = Ainv r (n = 3 NN <= 3 * kCoarseNodes per vector, R <= 8
// right-hand sides).  Every CTA stages all right-hand sides in shared memory;
// one warp per row i reads row i of Ainv coalesced (lanes over columns),
// accumulates the R products and reduces them with shuffles.
constexpr int kCoarseWarps = 8;
__global__ void __launch_bounds__(32 * kCoarseWarps) k_mg_coarse_solve(int NN, int R, const double* __restrict__ Ainv,
                                                                       const float* __restrict__ r, float* e) {
  __shared__ double sr[TOF_MAX_RHS][3 * kCoarseNodes];
  const int n = 3 * NN;
  for (int w = threadIdx.x; w < R * n; w += blockDim.x) {
    const int q = w / n, i = w % n;
    sr[q][i] = double(r[(size_t)q * NN * 4 + (i / 3) * 4 + i % 3]);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kCoarseWarps + (threadIdx.x >> 5);
  if (i >= n) return;
  double acc[TOF_MAX_RHS];
#pragma unroll
  for (int q = 0; q < TOF_MAX_RHS; ++q) acc[q] = 0.0;
  const double* row = Ainv + (size_t)i * n;
  for (int j = lane; j < n; j += 32) {
    const double a = row[j];
#pragma unroll
    for (int q = 0; q < TOF_MAX_RHS; ++q)
      if (q < R) acc[q] = fma(a, sr[q][j], acc[q]);
  }
#pragma unroll
  for (int q = 0; q < TOF_MAX_RHS; ++q) {
    if (q >= R) break;
    const double v = warp_sum(acc[q]);
    if (lane == 0) {
      float* er = e + (size_t)q * NN * 4;
      er[(i / 3) * 4 + i % 3] = float(v);
      if (i % 3 == 0) er[(i / 3) * 4 + 3] = 0.f;
    }
  }
}

static void launch_coarse_solve(int NN, int R, const double* Ainv, const float* r, float* e, cudaStream_t s) {
  k_mg_coarse_solve<<<ceil_div(3 * NN, kCoarseWarps), 32 * kCoarseWarps, 0, s>>>(NN, R, Ainv, r, e);
  count_launch();
}

// ---------------------------------------------------------------------------
// host: hierarchy, setup, V-cycle
// ---------------------------------------------------------------------------
static LevelView view(const MGLevel& L) {
  return LevelView{L.nx, L.ny, L.nz, L.NX, L.NY, L.NZ, L.NN, L.St, L.dinv, L.fix};
}
static Transfer transfer(const MGLevel& f, const MGLevel& c) {
  return Transfer{f.NX, f.NY, f.NZ, c.NX, c.NY, c.NZ, c.fx, c.fy, c.fz};
}

int mg_create(Ctx& c, int maxR) {
  MG* mg = new MG();
  c.mg = mg;
  mg->maxR = maxR;
  int nx = c.g.nx, ny = c.g.ny, nz = c.g.nz;
  int l = 0;
  while (true) {
    MGLevel& L = mg->L[l];
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.NX = nx + 1; L.NY = ny + 1; L.NZ = nz + 1;
    L.NN = L.NX * L.NY * L.NZ;
    L.NE = nx * ny * nz;
    if (l == 0) { L.fx = L.fy = L.fz = 1; }
    const bool can = nx >= 2 || ny >= 2 || nz >= 2;
    if (L.NN <= kCoarseNodes || !can || l == kMaxLevels - 1) { mg->nlev = l + 1; break; }
    MGLevel& C = mg->L[l + 1];
    C.fx = nx >= 2 ? 2 : 1; C.fy = ny >= 2 ? 2 : 1; C.fz = nz >= 2 ? 2 : 1;
    nx = (nx + C.fx - 1) / C.fx; ny = (ny + C.fy - 1) / C.fy; nz = (nz + C.fz - 1) / C.fz;
    ++l;
  }
  const MGLevel& last = mg->L[mg->nlev - 1];
  if (last.NN > kCoarseNodes) { c.last_error = "multigrid: coarsest level too large"; return -1; }
  mg->nc = 3 * last.NN;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  auto al = [&](auto** p, size_t n) {
    using T = std::remove_pointer_t<std::remove_reference_t<decltype(*p)>>;
    const size_t b = std::max<size_t>(n, 1) * sizeof(T);
    c.bytes += b;
    A(cudaMalloc((void**)p, b));
    A(cudaMemset(*p, 0, b));
  };
  for (int k = 0; k < mg->nlev; ++k) {
    MGLevel& L = mg->L[k];
    const size_t V = (size_t)L.NN * 4 * maxR;
    if (k > 0) {
      al(&L.Ae, (size_t)L.NE * 576);
      al(&L.dinv, (size_t)L.NN * 4);
      al(&L.fix, (size_t)L.NN);
      if (k < mg->nlev - 1) al(&L.St, (size_t)L.NN * 243);
    } else {
      L.dinv = c.dinvK32;
      L.fix = c.fix;
    }
    for (int ln = 0; ln < kLanes; ++ln) {
      MGBuf& B = mg->buf[ln][k];
      al(&B.r, V); al(&B.e, V); al(&B.e2, V); al(&B.t, V);
    }
  }
  const size_t n2 = (size_t)mg->nc * mg->nc;
  al(&mg->A, n2); al(&mg->Y, n2); al(&mg->Ainv, n2);
  const size_t V0 = (size_t)c.g.NN * 4 * maxR;
  al(&mg->x, V0); al(&mg->r, V0); al(&mg->z, V0); al(&mg->q, V0); al(&mg->p[0], V0); al(&mg->p[1], V0);
  al(&mg->S, 256); al(&mg->flags, 64); al(&mg->cnt, 16); al(&mg->info, 16);
  al(&mg->omega, kMaxLevels); al(&mg->lam, kMaxLevels); al(&mg->coef, kMaxLevels * kCoefStride);
  mg->part_blocks = std::max(c.g.ntiles, 4 * c.num_sms);
  al(&mg->part, (size_t)mg->part_blocks * 3 * 8);
  if (e != cudaSuccess) { c.last_error = std::string("multigrid alloc: ") + cudaGetErrorString(e); return -2; }
  const char* sm = getenv("TOF_MG_SMOOTHER");
  mg->smoother = (sm && std::string(sm) == "jacobi") ? 1 : 0;
  static_assert(kMaxNu >= 2, "smoothing sweeps");
  return 0;
}

void mg_destroy(Ctx& c) {
  MG* mg = c.mg;
  if (!mg) return;
  for (int k = 0; k < mg->nlev; ++k) {
    MGLevel& L = mg->L[k];
    if (k > 0) { cudaFree(L.Ae); cudaFree(L.dinv); cudaFree(L.fix); if (L.St) cudaFree(L.St); }
    for (int ln = 0; ln < kLanes; ++ln) {
      MGBuf& B = mg->buf[ln][k];
      cudaFree(B.r); cudaFree(B.e); cudaFree(B.e2); cudaFree(B.t);
    }
  }
  for (auto& lane : mg->vexec)
    for (auto& g : lane)
      if (g) cudaGraphExecDestroy(g);
  void* ps[] = {mg->A, mg->Y, mg->Ainv, mg->x, mg->r, mg->z, mg->q, mg->p[0], mg->p[1], mg->S, mg->flags, mg->cnt,
                mg->info, mg->part, mg->omega, mg->lam, mg->coef};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete mg;
  c.mg = nullptr;
}

// Rebuild coarse operators after a density change.
int mg_setup(Ctx& c, cudaStream_t s) {
  MG* mg = c.mg;
  for (int k = 1; k < mg->nlev; ++k) {
    MGLevel& F = mg->L[k - 1];
    MGLevel& C = mg->L[k];
    GalerkinArgs a;
    a.nx = F.nx; a.ny = F.ny; a.nz = F.nz; a.NX = F.NX; a.NY = F.NY;
    a.Ae_f = k == 1 ? nullptr : F.Ae;
    a.fK = c.fK64; a.Ke = c.Ke64; a.fix0 = c.fix;
    a.cx = C.nx; a.cy = C.ny; a.cz = C.nz;
    a.fx = C.fx; a.fy = C.fy; a.fz = C.fz;
    a.Ae_c = C.Ae;
    k_mg_galerkin<<<C.NE, 128, 0, s>>>(a);
    count_launch();
    k_mg_diag<<<ceil_div(C.NN, 128), 128, 0, s>>>(C.nx, C.ny, C.nz, C.Ae, C.dinv, C.fix);
    count_launch();
    if (C.St) {
      k_mg_stencil<<<int((27LL * C.NN + 255) / 256), 256, 0, s>>>(C.nx, C.ny, C.nz, C.Ae, C.St);
      count_launch();
    }
  }
  const MGLevel& L = mg->L[mg->nlev - 1];
  const size_t csm = coarse_setup_smem(mg->nc);
  cudaFuncSetAttribute(k_mg_coarse_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
  k_mg_coarse_setup<<<1, 1024, csm, s>>>(L.nx, L.ny, L.nz, mg->nlev > 1 ? L.Ae : nullptr, c.fK64, c.Ke64, L.fix, mg->A,
                                      mg->Y, mg->info);
  count_launch();
  k_mg_coarse_inverse<<<ceil_div(mg->nc, 8), 256, 0, s>>>(mg->nc, mg->A, mg->Y, L.fix, mg->Ainv);
  count_launch();
  // smoothing weights: power iteration on D^-1 A_l (scratch: the level's e, e2)
  for (int k = 0; k < mg->nlev - 1; ++k) {
    MGLevel& V = mg->L[k];
    float* x = mg->buf[0][k].e;
    float* y = mg->buf[0][k].e2;
    k_mg_power_init<<<ceil_div(V.NN, 256), 256, 0, s>>>(V.NN, V.fix, x);
    count_launch();
    for (int it = 0; it < kPowerIters; ++it) {
      if (k == 0) {
        if (launch_matvec(c, 0, false, x, y, 1, nullptr, s)) return -2;
        k_mg_scale_dinv<<<ceil_div(V.NN, 256), 256, 0, s>>>(V.NN, V.dinv, y);
        count_launch();
      } else {
        launch_mgs_op(view(V), 1, x, nullptr, y, nullptr, 2, s);
      }
      std::swap(x, y);
    }
    k_mg_lambda<<<1, 1024, 0, s>>>(V.NN, y, x, mg->lam + k, mg->omega + k, mg->coef + k * kCoefStride, mg->nu,
                                   mg->smoother);
    count_launch();
  }
  mg->dirty = false;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <int R>
static int vcycle_t(Ctx& c, int lane, cudaStream_t s) {
  MG* mg = c.mg;
  MGBuf* Bf = mg->buf[lane];
  const int nl = mg->nlev;
  auto grid1 = [](int n) { return ceil_div(n, 128); };
  // Smoothing sweeps ping-pong between e and e2; the first sweep writes to
  // whichever buffer makes the last sweep of the level land in e, so the
  // buffer roles are the same in every V-cycle (required for graph replay).
  float* cur[kMaxLevels];
  float* alt[kMaxLevels];
  for (int k = 0; k < nl; ++k) {
    const bool odd = ((2 * mg->nu - 1) & 1) != 0;   // sweeps after the first
    cur[k] = odd ? Bf[k].e2 : Bf[k].e;
    alt[k] = odd ? Bf[k].e : Bf[k].e2;
  }
  // downward
  for (int k = 0; k < nl - 1; ++k) {
    MGLevel& L = mg->L[k];
    const float* cf = mg->coef + k * kCoefStride;
    // sweep 0 from x = 0: x_1 = sr D^-1 r
    k_mg_jacobi0<<<ceil_div(L.NN * R, 256), 256, 0, s>>>(L.NN, R, L.dinv, Bf[k].r, cur[k], cf + 2);
    count_launch();
    for (int sw = 1; sw < mg->nu; ++sw) {
      const bool prev = sw >= 2;             // x_0 = 0: sweep 1 has no x_{k-1} term
      if (k == 0) { if (launch_smooth0(c, cur[k], alt[k], Bf[k].r, L.dinv, cf + 3 * sw, prev, R, s)) return -2; }
      else launch_mgs_op(view(L), R, cur[k], Bf[k].r, alt[k], cf + 3 * sw, prev ? 3 : 1, s);
      std::swap(cur[k], alt[k]);
    }
    if (k == 0) { if (launch_matvec(c, 0, false, cur[k], Bf[k].t, R, Bf[k].r, s)) return -2; }
    else launch_mgs_op(view(L), R, cur[k], Bf[k].r, Bf[k].t, nullptr, 0, s);
    MGLevel& C = mg->L[k + 1];
    k_mg_restrict_split<<<dim3(ceil_div(C.NN, 32), R), dim3(32, 3), 0, s>>>(transfer(L, C), R, Bf[k].t, C.fix,
                                                                       Bf[k + 1].r);
    count_launch();
  }
  {
    MGLevel& L = mg->L[nl - 1];
    launch_coarse_solve(L.NN, R, mg->Ainv, Bf[nl - 1].r, Bf[nl - 1].e, s);
    cur[nl - 1] = Bf[nl - 1].e;
  }
  // upward
  for (int k = nl - 2; k >= 0; --k) {
    MGLevel& L = mg->L[k];
    MGLevel& C = mg->L[k + 1];
    k_mg_prolong<<<grid1(L.NN * R), 128, 0, s>>>(transfer(L, C), R, cur[k + 1], L.fix, cur[k]);
    count_launch();
    const float* cf = mg->coef + k * kCoefStride;
    for (int sw = 0; sw < mg->nu; ++sw) {
      const bool prev = sw >= 1;             // alt holds x_{k-1} after the first sweep
      if (k == 0) { if (launch_smooth0(c, cur[k], alt[k], Bf[k].r, L.dinv, cf + 3 * sw, prev, R, s)) return -2; }
      else launch_mgs_op(view(L), R, cur[k], Bf[k].r, alt[k], cf + 3 * sw, prev ? 3 : 1, s);
      std::swap(cur[k], alt[k]);
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

static int vcycle_eager(Ctx& c, int R, int lane, cudaStream_t s) {
  if (c.mg->nlev == 1) {
    MGLevel& L = c.mg->L[0];
    launch_coarse_solve(L.NN, R, c.mg->Ainv, c.mg->buf[lane][0].r, c.mg->buf[lane][0].e, s);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
  }
  switch (R) {
    case 1: return vcycle_t<1>(c, lane, s);
    case 2: return vcycle_t<2>(c, lane, s);
    case 4: return vcycle_t<4>(c, lane, s);
    case 8: return vcycle_t<8>(c, lane, s);
  }
  return -1;
}

// Capture the V-cycle of one lane and R into a graph (recorded, not run).
static bool capture_vcycle(Ctx& c, int lane, int ri, int R, cudaStream_t s) {
  MG* mg = c.mg;
  cudaGraphExec_t& ge = mg->vexec[lane][ri];
  cudaGraph_t graph = nullptr;
  bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  capturing() = ok;
  if (ok) ok = vcycle_eager(c, R, lane, s) == 0;
  capturing() = false;
  const bool ended = cudaStreamEndCapture(s, &graph) == cudaSuccess;
  if (ok && ended && graph && cudaGraphInstantiate(&ge, graph, 0) == cudaSuccess) {
    cudaGraphGetNodes(graph, nullptr, &mg->vnodes[lane][ri]);
  } else {
    ge = nullptr;
    mg->vgraph_failed = true;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();   // clear a refused capture (e.g. the legacy default stream)
  return ge != nullptr;
}

// All V-cycle graphs (both lanes, every R the context supports), recorded
// once when the context is created: the buffers, tensor maps and smoothing
// coefficients they reference never move, so no solve pays a capture and an
// instantiation.
int mg_capture_all(Ctx& c) {
  MG* mg = c.mg;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) { cudaGetLastError(); return 0; }
  const int Rs[4] = {1, 2, 4, 8};
  for (int lane = 0; lane < kLanes && !mg->vgraph_failed; ++lane)
    for (int ri = 0; ri < 4 && !mg->vgraph_failed; ++ri)
      if (Rs[ri] <= mg->maxR && !mg->vexec[lane][ri]) capture_vcycle(c, lane, ri, Rs[ri], s);
  cudaStreamDestroy(s);
  return 0;
}

// Apply the V-cycle to mg_rhs(c, lane) (R vectors); result in mg_out(c, lane).
// Inside a stream capture (tof_time_kernel's graphs) the kernels are recorded as they
// are; otherwise the recorded graph of this lane and R is replayed, which
// removes the per-kernel launch overhead of ~40 short launches.
int mg_vcycle(Ctx& c, int R, cudaStream_t s, int lane) {
  MG* mg = c.mg;
  const int ri = R == 1 ? 0 : R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : -1;
  if (ri < 0 || lane < 0 || lane >= kLanes) return -1;
  if (capturing() || mg->vgraph_failed) return vcycle_eager(c, R, lane, s);
  cudaGraphExec_t& ge = mg->vexec[lane][ri];
  if (!ge && !capture_vcycle(c, lane, ri, R, s)) return vcycle_eager(c, R, lane, s);
  if (cudaGraphLaunch(ge, s) != cudaSuccess) return -2;
  count_launch((long long)mg->vnodes[lane][ri]);
  return 0;
}

int mg_query(Ctx& c, int level, int* dims, float* omega, cudaStream_t s) {
  MG* mg = c.mg;
  if (level < 0) return mg->nlev;
  if (level >= mg->nlev) return -1;
  if (mg->dirty && mg_setup(c, s)) return -2;
  if (dims) { dims[0] = mg->L[level].nx; dims[1] = mg->L[level].ny; dims[2] = mg->L[level].nz; }
  if (omega) {
    if (level < mg->nlev - 1) {
      cudaMemcpyAsync(omega, mg->omega + level, sizeof(float), cudaMemcpyDeviceToHost, s);
      cudaStreamSynchronize(s);
    } else {
      *omega = 0.f;
    }
  }
  return mg->nlev;
}

int mg_export(Ctx& c, int level, float* out, cudaStream_t s) {
  MG* mg = c.mg;
  if (level < 1 || level >= mg->nlev) return -1;
  if (mg->dirty && mg_setup(c, s)) return -2;
  const MGLevel& L = mg->L[level];
  return cudaMemcpyAsync(out, L.Ae, sizeof(float) * 576 * (size_t)L.NE, cudaMemcpyDeviceToDevice, s) == cudaSuccess
             ? 0
             : -2;
}

int mg_apply(Ctx& c, const float* r, float* e, int R, cudaStream_t s) {
  MG* mg = c.mg;
  if (R != 1 && R != 2 && R != 4 && R != 8) return -1;
  if (R > mg->maxR) return -1;
  if (mg->dirty && mg_setup(c, s)) return -2;
  const size_t bytes = sizeof(float) * 4 * (size_t)c.g.NN * R;
  cudaMemcpyAsync(mg->buf[0][0].r, r, bytes, cudaMemcpyDeviceToDevice, s);
  if (mg_vcycle(c, R, s)) return -2;
  return cudaMemcpyAsync(e, mg->buf[0][0].e, bytes, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? 0 : -2;
}

int mg_launch_level_op(Ctx& c, int level, int R, cudaStream_t s, long long* nodes) {
  MG* mg = c.mg;
  if (!mg || mg->dirty) { c.last_error = "the multigrid hierarchy is not set up (tof_mg_setup)"; return -1; }
  if (level < 1 || level > mg->nlev - 2) { c.last_error = "level must be a stencil level (1 .. levels - 2)"; return -1; }
  if ((R != 1 && R != 2 && R != 4 && R != 8) || R > mg->maxR) {
    c.last_error = "R must be 1, 2, 4 or 8 and at most the context's max_rhs";
    return -1;
  }
  MGLevel& L = mg->L[level];
  MGBuf& B = mg->buf[0][level];
  *nodes = L.NN;
  launch_mgs_op(view(L), R, B.e, B.r, B.e2, mg->coef + level * kCoefStride + 3, 3, s);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

void mg_mark_dirty(Ctx& c) {
  if (c.mg) c.mg->dirty = true;
}
int mg_ensure(Ctx& c, cudaStream_t s) { return c.mg->dirty ? mg_setup(c, s) : 0; }
float* mg_rhs(Ctx& c, int lane) { return c.mg->buf[lane][0].r; }
float* mg_out(Ctx& c, int lane) { return c.mg->buf[lane][0].e; }
int mg_levels(const Ctx& c) { return c.mg ? c.mg->nlev : 0; }

// ---------------------------------------------------------------------------
// FP64 PCG preconditioned by the FP32 V-cycle
// ---------------------------------------------------------------------------
// scalar layout per rhs k: S[k*8 + {0: rz, 1: alpha, 2: beta, 3: rr, 4: bnorm, 5: iters}]
// flags[k]: 0 active, 1 converged, 2 breakdown (p.q <= 0), 3 non-finite

// r = b - A x0 already computed into mg->r; r32 = (float) r; rr, bb
template <int R>
__global__ void __launch_bounds__(256) k_mgpcg_init(int NN, const double* __restrict__ b, const double* __restrict__ r,
                                                   float* r32, double* p0, double* S, int* flags, double* part,
                                                   unsigned* cnt, double rtol) {
  __shared__ double red[2 * R * 32];
  double v[2 * R];
#pragma unroll
  for (int k = 0; k < 2 * R; ++k) v[k] = 0.0;
  const long long vs = (long long)NN * 4;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const double4 rr = reinterpret_cast<const double4*>(r + k * vs)[n];
      const double4 bb = reinterpret_cast<const double4*>(b + k * vs)[n];
      reinterpret_cast<float4*>(r32 + k * vs)[n] = make_float4(float(rr.x), float(rr.y), float(rr.z), 0.f);
      reinterpret_cast<double4*>(p0 + k * vs)[n] = make_double4(0, 0, 0, 0);
      v[2 * k] += rr.x * rr.x + rr.y * rr.y + rr.z * rr.z;
      v[2 * k + 1] += bb.x * bb.x + bb.y * bb.y + bb.z * bb.z;
    }
  }
  double tot[2 * R];
  if (last_block<2 * R>(v, part, cnt, red, tot) && threadIdx.x == 0) {
    for (int k = 0; k < R; ++k) {
      const double bn = sqrt(tot[2 * k + 1]);
      S[k * 8 + 3] = tot[2 * k];
      S[k * 8 + 4] = bn;
      S[k * 8 + 6] = rtol;
      S[k * 8 + 5] = 0.0;
      S[k * 8 + 2] = 0.0;
      int f = 0;
      if (!isfinite(tot[2 * k]) || !isfinite(bn)) f = 3;
      else if (!(bn > 0.0) || sqrt(tot[2 * k]) <= rtol * bn) f = 1;
      flags[k] = f;
    }
  }
}

// z = (double) e0; rz = r.z; beta = rz / rz_prev (first: 0)
template <int R>
__global__ void __launch_bounds__(256) k_mgpcg_zrz(int NN, const float* __restrict__ e0, const double* __restrict__ r,
                                                  double* z, double* S, const int* flags, double* part, unsigned* cnt,
                                                  int first) {
  __shared__ double red[R * 32];
  double v[R];
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = 0.0;
  const long long vs = (long long)NN * 4;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const float4 e = reinterpret_cast<const float4*>(e0 + k * vs)[n];
      const double4 rr = reinterpret_cast<const double4*>(r + k * vs)[n];
      reinterpret_cast<double4*>(z + k * vs)[n] = make_double4(e.x, e.y, e.z, 0.0);
      v[k] += rr.x * e.x + rr.y * e.y + rr.z * e.z;
    }
  }
  double tot[R];
  if (last_block<R>(v, part, cnt, red, tot) && threadIdx.x == 0) {
    for (int k = 0; k < R; ++k) {
      if (flags[k]) continue;
      const double rz = tot[k];
      S[k * 8 + 2] = first ? 0.0 : rz / S[k * 8 + 0];
      S[k * 8 + 0] = rz;
    }
  }
}

// p_new = z + beta p_old; q = A p_new; alpha = rz / p.q (tile kernel, FP64)
template <int R>
__global__ void __launch_bounds__(256) k_mgpcg_pq(const __grid_constant__ CUtensorMap tmz,
                                                 const __grid_constant__ CUtensorMap tmp, Grid g,
                                                 const double* __restrict__ fK, const double* __restrict__ keb,
                                                 const uint8_t* __restrict__ fix, double* pn, double* q, double* S,
                                                 int* flags, double* part, unsigned* cnt) {
  extern __shared__ __align__(128) unsigned char smem[];
  using V4 = double4;
  const TileGeom tg = tile_geom(g, blockIdx.x);
  const unsigned hbytes = halo_bytes<double>(g, R);
  double* sz = reinterpret_cast<double*>(smem);
  double* sp = reinterpret_cast<double*>(smem + hbytes);
  double* sKe = reinterpret_cast<double*>(smem + 2 * hbytes);
  double* sf = sKe + kKeBlocksLen;
  const int nfe = tg.EX * tg.EY * tg.EZ;
  double* red = sf + nfe;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(red + R * 32);
  __shared__ double beta[R];
  __shared__ int fz[R];
  if (threadIdx.x == 0) {
    mbar_init(mbar, 1);
    mbar_arrive_expect_tx(mbar, 2 * hbytes);
    tma_load_5d(sz, &tmz, 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, mbar);
    tma_load_5d(sp, &tmp, 0, tg.i0 - 1, tg.j0 - 1, tg.k0 - 1, 0, mbar);
  }
  if (threadIdx.x < R) { beta[threadIdx.x] = S[threadIdx.x * 8 + 2]; fz[threadIdx.x] = flags[threadIdx.x]; }
  load_ke_blocks(keb, sKe);
  load_factor_tile(g, tg, fK, sf);
  __syncthreads();   // mbarrier initialised before anyone waits on it
  const bool ok = __syncthreads_and(mbar_wait(mbar, 0));
  const int hsr = tg.HX * tg.HY * tg.HZ;
  if (ok) {
    for (int idx = threadIdx.x; idx < R * hsr; idx += blockDim.x) {
      const int k = idx / hsr;
      const V4 z4 = reinterpret_cast<V4*>(sz)[idx];
      V4 p4 = reinterpret_cast<V4*>(sp)[idx];
      const double be = fz[k] ? 0.0 : beta[k];
      p4.x = fma(be, p4.x, z4.x); p4.y = fma(be, p4.y, z4.y); p4.z = fma(be, p4.z, z4.z); p4.w = 0.0;
      reinterpret_cast<V4*>(sp)[idx] = p4;
    }
  }
  __syncthreads();
  double v[R];
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = 0.0;
  int tx, ty, tz, n;
  if (ok && thread_node(g, tg, tx, ty, tz, n)) {
    double acc[R][3];
    stencil_node<double, R>(sp, tg, sf, sKe, tx, ty, tz, acc);
    const uint8_t fx = __ldg(fix + n);
    const long long vs = (long long)g.NN * 4;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const V4 pp = halo_center<double>(sp, tg, k, tx, ty, tz);
      const V4 qq = make_double4((fx & 1) ? 0.0 : acc[k][0], (fx & 2) ? 0.0 : acc[k][1], (fx & 4) ? 0.0 : acc[k][2], 0.0);
      reinterpret_cast<V4*>(q + k * vs)[n] = qq;
      reinterpret_cast<V4*>(pn + k * vs)[n] = pp;
      v[k] += pp.x * qq.x + pp.y * qq.y + pp.z * qq.z;
    }
  }
  double tot[R];
  if (last_block<R>(v, part, cnt, red, tot) && threadIdx.x == 0) {
    for (int k = 0; k < R; ++k) {
      if (flags[k]) { S[k * 8 + 1] = 0.0; continue; }
      if (!isfinite(tot[k])) { flags[k] = 3; S[k * 8 + 1] = 0.0; continue; }
      if (!(tot[k] > 0.0)) { flags[k] = 2; S[k * 8 + 1] = 0.0; continue; }
      S[k * 8 + 1] = S[k * 8 + 0] / tot[k];
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(flags + 8, ST_TIMEOUT);
}

// x += alpha p; r -= alpha q; r32 = (float) r; rr; convergence flags
template <int R>
__global__ void __launch_bounds__(256) k_mgpcg_xr(int NN, const double* __restrict__ p, const double* __restrict__ q,
                                                 double* x, double* r, float* r32, double* S, int* flags,
                                                 double* part, unsigned* cnt) {
  __shared__ double red[R * 32];
  __shared__ double al[R];
  __shared__ int fz[R];
  if (threadIdx.x < R) { al[threadIdx.x] = S[threadIdx.x * 8 + 1]; fz[threadIdx.x] = flags[threadIdx.x]; }
  __syncthreads();
  double v[R];
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = 0.0;
  const long long vs = (long long)NN * 4;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NN; n += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const size_t o = k * vs / 4 + n;
      double4 rr = reinterpret_cast<const double4*>(r)[o];
      if (!fz[k]) {
        const double a = al[k];
        const double4 pp = reinterpret_cast<const double4*>(p)[o];
        const double4 qq = reinterpret_cast<const double4*>(q)[o];
        double4 xx = reinterpret_cast<const double4*>(x)[o];
        xx.x = fma(a, pp.x, xx.x); xx.y = fma(a, pp.y, xx.y); xx.z = fma(a, pp.z, xx.z);
        rr.x = fma(-a, qq.x, rr.x); rr.y = fma(-a, qq.y, rr.y); rr.z = fma(-a, qq.z, rr.z);
        reinterpret_cast<double4*>(x)[o] = xx;
        reinterpret_cast<double4*>(r)[o] = rr;
      }
      reinterpret_cast<float4*>(r32)[o] = make_float4(float(rr.x), float(rr.y), float(rr.z), 0.f);
      v[k] += rr.x * rr.x + rr.y * rr.y + rr.z * rr.z;
    }
  }
  double tot[R];
  if (last_block<R>(v, part, cnt, red, tot) && threadIdx.x == 0) {
    for (int k = 0; k < R; ++k) {
      if (flags[k]) continue;
      S[k * 8 + 3] = tot[k];
      S[k * 8 + 5] += 1.0;
      if (!isfinite(tot[k])) flags[k] = 3;
      else if (sqrt(tot[k]) <= S[k * 8 + 6] * S[k * 8 + 4]) flags[k] = 1;
    }
  }
}

template <int R>
static int mgpcg_iter(Ctx& c, int pc, cudaStream_t s) {
  MG* mg = c.mg;
  const int eb = std::min(ceil_div(c.g.NN, 256), 2 * c.num_sms);
  std::string err;
  CUtensorMap tmz, tmp;
  if (!encode_node4_map(&tmz, mg->z, c.g, R, true, &err) || !encode_node4_map(&tmp, mg->p[pc], c.g, R, true, &err)) {
    c.last_error = err;
    return -2;
  }
  const int nfe = (c.g.TX + 1) * (c.g.TY + 1) * (c.g.TZ + 1);
  const size_t smem = 2 * size_t(halo_bytes<double>(c.g, R)) + 8 * (kKeBlocksLen + nfe) + 8 * R * 32 + 16;
  auto kern = k_mgpcg_pq<R>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<c.g.ntiles, c.g.TX * c.g.TY * c.g.TZ, smem, s>>>(tmz, tmp, c.g, c.fK64, c.keb64, c.fix, mg->p[pc ^ 1], mg->q,
                                                           mg->S, mg->flags, mg->part, mg->cnt + 0);
  count_launch();
  k_mgpcg_xr<R><<<eb, 256, 0, s>>>(c.g.NN, mg->p[pc ^ 1], mg->q, mg->x, mg->r, mg->buf[0][0].r, mg->S, mg->flags, mg->part,
                                   mg->cnt + 1);
  count_launch();
  if (mg_vcycle(c, R, s)) return -2;
  k_mgpcg_zrz<R><<<eb, 256, 0, s>>>(c.g.NN, mg->buf[0][0].e, mg->r, mg->z, mg->S, mg->flags, mg->part, mg->cnt + 2, 0);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Solve K x = b (R node4 FP64 rhs, x holds x0 and the result) to rtol.
template <int R>
static int mgpcg_t(Ctx& c, const double* b, double* x, double rtol, int maxiter, int* iters, int* status,
                   cudaStream_t s) {
  MG* mg = c.mg;
  const size_t V = (size_t)c.g.NN * 4;
  if (mg->dirty && mg_setup(c, s)) return -2;
  cudaMemsetAsync(mg->flags, 0, sizeof(int) * 16, s);
  cudaMemsetAsync(mg->cnt, 0, sizeof(unsigned) * 16, s);
  cudaMemcpyAsync(mg->x, x, sizeof(double) * R * V, cudaMemcpyDeviceToDevice, s);
  if (launch_matvec(c, 0, true, mg->x, mg->r, R, b, s)) return -2;
  const int eb = std::min(ceil_div(c.g.NN, 256), 2 * c.num_sms);
  k_mgpcg_init<R><<<eb, 256, 0, s>>>(c.g.NN, b, mg->r, mg->buf[0][0].r, mg->p[0], mg->S, mg->flags, mg->part, mg->cnt + 3,
                                     rtol);
  count_launch();
  if (mg_vcycle(c, R, s)) return -2;
  k_mgpcg_zrz<R><<<eb, 256, 0, s>>>(c.g.NN, mg->buf[0][0].e, mg->r, mg->z, mg->S, mg->flags, mg->part, mg->cnt + 2, 1);
  count_launch();
  int it = 0;
  int hf[9];
  while (true) {
    cudaMemcpyAsync(hf, mg->flags, sizeof(int) * 9, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { c.last_error = "multigrid PCG: CUDA error"; return -2; }
    bool all = true;
    for (int k = 0; k < R; ++k) all = all && hf[k] != 0;
    if (all || it >= maxiter || hf[8]) break;
    // kCheckIters iterations between two host checks of the flags, each
    // kernel launched on its own (never more than maxiter iterations)
    const int step = std::min(kCheckIters, maxiter - it);
    for (int q = 0; q < step; ++q)
      if (mgpcg_iter<R>(c, q & 1, s)) return -2;
    it += step;
  }
  cudaMemcpyAsync(x, mg->x, sizeof(double) * R * V, cudaMemcpyDeviceToDevice, s);
  double hs[64];
  cudaMemcpyAsync(hs, mg->S, sizeof(double) * 8 * R, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { c.last_error = "multigrid PCG: CUDA error"; return -2; }
  for (int k = 0; k < R; ++k) {
    iters[k] = int(hs[k * 8 + 5]);
    status[k] = hf[8] ? ST_TIMEOUT
                : hf[k] == 1 ? ST_OK
                : hf[k] == 2 ? ST_BREAKDOWN
                : hf[k] == 3 ? ST_NONFINITE
                             : ST_NOT_CONVERGED;
  }
  return 0;
}

int pcg_mg64(Ctx& c, const double* b, double* x, int R, double rtol, int maxiter, int* iters, int* status,
             cudaStream_t s) {
  switch (R) {
    case 1: return mgpcg_t<1>(c, b, x, rtol, maxiter, iters, status, s);
    case 2: return mgpcg_t<2>(c, b, x, rtol, maxiter, iters, status, s);
    case 4: return mgpcg_t<4>(c, b, x, rtol, maxiter, iters, status, s);
    case 8: return mgpcg_t<8>(c, b, x, rtol, maxiter, iters, status, s);
  }
  c.last_error = "multigrid PCG: nrhs must be 1, 2, 4 or 8";
  return -1;
}

// Load every kernel of this file now (CUDA loads device functions lazily,
// at first use, and a first use in the middle of a solve stalls it).
void preload_kernels_gmg() {
  auto touch = [](auto f) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(f));
  };
  touch(k_mg_galerkin); touch(k_mg_diag); touch(k_mg_stencil); touch(k_mg_coarse_setup);
  touch(k_mg_coarse_inverse); touch(k_mgs_op); touch(k_mgs_op_split); touch(k_mg_jacobi0); touch(k_mg_power_init); touch(k_mg_scale_dinv);
  touch(k_mg_lambda); touch(k_mg_restrict_split); touch(k_mg_prolong); touch(k_mg_coarse_solve);
  touch(k_mgpcg_init<1>); touch(k_mgpcg_init<2>); touch(k_mgpcg_init<4>); touch(k_mgpcg_init<8>);
  touch(k_mgpcg_zrz<1>); touch(k_mgpcg_zrz<2>); touch(k_mgpcg_zrz<4>); touch(k_mgpcg_zrz<8>);
  touch(k_mgpcg_pq<1>); touch(k_mgpcg_pq<2>); touch(k_mgpcg_pq<4>); touch(k_mgpcg_pq<8>);
  touch(k_mgpcg_xr<1>); touch(k_mgpcg_xr<2>); touch(k_mgpcg_xr<4>); touch(k_mgpcg_xr<8>);
}

}  // namespace tof

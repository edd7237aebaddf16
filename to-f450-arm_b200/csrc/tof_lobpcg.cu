// Block LOBPCG for the lowest modes of K x = lambda M x (sm_100a).
//
// The reference calls SciPy's lobpcg on the assembled K_ff, M_ff with a Jacobi
// preconditioner, tol 1e-4, maxiter 500 (src/fem.py:400-470; CuPy's lobpcg
// on the GPU, src/fem_gpu.py:101-173).  Here the FP64 block vectors live on
// the device in node4 layout; each iteration:
//   W = K X - M X diag(theta)           (k_lob_resid, FP64 norms; soft-locked
//                                        columns leave W)
//   W <- T W                            (Jacobi, a few FP32 PCG iterations,
//                                        or one FP32 multigrid V-cycle)
//   KW, MW                              (matrix-free block matvecs)
//   G_K = S^T K S, G_M = S^T M S        (S = [X W_act P_act], FP64 Gram)
//   Rayleigh-Ritz on (G_K, G_M)         (k_small_eig: one CTA; Cholesky of
//                                        the scaled G_M, or SVQB when the
//                                        basis is ill-conditioned; parallel
//                                        cyclic Jacobi for the small problem)
//   X, P, KX, MX, KP, MP <- S C         (k_lob_update)
// K X, M X, K P, M P are recomputed every kLobRefresh iterations and before
// convergence is accepted; a final FP64 Rayleigh-Ritz on fresh products gives
// the returned pairs.
#include <math.h>

#include <algorithm>
#include <stdio.h>

#include "tof_internal.h"
#include "tof_stencil.cuh"

namespace tof {

constexpr int kMaxBasis = 24;
#ifndef TOF_LOB_REFRESH
#define TOF_LOB_REFRESH 20
#endif
constexpr int kLobRefresh = TOF_LOB_REFRESH;   // iterations between fresh K / M products
// Below its rounding floor (~eps * lambda_max / lambda_1 of the pencil) the
// iteration stops converging and its basis can degrade.  The best iterate
// (smallest worst wanted residual) is kept aside.  Once that best is below
// kLobNearFloor (far from the plateaus near 1 that a Jacobi-preconditioned
// start goes through) the iteration stops, not converged, when the residual
// grows kLobDiverge-fold over the best or has not improved for
// max(kLobStall, iterations taken to reach the best), and the best iterate
// is returned.
constexpr int kLobStall = 500;
constexpr double kLobDiverge = 1e3;
constexpr double kLobNearFloor = 1e-3;
// The best iterate is copied aside only below this residual (at or above
// kLobNearFloor, where it is restarted from or returned; and at maxiter).
constexpr double kLobKeepBelow = 1e-2;
// Before stopping, a residual kLobRestartGrowth times above the best
// iterate's restarts the iteration from that iterate without P (at most
// kLobMaxRestarts times).
constexpr double kLobRestartGrowth = 10.0;
constexpr int kLobMaxRestarts = 3;
// A wanted residual within this factor of its FP64 rounding floor counts as
// converged when the floor lies above the requested tolerance.
constexpr double kLobFloorFactor = 10.0;

// y_k += theta_k m_k for nv vectors of n doubles (theta on the device)
__global__ void k_add_scaled_cols(long long n, int nv, const double* __restrict__ theta, const double* __restrict__ m,
                                  double* y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n * nv) y[i] = fma(theta[i / n], m[i], y[i]);
}

// ---------------------------------------------------------------------------
// residual W_j = KX_j - theta_j MX_j, optional Jacobi scaling, written to
// vector wslot.col[j] of S (skipped for wslot.col[j] < 0: a soft-locked
// column), and the norms ||W_j||^2, ||KX_j||^2 (unscaled residual) of every
// column, reduced by the last CTA into out[2j], out[2j+1]
// ---------------------------------------------------------------------------
// What the host reads of each LOBPCG iteration (pinned, mapped host memory
// written by the residual kernel): the residual and K X norms of each
// column, theta, and the rank word of the Rayleigh-Ritz step before it.
struct LobSlot {
  double r[16];
  double th[8];
  int info;
  int pad;
};

// One work item per (node, column): the residual column j of node n, its
// norms accumulated per thread and reduced by the last block; items
// nb .. nb + (R32 - na) - 1 zero the multigrid padding vectors na .. R32-1.
template <typename T>
__global__ void __launch_bounds__(256) k_lob_resid(int NN, int nb, long long vs, const T* __restrict__ KX,
                                                   const T* __restrict__ MX, const double* __restrict__ theta,
                                                   const T* __restrict__ dinv, T* S, ColMap wslot, double* part,
                                                   unsigned* counter, double* out, float* w32, int na, int R32,
                                                   const int* info, LobSlot* host) {
  using V4 = typename Vec4<T>::type;
  __shared__ double red[16 * 32];
  double v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = 0.0;
  const int npad = w32 ? R32 - na : 0;
  const long long items = (long long)NN * (nb + npad);
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < items;
       idx += (long long)gridDim.x * blockDim.x) {
    const int j = int(idx / NN), n = int(idx % NN);
    if (j >= nb) {
      reinterpret_cast<float4*>(w32 + (na + j - nb) * vs)[n] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    const size_t o = j * vs / 4 + n;
    const V4 kx = reinterpret_cast<const V4*>(KX)[o];
    const V4 mx = reinterpret_cast<const V4*>(MX)[o];
    const T th = T(theta[j]);
    V4 w;
    w.x = kx.x - th * mx.x; w.y = kx.y - th * mx.y; w.z = kx.z - th * mx.z; w.w = T(0);
    const double rr = double(w.x) * w.x + double(w.y) * w.y + double(w.z) * w.z;
    const double kk = double(kx.x) * kx.x + double(kx.y) * kx.y + double(kx.z) * kx.z;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k == j) { v[2 * k] += rr; v[2 * k + 1] += kk; }
    if (dinv) {
      const V4 di = reinterpret_cast<const V4*>(dinv)[n];
      w.x *= di.x; w.y *= di.y; w.z *= di.z;
    }
    int ws = -1;                     // wslot.col[j] without a dynamic index into the parameter
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k == j) ws = wslot.col[k];
    if (ws >= 0) {
      reinterpret_cast<V4*>(S + ws * vs)[n] = w;
      if (w32)
        reinterpret_cast<float4*>(w32 + (ws - nb) * vs)[n] = make_float4(float(w.x), float(w.y), float(w.z), 0.f);
    }
  }
  double tot[16];
  if (last_block<16>(v, part, counter, red, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 16; ++k) out[k] = tot[k];
    if (host) {
#pragma unroll
      for (int k = 0; k < 16; ++k) host->r[k] = tot[k];
      for (int j = 0; j < nb; ++j) host->th[j] = theta[j];
      host->info = *info;
      __threadfence_system();
    }
  }
}

// ---------------------------------------------------------------------------
// Symmetric eigensolver for K <= 24, one CTA, matrix in shared memory:
// cyclic two-sided Jacobi (Golub & Van Loan, Matrix Computations, 4th ed.,
// Alg. 8.5.2 / 8.5.3) with the parallel round-robin ordering (ibid.,
// Sec. 8.5.5): the NP / 2 disjoint index pairs of a round (NP = K rounded up
// to even; a pair holding the padding index is the identity) are rotated at
// once: NP / 2 threads compute the rotations, then thread (i, j) writes
// element (i, j) of J^T A J and of V J to the other buffer.  A pair (p, q) is rotated unless
// a_pq^2 <= tol^2 |a_pp a_qq| -- the relative criterion, which gives the
// small eigenvalues of a positive definite matrix to high relative accuracy
// (Demmel & Veselic, SIAM J. Matrix Anal. Appl. 13 (1992)) -- or
// |a_pq| <= kJacAbs ||A||_F, the rounding level of the rotations themselves
// (the backward error of QR), which ends the iteration on the nearly
// singular Gram matrices of the SVQB path.  The iteration ends at the first
// tested round whose input matrix meets the criterion everywhere.  A round
// is one rotation (~530 cycles on a B200: two dependent FP64 reciprocal
// square roots), a barrier, the element update of all 18 warps (~850
// cycles) and a barrier: 6-10 sweeps of K - 1 rounds on the graded
// Rayleigh-Ritz matrices of LOBPCG, against one Givens rotation per step of
// the serial QR bulge chase on one warp.  Computing the next round's
// rotations during the update (a spare warp, one barrier per round) was
// measured no faster: the rotation chain then competes with the update for
// issue slots.
// On return d[k] / V[:, k] are the eigenpairs (unsorted); false if
// kJacSweeps sweeps did not converge.  S (the input) is left unchanged; the
// iteration runs in JA / JV, two matrix buffers each, selected by the
// round's parity (indexing one shared array rather than swapping pointers
// keeps every access a shared-memory load).  The stopping test is evaluated
// on every kJacTestEvery-th round's input (up to kJacTestEvery - 1 extra
// rounds of rotations at the rounding level, for one test in four).
// ---------------------------------------------------------------------------
constexpr int LDA = kMaxBasis + 1;
constexpr int kEigThreads = kMaxBasis * kMaxBasis;   // one thread per element
constexpr int kJacSweeps = 40;
constexpr int kJacTestEvery = 4;
constexpr double kJacTol = 1e-14;
constexpr double kJacAbs = 1e-15;

__device__ __forceinline__ bool jac_offdiag_live(double apq, double app, double aqq, double floor2) {
  const double a2 = apq * apq;
  return a2 > kJacTol * kJacTol * fabs(app * aqq) && a2 > floor2;
}

__device__ bool cta_jacobi(const double (*S)[LDA], double (*JA)[kMaxBasis][LDA], double (*JV)[kMaxBasis][LDA],
                           double (*V)[LDA], double* d, int K) {
  // per index x of the round: the new row x of J^T A is
  // jal[x] A[x, :] + jbe[x] A[jmt[x], :] (the same for the columns of A J)
  __shared__ double jal[kMaxBasis + 1], jbe[kMaxBasis + 1];
  __shared__ int jmt[kMaxBasis + 1];
  __shared__ unsigned char jpq[kMaxBasis - 1][kMaxBasis / 2][2];   // the round-robin schedule
  __shared__ double red[kEigThreads / 32];
  __shared__ double fro2;
  const int t = threadIdx.x;
  const int i = t / kMaxBasis, j = t % kMaxBasis;
  const bool own = i < K && j < K;
  const int NP = K + (K & 1), M = NP - 1;
  if (t < M * (NP / 2)) {
    // pair k of round r on NP = M + 1 players (M odd): player 0 meets
    // circle position r, positions r + k and r - k meet each other
    const int r = t / (NP / 2), k = t % (NP / 2);
    int p = k == 0 ? 0 : (r + k) % M + 1;
    int q = k == 0 ? r + 1 : (r - k + M) % M + 1;
    jpq[r][k][0] = (unsigned char)min(p, q);
    jpq[r][k][1] = (unsigned char)max(p, q);
  }
  const double s0 = own ? S[i][j] : 0.0;
  const double a2 = warp_sum(s0 * s0);   // ||A||_F^2
  if ((t & 31) == 0) red[t >> 5] = a2;
  if (own) {
    JA[0][i][j] = s0;
    JV[0][i][j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (t == 0) {
    double f = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) f += red[w];
    fro2 = f;
  }
  __syncthreads();
  const double floor2 = kJacAbs * kJacAbs * fro2;
  int cur = 0;
  bool conv = M <= 0;
  for (int it = 0, r = 0; !conv && it < kJacSweeps * M; ++it, r = (r + 1 == M) ? 0 : r + 1) {
    if (t < NP / 2) {
      const int p = jpq[r][t][0], q = jpq[r][t][1];
      double c = 1.0, sn = 0.0;
      bool rot = false;
      if (q < K) {
        const double app = JA[cur][p][p], aqq = JA[cur][q][q], apq = JA[cur][p][q];
        if (jac_offdiag_live(apq, app, aqq, floor2)) {
          // tan(2 phi) = 2 a_pq / (a_qq - a_pp), |phi| <= pi / 4:
          // c = (r + |d|) / sqrt(2 r (r + |d|)), s = sgn(d) e / sqrt(2 r (r + |d|))
          const double dd = aqq - app, e = 2.0 * apq;
          const double r2 = fma(dd, dd, e * e);
          const double rr = r2 * rsqrt(r2);
          const double ad = fabs(dd);
          const double iw = rsqrt(2.0 * rr * (rr + ad));
          c = (rr + ad) * iw;
          sn = (dd >= 0.0 ? e : -e) * iw;
          rot = true;
        }
      }
      jal[p] = c; jbe[p] = -sn; jmt[p] = rot ? q : p;
      jal[q] = c; jbe[q] = sn;  jmt[q] = rot ? p : q;
    }
    __syncthreads();
    // untested rounds count as unconverged
    bool bad = it % kJacTestEvery != 0;
    if (own) {
      const double aij = JA[cur][i][j];
      if (!bad) bad = i != j && jac_offdiag_live(aij, JA[cur][i][i], JA[cur][j][j], floor2);
      const double ai = jal[i], bi = jbe[i], aj = jal[j], bj = jbe[j];
      const int mi = jmt[i], mj = jmt[j];
      double v;
      if (mi == j && mi != i) {
        v = 0.0;                           // the rotated pair's off-diagonal
      } else {
        const double t1 = (ai * aj) * aij;
        const double t2 = (ai * bj) * JA[cur][i][mj];
        const double t3 = (bi * aj) * JA[cur][mi][j];
        const double t4 = (bi * bj) * JA[cur][mi][mj];
        v = (t1 + (t2 + t3)) + t4;
      }
      JA[cur ^ 1][i][j] = v;
      JV[cur ^ 1][i][j] = fma(bj, JV[cur][i][mj], aj * JV[cur][i][j]);
    }
    // a tested round's input already met the criterion: nothing was rotated
    conv = !__syncthreads_or(bad);
    if (!conv) cur ^= 1;
  }
  if (own && i == j) d[i] = JA[cur][i][i];
  if (own) V[i][j] = JV[cur][i][j];
  __syncthreads();
  return conv;
}

// In-place Cholesky B = L L^T of a symmetric n x n matrix (lower triangle
// and diagonal become L); idiag[k] = 1 / L[k][k].  false (uniformly across
// the CTA) when a pivot is not above piv_min: the basis is too close to
// dependent for Cholesky-based orthonormalisation.  Right-looking, one
// barrier per column: at step k each thread (i, j), k < j <= i, applies
// B[i][j] -= B[i][k] B[j][k] / d_k with column k and the pivot d_k already
// final; the columns are scaled by d_k^-1/2 at the end.  Loops, not
// unrolled code: each step runs once, so straight-line code would be bound
// by instruction fetch.
// (The CTA has one thread per element of a kMaxBasis x kMaxBasis matrix:
// thread t owns (t / kMaxBasis, t % kMaxBasis), a compile-time divisor.)
__device__ bool cta_chol(double (*B)[LDA], double* idiag, int n, double piv_min) {
  const int t = threadIdx.x, i = t / kMaxBasis, j = t % kMaxBasis;
  for (int k = 0; k < n; ++k) {
    const double pk = B[k][k];
    if (!(pk > piv_min)) return false;               // the same value in every thread
    const double rp = rsqrt(pk);
    if (k < j && j <= i && i < n) B[i][j] = fma(-B[i][k] * (rp * rp), B[j][k], B[i][j]);
    __syncthreads();
  }
  if (t < n) idiag[t] = rsqrt(B[t][t]);
  __syncthreads();
  if (j <= i && i < n) B[i][j] *= idiag[j];
  __syncthreads();
  return true;
}

// T <- L^-1 T (forward substitution, n x nc), L the lower triangle of B and
// idiag = 1 / diag(L); one barrier per row.
__device__ void cta_forward(double (*T)[LDA], double (*B)[LDA], const double* idiag, int n, int nc) {
  const int t = threadIdx.x, i = t / kMaxBasis, j = t % kMaxBasis;
  for (int l = 0; l + 1 < n; ++l) {
    if (i > l && i < n && j < nc) T[i][j] = fma(-B[i][l] * idiag[l], T[l][j], T[i][j]);
    __syncthreads();
  }
  if (i < n && j < nc) T[i][j] *= idiag[i];
  __syncthreads();
}

// Rayleigh-Ritz: the m smallest eigenpairs of G_K c = theta G_M c (n x n).
// Both Grams are scaled by D = diag(G_M)^-1/2.  Fast path: Cholesky
// D G_M D = L L^T (pivots above kCholPivot, i.e. a well-conditioned basis)
// and the standard problem L^-1 (D G_K D) L^-T.  Otherwise the SVQB form
// (Stathopoulos & Wu, SIAM J. Sci. Comput. 23 (2002)): D G_M D is
// eigendecomposed, directions with eigenvalue below drop_tol * max are
// discarded, and the standard problem is solved in the remaining
// M-orthonormal basis.  One CTA, one thread per matrix element.
// Outputs: C (n x m, row-major), theta (m), info[0] = kept rank (or -1; -2
// for non-finite input).
constexpr double kCholPivot = 1e-8;

__global__ void __launch_bounds__(kEigThreads) k_small_eig(int n, int m, const double* __restrict__ GK,
                                                          const double* __restrict__ GM, double drop_tol, double* C,
                                                          double* theta, int* info) {
  __shared__ double A[kMaxBasis][LDA], B[kMaxBasis][LDA], V[kMaxBasis][LDA], Z[kMaxBasis][LDA];
  __shared__ double JA[2][kMaxBasis][LDA], JV[2][kMaxBasis][LDA];   // Jacobi work buffers
  __shared__ double D[kMaxBasis], ev[kMaxBasis], idg[kMaxBasis];
  __shared__ int keep[kMaxBasis], order[kMaxBasis];
  __shared__ int kr;
  const int tid = threadIdx.x;
  {
    // non-finite Gram entries (a NaN / Inf density or start block): info -2
    bool bad = false;
    for (int w = tid; w < n * n; w += blockDim.x) bad = bad || !isfinite(GK[w]) || !isfinite(GM[w]);
    if (__syncthreads_or(bad)) {
      if (tid == 0) info[0] = -2;
      return;
    }
  }
  if (tid < n) {
    const double b = GM[tid * n + tid];
    D[tid] = b > 0.0 ? rsqrt(b) : 0.0;
  }
  __syncthreads();
  for (int w = tid; w < n * n; w += blockDim.x) {
    const int i = w / n, j = w % n;
    A[i][j] = 0.5 * (GK[i * n + j] + GK[j * n + i]) * D[i] * D[j];
    B[i][j] = 0.5 * (GM[i * n + j] + GM[j * n + i]) * D[i] * D[j];
  }
  __syncthreads();
  const bool chol = cta_chol(B, idg, n, kCholPivot);
  bool ok = true;
  int K = n;
  if (chol) {
    // Z <- L^-1 (forward substitution on the identity, one barrier per row),
    // then A <- L^-1 A L^-T as two dense products of one step each; thread
    // (i, j) forms element (i, j) and element (j, i) of V L^-T in the same
    // order and stores their mean, so A stays exactly symmetric.  Z is kept
    // for the back-transformation of the eigenvectors (one more product).
    const int ti = tid / kMaxBasis, tj = tid % kMaxBasis;
    const bool te = ti < n && tj < n;
    if (te) Z[ti][tj] = ti == tj ? 1.0 : 0.0;
    __syncthreads();
    cta_forward(Z, B, idg, n, n);
    if (te) {                                              // V = L^-1 A
      double acc = 0.0;
      for (int k = 0; k <= ti; ++k) acc = fma(Z[ti][k], A[k][tj], acc);
      V[ti][tj] = acc;
    }
    __syncthreads();
    if (te) {
      double a1 = 0.0, a2 = 0.0;
      for (int k = 0; k <= tj; ++k) a1 = fma(V[ti][k], Z[tj][k], a1);
      for (int k = 0; k <= ti; ++k) a2 = fma(V[tj][k], Z[ti][k], a2);
      A[ti][tj] = 0.5 * (a1 + a2);
    }
    __syncthreads();
  } else {
    for (int w = tid; w < n * n; w += blockDim.x) {       // B was overwritten by the failed Cholesky
      const int i = w / n, j = w % n;
      B[i][j] = 0.5 * (GM[i * n + j] + GM[j * n + i]) * D[i] * D[j];
    }
    __syncthreads();
    ok = cta_jacobi(B, JA, JV, V, ev, n);
    if (tid == 0) {
      double bmax = 0.0;
      for (int i = 0; i < n; ++i) bmax = fmax(bmax, ev[i]);
      int k = 0;
      for (int i = 0; i < n; ++i)
        if (ev[i] > drop_tol * bmax) keep[k++] = i;
      kr = k;
    }
    __syncthreads();
    K = kr;
    for (int w = tid; w < n * K; w += blockDim.x) {        // Z = V[:, keep] / sqrt(lambda)
      const int i = w / K, a = w % K;
      Z[i][a] = V[i][keep[a]] / sqrt(ev[keep[a]]);
    }
    __syncthreads();
    for (int w = tid; w < n * K; w += blockDim.x) {        // V <- A Z
      const int i = w / K, a = w % K;
      double s = 0.0;
      for (int j = 0; j < n; ++j) s = fma(A[i][j], Z[j][a], s);
      V[i][a] = s;
    }
    __syncthreads();
    for (int w = tid; w < K * K; w += blockDim.x) {        // B <- Z^T V
      const int a = w / K, b = w % K;
      double s = 0.0;
      for (int j = 0; j < n; ++j) s = fma(Z[j][a], V[j][b], s);
      B[a][b] = s;
    }
    __syncthreads();
    for (int w = tid; w < K * K; w += blockDim.x) {
      const int a = w / K, b = w % K;
      A[a][b] = 0.5 * (B[a][b] + B[b][a]);
    }
    __syncthreads();
  }
  ok = cta_jacobi(A, JA, JV, V, ev, K) && ok;
  if (tid < K) {                                           // ascending order (ties by index)
    const double e = ev[tid];
    int rank = 0;
    for (int j = 0; j < K; ++j) rank += (ev[j] < e || (ev[j] == e && j < tid)) ? 1 : 0;
    order[rank] = tid;
  }
  if (tid == 0) info[0] = (K >= m && ok) ? K : -1;
  __syncthreads();
  if (K < m || !ok) return;
  if (tid < m) theta[tid] = ev[order[tid]];
  if (chol) {
    // C = D L^-T U[:, order[:m]] (Z holds L^-1, lower triangular)
    for (int w = tid; w < n * m; w += blockDim.x) {
      const int i = w / m, k = w % m, col = order[k];
      double acc = 0.0;
      for (int l = i; l < n; ++l) acc = fma(Z[l][i], V[l][col], acc);
      C[i * m + k] = D[i] * acc;
    }
  } else {
    for (int w = tid; w < n * m; w += blockDim.x) {        // C = D Z U[:, order[:m]]
      const int i = w / m, k = w % m;
      double s = 0.0;
      for (int a = 0; a < K; ++a) s = fma(Z[i][a], V[a][order[k]], s);
      C[i * m + k] = D[i] * s;
    }
  }
}


// ---------------------------------------------------------------------------
// block update: Xn = S C, Pn = S[:, nb:] C[nb:, :] for S, KS, MS
// ---------------------------------------------------------------------------
// One thread per (node, block in {S, KS, MS}, output half): the X half
// accumulates all ncols input columns, the P half the columns from nb on
// (two threads with nb accumulators each rather than one with 2 nb: half
// the registers, twice the threads in flight); the input node records
// stream in as whole (coalesced) 4-component loads, the outputs are stored
// with a zero 4th component.
template <typename T>
__global__ void __launch_bounds__(128) k_lob_update(int NN, int nb, int ncols, ColMap cols, long long vs,
                                                    const T* __restrict__ S, const T* __restrict__ KS,
                                                    const T* __restrict__ MS, const double* __restrict__ C,
                                                    T* S2, T* KS2, T* MS2, int only) {
  using V4 = typename Vec4<T>::type;
  __shared__ T sC[kMaxBasis * 8];
  for (int i = threadIdx.x; i < ncols * nb; i += blockDim.x) sC[i] = T(C[i]);
  __syncthreads();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (only >= 0 ? 3LL : 6LL) * NN) return;
  const int n = int(t % NN);
  const int b = int((t / NN) % 3);
  // 0: X = S C, 1: P = S[:, nb:] C[nb:, :] (`only` >= 0: that half alone)
  const int half = only >= 0 ? only : int(t / (3LL * NN));
  const T* src = b == 0 ? S : b == 1 ? KS : MS;
  T* dst = b == 0 ? S2 : b == 1 ? KS2 : MS2;
  const int j0 = half ? nb : 0;
  T x[8][3];
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) x[k][c] = T(0);
#pragma unroll
  for (int j = 0; j < kMaxBasis; ++j) {
    if (j >= j0 && j < ncols) {
      const V4 v = reinterpret_cast<const V4*>(src + cols.col[j] * vs)[n];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k < nb) {
          const T cf = sC[j * nb + k];
          x[k][0] = fma(cf, v.x, x[k][0]); x[k][1] = fma(cf, v.y, x[k][1]); x[k][2] = fma(cf, v.z, x[k][2]);
        }
      }
    }
  }
  T* out = dst + (half ? 2 * nb : 0) * vs;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k < nb) {
      V4 o;
      o.x = x[k][0]; o.y = x[k][1]; o.z = x[k][2]; o.w = T(0);
      reinterpret_cast<V4*>(out + k * vs)[n] = o;
    }
  }
}

template <typename T>
static void launch_lob_update(int NN, int nb, int ncols, const ColMap& cols, long long vs, const T* S, const T* KS,
                              const T* MS, const double* C, T* S2, T* KS2, T* MS2, cudaStream_t s, int only = -1) {
  const long long threads = (only >= 0 ? 3LL : 6LL) * NN;
  k_lob_update<T><<<int((threads + 127) / 128), 128, 0, s>>>(NN, nb, ncols, cols, vs, S, KS, MS, C, S2, KS2, MS2,
                                                             only);
  count_launch();
}

static ColMap identity_cols() {
  ColMap m;
  for (int k = 0; k < 24; ++k) m.col[k] = k;
  return m;
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct LobBufs {
  void* S[2];
  void* KS[2];
  void* MS[2];
};

template <typename T>
static inline T* vec(void* base, int j, long long vs) {
  return reinterpret_cast<T*>(base) + j * vs;
}

static int lob_small_eig(Ctx& c, int n, int m, double drop, cudaStream_t s, const double* GK = nullptr,
                         const double* GM = nullptr) {
  if (!GK) GK = c.gram;
  if (!GM) GM = c.gram + 576;
  double* C = c.gram + 2 * 576;
  double* th = c.gram + 3 * 576;
  int* info = c.status_m;
  k_small_eig<<<1, kEigThreads, 0, s>>>(n, m, GK, GM, drop, C, th, info);
  count_launch();
  return 0;
}

int lobpcg_run(Ctx& c, bool f64, int nmodes, int nb, double* X64, double* lam, double tol, int maxiter,
               int precond, int inner_iters, double inner_rtol, int* iters_out, double* resid_out, double* floor_out,
               cudaStream_t s);

// Implementation templated on the vector type.
template <typename T>
static int lobpcg_impl(Ctx& c, int nmodes, int nb, double* X64, double* lam, double tol, int maxiter, int precond,
                       int inner_iters, double inner_rtol, int* iters_out, double* resid_out, double* floor_out,
                       cudaStream_t s) {
  const bool f64 = sizeof(T) == 8;
  const long long vs = (long long)c.g.NN * 4;
  const int NN = c.g.NN;
  const long long blk = 3LL * c.max_modes * vs;   // one S / KS / MS block (elements)
  T* base = f64 ? reinterpret_cast<T*>(c.lw64 + 3 * (long long)c.max_modes * vs)
                : reinterpret_cast<T*>(c.lw32);
  LobBufs B;
  for (int q = 0; q < 2; ++q) {
    B.S[q] = base + (3 * q + 0) * blk;
    B.KS[q] = base + (3 * q + 1) * blk;
    B.MS[q] = base + (3 * q + 2) * blk;
  }
  const double drop = f64 ? 1e-12 : 1e-9;
  double* GK = c.gram;
  double* GM = c.gram + 576;
  double* C = c.gram + 2 * 576;
  double* th = c.gram + 3 * 576;
  double* rn = c.gram + 3 * 576 + 32;
  int* info = c.status_m;
  const int rblocks = 2 * c.num_sms;
  int cur = 0;
  if (precond == 2 && mg_ensure(c, s)) return -2;
  cudaStreamWaitEvent(s, c.lob_pev, 0);        // a P half still running from an earlier call
  // X <- X64 (first nb vectors), KX, MX
  launch_convert(X64, true, B.S[cur], f64, (long long)nb * vs, s);
  if (launch_matvec_km(c, f64, B.S[cur], B.KS[cur], B.MS[cur], nb, s)) return -2;
  // initial Rayleigh-Ritz on X alone
  launch_gram2_cols(c, f64, B.S[cur], B.KS[cur], B.MS[cur], identity_cols(), nb, GK, GM, s, c.gram_part_m);
  lob_small_eig(c, nb, nb, drop, s);
  const ColMap ident = identity_cols();
  launch_lob_update<T>(NN, nb, nb, ident, vs, (T*)B.S[cur], (T*)B.KS[cur], (T*)B.MS[cur], C, (T*)B.S[cur ^ 1],
                       (T*)B.KS[cur ^ 1], (T*)B.MS[cur ^ 1], s);
  cur ^= 1;
  int it = 0;
  double hr[16];
  double hth[8];
  int hinfo = 0;
  cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  if (hinfo == -2) { c.last_error = "LOBPCG: non-finite values in the initial block's products"; return -4; }
  if (hinfo < 0) { c.last_error = "LOBPCG: initial block is rank deficient"; return -3; }
  bool conv = false;
  // K X, M X, K P, M P follow the update recurrence (S C) between refreshes.
  // The recurrence mixes in K W, whose norm is up to lambda_max / lambda_1
  // times that of K X, so its rounding error grows relative to the small
  // wanted residuals; recomputing the products every kLobRefresh iterations
  // (and before convergence is accepted) bounds that drift.
  auto refresh = [&]() -> int {
    cudaStreamWaitEvent(s, c.lob_pev, 0);      // P of this iterate (side stream)
    void* S = B.S[cur];
    if (launch_matvec_km(c, f64, S, B.KS[cur], B.MS[cur], nb, s)) return -2;
    const T* P = vec<T>(S, 2 * nb, vs);
    if (launch_matvec_km(c, f64, P, vec<T>(B.KS[cur], 2 * nb, vs), vec<T>(B.MS[cur], 2 * nb, vs), nb, s)) return -2;
    return 0;
  };
  // Soft locking (as scipy.sparse.linalg.lobpcg's active mask): a wanted
  // column whose residual is below tol leaves the search space [W, P] but
  // stays in X, so later Rayleigh-Ritz steps still refine it.  Tiny residual
  // columns otherwise make the basis ill-conditioned and stall the slowest
  // (lowest) modes.  Guard columns (j >= nmodes) are never locked.
  bool locked[8] = {false, false, false, false, false, false, false, false};
  double rres[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int act[8];
  ColMap wslot;
  auto active_map = [&]() -> int {   // W_j of active column j goes to vector nb + k
    int k = 0;
    for (int j = 0; j < 24; ++j) wslot.col[j] = -1;
    for (int j = 0; j < nb; ++j)
      if (!locked[j]) { act[k] = j; wslot.col[j] = nb + k; ++k; }
    return k;
  };
  double worst = 0.0;
  bool finite = true;
  // The host reads each iteration's residual norms one iteration late: the
  // residual kernel of iteration k copies its norms (and the rank word of
  // the Rayleigh-Ritz step before it) into a pinned slot and records an
  // event; the host launches the rest of iteration k, then waits for that
  // event only when it prepares iteration k + 1, so the GPU always has
  // queued work and the host never drains the stream.  Locking, restart and
  // stopping decisions therefore act one iteration later than they were
  // observed.  Slots 0 / 1 alternate; slot 2 is for synchronous reads.
  LobSlot* hp = reinterpret_cast<LobSlot*>(c.lob_pin);
  LobSlot* hp_dev = reinterpret_cast<LobSlot*>(c.lob_pin_dev);
  // with the single-V-cycle preconditioner the residual kernel also writes
  // the multigrid right-hand sides (FP32 W of the active columns, zero
  // padding up to the cycle's block size)
  const bool w32_out = precond == 2 && inner_iters <= 1;
  auto launch_resid = [&](int slot) {
    const T* dinv = nullptr;
    if (precond == 0) dinv = f64 ? (const T*)c.dinvK64 : (const T*)c.dinvK32;
    int na_now = 0;
    for (int j = 0; j < nb; ++j) na_now += wslot.col[j] >= 0 ? 1 : 0;
    const int R32 = na_now <= 1 ? 1 : na_now <= 2 ? 2 : na_now <= 4 ? 4 : 8;
    k_lob_resid<T><<<rblocks, 256, 0, s>>>(NN, nb, vs, (T*)B.KS[cur], (T*)B.MS[cur], th, dinv, (T*)B.S[cur],
                                           wslot, c.gram_part_m, c.counters_m, rn,
                                           w32_out ? mg_rhs(c, 1) : nullptr, na_now, R32, info, hp_dev + slot);
    count_launch();
    cudaEventRecord(c.lob_ev[slot], s);
  };
  auto read_resid = [&](int slot) -> int {
    if (cudaEventSynchronize(c.lob_ev[slot]) != cudaSuccess) { c.last_error = "LOBPCG: CUDA error"; return -2; }
    worst = 0.0;
    finite = true;
    hinfo = hp[slot].info;
    for (int j = 0; j < 8; ++j) hth[j] = hp[slot].th[j];
    for (int j = 0; j < nmodes; ++j) {
      const double r = sqrt(hp[slot].r[2 * j]) / fmax(sqrt(hp[slot].r[2 * j + 1]), 1e-300);
      if (!isfinite(r)) finite = false;
      worst = fmax(worst, r);
      rres[j] = r;
      if (resid_out) resid_out[j] = r;
    }
    return 0;
  };
  auto residual = [&]() -> int {       // synchronous: launch and read at once
    launch_resid(2);
    return read_resid(2);
  };
  double best = INFINITY;
  int restarts = 0, ncols_prev = 0;
  double best_res[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int it_best = 0;
  bool use_best = false;
  bool have_best = false;                      // X6 holds the best iterate
  double* X6 = c.lw64;                         // holds the best iterate (free until the final step)
  int pending = -1;                            // slot of a residual launched but not yet read
  // Bookkeeping on the residual of the iterate before the current one (in
  // S[cur ^ 1] until this iteration's update).  Returns 1 to stop the
  // iteration, < 0 on error; sets drop_p for a restart.
  bool drop_p = false;
  auto observe = [&](int itk) -> int {
    if (!finite) { c.last_error = "LOBPCG: non-finite residual"; return -4; }
    if (hinfo == -2) { c.last_error = "LOBPCG: non-finite Rayleigh-Ritz matrices"; return -4; }
    if (hinfo < 0) { c.last_error = "LOBPCG: Rayleigh-Ritz basis rank deficient"; return -3; }
    // the Rayleigh-Ritz step before that iterate dropped directions (SVQB):
    // the basis had become ill-conditioned, so the next one leaves P out
    if (hinfo > 0 && hinfo < ncols_prev) drop_p = true;
    if (worst < best) {
      best = worst;
      it_best = itk;
      for (int j = 0; j < nmodes; ++j) best_res[j] = rres[j];
      // the iterate itself is kept only once it could be returned or
      // restarted from (a 5.5 MB copy on the 2 mm arm)
      if (worst < kLobKeepBelow) {
        cudaMemcpyAsync(X6, B.S[cur ^ 1], sizeof(double) * nb * vs, cudaMemcpyDeviceToDevice, s);
        have_best = true;
      }
    } else if (best < kLobNearFloor && worst > kLobRestartGrowth * best && restarts < kLobMaxRestarts) {
      // the residual grew well past the best iterate: continue from the best
      // iterate with fresh products and without P
      ++restarts;
      cudaMemcpyAsync(B.S[cur], X6, sizeof(double) * nb * vs, cudaMemcpyDeviceToDevice, s);
      if (launch_matvec_km(c, f64, B.S[cur], B.KS[cur], B.MS[cur], nb, s)) return -2;
      for (int j = 0; j < nmodes; ++j) locked[j] = false;
      drop_p = true;
    } else if (best < kLobNearFloor &&
               (worst > kLobDiverge * best || itk - it_best >= std::max(kLobStall, it_best))) {
      use_best = true;
      return 1;
    }
    return 0;
  };
  int ncols_at[2] = {nb, nb};                  // basis size of each iteration's Rayleigh-Ritz step
  for (it = 0; it < maxiter; ++it) {
    const bool fresh = it > 0 && it % kLobRefresh == 0;
    if (fresh && refresh()) return -2;
    if (pending >= 0) {
      if (read_resid(pending)) return -2;      // iteration it - 1 (rank word of the step before it)
      pending = -1;
      ncols_prev = it >= 2 ? ncols_at[(it - 2) & 1] : nb;
      bool all = true;
      for (int j = 0; j < nmodes; ++j) {
        if (!locked[j] && rres[j] <= tol) locked[j] = true;
        all = all && locked[j];
      }
      bool confirmed_open = false;
      if (all && finite) {                     // confirm on fresh products of the current iterate
        if (!fresh && refresh()) return -2;
        active_map();
        if (residual()) return -2;
        bool reopened = false;
        for (int j = 0; j < nmodes; ++j)
          if (!(rres[j] <= tol)) { locked[j] = false; reopened = true; }
        if (!reopened) { conv = true; break; }
        if (!finite) { c.last_error = "LOBPCG: non-finite residual"; return -4; }
        confirmed_open = true;
      }
      if (!confirmed_open) {
        const int o = observe(it - 1);
        if (o < 0) return o;
        if (o > 0) break;
      }
    }
    int na = active_map();
    launch_resid(it & 1);
    pending = it & 1;
#ifdef TOF_LOB_TRACE
    fprintf(stderr, "lobpcg it %d rank %d active %d fresh %d worst(prev) %.3e res", it, hinfo, na, int(fresh), worst);
    for (int j = 0; j < nmodes; ++j) fprintf(stderr, " %.2e", rres[j]);
    fprintf(stderr, " theta0 %.10e\n", hth[0]);
#endif
    T* W = vec<T>(B.S[cur], nb, vs);
    const int R = na <= 1 ? 1 : na <= 2 ? 2 : na <= 4 ? 4 : 8;
    if (precond == 2 && inner_iters <= 1) {
      // W <- V-cycle(W): the FP32 multigrid approximation of K^-1
      // (the right-hand sides were written by the residual kernel)
      if (mg_ensure(c, s)) return -2;
      if (mg_vcycle(c, R, s, 1)) return -2;
      launch_convert(mg_out(c, 1), false, W, f64, (long long)na * vs, s);
    } else if (precond == 2) {
      // inner_iters multigrid cycles as a stationary iteration on K e = W:
      // e <- e + B (W - K e), all in FP32 (the FP32 LOBPCG work area holds
      // the kept right-hand side and the accumulated correction)
      if (mg_ensure(c, s)) return -2;
      float* r32 = mg_rhs(c, 1);
      float* e32 = mg_out(c, 1);
      float* rk = c.lw32;
      float* ek = c.lw32 + 8 * vs;
      if (R > na) cudaMemsetAsync(rk, 0, sizeof(float) * R * vs, s);
      launch_convert(W, f64, rk, false, (long long)na * vs, s);
      cudaMemcpyAsync(r32, rk, sizeof(float) * R * vs, cudaMemcpyDeviceToDevice, s);
      if (mg_vcycle(c, R, s, 1)) return -2;
      cudaMemcpyAsync(ek, e32, sizeof(float) * R * vs, cudaMemcpyDeviceToDevice, s);
      for (int cyc = 1; cyc < inner_iters; ++cyc) {
        if (launch_matvec(c, 0, false, ek, r32, R, rk, s)) return -2;
        if (mg_vcycle(c, R, s, 1)) return -2;
        launch_add_f32(R * vs, e32, ek, s);
      }
      launch_convert(ek, false, W, f64, (long long)na * vs, s);
    } else if (precond == 1) {
      // W <- (inexact) K^-1 W by block PCG (FP32)
      const size_t pblk = (size_t)c.max_rhs * vs;
      double* b64 = c.pw64 + 6 * pblk;
      float* d32 = c.pw32 + 9 * pblk;
      cudaMemsetAsync(b64, 0, sizeof(double) * R * vs, s);
      launch_convert(W, f64, b64, true, (long long)na * vs, s);
      cudaMemsetAsync(d32, 0, sizeof(float) * R * vs, s);
      if (pcg_std32(c, b64, d32, R, inner_rtol, inner_iters, s)) return -2;
      launch_convert(d32, false, W, f64, (long long)na * vs, s);
    }
    // K W, M W: one launch for the R >= na vectors when they stay inside the
    // W block (the columns beyond na are never read)
    if (launch_matvec_km(c, f64, W, vec<T>(B.KS[cur], nb, vs), vec<T>(B.MS[cur], nb, vs), R <= nb ? R : na, s))
      return -2;
    // basis [X, W_active, P_active]
    ColMap cols;
    int ncols = 0;
    for (int j = 0; j < nb; ++j) cols.col[ncols++] = j;
    for (int k = 0; k < na; ++k) cols.col[ncols++] = nb + k;
    if (it > 0 && !drop_p)
      for (int k = 0; k < na; ++k) cols.col[ncols++] = 2 * nb + act[k];
    for (int k = ncols; k < 24; ++k) cols.col[k] = 0;
    drop_p = false;
    ncols_at[it & 1] = ncols;
    cudaStreamWaitEvent(s, c.lob_pev, 0);      // P, K P, M P of this iterate
    launch_gram2_cols(c, f64, B.S[cur], B.KS[cur], B.MS[cur], cols, ncols, GK, GM, s, c.gram_part_m);
    // keep a full-basis problem for tof_time_kernel: the first one, then
    // one every 16 iterations (a 9 KB copy), so it comes from the late,
    // well-conditioned iterations that make up most of a solve
    if (ncols == 3 * nb && (c.lob_last_n != ncols || (it & 15) == 15)) {
      cudaMemcpyAsync(c.gram + 10 * 576, GK, sizeof(double) * 2 * 576, cudaMemcpyDeviceToDevice, s);
      c.lob_last_n = ncols;
      c.lob_last_m = nb;
    }
    lob_small_eig(c, ncols, nb, drop, s);
    // the P half of the update on the side stream: the next iteration needs
    // only X, K X, M X until its Gram matrices (which wait for it)
    cudaEventRecord(c.lob_cev, s);
    cudaStreamWaitEvent(c.lob_side, c.lob_cev, 0);
    launch_lob_update<T>(NN, nb, ncols, cols, vs, (T*)B.S[cur], (T*)B.KS[cur], (T*)B.MS[cur], C,
                         (T*)B.S[cur ^ 1], (T*)B.KS[cur ^ 1], (T*)B.MS[cur ^ 1], c.lob_side, 1);
    cudaEventRecord(c.lob_pev, c.lob_side);
    launch_lob_update<T>(NN, nb, ncols, cols, vs, (T*)B.S[cur], (T*)B.KS[cur], (T*)B.MS[cur], C,
                         (T*)B.S[cur ^ 1], (T*)B.KS[cur ^ 1], (T*)B.MS[cur ^ 1], s, 0);
    cur ^= 1;
  }
  cudaStreamWaitEvent(s, c.lob_pev, 0);        // the last P half, before anything reads the buffers
  if (pending >= 0 && !conv && !use_best) {    // the last iterate's residual, not yet read
    if (read_resid(pending)) return -2;
    ncols_prev = it >= 2 ? ncols_at[(it - 2) & 1] : nb;
    const int o = observe(it - 1);
    if (o < 0) return o;
  }
  if (iters_out) *iters_out = it;
  if (!conv && it >= maxiter && worst > best && have_best) use_best = true;
  if (use_best && resid_out)
    for (int j = 0; j < nmodes; ++j) resid_out[j] = best_res[j];
  // final FP64 Rayleigh-Ritz on fresh FP64 products of X6 (the best iterate,
  // or the current one)
  double* KX6 = c.lw64 + (long long)c.max_modes * vs;
  double* MX6 = c.lw64 + 2LL * c.max_modes * vs;
  if (!use_best) cudaMemcpyAsync(X6, B.S[cur], sizeof(double) * nb * vs, cudaMemcpyDeviceToDevice, s);
  if (launch_matvec_km(c, true, X6, KX6, MX6, nb, s)) return -2;
  // (its Gram matrices go to slots 8 / 9)
  launch_gram2_cols(c, true, X6, KX6, MX6, ident, nb, c.gram + 8 * 576, c.gram + 9 * 576, s, c.gram_part_m);
  lob_small_eig(c, nb, nb, 1e-14, s, c.gram + 8 * 576, c.gram + 9 * 576);
  // X64 = X6 C: all nb Ritz vectors of the final step, the nmodes wanted
  // ones first (the rest warm-start the guard columns of the next solve)
  {
    double* out = X64;
    // reuse the update kernel: S = X6 (ncols = nb), P part unused -> KS2/MS2 scratch
    double* scratch = c.lw64 + 3LL * c.max_modes * vs;   // FP64 LOBPCG area (free in mixed mode)
    if (f64) scratch = (double*)B.S[cur ^ 1];
    launch_lob_update<double>(NN, nb, nb, ident, vs, X6, KX6, MX6, C, scratch, scratch + 3LL * c.max_modes * vs,
                              scratch + 6LL * c.max_modes * vs, s);
    cudaMemcpyAsync(out, scratch, sizeof(double) * nb * vs, cudaMemcpyDeviceToDevice, s);
    // rounding floor of each returned residual: eps ||(|K| + theta M)|x|||
    // / ||K x|| (M has no negative entries); the current-iterate buffers are
    // free by now
    double* ax = (double*)B.S[cur];
    double* y = (double*)B.KS[cur];
    double* mx = (double*)B.MS[cur];
    launch_abs64((long long)nmodes * vs, out, ax, s);
    if (launch_matvec(c, 2, true, ax, y, nmodes, nullptr, s)) return -2;
    if (launch_matvec(c, 1, true, ax, mx, nmodes, nullptr, s)) return -2;
    k_add_scaled_cols<<<int((4LL * NN * nmodes + 255) / 256), 256, 0, s>>>(4LL * NN, nmodes, th, mx, y);
    count_launch();
    launch_gram(c, true, y, nmodes, y, nmodes, c.gram + 6 * 576, s, c.gram_part_m);
    launch_gram(c, true, scratch + 3LL * c.max_modes * vs, nmodes, scratch + 3LL * c.max_modes * vs, nmodes,
                c.gram + 6 * 576 + 64, s, c.gram_part_m);
  }
  double gfl[2][64];
  cudaMemcpyAsync(gfl, c.gram + 6 * 576, sizeof(gfl), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hth, th, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { c.last_error = "LOBPCG: CUDA error"; return -2; }

  if (hinfo == -2) { c.last_error = "LOBPCG: non-finite final products"; return -4; }
  if (hinfo < 0) { c.last_error = "LOBPCG: final block rank deficient"; return -3; }
  for (int j = 0; j < nmodes; ++j) lam[j] = hth[j];
  // converged: every wanted residual at tol, or at a small multiple of its
  // FP64 rounding floor where that lies above tol (the lowest modes of soft
  // SIMP designs, eps lambda_max / lambda_1 ~ 1e-6)
  bool at_floor = true;
  for (int j = 0; j < nmodes; ++j) {
    const double kx = sqrt(gfl[1][j * nmodes + j]);
    const double fl = kx > 0.0 ? 2.220446049250313e-16 * sqrt(gfl[0][j * nmodes + j]) / kx : 0.0;
    if (floor_out) floor_out[j] = fl;
    const double r = use_best ? best_res[j] : rres[j];
    if (!(r <= std::max(tol, kLobFloorFactor * fl))) at_floor = false;
  }
  return (conv || at_floor) ? 0 : 1;
}

// The block vectors are FP64 in both modes: FP32 block vectors (with FP64
// Gram matrices and Rayleigh-Ritz) stalled at residual ~1 on the SIMP arm and
// cantilever (the K X / M X recurrences drift by eps_32 * cond), so the mixed
// mode puts FP32 where it is safe, in the multigrid preconditioner.
int lob_launch_rayleigh_ritz(Ctx& c, cudaStream_t s, int* n) {
  if (c.lob_last_n < 1) { c.last_error = "no LOBPCG iteration has run on this context"; return -1; }
  *n = c.lob_last_n;
  return lob_small_eig(c, c.lob_last_n, c.lob_last_m, 1e-12, s, c.gram + 10 * 576, c.gram + 11 * 576);
}

int lobpcg_run(Ctx& c, bool f64, int nmodes, int nb, double* X64, double* lam, double tol, int maxiter,
               int precond, int inner_iters, double inner_rtol, int* iters_out, double* resid_out, double* floor_out,
               cudaStream_t s) {
  if (!f64) precond = 2;
  return lobpcg_impl<double>(c, nmodes, nb, X64, lam, tol, maxiter, precond, inner_iters, inner_rtol, iters_out,
                             resid_out, floor_out, s);
}

// Load every kernel of this file now (CUDA loads device functions lazily,
// at first use, and a first use in the middle of a solve stalls it).
void preload_kernels_lobpcg() {
  auto touch = [](auto f) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(f));
  };
  touch(k_add_scaled_cols); touch(k_lob_resid<double>); touch(k_small_eig); touch(k_lob_update<double>);
}

}  // namespace tof

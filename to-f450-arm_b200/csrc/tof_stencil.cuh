// Matrix-free hex8 operator on the structured voxel grid (sm_100a).
//
// The reference assembles K = sum_e f_e Ke and M = sum_e m_e Me as COO->CSR
// (src/fem.py:311-398, 576 entries per element).  Here the product y = A x is
// formed per NODE without assembly: for node n and each of its 27 neighbours
// n+d, the 3x3 coupling block is the sum over the (1..8) elements containing
// both nodes of f_e * Ke[3 ln : 3 ln + 3, 3 lm : 3 lm + 3], where ln / lm are the
// local corner indices of n and n+d in that element.  That is 64 (element,
// corner) pairs = 576 FMAs per node to form the blocks, shared by all R
// right-hand sides, plus 27 * 9 FMAs per node and right-hand side to apply
// them.  No atomics, deterministic, and the fixed-DOF restriction
// K[free][:, free] (src/fem.py:437-438, 540) is a mask on the output.
//
// A CTA owns a TX*TY*TZ node tile.  Its input is the tile plus a one-node halo
// of the R vectors, fetched by one 5-D TMA load (coordinates start at the
// tile origin - 1; the TMA unit zero-fills whatever lies outside the grid, so
// the grid boundary needs no special case).  Element factors of the
// (TX+1)(TY+1)(TZ+1) elements touching the tile and the 64 Ke blocks live in
// shared memory next to it.
#pragma once

#include "tof_common.cuh"

namespace tof {

// Ke / Me stored as 64 3x3 blocks, block (ln, lm) at [(ln*8+lm)*12], rows
// padded to 4 so a row is one vector load.
constexpr int kKeBlockStride = 12;
constexpr int kKeBlocksLen = 64 * kKeBlockStride;

struct TileGeom {
  int i0, j0, k0;      // tile origin (node coords)
  int HX, HY, HZ;      // halo box dims (T + 2)
  int EX, EY, EZ;      // element box dims (T + 1)
};

__device__ __forceinline__ TileGeom tile_geom(const Grid& g, int t) {
  TileGeom tg;
  const int tix = t % g.ntx, tiy = (t / g.ntx) % g.nty, tiz = t / (g.ntx * g.nty);
  tg.i0 = tix * g.TX; tg.j0 = tiy * g.TY; tg.k0 = tiz * g.TZ;
  tg.HX = g.TX + 2; tg.HY = g.TY + 2; tg.HZ = g.TZ + 2;
  tg.EX = g.TX + 1; tg.EY = g.TY + 1; tg.EZ = g.TZ + 1;
  return tg;
}

// Bytes of one halo box of R node4 vectors.
template <typename T>
__host__ __device__ inline unsigned halo_bytes(const Grid& g, int R) {
  return unsigned(R) * (g.TX + 2) * (g.TY + 2) * (g.TZ + 2) * 4u * unsigned(sizeof(T));
}

// Stage element factors of the elements touching the tile into smem (zero
// outside the grid).  Factors are read-only for the lifetime of a launch.
template <typename T>
__device__ __forceinline__ void load_factor_tile(const Grid& g, const TileGeom& tg, const T* __restrict__ fe,
                                                 T* sf) {
  const int n = tg.EX * tg.EY * tg.EZ;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int ex = idx % tg.EX, ey = (idx / tg.EX) % tg.EY, ez = idx / (tg.EX * tg.EY);
    const int gx = tg.i0 - 1 + ex, gy = tg.j0 - 1 + ey, gz = tg.k0 - 1 + ez;
    T f = T(0);
    if (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz)
      f = __ldg(fe + (size_t(gz) * g.ny + gy) * g.nx + gx);
    sf[idx] = f;
  }
}

template <typename T>
__device__ __forceinline__ void load_ke_blocks(const T* __restrict__ keb, T* sKe) {
  for (int i = threadIdx.x; i < kKeBlocksLen; i += blockDim.x) sKe[i] = __ldg(keb + i);
}

// One node's y = A x for R vectors, from the staged tiles.  (tx,ty,tz) is the
// node's position inside the tile.  acc is overwritten.
template <typename T, int R>
__device__ __forceinline__ void stencil_node(const T* __restrict__ sx, const TileGeom& tg,
                                             const T* __restrict__ sf, const T* __restrict__ sKe, int tx,
                                             int ty, int tz, T (&acc)[R][3]) {
  using V4 = typename Vec4<T>::type;
  const int hsy = tg.HX, hsz = tg.HX * tg.HY, hsr = tg.HX * tg.HY * tg.HZ;
  const int fsy = tg.EX, fsz = tg.EX * tg.EY;
  // the 8 element factors around the node: fr[c+1][b+1][a+1] for the
  // element whose lowest corner sits at node offset (a, b, c), a,b,c in {-1,0}
  T fr[2][2][2];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) fr[c][b][a] = sf[(tz + c) * fsz + (ty + b) * fsy + (tx + a)];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r][0] = acc[r][1] = acc[r][2] = T(0);
  const V4* xv4 = reinterpret_cast<const V4*>(sx);
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        T C[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) C[q] = T(0);
#pragma unroll
        for (int c = (dz > 0 ? 0 : -1); c <= (dz < 0 ? -1 : 0); ++c)
#pragma unroll
          for (int b = (dy > 0 ? 0 : -1); b <= (dy < 0 ? -1 : 0); ++b)
#pragma unroll
            for (int a = (dx > 0 ? 0 : -1); a <= (dx < 0 ? -1 : 0); ++a) {
              const T f = fr[c + 1][b + 1][a + 1];
              const int ln = local_node(-a, -b, -c);
              const int lm = local_node(dx - a, dy - b, dz - c);
              const V4* kb = reinterpret_cast<const V4*>(sKe + (ln * 8 + lm) * kKeBlockStride);
#pragma unroll
              for (int rr = 0; rr < 3; ++rr) {
                const V4 kr = kb[rr];
                C[rr * 3 + 0] = fma(f, kr.x, C[rr * 3 + 0]);
                C[rr * 3 + 1] = fma(f, kr.y, C[rr * 3 + 1]);
                C[rr * 3 + 2] = fma(f, kr.z, C[rr * 3 + 2]);
              }
            }
        const int off = (tz + 1 + dz) * hsz + (ty + 1 + dy) * hsy + (tx + 1 + dx);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const V4 x = xv4[r * hsr + off];
#pragma unroll
          for (int rr = 0; rr < 3; ++rr)
            acc[r][rr] = fma(C[rr * 3 + 0], x.x, fma(C[rr * 3 + 1], x.y, fma(C[rr * 3 + 2], x.z, acc[r][rr])));
        }
      }
}

// Node of this thread inside the tile; false if the thread has no node.
__device__ __forceinline__ bool thread_node(const Grid& g, const TileGeom& tg, int& tx, int& ty, int& tz,
                                            int& n) {
  const int t = threadIdx.x;
  tx = t % g.TX; ty = (t / g.TX) % g.TY; tz = t / (g.TX * g.TY);
  const int i = tg.i0 + tx, j = tg.j0 + ty, k = tg.k0 + tz;
  n = (k * g.NY + j) * g.NX + i;
  return tz < g.TZ && i < g.NX && j < g.NY && k < g.NZ;
}

// The TMA-staged halo tile of a node4 vector block at node (tx,ty,tz) itself.
template <typename T>
__device__ __forceinline__ typename Vec4<T>::type halo_center(const T* sx, const TileGeom& tg, int r, int tx,
                                                              int ty, int tz) {
  using V4 = typename Vec4<T>::type;
  const int hsr = tg.HX * tg.HY * tg.HZ;
  return reinterpret_cast<const V4*>(sx)[r * hsr + ((tz + 1) * tg.HY + (ty + 1)) * tg.HX + (tx + 1)];
}

}  // namespace tof

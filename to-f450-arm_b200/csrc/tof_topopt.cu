// Density filter, OC update and SIMP glue kernels (sm_100a).
#include <math.h>

#include "tof_internal.h"

namespace tof {

// ---------------------------------------------------------------------------
// Masked normalised convolution filter (src/topopt.py:44-58):
//   num = conv(field * mask, w), den = conv(mask, w)   (zero padding)
//   out = num / max(den, 1e-12) on the mask, 0 elsewhere.
// conv is the true convolution of scipy.ndimage.convolve:
//   out_i = sum_q w_q in_{i - (q - c)}.
// Element grids are x-fastest (e = (ez*ny + ey)*nx + ex).
//
// mode 0: forward (as above).
// mode 1: exact transpose of mode 0 as a linear map of the field:
//   out_j = mask_j sum_q w_q mask_{j+d} g_{j+d} / den_{j+d},  d = q - c.
// mode 2: forward, then every active element outside the mask set to 1 (the
//   physical density composite of src/topopt.py:273-278); `fill` marks them.
// ---------------------------------------------------------------------------
struct FilterTap {
  int dx, dy, dz, pad;
  double w;
};

__global__ void k_filter(int nx, int ny, int nz, const FilterTap* __restrict__ taps, int ntaps,
                         const uint8_t* __restrict__ mask, const double* __restrict__ den,
                         const uint8_t* __restrict__ fill, const double* __restrict__ in, double* out, int mode) {
  extern __shared__ FilterTap st[];
  for (int i = threadIdx.x; i < ntaps; i += blockDim.x) st[i] = taps[i];
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int NE = nx * ny * nz;
  if (e >= NE) return;
  const int ex = e % nx, ey = (e / nx) % ny, ez = e / (nx * ny);
  double r = 0.0;
  if (mask[e]) {
    double s = 0.0;
    const int sgn = mode == 1 ? 1 : -1;
    for (int t = 0; t < ntaps; ++t) {
      const int x = ex + sgn * st[t].dx, y = ey + sgn * st[t].dy, z = ez + sgn * st[t].dz;
      if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
      const int j = (z * ny + y) * nx + x;
      if (!mask[j]) continue;
      if (mode == 1) s += st[t].w * in[j] / fmax(den[j], 1e-12);
      else s += st[t].w * in[j];
    }
    r = mode == 1 ? s : s / fmax(den[e], 1e-12);
  } else if (mode == 2 && fill && fill[e]) {
    r = 1.0;
  }
  out[e] = r;
}

// den = conv(mask, w) over the whole grid
__global__ void k_filter_den(int nx, int ny, int nz, const FilterTap* __restrict__ taps, int ntaps,
                             const uint8_t* __restrict__ mask, double* den) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nx * ny * nz) return;
  const int ex = e % nx, ey = (e / nx) % ny, ez = e / (nx * ny);
  double s = 0.0;
  for (int t = 0; t < ntaps; ++t) {
    const int x = ex - taps[t].dx, y = ey - taps[t].dy, z = ez - taps[t].dz;
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
    if (mask[(z * ny + y) * nx + x]) s += taps[t].w;
  }
  den[e] = s;
}

void launch_filter_den(int nx, int ny, int nz, const void* taps, int ntaps, const uint8_t* mask, double* den,
                       cudaStream_t s) {
  const int NE = nx * ny * nz;
  k_filter_den<<<ceil_div(NE, 256), 256, 0, s>>>(nx, ny, nz, (const FilterTap*)taps, ntaps, mask, den);
  count_launch();
}

void launch_filter(int nx, int ny, int nz, const void* taps, int ntaps, const uint8_t* mask, const double* den,
                   const uint8_t* fill, const double* in, double* out, int mode, cudaStream_t s) {
  const int NE = nx * ny * nz;
  k_filter<<<ceil_div(NE, 256), 256, ntaps * sizeof(FilterTap), s>>>(nx, ny, nz, (const FilterTap*)taps, ntaps,
                                                                      mask, den, fill, in, out, mode);
  count_launch();
}

size_t filter_tap_bytes() { return sizeof(FilterTap); }

// ---------------------------------------------------------------------------
// OC update with bisection on the Lagrange multiplier (src/topopt.py:190-214):
//   x_new = max(0.001, max(x - move, min(1, min(x + move, x sqrt(|dc| / (l V_e))))))
//   l in [1e-9, 1e9], bisect while (l2 - l1) / (l1 + l2) > 1e-4 on
//   sum(x_new) * V_e > target.  The result is x_new of the last midpoint, as
//   in the reference.  One CTA; the sum is a fixed-order block reduction.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_oc(int n, const double* __restrict__ x, const double* __restrict__ dc,
                                             double V_e, double target, double move, double* x_new,
                                             int* n_bisect) {
  __shared__ double red[32];
  double l1 = 1e-9, l2 = 1e9, lmid = 0.5 * (l1 + l2);
  int nb = 0;
  while ((l2 - l1) / (l1 + l2) > 1e-4) {
    lmid = 0.5 * (l1 + l2);
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double xi = x[i];
      const double t = xi * sqrt(fabs(dc[i]) / (lmid * V_e));
      s += fmax(0.001, fmax(xi - move, fmin(1.0, fmin(xi + move, t))));
    }
    double v[1] = {s};
    block_sum<1>(v, red);
    if (v[0] * V_e > target) l1 = lmid;
    else l2 = lmid;
    ++nb;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double xi = x[i];
    const double t = xi * sqrt(fabs(dc[i]) / (lmid * V_e));
    x_new[i] = fmax(0.001, fmax(xi - move, fmin(1.0, fmin(xi + move, t))));
  }
  if (threadIdx.x == 0 && n_bisect) *n_bisect = nb;
}

void launch_oc(int n, const double* x, const double* dc, double V_e, double target, double move, double* x_new,
               int* n_bisect, cudaStream_t s) {
  k_oc<<<1, 1024, 0, s>>>(n, x, dc, V_e, target, move, x_new, n_bisect);
  count_launch();
}

// ---------------------------------------------------------------------------
// SIMP glue, fused per element:
//   compliance sensitivity (src/topopt.py:296-306):
//     c += w_l f_e ce_le,   dc_e += w_l (-p (1-emin) rho^(p-1) ce_le)
//   eigenvalue sensitivity (src/fem.py:492-526):
//     dlam_e = ((1-emin) p max(rho,1e-9)^(p-1) qK_e - lam m'(rho_e) qM_e) / vMv
// Partial sums of c (and of m(rho) qM for vMv) per CTA go to `part`.
// ---------------------------------------------------------------------------
__global__ void k_compliance_sens(int NE, int nlc, const double* __restrict__ w, const double* __restrict__ rho,
                                  const double* __restrict__ ce, const uint8_t* __restrict__ active, SimpParams sp,
                                  double* dc, double* part) {
  __shared__ double red[32];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double csum = 0.0;
  if (e < NE) {
    double d = 0.0;
    if (active[e]) {
      const double r = rho[e];
      const double f = sp.emin + (1.0 - sp.emin) * pow(r, sp.penal);
      const double g = -sp.penal * (1.0 - sp.emin) * pow(r, sp.penal - 1.0);
      for (int l = 0; l < nlc; ++l) {
        const double c = ce[(size_t)l * NE + e];
        csum += w[l] * f * c;
        d += w[l] * (g * c);
      }
    }
    dc[e] = d;
  }
  double v[1] = {csum};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void k_sum_partials(int n, const double* __restrict__ part, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  double v[1] = {s};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) *out = v[0];
}

void launch_compliance_sens(int NE, int nlc, const double* w, const double* rho, const double* ce,
                            const uint8_t* active, SimpParams sp, double* dc, double* part, double* c_out,
                            cudaStream_t s) {
  const int blocks = ceil_div(NE, 256);
  k_compliance_sens<<<blocks, 256, 0, s>>>(NE, nlc, w, rho, ce, active, sp, dc, part);
  count_launch();
  k_sum_partials<<<1, 256, 0, s>>>(blocks, part, c_out);
  count_launch();
}

__global__ void k_mass_quad(int NE, const double* __restrict__ rho, const double* __restrict__ qM,
                            const uint8_t* __restrict__ active, SimpParams sp, double* part) {
  __shared__ double red[32];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (e < NE && active[e]) {
    const double r = rho[e];
    const double m = (r >= sp.mass_threshold) ? r
                                              : sp.mass_threshold * pow(fmax(r, 0.0) / sp.mass_threshold, sp.mass_q);
    s = m * qM[e];
  }
  double v[1] = {s};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void k_eig_sens(int NE, const double* __restrict__ rho, const double* __restrict__ qK,
                           const double* __restrict__ qM, const uint8_t* __restrict__ active, SimpParams sp,
                           double lam, const double* __restrict__ vMv_bulk, double vMv_tip, double* out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NE) return;
  if (!active[e]) { out[e] = 0.0; return; }
  double vMv = *vMv_bulk + vMv_tip;
  if (vMv <= 0.0) vMv = 1.0;
  const double r = rho[e];
  const double fKp = (1.0 - sp.emin) * sp.penal * pow(fmax(r, 1e-9), sp.penal - 1.0);
  const double fMp = (r >= sp.mass_threshold)
                         ? 1.0
                         : sp.mass_q * pow(fmax(r, 0.0) / sp.mass_threshold, sp.mass_q - 1.0);
  out[e] = (fKp * qK[e] - lam * fMp * qM[e]) / vMv;
}

void launch_eig_sens(int NE, const double* rho, const double* qK, const double* qM, const uint8_t* active,
                     SimpParams sp, double lam, double vMv_tip, double* out, double* part, double* scal,
                     cudaStream_t s) {
  const int blocks = ceil_div(NE, 256);
  k_mass_quad<<<blocks, 256, 0, s>>>(NE, rho, qM, active, sp, part);
  count_launch();
  k_sum_partials<<<1, 256, 0, s>>>(blocks, part, scal);
  count_launch();
  k_eig_sens<<<blocks, 256, 0, s>>>(NE, rho, qK, qM, active, sp, lam, scal, vMv_tip, out);
  count_launch();
}

// Load every kernel of this file now (CUDA loads device functions lazily,
// at first use, and a first use in the middle of a solve stalls it).
void preload_kernels_topopt() {
  auto touch = [](auto f) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(f));
  };
  touch(k_filter); touch(k_filter_den); touch(k_oc); touch(k_compliance_sens); touch(k_sum_partials);
  touch(k_mass_quad); touch(k_eig_sens);
}

}  // namespace tof

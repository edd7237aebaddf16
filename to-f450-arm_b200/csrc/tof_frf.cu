// Modal-superposition frequency response at selected DOFs (sm_100a).
//
// The reference evaluates, for one DOF d and a geometric grid of frequencies,
//   |H_dd(f)| = | sum_k v_k[d]^2 / ((w_k^2 - w^2) + 2 i zeta w_k w) |
// with proportional modal damping zeta (src/plotting.py:378-399).  Here one
// thread per (DOF, frequency) sums the modes in complex FP64 arithmetic, for
// any number of DOFs at once.
#include <math.h>

#include "tof_internal.h"

namespace tof {

__global__ void k_modal_frf(long long ndof, int m, const double* __restrict__ V, const double* __restrict__ fk_hz,
                            long long npts, const double* __restrict__ f_hz, double zeta, double* out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= ndof * npts) return;
  const long long d = t / npts, i = t % npts;
  const double w = 2.0 * M_PI * f_hz[i];
  double re = 0.0, im = 0.0;
  for (int k = 0; k < m; ++k) {
    const double wk = 2.0 * M_PI * fk_hz[k];
    const double v = V[d * m + k];
    const double a = wk * wk - w * w, b = 2.0 * zeta * wk * w;   // denominator a + i b
    const double s = v * v / (a * a + b * b);
    re = fma(s, a, re);
    im = fma(-s, b, im);
  }
  out[t] = hypot(re, im);
}

int launch_modal_frf(long long ndof, int m, const double* V, const double* fk_hz, long long npts, const double* f_hz,
                     double zeta, double* out, cudaStream_t s) {
  const long long n = ndof * npts;
  if (n <= 0) return 0;
  k_modal_frf<<<int((n + 255) / 256), 256, 0, s>>>(ndof, m, V, fk_hz, npts, f_hz, zeta, out);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace tof

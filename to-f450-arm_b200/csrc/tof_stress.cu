// Element stress recovery and the stress-life fatigue field (sm_100a).
//
// The reference computes, on the host, per active element
//   sigma_e = rho_e D B_c u_e            (src/fem.py:564-579, B_c = strain-
//                                         displacement matrix at the centre,
//                                         src/fem.py:153-176, linear rho scaling)
//   von Mises, largest principal stress   (src/fem.py:582-602)
// and, per element, a two-level fatigue cycle between the von Mises stresses
// of two load cases with the Goodman mean-stress correction and the PA12 S-N
// curve (src/fatigue.py:24-112).  Here both are element-local kernels on the
// device-resident displacements: one thread per (element, vector).
#include <math.h>

#include "tof_internal.h"

namespace tof {

struct StressArgs {
  Grid g;
  int nvec;
  const double* rho;          // [NE] full grid
  const uint8_t* active;      // [NE]
  double B[6 * 24];           // row-major, Voigt rows xx yy zz xy yz xz
  double D[6 * 6];
  double* sigma;              // [nvec][NE][6] or null
  double* vm;                 // [nvec][NE] or null
  double* smax;               // [nvec][NE] or null
};

// von Mises equivalent of a Voigt stress (src/fem.py:582-589)
__device__ __forceinline__ double von_mises6(const double* s) {
  const double a = s[0] - s[1], b = s[1] - s[2], c = s[2] - s[0];
  const double v = 0.5 * (a * a + b * b + c * c) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
  return sqrt(fmax(v, 0.0));
}

// Largest eigenvalue of the symmetric stress tensor (src/fem.py:592-602), by
// the closed-form trigonometric solution of the characteristic cubic
// (O. K. Smith, Comm. ACM 4(4):168, 1961).
__device__ __forceinline__ double principal_max6(const double* s) {
  const double a11 = s[0], a22 = s[1], a33 = s[2], a12 = s[3], a23 = s[4], a13 = s[5];
  const double p1 = a12 * a12 + a13 * a13 + a23 * a23;
  if (p1 == 0.0) return fmax(a11, fmax(a22, a33));
  const double q = (a11 + a22 + a33) / 3.0;
  const double d1 = a11 - q, d2 = a22 - q, d3 = a33 - q;
  const double p = sqrt((d1 * d1 + d2 * d2 + d3 * d3 + 2.0 * p1) / 6.0);
  const double ip = 1.0 / p;
  const double b11 = d1 * ip, b22 = d2 * ip, b33 = d3 * ip, b12 = a12 * ip, b23 = a23 * ip, b13 = a13 * ip;
  double r = 0.5 * (b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) + b13 * (b12 * b23 - b22 * b13));
  r = fmin(1.0, fmax(-1.0, r));
  return q + 2.0 * p * cos(acos(r) / 3.0);
}

template <typename T>
__global__ void __launch_bounds__(256) k_stress(StressArgs a, const T* __restrict__ u) {
  using V4 = typename Vec4<T>::type;
  const Grid& g = a.g;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)g.NE * a.nvec) return;
  const int e = int(t % g.NE), r = int(t / g.NE);
  double s[6] = {0, 0, 0, 0, 0, 0};
  if (a.active[e]) {
    const int ex = e % g.nx, ey = (e / g.nx) % g.ny, ez = e / (g.nx * g.ny);
    const V4* ur = reinterpret_cast<const V4*>(u + (size_t)r * g.NN * 4);
    double ue[24];
#pragma unroll
    for (int ln = 0; ln < 8; ++ln) {
      // local corner order of the reference: bottom face CCW, then top face
      const int ox = (ln == 1 || ln == 2 || ln == 5 || ln == 6), oy = (ln == 2 || ln == 3 || ln == 6 || ln == 7),
                oz = ln >= 4;
      const V4 v = ur[((ez + oz) * g.NY + (ey + oy)) * g.NX + (ex + ox)];
      ue[3 * ln] = double(v.x); ue[3 * ln + 1] = double(v.y); ue[3 * ln + 2] = double(v.z);
    }
    double eps[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 24; ++j) acc = fma(a.B[i * 24 + j], ue[j], acc);
      eps[i] = acc;
    }
    const double rho = a.rho[e];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) acc = fma(a.D[i * 6 + j], eps[j], acc);
      s[i] = rho * acc;
    }
  }
  if (a.sigma) {
    double* o = a.sigma + ((size_t)r * g.NE + e) * 6;
#pragma unroll
    for (int i = 0; i < 6; ++i) o[i] = s[i];
  }
  if (a.vm) a.vm[(size_t)r * g.NE + e] = von_mises6(s);
  if (a.smax) a.smax[(size_t)r * g.NE + e] = principal_max6(s);
}

__global__ void k_stress_invariants(long long n, const double* __restrict__ sigma, double* vm, double* smax) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) s[k] = sigma[i * 6 + k];
  if (vm) vm[i] = von_mises6(s);
  if (smax) smax[i] = principal_max6(s);
}

// ---------------------------------------------------------------------------
// Fatigue (src/fatigue.py).  The S-N curve of PA12 SLS at R = -1 (the
// reference's table, src/fatigue.py:20-21) is inverted to stress -> life by
// linear interpolation in log10-log10 space over the reversed table, ties of
// the repeated endurance stress nudged apart by 1e-12 (src/fatigue.py:38-56);
// the table is built on the host exactly as there.
// ---------------------------------------------------------------------------
constexpr int kSnPoints = 7;
struct SnTable {
  double xp[kSnPoints];   // log10 stress (MPa), increasing
  double fp[kSnPoints];   // log10 cycles
  double s_endurance;     // MPa, last table stress
  double s_top;           // MPa, first table stress
};

static SnTable sn_table() {
  static const double cycles[kSnPoints] = {1e2, 1e3, 1e4, 1e5, 1e6, 5e6, 1e7};
  static const double alt[kSnPoints] = {45.0, 38.0, 28.0, 20.0, 13.0, 12.0, 12.0};
  SnTable t;
  for (int i = 0; i < kSnPoints; ++i) {
    t.xp[i] = log10(alt[kSnPoints - 1 - i]);
    t.fp[i] = log10(cycles[kSnPoints - 1 - i]);
  }
  for (int i = 1; i < kSnPoints; ++i)
    if (t.xp[i] <= t.xp[i - 1]) t.xp[i] = t.xp[i - 1] + 1e-12;
  t.s_endurance = alt[kSnPoints - 1];
  t.s_top = alt[0];
  return t;
}

// np.interp(x, xp, fp, left=fp[0], right=fp[-1]) for the 7-point table
__device__ __forceinline__ double sn_interp(const SnTable& t, double x) {
  if (!(x >= t.xp[0])) return t.fp[0];
  if (x >= t.xp[kSnPoints - 1]) return t.fp[kSnPoints - 1];
  int j = 0;
#pragma unroll
  for (int k = 1; k < kSnPoints - 1; ++k)
    if (x >= t.xp[k]) j = k;
  const double slope = (t.fp[j + 1] - t.fp[j]) / (t.xp[j + 1] - t.xp[j]);
  double v = slope * (x - t.xp[j]) + t.fp[j];
  if (isnan(v)) v = slope * (x - t.xp[j + 1]) + t.fp[j + 1];
  return v;
}

// cycles to failure at an equivalent fully reversed stress s (Pa)
// (src/fatigue.py:24-65)
__device__ __forceinline__ double sn_life(const SnTable& t, double s_pa) {
  const double s = s_pa / 1e6;
  double life = pow(10.0, sn_interp(t, log10(s > 0.0 ? s : 1e-10)));
  if (s < t.s_endurance * 0.99) life = 1e9;
  if (s > t.s_top * 1.5) life = 1.0;
  return life;
}

// out rows: mean, alt, alt_eq, life, damage, factor of safety (src/fatigue.py:83-112)
__global__ void k_fatigue(long long n, SnTable t, const double* __restrict__ s1, const double* __restrict__ s2,
                          double uts, double s_design_pa, double* out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = s1[i], b = s2[i];
  const double peak = fmax(a, b), valley = fmin(a, b);
  const double mean = 0.5 * (peak + valley), alt = 0.5 * (peak - valley);
  const double denom = fmax(1.0 - fmax(mean, 0.0) / uts, 1e-6);      // Goodman (src/fatigue.py:68-80)
  const double eq = alt / denom;
  const double life = sn_life(t, eq);
  out[i] = mean;
  out[n + i] = alt;
  out[2 * n + i] = eq;
  out[3 * n + i] = life;
  out[4 * n + i] = 1.0 / fmax(life, 1.0);
  out[5 * n + i] = s_design_pa / fmax(eq, 1e-6);
}

__global__ void k_sn_life(long long n, SnTable t, const double* __restrict__ s, double* life) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) life[i] = sn_life(t, s[i]);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int launch_stress(Ctx& c, const double* B, const double* D, bool f64, const void* u, int nvec, const double* rho,
                  double* sigma, double* vm, double* smax, cudaStream_t s) {
  StressArgs a;
  a.g = c.g;
  a.nvec = nvec;
  a.rho = rho ? rho : c.rho;
  a.active = c.active;
  for (int i = 0; i < 144; ++i) a.B[i] = B[i];
  for (int i = 0; i < 36; ++i) a.D[i] = D[i];
  a.sigma = sigma; a.vm = vm; a.smax = smax;
  const long long n = (long long)c.g.NE * nvec;
  const int blocks = int((n + 255) / 256);
  if (f64) k_stress<double><<<blocks, 256, 0, s>>>(a, (const double*)u);
  else k_stress<float><<<blocks, 256, 0, s>>>(a, (const float*)u);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_stress_invariants(long long n, const double* sigma, double* vm, double* smax, cudaStream_t s) {
  if (n <= 0) return 0;
  k_stress_invariants<<<int((n + 255) / 256), 256, 0, s>>>(n, sigma, vm, smax);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_fatigue(long long n, const double* s1, const double* s2, double uts, double s_design_pa, double* out,
                   cudaStream_t s) {
  if (n <= 0) return 0;
  k_fatigue<<<int((n + 255) / 256), 256, 0, s>>>(n, sn_table(), s1, s2, uts, s_design_pa, out);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_sn_life(long long n, const double* sigma_eq, double* life, cudaStream_t s) {
  if (n <= 0) return 0;
  k_sn_life<<<int((n + 255) / 256), 256, 0, s>>>(n, sn_table(), sigma_eq, life);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace tof

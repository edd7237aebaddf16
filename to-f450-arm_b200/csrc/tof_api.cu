// C ABI of libtof: context management and the reference-facing entry points.
#include <math.h>
#include <stddef.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tof.h"
#include "tof_internal.h"
#include "tof_stencil.cuh"

namespace tof {
void launch_filter_den(int nx, int ny, int nz, const void* taps, int ntaps, const uint8_t* mask, double* den,
                       cudaStream_t s);
void launch_filter(int nx, int ny, int nz, const void* taps, int ntaps, const uint8_t* mask, const double* den,
                   const uint8_t* fill, const double* in, double* out, int mode, cudaStream_t s);
size_t filter_tap_bytes();
void launch_oc(int n, const double* x, const double* dc, double V_e, double target, double move, double* x_new,
               int* n_bisect, cudaStream_t s);
void launch_compliance_sens(int NE, int nlc, const double* w, const double* rho, const double* ce,
                            const uint8_t* active, SimpParams sp, double* dc, double* part, double* c_out,
                            cudaStream_t s);
void launch_eig_sens(int NE, const double* rho, const double* qK, const double* qM, const uint8_t* active,
                     SimpParams sp, double lam, double vMv_tip, double* out, double* part, double* scal,
                     cudaStream_t s);
int lobpcg_run(Ctx& c, bool f64, int nmodes, int nb, double* X64, double* lam, double tol, int maxiter,
               int precond, int inner_iters, double inner_rtol, int* iters_out, double* resid_out, double* floor_out,
               cudaStream_t s);

// ---------------------------------------------------------------------------
// tensor maps
// ---------------------------------------------------------------------------
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn get_encode() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  });
  return fn;
}

bool encode_node4_map(CUtensorMap* m, const void* base, const Grid& g, int R, bool f64, std::string* err) {
  EncodeFn enc = get_encode();
  if (!enc) { *err = "cuTensorMapEncodeTiled unavailable"; return false; }
  const cuuint64_t es = f64 ? 8 : 4;
  cuuint64_t dims[5] = {4, (cuuint64_t)g.NX, (cuuint64_t)g.NY, (cuuint64_t)g.NZ, (cuuint64_t)R};
  cuuint64_t strides[4] = {4 * es, 4 * es * g.NX, 4 * es * g.NX * g.NY, 4 * es * (cuuint64_t)g.NN};
  cuuint32_t box[5] = {4, (cuuint32_t)(g.TX + 2), (cuuint32_t)(g.TY + 2), (cuuint32_t)(g.TZ + 2), (cuuint32_t)R};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    *err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}

static int pow2ceil(int r) { return r <= 1 ? 1 : r <= 2 ? 2 : r <= 4 ? 4 : 8; }

std::atomic<long long>& launch_counter() {
  static std::atomic<long long> n{0};
  return n;
}
bool& capturing() {
  static thread_local bool f = false;
  return f;
}

}  // namespace tof

using namespace tof;

struct tof_ctx {
  Ctx c;
};

struct tof_filter {
  int nx, ny, nz, ntaps;
  void* taps;
  uint8_t* mask;
  uint8_t* fill;
  double* den;
};

static thread_local std::string g_create_error;

void tof::set_global_error(const std::string& msg) { g_create_error = msg; }

#define CUDA_TRY(expr)                                                    \
  do {                                                                    \
    cudaError_t _e = (expr);                                              \
    if (_e != cudaSuccess) {                                              \
      c.last_error = std::string(#expr) + ": " + cudaGetErrorString(_e); \
      return TOF_ERR_CUDA;                                                \
    }                                                                     \
  } while (0)

template <typename T>
static cudaError_t dalloc(Ctx& c, T** p, size_t n) {
  const size_t b = std::max<size_t>(n, 1) * sizeof(T);
  c.bytes += b;
  cudaError_t e = cudaMalloc((void**)p, b);
  if (e == cudaSuccess) e = cudaMemset(*p, 0, b);
  return e;
}

static void free_ctx(Ctx& c) {
  mg_destroy(c);
  for (cudaEvent_t& e : c.lob_ev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  if (c.lob_cev) { cudaEventDestroy(c.lob_cev); c.lob_cev = nullptr; }
  if (c.lob_pev) { cudaEventDestroy(c.lob_pev); c.lob_pev = nullptr; }
  if (c.lob_side) { cudaStreamDestroy(c.lob_side); c.lob_side = nullptr; }
  if (c.lob_pin) { cudaFreeHost(c.lob_pin); c.lob_pin = nullptr; }
  void* ptrs[] = {c.Ke64, c.Me64, c.keb64, c.meb64, c.kebabs64, c.keb32, c.meb32, c.active, c.fix, c.tip64, c.tip32,
                  c.fK64, c.fM64, c.fK32, c.fM32, c.rho, c.dK64, c.dM64, c.dinvK64, c.dinvK32, c.partials,
                  c.bar, c.status, c.scal, c.counters, c.pw32, c.pw64, c.lw32, c.lw64, c.gram, c.gram_part,
                  c.gram_part_m, c.counters_m, c.status_m, c.scal_m};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

// CUDA loads device functions lazily, at their first launch; a first launch
// in the middle of a solve (a block size reached only once soft locking has
// removed columns, say) then stalls that solve for tens of milliseconds.
// The first context created on each device loads every kernel up front.
static void preload_all_kernels(int dev) {
  static std::mutex mu;
  static bool done[64] = {};
  std::lock_guard<std::mutex> g(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  preload_kernels_core();
  preload_kernels_gmg();
  preload_kernels_lobpcg();
  preload_kernels_pcg();
  preload_kernels_topopt();
  cudaGetLastError();
  done[dev] = true;
}

extern "C" {

int tof_version(void) { return 100; }

long long tof_launch_count(void) { return launch_counter().load(); }

const char* tof_last_error(const tof_ctx* ctx) {
  if (!ctx) return g_create_error.c_str();
  static thread_local std::string copy;       // valid until this thread's next call
  copy = ctx->c.last_error.str();
  return copy.c_str();
}

int tof_ctx_create(int nx, int ny, int nz, const double h[3], const double Ke[576], const double Me[576],
                   const uint8_t* active, const uint8_t* fixed_dof, const double* tip_lump,
                   const tof_simp_params* simp, int max_rhs, int max_modes, const int tile[3], tof_ctx** out) {
  (void)h;
  if (!out || !Ke || !Me || !fixed_dof || nx < 1 || ny < 1 || nz < 1 || max_rhs < 1 || max_rhs > 8 ||
      max_modes < 1 || max_modes > 8) {
    g_create_error = "tof_ctx_create: invalid argument";
    return TOF_ERR_ARG;
  }
  int TX = 8, TY = 4, TZ = 4;
  if (tile) { TX = tile[0]; TY = tile[1]; TZ = tile[2]; }
  if (TX < 1 || TY < 1 || TZ < 1 || TX * TY * TZ > 256 || TX + 2 > 256 || TY + 2 > 256 || TZ + 2 > 256) {
    g_create_error = "tof_ctx_create: tile must have x*y*z <= 256";
    return TOF_ERR_ARG;
  }
  tof_ctx* h_ = new tof_ctx();
  Ctx& c = h_->c;
  c.g = make_grid(nx, ny, nz, TX, TY, TZ);
  if (simp) {
    c.sp.penal = simp->penal; c.sp.emin = simp->emin;
    c.sp.mass_threshold = simp->mass_threshold; c.sp.mass_q = simp->mass_q;
  }
  c.max_rhs = pow2ceil(std::max(max_rhs, max_modes));
  // the largest per-CTA shared memory any kernel of this context asks for:
  // the FP64 persistent PCG tile (two halo blocks of max_rhs vectors)
  {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t nfe = size_t(TX + 1) * (TY + 1) * (TZ + 1);
    size_t need = 2 * size_t(halo_bytes<double>(c.g, c.max_rhs)) + sizeof(double) * (kKeBlocksLen + nfe);
    need = ((need + 15) & ~size_t(15)) + sizeof(double) * 3 * c.max_rhs * 32 + 16;
    if (optin > 0 && need > size_t(optin)) {
      g_create_error = "tof_ctx_create: tile " + std::to_string(TX) + "x" + std::to_string(TY) + "x" +
                       std::to_string(TZ) + " needs " + std::to_string(need) + " B of shared memory per block with " +
                       std::to_string(c.max_rhs) + " vectors (limit " + std::to_string(optin) + " B)";
      delete h_;
      return TOF_ERR_ARG;
    }
  }
  c.max_modes = max_modes;
  const Grid& g = c.g;
  auto fail = [&](const std::string& m) {
    g_create_error = m;
    free_ctx(c);
    delete h_;
    return TOF_ERR_CUDA;
  };
  if (cudaGetDevice(&c.dev) != cudaSuccess) return fail("no CUDA device");
  preload_all_kernels(c.dev);
  cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.dev);

  // ---- host-side bookkeeping: active set, fixed + ghost DOFs, tip lump
  std::vector<uint8_t> act(g.NE, 1);
  if (active)
    for (int e = 0; e < g.NE; ++e) act[e] = active[e] ? 1 : 0;
  std::vector<uint8_t> used(g.NN, 0);
  for (int ez = 0; ez < nz; ++ez)
    for (int ey = 0; ey < ny; ++ey)
      for (int ex = 0; ex < nx; ++ex) {
        if (!act[(ez * ny + ey) * nx + ex]) continue;
        for (int oz = 0; oz < 2; ++oz)
          for (int oy = 0; oy < 2; ++oy)
            for (int ox = 0; ox < 2; ++ox) used[((ez + oz) * g.NY + ey + oy) * g.NX + ex + ox] = 1;
      }
  std::vector<uint8_t> fix(g.NN, 0);
  int nfree = 0;
  for (int n = 0; n < g.NN; ++n) {
    uint8_t f = 0;
    for (int q = 0; q < 3; ++q)
      if (fixed_dof[3 * (size_t)n + q] || !used[n]) f |= uint8_t(1u << q);
    fix[n] = f;
    nfree += 3 - __builtin_popcount(f);
  }
  c.n_free = nfree;
  c.host_fix = fix;
  std::vector<double> tip4((size_t)g.NN * 4, 0.0);
  std::vector<float> tip4f((size_t)g.NN * 4, 0.f);
  if (tip_lump)
    for (int n = 0; n < g.NN; ++n)
      for (int q = 0; q < 3; ++q)
        if (!((fix[n] >> q) & 1)) {
          tip4[4 * (size_t)n + q] = tip_lump[3 * (size_t)n + q];
          tip4f[4 * (size_t)n + q] = float(tip_lump[3 * (size_t)n + q]);
        }
  // 64-block layouts
  std::vector<double> kb(kKeBlocksLen, 0.0), mb(kKeBlocksLen, 0.0);
  std::vector<float> kbf(kKeBlocksLen, 0.f), mbf(kKeBlocksLen, 0.f);
  for (int ln = 0; ln < 8; ++ln)
    for (int lm = 0; lm < 8; ++lm)
      for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) {
          const int d = (ln * 8 + lm) * kKeBlockStride + r * 4 + q;
          const int s = (3 * ln + r) * 24 + 3 * lm + q;
          kb[d] = Ke[s]; mb[d] = Me[s];
          kbf[d] = float(Ke[s]); mbf[d] = float(Me[s]);
        }

  // ---- device memory (the only allocations of this context)
  const size_t NE = g.NE, NN = g.NN, V = NN * 4;
  const size_t R = c.max_rhs, MM = c.max_modes;
  c.partial_slots = 4 * c.num_sms;
  c.gram_blocks = 2 * c.num_sms;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  A(dalloc(c, &c.Ke64, 576)); A(dalloc(c, &c.Me64, 576));
  A(dalloc(c, &c.keb64, kKeBlocksLen)); A(dalloc(c, &c.meb64, kKeBlocksLen));
  A(dalloc(c, &c.kebabs64, kKeBlocksLen));
  A(dalloc(c, &c.keb32, kKeBlocksLen)); A(dalloc(c, &c.meb32, kKeBlocksLen));
  A(dalloc(c, &c.active, NE)); A(dalloc(c, &c.fix, NN));
  A(dalloc(c, &c.tip64, V)); A(dalloc(c, &c.tip32, V));
  A(dalloc(c, &c.fK64, NE)); A(dalloc(c, &c.fM64, NE)); A(dalloc(c, &c.fK32, NE)); A(dalloc(c, &c.fM32, NE));
  A(dalloc(c, &c.rho, NE));
  A(dalloc(c, &c.dK64, V)); A(dalloc(c, &c.dM64, V)); A(dalloc(c, &c.dinvK64, V)); A(dalloc(c, &c.dinvK32, V));
  A(dalloc(c, &c.partials, (size_t)c.partial_slots * 64));
  A(dalloc(c, &c.bar, 1)); A(dalloc(c, &c.status, 32)); A(dalloc(c, &c.scal, 256));
  A(dalloc(c, &c.counters, 16));
  A(dalloc(c, &c.pw32, 10 * R * V));
  A(dalloc(c, &c.pw64, 8 * R * V));
  A(dalloc(c, &c.lw32, 18 * MM * V));
  A(dalloc(c, &c.lw64, 21 * MM * V));
  A(dalloc(c, &c.gram, 12 * 576));
  A(dalloc(c, &c.gram_part, (size_t)c.gram_blocks * 1152));
  A(dalloc(c, &c.gram_part_m, (size_t)c.gram_blocks * 1152));
  A(dalloc(c, &c.counters_m, 16)); A(dalloc(c, &c.status_m, 16)); A(dalloc(c, &c.scal_m, 256));
  A(cudaHostAlloc(&c.lob_pin, 3 * 256, cudaHostAllocMapped));
  if (c.lob_pin) A(cudaHostGetDevicePointer(&c.lob_pin_dev, c.lob_pin, 0));
  for (cudaEvent_t& ev : c.lob_ev) A(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&c.lob_cev, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&c.lob_pev, cudaEventDisableTiming));
  A(cudaStreamCreateWithFlags(&c.lob_side, cudaStreamNonBlocking));
  if (e != cudaSuccess) return fail(std::string("tof_ctx_create: ") + cudaGetErrorString(e));
  if (mg_create(c, c.max_rhs)) return fail("tof_ctx_create: " + c.last_error.str());
  mg_capture_all(c);
  A(cudaMemcpy(c.Ke64, Ke, 576 * 8, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.Me64, Me, 576 * 8, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.keb64, kb.data(), kb.size() * 8, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.meb64, mb.data(), mb.size() * 8, cudaMemcpyHostToDevice));
  {
    std::vector<double> kabs(kb.size());
    for (size_t q = 0; q < kb.size(); ++q) kabs[q] = fabs(kb[q]);
    A(cudaMemcpy(c.kebabs64, kabs.data(), kabs.size() * 8, cudaMemcpyHostToDevice));
  }
  A(cudaMemcpy(c.keb32, kbf.data(), kbf.size() * 4, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.meb32, mbf.data(), mbf.size() * 4, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.active, act.data(), NE, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.fix, fix.data(), NN, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.tip64, tip4.data(), V * 8, cudaMemcpyHostToDevice));
  A(cudaMemcpy(c.tip32, tip4f.data(), V * 4, cudaMemcpyHostToDevice));
  if (e != cudaSuccess) return fail(std::string("tof_ctx_create: ") + cudaGetErrorString(e));
  // default density: solid everywhere active (src/fem.py:307-308)
  {
    std::vector<double> one(NE, 1.0);
    A(cudaMemcpy(c.rho, one.data(), NE * 8, cudaMemcpyHostToDevice));
    launch_factors(c, c.rho, 0);
    launch_diag(c, 0);
    A(cudaDeviceSynchronize());
  }
  if (e != cudaSuccess) return fail(std::string("tof_ctx_create: ") + cudaGetErrorString(e));
  *out = h_;
  return TOF_OK;
}

void tof_ctx_destroy(tof_ctx* ctx) {
  if (!ctx) return;
  cudaDeviceSynchronize();
  free_ctx(ctx->c);
  delete ctx;
}

int tof_ctx_set_wait_limit(tof_ctx* ctx, long long ns) {
  if (!ctx) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (ns < 1000 || ns > 60000000000LL) {
    c.last_error = "tof_ctx_set_wait_limit: the limit must be in [1 us, 60 s]";
    return TOF_ERR_ARG;
  }
  const unsigned long long w = (unsigned long long)ns;
  CUDA_TRY(cudaMemcpy(reinterpret_cast<char*>(c.bar) + offsetof(BarrierState, wait_ns), &w, sizeof(w),
                      cudaMemcpyHostToDevice));
  c.wait_ns = ns;
  return TOF_OK;
}

int tof_wait_selftest(tof_ctx* ctx, int extra_arrivals, void* stream) {
  if (!ctx || extra_arrivals < 0 || extra_arrivals > 1) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  cudaStream_t s = (cudaStream_t)stream;
  const int G = std::min(4, std::max(1, c.num_sms));
  CUDA_TRY(cudaMemsetAsync(c.bar, 0, kBarrierResetBytes, s));
  if (launch_barrier_selftest(c, G, G + extra_arrivals, s)) return TOF_ERR_CUDA;
  int err = 0;
  CUDA_TRY(cudaMemcpyAsync(&err, reinterpret_cast<char*>(c.bar) + offsetof(BarrierState, error), sizeof(int),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  // leave the barrier ready for the next persistent launch
  CUDA_TRY(cudaMemsetAsync(c.bar, 0, kBarrierResetBytes, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (err == ST_TIMEOUT) {
    c.last_error = "tof_wait_selftest: grid barrier wait budget expired";
    return TOF_ERR_TIMEOUT;
  }
  return err ? TOF_ERR_CUDA : TOF_OK;
}

long long tof_ctx_query(const tof_ctx* ctx, int what) {
  if (!ctx) return -1;
  const Ctx& c = ctx->c;
  switch (what) {
    case TOF_Q_NODES: return c.g.NN;
    case TOF_Q_ELEMS: return c.g.NE;
    case TOF_Q_FREE_DOFS: return c.n_free;
    case TOF_Q_TILE_X: return c.g.TX;
    case TOF_Q_TILE_Y: return c.g.TY;
    case TOF_Q_TILE_Z: return c.g.TZ;
    case TOF_Q_DEVICE_BYTES: return (long long)c.bytes;
    case TOF_Q_MAX_RHS: return c.max_rhs;
    case TOF_Q_MAX_MODES: return c.max_modes;
  }
  return -1;
}

int tof_set_density(tof_ctx* ctx, const double* rho, void* stream) {
  if (!ctx || !rho) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  cudaStream_t s = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(c.rho, rho, sizeof(double) * c.g.NE, cudaMemcpyDeviceToDevice, s));
  launch_factors(c, c.rho, s);
  launch_diag(c, s);
  mg_mark_dirty(c);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_set_tip_lump(tof_ctx* ctx, const double* tip_lump, void* stream) {
  if (!ctx) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t NN = c.g.NN;
  std::vector<double> t4(NN * 4, 0.0);
  std::vector<float> t4f(NN * 4, 0.f);
  if (tip_lump)
    for (size_t n = 0; n < NN; ++n)
      for (int q = 0; q < 3; ++q)
        if (!((c.host_fix[n] >> q) & 1)) {
          t4[4 * n + q] = tip_lump[3 * n + q];
          t4f[4 * n + q] = float(tip_lump[3 * n + q]);
        }
  CUDA_TRY(cudaMemcpyAsync(c.tip64, t4.data(), NN * 4 * 8, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(c.tip32, t4f.data(), NN * 4 * 4, cudaMemcpyHostToDevice, s));
  launch_diag(c, s);
  CUDA_TRY(cudaStreamSynchronize(s));   // host staging buffers go out of scope
  return TOF_OK;
}

int tof_pack(tof_ctx* ctx, const double* src, long long ld, void* dst, int dtype, int nvec, void* stream) {
  if (!ctx || !src || !dst || nvec < 1) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  launch_pack(c, src, ld, dst, dtype == TOF_F64, nvec, (cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_unpack(tof_ctx* ctx, const void* src, int dtype, double* dst, long long ld, int nvec, void* stream) {
  if (!ctx || !src || !dst || nvec < 1) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  launch_unpack(c, src, dtype == TOF_F64, dst, ld, nvec, (cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_matvec(tof_ctx* ctx, int op, int dtype, const void* x, void* y, int nvec, void* stream) {
  if (!ctx || !x || !y || nvec < 1 || (op != TOF_OP_K && op != TOF_OP_M)) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (launch_matvec(c, op, dtype == TOF_F64, x, y, nvec, nullptr, (cudaStream_t)stream)) return TOF_ERR_CUDA;
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_diag(tof_ctx* ctx, int op, double* out, void* stream) {
  if (!ctx || !out) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  CUDA_TRY(cudaMemcpyAsync(out, op == TOF_OP_K ? c.dK64 : c.dM64, sizeof(double) * 4 * c.g.NN,
                           cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return TOF_OK;
}

int tof_gram(tof_ctx* ctx, int dtype, const void* A, int na, const void* B, int nb, double* G, void* stream) {
  if (!ctx || !A || !B || !G || na < 1 || nb < 1 || na > 24 || nb > 24) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  launch_gram(c, dtype == TOF_F64, A, na, B, nb, G, (cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

// ---------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------
// rel[k] = ||b_k - K x_k|| / ||b_k|| recomputed in FP64, and the rounding
// floor of that residual, phi[k] = eps ||(|K| |x_k| + |b_k|)|| / ||b_k||:
// rounding the exact solution to FP64 alone leaves a residual up to
// eps |K| |x| (componentwise), so a true residual at or below phi is as
// small as FP64 can represent.  On soft SIMP designs |K||x| / |b| reaches
// 1e8, which puts phi above 1e-8 (a sparse LU solution then shows the same
// true residual).  Uses FP64 work slots 4, 5 and 7.
static int true_relres(Ctx& c, const double* b, const double* x, int R, double* rel, cudaStream_t s,
                       double* phi = nullptr) {
  const size_t V = (size_t)c.g.NN * 4;
  const size_t blk = (size_t)c.max_rhs * V;
  double* r64 = c.pw64 + 7 * blk;
  if (launch_matvec(c, 0, true, x, r64, R, b, s)) return TOF_ERR_CUDA;
  launch_gram(c, true, r64, R, r64, R, c.gram + 4 * 576, s);
  launch_gram(c, true, b, R, b, R, c.gram + 5 * 576, s);
  if (phi) {
    double* ax = c.pw64 + 5 * blk;
    double* y = c.pw64 + 4 * blk;
    launch_abs64((long long)R * V, x, ax, s);
    if (launch_matvec(c, 2, true, ax, y, R, nullptr, s)) return TOF_ERR_CUDA;
    launch_abs64((long long)R * V, b, ax, s);
    launch_axpy64((long long)R * V, ax, y, 1.0, s);
    launch_gram(c, true, y, R, y, R, c.gram + 7 * 576, s);
  }
  double G[3][64];
  CUDA_TRY(cudaMemcpyAsync(G[0], c.gram + 4 * 576, sizeof(double) * R * R, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(G[1], c.gram + 5 * 576, sizeof(double) * R * R, cudaMemcpyDeviceToHost, s));
  if (phi) CUDA_TRY(cudaMemcpyAsync(G[2], c.gram + 7 * 576, sizeof(double) * R * R, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int k = 0; k < R; ++k) {
    const double bn = sqrt(G[1][k * R + k]);
    rel[k] = bn > 0.0 ? sqrt(G[0][k * R + k]) / bn : 0.0;
    if (phi) phi[k] = bn > 0.0 ? 2.220446049250313e-16 * sqrt(G[2][k * R + k]) / bn : 0.0;
  }
  return TOF_OK;
}

// Status of one right-hand side after a PCG pass, given its true relative
// residual `rel` and the target max(rtol, rounding floor); sets `again`
// when the pass should be followed by a restart from the current x.  A
// pass that claims convergence above the target restarts (residual
// replacement).  So does a CG breakdown (p^T K p <= 0 in floating point):
// near the rounding floor the search direction is rounding noise and its
// energy can come out non-positive, and a restart recomputes the residual
// and the direction in FP64.  A breakdown at the target is convergence; one
// in the last allowed pass ends the solve not converged (the current x is
// the best one).
static int settle_pass(int status, double rel, double target, bool last, bool& again) {
  if (status == ST_BREAKDOWN) {
    if (rel <= target * 1.01) return ST_OK;
    if (last) return ST_NOT_CONVERGED;
    again = true;
    return ST_NOT_CONVERGED;
  }
  if (status == ST_OK && rel > target * 1.01) {
    again = true;
    return ST_NOT_CONVERGED;
  }
  return status;
}

int tof_pcg(tof_ctx* ctx, int mode, const double* b, double* x, int nrhs, double rtol, int maxiter,
            tof_solve_stats* stats, void* stream) {
  if (!ctx || !b || !x || nrhs < 1 || !(rtol > 0.0) || maxiter < 1) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (nrhs > c.max_rhs) { c.last_error = "tof_pcg: nrhs exceeds the context's max_rhs"; return TOF_ERR_ARG; }
  cudaStream_t s = (cudaStream_t)stream;
  const int R = pow2ceil(nrhs);
  const size_t V = (size_t)c.g.NN * 4;
  const size_t blk = (size_t)c.max_rhs * V;
  double* wx = c.pw64;            // slot 0: x
  double* wb = c.pw64 + 6 * blk;  // slot 6: b
  CUDA_TRY(cudaMemsetAsync(wb, 0, sizeof(double) * R * V, s));
  CUDA_TRY(cudaMemsetAsync(wx, 0, sizeof(double) * R * V, s));
  CUDA_TRY(cudaMemcpyAsync(wb, b, sizeof(double) * nrhs * V, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(wx, x, sizeof(double) * nrhs * V, cudaMemcpyDeviceToDevice, s));
  int st[16] = {0};
  double rel[8] = {0};
  double phi[8] = {0};
  int iters[8] = {0}, outer[8] = {0};
  int rc = TOF_OK;
  if (mode == TOF_MODE_FP64) {
    // SciPy's recurrence; when its recursive residual claims rtol but the
    // true residual (recomputed in FP64) exceeds max(rtol, rounding floor),
    // the iteration restarts from the current x (residual replacement), at
    // most kMaxRestarts times.  Right-hand sides already done restart from
    // their converged x and stop at once.
    constexpr int kMaxRestarts = 4;
    for (int o = 0; o <= kMaxRestarts; ++o) {
      const int budget = maxiter - *std::max_element(iters, iters + nrhs);
      if (budget <= 0) break;
      if (pcg_plain64(c, wb, wx, R, rtol, budget, nullptr, nullptr, nullptr, s)) return TOF_ERR_CUDA;
      int sto[16] = {0};
      CUDA_TRY(cudaMemcpyAsync(sto, c.status, sizeof(int) * 2 * R, cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      if (true_relres(c, wb, wx, R, rel, s, phi)) return TOF_ERR_CUDA;
      bool again = false;
      for (int k = 0; k < nrhs; ++k) {
        iters[k] += sto[R + k];
        outer[k] = o + 1;
        st[k] = settle_pass(sto[k], rel[k], std::max(rtol, phi[k]), o == kMaxRestarts, again);
      }
      if (!again) break;
    }
  } else if (mode == TOF_MODE_MIXED) {
    // FP64 PCG preconditioned by the FP32 multigrid V-cycle.  The recursive
    // residual drifts from the true one (by ~eps * cond); when it claims
    // convergence but the true residual b - K x does not meet rtol, the
    // iteration restarts from the current x (a restart recomputes r in FP64),
    // at most kMaxRestarts times.
    constexpr int kMaxRestarts = 4;
    int ist[8] = {0};
    for (int o = 0; o <= kMaxRestarts; ++o) {
      int it_o[8] = {0};
      const int budget = maxiter - *std::max_element(iters, iters + R);
      if (budget <= 0) break;
      if (pcg_mg64(c, wb, wx, R, rtol, budget, it_o, ist, s)) return TOF_ERR_CUDA;
      if (true_relres(c, wb, wx, R, rel, s, phi)) return TOF_ERR_CUDA;
      bool again = false;
      for (int k = 0; k < nrhs; ++k) {
        iters[k] += it_o[k];
        outer[k] = o + 1;
        st[k] = settle_pass(ist[k], rel[k], std::max(rtol, phi[k]), o == kMaxRestarts, again);
      }
      if (!again) break;
    }
  } else {
    // FP64 iterative refinement around the FP32 standard PCG
    double* r64 = c.pw64 + 7 * blk;
    float* d32 = c.pw32 + 9 * blk;
    double bn[8], rn[8];
    for (int k = 0; k < 8; ++k) st[k] = ST_NOT_CONVERGED;
    const int max_outer = 12;
    int budget = maxiter;
    for (int o = 0; o <= max_outer; ++o) {
      if (launch_matvec(c, 0, true, wx, r64, R, wb, s)) return TOF_ERR_CUDA;
      launch_gram(c, true, r64, R, r64, R, c.gram + 4 * 576, s);
      if (o == 0) launch_gram(c, true, wb, R, wb, R, c.gram + 5 * 576, s);
      double G[2][64];
      CUDA_TRY(cudaMemcpyAsync(G[0], c.gram + 4 * 576, sizeof(double) * R * R, cudaMemcpyDeviceToHost, s));
      if (o == 0)
        CUDA_TRY(cudaMemcpyAsync(G[1], c.gram + 5 * 576, sizeof(double) * R * R, cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      bool all = true;
      double need = 1.0;
      for (int k = 0; k < R; ++k) {
        if (o == 0) bn[k] = sqrt(G[1][k * R + k]);
        rn[k] = sqrt(G[0][k * R + k]);
        rel[k] = bn[k] > 0.0 ? rn[k] / bn[k] : 0.0;
        if (k < nrhs && !isfinite(rel[k])) { st[k] = ST_NONFINITE; continue; }
        if (k < nrhs && rel[k] > rtol) {
          all = false;
          need = std::min(need, rtol * bn[k] / rn[k]);
        } else if (k < nrhs) {
          st[k] = ST_OK;
        }
      }
      if (all || o == max_outer || budget <= 0) break;
      // inner tolerance: a bit below what the worst rhs still needs
      const double inner = std::min(0.1, std::max(2e-5, 0.3 * need));
      CUDA_TRY(cudaMemsetAsync(d32, 0, sizeof(float) * R * V, s));
      if (pcg_std32(c, r64, d32, R, inner, budget, s)) return TOF_ERR_CUDA;
      int ist[16];
      CUDA_TRY(cudaMemcpyAsync(ist, c.status, sizeof(int) * 2 * R, cudaMemcpyDeviceToHost, s));
      launch_add_f32_to_f64((long long)R * V, d32, wx, s);
      CUDA_TRY(cudaStreamSynchronize(s));
      int used = 0;
      for (int k = 0; k < nrhs; ++k) {
        iters[k] += ist[R + k];
        outer[k] += 1;
        used = std::max(used, ist[R + k]);
        if (ist[k] == ST_TIMEOUT) { c.last_error = "tof_pcg: grid barrier timed out"; return TOF_ERR_TIMEOUT; }
      }
      budget -= std::max(used, 1);
    }
  }
  CUDA_TRY(cudaMemcpyAsync(x, wx, sizeof(double) * nrhs * V, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int k = 0; k < nrhs; ++k) {
    if (st[k] == ST_TIMEOUT) { c.last_error = "tof_pcg: grid barrier timed out"; rc = TOF_ERR_TIMEOUT; }
    else if (st[k] < 0 && rc >= 0) rc = st[k];
    else if (st[k] == ST_NOT_CONVERGED && rc == TOF_OK) rc = TOF_NOT_CONVERGED;
    if (stats) {
      stats[k].status = st[k];
      stats[k].iters = iters[k];
      stats[k].outer = outer[k];
      stats[k].relres = rel[k];
      stats[k].floor = phi[k];
    }
  }
  return rc;
}

// ---------------------------------------------------------------------------
// kernel timing (diagnostics)
// ---------------------------------------------------------------------------
int tof_time_kernel(tof_ctx* ctx, int kernel, int level, int nvec, int reps, tof_kernel_timing* out, void* stream) {
  if (!ctx || !out || reps < 1 || reps > 1000 || !stream) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  cudaStream_t s = (cudaStream_t)stream;
  const int R = nvec;
  if (R != 1 && R != 2 && R != 4 && R != 8) { c.last_error = "tof_time_kernel: nvec must be 1, 2, 4 or 8"; return TOF_ERR_ARG; }
  const size_t V = (size_t)c.g.NN * 4;
  const size_t blk = (size_t)c.max_rhs * V;
  double bytes = 0.0, flops = 0.0;
  long long units = 0;
  int n_rr = 0;
  auto launch_once = [&]() -> int {
    switch (kernel) {
      case TOF_KERNEL_MATVEC_F32:
        if (R > c.max_rhs) return -1;
        units = c.g.NE;
        return launch_matvec(c, 0, false, c.pw32, c.pw32 + blk, R, nullptr, s);
      case TOF_KERNEL_MG_LEVEL_OP:
        return mg_launch_level_op(c, level, R, s, &units);
      case TOF_KERNEL_RAYLEIGH_RITZ:
        return lob_launch_rayleigh_ritz(c, s, &n_rr);
      case TOF_KERNEL_VCYCLE:
        units = c.g.NN;
        return mg_vcycle(c, R, s, 0);
    }
    c.last_error = "tof_time_kernel: unknown kernel";
    return -1;
  };
  if ((kernel == TOF_KERNEL_MG_LEVEL_OP || kernel == TOF_KERNEL_VCYCLE) && mg_ensure(c, s)) {
    c.last_error = "tof_time_kernel: multigrid setup failed";
    return TOF_ERR_CUDA;
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t ge = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  capturing() = true;
  int rc = 0;
  for (int r = 0; r < reps && rc == 0; ++r) rc = launch_once();
  capturing() = false;
  const cudaError_t ec = cudaStreamEndCapture(s, &graph);
  if (rc != 0 || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (ec != cudaSuccess && rc == 0) c.last_error = std::string("tof_time_kernel: capture: ") + cudaGetErrorString(ec);
    return rc == -1 ? TOF_ERR_ARG : TOF_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&ge, graph, 0);
  cudaGraphDestroy(graph);
  CUDA_TRY(ei);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  float ms = 0.f;
  cudaError_t e = cudaGraphLaunch(ge, s);                       // warm
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) e = cudaGraphLaunch(ge, s);
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(ge);
  CUDA_TRY(e);
  switch (kernel) {
    case TOF_KERNEL_MATVEC_F32:     // x read, y written (3 components), one factor per element
      bytes = 4.0 * (2.0 * 3.0 * c.g.NN * R) + 4.0 * c.g.NE;
      flops = 1152.0 * c.g.NE * R;
      break;
    case TOF_KERNEL_MG_LEVEL_OP:    // 27 3x3 FP32 stencil blocks per node; x, b, y_prev read, y written
      bytes = double(units) * (972.0 + 64.0 * R);
      flops = double(units) * 486.0 * R;
      break;
    case TOF_KERNEL_RAYLEIGH_RITZ:  // two n x n FP64 Gram matrices in, C and theta out
      units = n_rr;
      bytes = 8.0 * (2.0 * n_rr * n_rr + n_rr * c.lob_last_m + c.lob_last_m);
      break;
    default:
      break;
  }
  out->us = 1e3 * double(ms) / reps;
  out->bytes = bytes;
  out->flops = flops;
  out->units = units;
  return TOF_OK;
}

int tof_mg_query(tof_ctx* ctx, int level, int* dims, float* omega, void* stream) {
  if (!ctx) return TOF_ERR_ARG;
  const int r = mg_query(ctx->c, level, dims, omega, (cudaStream_t)stream);
  return r == -1 ? TOF_ERR_ARG : r == -2 ? TOF_ERR_CUDA : r;
}

int tof_mg_export(tof_ctx* ctx, int level, float* out, void* stream) {
  if (!ctx || !out) return TOF_ERR_ARG;
  const int r = mg_export(ctx->c, level, out, (cudaStream_t)stream);
  return r == -1 ? TOF_ERR_ARG : r == -2 ? TOF_ERR_CUDA : TOF_OK;
}

int tof_mg_setup(tof_ctx* ctx, void* stream) {
  if (!ctx) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (mg_ensure(c, (cudaStream_t)stream)) { c.last_error = "tof_mg_setup: multigrid setup failed"; return TOF_ERR_CUDA; }
  return TOF_OK;
}

int tof_mg_apply(tof_ctx* ctx, const float* r, float* e, int R, void* stream) {
  if (!ctx || !r || !e) return TOF_ERR_ARG;
  const int rc = mg_apply(ctx->c, r, e, R, (cudaStream_t)stream);
  return rc == -1 ? TOF_ERR_ARG : rc == -2 ? TOF_ERR_CUDA : TOF_OK;
}

// ---------------------------------------------------------------------------
// LOBPCG
// ---------------------------------------------------------------------------
int tof_lobpcg(tof_ctx* ctx, int mode, int nmodes, int block, double* X, double* lam, double tol, int maxiter,
               int precond, int inner_iters, double inner_rtol, tof_solve_stats* stats, double* resid,
               void* stream) {
  if (!ctx || !X || !lam || nmodes < 1 || block < nmodes || block > 8 || !(tol > 0.0) || maxiter < 1)
    return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (block > c.max_modes) { c.last_error = "tof_lobpcg: block exceeds the context's max_modes"; return TOF_ERR_ARG; }
  int it = 0;
  double res[8] = {0};
  double fl[8] = {0};
  const int rc = lobpcg_run(c, mode == TOF_MODE_FP64, nmodes, block, X, lam, tol, maxiter, precond,
                            std::max(inner_iters, 1), inner_rtol, &it, res, fl, (cudaStream_t)stream);
  if (resid)
    for (int j = 0; j < nmodes; ++j) resid[j] = res[j];
  if (stats) {
    stats->status = rc;
    stats->iters = it;
    stats->outer = 1;
    double w = 0.0;
    for (int j = 0; j < nmodes; ++j) w = std::max(w, res[j]);
    stats->relres = w;
    double f = 0.0;
    for (int j = 0; j < nmodes; ++j) f = std::max(f, fl[j]);
    stats->floor = f;
  }
  if (rc == -2) return TOF_ERR_CUDA;
  return rc;
}

// ---------------------------------------------------------------------------
// element quantities
// ---------------------------------------------------------------------------
int tof_elem_quadform(tof_ctx* ctx, int op, int dtype, const void* v, int nvec, double* out, void* stream) {
  if (!ctx || !v || !out || nvec < 1) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  launch_quadform(c, op, dtype == TOF_F64, v, nvec, out, (cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_compliance_sens(tof_ctx* ctx, int nlc, const double* w, const double* ce, double* dc, double* c_out,
                        void* stream) {
  if (!ctx || nlc < 1 || !w || !ce || !dc || !c_out) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (ceil_div(c.g.NE, 256) > (int)(c.gram_blocks * 576)) return TOF_ERR_ARG;
  launch_compliance_sens(c.g.NE, nlc, w, c.rho, ce, c.active, c.sp, dc, c.gram_part, c_out, (cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_eig_sens(tof_ctx* ctx, const double* qK, const double* qM, double lam, double vMv_tip, double* out,
                 void* stream) {
  if (!ctx || !qK || !qM || !out) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  launch_eig_sens(c.g.NE, c.rho, qK, qM, c.active, c.sp, lam, vMv_tip, out, c.gram_part_m, c.scal_m,
                  (cudaStream_t)stream);
  CUDA_TRY(cudaGetLastError());
  return TOF_OK;
}

int tof_stress(tof_ctx* ctx, const double* B_c, const double* D, int dtype, const void* u, int nvec,
               const double* rho, double* sigma, double* vm, double* smax, void* stream) {
  if (!ctx || !B_c || !D || !u || nvec < 1 || (dtype != TOF_F32 && dtype != TOF_F64)) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  if (launch_stress(c, B_c, D, dtype == TOF_F64, u, nvec, rho, sigma, vm, smax, (cudaStream_t)stream)) {
    c.last_error = "tof_stress: launch failed";
    return TOF_ERR_CUDA;
  }
  return TOF_OK;
}

int tof_stress_invariants(long long n, const double* sigma, double* vm, double* smax, void* stream) {
  if (n < 0 || (n > 0 && !sigma)) return TOF_ERR_ARG;
  return launch_stress_invariants(n, sigma, vm, smax, (cudaStream_t)stream) ? TOF_ERR_CUDA : TOF_OK;
}

int tof_fatigue(long long n, const double* s1, const double* s2, double sigma_uts, double s_design_pa, double* out,
                void* stream) {
  if (n < 0 || (n > 0 && (!s1 || !s2 || !out)) || !(sigma_uts > 0.0)) return TOF_ERR_ARG;
  return launch_fatigue(n, s1, s2, sigma_uts, s_design_pa, out, (cudaStream_t)stream) ? TOF_ERR_CUDA : TOF_OK;
}

int tof_sn_life(long long n, const double* sigma_eq, double* life, void* stream) {
  if (n < 0 || (n > 0 && (!sigma_eq || !life))) return TOF_ERR_ARG;
  return launch_sn_life(n, sigma_eq, life, (cudaStream_t)stream) ? TOF_ERR_CUDA : TOF_OK;
}

int tof_modal_frf(long long ndof, int m, const double* V, const double* fk_hz, long long npts, const double* f_hz,
                  double zeta, double* out, void* stream) {
  if (ndof < 0 || npts < 0 || m < 1 || (ndof * npts > 0 && (!V || !fk_hz || !f_hz || !out))) return TOF_ERR_ARG;
  return launch_modal_frf(ndof, m, V, fk_hz, npts, f_hz, zeta, out, (cudaStream_t)stream) ? TOF_ERR_CUDA : TOF_OK;
}

int tof_effective_mass(tof_ctx* ctx, const double* modes, int nmodes, int direction, double* out, void* stream) {
  if (!ctx || !modes || !out || nmodes < 1 || nmodes > 8 || direction < 0 || direction > 2) return TOF_ERR_ARG;
  Ctx& c = ctx->c;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t V = (size_t)c.g.NN * 4;
  // scratch in the FP64 LOBPCG area: [phi_1..phi_m, r] and M times them
  double* A = c.lw64 + 3 * (size_t)c.max_modes * V;
  double* MA = A + 9 * V;
  CUDA_TRY(cudaMemcpyAsync(A, modes, sizeof(double) * nmodes * V, cudaMemcpyDeviceToDevice, s));
  {
    // r: 1 on `direction` DOFs (packed, so fixed DOFs are 0)
    std::vector<double> r3(3 * (size_t)c.g.NN, 0.0);
    for (int n = 0; n < c.g.NN; ++n) r3[3 * (size_t)n + direction] = 1.0;
    double* tmp = MA;   // stage the DOF-major r through the MA area before packing
    CUDA_TRY(cudaMemcpyAsync(tmp, r3.data(), sizeof(double) * r3.size(), cudaMemcpyHostToDevice, s));
    launch_pack(c, tmp, 3 * (long long)c.g.NN, A + nmodes * V, true, 1, s);
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (launch_matvec(c, 1, true, A, MA, nmodes + 1, nullptr, s)) return TOF_ERR_CUDA;
  launch_gram(c, true, A, nmodes + 1, MA, nmodes + 1, c.gram + 6 * 576, s, c.gram_part_m);
  double G[81];
  CUDA_TRY(cudaMemcpyAsync(G, c.gram + 6 * 576, sizeof(double) * (nmodes + 1) * (nmodes + 1),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  const int n1 = nmodes + 1;
  const double total = G[nmodes * n1 + nmodes];
  for (int k = 0; k < nmodes; ++k) {
    const double gm = G[k * n1 + k];
    const double L = G[k * n1 + nmodes];   // phi_k^T M r
    out[k] = L * L / std::max(gm, 1e-30) / total;
  }
  return TOF_OK;
}

// ---------------------------------------------------------------------------
// filter / OC
// ---------------------------------------------------------------------------
int tof_filter_create(int nx, int ny, int nz, const double* w, int kx, int ky, int kz, const uint8_t* mask,
                      const uint8_t* fill, tof_filter** out) {
  if (!out || !w || !mask || nx < 1 || ny < 1 || nz < 1 || kx < 1 || ky < 1 || kz < 1 || !(kx & 1) ||
      !(ky & 1) || !(kz & 1)) {
    g_create_error = "tof_filter_create: invalid argument";
    return TOF_ERR_ARG;
  }
  struct Tap { int dx, dy, dz, pad; double w; };
  static_assert(sizeof(Tap) == 24, "tap layout");
  std::vector<Tap> taps;
  const int cx = kx / 2, cy = ky / 2, cz = kz / 2;
  for (int qz = 0; qz < kz; ++qz)
    for (int qy = 0; qy < ky; ++qy)
      for (int qx = 0; qx < kx; ++qx) {
        const double v = w[(qz * ky + qy) * kx + qx];
        if (v != 0.0) taps.push_back(Tap{qx - cx, qy - cy, qz - cz, 0, v});
      }
  if (taps.size() * sizeof(Tap) > 40 * 1024) { g_create_error = "tof_filter_create: kernel too large"; return TOF_ERR_ARG; }
  tof_filter* f = new tof_filter();
  f->nx = nx; f->ny = ny; f->nz = nz; f->ntaps = (int)taps.size();
  const size_t NE = (size_t)nx * ny * nz;
  cudaError_t e = cudaMalloc(&f->taps, std::max<size_t>(taps.size(), 1) * sizeof(Tap));
  if (e == cudaSuccess) e = cudaMalloc((void**)&f->mask, NE);
  if (e == cudaSuccess) e = cudaMalloc((void**)&f->fill, NE);
  if (e == cudaSuccess) e = cudaMalloc((void**)&f->den, NE * sizeof(double));
  if (e == cudaSuccess && !taps.empty()) e = cudaMemcpy(f->taps, taps.data(), taps.size() * sizeof(Tap), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(f->mask, mask, NE, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = fill ? cudaMemcpy(f->fill, fill, NE, cudaMemcpyHostToDevice) : cudaMemset(f->fill, 0, NE);
  if (e == cudaSuccess) {
    launch_filter_den(nx, ny, nz, f->taps, f->ntaps, f->mask, f->den, 0);
    e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) {
    g_create_error = std::string("tof_filter_create: ") + cudaGetErrorString(e);
    tof_filter_destroy(f);
    return TOF_ERR_CUDA;
  }
  *out = f;
  return TOF_OK;
}

int tof_filter_apply(tof_filter* f, int mode, const double* in, double* out, void* stream) {
  if (!f || !in || !out || mode < 0 || mode > 2) return TOF_ERR_ARG;
  launch_filter(f->nx, f->ny, f->nz, f->taps, f->ntaps, f->mask, f->den, f->fill, in, out, mode,
                (cudaStream_t)stream);
  return cudaGetLastError() == cudaSuccess ? TOF_OK : TOF_ERR_CUDA;
}

void tof_filter_destroy(tof_filter* f) {
  if (!f) return;
  if (f->taps) cudaFree(f->taps);
  if (f->mask) cudaFree(f->mask);
  if (f->fill) cudaFree(f->fill);
  if (f->den) cudaFree(f->den);
  delete f;
}

int tof_oc_update(int n, const double* x, const double* dc, double V_e, double target_volume, double move,
                  double* x_new, int* n_bisect, void* stream) {
  if (n < 1 || !x || !dc || !x_new || !(V_e > 0.0)) return TOF_ERR_ARG;
  launch_oc(n, x, dc, V_e, target_volume, move, x_new, n_bisect, (cudaStream_t)stream);
  return cudaGetLastError() == cudaSuccess ? TOF_OK : TOF_ERR_CUDA;
}

}  // extern "C"

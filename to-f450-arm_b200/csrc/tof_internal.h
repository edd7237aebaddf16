// Host-side internals of libtof: the design context and kernel launchers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "tof_common.cuh"

namespace tof {

// Host-side count of kernels this library launched (graph replays add their
// node count; launches recorded into a graph being captured are not counted).
// process-wide count of kernels launched (atomic: contexts may be driven
// from several host threads); launches recorded into a graph capture are
// counted when the graph is replayed instead
std::atomic<long long>& launch_counter();
bool& capturing();   // per host thread
inline void count_launch(long long n = 1) {
  if (!capturing()) launch_counter().fetch_add(n, std::memory_order_relaxed);
}
// Device functions of each source file, loaded eagerly when the first
// context is created on a device (see preload_all_kernels in tof_api.cu).
void preload_kernels_core();
void preload_kernels_gmg();
void preload_kernels_lobpcg();
void preload_kernels_pcg();
void preload_kernels_topopt();
// Error message of calls without a context (returned by tof_last_error(NULL)).
void set_global_error(const std::string& msg);

struct MG;

struct SimpParams {
  double penal = 3.0;          // SIMP exponent p (src/fem.py:204)
  double emin = 1e-9;          // E_min / E (src/fem.py:205)
  double mass_threshold = 0.1; // Pedersen threshold (src/fem.py:331)
  double mass_q = 6.0;         // Pedersen exponent (src/fem.py:332)
};

// One design: grid, element matrices, boundary conditions, SIMP factors and
// all solver workspace.  Everything is allocated in create(); solves never
// allocate.
// Error message of a context.  A static-family and a modal-family call may
// run at the same time from two host threads, so the message is set and read
// under a lock.
class ErrorSlot {
 public:
  ErrorSlot& operator=(const std::string& m) {
    std::lock_guard<std::mutex> g(mu_);
    msg_ = m;
    return *this;
  }
  ErrorSlot& operator=(const char* m) { return *this = std::string(m); }
  std::string str() const {
    std::lock_guard<std::mutex> g(mu_);
    return msg_;
  }

 private:
  mutable std::mutex mu_;
  std::string msg_;
};

struct Ctx {
  int dev = 0;
  int num_sms = 0;
  Grid g{};
  SimpParams sp{};
  int max_rhs = 0, max_modes = 0;
  int n_free = 0;

  // element matrices (FP64 dense 24x24 and the 64-block layout, FP32/FP64)
  double* Ke64 = nullptr; double* Me64 = nullptr;
  double* keb64 = nullptr; double* meb64 = nullptr;
  double* kebabs64 = nullptr;  // |Ke| in the 64-block layout (residual rounding floor)
  float* keb32 = nullptr; float* meb32 = nullptr;

  uint8_t* active = nullptr;   // [NE]
  uint8_t* fix = nullptr;      // [NN] bit c set: DOF c fixed (incl. ghost nodes)
  double* tip64 = nullptr;     // node4 lumped tip mass (0 at fixed DOFs)
  float* tip32 = nullptr;

  // per-element factors
  double *fK64 = nullptr, *fM64 = nullptr;
  float *fK32 = nullptr, *fM32 = nullptr;
  double* rho = nullptr;       // [NE] current density (0 outside the active set)
  // diagonals and Jacobi inverses (node4)
  double *dK64 = nullptr, *dM64 = nullptr, *dinvK64 = nullptr;
  float *dinvK32 = nullptr;

  // reductions / barrier
  double* partials = nullptr;  // [max grid][64]
  int partial_slots = 0;
  BarrierState* bar = nullptr;
  long long wait_ns = 0;       // wait budget of the persistent kernels (0: kWaitLimitNs)
  int* status = nullptr;       // [16] solver status words
  double* scal = nullptr;      // [256] solver scalars
  unsigned* counters = nullptr; // [16] last-block reduction counters (each kernel resets its own)

  // PCG workspace
  float* pw32 = nullptr;       // 10 node4 blocks of max_rhs vectors (FP32)
  double* pw64 = nullptr;      // 7 node4 blocks of max_rhs vectors (FP64)
  // LOBPCG workspace (FP32 node4): 2 sets x 3 blocks (S, KS, MS) of 3*max_modes
  float* lw32 = nullptr;
  double* lw64 = nullptr;      // FP64 refinement: X, KX, MX of max_modes
  double* gram = nullptr;      // [12][24*24]: modal 0-3, 6, 8-11; static 4, 5, 7
  // basis and block size of the last full-basis ([X W P], 3 x block)
  // in-loop Rayleigh-Ritz step, whose Gram matrices stay in slots 10 / 11
  int lob_last_n = 0, lob_last_m = 0;
  double* gram_part = nullptr; // [gram blocks][24*24]
  int gram_blocks = 0;
  // Scratch of the modal family (LOBPCG, eigenvalue sensitivities, effective
  // masses), apart from the static family's (PCG, true residuals, compliance
  // sensitivities), so one solve of each family may run at the same time on
  // two streams.  The multigrid V-cycle keeps one set of level vectors per
  // family (lane 0 static, lane 1 modal).
  double* gram_part_m = nullptr; // [gram blocks][24*24]
  unsigned* counters_m = nullptr; // [16]
  int* status_m = nullptr;       // [16]
  double* scal_m = nullptr;      // [256]
  // LOBPCG: pinned, mapped host slots for the residual norms read one
  // iteration late (written by the residual kernel through lob_pin_dev), and
  // the events that mark them complete
  void* lob_pin = nullptr;       // 3 slots of 256 bytes (cudaHostAlloc, mapped)
  void* lob_pin_dev = nullptr;
  // LOBPCG: a side stream for the P half of the block update (off the
  // critical path) and the events that order it: C ready, P half done
  cudaStream_t lob_side = nullptr;
  cudaEvent_t lob_cev = nullptr, lob_pev = nullptr;
  cudaEvent_t lob_ev[3] = {nullptr, nullptr, nullptr};

  // persistent-launch capacity for each kernel flavour
  int coop_pipe[9] = {0};
  int coop_plain[9] = {0};


  MG* mg = nullptr;                // multigrid hierarchy (tof_gmg.cu)
  std::vector<uint8_t> host_fix;   // host copy of `fix`
  size_t bytes = 0;
  ErrorSlot last_error;
};

// tensor-map encoding for a block of R node4 vectors (dtype float or double)
bool encode_node4_map(CUtensorMap* m, const void* base, const Grid& g, int R, bool f64, std::string* err);

// kernels (tof_kernels.cu)
void launch_factors(Ctx& c, const double* rho, cudaStream_t s);
void launch_diag(Ctx& c, cudaStream_t s);
// op: 0 K, 1 M, 2 |K| (entrywise absolute values; FP64 only)
int launch_matvec(Ctx& c, int op, bool f64, const void* x, void* y, int nrhs, const void* b_residual,
                  cudaStream_t s);
// yK = K x and yM = M x (with the tip lump) in one launch per chunk of <= 8
int launch_matvec_km(Ctx& c, bool f64, const void* x, void* yK, void* yM, int nrhs, cudaStream_t s);
int launch_smooth0(Ctx& c, const float* x, float* y, const float* b, const float* dinv, const float* coef, bool prev,
                   int R, cudaStream_t s);
void launch_pack(const Ctx& c, const double* src, long long ld, void* dst, bool f64, int nvec, cudaStream_t s);
void launch_unpack(const Ctx& c, const void* src, bool f64, double* dst, long long ld, int nvec, cudaStream_t s);
void launch_gram(Ctx& c, bool f64, const void* A, int na, const void* B, int nb, double* G, cudaStream_t s, double* part = nullptr);
// Column selection of a node4 block: vector k of the selection is vector
// col[k] of the block (up to 24).
struct ColMap {
  int col[24];
};
// G1 = A[:, cols]^T B1[:, cols], G2 = A[:, cols]^T B2[:, cols] (n x n) in one pass
void launch_gram2_cols(Ctx& c, bool f64, const void* A, const void* B1, const void* B2, const ColMap& cols, int n,
                       double* G1, double* G2, cudaStream_t s, double* part = nullptr);
// G = A[:, ma]^T B[:, mb] (na x nb), same kernels as launch_gram
void launch_gram_cols(Ctx& c, bool f64, const void* A, const ColMap& ma, int na, const void* B, const ColMap& mb,
                      int nb, double* G, cudaStream_t s, double* part = nullptr);
void launch_quadform(const Ctx& c, int op, bool f64, const void* v, int nvec, double* out, cudaStream_t s);
void launch_convert(const void* src, bool src64, void* dst, bool dst64, long long n, cudaStream_t s);
void launch_axpy64(long long n, const double* x, double* y, double a, cudaStream_t s);
// y += x (n floats)
void launch_add_f32(long long n, const float* x, float* y, cudaStream_t s);
// y = |x| (n doubles)
void launch_abs64(long long n, const double* x, double* y, cudaStream_t s);
void launch_add_f32_to_f64(long long n, const float* d, double* x, cudaStream_t s);

// stress and fatigue (tof_stress.cu)
int launch_stress(Ctx& c, const double* B, const double* D, bool f64, const void* u, int nvec, const double* rho,
                  double* sigma, double* vm, double* smax, cudaStream_t s);
int launch_stress_invariants(long long n, const double* sigma, double* vm, double* smax, cudaStream_t s);
int launch_fatigue(long long n, const double* s1, const double* s2, double uts, double s_design_pa, double* out,
                   cudaStream_t s);
int launch_sn_life(long long n, const double* sigma_eq, double* life, cudaStream_t s);

// modal FRF (tof_frf.cu)
int launch_modal_frf(long long ndof, int m, const double* V, const double* fk_hz, long long npts, const double* f_hz,
                     double zeta, double* out, cudaStream_t s);

// PCG (tof_pcg.cu)
// G CTAs meet at one grid barrier that expects `expected` arrivals (more than
// G: nobody releases it, every CTA gives up after the context's wait budget)
int launch_barrier_selftest(Ctx& c, int G, int expected, cudaStream_t s);
int pcg_plain64(Ctx& c, const double* b, double* x, int R, double rtol, int maxiter, int* iters, double* relres,
                int* status, cudaStream_t s);
int pcg_pipe32(Ctx& c, const double* b, float* d, int R, double rtol, int maxiter, int* iters, double* relres,
               int* status, cudaStream_t s);
// FP32 standard PCG from x = 0 (x must be zeroed by the caller)
int pcg_std32(Ctx& c, const double* b, float* x, int R, double rtol, int maxiter, cudaStream_t s);

// Diagnostic single launches for kernel timing (tof_time_kernel): the
// coarse-level stencil operator of multigrid level `level` in its smoothing
// form on the static lane's level vectors; the Rayleigh-Ritz eigensolver on
// the Gram matrices of the last full-basis LOBPCG step (slots 10 / 11).
int mg_launch_level_op(Ctx& c, int level, int R, cudaStream_t s, long long* nodes);
int lob_launch_rayleigh_ritz(Ctx& c, cudaStream_t s, int* n);

// multigrid (tof_gmg.cu)
int mg_create(Ctx& c, int maxR);
void mg_destroy(Ctx& c);
int mg_setup(Ctx& c, cudaStream_t s);
void mg_mark_dirty(Ctx& c);
int mg_ensure(Ctx& c, cudaStream_t s);
int mg_capture_all(Ctx& c);   // record every V-cycle graph once (context creation)
int mg_vcycle(Ctx& c, int R, cudaStream_t s, int lane = 0);   // mg_rhs -> mg_out
float* mg_rhs(Ctx& c, int lane = 0);
float* mg_out(Ctx& c, int lane = 0);
int mg_levels(const Ctx& c);
int mg_query(Ctx& c, int level, int* dims, float* omega, cudaStream_t s);
int mg_export(Ctx& c, int level, float* out, cudaStream_t s);
int mg_apply(Ctx& c, const float* r, float* e, int R, cudaStream_t s);
int pcg_mg64(Ctx& c, const double* b, double* x, int R, double rtol, int maxiter, int* iters, int* status,
             cudaStream_t s);

}  // namespace tof

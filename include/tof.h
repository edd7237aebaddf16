/* libtof — B200 (sm_100a) voxel SIMP hot path behind a plain C ABI.
 *
 * Every entry point takes plain pointers and sizes; device pointers are CUDA
 * global-memory addresses on the current device, `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).  Return value: 0 on
 * success, > 0 "finished but not converged", < 0 an error (see TOF_ERR_*;
 * tof_last_error() has the message).  Nothing here falls back to the CPU.
 *
 * Vector layout ("node4"): a nodal vector of the (nx+1)(ny+1)(nz+1)-node grid
 * stores node n = k*(nx+1)*(ny+1) + j*(nx+1) + i at [4n .. 4n+3] as
 * (ux, uy, uz, 0); a block of R vectors is R such arrays back to back.
 * tof_pack / tof_unpack convert from / to the reference's DOF-major layout
 * (DOF 3n + c).  All node4 inputs must be zero at fixed DOFs (tof_pack
 * guarantees it).
 *
 * Element arrays are over the full nx*ny*nz grid, x fastest:
 * e = (ez*ny + ey)*nx + ex.
 *
 * Citations are to the reference project (NinhGhoster/TO-F450-arm) by path
 * within it.
 */
#ifndef TOF_H
#define TOF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct tof_ctx tof_ctx;
typedef struct tof_filter tof_filter;

enum {
  TOF_OK = 0,
  TOF_NOT_CONVERGED = 1,
  TOF_ERR_ARG = -1,
  TOF_ERR_CUDA = -2,
  TOF_ERR_BREAKDOWN = -3,
  TOF_ERR_NONFINITE = -4,
  TOF_ERR_TIMEOUT = -5
};
enum { TOF_OP_K = 0, TOF_OP_M = 1 };
enum { TOF_F32 = 0, TOF_F64 = 1 };
/* PCG modes.  TOF_MODE_FP64: plain FP64 Jacobi PCG, the reference's
 * algorithm (the drop-in form).  TOF_MODE_MIXED: FP64 PCG preconditioned by
 * an FP32 geometric-multigrid V-cycle (Galerkin coarse levels).
 * TOF_MODE_IR: FP32 Jacobi PCG inside FP64 iterative refinement.
 * LOBPCG: block vectors, Gram matrices and Rayleigh-Ritz are FP64 in every
 * mode; TOF_MODE_FP64 uses the preconditioner requested, TOF_MODE_MIXED the
 * FP32 multigrid V-cycle. */
enum { TOF_MODE_FP64 = 0, TOF_MODE_MIXED = 1, TOF_MODE_IR = 2 };
enum { TOF_PRECOND_JACOBI = 0, TOF_PRECOND_PCG = 1, TOF_PRECOND_MG = 2 };
enum { TOF_FILTER_FORWARD = 0, TOF_FILTER_ADJOINT = 1, TOF_FILTER_PHYSICAL = 2 };
enum {
  TOF_Q_NODES = 0, TOF_Q_ELEMS = 1, TOF_Q_FREE_DOFS = 2, TOF_Q_TILE_X = 3, TOF_Q_TILE_Y = 4,
  TOF_Q_TILE_Z = 5, TOF_Q_DEVICE_BYTES = 6, TOF_Q_MAX_RHS = 7, TOF_Q_MAX_MODES = 8
};

typedef struct {
  int status;     /* TOF_OK, TOF_NOT_CONVERGED or a TOF_ERR_* */
  int iters;      /* Krylov / LOBPCG iterations (summed over refinement steps) */
  int outer;      /* refinement steps (mixed PCG), else 1 */
  double relres;  /* PCG: ||b - K x||_2 / ||b||_2 recomputed in FP64 at exit.
                     LOBPCG: largest ||K x - theta M x|| / ||K x|| of the modes */
  double floor;   /* PCG: FP64 rounding floor of relres, eps ||(|K||x| + |b|)|| / ||b||
                     (what rounding the exact solution to FP64 can leave); the
                     solve counts as converged when relres <= max(rtol, floor).
                     LOBPCG: the largest eps ||(|K| + theta M)|x||| / ||K x|| of
                     the modes; converged when each mode's residual is at most
                     max(tol, 10 x its floor) */
} tof_solve_stats;

/* SIMP interpolation constants: stiffness emin + (1-emin) rho^penal,
 * mass rho for rho >= mass_threshold else t (rho/t)^mass_q.
 * Reference: src/fem.py:204-205 (SIMP_PENALTY, E_MIN_FRAC), src/fem.py:331-349. */
typedef struct {
  double penal, emin, mass_threshold, mass_q;
} tof_simp_params;

int tof_version(void);
/* Number of CUDA kernels this library has launched in the process (CUDA-graph
 * replays count their kernel nodes).  Diagnostics; no reference counterpart. */
long long tof_launch_count(void);
/* ctx may be NULL: the calling thread's last create error.  The string stays
 * valid until the calling thread's next tof_last_error call. */
const char* tof_last_error(const tof_ctx* ctx);

/* Create a design context on the current CUDA device.
 * Replaces FEM3D.__init__ (src/fem.py:207-308): the element matrices are the
 * caller's 24x24 FP64 Ke / Me (src/fem.py:99-152; callers may overwrite them,
 * e.g. orthotropic D), `active` marks in_arm voxels (NULL = all), `fixed_dof`
 * (3*NN bytes, nonzero = clamped, src/fem.py:282-290) and the library adds
 * ghost nodes of no active element itself (src/fem.py:292-305).  `tip_lump`
 * (3*NN FP64 or NULL) is the lumped mass added to diag(M), i.e.
 * mass_kg / n_nodes on each DOF of the tip nodes (src/fem.py:383-398).
 * `tile` (node tile x, y, z; NULL = default 8x4x4) must have x*y*z <= 256.
 * max_rhs / max_modes (1..8) size the solver workspace; this is the only
 * call that allocates device memory.
 * Concurrency: calls on one context are issued in order on their streams,
 * except that one call of the static family (tof_pcg, tof_elem_quadform,
 * tof_compliance_sens) and one of the modal family (tof_lobpcg with the
 * Jacobi or multigrid preconditioner, tof_eig_sens, tof_effective_mass) may
 * run at the same time from two host threads on two streams: the families
 * keep separate scratch and multigrid vectors.  Both streams must first wait
 * on the stream that set the density (and, for the multigrid, ran
 * tof_mg_setup).  The error message of tof_last_error may then come from
 * either call. */
int tof_ctx_create(int nx, int ny, int nz, const double h[3], const double Ke[576], const double Me[576],
                   const uint8_t* active, const uint8_t* fixed_dof, const double* tip_lump,
                   const tof_simp_params* simp, int max_rhs, int max_modes, const int tile[3], tof_ctx** out);
void tof_ctx_destroy(tof_ctx* ctx);
long long tof_ctx_query(const tof_ctx* ctx, int what);
/* Wait budget of the context's persistent solver kernels (ns, 1 us .. 60 s;
 * default 2 s).  Every device-side wait of those kernels (grid barriers,
 * TMA tile arrivals) gives up after it: the solve then returns
 * TOF_ERR_TIMEOUT and the context stays usable.  No reference counterpart:
 * the reference's solvers run on the host and signal failure by `info != 0`
 * and a fallback solver (src/fem.py:548-550, src/fem_gpu.py:84-91). */
int tof_ctx_set_wait_limit(tof_ctx* ctx, long long ns);
/* Exercises that bounded wait: a few CTAs meet at one grid barrier that
 * expects `extra_arrivals` (0 or 1) more arrivals than the launch has.  With
 * 0 the barrier completes (TOF_OK); with 1 nobody releases it, every CTA
 * gives up after the wait budget and the call returns TOF_ERR_TIMEOUT.  The
 * barrier is reset either way.  Diagnostics; no reference counterpart. */
int tof_wait_selftest(tof_ctx* ctx, int extra_arrivals, void* stream);

/* Set element densities (device FP64 [NE]); computes SIMP stiffness and mass
 * factors and the diagonals.  Replaces the per-call assemble_K / assemble_M
 * (src/fem.py:311-398): no matrix is ever assembled. */
int tof_set_density(tof_ctx* ctx, const double* rho, void* stream);

/* Replace the lumped tip mass (host FP64 [3*NN], NULL = none) and refresh
 * diag(M).  FEM3D.modal_analysis / eigenvalue_sensitivity take the tip mass
 * per call (src/fem.py:400-435, 472-520); mass on fixed or ghost DOFs is
 * dropped as the reference's K[free][:, free] slicing drops it. */
int tof_set_tip_lump(tof_ctx* ctx, const double* tip_lump, void* stream);

/* DOF-major FP64 (ld doubles between vectors) <-> node4 of dtype. */
int tof_pack(tof_ctx* ctx, const double* src, long long ld, void* dst, int dtype, int nvec, void* stream);
int tof_unpack(tof_ctx* ctx, const void* src, int dtype, double* dst, long long ld, int nvec, void* stream);

/* y = A_ff x for A = K or M (matrix-free), nvec node4 vectors of dtype.
 * The reference forms K[free][:, free] @ x from the assembled CSR
 * (src/fem.py:437-438, src/fem_gpu.py:52-58). */
int tof_matvec(tof_ctx* ctx, int op, int dtype, const void* x, void* y, int nvec, void* stream);

/* diag(A_ff) as node4 FP64 (0 at fixed DOFs); src/fem.py:441-443, 543-544. */
int tof_diag(tof_ctx* ctx, int op, double* out, void* stream);

/* Solve K_ff u = b for nrhs node4 FP64 right-hand sides; x holds the start
 * vectors on entry and the solution on exit.  Replaces
 * FEM3D.apply_BCs_and_solve / FEM3D.solve (src/fem.py:529-561) and the GPU
 * drop-in _solve_cg_gpu (src/fem_gpu.py:46-98); stops at
 * ||b - K x||_2 <= rtol ||b||_2 like SciPy's cg, the residual recomputed in
 * FP64 at exit; where FP64 cannot represent a solution that good (the
 * rounding floor in tof_solve_stats.floor is above rtol) a true residual at
 * that floor counts as converged.  Synchronises `stream`;
 * stats (host, nrhs entries) may be NULL. */
int tof_pcg(tof_ctx* ctx, int mode, const double* b, double* x, int nrhs, double rtol, int maxiter,
            tof_solve_stats* stats, void* stream);

/* Kernel timing (diagnostics; no reference counterpart): `reps` launches of
 * one kernel, recorded into a CUDA graph on `stream` (not the legacy default
 * stream), replayed once to warm up and once between CUDA events; out->us is
 * the average device time of one launch, out->bytes / out->flops the
 * algorithmic traffic and arithmetic of one launch (0 where not meaningful),
 * out->units the nodes / elements / basis size it covers.  Kernels:
 * TOF_KERNEL_MATVEC_F32 (matrix-free FP32 K x on the fine grid, nvec
 * vectors, the multigrid smoother's operator), TOF_KERNEL_MG_LEVEL_OP (the
 * assembled-stencil operator of multigrid level `level` >= 1 in its
 * smoothing form), TOF_KERNEL_RAYLEIGH_RITZ (the LOBPCG Rayleigh-Ritz
 * eigensolver on the Gram matrices of the context's last LOBPCG iteration),
 * TOF_KERNEL_VCYCLE (a whole V-cycle, all its kernels).  The multigrid
 * kernels need the hierarchy of the current density (tof_mg_setup).  Work
 * vectors of the context are overwritten; the graph is created and
 * destroyed inside the call. */
enum { TOF_KERNEL_MATVEC_F32 = 0, TOF_KERNEL_MG_LEVEL_OP = 1, TOF_KERNEL_RAYLEIGH_RITZ = 2, TOF_KERNEL_VCYCLE = 3 };
typedef struct {
  double us;
  double bytes;
  double flops;
  long long units;
} tof_kernel_timing;
int tof_time_kernel(tof_ctx* ctx, int kernel, int level, int nvec, int reps, tof_kernel_timing* out, void* stream);

/* Multigrid preconditioner introspection (no reference counterpart: the
 * reference preconditions with diag(K) only).  tof_mg_query: number of
 * levels (return value); for `level` >= 0 also its element dims (dims[3]) and
 * the smoothing weight omega (host).  tof_mg_export: that level's Galerkin
 * element matrices, FP32 [NE][576] (device; level >= 1).  tof_mg_apply: one
 * V-cycle e = B r on R node4 FP32 vectors (R in 1, 2, 4, 8). */
int tof_mg_query(tof_ctx* ctx, int level, int* dims, float* omega, void* stream);
int tof_mg_export(tof_ctx* ctx, int level, float* out, void* stream);
int tof_mg_apply(tof_ctx* ctx, const float* r, float* e, int R, void* stream);
/* Build the multigrid hierarchy for the current density now, on `stream`
 * (otherwise the first solve that needs it builds it on its own stream).
 * Call it before issuing a static and a modal solve on two streams that both
 * wait on `stream` (see the concurrency note at tof_ctx_create). */
int tof_mg_setup(tof_ctx* ctx, void* stream);

/* Lowest `nmodes` eigenpairs of K_ff x = lam M_ff x with a block of `block`
 * vectors (nmodes <= block <= 8).  X (device node4 FP64, `block` vectors)
 * holds the start block on entry (warm start or random) and on exit the
 * `block` M-orthonormal Ritz vectors of the final Rayleigh-Ritz step,
 * ascending: the modes in its first nmodes vectors, then the guard vectors
 * (a warm start for the next solve);
 * lam (host, nmodes) gets the eigenvalues (rad/s)^2.  Replaces
 * FEM3D.modal_analysis (src/fem.py:400-470) and _modal_gpu
 * (src/fem_gpu.py:101-173).  precond: TOF_PRECOND_JACOBI (as the reference),
 * TOF_PRECOND_PCG (inner_iters FP32 PCG iterations to inner_rtol) or
 * TOF_PRECOND_MG (inner_iters FP32 multigrid V-cycles, at least one).
 * Synchronises `stream`.  resid (host, nmodes) may be NULL. */
int tof_lobpcg(tof_ctx* ctx, int mode, int nmodes, int block, double* X, double* lam, double tol, int maxiter,
               int precond, int inner_iters, double inner_rtol, tof_solve_stats* stats, double* resid,
               void* stream);

/* Per-element quadratic forms v_e^T A_e v_e (A_e = Ke or Me, unscaled), FP64
 * out [nvec][NE].  ce = u_e^T Ke u_e is FEM3D.elem_compliance
 * (src/fem.py:605-615); phi_e^T Ke phi_e and phi_e^T Me phi_e are the
 * contractions of FEM3D.eigenvalue_sensitivity (src/fem.py:498-501). */
int tof_elem_quadform(tof_ctx* ctx, int op, int dtype, const void* v, int nvec, double* out, void* stream);

/* G = A^T B (na x nb, row-major, device FP64) of node4 blocks, na, nb <= 24. */
int tof_gram(tof_ctx* ctx, int dtype, const void* A, int na, const void* B, int nb, double* G, void* stream);

/* The same G = A^T B without a context and without allocating any device
 * memory; no counterpart in the reference.  For callers that cannot allocate
 * device memory when they need it: a host application whose memory pool owns
 * the whole GPU and refuses other allocations, or a loop that must not take
 * cudaMalloc's implicit device synchronisation.  A, B: node4 blocks of
 * n_nodes nodes, dtype TOF_F32 or TOF_F64; G: device FP64 na x nb.
 * Limits: na, nb <= 24 and n_nodes <= INT_MAX, else TOF_ERR_ARG with a
 * message in tof_last_error(NULL).  Temporaries live in one fixed device
 * array of about 1.1 MiB that is part of this library's device code: it takes
 * its device memory at the first call on each device (CUDA loads device code
 * lazily) and keeps it until the process exits.  That first call also looks
 * up the array's device address, so make it before any stream capture and
 * before a memory pool takes over the GPU.  All calls on a GPU share the
 * array and it keeps the previous call's contents: calls whose executions
 * overlap on the same GPU race, so order them (one stream, or events). */
int tof_gram_noalloc(long long n_nodes, int dtype, const void* A, int na, const void* B, int nb, double* G,
                     void* stream);

/* Compliance and its sensitivity for nlc load cases from ce [nlc][NE]
 * (src/topopt.py:291-306): c = sum_l w_l sum_e f_e ce_le (device scalar
 * c_out), dc_e = sum_l w_l (-p (1-emin) rho_e^(p-1) ce_le) (device [NE]). */
int tof_compliance_sens(tof_ctx* ctx, int nlc, const double* w, const double* ce, double* dc, double* c_out,
                        void* stream);

/* d lambda / d rho_e (device [NE]) for one mode from its quadratic forms
 * qK, qM [NE] and the tip-mass term vMv_tip = m_node * sum(v_tip^2):
 * FEM3D.eigenvalue_sensitivity (src/fem.py:472-526). */
int tof_eig_sens(tof_ctx* ctx, const double* qK, const double* qM, double lam, double vMv_tip, double* out,
                 void* stream);

/* Effective-mass fractions (phi^T M r)^2 / (phi^T M phi) / (r^T M r) of
 * nmodes node4 FP64 modes, r = unit translation along `direction` (0, 1, 2)
 * on free DOFs; out (host, nmodes).  sims/modal_participation.py:37-57.
 * Synchronises `stream`. */
int tof_effective_mass(tof_ctx* ctx, const double* modes, int nmodes, int direction, double* out, void* stream);

/* Element stress at the element centres for nvec node4 displacement vectors
 * (dtype TOF_F32 / TOF_F64): sigma_e = rho_e D B_c u_e with the reference's
 * linear density scaling (FEM3D.compute_stress, src/fem.py:564-579).  B_c:
 * host 6x24 strain-displacement matrix at the centre (src/fem.py:153-176),
 * D: host 6x6 elasticity matrix, both row-major, Voigt order xx yy zz xy yz
 * xz.  rho: device FP64 [NE] over the full grid, or NULL for the density set
 * by tof_set_density.  Outputs, device FP64 over the full grid (x fastest,
 * 0 on inactive voxels), each may be NULL: sigma [nvec][NE][6], vm
 * [nvec][NE] (FEM3D.von_mises, src/fem.py:582-589), smax [nvec][NE]
 * (FEM3D.principal_stress_max, src/fem.py:592-602). */
int tof_stress(tof_ctx* ctx, const double* B_c, const double* D, int dtype, const void* u, int nvec,
               const double* rho, double* sigma, double* vm, double* smax, void* stream);

/* von Mises and largest principal stress of n Voigt stress rows (device FP64
 * [n][6]; outputs device FP64 [n], either may be NULL).  src/fem.py:582-602. */
int tof_stress_invariants(long long n, const double* sigma, double* vm, double* smax, void* stream);

/* Fatigue field of a cycle between two stress levels s1, s2 (Pa, device FP64
 * [n], e.g. the von Mises stresses of two load cases): mean and alternating
 * stress, Goodman-equivalent alternating stress for ultimate strength
 * sigma_uts, life from the PA12 S-N curve, damage per cycle and factor of
 * safety s_design_pa / equivalent stress (fatigue_life_field,
 * src/fatigue.py:83-112).  out: device FP64 [6][n] in that order. */
int tof_fatigue(long long n, const double* s1, const double* s2, double sigma_uts, double s_design_pa, double* out,
                void* stream);

/* Cycles to failure at n equivalent fully reversed stresses (Pa, device FP64)
 * from the PA12 S-N curve (sn_life, src/fatigue.py:24-65). */
int tof_sn_life(long long n, const double* sigma_eq, double* life, void* stream);

/* Modal-superposition FRF magnitude at ndof DOFs and npts frequencies:
 * out[d][i] = |sum_k V[d][k]^2 / ((w_k^2 - w_i^2) + 2 i zeta w_k w_i)|,
 * w = 2 pi f (modal_frf_at_dof, src/plotting.py:378-399).  V: device FP64
 * [ndof][m] mode-shape values at the DOFs, fk_hz: device [m] natural
 * frequencies, f_hz: device [npts]; out: device FP64 [ndof][npts]. */
int tof_modal_frf(long long ndof, int m, const double* V, const double* fk_hz, long long npts, const double* f_hz,
                  double zeta, double* out, void* stream);

/* Density filter on an nx*ny*nz element grid (x fastest) with a (kx,ky,kz)
 * weight array (z slowest: w[(qz*ky + qy)*kx + qx], odd sizes) and a mask
 * (NE bytes).  Replaces topopt.cone_kernel / filter_field
 * (src/topopt.py:32-58).  `fill` (NE bytes or NULL) marks active elements
 * outside the mask that TOF_FILTER_PHYSICAL sets to 1
 * (src/topopt.py:270-281). */
int tof_filter_create(int nx, int ny, int nz, const double* w, int kx, int ky, int kz, const uint8_t* mask,
                      const uint8_t* fill, tof_filter** out);
int tof_filter_apply(tof_filter* f, int mode, const double* in, double* out, void* stream);
void tof_filter_destroy(tof_filter* f);

/* OC update with bisection on the Lagrange multiplier
 * (SIMPOptimizer._oc_update, src/topopt.py:190-214); device FP64 arrays of
 * n design cells; n_bisect (device int or NULL) gets the step count. */
int tof_oc_update(int n, const double* x, const double* dc, double V_e, double target_volume, double move,
                  double* x_new, int* n_bisect, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* TOF_H */

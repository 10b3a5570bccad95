/*
 * hprmat_b200.h -- C ABI of the B200 (sm_100a) dense complex R-matrix solver.
 *
 * The library is a new solver type behind HPRMAT's `rmatrix` entry and its `solver_type`
 * dispatch.  Every entry point takes plain pointers and sizes.  Complex arrays are
 * interleaved (re, im) double pairs in Fortran column-major order, i.e. the memory of
 * `complex*16` / `complex(c_double_complex)` arrays, passed as `double*`.
 *
 * Reference interfaces (paths relative to the HPRMAT project root) that each entry point
 * replaces are cited next to it.  Errors are reported by the integer return value (see
 * HPRMAT_B200_* below).  Nothing falls back to a CPU solver: a missing or failing GPU is an
 * error.
 *
 * Threading: one context per host thread; calls on one context are ordered on the
 * context's CUDA stream and return after their results are complete.
 */
#ifndef HPRMAT_B200_H
#define HPRMAT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (return values). */
#define HPRMAT_B200_OK               0
#define HPRMAT_B200_ERR_ARG         -1   /* invalid argument (sizes, null pointers) */
#define HPRMAT_B200_ERR_CUDA        -2   /* CUDA runtime error (message: hprmat_b200_last_error) */
#define HPRMAT_B200_ERR_OOM         -3   /* device allocation failed */
#define HPRMAT_B200_ERR_TIMEOUT     -4   /* a bounded device-side wait gave up */
#define HPRMAT_B200_ERR_UNSUPPORTED -5   /* input outside what this build handles */
#define HPRMAT_B200_ERR_NODEVICE    -6   /* no usable sm_100 device */
#define HPRMAT_B200_SINGULAR         1   /* exactly zero pivot; stats.info = its 1-based column */
#define HPRMAT_B200_PIVOT_GROWTH     2   /* mixed path with opts.growth_error: the FP32 factors'
                                            pivot growth (stats.pivot_growth) exceeded the limit */
#define HPRMAT_B200_NOT_CONVERGED   99   /* refinement stopped above tol (as info=99 in
                                            src/cusolver_interface.cu:1577-1589) */

/* Arithmetic of the LU factorisation. */
#define HPRMAT_B200_PREC_FP64   0  /* plain FP64 complex LU (the "plain FP64 device LU") */
#define HPRMAT_B200_PREC_MIXED  1  /* complex LU with 3xTF32 tcgen05 trailing updates, FP32
                                      panels, FP64 residual refinement */

/* solver_type id of this backend in HPRMAT's dispatch (next free id after 1..6,
   src/rmatrix_hp.F90:299-322, src/rmat_solvers.F90:69-88). */
#define HPRMAT_SOLVER_B200      7

typedef struct hprmat_b200_ctx hprmat_b200_ctx;

typedef struct {
  int precision;   /* HPRMAT_B200_PREC_* (default MIXED) */
  int max_refine;  /* FP64 refinement steps, 0..8 (default 3) */
  double tol;      /* stop when ||B - C X||_F / ||B||_F < tol (default 1e-12); the same
                      relative Frobenius rule as src/rmat_solvers.F90:253-262 */
  double surface_tol; /* R-matrix path: or when a refinement step changes the surface
                         projection R = q2^T X (what the collision matrix depends on) by less
                         than surface_tol relative (Frobenius; default 1e-11) */
  int panel_nb;    /* LU block size; 0 = automatic */
  int reuse_factors; /* mixed path, one interval, local potentials: when nonzero and the previous
                        factorisation on this context was of the same channel block (same
                        potential -- checked by a fingerprint of cpot --, lval, mesh), rmatrix
                        keeps it as the preconditioner of the FP64 refinement instead of
                        factorising C(E) again: between energies C(E) changes only on the
                        diagonal (-k^2 and the closed-channel Bloch terms).  If the refinement
                        does not converge it factorises C(E) and solves again.  Default 0. */
  int estimate_condition; /* when nonzero, FP64 factorisations (the FP64 path and the mixed
                             path's FP64 fallback) also estimate the 1-norm condition number of
                             the matrix (stats.cond_estimate; LAPACK ZGECON's quantity, by the
                             Hager-Higham estimator on the factors: ~11 extra solves with one
                             right-hand side).  Default 0. */
  int growth_error;       /* mixed path: when nonzero, FP32 factors whose pivot growth exceeds the
                             limit (10^6) make the call return HPRMAT_B200_PIVOT_GROWTH instead of
                             factorising in FP64 (an exact zero FP32 pivot still falls back, as
                             the reference's Type 2 does).  Default 0: fall back. */
  int reserved[1];
} hprmat_b200_opts;

typedef struct {
  int status;               /* return value of the call */
  int info;                 /* LAPACK-style info: >0 = first zero pivot (1-based) */
  int refine_steps;         /* refinement corrections (outer steps) applied */
  int inner_iterations;     /* preconditioned FGMRES iterations (LU solves) over all steps */
  int nb;                   /* LU block size used */
  int n;                    /* order of the solved system */
  int nrhs;
  double rel_residual;      /* final ||B - C X||_F / ||B||_F, evaluated in FP64 */
  double surface_change;    /* relative change of R in the last refinement step (-1: n/a) */
  double residual_floor;    /* estimated rounding floor of the relative FP64 residual (0: n/a) */
  double floor_history[9];  /* the floor estimate at each outer step */
  double residual_history[9];
  double ms_assemble, ms_factor, ms_solve, ms_refine, ms_umatrix, ms_total;
  int factorizations;       /* LU factorisations the call ran (0: reused, opts.reuse_factors) */
  int fp64_fallback;        /* mixed path: 1 if the FP32 factorisation was replaced by the FP64 one
                               (pivot growth above the limit, or an exact zero FP32 pivot, as the
                               reference's Type 2 falls back on CGETRF info != 0) */
  double pivot_growth;      /* max |u_ij| / max |c_ij| (|re| + |im|) of the last factorisation */
  double cond_estimate;     /* opts.estimate_condition: estimate of ||C||_1 ||C^-1||_1 (largest
                               over the intervals); 0 when not estimated */
  double ms_condest;        /* host time of the condition estimate (included in ms_total) */
} hprmat_b200_stats;

/* Defaults for hprmat_b200_opts. */
void hprmat_b200_default_opts(hprmat_b200_opts* opts);

/* Create a context on CUDA device `device` (the reference auto-initialises device 0 in
   gpu_solver_init_, src/cusolver_interface.cu:193-220).  opts may be NULL. */
int hprmat_b200_create(int device, const hprmat_b200_opts* opts, hprmat_b200_ctx** out);
/* Release every device buffer of the context (gpu_solver_finalize_,
   src/cusolver_interface.cu:222-258). */
int hprmat_b200_destroy(hprmat_b200_ctx* ctx);
int hprmat_b200_set_opts(hprmat_b200_ctx* ctx, const hprmat_b200_opts* opts);
/* Order the context's work on an existing cudaStream_t (passed as void*); NULL = the
   context's own stream. */
int hprmat_b200_set_stream(hprmat_b200_ctx* ctx, void* stream);

/* Lagrange-Legendre mesh, kinetic and Bloch matrices: rmat_ini(nr, ns, rmax, zrma),
   src/rmatrix_hp.F90:61-159.  zrma (nr*ns doubles) may be NULL. */
int hprmat_b200_rmat_ini(hprmat_b200_ctx* ctx, int nr, int ns, double rmax, double* zrma);

/* Adjoint of the collision matrix (no counterpart in the reference).  For the arguments of
   hprmat_b200_rmatrix and the gradient gu of a real loss L with respect to U (complex (ndim,
   ndim), leading nopen x nopen block used; convention dL = Re sum conj(gu_ij) dU_ij, i.e.
   2 dL/dconj(U), so gu = 2 (U - T) for L = sum |U - T|^2), returns U in cu and in grad (complex
   (ncp1, ndim, ndim), as cpot) the gradient of L with respect to the potential at the mesh
   points in the same convention (dL = Re sum conj(grad) dcpot); rows >= nr are zero.  With a
   symmetric potential (cpot(i, c, c') = cpot(i, c', c)) C(E) is complex symmetric, so the
   adjoint solution is the forward solution times a small matrix: one forward solve at the
   context's precision (refined; opts.reuse_factors applies).  Otherwise the forward runs on
   the FP64 path and the adjoint solve with C^T reuses its LU factors. */
int hprmat_b200_rmatrix_adjoint(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk, const double* eta,
                                double rmax, int nr, int ns, const double* cpot, int ncp1, int ndim, const double* gu,
                                double* cu, int* nopen, double* grad, hprmat_b200_stats* stats);

/* The two halves of the adjoint for a symmetric potential, for callers that run all forward
   solves before the gradients (reverse-mode autodiff): hprmat_b200_rmatrix_x is
   hprmat_b200_rmatrix (ns = 1) that also copies the refined forward solution X = C^-1 Q
   (complex FP64, nch*nr x nch, column-major, leading dimension ldx) into the device buffer d_x;
   hprmat_b200_adjoint_from_x then returns the potential gradient of hprmat_b200_rmatrix_adjoint
   from that X and the forward's U (host cu) without solving again (Y = X M2^T, C^T = C).  It
   returns HPRMAT_B200_ERR_UNSUPPORTED for a potential that is not symmetric. */
int hprmat_b200_rmatrix_x(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk, const double* eta,
                          double rmax, int nr, const double* cpot, int ncp1, int ndim, double* cu, int* nopen,
                          void* d_x, long ldx, hprmat_b200_stats* stats);
int hprmat_b200_adjoint_from_x(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk, const double* eta,
                               double rmax, int nr, const double* cpot, int ncp1, int ndim, const double* cu,
                               const void* d_x, long ldx, const double* gu, double* grad);

/* Device-resident variants of the two halves above, for callers whose potential already lives
   in device memory (a torch CUDA tensor in reverse-mode autodiff): d_cpot, d_cu, d_x and d_grad
   are device pointers; lval/qk/eta, cu and gu (O(nch^2)) stay host arrays.  The potential's
   symmetry is checked on the device (HPRMAT_B200_ERR_UNSUPPORTED when it is not symmetric). */
int hprmat_b200_rmatrix_x_device(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk, const double* eta,
                                 double rmax, int nr, const void* d_cpot, int ncp1, int ndim, void* d_cu, int* nopen,
                                 void* d_x, long ldx, hprmat_b200_stats* stats);
int hprmat_b200_adjoint_from_x_device(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk,
                                      const double* eta, double rmax, int nr, const void* d_cpot, int ncp1, int ndim,
                                      const double* cu, const void* d_x, long ldx, const double* gu, void* d_grad);

/* One J-pi block of a batched energy scan (hprmat_b200_rmatrix_scan).  The reference has no
   batched entry: its drivers call rmatrix once per energy in a host loop
   (examples/Ex1/example1_hp.f90:102-110, examples/Ex4/example4_hp.f90:118-134). */
typedef struct {
  int nch;              /* channels of the block */
  const int* lval;      /* [nch] angular momenta */
  const double* cpot;   /* host, complex (ncp1, nch, nch) Fortran order; energy independent */
  int ncp1;             /* leading dimension of cpot (>= nr) */
  int nenergies;        /* energies of this block */
  const double* qk;     /* [nenergies][nch] signed wave numbers (negative: closed) */
  const double* eta;    /* [nenergies][nch] Sommerfeld parameters */
  double* cu;           /* out: [nenergies] complex (nch, nch) collision matrices, as rmatrix's cu */
  int* nopen;           /* out: [nenergies] open channels */
  int* status;          /* out: [nenergies] status of each solve */
} hprmat_b200_scan_block;

/* Collision matrices of every (block, energy) unit, one interval on the mesh (nr, rmax) shared by
   all blocks, precision and refinement from the context's options.  Each block's potential is
   copied to the device once; the units run largest first on nworkers concurrent worker streams
   (0: 4), each with its own working buffers, kept by the context for later scans.  Returns
   HPRMAT_B200_OK, HPRMAT_B200_NOT_CONVERGED if some unit stopped above its tolerance, or the
   error of the first unit that failed (the other units still run); seconds receives the wall
   time of the call. */
int hprmat_b200_rmatrix_scan(hprmat_b200_ctx* ctx, int nblocks, const hprmat_b200_scan_block* blocks, double rmax,
                             int nr, int nworkers, double* seconds);

/* The same scan by a structure-exploiting method (no counterpart in the reference, which solves
   every energy by its own LU): between the energies of one block C(E) changes only by a common
   shift of its diagonal and by the closed channels' Bloch terms, rank one each,
   C(E) = C0 + delta(E) I + Q D(E) Q^T with Q = blockdiag(q2).  Each block's C0 is reduced once
   on the device to Hessenberg form, C0 = P H P^H (Householder similarity transformations, FP64);
   every energy then costs O(N^2 nch) -- an LU of H + delta I with row-pair pivoting, the
   back substitution for P^H Q, and the Woodbury identity for the Bloch terms on an nch x nch
   system -- followed by FP64 refinement steps against the structured C(E) (at most
   opts.max_refine; converged when a step changes R by less than opts.surface_tol, or when the
   error that step leaves is predicted a thousand times below it).  Energies are solved in
   batches of independent units per launch.  Up to three blocks are in flight at once, each on a
   worker context (stream, working buffers, host thread) that the context creates on the first
   scan and keeps, as hprmat_b200_rmatrix_scan's workers; the results do not depend on how the
   blocks are dealt.  Units the shifted form cannot take
   (blocks with more than 64 channels, channels whose energy terms do not move together, a zero
   Hessenberg or Woodbury pivot) run the LU path of hprmat_b200_rmatrix.  Outputs, statuses and
   return value as hprmat_b200_rmatrix_scan; precision is FP64 throughout. */
int hprmat_b200_rmatrix_scan_shifted(hprmat_b200_ctx* ctx, int nblocks, const hprmat_b200_scan_block* blocks,
                                     double rmax, int nr, double* seconds);

/* Scan autotuner, run before hprmat_b200_rmatrix_scan on the same blocks (or a sample of them).
   For every distinct order N = nch nr among the blocks it times one energy of the block (the
   middle one in the scan's energy order; the first or last if that solve fails) solved on all
   nworkers worker streams at once -- the load the scan itself puts on the device -- and picks,
   one setting at a time from the context's own, the LU block size (128, 64, 32), the panel
   variant (thread-block cluster or grid), the panel's fewest rows per CTA (16, 32, 64), the
   solves' super-block size (automatic, 2, 1), the FGMRES cycle length (12, 8, 16) and the CTAs of
   the persistent trailing update (one per SM, half, a quarter: concurrent solves share the
   SMs); a change
   is kept when it is 5% faster than the incumbent twice (against its best trial, then against
   a fresh one).  The resulting table replaces the context's; later scans
   apply each unit's row (units of other orders run with the context's settings).  seconds
   receives the wall time of the tuning. */
int hprmat_b200_scan_autotune(hprmat_b200_ctx* ctx, int nblocks, const hprmat_b200_scan_block* blocks, double rmax,
                              int nr, int nworkers, double* seconds);

/* The autotuner's table: up to max rows of 7 ints (N, LU block size, panel cluster 0/1, panel
   rows per CTA, solve super-block size, FGMRES cycle length, trailing-update CTAs with 0 for one
   per SM) into rows and the tuned trial time
   in ms into ms (either may be NULL).  Returns the number of rows in the table; -1 for a null
   context. */
int hprmat_b200_scan_tune_get(hprmat_b200_ctx* ctx, int* rows, double* ms, int max);

/* Replace the table with n rows of 7 ints as above (a table kept from an earlier tuning on the
   same device model); n = 0 clears it. */
int hprmat_b200_scan_tune_set(hprmat_b200_ctx* ctx, const int* rows, int n);

/* Collision matrix for one (J, pi, E): rmatrix(nch, lval, qk, eta, rmax, nr, ns, cpot, cu,
   ncp1, ndim, nopen, ...) of src/rmatrix_hp.F90:175-368, for local potentials (ncp2 = 0), on
   one interval or propagated over ns > 1 intervals (:326-345).  Host buffers: cpot is complex (ncp1, ndim, ndim), cu is complex
   (ndim, ndim) and receives U in cu(1:nopen, 1:nopen); the rest of cu is zeroed as in the
   reference (:221).  The mesh must have been set by hprmat_b200_rmat_ini with the same
   nr, ns and rmax.  stats may be NULL. */
int hprmat_b200_rmatrix(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk,
                        const double* eta, double rmax, int nr, int ns, const double* cpot,
                        int ncp1, int ndim, double* cu, int* nopen, hprmat_b200_stats* stats);

/* Same as hprmat_b200_rmatrix with cpot and cu in device memory (cu: ndim x ndim complex,
   column-major).  lval/qk/eta stay host arrays (O(nch)). */
int hprmat_b200_rmatrix_device(hprmat_b200_ctx* ctx, int nch, const int* lval,
                               const double* qk, const double* eta, double rmax, int nr,
                               int ns, const void* d_cpot, int ncp1, int ndim, void* d_cu,
                               int* nopen, hprmat_b200_stats* stats);

/* rmatrix with wave functions (twf = .true.; the cf, nwf1, nwf2, nc, nvc arguments of
   src/rmatrix_hp.F90:175-186, computed at :378-431): as hprmat_b200_rmatrix, and for the nc
   entrance channels nvc[0..nc-1] (1-based indices among the open channels) the internal wave
   functions at the mesh points zrma in cf, complex (nwf1, nwf2, nc) with nwf1 >= nr*ns and
   nwf2 >= nch (rows 1..nr*ns of channels 1..nch are written), and the closed-channel
   amplitudes in cu(nopen+1.., ic).  The wave function applies C^-1 to the surface amplitudes,
   as Descouvemont's original (rmat_pierre/rmatrix.f:286-301); HPRMAT's rmatrix_hp.F90:407
   multiplies by C instead.  Built from the per-interval solutions of the R-matrix step: no
   further factorisation or solve. */
int hprmat_b200_rmatrix_wf(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk,
                           const double* eta, double rmax, int nr, int ns, const double* cpot,
                           int ncp1, int ndim, double* cu, int* nopen, int nc, const int* nvc,
                           double* cf, int nwf1, int nwf2, hprmat_b200_stats* stats);

/* The complete argument list of rmatrix (src/rmatrix_hp.F90:175-186, host buffers): twf != 0
   adds the wave functions (cf, nwf1, nwf2, nc, nvc as hprmat_b200_rmatrix_wf); ncp2 > 0 adds the
   non-local potential cpnl, complex (ncp2, ndim, ndim) with ncp2 >= nr*nr: channel block
   (c, c') of C(E) gains sqrt(w_i w_j) a cpnl((i-1) nr + j, c, c') (:283-288), one interval only
   (ns = 1, as :205-209).  With a non-local potential the FP64 refinement multiplies by a dense
   FP64 copy of C(E) (N^2 complex doubles on the device). */
int hprmat_b200_rmatrix_full(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk,
                             const double* eta, double rmax, int nr, int ns, const double* cpot,
                             int ncp1, int ndim, double* cu, int* nopen, int twf, double* cf, int nwf1,
                             int nwf2, int nc, const int* nvc, int ncp2, const double* cpnl,
                             hprmat_b200_stats* stats);

/* Same with cpot, cu and cf in device memory. */
int hprmat_b200_rmatrix_wf_device(hprmat_b200_ctx* ctx, int nch, const int* lval, const double* qk,
                                  const double* eta, double rmax, int nr, int ns, const void* d_cpot,
                                  int ncp1, int ndim, void* d_cu, int* nopen, int nc, const int* nvc,
                                  void* d_cf, int nwf1, int nwf2, hprmat_b200_stats* stats);

/* wf_print (src/rmatrix_hp.F90:678-734): the wave function of channel iv for entrance channel
   nom (both 1-based) at r = h, 2h, ..., npoin*h into cwftab (complex, npoin): a natural cubic
   spline of cf(1:nr*ns, iv, nom) over zrma for r <= rmax, the Coulomb (open) or Whittaker
   (closed) form with the amplitudes of cu beyond.  Host computation, no context. */
int hprmat_b200_wf_print(int nch, const int* lval, const double* qk, const double* eta, double rmax, int nr,
                         int ns, const double* cu, int ndim, int nopen, const double* cf, int nwf1,
                         int nwf2, const double* zrma, int iv, int nom, int npoin, double h,
                         double* cwftab);

/* Dense solve C X = B: the solve inside solve_rmatrix (src/rmat_solvers.F90:49-90), same
   layout as gpu_solve_mixed_ (src/cusolver_interface.cu:321-443).  A (n x n complex,
   column-major) is read only; B (n x nrhs complex) is overwritten with X.  Host buffers. */
int hprmat_b200_solve_linear(hprmat_b200_ctx* ctx, const double* A, double* B, int n,
                             int nrhs, hprmat_b200_stats* stats);
/* Same with A and B in device memory. */
int hprmat_b200_solve_linear_device(hprmat_b200_ctx* ctx, const void* d_A, void* d_B, int n,
                                    int nrhs, hprmat_b200_stats* stats);

/* solve_rmatrix(cmat, B_vector, nch, nlag, normfac, Rmat, solver_type=7)
   (src/rmat_solvers.F90:49-90 and the R extraction of :135-144): solves with the nch
   channel-surface right-hand sides blockdiag(B_vector) and returns
   Rmat(i, j) = normfac * sum_r B(r) X((i-1)*nlag + r, j) (bilinear, no conjugate).
   Host buffers: cmat (N x N), bvec (nlag), rmat (nch x nch), all complex. */
int hprmat_b200_solve_rmatrix(hprmat_b200_ctx* ctx, const double* cmat, const double* bvec,
                              int nch, int nlag, double normfac, double* rmat,
                              hprmat_b200_stats* stats);

/* Fortran-convention drop-ins (arguments by reference, trailing underscore) for the
   reference's C ABI, bound in src/gpu_solver_interface.F90:61-99.  They use a context on
   device 0 created on first use.  Return 0 on success, -1 on error; *info as in the
   reference (0 ok, -1 init, -2 alloc, >0 singular pivot, 99 refinement not converged). */
int gpu_b200_solve_mixed_(double* A, double* B, int* n, int* nrhs, int* max_refine,
                          double* tol, int* info);  /* cf. gpu_solve_mixed_  :321-329 */
int gpu_b200_solve_double_(double* A, double* B, int* n, int* nrhs,
                           int* info);              /* cf. gpu_solve_double_ :737-795 */
int gpu_b200_finalize_(void);                       /* cf. gpu_solver_finalize_ :222 */

/* Dense FP64 solve A X = B of small systems that allocates no device memory.  No
   counterpart in the reference: it is for callers that must not call cudaMalloc -- code that
   runs the solver inside another framework's device memory pool (where a cudaMalloc fails
   once the pool has reserved the memory) or in a latency-critical loop (where cudaFree
   stalls the whole device).  Same algorithm and kernels as the FP64 path of
   hprmat_b200_solve_linear_device; its working memory is a fixed array of about 5.8 MB
   inside the library that every GPU loading the library holds until the process exits.
   Limits: n <= 512, nrhs <= 64 (larger sizes return HPRMAT_B200_ERR_UNSUPPORTED).
   d_A (n x n complex double, column-major, read only) and d_B (n x nrhs, overwritten with
   X) are device pointers; the work is ordered on `stream` (a cudaStream_t, NULL = default
   stream) and complete when the call returns.  *info (may be NULL) receives the first zero
   pivot (1-based) when the status is HPRMAT_B200_SINGULAR.
   Every call looks up the array's device address on the current device
   (cudaGetSymbolAddress), so a device reset does not leave a stale address behind; the
   first call on a device also loads the array there, so make it before any stream capture.
   All calls share the one array: calls whose GPU work overlaps (other threads or streams)
   race and must be serialised by the caller. */
int hprmat_b200_solve_linear_noalloc(const void* d_A, void* d_B, int n, int nrhs, void* stream,
                                     int* info);

/* Boundary values of the R-matrix -> collision-matrix step at the channel radius a = rmax,
   per channel, as computed in rmatrix (src/rmatrix_hp.F90:224-244).  Host only, needs no
   GPU.  Open channels (qk > 0): co = G + iF and cop = (G' + iF') k a from COULFG
   (src/special_functions.f:1-275).  Closed channels: xc1 = a W'/W and xc2 = W from WHIT
   (src/special_functions.f:309-416).  co/cop are complex (nch entries each), xc1/xc2 real;
   entries that do not apply to a channel are zero.  Any output may be NULL. */
int hprmat_b200_boundary(int nch, const int* lval, const double* qk, const double* eta, double rmax,
                         double* co, double* cop, double* xc1, double* xc2, int* nopen);

/* Human-readable status and the last CUDA error message of this thread's calls. */
const char* hprmat_b200_status_string(int status);
const char* hprmat_b200_last_error(void);

/* Version of the ABI: the structs above and the entry points' signatures.  It changes whenever
   one of them does (101: stats gained factorizations, fp64_fallback, pivot_growth,
   cond_estimate and ms_condest; opts gained estimate_condition and growth_error).  A caller
   built against another value must be rebuilt. */
#define HPRMAT_B200_ABI_VERSION 101
int hprmat_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif /* HPRMAT_B200_H */

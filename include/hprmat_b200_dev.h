/*
 * hprmat_b200_dev.h -- kernel-level entry points of libhprmat_b200.so for tests and
 * benchmarks.  They run one device kernel of the solver on caller-provided device buffers,
 * ordered on the context's stream, and return after it completes.  They are not part of
 * the HPRMAT interface and have no counterpart in the reference.
 */
#ifndef HPRMAT_B200_DEV_H
#define HPRMAT_B200_DEV_H
#include "hprmat_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

/* C[M x Nc] -= A * B on the tensor cores: C complex float (interleaved, column-major, ldc),
   A and B as 4 planes (Re hi, Re lo, Im hi, Im lo of the TF32 split), K-major with nb
   floats per row / column, planes `plane` floats apart (the LU's operand buffers).
   nb a multiple of 16; bn = 128 or 256 columns per tile. */
int hprmat_b200_dev_tc_update(hprmat_b200_ctx* ctx, const float* aop, const float* bop, long plane, int nb,
                              void* C, long ldc, int M, int Nc, int bn);

/* C[M x N] -= A[M x K] B[K x N] in complex FP64 on the FP64 tensor cores (the DMMA kernel of the
   FP64 path's trailing updates, solves and dense residuals): device pointers to interleaved
   complex doubles, column-major with leading dimensions lda >= M, ldb >= K, ldc >= M. */
int hprmat_b200_dev_zgemm(hprmat_b200_ctx* ctx, const void* A, long lda, const void* B, long ldb, void* C, long ldc,
                          int M, int N, int K);

/* Householder reduction of A (device, N x N complex double, column-major, lda) in place to upper
   Hessenberg form H with A = P H P^H; P (device, N x N, leading dimension lda) receives the
   accumulated unitary factor.  The reduction of the shifted energy scan. */
int hprmat_b200_dev_hessenberg(hprmat_b200_ctx* ctx, void* A, long lda, int N, void* P);

/* Phase times of the shifted scans run on the context while profiling is enabled
   (hprmat_b200_dev_set_profile): ms[6] = reduction to Hessenberg form (with the assembly of C0),
   per-energy Hessenberg solves, products for S, T and X, refinement steps, collision matrices,
   units run by the LU path; counts[2] = refinement steps of the last batch, units sent to the LU
   path by the last scan.  reset != 0 clears the times. */
int hprmat_b200_dev_hess_timings(hprmat_b200_ctx* ctx, double* ms, int* counts, int reset);

/* Split complex float values into the 4 TF32 planes used by hprmat_b200_dev_tc_update:
   src is rows x nb (row-major complex float, i.e. K contiguous), dst gets 4 planes of
   rows x nb floats, `plane` floats apart. */
int hprmat_b200_dev_split_planes(hprmat_b200_ctx* ctx, const void* src, int rows, int nb, float* dst, long plane);

/* Benchmark counters.  With profiling enabled, every tensor-core trailing update of a
   factorisation is bracketed by CUDA events on the context's stream; the counters
   accumulate their elapsed time (ms), their algorithmic flops (8 M^2 nb per launch, the
   complex-LU convention) and their number.  `launches` counts every kernel the library
   launched on the context.  reset != 0 clears them after reading. */
int hprmat_b200_dev_set_profile(hprmat_b200_ctx* ctx, int enable);
int hprmat_b200_dev_counters(hprmat_b200_ctx* ctx, unsigned long long* launches, double* tc_ms, double* tc_flops,
                             int* tc_launches, int reset);

/* Tuning knobs for benchmarks and experiments (defaults in parentheses):
     "wave_un"        right-hand sides per unit of the wavefront solves: 64, 128 (0: 128 when
                      nrhs > 64, else 64);
     "wave_sb"        blocks per diagonal super block of the solves' scaled factors: 1, 2, 4
                      (0: 4, or 2 below 4 blocks); takes effect at the next factorisation;
     "wave"           wavefront solves on/off (1);
     "tc_trsm"        U12 by a tensor-core product with L11^-1 (1) or by substitution (0);
     "panel_rpc_min"  fewest panel rows per CTA (32);
     "panel_cluster"  panels that fit in one cluster of at most 16 CTAs exchange pivots in
                      distributed shared memory (1) or always through global memory (0);
     "tc_grid"        most CTAs of the persistent trailing update (0: one per SM);
     "growth_limit_exp" mixed path: an FP32 factorisation whose pivot growth exceeds 10^value
                      (-30..30) is replaced by the FP64 one (6);
     "gmres_m"        longest FGMRES cycle, <= 16 (12);
     "inner_tol0_exp" first cycle runs until the residual fell 10^-value (7);
     "zero_start"     refinement from X = 0 instead of the FP32 solution (0);
     "reuse_max_inner" with opts.reuse_factors, factorise again once a solve on the held
                      factors needed more FGMRES iterations than this (24);
     "f64_pair"       plain FP64 LU: two 64-column block steps share one K = 128 trailing
                      update (1) or each step updates on its own (0);
     "hess_blocked"   shifted scan: blocked Hessenberg reduction (1) or one reflector at a
                      time (0);
     "hess_cluster"   CTAs of the blocked reduction's column-step cluster: 8, 16, or 0 to
                      take 16 where the GPU holds such a cluster;
     "hess_workers"   shifted scan: J-pi blocks in flight at once, each on a worker context
                      of its own, 1..8 (3). */
int hprmat_b200_dev_set_tuning(hprmat_b200_ctx* ctx, const char* key, int value);

/* Failure-path check: one CTA waits, with a limit of `spins` polls (4096 .. 2^24), on a device
   counter that nothing increments -- the bounded wait of the panel's grid barrier.  Returns
   HPRMAT_B200_ERR_TIMEOUT with the site in the error message when the wait gave up, as it is
   meant to (the context stays usable); any other value is a failure of the check. */
int hprmat_b200_dev_wait_probe(hprmat_b200_ctx* ctx, int spins);

/* The binary architecture the library's kernels were compiled for, as the CUDA runtime reports
   it for one of them (cudaFuncAttributes.binaryVersion: 100 for sm_100a), on the current
   device; a negative status when no device can load them. */
int hprmat_b200_dev_binary_version(void);

/* LU factorisations run on the context and its scan workers since the last reset (opts.reuse_factors
   makes energy scans run fewer); reset != 0 clears the count after reading.  -1 for a null
   context. */
long long hprmat_b200_dev_factorizations(hprmat_b200_ctx* ctx, int reset);

/* The Lagrange-mesh matrices the device assembly uses, computed on the host (no context, no
   device): for every interval is (0-based, interval-major) tc[is][nr x nr] (kinetic + Bloch,
   column-major, / rmax0^2), blo[is][nr x nr] (the closed-channel Bloch matrix times rmax0:
   blo0 / rmax0 for the first interval, (blo2 / (is+1) - blo1 / is) / rmax0 after it), q2[is][nr],
   q1[is][nr] and zrma[nr ns] -- src/rmatrix_hp.F90:61-159 with rmax0 = rmax / ns.  Any output
   may be NULL. */
int hprmat_b200_dev_mesh(int nr, int ns, double rmax, double* tc, double* blo, double* q2, double* q1,
                         double* zrma);

/* Tracing of the wavefront triangular solves of the mixed path.  With enable != 0 every
   later sweep records, per unit (block row x right-hand-side group, in dependency order),
   four device-clock stamps in ns: the producer starts the unit, the last dependency flag
   was seen, the accumulator was complete, the block was published.
   hprmat_b200_dev_wave_trace_read copies the stamps of the last forward sweep followed by
   the last backward sweep (2 x units x 4 values, at most cap) and stores units. */
int hprmat_b200_dev_wave_trace(hprmat_b200_ctx* ctx, int enable);
int hprmat_b200_dev_wave_trace_read(hprmat_b200_ctx* ctx, long long* out, int cap, int* units);
/* With tracing enabled, the panel factorisations of block steps 0 and nsteps/2 also record
   per column `width` device-clock stamps: CTA 0 at column start, candidate posted, grid
   barrier passed, pivot row in place, update done, then each CTA's barrier arrival.
   Copies 2 x 128 x width values (at most cap). */
int hprmat_b200_dev_panel_trace_read(hprmat_b200_ctx* ctx, long long* out, int cap, int* width);

#ifdef __cplusplus
}
#endif
#endif

// Triangular solves of the mixed-precision LU as two persistent "wavefront" kernels on the
// tensor cores, plus the one-time preparation of the factors they read.
//
// After the blocked LU (nb = 128, row interchanges applied only to the right of each panel)
// the preparation
//   1. composes the row interchanges into, per block column k, the map from a final row
//      position to the row that held it after step k (sigma_k), and the final permutation;
//   2. copies the off-diagonal blocks, L rows gathered into their final order, transposed
//      into T (column-major TF32 planes);
//   3. writes the explicit inverses of the diagonal blocks (L_jj^-1, U_jj^-1) as planes;
//   4. replaces every off-diagonal block of the LU planes by its block-row scaled form
//        L'[j,k] = L_jj^-1 L[j,k]  (k < j),   U'[j,k] = U_jj^-1 U[j,k]  (k > j),
//      one 128 x 128 x 128 complex tensor-core product per block.
// A solve is then
//   forward   Y_j = L_jj^-1 (P B)_j - sum_{k<j} L'[j,k] Y_k
//   backward  X_j = U_jj^-1 Y_j     - sum_{k>j} U'[j,k] X_k
// each one persistent kernel: a unit is (block row j, group of UN right-hand sides); its
// accumulator lives in TMEM while its CTA streams the blocks of row j and the published
// solution blocks; the epilogue publishes block j through a per-unit flag.
// With super blocks of sb blocks the diagonal inverses are those of the sb*128-row diagonal
// blocks (built by doubling from the 128-row ones) and the sums skip the blocks of the own
// super block, so the sb block rows of a super block do not depend on each other and the
// dependency chain has nsteps / sb links.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <vector_types.h>

#include "tc_gemm.cuh"

namespace hprmat {

// sigma maps and the final permutation from the per-step interchange lists.
//   swaps: per step (stride swap_stride ints) top_src[kMaxNB], extra_dst[kMaxNB],
//          extra_src[kMaxNB], n_extra.
//   work:  2 N ints of scratch;  sig: nsteps rows of sig_ld ints;  perm0: N ints, the
//          original row of final position i.
int wave_perm_chain(const int* swaps, int swap_stride, int N, int nsteps, int* work, int* sig, long sig_ld,
                    int* perm0, cudaStream_t s);

// T[c][i] (column-major planes, ld ldt, plane tplane) = block (i, c) of the LU planes, rows
// of L blocks gathered through sigma; diagonal blocks are left untouched.
int wave_transpose_offdiag(const float* lup, long lup_ld, long lup_plane, const int* sig, long sig_ld, int N,
                           int nsteps, float* T, long ldt, long tplane, cudaStream_t s);

// DI planes, row-major h x h per block: row (2 J + u) * h + i (u = 0 for L_JJ^-1, 1 for
// U_JJ^-1), from the column-major float2 inverses inv[(2 J + u) * h * h], nblk blocks.
int wave_dinv_planes(const float2* inv, int nblk, int h, float* di, long di_plane, cudaStream_t s);

// Inverses of the 2h x 2h diagonal super blocks from those of the h x h blocks (dfh, nblk
// blocks) and the off-diagonal blocks in T; ptmp, otmp: 2 ceil(nblk/2) h^2 float2 each;
// df2h: 2 ceil(nblk/2) (2h)^2 float2.
int wave_dinv_double(const float2* dfh, int h, int nblk, const float* T, long ldt, long tplane, int N, float2* ptmp,
                     float2* otmp, float2* df2h, cudaStream_t s);

// Off-diagonal blocks of the LU planes outside the diagonal super blocks (sb blocks each)
// <- D_JJ^-1 * (block from T), on the tensor cores.
int wave_scale_offdiag(TcGemmPlan& p, const TcOperand& opD, const TcOperand& opT, int N, int nsteps, int sb,
                       float* lup, long lup_ld, long lup_plane, cudaStream_t s);

// B-operand planes of (P B): bp[p][c][i] = split(X[perm0[i] + c ldx]), i < N, c < nrhs.
int wave_rhs_planes(const float2* X, long ldx, const int* perm0, int N, int nrhs, float* bp, long bld, long bplane,
                    cudaStream_t s);

struct WaveSolve {
  int N = 0, nsteps = 0, nrhs = 0;
  int sb = 1;                  // blocks per diagonal super block of the scaled factors
  int un = 64;                 // right-hand sides per unit (64 or 128)
  float* xp = nullptr;         // output planes (column c, row i at xp[p*xp_plane + c*xp_ld + i])
  long xp_ld = 0, xp_plane = 0;
  float2* xout = nullptr;      // optional FP32 complex output (N x nrhs, ldx)
  long ldx = 0;
  int* flags = nullptr;        // [nsteps x groups] publication counters, zeroed by the sweep
  long long* trace = nullptr;  // optional: 4 device-clock stamps per unit
};

// One triangular sweep.  forward: A blocks from opM (L'), diagonal opD rows 2j, right side
// opB0, published blocks read back through opX (a view of ws.xp).  backward: U' and rows
// 2j + 1.  Cooperative launch of min(units, SMs) CTAs.
int wave_sweep(TcGemmPlan& p, bool forward, const TcOperand& opM, const TcOperand& opD, const TcOperand& opB0,
               const TcOperand& opX, const WaveSolve& ws, cudaStream_t s);

}  // namespace hprmat

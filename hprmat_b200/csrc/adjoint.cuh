// Adjoint of the collision matrix: solves with C^T from the FP64 LU factors of the forward solve
// and the gradient with respect to the potential at the mesh points.
//
// The forward solve applies, per block step s, the step's row interchanges P_s, the inverse of
// the unit-lower diagonal block and the update of the rows below (L21), then backwards the
// inverse of the upper diagonal block and the update of the rows above (U12).  C^-T is the
// product of the transposed step operators in the reverse order:
//   for s = 0 .. last:  X_s -= U(rows < s, s)^T X(rows < s);  X_s <- (U_ss^-1)^T X_s
//   for s = last .. 0:  X_s -= L(rows > s, s)^T X(rows > s);  X_s <- (L_ss^-1)^T X_s;  X <- P_s^-1 X
// with the factors exactly as stored (interchanges never applied to the left of a panel).
#pragma once
#include "common.cuh"

namespace hprmat {

// partial[sp][j + ncols * col] = sum over rows r of split sp of A(r, j) Y(r, col), for the
// rows [r0, r1) of A (column block of ncols <= 64 columns at acol, column-major, lda) and of Y
// (ldy), nrhs <= 128.  grid (nsplit), 256 threads; rows staged 8 at a time.
__global__ void __launch_bounds__(256) trans_partial_kernel(const double2* __restrict__ A, long lda, int acol,
                                                            int ncols, const double2* __restrict__ Y, long ldy,
                                                            int nrhs, int r0, int r1, int rows_per_split,
                                                            double2* partial) {
  constexpr int RB = 8;
  __shared__ double2 As[RB][64];
  __shared__ double2 Ys[RB][128];
  const int sp = blockIdx.x;
  const int a0 = r0 + sp * rows_per_split;
  const int a1 = min(r1, a0 + rows_per_split);
  const int tid = threadIdx.x;
  // thread -> outputs (j, col) = (tid % 64, tid / 64 + 4 q), q < 32: up to 64 x 128 outputs
  const int j = tid & 63;
  const int cb = tid >> 6;
  double2 acc[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) acc[q] = make_double2(0.0, 0.0);
  for (int rb = a0; rb < a1; rb += RB) {
    const int nrow = min(RB, a1 - rb);
    for (int idx = tid; idx < RB * 64; idx += 256) {
      const int r = idx % RB, jj = idx / RB;
      As[r][jj] = (r < nrow && jj < ncols) ? A[(size_t)(rb + r) + (size_t)(acol + jj) * lda] : make_double2(0.0, 0.0);
    }
    for (int idx = tid; idx < RB * 128; idx += 256) {
      const int r = idx % RB, c = idx / RB;
      Ys[r][c] = (r < nrow && c < nrhs) ? Y[(size_t)(rb + r) + (size_t)c * ldy] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int r = 0; r < nrow; ++r) {
      const double2 a = As[r][j];
#pragma unroll
      for (int q = 0; q < 32; ++q)
        if (cb + 4 * q < nrhs) cfma(acc[q], a, Ys[r][cb + 4 * q]);  // few right-hand sides: skip the rest
    }
    __syncthreads();
  }
  if (j < ncols)
#pragma unroll
    for (int q = 0; q < 32; ++q) {
      const int col = cb + 4 * q;
      if (col < nrhs) partial[(size_t)sp * ncols * 128 + j + (size_t)ncols * col] = acc[q];
    }
}

// X(k0 + j, col) -= sum_sp partial[sp][j + ncols col]  (splits summed in order)
__global__ void trans_reduce_kernel(const double2* __restrict__ partial, int nsplit, int ncols, int nrhs, double2* X,
                                    long ldx, int k0) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ncols * nrhs) return;
  const int j = idx % ncols, col = idx / ncols;
  double2 s = make_double2(0.0, 0.0);
  for (int sp = 0; sp < nsplit; ++sp) {
    const double2 v = partial[(size_t)sp * ncols * 128 + idx];
    s.x += v.x;
    s.y += v.y;
  }
  double2* x = X + (size_t)(k0 + j) + (size_t)col * ldx;
  x->x -= s.x;
  x->y -= s.y;
}

// X(k0.., col) <- Tinv^T X(k0.., col) with Tinv (NB x NB, column-major; ncols valid).  One
// CTA per right-hand side.
__global__ void __launch_bounds__(128) diag_trans_kernel(const double2* __restrict__ Tinv, int NB, int ncols, int k0,
                                                         double2* X, long ldx) {
  __shared__ double2 xs[256];
  const int col = blockIdx.x;
  double2* x = X + (size_t)col * ldx + k0;
  for (int i = threadIdx.x; i < ncols; i += blockDim.x) xs[i] = x[i];
  __syncthreads();
  for (int i = threadIdx.x; i < ncols; i += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int jj = 0; jj < ncols; ++jj) cfma(acc, Tinv[jj + (size_t)i * NB], xs[jj]);  // (Tinv^T)(i, jj)
    x[i] = acc;
  }
}

// X <- P_s^-1 X for the step's interchange list: the forward step moved row src(q) to q for
// the touched positions q, so row q goes back to src(q).  One CTA per right-hand side.
__global__ void __launch_bounds__(256) perm_inv_kernel(const int* __restrict__ sw, int kmaxnb, int k0, int ncols,
                                                       double2* X, long ldx) {
  __shared__ double2 v[512];
  __shared__ int dst[512];
  const int col = blockIdx.x;
  const int ne = sw[3 * kmaxnb];
  const int cnt = ncols + ne;
  double2* x = X + (size_t)col * ldx;
  for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
    const int q = t < ncols ? k0 + t : sw[kmaxnb + (t - ncols)];
    const int src = t < ncols ? sw[t] : sw[2 * kmaxnb + (t - ncols)];
    v[t] = x[q];
    dst[t] = src;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < cnt; t += blockDim.x) x[dst[t]] = v[t];
}

// grad(i, c, c') = -conj(sum_col Y[(c,i), col] X[(c',i), col]) * scale at the mesh points
// (complex (ncp1, ndim, ndim) Fortran layout); grid (nr, nch), thread c'.
__global__ void potential_grad_kernel(const double2* __restrict__ Y, const double2* __restrict__ X, long ld, int nr,
                                      int nch, int ncol, double scale, double2* grad, long ncp1, long ndim) {
  const int i = blockIdx.x, c = blockIdx.y;
  for (int cp = threadIdx.x; cp < nch; cp += blockDim.x) {
    double2 h = make_double2(0.0, 0.0);
    for (int col = 0; col < ncol; ++col)
      cfma(h, Y[(size_t)(c * nr + i) + (size_t)col * ld], X[(size_t)(cp * nr + i) + (size_t)col * ld]);
    grad[(size_t)i + ncp1 * ((size_t)c + ndim * (size_t)cp)] = make_double2(-h.x * scale, h.y * scale);
  }
}

// Sets *flag when the potential (complex (ncp1, ndim, ndim), rows < nr) is not symmetric in its
// channel indices: cpot(i, c, c') != cpot(i, c', c) for some mesh point i.  Grid (rows / 128,
// nch, nch), exact comparison as the host check does.
__global__ void potential_asym_kernel(const double2* __restrict__ cpot, long ncp1, long ndim, int nr, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y, cp = blockIdx.z;
  if (i >= nr || cp >= c) return;
  const double2 a = cpot[(size_t)i + ncp1 * ((size_t)c + ndim * (size_t)cp)];
  const double2 b = cpot[(size_t)i + ncp1 * ((size_t)cp + ndim * (size_t)c)];
  if (a.x != b.x || a.y != b.y) atomicExch(flag, 1);
}

}  // namespace hprmat

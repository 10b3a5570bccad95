// Complex FP64 GEMM update C -= A B of the plain FP64 path (trailing update of the FP64 LU,
// block updates of its triangular solves, the dense-operator residual of the refinement), on
// the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64).
#pragma once
#include <cuda_runtime.h>
#include <vector_types.h>

namespace hprmat {

// C[M x N] -= A[M x K] B[K x N]; A, B, C complex double (interleaved), column-major with
// leading dimensions lda, ldb, ldc (in complex elements).  Ordered on stream s.  Returns 0 or a
// negative status (launch error; message in the library's last error).
int zgemm_f64_update(int M, int N, int K, const double2* A, long lda, const double2* B, long ldb, double2* C,
                     long ldc, cudaStream_t s);

// The same for `batch` independent problems in one launch: problem z uses A + z sA, B + z sB,
// C + z sC (strides in complex elements; a stride 0 shares that operand).  A shared A (sA = 0)
// with sB = ldb N and sC = ldc N is computed as one problem of batch N columns.
int zgemm_f64_update_batched(int M, int N, int K, const double2* A, long lda, long sA, const double2* B, long ldb,
                             long sB, double2* C, long ldc, long sC, int batch, cudaStream_t s);

}  // namespace hprmat

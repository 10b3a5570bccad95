// Trailing update of the mixed-precision LU on the 5th-generation tensor cores.
#pragma once
#include <cuda_runtime.h>
#include <vector_types.h>

namespace hprmat {

struct TcGemmPlan {
  int device = -1;
  int nsm = 0;
  void* encode = nullptr;  // cuTensorMapEncodeTiled, fetched through the runtime
  int* d_err = nullptr;    // device word: nonzero if a bounded wait gave up
};

int tc_gemm_init(TcGemmPlan& p, int device);

// C[M x Nc] -= A * B for complex C (float2, column-major, ldc) with A and B given as the
// hi/lo TF32 splits of their real and imaginary parts ("planes" 0..3 = Re hi, Re lo,
// Im hi, Im lo), K-major with NB values per row (A: M rows, B: Nc columns), planes
// `plane` floats apart.  K = NB (zero padded).
int tc_trailing_update(TcGemmPlan& p, const float* aop, const float* bop, long plane, int NB, int K, float2* C,
                       long ldc, int M, int Nc, cudaStream_t s);

// Reads and clears the device error word (0 = no wait gave up).
int tc_gemm_check(TcGemmPlan& p, cudaStream_t s, int* err_out);

}  // namespace hprmat

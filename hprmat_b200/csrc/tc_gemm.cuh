// Complex GEMM updates of the mixed-precision LU and of its triangular solves on the
// 5th-generation tensor cores.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <vector_types.h>

namespace hprmat {

struct TcGemmPlan {
  int device = -1;
  int nsm = 0;
  void* encode = nullptr;  // cuTensorMapEncodeTiled, fetched through the runtime
  int* d_err = nullptr;    // device word: nonzero if a bounded wait gave up
  int max_grid = 0;        // most CTAs of a persistent update (0: one per SM); concurrent
                           // solves (scan workers) leave SMs to each other with a smaller grid
};

// A TMA view of an operand stored as 4 planes of floats (Re hi, Re lo, Im hi, Im lo of the
// TF32 split), each plane `rows` rows of `kext` contiguous K values (row stride `ld`
// floats, plane stride `plane` floats).  Boxes are 16 K values x box_rows rows x 4 planes.
struct TcOperand {
  CUtensorMap map;
  long kext = 0, rows = 0;
};

int tc_gemm_init(TcGemmPlan& p, int device);
int tc_make_operand(TcGemmPlan& p, TcOperand& op, const float* base, long kext, long rows, long ld, long plane,
                    int box_rows);

// C[M x Nc] -= A * B for complex C (float2, column-major, ldc).  Row m of A is operand row
// a_row0 + m, K values a_k0 .. a_k0 + K - 1; column n of B is operand row b_row0 + n, K values
// b_k0 ...  K is a multiple of 16.  bn = 128 or 256 columns per tile (the B view must have
// been made with box_rows = bn, the A view with box_rows = 128).
int tc_update(TcGemmPlan& p, const TcOperand& A, int a_k0, int a_row0, const TcOperand& B, int b_k0, int b_row0,
              int K, float2* C, long ldc, int M, int Nc, int bn, cudaStream_t s);

// Reads and clears the device error word (0 = no wait gave up).
int tc_gemm_check(TcGemmPlan& p, cudaStream_t s, int* err_out);

}  // namespace hprmat

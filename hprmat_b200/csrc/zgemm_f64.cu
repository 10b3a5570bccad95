// Complex FP64 GEMM update C -= A B on the FP64 tensor cores (sm_100a DMMA).
//
// The plain FP64 path of the solver (the "plain FP64 device LU" the mixed path is measured
// against, the mixed path's FP64 fallback, the condition estimate and the non-symmetric
// adjoint) spends its O(N^3) work in one shape of product: C[M x N] -= A[M x K] B[K x N] with
// complex double operands in column-major storage -- the LU's trailing update (K = the block
// size), the block updates of its triangular solves, and the dense operator's residual
// B - C X of the refinement (K = N).
//
// Each complex product is 4 real products on mma.sync.aligned.m8n8k4.f64 (DMMA):
//   Re += Ar Br + (-Ai) Bi,   Im += Ar Bi + Ai Br,
// FP64 products and FP64 accumulation throughout.  A CTA of 4 warps computes 64 x 64 complex
// tiles of C (each warp 32 x 32: 4 x 4 blocks of 8 x 8, Re and Im accumulators in registers),
// two persistent CTAs per SM, over K in chunks of 16 staged in shared memory by cp.async in a
// 3-deep ring that runs on across the CTA's tiles:
//   A chunk as [k][m] (m contiguous, as A's columns), row stride 66 complex, and
//   B chunk as [n][k] (k contiguous, as B's columns), row stride 20 complex,
// so that the fragment loads -- one 16-byte (re, im) load per 8 x 4 A block and per 4 x 8 B
// block -- hit 8 distinct 16-byte bank groups in every quarter warp.  Elements beyond M, N or K
// are zero-filled by the copies (src-size 0) and never stored.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "zgemm_f64.cuh"

namespace hprmat {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16;
constexpr int kStages = 3;
constexpr int kThreads = 128;
constexpr int kALd = kBM + 2;  // complex elements per k row of the A stage
constexpr int kBLd = kBK + 4;  // complex elements per n row of the B stage
constexpr int kAStage = kBK * kALd;
constexpr int kBStage = kBN * kBLd;
constexpr size_t kSmemBytes = (size_t)kStages * (kAStage + kBStage) * sizeof(double2);

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, bool valid) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  const int n = valid ? 16 : 0;  // 0: nothing read, 16 zero bytes written
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// d += a b for one 8 x 8 x 4 FP64 block (fragments as mma.m8n8k4 .f64 lays them out: a at
// row lane/4, column lane%4; b at row lane%4, column lane/4; d at row lane/4, columns
// 2 (lane%4) and 2 (lane%4) + 1).
// Not volatile: the compiler may interleave independent products to hide the DMMA latency.
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Persistent: a CTA walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... of all batch
// problems (rows fastest), and its K chunks form one stream across its tiles, so the ring
// prefetches the next tile's first chunks while the current tile finishes and writes C.
__global__ void __launch_bounds__(kThreads, 2)
    zgemm_dmma_kernel(int M, int N, int K, const double2* __restrict__ A, long lda, const double2* __restrict__ B,
                      long ldb, double2* __restrict__ C, long ldc, long sA, long sB, long sC, int batch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* As = reinterpret_cast<double2*>(smem_raw);
  double2* Bs = As + kStages * kAStage;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int nchunks = (K + kBK - 1) / kBK;
  const int mt = (M + kBM - 1) / kBM, nt = (N + kBN - 1) / kBN;
  const long ntiles = (long)mt * nt * batch;
  const long mytiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long nstream = mytiles * nchunks;  // chunks of all this CTA's tiles

  // chunk g of the stream -> its tile's operands
  auto load_chunk = [&](long g) {
    const long t = blockIdx.x + (g / nchunks) * (long)gridDim.x;
    const int kc = (int)(g % nchunks);
    const int z = (int)(t / ((long)mt * nt));
    const int r = (int)(t % ((long)mt * nt));
    const int m0 = (r % mt) * kBM, n0 = (r / mt) * kBN, k0 = kc * kBK;
    const double2* Az = A + (size_t)z * sA;
    const double2* Bz = B + (size_t)z * sB;
    const int stage = (int)(g % kStages);
    double2* as = As + stage * kAStage;
    double2* bs = Bs + stage * kBStage;
#pragma unroll
    for (int i = 0; i < (kBM * kBK) / kThreads; ++i) {
      const int idx = tid + i * kThreads;
      const int k = idx / kBM, m = idx % kBM;
      const bool ok = (m0 + m < M) && (k0 + k < K);
      const double2* src = ok ? Az + (size_t)(m0 + m) + (size_t)(k0 + k) * lda : Az;
      cp_async16(as + k * kALd + m, src, ok);
    }
#pragma unroll
    for (int i = 0; i < (kBN * kBK) / kThreads; ++i) {
      const int idx = tid + i * kThreads;
      const int n = idx / kBK, k = idx % kBK;
      const bool ok = (n0 + n < N) && (k0 + k < K);
      const double2* src = ok ? Bz + (size_t)(k0 + k) + (size_t)(n0 + n) * ldb : Bz;
      cp_async16(bs + n * kBLd + k, src, ok);
    }
  };

  double accr[4][4][2], acci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      accr[i][j][0] = accr[i][j][1] = 0.0;
      acci[i][j][0] = acci[i][j][1] = 0.0;
    }

#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nstream) load_chunk(s);
    cp_async_commit();
  }
  const int fr = lane >> 2, fk = lane & 3;
  for (long g = 0; g < nstream; ++g) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    // refill the slot consumed in the previous iteration (every warp has passed the barrier)
    if (g + kStages - 1 < nstream) load_chunk(g + kStages - 1);
    cp_async_commit();
    if (g % nchunks == 0) {
      // a new tile: its C lines (64 columns of 64 x 16 bytes) go to L2 now, so that the
      // epilogue's loads of C meet them there
      const long t = blockIdx.x + (g / nchunks) * (long)gridDim.x;
      const int z = (int)(t / ((long)mt * nt));
      const int r = (int)(t % ((long)mt * nt));
      const int m0 = (r % mt) * kBM, n0 = (r / mt) * kBN;
      const double2* Cz = C + (size_t)z * sC;
#pragma unroll
      for (int L = tid; L < kBN * 8; L += kThreads) {
        const int col = n0 + (L >> 3), row = m0 + (L & 7) * 8;
        if (row < M && col < N) asm volatile("prefetch.global.L2 [%0];" ::"l"(Cz + row + (size_t)col * ldc));
      }
    }
    const int stage = (int)(g % kStages);
    const double2* as = As + stage * kAStage;
    const double2* bs = Bs + stage * kBStage;
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[(kk + fk) * kALd + wm + 8 * i + fr];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[(wn + 8 * j + fr) * kBLd + kk + fk];
      // the 32 independent first products, then the 32 second ones (each accumulator's two
      // products 32 instructions apart)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(accr[i][j], a[i].x, b[j].x);
          dmma(acci[i][j], a[i].x, b[j].y);
        }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double nai = -a[i].y;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(accr[i][j], nai, b[j].y);
          dmma(acci[i][j], a[i].y, b[j].x);
        }
      }
    }
    if ((int)(g % nchunks) == nchunks - 1) {
      // the tile is complete: C -= acc, then start the next tile's accumulators at zero.  The C
      // loads of a row group of 8 go out before the previous group is written, so the loads'
      // latency overlaps instead of stalling on every element.
      const long t = blockIdx.x + (g / nchunks) * (long)gridDim.x;
      const int z = (int)(t / ((long)mt * nt));
      const int r = (int)(t % ((long)mt * nt));
      const int m0 = (r % mt) * kBM, n0 = (r / mt) * kBN;
      double2* Cz = C + (size_t)z * sC;
      double2 cv[2][4][2];
      auto load_group = [&](int i, double2 (&dst)[4][2]) {
        const int row = m0 + wm + 8 * i + fr;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int col = n0 + wn + 8 * j + 2 * fk + e;
            dst[j][e] = (row < M && col < N) ? Cz[(size_t)row + (size_t)col * ldc] : make_double2(0.0, 0.0);
          }
      };
      load_group(0, cv[0]);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (i + 1 < 4) load_group(i + 1, cv[(i + 1) & 1]);
        const int row = m0 + wm + 8 * i + fr;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int col = n0 + wn + 8 * j + 2 * fk + e;
            if (row < M && col < N) {
              double2 v = cv[i & 1][j][e];
              v.x -= accr[i][j][e];
              v.y -= acci[i][j][e];
              Cz[(size_t)row + (size_t)col * ldc] = v;
            }
            accr[i][j][e] = 0.0;
            acci[i][j][e] = 0.0;
          }
        }
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace

int zgemm_f64_update(int M, int N, int K, const double2* A, long lda, const double2* B, long ldb, double2* C,
                     long ldc, cudaStream_t s) {
  return zgemm_f64_update_batched(M, N, K, A, lda, 0, B, ldb, 0, C, ldc, 0, 1, s);
}

int zgemm_f64_update_batched(int M, int N, int K, const double2* A, long lda, long sA, const double2* B, long ldb,
                             long sB, double2* C, long ldc, long sC, int batch, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return 0;
  if (((uintptr_t)A & 15) || ((uintptr_t)B & 15) || ((uintptr_t)C & 15) || lda < M || ldb < K || ldc < M || sA < 0 ||
      sB < 0 || sC < 0) {
    set_last_error_msg("zgemm_f64_update: misaligned operand or leading dimension too small");
    return -1;
  }
  // a shared A with the problems' B and C blocks back to back (column-major) is one GEMM with
  // batch x N columns: whole 64-wide tiles instead of one partial tile column per problem
  if (batch > 1 && sA == 0 && sB == ldb * (long)N && sC == ldc * (long)N && (long)N * batch <= 0x7fffffffL) {
    N *= batch;
    batch = 1;
  }
  // per device and cheap next to a launch: set on every call (any thread, any device)
  HPR_CUDA_TRY(cudaFuncSetAttribute(zgemm_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  int dev = 0, nsm = 0;
  HPR_CUDA_TRY(cudaGetDevice(&dev));
  HPR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long ntiles = (long)((M + kBM - 1) / kBM) * ((N + kBN - 1) / kBN) * batch;
  const long grid = ntiles < 2L * nsm ? ntiles : 2L * nsm;  // two resident CTAs per SM
  zgemm_dmma_kernel<<<(unsigned)grid, kThreads, kSmemBytes, s>>>(M, N, K, A, lda, B, ldb, C, ldc, sA, sB, sC, batch);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace hprmat

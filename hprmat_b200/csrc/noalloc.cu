// Dense FP64 solve A X = B for small systems that allocates no device memory.
//
// Who needs it: code that drives the solver from inside another framework's device memory
// pool, or from a latency-critical loop.  There, a cudaMalloc/cudaFree either fails (the
// pool has already reserved the device memory) or stalls the whole device (cudaFree
// synchronises).  Every other entry point of this library grows device buffers on demand,
// so this one keeps all of its working memory in a fixed array that is part of the loaded
// library.  Its limits are n <= 512 and nrhs <= 64.
//
// The work is the same blocked LU with partial pivoting and blocked substitution as the
// FP64 path of hprmat_b200_solve_linear_device, run by the same kernels with block size 64.
// Only the source of the scratch memory differs.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/hprmat_b200.h"
#include "common.cuh"
#include "lu.cuh"

namespace hprmat {
namespace {

constexpr int kNoAllocMaxN = 512;
constexpr int kNoAllocMaxRhs = 64;
constexpr int kNoAllocNB = 64;
constexpr int kNoAllocSteps = kNoAllocMaxN / kNoAllocNB;
constexpr int kNoAllocMaxG = (kNoAllocMaxN + 31) / 32;
constexpr int kSwapStrideNA = 3 * kMaxNB + 4;

// Byte offsets into the scratch array (each 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffW = 0;
constexpr size_t kOffX = align256(kOffW + (size_t)kNoAllocMaxN * kNoAllocMaxN * sizeof(double2));
constexpr size_t kOffInv = align256(kOffX + (size_t)kNoAllocMaxN * kNoAllocMaxRhs * sizeof(double2));
constexpr size_t kOffSwaps =
    align256(kOffInv + (size_t)2 * kNoAllocSteps * kNoAllocNB * kNoAllocNB * sizeof(double2));
constexpr size_t kOffIpiv = align256(kOffSwaps + (size_t)kNoAllocSteps * kSwapStrideNA * sizeof(int));
constexpr size_t kOffCandRows = align256(kOffIpiv + (size_t)kNoAllocMaxN * sizeof(int));
constexpr size_t kOffKeys = align256(kOffCandRows + (size_t)2 * kNoAllocMaxG * kNoAllocNB * sizeof(double2));
constexpr size_t kOffRowj = align256(kOffKeys + (size_t)kNoAllocNB * sizeof(unsigned long long));
constexpr size_t kOffStatus = align256(kOffRowj + (size_t)2 * kNoAllocNB * sizeof(double2));
constexpr size_t kScratchBytes = align256(kOffStatus + 64 * sizeof(int));  // about 5.8 MB

// The scratch array.  Every device that loads the library holds it until the process
// exits.  In host code its name is only a host-side stand-in: the device address comes
// from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The array's device address on the current device, looked up on every call: a cached
// address would go stale if the application reset the device (cudaDeviceReset) or its
// primary context was created again.  The lookup is cheap next to the solve.
int scratch_for_current_device(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    set_last_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    return HPRMAT_B200_ERR_CUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return HPRMAT_B200_OK;
}

}  // namespace
}  // namespace hprmat

using namespace hprmat;

extern "C" int hprmat_b200_solve_linear_noalloc(const void* d_A, void* d_B, int n, int nrhs, void* stream,
                                                int* info) {
  if (info) *info = 0;
  if (!d_A || !d_B || n <= 0 || nrhs <= 0) {
    set_last_error_msg("solve_linear_noalloc: invalid arguments");
    return HPRMAT_B200_ERR_ARG;
  }
  if (n > kNoAllocMaxN || nrhs > kNoAllocMaxRhs) {
    set_last_error_msg("solve_linear_noalloc: n must be <= 512 and nrhs <= 64 (fixed scratch array)");
    return HPRMAT_B200_ERR_UNSUPPORTED;
  }
  unsigned char* base = nullptr;
  int s = scratch_for_current_device(&base);
  if (s != HPRMAT_B200_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0, nsm = 0;
  HPR_CUDA_TRY(cudaGetDevice(&dev));
  HPR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));

  constexpr int NB = kNoAllocNB, NT = 256;
  using T = double2;
  const int N = n;
  const long ld = N;
  T* W = reinterpret_cast<T*>(base + kOffW);
  T* X = reinterpret_cast<T*>(base + kOffX);
  T* inv = reinterpret_cast<T*>(base + kOffInv);
  int* swaps = reinterpret_cast<int*>(base + kOffSwaps);
  int* ipiv = reinterpret_cast<int*>(base + kOffIpiv);
  int* status = reinterpret_cast<int*>(base + kOffStatus);
  const int nsteps = (N + NB - 1) / NB;

  // The array keeps the previous call's contents: the status words and the barrier
  // counter must start at zero; A and B are copied in whole.
  HPR_CUDA_TRY(cudaMemsetAsync(status, 0, 64 * sizeof(int), st));
  HPR_CUDA_TRY(cudaMemcpyAsync(W, d_A, (size_t)N * N * sizeof(T), cudaMemcpyDeviceToDevice, st));
  HPR_CUDA_TRY(cudaMemcpyAsync(X, d_B, (size_t)N * nrhs * sizeof(T), cudaMemcpyDeviceToDevice, st));

  const int G0 = std::min(nsm, std::max(1, (N + 31) / 32));
  auto pk = panel_kernel<T, NB, NT>;
  for (int sidx = 0; sidx < nsteps; ++sidx) {
    const int k0 = sidx * NB;
    const int ncols = std::min(NB, N - k0);
    const int m = N - k0;
    const int G = std::min(G0, std::max(1, (m + 31) / 32));
    const int rpc = (m + G - 1) / G;
    const size_t smem = ((size_t)NB * (rpc | 1) + NB) * sizeof(T);
    if (smem > 48 * 1024) HPR_CUDA_TRY(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HPR_CUDA_TRY(cudaMemsetAsync(status + SW_BARRIER, 0, sizeof(int), st));
    HPR_CUDA_TRY(cudaMemsetAsync(base + kOffKeys, 0, (size_t)NB * sizeof(unsigned long long), st));
    PanelArgs<T> pa;
    pa.W = W;
    pa.ld = ld;
    pa.N = N;
    pa.k0 = k0;
    pa.ncols = ncols;
    pa.rpc = rpc;
    pa.G = G;
    pa.ipiv = ipiv;
    pa.cand_rows = reinterpret_cast<T*>(base + kOffCandRows);
    pa.keys = reinterpret_cast<unsigned long long*>(base + kOffKeys);
    pa.rowj = reinterpret_cast<T*>(base + kOffRowj);
    pa.status = status;
    int* swb = swaps + (size_t)sidx * kSwapStrideNA;
    pa.sw.top_src = swb;
    pa.sw.extra_dst = swb + kMaxNB;
    pa.sw.extra_src = swb + 2 * kMaxNB;
    pa.sw.n_extra = swb + 3 * kMaxNB;
    pa.growth_bits = nullptr;
    pa.lup = nullptr;
    pa.lup_ld = 0;
    pa.lup_plane = 0;
    void* args[] = {&pa};
    HPR_CUDA_TRY(cudaLaunchCooperativeKernel((void*)pk, dim3(G), dim3(NT), args, smem, st));
    if (k0 + ncols >= N) break;
    constexpr int CW = 32;
    auto tk = trsm_lower_kernel<T, NB, CW, NT>;
    const size_t tsm = (size_t)CW * (NB + 1) * sizeof(T) + (size_t)CW * NB * sizeof(T);
    if (tsm > 48 * 1024) HPR_CUDA_TRY(cudaFuncSetAttribute(tk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
    TrsmArgs<T> ta{};
    ta.W = W;
    ta.ld = ld;
    ta.k0 = k0;
    ta.ncols = ncols;
    ta.top_src = pa.sw.top_src;
    ta.extra_dst = pa.sw.extra_dst;
    ta.extra_src = pa.sw.extra_src;
    ta.n_extra = pa.sw.n_extra;
    ta.X = W;
    ta.ldx = ld;
    ta.c_begin = k0 + ncols;
    ta.c_end = N;
    tk<<<(N - k0 - ncols + CW - 1) / CW, NT, tsm, st>>>(ta);
    HPR_CUDA_TRY(cudaGetLastError());
    const int M2 = N - k0 - ncols;
    dim3 grid((M2 + 63) / 64, (M2 + 63) / 64);
    cgemm_update_kernel<T><<<grid, 256, 0, st>>>(M2, M2, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld,
                                                 W + k0 + (size_t)(k0 + ncols) * ld, ld,
                                                 W + (k0 + ncols) + (size_t)(k0 + ncols) * ld, ld);
    HPR_CUDA_TRY(cudaGetLastError());
  }
  auto ik = tri_inverse_kernel<T, NB, NT>;
  const size_t ism = ((size_t)NB * NB + NB) * sizeof(T);
  if (ism > 48 * 1024) HPR_CUDA_TRY(cudaFuncSetAttribute(ik, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ism));
  ik<<<dim3(nsteps, 2), NT, ism, st>>>(W, ld, N, NB, inv);
  HPR_CUDA_TRY(cudaGetLastError());
  // forward and backward substitution
  constexpr int DCW = 2;
  auto dk = diag_apply_kernel<T, NB, DCW>;
  const size_t dsm = ((size_t)NB * NB + 2 * DCW * NB) * sizeof(T);
  if (dsm > 48 * 1024) HPR_CUDA_TRY(cudaFuncSetAttribute(dk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
  for (int sidx = 0; sidx < nsteps; ++sidx) {
    const int k0 = sidx * NB, ncols = std::min(NB, N - k0);
    const int* sw = swaps + (size_t)sidx * kSwapStrideNA;
    dk<<<(nrhs + DCW - 1) / DCW, NB * DCW, dsm, st>>>(inv + (size_t)2 * sidx * NB * NB, ncols, k0, sw, sw + kMaxNB, sw + 2 * kMaxNB,
                            sw + 3 * kMaxNB, X, ld, nrhs, nullptr, 0);
    HPR_CUDA_TRY(cudaGetLastError());
    const int M2 = N - k0 - ncols;
    if (M2 > 0) {
      dim3 grid((M2 + 63) / 64, (nrhs + 63) / 64);
      cgemm_update_kernel<T><<<grid, 256, 0, st>>>(M2, nrhs, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld, X + k0,
                                                   ld, X + k0 + ncols, ld);
      HPR_CUDA_TRY(cudaGetLastError());
    }
  }
  for (int sidx = nsteps - 1; sidx >= 0; --sidx) {
    const int k0 = sidx * NB, ncols = std::min(NB, N - k0);
    dk<<<(nrhs + DCW - 1) / DCW, NB * DCW, dsm, st>>>(inv + ((size_t)2 * sidx + 1) * NB * NB, ncols, k0, nullptr, nullptr, nullptr, nullptr, X,
                            ld, nrhs, nullptr, 0);
    HPR_CUDA_TRY(cudaGetLastError());
    if (k0 > 0) {
      dim3 grid((k0 + 63) / 64, (nrhs + 63) / 64);
      cgemm_update_kernel<T><<<grid, 256, 0, st>>>(k0, nrhs, ncols, W + (size_t)k0 * ld, ld, X + k0, ld, X, ld);
      HPR_CUDA_TRY(cudaGetLastError());
    }
  }
  HPR_CUDA_TRY(cudaMemcpyAsync(d_B, X, (size_t)N * nrhs * sizeof(T), cudaMemcpyDeviceToDevice, st));
  int hs[SW_COUNT];
  HPR_CUDA_TRY(cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st));
  HPR_CUDA_TRY(cudaStreamSynchronize(st));
  if (hs[SW_TIMEOUT] != 0) {
    set_last_error_msg("solve_linear_noalloc: grid barrier wait limit exceeded");
    return HPRMAT_B200_ERR_TIMEOUT;
  }
  if (hs[SW_INFO] != 0) {
    if (info) *info = hs[SW_INFO];
    set_last_error_msg("solve_linear_noalloc: matrix is singular");
    return HPRMAT_B200_SINGULAR;
  }
  return HPRMAT_B200_OK;
}

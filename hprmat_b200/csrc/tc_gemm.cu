// Complex GEMM update of the mixed-precision LU (trailing update) and of its blocked
// triangular solves, on sm_100a tensor cores.
//
//   C[M x Nc] -= A[M x K] * B[K x Nc]       (complex, C interleaved float2, column-major)
//
// Each complex product is formed as 4 real products (4M), and each real product X*Y as
// the 3-term TF32 split hi(X)hi(Y) + hi(X)lo(Y) + lo(X)hi(Y) (3xTF32), so the bulk of the
// LU runs on tcgen05 kind::tf32 with FP32 accumulation at close to FP32 accuracy:
//   Re += Ar*Br - Ai*Bi,   Im += Ar*Bi + Ai*Br      -> 12 MMAs per K-step of 8.
// The minus sign comes from the A-negate bit of the instruction descriptor.
//
// Tile 128 (rows) x BN columns (BN = 128 for the LU and the solves; 256 kept for
// comparison).  Re and Im accumulate in 2 BN TMEM columns; with BN = 128 two such sets are
// used alternately so the epilogue of one tile overlaps the MMAs of the next.  One
// persistent CTA per SM, 10 warps:
//   warp 0     TMA producer: per K-chunk of 16 one 3-D box for the 4 A planes
//              (16 x 128 x 4 floats) and one for the 4 B planes (16 x BN x 4), 64-byte
//              swizzle, into a 3-stage ring (2 for BN = 256);
//   warp 1     TMEM allocator and single-thread MMA issuer;
//   warps 2-9  epilogue: tcgen05.ld of Re/Im, C -= acc, coalesced along rows (two warps per
//              TMEM lane quarter, each half of the tile's columns).
// Every mbarrier wait is bounded; on expiry the kernel records the site in *err, stops
// issuing work, waits (bounded) for its own TMA copies and frees its TMEM.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

namespace hprmat {

namespace {

using namespace tc;
constexpr int kBM = 128;
constexpr int kKC = 16;                                 // K values per stage (64 bytes)
constexpr int kABytes = 4 * kBM * kKC * 4;             // 32 KB
template <int BN> struct TileCfg {
  static constexpr int kBBytes = 4 * BN * kKC * 4;     // 64 KB (BN=256) / 32 KB (BN=128)
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kStages = (200 * 1024) / kStageBytes;   // 2 (BN=256) / 3 (BN=128)
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*barriers*/ + 1024 /*align*/;
  // accumulator sets (Re + Im, 2 BN columns each) in the 512 TMEM columns: with two, the
  // epilogue of one tile overlaps the MMAs of the next
  static constexpr int kBufs = (4 * BN <= 512) ? 2 : 1;
  static constexpr int kTmemCols = 512;
};
constexpr int kEpiWarps = 8;                         // 2 per TMEM lane quarter
constexpr int kThreads = 32 * (2 + kEpiWarps);
struct TcArgs {
  int a_k0, a_row0, b_k0, b_row0, kchunks;
  float2* C;
  long ldc;
  int M, Nc;
  int* err;
};

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    tc_update_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TcArgs p) {
  using Cfg = TileCfg<BN>;
  constexpr int kBN = BN;
  constexpr int kStages = Cfg::kStages;
  constexpr int kStageBytes = Cfg::kStageBytes;
  float2* C = p.C;
  const long ldc = p.ldc;
  const int M = p.M, Nc = p.Nc;
  int* err = p.err;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  constexpr int kBufs = Cfg::kBufs;
  uint64_t* acc_full = empty + kStages;       // [kBufs]
  uint64_t* acc_empty = acc_full + kBufs;     // [kBufs]
  uint64_t* drain = acc_empty + kBufs;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int mt = (M + kBM - 1) / kBM;
  const int nt = (Nc + kBN - 1) / kBN;
  const int ntiles = mt * nt;
  const int kChunks = p.kchunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 32 * kEpiWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(Cfg::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int inflight = 0;  // stages issued whose completion this thread has not observed
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const int m0 = (t % mt) * kBM;
        const int n0 = (t / mt) * kBN;
        for (int kc = 0; kc < kChunks; ++kc) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag, err, 11)) { ok = false; break; }
          unsigned char* sa = smem + stage * kStageBytes;
          mbar_expect_tx(&full[stage], kStageBytes);
          tma_load_3d(sa, &tmA, &full[stage], p.a_k0 + kc * kKC, p.a_row0 + m0, 0);
          tma_load_3d(sa + kABytes, &tmB, &full[stage], p.b_k0 + kc * kKC, p.b_row0 + n0, 0);
          inflight = min(inflight + 1, kStages);
          if (++stage == kStages) { stage = 0; phase ^= 1u; }
        }
      }
      if (!ok) {
        // let our own copies land before the CTA can exit: wait (bounded) on the fill
        // barriers of the stages issued last
        int s = stage, ph = phase;
        for (int i = 0; i < inflight; ++i) {
          if (--s < 0) { s = kStages - 1; ph ^= 1; }
          for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(&full[s], ph); ++it) {}
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      const uint32_t id_pos = idesc_tf32<BN>(false), id_neg = idesc_tf32<BN>(true);
      int local = 0;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++local) {
        const int buf = local % kBufs;
        const uint32_t use = (uint32_t)(local / kBufs);
        const uint32_t t_re = tmem + (uint32_t)(buf * 2 * kBN), t_im = t_re + kBN;
        if (!mbar_wait(&acc_empty[buf], (use & 1u) ^ 1u, abort_flag, err, 21)) break;
        tc_fence_after();
        for (int kc = 0; kc < kChunks; ++kc) {
          if (!mbar_wait(&full[stage], phase, abort_flag, err, 22)) { ok = false; break; }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * kStageBytes);
          const uint32_t sb = sa + kABytes;
#pragma unroll
          for (int kk = 0; kk < kKC / 8; ++kk) {
            const uint32_t off = kk * 32;
            const uint64_t a_rh = sdesc_k_sw64(sa + 0 * (kBM * 64) + off);
            const uint64_t a_rl = sdesc_k_sw64(sa + 1 * (kBM * 64) + off);
            const uint64_t a_ih = sdesc_k_sw64(sa + 2 * (kBM * 64) + off);
            const uint64_t a_il = sdesc_k_sw64(sa + 3 * (kBM * 64) + off);
            const uint64_t b_rh = sdesc_k_sw64(sb + 0 * (kBN * 64) + off);
            const uint64_t b_rl = sdesc_k_sw64(sb + 1 * (kBN * 64) + off);
            const uint64_t b_ih = sdesc_k_sw64(sb + 2 * (kBN * 64) + off);
            const uint64_t b_il = sdesc_k_sw64(sb + 3 * (kBN * 64) + off);
            const uint32_t first = (kc == 0 && kk == 0) ? 0u : 1u;
            // small terms first, then the hi*hi product
            mma_tf32(t_re, a_rh, b_rl, id_pos, first);
            mma_tf32(t_re, a_rl, b_rh, id_pos, 1u);
            mma_tf32(t_re, a_ih, b_il, id_neg, 1u);
            mma_tf32(t_re, a_il, b_ih, id_neg, 1u);
            mma_tf32(t_re, a_rh, b_rh, id_pos, 1u);
            mma_tf32(t_re, a_ih, b_ih, id_neg, 1u);
            mma_tf32(t_im, a_rh, b_il, id_pos, first);
            mma_tf32(t_im, a_rl, b_ih, id_pos, 1u);
            mma_tf32(t_im, a_ih, b_rl, id_pos, 1u);
            mma_tf32(t_im, a_il, b_rh, id_pos, 1u);
            mma_tf32(t_im, a_rh, b_ih, id_pos, 1u);
            mma_tf32(t_im, a_ih, b_rh, id_pos, 1u);
          }
          mma_commit(&empty[stage]);
          if (++stage == kStages) { stage = 0; phase ^= 1u; }
        }
        if (!ok) break;
        mma_commit(&acc_full[buf]);
      }
      if (!ok || *abort_flag) {
        // make sure no MMA of ours is still reading shared memory or writing TMEM
        mma_commit(drain);
        for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(drain, 0); ++it) {}
      }
    }
  } else {
    // epilogue warps 2..9: TMEM lane quarter q = warp % 4, column half (warp - 2) / 4
    const int q = warp & 3;
    const int c_begin = ((warp - 2) >> 2) * (kBN / 2);
    int local = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++local) {
      const int m0 = (t % mt) * kBM;
      const int n0 = (t / mt) * kBN;
      const int buf = local % kBufs;
      const uint32_t use = (uint32_t)(local / kBufs);
      const int row = m0 + q * 32 + lane;
      const bool rv = row < M;
      const int ncw = min(kBN / 2, Nc - (n0 + c_begin));  // columns of this warp (warp-uniform)
      // C does not depend on the accumulator: the first chunk's loads go out before the
      // wait, and each later chunk's loads before the previous chunk is consumed (two
      // chunks of 16 columns in flight per lane).
      float2 cv[2][16];
      auto load_chunk = [&](float2* dst, int c0) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j;
          dst[j] = (rv && col < Nc) ? C[row + (size_t)col * ldc] : make_float2(0.f, 0.f);
        }
      };
      if (ncw > 0) load_chunk(cv[0], c_begin);
      bool ok = true;
      if (lane == 0) ok = mbar_wait(&acc_full[buf], use & 1u, abort_flag, err, 31);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      __syncwarp();
      tc_fence_after();
      const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 2 * kBN);
#pragma unroll
      for (int i = 0; i < kBN / 32; ++i) {
        const int c0 = c_begin + 16 * i;
        if (16 * i >= ncw) break;  // warp-uniform
        if (i + 1 < kBN / 32 && 16 * (i + 1) < ncw) load_chunk(cv[(i + 1) & 1], c0 + 16);
        float re[16], im[16];
        tmem_ld16(tl + c0, re);
        tmem_ld16(tl + kBN + c0, im);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j;
          if (rv && col < Nc) C[row + (size_t)col * ldc] = make_float2(cv[i & 1][j].x - re[j], cv[i & 1][j].y - im[j]);
        }
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kTmemCols)
                 : "memory");
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

int tc_gemm_init(TcGemmPlan& p, int device) {
  p.device = device;
  int nsm = 0;
  HPR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  p.nsm = nsm;
  cudaDriverEntryPointQueryResult q;
  void* fn = nullptr;
  HPR_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (q != cudaDriverEntryPointSuccess || fn == nullptr) {
    set_last_error_msg("cuTensorMapEncodeTiled is not available from the driver");
    return -2;
  }
  p.encode = fn;
  if (!p.d_err) {
    HPR_CUDA_TRY(cudaMalloc(&p.d_err, sizeof(int)));
    HPR_CUDA_TRY(cudaMemset(p.d_err, 0, sizeof(int)));
  }
  HPR_CUDA_TRY(cudaFuncSetAttribute(tc_update_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    TileCfg<256>::kSmemBytes));
  HPR_CUDA_TRY(cudaFuncSetAttribute(tc_update_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    TileCfg<128>::kSmemBytes));
  return 0;
}

int tc_make_operand(TcGemmPlan& p, TcOperand& op, const float* base, long kext, long rows, long ld, long plane,
                    int box_rows) {
  if (((uintptr_t)base & 15) || (ld % 4) || (plane % 4) || kext < 16 || rows < 1 || ld < kext ||
      (box_rows != 64 && box_rows != 128 && box_rows != 256)) {
    set_last_error_msg("tensor-core operand: misaligned or invalid view");
    return -1;
  }
  EncodeTiledFn enc = reinterpret_cast<EncodeTiledFn>(p.encode);
  cuuint64_t dims[3] = {(cuuint64_t)kext, (cuuint64_t)rows, 4};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)plane * 4};
  cuuint32_t box[3] = {(cuuint32_t)kKC, (cuuint32_t)box_rows, 4};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(&op.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error_msg("cuTensorMapEncodeTiled failed for a tensor-core operand");
    return -2;
  }
  op.kext = kext;
  op.rows = rows;
  return 0;
}

int tc_update(TcGemmPlan& p, const TcOperand& A, int a_k0, int a_row0, const TcOperand& B, int b_k0, int b_row0,
              int K, float2* C, long ldc, int M, int Nc, int bn, cudaStream_t s) {
  if (M <= 0 || Nc <= 0 || K <= 0) return 0;
  // The K coordinate of every box is a multiple of 16 floats (64 bytes): TMA's 16-byte rule.
  if ((K % kKC) || (a_k0 % 4) || (b_k0 % 4) || a_k0 < 0 || b_k0 < 0 || a_row0 < 0 || b_row0 < 0) {
    set_last_error_msg("tensor-core update: K offsets must be multiples of 4 floats and K of 16");
    return -1;
  }
  TcArgs args{a_k0, a_row0, b_k0, b_row0, K / kKC, C, ldc, M, Nc, p.d_err};
  const int cap = (p.max_grid > 0 && p.max_grid < p.nsm) ? p.max_grid : p.nsm;
  if (bn == 256) {
    const int ntiles = ((M + kBM - 1) / kBM) * ((Nc + 255) / 256);
    const int grid = ntiles < cap ? ntiles : cap;
    tc_update_kernel<256><<<grid, kThreads, TileCfg<256>::kSmemBytes, s>>>(A.map, B.map, args);
  } else if (bn == 128) {
    const int ntiles = ((M + kBM - 1) / kBM) * ((Nc + 127) / 128);
    const int grid = ntiles < cap ? ntiles : cap;
    tc_update_kernel<128><<<grid, kThreads, TileCfg<128>::kSmemBytes, s>>>(A.map, B.map, args);
  } else {
    set_last_error_msg("tensor-core update: bn must be 128 or 256");
    return -5;
  }
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int tc_gemm_check(TcGemmPlan& p, cudaStream_t s, int* err_out) {
  int h = 0;
  HPR_CUDA_TRY(cudaMemcpyAsync(&h, p.d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  HPR_CUDA_TRY(cudaStreamSynchronize(s));
  if (h) HPR_CUDA_TRY(cudaMemsetAsync(p.d_err, 0, sizeof(int), s));
  *err_out = h;
  return 0;
}

}  // namespace hprmat

// Wavefront triangular solves of the mixed-precision LU and the preparation of the factors
// they read (interface and algorithm: tc_solve.cuh).
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "tc_common.cuh"
#include "tc_solve.cuh"

namespace hprmat {

namespace {

using namespace tc;

constexpr int kNB = 128;       // block size of the factorisation and of the tiles
constexpr int kKC = 16;        // K values per TMA box (64 bytes)
constexpr int kChunks = kNB / kKC;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr int kMaxNBSw = 128;  // kMaxNB of the interchange lists

// ------------------------------------------------------------------ interchange chain
// One CTA.  cur[i] = row that holds final row i after the step being undone; inv = cur^-1.
// Walking the steps backwards, step s moves the content of position T_s(q) to q for the
// positions q it touches, so sigma_{s-1} = T_s o sigma_s changes only there.
__global__ void __launch_bounds__(1024) perm_chain_kernel(const int* __restrict__ swaps, int swap_stride, int N,
                                                           int nsteps, int* cur, int* inv, int* sig, long sig_ld,
                                                           int* perm0) {
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += 1024) {
    cur[i] = i;
    inv[i] = i;
  }
  __syncthreads();
  for (int s = nsteps - 1; s >= 0; --s) {
    // sigma_s, needed for the L block column s (final rows below its diagonal block)
    const int lo = (s + 1) * kNB;
    int* dst = sig + (size_t)s * sig_ld;
    for (int i = lo + tid; i < N; i += 1024) dst[i] = cur[i];
    __syncthreads();
    const int k0 = s * kNB;
    const int ncols = min(kNB, N - k0);
    const int* sw = swaps + (size_t)s * swap_stride;
    const int ne = sw[3 * kMaxNBSw];
    const int cnt = ncols + ne;
    int fi = 0, src = 0;
    if (tid < cnt) {
      const int q = tid < ncols ? k0 + tid : sw[kMaxNBSw + (tid - ncols)];
      src = tid < ncols ? sw[tid] : sw[2 * kMaxNBSw + (tid - ncols)];
      fi = inv[q];
    }
    __syncthreads();
    if (tid < cnt) {
      cur[fi] = src;
      inv[src] = fi;
    }
    __syncthreads();
  }
  for (int i = tid; i < N; i += 1024) perm0[i] = cur[i];
}

// ------------------------------------------------------------------ transposed copy
// CTA (row chunk of 32, block column k): 32 rows x 128 columns of each plane through
// shared memory into T (column-major, rows contiguous).
__global__ void __launch_bounds__(256) transpose_offdiag_kernel(const float* __restrict__ lup, long lup_ld,
                                                                 long lup_plane, const int* __restrict__ sig,
                                                                 long sig_ld, int N, float* T, long ldt,
                                                                 long tplane) {
  __shared__ float tile[32][kNB + 1];
  __shared__ int srow[32];
  const int k = blockIdx.y;
  const int i0 = blockIdx.x * 32;
  const int j = i0 / kNB;
  if (j == k) return;
  const int tid = threadIdx.x;
  const int c0 = k * kNB;
  const int nc = min(kNB, N - c0);
  if (tid < 32) {
    const int i = i0 + tid;
    srow[tid] = (i < N) ? (j > k ? sig[(size_t)k * sig_ld + i] : i) : -1;
  }
  __syncthreads();
  for (int p = 0; p < 4; ++p) {
    const float* src = lup + (size_t)p * lup_plane;
    for (int idx = tid; idx < 32 * kNB; idx += 256) {
      const int r = idx / kNB, c = idx % kNB;
      const int sr = srow[r];
      tile[r][c] = (sr >= 0 && c < nc) ? src[(size_t)sr * lup_ld + c0 + c] : 0.f;
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    float* dstp = T + (size_t)p * tplane;
    if (i0 + lane < N)
      for (int c = warp; c < nc; c += 8) dstp[(size_t)(c0 + c) * ldt + i0 + lane] = tile[lane][c];
    __syncthreads();
  }
}

// ------------------------------------------------------------------ diagonal inverse planes
// Block b (= 2 J + u) of h x h column-major float2 inverses -> row-major planes of row length h.
__global__ void __launch_bounds__(256) dinv_planes_kernel(const float2* __restrict__ inv, int h, float* di,
                                                          long di_plane) {
  const int b = blockIdx.x;
  const float2* src = inv + (size_t)b * h * h;
  for (int idx = blockIdx.y * 256 + threadIdx.x; idx < h * h; idx += 256 * gridDim.y) {
    const int i = idx / h, r = idx % h;
    const float2 v = src[i + (size_t)r * h];
    float hr, lr, hi, li;
    tf32_split(v.x, hr, lr);
    tf32_split(v.y, hi, li);
    const size_t off = ((size_t)b * h + i) * h + r;
    di[off] = hr;
    di[di_plane + off] = lr;
    di[2 * di_plane + off] = hi;
    di[3 * di_plane + off] = li;
  }
}

// ------------------------------------------------------------------ super-block inverses
// One doubling step of the diagonal-block inverses, h -> 2h:
//   L: [A 0; B C]^-1 = [A^-1 0; -C^-1 (B A^-1)  C^-1],   U: [A B; 0 C]^-1 = [A^-1 -A^-1 (B C^-1); 0 C^-1]
// with A^-1, C^-1 the level-h inverses (dfh[(2 blk + u)], h x h column-major) of blocks
// 2J and 2J + 1, and B the off-diagonal block read from T (final-order factors, TF32 planes:
// the FP32 value is head + tail).  Pass 1 forms P = B A^-1 (L) / B C^-1 (U), pass 2
// Off = -C^-1 P (L) / -A^-1 P (U); FP32 SIMT tiles of 64 x 64, batch z = 2 J + u.
struct DinvDouble {
  const float2* dfh;  // level-h inverses
  const float* T;     // transposed off-diagonal planes
  long ldt, tplane;
  int N, h, nblk;     // nblk: blocks at level h
  const float2* P;    // pass-1 result (pass 2 input)
};

template <int PASS>
__global__ void __launch_bounds__(256) dinv_double_kernel(DinvDouble d, float2* out) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ float2 As[BK][BM];
  __shared__ float2 Bs[BK][BN + 1];
  const int z = blockIdx.z;
  const int J = z >> 1, u = z & 1;
  const int first = 2 * J, second = 2 * J + 1;
  if (second >= d.nblk) return;  // no second block: nothing to join
  const int h = d.h;
  const size_t hh = (size_t)h * h;
  const float2* Ainv = d.dfh + (size_t)(2 * first + u) * hh;
  const float2* Cinv = d.dfh + (size_t)(2 * second + u) * hh;
  const float2* P = d.P + (size_t)z * hh;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  auto tval = [&](int row, int col) -> float2 {  // factor entry (row, col) from T, 0 outside
    if (row >= d.N || col >= d.N) return make_float2(0.f, 0.f);
    const size_t o = (size_t)col * d.ldt + row;
    return make_float2(d.T[o] + d.T[d.tplane + o], d.T[2 * d.tplane + o] + d.T[3 * d.tplane + o]);
  };
  // A operand (m, k) and B operand (k, n) of this pass
  auto aop = [&](int m, int k) -> float2 {
    if (PASS == 1) return u == 0 ? tval(second * h + m, first * h + k) : tval(first * h + m, second * h + k);
    return u == 0 ? Cinv[m + (size_t)k * h] : Ainv[m + (size_t)k * h];
  };
  auto bop = [&](int k, int n) -> float2 {
    if (PASS == 1) return u == 0 ? Ainv[k + (size_t)n * h] : Cinv[k + (size_t)n * h];
    return P[k + (size_t)n * h];
  };
  float2 acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[r][q] = make_float2(0.f, 0.f);
  for (int k0 = 0; k0 < h; k0 += BK) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      const int mm = idx % BM, kk = idx / BM;
      As[kk][mm] = aop(m0 + mm, k0 + kk);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      const int kk = idx % BK, nn = idx / BK;
      Bs[kk][nn] = bop(k0 + kk, n0 + nn);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float2 av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = As[kk][tx + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = Bs[kk][ty + 16 * q];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) cfma(acc[r][q], av[r], bv[q]);
    }
    __syncthreads();
  }
  float2* o = out + (size_t)z * hh;
  const float sg = PASS == 2 ? -1.f : 1.f;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int m = m0 + tx + 16 * r, n = n0 + ty + 16 * q;
      o[m + (size_t)n * h] = make_float2(sg * acc[r][q].x, sg * acc[r][q].y);
    }
}

// The 2h x 2h inverse of super block J (u = 0: L, 1: U) from A^-1, C^-1 and Off (identity
// for a missing second block).
__global__ void __launch_bounds__(256) dinv_assemble_kernel(const float2* __restrict__ dfh,
                                                            const float2* __restrict__ off, int h, int nblk,
                                                            float2* df2h) {
  const int z = blockIdx.x;
  const int J = z >> 1, u = z & 1;
  const int first = 2 * J, second = 2 * J + 1;
  const bool has2 = second < nblk;
  const size_t hh = (size_t)h * h;
  const int h2 = 2 * h;
  float2* o = df2h + (size_t)z * h2 * h2;
  for (int idx = blockIdx.y * 256 + threadIdx.x; idx < h2 * h2; idx += 256 * gridDim.y) {
    const int r = idx % h2, c = idx / h2;
    float2 v = make_float2(0.f, 0.f);
    if (r < h && c < h) {
      v = dfh[(size_t)(2 * first + u) * hh + r + (size_t)c * h];
    } else if (r >= h && c >= h) {
      if (has2) v = dfh[(size_t)(2 * second + u) * hh + (r - h) + (size_t)(c - h) * h];
      else if (r == c) v.x = 1.f;
    } else if (has2 && u == 0 && r >= h && c < h) {
      v = off[(size_t)z * hh + (r - h) + (size_t)c * h];
    } else if (has2 && u == 1 && r < h && c >= h) {
      v = off[(size_t)z * hh + r + (size_t)(c - h) * h];
    }
    o[idx] = v;
  }
}

// ------------------------------------------------------------------ right-hand side planes
__global__ void __launch_bounds__(256) rhs_planes_kernel(const float2* __restrict__ X, long ldx,
                                                          const int* __restrict__ perm0, int N, float* bp, long bld,
                                                          long bplane) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= N) return;
  const float2 v = X[(size_t)perm0[i] + (size_t)c * ldx];
  float hr, lr, hi, li;
  tf32_split(v.x, hr, lr);
  tf32_split(v.y, hi, li);
  const size_t off = (size_t)c * bld + i;
  bp[off] = hr;
  bp[bplane + off] = lr;
  bp[2 * bplane + off] = hi;
  bp[3 * bplane + off] = li;
}

// ------------------------------------------------------------------ shared pieces of the
// two tensor-core kernels below: a 3xTF32 complex MMA chain over K = 128 from a ring of
// shared-memory stages, each stage one 16-deep K chunk of the A tile (4 planes x 128 rows)
// and of the B tile (4 planes x BN rows).
template <int BN>
struct Ring {
  static constexpr int kABytes = 4 * kNB * kKC * 4;
  static constexpr int kBBytes = 4 * BN * kKC * 4;
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kStages = (192 * 1024) / kStageBytes;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 1024;
};

template <int BN>
__device__ __forceinline__ void mma_chunk(unsigned char* smem, int stage, uint32_t t_re, uint32_t t_im,
                                          bool first_chunk, bool negate) {
  using R = Ring<BN>;
  const uint32_t sa = smem_u32(smem + stage * R::kStageBytes);
  const uint32_t sb = sa + R::kABytes;
#pragma unroll
  for (int kk = 0; kk < kKC / 8; ++kk) {
    const uint32_t off = kk * 32;
    uint64_t a[4], b[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a[q] = sdesc_k_sw64(sa + q * (kNB * 64) + off);
      b[q] = sdesc_k_sw64(sb + q * (BN * 64) + off);
    }
    cmma_3xtf32<BN>(t_re, t_im, a, b, (first_chunk && kk == 0) ? 0u : 1u, negate);
  }
}

__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

__device__ __forceinline__ long long globaltimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// ------------------------------------------------------------------ off-diagonal scaling
struct ScaleArgs {
  int N, nsteps, sb;  // sb: blocks per super block of the diagonal inverses
  float* lup;
  long lup_ld, lup_plane;
  int* err;
};

// Tile t -> block (j, k) with k outside j's super block J = j / sb: out = rows (j mod sb)*128..
// of D_JJ^-1 (DI super-block row 2J or 2J+1, K = sb*128) x the T rows of super block J at
// columns k*128.., written as the TF32 planes of the LU planes at rows j*128.., columns
// k*128..  Persistent, one CTA per SM, two TMEM accumulator sets so the epilogue of a tile
// overlaps the next tile's MMAs.
__global__ void __launch_bounds__(kThreads, 1)
    scale_offdiag_kernel(const __grid_constant__ CUtensorMap tmD, const __grid_constant__ CUtensorMap tmT,
                         ScaleArgs p) {
  constexpr int BN = kNB;
  using R = Ring<BN>;
  constexpr int kStages = R::kStages;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * R::kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;  // [2]
  uint64_t* acc_empty = acc_full + 2;    // [2]
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsteps = p.nsteps, N = p.N, sb = p.sb;
  const int ntiles = nsteps * nsteps;  // (j, k) pairs in the same super block are skipped
  const int nchunk = kChunks * sb;
  int* err = p.err;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 32 * kEpiWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0, inflight = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const int j = t / nsteps, k = t % nsteps;
        const int J = j / sb;
        if (k / sb == J) continue;
        const int drow = (2 * J + (k > j ? 1 : 0)) * sb * kNB + (j % sb) * kNB;
        for (int kc = 0; kc < nchunk; ++kc) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag, err, 51)) { ok = false; break; }
          unsigned char* sa = smem + stage * R::kStageBytes;
          mbar_expect_tx(&full[stage], R::kStageBytes);
          tma_load_3d(sa, &tmD, &full[stage], kc * kKC, drow, 0);
          tma_load_3d(sa + R::kABytes, &tmT, &full[stage], J * sb * kNB + kc * kKC, k * kNB, 0);
          inflight = min(inflight + 1, kStages);
          if (++stage == kStages) { stage = 0; phase ^= 1u; }
        }
      }
      if (!ok) {
        int s = stage;
        uint32_t ph = phase;
        for (int i = 0; i < inflight; ++i) {
          if (--s < 0) { s = kStages - 1; ph ^= 1u; }
          for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(&full[s], ph); ++it) {}
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0, local = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        if ((t % nsteps) / sb == (t / nsteps) / sb) continue;
        const int buf = local & 1;
        const uint32_t use = (uint32_t)(local >> 1);
        ++local;
        const uint32_t t_re = tmem + (uint32_t)(buf * 2 * BN), t_im = t_re + BN;
        if (!mbar_wait(&acc_empty[buf], (use & 1u) ^ 1u, abort_flag, err, 52)) break;
        tc_fence_after();
        for (int kc = 0; kc < nchunk; ++kc) {
          if (!mbar_wait(&full[stage], phase, abort_flag, err, 53)) { ok = false; break; }
          tc_fence_after();
          mma_chunk<BN>(smem, stage, t_re, t_im, kc == 0, false);
          mma_commit(&empty[stage]);
          if (++stage == kStages) { stage = 0; phase ^= 1u; }
        }
        if (!ok) break;
        mma_commit(&acc_full[buf]);
      }
      if (!ok || *abort_flag) {
        mma_commit(drain);
        for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(drain, 0); ++it) {}
      }
    }
  } else {
    const int q = warp & 3;
    const int c_begin = ((warp - 2) >> 2) * (BN / 2);
    int local = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int j = t / nsteps, k = t % nsteps;
      if (k / sb == j / sb) continue;
      const int buf = local & 1;
      const uint32_t use = (uint32_t)(local >> 1);
      ++local;
      bool ok = true;
      if (lane == 0) ok = mbar_wait(&acc_full[buf], use & 1u, abort_flag, err, 54);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      __syncwarp();
      tc_fence_after();
      const int row = j * kNB + q * 32 + lane;
      const bool rv = row < N;
      const int ncol = N - k * kNB;  // valid columns of the block (>= 1)
      const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 2 * BN);
#pragma unroll
      for (int i = 0; i < BN / 32; ++i) {
        const int c0 = c_begin + 16 * i;
        float re[16], im[16];
        tmem_ld16(tl + c0, re);
        tmem_ld16(tl + BN + c0, im);
        tmem_wait_ld();
        if (rv && c0 < ncol) {
          float hr[16], lr[16], hi[16], li[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            tf32_split(re[e], hr[e], lr[e]);
            tf32_split(im[e], hi[e], li[e]);
          }
          const size_t off = (size_t)row * p.lup_ld + (size_t)k * kNB + c0;
          float* d0 = p.lup + off;
          if (c0 + 16 <= ncol) {
#pragma unroll
            for (int e = 0; e < 16; e += 4) {
              *reinterpret_cast<float4*>(d0 + e) = make_float4(hr[e], hr[e + 1], hr[e + 2], hr[e + 3]);
              *reinterpret_cast<float4*>(d0 + p.lup_plane + e) = make_float4(lr[e], lr[e + 1], lr[e + 2], lr[e + 3]);
              *reinterpret_cast<float4*>(d0 + 2 * p.lup_plane + e) =
                  make_float4(hi[e], hi[e + 1], hi[e + 2], hi[e + 3]);
              *reinterpret_cast<float4*>(d0 + 3 * p.lup_plane + e) =
                  make_float4(li[e], li[e + 1], li[e + 2], li[e + 3]);
            }
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              if (c0 + e < ncol) {
                d0[e] = hr[e];
                d0[p.lup_plane + e] = lr[e];
                d0[2 * p.lup_plane + e] = hi[e];
                d0[3 * p.lup_plane + e] = li[e];
              }
            }
          }
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// ------------------------------------------------------------------ wavefront sweep
struct WaveArgs {
  int N, nsteps, G, nrhs, sb;
  float* xp;
  long xp_ld, xp_plane;
  float2* xout;
  long ldx;
  int* flags;  // zeroed before the launch; kEpiWarps once block (j, h) is published
  int* err;
  long long* trace;
};

// Waits until *flag >= target (acquire), bounded; false if the limit was reached or the
// kernel is being abandoned.
__device__ __forceinline__ bool wait_flag(const int* flag, int target, volatile int* abort_flag, int* err, int site) {
  for (unsigned it = 0;; ++it) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
    if (v >= target) return true;
    if ((it & 255u) == 255u) {
      int e;
      asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(e) : "l"(err) : "memory");
      if (*abort_flag || e != 0) return false;
      if (it >= (1u << 23)) {
        *abort_flag = 1;
        atomicCAS(err, 0, site);
        return false;
      }
    }
  }
}

// Unit u (u = rank * G + h, ranks in dependency order) handled by CTA u mod gridDim.x:
// block row j = rank (forward) or nsteps - 1 - rank (backward), right-hand sides
// h*UN .. h*UN + UN - 1, super block J = j / sb.  Groups: g0 is rows (j mod sb)*128.. of
// -D_JJ^-1 B_J (K = sb*128, no dependency); then one group per block k outside super block J
// (k < J*sb forward, k >= (J+1)*sb backward), each after the unit (k, h) has published.
// The unit's solution block is -acc.
// Schedule: a CTA takes its units in windows of kSlots (one TMEM accumulator each); in a
// window it issues every unit's g0, then the dependent groups block by block in dependency
// order (k ascending forward, descending backward), for each block the window's units in
// order.  A unit thus consumes each published block as soon as its CTA reaches it, instead of
// after its predecessors in the CTA have finished.  A unit completes at its last block; the
// units of a window complete in window order.
template <int UN, bool FWD>
__global__ void __launch_bounds__(kThreads, 1)
    wavefront_kernel(const __grid_constant__ CUtensorMap tmM, const __grid_constant__ CUtensorMap tmD,
                     const __grid_constant__ CUtensorMap tmB0, const __grid_constant__ CUtensorMap tmX, WaveArgs p) {
  using R = Ring<UN>;
  constexpr int kStages = R::kStages;
  constexpr int kSlots = 512 / (2 * UN);  // accumulators (Re + Im, 2 UN columns each)
  constexpr int kTmemCols = 512;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * R::kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;    // [kSlots]
  uint64_t* acc_empty = acc_full + kSlots;  // [kSlots]
  uint64_t* drain = acc_empty + kSlots;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsteps = p.nsteps, G = p.G, N = p.N, sb = p.sb;
  const int nunits = nsteps * G;
  const int nloc = nunits > (int)blockIdx.x ? (nunits - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
  int* err = p.err;
  // local unit l -> unit id, block row, super block, right-hand-side group
  auto unit_id = [&](int l) { return (int)blockIdx.x + l * (int)gridDim.x; };
  auto row_of = [&](int u) { const int r = u / G; return FWD ? r : nsteps - 1 - r; };
  // dependent blocks of a unit in super block J: forward [0, J sb), backward [(J+1) sb, nsteps)
  auto needs = [&](int J, int k) { return FWD ? k < J * sb : k >= (J + 1) * sb; };
  auto last_k = [&](int J) { return FWD ? J * sb - 1 : (J + 1) * sb; };  // valid if any dependent block
  auto has_dep = [&](int J) { return FWD ? J > 0 : (J + 1) * sb < nsteps; };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < kSlots; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 32 * kEpiWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0, inflight = 0;
      uint32_t phase = 0;
      bool ok = true;
      auto next_stage = [&]() {
        inflight = min(inflight + 1, kStages);
        if (++stage == kStages) { stage = 0; phase ^= 1u; }
      };
      // one dependent group: block k of unit u (block row j, group h)
      auto issue_dep = [&](int u, int j, int h, int k, bool last) {
        for (int kc = 0; kc < kChunks && ok; ++kc) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag, err, 61)) { ok = false; break; }
          unsigned char* sa = smem + stage * R::kStageBytes;
          mbar_expect_tx(&full[stage], R::kStageBytes);
          tma_load_3d(sa, &tmM, &full[stage], k * kNB + kc * kKC, j * kNB, 0);
          if (kc == 0) {
            // block k of this group's right-hand sides must have been published; on failure
            // the load is still issued so that the stage completes
            if (!wait_flag(p.flags + (size_t)k * G + h, kEpiWarps, abort_flag, err, 62)) ok = false;
            fence_proxy_async_global();
            if (p.trace && last) p.trace[4 * (size_t)u + 1] = globaltimer_ns();
          }
          tma_load_3d(sa + R::kABytes, &tmX, &full[stage], k * kNB + kc * kKC, h * UN, 0);
          next_stage();
        }
      };
      for (int l0 = 0; l0 < nloc && ok; l0 += kSlots) {
        const int nw = min(kSlots, nloc - l0);
        int kfirst = nsteps, klast = -1;  // range of dependent blocks of the window
        for (int i = 0; i < nw && ok; ++i) {
          const int u = unit_id(l0 + i), j = row_of(u), h = u % G, J = j / sb;
          if (p.trace) p.trace[4 * (size_t)u] = globaltimer_ns();
          for (int kc = 0; kc < kChunks * sb; ++kc) {
            if (!mbar_wait(&empty[stage], phase ^ 1u, abort_flag, err, 61)) { ok = false; break; }
            unsigned char* sa = smem + stage * R::kStageBytes;
            mbar_expect_tx(&full[stage], R::kStageBytes);
            tma_load_3d(sa, &tmD, &full[stage], kc * kKC, (2 * J + (FWD ? 0 : 1)) * sb * kNB + (j % sb) * kNB, 0);
            tma_load_3d(sa + R::kABytes, &tmB0, &full[stage], J * sb * kNB + kc * kKC, h * UN, 0);
            next_stage();
          }
          if (has_dep(J)) {
            kfirst = min(kfirst, FWD ? 0 : (J + 1) * sb);
            klast = max(klast, FWD ? J * sb - 1 : nsteps - 1);
          }
        }
        for (int s = 0; s <= klast - kfirst && ok; ++s) {
          const int k = FWD ? kfirst + s : klast - s;
          for (int i = 0; i < nw && ok; ++i) {
            const int u = unit_id(l0 + i), j = row_of(u), h = u % G, J = j / sb;
            if (needs(J, k)) issue_dep(u, j, h, k, k == last_k(J));
          }
        }
      }
      if (!ok) {
        int s = stage;
        uint32_t ph = phase;
        for (int i = 0; i < inflight; ++i) {
          if (--s < 0) { s = kStages - 1; ph ^= 1u; }
          for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(&full[s], ph); ++it) {}
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      auto mma_group = [&](int slot, int nch, bool first, bool negate) {
        const uint32_t t_re = tmem + (uint32_t)(slot * 2 * UN), t_im = t_re + UN;
        for (int kc = 0; kc < nch; ++kc) {
          if (!mbar_wait(&full[stage], phase, abort_flag, err, 64)) { ok = false; break; }
          tc_fence_after();
          mma_chunk<UN>(smem, stage, t_re, t_im, first && kc == 0, negate);
          mma_commit(&empty[stage]);
          if (++stage == kStages) { stage = 0; phase ^= 1u; }
        }
      };
      int win = 0;
      for (int l0 = 0; l0 < nloc && ok; l0 += kSlots, ++win) {
        const int nw = min(kSlots, nloc - l0);
        int kfirst = nsteps, klast = -1;
        for (int i = 0; i < nw && ok; ++i) {
          const int j = row_of(unit_id(l0 + i)), J = j / sb;
          if (!mbar_wait(&acc_empty[i], (uint32_t)(win & 1) ^ 1u, abort_flag, err, 63)) { ok = false; break; }
          tc_fence_after();
          mma_group(i, kChunks * sb, true, true);
          if (!ok) break;
          if (has_dep(J)) {
            kfirst = min(kfirst, FWD ? 0 : (J + 1) * sb);
            klast = max(klast, FWD ? J * sb - 1 : nsteps - 1);
          } else {
            mma_commit(&acc_full[i]);
          }
        }
        for (int s = 0; s <= klast - kfirst && ok; ++s) {
          const int k = FWD ? kfirst + s : klast - s;
          for (int i = 0; i < nw && ok; ++i) {
            const int J = row_of(unit_id(l0 + i)) / sb;
            if (!needs(J, k)) continue;
            mma_group(i, kChunks, false, false);
            if (ok && k == last_k(J)) mma_commit(&acc_full[i]);
          }
        }
      }
      if (!ok || *abort_flag) {
        mma_commit(drain);
        for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(drain, 0); ++it) {}
      }
    }
  } else {
    // epilogue: warp w reads TMEM lane quarter w % 4 (rows), half (w - 2) / 4 of the columns
    const int q = warp & 3;
    const int c_begin = ((warp - 2) >> 2) * (UN / 2);
    int win = 0;
    bool ok = true;
    for (int l0 = 0; l0 < nloc && ok; l0 += kSlots, ++win) {
      const int nw = min(kSlots, nloc - l0);
      for (int i = 0; i < nw; ++i) {
        const int u = unit_id(l0 + i), j = row_of(u), h = u % G;
        if (lane == 0) ok = mbar_wait(&acc_full[i], (uint32_t)(win & 1), abort_flag, err, 65);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        if (p.trace && warp == 2 && lane == 0) p.trace[4 * (size_t)u + 2] = globaltimer_ns();
        __syncwarp();
        tc_fence_after();
        const int row = j * kNB + q * 32 + lane;
        const bool rv = row < N;
        const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(i * 2 * UN);
        constexpr int kCh = UN / 32;  // chunks of 16 columns per warp, read two at a time
        // the planes are what other CTAs wait for: write them, make them visible to the TMA
        // (async proxy) loads of the CTAs that acquire the flag, publish, then the FP32 output
#pragma unroll
        for (int i0 = 0; i0 < kCh; i0 += 2) {
          float re[2][16], im[2][16];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            tmem_ld16(tl + c_begin + 16 * (i0 + c), re[c]);
            tmem_ld16(tl + UN + c_begin + 16 * (i0 + c), im[c]);
          }
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 2; ++c) {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const int col = h * UN + c_begin + 16 * (i0 + c) + e;
              if (rv && col < p.nrhs) {
                float hr, lr, hi, li;
                tf32_split(-re[c][e], hr, lr);
                tf32_split(-im[c][e], hi, li);
                float* d = p.xp + (size_t)col * p.xp_ld + row;
                d[0] = hr;
                d[p.xp_plane] = lr;
                d[2 * p.xp_plane] = hi;
                d[3 * p.xp_plane] = li;
              }
            }
          }
        }
        fence_proxy_async_global();
        __syncwarp();
        if (lane == 0) {
          // release: cumulative over the warp's writes ordered before it by the warp barrier
          asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(p.flags + (size_t)j * G + h) : "memory");
          if (p.trace && warp == 2) p.trace[4 * (size_t)u + 3] = globaltimer_ns();
        }
        if (p.xout) {
#pragma unroll
          for (int i0 = 0; i0 < kCh; i0 += 2) {
            float re[2][16], im[2][16];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              tmem_ld16(tl + c_begin + 16 * (i0 + c), re[c]);
              tmem_ld16(tl + UN + c_begin + 16 * (i0 + c), im[c]);
            }
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
              for (int e = 0; e < 16; ++e) {
                const int col = h * UN + c_begin + 16 * (i0 + c) + e;
                if (rv && col < p.nrhs)
                  p.xout[(size_t)row + (size_t)col * p.ldx] = make_float2(-re[c][e], -im[c][e]);
              }
          }
        }
        tc_fence_before();
        mbar_arrive(&acc_empty[i]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

template <int UN, bool FWD>
int launch_wave(TcGemmPlan& pl, const TcOperand& opM, const TcOperand& opD, const TcOperand& opB0,
                const TcOperand& opX, const WaveArgs& args, int nunits, cudaStream_t s) {
  auto kern = wavefront_kernel<UN, FWD>;
  const int smem = Ring<UN>::kSmemBytes;
  HPR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int grid = nunits < pl.nsm ? nunits : pl.nsm;
  CUtensorMap m = opM.map, d = opD.map, b0 = opB0.map, x = opX.map;
  WaveArgs a = args;
  void* kargs[] = {&m, &d, &b0, &x, &a};
  HPR_CUDA_TRY(cudaLaunchCooperativeKernel((void*)kern, dim3(grid), dim3(kThreads), kargs, (size_t)smem, s));
  return 0;
}

}  // namespace

int wave_perm_chain(const int* swaps, int swap_stride, int N, int nsteps, int* work, int* sig, long sig_ld,
                    int* perm0, cudaStream_t s) {
  perm_chain_kernel<<<1, 1024, 0, s>>>(swaps, swap_stride, N, nsteps, work, work + N, sig, sig_ld, perm0);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int wave_transpose_offdiag(const float* lup, long lup_ld, long lup_plane, const int* sig, long sig_ld, int N,
                           int nsteps, float* T, long ldt, long tplane, cudaStream_t s) {
  dim3 grid((N + 31) / 32, nsteps);
  transpose_offdiag_kernel<<<grid, 256, 0, s>>>(lup, lup_ld, lup_plane, sig, sig_ld, N, T, ldt, tplane);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int wave_dinv_planes(const float2* inv, int nblk, int h, float* di, long di_plane, cudaStream_t s) {
  dinv_planes_kernel<<<dim3(2 * nblk, (h * h + 256 * 64 - 1) / (256 * 64)), 256, 0, s>>>(inv, h, di, di_plane);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int wave_dinv_double(const float2* dfh, int h, int nblk, const float* T, long ldt, long tplane, int N, float2* ptmp,
                     float2* otmp, float2* df2h, cudaStream_t s) {
  const int nsup = (nblk + 1) / 2;
  DinvDouble d{dfh, T, ldt, tplane, N, h, nblk, ptmp};
  const dim3 grid(h / 64, h / 64, 2 * nsup);
  dinv_double_kernel<1><<<grid, 256, 0, s>>>(d, ptmp);
  HPR_CUDA_TRY(cudaGetLastError());
  dinv_double_kernel<2><<<grid, 256, 0, s>>>(d, otmp);
  HPR_CUDA_TRY(cudaGetLastError());
  dinv_assemble_kernel<<<dim3(2 * nsup, (4 * h * h + 256 * 64 - 1) / (256 * 64)), 256, 0, s>>>(dfh, otmp, h, nblk,
                                                                                                 df2h);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int wave_scale_offdiag(TcGemmPlan& pl, const TcOperand& opD, const TcOperand& opT, int N, int nsteps, int sb,
                       float* lup, long lup_ld, long lup_plane, cudaStream_t s) {
  if (nsteps <= sb) return 0;
  if (((uintptr_t)lup & 15) || (lup_ld % 4) || (lup_plane % 4)) {
    set_last_error_msg("off-diagonal scaling: LU planes must be 16-byte aligned");
    return -1;
  }
  const int smem = Ring<kNB>::kSmemBytes;
  HPR_CUDA_TRY(cudaFuncSetAttribute(scale_offdiag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int ntiles = nsteps * (nsteps - 1);
  const int grid = ntiles < pl.nsm ? ntiles : pl.nsm;
  ScaleArgs a{N, nsteps, sb, lup, lup_ld, lup_plane, pl.d_err};
  scale_offdiag_kernel<<<grid, kThreads, smem, s>>>(opD.map, opT.map, a);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int wave_rhs_planes(const float2* X, long ldx, const int* perm0, int N, int nrhs, float* bp, long bld, long bplane,
                    cudaStream_t s) {
  dim3 grid((N + 255) / 256, nrhs);
  rhs_planes_kernel<<<grid, 256, 0, s>>>(X, ldx, perm0, N, bp, bld, bplane);
  HPR_CUDA_TRY(cudaGetLastError());
  return 0;
}

int wave_sweep(TcGemmPlan& pl, bool forward, const TcOperand& opM, const TcOperand& opD, const TcOperand& opB0,
               const TcOperand& opX, const WaveSolve& ws, cudaStream_t s) {
  if (ws.un != 64 && ws.un != 128) {
    set_last_error_msg("wavefront solve: right-hand sides per unit must be 64 or 128");
    return -5;
  }
  const int G = (ws.nrhs + ws.un - 1) / ws.un;
  HPR_CUDA_TRY(cudaMemsetAsync(ws.flags, 0, (size_t)ws.nsteps * G * sizeof(int), s));
  WaveArgs a{ws.N,       ws.nsteps, G,      ws.nrhs, ws.sb,    ws.xp,   ws.xp_ld,
             ws.xp_plane, ws.xout,   ws.ldx, ws.flags, pl.d_err, ws.trace};
  const int nunits = ws.nsteps * G;
  if (ws.un == 64)
    return forward ? launch_wave<64, true>(pl, opM, opD, opB0, opX, a, nunits, s)
                   : launch_wave<64, false>(pl, opM, opD, opB0, opX, a, nunits, s);
  return forward ? launch_wave<128, true>(pl, opM, opD, opB0, opX, a, nunits, s)
                 : launch_wave<128, false>(pl, opM, opD, opB0, opX, a, nunits, s);
}

}  // namespace hprmat

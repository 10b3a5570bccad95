// Blocked right-looking complex LU with partial pivoting, and the triangular solves that
// use its factors.  Templates over the complex element type T (double2 = FP64 path,
// float2 = panels/solves of the mixed path).
//
// Storage: the matrix W is column-major with leading dimension ld (complex elements).
// Block step s factors columns [k0, k0+ncols) with k0 = s*nb:
//   1. panel_kernel      -- cooperative launch, the panel rows spread over all SMs and held
//                           in shared memory; one grid barrier per column: every CTA posts
//                           its local |re|+|im| maximum (the modulus LAPACK's izamax uses)
//                           and that row, then all CTAs pick the same pivot, swap and
//                           eliminate their rows.  Writes ipiv and the step's row-interchange
//                           list.
//   2. trsm_lower_kernel -- applies the step's row interchanges to the columns right of the
//                           panel (or to right-hand sides) and solves with the unit lower
//                           diagonal block: U12 = L11^-1 P A12.
//   3. trailing update   -- A22 -= L21 U12 (cgemm_update_kernel here; the mixed path uses
//                           the tcgen05 kernel of tc_gemm.cu).
// Row interchanges are applied only to columns at or right of the current panel; the
// forward solve applies each step's interchanges to the right-hand side just before that
// step's block column, which is consistent with the factors stored that way.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"

namespace hprmat {

constexpr int kMaxNB = 128;

// Row-interchange list of one block step (global row indices).
struct StepSwaps {
  int* top_src;    // [nbmax]  source row of final row k0+j, j < ncols
  int* extra_dst;  // [nbmax]  rows >= k0+ncols that receive a displaced row
  int* extra_src;  // [nbmax]
  int* n_extra;    // [1]
};

template <typename T>
struct PanelArgs {
  T* W;
  long ld;
  int N, k0, ncols, rpc, G;
  int* ipiv;                      // [N] global pivot rows (0-based)
  T* cand_rows;                   // [2][G][NB]
  unsigned long long* keys;       // [NB] winning pivot key per panel column (zeroed per launch)
  T* rowj;                        // [2][NB]
  int* status;                    // device status block
  StepSwaps sw;
  unsigned* growth_bits;          // running max |u_ij| (mag_hi key)
  // Optional (mixed path): the "LU planes", hi/lo TF32 splits of Re/Im of the factors,
  // row-major (row stride lup_ld floats, planes lup_plane floats apart).  The panel writes
  // its L21 rows there; they are the K-major A operand of the tensor-core updates.
  float* lup;
  long lup_ld;
  long lup_plane;
  // Optional timing trace, per column kPanelTraceW stamps: CTA 0 at column start, candidate
  // posted, barrier passed, pivot row in place, update done; then every CTA's arrival.
  long long* trace = nullptr;
};
constexpr int kPanelTraceW = 5 + 160;

// Pivot candidates are compared by PivotKey<T> (common.cuh): |re|+|im| as an integer key
// that orders over the element type's whole range (FP64 panels: magnitudes far outside the
// float range too), with the lowest row winning among equal moduli.

// End of a panel factorisation, shared by both panel kernels: the CTA's factored rows back
// into W, its L21 rows into the LU planes (mixed path), and from CTA 0 the pivots, the growth
// and the step's row-interchange list.
template <typename T, int NB, int NT>
__device__ void panel_finish(const PanelArgs<T>& a, const T* P, int rpcp, int r0, int nloc, const int* s_loc_ipiv,
                             unsigned s_growth, int b, int tid) {
  const int ncols = a.ncols;
  // write the factored rows back
  for (int c = 0; c < ncols; ++c)
    for (int lr = tid; lr < nloc; lr += NT)
      a.W[(size_t)(a.k0 + r0 + lr) + (size_t)(a.k0 + c) * a.ld] = P[(size_t)c * rpcp + lr];
  // L21 rows into the LU planes (mixed path): global row k0 + g, columns k0 .. k0+ncols
  if (a.lup != nullptr) {
    const int lr0 = max(ncols - r0, 0);
    const int nl = nloc - lr0;
    for (int idx = tid; idx < nl * ncols; idx += NT) {
      int c = idx % ncols;
      int lr = lr0 + idx / ncols;
      size_t off = (size_t)(a.k0 + r0 + lr) * a.lup_ld + (size_t)(a.k0 + c);
      float hr, lrr, hi_, li;
      T v = P[(size_t)c * rpcp + lr];
      tf32_split((float)v.x, hr, lrr);
      tf32_split((float)v.y, hi_, li);
      a.lup[off] = hr;
      a.lup[a.lup_plane + off] = lrr;
      a.lup[2 * a.lup_plane + off] = hi_;
      a.lup[3 * a.lup_plane + off] = li;
    }
  }
  if (b == 0) {
    __syncthreads();
    if (tid < ncols) a.ipiv[a.k0 + tid] = a.k0 + s_loc_ipiv[tid];
    if (tid == 0 && a.growth_bits) atomicMax(a.growth_bits, s_growth);
    // Row-interchange list of this step: simulate the swaps on the touched positions.
    if (tid < 32) {
      __shared__ int pos[2 * NB], src[2 * NB];
      __shared__ int cnt;
      for (int j = tid; j < ncols; j += 32) { pos[j] = a.k0 + j; src[j] = a.k0 + j; }
      if (tid == 0) cnt = ncols;
      __syncwarp();
      for (int j = 0; j < ncols; ++j) {
        int bp = a.k0 + s_loc_ipiv[j];
        if (bp == a.k0 + j) continue;
        int slot;
        if (bp < a.k0 + ncols) {
          slot = bp - a.k0;
        } else {
          int found = -1;
          for (int base = ncols; base < cnt; base += 32) {
            int s = base + tid;
            unsigned m_ = __ballot_sync(0xffffffffu, s < cnt && pos[s] == bp);
            if (m_) { found = base + __ffs(m_) - 1; break; }
          }
          if (found < 0) {
            if (tid == 0) { pos[cnt] = bp; src[cnt] = bp; cnt = cnt + 1; }
            __syncwarp();
            found = cnt - 1;
          }
          slot = found;
        }
        if (tid == 0) { int t = src[j]; src[j] = src[slot]; src[slot] = t; }
        __syncwarp();
      }
      for (int j = tid; j < ncols; j += 32) a.sw.top_src[j] = src[j];
      if (tid == 0) {
        int ne = 0;
        for (int s = ncols; s < cnt; ++s)
          if (src[s] != pos[s]) { a.sw.extra_dst[ne] = pos[s]; a.sw.extra_src[ne] = src[s]; ++ne; }
        *a.sw.n_extra = ne;
      }
    }
  }
}

template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT, 1) panel_kernel(PanelArgs<T> a) {
  using R = typename RealOf<T>::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = a.N - a.k0;
  const int b = blockIdx.x;
  const int r0 = b * a.rpc;
  const int r1 = min(r0 + a.rpc, m);
  const int nloc = max(r1 - r0, 0);
  const int rpcp = a.rpc | 1;  // odd column stride: conflict-free row gathers
  T* P = reinterpret_cast<T*>(smem_raw);                 // [NB][rpcp] column-major
  T* urow = P + (size_t)NB * rpcp;                       // [NB]
  using PK = PivotKey<T>;
  using PM = typename PK::M;
  __shared__ PM red_v[NT / 32];
  __shared__ int red_i[NT / 32];
  __shared__ int s_piv, s_loc_ipiv[NB];
  __shared__ unsigned s_growth;
  const int tid = threadIdx.x;
  const int ncols = a.ncols;

  // load rows [r0, r1) of the panel
  for (int c = 0; c < ncols; ++c)
    for (int lr = tid; lr < nloc; lr += NT)
      P[(size_t)c * rpcp + lr] = a.W[(size_t)(a.k0 + r0 + lr) + (size_t)(a.k0 + c) * a.ld];
  if (tid == 0) s_growth = 0u;
  __syncthreads();

  // Column jc's pivot candidate: the largest |re|+|im| of the local rows >= jc (lowest row on
  // ties) into s_piv, and its key into the column's global maximum.  v_of(lr) gives the
  // current value of column jc in local row lr.
  auto candidate = [&](int jc, PM bv, int bi) {
    for (int o = 16; o > 0; o >>= 1) {
      PM ov = __shfl_down_sync(0xffffffffu, bv, o);
      int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { red_v[tid >> 5] = bv; red_i[tid >> 5] = bi; }
    __syncthreads();
    if (tid < 32) {
      bv = (tid < NT / 32) ? red_v[tid] : PM(0);
      bi = (tid < NT / 32) ? red_i[tid] : 0x7fffffff;
      for (int o = 16; o > 0; o >>= 1) {
        PM ov = __shfl_down_sync(0xffffffffu, bv, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (tid == 0) {
        s_piv = bi;
        if (bi != 0x7fffffff) atomicMax(a.keys + jc, PK::key(bv, bi));
      }
    }
    __syncthreads();
  };
  // Post the candidate row of column jc and, from its owner, row jc.  Columns > jc still
  // wait for the rank-1 update of column jc - 1 (multipliers in column jc - 1, pivot row in
  // urow) when pend is set; the posted values include it.
  auto post = [&](int jc, bool pend) {
    const int pb = jc & 1;
    const int ci = s_piv;
    const bool have = ci != 0x7fffffff;
    const bool own = jc >= r0 && jc < r1;
    for (int c = tid; c < ncols; c += NT) {
      if (have) {
        T v = P[(size_t)c * rpcp + (ci - r0)];
        if (pend && c > jc) cfms(v, P[(size_t)(jc - 1) * rpcp + (ci - r0)], urow[c]);
        a.cand_rows[((size_t)pb * a.G + b) * NB + c] = v;
      }
      if (own) {
        T v = P[(size_t)c * rpcp + (jc - r0)];
        if (pend && c > jc) cfms(v, P[(size_t)(jc - 1) * rpcp + (jc - r0)], urow[c]);
        a.rowj[(size_t)pb * NB + c] = v;
      }
    }
  };
  auto arrive = [&](int jc) {
    __syncthreads();
    if (tid == 0) {
      if (a.trace) {
        const long long t = device_ns();
        long long* tr = a.trace + (size_t)jc * kPanelTraceW;
        if (b < 160) tr[5 + b] = t;
        if (b == 0) tr[1] = t;
      }
      grid_arrive(a.status + SW_BARRIER);
    }
  };

  // column 0: candidate, post, arrive
  {
    PM bv = 0;
    int bi = 0x7fffffff;
    for (int lr = max(-r0, 0) + tid; lr < nloc; lr += NT) {
      const PM v = PK::mag(P[lr]);
      if (v > bv) { bv = v; bi = r0 + lr; }
    }
    candidate(0, bv, bi);
    post(0, false);
    arrive(0);
  }
  const int warp = tid >> 5, lane = tid & 31;
  for (int j = 0; j < ncols; ++j) {
    const int buf = j & 1;
    long long* tr = a.trace ? a.trace + (size_t)j * kPanelTraceW : nullptr;
    if (tr && b == 0 && tid == 0) tr[0] = device_ns();
    // every CTA has posted its candidate of column j
    if (!grid_wait(a.status + SW_BARRIER, a.status + SW_TIMEOUT, (unsigned)a.G * (j + 1), 1)) return;
    if (tr && b == 0 && tid == 0) tr[2] = device_ns();
    // the winning key names the pivot row; its owner CTA is row / rpc
    if (tid == 0) {
      unsigned long long key = __ldcg(a.keys + j);
      s_piv = PK::row(key);
    }
    __syncthreads();
    const int p = s_piv;
    const int win = p / a.rpc;
    unsigned g = 0u;  // pivot growth: largest |re|+|im| in the U part of the pivot row (mag_hi key)
    for (int c = tid; c < ncols; c += NT) {
      T u = __ldcg(reinterpret_cast<const T*>(a.cand_rows) + ((size_t)buf * a.G + win) * NB + c);
      urow[c] = u;
      if (p != j && p >= r0 && p < r1)
        P[(size_t)c * rpcp + (p - r0)] = __ldcg(reinterpret_cast<const T*>(a.rowj) + (size_t)buf * NB + c);
      if (p != j && j >= r0 && j < r1) P[(size_t)c * rpcp + (j - r0)] = u;
      if (c >= j) g = max(g, mag_hi((double)cabs1(u)));
    }
    if (tid < ((ncols + 31) & ~31)) {  // whole warps that may hold entries
      for (int o = 16; o > 0; o >>= 1) g = max(g, __shfl_down_sync(0xffffffffu, g, o));
      if ((tid & 31) == 0 && g > 0u) atomicMax(&s_growth, g);
    }
    if (tid == 0) s_loc_ipiv[j] = p;
    __syncthreads();
    if (tr && b == 0 && tid == 0) tr[3] = device_ns();
    // scale column j below the diagonal (multipliers; a zero pivot leaves them unscaled, as
    // xGETF2 does, and is reported in info)
    const T piv = urow[j];
    const bool zero = (piv.x == R(0) && piv.y == R(0));
    if (zero && b == 0 && tid == 0) atomicCAS(a.status + SW_INFO, 0, a.k0 + j + 1);
    const T inv = zero ? czero<T>() : crecip(piv);
    const int lo = max(j + 1 - r0, 0);
    if (j + 1 < ncols) {
      // column j + 1 first: scale, update, candidate; post it and arrive, then finish the
      // rank-1 update of columns j + 2 .. while the other CTAs arrive
      const int jn = j + 1;
      PM bv = 0;
      int bi = 0x7fffffff;
      for (int lr = lo + tid; lr < nloc; lr += NT) {
        T l = P[(size_t)j * rpcp + lr];
        if (!zero) {
          l = cmul(l, inv);
          P[(size_t)j * rpcp + lr] = l;
        }
        T v = P[(size_t)jn * rpcp + lr];
        cfms(v, l, urow[jn]);
        P[(size_t)jn * rpcp + lr] = v;
        const PM av = PK::mag(v);
        if (av > bv) { bv = av; bi = r0 + lr; }
      }
      candidate(jn, bv, bi);
      post(jn, true);
      arrive(jn);
      // rank-1 update of columns j + 2 .. ncols - 1: lanes over rows, warps over columns,
      // four independent columns per step
      constexpr int NW = NT / 32;
      for (int lr = lo + lane; lr < nloc; lr += 32) {
        const T l = P[(size_t)j * rpcp + lr];
        int c = jn + 1 + warp;
        for (; c + 3 * NW < ncols; c += 4 * NW) {
          T v[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) v[q] = P[(size_t)(c + q * NW) * rpcp + lr];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            cfms(v[q], l, urow[c + q * NW]);
            P[(size_t)(c + q * NW) * rpcp + lr] = v[q];
          }
        }
        for (; c < ncols; c += NW) {
          T v = P[(size_t)c * rpcp + lr];
          cfms(v, l, urow[c]);
          P[(size_t)c * rpcp + lr] = v;
        }
      }
      __syncthreads();
    } else {
      for (int lr = lo + tid; lr < nloc; lr += NT) {
        if (!zero) P[(size_t)j * rpcp + lr] = cmul(P[(size_t)j * rpcp + lr], inv);
      }
      __syncthreads();
    }
    if (tr && b == 0 && tid == 0) tr[4] = device_ns();
  }

  panel_finish<T, NB, NT>(a, P, rpcp, r0, nloc, s_loc_ipiv, s_growth, b, tid);
}

// -------------------------------------------------------------------------------------
// The panel factorisation of panel_kernel for panels whose rows fit in one thread-block
// cluster (G <= 16 CTAs, the whole grid): the same algorithm and look-ahead, with the
// per-column exchange in distributed shared memory instead of global memory.  Each CTA pushes
// its pivot key into every CTA's shared memory and posts its candidate row and (the owner)
// row j in its own; after the hardware cluster barrier every CTA reduces the G keys locally,
// picks the same pivot and reads the two rows from their owners (one remote round trip).
// Double buffering by column parity is safe because a CTA posts column j + 2 only after the
// barrier of column j + 1, which every CTA reaches after reading column j.  There is no
// polling: the waits are the cluster barrier's.  Dynamic shared memory: P [NB][rpc|1],
// urow [NB], candidate rows [2][NB], rows j [2][NB], keys [2][16].
namespace cgx = cooperative_groups;

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

constexpr int kMaxClusterCTAs = 16;

template <typename T>
__host__ __device__ constexpr size_t panel_cluster_smem(int rpc, int nb) {
  return ((size_t)nb * (size_t)(rpc | 1) + 5 * (size_t)nb) * sizeof(T) +
         2 * kMaxClusterCTAs * sizeof(unsigned long long) + 16;
}

template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT, 1) panel_cluster_kernel(PanelArgs<T> a) {
  using R = typename RealOf<T>::R;
  cgx::cluster_group cluster = cgx::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = a.N - a.k0;
  const int b = (int)cluster.block_rank();
  const int r0 = b * a.rpc;
  const int r1 = min(r0 + a.rpc, m);
  const int nloc = max(r1 - r0, 0);
  const int rpcp = a.rpc | 1;
  T* P = reinterpret_cast<T*>(smem_raw);  // [NB][rpcp] column-major
  T* urow = P + (size_t)NB * rpcp;        // [NB]
  T* xrow = urow + NB;                    // [2][NB] candidate row posted by this CTA
  T* xrowj = xrow + 2 * NB;               // [2][NB] row j, posted by its owner
  // [2][kMaxClusterCTAs]: every CTA's pivot key, pushed into every CTA before the barrier
  unsigned long long* xkey = reinterpret_cast<unsigned long long*>(xrowj + 2 * NB);
  using PK = PivotKey<T>;
  using PM = typename PK::M;
  __shared__ PM red_v[NT / 32];
  __shared__ int red_i[NT / 32];
  __shared__ int s_piv, s_loc_ipiv[NB];
  __shared__ unsigned s_growth;
  const int tid = threadIdx.x;
  const int ncols = a.ncols;

  for (int c = 0; c < ncols; ++c)
    for (int lr = tid; lr < nloc; lr += NT)
      P[(size_t)c * rpcp + lr] = a.W[(size_t)(a.k0 + r0 + lr) + (size_t)(a.k0 + c) * a.ld];
  if (tid == 0) s_growth = 0u;
  __syncthreads();

  // column jc's local candidate into s_piv, and its key into slot b of xkey[jc & 1] of every
  // CTA of the cluster (lane t of warp 0 stores into CTA t)
  auto candidate = [&](int jc, PM bv, int bi) {
    for (int o = 16; o > 0; o >>= 1) {
      PM ov = __shfl_down_sync(0xffffffffu, bv, o);
      int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { red_v[tid >> 5] = bv; red_i[tid >> 5] = bi; }
    __syncthreads();
    if (tid < 32) {
      bv = (tid < NT / 32) ? red_v[tid] : PM(0);
      bi = (tid < NT / 32) ? red_i[tid] : 0x7fffffff;
      for (int o = 16; o > 0; o >>= 1) {
        PM ov = __shfl_down_sync(0xffffffffu, bv, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (tid == 0) s_piv = bi;
      const unsigned long long key = __shfl_sync(0xffffffffu, bi != 0x7fffffff ? PK::key(bv, bi) : 0ull, 0);
      if (tid < a.G) *cluster.map_shared_rank(xkey + (jc & 1) * kMaxClusterCTAs + b, (unsigned)tid) = key;
    }
    __syncthreads();
  };
  auto post = [&](int jc, bool pend) {
    const int pb = jc & 1;
    const int ci = s_piv;
    const bool have = ci != 0x7fffffff;
    const bool own = jc >= r0 && jc < r1;
    for (int c = tid; c < ncols; c += NT) {
      if (have) {
        T v = P[(size_t)c * rpcp + (ci - r0)];
        if (pend && c > jc) cfms(v, P[(size_t)(jc - 1) * rpcp + (ci - r0)], urow[c]);
        xrow[pb * NB + c] = v;
      }
      if (own) {
        T v = P[(size_t)c * rpcp + (jc - r0)];
        if (pend && c > jc) cfms(v, P[(size_t)(jc - 1) * rpcp + (jc - r0)], urow[c]);
        xrowj[pb * NB + c] = v;
      }
    }
  };

  {
    PM bv = 0;
    int bi = 0x7fffffff;
    for (int lr = tid; lr < nloc; lr += NT) {
      const PM v = PK::mag(P[lr]);
      if (v > bv) { bv = v; bi = r0 + lr; }
    }
    candidate(0, bv, bi);
    post(0, false);
    cluster_arrive();
  }
  const int warp = tid >> 5, lane = tid & 31;
  for (int j = 0; j < ncols; ++j) {
    const int buf = j & 1;
    cluster_wait();
    // the largest key names the pivot row (the lowest row among equal moduli); every warp
    // reduces the G keys, now in local shared memory, itself
    unsigned long long kmax;
    {
      const int lane_ = tid & 31;
      unsigned long long k = lane_ < a.G ? xkey[buf * kMaxClusterCTAs + lane_] : 0ull;
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, k, o);
        k = v > k ? v : k;
      }
      kmax = k;
    }
    const int p = PK::row(kmax);
    const T* wrow = cluster.map_shared_rank(xrow + buf * NB, (unsigned)(p / a.rpc));
    const T* jrow = cluster.map_shared_rank(xrowj + buf * NB, (unsigned)(j / a.rpc));
    unsigned g = 0u;
    for (int c = tid; c < ncols; c += NT) {
      T u = wrow[c];
      urow[c] = u;
      if (p != j && p >= r0 && p < r1) P[(size_t)c * rpcp + (p - r0)] = jrow[c];
      if (p != j && j >= r0 && j < r1) P[(size_t)c * rpcp + (j - r0)] = u;
      if (c >= j) g = max(g, mag_hi((double)cabs1(u)));
    }
    if (tid < ((ncols + 31) & ~31)) {
      for (int o = 16; o > 0; o >>= 1) g = max(g, __shfl_down_sync(0xffffffffu, g, o));
      if ((tid & 31) == 0 && g > 0u) atomicMax(&s_growth, g);
    }
    if (tid == 0) s_loc_ipiv[j] = p;
    __syncthreads();
    const T piv = urow[j];
    const bool zero = (piv.x == R(0) && piv.y == R(0));
    if (zero && b == 0 && tid == 0) atomicCAS(a.status + SW_INFO, 0, a.k0 + j + 1);
    const T inv = zero ? czero<T>() : crecip(piv);
    const int lo = max(j + 1 - r0, 0);
    if (j + 1 < ncols) {
      const int jn = j + 1;
      PM bv = 0;
      int bi = 0x7fffffff;
      for (int lr = lo + tid; lr < nloc; lr += NT) {
        T l = P[(size_t)j * rpcp + lr];
        if (!zero) {
          l = cmul(l, inv);
          P[(size_t)j * rpcp + lr] = l;
        }
        T v = P[(size_t)jn * rpcp + lr];
        cfms(v, l, urow[jn]);
        P[(size_t)jn * rpcp + lr] = v;
        const PM av = PK::mag(v);
        if (av > bv) { bv = av; bi = r0 + lr; }
      }
      candidate(jn, bv, bi);
      post(jn, true);
      cluster_arrive();
      constexpr int NW = NT / 32;
      for (int lr = lo + lane; lr < nloc; lr += 32) {
        const T l = P[(size_t)j * rpcp + lr];
        int c = jn + 1 + warp;
        for (; c + 3 * NW < ncols; c += 4 * NW) {
          T v[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) v[q] = P[(size_t)(c + q * NW) * rpcp + lr];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            cfms(v[q], l, urow[c + q * NW]);
            P[(size_t)(c + q * NW) * rpcp + lr] = v[q];
          }
        }
        for (; c < ncols; c += NW) {
          T v = P[(size_t)c * rpcp + lr];
          cfms(v, l, urow[c]);
          P[(size_t)c * rpcp + lr] = v;
        }
      }
      __syncthreads();
    } else {
      for (int lr = lo + tid; lr < nloc; lr += NT) {
        if (!zero) P[(size_t)j * rpcp + lr] = cmul(P[(size_t)j * rpcp + lr], inv);
      }
      __syncthreads();
    }
  }
  // no CTA leaves while another may still read its shared memory
  cluster_arrive();
  cluster_wait();
  panel_finish<T, NB, NT>(a, P, rpcp, r0, nloc, s_loc_ipiv, s_growth, b, tid);
}

// -------------------------------------------------------------------------------------
// Apply the step's row interchanges to columns [c_begin, c_end) of X and solve with the
// unit lower triangle L11 = W[k0:k0+ncols, k0:k0+ncols].  Optionally emit the result as the
// B-operand planes of the mixed path (per column, NB consecutive K values).
template <typename T>
struct TrsmArgs {
  const T* W;
  long ld;
  int k0, ncols;
  const int* top_src;
  const int* extra_dst;
  const int* extra_src;
  const int* n_extra;
  T* X;
  long ldx;
  int c_begin, c_end;
  float* bop;        // optional B-operand planes
  long bop_plane;
  int bop_col0;      // column of X that maps to B-operand column 0
  unsigned* growth_bits;
  float* lup;        // optional LU planes: U12 rows k0.. (row-major, see PanelArgs)
  long lup_ld;
  long lup_plane;
  int mode;          // 0: interchanges and solve; 1: interchanges only; 2: solve only (rows k0..)
};

template <typename T, int NB, int CW, int NT>
__global__ void __launch_bounds__(NT) trsm_lower_kernel(TrsmArgs<T> a) {
  using R = typename RealOf<T>::R;
  constexpr int NBP = NB + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);  // [CW][NBP]
  T* E = A + CW * NBP;                    // [CW][NB]
  const int tid = threadIdx.x;
  const int cb = a.c_begin + blockIdx.x * CW;
  const int ncw = min(CW, a.c_end - cb);
  if (ncw <= 0) return;
  const int ncols = a.ncols;
  const bool swap = a.mode != 2, solve = a.mode != 1;
  const int ne = swap ? *a.n_extra : 0;
  for (int idx = tid; idx < ncw * ncols; idx += NT) {
    int j = idx % ncols, cc = idx / ncols;
    A[cc * NBP + j] = a.X[(size_t)(swap ? a.top_src[j] : a.k0 + j) + (size_t)(cb + cc) * a.ldx];
  }
  for (int idx = tid; idx < ncw * ne; idx += NT) {
    int e = idx % ne, cc = idx / ne;
    E[cc * NB + e] = a.X[(size_t)a.extra_src[e] + (size_t)(cb + cc) * a.ldx];
  }
  __syncthreads();
  for (int idx = tid; idx < ncw * ne; idx += NT) {
    int e = idx % ne, cc = idx / ne;
    a.X[(size_t)a.extra_dst[e] + (size_t)(cb + cc) * a.ldx] = E[cc * NB + e];
  }
  for (int j = 0; j < (solve ? ncols - 1 : 0); ++j) {
    __syncthreads();
    const int nr = ncols - j - 1;
    const T* Lcol = a.W + (size_t)(a.k0 + j) * a.ld + a.k0;
    for (int idx = tid; idx < nr * ncw; idx += NT) {
      int i = j + 1 + idx % nr, cc = idx / nr;
      T l = Lcol[i];
      T v = A[cc * NBP + i];
      cfms(v, l, A[cc * NBP + j]);
      A[cc * NBP + i] = v;
    }
  }
  __syncthreads();
  R gmax = R(0);
  for (int idx = tid; idx < ncw * ncols; idx += NT) {
    int j = idx % ncols, cc = idx / ncols;
    T v = A[cc * NBP + j];
    a.X[(size_t)(a.k0 + j) + (size_t)(cb + cc) * a.ldx] = v;
    gmax = fmax(gmax, cabs1(v));
  }
  if (a.growth_bits && solve) {
    for (int o = 16; o > 0; o >>= 1) gmax = fmax(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
    if ((tid & 31) == 0) atomicMax(a.growth_bits, mag_hi((double)gmax));
  }
  if (a.lup != nullptr) {
    for (int idx = tid; idx < ncw * ncols; idx += NT) {
      int cc = idx % ncw, j = idx / ncw;
      float hr, lr, hi_, li;
      T v = A[cc * NBP + j];
      tf32_split((float)v.x, hr, lr);
      tf32_split((float)v.y, hi_, li);
      size_t off = (size_t)(a.k0 + j) * a.lup_ld + (size_t)(cb + cc);
      a.lup[off] = hr;
      a.lup[a.lup_plane + off] = lr;
      a.lup[2 * a.lup_plane + off] = hi_;
      a.lup[3 * a.lup_plane + off] = li;
    }
  }
  if (a.bop != nullptr) {
    for (int idx = tid; idx < ncw * NB; idx += NT) {
      int j = idx % NB, cc = idx / NB;
      float hr = 0.f, lr = 0.f, hi_ = 0.f, li = 0.f;
      if (j < ncols) {
        T v = A[cc * NBP + j];
        tf32_split((float)v.x, hr, lr);
        tf32_split((float)v.y, hi_, li);
      }
      size_t off = (size_t)(cb + cc - a.bop_col0) * NB + j;
      a.bop[0 * a.bop_plane + off] = hr;
      a.bop[1 * a.bop_plane + off] = lr;
      a.bop[2 * a.bop_plane + off] = hi_;
      a.bop[3 * a.bop_plane + off] = li;
    }
  }
}

// dst[i + j ldd] = W[src(i) + (col0 + j) ld], i < nr, j < ncol, src(i) = rows[i] (or row0 + i
// without a row list): a block of W, optionally with its rows gathered.
template <typename T>
__global__ void gather_block_kernel(const T* __restrict__ W, long ld, const int* __restrict__ rows, int row0, int nr,
                                    int col0, int ncol, T* __restrict__ dst, long ldd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  const int src = rows ? rows[i] : row0 + i;
  for (int j = blockIdx.y; j < ncol; j += gridDim.y) dst[(size_t)i + (size_t)j * ldd] = W[(size_t)src + (size_t)(col0 + j) * ld];
}

// The rows of a step's interchange list that move below the panel: dst[(extra_dst[e] - row0) +
// j ldd] = W[extra_src[e] + (col0 + j) ld], e < *n_extra, j < ncol.
template <typename T>
__global__ void patch_rows_kernel(const T* __restrict__ W, long ld, const int* __restrict__ extra_dst,
                                  const int* __restrict__ extra_src, const int* __restrict__ n_extra, int row0,
                                  int col0, int ncol, T* __restrict__ dst, long ldd) {
  const int ne = *n_extra;
  for (int idx = threadIdx.x; idx < ne * ncol; idx += blockDim.x) {
    const int e = idx % ne, j = idx / ne;
    dst[(size_t)(extra_dst[e] - row0) + (size_t)j * ldd] = W[(size_t)extra_src[e] + (size_t)(col0 + j) * ld];
  }
}

// Solve with the upper triangle U11 = W[k0:k0+ncols, k0:k0+ncols] (non-unit diagonal) for
// rows k0..k0+ncols of columns [c_begin, c_end) of X.
template <typename T, int NB, int CW, int NT>
__global__ void __launch_bounds__(NT) trsm_upper_kernel(const T* __restrict__ W, long ld, int k0,
                                                        int ncols, T* X, long ldx, int c_begin,
                                                        int c_end) {
  constexpr int NBP = NB + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);  // [CW][NBP]
  T* rd = A + CW * NBP;                   // [NB]
  const int tid = threadIdx.x;
  const int cb = c_begin + blockIdx.x * CW;
  const int ncw = min(CW, c_end - cb);
  if (ncw <= 0) return;
  for (int j = tid; j < ncols; j += NT) {
    T d = W[(size_t)(k0 + j) + (size_t)(k0 + j) * ld];
    rd[j] = (d.x == 0 && d.y == 0) ? czero<T>() : crecip(d);
  }
  for (int idx = tid; idx < ncw * ncols; idx += NT) {
    int j = idx % ncols, cc = idx / ncols;
    A[cc * NBP + j] = X[(size_t)(k0 + j) + (size_t)(cb + cc) * ldx];
  }
  for (int j = ncols - 1; j >= 0; --j) {
    __syncthreads();
    for (int cc = tid; cc < ncw; cc += NT) A[cc * NBP + j] = cmul(A[cc * NBP + j], rd[j]);
    __syncthreads();
    if (j == 0) break;
    const T* Ucol = W + (size_t)(k0 + j) * ld + k0;
    for (int idx = tid; idx < j * ncw; idx += NT) {
      int i = idx % j, cc = idx / j;
      T v = A[cc * NBP + i];
      cfms(v, Ucol[i], A[cc * NBP + j]);
      A[cc * NBP + i] = v;
    }
  }
  __syncthreads();
  for (int idx = tid; idx < ncw * ncols; idx += NT) {
    int j = idx % ncols, cc = idx / ncols;
    X[(size_t)(k0 + j) + (size_t)(cb + cc) * ldx] = A[cc * NBP + j];
  }
}

// -------------------------------------------------------------------------------------
// C[M x N] -= A[M x K] * B[K x N], all column-major complex (SIMT, FMA units).  Used for
// the FP64 LU's trailing update, the block updates of the triangular solves and the dense
// FP64 residual.  64 x 64 output tile per 256-thread CTA, 4 x 4 outputs per thread,
// K staged through shared memory 16 at a time.
template <typename T>
__global__ void __launch_bounds__(256) cgemm_update_kernel(int M, int N, int K, const T* __restrict__ A,
                                                           long lda, const T* __restrict__ B, long ldb,
                                                           T* C, long ldc) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ T As[BK][BM];
  __shared__ T Bs[BK][BN + 1];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = czero<T>();
  for (int kb = 0; kb < K; kb += BK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + 256 * q;
      int r = e & 63, k = e >> 6;
      int gm = m0 + r, gk = kb + k;
      As[k][r] = (gm < M && gk < K) ? A[(size_t)gm + (size_t)gk * lda] : czero<T>();
      int kk = e & 15, cc = e >> 4;
      int gn = n0 + cc, gk2 = kb + kk;
      Bs[kk][cc] = (gn < N && gk2 < K) ? B[(size_t)gk2 + (size_t)gn * ldb] : czero<T>();
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      T av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[k][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[k][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gm = m0 + tx + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + ty + 16 * j;
      if (gn >= N) continue;
      T* p = C + (size_t)gm + (size_t)gn * ldc;
      T v = *p;
      v.x -= acc[i][j].x;
      v.y -= acc[i][j].y;
      *p = v;
    }
  }
}

// C[M x N] -= A[M x K] * B[K x N] for few columns (N <= 8, K <= 128): the block updates of
// triangular solves with one or a few right-hand sides, where the 64 x 64 tiles of
// cgemm_update_kernel would compute mostly empty columns.  One thread per row of A (coalesced
// column reads), B staged in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) cgemv_update_kernel(int M, int N, int K, const T* __restrict__ A, long lda,
                                                           const T* __restrict__ B, long ldb, T* C, long ldc) {
  constexpr int kMaxN = 8, kMaxK = 128;
  __shared__ T Bs[kMaxN][kMaxK];
  for (int e = threadIdx.x; e < K * N; e += blockDim.x) {
    const int k = e % K, n = e / K;
    Bs[n][k] = B[(size_t)k + (size_t)n * ldb];
  }
  __syncthreads();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  T acc[kMaxN];
#pragma unroll
  for (int n = 0; n < kMaxN; ++n) acc[n] = czero<T>();
  for (int k = 0; k < K; ++k) {
    const T a = A[(size_t)m + (size_t)k * lda];
#pragma unroll
    for (int n = 0; n < kMaxN; ++n)
      if (n < N) cfma(acc[n], a, Bs[n][k]);
  }
#pragma unroll
  for (int n = 0; n < kMaxN; ++n) {
    if (n < N) {
      T* p = C + (size_t)m + (size_t)n * ldc;
      T v = *p;
      v.x -= acc[n].x;
      v.y -= acc[n].y;
      *p = v;
    }
  }
}

// -------------------------------------------------------------------------------------
// Explicit inverses of the diagonal blocks, used by the triangular solves with many
// right-hand sides (each block solve becomes a small dense product instead of a chain of
// nb dependent steps).  blockIdx.x = step, blockIdx.y = 0: unit lower L11, 1: upper U11.
// Output per step: inv[(2*s + y) * NB * NB], column-major NB x NB, zero outside the
// triangle, explicit unit diagonal for L11^-1.  In-place column sweeps as LAPACK's
// xTRTI2: lower from the last column backwards, upper from the first column onwards.
template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT) tri_inverse_kernel(const T* __restrict__ W, long ld, int N, int nb,
                                                         T* inv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);  // [NB][NB] column-major
  T* tmp = S + NB * NB;                   // [NB]
  const int s = blockIdx.x;
  const bool upper = blockIdx.y == 1;
  const int k0 = s * nb;
  const int nc = min(nb, N - k0);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NB * NB; idx += NT) {
    int i = idx % NB, j = idx / NB;
    T v = czero<T>();
    if (i < nc && j < nc) {
      if ((!upper && i > j) || (upper && i <= j)) v = W[(size_t)(k0 + i) + (size_t)(k0 + j) * ld];
      if (!upper && i == j) v.x = 1;
    }
    if (i >= nc && i == j) v.x = 1;  // identity padding keeps the padded block invertible
    S[idx] = v;
  }
  __syncthreads();
  if (!upper) {
    for (int j = nc - 2; j >= 0; --j) {
      for (int i = j + 1 + tid; i < nc; i += NT) tmp[i] = S[i + j * NB];
      __syncthreads();
      for (int i = j + 1 + tid; i < nc; i += NT) {
        T acc = czero<T>();
        for (int k = j + 1; k <= i; ++k) cfma(acc, S[i + k * NB], tmp[k]);  // S[i][i] = 1
        acc.x = -acc.x;
        acc.y = -acc.y;
        S[i + j * NB] = acc;
      }
      __syncthreads();
    }
  } else {
    for (int j = 0; j < nc; ++j) {
      for (int i = tid; i <= j; i += NT) tmp[i] = S[i + j * NB];
      __syncthreads();
      T d = tmp[j];
      T dinv = (d.x == 0 && d.y == 0) ? czero<T>() : crecip(d);
      for (int i = tid; i < j; i += NT) {
        T acc = czero<T>();
        for (int k = i; k < j; ++k) cfma(acc, S[i + k * NB], tmp[k]);
        acc = cmul(acc, dinv);
        acc.x = -acc.x;
        acc.y = -acc.y;
        S[i + j * NB] = acc;
      }
      if (tid == 0) S[j + j * NB] = dinv;
      __syncthreads();
    }
  }
  T* out = inv + ((size_t)2 * s + (upper ? 1 : 0)) * NB * NB;
  for (int idx = tid; idx < NB * NB; idx += NT) out[idx] = S[idx];
}

// One diagonal block of a triangular solve with many right-hand sides:
//   X[k0:k0+ncols, col] = Tinv * (P X)[k0:k0+ncols, col]
// where P is the step's row-interchange list (forward solve; pass top_src = nullptr for
// the backward solve).  Each CTA stages the NB x NB inverse in shared memory with wide
// independent loads, then handles CW right-hand sides: thread (i, cc) forms row i of
// column cc.  With rop != nullptr the result is also written as B-operand planes of the
// tensor-core update (per right-hand side NB consecutive values, zero padded; planes
// rop_plane apart).  Dynamic shared memory: NB*NB + 2*CW*NB elements of T.
template <typename T, int NB, int CW>
__global__ void __launch_bounds__(NB * CW) diag_apply_kernel(const T* __restrict__ Tinv, int ncols, int k0,
                                                             const int* top_src, const int* extra_dst,
                                                             const int* extra_src, const int* n_extra,
                                                             T* X, long ldx, int nrhs, float* rop, long rop_plane) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ts = reinterpret_cast<T*>(smem_raw);  // [NB * NB] column-major
  T* bv = ts + NB * NB;                     // [CW][NB]
  T* ev = bv + CW * NB;                     // [CW][NB]
  constexpr int NT = NB * CW;
  const int tid = threadIdx.x;
  const int i = tid % NB, cc = tid / NB;
  const int col = blockIdx.x * CW + cc;
  const bool active = col < nrhs;
  T* x = X + (size_t)(active ? col : 0) * ldx;
  const int ne = top_src ? *n_extra : 0;
  // stage the inverse: 16-byte loads, all independent
  {
    const float4* src = reinterpret_cast<const float4*>(Tinv);
    float4* dst = reinterpret_cast<float4*>(ts);
    constexpr int n16 = NB * NB * (int)sizeof(T) / 16;
#pragma unroll 8
    for (int q = tid; q < n16; q += NT) dst[q] = __ldg(src + q);
  }
  if (active && i < ncols) bv[cc * NB + i] = x[top_src ? top_src[i] : k0 + i];
  if (active && i < ne) ev[cc * NB + i] = x[extra_src[i]];
  __syncthreads();
  if (active && i < ne) x[extra_dst[i]] = ev[cc * NB + i];
  T acc0 = czero<T>(), acc1 = czero<T>();
  if (active && i < ncols) {
    const T* b = bv + cc * NB;
    int j = 0;
#pragma unroll 4
    for (; j + 1 < ncols; j += 2) {
      cfma(acc0, ts[i + j * NB], b[j]);
      cfma(acc1, ts[i + (j + 1) * NB], b[j + 1]);
    }
    if (j < ncols) cfma(acc0, ts[i + j * NB], b[j]);
    acc0 = cadd(acc0, acc1);
    x[k0 + i] = acc0;
  }
  if (active && rop != nullptr) {
    float hr, lr, hi_, li;
    tf32_split((float)acc0.x, hr, lr);
    tf32_split((float)acc0.y, hi_, li);
    size_t off = (size_t)col * NB + i;
    rop[off] = hr;
    rop[rop_plane + off] = lr;
    rop[2 * rop_plane + off] = hi_;
    rop[3 * rop_plane + off] = li;
  }
}

// -------------------------------------------------------------------------------------
// Tensor-core TRSM of the mixed path (U12 = L11^-1 P A12), in three steps per block step:
//   l11_inverse_planes_kernel: Linv = L11^-1 (unit lower, one CTA, column sweeps as xTRTI2)
//       written as the A-operand planes of (I - Linv), K-major rows;
//   swap_gather_kernel: applies the step's row interchanges to the columns right of the
//       panel, leaving P A12 in rows k0.. of W and as B-operand planes (per column K-major);
//   tc_update: C -= (I - Linv) (P A12) with C = those rows of W, i.e. C = Linv P A12 = U12;
//   u12_split_kernel: U12 -> B-operand planes of the trailing update and the LU planes.
// Inverse of the unit lower triangle L11 in shared memory by recursive blocking: the
// diagonal blocks of (up to) 16 x 16 are inverted by one warp each, all at once (column
// sweeps, as xTRTI2), then pairs of blocks are joined with
//   [A 0; B C]^-1 = [A^-1 0; -C^-1 B A^-1  C^-1]
// until the whole NB x NB block is done.  Dynamic shared memory: (NB*NB + (NB/2)^2) float2.
template <int NB, int NT>
__global__ void __launch_bounds__(NT) l11_inverse_planes_kernel(const float2* __restrict__ W, long ld, int k0,
                                                                 int ncols, float* planes, long plane) {
  constexpr int B0 = NB < 16 ? NB : 16;
  static_assert(NT >= 32 * (NB / B0), "one warp per diagonal block");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* S = reinterpret_cast<float2*>(smem_raw);  // [NB][NB] column-major, L11 -> L11^-1 in place
  float2* T = S + NB * NB;                          // [NB/2][NB/2] scratch
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  for (int idx = tid; idx < NB * NB; idx += NT) {
    int i = idx % NB, j = idx / NB;
    float2 v = make_float2(0.f, 0.f);
    if (i < ncols && j < ncols && i > j) v = W[(size_t)(k0 + i) + (size_t)(k0 + j) * ld];
    if (i == j) v.x = 1.f;
    S[idx] = v;
  }
  __syncthreads();
  // level 0: warp w inverts the diagonal block [B0 w, B0 w + B0)
  if (warp < NB / B0) {
    const int b = B0 * warp;
    const bool in = lane < B0;
    for (int j = B0 - 2; j >= 0; --j) {
      const float2 l = in ? S[(b + lane) + (b + j) * NB] : make_float2(0.f, 0.f);  // lane k: L[k][j]
      float2 acc = make_float2(0.f, 0.f);
      for (int k = j + 1; k < B0; ++k) {
        float2 lk;
        lk.x = __shfl_sync(0xffffffffu, l.x, k);
        lk.y = __shfl_sync(0xffffffffu, l.y, k);
        if (in && k <= lane) cfma(acc, S[(b + lane) + (b + k) * NB], lk);  // Linv[i][k], Linv[i][i] = 1
      }
      __syncwarp();
      if (in && lane > j) S[(b + lane) + (b + j) * NB] = make_float2(-acc.x, -acc.y);
      __syncwarp();
    }
  }
  __syncthreads();
  // join blocks of size h into blocks of size 2h; every thread computes 2 x 4 tiles of the
  // h x h products, so that six shared-memory loads feed eight complex FMAs.  The zeros above
  // the diagonal of S make the triangular ranges rectangular within a tile.
  for (int h = B0; h < NB; h *= 2) {
    const int npair = NB / (2 * h);
    const int th = h / 2, tw = h / 4;  // tiles per pair: th x tw
    // T = B * Ainv for every pair (B: rows [a+h, a+2h), cols [a, a+h); Ainv(k, j) = 0, k < j)
    for (int t = tid; t < npair * th * tw; t += NT) {
      const int pr = t / (th * tw), r = t % (th * tw);
      const int i0 = 2 * (r % th), j0 = 4 * (r / th);
      const int a = pr * 2 * h;
      float2 acc[2][4];
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[u][q] = make_float2(0.f, 0.f);
      for (int k = j0; k < h; ++k) {
        const float2 b0 = S[(a + h + i0) + (a + k) * NB], b1 = S[(a + h + i0 + 1) + (a + k) * NB];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 v = S[(a + k) + (a + j0 + q) * NB];
          cfma(acc[0][q], b0, v);
          cfma(acc[1][q], b1, v);
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) T[pr * h * h + (i0 + u) + (j0 + q) * h] = acc[u][q];
    }
    __syncthreads();
    // B := -Cinv * T  (Cinv: rows/cols [a+h, a+2h), lower: Cinv(i, k) = 0 for k > i)
    for (int t = tid; t < npair * th * tw; t += NT) {
      const int pr = t / (th * tw), r = t % (th * tw);
      const int i0 = 2 * (r % th), j0 = 4 * (r / th);
      const int a = pr * 2 * h;
      float2 acc[2][4];
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[u][q] = make_float2(0.f, 0.f);
      for (int k = 0; k <= i0 + 1; ++k) {
        const float2 c0 = S[(a + h + i0) + (a + h + k) * NB], c1 = S[(a + h + i0 + 1) + (a + h + k) * NB];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 v = T[pr * h * h + k + (j0 + q) * h];
          cfma(acc[0][q], c0, v);
          cfma(acc[1][q], c1, v);
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          S[(a + h + i0 + u) + (a + j0 + q) * NB] = make_float2(-acc[u][q].x, -acc[u][q].y);
    }
    __syncthreads();
  }
  // (I - Linv) as A-operand planes: row i, K index j contiguous
  for (int idx = tid; idx < NB * NB; idx += NT) {
    int j = idx % NB, i = idx / NB;
    float2 v = S[i + j * NB];
    float2 d = make_float2((i == j ? 1.f : 0.f) - v.x, -v.y);
    if (i >= ncols || j >= ncols) d = make_float2(0.f, 0.f);
    float hr, lr, hi_, li;
    tf32_split(d.x, hr, lr);
    tf32_split(d.y, hi_, li);
    planes[idx] = hr;
    planes[plane + idx] = lr;
    planes[2 * plane + idx] = hi_;
    planes[3 * plane + idx] = li;
  }
}

// Row interchanges of one step on columns [c_begin, c_end) of W, leaving P A12 in rows
// k0 .. k0+ncols and as B-operand planes bg[(col - c_begin) * NB + j] (zero padded).
template <int NB, int CW, int NT>
__global__ void __launch_bounds__(NT) swap_gather_kernel(float2* W, long ld, int k0, int ncols,
                                                         const int* __restrict__ top_src,
                                                         const int* __restrict__ extra_dst,
                                                         const int* __restrict__ extra_src,
                                                         const int* __restrict__ n_extra, int c_begin, int c_end,
                                                         float* bg, long plane) {
  constexpr int NBP = NB + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* A = reinterpret_cast<float2*>(smem_raw);  // [CW][NBP]
  float2* E = A + CW * NBP;                         // [CW][NB]
  const int tid = threadIdx.x;
  const int cb = c_begin + blockIdx.x * CW;
  const int ncw = min(CW, c_end - cb);
  if (ncw <= 0) return;
  const int ne = *n_extra;
  for (int idx = tid; idx < ncw * ncols; idx += NT) {
    int j = idx % ncols, cc = idx / ncols;
    A[cc * NBP + j] = W[(size_t)top_src[j] + (size_t)(cb + cc) * ld];
  }
  for (int idx = tid; idx < ncw * ne; idx += NT) {
    int e = idx % ne, cc = idx / ne;
    E[cc * NB + e] = W[(size_t)extra_src[e] + (size_t)(cb + cc) * ld];
  }
  __syncthreads();
  for (int idx = tid; idx < ncw * ne; idx += NT) {
    int e = idx % ne, cc = idx / ne;
    W[(size_t)extra_dst[e] + (size_t)(cb + cc) * ld] = E[cc * NB + e];
  }
  for (int idx = tid; idx < ncw * NB; idx += NT) {
    int j = idx % NB, cc = idx / NB;
    float2 v = j < ncols ? A[cc * NBP + j] : make_float2(0.f, 0.f);
    if (j < ncols) W[(size_t)(k0 + j) + (size_t)(cb + cc) * ld] = v;
    float hr, lr, hi_, li;
    tf32_split(v.x, hr, lr);
    tf32_split(v.y, hi_, li);
    size_t off = (size_t)(cb + cc - c_begin) * NB + j;
    bg[off] = hr;
    bg[plane + off] = lr;
    bg[2 * plane + off] = hi_;
    bg[3 * plane + off] = li;
  }
}

// U12 (rows k0 .. k0+ncols of W, columns [c_begin, c_end)) -> B-operand planes of the
// trailing update (per column K-major) and the row-major LU planes; tracks max |u_ij|.
template <int NB, int CW, int NT>
__global__ void __launch_bounds__(NT) u12_split_kernel(const float2* __restrict__ W, long ld, int k0, int ncols,
                                                       int c_begin, int c_end, float* bop, long bplane, float* lup,
                                                       long lup_ld, long lup_plane, unsigned* growth_bits) {
  const int tid = threadIdx.x;
  const int cb = c_begin + blockIdx.x * CW;
  const int ncw = min(CW, c_end - cb);
  if (ncw <= 0) return;
  float gmax = 0.f;
  // per column K-major operand: consecutive threads -> consecutive rows of one column
  for (int idx = tid; idx < ncw * NB; idx += NT) {
    int j = idx % NB, cc = idx / NB;
    float2 v = j < ncols ? W[(size_t)(k0 + j) + (size_t)(cb + cc) * ld] : make_float2(0.f, 0.f);
    gmax = fmaxf(gmax, fabsf(v.x) + fabsf(v.y));
    float hr, lr, hi_, li;
    tf32_split(v.x, hr, lr);
    tf32_split(v.y, hi_, li);
    size_t off = (size_t)(cb + cc - c_begin) * NB + j;
    bop[off] = hr;
    bop[bplane + off] = lr;
    bop[2 * bplane + off] = hi_;
    bop[3 * bplane + off] = li;
  }
  // row-major LU planes: consecutive threads -> consecutive columns of one row
  for (int idx = tid; idx < ncw * ncols; idx += NT) {
    int cc = idx % ncw, j = idx / ncw;
    float2 v = W[(size_t)(k0 + j) + (size_t)(cb + cc) * ld];
    float hr, lr, hi_, li;
    tf32_split(v.x, hr, lr);
    tf32_split(v.y, hi_, li);
    size_t off = (size_t)(k0 + j) * lup_ld + (size_t)(cb + cc);
    lup[off] = hr;
    lup[lup_plane + off] = lr;
    lup[2 * lup_plane + off] = hi_;
    lup[3 * lup_plane + off] = li;
  }
  if (growth_bits) {
    for (int o = 16; o > 0; o >>= 1) gmax = fmaxf(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
    if ((tid & 31) == 0 && gmax > 0.f) atomicMax(growth_bits, mag_hi((double)gmax));
  }
}

}  // namespace hprmat

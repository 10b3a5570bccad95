// Kernels of the shifted (Hessenberg) energy scan.
//
// Between the energies of one J-pi block the R-matrix C(E) changes only by a multiple of the
// identity and by the closed channels' Bloch terms, which are rank one per channel:
//   C(E) = C0 + delta(E) I + Q D(E) Q^T,   Q = blockdiag(q2) (N x nch),
// delta(E) the common change of the diagonal energy term (-k_c^2 for open, +k_c^2 for closed
// channels: -(E - threshold_c)/hm for every c), D(E) = diag(-xc_c / a) over the closed channels
// (the device Bloch matrix of one interval is q2 q2^T).  C0 is reduced once to upper Hessenberg
// form by Householder similarity transformations, C0 = P H P^H (P unitary); then for every
// energy (H + delta I) Y = P^H Q costs O(N^2 nch) (an LU of a Hessenberg matrix needs only
// row-pair pivoting and N - 1 eliminations) instead of the O(N^3) LU of C(E), and the Bloch
// terms enter through the Woodbury identity on the nch x nch matrix S = Q^T P Y:
//   Q^T C(E)^-1 Q = S (I + D S)^-1,   C(E)^-1 Q = P Y T,   T = I - D (I + S D)^-1 S.
// The reduction is backward stable in norm only (entries of C0 span many orders of magnitude),
// so every energy then takes FP64 refinement steps against the structured C(E) (r = Q - C(E) X,
// correction through the same Hessenberg factors).
//
// Householder convention: for x (m entries) with ||x|| > 0, gamma = -e^{i arg x0} ||x|| and
// u = (x - gamma e1) / ||x - gamma e1||; H = I - 2 u u^H is Hermitian and unitary with
// H x = gamma e1, and A <- H A H is a similarity.  After the steps k = 0 .. N-3,
// C0 = P H_final P^H with P = H_0 H_1 ... H_{N-3}.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace hprmat {

constexpr int kHessThreads = 256;

__device__ __forceinline__ double2 hz_conj(double2 a) { return make_double2(a.x, -a.y); }

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  const double out = red[0];
  __syncthreads();
  return out;
}

// Reflector of column k of A (N x N, column-major, lda): x = A[k+1 .., k], m = N - k - 1 >= 2.
// Writes u into ustore[k+1 .., k] (column k of the reflector store; u = 0 when x = 0) and
// replaces the column by gamma e1.  One CTA.
__global__ void __launch_bounds__(kHessThreads) hess_reflector_kernel(double2* A, long lda, int N, int k,
                                                                      double2* ustore, long ldu) {
  __shared__ double red[32];
  const int m = N - k - 1;
  double2* x = A + (size_t)k * lda + (k + 1);
  double2* u = ustore + (size_t)k * ldu + (k + 1);
  double ss = 0.0;
  for (int i = threadIdx.x; i < m; i += kHessThreads) ss += x[i].x * x[i].x + x[i].y * x[i].y;
  ss = block_sum<kHessThreads>(ss, red);
  const double2 x0 = x[0];
  __syncthreads();  // every thread has read x0 before thread 0 overwrites it
  if (ss == 0.0) {
    for (int i = threadIdx.x; i < m; i += kHessThreads) u[i] = make_double2(0.0, 0.0);
    return;
  }
  const double nrm = sqrt(ss);
  const double a0 = hypot(x0.x, x0.y);
  const double2 ph = a0 > 0.0 ? make_double2(x0.x / a0, x0.y / a0) : make_double2(1.0, 0.0);
  const double2 gamma = make_double2(-ph.x * nrm, -ph.y * nrm);
  // ||x - gamma e1||^2 = 2 ||x||^2 + 2 ||x|| |x0|
  const double winv = 1.0 / sqrt(2.0 * ss + 2.0 * nrm * a0);
  for (int i = threadIdx.x; i < m; i += kHessThreads) {
    double2 w = x[i];
    if (i == 0) {
      w.x -= gamma.x;
      w.y -= gamma.y;
    }
    u[i] = make_double2(w.x * winv, w.y * winv);
    x[i] = i == 0 ? gamma : make_double2(0.0, 0.0);
  }
}

// A[r0 .., c] <- H A[r0 .., c] for the columns c in [c0, N) of A (column-major, lda), H = I - 2 u u^H
// with u the m = N - r0 entries of column k of the reflector store (rows r0 ..): per column
// w = u^H A[r0.., c], A[r0.., c] -= 2 u w.  One warp per column.
__global__ void __launch_bounds__(kHessThreads) hess_left_kernel(double2* A, long lda, int N, int r0, int c0,
                                                                 const double2* ustore, long ldu, int k) {
  const int warp = (blockIdx.x * kHessThreads + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int c = c0 + warp;
  if (c >= N) return;
  const int m = N - r0;
  const double2* u = ustore + (size_t)k * ldu + r0;
  double2* a = A + (size_t)c * lda + r0;
  double wr = 0.0, wi = 0.0;  // sum conj(u_i) a_i
  for (int i = lane; i < m; i += 32) {
    const double2 ui = u[i], ai = a[i];
    wr += ui.x * ai.x + ui.y * ai.y;
    wi += ui.x * ai.y - ui.y * ai.x;
  }
  for (int o = 16; o > 0; o >>= 1) {
    wr += __shfl_xor_sync(0xffffffffu, wr, o);
    wi += __shfl_xor_sync(0xffffffffu, wi, o);
  }
  wr *= 2.0;
  wi *= 2.0;
  for (int i = lane; i < m; i += 32) {
    const double2 ui = u[i];
    double2 ai = a[i];
    ai.x -= ui.x * wr - ui.y * wi;
    ai.y -= ui.x * wi + ui.y * wr;
    a[i] = ai;
  }
}

// Right application A[:, k+1 ..] <- A[:, k+1 ..] H, rows 0 .. N-1: first p = A[:, k+1 ..] u in
// column chunks (part[chunk][row]), then A_ij -= 2 p_i conj(u_j).  Grid (row blocks of 256,
// column chunks of kHessChunk).
constexpr int kHessChunk = 64;
__global__ void __launch_bounds__(kHessThreads) hess_right_partial_kernel(const double2* __restrict__ A, long lda,
                                                                          int N, int k, const double2* ustore,
                                                                          long ldu, double2* part) {
  const int row = blockIdx.x * kHessThreads + threadIdx.x;
  const int j0 = k + 1 + blockIdx.y * kHessChunk;
  const int j1 = min(j0 + kHessChunk, N);
  __shared__ double2 us[kHessChunk];
  for (int j = j0 + threadIdx.x; j < j1; j += kHessThreads) us[j - j0] = ustore[(size_t)k * ldu + j];
  __syncthreads();
  if (row >= N) return;
  // four independent sums, eight loads in flight per thread
  double pr[4] = {0.0, 0.0, 0.0, 0.0}, pi[4] = {0.0, 0.0, 0.0, 0.0};
  int j = j0;
  for (; j + 7 < j1; j += 8) {
    double2 a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = A[(size_t)(j + q) * lda + row];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double2 u = us[j + q - j0];
      pr[q & 3] += a[q].x * u.x - a[q].y * u.y;
      pi[q & 3] += a[q].x * u.y + a[q].y * u.x;
    }
  }
  for (; j < j1; ++j) {
    const double2 a = A[(size_t)j * lda + row], u = us[j - j0];
    pr[0] += a.x * u.x - a.y * u.y;
    pi[0] += a.x * u.y + a.y * u.x;
  }
  part[(size_t)blockIdx.y * N + row] = make_double2(pr[0] + pr[1] + pr[2] + pr[3], pi[0] + pi[1] + pi[2] + pi[3]);
}

__global__ void __launch_bounds__(kHessThreads) hess_right_update_kernel(double2* A, long lda, int N, int k,
                                                                         const double2* ustore, long ldu,
                                                                         const double2* __restrict__ part,
                                                                         int nchunks) {
  const int row = blockIdx.x * kHessThreads + threadIdx.x;
  const int j0 = k + 1 + blockIdx.y * kHessChunk;
  const int j1 = min(j0 + kHessChunk, N);
  __shared__ double2 us[kHessChunk];
  for (int j = j0 + threadIdx.x; j < j1; j += kHessThreads) us[j - j0] = ustore[(size_t)k * ldu + j];
  __syncthreads();
  if (row >= N) return;
  double pr = 0.0, pi = 0.0;
  for (int c = 0; c < nchunks; ++c) {
    const double2 v = part[(size_t)c * N + row];
    pr += v.x;
    pi += v.y;
  }
  pr *= 2.0;
  pi *= 2.0;
  for (int j = j0; j < j1; ++j) {
    const double2 u = us[j - j0];
    double2 a = A[(size_t)j * lda + row];
    // a -= p conj(u)
    a.x -= pr * u.x + pi * u.y;
    a.y -= pi * u.x - pr * u.y;
    A[(size_t)j * lda + row] = a;
  }
}

// dst (row-major, ldd) = the upper Hessenberg part of src (column-major, lds) plus nothing else;
// and PH (column-major, ldp) = P^H.  Grid (N / 32, N / 32), block (32, 8).
__global__ void hess_transpose_kernel(const double2* __restrict__ src, long lds, int N, double2* dst, long ldd,
                                      bool conj_, bool hessenberg_only) {
  __shared__ double2 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += 8) {
    const int r = bx + threadIdx.x, c = by + j;
    if (r < N && c < N) {
      double2 v = src[(size_t)c * lds + r];
      if (hessenberg_only && r > c + 1) v = make_double2(0.0, 0.0);
      tile[j][threadIdx.x] = conj_ ? hz_conj(v) : v;
    }
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += 8) {
    const int r = by + threadIdx.x, c = bx + j;  // dst element (row c of src's transpose)
    if (r < N && c < N) dst[(size_t)c * ldd + r] = tile[threadIdx.x][j];
  }
}

// A (column-major, lda) = identity (N x N).
__global__ void identity_kernel(double2* A, long lda, int N) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r < N) A[(size_t)c * lda + r] = make_double2(r == c ? 1.0 : 0.0, 0.0);
}

// W (column-major, ldw) = P^H Q for Q = blockdiag(q2) (nch blocks of nr rows): W[i, c] =
// sum_r PH[i, c nr + r] q2[r].  Grid (N / 256, nch).
__global__ void hess_wq_kernel(const double2* __restrict__ PH, long ldp, int N, int nr, const double* __restrict__ q2,
                               double2* W, long ldw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= N) return;
  double wr = 0.0, wi = 0.0;
  for (int r = 0; r < nr; ++r) {
    const double2 p = PH[(size_t)(c * nr + r) * ldp + i];
    wr += p.x * q2[r];
    wi += p.y * q2[r];
  }
  W[(size_t)c * ldw + i] = make_double2(wr, wi);
}

// WH (column-major nch x N, ldwh) = W^H = (P^H Q)^H = Q^T P: WH[c, i] = sum_r q2[r] P[c nr + r, i].
// Grid (N / 256, nch).
__global__ void hess_whq_kernel(const double2* __restrict__ P, long ldp, int N, int nr, const double* __restrict__ q2,
                                double2* WH, long ldwh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= N) return;
  double wr = 0.0, wi = 0.0;
  const double2* col = P + (size_t)i * ldp + (size_t)c * nr;
  for (int r = 0; r < nr; ++r) {
    wr += col[r].x * q2[r];
    wi += col[r].y * q2[r];
  }
  WH[(size_t)i * ldwh + c] = make_double2(wr, wi);
}

// ---------------------------------------------------------------- blocked reduction
// Panels of kHbB columns (the method of LAPACK's xGEHRD with xLAHR2, in this file's reflector
// convention, tau = 2): the reflectors u_1 .. u_b of columns k .. k+b-1 are kept in V (the
// reflector store, column c holding u for column c, zero above row c+1), their product is
// H_1 ... H_b = I - V T V^H (T upper triangular, b x b) and Y = A0 V T for the matrix A0 at the
// panel's start.  Column c = k + i of the panel is first brought up to date,
//   x = A0[:, c] - Y[:, <i] V[c, <i]^H,   x[k+1..] -= V[k+1.., <i] T^H V[k+1.., <i]^H x[k+1..],
// its reflector is formed from x[c+1..], then y_i = tau (A0[:, c+1..] u_i - Y[:, <i] (V^H u_i)) and
// T[<i, i] = -tau T (V^H u_i).  After the panel the trailing columns get A -= Y V^H (all rows) and
// A[k+1.., ] -= V T^H (V^H A[k+1.., ]), three GEMMs.
constexpr int kHbB = 32;           // panel width


// The column step runs on one thread-block cluster (G = 8 or 16 CTAs of kHbCT threads, CTA q
// holding rows [q rpc, (q + 1) rpc) of x in shared memory); its three sums over all rows are one
// partial per CTA in shared memory, summed by every CTA through the cluster's distributed shared
// memory after a hardware cluster barrier.  The GEMV that follows each column needs the
// bandwidth of all SMs and is a launch of its own (hb_gemv_kernel).
constexpr int kHbCT = 256;
// The loops over the panel's earlier columns j < n (n runtime, at most kHbB) load in groups of 8
// predicated loads (zero beyond n) issued together, so that their L2 latencies overlap.
constexpr int kHbGrp = 8;

// acc -= sum_{j < n} Y[j * ldy] * s[j]  (column stride ldy; s in shared memory)
__device__ __forceinline__ void hb_sub_cols(double2& acc, const double2* Y, long ldy, const double2* s, int n) {
#pragma unroll
  for (int j0 = 0; j0 < kHbB; j0 += kHbGrp) {
    if (j0 >= n) break;
    double2 y[kHbGrp];
#pragma unroll
    for (int q = 0; q < kHbGrp; ++q) y[q] = j0 + q < n ? Y[(size_t)(j0 + q) * ldy] : make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < kHbGrp; ++q)
      if (j0 + q < n) cfms(acc, y[q], s[j0 + q]);
  }
}


// acc1 -= sum_{j < n} Y[j * ldy] s1[j] and acc2 -= sum_{j < n} Y[j * ldy] s2[j], one load of each Y
__device__ __forceinline__ void hb_sub_cols2(double2& acc1, const double2* s1, double2& acc2, const double2* s2,
                                             const double2* Y, long ldy, int n) {
#pragma unroll
  for (int j0 = 0; j0 < kHbB; j0 += kHbGrp) {
    if (j0 >= n) break;
    double2 y[kHbGrp];
#pragma unroll
    for (int q = 0; q < kHbGrp; ++q) y[q] = j0 + q < n ? Y[(size_t)(j0 + q) * ldy] : make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < kHbGrp; ++q)
      if (j0 + q < n) {
        cfms(acc1, y[q], s1[j0 + q]);
        cfms(acc2, y[q], s2[j0 + q]);
      }
  }
}

namespace cgh = cooperative_groups;

// out[j] = sum over rows r in [rlo, rhi) of conj(V[(k + j), r]) vec[r - r0], j < n (Vk = V + k ldv;
// vec and out in shared memory): warp w takes j = 4w .. 4w + 3 over all the rows (lanes on
// consecutive rows), then sums across its lanes.
static_assert((kHbCT / 32) * 4 >= kHbB, "four columns per warp cover the panel");
__device__ void hb_cta_dots(const double2* Vk, long ldv, const double2* vec, int rlo, int rhi, int r0, int n,
                            double2* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, jb = warp * 4;
  if (jb < n) {
    double2 acc[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[e] = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int r = rlo + lane; r < rhi; r += 32) {
      const double2 xr = vec[r - r0];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double2 v = jb + e < n ? Vk[(size_t)(jb + e) * ldv + r] : make_double2(0.0, 0.0);
        cfma(acc[e], make_double2(v.x, -v.y), xr);
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e)
      for (int o = 16; o > 0; o >>= 1) {
        acc[e].x += __shfl_xor_sync(0xffffffffu, acc[e].x, o);
        acc[e].y += __shfl_xor_sync(0xffffffffu, acc[e].y, o);
      }
    if (lane == 0)
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (jb + e < n) out[jb + e] = acc[e];
  }
  __syncthreads();
}

// tot[j] = sum over the cluster's ranks g < G of rank g's mine[j], j < n (tot shared; red: shared
// [kHbCT / 32][32]).  Thread t reads ranks t / 32, t / 32 + 8, .. of j = t % 32: the remote loads of
// all ranks are in flight together.
__device__ void hb_cluster_sum(const cgh::cluster_group& cl, int G, double2* mine, int n, double2* red, double2* tot) {
  const int j = threadIdx.x & 31, g0 = threadIdx.x >> 5;
  double2 t = make_double2(0.0, 0.0);
  if (j < n)
    for (int g = g0; g < G; g += kHbCT / 32) {
      const double2 m = cl.map_shared_rank(mine, (unsigned)g)[j];
      t.x += m.x;
      t.y += m.y;
    }
  red[g0 * 32 + j] = t;
  __syncthreads();
  if ((int)threadIdx.x < n) {
    double2 s = red[threadIdx.x];
    for (int w = 1; w < kHbCT / 32; ++w) {
      s.x += red[w * 32 + threadIdx.x].x;
      s.y += red[w * 32 + threadIdx.x].y;
    }
    tot[threadIdx.x] = s;
  }
  __syncthreads();
}

struct HbColArgs {
  double2* A;
  long lda;
  int N, k;
  int iy, ix;            // y of panel column iy (if >= 0), then column ix (if >= 0)
  int rpc;               // rows per CTA
  const double2* part;   // GEMV chunk sums of column k + iy: part[ch * N + r]
  int nchunk;
  double2* Y;            // N x kHbB, column-major (ldy)
  long ldy;
  double2* V;            // reflector store (ldv)
  long ldv;
  double2* T;            // kHbB x kHbB of this panel
  double2* s;            // kHbB: V[:, <i]^H u_i of the last column done (rank 0 writes it)
};

// (a) iy >= 0: Y[r, iy] = 2 (p_r - Y[r, <iy] s), p_r the GEMV chunk sums, s of column iy.
// (b) ix >= 0, column c = k + ix: x_r = A[r, c] - Y[r, <ix] conj(V[c, k + <ix]); w = V[k+1.., <ix]^H x;
// z = T^H w; x[k+1..] -= V z; the reflector of x[c+1..] into V[:, c] and A[:, c]; s = V[:, <ix]^H u
// and T[:, ix] (rank 0).  With both, ix = iy + 1, and one pass over Y[r, <iy] serves (a) and (b).
// Dynamic shared memory: rpc complex (x).
__global__ void __launch_bounds__(kHbCT) hb_col_cluster_kernel(HbColArgs a) {
  extern __shared__ __align__(16) double2 xs[];
  __shared__ double2 mine[kHbB];  // this CTA's partial sums, read by the whole cluster
  __shared__ double2 tot[kHbB], zv[kHbB], cv[kHbB], sv[kHbB];
  __shared__ double2 Ts[kHbB * kHbB];  // T of the panel (columns < ix are final)
  __shared__ double2 red[kHbCT];
  __shared__ double mine_ss, rd[kHbCT / 32], sst_s;
  __shared__ double2 mine_x0, x0_s;
  cgh::cluster_group cl = cgh::this_cluster();
  const int G = (int)cl.num_blocks(), q = (int)cl.block_rank();
  const int tid = threadIdx.x, N = a.N, k = a.k;
  const int r0 = q * a.rpc, r1 = min(N, r0 + a.rpc);
  const int i = a.ix, c = k + i;
  if (tid < a.iy) sv[tid] = a.s[tid];
  if (tid < i) {
    const double2 vc = a.V[(size_t)(k + tid) * a.ldv + c];
    cv[tid] = make_double2(vc.x, -vc.y);
  }
  if (i > 0)
    for (int e = tid; e < kHbB * i; e += kHbCT) Ts[e] = a.T[e];
  __syncthreads();
  for (int r = r0 + tid; r < r1; r += kHbCT) {
    double2 xr = i >= 0 ? a.A[(size_t)c * a.lda + r] : make_double2(0.0, 0.0);
    if (a.iy >= 0) {
      double pr[4] = {0.0, 0.0, 0.0, 0.0}, pi[4] = {0.0, 0.0, 0.0, 0.0};
      int ch = 0;
      for (; ch + 3 < a.nchunk; ch += 4) {
        double2 t[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) t[e] = a.part[(size_t)(ch + e) * N + r];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          pr[e] += t[e].x;
          pi[e] += t[e].y;
        }
      }
      for (; ch < a.nchunk; ++ch) {
        const double2 t = a.part[(size_t)ch * N + r];
        pr[0] += t.x;
        pi[0] += t.y;
      }
      double2 p = make_double2(pr[0] + pr[1] + pr[2] + pr[3], pi[0] + pi[1] + pi[2] + pi[3]);
      if (i >= 0)
        hb_sub_cols2(p, sv, xr, cv, a.Y + r, a.ldy, a.iy);
      else
        hb_sub_cols(p, a.Y + r, a.ldy, sv, a.iy);
      const double2 y = make_double2(2.0 * p.x, 2.0 * p.y);
      a.Y[(size_t)a.iy * a.ldy + r] = y;
      if (i >= 0) cfms(xr, y, cv[a.iy]);
    }
    if (i >= 0) xs[r - r0] = xr;
  }
  if (i < 0) return;  // uniform: no CTA of the cluster reads another's shared memory
  __syncthreads();
  if (i > 0) {
    hb_cta_dots(a.V + (size_t)k * a.ldv, a.ldv, xs, max(r0, k + 1), r1, r0, i, mine);
    cl.sync();
    hb_cluster_sum(cl, G, mine, i, red, tot);
    // z_j = sum_{l <= j} conj(T[l, j]) w_l
    if (tid < i) {
      double2 acc = make_double2(0.0, 0.0);
      for (int l = 0; l <= tid; ++l) {
        const double2 t = Ts[tid * kHbB + l];
        cfma(acc, make_double2(t.x, -t.y), tot[l]);
      }
      zv[tid] = acc;
    }
    __syncthreads();
  }
  double ss = 0.0;
  for (int r = r0 + tid; r < r1; r += kHbCT) {
    double2 v = xs[r - r0];
    if (i > 0 && r >= k + 1) {
      hb_sub_cols(v, a.V + (size_t)k * a.ldv + r, a.ldv, zv, i);
      xs[r - r0] = v;
    }
    if (r > c) ss += v.x * v.x + v.y * v.y;
    if (r == c + 1) mine_x0 = v;
  }
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
  if ((tid & 31) == 0) rd[tid >> 5] = ss;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kHbCT / 32; ++w) t += rd[w];
    mine_ss = t;
  }
  cl.sync();  // also: every CTA has read the w partials
  if (tid < 32) {
    double v = tid < G ? *cl.map_shared_rank(&mine_ss, (unsigned)tid) : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) {
      sst_s = v;
      x0_s = *cl.map_shared_rank(&mine_x0, (unsigned)((c + 1) / a.rpc));
    }
  }
  __syncthreads();
  const double sst = sst_s;
  const double2 x0 = x0_s;
  const double a0 = hypot(x0.x, x0.y);
  double2 gamma = x0;
  double winv = 0.0;
  if (sst > 0.0) {
    const double nrm = sqrt(sst);
    const double2 ph = a0 > 0.0 ? make_double2(x0.x / a0, x0.y / a0) : make_double2(1.0, 0.0);
    gamma = make_double2(-ph.x * nrm, -ph.y * nrm);
    winv = 1.0 / sqrt(2.0 * sst + 2.0 * nrm * a0);
  }
  for (int r = r0 + tid; r < r1; r += kHbCT) {
    const double2 xr = xs[r - r0];
    double2 u = make_double2(0.0, 0.0);
    if (r > c && sst > 0.0) {
      u = xr;
      if (r == c + 1) {
        u.x -= gamma.x;
        u.y -= gamma.y;
      }
      u.x *= winv;
      u.y *= winv;
    }
    a.V[(size_t)c * a.ldv + r] = u;
    a.A[(size_t)c * a.lda + r] = r <= c ? xr : (r == c + 1 ? gamma : make_double2(0.0, 0.0));
    xs[r - r0] = u;  // x is done with; u for the sums below
  }
  __syncthreads();
  // the w partials in mine were read by every CTA before the barrier after the norm
  if (i > 0) hb_cta_dots(a.V + (size_t)k * a.ldv, a.ldv, xs, max(r0, c + 1), r1, r0, i, mine);
  cl.sync();
  if (q == 0) {
    hb_cluster_sum(cl, G, mine, i, red, tot);
    if (tid < i) a.s[tid] = tot[tid];
    // T[:, i]: rows < i from -2 T[<i, <i] s, row i = 2 (or 0 for an identity reflector), rest 0
    if (tid < kHbB) {
      double2 t = make_double2(0.0, 0.0);
      if (tid < i) {
        for (int m = tid; m < i; ++m) cfma(t, Ts[m * kHbB + tid], tot[m]);
        t = make_double2(-2.0 * t.x, -2.0 * t.y);
      } else if (tid == i) {
        t = make_double2(sst > 0.0 ? 2.0 : 0.0, 0.0);
      }
      a.T[(size_t)i * kHbB + tid] = t;
    }
  }
  cl.sync();  // no CTA leaves while rank 0 reads its partials
}

// The GEMV of column c: part[ch * N + r] = sum over the 256 columns j of chunk ch (from c + 1) of
// A[r, j] u_j, u = V[:, c].  A CTA takes 32 rows and one chunk; warp w its 32 columns w * 32 ..,
// 16 loads in flight per thread; the 8 warps' sums are added in shared memory.
constexpr int kHbGemvCols = 256;
__global__ void __launch_bounds__(256) hb_gemv_kernel(const double2* __restrict__ A, long lda, int N, int c,
                                                      const double2* __restrict__ u, double2* part) {
  __shared__ double2 us[kHbGemvCols];
  __shared__ double2 red[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * 32 + lane;
  const int j0 = c + 1 + blockIdx.y * kHbGemvCols;
  const int j1 = min(j0 + kHbGemvCols, N);
  us[threadIdx.x] = j0 + (int)threadIdx.x < j1 ? u[j0 + threadIdx.x] : make_double2(0.0, 0.0);
  __syncthreads();
  double pr[4] = {0.0, 0.0, 0.0, 0.0}, pi[4] = {0.0, 0.0, 0.0, 0.0};
  const int jw = j0 + warp * 32;
  if (row < N && jw + 32 <= j1) {
    // all 32 columns in range: 16 unpredicated loads at a time
    const double2* Ar = A + (size_t)jw * lda + row;
#pragma unroll
    for (int b = 0; b < 32; b += 16) {
      double2 av[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) av[e] = __ldg(Ar + (size_t)(b + e) * lda);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const double2 uu = us[warp * 32 + b + e];
        pr[e & 3] += av[e].x * uu.x - av[e].y * uu.y;
        pi[e & 3] += av[e].x * uu.y + av[e].y * uu.x;
      }
    }
  } else if (row < N && jw < j1) {
#pragma unroll
    for (int b = 0; b < 32; b += 16) {
      double2 av[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int j = jw + b + e;
        av[e] = j < j1 ? A[(size_t)j * lda + row] : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const double2 uu = us[warp * 32 + b + e];
        pr[e & 3] += av[e].x * uu.x - av[e].y * uu.y;
        pi[e & 3] += av[e].x * uu.y + av[e].y * uu.x;
      }
    }
  }
  red[warp][lane] = make_double2(pr[0] + pr[1] + pr[2] + pr[3], pi[0] + pi[1] + pi[2] + pi[3]);
  __syncthreads();
  if (warp == 0 && row < N) {
    double2 t = red[0][lane];
    for (int w = 1; w < 8; ++w) {
      t.x += red[w][lane].x;
      t.y += red[w][lane].y;
    }
    part[(size_t)blockIdx.y * N + row] = t;
  }
}

// C (column-major, ldc, M x Nc) += sum of the split-K slices tmp[z] (same layout, slice stride
// ldc * Nc): the partial products of a GEMM cut along K.
__global__ void splitk_sum_kernel(double2* C, long ldc, int M, int Nc, const double2* __restrict__ tmp, int slices) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M * Nc) return;
  const int r = (int)(idx % M), col = (int)(idx / M);
  const size_t off = (size_t)col * ldc + r, stride = (size_t)ldc * Nc;
  double2 v = C[off];
  for (int z = 0; z < slices; ++z) {
    v.x += tmp[off + z * stride].x;
    v.y += tmp[off + z * stride].y;
  }
  C[off] = v;
}

// Per panel (b columns at k): VH = V[:, k..k+b)^H (b x N, column-major, ld kHbB) and
// VT = -V T^H (conj_t) or -V T (N x kHbB, column-major, ld N) for rows r of the grid.
__global__ void hb_prep_kernel(int N, int k, int b, const double2* __restrict__ V, long ldv,
                               const double2* __restrict__ T, double2* VH, double2* VT, bool conj_t) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  double2 v[kHbB];
#pragma unroll
  for (int j = 0; j < kHbB; ++j) v[j] = j < b ? V[(size_t)(k + j) * ldv + r] : make_double2(0.0, 0.0);
#pragma unroll
  for (int j = 0; j < kHbB; ++j) VH[(size_t)r * kHbB + j] = make_double2(v[j].x, -v[j].y);
  // (V T^H)[r, j] = sum_{l >= j} V[r, l] conj(T[j, l]);  (V T)[r, j] = sum_{l <= j} V[r, l] T[l, j].
  // Both loops fully unrolled (v stays in registers); V is zero in the columns l >= b.
#pragma unroll
  for (int j = 0; j < kHbB; ++j) {
    double2 acc = make_double2(0.0, 0.0);
    if (conj_t) {
#pragma unroll
      for (int l = j; l < kHbB; ++l) {
        const double2 t = l < b ? T[(size_t)l * kHbB + j] : make_double2(0.0, 0.0);
        cfma(acc, v[l], make_double2(t.x, -t.y));
      }
    } else {
#pragma unroll
      for (int l = 0; l <= j; ++l) cfma(acc, v[l], T[(size_t)j * kHbB + l]);
    }
    if (j >= b) acc = make_double2(0.0, 0.0);
    VT[(size_t)j * N + r] = make_double2(-acc.x, -acc.y);
  }
}

// ---------------------------------------------------------------- per-energy Hessenberg solves
// One CTA per unit (energy): the LU of Hs = H + delta I (H upper Hessenberg, row-major Hr,
// ldh) with partial pivoting between the two candidate rows of each column (the larger
// |re| + |im|, the working row on ties, as izamax), applied to the nch right-hand sides of
// W (column-major, ldw; shared by all units); then back substitution.  Per unit (stride
// arguments): the upper factor Ue (row-major, ldh), the multipliers lm[k] and row swaps sw[k]
// of step k, and the solution Y (column-major, ldy).  info[u] = first zero pivot (1-based).
struct HessSolveArgs {
  const double2* Hr;
  long ldh;
  int N, nch;
  const double* delta;   // [units]
  const double2* W;      // RHS (forward solve) or nullptr: refine from Y's own content
  long ldw;
  double2* Ue;           // [units] N x ldh row-major
  long sUe;
  double2* lm;           // [units] N
  int* sw;               // [units] N
  double2* Y;            // [units] N x nch column-major, ldy
  long ldy, sY;
  int* info;             // [units]
};

constexpr int kHsRows = 32;   // rows per back-substitution block
constexpr int kHsMaxRhs = 64;

// d += a b for one 8 x 8 x 4 FP64 block on the DMMA units (fragments as mma.m8n8k4 .f64 lays
// them out: a at row lane/4, column lane%4; b at row lane%4, column lane/4; d at row lane/4,
// columns 2 (lane%4) and 2 (lane%4) + 1).
__device__ __forceinline__ void hs_dmma(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}
__device__ __forceinline__ void hs_cp16(void* dst, const void* src, bool valid) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

constexpr int kHsUs = kHsRows + 4;       // row stride of the Ue tile (complex): conflict-free A fragments
constexpr int kHsYs = kHsMaxRhs + 2;     // row stride of the Y chunk: conflict-free B fragments
constexpr int kHsUsTile = kHsRows * kHsUs;
constexpr int kHsYsTile = kHsRows * kHsYs;

// Back substitution Y = Ue^-1 Z in place on the unit's Y (column-major, ldy).  Blocks of 32
// rows from the bottom.  The block's rows minus Ue[rows, below] Y[below] on the FP64 tensor
// units: 8 warps as 4 (8 rows) x 2 (32 right-hand sides), 32-column chunks of Ue and 32-row
// chunks of Y double-buffered in shared memory by cp.async; then the 32 x 32 triangle, one
// right-hand side per thread.
__device__ void hess_back_substitute(const double2* Ue, long ldh, int N, int nch, double2* Y, long ldy,
                                     double2* smem) {
  double2* us = smem;                       // [2][32][kHsUs]
  double2* ys = us + 2 * kHsUsTile;         // [2][32][kHsYs]
  // [32][kHsMaxRhs], used only after a block's chunk loop: over the Y chunk buffers, so that the
  // kernel fits two CTAs per SM
  double2* acc_s = ys;
  static_assert(kHsRows * kHsMaxRhs <= 2 * kHsYsTile, "the block's right-hand sides fit the chunk buffers");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = warp & 3, wc = warp >> 2;
  const int fr = lane >> 2, fk = lane & 3;
  const int nblk = (N + kHsRows - 1) / kHsRows;
  for (int b = nblk - 1; b >= 0; --b) {
    const int k0 = b * kHsRows, k1 = min(k0 + kHsRows, N);
    const int nrow = k1 - k0;
    double accr[4][2], acci[4][2];
#pragma unroll
    for (int q = 0; q < 4; ++q) accr[q][0] = accr[q][1] = acci[q][0] = acci[q][1] = 0.0;
    const int nchk = (N - k1 + kHsRows - 1) / kHsRows;
    auto load = [&](int ci, int buf) {
      const int j0 = k1 + ci * kHsRows;
      double2* u_ = us + buf * kHsUsTile;
      double2* y_ = ys + buf * kHsYsTile;
      for (int idx = tid; idx < kHsRows * kHsRows; idx += kHessThreads) {
        const int r = idx / kHsRows, j = idx % kHsRows;
        const bool ok = r < nrow && j0 + j < N;
        hs_cp16(u_ + r * kHsUs + j, ok ? Ue + (size_t)(k0 + r) * ldh + j0 + j : Ue, ok);
      }
      for (int idx = tid; idx < kHsRows * kHsMaxRhs; idx += kHessThreads) {
        const int j = idx % kHsRows, c = idx / kHsRows;
        const bool ok = c < nch && j0 + j < N;
        hs_cp16(y_ + j * kHsYs + c, ok ? Y + (size_t)c * ldy + j0 + j : Y, ok);
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (nchk > 0) load(0, 0);
    for (int ci = 0; ci < nchk; ++ci) {
      if (ci + 1 < nchk) {
        load(ci + 1, (ci + 1) & 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
      __syncthreads();
      const double2* u_ = us + (ci & 1) * kHsUsTile;
      const double2* y_ = ys + (ci & 1) * kHsYsTile;
#pragma unroll
      for (int kk = 0; kk < kHsRows; kk += 4) {
        const double2 a = u_[(8 * wr + fr) * kHsUs + kk + fk];
        double2 bb[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) bb[q] = y_[(kk + fk) * kHsYs + 32 * wc + 8 * q + fr];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          hs_dmma(accr[q], a.x, bb[q].x);
          hs_dmma(acci[q], a.x, bb[q].y);
        }
        const double nai = -a.y;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          hs_dmma(accr[q], nai, bb[q].y);
          hs_dmma(acci[q], a.y, bb[q].x);
        }
      }
      __syncthreads();  // the buffer is refilled two chunks later
    }
    // the block's right-hand sides minus the products, into shared memory
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = 8 * wr + fr, c = 32 * wc + 8 * q + 2 * fk + e;
        double2 z = (r < nrow && c < nch) ? Y[(size_t)c * ldy + k0 + r] : make_double2(0.0, 0.0);
        z.x -= accr[q][e];
        z.y -= acci[q][e];
        acc_s[r * kHsMaxRhs + c] = z;
      }
    // the diagonal tile
    for (int idx = tid; idx < kHsRows * kHsRows; idx += kHessThreads) {
      const int r = idx / kHsRows, j = idx % kHsRows;
      us[r * kHsUs + j] = (r < nrow && j < nrow) ? Ue[(size_t)(k0 + r) * ldh + k0 + j] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // the triangle, one right-hand side per thread
    if (tid < nch) {
      for (int r = nrow - 1; r >= 0; --r) {
        double2 v = acc_s[r * kHsMaxRhs + tid];
        for (int j = r + 1; j < nrow; ++j) cfms(v, us[r * kHsUs + j], acc_s[j * kHsMaxRhs + tid]);
        const double2 d = us[r * kHsUs + r];
        v = (d.x == 0.0 && d.y == 0.0) ? make_double2(0.0, 0.0) : cdiv(v, d);
        acc_s[r * kHsMaxRhs + tid] = v;
        Y[(size_t)tid * ldy + k0 + r] = v;
      }
    }
    __syncthreads();
  }
}

constexpr size_t kHessSolveSmem = (2 * (size_t)kHsUsTile + 2 * (size_t)kHsYsTile) * sizeof(double2);

// Factor and solve (W given) or re-solve with the stored factors (W == nullptr: the unit's Y
// holds the right-hand sides).  PHASE 1: the elimination (factor, or the forward pass of a
// re-solve) into Ue, lm, sw and Y; dynamic shared memory N complex with W, none without.
// PHASE 2: the back substitution on Y; dynamic shared memory kHessSolveSmem.  The two run as
// separate launches: the latency-bound eliminations of all units then share the SMs (several
// CTAs each), and the DMMA-bound back substitutions follow.
template <int PHASE>
__global__ void __launch_bounds__(kHessThreads) hess_solve_kernel(HessSolveArgs a) {
  extern __shared__ __align__(16) double2 hsm[];
  const int unit = blockIdx.x;
  const int N = a.N, nch = a.nch, tid = threadIdx.x;
  double2* Ue = a.Ue + (size_t)unit * a.sUe;
  double2* lm = a.lm + (size_t)unit * N;
  int* sw = a.sw + (size_t)unit * N;
  double2* Y = a.Y + (size_t)unit * a.sY;
  if (PHASE == 2) {
    hess_back_substitute(Ue, a.ldh, N, nch, Y, a.ldy, hsm);
    return;
  }
  if (a.W != nullptr) {
    // LU of Hs with the working row in shared memory; the right-hand sides follow row by row
    const double dl = a.delta[unit];
    double2* cur = hsm;  // working row, columns k .. N-1
    __shared__ int s_info;
    for (int j = tid; j < N; j += kHessThreads) {
      double2 v = a.Hr[j];
      if (j == 0) v.x += dl;
      cur[j] = v;
    }
    // right-hand-side working row (thread c < nch keeps column c)
    double2 zc = tid < nch ? a.W[(size_t)tid * a.ldw] : make_double2(0.0, 0.0);
    if (tid == 0) s_info = 0;
    __syncthreads();
    constexpr int kEV = 16;  // row values per thread held in registers (N <= kEV kHessThreads)
    if (N <= kEV * kHessThreads) {
      // Row k + 1 of H (columns k + tid + i kHessThreads), its subdiagonal entry and the
      // right-hand sides' entries are loaded one step ahead, all in flight together, so that a
      // step costs one barrier and no dependent load.
      double2 hv[kEV];
      auto load_row = [&](int k) {
        const double2* hn = a.Hr + (size_t)(k + 1) * a.ldh;
#pragma unroll
        for (int i = 0; i < kEV; ++i) {
          const int j = k + tid + i * kHessThreads;
          hv[i] = j < N ? hn[j] : make_double2(0.0, 0.0);
        }
      };
      load_row(0);
      double2 bk = a.Hr[(size_t)a.ldh];
      double2 zb = tid < nch ? a.W[(size_t)tid * a.ldw + 1] : make_double2(0.0, 0.0);
      for (int k = 0; k < N - 1; ++k) {
        const double2 ak = cur[k];
        const bool swap = (fabs(bk.x) + fabs(bk.y)) > (fabs(ak.x) + fabs(ak.y));
        const double2 piv = swap ? bk : ak, oth = swap ? ak : bk;
        const bool zero = piv.x == 0.0 && piv.y == 0.0;
        const double2 l = zero ? make_double2(0.0, 0.0) : cdiv(oth, piv);
        if (zero && tid == 0 && s_info == 0) s_info = k + 1;
#pragma unroll
        for (int i = 0; i < kEV; ++i) {
          const int j = k + tid + i * kHessThreads;
          if (j < N) {
            double2 b = hv[i];
            if (j == k + 1) b.x += dl;
            const double2 c = cur[j];
            const double2 p = swap ? b : c, o = swap ? c : b;
            Ue[(size_t)k * a.ldh + j] = p;
            if (j > k) {
              double2 nv = o;
              cfms(nv, l, p);
              cur[j] = nv;
            }
          }
        }
        if (tid == 0) {
          lm[k] = l;
          sw[k] = swap ? 1 : 0;
        }
        const double2 zk = zb;
        if (k + 2 < N) {
          load_row(k + 1);
          bk = a.Hr[(size_t)(k + 2) * a.ldh + k + 1];
          if (tid < nch) zb = a.W[(size_t)tid * a.ldw + k + 2];
        }
        if (tid < nch) {
          const double2 zp = swap ? zk : zc, zo = swap ? zc : zk;
          Y[(size_t)tid * a.ldy + k] = zp;
          double2 nz = zo;
          cfms(nz, l, zp);
          zc = nz;
        }
        __syncthreads();
      }
    } else {
      for (int k = 0; k < N - 1; ++k) {
        const double2* hn = a.Hr + (size_t)(k + 1) * a.ldh;  // row k + 1 of H (columns k ..)
        double2 bk = hn[k];
        const double2 ak = cur[k];
        const bool swap = (fabs(bk.x) + fabs(bk.y)) > (fabs(ak.x) + fabs(ak.y));
        const double2 piv = swap ? bk : ak, oth = swap ? ak : bk;
        const bool zero = piv.x == 0.0 && piv.y == 0.0;
        const double2 l = zero ? make_double2(0.0, 0.0) : cdiv(oth, piv);
        if (zero && tid == 0 && s_info == 0) s_info = k + 1;
        for (int j = k + tid; j < N; j += kHessThreads) {
          double2 b = hn[j];
          if (j == k + 1) b.x += dl;
          const double2 c = cur[j];
          const double2 p = swap ? b : c, o = swap ? c : b;
          Ue[(size_t)k * a.ldh + j] = p;
          if (j > k) {
            double2 nv = o;
            cfms(nv, l, p);
            cur[j] = nv;
          }
        }
        if (tid == 0) {
          lm[k] = l;
          sw[k] = swap ? 1 : 0;
        }
        if (tid < nch) {
          const double2 zb = a.W[(size_t)tid * a.ldw + k + 1];
          const double2 zp = swap ? zb : zc, zo = swap ? zc : zb;
          Y[(size_t)tid * a.ldy + k] = zp;
          double2 nz = zo;
          cfms(nz, l, zp);
          zc = nz;
        }
        __syncthreads();
      }
    }
    if (tid == 0) {
      const double2 d = cur[N - 1];
      Ue[(size_t)(N - 1) * a.ldh + (N - 1)] = d;
      if (d.x == 0.0 && d.y == 0.0 && s_info == 0) s_info = N;
      a.info[unit] = s_info;
    }
    if (tid < nch) Y[(size_t)tid * a.ldy + N - 1] = zc;
    __syncthreads();
  } else {
    // forward elimination of the unit's right-hand sides with the stored steps
    if (tid < nch) {
      // step k reads y[k + 1] before step k + 1 writes it: the loads of 8 steps go out together
      double2* y = Y + (size_t)tid * a.ldy;
      double2 zc = y[0];
      int k = 0;
      for (; k + 8 <= N - 1; k += 8) {
        double2 zb[8], l[8];
        int s[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          zb[e] = y[k + 1 + e];
          l[e] = lm[k + e];
          s[e] = sw[k + e];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const double2 zp = s[e] ? zb[e] : zc, zo = s[e] ? zc : zb[e];
          y[k + e] = zp;
          double2 nz = zo;
          cfms(nz, l[e], zp);
          zc = nz;
        }
      }
      for (; k < N - 1; ++k) {
        const double2 zb = y[k + 1];
        const bool swap = sw[k] != 0;
        const double2 zp = swap ? zb : zc, zo = swap ? zc : zb;
        y[k] = zp;
        double2 nz = zo;
        cfms(nz, lm[k], zp);
        zc = nz;
      }
      y[N - 1] = zc;
    }
  }
}

// ---------------------------------------------------------------- per-unit Woodbury terms
// One CTA per unit, nch <= 64, matrices column-major nch x nch with stride nch^2 per unit.
// mode 0 (after the first solve; S given as -S by the preceding GEMM):
//   F = (I + S D)^-1 S,  T = I - D F  (-> Tout),  R0 = S T = S - S D F  (-> Rout)
// mode 1 (refinement correction G = W^H y_r): Delta = (I + S D)^-1 G, Rout += Delta, and the
//   relative change ||Delta||_F / ||Rout||_F into chg[unit]; Delta also to Dout (for X updates).
// Gaussian elimination with partial pivoting (|re| + |im|) in shared memory.
__global__ void __launch_bounds__(kHessThreads) hess_woodbury_kernel(int nch, const double2* Sneg, const double* D,
                                                                     int ldD, int mode, const double2* G,
                                                                     double2* Tout, double2* Rout, double2* Dout,
                                                                     double* chg, int* info) {
  extern __shared__ __align__(16) double2 wsm[];
  const int unit = blockIdx.x, tid = threadIdx.x;
  const size_t nn = (size_t)nch * nch;
  const double2* Sg = Sneg + unit * nn;
  const double* d = D + (size_t)unit * ldD;
  double2* M = wsm;           // I + S D (column-major)
  double2* Bm = M + nn;       // right-hand sides (nch columns)
  double2* Sv = Bm + nn;      // S
  __shared__ int piv_row;
  __shared__ double red[32];
  for (int idx = tid; idx < (int)nn; idx += kHessThreads) {
    const int r = idx % nch, c = idx / nch;
    const double2 s = make_double2(-Sg[idx].x, -Sg[idx].y);
    Sv[idx] = s;
    double2 m = make_double2(s.x * d[c], s.y * d[c]);
    if (r == c) m.x += 1.0;
    M[idx] = m;
    Bm[idx] = mode == 0 ? s : G[unit * nn + idx];
  }
  __syncthreads();
  // elimination, column j: pivot search by warp 0, swap, eliminate below
  for (int j = 0; j < nch; ++j) {
    if (tid < 32) {
      double bv = -1.0;
      int bi = j;
      for (int r = j + tid; r < nch; r += 32) {
        const double v = fabs(M[j * nch + r].x) + fabs(M[j * nch + r].y);
        if (v > bv || (v == bv && r < bi)) {
          bv = v;
          bi = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, bv, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) {
          bv = ov;
          bi = oi;
        }
      }
      if (tid == 0) piv_row = bi;
    }
    __syncthreads();
    const int p = piv_row;
    if (p != j)
      for (int c = tid; c < 2 * nch; c += kHessThreads) {
        double2* base = c < nch ? M + (size_t)c * nch : Bm + (size_t)(c - nch) * nch;
        const double2 t = base[j];
        base[j] = base[p];
        base[p] = t;
      }
    __syncthreads();
    const double2 pv = M[j * nch + j];
    if (pv.x == 0.0 && pv.y == 0.0) {
      if (tid == 0) info[unit] = j + 1;
      continue;
    }
    // rows r > j: l_r = M[r, j] / pv; row r -= l_r row j (columns > j of M and all of Bm)
    for (int idx = tid; idx < (nch - j - 1) * (2 * nch - j - 1); idx += kHessThreads) {
      const int r = j + 1 + idx % (nch - j - 1);
      const int cc = j + 1 + idx / (nch - j - 1);  // column index over [M cols j+1.. | Bm cols]
      const double2 l = cdiv(M[j * nch + r], pv);
      double2* col = cc < nch ? M + (size_t)cc * nch : Bm + (size_t)(cc - nch) * nch;
      double2 v = col[r];
      cfms(v, l, col[j]);
      col[r] = v;
    }
    __syncthreads();
  }
  // back substitution, one right-hand side per thread
  if (tid < nch) {
    double2* b = Bm + (size_t)tid * nch;
    for (int r = nch - 1; r >= 0; --r) {
      double2 v = b[r];
      for (int c = r + 1; c < nch; ++c) cfms(v, M[(size_t)c * nch + r], b[c]);
      const double2 dd = M[(size_t)r * nch + r];
      b[r] = (dd.x == 0.0 && dd.y == 0.0) ? make_double2(0.0, 0.0) : cdiv(v, dd);
    }
  }
  __syncthreads();
  double2* R = Rout + unit * nn;
  if (mode == 0) {
    // F = Bm.  T = I - D F (T[r, c] = delta_rc - d_r F[r, c]);  R0 = S T = S - S D F
    double2* T = Tout + unit * nn;
    for (int idx = tid; idx < (int)nn; idx += kHessThreads) {
      const int r = idx % nch, c = idx / nch;
      const double2 f = Bm[idx];
      T[idx] = make_double2((r == c ? 1.0 : 0.0) - d[r] * f.x, -d[r] * f.y);
      double2 v = Sv[idx];
      for (int q = 0; q < nch; ++q) {
        const double2 s = Sv[(size_t)q * nch + r];
        const double2 df = make_double2(d[q] * Bm[(size_t)c * nch + q].x, d[q] * Bm[(size_t)c * nch + q].y);
        cfms(v, s, df);
      }
      R[idx] = v;
    }
  } else {
    double2* Dl = Dout + unit * nn;
    double dn = 0.0, rn = 0.0;
    for (int idx = tid; idx < (int)nn; idx += kHessThreads) {
      const double2 dv = Bm[idx];
      double2 v = R[idx];
      v.x += dv.x;
      v.y += dv.y;
      R[idx] = v;
      Dl[idx] = dv;
      dn += dv.x * dv.x + dv.y * dv.y;
      rn += v.x * v.x + v.y * v.y;
    }
    dn = block_sum<kHessThreads>(dn, red);
    rn = block_sum<kHessThreads>(rn, red);
    if (tid == 0) chg[unit] = rn > 0.0 ? sqrt(dn / rn) : 0.0;
  }
}

constexpr size_t hess_woodbury_smem(int nch) { return (size_t)3 * nch * nch * sizeof(double2); }

// out[unit] (nch x nch, column-major) = -diag(d_unit) Dl[unit]: the right factor of the X update
// X += P (y_r - Y D Delta).  Grid (nch^2 / 256, units).
__global__ void hess_scale_rows_kernel(const double2* __restrict__ Dl, const double* __restrict__ D, int ldD, int nch,
                                       double2* out) {
  const long nn = (long)nch * nch;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int unit = blockIdx.y;
  const double d = D[(size_t)unit * ldD + (i % nch)];
  const double2 v = Dl[(size_t)unit * nn + i];
  out[(size_t)unit * nn + i] = make_double2(-d * v.x, -d * v.y);
}

// C (column-major nch x nch, per unit stride nch^2) = scale * Rsrc, zeroing nothing else: the
// R-matrix of a unit R = (Q^T X) / a from the accumulated Q^T X.
__global__ void scale_copy_kernel(const double2* src, double2* dst, long n, double scale) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = make_double2(src[i].x * scale, src[i].y * scale);
}

}  // namespace hprmat

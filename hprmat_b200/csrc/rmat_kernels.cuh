// Device kernels of the R-matrix path around the LU: assembly of C(E), the FP64
// residual r = B - C X evaluated from C's generators, R-matrix extraction and the
// collision-matrix (U) step, and the per-column FGMRES kernels of the refinement.
#pragma once
#include <type_traits>
#include "common.cuh"

namespace hprmat {

// Per-channel data of one (J, pi, E), device resident.
struct ChannelData {
  const double* fac;     // [nch] l(l+1)
  const double* kk;      // [nch] -k^2 (open) or +k^2 (closed): diagonal energy term
  const double* bloch;   // [nch] xc(c,1) / a for closed channels, 0 for open ones
};

// One interval of the mesh (src/rmatrix_hp.F90:61-159).  The right-hand sides of a solve are
// nq1 columns blockdiag(q1) (inner-boundary values, intervals after the first of a propagated
// problem: nq1 = nch) followed by nch columns blockdiag(q2) (outer-boundary values).
struct MeshDev {
  const double* tc;      // [nr*nr] kinetic + Bloch matrix of the interval / a^2 (column-major)
  const double* blo0;    // [nr*nr] closed-channel Bloch matrix of the interval, times a:
                         //   blo0 / a (first interval), blo2 / is - blo1 / (is - 1) (interval is)
  const double* r;       // [nr] mesh radii of the interval
  const double* q2;      // [nr] outer-boundary values
  const double* q1;      // [nr] inner-boundary values (nullptr when nq1 = 0)
  int nr;
  int nq1;
};

// Non-local potential of an rmatrix call (src/rmatrix_hp.F90:283-288): block (c, c') of C(E)
// gains sqrt(w_i w_j) rmax0 cpnl(i nr + j, c, c'), cpnl complex (ncp2, ndim, ndim).  p = nullptr:
// local potentials only.
struct NonLocalDev {
  const double2* p = nullptr;
  long ncp2 = 0, ndim = 0;
  const double* wle = nullptr;  // Gauss-Legendre weights (nr)
  double rmax0 = 0.0;
};

// Right-hand side value at row (c, i), column col: blockdiag(q1) columns, then blockdiag(q2).
__device__ __forceinline__ double surface_value(const MeshDev& m, int c, int i, int col) {
  if (col < m.nq1) return c == col ? m.q1[i] : 0.0;
  return c == col - m.nq1 ? m.q2[i] : 0.0;
}

// Compensated accumulation (Ogita-Rump-Oishi Dot2): sum += a*b with the rounding errors of
// the product (FMA) and of the sum (TwoSum) kept in a second word.  Gives the residual of
// the outer refinement steps about twice the working precision, so that refinement
// converges to the solution rather than to the rounding noise of u |C| |X|.
struct Acc2 {
  double hi = 0.0, lo = 0.0;
  __device__ __forceinline__ void add_prod(double a, double b) {
    double p = a * b;
    double pe = fma(a, b, -p);
    double s = hi + p;
    double bb = s - hi;
    double e = (hi - (s - bb)) + (p - bb);
    hi = s;
    lo += e + pe;
  }
  __device__ __forceinline__ void add(double p) {
    double s = hi + p;
    double bb = s - hi;
    lo += (hi - (s - bb)) + (p - bb);
    hi = s;
  }
  __device__ __forceinline__ double value() const { return hi + lo; }
};

// Block-wide maximum of a non-negative magnitude into *out as a mag_hi key (orders like the
// values over the whole double range), one atomic per block.  All threads of the block call it.
__device__ __forceinline__ void block_max_atomic(double v, unsigned* out) {
  __shared__ unsigned red_m[32];
  unsigned k = mag_hi(v);
  for (int o = 16; o > 0; o >>= 1) k = max(k, __shfl_down_sync(0xffffffffu, k, o));
  if ((threadIdx.x & 31) == 0) red_m[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x < 32) {
    k = threadIdx.x < (blockDim.x >> 5) ? red_m[threadIdx.x] : 0u;
    for (int o = 16; o > 0; o >>= 1) k = max(k, __shfl_down_sync(0xffffffffu, k, o));
    if (threadIdx.x == 0 && k > 0u) atomicMax(out, k);
  }
}

// C(E) of src/rmatrix_hp.F90:246-293 (one interval):
//   channel block (c,c): tc + diag(l(l+1)/r^2 -+ k^2) - (xc/a) blo0 (closed channels)
//   every block (c,c'):  + diag(cpot(r_i, c, c'))  [+ the non-local term, nl]
// One thread per element, threads along rows (column-major, coalesced stores).  Writes T
// (double2 or float2).
// Also accumulates ||C||_F^2 (FP64) into *fro2 for the refinement's backward error and, with
// amax, the largest |re| + |im| of C for the pivot-growth check.
template <typename T>
__global__ void assemble_kernel(MeshDev mesh, ChannelData ch, int nch, const double2* __restrict__ cpot,
                                long ncp1, long ndim, T* W, long ld, int N, double* fro2, NonLocalDev nl = {},
                                unsigned* amax = nullptr) {
  // thread: one row; block: 256 rows of the columns blockIdx.y, blockIdx.y + gridDim.y, ...
  // (coalesced writes along the column), one atomic per block for ||C||_F^2
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  double am = 0.0;
  if (row < N) {
    const int nr = mesh.nr;
    const int c = row / nr, i = row - c * nr;
    const double rr = mesh.r[i];
    const double dg = ch.fac[c] / (rr * rr) + ch.kk[c];
    const double bl = ch.bloch[c];
    // column col = cp nr + j, stepped by gridDim.y without a division per element
    const int cstep = gridDim.y / nr, jstep = gridDim.y - cstep * nr;
    int cp = blockIdx.y / nr, j = blockIdx.y - cp * nr;
    for (int col = blockIdx.y; col < N; col += gridDim.y) {
      T out;
      if (c == cp || i == j || nl.p) {
        double re = 0.0, im = 0.0;
        if (c == cp) {
          re = mesh.tc[i + (size_t)j * nr] - bl * mesh.blo0[i + (size_t)j * nr];
          if (i == j) re += dg;
        }
        if (i == j) {
          double2 v = cpot[(size_t)i + ncp1 * ((size_t)c + ndim * (size_t)cp)];
          re += v.x;
          im += v.y;
        }
        if (nl.p) {
          const double wf = sqrt(nl.wle[i] * nl.wle[j]) * nl.rmax0;
          const double2 v = nl.p[(size_t)i * nr + j + nl.ncp2 * ((size_t)c + nl.ndim * (size_t)cp)];
          re += wf * v.x;
          im += wf * v.y;
        }
        out.x = (typename RealOf<T>::R)re;
        out.y = (typename RealOf<T>::R)im;
        sq += re * re + im * im;
        am = fmax(am, fabs(re) + fabs(im));
      } else {  // off the channel's block and off the mesh diagonal: C is zero there
        out.x = 0;
        out.y = 0;
      }
      W[(size_t)row + (size_t)col * ld] = out;
      cp += cstep;
      j += jstep;
      if (j >= nr) {
        j -= nr;
        ++cp;
      }
    }
  }
  if (amax) block_max_atomic(am, amax);
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x < 32) {
    sq = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if (threadIdx.x == 0 && sq != 0.0) atomicAdd(fro2, sq);
  }
}

// Channel-surface right-hand sides X = [blockdiag(q1) | blockdiag(q2)] (src/rmatrix_hp.F90:456-461,
// :604-609 for the propagated intervals), scaled.  grid (N / 256, nq1 + nch).
template <typename T>
__global__ void surface_rhs_kernel(MeshDev mesh, T* X, long ldx, int N, double scale) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (row >= N) return;
  const int nr = mesh.nr;
  const int c = row / nr, i = row - c * nr;
  T v = czero<T>();
  v.x = (typename RealOf<T>::R)(surface_value(mesh, c, i, col) * scale);
  X[(size_t)row + (size_t)col * ldx] = v;
}


// ------------------------------------------------------------------ tiled residual products
// The operator products of the refinement (structured C(E), FP64) as batched tiles:
//   kinetic:  batch c,  out[c*nr + i, col]  = b(i, col) - sum_j K_c(i, j) X[c*nr + j, col],
//             K_c = tc - bloch_c blo0 + diag(fac_c / r_i^2 + kk_c)  (real, built per tile);
//   coupling: batch i,  out[c*nr + i, col] -= sum_c' cpot(r_i, c, c') X[c'*nr + i, col]
// (src/rmatrix_hp.F90:246-293 for the matrix they multiply by).  resid_tile_kernel: 256
// threads compute a 64 x 64 tile (4 x 4 complex values each) from 16-deep K chunks staged in
// shared memory; resid_tile2_kernel the compensated and modulus variants of the outer steps.
struct KineticTile {
  MeshDev mesh;
  ChannelData ch;
  const double2* X;
  long ldx;
  int with_b;
  long sx = 0, sch = 0;  // per-unit strides of X and of the channel data (batched launches)
  __device__ KineticTile at(int u) const {
    KineticTile t = *this;
    t.X += (size_t)u * sx;
    t.ch.fac += (size_t)u * sch;
    t.ch.kk += (size_t)u * sch;
    t.ch.bloch += (size_t)u * sch;
    return t;
  }
  __device__ double a(int c, int i, int j) const {
    const int nr = mesh.nr;
    double k = mesh.tc[i + (size_t)j * nr] - ch.bloch[c] * mesh.blo0[i + (size_t)j * nr];
    if (i == j) {
      const double rr = mesh.r[i];
      k += ch.fac[c] / (rr * rr) + ch.kk[c];
    }
    return k;
  }
  __device__ double2 b(int c, int j, int col) const { return X[(size_t)c * mesh.nr + j + (size_t)col * ldx]; }
  __device__ size_t o(int c, int i, int col, long ldo) const { return (size_t)c * mesh.nr + i + (size_t)col * ldo; }
  __device__ double2 init(int c, int i, int col, const double2*, size_t) const {
    return make_double2(with_b ? surface_value(mesh, c, i, col) : 0.0, 0.0);
  }
};

struct CouplingTile {
  const double2* vt;  // cpot_transpose_kernel layout
  const double2* X;
  long ldx;
  int nr, nch;
  long sx = 0;  // per-unit stride of X (batched launches)
  __device__ CouplingTile at(int u) const {
    CouplingTile t = *this;
    t.X += (size_t)u * sx;
    return t;
  }
  __device__ double2 a(int i, int c, int cp) const { return vt[((size_t)i * nch + cp) * nch + c]; }
  __device__ double2 b(int i, int cp, int col) const { return X[(size_t)cp * nr + i + (size_t)col * ldx]; }
  __device__ size_t o(int i, int c, int col, long ldo) const { return (size_t)c * nr + i + (size_t)col * ldo; }
  __device__ double2 init(int, int, int, const double2* out, size_t idx) const { return out[idx]; }
};

template <class Op, bool REAL_A>
__global__ void __launch_bounds__(256, 2) resid_tile_kernel(Op op, int M, int Ncol, int K, double2* out, long ldo) {
  constexpr int BM = 64, BN = 64, BK = 16;
  using AT = typename std::conditional<REAL_A, double, double2>::type;
  __shared__ AT As[BK][BM];
  __shared__ double2 Bs[BK][BN + 1];
  const int z = blockIdx.z;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  double2 acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[r][q] = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < K; k0 += BK) {
    // A tile: consecutive threads along m
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      const int mm = idx % BM, kk = idx / BM;
      const int m = m0 + mm, k = k0 + kk;
      if constexpr (REAL_A) {
        As[kk][mm] = (m < M && k < K) ? op.a(z, m, k) : 0.0;
      } else {
        As[kk][mm] = (m < M && k < K) ? op.a(z, m, k) : make_double2(0.0, 0.0);
      }
    }
    // B tile: consecutive threads along k
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      const int kk = idx % BK, nn = idx / BK;
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < Ncol && k < K) ? op.b(z, k, n) : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      AT av[4];
      double2 bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = As[kk][tx + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = Bs[kk][ty + 16 * q];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if constexpr (REAL_A) {
            acc[r][q].x = fma(av[r], bv[q].x, acc[r][q].x);
            acc[r][q].y = fma(av[r], bv[q].y, acc[r][q].y);
          } else {
            acc[r][q].x = fma(av[r].x, bv[q].x, acc[r][q].x);
            acc[r][q].x = fma(-av[r].y, bv[q].y, acc[r][q].x);
            acc[r][q].y = fma(av[r].x, bv[q].y, acc[r][q].y);
            acc[r][q].y = fma(av[r].y, bv[q].x, acc[r][q].y);
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int m = m0 + tx + 16 * r, n = n0 + ty + 16 * q;
      if (m < M && n < Ncol) {
        const size_t idx = op.o(z, m, n, ldo);
        const double2 b = op.init(z, m, n, out, idx);
        out[idx] = make_double2(b.x - acc[r][q].x, b.y - acc[r][q].y);
      }
    }
}

// The outer-step variants of the same products, 32 x 64 tiles (2 x 4 values per thread):
//   kComp1:  kinetic, out = B - K_c X with compensated (Dot2) sums; the low words go to lo;
//   kComp2:  coupling, out = (out + lo) - V X with compensated sums, rounded once;
//   kAbs1:   kinetic, out = |B| + |K_c| |X| (real part; the rounding scale of the residual);
//   kAbs2:   coupling, out += |V| |X| (real part).
enum ResidTileMode { kComp1 = 0, kComp2 = 1, kAbs1 = 2, kAbs2 = 3 };

// Batched over units (energies): blockIdx.y = column tile + ytiles * unit; unit u works on
// op.at(u) and on out, lo + u * so.
template <class Op, bool REAL_A, int MODE>
__global__ void __launch_bounds__(256) resid_tile2_kernel(Op op_all, int M, int Ncol, int K, double2* out, long ldo,
                                                          double2* lo, int ytiles, long so) {
  constexpr int BM = 32, BN = 64, BK = 16;
  using AT = typename std::conditional<REAL_A, double, double2>::type;
  __shared__ AT As[BK][BM];
  __shared__ double2 Bs[BK][BN + 1];
  const int z = blockIdx.z;
  const int unit = blockIdx.y / ytiles;
  const Op op = op_all.at(unit);
  out += (size_t)unit * so;
  if (lo) lo += (size_t)unit * so;
  const int m0 = blockIdx.x * BM, n0 = (blockIdx.y - unit * ytiles) * BN;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  Acc2 sr[2][4], si[2][4];
  double ar[2][4];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ar[r][q] = 0.0;
      const int m = m0 + tx + 16 * r, n = n0 + ty + 16 * q;
      if (m < M && n < Ncol) {
        const size_t idx = op.o(z, m, n, ldo);
        if constexpr (MODE == kComp1) {
          sr[r][q].add(op.init(z, m, n, out, idx).x);
        } else if constexpr (MODE == kComp2) {
          const double2 o = out[idx], l = lo[idx];
          sr[r][q].hi = o.x;
          sr[r][q].lo = l.x;
          si[r][q].hi = o.y;
          si[r][q].lo = l.y;
        } else if constexpr (MODE == kAbs1) {
          ar[r][q] = fabs(op.init(z, m, n, out, idx).x);
        } else {
          ar[r][q] = out[idx].x;
        }
      }
    }
  for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int idx = tid + 256 * e;
      const int mm = idx % BM, kk = idx / BM;
      const int m = m0 + mm, k = k0 + kk;
      if constexpr (REAL_A) {
        As[kk][mm] = (m < M && k < K) ? op.a(z, m, k) : 0.0;
      } else {
        As[kk][mm] = (m < M && k < K) ? op.a(z, m, k) : make_double2(0.0, 0.0);
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = tid + 256 * e;
      const int kk = idx % BK, nn = idx / BK;
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < Ncol && k < K) ? op.b(z, k, n) : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < BK; ++kk) {
      AT av[2];
      double2 bv[4];
#pragma unroll
      for (int r = 0; r < 2; ++r) av[r] = As[kk][tx + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = Bs[kk][ty + 16 * q];
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if constexpr (MODE == kComp1) {
            sr[r][q].add_prod(-av[r], bv[q].x);
            si[r][q].add_prod(-av[r], bv[q].y);
          } else if constexpr (MODE == kComp2) {
            sr[r][q].add_prod(-av[r].x, bv[q].x);
            sr[r][q].add_prod(av[r].y, bv[q].y);
            si[r][q].add_prod(-av[r].x, bv[q].y);
            si[r][q].add_prod(-av[r].y, bv[q].x);
          } else if constexpr (MODE == kAbs1) {
            ar[r][q] = fma(fabs(av[r]), hypot(bv[q].x, bv[q].y), ar[r][q]);
          } else {
            ar[r][q] = fma(hypot(av[r].x, av[r].y), hypot(bv[q].x, bv[q].y), ar[r][q]);
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int m = m0 + tx + 16 * r, n = n0 + ty + 16 * q;
      if (m < M && n < Ncol) {
        const size_t idx = op.o(z, m, n, ldo);
        if constexpr (MODE == kComp1) {
          out[idx] = make_double2(sr[r][q].hi, si[r][q].hi);
          lo[idx] = make_double2(sr[r][q].lo, si[r][q].lo);
        } else if constexpr (MODE == kComp2) {
          out[idx] = make_double2(sr[r][q].value(), si[r][q].value());
        } else {
          out[idx] = make_double2(ar[r][q], 0.0);
        }
      }
    }
}

// Potential re-laid out per mesh point: vt[(i*nch + c')*nch + c] = cpot(r_i, c, c'), so the
// coupling residual reads it with consecutive channels in consecutive threads.
__global__ void cpot_transpose_kernel(const double2* __restrict__ cpot, long ncp1, long ndim, int nr, int nch,
                                      double2* vt) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)nr * nch * nch;
  if (idx >= total) return;
  const int c = (int)(idx % nch);
  const int cp = (int)((idx / nch) % nch);
  const int i = (int)(idx / ((long)nch * nch));
  vt[idx] = cpot[(size_t)i + ncp1 * ((size_t)c + ndim * (size_t)cp)];
}


// Per-column sums of |x|^2 of an N x ncol block; one CTA per column (deterministic).
__global__ void colnorm2_kernel(const double2* __restrict__ X, long ldx, int N, double* out) {
  const int col = blockIdx.x;
  const double2* x = X + (size_t)col * ldx;
  double s = 0.0;
  for (int r = threadIdx.x; r < N; r += blockDim.x) {
    double2 v = x[r];
    s = fma(v.x, v.x, fma(v.y, v.y, s));
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[col] = s;
  }
}

// Conversions between the FP64 refinement vectors and the LU's element type.
__global__ void d2f_kernel(const double2* __restrict__ src, long lds, float2* dst, long ldd, int N,
                           const double* __restrict__ colscale) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (r >= N) return;
  double s = colscale ? colscale[col] : 1.0;
  double2 v = src[(size_t)r + (size_t)col * lds];
  dst[(size_t)r + (size_t)col * ldd] = make_float2((float)(v.x * s), (float)(v.y * s));
}
__global__ void f2d_kernel(const float2* __restrict__ src, long lds, double2* dst, long ldd, int N,
                           const double* __restrict__ colscale) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (r >= N) return;
  double s = colscale ? colscale[col] : 1.0;
  float2 v = src[(size_t)r + (size_t)col * lds];
  dst[(size_t)r + (size_t)col * ldd] = make_double2((double)v.x * s, (double)v.y * s);
}
__global__ void copy_d_kernel(const double2* __restrict__ src, long lds, double2* dst, long ldd, int N) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (r >= N) return;
  dst[(size_t)r + (size_t)col * ldd] = src[(size_t)r + (size_t)col * lds];
}
// ||A||_F^2 of a dense FP64 complex matrix (column-major), accumulated into *fro2.
// ||A||_F^2 (N x N): block = 256 rows of the columns blockIdx.y + k gridDim.y, one atomic per
// block.
// ||A||_F^2 into *fro2 and, with amax, the largest |re| + |im| of A (pivot-growth check).
__global__ void fro2_kernel(const double2* __restrict__ A, long lda, int N, double* fro2, unsigned* amax = nullptr) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  double am = 0.0;
  if (r < N) {
    for (int col = blockIdx.y; col < N; col += gridDim.y) {
      double2 v = A[(size_t)r + (size_t)col * lda];
      sq += v.x * v.x + v.y * v.y;
      am = fmax(am, fabs(v.x) + fabs(v.y));
    }
  }
  if (amax) block_max_atomic(am, amax);
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x < 32) {
    sq = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if (threadIdx.x == 0 && sq != 0.0) atomicAdd(fro2, sq);
  }
}

// ||A||_1 = max over columns of sum_i |a_ij| (LAPACK's 1-norm, |z| the modulus) into *out as
// the bits of a non-negative double (which order like the values).  One block per column.
__global__ void colabs_max_kernel(const double2* __restrict__ A, long lda, int N, unsigned long long* out) {
  const double2* col = A + (size_t)blockIdx.x * lda;
  double s = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += hypot(col[i].x, col[i].y);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(s));
  }
}

// FP64 -> FP32 copy of a matrix; with amax also the largest |re| + |im| (pivot-growth check).
__global__ void d2f_matrix_kernel(const double2* __restrict__ src, long lds, float2* dst, long ldd, int N,
                                  unsigned* amax = nullptr) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  double am = 0.0;
  if (r < N) {
    double2 v = src[(size_t)r + (size_t)col * lds];
    dst[(size_t)r + (size_t)col * ldd] = make_float2((float)v.x, (float)v.y);
    am = fabs(v.x) + fabs(v.y);
  }
  if (amax) block_max_atomic(am, amax);
}

// ---------------------------------------------------------------- FGMRES (per column)
// Arnoldi step j of right-preconditioned (flexible) GMRES, one CTA per right-hand side:
//   H[0..j, j] = V_i^H w (classical Gram-Schmidt, applied twice), w -= sum_i H[i,j] V_i,
//   H[j+1, j] = |w|, V_{j+1} = w / |w|; then the Givens rotations of the column's
//   least-squares problem are updated.  V: (m+1) blocks of N x ncol, w is V_{j+1}'s slot.
// Per-column state (double): hess[(m+1) x m complex], cs[m] (real), sn[m] (complex),
// g[m+1] (complex).
constexpr int kGmresMaxM = 16;  // longest FGMRES cycle

// Per column |g_{j+1}| / beta: the cycle's residual reduction so far (for the host's
// stopping test).  One thread per column.
__global__ void gmres_estimate_kernel(const double2* __restrict__ g, const double* __restrict__ beta, int m, int j,
                                      int ncol, double* out) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  double2 v = g[(size_t)col * (m + 1) + j + 1];
  double b = beta[col];
  out[col] = b > 0 ? hypot(v.x, v.y) / b : 0.0;
}

struct GmresState {
  double2* V;     // [(m+1)][ldv * ncol]
  long ldv;
  long vstride;   // elements between V blocks
  double2* H;     // [ncol][(m+1)*m]
  double* cs;     // [ncol][m]
  double2* sn;    // [ncol][m]
  double2* g;     // [ncol][m+1]
  double* beta;   // [ncol] initial residual norm of each column
  int m, N, ncol;
};

template <int NT>
__device__ inline double2 block_sum2(double2 v, double2* red) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = (threadIdx.x < NT / 32) ? red[threadIdx.x] : make_double2(0, 0);
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_down_sync(0xffffffffu, v.x, o);
      v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    if (threadIdx.x == 0) red[32] = v;
  }
  __syncthreads();
  return red[32];
}

// V_0 = r / |r|, g = (|r|, 0, ...).  r is V block 0 on entry.
template <int NT>
__global__ void __launch_bounds__(NT) gmres_start_kernel(GmresState s) {
  __shared__ double2 red[33];
  const int col = blockIdx.x;
  double2* v = s.V + (size_t)col * s.ldv;
  double2 acc = make_double2(0, 0);
  for (int r = threadIdx.x; r < s.N; r += NT) {
    double2 x = v[r];
    acc.x = fma(x.x, x.x, fma(x.y, x.y, acc.x));
  }
  double beta = sqrt(block_sum2<NT>(acc, red).x);
  double inv = beta > 0 ? 1.0 / beta : 0.0;
  for (int r = threadIdx.x; r < s.N; r += NT) {
    double2 x = v[r];
    v[r] = make_double2(x.x * inv, x.y * inv);
  }
  for (int i = threadIdx.x; i <= s.m; i += NT) s.g[(size_t)col * (s.m + 1) + i] = make_double2(i == 0 ? beta : 0.0, 0.0);
  if (threadIdx.x == 0) s.beta[col] = beta;
}

// w -= V_{0..J} (V^H w), twice (classical Gram-Schmidt with one reorthogonalisation): all J + 1
// projections in one pass over w and the basis and one block reduction, then one update pass;
// the projections are added into h[0..J].  One CTA per right-hand side; J a compile-time bound
// so that the J + 1 accumulators stay in registers.
template <int NT, int J>
__device__ void cgs2(const GmresState& s, int col, double2* w, double2* h) {
  __shared__ double2 part[J + 1][NT / 32];
  __shared__ double2 hp[J + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double2* V = s.V + (size_t)col * s.ldv;
  for (int pass = 0; pass < 2; ++pass) {
    double2 acc[J + 1];
#pragma unroll
    for (int i = 0; i <= J; ++i) acc[i] = make_double2(0, 0);
    for (int r = threadIdx.x; r < s.N; r += NT) {
      const double2 b = w[r];
#pragma unroll
      for (int i = 0; i <= J; ++i) {
        const double2 a = V[(size_t)i * s.vstride + r];
        acc[i].x = fma(a.x, b.x, fma(a.y, b.y, acc[i].x));  // conj(a) * b
        acc[i].y = fma(a.x, b.y, fma(-a.y, b.x, acc[i].y));
      }
    }
#pragma unroll
    for (int i = 0; i <= J; ++i) {
      double2 v = acc[i];
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
      }
      if (lane == 0) part[i][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x <= J) {
      const int i = threadIdx.x;
      double2 v = make_double2(0, 0);
      for (int q = 0; q < NT / 32; ++q) {
        v.x += part[i][q].x;
        v.y += part[i][q].y;
      }
      hp[i] = v;
      h[i].x += v.x;
      h[i].y += v.y;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < s.N; r += NT) {
      double2 b = w[r];
#pragma unroll
      for (int i = 0; i <= J; ++i) {
        const double2 a = V[(size_t)i * s.vstride + r];
        const double2 hi = hp[i];
        b.x -= hi.x * a.x - hi.y * a.y;
        b.y -= hi.x * a.y + hi.y * a.x;
      }
      w[r] = b;
    }
    __syncthreads();
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) gmres_arnoldi_kernel(GmresState s, int j) {
  __shared__ double2 red[33];
  __shared__ double2 h[kGmresMaxM + 1];
  const int col = blockIdx.x;
  const int m = s.m;
  double2* w = s.V + (size_t)(j + 1) * s.vstride + (size_t)col * s.ldv;
  for (int i = threadIdx.x; i <= j; i += NT) h[i] = make_double2(0, 0);
  __syncthreads();
  switch (j) {  // the loops over the basis at compile-time length
#define HPR_CGS2_CASE(J) \
  case J: cgs2<NT, J>(s, col, w, h); break;
    HPR_CGS2_CASE(0) HPR_CGS2_CASE(1) HPR_CGS2_CASE(2) HPR_CGS2_CASE(3) HPR_CGS2_CASE(4) HPR_CGS2_CASE(5)
    HPR_CGS2_CASE(6) HPR_CGS2_CASE(7) HPR_CGS2_CASE(8) HPR_CGS2_CASE(9) HPR_CGS2_CASE(10) HPR_CGS2_CASE(11)
    HPR_CGS2_CASE(12) HPR_CGS2_CASE(13) HPR_CGS2_CASE(14) HPR_CGS2_CASE(15)
#undef HPR_CGS2_CASE
    default: break;
  }
  double2 acc = make_double2(0, 0);
  for (int r = threadIdx.x; r < s.N; r += NT) {
    double2 b = w[r];
    acc.x = fma(b.x, b.x, fma(b.y, b.y, acc.x));
  }
  double hn = sqrt(block_sum2<NT>(acc, red).x);
  const bool breakdown = !(hn > 1e-300);
  double inv = breakdown ? 0.0 : 1.0 / hn;
  for (int r = threadIdx.x; r < s.N; r += NT) {
    double2 b = w[r];
    w[r] = make_double2(b.x * inv, b.y * inv);
  }
  if (threadIdx.x == 0) {
    double2* H = s.H + (size_t)col * (m + 1) * m;
    double* cs = s.cs + (size_t)col * m;
    double2* sn = s.sn + (size_t)col * m;
    double2* g = s.g + (size_t)col * (m + 1);
    double2 hc[kGmresMaxM + 1];
    for (int i = 0; i <= j; ++i) hc[i] = h[i];
    hc[j + 1] = make_double2(breakdown ? 0.0 : hn, 0.0);
    // apply previous rotations: [c s; -conj(s) c]
    for (int i = 0; i < j; ++i) {
      double c = cs[i];
      double2 sv = sn[i];
      double2 a = hc[i], b = hc[i + 1];
      double2 t0 = make_double2(c * a.x + (sv.x * b.x - sv.y * b.y), c * a.y + (sv.x * b.y + sv.y * b.x));
      double2 t1 = make_double2(-(sv.x * a.x + sv.y * a.y) + c * b.x, -(sv.x * a.y - sv.y * a.x) + c * b.y);
      hc[i] = t0;
      hc[i + 1] = t1;
    }
    // new rotation zeroing hc[j+1]
    double2 a = hc[j], b = hc[j + 1];
    double na = hypot(a.x, a.y), nb = hypot(b.x, b.y);
    double c;
    double2 sv;
    if (nb == 0.0) {
      c = 1.0;
      sv = make_double2(0, 0);
    } else if (na == 0.0) {
      c = 0.0;
      sv = make_double2(b.x / nb, -b.y / nb);  // conj(b)/|b|
    } else {
      double nrm = hypot(na, nb);
      c = na / nrm;
      // s = (a/|a|) * conj(b) / nrm
      double2 ph = make_double2(a.x / na, a.y / na);
      sv = make_double2((ph.x * b.x + ph.y * b.y) / nrm, (ph.y * b.x - ph.x * b.y) / nrm);
    }
    cs[j] = c;
    sn[j] = sv;
    double2 r0 = make_double2(c * a.x + (sv.x * b.x - sv.y * b.y), c * a.y + (sv.x * b.y + sv.y * b.x));
    hc[j] = r0;
    hc[j + 1] = make_double2(0, 0);
    double2 gj = g[j];
    g[j] = make_double2(c * gj.x, c * gj.y);
    g[j + 1] = make_double2(-(sv.x * gj.x + sv.y * gj.y), -(sv.x * gj.y - sv.y * gj.x));
    for (int i = 0; i <= j + 1; ++i) H[(size_t)j * (m + 1) + i] = hc[i];
  }
}

// Solve the rotated (upper triangular) least-squares system for y and apply
// X += sum_i y_i Z_i (flexible GMRES: Z_i = M^-1 V_i).  One CTA per column.
template <int NT>
__global__ void __launch_bounds__(NT) gmres_update_kernel(GmresState s, int jdone, const double2* Z, long zstride,
                                                          long ldz, double2* X, long ldx, double sign) {
  __shared__ double2 y[kGmresMaxM];
  const int col = blockIdx.x;
  const int m = s.m;
  if (threadIdx.x == 0) {
    const double2* H = s.H + (size_t)col * (m + 1) * m;
    const double2* g = s.g + (size_t)col * (m + 1);
    for (int i = jdone - 1; i >= 0; --i) {
      double2 acc = g[i];
      for (int k = i + 1; k < jdone; ++k) {
        double2 hk = H[(size_t)k * (m + 1) + i];
        acc.x -= hk.x * y[k].x - hk.y * y[k].y;
        acc.y -= hk.x * y[k].y + hk.y * y[k].x;
      }
      double2 d = H[(size_t)i * (m + 1) + i];
      double dn = d.x * d.x + d.y * d.y;
      if (dn == 0.0) {
        y[i] = make_double2(0, 0);
      } else {
        y[i] = make_double2((acc.x * d.x + acc.y * d.y) / dn, (acc.y * d.x - acc.x * d.y) / dn);
      }
    }
  }
  __syncthreads();
  double2* x = X + (size_t)col * ldx;
  for (int r = threadIdx.x; r < s.N; r += NT) {
    double2 acc = x[r];
    for (int i = 0; i < jdone; ++i) {
      double2 z = Z[(size_t)i * zstride + (size_t)col * ldz + r];
      acc.x += sign * (y[i].x * z.x - y[i].y * z.y);
      acc.y += sign * (y[i].x * z.y + y[i].y * z.x);
    }
    x[r] = acc;
  }
}

// |a - b|^2 and |a|^2 of two complex vectors (one CTA): out[0], out[1].
__global__ void rel_change_kernel(const double2* __restrict__ a, const double2* __restrict__ b, int n, double* out) {
  double d = 0.0, s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 x = a[i], y = b[i];
    double dx = x.x - y.x, dy = x.y - y.y;
    d = fma(dx, dx, fma(dy, dy, d));
    s = fma(x.x, x.x, fma(x.y, x.y, s));
  }
  __shared__ double rd[32], rs[32];
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_down_sync(0xffffffffu, d, o);
    s += __shfl_down_sync(0xffffffffu, s, o);
  }
  if ((threadIdx.x & 31) == 0) { rd[threadIdx.x >> 5] = d; rs[threadIdx.x >> 5] = s; }
  __syncthreads();
  if (threadIdx.x == 0) {
    d = 0.0;
    s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { d += rd[w]; s += rs[w]; }
    out[0] = d;
    out[1] = s;
  }
}

// ---------------------------------------------------------------- R and U
// R(i, j) = sum_r q(r) X((i-1) nr + r, j) * scale for j < ncols, R with leading dimension nch
// (src/rmatrix_hp.F90:466-474 and :337 with q = q2, scale 1/a; :622-630 for the q1 and q2
// projections of a propagated interval).  grid (nch, ceil(ncols / 128)), 128 threads.
__global__ void rmat_extract_kernel(const double2* __restrict__ X, long ldx, const double* __restrict__ q2,
                                    int nr, int nch, int ncols, double inv_a, double2* R) {
  const int i = blockIdx.x;
  const int jc = threadIdx.x + blockIdx.y * blockDim.x;
  if (jc >= ncols) return;
  const double2* x = X + (size_t)jc * ldx + (size_t)i * nr;
  double ar = 0.0, ai = 0.0;
  for (int r = 0; r < nr; ++r) {
    double2 v = x[r];
    ar = fma(q2[r], v.x, ar);
    ai = fma(q2[r], v.y, ai);
  }
  R[i + (size_t)jc * nch] = make_double2(ar * inv_a, ai * inv_a);
}

// A Z = B in one CTA (A: n x n, ld n; B: n x nrhs, ld ldb; both overwritten, B <- Z) by
// Gaussian elimination with partial pivoting on |re| + |im| (the LAPACK izamax measure; the
// first row on ties).  *info = k + 1 at the first zero pivot k (0-based); the elimination
// continues with a zero reciprocal so that every thread reaches every barrier.
__device__ void cta_gauss_solve(double2* A, int n, double2* B, long ldb, int nrhs, int* info) {
  const int tid = threadIdx.x, NT = blockDim.x;
  __shared__ int s_p;
  __shared__ double s_v[32];
  __shared__ int s_i[32];
  for (int k = 0; k < n; ++k) {
    double bv = -1.0;
    int bi = 0x7fffffff;
    for (int r = k + tid; r < n; r += NT) {
      double v = fabs(A[r + (size_t)k * n].x) + fabs(A[r + (size_t)k * n].y);
      if (v > bv) { bv = v; bi = r; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_down_sync(0xffffffffu, bv, o);
      int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { s_v[tid >> 5] = bv; s_i[tid >> 5] = bi; }
    __syncthreads();
    if (tid < 32) {
      bv = (tid < NT / 32) ? s_v[tid] : -1.0;
      bi = (tid < NT / 32) ? s_i[tid] : 0x7fffffff;
      for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_down_sync(0xffffffffu, bv, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (tid == 0) {
        s_p = bi;
        if (bv == 0.0 && *info == 0) *info = k + 1;
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p != k) {
      for (int c = tid; c < n; c += NT) {
        double2 t = A[k + (size_t)c * n];
        A[k + (size_t)c * n] = A[p + (size_t)c * n];
        A[p + (size_t)c * n] = t;
      }
      for (int c = tid; c < nrhs; c += NT) {
        double2 t = B[k + (size_t)c * ldb];
        B[k + (size_t)c * ldb] = B[p + (size_t)c * ldb];
        B[p + (size_t)c * ldb] = t;
      }
    }
    __syncthreads();
    double2 piv = A[k + (size_t)k * n];
    double2 inv = (piv.x == 0 && piv.y == 0) ? make_double2(0, 0) : crecip(piv);
    for (int r = k + 1 + tid; r < n; r += NT) A[r + (size_t)k * n] = cmul(A[r + (size_t)k * n], inv);
    __syncthreads();
    const int nrow = n - k - 1;
    const int nca = n - k - 1;  // columns k+1.. of A
    const int total = nrow * (nca + nrhs);
    for (int idx = tid; idx < total; idx += NT) {
      int r = k + 1 + idx % nrow;
      int c = idx / nrow;
      double2 l = A[r + (size_t)k * n];
      if (c < nca) {
        int cc = k + 1 + c;
        double2 v = A[r + (size_t)cc * n];
        cfms(v, l, A[k + (size_t)cc * n]);
        A[r + (size_t)cc * n] = v;
      } else {
        int cc = c - nca;
        double2 v = B[r + (size_t)cc * ldb];
        cfms(v, l, B[k + (size_t)cc * ldb]);
        B[r + (size_t)cc * ldb] = v;
      }
    }
    __syncthreads();
  }
  // back substitution, columns of B in parallel
  for (int c = tid; c < nrhs; c += NT) {
    for (int k = n - 1; k >= 0; --k) {
      double2 v = B[k + (size_t)c * ldb];
      for (int q = k + 1; q < n; ++q) cfms(v, A[k + (size_t)q * n], B[q + (size_t)c * ldb]);
      double2 d = A[k + (size_t)k * n];
      v = (d.x == 0 && d.y == 0) ? make_double2(0, 0) : cdiv(v, d);
      B[k + (size_t)c * ldb] = v;
    }
  }
  __syncthreads();
}

// Collision matrix (src/rmatrix_hp.F90:348-368): Z_O U = Z_I with
//   Z_O = diag(co) - Rt diag(cop), Z_I = diag(conj co) - Rt diag(conj cop),
//   Rt(m1,m2) = R(i1,i2) sqrt(k_i1/k_i2) over open channels; solved by Gaussian
// elimination with partial pivoting (|re|+|im|) in one CTA.  cu (ndim x ndim) is zeroed
// and receives U in its leading nopen x nopen block.  Work arrays: zo, zi (nopen^2).
__device__ void umatrix_body(const double2* __restrict__ R, int nch, const int* __restrict__ open_idx,
                             const double* __restrict__ qk, const double2* __restrict__ co,
                             const double2* __restrict__ cop, int no, double2* zo, double2* zi, double2* cu, int ndim,
                             int* info) {
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int idx = tid; idx < ndim * ndim; idx += NT) cu[idx] = make_double2(0, 0);
  for (int idx = tid; idx < no * no; idx += NT) {
    int m1 = idx % no, m2 = idx / no;
    int i1 = open_idx[m1], i2 = open_idx[m2];
    double2 r = R[i1 + (size_t)i2 * nch];
    double s = sqrt(qk[i1] / qk[i2]);
    r.x *= s;
    r.y *= s;
    double2 p = cop[m2];
    // zo = -r * cop ; zi = -r * conj(cop)
    double2 a = make_double2(-(r.x * p.x - r.y * p.y), -(r.x * p.y + r.y * p.x));
    double2 b = make_double2(-(r.x * p.x + r.y * p.y), -(-r.x * p.y + r.y * p.x));
    if (m1 == m2) {
      a.x += co[m1].x;
      a.y += co[m1].y;
      b.x += co[m1].x;
      b.y -= co[m1].y;
    }
    zo[idx] = a;
    zi[idx] = b;
  }
  __syncthreads();
  cta_gauss_solve(zo, no, zi, no, no, info);
  for (int idx = tid; idx < no * no; idx += NT) {
    int m1 = idx % no, m2 = idx / no;
    cu[m1 + (size_t)m2 * ndim] = zi[idx];
  }
}

__global__ void __launch_bounds__(1024) umatrix_kernel(const double2* __restrict__ R, int nch,
                                                       const int* __restrict__ open_idx,
                                                       const double* __restrict__ qk,
                                                       const double2* __restrict__ co,
                                                       const double2* __restrict__ cop, int no,
                                                       double2* zo, double2* zi, double2* cu,
                                                       int ndim, int* info) {
  umatrix_body(R, nch, open_idx, qk, co, cop, no, zo, zi, cu, ndim, info);
}

// The collision-matrix step of many independent units in one launch, one CTA per unit; a unit
// whose skip word is nonzero is left alone.
struct UmatUnit {
  const double2* R;
  const int* open_idx;
  const double* qk;
  const double2* co;
  const double2* cop;
  int no;
  double2* zo;
  double2* zi;
  double2* cu;
  int* info;
  const int* skip;
};
__global__ void __launch_bounds__(1024) umatrix_batch_kernel(const UmatUnit* __restrict__ units, int nch) {
  const UmatUnit u = units[blockIdx.x];
  if (*u.skip != 0) return;
  umatrix_body(u.R, nch, u.open_idx, u.qk, u.co, u.cop, u.no, u.zo, u.zi, u.cu, nch, u.info);
}

// One step of the R-matrix propagation (src/rmatrix_hp.F90:337-345): with R00, R01, R11 the
// q1/q2 projections of interval is (nch x nch, ld nch) and rp the propagated R of the
// intervals before it,
//   rp <- (R11 - R01^T (R00 + rmax1 rp)^-1 R01) / rmax2      (plain transpose)
// The reference inverts R00 + rmax1 rp explicitly; here it is solved for R01.  One CTA;
// work arrays cz, z (nch^2).
__global__ void __launch_bounds__(1024) propagate_kernel(const double2* __restrict__ R00,
                                                         const double2* __restrict__ R01,
                                                         const double2* __restrict__ R11, double2* rp, int nch,
                                                         double rmax1, double rmax2, double2* cz, double2* z,
                                                         int* info) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nn = nch * nch;
  for (int idx = tid; idx < nn; idx += NT) {
    const double2 a = R00[idx], b = rp[idx];
    cz[idx] = make_double2(a.x + rmax1 * b.x, a.y + rmax1 * b.y);
    z[idx] = R01[idx];
  }
  __syncthreads();
  cta_gauss_solve(cz, nch, z, nch, nch, info);
  const double inv = 1.0 / rmax2;
  for (int idx = tid; idx < nn; idx += NT) {
    const int i = idx % nch, j = idx / nch;
    double2 v = R11[idx];
    for (int k = 0; k < nch; ++k) cfms(v, R01[k + (size_t)i * nch], z[k + (size_t)j * nch]);
    rp[idx] = make_double2(v.x * inv, v.y * inv);
  }
}


// Order-independent 64-bit fingerprint of the potential entries a call uses (rows < nrows,
// channels < nch of cpot (ncp1, ndim, ndim)): the sum over entries of a SplitMix64 mix of
// their bits and position.  Identifies the channel block for the reuse of a factorisation.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void fingerprint_kernel(const double2* __restrict__ cpot, long ncp1, long ndim, int nrows, int nch,
                                   unsigned long long* out) {
  const long total = (long)nrows * nch * nch;
  unsigned long long h = 0;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const long i = idx % nrows, cc = idx / nrows;
    const long c = cc % nch, cp = cc / nch;
    const double2 v = cpot[i + ncp1 * (c + ndim * cp)];
    const unsigned long long bx = (unsigned long long)__double_as_longlong(v.x);
    const unsigned long long by = (unsigned long long)__double_as_longlong(v.y);
    h += mix64(bx ^ mix64(by ^ mix64((unsigned long long)idx)));
  }
  for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, h);
}

// ------------------------------------------------------------------ wave functions
// Internal wave functions (rmatrix with twf, src/rmatrix_hp.F90:378-431), built from the
// solutions the R-matrix step already has: per interval X = C^-1 [blockdiag(q1) | blockdiag(q2)].
// cfp holds the channel-surface amplitudes, (ns + 1) columns of nch per entrance channel:
// element (i, is, ic) at i + nch (is + (ns + 1) ic), is = 0..ns (column 0 stays zero).

// cfp(i1, ns) = (conj(cop_m1) [i1 = i2] - U(m1, nvex) cop_m1 sqrt(k_i2 / k_i1)) / rmax over the
// open channels i1 = open_idx[m1], i2 = open_idx[nvex] (:380-386); everything else zero.
// One CTA.  nvc: 0-based open-channel indices of the entrance channels.
__global__ void wf_surface_kernel(const double2* __restrict__ cu, int ndim, const int* __restrict__ open_idx, int no,
                                  const double* __restrict__ qk, const double2* __restrict__ cop,
                                  const int* __restrict__ nvc, int nc, int nch, int ns, double rmax, double2* cfp) {
  const int tot = nch * (ns + 1) * nc;
  for (int i = threadIdx.x; i < tot; i += blockDim.x) cfp[i] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int idx = threadIdx.x; idx < no * nc; idx += blockDim.x) {
    const int m1 = idx % no, ic = idx / no;
    const int nvex = nvc[ic];
    const int i1 = open_idx[m1], i2 = open_idx[nvex];
    const double sc = sqrt(qk[i2] / qk[i1]);
    const double2 p = cop[m1];
    const double2 up = cmul(cu[m1 + (size_t)nvex * ndim], p);
    double2 v = make_double2(-up.x * sc, -up.y * sc);
    if (i1 == i2) {
      v.x += p.x;
      v.y -= p.y;
    }
    cfp[i1 + (size_t)nch * (ns + (size_t)(ns + 1) * ic)] = make_double2(v.x / rmax, v.y / rmax);
  }
}

// cfp(:, is) = Z cfp(:, is + 1), Z = (R00 + rin R)^-1 R01 of interval is + 1 as the propagation
// formed it (:388-394).  grid nc.
__global__ void wf_back_kernel(const double2* __restrict__ Z, int nch, int ns, int is, double2* cfp) {
  const int ic = blockIdx.x;
  const double2* src = cfp + (size_t)nch * (is + 1 + (size_t)(ns + 1) * ic);
  double2* dst = cfp + (size_t)nch * (is + (size_t)(ns + 1) * ic);
  for (int i = threadIdx.x; i < nch; i += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < nch; ++k) cfma(acc, Z[i + (size_t)k * nch], src[k]);
    dst[i] = acc;
  }
}

// Unnormalised wave function of interval is (1-based): cf = X2 cfp(:, is) - X1 cfp(:, is - 1),
// X1 the nq1 leading columns of X (C^-1 blockdiag(q1); none in the first interval), X2 the nch
// after them (C^-1 blockdiag(q2)) -- C^-1 applied to the surface amplitudes as in
// rmat_pierre/rmatrix.f:286-301.  cf complex (nwf1, nwf2, nc), rows (is - 1) nr + ir.
// grid (ceil(nch nr / 256), nc), 256 threads, 2 nch double2 of dynamic shared memory.
__global__ void wf_assemble_kernel(const double2* __restrict__ X, long ldx, int nq1, int nch, int nr, int ns, int is,
                                   const double2* __restrict__ cfp, double2* cf, long nwf1, long nwf2) {
  extern __shared__ double2 sc[];
  const int ic = blockIdx.y;
  const double2* c2 = cfp + (size_t)nch * (is + (size_t)(ns + 1) * ic);
  const double2* c1 = cfp + (size_t)nch * (is - 1 + (size_t)(ns + 1) * ic);
  for (int k = threadIdx.x; k < nch; k += blockDim.x) {
    sc[k] = c2[k];
    sc[nch + k] = c1[k];
  }
  __syncthreads();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nch * nr) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int k = 0; k < nch; ++k) cfma(acc, X[row + (size_t)(nq1 + k) * ldx], sc[k]);
  for (int k = 0; k < nq1; ++k) cfms(acc, X[row + (size_t)k * ldx], sc[nch + k]);
  const int i1 = row / nr, ir = row - i1 * nr;
  cf[(size_t)((is - 1) * nr + ir) + nwf1 * ((size_t)i1 + nwf2 * ic)] = acc;
}

// Closed-channel amplitudes (:414-419): cu(nopen + m, ic) = sum_ir cf((ns-1) nr + ir, i1, ic)
// q2(ir, ns) / W_i1 over the closed channels i1 = closed_idx[m], before the normalisation.
// grid nc.
__global__ void wf_closed_kernel(const double2* __restrict__ cf, long nwf1, long nwf2, int nr, int ns,
                                 const double* __restrict__ q2last, const int* __restrict__ closed_idx, int ncl,
                                 const double* __restrict__ xc2, int no, double2* cu, int ndim) {
  const int ic = blockIdx.x;
  for (int m = threadIdx.x; m < ncl; m += blockDim.x) {
    const int i1 = closed_idx[m];
    const double2* f = cf + (size_t)(ns - 1) * nr + nwf1 * ((size_t)i1 + nwf2 * ic);
    double ar = 0.0, ai = 0.0;
    for (int ir = 0; ir < nr; ++ir) {
      ar = fma(f[ir].x, q2last[ir], ar);
      ai = fma(f[ir].y, q2last[ir], ai);
    }
    const double w = xc2[i1];
    cu[(size_t)(no + m) + (size_t)ic * ndim] = make_double2(ar / w, ai / w);
  }
}

// cf(row, i1, ic) /= sqrt(rmax0 w_ir), row = (is - 1) nr + ir (:421-428).  grid
// (ceil(nr ns / 256), nch, nc).
__global__ void wf_normalize_kernel(double2* cf, long nwf1, long nwf2, int nr, int ns, const double* __restrict__ wle,
                                    double rmax0) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nr * ns) return;
  const double sc = 1.0 / sqrt(rmax0 * wle[row % nr]);
  double2* v = cf + (size_t)row + nwf1 * ((size_t)blockIdx.y + nwf2 * blockIdx.z);
  v->x *= sc;
  v->y *= sc;
}

}  // namespace hprmat

// Host runtime of the B200 R-matrix solver: context, mesh, LU / solve drivers, FP64
// refinement and the C ABI declared in include/hprmat_b200.h.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/hprmat_b200.h"
#include "../../include/hprmat_b200_dev.h"
#include "common.cuh"
#include "coulomb.cuh"
#include "lu.cuh"
#include "adjoint.cuh"
#include "hessenberg.cuh"
#include "rmat_kernels.cuh"
#include "tc_gemm.cuh"
#include "tc_solve.cuh"
#include "zgemm_f64.cuh"

using namespace hprmat;

// NVTX range over one phase of a solve (assembly, factorisation, triangular solves,
// refinement, condition estimate, collision matrix), visible on a profiler's timeline.
// Header-only NVTX v3: with no tool attached a range costs a few nanoseconds.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ------------------------------------------------------------------ error reporting
static thread_local std::string g_last_error;

void hprmat::set_last_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
  g_last_error = buf;
}
void hprmat::set_last_error_msg(const char* msg) { g_last_error = msg; }

static int fail(int status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

#define TRY(expr)                  \
  do {                             \
    int _s = (expr);               \
    if (_s != HPRMAT_B200_OK) return _s; \
  } while (0)

#define LAUNCH_CHECK()        \
  do {                        \
    ++c->launches;            \
    HPR_CUDA_TRY(cudaGetLastError()); \
  } while (0)

// ------------------------------------------------------------------ device buffers
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  int ensure(size_t b) {
    if (b <= bytes && p) return HPRMAT_B200_OK;
    release();
    if (b == 0) b = 16;
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
      p = nullptr;
      bytes = 0;
      cudaGetLastError();
      return fail(HPRMAT_B200_ERR_OOM, "cudaMalloc(%zu bytes) failed: %s", b, cudaGetErrorString(e));
    }
    bytes = b;
    return HPRMAT_B200_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

static constexpr int kSwapStride = 3 * kMaxNB + 4;  // ints per step in the swap store

// Threads per CTA of the FGMRES Arnoldi step (one CTA per right-hand side, 128 CTAs in a
// production solve): the step streams the basis, so more warps per SM keep more loads in
// flight.
constexpr int kArnoldiNT = 512;

// Status-block slots beyond the factorisation's own (SW_*; int offsets into the 64-int block):
// the largest |re| + |im| of the matrix about to be factorised (mag_hi key, written by the
// assembly / conversion kernels for the pivot-growth check) and ||C||_1 (double bits, 8-byte
// aligned, written by colabs_max_kernel when opts.estimate_condition is set).  The
// factorisation copies the first kStatusCopy ints to h_status when it ends.
constexpr int kAmaxSlot = 40;
constexpr int kAnormSlot = 42;
constexpr int kStatusCopy = 44;
constexpr int kSymSlot = 48;  // nonzero when a device potential is not symmetric (adjoint_from_x_device)

// One row of the scan autotuner's table: the settings chosen for the units of order N, and the
// time of the tuned trial (all workers solving one energy of order N at once).
struct ScanTune {
  int N, nb, cluster, rpc_min, sb, gmres_m, tc_grid;
  double ms;
};
constexpr int kTuneInts = 7;  // ints per row of the public table

struct hprmat_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  hprmat_b200_opts opts{};
  int nsm = 0;
  int smem_optin = 0;
  // mesh (rmat_ini)
  int nr = 0, ns = 0;
  double rmax = 0.0;
  // per interval is (nr values or nr x nr matrices each, interval-major): kinetic + Bloch tc,
  // closed-channel Bloch matrix blo0 (MeshDev), outer and inner boundary values q2, q1
  std::vector<double> xle, wle, tc, blo0, q2, q1, zrma;
  DevBuf mesh;  // tc | blo0 | r | q2 | q1, each ns intervals, then the weights wle (nr)
  // work buffers
  DevBuf W, A64, X, X64, R64, B64, V, Z, gm, swaps, ipiv, stage, status, ops, inv, chan, rmat,
      zwork, cpot, cu, norms, lup, rop, rsurf, vt, rlo, linv;
  // wave functions: per-interval solutions and propagation matrices, surface amplitudes, cf
  DevBuf wfx, wfz, wfc, wfcf;
  DevBuf fpbuf;  // potential fingerprint (opts.reuse_factors)
  DevBuf cond_v;  // condition estimate: one right-hand side (opts.estimate_condition)
  // tensor-core operand views of the current factorisation (mixed path)
  TcOperand op_lu, op_bop, op_rhs, op_linv;
  long lup_ld = 0, lup_plane = 0, rop_plane = 0;
  int rop_nrhs = 0, rop_nb = 0;  // key of the solves' right-hand-side planes and their TMA map
  // wavefront solves (mixed path, nb = 128): sigma maps and permutation, transposed
  // off-diagonal blocks, diagonal-inverse planes, right-side / solution planes, flags
  DevBuf wsig, wperm, wT, wdi, wbp, wyp, wxp, wflags, wdf1, wdf2, wptmp, wotmp;
  TcOperand op_wT, op_wdi, op_wbp, op_wyp, op_wxp;
  bool wave_ready = false;
  int wave_un = 0;        // right-hand sides per unit (64, 128; 0: 128 when nrhs > 64)
  int wave_sb = 0;        // blocks per diagonal super block of the scaled factors (1, 2, 4; 0: auto)
  int wave_sb_ready = 1;  // the value the current factors were prepared with
  bool wave_enabled = true;  // wavefront solves (else block-step solves)
  bool tc_trsm = true;       // U12 by the tensor cores from L11^-1 (else substitution)
  int panel_rpc_min = 32;    // fewest panel rows per CTA
  double growth_limit = 1e6;  // mixed path: pivot growth above which C(E) is factorised in FP64
  bool panel_cluster = true;  // panels that fit in one 16-CTA cluster use panel_cluster_kernel
  signed char cluster_ok[2][17] = {};  // per element size (float2, double2) and cluster size:
                                       // 0 unknown, 1 schedulable, -1 not
  int gmres_m = 12;          // longest FGMRES cycle per outer step (<= kGmresMaxM)
  double inner_tol0 = 1e-7;  // first cycle stops once the residual fell this much
  bool zero_start = false;   // refinement starts from X = 0 instead of the FP32 solution
  int w_N = 0, w_npad = 0, w_un = 0;  // key of the wave right-hand-side buffers and their TMA maps
  long w_xld = 0, w_xplane = 0;
  bool wave_trace = false;
  DevBuf wtrace, ptrace;
  // the mixed factorisation held in W / lup / the wave buffers, for opts.reuse_factors: its
  // LUState (N, ld, nb, nsteps) and the channel block it belongs to
  bool lu_held = false;
  int held_last_inner = 0;     // FGMRES iterations of the last solve on the held factors
  int reuse_max_inner = 24;    // factorise again once a reuse solve needed more than this
  long long factorizations = 0;  // LU factorisations run on this context
  int held_N = 0, held_nb = 0, held_nsteps = 0, held_nch = 0, held_nr = 0;
  long held_ld = 0;
  double held_rmax = 0.0;
  unsigned long long held_fp = 0;
  std::vector<int> held_lval;
  // last FP64 factorisation of rmatrix (for the adjoint): N, ld, nb, nsteps; adjoint scratch
  int f64_N = 0, f64_nb = 0, f64_nsteps = 0;
  long f64_ld = 0;
  DevBuf adj_y, adj_part, adj_grad;
  // shifted (Hessenberg) scan: per block C0 -> H (hA), P, P^H, reflectors, row-major H, partial
  // sums, W = P^H Q, W^H; per batch of energies the factors and work arrays of every unit
  DevBuf hA, hP, hPH, hU, hHr, hPart, hW, hWH, hChan, hUe, hLm, hSw, hY, hX, hR, hYr, hYT, hS, hT, hRacc, hG,
      hDl, hUnit, hCu, hZo;
  double hess_budget_gb = 48.0;  // device memory for one batch of energies
  int hess_steps_last = 0;       // refinement steps of the last batch
  int hess_fallback_last = 0;    // energies the last shifted scan sent to the LU path
  double hess_ms[6] = {};        // with profiling: reduce, solve, products, refine, U, fallback (ms)
  bool hess_blocked = true;      // blocked (panel + GEMM) Hessenberg reduction
  int hess_workers = 3;          // shifted scan: blocks in flight at once (worker contexts)
  DevBuf hbY, hbT, hbS, hbVH, hbVT, hbW, hbTmp, hUmat;
  bool f64_pair = true;  // plain FP64 LU: two block steps share one K = 128 trailing update
  DevBuf f64_pair_buf;
  int hb_cluster = 0;  // CTAs of the Hessenberg column step's cluster (0: not chosen yet)
  // batched energy scans: worker contexts (own stream and buffers) and the blocks' potentials
  std::vector<hprmat_b200_ctx*> scan_workers;
  std::vector<std::unique_ptr<DevBuf>> scan_cpot;
  std::vector<ScanTune> scan_tune;  // autotuner table, applied per unit by rmatrix_scan
  int wtrace_units = 0;
  int* h_status = nullptr;  // pinned
  double* h_norms = nullptr;  // pinned
  TcGemmPlan tcplan;
  // counters for benchmarks: kernel launches issued, and (when profiling) CUDA-event
  // time and algorithmic flops of the tensor-core trailing updates
  unsigned long long launches = 0;
  bool profile = false;
  std::vector<cudaEvent_t> ev;
  int ev_used = 0;
  std::vector<double> ev_flops;
  double tc_ms = 0.0, tc_flops = 0.0;
  int tc_launches = 0;
};

// ------------------------------------------------------------------ mesh (rmat_ini)
// Gauss-Legendre nodes and weights on (0,1): LEGZO, src/rmatrix_hp.F90:741-783.
static void legzo(int n, std::vector<double>& x, std::vector<double>& w) {
  const double pi = 3.1415926535898, one = 1.0;
  std::vector<double> X(n + 1, 0.0), Wt(n + 1, 0.0);
  int n0 = (n + 1) / 2;
  for (int nr = 1; nr <= n0; ++nr) {
    double z = cos(pi * (nr - 0.25) / (n + 0.5));
    double pd = 0.0, pf = 0.0;
    for (;;) {
      double z0 = z, p = 1.0;
      for (int i = 1; i <= nr - 1; ++i) p = p * (z - X[i]);
      double f0 = 1.0;
      if (nr == n0 && n != 2 * (n / 2)) z = 0.0;
      double f1 = z;
      for (int k = 2; k <= n; ++k) {
        pf = (2 - one / k) * z * f1 - (1 - one / k) * f0;
        pd = k * (f1 - z * pf) / (1 - z * z);
        f0 = f1;
        f1 = pf;
      }
      if (z == 0.0) break;
      double fd = pf / p, q = 0.0;
      for (int i = 1; i <= nr - 1; ++i) {
        double wp = 1.0;
        for (int j = 1; j <= nr - 1; ++j)
          if (j != i) wp = wp * (z - X[j]);
        q = q + wp;
      }
      double gd = (pd - q * fd) / p;
      z = z - fd / gd;
      if (!(fabs(z - z0) > fabs(z) * 1.0e-15)) break;
    }
    X[nr] = z;
    X[n + 1 - nr] = -z;
    Wt[nr] = 2 / ((1 - z * z) * pd * pd);
    Wt[n + 1 - nr] = Wt[nr];
  }
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    x[i] = (1 + X[n - i]) / 2;
    w[i] = Wt[n - i] / 2;
  }
}

// Kinetic + Bloch matrices, Bloch matrices and boundary values of every interval:
// src/rmatrix_hp.F90:85-151, scaled as at :146-151.  The closed-channel Bloch term of interval
// is (:268-276) is stored as one matrix times rmax0 so that the per-channel factor xc / rmax0
// is the same in every interval: blo0 (is = 1), blo2 / is - blo1 / (is - 1) (is > 1).
static void build_mesh_host(int nr, int ns, double rmax, std::vector<double>& xle, std::vector<double>& wle,
                            std::vector<double>& tc, std::vector<double>& blo, std::vector<double>& q2,
                            std::vector<double>& q1, std::vector<double>& zrma) {
  legzo(nr, xle, wle);
  const double rmax0 = rmax / ns;
  const size_t nn = (size_t)nr * nr;
  tc.assign(nn * ns, 0.0);
  blo.assign(nn * ns, 0.0);
  q2.assign((size_t)nr * ns, 0.0);
  q1.assign((size_t)nr * ns, 0.0);
  const double nn1 = (double)nr * (nr + 1);
  for (int is = 1; is <= ns; ++is) {
    double* t = tc.data() + (is - 1) * nn;
    double* b = blo.data() + (is - 1) * nn;
    for (int i1 = 1; i1 <= nr; ++i1) {
      const double xi = xle[i1 - 1], xi2 = xi * (1 - xi);
      double td, bd;
      if (is == 1) {
        td = (4 * nn1 + 3 + (1 - 6 * xi) / xi2) / (3 * xi2);
        bd = 1 / xi2;
      } else {
        const double xlb = xi / (1 - xi) * (nn1 - 1 / (1 - xi));
        const double xla = (1 - xi) / xi * (-nn1 + 1 / xi);
        td = (nn1 + 6 - 2 / xi2) / (3 * xi2) + xlb - xla;
        bd = xi / (1 - xi) / is - (1 - xi) / xi / (is - 1);
      }
      t[(i1 - 1) + (size_t)(i1 - 1) * nr] = td;
      b[(i1 - 1) + (size_t)(i1 - 1) * nr] = bd;
      for (int i2 = 1; i2 <= i1 - 1; ++i2) {
        const double xj = xle[i2 - 1], xj2 = xj * (1 - xj);
        double to, bo;
        if (is == 1) {
          const double d = xi - xj;
          to = (nn1 + 1 + (xi + xj - 2 * xi * xj) / (d * d) - 1 / (1 - xi) - 1 / (1 - xj)) / sqrt(xi2 * xj2);
          bo = 1 / sqrt(xi2 * xj2);
        } else {
          const double d = xj - xi;
          const double yy = sqrt(xj2 / (xi2 * xi2 * xi2)) * (2 * xi * xj + 3 * xi - xj - 4 * xi * xi) / (d * d);
          const double b2 = sqrt(xi * xj / (1 - xi) / (1 - xj));
          const double b1 = sqrt((1 - xi) * (1 - xj) / xi / xj);
          to = yy + b2 * (nn1 - 1 / (1 - xj)) - b1 * (-nn1 + 1 / xj);
          bo = b2 / is - b1 / (is - 1);
        }
        if ((i1 + i2) % 2 == 1) {
          to = -to;
          // the reference negates blo0 in the loop over every interval (:119-124), so the
          // first interval's matrix ends up negated ns times
          if (is > 1 || ns % 2 == 1) bo = -bo;
        }
        t[(i1 - 1) + (size_t)(i2 - 1) * nr] = to;
        t[(i2 - 1) + (size_t)(i1 - 1) * nr] = to;
        b[(i1 - 1) + (size_t)(i2 - 1) * nr] = bo;
        b[(i2 - 1) + (size_t)(i1 - 1) * nr] = bo;
      }
    }
    for (int i = 0; i < nr; ++i) {
      const double x = xle[i];
      double v2, v1;
      if (is == 1) {
        v2 = 1 / sqrt(x * (1 - x));
        v1 = 0.0;
      } else {
        v2 = sqrt(x / (1 - x));
        v1 = -1 / v2;
      }
      if (nr % 2 == 1) v2 = -v2;
      if (i % 2 == 0) {  // q(1:nr:2) = -q(1:nr:2)
        v2 = -v2;
        v1 = -v1;
      }
      q2[(size_t)(is - 1) * nr + i] = v2 / sqrt(rmax0);
      q1[(size_t)(is - 1) * nr + i] = v1 / sqrt(rmax0);
    }
  }
  for (auto& v : tc) v = v / (rmax0 * rmax0);
  for (auto& v : blo) v = v / rmax0;
  zrma.resize((size_t)nr * ns);
  for (int is = 0; is < ns; ++is)
    for (int i = 0; i < nr; ++i) zrma[(size_t)is * nr + i] = (is + xle[i]) * rmax0;
}

static void build_mesh(hprmat_b200_ctx* c, int nr, int ns, double rmax) {
  c->nr = nr;
  c->ns = ns;
  c->rmax = rmax;
  build_mesh_host(nr, ns, rmax, c->xle, c->wle, c->tc, c->blo0, c->q2, c->q1, c->zrma);
}

static int upload_mesh(hprmat_b200_ctx* c) {
  const size_t nn = (size_t)c->nr * c->nr, nv = (size_t)c->nr * c->ns;
  const size_t n = 2 * nn * c->ns + 3 * nv + c->nr;
  TRY(c->mesh.ensure(n * sizeof(double)));
  std::vector<double> h(n);
  double* p = h.data();
  p = std::copy(c->tc.begin(), c->tc.end(), p);
  p = std::copy(c->blo0.begin(), c->blo0.end(), p);
  p = std::copy(c->zrma.begin(), c->zrma.end(), p);
  p = std::copy(c->q2.begin(), c->q2.end(), p);
  p = std::copy(c->q1.begin(), c->q1.end(), p);
  std::copy(c->wle.begin(), c->wle.end(), p);
  HPR_CUDA_TRY(cudaMemcpyAsync(c->mesh.p, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return HPRMAT_B200_OK;
}

// Gauss-Legendre weights of the mesh on the device.
static const double* mesh_wle(const hprmat_b200_ctx* c) {
  return c->mesh.as<double>() + 2 * (size_t)c->ns * c->nr * c->nr + 3 * (size_t)c->nr * c->ns;
}

// Device view of interval is (0-based); nq1 leading right-hand sides blockdiag(q1).
static MeshDev mesh_dev(const hprmat_b200_ctx* c, int is = 0, int nq1 = 0) {
  const double* base = c->mesh.as<double>();
  const size_t nn = (size_t)c->nr * c->nr, nv = (size_t)c->nr * c->ns;
  MeshDev m;
  m.nr = c->nr;
  m.nq1 = nq1;
  m.tc = base + is * nn;
  m.blo0 = base + c->ns * nn + is * nn;
  m.r = base + 2 * c->ns * nn + (size_t)is * c->nr;
  m.q2 = base + 2 * c->ns * nn + nv + (size_t)is * c->nr;
  m.q1 = nq1 > 0 ? base + 2 * c->ns * nn + 2 * nv + (size_t)is * c->nr : nullptr;
  return m;
}

// ------------------------------------------------------------------ launch helpers
template <typename K>
static int set_smem(K kernel, size_t bytes) {
  // The 48 KB default covers static + dynamic shared memory.  Only ever raise the limit:
  // kernels instantiated in more than one file share it.  Contexts used from several host
  // threads (scan workers) read and raise it under one lock, so that no thread lowers the
  // limit another one has just raised.
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  cudaFuncAttributes fa;
  HPR_CUDA_TRY(cudaFuncGetAttributes(&fa, kernel));
  if ((int)bytes > fa.maxDynamicSharedSizeBytes || (int)(bytes + fa.sharedSizeBytes) > 48 * 1024)
    HPR_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      std::max((int)bytes, fa.maxDynamicSharedSizeBytes)));
  return HPRMAT_B200_OK;
}

static inline unsigned cdiv_u(long a, long b) { return (unsigned)((a + b - 1) / b); }

// ------------------------------------------------------------------ LU driver
struct LUState {
  int N = 0;
  long ld = 0;
  int nb = 0;
  int nsteps = 0;
};

static int pick_nb(const hprmat_b200_ctx* c, int N, size_t elem, int preferred) {
  if (c->opts.panel_nb > 0) preferred = c->opts.panel_nb;
  for (int nb = preferred; nb >= 16; nb /= 2) {
    int G = std::min(c->nsm, std::max(1, (N + 31) / 32));
    int rpc = (N + G - 1) / G;
    size_t smem = ((size_t)nb * (rpc | 1) + nb) * elem;
    if (smem + 8192 <= (size_t)c->smem_optin) return nb;
  }
  return 0;
}

// ------------------------------------------------------------------ wavefront solves
// One-time preparation after a mixed nb = 128 factorisation (tc_solve.cuh): L rows in their
// final order, off-diagonal blocks scaled by the inverse diagonal blocks of their block row,
// diagonal inverses as planes.  Overwrites the off-diagonal part of the LU planes.
static int wave_prepare(hprmat_b200_ctx* c, const LUState& st) {
  const int N = st.N, ns = st.nsteps;
  c->wave_ready = false;
  // super blocks of 4 blocks (2 for nsteps < 4): a quarter of the dependency links, at the
  // price of 4x larger diagonal inverses in the one-time preparation
  const int sb = c->wave_sb > 0 ? c->wave_sb : (ns >= 4 ? 4 : 2);
  const long sig_ld = (N + 3) / 4 * 4;
  TRY(c->wsig.ensure((size_t)ns * sig_ld * sizeof(int)));
  TRY(c->wperm.ensure((size_t)3 * N * sizeof(int) + 64));
  int* work = c->wperm.as<int>();
  int* perm0 = work + 2 * (size_t)N;
  const long ldt = (N + 3) / 4 * 4;
  const long tplane = ldt * (long)N;
  TRY(c->wT.ensure((size_t)4 * tplane * sizeof(float)));
  if (wave_perm_chain(c->swaps.as<int>(), kSwapStride, N, ns, work, c->wsig.as<int>(), sig_ld, perm0, c->stream) ||
      wave_transpose_offdiag(c->lup.as<float>(), c->lup_ld, c->lup_plane, c->wsig.as<int>(), sig_ld, N, ns,
                             c->wT.as<float>(), ldt, tplane, c->stream))
    return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
  // inverses of the diagonal super blocks: doubling from the 128-row blocks
  const float2* cur = c->inv.as<float2>();
  int nblk = ns;
  for (int h = 128, lvl = 0; h < 128 * sb; h *= 2, ++lvl) {
    const int nsup = (nblk + 1) / 2;
    TRY(c->wptmp.ensure((size_t)2 * nsup * h * h * sizeof(float2)));
    TRY(c->wotmp.ensure((size_t)2 * nsup * h * h * sizeof(float2)));
    DevBuf& dst = (lvl & 1) ? c->wdf2 : c->wdf1;
    TRY(dst.ensure((size_t)2 * nsup * 4 * h * h * sizeof(float2)));
    if (wave_dinv_double(cur, h, nblk, c->wT.as<float>(), ldt, tplane, N, c->wptmp.as<float2>(),
                         c->wotmp.as<float2>(), dst.as<float2>(), c->stream))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    cur = dst.as<float2>();
    nblk = nsup;
    c->launches += 3;
  }
  const int hs = 128 * sb;
  const long di_plane = (long)2 * nblk * hs * hs;
  TRY(c->wdi.ensure((size_t)4 * di_plane * sizeof(float)));
  if (wave_dinv_planes(cur, nblk, hs, c->wdi.as<float>(), di_plane, c->stream) ||
      tc_make_operand(c->tcplan, c->op_wdi, c->wdi.as<float>(), hs, (long)2 * nblk * hs, hs, di_plane, 128) ||
      tc_make_operand(c->tcplan, c->op_wT, c->wT.as<float>(), N, N, ldt, tplane, 128) ||
      wave_scale_offdiag(c->tcplan, c->op_wdi, c->op_wT, N, ns, sb, c->lup.as<float>(), c->lup_ld, c->lup_plane,
                         c->stream))
    return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
  c->launches += 5;
  c->wave_sb_ready = sb;
  c->wave_ready = true;
  return HPRMAT_B200_OK;
}

// X (N x nrhs, FP32 complex, ldx) <- (LU)^-1 P X with the prepared factors: right-hand side
// planes of P X, forward sweep into the Y planes, backward sweep into X.
static int lu_solve_wave(hprmat_b200_ctx* c, const LUState& st, float2* X, long ldx, int nrhs) {
  const int N = st.N, ns = st.nsteps;
  const int un = c->wave_un > 0 ? c->wave_un : (nrhs > 64 ? 128 : 64);
  const int G = (nrhs + un - 1) / un;
  const int npad = G * un;
  const long xld = (N + 3) / 4 * 4;
  const long xplane = xld * (long)npad;
  // the TMA maps' box is un rows: a new unit width needs new maps even when npad is unchanged
  if (c->w_N != N || c->w_npad != npad || c->w_xld != xld || c->w_un != un || !c->wbp.p) {
    c->w_N = 0;
    const size_t bytes = (size_t)4 * xplane * sizeof(float);
    TRY(c->wbp.ensure(bytes));
    TRY(c->wyp.ensure(bytes));
    TRY(c->wxp.ensure(bytes));
    HPR_CUDA_TRY(cudaMemsetAsync(c->wbp.p, 0, bytes, c->stream));
    HPR_CUDA_TRY(cudaMemsetAsync(c->wyp.p, 0, bytes, c->stream));
    HPR_CUDA_TRY(cudaMemsetAsync(c->wxp.p, 0, bytes, c->stream));
    if (tc_make_operand(c->tcplan, c->op_wbp, c->wbp.as<float>(), N, npad, xld, xplane, un) ||
        tc_make_operand(c->tcplan, c->op_wyp, c->wyp.as<float>(), N, npad, xld, xplane, un) ||
        tc_make_operand(c->tcplan, c->op_wxp, c->wxp.as<float>(), N, npad, xld, xplane, un))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    c->w_N = N;
    c->w_npad = npad;
    c->w_un = un;
    c->w_xld = xld;
    c->w_xplane = xplane;
  }
  TRY(c->wflags.ensure((size_t)2 * ns * G * sizeof(int)));
  const int* perm0 = c->wperm.as<int>() + 2 * (size_t)N;
  WaveSolve ws;
  ws.N = N;
  ws.nsteps = ns;
  ws.nrhs = nrhs;
  ws.un = un;
  ws.sb = c->wave_sb_ready;
  ws.xp = c->wyp.as<float>();
  ws.xp_ld = xld;
  ws.xp_plane = xplane;
  ws.flags = c->wflags.as<int>();
  if (c->wave_trace) {
    TRY(c->wtrace.ensure((size_t)2 * ns * G * 4 * sizeof(long long)));
    c->wtrace_units = ns * G;
    ws.trace = c->wtrace.as<long long>();
  }
  if (wave_rhs_planes(X, ldx, perm0, N, nrhs, c->wbp.as<float>(), xld, xplane, c->stream) ||
      wave_sweep(c->tcplan, true, c->op_lu, c->op_wdi, c->op_wbp, c->op_wyp, ws, c->stream))
    return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
  ws.xp = c->wxp.as<float>();
  ws.xout = X;
  ws.ldx = ldx;
  ws.flags = c->wflags.as<int>() + (size_t)ns * G;
  if (ws.trace) ws.trace += (size_t)ns * G * 4;
  if (wave_sweep(c->tcplan, false, c->op_lu, c->op_wdi, c->op_wyp, c->op_wxp, ws, c->stream))
    return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
  c->launches += 3;
  return HPRMAT_B200_OK;
}

// One CTA waits, with a limit of `limit` polls, on a counter that nothing increments: the
// bounded wait of the panel's grid barrier, run out on purpose to check the failure report.
__global__ void wait_probe_kernel(int* counter, int* timeout_flag, unsigned limit) {
  grid_wait(counter, timeout_flag, 1u, 99, limit);
}

// C[M x N] -= A[M x K] B[K x N] in complex FP64 (column-major) on the context's stream, by
// this library's DMMA kernel (zgemm_f64.cu).
static int zgemm_update(hprmat_b200_ctx* c, int M, int N, int K, const double2* A, long lda, const double2* B,
                        long ldb, double2* C, long ldc) {
  if (zgemm_f64_update(M, N, K, A, lda, B, ldb, C, ldc, c->stream))
    return fail(HPRMAT_B200_ERR_CUDA, "FP64 complex GEMM update: %s", hprmat_b200_last_error());
  ++c->launches;
  return HPRMAT_B200_OK;
}

template <typename T, int NB>
static int factor_impl(hprmat_b200_ctx* c, T* W, long ld, int N, bool mixed, LUState& st) {
  constexpr int NT = 256;
  const int nsteps = (N + NB - 1) / NB;
  c->lu_held = false;  // W, lup and the wave buffers are overwritten
  ++c->factorizations;
  st.N = N;
  st.ld = ld;
  st.nb = NB;
  st.nsteps = nsteps;
  int* status = c->status.as<int>();
  HPR_CUDA_TRY(cudaMemsetAsync(status, 0, SW_COUNT * sizeof(int), c->stream));
  const int G0 = std::min(c->nsm, std::max(1, (N + 31) / 32));
  TRY(c->stage.ensure((size_t)2 * G0 * NB * sizeof(T) + (size_t)NB * sizeof(unsigned long long) +
                      (size_t)2 * NB * sizeof(T) + 256));
  TRY(c->swaps.ensure((size_t)nsteps * kSwapStride * sizeof(int)));
  TRY(c->ipiv.ensure((size_t)N * sizeof(int) + 64));
  unsigned char* sp = c->stage.as<unsigned char>();
  T* cand_rows = reinterpret_cast<T*>(sp);
  sp += (size_t)2 * G0 * NB * sizeof(T);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(sp);
  sp += (size_t)NB * sizeof(unsigned long long);
  T* rowj = reinterpret_cast<T*>(sp);
  unsigned* growth = reinterpret_cast<unsigned*>(status + SW_COUNT - 1);

  float* bop = nullptr;
  long plane = 0;
  if (mixed) {
    // B operand of the trailing update (U12, K-major per column) and the LU planes
    plane = (long)(N + 256) * NB;
    TRY(c->ops.ensure((size_t)4 * plane * sizeof(float)));
    bop = c->ops.as<float>();
    c->lup_ld = (N + 3) / 4 * 4;
    c->lup_plane = c->lup_ld * (long)N;
    TRY(c->lup.ensure((size_t)4 * c->lup_plane * sizeof(float)));
    TRY(c->linv.ensure((size_t)4 * NB * NB * sizeof(float)));
    if (N > NB) {  // views are used only when there is more than one block step
      if (tc_make_operand(c->tcplan, c->op_linv, c->linv.as<float>(), NB, NB, NB, (long)NB * NB, 128))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      if (tc_make_operand(c->tcplan, c->op_lu, c->lup.as<float>(), N, N, c->lup_ld, c->lup_plane, 128))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      if (tc_make_operand(c->tcplan, c->op_bop, bop, NB, N, NB, plane, 128))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    }
  }

  // after the panel of step s: row interchanges, U12 = L11^-1 P A12 and the trailing update
  auto after_panel = [&](int s, int k0, int ncols, const StepSwaps& sw) -> int {
    (void)s;
    // row interchanges + U12 = L11^-1 A12
    if (mixed && c->tc_trsm) {
      // L11^-1 (as I - L11^-1 operand planes), P A12 gathered, U12 by one tensor-core GEMM
      constexpr int CW = 32;
      const size_t ism = ((size_t)NB * NB + (size_t)(NB / 2) * (NB / 2)) * sizeof(float2);
      constexpr int NTI = 512;
      auto ik = l11_inverse_planes_kernel<NB, NTI>;
      TRY(set_smem(ik, ism));
      ik<<<1, NTI, ism, c->stream>>>(reinterpret_cast<const float2*>(W), ld, k0, ncols, c->linv.as<float>(),
                                     (long)NB * NB);
      LAUNCH_CHECK();
      auto gk = swap_gather_kernel<NB, CW, NT>;
      const size_t gsm = (size_t)CW * (NB + 1) * sizeof(float2) + (size_t)CW * NB * sizeof(float2);
      TRY(set_smem(gk, gsm));
      gk<<<cdiv_u(N - k0 - ncols, CW), NT, gsm, c->stream>>>(reinterpret_cast<float2*>(W), ld, k0, ncols,
                                                              sw.top_src, sw.extra_dst, sw.extra_src,
                                                              sw.n_extra, k0 + ncols, N, bop, plane);
      LAUNCH_CHECK();
      if (tc_update(c->tcplan, c->op_linv, 0, 0, c->op_bop, 0, 0, NB,
                    reinterpret_cast<float2*>(W) + k0 + (size_t)(k0 + ncols) * ld, ld, ncols, N - k0 - ncols, 128,
                    c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      ++c->launches;
      auto uk = u12_split_kernel<NB, CW, NT>;
      uk<<<cdiv_u(N - k0 - ncols, CW), NT, 0, c->stream>>>(reinterpret_cast<const float2*>(W), ld, k0, ncols,
                                                             k0 + ncols, N, bop, plane, c->lup.as<float>(),
                                                             c->lup_ld, c->lup_plane, growth);
      LAUNCH_CHECK();
    } else {
      constexpr int CW = 32;
      auto tk = trsm_lower_kernel<T, NB, CW, NT>;
      size_t tsm = (size_t)CW * (NB + 1) * sizeof(T) + (size_t)CW * NB * sizeof(T);
      TRY(set_smem(tk, tsm));
      TrsmArgs<T> ta{};
      ta.W = W;
      ta.ld = ld;
      ta.k0 = k0;
      ta.ncols = ncols;
      ta.top_src = sw.top_src;
      ta.extra_dst = sw.extra_dst;
      ta.extra_src = sw.extra_src;
      ta.n_extra = sw.n_extra;
      ta.X = W;
      ta.ldx = ld;
      ta.c_begin = k0 + ncols;
      ta.c_end = N;
      ta.growth_bits = growth;
      if (mixed) {  // U12 also as the B operand of the trailing update and into the LU planes
        ta.bop = bop;
        ta.bop_plane = plane;
        ta.bop_col0 = k0 + ncols;
        ta.lup = c->lup.as<float>();
        ta.lup_ld = c->lup_ld;
        ta.lup_plane = c->lup_plane;
      }
      tk<<<cdiv_u(N - k0 - ncols, CW), NT, tsm, c->stream>>>(ta);
      LAUNCH_CHECK();
    }
    // trailing update A22 -= L21 U12
    const int M2 = N - k0 - ncols;
    if (mixed) {
      const bool prof = c->profile && c->ev_used + 2 <= (int)c->ev.size();
      if (prof) HPR_CUDA_TRY(cudaEventRecord(c->ev[c->ev_used], c->stream));
      if (tc_update(c->tcplan, c->op_lu, k0, k0 + ncols, c->op_bop, 0, 0, NB,
                    reinterpret_cast<float2*>(W) + (k0 + ncols) + (size_t)(k0 + ncols) * ld, ld, M2, M2, 128,
                    c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      ++c->launches;
      if (prof) {
        HPR_CUDA_TRY(cudaEventRecord(c->ev[c->ev_used + 1], c->stream));
        c->ev_flops.push_back(8.0 * (double)M2 * (double)M2 * (double)NB);
        c->ev_used += 2;
      }
    } else if constexpr (std::is_same<T, double2>::value) {
      // FP64 path: the trailing update C -= A B on the FP64 tensor cores (zgemm_f64.cu)
      if (M2 > 0) TRY(zgemm_update(c, M2, M2, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld,
                                   W + k0 + (size_t)(k0 + ncols) * ld, ld,
                                   W + (k0 + ncols) + (size_t)(k0 + ncols) * ld, ld));
    } else {
      dim3 grid(cdiv_u(M2, 64), cdiv_u(M2, 64));
      cgemm_update_kernel<T><<<grid, 256, 0, c->stream>>>(M2, M2, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld,
                                                         W + k0 + (size_t)(k0 + ncols) * ld, ld,
                                                         W + (k0 + ncols) + (size_t)(k0 + ncols) * ld, ld);
      LAUNCH_CHECK();
    }
    return HPRMAT_B200_OK;
  };

  // Plain FP64 path, NB = 64: block steps s (even) and s + 1 share one K = 128 trailing update,
  // so that the trailing matrix streams through memory once per two panels.  After panel s only
  // the next panel's columns are brought up to date (interchanges, U12, a 64-column update);
  // after panel s + 1, for the columns right of both panels: step s's interchanges and U12,
  // step s + 1's interchanges, rows k1 .. k2 minus step s's product (its L21 rows in step s + 1's
  // order), step s + 1's U12, and A22 -= [P L21(s) | L21(s+1)] [U12(s); U12(s+1)], the first
  // half of the A operand gathered in step s + 1's row order.  The factors are stored as the
  // single-step path stores them (L21 of a step in its own row order).
  constexpr bool kPairable = std::is_same<T, double2>::value && NB == 64;
  const bool pair = kPairable && !mixed && c->f64_pair && nsteps >= 3;
  auto step_swaps = [&](int s) {
    int* swb = c->swaps.as<int>() + (size_t)s * kSwapStride;
    return StepSwaps{swb, swb + kMaxNB, swb + 2 * kMaxNB, swb + 3 * kMaxNB};
  };
  auto trsm = [&](int k0, int ncols, const StepSwaps& sw, int c_begin, int c_end, int mode) -> int {
    if (c_end <= c_begin) return HPRMAT_B200_OK;
    constexpr int CW = 32;
    auto tk = trsm_lower_kernel<T, NB, CW, NT>;
    const size_t tsm = (size_t)CW * (NB + 1) * sizeof(T) + (size_t)CW * NB * sizeof(T);
    TRY(set_smem(tk, tsm));
    TrsmArgs<T> ta{};
    ta.W = W;
    ta.ld = ld;
    ta.k0 = k0;
    ta.ncols = ncols;
    ta.top_src = sw.top_src;
    ta.extra_dst = sw.extra_dst;
    ta.extra_src = sw.extra_src;
    ta.n_extra = sw.n_extra;
    ta.X = W;
    ta.ldx = ld;
    ta.c_begin = c_begin;
    ta.c_end = c_end;
    ta.growth_bits = growth;
    ta.mode = mode;
    tk<<<cdiv_u(c_end - c_begin, CW), NT, tsm, c->stream>>>(ta);
    LAUNCH_CHECK();
    return HPRMAT_B200_OK;
  };
  auto pair_first = [&](int s, int k0) -> int {  // after panel s: the next panel's columns
    const int k1 = k0 + NB;
    TRY(trsm(k0, NB, step_swaps(s), k1, k1 + NB, 0));
    if constexpr (kPairable)
      TRY(zgemm_update(c, N - k1, NB, NB, W + k1 + (size_t)k0 * ld, ld, W + k0 + (size_t)k1 * ld, ld,
                       W + k1 + (size_t)k1 * ld, ld));
    return HPRMAT_B200_OK;
  };
  auto pair_second = [&](int s, int k0) -> int {  // after panel s + 1: everything right of both
    if constexpr (kPairable) {
      const int k1 = k0 + NB, k2 = k1 + NB;
      const int m2 = N - k2;
      const StepSwaps s0 = step_swaps(s), s1 = step_swaps(s + 1);
      TRY(trsm(k0, NB, s0, k2, N, 0));
      TRY(trsm(k1, NB, s1, k2, N, 1));
      // rows k1 .. k2 minus L21(s) (rows in step s + 1's order) U12(s)
      TRY(c->f64_pair_buf.ensure(((size_t)NB * NB + (size_t)m2 * 2 * NB) * sizeof(T)));
      T* F = c->f64_pair_buf.as<T>();
      T* LL = F + (size_t)NB * NB;
      gather_block_kernel<T><<<dim3(1, 16), NB, 0, c->stream>>>(W, ld, s1.top_src, 0, NB, k0, NB, F, NB);
      LAUNCH_CHECK();
      TRY(zgemm_update(c, NB, m2, NB, F, NB, W + k0 + (size_t)k2 * ld, ld, W + k1 + (size_t)k2 * ld, ld));
      TRY(trsm(k1, NB, s1, k2, N, 2));
      // A operand [P L21(s) | L21(s+1)], rows k2 .., and the K = 128 update
      gather_block_kernel<T><<<dim3(cdiv_u(m2, 256), 32), 256, 0, c->stream>>>(W, ld, nullptr, k2, m2, k0, 2 * NB, LL,
                                                                              m2);
      LAUNCH_CHECK();
      patch_rows_kernel<T><<<1, 256, 0, c->stream>>>(W, ld, s1.extra_dst, s1.extra_src, s1.n_extra, k2, k0, NB, LL, m2);
      LAUNCH_CHECK();
      TRY(zgemm_update(c, m2, m2, 2 * NB, LL, m2, W + k0 + (size_t)k2 * ld, ld, W + k2 + (size_t)k2 * ld, ld));
    }
    return HPRMAT_B200_OK;
  };
  // what follows the panel of step s
  auto after_step = [&](int s, int k0, int ncols, const StepSwaps& sw) -> int {
    if (pair && s + 2 < nsteps && (s & 1) == 0) return pair_first(s, k0);
    if (pair && (s & 1) == 1 && s + 1 < nsteps) return pair_second(s - 1, k0 - NB);
    return after_panel(s, k0, ncols, sw);
  };
  auto pk = panel_kernel<T, NB, NT>;
  auto pkc = panel_cluster_kernel<T, NB, NT>;
  // the largest rows per CTA of a cluster panel (shared memory of the opt-in limit, less the
  // static arrays)
  int rpc_max_c = 0;
  while (panel_cluster_smem<T>(rpc_max_c + 1, NB) + 4096 <= (size_t)c->smem_optin) ++rpc_max_c;
  auto cluster_fits = [&](int g) -> bool {  // can the GPU hold a cluster of g such CTAs
    signed char& ok = c->cluster_ok[sizeof(T) == sizeof(double2)][g];
    if (ok == 0) {
      const size_t sm = panel_cluster_smem<T>(rpc_max_c, NB);
      ok = -1;
      if (cudaFuncSetAttribute((const void*)pkc, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
          set_smem(pkc, sm) == HPRMAT_B200_OK) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g);
        cfg.blockDim = dim3(NT);
        cfg.dynamicSmemBytes = sm;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = g;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void*)pkc, &cfg) == cudaSuccess && n >= 1) ok = 1;
      }
      cudaGetLastError();
    }
    return ok == 1;
  };
  for (int s = 0; s < nsteps; ++s) {
    const int k0 = s * NB;
    const int ncols = std::min(NB, N - k0);
    const int m = N - k0;
    if (c->panel_cluster && rpc_max_c > 0 && m <= 16 * rpc_max_c) {
      // the whole panel in one cluster: as many CTAs as panel_rpc_min rows allow, at most 16
      const int Gc = std::min(16, std::max((m + rpc_max_c - 1) / rpc_max_c, (m + c->panel_rpc_min - 1) / c->panel_rpc_min));
      if (cluster_fits(Gc)) {
        const int rpcc = (m + Gc - 1) / Gc;
        const size_t smc = panel_cluster_smem<T>(rpcc, NB);
        TRY(set_smem(pkc, smc));
        PanelArgs<T> pa;
        pa.W = W;
        pa.ld = ld;
        pa.N = N;
        pa.k0 = k0;
        pa.ncols = ncols;
        pa.rpc = rpcc;
        pa.G = Gc;
        pa.ipiv = c->ipiv.as<int>();
        pa.cand_rows = nullptr;
        pa.keys = nullptr;
        pa.rowj = nullptr;
        pa.status = status;
        int* swb = c->swaps.as<int>() + (size_t)s * kSwapStride;
        pa.sw.top_src = swb;
        pa.sw.extra_dst = swb + kMaxNB;
        pa.sw.extra_src = swb + 2 * kMaxNB;
        pa.sw.n_extra = swb + 3 * kMaxNB;
        pa.growth_bits = growth;
        pa.lup = (mixed && k0 + ncols < N) ? c->lup.as<float>() : nullptr;
        pa.lup_ld = c->lup_ld;
        pa.lup_plane = c->lup_plane;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(Gc);
        cfg.blockDim = dim3(NT);
        cfg.dynamicSmemBytes = smc;
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = Gc;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(&cfg, pkc, pa);
        if (e != cudaSuccess)
          return fail(HPRMAT_B200_ERR_CUDA, "cluster panel launch (step %d, %d CTAs of %d rows, %zu B shared): %s", s,
                      Gc, rpcc, smc, cudaGetErrorString(e));
        ++c->launches;
        if (k0 + ncols >= N) break;
        TRY(after_step(s, k0, ncols, pa.sw));
        continue;
      }
    }
    // CTAs of the panel: at least panel_rpc_min rows each (fewer CTAs contend less for the
    // per-column barrier), as many as the shared memory needs
    const int rpc_max = (int)(((size_t)c->smem_optin - 8192) / sizeof(T) / NB) - 2;
    const int G = std::min(G0, std::max(std::min(G0, std::max(1, (m + c->panel_rpc_min - 1) / c->panel_rpc_min)),
                                        (m + rpc_max - 1) / rpc_max));
    const int rpc = (m + G - 1) / G;
    const size_t smem = ((size_t)NB * (rpc | 1) + NB) * sizeof(T);
    TRY(set_smem(pk, smem));
    HPR_CUDA_TRY(cudaMemsetAsync(status + SW_BARRIER, 0, sizeof(int), c->stream));
    HPR_CUDA_TRY(cudaMemsetAsync(keys, 0, (size_t)NB * sizeof(unsigned long long), c->stream));
    PanelArgs<T> pa;
    pa.W = W;
    pa.ld = ld;
    pa.N = N;
    pa.k0 = k0;
    pa.ncols = ncols;
    pa.rpc = rpc;
    pa.G = G;
    pa.ipiv = c->ipiv.as<int>();
    pa.cand_rows = cand_rows;
    pa.keys = keys;
    pa.rowj = rowj;
    pa.status = status;
    int* swb = c->swaps.as<int>() + (size_t)s * kSwapStride;
    pa.sw.top_src = swb;
    pa.sw.extra_dst = swb + kMaxNB;
    pa.sw.extra_src = swb + 2 * kMaxNB;
    pa.sw.n_extra = swb + 3 * kMaxNB;
    pa.growth_bits = growth;
    pa.lup = (mixed && k0 + ncols < N) ? c->lup.as<float>() : nullptr;
    pa.lup_ld = c->lup_ld;
    pa.lup_plane = c->lup_plane;
    pa.trace = nullptr;
    if (c->wave_trace && (s == 0 || s == nsteps / 2)) {
      TRY(c->ptrace.ensure((size_t)2 * kMaxNB * kPanelTraceW * sizeof(long long)));
      if (s == 0) HPR_CUDA_TRY(cudaMemsetAsync(c->ptrace.p, 0, c->ptrace.bytes, c->stream));
      pa.trace = c->ptrace.as<long long>() + (s == 0 ? 0 : (size_t)kMaxNB * kPanelTraceW);
    }
    void* args[] = {&pa};
    {
      const cudaError_t e = cudaLaunchCooperativeKernel((void*)pk, dim3(G), dim3(NT), args, smem, c->stream);
      if (e != cudaSuccess) {
        int occ = -1;
        cudaGetLastError();
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pk, NT, smem);
        return fail(HPRMAT_B200_ERR_CUDA, "panel launch (step %d, %d CTAs of %d rows, %zu B shared, %d per SM): %s", s,
                    G, rpc, smem, occ, cudaGetErrorString(e));
      }
    }
    ++c->launches;
    if (k0 + ncols >= N) break;
    TRY(after_step(s, k0, ncols, pa.sw));
  }
  // explicit inverses of the diagonal blocks for the solves
  {
    TRY(c->inv.ensure((size_t)2 * nsteps * NB * NB * sizeof(T)));
    auto ik = tri_inverse_kernel<T, NB, NT>;
    size_t ism = ((size_t)NB * NB + NB) * sizeof(T);
    TRY(set_smem(ik, ism));
    ik<<<dim3(nsteps, 2), NT, ism, c->stream>>>(W, ld, N, NB, c->inv.as<T>());
    LAUNCH_CHECK();
  }
  c->wave_ready = false;
  if constexpr (NB == 128 && std::is_same<T, float2>::value) {
    if (mixed && nsteps >= 2 && c->wave_enabled) TRY(wave_prepare(c, st));
  }
  HPR_CUDA_TRY(cudaMemcpyAsync(c->h_status, status, kStatusCopy * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (c->h_status[SW_TIMEOUT] != 0)
    return fail(HPRMAT_B200_ERR_TIMEOUT, "panel factorisation: grid barrier wait limit exceeded (site %d)",
                c->h_status[SW_TIMEOUT]);
  if (c->profile) {
    for (int i = 0; i + 1 < c->ev_used; i += 2) {
      float ms = 0.f;
      HPR_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]));
      c->tc_ms += ms;
      c->tc_flops += c->ev_flops[i / 2];
      ++c->tc_launches;
    }
    c->ev_used = 0;
    c->ev_flops.clear();
  }
  if (mixed) {
    int err = 0;
    TRY(tc_gemm_check(c->tcplan, c->stream, &err));
    if (err) return fail(HPRMAT_B200_ERR_TIMEOUT, "tensor-core update: wait limit exceeded at site %d", err);
  }
  return HPRMAT_B200_OK;
}

template <typename T>
static int factor(hprmat_b200_ctx* c, T* W, long ld, int N, bool mixed, int nb, LUState& st) {
  NvtxRange nv(mixed ? "hprmat.factor.mixed" : "hprmat.factor.fp64");
  if (N >= PivotKey<T>::kMaxRows)
    return fail(HPRMAT_B200_ERR_UNSUPPORTED, "order %d beyond the pivot keys' row range", N);
  switch (nb) {
    case 128: return factor_impl<T, 128>(c, W, ld, N, mixed, st);
    case 64: return factor_impl<T, 64>(c, W, ld, N, mixed, st);
    case 32: return factor_impl<T, 32>(c, W, ld, N, mixed, st);
    case 16: return factor_impl<T, 16>(c, W, ld, N, mixed, st);
  }
  return fail(HPRMAT_B200_ERR_UNSUPPORTED, "unsupported block size %d", nb);
}

// Forward and backward substitution with the stored factors, in place on X (N x nrhs).
template <typename T, int NB>
static int lu_solve_impl(hprmat_b200_ctx* c, const T* W, const LUState& st, T* X, long ldx, int nrhs) {
  const int N = st.N;
  const long ld = st.ld;
  const T* inv = c->inv.as<T>();
  constexpr int DCW = 2;
  auto dk = diag_apply_kernel<T, NB, DCW>;
  const size_t dsm = ((size_t)NB * NB + 2 * DCW * NB) * sizeof(T);
  TRY(set_smem(dk, dsm));
  const int* swb = c->swaps.as<int>();
  for (int s = 0; s < st.nsteps; ++s) {
    const int k0 = s * NB, ncols = std::min(NB, N - k0);
    const int* sw = swb + (size_t)s * kSwapStride;
    dk<<<cdiv_u(nrhs, DCW), NB * DCW, dsm, c->stream>>>(inv + (size_t)2 * s * NB * NB, ncols, k0, sw, sw + kMaxNB, sw + 2 * kMaxNB,
                                   sw + 3 * kMaxNB, X, ldx, nrhs, nullptr, 0);
    LAUNCH_CHECK();
    const int M2 = N - k0 - ncols;
    if (M2 > 0 && nrhs <= 8) {
      cgemv_update_kernel<T><<<cdiv_u(M2, 256), 256, 0, c->stream>>>(
          M2, nrhs, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld, X + k0, ldx, X + k0 + ncols, ldx);
      LAUNCH_CHECK();
    } else if (M2 > 0) {
      if constexpr (std::is_same<T, double2>::value) {
        TRY(zgemm_update(c, M2, nrhs, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld, X + k0, ldx, X + k0 + ncols,
                         ldx));
      } else {
        dim3 grid(cdiv_u(M2, 64), cdiv_u(nrhs, 64));
        cgemm_update_kernel<T><<<grid, 256, 0, c->stream>>>(M2, nrhs, ncols, W + (k0 + ncols) + (size_t)k0 * ld, ld,
                                                           X + k0, ldx, X + k0 + ncols, ldx);
        LAUNCH_CHECK();
      }
    }
  }
  for (int s = st.nsteps - 1; s >= 0; --s) {
    const int k0 = s * NB, ncols = std::min(NB, N - k0);
    dk<<<cdiv_u(nrhs, DCW), NB * DCW, dsm, c->stream>>>(inv + ((size_t)2 * s + 1) * NB * NB, ncols, k0, nullptr, nullptr, nullptr,
                                   nullptr, X, ldx, nrhs, nullptr, 0);
    LAUNCH_CHECK();
    if (k0 > 0 && nrhs <= 8) {
      cgemv_update_kernel<T><<<cdiv_u(k0, 256), 256, 0, c->stream>>>(k0, nrhs, ncols, W + (size_t)k0 * ld, ld,
                                                                     X + k0, ldx, X, ldx);
      LAUNCH_CHECK();
    } else if (k0 > 0) {
      if constexpr (std::is_same<T, double2>::value) {
        TRY(zgemm_update(c, k0, nrhs, ncols, W + (size_t)k0 * ld, ld, X + k0, ldx, X, ldx));
      } else {
        dim3 grid(cdiv_u(k0, 64), cdiv_u(nrhs, 64));
        cgemm_update_kernel<T><<<grid, 256, 0, c->stream>>>(k0, nrhs, ncols, W + (size_t)k0 * ld, ld, X + k0, ldx,
                                                           X, ldx);
        LAUNCH_CHECK();
      }
    }
  }
  return HPRMAT_B200_OK;
}

// Mixed path: the same blocked substitution with the block updates on the tensor cores.
// Each diagonal block (explicit inverse) also emits its result as the B operand; the update
// reads L21 / U12 from the LU planes.
template <int NB>
static int lu_solve_tc_impl(hprmat_b200_ctx* c, const LUState& st, float2* X, long ldx, int nrhs) {
  if (NB == 128 && c->wave_ready) return lu_solve_wave(c, st, X, ldx, nrhs);
  const int N = st.N;
  const float2* inv = c->inv.as<float2>();
  constexpr int DCW = 2;
  auto dk = diag_apply_kernel<float2, NB, DCW>;
  const size_t dsm = ((size_t)NB * NB + 2 * DCW * NB) * sizeof(float2);
  TRY(set_smem(dk, dsm));
  const int npad = (nrhs + 127) / 128 * 128;
  if (c->rop_nrhs != npad || c->rop_nb != NB || !c->rop.p) {  // the map's K extent is NB
    c->rop_plane = (long)npad * NB;
    TRY(c->rop.ensure((size_t)4 * c->rop_plane * sizeof(float)));
    HPR_CUDA_TRY(cudaMemsetAsync(c->rop.p, 0, (size_t)4 * c->rop_plane * sizeof(float), c->stream));
    if (tc_make_operand(c->tcplan, c->op_rhs, c->rop.as<float>(), NB, npad, NB, c->rop_plane, 128))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    c->rop_nrhs = npad;
    c->rop_nb = NB;
  }
  float* rop = c->rop.as<float>();
  const int* swb = c->swaps.as<int>();
  for (int s = 0; s < st.nsteps; ++s) {
    const int k0 = s * NB, ncols = std::min(NB, N - k0);
    const int* sw = swb + (size_t)s * kSwapStride;
    const int M2 = N - k0 - ncols;
    dk<<<cdiv_u(nrhs, DCW), NB * DCW, dsm, c->stream>>>(inv + (size_t)2 * s * NB * NB, ncols, k0, sw, sw + kMaxNB, sw + 2 * kMaxNB,
                                   sw + 3 * kMaxNB, X, ldx, nrhs, M2 > 0 ? rop : nullptr, c->rop_plane);
    LAUNCH_CHECK();
    if (M2 > 0) {
      if (tc_update(c->tcplan, c->op_lu, k0, k0 + ncols, c->op_rhs, 0, 0, (ncols + 15) / 16 * 16, X + k0 + ncols,
                    ldx, M2, nrhs, 128, c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      ++c->launches;
    }
  }
  for (int s = st.nsteps - 1; s >= 0; --s) {
    const int k0 = s * NB, ncols = std::min(NB, N - k0);
    dk<<<cdiv_u(nrhs, DCW), NB * DCW, dsm, c->stream>>>(inv + ((size_t)2 * s + 1) * NB * NB, ncols, k0, nullptr, nullptr, nullptr,
                                   nullptr, X, ldx, nrhs, k0 > 0 ? rop : nullptr, c->rop_plane);
    LAUNCH_CHECK();
    if (k0 > 0) {
      if (tc_update(c->tcplan, c->op_lu, k0, 0, c->op_rhs, 0, 0, (ncols + 15) / 16 * 16, X, ldx, k0, nrhs, 128,
                    c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      ++c->launches;
    }
  }
  return HPRMAT_B200_OK;
}

static int lu_solve_tc(hprmat_b200_ctx* c, const LUState& st, float2* X, long ldx, int nrhs) {
  NvtxRange nv("hprmat.solve.mixed");
  switch (st.nb) {
    case 128: return lu_solve_tc_impl<128>(c, st, X, ldx, nrhs);
    case 64: return lu_solve_tc_impl<64>(c, st, X, ldx, nrhs);
    case 32: return lu_solve_tc_impl<32>(c, st, X, ldx, nrhs);
    case 16: return lu_solve_tc_impl<16>(c, st, X, ldx, nrhs);
  }
  return fail(HPRMAT_B200_ERR_UNSUPPORTED, "unsupported block size %d", st.nb);
}

template <typename T>
static int lu_solve(hprmat_b200_ctx* c, const T* W, const LUState& st, T* X, long ldx, int nrhs) {
  NvtxRange nv("hprmat.solve");
  switch (st.nb) {
    case 128: return lu_solve_impl<T, 128>(c, W, st, X, ldx, nrhs);
    case 64: return lu_solve_impl<T, 64>(c, W, st, X, ldx, nrhs);
    case 32: return lu_solve_impl<T, 32>(c, W, st, X, ldx, nrhs);
    case 16: return lu_solve_impl<T, 16>(c, W, st, X, ldx, nrhs);
  }
  return fail(HPRMAT_B200_ERR_UNSUPPORTED, "unsupported block size %d", st.nb);
}

// ------------------------------------------------------------------ operators for refinement
// out = with_b * B - C X (FP64).  Either the structured C(E) of the R-matrix problem or a
// dense FP64 matrix.
struct Operator {
  bool structured = false;
  // structured
  MeshDev mesh;
  ChannelData ch;
  int nch = 0;
  const double2* vt = nullptr;  // potential per mesh point (cpot_transpose_kernel layout)
  // dense
  const double2* A = nullptr;
  long lda = 0;
  const double2* B = nullptr;  // dense right-hand side (N x nrhs, ld = ldb)
  long ldb = 0;
  int N = 0;
  // R-matrix problems: surface projection R = q2^T X per channel block, for the stopping rule
  const double* q2 = nullptr;
  const double* q1 = nullptr;  // propagated intervals: leading blockdiag(q1) right-hand sides
  int nr = 0;
};

// absmode: out = |B| + |C| |X| instead (structured operator only).
static int apply_residual(hprmat_b200_ctx* c, const Operator& op, const double2* X, long ldx, int ncol,
                          double2* out, long ldo, bool with_b, bool absmode = false) {
  const int N = op.N;
  if (op.structured && !with_b && !absmode) {
    // plain product (inner iterations): tiled batched kernels
    const int nr = op.mesh.nr;
    KineticTile kt{op.mesh, op.ch, X, ldx, with_b ? 1 : 0};
    resid_tile_kernel<KineticTile, true>
        <<<dim3(cdiv_u(nr, 64), cdiv_u(ncol, 64), op.nch), 256, 0, c->stream>>>(kt, nr, ncol, nr, out, ldo);
    LAUNCH_CHECK();
    CouplingTile ct{op.vt, X, ldx, nr, op.nch};
    resid_tile_kernel<CouplingTile, false>
        <<<dim3(cdiv_u(op.nch, 64), cdiv_u(ncol, 64), nr), 256, 0, c->stream>>>(ct, op.nch, ncol, op.nch, out, ldo);
    LAUNCH_CHECK();
    return HPRMAT_B200_OK;
  }
  if (op.structured) {
    // outer residual (compensated, low words in rlo) or its rounding scale (absmode)
    const int nr = op.mesh.nr;
    double2* lo = nullptr;
    if (!absmode) {
      TRY(c->rlo.ensure((size_t)ldo * ncol * sizeof(double2)));
      lo = c->rlo.as<double2>();
    }
    KineticTile kt{op.mesh, op.ch, X, ldx, with_b ? 1 : 0};
    CouplingTile ct{op.vt, X, ldx, nr, op.nch};
    const int yt = (int)cdiv_u(ncol, 64);
    const dim3 gk(cdiv_u(nr, 32), yt, op.nch), gc(cdiv_u(op.nch, 32), yt, nr);
    if (absmode) {
      resid_tile2_kernel<KineticTile, true, kAbs1><<<gk, 256, 0, c->stream>>>(kt, nr, ncol, nr, out, ldo, lo, yt, 0);
      LAUNCH_CHECK();
      resid_tile2_kernel<CouplingTile, false, kAbs2><<<gc, 256, 0, c->stream>>>(ct, op.nch, ncol, op.nch, out, ldo,
                                                                               lo, yt, 0);
    } else {
      resid_tile2_kernel<KineticTile, true, kComp1><<<gk, 256, 0, c->stream>>>(kt, nr, ncol, nr, out, ldo, lo, yt, 0);
      LAUNCH_CHECK();
      resid_tile2_kernel<CouplingTile, false, kComp2><<<gc, 256, 0, c->stream>>>(ct, op.nch, ncol, op.nch, out,
                                                                                ldo, lo, yt, 0);
    }
    LAUNCH_CHECK();
    return HPRMAT_B200_OK;
  }
  {
    dim3 g0(cdiv_u(N, 256), ncol);
    if (with_b) {
      copy_d_kernel<<<g0, 256, 0, c->stream>>>(op.B, op.ldb, out, ldo, N);
    } else {
      HPR_CUDA_TRY(cudaMemset2DAsync(out, ldo * sizeof(double2), 0, (size_t)N * sizeof(double2), ncol, c->stream));
    }
    LAUNCH_CHECK();
    // dense operator (solve_linear, non-local potentials): a plain FP64 GEMM (zgemm_f64.cu)
    TRY(zgemm_update(c, N, ncol, N, op.A, op.lda, X, ldx, out, ldo));
  }
  return HPRMAT_B200_OK;
}

// The outer (compensated) residual out_u = B - C_u X_u of `units` structured operators that
// differ only in their channel data (unit u: X + u sx, out + u so, channel data + u sch
// doubles), two launches for all of them.  op holds unit 0's channel data.
static int apply_residual_units(hprmat_b200_ctx* c, const Operator& op, const double2* X, long ldx, long sx, int ncol,
                                double2* out, long ldo, long so, long sch, int units) {
  const int nr = op.mesh.nr;
  if (so < ldo * (long)ncol) return fail(HPRMAT_B200_ERR_ARG, "apply_residual_units: unit stride below one block");
  TRY(c->rlo.ensure((size_t)so * units * sizeof(double2)));
  double2* lo = c->rlo.as<double2>();
  KineticTile kt{op.mesh, op.ch, X, ldx, 1};
  kt.sx = sx;
  kt.sch = sch;
  CouplingTile ct{op.vt, X, ldx, nr, op.nch};
  ct.sx = sx;
  const int yt = (int)cdiv_u(ncol, 64);
  const dim3 gk(cdiv_u(nr, 32), yt * units, op.nch), gc(cdiv_u(op.nch, 32), yt * units, nr);
  resid_tile2_kernel<KineticTile, true, kComp1><<<gk, 256, 0, c->stream>>>(kt, nr, ncol, nr, out, ldo, lo, yt, so);
  LAUNCH_CHECK();
  resid_tile2_kernel<CouplingTile, false, kComp2><<<gc, 256, 0, c->stream>>>(ct, op.nch, ncol, op.nch, out, ldo, lo,
                                                                            yt, so);
  LAUNCH_CHECK();
  return HPRMAT_B200_OK;
}

static int frob_norm(hprmat_b200_ctx* c, const double2* X, long ldx, int N, int ncol, double* result) {
  TRY(c->norms.ensure((size_t)ncol * sizeof(double)));
  colnorm2_kernel<<<ncol, 256, 0, c->stream>>>(X, ldx, N, c->norms.as<double>());
  LAUNCH_CHECK();
  HPR_CUDA_TRY(cudaMemcpyAsync(c->h_norms, c->norms.p, (size_t)ncol * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (int i = 0; i < ncol; ++i) s += c->h_norms[i];
  *result = sqrt(s);
  return HPRMAT_B200_OK;
}

// Mixed path: X64 (N x nrhs, FP64) from the FP32 factors, refined with FGMRES on the FP64
// operator.  Each outer step: r = B - C X; stop when |r|_F/|B|_F < tol; otherwise run
// up to gmres_m flexible-GMRES iterations on C d = r, preconditioned by the FP32 LU solve, and
// X += d.  Returns NOT_CONVERGED if max_refine outer corrections did not reach tol.
static int refine_mixed(hprmat_b200_ctx* c, const Operator& op, const float2* W32, const LUState& st,
                        double2* X64, long ldx, int nrhs, double bnorm, double cnorm, hprmat_b200_stats* stats,
                        int max_outer = -1, bool error_based = false) {
  NvtxRange nv("hprmat.refine");
  // error_based (factors of another energy, opts.reuse_factors): a small residual alone does
  // not stop the refinement -- the surface rule, which measures the error in R, must hold
  if (max_outer < 0) max_outer = c->opts.max_refine;
  const int N = op.N;
  const int m = std::min(c->gmres_m, kGmresMaxM);
  const long ldv = st.ld;
  const long vstride = ldv * nrhs;
  TRY(c->V.ensure((size_t)(m + 1) * vstride * sizeof(double2)));
  TRY(c->Z.ensure((size_t)m * vstride * sizeof(double2)));
  TRY(c->gm.ensure((size_t)nrhs * ((m + 1) * m * sizeof(double2) + m * sizeof(double) + m * sizeof(double2) +
                                   (m + 1) * sizeof(double2) + 2 * sizeof(double)) + 256));
  TRY(c->X.ensure((size_t)ldv * nrhs * sizeof(float2)));
  double2* V = c->V.as<double2>();
  double2* Z = c->Z.as<double2>();
  float2* X32 = c->X.as<float2>();
  GmresState gs;
  gs.V = V;
  gs.ldv = ldv;
  gs.vstride = vstride;
  unsigned char* gp = c->gm.as<unsigned char>();
  gs.H = reinterpret_cast<double2*>(gp);
  gp += (size_t)nrhs * (m + 1) * m * sizeof(double2);
  gs.sn = reinterpret_cast<double2*>(gp);
  gp += (size_t)nrhs * m * sizeof(double2);
  gs.g = reinterpret_cast<double2*>(gp);
  gp += (size_t)nrhs * (m + 1) * sizeof(double2);
  gs.cs = reinterpret_cast<double*>(gp);
  gp += (size_t)nrhs * m * sizeof(double);
  gs.beta = reinterpret_cast<double*>(gp);
  gp += (size_t)nrhs * sizeof(double);
  double* d_est = reinterpret_cast<double*>(gp);
  gs.m = m;
  gs.N = N;
  gs.ncol = nrhs;
  dim3 gconv(cdiv_u(N, 256), nrhs);
  int steps = 0;
  int status = HPRMAT_B200_OK;
  double prev_rel = 0.0, prev_change = 0.0, floor_rel = 0.0, last_est = 1.0;
  int inner_total = 0;
  const bool surf = op.q2 != nullptr;
  const int nchs = surf ? N / op.nr : 0;
  // monitored surface projections: q2^T X, and q1^T X on a propagated interval
  const size_t nsurf = (size_t)nchs * nrhs * (op.q1 ? 2 : 1);
  if (surf) TRY(c->rsurf.ensure(2 * nsurf * sizeof(double2) + 64));
  (void)cnorm;
  if (stats) stats->surface_change = -1.0;
  for (int outer = 0;; ++outer) {
    TRY(apply_residual(c, op, X64, ldx, nrhs, V, ldv, true));
    double rn;
    TRY(frob_norm(c, V, ldv, N, nrhs, &rn));
    const double rel = rn / bnorm;
    double change = -1.0;
    if (surf) {
      // R of the current iterate into slot (outer & 1); compare with the previous one
      double2* Rn = c->rsurf.as<double2>() + (size_t)(outer & 1) * nsurf;
      const dim3 ge(nchs, cdiv_u(nrhs, 128));
      rmat_extract_kernel<<<ge, 128, 0, c->stream>>>(X64, ldx, op.q2, op.nr, nchs, nrhs, 1.0, Rn);
      LAUNCH_CHECK();
      if (op.q1) {
        rmat_extract_kernel<<<ge, 128, 0, c->stream>>>(X64, ldx, op.q1, op.nr, nchs, nrhs, 1.0,
                                                       Rn + (size_t)nchs * nrhs);
        LAUNCH_CHECK();
      }
      if (outer > 0) {
        const double2* Ro = c->rsurf.as<double2>() + (size_t)((outer - 1) & 1) * nsurf;
        TRY(c->norms.ensure(2 * sizeof(double) * 2));
        rel_change_kernel<<<1, 256, 0, c->stream>>>(Rn, Ro, (int)nsurf, c->norms.as<double>());
        LAUNCH_CHECK();
        HPR_CUDA_TRY(cudaMemcpyAsync(c->h_norms, c->norms.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        change = c->h_norms[1] > 0 ? sqrt(c->h_norms[0] / c->h_norms[1]) : 0.0;
      }
    }
    if (op.structured && outer == 0) {
      // rounding scale of the residual: u || |B| + |C||X| ||_F / ||B||_F (reported only)
      TRY(apply_residual(c, op, X64, ldx, nrhs, V + vstride, ldv, true, true));
      double fn;
      TRY(frob_norm(c, V + vstride, ldv, N, nrhs, &fn));
      floor_rel = 1.1102230246251565e-16 * fn / bnorm;
      if (stats) stats->floor_history[0] = floor_rel;
    }
    if (stats && outer < 9) stats->residual_history[outer] = rel;
    if (stats) {
      stats->rel_residual = rel;
      stats->surface_change = change;
      stats->residual_floor = floor_rel;
    }
    if (!(rel >= c->opts.tol) && !(error_based && surf && rel > 0.0)) break;  // converged (also on rel == 0)
    if (surf && outer > 0) {
      // change = size of the last correction in R, i.e. the error of the previous iterate;
      // the last cycle reduced that error by about last_est, which predicts the error left.
      // (the GMRES estimate bounds the residual, not the error in R: keep a wide margin)
      const double predicted = change * std::max(last_est, 1e-16);
      if (!(change >= c->opts.surface_tol) || 1e3 * predicted < c->opts.surface_tol) break;
      if (outer >= 2 && change > 0.5 * prev_change) {  // no longer improving
        // on factors of another energy a stall means the preconditioner is too far off:
        // report it, so that the caller factorises C(E) itself
        if (predicted > 1e-8 || error_based) status = HPRMAT_B200_NOT_CONVERGED;
        break;
      }
    } else if (!surf && outer >= 1 && rel > 0.5 * prev_rel) {  // dense operator: residual stalled
      if (rel > 1e-8) status = HPRMAT_B200_NOT_CONVERGED;
      break;
    }
    if (outer >= max_outer) {
      status = HPRMAT_B200_NOT_CONVERGED;
      break;
    }
    prev_rel = rel;
    prev_change = change;
    gmres_start_kernel<256><<<nrhs, 256, 0, c->stream>>>(gs);
    LAUNCH_CHECK();
    // the first cycle starts from the FP32 solution; a later cycle aims at what is left to
    // the tolerance (a tenth of tol / rel), so that one polishing cycle usually ends it
    const double inner_tol =
        outer == 0 ? c->inner_tol0 : std::min(1e-2, std::max(1e-8, 0.1 * c->opts.tol / std::max(rel, 1e-300)));
    int jdone = 0;
    double est = 1.0;
    for (int j = 0; j < m; ++j) {
      d2f_kernel<<<gconv, 256, 0, c->stream>>>(V + (size_t)j * vstride, ldv, X32, ldv, N, nullptr);
      LAUNCH_CHECK();
      TRY(lu_solve_tc(c, st, X32, ldv, nrhs));
      f2d_kernel<<<gconv, 256, 0, c->stream>>>(X32, ldv, Z + (size_t)j * vstride, ldv, N, nullptr);
      LAUNCH_CHECK();
      // V_{j+1} = -C Z_j: FGMRES runs on the operator -C, so the correction is subtracted
      TRY(apply_residual(c, op, Z + (size_t)j * vstride, ldv, nrhs, V + (size_t)(j + 1) * vstride, ldv, false));
      gmres_arnoldi_kernel<kArnoldiNT><<<nrhs, kArnoldiNT, 0, c->stream>>>(gs, j);
      LAUNCH_CHECK();
      jdone = j + 1;
      // residual estimate of the cycle (worst column) from the Givens-rotated right side
      gmres_estimate_kernel<<<cdiv_u(nrhs, 128), 128, 0, c->stream>>>(gs.g, gs.beta, m, j, nrhs, d_est);
      LAUNCH_CHECK();
      HPR_CUDA_TRY(cudaMemcpyAsync(c->h_norms, d_est, (size_t)nrhs * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream));
      HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
      est = 0.0;
      for (int q = 0; q < nrhs; ++q) est = std::max(est, c->h_norms[q]);
      if (est < inner_tol) break;
    }
    last_est = est;
    gmres_update_kernel<256><<<nrhs, 256, 0, c->stream>>>(gs, jdone, Z, vstride, ldv, X64, ldx, -1.0);
    LAUNCH_CHECK();
    inner_total += jdone;
    ++steps;
  }
  if (stats) {
    stats->refine_steps = steps;
    stats->inner_iterations = inner_total;
  }
  {
    // a bounded wait that gave up inside a tensor-core solve invalidates the result
    int err = 0;
    TRY(tc_gemm_check(c->tcplan, c->stream, &err));
    if (err) return fail(HPRMAT_B200_ERR_TIMEOUT, "tensor-core solve: wait limit exceeded at site %d", err);
  }
  return status;
}

// ------------------------------------------------------------------ boundary values
struct Boundary {
  int nopen = 0;
  std::vector<int> open_idx, closed_idx;
  std::vector<double> fac, kk, bloch, qk, xc2;  // xc2: W(rmax) of closed channels (xc(c, 2))
  std::vector<double2> co, cop;
};

// src/rmatrix_hp.F90:224-244 and the per-channel diagonal terms of :259-276.
static int boundary_values(int nch, const int* lval, const double* qk, const double* eta, double rmax, double rmax2,
                           Boundary& b) {
  b = Boundary();
  b.fac.resize(nch);
  b.kk.resize(nch);
  b.bloch.resize(nch);
  b.xc2.assign(nch, 0.0);
  b.qk.assign(qk, qk + nch);
  for (int c = 0; c < nch; ++c) {
    const int l = lval[c];
    if (l < 0) return fail(HPRMAT_B200_ERR_ARG, "lval(%d) = %d < 0", c + 1, l);
    b.fac[c] = (double)l * (l + 1);
    b.kk[c] = 0.0;
    b.bloch[c] = 0.0;
    if (qk[c] > 0) {
      b.kk[c] = -qk[c] * qk[c];
      CoulombFG f = coulfg_single(qk[c] * rmax, eta[c], (double)l);
      if (f.ifail != 0) return fail(HPRMAT_B200_ERR_ARG, "COULFG failed (ifail=%d) for channel %d", f.ifail, c + 1);
      b.open_idx.push_back(c);
      b.co.push_back(make_double2(f.g, f.f));
      b.cop.push_back(make_double2(f.gp * qk[c] * rmax, f.fp * qk[c] * rmax));
    } else {
      if (qk[c] < 0) b.kk[c] = qk[c] * qk[c];
      double qk2 = -qk[c];
      WhitOut w = whit_l(eta[c], rmax, qk2, l);
      double xc1 = rmax * w.wd / w.w;
      b.bloch[c] = xc1 / rmax2;
      b.xc2[c] = w.w;
      b.closed_idx.push_back(c);
    }
  }
  b.nopen = (int)b.open_idx.size();
  return HPRMAT_B200_OK;
}

// ------------------------------------------------------------------ public API helpers
static int check_ctx(hprmat_b200_ctx* c) {
  if (!c) return fail(HPRMAT_B200_ERR_ARG, "null context");
  HPR_CUDA_TRY(cudaSetDevice(c->device));
  return HPRMAT_B200_OK;
}

using Clock = std::chrono::steady_clock;
static double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}


static int condest_fp64(hprmat_b200_ctx* c, const double2* W, const LUState& st, double* kappa);

// Start of a condition estimate: ||A||_1 of the matrix about to be factorised in FP64.
static int anorm_begin(hprmat_b200_ctx* c, const double2* A, long lda, int N) {
  unsigned long long* d = reinterpret_cast<unsigned long long*>(c->status.as<int>() + kAnormSlot);
  HPR_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream));
  colabs_max_kernel<<<N, 256, 0, c->stream>>>(A, lda, N, d);
  LAUNCH_CHECK();
  return HPRMAT_B200_OK;
}

// Pivot growth of the last factorisation: the largest |re| + |im| of U (accumulated by the
// panel and U12 kernels into the status block) over that of the matrix (kAmaxSlot), both from
// the copy factor made.  0 for a zero matrix.
static int pivot_growth(hprmat_b200_ctx* c, double* rho) {
  const double am = mag_hi_value((unsigned)c->h_status[kAmaxSlot]);
  const double g = mag_hi_value((unsigned)c->h_status[SW_COUNT - 1]);
  *rho = am > 0.0 ? g / am : 0.0;
  return HPRMAT_B200_OK;
}

// One interval (0-based is) of an rmatrix call: C(E) of the interval assembled on the device
// (src/rmatrix_hp.F90:246-293), factorised, and solved for its md.nq1 + nch surface right-hand
// sides into X64 (ld ldx): FP64 LU and one solve, or the mixed LU with FP64 refinement.
// d_cpot points at the interval's first mesh row.  Statistics of the interval in *stats.
// With a non-local potential (nl.p set) C(E) has dense channel blocks: the refinement's FP64
// operator is then a dense copy of C (A64) with a dense right-hand side (B64).
// reuse: keep the held mixed factorisation (opts.reuse_factors) as the refinement's
// preconditioner instead of assembling and factorising C(E); up to 8 refinement cycles.
static int interval_solve(hprmat_b200_ctx* c, int is, int nch, const ChannelData& chd, const MeshDev& md,
                          const double2* d_cpot, int ncp1, int ndim, double2* X64, long ld,
                          hprmat_b200_stats* stats, const NonLocalDev& nl, bool reuse = false) {
  const int nr = md.nr;
  const int N = nch * nr;
  const int nrhs = md.nq1 + nch;
  const bool mixed = c->opts.precision == HPRMAT_B200_PREC_MIXED;
  Operator op;
  op.structured = nl.p == nullptr;
  op.mesh = md;
  op.ch = chd;
  op.nch = nch;
  op.N = N;
  TRY(c->vt.ensure((size_t)nr * nch * nch * sizeof(double2)));
  {
    const long tot = (long)nr * nch * nch;
    cpot_transpose_kernel<<<cdiv_u(tot, 256), 256, 0, c->stream>>>(d_cpot, ncp1, ndim, nr, nch, c->vt.as<double2>());
    LAUNCH_CHECK();
  }
  op.vt = c->vt.as<double2>();
  op.q2 = md.q2;
  op.q1 = md.q1;
  op.nr = nr;
  // |B|_F of [blockdiag(q1) | blockdiag(q2)]
  double qn = 0.0;
  for (int i = 0; i < nr; ++i) {
    const double v2 = c->q2[(size_t)is * nr + i], v1 = c->q1[(size_t)is * nr + i];
    qn += v2 * v2 + (md.nq1 > 0 ? v1 * v1 : 0.0);
  }
  const double bnorm = sqrt(qn * nch);
  LUState st;
  int status = HPRMAT_B200_OK;
  dim3 ga(cdiv_u(N, 256), std::min(N, 512));  // assemble_kernel strides over the columns
  dim3 gr(cdiv_u(N, 256), nrhs);
  double* d_fro2 = reinterpret_cast<double*>(c->status.as<int>() + 32);
  unsigned* d_amax = reinterpret_cast<unsigned*>(c->status.as<int>() + kAmaxSlot);
  HPR_CUDA_TRY(cudaMemsetAsync(d_fro2, 0, sizeof(double), c->stream));
  HPR_CUDA_TRY(cudaMemsetAsync(d_amax, 0, sizeof(unsigned), c->stream));
  if (!op.structured) {
    TRY(c->A64.ensure((size_t)ld * N * sizeof(double2)));
    TRY(c->B64.ensure((size_t)ld * nrhs * sizeof(double2)));
    assemble_kernel<double2><<<ga, 256, 0, c->stream>>>(md, chd, nch, d_cpot, ncp1, ndim, c->A64.as<double2>(), ld,
                                                        N, d_fro2, nl);
    LAUNCH_CHECK();
    surface_rhs_kernel<double2><<<gr, 256, 0, c->stream>>>(md, c->B64.as<double2>(), ld, N, 1.0);
    LAUNCH_CHECK();
    op.A = c->A64.as<double2>();
    op.lda = ld;
    op.B = c->B64.as<double2>();
    op.ldb = ld;
    HPR_CUDA_TRY(cudaMemsetAsync(d_fro2, 0, sizeof(double), c->stream));
  }
  if (mixed) {
    TRY(c->W.ensure((size_t)ld * N * sizeof(float2)));
    float2* W = c->W.as<float2>();
    if (reuse) {
      st.N = c->held_N;
      st.ld = c->held_ld;
      st.nb = c->held_nb;
      st.nsteps = c->held_nsteps;
    } else {
      {
        NvtxRange nv("hprmat.assemble");
        assemble_kernel<float2><<<ga, 256, 0, c->stream>>>(md, chd, nch, d_cpot, ncp1, ndim, W, ld, N, d_fro2, nl,
                                                           d_amax);
        LAUNCH_CHECK();
      }
      int nb = pick_nb(c, N, sizeof(float2), 128);
      if (!nb) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "N = %d too large for the panel kernel", N);
      auto t1 = Clock::now();
      TRY(factor<float2>(c, W, ld, N, true, nb, st));
      stats->ms_factor = ms_since(t1);
      stats->factorizations += 1;
      c->held_N = st.N;
      c->held_ld = st.ld;
      c->held_nb = st.nb;
      c->held_nsteps = st.nsteps;
      // FP32 factors with a large pivot growth (or an exact zero FP32 pivot) cannot carry the
      // refinement: factorise C(E) in FP64 instead (the reference's Type 2 falls back to ZGESV
      // on CGETRF info != 0, src/rmat_solvers.F90:233-236)
      TRY(pivot_growth(c, &stats->pivot_growth));
      if (c->h_status[SW_INFO] != 0 || !(stats->pivot_growth <= c->growth_limit)) {
        if (c->h_status[SW_INFO] == 0 && c->opts.growth_error)
          return fail(HPRMAT_B200_PIVOT_GROWTH, "C(E) of interval %d: pivot growth %.3g of the FP32 factors above %.3g",
                      is + 1, stats->pivot_growth, c->growth_limit);
        stats->fp64_fallback = 1;
        HPR_CUDA_TRY(cudaMemsetAsync(d_amax, 0, sizeof(unsigned), c->stream));
      }
    }
    if (!stats->fp64_fallback) {
      auto t2 = Clock::now();
      TRY(c->X.ensure((size_t)ld * nrhs * sizeof(float2)));
      float2* X32 = c->X.as<float2>();
      surface_rhs_kernel<float2><<<gr, 256, 0, c->stream>>>(md, X32, ld, N, 1.0);
      LAUNCH_CHECK();
      if (c->zero_start) {
        HPR_CUDA_TRY(cudaMemsetAsync(X64, 0, (size_t)ld * nrhs * sizeof(double2), c->stream));
      } else {
        TRY(lu_solve_tc(c, st, X32, ld, nrhs));
        f2d_kernel<<<gr, 256, 0, c->stream>>>(X32, ld, X64, ld, N, nullptr);
        LAUNCH_CHECK();
      }
      stats->ms_solve = ms_since(t2);
      auto t3 = Clock::now();
      status = refine_mixed(c, op, W, st, X64, ld, nrhs, bnorm, 0.0, stats, reuse ? 8 : -1, reuse);
      if (status != HPRMAT_B200_OK && status != HPRMAT_B200_NOT_CONVERGED) return status;
      stats->ms_refine = ms_since(t3);
    }
  }
  if (!mixed || stats->fp64_fallback) {
    TRY(c->W.ensure((size_t)ld * N * sizeof(double2)));
    double2* W = c->W.as<double2>();
    {
      NvtxRange nv("hprmat.assemble");
      assemble_kernel<double2><<<ga, 256, 0, c->stream>>>(md, chd, nch, d_cpot, ncp1, ndim, W, ld, N, d_fro2, nl,
                                                          d_amax);
      LAUNCH_CHECK();
    }
    surface_rhs_kernel<double2><<<gr, 256, 0, c->stream>>>(md, X64, ld, N, 1.0);
    LAUNCH_CHECK();
    int nb = pick_nb(c, N, sizeof(double2), 64);
    if (!nb) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "N = %d too large for the panel kernel", N);
    if (c->opts.estimate_condition) TRY(anorm_begin(c, W, ld, N));
    auto t1 = Clock::now();
    TRY(factor<double2>(c, W, ld, N, false, nb, st));
    stats->factorizations += 1;
    TRY(pivot_growth(c, &stats->pivot_growth));
    c->f64_N = st.N;
    c->f64_ld = st.ld;
    c->f64_nb = st.nb;
    c->f64_nsteps = st.nsteps;
    stats->ms_factor = ms_since(t1);
    auto t2 = Clock::now();
    TRY(lu_solve<double2>(c, W, st, X64, ld, nrhs));
    TRY(c->R64.ensure((size_t)ld * nrhs * sizeof(double2)));
    TRY(apply_residual(c, op, X64, ld, nrhs, c->R64.as<double2>(), ld, true));
    double rn;
    TRY(frob_norm(c, c->R64.as<double2>(), ld, N, nrhs, &rn));
    stats->surface_change = -1.0;
    stats->rel_residual = rn / bnorm;
    stats->residual_history[0] = rn / bnorm;
    stats->ms_solve = ms_since(t2);
    if (c->opts.estimate_condition && c->h_status[SW_INFO] == 0) {
      auto t4 = Clock::now();
      TRY(condest_fp64(c, W, st, &stats->cond_estimate));
      stats->ms_condest = ms_since(t4);
    }
  }
  stats->nb = st.nb;
  if ((!reuse || stats->fp64_fallback) && c->h_status[SW_INFO] != 0) {
    stats->info = c->h_status[SW_INFO];
    return fail(HPRMAT_B200_SINGULAR, "C(E) of interval %d is singular: zero pivot in column %d", is + 1,
                c->h_status[SW_INFO]);
  }
  return status;
}

// rmatrix (src/rmatrix_hp.F90:175-368) on the device.  One interval: R = q2^T C^-1 q2 / a.
// ns > 1 intervals (R-matrix propagation, :326-345 and :590-632): interval 1 gives
// R11 / rmax0; every later interval is solved for [blockdiag(q1) | blockdiag(q2)] on the same
// factors (the reference's second FP64 solve with 2 nch right-hand sides, done here at the
// context's precision with the same refinement) and its projections R00 = q1^T X_1,
// R01 = q1^T X_2, R11 = q2^T X_2 update the propagated R (propagate_kernel).
// Wave functions requested from rmatrix_core (the twf arguments of rmatrix): nc entrance
// channels nvc (host, 1-based indices among the open channels) and the device array cf,
// complex (nwf1, nwf2, nc).
struct WfRequest {
  int nc = 0;
  const int* nvc = nullptr;
  double2* d_cf = nullptr;
  long nwf1 = 0, nwf2 = 0;
};

static int rmatrix_core(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                        double rmax, int nr, int ns, const double2* d_cpot, int ncp1, int ndim, double2* d_cu,
                        int* nopen, hprmat_b200_stats* stats, const WfRequest* wf = nullptr,
                        const double2* d_cpnl = nullptr, int ncp2 = 0) {
  auto t_all = Clock::now();
  if (d_cpnl && (ns != 1 || ncp2 < nr * nr))
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix: non-local potentials need ns = 1 and ncp2 >= nr*nr");
  if (nch <= 0 || nr <= 0 || ns <= 0 || !lval || !qk || !eta || !d_cpot || !d_cu || !nopen)
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix: invalid arguments");
  if (wf && (wf->nc <= 0 || !wf->nvc || !wf->d_cf || wf->nwf1 < (long)nr * ns || wf->nwf2 < nch || wf->nc > ndim))
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix: wave functions need nc >= 1, nvc, cf with nwf1 >= nr*ns, "
                                     "nwf2 >= nch and nc <= ndim");
  if (ndim < nch || ncp1 < nr * ns) return fail(HPRMAT_B200_ERR_ARG, "rmatrix: ndim < nch or ncp1 < nr*ns");
  if (c->nr != nr || c->ns != ns || c->rmax != rmax)
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix: call rmat_ini(nr=%d, ns=%d, rmax=%g) first", nr, ns, rmax);
  const long Nl = (long)nch * nr;
  if (Nl > 200000) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "rmatrix: N = %ld too large", Nl);
  const int N = (int)Nl;
  const double rmax0 = rmax / ns;
  Boundary bnd;
  TRY(boundary_values(nch, lval, qk, eta, rmax, rmax0, bnd));
  *nopen = bnd.nopen;
  const int ncl = (int)bnd.closed_idx.size();
  const int nc = wf ? wf->nc : 0;
  if (wf)
    for (int ic = 0; ic < nc; ++ic)
      if (wf->nvc[ic] < 1 || wf->nvc[ic] > bnd.nopen)
        return fail(HPRMAT_B200_ERR_ARG, "rmatrix: entrance channel nvc(%d) = %d is not an open channel (nopen = %d)",
                    ic + 1, wf->nvc[ic], bnd.nopen);
  // channel data: fac | kk | bloch | qk | xc2 (doubles, padded to an even count so that the
  // double2 arrays after them stay 16-byte aligned), then co | cop (double2), then
  // open_idx | closed_idx | nvc - 1 (ints)
  const size_t nd = (5 * (size_t)nch + 1) / 2 * 2;
  const size_t bytes = nd * sizeof(double) + 2 * (size_t)std::max(1, bnd.nopen) * sizeof(double2) +
                       ((size_t)std::max(1, bnd.nopen) + std::max(1, ncl) + std::max(1, nc)) * sizeof(int) + 64;
  TRY(c->chan.ensure(bytes));
  std::vector<unsigned char> h(bytes, 0);
  double* hd = reinterpret_cast<double*>(h.data());
  std::copy(bnd.fac.begin(), bnd.fac.end(), hd);
  std::copy(bnd.kk.begin(), bnd.kk.end(), hd + nch);
  std::copy(bnd.bloch.begin(), bnd.bloch.end(), hd + 2 * nch);
  std::copy(bnd.qk.begin(), bnd.qk.end(), hd + 3 * nch);
  std::copy(bnd.xc2.begin(), bnd.xc2.end(), hd + 4 * nch);
  double2* hz = reinterpret_cast<double2*>(hd + nd);
  std::copy(bnd.co.begin(), bnd.co.end(), hz);
  std::copy(bnd.cop.begin(), bnd.cop.end(), hz + std::max(1, bnd.nopen));
  int* hi = reinterpret_cast<int*>(hz + 2 * std::max(1, bnd.nopen));
  std::copy(bnd.open_idx.begin(), bnd.open_idx.end(), hi);
  std::copy(bnd.closed_idx.begin(), bnd.closed_idx.end(), hi + std::max(1, bnd.nopen));
  for (int ic = 0; ic < nc; ++ic) hi[std::max(1, bnd.nopen) + std::max(1, ncl) + ic] = wf->nvc[ic] - 1;
  HPR_CUDA_TRY(cudaMemcpyAsync(c->chan.p, h.data(), bytes, cudaMemcpyHostToDevice, c->stream));
  const double* dd = c->chan.as<double>();
  ChannelData chd{dd, dd + nch, dd + 2 * nch};
  const double* d_qk = dd + 3 * nch;
  const double* d_xc2 = dd + 4 * nch;
  const double2* d_co = reinterpret_cast<const double2*>(dd + nd);
  const double2* d_cop = d_co + std::max(1, bnd.nopen);
  const int* d_open = reinterpret_cast<const int*>(d_cop + std::max(1, bnd.nopen));
  const int* d_closed = d_open + std::max(1, bnd.nopen);
  const int* d_nvc = d_closed + std::max(1, ncl);

  const long ld = (N + 3) / 4 * 4;
  const int nrhs_max = ns > 1 ? 2 * nch : nch;
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->n = N;
    stats->nrhs = nrhs_max;
    stats->rel_residual = -1.0;
    stats->surface_change = -1.0;
  }
  TRY(c->X64.ensure((size_t)ld * nrhs_max * sizeof(double2)));
  double2* X64 = c->X64.as<double2>();
  const int no = bnd.nopen;
  const size_t nn = (size_t)nch * nch;
  // R | R01 | R11 | propagated R (nch^2 each); work: 2 max(nopen^2, nch^2)
  TRY(c->rmat.ensure(4 * nn * sizeof(double2) + 64));
  TRY(c->zwork.ensure((size_t)2 * std::max<size_t>(1, std::max<size_t>((size_t)no * no, ns > 1 ? nn : 0)) *
                          sizeof(double2) + 64));
  double2* R = c->rmat.as<double2>();
  double2* R01 = R + nn;
  double2* R11 = R + 2 * nn;
  double2* rp = R + 3 * nn;
  double2* zo = c->zwork.as<double2>();
  int* d_info = c->status.as<int>() + SW_INFO;
  // with wave functions every interval keeps its solutions (slot is, ld x nrhs_max) and its
  // propagation matrix (R00 + rmax1 R)^-1 R01 (slot is, nch^2)
  const size_t xslot = (size_t)ld * nrhs_max;
  if (wf) {
    TRY(c->wfx.ensure((size_t)ns * xslot * sizeof(double2)));
    TRY(c->wfz.ensure((size_t)ns * nn * sizeof(double2)));
    TRY(c->wfc.ensure((size_t)nch * (ns + 1) * nc * sizeof(double2)));
  }
  // factor reuse (opts.reuse_factors): the held factorisation must be of this channel block
  const bool mixed = c->opts.precision == HPRMAT_B200_PREC_MIXED;
  const bool keyed = c->opts.reuse_factors && mixed && ns == 1 && !d_cpnl;
  unsigned long long fp = 0;
  if (keyed) {
    TRY(c->fpbuf.ensure(sizeof(unsigned long long)));
    HPR_CUDA_TRY(cudaMemsetAsync(c->fpbuf.p, 0, sizeof(unsigned long long), c->stream));
    const long tot = (long)nr * nch * nch;
    fingerprint_kernel<<<std::min<unsigned>(cdiv_u(tot, 256), 592), 256, 0, c->stream>>>(
        d_cpot, ncp1, ndim, nr, nch, c->fpbuf.as<unsigned long long>());
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaMemcpyAsync(&fp, c->fpbuf.p, sizeof(fp), cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  const bool try_reuse = keyed && c->lu_held && c->held_N == N && c->held_nch == nch && c->held_nr == nr &&
                         c->held_rmax == rmax && c->held_fp == fp && c->held_last_inner <= c->reuse_max_inner &&
                         std::equal(lval, lval + nch, c->held_lval.begin(), c->held_lval.end());
  int status = HPRMAT_B200_OK;
  for (int is = 0; is < ns; ++is) {
    const MeshDev md = mesh_dev(c, is, is > 0 ? nch : 0);
    if (wf) X64 = c->wfx.as<double2>() + (size_t)is * xslot;
    hprmat_b200_stats si;
    memset(&si, 0, sizeof(si));
    si.rel_residual = -1.0;
    si.surface_change = -1.0;
    NonLocalDev nl;
    if (d_cpnl) {
      nl.p = d_cpnl;
      nl.ncp2 = ncp2;
      nl.ndim = ndim;
      nl.wle = mesh_wle(c);
      nl.rmax0 = rmax0;
    }
    int s = interval_solve(c, is, nch, chd, md, d_cpot + (size_t)is * nr, ncp1, ndim, X64, ld, &si, nl, try_reuse);
    if (try_reuse && s == HPRMAT_B200_NOT_CONVERGED) {
      // the held factors were too far from C(E) for the refinement: factorise C(E)
      hprmat_b200_stats s2;
      memset(&s2, 0, sizeof(s2));
      s2.rel_residual = -1.0;
      s2.surface_change = -1.0;
      s = interval_solve(c, is, nch, chd, md, d_cpot + (size_t)is * nr, ncp1, ndim, X64, ld, &s2, nl, false);
      s2.refine_steps += si.refine_steps;
      s2.inner_iterations += si.inner_iterations;
      s2.ms_solve += si.ms_solve;
      s2.ms_refine += si.ms_refine;
      si = s2;
    }
    if (keyed && (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED))
      c->held_last_inner = si.factorizations > 0 ? 0 : si.inner_iterations;
    if (keyed && (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) && si.factorizations > 0 &&
        !si.fp64_fallback) {
      c->lu_held = true;
      c->held_nch = nch;
      c->held_nr = nr;
      c->held_rmax = rmax;
      c->held_fp = fp;
      c->held_lval.assign(lval, lval + nch);
    }
    if (stats) {
      stats->info = si.info;
      stats->nb = si.nb;
      stats->factorizations += si.factorizations;
      stats->fp64_fallback |= si.fp64_fallback;
      stats->pivot_growth = std::max(stats->pivot_growth, si.pivot_growth);
      stats->cond_estimate = std::max(stats->cond_estimate, si.cond_estimate);
      stats->ms_condest += si.ms_condest;
      stats->refine_steps += si.refine_steps;
      stats->inner_iterations += si.inner_iterations;
      stats->ms_factor += si.ms_factor;
      stats->ms_solve += si.ms_solve;
      stats->ms_refine += si.ms_refine;
      if (si.rel_residual > stats->rel_residual) {  // the worst interval's refinement record
        stats->rel_residual = si.rel_residual;
        stats->surface_change = si.surface_change;
        stats->residual_floor = si.residual_floor;
        memcpy(stats->residual_history, si.residual_history, sizeof(si.residual_history));
        memcpy(stats->floor_history, si.floor_history, sizeof(si.floor_history));
      }
    }
    if (s != HPRMAT_B200_OK && s != HPRMAT_B200_NOT_CONVERGED) return s;
    if (s == HPRMAT_B200_NOT_CONVERGED) status = s;
    const dim3 ge(nch, cdiv_u(nch, 128));
    if (is == 0) {
      // ns = 1: R / a;  ns > 1: the first interval's R11 / rmax2 (rmax2 = rmax0)
      rmat_extract_kernel<<<ge, 128, 0, c->stream>>>(X64, ld, md.q2, nr, nch, nch, 1.0 / rmax0, ns > 1 ? rp : R);
      LAUNCH_CHECK();
      continue;
    }
    rmat_extract_kernel<<<ge, 128, 0, c->stream>>>(X64, ld, md.q1, nr, nch, nch, 1.0, R);  // R00
    LAUNCH_CHECK();
    rmat_extract_kernel<<<ge, 128, 0, c->stream>>>(X64 + (size_t)nch * ld, ld, md.q1, nr, nch, nch, 1.0, R01);
    LAUNCH_CHECK();
    rmat_extract_kernel<<<ge, 128, 0, c->stream>>>(X64 + (size_t)nch * ld, ld, md.q2, nr, nch, nch, 1.0, R11);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(int), c->stream));
    propagate_kernel<<<1, 1024, 0, c->stream>>>(R, R01, R11, rp, nch, is * rmax0, (is + 1) * rmax0, zo,
                                                wf ? c->wfz.as<double2>() + (size_t)is * nn : zo + nn, d_info);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaMemcpyAsync(c->h_status, c->status.p, SW_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->h_status[SW_INFO] != 0)
      return fail(HPRMAT_B200_SINGULAR, "singular R00 + rmax1 R in the propagation to interval %d", is + 1);
  }
  // U
  auto t4 = Clock::now();
  NvtxRange nv_u("hprmat.umatrix");
  HPR_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(int), c->stream));
  umatrix_kernel<<<1, 1024, 0, c->stream>>>(ns > 1 ? rp : R, nch, d_open, d_qk, d_co, d_cop, no, zo,
                                            zo + std::max(1, no * no), d_cu, ndim, d_info);
  LAUNCH_CHECK();
  HPR_CUDA_TRY(cudaMemcpyAsync(c->h_status, c->status.p, SW_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (c->h_status[SW_INFO] != 0) return fail(HPRMAT_B200_SINGULAR, "singular Z_O in the collision-matrix step");
  if (wf) {
    // surface amplitudes from U, carried inwards, then the wave function per interval
    double2* cfp = c->wfc.as<double2>();
    wf_surface_kernel<<<1, 256, 0, c->stream>>>(d_cu, ndim, d_open, no, d_qk, d_cop, d_nvc, nc, nch, ns, rmax, cfp);
    LAUNCH_CHECK();
    for (int is = ns - 1; is >= 1; --is) {  // 1-based interval is from interval is + 1
      wf_back_kernel<<<nc, 128, 0, c->stream>>>(c->wfz.as<double2>() + (size_t)is * nn, nch, ns, is, cfp);
      LAUNCH_CHECK();
    }
    const size_t smem = 2 * (size_t)nch * sizeof(double2);
    if (smem > 48 * 1024) TRY(set_smem(wf_assemble_kernel, smem));
    for (int is = 1; is <= ns; ++is) {
      wf_assemble_kernel<<<dim3(cdiv_u(N, 256), nc), 256, smem, c->stream>>>(
          c->wfx.as<double2>() + (size_t)(is - 1) * xslot, ld, is > 1 ? nch : 0, nch, nr, ns, is, cfp, wf->d_cf,
          wf->nwf1, wf->nwf2);
      LAUNCH_CHECK();
    }
    if (ncl > 0) {
      wf_closed_kernel<<<nc, 128, 0, c->stream>>>(wf->d_cf, wf->nwf1, wf->nwf2, nr, ns,
                                                   mesh_dev(c, ns - 1).q2, d_closed, ncl, d_xc2, no, d_cu, ndim);
      LAUNCH_CHECK();
    }
    wf_normalize_kernel<<<dim3(cdiv_u(nr * ns, 256), nch, nc), 256, 0, c->stream>>>(wf->d_cf, wf->nwf1, wf->nwf2, nr,
                                                                                    ns, mesh_wle(c), rmax0);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  if (stats) {
    stats->ms_umatrix = ms_since(t4);
    stats->ms_total = ms_since(t_all);
    stats->status = status;
  }
  return status;
}

// X <- C^-T X with the FP64 factors in W (adjoint.cuh for the step order).
static int lu_solve_trans(hprmat_b200_ctx* c, const double2* W, long ld, int N, int nb, int nsteps, double2* X,
                          long ldx, int nrhs) {
  const double2* inv = c->inv.as<double2>();
  const int* swb = c->swaps.as<int>();
  constexpr int kRowsPerSplit = 256;
  auto update = [&](int acol, int ncols, int r0, int r1, int k0) -> int {  // X_block -= A(r0:r1, blk)^T X(r0:r1)
    if (r1 <= r0) return HPRMAT_B200_OK;
    const int nsplit = (r1 - r0 + kRowsPerSplit - 1) / kRowsPerSplit;
    TRY(c->adj_part.ensure((size_t)nsplit * ncols * 128 * sizeof(double2)));
    for (int cb = 0; cb < nrhs; cb += 128) {
      const int nc = std::min(128, nrhs - cb);
      trans_partial_kernel<<<nsplit, 256, 0, c->stream>>>(W, ld, acol, ncols, X + (size_t)cb * ldx, ldx, nc, r0, r1,
                                                          kRowsPerSplit, c->adj_part.as<double2>());
      LAUNCH_CHECK();
      trans_reduce_kernel<<<cdiv_u(ncols * nc, 256), 256, 0, c->stream>>>(c->adj_part.as<double2>(), nsplit, ncols,
                                                                          nc, X + (size_t)cb * ldx, ldx, k0);
      LAUNCH_CHECK();
    }
    return HPRMAT_B200_OK;
  };
  for (int s = 0; s < nsteps; ++s) {
    const int k0 = s * nb, ncols = std::min(nb, N - k0);
    TRY(update(k0, ncols, 0, k0, k0));
    diag_trans_kernel<<<nrhs, 128, 0, c->stream>>>(inv + ((size_t)2 * s + 1) * nb * nb, nb, ncols, k0, X, ldx);
    LAUNCH_CHECK();
  }
  for (int s = nsteps - 1; s >= 0; --s) {
    const int k0 = s * nb, ncols = std::min(nb, N - k0);
    TRY(update(k0, ncols, k0 + ncols, N, k0));
    diag_trans_kernel<<<nrhs, 128, 0, c->stream>>>(inv + (size_t)2 * s * nb * nb, nb, ncols, k0, X, ldx);
    LAUNCH_CHECK();
    perm_inv_kernel<<<nrhs, 256, 0, c->stream>>>(swb + (size_t)s * kSwapStride, kMaxNB, k0, ncols, X, ldx);
    LAUNCH_CHECK();
  }
  c->launches += (size_t)nsteps * 5;
  return HPRMAT_B200_OK;
}

// 1-norm condition number of the matrix factorised in FP64 (factors W, st; ||A||_1 left in the
// status block by anorm_begin and copied to h_status by factor): ||A^-1||_1 by the Hager-Higham estimator (N. J. Higham, ACM
// TOMS 14 (1988) 381-396, the method of LAPACK's ZLACN2 behind ZGECON): x = 1/n; repeat
// y = A^-1 x, stop when ||y||_1 no longer grows, x = e_j with j = argmax |(A^-H sign(y))_j|,
// stop when j repeats (at most 5 passes); then the extra vector x_i = (-1)^i (1 + i/(n-1)),
// estimate 2 ||A^-1 x||_1 / (3n), against matrices that defeat the iteration.  Solves with A on
// the factors (lu_solve), with A^H as conj(A^-T conj v) (lu_solve_trans); one right-hand side
// each, vectors on the host.  *kappa = 0 when not available (block size above 64).
static int condest_fp64(hprmat_b200_ctx* c, const double2* W, const LUState& st, double* kappa) {
  NvtxRange nv("hprmat.condest");
  *kappa = 0.0;
  const int N = st.N;
  if (N <= 0 || st.nb > 64) return HPRMAT_B200_OK;
  double anorm;  // from the copy factor made of the status block
  memcpy(&anorm, c->h_status + kAnormSlot, sizeof(double));
  if (!(anorm > 0.0)) return HPRMAT_B200_OK;
  TRY(c->cond_v.ensure((size_t)st.ld * sizeof(double2)));
  double2* dv = c->cond_v.as<double2>();
  std::vector<double2> v(N);
  auto solve = [&](bool herm) -> int {
    if (herm)
      for (auto& z : v) z.y = -z.y;
    HPR_CUDA_TRY(cudaMemcpyAsync(dv, v.data(), (size_t)N * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    if (herm) {
      TRY(lu_solve_trans(c, W, st.ld, N, st.nb, st.nsteps, dv, st.ld, 1));
    } else {
      TRY(lu_solve<double2>(c, W, st, dv, st.ld, 1));
    }
    HPR_CUDA_TRY(cudaMemcpyAsync(v.data(), dv, (size_t)N * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (herm)
      for (auto& z : v) z.y = -z.y;
    return HPRMAT_B200_OK;
  };
  auto norm1 = [&]() {
    double t = 0.0;
    for (const auto& z : v) t += hypot(z.x, z.y);
    return t;
  };
  for (auto& z : v) z = mk(1.0 / N, 0.0);
  double est = 0.0;
  int jlast = -1;
  for (int pass = 0; pass < 5; ++pass) {
    TRY(solve(false));
    const double e = norm1();
    if (!std::isfinite(e) || (pass > 0 && e <= est)) break;
    est = e;
    for (auto& z : v) {
      const double m = hypot(z.x, z.y);
      z = m > 0.0 ? mk(z.x / m, z.y / m) : mk(1.0, 0.0);
    }
    TRY(solve(true));
    int j = 0;
    double best = -1.0;
    for (int i = 0; i < N; ++i) {
      const double m = hypot(v[i].x, v[i].y);
      if (m > best) {
        best = m;
        j = i;
      }
    }
    if (j == jlast) break;
    jlast = j;
    std::fill(v.begin(), v.end(), mk(0.0, 0.0));
    v[j] = mk(1.0, 0.0);
  }
  for (int i = 0; i < N; ++i)
    v[i] = mk((i & 1 ? -1.0 : 1.0) * (1.0 + (N > 1 ? (double)i / (N - 1) : 0.0)), 0.0);
  TRY(solve(false));
  est = std::max(est, 2.0 * norm1() / (3.0 * N));
  *kappa = anorm * est;
  return HPRMAT_B200_OK;
}

// Small dense complex solve on the host (partial pivoting): A (n x n, column-major) X = B
// (n x m); A and B are overwritten.  Returns false if A is singular.
static bool host_csolve(std::vector<double2>& A, std::vector<double2>& B, int n, int m) {
  auto at = [&](int i, int j) -> double2& { return A[(size_t)i + (size_t)j * n]; };
  auto bt = [&](int i, int j) -> double2& { return B[(size_t)i + (size_t)j * n]; };
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = -1.0;
    for (int i = k; i < n; ++i) {
      const double v = fabs(at(i, k).x) + fabs(at(i, k).y);
      if (v > best) { best = v; p = i; }
    }
    if (!(best > 0.0)) return false;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(at(k, j), at(p, j));
      for (int j = 0; j < m; ++j) std::swap(bt(k, j), bt(p, j));
    }
    const double2 inv = crecip(at(k, k));
    for (int i = k + 1; i < n; ++i) {
      const double2 l = cmul(at(i, k), inv);
      for (int j = k + 1; j < n; ++j) cfms(at(i, j), l, at(k, j));
      for (int j = 0; j < m; ++j) cfms(bt(i, j), l, bt(k, j));
    }
  }
  for (int j = 0; j < m; ++j)
    for (int i = n - 1; i >= 0; --i) {
      double2 v = bt(i, j);
      for (int k = i + 1; k < n; ++k) cfms(v, at(i, k), bt(k, j));
      bt(i, j) = cmul(v, crecip(at(i, i)));
    }
  return true;
}

// Dense solve A X = B with device operands (A read only, B overwritten with X).
// surf_q2 (device, nlag doubles) enables the surface-projection stopping rule when the
// right-hand sides are the channel-surface vectors blockdiag(q2) of an R-matrix problem.
static int solve_dense_core(hprmat_b200_ctx* c, const double2* dA, double2* dB, int n, int nrhs,
                            hprmat_b200_stats* stats, const double* surf_q2 = nullptr, int nlag = 0) {
  auto t_all = Clock::now();
  if (n <= 0 || nrhs <= 0 || !dA || !dB) return fail(HPRMAT_B200_ERR_ARG, "solve_linear: invalid arguments");
  const int N = n;
  const long ld = (N + 3) / 4 * 4;
  const bool mixed = c->opts.precision == HPRMAT_B200_PREC_MIXED;
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->n = N;
    stats->nrhs = nrhs;
    stats->rel_residual = -1.0;
  }
  LUState st;
  int status = HPRMAT_B200_OK;
  dim3 ga(cdiv_u(N, 256), N);
  dim3 gr(cdiv_u(N, 256), nrhs);
  bool fallback = false;
  if (mixed) {
    TRY(c->W.ensure((size_t)ld * N * sizeof(float2)));
    float2* W = c->W.as<float2>();
    unsigned* d_amax = reinterpret_cast<unsigned*>(c->status.as<int>() + kAmaxSlot);
    HPR_CUDA_TRY(cudaMemsetAsync(d_amax, 0, sizeof(unsigned), c->stream));
    d2f_matrix_kernel<<<ga, 256, 0, c->stream>>>(dA, N, W, ld, N, d_amax);
    LAUNCH_CHECK();
    int nb = pick_nb(c, N, sizeof(float2), 128);
    if (!nb) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "N = %d too large for the panel kernel", N);
    auto t1 = Clock::now();
    TRY(factor<float2>(c, W, ld, N, true, nb, st));
    if (stats) stats->ms_factor = ms_since(t1);
    double rho = 0.0;
    TRY(pivot_growth(c, &rho));
    if (stats) {
      stats->factorizations = 1;
      stats->pivot_growth = rho;
    }
    // an exact zero FP32 pivot or a pivot growth beyond what the FP32 factors can carry through
    // the refinement: factorise A in FP64 (Type 2's ZGESV fallback, src/rmat_solvers.F90:233-236)
    fallback = c->h_status[SW_INFO] != 0 || !(rho <= c->growth_limit);
    if (fallback && c->h_status[SW_INFO] == 0 && c->opts.growth_error)
      return fail(HPRMAT_B200_PIVOT_GROWTH, "pivot growth %.3g of the FP32 factors above %.3g", rho, c->growth_limit);
    if (stats) stats->fp64_fallback = fallback;
  }
  if (mixed && !fallback) {
    float2* W = c->W.as<float2>();
    auto t2 = Clock::now();
    TRY(c->X.ensure((size_t)ld * nrhs * sizeof(float2)));
    TRY(c->X64.ensure((size_t)ld * nrhs * sizeof(double2)));
    float2* X32 = c->X.as<float2>();
    double2* X64 = c->X64.as<double2>();
    d2f_kernel<<<gr, 256, 0, c->stream>>>(dB, N, X32, ld, N, nullptr);
    LAUNCH_CHECK();
    TRY(lu_solve_tc(c, st, X32, ld, nrhs));
    f2d_kernel<<<gr, 256, 0, c->stream>>>(X32, ld, X64, ld, N, nullptr);
    LAUNCH_CHECK();
    if (stats) stats->ms_solve = ms_since(t2);
    Operator op;
    op.structured = false;
    op.A = dA;
    op.lda = N;
    op.B = dB;
    op.ldb = N;
    op.N = N;
    op.q2 = surf_q2;
    op.nr = nlag;
    double bn;
    TRY(frob_norm(c, dB, N, N, nrhs, &bn));
    if (bn == 0.0) bn = 1.0;
    double* d_fro2 = reinterpret_cast<double*>(c->status.as<int>() + 32);
    HPR_CUDA_TRY(cudaMemsetAsync(d_fro2, 0, sizeof(double), c->stream));
    fro2_kernel<<<dim3(cdiv_u(N, 256), std::min(N, 512)), 256, 0, c->stream>>>(dA, N, N, d_fro2);
    LAUNCH_CHECK();
    double cn2;
    HPR_CUDA_TRY(cudaMemcpyAsync(&cn2, d_fro2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    auto t3 = Clock::now();
    status = refine_mixed(c, op, W, st, X64, ld, nrhs, bn, sqrt(cn2), stats);
    if (status != HPRMAT_B200_OK && status != HPRMAT_B200_NOT_CONVERGED) return status;
    copy_d_kernel<<<gr, 256, 0, c->stream>>>(X64, ld, dB, N, N);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (stats) stats->ms_refine = ms_since(t3);
  }
  if (!mixed || fallback) {
    TRY(c->W.ensure((size_t)ld * N * sizeof(double2)));
    double2* W = c->W.as<double2>();
    HPR_CUDA_TRY(cudaMemcpy2DAsync(W, ld * sizeof(double2), dA, (size_t)N * sizeof(double2),
                                   (size_t)N * sizeof(double2), N, cudaMemcpyDeviceToDevice, c->stream));
    if (stats && !fallback) {  // max |a_ij| for the reported pivot growth (the mixed path has it)
      unsigned* d_amax = reinterpret_cast<unsigned*>(c->status.as<int>() + kAmaxSlot);
      double* d_fro2 = reinterpret_cast<double*>(c->status.as<int>() + 32);
      HPR_CUDA_TRY(cudaMemsetAsync(d_amax, 0, sizeof(unsigned), c->stream));
      fro2_kernel<<<dim3(cdiv_u(N, 256), std::min(N, 512)), 256, 0, c->stream>>>(dA, N, N, d_fro2, d_amax);
      LAUNCH_CHECK();
    }
    int nb = pick_nb(c, N, sizeof(double2), 64);
    if (!nb) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "N = %d too large for the panel kernel", N);
    if (stats && c->opts.estimate_condition) TRY(anorm_begin(c, dA, N, N));
    auto t1 = Clock::now();
    TRY(factor<double2>(c, W, ld, N, false, nb, st));
    if (stats) stats->ms_factor = ms_since(t1);
    if (stats) {
      stats->factorizations += 1;
      TRY(pivot_growth(c, &stats->pivot_growth));
    }
    if (c->h_status[SW_INFO] != 0) {
      if (stats) stats->info = c->h_status[SW_INFO];
      return fail(HPRMAT_B200_SINGULAR, "matrix is singular: zero pivot in column %d", c->h_status[SW_INFO]);
    }
    auto t2 = Clock::now();
    TRY(c->X64.ensure((size_t)ld * nrhs * sizeof(double2)));
    double2* X = c->X64.as<double2>();
    copy_d_kernel<<<gr, 256, 0, c->stream>>>(dB, N, X, ld, N);
    LAUNCH_CHECK();
    TRY(lu_solve<double2>(c, W, st, X, ld, nrhs));
    copy_d_kernel<<<gr, 256, 0, c->stream>>>(X, ld, dB, N, N);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (stats) stats->ms_solve = ms_since(t2);
    if (stats && c->opts.estimate_condition) {
      auto t4 = Clock::now();
      TRY(condest_fp64(c, W, st, &stats->cond_estimate));
      stats->ms_condest = ms_since(t4);
    }
  }
  if (stats) {
    stats->nb = st.nb;
    stats->ms_total = ms_since(t_all);
    stats->status = status;
  }
  return status;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

void hprmat_b200_default_opts(hprmat_b200_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->precision = HPRMAT_B200_PREC_MIXED;
  o->max_refine = 3;
  o->tol = 1.0e-12;
  o->surface_tol = 1.0e-11;
  o->panel_nb = 0;
}

static int validate_opts(const hprmat_b200_opts* o) {
  if (o->precision != HPRMAT_B200_PREC_FP64 && o->precision != HPRMAT_B200_PREC_MIXED)
    return fail(HPRMAT_B200_ERR_ARG, "opts.precision must be 0 (FP64) or 1 (mixed)");
  if (o->max_refine < 0 || o->max_refine > 8) return fail(HPRMAT_B200_ERR_ARG, "opts.max_refine must be in 0..8");
  if (!(o->tol >= 0.0)) return fail(HPRMAT_B200_ERR_ARG, "opts.tol must be >= 0");
  if (!(o->surface_tol >= 0.0)) return fail(HPRMAT_B200_ERR_ARG, "opts.surface_tol must be >= 0");
  if (o->panel_nb != 0 && o->panel_nb != 16 && o->panel_nb != 32 && o->panel_nb != 64 && o->panel_nb != 128)
    return fail(HPRMAT_B200_ERR_ARG, "opts.panel_nb must be 0, 16, 32, 64 or 128");
  return HPRMAT_B200_OK;
}

int hprmat_b200_create(int device, const hprmat_b200_opts* opts, hprmat_b200_ctx** out) {
  if (!out) return fail(HPRMAT_B200_ERR_ARG, "null output pointer");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(HPRMAT_B200_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  if (device < 0 || device >= ndev) return fail(HPRMAT_B200_ERR_ARG, "device %d out of range", device);
  cudaDeviceProp prop;
  HPR_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(HPRMAT_B200_ERR_NODEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device,
                prop.major, prop.minor);
  hprmat_b200_opts o;
  hprmat_b200_default_opts(&o);
  if (opts) o = *opts;
  TRY(validate_opts(&o));
  auto* c = new hprmat_b200_ctx();
  c->device = device;
  c->opts = o;
  c->nsm = prop.multiProcessorCount;
  c->smem_optin = (int)prop.sharedMemPerBlockOptin;
  HPR_CUDA_TRY(cudaSetDevice(device));
  HPR_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->own_stream = true;
  HPR_CUDA_TRY(cudaMallocHost(&c->h_status, 64 * sizeof(int)));
  HPR_CUDA_TRY(cudaMallocHost(&c->h_norms, 4096 * sizeof(double)));
  int s = c->status.ensure(64 * sizeof(int));
  if (s != HPRMAT_B200_OK) {
    delete c;
    return s;
  }
  HPR_CUDA_TRY(cudaMemset(c->status.p, 0, 64 * sizeof(int)));
  s = tc_gemm_init(c->tcplan, device);
  if (s != HPRMAT_B200_OK) {
    delete c;
    return s;
  }
  *out = c;
  return HPRMAT_B200_OK;
}

int hprmat_b200_destroy(hprmat_b200_ctx* c) {
  if (!c) return HPRMAT_B200_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  DevBuf* bufs[] = {&c->mesh, &c->W, &c->A64, &c->X, &c->X64, &c->R64, &c->B64, &c->V, &c->Z, &c->gm,
                    &c->swaps, &c->ipiv, &c->stage, &c->status, &c->ops, &c->inv, &c->chan, &c->rmat,
                    &c->zwork, &c->cpot, &c->cu, &c->norms, &c->lup, &c->rop, &c->rsurf, &c->vt, &c->rlo, &c->linv,
                    &c->wfx, &c->wfz, &c->wfc, &c->wfcf, &c->fpbuf};
  for (DevBuf* b : bufs) b->release();
  for (hprmat_b200_ctx* w : c->scan_workers) hprmat_b200_destroy(w);
  c->scan_workers.clear();
  c->scan_cpot.clear();
  for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->h_norms) cudaFreeHost(c->h_norms);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return HPRMAT_B200_OK;
}

int hprmat_b200_set_opts(hprmat_b200_ctx* c, const hprmat_b200_opts* o) {
  if (!c || !o) return fail(HPRMAT_B200_ERR_ARG, "null argument");
  TRY(validate_opts(o));
  c->opts = *o;
  return HPRMAT_B200_OK;
}

int hprmat_b200_set_stream(hprmat_b200_ctx* c, void* stream) {
  TRY(check_ctx(c));
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (stream) {
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
  } else {
    HPR_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  return HPRMAT_B200_OK;
}

int hprmat_b200_rmat_ini(hprmat_b200_ctx* c, int nr, int ns, double rmax, double* zrma) {
  TRY(check_ctx(c));
  if (nr < 2 || ns < 1 || !(rmax > 0)) return fail(HPRMAT_B200_ERR_ARG, "rmat_ini: need nr >= 2, ns >= 1, rmax > 0");
  build_mesh(c, nr, ns, rmax);
  TRY(upload_mesh(c));
  if (zrma) std::copy(c->zrma.begin(), c->zrma.end(), zrma);
  return HPRMAT_B200_OK;
}

int hprmat_b200_rmatrix_device(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                               double rmax, int nr, int ns, const void* d_cpot, int ncp1, int ndim, void* d_cu,
                               int* nopen, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  int s = rmatrix_core(c, nch, lval, qk, eta, rmax, nr, ns, (const double2*)d_cpot, ncp1, ndim, (double2*)d_cu, nopen,
                       stats);
  if (stats) stats->status = s;
  return s;
}

int hprmat_b200_rmatrix(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                        double rmax, int nr, int ns, const double* cpot, int ncp1, int ndim, double* cu, int* nopen,
                        hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!cpot || !cu || ndim <= 0 || ncp1 <= 0) return fail(HPRMAT_B200_ERR_ARG, "rmatrix: invalid arguments");
  const size_t pbytes = (size_t)ncp1 * ndim * ndim * sizeof(double2);
  const size_t ubytes = (size_t)ndim * ndim * sizeof(double2);
  TRY(c->cpot.ensure(pbytes));
  TRY(c->cu.ensure(ubytes));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->cpot.p, cpot, pbytes, cudaMemcpyHostToDevice, c->stream));
  int s = rmatrix_core(c, nch, lval, qk, eta, rmax, nr, ns, c->cpot.as<double2>(), ncp1, ndim, c->cu.as<double2>(),
                       nopen, stats);
  if (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) {
    HPR_CUDA_TRY(cudaMemcpyAsync(cu, c->cu.p, ubytes, cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  if (stats) stats->status = s;
  return s;
}

int hprmat_b200_rmatrix_wf_device(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                                  double rmax, int nr, int ns, const void* d_cpot, int ncp1, int ndim, void* d_cu,
                                  int* nopen, int nc, const int* nvc, void* d_cf, int nwf1, int nwf2,
                                  hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  WfRequest wf;
  wf.nc = nc;
  wf.nvc = nvc;
  wf.d_cf = (double2*)d_cf;
  wf.nwf1 = nwf1;
  wf.nwf2 = nwf2;
  int s = rmatrix_core(c, nch, lval, qk, eta, rmax, nr, ns, (const double2*)d_cpot, ncp1, ndim, (double2*)d_cu, nopen,
                       stats, &wf);
  if (stats) stats->status = s;
  return s;
}

int hprmat_b200_rmatrix_wf(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                           double rmax, int nr, int ns, const double* cpot, int ncp1, int ndim, double* cu, int* nopen,
                           int nc, const int* nvc, double* cf, int nwf1, int nwf2, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!cpot || !cu || !cf || ndim <= 0 || ncp1 <= 0 || nc <= 0 || nwf1 <= 0 || nwf2 <= 0)
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix_wf: invalid arguments");
  const size_t pbytes = (size_t)ncp1 * ndim * ndim * sizeof(double2);
  const size_t ubytes = (size_t)ndim * ndim * sizeof(double2);
  const size_t fbytes = (size_t)nwf1 * nwf2 * nc * sizeof(double2);
  TRY(c->cpot.ensure(pbytes));
  TRY(c->cu.ensure(ubytes));
  TRY(c->wfcf.ensure(fbytes));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->cpot.p, cpot, pbytes, cudaMemcpyHostToDevice, c->stream));
  WfRequest wf;
  wf.nc = nc;
  wf.nvc = nvc;
  wf.d_cf = c->wfcf.as<double2>();
  wf.nwf1 = nwf1;
  wf.nwf2 = nwf2;
  int s = rmatrix_core(c, nch, lval, qk, eta, rmax, nr, ns, c->cpot.as<double2>(), ncp1, ndim, c->cu.as<double2>(),
                       nopen, stats, &wf);
  if (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) {
    HPR_CUDA_TRY(cudaMemcpyAsync(cu, c->cu.p, ubytes, cudaMemcpyDeviceToHost, c->stream));
    // only the written part of cf: rows 1..nr*ns of channels 1..nch per entrance channel
    const size_t pitch = (size_t)nwf1 * sizeof(double2);
    for (int ic = 0; ic < nc; ++ic) {
      const size_t off = (size_t)ic * nwf1 * nwf2;
      HPR_CUDA_TRY(cudaMemcpy2DAsync(reinterpret_cast<double2*>(cf) + off, pitch, c->wfcf.as<double2>() + off, pitch,
                                     (size_t)nr * ns * sizeof(double2), nch, cudaMemcpyDeviceToHost, c->stream));
    }
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  if (stats) stats->status = s;
  return s;
}

// Complex value i of a caller's interleaved complex array, read as two doubles: a Fortran
// complex*16 array need not be 16-byte aligned.
static inline double2 host_c(const double* p, size_t i) { return mk(p[2 * i], p[2 * i + 1]); }

int hprmat_b200_rmatrix_full(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                             double rmax, int nr, int ns, const double* cpot, int ncp1, int ndim, double* cu,
                             int* nopen, int twf, double* cf, int nwf1, int nwf2, int nc, const int* nvc, int ncp2,
                             const double* cpnl, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!cpot || !cu || ndim <= 0 || ncp1 <= 0 || (twf && (!cf || nc <= 0 || nwf1 <= 0 || nwf2 <= 0)) ||
      (ncp2 > 0 && !cpnl) || ncp2 < 0)
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix_full: invalid arguments");
  const size_t pbytes = (size_t)ncp1 * ndim * ndim * sizeof(double2);
  const size_t ubytes = (size_t)ndim * ndim * sizeof(double2);
  const size_t nlbytes = (size_t)ncp2 * ndim * ndim * sizeof(double2);
  const size_t fbytes = twf ? (size_t)nwf1 * nwf2 * nc * sizeof(double2) : 0;
  TRY(c->cpot.ensure(pbytes + nlbytes));
  TRY(c->cu.ensure(ubytes));
  if (twf) TRY(c->wfcf.ensure(fbytes));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->cpot.p, cpot, pbytes, cudaMemcpyHostToDevice, c->stream));
  const double2* d_cpnl = nullptr;
  if (ncp2 > 0) {
    d_cpnl = c->cpot.as<double2>() + (size_t)ncp1 * ndim * ndim;
    HPR_CUDA_TRY(cudaMemcpyAsync((void*)d_cpnl, cpnl, nlbytes, cudaMemcpyHostToDevice, c->stream));
  }
  WfRequest wf;
  if (twf) {
    wf.nc = nc;
    wf.nvc = nvc;
    wf.d_cf = c->wfcf.as<double2>();
    wf.nwf1 = nwf1;
    wf.nwf2 = nwf2;
  }
  int s = rmatrix_core(c, nch, lval, qk, eta, rmax, nr, ns, c->cpot.as<double2>(), ncp1, ndim, c->cu.as<double2>(),
                       nopen, stats, twf ? &wf : nullptr, d_cpnl, ncp2);
  if (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) {
    HPR_CUDA_TRY(cudaMemcpyAsync(cu, c->cu.p, ubytes, cudaMemcpyDeviceToHost, c->stream));
    if (twf) {
      const size_t pitch = (size_t)nwf1 * sizeof(double2);
      for (int ic = 0; ic < nc; ++ic) {
        const size_t off = (size_t)ic * nwf1 * nwf2;
        HPR_CUDA_TRY(cudaMemcpy2DAsync(reinterpret_cast<double2*>(cf) + off, pitch, c->wfcf.as<double2>() + off,
                                       pitch, (size_t)nr * ns * sizeof(double2), nch, cudaMemcpyDeviceToHost,
                                       c->stream));
      }
    }
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  if (stats) stats->status = s;
  return s;
}

// Natural cubic spline through (x, y), n >= 2: second derivatives y2 by the tridiagonal
// (Thomas) elimination of the spline's continuity equations with y2 = 0 at both ends.
static void natural_spline(const double* x, const double* y, int n, std::vector<double>& y2) {
  y2.assign(n, 0.0);
  std::vector<double> u(n, 0.0);
  for (int i = 1; i < n - 1; ++i) {
    const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    const double p = sig * y2[i - 1] + 2.0;
    y2[i] = (sig - 1.0) / p;
    const double d = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    u[i] = (6.0 * d / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
  }
  y2[n - 1] = 0.0;
  for (int k = n - 2; k >= 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
}

// The spline's value at r: bracketing interval by bisection (the end intervals continue
// beyond the first and last node), then the cubic in its local coordinates.
static double spline_at(const double* x, const double* y, const std::vector<double>& y2, int n, double r) {
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int k = (hi + lo) / 2;
    if (x[k] > r)
      hi = k;
    else
      lo = k;
  }
  const double h = x[hi] - x[lo];
  const double a = (x[hi] - r) / h, b = (r - x[lo]) / h;
  return a * y[lo] + b * y[hi] + ((a * a * a - a) * y2[lo] + (b * b * b - b) * y2[hi]) * h * h / 6.0;
}

int hprmat_b200_wf_print(int nch, const int* lval, const double* qk, const double* eta, double rmax, int nr, int ns,
                         const double* cu, int ndim, int nopen, const double* cf, int nwf1, int nwf2,
                         const double* zrma, int iv, int nom, int npoin, double h, double* cwftab) {
  if (nch <= 0 || !lval || !qk || !eta || !cu || !cf || !zrma || !cwftab || nr * ns < 2 || nwf1 < nr * ns ||
      nwf2 < nch || iv < 1 || iv > nch || nom < 1 || nom > nch || npoin < 0 || ndim < nch)
    return fail(HPRMAT_B200_ERR_ARG, "wf_print: invalid arguments");
  const int nsr = nr * ns;
  int nop = 0, nclo = nopen;
  for (int w = 0; w < iv; ++w) {
    if (qk[w] > 0) ++nop;
    if (qk[w] < 0) ++nclo;
  }
  const size_t f0 = (size_t)nwf1 * ((size_t)(iv - 1) + (size_t)nwf2 * (nom - 1));
  std::vector<double> fr(nsr), fi(nsr), y2r, y2i;
  for (int i = 0; i < nsr; ++i) {
    fr[i] = cf[2 * (f0 + i)];
    fi[i] = cf[2 * (f0 + i) + 1];
  }
  natural_spline(zrma, fr.data(), nsr, y2r);
  natural_spline(zrma, fi.data(), nsr, y2i);
  const int l = lval[iv - 1];
  auto put = [&](int i, double2 v) {
    cwftab[2 * i] = v.x;
    cwftab[2 * i + 1] = v.y;
  };
  for (int i = 1; i <= npoin; ++i) {
    const double r = i * h;
    if (r <= rmax) {
      put(i - 1, mk(spline_at(zrma, fr.data(), y2r, nsr, r), spline_at(zrma, fi.data(), y2i, nsr, r)));
    } else if (qk[iv - 1] > 0) {
      const CoulombFG fg = coulfg_single(qk[iv - 1] * r, eta[iv - 1], (double)l);
      if (fg.ifail != 0) return fail(HPRMAT_B200_ERR_ARG, "wf_print: COULFG failed (ifail=%d) at r = %g", fg.ifail, r);
      const double sc = sqrt(qk[nom - 1] / qk[iv - 1]);
      const double2 co = mk(fg.g * sc, fg.f * sc);
      double2 v = cmul(host_c(cu, (size_t)(nop - 1) + (size_t)(nom - 1) * ndim), co);
      v = mk(-v.x, -v.y);
      if (iv == nom) v = mk(v.x + co.x, v.y - co.y);
      put(i - 1, v);
    } else {
      const WhitOut w = whit_l(eta[iv - 1], r, -qk[iv - 1], l);
      const double2 a = host_c(cu, (size_t)(nclo - 1) + (size_t)(nom - 1) * ndim);
      put(i - 1, mk(a.x * w.w, a.y * w.w));
    }
  }
  return HPRMAT_B200_OK;
}

// Batched energy scan: every block's potential is copied once; (block, energy) units are
// taken largest first by worker contexts, one host thread and one stream each, so that the
// solves of different units overlap on the device.  Each unit is rmatrix_core as for one
// energy, with the autotuner's settings for its order when the table has them.
static int scan_check_blocks(int nblocks, const hprmat_b200_scan_block* blocks, double rmax, int nr, const char* who) {
  if (nblocks < 0 || (nblocks > 0 && !blocks) || nr <= 0 || !(rmax > 0.0))
    return fail(HPRMAT_B200_ERR_ARG, "%s: invalid arguments", who);
  for (int b = 0; b < nblocks; ++b) {
    const hprmat_b200_scan_block& B = blocks[b];
    if (B.nch <= 0 || B.nenergies < 0 || !B.lval || !B.cpot || B.ncp1 < nr || !B.cu || !B.nopen || !B.status ||
        (B.nenergies > 0 && (!B.qk || !B.eta)))
      return fail(HPRMAT_B200_ERR_ARG, "%s: invalid block %d", who, b);
  }
  return HPRMAT_B200_OK;
}

// The blocks' potentials on the device (c->scan_cpot), once per block.
static int scan_upload(hprmat_b200_ctx* c, int nblocks, const hprmat_b200_scan_block* blocks) {
  HPR_CUDA_TRY(cudaSetDevice(c->device));
  c->scan_cpot.clear();
  for (int b = 0; b < nblocks; ++b) {
    const hprmat_b200_scan_block& B = blocks[b];
    const size_t pbytes = (size_t)B.ncp1 * B.nch * B.nch * sizeof(double2);
    c->scan_cpot.emplace_back(new DevBuf());
    TRY(c->scan_cpot.back()->ensure(pbytes));
    HPR_CUDA_TRY(cudaMemcpyAsync(c->scan_cpot.back()->p, B.cpot, pbytes, cudaMemcpyHostToDevice, c->stream));
  }
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return HPRMAT_B200_OK;
}

// nworkers worker contexts with the context's options and settings and the scan's mesh.
static int scan_workers_ready(hprmat_b200_ctx* c, int nworkers, int nr, double rmax) {
  while ((int)c->scan_workers.size() < nworkers) {
    hprmat_b200_ctx* w = nullptr;
    TRY(hprmat_b200_create(c->device, &c->opts, &w));
    c->scan_workers.push_back(w);
  }
  std::vector<double> zrma((size_t)nr);
  for (int i = 0; i < nworkers; ++i) {
    hprmat_b200_ctx* w = c->scan_workers[i];
    w->opts = c->opts;
    w->wave_sb = c->wave_sb;
    w->wave_un = c->wave_un;
    w->panel_cluster = c->panel_cluster;
    w->panel_rpc_min = c->panel_rpc_min;
    w->gmres_m = c->gmres_m;
    w->tcplan.max_grid = c->tcplan.max_grid;
    w->reuse_max_inner = c->reuse_max_inner;
    w->lu_held = false;
    TRY(hprmat_b200_rmat_ini(w, nr, 1, rmax, zrma.data()));
  }
  return HPRMAT_B200_OK;
}

// Settings of a worker for one unit: the row t, or the context's own settings (t null).
static void scan_apply(hprmat_b200_ctx* w, const hprmat_b200_ctx* c, const ScanTune* t) {
  w->tcplan.max_grid = t ? t->tc_grid : c->tcplan.max_grid;
  w->opts.panel_nb = t ? t->nb : c->opts.panel_nb;
  w->panel_cluster = t ? t->cluster != 0 : c->panel_cluster;
  w->panel_rpc_min = t ? t->rpc_min : c->panel_rpc_min;
  w->wave_sb = t ? t->sb : c->wave_sb;
  w->gmres_m = t ? t->gmres_m : c->gmres_m;
}

static const ScanTune* scan_row(const hprmat_b200_ctx* c, long N) {
  for (const ScanTune& t : c->scan_tune)
    if (t.N == N) return &t;
  return nullptr;
}

// The block's energies in the scan's order (the first channel's signed k^2).
static std::vector<int> scan_energy_order(const hprmat_b200_scan_block& B) {
  std::vector<int> order(B.nenergies);
  for (int e = 0; e < B.nenergies; ++e) order[e] = e;
  auto key = [&](int e) {
    const double k = B.qk[(size_t)e * B.nch];
    return k > 0 ? k * k : -k * k;
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key(x) < key(y); });
  return order;
}

int hprmat_b200_rmatrix_scan(hprmat_b200_ctx* c, int nblocks, const hprmat_b200_scan_block* blocks, double rmax,
                             int nr, int nworkers, double* seconds) {
  TRY(check_ctx(c));
  TRY(scan_check_blocks(nblocks, blocks, rmax, nr, "rmatrix_scan"));
  auto t0 = Clock::now();
  // work items: runs of up to kChunk energies of one block in energy order, largest blocks
  // first; with opts.reuse_factors a worker keeps one factorisation across the run
  constexpr int kChunk = 32;
  struct Unit {
    int b;
    std::vector<int> es;
    long n;
  };
  std::vector<Unit> units;
  for (int b = 0; b < nblocks; ++b) {
    const hprmat_b200_scan_block& B = blocks[b];
    const std::vector<int> order = scan_energy_order(B);
    for (int e0 = 0; e0 < B.nenergies; e0 += kChunk) {
      Unit u{b, {}, (long)B.nch * nr};
      u.es.assign(order.begin() + e0, order.begin() + std::min(B.nenergies, e0 + kChunk));
      units.push_back(std::move(u));
    }
  }
  std::stable_sort(units.begin(), units.end(), [](const Unit& x, const Unit& y) { return x.n > y.n; });
  TRY(scan_upload(c, nblocks, blocks));
  if (nworkers <= 0) nworkers = 4;
  nworkers = std::max(1, std::min<int>(nworkers, (int)std::max<size_t>(units.size(), 1)));
  TRY(scan_workers_ready(c, nworkers, nr, rmax));
  std::atomic<size_t> next{0};
  std::atomic<int> first_error{0};
  std::mutex err_mu;
  std::string err_msg;
  auto work = [&](int wi) {
    hprmat_b200_ctx* w = c->scan_workers[wi];
    cudaSetDevice(w->device);
    for (;;) {
      const size_t k = next.fetch_add(1);
      if (k >= units.size()) break;
      const Unit& u = units[k];
      const hprmat_b200_scan_block& B = blocks[u.b];
      const size_t ubytes = (size_t)B.nch * B.nch * sizeof(double2);
      scan_apply(w, c, scan_row(c, u.n));
      for (const int e : u.es) {
        int s = w->cu.ensure(ubytes);
        int nopen = 0;
        if (s == HPRMAT_B200_OK)
          s = rmatrix_core(w, B.nch, B.lval, B.qk + (size_t)e * B.nch, B.eta + (size_t)e * B.nch, rmax, nr, 1,
                           c->scan_cpot[u.b]->as<double2>(), B.ncp1, B.nch, w->cu.as<double2>(), &nopen, nullptr);
        if (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) {
          double* dst = B.cu + (size_t)e * B.nch * B.nch * 2;
          if (cudaMemcpyAsync(dst, w->cu.p, ubytes, cudaMemcpyDeviceToHost, w->stream) != cudaSuccess ||
              cudaStreamSynchronize(w->stream) != cudaSuccess)
            s = HPRMAT_B200_ERR_CUDA;
        }
        B.nopen[e] = nopen;
        B.status[e] = s;
        if (s != HPRMAT_B200_OK) {
          int z = 0;
          if (first_error.compare_exchange_strong(z, s)) {
            std::lock_guard<std::mutex> lk(err_mu);
            err_msg = hprmat_b200_last_error();
          }
        }
      }
    }
  };
  std::vector<std::thread> threads;
  for (int i = 1; i < nworkers; ++i) threads.emplace_back(work, i);
  work(0);
  for (auto& t : threads) t.join();
  if (seconds) *seconds = std::chrono::duration<double>(Clock::now() - t0).count();
  const int fe = first_error.load();
  if (fe != HPRMAT_B200_OK && fe != HPRMAT_B200_NOT_CONVERGED) return fail(fe, "rmatrix_scan: %s", err_msg.c_str());
  return fe;
}

// ------------------------------------------------------------------ shifted (Hessenberg) scan
// Householder reduction of A (N x N, column-major, ld) to upper Hessenberg form in place,
// A = P H P^H, with P (ld) accumulated from the reflectors (kept in hU, column k: rows k+1 ..).
static int hess_reduce_blocked(hprmat_b200_ctx* c, double2* A, long ld, int N, double2* P);

static int hess_reduce_unblocked(hprmat_b200_ctx* c, double2* A, long ld, int N, double2* P) {
  NvtxRange nv("hprmat.hess.reduce");
  TRY(c->hU.ensure((size_t)ld * N * sizeof(double2)));
  const int nchunk_max = (N + kHessChunk - 1) / kHessChunk;
  TRY(c->hPart.ensure((size_t)nchunk_max * N * sizeof(double2)));
  double2* U = c->hU.as<double2>();
  for (int k = 0; k + 2 < N; ++k) {
    hess_reflector_kernel<<<1, kHessThreads, 0, c->stream>>>(A, ld, N, k, U, ld);
    LAUNCH_CHECK();
    const int ncol = N - k - 1;
    hess_left_kernel<<<cdiv_u((long)ncol * 32, kHessThreads), kHessThreads, 0, c->stream>>>(A, ld, N, k + 1, k + 1, U,
                                                                                          ld, k);
    LAUNCH_CHECK();
    const int nchunk = (ncol + kHessChunk - 1) / kHessChunk;
    const dim3 gr(cdiv_u(N, kHessThreads), nchunk);
    hess_right_partial_kernel<<<gr, kHessThreads, 0, c->stream>>>(A, ld, N, k, U, ld, c->hPart.as<double2>());
    LAUNCH_CHECK();
    hess_right_update_kernel<<<gr, kHessThreads, 0, c->stream>>>(A, ld, N, k, U, ld, c->hPart.as<double2>(), nchunk);
    LAUNCH_CHECK();
  }
  // P = H_0 H_1 ... accumulated backwards from the identity
  identity_kernel<<<dim3(cdiv_u(N, 256), N), 256, 0, c->stream>>>(P, ld, N);
  LAUNCH_CHECK();
  for (int k = N - 3; k >= 0; --k) {
    hess_left_kernel<<<cdiv_u((long)(N - k - 1) * 32, kHessThreads), kHessThreads, 0, c->stream>>>(P, ld, N, k + 1,
                                                                                                   k + 1, U, ld, k);
    LAUNCH_CHECK();
  }
  return HPRMAT_B200_OK;
}


static int hess_reduce(hprmat_b200_ctx* c, double2* A, long ld, int N, double2* P) {
  if (c->hess_blocked && N > kHbB + 2) return hess_reduce_blocked(c, A, ld, N, P);
  return hess_reduce_unblocked(c, A, ld, N, P);
}

// The same reduction in panels of kHbB columns (hessenberg.cuh, "blocked reduction"): per column
// one thread-block cluster brings the column up to date and forms its reflector, and a GEMV of
// the trailing matrix gives the column of Y; per panel three DMMA GEMMs update the trailing
// columns.  P is accumulated backwards from the identity, panel by panel, by two GEMMs each.
static int hess_reduce_blocked(hprmat_b200_ctx* c, double2* A, long ld, int N, double2* P) {
  NvtxRange nv("hprmat.hess.reduce_blocked");
  const int ncols = N - 2;  // columns 0 .. N-3 get a reflector
  const int np = (ncols + kHbB - 1) / kHbB;
  const int nchunk_max = (N + kHessChunk - 1) / kHessChunk;
  TRY(c->hU.ensure((size_t)ld * N * sizeof(double2)));
  TRY(c->hPart.ensure((size_t)nchunk_max * N * sizeof(double2)));
  TRY(c->hbY.ensure((size_t)N * kHbB * sizeof(double2)));
  TRY(c->hbT.ensure((size_t)np * kHbB * kHbB * sizeof(double2)));
  TRY(c->hbVH.ensure((size_t)kHbB * N * sizeof(double2)));
  TRY(c->hbVT.ensure((size_t)N * kHbB * sizeof(double2)));
  TRY(c->hbW.ensure((size_t)kHbB * N * sizeof(double2)));
  double2* V = c->hU.as<double2>();
  double2* Y = c->hbY.as<double2>();
  double2* VH = c->hbVH.as<double2>();
  double2* VT = c->hbVT.as<double2>();
  double2* W = c->hbW.as<double2>();
  TRY(c->hbS.ensure((size_t)kHbB * sizeof(double2)));
  double2* part = c->hPart.as<double2>();
  // the column step's cluster: 16 CTAs where the GPU holds such a cluster, else 8 (portable)
  if (c->hb_cluster == 0) {
    c->hb_cluster = 8;
    if (cudaFuncSetAttribute((const void*)hb_col_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
            cudaSuccess &&
        set_smem(hb_col_cluster_kernel, (size_t)cdiv_u(N, 16) * sizeof(double2)) == HPRMAT_B200_OK) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(16);
      cfg.blockDim = dim3(kHbCT);
      cfg.dynamicSmemBytes = (size_t)cdiv_u(N, 16) * sizeof(double2);
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 16;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, (const void*)hb_col_cluster_kernel, &cfg) == cudaSuccess && n >= 1)
        c->hb_cluster = 16;
    }
    cudaGetLastError();
  }
  const int Gc = c->hb_cluster;
  if (Gc > 8)
    HPR_CUDA_TRY(cudaFuncSetAttribute((const void*)hb_col_cluster_kernel,
                                      cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  const int rpc = cdiv_u(N, Gc);
  const size_t xsm = (size_t)rpc * sizeof(double2);
  if (xsm + 16384 > (size_t)c->smem_optin) return hess_reduce_unblocked(c, A, ld, N, P);
  TRY(set_smem(hb_col_cluster_kernel, xsm));
  HbColArgs ca{};
  ca.A = A;
  ca.lda = ld;
  ca.N = N;
  ca.rpc = rpc;
  ca.part = part;
  ca.Y = Y;
  ca.ldy = N;
  ca.V = V;
  ca.ldv = ld;
  ca.s = c->hbS.as<double2>();
  auto column_step = [&]() -> int {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(Gc);
    cfg.blockDim = dim3(kHbCT);
    cfg.dynamicSmemBytes = xsm;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = Gc;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, hb_col_cluster_kernel, ca);
    if (e != cudaSuccess)
      return fail(HPRMAT_B200_ERR_CUDA, "Hessenberg column step (%d CTAs of %d rows): %s", Gc, rpc,
                  cudaGetErrorString(e));
    ++c->launches;
    return HPRMAT_B200_OK;
  };
  auto gemm = [&](int M, int Nc, int K, const double2* Aop, long lda, const double2* Bop, long ldb, double2* Cop,
                  long ldc) -> int {
    if (zgemm_f64_update(M, Nc, K, Aop, lda, Bop, ldb, Cop, ldc, c->stream))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    ++c->launches;
    return HPRMAT_B200_OK;
  };
  // the short-wide products (M = panel width, K up to N) cut along K into slices that run side
  // by side, then summed into C
  auto gemm_splitk = [&](int M, int Nc, int K, const double2* Aop, long lda, const double2* Bop, long ldb,
                         double2* Cop, long ldc) -> int {
    const int S = std::max(1, std::min(16, K / 256));
    if (S == 1) return gemm(M, Nc, K, Aop, lda, Bop, ldb, Cop, ldc);
    const int Ks = K / S, tail = K - S * Ks;
    const int slices = S + (tail > 0 ? 1 : 0);
    const size_t slice = (size_t)ldc * Nc;
    TRY(c->hbTmp.ensure((size_t)slices * slice * sizeof(double2)));
    double2* tmp = c->hbTmp.as<double2>();
    HPR_CUDA_TRY(cudaMemsetAsync(tmp, 0, (size_t)slices * slice * sizeof(double2), c->stream));
    if (zgemm_f64_update_batched(M, Nc, Ks, Aop, lda, (long)Ks * lda, Bop, ldb, Ks, tmp, ldc, (long)slice, S,
                                 c->stream))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    if (tail > 0) TRY(gemm(M, Nc, tail, Aop + (size_t)S * Ks * lda, lda, Bop + (size_t)S * Ks, ldb, tmp + S * slice, ldc));
    splitk_sum_kernel<<<cdiv_u((long)M * Nc, 256), 256, 0, c->stream>>>(Cop, ldc, M, Nc, tmp, slices);
    LAUNCH_CHECK();
    return HPRMAT_B200_OK;
  };
  for (int p = 0; p < np; ++p) {
    const int k = p * kHbB, b = std::min(kHbB, ncols - k);
    double2* Tp = c->hbT.as<double2>() + (size_t)p * kHbB * kHbB;
    // per column: the column step (with y of the column before) on the cluster, then the GEMV
    ca.k = k;
    ca.T = Tp;
    ca.iy = -1;
    ca.ix = 0;
    ca.nchunk = 0;
    TRY(column_step());
    for (int i = 0; i < b; ++i) {
      const int col = k + i;
      const int nchunk = cdiv_u(N - col - 1, kHbGemvCols);
      hb_gemv_kernel<<<dim3(cdiv_u(N, 32), nchunk), 256, 0, c->stream>>>(A, ld, N, col, V + (size_t)col * ld, part);
      LAUNCH_CHECK();
      ca.iy = i;
      ca.ix = i + 1 < b ? i + 1 : -1;
      ca.nchunk = nchunk;
      TRY(column_step());
    }
    if (k + b < N) {
      const int nt = N - k - b;
      hb_prep_kernel<<<cdiv_u(N, 128), 128, 0, c->stream>>>(N, k, b, V, ld, Tp, VH, VT, true);
      LAUNCH_CHECK();
      // A[:, k+b ..] -= Y V[k+b .., ]^H
      TRY(gemm(N, nt, b, Y, N, VH + (size_t)(k + b) * kHbB, kHbB, A + (size_t)(k + b) * ld, ld));
      // W = -V[k+1 .., ]^H A[k+1 .., k+b ..];  A[k+1 .., k+b ..] -= (-V T^H) W
      HPR_CUDA_TRY(cudaMemsetAsync(W, 0, (size_t)kHbB * nt * sizeof(double2), c->stream));
      TRY(gemm_splitk(b, nt, N - k - 1, VH + (size_t)(k + 1) * kHbB, kHbB, A + (k + 1) + (size_t)(k + b) * ld, ld, W,
                      kHbB));
      TRY(gemm(N - k - 1, nt, b, VT + (k + 1), N, W, kHbB, A + (k + 1) + (size_t)(k + b) * ld, ld));
    }
  }
  // P = Q_0 Q_1 ... (Q_p = I - V_p T_p V_p^H), backwards from the identity on rows/columns k+1 ..
  identity_kernel<<<dim3(cdiv_u(N, 256), N), 256, 0, c->stream>>>(P, ld, N);
  LAUNCH_CHECK();
  for (int p = np - 1; p >= 0; --p) {
    const int k = p * kHbB, b = std::min(kHbB, ncols - k);
    const double2* Tp = c->hbT.as<double2>() + (size_t)p * kHbB * kHbB;
    const int m = N - k - 1;
    hb_prep_kernel<<<cdiv_u(N, 128), 128, 0, c->stream>>>(N, k, b, V, ld, Tp, VH, VT, false);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaMemsetAsync(W, 0, (size_t)kHbB * m * sizeof(double2), c->stream));
    TRY(gemm_splitk(b, m, m, VH + (size_t)(k + 1) * kHbB, kHbB, P + (k + 1) + (size_t)(k + 1) * ld, ld, W, kHbB));
    TRY(gemm(m, m, b, VT + (k + 1), N, W, kHbB, P + (k + 1) + (size_t)(k + 1) * ld, ld));
  }
  return HPRMAT_B200_OK;
}

// One J-pi block of hprmat_b200_rmatrix_scan_shifted (hessenberg.cuh for the algebra): C0 is
// reduced to Hessenberg form once, then the block's energies are solved in batches by O(N^2 nch)
// work each, refined in FP64 against the structured C(E).  Energies whose kinematics do not fit
// the shifted form (channels whose diagonal energy terms do not move together) or whose
// Hessenberg or Woodbury pivots vanish are listed in `fallback` for the LU path.  COULFG
// failures get their status as in rmatrix.
static int hess_scan_block(hprmat_b200_ctx* c, const double2* d_cpot, const hprmat_b200_scan_block& B, double rmax,
                           int nr, std::vector<int>& fallback, int* first_error, std::string* err_msg) {
  const int nch = B.nch, N = nch * nr;
  const long ld = N;
  auto note = [&](int s) {
    if (s != HPRMAT_B200_OK && *first_error == HPRMAT_B200_OK) {
      *first_error = s;
      *err_msg = hprmat_b200_last_error();
    }
  };
  // host: boundary values of every energy, the shifts and the Bloch factors
  std::vector<Boundary> bd(B.nenergies);
  std::vector<int> good;
  for (int e = 0; e < B.nenergies; ++e) {
    const int s = boundary_values(nch, B.lval, B.qk + (size_t)e * nch, B.eta + (size_t)e * nch, rmax, rmax, bd[e]);
    B.status[e] = s;
    B.nopen[e] = s == HPRMAT_B200_OK ? bd[e].nopen : 0;
    if (s == HPRMAT_B200_OK) good.push_back(e);
    else note(s);
  }
  if (good.empty()) return HPRMAT_B200_OK;
  const std::vector<double>& kref = bd[good[0]].kk;
  std::vector<int> units;
  std::vector<double> delta;
  for (const int e : good) {
    const double dl = bd[e].kk[0] - kref[0];
    bool ok = true;
    for (int ch = 0; ch < nch && ok; ++ch) {
      const double d = bd[e].kk[ch] - kref[ch];
      ok = fabs(d - dl) <= 1e-12 * std::max({1.0, fabs(bd[e].kk[ch]), fabs(kref[ch])});
    }
    if (ok) {
      units.push_back(e);
      delta.push_back(dl);
    } else {
      fallback.push_back(e);
    }
  }
  if (units.empty()) return HPRMAT_B200_OK;
  const MeshDev md = mesh_dev(c, 0, 0);
  // with profiling, every phase ends with a stream synchronisation and adds its host time
  auto tmark = Clock::now();
  auto phase = [&](int slot) -> int {
    if (!c->profile) return HPRMAT_B200_OK;
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->hess_ms[slot] += ms_since(tmark);
    tmark = Clock::now();
    return HPRMAT_B200_OK;
  };
  // C0 = C(E_ref) without the closed channels' Bloch terms
  {
    std::vector<double> h(3 * (size_t)nch, 0.0);
    std::copy(bd[good[0]].fac.begin(), bd[good[0]].fac.end(), h.begin());
    std::copy(kref.begin(), kref.end(), h.begin() + nch);
    TRY(c->hChan.ensure(h.size() * sizeof(double)));
    HPR_CUDA_TRY(cudaMemcpyAsync(c->hChan.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double* dh = c->hChan.as<double>();
    ChannelData chd0{dh, dh + nch, dh + 2 * nch};
    TRY(c->hA.ensure((size_t)ld * N * sizeof(double2)));
    double* d_fro2 = reinterpret_cast<double*>(c->status.as<int>() + 32);
    NvtxRange nv("hprmat.hess.assemble");
    assemble_kernel<double2><<<dim3(cdiv_u(N, 256), std::min(N, 512)), 256, 0, c->stream>>>(
        md, chd0, nch, d_cpot, B.ncp1, nch, c->hA.as<double2>(), ld, N, d_fro2);
    LAUNCH_CHECK();
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));  // h outlives its copy
  }
  double2* A = c->hA.as<double2>();
  {
    TRY(c->hP.ensure((size_t)ld * N * sizeof(double2)));
    double2* P = c->hP.as<double2>();
    TRY(hess_reduce(c, A, ld, N, P));
    TRY(c->hHr.ensure((size_t)ld * N * sizeof(double2)));
    TRY(c->hPH.ensure((size_t)ld * N * sizeof(double2)));
    const dim3 gt(cdiv_u(N, 32), cdiv_u(N, 32)), bt(32, 8);
    hess_transpose_kernel<<<gt, bt, 0, c->stream>>>(A, ld, N, c->hHr.as<double2>(), ld, false, true);
    LAUNCH_CHECK();
    hess_transpose_kernel<<<gt, bt, 0, c->stream>>>(P, ld, N, c->hPH.as<double2>(), ld, true, false);
    LAUNCH_CHECK();
    TRY(c->hW.ensure((size_t)ld * nch * sizeof(double2)));
    TRY(c->hWH.ensure((size_t)nch * N * sizeof(double2)));
    hess_wq_kernel<<<dim3(cdiv_u(N, 256), nch), 256, 0, c->stream>>>(c->hPH.as<double2>(), ld, N, nr, md.q2,
                                                                     c->hW.as<double2>(), ld);
    LAUNCH_CHECK();
    hess_whq_kernel<<<dim3(cdiv_u(N, 256), nch), 256, 0, c->stream>>>(P, ld, N, nr, md.q2, c->hWH.as<double2>(),
                                                                      nch);
    LAUNCH_CHECK();
  }
  TRY(phase(0));
  // the potential per mesh point for the structured residual
  TRY(c->vt.ensure((size_t)nr * nch * nch * sizeof(double2)));
  {
    const long tot = (long)nr * nch * nch;
    cpot_transpose_kernel<<<cdiv_u(tot, 256), 256, 0, c->stream>>>(d_cpot, B.ncp1, nch, nr, nch, c->vt.as<double2>());
    LAUNCH_CHECK();
  }
  // batches of energies
  const size_t nn = (size_t)nch * nch;
  const size_t per_unit = (size_t)ld * N * sizeof(double2) + (size_t)N * (sizeof(double2) + sizeof(int)) +
                          5 * (size_t)ld * nch * sizeof(double2) + 6 * nn * sizeof(double2) + 4096;
  const int nb = (int)std::max<size_t>(1, std::min<size_t>(units.size(), (size_t)(c->hess_budget_gb * 1e9) / per_unit));
  TRY(c->hUe.ensure((size_t)nb * ld * N * sizeof(double2)));
  TRY(c->hLm.ensure((size_t)nb * N * sizeof(double2)));
  TRY(c->hSw.ensure((size_t)nb * N * sizeof(int)));
  for (DevBuf* b : {&c->hY, &c->hX, &c->hR, &c->hYr, &c->hYT}) TRY(b->ensure((size_t)nb * ld * nch * sizeof(double2)));
  for (DevBuf* b : {&c->hS, &c->hT, &c->hRacc, &c->hG, &c->hDl}) TRY(b->ensure((size_t)nb * nn * sizeof(double2)));
  TRY(c->hCu.ensure((size_t)nb * nn * sizeof(double2)));
  TRY(c->hZo.ensure((size_t)2 * std::max<size_t>(nn, 1) * sizeof(double2)));
  // per-unit block of the unit buffer: delta | D (nch) | kk (nch) | bloch (nch) | qk (nch) | fac (nch)
  // as doubles, then co | cop (nch each, double2), open_idx (nch ints), then info | info2 | uinfo
  const size_t ud = (1 + 5 * (size_t)nch + 1) / 2 * 2;  // doubles per unit, even: co follows 16-byte aligned
  const size_t ub = ud * sizeof(double) + 2 * (size_t)nch * sizeof(double2) + (size_t)nch * sizeof(int) + 16;
  const size_t ubp = (ub + 255) / 256 * 256;
  TRY(c->hUnit.ensure((size_t)nb * ubp + (size_t)3 * nb * sizeof(int) + (size_t)nb * sizeof(double) + 256));
  unsigned char* ubase = c->hUnit.as<unsigned char>();
  int* d_info = reinterpret_cast<int*>(ubase + (size_t)nb * ubp);
  int* d_info2 = d_info + nb;
  int* d_uinfo = d_info2 + nb;
  double* d_chg = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(d_uinfo + nb) + 8 -
                                           (reinterpret_cast<uintptr_t>(d_uinfo + nb) & 7));
  std::vector<double> d_delta_host(nb);
  TRY(c->hChan.ensure((size_t)nb * sizeof(double) + 64));
  const size_t smem_elim = (size_t)N * sizeof(double2);
  TRY(set_smem(hess_solve_kernel<1>, smem_elim));
  TRY(set_smem(hess_solve_kernel<2>, kHessSolveSmem));
  // a solve: the eliminations of all units (several CTAs per SM), then the back substitutions
  auto hess_solve = [&](const HessSolveArgs& args, int units) -> int {
    hess_solve_kernel<1><<<units, kHessThreads, args.W ? smem_elim : 0, c->stream>>>(args);
    LAUNCH_CHECK();
    hess_solve_kernel<2><<<units, kHessThreads, kHessSolveSmem, c->stream>>>(args);
    LAUNCH_CHECK();
    return HPRMAT_B200_OK;
  };
  TRY(set_smem(hess_woodbury_kernel, hess_woodbury_smem(nch)));
  std::vector<unsigned char> hu((size_t)nb * ubp);
  std::vector<int> hinfo(3 * (size_t)nb);
  std::vector<double> hchg(nb), hprev(nb);
  std::vector<char> hconv(nb);
  const double2* P = c->hP.as<double2>();
  const double2* PH = c->hPH.as<double2>();
  const double2* WH = c->hWH.as<double2>();
  for (size_t u0 = 0; u0 < units.size(); u0 += nb) {
    const int m = (int)std::min<size_t>(nb, units.size() - u0);
    // per-unit data
    std::fill(hu.begin(), hu.end(), 0);
    for (int j = 0; j < m; ++j) {
      const Boundary& b = bd[units[u0 + j]];
      double* hd = reinterpret_cast<double*>(hu.data() + (size_t)j * ubp);
      hd[0] = delta[u0 + j];
      for (int ch = 0; ch < nch; ++ch) {
        hd[1 + ch] = -b.bloch[ch];
        hd[1 + nch + ch] = b.kk[ch];
        hd[1 + 2 * nch + ch] = b.bloch[ch];
        hd[1 + 3 * nch + ch] = b.qk[ch];
        hd[1 + 4 * nch + ch] = b.fac[ch];
      }
      double2* hz = reinterpret_cast<double2*>(hd + ud);
      std::copy(b.co.begin(), b.co.end(), hz);
      std::copy(b.cop.begin(), b.cop.end(), hz + nch);
      int* hi = reinterpret_cast<int*>(hz + 2 * nch);
      std::copy(b.open_idx.begin(), b.open_idx.end(), hi);
      d_delta_host[j] = delta[u0 + j];
    }
    HPR_CUDA_TRY(cudaMemcpyAsync(ubase, hu.data(), (size_t)m * ubp, cudaMemcpyHostToDevice, c->stream));
    HPR_CUDA_TRY(cudaMemcpyAsync(c->hChan.p, d_delta_host.data(), (size_t)m * sizeof(double), cudaMemcpyHostToDevice,
                                 c->stream));
    HPR_CUDA_TRY(cudaMemsetAsync(d_info, 0, 3 * (size_t)nb * sizeof(int), c->stream));
    auto unit_d = [&](int j) { return reinterpret_cast<double*>(ubase + (size_t)j * ubp); };
    // D of every unit at stride ubp / 8 doubles: the Woodbury kernel reads D + unit * ldD
    const double* dD = unit_d(0) + 1;
    const int ldD = (int)(ubp / sizeof(double));
    // 1. Y = (H + delta I)^-1 W
    HessSolveArgs ha{};
    ha.Hr = c->hHr.as<double2>();
    ha.ldh = ld;
    ha.N = N;
    ha.nch = nch;
    ha.delta = c->hChan.as<double>();
    ha.W = c->hW.as<double2>();
    ha.ldw = ld;
    ha.Ue = c->hUe.as<double2>();
    ha.sUe = ld * N;
    ha.lm = c->hLm.as<double2>();
    ha.sw = c->hSw.as<int>();
    ha.Y = c->hY.as<double2>();
    ha.ldy = ld;
    ha.sY = ld * nch;
    ha.info = d_info;
    {
      NvtxRange nv("hprmat.hess.solve");
      TRY(hess_solve(ha, m));
    }
    TRY(phase(1));
    const long sN = ld * nch;
    // 2. -S = -W^H Y;  T, R0 = S T
    HPR_CUDA_TRY(cudaMemsetAsync(c->hS.p, 0, (size_t)m * nn * sizeof(double2), c->stream));
    if (zgemm_f64_update_batched(nch, nch, N, WH, nch, 0, c->hY.as<double2>(), ld, sN, c->hS.as<double2>(), nch,
                                 (long)nn, m, c->stream))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    hess_woodbury_kernel<<<m, kHessThreads, hess_woodbury_smem(nch), c->stream>>>(
        nch, c->hS.as<double2>(), dD, ldD, 0, nullptr, c->hT.as<double2>(), c->hRacc.as<double2>(), nullptr, nullptr,
        d_info2);
    LAUNCH_CHECK();
    // 3. X = P Y T  (-YT first)
    HPR_CUDA_TRY(cudaMemsetAsync(c->hYT.p, 0, (size_t)m * sN * sizeof(double2), c->stream));
    if (zgemm_f64_update_batched(N, nch, nch, c->hY.as<double2>(), ld, sN, c->hT.as<double2>(), nch, (long)nn,
                                 c->hYT.as<double2>(), ld, sN, m, c->stream))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    HPR_CUDA_TRY(cudaMemsetAsync(c->hX.p, 0, (size_t)m * sN * sizeof(double2), c->stream));
    if (zgemm_f64_update_batched(N, nch, N, P, ld, 0, c->hYT.as<double2>(), ld, sN, c->hX.as<double2>(), ld, sN, m,
                                 c->stream))
      return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
    TRY(phase(2));
    // 4. refinement steps against the structured C(E)
    int steps = 0;
    const int max_steps = std::max(1, c->opts.max_refine);
    for (; steps < max_steps; ++steps) {
      NvtxRange nv("hprmat.hess.refine");
      {
        // r = Q - C(E) X of every unit of the batch in two launches (unit blocks ubp bytes apart)
        const double* ud_ = unit_d(0);
        Operator op;
        op.structured = true;
        op.mesh = md;
        op.ch = ChannelData{ud_ + 1 + 4 * nch, ud_ + 1 + nch, ud_ + 1 + 2 * nch};
        op.nch = nch;
        op.N = N;
        op.vt = c->vt.as<double2>();
        op.q2 = md.q2;
        op.q1 = md.q1;
        op.nr = nr;
        TRY(apply_residual_units(c, op, c->hX.as<double2>(), ld, sN, nch, c->hR.as<double2>(), ld, sN, ldD, m));
      }
      // -y_r = -(H + delta I)^-1 P^H r
      HPR_CUDA_TRY(cudaMemsetAsync(c->hYr.p, 0, (size_t)m * sN * sizeof(double2), c->stream));
      if (zgemm_f64_update_batched(N, nch, N, PH, ld, 0, c->hR.as<double2>(), ld, sN, c->hYr.as<double2>(), ld, sN, m,
                                   c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      HessSolveArgs hr = ha;
      hr.W = nullptr;
      hr.Y = c->hYr.as<double2>();
      TRY(hess_solve(hr, m));
      // G = W^H y_r; Delta = (I + S D)^-1 G; R += Delta
      HPR_CUDA_TRY(cudaMemsetAsync(c->hG.p, 0, (size_t)m * nn * sizeof(double2), c->stream));
      if (zgemm_f64_update_batched(nch, nch, N, WH, nch, 0, c->hYr.as<double2>(), ld, sN, c->hG.as<double2>(), nch,
                                   (long)nn, m, c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      hess_woodbury_kernel<<<m, kHessThreads, hess_woodbury_smem(nch), c->stream>>>(
          nch, c->hS.as<double2>(), dD, ldD, 1, c->hG.as<double2>(), nullptr, c->hRacc.as<double2>(),
          c->hDl.as<double2>(), d_chg, d_info2);
      LAUNCH_CHECK();
      HPR_CUDA_TRY(cudaMemcpyAsync(hchg.data(), d_chg, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
      // Converged: the change is below surface_tol, or the error it leaves is predicted far below
      // it.  The change of step s is the error of the iterate before it; every step multiplies the
      // error by about the solver's relative accuracy, which is the first change itself (the same
      // Hessenberg solve made the first iterate's error) and later the ratio of two changes.
      bool all = true;
      for (int j = 0; j < m; ++j) {
        const double chg = hchg[j];
        const double rate = steps == 0 ? chg : (hprev[j] > 0.0 ? chg / hprev[j] : 0.0);
        hconv[j] = chg < c->opts.surface_tol || 1e3 * chg * std::max(rate, 1e-16) < c->opts.surface_tol;
        hprev[j] = chg;
        all = all && hconv[j];
      }
      if (all || steps + 1 == max_steps) {
        ++steps;
        break;
      }
      // X += P (y_r - Y D Delta):  hYr = -y_r + Y D Delta, then X -= P hYr
      hess_scale_rows_kernel<<<dim3(cdiv_u((long)nn, 256), m), 256, 0, c->stream>>>(c->hDl.as<double2>(), dD, ldD,
                                                                                    nch, c->hT.as<double2>());
      LAUNCH_CHECK();
      if (zgemm_f64_update_batched(N, nch, nch, c->hY.as<double2>(), ld, sN, c->hT.as<double2>(), nch, (long)nn,
                                   c->hYr.as<double2>(), ld, sN, m, c->stream) ||
          zgemm_f64_update_batched(N, nch, N, P, ld, 0, c->hYr.as<double2>(), ld, sN, c->hX.as<double2>(), ld, sN, m,
                                   c->stream))
        return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
      // T now holds -D Delta; the next step's Woodbury reads only S, D and G
    }
    TRY(phase(3));
    // 5. U of every unit from R = Racc / a
    HPR_CUDA_TRY(cudaMemcpyAsync(hinfo.data(), d_info, 2 * (size_t)nb * sizeof(int), cudaMemcpyDeviceToHost,
                                 c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    scale_copy_kernel<<<cdiv_u((long)m * nn, 256), 256, 0, c->stream>>>(c->hRacc.as<double2>(), c->hRacc.as<double2>(),
                                                                        (long)m * nn, 1.0 / rmax);
    LAUNCH_CHECK();
    // one launch for the batch's collision matrices (a unit with a zero Hessenberg or Woodbury
    // pivot is skipped: it goes to the LU path)
    {
      std::vector<UmatUnit> uu(m);
      TRY(c->hZo.ensure((size_t)2 * m * std::max<size_t>(nn, 1) * sizeof(double2)));
      for (int jj = 0; jj < m; ++jj) {
        const double* ud_ = unit_d(jj);
        const double2* dz = reinterpret_cast<const double2*>(ud_ + ud);
        UmatUnit& q = uu[jj];
        q.R = c->hRacc.as<double2>() + (size_t)jj * nn;
        q.open_idx = reinterpret_cast<const int*>(dz + 2 * nch);
        q.qk = ud_ + 1 + 3 * nch;
        q.co = dz;
        q.cop = dz + nch;
        q.no = bd[units[u0 + jj]].nopen;
        q.zo = c->hZo.as<double2>() + (size_t)2 * jj * std::max<size_t>(nn, 1);
        q.zi = q.zo + std::max<size_t>(nn, 1);
        q.cu = c->hCu.as<double2>() + (size_t)jj * nn;
        q.info = d_uinfo + jj;
        q.skip = hinfo[jj] != 0 ? d_info + jj : d_info2 + jj;
      }
      TRY(c->hUmat.ensure((size_t)m * sizeof(UmatUnit)));
      HPR_CUDA_TRY(cudaMemcpyAsync(c->hUmat.p, uu.data(), (size_t)m * sizeof(UmatUnit), cudaMemcpyHostToDevice,
                                   c->stream));
      umatrix_batch_kernel<<<m, 1024, 0, c->stream>>>(c->hUmat.as<UmatUnit>(), nch);
      LAUNCH_CHECK();
      HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));  // uu outlives its copy
    }
    HPR_CUDA_TRY(cudaMemcpyAsync(hinfo.data() + 2 * nb, d_uinfo, (size_t)nb * sizeof(int), cudaMemcpyDeviceToHost,
                                 c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int j = 0; j < m; ++j) {
      const int e = units[u0 + j];
      if (hinfo[j] != 0 || hinfo[nb + j] != 0) {
        fallback.push_back(e);
        continue;
      }
      int s = hinfo[2 * nb + j] != 0 ? HPRMAT_B200_SINGULAR : HPRMAT_B200_OK;
      if (s == HPRMAT_B200_OK && !hconv[j]) s = HPRMAT_B200_NOT_CONVERGED;
      if (s == HPRMAT_B200_SINGULAR) set_last_error_msg("rmatrix_scan_shifted: singular Z_O in the collision-matrix step");
      if (s != HPRMAT_B200_SINGULAR) {
        HPR_CUDA_TRY(cudaMemcpyAsync(B.cu + (size_t)e * nn * 2, c->hCu.as<double2>() + (size_t)j * nn,
                                     nn * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
      }
      B.status[e] = s;
      note(s);
    }
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    TRY(phase(4));
    c->hess_steps_last = steps;
  }
  return HPRMAT_B200_OK;
}

int hprmat_b200_rmatrix_scan_shifted(hprmat_b200_ctx* c, int nblocks, const hprmat_b200_scan_block* blocks,
                                     double rmax, int nr, double* seconds) {
  TRY(check_ctx(c));
  TRY(scan_check_blocks(nblocks, blocks, rmax, nr, "rmatrix_scan_shifted"));
  if (c->nr != nr || c->ns != 1 || c->rmax != rmax) TRY(hprmat_b200_rmat_ini(c, nr, 1, rmax, nullptr));
  auto t0 = Clock::now();
  TRY(scan_upload(c, nblocks, blocks));
  int first_error = HPRMAT_B200_OK;
  std::string err_msg;
  c->hess_fallback_last = 0;
  // one block on context w: the shifted form, then the LU path for what it does not take
  auto run_block = [&](hprmat_b200_ctx* w, int b, int* ferr, std::string* emsg) -> int {
    const hprmat_b200_scan_block& B = blocks[b];
    const double2* d_cpot = c->scan_cpot[b]->as<double2>();
    std::vector<int> fallback;
    if (B.nch > kHsMaxRhs) {
      for (int e = 0; e < B.nenergies; ++e) fallback.push_back(e);
    } else {
      TRY(hess_scan_block(w, d_cpot, B, rmax, nr, fallback, ferr, emsg));
    }
    w->hess_fallback_last += (int)fallback.size();
    auto tfb = Clock::now();
    const size_t ubytes = (size_t)B.nch * B.nch * sizeof(double2);
    for (const int e : fallback) {
      int nopen = 0;
      int s = w->cu.ensure(ubytes);
      if (s == HPRMAT_B200_OK)
        s = rmatrix_core(w, B.nch, B.lval, B.qk + (size_t)e * B.nch, B.eta + (size_t)e * B.nch, rmax, nr, 1, d_cpot,
                         B.ncp1, B.nch, w->cu.as<double2>(), &nopen, nullptr);
      if (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) {
        HPR_CUDA_TRY(cudaMemcpyAsync(B.cu + (size_t)e * B.nch * B.nch * 2, w->cu.p, ubytes, cudaMemcpyDeviceToHost,
                                     w->stream));
        HPR_CUDA_TRY(cudaStreamSynchronize(w->stream));
      }
      B.nopen[e] = nopen;
      B.status[e] = s;
      if (s != HPRMAT_B200_OK && *ferr == HPRMAT_B200_OK) {
        *ferr = s;
        *emsg = hprmat_b200_last_error();
      }
    }
    if (w->profile) w->hess_ms[5] += ms_since(tfb);
    return HPRMAT_B200_OK;
  };
  const int nw = std::max(1, std::min(c->hess_workers, nblocks));
  if (nw == 1) {
    for (int b = 0; b < nblocks; ++b) TRY(run_block(c, b, &first_error, &err_msg));
  } else {
    // Several blocks in flight, one worker context (stream, buffers, host thread) each, so that
    // one block's latency-bound reduction overlaps the others' GEMMs and solves.  Blocks go to
    // the least loaded worker, largest first (cost ~ N^3 for the reduction plus
    // nenergies N^2 nch for the energies); each worker gets its share of the batch budget.
    TRY(scan_workers_ready(c, nw, nr, rmax));
    c->hess_steps_last = 0;
    std::vector<std::vector<int>> mine((size_t)nw);
    {
      std::vector<int> order(nblocks);
      std::vector<double> cost(nblocks), load((size_t)nw, 0.0);
      for (int b = 0; b < nblocks; ++b) {
        order[b] = b;
        const double n = (double)blocks[b].nch * nr;
        cost[b] = n * n * n + (double)blocks[b].nenergies * n * n * blocks[b].nch;
      }
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
      for (const int b : order) {
        const int i = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        mine[i].push_back(b);
        load[i] += cost[b];
      }
    }
    std::vector<int> status((size_t)nw, HPRMAT_B200_OK), ferr((size_t)nw, HPRMAT_B200_OK);
    std::vector<std::string> fail_msg((size_t)nw), emsg((size_t)nw);
    std::vector<std::thread> th;
    for (int i = 0; i < nw; ++i) {
      hprmat_b200_ctx* w = c->scan_workers[i];
      w->hess_blocked = c->hess_blocked;
      w->hb_cluster = c->hb_cluster;
      w->hess_budget_gb = c->hess_budget_gb / nw;
      w->profile = c->profile;
      w->hess_fallback_last = 0;
      for (double& v : w->hess_ms) v = 0.0;
      th.emplace_back([&, i, w]() {
        cudaSetDevice(w->device);
        for (const int b : mine[i]) {
          const int s = run_block(w, b, &ferr[i], &emsg[i]);
          if (s != HPRMAT_B200_OK) {
            status[i] = s;
            fail_msg[i] = hprmat_b200_last_error();
            break;
          }
        }
        cudaStreamSynchronize(w->stream);
      });
    }
    for (std::thread& t : th) t.join();
    for (int i = 0; i < nw; ++i) {
      hprmat_b200_ctx* w = c->scan_workers[i];
      c->hess_fallback_last += w->hess_fallback_last;
      c->hess_steps_last = std::max(c->hess_steps_last, w->hess_steps_last);
      if (c->profile)
        for (int k = 0; k < 6; ++k) c->hess_ms[k] += w->hess_ms[k];
      if (ferr[i] != HPRMAT_B200_OK && first_error == HPRMAT_B200_OK) {
        first_error = ferr[i];
        err_msg = emsg[i];
      }
    }
    for (int i = 0; i < nw; ++i)
      if (status[i] != HPRMAT_B200_OK) return fail(status[i], "rmatrix_scan_shifted: %s", fail_msg[i].c_str());
  }
  if (seconds) *seconds = std::chrono::duration<double>(Clock::now() - t0).count();
  if (first_error != HPRMAT_B200_OK && first_error != HPRMAT_B200_NOT_CONVERGED)
    return fail(first_error, "rmatrix_scan_shifted: %s", err_msg.c_str());
  return first_error;
}

// Scan autotuner (see the header).  A trial runs one energy of a block on every worker at once
// (a warm-up round, then the best of two timed rounds, host wall clock around the joined
// threads, each worker's stream synchronised): the device under the scan's own concurrency.
int hprmat_b200_scan_autotune(hprmat_b200_ctx* c, int nblocks, const hprmat_b200_scan_block* blocks, double rmax,
                              int nr, int nworkers, double* seconds) {
  TRY(check_ctx(c));
  TRY(scan_check_blocks(nblocks, blocks, rmax, nr, "scan_autotune"));
  auto t0 = Clock::now();
  TRY(scan_upload(c, nblocks, blocks));
  if (nworkers <= 0) nworkers = 4;
  TRY(scan_workers_ready(c, nworkers, nr, rmax));
  std::vector<ScanTune> table;
  auto trial = [&](const ScanTune& t, int b, int e, double* ms) -> int {
    const hprmat_b200_scan_block& B = blocks[b];
    const size_t ubytes = (size_t)B.nch * B.nch * sizeof(double2);
    std::atomic<int> err{0};
    auto run = [&](int wi) {
      hprmat_b200_ctx* w = c->scan_workers[wi];
      cudaSetDevice(w->device);
      scan_apply(w, c, &t);
      w->lu_held = false;
      int nopen = 0;
      int s = w->cu.ensure(ubytes);
      if (s == HPRMAT_B200_OK)
        s = rmatrix_core(w, B.nch, B.lval, B.qk + (size_t)e * B.nch, B.eta + (size_t)e * B.nch, rmax, nr, 1,
                         c->scan_cpot[b]->as<double2>(), B.ncp1, B.nch, w->cu.as<double2>(), &nopen, nullptr);
      if ((s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) && cudaStreamSynchronize(w->stream) != cudaSuccess)
        s = HPRMAT_B200_ERR_CUDA;
      if (s != HPRMAT_B200_OK && s != HPRMAT_B200_NOT_CONVERGED) {
        int z = 0;
        err.compare_exchange_strong(z, s);
      }
    };
    double best = 0.0;
    for (int round = 0; round < 3; ++round) {
      auto r0 = Clock::now();
      std::vector<std::thread> th;
      for (int i = 1; i < nworkers; ++i) th.emplace_back(run, i);
      run(0);
      for (auto& x : th) x.join();
      const double dt = ms_since(r0);
      if (err.load() != 0) return err.load();
      if (round == 1 || (round == 2 && dt < best)) best = dt;
    }
    *ms = best;
    return HPRMAT_B200_OK;
  };
  std::vector<long> done;
  for (int b = 0; b < nblocks; ++b) {
    const hprmat_b200_scan_block& B = blocks[b];
    const long N = (long)B.nch * nr;
    if (B.nenergies == 0 || std::find(done.begin(), done.end(), N) != done.end()) continue;
    done.push_back(N);
    const std::vector<int> order = scan_energy_order(B);
    ScanTune cur{(int)N, c->opts.panel_nb > 0 ? c->opts.panel_nb : 128, c->panel_cluster ? 1 : 0, c->panel_rpc_min,
                 c->wave_sb, c->gmres_m, c->tcplan.max_grid, 0.0};
    // a representative energy whose solve succeeds: the middle one, else the first or last
    int e = -1;
    double best = 0.0;
    for (const int cand : {order[order.size() / 2], order.front(), order.back()}) {
      if (trial(cur, b, cand, &best) == HPRMAT_B200_OK) {
        e = cand;
        break;
      }
    }
    if (e < 0) continue;
    // a setting is taken when it is 5% faster twice: once against the incumbent's best time,
    // then again against a fresh trial of the incumbent (concurrent trials vary by a few %)
    auto consider = [&](ScanTune t) -> int {
      double ms = 0.0;
      if (trial(t, b, e, &ms) != HPRMAT_B200_OK || !(ms < 0.95 * best)) return HPRMAT_B200_OK;
      double ms_inc = 0.0, ms2 = 0.0;
      if (trial(cur, b, e, &ms_inc) != HPRMAT_B200_OK || trial(t, b, e, &ms2) != HPRMAT_B200_OK)
        return HPRMAT_B200_OK;
      ms = std::min(ms, ms2);
      best = std::min(best, ms_inc);
      if (ms < 0.95 * best) {
        best = ms;
        cur = t;
      }
      return HPRMAT_B200_OK;
    };
    for (const int v : {128, 64, 32}) {
      if (v == cur.nb || pick_nb(c, (int)N, sizeof(float2), v) != v) continue;
      ScanTune t = cur;
      t.nb = v;
      TRY(consider(t));
    }
    {
      ScanTune t = cur;
      t.cluster = !cur.cluster;
      TRY(consider(t));
    }
    for (const int v : {16, 32, 64}) {
      if (v == cur.rpc_min) continue;
      ScanTune t = cur;
      t.rpc_min = v;
      TRY(consider(t));
    }
    for (const int v : {0, 2, 1}) {
      if (v == cur.sb) continue;
      ScanTune t = cur;
      t.sb = v;
      TRY(consider(t));
    }
    for (const int v : {12, 8, 16}) {
      if (v == cur.gmres_m) continue;
      ScanTune t = cur;
      t.gmres_m = v;
      TRY(consider(t));
    }
    for (const int v : {0, c->nsm / 2, c->nsm / 4}) {  // trailing-update CTAs: all SMs, half, a quarter
      if (v == cur.tc_grid) continue;
      ScanTune t = cur;
      t.tc_grid = v;
      TRY(consider(t));
    }
    cur.ms = best;
    table.push_back(cur);
  }
  for (int i = 0; i < nworkers; ++i) scan_apply(c->scan_workers[i], c, nullptr);
  c->scan_tune = table;
  if (seconds) *seconds = std::chrono::duration<double>(Clock::now() - t0).count();
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_wait_probe(hprmat_b200_ctx* c, int spins) {
  TRY(check_ctx(c));
  if (spins < 4096 || spins > (1 << 24)) return fail(HPRMAT_B200_ERR_ARG, "wait_probe: spins must be in 4096..2^24");
  int* status = c->status.as<int>();
  HPR_CUDA_TRY(cudaMemsetAsync(status, 0, SW_COUNT * sizeof(int), c->stream));
  wait_probe_kernel<<<1, 32, 0, c->stream>>>(status + SW_BARRIER, status + SW_TIMEOUT, (unsigned)spins);
  LAUNCH_CHECK();
  HPR_CUDA_TRY(cudaMemcpyAsync(c->h_status, status, SW_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const int site = c->h_status[SW_TIMEOUT];
  HPR_CUDA_TRY(cudaMemsetAsync(status, 0, SW_COUNT * sizeof(int), c->stream));  // leave the block clean
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (site != 0) return fail(HPRMAT_B200_ERR_TIMEOUT, "wait_probe: bounded wait gave up as designed (site %d)", site);
  return HPRMAT_B200_OK;
}

int hprmat_b200_scan_tune_get(hprmat_b200_ctx* c, int* rows, double* ms, int max) {
  if (!c) return -1;
  const int n = (int)c->scan_tune.size();
  const int m = max > 0 ? std::min(max, n) : 0;
  for (int i = 0; i < m; ++i) {
    const ScanTune& t = c->scan_tune[i];
    if (rows) {
      int* r = rows + (size_t)kTuneInts * i;
      r[0] = t.N;
      r[1] = t.nb;
      r[2] = t.cluster;
      r[3] = t.rpc_min;
      r[4] = t.sb;
      r[5] = t.gmres_m;
      r[6] = t.tc_grid;
    }
    if (ms) ms[i] = t.ms;
  }
  return n;
}

int hprmat_b200_scan_tune_set(hprmat_b200_ctx* c, const int* rows, int n) {
  TRY(check_ctx(c));
  if (n < 0 || (n > 0 && !rows)) return fail(HPRMAT_B200_ERR_ARG, "scan_tune_set: invalid arguments");
  std::vector<ScanTune> table;
  for (int i = 0; i < n; ++i) {
    const int* r = rows + (size_t)kTuneInts * i;
    const bool ok = r[0] > 0 && (r[1] == 16 || r[1] == 32 || r[1] == 64 || r[1] == 128) && (r[2] == 0 || r[2] == 1) &&
                    r[3] >= 1 && (r[4] == 0 || r[4] == 1 || r[4] == 2 || r[4] == 4) && r[5] >= 1 &&
                    r[5] <= kGmresMaxM && r[6] >= 0;
    if (!ok) return fail(HPRMAT_B200_ERR_ARG, "scan_tune_set: invalid row %d", i);
    table.push_back(ScanTune{r[0], r[1], r[2], r[3], r[4], r[5], r[6], 0.0});
  }
  c->scan_tune = table;
  return HPRMAT_B200_OK;
}

// Adjoint of one collision matrix.  Symmetric potential: the forward solve at the context's
// precision and Y = X M2^T (C^T = C).  Otherwise the forward solve on the FP64 path, then one
// solve with C^T from the same factors (adjoint.cuh).  With G = gu (dL = Re sum conj(G) dU):
//   M = W G^H Z_O^-1,  W = diag(cop) U - diag(conj cop)       (dU = Z_O^-1 dRt W)
//   M2(i2, i1) = M(m2, m1) sqrt(k_i1 / k_i2)                  (Rt = R sqrt(k_i / k_j), open)
//   C^T Y = Q M2^T,  Q = blockdiag(q2)                         (R = Q^T X / a)
//   grad(r_i, c, c') = -conj(sum_col Y[(c,i), col] X[(c',i), col]) / a
// M2 of the adjoint (the rhs of C^T Y = Q M2^T is Q M2^T): from R (host, nch x nch, R/a as the
// U step uses it), U (host cu, ld ndim) and the loss gradient gu (ld ndim).  no = nopen.
static int adjoint_m2(int nch, const int* lval, const double* qk, const double* eta, double rmax, double a,
                      const std::vector<double2>& R, const double* cu, const double* gu, int ndim,
                      std::vector<double2>& M2, int* no_out) {
  Boundary bnd;
  TRY(boundary_values(nch, lval, qk, eta, rmax, a, bnd));
  const int no = bnd.nopen;
  *no_out = no;
  M2.assign((size_t)nch * nch, mk(0.0, 0.0));
  if (no == 0) return HPRMAT_B200_OK;
  auto sk = [&](int m1, int m2) { return sqrt(qk[bnd.open_idx[m1]] / qk[bnd.open_idx[m2]]); };
  std::vector<double2> Zt((size_t)no * no), Pt((size_t)no * no);  // Z_O^T and (W G^H)^T
  for (int m2 = 0; m2 < no; ++m2)
    for (int m1 = 0; m1 < no; ++m1) {
      double2 r = R[bnd.open_idx[m1] + (size_t)bnd.open_idx[m2] * nch];
      const double sc = sk(m1, m2);
      r.x *= sc;
      r.y *= sc;
      double2 z = cmul(r, bnd.cop[m2]);
      z.x = -z.x;
      z.y = -z.y;
      if (m1 == m2) {
        z.x += bnd.co[m1].x;
        z.y += bnd.co[m1].y;
      }
      Zt[m2 + (size_t)m1 * no] = z;  // (Z_O^T)(m2, m1) = Z_O(m1, m2)
    }
  for (int a1 = 0; a1 < no; ++a1)
    for (int b1 = 0; b1 < no; ++b1) {
      double2 acc = mk(0.0, 0.0);  // (W G^H)(a1, b1) = sum_k W(a1, k) conj(G(b1, k))
      for (int k = 0; k < no; ++k) {
        double2 w = cmul(bnd.cop[a1], host_c(cu, a1 + (size_t)k * ndim));
        if (a1 == k) {
          w.x -= bnd.cop[a1].x;
          w.y += bnd.cop[a1].y;
        }
        const double2 g = host_c(gu, b1 + (size_t)k * ndim);
        cfma(acc, w, mk(g.x, -g.y));
      }
      Pt[b1 + (size_t)a1 * no] = acc;
    }
  // M = (W G^H) Z_O^-1  <=>  Z_O^T M^T = (W G^H)^T
  if (!host_csolve(Zt, Pt, no, no)) return fail(HPRMAT_B200_SINGULAR, "rmatrix_adjoint: singular Z_O");
  // M2(i2, i1) = M(m2, m1) sqrt(k_i1/k_i2), stored at [i2 + i1 nch]
  for (int m1 = 0; m1 < no; ++m1)
    for (int m2 = 0; m2 < no; ++m2) {
      double2 v = Pt[m1 + (size_t)m2 * no];  // M^T(m1, m2) = M(m2, m1)
      const double sc = sk(m1, m2);
      M2[bnd.open_idx[m2] + (size_t)bnd.open_idx[m1] * nch] = mk(v.x * sc, v.y * sc);
    }
  return HPRMAT_B200_OK;
}

// Gradient at the mesh points for a symmetric C(E) from its forward solution X (device, N x nch,
// ld ldx): Y = X M2^T, grad(r_i, c, c') = -conj(sum_col Y[(c,i), col] X[(c',i), col]) / a into the
// device array d_grad (complex (ncp1, ndim, ndim), zeroed here).
static int adjoint_grad_symmetric(hprmat_b200_ctx* c, int nch, int nr, int ndim, int ncp1, double a,
                                  const std::vector<double2>& M2, const double2* X, long ldx, double2* d_grad) {
  const int N = nch * nr;
  HPR_CUDA_TRY(cudaMemsetAsync(d_grad, 0, (size_t)ncp1 * ndim * ndim * sizeof(double2), c->stream));
  TRY(c->adj_y.ensure((size_t)ldx * nch * sizeof(double2)));
  double2* Y = c->adj_y.as<double2>();
  // C -= A B with A = X, B(ch, col) = -M2(col, ch), C = 0
  std::vector<double2> nb((size_t)nch * nch);
  for (int col = 0; col < nch; ++col)
    for (int ch = 0; ch < nch; ++ch) {
      const double2 m = M2[col + (size_t)ch * nch];
      nb[ch + (size_t)col * nch] = mk(-m.x, -m.y);
    }
  TRY(c->adj_part.ensure(nb.size() * sizeof(double2)));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->adj_part.p, nb.data(), nb.size() * sizeof(double2), cudaMemcpyHostToDevice,
                               c->stream));
  HPR_CUDA_TRY(cudaMemsetAsync(Y, 0, (size_t)ldx * nch * sizeof(double2), c->stream));
  dim3 grid(cdiv_u(N, 64), cdiv_u(nch, 64));
  cgemm_update_kernel<double2><<<grid, 256, 0, c->stream>>>(N, nch, nch, X, ldx, c->adj_part.as<double2>(), nch, Y,
                                                            ldx);
  LAUNCH_CHECK();
  potential_grad_kernel<<<dim3(nr, nch), 128, 0, c->stream>>>(Y, X, ldx, nr, nch, nch, 1.0 / a, d_grad, ncp1, ndim);
  LAUNCH_CHECK();
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));  // nb must outlive its copy
  return HPRMAT_B200_OK;
}

static bool potential_symmetric(const double* cpot, int ncp1, int ndim, int nr, int nch) {
  for (int cp = 0; cp < nch; ++cp)
    for (int c1 = cp + 1; c1 < nch; ++c1)
      for (int i = 0; i < nr; ++i) {
        const size_t a1 = 2 * ((size_t)i + (size_t)ncp1 * (c1 + (size_t)ndim * cp));
        const size_t a2 = 2 * ((size_t)i + (size_t)ncp1 * (cp + (size_t)ndim * c1));
        if (cpot[a1] != cpot[a2] || cpot[a1 + 1] != cpot[a2 + 1]) return false;
      }
  return true;
}

int hprmat_b200_rmatrix_adjoint(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                                double rmax, int nr, int ns, const double* cpot, int ncp1, int ndim, const double* gu,
                                double* cu, int* nopen, double* grad, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!cpot || !cu || !gu || !grad || !nopen || ndim < nch || ncp1 < nr || nch <= 0)
    return fail(HPRMAT_B200_ERR_ARG, "rmatrix_adjoint: invalid arguments");
  if (ns != 1) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "rmatrix_adjoint: one interval (ns = 1) only");
  const size_t pbytes = (size_t)ncp1 * ndim * ndim * sizeof(double2);
  const size_t ubytes = (size_t)ndim * ndim * sizeof(double2);
  TRY(c->cpot.ensure(pbytes));
  TRY(c->cu.ensure(ubytes));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->cpot.p, cpot, pbytes, cudaMemcpyHostToDevice, c->stream));
  // C(E) is complex symmetric when the potential is (the kinetic, Bloch, centrifugal and energy
  // terms are): then C^-T = C^-1 and the adjoint solution is Y = X M2^T from the forward
  // solution X = C^-1 Q, at the context's precision (refined) -- no transposed solve.  Otherwise
  // the forward runs on the FP64 path and Y comes from a solve with C^T on its factors.
  const bool symmetric = potential_symmetric(cpot, ncp1, ndim, nr, nch);
  const int prec = c->opts.precision;
  if (!symmetric) c->opts.precision = HPRMAT_B200_PREC_FP64;
  int s = rmatrix_core(c, nch, lval, qk, eta, rmax, nr, ns, c->cpot.as<double2>(), ncp1, ndim, c->cu.as<double2>(),
                       nopen, stats);
  c->opts.precision = prec;
  if (s != HPRMAT_B200_OK && s != HPRMAT_B200_NOT_CONVERGED) return s;
  if (!symmetric && c->f64_nb > 64) return fail(HPRMAT_B200_ERR_UNSUPPORTED, "rmatrix_adjoint: panel_nb above 64");
  HPR_CUDA_TRY(cudaMemcpyAsync(cu, c->cu.p, ubytes, cudaMemcpyDeviceToHost, c->stream));
  std::vector<double2> R((size_t)nch * nch);
  HPR_CUDA_TRY(cudaMemcpyAsync(R.data(), c->rmat.p, R.size() * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const int N = nch * nr;
  const long ld = (N + 3) / 4 * 4;  // the layout rmatrix_core gave X (and the FP64 factors)
  const double a = rmax / ns;
  TRY(c->adj_grad.ensure(pbytes));
  HPR_CUDA_TRY(cudaMemsetAsync(c->adj_grad.p, 0, pbytes, c->stream));
  std::vector<double2> M2;
  int no = 0;
  TRY(adjoint_m2(nch, lval, qk, eta, rmax, a, R, cu, gu, ndim, M2, &no));
  if (no > 0) {
    if (symmetric) {
      TRY(adjoint_grad_symmetric(c, nch, nr, ndim, ncp1, a, M2, c->X64.as<double2>(), ld, c->adj_grad.as<double2>()));
    } else {
      // C^T Y = Q M2^T: rhs[(c,i), col] = q2_i M2(col, c)
      TRY(c->adj_y.ensure((size_t)ld * nch * sizeof(double2)));
      double2* Y = c->adj_y.as<double2>();
      std::vector<double2> rhs((size_t)ld * nch, mk(0.0, 0.0));
      for (int col = 0; col < nch; ++col)
        for (int ch = 0; ch < nch; ++ch) {
          const double2 m = M2[col + (size_t)ch * nch];
          if (m.x == 0.0 && m.y == 0.0) continue;
          for (int i = 0; i < nr; ++i)
            rhs[(size_t)(ch * nr + i) + (size_t)col * ld] = mk(c->q2[i] * m.x, c->q2[i] * m.y);
        }
      HPR_CUDA_TRY(cudaMemcpyAsync(Y, rhs.data(), rhs.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
      TRY(lu_solve_trans(c, c->W.as<double2>(), ld, N, c->f64_nb, c->f64_nsteps, Y, ld, nch));
      potential_grad_kernel<<<dim3(nr, nch), 128, 0, c->stream>>>(Y, c->X64.as<double2>(), ld, nr, nch, nch, 1.0 / a,
                                                                  c->adj_grad.as<double2>(), ncp1, ndim);
      LAUNCH_CHECK();
      HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));  // rhs must outlive its copy
    }
  }
  HPR_CUDA_TRY(cudaMemcpyAsync(grad, c->adj_grad.p, pbytes, cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return s;
}


int hprmat_b200_rmatrix_x(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                          double rmax, int nr, const double* cpot, int ncp1, int ndim, double* cu, int* nopen,
                          void* d_x, long ldx, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!d_x || ldx < (long)nch * nr) return fail(HPRMAT_B200_ERR_ARG, "rmatrix_x: need d_x with ldx >= nch*nr");
  int s = hprmat_b200_rmatrix(c, nch, lval, qk, eta, rmax, nr, 1, cpot, ncp1, ndim, cu, nopen, stats);
  if (s != HPRMAT_B200_OK && s != HPRMAT_B200_NOT_CONVERGED) return s;
  const long N = (long)nch * nr, ld = (N + 3) / 4 * 4;
  HPR_CUDA_TRY(cudaMemcpy2DAsync(d_x, (size_t)ldx * sizeof(double2), c->X64.p, (size_t)ld * sizeof(double2),
                                 (size_t)N * sizeof(double2), nch, cudaMemcpyDeviceToDevice, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return s;
}

int hprmat_b200_adjoint_from_x(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                               double rmax, int nr, const double* cpot, int ncp1, int ndim, const double* cu,
                               const void* d_x, long ldx, const double* gu, double* grad) {
  TRY(check_ctx(c));
  if (!cpot || !cu || !gu || !grad || !d_x || ndim < nch || ncp1 < nr || nch <= 0 || ldx < (long)nch * nr)
    return fail(HPRMAT_B200_ERR_ARG, "adjoint_from_x: invalid arguments");
  if (!potential_symmetric(cpot, ncp1, ndim, nr, nch))
    return fail(HPRMAT_B200_ERR_UNSUPPORTED, "adjoint_from_x: the potential is not symmetric; use rmatrix_adjoint");
  if (c->nr != nr || c->ns != 1 || c->rmax != rmax)
    return fail(HPRMAT_B200_ERR_ARG, "adjoint_from_x: call rmat_ini(nr=%d, ns=1, rmax=%g) first", nr, rmax);
  const double a = rmax;
  const size_t pbytes = (size_t)ncp1 * ndim * ndim * sizeof(double2);
  // R = q2^T X / a from the forward solution
  TRY(c->rmat.ensure((size_t)nch * nch * sizeof(double2) + 64));
  const MeshDev md = mesh_dev(c, 0);
  rmat_extract_kernel<<<dim3(nch, cdiv_u(nch, 128)), 128, 0, c->stream>>>((const double2*)d_x, ldx, md.q2, nr, nch,
                                                                         nch, 1.0 / a, c->rmat.as<double2>());
  LAUNCH_CHECK();
  std::vector<double2> R((size_t)nch * nch);
  HPR_CUDA_TRY(cudaMemcpyAsync(R.data(), c->rmat.p, R.size() * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  std::vector<double2> M2;
  int no = 0;
  TRY(adjoint_m2(nch, lval, qk, eta, rmax, a, R, cu, gu, ndim, M2, &no));
  TRY(c->adj_grad.ensure(pbytes));
  if (no > 0) {
    TRY(adjoint_grad_symmetric(c, nch, nr, ndim, ncp1, a, M2, (const double2*)d_x, ldx, c->adj_grad.as<double2>()));
  } else {
    HPR_CUDA_TRY(cudaMemsetAsync(c->adj_grad.p, 0, pbytes, c->stream));
  }
  HPR_CUDA_TRY(cudaMemcpyAsync(grad, c->adj_grad.p, pbytes, cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return HPRMAT_B200_OK;
}

int hprmat_b200_rmatrix_x_device(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk, const double* eta,
                                 double rmax, int nr, const void* d_cpot, int ncp1, int ndim, void* d_cu, int* nopen,
                                 void* d_x, long ldx, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!d_x || ldx < (long)nch * nr) return fail(HPRMAT_B200_ERR_ARG, "rmatrix_x_device: need d_x with ldx >= nch*nr");
  int s = hprmat_b200_rmatrix_device(c, nch, lval, qk, eta, rmax, nr, 1, d_cpot, ncp1, ndim, d_cu, nopen, stats);
  if (s != HPRMAT_B200_OK && s != HPRMAT_B200_NOT_CONVERGED) return s;
  const long N = (long)nch * nr, ld = (N + 3) / 4 * 4;
  HPR_CUDA_TRY(cudaMemcpy2DAsync(d_x, (size_t)ldx * sizeof(double2), c->X64.p, (size_t)ld * sizeof(double2),
                                 (size_t)N * sizeof(double2), nch, cudaMemcpyDeviceToDevice, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return s;
}

int hprmat_b200_adjoint_from_x_device(hprmat_b200_ctx* c, int nch, const int* lval, const double* qk,
                                      const double* eta, double rmax, int nr, const void* d_cpot, int ncp1, int ndim,
                                      const double* cu, const void* d_x, long ldx, const double* gu, void* d_grad) {
  TRY(check_ctx(c));
  if (!d_cpot || !cu || !gu || !d_grad || !d_x || ndim < nch || ncp1 < nr || nch <= 0 || ldx < (long)nch * nr)
    return fail(HPRMAT_B200_ERR_ARG, "adjoint_from_x_device: invalid arguments");
  if (c->nr != nr || c->ns != 1 || c->rmax != rmax)
    return fail(HPRMAT_B200_ERR_ARG, "adjoint_from_x_device: call rmat_ini(nr=%d, ns=1, rmax=%g) first", nr, rmax);
  // the potential must be symmetric (C(E) complex symmetric): checked on the device
  int* d_flag = c->status.as<int>() + kSymSlot;
  HPR_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), c->stream));
  potential_asym_kernel<<<dim3(cdiv_u(nr, 128), nch, nch), 128, 0, c->stream>>>((const double2*)d_cpot, ncp1, ndim, nr,
                                                                               d_flag);
  LAUNCH_CHECK();
  int asym = 0;
  HPR_CUDA_TRY(cudaMemcpyAsync(&asym, d_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  const double a = rmax;
  TRY(c->rmat.ensure((size_t)nch * nch * sizeof(double2) + 64));
  const MeshDev md = mesh_dev(c, 0);
  rmat_extract_kernel<<<dim3(nch, cdiv_u(nch, 128)), 128, 0, c->stream>>>((const double2*)d_x, ldx, md.q2, nr, nch,
                                                                         nch, 1.0 / a, c->rmat.as<double2>());
  LAUNCH_CHECK();
  std::vector<double2> R((size_t)nch * nch);
  HPR_CUDA_TRY(cudaMemcpyAsync(R.data(), c->rmat.p, R.size() * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (asym)
    return fail(HPRMAT_B200_ERR_UNSUPPORTED,
                "adjoint_from_x_device: the potential is not symmetric; use rmatrix_adjoint");
  std::vector<double2> M2;
  int no = 0;
  TRY(adjoint_m2(nch, lval, qk, eta, rmax, a, R, cu, gu, ndim, M2, &no));
  if (no > 0) {
    TRY(adjoint_grad_symmetric(c, nch, nr, ndim, ncp1, a, M2, (const double2*)d_x, ldx, (double2*)d_grad));
  } else {
    HPR_CUDA_TRY(cudaMemsetAsync(d_grad, 0, (size_t)ncp1 * ndim * ndim * sizeof(double2), c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  return HPRMAT_B200_OK;
}

int hprmat_b200_solve_linear_device(hprmat_b200_ctx* c, const void* d_A, void* d_B, int n, int nrhs,
                                    hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  int s = solve_dense_core(c, (const double2*)d_A, (double2*)d_B, n, nrhs, stats);
  if (stats) stats->status = s;
  return s;
}

int hprmat_b200_solve_linear(hprmat_b200_ctx* c, const double* A, double* B, int n, int nrhs,
                             hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!A || !B || n <= 0 || nrhs <= 0) return fail(HPRMAT_B200_ERR_ARG, "solve_linear: invalid arguments");
  const size_t abytes = (size_t)n * n * sizeof(double2);
  const size_t bbytes = (size_t)n * nrhs * sizeof(double2);
  TRY(c->A64.ensure(abytes));
  TRY(c->B64.ensure(bbytes));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->A64.p, A, abytes, cudaMemcpyHostToDevice, c->stream));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->B64.p, B, bbytes, cudaMemcpyHostToDevice, c->stream));
  int s = solve_dense_core(c, c->A64.as<double2>(), c->B64.as<double2>(), n, nrhs, stats);
  if (s == HPRMAT_B200_OK || s == HPRMAT_B200_NOT_CONVERGED) {
    HPR_CUDA_TRY(cudaMemcpyAsync(B, c->B64.p, bbytes, cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  if (stats) stats->status = s;
  return s;
}

int hprmat_b200_solve_rmatrix(hprmat_b200_ctx* c, const double* cmat, const double* bvec, int nch, int nlag,
                              double normfac, double* rmat, hprmat_b200_stats* stats) {
  TRY(check_ctx(c));
  if (!cmat || !bvec || !rmat || nch <= 0 || nlag <= 0) return fail(HPRMAT_B200_ERR_ARG, "solve_rmatrix: invalid arguments");
  const int N = nch * nlag;
  std::vector<double> X((size_t)2 * N * nch, 0.0);
  for (int ich = 0; ich < nch; ++ich)
    for (int r = 0; r < nlag; ++r) {
      size_t idx = (size_t)(ich * nlag + r) + (size_t)ich * N;
      X[2 * idx] = bvec[2 * r];
      X[2 * idx + 1] = bvec[2 * r + 1];
    }
  // Real surface vectors (the R-matrix case) enable the surface stopping rule.
  bool real_b = true;
  for (int r = 0; r < nlag; ++r) real_b = real_b && bvec[2 * r + 1] == 0.0;
  const double* d_q2 = nullptr;
  if (real_b) {
    std::vector<double> q(nlag);
    for (int r = 0; r < nlag; ++r) q[r] = bvec[2 * r];
    TRY(c->rmat.ensure(std::max(c->rmat.bytes, (size_t)nlag * sizeof(double) + 64)));
    HPR_CUDA_TRY(cudaMemcpy(c->rmat.p, q.data(), (size_t)nlag * sizeof(double), cudaMemcpyHostToDevice));
    d_q2 = c->rmat.as<double>();
  }
  const size_t abytes = (size_t)N * N * sizeof(double2);
  const size_t bbytes = (size_t)N * nch * sizeof(double2);
  TRY(c->A64.ensure(abytes));
  TRY(c->B64.ensure(bbytes));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->A64.p, cmat, abytes, cudaMemcpyHostToDevice, c->stream));
  HPR_CUDA_TRY(cudaMemcpyAsync(c->B64.p, X.data(), bbytes, cudaMemcpyHostToDevice, c->stream));
  int s = solve_dense_core(c, c->A64.as<double2>(), c->B64.as<double2>(), N, nch, stats, d_q2, nlag);
  if (stats) stats->status = s;
  if (s != HPRMAT_B200_OK && s != HPRMAT_B200_NOT_CONVERGED) return s;
  HPR_CUDA_TRY(cudaMemcpyAsync(X.data(), c->B64.p, bbytes, cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  // Rmat(ich, ichp) = normfac * sum_r B(r) X(r + (ich-1) nlag, ichp): complex products
  for (int jp = 0; jp < nch; ++jp)
    for (int i = 0; i < nch; ++i) {
      double ar = 0.0, ai = 0.0;
      for (int r = 0; r < nlag; ++r) {
        size_t idx = (size_t)(i * nlag + r) + (size_t)jp * N;
        double br = bvec[2 * r], bi = bvec[2 * r + 1];
        double xr = X[2 * idx], xi = X[2 * idx + 1];
        ar += br * xr - bi * xi;
        ai += br * xi + bi * xr;
      }
      rmat[2 * (i + (size_t)jp * nch)] = ar * normfac;
      rmat[2 * (i + (size_t)jp * nch) + 1] = ai * normfac;
    }
  return s;
}

// ---- Fortran-convention drop-ins on a lazily created device-0 context
static std::mutex g_default_mu;
static hprmat_b200_ctx* g_default = nullptr;

static int default_ctx(hprmat_b200_ctx** out) {
  if (!g_default) TRY(hprmat_b200_create(0, nullptr, &g_default));
  *out = g_default;
  return HPRMAT_B200_OK;
}

static int fortran_info(int s, const hprmat_b200_stats& st) {
  switch (s) {
    case HPRMAT_B200_OK: return 0;
    case HPRMAT_B200_SINGULAR: return st.info > 0 ? st.info : 1;
    case HPRMAT_B200_NOT_CONVERGED: return 99;
    case HPRMAT_B200_ERR_OOM: return -2;
    case HPRMAT_B200_ERR_NODEVICE: return -1;
    default: return -1;
  }
}

int gpu_b200_solve_mixed_(double* A, double* B, int* n, int* nrhs, int* max_refine, double* tol, int* info) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  hprmat_b200_ctx* c = nullptr;
  int s = default_ctx(&c);
  hprmat_b200_stats st{};
  if (s == HPRMAT_B200_OK) {
    hprmat_b200_opts o = c->opts;
    o.precision = HPRMAT_B200_PREC_MIXED;
    o.max_refine = max_refine ? std::max(0, std::min(8, *max_refine)) : 3;
    o.tol = (tol && *tol > 0) ? *tol : 1.0e-13;
    s = hprmat_b200_set_opts(c, &o);
    if (s == HPRMAT_B200_OK) s = hprmat_b200_solve_linear(c, A, B, *n, *nrhs, &st);
  }
  if (info) *info = fortran_info(s, st);
  return (s == HPRMAT_B200_OK) ? 0 : -1;
}

int gpu_b200_solve_double_(double* A, double* B, int* n, int* nrhs, int* info) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  hprmat_b200_ctx* c = nullptr;
  int s = default_ctx(&c);
  hprmat_b200_stats st{};
  if (s == HPRMAT_B200_OK) {
    hprmat_b200_opts o = c->opts;
    o.precision = HPRMAT_B200_PREC_FP64;
    s = hprmat_b200_set_opts(c, &o);
    if (s == HPRMAT_B200_OK) s = hprmat_b200_solve_linear(c, A, B, *n, *nrhs, &st);
  }
  if (info) *info = fortran_info(s, st);
  return (s == HPRMAT_B200_OK) ? 0 : -1;
}

int gpu_b200_finalize_(void) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  int s = hprmat_b200_destroy(g_default);
  g_default = nullptr;
  return s;
}

// ---- kernel-level hooks (include/hprmat_b200_dev.h)
int hprmat_b200_dev_set_profile(hprmat_b200_ctx* c, int enable) {
  TRY(check_ctx(c));
  c->profile = enable != 0;
  if (c->profile && c->ev.empty()) {
    c->ev.resize(2 * 2048);
    for (auto& e : c->ev) HPR_CUDA_TRY(cudaEventCreate(&e));
  }
  c->ev_used = 0;
  c->ev_flops.clear();
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_wave_trace(hprmat_b200_ctx* c, int enable) {
  TRY(check_ctx(c));
  c->wave_trace = enable != 0;
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_wave_trace_read(hprmat_b200_ctx* c, long long* out, int cap, int* units) {
  TRY(check_ctx(c));
  if (!out || !units || cap < 0) return fail(HPRMAT_B200_ERR_ARG, "null output");
  *units = c->wtrace_units;
  const size_t n = std::min((size_t)cap, (size_t)c->wtrace_units * 8);
  if (n && c->wtrace.p) {
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    HPR_CUDA_TRY(cudaMemcpy(out, c->wtrace.p, n * sizeof(long long), cudaMemcpyDeviceToHost));
  }
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_panel_trace_read(hprmat_b200_ctx* c, long long* out, int cap, int* width) {
  TRY(check_ctx(c));
  if (!out || !width || cap < 0) return fail(HPRMAT_B200_ERR_ARG, "null output");
  *width = kPanelTraceW;
  const size_t n = std::min((size_t)cap, c->ptrace.bytes / sizeof(long long));
  if (n && c->ptrace.p) {
    HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    HPR_CUDA_TRY(cudaMemcpy(out, c->ptrace.p, n * sizeof(long long), cudaMemcpyDeviceToHost));
  }
  return HPRMAT_B200_OK;
}

long long hprmat_b200_dev_factorizations(hprmat_b200_ctx* c, int reset) {
  if (!c) return -1;
  long long n = c->factorizations;
  for (hprmat_b200_ctx* w : c->scan_workers) n += w->factorizations;
  if (reset) {
    c->factorizations = 0;
    for (hprmat_b200_ctx* w : c->scan_workers) w->factorizations = 0;
  }
  return n;
}

int hprmat_b200_dev_mesh(int nr, int ns, double rmax, double* tc, double* blo, double* q2, double* q1,
                         double* zrma) {
  if (nr < 2 || ns < 1 || !(rmax > 0)) return fail(HPRMAT_B200_ERR_ARG, "dev_mesh: need nr >= 2, ns >= 1, rmax > 0");
  std::vector<double> xle, wle, t, b, v2, v1, z;
  build_mesh_host(nr, ns, rmax, xle, wle, t, b, v2, v1, z);
  if (tc) std::copy(t.begin(), t.end(), tc);
  if (blo) std::copy(b.begin(), b.end(), blo);
  if (q2) std::copy(v2.begin(), v2.end(), q2);
  if (q1) std::copy(v1.begin(), v1.end(), q1);
  if (zrma) std::copy(z.begin(), z.end(), zrma);
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_set_tuning(hprmat_b200_ctx* c, const char* key, int value) {
  TRY(check_ctx(c));
  if (!key) return fail(HPRMAT_B200_ERR_ARG, "null key");
  if (strcmp(key, "gmres_m") == 0) {
    if (value < 1 || value > kGmresMaxM) return fail(HPRMAT_B200_ERR_ARG, "gmres_m must be in 1..%d", kGmresMaxM);
    c->gmres_m = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "inner_tol0_exp") == 0) {
    if (value < 1 || value > 15) return fail(HPRMAT_B200_ERR_ARG, "inner_tol0_exp must be in 1..15");
    c->inner_tol0 = pow(10.0, -value);
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "zero_start") == 0) {
    c->zero_start = value != 0;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "panel_cluster") == 0) {
    c->panel_cluster = value != 0;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "tc_grid") == 0) {
    if (value < 0) return fail(HPRMAT_B200_ERR_ARG, "tc_grid must be >= 0");
    c->tcplan.max_grid = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "growth_limit_exp") == 0) {
    if (value < -30 || value > 30) return fail(HPRMAT_B200_ERR_ARG, "growth_limit_exp must be in -30..30");
    c->growth_limit = pow(10.0, value);
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "reuse_max_inner") == 0) {
    if (value < 0) return fail(HPRMAT_B200_ERR_ARG, "reuse_max_inner must be >= 0");
    c->reuse_max_inner = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "hess_blocked") == 0) {
    c->hess_blocked = value != 0;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "f64_pair") == 0) {
    c->f64_pair = value != 0;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "hess_workers") == 0) {  // shifted scan: blocks in flight at once, 1..8
    if (value < 1 || value > 8) return fail(HPRMAT_B200_ERR_ARG, "hess_workers must be 1..8");
    c->hess_workers = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "hess_cluster") == 0) {  // CTAs of the column step's cluster: 8 or 16 (0: choose)
    if (value != 0 && value != 8 && value != 16) return fail(HPRMAT_B200_ERR_ARG, "hess_cluster must be 0, 8 or 16");
    c->hb_cluster = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "panel_rpc_min") == 0) {
    if (value < 1) return fail(HPRMAT_B200_ERR_ARG, "panel_rpc_min must be positive");
    c->panel_rpc_min = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "wave") == 0) {
    c->wave_enabled = value != 0;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "tc_trsm") == 0) {
    c->tc_trsm = value != 0;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "wave_sb") == 0) {
    if (value != 0 && value != 1 && value != 2 && value != 4)
      return fail(HPRMAT_B200_ERR_ARG, "wave_sb must be 0 (automatic), 1, 2 or 4");
    c->wave_sb = value;
    return HPRMAT_B200_OK;
  }
  if (strcmp(key, "wave_un") == 0) {
    if (value != 0 && value != 64 && value != 128)
      return fail(HPRMAT_B200_ERR_ARG, "wave_un must be 0 (automatic), 64 or 128");
    c->wave_un = value;
    return HPRMAT_B200_OK;
  }
  return fail(HPRMAT_B200_ERR_ARG, "unknown tuning key '%s'", key);
}

int hprmat_b200_dev_counters(hprmat_b200_ctx* c, unsigned long long* launches, double* tc_ms, double* tc_flops,
                             int* tc_launches, int reset) {
  if (!c) return fail(HPRMAT_B200_ERR_ARG, "null context");
  if (launches) *launches = c->launches;
  if (tc_ms) *tc_ms = c->tc_ms;
  if (tc_flops) *tc_flops = c->tc_flops;
  if (tc_launches) *tc_launches = c->tc_launches;
  if (reset) {
    c->launches = 0;
    c->tc_ms = c->tc_flops = 0.0;
    c->tc_launches = 0;
  }
  return HPRMAT_B200_OK;
}

__global__ void split_planes_kernel(const float2* __restrict__ src, int rows, int nb, float* dst, long plane) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)rows * nb) return;
  float2 v = src[idx];
  float hr, lr, hi, li;
  tf32_split(v.x, hr, lr);
  tf32_split(v.y, hi, li);
  dst[idx] = hr;
  dst[plane + idx] = lr;
  dst[2 * plane + idx] = hi;
  dst[3 * plane + idx] = li;
}

int hprmat_b200_dev_zgemm(hprmat_b200_ctx* c, const void* A, long lda, const void* B, long ldb, void* C, long ldc,
                          int M, int N, int K) {
  TRY(check_ctx(c));
  if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return fail(HPRMAT_B200_ERR_ARG, "dev_zgemm: invalid arguments");
  TRY(zgemm_update(c, M, N, K, (const double2*)A, lda, (const double2*)B, ldb, (double2*)C, ldc));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_hess_timings(hprmat_b200_ctx* c, double* ms, int* counts, int reset) {
  TRY(check_ctx(c));
  if (ms) std::copy(c->hess_ms, c->hess_ms + 6, ms);
  if (counts) {
    counts[0] = c->hess_steps_last;
    counts[1] = c->hess_fallback_last;
  }
  if (reset) std::fill(c->hess_ms, c->hess_ms + 6, 0.0);
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_hessenberg(hprmat_b200_ctx* c, void* A, long lda, int N, void* P) {
  TRY(check_ctx(c));
  if (!A || !P || N < 3 || lda < N) return fail(HPRMAT_B200_ERR_ARG, "dev_hessenberg: invalid arguments");
  TRY(hess_reduce(c, (double2*)A, lda, N, (double2*)P));
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_binary_version(void) {
  cudaFuncAttributes fa;
  const cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)split_planes_kernel);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(HPRMAT_B200_ERR_NODEVICE, "no device can load the library's kernels: %s", cudaGetErrorString(e));
  }
  return fa.binaryVersion;
}

int hprmat_b200_dev_split_planes(hprmat_b200_ctx* c, const void* src, int rows, int nb, float* dst, long plane) {
  TRY(check_ctx(c));
  if (!src || !dst || rows <= 0 || nb <= 0 || plane < (long)rows * nb) return fail(HPRMAT_B200_ERR_ARG, "split_planes: invalid arguments");
  long n = (long)rows * nb;
  split_planes_kernel<<<cdiv_u(n, 256), 256, 0, c->stream>>>((const float2*)src, rows, nb, dst, plane);
  LAUNCH_CHECK();
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return HPRMAT_B200_OK;
}

int hprmat_b200_dev_tc_update(hprmat_b200_ctx* c, const float* aop, const float* bop, long plane, int nb, void* C,
                              long ldc, int M, int Nc, int bn) {
  TRY(check_ctx(c));
  if (!aop || !bop || !C || M <= 0 || Nc <= 0 || ldc < M || nb < 16 || (nb % 16) || (bn != 128 && bn != 256) ||
      plane < (long)std::max(M, Nc) * nb || ((uintptr_t)aop & 15) || ((uintptr_t)bop & 15) || (plane % 4))
    return fail(HPRMAT_B200_ERR_ARG, "dev_tc_update: invalid arguments");
  TcOperand A, B;
  if (tc_make_operand(c->tcplan, A, aop, nb, plane / nb, nb, plane, 128) ||
      tc_make_operand(c->tcplan, B, bop, nb, plane / nb, nb, plane, bn))
    return fail(HPRMAT_B200_ERR_ARG, "%s", hprmat_b200_last_error());
  if (tc_update(c->tcplan, A, 0, 0, B, 0, 0, nb, (float2*)C, ldc, M, Nc, bn, c->stream))
    return fail(HPRMAT_B200_ERR_CUDA, "%s", hprmat_b200_last_error());
  HPR_CUDA_TRY(cudaStreamSynchronize(c->stream));
  int err = 0;
  TRY(tc_gemm_check(c->tcplan, c->stream, &err));
  if (err) return fail(HPRMAT_B200_ERR_TIMEOUT, "tensor-core update: wait limit exceeded at site %d", err);
  return HPRMAT_B200_OK;
}

int hprmat_b200_boundary(int nch, const int* lval, const double* qk, const double* eta, double rmax, double* co,
                         double* cop, double* xc1, double* xc2, int* nopen) {
  if (nch <= 0 || !lval || !qk || !eta || !(rmax > 0)) return fail(HPRMAT_B200_ERR_ARG, "boundary: invalid arguments");
  int no = 0;
  for (int c = 0; c < nch; ++c) {
    if (co) co[2 * c] = co[2 * c + 1] = 0.0;
    if (cop) cop[2 * c] = cop[2 * c + 1] = 0.0;
    if (xc1) xc1[c] = 0.0;
    if (xc2) xc2[c] = 0.0;
    if (lval[c] < 0) return fail(HPRMAT_B200_ERR_ARG, "lval(%d) < 0", c + 1);
    if (qk[c] > 0) {
      CoulombFG f = coulfg_single(qk[c] * rmax, eta[c], (double)lval[c]);
      if (f.ifail != 0) return fail(HPRMAT_B200_ERR_ARG, "COULFG failed (ifail=%d) for channel %d", f.ifail, c + 1);
      if (co) { co[2 * c] = f.g; co[2 * c + 1] = f.f; }
      if (cop) { cop[2 * c] = f.gp * qk[c] * rmax; cop[2 * c + 1] = f.fp * qk[c] * rmax; }
      ++no;
    } else {
      WhitOut w = whit_l(eta[c], rmax, -qk[c], lval[c]);
      if (xc1) xc1[c] = rmax * w.wd / w.w;
      if (xc2) xc2[c] = w.w;
    }
  }
  if (nopen) *nopen = no;
  return HPRMAT_B200_OK;
}

const char* hprmat_b200_status_string(int s) {
  switch (s) {
    case HPRMAT_B200_OK: return "ok";
    case HPRMAT_B200_ERR_ARG: return "invalid argument";
    case HPRMAT_B200_ERR_CUDA: return "CUDA error";
    case HPRMAT_B200_ERR_OOM: return "device out of memory";
    case HPRMAT_B200_ERR_TIMEOUT: return "device wait limit exceeded";
    case HPRMAT_B200_ERR_UNSUPPORTED: return "unsupported input";
    case HPRMAT_B200_ERR_NODEVICE: return "no usable sm_100 device";
    case HPRMAT_B200_SINGULAR: return "singular matrix";
    case HPRMAT_B200_PIVOT_GROWTH: return "pivot growth exceeded";
    case HPRMAT_B200_NOT_CONVERGED: return "refinement did not converge";
  }
  return "unknown status";
}

const char* hprmat_b200_last_error(void) { return g_last_error.c_str(); }

int hprmat_b200_version(void) { return HPRMAT_B200_ABI_VERSION; }

}  // extern "C"

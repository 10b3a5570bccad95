"""Host-side mirror of HPRMAT's R-matrix interface on the B200 solver.

Names and argument meanings follow the reference:
  * ``rmat_ini(nr, ns, rmax) -> zrma``                     (src/rmatrix_hp.F90:61)
  * ``rmatrix(nch, lval, qk, eta, rmax, nr, ns, cpot) -> (cu, nopen)``
                                                            (src/rmatrix_hp.F90:175-176)
  * ``solve_rmatrix(cmat, B_vector, nch, nlag, normfac, solver_type=7) -> Rmat``
                                                            (src/rmat_solvers.F90:49)
  * ``RMatrixSolver(nr, ns, rmax).solve(lval, qk, eta, cpot) -> (cu, nopen)``
                                                            (bindings/python/hprmat.py:79-163)
``solver_type`` 7 is this backend; precision "mixed" (default) or "fp64" selects the
factorisation arithmetic.  Errors raise ``HprmatError``; a collision matrix whose
refinement stopped above the tolerance raises as well unless ``allow_unconverged``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat
from ._native import HprmatError, Stats

SOLVER_B200 = nat.SOLVER_B200

_PREC = {"mixed": nat.PREC_MIXED, "fp64": nat.PREC_FP64}


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _fortran_device(t):
    """A torch CUDA tensor (d0, d1, d2) as contiguous Fortran-order (column-major) memory: the
    returned tensor's storage is t laid out with d0 fastest (a copy only when t is not already
    so), for device pointers handed to the C ABI."""
    return t.permute(2, 1, 0).contiguous()


class Context:
    """One device context (stream + device buffers) of the C library."""

    def __init__(self, device: int = 0, precision: str = "mixed", max_refine: int = 3, tol: float = 1e-12,
                 panel_nb: int = 0, surface_tol: float = 1e-11, reuse_factors: bool = False):
        self._lib = nat.load()
        self._h = ctypes.c_void_p()
        self.opts = nat.Opts()
        self._lib.hprmat_b200_default_opts(ctypes.byref(self.opts))
        self.opts.precision = _PREC[precision]
        self.opts.max_refine = int(max_refine)
        self.opts.tol = float(tol)
        self.opts.surface_tol = float(surface_tol)
        self.opts.panel_nb = int(panel_nb)
        self.opts.reuse_factors = int(bool(reuse_factors))
        nat.check(self._lib.hprmat_b200_create(int(device), ctypes.byref(self.opts), ctypes.byref(self._h)))
        self.device = device
        self.mesh = None
        self._mesh_key = None
        self.last_stats = None

    def close(self):
        if self._h:
            self._lib.hprmat_b200_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_reuse_factors(self, enable: bool):
        """opts.reuse_factors: successive rmatrix calls on the same channel block (energy scans)
        refine with the held factorisation instead of factorising every energy."""
        self.opts.reuse_factors = int(bool(enable))
        nat.check(self._lib.hprmat_b200_set_opts(self._h, ctypes.byref(self.opts)))

    def set_estimate_condition(self, enable: bool):
        """opts.estimate_condition: FP64 factorisations also estimate the 1-norm condition number
        of the factorised matrix (``last_stats["cond_estimate"]``, as LAPACK ZGECON's 1/rcond)."""
        self.opts.estimate_condition = int(bool(enable))
        nat.check(self._lib.hprmat_b200_set_opts(self._h, ctypes.byref(self.opts)))

    def set_precision(self, precision: str, max_refine: int | None = None, tol: float | None = None,
                      surface_tol: float | None = None):
        self.opts.precision = _PREC[precision]
        if surface_tol is not None:
            self.opts.surface_tol = float(surface_tol)
        if max_refine is not None:
            self.opts.max_refine = int(max_refine)
        if tol is not None:
            self.opts.tol = float(tol)
        nat.check(self._lib.hprmat_b200_set_opts(self._h, ctypes.byref(self.opts)))

    def set_stream(self, stream_handle: int | None):
        nat.check(self._lib.hprmat_b200_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    # -- rmat_ini ---------------------------------------------------------------
    def rmat_ini(self, nr: int, ns: int, rmax: float) -> np.ndarray:
        zrma = np.zeros(nr * ns, dtype=np.float64)
        nat.check(self._lib.hprmat_b200_rmat_ini(self._h, int(nr), int(ns), float(rmax), _dptr(zrma)))
        self.mesh = zrma
        self._mesh_key = (int(nr), int(ns), float(rmax))
        return zrma

    def _ensure_mesh(self, nr, ns, rmax):
        if self._mesh_key != (int(nr), int(ns), float(rmax)):
            self.rmat_ini(nr, ns, rmax)

    # -- rmatrix ----------------------------------------------------------------
    def _full(self, nch, lval, qk, eta, rmax, nr, ns, cpot, ndim, nvc, cpnl, allow_unconverged):
        """hprmat_b200_rmatrix_full: wave functions when nvc is given, non-local cpnl if given."""
        self._ensure_mesh(nr, ns, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cpot = np.asfortranarray(cpot, dtype=np.complex128)
        ncp1 = cpot.shape[0]
        ndim = int(ndim or cpot.shape[1])
        cu = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        twf = nvc is not None
        nvc_a = np.ascontiguousarray(nvc if twf else [1], dtype=np.int32)
        cf = np.zeros((nr * ns, nch, len(nvc_a)) if twf else (1, 1, 1), dtype=np.complex128, order="F")
        if cpnl is not None:
            cpnl = np.asfortranarray(cpnl, dtype=np.complex128)
            ncp2, nl_ptr = cpnl.shape[0], _dptr(cpnl)
        else:
            ncp2, nl_ptr = 0, None
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix_full(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                               int(nr), int(ns), _dptr(cpot), int(ncp1), ndim, _dptr(cu),
                                               ctypes.byref(nopen), int(twf), _dptr(cf), cf.shape[0], cf.shape[1],
                                               len(nvc_a), _iptr(nvc_a), int(ncp2), nl_ptr, ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return cu, nopen.value, (cf if twf else None)

    def rmatrix(self, nch, lval, qk, eta, rmax, nr, ns, cpot, ndim=None, allow_unconverged=False, cpnl=None):
        """Collision matrix ``cu`` (ndim x ndim, U in cu[:nopen, :nopen]) and ``nopen``.
        ``cpnl``: non-local potential (ncp2 >= nr^2, nch, nch), one interval only."""
        if cpnl is not None:
            cu, nopen, _ = self._full(nch, lval, qk, eta, rmax, nr, ns, cpot, ndim, None, cpnl, allow_unconverged)
            return cu, nopen
        self._ensure_mesh(nr, ns, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cpot = np.asfortranarray(cpot, dtype=np.complex128)
        ncp1 = cpot.shape[0]
        ndim = int(ndim or cpot.shape[1])
        cu = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                          int(nr), int(ns), _dptr(cpot), int(ncp1), ndim,
                                          _dptr(cu), ctypes.byref(nopen), ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return cu, nopen.value

    def rmatrix_scan(self, blocks, rmax, nr, nworkers=0, allow_unconverged=False, raise_on_unit_error=True,
                     method="lu"):
        """Batched energy scan.  ``blocks``: sequence of (lval, cpot, qk, eta) with qk/eta of
        shape (nenergies, nch), cpot (ncp1, nch, nch) complex, Fortran order.  Returns a list of
        (cu (nenergies, nch, nch) with U in cu[e, :nopen, :nopen], nopen (nenergies,),
        status (nenergies,)) and sets ``last_scan_seconds``.  ``method``: "lu" (every energy
        by its own LU on concurrent worker streams, hprmat_b200_rmatrix_scan) or "shifted" (one
        Hessenberg reduction per block and O(N^2 nch) per energy, hprmat_b200_rmatrix_scan_shifted;
        up to three blocks in flight on worker contexts; ``nworkers`` is not used).  For blocks of
        at most 64 channels the shifted method is the faster one: 1.61-1.63 s against 6.5-7.1 s on
        the 12-block, 3072-energy scan."""
        keep, arr, out = self._scan_blocks(blocks)
        self._ensure_mesh(nr, 1, rmax)
        blocks_c = (nat.ScanBlock * len(arr))(*arr)
        secs = ctypes.c_double(0.0)
        if method == "shifted":
            s = self._lib.hprmat_b200_rmatrix_scan_shifted(self._h, len(arr), blocks_c, float(rmax), int(nr),
                                                           ctypes.byref(secs))
        elif method == "lu":
            s = self._lib.hprmat_b200_rmatrix_scan(self._h, len(arr), blocks_c, float(rmax), int(nr), int(nworkers),
                                                   ctypes.byref(secs))
        else:
            raise ValueError(f"unknown scan method {method!r}")
        self.last_scan_seconds = secs.value
        if raise_on_unit_error:
            nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        # the library writes each U column-major (Fortran) into its (nch, nch) slot
        return [(np.ascontiguousarray(cu.transpose(0, 2, 1)), nopen, status) for cu, nopen, status in out]

    TUNE_KEYS = ("N", "nb", "panel_cluster", "panel_rpc_min", "wave_sb", "gmres_m", "tc_grid")

    def scan_autotune(self, blocks, rmax, nr, nworkers=0):
        """Autotune the scan's per-order settings on these blocks (hprmat_b200_scan_autotune);
        returns the table (``scan_tune_table``) and sets ``last_autotune_seconds``."""
        keep, arr, _out = self._scan_blocks(blocks)
        self._ensure_mesh(nr, 1, rmax)
        blocks_c = (nat.ScanBlock * len(arr))(*arr)
        secs = ctypes.c_double(0.0)
        nat.check(self._lib.hprmat_b200_scan_autotune(self._h, len(arr), blocks_c, float(rmax), int(nr),
                                                      int(nworkers), ctypes.byref(secs)))
        self.last_autotune_seconds = secs.value
        del keep
        return self.scan_tune_table()

    def scan_tune_table(self):
        """The autotuner's rows as dicts (keys TUNE_KEYS and the trial time ``ms``)."""
        n = self._lib.hprmat_b200_scan_tune_get(self._h, None, None, 0)
        rows = np.zeros((max(n, 1), len(self.TUNE_KEYS)), np.int32)
        ms = np.zeros(max(n, 1))
        self._lib.hprmat_b200_scan_tune_get(self._h, _iptr(rows), _dptr(ms), n)
        return [dict(zip(self.TUNE_KEYS, map(int, rows[i])), ms=float(ms[i])) for i in range(n)]

    def set_scan_tune_table(self, table):
        """Load a table (rows as ``scan_tune_table`` returns them, e.g. from a JSON cache)."""
        rows = np.array([[int(r.get(k, 0)) for k in self.TUNE_KEYS] for r in table], np.int32).reshape(
            -1, len(self.TUNE_KEYS))
        nat.check(self._lib.hprmat_b200_scan_tune_set(self._h, _iptr(np.ascontiguousarray(rows)), len(rows)))

    @staticmethod
    def _scan_blocks(blocks):
        """ScanBlock records for (lval, cpot, qk, eta) blocks, the arrays they point into (keep
        them alive) and the output arrays (cu, nopen, status) per block."""
        keep, arr, out = [], [], []
        for lval, cpot, qk, eta in blocks:
            lval = np.ascontiguousarray(lval, dtype=np.int32)
            cpot = np.asfortranarray(cpot, dtype=np.complex128)
            qk = np.ascontiguousarray(np.atleast_2d(qk), dtype=np.float64)
            eta = np.ascontiguousarray(np.atleast_2d(eta), dtype=np.float64)
            nE, nch = qk.shape
            if cpot.shape[1] != nch or eta.shape != qk.shape or lval.shape[0] != nch:
                raise ValueError("rmatrix_scan: inconsistent block shapes")
            cu = np.zeros((nE, nch, nch), dtype=np.complex128)       # per energy (nch, nch) row-major view
            nopen = np.zeros(nE, dtype=np.int32)
            status = np.zeros(nE, dtype=np.int32)
            keep += [lval, cpot, qk, eta]
            b = nat.ScanBlock(nch, _iptr(lval), _dptr(cpot), cpot.shape[0], nE, _dptr(qk), _dptr(eta), _dptr(cu),
                              _iptr(nopen), _iptr(status))
            arr.append(b)
            out.append((cu, nopen, status))
        return keep, arr, out

    def rmatrix_adjoint(self, nch, lval, qk, eta, rmax, nr, cpot, gu):
        """Collision matrix and the gradient of a real loss with respect to the potential.
        ``gu``: dL/dU in the convention dL = Re sum conj(gu) dU (PyTorch's), nopen x nopen or
        larger.  Returns (cu, nopen, grad) with grad shaped like cpot (same convention)."""
        self._ensure_mesh(nr, 1, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cpot = np.asfortranarray(cpot, dtype=np.complex128)
        ncp1, ndim = cpot.shape[0], cpot.shape[1]
        g = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        gu = np.asarray(gu, dtype=np.complex128)
        g[:gu.shape[0], :gu.shape[1]] = gu
        cu = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        grad = np.zeros_like(cpot, order="F")
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix_adjoint(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                                  int(nr), 1, _dptr(cpot), int(ncp1), int(ndim), _dptr(g), _dptr(cu),
                                                  ctypes.byref(nopen), _dptr(grad), ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s)
        return cu, nopen.value, grad

    def rmatrix_wf(self, nch, lval, qk, eta, rmax, nr, ns, cpot, nvc=(1,), ndim=None, allow_unconverged=False,
                   cpnl=None):
        """Collision matrix and internal wave functions (rmatrix with twf = .true.).  ``nvc``:
        entrance channels, 1-based among the open channels.  Returns (cu, nopen, cf) with cf
        complex (nr*ns, nch, len(nvc)) at the mesh points and the closed-channel amplitudes in
        cu[nopen:, ic].  ``cpnl``: non-local potential as in ``rmatrix``."""
        if cpnl is not None:
            return self._full(nch, lval, qk, eta, rmax, nr, ns, cpot, ndim, list(nvc), cpnl, allow_unconverged)
        self._ensure_mesh(nr, ns, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        nvc = np.ascontiguousarray(nvc, dtype=np.int32)
        cpot = np.asfortranarray(cpot, dtype=np.complex128)
        ncp1 = cpot.shape[0]
        ndim = int(ndim or cpot.shape[1])
        cu = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        cf = np.zeros((nr * ns, nch, len(nvc)), dtype=np.complex128, order="F")
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix_wf(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                             int(nr), int(ns), _dptr(cpot), int(ncp1), ndim, _dptr(cu),
                                             ctypes.byref(nopen), len(nvc), _iptr(nvc), _dptr(cf), nr * ns, int(nch),
                                             ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return cu, nopen.value, cf

    def rmatrix_x(self, nch, lval, qk, eta, rmax, nr, cpot, allow_unconverged=False):
        """rmatrix (one interval) that also returns the refined forward solution X = C^-1 Q as a
        torch CUDA tensor (nch*nr, nch) complex128, for ``adjoint_from_x``."""
        import torch
        self._ensure_mesh(nr, 1, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cpot = np.asfortranarray(cpot, dtype=np.complex128)
        ncp1, ndim = cpot.shape[0], cpot.shape[1]
        n = int(nch) * int(nr)
        x = torch.empty((int(nch), n), dtype=torch.complex128, device=f"cuda:{self.device}")  # column-major X
        cu = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix_x(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                            int(nr), _dptr(cpot), int(ncp1), int(ndim), _dptr(cu),
                                            ctypes.byref(nopen), ctypes.c_void_p(x.data_ptr()), n, ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return cu, nopen.value, x.T

    def rmatrix_x_device(self, nch, lval, qk, eta, rmax, nr, cpot, allow_unconverged=False):
        """rmatrix_x with the potential already on this context's device: ``cpot`` is a torch
        CUDA tensor (ncp1, nch, nch) complex128 (any strides).  Returns (U as a torch CUDA tensor
        (ndim, ndim), nopen, X as a torch CUDA tensor (nch*nr, nch)); nothing of size cpot or X
        crosses to the host."""
        import torch
        self._ensure_mesh(nr, 1, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cf = _fortran_device(cpot)
        ncp1, ndim = cpot.shape[0], cpot.shape[1]
        n = int(nch) * int(nr)
        x = torch.empty((int(nch), n), dtype=torch.complex128, device=cpot.device)  # column-major X
        d_cu = torch.empty((ndim, ndim), dtype=torch.complex128, device=cpot.device)  # column-major U (as U^T)
        # the library works on the context's own stream: the potential (and its copy) must be complete
        torch.cuda.current_stream(cpot.device).synchronize()
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix_x_device(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta),
                                                   float(rmax), int(nr), ctypes.c_void_p(cf.data_ptr()), int(ncp1),
                                                   int(ndim), ctypes.c_void_p(d_cu.data_ptr()), ctypes.byref(nopen),
                                                   ctypes.c_void_p(x.data_ptr()), n, ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return d_cu.T, nopen.value, x.T

    def adjoint_from_x_device(self, nch, lval, qk, eta, rmax, nr, cpot, cu, x, gu):
        """adjoint_from_x with cpot, x and the returned gradient as torch CUDA tensors (the
        gradient has cpot's shape); cu and gu (nopen-sized) may be host or device."""
        import torch
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cf = _fortran_device(cpot)
        ncp1, ndim = cpot.shape[0], cpot.shape[1]
        cu_h = np.asfortranarray(cu.detach().cpu().numpy() if torch.is_tensor(cu) else cu, dtype=np.complex128)
        g = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        gu_h = np.asarray(gu.detach().cpu().numpy() if torch.is_tensor(gu) else gu, dtype=np.complex128)
        g[:gu_h.shape[0], :gu_h.shape[1]] = gu_h
        xt = x.T
        assert xt.is_contiguous() and xt.shape == (int(nch), int(nch) * int(nr))
        grad = torch.empty((ndim, ndim, ncp1), dtype=torch.complex128, device=cpot.device)  # Fortran (ncp1, ndim, ndim)
        torch.cuda.current_stream(cpot.device).synchronize()
        s = self._lib.hprmat_b200_adjoint_from_x_device(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta),
                                                        float(rmax), int(nr), ctypes.c_void_p(cf.data_ptr()),
                                                        int(ncp1), int(ndim), _dptr(cu_h),
                                                        ctypes.c_void_p(xt.data_ptr()), int(nch) * int(nr), _dptr(g),
                                                        ctypes.c_void_p(grad.data_ptr()))
        nat.check(s)
        return grad.permute(2, 1, 0)

    def adjoint_from_x(self, nch, lval, qk, eta, rmax, nr, cpot, cu, x, gu):
        """Potential gradient of a real loss from the forward solution ``x`` of ``rmatrix_x``
        (symmetric potentials), in the convention of ``rmatrix_adjoint``."""
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        cpot = np.asfortranarray(cpot, dtype=np.complex128)
        ncp1, ndim = cpot.shape[0], cpot.shape[1]
        cu = np.asfortranarray(cu, dtype=np.complex128)
        g = np.zeros((ndim, ndim), dtype=np.complex128, order="F")
        gu = np.asarray(gu, dtype=np.complex128)
        g[:gu.shape[0], :gu.shape[1]] = gu
        xt = x.T  # (nch, n) row-major == column-major (n, nch)
        assert xt.is_contiguous() and xt.shape == (int(nch), int(nch) * int(nr))
        grad = np.zeros_like(cpot, order="F")
        s = self._lib.hprmat_b200_adjoint_from_x(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                                 int(nr), _dptr(cpot), int(ncp1), int(ndim), _dptr(cu),
                                                 ctypes.c_void_p(xt.data_ptr()), int(nch) * int(nr), _dptr(g),
                                                 _dptr(grad))
        nat.check(s)
        return grad

    def rmatrix_device(self, nch, lval, qk, eta, rmax, nr, ns, d_cpot, ncp1, ndim, d_cu, allow_unconverged=False):
        """Device-resident variant: ``d_cpot``/``d_cu`` are device addresses (ints)."""
        self._ensure_mesh(nr, ns, rmax)
        lval = np.ascontiguousarray(lval, dtype=np.int32)
        qk = np.ascontiguousarray(qk, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        nopen = ctypes.c_int(0)
        st = Stats()
        s = self._lib.hprmat_b200_rmatrix_device(self._h, int(nch), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax),
                                                 int(nr), int(ns), ctypes.c_void_p(d_cpot), int(ncp1), int(ndim),
                                                 ctypes.c_void_p(d_cu), ctypes.byref(nopen), ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return nopen.value

    # -- dense solves -------------------------------------------------------------
    def solve_linear(self, A, B, allow_unconverged=False):
        """X with A X = B (A: n x n, B: n x nrhs complex)."""
        A = np.asfortranarray(A, dtype=np.complex128)
        X = np.array(B, dtype=np.complex128, order="F", copy=True)
        if X.ndim == 1:
            X = X.reshape(-1, 1, order="F")
        n, nrhs = X.shape
        st = Stats()
        s = self._lib.hprmat_b200_solve_linear(self._h, _dptr(A), _dptr(X), n,
                                               nrhs, ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return X

    def solve_linear_device(self, d_A, d_B, n, nrhs, allow_unconverged=False):
        st = Stats()
        s = self._lib.hprmat_b200_solve_linear_device(self._h, ctypes.c_void_p(d_A), ctypes.c_void_p(d_B), int(n),
                                                      int(nrhs), ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))

    def solve_rmatrix(self, cmat, B_vector, nch, nlag, normfac=1.0, allow_unconverged=False):
        cmat = np.asfortranarray(cmat, dtype=np.complex128)
        b = np.ascontiguousarray(B_vector, dtype=np.complex128)
        rm = np.zeros((nch, nch), dtype=np.complex128, order="F")
        st = Stats()
        s = self._lib.hprmat_b200_solve_rmatrix(self._h, _dptr(cmat), _dptr(b),
                                                int(nch), int(nlag), float(normfac), _dptr(rm),
                                                ctypes.byref(st))
        self.last_stats = st.as_dict()
        nat.check(s, (nat.OK, nat.NOT_CONVERGED) if allow_unconverged else (nat.OK,))
        return rm


def boundary_values(lval, qk, eta, rmax):
    """Per-channel (co, cop, xc1, xc2, nopen) at the channel radius (host computation)."""
    lib = nat.load()
    lval = np.ascontiguousarray(lval, dtype=np.int32)
    qk = np.ascontiguousarray(qk, dtype=np.float64)
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    n = len(lval)
    co = np.zeros(n, np.complex128)
    cop = np.zeros(n, np.complex128)
    xc1 = np.zeros(n)
    xc2 = np.zeros(n)
    nopen = ctypes.c_int(0)
    nat.check(lib.hprmat_b200_boundary(n, _iptr(lval), _dptr(qk), _dptr(eta), float(rmax), _dptr(co),
                                       _dptr(cop), _dptr(xc1), _dptr(xc2), ctypes.byref(nopen)))
    return co, cop, xc1, xc2, nopen.value


_default: Context | None = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context()
    return _default


def rmat_ini(nr: int, ns: int, rmax: float) -> np.ndarray:
    return default_context().rmat_ini(nr, ns, rmax)


def rmatrix(nch, lval, qk, eta, rmax, nr, ns, cpot, precision: str | None = None):
    ctx = default_context()
    if precision is not None:
        ctx.set_precision(precision)
    return ctx.rmatrix(nch, lval, qk, eta, rmax, nr, ns, cpot)


def solve_rmatrix(cmat, B_vector, nch, nlag, normfac=1.0, solver_type=SOLVER_B200, precision: str | None = None):
    if solver_type != SOLVER_B200:
        raise ValueError(f"this backend is solver_type {SOLVER_B200}")
    ctx = default_context()
    if precision is not None:
        ctx.set_precision(precision)
    return ctx.solve_rmatrix(cmat, B_vector, nch, nlag, normfac)


def wf_print(lval, qk, eta, rmax, nr, ns, cu, nopen, cf, zrma, iv, nom, npoin, h):
    """Wave function of channel ``iv`` for entrance channel ``nom`` (1-based) on r = h, ...,
    npoin*h (src/rmatrix_hp.F90:678-734): spline inside rmax, Coulomb/Whittaker outside."""
    lib = nat.load()
    lval = np.ascontiguousarray(lval, dtype=np.int32)
    qk = np.ascontiguousarray(qk, dtype=np.float64)
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    cu = np.asfortranarray(cu, dtype=np.complex128)
    cf = np.asfortranarray(cf, dtype=np.complex128)
    if cf.ndim == 2:
        cf = cf[:, :, None]
    zrma = np.ascontiguousarray(zrma, dtype=np.float64)
    out = np.zeros(int(npoin), dtype=np.complex128)
    s = lib.hprmat_b200_wf_print(len(lval), _iptr(lval), _dptr(qk), _dptr(eta), float(rmax), int(nr), int(ns),
                                 _dptr(cu), cu.shape[0], int(nopen), _dptr(cf), cf.shape[0], cf.shape[1],
                                 _dptr(zrma), int(iv), int(nom), int(npoin), float(h), _dptr(out))
    nat.check(s)
    return out


class RMatrixSolver:
    """Mirror of the reference Python binding's ``RMatrixSolver`` for solver type 7
    (bindings/python/hprmat.py:79-303)."""

    def __init__(self, nr, ns, rmax, solver=SOLVER_B200, device=0, precision="mixed"):
        if solver != SOLVER_B200:
            raise ValueError(f"this backend is solver type {SOLVER_B200}")
        self.nr, self.ns, self.rmax, self.solver = int(nr), int(ns), float(rmax), int(solver)
        self.ctx = Context(device=device, precision=precision)
        self.mesh = self.ctx.rmat_ini(self.nr, self.ns, self.rmax)

    def solve(self, lval, qk, eta, cpot, solver=None):
        lval = np.asarray(lval, dtype=np.int32)
        cu, nopen = self.ctx.rmatrix(len(lval), lval, qk, eta, self.rmax, self.nr, self.ns, cpot)
        return cu, nopen

    def solve_with_wavefunction(self, lval, qk, eta, cpot, entrance_channels=None, solver=None):
        """(cu, cf, nopen) with cf (nr*ns, nch, n_entrance) as the reference binding
        (bindings/python/hprmat.py:165-207); entrance channels 1-based, default [1]."""
        lval = np.asarray(lval, dtype=np.int32)
        nvc = [1] if entrance_channels is None else list(entrance_channels)
        cu, nopen, cf = self.ctx.rmatrix_wf(len(lval), lval, qk, eta, self.rmax, self.nr, self.ns, cpot, nvc)
        return cu, cf, nopen

    def solve_nonlocal(self, lval, qk, eta, cpot, cpnl, entrance_channels=None, solver=None):
        """(cu, cf, nopen) with a non-local potential cpnl (nr*nr, nch, nch), as the reference
        binding (bindings/python/hprmat.py:209-252)."""
        lval = np.asarray(lval, dtype=np.int32)
        nvc = [1] if entrance_channels is None else list(entrance_channels)
        cu, nopen, cf = self.ctx.rmatrix_wf(len(lval), lval, qk, eta, self.rmax, self.nr, self.ns, cpot, nvc,
                                            cpnl=cpnl)
        return cu, cf, nopen

    def interpolate_wavefunction(self, lval, qk, eta, cu, cf, nopen, channel, entrance, npoin, h=None):
        """(r, wf) on r = h, ..., npoin*h (bindings/python/hprmat.py:254-303); h defaults to
        2 rmax / npoin."""
        if h is None:
            h = 2.0 * self.rmax / npoin
        wf = wf_print(lval, qk, eta, self.rmax, self.nr, self.ns, cu, nopen, cf, self.mesh, channel, entrance,
                      npoin, h)
        return np.arange(1, npoin + 1) * h, wf

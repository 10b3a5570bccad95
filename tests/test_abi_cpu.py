"""C ABI checks that need no GPU: the library loads, exports every declared symbol, and
its host-side pieces agree with the oracle."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from hprmat_b200 import _native as nat
from hprmat_b200 import api, workloads
from oracle import rmatrix_oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in ("hprmat_b200.h", "hprmat_b200_dev.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b((?:hprmat_b200|gpu_b200)_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = nat.load()
    declared = _declared()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(nat.EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True, text=True).stdout
    for name in declared:
        assert re.search(r"\bT " + re.escape(name) + r"$", out, re.M), name


def test_abi_version_agrees_across_header_library_and_bindings():
    src = open(os.path.join(ROOT, "include", "hprmat_b200.h")).read()
    m = re.search(r"#define HPRMAT_B200_ABI_VERSION (\d+)", src)
    assert m and int(m.group(1)) == nat.ABI_VERSION == nat.load().hprmat_b200_version()


def test_library_build_targets_sm100a():
    """The build compiles every translation unit for sm_100a only (the runtime check of the
    loaded kernels' architecture is the GPU test test_kernels_report_sm100_binary)."""
    from hprmat_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_default_opts_and_status_strings():
    lib = nat.load()
    o = nat.Opts()
    lib.hprmat_b200_default_opts(ctypes.byref(o))
    assert o.precision == nat.PREC_MIXED and o.max_refine == 3 and o.tol == 1e-12 and o.surface_tol == 1e-11
    assert o.panel_nb == 0
    assert lib.hprmat_b200_status_string(nat.SINGULAR) == b"singular matrix"
    assert lib.hprmat_b200_status_string(nat.NOT_CONVERGED) == b"refinement did not converge"
    assert lib.hprmat_b200_status_string(nat.PIVOT_GROWTH) == b"pivot growth exceeded"
    assert o.estimate_condition == 0 and o.growth_error == 0


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(nat.HprmatError) as e:
        api.Context()
    assert e.value.status == nat.ERR_NODEVICE


@pytest.mark.parametrize("wl", ["small", "production", "sweep"])
def test_boundary_values_match_oracle(wl):
    w = {"small": workloads.small(), "production": workloads.production(nch=40),
         "sweep": workloads.sweep(20)}[wl]
    co, cop, xc1, xc2, nopen = api.boundary_values(w.lval, w.qk, w.eta, w.rmax)
    ref = orc.boundary_values(w.nch, w.lval, w.qk, w.eta, w.rmax)
    assert nopen == ref.nopen
    for m, c in enumerate(ref.npo_open):
        assert abs(co[c] - ref.co[m]) <= 1e-13 * abs(ref.co[m])
        assert abs(cop[c] - ref.cop[m]) <= 1e-13 * abs(ref.cop[m])
    for c in ref.npo_closed:
        assert abs(xc1[c] - ref.xc[c, 0]) <= 1e-13 * abs(ref.xc[c, 0])
        assert abs(xc2[c] - ref.xc[c, 1]) <= 1e-13 * abs(ref.xc[c, 1])


def test_boundary_values_ex1_jwkb_branch():
    """Ex1 at 10 MeV (l = 20, eta = 16) runs COULFG's JWKB branch; product == oracle."""
    from tests.example_inputs import ex1_setup
    mesh = orc.rmat_ini(60, 1, 14.0)
    _, kin = ex1_setup(mesh.zrma)
    for e in (10.0, 20.0, 50.0):
        lval, qk, eta = kin(e, 20)
        co, cop, _, _, _ = api.boundary_values(lval, qk, eta, 14.0)
        ref = orc.boundary_values(1, lval, qk, eta, 14.0)
        assert abs(co[0] - ref.co[0]) <= 1e-13 * abs(ref.co[0])
        assert abs(cop[0] - ref.cop[0]) <= 1e-13 * abs(ref.cop[0])


def test_boundary_rejects_bad_arguments():
    lib = nat.load()
    z = np.zeros(1)
    assert lib.hprmat_b200_boundary(0, None, None, None, 1.0, None, None, None, None, None) == nat.ERR_ARG
    lval = np.array([-1], np.int32)
    assert lib.hprmat_b200_boundary(1, lval.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1.0,
                                    None, None, None, None, None) == nat.ERR_ARG


@pytest.mark.parametrize("nr,ns,rmax", [(10, 1, 10.0), (30, 4, 16.0), (15, 3, 12.0), (40, 2, 20.0)])
def test_mesh_matches_oracle(nr, ns, rmax):
    """Per-interval kinetic/Bloch matrices and boundary values of the device assembly against
    the oracle's rmat_ini (src/rmatrix_hp.F90:61-159), odd and even nr, one to four intervals."""
    lib = nat.load()
    tc = np.zeros(ns * nr * nr)
    blo = np.zeros(ns * nr * nr)
    q2 = np.zeros(ns * nr)
    q1 = np.zeros(ns * nr)
    zr = np.zeros(ns * nr)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    nat.check(lib.hprmat_b200_dev_mesh(nr, ns, rmax, dp(tc), dp(blo), dp(q2), dp(q1), dp(zr)))
    m = orc.rmat_ini(nr, ns, rmax)
    for s in range(ns):
        t = tc[s * nr * nr:(s + 1) * nr * nr].reshape(nr, nr, order="F")
        b = blo[s * nr * nr:(s + 1) * nr * nr].reshape(nr, nr, order="F")
        np.testing.assert_allclose(t, m.tc[:, :, s], rtol=1e-13, atol=1e-13 * np.abs(m.tc[:, :, s]).max())
        # closed-channel Bloch term of interval s+1, times rmax0 (rmatrix_hp.F90:268-276)
        ref = m.blo0 if s == 0 else (m.blo2 / ((s + 1) * m.rmax0) - m.blo1 / (s * m.rmax0)) * m.rmax0
        np.testing.assert_allclose(b, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
        np.testing.assert_allclose(q2[s * nr:(s + 1) * nr], m.q2[:, s], rtol=1e-14)
        np.testing.assert_allclose(q1[s * nr:(s + 1) * nr], m.q1[:, s], rtol=1e-14, atol=0)
    np.testing.assert_allclose(zr, m.zrma, rtol=1e-15)


def test_wf_print_matches_oracle():
    """The library's host wf_print (spline inside rmax, Coulomb/Whittaker outside) against the
    oracle's restatement on Ex3's wave function (oracle cu and cf as input), every channel."""
    from tests.example_inputs import ex3_setup
    nr, ns, rmax, j = 50, 2, 14.0, 30
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin, nv = ex3_setup(mesh.zrma, j)
    lval, qk, eta = kin(34.0)
    cu, no, cf = orc.rmatrix_wf(nv, lval, qk, eta, rmax, mesh, cpot, [1])
    for iv in range(1, nv + 1):
        ref = orc.wf_print(nv, lval, qk, eta, rmax, mesh, cu, no, cf, iv, 1, 25, 0.8)
        got = api.wf_print(lval, qk, eta, rmax, nr, ns, cu, no, cf, mesh.zrma, iv, 1, 25, 0.8)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    with pytest.raises(nat.HprmatError):
        api.wf_print(lval, qk, eta, rmax, nr, ns, cu, no, cf, mesh.zrma, nv + 1, 1, 5, 1.0)


def test_wf_print_closed_channel_tail():
    """Closed channels outside rmax: the Whittaker form times the closed-channel amplitude."""
    from tests.example_inputs import ex4_setup
    nr, ns, rmax, j = 20, 4, 11.0, 3
    mesh = orc.rmat_ini(nr, ns, rmax)
    cpot, kin, nv = ex4_setup(mesh.zrma, j)
    lval, qk, eta = kin(4.0)
    assert (qk < 0).any()
    cu, no, cf = orc.rmatrix_wf(nv, lval, qk, eta, rmax, mesh, cpot, [1])
    for iv in range(1, nv + 1):
        ref = orc.wf_print(nv, lval, qk, eta, rmax, mesh, cu, no, cf, iv, 1, 16, 1.0)
        got = api.wf_print(lval, qk, eta, rmax, nr, ns, cu, no, cf, mesh.zrma, iv, 1, 16, 1.0)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14 * max(np.abs(ref).max(), 1e-300))


def test_struct_mirrors_match_the_header(tmp_path):
    """The ctypes mirrors of hprmat_b200_opts / hprmat_b200_stats / hprmat_b200_scan_block have
    the C header's size and field offsets (compiled with gcc against include/hprmat_b200.h)."""
    mirrors = {"hprmat_b200_opts": nat.Opts, "hprmat_b200_stats": nat.Stats, "hprmat_b200_scan_block": nat.ScanBlock}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "hprmat_b200.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _t in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            cname, field, val = ln.split()
            got[(cname, field)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _t in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_scan_blocks_are_checked_on_the_host():
    """Scan inputs are validated and laid out before any device call."""
    w = workloads.small()
    qk = np.tile(np.asarray(w.qk, float), (3, 1))
    eta = np.tile(np.asarray(w.eta, float), (3, 1))
    _keep, arr, out = api.Context._scan_blocks([(w.lval, w.cpot, qk, eta)])
    assert arr[0].nch == w.nch and arr[0].nenergies == 3 and arr[0].ncp1 == w.cpot.shape[0]
    assert out[0][0].shape == (3, w.nch, w.nch)
    with pytest.raises(ValueError):
        api.Context._scan_blocks([(w.lval, w.cpot, qk[:, :-1], eta)])
    with pytest.raises(ValueError):
        api.Context._scan_blocks([(w.lval[:-1], w.cpot, qk, eta)])

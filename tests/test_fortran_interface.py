"""The Fortran side of the boundary (fortran/b200_solver_interface.F90, fortran/solver_type7.patch)
checked against the C header without a Fortran compiler (none exists in this image).

* Every ``bind(C, name=...)`` interface names a function that include/hprmat_b200.h declares,
  with the same number and order of arguments; each argument's Fortran declaration passes what
  the C prototype expects (a VALUE scalar of the matching kind for int / long / double, a
  reference for pointers to numbers or structs, a VALUE ``type(c_ptr)`` for void* and the context
  handle), and functions return what C returns.
* The interoperable types mirror the C structs field by field (names, kinds, array lengths).
* The dispatch patch adds ``case (7)`` to both dispatches (src/rmatrix_hp.F90:299-322,
  src/rmat_solvers.F90:69-88), each calling the module's solve_rmatrix_b200 with the argument
  list of solve_rmatrix_dense (src/rmat_solvers.F90:98-148); where the reference sources are
  present, the patch applies to a copy of them.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "fortran", "b200_solver_interface.F90")
PATCH = os.path.join(ROOT, "fortran", "solver_type7.patch")
HEADER = os.path.join(ROOT, "include", "hprmat_b200.h")
REFERENCE = "/root/reference"


def _strip_c(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _c_prototypes():
    src = _strip_c(open(HEADER).read())
    out = {}
    for m in re.finditer(r"\b(int|void|long long|const char\*)\s+((?:hprmat_b200|gpu_b200)_\w+)\s*\(([^)]*)\)\s*;",
                         src, re.S):
        ret, name, args = m.group(1), m.group(2), " ".join(m.group(3).split())
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        out[name] = (ret, params)
    return out


def _c_param_type(p):
    """'const double* cpot' -> 'double*'; 'hprmat_b200_ctx** out' -> 'hprmat_b200_ctx**'."""
    p = p.replace("const ", "").strip()
    m = re.match(r"^(.*?)(\w+)$", p)
    assert m and m.group(1).strip(), p
    return re.sub(r"\s+", "", m.group(1))


def _strip_f(src):
    lines = []
    for ln in src.splitlines():
        ln = ln.split("!")[0].rstrip()
        lines.append(ln)
    joined = "\n".join(lines)
    return re.sub(r"&\s*\n\s*", " ", joined)  # continuation lines


def _f_interfaces():
    src = _strip_f(open(F90).read())
    body = src[src.index("interface"):src.index("end interface")]
    out = {}
    pat = re.compile(r"(?:(integer\(c_int\)|type\(c_ptr\))\s+)?(function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*"
                     r"bind\(C,\s*name=\"(\w+)\"\)(.*?)end\s+(?:function|subroutine)", re.S | re.I)
    for m in pat.finditer(body):
        rtype, kind, _fname, args, cname, decls = m.groups()
        argnames = [a.strip().lower() for a in args.split(",") if a.strip()]
        attrs = {}
        for d in decls.splitlines():
            d = d.strip()
            if "::" not in d or d.lower().startswith("import"):
                continue
            spec, names = d.split("::", 1)
            spec = spec.strip().lower()
            for nm in names.split(","):
                nm = nm.strip().lower()
                base = nm.split("(")[0].strip()
                attrs[base] = (spec, "(" in nm)
        out[cname] = (kind.lower(), rtype, argnames, attrs)
    return out


# C parameter type -> accepted Fortran declarations: (type spec prefix, by value?)
_BY_VALUE = {"int": "integer(c_int)", "long": "integer(c_long)", "double": "real(c_double)"}
_BY_REF = {"int*": ("integer(c_int)",), "double*": ("real(c_double)", "complex(c_double_complex)"),
           "hprmat_b200_opts*": ("type(b200_opts)",), "hprmat_b200_stats*": ("type(b200_stats)",),
           "hprmat_b200_scan_block*": ("type(b200_scan_block)",), "hprmat_b200_ctx**": ("type(c_ptr)",)}
_PTR_BY_VALUE = ("void*", "hprmat_b200_ctx*")


def _check_arg(cname, ctype, spec):
    by_value = "value" in spec
    base = spec.split(",")[0].strip()
    if ctype in _BY_VALUE:
        assert by_value and base == _BY_VALUE[ctype], (cname, ctype, spec)
    elif ctype in _PTR_BY_VALUE:
        assert by_value and base == "type(c_ptr)", (cname, ctype, spec)
    elif ctype in _BY_REF:
        assert not by_value and base in _BY_REF[ctype], (cname, ctype, spec)
    else:
        raise AssertionError(f"{cname}: no Fortran mapping for C type {ctype}")


def test_every_binding_matches_the_c_prototype():
    protos = _c_prototypes()
    ifaces = _f_interfaces()
    assert len(ifaces) >= 20
    for cname, (kind, rtype, argnames, attrs) in ifaces.items():
        assert cname in protos, cname
        ret, params = protos[cname]
        assert len(argnames) == len(params), (cname, argnames, params)
        if ret == "void":
            assert kind == "subroutine", cname
        elif ret == "int":
            assert kind == "function" and rtype == "integer(c_int)", cname
        elif ret == "const char*":
            assert kind == "function" and rtype == "type(c_ptr)", cname
        for a, p in zip(argnames, params):
            assert a in attrs, (cname, a)
            _check_arg(cname, _c_param_type(p), attrs[a][0])


def test_the_solver_entry_points_have_bindings():
    ifaces = _f_interfaces()
    for name in ("gpu_b200_solve_mixed_", "gpu_b200_solve_double_", "gpu_b200_finalize_", "hprmat_b200_create",
                 "hprmat_b200_destroy", "hprmat_b200_rmat_ini", "hprmat_b200_rmatrix", "hprmat_b200_rmatrix_full",
                 "hprmat_b200_solve_rmatrix", "hprmat_b200_solve_linear", "hprmat_b200_rmatrix_scan",
                 "hprmat_b200_last_error", "hprmat_b200_version"):
        assert name in ifaces, name


def _c_struct(name):
    src = _strip_c(open(HEADER).read())
    m = re.search(r"typedef struct \{([^{}]*)\}\s*" + name + r"\s*;", src)
    assert m, name
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        decl = decl.replace("const ", "")
        mt = re.match(r"(\w+)\s*(\*?)\s*(.*)$", decl)
        ctype, ptr, names = mt.group(1), mt.group(2), mt.group(3)
        for nm in names.split(","):
            nm = nm.strip()
            star = ptr or ("*" if nm.startswith("*") else "")
            nm = nm.lstrip("*")
            dim = re.search(r"\[(\d+)\]", nm)
            fields.append((nm.split("[")[0], ctype + star, int(dim.group(1)) if dim else None))
    return fields


def _f_type(name):
    src = _strip_f(open(F90).read())
    m = re.search(r"type,\s*bind\(C\)\s*::\s*" + name + r"\s*\n(.*?)end\s+type", src, re.S | re.I)
    assert m, name
    fields = []
    for d in m.group(1).splitlines():
        if "::" not in d:
            continue
        spec, names = d.split("::", 1)
        names = re.sub(r"=\s*[^,]+(?=,|$)", "", names)  # default initialisers
        for nm in re.split(r",(?![^(]*\))", names):
            nm = nm.strip()
            if not nm:
                continue
            dim = re.search(r"\((\d+)\)", nm)
            fields.append((nm.split("(")[0].strip().lower(), spec.strip().lower(), int(dim.group(1)) if dim else None))
    return fields


@pytest.mark.parametrize("cname,fname", [("hprmat_b200_opts", "b200_opts"), ("hprmat_b200_stats", "b200_stats"),
                                         ("hprmat_b200_scan_block", "b200_scan_block")])
def test_struct_mirrors_match_the_header(cname, fname):
    kinds = {"int": "integer(c_int)", "double": "real(c_double)"}
    cf = _c_struct(cname)
    ff = _f_type(fname)
    assert [n for n, _, _ in cf] == [n for n, _, _ in ff], (cname, cf, ff)
    for (n, ct, cd), (_, fs, fd) in zip(cf, ff):
        want = "type(c_ptr)" if ct.endswith("*") else kinds[ct]
        assert fs == want and cd == fd, (cname, n, ct, fs, cd, fd)


def test_abi_version_of_the_module_matches_the_header():
    m = re.search(r"#define HPRMAT_B200_ABI_VERSION (\d+)", open(HEADER).read())
    f = re.search(r"B200_ABI_VERSION\s*=\s*(\d+)", open(F90).read())
    assert m and f and m.group(1) == f.group(1)


def test_dispatch_patch_adds_case_7_to_both_dispatches():
    patch = open(PATCH).read()
    files = re.findall(r"^\+\+\+ b/(\S+)", patch, re.M)
    assert files == ["src/rmatrix_hp.F90", "src/rmat_solvers.F90", "Makefile"]
    added = [ln[1:] for ln in patch.splitlines() if ln.startswith("+") and not ln.startswith("+++")]
    calls = [ln.strip() for ln in added if "call solve_rmatrix_b200(" in ln]
    assert calls == ["call solve_rmatrix_b200(ch(:,:,is), B_vector, nch, nr, 1.0d0, Rmat_local)",
                     "call solve_rmatrix_b200(cmat, B_vector, nch, nlag, normfac, Rmat)"]
    assert sum(1 for ln in added if ln.strip() == "case (7)") == 2
    assert sum(1 for ln in added if "use b200_solver_interface, only: solve_rmatrix_b200" in ln) == 2
    src = _strip_f(open(F90).read())
    m = re.search(r"subroutine solve_rmatrix_b200\(([^)]*)\)", src)
    assert m and [a.strip() for a in m.group(1).split(",")] == ["cmat", "B_vector", "nch", "nlag", "normfac", "Rmat"]
    assert re.search(r"public ::[^\n]*\bsolve_rmatrix_b200\b", src)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "src")) or shutil.which("patch") is None,
                    reason="the reference sources (or patch) are not on this machine")
def test_dispatch_patch_applies_to_the_reference(tmp_path):
    for rel in ("src/rmatrix_hp.F90", "src/rmat_solvers.F90", "Makefile"):
        dst = tmp_path / rel
        dst.parent.mkdir(parents=True, exist_ok=True)
        shutil.copyfile(os.path.join(REFERENCE, rel), dst)
    r = subprocess.run(["patch", "-p1", "--dry-run", "-i", PATCH], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr

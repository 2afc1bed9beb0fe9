"""The C-ABI library builds for sm_100a, loads, and exports every symbol include/*.h declares.

No compute calls here (this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from cism_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(cismgpu_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_the_four_solvers():
    names = declared_symbols()
    for f in ("cismgpu_pcg_standard_3d", "cismgpu_pcg_chrongear_3d", "cismgpu_pcg_standard_2d",
              "cismgpu_pcg_chrongear_2d"):
        assert f in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string(lib):
    lib.cismgpu_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.cismgpu_version()


def test_built_for_sm100a_only():
    flags = build.flags()
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "--fmad=false" in flags


def _header_prototypes():
    text = ""
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text += re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(cismgpu_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return protos


def test_fortran_interfaces_match_the_header():
    """Every bind(C) interface of the Fortran module names a declared C function with the same
    number of arguments."""
    src = open(os.path.join(ROOT, "cism_b200", "fortran", "glissade_velo_higher_pcg_gpu.F90")).read()
    src = "\n".join(line.split("!")[0] for line in src.splitlines())  # drop comments
    src = re.sub(r"&\s*\n\s*", " ", src)                                 # join continuation lines
    protos = _header_prototypes()
    found = re.findall(r"function\s+\w+\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(cismgpu_[a-z0-9_]+)\"\)", src)
    assert len(found) >= 8
    for args, cname in found:
        n = 0 if not args.strip() else args.count(",") + 1
        assert cname in protos, cname
        assert protos[cname] == n, (cname, protos[cname], n)


def test_status_names_match_the_header():
    import cism_b200 as cg
    text = open(os.path.join(ROOT, "include", "cismgpu.h")).read()
    codes = {int(v): n for n, v in re.findall(r"#define\s+(CISMGPU_(?:OK|E[A-Z0-9_]+))\s+(\d+)", text)}
    assert codes == cg.STATUS_NAMES


def test_assembly_entry_points_validate_before_the_device(lib):
    """The assembly and boundary entry points reject bad arguments with the library's status
    (4 EINVAL) before any device call, so these run without a GPU."""
    import numpy as np
    import cism_b200 as cg
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=81)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    u = np.zeros((ny - 1, nx - 1, nz))
    ff = np.ones((ny, nx, nz - 1))
    act = g["ac"].astype(np.int32)
    base = [nx, ny, nz, 2, g["sigma"], act, g["xVertex"], g["yVertex"], u, u, g["stagusrf"], g["stagthck"], ff]
    cases = [(3, 1, {}), (None, None, {"whichefvs": 3}), (None, None, {"n_glen": 0.0})]
    for idx, val, kw in cases:
        args = list(base)
        if idx is not None:
            args[idx] = val  # nhalo = 1
        with pytest.raises(cg.CismGpuError) as e:
            cg.assemble_stiffness_matrix_3d(*args, **kw)
        assert e.value.status == 4
    u2 = np.zeros((ny - 1, nx - 1))
    with pytest.raises(cg.CismGpuError) as e:
        cg.assemble_stiffness_matrix_2d(nx, ny, nz, 1, g["sigma"], act, g["xVertex"], g["yVertex"], u2, u2,
                                        g["stagthck"], ff)
    assert e.value.status == 4
    A = [np.zeros((ny - 1, nx - 1, nz, 27)) for _ in range(2)]
    with pytest.raises(cg.CismGpuError) as e:  # whichassemble_beta is 0 (standard) or 1 (local)
        cg.basal_sliding_bc_3d(nx, ny, nz, 2, 1.0, 1.0, act, g["av"], np.zeros((ny - 1, nx - 1)), np.zeros((ny, nx)),
                               g["xVertex"], g["yVertex"], *A, whichassemble_beta=2)
    assert e.value.status == 4
    with pytest.raises(cg.CismGpuError) as e:  # the standard form reads cell vertices: nhalo >= 2
        cg.basal_sliding_bc_3d(nx, ny, nz, 1, 1.0, 1.0, act, g["av"], np.zeros((ny - 1, nx - 1)), np.zeros((ny, nx)),
                               g["xVertex"], g["yVertex"], *A, whichassemble_beta=0)
    assert e.value.status == 4
    A2 = [np.zeros((9, ny - 1, nx - 1)) for _ in range(2)]
    with pytest.raises(cg.CismGpuError) as e:
        cg.basal_sliding_bc_2d(nx, ny, 2, 1.0, 1.0, act, g["av"], np.zeros((ny - 1, nx - 1)), g["xVertex"],
                               g["yVertex"], *A2, whichassemble_beta=2)
    assert e.value.status == 4
    with pytest.raises(cg.CismGpuError) as e:
        cg.basal_sliding_bc_2d(nx, ny, 1, 1.0, 1.0, act, g["av"], np.zeros((ny - 1, nx - 1)), g["xVertex"],
                               g["yVertex"], *A2, whichassemble_beta=0)
    assert e.value.status == 4
    bad = np.arange(1, 28, dtype=np.int32)
    bad[5] = 99
    with pytest.raises(cg.CismGpuError) as e:  # indxA entry outside 1..27
        cg.assemble_stiffness_matrix_3d(*base, indxA_3d=bad)
    assert e.value.status == 4


def test_newer_assembly_entry_points_validate_before_the_device(lib):
    """DIVA, L1L2 and the load vector reject bad arguments (EINVAL) before any device call."""
    import numpy as np
    import cism_b200 as cg
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=82)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    act = g["ac"].astype(np.int32)
    z2 = np.zeros((ny - 1, nx - 1))
    zc = np.zeros((ny, nx))
    ff = np.ones((ny, nx, nz - 1))
    with pytest.raises(cg.CismGpuError) as e:  # n_glen must be 1 or 3 for the L1L2 viscosity
        cg.assemble_stiffness_matrix_2d_l1l2(nx, ny, nz, 2, g["sigma"], act, g["xVertex"], g["yVertex"], z2, z2,
                                             g["stagthck"], z2, z2, ff, ff, n_glen=2.0)
    assert e.value.status == 4
    eq = np.zeros((ny, nx, 4, nz - 1))
    with pytest.raises(cg.CismGpuError) as e:  # nhalo = 1
        cg.assemble_stiffness_matrix_2d_diva(nx, ny, nz, 1, g["sigma"], g["sigma"][:-1], act, g["xVertex"],
                                             g["yVertex"], z2, z2, g["stagthck"], zc, z2, z2, zc, zc, ff, eq)
    assert e.value.status == 4
    with pytest.raises(cg.CismGpuError) as e:  # whichassemble_taud is 0 or 1
        cg.load_vector_gravity(nx, ny, nz, 2, g["sigma"], np.linspace(0, 1, nz + 1), 1.0, 1.0, act, g["av"],
                               g["xVertex"], g["yVertex"], g["stagusrf"], g["stagthck"], z2, z2, whichassemble_taud=3)
    assert e.value.status == 4
    with pytest.raises(cg.CismGpuError) as e:
        cg.basal_sliding_bc_2d_diva(nx, ny, 2, 1.0, 1.0, act, g["av"], z2, z2, zc, g["xVertex"], g["yVertex"],
                                    np.zeros((9, ny - 1, nx - 1)), np.zeros((9, ny - 1, nx - 1)), whichassemble_beta=7)
    assert e.value.status == 4


def test_handle_method_bindings_reach_the_library(lib):
    """The DeviceSolver assembly methods pass their arguments through ctypes with the C
    signatures: on a NULL handle the library answers EINVAL (no device call), where a binding
    mismatch would raise a ctypes or Python error first."""
    import numpy as np
    import cism_b200 as cg
    from cism_b200 import assembly as asm
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=83, nz=5)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    act = g["ac"].astype(np.int32)
    av = g["av"].astype(np.int32)
    z2, zc = np.zeros((ny - 1, nx - 1)), np.zeros((ny, nx))
    ff = np.ones((ny, nx, nz - 1))
    for kind in ("3d", "2d"):
        s = cg.DeviceSolver.__new__(cg.DeviceSolver)
        s._lib = cg.load_library()
        s.handle = None
        P = asm.Problem(kind, nx, ny, nz if kind == "3d" else 1, None, None, None, None, None, None, av, {})
        s.problem = P
        u = np.zeros((ny - 1, nx - 1, nz)) if kind == "3d" else z2
        load = (u, u)
        calls = [lambda: s.assemble_stiffness(2, g["sigma"], act, g["xVertex"], g["yVertex"], g["stagusrf"],
                                              g["stagthck"], ff),
                 lambda: s.assemble_system(2, 1.0, 1.0, g["sigma"], act, av, g["xVertex"], g["yVertex"],
                                           g["stagusrf"], g["stagthck"], ff, *load, beta=z2, lsrf=zc,
                                           umask=np.zeros(u.shape, np.int32), vmask=np.zeros(u.shape, np.int32),
                                           whichassemble_beta=0)]
        if kind == "2d":
            sig = g["sigma"]
            calls += [lambda: s.assemble_stiffness_diva(nz, 2, sig, sig[:-1], act, g["xVertex"], g["yVertex"],
                                                        g["stagthck"], zc, z2, z2, zc, zc, ff, uvel=z2, vvel=z2,
                                                        efvs_qp_3d=np.zeros((ny, nx, 4, nz - 1))),
                      lambda: s.assemble_system_diva(nz, 2, 1.0, 1.0, sig, sig[:-1], act, av, g["xVertex"],
                                                     g["yVertex"], g["stagthck"], zc, z2, z2, zc, zc, ff, z2, z2,
                                                     beta_eff_x=z2, beta_eff_y=z2, lsrf=zc,
                                                     umask=np.zeros(z2.shape, np.int32),
                                                     vmask=np.zeros(z2.shape, np.int32))]
        for call in calls:
            with pytest.raises(cg.CismGpuError) as e:
                call()
            assert e.value.status == 4
        s.handle = None  # nothing to destroy


# ---------------------------------------------------------------------------------------------
# The Fortran module's bind(C) interfaces against the header's prototypes, parameter by parameter.
# No Fortran compiler is available, so the interfaces are read as text, each dummy argument's C
# type is derived from its ISO_C_BINDING kind and attributes (value: by value; otherwise a pointer
# to the kind, as Fortran passes by reference), and g++ checks them against the header's function
# types with static_asserts.  Integer kinds compare by size and signedness (the ABI), floating
# kinds and structs exactly, pointees without their const.
# ---------------------------------------------------------------------------------------------
_KINDS = {"c_int": ("int", 4), "c_int32_t": ("int", 4), "c_long_long": ("int", 8), "c_int64_t": ("int", 8),
          "c_size_t": ("uint", 8), "c_double": ("double", 8), "c_float": ("float", 4), "c_char": ("char", 1),
          "c_ptr": ("ptr", 8), "cismgpu_par_t": ("par", 0)}


def _fortran_interfaces():
    src = open(os.path.join(ROOT, "cism_b200", "fortran", "glissade_velo_higher_pcg_gpu.F90")).read()
    src = "\n".join(line.split("!")[0] for line in src.splitlines())
    src = re.sub(r"&\s*\n\s*", " ", src)
    block = src[src.index("\n    interface"):src.index("end interface")]
    out = []
    for m in re.finditer(r"(integer|type|real)\((\w+)\)\s+function\s+\w+\s*\(([^)]*)\)\s*"
                         r"bind\(C,\s*name=\"(cismgpu_[a-z0-9_]+)\"\)(.*?)end function", block, flags=re.S):
        _, rkind, args, cname, body = m.groups()
        names = [a.strip() for a in args.split(",") if a.strip()]
        decl = {}
        for line in body.splitlines():
            d = re.match(r"\s*(integer|real|type|character)\((?:kind=)?(\w+)\)\s*(,[^:]*)?::(.*)", line)
            if not d:
                continue
            attrs = d.group(3) or ""
            for ent in re.findall(r"(\w+)\s*(\([^)]*\))?", d.group(4)):
                decl[ent[0].lower()] = (d.group(2), "value" in attrs)
        out.append((cname, rkind, [(n, *decl[n.lower()]) for n in names]))
    return out


def _cxx_check(kind, value, t):
    base, size = _KINDS[kind]
    if kind == "c_ptr":
        return f"std::is_pointer<{t}>::value" if value else f"std::is_pointer<pointee<{t}>>::value"
    inner = t if value else f"pointee<{t}>"
    ptr = "true" if value else f"std::is_pointer<{t}>::value"
    if base in ("int", "uint"):
        sign = "true" if base == "int" else "false"
        return (f"{ptr} && std::is_integral<{inner}>::value && sizeof({inner}) == {size} && "
                f"std::is_signed<{inner}>::value == {sign}")
    ctype = {"double": "double", "float": "float", "char": "char", "par": "cismgpu_par_t"}[base]
    return f"{ptr} && std::is_same<{inner}, {ctype}>::value"


def test_fortran_interfaces_match_the_header_types(tmp_path):
    """Every parameter and result of every bind(C) interface of the Fortran module has the C type
    of the header's prototype (g++ static_asserts), and the module's bind(C) cismgpu_par_t has the
    header struct's members, types and offsets."""
    import shutil
    import subprocess
    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    ifaces = _fortran_interfaces()
    assert len(ifaces) >= 20
    lines = ["#include <cstddef>", "#include <cstdint>", "#include <tuple>", "#include <type_traits>",
             '#include "cismgpu.h"',
             "template <class P> using pointee = std::remove_cv_t<std::remove_pointer_t<P>>;",
             "template <class F> struct sig;",
             "template <class R, class... A> struct sig<R (*)(A...)> {",
             "  using ret = R; static constexpr int n = sizeof...(A);",
             "  template <int i> using arg = std::tuple_element_t<i, std::tuple<A...>>; };"]
    for cname, rkind, args in ifaces:
        s = f"sig<decltype(&{cname})>"
        lines.append(f'static_assert({s}::n == {len(args)}, "{cname}: argument count");')
        lines.append(f'static_assert({_cxx_check(rkind, True, f"{s}::ret")}, "{cname}: result type");')
        for i, (name, kind, value) in enumerate(args):
            t = f"{s}::arg<{i}>"
            lines.append(f'static_assert({_cxx_check(kind, value, t)}, "{cname}: argument {i + 1} ({name})");')
    src = open(os.path.join(ROOT, "cism_b200", "fortran", "glissade_velo_higher_pcg_gpu.F90")).read()
    body = re.search(r"type, bind\(C\) :: cismgpu_par_t(.*?)end type", src, flags=re.S).group(1)
    fields = []
    for kind, names in re.findall(r"integer\((\w+)\)\s*::\s*([^\n!]*)", body):
        assert kind == "c_int32_t"
        fields += [n.strip() for n in names.split(",") if n.strip()]
    assert len(fields) == 10
    for k, f in enumerate(fields):
        lines.append(f'static_assert(offsetof(cismgpu_par_t, {f}) == {4 * k}, "par member {f}");')
        lines.append(f'static_assert(std::is_same<decltype(cismgpu_par_t::{f}), int32_t>::value, "par {f}");')
    lines.append(f'static_assert(sizeof(cismgpu_par_t) == {4 * len(fields)}, "par size");')
    cpp = tmp_path / "fortran_abi_check.cpp"
    cpp.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(cpp)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


# ---------------------------------------------------------------------------------------------
# The Python package's ctypes signatures against the header's prototypes.
# ---------------------------------------------------------------------------------------------
def _header_signatures():
    """{name: (return type, [parameter types])} from include/*.h, names and array brackets
    dropped, whitespace normalised."""
    text = ""
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text += re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
    text = "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))
    text = text.replace('extern "C" {', ";")
    out = {}
    for m in re.finditer(r"([^;{}]*?)\b(cismgpu_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        ret = " ".join(m.group(1).split()).replace("typedef", "").strip()
        args = m.group(3).strip()
        params = []
        if args not in ("", "void"):
            for a in args.split(","):
                a = " ".join(a.split())
                a = re.sub(r"\b\w+(\[\w*\])?$", lambda mm: "*" if mm.group(1) else "", a).strip()
                params.append(re.sub(r"\s*\*", " *", a).replace("  ", " ").strip())
        out[m.group(2)] = (ret, params)
    return out


def _ctype_matches(ctype_text, ct):
    """Whether ctypes type ct passes the C type ctype_text the same way."""
    t = ctype_text.replace("const ", "").strip()
    if t.endswith("*"):
        if ct is ctypes.c_void_p or (t == "char *" and ct is ctypes.c_char_p):
            return True
        if not (isinstance(ct, type) and issubclass(ct, ctypes._Pointer)):
            return False
        pointee = t[:-1].strip()
        if pointee.endswith("*"):  # a handle's address: T **
            return ct._type_ is ctypes.c_void_p or issubclass(ct._type_, ctypes._Pointer)
        if pointee in ("cismgpu_par_t", "cismgpu_request_t"):
            return issubclass(ct._type_, ctypes.Structure)
        return _ctype_matches(pointee, ct._type_)
    scalars = {"int": ("i", 4, True), "int32_t": ("i", 4, True), "unsigned int": ("i", 4, False),
               "long long": ("i", 8, True), "int64_t": ("i", 8, True), "size_t": ("i", 8, False),
               "double": ("d", 8, True), "float": ("f", 4, True)}
    if t not in scalars or ct is None or not isinstance(ct, type) or not issubclass(ct, ctypes._SimpleCData):
        return False
    kind, size, signed = scalars[t]
    if ctypes.sizeof(ct) != size:
        return False
    if kind != "i":
        return ct._type_ == kind
    return ct._type_ in "bhilqBHILQ" and (ct._type_.islower() == signed)


def test_python_bindings_match_the_header():
    """Every function the package binds has the header's parameter count and, parameter by
    parameter, a ctypes type that passes the C type the same way (pointers as c_void_p or a
    POINTER of the same pointee, integers by size and signedness); functions returning a pointer
    or a non-int value declare a restype that carries it."""
    import cism_b200 as cg
    lib = cg.load_library()
    sigs = _header_signatures()
    checked = 0
    for name, (ret, params) in sorted(sigs.items()):
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        if fn.argtypes is not None:
            assert len(fn.argtypes) == len(params), (name, len(fn.argtypes), len(params))
            for i, (p, ct) in enumerate(zip(params, fn.argtypes)):
                assert _ctype_matches(p, ct), (name, i + 1, p, ct)
            checked += 1
        r = ret.replace("const ", "").strip()
        if r.endswith("*"):
            assert fn.restype in (ctypes.c_char_p, ctypes.c_void_p) or (
                isinstance(fn.restype, type) and issubclass(fn.restype, ctypes._Pointer)), (name, ret, fn.restype)
        elif r not in ("int", "void") and fn.argtypes is not None:
            assert _ctype_matches(r, fn.restype), (name, ret, fn.restype)
    assert checked >= 40, checked


_C_CALLER = r"""
#include <stdio.h>
#include <string.h>
#include "cismgpu.h"
int main(void) {
    const char *v = cismgpu_version();
    if (!v || !strstr(v, "sm_100a")) return 2;
    int prev = cismgpu_set_sum_order(CISMGPU_SUM_SEQUENTIAL);
    if (cismgpu_set_sum_order(prev) != CISMGPU_SUM_SEQUENTIAL) return 3;
    if (cismgpu_solver_mixed_layout(NULL, NULL) != CISMGPU_EINVAL) return 4;
    if (strlen(cismgpu_last_error()) == 0) return 5;
    printf("%s\n", v);
    return 0;
}
"""


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c", "c11"), ("c++", "c++11"), ("c++", "c++17")])
def test_header_compiles_strictly(tmp_path, lang, std):
    """include/cismgpu.h is plain C for C callers and C++ callers: no warning under -pedantic."""
    import shutil
    import subprocess
    cc = "gcc" if lang == "c" else "g++"
    if not shutil.which(cc):
        pytest.skip(f"no {cc}")
    src = tmp_path / ("hdr.c" if lang == "c" else "hdr.cpp")
    src.write_text('#include "cismgpu.h"\nint main(void) { return 0; }\n')
    r = subprocess.run([cc, f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_caller_links_and_calls(tmp_path, lib):
    """A C99 program built against the header links libcismgpu.so and calls its host-side entry
    points (version, sum order, an argument check and its message) without a GPU."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("no gcc")
    libdir = os.path.dirname(build.build())
    src = tmp_path / "caller.c"
    src.write_text(_C_CALLER)
    exe = tmp_path / "caller"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                        os.path.join(ROOT, "include"), str(src), "-L", libdir, "-lcismgpu",
                        f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and "sm_100a" in run.stdout, (run.returncode, run.stdout, run.stderr)

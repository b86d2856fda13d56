"""The C-ABI library loads and exports every entry point include/p2cuda.h
declares; without a GPU, p2_create fails cleanly (CPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "p2cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(p2_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for f in ("p2_stokes_solve", "p2_ronurecalc", "p2_set_grid", "p2_set_bc", "p2_set_nodes", "p2_create"):
        assert f in names


def test_library_exports_every_declared_symbol():
    from pardiso2_b200 import capi
    lib = capi.load()
    for f in declared_functions():
        assert hasattr(lib, f), f
    assert set(capi.EXPORTED) == set(declared_functions())


def test_library_is_sm100a_and_self_contained():
    from pardiso2_b200 import capi
    out = os.popen("ldd %s" % capi.LIB_PATH).read()
    assert "libcudart" not in out  # cudart linked statically: the .so travels alone


def test_create_without_gpu_reports_cuda_error(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    from pardiso2_b200 import capi
    lib = capi.load()
    h = ctypes.c_void_p()
    assert lib.p2_create(ctypes.byref(h), 0) == 2  # P2_ERR_CUDA
    assert not h.value


def test_default_params_are_the_reference_defaults():
    from pardiso2_b200 import capi
    p = capi.default_params()
    # pardiso/mode.t3c:89-93
    assert (p.p0koef, p.p1koef, p.p2koef, p.v0koef, p.v1koef) == (0.3, 1.0, 0.0, 1.0, 1.0)
    assert (p.nubeg, p.nuend, p.viscmod) == (1.0, 1e4, 0)
    assert p.tol == 1e-8 and p.precision == 0


def test_reference_shim_compiles_in_the_unity_build():
    """pardiso2_b200/csrc/move3mg_cuda.c replaces vpiterate()/ronurecalc()
    inside the reference's own unity build (needs the reference sources)."""
    import subprocess
    obj = os.path.join(ROOT, "oracle", "_ref", "shim_check.o")
    ref = os.environ.get("P2_REFERENCE_DIR")
    if ref and os.path.isdir(ref):
        r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "shimcheck", "REF=" + ref],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
    if not os.path.exists(obj):
        pytest.skip("shim check object not built (build() with the reference sources, or P2_REFERENCE_DIR)")
    syms = subprocess.run(["nm", obj], capture_output=True, text=True).stdout
    for name, kind in (("vpiterate", "T"), ("ronurecalc", "T"), ("vpiterate_cpu", "T"), ("ronurecalc_cpu", "T"),
                       ("p2_stokes_solve", "U"), ("p2_ronurecalc", "U"), ("p2_set_grid", "U")):
        assert any(ln.split()[-2:] == [kind, name] for ln in syms.splitlines()), (name, kind)


def test_ctypes_structs_match_the_header(tmp_path):
    """The ctypes mirrors of the parameter / result structs have the C
    layout (size and every field offset), checked against gcc on the header."""
    import shutil
    import subprocess

    from pardiso2_b200 import capi
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    structs = {"p2_params": capi.Params, "p2_solve_info": capi.SolveInfo, "p2_tune_info": capi.TuneInfo,
               "p2_effbulk": capi.EffBulk, "p2_heat_params": capi.HeatParams, "p2_heat_info": capi.HeatInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "p2cuda.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                           text=True).stdout.split("\n") if l)
    for cname, cls in structs.items():
        assert int(out["%s size" % cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(out["%s.%s" % (cname, f)]) == getattr(cls, f).offset, (cname, f)

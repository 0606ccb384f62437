"""The C-ABI library loads, exports every declared entry point, and its host-only
functions behave.  No compute call is made (no GPU here)."""
import ctypes as C
import os
import re

import numpy as np

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mgsb_[a-z0-9_]+)\s*\(", text)))


def test_all_declared_symbols_exported(lib):
    names = [n for n in _declared("mgsb.h")]
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header(lib):
    declared = set(_declared("mgsb.h"))
    bound = {n for n, _, _ in L.SIGNATURES}
    assert declared == bound, (declared - bound, bound - declared)


def test_default_params_are_reference_constants(lib):
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)
    # PDSolver::Init, PDSolver.cpp:166-176
    assert p.iterations == 20
    assert abs(p.dt - 1 / 60) < 1e-9
    assert abs(p.damping - 0.95) < 1e-7
    assert p.volume_stiffness == 8000.0 and p.collision_stiffness == 1000.0
    assert abs(p.cheb_rho - 0.9992) < 1e-7
    assert list(p.gravity) == [0.0, np.float32(-9.8), 0.0]
    assert abs(p.relaxation - 0.6) < 1e-7
    q = mg.default_params(mg.SOLVER_MULTIGRID)
    assert q.iterations == 10 and q.levels >= 2 and q.pre_sweeps == 2 and q.post_sweeps == 2


def test_bad_arguments_rejected(lib):
    p = mg.default_params()
    assert lib.mgsb_default_params(7, C.byref(p)) == 1
    out = C.POINTER(L.MeshData)()
    lo = np.zeros(3, np.float32)
    assert lib.mgsb_mesh_box(0, 1, 1, lo.ctypes.data_as(C.POINTER(C.c_float)),
                             lo.ctypes.data_as(C.POINTER(C.c_float)), C.byref(out)) == 1
    h = C.c_void_p()
    assert lib.mgsb_create(None, C.byref(p), C.byref(h)) == 1
    assert lib.mgsb_status_string(4) == b"diverged"


def _c_offsets(struct, fields):
    """Compile a tiny C program against include/mgsb.h printing offsetof/sizeof."""
    import shutil
    import subprocess
    import tempfile
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    body = "".join(f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields)
    src = (f'#include <stdio.h>\n#include <stddef.h>\n#include "mgsb.h"\n'
           f'int main(void){{{body} printf("%zu\\n", sizeof({struct})); return 0;}}\n')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run([cc, "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    return [int(v) for v in out]


def test_struct_layouts_match_c(lib):
    for cls, name in [(L.Params, "mgsb_params"), (L.Mesh, "mgsb_mesh"), (L.MeshData, "mgsb_mesh_data")]:
        fields = [f for f, _ in cls._fields_]
        got = _c_offsets(name, fields)
        assert got[:-1] == [getattr(cls, f).offset for f in fields], name
        assert got[-1] == C.sizeof(cls), name

"""CPU-only checks of the C ABI boundary: the library loads without a GPU, exports every
symbol include/ariel.h declares, and refuses to compute without an sm_100 device."""
import ctypes as C
import os
import re

import pytest

from ariel_b200 import _abi as A
from ariel_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "ariel.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ariel_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_defaults_match_reference_constants():
    L = _lib.lib()
    p = A.AsimParams()
    L.ariel_params_default(C.byref(p))
    assert abs(p.picflip - 0.95) < 1e-7 and p.subcell == 1 and p.resample_every == 1
    assert p.precond == A.PRECOND_REF and p.stop_rule == A.STOP_REF_ABS
    d = A.AsimSceneDesc()
    L.ariel_scene_dambreak(C.byref(d), 64)
    assert d.dim == 64 and d.density == 0.5 and abs(d.stepsize - 1 / 240) < 1e-9
    assert d.n_forces == 1 and abs(d.forces[0][1] + 9.8) < 1e-6
    assert L.ariel_abi_version() == 2


def test_status_strings():
    L = _lib.lib()
    for code in range(10):
        assert L.ariel_status_string(code)


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU behaviour")
def test_no_device_is_reported_not_faked():
    L = _lib.lib()
    d = A.scene_dambreak(16)
    p = A.params_default()
    h = C.c_void_p()
    assert L.ariel_create(C.byref(d), C.byref(p), C.byref(h)) == A.ARIEL_ERR_NO_DEVICE
    assert L.ariel_selftest_barrier_timeout(1.0) == A.ARIEL_ERR_NO_DEVICE


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirror (ariel_b200/_abi.py) against the C compiler's view of include/ariel.h:
    size of every struct and offset of a few late fields."""
    import shutil
    import subprocess
    structs = ["AsimBox", "AsimSphere", "AsimSceneDesc", "AsimParams", "AsimStats", "AsimSolverTotals",
               "AsimServerConfig", "AsimRequestInfo", "AsimServerStats", "AsimSceneInfo"]
    fields = [("AsimSceneDesc", "seed"), ("AsimSceneDesc", "n_mesh"), ("AsimSceneDesc", "mesh"),
              ("AsimParams", "sweep_brick"), ("AsimParams", "reseed_max"), ("AsimStats", "stage_ms"),
              ("AsimSceneInfo", "mesh_output")]
    src = tmp_path / "sizes.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ariel.h"', "int main(void) {"]
    lines += ['printf("%s %%zu\\n", sizeof(%s));' % (s, s) for s in structs]
    lines += ['printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (s, f, s, f) for s, f in fields]
    lines += ["return 0; }"]
    src.write_text("\n".join(lines))
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for s in structs:
        assert int(out[s]) == C.sizeof(getattr(A, s)), s
    for s, f in fields:
        assert int(out["%s.%s" % (s, f)]) == getattr(getattr(A, s), f).offset, (s, f)

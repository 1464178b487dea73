"""The C ABI library loads, exports every symbol include/csg.h declares, its
ctypes mirror matches the C struct layouts, and argument checks fail cleanly
(no GPU needed: validation happens before any CUDA call)."""
import ctypes as C
import pathlib
import re
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "csg.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(csg_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(csg):
    names = declared_functions()
    assert len(names) >= 16
    lib = C.CDLL(str(csg.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(csg.LIB_PATH)], check=True,
                         capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (csg_\w+)", out))
    assert set(names) <= exported


def test_struct_layouts_match_header(tmp_path, csg):
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "csg.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu\\n\","
        "sizeof(csg_config), offsetof(csg_config, H), offsetof(csg_config, betas),"
        "offsetof(csg_config, swap_log_rounds), sizeof(csg_observables),"
        "offsetof(csg_observables, boundary), sizeof(csg_device_obs), sizeof(csg_plan));"
        "return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [C.sizeof(csg.Config), csg.Config.H.offset, csg.Config.betas.offset,
            csg.Config.swap_log_rounds.offset, C.sizeof(csg.ObservablesC),
            csg.ObservablesC.boundary.offset, C.sizeof(csg.DeviceObs), C.sizeof(csg.Plan)]
    assert got == want


@pytest.mark.parametrize("kw,msg", [
    (dict(L=7), "even"),
    (dict(L=130), "outside"),
    (dict(n_words=0), "n_words"),
    (dict(n_copies=3), "n_copies"),
    (dict(T=6), "multiple of 4"),
    (dict(H=4.5), "H out of range"),
])
def test_invalid_configurations_are_rejected(csg, kw, msg):
    L = kw.get("L", 8)
    T = kw.get("T", 8)
    betas = np.linspace(2.0, 0.5, T)
    with pytest.raises(csg.CsgError, match=msg):
        csg.Engine(L, kw.get("n_words", 1), kw.get("n_copies", 2), betas, H=kw.get("H", 0.0))


def test_negative_beta_rejected(csg):
    with pytest.raises(csg.CsgError, match="betas"):
        csg.Engine(8, 1, 2, np.array([2.0, 1.0, -1.0, 0.5]))


def test_missing_library_fails_loudly(csg, monkeypatch, tmp_path):
    monkeypatch.setattr(csg, "_lib", None)
    monkeypatch.setattr(csg, "LIB_PATH", tmp_path / "nope.so")
    with pytest.raises(RuntimeError, match="missing"):
        csg.lib()


def test_flag_constants_match_header(tmp_path, csg):
    src = tmp_path / "fl.c"
    src.write_text(
        '#include <stdio.h>\n#include "csg.h"\n'
        'int main(void){printf("%d %d %d\\n", CSG_MEASURE_M, CSG_ENGINE_STREAM, '
        'CSG_STREAM_FUSED); return 0;}\n')
    exe = tmp_path / "fl"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert got == [csg.CSG_MEASURE_M, csg.CSG_ENGINE_STREAM, csg.CSG_STREAM_FUSED]

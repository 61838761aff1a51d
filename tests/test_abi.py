"""The C ABI library: loads, exports every declared symbol, and its struct
layouts agree with include/pgerosion.h (no GPU calls)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from pgerosion import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "pgerosion.h"


def declared():
    return re.findall(r"PGE_API\s+\w+\s+(pge_\w+)\(", HEADER.read_text())


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = declared()
    assert set(names) == set(_lib.EXPORTS)
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "pgerosion.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n",'
                   "sizeof(PgeGrid),sizeof(PgeState),sizeof(PgeSpawns),sizeof(PgeParams),sizeof(PgeStats),sizeof(PgeHalo),"
                   "offsetof(PgeGrid,max_droplets));return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.PgeGrid), ctypes.sizeof(_lib.PgeState), ctypes.sizeof(_lib.PgeSpawns), ctypes.sizeof(_lib.PgeParams),
            ctypes.sizeof(_lib.PgeStats), ctypes.sizeof(_lib.PgeHalo), _lib.PgeGrid.max_droplets.offset]
    assert got == want


def test_version_and_argument_errors_without_gpu():
    L = _lib.load()
    assert L.pge_version() == 1
    g = _lib.PgeGrid(F=6, N=16, H=2, spherical=1, deposit_on_exit=0, metric_shared=1, max_steps=64, max_droplets=1000, max_wave=256)
    assert L.pge_workspace_bytes(ctypes.byref(g)) > 0
    bad = _lib.PgeGrid(F=5, N=16, H=2, spherical=1, max_steps=64, max_droplets=10, max_wave=10)
    assert L.pge_workspace_bytes(ctypes.byref(bad)) == 0
    assert "6 faces" in _lib.last_error()
    rc = L.pge_trace_apply(ctypes.byref(g), None, None, None, None, None, None, 0, None)
    assert rc == _lib.PGE_E_ARG


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(_lib.PgeError):
        _lib.load(tmp_path / "libpgerosion.so")

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
    src.write_text('#include "pgerosion.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                   "sizeof(PgeGrid),sizeof(PgeState),sizeof(PgeSpawns),sizeof(PgeParams),sizeof(PgeStats),sizeof(PgeHalo),"
                   "offsetof(PgeGrid,max_droplets),offsetof(PgeState,lake_flag),offsetof(PgeState,roots),"
                   "offsetof(PgeParams,lateral_rate),offsetof(PgeParams,max_steps),sizeof(PgeLakeInfo));return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.PgeGrid), ctypes.sizeof(_lib.PgeState), ctypes.sizeof(_lib.PgeSpawns), ctypes.sizeof(_lib.PgeParams),
            ctypes.sizeof(_lib.PgeStats), ctypes.sizeof(_lib.PgeHalo), _lib.PgeGrid.max_droplets.offset,
            _lib.PgeState.lake_flag.offset, _lib.PgeState.roots.offset, _lib.PgeParams.lateral_rate.offset,
            _lib.PgeParams.max_steps.offset, ctypes.sizeof(_lib.PgeLakeInfo)]
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


def test_refresh_entries_reject_bad_arguments_without_gpu():
    """The lake, basin and window entries refuse what they cannot run before
    any device call: NULL inputs, the wrong kind of grid, bad rates."""
    import numpy as np

    L = _lib.load()
    sphere = _lib.PgeGrid(F=6, N=8, H=2, spherical=1, metric_shared=1, max_steps=8, max_droplets=16, max_wave=16)
    window = _lib.PgeGrid(F=1, N=8, H=2, spherical=0, metric_shared=1, max_steps=8, max_droplets=16, max_wave=16)
    a = np.zeros(6 * 12 * 12 * 3, np.float64)
    ptr = a.ctypes.data
    st = _lib.PgeState(height=ptr, sediment=ptr)  # no route
    assert L.pge_window_lakes(ctypes.byref(window), ctypes.byref(st), 0.1, ptr, None, None) == _lib.PGE_E_ARG
    assert "NULL" in _lib.last_error()
    st.route = ptr
    assert L.pge_window_lakes(ctypes.byref(window), ctypes.byref(st), -1.0, ptr, None, None) == _lib.PGE_E_ARG
    assert L.pge_basin_fill(ctypes.byref(window), ptr, ptr, ptr, 0.1, 0.0, ptr, None, None) == _lib.PGE_E_UNSUPPORTED
    assert L.pge_basin_fill(ctypes.byref(sphere), ptr, None, ptr, 0.1, 0.0, ptr, None, None) == _lib.PGE_E_ARG
    assert L.pge_basin_fill(ctypes.byref(sphere), ptr, ptr, ptr, -0.1, 0.0, ptr, None, None) == _lib.PGE_E_ARG
    assert L.pge_window_lake_balance(ctypes.byref(sphere), ptr, ptr, ptr, ptr, 1.0, 0.0, ptr, ptr, None) == _lib.PGE_E_UNSUPPORTED
    assert L.pge_window_lake_balance(ctypes.byref(window), ptr, ptr, ptr, ptr, 0.0, 0.0, ptr, ptr, None) == _lib.PGE_E_ARG
    info = _lib.PgeLakeInfo()
    assert L.pge_lake_balance(ctypes.byref(sphere), ptr, ptr, ptr, 1000.0, ptr, ptr, ptr, None, 6.0, 3.0, 0.1, ptr, None, None,
                              ctypes.byref(info)) == _lib.PGE_E_ARG
    assert L.pge_lake_balance(ctypes.byref(sphere), ptr, ptr, ptr, 0.0, ptr, ptr, ptr, ptr, 6.0, 3.0, 0.1, ptr, None, None,
                              ctypes.byref(info)) == _lib.PGE_E_ARG


def test_bank_cut_needs_room_for_two_entries_a_step_without_gpu():
    """erosion.lateral_rate > 0 writes two change-list entries a step: a
    workspace built for max_steps alone is refused before any device call."""
    import numpy as np

    L = _lib.load()
    g = _lib.PgeGrid(F=6, N=8, H=2, spherical=1, metric_shared=1, max_steps=32, max_droplets=16, max_wave=16, wave_tables=1)
    nbytes = int(L.pge_workspace_bytes(ctypes.byref(g)))
    raw = np.zeros(nbytes + 512, np.uint8)
    ws = (raw.ctypes.data + 255) & ~255
    a = np.zeros(64, np.float64)
    ptr = a.ctypes.data
    st = _lib.PgeState(**{n: ptr for n, _ in _lib.PgeState._fields_
                          if n not in ("mask", "erodibility", "route", "lake_flag", "roots", "lake_load", "lake_id", "lake_room",
                                       "lakes")})
    prm = _lib.PgeParams(max_steps=32, wave=16, precision=_lib.PREC_F64, apply=_lib.APPLY_WAVE, lateral_rate=0.5)
    stats = np.zeros(_lib.STATS_WORDS, np.int64)
    sp = _lib.PgeSpawns(count=0, volume0=1.0)
    rc = L.pge_trace_apply(ctypes.byref(g), ctypes.byref(st), ctypes.byref(sp), ctypes.byref(prm), None, stats.ctypes.data, ws,
                           nbytes, None)
    assert rc == _lib.PGE_E_ARG and "2 x max_steps" in _lib.last_error()
    prm.lateral_rate = -1.0
    rc = L.pge_trace_apply(ctypes.byref(g), ctypes.byref(st), ctypes.byref(sp), ctypes.byref(prm), None, stats.ctypes.data, ws,
                           nbytes, None)
    assert rc == _lib.PGE_E_ARG and "lateral_rate" in _lib.last_error()


def test_wave_tables_follow_max_threads_without_gpu():
    """PgeGrid.max_threads bounds the wave apply's per-thread own-change
    tables: a grid for 4096 resident droplet threads needs a smaller
    workspace than one for the whole GPU, and the ordered apply's workspace
    (no tables) does not depend on it."""
    L = _lib.load()
    kw = dict(F=6, N=64, H=2, spherical=1, metric_shared=1, max_steps=128, max_droplets=4096, max_wave=2048)
    full = int(L.pge_workspace_bytes(ctypes.byref(_lib.PgeGrid(**kw, wave_tables=1))))
    small = int(L.pge_workspace_bytes(ctypes.byref(_lib.PgeGrid(**kw, wave_tables=1, max_threads=4096))))
    assert 0 < small < full
    # 16 bytes a table slot (key and own change) a thread less
    slots = 16
    while slots < 2 * (128 + 8 + 2):
        slots <<= 1
    assert full - small >= 16 * slots * (148 * 1024 - 4096) - 4096
    a = int(L.pge_workspace_bytes(ctypes.byref(_lib.PgeGrid(**kw))))
    b = int(L.pge_workspace_bytes(ctypes.byref(_lib.PgeGrid(**kw, max_threads=4096))))
    assert a == b

"""The workspace-free thermal entry point (pge_thermal_noalloc).

Some callers cannot allocate device memory -- a host that owns the device
heap through its own pool, or a loop that must not pay cudaMalloc's latency
and synchronisation -- so the library offers one variant of the thermal pass
whose scratch is a static device array instead of a caller workspace.  This
file checks it against the workspace entry point (pge_thermal) through the C
ABI on two calls in a row, and that a grid larger than the static scratch is
refused.  It is collected last, and builds all of its own state, so it runs
the same alone in a fresh process or after every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from pgerosion import _lib
from pgerosion import maps as gm
from pgerosion import synth

pytestmark = pytest.mark.gpu


def _state(world, seed):
    st = gm.ErosionState.from_world(world)
    rng = np.random.default_rng(seed)
    # some loose sediment on the relief, so both the talus and the creep pass move material
    st.sediment.copy_(torch.as_tensor(rng.random(tuple(st.sediment.shape)) * 0.5))
    return st


def _thermal_args(ep, unit):
    return (float(ep.thermal_rate), float(ep.creep_rate), float(ep.thermal_max) / unit, float(ep.talus_slope_soft),
            float(ep.talus_slope_hard), float(ep.dep_floor_m) / unit)


def test_thermal_noalloc_matches_workspace_entry_point(cuda):
    L = _lib.load()
    world = synth.earth_world(seed=11, N=64, H=2, cell_size_m=50.0, land_fraction=0.3)
    params, _ = synth.config_params("small")
    a = _state(world, 1)
    b = _state(world, 1)
    a.reserve(1, 64, 1)
    targs = _thermal_args(params.erosion, a.height_unit_m)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h0 = a.height.clone()
    for call in range(2):
        rc = L.pge_thermal(ctypes.byref(a.pge_grid()), ctypes.byref(a.pge_state()), *targs, ctypes.c_void_p(a.workspace.data_ptr()),
                           a.workspace.numel(), stream)
        assert rc == _lib.PGE_OK, _lib.last_error()
        rc = L.pge_thermal_noalloc(ctypes.byref(b.pge_grid()), ctypes.byref(b.pge_state()), *targs, stream)
        assert rc == _lib.PGE_OK, _lib.last_error()
        torch.cuda.synchronize()
        for k in ("height", "sediment"):
            np.testing.assert_allclose(getattr(b, k).cpu().numpy(), getattr(a, k).cpu().numpy(), rtol=1e-12, atol=1e-12,
                                       err_msg=f"call {call}: {k}")
    assert not torch.equal(a.height, h0), "the pass moved no material: the comparison proves nothing"


def test_thermal_noalloc_refuses_grids_beyond_its_scratch(cuda):
    L = _lib.load()
    world = synth.earth_world(seed=11, N=64, H=2, cell_size_m=50.0, land_fraction=0.3)
    st = _state(world, 2)
    big = _lib.PgeGrid(F=6, N=256, H=2, spherical=1, deposit_on_exit=0, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    assert 6 * 260 * 260 > _lib.NOALLOC_MAX_CELLS
    rc = L.pge_thermal_noalloc(ctypes.byref(big), ctypes.byref(st.pge_state()), 0.5, 0.02, 1.0, 0.6, 1.2, 0.02,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.PGE_E_ARG
    assert "exceed the static scratch" in _lib.last_error()
    # the same grid rules as pge_thermal: a sphere has six faces, the halo fits the face
    for bad in (_lib.PgeGrid(F=1, N=64, H=2, spherical=1, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1),
                _lib.PgeGrid(F=6, N=4, H=3, spherical=1, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)):
        rc = L.pge_thermal_noalloc(ctypes.byref(bad), ctypes.byref(st.pge_state()), 0.5, 0.02, 1.0, 0.6, 1.2, 0.02,
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == _lib.PGE_E_ARG, "a grid pge_thermal refuses must be refused here too"

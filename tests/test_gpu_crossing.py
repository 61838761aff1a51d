"""The float64 trace's face crossing on the device, against the reference.

* The kernel's tan / atan / sin / cos (pge_crmath, the code the float64
  droplet kernel calls) equal the host build of the same code bit for bit on
  10^7 inputs of the crossing's ranges, which tests/test_crmath.py checks
  against the C library (the reference's functions) and against exact values.
  CUDA's own functions are measured beside them, for the record.
* The device to_sphere / from_sphere (pge_cubesphere_map) against the bake's
  own vector file (tests/data/cubesphere_vectors.bin, which the reference's
  scalar functions reproduce bit for bit: bake/tests/test_cubesphere.py:
  379-402; the reference's bar for its vectorised path is 2 ulp), and
  transfer_velocity against records the reference computed
  (tests/golden/cubesphere_vectors.npz).
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from pgerosion import _lib

from .test_crmath import OPS, host, inputs

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).parent / "golden"


def _dev(op, x):
    xd = torch.as_tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    rc = _lib.load().pge_crmath(op, xd.numel(), ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.PGE_OK, _lib.last_error()
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("op", sorted(OPS))
def test_device_trig_equals_host_build_and_tracks_the_c_library(cuda, op):
    n = 10_000_000 if op < 2 else 2_000_000  # tan and atan are the crossing's; sin / cos seed loaded droplets
    x = inputs(op, n, seed=100)
    dev = _dev(op, x)
    hst = host(op, x)
    assert np.array_equal(dev.view(np.int64), hst.view(np.int64)), f"{OPS[op]}: device and host builds differ"
    libm = orc.libm(op, x)
    ours = np.count_nonzero(dev != libm) / n
    cuda_own = _dev(op + 4, x)
    theirs = np.count_nonzero(cuda_own != libm) / n
    ulp_cuda = np.abs(cuda_own.view(np.int64) - libm.view(np.int64)).max()
    print(f"{OPS[op]} on {n} inputs: library vs C library {ours:.4%} differ (1 ulp, the C library's misroundings); "
          f"CUDA's {OPS[op]} vs C library {theirs:.4%} differ (max {ulp_cuda} ulp)")
    assert ours < 0.005


def _map(op, face, uv, ab, xyz):
    face = torch.as_tensor(np.ascontiguousarray(face, np.int32), device="cuda")
    uv = torch.as_tensor(np.ascontiguousarray(uv, np.float64), device="cuda")
    ab = torch.as_tensor(np.ascontiguousarray(ab, np.float64), device="cuda")
    xyz = torch.as_tensor(np.ascontiguousarray(xyz, np.float64), device="cuda")
    rc = _lib.load().pge_cubesphere_map(op, face.numel(), *(ctypes.c_void_p(t.data_ptr()) for t in (face, uv, ab, xyz)),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.PGE_OK, _lib.last_error()
    torch.cuda.synchronize()
    return face.cpu().numpy(), uv.cpu().numpy(), ab.cpu().numpy(), xyz.cpu().numpy()


def _ulp(a, b):
    return np.abs(np.asarray(a, np.float64).view(np.int64) - np.asarray(b, np.float64).view(np.int64))


def test_device_mapping_against_the_reference_vector_file(cuda):
    g = np.load(GOLD / "cubesphere_ref_vectors.npz")
    n = g["face"].size
    _, _, _, xyz = _map(0, g["face"], np.stack([g["u"], g["v"]], 1), np.zeros((n, 2)), np.zeros((n, 3)))
    u_xyz = _ulp(xyz, g["xyz"])
    f2, uv2, _, _ = _map(1, np.zeros(n, np.int32), np.zeros((n, 2)), np.zeros((n, 2)), g["xyz"])
    u_uv = _ulp(uv2, np.stack([g["u2"], g["v2"]], 1))
    print(f"reference vector file, {n} records: to_sphere bit-exact in {np.mean(u_xyz.max(1) == 0):.2%} (max {u_xyz.max()} ulp), "
          f"from_sphere bit-exact in {np.mean(u_uv.max(1) == 0):.2%} (max {u_uv.max()} ulp)")
    assert np.array_equal(f2, g["face2"])
    # the reference's bar for code other than its scalar functions: within 2 eps absolute
    # (bake/tests/test_cubesphere.py:396-402); a last-bit difference of u near 0 is many ulps of u
    eps = np.finfo(np.float64).eps
    assert np.abs(xyz - g["xyz"]).max() <= 2 * eps
    assert np.abs(uv2 - np.stack([g["u2"], g["v2"]], 1)).max() <= 2 * eps
    assert np.mean(u_xyz.max(1) == 0) > 0.99 and np.mean(u_uv.max(1) == 0) > 0.99


def test_device_transfer_velocity_against_reference_records(cuda):
    g = np.load(GOLD / "cubesphere_vectors.npz")
    n = g["t_face"].size
    f, uv, ab, _ = _map(2, g["t_face"], np.stack([g["t_u"], g["t_v"]], 1), np.stack([g["t_a"], g["t_b"]], 1), np.zeros((n, 3)))
    out = np.concatenate([uv, ab], 1)
    assert np.array_equal(f, g["t_face2"])
    exact = np.all(out == g["t_out"], 1)
    rel = np.abs(out - g["t_out"]).max() / np.abs(g["t_out"]).max()
    print(f"transfer_velocity, {n} crossings: bit-exact {exact.mean():.2%}, largest difference {rel:.2e} of the largest value")
    assert exact.mean() > 0.98
    assert rel < 1e-13

"""The float64 trace's own tan / atan / sin / cos (pge_crmath.cuh), on the host.

The reference's face crossing (bake/globe/cubesphere.py:70-220) and a
re-injected droplet's direction (bake/globe/erosion/particle.py:400-401) call
the C library's functions.  The library evaluates them in double-double and
rounds once.  These tests, with no GPU: (1) on the inputs the crossing and
the spawn see, the host build agrees with the C library except in a small
share of inputs, by one ulp at most; (2) wherever they disagree (and on
random agreeing inputs) the library's value is the correctly rounded one,
checked against 60-digit decimal arithmetic -- so the disagreements are the C
library's own last-bit errors; (3) signed zeros and edge inputs agree.
The device build is checked against this host build bit for bit in
tests/test_gpu_crossing.py.
"""
import ctypes
import math
from decimal import Decimal as D, getcontext

import numpy as np
import pytest

from oracle import oracle as orc
from pgerosion import _lib

OPS = {0: "tan", 1: "atan", 2: "sin", 3: "cos"}


def host(op, x):
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(x)
    rc = _lib.load().pge_crmath_host(op, x.size, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(y.ctypes.data))
    assert rc == _lib.PGE_OK, _lib.last_error()
    return y


def inputs(op, n, seed=0):
    """What the trace feeds each function: (u - 1/2) pi/2 for u a face coordinate up to a
    little past the edge (to_sphere, jacobian), s in [-1, 1] (from_sphere), a direction
    in [0, 2 pi) (the spawn of a loaded droplet)."""
    rng = np.random.default_rng(seed + op)
    if op == 0:
        return (rng.uniform(-0.02, 1.02, n) - 0.5) * (np.pi / 2)
    if op == 1:
        return rng.uniform(-1.0, 1.0, n)
    return rng.uniform(0.0, 2.0 * np.pi, n)


def exact(op, x: float) -> D:
    """The function's value to ~55 digits: Taylor series in decimal arithmetic."""
    getcontext().prec = 70
    xd = D(x)
    if op == 1:
        h = 0  # atan by argument halving, then its series
        while abs(xd) > D("0.02"):
            xd = xd / (1 + (1 + xd * xd).sqrt())
            h += 1
        s, t, n = D(0), xd, 0
        while abs(t) > D(10) ** -66:
            s += t / (2 * n + 1) if n % 2 == 0 else -t / (2 * n + 1)
            t *= xd * xd
            n += 1
        return s * (2 ** h)
    s, c, t, n = D(0), D(0), D(1), 0
    while abs(t) > D(10) ** -66 or n < 4:
        sign = 1 if (n // 2) % 2 == 0 else -1
        if n % 2 == 0:
            c += sign * t
        else:
            s += sign * t
        n += 1
        t = t * xd / n
    return s / c if op == 0 else s if op == 2 else c


def correctly_rounded(v: D) -> float:
    f = float(v)
    return min((math.nextafter(f, -math.inf), f, math.nextafter(f, math.inf)), key=lambda c: abs(D(c) - v))


@pytest.mark.parametrize("op", sorted(OPS))
def test_host_functions_against_the_c_library_and_exact_values(op):
    n = 400_000
    x = inputs(op, n)
    ours = host(op, x)
    libm = orc.libm(op, x)
    ulp = np.abs(ours.view(np.int64) - libm.view(np.int64))
    bad = np.flatnonzero(ulp)
    share = bad.size / n
    print(f"{OPS[op]}: {bad.size} of {n} inputs differ from the C library ({share:.4%}), max {ulp.max()} ulp")
    assert ulp.max() <= 1
    assert share < 0.005
    rng = np.random.default_rng(7)
    check = list(rng.choice(bad, min(60, bad.size), replace=False)) + list(rng.choice(n, 40, replace=False))
    for i in check:
        want = correctly_rounded(exact(op, float(x[i])))
        assert ours[i] == want, f"{OPS[op]}({x[i]!r}): ours {ours[i]!r}, correctly rounded {want!r}, C library {libm[i]!r}"


def test_edge_inputs_agree_with_the_c_library():
    x = np.array([0.0, -0.0, 5e-324, -1e-300, 1e-8, -3e-9, 1.0, -1.0, 0.999999999, 2.0, -7.5, 1e6, -1e10, np.pi / 4,
                  -np.pi / 4, np.pi / 2, 3 * np.pi / 2, 2 * np.pi])
    for op in OPS:
        ours = host(op, x)
        libm = orc.libm(op, x)
        assert np.array_equal(ours.view(np.int64), libm.view(np.int64)), (OPS[op], x[ours != libm], ours[ours != libm])

"""The deterministic transcendental functions (cindergs_b200/csrc/detmath.h)
used by Stages 1-3 on both host and device: within 3 ulp of the correctly
rounded value over the ranges the pipeline uses."""
import math

import numpy as np
import pytest

import oracle


def ulps(a: np.float32, b: np.float32) -> int:
    ia = int(np.float32(a).view(np.int32))
    ib = int(np.float32(b).view(np.int32))
    return abs(ia - ib)


@pytest.mark.parametrize("fn,ref,xs", [
    ("log", math.log, np.geomspace(1e-30, 1e30, 4001)),
    ("log", math.log, np.linspace(1.0, 255.0, 4001)),           # ln(255 alpha)
    ("exp", math.exp, np.linspace(-87.0, 88.0, 4001)),
    ("exp", math.exp, np.linspace(-4.0, 0.0, 4001)),            # compositor e^q
    ("acos", math.acos, np.linspace(-1.0, 1.0, 4001)),
    ("cos", math.cos, np.linspace(0.0, math.pi / 3, 4001)),     # Cardano phi
])
def test_within_3_ulp(fn, ref, xs):
    worst = 0
    for x in xs.astype(np.float32):
        got = np.float32(oracle.detmath(fn, float(x)))
        want = np.float32(ref(float(x)))
        worst = max(worst, ulps(got, want))
    assert worst <= 3, worst


def test_pow_relative_error():
    rng = np.random.default_rng(0)
    b = rng.uniform(1e-4, 0.999, 2000).astype(np.float32)
    e = rng.uniform(0.55, 1.7, 2000).astype(np.float32)
    for bi, ei in zip(b, e):
        got = oracle.detmath("pow", float(bi), float(ei))
        want = float(bi) ** float(ei)
        assert abs(got - want) <= 2e-6 * want


def test_special_values():
    assert oracle.detmath("log", 0.0) == -math.inf
    assert math.isnan(oracle.detmath("log", -1.0))
    assert oracle.detmath("exp", 100.0) == math.inf
    assert oracle.detmath("exp", -200.0) == 0.0
    assert oracle.detmath("log", 1.0) == 0.0
    assert oracle.detmath("exp", 0.0) == 1.0

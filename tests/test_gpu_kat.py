"""The library's device reconstruction functions against the reference's
reconstruction unit tests (GPU).

src/physics/hydro/tests/test_reconstruction.cpp:13-194 checks Reconstruct on
a cubic polynomial (exact to 5e-6 relative for every method and limiter) and
mirror symmetry on a steep tanh profile (the minus value of the reversed
stencil equals the plus value within 4 ulps).  The fixtures in
tests/golden/reconstruction_kat.json restate those inputs; here they run
through every device form the stage kernels use (kmy_reconstruct_stencils):
the FP64 per-task, brick and z-streamed forms, and the FP32 per-lane, brick
(packed) and z-streamed (packed) forms.  FP32 forms are held to the same exactness bound
(their rounding is far below 5e-6 on these values) and to 4 float ulps of
symmetry; the packed forms' two lanes must agree bit for bit.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import kamayan_b200 as K

pytestmark = pytest.mark.gpu

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "reconstruction_kat.json").read_text())
IMPLS = ["fp64_tasks", "fp64_brick", "fp32_lane", "fp32_brick", "fp32_slab", "fp64_slab"]


def ulps(a, b, f32):
    if f32:
        ia, ib = np.array([a], np.float32).view(np.int32)[0], np.array([b], np.float32).view(np.int32)[0]
    else:
        ia, ib = np.array([a]).view(np.int64)[0], np.array([b]).view(np.int64)[0]
    return abs(int(ia) - int(ib))


@pytest.mark.parametrize("impl", IMPLS)
def test_device_reconstruction_polynomial_exactness(kmy_lib, impl):
    for case in CASES:
        out = K.reconstruct_stencils(case["reconstruction"], case["slope_limiter"], impl, [case["stencil"]])
        vm, vp, lanes = out[0]
        assert lanes == 0.0, (impl, case["reconstruction"])
        assert abs((vm - case["exact_minus"]) / case["exact_minus"]) < case["rel_tol"], (impl, case)
        assert abs((vp - case["exact_plus"]) / case["exact_plus"]) < case["rel_tol"], (impl, case)


@pytest.mark.parametrize("impl", IMPLS)
def test_device_reconstruction_mirror_symmetry(kmy_lib, impl):
    f32 = impl.startswith("fp32")
    for case in CASES:
        fwd = case["tanh_stencil"]
        out = K.reconstruct_stencils(case["reconstruction"], case["slope_limiter"], impl, [fwd, fwd[::-1]])
        (vm1, vp1, l1), (vm2, vp2, l2) = out
        assert l1 == l2 == 0.0
        assert ulps(vm1, vp2, f32) <= case["symmetry_ulps"], (impl, case["reconstruction"], vm1, vp2)
        assert ulps(vp1, vm2, f32) <= case["symmetry_ulps"], (impl, case["reconstruction"], vp1, vm2)


@pytest.mark.parametrize("impl", IMPLS)
def test_device_reconstruction_matches_oracle(kmy_lib, oracle_mod, impl):
    """Random stencils (smooth, steep and flat): every device form against the
    CPU restatement, FP64 forms to 1e-13 and FP32 forms to 2e-6 of the
    stencil's scale."""
    rng = np.random.default_rng(5)
    st = np.concatenate([rng.normal(size=(200, 5)),
                         1.0 + 1e-3 * np.sin(np.arange(5)[None, :] * 0.3 + rng.uniform(size=(200, 1))),
                         np.where(np.arange(5)[None, :] < rng.integers(0, 6, size=(200, 1)), 1.0, 0.125)])
    tol = 2e-6 if impl.startswith("fp32") else 1e-13
    for recon, lim in [("fog", "minmod"), ("plm", "minmod"), ("plm", "mc"), ("plm", "van_leer"),
                       ("ppm", "minmod"), ("ppm", "mc"), ("wenoz", "mc")]:
        out = K.reconstruct_stencils(recon, lim, impl, st)
        for i in range(st.shape[0]):
            vm, vp = oracle_mod.reconstruct(recon, lim, list(st[i]))
            scale = max(np.abs(st[i]).max(), 1e-30)
            assert abs(out[i, 0] - vm) <= tol * scale and abs(out[i, 1] - vp) <= tol * scale, \
                (impl, recon, lim, st[i], out[i], (vm, vp))


def test_fp64_newton_raphson_math_vs_ieee(kmy_lib):
    """The z-streamed FP64 stage's reciprocal and square root (hardware
    approximation + two Newton-Raphson steps) against IEEE 1/x and sqrt(x):
    within 2 and 3 ulps over the magnitudes a hydro state takes (1e-300 .. 1e300),
    sqrt(0) = 0."""
    rng = np.random.default_rng(7)
    x = 10.0 ** rng.uniform(-300, 300, 20000)
    x[:4] = [1.0, 2.0, 3.0, 0.7]
    sgn = np.where(rng.random(x.size) < 0.5, -1.0, 1.0)
    st = np.zeros((x.size, 5))
    st[:, 0] = sgn * x
    st[:, 1] = x
    st[0, 1] = 0.0
    out = K.reconstruct_stencils("wenoz", "mc", "fp64_nr_math", st)
    want_r = 1.0 / st[:, 0]
    want_s = np.sqrt(st[:, 1])
    ur = np.abs(out[:, 0].view(np.int64) - want_r.view(np.int64))
    us = np.abs(out[:, 1].view(np.int64) - want_s.view(np.int64))
    assert ur.max() <= 2, (ur.max(), st[ur.argmax(), 0])
    assert us.max() <= 3, (us.max(), st[us.argmax(), 1])
    assert out[0, 1] == 0.0

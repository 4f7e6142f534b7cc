"""The compensated 16-bit scheme, emulated on the CPU oracle (no GPU): the state stored as a
16-bit number and an FP16 rounding residual, the stencil reading the compensated state
(tests/helpers.py compensated_stencil), against the same layer in FP64.  With FP64
arithmetic, what is left is the storage's error; it must stay below the FP32 path's own error
for FP16 numbers (the GPU kernel, which adds FP32 arithmetic, is held to 2x in
tests/test_gpu_compensated.py), and within a few times it for BF16 numbers, while any stencil
that reads the 16-bit numbers themselves sits two orders of magnitude above (the floor,
tests/helpers.py stencil_on_codes).  Kelvin-Helmholtz layer, 256^2, 100 steps at 0.9 of the
CFL step."""
import numpy as np
import pytest

import fg2_b200
from helpers import compensated_stencil, stencil_on_codes
from oracle.oracle import Oracle, reference_delta

N, STEPS = 256, 100


@pytest.fixture(scope="module")
def layer():
    x0 = fg2_b200.setup_evaluate("kh", N, N, seed=2)[0]
    d1, d2 = reference_delta(N, N, 1.0, 1.0)
    gam = 5.0 / 3.0
    cs = np.sqrt(gam * (gam - 1.0) * np.exp(x0[..., 3]))
    dt = 0.9 * 0.5 / ((np.abs(x0[..., 1]) + cs) / d1 + (np.abs(x0[..., 2]) + cs) / d2).max()

    def run(prec):
        o = Oracle("hydro", prec, "port")
        o.set_delta(d1, d2)
        u = o.padded(x0.astype(np.float64 if prec == "f64" else np.float32))
        v = o.empty(N, N)
        assert o.run(u, v, 0.0, dt, STEPS) == 0
        return o.interior(u).astype(np.float64)

    o64 = Oracle("hydro", "f64", "port")
    o64.set_delta(d1, d2)
    ref = run("f64")
    return x0, dt, o64, ref, rho_rel_l2(run("f32"), ref)


def rho_rel_l2(x, ref):
    a, b = np.exp(x[..., 0]), np.exp(ref[..., 0])
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("storage,bound", [("f16", 1.0), ("bf16", 4.0)])
def test_compensated_stencil_error_against_the_fp32_path(layer, storage, bound):
    x0, dt, o64, ref, e32 = layer
    e = rho_rel_l2(compensated_stencil(o64, x0, STEPS, dt, storage), ref)
    assert e <= bound * e32, (e, e32)


def test_a_stencil_on_the_16bit_numbers_sits_far_above(layer):
    x0, dt, o64, ref, e32 = layer
    floor = rho_rel_l2(stencil_on_codes(o64, x0, STEPS, dt, "f16"), ref)
    assert floor > 100.0 * e32, (floor, e32)

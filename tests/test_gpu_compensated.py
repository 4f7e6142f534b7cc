"""Compensated 16-bit deviation storage (storage f16 / bf16).

The state is held as the 16-bit number S (value bg + s h) less its rounding residual e,
which the library keeps beside it in a second 16-bit array (one per ping-pong parity of the
state, written by every stage that writes the state), so every rounding of the state is
compensated (two-sum) and the state itself is tracked to about 2^-23 (FP16) or 2^-20 (BF16)
of its tile scale (the residual is an FP16 number for both).  The stencil reads that compensated state, T = S - e, decoded from both
arrays, not the 16-bit numbers.

* Upload/download: the state comes back to within the residual's own rounding.
* Small increments: with a step that changes the state by less than half a 16-bit unit, the
  compensated state moves with the FP32 one (an uncompensated store would not move at all),
  to a small fraction of a unit after 20 steps.
* Accuracy against FP64 (Kelvin-Helmholtz layer, 256^2, 100 steps): FP16 storage keeps the
  density error within 2x of the FP32 path's; BF16 (8 + 8 significant bits) well below the
  floor of any scheme whose stencil reads the 16-bit numbers (an FP64 CPU run that keeps the
  state exact and evaluates the right-hand side on the coded state, tests/helpers.py
  stencil_on_codes on the oracle port)."""
import numpy as np
import pytest

import fg2_b200
from helpers import deviation_codes, stencil_on_codes
from oracle.oracle import Oracle, reference_delta

pytestmark = pytest.mark.gpu

UNIT = {"f16": 2.0 ** -11, "bf16": 2.0 ** -8}
# the residual is itself an FP16 number (11 significant bits) of e / s * 4096, |e| <= s unit / 2
RESID = {"f16": 2.0 ** -22, "bf16": 2.0 ** -19}


def run(storage, x0, steps, dt, n1, n2):
    with fg2_b200.Sim(n1, n2, storage=storage) as s:
        s.config()
        s.upload(x0.astype(np.float64 if storage == "f64" else np.float32))
        t = 0.0
        for _ in range(steps):
            assert s.step(t, dt) == 0
            t += dt
        return s.download().astype(np.float64)


def rho_rel_l2(x, ref):
    a, b = np.exp(x[..., 0]), np.exp(ref[..., 0])
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_upload_keeps_the_residual(storage, cuda):
    n1, n2 = 96, 130
    x = fg2_b200.setup_evaluate("kh", n1, n2, seed=4)[0].astype(np.float32)
    with fg2_b200.Sim(n1, n2, storage=storage) as s:
        s.config()
        s.upload(x)
        y = s.download().astype(np.float64)
    _, scale = deviation_codes(x.astype(np.float64))
    err = np.abs(y - x)
    # the residual's rounding plus the FP32 arithmetic of the encode (a few ulp of x)
    assert np.all(err <= RESID[storage] * scale + 4 * np.spacing(np.abs(x).astype(np.float32))), err.max()


@pytest.mark.parametrize("storage,dt", [("f16", 4e-6), ("bf16", 3.2e-5)])
def test_increments_below_half_a_unit_accumulate(storage, dt, cuda):
    """Grid-scale velocity noise (sigma 0.01) decays by viscosity at about a fifth of a 16-bit
    unit (of the tile scale) per step at this dt; over 20 steps the FP32 state moves by
    several units and the compensated 16-bit state follows it to a few percent of that."""
    n1, n2, steps = 128, 160, 20
    x0 = fg2_b200.setup_evaluate("noise", n1, n2, seed=5)[0]
    ref = run("f32", x0, steps, dt, n1, n2)
    out = run(storage, x0, steps, dt, n1, n2)
    _, scale = deviation_codes(x0)
    unit = UNIT[storage] * scale
    step = np.abs(run("f32", x0, 1, dt, n1, n2) - x0.astype(np.float32)) / unit
    moved = np.abs(ref - x0.astype(np.float32)) / unit
    assert step.max() < 0.5 and moved.max() > 2.0, (step.max(), moved.max())
    err = np.abs(out - ref) / unit
    assert err.max() <= 0.05 * moved.max(), (err.max(), moved.max())


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_density_error_against_fp64(storage, cuda):
    n, steps = 256, 100
    x0 = fg2_b200.setup_evaluate("kh", n, n, seed=2)[0]
    d1, d2 = reference_delta(n, n, 1.0, 1.0)
    gam = 5.0 / 3.0
    cs = np.sqrt(gam * (gam - 1.0) * np.exp(x0[..., 3]))
    dt = 0.9 * 0.5 / ((np.abs(x0[..., 1]) + cs) / d1 + (np.abs(x0[..., 2]) + cs) / d2).max()
    ref = run("f64", x0, steps, dt, n, n)
    e32 = rho_rel_l2(run("f32", x0, steps, dt, n, n), ref)
    e16 = rho_rel_l2(run(storage, x0, steps, dt, n, n), ref)
    o = Oracle("hydro", "f64", "port")
    o.set_delta(d1, d2)
    floor = rho_rel_l2(stencil_on_codes(o, x0, steps, dt, storage), ref)
    print(f"{storage}: density rel L2 vs FP64 {e16:.3e} = {e16 / e32:.2f}x FP32 ({e32:.3e}); "
          f"stencil-on-codes floor {floor:.3e}")
    assert e32 < floor
    if storage == "f16":
        assert e16 <= 2.0 * e32, (e16, e32)  # the mixed-precision accuracy bar
    else:
        assert e16 <= 0.25 * floor, (e16, floor)

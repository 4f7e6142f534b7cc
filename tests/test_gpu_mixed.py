"""The 16-bit deviation-storage path (storage f16 / bf16): the state is stored as FP16 or
BF16 numbers h with value bg + s h (per-field background, per-64x64-tile scale s), the
stencil runs in FP32.  Checks: the host codes round-trip within half a 16-bit unit; over ten
steps the state stays within the rounding budget around the FP32 path: each of the 30
substages rounds every value once, to at most half a unit (2^-11 for FP16, 2^-8 for BF16) of
its tile scale, and the stencil, which couples the fields, carries each rounding forward
within the CFL factor, so the budget is 30 units of the largest field scale (a decoding,
ghost or compensation fault shows errors orders of magnitude above it); walls, the device
CFL step, the FP64 sums and batches of 16-bit members work as on the FP32 path."""
import numpy as np
import pytest

import fg2_b200

pytestmark = pytest.mark.gpu

UNIT = {"f16": 2.0 ** -11, "bf16": 2.0 ** -8}


def scale_of(x):
    """Per-field largest deviation from the background (the field mean, 0 for u2, which a
    reflecting wall negates): the largest tile scale."""
    x = x.reshape(-1, x.shape[-1]).astype(np.float64)
    bg = x.mean(0)
    bg[2] = 0.0
    return np.abs(x - bg).max(0)


def run(storage, n1, n2, setup, steps, dt, scheme="hydro", box=(1.0, 1.0), bcond=(1, 1), seed=3):
    with fg2_b200.Sim(n1, n2, scheme=scheme, storage=storage) as s:
        s.set_box(*box)
        s.set_bcond(*bcond)
        s.config()
        s.init(setup, seed=seed)
        x0 = s.download()
        t = 0.0
        for _ in range(steps):
            assert s.step(t, dt) == 0
            t += dt
        return x0, s.download()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_codes_round_trip(storage, cuda):
    with fg2_b200.Sim(96, 130, storage=storage) as s:
        s.config()
        x = fg2_b200.setup_evaluate("kh", 96, 130, seed=4)[0].astype(np.float32)
        s.upload(x)
        y = s.download()
    # each value within half a unit of the largest deviation of the field
    err = np.abs(y.astype(np.float64) - x).reshape(-1, 4).max(0)
    assert np.all(err <= 0.5 * UNIT[storage] * scale_of(x) * 1.0001 + 1e-30), err


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("scheme,setup,box,bcond", [
    ("hydro", "kh", (1.0, 1.0), (1, 1)),
    ("hydro", "noise", (1.0, 1.0), (0, 0)),
    ("hydro-isot", "turb", (2 * np.pi, 2 * np.pi), (1, 1)),
])
def test_steps_stay_within_the_rounding_budget(storage, scheme, setup, box, bcond, cuda):
    n1, n2, steps = 128, 160, 10
    dt = 5e-4 if scheme == "hydro" else 4e-3
    if setup == "kh":
        dt = 2e-4
    _, ref = run("f32", n1, n2, setup, steps, dt, scheme, box, bcond)
    x0, out = run(storage, n1, n2, setup, steps, dt, scheme, box, bcond)
    assert np.all(np.isfinite(out))
    err = np.abs(out.astype(np.float64) - ref).reshape(-1, out.shape[-1]).max(0)
    budget = 2.0 * 3 * steps * 0.5 * UNIT[storage] * max(scale_of(x0).max(), scale_of(ref).max())
    assert np.all(err <= budget), (err, budget)
    if storage == "f16":  # the state moves like the FP32 one (no stagnation at the first rounding)
        moved = np.abs(ref.astype(np.float64) - x0).reshape(-1, out.shape[-1]).max(0)
        assert np.all(np.abs(out.astype(np.float64) - x0).reshape(-1, out.shape[-1]).max(0) > 0.5 * moved)


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_sums_decode_the_state(storage, cuda):
    with fg2_b200.Sim(70, 90, storage=storage) as s:
        s.config()
        s.init("kh", seed=2)
        assert s.step(0.0, 1e-4) == 0
        q = s.download().astype(np.float64)
        sums = s.sums()
    rho = np.exp(q[..., 0])
    terms = [rho, rho * q[..., 1], rho * q[..., 2], rho * (np.exp(q[..., 3]) + 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2))]
    # the sums decode the compensated state in FP64; the download rounds it to FP32
    for k in range(4):
        assert abs(sums[k] - terms[k].sum()) <= 2.0 ** -22 * np.abs(terms[k]).sum(), (k, sums[k], terms[k].sum())


def test_device_cfl_steps(cuda):
    with fg2_b200.Sim(128, 128, storage="f16") as a, fg2_b200.Sim(128, 128, storage="f32") as b:
        for s in (a, b):
            s.config()
            s.init("kh", seed=6)
            s.set_time(0.0)
            s.advance(8, 0.0, graph=True)
            assert s.sync() == 0
        # the CFL steps follow the (slightly different) states closely
        assert a.time() == pytest.approx(b.time(), rel=1e-3)


def test_batch_of_16_bit_members_matches_single_grids(cuda):
    sizes = [(96, 96), (64, 160), (130, 70)]
    with fg2_b200.Batch(sizes, scheme="hydro", storage="f16") as b:
        b.config()
        alone = []
        for k, (n1, n2) in enumerate(sizes):
            b.members[k].init("noise", seed=k)
            s = fg2_b200.Sim(n1, n2, scheme="hydro", storage="f16")
            s.config()
            s.init("noise", seed=k)
            alone.append(s)
        x0 = [m.download() for m in b.members]
        assert b.advance(6, 3e-4, graph=True) == 0 and b.sync() == 0
        for k, s in enumerate(alone):
            t = 0.0
            for _ in range(6):
                assert s.step(t, 3e-4) == 0
                t += 3e-4
            out = s.download()
            err = np.abs(b.members[k].download().astype(np.float64) - out).reshape(-1, 4).max(0)
            # the batch scales derivatives after the sum: results differ by rounding flips
            budget = 2 * 18 * 0.5 * UNIT["f16"] * max(scale_of(x0[k]).max(), scale_of(out).max())
            assert np.all(err <= budget), (k, err, budget)
            s.close()


def test_16_bit_drift_is_refused(cuda):
    with fg2_b200.Sim(32, 32, storage="f16") as s:
        s.config()
        s.init("noise")
        with pytest.raises(fg2_b200.FG2Error):
            s.drift(1e-4)

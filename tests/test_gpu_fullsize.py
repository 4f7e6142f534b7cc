"""Size-independent properties at the benchmark configurations' full sizes, where the CPU
oracle would take too long: the 4096^2 plain-FP32 grid, the 8192^2 precision grid, and the
512-member batch.

* Translation equivariance: on a periodic grid the hydro step does not depend on where a cell
  sits (no position enters its right-hand side, and each cell's arithmetic, the order of its
  sums included, is independent of the tile boundaries), so stepping a rolled state gives
  bitwise the rolled result of stepping the state.
* A uniform state stays uniform: every cell performs the same arithmetic (8192^2, and 14336^2,
  the largest grid of the reference's own benchmark list, 3.3 GB per array).
* The 16-bit deviation codes round-trip within half a unit of the tile scale at 8192^2.
* Tiling neutrality of the batch (strip width 64 or 128) on the 512 members of the batch
  benchmark, bitwise."""
import os
import sys

import numpy as np
import pytest

import fg2_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu

N = 4096


def steps(sim, x, nsteps, dt):
    sim.upload(x)
    t = 0.0
    for _ in range(nsteps):
        assert sim.step(t, dt) == 0
        t += dt
    return sim.download()


def test_translation_equivariance_4096(cuda):
    x = fg2_b200.setup_evaluate("kh", N, N, seed=2)[0].astype(np.float32)
    shift = (37, 129)  # not multiples of the tile height (35) or the strip width (128)
    with fg2_b200.Sim(N, N) as s:
        s.config()
        dt = 1.5e-5  # inside the CFL and diffusive limits of this state (about 1.86e-5)
        a = np.roll(steps(s, x, 3, dt), shift, axis=(0, 1))
        b = steps(s, np.ascontiguousarray(np.roll(x, shift, axis=(0, 1))), 3, dt)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n", [8192, 14336])  # 14336^2: the reference's largest benchmarked grid
def test_uniform_state_stays_uniform(n, cuda):
    x = np.empty((n, n, 4), np.float32)
    x[..., :] = np.array([0.25, 0.1, -0.2, np.log(0.9)], np.float32)
    with fg2_b200.Sim(n, n) as s:
        s.config()
        out = steps(s, x, 2, 1e-5)
    assert np.all(out == out[0, 0])
    assert np.allclose(out[0, 0], x[0, 0], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_codes_round_trip_8192(storage, cuda):
    n = 8192
    x = fg2_b200.setup_evaluate("kh", n, n, seed=2)[0].astype(np.float32)
    with fg2_b200.Sim(n, n, storage=storage) as s:
        s.config()
        s.upload(x)
        y = s.download()
    unit = {"f16": 2.0 ** -11, "bf16": 2.0 ** -8}[storage]
    flat = x.reshape(-1, 4).astype(np.float64)
    bg = flat.mean(0)
    bg[2] = 0.0
    scale = np.abs(flat - bg).max(0)
    err = np.abs(y.reshape(-1, 4).astype(np.float64) - flat).max(0)
    assert np.all(err <= 0.5 * unit * scale * 1.0001), err


def test_batch_strip_width_is_neutral_on_the_512_member_batch(cuda):
    sys.path.insert(0, ROOT)
    import bench
    sizes = bench.batch_sizes()
    outs = []
    for strip in (128, 64):
        with fg2_b200.Batch(sizes, scheme="hydro-isot") as b:
            b.set_box(2 * np.pi, 2 * np.pi)
            b.config()
            for k, m in enumerate(b.members):
                m.init("turb", seed=bench.BATCH_SEED * 100000 + k)
            b.set_strip(strip)
            assert b.advance(2, 1e-3, graph=True) == 0
            assert b.sync() == 0
            outs.append([m.download() for m in b.members[::37]])
    for a, c in zip(*outs):
        assert np.array_equal(a, c)

"""The single-grid autotuner (fg2_sim_autotune), the successor for one grid of the reference's
block-size heuristic (src/setup.cpp:39-58): it times steps of dt = 0 on the simulation's own
state for every tile height x occupancy candidate and keeps the fastest.  The state must come
out bitwise unchanged (FP32, and 16-bit storage with its rounding residual), and the chosen
tiling must give bitwise the results of the default one."""
import numpy as np
import pytest

import fg2_b200

pytestmark = pytest.mark.gpu


def steps(s, nsteps, dt):
    t = 0.0
    for _ in range(nsteps):
        assert s.step(t, dt) == 0
        t += dt
    return s.download()


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("n1,n2", [(300, 260), (1024, 1024)])
def test_autotune_leaves_the_state_and_the_results_unchanged(storage, n1, n2, cuda):
    x = fg2_b200.setup_evaluate("kh", n1, n2, seed=9)[0].astype(np.float32)
    dt = 2e-5
    with fg2_b200.Sim(n1, n2, storage=storage) as a, fg2_b200.Sim(n1, n2, storage=storage) as b:
        for s in (a, b):
            s.config()
            s.upload(x)
        before = a.download()
        ms = a.autotune(reps=2)
        assert ms > 0
        nb, ctas, tail = a.tiling()
        assert 1 <= nb <= 8 and ctas >= 0 and tail in (0, 1, 3)
        assert np.array_equal(a.download(), before)
        # the tuned tiling and the default one give bitwise the same steps
        assert np.array_equal(steps(a, 3, dt), steps(b, 3, dt))


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("n1,n2,walls", [(300, 260, False), (1000, 130, True), (64, 200, False)])
def test_tail_bands_give_the_default_results_bitwise(storage, n1, n2, walls, cuda):
    """Every tile height with and without one-block tail bands, in both launch directions (a
    step has three launches, so consecutive steps start in alternate directions), computes
    every row once and gives bitwise the default tiling's steps."""
    x = fg2_b200.setup_evaluate("kh", n1, n2, seed=4)[0].astype(np.float32)
    dt = 2e-5

    def run(tiling):
        with fg2_b200.Sim(n1, n2, storage=storage) as s:
            if walls:
                s.set_bcond(0, 0)
            s.config()
            s.upload(x)
            if tiling:
                s.set_tiling(*tiling)
                assert s.tiling() == tiling
            return steps(s, 4, dt)

    ref = run(None)
    for tiling in [(1, 0, 0), (3, 0, 1), (3, 1, 3), (5, 0, 2), (8, 0, 1), (8, 2, 0)]:
        assert np.array_equal(run(tiling), ref), tiling


def test_bad_tail_band_counts_are_refused(cuda):
    with fg2_b200.Sim(64, 64) as s:
        s.config()
        for bad in (-1, 65):
            with pytest.raises(fg2_b200.FG2Error):
                s.set_tiling(3, 0, bad)
        s.set_tiling(3, 0, 2)
        assert s.tiling() == (3, 0, 2)

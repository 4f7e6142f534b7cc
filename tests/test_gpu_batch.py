"""The batch path (fg2_batch_*): independent simulations of uneven sizes advanced by one
persistent substage launch per RK3 stage, checked member by member against the same
simulations advanced alone (the single-grid path, itself pinned to the reference's
arithmetic) and against the CPU port.  A batch applies 1/Delta to each derivative after the
weighted sum (as the reference's deriv.h does) instead of folding it into the weights, so
members agree with the single-grid path to rounding: per-field relative L2 <= 1e-5 after the
steps, the documented FP32 bar."""
import numpy as np
import pytest

import fg2_b200
from helpers import rel_l2
from oracle.oracle import Oracle, reference_delta

pytestmark = pytest.mark.gpu

SIZES = [(64, 64), (96, 128), (37, 53), (130, 67), (200, 260), (16, 300)]
TWO_PI = 2 * np.pi


def make_pair(scheme, sizes, setup, box=(1.0, 1.0), bconds=None, para=()):
    """A batch and, for each member, the same simulation alone, all initialised alike."""
    b = fg2_b200.Batch(sizes, scheme=scheme)
    b.set_box(*box)
    for kv in para:
        assert b.para(kv) is not None
    alone = []
    for k, (n1, n2) in enumerate(sizes):
        s = fg2_b200.Sim(n1, n2, scheme=scheme)
        s.set_box(*box)
        for kv in para:
            assert s.para(kv) is not None
        if bconds:
            s.set_bcond(*bconds[k])
            b.members[k].set_bcond(*bconds[k])
        s.config()
        s.init(setup, seed=100 + k)
        alone.append(s)
    b.config()
    for k, m in enumerate(b.members):
        m.init(setup, seed=100 + k)
    return b, alone


def close(b, alone):
    b.close()
    for s in alone:
        s.close()


def step_alone(s, steps, dt):
    t = 0.0
    for _ in range(steps):
        assert s.step(t, dt) == 0
        t += dt


@pytest.mark.parametrize("scheme,setup", [("hydro-isot", "turb"), ("hydro", "noise")])
@pytest.mark.parametrize("graph", [False, True])
def test_fixed_dt_members_match_single_grids(scheme, setup, graph, cuda):
    box = (TWO_PI, TWO_PI) if scheme == "hydro-isot" else (1.0, 1.0)
    b, alone = make_pair(scheme, SIZES, setup, box)
    try:
        dt = 2e-4 if scheme == "hydro" else 2e-3
        steps = 10
        assert b.advance(steps, dt, graph=graph) == 0
        assert b.sync() == 0
        for k, s in enumerate(alone):
            step_alone(s, steps, dt)
            err = rel_l2(b.members[k].download(), s.download())
            assert np.all(err <= 1e-5), (k, SIZES[k], err)
    finally:
        close(b, alone)


def test_device_cfl_members_match_single_grids(cuda):
    """dt <= 0: each member takes its own CFL step on the device, like Sim.advance(dt=0)."""
    b, alone = make_pair("hydro-isot", SIZES, "turb", (TWO_PI, TWO_PI))
    try:
        b.set_time(0.0)
        assert b.advance(8, 0.0, graph=True) == 0
        assert b.sync() == 0
        for k, s in enumerate(alone):
            s.set_time(0.0)
            s.advance(8, 0.0, graph=False)
            assert s.sync() == 0
            m = b.members[k]
            assert m.time() == pytest.approx(s.time(), rel=1e-6), k
            assert np.all(rel_l2(m.download(), s.download()) <= 1e-5), k
        # members of different sizes took different steps
        times = [m.time() for m in b.members]
        assert len(set(np.round(times, 12))) > 1
    finally:
        close(b, alone)


def test_mixed_boundaries_and_boxes(cuda):
    """Members with their own boundaries (walls / periodic) and boxes in one launch."""
    sizes = [(48, 40), (64, 96), (33, 70)]
    bconds = [(0, 0), (1, 0), (0, 1)]
    b, alone = make_pair("hydro", sizes, "noise", (1.0, 1.0), bconds)
    try:
        for s in (b.members[2], alone[2]):
            s.set_box(2.0, 0.5)
            s.config()
            s.init("noise", seed=102)
        assert b.advance(6, 1e-4, graph=False) == 0
        assert b.sync() == 0
        for k, s in enumerate(alone):
            step_alone(s, 6, 1e-4)
            assert np.all(rel_l2(b.members[k].download(), s.download()) <= 1e-5), k
    finally:
        close(b, alone)


def test_member_matches_cpu_port(cuda):
    """Members against the reference's arithmetic on the CPU (the port)."""
    sizes = [(40, 56), (72, 72)]
    with fg2_b200.Batch(sizes, scheme="hydro-isot") as b:
        b.set_box(TWO_PI, TWO_PI)
        b.config()
        x0 = []
        for k, m in enumerate(b.members):
            m.init("turb", seed=7 + k)
            x0.append(m.download())
        dt, steps = 2e-3, 10
        assert b.advance(steps, dt, graph=False) == 0
        assert b.sync() == 0
        o = Oracle("hydro-isot", "f32", "port")
        for k, (n1, n2) in enumerate(sizes):
            o.set_delta(*reference_delta(n1, n2, TWO_PI, TWO_PI))
            u = o.padded(x0[k])
            v = o.empty(n1, n2)
            o.run(u, v, 0.0, dt, steps)
            assert np.all(rel_l2(b.members[k].download(), o.interior(u)) <= 1e-5), k


def test_tiling_does_not_change_results(cuda):
    """Every strip width, tile height and CTA count gives bitwise the same state (each cell's
    arithmetic, the order of its sums included, does not depend on the tiling)."""
    outs = []
    for strip, nb, ctas in [(128, 5, 0), (128, 2, 1), (64, 8, 2), (128, 3, 3), (64, 3, 0), (64, 5, 6)]:
        b, alone = make_pair("hydro", SIZES[:4], "noise")
        try:
            b.set_strip(strip)
            b.set_tiling(nb, ctas)
            assert b.tiling() == (nb, ctas) and b.strip() == strip
            assert b.advance(4, 1e-4, graph=True) == 0
            assert b.sync() == 0
            outs.append([m.download() for m in b.members])
        finally:
            close(b, alone)
    for o in outs[1:]:
        for a, c in zip(outs[0], o):
            assert np.array_equal(a, c)


def test_autotune_keeps_state(cuda):
    b, alone = make_pair("hydro-isot", SIZES, "turb", (TWO_PI, TWO_PI))
    try:
        before = [m.download() for m in b.members]
        ms = b.autotune(reps=2)
        assert ms > 0
        nb, ctas = b.tiling()
        assert b.strip() in (64, 128)
        assert 1 <= nb <= 8 and 0 <= ctas <= 12 * 32 // b.strip()
        for a, m in zip(before, b.members):
            assert np.array_equal(a, m.download())
        assert b.advance(2, 1e-3) == 0 and b.sync() == 0
    finally:
        close(b, alone)


def test_autotune_keeps_16_bit_members_and_their_residuals(cuda):
    """A step of dt = 0 re-encodes 16-bit members and drops their rounding residuals, so the
    tuner keeps the members' arrays aside: the compensated states come back bitwise, and the
    next steps give what an untuned batch gives."""
    sizes = [(96, 96), (64, 160), (130, 70)]
    outs = []
    for tune in (True, False):
        with fg2_b200.Batch(sizes, scheme="hydro", storage="f16") as b:
            b.config()
            for k, m in enumerate(b.members):
                m.init("kh", seed=300 + k)
            before = [m.download() for m in b.members]
            if tune:
                assert b.autotune(reps=1) > 0
                for x, m in zip(before, b.members):
                    assert np.array_equal(x, m.download())
            assert b.advance(4, 1e-4, graph=True) == 0 and b.sync() == 0
            outs.append([m.download() for m in b.members])
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("storage", ["f16", "f64"])
def test_strip_width_does_not_change_results_of_other_storages(storage, cuda):
    """The 64-column strip with 16-bit deviation storage (its decode pass reads the narrower
    box) and with FP64 cells, bitwise against the default strip."""
    sizes = [(64, 64), (37, 130), (96, 40)]
    outs = []
    for strip in (128, 64):
        with fg2_b200.Batch(sizes, scheme="hydro", storage=storage) as b:
            b.config()
            for k, m in enumerate(b.members):
                m.init("noise", seed=200 + k)
            b.set_strip(strip)
            assert b.advance(4, 1e-4, graph=True) == 0
            assert b.sync() == 0
            outs.append([m.download() for m in b.members])
    for a, c in zip(*outs):
        assert np.array_equal(a, c)


def test_bad_strip_width_is_refused(cuda):
    with fg2_b200.Batch([(32, 32)], scheme="hydro") as b:
        with pytest.raises(fg2_b200.FG2Error):
            b.set_strip(96)
        assert b.strip() == 128


def test_nan_in_one_member_is_reported(cuda):
    sizes = [(32, 32), (48, 40)]
    with fg2_b200.Batch(sizes, scheme="hydro") as b:
        b.config()
        for k, m in enumerate(b.members):
            m.init("noise", seed=k)
        q = b.members[1].download()
        q[5, 7, 1] = np.nan
        b.members[1].upload(q)
        assert b.advance(1, 1e-4, graph=False) == 0
        assert b.sync() == 1
        assert b.members[1].sync() == 1
        assert b.members[0].sync() == 0


def test_member_shards_step_like_the_whole_batch(cuda):
    """A batch split over ranks by fg2_b200.shard_members: each shard, stepped as its own
    batch with device CFL steps, gives bitwise the member states and times of the whole batch
    (members share no data; each member's dt is its own)."""
    sizes = [(64, 64), (96, 128), (192, 64), (128, 128), (64, 96), (256, 192), (96, 96)]

    def run(idx):
        with fg2_b200.Batch([sizes[k] for k in idx], scheme="hydro-isot") as b:
            b.set_box(TWO_PI, TWO_PI)
            b.config()
            for m, k in zip(b.members, idx):
                m.init("turb", seed=50 + k)
            b.set_tiling(4, 0)
            b.set_time(0.0)
            assert b.advance(6, 0.0, graph=True) == 0
            assert b.sync() == 0
            return {k: (m.download(), m.time()) for m, k in zip(b.members, idx)}

    whole = run(list(range(len(sizes))))
    for world in (2, 3):
        for shard in fg2_b200.shard_members(sizes, world):
            for k, (x, t) in run(shard).items():
                assert np.array_equal(x, whole[k][0]) and t == whole[k][1], (world, k)

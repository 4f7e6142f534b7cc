"""The disk scheme (radiative torus on a log-r / theta grid, six fields per cell) through the
C ABI: the fused substage kernel with three field pairs and four mixed derivatives, the
scheme's own box and walls, its Euler hook (radiation-matter equilibrium), its curvilinear
CFL rate, and batches of disk members.  Tolerances as for the other schemes: per-field
relative L2 <= 1e-5 after 10 FP32 steps against the CPU port (itself bit-exact with the
reference's own disk headers on the golden vectors).

The reference's disk time step c / (n1/l1 + n2/l2) is far above the explicit limit of its
radiation diffusion (the reference blows up within a step at it), so stepping tests use a
fixed dt = 1e-4 on a smooth state, or a small Courant number."""
import os
import sys

import numpy as np
import pytest

import fg2_b200
from helpers import DEFAULTS, golden_cases, load_golden, rel_l2
from oracle.oracle import Oracle, disk_box, reference_delta, reference_dt

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import smooth_disk_state  # noqa: E402

pytestmark = pytest.mark.gpu

DT = 1e-4


def smooth(n1, n2, seed=1):
    l1, l2 = disk_box(n1, n2)
    return smooth_disk_state(np.random.default_rng(seed), n1, n2, l1, l2).astype(np.float32)


def port_steps(x0, steps, dt, para=None):
    n1, n2 = x0.shape[:2]
    o = Oracle("disk", "f32", "port")
    for k, v in {**DEFAULTS["disk"], **(para or {})}.items():
        o.set_para(k, v)
    o.set_delta(*reference_delta(n1, n2, *disk_box(n1, n2)))
    u = o.padded(x0)
    v = o.empty(n1, n2)
    assert o.run(u, v, 0.0, dt, steps, 0, 0) == 0
    return o.interior(u).copy()


def f64_euler(g):
    """The Euler hook in FP64 (the port at R = double) from the same inputs."""
    o = Oracle("disk", "f64", "port")
    for k, v in {**DEFAULTS["disk"], **g["para"]}.items():
        o.set_para(k, float(np.float32(v)) if g["prec"] == "f32" else v)
    o.set_delta(g["delta1"], g["delta2"])
    u = o.padded(g["x0"].astype(np.float64))
    o.euler(u, g["dt"])
    return o.interior(u).copy()


@pytest.mark.parametrize("name", [n for n in golden_cases() if n.startswith("disk")])
def test_euler_hook_matches_golden(name, cuda):
    """The same cells reach radiation-matter equilibrium.  The closed-form quartic root
    (src/disk/Euler.cuh:44-50) subtracts nearly equal numbers (b = a - x0 / 3a), so in FP32
    the reference's own result is about 1% (relative L2 of ln e) off FP64; the GPU must then
    stay within three times the reference's own FP32 error against FP64, as for kick."""
    g = load_golden(name)
    with fg2_b200.Sim(g["n1"], g["n2"], scheme="disk", storage=g["prec"]) as sim:
        for k, v in g["para"].items():
            assert sim.para(f"{k}={v!r}") is not None
        sim.config()
        sim.upload(g["x0"])
        sim.euler(g["dt"])
        out = sim.download()
    changed = (g["euler_out"] != g["x0"]).any(axis=2)
    assert np.array_equal((out != g["x0"]).any(axis=2), changed)
    if g["prec"] == "f64":
        assert np.all(rel_l2(out, g["euler_out"]) <= 1e-12), rel_l2(out, g["euler_out"])
        return
    truth = f64_euler(g)
    err_gpu, err_ref = rel_l2(out, truth), rel_l2(g["euler_out"], truth)
    assert np.all(err_gpu <= np.maximum(3 * err_ref, 1e-5)), (err_gpu, err_ref)


@pytest.mark.parametrize("n1,n2", [(64, 48), (130, 67), (37, 200), (256, 128)])
def test_port_parity_smooth_state(n1, n2, cuda):
    """Ragged and tile-straddling sizes; the simulation is never told its box or walls: the
    scheme's settings give them (src/disk/config.h:24-34), and the port runs with walls."""
    x0 = smooth(n1, n2)
    with fg2_b200.Sim(n1, n2, scheme="disk") as sim:
        sim.config()
        assert sim.getdt() == reference_dt(n1, n2, *disk_box(n1, n2))
        sim.upload(x0)
        for n in range(10):
            assert sim.step(n * DT, DT) == 0
        gpu = sim.download()
    err = rel_l2(gpu, port_steps(x0, 10, DT))
    assert np.all(err <= 1e-5), err


def test_hawley_setup_matches_host_evaluation(cuda):
    n1, n2 = 48, 64
    with fg2_b200.Sim(n1, n2, scheme="disk") as sim:
        sim.config()
        sim.init("Hawley")
        x = sim.download()
    l1, l2 = disk_box(n1, n2)
    # the host evaluation for an FP32 state (float arithmetic on the FP32 box, as the
    # reference's R = float) is what the simulation holds, bit for bit
    ref, known = fg2_b200.setup_evaluate("Hawley", n1, n2, scheme="disk", l1=l1, l2=l2, storage="f32")
    assert known
    assert np.array_equal(x, ref.astype(np.float32))
    assert x[..., 0].max() > np.log(0.5) and np.isclose(x[..., 0].min(), np.log(1e-4))


def test_cfl_getdt_matches_host_reduction(cuda):
    n1, n2 = 64, 80
    x0 = smooth(n1, n2, seed=3)
    with fg2_b200.Sim(n1, n2, scheme="disk") as s:
        s.config()
        s.upload(x0)
        s.set_dt_mode("cfl")
        dt = s.getdt()
    q = x0.astype(np.float64)
    p = {k: float(np.float32(v)) for k, v in DEFAULTS["disk"].items()}
    d1, d2 = reference_delta(n1, n2, *disk_box(n1, n2))
    i = np.arange(n1)[:, None]
    j = np.arange(n2)[None, :]
    th = (j + 0.5) * d2
    sphr = p["rin"] * np.exp((i + 0.5) * d1)
    cs = np.sqrt(p["gamma"] * (p["gamma"] - 1) * np.exp(q[..., 4]))
    u_r = np.sin(th) * q[..., 1] + np.cos(th) * q[..., 2]
    u_t = np.cos(th) * q[..., 1] - np.sin(th) * q[..., 2]
    rate = (((np.abs(u_r) + cs) / d1 + (np.abs(u_t) + cs) / d2) / sphr).max()
    D = max(p["nu"], p["dd"], p["ed"], p["rd"])
    dt_diff = 0.5 * 2.51 / (D * 1088 / 180 * (1 / d1 ** 2 + 1 / d2 ** 2))
    assert dt == pytest.approx(min(0.5 / rate, dt_diff), rel=1e-10)


def test_device_resident_cfl_steps_track_host_loop(cuda):
    """advance(dt <= 0): the curvilinear CFL rate folded into the last stage of the fused
    kernel, dt and t kept on the device; a small Courant number keeps the radiation
    diffusion stable."""
    n1, n2, nsteps = 64, 96, 8
    x0 = smooth(n1, n2, seed=5)
    with fg2_b200.Sim(n1, n2, scheme="disk") as a, fg2_b200.Sim(n1, n2, scheme="disk") as b:
        for s in (a, b):
            s.config()
            s.set_courant(2e-5)
            s.upload(x0)
            s.set_dt_mode("cfl")
        t = 0.0
        for _ in range(nsteps):
            dt = a.getdt()
            assert 0 < dt < 2e-4
            assert a.step(t, dt) == 0
            t += dt
        b.set_time(0.0)
        b.advance(nsteps, 0.0, graph=True)
        assert b.sync() == 0
        assert b.time() == pytest.approx(t, rel=1e-6)
        assert np.all(rel_l2(b.download(), a.download()) < 1e-5)


def test_batch_members_match_single_grids(cuda):
    sizes = [(40, 48), (64, 32), (24, 60), (130, 67)]
    states = [smooth(n1, n2, seed=10 + k) for k, (n1, n2) in enumerate(sizes)]
    runs = []
    for strip in (128, 64):  # both strip widths, bitwise alike
        with fg2_b200.Batch(sizes, scheme="disk") as b:
            b.config()
            b.set_strip(strip)
            for m, x in zip(b.members, states):
                m.upload(x)
            b.set_time(0.0)
            b.advance(10, DT, graph=True)
            assert b.sync() == 0
            runs.append([m.download() for m in b.members])
    got = runs[0]
    for a, c in zip(*runs):
        assert np.array_equal(a, c)
    for (n1, n2), x, out in zip(sizes, states, got):
        with fg2_b200.Sim(n1, n2, scheme="disk") as s:
            s.config()
            s.upload(x)
            for n in range(10):
                assert s.step(n * DT, DT) == 0
            alone = s.download()
        assert np.all(rel_l2(out, alone) <= 1e-5), ((n1, n2), rel_l2(out, alone))
        assert np.all(rel_l2(out, port_steps(x, 10, DT)) <= 1e-5)


def test_reference_mirror_api(cuda):
    """The function contract of src/fg2.h:70-84 on the disk library: setup / para / config /
    init / step give what the handle API gives (box and walls from the scheme's settings)."""
    lib = fg2_b200.load_library("disk")
    assert lib.fg2_setup(48, 64) > 0
    assert lib.fg2_para(b"alpha=0.02") == b"alpha = 0.02"
    lib.fg2_config()
    lib.fg2_init(b"smooth")
    assert lib.fg2_getdt() == reference_dt(48, 64, *disk_box(48, 64))
    for n in range(3):
        assert lib.fg2_step(n * DT, DT) == 0
    g = fg2_b200.Sim.__new__(fg2_b200.Sim)
    g.lib, g.h, g.n1, g.n2, g.nvar, g.host_dtype = lib, lib.fg2_global(), 48, 64, 6, np.float32
    ug = g.download()
    g.h = None  # not owned
    with fg2_b200.Sim(48, 64, scheme="disk") as s:
        s.para("alpha=0.02")
        s.config()
        s.init("smooth", seed=0)
        for n in range(3):
            assert s.step(n * DT, DT) == 0
        assert np.array_equal(s.download(), ug)

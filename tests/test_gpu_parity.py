"""Parity of the CUDA path (through the C ABI) with the reference's arithmetic: the
committed golden vectors (made by the reference's own headers compiled for the host) and
the CPU port on seeded inputs.  Tolerance: per-field relative L2 <= 1e-5 after 10 steps in
FP32 (the documented bar), <= 1e-12 in FP64."""
import numpy as np
import pytest

import fg2_b200
from helpers import DEFAULTS, golden_cases, load_golden, rel_l2
from oracle.oracle import Oracle, reference_delta, reference_dt

pytestmark = pytest.mark.gpu

TOL = {"f32": 1e-5, "f64": 1e-12}


def sim_for(g):
    sim = fg2_b200.Sim(g["n1"], g["n2"], scheme=g["scheme"], storage=g["prec"])
    sim.set_bcond(g["p1"], g["p2"])
    for k, v in g["para"].items():
        assert sim.para(f"{k}={v!r}") is not None
    sim.config()
    if g["has_rand"]:
        sim.set_forcing_phases(*g["rand"])
    sim.upload(g["x0"])
    return sim


@pytest.mark.parametrize("name", golden_cases())
def test_steps_match_golden(name, cuda):
    g = load_golden(name)
    with sim_for(g) as sim:
        t = 0.0
        for _ in range(g["steps"]):
            assert sim.step(t, g["dt"]) == 0
            t += g["dt"]
        out = sim.download()
    err = rel_l2(out, g["out"])
    assert np.all(err <= TOL[g["prec"]]), (name, err)


def f64_kick(g, v_in=None, beta=0.0):
    """The right-hand side in FP64 (the port at R = double) from the same FP32 inputs."""
    o = Oracle(g["scheme"], "f64", "port")
    for k, v in {**DEFAULTS[g["scheme"]], **g["para"]}.items():
        o.set_para(k, float(np.float32(v)) if g["prec"] == "f32" else v)
    o.set_delta(g["delta1"], g["delta2"])
    u = o.padded(g["x0"].astype(np.float64))
    o.bcond(u, g["p1"], g["p2"])
    v = o.empty(g["n1"], g["n2"]) if v_in is None else o.padded(v_in.astype(np.float64))
    o.kick(v, u, 0.0, beta)
    return o.interior(v).copy()


@pytest.mark.parametrize("name", golden_cases())
def test_kick_matches_golden(name, cuda):
    """One right-hand-side evaluation.  Its fields can be small differences of large terms
    (the pressure gradient of a pressure-balanced shear layer nearly cancels), so besides
    the golden comparison the GPU's rounding error against FP64 must stay within three times
    the reference's own FP32 rounding error, or 5e-6 (about 80 FP32 ulps), whichever is larger."""
    g = load_golden(name)
    with sim_for(g) as sim:
        sim.bcond()
        sim.kick(0.0, 0.0)
        f0 = sim.download_v()
        sim.upload_v(g["v_in"])
        sim.kick(0.0, -5.0 / 9.0)
        f1 = sim.download_v()
    tol = 1e-4 if g["prec"] == "f32" else 1e-12
    assert np.all(rel_l2(f0, g["kick0"]) <= tol), rel_l2(f0, g["kick0"])
    assert np.all(rel_l2(f1, g["kick1"]) <= tol), rel_l2(f1, g["kick1"])
    if g["prec"] == "f32":
        truth = f64_kick(g)
        assert np.all(rel_l2(f0, truth) <= np.maximum(3 * rel_l2(g["kick0"], truth), 5e-6))


@pytest.mark.parametrize("scheme,n1,n2", [("hydro", 256, 256), ("hydro", 37, 53), ("hydro", 64, 7),
                                          ("hydro", 130, 67), ("hydro-isot", 96, 160), ("hydro-isot", 5, 9)])
def test_port_parity_seeded(scheme, n1, n2, cuda):
    """The small plain configuration (256^2, Gaussian velocity noise, fixed dt) and ragged
    sizes: 10 GPU steps against 10 oracle steps from the same seeded state."""
    o = Oracle(scheme, "f32", "port")
    with fg2_b200.Sim(n1, n2, scheme=scheme) as sim:
        sim.config()
        sim.init("noise", seed=1)
        x0 = sim.download()
        l = (1.0, 1.0) if scheme == "hydro" else (2 * np.pi, 2 * np.pi)
        dt = reference_dt(n1, n2, *l)
        assert sim.getdt() == dt
        for n in range(10):
            assert sim.step(n * dt, dt) == 0
        gpu = sim.download()
    o.set_delta(*reference_delta(n1, n2, *l))
    u = o.padded(x0)
    v = o.empty(n1, n2)
    assert o.run(u, v, 0.0, dt, 10) == 0
    err = rel_l2(gpu, o.interior(u))
    assert np.all(err <= 1e-5), err


def test_small_plain_configuration_100_steps(cuda):
    """The small plain configuration in full: hydro 256^2 periodic, rho = 1, p = 1/gamma, Gaussian
    velocity noise (sigma 0.01, seed 1), the reference's dt = c / (n1/l1 + n2/l2) with c = 0.5,
    100 steps, against the reference's arithmetic on the CPU (the port, FP32) and against the
    FP64 port: the GPU's FP32 error against FP64 stays within 3x the CPU port's own FP32 error."""
    n1 = n2 = 256
    with fg2_b200.Sim(n1, n2) as sim:
        sim.config()
        sim.init("noise", seed=1)
        x0 = sim.download()
        dt = sim.getdt()
        assert dt == reference_dt(n1, n2, 1.0, 1.0)
        for n in range(100):
            assert sim.step(n * dt, dt) == 0
        gpu = sim.download()
    outs = {}
    for prec in ("f32", "f64"):
        o = Oracle("hydro", prec, "port")
        o.set_delta(*reference_delta(n1, n2, 1.0, 1.0) if prec == "f32" else (1.0 / n1, 1.0 / n2))
        u = o.padded(x0.astype(o.dtype))
        v = o.empty(n1, n2)
        assert o.run(u, v, 0.0, dt, 100) == 0
        outs[prec] = o.interior(u).astype(np.float64)
    assert np.all(rel_l2(gpu, outs["f32"]) <= 1e-5), rel_l2(gpu, outs["f32"])
    err_gpu, err_cpu = rel_l2(gpu, outs["f64"]), rel_l2(outs["f32"], outs["f64"])
    assert np.all(err_gpu <= np.maximum(3 * err_cpu, 1e-7)), (err_gpu, err_cpu)


def test_solve_frames_match_manual_steps(tmp_path, cuda):
    """solve() (src/solve.cpp:25-64) with the reference's getdt: the same steps as stepping by
    hand, frames dumped as %04d.raw with their times, the last step of each frame shortened."""
    n1, n2 = 48, 64
    with fg2_b200.Sim(n1, n2) as a, fg2_b200.Sim(n1, n2) as b:
        for s in (a, b):
            s.config()
            s.init("noise", seed=4)
        dt = a.getdt()
        t_final = 7.5 * dt
        rc, ms = a.solve(0.0, t_final, 0, 3, tmp_path)
        assert rc == 0 and ms > 0
        t = 0.0
        for k in range(1, 4):
            target = t_final - (3 - k) * (t_final / 3)
            while t < target:
                h = min(target - t, dt)
                assert b.step(t, h) == 0
                t = min(t + h, target)
            with fg2_b200.Sim(n1, n2) as c:
                c.config()
                assert c.load(tmp_path / f"{k:04d}.raw") == pytest.approx(target)
                assert np.array_equal(c.download(), b.download())
        assert np.array_equal(a.download(), b.download())


def test_solve_with_device_cfl_steps(tmp_path, cuda):
    with fg2_b200.Sim(64, 64) as s:
        s.config()
        s.init("kh", seed=2)
        s.set_dt_mode("cfl")
        rc, _ = s.solve(0.0, 2e-3, 0, 2, tmp_path)
        assert rc == 0
        assert s.time() == pytest.approx(2e-3, rel=1e-12)
        for k in (1, 2):
            with fg2_b200.Sim(64, 64) as c:
                c.config()
                assert c.load(tmp_path / f"{k:04d}.raw") == pytest.approx(1e-3 * k, rel=1e-12)


def test_fused_step_equals_reference_building_blocks(cuda):
    """step() == Euler + 3 x (bcond, kick, drift) through the separate entry points."""
    n1, n2 = 48, 40
    coef = [(0.0, 1.0 / 3.0), (-5.0 / 9.0, 15.0 / 16.0), (-153.0 / 128.0, 8.0 / 15.0)]
    with fg2_b200.Sim(n1, n2) as a, fg2_b200.Sim(n1, n2) as b:
        for s in (a, b):
            s.config()
            s.init("kh", seed=3)
        dt = a.getdt()
        assert a.step(0.0, dt) == 0
        for beta, gamma in coef:
            b.bcond()
            b.kick(0.0, beta)
            assert b.drift(float(np.float32(dt * gamma))) == 0
        ua, ub = a.download(), b.download()
    assert np.array_equal(ua, ub) or np.all(rel_l2(ua, ub) < 1e-7)


def test_graph_replay_is_bit_identical(cuda):
    with fg2_b200.Sim(96, 128) as a, fg2_b200.Sim(96, 128) as b:
        for s in (a, b):
            s.config()
            s.init("noise", seed=9)
        dt = a.getdt()
        a.advance(6, dt)
        b.advance(6, dt, graph=True)
        assert a.sync() == 0 and b.sync() == 0
        assert np.array_equal(a.download(), b.download())


def test_cfl_getdt_matches_host_reduction(cuda):
    n1, n2 = 64, 80
    with fg2_b200.Sim(n1, n2) as s:
        s.config()
        s.init("kh", seed=4)
        s.set_dt_mode("cfl")
        dt = s.getdt()
        q = s.download().astype(np.float64)
    gamma = float(np.float32(5 / 3))
    cs = np.sqrt(gamma * (gamma - 1) * np.exp(q[..., 3]))
    d1, d2 = reference_delta(n1, n2, 1.0, 1.0)
    rate = ((np.abs(q[..., 1]) + cs) / d1 + (np.abs(q[..., 2]) + cs) / d2).max()
    D = max(4 / 3 * float(np.float32(2e-4)), (gamma - 1) * float(np.float32(5e-4)))
    dt_diff = 0.5 * 2.51 / (D * 1088 / 180 * (1 / d1 ** 2 + 1 / d2 ** 2))
    assert dt == pytest.approx(min(0.5 / rate, dt_diff), rel=1e-12)


def test_getdt_after_a_step_reads_the_fused_max(cuda):
    """With CFL time steps, step() takes the signal max of the new state in its last stage and
    the next getdt() reads it: the same dt as a reduction pass over that state (the fused rate
    is evaluated in FP32, the pass in FP64), and the state is bitwise the one a step with the
    reference's getdt mode gives for the same dt."""
    n1, n2 = 64, 80
    with fg2_b200.Sim(n1, n2) as a, fg2_b200.Sim(n1, n2) as b, fg2_b200.Sim(n1, n2) as c:
        for s in (a, b, c):
            s.config()
            s.init("kh", seed=4)
        a.set_dt_mode("cfl")
        b.set_dt_mode("cfl")
        t = 0.0
        for _ in range(3):
            dt = a.getdt()
            assert a.step(t, dt) == 0 and c.step(t, dt) == 0
            t += dt
        fused = a.getdt()
        assert a.getdt() == fused  # no state change, no new max
        b.upload(a.download())
        assert fused == pytest.approx(b.getdt(), rel=1e-6)
        assert np.array_equal(a.download(), c.download())
        # a parameter or box change makes the kept max stale: getdt() takes a new one
        assert a.step(t, a.getdt()) == 0
        for s in (a, b):
            assert s.para("gamma=1.4") is not None
            s.set_box(1.0, 0.8)
        b.upload(a.download())
        assert a.getdt() == b.getdt()


def test_device_resident_dt_tracks_host_loop(cuda):
    """advance(dt <= 0): getdt fused into the last stage, dt and t kept on the device."""
    n1, n2, nsteps = 64, 64, 8
    with fg2_b200.Sim(n1, n2) as a, fg2_b200.Sim(n1, n2) as b:
        for s in (a, b):
            s.config()
            s.init("kh", seed=5)
            s.set_dt_mode("cfl")
        t = 0.0
        for _ in range(nsteps):
            dt = a.getdt()
            assert a.step(t, dt) == 0
            t += dt
        b.set_time(0.0)
        b.advance(nsteps, 0.0, graph=True)
        assert b.sync() == 0
        assert b.time() == pytest.approx(t, rel=1e-6)
        assert np.all(rel_l2(b.download(), a.download()) < 1e-5)


def test_t_end_caps_the_device_clock(cuda):
    with fg2_b200.Sim(32, 32) as s:
        s.config()
        s.init("noise", seed=1)
        s.set_time(0.0)
        s.advance(20, 0.0, t_end=1e-3)
        assert s.sync() == 0
        assert s.time() == pytest.approx(1e-3, rel=1e-12)


def test_nan_in_the_input_is_reported(cuda):
    with fg2_b200.Sim(32, 48) as s:
        s.config()
        s.init("noise", seed=1)
        x = s.download()
        x[10, 11, 1] = np.nan
        s.upload(x)
        assert s.step(0.0, 1e-3) == 1  # cudaErrorInvalidValue, src/step.cpp:38-40


def test_sums_are_reproducible_fp64(cuda):
    with fg2_b200.Sim(200, 160) as s:
        s.config()
        s.init("kh", seed=2)
        a, b = s.sums(), s.sums()
        q = s.download().astype(np.float64)
    assert np.array_equal(a, b)
    rho = np.exp(q[..., 0])
    ref = [rho.sum(), (rho * q[..., 1]).sum(), (rho * q[..., 2]).sum(),
           (rho * (np.exp(q[..., 3]) + 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2))).sum()]
    np.testing.assert_allclose(a, ref, rtol=1e-12, atol=1e-9)


def test_raw_frame_round_trip(cuda, tmp_path):
    path = tmp_path / "0001.raw"
    with fg2_b200.Sim(40, 56) as s:
        s.config()
        s.init("turb", seed=7)
        s.dump(path, 0.25)
        x = s.download()
    raw = np.fromfile(path, dtype=np.uint8)
    hdr = np.frombuffer(raw[:24].tobytes(), np.int32)
    assert list(hdr) == [40, 56, 4, 4, 1, 1]  # n1, n2, NVAR, sizeof(R), p1, p2 (src/io.cpp:62)
    assert np.frombuffer(raw[24:32].tobytes(), np.float64)[0] == 0.25
    data = np.frombuffer(raw[44:].tobytes(), np.float32).reshape(40, 56, 4)
    assert np.array_equal(data, x)
    with fg2_b200.Sim(40, 56) as s:
        assert s.load(path) == 0.25
        assert np.array_equal(s.download(), x)


def test_reference_mirror_api(cuda):
    """fg2_setup / fg2_para / fg2_config / fg2_init / fg2_getdt / fg2_step, the function
    contract of src/fg2.h:70-84, give what the handle API gives."""
    lib = fg2_b200.load_library("hydro")
    assert lib.fg2_setup(64, 48) > 0
    assert lib.fg2_para(b"--nus=3e-4") == b"nus = 0.0003"
    assert lib.fg2_para(b"nosuchkey=1") is None
    lib.fg2_config()
    lib.fg2_init(b"noise")
    dt = lib.fg2_getdt()
    for n in range(3):
        assert lib.fg2_step(n * dt, dt) == 0
    g = fg2_b200.Sim.__new__(fg2_b200.Sim)
    g.lib, g.h, g.n1, g.n2, g.nvar, g.host_dtype = lib, lib.fg2_global(), 64, 48, 4, np.float32
    ug = g.download()
    g.h = None  # not owned
    with fg2_b200.Sim(64, 48) as s:
        s.para("nus=3e-4")
        s.config()
        s.init("noise", seed=0)
        for n in range(3):
            assert s.step(n * dt, dt) == 0
        assert np.array_equal(s.download(), ug)


def test_reference_mirror_api_takes_interior_origin_pointers(cuda):
    """fg2_u/fg2_v/fg2_s hand out the arrays as the reference's globals hold them
    (global::u = base + HALF (s + NVAR), src/setup.cpp:64-72), and fg2_bcond / fg2_kick /
    fg2_drift, called with those pointers the way src/step.cpp:30-35 calls bcond / kick /
    drift, give what the handle API's bcond / kick / drift give."""
    import torch

    class DevArray:  # a view of device memory at a raw address (CUDA array interface)
        def __init__(self, ptr, n):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}

    lib = fg2_b200.load_library("hydro")
    n1, n2 = 40, 72
    assert lib.fg2_setup(n1, n2) > 0
    lib.fg2_config()
    lib.fg2_init(b"noise")
    s_el = lib.fg2_s()
    u, v = lib.fg2_u(), lib.fg2_v()
    g = fg2_b200.Sim.__new__(fg2_b200.Sim)
    g.lib, g.h, g.n1, g.n2, g.nvar, g.host_dtype = lib, lib.fg2_global(), n1, n2, 4, np.float32
    pitch, cell = g.layout()
    assert s_el == pitch and cell == 4
    x = g.download()
    # the interior-origin pointer indexes the interior like the reference: u[i s + j NVAR + f],
    # row -1 and column -1 are ghosts
    torch.cuda.synchronize()
    whole = torch.as_tensor(DevArray(u, (n1 - 1) * s_el + n2 * 4), device=cuda).cpu().numpy()
    for i, j in ((0, 0), (17, 33), (n1 - 1, n2 - 1)):
        assert np.array_equal(whole[i * s_el + j * 4: i * s_el + j * 4 + 4], x[i, j])
    # one RK3 substage by hand through the mirror API (src/step.cpp:30-35, i = 0)
    dt = lib.fg2_getdt()
    lib.fg2_bcond(u, 1, 1)
    lib.fg2_kick(v, u, 0.0, 0.0)
    lib.fg2_drift(u, v, dt / 3.0)
    torch.cuda.synchronize()
    ghost = torch.as_tensor(DevArray(u - 4 * (s_el + 4), 4), device=cuda).cpu().numpy()
    out_mirror = g.download()
    g.h = None  # not owned
    with fg2_b200.Sim(n1, n2) as s:
        s.config()
        s.upload(x)
        s.bcond()
        s.kick(0.0, 0.0)
        assert s.drift(dt / 3.0) == 0
        assert np.array_equal(s.download(), out_mirror)
    # ghost cell (-1, -1) after the periodic bcond is the image of interior cell (n1-1, n2-1)
    assert np.array_equal(ghost, x[n1 - 1, n2 - 1])

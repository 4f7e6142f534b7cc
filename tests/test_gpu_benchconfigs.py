"""Oracle parity at the benchmark configurations themselves, at their full sizes.

* The headline plain-FP32 workload: hydro 4096^2 periodic tanh Kelvin-Helmholtz layer (setup
  kh, seed 2), 10 RK3 steps of dt = 1.8e-5 (inside this state's CFL and diffusive limits),
  against the reference's own arithmetic compiled for the host (oracle/_ref, OpenMP on every
  host core; the port where that build is absent), the loop of src/step.cpp:22-43 around
  src/kick.cu:59-106 and src/drift.cu:21-39.
* The precision workload's grid: the same layer at 8192^2, 3 steps, against the port.
* The FP64 kernel the bench's accuracy and precision legs take as truth: the headline layer at
  4096^2, 3 steps in FP64, against the port in double (relative L2 <= 1e-12).
* Full-size batch members: the 512-member hydro-isot batch (sides 64..512, box 2 pi) and the
  64-member hydro batch (sides 512..2048), each advanced as one batch; members of the largest
  and smallest sides are compared with the port stepping them alone.

Bar: per-field relative L2 <= 1e-5 (FP32 against FP32 arithmetic, the documented bar).  The
turbulent batch members start from ln rho = 0 with a divergence-free velocity, so after a few
steps ln rho is a tiny field of its own rounding size; their first field is compared as the
density rho = exp(ln rho) instead."""
import os
import sys

import numpy as np
import pytest

import fg2_b200
from helpers import rel_l2
from oracle.oracle import Oracle, available, reference_delta

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def oracle(scheme, n1, n2, l1=1.0, l2=1.0, prefer="reference"):
    kind = prefer if available(scheme, "f32", prefer) else "port"
    o = Oracle(scheme, "f32", kind)
    o.threads(os.cpu_count() or 1)
    o.set_delta(*reference_delta(n1, n2, l1, l2))
    return o


def gpu_steps(n, x, nsteps, dt, storage="f32"):
    with fg2_b200.Sim(n, n, storage=storage) as s:
        s.config()
        s.upload(x)
        t = 0.0
        for _ in range(nsteps):
            assert s.step(t, dt) == 0
            t += dt
        return s.download()


def cpu_steps(o, x, nsteps, dt):
    n1, n2 = x.shape[:2]
    u = o.padded(x)
    v = o.empty(n1, n2)
    assert o.run(u, v, 0.0, dt, nsteps) == 0
    return o.interior(u)


def test_headline_workload_4096_against_the_reference(cuda):
    n, nsteps, dt = 4096, 10, 1.8e-5
    x = fg2_b200.setup_evaluate("kh", n, n, seed=2)[0].astype(np.float32)
    gpu = gpu_steps(n, x, nsteps, dt)
    ref = cpu_steps(oracle("hydro", n, n), x, nsteps, dt)
    err = rel_l2(gpu, ref)
    assert np.all(err <= 1e-5), err


def test_precision_grid_8192_against_the_port(cuda):
    n, nsteps, dt = 8192, 3, 8e-6
    x = fg2_b200.setup_evaluate("kh", n, n, seed=2)[0].astype(np.float32)
    gpu = gpu_steps(n, x, nsteps, dt)
    ref = cpu_steps(oracle("hydro", n, n, prefer="port"), x, nsteps, dt)
    err = rel_l2(gpu, ref)
    assert np.all(err <= 1e-5), err


def test_fp64_truth_at_4096_against_the_port(cuda):
    n, nsteps, dt = 4096, 3, 1.8e-5
    x = fg2_b200.setup_evaluate("kh", n, n, seed=2)[0]
    gpu = gpu_steps(n, x, nsteps, dt, storage="f64")
    o = Oracle("hydro", "f64", "port")
    o.threads(os.cpu_count() or 1)
    o.set_delta(1.0 / n, 1.0 / n)
    ref = cpu_steps(o, x, nsteps, dt)
    err = rel_l2(gpu, ref)
    assert np.all(err <= 1e-12), err


def batch_members_against_the_port(scheme, sizes, seed_of, box, dt, nsteps, setup):
    with fg2_b200.Batch(sizes, scheme=scheme) as b:
        b.set_box(*box)
        b.config()
        for k, m in enumerate(b.members):
            m.init(setup, seed=seed_of(k))
        sides = sorted({s[0] for s in sizes})
        sample = [sizes.index((sides[-1], sides[-1])), sizes.index((sides[0], sides[0]))]
        x0 = {k: b.members[k].download() for k in sample}
        assert b.advance(nsteps, dt, graph=True) == 0
        assert b.sync() == 0
        out = {k: b.members[k].download() for k in sample}

    def density_first(x):
        y = x.astype(np.float64)
        y[..., 0] = np.exp(y[..., 0])
        return y

    for k in sample:
        n1, n2 = sizes[k]
        ref = cpu_steps(oracle(scheme, n1, n2, *box, prefer="port"), x0[k], nsteps, dt)
        err = rel_l2(density_first(out[k]), density_first(ref))
        assert np.all(err <= 1e-5), (k, sizes[k], err)


def test_batch_c4_members_against_the_port(cuda):
    sys.path.insert(0, ROOT)
    import bench
    sizes = bench.batch_sizes()
    assert len(sizes) == 512
    batch_members_against_the_port("hydro-isot", sizes, lambda k: bench.BATCH_SEED * 100000 + k,
                                   (2 * np.pi, 2 * np.pi), 1e-3, 2, "turb")


def test_batch_c5_members_against_the_port(cuda):
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(bench.COMBINED_SEED)
    sizes = [(int(x), int(x)) for x in rng.choice(bench.COMBINED_SIDES, size=bench.COMBINED_COUNT)]
    batch_members_against_the_port("hydro", sizes, lambda k: bench.COMBINED_SEED * 1000 + k, (1.0, 1.0), 2e-5, 3,
                                   "turb")

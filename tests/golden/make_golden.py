"""Generate the golden vectors in tests/golden/*.npz from the REFERENCE's own arithmetic.

Runs only where the reference tree is present (it builds oracle/_ref/ from it): the
reference's src/deriv.h and src/<scheme>/eqns.cuh, Euler.cuh and bcond.cuh compiled for
the host by oracle/ref_harness.cpp, driven by the loops of oracle/loops.h that follow
src/step.cpp, src/kick.cu, src/drift.cu and src/bcond.cu.  The fixtures then travel
with the repository; tests read them, never the reference.

    python tests/golden/make_golden.py              (rebuilds oracle/, rewrites every fixture)
    python tests/golden/make_golden.py disk_torus   (only the cases whose name starts so)

Every case stores its inputs, parameters and outputs, so a test needs nothing else.
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle, default_box, disk_box, reference_delta, reference_dt  # noqa: E402


def noise_state(rng, n1, n2, nv, sigma=0.01, lne=np.log(0.9)):
    x = np.zeros((n1, n2, nv))
    x[..., 1:3] = rng.normal(0.0, sigma, (n1, n2, 2))
    if nv == 4:
        x[..., 3] = lne
    return x


def shear_state(rng, n1, n2, nv, gamma=5.0 / 3.0):
    """A small tanh shear layer with density contrast (the shape of the large-grid case)."""
    x1 = (np.arange(n1) + 0.5) / n1
    x2 = (np.arange(n2) + 0.5) / n2
    X, Y = np.meshgrid(x1, x2, indexing="ij")
    inside = np.abs(Y - 0.5) < 0.25
    rho = np.where(inside, 1.0, 2.0)
    ux = 0.5 * np.tanh((np.abs(Y - 0.5) - 0.25) / 0.05)
    uy = 0.01 * np.sin(4 * np.pi * X) + rng.normal(0, 1e-4, X.shape)
    x = np.zeros((n1, n2, nv))
    x[..., 0] = np.log(rho)
    x[..., 1] = ux
    x[..., 2] = uy
    if nv == 4:
        x[..., 3] = np.log(2.5 / (rho * (gamma - 1.0)))
    return x


def torus_state(rng, n1, n2, l1, l2, M=1.0, rin=3.0, gamma=5.0 / 3.0, ar=1.0e8, noise=1e-3):
    """The disk scheme's Hawley torus (src/disk/init.h:31-58) at cell centres
    (ln(r / r_in), theta), in double, with Gaussian noise on ln rho, u_R and u_z."""
    lnr = l1 * (np.arange(n1) + 0.5) / n1
    th = l2 * (np.arange(n2) + 0.5) / n2
    LR, TH = np.meshgrid(lnr, th, indexing="ij")
    r = rin * np.exp(LR)
    R = r * np.sin(TH)
    q0, r0, d0, e0, bg = 2.0, 16.0, 1.0, 0.01, 1.0e-4
    g1, q1 = gamma - 1.0, 2.0 * q0 - 2.0
    lK = np.sqrt(M * r0 ** (q1 - 1.0))
    K = g1 * e0 / d0 ** g1
    h = gamma * e0 - M / r0 + lK * lK / (r0 ** q1 * q1) + M / r - lK * lK / (R ** q1 * q1)
    den = np.sign(h) * (np.abs(h) * g1 / (gamma * K)) ** (1.0 / g1)
    Omg = lK * R ** (-q0)
    low = den < bg
    den = np.where(low, bg, den)
    Omg = np.where(low, Omg * np.sin(TH) ** 2, Omg)
    eng = K * den ** g1 / g1
    tbg = K * bg ** g1
    rad = ar * tbg ** 4 / bg
    x = np.zeros((n1, n2, 6))
    x[..., 0] = np.log(den) + rng.normal(0.0, noise, LR.shape)
    x[..., 1] = rng.normal(0.0, noise, LR.shape)
    x[..., 2] = rng.normal(0.0, noise, LR.shape)
    x[..., 3] = Omg
    x[..., 4] = np.log(eng)
    x[..., 5] = np.log(rad)
    return x


def smooth_disk_state(rng, n1, n2, l1, l2, gamma=5.0 / 3.0, ar=1.0e8, rin=3.0):
    """A smooth disk-scheme state: a density bump on the equator, Keplerian rotation, small
    long-wavelength poloidal velocities, a smooth temperature and radiation off its local
    equilibrium by a smooth factor (e_rad = a_r T^4 / rho exp(0.3 cos 2 theta), so that
    free-free heating / cooling is not a difference of equal numbers), plus a little noise
    on ln rho (the disk scheme's "smooth" setup, with numpy's generator)."""
    lnr = l1 * (np.arange(n1) + 0.5) / n1
    th = l2 * (np.arange(n2) + 0.5) / n2
    LR, TH = np.meshgrid(lnr, th, indexing="ij")
    r = rin * np.exp(LR)
    x = np.zeros((n1, n2, 6))
    bump = np.exp(-((LR - 0.5 * l1) ** 2 + (TH - 0.5 * np.pi) ** 2) / 0.3)
    x[..., 0] = -3.0 + 3.0 * bump + rng.normal(0.0, 1e-4, LR.shape)
    x[..., 1] = 1e-3 * np.sin(2 * np.pi * LR / l1) * np.sin(TH)
    x[..., 2] = 1e-3 * np.cos(2 * np.pi * LR / l1) * np.sin(2 * TH)
    x[..., 3] = (r * np.sin(TH) + 1.0) ** -1.5
    eng = 0.01 * (1.0 + 0.2 * np.cos(TH) * np.sin(np.pi * LR / l1))
    x[..., 4] = np.log(eng)
    temp = (gamma - 1.0) * eng
    x[..., 5] = np.log(ar * temp ** 4 / np.exp(x[..., 0])) + 0.3 * np.cos(2.0 * TH)
    return x


DEFAULTS = {
    "hydro": {"gamma": 5 / 3, "nus": 2e-4, "nub": 0.0, "kappa": 5e-4, "dd": 0.0},
    "hydro-isot": {"dd": 0.0, "nus": 2e-4, "nub": 0.0, "cs2": 1.0, "f": 0.0, "k": -8.0},
    "disk": {"M": 1.0, "rS": 2.0, "rin": 3.0, "gamma": 5 / 3, "nus": 0.0, "nub": 0.0, "kappa": 0.0,
             "alpha": 0.01, "ar": 1.0e8, "es": 1.0, "ff": 0.0, "dd": 1.0e-4, "nu": 2.0e-4, "ed": 5.0e-4,
             "rd": 5.0e-4},
}

# The disk's own time step (src/getdt.cpp:26 on its box) is far above the explicit limit of
# its radiation diffusion, and the reference blows up within one step at it; its cases use a
# fixed dt inside that limit instead, on a smooth state.  The torus (whose sharp edge makes
# the radiation terms stiffer still) is checked through its right-hand side alone (0 steps),
# and so is free-free cooling (ff > 0), which is stiffer again; disk cases also store one
# application of the Euler hook (radiation-matter equilibrium) to the initial state.
DISK_DT = 1.0e-4

CASES = [
    # name, scheme, prec, n1, n2, init, para, steps, p1, p2, euler rand
    ("hydro_noise_f32", "hydro", "f32", 24, 32, "noise", {}, 10, 1, 1, None),
    ("hydro_noise_f64", "hydro", "f64", 24, 32, "noise", {}, 10, 1, 1, None),
    ("hydro_shear_odd_f32", "hydro", "f32", 19, 37, "shear", {"dd": 1e-3}, 10, 1, 1, None),
    ("hydro_nub_f32", "hydro", "f32", 16, 24, "noise", {"nub": 1e-3, "gamma": 1.4, "kappa": 1e-3}, 10, 1, 1, None),
    ("hydro_walls_f32", "hydro", "f32", 20, 28, "shear", {}, 10, 0, 0, None),
    ("isot_noise_f32", "hydro-isot", "f32", 24, 32, "noise", {}, 10, 1, 1, None),
    ("isot_noise_f64", "hydro-isot", "f64", 24, 32, "noise", {}, 10, 1, 1, None),
    ("isot_kolmogorov_f32", "hydro-isot", "f32", 20, 24, "noise", {"f": 0.05, "k": -2, "dd": 1e-3}, 10, 1, 1, None),
    ("isot_forced_f32", "hydro-isot", "f32", 16, 20, "noise", {"f": 0.05, "k": 2}, 5, 1, 1, (1.234, 4.321)),
    ("isot_walls_f32", "hydro-isot", "f32", 18, 22, "noise", {}, 10, 0, 0, None),
    ("disk_torus_f32", "disk", "f32", 24, 32, "torus", {}, 0, 0, 0, None),
    ("disk_smooth_f32", "disk", "f32", 24, 32, "smooth", {}, 10, 0, 0, None),
    ("disk_smooth_f64", "disk", "f64", 24, 32, "smooth", {}, 10, 0, 0, None),
    ("disk_smooth_ff_f32", "disk", "f32", 20, 26, "smooth", {"ff": 1e-3, "nus": 1e-4, "kappa": 1e-3, "nub": 1e-4}, 0, 0, 0, None),
]


def make_case(name, scheme, prec, n1, n2, init, para, steps, p1, p2, rand, seed):
    o = Oracle(scheme, prec, "reference")
    rng = np.random.default_rng(seed)
    l1, l2 = disk_box(n1, n2, prec == "f64") if scheme == "disk" else default_box(scheme)
    if prec == "f32":  # Delta and getdt() in R = float (src/config.cpp:39, src/getdt.cpp:26)
        d1, d2 = reference_delta(n1, n2, l1, l2)
        dt = reference_dt(n1, n2, l1, l2)
    else:  # R = double
        d1, d2 = l1 / n1, l2 / n2
        dt = 0.5 / (n1 / l1 + n2 / l2)
    if scheme == "disk":
        dt = DISK_DT
    o.set_delta(d1, d2)
    for k, val in para.items():
        o.set_para(k, val)
    if init == "noise":
        x0 = noise_state(rng, n1, n2, o.nvar)
    elif init == "torus":
        x0 = torus_state(rng, n1, n2, l1, l2)
    elif init == "smooth":
        x0 = smooth_disk_state(rng, n1, n2, l1, l2)
    else:
        x0 = shear_state(rng, n1, n2, o.nvar)
    x0 = x0.astype(o.dtype)

    # one kick from the initial state (v = F(u) at beta = 0, then beta != 0 on a known v)
    u = o.padded(x0)
    o.bcond(u, p1, p2)
    v = o.empty(n1, n2)
    o.kick(v, u, 0.0, 0.0)
    f0 = o.interior(v).copy()
    v_in = rng.normal(0, 1.0, (n1, n2, o.nvar)).astype(o.dtype)
    v = o.padded(v_in)
    o.kick(v, u, 0.0, -5.0 / 9.0)
    f1 = o.interior(v).copy()

    # the Euler hook alone on the initial state (disk: radiation-matter equilibrium)
    extra = {}
    if scheme == "disk":
        u = o.padded(x0)
        o.euler(u, dt)
        extra["euler_out"] = o.interior(u).copy()

    # `steps` full RK3 steps at the reference's fixed dt
    u = o.padded(x0)
    v = o.empty(n1, n2)
    if rand is not None:
        o.set_rand(*rand)
    nan = 0
    t = 0.0
    for _ in range(steps):
        nan |= o.step(u, v, t, dt, p1, p2)
        t += dt
    # reset parameters for the next case (the harness keeps them in globals)
    for k, val in DEFAULTS[scheme].items():
        o.set_para(k, val)
    return dict(
        scheme=scheme, prec=prec, n1=n1, n2=n2, p1=p1, p2=p2, steps=steps, dt=dt,
        l1=l1, l2=l2, delta1=d1, delta2=d2,
        para_keys=np.array(list(para.keys()), dtype="U16"),
        para_vals=np.array(list(para.values()), dtype=np.float64),
        rand=np.array(rand if rand is not None else (0.0, 0.0)), has_rand=rand is not None,
        x0=x0, v_in=v_in, kick0=f0, kick1=f1, out=o.interior(u).copy(), nan=nan, **extra,
    )


# The reference tree these vectors are made from (read-only); FG2_REFERENCE overrides it.
REFERENCE_TREE = os.environ.get("FG2_REFERENCE", "/root/reference")


def main(prefixes=()):
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=" + REFERENCE_TREE])
    for seed, case in enumerate(CASES, start=1):
        if prefixes and not any(case[0].startswith(p) for p in prefixes):
            continue
        d = make_case(*case, seed=seed)
        path = os.path.join(HERE, case[0] + ".npz")
        np.savez_compressed(path, seed=seed, **d)
        print(f"{case[0]:24s} {os.path.getsize(path):7d} B  nan={d['nan']}  "
              f"|out|max={np.abs(d['out']).max():.4g}")


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))

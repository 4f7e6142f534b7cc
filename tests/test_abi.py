"""The C-ABI libraries (no GPU calls): every symbol include/fg2_b200.h declares is
exported by both scheme libraries, the scheme metadata matches the reference's plug-in
(field order, para keys, flop count), and the host-side initial conditions are the
documented seeded formulas."""
import ctypes
import os
import re

import numpy as np
import pytest

import fg2_b200
from fg2_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fg2_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fg2_\w+)\s*\(", text)))


def test_header_declares_the_reference_contract():
    names = declared_symbols()
    # src/fg2.h:70-84 mirrored one for one
    for ref in ("setup", "config", "para", "init", "load", "dump", "getdt", "step", "kick", "drift", "bcond",
                "Euler"):
        assert f"fg2_{ref}" in names
    assert len(names) > 50


@pytest.mark.parametrize("scheme", build.SCHEMES)
def test_library_exports_every_declared_symbol(scheme):
    lib = ctypes.CDLL(build.lib_path(scheme))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_scheme_metadata():
    h = fg2_b200.load_library("hydro")
    assert h.fg2_scheme_name() == b"hydro" and h.fg2_nvar() == 4 and h.fg2_eqns_flop() == 289
    assert [h.fg2_field_name(f) for f in range(4)] == [b"lnd", b"u1", b"u2", b"lne"]
    assert [h.fg2_para_key(k) for k in range(h.fg2_para_count())] == [b"gamma", b"nus", b"nub", b"kappa", b"dd"]
    i = fg2_b200.load_library("hydro-isot")
    assert i.fg2_scheme_name() == b"hydro-isot" and i.fg2_nvar() == 3 and i.fg2_eqns_flop() == 214
    assert [i.fg2_para_key(k) for k in range(i.fg2_para_count())] == [b"dd", b"nus", b"nub", b"cs2", b"f", b"k"]
    assert h.fg2_field_name(4) is None
    d = fg2_b200.load_library("disk")
    assert d.fg2_scheme_name() == b"disk" and d.fg2_nvar() == 6 and d.fg2_eqns_flop() == 733
    assert [d.fg2_field_name(f) for f in range(6)] == [b"lnd", b"ur", b"uz", b"Omg", b"lne", b"lner"]
    assert [d.fg2_para_key(k) for k in range(d.fg2_para_count())] == [
        b"M", b"rS", b"rin", b"gamma", b"nus", b"nub", b"kappa", b"alpha", b"ar", b"es", b"ff", b"dd", b"nu",
        b"ed", b"rd"]


def test_six_field_scheme_refuses_16bit_storage_before_any_device_call():
    lib = fg2_b200.load_library("disk")
    for code in (fg2_b200.STORAGE["f16"], fg2_b200.STORAGE["bf16"]):
        assert not lib.fg2_sim_create(64, 64, code, None)
        assert b"at most 4 fields" in lib.fg2_last_error()


def test_disk_host_setup_is_the_hawley_torus():
    """src/disk/init.h:31-58 at cell centres (ln(r / r_in), theta) of the scheme's own box."""
    from oracle.oracle import disk_box
    n1, n2 = 24, 32
    l1, l2 = disk_box(n1, n2, f64=True)
    x, known = fg2_b200.setup_evaluate("Hawley", n1, n2, scheme="disk", l1=l1, l2=l2)
    assert known and x.shape == (n1, n2, 6)
    assert np.all(x[..., 1:3] == 0.0) and np.all(x[..., 5] == x[0, 0, 5])
    assert np.isclose(x[..., 0].min(), np.log(1e-4)) and x[..., 0].max() > np.log(0.5)
    # pressure maximum of the torus at r0 = 16 on the equator, density d0 = 1 there
    lnr = l1 * (np.arange(n1) + 0.5) / n1
    i = int(np.argmin(np.abs(3.0 * np.exp(lnr) - 16.0)))
    assert abs(x[i, n2 // 2, 0]) < 0.2


def test_bad_sizes_rejected_before_any_device_call():
    lib = fg2_b200.load_library("hydro")
    assert not lib.fg2_sim_create(2, 64, 0, None)
    assert b"ghost width" in lib.fg2_last_error()
    assert not lib.fg2_sim_create(64, 64, 7, None)


def test_tiling_entry_points_reject_null_handles_and_bad_values():
    lib = fg2_b200.load_library("hydro")
    t = ctypes.c_int(-7)
    assert lib.fg2_sim_set_tail(None, 1) != 0
    assert lib.fg2_sim_get_tail(None, ctypes.byref(t)) != 0 and t.value == -7
    assert lib.fg2_sim_set_tiling(None, 3) != 0
    assert lib.fg2_sim_set_occupancy(None, 1) != 0


# ---- host-side initial conditions -------------------------------------------------------
M64 = (1 << 64) - 1


def splitmix_uniforms(seed, n):
    """The library's splitmix64 stream as uniforms in (0, 1] (pure Python, exact)."""
    out = np.empty(n)
    s = seed & M64
    for k in range(n):
        s = (s + 0x9E3779B97F4A7C15) & M64
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        z ^= z >> 31
        out[k] = ((z >> 11) + 1) * (1.0 / 9007199254740992.0)
    return out


def test_noise_setup_is_seeded_box_muller():
    n1, n2, seed, sigma = 6, 7, 1234, 0.01
    q, known = fg2_b200.setup_evaluate("noise", n1, n2, "hydro", seed=seed)
    assert known
    u = splitmix_uniforms(seed, 2 * n1 * n2).reshape(-1, 2)
    r = np.sqrt(-2 * np.log(u[:, 0]))
    t = 2 * np.pi * u[:, 1]
    np.testing.assert_allclose(q[..., 1].ravel(), sigma * r * np.cos(t), rtol=1e-13, atol=1e-17)
    np.testing.assert_allclose(q[..., 2].ravel(), sigma * r * np.sin(t), rtol=1e-13, atol=1e-17)
    assert np.all(q[..., 0] == 0)
    gamma = 5 / 3
    np.testing.assert_allclose(q[..., 3], np.log(1 / (gamma * (gamma - 1))), rtol=1e-15)


def test_kh_setup_profile():
    n = 64
    q, _ = fg2_b200.setup_evaluate("kh", n, n, "hydro", seed=2)
    y = (np.arange(n) + 0.5) / n
    s = np.tanh((np.abs(y - 0.5) - 0.25) / 0.01)
    np.testing.assert_allclose(q[0, :, 1], 0.5 * s, rtol=1e-12, atol=1e-15)
    rho = np.exp(q[0, :, 0])
    np.testing.assert_allclose(rho, 1.5 + 0.5 * s, rtol=1e-12)
    p = rho * (2 / 3) * np.exp(q[0, :, 3])  # p = (gamma - 1) rho e
    np.testing.assert_allclose(p, 2.5, rtol=1e-12)
    x = (np.arange(n) + 0.5) / n
    assert np.abs(q[:, 0, 2] - 0.01 * np.sin(4 * np.pi * x)).max() < 1e-3


@pytest.mark.parametrize("scheme,mach", [("hydro", 0.5), ("hydro-isot", 0.3)])
def test_turbulence_setup_spectrum(scheme, mach):
    n = 64
    q, _ = fg2_b200.setup_evaluate("turb", n, n, scheme, seed=5)
    u1, u2 = q[..., 1], q[..., 2]
    assert np.sqrt((u1 ** 2 + u2 ** 2).mean()) == pytest.approx(mach, rel=1e-12)
    f1, f2 = np.fft.fft2(u1), np.fft.fft2(u2)
    k = np.fft.fftfreq(n, 1.0 / n)
    K1, K2 = np.meshgrid(k, k, indexing="ij")
    kk = np.hypot(K1, K2)
    power = np.abs(f1) ** 2 + np.abs(f2) ** 2
    assert power[(kk < 2) | (kk > 16)].sum() < 1e-20 * power.sum()          # band limit
    assert np.abs(K1 * f1 + K2 * f2).max() < 1e-9 * np.abs(f1).max()      # solenoidal
    # shell energy ~ k^-2 on average: fit the slope over the band
    shells = np.arange(2, 17)
    e = np.array([power[(kk >= s - 0.5) & (kk < s + 0.5)].sum() for s in shells])
    slope = np.polyfit(np.log(shells), np.log(e), 1)[0]
    assert -2.6 < slope < -1.4


def test_unknown_setup_gives_zeros():
    q, known = fg2_b200.setup_evaluate("no-such-setup", 4, 4, "hydro")
    assert not known and np.all(q == 0)


def test_isot_setups_use_the_2pi_box():
    q, known = fg2_b200.setup_evaluate("Kf", 8, 8, "hydro-isot", para={"dd": 0, "nus": 0.01, "nub": 0, "cs2": 1,
                                                                       "f": 0.1, "k": 2}, seed=3)
    assert known
    x = 2 * np.pi * (np.arange(8) + 0.5) / 8
    np.testing.assert_allclose(q[:, 0, 2], 0.1 / (0.01 * 4) * np.cos(2 * x), atol=1e-7)


def _centres(n1, n2, l1=1.0, l2=1.0):
    x = l1 * (np.arange(n1) + 0.5) / n1 - 0.5 * l1
    y = l2 * (np.arange(n2) + 0.5) / n2 - 0.5 * l2
    return np.meshgrid(x, y, indexing="ij")


def _fermi_dirac(x, d):
    return 1.0 / (np.exp(x / d) + 1.0)


@pytest.mark.parametrize("name", ["blast", "bow", "implos", "Sod"])
def test_reference_hydro_setups(name):
    """The reference's named initial conditions (src/hydro/init.h:26-94) at cell centres of the
    unit box, restated here in numpy: (ln rho, u1, u2, ln e)."""
    n1, n2, g = 40, 56, 5.0 / 3.0
    q, known = fg2_b200.setup_evaluate(name, n1, n2, "hydro")
    assert known
    X, Y = _centres(n1, n2)
    zero = np.zeros_like(X)
    if name == "blast":
        e = np.where(X * X + Y * Y < 0.01, 1.0, 0.01) / (g - 1.0)
        ref = [zero, zero, zero, np.log(e)]
    elif name == "bow":
        d = 9.9 * _fermi_dirac(np.sqrt(X * X + Y * Y) - 0.01, 0.001) + 0.1
        ref = [np.log(d), (10.0 / d - 1.0) / 99.0, zero, np.log(0.01 / d / (g - 1.0))]
    elif name == "implos":
        f = _fermi_dirac(0.15 - np.abs(X) - np.abs(Y), 0.001)
        d, p = 0.125 + 0.875 * f, 0.14 + 0.86 * f
        ref = [np.log(d), zero, zero, np.log(p / d / (g - 1.0))]
    else:
        left = np.fmod(X - 2 * Y + 1.5, 1.0) < 0.5
        d, p = np.where(left, 1.0, 0.125), np.where(left, 1.0, 0.1)
        ref = [np.log(d), zero, zero, np.log(p / d / (g - 1.0))]
    np.testing.assert_allclose(q, np.stack(ref, axis=-1), rtol=1e-12, atol=1e-14)


def test_reference_kh_setup_is_a_seeded_step_profile():
    """src/hydro/init.h:60-76: rho 2 and u1 = 0.5 within |y| < 1/4, rho 1 and u1 = -0.5 outside,
    each u1 plus uniform noise in [-0.005, 0.005) (rand() replaced by the seeded generator),
    p = 2.5."""
    n1, n2, g = 32, 48, 5.0 / 3.0
    q, known = fg2_b200.setup_evaluate("KH", n1, n2, "hydro", seed=9)
    assert known
    _, Y = _centres(n1, n2)
    inner = np.abs(Y) < 0.25
    np.testing.assert_allclose(np.exp(q[..., 0]), np.where(inner, 2.0, 1.0), rtol=1e-14)
    noise = q[..., 1] - np.where(inner, 0.5, -0.5)
    assert np.all(np.abs(noise) <= 0.005 + 1e-15) and noise.std() > 0.002
    np.testing.assert_allclose(np.exp(q[..., 0]) * (g - 1) * np.exp(q[..., 3]), 2.5, rtol=1e-13)
    assert np.all(q[..., 2] == 0)
    q2, _ = fg2_b200.setup_evaluate("KH", n1, n2, "hydro", seed=9)
    assert np.array_equal(q, q2)

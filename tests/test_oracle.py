"""The oracle pinned against the reference: the port (oracle/port.cpp) and, where the
reference tree is present, the reference's own headers compiled for the host
(oracle/_ref/) reproduce the committed golden vectors bit for bit; stencil known-answer
tests on polynomials and a convergence-order check."""
import numpy as np
import pytest

from helpers import DEFAULTS, golden_cases, load_golden
from oracle.oracle import HALO, Oracle, available, reference_delta, reference_dt


def configured(g, kind):
    o = Oracle(g["scheme"], g["prec"], kind)
    for k, v in DEFAULTS[g["scheme"]].items():
        o.set_para(k, v)
    for k, v in g["para"].items():
        o.set_para(k, v)
    o.set_delta(g["delta1"], g["delta2"])
    o.set_rand(*g["rand"])
    return o


@pytest.mark.parametrize("kind", ["port", "reference"])
@pytest.mark.parametrize("name", golden_cases())
def test_golden_bit_exact(name, kind):
    g = load_golden(name)
    if not available(g["scheme"], g["prec"], kind):
        pytest.skip(f"{kind} checker not built here (the reference tree is absent)")
    o = configured(g, kind)
    n1, n2 = g["n1"], g["n2"]
    # kick from the initial state, beta = 0 and beta = -5/9 on a given v
    u = o.padded(g["x0"])
    o.bcond(u, g["p1"], g["p2"])
    v = o.empty(n1, n2)
    o.kick(v, u, 0.0, 0.0)
    assert np.array_equal(o.interior(v), g["kick0"])
    v = o.padded(g["v_in"])
    o.kick(v, u, 0.0, -5.0 / 9.0)
    assert np.array_equal(o.interior(v), g["kick1"])
    if "euler_out" in g:  # the Euler hook alone
        u = o.padded(g["x0"])
        o.euler(u, g["dt"])
        assert np.array_equal(o.interior(u), g["euler_out"])
    # full steps
    u = o.padded(g["x0"])
    v = o.empty(n1, n2)
    nan, t = 0, 0.0
    for _ in range(g["steps"]):
        nan |= o.step(u, v, t, g["dt"], g["p1"], g["p2"])
        t += g["dt"]
    assert nan == g["nan"] == 0
    assert np.array_equal(o.interior(u), g["out"])


def test_reference_dt_and_delta():
    # src/getdt.cpp:26 and src/config.cpp:39 evaluated in float with a double quotient
    assert reference_dt(256, 256, 1.0, 1.0) == pytest.approx(0.5 / 512, rel=1e-15)
    d1, d2 = reference_delta(48, 32, 1.0, 1.0)
    assert d1 == float(np.float32(1 / 48)) and d2 == float(np.float32(1 / 32))


def grid(n1, n2, h1, h2):
    x = np.arange(-HALO, n1 + HALO) * h1
    y = np.arange(-HALO, n2 + HALO) * h2
    return np.meshgrid(x, y, indexing="ij")


@pytest.mark.parametrize("kind", ["port", "reference"])
def test_stencils_exact_on_polynomials(kind):
    """D1/D2 exact to degree 6, D11/D22 to degree 7, D12 on x^a y^b for a, b <= 3."""
    if not available("hydro", "f64", kind):
        pytest.skip("reference checker not built here")
    o = Oracle("hydro", "f64", kind)
    n1, n2 = 14, 18
    h1, h2 = 0.37 / n1, 0.29 / n2
    o.set_delta(h1, h2)
    X, Y = grid(n1, n2, h1, h2)
    Xi, Yi = X[HALO:-HALO, HALO:-HALO], Y[HALO:-HALO, HALO:-HALO]
    rng = np.random.default_rng(7)
    for deg, which, var in ((6, 0, "x"), (6, 1, "y"), (7, 2, "x"), (7, 3, "y")):
        c = rng.normal(size=deg + 1)
        s = X if var == "x" else Y
        si = Xi if var == "x" else Yi
        u = np.zeros((n1 + 6, n2 + 6, 4))
        u[..., 2] = np.polynomial.polynomial.polyval(s, c)
        p = np.polynomial.polynomial.polyder(c, 1 if which < 2 else 2)
        exact = np.polynomial.polynomial.polyval(si, p)
        got = o.deriv(u, which, 2)
        assert np.abs(got - exact).max() <= 1e-8 * max(1.0, np.abs(exact).max())
    for a in range(4):
        for b in range(4):
            u = np.zeros((n1 + 6, n2 + 6, 4))
            u[..., 1] = X ** a * Y ** b
            exact = (a * b * Xi ** max(a - 1, 0) * Yi ** max(b - 1, 0)) if a and b else 0 * Xi
            assert np.abs(o.deriv(u, 4, 1) - exact).max() < 1e-9


def test_stencil_convergence_order_six():
    o = Oracle("hydro", "f64", "port")
    errs = []
    for n in (16, 32):
        h = 1.0 / n
        o.set_delta(h, h)
        X, Y = grid(n, n, h, h)
        u = np.zeros((n + 6, n + 6, 4))
        u[..., 0] = np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
        Xi, Yi = X[HALO:-HALO, HALO:-HALO], Y[HALO:-HALO, HALO:-HALO]
        exact = {0: 2 * np.pi * np.cos(2 * np.pi * Xi) * np.cos(2 * np.pi * Yi),
                 2: -(2 * np.pi) ** 2 * np.sin(2 * np.pi * Xi) * np.cos(2 * np.pi * Yi),
                 4: -(2 * np.pi) ** 2 * np.cos(2 * np.pi * Xi) * np.sin(2 * np.pi * Yi)}
        errs.append({w: np.abs(o.deriv(u, w, 0) - e).max() for w, e in exact.items()})
    for w in errs[0]:
        order = np.log2(errs[0][w] / errs[1][w])
        assert order > 5.7, (w, order)


def test_uniform_state_is_steady():
    o = Oracle("hydro", "f32", "port")
    n1 = n2 = 16
    o.set_delta(*reference_delta(n1, n2, 1.0, 1.0))
    x = np.zeros((n1, n2, 4), np.float32)
    x[..., 0], x[..., 1], x[..., 2], x[..., 3] = 0.3, 0.0, 0.0, -0.2
    u = o.padded(x)
    v = o.empty(n1, n2)
    for _ in range(3):
        assert o.step(u, v, 0.0, reference_dt(n1, n2, 1.0, 1.0)) == 0
    assert np.array_equal(o.interior(u), x)


def test_nan_input_flags_status():
    """A NaN planted in the oracle's input makes step() report it (src/step.cpp:38-40)."""
    o = Oracle("hydro", "f32", "port")
    n1 = n2 = 12
    o.set_delta(*reference_delta(n1, n2, 1.0, 1.0))
    x = np.zeros((n1, n2, 4), np.float32)
    x[5, 7, 1] = np.nan
    u = o.padded(x)
    v = o.empty(n1, n2)
    assert o.step(u, v, 0.0, 1e-3) == 1


@pytest.mark.parametrize("name,shape,seed", [("kh", (300, 257), 2), ("noise", (64, 37), 1)])
def test_numpy_setups_match_the_library(name, shape, seed):
    """oracle/setups.py (the input of the bench's reference arm, which must not load the
    product) gives the library's initial conditions to within one FP32 ulp."""
    import fg2_b200
    from oracle import setups
    a = getattr(setups, name)(*shape, seed=seed)
    b, _ = fg2_b200.setup_evaluate(name, shape[0], shape[1], seed=seed)
    a32, b32 = a.astype(np.float32), b.astype(np.float32)
    ulps = np.abs(a32.view(np.int32).astype(np.int64) - b32.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1
    assert np.abs(a - b).max() <= 1e-15 * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("name", ["blast", "bow", "implos", "Sod", "KH", "nosuch"])
def test_named_setups_match_the_reference(name, prec):
    """The reference's named initial conditions (src/hydro/init.h, compiled for the host from
    the reference tree and evaluated at the cell centres of src/init.cpp:30-36) against the
    library's setups for a state of the same precision, bit for bit.  KH draws its noise from
    rand() in the reference and from the seeded generator here, so its u1 is left out."""
    import ctypes
    import fg2_b200
    from oracle.oracle import lib_path
    if not available("hydro", prec, "reference"):
        pytest.skip("reference checker not built here (the reference tree is absent)")
    lib = ctypes.CDLL(lib_path("hydro", prec, "reference"))
    lib.orc_set_para.argtypes = [ctypes.c_char_p, ctypes.c_double]
    lib.orc_ref_setup.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_void_p]
    for key, val in DEFAULTS["hydro"].items():
        lib.orc_set_para(key.encode(), val)
    n1, n2 = 96, 80
    dtype = np.float32 if prec == "f32" else np.float64
    ref = np.zeros((n1, n2, 4), dtype)
    lib.orc_ref_setup(name.encode(), n1, n2, 1.0, 1.0, ref.ctypes.data)
    ours = fg2_b200.setup_evaluate(name, n1, n2, seed=1, storage=prec)[0].astype(dtype)
    fields = [0, 2, 3] if name == "KH" else [0, 1, 2, 3]
    assert np.array_equal(ours[..., fields], ref[..., fields])


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_disk_torus_matches_the_reference(prec):
    """The Hawley torus of the disk scheme (src/disk/init.h, compiled for the host) on the
    scheme's own box, against the library's setup for a state of the same precision, bit for
    bit."""
    import ctypes
    import fg2_b200
    from oracle.oracle import disk_box, lib_path
    if not available("disk", prec, "reference"):
        pytest.skip("reference checker not built here (the reference tree is absent)")
    lib = ctypes.CDLL(lib_path("disk", prec, "reference"))
    lib.orc_set_para.argtypes = [ctypes.c_char_p, ctypes.c_double]
    lib.orc_ref_setup.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_void_p]
    for key, val in DEFAULTS["disk"].items():
        lib.orc_set_para(key.encode(), val)
    n1, n2 = 48, 64
    l1, l2 = disk_box(n1, n2, prec == "f64")
    dtype = np.float32 if prec == "f32" else np.float64
    ref = np.zeros((n1, n2, 6), dtype)
    lib.orc_ref_setup(b"Hawley", n1, n2, l1, l2, ref.ctypes.data)
    ours = fg2_b200.setup_evaluate("Hawley", n1, n2, scheme="disk", l1=l1, l2=l2, seed=1, storage=prec)[0]
    assert np.array_equal(ours.astype(dtype), ref)

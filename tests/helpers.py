"""Shared helpers of the test suite."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# The reference's parameter defaults per scheme (src/hydro/eqns.cuh:19-24,
# src/hydro-isot/eqns.cuh:19-25, src/disk/eqns.cuh:19-36).
DEFAULTS = {
    "hydro": {"gamma": 5 / 3, "nus": 2e-4, "nub": 0.0, "kappa": 5e-4, "dd": 0.0},
    "hydro-isot": {"dd": 0.0, "nus": 2e-4, "nub": 0.0, "cs2": 1.0, "f": 0.0, "k": -8.0},
    "disk": {"M": 1.0, "rS": 2.0, "rin": 3.0, "gamma": 5 / 3, "nus": 0.0, "nub": 0.0, "kappa": 0.0,
             "alpha": 0.01, "ar": 1.0e8, "es": 1.0, "ff": 0.0, "dd": 1.0e-4, "nu": 2.0e-4, "ed": 5.0e-4,
             "rd": 5.0e-4},
}


def golden_cases():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        d = {k: z[k] for k in z.files}
    for k in ("scheme", "prec"):
        d[k] = str(d[k])
    for k in ("n1", "n2", "p1", "p2", "steps", "nan", "seed"):
        d[k] = int(d[k])
    for k in ("dt", "l1", "l2", "delta1", "delta2"):
        d[k] = float(d[k])
    d["para"] = dict(zip([str(k) for k in d["para_keys"]], [float(v) for v in d["para_vals"]]))
    d["has_rand"] = bool(d["has_rand"])
    return d


def rel_l2(a, b):
    """Per-field ||a - b||_2 / ||b||_2 over the last axis (fields)."""
    a = np.asarray(a, np.float64).reshape(-1, a.shape[-1])
    b = np.asarray(b, np.float64).reshape(-1, b.shape[-1])
    num = np.sqrt(((a - b) ** 2).sum(0))
    den = np.sqrt((b ** 2).sum(0))
    return num / np.where(den > 0, den, 1.0)


# ---- 16-bit deviation storage, emulated on the CPU ----------------------------------------
SCALE_TILE = 64


def round_bf16(a):
    """Round to the nearest BF16 number (ties to even), returned as float64."""
    b = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def round16(a, storage):
    return np.asarray(a, np.float16).astype(np.float64) if storage == "f16" else round_bf16(a)


def deviation_codes(x0, reflect=(2,)):
    """The storage's codes for the initial state x0 (n1, n2, NVAR): per-field background (the
    field mean; 0 for the fields a reflecting wall negates) and per-64x64-tile scale (the largest
    deviation on the tile, 1 where there is none), broadcast to cells."""
    n1, n2, nv = x0.shape
    bg = x0.reshape(-1, nv).mean(0)
    for f in reflect:
        bg[f] = 0.0
    t1, t2 = -(-n1 // SCALE_TILE), -(-n2 // SCALE_TILE)
    pad = np.full((t1 * SCALE_TILE, t2 * SCALE_TILE, nv), np.nan)
    pad[:n1, :n2] = np.abs(x0 - bg)
    s = np.nanmax(pad.reshape(t1, SCALE_TILE, t2, SCALE_TILE, nv), axis=(1, 3))
    # a field equal to its background on a tile (to the float rounding of the mean) has scale 1
    s[~(s > 1e-6 * np.maximum(np.abs(bg), 1.0))] = 1.0
    return bg, np.repeat(np.repeat(s, SCALE_TILE, 0), SCALE_TILE, 1)[:n1, :n2]


def stencil_on_codes(oracle, x0, steps, dt, storage, p1=1, p2=1):
    """The accuracy floor of any scheme whose stencil reads the 16-bit numbers: the state T is
    kept exactly (FP64, every rounding compensated), but each substage evaluates the right-hand
    side on the numbers the storage holds for T, bg + s round16((T - bg) / s).  `oracle` is
    an FP64 Oracle with its Delta set.  Returns T after `steps` RK3 steps."""
    from oracle.oracle import HALO
    beta = [0.0, -5.0 / 9.0, -153.0 / 128.0]
    gamma = [1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0]
    bg, s = deviation_codes(x0)
    T = np.asarray(x0, np.float64).copy()
    n1, n2, _ = T.shape
    up = oracle.padded(T)
    vp = oracle.padded(np.zeros_like(T))
    inner = (slice(HALO, HALO + n1), slice(HALO, HALO + n2))
    for _ in range(steps):
        for k in range(3):
            up[inner] = bg + s * round16((T - bg) / s, storage)
            oracle.bcond(up, p1, p2)
            oracle.kick(vp, up, 0.0, beta[k])
            T = T + gamma[k] * dt * vp[inner]
    return T


def compensated_stencil(oracle, x0, steps, dt, storage, p1=1, p2=1):
    """The library's compensated 16-bit scheme, emulated with FP64 arithmetic: each state is
    stored as the 16-bit number S = bg + s round16((u - bg) / s) and its residual as the FP16
    number r = (S - u) / s * 4096; every substage's stencil reads T = S - s r / 4096, v is
    stored as plain 16-bit numbers between substages.  Returns T after `steps` RK3 steps."""
    from oracle.oracle import HALO
    beta = [0.0, -5.0 / 9.0, -153.0 / 128.0]
    gamma = [1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0]
    bg, s = deviation_codes(x0)
    n1, n2, _ = x0.shape

    def store(u):  # (S, T) of a state u
        S = bg + s * round16((u - bg) / s, storage)
        r = round16((S - u) / s * 4096.0, "f16")
        return S - s * r / 4096.0

    T = store(np.asarray(x0, np.float64))
    up = oracle.padded(T)
    vp = oracle.padded(np.zeros_like(T))
    inner = (slice(HALO, HALO + n1), slice(HALO, HALO + n2))
    for _ in range(steps):
        for k in range(3):
            up[inner] = T
            oracle.bcond(up, p1, p2)
            oracle.kick(vp, up, 0.0, beta[k])
            v = vp[inner].copy()
            T = store(T + gamma[k] * dt * v)
            if k < 2:
                vp[inner] = round16(v, storage)
    return T

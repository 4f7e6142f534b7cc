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

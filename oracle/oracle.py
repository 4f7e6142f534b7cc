"""ctypes front end of the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg and the
`--impl reference` arm) import this module.  It loads one of

  oracle/lib/liborc_port_<scheme>_<prec>.so   this project's restatement (oracle/port.cpp)
  oracle/_ref/liborc_ref_<scheme>_<prec>.so   the reference's own stencil/RHS headers compiled
                                              for the host (oracle/ref_harness.cpp)

Arrays use the reference's host layout: numpy (n1 + 6, n2 + 6, NVAR), C order, three
ghost cells on every side (src/setup.cpp:60-72 with a dense row pitch).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HALO = 3
SCHEMES = {"hydro": ("hydro", 4), "hydro-isot": ("isot", 3), "isot": ("isot", 3), "disk": ("disk", 6)}


def lib_path(scheme="hydro", prec="f32", kind="port"):
    tag, _ = SCHEMES[scheme]
    if kind == "port":
        return os.path.join(HERE, "lib", f"liborc_port_{tag}_{prec}.so")
    if kind == "reference":
        return os.path.join(HERE, "_ref", f"liborc_ref_{tag}_{prec}.so")
    raise ValueError(kind)


def available(scheme="hydro", prec="f32", kind="port"):
    return os.path.exists(lib_path(scheme, prec, kind))


class Oracle:
    """One scheme at one precision; the C side keeps its parameters in globals, so use
    one Oracle object per (scheme, precision, kind) at a time."""

    def __init__(self, scheme="hydro", prec="f32", kind="port"):
        path = lib_path(scheme, prec, kind)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`)")
        self.lib = ctypes.CDLL(path)
        self.scheme, self.prec, self.kind = scheme, prec, kind
        self.dtype = np.float32 if prec == "f32" else np.float64
        L = self.lib
        P = ctypes.c_void_p
        I, D = ctypes.c_int, ctypes.c_double
        L.orc_nvar.restype = I
        L.orc_real_size.restype = I
        L.orc_set_para.argtypes = [ctypes.c_char_p, D]
        L.orc_set_para.restype = I
        L.orc_get_para.argtypes = [ctypes.c_char_p]
        L.orc_get_para.restype = D
        L.orc_set_delta.argtypes = [D, D]
        L.orc_set_rand.argtypes = [D, D]
        L.orc_threads.argtypes = [I]
        L.orc_threads.restype = I
        L.orc_kick.argtypes = [P, P, I, I, D, D]
        L.orc_drift.argtypes = [P, P, I, I, D]
        L.orc_drift.restype = I
        L.orc_bcond.argtypes = [P, I, I, I, I]
        L.orc_euler.argtypes = [P, I, I, D]
        L.orc_step.argtypes = [P, P, I, I, D, D, I, I]
        L.orc_step.restype = I
        L.orc_run.argtypes = [P, P, I, I, D, D, I, I, I]
        L.orc_run.restype = I
        L.orc_deriv.argtypes = [P, I, I, I, I, P]
        self.nvar = L.orc_nvar()
        assert L.orc_real_size() == np.dtype(self.dtype).itemsize

    # ---- arrays ---------------------------------------------------------------------
    def empty(self, n1, n2, fill=None):
        a = np.empty((n1 + 2 * HALO, n2 + 2 * HALO, self.nvar), dtype=self.dtype)
        a.fill(-np.finfo(self.dtype).max if fill is None else fill)  # src/setup.cpp:80-83
        return a

    def padded(self, interior):
        """(n1, n2, NVAR) interior -> padded array with ghosts unset (-max)."""
        n1, n2, nv = interior.shape
        assert nv == self.nvar
        a = self.empty(n1, n2)
        a[HALO:HALO + n1, HALO:HALO + n2] = interior
        return a

    @staticmethod
    def interior(a):
        return a[HALO:-HALO, HALO:-HALO]

    def _chk(self, a):
        assert a.dtype == self.dtype and a.flags.c_contiguous and a.shape[2] == self.nvar
        return a.ctypes.data

    # ---- parameters -----------------------------------------------------------------
    def set_para(self, key, val):
        if self.lib.orc_set_para(key.encode(), float(val)) != 0:
            raise KeyError(key)

    def get_para(self, key):
        return self.lib.orc_get_para(key.encode())

    def set_delta(self, d1, d2):
        self.lib.orc_set_delta(float(d1), float(d2))

    def set_rand(self, r1, r2):
        self.lib.orc_set_rand(float(r1), float(r2))

    def threads(self, n=0):
        return self.lib.orc_threads(int(n))

    # ---- the step -------------------------------------------------------------------
    def kick(self, v, u, t, beta):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        self.lib.orc_kick(self._chk(v), self._chk(u), n1, n2, float(t), float(beta))

    def drift(self, u, v, dt):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        return self.lib.orc_drift(self._chk(u), self._chk(v), n1, n2, float(dt))

    def bcond(self, u, p1=1, p2=1):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        self.lib.orc_bcond(self._chk(u), n1, n2, int(p1), int(p2))

    def euler(self, u, dt):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        self.lib.orc_euler(self._chk(u), n1, n2, float(dt))

    def step(self, u, v, t, dt, p1=1, p2=1):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        return self.lib.orc_step(self._chk(u), self._chk(v), n1, n2, float(t), float(dt), int(p1), int(p2))

    def run(self, u, v, t, dt, nsteps, p1=1, p2=1):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        return self.lib.orc_run(self._chk(u), self._chk(v), n1, n2, float(t), float(dt), int(nsteps),
                                int(p1), int(p2))

    def deriv(self, u, which, field):
        n1, n2 = u.shape[0] - 2 * HALO, u.shape[1] - 2 * HALO
        out = np.zeros((n1, n2), dtype=self.dtype)
        self.lib.orc_deriv(self._chk(u), n1, n2, int(which), int(field), out.ctypes.data)
        return out


# Reference-default parameters and the box each scheme forces (src/hydro/eqns.cuh:19-24,
# src/hydro-isot/eqns.cuh:19-25, src/hydro-isot/config.h:21-26, src/disk/config.h:24-34,
# src/global.cpp:28).
def default_box(scheme, n1=None, n2=None):
    tag = SCHEMES[scheme][0]
    if tag == "isot":
        return (2 * np.pi, 2 * np.pi)
    if tag == "disk":
        return disk_box(n1, n2)
    return (1.0, 1.0)


def disk_box(n1, n2, f64=False):
    """The disk scheme's box (src/disk/config.h:24-34): theta over the full pi wedge and a
    log-r extent 2 n1 asinh(pi / (2 n2)) that makes the cells about square, evaluated with
    R-typed intermediates (R = float unless f64)."""
    R = np.float64 if f64 else np.float32
    l2 = R(np.pi)
    hd2 = R(0.5 * np.float64(l2) / n2)
    hd1 = R(np.log(np.float64(hd2) + np.sqrt(np.float64(R(hd2 * hd2)) + 1.0)))
    l1 = R(2.0 * np.float64(hd1) * n1)
    return float(l1), float(l2)


def reference_dt(n1, n2, l1, l2, c=0.5):
    """getdt() of the reference (src/getdt.cpp:26): (E)c / (n1/l1 + n2/l2), where the
    quotients and their sum are evaluated in R = float and only the final division in E."""
    l1f, l2f, cf = np.float32(l1), np.float32(l2), np.float32(c)
    den = np.float32(np.float32(n1) / l1f) + np.float32(np.float32(n2) / l2f)
    return float(np.float64(cf) / np.float64(den))


def reference_delta(n1, n2, l1, l2):
    """Delta1, Delta2 = l1/n1, l2/n2 evaluated in R = float (src/config.cpp:39)."""
    return float(np.float32(np.float32(l1) / np.float32(n1))), float(np.float32(np.float32(l2) / np.float32(n2)))

"""fg2_b200 -- B200-native time step of fg2's 2D compressible hydrodynamics.

Python host side over the per-scheme C-ABI libraries (include/fg2_b200.h):

    import fg2_b200
    sim = fg2_b200.Sim(256, 256, scheme="hydro")        # setup()
    sim.para("nus=1e-4")                                # para("key=val")
    sim.config()                                        # config()
    sim.init("noise", seed=1)                           # init()
    dt = sim.getdt()                                    # getdt()
    status = sim.step(0.0, dt)                          # step(t, dt) -> 0, or 1 on NaN
    state = sim.download()                              # (n1, n2, NVAR) array

Names, argument meanings and return conventions follow the reference's function contract
(src/fg2.h:60-84).  There is no CPU fallback: constructing a Sim without the built
library, or without a CUDA device, raises.
"""
import ctypes
import os

import numpy as np

from .build import lib_path, SCHEMES

__all__ = ["Sim", "load_library", "setup_evaluate", "SCHEMES", "STORAGE", "FG2Error"]

STORAGE = {"f32": 0, "f64": 1, "f16": 2, "bf16": 3}
DT_REFERENCE, DT_CFL = 0, 1
_LIBS = {}


class FG2Error(RuntimeError):
    pass


def _bind(lib):
    P, I, D, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    U64, SZ, LL = ctypes.c_uint64, ctypes.c_size_t, ctypes.c_longlong
    sig = {
        "fg2_scheme_name": (S, []), "fg2_nvar": (I, []), "fg2_field_name": (S, [I]),
        "fg2_eqns_flop": (I, []), "fg2_para_count": (I, []), "fg2_para_key": (S, [I]),
        "fg2_last_error": (S, []),
        "fg2_setup_evaluate": (I, [S, I, I, D, D, P, U64, I, P]),
        "fg2_sim_create": (P, [I, I, I, P]), "fg2_sim_destroy": (None, [P]),
        "fg2_sim_device_bytes": (SZ, [P]), "fg2_sim_storage": (I, [P]),
        "fg2_sim_set_box": (I, [P, D, D]), "fg2_sim_set_courant": (I, [P, D]), "fg2_sim_set_tiling": (I, [P, I]),
        "fg2_sim_set_occupancy": (I, [P, I]), "fg2_sim_get_tiling": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "fg2_sim_autotune": (I, [P, I, ctypes.POINTER(D)]), "fg2_sim_set_tail": (I, [P, I]),
        "fg2_tile_bands": (I, [I, I, I, I, ctypes.POINTER(I), I]),
        "fg2_sim_get_tail": (I, [P, ctypes.POINTER(I)]),
        "fg2_sim_set_bcond": (I, [P, I, I]), "fg2_sim_para": (S, [P, S]),
        "fg2_sim_get_para": (I, [P, S, ctypes.POINTER(D)]), "fg2_sim_config": (I, [P]),
        "fg2_sim_init": (I, [P, S, U64]), "fg2_sim_upload": (I, [P, P]), "fg2_sim_download": (I, [P, P]),
        "fg2_sim_upload_v": (I, [P, P]), "fg2_sim_download_v": (I, [P, P]),
        "fg2_sim_set_dt_mode": (I, [P, I]), "fg2_sim_getdt": (D, [P]),
        "fg2_sim_step": (I, [P, D, D]), "fg2_sim_advance": (I, [P, I, D, D]),
        "fg2_sim_advance_graph": (I, [P, I, D, D]), "fg2_sim_sync": (I, [P]),
        "fg2_sim_stage": (I, [P, I, D]),
        "fg2_sim_set_time": (I, [P, D]), "fg2_sim_time": (D, [P]), "fg2_sim_last_dt": (D, [P]),
        "fg2_sim_clear_status": (None, [P]),
        "fg2_sim_kick": (I, [P, D, D]), "fg2_sim_drift": (I, [P, D]), "fg2_sim_bcond": (I, [P]),
        "fg2_sim_euler": (I, [P, D]), "fg2_sim_set_forcing_phases": (I, [P, D, D]),
        "fg2_sim_seed_forcing": (I, [P, U64]), "fg2_sim_sums": (I, [P, P]),
        "fg2_sim_u": (P, [P]), "fg2_sim_v": (P, [P]), "fg2_sim_stream": (P, [P]),
        "fg2_sim_layout": (I, [P, ctypes.POINTER(LL), ctypes.POINTER(LL)]),
        "fg2_sim_dump": (I, [P, S, D]), "fg2_sim_load": (I, [P, S, ctypes.POINTER(D)]),
        "fg2_setup": (SZ, [I, I]), "fg2_config": (None, []), "fg2_para": (S, [S]), "fg2_init": (None, [S]),
        "fg2_load": (D, [S]), "fg2_dump": (None, [S, D]), "fg2_getdt": (D, []), "fg2_step": (I, [D, D]),
        "fg2_kick": (None, [P, P, ctypes.c_float, ctypes.c_float]),
        "fg2_drift": (None, [P, P, ctypes.c_float]), "fg2_bcond": (None, [P, I, I]),
        "fg2_Euler": (None, [P, ctypes.c_float]), "fg2_global": (P, []),
        "fg2_u": (P, []), "fg2_v": (P, []), "fg2_s": (ctypes.c_longlong, []),
        "fg2_sums_noalloc": (I, [P, I, I, LL, I, P, P]),
        "fg2_sim_solve": (I, [P, D, D, I, I, S, ctypes.POINTER(D)]),
        "fg2_sim_test_stall_waits": (I, [P, I]),
        "fg2_batch_create": (P, [I, P, P, I, P]), "fg2_batch_destroy": (None, [P]),
        "fg2_batch_count": (I, [P]), "fg2_batch_cells": (LL, [P]), "fg2_batch_device_bytes": (SZ, [P]),
        "fg2_batch_stream": (P, [P]), "fg2_batch_member": (P, [P, I]),
        "fg2_batch_set_box": (I, [P, D, D]), "fg2_batch_set_courant": (I, [P, D]),
        "fg2_batch_set_bcond": (I, [P, I, I]), "fg2_batch_para": (S, [P, S]), "fg2_batch_config": (I, [P]),
        "fg2_batch_set_time": (I, [P, D]), "fg2_batch_advance": (I, [P, I, D, D, I]),
        "fg2_batch_sync": (I, [P]), "fg2_batch_set_tiling": (I, [P, I, I]),
        "fg2_batch_get_tiling": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "fg2_batch_set_strip": (I, [P, I]), "fg2_batch_get_strip": (I, [P]),
        "fg2_batch_autotune": (I, [P, I, ctypes.POINTER(D)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def load_library(scheme="hydro"):
    """The C-ABI library of `scheme` ('hydro' or 'hydro-isot'); raises when it is absent."""
    if scheme == "isot":
        scheme = "hydro-isot"
    if scheme not in SCHEMES:
        raise ValueError(f"unknown scheme {scheme!r}; available: {SCHEMES}")
    if scheme not in _LIBS:
        path = lib_path(scheme)
        if not os.path.exists(path):
            raise FG2Error(f"{path} is not built (python -m fg2_b200.build); there is no CPU fallback")
        _LIBS[scheme] = _bind(ctypes.CDLL(path))
    return _LIBS[scheme]


def setup_evaluate(name, n1, n2, scheme="hydro", l1=1.0, l2=1.0, para=None, seed=0, storage="f64"):
    """Evaluate an initial condition on the host: (n1, n2, NVAR) float64 array (no GPU).
    storage: the precision of the state it is for; with "f32" (or a 16-bit storage) the
    reference's named setups compute in float, as the reference does with R = float, which is
    what Sim.init uses for such states."""
    lib = load_library(scheme)
    nv = lib.fg2_nvar()
    out = np.empty((n1, n2, nv), np.float64)
    pa = None
    if para is not None:
        keys = [lib.fg2_para_key(k).decode() for k in range(lib.fg2_para_count())]
        pa = np.array([para[k] for k in keys], np.float64)
    rc = lib.fg2_setup_evaluate(name.encode(), n1, n2, l1, l2, None if pa is None else pa.ctypes.data,
                                int(seed), STORAGE[storage], out.ctypes.data)
    if rc < 0:
        raise FG2Error(lib.fg2_last_error().decode())
    return out, bool(rc)


def tile_bands(n1, nb=0, tail=0, reverse=False, scheme="hydro"):
    """The row bands (i0, iend, blocks) the fused kernel cuts a grid of n1 rows into, in the
    order a launch takes them (host only, no GPU)."""
    lib = load_library(scheme)
    n = lib.fg2_tile_bands(int(n1), int(nb), int(tail), int(reverse), None, 0)
    if n < 0:
        raise FG2Error("bad tile band arguments")
    out = (ctypes.c_int * (3 * max(n, 1)))()
    lib.fg2_tile_bands(int(n1), int(nb), int(tail), int(reverse), out, n)
    return [tuple(out[3 * q:3 * q + 3]) for q in range(n)]


class Sim:
    """One simulation on the current CUDA device (the handle API, fg2_sim_*)."""

    def __init__(self, n1, n2, scheme="hydro", storage="f32", stream=None, _member=None):
        self.lib = load_library(scheme)
        self.scheme = self.lib.fg2_scheme_name().decode()
        self.n1, self.n2 = int(n1), int(n2)
        self.storage = storage
        self.nvar = self.lib.fg2_nvar()
        self.host_dtype = np.float64 if storage == "f64" else np.float32
        self._owner = _member is None
        h = self.lib.fg2_sim_create(self.n1, self.n2, STORAGE[storage], stream) if self._owner else _member
        if not h:
            raise FG2Error(self.lib.fg2_last_error().decode())
        self.h = ctypes.c_void_p(h)

    def close(self):
        if getattr(self, "h", None):
            if self._owner:
                self.lib.fg2_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc < 0 or rc > 1:
            raise FG2Error(f"{what}: status {rc}: {self.lib.fg2_last_error().decode()}")
        return rc

    # ---- configuration -----------------------------------------------------------
    @property
    def fields(self):
        return [self.lib.fg2_field_name(f).decode() for f in range(self.nvar)]

    def para(self, keyval):
        r = self.lib.fg2_sim_para(self.h, keyval.encode())
        return None if r is None else r.decode()

    def get_para(self, key):
        v = ctypes.c_double()
        self._check(self.lib.fg2_sim_get_para(self.h, key.encode(), ctypes.byref(v)), "get_para")
        return v.value

    def set_box(self, l1, l2):
        self._check(self.lib.fg2_sim_set_box(self.h, l1, l2), "set_box")

    def set_courant(self, c):
        self._check(self.lib.fg2_sim_set_courant(self.h, c), "set_courant")

    def set_tiling(self, nb, ctas_per_sm=None, tail=None):
        """Tile height of the fused kernel in blocks of 7 rows (0: the default) and, if given,
        CTAs per SM of its persistent grid (0: as many as fit) and the number of one-block
        tail bands that end the grid (0: none)."""
        self._check(self.lib.fg2_sim_set_tiling(self.h, int(nb)), "set_tiling")
        if ctas_per_sm is not None:
            self._check(self.lib.fg2_sim_set_occupancy(self.h, int(ctas_per_sm)), "set_occupancy")
        if tail is not None:
            self._check(self.lib.fg2_sim_set_tail(self.h, int(tail)), "set_tail")

    def tiling(self):
        """(tile height in blocks of 7 rows, CTAs per SM, tail bands) the launches use."""
        nb, c, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fg2_sim_get_tiling(self.h, ctypes.byref(nb), ctypes.byref(c)), "tiling")
        self._check(self.lib.fg2_sim_get_tail(self.h, ctypes.byref(t)), "tiling")
        return nb.value, c.value, t.value

    def autotune(self, reps=3):
        """Time every tiling candidate on this simulation's state (left unchanged) and keep the
        fastest; returns its ms per step."""
        ms = ctypes.c_double()
        self._check(self.lib.fg2_sim_autotune(self.h, int(reps), ctypes.byref(ms)), "autotune")
        return ms.value

    def set_bcond(self, p1, p2):
        self._check(self.lib.fg2_sim_set_bcond(self.h, int(p1), int(p2)), "set_bcond")

    def config(self):
        self._check(self.lib.fg2_sim_config(self.h), "config")

    def set_dt_mode(self, mode):
        mode = {"reference": DT_REFERENCE, "cfl": DT_CFL}.get(mode, mode)
        self._check(self.lib.fg2_sim_set_dt_mode(self.h, int(mode)), "set_dt_mode")

    @property
    def device_bytes(self):
        return self.lib.fg2_sim_device_bytes(self.h)

    def layout(self):
        p, s = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.fg2_sim_layout(self.h, ctypes.byref(p), ctypes.byref(s)), "layout")
        return p.value, s.value

    # ---- state -------------------------------------------------------------------
    def init(self, name, seed=0):
        self._check(self.lib.fg2_sim_init(self.h, name.encode(), int(seed)), "init")

    def _host(self, a):
        a = np.ascontiguousarray(a, dtype=self.host_dtype)
        if a.shape != (self.n1, self.n2, self.nvar):
            raise ValueError(f"expected shape {(self.n1, self.n2, self.nvar)}, got {a.shape}")
        return a

    def upload(self, state):
        a = self._host(state)
        self._check(self.lib.fg2_sim_upload(self.h, a.ctypes.data), "upload")

    def download(self, out=None):
        out = np.empty((self.n1, self.n2, self.nvar), self.host_dtype) if out is None else out
        self._check(self.lib.fg2_sim_download(self.h, out.ctypes.data), "download")
        return out

    def upload_v(self, v):
        a = self._host(v)
        self._check(self.lib.fg2_sim_upload_v(self.h, a.ctypes.data), "upload_v")

    def download_v(self):
        out = np.empty((self.n1, self.n2, self.nvar), self.host_dtype)
        self._check(self.lib.fg2_sim_download_v(self.h, out.ctypes.data), "download_v")
        return out

    # ---- time step ----------------------------------------------------------------
    def getdt(self):
        return self.lib.fg2_sim_getdt(self.h)

    def step(self, t, dt):
        return self._check(self.lib.fg2_sim_step(self.h, float(t), float(dt)), "step")

    def advance(self, nsteps, dt=0.0, t_end=float("inf"), graph=False):
        f = self.lib.fg2_sim_advance_graph if graph else self.lib.fg2_sim_advance
        self._check(f(self.h, int(nsteps), float(dt), float(t_end)), "advance")

    def stage(self, k, dt):
        self._check(self.lib.fg2_sim_stage(self.h, int(k), float(dt)), "stage")

    def sync(self):
        return self._check(self.lib.fg2_sim_sync(self.h), "sync")

    def set_time(self, t):
        self._check(self.lib.fg2_sim_set_time(self.h, float(t)), "set_time")

    def time(self):
        return self.lib.fg2_sim_time(self.h)

    def last_dt(self):
        return self.lib.fg2_sim_last_dt(self.h)

    def clear_status(self):
        self.lib.fg2_sim_clear_status(self.h)

    def test_stall_waits(self, nbytes):
        """Tests of the timeout path: every data chunk of the substage kernel then waits for
        `nbytes` more than its copies deliver, so its bounded waits run out (0 restores)."""
        self._check(self.lib.fg2_sim_test_stall_waits(self.h, int(nbytes)), "test_stall_waits")

    def kick(self, t, beta):
        self._check(self.lib.fg2_sim_kick(self.h, float(t), float(beta)), "kick")

    def drift(self, dt):
        return self._check(self.lib.fg2_sim_drift(self.h, float(dt)), "drift")

    def bcond(self):
        self._check(self.lib.fg2_sim_bcond(self.h), "bcond")

    def euler(self, dt):
        self._check(self.lib.fg2_sim_euler(self.h, float(dt)), "euler")

    def set_forcing_phases(self, r1, r2):
        self._check(self.lib.fg2_sim_set_forcing_phases(self.h, float(r1), float(r2)), "set_forcing_phases")

    def sums(self):
        out = np.zeros(4, np.float64)
        self._check(self.lib.fg2_sim_sums(self.h, out.ctypes.data), "sums")
        return out

    @property
    def stream(self):
        return self.lib.fg2_sim_stream(self.h)

    # ---- frames -------------------------------------------------------------------
    def dump(self, path, time):
        self._check(self.lib.fg2_sim_dump(self.h, str(path).encode(), float(time)), "dump")

    def solve(self, t, t_final, i, n, directory):
        """The reference's frame loop: frames i+1 .. n up to t_final, dumped as
        directory/%04d.raw.  Returns (status, ms per step)."""
        ms = ctypes.c_double()
        rc = self.lib.fg2_sim_solve(self.h, float(t), float(t_final), int(i), int(n), str(directory).encode(),
                                    ctypes.byref(ms))
        return self._check(rc, "solve"), ms.value

    def load(self, path):
        t = ctypes.c_double()
        self._check(self.lib.fg2_sim_load(self.h, str(path).encode(), ctypes.byref(t)), "load")
        return t.value


class Batch:
    """Independent simulations of one scheme advanced together (the batch API, fg2_batch_*).

    `sizes` is a list of (n1, n2).  `members[k]` is a Sim view of member k (owned by the batch)
    for init, upload/download, sums, time and per-member status."""

    def __init__(self, sizes, scheme="hydro-isot", storage="f32", stream=None):
        self.lib = load_library(scheme)
        sizes = [(int(a), int(b)) for a, b in sizes]
        n = len(sizes)
        n1 = (ctypes.c_int * n)(*[a for a, _ in sizes])
        n2 = (ctypes.c_int * n)(*[b for _, b in sizes])
        h = self.lib.fg2_batch_create(n, ctypes.cast(n1, ctypes.c_void_p), ctypes.cast(n2, ctypes.c_void_p),
                                      STORAGE[storage], stream)
        if not h:
            raise FG2Error(self.lib.fg2_last_error().decode())
        self.h = ctypes.c_void_p(h)
        self.sizes = sizes
        self.members = [Sim(a, b, scheme, storage, _member=self.lib.fg2_batch_member(self.h, k))
                        for k, (a, b) in enumerate(sizes)]

    def close(self):
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None
            self.lib.fg2_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc < 0 or rc > 1:
            raise FG2Error(f"{what}: status {rc}: {self.lib.fg2_last_error().decode()}")
        return rc

    def __len__(self):
        return len(self.members)

    @property
    def cells(self):
        return self.lib.fg2_batch_cells(self.h)

    @property
    def device_bytes(self):
        return self.lib.fg2_batch_device_bytes(self.h)

    @property
    def stream(self):
        return self.lib.fg2_batch_stream(self.h)

    def para(self, keyval):
        r = self.lib.fg2_batch_para(self.h, keyval.encode())
        return None if r is None else r.decode()

    def set_box(self, l1, l2):
        self._check(self.lib.fg2_batch_set_box(self.h, l1, l2), "set_box")

    def set_courant(self, c):
        self._check(self.lib.fg2_batch_set_courant(self.h, c), "set_courant")

    def set_bcond(self, p1, p2):
        self._check(self.lib.fg2_batch_set_bcond(self.h, int(p1), int(p2)), "set_bcond")

    def config(self):
        self._check(self.lib.fg2_batch_config(self.h), "config")

    def set_time(self, t):
        self._check(self.lib.fg2_batch_set_time(self.h, float(t)), "set_time")

    def advance(self, nsteps, dt=0.0, t_end=float("inf"), graph=True):
        """nsteps RK3 steps of every member (dt <= 0: per-member device-resident CFL steps)."""
        return self._check(self.lib.fg2_batch_advance(self.h, int(nsteps), float(dt), float(t_end), int(bool(graph))),
                           "advance")

    def sync(self):
        return self.lib.fg2_batch_sync(self.h)

    def set_tiling(self, nb, ctas_per_sm=0):
        self._check(self.lib.fg2_batch_set_tiling(self.h, int(nb), int(ctas_per_sm)), "set_tiling")

    def tiling(self):
        nb, c = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fg2_batch_get_tiling(self.h, ctypes.byref(nb), ctypes.byref(c)), "tiling")
        return nb.value, c.value

    def set_strip(self, width):
        """Strip width of the batch launches: 64 or 128 columns per tile (2 or 4 warps per CTA)."""
        self._check(self.lib.fg2_batch_set_strip(self.h, int(width)), "set_strip")

    def strip(self):
        return self.lib.fg2_batch_get_strip(self.h)

    def autotune(self, reps=3):
        ms = ctypes.c_double()
        self._check(self.lib.fg2_batch_autotune(self.h, int(reps), ctypes.byref(ms)), "autotune")
        return ms.value


def shard_members(sizes, world):
    """Split a batch's members over `world` ranks by cell count: members in descending cell
    count (ties by index) each go to the rank holding the fewest cells so far (lowest rank on a
    tie).  Returns, per rank, the sorted member indices it owns.  Members are independent, so
    the ranks step their shards with no exchange; the heaviest rank holds at most the mean plus
    one member.  The reference runs one simulation on one device and has no multi-device path."""
    world = int(world)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    shards = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda k: (-sizes[k][0] * sizes[k][1], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        shards[r].append(k)
        load[r] += sizes[k][0] * sizes[k][1]
    return [sorted(s) for s in shards]

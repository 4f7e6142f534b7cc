"""Command-line driver with the reference's argument semantics (src/main.cpp:27-116).

    python -m fg2_b200.cli SCHEME [options] [key=val ...] [INPUT]

SCHEME picks the library, as the reference builds one binary per scheme directory
(Makefile:19-22): hydro, hydro-isot or disk.  The rest follows src/main.cpp:

  -n n0 [n1 [n2]]   frames to write (default 10), then the grid (default 1024 x 1024; one
                    number sets both sides)
  -l l0 [l1 [l2]]   simulated time (default 1), then the box (one number sets both sides)
  -b p1 [p2]        boundaries per axis: a value starting with p/P is periodic, anything else
                    the reference's non-periodic choice for that axis
  -c c              Courant number
  -d d              CUDA device
  key=val           scheme parameters, set after the grid exists (src/main.cpp:94-101)
  INPUT             a .raw frame to continue from (its frame number is the first number in
                    the name, src/misc.cpp:48-55), or else the name of an initial condition
                    (default "default"); a fresh start is dumped as frame 0

Frames i+1 .. i+n0 are written as %04d.raw in the working directory at equal time intervals
up to t + l0 (src/solve.cpp:25-64); a NaN stops the run and writes ****.raw.  An option given
without a value, or an unknown option, prints the usage and exits (src/usage.cpp).
"""
import os
import re
import sys

USAGE = __doc__

_FLOAT = re.compile(r"\s*[+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?)")
_INT = re.compile(r"\s*[+-]?\d+")


def atof(s):
    """C's atof: the longest leading number, 0 when there is none."""
    m = _FLOAT.match(s)
    return float(m.group(0)) if m else 0.0


def atoi(s):
    """C's atoi: the leading integer, 0 when there is none."""
    m = _INT.match(s)
    return int(m.group(0)) if m else 0


def _is_opt(a):
    """An option word: '-' followed by a letter (src/main.cpp:24)."""
    return len(a) > 1 and a[0] == "-" and a[1].isalpha()


def parse(argv):
    """The reference's parser (src/main.cpp:36-58) on argv (without the program and scheme):
    returns a dict of the settings, or raises SystemExit with the usage on a bad option.  As
    there, an option takes every following word up to its maximum count that is not itself an
    option ('-' and a letter), and converts it as atof / atoi do: give the input name and the
    key=val words before an option's values, not right after them."""
    cfg = {"input": "default", "n0": 10, "n1": 1024, "n2": 1024, "l0": 1.0, "l1": None, "l2": None,
           "p1": None, "p2": None, "c": None, "d": 0, "para": []}
    if "--help" in argv:
        raise SystemExit(USAGE)
    i = 0

    def noval(k):
        return k + 1 >= len(argv) or _is_opt(argv[k + 1])

    while i < len(argv):
        a = argv[i]
        if "=" in a:
            cfg["para"].append(a)
        elif not a.startswith("-"):
            cfg["input"] = a
        else:
            o = a[1:2]
            if o not in "bcdln" or o == "" or noval(i):
                raise SystemExit(f"unknown option or missing value: {a}\n\n{USAGE}")
            if o == "b":
                i += 1
                cfg["p1"] = argv[i][:1] in ("p", "P")
                if not noval(i):
                    i += 1
                    cfg["p2"] = argv[i][:1] in ("p", "P")
            elif o == "c":
                i += 1
                cfg["c"] = atof(argv[i])
            elif o == "d":
                i += 1
                cfg["d"] = atoi(argv[i])
            elif o == "l":
                i += 1
                cfg["l0"] = atof(argv[i])
                if not noval(i):
                    i += 1
                    cfg["l1"] = cfg["l2"] = atof(argv[i])
                    if not noval(i):
                        i += 1
                        cfg["l2"] = atof(argv[i])
            elif o == "n":
                i += 1
                cfg["n0"] = atoi(argv[i])
                if not noval(i):
                    i += 1
                    cfg["n1"] = cfg["n2"] = atoi(argv[i])
                    if not noval(i):
                        i += 1
                        cfg["n2"] = atoi(argv[i])
        i += 1
    return cfg


def frame_number(name):
    """The first number in the name as given (src/misc.cpp:48-55), 0 when there is none."""
    digits = ""
    for ch in name:
        if ch.isdigit():
            digits += ch
        elif digits:
            break
    return int(digits) if digits else 0


def run(scheme, argv, out=print):
    """Parse argv and run the reference's main(): returns the solve status (0, or 1 on NaN)."""
    import fg2_b200
    cfg = parse(argv)
    import torch
    torch.cuda.set_device(cfg["d"])
    out("2D finite grid code, B200 time step\n")
    n1, n2 = cfg["n1"], cfg["n2"]
    sim = fg2_b200.Sim(n1, n2, scheme=scheme)
    try:
        out(f"  Resolution   : {n1} x {n2} using {sim.device_bytes / 1048576.0:.3g}MiB of device memory")
        if cfg["p1"] is not None:  # an axis not given keeps the default, periodic (src/global.cpp:29)
            sim.set_bcond(int(cfg["p1"]), int(cfg["p2"]) if cfg["p2"] is not None else 1)
        if cfg["l1"] is not None:
            sim.set_box(cfg["l1"], cfg["l2"])
        if cfg["c"] is not None:
            sim.set_courant(cfg["c"])
        for kv in cfg["para"]:
            msg = sim.para(kv)
            out(f"  Parameter    : {msg}" if msg is not None else f'  Fail to set  : "{kv}"')
        inp = cfg["input"]
        if os.path.exists(inp):
            i = frame_number(inp)
            t = sim.load(inp)
            sim.config()
            out(f'  Input file   : "{inp}", start at frame {i}, time {t:g}')
        else:
            out(f'  Initialize   : "{inp}"')
            sim.config()
            sim.init(inp)
            i, t = 0, 0.0
            sim.dump(f"{i:04d}.raw", t)
        n0, l0 = cfg["n0"], cfg["l0"]
        out(f"  Time         : {l0:g} with {n0} frame{'s' if n0 > 1 else ''}")
        status, ms = sim.solve(t, t + l0, i, i + n0, ".")
        out(f"  {'Done' if status == 0 else 'Stopped on a NaN'} ({ms:.4g} ms per step)")
        return status
    finally:
        sim.close()


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] in ("--help", "-h"):
        print(USAGE)
        return 0
    return run(argv[0], argv[1:])


if __name__ == "__main__":
    sys.exit(main())

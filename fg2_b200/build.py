"""Build the per-scheme C-ABI libraries for sm_100a (nvcc, no GPU needed).

    python -m fg2_b200.build            # both schemes
    python -m fg2_b200.build hydro      # one scheme

Each scheme compiles the same sources with `-I csrc/schemes/<scheme>`, the way the
reference builds one binary per scheme directory (Makefile:19-22), into
fg2_b200/lib/libfg2_<scheme>.so.  Objects go to fg2_b200/_build/.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
SCHEMES = ("hydro", "hydro-isot", "disk")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"] + ARCH
SOURCES = ("kernels.cu", "noalloc.cu", "runtime.cpp", "batch.cpp")


def nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = os.path.join(cuda, "bin", "nvcc")
    return path if os.path.exists(path) else shutil.which("nvcc")


def lib_path(scheme):
    return os.path.join(LIB, f"libfg2_{scheme}.so")


def _headers(scheme):
    """Headers every source of `scheme` may include."""
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    sdir = os.path.join(CSRC, "schemes", scheme)
    out += [os.path.join(sdir, f) for f in os.listdir(sdir)]
    out.append(os.path.join(os.path.dirname(HERE), "include", "fg2_b200.h"))
    return out


def _deps():
    out = []
    for root, _, files in os.walk(CSRC):
        out += [os.path.join(root, f) for f in files]
    out.append(os.path.join(os.path.dirname(HERE), "include", "fg2_b200.h"))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _obj(scheme, src):
    return os.path.join(BUILD, scheme, src + ".o")


def _compile(scheme, src):
    obj = _obj(scheme, src)
    if not _stale(obj, [os.path.join(CSRC, src)] + _headers(scheme)):
        return obj  # up to date
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, "-I", CSRC, "-I", os.path.join(CSRC, "schemes", scheme),
           "-x", "cu" if src.endswith(".cu") else "c++", "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {scheme}/{src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(schemes=SCHEMES, force=False, jobs=4):
    deps = _deps()
    todo = [s for s in schemes if force or _stale(lib_path(s), deps)]
    if not todo:
        return [lib_path(s) for s in schemes]
    os.makedirs(LIB, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {(s, src): ex.submit(_compile, s, src) for s in todo for src in SOURCES}
        objs = {k: f.result() for k, f in futs.items()}
    for s in todo:
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib_path(s), *[objs[(s, src)] for src in SOURCES]]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed for {s}:\n{r.stdout}\n{r.stderr}")
    return [lib_path(s) for s in schemes]


if __name__ == "__main__":
    names = [a for a in sys.argv[1:] if not a.startswith("-")] or list(SCHEMES)
    for p in build(names, force="--force" in sys.argv):
        print(p)

"""Initial conditions of the benchmark workloads in numpy -- TEST INFRASTRUCTURE ONLY.

The `--impl reference` arm of bench.py builds its input with these, so the process that
times the reference's CPU arithmetic maps nothing of the product (fg2_b200's libraries).
Each function restates, in vectorised numpy, a setup of the library's scheme directory:

  kh     fg2_b200/csrc/schemes/hydro/init.h  (KHTanh: tanh shear layer, rho 1 inside / 2
         outside, p = 2.5, u2 = 0.01 sin(4 pi x) + N(0, 1e-4^2))
  noise  fg2_b200/csrc/schemes/hydro/init.h  (Noise: rho = 1, p = 1/gamma, u ~ N(0, sigma^2))

and the seeded generator of fg2_b200/csrc/setup_common.h (splitmix64, uniform in (0, 1],
Box-Muller pairs: the first deviate of a pair is r cos t, the second r sin t).  Cells draw in
row-major order.  numpy's transcendental functions may differ from the C library's in the
last bit of a double; after the cast to the state's FP32 the two agree to 1 ulp (tested).
"""
import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix_uniform(seed, count, start=0):
    """Uniform deviates number start .. start+count-1 of the generator seeded with `seed`:
    the k-th call advances the state by the golden gamma and mixes it (setup_common.h Rng)."""
    k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normals(seed, count):
    """The first `count` normal deviates of the generator: Box-Muller pairs in draw order."""
    npair = (count + 1) // 2
    u = splitmix_uniform(seed, 2 * npair)
    r = np.sqrt(-2.0 * np.log(u[0::2]))
    t = 6.283185307179586476925 * u[1::2]
    out = np.empty(2 * npair)
    out[0::2] = r * np.cos(t)
    out[1::2] = r * np.sin(t)
    return out[:count]


def kh(n1, n2, seed=2, l1=1.0, l2=1.0, gamma=5.0 / 3.0, w=0.01):
    """tanh Kelvin-Helmholtz layer: (n1, n2, 4) float64 cells (lnd, u1, u2, lne) at cell
    centres x = l1 (i + 1/2) / n1 (axis 1), y = l2 (j + 1/2) / n2 (axis 2)."""
    x = l1 * (np.arange(n1) + 0.5) / n1
    y = l2 * (np.arange(n2) + 0.5) / n2
    s = np.tanh((np.abs(y / l2 - 0.5) - 0.25) / w)
    rho = 1.5 + 0.5 * s
    q = np.empty((n1, n2, 4))
    q[:, :, 0] = np.log(rho)[None, :]
    q[:, :, 1] = (0.5 * s)[None, :]
    q[:, :, 2] = (0.01 * np.sin(4.0 * 3.14159265358979323846 * x / l1))[:, None] + \
        1e-4 * normals(seed, n1 * n2).reshape(n1, n2)
    q[:, :, 3] = np.log(2.5 / (rho * (gamma - 1.0)))[None, :]
    return q


def noise(n1, n2, seed=1, sigma=0.01, gamma=5.0 / 3.0):
    """rho = 1, p = 1/gamma, u1 and u2 i.i.d. N(0, sigma^2), drawn u1 then u2 per cell."""
    g = normals(seed, 2 * n1 * n2).reshape(n1, n2, 2)
    q = np.empty((n1, n2, 4))
    q[:, :, 0] = 0.0
    q[:, :, 1] = sigma * g[:, :, 0]
    q[:, :, 2] = sigma * g[:, :, 1]
    q[:, :, 3] = np.log(1.0 / (gamma * (gamma - 1.0)))
    return q

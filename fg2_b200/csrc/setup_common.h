// fg2_b200/csrc/setup_common.h -- host helpers for initial conditions: a portable seeded
// generator (splitmix64 + Box-Muller), the option parser of setup names
// ("name:key=val,key=val"), and the band-limited random-phase velocity field.
//
// The reference evaluates a setup function at cell centres x = l1 (i + 1/2) / n1,
// y = l2 (j + 1/2) / n2 in row order on the host (src/init.cpp:26-42) and draws its noise
// from rand(); here every seeded setup draws from splitmix64 in the same row order, so a
// (setup, seed, n1, n2) triple fixes the initial state on any machine.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace fg2 {

// splitmix64 (S. Vigna's public-domain generator) and Box-Muller normal deviates.
struct Rng {
  uint64_t s;
  bool have = false;
  double spare = 0;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next()
  {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform in (0, 1]
  double uniform() { return (double)((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
  double normal()
  {
    if (have) { have = false; return spare; }
    const double r = std::sqrt(-2.0 * std::log(uniform()));
    const double t = 6.283185307179586476925 * uniform();
    spare = r * std::sin(t);
    have = true;
    return r * std::cos(t);
  }
};

// Options of a setup name: "turb:mach=0.3,kmin=2" -> base "turb", opt("mach", d).
struct SetupName {
  std::string base;
  std::vector<std::pair<std::string, double>> kv;
  explicit SetupName(const char *name)
  {
    const char *c = std::strchr(name, ':');
    base = c ? std::string(name, c - name) : std::string(name);
    while (c && *c) {
      const char *k = c + 1;
      const char *e = std::strchr(k, '=');
      if (!e) break;
      const char *n = std::strchr(e, ',');
      kv.emplace_back(std::string(k, e - k), std::atof(e + 1));
      c = n;
    }
  }
  double opt(const char *key, double def) const
  {
    for (auto &p : kv)
      if (p.first == key) return p.second;
    return def;
  }
};

struct SetupCtx {
  int n1, n2;
  double l1, l2;
  const double *para;  // the scheme's parameter values by slot
  uint64_t seed;
  bool single = false;  // the state is FP32 (or 16-bit): the reference's setups compute in float
};

// Interface of one initial condition: fills row i (n2 cells x NVAR values, cell-interleaved,
// no ghosts) in double; rows are requested in order 0 .. n1-1.
struct Setup {
  virtual ~Setup() {}
  virtual void row(int i, double *out) = 0;
};

// Solenoidal random-phase velocity field on a periodic box, with integer wave vectors
// (kx, ky) in units of 2 pi / L and kmin <= |k| <= kmax.  A shell-integrated spectrum
// E(k) ~ k^-slope over a 2D shell holding ~k modes gives a mode amplitude ~ k^-(slope+1)/2.
// Each mode is a plane wave with direction (-ky, kx) / |k| (divergence free) and a uniform
// random phase; the field is scaled to the requested rms |u|.  Evaluated separably:
// u(x_i, y_j) = Re sum_kx e^{i kx x_i} [sum_ky c(kx, ky) e^{i ky y_j}].
struct RandomVelocity {
  int n1, n2, kmax;
  std::vector<double> g1re, g1im, g2re, g2im;  // [kx index][j] inner sums per component
  std::vector<double> ex_re, ex_im;            // scratch per row
  double scale = 1.0;

  RandomVelocity(int n1_, int n2_, double kmin, double kmax_, double slope, double rms, Rng &rng)
      : n1(n1_), n2(n2_), kmax((int)kmax_)
  {
    const int K = kmax;
    const int nkx = 2 * K + 1;
    // complex mode coefficients of u1 and u2, half plane kx > 0 or (kx == 0, ky > 0)
    std::vector<double> c1re(nkx * nkx, 0), c1im(nkx * nkx, 0), c2re(nkx * nkx, 0), c2im(nkx * nkx, 0);
    for (int kx = -K; kx <= K; ++kx)
      for (int ky = -K; ky <= K; ++ky) {
        if (kx < 0 || (kx == 0 && ky <= 0)) continue;
        const double k = std::sqrt((double)kx * kx + (double)ky * ky);
        if (k < kmin || k > kmax_) continue;
        const double a = std::pow(k, -(slope + 1.0) / 2.0);
        const double ph = 6.283185307179586476925 * rng.uniform();
        const int idx = (kx + K) * nkx + (ky + K);
        const double e1 = -ky / k, e2 = kx / k;
        c1re[idx] = a * e1 * std::cos(ph); c1im[idx] = a * e1 * std::sin(ph);
        c2re[idx] = a * e2 * std::cos(ph); c2im[idx] = a * e2 * std::sin(ph);
      }
    // inner sums over ky for every kx and column j
    g1re.assign((size_t)nkx * n2, 0); g1im.assign((size_t)nkx * n2, 0);
    g2re.assign((size_t)nkx * n2, 0); g2im.assign((size_t)nkx * n2, 0);
    for (int kx = -K; kx <= K; ++kx)
      for (int ky = -K; ky <= K; ++ky) {
        const int idx = (kx + K) * nkx + (ky + K);
        if (c1re[idx] == 0 && c1im[idx] == 0 && c2re[idx] == 0 && c2im[idx] == 0) continue;
        for (int j = 0; j < n2; ++j) {
          const double th = 6.283185307179586476925 * ky * (j + 0.5) / n2;
          const double cr = std::cos(th), ci = std::sin(th);
          const size_t o = (size_t)(kx + K) * n2 + j;
          g1re[o] += c1re[idx] * cr - c1im[idx] * ci; g1im[o] += c1re[idx] * ci + c1im[idx] * cr;
          g2re[o] += c2re[idx] * cr - c2im[idx] * ci; g2im[o] += c2re[idx] * ci + c2im[idx] * cr;
        }
      }
    // rms of the unscaled field: each mode contributes a^2 / 2 to <|u|^2>
    double ms = 0;
    for (int i = 0; i < nkx * nkx; ++i)
      ms += 0.5 * (c1re[i] * c1re[i] + c1im[i] * c1im[i] + c2re[i] * c2re[i] + c2im[i] * c2im[i]);
    scale = ms > 0 ? rms / std::sqrt(ms) : 0.0;
    ex_re.resize(nkx); ex_im.resize(nkx);
  }

  // u1, u2 along row i (stride `stride` doubles between cells, fields at +f1, +f2)
  void row(int i, double *out, int stride, int f1, int f2)
  {
    const int K = kmax, nkx = 2 * K + 1;
    for (int kx = -K; kx <= K; ++kx) {
      const double th = 6.283185307179586476925 * kx * (i + 0.5) / n1;
      ex_re[kx + K] = std::cos(th); ex_im[kx + K] = std::sin(th);
    }
    for (int j = 0; j < n2; ++j) {
      double a1 = 0, a2 = 0;
      for (int q = 0; q < nkx; ++q) {
        const size_t o = (size_t)q * n2 + j;
        a1 += ex_re[q] * g1re[o] - ex_im[q] * g1im[o];
        a2 += ex_re[q] * g2re[o] - ex_im[q] * g2im[o];
      }
      out[j * stride + f1] = scale * a1;
      out[j * stride + f2] = scale * a2;
    }
  }
};

}  // namespace fg2

// nbr_ic.cpp -- deterministic initial conditions (host code).
//
// The reference's initialisers (CPU/nbody_system.cpp:238-384) are a ring with
// a central mass and an unseeded random box (std::random_device,
// :242-243), so its runs are not reproducible.  Every sampler here draws from
// one documented generator -- xoshiro256** (Blackman & Vigna) whose state is
// filled by splitmix64 from the seed -- and maps 53 random bits to a double,
// so a seed gives the same bits on every host and in every process.
#include "nbr.h"

#include <cmath>
#include <cstdint>
#include <cstddef>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t z = seed;
    for (auto& w : s) w = splitmix64(z);
  }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return double(next() >> 11) * 0x1.0p-53; }          // [0, 1)
  double uniform_pos() { return double((next() >> 11) + 1) * 0x1.0p-53; }  // (0, 1]
};

// Isotropic vector of length r from two uniforms.
inline void isotropic(Rng& g, double r, double& x, double& y, double& z) {
  const double c = 1.0 - 2.0 * g.uniform();
  const double ph = 2.0 * kPi * g.uniform();
  const double s = std::sqrt(std::fmax(0.0, 1.0 - c * c));
  x = r * s * std::cos(ph);
  y = r * s * std::sin(ph);
  z = r * c;
}

void recentre(size_t n, double* a, double* b, double* c, const double* m) {
  long double sa = 0, sb = 0, sc = 0, sm = 0;
  for (size_t i = 0; i < n; ++i) {
    sa += (long double)m[i] * a[i]; sb += (long double)m[i] * b[i]; sc += (long double)m[i] * c[i];
    sm += m[i];
  }
  if (sm <= 0) return;
  const double ma = double(sa / sm), mb = double(sb / sm), mc = double(sc / sm);
  for (size_t i = 0; i < n; ++i) { a[i] -= ma; b[i] -= mb; c[i] -= mc; }
}

// Plummer sphere in N-body units (G = M = 1, E = -1/4, scale radius
// a = 3 pi / 16), after Aarseth, Henon & Wielen (1974, A&A 37, 183):
//   r = a / sqrt(X^{-2/3} - 1), X the enclosed mass fraction (<= 0.999);
//   speed v = q v_esc(r), v_esc = sqrt(2 / a) (1 + r^2/a^2)^{-1/4}, with q
//   drawn by von Neumann rejection from g(q) = q^2 (1 - q^2)^{7/2}
//   (max 0.092 < 0.1);  directions isotropic.
void plummer(size_t n, uint64_t seed, double* x, double* y, double* z, double* vx, double* vy,
             double* vz) {
  Rng g(seed);
  const double a = 3.0 * kPi / 16.0;
  const double vscale = std::sqrt(2.0 / a);
  for (size_t i = 0; i < n; ++i) {
    const double X = 0.999 * g.uniform_pos();
    const double r = a / std::sqrt(std::pow(X, -2.0 / 3.0) - 1.0);
    isotropic(g, r, x[i], y[i], z[i]);
    double q, h;
    do {
      q = g.uniform();
      h = 0.1 * g.uniform();
    } while (h > q * q * std::pow(1.0 - q * q, 3.5));
    const double v = q * vscale * std::pow(1.0 + r * r / (a * a), -0.25);
    isotropic(g, v, vx[i], vy[i], vz[i]);
  }
}

bool any_null(std::initializer_list<const void*> ps) {
  for (auto p : ps)
    if (!p) return true;
  return false;
}

}  // namespace

extern "C" {

int nbr_ic_plummer(size_t n, uint64_t seed, double* x, double* y, double* z, double* vx,
                   double* vy, double* vz, double* m) {
  if (n == 0 || any_null({x, y, z, vx, vy, vz, m})) return NBR_ERR_INVALID_ARG;
  plummer(n, seed, x, y, z, vx, vy, vz);
  for (size_t i = 0; i < n; ++i) m[i] = 1.0 / double(n);
  recentre(n, x, y, z, m);
  recentre(n, vx, vy, vz, m);
  return NBR_OK;
}

int nbr_ic_uniform_ball(size_t n, uint64_t seed, double* x, double* y, double* z, double* vx,
                        double* vy, double* vz, double* m) {
  if (n == 0 || any_null({x, y, z, vx, vy, vz, m})) return NBR_ERR_INVALID_ARG;
  Rng g(seed);
  for (size_t i = 0; i < n; ++i) {
    double a, b, c;
    do {
      a = 2.0 * g.uniform() - 1.0;
      b = 2.0 * g.uniform() - 1.0;
      c = 2.0 * g.uniform() - 1.0;
    } while (a * a + b * b + c * c > 1.0);
    x[i] = a; y[i] = b; z[i] = c;
    vx[i] = vy[i] = vz[i] = 0.0;
    m[i] = 1.0 / double(n);
  }
  return NBR_OK;
}

int nbr_ic_two_component(size_t n, size_t n_heavy, double ratio, uint64_t seed, double* x,
                         double* y, double* z, double* vx, double* vy, double* vz, double* m) {
  if (n == 0 || n_heavy > n || !(ratio > 0.0) || any_null({x, y, z, vx, vy, vz, m}))
    return NBR_ERR_INVALID_ARG;
  plummer(n, seed, x, y, z, vx, vy, vz);
  const double ml = 1.0 / (double(n - n_heavy) + ratio * double(n_heavy));
  for (size_t i = 0; i < n; ++i) m[i] = i < n_heavy ? ratio * ml : ml;
  recentre(n, x, y, z, m);
  recentre(n, vx, vy, vz, m);
  return NBR_OK;
}

// The reference's ring initial condition (init_stable_orbiting_particles,
// CPU/nbody_system.cpp:319-384): the ring mass follows from requiring the
// summed pull of the other ring particles plus the central mass to equal the
// centripetal force m R omega^2 (G = 1).
int nbr_ic_ring(size_t n, double R, double omega, double ratio, double* x, double* y, double* z,
                double* vx, double* vy, double* vz, double* m, double* fx, double* fy,
                double* fz) {
  if (n < 2 || any_null({x, y, z, vx, vy, vz, m})) return NBR_ERR_INVALID_ARG;
  const size_t r = n - 1;
  double sum = 0.0;
  for (size_t i = 1; i <= (r - 1) / 2; ++i)
    sum += (2.0 + 2.0 * std::cos((kPi * double(r - 2 * i)) / double(r))) /
           std::pow(2.0 - 2.0 * std::cos(double(i) * 2.0 * kPi / double(r)), 1.5);
  if (r % 2 == 0) sum += 0.25;
  sum += ratio;
  const double mr = R * R * R * omega * omega / sum;
  for (size_t i = 0; i < r; ++i) {
    const double th = double(i) * 2.0 * kPi / double(r);
    m[i] = mr;
    x[i] = R * std::cos(th); y[i] = R * std::sin(th); z[i] = 0.0;
    vx[i] = -R * omega * std::sin(th); vy[i] = R * omega * std::cos(th); vz[i] = 0.0;
    if (fx) fx[i] = -mr * R * omega * omega * std::cos(th);
    if (fy) fy[i] = -mr * R * omega * omega * std::sin(th);
    if (fz) fz[i] = 0.0;
  }
  m[r] = ratio * mr;
  x[r] = y[r] = z[r] = vx[r] = vy[r] = vz[r] = 0.0;
  if (fx) fx[r] = 0.0;
  if (fy) fy[r] = 0.0;
  if (fz) fz[r] = 0.0;
  return NBR_OK;
}

int nbr_ic_ring_predict(size_t n, double R, double omega, size_t step, size_t steps_per_rev,
                        double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  if (n < 2 || steps_per_rev == 0 || any_null({x, y, z, vx, vy, vz})) return NBR_ERR_INVALID_ARG;
  const size_t r = n - 1;
  const double off = double(step) / double(steps_per_rev);
  for (size_t i = 0; i < r; ++i) {
    const double th = (double(i) / double(r) + off) * 2.0 * kPi;
    x[i] = R * std::cos(th); y[i] = R * std::sin(th); z[i] = 0.0;
    vx[i] = -R * omega * std::sin(th); vy[i] = R * omega * std::cos(th); vz[i] = 0.0;
  }
  x[r] = y[r] = z[r] = vx[r] = vy[r] = vz[r] = 0.0;
  return NBR_OK;
}

int nbr_ic_batch_sizes(size_t nsys, uint64_t seed, size_t nmin, size_t nmax, size_t* sizes) {
  if (!sizes || nmin == 0 || nmax < nmin) return NBR_ERR_INVALID_ARG;
  Rng g(seed);
  const double l0 = std::log(double(nmin)), l1 = std::log(double(nmax));
  for (size_t s = 0; s < nsys; ++s) {
    const double v = std::floor(std::exp(l0 + g.uniform() * (l1 - l0)));
    size_t k = size_t(v);
    if (k < nmin) k = nmin;
    if (k > nmax) k = nmax;
    sizes[s] = k;
  }
  return NBR_OK;
}

uint64_t nbr_ic_system_seed(uint64_t seed, size_t s) {
  uint64_t z = seed ^ (0xD1B54A32D192ED03ull * (uint64_t(s) + 1));
  return splitmix64(z);
}

}  // extern "C"

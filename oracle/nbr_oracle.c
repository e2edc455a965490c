/* nbr_oracle.c -- CPU oracle for the all-pairs softened gravity path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke check and bench.py's CPU
 * baseline may load the library built from this file, and only as the checker
 * or the timed CPU baseline.  The product (libnbr.so) never links or calls it.
 *
 * This is a plain-C restatement of the reference's CPU path with the two
 * extensions the GPU solver needs:
 *   - Plummer softening: r^2 -> r^2 + eps^2 (the reference has none,
 *     CPU/force_calculation.cpp:75-82);
 *   - acceleration form a_i = G sum_j m_j (x_j - x_i) / (r^2+eps^2)^{3/2}
 *     instead of the force m_i a_i (the reference divides by the mass inside
 *     the kick, CPU/omp_solver.cpp:385-387).
 * It follows compute_forces_simple (CPU/force_calculation.cpp:34-107) pair by
 * pair -- difference, sqrt, divide by dist^3, skip q == k -- but without the
 * Newton-3 half-triangle, so every ordered pair is evaluated and the j sum runs
 * in index order.  At eps = 0 it reproduces the reference's forces divided by
 * the receiver's mass; tests/test_oracle.py pins it against the reference built
 * from source (oracle/_ref) and against the reference's analytic ring forces.
 *
 * Parity pin: the reference ships no golden vectors; its known-answer checks are
 * generated by formula (ring forces, CPU/nbody_system.cpp:319-384; rigid
 * rotation, :386-408).  Both are restated below and checked in the tests.
 */
#include <math.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

/* FP64 accelerations, summed over j in index order, skipping j == i
 * (CPU/force_calculation.cpp:62-86 with softening, no Newton-3). */
void orc_accel(size_t n, const double* x, const double* y, const double* z, const double* m,
               double G, double eps2, double* ax, double* ay, double* az) {
  long long N = (long long)n;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long i = 0; i < N; ++i) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (long long j = 0; j < N; ++j) {
      if (j == i) continue;
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      double dist = sqrt(dx * dx + dy * dy + dz * dz + eps2);
      double w = m[j] / (dist * dist * dist);
      sx += w * dx; sy += w * dy; sz += w * dz;
    }
    ax[i] = G * sx; ay[i] = G * sy; az[i] = G * sz;
  }
}

/* The same sum in x87 extended precision (64-bit mantissa): the "truth" the
 * error statistics are measured against. */
void orc_accel_ld(size_t n, const double* x, const double* y, const double* z, const double* m,
                  double G, double eps2, double* ax, double* ay, double* az) {
  long long N = (long long)n;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long i = 0; i < N; ++i) {
    long double sx = 0.0L, sy = 0.0L, sz = 0.0L;
    for (long long j = 0; j < N; ++j) {
      if (j == i) continue;
      long double dx = (long double)x[j] - x[i], dy = (long double)y[j] - y[i],
                  dz = (long double)z[j] - z[i];
      long double r2 = dx * dx + dy * dy + dz * dz + (long double)eps2;
      long double dist = sqrtl(r2);
      long double w = (long double)m[j] / (dist * r2);
      sx += w * dx; sy += w * dy; sz += w * dz;
    }
    ax[i] = (double)(G * sx); ay[i] = (double)(G * sy); az[i] = (double)(G * sz);
  }
}

/* orc_accel_ld restricted to the receivers idx[0..nidx) (sources: all n):
 * checks full-size systems on a sample of particles. */
void orc_accel_subset_ld(size_t n, const double* x, const double* y, const double* z,
                         const double* m, double G, double eps2, size_t nidx, const long long* idx,
                         double* ax, double* ay, double* az) {
  long long K = (long long)nidx, N = (long long)n;
#pragma omp parallel for schedule(dynamic, 1)
  for (long long q = 0; q < K; ++q) {
    long long i = idx[q];
    long double sx = 0.0L, sy = 0.0L, sz = 0.0L;
    for (long long j = 0; j < N; ++j) {
      if (j == i) continue;
      long double dx = (long double)x[j] - x[i], dy = (long double)y[j] - y[i],
                  dz = (long double)z[j] - z[i];
      long double r2 = dx * dx + dy * dy + dz * dz + (long double)eps2;
      long double w = (long double)m[j] / (sqrtl(r2) * r2);
      sx += w * dx; sy += w * dy; sz += w * dz;
    }
    ax[q] = (double)(G * sx); ay[q] = (double)(G * sy); az[q] = (double)(G * sz);
  }
}

/* Explicit Euler of reduced_solver_omp (CPU/omp_solver.cpp:121-135) in
 * acceleration form: a = accel(x); x += v dt; v += a dt. */
void orc_euler(size_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
               const double* m, double G, double eps2, double dt, size_t steps) {
  double* ax = (double*)malloc((n ? n : 1) * 3 * sizeof(double));
  double* ay = ax + n; double* az = ay + n;
  for (size_t t = 0; t < steps; ++t) {
    orc_accel(n, x, y, z, m, G, eps2, ax, ay, az);
    for (size_t i = 0; i < n; ++i) {
      x[i] += vx[i] * dt; y[i] += vy[i] * dt; z[i] += vz[i] * dt;
      vx[i] += ax[i] * dt; vy[i] += ay[i] * dt; vz[i] += az[i] * dt;
    }
  }
  free(ax);
}

/* Per-particle softened potential phi_i = -G sum_{j != i} m_j / sqrt(r^2+eps^2)
 * in extended precision.  The reference's unsoftened U
 * (calculate_potential_energy, CPU/force_calculation.cpp:1880-1904) is
 * U = 1/2 sum_i m_i phi_i at eps = 0. */
void orc_potential(size_t n, const double* x, const double* y, const double* z, const double* m,
                   double G, double eps2, double* phi) {
  long long N = (long long)n;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long i = 0; i < N; ++i) {
    long double s = 0.0L;
    for (long long j = 0; j < N; ++j) {
      if (j == i) continue;
      long double dx = (long double)x[j] - x[i], dy = (long double)y[j] - y[i],
                  dz = (long double)z[j] - z[i];
      s += (long double)m[j] / sqrtl(dx * dx + dy * dy + dz * dz + (long double)eps2);
    }
    phi[i] = (double)(-G * s);
  }
}

/* out[0..9] = T, U, E, Px, Py, Pz, Lx, Ly, Lz, M.  T as
 * compute_kinetic_energy (CPU/force_calculation.cpp:1740-1748); U softened. */
void orc_energy(size_t n, const double* x, const double* y, const double* z, const double* vx,
                const double* vy, const double* vz, const double* m, double G, double eps2,
                double* out) {
  double* phi = (double*)malloc((n ? n : 1) * sizeof(double));
  orc_potential(n, x, y, z, m, G, eps2, phi);
  long double T = 0, U = 0, P[3] = {0, 0, 0}, L[3] = {0, 0, 0}, M = 0;
  for (size_t i = 0; i < n; ++i) {
    T += 0.5L * m[i] * ((long double)vx[i] * vx[i] + (long double)vy[i] * vy[i] + (long double)vz[i] * vz[i]);
    U += 0.5L * m[i] * (long double)phi[i];
    P[0] += (long double)m[i] * vx[i]; P[1] += (long double)m[i] * vy[i]; P[2] += (long double)m[i] * vz[i];
    L[0] += (long double)m[i] * ((long double)y[i] * vz[i] - (long double)z[i] * vy[i]);
    L[1] += (long double)m[i] * ((long double)z[i] * vx[i] - (long double)x[i] * vz[i]);
    L[2] += (long double)m[i] * ((long double)x[i] * vy[i] - (long double)y[i] * vx[i]);
    M += m[i];
  }
  free(phi);
  out[0] = (double)T; out[1] = (double)U; out[2] = (double)(T + U);
  out[3] = (double)P[0]; out[4] = (double)P[1]; out[5] = (double)P[2];
  out[6] = (double)L[0]; out[7] = (double)L[1]; out[8] = (double)L[2];
  out[9] = (double)M;
}

/* Yoshida weights -> c[2w], d[2w-1] for orders 2/4/6/8; restated from
 * omp_main (CPU/omp_solver.cpp:677-726).  Returns lf_steps = 2w. */
int orc_yoshida(int order, double* c, double* d) {
  double w2[1] = {1.0};
  double cb = cbrt(2.0);
  double w4[2] = {-cb / (2.0 - cb), 1.0 / (2.0 - cb)};
  double w6[4] = {1.0, -1.17767998417887, 0.235573213359357, 0.78451361047756};
  double w8[8] = {1.0, -0.161582374150097e1, -0.244699182370524e1, -0.716989419708120e-2,
                  0.244002732616735e1, 0.157739928123617, 0.182020630970714e1, 0.104242620869991e1};
  for (int i = 1; i < 4; ++i) w6[0] -= 2.0 * w6[i];
  for (int i = 1; i < 8; ++i) w8[0] -= 2.0 * w8[i];
  const double* w = w2; int ws = 1;
  if (order == 4) { w = w4; ws = 2; }
  else if (order == 6) { w = w6; ws = 4; }
  else if (order == 8) { w = w8; ws = 8; }
  for (int i = 0; i < ws; ++i) {
    double ci = (i == 0) ? w[ws - 1] / 2.0 : (w[ws - i] + w[ws - 1 - i]) / 2.0;
    c[i] = ci; c[2 * ws - 1 - i] = ci;
    d[i] = w[ws - 1 - i]; d[2 * ws - 2 - i] = w[ws - 1 - i];
  }
  return 2 * ws;
}

/* Symplectic drift-kick-...-drift step with Yoshida c/d, the schedule of
 * reduced_solver_omp_lf (CPU/omp_solver.cpp:305-420): for each sub-step s,
 * x += c[s] v dt; a = accel(x); v += d[s] a dt; then x += c[last] v dt. */
void orc_dkd(size_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
             const double* m, double G, double eps2, double dt, size_t steps, int order) {
  double c[16], d[16];
  int lf = orc_yoshida(order, c, d);
  double* ax = (double*)malloc((n ? n : 1) * 3 * sizeof(double));
  double* ay = ax + n; double* az = ay + n;
  for (size_t t = 0; t < steps; ++t) {
    for (int s = 0; s < lf - 1; ++s) {
      for (size_t i = 0; i < n; ++i) {
        x[i] += c[s] * vx[i] * dt; y[i] += c[s] * vy[i] * dt; z[i] += c[s] * vz[i] * dt;
      }
      orc_accel(n, x, y, z, m, G, eps2, ax, ay, az);
      for (size_t i = 0; i < n; ++i) {
        vx[i] += d[s] * ax[i] * dt; vy[i] += d[s] * ay[i] * dt; vz[i] += d[s] * az[i] * dt;
      }
    }
    for (size_t i = 0; i < n; ++i) {
      x[i] += c[lf - 1] * vx[i] * dt; y[i] += c[lf - 1] * vy[i] * dt; z[i] += c[lf - 1] * vz[i] * dt;
    }
  }
  free(ax);
}

/* Kick-drift-kick leapfrog: v += a dt/2; x += v dt; a = accel(x); v += a dt/2.
 * The reference has only DKD; KDK is the scheme the softened workloads use. */
void orc_kdk(size_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
             const double* m, double G, double eps2, double dt, size_t steps) {
  double* ax = (double*)malloc((n ? n : 1) * 3 * sizeof(double));
  double* ay = ax + n; double* az = ay + n;
  orc_accel(n, x, y, z, m, G, eps2, ax, ay, az);
  for (size_t t = 0; t < steps; ++t) {
    for (size_t i = 0; i < n; ++i) {
      vx[i] += 0.5 * dt * ax[i]; vy[i] += 0.5 * dt * ay[i]; vz[i] += 0.5 * dt * az[i];
      x[i] += dt * vx[i]; y[i] += dt * vy[i]; z[i] += dt * vz[i];
    }
    orc_accel(n, x, y, z, m, G, eps2, ax, ay, az);
    for (size_t i = 0; i < n; ++i) {
      vx[i] += 0.5 * dt * ax[i]; vy[i] += 0.5 * dt * ay[i]; vz[i] += 0.5 * dt * az[i];
    }
  }
  free(ax);
}

/* Ring of n-1 equal masses on radius R plus a central mass ratio*m, with the
 * masses chosen so that omega is an exact circular orbit; restated from
 * init_stable_orbiting_particles (CPU/nbody_system.cpp:319-384).  f* receives
 * the analytic FORCE (mass times acceleration) the reference stores there. */
int orc_ring_init(size_t n, double R, double omega, double ratio, double* x, double* y, double* z,
                  double* vx, double* vy, double* vz, double* m, double* fx, double* fy, double* fz) {
  if (n < 2) return -1;
  size_t r = n - 1;
  double total = R * R * R * omega * omega;  /* G = 1 */
  double sum = 0.0;
  for (size_t i = 1; i <= (r - 1) / 2; ++i)
    sum += (2.0 + 2.0 * cos((ORC_PI * (double)(r - 2 * i)) / (double)r)) /
           pow(2.0 - 2.0 * cos((double)i * 2 * ORC_PI / (double)r), 1.5);
  if (r % 2 == 0) sum += 0.25;
  sum += ratio;
  double mr = total / sum;
  for (size_t i = 0; i < r; ++i) {
    double th = (double)i * 2 * ORC_PI / (double)r;
    m[i] = mr;
    x[i] = R * cos(th); y[i] = R * sin(th); z[i] = 0.0;
    vx[i] = -R * omega * sin(th); vy[i] = R * omega * cos(th); vz[i] = 0.0;
    fx[i] = -mr * R * omega * omega * cos(th);
    fy[i] = -mr * R * omega * omega * sin(th);
    fz[i] = 0.0;
  }
  m[r] = ratio * mr;
  x[r] = y[r] = z[r] = vx[r] = vy[r] = vz[r] = fx[r] = fy[r] = fz[r] = 0.0;
  return 0;
}

/* Rigid rotation by 2 pi * step / steps_per_rev
 * (predict_stable_orbiting_particles, CPU/nbody_system.cpp:386-408). */
int orc_ring_predict(size_t n, double R, double omega, size_t step, size_t steps_per_rev,
                     double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  if (n < 2) return -1;
  size_t r = n - 1;
  double off = (double)step / (double)steps_per_rev;
  for (size_t i = 0; i < r; ++i) {
    double th = ((double)i / (double)r + off) * 2 * ORC_PI;
    x[i] = R * cos(th); y[i] = R * sin(th); z[i] = 0.0;
    vx[i] = -R * omega * sin(th); vy[i] = R * omega * cos(th); vz[i] = 0.0;
  }
  x[r] = y[r] = z[r] = vx[r] = vy[r] = vz[r] = 0.0;
  return 0;
}

/* ------------------------------------------------------------ samplers ----
 * The seeded synthetic systems the benchmark and the tests run on, restated
 * here so that a process that must not load the product (the timed reference
 * arm) can build the same inputs.  Same algorithms and the same generator as
 * the product's samplers (nbr_ic_plummer & co.), so a seed gives the same bits:
 *   - xoshiro256** (Blackman & Vigna, 2018) seeded through splitmix64;
 *   - 53 random bits -> a double in [0, 1) or (0, 1];
 *   - Plummer sphere in N-body units (G = M = 1, scale radius a = 3 pi / 16),
 *     Aarseth, Henon & Wielen (1974): r = a / sqrt(X^(-2/3) - 1) with the
 *     enclosed mass fraction X <= 0.999, speed q v_esc(r) with q by von Neumann
 *     rejection from q^2 (1 - q^2)^(7/2) (bound 0.1), isotropic directions,
 *     then centre of mass and momentum moved to zero;
 *   - uniform ball by rejection from the cube [-1, 1]^3.
 * tests/test_oracle.py checks bit-identity with the product's samplers. */
typedef struct { unsigned long long s[4]; } orc_rng;

static unsigned long long orc_splitmix64(unsigned long long* s) {
  unsigned long long z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static unsigned long long orc_rotl(unsigned long long x, int k) { return (x << k) | (x >> (64 - k)); }
static void orc_rng_seed(orc_rng* g, unsigned long long seed) {
  unsigned long long z = seed;
  for (int i = 0; i < 4; ++i) g->s[i] = orc_splitmix64(&z);
}
static unsigned long long orc_rng_next(orc_rng* g) {
  unsigned long long* s = g->s;
  const unsigned long long r = orc_rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
  s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
  s[2] ^= t; s[3] = orc_rotl(s[3], 45);
  return r;
}
static double orc_u01(orc_rng* g) { return (double)(orc_rng_next(g) >> 11) * 0x1.0p-53; }
static double orc_u01_pos(orc_rng* g) { return (double)((orc_rng_next(g) >> 11) + 1) * 0x1.0p-53; }

static void orc_isotropic(orc_rng* g, double r, double* x, double* y, double* z) {
  const double c = 1.0 - 2.0 * orc_u01(g);
  const double ph = 2.0 * ORC_PI * orc_u01(g);
  const double s = sqrt(fmax(0.0, 1.0 - c * c));
  *x = r * s * cos(ph);
  *y = r * s * sin(ph);
  *z = r * c;
}

static void orc_recentre(size_t n, double* a, double* b, double* c, const double* m) {
  long double sa = 0, sb = 0, sc = 0, sm = 0;
  for (size_t i = 0; i < n; ++i) {
    sa += (long double)m[i] * a[i]; sb += (long double)m[i] * b[i]; sc += (long double)m[i] * c[i];
    sm += m[i];
  }
  if (sm <= 0) return;
  const double ma = (double)(sa / sm), mb = (double)(sb / sm), mc = (double)(sc / sm);
  for (size_t i = 0; i < n; ++i) { a[i] -= ma; b[i] -= mb; c[i] -= mc; }
}

static void orc_plummer_draw(size_t n, unsigned long long seed, double* x, double* y, double* z,
                             double* vx, double* vy, double* vz) {
  orc_rng g;
  orc_rng_seed(&g, seed);
  const double a = 3.0 * ORC_PI / 16.0;
  const double vscale = sqrt(2.0 / a);
  for (size_t i = 0; i < n; ++i) {
    const double X = 0.999 * orc_u01_pos(&g);
    const double r = a / sqrt(pow(X, -2.0 / 3.0) - 1.0);
    orc_isotropic(&g, r, &x[i], &y[i], &z[i]);
    double q, h;
    do {
      q = orc_u01(&g);
      h = 0.1 * orc_u01(&g);
    } while (h > q * q * pow(1.0 - q * q, 3.5));
    const double v = q * vscale * pow(1.0 + r * r / (a * a), -0.25);
    orc_isotropic(&g, v, &vx[i], &vy[i], &vz[i]);
  }
}

/* Plummer sphere of n equal masses 1/n. */
int orc_plummer(size_t n, unsigned long long seed, double* x, double* y, double* z, double* vx,
                double* vy, double* vz, double* m) {
  if (n == 0) return -1;
  orc_plummer_draw(n, seed, x, y, z, vx, vy, vz);
  for (size_t i = 0; i < n; ++i) m[i] = 1.0 / (double)n;
  orc_recentre(n, x, y, z, m);
  orc_recentre(n, vx, vy, vz, m);
  return 0;
}

/* Plummer positions and velocities; the first n_heavy particles are `ratio`
 * times heavier than the rest, total mass 1. */
int orc_two_component(size_t n, size_t n_heavy, double ratio, unsigned long long seed, double* x,
                      double* y, double* z, double* vx, double* vy, double* vz, double* m) {
  if (n == 0 || n_heavy > n || !(ratio > 0.0)) return -1;
  orc_plummer_draw(n, seed, x, y, z, vx, vy, vz);
  const double ml = 1.0 / ((double)(n - n_heavy) + ratio * (double)n_heavy);
  for (size_t i = 0; i < n; ++i) m[i] = i < n_heavy ? ratio * ml : ml;
  orc_recentre(n, x, y, z, m);
  orc_recentre(n, vx, vy, vz, m);
  return 0;
}

/* n equal masses uniform in the unit ball, at rest. */
int orc_uniform_ball(size_t n, unsigned long long seed, double* x, double* y, double* z, double* vx,
                     double* vy, double* vz, double* m) {
  if (n == 0) return -1;
  orc_rng g;
  orc_rng_seed(&g, seed);
  for (size_t i = 0; i < n; ++i) {
    double a, b, c;
    do {
      a = 2.0 * orc_u01(&g) - 1.0;
      b = 2.0 * orc_u01(&g) - 1.0;
      c = 2.0 * orc_u01(&g) - 1.0;
    } while (a * a + b * b + c * c > 1.0);
    x[i] = a; y[i] = b; z[i] = c;
    vx[i] = vy[i] = vz[i] = 0.0;
    m[i] = 1.0 / (double)n;
  }
  return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

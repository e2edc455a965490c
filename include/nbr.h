/* nbr.h -- C ABI of the B200 all-pairs N-body solver (libnbr.so).
 *
 * The solver is a drop-in for the force-and-integrate path of the reference
 * CPU solver (pc2/n-body-ring-solver, directory CPU/).  Each entry point
 * below names the reference interface it replaces.  Conventions:
 *
 *  - plain pointers and sizes only; every host array is a caller-owned
 *    contiguous double array of length n (structure of arrays, the layout of
 *    NBody_system, CPU/nbody_system.h:41-74);
 *  - every function returns an nbr_status; nothing aborts and no exception
 *    crosses the ABI (the reference has no error channel at all,
 *    CPU/force_calculation.cpp:1129);
 *  - one context = one GPU + one CUDA stream; a context is used by one host
 *    thread at a time;
 *  - units are the caller's: G is a parameter (the reference fixes G = 1,
 *    CPU/nbody_system.h:11); eps2 is the Plummer softening length squared
 *    (the reference has none: eps2 = 0 reproduces it, skipping coincident
 *    pairs the way the reference skips q == k).
 */
#ifndef NBR_H
#define NBR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum nbr_status {
  NBR_OK = 0,
  NBR_ERR_INVALID_ARG = 1,  /* bad pointer, size or enum value */
  NBR_ERR_CUDA = 2,         /* a CUDA call failed; see nbr_last_error_string */
  NBR_ERR_NO_MEMORY = 3,    /* device or host allocation failed */
  NBR_ERR_TIMEOUT = 4,      /* a bounded device wait gave up (kernel aborted cleanly) */
  NBR_ERR_NO_SYSTEM = 5,    /* no particles uploaded yet */
  NBR_ERR_UNSUPPORTED = 6,  /* no CUDA device / unsupported configuration */
  NBR_ERR_NONFINITE = 7,    /* an input contains NaN or Inf */
  NBR_ERR_IO = 8,           /* a snapshot file could not be opened, read or written */
  NBR_ERR_BOUNDS = 9        /* libnbr_checked.so only: a kernel index fell outside its
                               array; the access was skipped (a library defect) */
} nbr_status;

/* Arithmetic of the pair interaction. */
typedef enum nbr_precision {
  NBR_FP64 = 0,  /* plain FP64: matches the reference's double-precision forces */
  NBR_FP32C = 1  /* FP32 pair arithmetic on FP64 tile-relative coordinates,
                    TwoSum-compensated cross-tile sums, FP64 integration */
} nbr_precision;

/* Leapfrog schedule. */
typedef enum nbr_scheme {
  NBR_KDK = 0,  /* kick-drift-kick, force reused across steps */
  NBR_DKD = 1,  /* drift-kick-drift with Yoshida c/d coefficients, the schedule of
                   reduced_solver_omp_lf (CPU/omp_solver.cpp:257-456) */
  NBR_EULER = 2 /* explicit Euler, x += v dt then v += a dt: reduced_solver_omp
                   (CPU/omp_solver.cpp:16-178), the reference's default -i euler */
} nbr_scheme;

typedef struct nbr_ctx nbr_ctx;

/* Conserved quantities of the current state, all in FP64.  U is the softened
 * potential energy 1/2 sum_i m_i phi_i. */
typedef struct nbr_diag {
  double T, U, E;
  double P[3];
  double L[3];
  double M;
} nbr_diag;

/* Per-call statistics of nbr_run / nbr_batch_run. */
typedef struct nbr_run_stats {
  double force_evals;   /* force evaluations launched */
  double pairs;         /* ordered pairs i != j evaluated: force_evals * sum N(N-1) */
  double gpu_ms;        /* device time of the launch sequence (CUDA events) */
  double kernels;       /* kernel launches issued */
} nbr_run_stats;

/* ------------------------------------------------------------ context ---- */
/* Creates a context on `device` (its own stream and device error word). */
int nbr_ctx_create(int device, nbr_ctx** out);
int nbr_ctx_destroy(nbr_ctx* ctx);
/* Last error message of the context (or of the calling thread if ctx is NULL). */
const char* nbr_last_error_string(const nbr_ctx* ctx);
/* Library version, e.g. 1000 for 0.1.0. */
int nbr_version(void);
/* Number of visible CUDA devices (0 when none); never fails. */
int nbr_device_count(void);
/* The context's CUDA stream (a cudaStream_t as an opaque pointer), for callers
 * that time or order their own work against the solver's. */
void* nbr_ctx_stream(nbr_ctx* ctx);
/* Waits for all work issued on the context's stream; reports a bounded-wait
 * timeout (NBR_ERR_TIMEOUT) of asynchronous calls issued before it. */
int nbr_ctx_synchronize(nbr_ctx* ctx);

/* -------------------------------------------------------------- state ---- */
/* Copies a system of n particles in (replaces NBody_system::alloc_particles +
 * the initialisers' stores, CPU/nbody_system.cpp:177-193).  vx/vy/vz may be
 * NULL (zero velocities).  Rejects NaN/Inf (NBR_ERR_NONFINITE) and negative
 * masses (NBR_ERR_INVALID_ARG); the check runs on the device copy, and a
 * rejected upload leaves the context with no system. */
int nbr_system_upload(nbr_ctx* ctx, size_t n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz, const double* m);
/* Copies the current state out; any pointer may be NULL. */
int nbr_system_download(nbr_ctx* ctx, double* x, double* y, double* z, double* vx, double* vy,
                        double* vz);
/* Particle count of the uploaded system (0 if none). */
size_t nbr_system_size(const nbr_ctx* ctx);

/* ------------------------------------------------------------- forces ---- */
/* Accelerations (want_force = 0) or forces m_i a_i (want_force = 1) of the
 * uploaded system, a_i = G sum_{j != i} m_j (x_j - x_i) / (|x_j - x_i|^2 + eps2)^{3/2},
 * written (overwrite, not accumulate) to the host arrays.  Replaces the force
 * kernels compute_forces_simple / _avx2 / _avx2_blocked / _avx512_rsqrt(_4i)_blocked
 * (CPU/force_calculation.h:7-14) with their Newton-3 split summed: the
 * reference's force + recv_force (CPU/omp_solver.cpp:124-126). */
int nbr_forces(nbr_ctx* ctx, int precision, double G, double eps2, int want_force, double* ax,
               double* ay, double* az);

/* The same evaluation left on the device: accelerations of the current state
 * into the context's acceleration arrays (read back with nbr_forces_download).
 * One force-kernel launch (plus a one-off pack of the FP32C records after an
 * upload); for timing the kernel with the caller's own events on
 * nbr_ctx_stream.  Asynchronous: returns after enqueueing. */
int nbr_forces_device(nbr_ctx* ctx, int precision, double G, double eps2);
/* Copies the accelerations left by nbr_forces_device / nbr_run to the host. */
int nbr_forces_download(nbr_ctx* ctx, double* ax, double* ay, double* az);

/* Largest particle count nbr_forces_noalloc accepts. */
#define NBR_NOALLOC_MAX_N 32768

/* Accelerations of n particles (FP64 or FP32C, as nbr_forces with
 * want_force = 0) computed without allocating anything.  This entry point has
 * no counterpart in the reference.  It exists for callers that cannot let a
 * library allocate device memory: an application whose memory pool owns every
 * device allocation, a process held to a fixed device-memory budget, or a
 * latency-critical loop that cannot afford the synchronisation cudaMalloc and
 * cudaFree may imply.  The caller provides the inputs and outputs; all
 * scratch lives in one static device array inside libnbr.so (about 8.5 MB),
 * which every GPU that loads the library holds until the process exits.
 *  - x, y, z, m (n entries) and ax, ay, az (n entries) are device-accessible
 *    pointers (device, managed or mapped pinned memory) owned by the caller;
 *  - n <= NBR_NOALLOC_MAX_N, else NBR_ERR_INVALID_ARG and nothing runs;
 *  - stream: a cudaStream_t (NULL for the default stream); the call returns
 *    after the work on that stream has finished, so a bounded-wait timeout can
 *    be reported (NBR_ERR_TIMEOUT);
 *  - the first call on a device looks up the scratch array's device address
 *    (cudaGetSymbolAddress, with that device current); make that first call
 *    before any stream capture;
 *  - the looked-up address is kept for the life of the process: after a
 *    cudaDeviceReset of a device, do not call this entry point on it again;
 *  - all calls on a device share the scratch array, which keeps the last
 *    call's contents (each call clears what must start at zero); calls that
 *    overlap on the same GPU, from several streams or host threads, race on it
 *    and must be serialised by the caller.
 * Errors are reported through nbr_last_error_string(NULL). */
int nbr_forces_noalloc(int precision, size_t n, const double* x, const double* y, const double* z,
                       const double* m, double G, double eps2, double* ax, double* ay, double* az,
                       void* stream);

/* Accelerations or forces on n_i receivers from n_j sources (separate sets).
 * The block-pair call the reference's ring decomposition makes for a received
 * block (compute_forces_* with local_N, rank, comm_sz, recv_round,
 * CPU/hybrid_solver.cpp:84-95), evaluated in full rather than as a Newton-3
 * half.  mi (receiver masses) is needed only for want_force = 1.  Pairs at
 * zero distance are skipped when eps2 = 0 (the reference skips q == k). */
int nbr_accel_ij(nbr_ctx* ctx, int precision, size_t n_i, const double* xi, const double* yi,
                 const double* zi, const double* mi, size_t n_j, const double* xj,
                 const double* yj, const double* zj, const double* mj, double G, double eps2,
                 int want_force, double* ax, double* ay, double* az);

/* Per-particle softened potential phi_i = -G sum_{j != i} m_j / sqrt(r^2 + eps2)
 * (phi may be NULL) and U = 1/2 sum m_i phi_i, in FP64.  At eps2 = 0 U equals
 * calculate_potential_energy / compute_potential_energy_avx2
 * (CPU/force_calculation.cpp:1749-1904). */
int nbr_potential(nbr_ctx* ctx, double G, double eps2, double* phi, double* U);

/* T, U, E, P, L, M of the current state (FP64, block-reduced on the GPU).
 * T replaces compute_kinetic_energy (CPU/force_calculation.cpp:1740-1748). */
int nbr_diagnostics(nbr_ctx* ctx, double G, double eps2, nbr_diag* out);

/* ---------------------------------------------------------- integrate ---- */
/* Advances the uploaded system by `steps` steps of size dt.
 *   scheme NBR_DKD: Yoshida order 2/4/6/8, 2w-1 force evaluations per step,
 *     the schedule of reduced_solver_omp_lf (CPU/omp_solver.cpp:257-456) with
 *     the coefficients of omp_main (CPU/omp_solver.cpp:677-743);
 *   scheme NBR_KDK: order must be 2; one force evaluation per step, the last
 *     acceleration is reused by the next call (first-same-as-last);
 *   scheme NBR_EULER: order ignored; one force evaluation per step.
 * The launch sequence is captured in one CUDA graph.  diag (optional, 2
 * entries) receives the diagnostics before and after; stats may be NULL. */
int nbr_run(nbr_ctx* ctx, int precision, int scheme, int order, double dt, size_t steps, double G,
            double eps2, nbr_diag* diag, nbr_run_stats* stats);

/* Yoshida c[2w] / d[2w-1] of omp_main (CPU/omp_solver.cpp:677-726) for order
 * 2, 4, 6 or 8; returns lf_steps = 2w, or 0 for an unsupported order. */
int nbr_yoshida_coefficients(int order, double* c, double* d);

/* --------------------------------------------- multi-GPU i-partition ---- */
/* One process (and one context) per GPU; every context holds the whole system
 * and owns the receivers [i0, i0 + count).  A step is one force evaluation
 * of the owned receivers against all n sources, their kick and drift, then an
 * exchange that brings every context the new positions of all particles.
 * This replaces hybrid_full_solver (CPU/hybrid_solver.cpp:226-336): each MPI
 * rank owns local_N = N / comm_sz particles, computes their forces against
 * all N (compute_forces_full_avx2, :288), updates them (:290-299) and
 * MPI_Allgathers the positions (:310).  The exchange belongs to the caller
 * (e.g. an NCCL all-gather on the arrays nbr_state_pointers returns, ordered
 * after the step on nbr_ctx_stream); the library only computes. */

/* One force evaluation of receivers [i0, i0 + count) (count is clipped to
 * n - i0; i0 a multiple of 128) with the fused update, asynchronous on the
 * context's stream:
 *   scheme NBR_KDK or NBR_DKD: v += kick * a, then x' = x + drift * v;
 *   scheme NBR_EULER:          x' = x + drift * v_old, v += kick * a;
 * x' goes to the other position buffer, which becomes current.  Only the
 * range's entries of that buffer are written: the positions of every other
 * particle must be filled in (the exchange) before the next step, followed
 * by nbr_state_changed.  A KDK run of k steps from x_0 is k + 1 calls with
 * (kick, drift) = (dt/2, dt), then (dt, dt) k - 1 times, then (dt/2, 0).
 * A bounded-wait timeout is reported by the next synchronising call
 * (nbr_ctx_synchronize, a download). */
int nbr_step_range(nbr_ctx* ctx, int precision, int scheme, size_t i0, size_t count, double kick,
                   double drift, double G, double eps2);
/* Newton-3 across GPUs (the GPU image of hybrid_ring_solver's travelling
 * partial forces, CPU/hybrid_solver.cpp:52-107, with a fixed reduction order).
 * The block-pair triangle of the uploaded system is cut into nslices slices
 * of consecutive row groups with equal pair work; each unordered pair belongs
 * to exactly one slice.  nbr_n3_slice_accel writes the partial accelerations
 * (not multiplied by G) that each slice v in [slice_begin, slice_end) gives
 * EVERY particle, in FP64, into the device array dst[(v - slice_begin) * 3 *
 * ld + d * ld + i] (d = x, y, z; ld >= the system size rounded up to 1024),
 * asynchronous on the context's stream; the slices of the range share one
 * pair-kernel launch (each slice's partials are the same as when computed
 * alone).  A rank computes
 * its slices, the ranks exchange the columns of their owned ranges (an
 * all-to-all), and nbr_step_range_sum adds, for the receivers [i0, i0 +
 * count) (i0 a multiple of 128), the nslices partials in slice order --
 * src[v * vstride + d * ld + k] for receiver i0 + k, ld >= count rounded up
 * to 128 -- multiplies by G and applies the fused kick/drift of scheme
 * (NBR_KDK / NBR_DKD: v += kick a, x' = x + drift v; NBR_EULER: drift with
 * the old velocity) to them, like nbr_step_range.  With the same nslices the
 * result does not depend on how the slices are spread over ranks. */
int nbr_n3_slice_accel(nbr_ctx* ctx, int precision, double eps2, int slice_begin, int slice_end,
                       int nslices, double* dst, size_t ld);
/* The Newton-3 grid the library plans for a system of n particles on a device
 * of `sms` SMs (host only: no context or device needed).  The grid has one
 * CTA per (row group of 8 blocks of 256 particles, chunk of column blocks);
 * the chunk width and the launch order come from a list-scheduling model of
 * the launch.  Outputs (any may be NULL): *cols, column blocks per CTA of the
 * whole-system grid; *slice_cols, of its `nslices` row-group slices (the
 * multi-GPU partition; nslices >= 1); *efficiency, the model's pair work
 * spread evenly over the SMs / the grid's finishing time (1 at best); *ctas,
 * the whole-system grid's CTA count; order[0 .. min(order_cap, *ctas) - 1],
 * the launch order (launch index -> group-major CTA number, longest CTA
 * first).  NBR_ERR_INVALID_ARG for n < 1, sms < 1 or nslices < 1. */
int nbr_n3_grid_plan(size_t n, int sms, int nslices, int* cols, int* slice_cols,
                     double* efficiency, long long* ctas, int* order, long long order_cap);
int nbr_step_range_sum(nbr_ctx* ctx, int precision, int scheme, size_t i0, size_t count, double kick,
                       double drift, double G, const double* src, int nslices, size_t vstride,
                       size_t ld);
/* Device pointers of the current position and velocity arrays of the
 * uploaded system (any pointer may be NULL) and their allocated length
 * (*len >= n; entries >= n are zero-mass padding).  The position pointers
 * change with every step (double buffering): query them after each step. */
int nbr_state_pointers(nbr_ctx* ctx, double** x, double** y, double** z, double** vx, double** vy,
                       double** vz, size_t* len);
/* Declares that positions or velocities were written through
 * nbr_state_pointers: FP32C source records are rebuilt from the positions at
 * the next evaluation and stored accelerations are not reused. */
int nbr_state_changed(nbr_ctx* ctx);
/* ---------------------------------------------------------- snapshots ---- */
/* Checkpoints in the reference's binary snapshot format,
 * NBody_system::save_particles (CPU/nbody_system.cpp:133-152): per record the
 * time time_step * delta_t, then n masses, positions x, y, z, velocities
 * x, y, z and forces x, y, z, all native-endian doubles (8 + 80 n bytes).  The
 * reference names the file "NBody_<n>.dat"; here the caller names it.
 * time_step == 0 truncates the file, any other value appends a record. */

/* One record from host arrays (m, x, y, z required; velocities and forces may
 * be NULL: written as zeros).  No context and no GPU needed. */
int nbr_snapshot_write_arrays(const char* path, size_t n, size_t time_step, double delta_t,
                              const double* m, const double* x, const double* y, const double* z,
                              const double* vx, const double* vy, const double* vz,
                              const double* fx, const double* fy, const double* fz);
/* One record of the context's current state.  Forces are m_i a_i of the
 * current positions when the context holds those accelerations (after
 * nbr_forces with want_force = 0, nbr_forces_device or a KDK nbr_run), zeros
 * otherwise. */
int nbr_snapshot_save(nbr_ctx* ctx, const char* path, size_t time_step, double delta_t);
/* Number of whole n-particle records in the file (NBR_ERR_INVALID_ARG when the
 * size is not a whole number of records: wrong n or a truncated file). */
int nbr_snapshot_records(const char* path, size_t n, size_t* records);
/* Record `record` (0-based) into host arrays; any output may be NULL. */
int nbr_snapshot_read_arrays(const char* path, size_t n, size_t record, double* time, double* m,
                             double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             double* fx, double* fy, double* fz);
/* Resume: uploads record `record` (masses, positions, velocities) as the
 * context's system; *time (may be NULL) receives its time. */
int nbr_snapshot_load(nbr_ctx* ctx, const char* path, size_t n, size_t record, double* time);

/* ------------------------------------------------------------ tuning ---- */
/* Forces a kernel configuration for the given precision (ni receivers per
 * thread: 4 or 8; warps per CTA: 2, 4 or 8; split >= 1 or 0 = automatic;
 * ni = 1: the small-N kernel with warps = 2, 4 or 8 lane groups per warp;
 * ni = 3, warps = 8: the Newton-3 kernel, each unordered pair evaluated once
 * and applied to both particles, for FP32C and for FP64; for FP32C also
 * warps = 16, two warps per 256-particle row block; whole systems only,
 * receiver ranges and separate receiver and source sets fall back to the large
 * kernels; ni = 2, warps = 4, 8 or 16 lane groups per warp, split = 8 or 16
 * warps per CTA (0: 16; FP32C: 16 only): nbr_run of a system of at most 4096
 * particles as one cooperative launch for all steps (the default for such
 * systems, both precisions), evaluations outside nbr_run use the default
 * kernels).  ni = 0 restores the autotuner. */
int nbr_set_force_config(nbr_ctx* ctx, int precision, int ni, int warps, int split);
/* The j-tile (sources per stage of the shared-memory ring: 64, 128 or 256)
 * and the unroll depth of the source loop (2, 4 or 8) of the large kernels,
 * for a configuration forced with nbr_set_force_config (ni 4 or 8); 0 takes
 * the default (128; unroll 4 for FP32C, 2 for FP64).  Built for the default
 * large configurations FP32C (8, 2) and FP64 (4, 4); other (tile, unroll)
 * pairs return NBR_ERR_INVALID_ARG.  For the persistent small-system run (ni
 * = 2) tile is its receivers per lane instead: 4 (the default) or 8, the
 * latter with 8 or 16 lane groups. */
int nbr_set_force_tiling(nbr_ctx* ctx, int precision, int tile, int unroll);
/* The j-tile and unroll depth a force evaluation of the uploaded system would
 * use (0 and 0 when the chosen kernel is not a large one). */
int nbr_get_force_tiling(nbr_ctx* ctx, int precision, double eps2, int* tile, int* unroll);
/* The configuration a force evaluation of the uploaded system would use
 * (forced, autotuned or default): ni = 4 or 8 receivers per thread of the
 * large kernels, ni = 1 the small-N kernel (warps = lane groups per warp),
 * ni = 3 the Newton-3 kernel (each unordered pair once; the default of both
 * precisions from 16384 to 2^20 particles); split = j splits (unused by the
 * Newton-3 kernel). */
int nbr_get_force_config(nbr_ctx* ctx, int precision, double eps2, int* ni, int* warps, int* split);
/* Times the supported configurations for the uploaded system and stores the
 * fastest in the autotune cache file (see nbr_tune_cache_path) under the
 * system's (precision, log2 N, log2 source tiles, eps == 0) bucket: receivers
 * per thread and warps per CTA (the i-tile), three j-splits, the small-N and
 * Newton-3 kernels, and, when the large kernel's default configuration wins,
 * its j-tile (64, 128, 256) and unroll depth (2, 4, 8).  Later evaluations in
 * the same bucket use the stored winner. */
int nbr_autotune(nbr_ctx* ctx, int precision, double eps2);
/* Path of the JSON autotune cache ($NBR_TUNE_CACHE or the library directory). */
const char* nbr_tune_cache_path(void);

/* ------------------------------------------------------- init conditions ---- */
/* Deterministic samplers (xoshiro256** seeded through splitmix64; the same
 * seed gives the same bits on every host).  N-body units G = M = 1. */
/* Plummer sphere, scale radius a = 3 pi / 16, equal masses 1/n, positions by
 * the inverse cumulative mass (mass fraction <= 0.999), speeds by von Neumann
 * rejection from the isotropic distribution function; centre of mass and
 * mean velocity moved to zero. */
int nbr_ic_plummer(size_t n, uint64_t seed, double* x, double* y, double* z, double* vx,
                   double* vy, double* vz, double* m);
/* Uniform density in the unit ball, zero velocities, masses 1/n (not recentred). */
int nbr_ic_uniform_ball(size_t n, uint64_t seed, double* x, double* y, double* z, double* vx,
                        double* vy, double* vz, double* m);
/* Plummer sphere whose first n_heavy particles weigh `ratio` times the others,
 * total mass 1. */
int nbr_ic_two_component(size_t n, size_t n_heavy, double ratio, uint64_t seed, double* x,
                         double* y, double* z, double* vx, double* vy, double* vz, double* m);
/* The reference's ring: n-1 equal masses on radius R plus a central mass
 * ratio * m, exact circular orbit with angular velocity omega
 * (init_stable_orbiting_particles, CPU/nbody_system.cpp:319-384).  f* (may be
 * NULL) receive the analytic force. */
int nbr_ic_ring(size_t n, double R, double omega, double ratio, double* x, double* y, double* z,
                double* vx, double* vy, double* vz, double* m, double* fx, double* fy,
                double* fz);
/* Analytic rigid rotation of that ring after `step` of `steps_per_rev` steps
 * (predict_stable_orbiting_particles, CPU/nbody_system.cpp:386-408). */
int nbr_ic_ring_predict(size_t n, double R, double omega, size_t step, size_t steps_per_rev,
                        double* x, double* y, double* z, double* vx, double* vy, double* vz);
/* Sizes of nsys systems drawn log-uniform in [nmin, nmax] (seed). */
int nbr_ic_batch_sizes(size_t nsys, uint64_t seed, size_t nmin, size_t nmax, size_t* sizes);
/* Seed of system s of a batch drawn with `seed`. */
uint64_t nbr_ic_system_seed(uint64_t seed, size_t s);

/* ------------------------------------------------------------- batched ---- */
/* Uploads nsys independent systems stored back to back: system s owns
 * particles offsets[s] .. offsets[s+1]-1 (offsets has nsys+1 entries,
 * offsets[0] = 0).  Systems never interact. */
int nbr_batch_upload(nbr_ctx* ctx, size_t nsys, const size_t* offsets, const double* x,
                     const double* y, const double* z, const double* vx, const double* vy,
                     const double* vz, const double* m);
/* Copies the batch state out (any pointer may be NULL). */
int nbr_batch_download(nbr_ctx* ctx, double* x, double* y, double* z, double* vx, double* vy,
                       double* vz);
/* Accelerations of every batch particle (want_force as in nbr_forces). */
int nbr_batch_forces(nbr_ctx* ctx, int precision, double G, double eps2, int want_force,
                     double* ax, double* ay, double* az);
/* KDK leapfrog of every system for `steps` steps: one persistent launch per
 * step walking a device work queue of (system, receiver tile) items (FP32C
 * Newton-3 row blocks: one more launch, the epilogue that sums each
 * particle's action and reactions in a fixed order), the whole step loop
 * captured in one CUDA graph. */
int nbr_batch_run(nbr_ctx* ctx, int precision, double dt, size_t steps, double G, double eps2,
                  nbr_run_stats* stats);
/* Forces the batched kernel's configuration for a precision: wide = 1 pairs a
 * system's receiver tiles into two-tile work items (8 receivers per lane),
 * wide = 0 keeps one-tile items (4 per lane), wide = 2 evaluates the larger
 * systems by Newton-3 row blocks -- receiver tiles against the later column
 * tiles, each pair once: FP32C two-tile blocks for systems of three tiles
 * (257 particles) or more, the others as for wide = 1; FP64 one-tile blocks
 * for systems of two tiles (129 particles) or more, the others as for
 * wide = 0; ctas_per_sm = resident CTAs per SM of the persistent grid (0: the
 * occupancy limit).  wide = -1 restores the autotune cache or the default
 * (occupancy limit; Newton-3 row blocks).  Applies to the uploaded batch; an
 * upload starts from the autotune cache again.  The Newton-3 scratch (3
 * doubles per particle and 3 x 128 doubles per (row block, later column
 * tile)) is allocated at its first use.  Other values: NBR_ERR_INVALID_ARG. */
int nbr_batch_set_config(nbr_ctx* ctx, int precision, int wide, int ctas_per_sm);
/* Times every (item width, CTAs per SM) on the uploaded batch and stores the
 * fastest in the autotune cache under the batch's (precision, log2 system
 * count, log2 largest system, eps == 0) bucket; later uploads of a batch in
 * the same bucket use it. */
int nbr_batch_autotune(nbr_ctx* ctx, int precision, double eps2);
/* Per-system diagnostics (out has nsys entries). */
int nbr_batch_diagnostics(nbr_ctx* ctx, double G, double eps2, nbr_diag* out);

#ifdef __cplusplus
}
#endif
#endif /* NBR_H */

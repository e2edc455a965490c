"""ctypes access to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs import this module, and only to check or to time against.  The
product library never imports or links anything here.

Two libraries are wrapped:

* ``liboracle.so`` -- the plain-C softened restatement (nbr_oracle.c);
* ``_ref/libnbr_ref_*.so`` -- the reference's own CPU solver compiled from its
  sources (CPU/nbody_system.cpp, CPU/force_calculation.cpp, CPU/omp_solver.cpp)
  plus ref_glue.cpp.  The AVX-512 build is used when the host CPU has
  AVX-512F/VL, else the AVX build.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = C.POINTER(C.c_double)
_SZ = C.c_size_t
# State arrays of a system, in the order the samplers fill them.
KEYS = ("x", "y", "z", "vx", "vy", "vz", "m")

# Reference force kernels selectable through ref_forces().
REF_SIMPLE, REF_AVX2, REF_AVX2_BLOCKED, REF_AVX512_RSQRT, REF_AVX512_RSQRT_4I = range(5)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "")
    except OSError:
        return False
    toks = set(flags.split())
    return {"avx512f", "avx512vl", "avx512bw", "avx512dq", "avx512cd"} <= toks


class Oracle:
    """The plain-C softened restatement."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        L = self.lib = C.CDLL(path)
        arr7 = [_SZ, _D, _D, _D, _D, C.c_double, C.c_double, _D, _D, _D]
        for name in ("orc_accel", "orc_accel_ld"):
            getattr(L, name).argtypes = arr7
            getattr(L, name).restype = None
        L.orc_accel_subset_ld.argtypes = [_SZ, _D, _D, _D, _D, C.c_double, C.c_double, _SZ,
                                          C.POINTER(C.c_longlong), _D, _D, _D]
        L.orc_accel_subset_ld.restype = None
        L.orc_euler.argtypes = [_SZ] + [_D] * 7 + [C.c_double, C.c_double, C.c_double, _SZ]
        L.orc_potential.argtypes = [_SZ, _D, _D, _D, _D, C.c_double, C.c_double, _D]
        L.orc_energy.argtypes = [_SZ] + [_D] * 7 + [C.c_double, C.c_double, _D]
        L.orc_yoshida.argtypes = [C.c_int, _D, _D]
        L.orc_yoshida.restype = C.c_int
        L.orc_dkd.argtypes = [_SZ] + [_D] * 7 + [C.c_double, C.c_double, C.c_double, _SZ, C.c_int]
        L.orc_kdk.argtypes = [_SZ] + [_D] * 7 + [C.c_double, C.c_double, C.c_double, _SZ]
        L.orc_ring_init.argtypes = [_SZ, C.c_double, C.c_double, C.c_double] + [_D] * 10
        L.orc_ring_init.restype = C.c_int
        L.orc_ring_predict.argtypes = [_SZ, C.c_double, C.c_double, _SZ, _SZ] + [_D] * 6
        L.orc_ring_predict.restype = C.c_int
        L.orc_num_threads.restype = C.c_int
        samp = [_SZ, C.c_ulonglong] + [_D] * 7
        for name in ("orc_plummer", "orc_uniform_ball"):
            getattr(L, name).argtypes = samp
            getattr(L, name).restype = C.c_int
        L.orc_two_component.argtypes = [_SZ, _SZ, C.c_double, C.c_ulonglong] + [_D] * 7
        L.orc_two_component.restype = C.c_int

    def accel(self, x, y, z, m, G=1.0, eps2=0.0, extended=False):
        n = len(x)
        a = np.zeros((3, n))
        fn = self.lib.orc_accel_ld if extended else self.lib.orc_accel
        fn(n, _p(x), _p(y), _p(z), _p(m), G, eps2, _p(a[0]), _p(a[1]), _p(a[2]))
        return a

    def accel_subset(self, x, y, z, m, idx, G=1.0, eps2=0.0):
        """Extended-precision accelerations of the receivers idx (sources: all)."""
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        a = np.zeros((3, len(idx)))
        self.lib.orc_accel_subset_ld(len(x), _p(x), _p(y), _p(z), _p(m), G, eps2, len(idx),
                                     idx.ctypes.data_as(C.POINTER(C.c_longlong)),
                                     _p(a[0]), _p(a[1]), _p(a[2]))
        return a

    def euler(self, s, dt, steps, G=1.0, eps2=0.0):
        s = {k: v.copy() for k, v in s.items()}
        self.lib.orc_euler(len(s["x"]), *[_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")],
                           G, eps2, dt, steps)
        return s

    def potential(self, x, y, z, m, G=1.0, eps2=0.0):
        phi = np.zeros(len(x))
        self.lib.orc_potential(len(x), _p(x), _p(y), _p(z), _p(m), G, eps2, _p(phi))
        return phi

    def energy(self, s, G=1.0, eps2=0.0):
        """dict with T, U, E, P[3], L[3], M for a state dict of x,y,z,vx,vy,vz,m."""
        out = np.zeros(10)
        self.lib.orc_energy(len(s["x"]), *[_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")],
                            G, eps2, _p(out))
        return {"T": out[0], "U": out[1], "E": out[2], "P": out[3:6].copy(), "L": out[6:9].copy(),
                "M": out[9]}

    def yoshida(self, order):
        c = np.zeros(16); d = np.zeros(16)
        k = self.lib.orc_yoshida(order, _p(c), _p(d))
        return c[:k].copy(), d[:k - 1].copy()

    def dkd(self, s, dt, steps, order=2, G=1.0, eps2=0.0):
        s = {k: v.copy() for k, v in s.items()}
        self.lib.orc_dkd(len(s["x"]), *[_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")],
                         G, eps2, dt, steps, order)
        return s

    def kdk(self, s, dt, steps, G=1.0, eps2=0.0):
        s = {k: v.copy() for k, v in s.items()}
        self.lib.orc_kdk(len(s["x"]), *[_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")],
                         G, eps2, dt, steps)
        return s

    def ring_init(self, n, R=1.0, omega=2 * np.pi, ratio=1e5):
        arrs = [np.zeros(n) for _ in range(10)]
        rc = self.lib.orc_ring_init(n, R, omega, ratio, *[_p(a) for a in arrs])
        if rc != 0:
            raise ValueError("ring needs n >= 2")
        keys = ("x", "y", "z", "vx", "vy", "vz", "m", "fx", "fy", "fz")
        return dict(zip(keys, arrs))

    def _sample(self, fn, n, *args):
        s = {k: np.zeros(n) for k in KEYS}
        if fn(n, *args, *[_p(s[k]) for k in KEYS]) != 0:
            raise ValueError("bad sampler arguments")
        return s

    def plummer(self, n, seed):
        """Plummer sphere of n equal masses, the same bits as the product's
        nbr_ic_plummer for the same seed."""
        return self._sample(self.lib.orc_plummer, n, seed)

    def uniform_ball(self, n, seed):
        return self._sample(self.lib.orc_uniform_ball, n, seed)

    def two_component(self, n, n_heavy, ratio, seed):
        return self._sample(self.lib.orc_two_component, n, n_heavy, ratio, seed)

    def ring_predict(self, n, step, steps_per_rev, R=1.0, omega=2 * np.pi):
        arrs = [np.zeros(n) for _ in range(6)]
        self.lib.orc_ring_predict(n, R, omega, step, steps_per_rev, *[_p(a) for a in arrs])
        return dict(zip(("x", "y", "z", "vx", "vy", "vz"), arrs))


class Reference:
    """The reference's own CPU solver, compiled from its sources."""

    def __init__(self, path: str | None = None):
        if path is None:
            name = "libnbr_ref_avx512.so" if cpu_has_avx512() else "libnbr_ref_avx.so"
            path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources are")
        self.path = path
        L = self.lib = C.CDLL(path)
        L.ref_has_avx512.restype = C.c_int
        L.ref_max_threads.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_forces.argtypes = [C.c_int, _SZ] + [_D] * 7
        L.ref_forces.restype = C.c_int
        L.ref_lf.argtypes = [_SZ] + [_D] * 7 + [_SZ, C.c_double, C.c_int]
        L.ref_lf.restype = C.c_double
        L.ref_euler.argtypes = [_SZ] + [_D] * 7 + [_SZ, C.c_double, C.c_int]
        L.ref_euler.restype = C.c_double
        L.ref_ring_share.argtypes = [_SZ] + [_D] * 4 + [_SZ, C.c_int]
        L.ref_ring_share.restype = C.c_double
        L.ref_kinetic.argtypes = [_SZ] + [_D] * 4
        L.ref_kinetic.restype = C.c_double
        L.ref_potential.argtypes = [_SZ] + [_D] * 4 + [C.c_int]
        L.ref_potential.restype = C.c_double
        L.ref_ring_init.argtypes = [_SZ, C.c_double, C.c_double, C.c_double] + [_D] * 10
        L.ref_ring_init.restype = C.c_int
        L.ref_ring_predict.argtypes = [_SZ, C.c_double, C.c_double, _SZ, _SZ] + [_D] * 6
        L.ref_ring_predict.restype = C.c_int
        L.ref_yoshida.argtypes = [C.c_int, _D, _D]
        L.ref_yoshida.restype = C.c_int
        L.ref_save_snapshot.argtypes = [C.c_char_p, _SZ] + [_D] * 10 + [_SZ, C.c_double]
        L.ref_save_snapshot.restype = C.c_int

    @property
    def has_avx512(self) -> bool:
        return bool(self.lib.ref_has_avx512())

    def best_variant(self) -> int:
        return REF_AVX512_RSQRT_4I if self.has_avx512 else REF_AVX2_BLOCKED

    def threads(self) -> int:
        return self.lib.ref_max_threads()

    def set_threads(self, t: int):
        self.lib.ref_set_threads(int(t))

    def forces(self, x, y, z, m, variant=REF_AVX2_BLOCKED):
        n = len(x)
        f = np.zeros((3, n))
        rc = self.lib.ref_forces(variant, n, _p(x), _p(y), _p(z), _p(m), _p(f[0]), _p(f[1]), _p(f[2]))
        if rc != 0:
            raise ValueError(f"reference kernel {variant} unavailable in {self.path}")
        return f

    def lf(self, s, dt, steps, order=2):
        s = {k: v.copy() for k, v in s.items()}
        secs = self.lib.ref_lf(len(s["x"]), *[_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")],
                               steps, dt, order)
        return s, secs

    def euler(self, s, dt, steps, variant=REF_AVX2_BLOCKED):
        s = {k: v.copy() for k, v in s.items()}
        secs = self.lib.ref_euler(len(s["x"]), *[_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")],
                                  steps, dt, variant)
        return s, secs

    def ring_share(self, s, comm_sz, variant=None):
        variant = self.best_variant() if variant is None else variant
        return self.lib.ref_ring_share(len(s["x"]), _p(s["x"]), _p(s["y"]), _p(s["z"]), _p(s["m"]),
                                       comm_sz, variant)

    def kinetic(self, s):
        return self.lib.ref_kinetic(len(s["x"]), _p(s["vx"]), _p(s["vy"]), _p(s["vz"]), _p(s["m"]))

    def potential(self, s, variant=1):
        return self.lib.ref_potential(len(s["x"]), _p(s["x"]), _p(s["y"]), _p(s["z"]), _p(s["m"]), variant)

    def ring_init(self, n, R=1.0, omega=2 * np.pi, ratio=1e5):
        arrs = [np.zeros(n) for _ in range(10)]
        if self.lib.ref_ring_init(n, R, omega, ratio, *[_p(a) for a in arrs]) != 0:
            raise ValueError("ring needs n >= 2")
        keys = ("x", "y", "z", "vx", "vy", "vz", "m", "fx", "fy", "fz")
        return dict(zip(keys, arrs))

    def ring_predict(self, n, step, steps_per_rev, R=1.0, omega=2 * np.pi):
        arrs = [np.zeros(n) for _ in range(6)]
        self.lib.ref_ring_predict(n, R, omega, step, steps_per_rev, *[_p(a) for a in arrs])
        return dict(zip(("x", "y", "z", "vx", "vy", "vz"), arrs))

    def save_snapshot(self, directory, s, f, records, delta_t):
        """Writes `records` records of state s (forces f, (3, n)) with the
        reference's save_particles into directory/NBody_<n>.dat; returns the path."""
        n = len(s["x"])
        arr = [np.ascontiguousarray(a, dtype=np.float64) for a in
               (s["m"], s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], f[0], f[1], f[2])]
        rc = self.lib.ref_save_snapshot(str(directory).encode(), n, *[_p(a) for a in arr], records, delta_t)
        if rc != 0:
            raise OSError(f"ref_save_snapshot failed in {directory}")
        return os.path.join(str(directory), f"NBody_{n}.dat")

    def yoshida(self, order):
        c = np.zeros(16); d = np.zeros(16)
        k = self.lib.ref_yoshida(order, _p(c), _p(d))
        return c[:k].copy(), d[:k - 1].copy()


def reference_available() -> bool:
    name = "libnbr_ref_avx512.so" if cpu_has_avx512() else "libnbr_ref_avx.so"
    return os.path.exists(os.path.join(HERE, "_ref", name))

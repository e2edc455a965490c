"""ctypes binding of libnbr.so, the C ABI declared in include/nbr.h.

The product is the shared library; this module only marshals numpy arrays for
the tests and the benchmark.  There is no fallback: if libnbr.so is missing or
no sm_100 GPU is visible, the calls fail with NbrError.

State dictionaries use the keys x, y, z, vx, vy, vz, m (float64 arrays of one
length), the structure-of-arrays layout of the reference's NBody_system
(CPU/nbody_system.h:41-74).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# NBR_LIB_PATH selects another build of the library, e.g. libnbr_checked.so.
LIB_PATH = os.environ.get("NBR_LIB_PATH") or os.path.join(HERE, "libnbr.so")

NBR_OK = 0
STATUS = {0: "NBR_OK", 1: "NBR_ERR_INVALID_ARG", 2: "NBR_ERR_CUDA", 3: "NBR_ERR_NO_MEMORY",
          4: "NBR_ERR_TIMEOUT", 5: "NBR_ERR_NO_SYSTEM", 6: "NBR_ERR_UNSUPPORTED",
          7: "NBR_ERR_NONFINITE", 8: "NBR_ERR_IO",
          9: "NBR_ERR_BOUNDS"}
FP64, FP32C = 0, 1
KDK, DKD, EULER = 0, 1, 2
KEYS = ("x", "y", "z", "vx", "vy", "vz", "m")

_D = C.POINTER(C.c_double)
_SZ = C.c_size_t
_U64 = C.c_uint64


class NbrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Diag(C.Structure):
    _fields_ = [("T", C.c_double), ("U", C.c_double), ("E", C.c_double),
                ("P", C.c_double * 3), ("L", C.c_double * 3), ("M", C.c_double)]

    def as_dict(self):
        return {"T": self.T, "U": self.U, "E": self.E, "P": list(self.P), "L": list(self.L), "M": self.M}


class RunStats(C.Structure):
    _fields_ = [("force_evals", C.c_double), ("pairs", C.c_double), ("gpu_ms", C.c_double),
                ("kernels", C.c_double)]


_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads libnbr.so (raises FileNotFoundError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: build it with `make -C n-body-ring-solver_b200`")
    L = C.CDLL(path)
    P = C.POINTER(C.c_void_p)
    sig = {
        "nbr_ctx_create": ([C.c_int, P], C.c_int),
        "nbr_ctx_destroy": ([C.c_void_p], C.c_int),
        "nbr_last_error_string": ([C.c_void_p], C.c_char_p),
        "nbr_version": ([], C.c_int),
        "nbr_device_count": ([], C.c_int),
        "nbr_ctx_stream": ([C.c_void_p], C.c_void_p),
        "nbr_ctx_synchronize": ([C.c_void_p], C.c_int),
        "nbr_system_upload": ([C.c_void_p, _SZ] + [_D] * 7, C.c_int),
        "nbr_system_download": ([C.c_void_p] + [_D] * 6, C.c_int),
        "nbr_system_size": ([C.c_void_p], _SZ),
        "nbr_forces": ([C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, _D, _D, _D], C.c_int),
        "nbr_forces_device": ([C.c_void_p, C.c_int, C.c_double, C.c_double], C.c_int),
        "nbr_forces_download": ([C.c_void_p, _D, _D, _D], C.c_int),
        "nbr_accel_ij": ([C.c_void_p, C.c_int, _SZ, _D, _D, _D, _D, _SZ, _D, _D, _D, _D, C.c_double,
                          C.c_double, C.c_int, _D, _D, _D], C.c_int),
        "nbr_potential": ([C.c_void_p, C.c_double, C.c_double, _D, _D], C.c_int),
        "nbr_diagnostics": ([C.c_void_p, C.c_double, C.c_double, C.POINTER(Diag)], C.c_int),
        "nbr_run": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, _SZ, C.c_double, C.c_double,
                     C.POINTER(Diag), C.POINTER(RunStats)], C.c_int),
        "nbr_yoshida_coefficients": ([C.c_int, _D, _D], C.c_int),
        "nbr_set_force_config": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "nbr_get_force_config": ([C.c_void_p, C.c_int, C.c_double] + [C.POINTER(C.c_int)] * 3, C.c_int),
        "nbr_set_force_tiling": ([C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_int),
        "nbr_get_force_tiling": ([C.c_void_p, C.c_int, C.c_double] + [C.POINTER(C.c_int)] * 2, C.c_int),
        "nbr_autotune": ([C.c_void_p, C.c_int, C.c_double], C.c_int),
        "nbr_tune_cache_path": ([], C.c_char_p),
        "nbr_ic_plummer": ([_SZ, _U64] + [_D] * 7, C.c_int),
        "nbr_ic_uniform_ball": ([_SZ, _U64] + [_D] * 7, C.c_int),
        "nbr_ic_two_component": ([_SZ, _SZ, C.c_double, _U64] + [_D] * 7, C.c_int),
        "nbr_ic_ring": ([_SZ, C.c_double, C.c_double, C.c_double] + [_D] * 10, C.c_int),
        "nbr_ic_ring_predict": ([_SZ, C.c_double, C.c_double, _SZ, _SZ] + [_D] * 6, C.c_int),
        "nbr_ic_batch_sizes": ([_SZ, _U64, _SZ, _SZ, C.POINTER(_SZ)], C.c_int),
        "nbr_ic_system_seed": ([_U64, _SZ], _U64),
        "nbr_batch_upload": ([C.c_void_p, _SZ, C.POINTER(_SZ)] + [_D] * 7, C.c_int),
        "nbr_batch_download": ([C.c_void_p] + [_D] * 6, C.c_int),
        "nbr_batch_forces": ([C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, _D, _D, _D], C.c_int),
        "nbr_batch_run": ([C.c_void_p, C.c_int, C.c_double, _SZ, C.c_double, C.c_double,
                           C.POINTER(RunStats)], C.c_int),
        "nbr_batch_diagnostics": ([C.c_void_p, C.c_double, C.c_double, C.POINTER(Diag)], C.c_int),
        "nbr_batch_set_config": ([C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_int),
        "nbr_batch_autotune": ([C.c_void_p, C.c_int, C.c_double], C.c_int),
        "nbr_step_range": ([C.c_void_p, C.c_int, C.c_int, _SZ, _SZ, C.c_double, C.c_double, C.c_double,
                            C.c_double], C.c_int),
        "nbr_n3_slice_accel": ([C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                C.c_void_p, _SZ], C.c_int),
        "nbr_step_range_sum": ([C.c_void_p, C.c_int, C.c_int, _SZ, _SZ, C.c_double, C.c_double,
                                C.c_double, C.c_void_p, C.c_int, _SZ, _SZ], C.c_int),
        "nbr_n3_grid_plan": ([_SZ, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                              C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                              C.c_longlong], C.c_int),
        "nbr_state_pointers": ([C.c_void_p] + [C.POINTER(C.c_void_p)] * 6 + [C.POINTER(_SZ)], C.c_int),
        "nbr_state_changed": ([C.c_void_p], C.c_int),
        "nbr_snapshot_write_arrays": ([C.c_char_p, _SZ, _SZ, C.c_double] + [_D] * 10, C.c_int),
        "nbr_snapshot_save": ([C.c_void_p, C.c_char_p, _SZ, C.c_double], C.c_int),
        "nbr_snapshot_records": ([C.c_char_p, _SZ, C.POINTER(_SZ)], C.c_int),
        "nbr_snapshot_read_arrays": ([C.c_char_p, _SZ, _SZ, _D] + [_D] * 10, C.c_int),
        "nbr_snapshot_load": ([C.c_void_p, C.c_char_p, _SZ, _SZ, _D], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 C-contiguous arrays only"
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def device_count() -> int:
    return load().nbr_device_count()


def yoshida(order: int):
    c = np.zeros(16)
    d = np.zeros(16)
    k = load().nbr_yoshida_coefficients(order, _p(c), _p(d))
    if k == 0:
        raise ValueError(f"order {order} unsupported")
    return c[:k].copy(), d[:k - 1].copy()


# ----------------------------------------------------------------- snapshots --
SNAP_FIELDS = ("m", "x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz")


def snapshot_write(path: str, s: Dict[str, np.ndarray], time_step: int, delta_t: float,
                   forces: Optional[np.ndarray] = None):
    """One record in the reference's save_particles format (host arrays)."""
    n = len(s["x"])
    arr = {k: _f64(s[k]) for k in ("m", "x", "y", "z")}
    for k in ("vx", "vy", "vz"):
        arr[k] = _f64(s[k]) if s.get(k) is not None else None
    for d, k in enumerate(("fx", "fy", "fz")):
        arr[k] = _f64(forces[d]) if forces is not None else None
    _check(load().nbr_snapshot_write_arrays(str(path).encode(), n, time_step, delta_t,
                                            *[_p(arr[k]) for k in SNAP_FIELDS]), "snapshot_write")


def snapshot_records(path: str, n: int) -> int:
    out = _SZ()
    _check(load().nbr_snapshot_records(str(path).encode(), n, C.byref(out)), "snapshot_records")
    return int(out.value)


def snapshot_read(path: str, n: int, record: int) -> Dict[str, np.ndarray]:
    """Record `record` as a dict with t and the ten fields."""
    out = {k: np.zeros(n) for k in SNAP_FIELDS}
    t = C.c_double()
    _check(load().nbr_snapshot_read_arrays(str(path).encode(), n, record, C.byref(t),
                                           *[_p(out[k]) for k in SNAP_FIELDS]), "snapshot_read")
    out["t"] = t.value
    return out


# ------------------------------------------------------------------ samplers --
def _new_state(n: int) -> Dict[str, np.ndarray]:
    return {k: np.zeros(n) for k in KEYS}


def _check(rc: int, what: str, ctx=None):
    if rc != NBR_OK:
        L = load()
        msg = L.nbr_last_error_string(ctx).decode() if ctx is not None else L.nbr_last_error_string(None).decode()
        raise NbrError(rc, f"{what}: {msg}")


def plummer(n: int, seed: int) -> Dict[str, np.ndarray]:
    s = _new_state(n)
    _check(load().nbr_ic_plummer(n, seed, *[_p(s[k]) for k in KEYS]), "nbr_ic_plummer")
    return s


def uniform_ball(n: int, seed: int) -> Dict[str, np.ndarray]:
    s = _new_state(n)
    _check(load().nbr_ic_uniform_ball(n, seed, *[_p(s[k]) for k in KEYS]), "nbr_ic_uniform_ball")
    return s


def two_component(n: int, n_heavy: int, ratio: float, seed: int) -> Dict[str, np.ndarray]:
    s = _new_state(n)
    _check(load().nbr_ic_two_component(n, n_heavy, ratio, seed, *[_p(s[k]) for k in KEYS]),
           "nbr_ic_two_component")
    return s


def ring(n: int, R: float = 1.0, omega: float = 2 * np.pi, ratio: float = 1e5):
    s = _new_state(n)
    f = [np.zeros(n) for _ in range(3)]
    _check(load().nbr_ic_ring(n, R, omega, ratio, *[_p(s[k]) for k in KEYS], *[_p(a) for a in f]),
           "nbr_ic_ring")
    s["fx"], s["fy"], s["fz"] = f
    return s


def ring_predict(n: int, step: int, steps_per_rev: int, R: float = 1.0, omega: float = 2 * np.pi):
    arrs = [np.zeros(n) for _ in range(6)]
    _check(load().nbr_ic_ring_predict(n, R, omega, step, steps_per_rev, *[_p(a) for a in arrs]),
           "nbr_ic_ring_predict")
    return dict(zip(("x", "y", "z", "vx", "vy", "vz"), arrs))


def batch_sizes(nsys: int, seed: int, nmin: int = 64, nmax: int = 4096) -> np.ndarray:
    out = (_SZ * nsys)()
    _check(load().nbr_ic_batch_sizes(nsys, seed, nmin, nmax, out), "nbr_ic_batch_sizes")
    return np.array(out[:], dtype=np.int64)


def n3_grid_plan(n: int, sms: int = 148, nslices: int = 8, with_order: bool = False) -> dict:
    """The Newton-3 grid the library plans for n particles on `sms` SMs
    (nbr_n3_grid_plan; host only)."""
    cols, scols, ctas = C.c_int(), C.c_int(), C.c_longlong()
    eff = C.c_double()
    L = load()
    _check(L.nbr_n3_grid_plan(n, sms, nslices, C.byref(cols), C.byref(scols), C.byref(eff),
                              C.byref(ctas), None, 0), "nbr_n3_grid_plan")
    out = {"cols": cols.value, "slice_cols": scols.value, "efficiency": eff.value,
           "ctas": ctas.value}
    if with_order:
        buf = (C.c_int * ctas.value)()
        _check(L.nbr_n3_grid_plan(n, sms, nslices, None, None, None, None, buf, ctas.value),
               "nbr_n3_grid_plan")
        out["order"] = np.array(buf[:], dtype=np.int64)
    return out


def system_seed(seed: int, s: int) -> int:
    return int(load().nbr_ic_system_seed(seed, s))


def batch_plummer(nsys: int, seed: int, nmin: int = 64, nmax: int = 4096):
    """The batched workload: sizes log-uniform in [nmin, nmax], system s a
    Plummer sphere seeded by system_seed(seed, s).  Returns (offsets, state)."""
    sizes = batch_sizes(nsys, seed, nmin, nmax)
    off = np.zeros(nsys + 1, dtype=np.int64)
    off[1:] = np.cumsum(sizes)
    st = _new_state(int(off[-1]))
    for s in range(nsys):
        sub = plummer(int(sizes[s]), system_seed(seed, s))
        for k in KEYS:
            st[k][off[s]:off[s + 1]] = sub[k]
    return off, st


class _DeviceArray:
    """A float64 device array the library owns, exposed through
    __cuda_array_interface__ so torch can view it without a copy."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 2, "strides": None}


# ------------------------------------------------------------------- context --
def torch_float64():
    import torch
    return torch.float64


class Context:
    """One GPU context (its own CUDA stream); see include/nbr.h."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        rc = L.nbr_ctx_create(device, C.byref(h))
        _check(rc, "nbr_ctx_create")
        self.L = L
        self.h = h
        self.n = 0
        self.device = device

    def close(self):
        if self.h:
            self.L.nbr_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        _check(rc, what, self.h)

    @property
    def stream(self) -> int:
        return int(self.L.nbr_ctx_stream(self.h) or 0)

    def synchronize(self):
        self._chk(self.L.nbr_ctx_synchronize(self.h), "synchronize")

    # state
    def upload(self, s: Dict[str, np.ndarray]):
        arrs = {k: _f64(s[k]) for k in ("x", "y", "z", "m")}
        v = [_f64(s[k]) if k in s and s[k] is not None else None for k in ("vx", "vy", "vz")]
        n = len(arrs["x"])
        self._chk(self.L.nbr_system_upload(self.h, n, _p(arrs["x"]), _p(arrs["y"]), _p(arrs["z"]),
                                           *[_p(a) for a in v], _p(arrs["m"])), "upload")
        self.n = n

    def upload_raw(self, n, x, y, z, vx, vy, vz, m):
        """Upload from existing float64 arrays (no copies), e.g. pinned buffers."""
        self._chk(self.L.nbr_system_upload(self.h, n, _p(x), _p(y), _p(z), _p(vx), _p(vy), _p(vz), _p(m)),
                  "upload")
        self.n = n

    def download(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        n = self.L.nbr_system_size(self.h)
        out = out if out is not None else {k: np.zeros(n) for k in KEYS[:6]}
        self._chk(self.L.nbr_system_download(self.h, *[_p(out[k]) for k in KEYS[:6]]), "download")
        return out

    def download_raw(self, x, y, z, vx, vy, vz):
        self._chk(self.L.nbr_system_download(self.h, _p(x), _p(y), _p(z), _p(vx), _p(vy), _p(vz)),
                  "download")

    def forces(self, precision=FP64, G=1.0, eps2=0.0, want_force=False) -> np.ndarray:
        n = self.L.nbr_system_size(self.h)
        a = np.zeros((3, n))
        self._chk(self.L.nbr_forces(self.h, precision, G, eps2, int(want_force), _p(a[0]), _p(a[1]),
                                    _p(a[2])), "forces")
        return a

    def forces_device(self, precision=FP64, G=1.0, eps2=0.0):
        """Enqueues one force evaluation on the device (no host copies)."""
        self._chk(self.L.nbr_forces_device(self.h, precision, G, eps2), "forces_device")

    def forces_download(self) -> np.ndarray:
        n = self.L.nbr_system_size(self.h)
        a = np.zeros((3, n))
        self._chk(self.L.nbr_forces_download(self.h, _p(a[0]), _p(a[1]), _p(a[2])), "forces_download")
        return a

    def accel_ij(self, xi, yi, zi, xj, yj, zj, mj, mi=None, precision=FP64, G=1.0, eps2=0.0,
                 want_force=False) -> np.ndarray:
        xi, yi, zi = _f64(xi), _f64(yi), _f64(zi)
        xj, yj, zj, mj = _f64(xj), _f64(yj), _f64(zj), _f64(mj)
        mi = _f64(mi) if mi is not None else None
        a = np.zeros((3, len(xi)))
        self._chk(self.L.nbr_accel_ij(self.h, precision, len(xi), _p(xi), _p(yi), _p(zi), _p(mi), len(xj),
                                      _p(xj), _p(yj), _p(zj), _p(mj), G, eps2, int(want_force),
                                      _p(a[0]), _p(a[1]), _p(a[2])), "accel_ij")
        return a

    def potential(self, G=1.0, eps2=0.0, per_particle=False):
        n = self.L.nbr_system_size(self.h)
        phi = np.zeros(n) if per_particle else None
        U = C.c_double()
        self._chk(self.L.nbr_potential(self.h, G, eps2, _p(phi), C.byref(U)), "potential")
        return (U.value, phi) if per_particle else U.value

    def diagnostics(self, G=1.0, eps2=0.0) -> dict:
        d = Diag()
        self._chk(self.L.nbr_diagnostics(self.h, G, eps2, C.byref(d)), "diagnostics")
        return d.as_dict()

    def run(self, precision=FP64, scheme=KDK, order=2, dt=1e-3, steps=1, G=1.0, eps2=0.0, diag=False):
        d = (Diag * 2)()
        st = RunStats()
        self._chk(self.L.nbr_run(self.h, precision, scheme, order, dt, steps, G, eps2,
                                 d if diag else None, C.byref(st)), "run")
        out = {"force_evals": st.force_evals, "pairs": st.pairs, "gpu_ms": st.gpu_ms,
               "kernels": st.kernels}
        if diag:
            out["diag"] = (d[0].as_dict(), d[1].as_dict())
        return out

    # multi-GPU i-partition (see nbr_shard.py)
    def step_range(self, precision, scheme, i0, count, kick, drift, G=1.0, eps2=0.0):
        """One force evaluation of receivers [i0, i0 + count) with the fused
        kick/drift, asynchronous on the context's stream."""
        self._chk(self.L.nbr_step_range(self.h, precision, scheme, i0, count, kick, drift, G, eps2),
                  "step_range")

    def n3_slice_accel(self, precision, eps2, slice_, nslices, dst, slice_end=None):
        """Newton-3 partial accelerations of every particle from slices
        [slice_, slice_end) of `nslices` (slice_end: slice_ + 1 by default)
        into dst, a contiguous device tensor of shape (3, ld) for one slice or
        (slices, 3, ld) float64 (ld >= the padded size), asynchronous on the
        context's stream; the slices share one pair-kernel launch."""
        end = slice_ + 1 if slice_end is None else slice_end
        assert dst.dtype == torch_float64() and dst.is_contiguous()
        if dst.dim() == 2:
            assert end == slice_ + 1 and dst.shape[0] == 3
        else:
            assert dst.dim() == 3 and dst.shape[0] == end - slice_ and dst.shape[1] == 3
        ld = dst.stride(-2)
        self._chk(self.L.nbr_n3_slice_accel(self.h, precision, eps2, slice_, end, nslices,
                                            C.c_void_p(dst.data_ptr()), ld), "n3_slice_accel")

    def step_range_sum(self, precision, scheme, i0, count, kick, drift, G, src):
        """Kick/drift of receivers [i0, i0 + count) from the partial
        accelerations src (device tensor (nslices, 3, ld) float64, contiguous,
        receiver i0 + k at [:, :, k]) summed in slice order."""
        assert src.dtype == torch_float64() and src.is_contiguous() and src.dim() == 3
        self._chk(self.L.nbr_step_range_sum(self.h, precision, scheme, i0, count, kick, drift, G,
                                            C.c_void_p(src.data_ptr()), src.shape[0],
                                            src.stride(0), src.stride(1)), "step_range_sum")

    def state_pointers(self):
        """Device addresses of the current x, y, z, vx, vy, vz arrays and their length."""
        ptrs = [C.c_void_p() for _ in range(6)]
        ln = _SZ()
        self._chk(self.L.nbr_state_pointers(self.h, *[C.byref(p) for p in ptrs], C.byref(ln)),
                  "state_pointers")
        return dict(zip(KEYS[:6], [int(p.value or 0) for p in ptrs])), int(ln.value)

    def state_tensors(self):
        """The current x, y, z, vx, vy, vz as float64 torch tensors viewing
        the context's device memory (valid until the next upload; positions
        until the next step)."""
        import torch
        ptrs, ln = self.state_pointers()
        dev = torch.device("cuda", self.device)
        return {k: torch.as_tensor(_DeviceArray(p, ln), device=dev) for k, p in ptrs.items()}

    def state_changed(self):
        self._chk(self.L.nbr_state_changed(self.h), "state_changed")

    def snapshot_save(self, path, time_step, delta_t):
        self._chk(self.L.nbr_snapshot_save(self.h, str(path).encode(), time_step, delta_t),
                  "snapshot_save")

    def snapshot_load(self, path, n, record):
        t = C.c_double()
        self._chk(self.L.nbr_snapshot_load(self.h, str(path).encode(), n, record, C.byref(t)),
                  "snapshot_load")
        self.n = n
        return t.value

    def set_force_config(self, precision, ni=0, warps=0, split=0):
        self._chk(self.L.nbr_set_force_config(self.h, precision, ni, warps, split), "set_force_config")

    def get_force_config(self, precision, eps2=0.0):
        v = [C.c_int() for _ in range(3)]
        self._chk(self.L.nbr_get_force_config(self.h, precision, eps2, *[C.byref(x) for x in v]),
                  "get_force_config")
        return tuple(x.value for x in v)

    def set_force_tiling(self, precision, tile=0, unroll=0):
        """j-tile and unroll depth of a forced large-kernel configuration."""
        self._chk(self.L.nbr_set_force_tiling(self.h, precision, tile, unroll), "set_force_tiling")

    def get_force_tiling(self, precision, eps2=0.0):
        v = [C.c_int(), C.c_int()]
        self._chk(self.L.nbr_get_force_tiling(self.h, precision, eps2, *[C.byref(x) for x in v]),
                  "get_force_tiling")
        return tuple(x.value for x in v)

    def autotune(self, precision, eps2):
        self._chk(self.L.nbr_autotune(self.h, precision, eps2), "autotune")

    # batched
    def batch_upload(self, offsets, s):
        off = (_SZ * len(offsets))(*[int(v) for v in offsets])
        arrs = [_f64(s[k]) for k in KEYS]
        self._batch_keep = arrs
        self._chk(self.L.nbr_batch_upload(self.h, len(offsets) - 1, off, *[_p(a) for a in arrs]),
                  "batch_upload")
        self.batch_n = int(offsets[-1])
        self.nsys = len(offsets) - 1

    def batch_download(self):
        out = {k: np.zeros(self.batch_n) for k in KEYS[:6]}
        self._chk(self.L.nbr_batch_download(self.h, *[_p(out[k]) for k in KEYS[:6]]), "batch_download")
        return out

    def batch_forces(self, precision=FP64, G=1.0, eps2=0.0, want_force=False):
        a = np.zeros((3, self.batch_n))
        self._chk(self.L.nbr_batch_forces(self.h, precision, G, eps2, int(want_force), _p(a[0]),
                                          _p(a[1]), _p(a[2])), "batch_forces")
        return a

    def batch_run(self, precision=FP64, dt=1e-3, steps=1, G=1.0, eps2=0.0):
        st = RunStats()
        self._chk(self.L.nbr_batch_run(self.h, precision, dt, steps, G, eps2, C.byref(st)), "batch_run")
        return {"force_evals": st.force_evals, "pairs": st.pairs, "gpu_ms": st.gpu_ms,
                "kernels": st.kernels}

    def batch_set_config(self, precision, wide=-1, ctas_per_sm=0):
        """Work list of the batched kernel: 0 one-tile items, 1 two-tile items,
        2 Newton-3 row blocks for the larger systems (the default), -1 back to
        the autotune cache or the default; ctas_per_sm 0 = occupancy limit."""
        self._chk(self.L.nbr_batch_set_config(self.h, precision, wide, ctas_per_sm), "batch_set_config")

    def batch_autotune(self, precision, eps2=0.0):
        self._chk(self.L.nbr_batch_autotune(self.h, precision, eps2), "batch_autotune")

    def batch_diagnostics(self, G=1.0, eps2=0.0):
        d = (Diag * self.nsys)()
        self._chk(self.L.nbr_batch_diagnostics(self.h, G, eps2, d), "batch_diagnostics")
        return [d[i].as_dict() for i in range(self.nsys)]

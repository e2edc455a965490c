"""Drives the bounds-checked library build (libnbr_checked.so, selected with
NBR_LIB_PATH) through every kernel at edge sizes and prints one JSON line:
the number of calls made and the results of a few of them for comparison with
the normal build.  Any kernel index outside its array makes a call fail with
NBR_ERR_BOUNDS, which ends the script with a non-zero status.  Used by
tests/test_gpu_checked.py."""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..",
                                "n-body-ring-solver_b200"))
import nbr  # noqa: E402

FP64, FP32C = nbr.FP64, nbr.FP32C
calls = 0
out = {}
with nbr.Context(0) as ctx:
    for n in (1, 2, 31, 127, 128, 129, 1000, 4097, 33000):
        s = nbr.plummer(n, 3)
        ctx.upload(s)
        for prec in (FP64, FP32C):
            for eps2 in (0.0, 1e-6):
                a = ctx.forces(prec, eps2=eps2)
                calls += 1
                out[f"forces_{n}_{prec}_{eps2}"] = float(np.abs(a).sum())
            for cfg in ((4, 2, 1), (8, 4, 3), (4, 8, 64)):
                ctx.set_force_config(prec, *cfg)
                ctx.forces(prec, eps2=1e-6)
                calls += 1
            ctx.set_force_config(prec, 0)
        U = ctx.potential(eps2=1e-6)
        d = ctx.diagnostics(eps2=1e-6)
        calls += 2
        out[f"U_{n}"] = U
        for scheme, order in ((nbr.KDK, 2), (nbr.DKD, 4), (nbr.EULER, 2)):
            ctx.upload(s)
            ctx.run(FP32C, scheme, order, 1e-4, 3, eps2=1e-6)
            ctx.run(FP64, scheme, order, 1e-4, 2, eps2=1e-6)
            calls += 2
        if n >= 256:  # receiver ranges of the multi-GPU partition
            ctx.upload(s)
            for i0, cnt in ((0, 128), (128, n), (n - n % 128 if n % 128 else n - 128, 128)):
                ctx.step_range(FP32C, nbr.KDK, i0, cnt, 1e-4, 1e-4, 1.0, 1e-6)
                ctx.state_changed()
                calls += 1
            ctx.synchronize()
        ai = ctx.accel_ij(s["x"][: max(1, n // 2)], s["y"][: max(1, n // 2)], s["z"][: max(1, n // 2)],
                          s["x"], s["y"], s["z"], s["m"], precision=FP32C, eps2=1e-6)
        calls += 1
    sizes = [1, 2, 3, 16, 17, 33, 64, 65, 127, 128, 129, 255, 256, 257, 700]
    off = np.concatenate([[0], np.cumsum(sizes)])
    st = {k: np.concatenate([nbr.plummer(m, 20 + i)[k] for i, m in enumerate(sizes)]) for k in nbr.KEYS}
    ctx.batch_upload(off, st)
    for prec in (FP64, FP32C):
        for wide in (0, 1, 2):
            ctx.batch_set_config(prec, wide, 0)
            a = ctx.batch_forces(prec, eps2=1e-6)
            ctx.batch_run(prec, dt=1e-4, steps=2, eps2=1e-6)
            calls += 2
            out[f"batch_{prec}_{wide}"] = float(np.abs(a).sum())
    ctx.batch_diagnostics(eps2=1e-6)
    calls += 1
# the no-allocation entry point: its scratch regions inside the static array
# are checked against their own lengths
import ctypes as C  # noqa: E402
import torch  # noqa: E402
lib = nbr.load()
fna = lib.nbr_forces_noalloc
fna.argtypes = [C.c_int, C.c_size_t] + [C.c_void_p] * 4 + [C.c_double, C.c_double] + [C.c_void_p] * 4
fna.restype = C.c_int
for n in (1, 128, 1025, 32768):
    s = nbr.plummer(n, 50 + n)
    dev = {k: torch.from_numpy(s[k]).cuda() for k in ("x", "y", "z", "m")}
    for prec in (FP64, FP32C):
        a = torch.zeros((3, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = fna(prec, n, dev["x"].data_ptr(), dev["y"].data_ptr(), dev["z"].data_ptr(),
                 dev["m"].data_ptr(), 1.0, 1e-6, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(),
                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc != 0:
            raise SystemExit(f"nbr_forces_noalloc n={n} prec={prec}: status {rc}: "
                             f"{lib.nbr_last_error_string(None)}")
        calls += 1
        out[f"noalloc_{n}_{prec}"] = float(a.abs().sum().item())
print(json.dumps({"calls": calls, "results": out}))

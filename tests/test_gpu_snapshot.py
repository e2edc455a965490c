"""Checkpoint / resume through the C ABI and the CLI, on the GPU.

nbr_snapshot_save writes the context's state in the reference's
save_particles format (checked byte-for-byte against the reference on the
host in test_snapshot.py); nbr_snapshot_load resumes from any record.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu
FP64, KDK = 0, 0


def test_save_records_state_and_forces(ctx, nbr, tmp_path):
    n, dt, eps2 = 3000, 1e-3, 1e-6
    s = nbr.plummer(n, 4)
    ctx.upload(s)
    p = tmp_path / "NBody_3000.dat"
    ctx.snapshot_save(p, 0, dt)  # no accelerations yet: forces are zeros
    a0 = ctx.forces(FP64, eps2=eps2)
    ctx.snapshot_save(p, 1, dt)  # after nbr_forces: m a of the current positions
    ctx.run(FP64, KDK, 2, dt, 3, eps2=eps2)
    ctx.snapshot_save(p, 4, dt)
    acc = ctx.forces_download()
    state = ctx.download()
    assert nbr.snapshot_records(p, n) == 3
    r0, r1, r2 = (nbr.snapshot_read(p, n, k) for k in range(3))
    assert (r0["t"], r1["t"], r2["t"]) == (0.0, dt, 4 * dt)
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(r0[k], s[k])
    assert not r0["fx"].any()
    for d, k in enumerate(("fx", "fy", "fz")):
        np.testing.assert_array_equal(r1[k], s["m"] * a0[d])
        np.testing.assert_array_equal(r2[k], s["m"] * acc[d])
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(r2[k], state[k])


def test_resume_continues_the_run(nbr, tmp_path):
    n, dt, eps2 = 2048, 1e-3, 1e-6
    s = nbr.plummer(n, 5)
    p = tmp_path / "ck.dat"
    with nbr.Context(0) as a:
        a.upload(s)
        a.run(FP64, KDK, 2, dt, 4, eps2=eps2)
        a.snapshot_save(p, 4, dt)
        a.run(FP64, KDK, 2, dt, 3, eps2=eps2)
        want = a.download()
    with nbr.Context(0) as b:
        t = b.snapshot_load(p, n, 0)
        assert t == 4 * dt
        b.run(FP64, KDK, 2, dt, 3, eps2=eps2)
        got = b.download()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_allclose(got[k], want[k], rtol=0, atol=1e-14 * np.abs(want[k]).max())


def test_cli_save_and_resume(tmp_path):
    exe = os.path.join(PKG, "nbr_main")
    args = ["-t", "gpu", "-N", "1000", "-i", "lf", "-scheme", "kdk", "-ic", "plummer", "-seed", "1",
            "-eps", "1e-3", "-dt", "1e-3"]
    out = subprocess.run([exe, *args, "-s", "20", "-save", "5"], capture_output=True, text=True,
                         cwd=tmp_path, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    p = tmp_path / "NBody_1000.dat"
    raw = np.fromfile(p, dtype=np.float64).reshape(-1, 1 + 10 * 1000)
    np.testing.assert_allclose(raw[:, 0], [0, 5e-3, 10e-3, 15e-3, 20e-3], rtol=1e-15)
    out = subprocess.run([exe, *args, "-s", "10", "-save", "10", "-resume", str(p)],
                         capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "Resumed from" in out.stdout
    raw = np.fromfile(p, dtype=np.float64).reshape(-1, 1 + 10 * 1000)
    assert raw.shape[0] == 6 and abs(raw[-1, 0] - 30e-3) < 1e-15

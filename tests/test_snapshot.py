"""Snapshot files in the reference's save_particles format (host side, no GPU).

The writer must produce the same bytes as the reference's own
NBody_system::save_particles (CPU/nbody_system.cpp:133-152), compiled from
its sources into oracle/_ref, on the same arrays.
"""
import numpy as np
import pytest


def _state(n, seed):
    rng = np.random.default_rng(seed)
    s = {k: rng.standard_normal(n) for k in ("x", "y", "z", "vx", "vy", "vz")}
    s["m"] = rng.uniform(0.1, 1.0, n)
    f = rng.standard_normal((3, n))
    return s, f


def test_bytes_match_reference_save_particles(nbr, reference, tmp_path):
    n, dt = 1000, 0.015625 / 3
    s, f = _state(n, 1)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    ref_path = reference.save_snapshot(ref_dir, s, f, 3, dt)
    ours = tmp_path / "ours.dat"
    for t in range(3):
        nbr.snapshot_write(ours, s, t, dt, forces=f)
    a, b = open(ref_path, "rb").read(), open(ours, "rb").read()
    assert len(a) == 3 * (8 + 80 * n)
    assert a == b


def test_layout_and_round_trip(nbr, tmp_path):
    n, dt = 300, 1e-3
    s, f = _state(n, 2)
    p = tmp_path / "snap.dat"
    nbr.snapshot_write(p, s, 0, dt, forces=f)
    s2 = {k: v * 2 for k, v in s.items()}
    nbr.snapshot_write(p, s2, 7, dt)  # no forces: zeros
    raw = np.fromfile(p, dtype=np.float64)
    assert raw.size == 2 * (1 + 10 * n)
    rec = raw[: 1 + 10 * n]
    assert rec[0] == 0.0
    for i, k in enumerate(("m", "x", "y", "z", "vx", "vy", "vz")):
        np.testing.assert_array_equal(rec[1 + i * n:1 + (i + 1) * n], s[k])
    np.testing.assert_array_equal(rec[1 + 7 * n:], f.reshape(-1))
    assert nbr.snapshot_records(p, n) == 2
    r1 = nbr.snapshot_read(p, n, 1)
    assert r1["t"] == 7 * dt
    for k in ("m", "x", "vz"):
        np.testing.assert_array_equal(r1[k], s2[k])
    assert not r1["fx"].any() and not r1["fz"].any()
    # time step 0 truncates
    nbr.snapshot_write(p, s, 0, dt)
    assert nbr.snapshot_records(p, n) == 1


def test_snapshot_errors(nbr, tmp_path):
    n = 100
    s, _ = _state(n, 3)
    p = tmp_path / "e.dat"
    nbr.snapshot_write(p, s, 0, 1.0)
    with pytest.raises(nbr.NbrError) as e:
        nbr.snapshot_records(p, n + 1)  # not a whole number of records
    assert e.value.status == 1
    with pytest.raises(nbr.NbrError) as e:
        nbr.snapshot_read(p, n, 1)  # only record 0 exists
    assert e.value.status == 1
    with pytest.raises(nbr.NbrError) as e:
        nbr.snapshot_records(tmp_path / "missing.dat", n)
    assert e.value.status == 8
    with pytest.raises(nbr.NbrError) as e:
        nbr.snapshot_write(tmp_path / "no_such_dir" / "x.dat", s, 0, 1.0)
    assert e.value.status == 8

"""Pins the CPU oracle (oracle/nbr_oracle.c) before anything is checked against it.

Three anchors, all unsoftened because the reference has no softening:
  * golden fixtures produced by the reference's own CPU solver
    (tests/golden/make_golden.py, built from the reference sources);
  * the same solver called live where oracle/_ref was built;
  * the reference's formula-generated known answers: analytic ring forces
    (CPU/nbody_system.cpp:319-384) and the rigid rotation (:386-408).
"""
import numpy as np
import pytest

from conftest import golden, rel_err, state_copy

KEYS6 = ("x", "y", "z", "vx", "vy", "vz")


def _split(fx):
    return {k[3:]: v for k, v in fx.items() if k.startswith("in_")}, \
           {k[4:]: v for k, v in fx.items() if k.startswith("out_")}


@pytest.mark.parametrize("name", ["ref_forces_random_n1000.npz", "ref_forces_plummer_n2048.npz"])
def test_oracle_forces_match_reference_golden(oracle, name):
    g = golden(name)
    a = oracle.accel(g["x"], g["y"], g["z"], g["m"], G=1.0, eps2=0.0)
    F = a * g["m"]
    for key in [k for k in g if k.startswith("F_")]:
        err = rel_err(F, g[key])
        assert err.max() < 1e-13, (key, err.max())


def test_oracle_extended_precision_agrees(oracle):
    g = golden("ref_forces_random_n1000.npz")
    a = oracle.accel(g["x"], g["y"], g["z"], g["m"])
    al = oracle.accel(g["x"], g["y"], g["z"], g["m"], extended=True)
    assert rel_err(a, al).max() < 1e-14


def test_oracle_ring_known_answer(oracle):
    g = golden("ref_ring_n1001.npz")
    a = oracle.accel(g["x"], g["y"], g["z"], g["m"])
    F = a * g["m"]
    # Ring particles: exact circular-orbit force; central particle: zero by symmetry.
    err = rel_err(F[:, :-1], g["F_analytic"][:, :-1])
    assert err.max() < 1e-11, err.max()
    assert np.abs(F[:, -1]).max() < 1e-9 * np.abs(g["F_analytic"]).max()
    assert rel_err(F[:, :-1], g["F_simple"][:, :-1]).max() < 1e-13


def test_oracle_ring_init_matches_reference(oracle):
    g = golden("ref_ring_n1001.npz")
    r = oracle.ring_init(1001, ratio=1e5)
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(r[k], g[k])
    np.testing.assert_array_equal(np.stack([r["fx"], r["fy"], r["fz"]]), g["F_analytic"])
    p = golden("ref_ring_predict_n101_s7_of100.npz")
    q = oracle.ring_predict(101, 7, 100)
    for k in KEYS6:
        np.testing.assert_allclose(q[k], p[k], rtol=0, atol=1e-15)


def test_oracle_energy_matches_reference(oracle):
    g = golden("ref_energy_plummer_n2048.npz")
    e = oracle.energy(g, G=1.0, eps2=0.0)
    assert abs(e["T"] - g["T"]) <= 1e-14 * abs(g["T"])
    assert abs(e["U"] - g["U_scalar"]) <= 1e-13 * abs(g["U_scalar"])
    assert abs(e["U"] - g["U_avx2"]) <= 1e-13 * abs(g["U_avx2"])


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_oracle_dkd_matches_reference_lf(oracle, order):
    g = golden(f"ref_lf_order{order}_plummer_n256.npz")
    s_in, s_out = _split(g)
    got = oracle.dkd(s_in, float(g["dt"]), int(g["steps"]), order=order, eps2=0.0)
    for k in KEYS6:
        scale = np.abs(s_out[k]).max()
        assert np.abs(got[k] - s_out[k]).max() <= 1e-12 * scale, (k, np.abs(got[k] - s_out[k]).max())


def test_yoshida_tables_match_reference(oracle, nbr):
    g = golden("ref_yoshida.npz")
    for o in (2, 4, 6, 8):
        c, d = oracle.yoshida(o)
        np.testing.assert_array_equal(c, g[f"c{o}"])
        np.testing.assert_array_equal(d, g[f"d{o}"])
        c2, d2 = nbr.yoshida(o)
        np.testing.assert_array_equal(c2, g[f"c{o}"])
        np.testing.assert_array_equal(d2, g[f"d{o}"])
        assert abs(c.sum() - 1) < 1e-14 and abs(d.sum() - 1) < 1e-14


def test_oracle_kdk_is_second_order_and_conservative(oracle, nbr):
    s = nbr.plummer(256, 3)
    eps2 = 1e-4
    e0 = oracle.energy(s, eps2=eps2)["E"]
    drift = []
    for dt, steps in ((2e-3, 50), (1e-3, 100)):
        out = oracle.kdk(s, dt, steps, eps2=eps2)
        drift.append(abs(oracle.energy(out, eps2=eps2)["E"] - e0))
    # halving dt at fixed end time cuts the energy error by about 4
    assert drift[1] < drift[0] / 2.5


def test_oracle_kdk_equals_dkd_structure(oracle, nbr):
    """KDK and order-2 DKD are both second order: trajectories agree to O(dt^2)."""
    s = nbr.plummer(128, 9)
    a = oracle.kdk(s, 1e-4, 20, eps2=1e-4)
    b = oracle.dkd(s, 1e-4, 20, order=2, eps2=1e-4)
    for k in ("x", "y", "z"):
        assert np.abs(a[k] - b[k]).max() < 1e-6


# ---- live reference (only where oracle/_ref was built from the sources) ----
def test_oracle_matches_live_reference_all_kernels(oracle, reference, nbr):
    from oracle import REF_AVX2, REF_AVX2_BLOCKED, REF_AVX512_RSQRT, REF_AVX512_RSQRT_4I, REF_SIMPLE
    s = nbr.plummer(777, 21)
    a = oracle.accel(s["x"], s["y"], s["z"], s["m"])
    variants = [REF_SIMPLE, REF_AVX2, REF_AVX2_BLOCKED]
    if reference.has_avx512:
        variants += [REF_AVX512_RSQRT, REF_AVX512_RSQRT_4I]
    for v in variants:
        F = reference.forces(s["x"], s["y"], s["z"], s["m"], v)
        assert rel_err(a * s["m"], F).max() < 1e-12, v


def test_oracle_dkd_matches_live_reference(oracle, reference, nbr):
    r = nbr.ring(301, ratio=1e3)
    s = {k: r[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    out, _ = reference.lf(s, 1e-3, 20, order=4)
    got = oracle.dkd(s, 1e-3, 20, order=4)
    for k in KEYS6:
        assert np.abs(got[k] - out[k]).max() <= 1e-12 * max(1.0, np.abs(out[k]).max())


def test_golden_fixtures_reproduce(reference):
    """The committed fixtures are what the reference computes today."""
    g = golden("ref_forces_random_n1000.npz")
    from oracle import REF_SIMPLE
    F = reference.forces(g["x"], g["y"], g["z"], g["m"], REF_SIMPLE)
    np.testing.assert_array_equal(F, g["F_simple"])


def test_oracle_euler_matches_reference_golden(oracle):
    g = golden("ref_euler_plummer_n256.npz")
    s_in, s_out = _split(g)
    got = oracle.euler(s_in, float(g["dt"]), int(g["steps"]))
    for k in KEYS6:
        assert np.abs(got[k] - s_out[k]).max() <= 1e-12 * np.abs(s_out[k]).max(), k


def test_oracle_subset_matches_full(oracle, nbr):
    s = nbr.plummer(3000, 8)
    idx = np.array([0, 5, 1234, 2999])
    full = oracle.accel(s["x"], s["y"], s["z"], s["m"], eps2=1e-6, extended=True)
    sub = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=1e-6)
    np.testing.assert_array_equal(sub, full[:, idx])


@pytest.mark.parametrize("kind, args", [("plummer", (2048, 0)), ("plummer", (262144, 2)),
                                        ("plummer", (1000, 7)), ("uniform_ball", (32768, 1)),
                                        ("two_component", (131072, 1311, 1000.0, 4))])
def test_oracle_samplers_are_bit_identical_to_the_products(oracle, nbr, kind, args):
    """The oracle's samplers build the benchmark inputs in processes that must
    not load the product (the timed reference arm); they must give exactly
    the product's inputs."""
    a = getattr(oracle, kind)(*args)
    b = getattr(nbr, kind)(*args)
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        assert np.array_equal(a[k], b[k]), k

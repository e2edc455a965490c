"""Generates the golden fixtures in this directory from the reference itself.

The reference ships no golden vectors (its checks are formula-generated,
CPU/nbody_system.cpp:319-408).  This script runs the reference's own CPU solver,
compiled from its sources by oracle/Makefile into oracle/_ref/, on seeded
inputs and stores inputs and outputs together, so the fixtures are
self-contained and usable where the reference is absent (the GPU box).

    make -C oracle ref && python tests/golden/make_golden.py

Every fixture is unsoftened (the reference has no softening) and in the
reference's force form (F = m a) where it stores forces.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "n-body-ring-solver_b200"))

from oracle import (REF_AVX2_BLOCKED, REF_AVX512_RSQRT_4I, REF_SIMPLE,  # noqa: E402
                    Reference)


def plummer_np(n, seed):
    """Plummer positions/velocities from numpy's PCG64 (inputs only; the
    product's own sampler is tested separately)."""
    rng = np.random.default_rng(seed)
    a = 3 * np.pi / 16
    X = 0.999 * rng.uniform(1e-12, 1.0, n)
    r = a / np.sqrt(X ** (-2 / 3) - 1)
    c = 1 - 2 * rng.uniform(size=n)
    ph = 2 * np.pi * rng.uniform(size=n)
    s = np.sqrt(1 - c * c)
    x, y, z = r * s * np.cos(ph), r * s * np.sin(ph), r * c
    v = 0.5 * np.sqrt(2 / a) * (1 + r * r / a / a) ** -0.25 * rng.uniform(0.2, 0.9, n)
    c = 1 - 2 * rng.uniform(size=n)
    ph = 2 * np.pi * rng.uniform(size=n)
    s = np.sqrt(1 - c * c)
    st = {"x": x - x.mean(), "y": y - y.mean(), "z": z - z.mean(),
          "vx": v * s * np.cos(ph), "vy": v * s * np.sin(ph), "vz": v * c, "m": np.full(n, 1.0 / n)}
    for k in ("vx", "vy", "vz"):
        st[k] = st[k] - st[k].mean()
    return st


def main():
    ref = Reference()
    out = {}

    rng = np.random.default_rng(11)
    n = 1000
    x, y, z = rng.uniform(-1, 1, (3, n))
    m = rng.uniform(0.5, 1.5, n)
    rec = {"x": x, "y": y, "z": z, "m": m,
           "F_simple": ref.forces(x, y, z, m, REF_SIMPLE),
           "F_avx2_blocked": ref.forces(x, y, z, m, REF_AVX2_BLOCKED)}
    if ref.has_avx512:
        rec["F_avx512_rsqrt_4i"] = ref.forces(x, y, z, m, REF_AVX512_RSQRT_4I)
    out["ref_forces_random_n1000.npz"] = rec

    s = plummer_np(2048, 7)
    out["ref_forces_plummer_n2048.npz"] = {
        "x": s["x"], "y": s["y"], "z": s["z"], "m": s["m"],
        "F_simple": ref.forces(s["x"], s["y"], s["z"], s["m"], REF_SIMPLE),
        "F_avx2_blocked": ref.forces(s["x"], s["y"], s["z"], s["m"], REF_AVX2_BLOCKED)}
    out["ref_energy_plummer_n2048.npz"] = {
        **s, "T": np.array(ref.kinetic(s)), "U_scalar": np.array(ref.potential(s, 0)),
        "U_avx2": np.array(ref.potential(s, 1))}

    r = ref.ring_init(1001, ratio=1e5)
    out["ref_ring_n1001.npz"] = {**{k: r[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")},
                                 "F_analytic": np.stack([r["fx"], r["fy"], r["fz"]]),
                                 "F_simple": ref.forces(r["x"], r["y"], r["z"], r["m"], REF_SIMPLE)}
    p = ref.ring_predict(101, 7, 100)
    out["ref_ring_predict_n101_s7_of100.npz"] = p

    s = plummer_np(256, 5)
    for order, steps in ((2, 10), (4, 4), (6, 2), (8, 1)):
        after, _ = ref.lf(s, 1e-4, steps, order)
        out[f"ref_lf_order{order}_plummer_n256.npz"] = {
            **{"in_" + k: v for k, v in s.items()},
            **{"out_" + k: after[k] for k in ("x", "y", "z", "vx", "vy", "vz")},
            "dt": np.array(1e-4), "steps": np.array(steps), "order": np.array(order)}
    after, _ = ref.euler(s, 1e-4, 10, REF_AVX2_BLOCKED)
    out["ref_euler_plummer_n256.npz"] = {
        **{"in_" + k: v for k, v in s.items()},
        **{"out_" + k: after[k] for k in ("x", "y", "z", "vx", "vy", "vz")},
        "dt": np.array(1e-4), "steps": np.array(10)}
    out["ref_yoshida.npz"] = {f"c{o}": ref.yoshida(o)[0] for o in (2, 4, 6, 8)}
    out["ref_yoshida.npz"].update({f"d{o}": ref.yoshida(o)[1] for o in (2, 4, 6, 8)})

    for name, arrays in out.items():
        np.savez_compressed(os.path.join(HERE, name), **arrays)
        print("wrote", name)


if __name__ == "__main__":
    main()

"""CPU-side checks of the C ABI: the library loads and exports every declared
symbol, host-only entry points (samplers, coefficients) behave, and without a
GPU the compute entry points fail loudly instead of falling back."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG, REFERENCE_CPU, ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(nbr_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_functions():
    names = declared_functions()
    assert "nbr_forces" in names and "nbr_run" in names and len(names) >= 30


def test_library_exports_every_declared_symbol(nbr):
    lib = ctypes.CDLL(nbr.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_device_count(nbr):
    L = nbr.load()
    assert L.nbr_version() >= 1000
    assert L.nbr_device_count() >= 0


def test_no_gpu_fails_loudly(nbr):
    if nbr.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(nbr.NbrError) as ei:
        nbr.Context(0)
    assert ei.value.status == 6  # NBR_ERR_UNSUPPORTED


def test_null_context_is_rejected(nbr):
    L = nbr.load()
    assert L.nbr_forces(None, 0, 1.0, 0.0, 0, None, None, None) == 1
    assert L.nbr_run(None, 0, 0, 2, 1e-3, 1, 1.0, 0.0, None, None) == 1
    assert L.nbr_ctx_destroy(None) == 0
    assert b"NULL" in L.nbr_last_error_string(None)


# ------------------------------------------------------------------ samplers --
def test_plummer_deterministic(nbr):
    a = nbr.plummer(1000, 42)
    b = nbr.plummer(1000, 42)
    c = nbr.plummer(1000, 43)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert not np.array_equal(a["x"], c["x"])


def test_plummer_statistics(nbr, oracle):
    s = nbr.plummer(20000, 0)
    assert abs(s["m"].sum() - 1.0) < 1e-12
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert abs(np.dot(s["m"], s[k])) < 1e-12
    e = oracle.energy(s, eps2=0.0)
    # N-body units: E = -1/4 for the full model; the 0.999 mass cut changes it slightly.
    assert abs(e["E"] + 0.25) < 0.01
    assert abs(2 * e["T"] / abs(e["U"]) - 1.0) < 0.03
    r = np.sqrt(s["x"] ** 2 + s["y"] ** 2 + s["z"] ** 2)
    a = 3 * np.pi / 16
    r_half = a / np.sqrt(0.5 ** (-2 / 3) - 1)
    assert abs(np.median(r) / r_half - 1) < 0.03


def test_uniform_ball(nbr):
    s = nbr.uniform_ball(20000, 1)
    r = np.sqrt(s["x"] ** 2 + s["y"] ** 2 + s["z"] ** 2)
    assert r.max() <= 1.0
    assert abs((r < 0.5).mean() - 0.125) < 0.01
    assert np.all(s["vx"] == 0) and np.all(s["m"] == 1.0 / 20000)


def test_two_component(nbr):
    n, nh = 131072, 1311
    s = nbr.two_component(n, nh, 1000.0, 4)
    m = s["m"]
    assert abs(m.sum() - 1.0) < 1e-12
    assert np.all(m[:nh] == m[0]) and np.all(m[nh:] == m[-1])
    assert abs(m[0] / m[-1] - 1000.0) < 1e-9
    assert abs(m[-1] - 1.0 / (n - nh + 1000 * nh)) < 1e-20


def test_batch_sizes(nbr):
    sz = nbr.batch_sizes(4096, 3)
    assert sz.min() >= 64 and sz.max() <= 4096
    # log-uniform: median near sqrt(64 * 4096) = 512
    assert 400 < np.median(sz) < 650
    assert 3.5e6 < sz.sum() < 4.5e6
    assert nbr.system_seed(3, 0) != nbr.system_seed(3, 1)


def test_ring_matches_reference_golden(nbr):
    from conftest import golden
    g = golden("ref_ring_n1001.npz")
    r = nbr.ring(1001, ratio=1e5)
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(r[k], g[k])
    np.testing.assert_array_equal(np.stack([r["fx"], r["fy"], r["fz"]]), g["F_analytic"])
    p = golden("ref_ring_predict_n101_s7_of100.npz")
    q = nbr.ring_predict(101, 7, 100)
    for k in q:
        np.testing.assert_allclose(q[k], p[k], rtol=0, atol=1e-15)


def test_sampler_argument_errors(nbr):
    with pytest.raises(nbr.NbrError):
        nbr.plummer(0, 1)
    with pytest.raises(nbr.NbrError):
        nbr.ring(1)
    with pytest.raises(nbr.NbrError):
        nbr.two_component(10, 11, 1000.0, 1)


def test_adapter_header_compiles_with_reference_layout(tmp_path):
    """compute_forces_gpu binds to a type with NBody_system's members."""
    src = tmp_path / "t.cpp"
    src.write_text(
        '#include "nbr_compute_forces.hpp"\n'
        "struct Sys { size_t N; double* mass; double* pos[3]; double* vel[3]; double* force[3];\n"
        "             static constexpr double G = 1; };\n"
        "void f(Sys& s, double* rp[3], double* rf[3]) { compute_forces_gpu(s, rp, rf, nullptr, nullptr, 4, 0, 1, 0, 1); }\n")
    out = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_adapter_compiles_against_reference_header(tmp_path):
    ref = REFERENCE_CPU
    if not os.path.isdir(ref):
        pytest.skip("reference sources not present")
    src = tmp_path / "t.cpp"
    src.write_text(
        '#include "nbody_system.h"\n#include "nbr_compute_forces.hpp"\n'
        "void f(NBody_system& s, double* rp[3], double* rf[3], double*** lf, double*** lrf) {\n"
        "  compute_forces_gpu(s, rp, rf, lf, lrf, s.N, 0, 1, 0, 1); }\n")
    out = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                          "-I", ref, str(src)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_cli_without_gpu_reports_and_fails():
    exe = os.path.join(PKG, "nbr_main")
    if not os.path.exists(exe):
        pytest.skip("nbr_main not built")
    import nbr as mod
    if mod.device_count() > 0:
        pytest.skip("a GPU is visible")
    out = subprocess.run([exe, "-N", "100", "-s", "1"], capture_output=True, text=True)
    assert out.returncode == 1 and "No GPU context" in out.stdout


def _n3_costs(nb, cols):
    """The grid model's CTA costs, group-major (a restatement of the model:
    0.15 per CTA plus 1 per column block, 0.8 for a row group's first 8)."""
    out = []
    for r0 in range(0, nb, 8):
        cs = r0
        while cs < nb:
            ce = min(cs + cols, nb)
            diag = max(0, min(ce, r0 + 8) - cs)
            out.append(0.15 + 0.8 * diag + (ce - cs - diag))
            cs += cols
    return out


@pytest.mark.parametrize("n", [1, 300, 20000, 32768, 131072, 262144, 1048576])
def test_n3_grid_plan_invariants(nbr, n):
    """The Newton-3 grid plan (host only): widths within 1 .. 32, the CTA
    count of that width, a launch order that is a permutation of the CTAs
    with non-increasing modeled cost, an efficiency in (0, 1], and the same
    answer on a second call."""
    plan = nbr.n3_grid_plan(n, 148, 8, with_order=True)
    assert 1 <= plan["cols"] <= 32 and 1 <= plan["slice_cols"] <= 32
    nb = -(-n // 256)
    cost = _n3_costs(nb, plan["cols"])
    assert plan["ctas"] == len(cost)
    order = plan["order"]
    assert sorted(order.tolist()) == list(range(len(cost)))
    c = np.array(cost)[order]
    assert np.all(np.diff(c) <= 1e-12)
    assert 0.0 < plan["efficiency"] <= 1.0 + 1e-9
    again = nbr.n3_grid_plan(n, 148, 8, with_order=True)
    assert again["cols"] == plan["cols"] and np.array_equal(again["order"], order)


def test_n3_grid_plan_known_choices(nbr):
    """The widths measured best on B200 (148 SMs): 28 columns for the whole
    N = 262144 grid (a sweep of 24 .. 32 confirmed it), 31 for its 8
    multi-GPU slices; 32 from about 2^20."""
    assert nbr.n3_grid_plan(262144, 148, 8)["cols"] == 28
    assert nbr.n3_grid_plan(262144, 148, 8)["slice_cols"] == 31
    assert nbr.n3_grid_plan(1048576, 148, 8)["cols"] == 32


def test_n3_grid_plan_rejects_bad_arguments(nbr):
    L = nbr.load()
    assert L.nbr_n3_grid_plan(0, 148, 8, None, None, None, None, None, 0) == 1
    assert L.nbr_n3_grid_plan(1000, 0, 8, None, None, None, None, None, 0) == 1
    assert L.nbr_n3_grid_plan(1000, 148, 0, None, None, None, None, None, 0) == 1

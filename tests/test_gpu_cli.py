"""The nbr_main driver with the reference's flag surface (CPU/main.cpp), on the GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu
EXE = os.path.join(PKG, "nbr_main")


def run(args, cwd):
    out = subprocess.run([EXE, *args], capture_output=True, text=True, cwd=cwd, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return out.stdout


def test_cli_omp_main_equivalent_lf(tmp_path):
    """-t gpu -i lf -order 2 on the reference's ring: after one revolution
    the deviation from the initial state is small (omp_main's check)."""
    out = run(["-t", "gpu", "-N", "513", "-s", "1000", "-T", "1.0", "-i", "lf", "-order", "2", "-r", "1e6"], tmp_path)
    assert "Performance:" in out
    dev = float(out.split("Average position deviation from reference:")[1].split()[0])
    assert dev < 1e-3


def test_cli_euler_default(tmp_path):
    out = run(["-N", "200", "-s", "10"], tmp_path)
    assert "Euler" in out and "Performance:" in out


def test_cli_bench_csv_schema(tmp_path):
    csv = tmp_path / "scaling.csv"
    for _ in range(2):
        run(["-t", "gpu-bench", "-N", "4096", "-s", "5", "-i", "lf", "-scheme", "kdk", "-ic", "plummer",
             "-seed", "2", "-eps", "1e-3", "-dt", "5e-4", "-p", "sp", "-o", str(csv)], tmp_path)
    lines = csv.read_text().strip().splitlines()
    assert lines[0] == "#Nodes, Cores, N, t_total[s], performance[Mpairs/s], time_steps/s, ms/time_step"
    assert len(lines) == 3  # header written once, rows appended
    assert int(lines[1].split(",")[2]) == 4096


def test_cli_accuracy_csv(tmp_path):
    csv = tmp_path / "acc.csv"
    run(["-t", "gpu-accuracy", "-start", "1000", "-step", "2", "-n", "2", "-ratio-start", "1e3",
         "-ratio-stop", "1e5", "-ratio-steps", "2", "-o", str(csv)], tmp_path)
    lines = csv.read_text().strip().splitlines()
    assert lines[0].startswith("N, precision, ratio, average_force_length_error")
    assert len(lines) == 1 + 3 * 2
    errs = np.array([float(l.split(",")[3]) for l in lines[1:]])
    assert np.all(errs < 1e-9)  # percent; FP64 against the analytic ring force


def test_cli_ratio_csv(tmp_path):
    csv = tmp_path / "ratio.csv"
    run(["-t", "gpu-ratio", "-start", "101", "-step", "100", "-n", "1", "-s", "50", "-rev-steps", "100",
         "-ratio-start", "1e4", "-ratio-stop", "1e5", "-ratio-steps", "1", "-max-error", "0.5",
         "-o", str(csv)], tmp_path)
    lines = csv.read_text().strip().splitlines()
    assert lines[0].startswith("N, precision, s, s_collapse")
    assert len(lines) == 3
    assert int(lines[1].split(",")[3]) == 50  # no collapse within 50 steps


def test_cli_batch(tmp_path):
    out = run(["-t", "gpu-batch", "-nsys", "64", "-nmin", "64", "-nmax", "512", "-s", "5", "-dt", "1e-3",
               "-eps", "1e-3", "-p", "sp"], tmp_path)
    assert "systems*steps/s" in out


@pytest.mark.parametrize("prec,tol", [("dp", 1e-11), ("sp", 1e-6)])
def test_cli_multi_gpu_newton3(tmp_path, nbr, oracle, prec, tol):
    """-t gpu-multi: the C++ multi-GPU host (NCCL communicator per GPU,
    Newton-3 slices, all-to-all of partial forces, all-gather of positions) on
    the one GPU this runs on; the end state against the oracle's KDK run."""
    final = tmp_path / "final.dat"
    csv = tmp_path / "multi.csv"
    out = run(["-t", "gpu-multi", "-ngpu", "1", "-slices", "5", "-N", "3000", "-ic", "plummer",
               "-seed", "4", "-eps", "1e-3", "-i", "lf", "-scheme", "kdk", "-s", "3", "-dt", "1e-3",
               "-p", prec, "-final", str(final), "-o", str(csv)], tmp_path)
    assert "GPU multi solver" in out
    got = nbr.snapshot_read(str(final), 3000, 0)
    s = nbr.plummer(3000, 4)
    want = oracle.kdk(s, 1e-3, 3, eps2=1e-6)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= tol, k
    lines = csv.read_text().strip().splitlines()
    assert lines[0].startswith("#Nodes, Cores, N") and lines[1].startswith("1,")

"""The reference arm of bench.py on the host cores (no GPU).

`bench.py --impl reference` times the reference's own CPU solver, built from
its sources into oracle/_ref, on the bench workload's inputs: its fastest force
kernel (the line's value) and its end-to-end leapfrog solver
reduced_solver_omp_lf (the line's e2e).  Its one JSON line must carry the keys
the driver reads, and the process must never load the product library (the
inputs come from the oracle's samplers).  A small N keeps the run to seconds.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    # run bench.py's main, then report on stderr whether libnbr.so was mapped
    probe = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--n', '4096', "
             "'--steps', '2', '--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
             "maps = open('/proc/self/maps').read(); "
             "sys.stderr.write('LIBNBR_MAPPED=%d' % ('libnbr.so' in maps))")
    p = subprocess.run([sys.executable, "-c", probe], capture_output=True, text=True, cwd=ROOT,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    if "unavailable" in line:
        pytest.skip(line["unavailable"])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "dtype", "data", "config"):
        assert k in line, k
    assert line["value"] > 0 and line["unit"] == "GPairs/s" and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1 and line["config"]["n"] == 4096
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"]
    assert set(cb["legs"]) == {"force_only", "end_to_end", "config0"}
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["unit"] == line["unit"] and e2e["steps"] >= 1
    assert e2e["value"] == cb["legs"]["end_to_end"]["value"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config0"]["steps_per_s"] > 0
    assert "LIBNBR_MAPPED=0" in p.stderr, p.stderr[-500:]

"""bench.py --impl reference on the host (the reference arm needs no GPU): the
C++ restatement runs real registrations step by step (a step is one GN
iteration) and the line carries the contract's keys."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "16",
                          "--nt", "2", "--steps", "4", "--warmup", "1", "--maxit", "2"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "higher_is_better", "cpu_baseline",
                "e2e", "config"):
        assert key in line
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    cfg = line["config"]
    # maxit 2 and four GN-iteration steps: two complete registrations, measured not extrapolated
    assert cfg["registrations_completed"] == 2 and not cfg["extrapolated_from_gn_iterations"]
    work = cfg["work_per_registration"]
    assert work["iters"] == 2 and work["hess_matvecs"] == work["pcg_iters"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1

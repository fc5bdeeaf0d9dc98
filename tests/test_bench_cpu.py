"""The benchmark's CPU-side pieces: the reference arm (the reference's own CPU
implementation of the path, compiled from its sources when present, else the
oracle restatement) prints one well-formed JSON line, and the algorithmic
byte counts used for the rooflines follow the problem sizes."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_byte_models(product):
    sys.path.insert(0, ROOT)
    import bench
    from karam_b200 import circuits
    info = product.Problem(None, circuits.config2()).info
    n, nm, nv, nc = info["n"], info["n_mos"], info["n_slots"], info["n_cap"]
    assert bench.eval_stamp_bytes(info, True) == 8 * nm + 24 * n + 4 * nv
    assert bench.eval_stamp_bytes(info, False, True) == 8 * nm + 24 * n + 8 * nv + 8 * nc
    assert bench.lu_bytes(info, True) == 4 * nv + 40 * n + 208


@pytest.mark.timeout(600)
def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0", "--cpu-sample", "2"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["unit"] == "solves/s" and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] in ("reference", "port")
    assert rec["e2e"]["h2d_bytes_per_step"] == 0


@pytest.mark.timeout(300)
def test_multi_gpu_request_without_gpus_is_refused():
    """`--gpus N` outside a launcher starts N ranks itself; with fewer visible
    GPUs than asked for it refuses (exit 2, an error line) instead of
    measuring fewer GPUs."""
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                          "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 2
    rec = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][0])
    assert "2 visible GPUs" in rec["error"]

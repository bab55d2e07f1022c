"""The benchmark's CPU arm (`bench.py --impl reference`) on a tiny sample: the line a benchmark
driver parses must carry the contract's keys, with the CPU port timed on the host (kind "port",
no host<->device bytes), and the arm must load no product library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    code = ("import runpy, sys, json\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--cpu-nts', '3']\n"
            "try:\n"
            "    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit as e:\n"
            "    assert not e.code, e.code\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('PRODUCT_LOADED' if 'libaio_b200' in maps else 'PRODUCT_NOT_LOADED')\n")
    env = dict(os.environ, OMP_NUM_THREADS="4")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert lines, out.stdout[-2000:]
    line = json.loads(lines[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "Gpts/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"].startswith("batched Born forward+adjoint")
    assert "PRODUCT_NOT_LOADED" in out.stdout

"""``bench.py --impl reference`` in a fresh process: one JSON line with the contract's keys."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_its_line():
    """The reference arm on the D = 8 layout of the benchmark geometry (the default
    D = 32 arm builds the oracle on 5.8 M cells, minutes and about 19 GB of host memory)."""
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload",
                          "d8_oscillating_sphere", "--steps", "1", "--warmup", "3"],
                         capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    # full layout of the workload, real iterations, the extrapolation labelled
    assert line["config"]["workload"] == "d8_oscillating_sphere" and line["config"]["cells"] == 90_112
    assert line["extrapolated"] is True and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value_one_blas_thread"] > 0 and line["cpu_baseline"]["cpu_model"]


def test_pressure_reference_arm_prints_its_line():
    """The offline pressure recovery's reference arm: the oracle (scipy cg, the
    reference's algorithm) on the 64^3 sample, row-iterations/s."""
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload",
                          "pressure_recovery_128", "--steps", "1", "--warmup", "3"],
                         capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "row-iterations/s"
    assert line["config"]["workload"] == "pressure_recovery_128"
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["value"] == line["value"]

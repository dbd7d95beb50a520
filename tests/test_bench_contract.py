"""bench.py's reference arm (the oracle on the host cores) on a small cell:
one JSON line with the keys the measurement contract asks for; and the
algorithmic byte model the roofline uses."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--n", "5", "--steps", "2",
                          "--warmup", "1", "--ref-seconds", "2"], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["config"]["atoms"] == 250
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0


def test_byte_model():
    sys.path.insert(0, ROOT)
    import bench
    n_half, n_full, n_mid = 42.1, 14.06, 15.87
    m = bench.kernel_bytes_per_atom("screen_density", n_half, n_full, n_mid, mixed=True)
    d = bench.kernel_bytes_per_atom("screen_density", n_half, n_full, n_mid, mixed=False)
    assert abs(m - (4 * n_mid + 4 * n_full + 56)) < 1e-9 and abs(d - m - 32) < 1e-9
    f = bench.kernel_bytes_per_atom("forces", n_half, n_full, n_mid, mixed=True)
    assert abs(f - (4 * n_full + 160)) < 1e-9
    assert bench.kernel_bytes_per_atom("no_such_kernel", n_half, n_full, n_mid) is None

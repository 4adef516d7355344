"""bench.py output contract, on the CPU: the reference arm's JSON line (the
CPU port of the reference path on the small L=31 case) and the helpers that
feed the GPU line's roofline fields."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _json_line(out: str) -> dict:
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out
    return json.loads(lines[0])


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "cfg1",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = _json_line(r.stdout)
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["unit"] == "cycles/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"] == "L31_Nr33"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("port", "reference") and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_roofline_helpers():
    import bench
    from kemorin_mhd_b200.config import SphConfig
    cfg = SphConfig(511, 768, 1536, 257)
    # the committed full-size ncu summaries carry the per-launch DRAM bytes
    t_gemm = bench.read_traffic("k_split_gemm", "L511_Nr257")
    t_fft = bench.read_traffic("k_fft_cycle_f", "L511_Nr257")
    assert t_gemm is not None and 1e10 < t_gemm < 1e11
    assert t_fft is not None and 1e10 < t_fft < 1e11
    assert bench.read_traffic("k_split_gemm", "no_such_workload") is None
    # executed INT8 ops: proportional to the slice-product count, and at least
    # the useful work of 26 products per useful multiply-add
    e26 = bench.split_executed_ops(cfg, 26)
    e10 = bench.split_executed_ops(cfg, 10)
    assert abs(e26 / e10 - 2.6) < 1e-12
    useful = 2.0 * cfg.nh * cfg.J * cfg.nr * (5 * 3 + 1)  # default set: 3 vectors + 1 scalar
    assert e26 > 26 * useful

"""The bench's reference arm on the CPU: `bench.py --impl reference` times the
reference's own H-apply (compiled from its sources into oracle/_ref) and prints one
JSON line with the contract's keys (impl, metric, unit, cpu_baseline, e2e with zero
host-device bytes). Skipped where the reference harness has not been built."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libqumasun_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference harness not built")
@pytest.mark.timeout(300)
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=280, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "H|psi> GB/s (algorithmic)" and d["unit"] == "GB/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
    assert d["steps"] == 1 and d["warmup"] == 1
    # a step is the whole 256-state workload, measured (not extrapolated)
    assert d["config"]["n_states"] == 256 and abs(d["ms_per_step"] - 256 / d["state_applications_per_s"] * 1e3) < 1.0
    sys.path.insert(0, ROOT)
    import bench
    from qumasun_b200.cell import build_cell
    assert d["config"] == bench.bench_config(build_cell(reps=bench.REPS), 1)

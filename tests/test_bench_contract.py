"""The bench's reference arm on CPU: one JSON line with the fields the measurement
contract needs (the CPU port of the reference sweep, timed on the host cores), and
the bench's committed DRAM-traffic record."""
import json
import pathlib
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "spin-updates/s" and d["unit"] == "attempts/s"
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    # the default workload is the large frustrated configuration, and the reference arm
    # runs the oracle's port alone: the CUDA library is never mapped into that process
    assert d["config"]["workload"].startswith("fcc64") and d["config"]["sites_per_chain"] == 4 * 64 ** 3
    assert d["config"]["libscemc_cuda_loaded"] is False


def test_dram_traffic_record_names_the_default_workload():
    d = json.loads((ROOT / "profiles" / "dram_traffic.json").read_text())
    recs = d["fcc64_l2_tri_zeeman_32rungs_metropolis+OR+exchange"]
    assert "3" in recs  # by kernel id of the launch form the autotuner may pick
    for rec in recs.values():
        assert 100 < rec["bytes_per_attempt"] < 5000 and rec["source"] and rec["kernel"]

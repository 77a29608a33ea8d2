"""The bench's JSON contract on the CPU: the reference arm's line (the reference's own CPU path
on a bounded sample of the workload), and the clock sampler's restriction of its samples to
the timed region."""
import importlib.util
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _bench_module():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:  # the compiled reference is missing: the arm says why and exits 0
        assert line["unavailable"]
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["unit"] == "particle-substeps/s" and line["higher_is_better"] is True
    assert line["config"]["workload"] == "dp_two_boxes_dx256_8ppc"
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    # a sample of the 30 M-particle workload: the line says how many particles it ran
    assert 0 < line["extrapolated_from"] < line["config"]["particles"]
    assert line["extrapolation"]


def test_g2p_bytes_follow_the_survey_accounting():
    bench = _bench_module()
    # 188 B per plastic particle (180 + logJp read and write) and 12 B per active cell
    assert bench.g2p_algorithmic_bytes(30_089_900, 10_450, True) == 30_089_900 * 188 + 10_450 * 512 * 12
    assert bench.g2p_algorithmic_bytes(1, 0, False) == 180
    assert bench.g2p_implementation_bytes(1, 0, True) == 212
    assert bench.substep_algorithmic_bytes(1, 0, True) == 304


def test_clock_sampler_keeps_the_timed_region():
    bench = _bench_module()
    c = bench.ClockSampler(0)
    c.thread = object()  # as if the NVML thread ran: only the summary is under test
    c.samples = [(1.0, 1965, 1965, 0), (2.0, 1900, 1965, 0x4), (3.0, 1965, 1965, 0), (9.0, 900, 1965, 0x48)]
    c.t0, c.t1 = 1.5, 3.5
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1932.5 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"]
    c.t0, c.t1 = 8.0, 10.0
    assert c.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
    c.t0, c.t1 = 4.0, 5.0
    assert c.summary()["reasons"] == ["no samples"]

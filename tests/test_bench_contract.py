"""The JSON line of bench.py: the reference arm (the reference's own host
solver, or the oracle port where that build is absent) runs on the CPU and
prints the contract's keys; the byte accounting and the figures read from the
committed files are the ones the GPU arm reports."""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..")
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    # the line names the sample it times: 64^3, with a 128^3 sample beside it
    assert d["config"]["mesh"] == [64, 64, 64] and "64^3 sample" in d["config"]["workload"]
    assert set(d["config"]["samples"]) == {"64^3", "128^3"}
    assert d["config"]["samples"]["64^3"]["value"] == pytest.approx(d["value"])
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    if cb["kind"] == "reference":  # the build flags are stated
        assert "-O3" in cb["sample"] and "-march=" in cb["sample"]
    assert cb["value"] == pytest.approx(d["value"])
    e = d["e2e"]
    assert e["value"] == pytest.approx(d["value"]) and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_algorithmic_bytes_per_step():
    # s = 0 reads in and writes out; s = 1, 2 read in and out and write out:
    # 8 array touches of 8 fields per step; a mixed value is 4 + 2 bytes
    n = 512
    assert bench.alg_bytes_per_step("sp", n) == 8 * 4 * 8 * n ** 3
    assert bench.alg_bytes_per_step("mixed", n) == 8 * 6 * 8 * n ** 3
    assert bench.alg_bytes_per_step("dp", n) == 8 * 8 * 8 * n ** 3


def test_traffic_and_peak_come_from_committed_files():
    t = bench.profile_traffic("solve_mixed_256.json", 512)
    # a 512^3 step's three launches move about 128 B per cell each on average
    # (s = 0: hi and bf16 lo of in read, out written, 96 B; s = 1, 2: also out
    # read, 144 B); the committed capture is within 10 % of that
    assert t is not None and abs(t / (128 * 512 ** 3) - 1.0) < 0.10
    # the peak: the measured copy bandwidth where the machine's record of it
    # exists, else the stated fallback
    peak, kind = bench.measured_peak_hbm()
    measured = os.path.exists(os.path.join(bench.HERE, "MEASURED_PEAKS.json"))
    assert kind == ("measured" if measured else "fallback") and 5000.0 < peak < 8000.0


def test_cpu_oracle_sample_reports_all_cores():
    """The multi-core CPU figure: the oracle's FP64 solver with OpenMP on the
    host cores this process may use, a bounded sample; `cores` is the thread
    count the oracle's OpenMP loops ran with."""
    import bench
    import oracle_lib as O

    r = bench.cpu_oracle_sample(budget_s=0.2, n=16)
    assert r["kind"] == "port" and r["unit"] == bench.UNIT
    assert r["cores"] == O.omp_threads()
    assert r["cpus_available"] == len(os.sched_getaffinity(0))
    assert r["value"] > 0 and "FP64" in r["sample"]

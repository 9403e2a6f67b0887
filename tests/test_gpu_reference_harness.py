"""The reference's own benchmark harness run through the drop-in.

`ac_run -b` (samples/standalone/benchmark.cc:49-118), its sources unchanged and
linked against the FP32 library, integrates a 512^3 mesh from the ABC-flow
initial state: 10 warm-up steps of acIntegrate(0), then 100 steps of
acIntegrate(FLT_EPSILON) + acSynchronize, each timed by the host clock; it
prints the mean and the 90th percentile per step. The same library, driven
through acDeviceIntegrateStep with a synchronisation after every step, is timed
here on a 512^3 mesh of seeded noise, by the host clock and by CUDA events.
The harness's figures must agree with these within 10 %: the kernels do not
branch on the data, so the initial state does not change the work. Both sets of
figures are printed (pytest -s)."""
import json
import os
import re
import statistics
import subprocess
import time

import numpy as np
import pytest

from astaroth_b200 import Device, abi, init

pytestmark = pytest.mark.gpu
N = 512


def test_reference_benchmark_harness_agrees_with_library_timing(tmp_path):
    exe = os.path.join(abi.REPO, "oracle", "_ref", "ac_run_sp")
    if not os.path.exists(exe):
        pytest.skip("standalone binary not built (needs the reference sources at build time)")
    # the harness overrides the mesh size (512^3) and keeps the rest of the
    # configuration file it is given: the reference's default one
    conf = tmp_path / "astaroth.conf"
    conf.write_text("".join(f"{k} = {v}\n" for k, v in abi.DEFAULT_CONFIG.items()))
    r = subprocess.run([exe, "--benchmark", "--config", str(conf)], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    mean = re.search(r"Time per step: ([0-9.]+) ms", r.stdout)
    p90 = re.search(r"90th percentile per step: ([0-9.]+) ms", r.stdout)
    assert mean and p90, r.stdout[-3000:]
    harness = {"mean_ms": float(mean.group(1)), "p90_ms": float(p90.group(1))}
    with open(tmp_path / "nprocs_1_result_strong.bench") as f:
        assert f.read().splitlines()[0].startswith("num_processes")

    # the same step through the library's own entry point
    import torch

    info = abi.make_info(abi.SP, N)
    fields = init.workload_fields(N, N, N, np.float32, seed=7, amplitude=1e-3,
                                  velocity_mode=0.1)
    host = abi.HostMesh(abi.SP, info, fields)
    del fields
    dt = float(np.finfo(np.float32).eps)
    with Device("sp", info, 0) as dev:
        dev.load_mesh(host)
        del host
        st = torch.cuda.ExternalStream(dev.cuda_stream(0))
        for _ in range(10):
            dev.integrate_step(0.0)
        dev.synchronize()
        wall, evt = [], []
        for _ in range(100):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(st)
            dev.integrate_step(dt)
            e1.record(st)
            dev.synchronize()
            wall.append((time.perf_counter() - t0) * 1e3)
            evt.append(e0.elapsed_time(e1))
        assert dev.status() == 0
    wall.sort()
    library = {"mean_ms": statistics.mean(wall), "p90_ms": wall[int(0.9 * len(wall))],
               "device_mean_ms": statistics.mean(evt)}
    print("reference harness (ac_run -b, 512^3 FP32):", json.dumps(harness))
    print("library, acDeviceIntegrateStep + synchronize:", json.dumps(library))
    assert harness["mean_ms"] == pytest.approx(library["mean_ms"], rel=0.10)
    assert harness["p90_ms"] == pytest.approx(library["p90_ms"], rel=0.10)

#!/usr/bin/env python
"""RK3 cell-updates/s of the single-device MHD solver, 512^3 workload.

Workload (the headline configuration): 512^3 mesh, eight fields
(lnrho, ux, uy, uz, ax, ay, az, entropy), seeded 1e-3 * U(-1,1) noise plus the
k = 2 velocity mode u = 0.1 (sin 2y, sin 2z, sin 2x), dx = 2 pi / 512,
nu = eta = 5e-3, cs = 1, gamma = 5/3, cp = 1, dt = 1e-3, periodic.
The measured arm is the mixed-precision library (FP32 stencils and right-hand
sides, compensated state: FP32 hi part and bfloat16 lo part, FP64 reductions);
the plain FP64 and
FP32 libraries run the same steps beside it for the comparison and the error.

One step = three substeps, each a periodic ghost fill of all fields plus one
fused solve launch, all through the C ABI (acDevicePeriodicBoundconds,
acDeviceIntegrateSubstep, acDeviceSwapBuffers). Inputs are larger than L2
(8.9 GB of state per block), so no L2 flush is needed between steps.

Beside the headline line: the FP64 and FP32 libraries on the same steps (and
the per-field error against FP64), an end-to-end run from pinned host memory,
the 64-member ensemble, the 256^3 FP32 and FP64 runs with four reductions read
back every step, simulation loops whose time step follows the state (64^3 and
128^3 FP32: the time step chosen on the host after a synchronising reduction,
as the reference standalone does, against the time step chosen on the device),
and the forced large-mesh run (1024^3 mixed, helical forcing from a seeded
generator and four FP64 diagnostics every step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs are replicas (the path has no exchange step on one device):
every rank advances its own mesh; value = all ranks' cell updates / max time.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import statistics
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "RK3 cell-updates/s at 512^3 (mixed precision; FP64 and FP32 alongside)"
UNIT = "cell-updates/s"
N_DEFAULT = 512
DT = 1e-3
PHYS = dict(gamma=5.0 / 3.0, nu_visc=5e-3, eta=5e-3, cs_sound=1.0, cp_sound=1.0)


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_DEFAULT, help="mesh size (default 512)")
    ap.add_argument("--flavour", choices=["mixed", "sp", "dp"], default="mixed",
                    help="library of the measured arm (default mixed; the others for "
                         "profiling their kernels with the same driver)")
    ap.add_argument("--no-variants", action="store_true", help="skip the FP64/FP32 side runs")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-member ensemble")
    ap.add_argument("--no-cfl", action="store_true",
                    help="skip the loops whose time step follows the state")
    ap.add_argument("--no-forced", action="store_true",
                    help="skip the forced large-mesh run (helical forcing + diagnostics)")
    ap.add_argument("--forced-n", type=int, default=1024, help="mesh size of the forced run")
    ap.add_argument("--no-oracle", action="store_true",
                    help="skip the comparisons with the f64 oracle (512^3 after 2 steps; "
                         "256^3 diagnostics over 100 steps)")
    ap.add_argument("--no-diagnostics", action="store_true",
                    help="skip the 256^3 FP32/FP64 run with reductions every step")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# ranks
# ---------------------------------------------------------------------------
class Ranks:
    """One process per GPU (torchrun environment). Replicas only: the group is
    used for the barrier around the timed region and the max of the timings,
    never on the data path. backend "nccl" on GPUs; "gloo" runs the same logic
    on CPU processes (tests)."""

    def __init__(self, gpus: int, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
            self.dist = dist

    def _sync(self):
        if self.backend == "nccl":
            import torch

            torch.cuda.synchronize()

    def barrier(self):
        self._sync()
        if self.dist:
            self.dist.barrier()
        self._sync()

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, cells_per_rank: int, steps: int, ms: float) -> float:
        """Whole-job cell updates per second: every rank's cells over the max
        time (pass `ms` already reduced with max())."""
        return self.world * cells_per_rank * steps / (ms * 1e-3)

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            text, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            text, _ = self.proc.communicate()
        rows = [r for r in csv.reader(io.StringIO(text)) if len(r) >= 9]
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload_info(prec, n: int):
    from astaroth_b200 import abi

    ds = 2.0 * math.pi / n
    return abi.make_info(prec, n, n, n, dsx=ds, dsy=ds, dsz=ds, **PHYS)


def host_mesh(flavour: str, n: int, pinned: bool = True, velocity_mode: float = 0.1):
    """The seeded initial state as a pinned host AcMesh of the flavour's AcReal:
    1e-3 noise (seed 1) plus the k = 2 velocity mode of amplitude
    velocity_mode. Values are generated on the GPU (bit-identical to the numpy
    generator), rounded to float32 once; the FP64 library gets the same
    float32 values."""
    import torch

    from astaroth_b200 import abi, init

    prec = abi.PRECISIONS[flavour]
    info = workload_info(prec, n)
    tdt = torch.float64 if prec.double else torch.float32
    host = abi.HostMesh(prec, info, pinned=pinned)
    gen = init.workload_fields_torch(n, n, n, torch.float32, seed=1, amplitude=1e-3,
                                     velocity_mode=velocity_mode, device="cuda")
    for w, g in enumerate(gen):
        host.fields[w][...] = g.to(tdt).cpu().numpy()
    del gen
    torch.cuda.empty_cache()
    return host


def alg_bytes_per_step(flavour: str, n: int) -> int:
    """Algorithmic HBM bytes of the three solve launches of one step: every
    array touched once per substep (s = 0: read in, write out; s = 1, 2: read
    in, read out, write out), eight fields. FP32 4 B, FP64 8 B, mixed 6 B
    (float hi + bfloat16 lo) per value: 256, 512 and 384 B per cell and step."""
    w = {"sp": 4, "dp": 8, "mixed": 6}[flavour]
    return 8 * w * (2 + 3 + 3) * n ** 3


def timed_steps(dev, steps: int, warmup: int, ranks, sample_clocks=False, gpu_index=0):
    """Runs warmup + steps RK3 steps through the C ABI; returns device-timed
    figures (CUDA events on the device's stream, max over ranks)."""
    import torch

    st = torch.cuda.ExternalStream(dev.cuda_stream(0))
    for _ in range(warmup):
        for s in range(3):
            dev.periodic_boundconds()
            dev.integrate_substep(s, DT)
            dev.swap_buffers()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    pairs = [[(ev(), ev()) for _ in range(3)] for _ in range(steps)]
    e0, e1 = ev(), ev()
    clocks = ClockSampler(gpu_index) if sample_clocks else None
    ranks.barrier()
    launches0 = dev.launch_count()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0.record(st)
    for k in range(steps):
        for s in range(3):
            dev.periodic_boundconds()
            pairs[k][s][0].record(st)
            dev.integrate_substep(s, DT)
            pairs[k][s][1].record(st)
            dev.swap_buffers()
    e1.record(st)
    e1.synchronize()
    ranks.barrier()
    clk = clocks.stop() if clocks else None
    launches = dev.launch_count() - launches0
    total_ms = ranks.max(e0.elapsed_time(e1))
    solve_ms = [[a.elapsed_time(b) for a, b in row] for row in pairs]
    solve_total = ranks.max(sum(sum(r) for r in solve_ms))
    per_substep = [statistics.mean(r[s] for r in solve_ms) for s in range(3)]
    return {"total_ms": total_ms, "ms_per_step": total_ms / steps,
            "solve_ms_total": solve_total, "solve_ms_per_substep": per_substep,
            "launches": launches, "clocks": clk}


def field_errors(dev_a, dev_b, n: int) -> list[float]:
    """Per-field normwise error max|a - b| / max|b| over the interior, from the
    double views of the two devices' current states."""
    import torch

    g = 3
    errs = []
    for w in range(8):
        a = torch.from_numpy(dev_a.store_double(w)).cuda()[g:-g, g:-g, g:-g]
        b = torch.from_numpy(dev_b.store_double(w)).cuda()[g:-g, g:-g, g:-g]
        den = float(b.abs().max())
        errs.append(float((a - b).abs().max()) / den if den > 0 else float((a - b).abs().max()))
        del a, b
    torch.cuda.empty_cache()
    return errs


def e2e_run(flavour: str, host, steps: int, ranks) -> dict:
    """The same steps end to end through the public C ABI with host buffers:
    load the mesh from pinned host memory, per step one RK3 step
    (acDeviceIntegrateStep) and one diagnostic reduction read back to the host
    (max |u|, as a CFL check does), then store the mesh to pinned host memory.
    The reduction is folded into each step's last substep
    (acDeviceSetStepDiagnostics), so acDeviceReduceVec(MAX) returns it with one
    small device-to-host copy instead of another pass over the fields."""
    import torch

    from astaroth_b200 import Device, abi

    n = abi.dims(host.info)[0]
    dev = Device(flavour, host.info, torch.cuda.current_device())
    out = abi.HostMesh(host.prec, host.info, pinned=True)
    dev.set_step_diagnostics(True)
    dev.load_mesh(host)
    dev.integrate_step(DT)  # warm the kernels and graph-free path
    dev.synchronize()
    ranks.barrier()
    t0 = time.perf_counter()
    dev.load_mesh(host)
    umax = 0.0
    for _ in range(steps):
        dev.integrate_step(DT)
        umax = dev.reduce_vec(abi.RTYPE_MAX, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
    dev.store_mesh(out)
    dev.synchronize()
    t = ranks.max(time.perf_counter() - t0)
    mesh_bytes = 8 * host.fields[0].nbytes
    dev.destroy()
    del out
    return {"seconds": t, "cells_per_s": ranks.world * n ** 3 * steps / t,
            "h2d_bytes_per_step": mesh_bytes / steps, "d2h_bytes_per_step": 32 + mesh_bytes / steps,
            "umax": umax}


def cpu_oracle_sample(budget_s: float = 6.0, n: int = 64) -> dict:
    """The CPU restatement of the reference host solver (oracle/mhd_oracle.c,
    its row-wise form) in double precision with OpenMP on the host cores this
    process may use, on an n^3 sample of the same physics: the multi-core CPU
    figure beside the reference's own single-threaded solver."""
    sys.path.insert(0, os.path.join(HERE, "tests"))
    import numpy as np

    import oracle_lib as O
    from astaroth_b200 import abi, init

    info = workload_info(abi.DP, n)
    fields = init.workload_fields(n, n, n, np.float64, seed=1, amplitude=1e-3, velocity_mode=0.1)
    om = O.OracleMesh("f64", fields, n, n, n)
    p = O.params_from(info)
    om.step(p, DT)  # warm-up (thread pool, first touch)
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s:
        om.step(p, DT)
        steps += 1
    t = time.perf_counter() - t0
    threads = O.omp_threads()
    return {"value": n ** 3 * steps / t, "unit": UNIT, "cores": threads,
            "cpus_available": len(os.sched_getaffinity(0)), "kind": "port",
            "sample": f"{steps} RK3 steps of a {n}^3 mesh; oracle/mhd_oracle.c (row-wise form) "
                      f"in FP64, OpenMP with {threads} threads"}


# the reference's host utils as timed: its Release flags (-O3 on x86-64; the
# pinning build, which also turns contraction off) and an AVX2/FMA build
REF_BUILDS = {"": "-O3 -march=x86-64-v2 -ffp-contract=off",
              "avx2": "-O3 -march=x86-64-v3 (AVX2, FMA contraction on)"}


def cpu_reference_sample(budget_s: float = 12.0, n: int = 64, max_steps: int | None = None,
                         warmup: int = 0, build: str | None = None) -> dict:
    """The reference's own host solver (src/utils/modelsolver.c acHostIntegrateStep,
    FP32, built from its sources into oracle/_ref; its OpenMP pragmas are
    commented out, so one thread) on an n^3 sample of the same physics; the
    oracle port (OpenMP) where that build is absent. build None: the faster
    of the two builds (one warm-up step of each decides)."""
    sys.path.insert(0, os.path.join(HERE, "tests"))
    import numpy as np

    import oracle_lib as O
    from astaroth_b200 import abi, init

    info = workload_info(abi.SP, n)
    fields = init.workload_fields(n, n, n, np.float32, seed=1, amplitude=1e-3, velocity_mode=0.1)
    libs = {b: O.ref_lib("sp", b) for b in REF_BUILDS}
    libs = {b: l for b, l in libs.items() if l is not None}
    if libs:
        hm = abi.HostMesh(abi.SP, info, fields)
        if build is None:
            pick = {}
            for b, lib in libs.items():
                t0 = time.perf_counter()
                lib.acHostIntegrateStep(hm.cmesh, abi.SP.real(DT))
                pick[b] = time.perf_counter() - t0
            build = min(pick, key=pick.get)
        ref = libs[build]

        def step():
            ref.acHostIntegrateStep(hm.cmesh, abi.SP.real(DT))

        kind, cores = "reference", 1
        what = ("reference src/utils/modelsolver.c acHostIntegrateStep (FP32), 1 thread, "
                f"built {REF_BUILDS[build]}")
    else:
        om = O.OracleMesh("f32", fields, n, n, n)
        p = O.params_from(info)

        def step():
            om.step(p, float(np.float32(DT)))

        kind, cores, build = "port", O.omp_threads(), "port"
        what = f"oracle/mhd_oracle.c (FP32 restatement), OpenMP with {cores} threads"
    for _ in range(warmup):
        step()
    times = []
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
        if max_steps is not None and len(times) >= max_steps:
            break
        if max_steps is None and time.perf_counter() - t_start >= budget_s:
            break
    tot = sum(times)
    return {"value": n ** 3 * len(times) / tot, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{len(times)} RK3 steps of a {n}^3 mesh of the same physics; {what}",
            "ms_per_step": 1e3 * tot / len(times), "steps": len(times), "build": build,
            "mesh": [n, n, n]}


def oracle_errors(n: int, steps: int, gpu: int) -> dict:
    """Per-field error of the three libraries against the f64 oracle at n^3:
    the headline's seeded initial state, `steps` RK3 steps through
    acDeviceIntegrateStep in each library, the oracle (row-wise form, OpenMP)
    stepped from the same float32 values; max|x - x_oracle| / max|x_oracle| per
    field over the interior, evaluated on the GPU in double precision."""
    import torch

    sys.path.insert(0, os.path.join(HERE, "tests"))
    import oracle_lib as O
    from astaroth_b200 import Device, abi

    t0 = time.perf_counter()
    host = host_mesh("sp", n)
    om = O.OracleMesh("f64", host.fields, n, n, n)
    om.step(O.params_from(workload_info(abi.DP, n)), DT, steps)
    oracle_s = time.perf_counter() - t0
    g = abi.NGHOST
    out = {"metric": f"max|x - x_oracle| / max|x_oracle| per field after {steps} steps at "
                     f"{n}^3 (f64 oracle, row-wise form)",
           "fields": list(abi.VTXBUFS), "oracle_seconds": oracle_s,
           "oracle_threads": O.omp_threads()}
    for flav in ("mixed", "sp", "dp"):
        h = host if flav != "dp" else host_mesh("dp", n)
        dev = Device(flav, h.info, gpu)
        try:
            dev.load_mesh(h)
            for _ in range(steps):
                dev.integrate_step(DT)
            dev.synchronize()
            errs = []
            for w in range(8):
                a = torch.from_numpy(dev.store_double(w)).cuda()[g:-g, g:-g, g:-g]
                b = torch.from_numpy(om.interior(w)).cuda()
                errs.append(float((a - b).abs().max()) / float(b.abs().max()))
                del a, b
            out[{"mixed": "mixed_vs_oracle", "sp": "fp32_vs_oracle", "dp": "fp64_vs_oracle"}[flav]] = errs
        finally:
            dev.destroy()
            torch.cuda.empty_cache()
    del om, host
    return out


def ensemble_run(steps: int, ranks) -> dict:
    """The ensemble workload: 64 independent FP32 meshes, 16 each of 32^3,
    48^3, 96^3 and 128^3, nu and eta log-uniform in [1e-3, 1e-2] per member
    (seeded), seeded 1e-3 noise. Steps/s of (a) the ensemble, one ghost fill +
    one solve launch per substep replayed from a CUDA graph, against looping
    single-mesh Devices (b) launching asynchronously (each Device on its own
    streams, so the GPU overlaps members) and (c) synchronising each member's
    step as the reference's Node/Legacy integrate does."""
    import numpy as np
    import torch

    from astaroth_b200 import Device, Ensemble, abi, init

    prec = abi.SP
    sizes = [32] * 16 + [48] * 16 + [96] * 16 + [128] * 16
    rng = np.random.default_rng(2024)
    infos, hosts = [], []
    for k, n in enumerate(sizes):
        nu, eta = 10 ** rng.uniform(-3, -2, 2)
        ds = 2 * math.pi / n
        info = abi.make_info(prec, n, dsx=ds, dsy=ds, dsz=ds, gamma=5 / 3, cs_sound=1.0,
                             cp_sound=1.0, nu_visc=nu, eta=eta)
        h = abi.HostMesh(prec, info)
        gen = init.workload_fields_torch(n, n, n, torch.float32, seed=100 + k, amplitude=1e-3,
                                         device="cuda")
        for w, g in enumerate(gen):
            h.fields[w][...] = g.cpu().numpy()
        infos.append(info)
        hosts.append(h)
    cells = sum(n ** 3 for n in sizes)
    dev_index = torch.cuda.current_device()

    ens = Ensemble("sp", infos, dev_index)
    for k in range(len(sizes)):
        ens.load_member(k, hosts[k])
    ens.auto_optimize()
    st = torch.cuda.ExternalStream(ens.cuda_stream())
    ens.integrate_steps(DT, 2)
    ens.synchronize()
    ranks.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ens.launch_count()
    e0.record(st)
    ens.integrate_steps(DT, steps)
    e1.record(st)
    e1.synchronize()
    ens_ms = ranks.max(e0.elapsed_time(e1) / steps)
    ens_launches = ens.launch_count() - l0
    cfg, seg = ens.schedule()
    ens.destroy()

    devs = [Device("sp", infos[k], dev_index) for k in range(len(sizes))]
    for k, d in enumerate(devs):
        d.load_mesh(hosts[k])

    def loop(sync_each: bool) -> float:
        for d in devs:
            d.integrate_step(DT)
        torch.cuda.synchronize()
        ranks.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            for d in devs:
                d.integrate_step(DT)
                if sync_each:
                    d.synchronize(0)
        torch.cuda.synchronize()
        return ranks.max((time.perf_counter() - t0) * 1e3 / steps)

    loop_async = loop(False)
    loop_sync = loop(True)
    for d in devs:
        d.destroy()
    return {"members": "16 x 32^3, 16 x 48^3, 16 x 96^3, 16 x 128^3 (FP32)",
            "cells": cells, "ensemble_ms_per_step": ens_ms,
            "ensemble_steps_per_s": 1e3 / ens_ms,
            "ensemble_cell_updates_per_s": ranks.world * cells / (ens_ms * 1e-3),
            "ensemble_launches_per_step": ens_launches / steps,
            "schedule": {"tile_config": cfg, "segment_planes": seg},
            "loop_async_ms_per_step": loop_async, "loop_sync_ms_per_step": loop_sync,
            "speedup_vs_loop_async": loop_async / ens_ms,
            "speedup_vs_loop_sync": loop_sync / ens_ms}


def forced_run(n: int, steps: int, warmup: int, ranks, gpu: int) -> dict:
    """The forced large-mesh workload: an n^3 mixed-precision mesh (1024^3:
    105 GB of state, float hi and bfloat16 lo parts in two buffers), the seeded initial state of the
    headline workload, and every step a new helical forcing (|k| in [1, 3],
    magnitude 0.05, relhel 0, from the seeded generator acForcingParamsGenerate,
    seed 5) then one RK3 step then the diagnostics: max, min and rms of |u|
    and rms_exp of lnrho (FP64 reductions, each read back). The initial fields
    are generated on the device one at a time and loaded device to device.

    The time step is the headline's 1e-3 scaled by dx^2 (2.5e-4 at 1024^3): the
    diffusion number nu_long dt / dx^2 of the 512^3 workload, with
    nu_long = 4/3 nu + zeta = 0.0167, is already near the real-axis limit of
    the three-stage Runge-Kutta scheme, and dt = 1e-3 at dx = 2 pi / 1024 makes
    grid-scale modes grow (the f64 oracle reaches NaN within 6 steps)."""
    import ctypes as C

    import torch

    from astaroth_b200 import Device, abi, init
    from astaroth_b200.device import ForcingGenerator

    prec = abi.PRECISIONS["mixed"]
    ds = 2.0 * math.pi / n
    info = abi.make_info(prec, n, n, n, dsx=ds, dsy=ds, dsz=ds, kmin=1.0, kmax=3.0, relhel=0.0,
                         forcing_magnitude=0.05, **PHYS)
    torch.cuda.empty_cache()
    free_b, _ = torch.cuda.mem_get_info(gpu)
    dev = Device("mixed", info, gpu)
    try:
        footprint = dev.memory_footprint()
        mesh = abi.mesh_type(prec)()
        mesh.info = info
        for w in range(abi.NUM_VTXBUF_HANDLES):
            g = init.workload_field_torch(w, n, n, n, torch.float32, seed=1, amplitude=1e-3,
                                          velocity_mode=0.1, device=f"cuda:{gpu}")
            torch.cuda.synchronize(gpu)
            mesh.vertex_buffer[w] = C.cast(C.c_void_p(g.data_ptr()), C.POINTER(prec.real))
            if dev.lib.acDeviceLoadVertexBuffer(dev.handle, 0, mesh, w) != abi.AC_SUCCESS:
                raise RuntimeError("acDeviceLoadVertexBuffer failed")
            dev.synchronize()
            mesh.vertex_buffer[w] = C.POINTER(prec.real)()
            del g
            torch.cuda.empty_cache()
        dev.set_forcing(True)
        dev.set_step_diagnostics(True)  # the four diagnostics folded into substep 2
        gen = ForcingGenerator("mixed", info, seed=5)
        st = torch.cuda.ExternalStream(dev.cuda_stream(0))
        diag = {}

        dt = DT * (N_DEFAULT / n) ** 2

        def step():
            dev.load_forcing_params(gen.next())
            dev.integrate_step(dt)
            diag["umax"] = dev.reduce_vec_double(abi.RTYPE_MAX, abi.VTXBUF_UUX, abi.VTXBUF_UUY,
                                                 abi.VTXBUF_UUZ)
            diag["umin"] = dev.reduce_vec_double(abi.RTYPE_MIN, abi.VTXBUF_UUX, abi.VTXBUF_UUY,
                                                 abi.VTXBUF_UUZ)
            diag["urms_sum"] = dev.reduce_vec_double(abi.RTYPE_RMS, abi.VTXBUF_UUX,
                                                     abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
            diag["rhorms_sum"] = dev.reduce_scal_double(abi.RTYPE_RMS_EXP, abi.VTXBUF_LNRHO)

        for _ in range(warmup):
            step()
        dev.synchronize()
        ranks.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(st)
        for _ in range(steps):
            step()
        e1.record(st)
        e1.synchronize()
        wall_ms = (time.perf_counter() - t0) * 1e3
        ranks.barrier()
        ms = ranks.max(e0.elapsed_time(e1))
        # the same steps without reading the diagnostics: their share of a step
        def bare():
            dev.load_forcing_params(gen.next())
            dev.integrate_step(dt)

        dev.synchronize()
        ranks.barrier()
        e0.record(st)
        for _ in range(steps):
            bare()
        e1.record(st)
        e1.synchronize()
        bare_ms = ranks.max(e0.elapsed_time(e1))
        cells = n ** 3
        return {"mesh": [n, n, n], "steps": steps, "warmup": warmup,
                "ms_per_step": ms / steps, "wall_ms_per_step": wall_ms / steps,
                "ms_per_step_without_diagnostics": bare_ms / steps,
                "diagnostics_share_of_step": (ms - bare_ms) / ms,
                "cell_updates_per_s": ranks.world * cells * steps / (ms * 1e-3),
                "device_state_gb": footprint / 1e9, "free_gb_before": free_b / 1e9, "dt": dt,
                "step": "forcing params load + 3 x (ghost fill + forced solve) + 4 FP64 "
                        "diagnostics read back (folded into the last substep's solve)",
                "forcing": "helical, |k| in [1, 3], magnitude 0.05, relhel 0, seed 5",
                "last_step_diagnostics": {"umax": diag["umax"], "umin": diag["umin"],
                                          "urms": math.sqrt(diag["urms_sum"] / cells),
                                          "rho_rms": math.sqrt(diag["rhorms_sum"] / cells)},
                "state_finite": all(math.isfinite(v) for v in diag.values())}
    finally:
        dev.destroy()
        torch.cuda.empty_cache()


def diagnostics_run(n: int, steps: int, warmup: int, ranks, gpu: int,
                    check_steps: int = 0) -> dict:
    """The diagnostics workload: an n^3 mesh (256^3) of seeded 1e-3 noise in
    FP32 and in FP64, each step an RK3 step followed by max, min and rms of |u|
    and rms_exp of lnrho, each read back (FP64 accumulation); reported as
    step-only time, step + diagnostics time and the time of one reduction.
    With check_steps > 0, also the error of both libraries against the f64
    oracle over that many steps from the initial state: every step's four
    diagnostics (relative) and the final fields (normwise)."""
    import torch

    from astaroth_b200 import Device, abi

    out = {"mesh": [n, n, n], "steps": steps, "warmup": warmup, "init": "seeded 1e-3 noise",
           "diagnostics": "max, min, rms of |u|; rms_exp of lnrho; each read back",
           "folded": "acDeviceSetStepDiagnostics: the last substep folds the four; "
                     "diagnostics_share_of_step = (step + diagnostics, folded) / step alone - 1 "
                     "as a share of the former"}
    if check_steps > 0:
        out["errors_vs_oracle"] = diagnostics_errors(n, check_steps, gpu)
    for flav in ("sp", "dp"):
        host = host_mesh(flav, n, velocity_mode=0.0)
        dev = Device(flav, host.info, gpu)
        try:
            dev.load_mesh(host)
            st = torch.cuda.ExternalStream(dev.cuda_stream(0))

            def diag():
                dev.reduce_vec(abi.RTYPE_MAX, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
                dev.reduce_vec(abi.RTYPE_MIN, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
                dev.reduce_vec(abi.RTYPE_RMS, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
                dev.reduce_scal(abi.RTYPE_RMS_EXP, abi.VTXBUF_LNRHO)

            def timed(fn, k):
                for _ in range(warmup):
                    fn()
                dev.synchronize()
                ranks.barrier()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(k):
                    fn()
                e1.record(st)
                e1.synchronize()
                return ranks.max(e0.elapsed_time(e1)) / k

            step_ms = timed(lambda: dev.integrate_step(DT), steps)
            both_ms = timed(lambda: (dev.integrate_step(DT), diag()), steps)
            red_ms = timed(diag, steps) / 4
            # the same with the diagnostics folded into the last substep
            dev.set_step_diagnostics(True)
            fold_step_ms = timed(lambda: dev.integrate_step(DT), steps)
            fold_both_ms = timed(lambda: (dev.integrate_step(DT), diag()), steps)
            dev.set_step_diagnostics(False)
            out[flav] = {"ms_per_step": step_ms, "ms_per_step_with_diagnostics": both_ms,
                         "ms_per_reduction": red_ms,
                         "cell_updates_per_s_with_diagnostics":
                             ranks.world * n ** 3 / (both_ms * 1e-3),
                         "folded": {"ms_per_step": fold_step_ms,
                                    "ms_per_step_with_diagnostics": fold_both_ms,
                                    "diagnostics_share_of_step":
                                        (fold_both_ms - step_ms) / fold_both_ms,
                                    "cell_updates_per_s_with_diagnostics":
                                        ranks.world * n ** 3 / (fold_both_ms * 1e-3)}}
        finally:
            dev.destroy()
            del host
            torch.cuda.empty_cache()
    return out


def diagnostics_errors(n: int, steps: int, gpu: int) -> dict:
    """FP32 and FP64 against the f64 oracle (row-wise form, OpenMP) over
    `steps` RK3 steps of the diagnostics workload: after every step the four
    diagnostics (relative error; the oracle's sums in long double) and at the
    end every field (normwise, interior)."""
    import torch

    sys.path.insert(0, os.path.join(HERE, "tests"))
    import oracle_lib as O
    from astaroth_b200 import Device, abi

    t0 = time.perf_counter()
    host = host_mesh("sp", n, velocity_mode=0.0)
    om = O.OracleMesh("f64", host.fields, n, n, n)
    p = O.params_from(workload_info(abi.DP, n))
    want = []
    for _ in range(steps):
        om.step(p, DT)
        want.append(om.diagnostics())
    out = {"steps": steps, "oracle": "f64, row-wise form", "oracle_seconds": time.perf_counter() - t0,
           "oracle_threads": O.omp_threads(),
           "metric": "per step: max over the four diagnostics of |x - x_oracle| / |x_oracle| "
                     "(min |u| against max |u|, the scale of the field); fields: "
                     "max|x - x_oracle| / max|x_oracle| per field after the last step"}
    U = (abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
    g = abi.NGHOST
    cells = n ** 3
    for flav in ("sp", "dp"):
        h = host if flav == "sp" else host_mesh("dp", n, velocity_mode=0.0)
        dev = Device(flav, h.info, gpu)
        try:
            dev.load_mesh(h)
            per_step = []
            for k in range(steps):
                dev.integrate_step(DT)
                got = (dev.reduce_vec_double(abi.RTYPE_MAX, *U),
                       dev.reduce_vec_double(abi.RTYPE_MIN, *U),
                       math.sqrt(dev.reduce_vec_double(abi.RTYPE_RMS, *U) / cells),
                       math.sqrt(dev.reduce_scal_double(abi.RTYPE_RMS_EXP, abi.VTXBUF_LNRHO)
                                 / cells))
                w_ = want[k]
                scale = (w_[0], w_[0], w_[2], w_[3])  # min |u| against max |u|
                per_step.append(max(abs(a - b) / abs(c) for a, b, c in zip(got, w_, scale)))
            dev.synchronize()
            fields = []
            for w in range(8):
                a = torch.from_numpy(dev.store_double(w)).cuda()[g:-g, g:-g, g:-g]
                b = torch.from_numpy(om.interior(w)).cuda()
                fields.append(float((a - b).abs().max()) / float(b.abs().max()))
                del a, b
            out[flav] = {"diagnostics_max_rel_error": max(per_step),
                         "diagnostics_rel_error_last_step": per_step[-1],
                         "fields": fields, "fields_max": max(fields)}
        finally:
            dev.destroy()
            torch.cuda.empty_cache()
    return out


def cfl_run(sizes, steps: int, warmup: int, ranks, gpu: int) -> dict:
    """Simulation loops whose time step follows the state (FP32, seeded state
    of the headline workload at smaller n, AC_cdt = 0.4, AC_cdtv = 0.3): the
    reference standalone's loop, each step a synchronising max |u| reduction
    read back, the Courant time step on the host (host_timestep) and an RK3
    step, against acDeviceIntegrateStepsCFL, where the reduction, the time
    step and the RK3 step run on the device from one CUDA graph per step.
    Steps per second of each, timed by CUDA events on the Device's stream."""
    import torch

    from astaroth_b200 import Device, abi

    def host_timestep(info, umax):
        g = lambda k: abi.get_real(info, k)  # noqa: E731
        dsmin = min(g("dsx"), g("dsy"), g("dsz"))
        uu_dt = g("cdt") * dsmin / (abs(umax) + math.sqrt(g("cs2_sound")))
        visc_dt = g("cdtv") * dsmin * dsmin / max(g("nu_visc"), g("eta"), g("gamma"), 0.0)
        return min(uu_dt, visc_dt)

    out = {"precision": "FP32", "steps": steps,
           "host_loop": "acDeviceReduceVec(MAX |u|) read back + host_timestep + acDeviceIntegrateStep",
           "device_loop": "acDeviceIntegrateStepsCFL (reduction, time step, RK3 step in one graph)"}
    for n in sizes:
        host = host_mesh("sp", n)
        abi.set_real(host.info, "cs2_sound", 1.0)
        dev = Device("sp", host.info, gpu)
        try:
            dev.load_mesh(host)
            st = torch.cuda.ExternalStream(dev.cuda_stream(0))

            def host_step():
                u = dev.reduce_vec(abi.RTYPE_MAX, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
                dev.integrate_step(host_timestep(host.info, u))

            def timed(fn, k):
                for _ in range(warmup):
                    fn()
                dev.synchronize()
                ranks.barrier()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(k):
                    fn()
                e1.record(st)
                e1.synchronize()
                return ranks.max(e0.elapsed_time(e1)) / k

            host_ms = timed(host_step, steps)
            dev_ms = timed(lambda: dev.integrate_steps_cfl(1), steps)
            dt, t, k = dev.timestep_record()
            out[f"{n}^3"] = {"host_loop_ms_per_step": host_ms, "device_loop_ms_per_step": dev_ms,
                             "speedup": host_ms / dev_ms, "last_dt": dt, "device_steps": k}
        finally:
            dev.destroy()
            del host
            torch.cuda.empty_cache()
    return out


def profile_traffic(name: str, n: int):
    """DRAM bytes per solve launch of an n^3 step from a committed ncu capture
    (profiles/<name>, JSON): the mean over the step's three launches (s = 2 as
    recorded in the file) of dram__bytes_read.sum + dram__bytes_write.sum,
    scaled from the captured mesh by the cells (a launch's bytes grow with the
    cells it updates); None when the file is absent."""
    path = os.path.join(HERE, "profiles", name)
    try:
        with open(path) as f:
            p = json.load(f)
        launches = p["launches"]
        per = []
        for s in ("s0", "s1", "s2"):
            rec = launches.get(s) or launches[p[s + "_as"]]
            per.append(rec["dram_bytes_read"] + rec["dram_bytes_write"])
        return sum(per) / len(per) * n ** 3 / p["cells"]
    except (OSError, KeyError, ValueError, TypeError):
        return None


def measured_peak_hbm():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def config_block(n: int, world: int) -> dict:
    return {"workload": f"MHD RK3, {n}^3, 8 fields, mixed precision (FP32 RHS, compensated state "
                        f"FP32 hi + bf16 lo, FP64 reductions); seeded 1e-3 noise + k=2 velocity "
                        f"mode 0.1",
            "mesh": [n, n, n], "fields": 8, "dt": DT, "dx": "2*pi/n", "nu": 5e-3, "eta": 5e-3,
            "cs": 1.0, "gamma": 5.0 / 3.0, "cp": 1.0,
            "step": "3 x (periodic ghost fill + fused solve launch + swap) through the C ABI",
            "l2": "inputs larger than L2 (8.9 GB per state block); no flush",
            "parallelism": f"replicas x{world}" if world > 1 else "single device"}


def run_reference(args) -> None:
    """The reference's own host solver on the box's cores: `steps` RK3 steps of
    a 64^3 sample of the headline physics (the faster of its two builds), and
    two steps of a 128^3 sample beside it. Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return  # the reference CPU arm runs on rank 0 only
    r = cpu_reference_sample(n=64, max_steps=args.steps, warmup=args.warmup)
    r128 = cpu_reference_sample(n=128, max_steps=2, warmup=0, build=r["build"])
    cfg = config_block(64, 1)
    cfg["workload"] = ("the headline workload's physics (seeded 1e-3 noise + k=2 velocity mode "
                       "0.1, nu = eta = 5e-3, dt = 1e-3, dx = 2 pi / n) on a 64^3 sample; the "
                       "reference's host solver in FP32")
    cfg["samples"] = {"64^3": {k: r[k] for k in ("value", "ms_per_step", "steps")},
                      "128^3": {k: r128[k] for k in ("value", "ms_per_step", "steps")}}
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference", "config": cfg,
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch

    from astaroth_b200 import Device, abi

    ranks = Ranks(args.gpus)
    gpu = ranks.local
    torch.cuda.set_device(gpu)
    n = args.n
    arm = args.flavour  # the measured library (the mixed build unless asked)
    host = host_mesh(arm, n)
    dev = Device(arm, host.info, gpu)
    tile_config = dev.solve_config()[2]  # the library's default tile configuration
    dev.load_mesh(host)
    res = timed_steps(dev, args.steps, args.warmup, ranks, sample_clocks=True, gpu_index=gpu)
    value = ranks.throughput(n ** 3, args.steps, res["total_ms"])  # total_ms: max over ranks

    # roofline of the dominant kernel (the fused solve): algorithmic bytes per
    # launch over the average launch time from the events around every launch
    alg = alg_bytes_per_step(arm, n)
    achieved_gbs = alg * args.steps / (res["solve_ms_total"] * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    # DRAM bytes per solve launch at this size (mean over the step's three
    # launches), from the committed ncu capture of a 256^3 step scaled by the
    # cells (bytes grow with them)
    traffic = profile_traffic(f"solve_{arm}_256.json", n)

    variants = {}
    errors = None
    if not args.no_variants:
        # the same warmup + steps from the same float32 initial values
        side = {}
        for flav in ("dp", "sp"):
            h = host_mesh(flav, n)
            d = Device(flav, h.info, gpu)
            d.load_mesh(h)
            del h
            r = timed_steps(d, args.steps, args.warmup, ranks)
            variants[flav] = {
                "value": ranks.world * n ** 3 * args.steps / (r["total_ms"] * 1e-3),
                "ms_per_step": r["ms_per_step"],
                "solve_ms_per_substep": r["solve_ms_per_substep"],
                "solve_hbm_gbs_alg": alg_bytes_per_step(flav, n) * args.steps
                / (r["solve_ms_total"] * 1e-3) / 1e9}
            side[flav] = d
        # per-field normwise error (interior) after warmup + steps steps
        errors = {"metric": "max|x - x_fp64| / max|x_fp64| per field after "
                            f"{args.warmup + args.steps} steps",
                  "fields": list(abi.VTXBUFS),
                  "mixed_vs_fp64": field_errors(dev, side["dp"], n),
                  "fp32_vs_fp64": field_errors(side["sp"], side["dp"], n)}
        for d in side.values():
            d.destroy()
        variants["speedup_mixed_over_fp64"] = value / variants["dp"]["value"]
    dev.destroy()
    del host
    torch.cuda.empty_cache()
    # the oracle runs on the host cores: one-GPU runs only
    check = not args.no_oracle and ranks.world == 1
    if check:
        errors = errors or {}
        errors["vs_oracle"] = oracle_errors(n, 2, gpu)

    e2e = None
    if not args.no_e2e:
        h = host_mesh("mixed", n)
        e = e2e_run("mixed", h, args.steps, ranks)
        e2e = {"value": e["cells_per_s"], "unit": UNIT,
               "h2d_bytes_per_step": e["h2d_bytes_per_step"],
               "d2h_bytes_per_step": e["d2h_bytes_per_step"],
               "includes": "mesh load from pinned host, per-step max|u| (folded into the step's "
                           "last substep) read back, mesh store"}
        del h

    ensemble = None
    if not args.no_ensemble:
        ensemble = ensemble_run(min(args.steps, 20), ranks)

    diagnostics = None
    if not args.no_diagnostics:
        diagnostics = diagnostics_run(256, 100, max(args.warmup, 3), ranks, gpu,
                                      check_steps=100 if check else 0)

    cfl = None
    if not args.no_cfl:
        cfl = cfl_run((64, 128), 200, max(args.warmup, 3), ranks, gpu)

    forced = None
    if not args.no_forced:
        torch.cuda.empty_cache()
        forced = forced_run(args.forced_n, min(args.steps, 20), max(args.warmup, 3), ranks, gpu)

    # the reference host solver's baseline: one process on the host cores, so
    # only in a one-GPU run (a multi-rank run reports none)
    cpu = cpu_all = None
    if ranks.world == 1 and not args.no_cpu:
        c = cpu_reference_sample(budget_s=12.0)
        cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cpu_all = cpu_oracle_sample()

    if ranks.rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": {"mixed": "f32 (compensated state: f32 hi + bf16 lo, f64 reductions)",
                          "sp": "f32", "dp": "f64"}[arm],
                "data": "synthetic",
                "config": config_block(n, ranks.world),
                "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak,
                             "unit": "GB/s", "frac": achieved_gbs / peak,
                             "traffic": traffic, "peak_source": peak_kind,
                             "kernel": f"solve_kernel ({arm}, {tile_config})",
                             "alg_bytes_per_cell_step": alg // n ** 3,
                             "solve_ms_per_substep": res["solve_ms_per_substep"]},
                "clocks": res["clocks"], "gpu_launches": res["launches"],
                "e2e": e2e, "cpu_baseline": cpu, "cpu_oracle_all_cores": cpu_all,
                "variants": variants, "errors": errors,
                "ensemble": ensemble, "diagnostics_256": diagnostics, "cfl_loop": cfl,
                "forced": forced}
        print(json.dumps(line), flush=True)
    ranks.close()


def main(argv=None) -> None:
    args = parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

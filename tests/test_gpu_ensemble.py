"""Ensembles (include/astaroth_b200.h acEnsemble*): many meshes of uneven sizes
and parameters advanced by one launch per substep. Every member must equal,
bit for bit, the same mesh advanced alone through the Device interface, for
every tile configuration and z-segment length, with and without graph replay;
the autotuner must keep the members' states and cache its choice.
"""
import math
import os

import numpy as np
import pytest

from astaroth_b200 import Device, Ensemble, abi, init

pytestmark = pytest.mark.gpu

SIZES = [(24, 24, 24), (37, 29, 23), (48, 32, 40), (16, 16, 64), (32, 48, 20), (136, 12, 8)]


def member_info(prec, n, k):
    nx, ny, nz = n
    rng = np.random.default_rng(100 + k)
    nu, eta = 10 ** rng.uniform(-3, -2, 2)
    return abi.make_info(prec, nx, ny, nz, dsx=2 * math.pi / nx, dsy=2 * math.pi / ny,
                         dsz=2 * math.pi / nz, gamma=5 / 3, nu_visc=nu, eta=eta)


def member_fields(prec, n, k):
    return init.workload_fields(*n, prec.np_dtype, seed=k + 1, amplitude=0.02, velocity_mode=0.05)


def single_results(flavour, steps, dt):
    prec = abi.PRECISIONS[flavour]
    out = []
    for k, n in enumerate(SIZES):
        info = member_info(prec, n, k)
        host = abi.HostMesh(prec, info, member_fields(prec, n, k))
        with Device(flavour, info) as dev:
            dev.load_mesh(host)
            for _ in range(steps):
                dev.integrate_step(dt)
            dev.store_mesh(host)
        out.append([f.copy() for f in host.fields])
    return out


def run_ensemble(flavour, steps, dt, schedule=None, graph=False):
    prec = abi.PRECISIONS[flavour]
    infos = [member_info(prec, n, k) for k, n in enumerate(SIZES)]
    with Ensemble(flavour, infos) as ens:
        if schedule is not None:
            ens.set_schedule(*schedule)
        for k, n in enumerate(SIZES):
            ens.load_member(k, abi.HostMesh(prec, infos[k], member_fields(prec, n, k)))
        if graph:
            ens.integrate_steps(dt, steps)
        else:
            for _ in range(steps):
                ens.integrate_step(dt)
        ens.synchronize()
        assert ens.status() == 0
        res = []
        for k in range(len(SIZES)):
            h = abi.HostMesh(prec, infos[k])
            ens.store_member(k, h)
            res.append(h.fields)
    return res


@pytest.mark.parametrize("flavour", ["sp", "dp", "mixed"])
def test_ensemble_members_equal_single_meshes(flavour):
    ref = single_results(flavour, 3, 1e-3)
    got = run_ensemble(flavour, 3, 1e-3)
    for k in range(len(SIZES)):
        for w in range(8):
            assert np.array_equal(got[k][w], ref[k][w]), (k, w)


@pytest.mark.parametrize("schedule,graph", [((0, 0), True), ((1, 16), False), ((2, 32), True),
                                            ((0, 64), False)])
def test_ensemble_schedules_and_graphs_bitwise(schedule, graph):
    ref = single_results("sp", 2, 1e-3)
    got = run_ensemble("sp", 2, 1e-3, schedule=schedule, graph=graph)
    for k in range(len(SIZES)):
        for w in range(8):
            assert np.array_equal(got[k][w], ref[k][w]), (schedule, k, w)


def test_autotuner_keeps_state_and_caches(tmp_path):
    prec = abi.SP
    infos = [member_info(prec, n, k) for k, n in enumerate(SIZES)]
    cache = str(tmp_path / "tune.txt")
    with Ensemble("sp", infos) as ens:
        for k, n in enumerate(SIZES):
            ens.load_member(k, abi.HostMesh(prec, infos[k], member_fields(prec, n, k)))
        ens.integrate_step(1e-3)
        before = []
        for k in range(len(SIZES)):
            h = abi.HostMesh(prec, infos[k])
            ens.store_member(k, h)
            before.append(h.fields)
        ens.auto_optimize(cache)
        chosen = ens.schedule()
        for k in range(len(SIZES)):
            h = abi.HostMesh(prec, infos[k])
            ens.store_member(k, h)
            for w in range(8):
                assert np.array_equal(h.fields[w], before[k][w])
    text = open(cache).read().split()
    assert len(text) == 3 and int(text[1]) == chosen[0] and int(text[2]) == chosen[1]
    with Ensemble("sp", infos) as ens2:  # a second ensemble of the same sizes reads the cache
        ens2.auto_optimize(cache)
        assert ens2.schedule() == chosen
    assert len(open(cache).read().split()) == 3


def test_ensemble_larger_than_one_launch_group():
    """An ensemble of more members than one launch carries parameters for (64)
    runs in several launches per substep; every member must still equal its
    mesh advanced alone, bit for bit."""
    prec = abi.SP
    sizes = [(8 + k % 5, 7 + k % 3, 6 + k % 4) for k in range(70)]
    infos = [member_info(prec, n, k) for k, n in enumerate(sizes)]
    fields = [member_fields(prec, n, k) for k, n in enumerate(sizes)]
    with Ensemble("sp", infos) as ens:
        for k in range(len(sizes)):
            ens.load_member(k, abi.HostMesh(prec, infos[k], fields[k]))
        ens.integrate_step(1e-3)
        ens.synchronize()
        assert ens.status() == 0
        got = []
        for k in range(len(sizes)):
            h = abi.HostMesh(prec, infos[k])
            ens.store_member(k, h)
            got.append(h.fields)
    for k in range(len(sizes)):  # members of both launch groups
        host = abi.HostMesh(prec, infos[k], [f.copy() for f in fields[k]])
        with Device("sp", infos[k]) as dev:
            dev.load_mesh(host)
            dev.integrate_step(1e-3)
            dev.store_mesh(host)
        for w in range(8):
            assert np.array_equal(got[k][w], host.fields[w]), (k, w)

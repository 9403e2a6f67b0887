"""Steps whose time step is chosen on the device (include/astaroth_b200.h
acDeviceIntegrateStepCFL, acDeviceIntegrateStepsCFL, acDeviceGetTimestepRecord,
acDeviceSetSimulationTime).

The reference standalone picks each step's dt on the host from a synchronising
max |u| reduction (samples/standalone/simulation.cc:429-436) and
host_timestep (samples/standalone/model/host_timestep.cc:33-60). Here the same
formula runs on the device. Each step must use exactly the dt that a host loop
computes from acDeviceReduceVec(RTYPE_MAX) with that formula in double
precision, and so must leave the same state bit for bit as that loop through
acDeviceIntegrateStep. The dt must also lie within one AcReal ulp (two in
double precision) of the reference's own long-double host_timestep, compiled
into oracle/_ref. Graph replay must equal single steps.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

import oracle_lib as O
from astaroth_b200 import Device, abi, init
from astaroth_b200.device import AcError

pytestmark = pytest.mark.gpu

FLAVOURS = ["sp", "dp", "mixed"]
N = 32
STEPS = 5


def workload(flavour, **over):
    prec = abi.PRECISIONS[flavour]
    ds = 2 * math.pi / N
    # cdt small enough that the advective limit, which depends on max|u|,
    # binds (about 3.4e-3 here; the viscous limit with gamma = 5/3 is 6.9e-3)
    kw = dict(dsx=ds, dsy=ds, dsz=ds, gamma=5 / 3, nu_visc=5e-3, eta=5e-3, cs2_sound=1.0,
              cdt=0.02, cdtv=0.3)
    kw.update(over)
    info = abi.make_info(prec, N, **kw)
    abi.set_real(info, "dsmin", ds)  # as the standalone's config loader sets it
    fields = init.workload_fields(N, N, N, prec.np_dtype, seed=3, amplitude=1e-3,
                                  velocity_mode=0.1)
    return prec, info, fields


def reference_dt(flavour, info, umax):
    """The reference standalone's host_timestep (long double), compiled
    unchanged into oracle/_ref, or None where it was not built."""
    kind = "dp" if flavour == "dp" else "sp"
    path = os.path.join(O.ORACLE_DIR, "_ref", f"libref_timestep_{kind}.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.ref_host_timestep.argtypes = [C.c_double, C.c_void_p, C.c_double]
    lib.ref_host_timestep.restype = C.c_double
    return lib.ref_host_timestep(umax, C.addressof(info), 1.0)


def stored(dev, prec, info):
    h = abi.HostMesh(prec, info)
    dev.store_mesh(h)
    return [f.copy() for f in h.fields]


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_device_time_step_equals_host_loop(flavour):
    prec, info, fields = workload(flavour)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    with Device(flavour, info) as a, Device(flavour, info) as b:
        a.load_mesh(host)
        b.load_mesh(host)
        a.set_simulation_time(0.25)
        t_host, dts = 0.25, []
        for k in range(STEPS):
            a.integrate_step_cfl()
            dt_dev, t_dev, steps = a.timestep_record()
            # the host loop of the reference standalone, through the C ABI
            umax = b.reduce_vec(abi.RTYPE_MAX, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
            dt = O.cfl_dt(prec, info, umax)
            assert dt_dev == dt, (k, dt_dev, dt)
            ref = reference_dt(flavour, info, umax)
            if ref is not None:
                ulp = float(np.spacing(prec.np_dtype(ref)))
                assert abs(dt_dev - ref) <= (2 if prec.double else 1) * ulp, (k, dt_dev, ref)
            b.integrate_step(dt)
            t_host += dt
            dts.append(dt)
            assert steps == k + 1
            assert t_dev == t_host
        # the advective limit bound (dt followed max|u|), not the viscous one
        ds = 2 * math.pi / N
        visc_dt = 0.3 * ds * ds / (5 / 3)
        assert max(dts) < 0.9 * visc_dt
        assert a.status() == 0
        got, want = stored(a, prec, info), stored(b, prec, info)
    for w in range(8):
        assert np.array_equal(got[w], want[w]), w


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_device_time_step_graph_replay_bitwise(flavour):
    prec, info, fields = workload(flavour)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    with Device(flavour, info) as a, Device(flavour, info) as c:
        a.load_mesh(host)
        c.load_mesh(host)
        for _ in range(STEPS):
            a.integrate_step_cfl(0.5)
        c.integrate_steps_cfl(2, 0.5)
        c.integrate_steps_cfl(STEPS - 2, 0.5)
        assert a.timestep_record() == c.timestep_record()
        got, want = stored(c, prec, info), stored(a, prec, info)
    for w in range(8):
        assert np.array_equal(got[w], want[w]), w


def test_device_time_step_refuses_what_it_cannot_choose():
    prec, info, fields = workload("sp", cdt=0.0)
    with Device("sp", info) as d:
        d.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
        with pytest.raises(AcError):
            d.integrate_step_cfl()
        with pytest.raises(AcError):
            d.integrate_steps_cfl(2)
        _, _, steps = d.timestep_record()
        assert steps == 0
    prec, info, fields = workload("sp")
    with Device("sp", info) as d:
        d.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
        with pytest.raises(AcError):
            d.integrate_step_cfl(0.0)
        d.set_forcing(True)
        with pytest.raises(AcError):
            d.integrate_step_cfl()
        d.set_forcing(False)
        d.integrate_step_cfl()
        assert d.timestep_record()[2] == 1

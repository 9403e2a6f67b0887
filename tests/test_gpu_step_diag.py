"""Step diagnostics folded into the last substep (acDeviceSetStepDiagnostics).

With them enabled, substep 2 over the whole interior also accumulates max, min
and sum of |u|^2 and sum of exp(lnrho)^2 of the state it writes; the step's
diagnostics (acDeviceReduceVec MAX / MIN / RMS of u, acDeviceReduceScal RMS_EXP
of lnrho) then come from that record. Checked here, for every build:
  - the states equal those of the same steps without the diagnostics, bit for bit;
  - MAX and MIN equal a separate reduction pass bit for bit, RMS and RMS_EXP
    within 1e-12 relative (their summation order differs);
  - single steps, graph-replayed steps, forced steps and steps whose time step
    the device chooses;
  - the four requests launch nothing once the step has run; a load drops the
    record; other fields are never served from it.
"""
import numpy as np
import pytest

from astaroth_b200 import Device, abi, init
from astaroth_b200.device import ForcingGenerator

pytestmark = pytest.mark.gpu
U = (abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
A = (abi.VTXBUF_AX, abi.VTXBUF_AY, abi.VTXBUF_AZ)


def info_for(prec, dims, **kw):
    nx, ny, nz = dims
    return abi.make_info(prec, nx, ny, nz, dsx=0.2, dsy=0.17, dsz=0.23, gamma=5 / 3,
                         nu_visc=5e-3, eta=5e-3, cs_sound=1.0, cp_sound=1.0, **kw)


def diagnostics(dev):
    return (dev.reduce_vec_double(abi.RTYPE_MAX, *U), dev.reduce_vec_double(abi.RTYPE_MIN, *U),
            dev.reduce_vec_double(abi.RTYPE_RMS, *U),
            dev.reduce_scal_double(abi.RTYPE_RMS_EXP, abi.VTXBUF_LNRHO))


def check_same(folded, separate):
    assert folded[0] == separate[0] and folded[1] == separate[1], (folded, separate)
    for q in (2, 3):
        assert folded[q] == pytest.approx(separate[q], rel=1e-12), (q, folded, separate)


def states(dev):
    return [dev.store_double(w) for w in range(8)]


@pytest.mark.parametrize("flavour", ["sp", "dp", "mixed"])
@pytest.mark.parametrize("mode", ["steps", "graph", "forced", "cfl"])
def test_folded_diagnostics_equal_a_separate_pass(flavour, mode):
    prec = abi.PRECISIONS[flavour]
    dims = (37, 29, 23)
    extra = dict(kmin=1.0, kmax=3.0, relhel=0.3, forcing_magnitude=0.05) if mode == "forced" else {}
    info = info_for(prec, dims, **extra)
    fields = init.workload_fields(*dims, prec.np_dtype, seed=9, amplitude=0.02, velocity_mode=0.1)
    dt = float(prec.np_dtype(1e-3))
    gen = ForcingGenerator(flavour, info, seed=3) if mode == "forced" else None
    params = [gen.next() for _ in range(3)] if gen else None
    runs = {}
    for folded in (False, True):
        with Device(flavour, info) as dev:
            dev.set_step_diagnostics(folded)
            dev.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
            if mode == "forced":
                dev.set_forcing(True)
            got = []
            for k in range(3):
                if mode == "steps":
                    dev.integrate_step(dt)
                elif mode == "graph":
                    dev.integrate_steps(dt, 1)
                elif mode == "forced":
                    dev.load_forcing_params(params[k])
                    dev.integrate_step(dt)
                else:
                    dev.integrate_steps_cfl(1)
                before = dev.launch_count()
                got.append(diagnostics(dev))
                launched = dev.launch_count() - before
                if folded:
                    assert launched == 0, (k, launched)  # served from the record
                else:
                    assert launched == 2  # the MAX/MIN/RMS pass and the RMS_EXP pass
            dev.synchronize()
            assert dev.status() == 0
            runs[folded] = (got, states(dev))
    for k in range(3):
        check_same(runs[True][0][k], runs[False][0][k])
    for w in range(8):
        assert np.array_equal(runs[True][1][w], runs[False][1][w]), w


@pytest.mark.parametrize("flavour", ["sp", "mixed"])
def test_record_is_dropped_when_the_block_changes_and_serves_only_its_fields(flavour):
    prec = abi.PRECISIONS[flavour]
    dims = (24, 20, 16)
    info = info_for(prec, dims)
    a = init.workload_fields(*dims, prec.np_dtype, seed=1, amplitude=0.02, velocity_mode=0.1)
    b = init.workload_fields(*dims, prec.np_dtype, seed=2, amplitude=0.05, velocity_mode=0.2)
    with Device(flavour, info) as dev, Device(flavour, info) as ref:
        dev.set_step_diagnostics(True)
        dev.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in a]))
        dev.integrate_step(1e-3)
        diagnostics(dev)
        # other fields and other reduction types run their own pass
        n0 = dev.launch_count()
        dev.reduce_vec_double(abi.RTYPE_MAX, *A)
        dev.reduce_scal_double(abi.RTYPE_RMS_EXP, abi.VTXBUF_ENTROPY)
        dev.reduce_vec_double(abi.RTYPE_SUM, *U)
        assert dev.launch_count() - n0 == 3
        # a load changes the block: the next requests read the new state
        dev.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in b]))
        n0 = dev.launch_count()
        after = diagnostics(dev)
        assert dev.launch_count() - n0 == 2
        ref.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in b]))
        assert after == diagnostics(ref)
        # a step over a sub-box does not fold (and the record stays dropped)
        s, e = abi.int3(4, 4, 4), abi.int3(20, 18, 15)
        for step in range(3):
            dev.integrate_substep(step, 1e-3, s, e)
            dev.swap_buffers()
        n0 = dev.launch_count()
        diagnostics(dev)
        assert dev.launch_count() - n0 == 2

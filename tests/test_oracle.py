"""Pins the CPU oracle (oracle/mhd_oracle.c) against the reference's own host
model. Runs without a GPU.

- golden fixtures (tests/golden/ref_*.npz) were produced by the reference's
  src/utils/modelsolver.c + modelreduce.c (see tests/golden/make_golden.py);
- where the reference build is present (oracle/_ref), it is also run live on
  other sizes.
Tolerances: the double and float builds follow the reference's arithmetic
order and are expected to agree to rounding (bit-exact in practice); the long
double build must agree with the double reference to 1e-13 normwise.
"""
import glob
import math
import os

import numpy as np
import pytest

from astaroth_b200 import abi, init
import oracle_lib as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))
PHYS = dict(gamma=5.0 / 3.0, nu_visc=5e-3, eta=5e-3, cs_sound=1.0, cp_sound=1.0)
RTYPES = (0, 1, 2, 3, 7)  # MAX MIN RMS RMS_EXP SUM


def _case(path):
    d = np.load(path)
    nx, ny, nz, steps = (int(v) for v in d["meta"])
    dt, amp, vel = (float(v) for v in d["dt_amp_vel"])
    pname = os.path.basename(path).split("_")[1]
    return d, pname, nx, ny, nz, steps, dt, amp, vel


def _run_oracle(kind, pname, nx, ny, nz, steps, dt, amp, vel):
    prec = abi.PRECISIONS[pname]
    info = abi.make_info(prec, nx, ny, nz, dsx=2 * math.pi / nx, dsy=2 * math.pi / ny,
                         dsz=2 * math.pi / nz, **PHYS)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=7, amplitude=amp,
                                  velocity_mode=vel)
    om = O.OracleMesh(kind, fields, nx, ny, nz)
    om.step(O.params_from(info), float(prec.np_dtype(dt)), steps)
    om.periodic()
    return om


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 4


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    d, pname, nx, ny, nz, steps, dt, amp, vel = _case(path)
    kind = "f64" if pname == "dp" else "f32"
    om = _run_oracle(kind, pname, nx, ny, nz, steps, dt, amp, vel)
    tol = 1e-15 if pname == "dp" else 1e-7
    for w in range(8):
        err = O.normwise_error(om.fields[w], d[f"f{w}"])
        assert err <= tol, (w, err)
    # reductions, in the reference's order: per rtype, 8 scalar fields then uu, aa
    red = d["reductions"]
    k = 0
    for rt in RTYPES:
        for w in range(8):
            v = om.reduce(rt, [w])
            assert v == pytest.approx(red[k], rel=tol * 10, abs=1e-30), (rt, w)
            k += 1
        for h in ([1, 2, 3], [4, 5, 6]):
            v = om.reduce(rt, h)
            assert v == pytest.approx(red[k], rel=tol * 10, abs=1e-30), (rt, h)
            k += 1


@pytest.mark.parametrize("path", [p for p in GOLDEN if "_dp_" in p],
                         ids=lambda p: os.path.basename(p))
def test_long_double_oracle_close_to_reference(path):
    d, pname, nx, ny, nz, steps, dt, amp, vel = _case(path)
    om = _run_oracle("f80", pname, nx, ny, nz, steps, dt, amp, vel)
    for w in range(8):
        assert O.normwise_error(d[f"f{w}"], om.fields[w]) <= 1e-13


@pytest.mark.parametrize("pname,n", [("dp", (12, 8, 10)), ("sp", (10, 12, 8))])
def test_oracle_matches_reference_live(pname, n):
    lib = O.ref_lib(pname)
    if lib is None:
        pytest.skip("reference host utils not built here (no reference sources)")
    prec = abi.PRECISIONS[pname]
    nx, ny, nz = n
    info = abi.make_info(prec, nx, ny, nz, dsx=0.3, dsy=0.25, dsz=0.2, **PHYS)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=3, amplitude=0.2)
    hm = abi.HostMesh(prec, info, [f.copy() for f in fields])
    lib.acHostIntegrateStep(hm.cmesh, prec.real(2e-3))
    om = O.OracleMesh("f64" if pname == "dp" else "f32", fields, nx, ny, nz)
    om.step(O.params_from(info), float(prec.np_dtype(2e-3)))
    for w in range(8):
        assert O.normwise_error(om.interior(w), hm.interior(w)) <= (1e-15 if pname == "dp" else 1e-7)


def test_periodic_fill_matches_numpy_wrap():
    nx, ny, nz = 7, 9, 8
    rng = np.random.default_rng(0)
    inter = [rng.standard_normal((nz, ny, nx)) for _ in range(8)]
    full = [np.zeros((nz + 6, ny + 6, nx + 6)) for _ in range(8)]
    for w in range(8):
        full[w][3:-3, 3:-3, 3:-3] = inter[w]
    om = O.OracleMesh("f64", full, nx, ny, nz)
    om.periodic()
    for w in range(8):
        assert np.array_equal(om.fields[w], init.wrap_ghosts(inter[w]))


@pytest.mark.parametrize("kind", ["f32", "f64"])
@pytest.mark.parametrize("forcing", [False, True])
def test_rowwise_step_equals_vertexwise_step(kind, forcing):
    """The oracle's row-wise step (oracle_step_rows, used at large sizes) is
    the vertex-wise step (oracle_step, the restatement of modelsolver.c)
    evaluated in another loop order: equal bit for bit, forcing included."""
    nx, ny, nz = 19, 13, 11
    dtype = O.KIND_DTYPE[kind]
    prec = abi.SP if kind == "f32" else abi.DP
    info = abi.make_info(prec, nx, ny, nz, dsx=0.31, dsy=0.27, dsz=0.23, **PHYS)
    fields = init.workload_fields(nx, ny, nz, dtype, seed=17, amplitude=0.3, velocity_mode=0.2)
    extra = {}
    if forcing:
        extra = dict(forcing=1, forcing_magnitude=0.05, forcing_phase=0.4, kaver=1.0,
                     k_force=[1.0, -2.0, 1.0], ff_re=[0.1, 0.2, -0.3], ff_im=[0.3, -0.1, 0.2])
    p = O.params_from(info, **extra)
    a = O.OracleMesh(kind, fields, nx, ny, nz)
    b = O.OracleMesh(kind, fields, nx, ny, nz)
    a.step(p, 2e-3, 2, vertexwise=True)
    b.step(p, 2e-3, 2)
    for w in range(8):
        assert np.array_equal(a.fields[w], b.fields[w]), w
        assert a.fields[w].tobytes() == b.fields[w].tobytes(), w

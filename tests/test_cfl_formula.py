"""The Courant time step that acDeviceIntegrateStepCFL evaluates on the device,
against the reference standalone's own host_timestep
(samples/standalone/model/host_timestep.cc:33-60), compiled unchanged into
oracle/_ref/libref_timestep_{sp,dp}.so.

The GPU tests (tests/test_gpu_cfl.py) check that the device's dt equals
oracle_lib.cfl_dt bit for bit. Here cfl_dt (double precision) is pinned to the
reference function (long double): in single precision within one ulp and
equal for all but a small fraction of cases; in double precision, where the
formula's four roundings in double are not hidden by a final rounding to a
narrower type, within two ulp.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from astaroth_b200 import abi
import oracle_lib as O

REF_DIR = os.path.join(O.ORACLE_DIR, "_ref")


def ref_lib(flavour):
    kind = "dp" if flavour == "dp" else "sp"
    path = os.path.join(REF_DIR, f"libref_timestep_{kind}.so")
    if not os.path.exists(path):
        pytest.skip("reference time step not built (oracle/_ref needs the reference sources)")
    lib = C.CDLL(path)
    lib.ref_host_timestep.argtypes = [C.c_double, C.c_void_p, C.c_double]
    lib.ref_host_timestep.restype = C.c_double
    return lib


@pytest.mark.parametrize("flavour", ["sp", "dp", "mixed"])
def test_device_formula_within_one_ulp_of_reference(flavour):
    prec = abi.PRECISIONS[flavour]
    lib = ref_lib(flavour)
    R = prec.np_dtype
    rng = np.random.default_rng(7)
    exact = total = 0
    for case in range(400):
        n = int(rng.choice([32, 64, 128, 512]))
        ds = [2 * math.pi / n * float(f) for f in rng.uniform(0.5, 2.0, 3)]
        info = abi.make_info(prec, n, dsx=ds[0], dsy=ds[1], dsz=ds[2],
                             cdt=float(rng.uniform(0.01, 0.9)), cdtv=float(rng.uniform(0.05, 0.9)),
                             nu_visc=float(10 ** rng.uniform(-4, -1)),
                             eta=float(10 ** rng.uniform(-4, -1)),
                             gamma=float(rng.choice([5 / 3, 1.0, 0.5, 1e-3])),
                             cs2_sound=float(rng.uniform(0.1, 4.0)))
        # the standalone's config loader sets dsmin (config_loader.cc:102)
        abi.set_real(info, "dsmin", min(abi.get_real(info, k) for k in ("dsx", "dsy", "dsz")))
        ts = float(rng.choice([1.0, 0.5, 0.25]))
        for umax in rng.uniform(0, 3, 5):
            ours = O.cfl_dt(prec, info, float(umax), ts)
            ref = lib.ref_host_timestep(float(R(umax)), C.addressof(info), ts)
            ulp = float(np.spacing(R(abs(ref))))
            assert abs(ours - ref) <= (2 if prec.double else 1) * ulp, (case, umax, ours, ref)
            exact += ours == ref
            total += 1
    if not prec.double:
        assert exact >= 0.99 * total, (exact, total)


def test_device_formula_uses_smallest_spacing_when_dsmin_unset():
    prec = abi.SP
    info = abi.make_info(prec, 64, dsx=0.1, dsy=0.05, dsz=0.2, cs2_sound=1.0)
    assert not abi.get_real(info, "dsmin") > 0  # unset (NaN)
    with_min = abi.make_info(prec, 64, dsx=0.1, dsy=0.05, dsz=0.2, cs2_sound=1.0, dsmin=0.05)
    assert O.cfl_dt(prec, info, 0.3) == O.cfl_dt(prec, with_min, 0.3)

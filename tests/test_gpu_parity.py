"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (normwise per field: max|cand - model| / max|model| over the interior):
  FP32  <= 1e-5     FP64 <= 1e-12     mixed <= 1e-6
against the long-double oracle (the f64 oracle at 256^3 and above, where the
long-double build would take minutes); mixed also <= 1e-6 against the FP64 GPU
path.
Load/store, ghost fill, sub-box updates, graph replay and tile choice are
checked bit-exactly. Full-size behaviour is checked through size-independent
properties (periodic-shift equivariance, reductions of a stored mesh).
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

from astaroth_b200 import Device, abi, init
import oracle_lib as O

pytestmark = pytest.mark.gpu
FLAVOURS = ("sp", "dp", "mixed")
TOL = {"sp": 1e-5, "dp": 1e-12, "mixed": 1e-6}
PHYS = dict(gamma=5.0 / 3.0, nu_visc=5e-3, eta=5e-3, cs_sound=1.0, cp_sound=1.0)


def workload_info(prec, nx, ny=None, nz=None, **kw):
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = dict(PHYS)
    p.update(kw)
    return abi.make_info(prec, nx, ny, nz, dsx=2 * math.pi / nx, dsy=2 * math.pi / ny,
                         dsz=2 * math.pi / nz, **p)


def new_device(flavour, info):
    return Device(flavour, info)


def run_gpu(flavour, fields, info, dt, steps, graph=False):
    prec = abi.PRECISIONS[flavour]
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        if graph:
            dev.integrate_steps(dt, steps)
        else:
            for _ in range(steps):
                dev.integrate_step(dt)
        dev.periodic_boundconds()
        dev.synchronize()
        assert dev.status() == 0
        out = [dev.store_double(w) for w in range(8)]
    return out


def interior(a):
    g = abi.NGHOST
    return a[g:-g, g:-g, g:-g]


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_load_store_roundtrip(flavour):
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz = 37, 29, 23
    info = abi.make_info(prec, nx, ny, nz)
    rng = np.random.default_rng(1)
    fields = [rng.standard_normal((nz + 6, ny + 6, nx + 6)).astype(prec.np_dtype) for _ in range(8)]
    host = abi.HostMesh(prec, info, fields)
    back = abi.HostMesh(prec, info)
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        dev.store_mesh(back)
        for w in range(8):
            assert np.array_equal(back.fields[w], fields[w])
        # a flat sub-range that starts and ends mid-row
        part = abi.HostMesh(prec, info)
        start, count = 1234, 5 * (nx + 6) + 17
        k, rem = divmod(start, (nx + 6) * (ny + 6))
        j, i = divmod(rem, nx + 6)
        off = abi.int3(i, j, k)
        rc = dev.lib.acDeviceStoreVertexBufferWithOffset(dev.handle, 0, 3, off, off, count,
                                                         C.byref(part.cmesh))
        assert rc == 0
        dev.synchronize()
        flat = part.fields[3].reshape(-1)
        assert np.array_equal(flat[start:start + count], fields[3].reshape(-1)[start:start + count])


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_periodic_boundconds_exact(flavour):
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz = 21, 18, 13
    info = abi.make_info(prec, nx, ny, nz)
    rng = np.random.default_rng(2)
    inter = [rng.standard_normal((nz, ny, nx)).astype(prec.np_dtype) for _ in range(8)]
    fields = [np.zeros((nz + 6, ny + 6, nx + 6), prec.np_dtype) for _ in range(8)]
    for f, v in zip(fields, inter):
        f[3:-3, 3:-3, 3:-3] = v
    host = abi.HostMesh(prec, info, fields)
    back = abi.HostMesh(prec, info)
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        dev.periodic_boundconds()
        dev.store_mesh(back)
        for w in range(8):
            assert np.array_equal(back.fields[w], init.wrap_ghosts(inter[w]))
        # a sub-box fill touches only ghost vertices inside the box
        dev.load_mesh(host)
        s, e = abi.int3(0, 2, 1), abi.int3(nx + 6, 9, nz + 6)
        assert dev.lib.acDevicePeriodicBoundcondStep(dev.handle, 0, 5, s, e) == 0
        dev.store_mesh(back)
        want = fields[5].copy()
        full = init.wrap_ghosts(inter[5])
        want[1:, 2:9, :] = full[1:, 2:9, :]
        assert np.array_equal(back.fields[5], want)
        assert np.array_equal(back.fields[4], fields[4])


@pytest.fixture(scope="module")
def oracle_64():
    """Config 1: 64^3, 1e-3 noise (seed 1), dt = 1e-3, 10 steps, long double."""
    n, steps, dt = 64, 10, 1e-3
    info = workload_info(abi.DP, n)
    fields = init.workload_fields(n, n, n, np.float32, seed=1, amplitude=1e-3)
    om = O.OracleMesh("f80", fields, n, n, n)
    om.step(O.params_from(info), float(np.float32(dt)), steps)
    om.periodic()
    return fields, om


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_config1_64cube_10_steps_vs_oracle(flavour, oracle_64):
    fields, om = oracle_64
    prec = abi.PRECISIONS[flavour]
    n, steps, dt = 64, 10, float(np.float32(1e-3))
    info = workload_info(prec, n)
    out = run_gpu(flavour, [f.astype(prec.np_dtype) for f in fields], info, dt, steps)
    errs = [O.normwise_error(interior(out[w]), om.interior(w)) for w in range(8)]
    print(flavour, ["%.2e" % e for e in errs])
    assert max(errs) <= TOL[flavour], errs


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_ragged_mesh_vs_oracle(flavour):
    """Sizes that are not multiples of any tile, anisotropic spacing, larger amplitude."""
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz, steps = 37, 29, 23, 2
    info = abi.make_info(prec, nx, ny, nz, dsx=0.21, dsy=0.17, dsz=0.25, **PHYS)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=11, amplitude=0.05,
                                  velocity_mode=0.1)
    dt = float(prec.np_dtype(2e-3))
    out = run_gpu(flavour, fields, info, dt, steps)
    om = O.OracleMesh("f80", fields, nx, ny, nz)
    om.step(O.params_from(info), dt, steps)
    errs = [O.normwise_error(interior(out[w]), om.interior(w)) for w in range(8)]
    print(flavour, ["%.2e" % e for e in errs])
    assert max(errs) <= TOL[flavour], errs


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_reductions_vs_oracle(flavour):
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz = 40, 33, 26
    info = abi.make_info(prec, nx, ny, nz)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=4, amplitude=0.3)
    host = abi.HostMesh(prec, info, fields)
    om = O.OracleMesh("f80", fields, nx, ny, nz)
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        for rt in (abi.RTYPE_MAX, abi.RTYPE_MIN, abi.RTYPE_RMS, abi.RTYPE_RMS_EXP, abi.RTYPE_SUM):
            for w in (0, 3, 7):
                got = dev.reduce_scal_double(rt, w)
                want = om.reduce(rt, [w], normalise=False)  # device layer: raw sums
                assert got == pytest.approx(want, rel=1e-12, abs=1e-12), (rt, w)
            got = dev.reduce_vec_double(rt, 1, 2, 3)
            want = om.reduce(rt, [1, 2, 3], normalise=False)
            assert got == pytest.approx(want, rel=1e-12, abs=1e-12), rt
            # the AcReal-returning entry points round the same accumulator
            assert dev.reduce_scal(rt, 3) == pytest.approx(dev.reduce_scal_double(rt, 3),
                                                           rel=1e-7 if prec.np_dtype == np.float32 else 1e-15)
        # unsupported types fail instead of returning garbage
        with pytest.raises(Exception):
            dev.reduce_scal(abi.RTYPE_ALFVEN_MAX, 0)


def test_node_reductions_are_normalised():
    prec = abi.SP
    n = 24
    info = abi.make_info(prec, n)
    fields = init.workload_fields(n, n, n, np.float32, seed=9, amplitude=0.2)
    host = abi.HostMesh(prec, info, fields)
    from astaroth_b200 import library

    lib = library.load("sp")
    node = C.c_void_p()
    assert lib.acNodeCreate(0, info, C.byref(node)) == 0
    try:
        assert lib.acNodeLoadMesh(node, 0, host.cmesh) == 0
        om = O.OracleMesh("f80", fields, n, n, n)
        r = C.c_float()
        assert lib.acNodeReduceScal(node, 0, abi.RTYPE_RMS, 2, C.byref(r)) == 0
        assert r.value == pytest.approx(om.reduce(abi.RTYPE_RMS, [2], normalise=True), rel=1e-6)
        assert lib.acNodeReduceVec(node, 0, abi.RTYPE_RMS_EXP, 1, 2, 3, C.byref(r)) == 0
        assert r.value == pytest.approx(om.reduce(abi.RTYPE_RMS_EXP, [1, 2, 3], normalise=True),
                                        rel=1e-6)
    finally:
        lib.acNodeDestroy(node)


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_subbox_substep_matches_full(flavour):
    prec = abi.PRECISIONS[flavour]
    n = 40
    info = workload_info(prec, n)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=5, amplitude=0.05)
    host = abi.HostMesh(prec, info, fields)
    dt = 1e-3
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        dev.periodic_boundconds()
        dev.integrate_substep(0, dt)
        dev.swap_buffers()
        full = [dev.store_double(w) for w in range(8)]
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        dev.swap_buffers()  # out := the initial state, to see what is left untouched
        dev.load_mesh(host)
        dev.periodic_boundconds()
        # the same substep over a box whose x start is not tile aligned
        s, e = abi.int3(6, 4, 9), abi.int3(40, 31, 22)
        dev.integrate_substep(0, dt, s, e)
        dev.swap_buffers()
        part = [dev.store_double(w) for w in range(8)]
    for w in range(8):
        box = (slice(9, 22), slice(4, 31), slice(6, 40))
        assert np.array_equal(part[w][box], full[w][box])
        mask = np.ones_like(part[w], dtype=bool)
        mask[box] = False
        assert np.array_equal(part[w][mask], fields[w].astype(np.float64)[mask])


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_graph_replay_and_tile_configs_bitwise(flavour):
    prec = abi.PRECISIONS[flavour]
    n = 48
    info = workload_info(prec, n)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=6, amplitude=0.05)
    ref = run_gpu(flavour, fields, info, 1e-3, 3, graph=False)
    got = run_gpu(flavour, fields, info, 1e-3, 3, graph=True)
    for w in range(8):
        assert np.array_equal(ref[w], got[w])
    host = abi.HostMesh(prec, info, fields)
    with new_device(flavour, info) as dev:
        _, ncfg, _ = dev.solve_config()
        for c in range(ncfg):
            dev.set_solve_config(c)
            dev.load_mesh(host)
            for _ in range(3):
                dev.integrate_step(1e-3)
            dev.periodic_boundconds()
            for w in range(8):
                assert np.array_equal(dev.store_double(w), ref[w]), (c, w)


def test_legacy_interface_matches_device_path():
    prec = abi.SP
    n = 32
    info = workload_info(prec, n)
    fields = init.workload_fields(n, n, n, np.float32, seed=8, amplitude=0.01)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    from astaroth_b200 import library

    lib = library.load("sp")
    assert lib.acInit(info) == 0
    try:
        assert lib.acLoad(host.cmesh) == 0
        for _ in range(2):
            assert lib.acIntegrate(np.float32(1e-3)) == 0
        assert lib.acBoundcondStep() == 0
        out = abi.HostMesh(prec, info)
        assert lib.acStore(C.byref(out.cmesh)) == 0
        umax = lib.acReduceVec(abi.RTYPE_MAX, 1, 2, 3)
    finally:
        lib.acQuit()
    ref = run_gpu("sp", fields, info, float(np.float32(1e-3)), 2)
    for w in range(8):
        assert np.array_equal(out.fields[w].astype(np.float64), ref[w])
    assert umax == pytest.approx(np.max(np.sqrt(sum(interior(ref[c]) ** 2 for c in (1, 2, 3)))),
                                 rel=1e-6)


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_forcing_vs_oracle(flavour):
    prec = abi.PRECISIONS[flavour]
    n, steps = 24, 2
    kf, ffr, ffi = (1.0, -2.0, 1.0), (0.1, 0.2, -0.3), (0.3, -0.1, 0.2)
    extra = dict(forcing_magnitude=0.05, forcing_phase=0.7, kaver=1.0, k_forcex=kf[0],
                 k_forcey=kf[1], k_forcez=kf[2], ff_hel_rex=ffr[0], ff_hel_rey=ffr[1],
                 ff_hel_rez=ffr[2], ff_hel_imx=ffi[0], ff_hel_imy=ffi[1], ff_hel_imz=ffi[2])
    info = workload_info(prec, n, **extra)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=12, amplitude=1e-3)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    dt = float(prec.np_dtype(1e-3))
    with new_device(flavour, info) as dev:
        dev.set_forcing(True)
        dev.load_mesh(host)
        for _ in range(steps):
            dev.integrate_step(dt)
        out = [dev.store_double(w) for w in range(8)]
    p = O.params_from(info, forcing=1, forcing_magnitude=abi.get_real(info, "forcing_magnitude"),
                      forcing_phase=abi.get_real(info, "forcing_phase"), kaver=1.0,
                      k_force=[abi.get_real(info, k) for k in ("k_forcex", "k_forcey", "k_forcez")],
                      ff_re=[abi.get_real(info, k) for k in ("ff_hel_rex", "ff_hel_rey", "ff_hel_rez")],
                      ff_im=[abi.get_real(info, k) for k in ("ff_hel_imx", "ff_hel_imy", "ff_hel_imz")])
    om = O.OracleMesh("f80", fields, n, n, n)
    om.step(p, dt, steps)
    errs = [O.normwise_error(interior(out[w]), om.interior(w)) for w in range(8)]
    print("forcing", flavour, ["%.2e" % e for e in errs])
    assert max(errs) <= TOL[flavour], errs


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_generated_forcing_each_step_vs_oracle(flavour):
    """Every step a new forcing from the seeded generator, loaded with
    acDeviceLoadForcingParams (the reference standalone's per-step
    generateForcingParams + loadForcingParamsToDevice); the oracle steps with
    the same parameters."""
    from astaroth_b200.device import ForcingGenerator

    prec = abi.PRECISIONS[flavour]
    n, steps = 24, 3
    info = workload_info(prec, n, kmin=1.0, kmax=3.0, relhel=0.5, forcing_magnitude=0.05)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=21, amplitude=1e-3)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    dt = float(prec.np_dtype(1e-3))
    gen = ForcingGenerator(flavour, info, seed=77)
    params = [gen.next() for _ in range(steps)]
    with new_device(flavour, info) as dev:
        dev.set_forcing(True)
        dev.load_mesh(host)
        for fp in params:
            dev.load_forcing_params(fp)
            dev.integrate_step(dt)
        dev.synchronize()
        assert dev.status() == 0
        out = [dev.store_double(w) for w in range(8)]
    om = O.OracleMesh("f80", fields, n, n, n)
    for fp in params:
        p = O.params_from(info, forcing=1, forcing_magnitude=fp.magnitude,
                          forcing_phase=fp.phase, kaver=fp.kaver, k_force=list(fp.k_force),
                          ff_re=list(fp.ff_hel_re), ff_im=list(fp.ff_hel_im))
        om.step(p, dt, 1)
    errs = [O.normwise_error(interior(out[w]), om.interior(w)) for w in range(8)]
    print("generated forcing", flavour, ["%.2e" % e for e in errs])
    assert max(errs) <= TOL[flavour], errs
    # the forcing moved the velocity well beyond the tolerance
    free = O.OracleMesh("f80", fields, n, n, n)
    free.step(O.params_from(info), dt, steps)
    assert O.normwise_error(free.interior(1), om.interior(1)) > 100 * TOL[flavour]


def test_mixed_tracks_fp64():
    """The mixed state stays close to the FP64 GPU path (64^3, 10 steps)."""
    n, steps, dt = 64, 10, float(np.float32(1e-3))
    fields = init.workload_fields(n, n, n, np.float32, seed=1, amplitude=1e-3, velocity_mode=0.1)
    d = run_gpu("dp", [f.astype(np.float64) for f in fields], workload_info(abi.DP, n), dt, steps)
    m = run_gpu("mixed", fields, workload_info(abi.MIXED, n), dt, steps)
    s = run_gpu("sp", fields, workload_info(abi.SP, n), dt, steps)
    em = [O.normwise_error(interior(m[w]), interior(d[w])) for w in range(8)]
    es = [O.normwise_error(interior(s[w]), interior(d[w])) for w in range(8)]
    print("mixed vs dp", ["%.2e" % e for e in em])
    print("sp    vs dp", ["%.2e" % e for e in es])
    assert max(em) <= 1e-6


@pytest.mark.parametrize("flavour", ["sp", "mixed"])
def test_shift_equivariance_256(flavour):
    """Full-size property: a periodic shift of the initial state shifts the
    result exactly (every vertex runs the same arithmetic)."""
    prec = abi.PRECISIONS[flavour]
    n = 256
    info = workload_info(prec, n)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=3, amplitude=1e-3, velocity_mode=0.1)
    shift = (5, -37, 101)
    shifted = [init.wrap_ghosts(np.roll(f[3:-3, 3:-3, 3:-3], shift, axis=(0, 1, 2)))
               for f in fields]
    a = run_gpu(flavour, fields, info, 1e-3, 1)
    b = run_gpu(flavour, shifted, info, 1e-3, 1)
    for w in range(8):
        assert np.array_equal(np.roll(interior(a[w]), shift, axis=(0, 1, 2)), interior(b[w]))


def test_reference_ctest_sample_runs(tmp_path):
    exe = os.path.join(abi.REPO, "oracle", "_ref", "ctest_sp")
    if not os.path.exists(exe):
        pytest.skip("ctest binary not built (needs the reference sources at build time)")
    cfg = tmp_path / "astaroth.conf"
    lines = [f"{k} = {v}" for k, v in abi.DEFAULT_CONFIG.items() if k != "AC_bin_save_t"]
    cfg.write_text("\n".join(lines) + "\n")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ctest complete." in r.stdout
    assert "FAIL" not in r.stdout


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_transfer_moves_whole_values(flavour):
    """acDeviceTransferMesh between two Devices on one GPU copies the whole
    state: in the mixed build the (hi, lo) pairs, and after a whole-box ghost
    fill (which writes only the hi parts on the integration path) the ghosts'
    lo parts too; the double views of source and destination are identical."""
    prec = abi.PRECISIONS[flavour]
    n = 16
    info = workload_info(prec, n)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=41, amplitude=0.05,
                                  velocity_mode=0.1)
    with new_device(flavour, info) as a, new_device(flavour, info) as b:
        a.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
        for _ in range(2):
            a.integrate_step(1e-3)
        a.periodic_boundconds()
        assert a.lib.acDeviceTransferMesh(a.handle, 0, b.handle) == abi.AC_SUCCESS
        a.synchronize()
        src = [a.store_double(w) for w in range(8)]
        dst = [b.store_double(w) for w in range(8)]
    for w in range(8):
        assert np.array_equal(src[w], dst[w]), w
        assert np.array_equal(src[w], init.wrap_ghosts(interior(src[w]))), w


def mirror_fill_numpy(a, sign):
    """Restatement of the symmetric/antisymmetric fill as the reference intends it
    (src/core/kernels/boundconds.cuh:3-128): each ghost vertex takes sign times
    the vertex mirrored about the first/last interior point on every axis where
    it lies outside the interior."""
    g = abi.NGHOST
    out = a.copy()
    mz, my, mx = a.shape

    def mir(c, m):
        n = m - 2 * g
        return 2 * g - c if c < g else (2 * (n + g - 1) - c if c > n + g - 1 else c)

    for k in range(mz):
        for j in range(my):
            for i in range(mx):
                if g <= i < mx - g and g <= j < my - g and g <= k < mz - g:
                    continue
                out[k, j, i] = sign * a[mir(k, mz), mir(j, my), mir(i, mx)]
    return out


@pytest.mark.parametrize("flavour", FLAVOURS)
@pytest.mark.parametrize("bc", [abi.AC_BOUNDCOND_SYMMETRIC, abi.AC_BOUNDCOND_ANTISYMMETRIC])
def test_symmetric_boundaries_exact(flavour, bc):
    """acDeviceGeneralBoundconds with a symmetric or antisymmetric condition
    (selected by AC_bc_type_top_x, as in the reference): ghosts equal sign
    times the mirrored interior, bit for bit, on a non-cubic mesh; the interior
    is untouched; a later periodic fill is not skipped."""
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz = 9, 7, 5
    info = workload_info(prec, nx, ny, nz, bc_type_top_x=bc)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=31, amplitude=0.5)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    sign = 1.0 if bc == abi.AC_BOUNDCOND_SYMMETRIC else -1.0
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        dev.periodic_boundconds()  # the ghosts hold periodic images first
        s, e = dev.full_box()
        rc = dev.lib.acDeviceGeneralBoundconds(dev.handle, 0, s, e, info, abi.int3(-1, -1, -1))
        assert rc == abi.AC_SUCCESS
        got = [dev.store_double(w) for w in range(8)]
        dev.periodic_boundconds()  # must run again: the ghosts are mirror images now
        back = [dev.store_double(w) for w in range(8)]
    for w in range(8):
        want = mirror_fill_numpy(fields[w].astype(np.float64), sign)
        assert np.array_equal(got[w], want), w
        assert np.array_equal(back[w], init.wrap_ghosts(interior(fields[w].astype(np.float64)))), w


def test_symmetric_boundaries_through_legacy_integrate():
    """acIntegrateGBC with a symmetric condition (the standalone's integration
    call) equals the Device sequence general fill + substep + swap, bit for bit."""
    prec = abi.SP
    n = 12
    info = workload_info(prec, n, bc_type_top_x=abi.AC_BOUNDCOND_SYMMETRIC)
    fields = init.workload_fields(n, n, n, np.float32, seed=32, amplitude=0.01)
    dt = float(np.float32(1e-3))
    with new_device("sp", info) as dev:
        dev.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
        s, e = dev.full_box()
        for step in range(3):
            assert dev.lib.acDeviceGeneralBoundconds(dev.handle, 0, s, e, info,
                                                     abi.int3(-1, -1, -1)) == abi.AC_SUCCESS
            dev.integrate_substep(step, dt)
            dev.swap_buffers()
        dev.synchronize()
        ref = [dev.store_double(w) for w in range(8)]
    from astaroth_b200 import library

    lib = library.load("sp")
    assert lib.acInit(info) == 0
    try:
        assert lib.acLoad(abi.HostMesh(prec, info, [f.copy() for f in fields]).cmesh) == 0
        assert lib.acIntegrateGBC(info, C.c_float(dt)) == 0
        out = abi.HostMesh(prec, info)
        assert lib.acStore(C.byref(out.cmesh)) == 0
    finally:
        lib.acQuit()
    for w in range(8):
        assert np.array_equal(interior(out.fields[w].astype(np.float64)), interior(ref[w])), w


def test_reference_standalone_simulation_runs_and_matches_oracle(tmp_path):
    """The reference's standalone sample (samples/standalone, sources unchanged,
    linked against the FP32 library) runs its simulation mode: Legacy API steps
    with the host CFL time step, diagnostics every step into timeseries.ts and
    .mesh snapshots at steps 0 and 4. The oracle, started from the step-0
    snapshot and stepped with the time steps the sample reports, must reproduce
    the step-4 snapshot, and the sample's max|u| must be that of the snapshot."""
    exe = os.path.join(abi.REPO, "oracle", "_ref", "ac_run_sp")
    if not os.path.exists(exe):
        pytest.skip("standalone binary not built (needs the reference sources at build time)")
    n, steps = 24, 4
    cfg = dict(abi.DEFAULT_CONFIG)
    cfg.update({"AC_nx": n, "AC_ny": n, "AC_nz": n, "AC_dsx": 2 * math.pi / n,
                "AC_dsy": 2 * math.pi / n, "AC_dsz": 2 * math.pi / n,
                "AC_max_steps": steps + 1, "AC_save_steps": 1, "AC_bin_steps": steps,
                "AC_bin_save_t": "1e666"})
    conf = tmp_path / "sim.conf"
    conf.write_text("".join(f"{k} = {v}\n" for k, v in cfg.items()))
    r = subprocess.run([exe, "--simulate", "--config", str(conf)], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    m = n + 6

    def snapshot(step):
        out = []
        for name in abi.VTXBUFS:
            raw = np.fromfile(tmp_path / f"{name}_{step}.mesh", dtype=np.float32)
            assert raw.size == 1 + m ** 3, name
            out.append(raw[1:].reshape(m, m, m).astype(np.float64))
        return float(raw[0]), out

    t0, s0 = snapshot(0)
    t4, s4 = snapshot(steps)
    rows = [ln.split() for ln in (tmp_path / "timeseries.ts").read_text().splitlines()[1:] if ln.strip()]
    dts = {int(row[0]): float(row[2]) for row in rows}
    assert sorted(dts) == list(range(steps + 1))
    assert all(np.isfinite(f).all() for f in s4)
    assert t4 == pytest.approx(sum(dts[i] for i in range(1, steps + 1)), rel=1e-5)

    info = abi.make_info(abi.SP, n, **{k: v for k, v in cfg.items() if k in abi.REAL_PARAMS
                                       and k not in ("AC_bin_save_t",)})
    p = O.params_from(info)
    om = O.OracleMesh("f80", [np.ascontiguousarray(f) for f in s0], n, n, n)
    for i in range(1, steps + 1):
        om.step(p, dts[i], 1)
    errs = [O.normwise_error(interior(s4[w]), om.interior(w)) for w in range(8)]
    assert max(errs) <= TOL["sp"], errs
    umax_sample = float(rows[-1][5])
    umax_snap = np.max(np.sqrt(sum(interior(s4[c]) ** 2 for c in (1, 2, 3))))
    assert umax_sample == pytest.approx(umax_snap, rel=1e-5)


@pytest.mark.parametrize("flavour", FLAVOURS)
@pytest.mark.parametrize("dims", [(20, 14, 11), (131, 5, 4), (7, 4, 5)])
def test_whole_box_fill_after_substep_is_exact(flavour, dims):
    """The whole-box ghost fill (interior-row x-ghosts and ghost rows as
    separate work units, rows wider than one 128-vertex chunk included) must
    leave every ghost equal to its periodic image of the interior that the
    substep just wrote; a second fill of the same block is skipped and must
    change nothing."""
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz = dims
    info = workload_info(prec, nx, ny, nz)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=13, amplitude=0.05)
    host = abi.HostMesh(prec, info, fields)
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        dev.periodic_boundconds()
        dev.integrate_substep(0, 1e-3)
        dev.swap_buffers()
        dev.periodic_boundconds()
        first = [dev.store_double(w) for w in range(8)]
        dev.periodic_boundconds()
        second = [dev.store_double(w) for w in range(8)]
    for w in range(8):
        assert np.array_equal(first[w], init.wrap_ghosts(interior(first[w]))), w
        assert np.array_equal(first[w], second[w]), w


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_staged_loads(flavour):
    """Loads go through a device staging buffer (a contiguous copy per chunk,
    then a scatter into the padded rows): a partial range loaded from one
    offset of the host mesh to another of the device lands exactly there and
    nowhere else; a field larger than one staging chunk (64 MB) loads whole;
    and loaded values carry no lo part in the mixed build, even where the
    block held a nonzero lo part before."""
    prec = abi.PRECISIONS[flavour]
    rng = np.random.default_rng(5)
    nx, ny, nz = 37, 29, 23
    info = abi.make_info(prec, nx, ny, nz)
    shape = (nz + 6, ny + 6, nx + 6)
    base = [rng.standard_normal(shape).astype(prec.np_dtype) for _ in range(8)]
    new = [rng.standard_normal(shape).astype(prec.np_dtype) for _ in range(8)]
    with new_device(flavour, info) as dev:
        dev.load_mesh(abi.HostMesh(prec, info, base))
        src_flat, dst_flat, count = 777, 2345, 4 * (nx + 6) + 29

        def int3_of(flat):
            k, rem = divmod(flat, (nx + 6) * (ny + 6))
            j, i = divmod(rem, nx + 6)
            return abi.int3(i, j, k)

        src_mesh = abi.HostMesh(prec, info, new)
        rc = dev.lib.acDeviceLoadVertexBufferWithOffset(dev.handle, 0, src_mesh.cmesh, 5,
                                                        int3_of(src_flat), int3_of(dst_flat),
                                                        count)
        assert rc == 0
        back = abi.HostMesh(prec, info)
        dev.store_mesh(back)
        want = base[5].reshape(-1).copy()
        want[dst_flat:dst_flat + count] = new[5].reshape(-1)[src_flat:src_flat + count]
        assert np.array_equal(back.fields[5].reshape(-1), want)
        for w in (0, 1, 2, 3, 4, 6, 7):
            assert np.array_equal(back.fields[w], base[w]), w

        if flavour == "mixed":
            # give both blocks nonzero lo parts, then load over them
            for s in range(3):
                dev.periodic_boundconds()
                dev.integrate_substep(s, 1e-3)
                dev.swap_buffers()
            dev.load_mesh(abi.HostMesh(prec, info, new))
            for w in range(8):
                assert np.array_equal(dev.store_double(w), new[w].astype(np.float64)), w

    n = 256  # 262^3 values per field: more than one staging chunk
    info = abi.make_info(prec, n)
    big = [rng.standard_normal((n + 6,) * 3).astype(prec.np_dtype) for _ in range(2)]
    fields = [big[w % 2] for w in range(8)]
    with new_device(flavour, info) as dev:
        dev.load_mesh(abi.HostMesh(prec, info, fields))
        back = abi.HostMesh(prec, info)
        dev.store_mesh(back)
        for w in range(8):
            assert np.array_equal(back.fields[w], fields[w]), w


def test_bounded_wait_gives_up_and_device_stays_usable():
    """Failure detection without a fault: a kernel waits, with the solve
    pipeline's bounded wait and a 0.2 s limit, on a barrier phase that nothing
    completes. The wait gives up, the status word reports it, a whole-device
    synchronisation returns AC_FAILURE, and after the status is reset the same
    Device integrates exactly as a fresh one does."""
    import time

    from astaroth_b200.device import AcError

    prec = abi.PRECISIONS["sp"]
    n = 16
    info = workload_info(prec, n)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=23, amplitude=1e-3)
    with new_device("sp", info) as dev:
        assert dev.status() == 0
        t0 = time.perf_counter()
        dev.check_wait_limit(0.2)
        waited = time.perf_counter() - t0
        assert 0.2 <= waited < 5.0
        assert dev.status() == 1
        with pytest.raises(AcError):
            dev.synchronize()
        dev.reset_status()
        assert dev.status() == 0
        dev.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in fields]))
        dev.integrate_step(1e-3)
        dev.synchronize()
        assert dev.status() == 0
        got = [dev.store_double(w) for w in range(8)]
    ref = run_gpu("sp", fields, info, 1e-3, 1)
    for w in range(8):
        assert np.array_equal(interior(got[w]), interior(ref[w])), w


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_diagnostics_print_reads_each_array_once(flavour):
    """The standalone's diagnostics print (samples/standalone/simulation.cc:250-310:
    MAX, MIN and RMS of |u|, then of each of the eight fields). Once a caller has
    reduced two arrays of one state, a pass serves every request whose bytes it
    reads, so from the second print on a print takes two passes in the
    single-precision builds (u with the A components that share its elements;
    lnrho with s) and six in FP64 (u with its components; lnrho, ax, ay, az, s);
    the first takes five (nine in FP64). Every value equals that of a
    three-in-one pass made for its request alone on a new Device, bit for bit;
    max and min equal the host values' and the sums agree within 1e-12."""
    prec = abi.PRECISIONS[flavour]
    dims = (20, 14, 11)
    info = workload_info(prec, *dims)
    fields = init.workload_fields(*dims, prec.np_dtype, seed=5, amplitude=0.05, velocity_mode=0.1)
    host = abi.HostMesh(prec, info, [f.copy() for f in fields])
    U = (abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
    kinds = (abi.RTYPE_MAX, abi.RTYPE_MIN, abi.RTYPE_RMS)

    def print_stats(dev):
        l0 = dev.launch_count()
        u = [dev.reduce_vec_double(k, *U) for k in kinds]
        f = {w: [dev.reduce_scal_double(k, w) for k in kinds] for w in range(8)}
        return u, f, dev.launch_count() - l0

    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        u1, f1, p1 = print_stats(dev)
        dev.load_mesh(host)  # a new state: the record starts again
        u2, f2, p2 = print_stats(dev)
    assert (p1, p2) == ((9, 6) if flavour == "dp" else (5, 2)), (p1, p2)
    alone = {}
    for w in range(8):
        with new_device(flavour, info) as dev:
            dev.load_mesh(host)
            alone[w] = [dev.reduce_scal_double(k, w) for k in kinds]
    with new_device(flavour, info) as dev:
        dev.load_mesh(host)
        alone_u = [dev.reduce_vec_double(k, *U) for k in kinds]
    assert u1 == alone_u and u2 == alone_u
    for w in range(8):
        assert f1[w] == alone[w] and f2[w] == alone[w], w
        v = interior(fields[w].astype(np.float64))
        assert f2[w][0] == v.max() and f2[w][1] == v.min(), w
        assert f2[w][2] == pytest.approx(float(np.sum(v * v)), rel=1e-12), w


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_reduction_record_follows_every_write(flavour):
    """MAX, MIN and RMS of one field or of a vector's length come from one pass
    and are kept while nothing has written the device's blocks; a step, a
    fill, a load and a transfer must each make the next request read the new
    values: device A (which holds a record) must return what device B (which
    reduces the same state for the first time) returns."""
    prec = abi.PRECISIONS[flavour]
    n = 24
    info = workload_info(prec, n)
    f1 = init.workload_fields(n, n, n, prec.np_dtype, seed=31, amplitude=0.05)
    f2 = init.workload_fields(n, n, n, prec.np_dtype, seed=32, amplitude=0.07)
    U = (abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
    kinds = (abi.RTYPE_MAX, abi.RTYPE_MIN, abi.RTYPE_RMS)

    def stats(dev):
        v = [dev.reduce_vec_double(r, *U) for r in kinds]
        s = [dev.reduce_scal_double(r, abi.VTXBUF_LNRHO) for r in kinds]
        # asked again: the same values
        assert [dev.reduce_vec_double(r, *U) for r in kinds] == v
        return v + s

    def fresh(setup):
        with new_device(flavour, info) as b:
            setup(b)
            return stats(b)

    with new_device(flavour, info) as a:
        a.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in f1]))
        s0 = stats(a)
        assert s0 == fresh(lambda b: b.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in f1])))

        a.integrate_step(1e-3)
        s1 = stats(a)
        assert s1 != s0

        def stepped(b):
            b.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in f1]))
            b.integrate_step(1e-3)
        assert s1 == fresh(stepped)

        a.set_vertex_buffer(abi.VTXBUF_UUX, 0.25)
        s2 = stats(a)

        def filled(b):
            stepped(b)
            b.set_vertex_buffer(abi.VTXBUF_UUX, 0.25)
        assert s2 == fresh(filled)

        a.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in f2]))
        assert stats(a) == fresh(lambda b: b.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in f2])))

        with new_device(flavour, info) as c:
            c.load_mesh(abi.HostMesh(prec, info, [f.copy() for f in f1]))
            rc = c.lib.acDeviceTransferMesh(c.handle, 0, a.handle)
            assert rc == 0
            c.synchronize()
            assert stats(a) == s0

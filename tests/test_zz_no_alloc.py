"""acReduceScalNoAlloc, the reduction entry point that allocates no device
memory (for callers that cannot call cudaMalloc: frameworks that own all
device memory through their own pool, or loops that must not pay cudaMalloc's
implicit synchronisation).

Checked through the C ABI against the existing entry point acDeviceReduceScal
(its FP64-accumulator form), within the reductions' tolerance (1e-12 relative),
on two calls in a row for every reduction type. The field and the result live
in device memory the test owns. This file sorts last so a stop-at-first-failure
run has already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from astaroth_b200 import Device, abi, init, library

pytestmark = pytest.mark.gpu

RTYPES = (abi.RTYPE_MAX, abi.RTYPE_MIN, abi.RTYPE_RMS, abi.RTYPE_RMS_EXP, abi.RTYPE_SUM)


@pytest.mark.parametrize("flavour", ["sp", "dp", "mixed"])
def test_noalloc_reduction_matches_device_reduction(flavour):
    import torch

    prec = abi.PRECISIONS[flavour]
    lib = library.load(flavour)
    nx, ny, nz = 45, 38, 29
    info = abi.make_info(prec, nx, ny, nz)
    tdt = torch.float64 if prec.double else torch.float32
    # two different fields, reduced one after the other
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=21, amplitude=0.4)
    host = abi.HostMesh(prec, info, fields)
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    with Device(flavour, info) as dev:
        dev.load_mesh(host)
        for rt in RTYPES:
            for w in (2, 7):  # two calls in a row
                dfield = torch.from_numpy(fields[w]).to(device="cuda", dtype=tdt).contiguous()
                rc = lib.acReduceScalNoAlloc(C.c_void_p(stream.cuda_stream), rt,
                                             C.c_void_p(dfield.data_ptr()), nx, ny, nz,
                                             C.c_void_p(result.data_ptr()))
                assert rc == abi.AC_SUCCESS
                torch.cuda.synchronize()
                got = float(result.item())
                want = dev.reduce_scal_double(rt, w)
                assert got == pytest.approx(want, rel=1e-12, abs=1e-300), (rt, w, got, want)


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_noalloc_at_the_largest_accepted_mesh_allocates_nothing(flavour):
    """ny * nz = 1,048,576 rows is the largest mesh the fixed scratch takes: every
    one of its 16,384 per-block partials is written and folded by the last
    block. The results equal an FP64 reduction of the same interior (torch, on
    the device) within 1e-12, and across the calls the device's free memory does
    not change (the entry point allocates nothing; the first call, which loads
    the library's kernels, comes before the measurement)."""
    import torch

    prec = abi.PRECISIONS[flavour]
    lib = library.load(flavour)
    nx, ny, nz = 8, 1024, 1024
    tdt = torch.float64 if prec.double else torch.float32
    g = abi.NGHOST
    gen = torch.Generator(device="cuda").manual_seed(5)
    field = (0.5 * torch.rand((nz + 2 * g, ny + 2 * g, nx + 2 * g), generator=gen,
                              device="cuda", dtype=torch.float64) - 0.25).to(tdt).contiguous()
    inner = field[g:-g, g:-g, g:-g].to(torch.float64)
    want = {abi.RTYPE_MAX: float(inner.max()), abi.RTYPE_MIN: float(inner.min()),
            abi.RTYPE_RMS: float((inner * inner).sum()),
            abi.RTYPE_RMS_EXP: float((torch.exp(inner) ** 2).sum()),
            abi.RTYPE_SUM: float(inner.sum())}
    del inner
    results = torch.zeros(2 * len(RTYPES), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def call(rt, slot):
        return lib.acReduceScalNoAlloc(C.c_void_p(stream.cuda_stream), rt,
                                       C.c_void_p(field.data_ptr()), nx, ny, nz,
                                       C.c_void_p(results.data_ptr() + 8 * slot))

    assert call(abi.RTYPE_SUM, 0) == abi.AC_SUCCESS  # loads the module
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for slot, rt in enumerate(RTYPES):
        for rep in range(2):  # two calls in a row
            assert call(rt, 2 * slot + rep) == abi.AC_SUCCESS
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    got = results.cpu().numpy()
    for slot, rt in enumerate(RTYPES):
        for rep in range(2):
            assert got[2 * slot + rep] == pytest.approx(want[rt], rel=1e-12), (rt, rep)


def test_noalloc_rejects_meshes_beyond_its_scratch():
    import torch

    lib = library.load("sp")
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    # ny * nz = 2048 * 1024 > 1,048,576 rows: rejected before any launch
    rc = lib.acReduceScalNoAlloc(None, abi.RTYPE_MAX, C.c_void_p(dummy.data_ptr()), 8, 2048,
                                 1024, C.c_void_p(result.data_ptr()))
    assert rc == abi.AC_FAILURE
    # one row past the limit (ny * nz = 1,048,577 needs 16,385 partials)
    rc = lib.acReduceScalNoAlloc(None, abi.RTYPE_MAX, C.c_void_p(dummy.data_ptr()), 8, 1048577,
                                 1, C.c_void_p(result.data_ptr()))
    assert rc == abi.AC_FAILURE
    rc = lib.acReduceScalNoAlloc(None, abi.RTYPE_ALFVEN_MAX, C.c_void_p(dummy.data_ptr()), 1, 1,
                                 1, C.c_void_p(result.data_ptr()))
    assert rc == abi.AC_FAILURE
    np.testing.assert_equal(result.item(), 0.0)

"""Python host mirror of the reference's Device interface (include/astaroth.h
acDevice*, reference src/core/device.cc). Each method is a thin call through
the C ABI of the in-tree library; a non-zero AcResult raises AcError.

    dev = Device("sp", info)
    dev.load_mesh(host)                 # acDeviceLoadMesh
    for s in range(3):
        dev.periodic_boundconds()       # acDevicePeriodicBoundconds
        dev.integrate_substep(s, dt)    # acDeviceIntegrateSubstep
        dev.swap_buffers()              # acDeviceSwapBuffers
    umax = dev.reduce_vec(abi.RTYPE_MAX, abi.VTXBUF_UUX, abi.VTXBUF_UUY, abi.VTXBUF_UUZ)
    dev.store_mesh(host)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, library


class AcError(RuntimeError):
    pass


def _check(rc: int, what: str) -> None:
    if rc != abi.AC_SUCCESS:
        raise AcError(f"{what} returned AC_FAILURE")


def i3(x: int, y: int, z: int) -> abi.int3:
    return abi.int3(int(x), int(y), int(z))


class Device:
    def __init__(self, flavour: str, info, device_id: int = 0):
        self.flavour = flavour
        self.prec = abi.PRECISIONS[flavour]
        self.lib = library.load(flavour)
        self.info = info
        self.n = abi.dims(info)
        self.handle = C.c_void_p()
        _check(self.lib.acDeviceCreate(device_id, info, C.byref(self.handle)), "acDeviceCreate")

    # --- lifetime ---------------------------------------------------------
    def destroy(self) -> None:
        if self.handle:
            self.lib.acDeviceDestroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    # --- boxes ------------------------------------------------------------
    def interior_box(self):
        nx, ny, nz = self.n
        g = abi.NGHOST
        return i3(g, g, g), i3(g + nx, g + ny, g + nz)

    def full_box(self):
        nx, ny, nz = self.n
        g = abi.NGHOST
        return i3(0, 0, 0), i3(nx + 2 * g, ny + 2 * g, nz + 2 * g)

    # --- data -------------------------------------------------------------
    def load_mesh(self, host: abi.HostMesh, stream: int = 0) -> None:
        _check(self.lib.acDeviceLoadMesh(self.handle, stream, host.cmesh), "acDeviceLoadMesh")

    def store_mesh(self, host: abi.HostMesh, stream: int = 0) -> None:
        _check(self.lib.acDeviceStoreMesh(self.handle, stream, C.byref(host.cmesh)),
               "acDeviceStoreMesh")
        self.synchronize(stream)

    def load_double(self, handle: int, arr: np.ndarray, stream: int = 0) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _check(self.lib.acDeviceLoadVertexBufferDouble(self.handle, stream, handle, a.ctypes.data),
               "acDeviceLoadVertexBufferDouble")

    def store_double(self, handle: int, stream: int = 0) -> np.ndarray:
        nx, ny, nz = self.n
        g = abi.NGHOST
        out = np.empty((nz + 2 * g, ny + 2 * g, nx + 2 * g), dtype=np.float64)
        _check(self.lib.acDeviceStoreVertexBufferDouble(self.handle, stream, handle,
                                                         out.ctypes.data),
               "acDeviceStoreVertexBufferDouble")
        return out

    def set_vertex_buffer(self, handle: int, value: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceSetVertexBuffer(self.handle, stream, handle, value),
               "acDeviceSetVertexBuffer")

    # --- uniforms ---------------------------------------------------------
    def load_scalar_uniform(self, param: int, value: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceLoadScalarUniform(self.handle, stream, param, value),
               "acDeviceLoadScalarUniform")

    def load_mesh_info(self, info) -> None:
        _check(self.lib.acDeviceLoadMeshInfo(self.handle, info), "acDeviceLoadMeshInfo")

    # --- hot path ---------------------------------------------------------
    def integrate_substep(self, step: int, dt: float, start=None, end=None, stream: int = 0) -> None:
        if start is None:
            start, end = self.interior_box()
        _check(self.lib.acDeviceIntegrateSubstep(self.handle, stream, step, start, end, dt),
               "acDeviceIntegrateSubstep")

    def periodic_boundconds(self, stream: int = 0, start=None, end=None) -> None:
        if start is None:
            start, end = self.full_box()
        _check(self.lib.acDevicePeriodicBoundconds(self.handle, stream, start, end),
               "acDevicePeriodicBoundconds")

    def swap_buffers(self) -> None:
        _check(self.lib.acDeviceSwapBuffers(self.handle), "acDeviceSwapBuffers")

    def integrate_step(self, dt: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceIntegrateStep(self.handle, stream, dt), "acDeviceIntegrateStep")

    def integrate_steps(self, dt: float, n: int, stream: int = 0) -> None:
        _check(self.lib.acDeviceIntegrateSteps(self.handle, stream, dt, n),
               "acDeviceIntegrateSteps")

    # --- steps whose time step is chosen on the device ----------------------
    def integrate_step_cfl(self, timescale: float = 1.0, stream: int = 0) -> None:
        _check(self.lib.acDeviceIntegrateStepCFL(self.handle, stream, timescale),
               "acDeviceIntegrateStepCFL")

    def integrate_steps_cfl(self, n: int, timescale: float = 1.0, stream: int = 0) -> None:
        _check(self.lib.acDeviceIntegrateStepsCFL(self.handle, stream, timescale, n),
               "acDeviceIntegrateStepsCFL")

    def timestep_record(self, stream: int = 0) -> tuple[float, float, int]:
        """(dt of the last such step, simulated time, steps taken)."""
        dt, t, k = self.prec.real(), C.c_double(), C.c_ulonglong()
        _check(self.lib.acDeviceGetTimestepRecord(self.handle, stream, C.byref(dt), C.byref(t),
                                                  C.byref(k)), "acDeviceGetTimestepRecord")
        return float(dt.value), float(t.value), int(k.value)

    def set_simulation_time(self, t: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceSetSimulationTime(self.handle, stream, t),
               "acDeviceSetSimulationTime")

    def set_step_diagnostics(self, enabled: bool) -> None:
        _check(self.lib.acDeviceSetStepDiagnostics(self.handle, int(bool(enabled))),
               "acDeviceSetStepDiagnostics")

    def set_forcing(self, enabled: bool) -> None:
        _check(self.lib.acDeviceSetForcing(self.handle, int(bool(enabled))), "acDeviceSetForcing")

    def load_forcing_params(self, params, stream: int = 0) -> None:
        _check(self.lib.acDeviceLoadForcingParams(self.handle, stream, params),
               "acDeviceLoadForcingParams")


    # --- reductions (device layer: RMS/RMS_EXP are raw sums) --------------
    def reduce_scal(self, rtype: int, handle: int, stream: int = 0) -> float:
        r = self.prec.real()
        _check(self.lib.acDeviceReduceScal(self.handle, stream, rtype, handle, C.byref(r)),
               "acDeviceReduceScal")
        return float(r.value)

    def reduce_vec(self, rtype: int, a: int, b: int, c: int, stream: int = 0) -> float:
        r = self.prec.real()
        _check(self.lib.acDeviceReduceVec(self.handle, stream, rtype, a, b, c, C.byref(r)),
               "acDeviceReduceVec")
        return float(r.value)

    def reduce_scal_double(self, rtype: int, handle: int, stream: int = 0) -> float:
        r = C.c_double()
        _check(self.lib.acDeviceReduceScalDouble(self.handle, stream, rtype, handle, C.byref(r)),
               "acDeviceReduceScalDouble")
        return r.value

    def reduce_vec_double(self, rtype: int, a: int, b: int, c: int, stream: int = 0) -> float:
        r = C.c_double()
        _check(self.lib.acDeviceReduceVecDouble(self.handle, stream, rtype, a, b, c, C.byref(r)),
               "acDeviceReduceVecDouble")
        return r.value

    # --- plumbing -----------------------------------------------------------
    def synchronize(self, stream: int = abi.STREAM_ALL) -> None:
        _check(self.lib.acDeviceSynchronizeStream(self.handle, stream), "acDeviceSynchronizeStream")

    def status(self) -> int:
        s = C.c_uint()
        _check(self.lib.acDeviceGetStatus(self.handle, C.byref(s)), "acDeviceGetStatus")
        return s.value

    def reset_status(self) -> None:
        _check(self.lib.acDeviceResetStatus(self.handle), "acDeviceResetStatus")

    def check_wait_limit(self, seconds: float) -> None:
        """acDeviceCheckWaitLimit: a bounded wait on a barrier nothing completes
        must give up after `seconds` and raise status bit 0."""
        _check(self.lib.acDeviceCheckWaitLimit(self.handle, float(seconds)),
               "acDeviceCheckWaitLimit")

    def cuda_stream(self, stream: int = 0) -> int:
        p = C.c_void_p()
        _check(self.lib.acDeviceGetCudaStream(self.handle, stream, C.byref(p)),
               "acDeviceGetCudaStream")
        return p.value or 0

    def launch_count(self) -> int:
        c = C.c_ulonglong()
        _check(self.lib.acDeviceGetLaunchCount(self.handle, C.byref(c)), "acDeviceGetLaunchCount")
        return c.value

    def set_solve_config(self, cfg: int) -> None:
        _check(self.lib.acDeviceSetSolveConfig(self.handle, cfg), "acDeviceSetSolveConfig")

    def solve_config(self) -> tuple[int, int, str]:
        c, n = C.c_int(), C.c_int()
        _check(self.lib.acDeviceGetSolveConfig(self.handle, C.byref(c), C.byref(n)),
               "acDeviceGetSolveConfig")
        return c.value, n.value, self.lib.acSolveConfigName(c.value).decode()

    def auto_optimize(self) -> None:
        _check(self.lib.acDeviceAutoOptimize(self.handle), "acDeviceAutoOptimize")

    def memory_footprint(self) -> int:
        b = C.c_size_t()
        _check(self.lib.acDeviceGetMemoryFootprint(self.handle, C.byref(b)),
               "acDeviceGetMemoryFootprint")
        return b.value


class Ensemble:
    """Python mirror of the ensemble entry points (include/astaroth_b200.h):
    many independent meshes advanced by one launch per substep."""

    def __init__(self, flavour: str, infos, device_id: int = 0):
        self.flavour = flavour
        self.prec = abi.PRECISIONS[flavour]
        self.lib = library.load(flavour)
        Info = abi.info_type(self.prec)
        arr = (Info * len(infos))(*infos)
        self.infos = list(infos)
        self.handle = C.c_void_p()
        _check(self.lib.acEnsembleCreate(device_id, len(infos), arr, C.byref(self.handle)),
               "acEnsembleCreate")

    def destroy(self) -> None:
        if self.handle:
            self.lib.acEnsembleDestroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def load_member(self, m: int, host: abi.HostMesh) -> None:
        _check(self.lib.acEnsembleLoadMember(self.handle, m, host.cmesh), "acEnsembleLoadMember")

    def store_member(self, m: int, host: abi.HostMesh) -> None:
        _check(self.lib.acEnsembleStoreMember(self.handle, m, C.byref(host.cmesh)),
               "acEnsembleStoreMember")

    def integrate_step(self, dt: float) -> None:
        _check(self.lib.acEnsembleIntegrateStep(self.handle, dt), "acEnsembleIntegrateStep")

    def integrate_steps(self, dt: float, n: int) -> None:
        _check(self.lib.acEnsembleIntegrateSteps(self.handle, dt, n), "acEnsembleIntegrateSteps")

    def synchronize(self) -> None:
        _check(self.lib.acEnsembleSynchronize(self.handle), "acEnsembleSynchronize")

    def status(self) -> int:
        s = C.c_uint()
        _check(self.lib.acEnsembleGetStatus(self.handle, C.byref(s)), "acEnsembleGetStatus")
        return s.value

    def cuda_stream(self) -> int:
        p = C.c_void_p()
        _check(self.lib.acEnsembleGetCudaStream(self.handle, C.byref(p)), "acEnsembleGetCudaStream")
        return p.value or 0

    def launch_count(self) -> int:
        c = C.c_ulonglong()
        _check(self.lib.acEnsembleGetLaunchCount(self.handle, C.byref(c)), "acEnsembleGetLaunchCount")
        return c.value

    def set_schedule(self, config: int, segment_planes: int) -> None:
        _check(self.lib.acEnsembleSetSchedule(self.handle, config, segment_planes),
               "acEnsembleSetSchedule")

    def schedule(self) -> tuple[int, int]:
        c, s = C.c_int(), C.c_int()
        _check(self.lib.acEnsembleGetSchedule(self.handle, C.byref(c), C.byref(s)),
               "acEnsembleGetSchedule")
        return c.value, s.value

    def auto_optimize(self, cache_path: str | None = None) -> None:
        _check(self.lib.acEnsembleAutoOptimize(self.handle,
                                               cache_path.encode() if cache_path else None),
               "acEnsembleAutoOptimize")


def forcing_params_from_uniforms(flavour: str, info, u) -> object:
    """acForcingParamsFromUniforms: the step's forcing from five draws in [0, 1]."""
    prec = abi.PRECISIONS[flavour]
    lib = library.load(flavour)
    out = abi.forcing_type(prec)()
    arr = (prec.real * 5)(*[float(x) for x in u])
    _check(lib.acForcingParamsFromUniforms(info, arr, C.byref(out)), "acForcingParamsFromUniforms")
    return out


class ForcingGenerator:
    """acForcingParamsGenerate: a reproducible stream of per-step forcing
    parameters from a seed."""

    def __init__(self, flavour: str, info, seed: int):
        self.prec = abi.PRECISIONS[flavour]
        self.lib = library.load(flavour)
        self.info = info
        self.state = C.c_ulonglong(seed)

    def next(self):
        out = abi.forcing_type(self.prec)()
        _check(self.lib.acForcingParamsGenerate(self.info, C.byref(self.state), C.byref(out)),
               "acForcingParamsGenerate")
        return out


"""Loads the in-tree C-ABI libraries (astaroth_b200/lib/libastaroth_{sp,dp,mixed}.so)
and declares the prototypes of include/astaroth.h, astaroth_utils.h and
astaroth_b200.h for ctypes.

There is no fallback: if a library is missing, loading raises. Build with
`python -m astaroth_b200.build`.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

LIBDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

# every function the three headers declare (the boundary a caller binds)
ASTAROTH_H = [
    "acInit", "acQuit", "acCheckDeviceAvailability", "acSynchronizeStream", "acSynchronizeMesh",
    "acLoadDeviceConstant", "acLoad", "acSetVertexBuffer", "acStore", "acIntegrate",
    "acIntegrateGBC", "acBoundcondStep", "acBoundcondStepGBC", "acReduceScal", "acReduceVec",
    "acReduceVecScal", "acStoreWithOffset", "acIntegrateStep", "acIntegrateStepWithOffset",
    "acSynchronize", "acLoadWithOffset", "acGetNumDevicesPerNode", "acGetNode",
    "acNodeCreate", "acNodeDestroy", "acNodePrintInfo", "acNodeQueryDeviceConfiguration",
    "acNodeAutoOptimize", "acNodeSynchronizeStream", "acNodeSynchronizeVertexBuffer",
    "acNodeSynchronizeMesh", "acNodeSwapBuffers", "acNodeLoadConstant",
    "acNodeLoadVertexBufferWithOffset", "acNodeLoadMeshWithOffset", "acNodeLoadVertexBuffer",
    "acNodeLoadMesh", "acNodeSetVertexBuffer", "acNodeStoreVertexBufferWithOffset",
    "acNodeStoreMeshWithOffset", "acNodeStoreVertexBuffer", "acNodeStoreMesh",
    "acNodeIntegrateSubstep", "acNodeIntegrate", "acNodeIntegrateGBC",
    "acNodePeriodicBoundcondStep", "acNodePeriodicBoundconds", "acNodeGeneralBoundcondStep",
    "acNodeGeneralBoundconds", "acNodeReduceScal", "acNodeReduceVec", "acNodeReduceVecScal",
    "acDeviceCreate", "acDeviceDestroy", "acDevicePrintInfo", "acDeviceAutoOptimize",
    "acDeviceSynchronizeStream", "acDeviceSwapBuffers", "acDeviceLoadScalarUniform",
    "acDeviceLoadVectorUniform", "acDeviceLoadIntUniform", "acDeviceLoadInt3Uniform",
    "acDeviceLoadScalarArray", "acDeviceLoadMeshInfo", "acDeviceLoadDefaultUniforms",
    "acDeviceLoadVertexBufferWithOffset", "acDeviceLoadMeshWithOffset", "acDeviceLoadVertexBuffer",
    "acDeviceLoadMesh", "acDeviceSetVertexBuffer", "acDeviceStoreVertexBufferWithOffset",
    "acDeviceStoreMeshWithOffset", "acDeviceStoreVertexBuffer", "acDeviceStoreMesh",
    "acDeviceTransferVertexBufferWithOffset", "acDeviceTransferMeshWithOffset",
    "acDeviceTransferVertexBuffer", "acDeviceTransferMesh", "acDeviceIntegrateSubstep",
    "acDevicePeriodicBoundcondStep", "acDevicePeriodicBoundconds", "acDeviceGeneralBoundcondStep",
    "acDeviceGeneralBoundconds", "acDeviceReduceScal", "acDeviceReduceVec",
    "acDeviceReduceVecScal", "acDeviceRunMPITest",
    "acHostUpdateBuiltinParams", "acHostMeshCreate", "acHostMeshRandomize", "acHostMeshDestroy",
]
ASTAROTH_UTILS_H = [
    "acLoadConfig", "acHostVertexBufferSet", "acHostMeshSet", "acHostMeshApplyPeriodicBounds",
    "acHostMeshClear", "acHostIntegrateStep", "acHostReduceScal", "acHostReduceVec", "acGetError",
    "acEvalError", "acVerifyMesh",
]
ASTAROTH_B200_H = [
    "acDeviceGetStatus", "acDeviceResetStatus", "acDeviceCheckWaitLimit",
    "acDeviceGetCudaStream", "acDeviceGetLaunchCount",
    "acDeviceSetSolveConfig", "acDeviceGetSolveConfig", "acSolveConfigName",
    "acDeviceGetMemoryFootprint", "acDeviceIntegrateStep", "acDeviceIntegrateSteps",
    "acDeviceIntegrateStepCFL", "acDeviceIntegrateStepsCFL", "acDeviceGetTimestepRecord",
    "acDeviceSetSimulationTime",
    "acDeviceSetStepDiagnostics", "acDeviceSetForcing", "acDeviceLoadVertexBufferDouble", "acDeviceStoreVertexBufferDouble",
    "acDeviceReduceScalDouble", "acDeviceReduceVecDouble", "acReduceScalNoAlloc",
    "acForcingParamsFromUniforms", "acForcingParamsGenerate", "acDeviceLoadForcingParams",
    "acEnsembleCreate", "acEnsembleDestroy", "acEnsembleLoadMember", "acEnsembleStoreMember",
    "acEnsembleIntegrateStep", "acEnsembleIntegrateSteps", "acEnsembleSynchronize",
    "acEnsembleGetStatus", "acEnsembleGetCudaStream", "acEnsembleGetLaunchCount",
    "acEnsembleSetSchedule", "acEnsembleGetSchedule", "acEnsembleAutoOptimize",
]
ALL_SYMBOLS = ASTAROTH_H + ASTAROTH_UTILS_H + ASTAROTH_B200_H


def lib_file(flavour: str) -> str:
    return os.path.join(LIBDIR, f"libastaroth_{flavour}.so")


def _declare(lib: C.CDLL, prec: abi.Precision) -> None:
    R = prec.real
    Info = abi.info_type(prec)
    Mesh = abi.mesh_type(prec)
    Frc = abi.forcing_type(prec)
    I3 = abi.int3
    Dev = C.c_void_p
    res = C.c_int
    i = C.c_int
    d = lib
    sig = {
        "acDeviceCreate": (res, [i, Info, C.POINTER(Dev)]),
        "acDeviceDestroy": (res, [Dev]),
        "acDevicePrintInfo": (res, [Dev]),
        "acDeviceAutoOptimize": (res, [Dev]),
        "acDeviceSynchronizeStream": (res, [Dev, i]),
        "acDeviceSwapBuffers": (res, [Dev]),
        "acDeviceLoadScalarUniform": (res, [Dev, i, i, R]),
        "acDeviceLoadIntUniform": (res, [Dev, i, i, i]),
        "acDeviceLoadInt3Uniform": (res, [Dev, i, i, I3]),
        "acDeviceLoadMeshInfo": (res, [Dev, Info]),
        "acDeviceLoadDefaultUniforms": (res, [Dev]),
        "acDeviceLoadVertexBufferWithOffset": (res, [Dev, i, Mesh, i, I3, I3, i]),
        "acDeviceLoadMeshWithOffset": (res, [Dev, i, Mesh, I3, I3, i]),
        "acDeviceLoadVertexBuffer": (res, [Dev, i, Mesh, i]),
        "acDeviceLoadMesh": (res, [Dev, i, Mesh]),
        "acDeviceSetVertexBuffer": (res, [Dev, i, i, R]),
        "acDeviceStoreVertexBufferWithOffset": (res, [Dev, i, i, I3, I3, i, C.POINTER(Mesh)]),
        "acDeviceStoreMeshWithOffset": (res, [Dev, i, I3, I3, i, C.POINTER(Mesh)]),
        "acDeviceStoreVertexBuffer": (res, [Dev, i, i, C.POINTER(Mesh)]),
        "acDeviceStoreMesh": (res, [Dev, i, C.POINTER(Mesh)]),
        "acDeviceTransferVertexBufferWithOffset": (res, [Dev, i, i, I3, I3, i, Dev]),
        "acDeviceTransferVertexBuffer": (res, [Dev, i, i, Dev]),
        "acDeviceTransferMesh": (res, [Dev, i, Dev]),
        "acDeviceIntegrateSubstep": (res, [Dev, i, i, I3, I3, R]),
        "acDevicePeriodicBoundcondStep": (res, [Dev, i, i, I3, I3]),
        "acDevicePeriodicBoundconds": (res, [Dev, i, I3, I3]),
        "acDeviceGeneralBoundcondStep": (res, [Dev, i, i, I3, I3, Info, I3]),
        "acDeviceGeneralBoundconds": (res, [Dev, i, I3, I3, Info, I3]),
        "acDeviceReduceScal": (res, [Dev, i, i, i, C.POINTER(R)]),
        "acDeviceReduceVec": (res, [Dev, i, i, i, i, i, C.POINTER(R)]),
        "acDeviceReduceVecScal": (res, [Dev, i, i, i, i, i, i, C.POINTER(R)]),
        # node
        "acNodeCreate": (res, [i, Info, C.POINTER(Dev)]),
        "acNodeDestroy": (res, [Dev]),
        "acNodeIntegrate": (res, [Dev, R]),
        "acNodeIntegrateSubstep": (res, [Dev, i, i, I3, I3, R]),
        "acNodeLoadMesh": (res, [Dev, i, Mesh]),
        "acNodeStoreMesh": (res, [Dev, i, C.POINTER(Mesh)]),
        "acNodePeriodicBoundconds": (res, [Dev, i]),
        "acNodeReduceScal": (res, [Dev, i, i, i, C.POINTER(R)]),
        "acNodeReduceVec": (res, [Dev, i, i, i, i, i, C.POINTER(R)]),
        "acNodeSynchronizeStream": (res, [Dev, i]),
        "acNodeSwapBuffers": (res, [Dev]),
        # legacy
        "acInit": (res, [Info]),
        "acQuit": (res, []),
        "acIntegrateGBC": (res, [Info, R]),
        "acBoundcondStepGBC": (res, [Info]),
        "acLoad": (res, [Mesh]),
        "acStore": (res, [C.POINTER(Mesh)]),
        "acIntegrate": (res, [R]),
        "acIntegrateStep": (res, [i, R]),
        "acBoundcondStep": (res, []),
        "acReduceScal": (R, [i, i]),
        "acReduceVec": (R, [i, i, i, i]),
        "acSynchronize": (res, []),
        "acCheckDeviceAvailability": (res, []),
        "acGetNumDevicesPerNode": (i, []),
        # host helpers and utils
        "acHostUpdateBuiltinParams": (res, [C.POINTER(Info)]),
        "acHostMeshCreate": (res, [Info, C.POINTER(Mesh)]),
        "acHostMeshRandomize": (res, [C.POINTER(Mesh)]),
        "acHostMeshDestroy": (res, [C.POINTER(Mesh)]),
        "acLoadConfig": (res, [C.c_char_p, C.POINTER(Info)]),
        "acHostMeshApplyPeriodicBounds": (res, [C.POINTER(Mesh)]),
        "acHostIntegrateStep": (res, [Mesh, R]),
        "acHostReduceScal": (R, [Mesh, i, i]),
        "acHostReduceVec": (R, [Mesh, i, i, i, i]),
        "acVerifyMesh": (res, [C.c_char_p, Mesh, Mesh]),
        # additions
        "acDeviceGetStatus": (res, [Dev, C.POINTER(C.c_uint)]),
        "acDeviceResetStatus": (res, [Dev]),
        "acDeviceCheckWaitLimit": (res, [Dev, C.c_double]),
        "acDeviceGetCudaStream": (res, [Dev, i, C.POINTER(C.c_void_p)]),
        "acDeviceGetLaunchCount": (res, [Dev, C.POINTER(C.c_ulonglong)]),
        "acDeviceSetSolveConfig": (res, [Dev, i]),
        "acDeviceGetSolveConfig": (res, [Dev, C.POINTER(i), C.POINTER(i)]),
        "acSolveConfigName": (C.c_char_p, [i]),
        "acDeviceGetMemoryFootprint": (res, [Dev, C.POINTER(C.c_size_t)]),
        "acDeviceIntegrateStep": (res, [Dev, i, R]),
        "acDeviceIntegrateSteps": (res, [Dev, i, R, i]),
        "acDeviceIntegrateStepCFL": (res, [Dev, i, R]),
        "acDeviceIntegrateStepsCFL": (res, [Dev, i, R, i]),
        "acDeviceGetTimestepRecord": (res, [Dev, i, C.POINTER(R), C.POINTER(C.c_double),
                                            C.POINTER(C.c_ulonglong)]),
        "acDeviceSetSimulationTime": (res, [Dev, i, C.c_double]),
        "acDeviceSetStepDiagnostics": (res, [Dev, i]),
        "acDeviceSetForcing": (res, [Dev, i]),
        "acDeviceLoadVertexBufferDouble": (res, [Dev, i, i, C.c_void_p]),
        "acDeviceStoreVertexBufferDouble": (res, [Dev, i, i, C.c_void_p]),
        "acDeviceReduceScalDouble": (res, [Dev, i, i, i, C.POINTER(C.c_double)]),
        "acDeviceReduceVecDouble": (res, [Dev, i, i, i, i, i, C.POINTER(C.c_double)]),
        "acReduceScalNoAlloc": (res, [C.c_void_p, i, C.c_void_p, i, i, i, C.c_void_p]),
        "acForcingParamsFromUniforms": (res, [Info, C.POINTER(R), C.POINTER(Frc)]),
        "acForcingParamsGenerate": (res, [Info, C.POINTER(C.c_ulonglong), C.POINTER(Frc)]),
        "acDeviceLoadForcingParams": (res, [Dev, i, Frc]),
        # ensembles
        "acEnsembleCreate": (res, [i, i, C.POINTER(Info), C.POINTER(Dev)]),
        "acEnsembleDestroy": (res, [Dev]),
        "acEnsembleLoadMember": (res, [Dev, i, Mesh]),
        "acEnsembleStoreMember": (res, [Dev, i, C.POINTER(Mesh)]),
        "acEnsembleIntegrateStep": (res, [Dev, R]),
        "acEnsembleIntegrateSteps": (res, [Dev, R, i]),
        "acEnsembleSynchronize": (res, [Dev]),
        "acEnsembleGetStatus": (res, [Dev, C.POINTER(C.c_uint)]),
        "acEnsembleGetCudaStream": (res, [Dev, C.POINTER(C.c_void_p)]),
        "acEnsembleGetLaunchCount": (res, [Dev, C.POINTER(C.c_ulonglong)]),
        "acEnsembleSetSchedule": (res, [Dev, i, i]),
        "acEnsembleGetSchedule": (res, [Dev, C.POINTER(i), C.POINTER(i)]),
        "acEnsembleAutoOptimize": (res, [Dev, C.c_char_p]),
    }
    for name, (rt, args) in sig.items():
        fn = getattr(d, name)
        fn.restype = rt
        fn.argtypes = args


_CACHE: dict[str, C.CDLL] = {}


def load(flavour: str) -> C.CDLL:
    """The library of one flavour ("sp", "dp" or "mixed"), prototypes declared.
    Raises if it was not built: there is no CPU fallback."""
    if flavour not in _CACHE:
        path = lib_file(flavour)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run `python -m astaroth_b200.build`")
        lib = C.CDLL(path)
        _declare(lib, abi.PRECISIONS[flavour])
        _CACHE[flavour] = lib
    return _CACHE[flavour]


def missing_symbols(flavour: str) -> list[str]:
    """Names declared by the headers that the library does not export."""
    lib = C.CDLL(lib_file(flavour))
    out = []
    for s in ALL_SYMBOLS:
        try:
            getattr(lib, s)
        except AttributeError:
            out.append(s)
    return out

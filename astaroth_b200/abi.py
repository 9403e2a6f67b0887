"""ctypes mirror of the C interface in include/astaroth.h.

The enum tables are parsed from include/user_defines.h at import time, so the
Python side can never drift from the header the C libraries are built from.
Layouts follow the reference's include/astaroth.h:109-119 (AcMeshInfo: ints,
int3s, reals, real3s; AcMesh: eight vertex-buffer pointers then the info).
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE_DIR = os.path.join(REPO, "include")

STENCIL_ORDER = 6
NGHOST = STENCIL_ORDER // 2


def _parse_xmacro(text: str, name: str) -> list[str]:
    m = re.search(r"#define\s+" + name + r"\(FUNC\)((?:[^\n]*\\\n)*[^\n]*)", text)
    if m is None:
        raise RuntimeError(f"{name} not found in user_defines.h")
    return re.findall(r"FUNC\((\w+)\)", m.group(1))


with open(os.path.join(INCLUDE_DIR, "user_defines.h")) as _f:
    _UD = _f.read()

INT_PARAMS = _parse_xmacro(_UD, "AC_FOR_USER_INT_PARAM_TYPES")
INT3_PARAMS = _parse_xmacro(_UD, "AC_FOR_USER_INT3_PARAM_TYPES")
REAL_PARAMS = _parse_xmacro(_UD, "AC_FOR_USER_REAL_PARAM_TYPES")
REAL3_PARAMS = _parse_xmacro(_UD, "AC_FOR_USER_REAL3_PARAM_TYPES")
VTXBUFS = _parse_xmacro(_UD, "AC_FOR_VTXBUF_HANDLES")
RTYPES = _parse_xmacro(_UD, "AC_FOR_RTYPES")
NUM_STREAMS = int(re.search(r"#define NUM_STREAMS \((\d+)\)", _UD).group(1))
STREAM_DEFAULT = 0
STREAM_ALL = NUM_STREAMS

# enum values as module attributes: AC_nx, AC_dsx, VTXBUF_UUX, RTYPE_RMS, ...
for _table in (INT_PARAMS, INT3_PARAMS, REAL_PARAMS, REAL3_PARAMS, VTXBUFS, RTYPES):
    for _i, _n in enumerate(_table):
        globals()[_n] = _i

NUM_INT_PARAMS = len(INT_PARAMS)
NUM_INT3_PARAMS = len(INT3_PARAMS)
NUM_REAL_PARAMS = len(REAL_PARAMS)
NUM_REAL3_PARAMS = len(REAL3_PARAMS)
NUM_VTXBUF_HANDLES = len(VTXBUFS)
AC_SUCCESS, AC_FAILURE = 0, 1
# include/astaroth.h AcBoundcond
AC_BOUNDCOND_PERIODIC, AC_BOUNDCOND_SYMMETRIC, AC_BOUNDCOND_ANTISYMMETRIC = 0, 1, 2


class int3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


@dataclass(frozen=True)
class Precision:
    """One build flavour of the library: the C type of AcReal and its name."""

    name: str  # "sp", "dp" or "mixed"
    real: type  # ctypes.c_float or ctypes.c_double
    np_dtype: type

    @property
    def double(self) -> bool:
        return self.real is C.c_double


def _make_types(real):
    class real3(C.Structure):
        _fields_ = [("x", real), ("y", real), ("z", real)]

    class AcMeshInfo(C.Structure):
        _fields_ = [
            ("int_params", C.c_int * NUM_INT_PARAMS),
            ("int3_params", int3 * NUM_INT3_PARAMS),
            ("real_params", real * NUM_REAL_PARAMS),
            ("real3_params", real3 * NUM_REAL3_PARAMS),
        ]

    class AcMesh(C.Structure):
        _fields_ = [
            ("vertex_buffer", C.POINTER(real) * NUM_VTXBUF_HANDLES),
            ("info", AcMeshInfo),
        ]

    return real3, AcMeshInfo, AcMesh


_F_REAL3, AcMeshInfoF, AcMeshF = _make_types(C.c_float)
_D_REAL3, AcMeshInfoD, AcMeshD = _make_types(C.c_double)

SP = Precision("sp", C.c_float, np.float32)
DP = Precision("dp", C.c_double, np.float64)
MIXED = Precision("mixed", C.c_float, np.float32)
PRECISIONS = {"sp": SP, "dp": DP, "mixed": MIXED}


def info_type(prec: Precision):
    return AcMeshInfoD if prec.double else AcMeshInfoF


def mesh_type(prec: Precision):
    return AcMeshD if prec.double else AcMeshF


def _forcing_fields(R):
    return [("magnitude", R), ("k_force", R * 3), ("ff_hel_re", R * 3), ("ff_hel_im", R * 3),
            ("phase", R), ("kaver", R)]


class AcForcingParamsF(C.Structure):
    """include/astaroth_b200.h AcForcingParams, single-precision builds."""
    _fields_ = _forcing_fields(C.c_float)


class AcForcingParamsD(C.Structure):
    """include/astaroth_b200.h AcForcingParams, double-precision build."""
    _fields_ = _forcing_fields(C.c_double)


def forcing_type(prec: Precision):
    return AcForcingParamsD if prec.double else AcForcingParamsF


def real3_type(prec: Precision):
    return _D_REAL3 if prec.double else _F_REAL3


# Values of config/astaroth.conf in the reference (the AC_DEFAULT_CONFIG the
# samples load), used for every parameter a workload does not set.
DEFAULT_CONFIG = {
    "AC_nx": 64, "AC_ny": 64, "AC_nz": 64,
    "AC_dsx": 0.04908738521, "AC_dsy": 0.04908738521, "AC_dsz": 0.04908738521,
    "AC_bc_type_top_x": 0, "AC_bc_type_top_y": 0, "AC_bc_type_top_z": 0,
    "AC_bc_type_bot_x": 0, "AC_bc_type_bot_y": 0, "AC_bc_type_bot_z": 0,
    "AC_max_steps": 1001, "AC_save_steps": 10, "AC_bin_steps": 1000,
    "AC_bin_save_t": float("inf"), "AC_start_step": 0, "AC_max_time": -1.0,
    "AC_cdt": 0.4, "AC_cdtv": 0.3, "AC_cdts": 1.0,
    "AC_nu_visc": 5e-3, "AC_cs_sound": 1.0, "AC_zeta": 0.01,
    "AC_eta": 5e-3, "AC_mu0": 1.4,
    "AC_relhel": 0.0, "AC_forcing_magnitude": 1e-5, "AC_kmin": 0.8, "AC_kmax": 1.2,
    "AC_switch_accretion": 0.0,
    "AC_cp_sound": 1.0, "AC_gamma": 0.5, "AC_lnT0": 1.2, "AC_lnrho0": 1.3,
    "AC_sink_pos_x": 3.14, "AC_sink_pos_y": 3.14, "AC_sink_pos_z": 3.14,
    "AC_M_sink_Msun": 1.0, "AC_soft": 0.12, "AC_accretion_range": 2.0,
    "AC_unit_velocity": 1.0, "AC_unit_density": 1.0, "AC_unit_length": 1.0,
    "AC_ampl_lnrho": 0.0, "AC_ampl_uu": 1.0,
}


def update_builtin_params(info) -> None:
    """Python twin of acHostUpdateBuiltinParams (reference src/core/astaroth.cc:190-227)."""
    ip = info.int_params
    ip[AC_mx] = ip[AC_nx] + STENCIL_ORDER
    ip[AC_my] = ip[AC_ny] + STENCIL_ORDER
    ip[AC_mz] = ip[AC_nz] + STENCIL_ORDER
    ip[AC_nx_min] = ip[AC_ny_min] = ip[AC_nz_min] = NGHOST
    ip[AC_nx_max] = NGHOST + ip[AC_nx]
    ip[AC_ny_max] = NGHOST + ip[AC_ny]
    ip[AC_nz_max] = NGHOST + ip[AC_nz]
    rp = info.real_params
    for a, inv in (("AC_dsx", "AC_inv_dsx"), ("AC_dsy", "AC_inv_dsy"), ("AC_dsz", "AC_inv_dsz")):
        ds = rp[globals()[a]]
        if isinstance(info, AcMeshInfoF):
            rp[globals()[inv]] = float(np.float32(1.0) / np.float32(ds))
        else:
            rp[globals()[inv]] = 1.0 / ds
    ip[AC_mxy] = ip[AC_mx] * ip[AC_my]
    ip[AC_nxy] = ip[AC_nx] * ip[AC_ny]
    ip[AC_nxyz] = ip[AC_nxy] * ip[AC_nz]


def make_info(prec: Precision, nx: int, ny: int | None = None, nz: int | None = None,
              unset_nan: bool = True, **overrides):
    """Build an AcMeshInfo the way acLoadConfig does (src/utils/config_loader.c:81-112):
    every word starts as 0xFF.. (NaN reals, -1 ints), the config values are
    applied, then the built-in params are derived. `overrides` use the enum
    names without the AC_ prefix or with it (nu_visc=... or AC_nu_visc=...)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    info = info_type(prec)()
    if unset_nan:
        C.memset(C.addressof(info), 0xFF, C.sizeof(info))
    cfg = dict(DEFAULT_CONFIG)
    cfg.update({"AC_nx": nx, "AC_ny": ny, "AC_nz": nz})
    for k, v in overrides.items():
        key = k if k.startswith("AC_") else "AC_" + k
        cfg[key] = v
    for k, v in cfg.items():
        if k in INT_PARAMS:
            info.int_params[INT_PARAMS.index(k)] = int(v)
        elif k in REAL_PARAMS:
            info.real_params[REAL_PARAMS.index(k)] = float(v)
        else:
            raise KeyError(f"unknown parameter {k}")
    update_builtin_params(info)
    return info


def set_real(info, name: str, value: float) -> None:
    key = name if name.startswith("AC_") else "AC_" + name
    info.real_params[REAL_PARAMS.index(key)] = float(value)


def get_real(info, name: str) -> float:
    key = name if name.startswith("AC_") else "AC_" + name
    return float(info.real_params[REAL_PARAMS.index(key)])


def get_int(info, name: str) -> int:
    key = name if name.startswith("AC_") else "AC_" + name
    return int(info.int_params[INT_PARAMS.index(key)])


def dims(info) -> tuple[int, int, int]:
    ip = info.int_params
    return ip[AC_nx], ip[AC_ny], ip[AC_nz]


class HostMesh:
    """A host AcMesh whose eight buffers are numpy arrays shaped (mz, my, mx)
    (C order, so flat index i + j*mx + k*mx*my as in the reference)."""

    def __init__(self, prec: Precision, info, fields: list[np.ndarray] | None = None,
                 pinned: bool = False):
        self.prec = prec
        nx, ny, nz = dims(info)
        shape = (nz + 2 * NGHOST, ny + 2 * NGHOST, nx + 2 * NGHOST)
        self.info = info
        self._pinned = None
        if fields is None:
            if pinned:
                import torch  # pinned host memory for end-to-end timing

                self._pinned = [torch.empty(shape, dtype=torch.float64 if prec.double else torch.float32)
                                .pin_memory() for _ in range(NUM_VTXBUF_HANDLES)]
                fields = [t.numpy() for t in self._pinned]
            else:
                fields = [np.zeros(shape, dtype=prec.np_dtype) for _ in range(NUM_VTXBUF_HANDLES)]
        self.fields = [np.ascontiguousarray(f, dtype=prec.np_dtype) for f in fields]
        for f in self.fields:
            assert f.shape == shape
        self.cmesh = mesh_type(prec)()
        for w, f in enumerate(self.fields):
            self.cmesh.vertex_buffer[w] = f.ctypes.data_as(C.POINTER(prec.real))
        self.cmesh.info = info

    def interior(self, w: int) -> np.ndarray:
        g = NGHOST
        return self.fields[w][g:-g, g:-g, g:-g]

    def copy(self) -> "HostMesh":
        return HostMesh(self.prec, self.info, [f.copy() for f in self.fields])

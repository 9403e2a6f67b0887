"""Test-side loaders for the CPU checker under oracle/.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module. It wraps
  - oracle/_build/liboracle_{f32,f64,f80}.so : the C restatement (mhd_oracle.c)
  - oracle/_ref/libref_utils_{sp,dp}.so      : the reference's own host utils
                                               (built only where the reference
                                               sources exist; optional)
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

from astaroth_b200 import abi

REPO = abi.REPO
ORACLE_DIR = os.path.join(REPO, "oracle")
# the reference sources (present only where the checker is built; the built
# files travel with the repository)
REFERENCE = os.environ.get("ASTAROTH_REFERENCE", "/root/reference")
KIND_DTYPE = {"f32": np.float32, "f64": np.float64, "f80": np.longdouble}


class OracleParams(C.Structure):
    _fields_ = [
        ("dsx", C.c_double), ("dsy", C.c_double), ("dsz", C.c_double),
        ("nu_visc", C.c_double), ("eta", C.c_double), ("mu0", C.c_double),
        ("cs_sound", C.c_double), ("cp_sound", C.c_double), ("gamma", C.c_double),
        ("lnT0", C.c_double), ("lnrho0", C.c_double), ("zeta", C.c_double),
        ("forcing", C.c_int),
        ("forcing_magnitude", C.c_double), ("forcing_phase", C.c_double), ("kaver", C.c_double),
        ("k_force", C.c_double * 3), ("ff_re", C.c_double * 3), ("ff_im", C.c_double * 3),
    ]


def ensure_built() -> None:
    need = [os.path.join(ORACLE_DIR, "_build", f"liboracle_{k}.so") for k in KIND_DTYPE]
    if not all(os.path.exists(p) for p in need):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


_LIBS: dict[str, C.CDLL] = {}


def oracle_lib(kind: str) -> C.CDLL:
    if kind not in _LIBS:
        ensure_built()
        lib = C.CDLL(os.path.join(ORACLE_DIR, "_build", f"liboracle_{kind}.so"))
        lib.oracle_step.restype = C.c_int
        lib.oracle_step.argtypes = [C.c_void_p * 8, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(OracleParams), C.c_double]
        if kind != "f80":  # the row-wise form (float and double builds)
            lib.oracle_step_rows.restype = C.c_int
            lib.oracle_step_rows.argtypes = lib.oracle_step.argtypes
        lib.oracle_periodic.restype = None
        lib.oracle_periodic.argtypes = [C.c_void_p * 8, C.c_int, C.c_int, C.c_int]
        lib.oracle_reduce.restype = C.c_double
        lib.oracle_reduce.argtypes = [C.c_void_p * 8, C.c_int, C.c_int * 3, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int]
        lib.oracle_diagnostics.restype = None
        lib.oracle_diagnostics.argtypes = [C.c_void_p * 8, C.c_int, C.c_int, C.c_int,
                                           C.c_double * 4]
        lib.oracle_omp_threads.restype = C.c_int
        lib.oracle_real_size.restype = C.c_int
        assert lib.oracle_real_size() == np.dtype(KIND_DTYPE[kind]).itemsize or kind == "f80"
        _LIBS[kind] = lib
    return _LIBS[kind]


def omp_threads() -> int:
    """Threads the oracle's OpenMP loops use in this process."""
    return int(oracle_lib("f64").oracle_omp_threads())


def params_from(info=None, **kw) -> OracleParams:
    """Oracle parameters, from an AcMeshInfo (the values the GPU sees) and/or keywords."""
    p = OracleParams()
    names = ["dsx", "dsy", "dsz", "nu_visc", "eta", "mu0", "cs_sound", "cp_sound", "gamma",
             "lnT0", "lnrho0", "zeta"]
    for n in names:
        if info is not None:
            setattr(p, n, abi.get_real(info, n))
    for k, v in kw.items():
        if k in ("k_force", "ff_re", "ff_im"):
            getattr(p, k)[:] = list(v)
        else:
            setattr(p, k, v)
    return p


def _ptrs(fields):
    arr = (C.c_void_p * 8)()
    for i, f in enumerate(fields):
        assert f.flags.c_contiguous
        arr[i] = f.ctypes.data
    return arr


class OracleMesh:
    """Eight (mz, my, mx) arrays of one oracle precision and a step method."""

    def __init__(self, kind: str, fields, nx: int, ny: int, nz: int):
        self.kind = kind
        self.lib = oracle_lib(kind)
        self.fields = [np.ascontiguousarray(f, dtype=KIND_DTYPE[kind]) for f in fields]
        self.n = (nx, ny, nz)

    def step(self, params: OracleParams, dt: float, nsteps: int = 1,
             vertexwise: bool = False) -> None:
        """nsteps RK3 steps. The float and double builds take the row-wise
        evaluation (oracle_step_rows, bit-identical to the vertex-wise
        oracle_step and many times faster) unless vertexwise is set."""
        fn = self.lib.oracle_step if vertexwise or self.kind == "f80" else self.lib.oracle_step_rows
        for _ in range(nsteps):
            rc = fn(_ptrs(self.fields), *self.n, C.byref(params), float(dt))
            assert rc == 0

    def periodic(self) -> None:
        self.lib.oracle_periodic(_ptrs(self.fields), *self.n)

    def reduce(self, rtype: int, handles, normalise: bool = True) -> float:
        h = (C.c_int * 3)(*(list(handles) + [0, 0, 0])[:3])
        return self.lib.oracle_reduce(_ptrs(self.fields), len(handles), h, *self.n, int(rtype),
                                      int(normalise))

    def diagnostics(self) -> tuple[float, float, float, float]:
        """max, min and rms of |u| and rms_exp of lnrho (oracle_diagnostics:
        OpenMP, long-double sums, RMS normalised as sqrt(sum / N))."""
        out = (C.c_double * 4)()
        self.lib.oracle_diagnostics(_ptrs(self.fields), *self.n, out)
        return tuple(out)

    def interior(self, w: int) -> np.ndarray:
        g = abi.NGHOST
        return self.fields[w][g:-g, g:-g, g:-g]


# --- the reference's own host utils (optional) ------------------------------
def ref_lib(prec_name: str, build: str = ""):
    """The reference's host utils: build "" is the bit-exact pinning build
    (-O3 -march=x86-64-v2 -ffp-contract=off), "avx2" the speed build
    (-O3 -march=x86-64-v3, GCC's default contraction), used only for timing."""
    suffix = f"_{build}" if build else ""
    path = os.path.join(ORACLE_DIR, "_ref", f"libref_utils_{prec_name}{suffix}.so")
    if not os.path.exists(path):
        return None
    prec = abi.PRECISIONS[prec_name]
    lib = C.CDLL(path)
    Mesh = abi.mesh_type(prec)
    lib.acHostIntegrateStep.restype = C.c_int
    lib.acHostIntegrateStep.argtypes = [Mesh, prec.real]
    lib.acHostReduceScal.restype = prec.real
    lib.acHostReduceScal.argtypes = [Mesh, C.c_int, C.c_int]
    lib.acHostReduceVec.restype = prec.real
    lib.acHostReduceVec.argtypes = [Mesh, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.acHostMeshApplyPeriodicBounds.restype = C.c_int
    lib.acHostMeshApplyPeriodicBounds.argtypes = [C.POINTER(Mesh)]
    lib.acLoadConfig.restype = C.c_int
    lib.acLoadConfig.argtypes = [C.c_char_p, C.POINTER(abi.info_type(prec))]
    return lib


def diagnostics(lnrho, ux, uy, uz):
    """The standalone's four step diagnostics of interior arrays: max, min and
    rms of |u| and rms_exp of lnrho, RMS as sqrt(sum / N) (modelreduce.c:76-209
    with the host normalisation), in double precision with pairwise sums (for
    candidate states held as arrays; OracleMesh.diagnostics for the oracle's)."""
    a = np.asarray(ux, dtype=np.float64)
    b = np.asarray(uy, dtype=np.float64)
    c = np.asarray(uz, dtype=np.float64)
    sq = a * a + b * b + c * c
    ln = np.sqrt(sq)
    e = np.exp(np.asarray(lnrho, dtype=np.float64))
    n = sq.size
    return (float(ln.max()), float(ln.min()), math.sqrt(float(sq.sum()) / n),
            math.sqrt(float((e * e).sum()) / n))


def normwise_error(candidate: np.ndarray, model: np.ndarray) -> float:
    """max |cand - model| / max |model| over the given arrays, in long double."""
    c = np.asarray(candidate, dtype=np.longdouble)
    m = np.asarray(model, dtype=np.longdouble)
    den = np.max(np.abs(m))
    num = np.max(np.abs(c - m))
    return float(num / den) if den > 0 else float(num)


def cfl_dt(prec, info, umax: float, timescale: float = 1.0) -> float:
    """The Courant time step as the library evaluates it on the device
    (astaroth_b200/csrc/device.cu: cfl_kernel): the reference standalone's
    host_timestep (samples/standalone/model/host_timestep.cc:33-60, vAmax = 0)
    in double precision instead of long double, umax rounded to AcReal first,
    AC_dsmin or else the smallest spacing, the product with timescale in AcReal."""
    R = prec.np_dtype
    g = lambda k: abi.get_real(info, k)  # noqa: E731
    u = float(R(umax))
    dsmin = g("dsmin")
    if not dsmin > 0:
        dsmin = min(g("dsx"), g("dsy"), g("dsz"))
    uu_dt = g("cdt") * dsmin / (abs(u) + math.sqrt(g("cs2_sound")))
    visc_dt = g("cdtv") * dsmin * dsmin / max(max(g("nu_visc"), g("eta")), max(g("gamma"), 0.0))
    return float(R(timescale) * R(min(uu_dt, visc_dt)))

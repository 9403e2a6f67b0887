"""The C-ABI boundary, checked without a GPU:
  - every function include/*.h declares is exported by all three libraries;
  - AcMeshInfo/AcMesh layouts seen by a C compiler equal the ctypes mirror;
  - the host utils (CPU functions of the library) agree with the reference's
    own host utils built from its sources (when present) and with the oracle;
  - the reference's ctest sample compiles and links against this library
    unchanged (when the reference sources are present).
No GPU compute is called here.
"""
import ctypes as C
import math
import os
import re
import subprocess

import numpy as np
import pytest

from astaroth_b200 import abi, init, library
import oracle_lib as O

REPO = abi.REPO
FLAVOURS = ("sp", "dp", "mixed")


def _header_functions():
    names = set()
    for h in ("astaroth.h", "astaroth_utils.h", "astaroth_b200.h"):
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"static inline[^{]*\{.*?\n\}", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?(?:AcResult|AcReal|int|Node|Error|bool|const char\s*\*)\s+"
                             r"(ac\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_function_count():
    names = _header_functions()
    # reference astaroth.h + astaroth_utils.h functions, plus the additions
    assert len(names) >= len(library.ASTAROTH_H) + len(library.ASTAROTH_UTILS_H)
    assert set(library.ALL_SYMBOLS) <= set(names) | {"acDeviceRunMPITest"}


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_library_exports_every_declared_symbol(flavour):
    path = library.lib_file(flavour)
    assert os.path.exists(path), "build the library first (python -m astaroth_b200.build)"
    lib = C.CDLL(path)  # loads without a GPU
    missing = [s for s in _header_functions() if not hasattr(lib, s)]
    assert not missing, missing


def test_enum_tables():
    assert abi.NUM_INT_PARAMS == 25
    assert abi.NUM_INT3_PARAMS == 2
    assert abi.NUM_REAL_PARAMS == 75
    assert abi.NUM_REAL3_PARAMS == 0
    assert abi.VTXBUFS == ["VTXBUF_LNRHO", "VTXBUF_UUX", "VTXBUF_UUY", "VTXBUF_UUZ",
                           "VTXBUF_AX", "VTXBUF_AY", "VTXBUF_AZ", "VTXBUF_ENTROPY"]
    assert abi.RTYPES[:4] == ["RTYPE_MAX", "RTYPE_MIN", "RTYPE_RMS", "RTYPE_RMS_EXP"]
    assert abi.RTYPE_SUM == 7
    assert abi.NUM_STREAMS == 32


_LAYOUT_C = r"""
#include <stddef.h>
#include <stdio.h>
#include "astaroth.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu\n", sizeof(AcMeshInfo), offsetof(AcMeshInfo, int3_params),
           offsetof(AcMeshInfo, real_params), sizeof(AcMesh), offsetof(AcMesh, info),
           sizeof(AcReal));
    return 0;
}
"""


@pytest.mark.parametrize("dp", [0, 1])
def test_struct_layout_matches_c_compiler(tmp_path, dp):
    src = tmp_path / "layout.c"
    src.write_text(_LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-DAC_DOUBLE_PRECISION={dp}", f"-I{REPO}/include",
                    "-I/usr/local/cuda/include", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    prec = abi.DP if dp else abi.SP
    Info, Mesh = abi.info_type(prec), abi.mesh_type(prec)
    want = [C.sizeof(Info), Info.int3_params.offset, Info.real_params.offset, C.sizeof(Mesh),
            Mesh.info.offset, C.sizeof(prec.real)]
    assert got == want


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_update_builtin_params_and_load_config(tmp_path, flavour):
    lib = library.load(flavour)
    prec = abi.PRECISIONS[flavour]
    cfg = tmp_path / "astaroth.conf"
    lines = [f"{k} = {v}" for k, v in abi.DEFAULT_CONFIG.items() if k != "AC_bin_save_t"]
    lines.append("AC_bin_save_t = 1e666")
    lines.append("AC_chi = 0.0001")  # unknown keys are ignored
    cfg.write_text("\n".join(lines) + "\n")
    info = abi.info_type(prec)()
    rc = lib.acLoadConfig(str(cfg).encode(), C.byref(info))
    assert rc == abi.AC_FAILURE  # int3 params are never set by a config file
    want = abi.make_info(prec, 64)
    for name in ("AC_mx", "AC_nx_max", "AC_nxyz", "AC_mxy"):
        assert abi.get_int(info, name) == abi.get_int(want, name)
    for name in ("AC_inv_dsx", "AC_nu_visc", "AC_gamma", "AC_lnrho0"):
        assert abi.get_real(info, name) == abi.get_real(want, name)
    assert math.isnan(abi.get_real(info, "AC_cs2_sound"))  # unset reals stay NaN
    ref = O.ref_lib(flavour)
    if ref is not None:
        info2 = abi.info_type(prec)()
        ref.acLoadConfig(str(cfg).encode(), C.byref(info2))
        assert bytes(info2) == bytes(info) or all(
            (a == b) or (math.isnan(a) and math.isnan(b))
            for a, b in zip(info.real_params, info2.real_params))


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_host_periodic_bounds_and_reductions(flavour):
    lib = library.load(flavour)
    prec = abi.PRECISIONS[flavour]
    nx, ny, nz = 9, 7, 8
    info = abi.make_info(prec, nx, ny, nz)
    rng = np.random.default_rng(5)
    fields = [np.zeros((nz + 6, ny + 6, nx + 6), prec.np_dtype) for _ in range(8)]
    inter = []
    for f in fields:
        v = rng.uniform(-0.5, 0.5, (nz, ny, nx)).astype(prec.np_dtype)
        f[3:-3, 3:-3, 3:-3] = v
        inter.append(v)
    hm = abi.HostMesh(prec, info, fields)
    lib.acHostMeshApplyPeriodicBounds(C.byref(hm.cmesh))
    for w in range(8):
        assert np.array_equal(hm.fields[w], init.wrap_ghosts(inter[w]))
    om = O.OracleMesh("f64" if flavour == "dp" else "f32", hm.fields, nx, ny, nz)
    tol = 1e-13 if flavour == "dp" else 1e-5
    for rt in (0, 1, 2, 3, 7):
        got = float(lib.acHostReduceScal(hm.cmesh, rt, 2))
        assert got == pytest.approx(om.reduce(rt, [2]), rel=tol)
        got = float(lib.acHostReduceVec(hm.cmesh, rt, 1, 2, 3))
        assert got == pytest.approx(om.reduce(rt, [1, 2, 3]), rel=tol)


@pytest.mark.parametrize("flavour", ["sp", "dp"])
def test_host_integrate_step_matches_oracle(flavour):
    lib = library.load(flavour)
    prec = abi.PRECISIONS[flavour]
    n = 12
    info = abi.make_info(prec, n, n, n, dsx=2 * math.pi / n, dsy=2 * math.pi / n,
                         dsz=2 * math.pi / n, gamma=5 / 3)
    fields = init.workload_fields(n, n, n, prec.np_dtype, seed=2, amplitude=0.05)
    hm = abi.HostMesh(prec, info, [f.copy() for f in fields])
    lib.acHostIntegrateStep(hm.cmesh, prec.real(1e-3))
    om = O.OracleMesh("f80", fields, n, n, n)
    om.step(O.params_from(info), float(prec.np_dtype(1e-3)))
    tol = 1e-13 if flavour == "dp" else 2e-6
    for w in range(8):
        assert O.normwise_error(hm.interior(w), om.interior(w)) <= tol, w


def ctest_binary():
    """The reference's samples/ctest/main.c compiled, unchanged, against
    include/ and linked to libastaroth_sp.so (built where the reference exists)."""
    return os.path.join(REPO, "oracle", "_ref", "ctest_sp")


def test_reference_ctest_links_unchanged():
    src = os.path.join(O.REFERENCE, "samples", "ctest", "main.c")
    if not os.path.exists(src):
        if os.path.exists(ctest_binary()):
            return
        pytest.skip("reference sources absent")
    os.makedirs(os.path.dirname(ctest_binary()), exist_ok=True)
    subprocess.run(["gcc", "-O2", "-DAC_DOUBLE_PRECISION=0", '-DAC_DEFAULT_CONFIG="astaroth.conf"',
                    f"-I{REPO}/include", "-I/usr/local/cuda/include", src, "-o", ctest_binary(),
                    f"-L{library.LIBDIR}", "-lastaroth_sp", f"-Wl,-rpath,{library.LIBDIR}"],
                   check=True)
    assert os.path.exists(ctest_binary())


def _header_arity():
    """Parameter count of every function include/*.h declares."""
    arity = {}
    for h in ("astaroth.h", "astaroth_utils.h", "astaroth_b200.h"):
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"static inline[^{]*\{.*?\n\}", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?(?:AcResult|AcReal|int|Node|Error|bool|const char\s*\*)"
                             r"\s+(ac\w+)\s*\(([^;{]*?)\)\s*;", text, flags=re.M | re.S):
            params = " ".join(m.group(2).split())
            arity[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return arity


@pytest.mark.parametrize("flavour", FLAVOURS)
def test_binding_prototypes_match_header_arity(flavour):
    """Every prototype the Python binding declares takes as many arguments as
    the header declares (catches a binding left behind by a header change)."""
    arity = _header_arity()
    lib = library.load(flavour)
    checked = 0
    for name in library.ALL_SYMBOLS:
        fn = getattr(lib, name, None)
        if fn is None or fn.argtypes is None or name not in arity:
            continue
        assert len(fn.argtypes) == arity[name], (name, len(fn.argtypes), arity[name])
        checked += 1
    assert checked >= 60, checked

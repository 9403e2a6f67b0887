"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own host
model (src/utils/modelsolver.c, modelreduce.c, memory.c), compiled from its
sources by oracle/Makefile into oracle/_ref/libref_utils_{sp,dp}.so.

The reference ships no golden vectors for this path; these fixtures are its
own outputs on small seeded meshes, so the oracle restatement (and through it
the GPU path) can be pinned on machines where the reference is absent.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from astaroth_b200 import abi, init  # noqa: E402
import oracle_lib as O  # noqa: E402

# name: (precision, nx, ny, nz, amplitude, velocity mode, steps, dt)
CASES = {
    "dp_8x10x12_a0.3": ("dp", 8, 10, 12, 0.3, 0.0, 2, 1e-3),
    "sp_8x10x12_a0.3": ("sp", 8, 10, 12, 0.3, 0.0, 2, 1e-3),
    "dp_16_a1e-3": ("dp", 16, 16, 16, 1e-3, 0.1, 3, 1e-3),
    "sp_16_a1e-3": ("sp", 16, 16, 16, 1e-3, 0.1, 3, 1e-3),
}
PHYS = dict(gamma=5.0 / 3.0, nu_visc=5e-3, eta=5e-3, cs_sound=1.0, cp_sound=1.0)


def case_info(prec, nx, ny, nz):
    return abi.make_info(prec, nx, ny, nz, dsx=2 * math.pi / nx, dsy=2 * math.pi / ny,
                         dsz=2 * math.pi / nz, **PHYS)


def run_case(name):
    pname, nx, ny, nz, amp, vel, steps, dt = CASES[name]
    prec = abi.PRECISIONS[pname]
    info = case_info(prec, nx, ny, nz)
    fields = init.workload_fields(nx, ny, nz, prec.np_dtype, seed=7, amplitude=amp,
                                  velocity_mode=vel)
    lib = O.ref_lib(pname)
    if lib is None:
        raise SystemExit("reference utils not built (oracle/_ref); run make -C oracle")
    hm = abi.HostMesh(prec, info, [f.copy() for f in fields])
    for _ in range(steps):
        lib.acHostIntegrateStep(hm.cmesh, prec.real(dt))
    lib.acHostMeshApplyPeriodicBounds(C_ptr(hm))
    out = {f"f{w}": hm.fields[w] for w in range(8)}
    red = []
    for rt in (0, 1, 2, 3, 7):
        for w in range(8):
            red.append(float(lib.acHostReduceScal(hm.cmesh, rt, w)))
        red.append(float(lib.acHostReduceVec(hm.cmesh, rt, 1, 2, 3)))
        red.append(float(lib.acHostReduceVec(hm.cmesh, rt, 4, 5, 6)))
    out["reductions"] = np.array(red, dtype=np.float64)
    out["meta"] = np.array([nx, ny, nz, steps], dtype=np.int64)
    out["dt_amp_vel"] = np.array([dt, amp, vel], dtype=np.float64)
    return out


def C_ptr(hm):
    import ctypes

    return ctypes.byref(hm.cmesh)


def main():
    for name in CASES:
        data = run_case(name)
        path = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(path, **data)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

// Shared definitions of the B200 MHD solver library.
//
// One source tree is compiled three times (see astaroth_b200/build.py):
//   sp     AC_DOUBLE_PRECISION=0                   float state, FP32 kernels
//   dp     AC_DOUBLE_PRECISION=1                   double state, FP64 kernels
//   mixed  AC_DOUBLE_PRECISION=0 ACB_MIXED=1       float interface; (hi, lo)
//          float state, FP32 stencils/RHS, compensated RK3 update, FP64 sums
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "astaroth.h"

#ifndef ACB_MIXED
#define ACB_MIXED 0
#endif

#define ACB_NF 8 // fields of the MHD module: lnrho, ux, uy, uz, ax, ay, az, entropy

// Stencil state element type (the hi part in the mixed build).
typedef AcReal state_t;

// ---------------------------------------------------------------------------
// Device memory layout of one field block (8 fields contiguous).
//
// Field f, vertex (i, j, k) with i in [0, mx), j in [0, my), k in [0, mz):
//     block + f * fstride + offx + i + j * mxp + k * mxp * my
// - mxp (row pitch) is a multiple of 32 bytes and >= offx + mx;
// - offx puts the first interior vertex (i = 3) of every row on a 32-byte
//   (one DRAM sector) boundary, so rows of interior stores are whole sectors;
// - fstride is a multiple of 256 bytes.
// The row pitch is the reason for the padding: TMA needs every global stride to
// be a multiple of 16 bytes, and mx = n + 6 is not in general.
// ---------------------------------------------------------------------------
struct Layout {
    int mx, my, mz;    // logical extents (n + 6)
    int nx, ny, nz;    // interior extents
    int mxp;           // row pitch, elements
    int offx;          // leading offset, elements
    long long plane;   // mxp * my
    long long fstride; // elements between fields
};

static inline Layout
make_layout(int nx, int ny, int nz, int elem_bytes)
{
    Layout L;
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.mx = nx + 2 * NGHOST;
    L.my = ny + 2 * NGHOST;
    L.mz = nz + 2 * NGHOST;
    const int sector = 32 / elem_bytes; // elements per 32-byte sector
    L.offx           = sector - NGHOST;
    L.mxp            = ((L.offx + L.mx + sector - 1) / sector) * sector;
    L.plane          = (long long)L.mxp * L.my;
    const long long q = 256 / elem_bytes;
    L.fstride         = ((L.offx + L.plane * L.mz + q - 1) / q) * q;
    return L;
}

__host__ __device__ __forceinline__ long long
lidx(const Layout& L, int i, int j, int k)
{
    return (long long)L.offx + i + (long long)j * L.mxp + (long long)k * L.plane;
}

// Status bits a kernel may raise in the per-device status word.
enum : unsigned {
    ACB_STATUS_TMA_TIMEOUT = 1u, // a bounded wait on a TMA barrier gave up
    ACB_STATUS_BAD_ARG     = 2u,
};

#define ACB_CUDA_CHECK(call)                                                                       \
    do {                                                                                           \
        cudaError_t err__ = (call);                                                                \
        if (err__ != cudaSuccess) {                                                                \
            fprintf(stderr, "astaroth_b200: CUDA error %s at %s:%d: %s\n", #call, __FILE__,       \
                    __LINE__, cudaGetErrorString(err__));                                          \
            return AC_FAILURE;                                                                     \
        }                                                                                          \
    } while (0)

// Shared definitions of the B200 MHD solver library.
//
// One source tree is compiled three times (see astaroth_b200/build.py):
//   sp     AC_DOUBLE_PRECISION=0                   float state, FP32 kernels
//   dp     AC_DOUBLE_PRECISION=1                   double state, FP64 kernels
//   mixed  AC_DOUBLE_PRECISION=0 ACB_MIXED=1       float interface; state of a
//          float hi and a bfloat16 lo part, FP32 stencils/RHS, compensated RK3
//          update, FP64 sums
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
// Device memory layout of one field block: ACB_NARR arrays of 8-byte elements,
// one element per vertex.
//   FP64 build: eight arrays, array f = field f (a double per vertex).
//   FP32 and mixed builds: four arrays of interleaved field pairs, (lnrho, ss),
//     (ux, ax), (uy, ay), (uz, az): element = (field A, field B) as two floats,
//     so one 8-byte load brings a stencil point of both fields of a pair (the
//     pairs are the fields whose stencils have the same shape). The mixed
//     build's lo parts use the same layout.
//
// Element of vertex (i, j, k), i in [0, mx), j in [0, my), k in [0, mz), of
// array a:  block + a * fstride + offx + i + j * mxp + k * mxp * my  (elements)
// - mxp (row pitch) is a multiple of 32 bytes and >= offx + mx;
// - offx puts the first interior vertex (i = 3) of every row on a 32-byte
//   (one DRAM sector) boundary, so rows of interior stores are whole sectors;
// - fstride is a multiple of 256 bytes.
// The row pitch is the reason for the padding: TMA needs every global stride to
// be a multiple of 16 bytes, and mx = n + 6 is not in general.
// ---------------------------------------------------------------------------
#define ACB_PAIRED (sizeof(state_t) == 4)
static constexpr int ACB_NARR  = ACB_PAIRED ? 4 : ACB_NF; // arrays of a block
static constexpr int ACB_LANES = ACB_PAIRED ? 2 : 1;      // state values per element
static constexpr int ACB_ELEM  = 8;                       // bytes per element

// array and lane of field f (lnrho 0, ux 1, uy 2, uz 3, ax 4, ay 5, az 6, ss 7)
__host__ __device__ constexpr int
acb_array(int f)
{
    return ACB_PAIRED ? (f < 4 ? f : (f == 7 ? 0 : f - 3)) : f;
}
__host__ __device__ constexpr int
acb_lane(int f)
{
    return ACB_PAIRED ? (f < 4 ? 0 : 1) : 0;
}
// the field held in lane l of array a
__host__ __device__ constexpr int
acb_field(int a, int l)
{
    return ACB_PAIRED ? (l == 0 ? a : (a == 0 ? 7 : a + 3)) : a;
}

// Mixed build: the lo parts of a block are stored in bfloat16. A pair array's
// two lo values (A, B) form one 32-bit bf16x2 word, and two pair arrays share an
// 8-byte element: lo array 0 holds (lnrho, ss) | (ux, ax), lo array 1 holds
// (uy, ay) | (uz, az), low word first. The lo block thus has ACB_LO_NARR arrays
// with the hi block's geometry (row pitch, offsets, array stride) and half its
// bytes. The state (hi, lo) keeps 24 + 8 significant bits plus the sign of lo:
// storing lo rounds it by at most 2^-9 of itself, at most 2^-34 of hi, far below
// the single-precision stencils' rounding.
typedef unsigned short lo16_t;
static constexpr int ACB_LO_NARR = 2; // lo arrays of a block
static constexpr int ACB_LO_STEP = 4; // bf16 values per 8-byte element

struct Layout {
    int mx, my, mz;    // logical extents (n + 6)
    int nx, ny, nz;    // interior extents
    int mxp;           // row pitch, elements
    int offx;          // leading offset, elements
    long long plane;   // mxp * my
    long long fstride; // elements between arrays
};

static inline Layout
make_layout(int nx, int ny, int nz)
{
    Layout L;
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.mx = nx + 2 * NGHOST;
    L.my = ny + 2 * NGHOST;
    L.mz = nz + 2 * NGHOST;
    const int sector = 32 / ACB_ELEM; // elements per 32-byte sector
    L.offx           = sector - NGHOST;
    L.mxp            = ((L.offx + L.mx + sector - 1) / sector) * sector;
    L.plane          = (long long)L.mxp * L.my;
    const long long q = 256 / ACB_ELEM;
    L.fstride         = ((L.offx + L.plane * L.mz + q - 1) / q) * q;
    return L;
}

// bytes of one block (hi, or the lo parts in the mixed build)
static inline size_t
block_bytes(const Layout& L)
{
    return (size_t)L.fstride * ACB_NARR * ACB_ELEM;
}

__host__ __device__ __forceinline__ long long
lidx(const Layout& L, int i, int j, int k)
{
    return (long long)L.offx + i + (long long)j * L.mxp + (long long)k * L.plane;
}

// Offset, in state values (floats or doubles), of field f at the element
// index id of a vertex (lidx): the field's value there is block[fidx(L, f, id)].
// A field's values are ACB_LANES apart: block + fidx(L, f, 0) is the field's
// base and its vertex id sits at base[id * ACB_LANES].
__host__ __device__ __forceinline__ long long
fidx(const Layout& L, int f, long long id)
{
    return ((long long)acb_array(f) * L.fstride + id) * ACB_LANES + acb_lane(f);
}

// bytes of one lo block (mixed build)
static inline size_t
lo_block_bytes(const Layout& L)
{
    return (size_t)L.fstride * ACB_LO_NARR * ACB_ELEM;
}

// The lo part of field f in a lo block, as bf16 values: the field's lo at
// vertex element id (lidx) is lo_field(...)[id * ACB_LO_STEP]. Null for a
// null block (builds without lo parts).
__host__ __device__ __forceinline__ lo16_t*
lo_field(lo16_t* lo_block, const Layout& L, int f)
{
    if (!lo_block)
        return nullptr;
    const int a = acb_array(f);
    return lo_block + (long long)(a >> 1) * L.fstride * ACB_LO_STEP + (a & 1) * 2 + acb_lane(f);
}

__device__ __forceinline__ float
lo16_to_float(lo16_t h)
{
    return __uint_as_float((uint32_t)h << 16);
}

// round to nearest even
__device__ __forceinline__ lo16_t
float_to_lo16(float f)
{
    unsigned short r;
    asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(r) : "f"(f));
    return r;
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

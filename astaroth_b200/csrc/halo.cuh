// Periodic ghost-zone fill.
//
// Reference behaviour (src/core/kernels/boundconds.cuh:131-190): every ghost
// vertex (i, j, k) of the box [start, end) takes the value of the interior
// vertex ((c - 3 + n) mod n) + 3 on each axis. Every source is an interior
// vertex, so all ghost vertices can be written concurrently.
//
// The reference launches one thread per vertex of the whole m^3 box per field
// (8 launches per call) and returns early for the 96.5% interior threads.
//
// Whole-box fill (the case every integration step takes): the ghost vertices
// split into two kinds of independent work units, all in one launch.
//   A. interior rows (j, k both interior): only the 3 + 3 x-ghosts. One thread
//      per (row, array) copies the six elements of both sides: 6 independent
//      loads before any store, or, with nx % 4 == 0, the two 32-byte sectors
//      that hold the ghosts (with one padding element each) as whole sectors.
//   B. ghost rows (j or k in the ghost zone): the whole row. One thread per
//      (row, array, 128-element chunk, lane) copies four elements 32 apart, so
//      each warp instruction is one coalesced 256-byte row segment and each
//      thread has 4 loads in flight.
// Both kinds move 8-byte elements of the block's arrays (a field pair, or one
// double), whatever the fields.
// A thread never stores before all its loads are issued, so memory-level
// parallelism comes from the thread count, not from the warp count per row.
// The mixed build's integration path fills the hi parts only (the stencils
// never read the lo parts of ghosts), and fills the lo block on its own (its
// ACB_LO_NARR arrays of 8-byte elements) only when the lo parts are read.
//
// Sub-box fill (any start/end, any field range): one warp per (j, k) row of the
// box, lane-strided; kept for the reference's partial-box API calls.
#pragma once
#include "common.cuh"

struct HaloArgs {
    Layout L;
    state_t* block; // block (in)
    lo16_t* lo;     // mixed build: lo block of `in` (bf16, see common.cuh; else null)
    int3 start, end;
    int f0, f1; // fields [f0, f1)
    long long rows;
};

__device__ __forceinline__ int
wrap_interior(int c, int n)
{
    return ((c - NGHOST + n) % n) + NGHOST;
}

// Fills the ghost vertices of row (j, k) of the box [start, end) for fields
// [f0, f1), with the 32 lanes of one warp.
__device__ __forceinline__ void
halo_row(const Layout& L, state_t* block, lo16_t* lo, int3 start, int3 end, int f0, int f1, int j,
         int k, int lane)
{
    const bool ghost_row = j < NGHOST || j >= NGHOST + L.ny || k < NGHOST || k >= NGHOST + L.nz;
    const int js         = wrap_interior(j, L.ny);
    const int ks         = wrap_interior(k, L.nz);
    const long long drow = lidx(L, 0, j, k);
    const long long srow = lidx(L, 0, js, ks);
    // field f's vertex id is at F[id * ACB_LANES], F = block + fidx(L, f, 0)
    constexpr int W = ACB_LANES;
    if (ghost_row) {
        for (int f = f0; f < f1; ++f) {
            state_t* F = block + fidx(L, f, 0);
            for (int i = start.x + lane; i < end.x; i += 32)
                F[(drow + i) * W] = F[(srow + wrap_interior(i, L.nx)) * W];
            if (ACB_MIXED && lo) {
                lo16_t* G = lo_field(lo, L, f);
                for (int i = start.x + lane; i < end.x; i += 32)
                    G[(drow + i) * ACB_LO_STEP] = G[(srow + wrap_interior(i, L.nx)) * ACB_LO_STEP];
            }
        }
    }
    else if (lane < 2 * NGHOST) {
        const int i = lane < NGHOST ? lane : L.nx + lane; // 0,1,2 and nx+3..nx+5
        if (i >= start.x && i < end.x) {
            const int is = wrap_interior(i, L.nx);
            for (int f = f0; f < f1; ++f) {
                state_t* F         = block + fidx(L, f, 0);
                F[(drow + i) * W] = F[(srow + is) * W];
                if (ACB_MIXED && lo) {
                    lo16_t* G                    = lo_field(lo, L, f);
                    G[(drow + i) * ACB_LO_STEP] = G[(srow + is) * ACB_LO_STEP];
                }
            }
        }
    }
}

static __global__ void __launch_bounds__(256)
halo_kernel(const HaloArgs a)
{
    const int lane       = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int ry = a.end.y - a.start.y;
    for (long long r = warp; r < a.rows; r += nwarps) {
        const int j = a.start.y + (int)(r % ry);
        const int k = a.start.z + (int)(r / ry);
        halo_row(a.L, a.block, a.lo, a.start, a.end, a.f0, a.f1, j, k, lane);
    }
}

// ---------------------------------------------------------------------------
// Whole-box fill of all fields (n >= NGHOST on every axis).

// 128-vertex chunks per ghost row.
__host__ __device__ __forceinline__ unsigned
halo_chunks(const Layout& L)
{
    return (unsigned)(L.mx + 127) / 128;
}

// Work units of kind A (interior rows x arrays) and A + B of one block of
// narr arrays (ACB_NARR for the fields, ACB_LO_NARR for the mixed lo block).
static inline long long
halo_units_a(const Layout& L, int narr = ACB_NARR)
{
    return (long long)L.ny * L.nz * narr;
}

static inline long long
halo_units(const Layout& L, int narr = ACB_NARR)
{
    const long long ghost_rows = (long long)L.my * L.mz - (long long)L.ny * L.nz;
    return halo_units_a(L, narr) + ghost_rows * narr * halo_chunks(L) * 32;
}

// Periodic source of ghost-or-interior coordinate c in [0, n + 6), n >= NGHOST.
__device__ __forceinline__ int
wrap_near(int c, int n)
{
    return c < NGHOST ? c + n : (c >= n + NGHOST ? c - n : c);
}

// The block's elements as 8-byte units (a field pair, or a double).
typedef unsigned long long helem_t;

// Kind A or B unit u of one block of narr arrays (the fields, or the mixed
// build's lo block: the same geometry).
__device__ __forceinline__ void
halo_unit_block(const Layout& L, helem_t* block, unsigned units_a, unsigned u, unsigned narr)
{
    if (u < units_a) {
        // kind A: x-ghosts of interior row r, array a
        const unsigned ar    = u % narr;
        const unsigned r     = u / narr;
        const unsigned kq    = r / (unsigned)L.ny;
        const int j          = NGHOST + (int)(r - kq * (unsigned)L.ny);
        const int k          = NGHOST + (int)kq;
        helem_t* F           = block + (long long)ar * L.fstride + lidx(L, 0, j, k);
        if ((L.nx & 3) == 0) {
            // offx = 1, nx % 4 == 0: x = -1..2 and x = nx+3..nx+6 are whole
            // 32-byte sectors of the row (x = -1 and x = nx+6 are row padding,
            // inside the row, and get their periodic images too), and so are
            // their sources x = nx-1..nx+2 and x = 3..6. Sector of x:
            // (offx + x) / 4.
            ulonglong2* R = reinterpret_cast<ulonglong2*>(F - L.offx);
            const int gl  = 2 * ((L.offx - 1) >> 2);        // x = -1
            const int gr  = 2 * ((L.offx + L.nx + 3) >> 2); // x = nx + 3
            const int sl  = 2 * ((L.offx + L.nx - 1) >> 2); // x = nx - 1
            const int sr  = 2 * ((L.offx + 3) >> 2);        // x = 3
            const ulonglong2 l0 = R[sl], l1 = R[sl + 1];
            const ulonglong2 r0 = R[sr], r1 = R[sr + 1];
            R[gl]     = l0;
            R[gl + 1] = l1;
            R[gr]     = r0;
            R[gr + 1] = r1;
            return;
        }
        helem_t v[2 * NGHOST];
#pragma unroll
        for (int q = 0; q < NGHOST; ++q) {
            v[q]          = F[L.nx + q];   // source of ghost q is nx + q
            v[NGHOST + q] = F[NGHOST + q]; // source of ghost nx + 3 + q is 3 + q
        }
#pragma unroll
        for (int q = 0; q < NGHOST; ++q) {
            F[q]                 = v[q];
            F[L.nx + NGHOST + q] = v[NGHOST + q];
        }
        return;
    }
    // kind B: 4 elements, 32 apart, of a 128-element chunk of ghost row `row`
    u -= units_a;
    const unsigned lane = u & 31;
    unsigned wq         = u >> 5;
    const unsigned ar   = wq % narr;
    wq /= narr;
    const unsigned nch   = halo_chunks(L);
    const unsigned row   = wq / nch;
    const unsigned chunk = wq - row * nch;
    // ghost rows: first the 6 ghost z planes (all j), then the 6 ghost j rows
    // of every interior z plane
    const unsigned zrows = 2 * NGHOST * (unsigned)L.my;
    int j, k;
    if (row < zrows) {
        const unsigned kk = row / (unsigned)L.my;
        j                 = (int)(row - kk * (unsigned)L.my);
        k                 = kk < NGHOST ? (int)kk : L.nz + (int)kk;
    }
    else {
        const unsigned rr = row - zrows;
        const unsigned kk = rr / (2 * NGHOST);
        const unsigned jj = rr - kk * (2 * NGHOST);
        k                 = NGHOST + (int)kk;
        j                 = jj < NGHOST ? (int)jj : L.ny + (int)jj;
    }
    const long long ao = (long long)ar * L.fstride;
    const long long d  = ao + lidx(L, 0, j, k);
    const long long sr = ao + lidx(L, 0, wrap_near(j, L.ny), wrap_near(k, L.nz));
    const int x0       = (int)(chunk * 128 + lane);
    helem_t v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int x = x0 + 32 * q;
        if (x < L.mx)
            v[q] = block[sr + wrap_near(x, L.nx)];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int x = x0 + 32 * q;
        if (x < L.mx)
            block[d + x] = v[q];
    }
}

// the field block (ACB_NARR arrays) of a whole-box fill
__device__ __forceinline__ void
halo_unit(const Layout& L, void* block, unsigned units_a, unsigned u)
{
    halo_unit_block(L, static_cast<helem_t*>(block), units_a, u, ACB_NARR);
}

// Whole-box fill of one block of narr arrays of 8-byte elements (the fields,
// or the mixed build's lo block).
static __global__ void __launch_bounds__(256)
halo_full_kernel(const Layout L, void* block, unsigned units_a, unsigned units, unsigned narr)
{
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned u = blockIdx.x * blockDim.x + threadIdx.x; u < units; u += stride)
        halo_unit_block(L, static_cast<helem_t*>(block), units_a, u, narr);
}

// One member of a batched ghost fill (whole m-box of every field).
struct HaloMember {
    Layout L;
    state_t* block;
    long long unit_begin; // first global work unit of this member
    unsigned units_a;     // its kind-A units
};

// Members whose first work units a fill block keeps in shared memory.
constexpr int ACB_HALO_SEARCH = 1024;

// Ghost fill of every field of many meshes in one launch; threads take the
// concatenated work units of all members. A unit's member is found by binary
// search over the members' first units, held in shared memory (the first
// ACB_HALO_SEARCH members; any further ones are read from the table), so the
// search costs shared loads instead of a chain of dependent global ones.
static __global__ void __launch_bounds__(256)
halo_batch_kernel(const HaloMember* __restrict__ mem, int n, long long total_units)
{
    __shared__ long long first[ACB_HALO_SEARCH];
    const int ns = n < ACB_HALO_SEARCH ? n : ACB_HALO_SEARCH;
    for (int i = threadIdx.x; i < ns; i += blockDim.x)
        first[i] = mem[i].unit_begin;
    __syncthreads();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < total_units;
         u += stride) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if ((mid < ns ? first[mid] : mem[mid].unit_begin) <= u)
                lo = mid;
            else
                hi = mid - 1;
        }
        const HaloMember& m = mem[lo];
        halo_unit(m.L, m.block, m.units_a, (unsigned)(u - m.unit_begin));
    }
}

// ---------------------------------------------------------------------------
// Symmetric / antisymmetric ghost fill (reference src/core/kernels/
// boundconds.cuh:3-128 as intended): every ghost vertex takes sign times the
// vertex mirrored about the first or last interior point on each axis where
// it lies outside the interior, c' = 2 * 3 - c below and 2 * (n + 2) - c
// above (vertex-centred walls), the sign applied once (+1 symmetric, -1
// antisymmetric). The reference kernel writes sign * src * 0 + 1 instead
// (:127) and compares y against the x bound (:62, :93); both are corrected.
// With n >= 4 on every axis every source is an interior vertex, so all
// writes are independent.
__device__ __forceinline__ int
mirror_interior(int c, int n)
{
    return c < NGHOST ? 2 * NGHOST - c : (c > n + NGHOST - 1 ? 2 * (n + NGHOST - 1) - c : c);
}

static __global__ void __launch_bounds__(256)
mirror_kernel(const HaloArgs a, const float sign)
{
    const int lane         = threadIdx.x & 31;
    const long long warp   = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const Layout& L        = a.L;
    const int ry           = a.end.y - a.start.y;
    for (long long r = warp; r < a.rows; r += nwarps) {
        const int j          = a.start.y + (int)(r % ry);
        const int k          = a.start.z + (int)(r / ry);
        const bool ghost_row = j < NGHOST || j >= NGHOST + L.ny || k < NGHOST || k >= NGHOST + L.nz;
        const long long drow = lidx(L, 0, j, k);
        const long long srow = lidx(L, 0, mirror_interior(j, L.ny), mirror_interior(k, L.nz));
        for (int i = a.start.x + lane; i < a.end.x; i += 32) {
            if (!ghost_row && i >= NGHOST && i < NGHOST + L.nx)
                continue; // interior vertex
            const int is = mirror_interior(i, L.nx);
            constexpr int W = ACB_LANES;
            for (int f = a.f0; f < a.f1; ++f) {
                state_t* F        = a.block + fidx(L, f, 0);
                F[(drow + i) * W] = (state_t)sign * F[(srow + is) * W];
                if (ACB_MIXED && a.lo) {
                    // a bf16 value times -1 is its sign bit flipped
                    lo16_t* G = lo_field(a.lo, L, f);
                    const lo16_t v = G[(srow + is) * ACB_LO_STEP];
                    G[(drow + i) * ACB_LO_STEP] = sign < 0 ? (lo16_t)(v ^ 0x8000u) : v;
                }
            }
        }
    }
}

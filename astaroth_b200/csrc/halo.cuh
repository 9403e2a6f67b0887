// Periodic ghost-zone fill, all requested fields in one launch.
//
// Reference behaviour (src/core/kernels/boundconds.cuh:131-190): every ghost
// vertex (i, j, k) of the box [start, end) takes the value of the interior
// vertex ((c - 3 + n) mod n) + 3 on each axis. Every source is an interior
// vertex, so all ghost vertices can be written concurrently.
//
// The reference launches one thread per vertex of the whole m^3 box per field
// (8 launches per call) and returns early for the 96.5% interior threads. Here
// one warp owns one (j, k) row of the box and loops over the fields:
//   - a row whose j or k lies in the ghost zone is copied whole, lane-strided
//     (coalesced) from its wrapped source row;
//   - an interior row only has its 3 + 3 x-ghosts, filled by six lanes.
#pragma once
#include "common.cuh"

struct HaloArgs {
    Layout L;
    state_t* block; // field block (in)
    float* lo;      // mixed build: lo block of `in` (else null)
    int3 start, end;
    int f0, f1; // fields [f0, f1)
    long long rows;
};

__device__ __forceinline__ int
wrap_interior(int c, int n)
{
    return ((c - NGHOST + n) % n) + NGHOST;
}

__global__ void __launch_bounds__(256)
halo_kernel(const HaloArgs a)
{
    const Layout& L  = a.L;
    const int lane   = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int ry = a.end.y - a.start.y;
    for (long long r = warp; r < a.rows; r += nwarps) {
        const int j = a.start.y + (int)(r % ry);
        const int k = a.start.z + (int)(r / ry);
        const bool ghost_row = j < NGHOST || j >= NGHOST + L.ny || k < NGHOST || k >= NGHOST + L.nz;
        const int js = wrap_interior(j, L.ny);
        const int ks = wrap_interior(k, L.nz);
        const long long drow = lidx(L, 0, j, k);
        const long long srow = lidx(L, 0, js, ks);
        if (ghost_row) {
            for (int f = a.f0; f < a.f1; ++f) {
                state_t* F = a.block + f * L.fstride;
                for (int i = a.start.x + lane; i < a.end.x; i += 32)
                    F[drow + i] = F[srow + wrap_interior(i, L.nx)];
                if (ACB_MIXED && a.lo) {
                    float* G = a.lo + f * L.fstride;
                    for (int i = a.start.x + lane; i < a.end.x; i += 32)
                        G[drow + i] = G[srow + wrap_interior(i, L.nx)];
                }
            }
        }
        else if (lane < 2 * NGHOST) {
            const int i = lane < NGHOST ? lane : L.nx + lane; // 0,1,2 and nx+3..nx+5
            if (i >= a.start.x && i < a.end.x) {
                const int is = wrap_interior(i, L.nx);
                for (int f = a.f0; f < a.f1; ++f) {
                    state_t* F = a.block + f * L.fstride;
                    F[drow + i] = F[srow + is];
                    if (ACB_MIXED && a.lo) {
                        float* G = a.lo + f * L.fstride;
                        G[drow + i] = G[srow + is];
                    }
                }
            }
        }
    }
}

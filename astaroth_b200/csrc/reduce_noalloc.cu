// acReduceScalNoAlloc: a scalar reduction over a caller-owned device field
// that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc -- a host application or
// framework that owns every byte of device memory through its own pool (so a
// library allocation would bypass its accounting, or fail under a hard memory
// cap), or a time-critical loop that must not pay the implicit device-wide
// synchronisation cudaMalloc/cudaFree can cause. The Device interface
// (acDeviceReduceScal) allocates its scratch in acDeviceCreate; this entry
// point instead keeps its scratch in a fixed array of this library.
//
// Scratch: one FP64 partial per CTA and a finishing counter, in the
// file-scope arrays below (kNoAllocMaxPartials doubles = 128 KiB plus one
// counter). Every GPU that loads the library holds them until the process
// exits. A CTA covers 64 rows (j, k) of the interior, so the largest accepted
// mesh has ny * nz <= kNoAllocMaxPartials * 64 = 1,048,576 (e.g. 1024^3);
// larger meshes are rejected with an error message and AC_FAILURE.
//
// The arrays are shared by every call: calls whose kernels overlap on the GPU
// (different streams, or different host threads, without ordering) race on
// them and give wrong results. The counter must start at zero, so each call
// clears it on its stream before the kernel; the partials are always written
// before they are read.
//
// Set-up: host code cannot use the arrays' names as device addresses (on the
// host the name is only a stand-in). On its first call on a device, the entry
// point asks the runtime for the device address of each array with
// cudaGetSymbolAddress, with that device current, and caches it per device.
// That first call should therefore come before any stream capture. The cache
// lives as long as the process: after cudaDeviceReset (or the destruction of
// the device's primary context) the library's module is loaded anew at other
// addresses, and the cached ones would point into freed memory, so resetting a
// device between calls is not supported.
#include <math.h>
#include <stdio.h>

#include <mutex>

#include "astaroth.h"
#include "astaroth_b200.h"

namespace {

constexpr int kNoAllocMaxPartials = 16384;
constexpr int kRowsPerBlock       = 64; // 8 warps x 8 rows
constexpr int kThreads            = 256;
constexpr int kMaxDevices         = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxPartials];
static __device__ __align__(256) unsigned g_noalloc_counter[1];

struct NoAllocScratch {
    double* partials;
    unsigned* counter;
    bool ready;
};
NoAllocScratch g_scratch[kMaxDevices];
std::mutex g_scratch_mutex;

__device__ __forceinline__ double
na_combine(int rtype, double a, double b)
{
    if (rtype == RTYPE_MAX)
        return fmax(a, b);
    if (rtype == RTYPE_MIN)
        return fmin(a, b);
    return a + b;
}

__device__ __forceinline__ double
na_identity(int rtype)
{
    return rtype == RTYPE_MAX ? -INFINITY : (rtype == RTYPE_MIN ? INFINITY : 0.0);
}

// Field in the reference's flat layout: idx = i + j*mx + k*mx*my, interior
// [3, 3+n) on each axis.
__global__ void __launch_bounds__(kThreads)
noalloc_reduce_kernel(const AcReal* __restrict__ field, int nx, int ny, int nz, int rtype,
                      double* __restrict__ partials, unsigned* __restrict__ counter,
                      double* __restrict__ result)
{
    const int mx = nx + 2 * NGHOST, my = ny + 2 * NGHOST;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long rows = (long long)ny * nz;
    double acc = na_identity(rtype);
    for (int q = 0; q < kRowsPerBlock / (kThreads / 32); ++q) {
        const long long r = (long long)blockIdx.x * kRowsPerBlock + q * (kThreads / 32) + wid;
        if (r >= rows)
            break;
        const int j = NGHOST + (int)(r % ny), k = NGHOST + (int)(r / ny);
        const AcReal* row = field + (size_t)j * mx + (size_t)k * mx * my + NGHOST;
        for (int i = lane; i < nx; i += 32) {
            const double v = (double)row[i];
            double f       = v;
            if (rtype == RTYPE_RMS)
                f = v * v;
            else if (rtype == RTYPE_RMS_EXP) {
                const double e = exp(v);
                f              = e * e;
            }
            acc = na_combine(rtype, acc, f);
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        acc = na_combine(rtype, acc, __shfl_xor_sync(0xffffffffu, acc, o));
    __shared__ double wsum[kThreads / 32];
    __shared__ bool last;
    if (lane == 0)
        wsum[wid] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wsum[0];
        for (int w = 1; w < kThreads / 32; ++w)
            b = na_combine(rtype, b, wsum[w]);
        partials[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double v = na_identity(rtype);
        for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads)
            v = na_combine(rtype, v, ((volatile double*)partials)[b]);
        for (int o = 16; o > 0; o >>= 1)
            v = na_combine(rtype, v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0)
            wsum[wid] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = wsum[0];
            for (int w = 1; w < kThreads / 32; ++w)
                b = na_combine(rtype, b, wsum[w]);
            *result = b;
        }
    }
}

// Device addresses of the scratch arrays for the current device; looked up
// once per device (with that device current) and cached.
bool
scratch_for_current_device(NoAllocScratch* out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        fprintf(stderr, "acReduceScalNoAlloc: no usable current device\n");
        return false;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    NoAllocScratch& s = g_scratch[dev];
    if (!s.ready) {
        cudaError_t e1 = cudaGetSymbolAddress((void**)&s.partials, g_noalloc_partials);
        cudaError_t e2 = cudaGetSymbolAddress((void**)&s.counter, g_noalloc_counter);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            fprintf(stderr, "acReduceScalNoAlloc: cudaGetSymbolAddress failed: %s\n",
                    cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            s.partials = nullptr;
            s.counter  = nullptr;
            return false;
        }
        s.ready = true;
    }
    *out = s;
    return true;
}

} // namespace

extern "C" AcResult
acReduceScalNoAlloc(void* cuda_stream, const ReductionType rtype, const AcReal* field,
                    const int nx, const int ny, const int nz, double* result)
{
    if (!(rtype == RTYPE_MAX || rtype == RTYPE_MIN || rtype == RTYPE_RMS ||
          rtype == RTYPE_RMS_EXP || rtype == RTYPE_SUM)) {
        fprintf(stderr, "acReduceScalNoAlloc: unsupported reduction type %d\n", (int)rtype);
        return AC_FAILURE;
    }
    if (!field || !result || nx < 1 || ny < 1 || nz < 1) {
        fprintf(stderr, "acReduceScalNoAlloc: invalid field, result or sizes\n");
        return AC_FAILURE;
    }
    const long long rows   = (long long)ny * nz;
    const long long blocks = (rows + kRowsPerBlock - 1) / kRowsPerBlock;
    if (blocks > kNoAllocMaxPartials) {
        fprintf(stderr,
                "acReduceScalNoAlloc: mesh %d x %d x %d needs %lld partials; the fixed scratch "
                "holds %d (ny * nz must be <= %d)\n",
                nx, ny, nz, blocks, kNoAllocMaxPartials, kNoAllocMaxPartials * kRowsPerBlock);
        return AC_FAILURE;
    }
    NoAllocScratch s;
    if (!scratch_for_current_device(&s))
        return AC_FAILURE;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (cudaMemsetAsync(s.counter, 0, sizeof(unsigned), st) != cudaSuccess) {
        fprintf(stderr, "acReduceScalNoAlloc: clearing the counter failed\n");
        return AC_FAILURE;
    }
    noalloc_reduce_kernel<<<(unsigned)blocks, kThreads, 0, st>>>(field, nx, ny, nz, (int)rtype,
                                                                  s.partials, s.counter, result);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        fprintf(stderr, "acReduceScalNoAlloc: launch failed: %s\n", cudaGetErrorString(err));
        return AC_FAILURE;
    }
    return AC_SUCCESS;
}

// Single-pass reductions over the interior: MAX, MIN, RMS (raw sum of
// squares), RMS_EXP (raw sum of exp^2), SUM, for one field, a vector of three
// fields (by length), or the Alfven speed of three fields plus a density.
//
// Reference behaviour (src/core/kernels/reductions.cuh:18-343, device layer
// src/core/device.cc:477-537): filter functions
//     scalar  v, v^2, exp(v)^2
//     vector  |v|, |v|^2, sum_i exp(v_i)^2         (SUM of a vector sums |v|)
//     Alfven  |B| / sqrt(4 pi exp(rho)),  |B|^2 / (4 pi exp(rho))
// over [n_min, n_max); the device layer returns the unnormalised sum for RMS
// and RMS_EXP.
//
// The reference runs a filter kernel into an n^3 scratch array, a 128-wide
// shared-memory tree, then a single thread folding n^3/128 partials serially,
// all accumulating in AcReal. Here: one kernel, one read of each input; per
// thread FP64 accumulation over warp-owned rows, a warp-shuffle tree, a block
// tree, one FP64 partial per block in scratch, and the last block to finish
// folds the partials in a fixed order (deterministic, no atomics on data).
#pragma once
#include "common.cuh"

enum { RED_SCAL = 1, RED_VEC = 3, RED_ALFVEN = 4 };

// sets of one multi-set pass at most: a vector and six scalar fields
constexpr int ACB_RED_SETS = 7;
// entries a Device keeps of the passes on its current block (all eight fields
// and a vector, with room to spare)
constexpr int ACB_RED_RECORD = 16;

struct ReduceArgs {
    Layout L;
    const state_t* f[6];
    const lo16_t* lo[6]; // mixed build: lo parts, lo_field views (else null)
    int nin;            // 1, 3 or 4
    int rtype;          // ReductionType
    int3 start, end;
    long long rows;
    double* partials;   // gridDim.x doubles of scratch
    unsigned* counter;  // scratch counter, zero between launches
    double* result;
};

__device__ __forceinline__ double
red_combine(int rtype, double a, double b)
{
    if (rtype == RTYPE_MAX || rtype == RTYPE_ALFVEN_MAX)
        return fmax(a, b);
    if (rtype == RTYPE_MIN || rtype == RTYPE_ALFVEN_MIN)
        return fmin(a, b);
    return a + b;
}

__device__ __forceinline__ double
red_identity(int rtype)
{
    if (rtype == RTYPE_MAX || rtype == RTYPE_ALFVEN_MAX)
        return -INFINITY;
    if (rtype == RTYPE_MIN || rtype == RTYPE_ALFVEN_MIN)
        return INFINITY;
    return 0.0;
}

__device__ __forceinline__ double
red_load(const ReduceArgs& a, int w, long long id)
{
    // a.f[w] is the field's base in the block: its vertex id is ACB_LANES
    // values further per element
    double v = (double)a.f[w][id * ACB_LANES];
#if ACB_MIXED
    v += (double)lo16_to_float(a.lo[w][id * ACB_LO_STEP]);
#endif
    return v;
}

// |v|^2 of a vector, with one fixed rounding sequence for every reduction
// that uses it (the length for MAX / MIN, the square for RMS), so that a pass
// computing several of them returns what separate passes return, bit for bit.
__device__ __forceinline__ double
red_len2(double x, double y, double z)
{
    return __fma_rn(z, z, __fma_rn(y, y, __dmul_rn(x, x)));
}

__device__ __forceinline__ double
red_filter(const ReduceArgs& a, long long id)
{
    const int rt = a.rtype;
    if (a.nin == RED_SCAL) {
        const double v = red_load(a, 0, id);
        if (rt == RTYPE_RMS)
            return __dmul_rn(v, v);
        if (rt == RTYPE_RMS_EXP) {
            const double e = exp(v);
            return e * e;
        }
        return v; // MAX, MIN, SUM
    }
    const double x = red_load(a, 0, id), y = red_load(a, 1, id), z = red_load(a, 2, id);
    if (a.nin == RED_VEC) {
        if (rt == RTYPE_RMS)
            return red_len2(x, y, z);
        if (rt == RTYPE_RMS_EXP) {
            const double ex = exp(x), ey = exp(y), ez = exp(z);
            return ex * ex + ey * ey + ez * ez;
        }
        return sqrt(red_len2(x, y, z)); // MAX, MIN, SUM of the length
    }
    // Alfven speed with density exponent d
    const double d  = red_load(a, 3, id);
    const double b2 = x * x + y * y + z * z;
    const double q  = 4.0 * M_PI * exp(d);
    if (rt == RTYPE_ALFVEN_RMS)
        return b2 / q;
    return sqrt(b2) / sqrt(q);
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS)
reduce_kernel(const ReduceArgs a)
{
    const Layout& L = a.L;
    const int lane  = threadIdx.x & 31;
    const int wid   = threadIdx.x >> 5;
    const long long gw  = ((long long)blockIdx.x * THREADS + threadIdx.x) >> 5;
    const long long nw  = ((long long)gridDim.x * THREADS) >> 5;
    const int rx        = a.end.x - a.start.x;
    const int ry        = a.end.y - a.start.y;
    double acc          = red_identity(a.rtype);
    for (long long r = gw; r < a.rows; r += nw) {
        const int j          = a.start.y + (int)(r % ry);
        const int k          = a.start.z + (int)(r / ry);
        const long long base = lidx(L, a.start.x, j, k);
        for (int i = lane; i < rx; i += 32)
            acc = red_combine(a.rtype, acc, red_filter(a, base + i));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        acc = red_combine(a.rtype, acc, __shfl_xor_sync(0xffffffffu, acc, o));
    __shared__ double wsum[THREADS / 32];
    __shared__ bool last;
    if (lane == 0)
        wsum[wid] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wsum[0];
        for (int w = 1; w < THREADS / 32; ++w)
            b = red_combine(a.rtype, b, wsum[w]);
        a.partials[blockIdx.x] = b;
        __threadfence();
        const unsigned done = atomicAdd(a.counter, 1u);
        last                = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        // fixed-order fold of the partials: lanes stride, then a fixed tree
        __threadfence();
        double v = red_identity(a.rtype);
        for (int b = threadIdx.x; b < (int)gridDim.x; b += THREADS)
            v = red_combine(a.rtype, v, ((volatile double*)a.partials)[b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v = red_combine(a.rtype, v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0)
            wsum[wid] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = wsum[0];
            for (int w = 1; w < THREADS / 32; ++w)
                b = red_combine(a.rtype, b, wsum[w]);
            *a.result  = b;
            *a.counter = 0u; // ready for the next launch on this stream
        }
    }
}

// MAX, MIN and the RMS sum of one scalar field or one vector's length in a
// single pass (a.rtype unused): three accumulators, each combined in exactly
// the order reduce_kernel combines its one, so result[0..2] equal the MAX,
// MIN and RMS passes' results bit for bit. partials holds 3 * gridDim.x.
template <int THREADS>
__global__ void __launch_bounds__(THREADS)
reduce3_kernel(const ReduceArgs a)
{
    const Layout& L = a.L;
    const int lane  = threadIdx.x & 31;
    const int wid   = threadIdx.x >> 5;
    const long long gw  = ((long long)blockIdx.x * THREADS + threadIdx.x) >> 5;
    const long long nw  = ((long long)gridDim.x * THREADS) >> 5;
    const int rx        = a.end.x - a.start.x;
    const int ry        = a.end.y - a.start.y;
    double mx = -INFINITY, mn = INFINITY, sm = 0.0;
    for (long long r = gw; r < a.rows; r += nw) {
        const int j          = a.start.y + (int)(r % ry);
        const int k          = a.start.z + (int)(r / ry);
        const long long base = lidx(L, a.start.x, j, k);
        for (int i = lane; i < rx; i += 32) {
            const long long id = base + i;
            double m, q;
            if (a.nin == RED_SCAL) {
                m = red_load(a, 0, id);
                q = __dmul_rn(m, m);
            }
            else {
                q = red_len2(red_load(a, 0, id), red_load(a, 1, id), red_load(a, 2, id));
                m = sqrt(q);
            }
            mx = fmax(mx, m);
            mn = fmin(mn, m);
            sm = sm + q;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        sm = sm + __shfl_xor_sync(0xffffffffu, sm, o);
    }
    __shared__ double wmx[THREADS / 32], wmn[THREADS / 32], wsm[THREADS / 32];
    __shared__ bool last;
    if (lane == 0) {
        wmx[wid] = mx;
        wmn[wid] = mn;
        wsm[wid] = sm;
    }
    __syncthreads();
    const unsigned G = gridDim.x;
    if (threadIdx.x == 0) {
        double bx = wmx[0], bn = wmn[0], bs = wsm[0];
        for (int w = 1; w < THREADS / 32; ++w) {
            bx = fmax(bx, wmx[w]);
            bn = fmin(bn, wmn[w]);
            bs = bs + wsm[w];
        }
        a.partials[blockIdx.x]         = bx;
        a.partials[G + blockIdx.x]     = bn;
        a.partials[2 * G + blockIdx.x] = bs;
        __threadfence();
        const unsigned done = atomicAdd(a.counter, 1u);
        last                = (done == G - 1);
    }
    __syncthreads();
    if (last) {
        // the fixed-order fold of reduce_kernel, for each accumulator
        __threadfence();
        const volatile double* P = a.partials;
        double vx = -INFINITY, vn = INFINITY, vs = 0.0;
        for (int b = threadIdx.x; b < (int)G; b += THREADS) {
            vx = fmax(vx, P[b]);
            vn = fmin(vn, P[G + b]);
            vs = vs + P[2 * G + b];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            vx = fmax(vx, __shfl_xor_sync(0xffffffffu, vx, o));
            vn = fmin(vn, __shfl_xor_sync(0xffffffffu, vn, o));
            vs = vs + __shfl_xor_sync(0xffffffffu, vs, o);
        }
        if (lane == 0) {
            wmx[wid] = vx;
            wmn[wid] = vn;
            wsm[wid] = vs;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bx = wmx[0], bn = wmn[0], bs = wsm[0];
            for (int w = 1; w < THREADS / 32; ++w) {
                bx = fmax(bx, wmx[w]);
                bn = fmin(bn, wmn[w]);
                bs = bs + wsm[w];
            }
            a.result[0] = bx;
            a.result[1] = bn;
            a.result[2] = bs;
            *a.counter  = 0u; // ready for the next launch on this stream
        }
    }
}

// MAX, MIN and the RMS sum of several sets in one pass: set 0 is one scalar
// field (NIN = RED_SCAL, input 0) or one vector's length (NIN = RED_VEC, inputs
// 0-2); sets 1 .. NS-1 are the scalar fields of the inputs that follow
// (input s for a scalar request, s - 1 for a vector one): the vector's
// components and, in the single-precision builds, the fields that share their
// 8-byte elements, whose bytes the pass reads anyway. Every set's accumulators
// are combined in exactly the order reduce3_kernel combines its three, so each
// set's results equal a reduce3_kernel pass over it, bit for bit. partials
// holds 3 * NS * gridDim.x doubles, result 3 * NS (set s at 3 s).
template <int THREADS, int NIN, int NS>
__global__ void __launch_bounds__(THREADS)
reduce_sets_kernel(const ReduceArgs a)
{
    constexpr int NF = NIN == RED_SCAL ? NS : (NS - 1 > 3 ? NS - 1 : 3); // inputs
    static_assert(NF <= 6, "at most six inputs");
    const Layout& L = a.L;
    const int lane  = threadIdx.x & 31;
    const int wid   = threadIdx.x >> 5;
    const long long gw  = ((long long)blockIdx.x * THREADS + threadIdx.x) >> 5;
    const long long nw  = ((long long)gridDim.x * THREADS) >> 5;
    const int rx        = a.end.x - a.start.x;
    const int ry        = a.end.y - a.start.y;
    double mx[NS], mn[NS], sm[NS];
#pragma unroll
    for (int t = 0; t < NS; ++t) {
        mx[t] = -INFINITY;
        mn[t] = INFINITY;
        sm[t] = 0.0;
    }
    for (long long r = gw; r < a.rows; r += nw) {
        const int j          = a.start.y + (int)(r % ry);
        const int k          = a.start.z + (int)(r / ry);
        const long long base = lidx(L, a.start.x, j, k);
        for (int i = lane; i < rx; i += 32) {
            const long long id = base + i;
            double v[NF];
#pragma unroll
            for (int w = 0; w < NF; ++w)
                v[w] = red_load(a, w, id);
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                double m, q;
                if (t == 0 && NIN == RED_VEC) {
                    q = red_len2(v[0], v[1], v[2]);
                    m = sqrt(q);
                }
                else {
                    m = v[NIN == RED_SCAL ? t : t - 1];
                    q = __dmul_rn(m, m);
                }
                mx[t] = fmax(mx[t], m);
                mn[t] = fmin(mn[t], m);
                sm[t] = sm[t] + q;
            }
        }
    }
#pragma unroll
    for (int t = 0; t < NS; ++t)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mx[t] = fmax(mx[t], __shfl_xor_sync(0xffffffffu, mx[t], o));
            mn[t] = fmin(mn[t], __shfl_xor_sync(0xffffffffu, mn[t], o));
            sm[t] = sm[t] + __shfl_xor_sync(0xffffffffu, sm[t], o);
        }
    __shared__ double wmx[NS][THREADS / 32], wmn[NS][THREADS / 32], wsm[NS][THREADS / 32];
    __shared__ bool last;
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < NS; ++t) {
            wmx[t][wid] = mx[t];
            wmn[t][wid] = mn[t];
            wsm[t][wid] = sm[t];
        }
    __syncthreads();
    const unsigned G = gridDim.x;
    if (threadIdx.x == 0) {
        for (int t = 0; t < NS; ++t) {
            double bx = wmx[t][0], bn = wmn[t][0], bs = wsm[t][0];
            for (int w = 1; w < THREADS / 32; ++w) {
                bx = fmax(bx, wmx[t][w]);
                bn = fmin(bn, wmn[t][w]);
                bs = bs + wsm[t][w];
            }
            a.partials[(3 * t) * G + blockIdx.x]     = bx;
            a.partials[(3 * t + 1) * G + blockIdx.x] = bn;
            a.partials[(3 * t + 2) * G + blockIdx.x] = bs;
        }
        __threadfence();
        const unsigned done = atomicAdd(a.counter, 1u);
        last                = (done == G - 1);
    }
    __syncthreads();
    if (last) {
        // the fixed-order fold of reduce_kernel, for each accumulator
        __threadfence();
        const volatile double* P = a.partials;
        for (int t = 0; t < NS; ++t) {
            double vx = -INFINITY, vn = INFINITY, vs = 0.0;
            for (int b = threadIdx.x; b < (int)G; b += THREADS) {
                vx = fmax(vx, P[(3 * t) * G + b]);
                vn = fmin(vn, P[(3 * t + 1) * G + b]);
                vs = vs + P[(3 * t + 2) * G + b];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                vx = fmax(vx, __shfl_xor_sync(0xffffffffu, vx, o));
                vn = fmin(vn, __shfl_xor_sync(0xffffffffu, vn, o));
                vs = vs + __shfl_xor_sync(0xffffffffu, vs, o);
            }
            if (lane == 0) {
                wmx[t][wid] = vx;
                wmn[t][wid] = vn;
                wsm[t][wid] = vs;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int t = 0; t < NS; ++t) {
                double bx = wmx[t][0], bn = wmn[t][0], bs = wsm[t][0];
                for (int w = 1; w < THREADS / 32; ++w) {
                    bx = fmax(bx, wmx[t][w]);
                    bn = fmin(bn, wmn[t][w]);
                    bs = bs + wsm[t][w];
                }
                a.result[3 * t]     = bx;
                a.result[3 * t + 1] = bn;
                a.result[3 * t + 2] = bs;
            }
            *a.counter = 0u; // ready for the next launch on this stream
        }
    }
}

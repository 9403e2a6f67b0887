// Fused RK3 substep of the MHD module: 6th-order stencils of the eight input
// fields, the continuity / momentum / induction / entropy right-hand sides and
// the Williamson 2N update, in one pass.
//
// Reference behaviour being reproduced:
//   kernel body            acc/mhd_solver/stencil_kernel.ac:693-734
//   stencils               acc/stdlib/stdderiv.h:13-262
//   RHS                    acc/mhd_solver/stencil_kernel.ac:355-528
//   2N update, "previous   src/core/kernels/integration.cuh:14-52
//   state" form:  s = 0   : out = in + beta1 * dt * f
//                 s = 1, 2: out = in + beta_{s+1} (alpha_{s+1}/beta_s (in - out) + dt f)
//   forcing (s = 2 only)   acc/mhd_solver/stencil_kernel.ac:611-648,713-717
//
// B200 structure (no counterpart in the reference, which reads 55 stencil points
// per field straight from global memory with one thread per vertex):
//   - persistent CTAs: the (x-y tile, z-plane) work of the region is linearised
//     and split into equal contiguous ranges, one per CTA, so the grid is a
//     multiple of the SM count and the tail is at most one plane per CTA;
//   - each CTA streams its tile along z (2.5D): one TMA load per plane brings
//     all eight fields of a (TX+8) x (TY+6) halo'd tile into a ring of NP
//     plane slots in shared memory, NP - 7 planes ahead of the consumer;
//   - one thread per (x, y) column; every stencil operand, including the
//     z-neighbours and the xz/yz diagonals, is read from the ring;
//   - derivative coefficients arrive pre-scaled by 1/ds (and 1/ds^2) so each
//     pencil costs 6-7 FP ops; only the 21 first, 24 second and 12 cross
//     derivatives the right-hand sides use are formed;
//   - the mixed build keeps the state as an unevaluated float pair (hi, lo):
//     stencils read hi, the update is a compensated two-sum.
#pragma once
#include "common.cuh"
#include "tma.cuh"

template <typename T>
struct SolveParams {
    T c1[3][3];   // first derivative: axis, k-1; pre-scaled by 1/ds
    T c2[3][4];   // second derivative: axis, {centre, k=1..3}; pre-scaled by 1/ds^2
    T cx[3][3];   // diagonal cross derivative: pair {xy, xz, yz}, k-1; pre-scaled
    T nu, eta, inv_mu0, eta_mu0, zeta;
    T cs2_sound, inv_cp, gamma, gm1, gamma_inv_cp, lnrho0, lnT0, k_heat;
    T rkA, rkB; // out = cur + rkA * (cur - prev) + rkB * rate; rkA unused at s = 0
    // helical forcing, applied after the update at s = 2 when `forcing` != 0
    int forcing;
    T fk[3], ff_re[3], ff_im[3], fcphi, fsphi, fscale, fxs[3], fds[3];
};

struct SolveGeom {
    Layout L;
    int3 start, end; // region of interior vertices to update, [start, end)
    int tx0;         // index of the first x tile; x tiles are anchored at i = 3 + TX * t
                     // so that every TMA box starts on a 16-byte boundary
    int ntx, nty;    // tiles covering the region
    int nzr;         // planes of the region
    long long units; // ntx * nty * nzr
};

template <typename T>
struct SolveArgs {
    SolveGeom g;
    state_t* out;    // out block (previous state at s > 0; result)
    float* in_lo;    // mixed build: lo parts of `in`
    float* out_lo;   // mixed build: lo parts of `out`
    unsigned* status;
    SolveParams<T> P;
};

template <int TX_, int TY_, int NP_, int MINB_>
struct TileCfg {
    static constexpr int TX = TX_, TY = TY_, NP = NP_, MINB = MINB_;
    static constexpr int BX = TX_ + 8, BY = TY_ + 6;
    static constexpr int THREADS = TX_ * TY_;
    static constexpr int FIELD   = BX * BY;
    static constexpr int PLANE   = ACB_NF * FIELD; // elements per ring slot
    static constexpr size_t smem_bytes() { return (size_t)NP * PLANE * sizeof(state_t); }
};

namespace acb {

template <typename T>
__device__ __forceinline__ T
rexp(T x)
{
    return exp(x);
}
template <>
__device__ __forceinline__ float
rexp<float>(float x)
{
    return expf(x);
}

// first and second derivative from the six neighbours of a pencil
template <typename T>
__device__ __forceinline__ void
d12(T f0, T m1, T p1, T m2, T p2, T m3, T p3, const T* c1, const T* c2, T& d1, T& d2)
{
    d1 = c1[0] * (p1 - m1) + c1[1] * (p2 - m2) + c1[2] * (p3 - m3);
    d2 = c2[0] * f0 + c2[1] * (p1 + m1) + c2[2] * (p2 + m2) + c2[3] * (p3 + m3);
}

template <typename T>
__device__ __forceinline__ T
dd2(T f0, T m1, T p1, T m2, T p2, T m3, T p3, const T* c2)
{
    return c2[0] * f0 + c2[1] * (p1 + m1) + c2[2] * (p2 + m2) + c2[3] * (p3 + m3);
}

// all derivatives of one field at the thread's vertex, read from the ring
template <typename T>
struct FieldDerivs {
    T v;          // value
    T gx, gy, gz; // first derivatives
    T xx, yy, zz; // pure second derivatives
    T xy, xz, yz; // cross derivatives (only those requested are formed)
};

// c: pointer to the field's centre element in the centre slot;
// zo[0..6]: element offsets of the slots of planes z-3 .. z+3 from the centre slot.
template <typename T, int BX, bool GX, bool GY, bool GZ, bool XY, bool XZ, bool YZ>
__device__ __forceinline__ FieldDerivs<T>
field_derivs(const state_t* __restrict__ c, const int* zo, const SolveParams<T>& P)
{
    FieldDerivs<T> r;
    const T f0 = (T)c[0];
    r.v        = f0;
    // x pencil
    {
        const T m1 = c[-1], p1 = c[1], m2 = c[-2], p2 = c[2], m3 = c[-3], p3 = c[3];
        if (GX)
            d12(f0, m1, p1, m2, p2, m3, p3, P.c1[0], P.c2[0], r.gx, r.xx);
        else
            r.xx = dd2(f0, m1, p1, m2, p2, m3, p3, P.c2[0]);
    }
    // y pencil
    {
        const T m1 = c[-BX], p1 = c[BX], m2 = c[-2 * BX], p2 = c[2 * BX], m3 = c[-3 * BX],
                p3 = c[3 * BX];
        if (GY)
            d12(f0, m1, p1, m2, p2, m3, p3, P.c1[1], P.c2[1], r.gy, r.yy);
        else
            r.yy = dd2(f0, m1, p1, m2, p2, m3, p3, P.c2[1]);
    }
    // z pencil
    {
        const T m1 = c[zo[2]], p1 = c[zo[4]], m2 = c[zo[1]], p2 = c[zo[5]], m3 = c[zo[0]],
                p3 = c[zo[6]];
        if (GZ)
            d12(f0, m1, p1, m2, p2, m3, p3, P.c1[2], P.c2[2], r.gz, r.zz);
        else
            r.zz = dd2(f0, m1, p1, m2, p2, m3, p3, P.c2[2]);
    }
    // diagonal cross derivatives: sum_k e_k (f(+k,+k) + f(-k,-k) - f(+k,-k) - f(-k,+k))
    if (XY) {
        T s = 0;
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            const T a = (T)c[k + k * BX] + (T)c[-k - k * BX];
            const T b = (T)c[k - k * BX] + (T)c[-k + k * BX];
            s += P.cx[0][k - 1] * (a - b);
        }
        r.xy = s;
    }
    if (XZ) {
        T s = 0;
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            const T a = (T)c[zo[3 + k] + k] + (T)c[zo[3 - k] - k];
            const T b = (T)c[zo[3 - k] + k] + (T)c[zo[3 + k] - k];
            s += P.cx[1][k - 1] * (a - b);
        }
        r.xz = s;
    }
    if (YZ) {
        T s = 0;
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            const T a = (T)c[zo[3 + k] + k * BX] + (T)c[zo[3 - k] - k * BX];
            const T b = (T)c[zo[3 - k] + k * BX] + (T)c[zo[3 + k] - k * BX];
            s += P.cx[2][k - 1] * (a - b);
        }
        r.yz = s;
    }
    return r;
}

// Right-hand sides of the eight fields at one vertex (stencil_kernel.ac:355-528,
// restated; same terms, evaluated from the derivative set above).
template <typename T, int BX, int FIELD>
__device__ __forceinline__ void
mhd_rhs(const state_t* __restrict__ c, const int* zo, const SolveParams<T>& P, T roc[ACB_NF],
        T cur[ACB_NF])
{
    //                                       GX     GY     GZ     XY     XZ     YZ
    const auto lr = field_derivs<T, BX, true, true, true, false, false, false>(c + 0 * FIELD, zo, P);
    const auto ux = field_derivs<T, BX, true, true, true, true, true, false>(c + 1 * FIELD, zo, P);
    const auto uy = field_derivs<T, BX, true, true, true, true, false, true>(c + 2 * FIELD, zo, P);
    const auto uz = field_derivs<T, BX, true, true, true, false, true, true>(c + 3 * FIELD, zo, P);
    const auto ax = field_derivs<T, BX, false, true, true, true, true, false>(c + 4 * FIELD, zo, P);
    const auto ay = field_derivs<T, BX, true, false, true, true, false, true>(c + 5 * FIELD, zo, P);
    const auto az = field_derivs<T, BX, true, true, false, false, true, true>(c + 6 * FIELD, zo, P);
    const auto ss = field_derivs<T, BX, true, true, true, false, false, false>(c + 7 * FIELD, zo, P);

    cur[0] = lr.v;
    cur[1] = ux.v;
    cur[2] = uy.v;
    cur[3] = uz.v;
    cur[4] = ax.v;
    cur[5] = ay.v;
    cur[6] = az.v;
    cur[7] = ss.v;

    const T u0 = ux.v, u1 = uy.v, u2 = uz.v;
    const T divu = ux.gx + uy.gy + uz.gz;

    // continuity: -u.grad(lnrho) - div(u)
    roc[0] = -(u0 * lr.gx + u1 * lr.gy + u2 * lr.gz) - divu;

    // B = curl A
    const T B0 = az.gy - ay.gz;
    const T B1 = ax.gz - az.gx;
    const T B2 = ay.gx - ax.gy;
    const T lapA0 = ax.xx + ax.yy + ax.zz;
    const T lapA1 = ay.xx + ay.yy + ay.zz;
    const T lapA2 = az.xx + az.yy + az.zz;

    // induction: u x B + eta lap(A)
    roc[4] = (u1 * B2 - u2 * B1) + P.eta * lapA0;
    roc[5] = (u2 * B0 - u0 * B2) + P.eta * lapA1;
    roc[6] = (u0 * B1 - u1 * B0) + P.eta * lapA2;

    // j = (grad div A - lap A) / mu0
    const T j0 = P.inv_mu0 * ((ax.xx + ay.xy + az.xz) - lapA0);
    const T j1 = P.inv_mu0 * ((ax.xy + ay.yy + az.yz) - lapA1);
    const T j2 = P.inv_mu0 * ((ax.xz + ay.yz + az.zz) - lapA2);

    // traceless strain S
    const T third = (T)1 / (T)3, twothird = (T)2 / (T)3, half = (T)0.5;
    const T S00   = twothird * ux.gx - third * (uy.gy + uz.gz);
    const T S11   = twothird * uy.gy - third * (ux.gx + uz.gz);
    const T S22   = twothird * uz.gz - third * (ux.gx + uy.gy);
    const T S01   = half * (ux.gy + uy.gx);
    const T S02   = half * (ux.gz + uz.gx);
    const T S12   = half * (uy.gz + uz.gy);

    // thermodynamics: E = gamma s / cp + (gamma - 1)(lnrho - lnrho0)
    const T E       = P.gamma * ss.v * P.inv_cp + P.gm1 * (lr.v - P.lnrho0);
    const T expE    = rexp<T>(E);
    const T cs2     = P.cs2_sound * expE;
    const T rho     = rexp<T>(lr.v);
    const T inv_rho = (T)1 / rho;

    // momentum
    const T gd0 = ux.xx + uy.xy + uz.xz;
    const T gd1 = ux.xy + uy.yy + uz.yz;
    const T gd2 = ux.xz + uy.yz + uz.zz;
    const T jxB0 = j1 * B2 - j2 * B1;
    const T jxB1 = j2 * B0 - j0 * B2;
    const T jxB2 = j0 * B1 - j1 * B0;
    const T lapu0 = ux.xx + ux.yy + ux.zz;
    const T lapu1 = uy.xx + uy.yy + uy.zz;
    const T lapu2 = uz.xx + uz.yy + uz.zz;
    const T Sg0   = S00 * lr.gx + S01 * lr.gy + S02 * lr.gz;
    const T Sg1   = S01 * lr.gx + S11 * lr.gy + S12 * lr.gz;
    const T Sg2   = S02 * lr.gx + S12 * lr.gy + S22 * lr.gz;
    roc[1] = -(ux.gx * u0 + ux.gy * u1 + ux.gz * u2) - cs2 * (P.inv_cp * ss.gx + lr.gx) +
             inv_rho * jxB0 + P.nu * (lapu0 + third * gd0 + (T)2 * Sg0) + P.zeta * gd0;
    roc[2] = -(uy.gx * u0 + uy.gy * u1 + uy.gz * u2) - cs2 * (P.inv_cp * ss.gy + lr.gy) +
             inv_rho * jxB1 + P.nu * (lapu1 + third * gd1 + (T)2 * Sg1) + P.zeta * gd1;
    roc[3] = -(uz.gx * u0 + uz.gy * u1 + uz.gz * u2) - cs2 * (P.inv_cp * ss.gz + lr.gz) +
             inv_rho * jxB2 + P.nu * (lapu2 + third * gd2 + (T)2 * Sg2) + P.zeta * gd2;

    // entropy
    const T lnT    = P.lnT0 + E;
    const T inv_pT = (T)1 / (rho * rexp<T>(lnT));
    const T SS     = S00 * S00 + S01 * S01 + S02 * S02 + S01 * S01 + S11 * S11 + S12 * S12 +
                 S02 * S02 + S12 * S12 + S22 * S22;
    const T heat = P.eta_mu0 * (j0 * j0 + j1 * j1 + j2 * j2) + (T)2 * rho * P.nu * SS +
                   P.zeta * rho * divu * divu;
    const T lap_s  = ss.xx + ss.yy + ss.zz;
    const T lap_lr = lr.xx + lr.yy + lr.zz;
    const T first  = P.gamma_inv_cp * lap_s + P.gm1 * lap_lr;
    const T sec0 = P.gamma_inv_cp * ss.gx + P.gm1 * lr.gx;
    const T sec1 = P.gamma_inv_cp * ss.gy + P.gm1 * lr.gy;
    const T sec2 = P.gamma_inv_cp * ss.gz + P.gm1 * lr.gz;
    const T thi0 = P.gamma * (P.inv_cp * ss.gx + lr.gx) - lr.gx;
    const T thi1 = P.gamma * (P.inv_cp * ss.gy + lr.gy) - lr.gy;
    const T thi2 = P.gamma * (P.inv_cp * ss.gz + lr.gz) - lr.gz;
    // cp * chi with chi = K / (rho cp)
    const T hc = P.k_heat * inv_rho * (first + (sec0 * thi0 + sec1 * thi1 + sec2 * thi2));
    roc[7]     = -(u0 * ss.gx + u1 * ss.gy + u2 * ss.gz) + inv_pT * heat + hc;
}

// Helical forcing at interior vertex (i, j, k) (stencil_kernel.ac:611-648 with
// a single device: global index = local index, global grid = local grid).
template <typename T>
__device__ __forceinline__ void
forcing_at(const SolveParams<T>& P, int i, int j, int k, T f[3])
{
    const T x0 = (T)(i - NGHOST) * P.fds[0] * P.fxs[0];
    const T x1 = (T)(j - NGHOST) * P.fds[1] * P.fxs[1];
    const T x2 = (T)(k - NGHOST) * P.fds[2] * P.fxs[2];
    const T kx = P.fk[0] * x0 + P.fk[1] * x1 + P.fk[2] * x2;
    T skx, ckx;
    if constexpr (sizeof(T) == 4) {
        sincosf((float)kx, (float*)&skx, (float*)&ckx);
    }
    else {
        sincos((double)kx, (double*)&skx, (double*)&ckx);
    }
    const T re = ckx * P.fcphi - skx * P.fsphi;
    const T im = ckx * P.fsphi + skx * P.fcphi;
    bool ok    = true;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        f[c] = P.fscale * (P.ff_re[c] * re - P.ff_im[c] * im);
        ok   = ok && isfinite(f[c]);
    }
    if (!ok)
        f[0] = f[1] = f[2] = 0;
}

// Compensated sum of the float pair (hi, lo) and a float increment d.
__device__ __forceinline__ void
pair_add(float hi, float lo, float d, float& ohi, float& olo)
{
    const float s  = hi + d;
    const float bb = s - hi;
    const float e  = (hi - (s - bb)) + (d - bb); // two-sum error
    const float l  = lo + e;
    ohi            = s + l; // renormalise
    olo            = l - (ohi - s);
}

} // namespace acb

template <class Cfg, int STEP>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MINB)
    solve_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ SolveArgs<AcReal> a)
{
    using T = AcReal;
    constexpr int TX = Cfg::TX, TY = Cfg::TY, NP = Cfg::NP, BX = Cfg::BX;
    constexpr int FIELD = Cfg::FIELD, PLANE = Cfg::PLANE;
    constexpr uint32_t PLANE_BYTES = PLANE * sizeof(state_t);

    extern __shared__ __align__(128) unsigned char smem_raw[];
    state_t* ring = reinterpret_cast<state_t*>(smem_raw);
    __shared__ __align__(8) uint64_t bars[NP];
    __shared__ int abort_flag;

    const int tid = threadIdx.x;
    const int tx  = tid % TX;
    const int ty  = tid / TX;
    if (tid == 0) {
        for (int s = 0; s < NP; ++s)
            mbar_init(&bars[s], 1);
        fence_barrier_init();
        abort_flag = 0;
        prefetch_tensormap(&tin);
    }
    __syncthreads();

    const SolveGeom& g = a.g;
    const Layout& L    = g.L;
    const long long U  = g.units;
    const long long u0 = U * blockIdx.x / gridDim.x;
    const long long u1 = U * (blockIdx.x + 1) / gridDim.x;

    uint32_t q = 0; // planes this CTA has consumed the ring for so far
    long long u = u0;
    while (u < u1) {
        const long long tile = u / g.nzr;
        const int za         = (int)(u - tile * g.nzr);
        const int zb         = (int)min((long long)g.nzr, za + (u1 - u));
        u += zb - za;
        const int tile_x = (int)(tile % g.ntx);
        const int tile_y = (int)(tile / g.ntx);
        const int i0     = NGHOST + (g.tx0 + tile_x) * TX;
        const int j0     = g.start.y + tile_y * TY;
        const int k0     = g.start.z + za;
        const int nout   = zb - za;
        const int nload  = nout + 2 * NGHOST;
        const int xt     = L.offx + i0 - 4; // multiple of 16 bytes by construction
        const int yt     = j0 - NGHOST;

        int issued = 0;
        if (tid == 0) {
            const int first = nload < NP ? nload : NP;
            for (int l = 0; l < first; ++l) {
                const uint32_t s = (q + l) % NP;
                mbar_arrive_expect_tx(&bars[s], PLANE_BYTES);
                tma_load_4d(ring + (size_t)s * PLANE, &tin, xt, yt, k0 - NGHOST + l, 0, &bars[s]);
            }
            issued = first;
        }
        // the first output needs planes 0..6
        bool ok = true;
        for (int l = 0; l < 2 * NGHOST && ok; ++l)
            ok = mbar_wait_bounded(&bars[(q + l) % NP], ((q + l) / NP) & 1u);

        const int i    = i0 + tx;
        const int j    = j0 + ty;
        const bool act = (i >= g.start.x) && (i < g.end.x) && (j < g.end.y);

        for (int p = 0; p < nout; ++p) {
            if (ok) {
                const uint32_t l = p + 2 * NGHOST;
                ok               = mbar_wait_bounded(&bars[(q + l) % NP], ((q + l) / NP) & 1u);
            }
            if (!ok) {
                atomicOr(a.status, (unsigned)ACB_STATUS_TMA_TIMEOUT);
                abort_flag = 1;
            }
            if (ok && act) {
                const int k      = k0 + p;
                const uint32_t sc = (q + p + NGHOST) % NP;
                int zo[7];
#pragma unroll
                for (int dz = -NGHOST; dz <= NGHOST; ++dz) {
                    const int sd   = (int)((q + p + NGHOST + dz) % NP);
                    zo[dz + NGHOST] = (sd - (int)sc) * PLANE;
                }
                const state_t* c = ring + (size_t)sc * PLANE + (ty + NGHOST) * BX + (tx + 4);
                const long long id = lidx(L, i, j, k);

                T prev[ACB_NF];
                if (STEP > 0) {
#pragma unroll
                    for (int f = 0; f < ACB_NF; ++f)
                        prev[f] = a.out[f * L.fstride + id];
                }
#if ACB_MIXED
                float cur_lo[ACB_NF], prev_lo[ACB_NF];
#pragma unroll
                for (int f = 0; f < ACB_NF; ++f) {
                    cur_lo[f]  = a.in_lo[f * L.fstride + id];
                    prev_lo[f] = STEP > 0 ? a.out_lo[f * L.fstride + id] : 0.f;
                }
#endif
                T roc[ACB_NF], cur[ACB_NF];
                acb::mhd_rhs<T, BX, FIELD>(c, zo, a.P, roc, cur);

                T fo[3] = {0, 0, 0};
                if (STEP == 2 && a.P.forcing)
                    acb::forcing_at<T>(a.P, i, j, k, fo);

#pragma unroll
                for (int f = 0; f < ACB_NF; ++f) {
#if ACB_MIXED
                    float d = a.P.rkB * roc[f];
                    if (STEP > 0)
                        d += a.P.rkA * ((cur[f] - prev[f]) + (cur_lo[f] - prev_lo[f]));
                    float hi, lo;
                    acb::pair_add(cur[f], cur_lo[f], d, hi, lo);
                    if (STEP == 2 && f >= 1 && f <= 3)
                        acb::pair_add(hi, lo, fo[f - 1], hi, lo);
                    a.out[f * L.fstride + id]    = hi;
                    a.out_lo[f * L.fstride + id] = lo;
#else
                    T r;
                    if (STEP == 0)
                        r = cur[f] + a.P.rkB * roc[f];
                    else
                        r = cur[f] + a.P.rkA * (cur[f] - prev[f]) + a.P.rkB * roc[f];
                    if (STEP == 2 && f >= 1 && f <= 3)
                        r += fo[f - 1];
                    a.out[f * L.fstride + id] = r;
#endif
                }
            }
            __syncthreads(); // every thread is done with plane p: its slot may be refilled
            if (abort_flag)
                break;
            if (tid == 0 && issued < nload) {
                const uint32_t l = issued; // == p + NP
                const uint32_t s = (q + l) % NP;
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&bars[s], PLANE_BYTES);
                tma_load_4d(ring + (size_t)s * PLANE, &tin, xt, yt, k0 - NGHOST + l, 0, &bars[s]);
                ++issued;
            }
        }
        if (abort_flag) {
            // drain (bounded) whatever this CTA still has in flight, then leave
            if (tid == 0) {
                for (int l = issued > NP ? issued - NP : 0; l < issued; ++l)
                    (void)mbar_wait_bounded(&bars[(q + l) % NP], ((q + l) / NP) & 1u);
            }
            return;
        }
        q += nload;
    }
}

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
//                          (STEP 3 = substep 2 with forcing; STEP 2 leaves it out)
//
// B200 structure (no counterpart in the reference, which reads 55 stencil points
// per field straight from global memory with one thread per vertex):
//   - persistent CTAs (one per SM slot) take tasks = (x-y tile, z segment)
//     round-robin, segment-major, so the CTAs of one wave stream neighbouring
//     tiles at the same z and read each other's halo planes from L2;
//   - each CTA streams its tile along z (2.5D): a producer warp issues one TMA
//     load per plane bringing all eight fields of a (TX+8) x (TY+6) halo'd tile
//     into a ring of NP plane slots in shared memory (mbarrier `full` with
//     transaction bytes); consumer warps release a slot through an `empty`
//     mbarrier when done, so no block-wide barrier sits in the plane loop;
//   - single precision: the layout interleaves the fields in pairs with the
//     same stencils, (lnrho, ss), (ux, ax), (uy, ay), (uz, az), so a stencil
//     point of a pair is one 8-byte shared load and its arithmetic runs in
//     packed f32x2 lanes;
//   - one consumer thread per (x, y) column; in single precision each thread
//     keeps a register queue along z (its column's values of the three planes
//     below, and running sums of the lower halves of the xz / yz diagonals),
//     so the ring is read for the centre plane and the three above it only
//     (112 8-byte shared loads per vertex instead of 296 values) and a plane's
//     slot is released as soon as its own outputs are done; double precision
//     reads all seven planes from the ring; the centre-only values (previous
//     state, lo parts) arrive by TMA in a ring of output-plane slots (mixed
//     substeps 1 and 2) or by plain loads (a plane ahead in double precision);
//   - derivative coefficients arrive pre-scaled by 1/ds (and 1/ds^2) so each
//     pencil costs 6-7 FP ops; only the 21 first, 24 second and 12 cross
//     derivatives the right-hand sides use are formed;
//   - the mixed build keeps the state as an unevaluated sum hi + lo of a float
//     and a bfloat16 (stored as such, widened to float in registers): stencils
//     read hi, the update is a compensated two-sum.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "tma.cuh"

template <typename T>
struct SolveParams {
    T c1[3][3];   // first derivative: axis, k-1; pre-scaled by 1/ds
    T c2[3][4];   // second derivative: axis, {centre, k=1..3}; pre-scaled by 1/ds^2
    T cx[3][3];   // diagonal cross derivative: pair {xy, xz, yz}, k-1; pre-scaled
    // single precision: c1, c2 and cx as (c, c) pairs of FP32 lanes, the
    // coefficient operands of packed sums over the two fields of a pair
    unsigned long long c1p[3][3], c2p[3][4], cxp[3][3];
    T nu, eta, inv_mu0, eta_mu0, zeta;
    T cs2_sound, inv_cp, gamma, gm1, gamma_inv_cp, lnrho0, lnT0, k_heat;
    T exp_lnT0; // exp(lnT0): T = exp(lnT0 + E) = exp_lnT0 * exp(E)
    T rkA, rkB; // out = cur + rkA * (cur - prev) + rkB * rate; rkA unused at s = 0
    // helical forcing, applied after the update at s = 2 when `forcing` != 0
    int forcing;
    T fk[3], ff_re[3], ff_im[3], fcphi, fsphi, fscale, fxs[3], fds[3];
    // time step chosen on the device (acDeviceIntegrateStepCFL): the kernels
    // built with DTDEV take rkB = (T)(rk_beta * *dt_dev) instead of rkB above
    const double* dt_dev;
    double rk_beta;
    // 2 pi / (ds n) per axis in double precision: the single-precision builds
    // form the forcing phase in double (forcing_column, forcing_plane)
    double fxs_d[3];
};

struct SolveGeom {
    Layout L;
    int3 start, end; // region of interior vertices to update, [start, end)
    int tx0;         // index of the first x tile; x tiles are anchored at i = 3 + TX * t
                     // so that every TMA box starts on a 16-byte boundary
    int ntx, nty;    // tiles covering the region
    int nzr;         // planes of the region
    int zseg;        // planes per task (the region's z range is cut into nseg segments)
    int nseg;
    long long tasks; // ntx * nty * nseg; task t = (segment t / tiles, tile t % tiles)
};

// One member of an ensemble (many independent meshes advanced by one launch):
// the TMA map of its `in` block, its geometry and task range and its buffers.
// Kept in global memory, one table per buffer parity; its parameters travel
// with the launch (MemberParams below).
template <typename T>
struct __align__(128) MemberDesc {
    CUtensorMap tmap;
    SolveGeom g;
    long long task_begin; // first global task of this member (tasks are member-major)
    state_t* out;
    lo16_t* in_lo;
    lo16_t* out_lo;
};

template <typename T>
struct SolveArgs {
    SolveGeom g;
    state_t* out;    // out block (previous state at s > 0; result)
    lo16_t* in_lo;   // mixed build: lo block of `in` (bf16, see common.cuh)
    lo16_t* out_lo;  // mixed build: lo block of `out`
    unsigned* status;
    SolveParams<T> P;
    // step diagnostics (kernels built with DIAG): four FP64 partials per CTA,
    // a finishing counter (zero between launches; the last CTA resets it) and
    // the folded result {max |u|^2, min |u|^2, sum |u|^2, sum exp(lnrho)^2}
    double* diag_partials;
    unsigned* diag_counter;
    double* diag_result;
    // ensemble launches only
    const MemberDesc<T>* members;
    int nmembers;
    long long total_tasks;
};

// Parameters of one ensemble member as the stencils and right-hand sides read
// them, carried in the launch's parameter space (the constant bank, as a single
// mesh's SolveParams are) instead of being read from memory at every use.
template <typename T>
struct MemberParams;
template <>
struct MemberParams<float> {
    unsigned long long c1p[3][3], c2p[3][4], cxp[3][3]; // (c, c) coefficient pairs
    float nu, eta, inv_mu0, eta_mu0, zeta;
    float cs2_sound, inv_cp, gamma, gm1, gamma_inv_cp, lnrho0, lnT0, k_heat, exp_lnT0;
};
template <>
struct MemberParams<double> {
    double c1[3][3], c2[3][4], cx[3][3];
    double nu, eta, inv_mu0, eta_mu0, zeta;
    double cs2_sound, inv_cp, gamma, gm1, gamma_inv_cp, lnrho0, lnT0, k_heat, exp_lnT0;
};

// Members per ensemble launch (a launch's parameters stay within 32 KB; a
// larger ensemble takes one launch per group of members).
constexpr int ACB_ENS_GROUP = 64;

template <typename T>
struct EnsSolveArgs : SolveArgs<T> {
    long long task_base;                 // first task of the group (tasks of all groups
                                         // are numbered as one list, member-major)
    MemberParams<T> mp[ACB_ENS_GROUP];   // by position in the group
};

// Centre-only arrays of a substep that the ring does not carry: the previous
// state (s > 0) and, in the mixed build, the lo parts of `in` and (s > 0) of
// `out` (two lo arrays each, bf16). Map slots: 0 = out hi, 1 = in lo, 2 = out lo.
template <int STEP>
struct CentreSet {
    static constexpr bool PREV = STEP > 0;
    static constexpr bool LO   = ACB_MIXED != 0;
    static constexpr int N     = (PREV ? 1 : 0) + (LO ? (PREV ? 2 : 1) : 0);
    // staged by TMA in the single-precision builds' configurations with a
    // centre ring (the mixed build's): the three arrays of substeps 1 and 2
    // and the lo parts of substep 0, whose plain loads left its warps waiting
    // on memory (long-scoreboard stalls 1.66 per issued instruction at 256^3;
    // the 512^3 step 17.43 -> 17.22 ms, same-box A/B)
    static constexpr bool STAGE = N >= 1;
};

struct CentreMaps {
    CUtensorMap m[3]; // (TX, TY, 1, arrays) boxes over out hi, in lo, out lo
};

template <int TX_, int TY_, int NP_, int MINB_, int NC_ = 0>
struct TileCfg {
    static constexpr int TX = TX_, TY = TY_, NP = NP_, MINB = MINB_;
    // NC > 0: the centre-only values of single-mesh single-precision substeps
    // arrive by TMA in a ring of NC output-plane slots (else plain loads)
    static constexpr int NC = NC_;
    static constexpr int CENTRE = TX_ * TY_ * ACB_NARR; // elements of one centre array set
    static constexpr int CENTRE_LO = TX_ * TY_ * ACB_LO_NARR; // the same for a lo block
    static constexpr int BX = TX_ + 8, BY = TY_ + 6;
    static constexpr int CONSUMERS = TX_ * TY_;        // one thread per (x, y) column
    static constexpr int CWARPS    = CONSUMERS / 32;   // consumer warps
    // Single precision with 8 or 12 consumer warps: the producer is a whole
    // warpgroup (4 warps, one of them working) that hands its registers to the
    // consumers (setmaxnreg), so each consumer thread gets the registers its z
    // queues need. An SM sub-partition's 16K registers hold 2 consumer warps
    // and 1 producer warp (2 * 232 + 40 = 504 <= 512 registers a lane), or 3
    // and 1 (3 * 160 + 32 = 512): more warps to hide latency, fewer registers.
    static constexpr bool WGSPEC = sizeof(state_t) == 4 && (CWARPS == 8 || CWARPS == 12);
    static constexpr int THREADS = CONSUMERS + (WGSPEC ? 128 : 32); // plus the producer
    static constexpr int REG_CONSUMER = CWARPS == 12 ? 160 : 232;
    static constexpr int REG_PRODUCER = CWARPS == 12 ? 32 : 40;
    // registers a thread the launch must hold for the reallocation to balance
    static constexpr int REG_LAUNCH =
        WGSPEC ? (REG_CONSUMER * CONSUMERS + REG_PRODUCER * 128 + THREADS - 1) / THREADS : 0;
    static constexpr int FIELD   = BX * BY;           // elements per array of a ring slot
    static constexpr int PLANE   = ACB_NARR * FIELD;  // elements per ring slot
    static constexpr size_t ring_bytes() { return (size_t)NP * PLANE * ACB_ELEM; }
    // prev hi, then (mixed) cur lo and prev lo
    static constexpr size_t centre_slot_bytes()
    {
        return (size_t)(ACB_MIXED ? CENTRE + 2 * CENTRE_LO : CENTRE) * ACB_ELEM;
    }
    static constexpr size_t smem_bytes() { return ring_bytes() + NC * centre_slot_bytes(); }
    // A task starts once the first 2 NGHOST planes are in the ring (the queue
    // priming and the first output plane's upper half), and without queues an
    // output plane needs all 2 NGHOST + 1 of its planes at once: a shallower
    // ring could never hold them.
    static_assert(NP >= (sizeof(state_t) == 4 ? 2 * NGHOST : 2 * NGHOST + 1),
                  "ring too shallow for the planes a task waits for");
    static_assert(smem_bytes() <= 227 * 1024, "shared memory of one CTA exceeded");
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

// 1 / x: correctly rounded in double precision; in single precision the fast
// division (within 2 ulp of the IEEE quotient for the arguments here, 1/rho and
// 1/(rho T) of order one), 4 % of a step cheaper than the correctly rounded
// reciprocal, whose special-case path it avoids
template <typename T>
__device__ __forceinline__ T
rrcp(T x)
{
    return __drcp_rn(x);
}
template <>
__device__ __forceinline__ float
rrcp<float>(float x)
{
    return __fdividef(1.0f, x);
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
template <typename T, int BX, bool GX, bool GY, bool GZ, bool XY, bool XZ, bool YZ, class PT>
__device__ __forceinline__ FieldDerivs<T>
field_derivs(const state_t* __restrict__ c, const int* zo, const PT& P)
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

// ---- pairs of fields in packed FP32 lanes ----------------------------------
// add/sub/mul/fma.rn.f32x2 operate on two independent FP32 lanes with the
// rounding of the scalar operations, so a pair of fields whose stencils have
// the same shape forms its sums and differences in half the instructions, bit
// for bit as one field at a time. In the single-precision layout a pair is one
// array of 8-byte (A, B) elements, so an F2 is also one 8-byte load.
struct F2 {
    unsigned long long v;
};

__device__ __forceinline__ F2
pk2(float a, float b)
{
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}

__device__ __forceinline__ void
upk2(F2 r, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r.v));
}

__device__ __forceinline__ F2
add2(F2 a, F2 b)
{
    F2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}

__device__ __forceinline__ F2
sub2(F2 a, F2 b)
{
    F2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}

__device__ __forceinline__ F2
mul2(F2 a, F2 b)
{
    F2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}

__device__ __forceinline__ F2
fma2(F2 a, F2 b, F2 c)
{
    F2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}

// Register queue of one pair array along z (2.5D streaming): the (A, B)
// values of the thread's own column at the three planes below the current one
// and, where the pair has an xz (yz) cross derivative, the lower half of that
// derivative as running sums, both fields in packed lanes. The diagonal cross
// derivative at plane z,
//   sum_k e_k (f(+k,+k) + f(-k,-k) - f(+k,-k) - f(-k,+k))
//     = U(z) - L(z),  U(z) = sum_k e_k d_k(z+k),  L(z) = sum_k e_k d_k(z-k),
// with d_k(w) = f(+k) - f(-k) the x (y) difference at plane w: the differences
// of the current plane are formed for the first derivative anyway, and each
// contributes e_k d_k(z) to L(z+k). So the queue keeps
//   a1 = L(z),  a2 = the part of L(z+1) known so far,  a3 = that of L(z+2),
// and advancing a plane is three fused multiply-adds (no register moves):
//   a1 <- e1 d1(z) + a2,  a2 <- e2 d2(z) + a3,  a3 <- e3 d3(z).
// Only the upper half U is read from the ring.
struct PairQ {
    F2 v1, v2, v3;    // (A, B) at z-1, z-2, z-3
    F2 xa1, xa2, xa3; // xz lower half: L(z), partial L(z+1), partial L(z+2)
    F2 ya1, ya2, ya3; // the same for yz
};

// Advances the lower-half sums of one z diagonal past the plane whose
// differences are d1, d2, d3 (e: the diagonal's (c, c) coefficient pairs).
// The rounding sequence is fixed, so prime_pair below reproduces the sums a
// streaming task would have built, bit for bit.
__device__ __forceinline__ void
zacc_push(F2& a1, F2& a2, F2& a3, const unsigned long long* e, F2 d1, F2 d2, F2 d3)
{
    a1 = fma2(F2{e[0]}, d1, a2);
    a2 = fma2(F2{e[1]}, d2, a3);
    a3 = mul2(F2{e[2]}, d3);
}

// Upper half U of one z diagonal (u1..u3: d_k at plane z+k).
__device__ __forceinline__ F2
zacc_upper(const unsigned long long* e, F2 u1, F2 u2, F2 u3)
{
    return fma2(F2{e[2]}, u3, fma2(F2{e[1]}, u2, mul2(F2{e[0]}, u1)));
}

// Lower-half sums of a z diagonal at the first plane of a task from the three
// planes below it (zo[0..2]); step: 1 for xz, the row pitch for yz.
__device__ __forceinline__ void
zacc_prime(const F2* __restrict__ c, const int* zo, int step, const unsigned long long* e, F2& a1,
           F2& a2, F2& a3)
{
    auto d = [&](int plane, int k) { return sub2(c[zo[plane] + k * step], c[zo[plane] - k * step]); };
    // plane z-3: only its third difference reaches L(z)
    const F2 t3 = mul2(F2{e[2]}, d(0, 3));
    // plane z-2
    const F2 b2 = fma2(F2{e[1]}, d(1, 2), t3);
    const F2 b3 = mul2(F2{e[2]}, d(1, 3));
    // plane z-1
    a1 = fma2(F2{e[0]}, d(2, 1), b2);
    a2 = fma2(F2{e[1]}, d(2, 2), b3);
    a3 = mul2(F2{e[2]}, d(2, 3));
}

// Fills the queue of one pair array c from the ring at the first plane of a
// task (zo[0..2]: the three planes below it).
template <int BX, bool XZ, bool YZ, class PT>
__device__ __forceinline__ void
prime_pair(const F2* __restrict__ c, const int* zo, const PT& P, PairQ& Q)
{
    Q.v1 = c[zo[2]];
    Q.v2 = c[zo[1]];
    Q.v3 = c[zo[0]];
    if (XZ)
        zacc_prime(c, zo, 1, P.cxp[1], Q.xa1, Q.xa2, Q.xa3);
    if (YZ)
        zacc_prime(c, zo, BX, P.cxp[2], Q.ya1, Q.ya2, Q.ya3);
}

template <bool GX_, bool GY_, bool GZ_, bool XY_, bool XZ_, bool YZ_>
struct DFlags {
    static constexpr bool GX = GX_, GY = GY_, GZ = GZ_, XY = XY_, XZ = XZ_, YZ = YZ_;
};

// The z-diagonal cross derivative of kind XK (xz, else yz) of both fields of
// a pair, in packed lanes: upper half from the ring, lower half queued.
template <bool XK, int BX, class PT>
__device__ __forceinline__ void
zcross_pair(const F2* __restrict__ c, const int* zo, const PT& P, const PairQ& Q,
            float& sA, float& sB)
{
    constexpr int step = XK ? 1 : BX;
    F2 u[3];
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const int z = zo[3 + k];
        u[k - 1]    = sub2(c[z + k * step], c[z - k * step]);
    }
    const F2 s = sub2(zacc_upper(P.cxp[XK ? 1 : 2], u[0], u[1], u[2]), XK ? Q.xa1 : Q.ya1);
    upk2(s, sA, sB);
}

// Advances a pair's queue by one plane (after every use of it): F0 and the
// x / y differences DX, DY of the plane just done.
template <bool XZ, bool YZ, class PT>
__device__ __forceinline__ void
push_queue(PairQ& Q, const PT& P, F2 F0, const F2* DX, const F2* DY)
{
    if (XZ)
        zacc_push(Q.xa1, Q.xa2, Q.xa3, P.cxp[1], DX[0], DX[1], DX[2]);
    if (YZ)
        zacc_push(Q.ya1, Q.ya2, Q.ya3, P.cxp[2], DY[0], DY[1], DY[2]);
    Q.v3 = Q.v2;
    Q.v2 = Q.v1;
    Q.v1 = F0;
}

// The derivatives of the two fields of one pair array c at once: every pencil
// sum and difference, the xy diagonals and the z diagonals in packed lanes
// (each stencil point one 8-byte load); the coefficient sums. Second
// derivatives in difference form (below). F0 returns the pair's centre values.
template <int BX, class FA, class FB, class PT>
__device__ __forceinline__ void
pair_derivs_q(const F2* __restrict__ c, const int* zo, const PT& P,
              PairQ& Q, FieldDerivs<float>& rA, FieldDerivs<float>& rB, F2& F0)
{
    static_assert(FA::XY == FB::XY && FA::XZ == FB::XZ && FA::YZ == FB::YZ,
                  "the fields of a pair have the same cross derivatives");
    F0 = c[0];
    float a0, b0;
    upk2(F0, a0, b0);
    rA.v = a0;
    rB.v = b0;
    F2 DX[3], SX[3], DY[3], SY[3], DZ[3], SZ[3];
    // Second differences as u + v with u = f(+k) - f0, v = f(-k) - f0: for a
    // smooth field u and v are exact in FP32 (Sterbenz), so f(+k) + f(-k) - 2 f0
    // keeps its digits instead of cancelling terms of size |c0 f0| (about
    // 2.7 f / ds^2); mathematically the same stencil (c0 = -2 (c1 + c2 + c3)).
    // The FP32 build, whose error is that of its FP32 state, keeps the plain
    // sums f(+k) + f(-k) and adds c0 f0 (two packed operations per point pair
    // instead of three); the difference form is what brings the mixed build
    // within 2.2e-7 of FP64.
    // First differences f(+k) - f(-k) directly, as prime_pair forms the queued
    // ones, so results do not depend on where a task's z segment starts.
    // The difference form is evaluated as S = 2 (f(-k) - f0) + (f(+k) - f(-k)),
    // one fused multiply-add on the two exact differences (the first
    // difference is formed anyway): a single rounding of the same value,
    // three packed operations per point pair instead of four.
    constexpr bool DIFF_FORM = ACB_MIXED != 0;
    auto dsum = [&](F2 p, F2 m, F2& D, F2& S) {
        D = sub2(p, m);
        if constexpr (DIFF_FORM)
            S = fma2(F2{0x4000000040000000ull}, sub2(m, F0), D); // (2, 2) * (m - f0) + D
        else
            S = add2(p, m);
    };
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        dsum(c[k], c[-k], DX[k - 1], SX[k - 1]);
        dsum(c[k * BX], c[-k * BX], DY[k - 1], SY[k - 1]);
    }
    dsum(c[zo[4]], Q.v1, DZ[0], SZ[0]);
    dsum(c[zo[5]], Q.v2, DZ[1], SZ[1]);
    dsum(c[zo[6]], Q.v3, DZ[2], SZ[2]);
    // Coefficient sums sum_k c_k d_k of both fields at once, with (c, c)
    // coefficient pairs from the kernel parameters.
    auto sum3 = [&](const unsigned long long* cp, const F2* d, float& oa, float& ob) {
        F2 r = mul2(F2{cp[0]}, d[0]);
        r    = fma2(F2{cp[1]}, d[1], r);
        upk2(fma2(F2{cp[2]}, d[2], r), oa, ob);
    };
    float gA, gB;
    if (FA::GX || FB::GX) {
        sum3(P.c1p[0], DX, gA, gB);
        if (FA::GX) rA.gx = gA;
        if (FB::GX) rB.gx = gB;
    }
    if (FA::GY || FB::GY) {
        sum3(P.c1p[1], DY, gA, gB);
        if (FA::GY) rA.gy = gA;
        if (FB::GY) rB.gy = gB;
    }
    if (FA::GZ || FB::GZ) {
        sum3(P.c1p[2], DZ, gA, gB);
        if (FA::GZ) rA.gz = gA;
        if (FB::GZ) rB.gz = gB;
    }
    if constexpr (DIFF_FORM) {
        sum3(P.c2p[0] + 1, SX, rA.xx, rB.xx);
        sum3(P.c2p[1] + 1, SY, rA.yy, rB.yy);
        sum3(P.c2p[2] + 1, SZ, rA.zz, rB.zz);
    }
    else {
        // c0 f0 + sum_k c_k (f(+k) + f(-k))
        auto sum4 = [&](const unsigned long long* cp, const F2* d, float& oa, float& ob) {
            F2 r = mul2(F2{cp[0]}, F0);
            r    = fma2(F2{cp[1]}, d[0], r);
            r    = fma2(F2{cp[2]}, d[1], r);
            upk2(fma2(F2{cp[3]}, d[2], r), oa, ob);
        };
        sum4(P.c2p[0], SX, rA.xx, rB.xx);
        sum4(P.c2p[1], SY, rA.yy, rB.yy);
        sum4(P.c2p[2], SZ, rA.zz, rB.zz);
    }

    // xy diagonals (the whole stencil from the centre plane)
    if (FA::XY) {
        F2 E[3];
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            const int pp = k + k * BX, mm = -k - k * BX, pm = k - k * BX, mp = -k + k * BX;
            E[k - 1] = sub2(add2(c[pp], c[mm]), add2(c[pm], c[mp]));
        }
        sum3(P.cxp[0], E, rA.xy, rB.xy);
    }

    // z diagonals (both fields have the same kinds)
    if (FA::XZ)
        zcross_pair<true, BX>(c, zo, P, Q, rA.xz, rB.xz);
    if (FA::YZ)
        zcross_pair<false, BX>(c, zo, P, Q, rA.yz, rB.yz);

    push_queue<FA::XZ, FA::YZ>(Q, P, F0, DX, DY);
}

// Derivative flags of the eight fields: what the right-hand sides use.
//                   GX     GY     GZ     XY     XZ     YZ
#define ACB_D_LNRHO true, true, true, false, false, false
#define ACB_D_UUX true, true, true, true, true, false
#define ACB_D_UUY true, true, true, true, false, true
#define ACB_D_UUZ true, true, true, false, true, true
#define ACB_D_AX false, true, true, true, true, false
#define ACB_D_AY true, false, true, true, false, true
#define ACB_D_AZ true, true, false, false, true, true
#define ACB_D_SS true, true, true, false, false, false

template <typename T, class PT>
__device__ __forceinline__ void rhs_terms(const FieldDerivs<T>& lr, const FieldDerivs<T>& ux,
                                          const FieldDerivs<T>& uy, const FieldDerivs<T>& uz,
                                          const FieldDerivs<T>& ax, const FieldDerivs<T>& ay,
                                          const FieldDerivs<T>& az, const FieldDerivs<T>& ss,
                                          const PT& P, T roc[ACB_NF], T cur[ACB_NF]);

// Right-hand sides of the eight fields at one vertex, every stencil operand
// read from the ring.
template <typename T, int BX, int FIELD, class PT>
__device__ __forceinline__ void
mhd_rhs(const state_t* __restrict__ c, const int* zo, const PT& P, T roc[ACB_NF],
        T cur[ACB_NF])
{
    const auto lr = field_derivs<T, BX, ACB_D_LNRHO>(c + 0 * FIELD, zo, P);
    const auto ux = field_derivs<T, BX, ACB_D_UUX>(c + 1 * FIELD, zo, P);
    const auto uy = field_derivs<T, BX, ACB_D_UUY>(c + 2 * FIELD, zo, P);
    const auto uz = field_derivs<T, BX, ACB_D_UUZ>(c + 3 * FIELD, zo, P);
    const auto ax = field_derivs<T, BX, ACB_D_AX>(c + 4 * FIELD, zo, P);
    const auto ay = field_derivs<T, BX, ACB_D_AY>(c + 5 * FIELD, zo, P);
    const auto az = field_derivs<T, BX, ACB_D_AZ>(c + 6 * FIELD, zo, P);
    const auto ss = field_derivs<T, BX, ACB_D_SS>(c + 7 * FIELD, zo, P);
    rhs_terms(lr, ux, uy, uz, ax, ay, az, ss, P, roc, cur);
}

// The same with the z register queues (single-precision stencils), one pair
// array at a time: (lnrho, ss), (ux, ax), (uy, ay), (uz, az). cur2 returns the
// centre values of each array.
template <int BX, int FIELD, class PT>
__device__ __forceinline__ void
mhd_rhs_q(const F2* __restrict__ c, const int* zo, const PT& P,
          float roc[ACB_NF], float cur[ACB_NF], F2 cur2[ACB_NARR], PairQ (&Q)[ACB_NARR])
{
    FieldDerivs<float> lr, ux, uy, uz, ax, ay, az, ss;
    pair_derivs_q<BX, DFlags<ACB_D_LNRHO>, DFlags<ACB_D_SS>>(c + 0 * FIELD, zo, P, Q[0], lr, ss,
                                                             cur2[0]);
    pair_derivs_q<BX, DFlags<ACB_D_UUX>, DFlags<ACB_D_AX>>(c + 1 * FIELD, zo, P, Q[1], ux, ax,
                                                           cur2[1]);
    pair_derivs_q<BX, DFlags<ACB_D_UUY>, DFlags<ACB_D_AY>>(c + 2 * FIELD, zo, P, Q[2], uy, ay,
                                                           cur2[2]);
    pair_derivs_q<BX, DFlags<ACB_D_UUZ>, DFlags<ACB_D_AZ>>(c + 3 * FIELD, zo, P, Q[3], uz, az,
                                                           cur2[3]);
    rhs_terms(lr, ux, uy, uz, ax, ay, az, ss, P, roc, cur);
}

template <int BX, int FIELD, class PT>
__device__ __forceinline__ void
prime_queues(const F2* __restrict__ c, const int* zo, const PT& P,
             PairQ (&Q)[ACB_NARR])
{
    prime_pair<BX, false, false>(c + 0 * FIELD, zo, P, Q[0]);
    prime_pair<BX, true, false>(c + 1 * FIELD, zo, P, Q[1]);
    prime_pair<BX, false, true>(c + 2 * FIELD, zo, P, Q[2]);
    prime_pair<BX, true, true>(c + 3 * FIELD, zo, P, Q[3]);
}

// Right-hand sides from the derivative sets (stencil_kernel.ac:355-528,
// restated; same terms).
template <typename T, class PT>
__device__ __forceinline__ void
rhs_terms(const FieldDerivs<T>& lr, const FieldDerivs<T>& ux, const FieldDerivs<T>& uy,
          const FieldDerivs<T>& uz, const FieldDerivs<T>& ax, const FieldDerivs<T>& ay,
          const FieldDerivs<T>& az, const FieldDerivs<T>& ss, const PT& P,
          T roc[ACB_NF], T cur[ACB_NF])
{
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
    const T inv_rho = rrcp<T>(rho);

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
    // T = exp(lnT0 + E) = exp(lnT0) exp(E): the exponential of E is formed
    // above already
    const T inv_pT = rrcp<T>(rho * (P.exp_lnT0 * expE));
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
// a single device: global index = local index, global grid = local grid), the
// double-precision build's; the single-precision builds form the phase by
// parts (forcing_column, forcing_plane and forcing_from below).
template <typename T>
__device__ __forceinline__ void
forcing_at(const SolveParams<T>& P, int i, int j, int k, T f[3])
{
    static_assert(sizeof(T) == 8, "the single-precision builds use forcing_from");
    T skx, ckx;
    const T x0 = (T)(i - NGHOST) * P.fds[0] * P.fxs[0];
    const T x1 = (T)(j - NGHOST) * P.fds[1] * P.fxs[1];
    const T x2 = (T)(k - NGHOST) * P.fds[2] * P.fxs[2];
    const T kx = P.fk[0] * x0 + P.fk[1] * x1 + P.fk[2] * x2;
    sincos(kx, &skx, &ckx);
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

// sin and cos of a double-precision phase, reduced to [-pi, pi] in double
// precision first
__device__ __forceinline__ void
sincos_reduced(double ph, float& s, float& c)
{
    const double red = ph - 6.283185307179586 * rint(ph * 0.15915494309189535);
    sincosf((float)red, &s, &c);
}

// The single-precision builds' forcing, by parts: the phase k.x + phi of
// vertex (i, j, k) is (k_x x + k_y y) + k_z z + phi, and exp(i (k.x + phi)) is
// the product of exp(i (k_x x + k_y y + phi)), formed once per column of a task
// (forcing_column), and exp(i k_z z), once per plane (forcing_plane; a warp's
// lanes form 32 planes' at a time, shuffled to the vertex's plane). Each part's
// phase is formed in double precision and reduced before its sin and cos, as
// forcing_at does for the whole phase; the product adds one rounding of a unit
// complex number. The exponentials then cost once per column and plane instead
// of once per vertex (the forced substep 2: 5.79 -> 5.44 ms at 512^3, 49.4 ->
// 46.3 ms at 1024^3, same-box A/B).
template <typename T>
__device__ __forceinline__ void
forcing_column(const SolveParams<T>& P, int i, int j, float& cxy, float& sxy)
{
    const double x0 = ((double)(i - NGHOST) * (double)P.fds[0]) * P.fxs_d[0];
    const double x1 = ((double)(j - NGHOST) * (double)P.fds[1]) * P.fxs_d[1];
    float s, c;
    sincos_reduced((double)P.fk[0] * x0 + (double)P.fk[1] * x1, s, c);
    cxy = c * (float)P.fcphi - s * (float)P.fsphi; // times exp(i phi)
    sxy = s * (float)P.fcphi + c * (float)P.fsphi;
}

template <typename T>
__device__ __forceinline__ void
forcing_plane(const SolveParams<T>& P, int k, float& cz, float& sz)
{
    const double x2 = ((double)(k - NGHOST) * (double)P.fds[2]) * P.fxs_d[2];
    sincos_reduced((double)P.fk[2] * x2, sz, cz);
}

template <typename T>
__device__ __forceinline__ void
forcing_from(const SolveParams<T>& P, float cxy, float sxy, float cz, float sz, T f[3])
{
    const float re = cxy * cz - sxy * sz;
    const float im = sxy * cz + cxy * sz;
    bool ok        = true;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        f[c] = (T)(P.fscale * (P.ff_re[c] * re - P.ff_im[c] * im));
        ok   = ok && isfinite(f[c]);
    }
    if (!ok)
        f[0] = f[1] = f[2] = 0;
}

// Compensated sum of float pairs (hi, lo) and float increments d, two fields
// in packed lanes: a two-sum of hi and d (s and its exact error e), the error
// added to lo, and the result renormalised so that |olo| <= ulp(ohi) / 2.
__device__ __forceinline__ void
pair_add2(F2 hi, F2 lo, F2 d, F2& ohi, F2& olo)
{
    const F2 s  = add2(hi, d);
    const F2 bb = sub2(s, hi);
    const F2 e  = add2(sub2(hi, sub2(s, bb)), sub2(d, bb)); // two-sum error
    const F2 l  = add2(lo, e);
    ohi         = add2(s, l); // renormalise
    olo         = sub2(l, sub2(ohi, s));
}

} // namespace acb

// Step diagnostics of the output state, accumulated per consumer thread while
// the last substep writes it: max, min and sum of |u|^2 and sum of
// exp(lnrho)^2, in FP64 from the stored values (hi + lo in the mixed build),
// each value formed exactly as the reduction kernels form it (reduce.cuh:
// red_load, red_len2, the RMS_EXP filter), so max and min equal a separate
// pass bit for bit (sqrt is monotonic) and the sums differ only in their order.
struct DiagAcc {
    double mx, mn, su, se;
};

__device__ __forceinline__ void
diag_init(DiagAcc& a)
{
    a.mx = -INFINITY;
    a.mn = INFINITY;
    a.su = 0.0;
    a.se = 0.0;
}

__device__ __forceinline__ void
diag_add(DiagAcc& a, double lnrho, double ux, double uy, double uz)
{
    const double l2 = __fma_rn(uz, uz, __fma_rn(uy, uy, __dmul_rn(ux, ux)));
    a.mx            = fmax(a.mx, l2);
    a.mn            = fmin(a.mn, l2);
    a.su += l2;
    const double e = exp(lnrho);
    a.se += e * e;
}

// Values of the vertex's own column that the update needs besides the ring:
// the previous state (s > 0) and, in the mixed build, the lo parts.
// FP64 build: one value per field.
struct CentreVals {
    AcReal prev[ACB_NF];
};

template <int STEP>
__device__ __forceinline__ void
load_centre(const Layout& L, const state_t* out, long long id, CentreVals& c)
{
#pragma unroll
    for (int f = 0; f < ACB_NF; ++f)
        if (STEP > 0)
            c.prev[f] = out[fidx(L, f, id)];
}

// The lo parts of pair array ar from a lo element (two bf16x2 words, the
// even array's in the low one) as a float pair, and a float pair as a bf16x2
// word (lane A in the low half); bf16 to float is exact.
__device__ __forceinline__ acb::F2
lo_unpack(unsigned long long e, int ar)
{
    const uint32_t x = (ar & 1) ? (uint32_t)(e >> 32) : (uint32_t)e;
    return acb::pk2(__uint_as_float(x << 16), __uint_as_float(x & 0xffff0000u));
}

__device__ __forceinline__ uint32_t
lo_pack(acb::F2 v)
{
    float a, b;
    acb::upk2(v, a, b);
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a)); // b high, a low
    return r;
}

// Single-precision layout: one (A, B) element per pair array; lo parts in
// the mixed build.
struct CentreVals2 {
    acb::F2 prev[ACB_NARR];
    acb::F2 cur_lo[ACB_NARR];
    acb::F2 prev_lo[ACB_NARR];
};

template <int STEP>
__device__ __forceinline__ void
load_centre2(const Layout& L, const state_t* out, const lo16_t* in_lo, const lo16_t* out_lo,
             long long id, CentreVals2& c)
{
    const acb::F2* o               = reinterpret_cast<const acb::F2*>(out);
    const unsigned long long* il   = reinterpret_cast<const unsigned long long*>(in_lo);
    const unsigned long long* ol   = reinterpret_cast<const unsigned long long*>(out_lo);
#pragma unroll
    for (int a = 0; a < ACB_NARR; ++a) {
        const long long e = a * L.fstride + id;
        if (STEP > 0)
            c.prev[a] = o[e];
#if ACB_MIXED
        const long long el = (a >> 1) * L.fstride + id;
        c.cur_lo[a]        = lo_unpack(il[el], a);
        c.prev_lo[a]       = STEP > 0 ? lo_unpack(ol[el], a) : acb::F2{0ull};
#endif
    }
    (void)il;
    (void)ol;
}

// The same values of the vertex a plane above into L1, while this plane's
// right-hand sides run (their plain loads then hit L1 instead of waiting on
// memory: FP32 512^3 step 13.17 -> 13.07 ms, FP32 ensemble step 5.52 -> 5.41 ms).
template <int STEP>
__device__ __forceinline__ void
prefetch_centre2(const Layout& L, const state_t* out, const lo16_t* in_lo, const lo16_t* out_lo,
                 long long id)
{
    const acb::F2* o             = reinterpret_cast<const acb::F2*>(out);
    const unsigned long long* il = reinterpret_cast<const unsigned long long*>(in_lo);
    const unsigned long long* ol = reinterpret_cast<const unsigned long long*>(out_lo);
#pragma unroll
    for (int a = 0; a < ACB_NARR; ++a) {
        if (STEP > 0)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(o + a * L.fstride + id));
#if ACB_MIXED
        if ((a & 1) == 0) {
            const long long el = (a >> 1) * L.fstride + id;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(il + el));
            if (STEP > 0)
                asm volatile("prefetch.global.L1 [%0];" ::"l"(ol + el));
        }
#endif
    }
    (void)o;
    (void)il;
    (void)ol;
}

template <class Cfg>
struct TaskGeom {
    int i0, j0, k0, nout;
    __device__ __forceinline__ TaskGeom(const SolveGeom& g, long long t, long long ntiles)
    {
        const long long seg  = t / ntiles;
        const long long tile = t - seg * ntiles;
        const int tile_x     = (int)(tile % g.ntx);
        const int tile_y     = (int)(tile / g.ntx);
        i0                   = NGHOST + (g.tx0 + tile_x) * Cfg::TX;
        j0                   = g.start.y + tile_y * Cfg::TY;
        k0                   = g.start.z + (int)seg * g.zseg;
        nout                 = min(g.zseg, g.nzr - (int)seg * g.zseg);
    }
};

__device__ __forceinline__ void
fence_tensormap_acquire(const CUtensorMap* map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                     reinterpret_cast<uint64_t>(map))
                 : "memory");
}

// Which member an ensemble task belongs to (binary search on task_begin).
template <typename T>
__device__ __forceinline__ int
member_of(const MemberDesc<T>* md, int n, long long t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (md[mid].task_begin <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}


// One task of a consumer warp: the planes of one (tile, z segment) column.
// Waits for the ring, computes and stores every output plane, releases the
// slots, and advances the plane counter q. Returns false if the CTA aborts.
template <class Cfg, int STEP, bool ENS, bool DTDEV, bool DIAG, class PT>
__device__ __forceinline__ bool
consume_task(const SolveArgs<AcReal>& a, const SolveGeom& gv, const PT& P,
             long long lt, state_t* out, lo16_t* in_lo, lo16_t* out_lo, const void* ring,
             uint64_t* full, uint64_t* empty, volatile int* abort_flag, uint32_t& q,
             const void* centre, uint64_t* full_c, uint64_t* empty_c, uint32_t& oq,
             DiagAcc& dacc)
{
    using CS          = CentreSet<STEP>;
    constexpr bool CT = Cfg::NC > 0 && !ENS && CS::STAGE;
    using T = AcReal;
    constexpr int TX = Cfg::TX, NP = Cfg::NP, BX = Cfg::BX;
    constexpr int FIELD = Cfg::FIELD, PLANE = Cfg::PLANE;
    const int tid  = threadIdx.x;
    const int lane = tid & 31;
    const int tx   = tid % TX;
    const int ty   = tid / TX;
    const Layout& L = gv.L;
    const TaskGeom<Cfg> tg(gv, lt, (long long)gv.ntx * gv.nty);
    const int nload = tg.nout + 2 * NGHOST;
    const int i     = tg.i0 + tx;
    const int j     = tg.j0 + ty;
    const bool act  = (i >= gv.start.x) && (i < gv.end.x) && (j < gv.end.y);
    const T rkA     = a.P.rkA;
    T rkB           = a.P.rkB;
    if constexpr (DTDEV)
        rkB = (T)(a.P.rk_beta * *a.P.dt_dev);
    // this thread's column in a ring slot (elements)
    const int col = (ty + NGHOST) * BX + (tx + 4);

    bool ok = true;
    for (int l = 0; l < 2 * NGHOST && ok; ++l)
        ok = mbar_wait_bounded(&full[(q + l) % NP], ((q + l) / NP) & 1u);
    ok = __all_sync(0xffffffffu, ok);

    // single precision streams with the z register queues (2.5D) over the pair
    // arrays; double precision has no registers to spare for them and reads
    // every operand from the ring
    constexpr bool QZ = ACB_PAIRED;
    acb::PairQ Q[ACB_NARR];
    if constexpr (QZ) {
        if (ok && act) {
            const uint32_t sc = (q + NGHOST) % NP;
            int zo[7];
#pragma unroll
            for (int dz = -NGHOST; dz <= NGHOST; ++dz)
                zo[dz + NGHOST] = ((int)((q + NGHOST + dz) % NP) - (int)sc) * PLANE;
            const acb::F2* c = reinterpret_cast<const acb::F2*>(ring) + (size_t)sc * PLANE + col;
            acb::prime_queues<BX, FIELD>(c, zo, P, Q);
        }
        // the three planes below the first output plane now live in the queues
        __syncwarp();
        if (lane == 0 && ok)
            for (int l = 0; l < NGHOST; ++l)
                mbar_arrive(&empty[(q + l) % NP]);
    }

    // forcing (s = 2 with forcing; single precision): the column's phase factor
    float fcxy = 0.f, fsxy = 0.f, fcz = 0.f, fsz = 0.f;
    if constexpr (STEP == 3 && QZ)
        acb::forcing_column(a.P, i, j, fcxy, fsxy);
    (void)fcxy;
    (void)fsxy;

    // double precision (no queues, registers to spare for it): the centre
    // values of the next plane are loaded a plane ahead
    constexpr bool PREF = !QZ;
    CentreVals cv_next;
    if constexpr (PREF)
        if (act)
            load_centre<STEP>(L, out, lidx(L, i, j, tg.k0), cv_next);

    for (int p = 0; p < tg.nout; ++p) {
        if (ok) {
            const uint32_t l = q + p + 2 * NGHOST;
            ok = mbar_wait_bounded(&full[l % NP], (l / NP) & 1u);
            ok = __all_sync(0xffffffffu, ok);
        }
        if constexpr (CT) {
            if (ok) {
                ok = mbar_wait_bounded(&full_c[oq % Cfg::NC], (oq / Cfg::NC) & 1u);
                ok = __all_sync(0xffffffffu, ok);
            }
        }
        if (!ok || *abort_flag) {
            if (lane == 0) {
                atomicOr(a.status, (unsigned)ACB_STATUS_TMA_TIMEOUT);
                *abort_flag = 1;
            }
            return false;
        }
        const int k = tg.k0 + p;
        float fcb = 0.f, fsb = 0.f; // the plane's forcing phase factor
        if constexpr (STEP == 3 && QZ) {
            if ((p & 31) == 0) // lane l: plane p + l
                acb::forcing_plane(a.P, k + lane, fcz, fsz);
            fcb = __shfl_sync(0xffffffffu, fcz, p & 31);
            fsb = __shfl_sync(0xffffffffu, fsz, p & 31);
        }
        (void)fcb;
        (void)fsb;
        if (act) {
            const long long id = lidx(L, i, j, k);
            const uint32_t sc  = (q + p + NGHOST) % NP;
            int zo[7];
#pragma unroll
            for (int dz = -NGHOST; dz <= NGHOST; ++dz) {
                if (QZ && dz < 0)
                    continue;
                const int sd    = (int)((q + p + NGHOST + dz) % NP);
                zo[dz + NGHOST] = (sd - (int)sc) * PLANE;
            }
            T fo[3] = {0, 0, 0};
            if constexpr (QZ) {
                // previous state and lo parts of this vertex: plain loads issued
                // first, or (CT) read from the centre slot after the right-hand
                // sides, which keeps their registers free through the stencils
                CentreVals2 cv;
                if constexpr (!CT) {
                    load_centre2<STEP>(L, out, in_lo, out_lo, id, cv);
                    if (p + 1 < tg.nout)
                        prefetch_centre2<STEP>(L, out, in_lo, out_lo, id + L.plane);
                }
                const acb::F2* c = reinterpret_cast<const acb::F2*>(ring) + (size_t)sc * PLANE + col;
                float roc[ACB_NF], cur[ACB_NF];
                acb::F2 cur2[ACB_NARR];
                acb::mhd_rhs_q<BX, FIELD>(c, zo, P, roc, cur, cur2, Q);
                if constexpr (STEP == 3)
                    acb::forcing_from<T>(a.P, fcxy, fsxy, fcb, fsb, fo);
                if constexpr (CT) {
                    // from the centre slot the producer filled by TMA
                    // slot: prev hi [array][TY][TX], then cur lo and prev lo
                    // [lo array][TY][TX], 8-byte elements
                    const acb::F2* cs = reinterpret_cast<const acb::F2*>(centre) +
                                        (size_t)(oq % Cfg::NC) * (Cfg::centre_slot_bytes() / 8) +
                                        ty * TX + tx;
                    const unsigned long long* csu =
                        reinterpret_cast<const unsigned long long*>(cs);
                    constexpr int FS  = Cfg::TX * Cfg::TY;
                    constexpr int OCL = CS::PREV ? Cfg::CENTRE : 0; // cur lo
                    constexpr int OPL = OCL + Cfg::CENTRE_LO;       // prev lo
#pragma unroll
                    for (int ar = 0; ar < ACB_NARR; ++ar) {
                        if constexpr (CS::PREV)
                            cv.prev[ar] = cs[ar * FS];
#if ACB_MIXED
                        cv.cur_lo[ar] = lo_unpack(csu[OCL + (ar >> 1) * FS], ar);
                        if constexpr (CS::PREV)
                            cv.prev_lo[ar] = lo_unpack(csu[OPL + (ar >> 1) * FS], ar);
                        else
                            cv.prev_lo[ar] = acb::F2{0ull};
#endif
                    }
                    (void)csu;
                }
                // The update, two fields per instruction (one pair array):
                //   FP32:  out = cur + rkA (cur - prev) + rkB roc  [+ forcing]
                //   mixed: d = rkB roc (+ rkA ((cur - prev) + (cur_lo - prev_lo)))
                //          (hi, lo) = (cur, cur_lo) + d, a two-sum  [+ forcing]
                // Forcing acts on ux, uy, uz, lane 0 of arrays 1-3; the lane of
                // ax, ay, az adds 0 (for the mixed pair, adding 0 to a pair that
                // pair_add2 returned leaves it as it is).
                const acb::F2 rkA2 = acb::pk2(rkA, rkA), rkB2 = acb::pk2(rkB, rkB);
                acb::F2* o2 = reinterpret_cast<acb::F2*>(out);
#if ACB_MIXED
                unsigned long long* ol2 = reinterpret_cast<unsigned long long*>(out_lo);
                uint32_t lo_even = 0; // the even array's bf16x2 word, stored with the odd one's
#endif
                // lane 0 of arrays 0..3 holds lnrho, ux, uy, uz: their stored
                // values for the step diagnostics (hi and, mixed, lo)
                float dh[ACB_NARR], dl[ACB_NARR];
#pragma unroll
                for (int ar = 0; ar < ACB_NARR; ++ar) {
                    const int fa = acb_field(ar, 0), fb = acb_field(ar, 1);
                    const long long e = ar * L.fstride + id;
                    const acb::F2 roc2 = acb::pk2(roc[fa], roc[fb]);
#if ACB_MIXED
                    const acb::F2 l2 = cv.cur_lo[ar];
                    acb::F2 d2       = acb::mul2(rkB2, roc2);
                    if (STEP > 0) {
                        const acb::F2 x = acb::add2(acb::sub2(cur2[ar], cv.prev[ar]),
                                                    acb::sub2(l2, cv.prev_lo[ar]));
                        d2 = acb::fma2(rkA2, x, d2);
                    }
                    acb::F2 h2, w2;
                    acb::pair_add2(cur2[ar], l2, d2, h2, w2);
                    if (STEP == 3 && ar >= 1)
                        acb::pair_add2(h2, w2, acb::pk2(fo[ar - 1], 0.f), h2, w2);
                    o2[e] = h2;
                    const uint32_t wl = lo_pack(w2); // lo rounded to bf16 as stored
                    if (ar & 1)
                        ol2[(ar >> 1) * L.fstride + id] =
                            (unsigned long long)lo_even | ((unsigned long long)wl << 32);
                    else
                        lo_even = wl;
                    if constexpr (DIAG) {
                        float t_;
                        acb::upk2(h2, dh[ar], t_);
                        acb::upk2(lo_unpack(wl, 0), dl[ar], t_);
                    }
#else
                    acb::F2 r;
                    if (STEP == 0)
                        r = acb::fma2(rkB2, roc2, cur2[ar]);
                    else
                        r = acb::fma2(rkB2, roc2,
                                      acb::fma2(rkA2, acb::sub2(cur2[ar], cv.prev[ar]), cur2[ar]));
                    if (STEP == 3 && ar >= 1)
                        r = acb::add2(r, acb::pk2(fo[ar - 1], 0.f));
                    o2[e] = r;
                    if constexpr (DIAG) {
                        float t_;
                        acb::upk2(r, dh[ar], t_);
                        dl[ar] = 0.f;
                    }
#endif
                }
                if constexpr (DIAG) {
                    // (double)hi + (double)lo, as the reductions read a value
                    double v[4];
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        v[f] = (double)dh[f];
#if ACB_MIXED
                        v[f] += (double)dl[f];
#endif
                    }
                    diag_add(dacc, v[0], v[1], v[2], v[3]);
                }
                (void)cur;
                (void)dh;
                (void)dl;
            }
            else {
                // double precision: previous state loaded a plane ahead
                CentreVals cv = cv_next;
                if (p + 1 < tg.nout)
                    load_centre<STEP>(L, out, id + L.plane, cv_next);
                const state_t* c = reinterpret_cast<const state_t*>(ring) + (size_t)sc * PLANE + col;
                T roc[ACB_NF], cur[ACB_NF];
                acb::mhd_rhs<T, BX, FIELD>(c, zo, P, roc, cur);
                if constexpr (STEP == 3)
                    acb::forcing_at<T>(a.P, i, j, k, fo);
                T dv[4];
#pragma unroll
                for (int f = 0; f < ACB_NF; ++f) {
                    T r;
                    if (STEP == 0)
                        r = cur[f] + rkB * roc[f];
                    else
                        r = cur[f] + rkA * (cur[f] - cv.prev[f]) + rkB * roc[f];
                    if (STEP == 3 && f >= 1 && f <= 3)
                        r += fo[f - 1];
                    out[fidx(L, f, id)] = r;
                    if (f < 4)
                        dv[f] = r;
                }
                if constexpr (DIAG)
                    diag_add(dacc, (double)dv[0], (double)dv[1], (double)dv[2], (double)dv[3]);
                (void)dv;
            }
        }
        __syncwarp();
        // with the queues the centre plane is done with; without them the
        // plane three below it
        if (lane == 0)
            mbar_arrive(&empty[(q + p + (QZ ? NGHOST : 0)) % NP]);
        if constexpr (CT) {
            if (lane == 0)
                mbar_arrive(&empty_c[oq % Cfg::NC]);
            ++oq;
        }
    }
    // the planes of the task not released yet
    __syncwarp();
    if (lane == 0)
        for (int l = tg.nout + (QZ ? NGHOST : 0); l < nload; ++l)
            mbar_arrive(&empty[(q + l) % NP]);
    q += nload;
    return true;
}

// Warp-specialised pipeline. Warp CWARPS is the producer: one lane issues one
// TMA load per plane (all 8 fields of the halo'd tile) into a ring of NP
// slots, each guarded by a `full` barrier (transaction bytes) and an `empty`
// barrier on which every consumer warp arrives once it has finished with the
// plane. Consumer warps own one vertex column each and never wait for each
// other except through the ring. Tasks (tile, z segment) are dealt round-robin
// so the CTAs of one wave stream neighbouring tiles at the same z and their
// halo reads of each other's planes hit L2. With ENS the tasks of all members
// of an ensemble form one list (member-major) and each task reads its member's
// map, geometry, buffers and parameters from the descriptor table.
template <bool ENS>
using SolveKernelArgs = typename std::conditional<ENS, EnsSolveArgs<AcReal>, SolveArgs<AcReal>>::type;

// Folds the consumer threads' step diagnostics: a warp butterfly, the warps
// in order, one partial per CTA, and the last CTA to finish folds the partials
// (its first warp: lane l takes CTAs l, l + 32, ... in order, then a fixed
// butterfly) into a.diag_result. Deterministic; no atomics on data. Every
// consumer warp reaches it, also after an abort (its waits are bounded).
template <class Cfg>
__device__ __forceinline__ void
diag_finish(const SolveArgs<AcReal>& a, DiagAcc d)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        d.mx = fmax(d.mx, __shfl_xor_sync(0xffffffffu, d.mx, o));
        d.mn = fmin(d.mn, __shfl_xor_sync(0xffffffffu, d.mn, o));
        d.su += __shfl_xor_sync(0xffffffffu, d.su, o);
        d.se += __shfl_xor_sync(0xffffffffu, d.se, o);
    }
    __shared__ double wred[Cfg::CWARPS][4];
    __shared__ int dlast;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        wred[warp][0] = d.mx;
        wred[warp][1] = d.mn;
        wred[warp][2] = d.su;
        wred[warp][3] = d.se;
    }
    // the consumer warps only: the producer warps have left
    asm volatile("bar.sync 1, %0;" ::"n"(Cfg::CONSUMERS) : "memory");
    if (threadIdx.x == 0) {
        double r[4] = {wred[0][0], wred[0][1], wred[0][2], wred[0][3]};
        for (int w = 1; w < Cfg::CWARPS; ++w) {
            r[0] = fmax(r[0], wred[w][0]);
            r[1] = fmin(r[1], wred[w][1]);
            r[2] += wred[w][2];
            r[3] += wred[w][3];
        }
        double* p = a.diag_partials + 4 * (size_t)blockIdx.x;
        p[0]      = r[0];
        p[1]      = r[1];
        p[2]      = r[2];
        p[3]      = r[3];
        __threadfence();
        dlast = atomicAdd(a.diag_counter, 1u) == gridDim.x - 1;
    }
    asm volatile("bar.sync 1, %0;" ::"n"(Cfg::CONSUMERS) : "memory");
    if (!dlast || warp != 0)
        return;
    __threadfence();
    const volatile double* v = a.diag_partials;
    double f0 = -INFINITY, f1 = INFINITY, f2 = 0.0, f3 = 0.0;
    for (unsigned b = lane; b < gridDim.x; b += 32) {
        f0 = fmax(f0, v[4 * b + 0]);
        f1 = fmin(f1, v[4 * b + 1]);
        f2 += v[4 * b + 2];
        f3 += v[4 * b + 3];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        f0 = fmax(f0, __shfl_xor_sync(0xffffffffu, f0, o));
        f1 = fmin(f1, __shfl_xor_sync(0xffffffffu, f1, o));
        f2 += __shfl_xor_sync(0xffffffffu, f2, o);
        f3 += __shfl_xor_sync(0xffffffffu, f3, o);
    }
    if (lane == 0) {
        a.diag_result[0] = f0;
        a.diag_result[1] = f1;
        a.diag_result[2] = f2;
        a.diag_result[3] = f3;
        *a.diag_counter  = 0u; // zero for the next launch
        __threadfence();
    }
}

// DTDEV: the time step is read from device memory (SolveParams::dt_dev), for
// steps whose time step the device chooses; single meshes, no forcing.
// DIAG: the launch also folds the step diagnostics of its output (diag_finish);
// single meshes, the last substep over the whole interior.
template <class Cfg, int STEP, bool ENS, bool DTDEV = false, bool DIAG = false>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MINB)
    solve_kernel(const __grid_constant__ CUtensorMap tin,
                 const __grid_constant__ SolveKernelArgs<ENS> a,
                 const __grid_constant__ CentreMaps cm)
{
    using T = AcReal;
    constexpr int TX = Cfg::TX, NP = Cfg::NP, BX = Cfg::BX;
    constexpr int FIELD = Cfg::FIELD, PLANE = Cfg::PLANE, CWARPS = Cfg::CWARPS;
    constexpr uint32_t PLANE_BYTES = PLANE * ACB_ELEM;

    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* ring = smem_raw; // NP slots of PLANE_BYTES
    __shared__ __align__(8) uint64_t full[NP];
    __shared__ __align__(8) uint64_t empty[NP];
    // centre ring (CT): one slot per output plane, filled by the producer
    // together with the deepest stencil plane that output needs
    using CS             = CentreSet<STEP>;
    constexpr bool CT    = Cfg::NC > 0 && !ENS && CS::STAGE;
    constexpr int NCS    = CT ? Cfg::NC : 1;
    __shared__ __align__(8) uint64_t full_c[NCS];
    __shared__ __align__(8) uint64_t empty_c[NCS];
    unsigned char* centre = smem_raw + Cfg::ring_bytes(); // NC slots of centre_slot_bytes
    __shared__ volatile int abort_flag;

    const int tid  = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < NP; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CWARPS);
        }
        for (int s = 0; s < NCS; ++s) {
            mbar_init(&full_c[s], 1);
            mbar_init(&empty_c[s], CWARPS);
        }
        fence_barrier_init();
        abort_flag = 0;
    }
    __syncthreads();

    const long long ntasks = ENS ? a.total_tasks : a.g.tasks; // (ENS: the group's tasks)

    if constexpr (Cfg::WGSPEC) {
        // whole warpgroups: warps 0..7 consume, warps 8..11 produce
        if (warp >= CWARPS)
            asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(Cfg::REG_PRODUCER));
        else
            asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(Cfg::REG_CONSUMER));
    }

    if (warp >= CWARPS) {
        // ------------------------------------------------------------ producer
        if (warp == CWARPS && lane == 0) {
            if (!ENS)
                prefetch_tensormap(&tin);
            uint32_t q  = 0;
            uint32_t oq = 0; // output planes whose centre arrays were issued
            bool ok     = true;
            int last_m  = -1;
            for (long long t = blockIdx.x; t < ntasks && ok; t += gridDim.x) {
                const CUtensorMap* map = &tin;
                const SolveGeom* g     = &a.g;
                long long lt           = t;
                if constexpr (ENS) {
                    const long long tg_      = t + a.task_base; // task in the whole list
                    const int m              = member_of(a.members, a.nmembers, tg_);
                    const MemberDesc<T>* md  = a.members + m;
                    map                      = &md->tmap;
                    g                        = &md->g;
                    lt                       = tg_ - md->task_begin;
                    if (m != last_m) {
                        fence_tensormap_acquire(map);
                        prefetch_tensormap(map);
                        last_m = m;
                    }
                }
                const TaskGeom<Cfg> tg(*g, lt, (long long)g->ntx * g->nty);
                const int xt    = g->L.offx + tg.i0 - 4; // a multiple of 16 bytes by construction
                const int yt    = tg.j0 - NGHOST;
                const int nload = tg.nout + 2 * NGHOST;
                for (int l = 0; l < nload; ++l) {
                    const uint32_t s = q % NP, use = q / NP;
                    if (use > 0 && !mbar_wait_bounded(&empty[s], (use - 1) & 1u)) {
                        ok = false;
                        break;
                    }
                    if (abort_flag) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[s], PLANE_BYTES);
                    tma_load_4d(ring + (size_t)s * PLANE_BYTES, map, xt, yt, tg.k0 - NGHOST + l, 0,
                                &full[s]);
                    ++q;
                    if constexpr (CT) {
                        // plane l is the top one output l - 6 needs: its centre
                        // arrays go out now, into the next centre slot
                        if (l >= 2 * NGHOST) {
                            const uint32_t sc = oq % Cfg::NC, usec = oq / Cfg::NC;
                            if (usec > 0 && !mbar_wait_bounded(&empty_c[sc], (usec - 1) & 1u)) {
                                ok = false;
                                break;
                            }
                            constexpr uint32_t CB = Cfg::CENTRE * ACB_ELEM;    // prev hi
                            constexpr uint32_t CL = Cfg::CENTRE_LO * ACB_ELEM; // a lo set
                            constexpr uint32_t OC = CS::PREV ? CB : 0;        // cur lo
                            constexpr uint32_t OP = OC + CL;                   // prev lo
                            constexpr uint32_t TXB = (CS::PREV ? CB : 0) + (CS::LO ? CL : 0) +
                                                     ((CS::LO && CS::PREV) ? CL : 0);
                            unsigned char* dst = centre + (size_t)sc * Cfg::centre_slot_bytes();
                            const int xc = g->L.offx + tg.i0; // interior tile start: 32-byte aligned
                            const int zc = tg.k0 + (l - 2 * NGHOST);
                            mbar_arrive_expect_tx(&full_c[sc], TXB);
                            if (CS::PREV)
                                tma_load_4d(dst, &cm.m[0], xc, tg.j0, zc, 0, &full_c[sc]);
                            if (CS::LO)
                                tma_load_4d(dst + OC, &cm.m[1], xc, tg.j0, zc, 0, &full_c[sc]);
                            if (CS::LO && CS::PREV)
                                tma_load_4d(dst + OP, &cm.m[2], xc, tg.j0, zc, 0, &full_c[sc]);
                            ++oq;
                        }
                    }
                }
            }
            if (!ok) {
                atomicOr(a.status, (unsigned)ACB_STATUS_TMA_TIMEOUT);
                abort_flag = 1;
                // wait (bounded) for this CTA's loads still in flight before leaving
                for (uint32_t r = q > (uint32_t)NP ? q - NP : 0; r < q; ++r)
                    (void)mbar_wait_bounded(&full[r % NP], (r / NP) & 1u);
                if constexpr (CT)
                    for (uint32_t r = oq > (uint32_t)Cfg::NC ? oq - Cfg::NC : 0; r < oq; ++r)
                        (void)mbar_wait_bounded(&full_c[r % Cfg::NC], (r / Cfg::NC) & 1u);
            }
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    uint32_t q = 0, oq = 0;
    DiagAcc dacc;
    diag_init(dacc);
    for (long long t = blockIdx.x; t < ntasks; t += gridDim.x) {
        bool ok;
        if constexpr (ENS) {
            // the group's members: descriptor table and parameters from the
            // launch (a.members points at the group's first descriptor)
            const long long tg_     = t + a.task_base;
            const int m             = member_of(a.members, a.nmembers, tg_);
            const MemberDesc<T>* md = a.members + m;
            const SolveGeom gv      = md->g;
            ok = consume_task<Cfg, STEP, ENS, DTDEV, false>(a, gv, a.mp[m], tg_ - md->task_begin,
                                                     md->out, md->in_lo, md->out_lo, ring, full,
                                                     empty, &abort_flag, q, centre, full_c,
                                                     empty_c, oq, dacc);
        }
        else {
            ok = consume_task<Cfg, STEP, ENS, DTDEV, DIAG>(a, a.g, a.P, t, a.out, a.in_lo, a.out_lo,
                                                    ring, full, empty, &abort_flag, q, centre,
                                                    full_c, empty_c, oq, dacc);
        }
        if (!ok) {
            if constexpr (DIAG)
                break; // every consumer warp still reaches the fold
            else
                return;
        }
    }
    if constexpr (DIAG)
        diag_finish<Cfg>(a, dacc);
}

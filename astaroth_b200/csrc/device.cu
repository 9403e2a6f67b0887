// Device layer of the B200 MHD solver: the acDevice* entry points of
// include/astaroth.h (reference src/core/device.cc:23-538 and
// src/core/kernels/kernels.cu:102-251) over the kernels in solve.cuh, halo.cuh
// and reduce.cuh, plus the additions declared in include/astaroth_b200.h.
//
// Differences of design from the reference, all invisible at the interface:
//   - the eight fields of `in` (and of `out`) live in one allocation with a
//     padded row pitch, in single precision as four arrays of interleaved
//     field pairs (common.cuh: Layout, fidx); load/store translate between the
//     caller's flat mx*my*mz arrays and that layout through a device staging
//     buffer and a scatter / gather kernel;
//   - the run-time parameters ("uniforms") are a per-Device host mirror of
//     AcMeshInfo, turned into pre-scaled kernel arguments at each launch,
//     instead of one __constant__ AcMeshInfo per GPU; loads keep the
//     reference's rule of skipping NaN/inf values with a warning;
//   - reductions use per-device FP64 scratch of one double per CTA.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "astaroth.h"
#include "astaroth_b200.h"
#include "common.cuh"
#include "halo.cuh"
#include "reduce.cuh"
#include "solve.cuh"
#include "internal.cuh"

using namespace acb_host;

const SolveConfig*
acb_host::solve_configs(int* n)
{
#if AC_DOUBLE_PRECISION == 1
    static const SolveConfig table[] = {
        make_solve_config<SolveCfg0, false>(),
        make_solve_config<SolveCfg1, false>(),
        make_solve_config<SolveCfg2, false>(),
    };
#else
    static const SolveConfig table[] = {
        make_solve_config<SolveCfg0, false>(),
        make_solve_config<SolveCfg1, false>(),
        make_solve_config<SolveCfg2, false>(),
    };
#endif
    *n = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

// ---------------------------------------------------------------------------
// The device object
// ---------------------------------------------------------------------------
// One captured whole step and the host-side block state a replay leaves.
struct StepGraph {
    cudaGraphExec_t exec;
    unsigned long long key;
    double extra; // a launch parameter the graph was captured with (CFL: time scale)
    unsigned long long launches;
    bool ghost[2]; // ghost_ok of both blocks after a replay
    bool lo[2];    // lo_stale of both blocks after a replay
    bool diag;     // the captured step's last substep folds the step diagnostics
};

enum { STEP_FIXED = 0, STEP_CFL = 1 };

struct device_s {
    int id;
    AcMeshInfo local_config;
    AcMeshInfo uniforms; // host mirror of the device parameters
    cudaStream_t streams[NUM_STREAMS];
    int num_sms;

    Layout L;
    state_t* blk[2]; // the two field blocks; blk[cur] is `in`
    lo16_t* lo[2];   // mixed build: lo blocks (bf16, see common.cuh)
    int cur;
    // ghost_ok[b]: block b's ghost zone holds the periodic images of its
    // interior (set by a full-box fill of all fields; cleared by any write to
    // the block). A fill of a block whose ghosts are already valid is skipped.
    bool ghost_ok[2];
    // lo_stale[b] (mixed build): the last whole-box fill of block b wrote the
    // hi parts of its ghosts only (the stencils never read the lo parts); the
    // lo parts are filled before anything reads or partly overwrites them
    bool lo_stale[2];

    CUtensorMap tmap[2];
    CentreMaps cmap[2]; // by parity of `in`: centre boxes over out hi, in lo, out lo
    int tmap_cfg;       // configuration the maps were encoded for (-1: none)

    double* red_partials; // 3 * ACB_RED_SETS * red_max_blocks (the multi-set pass)
    int red_max_blocks;
    unsigned* red_counter;
    double* red_result; // 3 * ACB_RED_SETS doubles
    double* h_result;   // pinned, 3 * ACB_RED_SETS doubles
    // Interiors written so far: bumped by every operation that can change a
    // block's interior values (the solve, loads, fills of whole fields,
    // transfers, graph replays). A MAX / MIN / RMS reduction of one field or
    // one vector's length computes all three in one pass, together with those
    // of the scalar fields whose bytes the pass reads anyway (a vector's
    // components and, in the single-precision builds, the fields sharing
    // their 8-byte elements), and keeps them here with the block and the epoch
    // they were taken at; later requests for any of them come from this record
    // while nothing has changed.
    unsigned long long write_epoch;
    struct {
        bool valid;
        const void* block;
        unsigned long long epoch;
        int n;     // entries, of every pass taken on this block and epoch
        bool wide; // the caller reduces several arrays of one state: passes
                   // also take the fields they read anyway (set by a second
                   // pass on one block and epoch, and kept)
        struct {
            int nin, handles[3];
            double vals[3]; // MAX, MIN, RMS sum
        } e[ACB_RED_RECORD];
    } red3;

    // Step diagnostics folded by the last substep's solve launch (enabled by
    // acDeviceSetStepDiagnostics): max, min and sum of |u|^2 and the sum of
    // exp(lnrho)^2 of the block it wrote, kept with that block and the epoch
    // after the launch; a reduction asking for one of them while nothing has
    // changed reads the record (one copy to the host for all four).
    bool step_diag;
    double* diag_partials; // 4 per CTA, diag_max_ctas CTAs
    int diag_max_ctas;
    unsigned* diag_counter;
    double* diag_result;   // 4 doubles
    double* h_diag;        // pinned, 4 doubles
    struct {
        bool valid, fetched;
        const void* block;
        unsigned long long epoch;
        double vals[4];
    } diag;

    double* xfer; // device staging buffer for the double-precision views
    size_t xfer_elems;
    StageBuf stage; // staging buffer of mesh loads

    unsigned* status;
    int solve_cfg;
    int forcing;
    unsigned long long launches;
    unsigned long long uniform_version;

    // whole-step graphs: [kind][starting buffer parity], kind 0 steps with
    // the time step given by the caller, kind 1 with the time step chosen on
    // the device (STEP_CFL)
    StepGraph graph[2][2];

    // time-step record of the steps whose dt is chosen on the device
    // (device memory): dt of the last such step, simulated time, steps taken
    double* cfl;
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static inline bool
real_is_valid(double v)
{
    return !isnan(v) && !isinf(v);
}

static inline cudaStream_t
stream_of(const Device d, Stream s)
{
    if (s < 0 || s >= NUM_STREAMS)
        s = STREAM_DEFAULT;
    return d->streams[s];
}

typedef CUresult (*PFN_encodeTiled_t)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                      const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                      const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                      CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled_t
get_encode_tiled()
{
    static PFN_encodeTiled_t fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_encodeTiled_t)p;
    }
    return fn;
}

AcResult
acb_host::encode_block_map(const Layout& L, const state_t* block, const SolveConfig& cfg,
                           CUtensorMap* map)
{
    PFN_encodeTiled_t enc = get_encode_tiled();
    if (!enc) {
        fprintf(stderr, "astaroth_b200: cuTensorMapEncodeTiled unavailable\n");
        return AC_FAILURE;
    }
    // the block's arrays of 8-byte elements (a field pair or a double); the
    // copy moves bits, so FLOAT64 serves both layouts
    const cuuint64_t esz     = ACB_ELEM;
    const cuuint64_t dim[4]  = {(cuuint64_t)L.mxp, (cuuint64_t)L.my, (cuuint64_t)L.mz, ACB_NARR};
    const cuuint64_t str[3]  = {(cuuint64_t)L.mxp * esz, (cuuint64_t)L.plane * esz,
                               (cuuint64_t)L.fstride * esz};
    const cuuint32_t box[4]  = {(cuuint32_t)(cfg.TX + 8), (cuuint32_t)(cfg.TY + 2 * NGHOST), 1,
                               ACB_NARR};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUresult r = enc(map, dt, 4, (void*)block, dim, str, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fprintf(stderr, "astaroth_b200: cuTensorMapEncodeTiled failed (%d)\n", (int)r);
        return AC_FAILURE;
    }
    return AC_SUCCESS;
}

AcResult
acb_host::encode_centre_map(const Layout& L, const void* block, const SolveConfig& cfg,
                            CUtensorMap* map, int narr)
{
    PFN_encodeTiled_t enc = get_encode_tiled();
    if (!enc) {
        fprintf(stderr, "astaroth_b200: cuTensorMapEncodeTiled unavailable\n");
        return AC_FAILURE;
    }
    const cuuint64_t esz     = ACB_ELEM;
    const cuuint64_t dim[4]  = {(cuuint64_t)L.mxp, (cuuint64_t)L.my, (cuuint64_t)L.mz,
                               (cuuint64_t)narr};
    const cuuint64_t str[3]  = {(cuuint64_t)L.mxp * esz, (cuuint64_t)L.plane * esz,
                               (cuuint64_t)L.fstride * esz};
    const cuuint32_t box[4]  = {(cuuint32_t)cfg.TX, (cuuint32_t)cfg.TY, 1, (cuuint32_t)narr};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(block), dim, str,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fprintf(stderr, "astaroth_b200: cuTensorMapEncodeTiled (centre) failed (%d)\n", (int)r);
        return AC_FAILURE;
    }
    return AC_SUCCESS;
}

static AcResult
ensure_maps(const Device d)
{
    if (d->tmap_cfg == d->solve_cfg)
        return AC_SUCCESS;
    int n;
    const SolveConfig* cfgs = solve_configs(&n);
    const SolveConfig& cfg = cfgs[d->solve_cfg];
    for (int b = 0; b < 2; ++b)
        if (encode_block_map(d->L, d->blk[b], cfg, &d->tmap[b]) != AC_SUCCESS)
            return AC_FAILURE;
    memset(d->cmap, 0, sizeof(d->cmap));
    if (cfg.NC > 0) {
        for (int p = 0; p < 2; ++p) {
            if (encode_centre_map(d->L, d->blk[p ^ 1], cfg, &d->cmap[p].m[0], ACB_NARR) != AC_SUCCESS)
                return AC_FAILURE;
            if (d->lo[p] &&
                (encode_centre_map(d->L, d->lo[p], cfg, &d->cmap[p].m[1], ACB_LO_NARR) != AC_SUCCESS ||
                 encode_centre_map(d->L, d->lo[p ^ 1], cfg, &d->cmap[p].m[2], ACB_LO_NARR) != AC_SUCCESS))
                return AC_FAILURE;
        }
    }
    d->tmap_cfg = d->solve_cfg;
    return AC_SUCCESS;
}

AcResult
acb_host::prepare_table(const SolveConfig* cfgs, int n)
{
    for (int c = 0; c < n; ++c)
        for (int st = 0; st < 10; ++st) {
            // kern[0..3], then kern_dt[0..2], then kern_diag[0..2]
            const void* k = st < 4   ? cfgs[c].kern[st]
                            : st < 7 ? cfgs[c].kern_dt[st - 4]
                                     : cfgs[c].kern_diag[st - 7];
            if (!k)
                continue;
            ACB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)cfgs[c].smem));
            // kernels that move registers between warpgroups must start with
            // enough of them, or the consumers' increase would wait for ever
            cudaFuncAttributes fa;
            ACB_CUDA_CHECK(cudaFuncGetAttributes(&fa, k));
            if (fa.numRegs < cfgs[c].launch_regs) {
                fprintf(stderr,
                        "astaroth_b200: solve kernel %s built with %d registers a thread, "
                        "needs %d for its register reallocation; refusing to launch it\n",
                        cfgs[c].name, fa.numRegs, cfgs[c].launch_regs);
                return AC_FAILURE;
            }
        }
    return AC_SUCCESS;
}

static AcResult
prepare_kernels_once()
{
    static bool done = false;
    if (done)
        return AC_SUCCESS;
    int n;
    const SolveConfig* cfgs = solve_configs(&n);
    if (prepare_table(cfgs, n) != AC_SUCCESS)
        return AC_FAILURE;
    done = true;
    return AC_SUCCESS;
}

// beta of the Williamson (1980) 2N scheme: rkB = beta[s] dt
static const double kRkBeta[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

// Kernel arguments from the uniform mirror (coefficients pre-scaled in double,
// rounded once to AcReal).
SolveParams<AcReal>
acb_host::make_params(const AcMeshInfo& uniforms, const Layout& L, int step, int forcing)
{
    const AcReal* rp = uniforms.real_params;
    SolveParams<AcReal> P;
    memset(&P, 0, sizeof(P));
    const double inv[3] = {rp[AC_inv_dsx], rp[AC_inv_dsy], rp[AC_inv_dsz]};
    const double c1[3]  = {3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0};
    const double c2[4]  = {-49.0 / 18.0, 3.0 / 2.0, -3.0 / 20.0, 1.0 / 90.0};
    const double cx[3]  = {270.0 / 720.0, -27.0 / 720.0, 2.0 / 720.0};
    for (int a = 0; a < 3; ++a) {
        for (int k = 0; k < 3; ++k)
            P.c1[a][k] = (AcReal)(c1[k] * inv[a]);
        for (int k = 0; k < 4; ++k)
            P.c2[a][k] = (AcReal)(c2[k] * inv[a] * inv[a]);
    }
    const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2}; // xy, xz, yz
    for (int p = 0; p < 3; ++p)
        for (int k = 0; k < 3; ++k)
            P.cx[p][k] = (AcReal)(cx[k] * inv[pa[p]] * inv[pb[p]]);
    if (sizeof(AcReal) == 4) {
        // the same coefficients as (c, c) lane pairs for the packed stencil sums
        auto dup = [](AcReal c) {
            uint32_t b;
            memcpy(&b, &c, 4);
            return ((unsigned long long)b << 32) | b;
        };
        for (int a = 0; a < 3; ++a) {
            for (int k = 0; k < 3; ++k)
                P.c1p[a][k] = dup(P.c1[a][k]);
            for (int k = 0; k < 4; ++k)
                P.c2p[a][k] = dup(P.c2[a][k]);
        }
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k)
                P.cxp[r][k] = dup(P.cx[r][k]);
    }

    const double gamma = rp[AC_gamma], cp = rp[AC_cp_sound], mu0 = rp[AC_mu0];
    P.nu           = rp[AC_nu_visc];
    P.eta          = rp[AC_eta];
    P.inv_mu0      = (AcReal)(1.0 / mu0);
    P.eta_mu0      = (AcReal)((double)rp[AC_eta] * mu0);
    P.zeta         = rp[AC_zeta];
    P.cs2_sound    = rp[AC_cs2_sound];
    P.inv_cp       = (AcReal)(1.0 / cp);
    P.gamma        = (AcReal)gamma;
    P.gm1          = (AcReal)(gamma - 1.0);
    P.gamma_inv_cp = (AcReal)(gamma / cp);
    P.lnrho0       = rp[AC_lnrho0];
    P.lnT0         = rp[AC_lnT0];
    P.exp_lnT0     = (AcReal)exp((double)rp[AC_lnT0]);
    P.k_heat       = (AcReal)0.001; // AC_THERMAL_CONDUCTIVITY of the module

    // Williamson (1980) 2N coefficients, "previous state" form
    const double alpha[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double* beta    = kRkBeta;
    const double dt       = rp[AC_dt];
    P.rkB                 = (AcReal)(beta[step] * dt);
    P.rkA                 = step > 0 ? (AcReal)(beta[step] * alpha[step] / beta[step - 1]) : 0;

    P.forcing = forcing;
    if (forcing) {
        const double cs    = sqrt((double)rp[AC_cs2_sound]);
        const double kaver = rp[AC_kaver];
        const double NN    = cs * (double)rp[AC_forcing_magnitude] * sqrt(kaver * cs);
        P.fscale           = (AcReal)(sqrt(dt) * NN);
        P.fk[0]            = rp[AC_k_forcex];
        P.fk[1]            = rp[AC_k_forcey];
        P.fk[2]            = rp[AC_k_forcez];
        P.ff_re[0]         = rp[AC_ff_hel_rex];
        P.ff_re[1]         = rp[AC_ff_hel_rey];
        P.ff_re[2]         = rp[AC_ff_hel_rez];
        P.ff_im[0]         = rp[AC_ff_hel_imx];
        P.ff_im[1]         = rp[AC_ff_hel_imy];
        P.ff_im[2]         = rp[AC_ff_hel_imz];
        P.fcphi            = (AcReal)cos((double)rp[AC_forcing_phase]);
        P.fsphi            = (AcReal)sin((double)rp[AC_forcing_phase]);
        const int3 gn      = uniforms.int3_params[AC_global_grid_n];
        const int nn[3]    = {gn.x > 0 ? gn.x : L.nx, gn.y > 0 ? gn.y : L.ny,
                           gn.z > 0 ? gn.z : L.nz};
        const double ds[3] = {rp[AC_dsx], rp[AC_dsy], rp[AC_dsz]};
        for (int c = 0; c < 3; ++c) {
            P.fds[c]   = (AcReal)ds[c];
            P.fxs[c]   = (AcReal)(2.0 * M_PI / (ds[c] * nn[c]));
            P.fxs_d[c] = 2.0 * M_PI / (ds[c] * nn[c]);
        }
    }
    return P;
}

// Cuts z into 1..8 segments of at least `min_planes` planes so that the last
// wave of (tile, segment) tasks is as full as possible; fewer segments win
// near-ties because each segment re-reads 6 halo planes.
int
acb_host::choose_segments(long long ntiles, int nzr, long long slots, int min_planes)
{
    int best_seg    = 1;
    double best_eff = -1.0;
    for (int ns = 1; ns <= 8; ++ns) {
        if (ns > 1 && nzr / ns < min_planes)
            break;
        const long long T    = ntiles * ns;
        const long long wave = (T + slots - 1) / slots;
        const double eff     = (double)T / (double)(wave * slots) - 0.01 * (ns - 1);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best_seg = ns;
        }
    }
    return best_seg;
}

static bool
box_in_interior(const Device d, int3 s, int3 e)
{
    const Layout& L = d->L;
    return s.x >= NGHOST && s.y >= NGHOST && s.z >= NGHOST && e.x <= NGHOST + L.nx &&
           e.y <= NGHOST + L.ny && e.z <= NGHOST + L.nz;
}

// dt_dev: when given, the solve reads the time step from this device double
// (the record of acDeviceIntegrateStepCFL) instead of the AC_dt uniform.
static AcResult
launch_solve(const Device d, cudaStream_t st, int step, int3 s, int3 e,
             const double* dt_dev = nullptr)
{
    if (step < 0 || step > 2) {
        fprintf(stderr, "astaroth_b200: invalid substep %d\n", step);
        return AC_FAILURE;
    }
    if (!box_in_interior(d, s, e)) {
        fprintf(stderr, "astaroth_b200: integration box outside the computational domain\n");
        return AC_FAILURE;
    }
    if (e.x <= s.x || e.y <= s.y || e.z <= s.z)
        return AC_SUCCESS;
    if (prepare_kernels_once() != AC_SUCCESS || ensure_maps(d) != AC_SUCCESS)
        return AC_FAILURE;
    int n;
    const SolveConfig& cfg = solve_configs(&n)[d->solve_cfg];

    SolveArgs<AcReal> a;
    memset(&a, 0, sizeof(a));
    SolveGeom& g = a.g;
    g.L          = d->L;
    g.start      = s;
    g.end        = e;
    g.tx0        = (s.x - NGHOST) / cfg.TX;
    g.ntx        = (e.x - 1 - NGHOST) / cfg.TX - g.tx0 + 1;
    g.nty        = (e.y - s.y + cfg.TY - 1) / cfg.TY;
    g.nzr        = e.z - s.z;
    a.out        = d->blk[d->cur ^ 1];
    a.in_lo      = d->lo[d->cur];
    a.out_lo     = d->lo[d->cur ^ 1];
    a.status     = d->status;
    a.P          = make_params(d->uniforms, d->L, step, d->forcing);
    if (dt_dev) {
        a.P.dt_dev  = dt_dev;
        a.P.rk_beta = kRkBeta[step];
    }

    // the last substep over the whole interior folds the step diagnostics
    // when they are enabled
    const bool whole = s.x == NGHOST && s.y == NGHOST && s.z == NGHOST &&
                       e.x == NGHOST + d->L.nx && e.y == NGHOST + d->L.ny &&
                       e.z == NGHOST + d->L.nz;
    const bool diag = d->step_diag && step == 2 && whole;
    SolveKernelFn kern;
    if (diag)
        kern = (SolveKernelFn)cfg.kern_diag[dt_dev ? 2 : (d->forcing ? 1 : 0)];
    else
        kern = dt_dev ? (SolveKernelFn)cfg.kern_dt[step]
                      : (SolveKernelFn)cfg.kern[step == 2 && d->forcing ? 3 : step];
    int per_sm = 0;
    ACB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern,
                                                                 cfg.threads, cfg.smem));
    if (per_sm < 1)
        per_sm = 1;
    const long long slots = (long long)d->num_sms * per_sm;
    const long long ntiles = (long long)g.ntx * g.nty;
    const int best_seg     = choose_segments(ntiles, g.nzr, slots, 16);
    g.nseg  = best_seg;
    g.zseg  = (g.nzr + best_seg - 1) / best_seg;
    g.nseg  = (g.nzr + g.zseg - 1) / g.zseg;
    g.tasks = ntiles * g.nseg;
    long long grid = std::min(slots, g.tasks);
    if (diag) {
        if (grid > d->diag_max_ctas) {
            fprintf(stderr, "astaroth_b200: %lld CTAs exceed the step diagnostics' %d partials\n",
                    grid, d->diag_max_ctas);
            return AC_FAILURE;
        }
        a.diag_partials = d->diag_partials;
        a.diag_counter  = d->diag_counter;
        a.diag_result   = d->diag_result;
    }
    kern<<<(unsigned)grid, cfg.threads, cfg.smem, st>>>(d->tmap[d->cur], a, d->cmap[d->cur]);
    ACB_CUDA_CHECK(cudaGetLastError());
    d->launches++;
    d->write_epoch++;
    if (diag) {
        d->diag.valid   = true;
        d->diag.fetched = false;
        d->diag.block   = d->blk[d->cur ^ 1];
        d->diag.epoch   = d->write_epoch;
    }
    d->ghost_ok[d->cur ^ 1] = false; // the out block's ghosts are stale now
    d->lo_stale[d->cur ^ 1] = false; // (all of them, hi and lo alike)
    return AC_SUCCESS;
}

// Fills the lo parts of block b's ghosts with their periodic images if the last
// whole-box fill of b left them (see lo_stale): the lo block has the layout of
// the hi block with ACB_LO_NARR arrays of 8-byte elements (four bfloat16 lo
// parts each), filled like the hi parts.
static AcResult
ensure_lo_ghosts(const Device d, cudaStream_t st, int b)
{
    if (!d->lo[b] || !d->lo_stale[b])
        return AC_SUCCESS;
    const Layout& L       = d->L;
    const long long units = halo_units(L, ACB_LO_NARR);
    const int blocks =
        (int)std::max(1LL, std::min((units + 255) / 256, (long long)d->num_sms * 32));
    halo_full_kernel<<<blocks, 256, 0, st>>>(L, d->lo[b], (unsigned)halo_units_a(L, ACB_LO_NARR),
                                             (unsigned)units, ACB_LO_NARR);
    ACB_CUDA_CHECK(cudaGetLastError());
    d->launches++;
    d->lo_stale[b] = false;
    return AC_SUCCESS;
}

static AcResult
launch_halo(const Device d, cudaStream_t st, int3 s, int3 e, int f0, int f1)
{
    const Layout& L = d->L;
    s.x             = std::max(s.x, 0);
    s.y             = std::max(s.y, 0);
    s.z             = std::max(s.z, 0);
    e.x             = std::min(e.x, L.mx);
    e.y             = std::min(e.y, L.my);
    e.z             = std::min(e.z, L.mz);
    if (e.x <= s.x || e.y <= s.y || e.z <= s.z)
        return AC_SUCCESS;
    if (d->ghost_ok[d->cur])
        return AC_SUCCESS; // every ghost already holds its periodic image
    const bool whole = f0 == 0 && f1 == NUM_VTXBUF_HANDLES && s.x == 0 && s.y == 0 && s.z == 0 &&
                       e.x == L.mx && e.y == L.my && e.z == L.mz;
    if (whole) {
        const long long units = halo_units(L);
        const long long want  = (units + 255) / 256;
        const int blocks = (int)std::max(1LL, std::min(want, (long long)d->num_sms * 32));
        halo_full_kernel<<<blocks, 256, 0, st>>>(L, d->blk[d->cur], (unsigned)halo_units_a(L),
                                                 (unsigned)units, ACB_NARR);
        ACB_CUDA_CHECK(cudaGetLastError());
        d->launches++;
        d->ghost_ok[d->cur] = true;
        d->lo_stale[d->cur] = d->lo[d->cur] != nullptr;
        return AC_SUCCESS;
    }
    if (ensure_lo_ghosts(d, st, d->cur) != AC_SUCCESS)
        return AC_FAILURE;
    HaloArgs a;
    a.L     = L;
    a.block = d->blk[d->cur];
    a.lo    = d->lo[d->cur];
    a.start = s;
    a.end   = e;
    a.f0    = f0;
    a.f1    = f1;
    a.rows  = (long long)(e.y - s.y) * (e.z - s.z);
    long long blocks = (a.rows + 7) / 8;
    blocks           = std::min(blocks, (long long)d->num_sms * 16);
    halo_kernel<<<(unsigned)blocks, 256, 0, st>>>(a);
    ACB_CUDA_CHECK(cudaGetLastError());
    d->launches++;
    return AC_SUCCESS;
}

// Arguments and grid of a reduction over the interior of the current block
// into the Device's scratch (result in d->red_result).
static AcResult
reduce_args(const Device d, int rtype, int nin, const int* handles, ReduceArgs& a,
            long long& blocks)
{
    const Layout& L = d->L;
    memset(&a, 0, sizeof(a));
    a.L = L;
    for (int w = 0; w < nin; ++w) {
        if (handles[w] < 0 || handles[w] >= NUM_VTXBUF_HANDLES)
            return AC_FAILURE;
        a.f[w]  = d->blk[d->cur] + fidx(L, handles[w], 0);
        a.lo[w] = lo_field(d->lo[d->cur], L, handles[w]);
    }
    a.nin      = nin;
    a.rtype    = rtype;
    a.start    = make_int3(NGHOST, NGHOST, NGHOST);
    a.end      = make_int3(NGHOST + L.nx, NGHOST + L.ny, NGHOST + L.nz);
    a.rows     = (long long)L.ny * L.nz;
    a.partials = d->red_partials;
    a.counter  = d->red_counter;
    a.result   = d->red_result;
    blocks     = (a.rows + 7) / 8;
    blocks     = std::max(1LL, std::min(blocks, (long long)d->red_max_blocks));
    return AC_SUCCESS;
}

static AcResult
run_reduce(const Device d, cudaStream_t st, int rtype, int nin, const int* handles,
           double* result)
{
    ReduceArgs a;
    long long blocks;
    if (reduce_args(d, rtype, nin, handles, a, blocks) != AC_SUCCESS)
        return AC_FAILURE;
    const int which  = rtype == RTYPE_MAX ? 0 : (rtype == RTYPE_MIN ? 1 : (rtype == RTYPE_RMS ? 2 : -1));
    // the step diagnostics the last solve folded, while the block is unchanged
    const bool is_u = nin == RED_VEC && handles[0] == VTXBUF_UUX && handles[1] == VTXBUF_UUY &&
                      handles[2] == VTXBUF_UUZ;
    const int dq = is_u && which >= 0 ? which
                   : (nin == RED_SCAL && rtype == RTYPE_RMS_EXP && handles[0] == VTXBUF_LNRHO)
                       ? 3
                       : -1;
    if (dq >= 0 && d->diag.valid && d->diag.block == d->blk[d->cur] &&
        d->diag.epoch == d->write_epoch) {
        if (!d->diag.fetched) {
            ACB_CUDA_CHECK(cudaMemcpyAsync(d->h_diag, d->diag_result, 4 * sizeof(double),
                                           cudaMemcpyDeviceToHost, st));
            ACB_CUDA_CHECK(cudaStreamSynchronize(st));
            for (int q = 0; q < 4; ++q)
                d->diag.vals[q] = d->h_diag[q];
            d->diag.fetched = true;
        }
        // max and min were folded as |u|^2: sqrt is monotonic and correctly
        // rounded, so this is the max (min) of the lengths a pass would take
        *result = dq <= 1 ? sqrt(d->diag.vals[dq]) : d->diag.vals[dq];
        return AC_SUCCESS;
    }
    if (which >= 0 && (nin == RED_SCAL || nin == RED_VEC)) {
        // MAX, MIN and RMS together: one pass serves all three requests, and
        // those of the scalar fields whose bytes it reads, while the block is
        // unchanged (the diagnostics of a step)
        auto& c    = d->red3;
        auto match = [&](int e) {
            return c.e[e].nin == nin && c.e[e].handles[0] == handles[0] &&
                   (nin == RED_SCAL ||
                    (c.e[e].handles[1] == handles[1] && c.e[e].handles[2] == handles[2]));
        };
        if (c.valid && c.block == d->blk[d->cur] && c.epoch == d->write_epoch)
            for (int e = 0; e < c.n; ++e)
                if (match(e)) {
                    *result = c.e[e].vals[which];
                    return AC_SUCCESS;
                }
        // a second pass on this block and epoch: from now on the passes take
        // every field they read (the first pass of a state, all that a caller
        // reducing one quantity makes, stays the three-in-one pass)
        if (c.valid && c.block == d->blk[d->cur] && c.epoch == d->write_epoch && c.n > 0)
            c.wide = true;
        // the pass's inputs: the request's fields, then (single precision)
        // the fields sharing their elements
        int in[6], nf = 0;
        for (int w = 0; w < nin; ++w)
            in[nf++] = handles[w];
        if (ACB_PAIRED && c.wide) {
            for (int w = 0; w < nin; ++w)
                in[nf++] = acb_field(acb_array(handles[w]), 1 - acb_lane(handles[w]));
            for (int x = 0; x < nf; ++x) // all distinct, or the request alone
                for (int y = x + 1; y < nf; ++y)
                    if (in[x] == in[y])
                        nf = nin;
        }
        for (int w = 0; w < nf; ++w) {
            a.f[w]  = d->blk[d->cur] + fidx(d->L, in[w], 0);
            a.lo[w] = lo_field(d->lo[d->cur], d->L, in[w]);
        }
        // sets: the request, then each input as a scalar (a scalar request's
        // own field excepted)
        const int ns = !c.wide ? 1 : (nin == RED_SCAL ? nf : 1 + nf);
        if (ns == 1)
            reduce3_kernel<256><<<(unsigned)blocks, 256, 0, st>>>(a);
        else if (nin == RED_SCAL)
            reduce_sets_kernel<256, RED_SCAL, 2><<<(unsigned)blocks, 256, 0, st>>>(a);
        else if (ns == 4)
            reduce_sets_kernel<256, RED_VEC, 4><<<(unsigned)blocks, 256, 0, st>>>(a);
        else
            reduce_sets_kernel<256, RED_VEC, 7><<<(unsigned)blocks, 256, 0, st>>>(a);
        ACB_CUDA_CHECK(cudaGetLastError());
        d->launches++;
        ACB_CUDA_CHECK(cudaMemcpyAsync(d->h_result, d->red_result, 3 * ns * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
        ACB_CUDA_CHECK(cudaStreamSynchronize(st));
        // kept beside the entries of earlier passes on this block and epoch
        if (!(c.valid && c.block == d->blk[d->cur] && c.epoch == d->write_epoch) ||
            c.n + ns > ACB_RED_RECORD)
            c.n = 0;
        c.valid = true;
        c.block = d->blk[d->cur];
        c.epoch = d->write_epoch;
        for (int t = 0; t < ns; ++t) {
            auto& e        = c.e[c.n + t];
            const bool req = t == 0;
            e.nin          = req ? nin : RED_SCAL;
            for (int w = 0; w < 3; ++w)
                e.handles[w] = req ? (w < nin ? handles[w] : -1)
                                   : (w == 0 ? in[nin == RED_SCAL ? t : t - 1] : -1);
            for (int q = 0; q < 3; ++q)
                e.vals[q] = d->h_result[3 * t + q];
        }
        *result = c.e[c.n].vals[which];
        c.n += ns;
        return AC_SUCCESS;
    }
    reduce_kernel<256><<<(unsigned)blocks, 256, 0, st>>>(a);
    ACB_CUDA_CHECK(cudaGetLastError());
    d->launches++;
    ACB_CUDA_CHECK(cudaMemcpyAsync(d->h_result, d->red_result, sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    *result = *d->h_result;
    return AC_SUCCESS;
}

// Element index (lidx) of the vertex at flat reference-order index idx.
__device__ __forceinline__ long long
flat_to_elem(const Layout& L, unsigned long long idx)
{
    const unsigned long long mx = (unsigned long long)L.mx, row = idx / mx;
    return (long long)L.offx + (long long)row * L.mxp + (long long)(idx - row * mx);
}

// Scatters n consecutive values of a field (field: its base, fidx(L, f, 0)) in
// reference order, starting at flat index s, from a staging buffer into the
// padded layout (and zeroes their lo parts when given: fresh values carry none).
__global__ void
scatter_rows_kernel(const Layout L, state_t* __restrict__ field, lo16_t* __restrict__ lo,
                    const state_t* __restrict__ flat, unsigned long long s, unsigned long long n)
{
    for (unsigned long long u = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
         u += (unsigned long long)gridDim.x * blockDim.x) {
        const long long e = flat_to_elem(L, s + u);
        field[e * ACB_LANES] = flat[u];
        if (lo)
            lo[e * ACB_LO_STEP] = 0;
    }
}

// The reverse: n values of a field from the padded layout into a staging
// buffer in reference order.
__global__ void
gather_rows_kernel(const Layout L, const state_t* __restrict__ field, state_t* __restrict__ flat,
                   unsigned long long s, unsigned long long n)
{
    for (unsigned long long u = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
         u += (unsigned long long)gridDim.x * blockDim.x)
        flat[u] = field[flat_to_elem(L, s + u) * ACB_LANES];
}

AcResult
acb_host::stage_create(StageBuf* stage, size_t max_elems)
{
    const size_t cap = ((size_t)64 << 20) / sizeof(state_t);
    stage->elems     = std::max<size_t>(1, std::min(max_elems, cap));
    stage->buf       = nullptr;
    stage->done      = nullptr;
    ACB_CUDA_CHECK(cudaMalloc((void**)&stage->buf, stage->elems * sizeof(state_t)));
    ACB_CUDA_CHECK(cudaEventCreateWithFlags(&stage->done, cudaEventDisableTiming));
    return AC_SUCCESS;
}

void
acb_host::stage_destroy(StageBuf* stage)
{
    if (stage->buf)
        cudaFree(stage->buf);
    if (stage->done)
        cudaEventDestroy(stage->done);
    stage->buf  = nullptr;
    stage->done = nullptr;
}

AcResult
acb_host::copy_field_range(cudaStream_t st, const Layout& L, state_t* field, size_t s,
                           AcReal* host, size_t count, bool h2d, lo16_t* lo_field,
                           StageBuf* stage)
{
    const size_t w     = sizeof(state_t);
    const size_t total = (size_t)L.mx * L.my * L.mz;
    if (s > total || count > total - s) {
        fprintf(stderr, "astaroth_b200: transfer range outside the mesh\n");
        return AC_FAILURE;
    }
    if (count == 0)
        return AC_SUCCESS;
    if (!stage || !stage->buf) {
        fprintf(stderr, "astaroth_b200: transfer without a staging buffer\n");
        return AC_FAILURE;
    }
    ACB_CUDA_CHECK(cudaStreamWaitEvent(st, stage->done, 0));
    for (size_t t = 0; t < count; t += stage->elems) {
        const size_t n   = std::min(stage->elems, count - t);
        const int blocks = (int)std::min<size_t>((n + 255) / 256, 4096);
        // cudaMemcpyDefault: the caller's mesh buffers are normally host
        // memory, but a device-resident mesh is copied the same way
        cudaError_t err;
        if (h2d) {
            err = cudaMemcpyAsync(stage->buf, host + t, n * w, cudaMemcpyDefault, st);
            if (err == cudaSuccess) {
                scatter_rows_kernel<<<blocks, 256, 0, st>>>(L, field, lo_field, stage->buf,
                                                            (unsigned long long)(s + t),
                                                            (unsigned long long)n);
                err = cudaGetLastError();
            }
        }
        else {
            gather_rows_kernel<<<blocks, 256, 0, st>>>(L, field, stage->buf,
                                                       (unsigned long long)(s + t),
                                                       (unsigned long long)n);
            err = cudaGetLastError();
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(host + t, stage->buf, n * w, cudaMemcpyDefault, st);
        }
        if (err != cudaSuccess) {
            fprintf(stderr, "astaroth_b200: transfer failed: %s\n", cudaGetErrorString(err));
            return AC_FAILURE;
        }
    }
    ACB_CUDA_CHECK(cudaEventRecord(stage->done, st));
    return AC_SUCCESS;
}

// flat (reference-order) double <-> padded field, for the double views and fills
__global__ void
pack_kernel(const Layout L, state_t* __restrict__ field, lo16_t* __restrict__ lo,
            double* __restrict__ flat, int to_flat, int fill, double value)
{
    const long long total = (long long)L.mx * L.my * L.mz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / L.mx;
        const int i         = (int)(t - row * L.mx);
        const long long e   = L.offx + row * L.mxp + i; // element index
        const long long id  = e * ACB_LANES;
        if (to_flat) {
            double v = (double)field[id];
            if (ACB_MIXED && lo)
                v += (double)lo16_to_float(lo[e * ACB_LO_STEP]);
            flat[t] = v;
        }
        else {
            const double v = fill ? value : flat[t];
            const state_t h = (state_t)v;
            field[id]       = h;
            if (ACB_MIXED && lo)
                lo[e * ACB_LO_STEP] = float_to_lo16((float)(v - (double)h));
        }
    }
}

static AcResult
launch_pack(const Device d, cudaStream_t st, int blk, int handle, double* flat, int to_flat,
            int fill, double value)
{
    const Layout& L = d->L;
    if (ensure_lo_ghosts(d, st, blk) != AC_SUCCESS)
        return AC_FAILURE;
    state_t* f      = d->blk[blk] + fidx(L, handle, 0);
    lo16_t* lo      = lo_field(d->lo[blk], L, handle);
    pack_kernel<<<d->num_sms * 8, 256, 0, st>>>(L, f, lo, flat, to_flat, fill, value);
    ACB_CUDA_CHECK(cudaGetLastError());
    d->launches++;
    if (!to_flat)
        d->write_epoch++;
    return AC_SUCCESS;
}

static AcResult
ensure_xfer(const Device d)
{
    const size_t need = (size_t)d->L.mx * d->L.my * d->L.mz;
    if (d->xfer && d->xfer_elems >= need)
        return AC_SUCCESS;
    if (d->xfer)
        cudaFree(d->xfer);
    d->xfer = nullptr;
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->xfer, need * sizeof(double)));
    d->xfer_elems = need;
    return AC_SUCCESS;
}

static void
invalidate_graphs(const Device d)
{
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < 2; ++p) {
            StepGraph& g = d->graph[k][p];
            if (g.exec)
                cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
            g.key  = 0;
        }
}

// Replays num_steps whole steps of one kind from CUDA graphs, one per
// starting buffer parity, capturing a graph (enqueue) when none matches the
// key; the Device's host-side block state follows what the captured step left.
template <class F>
static AcResult
replay_steps(const Device device, cudaStream_t st, int kind, unsigned long long base,
             double extra, int num_steps, F enqueue)
{
    for (int i = 0; i < num_steps; ++i) {
        const int p  = device->cur;
        StepGraph& G = device->graph[kind][p];
        // a captured step contains the ghost fill only when the ghosts were stale
        const unsigned long long key = base ^ (device->ghost_ok[p] ? 2ull : 0ull);
        if (!G.exec || G.key != key || G.extra != extra) {
            if (G.exec)
                cudaGraphExecDestroy(G.exec);
            G.exec = nullptr;
            cudaGraph_t g;
            ACB_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const unsigned long long before = device->launches;
            const AcResult rc               = enqueue(device, st);
            ACB_CUDA_CHECK(cudaStreamEndCapture(st, &g));
            device->cur = p; // capture advanced the roles; replay does it below
            G.launches  = device->launches - before;
            G.ghost[0]  = device->ghost_ok[0];
            G.ghost[1]  = device->ghost_ok[1];
            G.lo[0]     = device->lo_stale[0];
            G.lo[1]     = device->lo_stale[1];
            G.diag      = device->step_diag;
            device->launches = before;
            if (rc != AC_SUCCESS) {
                cudaGraphDestroy(g);
                return AC_FAILURE;
            }
            ACB_CUDA_CHECK(cudaGraphInstantiate(&G.exec, g, 0));
            cudaGraphDestroy(g);
            G.key   = key;
            G.extra = extra;
        }
        ACB_CUDA_CHECK(cudaGraphLaunch(G.exec, st));
        device->write_epoch++; // the replayed solves wrote both blocks
        device->launches += G.launches;
        device->ghost_ok[0] = G.ghost[0]; // as the captured step left them
        device->ghost_ok[1] = G.ghost[1];
        device->lo_stale[0] = G.lo[0];
        device->lo_stale[1] = G.lo[1];
        device->cur ^= 1; // three swaps per step
        if (G.diag) { // the replayed last substep folded the new block's diagnostics
            device->diag.valid   = true;
            device->diag.fetched = false;
            device->diag.block   = device->blk[device->cur];
            device->diag.epoch   = device->write_epoch;
        }
        else
            device->diag.valid = false;
    }
    return AC_SUCCESS;
}

// ---------------------------------------------------------------------------
// Time step chosen on the device
// ---------------------------------------------------------------------------
// The reference standalone's loop picks each step's dt on the host
// (samples/standalone/simulation.cc:429-436 with LSINK = LBFIELD = 0;
// model/host_timestep.cc:33-60): a synchronising max |u| reduction, then
//   uu_dt   = cdt dsmin / (|umax| + sqrt(cs2_sound))
//   visc_dt = cdtv dsmin^2 / max(max(nu, eta), max(gamma, chi = 0))
//   dt      = (AcReal)timescale * (AcReal)min(uu_dt, visc_dt)
// Here the same formula runs in one GPU thread on the max |u| that
// reduce3_kernel left in device memory, in double precision (the reference
// host code uses long double), with umax first rounded to AcReal as the
// reference's acReduceVec returns it. Nothing returns to the host, so a whole
// simulation step, time step included, is one CUDA graph.
struct CflParams {
    double cdt, cdtv, dsmin, cs2, nu, eta, gamma;
    AcReal timescale;
};

// rec: dt of the last step, simulated time, steps taken
static __global__ void
cfl_kernel(const double* umax, double* rec, const CflParams p)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    const double u       = (double)(AcReal)umax[0];
    const double uu_dt   = p.cdt * p.dsmin / (fabs(u) + sqrt(p.cs2));
    const double visc_dt = p.cdtv * p.dsmin * p.dsmin / fmax(fmax(p.nu, p.eta), fmax(p.gamma, 0.0));
    const AcReal dt      = p.timescale * (AcReal)fmin(uu_dt, visc_dt);
    rec[0]               = (double)dt;
    rec[1] += (double)dt;
    rec[2] += 1.0;
}

// The formula's parameters from the uniform mirror. AC_dsmin as the
// standalone's config loader sets it (min of AC_dsx, AC_dsy, AC_dsz) where the
// caller left it unset; AC_cdt and AC_cdtv must be positive.
static AcResult
cfl_params(const Device d, AcReal timescale, CflParams& cp)
{
    const AcReal* rp = d->uniforms.real_params;
    cp.cdt           = rp[AC_cdt];
    cp.cdtv          = rp[AC_cdtv];
    cp.dsmin         = rp[AC_dsmin] > 0
                           ? (double)rp[AC_dsmin]
                           : (double)std::min(rp[AC_dsx], std::min(rp[AC_dsy], rp[AC_dsz]));
    cp.cs2           = rp[AC_cs2_sound];
    cp.nu            = rp[AC_nu_visc];
    cp.eta           = rp[AC_eta];
    cp.gamma         = rp[AC_gamma];
    cp.timescale     = timescale;
    if (!(cp.cdt > 0) || !(cp.cdtv > 0) || !(cp.dsmin > 0) || !(timescale > 0)) {
        fprintf(stderr, "astaroth_b200: a time step chosen on the device needs AC_cdt, AC_cdtv, "
                        "the grid spacings and the time scale positive\n");
        return AC_FAILURE;
    }
    if (d->forcing) {
        fprintf(stderr, "astaroth_b200: forcing scales with sqrt(dt) on the host; it does not "
                        "combine with a time step chosen on the device\n");
        return AC_FAILURE;
    }
    return AC_SUCCESS;
}

// max |u| into d->red_result, the time step into d->cfl, then the three
// substeps reading it: 3 x (ghost fill, solve, swap).
static AcResult
enqueue_step_cfl(const Device d, cudaStream_t st, const CflParams& cp)
{
    const int hu[3] = {VTXBUF_UUX, VTXBUF_UUY, VTXBUF_UUZ};
    ReduceArgs a;
    long long blocks;
    if (reduce_args(d, RTYPE_MAX, RED_VEC, hu, a, blocks) != AC_SUCCESS)
        return AC_FAILURE;
    reduce3_kernel<256><<<(unsigned)blocks, 256, 0, st>>>(a);
    ACB_CUDA_CHECK(cudaGetLastError());
    cfl_kernel<<<1, 32, 0, st>>>(d->red_result, d->cfl, cp);
    ACB_CUDA_CHECK(cudaGetLastError());
    d->launches += 2;
    const int3 m0 = make_int3(0, 0, 0);
    const int3 m1 = make_int3(d->L.mx, d->L.my, d->L.mz);
    const int3 n0 = make_int3(NGHOST, NGHOST, NGHOST);
    const int3 n1 = make_int3(NGHOST + d->L.nx, NGHOST + d->L.ny, NGHOST + d->L.nz);
    for (int s = 0; s < 3; ++s) {
        if (launch_halo(d, st, m0, m1, 0, NUM_VTXBUF_HANDLES) != AC_SUCCESS)
            return AC_FAILURE;
        if (launch_solve(d, st, s, n0, n1, d->cfl) != AC_SUCCESS)
            return AC_FAILURE;
        d->cur ^= 1;
    }
    return AC_SUCCESS;
}

// ---------------------------------------------------------------------------
// Interface
// ---------------------------------------------------------------------------
extern "C" {

AcResult
acDevicePrintInfo(const Device device)
{
    cudaDeviceProp p;
    ACB_CUDA_CHECK(cudaGetDeviceProperties(&p, device->id));
    size_t free_b = 0, total_b = 0;
    cudaSetDevice(device->id);
    cudaMemGetInfo(&free_b, &total_b);
    int n;
    const SolveConfig* cfgs = solve_configs(&n);
    printf("--------------------------------------------------\n");
    printf("Device Number: %d\n", device->id);
    printf("    Device name: %s\n", p.name);
    printf("    Compute capability: %d.%d\n", p.major, p.minor);
    printf("    Multiprocessors: %d\n", p.multiProcessorCount);
    printf("    Global memory: %.2f GiB (%.2f GiB free)\n", total_b / 1073741824.0,
           free_b / 1073741824.0);
    printf("    L2 size: %d KiB\n", p.l2CacheSize / 1024);
    printf("    Shared memory per block (opt-in): %zu KiB\n", p.sharedMemPerBlockOptin / 1024);
    printf("  Mesh %d x %d x %d, row pitch %d, %s state\n", device->L.nx, device->L.ny,
           device->L.nz, device->L.mxp,
           ACB_MIXED ? "mixed (float hi, bfloat16 lo)" : (sizeof(AcReal) == 8 ? "double" : "float"));
    printf("  Solve configuration: %s\n", cfgs[device->solve_cfg].name);
    printf("--------------------------------------------------\n");
    return AC_SUCCESS;
}

AcResult
acDeviceSynchronizeStream(const Device device, const Stream stream)
{
    cudaSetDevice(device->id);
    if (stream == STREAM_ALL) {
        ACB_CUDA_CHECK(cudaDeviceSynchronize());
        unsigned st = 0;
        ACB_CUDA_CHECK(cudaMemcpy(&st, device->status, sizeof(st), cudaMemcpyDeviceToHost));
        if (st) {
            fprintf(stderr, "astaroth_b200: device %d status 0x%x (a kernel gave up waiting)\n",
                    device->id, st);
            return AC_FAILURE;
        }
    }
    else {
        ACB_CUDA_CHECK(cudaStreamSynchronize(stream_of(device, stream)));
    }
    return AC_SUCCESS;
}

AcResult
acDeviceLoadScalarUniform(const Device device, const Stream stream, const AcRealParam param,
                          const AcReal value)
{
    (void)stream;
    if (param < 0 || param >= NUM_REAL_PARAMS) {
        fprintf(stderr, "WARNING: invalid AcRealParam %d.\n", param);
        return AC_FAILURE;
    }
    if (!real_is_valid((double)value)) {
        fprintf(stderr, "WARNING: Passed an invalid value %g to device constant %s. Skipping.\n",
                (double)value, realparam_names[param]);
        return AC_FAILURE;
    }
    if (device->uniforms.real_params[param] != value) {
        device->uniforms.real_params[param] = value;
        device->uniform_version++;
    }
    return AC_SUCCESS;
}

AcResult
acDeviceLoadVectorUniform(const Device device, const Stream stream, const AcReal3Param param,
                          const AcReal3 value)
{
    (void)device;
    (void)stream;
    (void)value;
    // the module declares no vector uniforms (NUM_REAL3_PARAMS == 0)
    fprintf(stderr, "WARNING: invalid AcReal3Param %d\n", (int)param);
    return AC_FAILURE;
}

AcResult
acDeviceLoadIntUniform(const Device device, const Stream stream, const AcIntParam param,
                       const int value)
{
    (void)stream;
    if (param < 0 || param >= NUM_INT_PARAMS) {
        fprintf(stderr, "WARNING: invalid AcIntParam %d\n", param);
        return AC_FAILURE;
    }
    device->uniforms.int_params[param] = value;
    device->uniform_version++;
    return AC_SUCCESS;
}

AcResult
acDeviceLoadInt3Uniform(const Device device, const Stream stream, const AcInt3Param param,
                        const int3 value)
{
    (void)stream;
    if (param < 0 || param >= NUM_INT3_PARAMS) {
        fprintf(stderr, "WARNING: invalid AcInt3Param %d\n", param);
        return AC_FAILURE;
    }
    device->uniforms.int3_params[param] = value;
    device->uniform_version++;
    return AC_SUCCESS;
}

AcResult
acDeviceLoadScalarArray(const Device device, const Stream stream, const ScalarArrayHandle handle,
                        const size_t start, const AcReal* data, const size_t num)
{
    (void)device;
    (void)stream;
    (void)handle;
    (void)start;
    (void)data;
    (void)num;
    return AC_FAILURE; // the module declares no scalar arrays
}

AcResult
acDeviceLoadMeshInfo(const Device device, const AcMeshInfo config)
{
    const int* a = config.int_params;
    const int* b = device->local_config.int_params;
    if (a[AC_nx] != b[AC_nx] || a[AC_ny] != b[AC_ny] || a[AC_nz] != b[AC_nz] ||
        config.int3_params[AC_multigpu_offset].x !=
            device->local_config.int3_params[AC_multigpu_offset].x ||
        config.int3_params[AC_multigpu_offset].y !=
            device->local_config.int3_params[AC_multigpu_offset].y ||
        config.int3_params[AC_multigpu_offset].z !=
            device->local_config.int3_params[AC_multigpu_offset].z) {
        fprintf(stderr, "astaroth_b200: acDeviceLoadMeshInfo with other dimensions\n");
        return AC_FAILURE;
    }
    for (int i = 0; i < NUM_INT_PARAMS; ++i)
        acDeviceLoadIntUniform(device, STREAM_DEFAULT, (AcIntParam)i, config.int_params[i]);
    for (int i = 0; i < NUM_INT3_PARAMS; ++i)
        acDeviceLoadInt3Uniform(device, STREAM_DEFAULT, (AcInt3Param)i, config.int3_params[i]);
    for (int i = 0; i < NUM_REAL_PARAMS; ++i)
        if (real_is_valid((double)config.real_params[i]))
            acDeviceLoadScalarUniform(device, STREAM_DEFAULT, (AcRealParam)i,
                                      config.real_params[i]);
    return AC_SUCCESS;
}

AcResult
acDeviceLoadDefaultUniforms(const Device device)
{
    // Defaults of the module's uniforms: zero unless the module gives a value
    // (acc/stdlib/stdderiv.h:6-11, acc/mhd_solver/stencil_kernel.ac:69,112).
    memset(&device->uniforms, 0, sizeof(device->uniforms));
    AcReal* rp          = device->uniforms.real_params;
    const AcReal ds     = (AcReal)0.04908738521;
    rp[AC_dsx]          = ds;
    rp[AC_dsy]          = ds;
    rp[AC_dsz]          = ds;
    rp[AC_inv_dsx]      = (AcReal)1.0 / ds;
    rp[AC_inv_dsy]      = (AcReal)1.0 / ds;
    rp[AC_inv_dsz]      = (AcReal)1.0 / ds;
    rp[AC_cs_sound]     = (AcReal)1.0;
    rp[AC_cs2_sound]    = rp[AC_cs_sound] * rp[AC_cs_sound];
    device->uniform_version++;
    return AC_SUCCESS;
}

AcResult
acDeviceCreate(const int id, const AcMeshInfo config, Device* device_handle)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || id < 0 || id >= ndev) {
        fprintf(stderr, "astaroth_b200: no CUDA device %d\n", id);
        return AC_FAILURE;
    }
    const int nx = config.int_params[AC_nx], ny = config.int_params[AC_ny],
              nz = config.int_params[AC_nz];
    if (nx < NGHOST || ny < NGHOST || nz < NGHOST) {
        fprintf(stderr, "astaroth_b200: mesh %d x %d x %d too small\n", nx, ny, nz);
        return AC_FAILURE;
    }
    ACB_CUDA_CHECK(cudaSetDevice(id));
    struct device_s* d = (struct device_s*)calloc(1, sizeof(struct device_s));
    if (!d)
        return AC_FAILURE;
    d->id           = id;
    d->local_config = config;
    d->tmap_cfg     = -1;
    d->solve_cfg    = kDefaultSolveConfig;
    ACB_CUDA_CHECK(cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, id));

    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    for (int i = 0; i < NUM_STREAMS; ++i) {
        int prio = prio_lo - i; // stream 0 lowest priority, as the reference's 0..31 clamped
        if (prio < prio_hi)
            prio = prio_hi;
        ACB_CUDA_CHECK(cudaStreamCreateWithPriority(&d->streams[i], cudaStreamNonBlocking, prio));
    }

    d->L               = make_layout(nx, ny, nz);
    const size_t bytes = block_bytes(d->L);
    for (int b = 0; b < 2; ++b) {
        ACB_CUDA_CHECK(cudaMalloc((void**)&d->blk[b], bytes));
        ACB_CUDA_CHECK(cudaMemset(d->blk[b], 0, bytes));
#if ACB_MIXED
        ACB_CUDA_CHECK(cudaMalloc((void**)&d->lo[b], lo_block_bytes(d->L)));
        ACB_CUDA_CHECK(cudaMemset(d->lo[b], 0, lo_block_bytes(d->L)));
#endif
    }
    d->red_max_blocks = d->num_sms * 8;
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->red_partials,
                              3 * ACB_RED_SETS * sizeof(double) * d->red_max_blocks));
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->red_counter, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMemset(d->red_counter, 0, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->red_result, 3 * ACB_RED_SETS * sizeof(double)));
    ACB_CUDA_CHECK(cudaMallocHost((void**)&d->h_result, 3 * ACB_RED_SETS * sizeof(double)));
    d->diag_max_ctas = d->num_sms * 8;
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->diag_partials, 4 * sizeof(double) * d->diag_max_ctas));
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->diag_counter, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMemset(d->diag_counter, 0, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->diag_result, 4 * sizeof(double)));
    ACB_CUDA_CHECK(cudaMallocHost((void**)&d->h_diag, 4 * sizeof(double)));
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->status, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMemset(d->status, 0, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMalloc((void**)&d->cfl, 3 * sizeof(double)));
    ACB_CUDA_CHECK(cudaMemset(d->cfl, 0, 3 * sizeof(double)));
    if (stage_create(&d->stage, (size_t)d->L.mx * d->L.my * d->L.mz) != AC_SUCCESS)
        return AC_FAILURE;

    acDeviceLoadDefaultUniforms(d);
    acDeviceLoadMeshInfo(d, config);
    if (prepare_kernels_once() != AC_SUCCESS)
        return AC_FAILURE;
    ACB_CUDA_CHECK(cudaDeviceSynchronize());
    *device_handle = d;
    // The tile configuration is not timed here, unlike device.cc:175-176: on
    // the zeros a new Device holds, the GPU draws less power and runs at higher
    // clocks than on a real state, and under the power cap the ranking of the
    // configurations changes (512^3 mixed: 64x4 tiles fastest on zeros, 32x8
    // tiles 1.2 % faster on the seeded workload). The default is the
    // configuration fastest on real states; acDeviceAutoOptimize times the
    // configurations on the Device's current state.
    return AC_SUCCESS;
}

AcResult
acDeviceDestroy(Device device)
{
    if (!device)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    cudaDeviceSynchronize();
    invalidate_graphs(device);
    for (int b = 0; b < 2; ++b) {
        cudaFree(device->blk[b]);
        if (device->lo[b])
            cudaFree(device->lo[b]);
    }
    cudaFree(device->red_partials);
    cudaFree(device->red_counter);
    cudaFree(device->red_result);
    cudaFreeHost(device->h_result);
    cudaFree(device->diag_partials);
    cudaFree(device->diag_counter);
    cudaFree(device->diag_result);
    cudaFreeHost(device->h_diag);
    cudaFree(device->status);
    cudaFree(device->cfl);
    if (device->xfer)
        cudaFree(device->xfer);
    stage_destroy(&device->stage);
    for (int i = 0; i < NUM_STREAMS; ++i)
        cudaStreamDestroy(device->streams[i]);
    free(device);
    return AC_SUCCESS;
}

AcResult
acDeviceAutoOptimize(const Device device)
{
    // Times every compiled tile configuration on one full-domain substep (s = 1)
    // and keeps the fastest; the buffers are restored afterwards.
    cudaSetDevice(device->id);
    int n;
    solve_configs(&n);
    const cudaStream_t st = device->streams[STREAM_DEFAULT];
    const int3 s          = make_int3(NGHOST, NGHOST, NGHOST);
    const int3 e = make_int3(NGHOST + device->L.nx, NGHOST + device->L.ny, NGHOST + device->L.nz);
    // keep the out block (the substep overwrites it)
    const size_t bytes = block_bytes(device->L);
    state_t* save      = nullptr;
    ACB_CUDA_CHECK(cudaMalloc((void**)&save, bytes));
    ACB_CUDA_CHECK(cudaMemcpyAsync(save, device->blk[device->cur ^ 1], bytes,
                                   cudaMemcpyDeviceToDevice, st));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    const int saved_cfg = device->solve_cfg;
    int best            = saved_cfg;
    float best_ms       = INFINITY;
    for (int c = 0; c < n; ++c) {
        device->solve_cfg = c;
        if (launch_solve(device, st, 1, s, e) != AC_SUCCESS) // warm-up
            continue;
        cudaEventRecord(t0, st);
        const int reps = 3;
        for (int r = 0; r < reps; ++r)
            launch_solve(device, st, 1, s, e);
        cudaEventRecord(t1, st);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        if (cudaGetLastError() == cudaSuccess && ms < best_ms) {
            best_ms = ms;
            best    = c;
        }
    }
    device->solve_cfg = best;
    device->write_epoch++;
    ACB_CUDA_CHECK(cudaMemcpyAsync(device->blk[device->cur ^ 1], save, bytes,
                                   cudaMemcpyDeviceToDevice, st));
    device->ghost_ok[device->cur ^ 1] = false;
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    cudaFree(save);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    invalidate_graphs(device);
    (void)saved_cfg;
    return AC_SUCCESS;
}

AcResult
acDeviceSwapBuffers(const Device device)
{
    device->cur ^= 1;
    return AC_SUCCESS;
}

AcResult
acDeviceLoadVertexBufferWithOffset(const Device device, const Stream stream,
                                   const AcMesh host_mesh, const VertexBufferHandle h,
                                   const int3 src, const int3 dst, const int num_vertices)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES || num_vertices < 0)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    const size_t sidx = acVertexBufferIdx(src.x, src.y, src.z, host_mesh.info);
    const size_t didx = acVertexBufferIdx(dst.x, dst.y, dst.z, device->local_config);
    const Layout& L   = device->L;
    lo16_t* lo        = lo_field(device->lo[device->cur], L, h);
    device->ghost_ok[device->cur] = false;
    device->write_epoch++;
    if (ensure_lo_ghosts(device, stream_of(device, stream), device->cur) != AC_SUCCESS)
        return AC_FAILURE;
    return copy_field_range(stream_of(device, stream), L,
                            device->blk[device->cur] + fidx(L, h, 0), didx,
                            host_mesh.vertex_buffer[h] + sidx, (size_t)num_vertices, true, lo,
                            &device->stage);
}

AcResult
acDeviceLoadMeshWithOffset(const Device device, const Stream stream, const AcMesh host_mesh,
                           const int3 src, const int3 dst, const int num_vertices)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceLoadVertexBufferWithOffset(device, stream, host_mesh, (VertexBufferHandle)i,
                                               src, dst, num_vertices) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acDeviceLoadVertexBuffer(const Device device, const Stream stream, const AcMesh host_mesh,
                         const VertexBufferHandle h)
{
    const int3 z = make_int3(0, 0, 0);
    return acDeviceLoadVertexBufferWithOffset(device, stream, host_mesh, h, z, z,
                                              (int)acVertexBufferSize(device->local_config));
}

AcResult
acDeviceLoadMesh(const Device device, const Stream stream, const AcMesh host_mesh)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceLoadVertexBuffer(device, stream, host_mesh, (VertexBufferHandle)i) !=
            AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acDeviceSetVertexBuffer(const Device device, const Stream stream, const VertexBufferHandle h,
                        const AcReal value)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    const cudaStream_t st = stream_of(device, stream);
    // both in and out, as the reference does (src/core/device.cc:296-314)
    device->ghost_ok[0] = device->ghost_ok[1] = false;
    for (int b = 0; b < 2; ++b)
        if (launch_pack(device, st, b, h, nullptr, 0, 1, (double)value) != AC_SUCCESS)
            return AC_FAILURE;
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    return AC_SUCCESS;
}

AcResult
acDeviceStoreVertexBufferWithOffset(const Device device, const Stream stream,
                                    const VertexBufferHandle h, const int3 src, const int3 dst,
                                    const int num_vertices, AcMesh* host_mesh)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES || num_vertices < 0)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    const size_t sidx = acVertexBufferIdx(src.x, src.y, src.z, device->local_config);
    const size_t didx = acVertexBufferIdx(dst.x, dst.y, dst.z, host_mesh->info);
    const Layout& L   = device->L;
    return copy_field_range(stream_of(device, stream), L,
                            device->blk[device->cur] + fidx(L, h, 0), sidx,
                            host_mesh->vertex_buffer[h] + didx, (size_t)num_vertices, false,
                            nullptr, &device->stage);
}

AcResult
acDeviceStoreMeshWithOffset(const Device device, const Stream stream, const int3 src,
                            const int3 dst, const int num_vertices, AcMesh* host_mesh)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceStoreVertexBufferWithOffset(device, stream, (VertexBufferHandle)i, src, dst,
                                                num_vertices, host_mesh) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acDeviceStoreVertexBuffer(const Device device, const Stream stream, const VertexBufferHandle h,
                          AcMesh* host_mesh)
{
    const int3 z = make_int3(0, 0, 0);
    return acDeviceStoreVertexBufferWithOffset(device, stream, h, z, z,
                                               (int)acVertexBufferSize(device->local_config),
                                               host_mesh);
}

AcResult
acDeviceStoreMesh(const Device device, const Stream stream, AcMesh* host_mesh)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceStoreVertexBuffer(device, stream, (VertexBufferHandle)i, host_mesh) !=
            AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

// device-to-device flat-range copy between two padded layouts
__global__ void
transfer_kernel(const Layout Ls, const state_t* __restrict__ src, const lo16_t* __restrict__ slo,
                long long s0, const Layout Ld, state_t* __restrict__ dst, lo16_t* __restrict__ dlo,
                long long d0, long long count)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const long long a = s0 + t, b = d0 + t;
        const long long ra = a / Ls.mx, rb = b / Ld.mx;
        const long long ea = Ls.offx + ra * Ls.mxp + (a - ra * Ls.mx); // element indices
        const long long eb = Ld.offx + rb * Ld.mxp + (b - rb * Ld.mx);
        dst[eb * ACB_LANES] = src[ea * ACB_LANES];
        if (ACB_MIXED && dlo) // the (hi, lo) pair moves whole
            dlo[eb * ACB_LO_STEP] = slo ? slo[ea * ACB_LO_STEP] : (lo16_t)0;
    }
}

AcResult
acDeviceTransferVertexBufferWithOffset(const Device src_device, const Stream stream,
                                       const VertexBufferHandle h, const int3 src,
                                       const int3 dst, const int num_vertices, Device dst_device)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES || num_vertices < 0)
        return AC_FAILURE;
    const size_t sidx = acVertexBufferIdx(src.x, src.y, src.z, src_device->local_config);
    const size_t didx = acVertexBufferIdx(dst.x, dst.y, dst.z, dst_device->local_config);
    const size_t st   = acVertexBufferSize(src_device->local_config);
    const size_t dt   = acVertexBufferSize(dst_device->local_config);
    if (sidx + num_vertices > st || didx + num_vertices > dt)
        return AC_FAILURE;
    if (src_device->id != dst_device->id) {
        fprintf(stderr, "astaroth_b200: transfers between GPUs are not supported\n");
        return AC_FAILURE;
    }
    cudaSetDevice(src_device->id);
    dst_device->ghost_ok[dst_device->cur] = false;
    dst_device->write_epoch++;
    const cudaStream_t tst = stream_of(src_device, stream);
    if (ensure_lo_ghosts(src_device, tst, src_device->cur) != AC_SUCCESS ||
        ensure_lo_ghosts(dst_device, tst, dst_device->cur) != AC_SUCCESS)
        return AC_FAILURE;
    const lo16_t* slo = lo_field(src_device->lo[src_device->cur], src_device->L, h);
    lo16_t* dlo       = lo_field(dst_device->lo[dst_device->cur], dst_device->L, h);
    transfer_kernel<<<src_device->num_sms * 4, 256, 0, tst>>>(
        src_device->L, src_device->blk[src_device->cur] + fidx(src_device->L, h, 0), slo,
        (long long)sidx, dst_device->L, dst_device->blk[dst_device->cur] + fidx(dst_device->L, h, 0),
        dlo, (long long)didx, (long long)num_vertices);
    ACB_CUDA_CHECK(cudaGetLastError());
    src_device->launches++;
    return AC_SUCCESS;
}

AcResult
acDeviceTransferMeshWithOffset(const Device src_device, const Stream stream, const int3 src,
                               const int3 dst, const int num_vertices, Device* dst_device)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceTransferVertexBufferWithOffset(src_device, stream, (VertexBufferHandle)i, src,
                                                   dst, num_vertices, *dst_device) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acDeviceTransferVertexBuffer(const Device src_device, const Stream stream,
                             const VertexBufferHandle h, Device dst_device)
{
    const int3 z = make_int3(0, 0, 0);
    return acDeviceTransferVertexBufferWithOffset(src_device, stream, h, z, z,
                                                  (int)acVertexBufferSize(src_device->local_config),
                                                  dst_device);
}

AcResult
acDeviceTransferMesh(const Device src_device, const Stream stream, Device dst_device)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceTransferVertexBuffer(src_device, stream, (VertexBufferHandle)i, dst_device) !=
            AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acDeviceIntegrateSubstep(const Device device, const Stream stream, const int step_number,
                         const int3 start, const int3 end, const AcReal dt)
{
    cudaSetDevice(device->id);
    if (acDeviceLoadScalarUniform(device, stream, AC_dt, dt) != AC_SUCCESS)
        return AC_FAILURE;
    return launch_solve(device, stream_of(device, stream), step_number, start, end);
}

AcResult
acDevicePeriodicBoundcondStep(const Device device, const Stream stream,
                              const VertexBufferHandle h, const int3 start, const int3 end)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    return launch_halo(device, stream_of(device, stream), start, end, (int)h, (int)h + 1);
}

AcResult
acDevicePeriodicBoundconds(const Device device, const Stream stream, const int3 start,
                           const int3 end)
{
    cudaSetDevice(device->id);
    return launch_halo(device, stream_of(device, stream), start, end, 0, NUM_VTXBUF_HANDLES);
}

AcResult
acDeviceGeneralBoundcondStep(const Device device, const Stream stream,
                             const VertexBufferHandle h, const int3 start, const int3 end,
                             const AcMeshInfo config, const int3 bindex)
{
    (void)bindex; // the reference mirrors only for bindex.x < 0, which its Node always passes
    // As the reference (src/core/kernels/boundconds.cuh:192-242), the x-top
    // condition selects the fill of every face.
    const int bc = config.int_params[AC_bc_type_top_x];
    if (bc == AC_BOUNDCOND_PERIODIC)
        return acDevicePeriodicBoundcondStep(device, stream, h, start, end);
    if (bc != AC_BOUNDCOND_SYMMETRIC && bc != AC_BOUNDCOND_ANTISYMMETRIC) {
        fprintf(stderr, "ERROR: Boundary condition not recognized! (%d)\n", bc);
        return AC_FAILURE;
    }
    if (h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    const Layout& L = device->L;
    if (L.nx < NGHOST + 1 || L.ny < NGHOST + 1 || L.nz < NGHOST + 1) {
        fprintf(stderr, "astaroth_b200: symmetric boundaries need n >= 4 on every axis\n");
        return AC_FAILURE;
    }
    int3 s = start, e = end;
    s.x = std::max(s.x, 0);
    s.y = std::max(s.y, 0);
    s.z = std::max(s.z, 0);
    e.x = std::min(e.x, L.mx);
    e.y = std::min(e.y, L.my);
    e.z = std::min(e.z, L.mz);
    if (e.x <= s.x || e.y <= s.y || e.z <= s.z)
        return AC_SUCCESS;
    if (ensure_lo_ghosts(device, stream_of(device, stream), device->cur) != AC_SUCCESS)
        return AC_FAILURE;
    HaloArgs a;
    a.L     = L;
    a.block = device->blk[device->cur];
    a.lo    = device->lo[device->cur];
    a.start = s;
    a.end   = e;
    a.f0    = (int)h;
    a.f1    = (int)h + 1;
    a.rows  = (long long)(e.y - s.y) * (e.z - s.z);
    const long long blocks = std::min((a.rows + 7) / 8, (long long)device->num_sms * 16);
    mirror_kernel<<<(unsigned)blocks, 256, 0, stream_of(device, stream)>>>(
        a, bc == AC_BOUNDCOND_SYMMETRIC ? 1.0f : -1.0f);
    ACB_CUDA_CHECK(cudaGetLastError());
    device->launches++;
    device->ghost_ok[device->cur] = false; // no longer the periodic images
    return AC_SUCCESS;
}

AcResult
acDeviceGeneralBoundconds(const Device device, const Stream stream, const int3 start,
                          const int3 end, const AcMeshInfo config, const int3 bindex)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acDeviceGeneralBoundcondStep(device, stream, (VertexBufferHandle)i, start, end, config,
                                         bindex) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

static bool
rtype_ok(int rtype, int nin)
{
    if (nin == RED_ALFVEN)
        return rtype == RTYPE_ALFVEN_MAX || rtype == RTYPE_ALFVEN_MIN || rtype == RTYPE_ALFVEN_RMS;
    return rtype == RTYPE_MAX || rtype == RTYPE_MIN || rtype == RTYPE_RMS ||
           rtype == RTYPE_RMS_EXP || rtype == RTYPE_SUM;
}

AcResult
acDeviceReduceScalDouble(const Device device, const Stream stream, const ReductionType rtype,
                         const VertexBufferHandle h, double* result)
{
    if (!rtype_ok(rtype, RED_SCAL)) {
        fprintf(stderr, "astaroth_b200: unsupported reduction type %d\n", (int)rtype);
        *result = NAN;
        return AC_FAILURE;
    }
    cudaSetDevice(device->id);
    const int hs[1] = {(int)h};
    return run_reduce(device, stream_of(device, stream), rtype, RED_SCAL, hs, result);
}

AcResult
acDeviceReduceVecDouble(const Device device, const Stream stream, const ReductionType rtype,
                        const VertexBufferHandle a, const VertexBufferHandle b,
                        const VertexBufferHandle c, double* result)
{
    if (!rtype_ok(rtype, RED_VEC)) {
        fprintf(stderr, "astaroth_b200: unsupported reduction type %d\n", (int)rtype);
        *result = NAN;
        return AC_FAILURE;
    }
    cudaSetDevice(device->id);
    const int hs[3] = {(int)a, (int)b, (int)c};
    return run_reduce(device, stream_of(device, stream), rtype, RED_VEC, hs, result);
}

AcResult
acDeviceReduceScal(const Device device, const Stream stream, const ReductionType rtype,
                   const VertexBufferHandle h, AcReal* result)
{
    double r      = NAN;
    AcResult rc   = acDeviceReduceScalDouble(device, stream, rtype, h, &r);
    *result       = (AcReal)r;
    return rc;
}

AcResult
acDeviceReduceVec(const Device device, const Stream stream, const ReductionType rtype,
                  const VertexBufferHandle a, const VertexBufferHandle b,
                  const VertexBufferHandle c, AcReal* result)
{
    double r    = NAN;
    AcResult rc = acDeviceReduceVecDouble(device, stream, rtype, a, b, c, &r);
    *result     = (AcReal)r;
    return rc;
}

AcResult
acDeviceReduceVecScal(const Device device, const Stream stream, const ReductionType rtype,
                      const VertexBufferHandle a, const VertexBufferHandle b,
                      const VertexBufferHandle c, const VertexBufferHandle d, AcReal* result)
{
    if (!rtype_ok(rtype, RED_ALFVEN)) {
        fprintf(stderr, "astaroth_b200: unsupported reduction type %d\n", (int)rtype);
        *result = (AcReal)NAN;
        return AC_FAILURE;
    }
    cudaSetDevice(device->id);
    const int hs[4] = {(int)a, (int)b, (int)c, (int)d};
    double r        = NAN;
    AcResult rc     = run_reduce(device, stream_of(device, stream), rtype, RED_ALFVEN, hs, &r);
    *result         = (AcReal)r;
    return rc;
}

AcResult
acDeviceRunMPITest(void)
{
    fprintf(stderr, "astaroth_b200: acDeviceRunMPITest: no MPI layer in this build\n");
    return AC_FAILURE;
}

// ---------------------------------------------------------------------------
// additions (include/astaroth_b200.h)
// ---------------------------------------------------------------------------
AcResult
acDeviceGetStatus(const Device device, unsigned* status)
{
    cudaSetDevice(device->id);
    ACB_CUDA_CHECK(cudaDeviceSynchronize());
    ACB_CUDA_CHECK(cudaMemcpy(status, device->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return AC_SUCCESS;
}

AcResult
acDeviceResetStatus(const Device device)
{
    cudaSetDevice(device->id);
    ACB_CUDA_CHECK(cudaDeviceSynchronize());
    ACB_CUDA_CHECK(cudaMemset(device->status, 0, sizeof(unsigned)));
    return AC_SUCCESS;
}

// One warp waits, with the pipelines' bounded wait and a limit of limit_ns,
// on phase 0 of an mbarrier that expects one arrival and gets none; when the
// wait gives up, the warp raises the status bit a pipeline kernel raises and
// the kernel returns.
__global__ void
wait_check_kernel(unsigned* status, unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncwarp();
    const bool ok = mbar_wait_limit(&bar, 0u, limit_ns);
    if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0)
        atomicOr(status, (unsigned)ACB_STATUS_TMA_TIMEOUT);
}

AcResult
acDeviceCheckWaitLimit(const Device device, const double seconds)
{
    if (!(seconds > 0.0 && seconds <= 10.0))
        return AC_FAILURE;
    cudaSetDevice(device->id);
    const cudaStream_t st = device->streams[STREAM_DEFAULT];
    wait_check_kernel<<<1, 32, 0, st>>>(device->status, (unsigned long long)(seconds * 1e9));
    ACB_CUDA_CHECK(cudaGetLastError());
    device->launches++;
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    unsigned s = 0;
    ACB_CUDA_CHECK(cudaMemcpy(&s, device->status, sizeof(s), cudaMemcpyDeviceToHost));
    return (s & ACB_STATUS_TMA_TIMEOUT) ? AC_SUCCESS : AC_FAILURE;
}

AcResult
acDeviceGetCudaStream(const Device device, const Stream stream, void** cuda_stream)
{
    *cuda_stream = (void*)stream_of(device, stream);
    return AC_SUCCESS;
}

AcResult
acDeviceGetLaunchCount(const Device device, unsigned long long* count)
{
    *count = device->launches;
    return AC_SUCCESS;
}

AcResult
acDeviceSetSolveConfig(const Device device, const int config)
{
    int n;
    solve_configs(&n);
    const int c = config < 0 ? kDefaultSolveConfig : config;
    if (c >= n)
        return AC_FAILURE;
    if (device->solve_cfg != c) {
        device->solve_cfg = c;
        invalidate_graphs(device);
    }
    return AC_SUCCESS;
}

AcResult
acDeviceGetSolveConfig(const Device device, int* config, int* num_configs)
{
    solve_configs(num_configs);
    *config = device->solve_cfg;
    return AC_SUCCESS;
}

const char*
acSolveConfigName(const int config)
{
    int n;
    const SolveConfig* cfgs = solve_configs(&n);
    return (config >= 0 && config < n) ? cfgs[config].name : "invalid";
}

AcResult
acDeviceGetMemoryFootprint(const Device device, size_t* bytes)
{
    size_t b = 2 * block_bytes(device->L);
    if (device->lo[0])
        b += 2 * lo_block_bytes(device->L);
    *bytes = b;
    return AC_SUCCESS;
}

AcResult
acDeviceSetStepDiagnostics(const Device device, const int enabled)
{
    device->step_diag = enabled != 0;
    device->diag.valid = false;
    device->uniform_version++; // whole-step graphs are captured again
    return AC_SUCCESS;
}

AcResult
acDeviceSetForcing(const Device device, const int enabled)
{
    device->forcing = enabled ? 1 : 0;
    device->uniform_version++;
    return AC_SUCCESS;
}

AcResult
acDeviceLoadForcingParams(const Device device, const Stream stream, const AcForcingParams params)
{
    const struct {
        AcRealParam param;
        AcReal value;
    } v[] = {
        {AC_forcing_magnitude, params.magnitude}, {AC_forcing_phase, params.phase},
        {AC_k_forcex, params.k_force[0]},         {AC_k_forcey, params.k_force[1]},
        {AC_k_forcez, params.k_force[2]},         {AC_ff_hel_rex, params.ff_hel_re[0]},
        {AC_ff_hel_rey, params.ff_hel_re[1]},     {AC_ff_hel_rez, params.ff_hel_re[2]},
        {AC_ff_hel_imx, params.ff_hel_im[0]},     {AC_ff_hel_imy, params.ff_hel_im[1]},
        {AC_ff_hel_imz, params.ff_hel_im[2]},     {AC_kaver, params.kaver},
    };
    AcResult rc = AC_SUCCESS;
    for (const auto& e : v)
        if (acDeviceLoadScalarUniform(device, stream, e.param, e.value) != AC_SUCCESS)
            rc = AC_FAILURE;
    return rc;
}

static AcResult
enqueue_step(const Device d, cudaStream_t st)
{
    const int3 m0 = make_int3(0, 0, 0);
    const int3 m1 = make_int3(d->L.mx, d->L.my, d->L.mz);
    const int3 n0 = make_int3(NGHOST, NGHOST, NGHOST);
    const int3 n1 = make_int3(NGHOST + d->L.nx, NGHOST + d->L.ny, NGHOST + d->L.nz);
    for (int s = 0; s < 3; ++s) {
        if (launch_halo(d, st, m0, m1, 0, NUM_VTXBUF_HANDLES) != AC_SUCCESS)
            return AC_FAILURE;
        if (launch_solve(d, st, s, n0, n1) != AC_SUCCESS)
            return AC_FAILURE;
        d->cur ^= 1;
    }
    return AC_SUCCESS;
}

AcResult
acDeviceIntegrateStep(const Device device, const Stream stream, const AcReal dt)
{
    cudaSetDevice(device->id);
    if (acDeviceLoadScalarUniform(device, stream, AC_dt, dt) != AC_SUCCESS)
        return AC_FAILURE;
    return enqueue_step(device, stream_of(device, stream));
}

AcResult
acDeviceIntegrateSteps(const Device device, const Stream stream, const AcReal dt,
                       const int num_steps)
{
    cudaSetDevice(device->id);
    if (num_steps <= 0)
        return AC_SUCCESS;
    if (acDeviceLoadScalarUniform(device, stream, AC_dt, dt) != AC_SUCCESS)
        return AC_FAILURE;
    if (prepare_kernels_once() != AC_SUCCESS || ensure_maps(device) != AC_SUCCESS)
        return AC_FAILURE;
    const cudaStream_t st = stream_of(device, stream);
    // key: parameters, configuration and stream the graph was captured with
    const unsigned long long base = (device->uniform_version << 8) ^
                                    ((unsigned long long)device->solve_cfg << 2) ^
                                    ((unsigned long long)stream << 40) ^ 1ull;
    return replay_steps(device, st, STEP_FIXED, base, 0.0, num_steps,
                        [](const Device d, cudaStream_t s) { return enqueue_step(d, s); });
}

AcResult
acDeviceIntegrateStepCFL(const Device device, const Stream stream, const AcReal timescale)
{
    cudaSetDevice(device->id);
    CflParams cp;
    if (cfl_params(device, timescale, cp) != AC_SUCCESS)
        return AC_FAILURE;
    return enqueue_step_cfl(device, stream_of(device, stream), cp);
}

AcResult
acDeviceIntegrateStepsCFL(const Device device, const Stream stream, const AcReal timescale,
                          const int num_steps)
{
    cudaSetDevice(device->id);
    if (num_steps <= 0)
        return AC_SUCCESS;
    CflParams cp;
    if (cfl_params(device, timescale, cp) != AC_SUCCESS)
        return AC_FAILURE;
    if (prepare_kernels_once() != AC_SUCCESS || ensure_maps(device) != AC_SUCCESS)
        return AC_FAILURE;
    const cudaStream_t st = stream_of(device, stream);
    const unsigned long long base = (device->uniform_version << 8) ^
                                    ((unsigned long long)device->solve_cfg << 2) ^
                                    ((unsigned long long)stream << 40) ^ 1ull;
    return replay_steps(device, st, STEP_CFL, base, (double)timescale, num_steps,
                        [cp](const Device d, cudaStream_t s) { return enqueue_step_cfl(d, s, cp); });
}

AcResult
acDeviceGetTimestepRecord(const Device device, const Stream stream, AcReal* dt, double* time,
                          unsigned long long* steps)
{
    cudaSetDevice(device->id);
    const cudaStream_t st = stream_of(device, stream);
    double h[3];
    ACB_CUDA_CHECK(cudaMemcpyAsync(h, device->cfl, sizeof(h), cudaMemcpyDeviceToHost, st));
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    if (dt)
        *dt = (AcReal)h[0];
    if (time)
        *time = h[1];
    if (steps)
        *steps = (unsigned long long)h[2];
    return AC_SUCCESS;
}

AcResult
acDeviceSetSimulationTime(const Device device, const Stream stream, const double time)
{
    cudaSetDevice(device->id);
    const cudaStream_t st = stream_of(device, stream);
    const double h[3]     = {0.0, time, 0.0};
    ACB_CUDA_CHECK(cudaMemcpyAsync(device->cfl, h, sizeof(h), cudaMemcpyHostToDevice, st));
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    return AC_SUCCESS;
}

AcResult
acDeviceLoadVertexBufferDouble(const Device device, const Stream stream,
                               const VertexBufferHandle h, const double* src)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    if (ensure_xfer(device) != AC_SUCCESS)
        return AC_FAILURE;
    const cudaStream_t st = stream_of(device, stream);
    const size_t n        = (size_t)device->L.mx * device->L.my * device->L.mz;
    device->ghost_ok[device->cur] = false;
    ACB_CUDA_CHECK(cudaMemcpyAsync(device->xfer, src, n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (launch_pack(device, st, device->cur, h, device->xfer, 0, 0, 0.0) != AC_SUCCESS)
        return AC_FAILURE;
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    return AC_SUCCESS;
}

AcResult
acDeviceStoreVertexBufferDouble(const Device device, const Stream stream,
                                const VertexBufferHandle h, double* dst)
{
    if (h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    cudaSetDevice(device->id);
    if (ensure_xfer(device) != AC_SUCCESS)
        return AC_FAILURE;
    const cudaStream_t st = stream_of(device, stream);
    const size_t n        = (size_t)device->L.mx * device->L.my * device->L.mz;
    if (launch_pack(device, st, device->cur, h, device->xfer, 1, 0, 0.0) != AC_SUCCESS)
        return AC_FAILURE;
    ACB_CUDA_CHECK(cudaMemcpyAsync(dst, device->xfer, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ACB_CUDA_CHECK(cudaStreamSynchronize(st));
    return AC_SUCCESS;
}

} // extern "C"

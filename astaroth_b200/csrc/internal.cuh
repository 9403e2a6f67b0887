// Host-side pieces shared by the Device layer (device.cu) and the ensemble
// (ensemble.cu): the table of compiled solve-kernel tile shapes, tensor-map
// encoding, kernel arguments from a parameter mirror, the work split, and the
// flat <-> padded copies.
#pragma once
#include <stdio.h>
#include "astaroth.h"
#include "common.cuh"
#include "solve.cuh"

// Solve tile shapes (tile width, tile height, ring depth, CTAs per SM hint)
#if AC_DOUBLE_PRECISION == 1
using SolveCfg0 = TileCfg<32, 4, 8, 1>;
using SolveCfg1 = TileCfg<16, 8, 8, 1>;
using SolveCfg2 = TileCfg<32, 2, 10, 2>;
#elif ACB_MIXED
// all three stage the centre values of substeps 1 and 2 by TMA; the first (the
// default, 12 consumer warps) is the fastest on the 512^3 workload
using SolveCfg0 = TileCfg<32, 12, 6, 1, 2>;
using SolveCfg1 = TileCfg<64, 4, 6, 1, 3>;
using SolveCfg2 = TileCfg<32, 8, 7, 1, 3>;
#else
// the first (the default, 12 consumer warps) is the fastest at 512^3 (12.53
// against 12.63 ms per step for 64 x 6 tiles, same-box A/B); 32-wide tiles also
// waste fewer columns on meshes whose nx is an odd multiple of 32
using SolveCfg0 = TileCfg<32, 12, 7, 1>;
using SolveCfg1 = TileCfg<32, 8, 9, 1>;
using SolveCfg2 = TileCfg<64, 6, 7, 1>;
#endif

typedef void (*SolveKernelFn)(const CUtensorMap, const SolveArgs<AcReal>, const CentreMaps);
typedef void (*EnsKernelFn)(const CUtensorMap, const EnsSolveArgs<AcReal>, const CentreMaps);

struct SolveConfig {
    const char* name;
    int TX, TY, NP, threads;
    int launch_regs; // registers a thread the kernels must be launched with (0: any)
    int NC;          // centre ring slots (0: the centre values are plain loads)
    size_t smem;
    // substeps 0, 1, 2, and 2 with helical forcing (single mesh only): a
    // SolveKernelFn, or an EnsKernelFn in the ensemble table
    const void* kern[4];
    // single mesh: substeps 0, 1, 2 reading the time step from device memory
    // (null in the ensemble table)
    const void* kern_dt[3];
    // single mesh, substep 2 also folding the step diagnostics of its output:
    // plain, with helical forcing, and reading the time step from device memory
    // (null in the ensemble table)
    const void* kern_diag[3];
};

// "tile32x8_ring9", "..._tmacentre" when the centre values are staged by TMA
template <class Cfg, bool ENS>
const char*
solve_config_name()
{
    static char buf[48];
    if (!buf[0])
        snprintf(buf, sizeof(buf), "tile%dx%d_ring%d%s", Cfg::TX, Cfg::TY, Cfg::NP,
                 (!ENS && Cfg::NC > 0) ? "_tmacentre" : "");
    return buf;
}

template <class Cfg, bool ENS>
SolveConfig
make_solve_config()
{
    SolveConfig c;
    c.name    = solve_config_name<Cfg, ENS>();
    c.TX      = Cfg::TX;
    c.TY      = Cfg::TY;
    c.NP      = Cfg::NP;
    c.threads = Cfg::THREADS;
    c.launch_regs = Cfg::REG_LAUNCH;
    c.NC          = ENS ? 0 : Cfg::NC;
    c.smem    = ENS ? Cfg::ring_bytes() : Cfg::smem_bytes(); // ensembles load centres directly
    c.kern[0] = (const void*)solve_kernel<Cfg, 0, ENS>;
    c.kern[1] = (const void*)solve_kernel<Cfg, 1, ENS>;
    c.kern[2] = (const void*)solve_kernel<Cfg, 2, ENS>;
    if constexpr (ENS) {
        c.kern[3]    = nullptr;
        c.kern_dt[0] = c.kern_dt[1] = c.kern_dt[2] = nullptr;
        c.kern_diag[0] = c.kern_diag[1] = c.kern_diag[2] = nullptr;
    }
    else {
        c.kern[3]    = (const void*)solve_kernel<Cfg, 3, ENS>;
        c.kern_dt[0] = (const void*)solve_kernel<Cfg, 0, ENS, true>;
        c.kern_dt[1] = (const void*)solve_kernel<Cfg, 1, ENS, true>;
        c.kern_dt[2] = (const void*)solve_kernel<Cfg, 2, ENS, true>;
        c.kern_diag[0] = (const void*)solve_kernel<Cfg, 2, ENS, false, true>;
        c.kern_diag[1] = (const void*)solve_kernel<Cfg, 3, ENS, false, true>;
        c.kern_diag[2] = (const void*)solve_kernel<Cfg, 2, ENS, true, true>;
    }
    return c;
}

namespace acb_host {

constexpr int kDefaultSolveConfig = 0;

// single-mesh kernels (device.cu) and ensemble kernels (ensemble.cu), same tiles
const SolveConfig* solve_configs(int* n);
const SolveConfig* ensemble_configs(int* n);

// raises the dynamic shared-memory limit of every kernel of a table, once
AcResult prepare_table(const SolveConfig* cfgs, int n);

// 4-D map (x, y, z, field) over a field block with a (TX+8, TY+6, 1, 8) box
AcResult encode_block_map(const Layout& L, const state_t* block, const SolveConfig& cfg,
                          CUtensorMap* map);
// the same with a (TX, TY, 1, narr) box over a block of narr arrays: a tile's
// centre values (the fields' narr = ACB_NARR, the mixed lo block's ACB_LO_NARR)
AcResult encode_centre_map(const Layout& L, const void* block, const SolveConfig& cfg,
                           CUtensorMap* map, int narr);

// kernel arguments from a parameter mirror: coefficients pre-scaled in double
// and rounded once to AcReal; rkA/rkB for `step` from AC_dt
SolveParams<AcReal> make_params(const AcMeshInfo& uniforms, const Layout& L, int step,
                                int forcing);

// z segments per tile column so that tiles*segments fills the last wave best
int choose_segments(long long ntiles, int nzr, long long slots, int min_planes);

// Device staging buffer of loads and stores: the caller's values pass through
// it in one contiguous transfer per chunk, and a kernel scatters them into (or
// gathers them from) the padded layout, where a field's values are ACB_LANES
// apart (a pitched host-to-device copy of rows a few KB long ran at about a
// third of the contiguous rate, and the pair layout interleaves two fields).
// `done` is recorded after each use, and the next use, on whatever stream,
// waits for it.
struct StageBuf {
    state_t* buf;
    size_t elems;
    cudaEvent_t done;
};
// a buffer of min(max_elems, 64 MB) values
AcResult stage_create(StageBuf* stage, size_t max_elems);
void stage_destroy(StageBuf* stage);

// copies a flat range of a field (field: its base, block + fidx(L, f, 0))
// between host memory (reference order) and the padded device layout through
// the staging buffer; zeroes the lo parts of loaded values when given.
AcResult copy_field_range(cudaStream_t st, const Layout& L, state_t* field, size_t s,
                          AcReal* host, size_t count, bool h2d, lo16_t* lo_field,
                          StageBuf* stage);

} // namespace acb_host

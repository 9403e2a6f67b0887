// Ensembles: many independent meshes of uneven sizes and parameters on one GPU,
// advanced by ONE persistent solve launch and ONE ghost-fill launch per
// substep, with whole steps captured in CUDA graphs and the tile shape /
// z-segment length chosen per ensemble by a timing autotuner with an on-disk
// cache. No counterpart in the reference (its Device owns one mesh and a GPU
// holds one __constant__ parameter block, src/core/kernels/kernels.cu:9).
//
// Members keep the Device layout (common.cuh: Layout) and the solve kernel of
// solve.cuh in its ensemble form: each (tile, z segment) task finds its member
// in a descriptor table in global memory (TMA map, geometry, buffers,
// parameters), one table per buffer parity.
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "astaroth.h"
#include "astaroth_b200.h"
#include "common.cuh"
#include "halo.cuh"
#include "internal.cuh"
#include "solve.cuh"

using namespace acb_host;

const SolveConfig*
acb_host::ensemble_configs(int* n)
{
#if AC_DOUBLE_PRECISION == 1
    static const SolveConfig table[] = {
        make_solve_config<SolveCfg0, true>(),
        make_solve_config<SolveCfg1, true>(),
        make_solve_config<SolveCfg2, true>(),
    };
#else
    static const SolveConfig table[] = {
        make_solve_config<SolveCfg0, true>(),
        make_solve_config<SolveCfg1, true>(),
        make_solve_config<SolveCfg2, true>(),
    };
#endif
    *n = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

namespace {

struct Member {
    AcMeshInfo config;
    AcMeshInfo uniforms; // defaults of the module overlaid with the member's valid values
    Layout L;
    state_t* blk[2];
    lo16_t* lo[2]; // mixed build: lo blocks (bf16, see common.cuh)
};

bool
valid_real(double v)
{
    return !isnan(v) && !isinf(v);
}

// Module defaults (acc/stdlib/stdderiv.h:6-11, acc/mhd_solver/stencil_kernel.ac:69,112)
// overlaid with the valid entries of a member's configuration, as a Device does.
AcMeshInfo
member_uniforms(const AcMeshInfo& c)
{
    AcMeshInfo u;
    memset(&u, 0, sizeof(u));
    const AcReal ds            = (AcReal)0.04908738521;
    u.real_params[AC_dsx]      = ds;
    u.real_params[AC_dsy]      = ds;
    u.real_params[AC_dsz]      = ds;
    u.real_params[AC_inv_dsx]  = (AcReal)1.0 / ds;
    u.real_params[AC_inv_dsy]  = (AcReal)1.0 / ds;
    u.real_params[AC_inv_dsz]  = (AcReal)1.0 / ds;
    u.real_params[AC_cs_sound] = (AcReal)1.0;
    u.real_params[AC_cs2_sound] = (AcReal)1.0;
    for (int i = 0; i < NUM_INT_PARAMS; ++i)
        u.int_params[i] = c.int_params[i];
    for (int i = 0; i < NUM_INT3_PARAMS; ++i)
        u.int3_params[i] = c.int3_params[i];
    for (int i = 0; i < NUM_REAL_PARAMS; ++i)
        if (valid_real((double)c.real_params[i]))
            u.real_params[i] = c.real_params[i];
    return u;
}

} // namespace

struct ensemble_s {
    int id;
    int num_sms;
    std::vector<Member> m;
    cudaStream_t stream;
    unsigned* status;
    int cur; // buffer parity: blk[cur] is `in` for every member
    int cfg;
    int seg_planes; // target planes per z segment (0: whole columns)
    // ghost_ok[p]: the ghosts of every member's block p hold periodic images
    bool ghost_ok[2];
    StageBuf stage; // staging buffer of member loads

    bool desc_valid;
    std::vector<MemberDesc<AcReal>> h_desc[2];
    std::vector<MemberParams<AcReal>> h_mp; // by task-list position (both parities)
    // launch arguments of one group of members (about 20 KB, kept off the
    // stack; the launch copies them)
    std::unique_ptr<EnsSolveArgs<AcReal>> args;
    MemberDesc<AcReal>* d_desc[2];
    HaloMember* d_halo[2];
    long long halo_total; // work units of one batched ghost fill
    long long total_tasks;
    int grid;

    unsigned long long launches;
    unsigned long long version; // bumped on any schedule change
    cudaGraphExec_t graph[2];
    unsigned long long graph_key[2];
    float graph_dt[2];
    unsigned long long graph_launches[2];
    bool graph_ghost[2][2]; // ghost_ok of both blocks after a replay of graph[p]
};

namespace {

// The parts of a member's kernel parameters that its stencils and right-hand
// sides read (MemberParams), from its full parameter set.
MemberParams<AcReal>
member_params(const SolveParams<AcReal>& P)
{
    MemberParams<AcReal> m;
    memset(&m, 0, sizeof(m));
#if AC_DOUBLE_PRECISION == 1
    memcpy(m.c1, P.c1, sizeof(m.c1));
    memcpy(m.c2, P.c2, sizeof(m.c2));
    memcpy(m.cx, P.cx, sizeof(m.cx));
#else
    memcpy(m.c1p, P.c1p, sizeof(m.c1p));
    memcpy(m.c2p, P.c2p, sizeof(m.c2p));
    memcpy(m.cxp, P.cxp, sizeof(m.cxp));
#endif
    m.nu           = P.nu;
    m.eta          = P.eta;
    m.inv_mu0      = P.inv_mu0;
    m.eta_mu0      = P.eta_mu0;
    m.zeta         = P.zeta;
    m.cs2_sound    = P.cs2_sound;
    m.inv_cp       = P.inv_cp;
    m.gamma        = P.gamma;
    m.gm1          = P.gm1;
    m.gamma_inv_cp = P.gamma_inv_cp;
    m.lnrho0       = P.lnrho0;
    m.lnT0         = P.lnT0;
    m.exp_lnT0     = P.exp_lnT0;
    m.k_heat       = P.k_heat;
    return m;
}


void
drop_graphs(Ensemble e)
{
    for (int p = 0; p < 2; ++p) {
        if (e->graph[p])
            cudaGraphExecDestroy(e->graph[p]);
        e->graph[p]     = nullptr;
        e->graph_key[p] = 0;
    }
}

// (Re)builds both parities' descriptor tables and ghost-fill tables for the
// current tile configuration and segment length, and uploads them.
AcResult
build_tables(Ensemble e)
{
    int ncfg;
    const SolveConfig* cfgs = ensemble_configs(&ncfg);
    if (prepare_table(cfgs, ncfg) != AC_SUCCESS)
        return AC_FAILURE;
    const SolveConfig& cfg = cfgs[e->cfg];
    const int n            = (int)e->m.size();
    int per_sm             = 0;
    ACB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfg.kern[1], cfg.threads,
                                                                 cfg.smem));
    per_sm = std::max(per_sm, 1);
    e->h_mp.assign(n, MemberParams<AcReal>());
    for (int p = 0; p < 2; ++p) {
        std::vector<MemberDesc<AcReal>>& D = e->h_desc[p];
        D.assign(n, MemberDesc<AcReal>());
        std::vector<HaloMember> H(n);
        long long tasks = 0, units = 0;
        // Task list order: members with the longest tasks (z segment + halo
        // planes) first, so that the persistent CTAs, which take tasks
        // round-robin, finish the launch on short tasks instead of idling
        // behind a few long ones (longest-processing-time-first).
        auto zseg_of = [&](const Layout& L) {
            int nseg = 1;
            if (e->seg_planes > 0)
                nseg = std::max(1, (int)lround((double)L.nz / e->seg_planes));
            return (L.nz + nseg - 1) / nseg;
        };
        std::vector<int> order(n);
        for (int i = 0; i < n; ++i)
            order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return zseg_of(e->m[a].L) > zseg_of(e->m[b].L);
        });
        for (int pos = 0; pos < n; ++pos) {
            const int i      = order[pos];
            const Member& mb = e->m[i];
            const Layout& L  = mb.L;
            MemberDesc<AcReal>& d = D[pos];
            memset(&d, 0, sizeof(d));
            if (encode_block_map(L, mb.blk[p], cfg, &d.tmap) != AC_SUCCESS)
                return AC_FAILURE;
            SolveGeom& g = d.g;
            g.L          = L;
            g.start      = make_int3(NGHOST, NGHOST, NGHOST);
            g.end        = make_int3(NGHOST + L.nx, NGHOST + L.ny, NGHOST + L.nz);
            g.tx0        = 0;
            g.ntx        = (L.nx + cfg.TX - 1) / cfg.TX;
            g.nty        = (L.ny + cfg.TY - 1) / cfg.TY;
            g.nzr        = L.nz;
            g.zseg        = zseg_of(L);
            g.nseg        = (L.nz + g.zseg - 1) / g.zseg;
            g.tasks       = (long long)g.ntx * g.nty * g.nseg;
            d.task_begin  = tasks;
            tasks += g.tasks;
            d.out         = mb.blk[p ^ 1];
            d.in_lo       = mb.lo[p];
            d.out_lo      = mb.lo[p ^ 1];
            if (p == 0)
                e->h_mp[pos] = member_params(make_params(mb.uniforms, L, 0, 0));
            H[pos].L          = L;
            H[pos].block      = mb.blk[p];
            H[pos].unit_begin = units;
            H[pos].units_a    = (unsigned)halo_units_a(L);
            units += halo_units(L);
        }
        e->total_tasks = tasks;
        e->halo_total  = units;
        ACB_CUDA_CHECK(cudaMemcpy(e->d_desc[p], D.data(), sizeof(MemberDesc<AcReal>) * n,
                                  cudaMemcpyHostToDevice));
        ACB_CUDA_CHECK(cudaMemcpy(e->d_halo[p], H.data(), sizeof(HaloMember) * n,
                                  cudaMemcpyHostToDevice));
    }
    e->grid       = (int)std::min<long long>((long long)e->num_sms * per_sm, e->total_tasks);
    e->desc_valid = true;
    drop_graphs(e);
    return AC_SUCCESS;
}

AcResult
launch_halo_all(Ensemble e, cudaStream_t st)
{
    const int n          = (int)e->m.size();
    const long long want = (e->halo_total + 255) / 256;
    const int blocks     = (int)std::max<long long>(1, std::min<long long>(want, e->num_sms * 32));
    halo_batch_kernel<<<blocks, 256, 0, st>>>(e->d_halo[e->cur], n, e->halo_total);
    ACB_CUDA_CHECK(cudaGetLastError());
    e->launches++;
    e->ghost_ok[e->cur] = true;
    return AC_SUCCESS;
}

AcResult
launch_solve_all(Ensemble e, cudaStream_t st, int step, AcReal dt)
{
    int ncfg;
    const SolveConfig& cfg = ensemble_configs(&ncfg)[e->cfg];
    const int n            = (int)e->m.size();
    // the launch arguments carry up to ACB_ENS_GROUP members' parameters, so
    // a larger ensemble takes one launch per group of members (in task order)
    if (!e->args)
        e->args.reset(new EnsSolveArgs<AcReal>());
    EnsSolveArgs<AcReal>& a = *e->args;
    memset(&a, 0, sizeof(a));
    // Williamson (1980) 2N coefficients, "previous state" form (as the Device path)
    const double alpha[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double beta[3]  = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
    a.P.rkB               = (AcReal)(beta[step] * (double)dt);
    a.P.rkA               = step > 0 ? (AcReal)(beta[step] * alpha[step] / beta[step - 1]) : 0;
    a.status              = e->status;
    // ensemble kernels take their centre values by plain loads: no centre maps
    static const CentreMaps no_centre_maps = {};
    const std::vector<MemberDesc<AcReal>>& D = e->h_desc[e->cur];
    for (int g0 = 0; g0 < n; g0 += ACB_ENS_GROUP) {
        const int gn            = std::min(ACB_ENS_GROUP, n - g0);
        const long long t_begin = D[g0].task_begin;
        const long long t_end   = g0 + gn < n ? D[g0 + gn].task_begin : e->total_tasks;
        a.members               = e->d_desc[e->cur] + g0;
        a.nmembers              = gn;
        a.task_base             = t_begin;
        a.total_tasks           = t_end - t_begin;
        for (int i = 0; i < gn; ++i)
            a.mp[i] = e->h_mp[g0 + i];
        const int grid = (int)std::min<long long>(e->grid, a.total_tasks);
        // the map parameter is not read in ensemble mode; any valid map fills it
        ((EnsKernelFn)cfg.kern[step])<<<grid, cfg.threads, cfg.smem, st>>>(D[0].tmap, a,
                                                                           no_centre_maps);
        ACB_CUDA_CHECK(cudaGetLastError());
        e->launches++;
    }
    e->ghost_ok[e->cur ^ 1] = false; // the out blocks' ghosts are stale now
    return AC_SUCCESS;
}

AcResult
enqueue_step(Ensemble e, cudaStream_t st, AcReal dt)
{
    for (int s = 0; s < 3; ++s) {
        if (!e->ghost_ok[e->cur] && launch_halo_all(e, st) != AC_SUCCESS)
            return AC_FAILURE;
        if (launch_solve_all(e, st, s, dt) != AC_SUCCESS)
            return AC_FAILURE;
        e->cur ^= 1;
    }
    return AC_SUCCESS;
}

std::string
cache_key(Ensemble e)
{
    std::string k = ACB_MIXED ? "mixed" : (sizeof(AcReal) == 8 ? "dp" : "sp");
    std::vector<std::string> dims;
    for (const Member& mb : e->m)
        dims.push_back(std::to_string(mb.L.nx) + "x" + std::to_string(mb.L.ny) + "x" +
                       std::to_string(mb.L.nz));
    std::sort(dims.begin(), dims.end());
    // run-length encode the sorted sizes: 16*32x32x32,16*48x48x48,...
    for (size_t i = 0; i < dims.size();) {
        size_t j = i;
        while (j < dims.size() && dims[j] == dims[i])
            ++j;
        k += "|" + std::to_string(j - i) + "*" + dims[i];
        i = j;
    }
    return k;
}

std::string
cache_file(const char* path)
{
    if (path && path[0])
        return path;
    const char* env = getenv("ACB_TUNE_CACHE");
    if (env && env[0])
        return env;
    const char* home = getenv("HOME");
    std::string dir  = std::string(home ? home : "/tmp") + "/.cache";
    mkdir(dir.c_str(), 0755);
    dir += "/astaroth_b200";
    mkdir(dir.c_str(), 0755);
    return dir + "/tune.txt";
}

bool
cache_lookup(const std::string& file, const std::string& key, int* cfg, int* seg)
{
    FILE* f = fopen(file.c_str(), "r");
    if (!f)
        return false;
    char kbuf[4096];
    int c, s;
    bool found = false;
    while (fscanf(f, "%4095s %d %d", kbuf, &c, &s) == 3)
        if (key == kbuf) { // the last entry for a key wins
            *cfg  = c;
            *seg  = s;
            found = true;
        }
    fclose(f);
    return found;
}

} // namespace

extern "C" {

AcResult
acEnsembleCreate(const int device_id, const int num_members, const AcMeshInfo* configs,
                 Ensemble* ensemble)
{
    int ndev = 0;
    if (num_members < 1 || !configs || cudaGetDeviceCount(&ndev) != cudaSuccess || device_id < 0 ||
        device_id >= ndev) {
        fprintf(stderr, "astaroth_b200: acEnsembleCreate: invalid arguments\n");
        return AC_FAILURE;
    }
    ACB_CUDA_CHECK(cudaSetDevice(device_id));
    Ensemble e = new ensemble_s();
    e->id      = device_id;
    e->cfg     = kDefaultSolveConfig;
    e->seg_planes = 32;
    ACB_CUDA_CHECK(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device_id));
    ACB_CUDA_CHECK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    ACB_CUDA_CHECK(cudaMalloc((void**)&e->status, sizeof(unsigned)));
    ACB_CUDA_CHECK(cudaMemset(e->status, 0, sizeof(unsigned)));
    e->m.resize(num_members);
    for (int i = 0; i < num_members; ++i) {
        Member& mb = e->m[i];
        memset(&mb, 0, sizeof(mb));
        mb.config   = configs[i];
        mb.uniforms = member_uniforms(configs[i]);
        const int nx = configs[i].int_params[AC_nx], ny = configs[i].int_params[AC_ny],
                  nz = configs[i].int_params[AC_nz];
        if (nx < NGHOST || ny < NGHOST || nz < NGHOST) {
            fprintf(stderr, "astaroth_b200: ensemble member %d too small\n", i);
            acEnsembleDestroy(e);
            return AC_FAILURE;
        }
        mb.L               = make_layout(nx, ny, nz);
        const size_t bytes = block_bytes(mb.L);
        for (int b = 0; b < 2; ++b) {
            ACB_CUDA_CHECK(cudaMalloc((void**)&mb.blk[b], bytes));
            ACB_CUDA_CHECK(cudaMemset(mb.blk[b], 0, bytes));
#if ACB_MIXED
            const size_t lb = lo_block_bytes(mb.L);
            ACB_CUDA_CHECK(cudaMalloc((void**)&mb.lo[b], lb));
            ACB_CUDA_CHECK(cudaMemset(mb.lo[b], 0, lb));
#endif
        }
    }
    size_t largest = 0;
    for (const Member& mb : e->m)
        largest = std::max(largest, (size_t)mb.L.mx * mb.L.my * mb.L.mz);
    if (stage_create(&e->stage, largest) != AC_SUCCESS) {
        acEnsembleDestroy(e);
        return AC_FAILURE;
    }
    for (int p = 0; p < 2; ++p) {
        ACB_CUDA_CHECK(cudaMalloc((void**)&e->d_desc[p], sizeof(MemberDesc<AcReal>) * num_members));
        ACB_CUDA_CHECK(cudaMalloc((void**)&e->d_halo[p], sizeof(HaloMember) * num_members));
    }
    if (build_tables(e) != AC_SUCCESS) {
        acEnsembleDestroy(e);
        return AC_FAILURE;
    }
    *ensemble = e;
    return AC_SUCCESS;
}

AcResult
acEnsembleDestroy(Ensemble e)
{
    if (!e)
        return AC_FAILURE;
    cudaSetDevice(e->id);
    cudaDeviceSynchronize();
    drop_graphs(e);
    for (Member& mb : e->m)
        for (int b = 0; b < 2; ++b) {
            if (mb.blk[b])
                cudaFree(mb.blk[b]);
            if (mb.lo[b])
                cudaFree(mb.lo[b]);
        }
    for (int p = 0; p < 2; ++p) {
        if (e->d_desc[p])
            cudaFree(e->d_desc[p]);
        if (e->d_halo[p])
            cudaFree(e->d_halo[p]);
    }
    if (e->status)
        cudaFree(e->status);
    stage_destroy(&e->stage);
    if (e->stream)
        cudaStreamDestroy(e->stream);
    delete e;
    return AC_SUCCESS;
}

AcResult
acEnsembleLoadMember(Ensemble e, const int member, const AcMesh host_mesh)
{
    if (member < 0 || member >= (int)e->m.size())
        return AC_FAILURE;
    cudaSetDevice(e->id);
    Member& mb     = e->m[member];
    const size_t n = (size_t)mb.L.mx * mb.L.my * mb.L.mz;
    if (acVertexBufferSize(host_mesh.info) != n) {
        fprintf(stderr, "astaroth_b200: acEnsembleLoadMember: mesh size mismatch\n");
        return AC_FAILURE;
    }
    e->ghost_ok[e->cur] = false;
    for (int f = 0; f < NUM_VTXBUF_HANDLES; ++f) {
        lo16_t* lo = lo_field(mb.lo[e->cur], mb.L, f);
        if (copy_field_range(e->stream, mb.L, mb.blk[e->cur] + fidx(mb.L, f, 0), 0,
                             host_mesh.vertex_buffer[f], n, true, lo, &e->stage) != AC_SUCCESS)
            return AC_FAILURE;
    }
    ACB_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return AC_SUCCESS;
}

AcResult
acEnsembleStoreMember(Ensemble e, const int member, AcMesh* host_mesh)
{
    if (member < 0 || member >= (int)e->m.size())
        return AC_FAILURE;
    cudaSetDevice(e->id);
    Member& mb     = e->m[member];
    const size_t n = (size_t)mb.L.mx * mb.L.my * mb.L.mz;
    if (acVertexBufferSize(host_mesh->info) != n) {
        fprintf(stderr, "astaroth_b200: acEnsembleStoreMember: mesh size mismatch\n");
        return AC_FAILURE;
    }
    for (int f = 0; f < NUM_VTXBUF_HANDLES; ++f)
        if (copy_field_range(e->stream, mb.L, mb.blk[e->cur] + fidx(mb.L, f, 0), 0,
                             host_mesh->vertex_buffer[f], n, false, nullptr, &e->stage) !=
            AC_SUCCESS)
            return AC_FAILURE;
    ACB_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return AC_SUCCESS;
}

AcResult
acEnsembleIntegrateStep(Ensemble e, const AcReal dt)
{
    cudaSetDevice(e->id);
    if (!valid_real((double)dt))
        return AC_FAILURE;
    return enqueue_step(e, e->stream, dt);
}

AcResult
acEnsembleIntegrateSteps(Ensemble e, const AcReal dt, const int num_steps)
{
    cudaSetDevice(e->id);
    if (!valid_real((double)dt))
        return AC_FAILURE;
    for (int i = 0; i < num_steps; ++i) {
        const int p = e->cur;
        // a captured step contains the ghost fill only when the ghosts were stale
        const unsigned long long key = (e->version << 2) | (e->ghost_ok[p] ? 2ull : 0ull) | 1ull;
        if (!e->graph[p] || e->graph_key[p] != key || e->graph_dt[p] != (float)dt) {
            if (e->graph[p])
                cudaGraphExecDestroy(e->graph[p]);
            e->graph[p] = nullptr;
            cudaGraph_t g;
            ACB_CUDA_CHECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            const unsigned long long before = e->launches;
            const AcResult rc               = enqueue_step(e, e->stream, dt);
            ACB_CUDA_CHECK(cudaStreamEndCapture(e->stream, &g));
            e->cur               = p; // capture advanced the parity; the replay below does
            e->graph_launches[p] = e->launches - before;
            e->graph_ghost[p][0] = e->ghost_ok[0];
            e->graph_ghost[p][1] = e->ghost_ok[1];
            e->launches          = before;
            if (rc != AC_SUCCESS) {
                cudaGraphDestroy(g);
                return AC_FAILURE;
            }
            ACB_CUDA_CHECK(cudaGraphInstantiate(&e->graph[p], g, 0));
            cudaGraphDestroy(g);
            e->graph_key[p] = key;
            e->graph_dt[p]  = (float)dt;
        }
        ACB_CUDA_CHECK(cudaGraphLaunch(e->graph[p], e->stream));
        e->launches += e->graph_launches[p];
        e->ghost_ok[0] = e->graph_ghost[p][0]; // as the captured step left them
        e->ghost_ok[1] = e->graph_ghost[p][1];
        e->cur ^= 1; // three swaps per step
    }
    return AC_SUCCESS;
}

AcResult
acEnsembleSynchronize(Ensemble e)
{
    cudaSetDevice(e->id);
    ACB_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return AC_SUCCESS;
}

AcResult
acEnsembleGetStatus(Ensemble e, unsigned* status)
{
    cudaSetDevice(e->id);
    ACB_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    ACB_CUDA_CHECK(cudaMemcpy(status, e->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return AC_SUCCESS;
}

AcResult
acEnsembleGetCudaStream(Ensemble e, void** cuda_stream)
{
    *cuda_stream = (void*)e->stream;
    return AC_SUCCESS;
}

AcResult
acEnsembleGetLaunchCount(Ensemble e, unsigned long long* count)
{
    *count = e->launches;
    return AC_SUCCESS;
}

AcResult
acEnsembleSetSchedule(Ensemble e, const int config, const int segment_planes)
{
    int n;
    ensemble_configs(&n);
    if (config < 0 || config >= n || segment_planes < 0)
        return AC_FAILURE;
    cudaSetDevice(e->id);
    ACB_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    e->cfg        = config;
    e->seg_planes = segment_planes;
    e->version++;
    return build_tables(e);
}

AcResult
acEnsembleGetSchedule(Ensemble e, int* config, int* segment_planes)
{
    *config         = e->cfg;
    *segment_planes = e->seg_planes;
    return AC_SUCCESS;
}

AcResult
acEnsembleAutoOptimize(Ensemble e, const char* cache_path)
{
    cudaSetDevice(e->id);
    const std::string file = cache_file(cache_path);
    const std::string key  = cache_key(e);
    int cfg = 0, seg = 0;
    if (cache_lookup(file, key, &cfg, &seg))
        return acEnsembleSetSchedule(e, cfg, seg);

    // time substep s = 1 (reads in and out, writes out): `in` holds the state
    // between whole steps and is never written, so the members keep their state
    int ncfg;
    ensemble_configs(&ncfg);
    const int segs[] = {0, 64, 32, 16};
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best_ms = INFINITY;
    int best_cfg = e->cfg, best_seg = e->seg_planes;
    for (int c = 0; c < ncfg; ++c)
        for (int s : segs) {
            if (acEnsembleSetSchedule(e, c, s) != AC_SUCCESS)
                continue;
            if (launch_solve_all(e, e->stream, 1, (AcReal)1e-3) != AC_SUCCESS) // warm-up
                continue;
            cudaEventRecord(t0, e->stream);
            for (int r = 0; r < 3; ++r)
                launch_solve_all(e, e->stream, 1, (AcReal)1e-3);
            cudaEventRecord(t1, e->stream);
            cudaEventSynchronize(t1);
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            if (cudaGetLastError() == cudaSuccess && ms < best_ms) {
                best_ms  = ms;
                best_cfg = c;
                best_seg = s;
            }
        }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (acEnsembleSetSchedule(e, best_cfg, best_seg) != AC_SUCCESS)
        return AC_FAILURE;
    FILE* f = fopen(file.c_str(), "a");
    if (f) {
        fprintf(f, "%s %d %d\n", key.c_str(), best_cfg, best_seg);
        fclose(f);
    }
    return AC_SUCCESS;
}

} // extern "C"

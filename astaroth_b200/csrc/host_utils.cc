// Host-side helpers of include/astaroth_utils.h (reference src/utils/*.c):
// config loading, host mesh filling and periodic bounds, host reductions,
// mesh verification, and the CPU model step acHostIntegrateStep.
//
// Everything here runs on the CPU and is independent of the GPU path; callers
// use it to prepare meshes and to check GPU results, exactly as with the
// reference's utils library.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "astaroth.h"
#include "astaroth_utils.h"

static inline bool
finite_real(long double v)
{
    return !isnan(v) && !isinf(v);
}

extern "C" {

// ---------------------------------------------------------------------------
// config (src/utils/config_loader.c:39-112)
// ---------------------------------------------------------------------------
static int
name_index(const char* key, const char* const* names, int n)
{
    for (int i = 0; i < n; ++i)
        if (!strcmp(key, names[i]))
            return i;
    return -1;
}

AcResult
acLoadConfig(const char* config_path, AcMeshInfo* config)
{
    if (!config_path) {
        fprintf(stderr, "ERROR: acLoadConfig without a path\n");
        exit(EXIT_FAILURE);
    }
    memset(config, 0xFF, sizeof(*config));
    printf("Config file path: %s\n", config_path);
    FILE* fp = fopen(config_path, "r");
    if (!fp) {
        fprintf(stderr, "ERROR: cannot open config file %s\n", config_path);
        exit(EXIT_FAILURE);
    }
    char key[128], value[128];
    int matched;
    while ((matched = fscanf(fp, "%127s = %127s", key, value)) != EOF) {
        if (matched < 2)
            continue;
        int idx;
        if ((idx = name_index(key, intparam_names, NUM_INT_PARAMS)) >= 0)
            config->int_params[idx] = atoi(value);
        else if ((idx = name_index(key, realparam_names, NUM_REAL_PARAMS)) >= 0)
            config->real_params[idx] = (AcReal)atof(value);
    }
    fclose(fp);
    acHostUpdateBuiltinParams(config);

    AcResult rc = AC_SUCCESS;
    const uint32_t* words = (const uint32_t*)config;
    for (size_t i = 0; i < sizeof(*config) / sizeof(uint32_t); ++i)
        if (words[i] == 0xFFFFFFFFu)
            rc = AC_FAILURE; // some parameter was left unset
    return rc;
}

// ---------------------------------------------------------------------------
// host mesh memory (src/utils/memory.c:23-111)
// ---------------------------------------------------------------------------
AcResult
acHostVertexBufferSet(const VertexBufferHandle handle, const AcReal value, AcMesh* mesh)
{
    const size_t n = acVertexBufferSize(mesh->info);
    for (size_t i = 0; i < n; ++i)
        mesh->vertex_buffer[handle][i] = value;
    return AC_SUCCESS;
}

AcResult
acHostMeshSet(const AcReal value, AcMesh* mesh)
{
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w)
        acHostVertexBufferSet((VertexBufferHandle)w, value, mesh);
    return AC_SUCCESS;
}

AcResult
acHostMeshClear(AcMesh* mesh)
{
    return acHostMeshSet(0, mesh);
}

AcResult
acHostMeshApplyPeriodicBounds(AcMesh* mesh)
{
    const AcMeshInfo& I = mesh->info;
    const int nx = I.int_params[AC_nx], ny = I.int_params[AC_ny], nz = I.int_params[AC_nz];
    const int mx = I.int_params[AC_mx], my = I.int_params[AC_my], mz = I.int_params[AC_mz];
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        AcReal* f = mesh->vertex_buffer[w];
#pragma omp parallel for schedule(static)
        for (int k = 0; k < mz; ++k)
            for (int j = 0; j < my; ++j) {
                const bool inner_row = j >= NGHOST && j < NGHOST + ny && k >= NGHOST &&
                                       k < NGHOST + nz;
                const int js = (j - NGHOST + ny) % ny + NGHOST;
                const int ks = (k - NGHOST + nz) % nz + NGHOST;
                for (int i = 0; i < mx; ++i) {
                    if (inner_row && i >= NGHOST && i < NGHOST + nx)
                        continue;
                    const int is = (i - NGHOST + nx) % nx + NGHOST;
                    f[acVertexBufferIdx(i, j, k, I)] = f[acVertexBufferIdx(is, js, ks, I)];
                }
            }
    }
    return AC_SUCCESS;
}

// ---------------------------------------------------------------------------
// host reductions (src/utils/modelreduce.c:76-209); AcReal accumulation and
// normalised RMS as in the reference
// ---------------------------------------------------------------------------
static AcReal
host_reduce(const AcMesh& mesh, const ReductionType rtype, int nvec, const int* h)
{
    const AcMeshInfo& I = mesh.info;
    const bool mm       = rtype == RTYPE_MAX || rtype == RTYPE_MIN;
    AcReal res          = 0;
    bool first          = true;
    for (int k = I.int_params[AC_nz_min]; k < I.int_params[AC_nz_max]; ++k)
        for (int j = I.int_params[AC_ny_min]; j < I.int_params[AC_ny_max]; ++j)
            for (int i = I.int_params[AC_nx_min]; i < I.int_params[AC_nx_max]; ++i) {
                const size_t id = acVertexBufferIdx(i, j, k, I);
                const AcReal a  = mesh.vertex_buffer[h[0]][id];
                AcReal v;
                if (nvec == 1) {
                    if (rtype == RTYPE_RMS)
                        v = a * a;
                    else if (rtype == RTYPE_RMS_EXP)
                        v = (AcReal)exp(a) * (AcReal)exp(a);
                    else
                        v = a;
                }
                else {
                    const AcReal b = mesh.vertex_buffer[h[1]][id];
                    const AcReal c = mesh.vertex_buffer[h[2]][id];
                    if (rtype == RTYPE_RMS)
                        v = a * a + b * b + c * c;
                    else if (rtype == RTYPE_RMS_EXP)
                        v = (AcReal)exp(a) * (AcReal)exp(a) + (AcReal)exp(b) * (AcReal)exp(b) +
                            (AcReal)exp(c) * (AcReal)exp(c);
                    else
                        v = (AcReal)sqrt(a * a + b * b + c * c);
                }
                if (mm && first) {
                    res   = v;
                    first = false;
                }
                else if (rtype == RTYPE_MAX)
                    res = v > res ? v : res;
                else if (rtype == RTYPE_MIN)
                    res = v < res ? v : res;
                else
                    res = res + v;
            }
    if (rtype == RTYPE_RMS || rtype == RTYPE_RMS_EXP) {
        const AcReal inv_n = (AcReal)1.0 / I.int_params[AC_nxyz];
        return (AcReal)sqrt(inv_n * res);
    }
    return res;
}

AcReal
acHostReduceScal(const AcMesh mesh, const ReductionType rtype, const VertexBufferHandle a)
{
    if (!(rtype == RTYPE_MAX || rtype == RTYPE_MIN || rtype == RTYPE_RMS ||
          rtype == RTYPE_RMS_EXP || rtype == RTYPE_SUM)) {
        fprintf(stderr, "ERROR: Unrecognized RTYPE\n");
        exit(EXIT_FAILURE);
    }
    const int h[1] = {(int)a};
    return host_reduce(mesh, rtype, 1, h);
}

AcReal
acHostReduceVec(const AcMesh mesh, const ReductionType rtype, const VertexBufferHandle a,
                const VertexBufferHandle b, const VertexBufferHandle c)
{
    if (!(rtype == RTYPE_MAX || rtype == RTYPE_MIN || rtype == RTYPE_RMS ||
          rtype == RTYPE_RMS_EXP || rtype == RTYPE_SUM)) {
        fprintf(stderr, "ERROR: Unrecognized RTYPE\n");
        exit(EXIT_FAILURE);
    }
    const int h[3] = {(int)a, (int)b, (int)c};
    return host_reduce(mesh, rtype, 3, h);
}

// ---------------------------------------------------------------------------
// verification (src/utils/verification.c:30-168)
// ---------------------------------------------------------------------------
Error
acGetError(const AcReal model, const AcReal candidate)
{
    Error e;
    memset(&e, 0, sizeof(e));
    e.model     = model;
    e.candidate = candidate;
    if (model == candidate || fabsl((long double)model - (long double)candidate) == 0) {
        e.abs_error = e.rel_error = e.ulp_error = 0;
    }
    else if (!finite_real(model) || !finite_real(candidate)) {
        e.abs_error = e.rel_error = e.ulp_error = INFINITY;
    }
    else {
        const int p            = sizeof(AcReal) == 4 ? 24 : 53; // significand bits
        const long double ex   = floorl(logl(fabsl((long double)model)) / logl(2.0L));
        const long double ulp  = powl(2.0L, ex - (p - 1));
        const long double meps = 0.5L * powl(2.0L, -(p - 1));
        e.abs_error            = fabsl((long double)model - (long double)candidate);
        e.ulp_error            = e.abs_error / ulp;
        e.rel_error = fabsl(1.0L - (long double)candidate / (long double)model) / meps;
    }
    e.maximum_magnitude = e.minimum_magnitude = 0;
    return e;
}

bool
acEvalError(const char* label, const Error error)
{
    const long double max_ulp = 5;
    bool ok;
    if (error.ulp_error < max_ulp)
        ok = true;
    else if (error.abs_error < error.minimum_magnitude * AC_REAL_EPSILON)
        ok = true;
    else
        ok = false;
    printf("%-15s... %s ", label, ok ? "\x1B[32mOK! \x1B[0m" : "\x1B[31mFAIL! \x1B[0m");
    printf("| %.3Lg (abs), %.3Lg (ulps), %.3Lg (rel). Range: [%.3g, %.3g]\n", error.abs_error,
           error.ulp_error, error.rel_error, (double)error.minimum_magnitude,
           (double)error.maximum_magnitude);
    FILE* f = fopen("verification.out", "a");
    if (f) {
        fprintf(f, "%s, %Lg, %Lg, %Lg, %g, %g\n", label, error.ulp_error, error.abs_error,
                error.rel_error, (double)error.maximum_magnitude, (double)error.minimum_magnitude);
        fclose(f);
    }
    return ok;
}

AcResult
acVerifyMesh(const char* label, const AcMesh model, const AcMesh candidate)
{
    printf("---Test: %s---\n", label);
    fflush(stdout);
    printf("Errors at the point of the maximum absolute error:\n");
    int errors     = 0;
    const size_t n = acVertexBufferSize(model.info);
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        const AcReal* m = model.vertex_buffer[w];
        const AcReal* c = candidate.vertex_buffer[w];
        Error worst;
        memset(&worst, 0, sizeof(worst));
        worst.abs_error = -1;
        AcReal maxmag = -INFINITY, minmag = INFINITY;
        for (size_t i = 0; i < n; ++i) {
            const Error e = acGetError(m[i], c[i]);
            if (e.abs_error > worst.abs_error)
                worst = e;
            const AcReal a = (AcReal)fabs((double)m[i]);
            maxmag         = a > maxmag ? a : maxmag;
            minmag         = a < minmag ? a : minmag;
        }
        worst.maximum_magnitude = maxmag;
        worst.minimum_magnitude = minmag;
        if (!acEvalError(vtxbuf_names[w], worst))
            ++errors;
    }
    if (errors)
        printf("Failure. Found %d errors\n", errors);
    return errors ? AC_FAILURE : AC_SUCCESS;
}

} // extern "C"

/*
 * astaroth_utils.h -- host-side helpers of the reference utils library
 * (include/astaroth_utils.h:25-77): config loading, host mesh filling and
 * periodic bounds, host reductions and mesh verification.
 *
 * They are exported by the same shared library as astaroth.h. All of them
 * run on the CPU; none is on the GPU path.
 */
#pragma once
#include "astaroth.h"

#ifdef __cplusplus
extern "C" {
#endif

#include <stdbool.h>

typedef struct {
    AcReal model;
    AcReal candidate;
    long double abs_error;
    long double ulp_error;
    long double rel_error;
    AcReal maximum_magnitude;
    AcReal minimum_magnitude;
} Error;

/* Parses `key = value` lines (src/utils/config_loader.c:81-112). Unset words
 * stay 0xFF-filled; returns AC_FAILURE when any word is left unset. */
AcResult acLoadConfig(const char* config_path, AcMeshInfo* config);

AcResult acHostVertexBufferSet(const VertexBufferHandle handle, const AcReal value, AcMesh* mesh);
AcResult acHostMeshSet(const AcReal value, AcMesh* mesh);
/* Fills the ghost zones by periodic wrap (src/utils/memory.c:41-105). */
AcResult acHostMeshApplyPeriodicBounds(AcMesh* mesh);
AcResult acHostMeshClear(AcMesh* mesh);

/* One full RK3 step of the MHD module on the CPU (src/utils/modelsolver.c:987-1041). */
AcResult acHostIntegrateStep(AcMesh mesh, const AcReal dt);

/* Host reductions over the interior; RMS and RMS_EXP are normalised
 * (src/utils/modelreduce.c:76-209). */
AcReal acHostReduceScal(const AcMesh mesh, const ReductionType rtype, const VertexBufferHandle a);
AcReal acHostReduceVec(const AcMesh mesh, const ReductionType rtype, const VertexBufferHandle a,
                       const VertexBufferHandle b, const VertexBufferHandle c);

/* Error at one point and the acceptance rule of src/utils/verification.c:30-102:
 * < 5 ulp, or below the smallest model magnitude times machine epsilon. */
Error acGetError(const AcReal model, const AcReal candidate);
bool acEvalError(const char* label, const Error error);
AcResult acVerifyMesh(const char* label, const AcMesh model, const AcMesh candidate);

#ifdef __cplusplus
} /* extern "C" */
#endif

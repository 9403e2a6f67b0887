/*
 * astaroth.h -- public C interface of the single-device MHD solver.
 *
 * This header is the drop-in boundary: every type, enum value and function
 * prototype below is binary-compatible with the reference interface
 * include/astaroth.h:19-663, so that code written against the reference
 * (its ctest/cpptest/standalone samples, Fortran-style device callers)
 * compiles and links against this library unchanged. The names, argument
 * order and meaning are therefore fixed by the reference; the implementation
 * behind them (astaroth_b200/csrc) is new and B200-specific.
 *
 * Precision is chosen at compile time exactly as in the reference
 * (include/astaroth.h:29-42): AC_DOUBLE_PRECISION=1 selects double, anything
 * else float. Link against the library built for the same precision:
 *   libastaroth_sp.so     AcReal = float,  FP32 kernels
 *   libastaroth_dp.so     AcReal = double, FP64 kernels
 *   libastaroth_mixed.so  AcReal = float at the interface; FP32 stencils and
 *                         right-hand sides with a compensated state (a float hi
 *                         and a bfloat16 lo part) and FP64 reductions inside.
 */
#pragma once
#include <cuda_runtime_api.h> /* int3, float3, double3 */
#include <float.h>            /* FLT_EPSILON, DBL_EPSILON */
#include <stdio.h>            /* printf in acPrintMeshInfo */
#include <stdlib.h>           /* size_t */

/* Sixth-order central differences: three ghost cells on each side. */
#define STENCIL_ORDER (6)
#define NGHOST (STENCIL_ORDER / 2)

#if AC_DOUBLE_PRECISION == 1
typedef double AcReal;
typedef double3 AcReal3;
#define AC_REAL_MAX (DBL_MAX)
#define AC_REAL_MIN (DBL_MIN)
#define AC_REAL_EPSILON (DBL_EPSILON)
#else
typedef float AcReal;
typedef float3 AcReal3;
#define AC_REAL_MAX (FLT_MAX)
#define AC_REAL_MIN (FLT_MIN)
#define AC_REAL_EPSILON (FLT_EPSILON)
#endif

typedef struct {
    AcReal3 row[3];
} AcMatrix;

#include "user_defines.h"

typedef enum { AC_SUCCESS = 0, AC_FAILURE = 1 } AcResult;

typedef enum {
    AC_BOUNDCOND_PERIODIC      = 0,
    AC_BOUNDCOND_SYMMETRIC     = 1,
    AC_BOUNDCOND_ANTISYMMETRIC = 2
} AcBoundcond;

/* Enumerations generated from the tables of user_defines.h. */
#define AC_ENUM_ENTRY(X) X,
typedef enum { AC_FOR_RTYPES(AC_ENUM_ENTRY) NUM_RTYPES } ReductionType;
typedef enum { AC_FOR_USER_INT_PARAM_TYPES(AC_ENUM_ENTRY) NUM_INT_PARAMS } AcIntParam;
typedef enum { AC_FOR_USER_INT3_PARAM_TYPES(AC_ENUM_ENTRY) NUM_INT3_PARAMS } AcInt3Param;
typedef enum { AC_FOR_USER_REAL_PARAM_TYPES(AC_ENUM_ENTRY) NUM_REAL_PARAMS } AcRealParam;
typedef enum { AC_FOR_USER_REAL3_PARAM_TYPES(AC_ENUM_ENTRY) NUM_REAL3_PARAMS } AcReal3Param;
typedef enum {
    AC_FOR_SCALARARRAY_HANDLES(AC_ENUM_ENTRY) NUM_SCALARARRAY_HANDLES
} ScalarArrayHandle;
typedef enum { AC_FOR_VTXBUF_HANDLES(AC_ENUM_ENTRY) NUM_VTXBUF_HANDLES } VertexBufferHandle;
#undef AC_ENUM_ENTRY

/* Printable names, indexed by the enums above (terminated by "-end-"). */
#define AC_NAME_ENTRY(X) #X,
#define AC_MAYBE_UNUSED __attribute__((unused))
static const char* rtype_names[] AC_MAYBE_UNUSED     = {AC_FOR_RTYPES(AC_NAME_ENTRY) "-end-"};
static const char* intparam_names[] AC_MAYBE_UNUSED  = {
    AC_FOR_USER_INT_PARAM_TYPES(AC_NAME_ENTRY) "-end-"};
static const char* int3param_names[] AC_MAYBE_UNUSED = {
    AC_FOR_USER_INT3_PARAM_TYPES(AC_NAME_ENTRY) "-end-"};
static const char* realparam_names[] AC_MAYBE_UNUSED = {
    AC_FOR_USER_REAL_PARAM_TYPES(AC_NAME_ENTRY) "-end-"};
static const char* real3param_names[] AC_MAYBE_UNUSED = {
    AC_FOR_USER_REAL3_PARAM_TYPES(AC_NAME_ENTRY) "-end-"};
static const char* scalararray_names[] AC_MAYBE_UNUSED = {
    AC_FOR_SCALARARRAY_HANDLES(AC_NAME_ENTRY) "-end-"};
static const char* vtxbuf_names[] AC_MAYBE_UNUSED = {AC_FOR_VTXBUF_HANDLES(AC_NAME_ENTRY) "-end-"};
#undef AC_NAME_ENTRY
#undef AC_MAYBE_UNUSED

/* Run-time parameters. The layout (ints, int3s, reals, real3s) is fixed by
 * the reference (include/astaroth.h:109-114). */
typedef struct {
    int int_params[NUM_INT_PARAMS];
    int3 int3_params[NUM_INT3_PARAMS];
    AcReal real_params[NUM_REAL_PARAMS];
    AcReal3 real3_params[NUM_REAL3_PARAMS];
} AcMeshInfo;

/* A host mesh: one mx*my*mz array per field, idx = i + j*mx + k*mx*my. */
typedef struct {
    AcReal* vertex_buffer[NUM_VTXBUF_HANDLES];
    AcMeshInfo info;
} AcMesh;

typedef struct device_s* Device; /* opaque, owned by acDeviceCreate/Destroy */
typedef struct node_s* Node;     /* opaque, owned by acNodeCreate/Destroy */

typedef struct {
    int3 m;
    int3 n;
} GridDims;

typedef struct {
    int num_devices;
    Device* devices;

    GridDims grid;
    GridDims subgrid;
} DeviceConfiguration;

#ifdef __cplusplus
extern "C" {
#endif

/* ---- inline index helpers (include/astaroth.h:153-199) ------------------ */
static inline size_t
acVertexBufferSize(const AcMeshInfo info)
{
    return (size_t)info.int_params[AC_mx] * (size_t)info.int_params[AC_my] *
           (size_t)info.int_params[AC_mz];
}

static inline size_t
acVertexBufferSizeBytes(const AcMeshInfo info)
{
    return sizeof(AcReal) * acVertexBufferSize(info);
}

static inline size_t
acVertexBufferCompdomainSize(const AcMeshInfo info)
{
    return (size_t)info.int_params[AC_nx] * (size_t)info.int_params[AC_ny] *
           (size_t)info.int_params[AC_nz];
}

static inline size_t
acVertexBufferCompdomainSizeBytes(const AcMeshInfo info)
{
    return sizeof(AcReal) * acVertexBufferCompdomainSize(info);
}

static inline size_t
acVertexBufferIdx(const int i, const int j, const int k, const AcMeshInfo info)
{
    return (size_t)i + (size_t)j * (size_t)info.int_params[AC_mx] +
           (size_t)k * (size_t)info.int_params[AC_mx] * (size_t)info.int_params[AC_my];
}

static inline void
acPrintMeshInfo(const AcMeshInfo config)
{
    for (int i = 0; i < NUM_INT_PARAMS; ++i)
        printf("[%s]: %d\n", intparam_names[i], config.int_params[i]);
    for (int i = 0; i < NUM_INT3_PARAMS; ++i)
        printf("[%s]: (%d, %d, %d)\n", int3param_names[i], config.int3_params[i].x,
               config.int3_params[i].y, config.int3_params[i].z);
    for (int i = 0; i < NUM_REAL_PARAMS; ++i)
        printf("[%s]: %g\n", realparam_names[i], (double)(config.real_params[i]));
}

/* ---- Legacy interface: one node, synchronous (include/astaroth.h:208-283) */
AcResult acInit(const AcMeshInfo mesh_info);
AcResult acQuit(void);
AcResult acCheckDeviceAvailability(void);
AcResult acSynchronizeStream(const Stream stream);
AcResult acSynchronizeMesh(void);
AcResult acLoadDeviceConstant(const AcRealParam param, const AcReal value);
AcResult acLoad(const AcMesh host_mesh);
AcResult acSetVertexBuffer(const VertexBufferHandle handle, const AcReal value);
AcResult acStore(AcMesh* host_mesh);
/* One full RK3 step; boundary conditions are NOT applied after the last
 * substep (call acBoundcondStep before reading ghost zones). */
AcResult acIntegrate(const AcReal dt);
AcResult acIntegrateGBC(const AcMeshInfo config, const AcReal dt);
AcResult acBoundcondStep(void);
AcResult acBoundcondStepGBC(const AcMeshInfo config);
AcReal acReduceScal(const ReductionType rtype, const VertexBufferHandle vtxbuf_handle);
AcReal acReduceVec(const ReductionType rtype, const VertexBufferHandle a,
                   const VertexBufferHandle b, const VertexBufferHandle c);
AcReal acReduceVecScal(const ReductionType rtype, const VertexBufferHandle a,
                       const VertexBufferHandle b, const VertexBufferHandle c,
                       const VertexBufferHandle d);
AcResult acStoreWithOffset(const int3 dst, const size_t num_vertices, AcMesh* host_mesh);
AcResult acIntegrateStep(const int isubstep, const AcReal dt);
AcResult acIntegrateStepWithOffset(const int isubstep, const AcReal dt, const int3 start,
                                   const int3 end);
AcResult acSynchronize(void);
AcResult acLoadWithOffset(const AcMesh host_mesh, const int3 src, const int num_vertices);
int acGetNumDevicesPerNode(void);
Node acGetNode(void);

/* ---- Node interface, single device (include/astaroth.h:360-499) --------- */
AcResult acNodeCreate(const int id, const AcMeshInfo node_config, Node* node);
AcResult acNodeDestroy(Node node);
AcResult acNodePrintInfo(const Node node);
AcResult acNodeQueryDeviceConfiguration(const Node node, DeviceConfiguration* config);
AcResult acNodeAutoOptimize(const Node node);
AcResult acNodeSynchronizeStream(const Node node, const Stream stream);
AcResult acNodeSynchronizeVertexBuffer(const Node node, const Stream stream,
                                       const VertexBufferHandle vtxbuf_handle);
AcResult acNodeSynchronizeMesh(const Node node, const Stream stream);
AcResult acNodeSwapBuffers(const Node node);
AcResult acNodeLoadConstant(const Node node, const Stream stream, const AcRealParam param,
                            const AcReal value);
AcResult acNodeLoadVertexBufferWithOffset(const Node node, const Stream stream,
                                          const AcMesh host_mesh,
                                          const VertexBufferHandle vtxbuf_handle, const int3 src,
                                          const int3 dst, const int num_vertices);
AcResult acNodeLoadMeshWithOffset(const Node node, const Stream stream, const AcMesh host_mesh,
                                  const int3 src, const int3 dst, const int num_vertices);
AcResult acNodeLoadVertexBuffer(const Node node, const Stream stream, const AcMesh host_mesh,
                                const VertexBufferHandle vtxbuf_handle);
AcResult acNodeLoadMesh(const Node node, const Stream stream, const AcMesh host_mesh);
AcResult acNodeSetVertexBuffer(const Node node, const Stream stream,
                               const VertexBufferHandle handle, const AcReal value);
AcResult acNodeStoreVertexBufferWithOffset(const Node node, const Stream stream,
                                           const VertexBufferHandle vtxbuf_handle, const int3 src,
                                           const int3 dst, const int num_vertices,
                                           AcMesh* host_mesh);
AcResult acNodeStoreMeshWithOffset(const Node node, const Stream stream, const int3 src,
                                   const int3 dst, const int num_vertices, AcMesh* host_mesh);
AcResult acNodeStoreVertexBuffer(const Node node, const Stream stream,
                                 const VertexBufferHandle vtxbuf_handle, AcMesh* host_mesh);
AcResult acNodeStoreMesh(const Node node, const Stream stream, AcMesh* host_mesh);
AcResult acNodeIntegrateSubstep(const Node node, const Stream stream, const int step_number,
                                const int3 start, const int3 end, const AcReal dt);
AcResult acNodeIntegrate(const Node node, const AcReal dt);
AcResult acNodeIntegrateGBC(const Node node, const AcMeshInfo config, const AcReal dt);
AcResult acNodePeriodicBoundcondStep(const Node node, const Stream stream,
                                     const VertexBufferHandle vtxbuf_handle);
AcResult acNodePeriodicBoundconds(const Node node, const Stream stream);
AcResult acNodeGeneralBoundcondStep(const Node node, const Stream stream,
                                    const VertexBufferHandle vtxbuf_handle,
                                    const AcMeshInfo config);
AcResult acNodeGeneralBoundconds(const Node node, const Stream stream, const AcMeshInfo config);
AcResult acNodeReduceScal(const Node node, const Stream stream, const ReductionType rtype,
                          const VertexBufferHandle vtxbuf_handle, AcReal* result);
AcResult acNodeReduceVec(const Node node, const Stream stream_type, const ReductionType rtype,
                         const VertexBufferHandle vtxbuf0, const VertexBufferHandle vtxbuf1,
                         const VertexBufferHandle vtxbuf2, AcReal* result);
AcResult acNodeReduceVecScal(const Node node, const Stream stream_type, const ReductionType rtype,
                             const VertexBufferHandle vtxbuf0, const VertexBufferHandle vtxbuf1,
                             const VertexBufferHandle vtxbuf2, const VertexBufferHandle vtxbuf3,
                             AcReal* result);

/* ---- Device interface: the hot path (include/astaroth.h:506-642) -------- */
AcResult acDeviceCreate(const int id, const AcMeshInfo device_config, Device* device);
AcResult acDeviceDestroy(Device device);
AcResult acDevicePrintInfo(const Device device);
AcResult acDeviceAutoOptimize(const Device device);
AcResult acDeviceSynchronizeStream(const Device device, const Stream stream);
AcResult acDeviceSwapBuffers(const Device device);
AcResult acDeviceLoadScalarUniform(const Device device, const Stream stream,
                                   const AcRealParam param, const AcReal value);
AcResult acDeviceLoadVectorUniform(const Device device, const Stream stream,
                                   const AcReal3Param param, const AcReal3 value);
AcResult acDeviceLoadIntUniform(const Device device, const Stream stream, const AcIntParam param,
                                const int value);
AcResult acDeviceLoadInt3Uniform(const Device device, const Stream stream, const AcInt3Param param,
                                 const int3 value);
AcResult acDeviceLoadScalarArray(const Device device, const Stream stream,
                                 const ScalarArrayHandle handle, const size_t start,
                                 const AcReal* data, const size_t num);
AcResult acDeviceLoadMeshInfo(const Device device, const AcMeshInfo device_config);
AcResult acDeviceLoadDefaultUniforms(const Device device);
AcResult acDeviceLoadVertexBufferWithOffset(const Device device, const Stream stream,
                                            const AcMesh host_mesh,
                                            const VertexBufferHandle vtxbuf_handle, const int3 src,
                                            const int3 dst, const int num_vertices);
AcResult acDeviceLoadMeshWithOffset(const Device device, const Stream stream,
                                    const AcMesh host_mesh, const int3 src, const int3 dst,
                                    const int num_vertices);
AcResult acDeviceLoadVertexBuffer(const Device device, const Stream stream, const AcMesh host_mesh,
                                  const VertexBufferHandle vtxbuf_handle);
AcResult acDeviceLoadMesh(const Device device, const Stream stream, const AcMesh host_mesh);
AcResult acDeviceSetVertexBuffer(const Device device, const Stream stream,
                                 const VertexBufferHandle handle, const AcReal value);
AcResult acDeviceStoreVertexBufferWithOffset(const Device device, const Stream stream,
                                             const VertexBufferHandle vtxbuf_handle, const int3 src,
                                             const int3 dst, const int num_vertices,
                                             AcMesh* host_mesh);
AcResult acDeviceStoreMeshWithOffset(const Device device, const Stream stream, const int3 src,
                                     const int3 dst, const int num_vertices, AcMesh* host_mesh);
AcResult acDeviceStoreVertexBuffer(const Device device, const Stream stream,
                                   const VertexBufferHandle vtxbuf_handle, AcMesh* host_mesh);
AcResult acDeviceStoreMesh(const Device device, const Stream stream, AcMesh* host_mesh);
AcResult acDeviceTransferVertexBufferWithOffset(const Device src_device, const Stream stream,
                                                const VertexBufferHandle vtxbuf_handle,
                                                const int3 src, const int3 dst,
                                                const int num_vertices, Device dst_device);
AcResult acDeviceTransferMeshWithOffset(const Device src_device, const Stream stream,
                                        const int3 src, const int3 dst, const int num_vertices,
                                        Device* dst_device);
AcResult acDeviceTransferVertexBuffer(const Device src_device, const Stream stream,
                                      const VertexBufferHandle vtxbuf_handle, Device dst_device);
AcResult acDeviceTransferMesh(const Device src_device, const Stream stream, Device dst_device);
/* One RK3 substep over the box [start, end): reads the stencils of the `in`
 * buffers and the previous state from `out`, writes `out` (interior only). */
AcResult acDeviceIntegrateSubstep(const Device device, const Stream stream, const int step_number,
                                  const int3 start, const int3 end, const AcReal dt);
AcResult acDevicePeriodicBoundcondStep(const Device device, const Stream stream,
                                       const VertexBufferHandle vtxbuf_handle, const int3 start,
                                       const int3 end);
AcResult acDevicePeriodicBoundconds(const Device device, const Stream stream, const int3 start,
                                    const int3 end);
AcResult acDeviceGeneralBoundcondStep(const Device device, const Stream stream,
                                      const VertexBufferHandle vtxbuf_handle, const int3 start,
                                      const int3 end, const AcMeshInfo config, const int3 bindex);
AcResult acDeviceGeneralBoundconds(const Device device, const Stream stream, const int3 start,
                                   const int3 end, const AcMeshInfo config, const int3 bindex);
/* Reductions over the interior of `in`. RTYPE_RMS and RTYPE_RMS_EXP return
 * the raw sum of squares here; the Node and Legacy layers normalise it. */
AcResult acDeviceReduceScal(const Device device, const Stream stream, const ReductionType rtype,
                            const VertexBufferHandle vtxbuf_handle, AcReal* result);
AcResult acDeviceReduceVec(const Device device, const Stream stream_type, const ReductionType rtype,
                           const VertexBufferHandle vtxbuf0, const VertexBufferHandle vtxbuf1,
                           const VertexBufferHandle vtxbuf2, AcReal* result);
AcResult acDeviceReduceVecScal(const Device device, const Stream stream_type,
                               const ReductionType rtype, const VertexBufferHandle vtxbuf0,
                               const VertexBufferHandle vtxbuf1, const VertexBufferHandle vtxbuf2,
                               const VertexBufferHandle vtxbuf3, AcReal* result);
/* Declared by the reference (include/astaroth.h:642) but never defined
 * there; here it reports AC_FAILURE (no MPI layer). */
AcResult acDeviceRunMPITest(void);

/* ---- Host helpers (include/astaroth.h:650-659) -------------------------- */
AcResult acHostUpdateBuiltinParams(AcMeshInfo* config);
AcResult acHostMeshCreate(const AcMeshInfo mesh_info, AcMesh* mesh);
AcResult acHostMeshRandomize(AcMesh* mesh);
AcResult acHostMeshDestroy(AcMesh* mesh);

#ifdef __cplusplus
} /* extern "C" */
#endif

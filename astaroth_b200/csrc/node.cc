// Node and Legacy layers of include/astaroth.h on one device, and the host
// mesh helpers.
//
// Reference: src/core/node.cc:133-1007 (Node), src/core/astaroth.cc:24-267
// (Legacy and host helpers). The reference Node splits the mesh into z-slabs
// over every visible GPU and splits each substep into an inner box and six
// boundary slabs on seven streams so that halo transfers can overlap. With one
// device there is nothing to overlap: a substep here is one periodic fill of
// all fields and one launch of the fused kernel over the whole interior.
#include <cuda_runtime.h> // make_int3
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "astaroth.h"
#include "astaroth_b200.h"

struct node_s {
    int id;
    Device device;
    GridDims grid;
    AcMeshInfo config;
};

static GridDims
grid_dims(const AcMeshInfo& c)
{
    GridDims g;
    g.m = make_int3(c.int_params[AC_mx], c.int_params[AC_my], c.int_params[AC_mz]);
    g.n = make_int3(c.int_params[AC_nx], c.int_params[AC_ny], c.int_params[AC_nz]);
    return g;
}

static inline int3
max3(int3 a, int3 b)
{
    return make_int3(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z);
}

static inline int3
min3(int3 a, int3 b)
{
    return make_int3(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z);
}

extern "C" {

// ---------------------------------------------------------------------------
// host helpers (src/core/astaroth.cc:190-267)
// ---------------------------------------------------------------------------
AcResult
acHostUpdateBuiltinParams(AcMeshInfo* c)
{
    int* ip       = c->int_params;
    ip[AC_mx]     = ip[AC_nx] + STENCIL_ORDER;
    ip[AC_my]     = ip[AC_ny] + STENCIL_ORDER;
    ip[AC_mz]     = ip[AC_nz] + STENCIL_ORDER;
    ip[AC_nx_min] = STENCIL_ORDER / 2;
    ip[AC_nx_max] = ip[AC_nx_min] + ip[AC_nx];
    ip[AC_ny_min] = STENCIL_ORDER / 2;
    ip[AC_ny_max] = ip[AC_ny] + STENCIL_ORDER / 2;
    ip[AC_nz_min] = STENCIL_ORDER / 2;
    ip[AC_nz_max] = ip[AC_nz] + STENCIL_ORDER / 2;
    c->real_params[AC_inv_dsx] = (AcReal)(1.) / c->real_params[AC_dsx];
    c->real_params[AC_inv_dsy] = (AcReal)(1.) / c->real_params[AC_dsy];
    c->real_params[AC_inv_dsz] = (AcReal)(1.) / c->real_params[AC_dsz];
    ip[AC_mxy]  = ip[AC_mx] * ip[AC_my];
    ip[AC_nxy]  = ip[AC_nx] * ip[AC_ny];
    ip[AC_nxyz] = ip[AC_nxy] * ip[AC_nz];
    return AC_SUCCESS;
}

AcResult
acHostMeshCreate(const AcMeshInfo info, AcMesh* mesh)
{
    mesh->info         = info;
    const size_t bytes = acVertexBufferSizeBytes(info);
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        mesh->vertex_buffer[w] = (AcReal*)malloc(bytes);
        if (!mesh->vertex_buffer[w]) {
            fprintf(stderr, "acHostMeshCreate: out of host memory\n");
            exit(EXIT_FAILURE);
        }
    }
    return AC_SUCCESS;
}

AcResult
acHostMeshRandomize(AcMesh* mesh)
{
    const size_t n = acVertexBufferSize(mesh->info);
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w)
        for (size_t i = 0; i < n; ++i)
            mesh->vertex_buffer[w][i] = (AcReal)rand() / (AcReal)RAND_MAX;
    return AC_SUCCESS;
}

AcResult
acHostMeshDestroy(AcMesh* mesh)
{
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        free(mesh->vertex_buffer[w]);
        mesh->vertex_buffer[w] = NULL;
    }
    return AC_SUCCESS;
}

// ---------------------------------------------------------------------------
// Node (single device)
// ---------------------------------------------------------------------------
AcResult
acNodeCreate(const int id, const AcMeshInfo node_config, Node* node_handle)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        fprintf(stderr, "ERROR: No CUDA devices found!\n");
        return AC_FAILURE;
    }
    struct node_s* node = (struct node_s*)calloc(1, sizeof(struct node_s));
    node->id            = id;
    node->config        = node_config;
    node->grid          = grid_dims(node_config);
    if (node->grid.n.x < STENCIL_ORDER || node->grid.n.y < STENCIL_ORDER ||
        node->grid.n.z < STENCIL_ORDER) {
        fprintf(stderr, "ERROR: mesh smaller than the stencil\n");
        free(node);
        return AC_FAILURE;
    }
    AcMeshInfo dev_config                       = node_config;
    dev_config.int3_params[AC_global_grid_n]    = node->grid.n;
    dev_config.int3_params[AC_multigpu_offset]  = make_int3(0, 0, 0);
    node->config                                = dev_config;
    if (acDeviceCreate(0, dev_config, &node->device) != AC_SUCCESS) {
        free(node);
        return AC_FAILURE;
    }
    *node_handle = node;
    return AC_SUCCESS;
}

AcResult
acNodeDestroy(Node node)
{
    if (!node)
        return AC_FAILURE;
    acDeviceDestroy(node->device);
    free(node);
    return AC_SUCCESS;
}

AcResult
acNodePrintInfo(const Node node)
{
    return acDevicePrintInfo(node->device);
}

AcResult
acNodeQueryDeviceConfiguration(const Node node, DeviceConfiguration* config)
{
    config->num_devices = 1;
    config->devices     = &node->device;
    config->grid        = node->grid;
    config->subgrid     = node->grid;
    return AC_SUCCESS;
}

AcResult
acNodeAutoOptimize(const Node node)
{
    return acDeviceAutoOptimize(node->device);
}

AcResult
acNodeSynchronizeStream(const Node node, const Stream stream)
{
    return acDeviceSynchronizeStream(node->device, stream);
}

AcResult
acNodeSynchronizeVertexBuffer(const Node node, const Stream stream,
                              const VertexBufferHandle vtxbuf_handle)
{
    (void)vtxbuf_handle; // no neighbouring subgrids with one device
    return acNodeSynchronizeStream(node, stream);
}

AcResult
acNodeSynchronizeMesh(const Node node, const Stream stream)
{
    return acNodeSynchronizeStream(node, stream);
}

AcResult
acNodeSwapBuffers(const Node node)
{
    return acDeviceSwapBuffers(node->device);
}

AcResult
acNodeLoadConstant(const Node node, const Stream stream, const AcRealParam param,
                   const AcReal value)
{
    acNodeSynchronizeStream(node, stream);
    return acDeviceLoadScalarUniform(node->device, stream, param, value);
}

AcResult
acNodeLoadVertexBufferWithOffset(const Node node, const Stream stream, const AcMesh host_mesh,
                                 const VertexBufferHandle vtxbuf_handle, const int3 src,
                                 const int3 dst, const int num_vertices)
{
    (void)dst; // the reference maps src to both ends (src/core/node.cc:497-520)
    acNodeSynchronizeStream(node, stream);
    return acDeviceLoadVertexBufferWithOffset(node->device, stream, host_mesh, vtxbuf_handle, src,
                                              src, num_vertices);
}

AcResult
acNodeLoadMeshWithOffset(const Node node, const Stream stream, const AcMesh host_mesh,
                         const int3 src, const int3 dst, const int num_vertices)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acNodeLoadVertexBufferWithOffset(node, stream, host_mesh, (VertexBufferHandle)i, src,
                                             dst, num_vertices) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acNodeLoadVertexBuffer(const Node node, const Stream stream, const AcMesh host_mesh,
                       const VertexBufferHandle vtxbuf_handle)
{
    const int3 z = make_int3(0, 0, 0);
    return acNodeLoadVertexBufferWithOffset(node, stream, host_mesh, vtxbuf_handle, z, z,
                                            (int)acVertexBufferSize(host_mesh.info));
}

AcResult
acNodeLoadMesh(const Node node, const Stream stream, const AcMesh host_mesh)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acNodeLoadVertexBuffer(node, stream, host_mesh, (VertexBufferHandle)i) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acNodeSetVertexBuffer(const Node node, const Stream stream, const VertexBufferHandle handle,
                      const AcReal value)
{
    acNodeSynchronizeStream(node, stream);
    const AcResult r = acDeviceSetVertexBuffer(node->device, stream, handle, value);
    acNodeSynchronizeStream(node, stream);
    return r;
}

AcResult
acNodeStoreVertexBufferWithOffset(const Node node, const Stream stream,
                                  const VertexBufferHandle vtxbuf_handle, const int3 src,
                                  const int3 dst, const int num_vertices, AcMesh* host_mesh)
{
    (void)dst;
    acNodeSynchronizeStream(node, stream);
    return acDeviceStoreVertexBufferWithOffset(node->device, stream, vtxbuf_handle, src, src,
                                               num_vertices, host_mesh);
}

AcResult
acNodeStoreMeshWithOffset(const Node node, const Stream stream, const int3 src, const int3 dst,
                          const int num_vertices, AcMesh* host_mesh)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acNodeStoreVertexBufferWithOffset(node, stream, (VertexBufferHandle)i, src, dst,
                                              num_vertices, host_mesh) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acNodeStoreVertexBuffer(const Node node, const Stream stream,
                        const VertexBufferHandle vtxbuf_handle, AcMesh* host_mesh)
{
    const int3 z = make_int3(0, 0, 0);
    return acNodeStoreVertexBufferWithOffset(node, stream, vtxbuf_handle, z, z,
                                             (int)acVertexBufferSize(host_mesh->info), host_mesh);
}

AcResult
acNodeStoreMesh(const Node node, const Stream stream, AcMesh* host_mesh)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acNodeStoreVertexBuffer(node, stream, (VertexBufferHandle)i, host_mesh) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acNodeIntegrateSubstep(const Node node, const Stream stream, const int isubstep,
                       const int3 start, const int3 end, const AcReal dt)
{
    acNodeSynchronizeStream(node, stream);
    const int3 d0 = make_int3(NGHOST, NGHOST, NGHOST);
    const int3 d1 = make_int3(NGHOST + node->grid.n.x, NGHOST + node->grid.n.y,
                              NGHOST + node->grid.n.z);
    const int3 da = max3(start, d0);
    const int3 db = min3(end, d1);
    if (db.x <= da.x || db.y <= da.y || db.z <= da.z)
        return AC_SUCCESS;
    return acDeviceIntegrateSubstep(node->device, stream, isubstep, da, db, dt);
}

AcResult
acNodeIntegrate(const Node node, const AcReal dt)
{
    acNodeSynchronizeStream(node, STREAM_ALL);
    // Boundary conditions before each substep, not after the last one
    // (src/core/node.cc:728-805).
    if (acDeviceIntegrateStep(node->device, STREAM_DEFAULT, dt) != AC_SUCCESS)
        return AC_FAILURE;
    return acNodeSynchronizeStream(node, STREAM_ALL);
}

AcResult
acNodePeriodicBoundcondStep(const Node node, const Stream stream,
                            const VertexBufferHandle vtxbuf_handle)
{
    acNodeSynchronizeStream(node, stream);
    const int3 z = make_int3(0, 0, 0);
    return acDevicePeriodicBoundcondStep(node->device, stream, vtxbuf_handle, z, node->grid.m);
}

AcResult
acNodePeriodicBoundconds(const Node node, const Stream stream)
{
    acNodeSynchronizeStream(node, stream);
    const int3 z = make_int3(0, 0, 0);
    return acDevicePeriodicBoundconds(node->device, stream, z, node->grid.m);
}

AcResult
acNodeGeneralBoundcondStep(const Node node, const Stream stream,
                           const VertexBufferHandle vtxbuf_handle, const AcMeshInfo config)
{
    acNodeSynchronizeStream(node, stream);
    const int3 z      = make_int3(0, 0, 0);
    const int3 bindex = make_int3(-1, -1, -1);
    return acDeviceGeneralBoundcondStep(node->device, stream, vtxbuf_handle, z, node->grid.m,
                                        config, bindex);
}

AcResult
acNodeGeneralBoundconds(const Node node, const Stream stream, const AcMeshInfo config)
{
    for (int i = 0; i < NUM_VTXBUF_HANDLES; ++i)
        if (acNodeGeneralBoundcondStep(node, stream, (VertexBufferHandle)i, config) != AC_SUCCESS)
            return AC_FAILURE;
    return AC_SUCCESS;
}

AcResult
acNodeIntegrateGBC(const Node node, const AcMeshInfo config, const AcReal dt)
{
    acNodeSynchronizeStream(node, STREAM_ALL);
    const int3 d0 = make_int3(NGHOST, NGHOST, NGHOST);
    const int3 d1 = make_int3(NGHOST + node->grid.n.x, NGHOST + node->grid.n.y,
                              NGHOST + node->grid.n.z);
    for (int s = 0; s < 3; ++s) {
        if (acNodeGeneralBoundconds(node, STREAM_DEFAULT, config) != AC_SUCCESS)
            return AC_FAILURE;
        if (acDeviceIntegrateSubstep(node->device, STREAM_DEFAULT, s, d0, d1, dt) != AC_SUCCESS)
            return AC_FAILURE;
        acDeviceSwapBuffers(node->device);
    }
    return acNodeSynchronizeStream(node, STREAM_ALL);
}

// RMS, RMS_EXP and ALFVEN_RMS are normalised here, not in the device layer
// (src/core/node.cc:931-956).
static AcReal
node_finalise(const Node node, const ReductionType rtype, double raw)
{
    if (rtype == RTYPE_RMS || rtype == RTYPE_RMS_EXP || rtype == RTYPE_ALFVEN_RMS) {
        const double inv_n = 1.0 / ((double)node->grid.n.x * node->grid.n.y * node->grid.n.z);
        return (AcReal)sqrt(inv_n * raw);
    }
    return (AcReal)raw;
}

AcResult
acNodeReduceScal(const Node node, const Stream stream, const ReductionType rtype,
                 const VertexBufferHandle vtxbuf_handle, AcReal* result)
{
    acNodeSynchronizeStream(node, STREAM_ALL);
    double raw        = 0;
    const AcResult rc = acDeviceReduceScalDouble(node->device, stream, rtype, vtxbuf_handle, &raw);
    *result           = node_finalise(node, rtype, raw);
    return rc;
}

AcResult
acNodeReduceVec(const Node node, const Stream stream, const ReductionType rtype,
                const VertexBufferHandle a, const VertexBufferHandle b, const VertexBufferHandle c,
                AcReal* result)
{
    acNodeSynchronizeStream(node, STREAM_ALL);
    double raw        = 0;
    const AcResult rc = acDeviceReduceVecDouble(node->device, stream, rtype, a, b, c, &raw);
    *result           = node_finalise(node, rtype, raw);
    return rc;
}

AcResult
acNodeReduceVecScal(const Node node, const Stream stream, const ReductionType rtype,
                    const VertexBufferHandle a, const VertexBufferHandle b,
                    const VertexBufferHandle c, const VertexBufferHandle d, AcReal* result)
{
    acNodeSynchronizeStream(node, STREAM_ALL);
    AcReal raw        = 0;
    const AcResult rc = acDeviceReduceVecScal(node->device, stream, rtype, a, b, c, d, &raw);
    *result           = node_finalise(node, rtype, (double)raw);
    return rc;
}

// ---------------------------------------------------------------------------
// Legacy interface (src/core/astaroth.cc:24-188): one static node
// ---------------------------------------------------------------------------
static Node g_node = NULL;

AcResult
acInit(const AcMeshInfo mesh_info)
{
    return acNodeCreate(0, mesh_info, &g_node);
}

AcResult
acQuit(void)
{
    const AcResult r = acNodeDestroy(g_node);
    g_node           = NULL;
    return r;
}

AcResult
acCheckDeviceAvailability(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
        return AC_FAILURE;
    return n > 0 ? AC_SUCCESS : AC_FAILURE;
}

AcResult
acSynchronize(void)
{
    return acNodeSynchronizeStream(g_node, STREAM_ALL);
}

AcResult
acSynchronizeStream(const Stream stream)
{
    return acNodeSynchronizeStream(g_node, stream);
}

AcResult
acLoadDeviceConstant(const AcRealParam param, const AcReal value)
{
    return acNodeLoadConstant(g_node, STREAM_DEFAULT, param, value);
}

AcResult
acLoad(const AcMesh host_mesh)
{
    return acNodeLoadMesh(g_node, STREAM_DEFAULT, host_mesh);
}

AcResult
acSetVertexBuffer(const VertexBufferHandle handle, const AcReal value)
{
    return acNodeSetVertexBuffer(g_node, STREAM_DEFAULT, handle, value);
}

AcResult
acStore(AcMesh* host_mesh)
{
    const AcResult r = acNodeStoreMesh(g_node, STREAM_DEFAULT, host_mesh);
    acNodeSynchronizeStream(g_node, STREAM_DEFAULT);
    return r;
}

AcResult
acIntegrate(const AcReal dt)
{
    return acNodeIntegrate(g_node, dt);
}

AcResult
acIntegrateGBC(const AcMeshInfo config, const AcReal dt)
{
    return acNodeIntegrateGBC(g_node, config, dt);
}

AcResult
acIntegrateStep(const int isubstep, const AcReal dt)
{
    const int3 start = make_int3(NGHOST, NGHOST, NGHOST);
    const int3 end   = make_int3(NGHOST + g_node->grid.n.x, NGHOST + g_node->grid.n.y,
                               NGHOST + g_node->grid.n.z);
    return acNodeIntegrateSubstep(g_node, STREAM_DEFAULT, isubstep, start, end, dt);
}

AcResult
acIntegrateStepWithOffset(const int isubstep, const AcReal dt, const int3 start, const int3 end)
{
    return acNodeIntegrateSubstep(g_node, STREAM_DEFAULT, isubstep, start, end, dt);
}

AcResult
acBoundcondStep(void)
{
    return acNodePeriodicBoundconds(g_node, STREAM_DEFAULT);
}

AcResult
acBoundcondStepGBC(const AcMeshInfo config)
{
    return acNodeGeneralBoundconds(g_node, STREAM_DEFAULT, config);
}

AcReal
acReduceScal(const ReductionType rtype, const VertexBufferHandle vtxbuf_handle)
{
    AcReal result = 0;
    acNodeReduceScal(g_node, STREAM_DEFAULT, rtype, vtxbuf_handle, &result);
    return result;
}

AcReal
acReduceVec(const ReductionType rtype, const VertexBufferHandle a, const VertexBufferHandle b,
            const VertexBufferHandle c)
{
    AcReal result = 0;
    acNodeReduceVec(g_node, STREAM_DEFAULT, rtype, a, b, c, &result);
    return result;
}

AcReal
acReduceVecScal(const ReductionType rtype, const VertexBufferHandle a, const VertexBufferHandle b,
                const VertexBufferHandle c, const VertexBufferHandle d)
{
    AcReal result = 0;
    acNodeReduceVecScal(g_node, STREAM_DEFAULT, rtype, a, b, c, d, &result);
    return result;
}

AcResult
acStoreWithOffset(const int3 dst, const size_t num_vertices, AcMesh* host_mesh)
{
    const AcResult r = acNodeStoreMeshWithOffset(g_node, STREAM_DEFAULT, dst, dst,
                                                 (int)num_vertices, host_mesh);
    acNodeSynchronizeStream(g_node, STREAM_DEFAULT);
    return r;
}

AcResult
acLoadWithOffset(const AcMesh host_mesh, const int3 src, const int num_vertices)
{
    return acNodeLoadMeshWithOffset(g_node, STREAM_DEFAULT, host_mesh, src, src, num_vertices);
}

AcResult
acSynchronizeMesh(void)
{
    return acNodeSynchronizeMesh(g_node, STREAM_DEFAULT);
}

int
acGetNumDevicesPerNode(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
        return 0;
    return n;
}

Node
acGetNode(void)
{
    if (!g_node) {
        fprintf(stderr, "ERROR: acGetNode before acInit\n");
        exit(EXIT_FAILURE);
    }
    return g_node;
}

} // extern "C"

/*
 * ref_shim.c -- TEST INFRASTRUCTURE ONLY. Link-time helpers for building the
 * reference's own host utils (src/utils/*.c) into oracle/_ref without its CUDA
 * core library.
 *
 * The reference's modelsolver.c calls acHostMeshCreate/acHostMeshDestroy and
 * its config loader calls acHostUpdateBuiltinParams; the reference defines all
 * three in its GPU core library (src/core/astaroth.cc:190-267). This shim gives
 * plain host definitions with the same behaviour (malloc'd mx*my*mz buffers;
 * m = n + 6, bounds [3, 3+n), inverse spacings) so the utils build as a
 * standalone CPU library.
 */
#include <stdlib.h>

#include "astaroth.h"

AcResult
acHostUpdateBuiltinParams(AcMeshInfo* config)
{
    int* ip                = config->int_params;
    ip[AC_mx]              = ip[AC_nx] + STENCIL_ORDER;
    ip[AC_my]              = ip[AC_ny] + STENCIL_ORDER;
    ip[AC_mz]              = ip[AC_nz] + STENCIL_ORDER;
    ip[AC_nx_min]          = NGHOST;
    ip[AC_ny_min]          = NGHOST;
    ip[AC_nz_min]          = NGHOST;
    ip[AC_nx_max]          = NGHOST + ip[AC_nx];
    ip[AC_ny_max]          = NGHOST + ip[AC_ny];
    ip[AC_nz_max]          = NGHOST + ip[AC_nz];
    config->real_params[AC_inv_dsx] = (AcReal)(1.) / config->real_params[AC_dsx];
    config->real_params[AC_inv_dsy] = (AcReal)(1.) / config->real_params[AC_dsy];
    config->real_params[AC_inv_dsz] = (AcReal)(1.) / config->real_params[AC_dsz];
    ip[AC_mxy]             = ip[AC_mx] * ip[AC_my];
    ip[AC_nxy]             = ip[AC_nx] * ip[AC_ny];
    ip[AC_nxyz]            = ip[AC_nxy] * ip[AC_nz];
    return AC_SUCCESS;
}

AcResult
acHostMeshCreate(const AcMeshInfo info, AcMesh* mesh)
{
    mesh->info         = info;
    const size_t bytes = acVertexBufferSizeBytes(info);
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        mesh->vertex_buffer[w] = (AcReal*)malloc(bytes);
        if (!mesh->vertex_buffer[w])
            return AC_FAILURE;
    }
    return AC_SUCCESS;
}

AcResult
acHostMeshDestroy(AcMesh* mesh)
{
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w)
        free(mesh->vertex_buffer[w]);
    return AC_SUCCESS;
}

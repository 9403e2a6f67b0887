// TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Links the reference standalone's forcing generator
// (samples/standalone/model/host_forcing.cc, compiled from where it lies) into
// oracle/_ref/libref_forcing_{sp,dp}.so and exposes generateForcingParams
// after srand(seed), so tests can feed the library's generator the same
// rand() / RAND_MAX draws and compare bit for bit.
#include <stdlib.h>

#include "host_forcing.h"

// the generator file also holds device-loading helpers; the checker never
// calls them, so these entry points only satisfy the link
AcResult
acLoadDeviceConstant(const AcRealParam, const AcReal)
{
    return AC_FAILURE;
}

AcResult
acSynchronizeStream(const Stream)
{
    return AC_FAILURE;
}

extern "C" int
ref_forcing_generate(unsigned seed, const AcMeshInfo* info, double out[14])
{
    srand(seed);
    const ForcingParams p = generateForcingParams(*info);
    const double v[14]    = {p.magnitude,   p.k_force.x,   p.k_force.y,   p.k_force.z,
                          p.ff_hel_re.x, p.ff_hel_re.y, p.ff_hel_re.z, p.ff_hel_im.x,
                          p.ff_hel_im.y, p.ff_hel_im.z, p.phase,       p.kaver};
    for (int i = 0; i < 12; ++i)
        out[i] = v[i];
    out[12] = out[13] = 0.0;
    return 0;
}

// TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Links the reference standalone's time-step function
// (samples/standalone/model/host_timestep.cc, compiled from where it lies) into
// oracle/_ref/libref_timestep_{sp,dp}.so and exposes it with plain C types, so
// tests can compare the library's device-side time step formula with it.
#include "host_timestep.h"

// dt = host_timestep(umax, vAmax = 0, info): the call the standalone makes
// with LBFIELD = 0 (samples/standalone/simulation.cc:435-436)
extern "C" double
ref_host_timestep(double umax, const AcMeshInfo* info, double timescale)
{
    set_timescale((AcReal)timescale);
    return (double)host_timestep((AcReal)umax, (AcReal)0.0, *info);
}

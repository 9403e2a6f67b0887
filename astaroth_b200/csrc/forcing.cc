// Helical forcing parameters of one step (host side).
//
// Restates the reference standalone's generator
// (samples/standalone/model/host_forcing.cc:85-182 and 287-320):
//   - a wavevector drawn in spherical coordinates, azimuth 2 pi u0, polar angle
//     pi u1, length (kmax - kmin) u2 + kmin, then each component rounded to an
//     integer so that whole waves fit the box;
//   - a phase 2 pi u3;
//   - a unit vector e perpendicular to k: starting from x^ (or y^ when k lies
//     on the x axis), e = cos(2 pi u4) (k x e)^ + sin(2 pi u4) (k x (k x e)^)^;
//   - the helical amplitude vectors
//       ff_im = |k| (k x e) / D,   ff_re = relhel k x (k x e) / D,
//       D = sqrt(1 + relhel^2) |k| sqrt(|k|^2 - |k o e|^2),
//     where k o e is the componentwise product (the reference's "k dot e"
//     vector; kept as it is);
//   - kaver = (kmax - kmin) / 2 (the reference's definition, kept as it is).
// Every operation is done in AcReal in the reference's order, so the same five
// draws give the same bits in single and in double precision.
#include <math.h>
#include <stdio.h>

#include <cmath>

#include "astaroth.h"
#include "astaroth_b200.h"

namespace {

struct V3 {
    AcReal x, y, z;
};

V3
cross3(const V3& a, const V3& b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

V3
unit3(const V3& a)
{
    const AcReal n2 = a.x * a.x + a.y * a.y + a.z * a.z;
    return {a.x / std::sqrt(n2), a.y / std::sqrt(n2), a.z / std::sqrt(n2)};
}

// SplitMix64 (Steele, Lea and Flood 2014): one 64-bit output per call.
unsigned long long
splitmix64(unsigned long long* s)
{
    unsigned long long z = (*s += 0x9E3779B97F4A7C15ull);
    z                    = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z                    = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

} // namespace

extern "C" {

AcResult
acForcingParamsFromUniforms(const AcMeshInfo info, const AcReal u[5], AcForcingParams* params)
{
    if (!u || !params)
        return AC_FAILURE;
    const AcReal relhel = info.real_params[AC_relhel];
    const AcReal kmin   = info.real_params[AC_kmin];
    const AcReal kmax   = info.real_params[AC_kmax];
    const AcReal two_pi = AcReal(2.0) * AcReal(M_PI);

    // wavevector: spherical draw, components rounded
    const AcReal phi   = two_pi * u[0];
    const AcReal theta = AcReal(M_PI) * u[1];
    const AcReal kk    = (kmax - kmin) * u[2] + kmin;
    V3 k               = {AcReal(kk * std::sin(theta) * std::cos(phi)),
                          AcReal(kk * std::sin(theta) * std::sin(phi)), AcReal(kk * std::cos(theta))};
    k                  = {std::round(k.x), std::round(k.y), std::round(k.z)};

    const AcReal phase = two_pi * u[3];

    // e perpendicular to k, at a random angle about it
    V3 e = (k.y == AcReal(0.0) && k.z == AcReal(0.0)) ? V3{0, 1, 0} : V3{1, 0, 0};
    {
        const V3 a        = unit3(cross3(k, e));
        const V3 b        = unit3(cross3(k, a));
        const AcReal ang  = two_pi * u[4];
        const AcReal c    = std::cos(ang);
        const AcReal s    = std::sin(ang);
        e                 = {a.x * c + b.x * s, a.y * c + b.y * s, a.z * c + b.z * s};
    }

    // helical amplitude vectors
    const V3 ke     = {k.x * e.x, k.y * e.y, k.z * e.z};
    const V3 kxe    = cross3(k, e);
    const V3 kxkxe  = cross3(k, kxe);
    const AcReal ka = std::sqrt(k.x * k.x + k.y * k.y + k.z * k.z);
    const AcReal D  = std::sqrt(AcReal(1.0) + relhel * relhel) * ka *
                     std::sqrt(ka * ka - (ke.x * ke.x + ke.y * ke.y + ke.z * ke.z));

    params->magnitude    = info.real_params[AC_forcing_magnitude];
    params->k_force[0]   = k.x;
    params->k_force[1]   = k.y;
    params->k_force[2]   = k.z;
    params->ff_hel_im[0] = ka * kxe.x / D;
    params->ff_hel_im[1] = ka * kxe.y / D;
    params->ff_hel_im[2] = ka * kxe.z / D;
    params->ff_hel_re[0] = relhel * kxkxe.x / D;
    params->ff_hel_re[1] = relhel * kxkxe.y / D;
    params->ff_hel_re[2] = relhel * kxkxe.z / D;
    params->phase        = phase;
    params->kaver        = (kmax - kmin) / AcReal(2.0);
    return AC_SUCCESS;
}

AcResult
acForcingParamsGenerate(const AcMeshInfo info, unsigned long long* state, AcForcingParams* params)
{
    if (!state || !params)
        return AC_FAILURE;
    AcReal u[5];
    for (int i = 0; i < 5; ++i)
        u[i] = AcReal((double)(splitmix64(state) >> 11) * 0x1.0p-53); // [0, 1)
    return acForcingParamsFromUniforms(info, u, params);
}

} // extern "C"

// acHostIntegrateStep: the CPU model of one RK3 step of the MHD module, part of
// the utils interface (reference src/utils/modelsolver.c:987-1041). Callers use
// it as the host-side model they compare device results with; the GPU path
// never calls it.
//
// Same scheme as the reference host model: periodic bounds on the state before
// each substep, the 2N register w = alpha_s w + dt f(u) over the interior,
// then u += beta_s w. Arithmetic is in AcReal; inverse spacings and cs^2 are
// re-derived from AC_ds* and AC_cs_sound as the reference does (:993-997).
// The vertex loop is OpenMP-parallel.
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "astaroth.h"
#include "astaroth_utils.h"

namespace {

typedef AcReal R;

struct Model {
    int mx, my;
    R inv[3];
    R nu, eta, mu0, cs2, cp, gamma, lnT0, lnrho0, zeta;
    size_t at(int i, int j, int k) const { return (size_t)i + (size_t)j * mx + (size_t)k * mx * my; }
};

struct SD {
    R v, g[3], h[3][3];
};

inline R
rexp(R x)
{
    return (R)exp(x);
}

void
derivs(const Model& M, const R* f, int i, int j, int k, SD& s)
{
    const R c1[3] = {(R)(3.0 / 4.0), (R)(-3.0 / 20.0), (R)(1.0 / 60.0)};
    const R c2[4] = {(R)(-49.0 / 18.0), (R)(3.0 / 2.0), (R)(-3.0 / 20.0), (R)(1.0 / 90.0)};
    const R fac   = (R)(1. / 720.);
    const R cx[3] = {(R)270.0 * fac, (R)(-27.0) * fac, (R)2.0 * fac};
    const int di[3] = {1, 0, 0}, dj[3] = {0, 1, 0}, dk[3] = {0, 0, 1};
    s.v = f[M.at(i, j, k)];
    for (int a = 0; a < 3; ++a) {
        R g = 0, h = c2[0] * s.v;
        for (int o = 1; o <= 3; ++o) {
            const R p = f[M.at(i + o * di[a], j + o * dj[a], k + o * dk[a])];
            const R m = f[M.at(i - o * di[a], j - o * dj[a], k - o * dk[a])];
            g += c1[o - 1] * (p - m);
            h += c2[o] * (p + m);
        }
        s.g[a]    = g * M.inv[a];
        s.h[a][a] = h * M.inv[a] * M.inv[a];
    }
    const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
    for (int q = 0; q < 3; ++q) {
        const int a = pa[q], b = pb[q];
        R r = 0;
        for (int o = 1; o <= 3; ++o) {
            const int ia = o * di[a], ja = o * dj[a], ka = o * dk[a];
            const int ib = o * di[b], jb = o * dj[b], kb = o * dk[b];
            const R pp = f[M.at(i + ia + ib, j + ja + jb, k + ka + kb)];
            const R mm = f[M.at(i - ia - ib, j - ja - jb, k - ka - kb)];
            const R pm = f[M.at(i + ia - ib, j + ja - jb, k + ka - kb)];
            const R mp = f[M.at(i - ia + ib, j - ja + jb, k - ka + kb)];
            r += cx[o - 1] * (pp + mm - pm - mp);
        }
        s.h[a][b] = s.h[b][a] = r * M.inv[a] * M.inv[b];
    }
}

void
rates(const Model& M, R* const* in, int i, int j, int k, R roc[8])
{
    SD lr, u[3], A[3], ss;
    derivs(M, in[VTXBUF_LNRHO], i, j, k, lr);
    for (int c = 0; c < 3; ++c) {
        derivs(M, in[VTXBUF_UUX + c], i, j, k, u[c]);
        derivs(M, in[VTXBUF_AX + c], i, j, k, A[c]);
    }
    derivs(M, in[VTXBUF_ENTROPY], i, j, k, ss);
    const R uv[3] = {u[0].v, u[1].v, u[2].v};
    const R divu  = u[0].g[0] + u[1].g[1] + u[2].g[2];
    roc[VTXBUF_LNRHO] = -(uv[0] * lr.g[0] + uv[1] * lr.g[1] + uv[2] * lr.g[2]) - divu;

    R B[3] = {A[2].g[1] - A[1].g[2], A[0].g[2] - A[2].g[0], A[1].g[0] - A[0].g[1]};
    R lapA[3], gdA[3], gdu[3], lapu[3], jj[3];
    for (int c = 0; c < 3; ++c) {
        lapA[c] = A[c].h[0][0] + A[c].h[1][1] + A[c].h[2][2];
        lapu[c] = u[c].h[0][0] + u[c].h[1][1] + u[c].h[2][2];
        gdA[c]  = A[0].h[c][0] + A[1].h[c][1] + A[2].h[c][2];
        gdu[c]  = u[0].h[c][0] + u[1].h[c][1] + u[2].h[c][2];
        jj[c]   = ((R)1 / M.mu0) * (gdA[c] - lapA[c]);
    }
    const R uxB[3] = {uv[1] * B[2] - uv[2] * B[1], uv[2] * B[0] - uv[0] * B[2],
                      uv[0] * B[1] - uv[1] * B[0]};
    for (int c = 0; c < 3; ++c)
        roc[VTXBUF_AX + c] = uxB[c] + M.eta * lapA[c];

    R S[3][3];
    S[0][0] = (R)(2. / 3.) * u[0].g[0] - (R)(1. / 3.) * (u[1].g[1] + u[2].g[2]);
    S[1][1] = (R)(2. / 3.) * u[1].g[1] - (R)(1. / 3.) * (u[0].g[0] + u[2].g[2]);
    S[2][2] = (R)(2. / 3.) * u[2].g[2] - (R)(1. / 3.) * (u[0].g[0] + u[1].g[1]);
    S[0][1] = S[1][0] = (R)(1. / 2.) * (u[0].g[1] + u[1].g[0]);
    S[0][2] = S[2][0] = (R)(1. / 2.) * (u[0].g[2] + u[2].g[0]);
    S[1][2] = S[2][1] = (R)(1. / 2.) * (u[1].g[2] + u[2].g[1]);
    const R E   = M.gamma * ss.v / M.cp + (M.gamma - 1) * (lr.v - M.lnrho0);
    const R cs2 = M.cs2 * rexp(E);
    const R jxB[3] = {jj[1] * B[2] - jj[2] * B[1], jj[2] * B[0] - jj[0] * B[2],
                      jj[0] * B[1] - jj[1] * B[0]};
    const R inv_rho = (R)1 / rexp(lr.v);
    for (int c = 0; c < 3; ++c) {
        const R ugu = u[c].g[0] * uv[0] + u[c].g[1] * uv[1] + u[c].g[2] * uv[2];
        const R Sg  = S[c][0] * lr.g[0] + S[c][1] * lr.g[1] + S[c][2] * lr.g[2];
        roc[VTXBUF_UUX + c] = -ugu - cs2 * (((R)1 / M.cp) * ss.g[c] + lr.g[c]) + inv_rho * jxB[c] +
                              M.nu * (lapu[c] + (R)(1. / 3.) * gdu[c] + (R)2 * Sg) + M.zeta * gdu[c];
    }
    const R lnT    = M.lnT0 + E;
    const R inv_pT = (R)1 / (rexp(lr.v) * rexp(lnT));
    R SS           = 0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            SS += S[a][b] * S[a][b];
    const R heat = M.eta * M.mu0 * (jj[0] * jj[0] + jj[1] * jj[1] + jj[2] * jj[2]) +
                   (R)2 * rexp(lr.v) * M.nu * SS + M.zeta * rexp(lr.v) * divu * divu;
    const R icp   = (R)1 / M.cp;
    const R first = M.gamma * icp * (ss.h[0][0] + ss.h[1][1] + ss.h[2][2]) +
                    (M.gamma - 1) * (lr.h[0][0] + lr.h[1][1] + lr.h[2][2]);
    R st = 0;
    for (int c = 0; c < 3; ++c) {
        const R sec = M.gamma * icp * ss.g[c] + (M.gamma - 1) * lr.g[c];
        const R thi = M.gamma * (icp * ss.g[c] + lr.g[c]) - lr.g[c];
        st += sec * thi;
    }
    const R chi = (R)0.001 / (rexp(lr.v) * M.cp);
    roc[VTXBUF_ENTROPY] = -(uv[0] * ss.g[0] + uv[1] * ss.g[1] + uv[2] * ss.g[2]) + inv_pT * heat +
                          M.cp * chi * (first + st);
}

} // namespace

extern "C" AcResult
acHostIntegrateStep(AcMesh mesh, const AcReal dt)
{
    AcMeshInfo& I = mesh.info;
    Model M;
    M.mx     = I.int_params[AC_mx];
    M.my     = I.int_params[AC_my];
    M.inv[0] = (R)1 / I.real_params[AC_dsx];
    M.inv[1] = (R)1 / I.real_params[AC_dsy];
    M.inv[2] = (R)1 / I.real_params[AC_dsz];
    M.nu     = I.real_params[AC_nu_visc];
    M.eta    = I.real_params[AC_eta];
    M.mu0    = I.real_params[AC_mu0];
    M.cs2    = I.real_params[AC_cs_sound] * I.real_params[AC_cs_sound];
    M.cp     = I.real_params[AC_cp_sound];
    M.gamma  = I.real_params[AC_gamma];
    M.lnT0   = I.real_params[AC_lnT0];
    M.lnrho0 = I.real_params[AC_lnrho0];
    M.zeta   = I.real_params[AC_zeta];

    const size_t cnt = acVertexBufferSize(I);
    std::vector<std::vector<R>> w(NUM_VTXBUF_HANDLES, std::vector<R>(cnt, (R)0));
    const R alpha[3] = {(R)0, (R)(-5. / 9.), (R)(-153. / 128.)};
    const R beta[3]  = {(R)(1. / 3.), (R)(15. / 16.), (R)(8. / 15.)};
    const int x0 = I.int_params[AC_nx_min], x1 = I.int_params[AC_nx_max];
    const int y0 = I.int_params[AC_ny_min], y1 = I.int_params[AC_ny_max];
    const int z0 = I.int_params[AC_nz_min], z1 = I.int_params[AC_nz_max];
    for (int s = 0; s < 3; ++s) {
        acHostMeshApplyPeriodicBounds(&mesh);
#pragma omp parallel for schedule(static)
        for (int k = z0; k < z1; ++k)
            for (int j = y0; j < y1; ++j)
                for (int i = x0; i < x1; ++i) {
                    R roc[8];
                    rates(M, mesh.vertex_buffer, i, j, k, roc);
                    const size_t id = M.at(i, j, k);
                    for (int c = 0; c < NUM_VTXBUF_HANDLES; ++c)
                        w[c][id] = s == 0 ? roc[c] * dt : alpha[s] * w[c][id] + roc[c] * dt;
                }
#pragma omp parallel for schedule(static)
        for (int k = z0; k < z1; ++k)
            for (int j = y0; j < y1; ++j)
                for (int i = x0; i < x1; ++i) {
                    const size_t id = M.at(i, j, k);
                    for (int c = 0; c < NUM_VTXBUF_HANDLES; ++c)
                        mesh.vertex_buffer[c][id] += beta[s] * w[c][id];
                }
    }
    return AC_SUCCESS;
}

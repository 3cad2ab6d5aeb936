// Engine inlet conditions on level 1 (setBCsOnSolutionField, SolverSource/
// mgnsg3d_def_par.F90:4541-4918), after a node pass has written every node's
// state:
//   k_engine_sums    the sums over the engine inlet sides: the mass flow
//                    (engineFlowType 1, def_par:4541-4599) or the mass flow,
//                    total-pressure function and area (engineFlowType 2,
//                    :4689-4806), and from them each inlet's momentum factor
//   k_engine_finish  the scaling of the inlet momenta with the internal
//                    energy kept (:4615-4649, 4827-4860), the pressure the
//                    reference leaves in grp%p (the exhaust pressure, or
//                    makePressureField of engineFlowType 2, :4864), the
//                    no-inflow correction (:4653-4686), and the steps of the
//                    node pass that follow setBCsOnSolutionField, which the
//                    pass deferred for these nodes (limitDensity and
//                    setOuterBoundaryConditions of an RK stage, the increment
//                    of restrictGrid's fine step, prolongateGrid's floors)
// The exhaust states and the increment conditions are pointwise and stay in
// the node passes.  Each sum is taken in a fixed order: side s goes to the
// partial sum of lane s mod kEngineLanes in side order, and the partials meet
// in a pairwise tree; the CPU restatement sums in the same order.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace flite {

namespace {
__device__ __forceinline__ double ke3(const double *u, int N, int i) {
    const double a = u[N + i], b = u[2 * (size_t)N + i], c = u[3 * (size_t)N + i];
    return (a * a + b * b) + c * c;
}
}  // namespace

__global__ void __launch_bounds__(kEngineLanes) k_engine_sums(Params P, LevelView L, int mode) {
    const EngineView &E = L.eng;
    const double *T = mode == MODE_RFINE ? L.rhs : L.u;
    const int N = L.N, t = threadIdx.x;
    const bool ft2 = P.eftype == 2;
    double acc[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int s = t; s < E.nside; s += kEngineLanes) {
        const int2 nd = E.side[s];
        const int a = nd.x, b = nd.y, e = E.inlet[s];
        const double w0 = E.wx[s], w1 = E.wy[s], w2 = E.wz[s];
        const double s1 = (T[N + a] * w0 + T[2 * (size_t)N + a] * w1) + T[3 * (size_t)N + a] * w2;
        const double s2 = (T[N + b] * w0 + T[2 * (size_t)N + b] * w1) + T[3 * (size_t)N + b] * w2;
        acc[e][0] += s1 + s2;
        if (ft2) {
            // grp%p: the stage's pressure, or the exhaust pressure this call set
            const double pa = is_exhaust(L.bc[a]) ? E.pbc[a] : L.p[a];
            const double pb = is_exhaust(L.bc[b]) ? E.pbc[b] : L.p[b];
            const double ka = ke3(T, N, a), kb = ke3(T, N, b);
            const double ra = T[a], rb = T[b];
            const double press = 0.5 * ((pa + 0.5 * ka / ra) + (pb + 0.5 * kb / rb));
            const double temp1 = (P.gamma / ra) * (T[4 * (size_t)N + a] - (0.5 * ka) / ra);
            const double temp2 = (P.gamma / rb) * (T[4 * (size_t)N + b] - (0.5 * kb) / rb);
            const double temp = 0.5 * (temp1 + temp2);
            const double wn = sqrt((w0 * w0 + w1 * w1) + w2 * w2);
            acc[e][1] += (sqrt(temp) / press) * 2.0 * wn;
            acc[e][2] += 2.0 * wn;
        }
    }
    __shared__ double part[6][kEngineLanes];
    for (int e = 0; e < 2; ++e)
        for (int k = 0; k < 3; ++k) part[3 * e + k][t] = acc[e][k];
    __syncthreads();
    for (int w = kEngineLanes / 2; w >= 1; w >>= 1) {
        if (t < w)
            for (int j = 0; j < 6; ++j) part[j][t] = part[j][t] + part[j][t + w];
        __syncthreads();
    }
    if (t != 0) return;
    // an inlet whose flow sum is not positive keeps factor 1 (the
    // reference's factor is then an uninitialised local)
    EngineFactors F;
    F.fac[0] = 1.0; F.fac[1] = 1.0;
    F.scale = 1;
    if (P.eftype == 1) {
        for (int e = 0; e < 2; ++e)
            if (part[3 * e][0] > 0.0) F.fac[e] = P.front[e] / part[3 * e][0];
    } else if (ft2) {
        for (int e = 0; e < 2 && F.scale; ++e) {
            const double flow = part[3 * e][0];
            if (!(flow > 0.0)) continue;
            const double mff = flow * (part[3 * e + 1][0] / part[3 * e + 2][0]);
            F.fac[e] = P.front[e] / mff;
            if (F.fac[e] > 99999999999.) F.scale = 0;  // the jump past the scaling (def_par:4784-4801)
        }
    }
    *E.f = F;
}

__global__ void k_engine_finish(Params P, LevelView L, int mode, int all) {
    const EngineView &E = L.eng;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (all ? L.N : E.nnode)) return;
    const int i = all ? t : E.node[t];
    const int N = L.N;
    const unsigned char cls = L.bc[i];
    double *T = mode == MODE_RFINE ? L.rhs : L.u;
    double un[5];
    for (int c = 0; c < 5; ++c) un[c] = T[(size_t)c * N + i];
    const bool inlets = P.eftype == 1 || P.eftype == 2;
    const EngineFactors F = *E.f;
    if (inlets && F.scale && is_inlet(cls)) {
        // internal energy of grp%u (the node's state before the scaling in
        // every pass but restrictGrid's fine step)
        const double intE = L.u[4 * (size_t)N + i] - 0.5 * ke3(L.u, N, i) / L.u[i];
        const double fac = F.fac[cls == BC_EIN1 ? 0 : 1];
        for (int c = 1; c < 4; ++c) un[c] = un[c] * fac;
        un[4] = intE + 0.5 * ((un[1] * un[1] + un[2] * un[2]) + un[3] * un[3]) / un[0];
        if (P.sa) {
            const size_t o6 = 5 * (size_t)N + i;
            if (mode == MODE_RFINE) L.rhs[o6] = 0.0 - L.uprev[o6];
            else L.u[o6] = 0.0;
        }
    }
    // the pressure setBCsOnSolutionField leaves in grp%p
    double p = is_exhaust(cls) ? E.pbc[i] : L.p[i];
    if (P.eftype == 2 && F.scale) {
        if (mode == MODE_RFINE)
            p = pressure(P, L.u[i], L.u[N + i], L.u[2 * (size_t)N + i], L.u[3 * (size_t)N + i], L.u[4 * (size_t)N + i]);
        else
            p = pressure(P, un[0], un[1], un[2], un[3], un[4]);
    }
    L.p[i] = p;
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = L.nx[i]; n1 = L.ny[i]; n2 = L.nz[i]; }
    if (inlets && is_inlet(cls)) {  // no inflow through an inlet
        const double nv = (((-n0) * un[1] + (-n1) * un[2]) + (-n2) * un[3]) / un[0];
        if (nv < 0.00) {
            un[1] = un[1] + un[0] * (nv - 0.01) * n0;
            un[2] = un[2] + un[0] * (nv - 0.01) * n1;
            un[3] = un[3] + un[0] * (nv - 0.01) * n2;
        }
    }
    if (mode == MODE_STAGE) {  // limitDensity, setOuterBoundaryConditions
        un[0] = dmax(un[0], P.minRho);
        bc_outer(P, cls, n0, n1, n2, p, un);
    } else if (mode == MODE_PROLONG) {  // setOuterBoundaryConditions, the density floor
        bc_outer(P, cls, n0, n1, n2, p, un);
        un[0] = dmax(un[0], P.minRho);
    } else if (mode == MODE_RFINE) {  // setOuterBoundaryConditions, rhs = candidate - uprev
        bc_outer(P, cls, n0, n1, n2, p, un);
        for (int c = 0; c < 5; ++c) un[c] = un[c] - L.uprev[(size_t)c * N + i];
    }
    for (int c = 0; c < 5; ++c) T[(size_t)c * N + i] = un[c];
}

}  // namespace flite

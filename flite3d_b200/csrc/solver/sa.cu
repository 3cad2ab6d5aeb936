// Spalart-Allmaras one-equation model (turbulenceModel 1) on the device.
//
// nu~ is component 6 of the level's state arrays ([6][N]).  Each edge loop
// of the reference becomes a node gather over the CSR incidence lists in
// edge order (then the boundary edges in their order), and every expression
// keeps the reference's operation order, so the results equal the CPU
// restatement bit for bit:
//   k_sa_timestep  makeTurbulentTimeSteps  (def_par:12878-13100)
//   k_sa_grad      makeSADiffusion pass 1  (def_par:7436-7560): Galerkin
//                  gradient of nu~ and the cb2 term
//   k_sa_diff      makeSADiffusion pass 2  (def_par:7560-7809)
//   k_sa_conv      makeSARHS               (def_par:6809-6950)
//   k_sa_stage     the nu~ part of one RK stage / of restrictGrid's coarse
//                  and fine one-step updates: makeSASourceTerm (def_par:
//                  9285-9371), the diffusion term, solveTurbulenceSystem,
//                  the increment and solution conditions, nullifyOuterBoundary,
//                  updateSolutionVector, the FAS source, limitTurbulence and
//                  the far-field value (def_par:1002-1181, 12141-12430)
// k_sa_stage runs before the mean-flow node update of the same stage: it
// reads the stage-start density, which that update overwrites.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"
#include "pinned_math.h"

namespace flite {

namespace {
__device__ __forceinline__ int tid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ bool sa_wall(unsigned char cls) { return cls == BC_WALL || cls == BC_IWALL; }
__device__ __forceinline__ bool sa_far(unsigned char cls) { return cls == BC_FAR3 || cls == BC_FAR4; }
__device__ __forceinline__ double rp_exhaust(const Params &P, const LevelView &L, unsigned char cls) {
    return sa_exhaust(P, cls, eo_relax(P, *L.cyc));
}
}  // namespace

__global__ void k_sa_timestep(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double* __restrict__ nt = L.u + 5 * (size_t)N;
    const double oneOverSigma = 3.0 / 2.0, oneOverKappaSquared = 1.0 / (0.41 * 0.41);
    const double cb1 = 0.1355, cb2 = 0.622, ct3 = 1.1;
    const double cw1 = cb1 * oneOverKappaSquared + (1.0 + cb2) * oneOverSigma;
    const double oRe = 1.0 / P.Re;
    const double ro = 1. / L.u[i];
    const double m1 = L.u[N + i], m2 = L.u[2 * N + i], m3 = L.u[3 * N + i];
    double acc = 0.0, h = 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x, j = t.y;
        const double wx = L.wx[e], wy = L.wy[e], wz = L.wz[e];
        const double al = (wx * wx + wy * wy) + wz * wz;
        double vn = ((wx * m1 + wy * m2) + wz * m3) * ro;
        vn = P.turbK * sqrt(al) + fabs(vn);
        acc = acc + vn;
        // the other node's diffusion term (def_par:12930-12935)
        const double vis = oneOverSigma * (L.mu[j] + 3.0 * cb2 * nt[j] * oRe);
        const double dv = 2.0 * vis * al;
        h = h + dv;
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
        const double al = (wx * wx + wy * wy) + wz * wz;
        const int j1 = nd.x, j2 = nd.y;
        const double ro1 = 1. / L.u[j1], ro2 = 1. / L.u[j2];
        double vn1 = ((wx * L.u[N + j1] + wy * L.u[2 * N + j1]) + wz * L.u[3 * N + j1]) * ro1;
        double vn2 = ((wx * L.u[N + j2] + wy * L.u[2 * N + j2]) + wz * L.u[3 * N + j2]) * ro2;
        vn1 = P.turbK * sqrt(al) + fabs(vn1);
        vn2 = P.turbK * sqrt(al) + fabs(vn2);
        const double vnm = vn1 + vn2;
        acc = side == 0 ? (acc + vn1) + vnm : (acc + vn2) + vnm;
        const double vis1 = oneOverSigma * (L.mu[j1] + 3.0 * cb2 * nt[j1] * oRe);
        const double vis2 = oneOverSigma * (L.mu[j2] + 3.0 * cb2 * nt[j2] * oRe);
        const double dv1 = 2.0 * vis1 * al, dv2 = 2.0 * vis2 * al;
        const double dvm = dv1 + dv2;
        h = side == 0 ? (h + dv1) + dvm : (h + dv2) + dvm;
    }
    const double V = L.V[i];
    const double dt = 0.5 / (acc / V + h / (V * V));
    double dInvSquared = L.wdist[i] > 1.0e-10 ? 1.0 / L.wdist[i] : 1.0e10;
    dInvSquared = dInvSquared * dInvSquared;
    const double S = (fabs(L.divg[i]) +
                      cb1 * (L.vort[i] + (1.0 + ct3) * nt[i] * oneOverKappaSquared * dInvSquared * oRe)) +
                     cw1 * nt[i] * dInvSquared * oRe;
    L.dtT[i] = dt / (1.0 + 0.5 * S * dt);
}

__global__ void k_sa_grad(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double* __restrict__ nt = L.u + 5 * (size_t)N;
    const double ti = nt[i];
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const double tj = nt[t.y];
        const double s = t.x >= 0 ? ti + tj : tj + ti;  // (nu1 + nu2) in the edge's order
        const double f1 = L.wx[e] * s, f2 = L.wy[e] * s, f3 = L.wz[e] * s;
        if (t.x >= 0) { g0 = g0 + f1; g1 = g1 + f2; g2 = g2 + f3; }
        else { g0 = g0 - f1; g1 = g1 - f2; g2 = g2 - f3; }
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
        const double t1 = nt[nd.x], t2 = nt[nd.y];
        if (P.boundaryTerm == 1) {
            const double a = side == 0 ? 3. * t1 + t2 : t1 + 3. * t2;
            g0 = g0 + a * wx; g1 = g1 + a * wy; g2 = g2 + a * wz;
        } else {
            const double a = side == 0 ? t1 : t2;
            g0 = g0 + 4. * a * wx; g1 = g1 + 4. * a * wy; g2 = g2 + 4. * a * wz;
        }
    }
    const double sigma = 2. / 3., cb2 = 0.622, oRe = 1. / P.Re;
    const double fact = oRe * cb2 / sigma;
    const double vt = 1. / L.V[i];
    const double dx = g0 * vt, dy = g1 * vt, dz = g2 * vt;
    L.sag[i] = dx;
    L.sag[N + i] = dy;
    L.sag[2 * N + i] = dz;
    const double vp = (g0 * dx + g1 * dy) + g2 * dz;
    L.sanh[i] = 0.0 - fact * vp;
}

__global__ void k_sa_diff(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double* __restrict__ nt = L.u + 5 * (size_t)N;
    const double sigma = 2. / 3., oRe = 1. / P.Re;
    const double fact = oRe / sigma;
    auto visc = [&](int n) { return P.Re * L.mu[n] / L.u[n] + nt[n]; };
    auto fd = [&](int n, double wx, double wy, double wz) {
        return visc(n) * ((wx * L.sag[n] + wy * L.sag[N + n]) + wz * L.sag[2 * N + n]);
    };
    double acc = 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const int n1 = t.x >= 0 ? i : t.y, n2 = t.x >= 0 ? t.y : i;
        const double wx = L.wx[e], wy = L.wy[e], wz = L.wz[e];
        const double fd1 = fd(n1, wx, wy, wz), fd2 = fd(n2, wx, wy, wz);
        acc = t.x >= 0 ? acc - fact * (fd1 + fd2) : acc + fact * (fd1 + fd2);
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
        const double fd1 = fd(nd.x, wx, wy, wz), fd2 = fd(nd.y, wx, wy, wz);
        if (P.boundaryTerm == 1) acc = acc - fact * (side == 0 ? 3. * fd1 + fd2 : fd1 + 3. * fd2);
        else acc = acc - fact * 4. * (side == 0 ? fd1 : fd2);
    }
    L.turbDiff[i] = acc + L.sanh[i];
}

__global__ void k_sa_conv(Params P, LevelView L, int td) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double* __restrict__ nt = L.u + 5 * (size_t)N;
    auto prim = [&](int n, double *q) {
        const double rinv = 1. / L.u[n];
        q[0] = rinv * L.u[N + n]; q[1] = rinv * L.u[2 * N + n]; q[2] = rinv * L.u[3 * N + n];
        q[3] = nt[n];
    };
    double qi[4];
    prim(i, qi);
    // an unsteady stage's time difference comes first (def_par:1073)
    double acc = td ? time_difference(P, L, i, 5) : 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        double qj[4];
        prim(t.y, qj);
        const double *a = t.x >= 0 ? qi : qj, *b = t.x >= 0 ? qj : qi;
        const double u1 = a[0], v1 = a[1], w1 = a[2], t1 = a[3];
        const double u2 = b[0], v2 = b[1], w2 = b[2], t2 = b[3];
        const double wx = L.wx[e], wy = L.wy[e], wz = L.wz[e];
        double fconv = (wx * (u1 * t1 + u2 * t2) + wy * (v1 * t1 + v2 * t2)) + wz * (w1 * t1 + w2 * t2);
        if (fabs(t1 - t2) > 1.0e-20) {
            const double ax = (u2 * t2 - u1 * t1) / (t1 - t2);
            const double ay = (v2 * t2 - v1 * t1) / (t1 - t2);
            const double az = (w2 * t2 - w1 * t1) / (t1 - t2);
            fconv = fconv + fabs((wx * ax + wy * ay) + wz * az) * (t1 - t2);
        }
        acc = t.x >= 0 ? acc + fconv : acc - fconv;
    }
    L.rhs[5 * (size_t)N + i] = acc;
}

// makeSASourceTerm at node i added to r; the laminar viscosity floor writes
// 0.1*Re into the array, as the reference does (def_par:9321-9323)
__device__ __forceinline__ double sa_source(const Params &P, const LevelView &L, int i, double r) {
    using namespace flite_pm;
    const int N = L.N;
    const double oRe = 1. / P.Re;
    const double cb1 = 0.1355, cb2 = 0.622, kappa = 0.41, kappaSquared = kappa * kappa, sigma = 2. / 3.;
    const double cw1 = cb1 / kappaSquared + (1.0 + cb2) / sigma;
    const double cw2 = 0.3, cw3 = 2.0, cv1 = 7.1, ct3 = 1.1, ct4 = 2.0;
    const double cv1Tripled = pm_cube(cv1), cw3InSixth = pm_pow6(cw3), oneOverSix = 1. / 6.;
    const double vt = L.V[i];
    const double mucurl = dmax(L.u[5 * (size_t)N + i], 0.0);
    double mu = L.mu[i];
    if (mu < 0.1 / P.Re) {
        mu = 0.1 * P.Re;
        L.mu[i] = mu;
    }
    double Ksi = L.u[i] * oRe * mucurl / mu;
    Ksi = dmax(Ksi, 0.001);
    const double ft2 = ct3 * pm_exp(-ct4 * Ksi * Ksi);
    const double K3 = pm_cube(Ksi);
    const double d = dmax(L.wdist[i], 1.0e-10);
    const double muOverd = mucurl / d, dSquared = d * d;
    const double fv1 = K3 / (K3 + cv1Tripled);
    const double fv2 = 1.0 - (Ksi / (1.0 + Ksi * fv1));
    const double fv3 = 1.0;
    const double Scurl = fv3 * L.vort[i] + oRe * mucurl * fv2 / (kappaSquared * dSquared);
    double rr;
    if (fabs(Scurl) > 1.0e-10) {
        rr = oRe * mucurl / (Scurl * kappaSquared * dSquared);
        if (rr < 0.0) rr = 0.0;
        if (rr > 100.0) rr = 100.0;
    } else {
        rr = 100.0;
    }
    const double gg = rr + cw2 * (pm_pow6(rr) - rr);
    const double radicand = (1.0 + cw3InSixth) / (pm_pow6(gg) + cw3InSixth);
    const double fw = radicand > 1.0e-10 ? gg * pm_exp(oneOverSix * pm_log(radicand))
                                         : pm_exp(oneOverSix * pm_log(1.0 + cw3InSixth));
    r = r - vt * cb1 * (1.0 - ft2) * Scurl * mucurl;
    r = r + oRe * vt * (cw1 * fw - cb1 * ft2 / kappaSquared) * muOverd * muOverd;
    r = r - vt * mucurl * L.divg[i];
    return r;
}

__global__ void k_sa_stage(Params P, LevelView L, int mode, int stage, int turb) {
    int i = tid();
    if (i >= L.N) return;
    const size_t o6 = 5 * (size_t)L.N + i;
    const unsigned char cls = L.bc[i];
    // convection from k_sa_conv (after the time difference of an unsteady
    // stage, which is all of it when the turbulence is not recomputed)
    double r = turb ? L.rhs[o6] : (P.addts && mode == MODE_STAGE ? time_difference(P, L, i, 5) : 0.0);
    if (turb) r = sa_source(P, L, i, r);
    // restrictGrid adds the (last computed) diffusion term whether or not
    // the turbulence is recomputed (def_par:12238-12240, 12315-12317)
    if (turb || mode != MODE_STAGE) r = r + L.turbDiff[i];
    // solveTurbulenceSystem: the local step, or the explicit global one
    r = ((P.unsteady && P.explicit_) ? *L.ptsg : L.dtT[i]) * r / L.V[i];
    if (sa_wall(cls) || is_exhaust(cls)) r = 0.0;
    if (is_inlet(cls)) r = P.engRelax * r;  // the engine inlets' relaxation (def_par:5084-5099)
    if (L.grid > 1 && (cls == BC_FAR3 || is_engine(cls))) r = 0.0;  // nullifyOuterBoundary
    const double dtJ = stage > 0 ? P.turbCFL * P.RK[stage - 1] : P.turbCFL;
    double un = L.uprev[o6] - dtJ * r;
    un = dmax(un, 0.0);
    if (sa_wall(cls)) un = 0.0;
    // the exhausts' nu~; an inlet's is zeroed on level 1 by k_engine_finish
    // when its momenta are scaled
    if (is_exhaust(cls)) un = rp_exhaust(P, L, cls);
    if (mode == MODE_STAGE) {
        if (L.grid > 1 && turb) un = un - P.RK[stage - 1] * L.src[o6];
        if (turb) {  // limitTurbulence
            un = dmax(un, 0.0);
            if (un > P.maxTurb) un = P.maxTurb;
        }
        if (sa_far(cls)) un = 0.1;
        L.u[o6] = un;
    } else if (mode == MODE_RCOARSE) {
        if (sa_far(cls)) un = 0.1;
        L.src[o6] = un - L.uprev[o6];
    } else {  // MODE_RFINE
        if (L.grid > 1) un = un - L.src[o6];
        // limitTurbulence(finegrp, rhs(:,6)): floors the increment array and
        // caps the state's nu~ (def_par:1259-1290, 12361-12363)
        un = dmax(un, 0.0);
        if (L.u[o6] > P.maxTurb) L.u[o6] = P.maxTurb;
        if (sa_far(cls)) un = 0.1;
        L.rhs[o6] = un - L.uprev[o6];
    }
}

}  // namespace flite

// CUDA kernels of the flow-solver hot path (sm_100a, FP64).
//
// Layout and scheduling:
//  * node state is SoA [component][node] so node kernels read and write each
//    component coalesced;
//  * the interior-edge flux is computed once per edge into an edge buffer
//    [E][5]; a node kernel then sums it through a CSR list of incident
//    edges kept in edge order.  Summing in edge order reproduces the
//    reference's scatter loop (rhs(i1)+=f, rhs(i2)-=f in edge order) bit for
//    bit, with no atomics;
//  * cheap edge terms (time step, JST Laplacian and sensor, JST flux,
//    gradients, min/max) are recomputed by both endpoints inside a node
//    gather, which replaces an edge buffer round trip by reads of the
//    neighbour's state;
//  * everything the reference does per node after the residual (add the
//    dissipation, multiply by dt/V, boundary conditions on the increment,
//    the clipped update, boundary conditions on the solution, the FAS
//    source, the density floor, the far-field conditions) is fused into the
//    node kernel that gathers the residual;
//  * the kernels of the multigrid cycle also have a group form (template
//    flag B): one launch serves every case of a batch's case group, the
//    case in blockIdx.y and its parameters and level views among the
//    arguments (FLITE_CASE_P / FLITE_CASE_L).
#include <cuda_runtime.h>

#include "flux.cuh"
#include "kernels.h"
#include "pinned_math.h"

namespace flite {

static __device__ __forceinline__ int tid() { return blockIdx.x * blockDim.x + threadIdx.x; }

// Group-per-node gathers (small levels): U lanes (a power of two up to 32)
// serve one node.  Lane l of a group evaluates the terms of incidence k0 + l;
// the group then applies them to the node's accumulators in incidence order,
// every lane doing the same additions on broadcast terms, so the sums are
// those of the serial loop bit for bit.  Groups past the last node stay in
// the loop (the shuffles need every lane) but apply nothing.
template <int U, int K, class T, class Terms, class Add>
__device__ __forceinline__ void group_gather(int beg, int end, bool active, int gl, Terms &&terms, Add &&add) {
    const int span = active ? end - beg : 0;
    const unsigned trips = (unsigned)((span + U - 1) / U);
    const unsigned maxtrips = __reduce_max_sync(0xffffffffu, trips);
    for (unsigned t = 0; t < maxtrips; ++t) {
        const int k0 = beg + (int)t * U;
        T v[K];
#pragma unroll
        for (int c = 0; c < K; ++c) v[c] = T(0);
        if (active && k0 + gl < end) terms(k0 + gl, v);
        const int n = active ? min(U, end - k0) : 0;
        for (int q = 0; q < U; ++q) {
            T x[K];
#pragma unroll
            for (int c = 0; c < K; ++c) x[c] = __shfl_sync(0xffffffffu, v[c], q, U);
            if (q < n) add(x);
        }
    }
}

// ---- makePressureField (def_par:13612-13630) ------------------------------
template <bool B>
__global__ void k_pressure(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double r = L.u[i], ru = L.u[N + i], rv = L.u[2 * N + i], rw = L.u[3 * N + i], E = L.u[4 * N + i];
    const double p = pressure(P, r, ru, rv, rw, E);
    L.p[i] = p;
    store_node(L.q, i, r, ru, rv, rw, E, p);
}

// ---- makeTimeSteps (def_par:13335-13610) as a node gather -----------------
// The pieces of a thread-per-node gather, shared by the separate kernel, its
// incidence-row form and the fused walks below.
//
// interior edge t of node i (momentum m, 1/rho ro, cc = max(gamma p/rho,
// 0.001)): the convective and acoustic terms, and with viscosity the other
// node's viscous term (def_par:13432-13433; with SA the viscosity is
// mu + nu~/Re)
__device__ __forceinline__ void ts_inc(const Params &P, const LevelView &L, int2 t, double m1, double m2, double m3,
                                       double ro, double cc, double &acc, double &h) {
    const int N = L.N;
    const int e = t.x >= 0 ? t.x : ~t.x;
    const double wx = L.wx[e], wy = L.wy[e], wz = L.wz[e];
    const double al = (wx * wx + wy * wy) + wz * wz;
    const double vn = ((wx * m1 + wy * m2) + wz * m3) * ro;
    acc = (acc + fabs(vn)) + sqrt(cc * al);
    if (P.viscous) {
        const int j = t.y;
        const double vis = dmax(P.am, P.sa ? L.mu[j] + L.u[5 * N + j] / P.Re : L.mu[j]);
        const double dv = 2.0 * vis * al / L.u[j];
        h = h + dv;
    }
}
// boundary edge binc[k]: v[0..3] the convective and acoustic terms of the
// node's side and of both, v[4..5] the viscous ones
__device__ __forceinline__ void ts_bterms(const Params &P, const LevelView &L, int k, double *v) {
    const int N = L.N;
    const double c1 = P.gamma;
    const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
    const int2 nd = L.bedge[b];
    const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
    const double al = (wx * wx + wy * wy) + wz * wz;
    const int j1 = nd.x, j2 = nd.y;
    const double ro1 = 1. / L.u[j1], ro2 = 1. / L.u[j2];
    double cc1 = dmax(c1 * L.p[j1] * ro1, 0.001);
    double cc2 = dmax(c1 * L.p[j2] * ro2, 0.001);
    double vn1 = ((wx * L.u[N + j1] + wy * L.u[2 * N + j1]) + wz * L.u[3 * N + j1]) * ro1;
    double vn2 = ((wx * L.u[N + j2] + wy * L.u[2 * N + j2]) + wz * L.u[3 * N + j2]) * ro2;
    vn1 = fabs(vn1); vn2 = fabs(vn2);
    cc1 = sqrt(cc1 * al); cc2 = sqrt(cc2 * al);
    v[0] = side == 0 ? vn1 : vn2;
    v[1] = vn1 + vn2;
    v[2] = side == 0 ? cc1 : cc2;
    v[3] = cc1 + cc2;
    if (P.viscous) {
        const double vis1 = dmax(P.am, P.sa ? L.mu[j1] + L.u[5 * N + j1] / P.Re : L.mu[j1]);
        const double vis2 = dmax(P.am, P.sa ? L.mu[j2] + L.u[5 * N + j2] / P.Re : L.mu[j2]);
        const double dv1 = 2.0 * vis1 * al / L.u[j1];
        const double dv2 = 2.0 * vis2 * al / L.u[j2];
        v[4] = side == 0 ? dv1 : dv2;
        v[5] = dv1 + dv2;
    } else {
        v[4] = v[5] = 0.0;
    }
}
__device__ __forceinline__ void ts_badd(const Params &P, const double *x, double &acc, double &h) {
    acc = (((acc + x[0]) + x[1]) + x[2]) + x[3];
    if (P.viscous) h = (h + x[4]) + x[5];
}
__device__ __forceinline__ void ts_store(const LevelView &L, int i, double acc, double h) {
    const double V = L.V[i];
    const double dt = 0.5 / (acc / V + h / (V * V));
    L.dt[i] = dt;
    L.vdt[i] = V / dt;  // V/dt of the dissipation coefficient d0
}
// the boundary edges of node i in order, then dt and V/dt
__device__ __forceinline__ void ts_finish(const Params &P, const LevelView &L, int i, double acc, double h) {
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        double v[6];
        ts_bterms(P, L, k, v);
        ts_badd(P, v, acc, h);
    }
    ts_store(L, i, acc, h);
}

template <int U, bool B>
__global__ void k_timestep(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    const double c1 = P.gamma;
    const double ri = L.u[i], ro = 1. / ri;
    const double m1 = L.u[N + i], m2 = L.u[2 * N + i], m3 = L.u[3 * N + i];
    const double cc = dmax(c1 * L.p[i] * ro, 0.001);
    double acc = 0.0, h = 0.0;
    if constexpr (U > 1) {
        const int beg = L.inc_ptr[i], end = L.inc_ptr[i + 1];
        group_gather<U, 3, double>(
            beg, end, active, gl,
            [&](int k, double *v) {
            const int2 t = L.inc[k];
            const int e = t.x >= 0 ? t.x : ~t.x;
            const double wx = L.wx[e], wy = L.wy[e], wz = L.wz[e];
            const double al = (wx * wx + wy * wy) + wz * wz;
            const double vn = ((wx * m1 + wy * m2) + wz * m3) * ro;
            v[0] = fabs(vn);
            v[1] = sqrt(cc * al);
            if (P.viscous) {
                const int j = t.y;
                const double vis = dmax(P.am, P.sa ? L.mu[j] + L.u[5 * N + j] / P.Re : L.mu[j]);
                v[2] = 2.0 * vis * al / L.u[j];
            }
            },
            [&](const double *x) {
            acc = (acc + x[0]) + x[1];
            if (P.viscous) h = h + x[2];
            });
    } else
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) ts_inc(P, L, L.inc[k], m1, m2, m3, ro, cc, acc, h);
    auto bterms = [&](int k, double *v) { ts_bterms(P, L, k, v); };
    auto badd = [&](const double *x) { ts_badd(P, x, acc, h); };
    if constexpr (U > 1) {
        group_gather<U, 6, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, bterms, badd);
        if (!active || gl) return;
        ts_store(L, i, acc, h);
    } else {
        ts_finish(P, L, i, acc, h);
    }
}

// ---- makeArtificialDissipation2, passes 1-2 and the node finish -----------
// (def_par:11513-11780): undivided Laplacian with dE+dp, pressure sensor
struct LapAcc {
    double l[5], s7, s8;
};
// interior edge t of node i (state ui, pressure pi)
__device__ __forceinline__ void lap_inc(const Params &P, const LevelView &L, int2 t, const double *ui, double pi,
                                        LapAcc &a) {
    const int N = L.N;
    const int j = t.y;
    double df = 1.0;
    if (P.useDissW) df = 1. / L.slen[t.x >= 0 ? t.x : ~t.x];
    const double uj[5] = {L.u[j], L.u[N + j], L.u[2 * N + j], L.u[3 * N + j], L.u[4 * N + j]};
    const double pj = L.p[j];
    if (t.x >= 0) {  // this node is i1: d = u(i) - u(j)
#pragma unroll
        for (int c = 0; c < 4; ++c) a.l[c] = a.l[c] - (ui[c] - uj[c]) * df;
        const double d4 = ((ui[4] - uj[4]) + pi) - pj;
        a.l[4] = a.l[4] - d4 * df;
        const double dp = pi - pj, sp = pi + pj;
        a.s7 = a.s7 - dp; a.s8 = a.s8 + sp;
    } else {         // i2: d = u(j) - u(i)
#pragma unroll
        for (int c = 0; c < 4; ++c) a.l[c] = a.l[c] + (uj[c] - ui[c]) * df;
        const double d4 = ((uj[4] - ui[4]) + pj) - pi;
        a.l[4] = a.l[4] + d4 * df;
        const double dp = pj - pi, sp = pj + pi;
        a.s7 = a.s7 + dp; a.s8 = a.s8 + sp;
    }
}
__device__ __forceinline__ void lap_store(const LevelView &L, int i, const LapAcc &a) {
    const int N = L.N;
    const double fact = 1. / L.conn[i];
    L.sens[i] = 12. * fabs(a.s7 / a.s8);
#pragma unroll
    for (int c = 0; c < 5; ++c) L.lap[c * N + i] = fact * a.l[c];
}

template <int U, bool B>
__global__ void k_jst_lap(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    double l0 = 0, l1 = 0, l2 = 0, l3 = 0, l4 = 0, s7 = 0, s8 = 0;
    const double ui0 = L.u[i], ui1 = L.u[N + i], ui2 = L.u[2 * N + i], ui3 = L.u[3 * N + i], ui4 = L.u[4 * N + i];
    const double pi = L.p[i];
    if constexpr (U > 1) {
        const int beg = L.inc_ptr[i], end = L.inc_ptr[i + 1];
        group_gather<U, 7, double>(
            beg, end, active, gl,
            [&](int k, double *v) {
            const int2 t = L.inc[k];
            const int j = t.y;
            double df = 1.0;
            if (P.useDissW) df = 1. / L.slen[t.x >= 0 ? t.x : ~t.x];
            const double uj0 = L.u[j], uj1 = L.u[N + j], uj2 = L.u[2 * N + j], uj3 = L.u[3 * N + j];
            const double uj4 = L.u[4 * N + j], pj = L.p[j];
            // x - y is x + (-y): the subtractions of the serial loop become
            // additions of negated terms
            if (t.x >= 0) {
                v[0] = -((ui0 - uj0) * df); v[1] = -((ui1 - uj1) * df); v[2] = -((ui2 - uj2) * df);
                v[3] = -((ui3 - uj3) * df); v[4] = -((((ui4 - uj4) + pi) - pj) * df);
                v[5] = -(pi - pj); v[6] = pi + pj;
            } else {
                v[0] = (uj0 - ui0) * df; v[1] = (uj1 - ui1) * df; v[2] = (uj2 - ui2) * df;
                v[3] = (uj3 - ui3) * df; v[4] = (((uj4 - ui4) + pj) - pi) * df;
                v[5] = pj - pi; v[6] = pj + pi;
            }
            },
            [&](const double *x) {
            l0 = l0 + x[0]; l1 = l1 + x[1]; l2 = l2 + x[2]; l3 = l3 + x[3]; l4 = l4 + x[4];
            s7 = s7 + x[5]; s8 = s8 + x[6];
            });
        if (!active || gl) return;
    } else {
        LapAcc a = {{0, 0, 0, 0, 0}, 0, 0};
        const double ui[5] = {ui0, ui1, ui2, ui3, ui4};
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) lap_inc(P, L, L.inc[k], ui, pi, a);
        lap_store(L, i, a);
        return;
    }
    LapAcc a = {{l0, l1, l2, l3, l4}, s7, s8};
    lap_store(L, i, a);
}

// ---- makeArtificialDissipation2, pass 3 (def_par:11770-11906), scalar -----
// interior edge t of node i (Laplacian Li, state Ui, V/dt vdi, connectivity
// coni, sensor si): the fourth- and second-order terms with the sign of
// this node
__device__ __forceinline__ void jflux_inc(const Params &P, const LevelView &L, int2 t, double k4, double vdi,
                                          double coni, double si, const double *Li, const double *Ui, double *acc) {
    const int N = L.N;
    const int j = t.y;
    const double vdj = L.vdt[j];
    const bool first = t.x >= 0;
    double d0 = first ? dmin(vdi, vdj) : dmin(vdj, vdi);
    d0 = d0 / (first ? (coni + L.conn[j]) : (L.conn[j] + coni));
    const double sj = L.sens[j];
    const double d2 = d0 * P.k2 * (first ? dmax(si, sj) : dmax(sj, si));
    double d4 = d0 * k4;
    d4 = d4 > d2 ? d4 - d2 : 0.0;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const double Lj = L.lap[c * N + j], Uj = L.u[c * N + j];
        if (first) {
            const double d4v = Li[c] - Lj, d2v = Ui[c] - Uj;
            acc[c] = (acc[c] - d4v * d4) + d2v * d2;
        } else {
            const double d4v = Lj - Li[c], d2v = Uj - Ui[c];
            acc[c] = (acc[c] + d4v * d4) - d2v * d2;
        }
    }
}

template <int U, bool B>
__global__ void __launch_bounds__(256, U == 1 ? 4 : 1) k_jst_flux(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    const double k4 = L.grid == 1 ? P.k4 : P.cgdf;
    double acc[5] = {0, 0, 0, 0, 0};
    double Li[5], Ui[5];
    for (int c = 0; c < 5; ++c) { Li[c] = L.lap[c * N + i]; Ui[c] = L.u[c * N + i]; }
    const double vdi = L.vdt[i], coni = L.conn[i], si = L.sens[i];
    if constexpr (U > 1) {
        const int beg = L.inc_ptr[i], end = L.inc_ptr[i + 1];
        group_gather<U, 10, double>(
            beg, end, active, gl,
            [&](int k, double *v) {
            const int2 t = L.inc[k];
            const int j = t.y;
            const double vdj = L.vdt[j];
            const bool first = t.x >= 0;
            double d0 = first ? dmin(vdi, vdj) : dmin(vdj, vdi);
            d0 = d0 / (first ? (coni + L.conn[j]) : (L.conn[j] + coni));
            const double sj = L.sens[j];
            const double d2 = d0 * P.k2 * (first ? dmax(si, sj) : dmax(sj, si));
            double d4 = d0 * k4;
            d4 = d4 > d2 ? d4 - d2 : 0.0;
            for (int c = 0; c < 5; ++c) {
                const double Lj = L.lap[c * N + j], Uj = L.u[c * N + j];
                if (first) {
                    v[2 * c] = -((Li[c] - Lj) * d4);
                    v[2 * c + 1] = (Ui[c] - Uj) * d2;
                } else {
                    v[2 * c] = (Lj - Li[c]) * d4;
                    v[2 * c + 1] = -((Uj - Ui[c]) * d2);
                }
            }
            },
            [&](const double *x) {
            for (int c = 0; c < 5; ++c) acc[c] = (acc[c] + x[2 * c]) + x[2 * c + 1];
            });
        if (!active || gl) return;
    } else
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) jflux_inc(P, L, L.inc[k], k4, vdi, coni, si, Li, Ui, acc);
    for (int c = 0; c < 5; ++c) L.diss[c * N + i] = acc[c];
}

// ---- makeArtificialDissipation2, pass 3, matrix variant (def_par:11814-
// 11898): the one-dimensional Roe matrix |A| along edge e (i1 -> i2), with
// Harten's correction, applied to the Laplacian and state differences
__device__ __forceinline__ void matrix_diss(const Params &P, const LevelView &L, int e, int i1, int i2,
                                            double *d4v, double *d2v) {
    const int N = L.N;
    const double H = P.harten;
    const double eps1 = 1. / dmax(H, 1.e-5), gam1 = P.gm1;
    double rnx = L.wx[e], rny = L.wy[e], rnz = L.wz[e];
    const double al = sqrt((rnx * rnx + rny * rny) + rnz * rnz);
    const double vmo1 = 1. / al;
    rnx = rnx * vmo1; rny = rny * vmo1; rnz = rnz * vmo1;
    const double rhol = L.u[i1];
    double rho1 = 1. / rhol;
    const double uxl = L.u[N + i1] * rho1, vyl = L.u[2 * N + i1] * rho1, wzl = L.u[3 * N + i1] * rho1;
    const double hl = (L.u[4 * N + i1] + L.p[i1]) * rho1;
    const double rhor = L.u[i2];
    rho1 = 1. / rhor;
    const double uxr = L.u[N + i2] * rho1, vyr = L.u[2 * N + i2] * rho1, wzr = L.u[3 * N + i2] * rho1;
    const double hr = (L.u[4 * N + i2] + L.p[i2]) * rho1;
    const double di = sqrt(rhor / rhol), d1 = 1.0 / (di + 1.0);
    const double ui = (di * uxr + uxl) * d1, vi = (di * vyr + vyl) * d1, wi = (di * wzr + wzl) * d1;
    const double hi = (di * hr + hl) * d1;
    const double ci2 = gam1 * (hi - 0.5 * ((ui * ui + vi * vi) + wi * wi));
    const double ci = sqrt(ci2);
    const double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
    const double ucp = (ui * rnx + vi * rny) + wi * rnz;
    double l1 = fabs(ucp + ci), l2 = fabs(ucp - ci), l3 = fabs(ucp);
    if (l1 < H) l1 = 0.5 * (l1 * l1 * eps1 + H);
    if (l2 < H) l2 = 0.5 * (l2 * l2 * eps1 + H);
    if (l3 < H) l3 = 0.5 * (l3 * l3 * eps1 + H);
    const double s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
    auto apply = [&](double *d) {
        const double al1x = gam1 * ((((af * d[0] - ui * d[1]) - vi * d[2]) - wi * d[3]) + d[4]);
        const double al2x = ((-ucp * d[0] + d[1] * rnx) + d[2] * rny) + d[3] * rnz;
        const double cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci);
        const double cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
        d[0] = al * (l3 * d[0] + cc1);
        d[1] = al * ((l3 * d[1] + cc1 * ui) + cc2 * rnx);
        d[2] = al * ((l3 * d[2] + cc1 * vi) + cc2 * rny);
        d[3] = al * ((l3 * d[3] + cc1 * wi) + cc2 * rnz);
        d[4] = al * ((l3 * d[4] + cc1 * hi) + cc2 * ucp);
    };
    apply(d4v);
    apply(d2v);
}

// the matrix variant's pass 3 as a node gather in edge order; each edge's
// matrix terms are evaluated in the edge's own node order at both ends
__global__ void k_jst_flux_matrix(Params P, LevelView L) {
    const int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double k4 = L.grid == 1 ? P.k4 : P.cgdf;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const bool first = t.x >= 0;
        const int e = first ? t.x : ~t.x;
        const int i1 = first ? i : t.y, i2 = first ? t.y : i;
        double d4v[5], d2v[5];
        for (int c = 0; c < 5; ++c) {
            d4v[c] = L.lap[c * N + i1] - L.lap[c * N + i2];
            d2v[c] = L.u[c * N + i1] - L.u[c * N + i2];
        }
        matrix_diss(P, L, e, i1, i2, d4v, d2v);
        const double d2 = P.k2 * dmax(L.sens[i1], L.sens[i2]);
        const double d4 = k4 > d2 ? k4 - d2 : 0.0;
        for (int c = 0; c < 5; ++c)
            acc[c] = first ? (acc[c] - d4v[c] * d4) + d2v[c] * d2 : (acc[c] + d4v[c] * d4) - d2v[c] * d2;
    }
    for (int c = 0; c < 5; ++c) L.diss[c * N + i] = acc[c];
}

// ---- makeArtificialDissipation1 (def_par:10706-11482), level 1 -----------
// the linearity-preserving dissipation of Crumpton et al.  Pass 1, per node
// in edge order: the gradient sums of (rho, rho u, rho v, rho w, rho E), the
// undivided Laplacian L(U), the sum of the edge factors and L(x); then the
// boundary faces, the volume scaling, L^(U) = L(U) - (grad U).L(x) (L(x) = 0
// on boundary nodes) and the pressure sensor.  Writes L^ to lap, the sensor
// to sens and the factor sum to lpw.
__global__ void k_lp_sums(Params P, LevelView L) {
    const int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    double g[15], l[5], lx[3] = {0.0, 0.0, 0.0}, s21 = 0.0, pd = 0.0, ps = 0.0;
    for (int c = 0; c < 15; ++c) g[c] = 0.0;
    for (int c = 0; c < 5; ++c) l[c] = 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const bool first = t.x >= 0;
        const int e = first ? t.x : ~t.x;
        const int i1 = first ? i : t.y, i2 = first ? t.y : i;
        const EdgeW ew = load_edgew(L.ew, e);
        const double w[3] = {ew.wx, ew.wy, ew.wz};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 5; ++c) {
                const double sv = (L.u[c * N + i1] + L.u[c * N + i2]) * w[a];
                g[5 * a + c] = first ? g[5 * a + c] + sv : g[5 * a + c] - sv;
            }
        double df = 1.0;
        if (P.useDissW) df = 1. / L.slen[e];
        for (int c = 0; c < 5; ++c) {
            const double d = L.u[c * N + i1] - L.u[c * N + i2];
            l[c] = first ? l[c] - d * df : l[c] + d * df;
        }
        s21 = s21 + df;
        const double dx[3] = {L.cx[i1] - L.cx[i2], L.cy[i1] - L.cy[i2], L.cz[i1] - L.cz[i2]};
        for (int a = 0; a < 3; ++a) lx[a] = first ? lx[a] - dx[a] * df : lx[a] + dx[a] * df;
        const double dp = L.p[i1] - L.p[i2], sp = L.p[i1] + L.p[i2];
        pd = first ? pd - dp : pd + dp;
        ps = ps + sp;
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 5; ++c) {
                const double q1 = L.u[c * N + nd.x], q2 = L.u[c * N + nd.y];
                double v;
                if (P.boundaryTerm == 1) v = side == 0 ? (3. * q1 + q2) * w[a] : (q1 + 3. * q2) * w[a];
                else v = side == 0 ? 4. * q1 * w[a] : 4. * w[a];  // the reference's second term has no state
                g[5 * a + c] = g[5 * a + c] + v;
            }
    }
    if (P.useDissW) s21 = 3.0 * s21;
    const double vt = 1. / L.V[i];
    for (int c = 0; c < 15; ++c) g[c] = g[c] * vt;
    if (i < L.Nb) lx[0] = lx[1] = lx[2] = 0.0;
    for (int c = 0; c < 5; ++c)
        L.lap[c * N + i] = ((l[c] + g[c] * lx[0]) + g[5 + c] * lx[1]) + g[10 + c] * lx[2];
    L.sens[i] = 12. * fabs(pd / ps);
    L.lpw[i] = s21;
}

// pass 2: the edge terms, as a node gather in edge order; under
// useMatrixDissipation the scalar coefficient divided by each end's factor
// sum, otherwise the Roe matrix (the reference's branch order)
__global__ void k_lp_flux(Params P, LevelView L) {
    const int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const bool first = t.x >= 0;
        const int e = first ? t.x : ~t.x;
        const int i1 = first ? i : t.y, i2 = first ? t.y : i;
        double d4v[5], d2v[5];
        for (int c = 0; c < 5; ++c) {
            d4v[c] = L.lap[c * N + i1] - L.lap[c * N + i2];
            d2v[c] = L.u[c * N + i1] - L.u[c * N + i2];
        }
        double d2, d4, d41, d42;
        if (P.matrixDiss) {
            const double d0 = dmin(L.vdt[i1], L.vdt[i2]) / (L.conn[i1] + L.conn[i2]);
            d2 = d0 * P.k2 * dmax(L.sens[i1], L.sens[i2]);
            d4 = d0 * P.k4;
            d4 = d4 > d2 ? d4 - d2 : 0.0;
            d41 = d4 / L.lpw[i1];
            d42 = d4 / L.lpw[i2];
        } else {
            matrix_diss(P, L, e, i1, i2, d4v, d2v);
            d2 = P.k2 * dmax(L.sens[i1], L.sens[i2]);
            d4 = P.k4;
            d4 = d4 > d2 ? d4 - d2 : 0.0;
            d41 = d42 = d4;
        }
        for (int c = 0; c < 5; ++c)
            acc[c] = first ? (acc[c] - d4v[c] * d41) + d2v[c] * d2 : (acc[c] + d4v[c] * d42) - d2v[c] * d2;
    }
    for (int c = 0; c < 5; ++c) L.diss[c * N + i] = acc[c];
}

// ---- makeArtificialDissipation3 (def_par:11995-12139) ---------------------
template <int U>
__global__ void k_first_order_diss(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    double acc[5] = {0, 0, 0, 0, 0};
    const double vdi = L.vdt[i], coni = L.conn[i];
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        int2 t = L.inc[k];
        int j = t.y;
        double vdj = L.vdt[j];
        const bool first = t.x >= 0;
        double d0 = first ? dmin(vdi, vdj) : dmin(vdj, vdi);
        d0 = d0 / (first ? (coni + L.conn[j]) : (L.conn[j] + coni));
        double d2 = d0 * P.cgdf;
        for (int c = 0; c < 5; ++c) {
            double dk = first ? L.u[c * N + i] - L.u[c * N + j] : L.u[c * N + j] - L.u[c * N + i];
            acc[c] = first ? acc[c] + dk * d2 : acc[c] - dk * d2;
        }
    }
    for (int c = 0; c < 5; ++c) L.diss[c * N + i] = acc[c];
}

// ---- makeViscosityTerm, wide stencil (def_par:5198-5893) ------------------
// pass 1: Galerkin gradients of (u, v, w, T), then per node the Sutherland
// viscosity (T^1.5 evaluated as T*sqrt(T)), the stress tensor and heat
// flux, the adiabatic-wall projection and the wall stress (level 1)
// per node (u, v, w, T) of the viscous routine (def_par:5260-5270): each
// edge of the reference divides again; the quotients are the same numbers
template <bool B>
__global__ void k_visc_prim(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double gOg = P.gamma / (P.gamma - 1.0);
    const double r = L.u[i];
    L.prim[i] = L.u[N + i] / r;
    L.prim[N + i] = L.u[2 * N + i] / r;
    L.prim[2 * N + i] = L.u[3 * N + i] / r;
    L.prim[3 * N + i] = gOg * L.p[i] / r;
}

// the boundary-face terms of node i's Galerkin gradients of (u, v, w, T)
// (def_par:5322-5409), added to g in boundary-edge order
__device__ __forceinline__ void visc_grad_bterms(const LevelView &L, int k, double *d) {
    const int N = L.N;
    int b = L.binc[k] >> 1, side = L.binc[k] & 1;
    int2 nd = L.bedge[b];
    const double q1[4] = {L.prim[nd.x], L.prim[N + nd.x], L.prim[2 * N + nd.x], L.prim[3 * N + nd.x]};
    const double q2[4] = {L.prim[nd.y], L.prim[N + nd.y], L.prim[2 * N + nd.y], L.prim[3 * N + nd.y]};
    const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 4; ++c) {
            double sm = q1[c] + q2[c];
            double own = side == 0 ? q1[c] : q2[c];
            d[a * 4 + c] = (2. * own + sm) * w[a];
        }
}

// from node i's summed gradients g: Sutherland's viscosity, the SA eddy
// viscosity, vorticity and divergence, the stress tensor and heat flux, the
// adiabatic-wall projection and the wall stress (def_par:5460-5640)
__device__ __forceinline__ void visc_grad_finish(const Params &P, const LevelView &L, int i, const double *g) {
    const int N = L.N;
    const double gOg = P.gamma / (P.gamma - 1.0);
    const double vt = 1. / L.V[i];
    double dudx = g[0] * vt, dvdx = g[1] * vt, dwdx = g[2] * vt, dTdx = g[3] * vt;
    double dudy = g[4] * vt, dvdy = g[5] * vt, dwdy = g[6] * vt, dTdy = g[7] * vt;
    double dudz = g[8] * vt, dvdz = g[9] * vt, dwdz = g[10] * vt, dTdz = g[11] * vt;
    const double tempConv = (P.gamma - 1.0) * P.mach * P.mach;
    double T = gOg * L.p[i] / L.u[i];
    if (T <= 0.001) T = 0.001;
    double a = tempConv * T;
    double mu = (1. / P.Re) * ((a * sqrt(a)) * ((P.Tinf + 198.6) / (tempConv * P.Tinf * T + 198.6)));
    double kc = (1. / P.Pr) * mu;
    L.mu[i] = mu;
    if (P.sa) {
        const double a1 = dudy - dvdx, a2 = dvdz - dwdy, a3 = dwdx - dudz;
        L.vort[i] = sqrt((a1 * a1 + a2 * a2) + a3 * a3);
        L.divg[i] = (dudx + dvdy) + dwdz;
        // turbulent viscosity of the SA model (def_par:5556-5566)
        double tvc = (1. / P.Re) * L.u[i] * L.u[5 * N + i];
        const double ksi3 = flite_pm::pm_cube(tvc / mu);
        tvc = tvc * ksi3 / (ksi3 + 357.9);
        mu = mu + tvc;
        kc = kc + tvc * P.oPrt;
    }
    const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
    double tau[9];
    tau[0] = mu * (fourThirds * dudx - twoThirds * (dvdy + dwdz));
    tau[1] = mu * (dudy + dvdx);
    tau[2] = mu * (dudz + dwdx);
    tau[3] = mu * (fourThirds * dvdy - twoThirds * (dudx + dwdz));
    tau[4] = mu * (dvdz + dwdy);
    tau[5] = mu * (fourThirds * dwdz - twoThirds * (dudx + dvdy));
    tau[6] = kc * dTdx;
    tau[7] = kc * dTdy;
    tau[8] = kc * dTdz;
    const unsigned char cls = L.bc[i];
    if (L.grid == 1 && cls != BC_NONE) {
        double n0 = L.nx[i], n1 = L.ny[i], n2 = L.nz[i];
        if (cls == BC_WALL) {  // setTemperatureForAdiabaticWall (def_par:5170-5196)
            double nt = (tau[6] * n0 + tau[7] * n1) + tau[8] * n2;
            tau[6] = tau[6] - nt * n0;
            tau[7] = tau[7] - nt * n1;
            tau[8] = tau[8] - nt * n2;
        }
        L.wstress[i] = (tau[0] * n0 + tau[1] * n1) + tau[2] * n2;
        L.wstress[N + i] = (tau[1] * n0 + tau[3] * n1) + tau[4] * n2;
        L.wstress[2 * N + i] = (tau[2] * n0 + tau[4] * n1) + tau[5] * n2;
    }
    for (int c = 0; c < 9; ++c) L.tau[c * N + i] = tau[c];
}

// interior edge t of node i (u, v, w, T of the node qi): the edge's terms
// of the 12 gradient sums, added with the sign of this node
__device__ __forceinline__ void vgrad_inc(const LevelView &L, int2 t, const double *qi, double *g) {
    const int N = L.N;
    const int e = t.x >= 0 ? t.x : ~t.x, j = t.y;
    const double qj[4] = {L.prim[j], L.prim[N + j], L.prim[2 * N + j], L.prim[3 * N + j]};
    const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double x = (t.x >= 0 ? qi[c] + qj[c] : qj[c] + qi[c]) * w[a];
            g[a * 4 + c] = t.x >= 0 ? g[a * 4 + c] + x : g[a * 4 + c] - x;
        }
}
// the boundary edges of node i in order
__device__ __forceinline__ void visc_grad_boundary(const LevelView &L, int i, double *g) {
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        double v[12];
        visc_grad_bterms(L, k, v);
#pragma unroll
        for (int c = 0; c < 12; ++c) g[c] = g[c] + v[c];
    }
}

template <int U, bool B>
__global__ void __launch_bounds__(256, U == 1 ? 3 : 1) k_visc_grad(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    double g[12];
    for (int c = 0; c < 12; ++c) g[c] = 0.0;
    auto prim = [&](int j, double *q) {
        q[0] = L.prim[j]; q[1] = L.prim[N + j]; q[2] = L.prim[2 * N + j]; q[3] = L.prim[3 * N + j];
    };
    double qi[4];
    prim(i, qi);
    auto iterms = [&](int k, double *d) {
        int2 t = L.inc[k];
        int e = t.x >= 0 ? t.x : ~t.x;
        double qj[4];
        prim(t.y, qj);
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 4; ++c) {
                double x = (t.x >= 0 ? qi[c] + qj[c] : qj[c] + qi[c]) * w[a];
                d[a * 4 + c] = t.x >= 0 ? x : -x;  // g - x is g + (-x)
            }
    };
    auto bterms = [&](int k, double *d) { visc_grad_bterms(L, k, d); };
    auto add = [&](const double *d) {
        for (int c = 0; c < 12; ++c) g[c] = g[c] + d[c];
    };
    if constexpr (U > 1) {
        group_gather<U, 12, double>(L.inc_ptr[i], L.inc_ptr[i + 1], active, gl, iterms, add);
        group_gather<U, 12, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, bterms, add);
        if (!active || gl) return;
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) vgrad_inc(L, L.inc[k], qi, g);
        visc_grad_boundary(L, i, g);
    }
    visc_grad_finish(P, L, i, g);
}

// the viscous flux of an edge from the stress/heat-flux and velocity of its
// first (a, ua) and second (b, ub) node (def_par:5688-5720)
__device__ __forceinline__ void visc_edge_flux(const double *a, const double *b, const double *ua, const double *ub,
                                               double wx, double wy, double wz, double *f) {
    double dt[9];
    for (int c = 0; c < 9; ++c) dt[c] = a[c] + b[c];
    double dut1 = ((((ua[0] * a[0] + ub[0] * b[0]) + ua[1] * a[1]) + ub[1] * b[1]) + ua[2] * a[2]) + ub[2] * b[2];
    double dut2 = ((((ua[0] * a[1] + ub[0] * b[1]) + ua[1] * a[3]) + ub[1] * b[3]) + ua[2] * a[4]) + ub[2] * b[4];
    double dut3 = ((((ua[0] * a[2] + ub[0] * b[2]) + ua[1] * a[4]) + ub[1] * b[4]) + ua[2] * a[5]) + ub[2] * b[5];
    f[0] = (wx * dt[0] + wy * dt[1]) + wz * dt[2];
    f[1] = (wx * dt[1] + wy * dt[3]) + wz * dt[4];
    f[2] = (wx * dt[2] + wy * dt[4]) + wz * dt[5];
    f[3] = (wx * (dt[6] + dut1) + wy * (dt[7] + dut2)) + wz * (dt[8] + dut3);
}

// the two terms of each component of boundary edge binc[k] for its node
// (def_par:5730-5800); g[8] = 0 for symmetry and inviscid-wall faces,
// which contribute nothing
__device__ __forceinline__ void visc_flux_bterms(const LevelView &L, int k, double *g) {
    const int N = L.N;
    int bb = L.binc[k] >> 1, side = L.binc[k] & 1;
    int ind = L.bind[bb];
    g[8] = (ind == 2 || ind == 9) ? 0.0 : 1.0;
    if (g[8] == 0.0) return;
    int2 nd = L.bedge[bb];
    double a[9], b[9], ua[3], ub[3];
    for (int c = 0; c < 9; ++c) { a[c] = L.tau[c * N + nd.x]; b[c] = L.tau[c * N + nd.y]; }
    ua[0] = L.prim[nd.x]; ua[1] = L.prim[N + nd.x]; ua[2] = L.prim[2 * N + nd.x];
    ub[0] = L.prim[nd.y]; ub[1] = L.prim[N + nd.y]; ub[2] = L.prim[2 * N + nd.y];
    const double wx = L.bwx[bb], wy = L.bwy[bb], wz = L.bwz[bb];
    double dt[9];
    for (int c = 0; c < 9; ++c) dt[c] = a[c] + b[c];
    double d11 = (ua[0] * a[0] + ua[1] * a[1]) + ua[2] * a[2];
    double d12 = (ub[0] * b[0] + ub[1] * b[1]) + ub[2] * b[2];
    double d21 = (ua[0] * a[1] + ua[1] * a[3]) + ua[2] * a[4];
    double d22 = (ub[0] * b[1] + ub[1] * b[3]) + ub[2] * b[4];
    double d31 = (ua[0] * a[2] + ua[1] * a[4]) + ua[2] * a[5];
    double d32 = (ub[0] * b[2] + ub[1] * b[4]) + ub[2] * b[5];
    double dut1 = d11 + d12, dut2 = d21 + d22, dut3 = d31 + d32;
    g[0] = (wx * dt[0] + wy * dt[1]) + wz * dt[2];
    g[1] = (wx * dt[1] + wy * dt[3]) + wz * dt[4];
    g[2] = (wx * dt[2] + wy * dt[4]) + wz * dt[5];
    g[3] = (wx * (dt[6] + dut1) + wy * (dt[7] + dut2)) + wz * (dt[8] + dut3);
    const double *o = side == 0 ? a : b;
    double do1 = side == 0 ? d11 : d12, do2 = side == 0 ? d21 : d22, do3 = side == 0 ? d31 : d32;
    g[4] = 2.0 * ((wx * o[0] + wy * o[1]) + wz * o[2]);
    g[5] = 2.0 * ((wx * o[1] + wy * o[3]) + wz * o[4]);
    g[6] = 2.0 * ((wx * o[2] + wy * o[4]) + wz * o[5]);
    g[7] = 2.0 * ((wx * (o[6] + do1) + wy * (o[7] + do2)) + wz * (o[8] + do3));
}

// node i's boundary-edge terms added to acc in boundary-edge order
__device__ __forceinline__ void visc_flux_boundary(const LevelView &L, int i, double *acc) {
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        double v[9];
        visc_flux_bterms(L, k, v);
        if (v[8] == 0.0) continue;
        for (int c = 0; c < 4; ++c) acc[c] = (acc[c] + v[c]) + v[4 + c];
    }
}

// pass 2: viscous edge fluxes gathered per node and subtracted from the
// dissipation vector (def_par:5662-5892)
template <int U, bool B>
__global__ void __launch_bounds__(256, U == 1 ? 3 : 1) k_visc_flux(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    double ti[9], ui[3];
    for (int c = 0; c < 9; ++c) ti[c] = L.tau[c * N + i];
    ui[0] = L.prim[i]; ui[1] = L.prim[N + i]; ui[2] = L.prim[2 * N + i];
    double acc[4] = {0, 0, 0, 0};
    // interior edge: the edge flux with the sign of this node (x - y is x + (-y))
    auto iterms = [&](int k, double *g) {
        int2 t = L.inc[k];
        int e = t.x >= 0 ? t.x : ~t.x, j = t.y;
        double tj[9], uj[3];
        for (int c = 0; c < 9; ++c) tj[c] = L.tau[c * N + j];
        uj[0] = L.prim[j]; uj[1] = L.prim[N + j]; uj[2] = L.prim[2 * N + j];
        const bool first = t.x >= 0;
        double f[4];
        visc_edge_flux(first ? ti : tj, first ? tj : ti, first ? ui : uj, first ? uj : ui, L.wx[e], L.wy[e], L.wz[e],
                       f);
        for (int c = 0; c < 4; ++c) g[c] = first ? f[c] : -f[c];
    };
    auto iadd = [&](const double *g) {
        for (int c = 0; c < 4; ++c) acc[c] = acc[c] + g[c];
    };
    // boundary edge: the two terms of each component, g[8] = 1 if it counts
    auto bterms = [&](int k, double *g) { visc_flux_bterms(L, k, g); };
    auto badd = [&](const double *g) {
        if (g[8] == 0.0) return;
        for (int c = 0; c < 4; ++c) acc[c] = (acc[c] + g[c]) + g[4 + c];
    };
    if constexpr (U > 1) {
        group_gather<U, 4, double>(L.inc_ptr[i], L.inc_ptr[i + 1], active, gl, iterms, iadd);
        group_gather<U, 9, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, bterms, badd);
        if (!active || gl) return;
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
            double v[4];
            iterms(k, v);
            iadd(v);
        }
        for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
            double v[9];
            bterms(k, v);
            badd(v);
        }
    }
    for (int c = 0; c < 4; ++c) L.diss[(1 + c) * N + i] = L.diss[(1 + c) * N + i] - acc[c];
}

// ---- fused walks of one incidence list (thread per node) -------------------
// Gathers that read the same neighbours and write disjoint arrays share one
// walk of the node's incidence list: the incidences, their edges and the
// neighbours' state are read once for both.  Each sum keeps its own
// accumulators and its own order, so the results are those of the separate
// kernels bit for bit.
//
// makeTimeSteps with passes 1-2 of makeArtificialDissipation2: the time
// step reads mu of the neighbours (the previous viscous pass) and writes dt
// and V/dt; the Laplacian reads u and p and writes the Laplacian and sensor
template <bool B>
__global__ void __launch_bounds__(256, 3) k_ts_lap(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double ui[5] = {L.u[i], L.u[N + i], L.u[2 * N + i], L.u[3 * N + i], L.u[4 * N + i]};
    const double pi = L.p[i];
    const double ro = 1. / ui[0];
    const double cc = dmax(P.gamma * pi * ro, 0.001);
    double acc = 0.0, h = 0.0;
    LapAcc a = {{0, 0, 0, 0, 0}, 0, 0};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        ts_inc(P, L, t, ui[1], ui[2], ui[3], ro, cc, acc, h);
        lap_inc(P, L, t, ui, pi, a);
    }
    lap_store(L, i, a);
    ts_finish(P, L, i, acc, h);
}

// pass 3 of makeArtificialDissipation2 (scalar) with pass 1 of
// makeViscosityTerm: the JST terms read the Laplacian, sensor, V/dt and u of
// the neighbours and write the dissipation; the gradients read u, v, w, T
// and write mu, the stress tensor and the wall stress
template <bool B>
__global__ void __launch_bounds__(256, 2) k_jflux_vgrad(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double k4 = L.grid == 1 ? P.k4 : P.cgdf;
    double acc[5] = {0, 0, 0, 0, 0};
    double Li[5], Ui[5];
    for (int c = 0; c < 5; ++c) { Li[c] = L.lap[c * N + i]; Ui[c] = L.u[c * N + i]; }
    const double vdi = L.vdt[i], coni = L.conn[i], si = L.sens[i];
    const double qi[4] = {L.prim[i], L.prim[N + i], L.prim[2 * N + i], L.prim[3 * N + i]};
    double g[12];
    for (int c = 0; c < 12; ++c) g[c] = 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        jflux_inc(P, L, t, k4, vdi, coni, si, Li, Ui, acc);
        vgrad_inc(L, t, qi, g);
    }
    for (int c = 0; c < 5; ++c) L.diss[c * N + i] = acc[c];
    visc_grad_boundary(L, i, g);
    visc_grad_finish(P, L, i, g);
}

// ---- makeViscosityTerm2, the compact stencil (def_par:5896-6807) ---------
// pass 1: the Galerkin gradients of (u, v, w, T) as in k_visc_grad (with the
// FV boundary form under boundaryTerm 2), then per node the viscosity and
// the gradients scaled by mu (velocity) and k (temperature), stored with mu
// and k as tau[14][N]; the adiabatic-wall projection and the wall stress of
// the wall nodes on level 1; zero temperature gradients on every boundary
// node of isentropic (adiabatic) walls
__device__ __forceinline__ void visc2_grad_finish(const Params &P, const LevelView &L, int i, const double *g) {
    const int N = L.N;
    const double gOg = P.gamma / (P.gamma - 1.0);
    const double vt = 1. / L.V[i];
    double gs[12];
    for (int c = 0; c < 12; ++c) gs[c] = g[c] * vt;
    const double dudx = gs[0], dvdx = gs[1], dwdx = gs[2];
    const double dudy = gs[4], dvdy = gs[5], dwdy = gs[6];
    const double dudz = gs[8], dvdz = gs[9], dwdz = gs[10];
    const double tempConv = (P.gamma - 1.0) * P.mach * P.mach;
    double T = gOg * L.p[i] / L.u[i];
    if (T <= 0.001) T = 0.001;
    double a = tempConv * T;
    double mu = (1. / P.Re) * ((a * sqrt(a)) * ((P.Tinf + 198.6) / (tempConv * P.Tinf * T + 198.6)));
    double kc = (1. / P.Pr) * mu;
    L.mu[i] = mu;
    if (P.sa) {
        const double a1 = dudy - dvdx, a2 = dvdz - dwdy, a3 = dwdx - dudz;
        L.vort[i] = sqrt((a1 * a1 + a2 * a2) + a3 * a3);
        L.divg[i] = (dudx + dvdy) + dwdz;
        double tvc = (1. / P.Re) * L.u[i] * L.u[5 * N + i];
        const double ksi3 = flite_pm::pm_cube(tvc / mu);
        tvc = tvc * ksi3 / (ksi3 + 357.9);
        mu = mu + tvc;
        kc = kc + tvc * P.oPrt;
    }
#pragma unroll
    for (int q = 0; q < 12; ++q) gs[q] = ((q & 3) == 3 ? kc : mu) * gs[q];
    const unsigned char cls = L.bc[i];
    if (L.grid == 1 && cls == BC_WALL) {
        const double n0 = L.nx[i], n1 = L.ny[i], n2 = L.nz[i];
        const double nt = (gs[3] * n0 + gs[7] * n1) + gs[11] * n2;
        gs[3] = gs[3] - nt * n0;
        gs[7] = gs[7] - nt * n1;
        gs[11] = gs[11] - nt * n2;
        const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
        const double c1 = fourThirds * gs[0] - twoThirds * (gs[5] + gs[10]), c2 = gs[4] + gs[1];
        const double c3 = gs[8] + gs[2], c4 = fourThirds * gs[5] - twoThirds * (gs[0] + gs[10]);
        const double c5 = gs[9] + gs[6], c6 = fourThirds * gs[10] - twoThirds * (gs[0] + gs[5]);
        L.wstress[i] = (c1 * n0 + c2 * n1) + c3 * n2;
        L.wstress[N + i] = (c2 * n0 + c4 * n1) + c5 * n2;
        L.wstress[2 * N + i] = (c3 * n0 + c5 * n1) + c6 * n2;
    }
    if (P.isentropic && i < L.Nb) gs[3] = gs[7] = gs[11] = 0.0;
    for (int q = 0; q < 12; ++q) L.tau[q * N + i] = gs[q];
    L.tau[12 * N + i] = mu;
    L.tau[13 * N + i] = kc;
}

template <int U, bool B>
__global__ void __launch_bounds__(256, U == 1 ? 3 : 1) k_visc2_grad(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    double g[12];
    for (int c = 0; c < 12; ++c) g[c] = 0.0;
    auto prim = [&](int j, double *q) {
        q[0] = L.prim[j]; q[1] = L.prim[N + j]; q[2] = L.prim[2 * N + j]; q[3] = L.prim[3 * N + j];
    };
    double qi[4];
    prim(i, qi);
    auto iterms = [&](int k, double *d) {
        int2 t = L.inc[k];
        int e = t.x >= 0 ? t.x : ~t.x;
        double qj[4];
        prim(t.y, qj);
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 4; ++c) {
                double x = (t.x >= 0 ? qi[c] + qj[c] : qj[c] + qi[c]) * w[a];
                d[a * 4 + c] = t.x >= 0 ? x : -x;
            }
    };
    auto bterms = [&](int k, double *d) {
        if (P.boundaryTerm == 1) {
            visc_grad_bterms(L, k, d);
            return;
        }
        // boundaryTerm 2: 4 q w_b of the node itself (def_par:6113-6138)
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const int j = side == 0 ? nd.x : nd.y;
        double q[4];
        prim(j, q);
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 4; ++c) d[a * 4 + c] = 4. * q[c] * w[a];
    };
    auto add = [&](const double *d) {
        for (int c = 0; c < 12; ++c) g[c] = g[c] + d[c];
    };
    if constexpr (U > 1) {
        group_gather<U, 12, double>(L.inc_ptr[i], L.inc_ptr[i + 1], active, gl, iterms, add);
        group_gather<U, 12, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, bterms, add);
        if (!active || gl) return;
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
            double v[12];
            iterms(k, v);
            add(v);
        }
        for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
            double v[12];
            bterms(k, v);
            add(v);
        }
    }
    visc2_grad_finish(P, L, i, g);
}

// node j's data of the compact flux: scaled gradients (12), mu, k,
// velocity and temperature (from 1/rho as the routine forms them) and
// coordinates (zero on coarse levels)
struct Visc2Node {
    double G[12], mu, k, v[4], x[3];
};
__device__ __forceinline__ void load_visc2(const Params &P, const LevelView &L, int j, Visc2Node &o) {
    const int N = L.N;
    for (int q = 0; q < 12; ++q) o.G[q] = L.tau[q * N + j];
    o.mu = L.tau[12 * N + j];
    o.k = L.tau[13 * N + j];
    const double ri = 1.0 / L.u[j];
    o.v[0] = L.u[N + j] * ri; o.v[1] = L.u[2 * N + j] * ri; o.v[2] = L.u[3 * N + j] * ri;
    o.v[3] = (P.gamma / (P.gamma - 1.0)) * L.p[j] * ri;
    o.x[0] = L.cx[j]; o.x[1] = L.cy[j]; o.x[2] = L.cz[j];
}

// the compact flux of an edge from its first (a) and second (b) node
// (def_par:6432-6556)
__device__ __forceinline__ void visc2_edge_flux(const Visc2Node &a, const Visc2Node &b, double slen, double wx,
                                                double wy, double wz, double *f) {
    const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
    const double inv = 1.0 / slen;
    const double r[3] = {(b.x[0] - a.x[0]) * inv, (b.x[1] - a.x[1]) * inv, (b.x[2] - a.x[2]) * inv};
    double G[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int d = 0; d < 3; ++d) G[q][d] = a.G[d * 4 + q] + b.G[d * 4 + q];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double dr = (G[q][0] * r[0] + G[q][1] * r[1]) + G[q][2] * r[2];
#pragma unroll
        for (int d = 0; d < 3; ++d) G[q][d] = G[q][d] - dr * r[d];
        const double cf = q < 3 ? a.mu + b.mu : a.k + b.k;
        const double dq = cf * (b.v[q] - a.v[q]) * inv;
#pragma unroll
        for (int d = 0; d < 3; ++d) G[q][d] = G[q][d] + dq * r[d];
    }
    const double dt1 = fourThirds * G[0][0] - twoThirds * (G[1][1] + G[2][2]), dt2 = G[0][1] + G[1][0];
    const double dt3 = G[0][2] + G[2][0], dt4 = fourThirds * G[1][1] - twoThirds * (G[0][0] + G[2][2]);
    const double dt5 = G[1][2] + G[2][1], dt6 = fourThirds * G[2][2] - twoThirds * (G[0][0] + G[1][1]);
    const double dt7 = G[3][0], dt8 = G[3][1], dt9 = G[3][2];
    const double au = 0.5 * (a.v[0] + b.v[0]), av = 0.5 * (a.v[1] + b.v[1]), aw = 0.5 * (a.v[2] + b.v[2]);
    const double dut1 = (au * dt1 + av * dt2) + aw * dt3;
    const double dut2 = (au * dt2 + av * dt4) + aw * dt5;
    const double dut3 = (au * dt3 + av * dt5) + aw * dt6;
    f[0] = (wx * dt1 + wy * dt2) + wz * dt3;
    f[1] = (wx * dt2 + wy * dt4) + wz * dt5;
    f[2] = (wx * dt3 + wy * dt5) + wz * dt6;
    f[3] = (wx * (dt7 + dut1) + wy * (dt8 + dut2)) + wz * (dt9 + dut3);
}

// pass 2: the compact edge fluxes and the boundary faces' 4 w_b times each
// node's own stress, gathered per node and subtracted from the dissipation
template <int U, bool B>
__global__ void __launch_bounds__(256, U == 1 ? 2 : 1) k_visc2_flux(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    const int N = L.N;
    Visc2Node me;
    load_visc2(P, L, i, me);
    double acc[4] = {0, 0, 0, 0};
    auto iterms = [&](int k, double *g) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        Visc2Node nb;
        load_visc2(P, L, t.y, nb);
        double f[4];
        if (t.x >= 0) visc2_edge_flux(me, nb, L.slen[e], L.wx[e], L.wy[e], L.wz[e], f);
        else visc2_edge_flux(nb, me, L.slen[e], L.wx[e], L.wy[e], L.wz[e], f);
        for (int c = 0; c < 4; ++c) g[c] = t.x >= 0 ? f[c] : -f[c];
    };
    // a boundary face of this node: g[4] = 1 when it counts (not symmetry or
    // inviscid wall)
    auto bterms = [&](int k, double *g) {
        const int bb = L.binc[k] >> 1;
        const int ind = L.bind[bb];
        g[4] = (ind == 2 || ind == 9) ? 0.0 : 1.0;
        if (g[4] == 0.0) return;
        const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
        const double wx = L.bwx[bb], wy = L.bwy[bb], wz = L.bwz[bb];
        const double *G = me.G;
        const double t1 = fourThirds * G[0] - twoThirds * (G[5] + G[10]), t2 = G[4] + G[1], t3 = G[8] + G[2];
        const double t4 = fourThirds * G[5] - twoThirds * (G[0] + G[10]), t5 = G[9] + G[6];
        const double t6 = fourThirds * G[10] - twoThirds * (G[0] + G[5]);
        double t7 = G[3], t8 = G[7], t9 = G[11];
        if (P.isentropic) t7 = t8 = t9 = 0.0;
        const double *v = me.v;
        const double d1 = (v[0] * t1 + v[1] * t2) + v[2] * t3;
        const double d2 = (v[0] * t2 + v[1] * t4) + v[2] * t5;
        const double d3 = (v[0] * t3 + v[1] * t5) + v[2] * t6;
        g[0] = 4.0 * ((wx * t1 + wy * t2) + wz * t3);
        g[1] = 4.0 * ((wx * t2 + wy * t4) + wz * t5);
        g[2] = 4.0 * ((wx * t3 + wy * t5) + wz * t6);
        g[3] = 4.0 * ((wx * (t7 + d1) + wy * (t8 + d2)) + wz * (t9 + d3));
    };
    auto iadd = [&](const double *g) {
        for (int c = 0; c < 4; ++c) acc[c] = acc[c] + g[c];
    };
    auto badd = [&](const double *g) {
        if (g[4] == 0.0) return;
        for (int c = 0; c < 4; ++c) acc[c] = acc[c] + g[c];
    };
    if constexpr (U > 1) {
        group_gather<U, 4, double>(L.inc_ptr[i], L.inc_ptr[i + 1], active, gl, iterms, iadd);
        group_gather<U, 5, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, bterms, badd);
        if (!active || gl) return;
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
            double v[4];
            iterms(k, v);
            iadd(v);
        }
        for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
            double v[5];
            bterms(k, v);
            badd(v);
        }
    }
    for (int c = 0; c < 4; ++c) L.diss[(1 + c) * N + i] = L.diss[(1 + c) * N + i] - acc[c];
}

__global__ void k_fill(double *a, size_t n, double v) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// ---- computeGradient, Galerkin (def_par:2923-3245) ------------------------
__global__ void k_gradient(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    double g[15];
    for (int c = 0; c < 15; ++c) g[c] = 0.0;
    const double ri = L.u[i];
    const double qi[5] = {ri, L.u[N + i] / ri, L.u[2 * N + i] / ri, L.u[3 * N + i] / ri, L.u[4 * N + i]};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        int2 t = L.inc[k];
        int e = t.x >= 0 ? t.x : ~t.x, j = t.y;
        const double rj = L.u[j];
        const double qj[5] = {rj, L.u[N + j] / rj, L.u[2 * N + j] / rj, L.u[3 * N + j] / rj, L.u[4 * N + j]};
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 5; ++c) {
                double s = t.x >= 0 ? qi[c] + qj[c] : qj[c] + qi[c];
                double dq = s * w[a];
                g[a * 5 + c] = t.x >= 0 ? g[a * 5 + c] + dq : g[a * 5 + c] - dq;
            }
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        int2 nd = L.bedge[b];
        const double r1 = L.u[nd.x], r2 = L.u[nd.y];
        const double q1[5] = {r1, L.u[N + nd.x] / r1, L.u[2 * N + nd.x] / r1, L.u[3 * N + nd.x] / r1, L.u[4 * N + nd.x]};
        const double q2[5] = {r2, L.u[N + nd.y] / r2, L.u[2 * N + nd.y] / r2, L.u[3 * N + nd.y] / r2, L.u[4 * N + nd.y]};
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 5; ++c) {
                double s = q1[c] + q2[c];
                double own = side == 0 ? q1[c] : q2[c];
                g[a * 5 + c] = g[a * 5 + c] + (2. * own + s) * w[a];
            }
    }
    const double vt = 1. / L.V[i];
    for (int c = 0; c < 15; ++c) L.grad[c * N + i] = g[c] * vt;
}

// ---- the upwind extension's level-1 records (no reference counterpart) ----
// primitives (rho, (rho u)/rho, ..., rho E) and coordinates of every node
__global__ void k_prim_rec(LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    const double r = L.u[i];
    PrimRec o;
    o.r = r; o.u = L.u[N + i] / r; o.v = L.u[2 * N + i] / r; o.w = L.u[3 * N + i] / r; o.E = L.u[4 * N + i];
    o.x = L.cx[i]; o.y = L.cy[i]; o.z = L.cz[i];
    store_rec<PrimRec, 4>(L.qp, i, o);
}
// the Galerkin gradient of k_gradient (computeGradient, def_par:2923-3245),
// in the same summation order, from the primitive records, stored as
// component-major records
__global__ void k_gradient_rec(LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    double g[15];
#pragma unroll
    for (int c = 0; c < 15; ++c) g[c] = 0.0;
    const PrimRec Qi = load_prim(L.qp, i);
    const double qi[5] = {Qi.r, Qi.u, Qi.v, Qi.w, Qi.E};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const PrimRec Qj = load_prim(L.qp, t.y);
        const double qj[5] = {Qj.r, Qj.u, Qj.v, Qj.w, Qj.E};
        const EdgeW ew = load_edgew(L.ew, e);
        const double w[3] = {ew.wx, ew.wy, ew.wz};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const double sum = t.x >= 0 ? qi[c] + qj[c] : qj[c] + qi[c];
                const double dq = sum * w[a];
                g[a * 5 + c] = t.x >= 0 ? g[a * 5 + c] + dq : g[a * 5 + c] - dq;
            }
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const PrimRec Q1 = load_prim(L.qp, nd.x), Q2 = load_prim(L.qp, nd.y);
        const double q1[5] = {Q1.r, Q1.u, Q1.v, Q1.w, Q1.E}, q2[5] = {Q2.r, Q2.u, Q2.v, Q2.w, Q2.E};
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const double sum = q1[c] + q2[c];
                const double own = side == 0 ? q1[c] : q2[c];
                g[a * 5 + c] = g[a * 5 + c] + (2. * own + sum) * w[a];
            }
    }
    const double vt = 1. / L.V[i];
    GradRec o;
#pragma unroll
    for (int c = 0; c < 5; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) o.g[3 * c + a] = g[a * 5 + c] * vt;
    o.g[15] = 0.0;
    store_rec<GradRec, 8>(L.gq, i, o);
}

// ---- LSComputeGradient + computegradhat (def_par:2593-2920) ---------------
// the moment matrix is the same for the five scalars and is built once; the
// right-hand sides of the five scalars are gathered in the same edge order
__global__ void k_ls_gradient(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    double m[6] = {0, 0, 0, 0, 0, 0}, b[5][3];
    for (int sc = 0; sc < 5; ++sc) b[sc][0] = b[sc][1] = b[sc][2] = 0.0;
    const double ri = L.u[i];
    const double qi[5] = {ri, L.u[N + i] / ri, L.u[2 * N + i] / ri, L.u[3 * N + i] / ri, L.u[4 * N + i]};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        int2 t = L.inc[k];
        int j = t.y;
        const bool first = t.x >= 0;
        const int i1 = first ? i : j, i2 = first ? j : i;
        double dx = L.cx[i2] - L.cx[i1], dy = L.cy[i2] - L.cy[i1], dz = L.cz[i2] - L.cz[i1];
        double dist1 = 1. / ((dx * dx + dy * dy) + dz * dz);
        m[0] = m[0] + dx * dx * dist1; m[1] = m[1] + dx * dy * dist1; m[2] = m[2] + dx * dz * dist1;
        m[3] = m[3] + dy * dy * dist1; m[4] = m[4] + dy * dz * dist1; m[5] = m[5] + dz * dz * dist1;
        const double rj = L.u[j];
        const double qj[5] = {rj, L.u[N + j] / rj, L.u[2 * N + j] / rj, L.u[3 * N + j] / rj, L.u[4 * N + j]};
        for (int sc = 0; sc < 5; ++sc) {
            double dr2 = first ? qj[sc] - qi[sc] : qi[sc] - qj[sc];  // q(i2) - q(i1)
            b[sc][0] = b[sc][0] + dr2 * dx * dist1;
            b[sc][1] = b[sc][1] + dr2 * dy * dist1;
            b[sc][2] = b[sc][2] + dr2 * dz * dist1;
        }
    }
    double a11 = m[0], a12 = m[1], a13 = m[2], a21 = m[1], a22 = m[3], a23 = m[4], a31 = m[2], a32 = m[4], a33 = m[5];
    double c11 = a22 * a33 - a23 * a32, c21 = a23 * a31 - a21 * a33, c31 = a21 * a32 - a22 * a31;
    double det = (a11 * c11 + a12 * c21) + a13 * c31;
    if (fabs(det) > 0.0) det = 1.0 / det;
    c11 = det * c11; c21 = det * c21; c31 = det * c31;
    double c12 = det * (a13 * a32 - a12 * a33), c22 = det * (a11 * a33 - a13 * a31);
    double c32 = det * (a12 * a31 - a11 * a32), c13 = det * (a12 * a23 - a13 * a22);
    double c23 = det * (a13 * a21 - a23 * a11), c33 = det * (a11 * a22 - a12 * a21);
    for (int sc = 0; sc < 5; ++sc) {
        double b1 = b[sc][0], b2 = b[sc][1], b3 = b[sc][2];
        L.grad[sc * N + i] = (c11 * b1 + c12 * b2) + c13 * b3;
        L.grad[(5 + sc) * N + i] = (c21 * b1 + c22 * b2) + c23 * b3;
        L.grad[(10 + sc) * N + i] = (c31 * b1 + c32 * b2) + c33 * b3;
    }
}

// ---- LocalMinMax (def_par:3248-3459) ---------------------------------------
__global__ void k_minmax(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    double mn[5], mx[5];
    for (int c = 0; c < 5; ++c) { mn[c] = 1.0e15; mx[c] = 1.0e15; }
    const double ri = L.u[i];
    const double qi[5] = {ri, L.u[N + i] / ri, L.u[2 * N + i] / ri, L.u[3 * N + i] / ri, L.u[4 * N + i]};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        int2 t = L.inc[k];
        int j = t.y;
        const double rj = L.u[j];
        const double qj[5] = {rj, L.u[N + j] / rj, L.u[2 * N + j] / rj, L.u[3 * N + j] / rj, L.u[4 * N + j]};
        // amin1(q(i1), q(i2)) with the edge's own node order
        for (int c = 0; c < 5; ++c) {
            double a = t.x >= 0 ? qi[c] : qj[c], b = t.x >= 0 ? qj[c] : qi[c];
            mn[c] = dmin(mn[c], dmin(a, b));
            mx[c] = dmin(mx[c], dmin(-a, -b));
        }
    }
    for (int c = 0; c < 5; ++c) {
        L.bnd[c * N + i] = mn[c] - qi[c];
        L.bnd[(c + 5) * N + i] = -mx[c] - qi[c];
    }
}

// ---- interior edge flux into the edge buffer ------------------------------
// The block's fluxes (at most 256 x 5) are staged in shared memory and
// written as one contiguous run of 16-byte stores; the block size is even,
// so the run starts on a 16-byte boundary.
__device__ __forceinline__ void store_block_fluxes(double *flux, const double *sf, int e0, int count) {
    const int n = 5 * count;
    double2 *o = reinterpret_cast<double2 *>(flux + (size_t)e0 * 5);
    const double2 *src = reinterpret_cast<const double2 *>(sf);
    for (int k = threadIdx.x; k < n / 2; k += blockDim.x) o[k] = src[k];
    if ((n & 1) && threadIdx.x == 0) flux[(size_t)e0 * 5 + n - 1] = sf[n - 1];
}
template <int FT, bool O2>
__global__ void __launch_bounds__(256) k_edge_flux(Params P, LevelView L) {
    __shared__ __align__(16) double sf[256 * 5];
    const int e0 = blockIdx.x * blockDim.x, e = e0 + threadIdx.x;
    if (e < L.E) {
        const int2 nd = L.edge[e];
        double f[5];
        edge_flux<FT, O2>(P, L, e, nd.x, nd.y, f);
#pragma unroll
        for (int k = 0; k < 5; ++k) sf[threadIdx.x * 5 + k] = f[k];
    }
    __syncthreads();
    store_block_fluxes(L.flux, sf, e0, min((int)blockDim.x, L.E - e0));
}
template __global__ void k_edge_flux<1, false>(Params, LevelView);
template __global__ void k_edge_flux<2, false>(Params, LevelView);
template __global__ void k_edge_flux<3, false>(Params, LevelView);
template __global__ void k_edge_flux<3, true>(Params, LevelView);
template __global__ void k_edge_flux<4, false>(Params, LevelView);
template __global__ void k_edge_flux<4, true>(Params, LevelView);

// the upwind extension's level-1 edge flux into the edge buffer, stored as
// k_edge_flux stores
__global__ void __launch_bounds__(256) k_edge_flux_muscl(Params P, LevelView L) {
    __shared__ __align__(16) double sf[256 * 5];
    const int e0 = blockIdx.x * blockDim.x, e = e0 + threadIdx.x;
    if (e < L.E) {
        const int2 nd = L.edge[e];
        double f[5];
        edge_flux_muscl(P, L, e, nd.x, nd.y, f);
#pragma unroll
        for (int k = 0; k < 5; ++k) sf[threadIdx.x * 5 + k] = f[k];
    }
    __syncthreads();
    store_block_fluxes(L.flux, sf, e0, min((int)blockDim.x, L.E - e0));
}

// ---- boundary-edge contributions ------------------------------------------
template <bool B>
__global__ void k_bnd_flux(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    int b = tid();
    if (b >= L.B) return;
    double g1[5], g2[5];
    boundary_flux(P, L, b, g1, g2);
    double *o = L.bflux + (size_t)b * 10;
    for (int k = 0; k < 5; ++k) { o[k] = g1[k]; o[5 + k] = g2[k]; }
    if (L.bgterm) {
        boundary_gcl(P, L, b, g1, g2);
        double *t = L.bgterm + (size_t)b * 10;
        for (int k = 0; k < 5; ++k) { t[k] = g1[k]; t[5 + k] = g2[k]; }
    }
}

// ---- mixed precision ------------------------------------------------------
// The interior central flux of an edge is G(u1; w) + G(u2; w) with the
// one-sided flux G(u; w) = F(u).w.  FLITE_MIXED evaluates it as
//   G(u; w) = G(ua; w) + dG,
// where ua is an FP64 anchor state whose interior-edge residual was summed in
// FP64, and dG is computed in FP32 from the increments du = u - ua and
// dp = p - pa in a form whose every term carries an increment:
//   dv   = (dm - va drho) / rho
//   dG_0 = dm.w
//   dG_k = dm_k (v.w) + ma_k (dv.w) + dp w_k          k = 1..3
//   dG_4 = (dE + dp)(v.w) + (Ea + pa)(dv.w)
// so its rounding error is relative to the increment, not to the flux: the
// iteration converges to the FP64 fixed point.  The anchor is refreshed by an
// FP64 evaluation at the first stage of every relaxation step (and at the
// coarse-level evaluation of restrictGrid).

// the node's record for the increments: anchor primitives and u - ua (FP64
// difference, rounded once), p - pa
template <bool B>
__global__ void k_delta_state(CaseArg<B, LevelView> L_) {
    FLITE_CASE_L(B, L);
    int i = tid();
    if (i >= L.N) return;
    const int N = L.N;
    DeltaRec o;
    o.ra = L.a32[i]; o.vax = L.a32[N + i]; o.vay = L.a32[2 * N + i]; o.vaz = L.a32[3 * N + i];
    o.ha = L.a32[4 * N + i];
    o.dr = (float)(L.u[i] - L.ua[i]);
    o.dmx = (float)(L.u[N + i] - L.ua[N + i]);
    o.dmy = (float)(L.u[2 * N + i] - L.ua[2 * N + i]);
    o.dmz = (float)(L.u[3 * N + i] - L.ua[3 * N + i]);
    o.dE = (float)(L.u[4 * N + i] - L.ua[4 * N + i]);
    o.dp = (float)(L.p[i] - L.pa[i]);
    o.pad = 0.f;
    float4 *p = reinterpret_cast<float4 *>(L.dq + i);
    const float4 *d = reinterpret_cast<const float4 *>(&o);
    p[0] = d[0]; p[1] = d[1]; p[2] = d[2];
}

// FP32 incidences of the increments (w rounded once; j is ~j when the node
// is the edge's second node)
__global__ void k_make_inc32(const int2 *inc, const EdgeW *ew, int n, IncRec32 *o) {
    int k = tid();
    if (k >= n) return;
    const int2 t = inc[k];
    const EdgeW w = ew[t.x >= 0 ? t.x : ~t.x];
    o[k] = IncRec32{(float)w.wx, (float)w.wy, (float)w.wz, t.x >= 0 ? t.y : ~t.y};
}

__device__ __forceinline__ DeltaRec load_delta(const DeltaRec *q, int j) {
    const float4 *p = reinterpret_cast<const float4 *>(q + j);
    DeltaRec o;
    float4 *d = reinterpret_cast<float4 *>(&o);
    d[0] = __ldg(p); d[1] = __ldg(p + 1); d[2] = __ldg(p + 2);
    return o;
}

// increment of the one-sided flux G(u; w) of one node
__device__ __forceinline__ void delta_flux(const DeltaRec &n, float wx, float wy, float wz, float *g) {
    const float rinv = 1.f / (n.ra + n.dr);
    const float dvx = (n.dmx - n.vax * n.dr) * rinv, dvy = (n.dmy - n.vay * n.dr) * rinv;
    const float dvz = (n.dmz - n.vaz * n.dr) * rinv;
    const float vw = ((n.vax + dvx) * wx + (n.vay + dvy) * wy) + (n.vaz + dvz) * wz;
    const float dvw = (dvx * wx + dvy * wy) + dvz * wz;
    g[0] = (n.dmx * wx + n.dmy * wy) + n.dmz * wz;
    g[1] = (n.dmx * vw + (n.ra * n.vax) * dvw) + n.dp * wx;
    g[2] = (n.dmy * vw + (n.ra * n.vay) * dvw) + n.dp * wy;
    g[3] = (n.dmz * vw + (n.ra * n.vaz) * dvw) + n.dp * wz;
    g[4] = (n.dE + n.dp) * vw + n.ha * dvw;
}

// interior residual of node i as the anchor's FP64 sum plus the FP32 sum of
// the flux increments of its edges
template <int U>
__device__ __forceinline__ void gather_interior_delta(const LevelView &L, int i, double *r, bool active = true,
                                         int gl = 0) {
    float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    const DeltaRec me = load_delta(L.dq, i);
    auto terms = [&](int k, float *s5, bool &first) {
        const IncRec32 t = load_inc32(L.inc32, k);
        first = t.j >= 0;
        const DeltaRec nb = load_delta(L.dq, first ? t.j : ~t.j);
        float g1[5], g2[5];
        delta_flux(first ? me : nb, t.wx, t.wy, t.wz, g1);
        delta_flux(first ? nb : me, t.wx, t.wy, t.wz, g2);
        for (int c = 0; c < 5; ++c) s5[c] = g1[c] + g2[c];
    };
    if constexpr (U > 1) {
        // the terms carry the node's sign of the edge as a sixth value
        group_gather<U, 6, float>(
            L.inc_ptr[i], L.inc_ptr[i + 1], active, gl,
            [&](int k, float *v) {
                bool first;
                terms(k, v, first);
                v[5] = first ? 1.f : 0.f;
            },
            [&](const float *x) {
                const bool f = x[5] != 0.f;
                for (int c = 0; c < 5; ++c) acc[c] = f ? acc[c] + x[c] : acc[c] - x[c];
            });
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
            float v[5];
            bool first;
            terms(k, v, first);
            if (first) {
                for (int c = 0; c < 5; ++c) acc[c] += v[c];
            } else {
                for (int c = 0; c < 5; ++c) acc[c] -= v[c];
            }
        }
    }
    const int N = L.N;
    for (int c = 0; c < 5; ++c) r[c] = L.ra[c * N + i] + (double)acc[c];
}

// the same sum with the loads of two incidences issued before either flux
// is computed (more loads in flight per thread); the additions stay in edge
// order, so the result is the same bit for bit
__device__ __forceinline__ void gather_interior_central2(const LevelView &L, int i, double *r) {
    r[0] = r[1] = r[2] = r[3] = r[4] = 0.0;
    const NodeRec si = load_node(L.q, i);
    const int end = L.inc_ptr[i + 1];
    int k = L.inc_ptr[i];
    auto add = [&](const int2 t, const EdgeW &w, const NodeRec &n) {
        const NodeRec &sj = n;
        double f[5];
        if (t.x >= 0) {
            central_flux_rec(si, sj, w.wx, w.wy, w.wz, f);
            r[0] = r[0] + f[0]; r[1] = r[1] + f[1]; r[2] = r[2] + f[2]; r[3] = r[3] + f[3]; r[4] = r[4] + f[4];
        } else {
            central_flux_rec(sj, si, w.wx, w.wy, w.wz, f);
            r[0] = r[0] - f[0]; r[1] = r[1] - f[1]; r[2] = r[2] - f[2]; r[3] = r[3] - f[3]; r[4] = r[4] - f[4];
        }
    };
    for (; k + 1 < end; k += 2) {
        const int2 t0 = L.inc[k], t1 = L.inc[k + 1];
        const EdgeW w0 = load_edgew(L.ew, t0.x >= 0 ? t0.x : ~t0.x);
        const EdgeW w1 = load_edgew(L.ew, t1.x >= 0 ? t1.x : ~t1.x);
        const NodeRec n0 = load_node(L.q, t0.y), n1 = load_node(L.q, t1.y);
        add(t0, w0, n0);
        add(t1, w1, n1);
    }
    if (k < end) {
        const int2 t0 = L.inc[k];
        add(t0, load_edgew(L.ew, t0.x >= 0 ? t0.x : ~t0.x), load_node(L.q, t0.y));
    }
}

// interior central fluxes of node i computed from the two node records of
// each incident edge, summed in edge order: the same numbers, in the same
// order, as the edge kernel followed by the buffer gather
template <int U>
__device__ __forceinline__ void gather_interior_central(const LevelView &L, int i, double *r, bool active = true,
                                         int gl = 0) {
    r[0] = r[1] = r[2] = r[3] = r[4] = 0.0;
    const NodeRec si = load_node(L.q, i);
    // the flux of incidence k with this node's sign (x - y is x + (-y))
    auto terms = [&](int k, double *g) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const EdgeW w = load_edgew(L.ew, e);
        const NodeRec n = load_node(L.q, t.y);
        double f[5];
        if (t.x >= 0) {
            central_flux_rec(si, n, w.wx, w.wy, w.wz, f);
            for (int c = 0; c < 5; ++c) g[c] = f[c];
        } else {
            central_flux_rec(n, si, w.wx, w.wy, w.wz, f);
            for (int c = 0; c < 5; ++c) g[c] = -f[c];
        }
    };
    auto add = [&](const double *g) {
        r[0] = r[0] + g[0]; r[1] = r[1] + g[1]; r[2] = r[2] + g[2]; r[3] = r[3] + g[3]; r[4] = r[4] + g[4];
    };
    if constexpr (U > 1) {
        group_gather<U, 5, double>(L.inc_ptr[i], L.inc_ptr[i + 1], active, gl, terms, add);
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
            double v[5];
            terms(k, v);
            add(v);
        }
    }
}

// interior edges of node i from the FP64 edge buffer, in edge order
template <int U>
__device__ __forceinline__ void gather_interior(const LevelView &L, int i, double *r, bool active = true,
                                         int gl = 0) {
    r[0] = r[1] = r[2] = r[3] = r[4] = 0.0;
    auto terms = [&](int k, double *g) {
        const int s = L.inc[k].x;
        const double *f = L.flux + (size_t)(s >= 0 ? s : ~s) * 5;
        for (int c = 0; c < 5; ++c) g[c] = s >= 0 ? f[c] : -f[c];  // x - y is x + (-y)
    };
    auto add = [&](const double *g) {
        r[0] = r[0] + g[0]; r[1] = r[1] + g[1]; r[2] = r[2] + g[2]; r[3] = r[3] + g[3]; r[4] = r[4] + g[4];
    };
    if constexpr (U > 1) {
        group_gather<U, 5, double>(L.inc_ptr[i], L.inc_ptr[i + 1], active, gl, terms, add);
    } else {
        for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
            double v[5];
            terms(k, v);
            add(v);
        }
    }
}

// boundary edges of node i (FP64).  On a moving mesh each boundary edge
// first subtracts its GCL terms from both its nodes, then adds its fluxes
// (def_par:2124-2177): per node -t, +g; an edge with both ends at node i (a
// coarse level's self-edge) gives -t1, -t2, +g1, +g2, its second end's
// entry following its first in the node's list
template <int U>
__device__ __forceinline__ void gather_boundary(const LevelView &L, int i, double *r, bool active = true,
                                         int gl = 0) {
    auto terms = [&](int k, double *g) {
        const int v = L.binc[k];
        const double *b = L.bflux + (size_t)(v >> 1) * 10 + (v & 1) * 5;
        for (int c = 0; c < 5; ++c) g[c] = b[c];
    };
    auto add = [&](const double *g) {
        r[0] = r[0] + g[0]; r[1] = r[1] + g[1]; r[2] = r[2] + g[2]; r[3] = r[3] + g[3]; r[4] = r[4] + g[4];
    };
    // g[0..4] the GCL term, g[5..9] the flux, g[10] 0 (an edge between two
    // nodes), 1 or 2 (first or second end of a self-edge)
    auto terms_gcl = [&](int k, double *g) {
        const int v = L.binc[k];
        const size_t o = (size_t)(v >> 1) * 10 + (v & 1) * 5;
        for (int c = 0; c < 5; ++c) { g[c] = L.bgterm[o + c]; g[5 + c] = L.bflux[o + c]; }
        const int2 nd = L.bedge[v >> 1];
        g[10] = nd.x == nd.y ? (double)(1 + (v & 1)) : 0.0;
    };
    double pend[5];  // the flux of a self-edge's first end, added after its second GCL term
    auto add_gcl = [&](const double *g) {
        if (g[10] == 1.0) {
            for (int c = 0; c < 5; ++c) { r[c] = r[c] - g[c]; pend[c] = g[5 + c]; }
        } else if (g[10] == 2.0) {
            for (int c = 0; c < 5; ++c) r[c] = ((r[c] - g[c]) + pend[c]) + g[5 + c];
        } else {
            for (int c = 0; c < 5; ++c) r[c] = (r[c] - g[c]) + g[5 + c];
        }
    };
    if constexpr (U > 1) {
        if (L.bgterm) group_gather<U, 11, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, terms_gcl, add_gcl);
        else group_gather<U, 5, double>(L.binc_ptr[i], L.binc_ptr[i + 1], active, gl, terms, add);
    } else if (L.bgterm) {
        for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
            double v[11];
            terms_gcl(k, v);
            add_gcl(v);
        }
    } else {
        for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
            double v[5];
            terms(k, v);
            add(v);
        }
    }
}

// the FP64 evaluation becomes the new anchor of node i
__device__ __forceinline__ void store_anchor(const LevelView &L, int i, const double *rint) {
    const int N = L.N;
    double u[5];
    for (int c = 0; c < 5; ++c) {
        u[c] = L.u[c * N + i];
        L.ua[c * N + i] = u[c];
        L.ra[c * N + i] = rint[c];
    }
    const double p = L.p[i];
    L.pa[i] = p;
    const double rinv = 1.0 / u[0];
    L.a32[i] = (float)u[0];
    L.a32[N + i] = (float)(u[1] * rinv);
    L.a32[2 * N + i] = (float)(u[2] * rinv);
    L.a32[3 * N + i] = (float)(u[3] * rinv);
    L.a32[4 * N + i] = (float)(u[4] + p);
}

// the node part of a stage after the residual r of node i is summed:
// time differences, dissipation, solveSystem, the increment conditions, the
// clipped update and the solution and outer conditions, or the restrictGrid
// one-step forms (modes as in k_node_update)
// LEAN: a run without engine conditions and without explicit time stepping
// (the branches for those are left out of the code)
template <bool LEAN = false>
__device__ __forceinline__ void node_tail(const Params &P, const LevelView &L, int i, double *r, int mode,
                                          int stage) {
    const int N = L.N;
    if (mode == MODE_RESID) {
        for (int c = 0; c < 5; ++c) L.rhs[c * N + i] = r[c];
        return;
    }
    if (P.addts && mode == MODE_STAGE)  // addTimeDifferences (def_par:1184-1241)
        for (int c = 0; c < 5; ++c) r[c] = r[c] + time_difference(P, L, i, c);
    for (int c = 0; c < 5; ++c) r[c] = r[c] + L.diss[c * N + i];
    double dt = L.dt[i];
    const double V = L.V[i];
    // solveSystem's dual-time step, or the explicit global step (def_par:1427-1442)
    if (P.unsteady) dt = (!LEAN && P.explicit_) ? *L.ptsg : dt / (1.0 + 1.5 * dt / P.dtp);
    for (int c = 0; c < 5; ++c) r[c] = dt * r[c] / V;  // solveSystem
    const unsigned char cls = L.bc[i];
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = L.nx[i]; n1 = L.ny[i]; n2 = L.nz[i]; }
    bc_increment<!LEAN>(P, cls, n0, n1, n2, r);
    // nullifyOuterBoundary (coarse levels): zeroes the far-field (indicator
    // 3) and engine increments for the SA model and is a no-op otherwise
    if (P.sa && L.grid > 1 && (cls == BC_FAR3 || (!LEAN && is_engine(cls)))) r[0] = r[1] = r[2] = r[3] = r[4] = 0.0;
    const double dtJ = stage > 0 ? P.CFL * P.RK[stage - 1] : P.CFL;
    double d[5], up[5], un[5];
    for (int c = 0; c < 5; ++c) { d[c] = dtJ * r[c]; up[c] = L.uprev[c * N + i]; }
    clipped_update(P, up, d, un);
    if (mode == MODE_RFINE) {
        // the density floor of updateSolutionVector acts on grp%u, which is
        // not the array being updated in this call (def_par:1398-1403)
        if (L.u[i] < P.minRho) L.u[i] = P.minRho;
    } else {
        if (un[0] < P.minRho) un[0] = P.minRho;
    }
    double cm0 = 0, cm1 = 0, cm2 = 0;
    if (cls == BC_WALL && P.viscous) { cm0 = L.cmx[i]; cm1 = L.cmy[i]; cm2 = L.cmz[i]; }
    bc_solution(P, cls, n0, n1, n2, cm0, cm1, cm2, relax_param(P, *L.cyc), un);
    if (!LEAN && is_exhaust(cls)) {
        // the exhaust pressure matters on level 1 only: coarse pressures are
        // recomputed before anything reads them
        const double pex = bc_exhaust(P, cls, eo_relax(P, *L.cyc), un);
        if (L.eng.f) L.eng.pbc[i] = pex;
    }
    if (!LEAN && L.eng.f && mode != MODE_RCOARSE && (P.eftype == 2 || is_engine(cls))) {
        // level 1: the engine inlet terms need every node's state first;
        // k_engine_finish completes the node (the candidate state of
        // restrictGrid's fine step goes to rhs)
        double *T = mode == MODE_RFINE ? L.rhs : L.u;
        for (int c = 0; c < 5; ++c) T[c * N + i] = un[c];
        return;
    }
    if (mode == MODE_STAGE) {
        if (L.grid > 1) {
            const double a = P.RK[stage - 1];
            for (int c = 0; c < 5; ++c) un[c] = un[c] - a * L.src[c * N + i];
        }
        un[0] = dmax(un[0], P.minRho);  // limitDensity
        bc_outer(P, cls, n0, n1, n2, L.p[i], un);
        for (int c = 0; c < 5; ++c) L.u[c * N + i] = un[c];
    } else if (mode == MODE_RCOARSE) {
        bc_outer(P, cls, n0, n1, n2, L.p[i], un);
        for (int c = 0; c < 5; ++c) L.src[c * N + i] = un[c] - up[c];
    } else {  // MODE_RFINE
        if (L.grid > 1)
            for (int c = 0; c < 5; ++c) un[c] = un[c] - L.src[c * N + i];
        bc_outer(P, cls, n0, n1, n2, L.p[i], un);
        for (int c = 0; c < 5; ++c) L.rhs[c * N + i] = un[c] - up[c];
    }
}

// ---- the node part of one RK stage (def_par:1069-1178), fused -------------
// mode STAGE:   u <- update of stage `stage`
// mode RCOARSE: restrictGrid coarse one-step (def_par:12244-12263): src
// mode RFINE:   restrictGrid fine increment (def_par:12356-12383): rhs
// mode RESID:   rhs <- makeRHS only
// PREC: GATHER_BUFFER (FP64 edge buffer of the upwind fluxes),
// GATHER_CENTRAL (central fluxes computed in the gather), GATHER_ANCHOR (the
// same, stored as the new mixed-precision anchor), GATHER_DELTA (anchor +
// FP32 increments)
template <int PREC, int U, bool B>
__global__ void __launch_bounds__(256, PREC == GATHER_CENTRAL2 ? 2 : (U == 1 ? 3 : 1))
    k_node_update(CaseArg<B, Params> P_, CaseArg<B, LevelView> L_, int mode, int stage) {
    FLITE_CASE_P(B, P, L);
    FLITE_CASE_L(B, L);
    const int gl = U > 1 ? (int)(threadIdx.x % U) : 0;  // lane in the node's group
    const int i_raw = U > 1 ? tid() / U : tid();
    if (U == 1 && i_raw >= L.N) return;
    const bool active = i_raw < L.N;
    const int i = active ? i_raw : L.N - 1;  // idle groups read a valid node
    double r[5];
    if constexpr (PREC == GATHER_DELTA) {
        gather_interior_delta<U>(L, i, r, active, gl);
    } else if constexpr (PREC == GATHER_BUFFER) {
        gather_interior<U>(L, i, r, active, gl);
    } else if constexpr (PREC == GATHER_CENTRAL2) {
        gather_interior_central2(L, i, r);
    } else {
        gather_interior_central<U>(L, i, r, active, gl);
    }
    double rint[5];
    if constexpr (PREC == GATHER_ANCHOR)
        for (int c = 0; c < 5; ++c) rint[c] = r[c];
    gather_boundary<U>(L, i, r, active, gl);
    // with a group per node every lane holds the same sums; one lane goes on
    if constexpr (U > 1)
        if (!active || gl) return;
    if constexpr (PREC == GATHER_ANCHOR) store_anchor(L, i, rint);
    node_tail<PREC == GATHER_LEAN>(P, L, i, r, mode, stage);
}
// ---- the same node update with the central fluxes gathered from a
// shared-memory stage of the node block (GATHER_CENTRAL, a thread per node).
// Block t handles the kTile nodes t*kTile.. of the level; it first copies
// their 48-byte records and those of the block's halo (the other nodes its
// edges reach, in increasing node order) into shared memory with coalesced
// or independent loads, then every thread walks its node's incidences in
// edge order through the block's incidence rows (row k holds incidence k of
// every node of the block: the coefficients and the staged slot of the
// other node, read with coalesced loads).  A neighbour beyond the stage's
// capacity is read from the global records.  The flux of each incidence and
// the order of the additions are those of k_node_update, so the results are
// identical bit for bit.
__device__ __forceinline__ NodeRec load_node_shared(const NodeRec *rec, int slot) {
    const float4 *p = reinterpret_cast<const float4 *>(rec + slot);
    NodeRec o;
    float4 *d = reinterpret_cast<float4 *>(&o);
    d[0] = p[0]; d[1] = p[1]; d[2] = p[2];
    return o;
}

template <bool STAGE, bool AHEAD>
__global__ void __launch_bounds__(kTile, AHEAD ? 2 : 3) k_node_update_tiled(Params P, LevelView L, int mode,
                                                                            int stage) {
    extern __shared__ float4 stage_mem[];
    NodeRec *rec = reinterpret_cast<NodeRec *>(stage_mem);
    const TileView &T = L.tile;
    const int t = blockIdx.x, n0 = t * kTile;
    const int cnt = min(kTile, L.N - n0);
    if (STAGE) {
        const int h0 = T.halo_ptr[t];
        const int nh = min(T.halo_ptr[t + 1] - h0, kTileStageMax - kTile);
        const float4 *q = reinterpret_cast<const float4 *>(L.q);
        // 16-byte pieces: 3 per record, own records then the halo's
        for (int s = threadIdx.x; s < 3 * (cnt + nh); s += blockDim.x) {
            const int r = s / 3, part = s - 3 * r;
            const int j = r < cnt ? n0 + r : T.halo[h0 + (r - cnt)];
            const int slot = r < cnt ? r : kTile + (r - cnt);
            stage_mem[3 * slot + part] = __ldg(q + 3 * (size_t)j + part);
        }
        __syncthreads();
    }
    if ((int)threadIdx.x >= cnt) return;
    const int i = n0 + threadIdx.x;
    const NodeRec si = STAGE ? load_node_shared(rec, threadIdx.x) : load_node(L.q, i);
    const int deg = L.inc_ptr[i + 1] - L.inc_ptr[i];
    const size_t base = (size_t)T.row[t] * kTile + threadIdx.x;
    const unsigned *meta = STAGE ? T.meta : T.nmeta;
    auto fetch = [&](unsigned m) -> NodeRec {
        const int v = (int)(m & kTileIndexMask);
        if (!STAGE || (m & kTileGlobal)) return load_node(L.q, v);
        return load_node_shared(rec, v);
    };
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (!AHEAD) {
        for (int k = 0; k < deg; ++k) {
            const size_t x = base + (size_t)k * kTile;
            const unsigned m = __ldg(meta + x);
            const double wx = __ldg(T.wx + x), wy = __ldg(T.wy + x), wz = __ldg(T.wz + x);
            const NodeRec n = fetch(m);
            double f[5];
            if (!(m & kTileSecond)) {
                central_flux_rec(si, n, wx, wy, wz, f);
                r[0] = r[0] + f[0]; r[1] = r[1] + f[1]; r[2] = r[2] + f[2]; r[3] = r[3] + f[3]; r[4] = r[4] + f[4];
            } else {
                central_flux_rec(n, si, wx, wy, wz, f);
                r[0] = r[0] + (-f[0]); r[1] = r[1] + (-f[1]); r[2] = r[2] + (-f[2]); r[3] = r[3] + (-f[3]);
                r[4] = r[4] + (-f[4]);
            }
        }
        gather_boundary<1>(L, i, r);
        node_tail(P, L, i, r, mode, stage);
        return;
    }
    // the loads of incidence k+1 are issued before incidence k is evaluated
    unsigned m0 = 0;
    double wx0 = 0, wy0 = 0, wz0 = 0;
    NodeRec n0r{};
    if (deg > 0) {
        m0 = __ldg(meta + base);
        wx0 = __ldg(T.wx + base); wy0 = __ldg(T.wy + base); wz0 = __ldg(T.wz + base);
        n0r = fetch(m0);
    }
    for (int k = 0; k < deg; ++k) {
        unsigned m1 = 0;
        double wx1 = 0, wy1 = 0, wz1 = 0;
        NodeRec n1r{};
        if (k + 1 < deg) {
            const size_t x = base + (size_t)(k + 1) * kTile;
            m1 = __ldg(meta + x);
            wx1 = __ldg(T.wx + x); wy1 = __ldg(T.wy + x); wz1 = __ldg(T.wz + x);
            n1r = fetch(m1);
        }
        double f[5];
        if (!(m0 & kTileSecond)) {
            central_flux_rec(si, n0r, wx0, wy0, wz0, f);
            r[0] = r[0] + f[0]; r[1] = r[1] + f[1]; r[2] = r[2] + f[2]; r[3] = r[3] + f[3]; r[4] = r[4] + f[4];
        } else {
            central_flux_rec(n0r, si, wx0, wy0, wz0, f);
            r[0] = r[0] + (-f[0]); r[1] = r[1] + (-f[1]); r[2] = r[2] + (-f[2]); r[3] = r[3] + (-f[3]);
            r[4] = r[4] + (-f[4]);
        }
        m0 = m1; wx0 = wx1; wy0 = wy1; wz0 = wz1; n0r = n1r;
    }
    gather_boundary<1>(L, i, r);
    node_tail(P, L, i, r, mode, stage);
}

// ---- the other gathers of a level through the incidence rows of node blocks
// Each kernel walks its node's incidences in edge order through the block's
// incidence rows (row k holds incidence k of each node of the block), with
// the loads of incidence k+1 issued before incidence k is evaluated.  With
// STAGE the K node fields (SoA arrays) it reads at the other node are first
// copied for the block and its halo into shared memory as sm[slot*K + c];
// without, they are read from the global arrays.  The per-incidence
// arithmetic and the order of the additions are those of the kernels'
// thread-per-node forms above, so the results are identical bit for bit.
template <int K>
__device__ __forceinline__ void stage_fields(double *sm, const TileView &T, const double *const *f, int n0, int cnt,
                                             int h0, int nh) {
#pragma unroll 1
    for (int c = 0; c < K; ++c)
        for (int s = threadIdx.x; s < cnt + nh; s += blockDim.x) {
            const int j = s < cnt ? n0 + s : T.halo[h0 + (s - cnt)];
            const int slot = s < cnt ? s : kTile + (s - cnt);
            sm[slot * K + c] = __ldg(f[c] + j);
        }
}

// the block of the calling thread and its halo (staged part), with the
// fields staged when STAGE; returns the node, or -1 for the block's idle
// threads
template <int K, bool STAGE>
__device__ __forceinline__ int tile_begin(double *sm, const LevelView &L, const double *const *f) {
    const int n0 = blockIdx.x * kTile;
    const int cnt = min(kTile, L.N - n0);
    if (STAGE && K > 0) {
        const int h0 = L.tile.halo_ptr[blockIdx.x];
        const int nh = min(L.tile.halo_ptr[blockIdx.x + 1] - h0, kTileStageMax - kTile);
        stage_fields<K>(sm, L.tile, f, n0, cnt, h0, nh);
        __syncthreads();
    }
    return (int)threadIdx.x < cnt ? n0 + (int)threadIdx.x : -1;
}

// one incidence of the row walk: the other node's K fields, the flags and
// (when W) the edge coefficients
template <int K, bool STAGE, bool W>
struct Inc {
    unsigned m;
    double w[3];
    double v[K > 0 ? K : 1];
    __device__ __forceinline__ void load(const LevelView &L, const double *sm, const double *const *f, size_t x) {
        m = __ldg((STAGE ? L.tile.meta : L.tile.nmeta) + x);
        if (W) { w[0] = __ldg(L.tile.wx + x); w[1] = __ldg(L.tile.wy + x); w[2] = __ldg(L.tile.wz + x); }
        const int idx = (int)(m & kTileIndexMask);
        if (!STAGE || (m & kTileGlobal)) {
#pragma unroll
            for (int c = 0; c < K; ++c) v[c] = __ldg(f[c] + idx);
        } else {
#pragma unroll
            for (int c = 0; c < K; ++c) v[c] = sm[idx * K + c];
        }
    }
    __device__ __forceinline__ bool first() const { return !(m & kTileSecond); }
};

// walk node i's incidence rows calling fn(inc) in edge order (AHEAD: the
// loads of incidence k+1 issued before fn sees incidence k)
template <int K, bool STAGE, bool W, bool AHEAD, class Fn>
__device__ __forceinline__ void row_walk(const LevelView &L, const double *sm, const double *const *f, int i,
                                         Fn &&fn) {
    const int deg = L.inc_ptr[i + 1] - L.inc_ptr[i];
    const size_t base = (size_t)L.tile.row[blockIdx.x] * kTile + threadIdx.x;
    if (deg <= 0) return;
    if (!AHEAD) {
        for (int k = 0; k < deg; ++k) {
            Inc<K, STAGE, W> a;
            a.load(L, sm, f, base + (size_t)k * kTile);
            fn(a);
        }
        return;
    }
    Inc<K, STAGE, W> a, b;
    a.load(L, sm, f, base);
    for (int k = 0; k < deg; ++k) {
        if (k + 1 < deg) b.load(L, sm, f, base + (size_t)(k + 1) * kTile);
        fn(a);
        a = b;
    }
}

// makeTimeSteps: K = 0 (inviscid: the other node is not read), 2 (mu, rho),
// 3 (with the SA nu~)
template <int K, bool STAGE, bool AHEAD>
__global__ void __launch_bounds__(kTile, 3) k_timestep_tiled(Params P, LevelView L) {
    extern __shared__ double sm[];
    const int N = L.N;
    const double *f[3] = {L.mu, L.u, L.u + 5 * (size_t)N};
    const int i = tile_begin<K, STAGE>(sm, L, f);
    if (i < 0) return;
    const double c1 = P.gamma;
    const double ri = L.u[i], ro = 1. / ri;
    const double m1 = L.u[N + i], m2 = L.u[2 * N + i], m3 = L.u[3 * N + i];
    const double cc = dmax(c1 * L.p[i] * ro, 0.001);
    double acc = 0.0, h = 0.0;
    row_walk<K, STAGE, true, AHEAD>(L, sm, f, i, [&](const Inc<K, STAGE, true> &t) {
        const double wx = t.w[0], wy = t.w[1], wz = t.w[2];
        double al = (wx * wx + wy * wy) + wz * wz;
        double vn = ((wx * m1 + wy * m2) + wz * m3) * ro;
        acc = (acc + fabs(vn)) + sqrt(cc * al);
        if (K > 0) {
            double vis = dmax(P.am, K == 3 ? t.v[0] + t.v[K == 3 ? 2 : 0] / P.Re : t.v[0]);
            double dv = 2.0 * vis * al / t.v[K > 1 ? 1 : 0];
            h = h + dv;
        }
    });
    ts_finish(P, L, i, acc, h);
}

// makeArtificialDissipation2 passes 1-2 (no dissipation weighting): the
// other node's u and p
template <bool STAGE, bool AHEAD>
__global__ void __launch_bounds__(kTile, 3) k_jst_lap_tiled(Params P, LevelView L) {
    extern __shared__ double sm[];
    const int N = L.N;
    const double *f[6] = {L.u, L.u + N, L.u + 2 * (size_t)N, L.u + 3 * (size_t)N, L.u + 4 * (size_t)N, L.p};
    const int i = tile_begin<6, STAGE>(sm, L, f);
    if (i < 0) return;
    double l0 = 0, l1 = 0, l2 = 0, l3 = 0, l4 = 0, s7 = 0, s8 = 0;
    const double ui0 = L.u[i], ui1 = L.u[N + i], ui2 = L.u[2 * N + i], ui3 = L.u[3 * N + i], ui4 = L.u[4 * N + i];
    const double pi = L.p[i];
    const double df = 1.0;
    row_walk<6, STAGE, false, AHEAD>(L, sm, f, i, [&](const Inc<6, STAGE, false> &t) {
        const double uj0 = t.v[0], uj1 = t.v[1], uj2 = t.v[2], uj3 = t.v[3], uj4 = t.v[4], pj = t.v[5];
        if (t.first()) {
            double d0 = ui0 - uj0, d1 = ui1 - uj1, d2 = ui2 - uj2, d3 = ui3 - uj3;
            double d4 = ((ui4 - uj4) + pi) - pj;
            l0 = l0 - d0 * df; l1 = l1 - d1 * df; l2 = l2 - d2 * df; l3 = l3 - d3 * df; l4 = l4 - d4 * df;
            double dp = pi - pj, sp = pi + pj;
            s7 = s7 - dp; s8 = s8 + sp;
        } else {
            double d0 = uj0 - ui0, d1 = uj1 - ui1, d2 = uj2 - ui2, d3 = uj3 - ui3;
            double d4 = ((uj4 - ui4) + pj) - pi;
            l0 = l0 + d0 * df; l1 = l1 + d1 * df; l2 = l2 + d2 * df; l3 = l3 + d3 * df; l4 = l4 + d4 * df;
            double dp = pj - pi, sp = pj + pi;
            s7 = s7 + dp; s8 = s8 + sp;
        }
    });
    double fact = 1. / L.conn[i];
    L.sens[i] = 12. * fabs(s7 / s8);
    L.lap[i] = fact * l0;
    L.lap[N + i] = fact * l1;
    L.lap[2 * N + i] = fact * l2;
    L.lap[3 * N + i] = fact * l3;
    L.lap[4 * N + i] = fact * l4;
}

// makeArtificialDissipation2 pass 3, scalar: the other node's V/dt,
// connectivity, sensor, Laplacian and u
template <bool STAGE, bool AHEAD>
__global__ void __launch_bounds__(kTile, AHEAD ? 2 : 3) k_jst_flux_tiled(Params P, LevelView L) {
    extern __shared__ double sm[];
    const int N = L.N;
    const double *f[13] = {L.vdt, L.conn, L.sens,
                           L.lap, L.lap + N, L.lap + 2 * (size_t)N, L.lap + 3 * (size_t)N, L.lap + 4 * (size_t)N,
                           L.u, L.u + N, L.u + 2 * (size_t)N, L.u + 3 * (size_t)N, L.u + 4 * (size_t)N};
    const int i = tile_begin<13, STAGE>(sm, L, f);
    if (i < 0) return;
    const double k4 = L.grid == 1 ? P.k4 : P.cgdf;
    double acc[5] = {0, 0, 0, 0, 0};
    double Li[5], Ui[5];
    for (int c = 0; c < 5; ++c) { Li[c] = L.lap[c * N + i]; Ui[c] = L.u[c * N + i]; }
    const double vdi = L.vdt[i], coni = L.conn[i], si = L.sens[i];
    row_walk<13, STAGE, false, AHEAD>(L, sm, f, i, [&](const Inc<13, STAGE, false> &t) {
        const bool first = t.first();
        const double vdj = t.v[0], conj = t.v[1];
        double d0 = first ? dmin(vdi, vdj) : dmin(vdj, vdi);
        d0 = d0 / (first ? (coni + conj) : (conj + coni));
        const double sj = t.v[2];
        double d2 = d0 * P.k2 * (first ? dmax(si, sj) : dmax(sj, si));
        double d4 = d0 * k4;
        d4 = d4 > d2 ? d4 - d2 : 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const double Lj = t.v[3 + c], Uj = t.v[8 + c];
            if (first) {
                double d4v = Li[c] - Lj, d2v = Ui[c] - Uj;
                acc[c] = (acc[c] - d4v * d4) + d2v * d2;
            } else {
                double d4v = Lj - Li[c], d2v = Uj - Ui[c];
                acc[c] = (acc[c] + d4v * d4) - d2v * d2;
            }
        }
    });
    for (int c = 0; c < 5; ++c) L.diss[c * N + i] = acc[c];
}

// makeViscosityTerm pass 1 (gradients, then the node's stress and heat
// flux as in k_visc_grad): the other node's (u, v, w, T)
template <bool STAGE, bool AHEAD>
__global__ void __launch_bounds__(kTile, 3) k_visc_grad_tiled(Params P, LevelView L) {
    extern __shared__ double sm[];
    const int N = L.N;
    const double *f[4] = {L.prim, L.prim + N, L.prim + 2 * (size_t)N, L.prim + 3 * (size_t)N};
    const int i = tile_begin<4, STAGE>(sm, L, f);
    if (i < 0) return;
    double g[12];
    for (int c = 0; c < 12; ++c) g[c] = 0.0;
    const double qi[4] = {L.prim[i], L.prim[N + i], L.prim[2 * N + i], L.prim[3 * N + i]};
    row_walk<4, STAGE, true, AHEAD>(L, sm, f, i, [&](const Inc<4, STAGE, true> &t) {
        const bool first = t.first();
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                double v = (first ? qi[c] + t.v[c] : t.v[c] + qi[c]) * t.w[a];
                g[a * 4 + c] = g[a * 4 + c] + (first ? v : -v);
            }
    });
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        double v[12];
        visc_grad_bterms(L, k, v);
        for (int c = 0; c < 12; ++c) g[c] = g[c] + v[c];
    }
    visc_grad_finish(P, L, i, g);
}

// makeViscosityTerm pass 2 (as k_visc_flux): the other node's stress, heat
// flux and velocity
template <bool STAGE, bool AHEAD>
__global__ void __launch_bounds__(kTile, AHEAD ? 2 : 3) k_visc_flux_tiled(Params P, LevelView L) {
    extern __shared__ double sm[];
    const int N = L.N;
    const double *f[12] = {L.tau, L.tau + N, L.tau + 2 * (size_t)N, L.tau + 3 * (size_t)N, L.tau + 4 * (size_t)N,
                           L.tau + 5 * (size_t)N, L.tau + 6 * (size_t)N, L.tau + 7 * (size_t)N,
                           L.tau + 8 * (size_t)N, L.prim, L.prim + N, L.prim + 2 * (size_t)N};
    const int i = tile_begin<12, STAGE>(sm, L, f);
    if (i < 0) return;
    double ti[9], ui[3];
    for (int c = 0; c < 9; ++c) ti[c] = L.tau[c * N + i];
    ui[0] = L.prim[i]; ui[1] = L.prim[N + i]; ui[2] = L.prim[2 * N + i];
    double acc[4] = {0, 0, 0, 0};
    row_walk<12, STAGE, true, AHEAD>(L, sm, f, i, [&](const Inc<12, STAGE, true> &t) {
        const bool first = t.first();
        const double *tj = t.v, *uj = t.v + 9;
        double fl[4];
        visc_edge_flux(first ? ti : tj, first ? tj : ti, first ? ui : uj, first ? uj : ui, t.w[0], t.w[1], t.w[2],
                       fl);
        for (int c = 0; c < 4; ++c) acc[c] = acc[c] + (first ? fl[c] : -fl[c]);
    });
    visc_flux_boundary(L, i, acc);
    for (int c = 0; c < 4; ++c) L.diss[(1 + c) * N + i] = L.diss[(1 + c) * N + i] - acc[c];
}

#define FLITE_TILED_INST(STAGE, AHEAD)                                                     \
    template __global__ void k_timestep_tiled<0, STAGE, AHEAD>(Params, LevelView);         \
    template __global__ void k_timestep_tiled<2, STAGE, AHEAD>(Params, LevelView);         \
    template __global__ void k_timestep_tiled<3, STAGE, AHEAD>(Params, LevelView);         \
    template __global__ void k_jst_lap_tiled<STAGE, AHEAD>(Params, LevelView);            \
    template __global__ void k_jst_flux_tiled<STAGE, AHEAD>(Params, LevelView);           \
    template __global__ void k_visc_grad_tiled<STAGE, AHEAD>(Params, LevelView);          \
    template __global__ void k_visc_flux_tiled<STAGE, AHEAD>(Params, LevelView);
FLITE_TILED_INST(true, true)
FLITE_TILED_INST(true, false)
FLITE_TILED_INST(false, true)
FLITE_TILED_INST(false, false)
#undef FLITE_TILED_INST

template __global__ void k_node_update_tiled<true, true>(Params, LevelView, int, int);
template __global__ void k_node_update_tiled<true, false>(Params, LevelView, int, int);
template __global__ void k_node_update_tiled<false, true>(Params, LevelView, int, int);
template __global__ void k_node_update_tiled<false, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 1, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 1, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 4, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 4, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 8, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 8, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 16, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 16, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 32, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_BUFFER, 32, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_LEAN, 1, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_LEAN, 1, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 1, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 1, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 4, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 4, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 8, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 8, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 16, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 16, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 32, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_CENTRAL, 32, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 1, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 1, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 4, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 4, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 8, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 8, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 16, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 16, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 32, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_ANCHOR, 32, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_DELTA, 1, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_DELTA, 1, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_DELTA, 4, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_DELTA, 4, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_DELTA, 8, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_DELTA, 8, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_DELTA, 16, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_DELTA, 16, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_DELTA, 32, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_DELTA, 32, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_node_update<GATHER_CENTRAL2, 1, false>(Params, LevelView, int, int);
template __global__ void k_node_update<GATHER_CENTRAL2, 1, true>(CaseTab<Params>, CaseTab<LevelView>, int, int);
template __global__ void k_timestep<1, false>(Params, LevelView);
template __global__ void k_timestep<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_timestep<4, false>(Params, LevelView);
template __global__ void k_timestep<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_timestep<8, false>(Params, LevelView);
template __global__ void k_timestep<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_timestep<16, false>(Params, LevelView);
template __global__ void k_timestep<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_timestep<32, false>(Params, LevelView);
template __global__ void k_timestep<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_lap<1, false>(Params, LevelView);
template __global__ void k_jst_lap<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_lap<4, false>(Params, LevelView);
template __global__ void k_jst_lap<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_lap<8, false>(Params, LevelView);
template __global__ void k_jst_lap<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_lap<16, false>(Params, LevelView);
template __global__ void k_jst_lap<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_lap<32, false>(Params, LevelView);
template __global__ void k_jst_lap<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_flux<1, false>(Params, LevelView);
template __global__ void k_jst_flux<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_flux<4, false>(Params, LevelView);
template __global__ void k_jst_flux<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_flux<8, false>(Params, LevelView);
template __global__ void k_jst_flux<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_flux<16, false>(Params, LevelView);
template __global__ void k_jst_flux<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jst_flux<32, false>(Params, LevelView);
template __global__ void k_jst_flux<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_grad<1, false>(Params, LevelView);
template __global__ void k_visc_grad<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_grad<4, false>(Params, LevelView);
template __global__ void k_visc_grad<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_grad<8, false>(Params, LevelView);
template __global__ void k_visc_grad<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_grad<16, false>(Params, LevelView);
template __global__ void k_visc_grad<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_grad<32, false>(Params, LevelView);
template __global__ void k_visc_grad<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_grad<1, false>(Params, LevelView);
template __global__ void k_visc2_grad<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_grad<4, false>(Params, LevelView);
template __global__ void k_visc2_grad<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_grad<8, false>(Params, LevelView);
template __global__ void k_visc2_grad<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_grad<16, false>(Params, LevelView);
template __global__ void k_visc2_grad<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_grad<32, false>(Params, LevelView);
template __global__ void k_visc2_grad<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_flux<1, false>(Params, LevelView);
template __global__ void k_visc2_flux<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_flux<4, false>(Params, LevelView);
template __global__ void k_visc2_flux<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_flux<8, false>(Params, LevelView);
template __global__ void k_visc2_flux<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_flux<16, false>(Params, LevelView);
template __global__ void k_visc2_flux<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc2_flux<32, false>(Params, LevelView);
template __global__ void k_visc2_flux<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_flux<1, false>(Params, LevelView);
template __global__ void k_visc_flux<1, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_flux<4, false>(Params, LevelView);
template __global__ void k_visc_flux<4, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_flux<8, false>(Params, LevelView);
template __global__ void k_visc_flux<8, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_flux<16, false>(Params, LevelView);
template __global__ void k_visc_flux<16, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_flux<32, false>(Params, LevelView);
template __global__ void k_visc_flux<32, true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_first_order_diss<1>(Params, LevelView);
template __global__ void k_pressure<false>(Params, LevelView);
template __global__ void k_pressure<true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_visc_prim<false>(Params, LevelView);
template __global__ void k_visc_prim<true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_ts_lap<false>(Params, LevelView);
template __global__ void k_ts_lap<true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_jflux_vgrad<false>(Params, LevelView);
template __global__ void k_jflux_vgrad<true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_bnd_flux<false>(Params, LevelView);
template __global__ void k_bnd_flux<true>(CaseTab<Params>, CaseTab<LevelView>);
template __global__ void k_delta_state<false>(LevelView);
template __global__ void k_delta_state<true>(CaseTab<LevelView>);
template __global__ void k_restrict_u<false>(LevelView, LevelView);
template __global__ void k_restrict_u<true>(CaseTab<LevelView>, CaseTab<LevelView>);
template __global__ void k_restrict_state<false>(Params, LevelView, LevelView);
template __global__ void k_restrict_state<true>(CaseTab<Params>, CaseTab<LevelView>, CaseTab<LevelView>);
template __global__ void k_restrict_incr<false>(Params, LevelView, LevelView);
template __global__ void k_restrict_incr<true>(CaseTab<Params>, CaseTab<LevelView>, CaseTab<LevelView>);
template __global__ void k_prolong_coarse<false>(Params, LevelView, LevelView);
template __global__ void k_prolong_coarse<true>(CaseTab<Params>, CaseTab<LevelView>, CaseTab<LevelView>);
template __global__ void k_prolong_fine<false>(Params, LevelView, LevelView);
template __global__ void k_prolong_fine<true>(CaseTab<Params>, CaseTab<LevelView>, CaseTab<LevelView>);
template __global__ void k_inject_u<false>(LevelView, LevelView);
template __global__ void k_inject_u<true>(CaseTab<LevelView>, CaseTab<LevelView>);

// ---- copy u -> uprev (doTimeIterations def_par:983-987) -------------------
__global__ void k_copy(const double *a, double *b, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// mapFineToCoarse (def_par:12572-12596) as a gather over each coarse node's
// children in increasing fine order: the same additions in the same order as
// the reference's scatter over fine nodes
__device__ __forceinline__ void restrict_gather(const LevelView &C, const double *fine, int nf, int c, int ncomp,
                                                double *out) {
    for (int k = 0; k < ncomp; ++k) out[k] = 0.0;
    for (int q = C.child_ptr[c]; q < C.child_ptr[c + 1]; ++q) {
        int f = C.child[q];
        double w = C.rweight[f];
        for (int k = 0; k < ncomp; ++k) out[k] = out[k] + w * fine[(size_t)k * nf + f];
    }
}

// C.u = R(F.u) (plain mapFineToCoarse of the solution)
template <bool B>
__global__ void k_restrict_u(CaseArg<B, LevelView> C_, CaseArg<B, LevelView> F_) {
    FLITE_CASE_L(B, C);
    FLITE_CASE_L(B, F);
    int c = tid();
    if (c >= C.N) return;
    double v[6];
    restrict_gather(C, F.u, F.N, c, C.nvar, v);
    for (int k = 0; k < C.nvar; ++k) C.u[k * C.N + c] = v[k];
}

// mapFineToCoarse of another array (def_par:12572-12679)
__global__ void k_restrict_arr(LevelView C, LevelView F, const double *fsrc, double *cdst, int ncomp) {
    int c = tid();
    if (c >= C.N) return;
    double v[6];
    restrict_gather(C, fsrc, F.N, c, ncomp, v);
    for (int k = 0; k < ncomp; ++k) cdst[k * C.N + c] = v[k];
}

// the nu~ solution conditions: zero on walls (def_par:4416-4418, 4446-4448,
// 4469-4471), the ramped exhaust value on engine exhausts (:4507-4530), 0.1
// on the far field (def_par:4076-4140); rp is the exhaust ramp
__device__ __forceinline__ double sa_bc_solution(const Params &P, unsigned char cls, double rp, double v) {
    if (cls == BC_WALL || cls == BC_IWALL) return 0.0;
    if (is_exhaust(cls)) return sa_exhaust(P, cls, rp);
    if (cls == BC_FAR3 || cls == BC_FAR4) return 0.1;
    return v;
}
// the nu~ increment conditions (def_par:4978-5125)
__device__ __forceinline__ double sa_bc_increment(const Params &P, unsigned char cls, double r) {
    if (cls == BC_WALL || cls == BC_IWALL || is_exhaust(cls)) return 0.0;
    if (is_inlet(cls)) return P.engRelax * r;
    return r;
}

// restrictGrid head (def_par:12159-12185): C.u = R(F.u), C.mu = R(F.mu),
// pressure, boundary conditions, uprev = u, pressure again
template <bool B>
__global__ void k_restrict_state(CaseArg<B, Params> P_, CaseArg<B, LevelView> C_, CaseArg<B, LevelView> F_) {
    FLITE_CASE_P(B, P, C);
    FLITE_CASE_L(B, C);
    FLITE_CASE_L(B, F);
    int c = tid();
    if (c >= C.N) return;
    const int N = C.N;
    double v[5], m;
    restrict_gather(C, F.u, F.N, c, 5, v);
    restrict_gather(C, F.mu, F.N, c, 1, &m);
    C.mu[c] = m;
    double p0 = pressure(P, v[0], v[1], v[2], v[3], v[4]);
    const unsigned char cls = C.bc[c];
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = C.nx[c]; n1 = C.ny[c]; n2 = C.nz[c]; }
    bc_solution(P, cls, n0, n1, n2, 0.0, 0.0, 0.0, relax_param(P, *C.cyc), v);
    const double rp = eo_relax(P, *C.cyc);
    if (is_exhaust(cls)) bc_exhaust(P, cls, rp, v);
    bc_outer(P, cls, n0, n1, n2, p0, v);
    for (int k = 0; k < 5; ++k) { C.u[k * N + c] = v[k]; C.uprev[k * N + c] = v[k]; }
    if (P.sa) {
        double t;
        restrict_gather(C, F.u + 5 * (size_t)F.N, F.N, c, 1, &t);
        t = sa_bc_solution(P, cls, rp, t);
        C.u[5 * N + c] = t;
        C.uprev[5 * N + c] = t;
    }
    C.p[c] = fabs(pressure(P, v[0], v[1], v[2], v[3], v[4]));
    store_node(C.q, c, v[0], v[1], v[2], v[3], v[4], C.p[c]);
}

// restrictGrid tail (def_par:12385-12427): C.rhs = R(F.rhs), increment
// conditions, src -= rhs, u += rhs
template <bool B>
__global__ void k_restrict_incr(CaseArg<B, Params> P_, CaseArg<B, LevelView> C_, CaseArg<B, LevelView> F_) {
    FLITE_CASE_P(B, P, C);
    FLITE_CASE_L(B, C);
    FLITE_CASE_L(B, F);
    int c = tid();
    if (c >= C.N) return;
    const int N = C.N;
    double r[5];
    restrict_gather(C, F.rhs, F.N, c, 5, r);
    const unsigned char cls = C.bc[c];
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = C.nx[c]; n1 = C.ny[c]; n2 = C.nz[c]; }
    bc_increment(P, cls, n0, n1, n2, r);
    for (int k = 0; k < 5; ++k) {
        C.rhs[k * N + c] = r[k];
        C.src[k * N + c] = C.src[k * N + c] - r[k];
        C.u[k * N + c] = C.u[k * N + c] + r[k];
    }
    if (P.sa) {
        double t;
        restrict_gather(C, F.rhs + 5 * (size_t)F.N, F.N, c, 1, &t);
        t = sa_bc_increment(P, cls, t);
        C.rhs[5 * N + c] = t;
        C.src[5 * N + c] = C.src[5 * N + c] - t;
        C.u[5 * N + c] = C.u[5 * N + c] + t;
    }
}

// prolongateGrid coarse part (def_par:12445-12468): uprev = R(F.u) with the
// solution conditions, rhs = u - uprev with the increment conditions
template <bool B>
__global__ void k_prolong_coarse(CaseArg<B, Params> P_, CaseArg<B, LevelView> C_, CaseArg<B, LevelView> F_) {
    FLITE_CASE_P(B, P, C);
    FLITE_CASE_L(B, C);
    FLITE_CASE_L(B, F);
    int c = tid();
    if (c >= C.N) return;
    const int N = C.N;
    double v[5];
    restrict_gather(C, F.u, F.N, c, 5, v);
    const unsigned char cls = C.bc[c];
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = C.nx[c]; n1 = C.ny[c]; n2 = C.nz[c]; }
    bc_solution(P, cls, n0, n1, n2, 0.0, 0.0, 0.0, relax_param(P, *C.cyc), v);
    const double rp = eo_relax(P, *C.cyc);
    if (is_exhaust(cls)) bc_exhaust(P, cls, rp, v);
    bc_outer(P, cls, n0, n1, n2, C.p[c], v);
    double r[5];
    for (int k = 0; k < 5; ++k) {
        C.uprev[k * N + c] = v[k];
        r[k] = C.u[k * N + c] - v[k];
    }
    double r6 = 0.0;
    if (P.sa) {
        double t;
        restrict_gather(C, F.u + 5 * (size_t)F.N, F.N, c, 1, &t);
        t = sa_bc_solution(P, cls, rp, t);
        C.uprev[5 * N + c] = t;
        r6 = C.u[5 * N + c] - t;
        // nullifyOuterBoundary, then the increment conditions
        if (cls == BC_FAR3 || is_engine(cls)) { r[0] = r[1] = r[2] = r[3] = r[4] = 0.0; r6 = 0.0; }
        r6 = sa_bc_increment(P, cls, r6);
    }
    bc_increment(P, cls, n0, n1, n2, r);
    for (int k = 0; k < 5; ++k) C.rhs[k * N + c] = r[k];
    if (P.sa) C.rhs[5 * N + c] = r6;
}

// prolongateGrid fine part (def_par:12470-12567): injection, relaxation,
// u += correction, boundary conditions, floors
template <bool B>
__global__ void k_prolong_fine(CaseArg<B, Params> P_, CaseArg<B, LevelView> C_, CaseArg<B, LevelView> F_) {
    FLITE_CASE_P(B, P, C);
    FLITE_CASE_L(B, C);
    FLITE_CASE_L(B, F);
    int i = tid();
    if (i >= F.N) return;
    const int N = F.N;
    int pc = C.parent[i];
    const unsigned char cls = F.bc[i];
    // nullifyOuterBoundary of the injected correction (SA runs only)
    const bool nul = P.sa && (cls == BC_FAR3 || is_engine(cls));
    double un[5];
    for (int k = 0; k < 5; ++k) un[k] = F.u[k * N + i];
    for (int k = 0; k < 5; ++k) {
        double r = pc >= 0 ? C.rhs[k * C.N + pc] : F.rhs[k * N + i];
        if (nul) r = 0.0;
        r = P.prolRelax * r;
        if (i < F.Nb) r = P.mgBCRelax * r;
        F.rhs[k * N + i] = r;
        un[k] = un[k] + r;
    }
    double un6 = 0.0;
    if (P.sa) {
        double r = pc >= 0 ? C.rhs[5 * C.N + pc] : F.rhs[5 * N + i];
        if (nul) r = 0.0;
        r = P.turbProlRelax * r;
        F.rhs[5 * N + i] = r;
        un6 = F.u[5 * N + i];
        // the nu~ correction reaches the levels finer than
        // numberOfTurbulenceGrids (def_par:12540-12552)
        if (F.grid < P.nTurbGrids) un6 = un6 + r;
        un6 = sa_bc_solution(P, cls, eo_relax(P, *F.cyc), un6);
        un6 = dmax(un6, 0.0);
        F.u[5 * N + i] = un6;
    }
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = F.nx[i]; n1 = F.ny[i]; n2 = F.nz[i]; }
    double cm0 = 0, cm1 = 0, cm2 = 0;
    if (cls == BC_WALL && P.viscous && F.grid == 1) { cm0 = F.cmx[i]; cm1 = F.cmy[i]; cm2 = F.cmz[i]; }
    bc_solution(P, cls, n0, n1, n2, cm0, cm1, cm2, relax_param(P, *F.cyc), un);
    if (is_exhaust(cls)) {
        const double pex = bc_exhaust(P, cls, eo_relax(P, *F.cyc), un);
        if (F.eng.f) F.eng.pbc[i] = pex;
    }
    if (F.eng.f && (P.eftype == 2 || is_engine(cls))) {  // completed by k_engine_finish
        for (int k = 0; k < 5; ++k) F.u[k * N + i] = un[k];
        return;
    }
    bc_outer(P, cls, n0, n1, n2, F.p[i], un);
    un[0] = dmax(un[0], P.minRho);
    for (int k = 0; k < 5; ++k) F.u[k * N + i] = un[k];
}

// mapCoarseToFine of the solution (injection, def_par:12694-12700)
template <bool B>
__global__ void k_inject_u(CaseArg<B, LevelView> C_, CaseArg<B, LevelView> F_) {
    FLITE_CASE_L(B, C);
    FLITE_CASE_L(B, F);
    int i = tid();
    if (i >= F.N) return;
    int pc = C.parent[i];
    if (pc < 0) return;
    for (int k = 0; k < F.nvar; ++k) F.u[k * F.N + i] = C.u[k * C.N + pc];
}

// setBCsOnSolutionField on a level's solution (start-up, def_par:3994)
__global__ void k_bc_solution(Params P, LevelView L) {
    int i = tid();
    if (i >= L.N) return;
    const unsigned char cls = L.bc[i];
    if (cls == BC_NONE) return;
    const int N = L.N;
    double un[5];
    for (int k = 0; k < 5; ++k) un[k] = L.u[k * N + i];
    double cm0 = 0, cm1 = 0, cm2 = 0;
    if (cls == BC_WALL && P.viscous) { cm0 = L.cmx[i]; cm1 = L.cmy[i]; cm2 = L.cmz[i]; }
    bc_solution(P, cls, L.nx[i], L.ny[i], L.nz[i], cm0, cm1, cm2, relax_param(P, *L.cyc), un);
    if (is_exhaust(cls)) {
        const double rp = eo_relax(P, *L.cyc);
        const double pex = bc_exhaust(P, cls, rp, un);
        if (L.eng.f) L.eng.pbc[i] = pex;
        if (P.sa) L.u[5 * N + i] = sa_exhaust(P, cls, rp);
    }
    for (int k = 0; k < 5; ++k) L.u[k * N + i] = un[k];
    if (P.sa && (cls == BC_WALL || cls == BC_IWALL)) L.u[5 * N + i] = 0.0;
}

__global__ void k_set_int(int *dst, const int *src) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *src;
}

// ivd%physicalTimeStep = the smallest local time step of the level
// (makeTimeSteps under explicit time stepping, def_par:13598-13607): the
// minimum of positive doubles as the minimum of their bit patterns, which
// integer atomics take in any order to the same value.  k_min_dt_init
// starts it at the reference's 9999999.9.
__global__ void k_min_dt_init(LevelView L) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *L.ptsg = 9999999.9;
}
__global__ void k_min_dt(LevelView L) {
    __shared__ unsigned long long m[256];
    unsigned long long v = __double_as_longlong(9999999.9);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.N; i += gridDim.x * blockDim.x) {
        const double d = L.dt[i];
        if (d < __longlong_as_double((long long)v)) v = (unsigned long long)__double_as_longlong(d);
    }
    m[threadIdx.x] = v;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w && m[threadIdx.x + w] < m[threadIdx.x]) m[threadIdx.x] = m[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicMin(reinterpret_cast<unsigned long long *>(L.ptsg), m[0]);
}

// The same steps of the multigrid cycle on a level's view, so that a case
// group runs them for every case in one launch: the level's cycle number
// (doTimeIterations), uprev = u over n = nvar N values, and the zeroed
// dissipation (which 0) or FAS source (which 1) over n values.
template <bool B>
__global__ void k_case_cycle(CaseArg<B, LevelView> L_, const int *src) {
    FLITE_CASE_L(B, L);
    if (threadIdx.x == 0 && blockIdx.x == 0) *L.cyc = *src;
}
template <bool B>
__global__ void k_case_save_u(CaseArg<B, LevelView> L_, size_t n) {
    FLITE_CASE_L(B, L);
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) L.uprev[i] = L.u[i];
}
template <bool B>
__global__ void k_case_zero(CaseArg<B, LevelView> L_, int which, size_t n) {
    FLITE_CASE_L(B, L);
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) (which ? L.src : L.diss)[i] = 0.0;
}
template __global__ void k_case_cycle<false>(LevelView, const int *);
template __global__ void k_case_cycle<true>(CaseTab<LevelView>, const int *);
template __global__ void k_case_save_u<false>(LevelView, size_t);
template __global__ void k_case_save_u<true>(CaseTab<LevelView>, size_t);
template __global__ void k_case_zero<false>(LevelView, int, size_t);
template __global__ void k_case_zero<true>(CaseTab<LevelView>, int, size_t);

// ---- residual norms (writeResiduals mg_par:1299-1443) ---------------------
// per block: sum (u-uprev)^2 and max |u-uprev| with its first index
__global__ void k_resid_partial(LevelView L, double *part, int nblk) {
    __shared__ double ss[6][256];
    __shared__ double sm[6][256];
    __shared__ int si[6][256];
    const int N = L.N, nv = L.nvar;
    double s[6] = {0, 0, 0, 0, 0, 0}, m[6] = {0, 0, 0, 0, 0, 0};
    int mi[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, 0x7fffffff, 0x7fffffff, 0x7fffffff};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        // the first node in the caller's numbering wins a tie (mg_par:1387-1396)
        const int oi = L.perm ? L.perm[i] : i;
        for (int k = 0; k < nv; ++k) {
            double d = L.u[k * N + i] - L.uprev[k * N + i];
            s[k] = s[k] + d * d;
            double a = fabs(d);
            if (a > m[k] || (a == m[k] && a > 0.0 && oi < mi[k])) { m[k] = a; mi[k] = oi; }
        }
    }
    for (int k = 0; k < 6; ++k) { ss[k][threadIdx.x] = s[k]; sm[k][threadIdx.x] = m[k]; si[k][threadIdx.x] = mi[k]; }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            for (int k = 0; k < 6; ++k) {
                ss[k][threadIdx.x] += ss[k][threadIdx.x + w];
                double a = sm[k][threadIdx.x], b = sm[k][threadIdx.x + w];
                int ia = si[k][threadIdx.x], ib = si[k][threadIdx.x + w];
                if (b > a || (b == a && ib < ia)) { sm[k][threadIdx.x] = b; si[k][threadIdx.x] = ib; }
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 6; ++k) {
            part[blockIdx.x * 18 + k] = ss[k][0];
            part[blockIdx.x * 18 + 6 + k] = sm[k][0];
            part[blockIdx.x * 18 + 12 + k] = (double)si[k][0];
        }
    }
}

// one warp per component (blockDim.x = 192); each lane folds the block
// partials b = lane, lane+32, ... and the warp combines the lanes in a fixed
// tree, so the result does not depend on timing
__global__ void k_resid_final(const double *part, int nblk, double *out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= 6) return;
    double s = 0, m = 0;
    int mi = 0x7fffffff;
    for (int b = lane; b < nblk; b += 32) {
        s += part[b * 18 + k];
        double v = part[b * 18 + 6 + k];
        int iv = (int)part[b * 18 + 12 + k];
        if (v > m || (v == m && iv < mi)) { m = v; mi = iv; }
    }
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        double v = __shfl_down_sync(0xffffffffu, m, off);
        int iv = __shfl_down_sync(0xffffffffu, mi, off);
        if (v > m || (v == m && iv < mi)) { m = v; mi = iv; }
    }
    if (lane == 0) {
        out[k] = sqrt(s);
        out[6 + k] = m;
        out[12 + k] = (double)(mi == 0x7fffffff ? 0 : mi);
    }
}

// ---- forces (calculateLiftAndDrag def_par:14710-14805): block partials ---
// part[6*block + k]; k_forces_final sums the partials in block order
__global__ void k_forces(Params P, LevelView L, const int *wall, int nwall, double alphaR, double betaR,
                         double ground, double d0, double d1, double d2, double *part) {
    __shared__ double red[6][256];
    double ft[3] = {cos(alphaR) * cos(betaR), sin(betaR), sin(alphaR)};
    double fn1[3] = {-ft[2], 0.0, ft[0]}, fn2[3] = {-ft[1], ft[0], 0.0};
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const double pinf = 1. / (P.gamma * P.mach * P.mach);
    const int N = L.N;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nwall; q += gridDim.x * blockDim.x) {
        int ip = wall[q];
        double h = L.cz[ip];
        if (!(h > (ground + 0.01))) continue;
        double xd = L.cx[ip] - d0, yd = L.cy[ip] - d1, zd = L.cz[ip] - d2;
        double n[3] = {L.nx[ip], L.ny[ip], L.nz[ip]};
        double A = L.wallArea[ip], dp = L.p[ip] - pinf;
        double dn1 = (n[0] * fn1[0] + n[1] * fn1[1]) + n[2] * fn1[2];
        double dn2 = (n[0] * fn2[0] + n[1] * fn2[1]) + n[2] * fn2[2];
        double dt = (n[0] * ft[0] + n[1] * ft[1]) + n[2] * ft[2];
        acc[0] -= A * dp * dn1;
        acc[1] -= A * dp * dt;
        acc[2] -= A * dp * dn2;
        acc[4] += xd * A * dp * dn2 - yd * A * dp * dt;
        acc[5] += xd * A * dp * dn1 - zd * A * dp * dt;
        if (P.viscous) {
            double s0 = L.wstress[ip], s1 = L.wstress[N + ip], s2 = L.wstress[2 * N + ip];
            double sn1 = (s0 * fn1[0] + s1 * fn1[1]) + s2 * fn1[2];
            double sn2 = (s0 * fn2[0] + s1 * fn2[1]) + s2 * fn2[2];
            double st = (s0 * ft[0] + s1 * ft[1]) + s2 * ft[2];
            acc[0] += A * sn1;
            acc[2] += A * sn2;
            acc[1] += A * st;
            acc[3] += A * st;
            acc[4] += -xd * A * sn2 + yd * A * st;
            acc[5] += -xd * A * sn1 + zd * A * st;
        }
    }
    for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 6; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) part[6 * blockIdx.x + k] = red[k][0];
}

__global__ void k_permute_nodes(double *dst, const double *src, const int *map, int N, int ncomp) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)N * ncomp) return;
    const int c = (int)(t / N), i = (int)(t - (size_t)c * N);
    dst[t] = src[(size_t)c * N + map[i]];
}

// ---- forces of forceCalcType 3 (calculateLiftAndDrag3 def_par:15129-15313)
// Per wall node (indicator register -20..-19) the face loads of its wall and
// inviscid-wall faces (codes 1, 9) with a node above the ground plane, in
// boundary-edge order as the reference's scatter adds them: 4 w_b (p - p_inf)
// and, in viscous runs on code-1 faces, 4 tau_w |w_b|.  Then the seven sums
// part[7*block + k] = (lift, drag, latF, latM, longMl, longMd, rollM).
__global__ void k_forces3(Params P, LevelView L, const int *wall, int nwall, double alphaR, double betaR,
                          double ground, double d0, double d1, double d2, double *part) {
    __shared__ double red[7][256];
    double ft[3] = {cos(alphaR) * cos(betaR), sin(betaR), sin(alphaR)};
    double fn1[3] = {-ft[2], 0.0, ft[0]}, fn2[3] = {-ft[1], ft[0], 0.0};
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const double pinf = 1. / (P.gamma * P.mach * P.mach);
    const int N = L.N;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nwall; q += gridDim.x * blockDim.x) {
        const int ip = wall[q];
        double h0 = 0.0, h1 = 0.0, h2 = 0.0;
        for (int k = L.binc_ptr[ip]; k < L.binc_ptr[ip + 1]; ++k) {
            const int b = L.binc[k] >> 1;
            const int code = L.bind[b];
            if (!(code == 1 || code == 9)) continue;
            const int2 nd = L.bedge[b];
            if (!((L.cz[nd.x] > (ground + 0.01)) || (L.cz[nd.y] > (ground + 0.01)))) continue;
            const double pp = L.p[ip] - pinf;
            const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
            h0 = h0 + 4.0 * wx * pp;
            h1 = h1 + 4.0 * wy * pp;
            h2 = h2 + 4.0 * wz * pp;
            if (P.viscous && code == 1) {
                const double area = sqrt((wx * wx + wy * wy) + wz * wz);
                h0 = h0 + 4.0 * L.wstress[ip] * area;
                h1 = h1 + 4.0 * L.wstress[N + ip] * area;
                h2 = h2 + 4.0 * L.wstress[2 * N + ip] * area;
            }
        }
        const double xd = L.cx[ip] - d0, yd = L.cy[ip] - d1, zd = L.cz[ip] - d2;
        const double hn1 = (h0 * fn1[0] + h1 * fn1[1]) + h2 * fn1[2];
        const double hn2 = (h0 * fn2[0] + h1 * fn2[1]) + h2 * fn2[2];
        const double ht = (h0 * ft[0] + h1 * ft[1]) + h2 * ft[2];
        acc[0] += hn1;
        acc[1] += ht;
        acc[2] += hn2;
        acc[3] += -xd * hn2 + yd * ht;
        acc[4] += -xd * hn1;
        acc[5] += zd * ht;
        acc[6] += -yd * hn1 + zd * hn2;
    }
    for (int k = 0; k < 7; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 7; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 7; ++k) part[7 * blockIdx.x + k] = red[k][0];
}

// out[k] = sum over blocks of part[nval*block + k], in block order
__global__ void k_forces_final(const double *part, int nblk, int nval, double *out) {
    if (threadIdx.x >= nval) return;
    const int k = threadIdx.x;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[nval * b + k];
    out[k] = s;
}
}  // namespace flite

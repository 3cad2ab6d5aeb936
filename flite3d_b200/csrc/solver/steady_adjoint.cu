// Steady discrete adjoint of the level-1 smoother: dCL/dCD with respect to the
// level-1 geometry (edge coefficients side_w, boundary coefficients bnd_w,
// volumes) through the converged solution.
//
// One smoother iteration G (doTimeIterations with calcDiss, def_par:966-1181,
// for the central flux, scalar JST dissipation and an inviscid run) maps the
// level-1 state u to the next one; a converged solution is a fixed point
// u* = G(u*; g) of it (the multigrid corrections vanish there).  For an
// objective J(u; g),
//   dJ/dg = J_g + lam^T G_g   with   lam = P (G_u^T lam + J_u^T),
// the fixed-point form of the adjoint equation, iterated like the primal
// smoother and so converging at its rate.  P removes the energy of the
// subsonic inflow nodes: setOuterBoundaryConditions (def_par:4056-4146) sets
// their density and momentum and rebuilds their energy from the pressure of
// the previous stage, which leaves that energy where the initial state put it
// (an eigenvalue 1 of G_u); the solution, and every finite difference of it,
// keeps it fixed, so the adjoint treats it as a constant.
//
// G_u^T lam is the reverse sweep of the iteration:
//   stages 3, 2, 1 (k_adj_stage): outer, solution and increment boundary
//     conditions, density clip and floors, the update u - CFL a_k dt (Q+D)/V;
//     then the transpose of the residual Jacobian Q at the stage's input state
//     (k_vjp_farfield, k_vjp_node), whose output is the next stage's adjoint;
//   the JST dissipation (k_adj_jst_edges, k_adj_jst_lap): the sensor and
//     undivided Laplacian of def_par:11484-11993 in reverse;
//   the local time step (k_adj_timestep) of def_par:13335-13610 and the
//     pressure of the iteration's start.
// The state of every stage is recorded once per linearisation point by the
// primal kernels themselves.  Each kernel is a node gather over the
// incidence lists (or a node-local pass), so the sums are deterministic.
// The geometry sweep adds the coefficient, normal and wall-area parts and
// runs once, after the adjoint has converged.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "adjoint.cuh"
#include "context.h"

namespace flite {

namespace {

__device__ __forceinline__ int tidx() { return blockIdx.x * blockDim.x + threadIdx.x; }
// |w.m| below kKink |w||m| counts as zero (on the kink of |vn|)
constexpr double kKink = 1.0e-12;
__device__ __forceinline__ double sgn0(double x) { return x < 0 ? -1.0 : 1.0; }  // d|x|/dx, +1 at 0

// x <- x - scale (x.n) n on the momentum of x (components 1..3): reverse.
// xb holds the adjoint of the projected vector on entry and of the input on
// exit; nb (may be null) accumulates the normal's adjoint; x is the input.
__device__ __forceinline__ void remove_normal_rev(const double *x, double n0, double n1, double n2,
                                                  double scale, double *xb, double *nb) {
    const double n[3] = {n0, n1, n2};
    const double xm[3] = {x[1], x[2], x[3]};
    const double bm[3] = {xb[1], xb[2], xb[3]};
    const double xn = (xm[0] * n[0] + xm[1] * n[1]) + xm[2] * n[2];
    const double bn = (bm[0] * n[0] + bm[1] * n[1]) + bm[2] * n[2];
    for (int c = 0; c < 3; ++c) xb[1 + c] = bm[c] - scale * bn * n[c];
    if (nb)
        for (int c = 0; c < 3; ++c) nb[c] -= scale * (bn * xm[c] + xn * bm[c]);
}

// far-field Roe flux (def_par:2258-2419) with the state and the normal as
// dual numbers
__device__ void farfield_dn(const Params &P, const Dual *q, Dual pr, const Dual *n, const double *inf, Dual *F) {
    const double gam1 = P.gm1;
    double ro = inf[0], ro1 = 1. / ro, uo = inf[1], vo = inf[2], wo = inf[3], eo = inf[4], po = inf[5];
    Dual rhol = q[0], rinvl = Dual(1.0) / rhol;
    Dual rhl = q[4] + pr;
    Dual ul = q[1] * rinvl, vl = q[2] * rinvl, wl = q[3] * rinvl;
    Dual epsl = q[4], hl = rhl * rinvl;
    Dual nvl = (ul * n[0] + vl * n[1]) + wl * n[2];
    Dual fl1 = rhol * nvl, fl2 = pr * n[0] + rhol * ul * nvl, fl3 = pr * n[1] + rhol * vl * nvl;
    Dual fl4 = pr * n[2] + rhol * wl * nvl, fl5 = rhl * nvl;
    double rhor = ro, uxr = uo, vyr = vo, wzr = wo, epsr = eo * ro, presr = po, hr = eo + po * ro1;
    Dual unr = (Dual(uxr) * n[0] + Dual(vyr) * n[1]) + Dual(wzr) * n[2];
    Dual fr1 = Dual(rhor) * unr, fr2 = n[0] * presr + Dual(rhor * uxr) * unr;
    Dual fr3 = n[1] * presr + Dual(rhor * vyr) * unr, fr4 = n[2] * presr + Dual(rhor * wzr) * unr;
    Dual fr5 = Dual(epsr + presr) * unr;
    Dual di = dsqrt(Dual(rhor) / rhol), d1 = Dual(1.0) / (di + Dual(1.0));
    Dual ui = (di * uxr + ul) * d1, vi = (di * vyr + vl) * d1, wi = (di * wzr + wl) * d1;
    Dual hi = (di * hr + hl) * d1;
    Dual ci2 = Dual(gam1) * (hi - Dual(0.5) * ((ui * ui + vi * vi) + wi * wi));
    ci2 = dmaxc(ci2, 1.0e-5);
    Dual ci = dsqrt(ci2);
    Dual af = Dual(0.5) * ((ui * ui + vi * vi) + wi * wi);
    Dual ucp = (ui * n[0] + vi * n[1]) + wi * n[2];
    Dual du1 = Dual(rhor) - rhol, du2 = Dual(rhor * uxr) - rhol * ul, du3 = Dual(rhor * vyr) - rhol * vl;
    Dual du4 = Dual(rhor * wzr) - rhol * wl, du5 = Dual(epsr) - epsl;
    Dual l1 = dfabs(ucp + ci), l2 = dfabs(ucp - ci), l3 = dfabs(ucp);
    Dual s1 = Dual(0.5) * (l1 + l2), s2 = Dual(0.5) * (l1 - l2);
    Dual al1x = Dual(gam1) * ((((af * du1 - ui * du2) - vi * du3) - wi * du4) + du5);
    Dual al2x = ((-ucp * du1 + du2 * n[0]) + du3 * n[1]) + du4 * n[2];
    Dual cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci);
    Dual cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
    F[0] = Dual(0.5) * (fr1 + fl1) - Dual(0.5) * (l3 * du1 + cc1);
    F[1] = Dual(0.5) * (fr2 + fl2) - Dual(0.5) * ((l3 * du2 + cc1 * ui) + cc2 * n[0]);
    F[2] = Dual(0.5) * (fr3 + fl3) - Dual(0.5) * ((l3 * du3 + cc1 * vi) + cc2 * n[1]);
    F[3] = Dual(0.5) * (fr4 + fl4) - Dual(0.5) * ((l3 * du4 + cc1 * wi) + cc2 * n[2]);
    F[4] = Dual(0.5) * (fr5 + fl5) - Dual(0.5) * ((l3 * du5 + cc1 * hi) + cc2 * ucp);
}

// the one-sided flux F(u) in the three directions: A[d][c] = F_c(u; e_d)
__device__ __forceinline__ void flux_dirs(const Params &P, const double *u, double A[3][5]) {
    double p, dp[5];
    pressure_grad(P, u, &p, dp);
    const double r = u[0], E = u[4];
    const double m[3] = {u[1], u[2], u[3]};
    for (int d = 0; d < 3; ++d) {
        const double vd = m[d] / r;
        A[d][0] = m[d];
        for (int c = 0; c < 3; ++c) A[d][1 + c] = m[c] * vd + (c == d ? p : 0.0);
        A[d][4] = (E + p) * vd;
    }
}

}  // namespace

// ---- forward record ------------------------------------------------------
// nh6 = sum -+(p_i - p_j) and nh7 = sum (p_i + p_j) of the pressure sensor
// (def_par:11570-11620) at the iteration's start
__global__ void k_adj_sensor_parts(LevelView L, const double *p, double *nh6, double *nh7) {
    const int i = tidx();
    if (i >= L.N) return;
    double s6 = 0.0, s7 = 0.0;
    const double pi = p[i];
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const double pj = p[t.y];
        if (t.x >= 0) s6 -= pi - pj;
        else s6 += pj - pi;
        s7 += pi + pj;
    }
    nh6[i] = s6;
    nh7[i] = s7;
}

// ---- reverse of one RK stage, node part (def_par:1069-1178) --------------
// vbar: adjoint of the stage's output; u0 = uprev; x = the stage's input
// state; Q its residual (makeRHS); D, dt the iteration's dissipation and time
// step.  Adds the uprev part to ubar, stores Qbar (the adjoint of Q) and the
// adjoint of the stage's pressure (outer boundary condition), and adds to the
// adjoints of D, dt and (geometry sweep) V and the node normals.
__global__ void k_adj_stage(Params P, LevelView L, int stage, const double *vbar, const double *u0, const double *x,
                            const double *Q, const double *D, const double *dt, double *ubar, double *Qbar,
                            double *Dbar, double *dtbar, double *pbar, double *Vbar, double *nbar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double up[5], xs[5], t[5];
    for (int c = 0; c < 5; ++c) {
        up[c] = u0[(size_t)c * N + i];
        xs[c] = x[(size_t)c * N + i];
        t[c] = Q[(size_t)c * N + i] + D[(size_t)c * N + i];
    }
    const double dti = dt[i], Vi = L.V[i];
    double s[5], sp[5], d[5], z[5], z2[5];
    for (int c = 0; c < 5; ++c) s[c] = dti * t[c] / Vi;
    const unsigned char cls = L.bc[i];
    double n0 = 0, n1 = 0, n2 = 0;
    if (cls != BC_NONE) { n0 = L.nx[i]; n1 = L.ny[i]; n2 = L.nz[i]; }
    const bool inc_proj = cls == BC_WALL || cls == BC_IWALL || cls == BC_SYM;  // inviscid
    for (int c = 0; c < 5; ++c) sp[c] = s[c];
    if (inc_proj) remove_normal(sp, n0, n1, n2, 1.0);
    const double dtJ = P.CFL * P.RK[stage - 1];
    for (int c = 0; c < 5; ++c) d[c] = dtJ * sp[c];
    const bool clip = !(fabs(d[0] / up[0]) < P.maxInc);
    clipped_update(P, up, d, z);
    const bool lim1 = z[0] < P.minRho;
    if (lim1) z[0] = P.minRho;
    const double relax = relax_param(P, *L.cyc);
    for (int c = 0; c < 5; ++c) z2[c] = z[c];
    double m2[3] = {0, 0, 0};
    if (cls == BC_WALL || cls == BC_SYM) remove_normal(z2, n0, n1, n2, 1.0);
    if (cls == BC_IWALL) {
        remove_normal(z2, n0, n1, n2, relax);
        m2[0] = z2[1]; m2[1] = z2[2]; m2[2] = z2[3];
    }
    const bool lim2 = z2[0] < P.minRho;  // limitDensity
    double z3[5];
    for (int c = 0; c < 5; ++c) z3[c] = z2[c];
    if (lim2) z3[0] = P.minRho;

    // reverse
    double vb[5], zb[5], pb = 0.0;
    for (int c = 0; c < 5; ++c) vb[c] = vbar[(size_t)c * N + i];
    for (int c = 0; c < 5; ++c) zb[c] = vb[c];
    if (cls == BC_FAR3 || cls == BC_FAR4) {  // setOuterBoundaryConditions
        const double *inf = &P.inf[cls == BC_FAR3 ? 0 : 6];
        const double nvel = (inf[1] * n0 + inf[2] * n1) + inf[3] * n2;
        if (nvel > 0.00) {
            for (int c = 0; c < 5; ++c) zb[c] = 0.0;
            if (!(P.mach > 1.0)) pb = vb[4] / P.gm1;
        } else if (P.mach < 1.0) {
            const double r = z3[0], q = (z3[1] * z3[1] + z3[2] * z3[2]) + z3[3] * z3[3];
            zb[4] = 0.0;
            for (int c = 0; c < 3; ++c) zb[1 + c] += vb[4] * z3[1 + c] / r;
            zb[0] += -vb[4] * 0.5 * q / (r * r);
        }
    }
    if (lim2) zb[0] = 0.0;
    double nb[3] = {0, 0, 0};
    if (cls == BC_WALL || cls == BC_SYM) remove_normal_rev(z, n0, n1, n2, 1.0, zb, nb);
    if (cls == BC_IWALL) {
        if (!P.isentropic) {  // E = rho Tinf / gamma + ke / (2 rho) of the projected momentum
            const double r = z2[0], ke = (m2[0] * m2[0] + m2[1] * m2[1]) + m2[2] * m2[2];
            for (int c = 0; c < 3; ++c) zb[1 + c] += zb[4] * m2[c] / r;
            zb[0] += zb[4] * (P.Tinf / P.gamma - 0.5 * ke / (r * r));
            zb[4] = 0.0;
        }
        remove_normal_rev(z, n0, n1, n2, relax, zb, nb);
    }
    if (lim1) zb[0] = 0.0;
    double ub[5], db[5];
    if (!clip) {
        ub[0] = zb[0];
        db[0] = -zb[0];
    } else {
        const double sign = d[0] / fabs(d[0]);
        ub[0] = zb[0] * (1.0 - sign * P.maxInc);
        db[0] = 0.0;
    }
    for (int c = 1; c < 5; ++c) { ub[c] = zb[c]; db[c] = -zb[c]; }
    double sb[5];
    for (int c = 0; c < 5; ++c) sb[c] = dtJ * db[c];
    if (inc_proj) remove_normal_rev(s, n0, n1, n2, 1.0, sb, nb);
    double dtb = 0.0, vbv = 0.0;
    for (int c = 0; c < 5; ++c) {
        const double tb = sb[c] * dti / Vi;
        Qbar[(size_t)c * N + i] = tb;
        Dbar[(size_t)c * N + i] += tb;
        ubar[(size_t)c * N + i] += ub[c];
        dtb += sb[c] * t[c] / Vi;
        vbv -= sb[c] * dti * t[c] / (Vi * Vi);
    }
    dtbar[i] += dtb;
    pbar[i] = pb;
    if (Vbar) Vbar[i] += vbv;
    if (nbar)
        for (int c = 0; c < 3; ++c) nbar[(size_t)c * N + i] += nb[c];
}

// ---- JST dissipation (def_par:11484-11993), reverse ----------------------
// Edge part (pass 3) gathered per node: the adjoints of this node's undivided
// Laplacian (scaled back to nodeHelpArray 1:5), of its sensor terms nh6/nh7
// and of its V/dt; the direct u part goes to ubar.
__global__ void k_adj_jst_edges(Params P, LevelView L, const double *u0, const double *dt, const double *lap,
                                const double *sens, const double *nh6, const double *nh7, const double *Dbar,
                                double *ubar, double *dtbar, double *nhbar, double *nh6bar, double *nh7bar,
                                double *Vbar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    const double k2 = P.k2, k4 = L.grid == 1 ? P.k4 : P.cgdf;
    double lapb[5] = {0, 0, 0, 0, 0}, ubd[5] = {0, 0, 0, 0, 0}, sensb = 0.0, rb = 0.0;
    const double Vi = L.V[i], dti = dt[i], ri = Vi / dti, ci = L.conn[i], si = sens[i];
    double ui[5], li[5], Dbi[5];
    for (int c = 0; c < 5; ++c) {
        ui[c] = u0[(size_t)c * N + i];
        li[c] = lap[(size_t)c * N + i];
        Dbi[c] = Dbar[(size_t)c * N + i];
    }
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int j = t.y;
        const bool first = t.x >= 0;  // this node is the edge's i1
        const double rj = L.V[j] / dt[j], cj = L.conn[j], sj = sens[j];
        // edge quantities in (i1, i2) order
        const double r1 = first ? ri : rj, r2 = first ? rj : ri;
        const double s1 = first ? si : sj, s2 = first ? sj : si;
        const double cs = first ? ci + cj : cj + ci;
        const double d0 = dmin(r1, r2) / cs;
        const double smax = dmax(s1, s2);
        const double d2 = d0 * k2 * smax;
        const double d4a = d0 * k4;
        const bool act = d4a > d2;
        const double d4 = act ? d4a - d2 : 0.0;
        double db[5], d4v[5], d2v[5];
        for (int c = 0; c < 5; ++c) {
            const double dbj = Dbar[(size_t)c * N + j];
            const double lj = lap[(size_t)c * N + j], uj = u0[(size_t)c * N + j];
            db[c] = first ? Dbi[c] - dbj : dbj - Dbi[c];
            d4v[c] = first ? li[c] - lj : lj - li[c];
            d2v[c] = first ? ui[c] - uj : uj - ui[c];
        }
        const double sig = first ? 1.0 : -1.0;
        double d4b = 0.0, d2b = 0.0;
        for (int c = 0; c < 5; ++c) {
            lapb[c] += -sig * d4 * db[c];
            ubd[c] += sig * d2 * db[c];
            d4b -= d4v[c] * db[c];
            d2b += d2v[c] * db[c];
        }
        double d0b = 0.0;
        if (act) {
            d0b += k4 * d4b;
            d2b -= d4b;
        }
        d0b += k2 * smax * d2b;
        // max(s1, s2) = (s1 < s2) ? s2 : s1; min(r1, r2) = (r2 < r1) ? r2 : r1
        const bool max_is_2 = s1 < s2, min_is_2 = r2 < r1;
        if (max_is_2 != first) sensb += d0 * k2 * d2b;
        if (min_is_2 != first) rb += d0b / cs;
    }
    const double fact = 1. / ci;
    for (int c = 0; c < 5; ++c) {
        nhbar[(size_t)c * N + i] = fact * lapb[c];
        ubar[(size_t)c * N + i] += ubd[c];
    }
    // sens = 12 |nh6 / nh7|
    const double q = nh6[i] / nh7[i];
    const double qb = 12. * sgn0(q) * sensb;
    nh6bar[i] = qb / nh7[i];
    nh7bar[i] = -qb * q / nh7[i];
    // r = V / dt
    dtbar[i] += -rb * Vi / (dti * dti);
    if (Vbar) Vbar[i] += rb / dti;
}

// passes 1 and 2 in reverse: the undivided Laplacian and the sensor sums
// gathered back to the state and the pressure of the iteration's start
__global__ void k_adj_jst_lap(LevelView L, const double *nhbar, const double *nh6bar, const double *nh7bar,
                              double *ubar, double *p0bar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double nbi[5];
    for (int c = 0; c < 5; ++c) nbi[c] = nhbar[(size_t)c * N + i];
    const double b6i = nh6bar[i], b7i = nh7bar[i];
    double ub[5] = {0, 0, 0, 0, 0}, pb = 0.0;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int j = L.inc[k].y;
        for (int c = 0; c < 5; ++c) ub[c] += nhbar[(size_t)c * N + j] - nbi[c];
        pb += nhbar[(size_t)4 * N + j] - nbi[4];
        pb += nh6bar[j] - b6i;
        pb += nh7bar[j] + b7i;
    }
    for (int c = 0; c < 5; ++c) ubar[(size_t)c * N + i] += ub[c];
    p0bar[i] += pb;
}

// ---- local time step (def_par:13335-13610), inviscid, reverse -------------
// f(u, p; w) = |w.m/rho| + sqrt(max(gamma p/rho, 0.001) |w|^2): one edge end's
// term; df/du, df/dp and (geometry) df/dw
__device__ __forceinline__ void ts_term_grad(const Params &P, const double *u, double p, const double *w,
                                             double *fu, double *fp, double *fw) {
    const double r = u[0], ro = 1. / r;
    const double al = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
    const double wm = (w[0] * u[1] + w[1] * u[2]) + w[2] * u[3];
    const double vn = wm * ro;
    // |vn| at a slip wall or symmetry plane sits on its kink (the momentum is
    // projected onto the plane, vn is rounding noise): there the derivative
    // is the mean of the one-sided ones, 0, which is what a symmetric
    // displacement of the geometry sees
    const double mm = sqrt((u[1] * u[1] + u[2] * u[2]) + u[3] * u[3]);
    const double sg = fabs(wm) <= kKink * sqrt(al) * mm ? 0.0 : sgn0(vn);
    const double cc0 = P.gamma * p * ro;
    const bool floor = cc0 < 0.001;
    const double cc = floor ? 0.001 : cc0;
    const double g = sqrt(cc * al);
    const double gcc = g > 0 ? 0.5 * al / g : 0.0;  // dg/dcc
    fu[0] = -sg * vn * ro + (floor ? 0.0 : gcc * (-P.gamma * p * ro * ro));
    for (int c = 0; c < 3; ++c) fu[1 + c] = sg * w[c] * ro;
    fu[4] = 0.0;
    *fp = floor ? 0.0 : gcc * P.gamma * ro;
    if (fw) {
        const double gal = g > 0 ? 0.5 * cc / g : 0.0;  // dg/dal
        for (int c = 0; c < 3; ++c) fw[c] = sg * u[1 + c] * ro + gal * 2.0 * w[c];
    }
}

// Sbar = dJ/dS of dt = 0.5 / (S/V): the interior edges add f of this node's
// own state, each boundary edge 2 f(own) + f(other); then the pressure of the
// iteration's start goes back to the state
__global__ void k_adj_timestep(Params P, LevelView L, const double *u0, const double *p0, const double *dt,
                               const double *dtbar, const double *p0bar, double *ubar, double *Sbar, double *Vbar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    const double Vi = L.V[i], dti = dt[i];
    const double tt = 0.5 / dti;  // S/V
    const double tb = -0.5 * dtbar[i] / (tt * tt);
    const double sbi = tb / Vi;
    Sbar[i] = sbi;
    if (Vbar) Vbar[i] += -tb * tt / Vi;
    double ui[5];
    for (int c = 0; c < 5; ++c) ui[c] = u0[(size_t)c * N + i];
    const double pi = p0[i];
    double ub[5] = {0, 0, 0, 0, 0}, pb = 0.0;
    double fu[5], fp;
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int e = L.inc[k].x >= 0 ? L.inc[k].x : ~L.inc[k].x;
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        ts_term_grad(P, ui, pi, w, fu, &fp, nullptr);
        for (int c = 0; c < 5; ++c) ub[c] += sbi * fu[c];
        pb += sbi * fp;
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const int j = side == 0 ? nd.y : nd.x;
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        // Sbar of the other node is read after this kernel's writes are not
        // needed: it is recomputed from its own dtbar
        const double ttj = 0.5 / dt[j];
        const double sbj = (-0.5 * dtbar[j] / (ttj * ttj)) / L.V[j];
        const double wgt = 2.0 * sbi + sbj;
        ts_term_grad(P, ui, pi, w, fu, &fp, nullptr);
        for (int c = 0; c < 5; ++c) ub[c] += wgt * fu[c];
        pb += wgt * fp;
    }
    pb += p0bar[i];
    double p, dp[5];
    pressure_grad(P, ui, &p, dp);
    for (int c = 0; c < 5; ++c) ubar[(size_t)c * N + i] += ub[c] + pb * dp[c];
}

// geometry sweep: the coefficient adjoints of the time step, per edge
__global__ void k_adj_timestep_w(Params P, LevelView L, const double *u0, const double *p0, const double *Sbar,
                                 double *swbar) {
    const int e = tidx();
    if (e >= L.E) return;
    const int N = L.N, E = L.E;
    const int2 nd = L.edge[e];
    const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
    double acc[3] = {0, 0, 0};
    for (int side = 0; side < 2; ++side) {
        const int n = side == 0 ? nd.x : nd.y;
        double u[5], fu[5], fp, fw[3];
        for (int c = 0; c < 5; ++c) u[c] = u0[(size_t)c * N + n];
        ts_term_grad(P, u, p0[n], w, fu, &fp, fw);
        for (int c = 0; c < 3; ++c) acc[c] += Sbar[n] * fw[c];
    }
    for (int c = 0; c < 3; ++c) swbar[(size_t)c * E + e] += acc[c];
}

__global__ void k_adj_timestep_bw(Params P, LevelView L, const double *u0, const double *p0, const double *Sbar,
                                  double *bwbar) {
    const int b = tidx();
    if (b >= L.B) return;
    const int N = L.N, B = L.B;
    const int2 nd = L.bedge[b];
    const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
    double acc[3] = {0, 0, 0};
    for (int side = 0; side < 2; ++side) {
        const int n = side == 0 ? nd.x : nd.y, o = side == 0 ? nd.y : nd.x;
        double u[5], fu[5], fp, fw[3];
        for (int c = 0; c < 5; ++c) u[c] = u0[(size_t)c * N + n];
        ts_term_grad(P, u, p0[n], w, fu, &fp, fw);
        const double wgt = 2.0 * Sbar[n] + Sbar[o];
        for (int c = 0; c < 3; ++c) acc[c] += wgt * fw[c];
    }
    for (int c = 0; c < 3; ++c) bwbar[(size_t)c * B + b] += acc[c];
}

// geometry sweep: coefficient adjoints of the stage residual Q at the state x
// (central flux per edge; wall and far-field fluxes per boundary edge)
__global__ void k_adj_flux_w(Params P, LevelView L, const double *x, const double *Qbar, double *swbar) {
    const int e = tidx();
    if (e >= L.E) return;
    const int N = L.N, E = L.E;
    const int2 nd = L.edge[e];
    double u1[5], u2[5], A1[3][5], A2[3][5], a[5];
    for (int c = 0; c < 5; ++c) {
        u1[c] = x[(size_t)c * N + nd.x];
        u2[c] = x[(size_t)c * N + nd.y];
        a[c] = Qbar[(size_t)c * N + nd.x] - Qbar[(size_t)c * N + nd.y];
    }
    flux_dirs(P, u1, A1);
    flux_dirs(P, u2, A2);
    for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int c = 0; c < 5; ++c) s += a[c] * (A1[d][c] + A2[d][c]);
        swbar[(size_t)d * E + e] += s;
    }
}

__global__ void k_adj_flux_bw(Params P, LevelView L, const double *x, const double *Qbar, double *bwbar) {
    const int b = tidx();
    if (b >= L.B) return;
    const int N = L.N, B = L.B;
    const int ind = L.bind[b];
    const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
    const double rnorm = sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]);
    if (!(rnorm > 1.0e-10)) return;
    const int2 nd = L.bedge[b];
    const bool fe = P.boundaryTerm == 1;
    double u1[5], u2[5], r1[5], r2[5];
    for (int c = 0; c < 5; ++c) {
        u1[c] = x[(size_t)c * N + nd.x];
        u2[c] = x[(size_t)c * N + nd.y];
        r1[c] = Qbar[(size_t)c * N + nd.x];
        r2[c] = Qbar[(size_t)c * N + nd.y];
    }
    double acc[3] = {0, 0, 0};
    if (ind <= 2 || ind == 9) {
        // g1 = 3 F(u1; w) + F(u2; w), g2 = F(u1; w) + 3 F(u2; w): linear in w
        double A1[3][5], A2[3][5];
        flux_dirs(P, u1, A1);
        flux_dirs(P, u2, A2);
        for (int d = 0; d < 3; ++d)
            for (int c = 0; c < 5; ++c) {
                const double g1 = fe ? 3. * A1[d][c] + A2[d][c] : 4. * A1[d][c];
                const double g2 = fe ? A1[d][c] + 3. * A2[d][c] : 4. * A2[d][c];
                acc[d] += r1[c] * g1 + r2[c] * g2;
            }
    } else if (ind == 3 || ind == 4) {
        const double *inf = &P.inf[(ind - 3) * 6];
        double p1, p2, dp[5];
        pressure_grad(P, u1, &p1, dp);
        pressure_grad(P, u2, &p2, dp);
        for (int d = 0; d < 3; ++d) {
            Dual wd[3] = {Dual(w[0], d == 0 ? 1.0 : 0.0), Dual(w[1], d == 1 ? 1.0 : 0.0),
                          Dual(w[2], d == 2 ? 1.0 : 0.0)};
            Dual rn = dsqrt((wd[0] * wd[0] + wd[1] * wd[1]) + wd[2] * wd[2]);
            Dual n[3] = {wd[0] / rn, wd[1] / rn, wd[2] / rn};
            Dual q1[5], q2[5], F1[5], F2[5];
            for (int c = 0; c < 5; ++c) { q1[c] = Dual(u1[c]); q2[c] = Dual(u2[c]); }
            farfield_dn(P, q1, Dual(p1), n, inf, F1);
            farfield_dn(P, q2, Dual(p2), n, inf, F2);
            for (int c = 0; c < 5; ++c) {
                Dual g1 = fe ? rn * (Dual(3.) * F1[c] + F2[c]) : rn * Dual(4.) * F1[c];
                Dual g2 = fe ? rn * (F1[c] + Dual(3.) * F2[c]) : rn * Dual(4.) * F2[c];
                acc[d] += r1[c] * g1.d + r2[c] * g2.d;
            }
        }
    }
    for (int d = 0; d < 3; ++d) bwbar[(size_t)d * B + b] += acc[d];
}

// ---- objective -----------------------------------------------------------
// J = 2/A_ref sum over wall nodes (above the ground plane) of
// -A_i (p_i - p_inf) (n_i . e) (calculateLiftAndDrag def_par:14710-14870,
// inviscid part, pressure of the state): J, dJ/du, dJ/dA and dJ/dn.  One
// thread walks the wall list in order (a node listed twice counts twice).
__global__ void k_adj_objective(Params P, LevelView L, const int *wall, int nwall, double ground, double e0,
                                double e1, double e2, double aref, const double *u, double *J, double *Ju,
                                double *Abar, double *nbar) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int N = L.N;
    const double pinf = 1. / (P.gamma * P.mach * P.mach);
    const double f = 2.0 / aref;
    double acc = 0.0;
    for (int q = 0; q < nwall; ++q) {
        const int ip = wall[q];
        if (!(L.cz[ip] > (ground + 0.01))) continue;
        double x[5], p, dp[5];
        for (int c = 0; c < 5; ++c) x[c] = u[(size_t)c * N + ip];
        pressure_grad(P, x, &p, dp);
        const double n[3] = {L.nx[ip], L.ny[ip], L.nz[ip]};
        const double dn = (n[0] * e0 + n[1] * e1) + n[2] * e2;
        const double A = L.wallArea[ip], dpi = p - pinf;
        acc -= A * dpi * dn;
        for (int c = 0; c < 5; ++c) Ju[(size_t)c * N + ip] += -f * A * dn * dp[c];
        Abar[ip] += -f * dpi * dn;
        nbar[ip] += -f * A * dpi * e0;
        nbar[(size_t)N + ip] += -f * A * dpi * e1;
        nbar[2 * (size_t)N + ip] += -f * A * dpi * e2;
    }
    *J = f * acc;
}

// the same with a thread per wall-list entry, for a list without repeated
// nodes: the terms of J summed per block, the blocks in order by
// k_gm_dots_final
constexpr int kObjBlocks = 64;
__global__ void k_adj_objective_par(Params P, LevelView L, const int *wall, int nwall, double ground, double e0,
                                    double e1, double e2, double aref, const double *u, double *part, double *Ju,
                                    double *Abar, double *nbar) {
    __shared__ double red[256];
    const int N = L.N;
    const double pinf = 1. / (P.gamma * P.mach * P.mach);
    const double f = 2.0 / aref;
    double acc = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nwall; q += gridDim.x * blockDim.x) {
        const int ip = wall[q];
        if (!(L.cz[ip] > (ground + 0.01))) continue;
        double x[5], p, dp[5];
        for (int c = 0; c < 5; ++c) x[c] = u[(size_t)c * N + ip];
        pressure_grad(P, x, &p, dp);
        const double n[3] = {L.nx[ip], L.ny[ip], L.nz[ip]};
        const double dn = (n[0] * e0 + n[1] * e1) + n[2] * e2;
        const double A = L.wallArea[ip], dpi = p - pinf;
        acc -= A * dpi * dn;
        for (int c = 0; c < 5; ++c) Ju[(size_t)c * N + ip] += -f * A * dn * dp[c];
        Abar[ip] += -f * dpi * dn;
        nbar[ip] += -f * A * dpi * e0;
        nbar[(size_t)N + ip] += -f * A * dpi * e1;
        nbar[2 * (size_t)N + ip] += -f * A * dpi * e2;
    }
    red[threadIdx.x] = f * acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ---- node normals and wall areas from the boundary coefficients ------------
// n_i = a_i/|a_i|, a_i = -sum over the node's boundary edges of w_b
// (makeBoundaryNormals def_par:15394-15521): abar_i = (nbar - (nbar.n) n)/|a|
__global__ void k_adj_normals(LevelView L, const double *nbar, double *abar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double a[3] = {0, 0, 0};
    if (i < L.Nb)
        for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
            const int b = L.binc[k] >> 1;
            a[0] -= L.bwx[b]; a[1] -= L.bwy[b]; a[2] -= L.bwz[b];
        }
    const double nrm = sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]);
    double o[3] = {0, 0, 0};
    if (i < L.Nb && nrm > 1.0e-10) {
        const double n[3] = {a[0] / nrm, a[1] / nrm, a[2] / nrm};
        const double b[3] = {nbar[i], nbar[(size_t)N + i], nbar[2 * (size_t)N + i]};
        const double bn = (b[0] * n[0] + b[1] * n[1]) + b[2] * n[2];
        for (int c = 0; c < 3; ++c) o[c] = (b[c] - bn * n[c]) / nrm;
    }
    for (int c = 0; c < 3; ++c) abar[(size_t)c * N + i] = o[c];
}

// per boundary edge: -(abar_1 + abar_2) of the normals and 4 (Abar_1 + Abar_2)
// w/|w| of the wall areas A_i = sum 4|w_b| (makeSurfaceArea def_par:15523)
__global__ void k_adj_bedge_geom(LevelView L, const double *abar, const double *Abar, double *bwbar) {
    const int b = tidx();
    if (b >= L.B) return;
    const int N = L.N, B = L.B;
    const int2 nd = L.bedge[b];
    const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
    const double ai = sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]);
    const double Ab = Abar[nd.x] + Abar[nd.y];
    for (int c = 0; c < 3; ++c) {
        double v = -(abar[(size_t)c * N + nd.x] + abar[(size_t)c * N + nd.y]);
        if (ai > 0) v += 4.0 * Ab * w[c] / ai;
        bwbar[(size_t)c * B + b] += v;
    }
}

// ---- iteration: lam_new = P (ubar + Ju), with the norms of the change ------
constexpr int kAdjBlocks = 128;
__global__ void k_adj_update(Params P, LevelView L, const double *ubar, const double *Ju, double *lam,
                             double *part) {
    __shared__ double red[2][256];
    const int N = L.N;
    double dd = 0.0, ll = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        bool fixE = false;
        const unsigned char cls = L.bc[i];
        if ((cls == BC_FAR3 || cls == BC_FAR4) && !(P.mach > 1.0)) {
            const double *inf = &P.inf[cls == BC_FAR3 ? 0 : 6];
            fixE = ((inf[1] * L.nx[i] + inf[2] * L.ny[i]) + inf[3] * L.nz[i]) > 0.00;
        }
        for (int c = 0; c < 5; ++c) {
            const size_t k = (size_t)c * N + i;
            double v = ubar[k] + Ju[k];
            if (c == 4 && fixE) v = 0.0;
            const double d = v - lam[k];
            dd += d * d;
            ll += v * v;
            lam[k] = v;
        }
    }
    red[0][threadIdx.x] = dd;
    red[1][threadIdx.x] = ll;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[0][threadIdx.x] += red[0][threadIdx.x + w];
            red[1][threadIdx.x] += red[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = red[0][0];
        part[2 * blockIdx.x + 1] = red[1][0];
    }
}

__global__ void k_adj_norms(const double *part, int nblk, double *out) {
    if (threadIdx.x >= 2) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[2 * b + threadIdx.x];
    out[threadIdx.x] = s;
}

__global__ void k_adj_zero(double *a, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a[i] = 0.0;
}

// ---- host side ----------------------------------------------------------
// ---- GMRES on (I - A) lam = b, A = P G_u^T, b = P Ju ------------------------
// Restarted GMRES (Saad and Schultz 1986) with classical Gram-Schmidt applied
// twice; the Krylov vectors stay on the device, the Hessenberg matrix and
// its Givens rotations on the host.  Every reduction sums block partials in
// block order, so a solve is deterministic.
constexpr int kDotBlocks = 148;
__global__ void k_gm_dots(const double *V, size_t n, const double *w, double *part) {
    __shared__ double red[256];
    const double *v = V + (size_t)blockIdx.y * n;
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += v[i] * w[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = red[0];
}
__global__ void k_gm_dots_final(const double *part, int nblk, int k, double *h) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)j * nblk + b];
    h[j] = s;
}
// w += sgn sum_j c[j] V_j
__global__ void k_gm_combine(const double *V, size_t n, int k, const double *c, double sgn, double *w) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s += c[j] * V[(size_t)j * n + i];
        w[i] = w[i] + sgn * s;
    }
}
__global__ void k_gm_scale(double *w, size_t n, double a) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        w[i] = a * w[i];
}
__device__ __forceinline__ bool inflow_energy_fixed(const Params &P, const LevelView &L, int i) {
    const unsigned char cls = L.bc[i];
    if (!((cls == BC_FAR3 || cls == BC_FAR4) && !(P.mach > 1.0))) return false;
    const double *inf = &P.inf[cls == BC_FAR3 ? 0 : 6];
    return ((inf[1] * L.nx[i] + inf[2] * L.ny[i]) + inf[3] * L.nz[i]) > 0.00;
}
// mode 0: w = v - P ubar; mode 1: w = b - (v - P ubar); mode 2: w = P v
__global__ void k_gm_apply(Params P, LevelView L, const double *v, const double *ubar, const double *b, double *w,
                           int mode) {
    const int N = L.N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const bool fixE = inflow_energy_fixed(P, L, i);
        for (int c = 0; c < 5; ++c) {
            const size_t k = (size_t)c * N + i;
            double pu = mode == 2 ? v[k] : ubar[k];
            if (c == 4 && fixE) pu = 0.0;
            w[k] = mode == 2 ? pu : (mode == 0 ? v[k] - pu : b[k] - (v[k] - pu));
        }
    }
}

struct SteadyAdjoint {
    int N = 0, E = 0, B = 0;
    double *u0, *v1, *v2, *Q[3], *p0, *dt, *D, *lap, *sens, *nh6, *nh7;
    double *lam, *vb[2], *ubar, *Qbar, *Dbar, *dtbar, *pbar, *p0bar, *nhbar, *nh6bar, *nh7bar, *Sbar, *bvjp;
    double *Vbar, *nbar, *swbar, *bwbar, *Abar, *abar, *Ju, *part, *out;
    // GMRES: Krylov vectors [(m+1)][5N], right-hand side, dot partials
    double *kry = nullptr, *rhs = nullptr, *gpart = nullptr, *gh = nullptr;
    int kry_m = 0;
    bool recorded = false;
};

void destroy_steady_adjoint(SteadyAdjoint *a) { delete a; }

static const char *steady_adjoint_unsupported(const flite_ctx &X) {
    const flite_controls &c = X.c;
    if (c.fluxType != 1) return "the steady adjoint takes the central flux (fluxType 1)";
    if (c.precision != FLITE_FP64) return "the steady adjoint runs in FP64";
    if (c.ReynoldsNumber > 0) return "the steady adjoint covers inviscid runs (ReynoldsNumber 0)";
    if (c.dissipationScheme == 3) return "the steady adjoint takes the scalar JST dissipation (scheme 2)";
    if (c.useDissipationWeighting) return "the steady adjoint takes unweighted dissipation";
    return nullptr;
}

static SteadyAdjoint &buffers(flite_ctx &X) {
    LevelView &L = X.V(0);
    if (!X.sadj) {
        auto *a = new SteadyAdjoint();
        X.sadj = a;
        a->N = L.N; a->E = L.E; a->B = L.B;
        const size_t n5 = 5 * (size_t)L.N, N = L.N;
        for (double **p : {&a->u0, &a->v1, &a->v2, &a->Q[0], &a->Q[1], &a->Q[2], &a->D, &a->lap, &a->lam,
                           &a->vb[0], &a->vb[1], &a->ubar, &a->Qbar, &a->Dbar, &a->nhbar, &a->Ju})
            *p = X.alloc<double>(n5);
        for (double **p : {&a->p0, &a->dt, &a->sens, &a->nh6, &a->nh7, &a->dtbar, &a->pbar, &a->p0bar, &a->nh6bar,
                           &a->nh7bar, &a->Sbar, &a->Vbar, &a->Abar})
            *p = X.alloc<double>(N);
        a->nbar = X.alloc<double>(3 * N);
        a->abar = X.alloc<double>(3 * N);
        a->swbar = X.alloc<double>(3 * (size_t)L.E);
        a->bwbar = X.alloc<double>(3 * (size_t)std::max(L.B, 1));
        a->bvjp = X.alloc<double>(10 * (size_t)std::max(L.B, 1));
        a->part = X.alloc<double>(2 * kAdjBlocks);
        a->out = X.alloc<double>(4);
    }
    return *X.sadj;
}

static void zero(flite_ctx &X, double *p, size_t n);

// J into out[0], and its adjoints dJ/du (Ju), dJ/dA (Abar), dJ/dn (nbar),
// which the caller has zeroed
static void objective_terms(flite_ctx &X, SteadyAdjoint &A, int objective, const double *u) {
    LevelView &L = X.V(0);
    DevLevel &D = X.lv[0];
    const double PI = 4.0 * std::atan(1.0);
    const double aR = X.c.alpha * PI / 180., bR = X.c.beta * PI / 180.;
    const double ft[3] = {std::cos(aR) * std::cos(bR), std::sin(bR), std::sin(aR)};
    const double fn1[3] = {-ft[2], 0.0, ft[0]};
    const double *dir = objective == FLITE_OBJ_CL ? fn1 : ft;
    const int nw = (int)D.wall.size();
    if (nw == 0) {
        zero(X, A.out, 1);
        return;
    }
    std::vector<int> w(D.wall);
    std::sort(w.begin(), w.end());
    if (std::adjacent_find(w.begin(), w.end()) == w.end()) {
        k_adj_objective_par<<<kObjBlocks, 256, 0, X.s>>>(X.P, L, D.d_wall, nw, X.c.groundplane, dir[0], dir[1],
                                                         dir[2], X.c.referenceArea, u, A.part, A.Ju, A.Abar, A.nbar);
        k_gm_dots_final<<<1, 32, 0, X.s>>>(A.part, kObjBlocks, 1, A.out);
    } else {
        k_adj_objective<<<1, 1, 0, X.s>>>(X.P, L, D.d_wall, nw, X.c.groundplane, dir[0], dir[1], dir[2],
                                          X.c.referenceArea, u, A.out, A.Ju, A.Abar, A.nbar);
    }
}

static void zero(flite_ctx &X, double *p, size_t n) {
    k_adj_zero<<<std::min<size_t>((n + 255) / 256, 4096), 256, 0, X.s>>>(p, n);
}
static void copy(flite_ctx &X, const double *a, double *b, size_t n) {
    CK(cudaMemcpyAsync(b, a, n * sizeof(double), cudaMemcpyDeviceToDevice, X.s));
}

// the primal iteration from A.u0, recording the stage states, their
// residuals and the iteration's time step and dissipation
static void record(flite_ctx &X, SteadyAdjoint &A) {
    LevelView &L = X.V(0);
    const size_t n5 = 5 * (size_t)L.N, N = L.N;
    copy(X, A.u0, L.u, n5);
    copy(X, A.u0, L.uprev, n5);
    X.pressure(0);
    X.timesteps(0);
    X.dissipation(0);
    copy(X, L.p, A.p0, N);
    copy(X, L.dt, A.dt, N);
    copy(X, L.diss, A.D, n5);
    copy(X, L.lap, A.lap, n5);
    copy(X, L.sens, A.sens, N);
    k_adj_sensor_parts<<<X.nblk(N), X.nb, 0, X.s>>>(L, A.p0, A.nh6, A.nh7);
    double *in[3] = {A.u0, A.v1, A.v2};
    for (int st = 1; st <= 3; ++st) {
        if (st > 1) copy(X, L.u, in[st - 1], n5);
        X.pressure(0);
        X.rhs_terms(0, false);
        X.launch_node_update(0, MODE_RESID, 0, true);
        copy(X, L.rhs, A.Q[st - 1], n5);
        X.launch_node_update(0, MODE_STAGE, st, st == 1);
    }
    A.recorded = true;
}

// ubar = G_u^T lam (geometry sweep: and the geometry adjoints)
static void reverse(flite_ctx &X, SteadyAdjoint &A, const double *lam, bool geom) {
    LevelView &L = X.V(0);
    const size_t n5 = 5 * (size_t)L.N, N = L.N;
    const unsigned nbk = X.nblk(N);
    zero(X, A.ubar, n5);
    zero(X, A.Dbar, n5);
    zero(X, A.dtbar, N);
    zero(X, A.p0bar, N);
    double *Vb = geom ? A.Vbar : nullptr, *nb = geom ? A.nbar : nullptr;
    const double *in[3] = {A.u0, A.v1, A.v2};
    const double *vin = lam;
    for (int k = 3; k >= 1; --k) {
        const double *x = in[k - 1];
        k_adj_stage<<<nbk, X.nb, 0, X.s>>>(X.P, L, k, vin, A.u0, x, A.Q[k - 1], A.D, A.dt, A.ubar, A.Qbar, A.Dbar,
                                           A.dtbar, A.pbar, Vb, nb);
        if (L.B > 0) k_vjp_farfield<<<X.eblk(L.B), X.eb, 0, X.s>>>(X.P, L, x, A.Qbar, A.bvjp);
        double *vout = A.vb[k & 1];
        if (k > 1) k_vjp_node<<<nbk, X.nb, 0, X.s>>>(X.P, L, x, A.Qbar, A.bvjp, A.pbar, vout, 0);
        else k_vjp_node<<<nbk, X.nb, 0, X.s>>>(X.P, L, x, A.Qbar, A.bvjp, A.pbar, A.ubar, 1);
        if (geom) {
            k_adj_flux_w<<<X.eblk(L.E), X.eb, 0, X.s>>>(X.P, L, x, A.Qbar, A.swbar);
            if (L.B > 0) k_adj_flux_bw<<<X.eblk(L.B), X.eb, 0, X.s>>>(X.P, L, x, A.Qbar, A.bwbar);
        }
        vin = vout;
    }
    const bool jst = !(X.c.fourthOrderDissipationFactor == 0 && X.c.secondOrderDissipationFactor == 0);
    if (jst) {
        k_adj_jst_edges<<<nbk, X.nb, 0, X.s>>>(X.P, L, A.u0, A.dt, A.lap, A.sens, A.nh6, A.nh7, A.Dbar, A.ubar,
                                               A.dtbar, A.nhbar, A.nh6bar, A.nh7bar, Vb);
        k_adj_jst_lap<<<nbk, X.nb, 0, X.s>>>(L, A.nhbar, A.nh6bar, A.nh7bar, A.ubar, A.p0bar);
    }
    k_adj_timestep<<<nbk, X.nb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.dt, A.dtbar, A.p0bar, A.ubar, A.Sbar, Vb);
    if (geom) {
        k_adj_timestep_w<<<X.eblk(L.E), X.eb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.Sbar, A.swbar);
        if (L.B > 0) k_adj_timestep_bw<<<X.eblk(L.B), X.eb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.Sbar, A.bwbar);
    }
}

// geometry adjoints: zeroed, swept, the normals and wall areas chained to bnd_w
static void geometry_sweep(flite_ctx &X, SteadyAdjoint &A, const double *lam) {
    LevelView &L = X.V(0);
    const size_t N = L.N;
    zero(X, A.swbar, 3 * (size_t)L.E);
    zero(X, A.bwbar, 3 * (size_t)std::max(L.B, 1));
    reverse(X, A, lam, true);
    k_adj_normals<<<X.nblk(N), X.nb, 0, X.s>>>(L, A.nbar, A.abar);
    if (L.B > 0) k_adj_bedge_geom<<<X.eblk(L.B), X.eb, 0, X.s>>>(L, A.abar, A.Abar, A.bwbar);
}

static void download_geometry(flite_ctx &X, SteadyAdjoint &A, double *swb, double *bwb, double *vb) {
    LevelView &L = X.V(0);
    if (swb) CK(cudaMemcpyAsync(swb, A.swbar, 3 * (size_t)L.E * sizeof(double), cudaMemcpyDeviceToHost, X.s));
    if (bwb && L.B > 0)
        CK(cudaMemcpyAsync(bwb, A.bwbar, 3 * (size_t)L.B * sizeof(double), cudaMemcpyDeviceToHost, X.s));
    if (vb) CK(cudaMemcpyAsync(vb, A.Vbar, (size_t)L.N * sizeof(double), cudaMemcpyDeviceToHost, X.s));
}

// lam <- P (G_u^T lam + Ju) from lam = P Ju, `check` iterations per launch of
// one captured graph, until |dlam| <= tol |P Ju|
static int fixed_point_solve(flite_ctx &X, SteadyAdjoint &A, double ref, double tol, int max_iter, int *its,
                             double *res_out) {
    LevelView &L = X.V(0);
    const int check = 10;
    auto iterate = [&]() {
        reverse(X, A, A.lam, false);
        k_adj_update<<<kAdjBlocks, 256, 0, X.s>>>(X.P, L, A.ubar, A.Ju, A.lam, A.part);
    };
    cudaGraphExec_t gexec = nullptr;
    if (max_iter >= check) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(X.s, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < check; ++k) iterate();
        k_adj_norms<<<1, 32, 0, X.s>>>(A.part, kAdjBlocks, A.out + 2);
        CK(cudaStreamEndCapture(X.s, &g));
        cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }
    struct GraphGuard {
        cudaGraphExec_t &g;
        ~GraphGuard() { if (g) cudaGraphExecDestroy(g); }
    } guard{gexec};
    int it = 0;
    double res = 1.0, h[2];
    while (it < max_iter && res > tol) {
        if (gexec && it + check <= max_iter) {
            CK(cudaGraphLaunch(gexec, X.s));
            it += check;
        } else {
            for (int k = 0; k < check && it < max_iter; ++k, ++it) iterate();
            k_adj_norms<<<1, 32, 0, X.s>>>(A.part, kAdjBlocks, A.out + 2);
        }
        CK(cudaMemcpyAsync(h, A.out + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
        if (!std::isfinite(h[0])) return FLITE_ENAN;
        res = std::sqrt(h[0]) / ref;
    }
    *its = it;
    *res_out = res;
    return FLITE_OK;
}

// GMRES(m) for (I - P G_u^T) lam = P Ju from lam = P Ju; `its` counts
// products with G_u^T (one per Arnoldi step plus one per restart)
static int gmres_solve(flite_ctx &X, SteadyAdjoint &A, double bnorm, double tol, int max_iter, int m, int *its,
                       double *res_out) {
    LevelView &L = X.V(0);
    const size_t n = 5 * (size_t)L.N;
    if (A.kry_m < m) {
        // the vectors of a smaller restart length stay allocated until the context goes
        A.kry = X.alloc<double>((size_t)(m + 1) * n);
        A.gpart = X.alloc<double>((size_t)kDotBlocks * (m + 1));
        A.gh = X.alloc<double>(m + 1);
        if (!A.rhs) A.rhs = X.alloc<double>(n);
        A.kry_m = m;
    }
    const unsigned eb = 592;
    k_gm_apply<<<eb, 256, 0, X.s>>>(X.P, L, A.Ju, nullptr, nullptr, A.rhs, 2);  // b = P Ju
    auto Vj = [&](int j) { return A.kry + (size_t)j * n; };
    // h[0..k) = V[0..k)^T w, copied to the host
    auto dots = [&](int k, const double *w, double *h) {
        k_gm_dots<<<dim3(kDotBlocks, k), 256, 0, X.s>>>(A.kry, n, w, A.gpart);
        k_gm_dots_final<<<(k + 127) / 128, 128, 0, X.s>>>(A.gpart, kDotBlocks, k, A.gh);
        CK(cudaMemcpyAsync(h, A.gh, k * sizeof(double), cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
    };
    auto norm = [&](const double *w) {
        k_gm_dots<<<dim3(kDotBlocks, 1), 256, 0, X.s>>>(w, n, w, A.gpart);
        k_gm_dots_final<<<1, 32, 0, X.s>>>(A.gpart, kDotBlocks, 1, A.gh);
        double h;
        CK(cudaMemcpyAsync(&h, A.gh, sizeof(double), cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
        return std::sqrt(h);
    };
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), hv(m + 1), y(m);
    auto Hij = [&](int i, int j) -> double & { return H[(size_t)j * (m + 1) + i]; };
    int total = 0;
    double res = 1.0;
    while (true) {
        // r = b - (I - A) lam in V_0
        reverse(X, A, A.lam, false);
        k_gm_apply<<<eb, 256, 0, X.s>>>(X.P, L, A.lam, A.ubar, A.rhs, Vj(0), 1);
        ++total;
        const double beta = norm(Vj(0));
        if (!std::isfinite(beta)) return FLITE_ENAN;
        res = beta / bnorm;
        if (res <= tol || total >= max_iter) break;
        k_gm_scale<<<eb, 256, 0, X.s>>>(Vj(0), n, 1.0 / beta);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        for (; k < m && total < max_iter; ++k) {
            double *w = Vj(k + 1);
            reverse(X, A, Vj(k), false);
            k_gm_apply<<<eb, 256, 0, X.s>>>(X.P, L, Vj(k), A.ubar, nullptr, w, 0);
            ++total;
            for (int i = 0; i <= k; ++i) Hij(i, k) = 0.0;
            for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
                dots(k + 1, w, hv.data());  // also left in A.gh
                k_gm_combine<<<eb, 256, 0, X.s>>>(A.kry, n, k + 1, A.gh, -1.0, w);
                for (int i = 0; i <= k; ++i) Hij(i, k) += hv[i];
            }
            const double hn = norm(w);
            if (!std::isfinite(hn)) return FLITE_ENAN;
            Hij(k + 1, k) = hn;
            if (hn > 0) k_gm_scale<<<eb, 256, 0, X.s>>>(w, n, 1.0 / hn);
            for (int i = 0; i < k; ++i) {  // earlier rotations
                const double a = Hij(i, k), b = Hij(i + 1, k);
                Hij(i, k) = cs[i] * a + sn[i] * b;
                Hij(i + 1, k) = -sn[i] * a + cs[i] * b;
            }
            const double a = Hij(k, k), b = Hij(k + 1, k);
            const double r = std::hypot(a, b);
            cs[k] = r > 0 ? a / r : 1.0;
            sn[k] = r > 0 ? b / r : 0.0;
            Hij(k, k) = r;
            Hij(k + 1, k) = 0.0;
            g[k + 1] = -sn[k] * g[k];
            g[k] = cs[k] * g[k];
            if (std::fabs(g[k + 1]) / bnorm <= tol || hn == 0) {
                ++k;
                break;
            }
        }
        // lam += V y with H y = g (upper triangular, k columns)
        for (int i = k - 1; i >= 0; --i) {
            double s = g[i];
            for (int j = i + 1; j < k; ++j) s -= Hij(i, j) * y[j];
            y[i] = s / Hij(i, i);
        }
        CK(cudaMemcpyAsync(A.gh, y.data(), k * sizeof(double), cudaMemcpyHostToDevice, X.s));
        k_gm_combine<<<eb, 256, 0, X.s>>>(A.kry, n, k, A.gh, 1.0, A.lam);
    }
    *its = total;
    *res_out = res;
    return FLITE_OK;
}

}  // namespace flite

using namespace flite;

extern "C" int flite_iteration_vjp(flite_ctx *ctx, const double *u, const double *lam, double *ubar,
                                   double *side_w_bar, double *bnd_w_bar, double *volume_bar) {
    if (!ctx || !u || !lam || !ubar) return FLITE_EINVAL;
    if (const char *why = steady_adjoint_unsupported(*ctx)) {
        ctx->err = why;
        return FLITE_EUNSUPPORTED;
    }
    try {
        flite_ctx &X = *ctx;
        SteadyAdjoint &A = buffers(X);
        LevelView &L = X.V(0);
        const size_t n5 = 5 * (size_t)L.N, N = L.N;
        // the primal state of level 1 is kept: the record overwrites u, uprev,
        // p, dt, the dissipation and rhs
        std::vector<double> keep(n5);
        CK(cudaMemcpyAsync(keep.data(), L.u, n5 * sizeof(double), cudaMemcpyDeviceToHost, X.s));
        CK(cudaMemcpyAsync(A.u0, u, n5 * sizeof(double), cudaMemcpyHostToDevice, X.s));
        CK(cudaMemcpyAsync(A.lam, lam, n5 * sizeof(double), cudaMemcpyHostToDevice, X.s));
        record(X, A);
        zero(X, A.Vbar, N);
        zero(X, A.nbar, 3 * N);
        zero(X, A.Abar, N);
        const bool geom = side_w_bar || bnd_w_bar || volume_bar;
        if (geom) geometry_sweep(X, A, A.lam);
        else reverse(X, A, A.lam, false);
        CK(cudaMemcpyAsync(ubar, A.ubar, n5 * sizeof(double), cudaMemcpyDeviceToHost, X.s));
        if (geom) download_geometry(X, A, side_w_bar, bnd_w_bar, volume_bar);
        CK(cudaStreamSynchronize(X.s));
        CK(cudaMemcpy(L.u, keep.data(), n5 * sizeof(double), cudaMemcpyHostToDevice));
        X.drop_graph();
        return FLITE_OK;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return FLITE_ECUDA;
    }
}

extern "C" int flite_adjoint_solve(flite_ctx *ctx, int objective, double tol, int max_iter, double *J,
                                   double *side_w_bar, double *bnd_w_bar, double *volume_bar, int *iterations,
                                   double *residual) {
    if (!ctx || objective < FLITE_OBJ_CL || objective > FLITE_OBJ_CD || !(tol > 0) || max_iter < 1 || !J)
        return FLITE_EINVAL;
    if (const char *why = steady_adjoint_unsupported(*ctx)) {
        ctx->err = why;
        return FLITE_EUNSUPPORTED;
    }
    try {
        flite_ctx &X = *ctx;
        SteadyAdjoint &A = buffers(X);
        LevelView &L = X.V(0);
        const size_t n5 = 5 * (size_t)L.N, N = L.N;
        // linearisation point: the context's level-1 state
        copy(X, L.u, A.u0, n5);
        zero(X, A.Ju, n5);
        zero(X, A.Abar, N);
        zero(X, A.Vbar, N);
        zero(X, A.nbar, 3 * N);
        objective_terms(X, A, objective, A.u0);
        record(X, A);
        // lam_0 = P Ju
        zero(X, A.lam, n5);
        zero(X, A.ubar, n5);
        k_adj_update<<<kAdjBlocks, 256, 0, X.s>>>(X.P, L, A.ubar, A.Ju, A.lam, A.part);
        k_adj_norms<<<1, 32, 0, X.s>>>(A.part, kAdjBlocks, A.out + 2);
        double h[4];
        CK(cudaMemcpyAsync(h, A.out, 4 * sizeof(double), cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
        *J = h[0];
        const double ref = std::sqrt(h[3]);
        int it = 0;
        double res = ref > 0 ? 1.0 : 0.0;
        int rc = FLITE_OK;
        if (ref > 0) {
            rc = X.adj_method == 1 ? gmres_solve(X, A, ref, tol, max_iter, X.adj_restart, &it, &res)
                                   : fixed_point_solve(X, A, ref, tol, max_iter, &it, &res);
        }
        if (rc != FLITE_OK) {
            copy(X, A.u0, L.u, n5);
            cudaStreamSynchronize(X.s);
            ctx->err = "the adjoint iteration diverged";
            return rc;
        }
        if (iterations) *iterations = it;
        if (residual) *residual = res;
        // dJ/dg = J_g + lam^T G_g (the objective's own A and n adjoints are
        // already in Abar and nbar)
        geometry_sweep(X, A, A.lam);
        download_geometry(X, A, side_w_bar, bnd_w_bar, volume_bar);
        CK(cudaStreamSynchronize(X.s));
        // the record left the iterate in u: put the solution back
        copy(X, A.u0, L.u, n5);
        CK(cudaStreamSynchronize(X.s));
        X.drop_graph();
        return FLITE_OK;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return FLITE_ECUDA;
    }
}

extern "C" int flite_objective(flite_ctx *ctx, int objective, double *J) {
    if (!ctx || objective < FLITE_OBJ_CL || objective > FLITE_OBJ_CD || !J) return FLITE_EINVAL;
    if (const char *why = steady_adjoint_unsupported(*ctx)) {
        ctx->err = why;
        return FLITE_EUNSUPPORTED;
    }
    try {
        flite_ctx &X = *ctx;
        SteadyAdjoint &A = buffers(X);
        LevelView &L = X.V(0);
        const size_t n5 = 5 * (size_t)L.N, N = L.N;
        zero(X, A.Ju, n5);
        zero(X, A.Abar, N);
        zero(X, A.nbar, 3 * N);
        objective_terms(X, A, objective, L.u);
        CK(cudaMemcpyAsync(J, A.out, sizeof(double), cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
        return FLITE_OK;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return FLITE_ECUDA;
    }
}

extern "C" int flite_set_adjoint_method(flite_ctx *ctx, int method, int restart) {
    if (!ctx || method < 0 || method > 1 || (method == 1 && (restart < 1 || restart > 500))) return FLITE_EINVAL;
    ctx->adj_method = method;
    if (method == 1) ctx->adj_restart = restart;
    return FLITE_OK;
}

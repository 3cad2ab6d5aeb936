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
    // setBCsOnIncrementField: slip projection, or the no-slip wall of a
    // viscous run (momentum, and the energy of a non-isentropic wall, zeroed)
    const bool vwall = cls == BC_WALL && P.viscous;
    const bool inc_proj = (cls == BC_WALL && !P.viscous) || cls == BC_IWALL || cls == BC_SYM;
    for (int c = 0; c < 5; ++c) sp[c] = s[c];
    if (inc_proj) remove_normal(sp, n0, n1, n2, 1.0);
    if (vwall) {
        sp[1] = 0.0; sp[2] = 0.0; sp[3] = 0.0;
        if (!P.isentropic) sp[4] = 0.0;
    }
    const double dtJ = P.CFL * P.RK[stage - 1];
    for (int c = 0; c < 5; ++c) d[c] = dtJ * sp[c];
    const bool clip = !(fabs(d[0] / up[0]) < P.maxInc);
    clipped_update(P, up, d, z);
    const bool lim1 = z[0] < P.minRho;
    if (lim1) z[0] = P.minRho;
    const double relax = relax_param(P, *L.cyc);
    for (int c = 0; c < 5; ++c) z2[c] = z[c];
    double m2[3] = {0, 0, 0};
    if ((cls == BC_WALL && !P.viscous) || cls == BC_SYM) remove_normal(z2, n0, n1, n2, 1.0);
    if (vwall) {  // momentum rho * coordinateMovement / physicalTimeStep
        z2[1] = z2[0] * L.cmx[i] / P.pts;
        z2[2] = z2[0] * L.cmy[i] / P.pts;
        z2[3] = z2[0] * L.cmz[i] / P.pts;
        if (!P.isentropic) z2[4] = z2[0] * P.Tinf / P.gamma;
    }
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
    if ((cls == BC_WALL && !P.viscous) || cls == BC_SYM) remove_normal_rev(z, n0, n1, n2, 1.0, zb, nb);
    if (vwall) {
        zb[0] += ((zb[1] * L.cmx[i] + zb[2] * L.cmy[i]) + zb[3] * L.cmz[i]) / P.pts;
        zb[1] = 0.0; zb[2] = 0.0; zb[3] = 0.0;
        if (!P.isentropic) {
            zb[0] += zb[4] * P.Tinf / P.gamma;
            zb[4] = 0.0;
        }
    }
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
    if (vwall) {
        sb[1] = 0.0; sb[2] = 0.0; sb[3] = 0.0;
        if (!P.isentropic) sb[4] = 0.0;
    }
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

// the viscous term of one edge end: dv = 2 max(1/Re, mu) |w|^2 / rho
__device__ __forceinline__ double visc_ts_term(const Params &P, double mu, double r, double al, double *dvr,
                                               double *dvmu, double *dval) {
    const bool m = P.am < mu;
    const double vis = m ? mu : P.am;
    const double dv = 2.0 * vis * al / r;
    *dvr = -dv / r;
    *dvmu = m ? 2.0 * al / r : 0.0;
    *dval = 2.0 * vis / r;
    return dv;
}

// dt = 0.5 / t with t = S/V + h/V^2: S sums the convective terms (each
// interior edge f of this node's own state, each boundary edge 2 f(own) +
// f(other)), h the viscous ones (each interior edge the other end's dv, each
// boundary edge 2 dv(own) + dv(other)); the adjoints of S and h per node
// (Sbar, Hbar), this node's own terms in reverse, then the pressure of the
// iteration's start back to the state.  mu: the viscosity the step read;
// mubar its adjoint (laminar runs)
__global__ void k_adj_timestep(Params P, LevelView L, const double *u0, const double *p0, const double *dt,
                               const double *dtbar, const double *p0bar, const double *mu, double *ubar,
                               double *mubar, double *Sbar, double *Hbar, double *Vbar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    const double Vi = L.V[i], dti = dt[i];
    const double tt = 0.5 / dti;  // S/V + h/V^2
    const double tb = -0.5 * dtbar[i] / (tt * tt);
    const double sbi = tb / Vi, hbi = tb / (Vi * Vi);
    Sbar[i] = sbi;
    Hbar[i] = hbi;
    auto hbar_of = [&](int j) {
        const double tj = 0.5 / dt[j];
        return (-0.5 * dtbar[j] / (tj * tj)) / (L.V[j] * L.V[j]);
    };
    double h = 0.0, mb = 0.0, rvb = 0.0;  // viscous sum, and this node's rho / mu adjoints from it
    const bool visc = P.viscous;
    const double mui = visc ? mu[i] : 0.0;
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
        if (visc) {
            const int j = L.inc[k].y;
            const double al = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
            double dr, dm, da;
            h += visc_ts_term(P, mu[j], u0[j], al, &dr, &dm, &da);  // the other end's term
            visc_ts_term(P, mui, ui[0], al, &dr, &dm, &da);         // this end's, in the other's h
            const double hj = hbar_of(j);
            rvb += hj * dr;
            mb += hj * dm;
        }
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
        if (visc) {
            const double al = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
            double dr, dm, da;
            const double own = visc_ts_term(P, mui, ui[0], al, &dr, &dm, &da);
            double drj, dmj, daj;
            h += 2.0 * own + visc_ts_term(P, mu[j], u0[j], al, &drj, &dmj, &daj);
            const double hw = 2.0 * hbi + hbar_of(j);
            rvb += hw * dr;
            mb += hw * dm;
        }
    }
    ub[0] += rvb;
    if (visc && mubar) mubar[i] = mb;
    // V: t = S/V + h/V^2
    if (Vbar) Vbar[i] += tb * (-tt / Vi - h / (Vi * Vi * Vi));
    pb += p0bar[i];
    double p, dp[5];
    pressure_grad(P, ui, &p, dp);
    for (int c = 0; c < 5; ++c) ubar[(size_t)c * N + i] += ub[c] + pb * dp[c];
}

// geometry sweep: the coefficient adjoints of the time step, per edge
__global__ void k_adj_timestep_w(Params P, LevelView L, const double *u0, const double *p0, const double *Sbar,
                                 const double *Hbar, const double *mu, double *swbar) {
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
        if (P.viscous) {  // this end's dv goes to the other end's h
            const double al = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
            double dr, dm, da;
            visc_ts_term(P, mu[n], u[0], al, &dr, &dm, &da);
            const double hw = Hbar[side == 0 ? nd.y : nd.x];
            for (int c = 0; c < 3; ++c) acc[c] += hw * da * 2.0 * w[c];
        }
    }
    for (int c = 0; c < 3; ++c) swbar[(size_t)c * E + e] += acc[c];
}

__global__ void k_adj_timestep_bw(Params P, LevelView L, const double *u0, const double *p0, const double *Sbar,
                                  const double *Hbar, const double *mu, double *bwbar) {
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
        if (P.viscous) {
            const double al = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
            double dr, dm, da;
            visc_ts_term(P, mu[n], u[0], al, &dr, &dm, &da);
            const double hw = 2.0 * Hbar[n] + Hbar[o];
            for (int c = 0; c < 3; ++c) acc[c] += hw * da * 2.0 * w[c];
        }
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

// ---- makeViscosityTerm (def_par:5198-5893), laminar, reverse ---------------
// Layout: G [12][N] Galerkin sums of the primitives (u, v, w, T = gamma/(gamma-1)
// p/rho) per direction (index 4a + k), tau [9][N] (stress xx, xy, xz, yy, yz,
// zz, then the heat flux, projected at adiabatic walls), prim [4][N].

// forward helper of the record: the sums G of def_par:5380-5480 at the
// iteration's start (the primal keeps them in registers)
__global__ void k_adj_visc_sums(LevelView L, const double *prim, double *G) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double g[12];
    for (int c = 0; c < 12; ++c) g[c] = 0.0;
    double qi[4];
    for (int c = 0; c < 4; ++c) qi[c] = prim[(size_t)c * N + i];
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        for (int c = 0; c < 4; ++c) {
            const double sq = qi[c] + prim[(size_t)c * N + t.y];
            for (int a = 0; a < 3; ++a) g[a * 4 + c] += (t.x >= 0 ? sq : -sq) * w[a];
        }
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const int j = side == 0 ? nd.y : nd.x;
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        for (int c = 0; c < 4; ++c) {
            const double q = 3. * qi[c] + prim[(size_t)c * N + j];
            for (int a = 0; a < 3; ++a) g[a * 4 + c] += q * w[a];
        }
    }
    for (int c = 0; c < 12; ++c) G[(size_t)c * N + i] = g[c];
}

// adjoint of one viscous edge flux (f2..f5 of def_par:5700-5760) to one end:
// W = the adjoints of f2..f5, w the coefficients, t (9) and v (3) that end's
// tensor and velocity; adds to tb (9) and vb (3)
__device__ __forceinline__ void visc_flux_end_rev(const double *W, const double *w, const double *t,
                                                  const double *v, double *tb, double *vb) {
    const double wx = w[0], wy = w[1], wz = w[2];
    tb[0] += wx * W[0];
    tb[1] += wy * W[0] + wx * W[1];
    tb[2] += wz * W[0] + wx * W[2];
    tb[3] += wy * W[1];
    tb[4] += wz * W[1] + wy * W[2];
    tb[5] += wz * W[2];
    tb[6] += wx * W[3];
    tb[7] += wy * W[3];
    tb[8] += wz * W[3];
    const double D0 = wx * W[3], D1 = wy * W[3], D2 = wz * W[3];  // adjoints of dut1..dut3
    tb[0] += v[0] * D0;
    tb[1] += v[1] * D0 + v[0] * D1;
    tb[2] += v[2] * D0 + v[0] * D2;
    tb[3] += v[1] * D1;
    tb[4] += v[2] * D1 + v[1] * D2;
    tb[5] += v[2] * D2;
    vb[0] += (t[0] * D0 + t[1] * D1) + t[2] * D2;
    vb[1] += (t[1] * D0 + t[3] * D1) + t[4] * D2;
    vb[2] += (t[2] * D0 + t[4] * D1) + t[5] * D2;
}
// d f2..f5 / d w of the same terms (dt = the summed tensors, dut the summed
// velocity products)
__device__ __forceinline__ void visc_flux_w_rev(const double *W, const double *dt, const double *dut, double *wb) {
    wb[0] += ((W[0] * dt[0] + W[1] * dt[1]) + W[2] * dt[2]) + W[3] * (dt[6] + dut[0]);
    wb[1] += ((W[0] * dt[1] + W[1] * dt[3]) + W[2] * dt[4]) + W[3] * (dt[7] + dut[1]);
    wb[2] += ((W[0] * dt[2] + W[1] * dt[4]) + W[2] * dt[5]) + W[3] * (dt[8] + dut[2]);
}
__device__ __forceinline__ void visc_dut(const double *t, const double *v, double *dut) {
    dut[0] = (v[0] * t[0] + v[1] * t[1]) + v[2] * t[2];
    dut[1] = (v[0] * t[1] + v[1] * t[3]) + v[2] * t[4];
    dut[2] = (v[0] * t[2] + v[1] * t[4]) + v[2] * t[5];
}

// pass 2 in reverse, gathered per node: the adjoints of this node's tensor and
// velocity from the adjoints of the viscous fluxes (diss(:,2:5) -= flux)
__global__ void k_adj_visc_flux(LevelView L, const double *Dbar, const double *tau, const double *prim,
                                double *tbar, double *velbar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double ti[9], vi[3], Wi[4], tb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, vb[3] = {0, 0, 0};
    for (int c = 0; c < 9; ++c) ti[c] = tau[(size_t)c * N + i];
    for (int c = 0; c < 3; ++c) vi[c] = prim[(size_t)c * N + i];
    for (int c = 0; c < 4; ++c) Wi[c] = -Dbar[(size_t)(1 + c) * N + i];
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        double W[4];
        for (int c = 0; c < 4; ++c) {
            const double Wj = -Dbar[(size_t)(1 + c) * N + t.y];
            W[c] = t.x >= 0 ? Wi[c] - Wj : Wj - Wi[c];  // +f to node 1, -f to node 2
        }
        visc_flux_end_rev(W, w, ti, vi, tb, vb);
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int ind = L.bind[b];
        if (ind == 2 || ind == 9) continue;
        const int2 nd = L.bedge[b];
        const int j = side == 0 ? nd.y : nd.x;
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        double W[4];
        // +f to both ends and 2 g(own) to each: f's weight W_i + W_j, g's 2 W_i
        for (int c = 0; c < 4; ++c) W[c] = 3. * Wi[c] - Dbar[(size_t)(1 + c) * N + j];
        visc_flux_end_rev(W, w, ti, vi, tb, vb);
    }
    for (int c = 0; c < 9; ++c) tbar[(size_t)c * N + i] = tb[c];
    for (int c = 0; c < 3; ++c) velbar[(size_t)c * N + i] = vb[c];
}

// the node part in reverse (def_par:5500-5635): tensor and heat flux from the
// gradients, Sutherland's viscosity of T (and the viscosity's own adjoint
// mubar_out, when given), the adiabatic-wall projection; out: the adjoint of
// the sums G, and the parts of ubar (rho) and p0bar; geometry: V and normals
__global__ void k_adj_visc_node(Params P, LevelView L, const double *u0, const double *p0, const double *G,
                                const double *tbar, const double *lam_mu, double *Gbar, double *ubar, double *p0bar,
                                double *Vbar, double *nbar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    const double gOg = P.gamma / (P.gamma - 1.0);
    const double tc = (P.gamma - 1.0) * P.mach * P.mach;
    const double Vi = L.V[i], vt = 1. / Vi;
    double gr[12];
    for (int c = 0; c < 12; ++c) gr[c] = G[(size_t)c * N + i] * vt;
    const double ux = gr[0], vx = gr[1], wx = gr[2], Tx = gr[3];
    const double uy = gr[4], vy = gr[5], wy = gr[6], Ty = gr[7];
    const double uz = gr[8], vz = gr[9], wz = gr[10], Tz = gr[11];
    const double r = u0[i];
    double T = gOg * p0[i] / r;
    const bool tfloor = T <= 0.001;
    if (tfloor) T = 0.001;
    const double a = tc * T, sa = sqrt(a);
    const double C = P.Tinf + 198.6, Dn = tc * P.Tinf * T + 198.6;
    const double oRe = 1. / P.Re, oPr = 1. / P.Pr;
    const double mu = oRe * ((a * sa) * (C / Dn));
    const double kc = oPr * mu;
    double tb[9];
    for (int c = 0; c < 9; ++c) tb[c] = tbar[(size_t)c * N + i];
    const double f43 = 4. / 3., f23 = 2. / 3.;
    const double lin[6] = {f43 * ux - f23 * (vy + wz), uy + vx, uz + wx, f43 * vy - f23 * (ux + wz), vz + wy,
                           f43 * wz - f23 * (ux + vy)};
    double mub = lam_mu ? lam_mu[i] : 0.0;
    for (int c = 0; c < 6; ++c) mub += tb[c] * lin[c];
    // heat flux h = kc grad T, projected at adiabatic walls of level 1
    double h[3] = {kc * Tx, kc * Ty, kc * Tz}, hb[3] = {tb[6], tb[7], tb[8]};
    if (L.grid == 1 && L.bc[i] == BC_WALL) {
        const double n[3] = {L.nx[i], L.ny[i], L.nz[i]};
        const double hn = (h[0] * n[0] + h[1] * n[1]) + h[2] * n[2];
        const double bn = (hb[0] * n[0] + hb[1] * n[1]) + hb[2] * n[2];
        if (nbar)
            for (int c = 0; c < 3; ++c) nbar[(size_t)c * N + i] -= bn * h[c] + hn * hb[c];
        for (int c = 0; c < 3; ++c) hb[c] -= bn * n[c];
    }
    mub += oPr * ((hb[0] * Tx + hb[1] * Ty) + hb[2] * Tz);
    double gb[12];
    gb[0] = mu * (f43 * tb[0] - f23 * tb[3] - f23 * tb[5]);  // u_x
    gb[5] = mu * (-f23 * tb[0] + f43 * tb[3] - f23 * tb[5]);  // v_y
    gb[10] = mu * (-f23 * tb[0] - f23 * tb[3] + f43 * tb[5]);  // w_z
    gb[4] = mu * tb[1];  // u_y
    gb[1] = mu * tb[1];  // v_x
    gb[8] = mu * tb[2];  // u_z
    gb[2] = mu * tb[2];  // w_x
    gb[9] = mu * tb[4];  // v_z
    gb[6] = mu * tb[4];  // w_y
    gb[3] = kc * hb[0];
    gb[7] = kc * hb[1];
    gb[11] = kc * hb[2];
    double vb = 0.0;
    for (int c = 0; c < 12; ++c) {
        Gbar[(size_t)c * N + i] = gb[c] * vt;
        vb -= gb[c] * gr[c] * vt;
    }
    if (Vbar) Vbar[i] += vb;
    // mu(T) = oRe (tc T)^1.5 C / (tc Tin T + 198.6)
    const double dmu = tfloor ? 0.0 : oRe * C * (1.5 * tc * sa / Dn - (a * sa) * tc * P.Tinf / (Dn * Dn));
    const double Tb = mub * dmu;
    p0bar[i] += Tb * gOg / r;
    ubar[i] += -Tb * (gOg * p0[i] / r) / r;
}

// pass 1 in reverse, gathered per node: the primitives' adjoints from the
// sums' adjoints (interior edges: G(1) += (q1+q2) w, G(2) -= (q1+q2) w;
// boundary edges: G(own) += (3 q_own + q_other) w), plus the velocities'
// adjoints of the flux pass, to the state and the pressure
__global__ void k_adj_visc_prim(Params P, LevelView L, const double *u0, const double *p0, const double *Gbar,
                                const double *velbar, double *ubar, double *p0bar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double gi[12], qb[4] = {0, 0, 0, 0};
    for (int c = 0; c < 12; ++c) gi[c] = Gbar[(size_t)c * N + i];
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        const int2 t = L.inc[k];
        const int e = t.x >= 0 ? t.x : ~t.x;
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        for (int c = 0; c < 4; ++c)
            for (int a = 0; a < 3; ++a) {
                const double gj = Gbar[(size_t)(a * 4 + c) * N + t.y];
                qb[c] += w[a] * (t.x >= 0 ? gi[a * 4 + c] - gj : gj - gi[a * 4 + c]);
            }
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        const int b = L.binc[k] >> 1, side = L.binc[k] & 1;
        const int2 nd = L.bedge[b];
        const int j = side == 0 ? nd.y : nd.x;
        const double w[3] = {L.bwx[b], L.bwy[b], L.bwz[b]};
        for (int c = 0; c < 4; ++c)
            for (int a = 0; a < 3; ++a)
                qb[c] += w[a] * (3. * gi[a * 4 + c] + Gbar[(size_t)(a * 4 + c) * N + j]);
    }
    for (int c = 0; c < 3; ++c) qb[c] += velbar[(size_t)c * N + i];
    const double gOg = P.gamma / (P.gamma - 1.0);
    const double r = u0[i];
    double rb = 0.0;
    for (int c = 0; c < 3; ++c) {
        const double m = u0[(size_t)(1 + c) * N + i];
        ubar[(size_t)(1 + c) * N + i] += qb[c] / r;
        rb -= qb[c] * (m / r) / r;
    }
    const double q3 = gOg * p0[i] / r;
    p0bar[i] += qb[3] * gOg / r;
    rb -= qb[3] * q3 / r;
    ubar[i] += rb;
}

// geometry sweep: coefficient adjoints of both viscous passes, per edge
__global__ void k_adj_visc_w(LevelView L, const double *Dbar, const double *tau, const double *prim,
                             const double *Gbar, double *swbar) {
    const int e = tidx();
    if (e >= L.E) return;
    const int N = L.N, E = L.E;
    const int2 nd = L.edge[e];
    double a[9], b[9], va[3], vb[3], dt[9], da[3], db[3], dut[3], W[4], wb[3] = {0, 0, 0};
    for (int c = 0; c < 9; ++c) {
        a[c] = tau[(size_t)c * N + nd.x];
        b[c] = tau[(size_t)c * N + nd.y];
        dt[c] = a[c] + b[c];
    }
    for (int c = 0; c < 3; ++c) { va[c] = prim[(size_t)c * N + nd.x]; vb[c] = prim[(size_t)c * N + nd.y]; }
    visc_dut(a, va, da);
    visc_dut(b, vb, db);
    for (int c = 0; c < 3; ++c) dut[c] = da[c] + db[c];
    for (int c = 0; c < 4; ++c) W[c] = -Dbar[(size_t)(1 + c) * N + nd.x] + Dbar[(size_t)(1 + c) * N + nd.y];
    visc_flux_w_rev(W, dt, dut, wb);
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 3; ++k) {
            const double sq = prim[(size_t)c * N + nd.x] + prim[(size_t)c * N + nd.y];
            wb[k] += sq * (Gbar[(size_t)(k * 4 + c) * N + nd.x] - Gbar[(size_t)(k * 4 + c) * N + nd.y]);
        }
    for (int k = 0; k < 3; ++k) swbar[(size_t)k * E + e] += wb[k];
}

__global__ void k_adj_visc_bw(LevelView L, const double *Dbar, const double *tau, const double *prim,
                              const double *Gbar, double *bwbar) {
    const int b = tidx();
    if (b >= L.B) return;
    const int N = L.N, B = L.B;
    const int2 nd = L.bedge[b];
    double wb[3] = {0, 0, 0};
    if (!(L.bind[b] == 2 || L.bind[b] == 9)) {
        double ta[9], tbb[9], va[3], vb[3], dt[9], da[3], db[3], dut[3], W1[4], W2[4], Wf[4];
        for (int c = 0; c < 9; ++c) {
            ta[c] = tau[(size_t)c * N + nd.x];
            tbb[c] = tau[(size_t)c * N + nd.y];
            dt[c] = ta[c] + tbb[c];
        }
        for (int c = 0; c < 3; ++c) { va[c] = prim[(size_t)c * N + nd.x]; vb[c] = prim[(size_t)c * N + nd.y]; }
        visc_dut(ta, va, da);
        visc_dut(tbb, vb, db);
        for (int c = 0; c < 3; ++c) dut[c] = da[c] + db[c];
        for (int c = 0; c < 4; ++c) {
            W1[c] = -Dbar[(size_t)(1 + c) * N + nd.x];
            W2[c] = -Dbar[(size_t)(1 + c) * N + nd.y];
            Wf[c] = W1[c] + W2[c];
        }
        visc_flux_w_rev(Wf, dt, dut, wb);
        for (int c = 0; c < 4; ++c) { W1[c] *= 2.; W2[c] *= 2.; }
        visc_flux_w_rev(W1, ta, da, wb);
        visc_flux_w_rev(W2, tbb, db, wb);
    }
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 3; ++k) {
            const double q1 = prim[(size_t)c * N + nd.x], q2 = prim[(size_t)c * N + nd.y];
            wb[k] += (3. * q1 + q2) * Gbar[(size_t)(k * 4 + c) * N + nd.x] +
                     (3. * q2 + q1) * Gbar[(size_t)(k * 4 + c) * N + nd.y];
        }
    for (int k = 0; k < 3; ++k) bwbar[(size_t)k * B + b] += wb[k];
}

// the objective's wall-stress part: tbar seeds of sum over wall nodes of
// f A (S n).e (S the stress of tau), with its A and n adjoints
__global__ void k_adj_objective_stress(Params P, LevelView L, const int *wall, int nwall, double ground, double e0,
                                       double e1, double e2, double aref, const double *tau, double *tJ,
                                       double *Abar, double *nbar) {
    const int N = L.N;
    const double f = 2.0 / aref;
    const double e[3] = {e0, e1, e2};
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nwall; q += gridDim.x * blockDim.x) {
        const int ip = wall[q];
        if (!(L.cz[ip] > (ground + 0.01))) continue;
        const double n[3] = {L.nx[ip], L.ny[ip], L.nz[ip]};
        double t[6];
        for (int c = 0; c < 6; ++c) t[c] = tau[(size_t)c * N + ip];
        const double S[3][3] = {{t[0], t[1], t[2]}, {t[1], t[3], t[4]}, {t[2], t[4], t[5]}};
        const double A = L.wallArea[ip];
        double sd = 0.0;
        for (int d = 0; d < 3; ++d)
            for (int c = 0; c < 3; ++c) sd += e[d] * S[d][c] * n[c];
        Abar[ip] += f * sd;
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int d = 0; d < 3; ++d) s += e[d] * S[d][c];
            nbar[(size_t)c * N + ip] += f * A * s;
        }
        const double fA = f * A;
        tJ[ip] += fA * e[0] * n[0];
        tJ[(size_t)N + ip] += fA * (e[0] * n[1] + e[1] * n[0]);
        tJ[2 * (size_t)N + ip] += fA * (e[0] * n[2] + e[2] * n[0]);
        tJ[3 * (size_t)N + ip] += fA * e[1] * n[1];
        tJ[4 * (size_t)N + ip] += fA * (e[1] * n[2] + e[2] * n[1]);
        tJ[5 * (size_t)N + ip] += fA * e[2] * n[2];
    }
}

// pbar (of the iteration's starting pressure) onto the state
__global__ void k_adj_pbar_to_u(Params P, LevelView L, const double *u0, const double *pbar, double *ubar) {
    const int i = tidx();
    if (i >= L.N) return;
    const int N = L.N;
    double x[5], p, dp[5];
    for (int c = 0; c < 5; ++c) x[c] = u0[(size_t)c * N + i];
    pressure_grad(P, x, &p, dp);
    for (int c = 0; c < 5; ++c) ubar[(size_t)c * N + i] += pbar[i] * dp[c];
}

// ---- objective -----------------------------------------------------------
// J = 2/A_ref sum over wall nodes (above the ground plane) of
// -A_i (p_i - p_inf) (n_i . e) (calculateLiftAndDrag def_par:14710-14870,
// inviscid part, pressure of the state): J, dJ/du, dJ/dA and dJ/dn.  One
// thread walks the wall list in order (a node listed twice counts twice).
// the wall-stress term A (S n).e of a laminar run, S the stress part of tau
__device__ __forceinline__ double stress_term(const LevelView &L, const double *tau, int ip, double e0, double e1,
                                              double e2) {
    const size_t N = L.N;
    const double t0 = tau[ip], t1 = tau[N + ip], t2 = tau[2 * N + ip], t3 = tau[3 * N + ip];
    const double t4 = tau[4 * N + ip], t5 = tau[5 * N + ip];
    const double n0 = L.nx[ip], n1 = L.ny[ip], n2 = L.nz[ip];
    const double s0 = (t0 * n0 + t1 * n1) + t2 * n2, s1 = (t1 * n0 + t3 * n1) + t4 * n2;
    const double s2 = (t2 * n0 + t4 * n1) + t5 * n2;
    return L.wallArea[ip] * ((s0 * e0 + s1 * e1) + s2 * e2);
}

__global__ void k_adj_objective(Params P, LevelView L, const int *wall, int nwall, double ground, double e0,
                                double e1, double e2, double aref, const double *u, const double *tau, double *J,
                                double *Ju, double *Abar, double *nbar) {
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
        if (tau) acc += stress_term(L, tau, ip, e0, e1, e2);
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
                                    double e1, double e2, double aref, const double *u, const double *tau,
                                    double *part, double *Ju, double *Abar, double *nbar) {
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
        if (tau) acc += stress_term(L, tau, ip, e0, e1, e2);
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
__global__ void k_adj_update(Params P, LevelView L, int ncomp, const double *ubar, const double *Ju, double *lam,
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
        for (int c = 0; c < ncomp; ++c) {
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

__global__ void k_adj_add(const double *a, size_t n, double *w) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        w[i] = w[i] + a[i];
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
__global__ void k_gm_apply(Params P, LevelView L, int ncomp, const double *v, const double *ubar, const double *b,
                           double *w, int mode) {
    const int N = L.N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const bool fixE = inflow_energy_fixed(P, L, i);
        for (int c = 0; c < ncomp; ++c) {
            const size_t k = (size_t)c * N + i;
            double pu = mode == 2 ? v[k] : ubar[k];
            if (c == 4 && fixE) pu = 0.0;
            w[k] = mode == 2 ? pu : (mode == 0 ? v[k] - pu : b[k] - (v[k] - pu));
        }
    }
}

// The adjoint's unknowns are the level-1 state (5 components) and, in a
// laminar run, the laminar viscosity that the next iteration's time step reads
// (makeTimeSteps runs before makeViscosityTerm recomputes it, def_par:
// 1010-1035): lam, ubar, Ju and the Krylov vectors hold nc = 5 or 6
// components of N values.
struct SteadyAdjoint {
    int N = 0, E = 0, B = 0, nc = 5;
    double *u0, *v1, *v2, *Q[3], *p0, *dt, *D, *lap, *sens, *nh6, *nh7;
    double *lam, *vb[2], *ubar, *Qbar, *Dbar, *dtbar, *pbar, *p0bar, *nhbar, *nh6bar, *nh7bar, *Sbar, *Hbar, *bvjp;
    double *Vbar, *nbar, *swbar, *bwbar, *Abar, *abar, *Ju, *part, *out;
    // laminar runs: the viscosity the time step reads, the tensor, primitives
    // and gradient sums of the iteration's start, their adjoints, the
    // objective's tensor seeds and the primal's viscosity kept aside
    double *mu0 = nullptr, *tau = nullptr, *prim = nullptr, *Gv = nullptr, *tbar = nullptr, *velbar = nullptr;
    double *Gbar = nullptr, *tJ = nullptr, *mu_keep = nullptr, *ws_keep = nullptr;
    // GMRES: Krylov vectors [(m+1)][nc N], right-hand side, dot partials
    double *kry = nullptr, *rhs = nullptr, *gpart = nullptr, *gh = nullptr;
    int kry_m = 0;
    bool recorded = false;
};

void destroy_steady_adjoint(SteadyAdjoint *a) { delete a; }

static const char *steady_adjoint_unsupported(const flite_ctx &X) {
    const flite_controls &c = X.c;
    if (c.fluxType != 1) return "the steady adjoint takes the central flux (fluxType 1)";
    if (c.flowType != 0) return "the steady adjoint takes steady runs (flowType 0)";
    if (X.P.engines) return "the steady adjoint covers meshes without engine boundary conditions";
    if (c.rungeKuttaStages != 3) return "the steady adjoint takes the reference's three stages";
    if (c.turbulenceModel != 0) return "the steady adjoint covers inviscid and laminar runs (no turbulence model)";
    if (c.dissipationScheme == 1 || c.dissipationScheme == 3) return "the steady adjoint takes the scalar JST dissipation (scheme 2)";
    if (c.useDissipationWeighting) return "the steady adjoint takes unweighted dissipation";
    if (c.useMatrixDissipation) return "the steady adjoint takes the scalar JST dissipation";
    if (c.ReynoldsNumber > 0 && c.viscosityScheme != 1)
        return "the steady adjoint takes the viscous term of viscosityScheme 1";
    return nullptr;
}

static SteadyAdjoint &buffers(flite_ctx &X) {
    LevelView &L = X.V(0);
    if (!X.sadj) {
        auto *a = new SteadyAdjoint();
        X.sadj = a;
        a->N = L.N; a->E = L.E; a->B = L.B;
        a->nc = X.P.viscous ? 6 : 5;
        const size_t n5 = 5 * (size_t)L.N, N = L.N, na = (size_t)a->nc * N;
        for (double **p : {&a->u0, &a->v1, &a->v2, &a->Q[0], &a->Q[1], &a->Q[2], &a->D, &a->lap, &a->vb[0],
                           &a->vb[1], &a->Qbar, &a->Dbar, &a->nhbar})
            *p = X.alloc<double>(n5);
        for (double **p : {&a->lam, &a->ubar, &a->Ju}) *p = X.alloc<double>(na);
        for (double **p : {&a->p0, &a->dt, &a->sens, &a->nh6, &a->nh7, &a->dtbar, &a->pbar, &a->p0bar, &a->nh6bar,
                           &a->nh7bar, &a->Sbar, &a->Hbar, &a->Vbar, &a->Abar})
            *p = X.alloc<double>(N);
        if (X.P.viscous) {
            a->mu0 = X.alloc<double>(N);
            a->mu_keep = X.alloc<double>(N);
            a->ws_keep = X.alloc<double>(3 * N);
            a->tau = X.alloc<double>(9 * N);
            a->tbar = X.alloc<double>(9 * N);
            a->tJ = X.alloc<double>(9 * N);
            a->prim = X.alloc<double>(4 * N);
            a->velbar = X.alloc<double>(3 * N);
            a->Gv = X.alloc<double>(12 * N);
            a->Gbar = X.alloc<double>(12 * N);
        }
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
static void objective_terms(flite_ctx &X, SteadyAdjoint &A, int objective, const double *u,
                            const double *tau = nullptr) {
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
    const bool unique = std::adjacent_find(w.begin(), w.end()) == w.end();
    if (unique) {
        k_adj_objective_par<<<kObjBlocks, 256, 0, X.s>>>(X.P, L, D.d_wall, nw, X.c.groundplane, dir[0], dir[1],
                                                         dir[2], X.c.referenceArea, u, tau, A.part, A.Ju, A.Abar,
                                                         A.nbar);
        k_gm_dots_final<<<1, 32, 0, X.s>>>(A.part, kObjBlocks, 1, A.out);
    } else {
        k_adj_objective<<<1, 1, 0, X.s>>>(X.P, L, D.d_wall, nw, X.c.groundplane, dir[0], dir[1], dir[2],
                                          X.c.referenceArea, u, tau, A.out, A.Ju, A.Abar, A.nbar);
    }
    if (tau && A.tJ) {  // the wall stress: seeds of the tensor's adjoint, kept for the geometry sweep
        zero(X, A.tJ, 9 * (size_t)L.N);
        k_adj_objective_stress<<<unique ? kObjBlocks : 1, unique ? 256 : 1, 0, X.s>>>(
            X.P, L, D.d_wall, nw, X.c.groundplane, dir[0], dir[1], dir[2], X.c.referenceArea, tau, A.tJ, A.Abar,
            A.nbar);
    }
}

static void zero(flite_ctx &X, double *p, size_t n) {
    k_adj_zero<<<std::min<size_t>((n + 255) / 256, 4096), 256, 0, X.s>>>(p, n);
}
static void copy(flite_ctx &X, const double *a, double *b, size_t n) {
    CK(cudaMemcpyAsync(b, a, n * sizeof(double), cudaMemcpyDeviceToDevice, X.s));
}

// the laminar part of the reverse sweep: the viscous fluxes' adjoints (from
// Dbar; with tseed added, the objective's tensor seeds), the node part with
// the viscosity's own adjoint lam_mu, the gradient sums; into ubar and p0bar
static void viscous_reverse(flite_ctx &X, SteadyAdjoint &A, const double *lam_mu, const double *tseed,
                            bool from_fluxes, bool geom) {
    LevelView &L = X.V(0);
    const size_t N = L.N;
    const unsigned nbk = X.nblk(N);
    if (from_fluxes) {
        k_adj_visc_flux<<<nbk, X.nb, 0, X.s>>>(L, A.Dbar, A.tau, A.prim, A.tbar, A.velbar);
    } else {
        zero(X, A.tbar, 9 * N);
        zero(X, A.velbar, 3 * N);
    }
    if (tseed) k_adj_add<<<592, 256, 0, X.s>>>(tseed, 9 * N, A.tbar);
    k_adj_visc_node<<<nbk, X.nb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.Gv, A.tbar, lam_mu, A.Gbar, A.ubar, A.p0bar,
                                           geom ? A.Vbar : nullptr, geom ? A.nbar : nullptr);
    k_adj_visc_prim<<<nbk, X.nb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.Gbar, A.velbar, A.ubar, A.p0bar);
    if (geom) {
        k_adj_visc_w<<<X.eblk(L.E), X.eb, 0, X.s>>>(L, A.Dbar, A.tau, A.prim, A.Gbar, A.swbar);
        if (L.B > 0) k_adj_visc_bw<<<X.eblk(L.B), X.eb, 0, X.s>>>(L, A.Dbar, A.tau, A.prim, A.Gbar, A.bwbar);
    }
}

// laminar runs: the objective's wall-stress part of dJ/du, through the
// gradient chain at the recorded state, added to Ju
static void objective_stress_u(flite_ctx &X, SteadyAdjoint &A) {
    LevelView &L = X.V(0);
    const size_t N = L.N, n5 = 5 * N;
    zero(X, A.ubar, n5);
    zero(X, A.p0bar, N);
    zero(X, A.Dbar, n5);
    viscous_reverse(X, A, nullptr, A.tJ, false, false);
    k_adj_pbar_to_u<<<X.nblk(N), X.nb, 0, X.s>>>(X.P, L, A.u0, A.p0bar, A.ubar);
    k_adj_add<<<592, 256, 0, X.s>>>(A.ubar, n5, A.Ju);
}

// the primal iteration from A.u0, recording the stage states, their
// residuals and the iteration's time step and dissipation
static void record(flite_ctx &X, SteadyAdjoint &A) {
    LevelView &L = X.V(0);
    const size_t n5 = 5 * (size_t)L.N, N = L.N;
    // a FLITE_MIXED run converges to the FP64 iteration's fixed point: its
    // adjoint is the FP64 one, recorded with the FP64 kernels
    struct PrecisionGuard {
        flite_ctx &X;
        int keep;
        ~PrecisionGuard() { X.c.precision = keep; }
    } guard{X, X.c.precision};
    X.c.precision = FLITE_FP64;
    copy(X, A.u0, L.u, n5);
    copy(X, A.u0, L.uprev, n5);
    if (X.P.viscous) copy(X, A.mu0, L.mu, N);
    X.pressure(0);
    X.timesteps(0);
    X.dissipation(0);
    if (X.P.viscous) {
        X.viscous(0);
        copy(X, L.tau, A.tau, 9 * N);
        copy(X, L.prim, A.prim, 4 * N);
        k_adj_visc_sums<<<X.nblk(N), X.nb, 0, X.s>>>(L, A.prim, A.Gv);
    }
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

// ubar = G_u^T lam (geometry sweep: and the geometry adjoints); lam and ubar
// hold nc components (the state, and in laminar runs the viscosity)
static void reverse(flite_ctx &X, SteadyAdjoint &A, const double *lam, bool geom, const double *tseed = nullptr) {
    LevelView &L = X.V(0);
    const size_t n5 = 5 * (size_t)L.N, N = L.N;
    const unsigned nbk = X.nblk(N);
    zero(X, A.ubar, (size_t)A.nc * N);
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
    if (X.P.viscous) viscous_reverse(X, A, lam + n5, geom ? tseed : nullptr, true, geom);
    const bool jst = !(X.c.fourthOrderDissipationFactor == 0 && X.c.secondOrderDissipationFactor == 0);
    if (jst) {
        k_adj_jst_edges<<<nbk, X.nb, 0, X.s>>>(X.P, L, A.u0, A.dt, A.lap, A.sens, A.nh6, A.nh7, A.Dbar, A.ubar,
                                               A.dtbar, A.nhbar, A.nh6bar, A.nh7bar, Vb);
        k_adj_jst_lap<<<nbk, X.nb, 0, X.s>>>(L, A.nhbar, A.nh6bar, A.nh7bar, A.ubar, A.p0bar);
    }
    k_adj_timestep<<<nbk, X.nb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.dt, A.dtbar, A.p0bar, A.mu0, A.ubar,
                                          X.P.viscous ? A.ubar + n5 : nullptr, A.Sbar, A.Hbar, Vb);
    if (geom) {
        k_adj_timestep_w<<<X.eblk(L.E), X.eb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.Sbar, A.Hbar, A.mu0, A.swbar);
        if (L.B > 0)
            k_adj_timestep_bw<<<X.eblk(L.B), X.eb, 0, X.s>>>(X.P, L, A.u0, A.p0, A.Sbar, A.Hbar, A.mu0, A.bwbar);
    }
}

// geometry adjoints: zeroed, swept, the normals and wall areas chained to bnd_w
static void geometry_sweep(flite_ctx &X, SteadyAdjoint &A, const double *lam, const double *tseed = nullptr) {
    LevelView &L = X.V(0);
    const size_t N = L.N;
    zero(X, A.swbar, 3 * (size_t)L.E);
    zero(X, A.bwbar, 3 * (size_t)std::max(L.B, 1));
    reverse(X, A, lam, true, tseed);
    k_adj_normals<<<X.nblk(N), X.nb, 0, X.s>>>(L, A.nbar, A.abar);
    if (L.B > 0) k_adj_bedge_geom<<<X.eblk(L.B), X.eb, 0, X.s>>>(L, A.abar, A.Abar, A.bwbar);
}

static void download_geometry(flite_ctx &X, SteadyAdjoint &A, double *swb, double *bwb, double *vb) {
    LevelView &L = X.V(0);
    if (swb) CK(cudaMemcpyAsync(swb, A.swbar, 3 * (size_t)L.E * sizeof(double), cudaMemcpyDeviceToHost, X.s));
    if (bwb && L.B > 0)
        CK(cudaMemcpyAsync(bwb, A.bwbar, 3 * (size_t)L.B * sizeof(double), cudaMemcpyDeviceToHost, X.s));
    if (vb) X.get_nodes(0, vb, A.Vbar, 1);
}

// lam <- P (G_u^T lam + Ju) from lam = P Ju, `check` iterations per launch of
// one captured graph, until |dlam| <= tol |P Ju|
static int fixed_point_solve(flite_ctx &X, SteadyAdjoint &A, double ref, double tol, int max_iter, int *its,
                             double *res_out) {
    LevelView &L = X.V(0);
    const int check = 10;
    auto iterate = [&]() {
        reverse(X, A, A.lam, false);
        k_adj_update<<<kAdjBlocks, 256, 0, X.s>>>(X.P, L, A.nc, A.ubar, A.Ju, A.lam, A.part);
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
    const size_t n = (size_t)A.nc * L.N;
    if (A.kry_m < m) {
        // the vectors of a smaller restart length stay allocated until the context goes
        A.kry = X.alloc<double>((size_t)(m + 1) * n);
        A.gpart = X.alloc<double>((size_t)kDotBlocks * (m + 1));
        A.gh = X.alloc<double>(m + 1);
        if (!A.rhs) A.rhs = X.alloc<double>(n);
        A.kry_m = m;
    }
    const unsigned eb = 592;
    k_gm_apply<<<eb, 256, 0, X.s>>>(X.P, L, A.nc, A.Ju, nullptr, nullptr, A.rhs, 2);  // b = P Ju
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
    double res = 1.0, prev = -1.0;
    while (true) {
        // r = b - (I - A) lam in V_0
        reverse(X, A, A.lam, false);
        k_gm_apply<<<eb, 256, 0, X.s>>>(X.P, L, A.nc, A.lam, A.ubar, A.rhs, Vj(0), 1);
        ++total;
        double beta = norm(Vj(0));
        if (!std::isfinite(beta)) return FLITE_ENAN;
        res = beta / bnorm;
        if (res <= tol || total >= max_iter) break;
        if (prev > 0 && res > 0.9 * prev) {
            // Restarted GMRES can stall where G_u^T is far from normal (its
            // powers grow for a while before they decay): the fixed-point
            // iteration, which converges at the smoother's rate whatever the
            // transient, takes over for a stretch, then GMRES again
            int fit = 0;
            double fres = res;
            const int rc = fixed_point_solve(X, A, bnorm, tol, std::min(max_iter - total, 20 * (m + 1)), &fit, &fres);
            if (rc != FLITE_OK) return rc;
            total += fit;
            prev = -1.0;
            if (fres <= tol || total >= max_iter) {
                res = fres;
                break;
            }
            continue;
        }
        prev = res;
        k_gm_scale<<<eb, 256, 0, X.s>>>(Vj(0), n, 1.0 / beta);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        for (; k < m && total < max_iter; ++k) {
            double *w = Vj(k + 1);
            reverse(X, A, Vj(k), false);
            k_gm_apply<<<eb, 256, 0, X.s>>>(X.P, L, A.nc, Vj(k), A.ubar, nullptr, w, 0);
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
                                   double *side_w_bar, double *bnd_w_bar, double *volume_bar, const double *mu,
                                   const double *lam_mu, double *mu_bar) {
    if (!ctx || !u || !lam || !ubar) return FLITE_EINVAL;
    if (const char *why = steady_adjoint_unsupported(*ctx)) {
        ctx->err = why;
        return FLITE_EUNSUPPORTED;
    }
    if (ctx->P.viscous && !mu) {
        ctx->err = "a laminar run's iteration needs the viscosity its time step reads";
        return FLITE_EINVAL;
    }
    try {
        flite_ctx &X = *ctx;
        SteadyAdjoint &A = buffers(X);
        LevelView &L = X.V(0);
        const size_t n5 = 5 * (size_t)L.N, N = L.N;
        const bool visc = X.P.viscous;
        // the primal state of level 1 is kept: the record overwrites u, uprev,
        // p, dt, the dissipation and rhs (and the viscosity and wall stress)
        std::vector<double> keep(n5);
        CK(cudaMemcpyAsync(keep.data(), L.u, n5 * sizeof(double), cudaMemcpyDeviceToHost, X.s));
        if (visc) {
            copy(X, L.mu, A.mu_keep, N);
            copy(X, L.wstress, A.ws_keep, 3 * N);
            X.put_nodes(0, A.mu0, mu, 1);
            if (lam_mu) X.put_nodes(0, A.lam + n5, lam_mu, 1);
            else zero(X, A.lam + n5, N);
        }
        X.put_nodes(0, A.u0, u, 5);
        X.put_nodes(0, A.lam, lam, 5);
        record(X, A);
        zero(X, A.Vbar, N);
        zero(X, A.nbar, 3 * N);
        zero(X, A.Abar, N);
        const bool geom = side_w_bar || bnd_w_bar || volume_bar;
        if (geom) geometry_sweep(X, A, A.lam);
        else reverse(X, A, A.lam, false);
        X.get_nodes(0, ubar, A.ubar, 5);
        if (visc && mu_bar) X.get_nodes(0, mu_bar, A.ubar + n5, 1);
        if (geom) download_geometry(X, A, side_w_bar, bnd_w_bar, volume_bar);
        if (visc) {
            copy(X, A.mu_keep, L.mu, N);
            copy(X, A.ws_keep, L.wstress, 3 * N);
        }
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
        const size_t n5 = 5 * (size_t)L.N, N = L.N, na = (size_t)A.nc * N;
        const bool visc = X.P.viscous;
        // linearisation point: the context's level-1 state and, in a laminar
        // run, the viscosity its next time step reads
        copy(X, L.u, A.u0, n5);
        if (visc) {
            copy(X, L.mu, A.mu0, N);
            copy(X, L.mu, A.mu_keep, N);
            copy(X, L.wstress, A.ws_keep, 3 * N);
        }
        zero(X, A.Ju, na);
        zero(X, A.Abar, N);
        zero(X, A.Vbar, N);
        zero(X, A.nbar, 3 * N);
        record(X, A);
        objective_terms(X, A, objective, A.u0, visc ? A.tau : nullptr);
        if (visc) objective_stress_u(X, A);
        // lam_0 = P Ju
        zero(X, A.lam, na);
        zero(X, A.ubar, na);
        k_adj_update<<<kAdjBlocks, 256, 0, X.s>>>(X.P, L, A.nc, A.ubar, A.Ju, A.lam, A.part);
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
        auto restore = [&]() {
            copy(X, A.u0, L.u, n5);
            if (visc) {
                copy(X, A.mu_keep, L.mu, N);
                copy(X, A.ws_keep, L.wstress, 3 * N);
            }
        };
        if (rc != FLITE_OK) {
            restore();
            cudaStreamSynchronize(X.s);
            ctx->err = "the adjoint iteration diverged";
            return rc;
        }
        if (iterations) *iterations = it;
        if (residual) *residual = res;
        // dJ/dg = J_g + lam^T G_g (the objective's own A and n adjoints are
        // already in Abar and nbar; its wall-stress seeds join the sweep)
        geometry_sweep(X, A, A.lam, visc ? A.tJ : nullptr);
        download_geometry(X, A, side_w_bar, bnd_w_bar, volume_bar);
        // the record left the iterate in u: put the solution back
        restore();
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
        zero(X, A.out, 1);
        const double *tau = nullptr;
        if (X.P.viscous) {
            // the tensor of makeViscosityTerm at the state (its viscosity and
            // wall stress, which the next iteration and flite_forces read,
            // are put back)
            copy(X, L.mu, A.mu_keep, N);
            copy(X, L.wstress, A.ws_keep, 3 * N);
            X.pressure(0);
            k_visc_prim<<<X.nblk(N), X.nb, 0, X.s>>>(X.P, L);
            X.visc_grad(0);
            copy(X, L.tau, A.tau, 9 * N);
            copy(X, A.mu_keep, L.mu, N);
            copy(X, A.ws_keep, L.wstress, 3 * N);
            tau = A.tau;
        }
        objective_terms(X, A, objective, L.u, tau);
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

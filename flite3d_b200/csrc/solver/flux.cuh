// Edge and boundary-edge fluxes of makeRHS (def_par:1525-2512).
#pragma once
#include "device.cuh"

namespace flite {

struct NodeState {
    double r, ru, rv, rw, E, p;
};

__device__ __forceinline__ NodeState load_state(const LevelView &L, int i) {
    NodeState s;
    s.r = L.u[i];
    s.ru = L.u[L.N + i];
    s.rv = L.u[2 * L.N + i];
    s.rw = L.u[3 * L.N + i];
    s.E = L.u[4 * L.N + i];
    s.p = L.p[i];
    return s;
}

// LED limiter of the HLLC reconstruction (def_par:1856-1867); the root
// (1+t^nsig)^(1/nsig) is sqrt(sqrt(.)) for nsig=4 and sqrt(.) for nsig=2
__device__ __forceinline__ double led(double a, double bmin, double bmax, int nsig) {
    double cc = a;
    double a1 = 2.0 * a;
    if (a1 > 0.0) {
        double invmax = 0.0;
        if (bmax > 0.0) invmax = 1.0 / bmax;
        double t = a1 * invmax;
        double tn = nsig == 4 ? (t * t) * (t * t) : t * t;
        double root = nsig == 4 ? sqrt(sqrt(1. + tn)) : sqrt(1. + tn);
        cc = 0.5 * bmax * t / root;
    } else if (a1 < 0.0) {
        double invmin = 0.0;
        if (bmin < 0.0) invmin = 1.0 / bmin;
        double t = a1 * invmin;
        double tn = nsig == 4 ? (t * t) * (t * t) : t * t;
        double root = nsig == 4 ? sqrt(sqrt(1. + tn)) : sqrt(1. + tn);
        cc = 0.5 * bmin * t / root;
    }
    return cc;
}

// central flux of an edge from its two node states (def_par:1664-1669)
__device__ __forceinline__ void central_flux(const NodeState &a, const NodeState &b, double wx, double wy,
                                             double wz, double *f) {
    double pr1 = a.p, rinv1 = 1. / a.r;
    double ru1 = a.ru, rv1 = a.rv, rw1 = a.rw;
    double u1 = rinv1 * ru1, v1 = rinv1 * rv1, w1 = rinv1 * rw1;
    double rh1 = a.E + pr1;
    double pr2 = b.p, rinv2 = 1. / b.r;
    double ru2 = b.ru, rv2 = b.rv, rw2 = b.rw;
    double u2 = rinv2 * ru2, v2 = rinv2 * rv2, w2 = rinv2 * rw2;
    double rh2 = b.E + pr2;
    f[0] = (wx * (ru1 + ru2) + wy * (rv1 + rv2)) + wz * (rw1 + rw2);
    f[1] = (wx * (((ru1 * u1 + pr1) + ru2 * u2) + pr2) + wy * (ru1 * v1 + ru2 * v2)) + wz * (ru1 * w1 + ru2 * w2);
    f[2] = (wx * (rv1 * u1 + rv2 * u2) + wy * (((rv1 * v1 + pr1) + rv2 * v2) + pr2)) + wz * (rv1 * w1 + rv2 * w2);
    f[3] = (wx * (rw1 * u1 + rw2 * u2) + wy * (rw1 * v1 + rw2 * v2)) + wz * (((rw1 * w1 + pr1) + rw2 * w2) + pr2);
    f[4] = (wx * (rh1 * u1 + rh2 * u2) + wy * (rh1 * v1 + rh2 * v2)) + wz * (rh1 * w1 + rh2 * w2);
}

// the same central flux from two node records (1/rho and E + p formed once
// per node by k_pressure with the same operations)
__device__ __forceinline__ void central_flux_rec(const NodeRec &a, const NodeRec &b, double wx, double wy,
                                                 double wz, double *f) {
    const double pr1 = a.p, rinv1 = a.rinv, ru1 = a.ru, rv1 = a.rv, rw1 = a.rw, rh1 = a.rh;
    const double u1 = rinv1 * ru1, v1 = rinv1 * rv1, w1 = rinv1 * rw1;
    const double pr2 = b.p, rinv2 = b.rinv, ru2 = b.ru, rv2 = b.rv, rw2 = b.rw, rh2 = b.rh;
    const double u2 = rinv2 * ru2, v2 = rinv2 * rv2, w2 = rinv2 * rw2;
    f[0] = (wx * (ru1 + ru2) + wy * (rv1 + rv2)) + wz * (rw1 + rw2);
    f[1] = (wx * (((ru1 * u1 + pr1) + ru2 * u2) + pr2) + wy * (ru1 * v1 + ru2 * v2)) + wz * (ru1 * w1 + ru2 * w2);
    f[2] = (wx * (rv1 * u1 + rv2 * u2) + wy * (((rv1 * v1 + pr1) + rv2 * v2) + pr2)) + wz * (rv1 * w1 + rv2 * w2);
    f[3] = (wx * (rw1 * u1 + rw2 * u2) + wy * (rw1 * v1 + rw2 * v2)) + wz * (((rw1 * w1 + pr1) + rw2 * w2) + pr2);
    f[4] = (wx * (rh1 * u1 + rh2 * u2) + wy * (rh1 * v1 + rh2 * v2)) + wz * (rh1 * w1 + rh2 * w2);
}

// The Van Albada limited slope of the upwind-biased difference a and the
// edge difference b (an extension, no reference counterpart): ab(a+b) /
// (a^2+b^2) when a and b have the same sign, else 0.
__device__ __forceinline__ double van_albada(double a, double b) {
    const double ab = a * b;
    if (ab <= 0.0) return 0.0;
    return (ab * (a + b)) / (a * a + b * b);
}

// Interior edge flux f of edge e (i1 -> i2), added to rhs(i1) and
// subtracted from rhs(i2).  FT is the fluxType and O2 selects the HLLC
// reconstruction (with the Roe flux: the upwind sign of the extension); both are compile-time so that each kernel instance only
// holds the registers of its own flux.
template <int FT, bool O2>
__device__ __forceinline__ void edge_flux(const Params &P, const LevelView &L, int e, int i1, int i2, double *f) {
    const NodeState a = load_state(L, i1), b = load_state(L, i2);
    const double gam = P.gamma, gam1 = P.gm1;
    double pr1 = a.p, r1 = a.r, rinv1 = 1. / a.r;
    double ru1 = a.ru, rv1 = a.rv, rw1 = a.rw;
    double u1 = rinv1 * ru1, v1 = rinv1 * rv1, w1 = rinv1 * rw1;
    double E1 = a.E, rh1 = a.E + pr1;
    double pr2 = b.p, r2 = b.r, rinv2 = 1. / b.r;
    double ru2 = b.ru, rv2 = b.rv, rw2 = b.rw;
    double u2 = rinv2 * ru2, v2 = rinv2 * rv2, w2 = rinv2 * rw2;
    double E2 = b.E, rh2 = b.E + pr2;
    const double wx = L.wx[e], wy = L.wy[e], wz = L.wz[e];
    f[0] = f[1] = f[2] = f[3] = f[4] = 0.0;
    // moving meshes: the GCL term -q wgcl (def_par:1662-1791)
    const double wgcl = L.gclw ? L.gclw[e] : 0.0;
    auto gcl_sum = [&]() {
        if (!L.gclw) return;
        f[0] = f[0] - (r1 + r2) * wgcl; f[1] = f[1] - (ru1 + ru2) * wgcl; f[2] = f[2] - (rv1 + rv2) * wgcl;
        f[3] = f[3] - (rw1 + rw2) * wgcl; f[4] = f[4] - (E1 + E2) * wgcl;
    };
    if constexpr (FT == 1 || FT == 4) {
        // central flux; HLLC starts from it too (def_par:1798)
        central_flux(a, b, wx, wy, wz, f);
        if constexpr (FT == 1) {
            gcl_sum();
            return;
        }
    }
    if constexpr (FT == 2) {  // local Lax-Friedrichs (def_par:1670-1724)
        double rnorm = sqrt((wx * wx + wy * wy) + wz * wz);
        if (rnorm > 1.0e-10) {
            double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
            double c1 = sqrt(gam * pr1 * rinv1);
            double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
            double c2 = sqrt(gam * pr2 * rinv2);
            double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
            double l11 = fabs(nv1 + c1), l12 = fabs(nv2 + c2);
            double l1 = l11; if (l1 < l12) l1 = l12;
            double l21 = fabs(nv1 - c1), l22 = fabs(nv2 - c2);
            double l2 = l21; if (l2 < l22) l2 = l22;
            double lam = l1; if (lam < l2) lam = l2;
            f[0] = rnorm * ((r1 * nv1 + r2 * nv2) - lam * (r1 - r2));
            f[1] = rnorm * (((pr1 * rnx + ru1 * nv1) + (pr2 * rnx + ru2 * nv2)) - lam * (ru1 - ru2));
            f[2] = rnorm * (((pr1 * rny + rv1 * nv1) + (pr2 * rny + rv2 * nv2)) - lam * (rv1 - rv2));
            f[3] = rnorm * (((pr1 * rnz + rw1 * nv1) + (pr2 * rnz + rw2 * nv2)) - lam * (rw1 - rw2));
            f[4] = rnorm * ((rh1 * nv1 + rh2 * nv2) - lam * (E1 - E2));
            gcl_sum();
        }
        return;
    }
    if constexpr (FT == 3) {  // Roe (def_par:1725-1792)
        double rnorm = sqrt((wx * wx + wy * wy) + wz * wz);
        if (rnorm > 1.0e-10) {
            double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
            u1 = ru1 * rinv1; v1 = rv1 * rinv1; w1 = rw1 * rinv1;
            double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
            double f11 = r1 * nv1, f21 = pr1 * rnx + ru1 * nv1, f31 = pr1 * rny + rv1 * nv1;
            double f41 = pr1 * rnz + rw1 * nv1, f51 = rh1 * nv1;
            double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
            double f12 = r2 * nv2, f22 = pr2 * rnx + ru2 * nv2, f32 = pr2 * rny + rv2 * nv2;
            double f42 = pr2 * rnz + rw2 * nv2, f52 = rh2 * nv2;
            double h1 = rh1 * rinv1, h2 = rh2 * rinv2;
            double di = sqrt(r1 / r2), d1 = 1.0 / (di + 1.0);
            double ui = (di * u1 + u2) * d1, vi = (di * v1 + v2) * d1, wi = (di * w1 + w2) * d1;
            double hi = (di * h1 + h2) * d1;
            double ci2 = gam1 * (hi - 0.5 * ((ui * ui + vi * vi) + wi * wi));
            ci2 = dmax(ci2, 1.0e-5);
            double ci = sqrt(ci2);
            double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
            double ucp = (ui * rnx + vi * rny) + wi * rnz;
            double du1 = r1 - r2, du2 = ru1 - ru2, du3 = rv1 - rv2, du4 = rw1 - rw2, du5 = E1 - E2;
            if constexpr (O2) {
                // the extension (coarse levels) adds the Roe dissipation with
                // the upwind sign; the reference's interior branch subtracts it
                du1 = r2 - r1; du2 = ru2 - ru1; du3 = rv2 - rv1; du4 = rw2 - rw1; du5 = E2 - E1;
            }
            double l1 = fabs(ucp + ci), l2 = fabs(ucp - ci), l3 = fabs(ucp);
            double s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
            double al1x = gam1 * ((((af * du1 - ui * du2) - vi * du3) - wi * du4) + du5);
            double al2x = ((-ucp * du1 + du2 * rnx) + du3 * rny) + du4 * rnz;
            double cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci);
            double cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
            f[0] = rnorm * ((f11 + f12) - (l3 * du1 + cc1));
            f[1] = rnorm * ((f21 + f22) - ((l3 * du2 + cc1 * ui) + cc2 * rnx));
            f[2] = rnorm * ((f31 + f32) - ((l3 * du3 + cc1 * vi) + cc2 * rny));
            f[3] = rnorm * ((f41 + f42) - ((l3 * du4 + cc1 * wi) + cc2 * rnz));
            f[4] = rnorm * ((f51 + f52) - ((l3 * du5 + cc1 * hi) + cc2 * ucp));
            gcl_sum();
        }
        return;
    }
    if constexpr (FT == 4) {
    // HLLC (def_par:1794-2085)
    double roe1 = a.r, roe2 = b.r, re1 = a.E, re2 = b.E;
    double wx2 = 2.0 * wx, wy2 = 2.0 * wy, wz2 = 2.0 * wz;
    double rnorm = sqrt((wx2 * wx2 + wy2 * wy2) + wz2 * wz2);
    double rnorm1 = rnorm;
    if (rnorm > 0.0) rnorm = 1.0 / rnorm;
    double rnx = wx2 * rnorm, rny = wy2 * rnorm, rnz = wz2 * rnorm;
    if constexpr (O2) {
        double dpvl[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (L.grid == 1) {
            // coarse levels have zero coordinates: dx = 0 gives dpvl = 0
            double dx = L.cx[i2] - L.cx[i1], dy = L.cy[i2] - L.cy[i1], dz = L.cz[i2] - L.cz[i1];
            double hlength = 0.5 * P.clip * sqrt((dx * dx + dy * dy) + dz * dz);
            const int N = L.N;
            for (int j = 0; j < 5; ++j) {
                double dpv1 = 0.5 * ((L.grad[j * N + i1] * dx + L.grad[(j + 5) * N + i1] * dy) + L.grad[(j + 10) * N + i1] * dz);
                double dpv11 = 0.5 * ((L.grad[j * N + i2] * dx + L.grad[(j + 5) * N + i2] * dy) + L.grad[(j + 10) * N + i2] * dz);
                if (P.autoClip == 1) {
                    dpv1 = led(dpv1, L.bnd[j * N + i1], L.bnd[(j + 5) * N + i1], P.nsig);
                    dpv11 = -led(-dpv11, L.bnd[j * N + i2], L.bnd[(j + 5) * N + i2], P.nsig);
                }
                double aa = dpv1, bb = dpv11, cc;
                if (aa * bb <= 0.0) {
                    cc = 0.0;
                } else {
                    cc = fabs(aa) <= fabs(bb) ? aa : bb;
                    if (fabs(cc) > hlength && hlength > 0.0) cc = hlength * cc / fabs(cc);
                }
                dpvl[j] = cc;
            }
        }
        if ((roe1 + dpvl[0]) > 0.1) roe1 = roe1 + dpvl[0];
        u1 = u1 + dpvl[1]; v1 = v1 + dpvl[2]; w1 = w1 + dpvl[3];
        if ((re1 + dpvl[4]) > 0.0001) re1 = re1 + dpvl[4];
        pr1 = gam1 * (re1 - 0.5 * ((u1 * u1 + v1 * v1) + w1 * w1) * roe1);
        pr1 = dmax(pr1, 0.1);
        rh1 = re1 + pr1; rinv1 = 1 / roe1;
        ru1 = roe1 * u1; rv1 = roe1 * v1; rw1 = roe1 * w1;
        if ((roe2 - dpvl[0]) > 0.1) roe2 = roe2 - dpvl[0];
        u2 = u2 - dpvl[1]; v2 = v2 - dpvl[2]; w2 = w2 - dpvl[3];
        if ((re2 - dpvl[4]) > 0.0001) re2 = re2 - dpvl[4];
        pr2 = gam1 * (re2 - 0.5 * ((u2 * u2 + v2 * v2) + w2 * w2) * roe2);
        pr2 = dmax(pr2, 0.1);
        rh2 = re2 + pr2; rinv2 = 1 / roe2;
        ru2 = roe2 * u2; rv2 = roe2 * v2; rw2 = roe2 * w2;
    }
    double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
    double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
    const double beta0 = P.hllcBeta0;
    double rroe = sqrt(roe2 / roe1);
    double ut = (u1 + u2 * rroe) / (1 + rroe), vt = (v1 + v2 * rroe) / (1 + rroe);
    double wt = (w1 + w2 * rroe) / (1 + rroe);
    double qt = (ut * rnx + vt * rny) + wt * rnz;
    double ht = (rh1 * rinv1 + rh2 * rinv2 * rroe) / (1 + rroe);
    double ct = gam1 * (ht - 0.5 * ((ut * ut + vt * vt) + wt * wt));
    ct = sqrt(fabs(ct));
    double c1 = sqrt(gam1 * fabs(rh1 * rinv1 - 0.5 * ((u1 * u1 + v1 * v1) + w1 * w1)));
    double c2 = sqrt(gam1 * fabs(rh2 * rinv2 - 0.5 * ((u2 * u2 + v2 * v2) + w2 * w2)));
    double sl = dmin(nv1 - beta0 * c1, qt - ct);
    double sr = dmax(nv2 + beta0 * c2, qt + ct);
    sl = dmin(sl, nv2 - beta0 * c2);
    sr = dmax(sr, nv1 + beta0 * c1);
    double sm = roe2 * nv2 * (sr - nv2) - roe1 * nv1 * (sl - nv1);
    sm = (sm + pr1) - pr2;
    double fact = roe2 * (sr - nv2) - roe1 * (sl - nv1);
    if (fact != 0.0) fact = 1.0 / fact;
    sm = fact * sm;
    // the state of the GCL term: rho and E of the node with the
    // (reconstructed) momentum outside the star region, the star state
    // inside it (def_par:2046-2085)
    double q[5] = {r1, ru1, rv1, rw1, E1};
    if (sl > 0.0) {
        f[0] = ((rnx * ru1 + rny * rv1) + rnz * rw1) * rnorm1;
        f[1] = ((rnx * (ru1 * u1 + pr1) + rny * (ru1 * v1)) + rnz * (ru1 * w1)) * rnorm1;
        f[2] = ((rnx * (rv1 * u1) + rny * (rv1 * v1 + pr1)) + rnz * (rv1 * w1)) * rnorm1;
        f[3] = ((rnx * (rw1 * u1) + rny * (rw1 * v1)) + rnz * (rw1 * w1 + pr1)) * rnorm1;
        f[4] = ((rnx * (rh1 * u1) + rny * (rh1 * v1)) + rnz * (rh1 * w1)) * rnorm1;
    } else if (sl <= 0.0 && sm > 0.0) {
        double fl0 = (rnx * ru1 + rny * rv1) + rnz * rw1;
        double fl1 = (rnx * (ru1 * u1 + pr1) + rny * (ru1 * v1)) + rnz * (ru1 * w1);
        double fl2 = (rnx * (rv1 * u1) + rny * (rv1 * v1 + pr1)) + rnz * (rv1 * w1);
        double fl3 = (rnx * (rw1 * u1) + rny * (rw1 * v1)) + rnz * (rw1 * w1 + pr1);
        double fl4 = (rnx * (rh1 * u1) + rny * (rh1 * v1)) + rnz * (rh1 * w1);
        double pls = roe1 * (nv1 - sl) * (nv1 - sm) + pr1;
        double ls0, ls1, ls2, ls3, ls4;
        double factl = sl - sm;
        if (factl != 0.0) {
            factl = 1.0 / factl;
            ls0 = roe1 * (sl - nv1) * factl;
            ls1 = ((sl - nv1) * roe1 * u1 + (pls - pr1) * rnx) * factl;
            ls2 = ((sl - nv1) * roe1 * v1 + (pls - pr1) * rny) * factl;
            ls3 = ((sl - nv1) * roe1 * w1 + (pls - pr1) * rnz) * factl;
            ls4 = (((sl - nv1) * re1 - pr1 * nv1) + pls * sm) * factl;
        } else {
            ls0 = roe1; ls1 = ru1; ls2 = rv1; ls3 = rw1; ls4 = re1;
        }
        f[0] = (fl0 + sl * (ls0 - roe1)) * rnorm1;
        f[1] = (fl1 + sl * (ls1 - ru1)) * rnorm1;
        f[2] = (fl2 + sl * (ls2 - rv1)) * rnorm1;
        f[3] = (fl3 + sl * (ls3 - rw1)) * rnorm1;
        f[4] = (fl4 + sl * (ls4 - re1)) * rnorm1;
        q[0] = ls0; q[1] = ls1; q[2] = ls2; q[3] = ls3; q[4] = ls4;
    } else if (sm <= 0.0 && sr >= 0.0) {
        double fr0 = (rnx * ru2 + rny * rv2) + rnz * rw2;
        double fr1 = (rnx * (ru2 * u2 + pr2) + rny * (ru2 * v2)) + rnz * (ru2 * w2);
        double fr2 = (rnx * (rv2 * u2) + rny * (rv2 * v2 + pr2)) + rnz * (rv2 * w2);
        double fr3 = (rnx * (rw2 * u2) + rny * (rw2 * v2)) + rnz * (rw2 * w2 + pr2);
        double fr4 = (rnx * (rh2 * u2) + rny * (rh2 * v2)) + rnz * (rh2 * w2);
        double prs = roe2 * (nv2 - sr) * (nv2 - sm) + pr2;
        double rs0, rs1, rs2, rs3, rs4;
        double factr = sr - sm;
        if (factr != 0.0) {
            factr = 1.0 / factr;
            rs0 = roe2 * (sr - nv2) * factr;
            rs1 = ((sr - nv2) * roe2 * u2 + (prs - pr2) * rnx) * factr;
            rs2 = ((sr - nv2) * roe2 * v2 + (prs - pr2) * rny) * factr;
            rs3 = ((sr - nv2) * roe2 * w2 + (prs - pr2) * rnz) * factr;
            rs4 = (((sr - nv2) * re2 - pr2 * nv2) + prs * sm) * factr;
        } else {
            rs0 = roe2; rs1 = ru2; rs2 = rv2; rs3 = rw2; rs4 = re2;
        }
        f[0] = (fr0 + sr * (rs0 - roe2)) * rnorm1;
        f[1] = (fr1 + sr * (rs1 - ru2)) * rnorm1;
        f[2] = (fr2 + sr * (rs2 - rv2)) * rnorm1;
        f[3] = (fr3 + sr * (rs3 - rw2)) * rnorm1;
        f[4] = (fr4 + sr * (rs4 - re2)) * rnorm1;
        q[0] = rs0; q[1] = rs1; q[2] = rs2; q[3] = rs3; q[4] = rs4;
    } else if (sr < 0.0) {
        f[0] = ((rnx * ru2 + rny * rv2) + rnz * rw2) * rnorm1;
        f[1] = ((rnx * (ru2 * u2 + pr2) + rny * (ru2 * v2)) + rnz * (ru2 * w2)) * rnorm1;
        f[2] = ((rnx * (rv2 * u2) + rny * (rv2 * v2 + pr2)) + rnz * (rv2 * w2)) * rnorm1;
        f[3] = ((rnx * (rw2 * u2) + rny * (rw2 * v2)) + rnz * (rw2 * w2 + pr2)) * rnorm1;
        f[4] = ((rnx * (rh2 * u2) + rny * (rh2 * v2)) + rnz * (rh2 * w2)) * rnorm1;
        q[0] = r2; q[1] = ru2; q[2] = rv2; q[3] = rw2; q[4] = E2;
    }
    if (L.gclw)
        for (int k = 0; k < 5; ++k) f[k] = f[k] - q[k] * wgcl;
    }
}

// wall/symmetry own-state flux (def_par:2194-2230)
__device__ __forceinline__ void wall_flux(const NodeState &s, double rnx, double rny, double rnz, double *F) {
    double pr = s.p, rho = s.r, rinv = 1. / rho;
    double rh = s.E + pr;
    double uu = s.ru * rinv, vv = s.rv * rinv, ww = s.rw * rinv;
    double nv = (uu * rnx + vv * rny) + ww * rnz;
    F[0] = rho * nv;
    F[1] = pr * rnx + rho * uu * nv;
    F[2] = pr * rny + rho * vv * nv;
    F[3] = pr * rnz + rho * ww * nv;
    F[4] = rh * nv;
}

// Roe flux between a node state and the freestream (def_par:2268-2346)
__device__ __forceinline__ void farfield_flux(const Params &P, const NodeState &s, double rnx, double rny, double rnz,
                                              const double *inf, double *F) {
    const double gam1 = P.gm1;
    double ro = inf[0], ro1 = 1. / ro, uo = inf[1], vo = inf[2], wo = inf[3], eo = inf[4], po = inf[5];
    double prl = s.p, rhol = s.r, rinvl = 1. / rhol;
    double rhl = s.E + prl;
    double ul = s.ru * rinvl, vl = s.rv * rinvl, wl = s.rw * rinvl;
    double epsl = s.E, hl = rhl * rinvl;
    double nvl = (ul * rnx + vl * rny) + wl * rnz;
    double fl1 = rhol * nvl, fl2 = prl * rnx + rhol * ul * nvl, fl3 = prl * rny + rhol * vl * nvl;
    double fl4 = prl * rnz + rhol * wl * nvl, fl5 = rhl * nvl;
    double rhor = ro, uxr = uo, vyr = vo, wzr = wo, epsr = eo * ro, presr = po, hr = eo + po * ro1;
    double unr = (uxr * rnx + vyr * rny) + wzr * rnz;
    double fr1 = rhor * unr, fr2 = rnx * presr + rhor * uxr * unr, fr3 = rny * presr + rhor * vyr * unr;
    double fr4 = rnz * presr + rhor * wzr * unr, fr5 = (epsr + presr) * unr;
    double di = sqrt(rhor / rhol), d1 = 1.0 / (di + 1.0);
    double ui = (di * uxr + ul) * d1, vi = (di * vyr + vl) * d1, wi = (di * wzr + wl) * d1;
    double hi = (di * hr + hl) * d1;
    double ci2 = gam1 * (hi - 0.5 * ((ui * ui + vi * vi) + wi * wi));
    ci2 = dmax(ci2, 1.0e-5);
    double ci = sqrt(ci2);
    double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
    double ucp = (ui * rnx + vi * rny) + wi * rnz;
    double du1 = rhor - rhol, du2 = rhor * uxr - rhol * ul, du3 = rhor * vyr - rhol * vl;
    double du4 = rhor * wzr - rhol * wl, du5 = epsr - epsl;
    double l1 = fabs(ucp + ci), l2 = fabs(ucp - ci), l3 = fabs(ucp);
    double s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
    double al1x = gam1 * ((((af * du1 - ui * du2) - vi * du3) - wi * du4) + du5);
    double al2x = ((-ucp * du1 + du2 * rnx) + du3 * rny) + du4 * rnz;
    double cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci);
    double cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
    F[0] = 0.5 * (fr1 + fl1) - 0.5 * (l3 * du1 + cc1);
    F[1] = 0.5 * (fr2 + fl2) - 0.5 * ((l3 * du2 + cc1 * ui) + cc2 * rnx);
    F[2] = 0.5 * (fr3 + fl3) - 0.5 * ((l3 * du3 + cc1 * vi) + cc2 * rny);
    F[3] = 0.5 * (fr4 + fl4) - 0.5 * ((l3 * du4 + cc1 * wi) + cc2 * rnz);
    F[4] = 0.5 * (fr5 + fl5) - 0.5 * ((l3 * du5 + cc1 * hi) + cc2 * ucp);
}

// The flux of a node state through an engine face's coefficients
// (def_par:2448-2491)
__device__ __forceinline__ void engine_flux(const NodeState &s, double wx, double wy, double wz, double *F) {
    const double pr = s.p, r = s.r, rinv = 1. / s.r;
    const double uu = rinv * s.ru, vv = rinv * s.rv, ww = rinv * s.rw;
    const double pu = pr * rinv * s.ru, pv = pr * rinv * s.rv, pw = pr * rinv * s.rw;
    F[0] = (wx * r * uu + wy * r * vv) + wz * r * ww;
    F[1] = (wx * (s.ru * uu + pr) + wy * s.ru * vv) + wz * s.ru * ww;
    F[2] = (wx * s.rv * uu + wy * (s.rv * vv + pr)) + wz * s.rv * ww;
    F[3] = (wx * s.rw * uu + wy * s.rw * vv) + wz * (s.rw * ww + pr);
    F[4] = (wx * (s.E * uu + pu) + wy * (s.E * vv + pv)) + wz * (s.E * ww + pw);
}

// The GCL terms of boundary edge b of a moving mesh, subtracted from its
// two nodes' residuals before the edge's flux (def_par:2124-2177)
__device__ __forceinline__ void boundary_gcl(const Params &P, const LevelView &L, int b, double *t1, double *t2) {
    const int2 nd = L.bedge[b];
    const NodeState s1 = load_state(L, nd.x), s2 = load_state(L, nd.y);
    const double q1[5] = {s1.r, s1.ru, s1.rv, s1.rw, s1.E}, q2[5] = {s2.r, s2.ru, s2.rv, s2.rw, s2.E};
    const double w1 = L.bgclw[b], w2 = L.bgclw[L.B + b];
    for (int k = 0; k < 5; ++k) {
        if (P.boundaryTerm == 1) {
            t1[k] = (3. * q1[k] + q2[k]) * w1;
            t2[k] = (q1[k] + 3. * q2[k]) * w2;
        } else {
            t1[k] = q1[k] * w1;
            t2[k] = q2[k] * w2;
        }
    }
}

// Contributions g1 (to node 1) and g2 (to node 2) of boundary edge b
// (def_par:2182-2511)
__device__ __forceinline__ void boundary_flux(const Params &P, const LevelView &L, int b, double *g1, double *g2) {
    const int2 nd = L.bedge[b];
    const int ind = L.bind[b];
    const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
    for (int k = 0; k < 5; ++k) { g1[k] = 0.0; g2[k] = 0.0; }
    const NodeState s1 = load_state(L, nd.x), s2 = load_state(L, nd.y);
    const bool fe = P.boundaryTerm == 1;
    double F1[5], F2[5];
    if (ind <= 2 || ind == 9) {
        double rnorm = sqrt((wx * wx + wy * wy) + wz * wz);
        if (!(rnorm > 1.0e-10)) return;
        double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
        wall_flux(s1, rnx, rny, rnz, F1);
        wall_flux(s2, rnx, rny, rnz, F2);
    } else if (ind <= 4) {
        double rnorm = sqrt((wx * wx + wy * wy) + wz * wz);
        if (!(rnorm > 1.0e-10)) return;
        double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
        const double *inf = &P.inf[(ind - 3) * 6];
        farfield_flux(P, s1, rnx, rny, rnz, inf, F1);
        farfield_flux(P, s2, rnx, rny, rnz, inf, F2);
    } else {  // engine faces: the two fluxes' sum plus twice the node's own (def_par:2493-2505)
        engine_flux(s1, wx, wy, wz, F1);
        engine_flux(s2, wx, wy, wz, F2);
        for (int k = 0; k < 5; ++k) {
            const double fs = F1[k] + F2[k];
            g1[k] = fs + 2.0 * F1[k];
            g2[k] = fs + 2.0 * F2[k];
        }
        return;
    }
    const double rnorm = sqrt((wx * wx + wy * wy) + wz * wz);
    for (int k = 0; k < 5; ++k) {
        if (fe) {
            g1[k] = rnorm * (3. * F1[k] + F2[k]);
            g2[k] = rnorm * (F1[k] + 3. * F2[k]);
        } else {
            g1[k] = rnorm * 4. * F1[k];
            g2[k] = rnorm * 4. * F2[k];
        }
    }
}


// ---- the upwind extension on level 1 (no reference counterpart) -----------
// Roe flux of the MUSCL / Van Albada states of edge e (i1 -> i2), from the
// primitive and gradient records.  The states are (rho, u, v, w, rho E) with
// u = (rho u)/rho, reconstructed as
//     q_L = q1 + va(2 g1.d - dq, dq) / 2,  q_R = q2 - va(2 g2.d - dq, dq) / 2,
// d = x2 - x1, dq = q2 - q1; an edge whose reconstructed density or pressure
// is not positive takes the unreconstructed states.  p = (gamma-1)(rho E -
// rho |u|^2 / 2) of each state; the Roe average and wave strengths are those
// of the reference's Roe branch (def_par:1725-1792) with the dissipation
// added with the upwind sign.
__device__ __forceinline__ double prim_pressure(double gam1, const double *q) {
    return gam1 * (q[4] - 0.5 * ((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]) * q[0]);
}
__device__ __forceinline__ void edge_flux_muscl(const Params &P, const LevelView &L, int e, int i1, int i2,
                                                double *f) {
    const double gam1 = P.gm1;
    const PrimRec A = load_prim(L.qp, i1), B = load_prim(L.qp, i2);
    const double dx = B.x - A.x, dy = B.y - A.y, dz = B.z - A.z;
    const double q1[5] = {A.r, A.u, A.v, A.w, A.E}, q2[5] = {B.r, B.u, B.v, B.w, B.E};
    // g.d at each end, one gradient record (eight 16-byte loads) at a time
    double g1[5], g2[5];
    {
        const GradRec G = load_rec<GradRec, 8>(L.gq, i1);
#pragma unroll
        for (int j = 0; j < 5; ++j) g1[j] = (G.g[3 * j] * dx + G.g[3 * j + 1] * dy) + G.g[3 * j + 2] * dz;
    }
    {
        const GradRec G = load_rec<GradRec, 8>(L.gq, i2);
#pragma unroll
        for (int j = 0; j < 5; ++j) g2[j] = (G.g[3 * j] * dx + G.g[3 * j + 1] * dy) + G.g[3 * j + 2] * dz;
    }
    double qa[5], qb[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const double dq = q2[j] - q1[j];
        qa[j] = q1[j] + 0.5 * van_albada(2.0 * g1[j] - dq, dq);
        qb[j] = q2[j] - 0.5 * van_albada(2.0 * g2[j] - dq, dq);
    }
    double pa = prim_pressure(gam1, qa), pb = prim_pressure(gam1, qb);
    if (!(qa[0] > 0.0 && qb[0] > 0.0 && pa > 0.0 && pb > 0.0)) {
#pragma unroll
        for (int j = 0; j < 5; ++j) { qa[j] = q1[j]; qb[j] = q2[j]; }
        pa = prim_pressure(gam1, qa);
        pb = prim_pressure(gam1, qb);
    }
    f[0] = f[1] = f[2] = f[3] = f[4] = 0.0;
    const EdgeW w = load_edgew(L.ew, e);
    const double rnorm = sqrt((w.wx * w.wx + w.wy * w.wy) + w.wz * w.wz);
    if (!(rnorm > 1.0e-10)) return;
    const double rn = 1.0 / rnorm;
    const double rnx = w.wx * rn, rny = w.wy * rn, rnz = w.wz * rn;
    const double r1 = qa[0], u1 = qa[1], v1 = qa[2], w1 = qa[3], E1 = qa[4];
    const double r2 = qb[0], u2 = qb[1], v2 = qb[2], w2 = qb[3], E2 = qb[4];
    const double ru1 = r1 * u1, rv1 = r1 * v1, rw1 = r1 * w1, rh1 = E1 + pa;
    const double ru2 = r2 * u2, rv2 = r2 * v2, rw2 = r2 * w2, rh2 = E2 + pb;
    const double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
    const double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
    const double h1 = rh1 / r1, h2 = rh2 / r2;
    const double di = sqrt(r1 / r2), d1 = 1.0 / (di + 1.0);
    const double ui = (di * u1 + u2) * d1, vi = (di * v1 + v2) * d1, wi = (di * w1 + w2) * d1;
    const double hi = (di * h1 + h2) * d1;
    const double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
    const double ci2 = dmax(gam1 * (hi - af), 1.0e-5);
    const double ci = sqrt(ci2), ici = 1.0 / ci, ici2 = 1.0 / ci2;
    const double ucp = (ui * rnx + vi * rny) + wi * rnz;
    const double du1 = r2 - r1, du2 = ru2 - ru1, du3 = rv2 - rv1, du4 = rw2 - rw1, du5 = E2 - E1;
    const double l1 = fabs(ucp + ci), l2 = fabs(ucp - ci), l3 = fabs(ucp);
    const double s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
    const double al1x = gam1 * ((((af * du1 - ui * du2) - vi * du3) - wi * du4) + du5);
    const double al2x = ((-ucp * du1 + du2 * rnx) + du3 * rny) + du4 * rnz;
    const double cc1 = (s1 - l3) * al1x * ici2 + s2 * al2x * ici;
    const double cc2 = s2 * al1x * ici + (s1 - l3) * al2x;
    f[0] = rnorm * ((r1 * nv1 + r2 * nv2) - (l3 * du1 + cc1));
    f[1] = rnorm * (((pa * rnx + ru1 * nv1) + (pb * rnx + ru2 * nv2)) - ((l3 * du2 + cc1 * ui) + cc2 * rnx));
    f[2] = rnorm * (((pa * rny + rv1 * nv1) + (pb * rny + rv2 * nv2)) - ((l3 * du3 + cc1 * vi) + cc2 * rny));
    f[3] = rnorm * (((pa * rnz + rw1 * nv1) + (pb * rnz + rw2 * nv2)) - ((l3 * du4 + cc1 * wi) + cc2 * rnz));
    f[4] = rnorm * ((rh1 * nv1 + rh2 * nv2) - ((l3 * du5 + cc1 * hi) + cc2 * ucp));
}

}  // namespace flite

// Device helpers of the discrete adjoint shared by the residual product
// (adjoint.cu) and the steady adjoint solve (steady_adjoint.cu): dual
// numbers, the far-field Roe flux on dual numbers, the pressure gradient and
// the transposed flux Jacobian of the central and wall fluxes.
#pragma once
#include "device.cuh"

namespace flite {

struct Dual {
    double v, d;
    __device__ Dual() : v(0), d(0) {}
    __device__ Dual(double a) : v(a), d(0) {}
    __device__ Dual(double a, double b) : v(a), d(b) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    double s = sqrt(a.v);
    return Dual(s, s > 0 ? 0.5 * a.d / s : 0.0);
}
__device__ __forceinline__ Dual dfabs(Dual a) { return a.v < 0 ? -a : a; }
__device__ __forceinline__ Dual dmaxc(Dual a, double c) { return (a.v < c) ? Dual(c) : a; }

// far-field Roe flux of def_par:2268-2346 on the left (node) state
__device__ __forceinline__ void farfield_dual(const Params &P, const Dual *q, Dual pr, double rnx, double rny, double rnz,
                              const double *inf, Dual *F) {
    const double gam1 = P.gm1;
    double ro = inf[0], ro1 = 1. / ro, uo = inf[1], vo = inf[2], wo = inf[3], eo = inf[4], po = inf[5];
    Dual rhol = q[0], rinvl = Dual(1.0) / rhol;
    Dual rhl = q[4] + pr;
    Dual ul = q[1] * rinvl, vl = q[2] * rinvl, wl = q[3] * rinvl;
    Dual epsl = q[4], hl = rhl * rinvl;
    Dual nvl = (ul * rnx + vl * rny) + wl * rnz;
    Dual fl1 = rhol * nvl, fl2 = pr * rnx + rhol * ul * nvl, fl3 = pr * rny + rhol * vl * nvl;
    Dual fl4 = pr * rnz + rhol * wl * nvl, fl5 = rhl * nvl;
    double rhor = ro, uxr = uo, vyr = vo, wzr = wo, epsr = eo * ro, presr = po, hr = eo + po * ro1;
    double unr = (uxr * rnx + vyr * rny) + wzr * rnz;
    double fr1 = rhor * unr, fr2 = rnx * presr + rhor * uxr * unr, fr3 = rny * presr + rhor * vyr * unr;
    double fr4 = rnz * presr + rhor * wzr * unr, fr5 = (epsr + presr) * unr;
    Dual di = dsqrt(Dual(rhor) / rhol), d1 = Dual(1.0) / (di + Dual(1.0));
    Dual ui = (di * uxr + ul) * d1, vi = (di * vyr + vl) * d1, wi = (di * wzr + wl) * d1;
    Dual hi = (di * hr + hl) * d1;
    Dual ci2 = Dual(gam1) * (hi - Dual(0.5) * ((ui * ui + vi * vi) + wi * wi));
    ci2 = dmaxc(ci2, 1.0e-5);
    Dual ci = dsqrt(ci2);
    Dual af = Dual(0.5) * ((ui * ui + vi * vi) + wi * wi);
    Dual ucp = (ui * rnx + vi * rny) + wi * rnz;
    Dual du1 = Dual(rhor) - rhol, du2 = Dual(rhor * uxr) - rhol * ul, du3 = Dual(rhor * vyr) - rhol * vl;
    Dual du4 = Dual(rhor * wzr) - rhol * wl, du5 = Dual(epsr) - epsl;
    Dual l1 = dfabs(ucp + ci), l2 = dfabs(ucp - ci), l3 = dfabs(ucp);
    Dual s1 = Dual(0.5) * (l1 + l2), s2 = Dual(0.5) * (l1 - l2);
    Dual al1x = Dual(gam1) * ((((af * du1 - ui * du2) - vi * du3) - wi * du4) + du5);
    Dual al2x = ((-ucp * du1 + du2 * rnx) + du3 * rny) + du4 * rnz;
    Dual cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci);
    Dual cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
    F[0] = Dual(0.5) * (Dual(fr1) + fl1) - Dual(0.5) * (l3 * du1 + cc1);
    F[1] = Dual(0.5) * (Dual(fr2) + fl2) - Dual(0.5) * ((l3 * du2 + cc1 * ui) + cc2 * rnx);
    F[2] = Dual(0.5) * (Dual(fr3) + fl3) - Dual(0.5) * ((l3 * du3 + cc1 * vi) + cc2 * rny);
    F[3] = Dual(0.5) * (Dual(fr4) + fl4) - Dual(0.5) * ((l3 * du4 + cc1 * wi) + cc2 * rnz);
    F[4] = Dual(0.5) * (Dual(fr5) + fl5) - Dual(0.5) * ((l3 * du5 + cc1 * hi) + cc2 * ucp);
}

// pressure and its gradient wrt the conserved state (0 under the floor)
__device__ __forceinline__ void pressure_grad(const Params &P, const double *u, double *p, double *dp) {
    double r = u[0], m1 = u[1], m2 = u[2], m3 = u[3], E = u[4];
    double q = (m1 * m1 + m2 * m2) + m3 * m3;
    double pp = P.gm1 * (E - 0.5 * q / r);
    if (pp < 0.1) {
        *p = 0.1;
        for (int k = 0; k < 5; ++k) dp[k] = 0.0;
        return;
    }
    *p = pp;
    dp[0] = P.gm1 * 0.5 * q / (r * r);
    dp[1] = -P.gm1 * m1 / r;
    dp[2] = -P.gm1 * m2 / r;
    dp[3] = -P.gm1 * m3 / r;
    dp[4] = P.gm1;
}

// A_d(u)^T b accumulated into ubar for the three directions d
__device__ __forceinline__ void apply_flux_jacobian_t(const Params &P, const double *u, const double b[3][5],
                                                      double *ub) {
    double p, dp[5];
    pressure_grad(P, u, &p, dp);
    const double r = u[0], E = u[4];
    const double m[3] = {u[1], u[2], u[3]};
    for (int k = 0; k < 5; ++k) ub[k] = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double *a = b[d];
        const double md = m[d];
        // F_0 = m_d; F_{1+c} = m_c m_d / r + p [c==d]; F_4 = (E+p) m_d / r
        double pbar = a[1 + d] + a[4] * md / r;
        double rbar = 0.0, mbar[3] = {0, 0, 0}, Ebar = a[4] * md / r;
        double s = a[0] + a[4] * (E + p) / r;  // d/dm_d of the parts linear in m_d
        for (int c = 0; c < 3; ++c) {
            rbar -= a[1 + c] * m[c] * md / (r * r);
            mbar[c] += a[1 + c] * md / r;
            s += a[1 + c] * m[c] / r;
        }
        rbar -= a[4] * (E + p) * md / (r * r);
        mbar[d] += s;
        ub[0] += rbar + pbar * dp[0];
        ub[1] += mbar[0] + pbar * dp[1];
        ub[2] += mbar[1] + pbar * dp[2];
        ub[3] += mbar[2] + pbar * dp[3];
        ub[4] += Ebar + pbar * dp[4];
    }
}

}  // namespace flite

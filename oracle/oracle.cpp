// CPU restatement of the reference flow solver -- test infrastructure only.
//
// Every routine below restates the Fortran routine cited beside it, in the
// same operation order: the same edge-order scatter, left-to-right
// evaluation of every expression, and no fused multiply-add (this file is
// compiled with -ffp-contract=off).  The shared nodeHelpArray of the
// reference (one array for all levels, def_par:14231) is kept shared here
// too, so any state that would leak between levels in the reference leaks
// the same way here.
//
// Pinned choices where the reference reads undefined values:
//  * Roe and LLF read rho1/rho2/h1/h2 that the interior loop never sets
//    (def_par:1682,1693,1738,1748,1760): rho = r and h = (E+p)/rho.
//  * LLF/Roe leave f unchanged when |w| <= 1e-10 (def_par:1672,1727),
//    i.e. the previous edge's flux is added again: pinned to f = 0.
//  * nullifyOuterBoundary declares its own uninitialised ivd (def_par:4259):
//    a no-op for turbulenceModel 0, components 1..6 zeroed for SA.
//  * numberOfIONodes is never set (makeIORegister is commented out,
//    mg_par:1248,1262): pinned to 0.
//  * coarse-level coordinates are allocated but never filled
//    (def_par:14002-14011,14071): pinned to 0.
//  * the cycle number of a coarse level before its first relaxation is 0.
//  * the LED limiter's (1+t^nsig)^(1/nsig) (def_par:1861) is evaluated as
//    sqrt(sqrt(1+(t*t)*(t*t))) for nsig=4 and sqrt(1+t*t) for nsig=2.
//  * the engine mass-flow factor of an inlet whose flow sum is not positive
//    is an uninitialised local (def_par:4593-4598, 4779-4806): pinned to 1.
//    The sums over the engine inlet sides follow the device's fixed order
//    (engine_sums) in place of the reference's side order.
#include "oracle.h"
#include "pinned_math.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using vec = std::vector<double>;

struct Level {
    int N = 0, E = 0, B = 0, Nb = 0, nnorm = 0, grid = 1;
    std::vector<int> s1, s2;  // 0-based
    vec wx, wy, wz, slen;
    std::vector<int> b1, b2, bind;
    vec bwx, bwy, bwz;
    int reg[21];
    std::vector<int> node_ind;  // 0-based node numbers
    vec V, wdist, cx, cy, cz, cmx, cmy, cmz;
    // moving meshes (flowType 2): GCLWeightsArray of the sides and of the
    // boundary sides' two nodes as the reader leaves them (combined for
    // timeScheme 2 on level 1), and the previous volumes (level 1)
    vec gcl, bgcl1, bgcl2, Vp, Vp2;
    std::vector<int> parent;  // [N_finer], 0-based coarse node or -1
    vec rweight;
    // engine inlet sides: 0-based nodes, inlet 0|1, coefficients
    std::vector<int> e1, e2, ein;
    vec ewx, ewy, ewz;
    // state
    vec u[6], uprev[6], rhs[6], src[6], diss[5];
    vec uold[6], uold2[6];  // unsteady runs: previous physical time steps
    vec p, dt, mu, conn, wallArea, nx, ny, nz, wallStress[3];
    // Spalart-Allmaras: turbulenceDiffusionTerm, localTurbulentTimeSteps,
    // vorticity and divergence of the viscous routine
    vec turbDiff, dtT, vort, divg;
    int cycleNumber = 0;
    int R(int i) const { return reg[i + 20]; }  // nodeIndicatorRegister(i)
    // colouring of edge blocks for the threaded timing mode (built on first
    // use): blocks of colour k are cord[cptr[k] .. cptr[k+1])
    std::vector<int> cptr, cord, bcptr, bcord;
};

// Threads of the timing mode.  1 (the default) runs every loop in the
// reference's order; more threads run each edge loop colour by colour in
// parallel, which changes the order of the sums at a node (results then
// differ in the last bits) but not the algorithm.  Used only to time the
// CPU baseline on all host cores.
int g_threads = 1;

// Edges are grouped in blocks of consecutive edges (kept in the
// reference's order inside a block, for locality), and the blocks coloured
// greedily so that no two blocks of a colour share a node.
constexpr int kEdgeBlock = 2048;

void colour_blocks(int n, const int *a, const int *b, int nnodes, std::vector<int> &cptr,
                   std::vector<int> &cord) {
    const int nb = (n + kEdgeBlock - 1) / kEdgeBlock;
    std::vector<uint64_t> mask(nnodes, 0);
    std::vector<int> col(nb, 0);
    int ncol = 0;
    for (int q = 0; q < nb; ++q) {
        const int e0 = q * kEdgeBlock, e1 = std::min(n, e0 + kEdgeBlock);
        uint64_t m = 0;
        for (int e = e0; e < e1; ++e) m |= mask[a[e]] | mask[b[e]];
        int k = 0;
        while (k < 64 && (m >> k & 1)) ++k;
        if (k == 64) {  // too many colours: one block per colour from here
            k = ncol;
        } else {
            for (int e = e0; e < e1; ++e) {
                mask[a[e]] |= uint64_t(1) << k;
                mask[b[e]] |= uint64_t(1) << k;
            }
        }
        col[q] = k;
        ncol = std::max(ncol, k + 1);
    }
    cptr.assign(ncol + 1, 0);
    for (int q = 0; q < nb; ++q) ++cptr[col[q] + 1];
    for (int k = 0; k < ncol; ++k) cptr[k + 1] += cptr[k];
    cord.resize(nb);
    std::vector<int> at(cptr.begin(), cptr.end() - 1);
    for (int q = 0; q < nb; ++q) cord[at[col[q]]++] = q;
}

template <class F>
void for_blocks(int n, const std::vector<int> &cptr, const std::vector<int> &cord, F &&f) {
    const int ncol = (int)cptr.size() - 1;
    for (int k = 0; k < ncol; ++k) {
        const int a = cptr[k], b = cptr[k + 1];
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
        for (int q = a; q < b; ++q) {
            const int e0 = cord[q] * kEdgeBlock, e1 = std::min(n, e0 + kEdgeBlock);
            for (int e = e0; e < e1; ++e) f(e);
        }
    }
}

template <class F>
void for_edges(Level &g, F &&f) {
    if (g_threads <= 1) {
        for (int e = 0; e < g.E; ++e) f(e);
        return;
    }
    if (g.cptr.empty()) colour_blocks(g.E, g.s1.data(), g.s2.data(), g.N, g.cptr, g.cord);
    for_blocks(g.E, g.cptr, g.cord, f);
}

// boundary edges, likewise
template <class F>
void for_bedges(Level &g, F &&f) {
    if (g_threads <= 1) {
        for (int b = 0; b < g.B; ++b) f(b);
        return;
    }
    if (g.bcptr.empty()) colour_blocks(g.B, g.b1.data(), g.b2.data(), g.N, g.bcptr, g.bcord);
    for_blocks(g.B, g.bcptr, g.bcord, f);
}

template <class F>
void for_nodes(int n, F &&f) {
    if (g_threads <= 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int i = 0; i < n; ++i) f(i);
}

// the Van Albada limited slope of the upwind-biased difference a and the
// edge difference b (an extension, no reference counterpart)
static inline double van_albada(double a, double b) {
    const double ab = a * b;
    if (ab <= 0.0) return 0.0;
    return (ab * (a + b)) / (a * a + b * b);
}

struct Oracle {
    flite_controls c;
    std::vector<Level> lv;
    int nvar = 5;
    bool engines = false;
    // ivd%physicalTimeStep: the control's value, and under explicit time
    // stepping the smallest local time step of the last makeTimeSteps
    // (def_par:13598-13607), whichever level it ran on
    double pts_global = 0.0;  // the mesh has engine faces or nodes (indicators 5..8)
    std::vector<vec> nh;  // nodeHelpArray(:,1:25), sized for level 1
    double RK[5] = {0.6, 0.6, 1.0, 0.0, 0.0};  // def_par:14240-14244
    int nstage = 3;
    // the five-stage extension (no reference counterpart)
    void set_stages(int n) {
        nstage = n;
        if (n == 5) {
            RK[0] = 0.25; RK[1] = 1. / 6.; RK[2] = 0.375; RK[3] = 0.5; RK[4] = 1.0;
        }
    }

    // ---- makePressureField (def_par:13612-13630) --------------------------
    void makePressureField(Level &g, vec *u) {
        const double gm1 = c.gamma - 1.0;
        for_nodes(g.N, [&](int i) {
            double pp = gm1 * (u[4][i] - 0.5 * ((u[1][i] * u[1][i] + u[2][i] * u[2][i]) + u[3][i] * u[3][i]) / u[0][i]);
            g.p[i] = std::max(pp, 0.1);
        });
    }

    // ---- makeTimeSteps (def_par:13335-13610) ------------------------------
    void makeTimeSteps(Level &g) {
        const double c1 = c.gamma;
        vec &h1 = nh[0];
        for (int i = 0; i < g.N; ++i) { g.dt[i] = 0.0; }
        std::fill(h1.begin(), h1.end(), 0.0);
        const bool visc = c.ReynoldsNumber > 0.0;
        const double am = 1.0 / c.ReynoldsNumber;
        auto visc_of = [&](int i) {
            if (c.turbulenceModel == 1) return g.mu[i] + g.u[5][i] / c.ReynoldsNumber;
            return g.mu[i];
        };
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
            double al = (wx * wx + wy * wy) + wz * wz;
            double ro1 = 1. / g.u[0][i1], ro2 = 1. / g.u[0][i2];
            double cc1 = std::max(c1 * g.p[i1] * ro1, 0.001);
            double cc2 = std::max(c1 * g.p[i2] * ro2, 0.001);
            double vn1 = ((wx * g.u[1][i1] + wy * g.u[2][i1]) + wz * g.u[3][i1]) * ro1;
            double vn2 = ((wx * g.u[1][i2] + wy * g.u[2][i2]) + wz * g.u[3][i2]) * ro2;
            g.dt[i1] = (g.dt[i1] + std::fabs(vn1)) + std::sqrt(cc1 * al);
            g.dt[i2] = (g.dt[i2] + std::fabs(vn2)) + std::sqrt(cc2 * al);
            if (visc) {
                double vis1 = std::max(am, visc_of(i1)), vis2 = std::max(am, visc_of(i2));
                double dv1 = 2.0 * vis1 * al / g.u[0][i1];
                double dv2 = 2.0 * vis2 * al / g.u[0][i2];
                h1[i1] = h1[i1] + dv2;
                h1[i2] = h1[i2] + dv1;
            }
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double wx = g.bwx[b], wy = g.bwy[b], wz = g.bwz[b];
            double al = (wx * wx + wy * wy) + wz * wz;
            double ro1 = 1. / g.u[0][i1], ro2 = 1. / g.u[0][i2];
            double cc1 = std::max(c1 * g.p[i1] * ro1, 0.001);
            double cc2 = std::max(c1 * g.p[i2] * ro2, 0.001);
            double vn1 = ((wx * g.u[1][i1] + wy * g.u[2][i1]) + wz * g.u[3][i1]) * ro1;
            double vn2 = ((wx * g.u[1][i2] + wy * g.u[2][i2]) + wz * g.u[3][i2]) * ro2;
            vn1 = std::fabs(vn1); vn2 = std::fabs(vn2);
            double vnm = vn1 + vn2;
            cc1 = std::sqrt(cc1 * al); cc2 = std::sqrt(cc2 * al);
            double ccm = cc1 + cc2;
            g.dt[i1] = (((g.dt[i1] + vn1) + vnm) + cc1) + ccm;
            g.dt[i2] = (((g.dt[i2] + vn2) + vnm) + cc2) + ccm;
            if (visc) {
                double vis1 = std::max(am, visc_of(i1)), vis2 = std::max(am, visc_of(i2));
                double dv1 = 2.0 * vis1 * al / g.u[0][i1];
                double dv2 = 2.0 * vis2 * al / g.u[0][i2];
                double dvm = dv1 + dv2;
                h1[i1] = (h1[i1] + dv1) + dvm;
                h1[i2] = (h1[i2] + dv2) + dvm;
            }
        });
        for_nodes(g.N, [&](int i) { g.dt[i] = 0.5 / (g.dt[i] / g.V[i] + h1[i] / (g.V[i] * g.V[i])); });
        if (c.explicit_) {
            double minVal = 9999999.9;
            for (int i = 0; i < g.N; ++i)
                if (g.dt[i] < minVal) minVal = g.dt[i];
            pts_global = minVal;
        }
    }

    // ---- makeArtificialDissipation2, scalar form (def_par:11484-11993) ----
    void makeArtificialDissipation2(Level &g) {
        for (int k = 0; k < 5; ++k) std::fill(g.diss[k].begin(), g.diss[k].end(), 0.0);
        for (auto &col : nh) std::fill(col.begin(), col.end(), 0.0);
        if (c.fluxType == 4 && g.grid == 1) return;
        if (c.fourthOrderDissipationFactor == 0 && c.secondOrderDissipationFactor == 0) return;
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double d[5];
            for (int k = 0; k < 4; ++k) d[k] = g.u[k][i1] - g.u[k][i2];
            d[4] = ((g.u[4][i1] - g.u[4][i2]) + g.p[i1]) - g.p[i2];
            double df = 1.0;
            if (c.useDissipationWeighting) df = 1. / g.slen[e];
            for (int k = 0; k < 5; ++k) {
                nh[k][i1] = nh[k][i1] - d[k] * df;
                nh[k][i2] = nh[k][i2] + d[k] * df;
            }
            nh[5][i1] = nh[5][i1] + df;
            nh[5][i2] = nh[5][i2] + df;
        });
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double dp = g.p[i1] - g.p[i2], sp = g.p[i1] + g.p[i2];
            nh[6][i1] = nh[6][i1] - dp;
            nh[7][i1] = nh[7][i1] + sp;
            nh[6][i2] = nh[6][i2] + dp;
            nh[7][i2] = nh[7][i2] + sp;
        });
        for_nodes(g.N, [&](int i) {
            double fact = 1. / g.conn[i];
            nh[8][i] = 12. * std::fabs(nh[6][i] / nh[7][i]);
            for (int k = 0; k < 5; ++k) nh[k][i] = fact * nh[k][i];
        });
        const double k2 = c.secondOrderDissipationFactor;
        const double k4 = g.grid == 1 ? c.fourthOrderDissipationFactor : c.coarseGridDissipationFactor;
        const bool matrix = c.useMatrixDissipation != 0;
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double d4v[5], d2v[5];
            for (int k = 0; k < 5; ++k) d4v[k] = nh[k][i1] - nh[k][i2];
            for (int k = 0; k < 5; ++k) d2v[k] = g.u[k][i1] - g.u[k][i2];
            double d2, d4;
            if (!matrix) {
                double d0 = std::min(g.V[i1] / g.dt[i1], g.V[i2] / g.dt[i2]) / (g.conn[i1] + g.conn[i2]);
                d2 = d0 * k2 * std::max(nh[8][i1], nh[8][i2]);
                d4 = d0 * k4;
            } else {
                matrix_dissipation(g, e, i1, i2, d4v, d2v);
                d2 = k2 * std::max(nh[8][i1], nh[8][i2]);
                d4 = k4;
            }
            d4 = d4 > d2 ? d4 - d2 : 0.0;  // dim(d4,d2)
            for (int k = 0; k < 5; ++k) {
                g.diss[k][i1] = (g.diss[k][i1] - d4v[k] * d4) + d2v[k] * d2;
                g.diss[k][i2] = (g.diss[k][i2] + d4v[k] * d4) - d2v[k] * d2;
            }
        });
    }

    // ---- the matrix variant of makeArtificialDissipation2 (def_par:11814-
    // 11898): the one-dimensional Roe matrix |A| along the edge, with
    // Harten's correction of small eigenvalues, applied to the Laplacian
    // differences d4v and the state differences d2v (both i1 - i2)
    void matrix_dissipation(const Level &g, int e, int i1, int i2, double *d4v, double *d2v) {
        const double H = c.HartensCorrectionFactor;
        const double eps1 = 1. / std::max(H, 1.e-5), gam1 = c.gamma - 1.;
        double rnx = g.wx[e], rny = g.wy[e], rnz = g.wz[e];
        const double al = std::sqrt((rnx * rnx + rny * rny) + rnz * rnz);
        const double vmo1 = 1. / al;
        rnx = rnx * vmo1; rny = rny * vmo1; rnz = rnz * vmo1;
        const double rhol = g.u[0][i1];
        double rho1 = 1. / rhol;
        const double uxl = g.u[1][i1] * rho1, vyl = g.u[2][i1] * rho1, wzl = g.u[3][i1] * rho1;
        const double hl = (g.u[4][i1] + g.p[i1]) * rho1;
        const double rhor = g.u[0][i2];
        rho1 = 1. / rhor;
        const double uxr = g.u[1][i2] * rho1, vyr = g.u[2][i2] * rho1, wzr = g.u[3][i2] * rho1;
        const double hr = (g.u[4][i2] + g.p[i2]) * rho1;
        const double di = std::sqrt(rhor / rhol), d1 = 1.0 / (di + 1.0);
        const double ui = (di * uxr + uxl) * d1, vi = (di * vyr + vyl) * d1, wi = (di * wzr + wzl) * d1;
        const double hi = (di * hr + hl) * d1;
        const double ci2 = gam1 * (hi - 0.5 * ((ui * ui + vi * vi) + wi * wi));
        const double ci = std::sqrt(ci2);
        const double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
        const double ucp = (ui * rnx + vi * rny) + wi * rnz;
        double l1 = std::fabs(ucp + ci), l2 = std::fabs(ucp - ci), l3 = std::fabs(ucp);
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

    // ---- makeArtificialDissipation1 (def_par:10706-11482): the linearity-
    // preserving dissipation of Crumpton et al. on level 1.  Help columns
    // (0-based): 0-14 the gradient sums of (rho, rho u, rho v, rho w, rho E)
    // in x, y, z; 15-19 L(U), then L^(U); 20 the sum of the edge factors;
    // 21-23 L(x).  The far-field zeroing of the reference's columns 9-12 (def_par:11120-
    // 11126) touches columns that are not read again.
    void makeArtificialDissipation1(Level &g) {
        for (int k = 0; k < 5; ++k) std::fill(g.diss[k].begin(), g.diss[k].end(), 0.0);
        for (auto &col : nh) std::fill(col.begin(), col.end(), 0.0);
        for_edges(g, [&](int e) {
            const int i1 = g.s1[e], i2 = g.s2[e];
            const double w[3] = {g.wx[e], g.wy[e], g.wz[e]};
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 5; ++k) {
                    const double sv = (g.u[k][i1] + g.u[k][i2]) * w[a];
                    nh[5 * a + k][i1] = nh[5 * a + k][i1] + sv;
                    nh[5 * a + k][i2] = nh[5 * a + k][i2] - sv;
                }
            double df = 1.0;
            if (c.useDissipationWeighting) df = 1. / g.slen[e];
            for (int k = 0; k < 5; ++k) {
                const double d = g.u[k][i1] - g.u[k][i2];
                nh[15 + k][i1] = nh[15 + k][i1] - d * df;
                nh[15 + k][i2] = nh[15 + k][i2] + d * df;
            }
            nh[20][i1] = nh[20][i1] + df;
            nh[20][i2] = nh[20][i2] + df;
            const double dx[3] = {g.cx[i1] - g.cx[i2], g.cy[i1] - g.cy[i2], g.cz[i1] - g.cz[i2]};
            for (int a = 0; a < 3; ++a) {
                nh[21 + a][i1] = nh[21 + a][i1] - dx[a] * df;
                nh[21 + a][i2] = nh[21 + a][i2] + dx[a] * df;
            }
        });
        // boundary faces; with boundaryTerm != 1 the second node's term
        // carries no state (4 w, def_par:10974-10988), restated as is
        for_bedges(g, [&](int b) {
            const int i1 = g.b1[b], i2 = g.b2[b];
            const double w[3] = {g.bwx[b], g.bwy[b], g.bwz[b]};
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 5; ++k) {
                    const double q1 = g.u[k][i1], q2 = g.u[k][i2];
                    if (c.boundaryTerm == 1) {
                        nh[5 * a + k][i1] = nh[5 * a + k][i1] + (3. * q1 + q2) * w[a];
                        nh[5 * a + k][i2] = nh[5 * a + k][i2] + (q1 + 3. * q2) * w[a];
                    } else {
                        nh[5 * a + k][i1] = nh[5 * a + k][i1] + 4. * q1 * w[a];
                        nh[5 * a + k][i2] = nh[5 * a + k][i2] + 4. * w[a];
                    }
                }
        });
        if (c.useDissipationWeighting)
            for (int i = 0; i < g.N; ++i) nh[20][i] = 3.0 * nh[20][i];
        for (int i = 0; i < g.N; ++i) {
            const double vt = 1. / g.V[i];
            for (int k = 0; k < 15; ++k) nh[k][i] = nh[k][i] * vt;
        }
        for (int i = 0; i < g.Nb; ++i) nh[21][i] = nh[22][i] = nh[23][i] = 0.0;
        for (int i = 0; i < g.N; ++i)
            for (int k = 0; k < 5; ++k)
                nh[15 + k][i] = ((nh[15 + k][i] + nh[k][i] * nh[21][i]) + nh[5 + k][i] * nh[22][i]) +
                                nh[10 + k][i] * nh[23][i];
        // pressure switch
        std::fill(nh[0].begin(), nh[0].end(), 0.0);
        std::fill(nh[1].begin(), nh[1].end(), 0.0);
        for_edges(g, [&](int e) {
            const int i1 = g.s1[e], i2 = g.s2[e];
            const double dp = g.p[i1] - g.p[i2], sp = g.p[i1] + g.p[i2];
            nh[0][i1] = nh[0][i1] - dp;
            nh[1][i1] = nh[1][i1] + sp;
            nh[0][i2] = nh[0][i2] + dp;
            nh[1][i2] = nh[1][i2] + sp;
        });
        for (int i = 0; i < g.N; ++i) nh[8][i] = 12. * std::fabs(nh[0][i] / nh[1][i]);
        const double k2 = c.secondOrderDissipationFactor, k4 = c.fourthOrderDissipationFactor;
        for_edges(g, [&](int e) {
            const int i1 = g.s1[e], i2 = g.s2[e];
            double d4v[5], d2v[5];
            for (int k = 0; k < 5; ++k) d4v[k] = nh[15 + k][i1] - nh[15 + k][i2];
            for (int k = 0; k < 5; ++k) d2v[k] = g.u[k][i1] - g.u[k][i2];
            double d2, d4, d41, d42;
            // the branches as the reference orders them: the scalar
            // coefficient under useMatrixDissipation, the matrix otherwise
            if (c.useMatrixDissipation) {
                const double d0 = std::min(g.V[i1] / g.dt[i1], g.V[i2] / g.dt[i2]) / (g.conn[i1] + g.conn[i2]);
                d2 = d0 * k2 * std::max(nh[8][i1], nh[8][i2]);
                d4 = d0 * k4;
                d4 = d4 > d2 ? d4 - d2 : 0.0;
                d41 = d4 / nh[20][i1];
                d42 = d4 / nh[20][i2];
            } else {
                matrix_dissipation(g, e, i1, i2, d4v, d2v);
                d2 = k2 * std::max(nh[8][i1], nh[8][i2]);
                d4 = k4;
                d4 = d4 > d2 ? d4 - d2 : 0.0;
                d41 = d42 = d4;
            }
            for (int k = 0; k < 5; ++k) {
                g.diss[k][i1] = (g.diss[k][i1] - d4v[k] * d41) + d2v[k] * d2;
                g.diss[k][i2] = (g.diss[k][i2] + d4v[k] * d42) - d2v[k] * d2;
            }
        });
    }

    // ---- makeArtificialDissipation3 (def_par:11995-12139) -----------------
    void makeArtificialDissipation3(Level &g) {
        for (int k = 0; k < 5; ++k) std::fill(g.diss[k].begin(), g.diss[k].end(), 0.0);
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double d0 = std::min(g.V[i1] / g.dt[i1], g.V[i2] / g.dt[i2]) / (g.conn[i1] + g.conn[i2]);
            double d2 = d0 * c.coarseGridDissipationFactor;
            for (int k = 0; k < 5; ++k) {
                double dk = g.u[k][i1] - g.u[k][i2];
                g.diss[k][i1] = g.diss[k][i1] + dk * d2;
                g.diss[k][i2] = g.diss[k][i2] - dk * d2;
            }
        });
    }

    // ---- makeViscosityTerm, wide stencil (def_par:5198-5893) --------------
    // Sutherland's (T)^1.5 is evaluated as T*sqrt(T).
    void makeViscosityTerm(Level &g) {
        const double gOg = c.gamma / (c.gamma - 1.0);
        const double tempConv = (c.gamma - 1.0) * c.MachNumber * c.MachNumber;
        const double Tin = c.inflowTemperature;
        for (int k = 0; k < 12; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        auto prim = [&](int i, double *q) {
            double r = g.u[0][i];
            q[0] = g.u[1][i] / r; q[1] = g.u[2][i] / r; q[2] = g.u[3][i] / r;
            q[3] = gOg * g.p[i] / r;
        };
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double w[3] = {g.wx[e], g.wy[e], g.wz[e]};
            double q1[4], q2[4];
            prim(i1, q1); prim(i2, q2);
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    double d = (q1[k] + q2[k]) * w[a];
                    nh[a * 4 + k][i1] = nh[a * 4 + k][i1] + d;
                    nh[a * 4 + k][i2] = nh[a * 4 + k][i2] - d;
                }
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double w[3] = {g.bwx[b], g.bwy[b], g.bwz[b]};
            double q1[4], q2[4];
            prim(i1, q1); prim(i2, q2);
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    double s = q1[k] + q2[k];
                    nh[a * 4 + k][i1] = nh[a * 4 + k][i1] + (2. * q1[k] + s) * w[a];
                }
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    double s = q1[k] + q2[k];
                    nh[a * 4 + k][i2] = nh[a * 4 + k][i2] + (2. * q2[k] + s) * w[a];
                }
        });
        const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
        const double oRe = 1. / c.ReynoldsNumber, oPr = 1. / c.PrandtlNumber;
        for_nodes(g.N, [&](int i) {
            double vt = 1. / g.V[i];
            double dudx = nh[0][i] * vt, dvdx = nh[1][i] * vt, dwdx = nh[2][i] * vt, dTdx = nh[3][i] * vt;
            double dudy = nh[4][i] * vt, dvdy = nh[5][i] * vt, dwdy = nh[6][i] * vt, dTdy = nh[7][i] * vt;
            double dudz = nh[8][i] * vt, dvdz = nh[9][i] * vt, dwdz = nh[10][i] * vt, dTdz = nh[11][i] * vt;
            double T = gOg * g.p[i] / g.u[0][i];
            if (T <= 0.001) T = 0.001;
            double a = tempConv * T;
            double mu = oRe * ((a * std::sqrt(a)) * ((Tin + 198.6) / (tempConv * Tin * T + 198.6)));
            double k = oPr * mu;
            g.mu[i] = mu;
            {
                const double a1 = dudy - dvdx, a2 = dvdz - dwdy, a3 = dwdx - dudz;
                g.vort[i] = std::sqrt((a1 * a1 + a2 * a2) + a3 * a3);
                g.divg[i] = (dudx + dvdy) + dwdz;
            }
            if (sa()) {  // def_par:5556-5566
                double tvc = oRe * g.u[0][i] * g.u[5][i];
                const double ksi3 = flite_pm::pm_cube(tvc / mu);
                tvc = tvc * ksi3 / (ksi3 + 357.9);
                mu = mu + tvc;
                k = k + tvc * (1. / c.turbulentPrandtlNumber);
            }
            nh[0][i] = mu * (fourThirds * dudx - twoThirds * (dvdy + dwdz));
            nh[1][i] = mu * (dudy + dvdx);
            nh[2][i] = mu * (dudz + dwdx);
            nh[3][i] = mu * (fourThirds * dvdy - twoThirds * (dudx + dwdz));
            nh[4][i] = mu * (dvdz + dwdy);
            nh[5][i] = mu * (fourThirds * dwdz - twoThirds * (dudx + dvdy));
            nh[6][i] = k * dTdx;
            nh[7][i] = k * dTdy;
            nh[8][i] = k * dTdz;
        });
        if (g.grid == 1) {
            // setTemperatureForAdiabaticWall (def_par:5170-5196)
            for_range(g, -20, -19, [&](int ip) {
                double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
                double dT[3] = {nh[6][ip], nh[7][ip], nh[8][ip]};
                double nt = (dT[0] * n[0] + dT[1] * n[1]) + dT[2] * n[2];
                for (int k = 0; k < 3; ++k) nh[6 + k][ip] = dT[k] - nt * n[k];
            });
            // wall stress of the boundary nodes (def_par:5620-5635)
            for (int ib = 0; ib < std::min(g.Nb, g.nnorm); ++ib) {
                int ip = g.node_ind[ib];
                double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
                g.wallStress[0][ip] = (nh[0][ip] * n[0] + nh[1][ip] * n[1]) + nh[2][ip] * n[2];
                g.wallStress[1][ip] = (nh[1][ip] * n[0] + nh[3][ip] * n[1]) + nh[4][ip] * n[2];
                g.wallStress[2][ip] = (nh[2][ip] * n[0] + nh[4][ip] * n[1]) + nh[5][ip] * n[2];
            }
        }
        for (int k = 9; k < 13; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        auto loadt = [&](int i, double *t, double *uu) {
            for (int k = 0; k < 9; ++k) t[k] = nh[k][i];
            uu[0] = g.u[1][i] / g.u[0][i]; uu[1] = g.u[2][i] / g.u[0][i]; uu[2] = g.u[3][i] / g.u[0][i];
        };
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
            double a[9], b[9], ua[3], ub[3];
            loadt(i1, a, ua); loadt(i2, b, ub);
            double dt[9];
            for (int k = 0; k < 9; ++k) dt[k] = a[k] + b[k];
            double dut1 = ((((ua[0] * a[0] + ub[0] * b[0]) + ua[1] * a[1]) + ub[1] * b[1]) + ua[2] * a[2]) + ub[2] * b[2];
            double dut2 = ((((ua[0] * a[1] + ub[0] * b[1]) + ua[1] * a[3]) + ub[1] * b[3]) + ua[2] * a[4]) + ub[2] * b[4];
            double dut3 = ((((ua[0] * a[2] + ub[0] * b[2]) + ua[1] * a[4]) + ub[1] * b[4]) + ua[2] * a[5]) + ub[2] * b[5];
            double f2 = (wx * dt[0] + wy * dt[1]) + wz * dt[2];
            double f3 = (wx * dt[1] + wy * dt[3]) + wz * dt[4];
            double f4 = (wx * dt[2] + wy * dt[4]) + wz * dt[5];
            double f5 = (wx * (dt[6] + dut1) + wy * (dt[7] + dut2)) + wz * (dt[8] + dut3);
            double f[4] = {f2, f3, f4, f5};
            for (int k = 0; k < 4; ++k) {
                nh[9 + k][i1] = nh[9 + k][i1] + f[k];
                nh[9 + k][i2] = nh[9 + k][i2] - f[k];
            }
        });
        for (int bb = 0; bb < g.B; ++bb) {
            int ind = g.bind[bb];
            if (ind == 2 || ind == 9) continue;
            int i1 = g.b1[bb], i2 = g.b2[bb];
            double wx = g.bwx[bb], wy = g.bwy[bb], wz = g.bwz[bb];
            double a[9], b[9], ua[3], ub[3];
            loadt(i1, a, ua); loadt(i2, b, ub);
            double dt[9];
            for (int k = 0; k < 9; ++k) dt[k] = a[k] + b[k];
            double d11 = (ua[0] * a[0] + ua[1] * a[1]) + ua[2] * a[2];
            double d12 = (ub[0] * b[0] + ub[1] * b[1]) + ub[2] * b[2];
            double d21 = (ua[0] * a[1] + ua[1] * a[3]) + ua[2] * a[4];
            double d22 = (ub[0] * b[1] + ub[1] * b[3]) + ub[2] * b[4];
            double d31 = (ua[0] * a[2] + ua[1] * a[4]) + ua[2] * a[5];
            double d32 = (ub[0] * b[2] + ub[1] * b[4]) + ub[2] * b[5];
            double dut1 = d11 + d12, dut2 = d21 + d22, dut3 = d31 + d32;
            double f2 = (wx * dt[0] + wy * dt[1]) + wz * dt[2];
            double f3 = (wx * dt[1] + wy * dt[3]) + wz * dt[4];
            double f4 = (wx * dt[2] + wy * dt[4]) + wz * dt[5];
            double f5 = (wx * (dt[6] + dut1) + wy * (dt[7] + dut2)) + wz * (dt[8] + dut3);
            nh[9][i1] = (nh[9][i1] + f2) + 2.0 * ((wx * a[0] + wy * a[1]) + wz * a[2]);
            nh[10][i1] = (nh[10][i1] + f3) + 2.0 * ((wx * a[1] + wy * a[3]) + wz * a[4]);
            nh[11][i1] = (nh[11][i1] + f4) + 2.0 * ((wx * a[2] + wy * a[4]) + wz * a[5]);
            nh[12][i1] = (nh[12][i1] + f5) + 2.0 * ((wx * (a[6] + d11) + wy * (a[7] + d21)) + wz * (a[8] + d31));
            nh[9][i2] = (nh[9][i2] + f2) + 2.0 * ((wx * b[0] + wy * b[1]) + wz * b[2]);
            nh[10][i2] = (nh[10][i2] + f3) + 2.0 * ((wx * b[1] + wy * b[3]) + wz * b[4]);
            nh[11][i2] = (nh[11][i2] + f4) + 2.0 * ((wx * b[2] + wy * b[4]) + wz * b[5]);
            nh[12][i2] = (nh[12][i2] + f5) + 2.0 * ((wx * (b[6] + d12) + wy * (b[7] + d22)) + wz * (b[8] + d32));
        }
        for_nodes(g.N, [&](int i) { for (int k = 0; k < 4; ++k) g.diss[1 + k][i] = g.diss[1 + k][i] - nh[9 + k][i]; });
    }

    // the viscous routine of the run: makeViscosityTerm, or the compact
    // makeViscosityTerm2 with viscosityScheme 2 (def_par:1038-1043)
    void viscousTerm(Level &g) {
        if (c.viscosityScheme == 2) makeViscosityTerm2(g);
        else makeViscosityTerm(g);
    }

    // ---- makeViscosityTerm2, compact stencil (def_par:5896-6807) -----------
    // Galerkin gradients of (u, v, w, T) as in makeViscosityTerm (with the FV
    // boundary form under boundaryTerm 2), scaled per node by mu (velocity)
    // and k (temperature); per edge the sum of both ends' scaled gradients
    // with its component along the edge replaced by the compact difference
    // (mu1 + mu2)(q2 - q1)/|dx| (coordinates of level 1; zero on coarse
    // levels, where the correction vanishes); boundary faces take 4 w_b
    // times each node's own stress.
    void makeViscosityTerm2(Level &g) {
        const double gOg = c.gamma / (c.gamma - 1.0);
        const double tempConv = (c.gamma - 1.0) * c.MachNumber * c.MachNumber;
        const double Tin = c.inflowTemperature;
        for (int k = 0; k < 14; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        auto prim = [&](int i, double *q) {
            double r = g.u[0][i];
            q[0] = g.u[1][i] / r; q[1] = g.u[2][i] / r; q[2] = g.u[3][i] / r;
            q[3] = gOg * g.p[i] / r;
        };
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double w[3] = {g.wx[e], g.wy[e], g.wz[e]};
            double q1[4], q2[4];
            prim(i1, q1); prim(i2, q2);
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    double d = (q1[k] + q2[k]) * w[a];
                    nh[a * 4 + k][i1] = nh[a * 4 + k][i1] + d;
                    nh[a * 4 + k][i2] = nh[a * 4 + k][i2] - d;
                }
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double w[3] = {g.bwx[b], g.bwy[b], g.bwz[b]};
            double q1[4], q2[4];
            prim(i1, q1); prim(i2, q2);
            if (c.boundaryTerm == 1) {
                for (int a = 0; a < 3; ++a)
                    for (int k = 0; k < 4; ++k) nh[a * 4 + k][i1] = nh[a * 4 + k][i1] + (2. * q1[k] + (q1[k] + q2[k])) * w[a];
                for (int a = 0; a < 3; ++a)
                    for (int k = 0; k < 4; ++k) nh[a * 4 + k][i2] = nh[a * 4 + k][i2] + (2. * q2[k] + (q1[k] + q2[k])) * w[a];
            } else {
                for (int a = 0; a < 3; ++a)
                    for (int k = 0; k < 4; ++k) nh[a * 4 + k][i1] = nh[a * 4 + k][i1] + 4. * q1[k] * w[a];
                for (int a = 0; a < 3; ++a)
                    for (int k = 0; k < 4; ++k) nh[a * 4 + k][i2] = nh[a * 4 + k][i2] + 4. * q2[k] * w[a];
            }
        });
        const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
        const double oRe = 1. / c.ReynoldsNumber, oPr = 1. / c.PrandtlNumber;
        for_nodes(g.N, [&](int i) {
            const double vt = 1. / g.V[i];
            for (int k = 0; k < 12; ++k) nh[k][i] = nh[k][i] * vt;
            const double dudx = nh[0][i], dvdx = nh[1][i], dwdx = nh[2][i];
            const double dudy = nh[4][i], dvdy = nh[5][i], dwdy = nh[6][i];
            const double dudz = nh[8][i], dvdz = nh[9][i], dwdz = nh[10][i];
            double T = gOg * g.p[i] / g.u[0][i];
            if (T <= 0.001) T = 0.001;
            double a = tempConv * T;
            double mu = oRe * ((a * std::sqrt(a)) * ((Tin + 198.6) / (tempConv * Tin * T + 198.6)));
            double k = oPr * mu;
            g.mu[i] = mu;
            {
                const double a1 = dudy - dvdx, a2 = dvdz - dwdy, a3 = dwdx - dudz;
                g.vort[i] = std::sqrt((a1 * a1 + a2 * a2) + a3 * a3);
                g.divg[i] = (dudx + dvdy) + dwdz;
            }
            if (sa()) {  // def_par:6290-6300
                double tvc = oRe * g.u[0][i] * g.u[5][i];
                const double ksi3 = flite_pm::pm_cube(tvc / mu);
                tvc = tvc * ksi3 / (ksi3 + 357.9);
                mu = mu + tvc;
                k = k + tvc * (1. / c.turbulentPrandtlNumber);
            }
            for (int q : {0, 1, 2, 4, 5, 6, 8, 9, 10}) nh[q][i] = mu * nh[q][i];
            for (int q : {3, 7, 11}) nh[q][i] = k * nh[q][i];
            nh[12][i] = mu;
            nh[13][i] = k;
        });
        if (g.grid == 1) {
            // setTemperatureForAdiabaticWall on the scaled temperature
            // gradients (def_par:6346-6349), then the wall stress of the wall
            // nodes (:6351-6393)
            for_range(g, -20, -19, [&](int ip) {
                double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
                double dT[3] = {nh[3][ip], nh[7][ip], nh[11][ip]};
                double nt = (dT[0] * n[0] + dT[1] * n[1]) + dT[2] * n[2];
                nh[3][ip] = dT[0] - nt * n[0];
                nh[7][ip] = dT[1] - nt * n[1];
                nh[11][ip] = dT[2] - nt * n[2];
            });
            for_range(g, -20, -19, [&](int ip) {
                double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
                const double dudx = nh[0][ip], dvdx = nh[1][ip], dwdx = nh[2][ip];
                const double dudy = nh[4][ip], dvdy = nh[5][ip], dwdy = nh[6][ip];
                const double dudz = nh[8][ip], dvdz = nh[9][ip], dwdz = nh[10][ip];
                const double c1 = fourThirds * dudx - twoThirds * (dvdy + dwdz), c2 = dudy + dvdx, c3 = dudz + dwdx;
                const double c4 = fourThirds * dvdy - twoThirds * (dudx + dwdz), c5 = dvdz + dwdy;
                const double c6 = fourThirds * dwdz - twoThirds * (dudx + dvdy);
                g.wallStress[0][ip] = (c1 * n[0] + c2 * n[1]) + c3 * n[2];
                g.wallStress[1][ip] = (c2 * n[0] + c4 * n[1]) + c5 * n[2];
                g.wallStress[2][ip] = (c3 * n[0] + c5 * n[1]) + c6 * n[2];
            });
        }
        if (c.wallsAreIsentropic)  // def_par:6399-6405
            for (int i = 0; i < g.Nb; ++i) nh[3][i] = nh[7][i] = nh[11][i] = 0.0;
        for (int k = 14; k < 18; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        auto vel = [&](int i, double *v) {
            const double ri = 1.0 / g.u[0][i];
            v[0] = g.u[1][i] * ri; v[1] = g.u[2][i] * ri; v[2] = g.u[3][i] * ri;
            v[3] = gOg * g.p[i] * ri;
        };
        for_edges(g, [&](int e) {
            const int i1 = g.s1[e], i2 = g.s2[e];
            double f[4];
            visc2_edge(g, e, i1, i2, vel, f);
            for (int k = 0; k < 4; ++k) {
                nh[14 + k][i1] = nh[14 + k][i1] + f[k];
                nh[14 + k][i2] = nh[14 + k][i2] - f[k];
            }
        });
        for (int bb = 0; bb < g.B; ++bb) {
            const int ind = g.bind[bb];
            if (ind == 2 || ind == 9) continue;
            const int i1 = g.b1[bb], i2 = g.b2[bb];
            const double wx = g.bwx[bb], wy = g.bwy[bb], wz = g.bwz[bb];
            for (int side = 0; side < 2; ++side) {
                const int ip = side == 0 ? i1 : i2;
                double v[4];
                vel(ip, v);
                const double dudx = nh[0][ip], dvdx = nh[1][ip], dwdx = nh[2][ip], dTdx = nh[3][ip];
                const double dudy = nh[4][ip], dvdy = nh[5][ip], dwdy = nh[6][ip], dTdy = nh[7][ip];
                const double dudz = nh[8][ip], dvdz = nh[9][ip], dwdz = nh[10][ip], dTdz = nh[11][ip];
                const double t1 = fourThirds * dudx - twoThirds * (dvdy + dwdz), t2 = dudy + dvdx, t3 = dudz + dwdx;
                const double t4 = fourThirds * dvdy - twoThirds * (dudx + dwdz), t5 = dvdz + dwdy;
                const double t6 = fourThirds * dwdz - twoThirds * (dudx + dvdy);
                double t7 = dTdx, t8 = dTdy, t9 = dTdz;
                if (c.wallsAreIsentropic) t7 = t8 = t9 = 0.0;
                const double d1 = (v[0] * t1 + v[1] * t2) + v[2] * t3;
                const double d2 = (v[0] * t2 + v[1] * t4) + v[2] * t5;
                const double d3 = (v[0] * t3 + v[1] * t5) + v[2] * t6;
                nh[14][ip] = nh[14][ip] + 4.0 * ((wx * t1 + wy * t2) + wz * t3);
                nh[15][ip] = nh[15][ip] + 4.0 * ((wx * t2 + wy * t4) + wz * t5);
                nh[16][ip] = nh[16][ip] + 4.0 * ((wx * t3 + wy * t5) + wz * t6);
                nh[17][ip] = nh[17][ip] + 4.0 * ((wx * (t7 + d1) + wy * (t8 + d2)) + wz * (t9 + d3));
            }
        }
        for_nodes(g.N, [&](int i) { for (int k = 0; k < 4; ++k) g.diss[1 + k][i] = g.diss[1 + k][i] - nh[14 + k][i]; });
    }

    // the compact viscous flux of edge e = (i1, i2) (def_par:6432-6556)
    template <class Vel>
    void visc2_edge(const Level &g, int e, int i1, int i2, Vel &&vel, double *f) {
        const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
        const double inv = 1.0 / g.slen[e];
        const double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
        const double mmu1 = nh[12][i1], mmu2 = nh[12][i2], k1 = nh[13][i1], k2 = nh[13][i2];
        double v1[4], v2[4];
        vel(i1, v1);
        vel(i2, v2);
        const double r[3] = {(g.cx[i2] - g.cx[i1]) * inv, (g.cy[i2] - g.cy[i1]) * inv, (g.cz[i2] - g.cz[i1]) * inv};
        // summed scaled gradients: G[q][a] = d q / d x_a, q = u, v, w, T
        double G[4][3];
        for (int q = 0; q < 4; ++q)
            for (int a = 0; a < 3; ++a) G[q][a] = nh[a * 4 + q][i1] + nh[a * 4 + q][i2];
        const double cf[4] = {mmu1 + mmu2, mmu1 + mmu2, mmu1 + mmu2, k1 + k2};
        for (int q = 0; q < 4; ++q) {
            const double dr = (G[q][0] * r[0] + G[q][1] * r[1]) + G[q][2] * r[2];
            for (int a = 0; a < 3; ++a) G[q][a] = G[q][a] - dr * r[a];
            const double dq = cf[q] * (v2[q] - v1[q]) * inv;
            for (int a = 0; a < 3; ++a) G[q][a] = G[q][a] + dq * r[a];
        }
        const double dudx = G[0][0], dudy = G[0][1], dudz = G[0][2];
        const double dvdx = G[1][0], dvdy = G[1][1], dvdz = G[1][2];
        const double dwdx = G[2][0], dwdy = G[2][1], dwdz = G[2][2];
        const double dt1 = fourThirds * dudx - twoThirds * (dvdy + dwdz), dt2 = dudy + dvdx, dt3 = dudz + dwdx;
        const double dt4 = fourThirds * dvdy - twoThirds * (dudx + dwdz), dt5 = dvdz + dwdy;
        const double dt6 = fourThirds * dwdz - twoThirds * (dudx + dvdy);
        const double dt7 = G[3][0], dt8 = G[3][1], dt9 = G[3][2];
        const double au = 0.5 * (v1[0] + v2[0]), av = 0.5 * (v1[1] + v2[1]), aw = 0.5 * (v1[2] + v2[2]);
        const double dut1 = (au * dt1 + av * dt2) + aw * dt3;
        const double dut2 = (au * dt2 + av * dt4) + aw * dt5;
        const double dut3 = (au * dt3 + av * dt5) + aw * dt6;
        f[0] = (wx * dt1 + wy * dt2) + wz * dt3;
        f[1] = (wx * dt2 + wy * dt4) + wz * dt5;
        f[2] = (wx * dt3 + wy * dt5) + wz * dt6;
        f[3] = (wx * (dt7 + dut1) + wy * (dt8 + dut2)) + wz * (dt9 + dut3);
    }

    // ---- computeGradient, Galerkin (def_par:2923-3245) --------------------
    void computeGradient(Level &g, vec *u) {
        for (int k = 0; k < 15; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double w[3] = {g.wx[e], g.wy[e], g.wz[e]};
            double r1 = u[0][i1], q1[5] = {r1, u[1][i1] / r1, u[2][i1] / r1, u[3][i1] / r1, u[4][i1]};
            double r2 = u[0][i2], q2[5] = {r2, u[1][i2] / r2, u[2][i2] / r2, u[3][i2] / r2, u[4][i2]};
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 5; ++k) {
                    double dq = (q1[k] + q2[k]) * w[a];
                    nh[a * 5 + k][i1] = nh[a * 5 + k][i1] + dq;
                    nh[a * 5 + k][i2] = nh[a * 5 + k][i2] - dq;
                }
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double w[3] = {g.bwx[b], g.bwy[b], g.bwz[b]};
            double r1 = u[0][i1], q1[5] = {r1, u[1][i1] / r1, u[2][i1] / r1, u[3][i1] / r1, u[4][i1]};
            double r2 = u[0][i2], q2[5] = {r2, u[1][i2] / r2, u[2][i2] / r2, u[3][i2] / r2, u[4][i2]};
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 5; ++k) {
                    double s = q1[k] + q2[k];
                    nh[a * 5 + k][i1] = nh[a * 5 + k][i1] + (2. * q1[k] + s) * w[a];
                }
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 5; ++k) {
                    double s = q1[k] + q2[k];
                    nh[a * 5 + k][i2] = nh[a * 5 + k][i2] + (2. * q2[k] + s) * w[a];
                }
        });
        for (int i = 0; i < g.N; ++i) {
            double vt = 1. / g.V[i];
            for (int k = 0; k < 15; ++k) nh[k][i] = nh[k][i] * vt;
        }
    }

    // ---- LSComputeGradient + computegradhat (def_par:2593-2920) -----------
    // five scalar passes (rho, u, v, w, E) of the least-squares gradient with
    // 1/|dx|^2 weights and the adjugate inverse of the 3x3 moment matrix
    void LSComputeGradient(Level &g, vec *u) {
        vec grad[15];
        for (auto &a : grad) a.assign(g.N, 0.0);
        for (int k = 0; k < 15; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        vec v(g.N);
        for (int sc = 0; sc < 5; ++sc) {
            for (int i = 0; i < g.N; ++i) v[i] = (sc == 0 || sc == 4) ? u[sc][i] : u[sc][i] / u[0][i];
            computegradhat(g, v);
            for (int i = 0; i < g.N; ++i) {
                grad[sc][i] = nh[9][i];
                grad[5 + sc][i] = nh[10][i];
                grad[10 + sc][i] = nh[11][i];
            }
        }
        for (int k = 0; k < 15; ++k) nh[k] = grad[k].size() == nh[k].size() ? grad[k] : nh[k];
        for (int k = 0; k < 15; ++k)
            for (int i = 0; i < g.N; ++i) nh[k][i] = grad[k][i];
    }
    void computegradhat(Level &g, const vec &q) {
        for (int k = 0; k < 9; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double dx = g.cx[i2] - g.cx[i1], dy = g.cy[i2] - g.cy[i1], dz = g.cz[i2] - g.cz[i1];
            double dist1 = 1. / ((dx * dx + dy * dy) + dz * dz);
            double dr2 = q[i2] - q[i1];
            double m[6] = {dx * dx * dist1, dx * dy * dist1, dx * dz * dist1,
                           dy * dy * dist1, dy * dz * dist1, dz * dz * dist1};
            for (int k = 0; k < 6; ++k) nh[k][i1] = nh[k][i1] + m[k];
            for (int k = 0; k < 6; ++k) nh[k][i2] = nh[k][i2] + m[k];
            double b[3] = {dr2 * dx * dist1, dr2 * dy * dist1, dr2 * dz * dist1};
            for (int k = 0; k < 3; ++k) nh[6 + k][i1] = nh[6 + k][i1] + b[k];
            for (int k = 0; k < 3; ++k) nh[6 + k][i2] = nh[6 + k][i2] + b[k];
        });
        for_nodes(g.N, [&](int i) {
            double a11 = nh[0][i], a12 = nh[1][i], a13 = nh[2][i];
            double a21 = nh[1][i], a22 = nh[3][i], a23 = nh[4][i];
            double a31 = nh[2][i], a32 = nh[4][i], a33 = nh[5][i];
            double c11 = a22 * a33 - a23 * a32, c21 = a23 * a31 - a21 * a33, c31 = a21 * a32 - a22 * a31;
            double det = (a11 * c11 + a12 * c21) + a13 * c31;
            if (std::fabs(det) > 0.0) det = 1.0 / det;
            c11 = det * c11; c21 = det * c21; c31 = det * c31;
            double c12 = det * (a13 * a32 - a12 * a33), c22 = det * (a11 * a33 - a13 * a31);
            double c32 = det * (a12 * a31 - a11 * a32), c13 = det * (a12 * a23 - a13 * a22);
            double c23 = det * (a13 * a21 - a23 * a11), c33 = det * (a11 * a22 - a12 * a21);
            double b1 = nh[6][i], b2 = nh[7][i], b3 = nh[8][i];
            nh[9][i] = (c11 * b1 + c12 * b2) + c13 * b3;
            nh[10][i] = (c21 * b1 + c22 * b2) + c23 * b3;
            nh[11][i] = (c31 * b1 + c32 * b2) + c33 * b3;
        });
    }

    // ---- LocalMinMax (def_par:3248-3459) ----------------------------------
    void LocalMinMax(Level &g) {
        for (int k = 15; k < 25; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 1.0e15);
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double r1 = g.u[0][i1], q1[5] = {r1, g.u[1][i1] / r1, g.u[2][i1] / r1, g.u[3][i1] / r1, g.u[4][i1]};
            double r2 = g.u[0][i2], q2[5] = {r2, g.u[1][i2] / r2, g.u[2][i2] / r2, g.u[3][i2] / r2, g.u[4][i2]};
            double mn[5], mx[5];
            for (int k = 0; k < 5; ++k) { mn[k] = std::min(q1[k], q2[k]); mx[k] = std::min(-q1[k], -q2[k]); }
            for (int k = 0; k < 5; ++k) nh[15 + k][i1] = std::min(nh[15 + k][i1], mn[k]);
            for (int k = 0; k < 5; ++k) nh[15 + k][i2] = std::min(nh[15 + k][i2], mn[k]);
            for (int k = 0; k < 5; ++k) nh[20 + k][i1] = std::min(nh[20 + k][i1], mx[k]);
            for (int k = 0; k < 5; ++k) nh[20 + k][i2] = std::min(nh[20 + k][i2], mx[k]);
        });
        for_nodes(g.N, [&](int i) {
            double r = g.u[0][i];
            double q[5] = {r, g.u[1][i] / r, g.u[2][i] / r, g.u[3][i] / r, g.u[4][i]};
            for (int k = 0; k < 5; ++k) nh[15 + k][i] = nh[15 + k][i] - q[k];
            for (int k = 0; k < 5; ++k) nh[20 + k][i] = -nh[20 + k][i] - q[k];
        });
    }

    // LED limiter branch of the HLLC reconstruction (def_par:1856-1867)
    static double led(double a, double bmin, double bmax, int nsig) {
        double cc = a;
        double a1 = 2.0 * a;
        if (a1 > 0.0) {
            double invmax = 0.0;
            if (bmax > 0.0) invmax = 1.0 / bmax;
            double t = a1 * invmax;
            double tn = nsig == 4 ? (t * t) * (t * t) : t * t;
            double root = nsig == 4 ? std::sqrt(std::sqrt(1. + tn)) : std::sqrt(1. + tn);
            cc = 0.5 * bmax * t / root;
        } else if (a1 < 0.0) {
            double invmin = 0.0;
            if (bmin < 0.0) invmin = 1.0 / bmin;
            double t = a1 * invmin;
            double tn = nsig == 4 ? (t * t) * (t * t) : t * t;
            double root = nsig == 4 ? std::sqrt(std::sqrt(1. + tn)) : std::sqrt(1. + tn);
            cc = 0.5 * bmin * t / root;
        }
        return cc;
    }

    // ---- makeRHS (def_par:1525-2590) --------------------------------------
    // ---- the upwind extension on level 1 (no reference counterpart) -------
    // Roe flux of the MUSCL / Van Albada states of edge i1 -> i2: states
    // (rho, (rho u)/rho, ..., rho E) reconstructed from the Galerkin gradient
    // nh, q_L = q1 + va(2 g1.d - dq, dq)/2, q_R = q2 - va(2 g2.d - dq, dq)/2;
    // unreconstructed states where a reconstructed density or pressure is
    // not positive; p = (gamma-1)(rho E - rho |u|^2/2); the Roe average and
    // wave strengths of def_par:1725-1792 with the upwind sign
    static double prim_pressure(double gam1, const double *q) {
        return gam1 * (q[4] - 0.5 * ((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]) * q[0]);
    }
    void muscl_roe_flux(const Level &g, int i1, int i2, double wx, double wy, double wz, double *f) {
        const double gam1 = c.gamma - 1.0;
        const double ra = g.u[0][i1], rb = g.u[0][i2];
        const double q1[5] = {ra, g.u[1][i1] / ra, g.u[2][i1] / ra, g.u[3][i1] / ra, g.u[4][i1]};
        const double q2[5] = {rb, g.u[1][i2] / rb, g.u[2][i2] / rb, g.u[3][i2] / rb, g.u[4][i2]};
        const double dx = g.cx[i2] - g.cx[i1], dy = g.cy[i2] - g.cy[i1], dz = g.cz[i2] - g.cz[i1];
        double qa[5], qb[5];
        for (int j = 0; j < 5; ++j) {
            const double dq = q2[j] - q1[j];
            const double g1 = (nh[j][i1] * dx + nh[j + 5][i1] * dy) + nh[j + 10][i1] * dz;
            const double g2 = (nh[j][i2] * dx + nh[j + 5][i2] * dy) + nh[j + 10][i2] * dz;
            qa[j] = q1[j] + 0.5 * van_albada(2.0 * g1 - dq, dq);
            qb[j] = q2[j] - 0.5 * van_albada(2.0 * g2 - dq, dq);
        }
        double pa = prim_pressure(gam1, qa), pb = prim_pressure(gam1, qb);
        if (!(qa[0] > 0.0 && qb[0] > 0.0 && pa > 0.0 && pb > 0.0)) {
            for (int j = 0; j < 5; ++j) { qa[j] = q1[j]; qb[j] = q2[j]; }
            pa = prim_pressure(gam1, qa);
            pb = prim_pressure(gam1, qb);
        }
        for (int k = 0; k < 5; ++k) f[k] = 0.0;
        const double rnorm = std::sqrt((wx * wx + wy * wy) + wz * wz);
        if (!(rnorm > 1.0e-10)) return;
        const double rn = 1.0 / rnorm;
        const double rnx = wx * rn, rny = wy * rn, rnz = wz * rn;
        const double r1 = qa[0], u1 = qa[1], v1 = qa[2], w1 = qa[3], E1 = qa[4];
        const double r2 = qb[0], u2 = qb[1], v2 = qb[2], w2 = qb[3], E2 = qb[4];
        const double ru1 = r1 * u1, rv1 = r1 * v1, rw1 = r1 * w1, rh1 = E1 + pa;
        const double ru2 = r2 * u2, rv2 = r2 * v2, rw2 = r2 * w2, rh2 = E2 + pb;
        const double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
        const double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
        const double h1 = rh1 / r1, h2 = rh2 / r2;
        const double di = std::sqrt(r1 / r2), d1 = 1.0 / (di + 1.0);
        const double ui = (di * u1 + u2) * d1, vi = (di * v1 + v2) * d1, wi = (di * w1 + w2) * d1;
        const double hi = (di * h1 + h2) * d1;
        const double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
        const double ci2 = std::max(gam1 * (hi - af), 1.0e-5);
        const double ci = std::sqrt(ci2), ici = 1.0 / ci, ici2 = 1.0 / ci2;
        const double ucp = (ui * rnx + vi * rny) + wi * rnz;
        const double du1 = r2 - r1, du2 = ru2 - ru1, du3 = rv2 - rv1, du4 = rw2 - rw1, du5 = E2 - E1;
        const double l1 = std::fabs(ucp + ci), l2 = std::fabs(ucp - ci), l3 = std::fabs(ucp);
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

    void makeRHS(Level &g) {
        const double gam = c.gamma, gam1 = c.gamma - 1.0;
        int hllcflux = 1, autoClip = 0, nsig = 4;
        double clip = 0;
        if (c.fluxType == 4) {
            hllcflux = c.HLLCFluxOrder;
            clip = c.HLLCClipping;
            autoClip = c.Automaticlipping;
            nsig = c.ReynoldsNumber < 1 ? 4 : 2;
            if (hllcflux > 1) {
                if (c.GradientMethod == 1) computeGradient(g, g.u);
                else LSComputeGradient(g, g.u);
                if (autoClip == 1) LocalMinMax(g);
            }
        }
        // the upwind MUSCL / Van Albada extension of the Roe flux (no
        // reference counterpart): Galerkin gradients, level 1 only
        const bool upwind = c.fluxType == 3 && c.reconstruction == FLITE_RECON_VAN_ALBADA;
        const bool muscl = upwind && g.grid == 1;
        if (muscl) computeGradient(g, g.u);
        for_edges(g, [&](int e) {
            const int i1 = g.s1[e], i2 = g.s2[e];
            double pr1 = g.p[i1], r1 = g.u[0][i1], rinv1 = 1. / g.u[0][i1];
            double ru1 = g.u[1][i1], rv1 = g.u[2][i1], rw1 = g.u[3][i1];
            double u1 = rinv1 * ru1, v1 = rinv1 * rv1, w1 = rinv1 * rw1;
            double E1 = g.u[4][i1], rh1 = g.u[4][i1] + pr1;
            double pr2 = g.p[i2], r2 = g.u[0][i2], rinv2 = 1. / g.u[0][i2];
            double ru2 = g.u[1][i2], rv2 = g.u[2][i2], rw2 = g.u[3][i2];
            double u2 = rinv2 * ru2, v2 = rinv2 * rv2, w2 = rinv2 * rw2;
            double E2 = g.u[4][i2], rh2 = g.u[4][i2] + pr2;
            double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
            double f[5] = {0, 0, 0, 0, 0};
            // the GCL term of a moving mesh, -q wgcl (def_par:1662-1791)
            const bool ale = c.flowType == 2;
            const double wgcl = ale ? g.gcl[e] / c.physicalTimeStep : 0.0;
            auto gcl_sum = [&]() {
                f[0] = f[0] - (r1 + r2) * wgcl; f[1] = f[1] - (ru1 + ru2) * wgcl; f[2] = f[2] - (rv1 + rv2) * wgcl;
                f[3] = f[3] - (rw1 + rw2) * wgcl; f[4] = f[4] - (E1 + E2) * wgcl;
            };
            if (c.fluxType == 1) {
                f[0] = (wx * (ru1 + ru2) + wy * (rv1 + rv2)) + wz * (rw1 + rw2);
                f[1] = (wx * (((ru1 * u1 + pr1) + ru2 * u2) + pr2) + wy * (ru1 * v1 + ru2 * v2)) + wz * (ru1 * w1 + ru2 * w2);
                f[2] = (wx * (rv1 * u1 + rv2 * u2) + wy * (((rv1 * v1 + pr1) + rv2 * v2) + pr2)) + wz * (rv1 * w1 + rv2 * w2);
                f[3] = (wx * (rw1 * u1 + rw2 * u2) + wy * (rw1 * v1 + rw2 * v2)) + wz * (((rw1 * w1 + pr1) + rw2 * w2) + pr2);
                f[4] = (wx * (rh1 * u1 + rh2 * u2) + wy * (rh1 * v1 + rh2 * v2)) + wz * (rh1 * w1 + rh2 * w2);
                if (ale) gcl_sum();
            } else if (c.fluxType == 2) {  // LLF (def_par:1670-1724)
                double rnorm = std::sqrt((wx * wx + wy * wy) + wz * wz);
                if (rnorm > 1.0e-10) {
                    double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
                    double c1 = std::sqrt(gam * pr1 * rinv1);
                    double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
                    double f11 = r1 * nv1, f21 = pr1 * rnx + ru1 * nv1, f31 = pr1 * rny + rv1 * nv1;
                    double f41 = pr1 * rnz + rw1 * nv1, f51 = rh1 * nv1;
                    double c2 = std::sqrt(gam * pr2 * rinv2);
                    double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
                    double f12 = r2 * nv2, f22 = pr2 * rnx + ru2 * nv2, f32 = pr2 * rny + rv2 * nv2;
                    double f42 = pr2 * rnz + rw2 * nv2, f52 = rh2 * nv2;
                    double du[5] = {r1 - r2, ru1 - ru2, rv1 - rv2, rw1 - rw2, E1 - E2};
                    double l11 = std::fabs(nv1 + c1), l12 = std::fabs(nv2 + c2);
                    double l1 = l11; if (l1 < l12) l1 = l12;
                    double l21 = std::fabs(nv1 - c1), l22 = std::fabs(nv2 - c2);
                    double l2 = l21; if (l2 < l22) l2 = l22;
                    double lam = l1; if (lam < l2) lam = l2;
                    f[0] = rnorm * ((f11 + f12) - lam * du[0]);
                    f[1] = rnorm * ((f21 + f22) - lam * du[1]);
                    f[2] = rnorm * ((f31 + f32) - lam * du[2]);
                    f[3] = rnorm * ((f41 + f42) - lam * du[3]);
                    f[4] = rnorm * ((f51 + f52) - lam * du[4]);
                    if (ale) gcl_sum();
                }
            } else if (c.fluxType == 3 && muscl) {
                muscl_roe_flux(g, i1, i2, wx, wy, wz, f);
            } else if (c.fluxType == 3) {  // Roe (def_par:1725-1792)
                double rnorm = std::sqrt((wx * wx + wy * wy) + wz * wz);
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
                    double di = std::sqrt(r1 / r2), d1 = 1.0 / (di + 1.0);
                    double ui = (di * u1 + u2) * d1, vi = (di * v1 + v2) * d1, wi = (di * w1 + w2) * d1;
                    double hi = (di * h1 + h2) * d1;
                    double ci2 = gam1 * (hi - 0.5 * ((ui * ui + vi * vi) + wi * wi));
                    ci2 = std::max(ci2, 1.0e-5);
                    double ci = std::sqrt(ci2);
                    double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
                    double ucp = (ui * rnx + vi * rny) + wi * rnz;
                    double du1 = r1 - r2, du2 = ru1 - ru2, du3 = rv1 - rv2, du4 = rw1 - rw2, du5 = E1 - E2;
                    if (upwind) {
                        // the extension (coarse levels) adds the Roe
                        // dissipation with the upwind sign; the reference's
                        // branch subtracts it
                        du1 = r2 - r1; du2 = ru2 - ru1; du3 = rv2 - rv1; du4 = rw2 - rw1; du5 = E2 - E1;
                    }
                    double l1 = std::fabs(ucp + ci), l2 = std::fabs(ucp - ci), l3 = std::fabs(ucp);
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
                    if (ale) gcl_sum();
                }
            } else {  // HLLC (def_par:1794-2085)
                // central flux of the unreconstructed states (def_par:1798-
                // 1802); it stays only if no wave-speed branch applies
                f[0] = (wx * (ru1 + ru2) + wy * (rv1 + rv2)) + wz * (rw1 + rw2);
                f[1] = (wx * (((ru1 * u1 + pr1) + ru2 * u2) + pr2) + wy * (ru1 * v1 + ru2 * v2)) + wz * (ru1 * w1 + ru2 * w2);
                f[2] = (wx * (rv1 * u1 + rv2 * u2) + wy * (((rv1 * v1 + pr1) + rv2 * v2) + pr2)) + wz * (rv1 * w1 + rv2 * w2);
                f[3] = (wx * (rw1 * u1 + rw2 * u2) + wy * (rw1 * v1 + rw2 * v2)) + wz * (((rw1 * w1 + pr1) + rw2 * w2) + pr2);
                f[4] = (wx * (rh1 * u1 + rh2 * u2) + wy * (rh1 * v1 + rh2 * v2)) + wz * (rh1 * w1 + rh2 * w2);
                double roe1 = g.u[0][i1], roe2 = g.u[0][i2], re1 = g.u[4][i1], re2 = g.u[4][i2];
                double wx2 = 2.0 * wx, wy2 = 2.0 * wy, wz2 = 2.0 * wz;
                double rnorm = std::sqrt((wx2 * wx2 + wy2 * wy2) + wz2 * wz2);
                double rnorm1 = rnorm;
                if (rnorm > 0.0) rnorm = 1.0 / rnorm;
                double rnx = wx2 * rnorm, rny = wy2 * rnorm, rnz = wz2 * rnorm;
                if (hllcflux > 1) {
                    double dx = g.cx[i2] - g.cx[i1], dy = g.cy[i2] - g.cy[i1], dz = g.cz[i2] - g.cz[i1];
                    double hlength = 0.5 * clip * std::sqrt((dx * dx + dy * dy) + dz * dz);
                    double dpvl[5];
                    for (int j = 0; j < 5; ++j) {
                        double dpv1 = 0.5 * ((nh[j][i1] * dx + nh[j + 5][i1] * dy) + nh[j + 10][i1] * dz);
                        double dpv11 = 0.5 * ((nh[j][i2] * dx + nh[j + 5][i2] * dy) + nh[j + 10][i2] * dz);
                        if (autoClip == 1) {
                            dpv1 = led(dpv1, nh[j + 15][i1], nh[j + 20][i1], nsig);
                            dpv11 = -led(-dpv11, nh[j + 15][i2], nh[j + 20][i2], nsig);
                        }
                        double a = dpv1, b = dpv11, cc;
                        if (a * b <= 0.0) {
                            cc = 0.0;
                        } else {
                            cc = std::fabs(a) <= std::fabs(b) ? a : b;
                            if (std::fabs(cc) > hlength && hlength > 0.0) cc = hlength * cc / std::fabs(cc);
                        }
                        dpvl[j] = cc;
                    }
                    if ((roe1 + dpvl[0]) > 0.1) roe1 = roe1 + dpvl[0];
                    u1 = u1 + dpvl[1]; v1 = v1 + dpvl[2]; w1 = w1 + dpvl[3];
                    if ((re1 + dpvl[4]) > 0.0001) re1 = re1 + dpvl[4];
                    pr1 = gam1 * (re1 - 0.5 * ((u1 * u1 + v1 * v1) + w1 * w1) * roe1);
                    pr1 = std::max(pr1, 0.1);
                    rh1 = re1 + pr1; rinv1 = 1 / roe1;
                    ru1 = roe1 * u1; rv1 = roe1 * v1; rw1 = roe1 * w1;
                    if ((roe2 - dpvl[0]) > 0.1) roe2 = roe2 - dpvl[0];
                    u2 = u2 - dpvl[1]; v2 = v2 - dpvl[2]; w2 = w2 - dpvl[3];
                    if ((re2 - dpvl[4]) > 0.0001) re2 = re2 - dpvl[4];
                    pr2 = gam1 * (re2 - 0.5 * ((u2 * u2 + v2 * v2) + w2 * w2) * roe2);
                    pr2 = std::max(pr2, 0.1);
                    rh2 = re2 + pr2; rinv2 = 1 / roe2;
                    ru2 = roe2 * u2; rv2 = roe2 * v2; rw2 = roe2 * w2;
                }
                double nv1 = (u1 * rnx + v1 * rny) + w1 * rnz;
                double nv2 = (u2 * rnx + v2 * rny) + w2 * rnz;
                double beta0 = std::sqrt(gam1 / (2 * gam));
                double rroe = std::sqrt(roe2 / roe1);
                double ut = (u1 + u2 * rroe) / (1 + rroe), vt = (v1 + v2 * rroe) / (1 + rroe);
                double wt = (w1 + w2 * rroe) / (1 + rroe);
                double qt = (ut * rnx + vt * rny) + wt * rnz;
                double ht = (rh1 * rinv1 + rh2 * rinv2 * rroe) / (1 + rroe);
                double ct = gam1 * (ht - 0.5 * ((ut * ut + vt * vt) + wt * wt));
                ct = std::sqrt(std::fabs(ct));
                double c1 = std::sqrt(gam1 * std::fabs(rh1 * rinv1 - 0.5 * ((u1 * u1 + v1 * v1) + w1 * w1)));
                double c2 = std::sqrt(gam1 * std::fabs(rh2 * rinv2 - 0.5 * ((u2 * u2 + v2 * v2) + w2 * w2)));
                double sl = std::min(nv1 - beta0 * c1, qt - ct);
                double sr = std::max(nv2 + beta0 * c2, qt + ct);
                sl = std::min(sl, nv2 - beta0 * c2);
                sr = std::max(sr, nv1 + beta0 * c1);
                double sm = roe2 * nv2 * (sr - nv2) - roe1 * nv1 * (sl - nv1);
                sm = (sm + pr1) - pr2;
                double fact = roe2 * (sr - nv2) - roe1 * (sl - nv1);
                if (fact != 0.0) fact = 1.0 / fact;
                sm = fact * sm;
                double fl[5] = {(rnx * ru1 + rny * rv1) + rnz * rw1,
                                (rnx * (ru1 * u1 + pr1) + rny * (ru1 * v1)) + rnz * (ru1 * w1),
                                (rnx * (rv1 * u1) + rny * (rv1 * v1 + pr1)) + rnz * (rv1 * w1),
                                (rnx * (rw1 * u1) + rny * (rw1 * v1)) + rnz * (rw1 * w1 + pr1),
                                (rnx * (rh1 * u1) + rny * (rh1 * v1)) + rnz * (rh1 * w1)};
                double fr[5] = {(rnx * ru2 + rny * rv2) + rnz * rw2,
                                (rnx * (ru2 * u2 + pr2) + rny * (ru2 * v2)) + rnz * (ru2 * w2),
                                (rnx * (rv2 * u2) + rny * (rv2 * v2 + pr2)) + rnz * (rv2 * w2),
                                (rnx * (rw2 * u2) + rny * (rw2 * v2)) + rnz * (rw2 * w2 + pr2),
                                (rnx * (rh2 * u2) + rny * (rh2 * v2)) + rnz * (rh2 * w2)};
                double pls = roe1 * (nv1 - sl) * (nv1 - sm) + pr1;
                double prs = roe2 * (nv2 - sr) * (nv2 - sm) + pr2;
                double ls[5], rs[5];
                double factl = sl - sm;
                if (factl != 0.0) {
                    factl = 1.0 / factl;
                    ls[0] = roe1 * (sl - nv1) * factl;
                    ls[1] = ((sl - nv1) * roe1 * u1 + (pls - pr1) * rnx) * factl;
                    ls[2] = ((sl - nv1) * roe1 * v1 + (pls - pr1) * rny) * factl;
                    ls[3] = ((sl - nv1) * roe1 * w1 + (pls - pr1) * rnz) * factl;
                    ls[4] = (((sl - nv1) * re1 - pr1 * nv1) + pls * sm) * factl;
                } else {
                    ls[0] = roe1; ls[1] = ru1; ls[2] = rv1; ls[3] = rw1; ls[4] = re1;
                }
                double factr = sr - sm;
                if (factr != 0.0) {
                    factr = 1.0 / factr;
                    rs[0] = roe2 * (sr - nv2) * factr;
                    rs[1] = ((sr - nv2) * roe2 * u2 + (prs - pr2) * rnx) * factr;
                    rs[2] = ((sr - nv2) * roe2 * v2 + (prs - pr2) * rny) * factr;
                    rs[3] = ((sr - nv2) * roe2 * w2 + (prs - pr2) * rnz) * factr;
                    rs[4] = (((sr - nv2) * re2 - pr2 * nv2) + prs * sm) * factr;
                } else {
                    rs[0] = roe2; rs[1] = ru2; rs[2] = rv2; rs[3] = rw2; rs[4] = re2;
                }
                double L0[5] = {roe1, ru1, rv1, rw1, re1}, R0[5] = {roe2, ru2, rv2, rw2, re2};
                // the state of the GCL term: r, E of the node and the
                // (reconstructed) momentum outside the star region, the star
                // state inside it (def_par:2046-2085)
                double q[5] = {r1, ru1, rv1, rw1, E1};
                if (sl > 0.0) {
                    for (int k = 0; k < 5; ++k) f[k] = fl[k] * rnorm1;
                } else if (sl <= 0.0 && sm > 0.0) {
                    for (int k = 0; k < 5; ++k) f[k] = (fl[k] + sl * (ls[k] - L0[k])) * rnorm1;
                    for (int k = 0; k < 5; ++k) q[k] = ls[k];
                } else if (sm <= 0.0 && sr >= 0.0) {
                    for (int k = 0; k < 5; ++k) f[k] = (fr[k] + sr * (rs[k] - R0[k])) * rnorm1;
                    for (int k = 0; k < 5; ++k) q[k] = rs[k];
                } else if (sr < 0.0) {
                    for (int k = 0; k < 5; ++k) f[k] = fr[k] * rnorm1;
                    q[0] = r2; q[1] = ru2; q[2] = rv2; q[3] = rw2; q[4] = E2;
                }
                if (ale)
                    for (int k = 0; k < 5; ++k) f[k] = f[k] - q[k] * wgcl;
            }
            for (int k = 0; k < 5; ++k) {
                g.rhs[k][i1] = g.rhs[k][i1] + f[k];
                g.rhs[k][i2] = g.rhs[k][i2] - f[k];
            }
        });
        // boundary faces (def_par:2116-2512), after the GCL terms of each
        // boundary side (def_par:2124-2177; moving meshes)
        const bool ale = c.flowType == 2;
        for_bedges(g, [&](int b) {
            const int i1 = g.b1[b], i2 = g.b2[b], ind = g.bind[b];
            if (ale) {
                const double q1[5] = {g.u[0][i1], g.u[1][i1], g.u[2][i1], g.u[3][i1], g.u[4][i1]};
                const double q2[5] = {g.u[0][i2], g.u[1][i2], g.u[2][i2], g.u[3][i2], g.u[4][i2]};
                if (c.boundaryTerm == 1) {
                    double wgcl = g.bgcl1[b] / c.physicalTimeStep;
                    for (int k = 0; k < 5; ++k) g.rhs[k][i1] = g.rhs[k][i1] - (3. * q1[k] + q2[k]) * wgcl;
                    wgcl = g.bgcl2[b] / c.physicalTimeStep;
                    for (int k = 0; k < 5; ++k) g.rhs[k][i2] = g.rhs[k][i2] - (q1[k] + 3. * q2[k]) * wgcl;
                } else {
                    double wgcl = 4.0 * g.bgcl1[b] / c.physicalTimeStep;
                    for (int k = 0; k < 5; ++k) g.rhs[k][i1] = g.rhs[k][i1] - q1[k] * wgcl;
                    wgcl = 4.0 * g.bgcl2[b] / c.physicalTimeStep;
                    for (int k = 0; k < 5; ++k) g.rhs[k][i2] = g.rhs[k][i2] - q2[k] * wgcl;
                }
            }
            double g1[5], g2[5];
            boundary_flux(g, i1, i2, ind, g.bwx[b], g.bwy[b], g.bwz[b], g1, g2);
            for (int k = 0; k < 5; ++k) g.rhs[k][i1] = g.rhs[k][i1] + g1[k];
            for (int k = 0; k < 5; ++k) g.rhs[k][i2] = g.rhs[k][i2] + g2[k];
        });
    }

    // contributions of one boundary edge to its two nodes
    void boundary_flux(Level &g, int i1, int i2, int ind, double wx, double wy, double wz,
                       double *g1, double *g2) {
        const double gam1 = c.gamma - 1.0;
        for (int k = 0; k < 5; ++k) { g1[k] = 0.0; g2[k] = 0.0; }
        const bool fe = c.boundaryTerm == 1;
        if (ind <= 2 || ind == 9) {  // wall or symmetry (def_par:2182-2257)
            double rnorm = std::sqrt((wx * wx + wy * wy) + wz * wz);
            if (rnorm > 1.0e-10) {
                double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
                double F1[5], F2[5];
                wall_flux(g, i1, rnx, rny, rnz, F1);
                wall_flux(g, i2, rnx, rny, rnz, F2);
                for (int k = 0; k < 5; ++k) {
                    if (fe) { g1[k] = rnorm * (3. * F1[k] + F2[k]); g2[k] = rnorm * (F1[k] + 3. * F2[k]); }
                    else { g1[k] = rnorm * 4. * F1[k]; g2[k] = rnorm * 4. * F2[k]; }
                }
            }
        } else if (ind <= 4) {  // far field: Roe flux against freestream
            double rnorm = std::sqrt((wx * wx + wy * wy) + wz * wz);
            if (rnorm > 1.0e-10) {
                double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
                const double *inf = &c.inflowField[(ind - 3) * 6];
                double F1[5], F2[5];
                farfield_flux(g, i1, rnx, rny, rnz, inf, gam1, F1);
                farfield_flux(g, i2, rnx, rny, rnz, inf, gam1, F2);
                for (int k = 0; k < 5; ++k) {
                    if (fe) { g1[k] = rnorm * (3. * F1[k] + F2[k]); g2[k] = rnorm * (F1[k] + 3. * F2[k]); }
                    else { g1[k] = rnorm * 4. * F1[k]; g2[k] = rnorm * 4. * F2[k]; }
                }
            }
        } else {  // engine faces: average flux (def_par:2447-2511)
            double q1[5], q2[5];
            engine_flux(g, i1, wx, wy, wz, q1);
            engine_flux(g, i2, wx, wy, wz, q2);
            for (int k = 0; k < 5; ++k) {
                double fs = q1[k] + q2[k];
                g1[k] = fs + 2.0 * q1[k];
                g2[k] = fs + 2.0 * q2[k];
            }
        }
    }

    void wall_flux(Level &g, int i, double rnx, double rny, double rnz, double *F) {
        double pr = g.p[i], rho = g.u[0][i], rinv = 1. / rho;
        double ru = g.u[1][i], rv = g.u[2][i], rw = g.u[3][i], rh = g.u[4][i] + pr;
        double uu = ru * rinv, vv = rv * rinv, ww = rw * rinv;
        double nv = (uu * rnx + vv * rny) + ww * rnz;
        F[0] = rho * nv;
        F[1] = pr * rnx + rho * uu * nv;
        F[2] = pr * rny + rho * vv * nv;
        F[3] = pr * rnz + rho * ww * nv;
        F[4] = rh * nv;
    }

    // Roe flux between a node state and the freestream (def_par:2258-2419)
    void farfield_flux(Level &g, int i, double rnx, double rny, double rnz, const double *inf,
                       double gam1, double *F) {
        double ro = inf[0], ro1 = 1. / ro, uo = inf[1], vo = inf[2], wo = inf[3], eo = inf[4], po = inf[5];
        double prl = g.p[i], rhol = g.u[0][i], rinvl = 1. / rhol;
        double rul = g.u[1][i], rvl = g.u[2][i], rwl = g.u[3][i], rhl = g.u[4][i] + prl;
        double ul = rul * rinvl, vl = rvl * rinvl, wl = rwl * rinvl;
        double epsl = g.u[4][i], hl = rhl * rinvl;
        double nvl = (ul * rnx + vl * rny) + wl * rnz;
        double fl1 = rhol * nvl, fl2 = prl * rnx + rhol * ul * nvl, fl3 = prl * rny + rhol * vl * nvl;
        double fl4 = prl * rnz + rhol * wl * nvl, fl5 = rhl * nvl;
        double rhor = ro, uxr = uo, vyr = vo, wzr = wo, epsr = eo * ro, presr = po, hr = eo + po * ro1;
        double unr = (uxr * rnx + vyr * rny) + wzr * rnz;
        double fr1 = rhor * unr, fr2 = rnx * presr + rhor * uxr * unr, fr3 = rny * presr + rhor * vyr * unr;
        double fr4 = rnz * presr + rhor * wzr * unr, fr5 = (epsr + presr) * unr;
        double di = std::sqrt(rhor / rhol), d1 = 1.0 / (di + 1.0);
        double ui = (di * uxr + ul) * d1, vi = (di * vyr + vl) * d1, wi = (di * wzr + wl) * d1;
        double hi = (di * hr + hl) * d1;
        double ci2 = gam1 * (hi - 0.5 * ((ui * ui + vi * vi) + wi * wi));
        ci2 = std::max(ci2, 1.0e-5);
        double ci = std::sqrt(ci2);
        double af = 0.5 * ((ui * ui + vi * vi) + wi * wi);
        double ucp = (ui * rnx + vi * rny) + wi * rnz;
        double du1 = rhor - rhol, du2 = rhor * uxr - rhol * ul, du3 = rhor * vyr - rhol * vl;
        double du4 = rhor * wzr - rhol * wl, du5 = epsr - epsl;
        double l1 = std::fabs(ucp + ci), l2 = std::fabs(ucp - ci), l3 = std::fabs(ucp);
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

    void engine_flux(Level &g, int i, double wx, double wy, double wz, double *F) {
        double pr = g.p[i], r = g.u[0][i], rinv = 1. / g.u[0][i];
        double ru = g.u[1][i], rv = g.u[2][i], rw = g.u[3][i];
        double uu = rinv * ru, vv = rinv * rv, ww = rinv * rw, E = g.u[4][i];
        double pu = pr * rinv * ru, pv = pr * rinv * rv, pw = pr * rinv * rw;
        F[0] = (wx * r * uu + wy * r * vv) + wz * r * ww;
        F[1] = (wx * (ru * uu + pr) + wy * ru * vv) + wz * ru * ww;
        F[2] = (wx * rv * uu + wy * (rv * vv + pr)) + wz * rv * ww;
        F[3] = (wx * rw * uu + wy * rw * vv) + wz * (rw * ww + pr);
        F[4] = (wx * (E * uu + pu) + wy * (E * vv + pv)) + wz * (E * ww + pw);
    }

    bool sa() const { return c.turbulenceModel == 1; }

    // ---- makeTurbulentTimeSteps (def_par:12878-13100) ---------------------
    void makeTurbulentTimeSteps(Level &g) {
        const double oneOverSigma = 3.0 / 2.0, oneOverKappaSquared = 1.0 / (0.41 * 0.41);
        const double cb1 = 0.1355, cb2 = 0.622, ct3 = 1.1;
        const double cw1 = cb1 * oneOverKappaSquared + (1.0 + cb2) * oneOverSigma;
        const double oRe = 1.0 / c.ReynoldsNumber;
        vec &h = nh[0];
        std::fill(g.dtT.begin(), g.dtT.end(), 0.0);
        std::fill(h.begin(), h.end(), 0.0);
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
            double al = (wx * wx + wy * wy) + wz * wz;
            double ro1 = 1. / g.u[0][i1], ro2 = 1. / g.u[0][i2];
            double vn1 = ((wx * g.u[1][i1] + wy * g.u[2][i1]) + wz * g.u[3][i1]) * ro1;
            double vn2 = ((wx * g.u[1][i2] + wy * g.u[2][i2]) + wz * g.u[3][i2]) * ro2;
            vn1 = c.turbK * std::sqrt(al) + std::fabs(vn1);
            vn2 = c.turbK * std::sqrt(al) + std::fabs(vn2);
            g.dtT[i1] = g.dtT[i1] + vn1;
            g.dtT[i2] = g.dtT[i2] + vn2;
            double vis1 = oneOverSigma * (g.mu[i1] + 3.0 * cb2 * g.u[5][i1] * oRe);
            double vis2 = oneOverSigma * (g.mu[i2] + 3.0 * cb2 * g.u[5][i2] * oRe);
            double dv1 = 2.0 * vis1 * al, dv2 = 2.0 * vis2 * al;
            h[i1] = h[i1] + dv2;
            h[i2] = h[i2] + dv1;
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double wx = g.bwx[b], wy = g.bwy[b], wz = g.bwz[b];
            double al = (wx * wx + wy * wy) + wz * wz;
            double ro1 = 1. / g.u[0][i1], ro2 = 1. / g.u[0][i2];
            double vn1 = ((wx * g.u[1][i1] + wy * g.u[2][i1]) + wz * g.u[3][i1]) * ro1;
            double vn2 = ((wx * g.u[1][i2] + wy * g.u[2][i2]) + wz * g.u[3][i2]) * ro2;
            vn1 = c.turbK * std::sqrt(al) + std::fabs(vn1);
            vn2 = c.turbK * std::sqrt(al) + std::fabs(vn2);
            double vnm = vn1 + vn2;
            g.dtT[i1] = (g.dtT[i1] + vn1) + vnm;
            g.dtT[i2] = (g.dtT[i2] + vn2) + vnm;
            double vis1 = oneOverSigma * (g.mu[i1] + 3.0 * cb2 * g.u[5][i1] * oRe);
            double vis2 = oneOverSigma * (g.mu[i2] + 3.0 * cb2 * g.u[5][i2] * oRe);
            double dv1 = 2.0 * vis1 * al, dv2 = 2.0 * vis2 * al;
            double dvm = dv1 + dv2;
            h[i1] = (h[i1] + dv1) + dvm;
            h[i2] = (h[i2] + dv2) + dvm;
        });
        for_nodes(g.N, [&](int i) {
            double V = g.V[i];
            g.dtT[i] = 0.5 / (g.dtT[i] / V + h[i] / (V * V));
            double dt = g.dtT[i];
            double dInvSquared = g.wdist[i] > 1.0e-10 ? 1.0 / g.wdist[i] : 1.0e10;
            dInvSquared = dInvSquared * dInvSquared;
            double S = (std::fabs(g.divg[i]) +
                        cb1 * (g.vort[i] + (1.0 + ct3) * g.u[5][i] * oneOverKappaSquared * dInvSquared * oRe)) +
                       cw1 * g.u[5][i] * dInvSquared * oRe;
            g.dtT[i] = dt / (1.0 + 0.5 * S * dt);
        });
    }

    // ---- makeSADiffusion (def_par:7436-7809) ------------------------------
    void makeSADiffusion(Level &g) {
        const double sigma = 2. / 3., cb2 = 0.622, oRe = 1. / c.ReynoldsNumber;
        std::fill(g.turbDiff.begin(), g.turbDiff.end(), 0.0);
        for (int k = 8; k < 14; ++k) std::fill(nh[k].begin(), nh[k].begin() + g.N, 0.0);
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double t1 = g.u[5][i1], t2 = g.u[5][i2];
            double f1 = g.wx[e] * (t1 + t2), f2 = g.wy[e] * (t1 + t2), f3 = g.wz[e] * (t1 + t2);
            nh[8][i1] = nh[8][i1] + f1; nh[8][i2] = nh[8][i2] - f1;
            nh[9][i1] = nh[9][i1] + f2; nh[9][i2] = nh[9][i2] - f2;
            nh[10][i1] = nh[10][i1] + f3; nh[10][i2] = nh[10][i2] - f3;
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double wx = g.bwx[b], wy = g.bwy[b], wz = g.bwz[b];
            double t1 = g.u[5][i1], t2 = g.u[5][i2];
            if (c.boundaryTerm == 1) {
                nh[8][i1] = nh[8][i1] + (3. * t1 + t2) * wx; nh[8][i2] = nh[8][i2] + (t1 + 3. * t2) * wx;
                nh[9][i1] = nh[9][i1] + (3. * t1 + t2) * wy; nh[9][i2] = nh[9][i2] + (t1 + 3. * t2) * wy;
                nh[10][i1] = nh[10][i1] + (3. * t1 + t2) * wz; nh[10][i2] = nh[10][i2] + (t1 + 3. * t2) * wz;
            } else {
                nh[8][i1] = nh[8][i1] + 4. * t1 * wx; nh[8][i2] = nh[8][i2] + 4. * t2 * wx;
                nh[9][i1] = nh[9][i1] + 4. * t1 * wy; nh[9][i2] = nh[9][i2] + 4. * t2 * wy;
                nh[10][i1] = nh[10][i1] + 4. * t1 * wz; nh[10][i2] = nh[10][i2] + 4. * t2 * wz;
            }
        });
        std::fill(nh[0].begin(), nh[0].end(), 0.0);
        double fact = oRe * cb2 / sigma;
        for_nodes(g.N, [&](int i) {
            double vt = 1. / g.V[i];
            double dx = nh[8][i] * vt, dy = nh[9][i] * vt, dz = nh[10][i] * vt;
            nh[11][i] = dx; nh[12][i] = dy; nh[13][i] = dz;
            double vp = (nh[8][i] * dx + nh[9][i] * dy) + nh[10][i] * dz;
            nh[0][i] = nh[0][i] - fact * vp;
        });
        fact = oRe / sigma;
        auto visc = [&](int i) { return c.ReynoldsNumber * g.mu[i] / g.u[0][i] + g.u[5][i]; };
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
            double fd1 = visc(i1) * ((wx * nh[11][i1] + wy * nh[12][i1]) + wz * nh[13][i1]);
            double fd2 = visc(i2) * ((wx * nh[11][i2] + wy * nh[12][i2]) + wz * nh[13][i2]);
            g.turbDiff[i1] = g.turbDiff[i1] - fact * (fd1 + fd2);
            g.turbDiff[i2] = g.turbDiff[i2] + fact * (fd1 + fd2);
        });
        for_bedges(g, [&](int b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            double wx = g.bwx[b], wy = g.bwy[b], wz = g.bwz[b];
            double fd1 = visc(i1) * ((wx * nh[11][i1] + wy * nh[12][i1]) + wz * nh[13][i1]);
            double fd2 = visc(i2) * ((wx * nh[11][i2] + wy * nh[12][i2]) + wz * nh[13][i2]);
            if (c.boundaryTerm == 1) {
                g.turbDiff[i1] = g.turbDiff[i1] - fact * (3. * fd1 + fd2);
                g.turbDiff[i2] = g.turbDiff[i2] - fact * (fd1 + 3. * fd2);
            } else {
                g.turbDiff[i1] = g.turbDiff[i1] - fact * 4. * fd1;
                g.turbDiff[i2] = g.turbDiff[i2] - fact * 4. * fd2;
            }
        });
        for_nodes(g.N, [&](int i) { g.turbDiff[i] = g.turbDiff[i] + nh[0][i]; });
    }

    // ---- makeSARHS (def_par:6809-6950): upwinded convection of nu~ ---------
    void makeSARHS(Level &g) {
        for_edges(g, [&](int e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            double rinv1 = 1. / g.u[0][i1], t1 = g.u[5][i1];
            double u1 = rinv1 * g.u[1][i1], v1 = rinv1 * g.u[2][i1], w1 = rinv1 * g.u[3][i1];
            double rinv2 = 1. / g.u[0][i2], t2 = g.u[5][i2];
            double u2 = rinv2 * g.u[1][i2], v2 = rinv2 * g.u[2][i2], w2 = rinv2 * g.u[3][i2];
            double wx = g.wx[e], wy = g.wy[e], wz = g.wz[e];
            double fconv = (wx * (u1 * t1 + u2 * t2) + wy * (v1 * t1 + v2 * t2)) + wz * (w1 * t1 + w2 * t2);
            if (std::fabs(t1 - t2) > 1.0e-20) {
                double ax = (u2 * t2 - u1 * t1) / (t1 - t2);
                double ay = (v2 * t2 - v1 * t1) / (t1 - t2);
                double az = (w2 * t2 - w1 * t1) / (t1 - t2);
                fconv = fconv + std::fabs((wx * ax + wy * ay) + wz * az) * (t1 - t2);
            }
            g.rhs[5][i1] = g.rhs[5][i1] + fconv;
            g.rhs[5][i2] = g.rhs[5][i2] - fconv;
        });
    }

    // ---- makeSASourceTerm (def_par:9285-9371) -----------------------------
    // The laminar viscosity floor writes 0.1*Re (not 0.1/Re) into the array,
    // as the reference does (def_par:9321-9323).
    void makeSASourceTerm(Level &g) {
        using namespace flite_pm;
        const double oRe = 1. / c.ReynoldsNumber;
        const double cb1 = 0.1355, cb2 = 0.622, kappa = 0.41, kappaSquared = kappa * kappa, sigma = 2. / 3.;
        const double cw1 = cb1 / kappaSquared + (1.0 + cb2) / sigma;
        const double cw2 = 0.3, cw3 = 2.0, cv1 = 7.1, ct3 = 1.1, ct4 = 2.0;
        const double cv1Tripled = pm_cube(cv1), cw3InSixth = pm_pow6(cw3), oneOverSix = 1. / 6.;
        const double cFact = pm_exp(oneOverSix * pm_log(1.0 + cw3InSixth));
        for_nodes(g.N, [&](int i) {
            double vt = g.V[i];
            double mucurl = std::max(g.u[5][i], 0.0);
            if (g.mu[i] < 0.1 / c.ReynoldsNumber) g.mu[i] = 0.1 * c.ReynoldsNumber;
            double Ksi = g.u[0][i] * oRe * mucurl / g.mu[i];
            Ksi = std::max(Ksi, 0.001);
            double ft2 = ct3 * pm_exp(-ct4 * Ksi * Ksi);
            double K3 = pm_cube(Ksi);
            double d = std::max(g.wdist[i], 1.0e-10);
            double muOverd = mucurl / d, dSquared = d * d;
            double fv1 = K3 / (K3 + cv1Tripled);
            double fv2 = 1.0 - (Ksi / (1.0 + Ksi * fv1));
            double fv3 = 1.0;
            double Scurl = fv3 * g.vort[i] + oRe * mucurl * fv2 / (kappaSquared * dSquared);
            double r;
            if (std::fabs(Scurl) > 1.0e-10) {
                r = oRe * mucurl / (Scurl * kappaSquared * dSquared);
                if (r < 0.0) r = 0.0;
                if (r > 100.0) r = 100.0;
            } else {
                r = 100.0;
            }
            double gg = r + cw2 * (pm_pow6(r) - r);
            double radicand = (1.0 + cw3InSixth) / (pm_pow6(gg) + cw3InSixth);
            double fw = radicand > 1.0e-10 ? gg * pm_exp(oneOverSix * pm_log(radicand)) : cFact;
            g.rhs[5][i] = g.rhs[5][i] - vt * cb1 * (1.0 - ft2) * Scurl * mucurl;
            g.rhs[5][i] = g.rhs[5][i] + oRe * vt * (cw1 * fw - cb1 * ft2 / kappaSquared) * muOverd * muOverd;
            g.rhs[5][i] = g.rhs[5][i] - vt * mucurl * g.divg[i];
        });
    }

    // ---- limitTurbulence (def_par:1259-1290): a is floored at zero; the
    // state's nu~ (not a) is capped at maxTurbulenceValue
    void limitTurbulence(Level &g, vec &a) {
        for (int i = 0; i < g.N; ++i) {
            a[i] = std::max(a[i], 0.0);
            if (g.u[5][i] > c.maxTurbulenceValue) g.u[5][i] = c.maxTurbulenceValue;
        }
    }

    // ---- nullifyOuterBoundary (def_par:4254-4362), SA: components 1..6 of
    // the far-field (indicator 3) and engine nodes
    void nullifyOuterBoundary(Level &g, vec *u) {
        if (!sa()) return;
        const int ranges[5][2] = {{-16, -15}, {-12, -11}, {-10, -9}, {-8, -7}, {-6, -5}};
        for (auto &rg : ranges)
            for_range(g, rg[0], rg[1], [&](int ip) {
                for (int k = 0; k < 6; ++k) u[k][ip] = 0.0;
            });
    }

    // ---- solveSystem (def_par:1407-1479) + solveTurbulenceSystem
    // (def_par:1481-1522) -------------------------------------------------
    void solveSystem(Level &g, vec *rhs) {
        // flowType != 0: the dual-time step dt / (1 + 1.5 dt / physicalTimeStep),
        // or under explicit time stepping ivd%physicalTimeStep for every node
        // (def_par:1427-1442; solveTurbulenceSystem :1505-1517)
        const bool unsteady = c.flowType != 0;
        const bool glob = unsteady && c.explicit_;
        for_nodes(g.N, [&](int i) {
            double dt = g.dt[i];
            if (glob) dt = pts_global;
            else if (unsteady) dt = dt / (1.0 + 1.5 * dt / c.physicalTimeStep);
            for (int k = 0; k < 5; ++k) rhs[k][i] = dt * rhs[k][i] / g.V[i];
        });
        if (sa()) for_nodes(g.N, [&](int i) { rhs[5][i] = (glob ? pts_global : g.dtT[i]) * rhs[5][i] / g.V[i]; });
    }

    double relaxation_param(const Level &g) const {
        if (c.numberOfCFLIncrements > 0) {
            double r = (double)(g.cycleNumber - 1) / (double)c.numberOfCFLIncrements;
            return std::min(r, 1.0);
        }
        return 1.0;
    }

    template <class Fn>
    void for_range(const Level &g, int a, int b, Fn fn) {
        for (int ib = g.R(a); ib <= g.R(b); ++ib) fn(g.node_ind[ib - 1]);
    }

    void remove_normal(Level &g, vec *x, int ip, double scale) {
        double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
        double nv = (x[1][ip] * n[0] + x[2][ip] * n[1]) + x[3][ip] * n[2];
        for (int k = 0; k < 3; ++k) x[1 + k][ip] = x[1 + k][ip] - scale * nv * n[k];
    }

    // ---- setBCsOnIncrementField (def_par:4978-5140) -----------------------
    void setBCsOnIncrementField(Level &g, vec *rhs) {
        const bool t = sa();
        if (c.ReynoldsNumber > 0) {
            for_range(g, -20, -19, [&](int ip) {
                rhs[1][ip] = 0.0; rhs[2][ip] = 0.0; rhs[3][ip] = 0.0;
                if (!c.wallsAreIsentropic) rhs[4][ip] = 0.0;
                if (t) rhs[5][ip] = 0.0;
            });
        } else {
            for_range(g, -20, -19, [&](int ip) {
                remove_normal(g, rhs, ip, 1.0);
                if (t) rhs[5][ip] = 0.0;
            });
        }
        for_range(g, -4, -3, [&](int ip) {
            remove_normal(g, rhs, ip, 1.0);
            if (t) rhs[5][ip] = 0.0;
        });
        for_range(g, -18, -17, [&](int ip) { remove_normal(g, rhs, ip, 1.0); });
        // engine inlets relaxed, engine exhausts held (def_par:5084-5125)
        for (int r : {-12, -10})
            for_range(g, r, r + 1, [&](int ip) {
                for (int k = 0; k < nvar; ++k) rhs[k][ip] = c.engineBCRelaxation * rhs[k][ip];
            });
        for (int r : {-8, -6})
            for_range(g, r, r + 1, [&](int ip) {
                for (int k = 0; k < nvar; ++k) rhs[k][ip] = 0.0;
            });
    }

    // ---- updateSolutionVector (def_par:1292-1405); u may alias delu -------
    void updateSolutionVector(Level &g, vec *u, vec *uprev, vec *delu, int rk) {
        double dtJ = rk > 0 ? c.CFLNumber * RK[rk - 1] : c.CFLNumber;
        for (int k = 0; k < 5; ++k)
            for_nodes(g.N, [&](int i) { delu[k][i] = dtJ * delu[k][i]; });
        for_nodes(g.N, [&](int i) {
            double inc = delu[0][i];
            if (std::fabs(inc / uprev[0][i]) < c.maxIncrementFactor) {
                u[0][i] = uprev[0][i] - inc;
            } else {
                double sign = inc / std::fabs(inc);
                u[0][i] = uprev[0][i] - sign * c.maxIncrementFactor * uprev[0][i];
            }
            for (int k = 1; k < 5; ++k) u[k][i] = uprev[k][i] - delu[k][i];
        });
        if (sa()) {
            const double dtT = rk > 0 ? c.turbulentCFLNumber * RK[rk - 1] : c.turbulentCFLNumber;
            for_nodes(g.N, [&](int i) {
                delu[5][i] = dtT * delu[5][i];
                u[5][i] = uprev[5][i] - delu[5][i];
                u[5][i] = std::max(u[5][i], 0.0);
            });
        }
        for_nodes(g.N, [&](int i) { if (g.u[0][i] < c.minimumDensity) g.u[0][i] = c.minimumDensity; });
    }

    // ---- setBCsOnSolutionField (def_par:4364-4976), static walls ----------
    void setBCsOnSolutionField(Level &g, vec *u) {
        const double relax = relaxation_param(g);
        if (c.ReynoldsNumber > 0) {
            for_range(g, -20, -19, [&](int ip) {
                double cm[3] = {g.cmx[ip], g.cmy[ip], g.cmz[ip]};
                for (int k = 0; k < 3; ++k) u[1 + k][ip] = u[0][ip] * cm[k] / c.physicalTimeStep;
                if (!c.wallsAreIsentropic) u[4][ip] = u[0][ip] * c.inflowTemperature / c.gamma;
                if (sa()) u[5][ip] = 0.0;
            });
        } else {
            // the wall velocity term adds grp%u(ip,1)*0*normal for a steady
            // run (def_par:4445-4456): the tangential projection only
            for_range(g, -20, -19, [&](int ip) {
                remove_normal(g, u, ip, 1.0);
                if (sa()) u[5][ip] = 0.0;
            });
        }
        for_range(g, -4, -3, [&](int ip) {
            remove_normal(g, u, ip, relax);
            if (!c.wallsAreIsentropic) {
                double ke = (u[1][ip] * u[1][ip] + u[2][ip] * u[2][ip]) + u[3][ip] * u[3][ip];
                u[4][ip] = u[0][ip] * c.inflowTemperature / c.gamma + 0.5 * ke / u[0][ip];
            }
            if (sa()) u[5][ip] = 0.0;
        });
        for_range(g, -18, -17, [&](int ip) { remove_normal(g, u, ip, 1.0); });
        if (engines) engine_conditions(g, u);
    }

    // ---- engine conditions of setBCsOnSolutionField (def_par:4488-4918) ----
    // The exhausts take the ramped exhaust state, and its pressure into grp%p;
    // on level 1 the inlets' momenta are scaled to the target mass flow
    // (engineFlowType 1) or mass flow function (2) with the internal energy
    // of grp%u kept, and an inflow through an inlet is turned out.  u is the
    // array the conditions act on (grp%u, or the candidate state of
    // restrictGrid's fine step); grp%u and grp%p are the level's.
    double eo_relax(const Level &g) const {  // def_par:4490-4495
        if (c.numberOfEORelaxationSteps > 0) {
            double r = (double)(g.cycleNumber - 1) / (double)c.numberOfEORelaxationSteps;
            return std::min(r, 1.0);
        }
        return 1.0;
    }
    static double ke(const vec *u, int i) { return (u[1][i] * u[1][i] + u[2][i] * u[2][i]) + u[3][i] * u[3][i]; }

    // Sums over the engine inlet sides in the device's fixed order: side s
    // goes to partial kEngineLanes-strided sums (s mod kEngineLanes), in side
    // order, and the partials meet in a pairwise tree.  The reference sums in
    // side order on each domain and then over the domains.
    static constexpr int kEngineLanes = 256;
    template <class Term>
    void engine_sums(const Level &g, int nq, Term term, double (*out)[2]) {
        std::vector<double> part((size_t)nq * 2 * kEngineLanes, 0.0);
        const int n = (int)g.e1.size();
        for (int s = 0; s < n; ++s) {
            double q[3];
            term(s, q);
            const size_t base = ((size_t)g.ein[s] * nq) * kEngineLanes + s % kEngineLanes;
            for (int k = 0; k < nq; ++k) part[base + (size_t)k * kEngineLanes] += q[k];
        }
        for (int e = 0; e < 2; ++e)
            for (int k = 0; k < nq; ++k) {
                double *a = &part[((size_t)e * nq + k) * kEngineLanes];
                for (int w = kEngineLanes / 2; w >= 1; w /= 2)
                    for (int t = 0; t < w; ++t) a[t] = a[t] + a[t + w];
                out[k][e] = a[0];
            }
    }

    void engine_conditions(Level &g, vec *u) {
        const double rp = eo_relax(g);
        for (int e = 0; e < 2; ++e) {  // exhausts (def_par:4497-4540)
            const double *rear = &c.enginesRearParameters[7 * e];
            for_range(g, e == 0 ? -8 : -6, e == 0 ? -7 : -5, [&](int ip) {
                for (int k = 0; k < 5; ++k) u[k][ip] = (1.0 - rp) * c.inflowField[k] + rp * rear[k];
                g.p[ip] = (1.0 - rp) * c.inflowField[5] + rp * rear[5];
                if (sa()) u[5][ip] = rp * rear[6];
            });
        }
        if (g.grid != 1) return;  // the inlet terms act on level 1 only
        double fac[2] = {1.0, 1.0};  // the reference's is uninitialised where the flow is not positive
        bool scale = true;
        if (c.engineFlowType == 1) {  // def_par:4541-4599
            double s[1][2];
            engine_sums(g, 1, [&](int q, double *t) {
                const int a = g.e1[q], b = g.e2[q];
                const double w[3] = {g.ewx[q], g.ewy[q], g.ewz[q]};
                const double s1 = (u[1][a] * w[0] + u[2][a] * w[1]) + u[3][a] * w[2];
                const double s2 = (u[1][b] * w[0] + u[2][b] * w[1]) + u[3][b] * w[2];
                t[0] = s1 + s2;
            }, s);
            for (int e = 0; e < 2; ++e)
                if (s[0][e] > 0.0) fac[e] = c.enginesFrontMassFlow[e] / s[0][e];
        } else if (c.engineFlowType == 2) {  // def_par:4689-4806
            double s[3][2];
            engine_sums(g, 3, [&](int q, double *t) {
                const int a = g.e1[q], b = g.e2[q];
                const double w[3] = {g.ewx[q], g.ewy[q], g.ewz[q]};
                const double s1 = (u[1][a] * w[0] + u[2][a] * w[1]) + u[3][a] * w[2];
                const double s2 = (u[1][b] * w[0] + u[2][b] * w[1]) + u[3][b] * w[2];
                const double press = 0.5 * ((g.p[a] + 0.5 * ke(u, a) / u[0][a]) + (g.p[b] + 0.5 * ke(u, b) / u[0][b]));
                const double temp1 = (c.gamma / u[0][a]) * (u[4][a] - (0.5 * ke(u, a)) / u[0][a]);
                const double temp2 = (c.gamma / u[0][b]) * (u[4][b] - (0.5 * ke(u, b)) / u[0][b]);
                const double temp = 0.5 * (temp1 + temp2);
                const double wn = std::sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]);
                t[0] = s1 + s2;
                t[1] = (std::sqrt(temp) / press) * 2.0 * wn;
                t[2] = 2.0 * wn;
            }, s);
            for (int e = 0; e < 2 && scale; ++e) {
                if (!(s[0][e] > 0.0)) continue;
                const double mff = s[0][e] * (s[1][e] / s[2][e]);
                fac[e] = c.enginesFrontMassFlow[e] / mff;
                if (fac[e] > 99999999999.) scale = false;  // the goto 9999 past the scaling
            }
        }
        if (scale) {  // def_par:4615-4649, 4827-4860
            for (int e = 0; e < 2; ++e)
                for_range(g, e == 0 ? -12 : -10, e == 0 ? -11 : -9, [&](int ip) {
                    const double intE = g.u[4][ip] - 0.5 * ke(g.u, ip) / g.u[0][ip];
                    for (int k = 1; k < 4; ++k) u[k][ip] = u[k][ip] * fac[e];
                    u[4][ip] = intE + 0.5 * ke(u, ip) / u[0][ip];
                    if (sa()) u[5][ip] = 0.0;
                });
            if (c.engineFlowType == 2) makePressureField(g, g.u);  // def_par:4864
        }
        for (int e = 0; e < 2; ++e)  // no inflow through an inlet (def_par:4653-4686)
            for_range(g, e == 0 ? -12 : -10, e == 0 ? -11 : -9, [&](int ip) {
                const double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
                const double nv = (((-n[0]) * u[1][ip] + (-n[1]) * u[2][ip]) + (-n[2]) * u[3][ip]) / u[0][ip];
                if (nv < 0.00)
                    for (int k = 0; k < 3; ++k) u[1 + k][ip] = u[1 + k][ip] + u[0][ip] * (nv - 0.01) * n[k];
            });
    }

    // ---- setOuterBoundaryConditions (def_par:4018-4251) -------------------
    void setOuterBoundaryConditions(Level &g, vec *u, const vec &p) {
        const double gm1 = c.gamma - 1.0;
        for (int side = 0; side < 2; ++side) {
            const double *inf = &c.inflowField[side * 6];
            double iR = inf[0], iU1 = inf[1], iU2 = inf[2], iU3 = inf[3], iE = inf[4], iP = inf[5];
            for_range(g, side == 0 ? -16 : -14, side == 0 ? -15 : -13, [&](int ip) {
                double rho = u[0][ip], U1 = u[1][ip], U2 = u[2][ip], U3 = u[3][ip];
                double nvel = (iU1 * g.nx[ip] + iU2 * g.ny[ip]) + iU3 * g.nz[ip];
                if (nvel > 0.00) {
                    if (c.MachNumber > 1.0) {
                        u[0][ip] = iR; u[1][ip] = iU1 * iR; u[2][ip] = iU2 * iR; u[3][ip] = iU3 * iR;
                        u[4][ip] = iE * iR;
                    } else {
                        u[0][ip] = iR; u[1][ip] = iU1 * iR; u[2][ip] = iU2 * iR; u[3][ip] = iU3 * iR;
                        u[4][ip] = p[ip] / gm1 + 0.5 * ((iU1 * iU1 + iU2 * iU2) + iU3 * iU3) * iR;
                    }
                } else {
                    if (c.MachNumber < 1.0) u[4][ip] = iP / gm1 + 0.5 * ((U1 * U1 + U2 * U2) + U3 * U3) / rho;
                }
                if (sa()) u[5][ip] = 0.1;  // every branch (def_par:4076-4140)
            });
        }
    }

    void limitDensity(Level &g) {
        for_nodes(g.N, [&](int i) { g.u[0][i] = std::max(g.u[0][i], c.minimumDensity); });
    }

    // singleIteration (def_par:1030-1036) and restrictGrid's fine part
    // (def_par:12269-12273): scheme 1 acts on level 1 only
    void dissipation_for(Level &g, bool in_restrict_fine) {
        if (c.dissipationScheme == 1 && g.grid == 1) { makeArtificialDissipation1(g); return; }
        if (in_restrict_fine) { makeArtificialDissipation2(g); return; }
        if (c.dissipationScheme == 3) makeArtificialDissipation3(g);
        else makeArtificialDissipation2(g);
    }

    // ---- addTimeDifferences (def_par:1184-1241): on a static mesh the
    // previous volumes are the volumes ----------------------------------------
    void addTimeDifferences(Level &g) {
        if (c.flowType == 0 || c.explicit_) return;  // addTimeStep (def_par:386-394, 1195)
        const double dtp = c.physicalTimeStep;
        if (g.grid == 1 && c.timeScheme == 2) {
            const vec &Vp = c.flowType == 2 ? g.Vp : g.V, &Vp2 = c.flowType == 2 ? g.Vp2 : g.V;
            for (int i = 0; i < g.N; ++i)
                for (int k = 0; k < nvar; ++k)
                    g.rhs[k][i] = g.rhs[k][i] + (((1.5 * g.V[i]) * g.u[k][i] - (2.0 * Vp[i]) * g.uold[k][i]) +
                                                 (0.5 * Vp2[i]) * g.uold2[k][i]) / dtp;
        } else {
            for (int i = 0; i < g.N; ++i)
                for (int k = 0; k < nvar; ++k)
                    g.rhs[k][i] = g.rhs[k][i] + g.V[i] * (g.u[k][i] - g.uold[k][i]) / dtp;
        }
    }

    // ---- singleIteration (def_par:1002-1181) ------------------------------
    void singleIteration(Level &g, bool calcDiss, bool calcTurb) {
        const bool turb = sa() && calcTurb;
        if (calcDiss) {
            makePressureField(g, g.u);
            for_nodes(g.N, [&](int i) { g.p[i] = std::fabs(g.p[i]); });
            makeTimeSteps(g);
            dissipation_for(g, false);
            if (c.ReynoldsNumber > 0.0) {
                viscousTerm(g);
                if (turb) {
                    makeTurbulentTimeSteps(g);
                    makeSADiffusion(g);
                }
            }
        }
        for (int st = 1; st <= nstage; ++st) {
            makePressureField(g, g.u);
            for (int k = 0; k < nvar; ++k) std::fill(g.rhs[k].begin(), g.rhs[k].end(), 0.0);
            makeRHS(g);
            addTimeDifferences(g);
            if (turb) {
                // triggerTurbulenceField and makeSATripTerm act on the trip
                // field nodes of a .wid file; none are read (no trip lines)
                makeSARHS(g);
                makeSASourceTerm(g);
            }
            for (int k = 0; k < 5; ++k)
                for_nodes(g.N, [&](int i) { g.rhs[k][i] = g.rhs[k][i] + g.diss[k][i]; });
            if (turb) for_nodes(g.N, [&](int i) { g.rhs[5][i] = g.rhs[5][i] + g.turbDiff[i]; });
            solveSystem(g, g.rhs);
            setBCsOnIncrementField(g, g.rhs);
            if (g.grid > 1) nullifyOuterBoundary(g, g.rhs);
            updateSolutionVector(g, g.u, g.uprev, g.rhs, st);
            setBCsOnSolutionField(g, g.u);
            if (g.grid > 1) {
                for (int k = 0; k < 5; ++k)
                    for_nodes(g.N, [&](int i) { g.u[k][i] = g.u[k][i] - RK[st - 1] * g.src[k][i]; });
                if (turb) for_nodes(g.N, [&](int i) { g.u[5][i] = g.u[5][i] - RK[st - 1] * g.src[5][i]; });
            }
            limitDensity(g);
            if (turb) limitTurbulence(g, g.u[5]);
            setOuterBoundaryConditions(g, g.u, g.p);
        }
    }

    bool calcTurbOfCycle = true;  // cycleNo <= numberOfTurbulenceSteps (mg_par:922-926)

    void doTimeIterations(int l, int nsteps, bool calcDiss, int cycle) {
        Level &g = lv[l];
        g.cycleNumber = cycle;
        for (int s = 0; s < nsteps; ++s) {
            for (int k = 0; k < nvar; ++k) g.uprev[k] = g.u[k];
            singleIteration(g, calcDiss, calcTurbOfCycle);
        }
    }

    // ---- mapFineToCoarse (def_par:12572-12679) ----------------------------
    void mapFineToCoarse(const Level &f, const Level &cg, vec *fu, vec *cu, int ncomp) {
        for (int k = 0; k < ncomp; ++k) {
            std::fill(cu[k].begin(), cu[k].end(), 0.0);
            for (int i = 0; i < f.N; ++i) {
                int pp = cg.parent[i];
                if (pp >= 0) cu[k][pp] = cu[k][pp] + cg.rweight[i] * fu[k][i];
            }
        }
    }
    // ---- mapCoarseToFine, injection (def_par:12681-12783) -----------------
    void mapCoarseToFine(const Level &cg, const Level &f, vec *cu, vec *fu, int ncomp) {
        for (int i = 0; i < f.N; ++i) {
            int pp = cg.parent[i];
            if (pp >= 0)
                for (int k = 0; k < ncomp; ++k) fu[k][i] = cu[k][pp];
        }
    }

    // ---- restrictGrid (def_par:12141-12430) -------------------------------
    void restrictGrid(int fl, bool calcTurb) {
        Level &F = lv[fl], &C = lv[fl + 1];
        const bool turb = sa() && calcTurb;
        const int nv = nvar;
        mapFineToCoarse(F, C, F.u, C.u, nv);
        {   // mapScalarFineToCoarse of the laminar viscosity
            vec m(C.N, 0.0);
            for (int i = 0; i < F.N; ++i) {
                int pp = C.parent[i];
                if (pp >= 0) m[pp] = m[pp] + C.rweight[i] * F.mu[i];
            }
            C.mu = m;
        }
        makePressureField(C, C.u);
        setBCsOnSolutionField(C, C.u);
        setOuterBoundaryConditions(C, C.u, C.p);
        for (int k = 0; k < nv; ++k) C.uprev[k] = C.u[k];
        makePressureField(C, C.u);
        for (int i = 0; i < C.N; ++i) C.p[i] = std::fabs(C.p[i]);
        makeTimeSteps(C);
        if (c.coarseGridDissipationScheme == 2) makeArtificialDissipation2(C);
        else if (c.coarseGridDissipationScheme == 3) makeArtificialDissipation3(C);
        if (c.ReynoldsNumber > 0.0) viscousTerm(C);
        for (int k = 0; k < nv; ++k) std::fill(C.rhs[k].begin(), C.rhs[k].end(), 0.0);
        makeRHS(C);
        if (turb) {
            makeTurbulentTimeSteps(C);
            makeSADiffusion(C);
            makeSARHS(C);
            makeSASourceTerm(C);
        }
        for (int k = 0; k < 5; ++k)
            for (int i = 0; i < C.N; ++i) C.rhs[k][i] = C.rhs[k][i] + C.diss[k][i];
        // the turbulent diffusion is added with or without calculateTurbulence
        // (def_par:12238-12240): the last computed one
        if (sa()) for (int i = 0; i < C.N; ++i) C.rhs[5][i] = C.rhs[5][i] + C.turbDiff[i];
        solveSystem(C, C.rhs);
        setBCsOnIncrementField(C, C.rhs);
        nullifyOuterBoundary(C, C.rhs);
        updateSolutionVector(C, C.u, C.uprev, C.rhs, 0);
        setBCsOnSolutionField(C, C.u);
        setOuterBoundaryConditions(C, C.u, C.p);
        for (int k = 0; k < nv; ++k)
            for (int i = 0; i < C.N; ++i) C.src[k][i] = C.u[k][i] - C.uprev[k][i];
        for (int k = 0; k < nv; ++k) C.u[k] = C.uprev[k];
        // fine-grid one-step increment at the current fine state
        makePressureField(F, F.u);
        for (int i = 0; i < F.N; ++i) F.p[i] = std::fabs(F.p[i]);
        dissipation_for(F, true);
        if (c.ReynoldsNumber > 0.0) viscousTerm(F);
        for (int k = 0; k < nv; ++k) std::fill(F.rhs[k].begin(), F.rhs[k].end(), 0.0);
        makeRHS(F);
        if (turb) {
            makeSADiffusion(F);
            makeSARHS(F);
            makeSASourceTerm(F);
        }
        for (int k = 0; k < 5; ++k)
            for (int i = 0; i < F.N; ++i) F.rhs[k][i] = F.rhs[k][i] + F.diss[k][i];
        if (sa()) for (int i = 0; i < F.N; ++i) F.rhs[5][i] = F.rhs[5][i] + F.turbDiff[i];
        solveSystem(F, F.rhs);
        setBCsOnIncrementField(F, F.rhs);
        if (F.grid > 1) nullifyOuterBoundary(F, F.rhs);  // FAS source term allocated
        updateSolutionVector(F, F.rhs, F.uprev, F.rhs, 0);
        setBCsOnSolutionField(F, F.rhs);
        if (F.grid > 1)
            for (int k = 0; k < nv; ++k)
                for (int i = 0; i < F.N; ++i) F.rhs[k][i] = F.rhs[k][i] - F.src[k][i];
        if (sa()) limitTurbulence(F, F.rhs[5]);
        setOuterBoundaryConditions(F, F.rhs, F.p);
        for (int k = 0; k < nv; ++k)
            for (int i = 0; i < F.N; ++i) F.rhs[k][i] = F.rhs[k][i] - F.uprev[k][i];
        mapFineToCoarse(F, C, F.rhs, C.rhs, nv);
        setBCsOnIncrementField(C, C.rhs);
        for (int k = 0; k < nv; ++k)
            for (int i = 0; i < C.N; ++i) C.src[k][i] = C.src[k][i] - C.rhs[k][i];
        for (int k = 0; k < nv; ++k)
            for (int i = 0; i < C.N; ++i) C.u[k][i] = C.u[k][i] + C.rhs[k][i];
    }

    // ---- prolongateGrid (def_par:12432-12570) -----------------------------
    void prolongateGrid(int cl) {
        Level &C = lv[cl], &F = lv[cl - 1];
        const int nv = nvar;
        mapFineToCoarse(F, C, F.u, C.uprev, nv);
        setBCsOnSolutionField(C, C.uprev);
        setOuterBoundaryConditions(C, C.uprev, C.p);
        for (int k = 0; k < nv; ++k)
            for (int i = 0; i < C.N; ++i) C.rhs[k][i] = C.u[k][i] - C.uprev[k][i];
        nullifyOuterBoundary(C, C.rhs);
        setBCsOnIncrementField(C, C.rhs);
        mapCoarseToFine(C, F, C.rhs, F.rhs, nv);
        nullifyOuterBoundary(F, F.rhs);
        for (int k = 0; k < 5; ++k)
            for (int i = 0; i < F.N; ++i) F.rhs[k][i] = c.prolongationRelaxation * F.rhs[k][i];
        if (sa())
            for (int i = 0; i < F.N; ++i) F.rhs[5][i] = c.turbProlongationRelaxation * F.rhs[5][i];
        for (int k = 0; k < 5; ++k)
            for (int i = 0; i < F.Nb; ++i) F.rhs[k][i] = c.multigridBCRelaxation * F.rhs[k][i];
        // the nu~ correction reaches levels finer than numberOfTurbulenceGrids
        const int ncomp = (sa() && F.grid < c.numberOfTurbulenceGrids) ? 6 : 5;
        for (int i = 0; i < F.N; ++i)
            for (int k = 0; k < ncomp; ++k) F.u[k][i] = F.u[k][i] + F.rhs[k][i];
        setBCsOnSolutionField(F, F.u);
        setOuterBoundaryConditions(F, F.u, F.p);
        for (int i = 0; i < F.N; ++i) {
            if (sa()) F.u[5][i] = std::max(F.u[5][i], 0.0);
            F.u[0][i] = std::max(F.u[0][i], c.minimumDensity);
        }
    }

    // ---- oneCycle (mg_par:907-1196) ---------------------------------------
    void oneCycle(int cyc) {
        const int G = (int)lv.size();
        calcTurbOfCycle = cyc <= c.numberOfTurbulenceSteps;
        const bool ct = calcTurbOfCycle;
        const int nr = c.numberOfRelaxationSteps;
        auto relax = [&](int j1, int steps, bool calc) { doTimeIterations(j1 - 1, steps, calc, cyc); };
        auto restr = [&](int j1) { restrictGrid(j1 - 1, ct); };
        auto prol = [&](int j1) { prolongateGrid(j1 - 1); };
        const int s = c.multigridScheme;
        if (s <= 0) {
            for (int i = 1; i <= G - 1; ++i) {
                for (int k = 0; k < nvar; ++k) lv[i - 1].uprev[k] = lv[i - 1].u[k];
                mapFineToCoarse(lv[i - 1], lv[i], lv[i - 1].u, lv[i].u, nvar);
            }
            for (int k = 0; k < nvar; ++k) std::fill(lv[G - 1].src[k].begin(), lv[G - 1].src[k].end(), 0.0);
            relax(G, nr, true);
            for (int i = G; i >= 2; --i) mapCoarseToFine(lv[i - 1], lv[i - 2], lv[i - 1].u, lv[i - 2].u, nvar);
        } else if (s == 1) {
            for (int i = 1; i <= G - 1; ++i) {
                relax(i, nr, i == 1);
                restr(i);
                mapFineToCoarse(lv[i - 1], lv[i], lv[i - 1].u, lv[i].u, nvar);
            }
            relax(G, nr, G == 1);
            for (int i = G; i >= 2; --i) { prol(i); relax(i - 1, nr, (i - 1) == 1); }
        } else if (s == 2 || s == 5) {
            int nsw = G <= 2 ? 1 : 2 * G - 4;
            int fsl = 1;
            for (int i = 1; i <= nsw; ++i) {
                for (int j = fsl; j <= G - 1; ++j) {
                    relax(j, s == 5 ? j : nr, j == fsl);
                    restr(j);
                }
                relax(G, s == 5 ? G : nr, G == 1);
                if (fsl == 1) fsl = G > 2 ? G - 1 : G;
                else if (i <= nsw / 2) fsl = fsl - 1;
                else fsl = fsl + 1;
                for (int j = G; j >= fsl + 1; --j) { prol(j); relax(j - 1, nr, (j - 1) == 1); }
            }
            for (int j = G; j >= 2; --j) { prol(j); relax(j - 1, nr, (j - 1) == 1); }
        } else if (s == 3 || s == 7) {
            int nsw = G == 1 ? 1 : G - 1;
            int fsl = 1;
            for (int i = 1; i <= nsw; ++i) {
                for (int j = fsl; j <= G - 1; ++j) { relax(j, nr, j == fsl); restr(j); }
                relax(G, nr, G == 1);
                if (fsl == 1) fsl = G >= 2 ? G - 1 : G;
                else fsl = fsl - 1;
                for (int j = G; j >= fsl + 1; --j) {
                    prol(j);
                    if (s == 7) relax(j - 1, nr, (j - 1) == 1);
                }
            }
        } else if (s == 4) {
            int nsw = G == 1 ? 1 : G - 1;
            int fsl = 1;
            for (int i = 1; i <= nsw; ++i) {
                for (int j = fsl; j <= G - 1; ++j) { relax(j, nr, j == fsl); restr(j); }
                relax(G, nr, G == 1);
                fsl = fsl + 1;
                for (int j = G; j >= fsl + 1; --j) { prol(j); relax(j - 1, nr, (j - 1) == 1); }
            }
            for (int j = G; j >= 2; --j) { prol(j); relax(j - 1, nr, (j - 1) == 1); }
        } else {
            throw std::runtime_error("Specified multigrid scheme not implemented");
        }
    }

    // ---- geometry set-up of readGridComputationData -----------------------
    void setup_level(Level &g) {
        // makeBoundaryNormals (def_par:15394-15521)
        g.nx.assign(g.N, 0.0); g.ny.assign(g.N, 0.0); g.nz.assign(g.N, 0.0);
        for (int b = 0; b < g.B; ++b) {
            int a = g.b1[b], d = g.b2[b];
            g.nx[a] = g.nx[a] - g.bwx[b]; g.ny[a] = g.ny[a] - g.bwy[b]; g.nz[a] = g.nz[a] - g.bwz[b];
            g.nx[d] = g.nx[d] - g.bwx[b]; g.ny[d] = g.ny[d] - g.bwy[b]; g.nz[d] = g.nz[d] - g.bwz[b];
        }
        for (int i = 0; i < g.Nb; ++i) {
            double nrm = std::sqrt((g.nx[i] * g.nx[i] + g.ny[i] * g.ny[i]) + g.nz[i] * g.nz[i]);
            if (nrm > 1.0e-10) { g.nx[i] = g.nx[i] / nrm; g.ny[i] = g.ny[i] / nrm; g.nz[i] = g.nz[i] / nrm; }
            else { g.nx[i] = 0.0; g.ny[i] = 0.0; g.nz[i] = 0.0; }
        }
        // makeSurfaceArea (def_par:15523-15634), level 1 only
        g.wallArea.assign(g.N, 0.0);
        if (g.grid == 1)
            for (int b = 0; b < g.B; ++b) {
                double ai = std::sqrt((g.bwx[b] * g.bwx[b] + g.bwy[b] * g.bwy[b]) + g.bwz[b] * g.bwz[b]);
                g.wallArea[g.b1[b]] = g.wallArea[g.b1[b]] + 4.0 * ai;
                g.wallArea[g.b2[b]] = g.wallArea[g.b2[b]] + 4.0 * ai;
            }
        // nodeConnectivityArray (def_par:14262-14275)
        g.conn.assign(g.N, 0.0);
        for (int e = 0; e < g.E; ++e) { g.conn[g.s1[e]] += 1.0; g.conn[g.s2[e]] += 1.0; }
    }

    // ---- calculateLiftAndDrag (def_par:14710-14870) -----------------------
    void forces(double *out) {
        Level &g = lv[0];
        const double PI = 4.0 * std::atan(1.0);
        double aR = c.alpha * PI / 180., bR = c.beta * PI / 180.;
        double ft[3] = {std::cos(aR) * std::cos(bR), std::sin(bR), std::sin(aR)};
        double fn1[3] = {-ft[2], 0.0, ft[0]}, fn2[3] = {-ft[1], ft[0], 0.0};
        double lift = 0, drag = 0, latF = 0, fric = 0, latM = 0, longM = 0;
        const double pinf = 1. / (c.gamma * c.MachNumber * c.MachNumber);
        for_range(g, -20, -19, [&](int ip) {
            double h = g.cz[ip];
            double xd = g.cx[ip] - c.datum[0], yd = g.cy[ip] - c.datum[1], zd = g.cz[ip] - c.datum[2];
            if (!(h > (c.groundplane + 0.01))) return;
            double n[3] = {g.nx[ip], g.ny[ip], g.nz[ip]};
            auto dot = [&](const double *a) { return (n[0] * a[0] + n[1] * a[1]) + n[2] * a[2]; };
            double A = g.wallArea[ip], dp = g.p[ip] - pinf;
            lift = lift - A * dp * dot(fn1);
            latF = latF - A * dp * dot(fn2);
            drag = drag - A * dp * dot(ft);
            latM = latM + xd * A * dp * dot(fn2);
            latM = latM - yd * A * dp * dot(ft);
            longM = longM + xd * A * dp * dot(fn1);
            longM = longM - zd * A * dp * dot(ft);
            if (c.ReynoldsNumber > 0.0) {
                double s[3] = {g.wallStress[0][ip], g.wallStress[1][ip], g.wallStress[2][ip]};
                auto sd = [&](const double *a) { return (s[0] * a[0] + s[1] * a[1]) + s[2] * a[2]; };
                lift = lift + A * sd(fn1);
                latF = latF + A * sd(fn2);
                drag = drag + A * sd(ft);
                fric = fric + A * sd(ft);
                latM = latM - xd * A * sd(fn2);
                latM = latM + yd * A * sd(ft);
                longM = longM - xd * A * sd(fn1);
                longM = longM + zd * A * sd(ft);
            }
        });
        out[0] = 2.0 * lift / c.referenceArea;
        out[1] = 2.0 * drag / c.referenceArea;
        out[2] = 2.0 * latF / c.referenceArea;
        out[3] = 2.0 * fric / c.referenceArea;
        out[4] = latM;
        out[5] = longM;
        out[6] = out[7] = out[8] = 0.0;
        if (c.forceCalcType == 3) {
            // writeResiduals (mg_par:1364-1366): calculateLiftAndDrag3
            // replaces lift, drag, latF, latM and adds longMl, longMd, rollM
            double f3[7];
            forces3(f3);
            out[0] = f3[0]; out[1] = f3[1]; out[2] = f3[2]; out[4] = f3[3];
            out[6] = f3[4]; out[7] = f3[5]; out[8] = f3[6];
        }
    }

    // ---- calculateLiftAndDrag3 (def_par:15129-15313) ------------------------
    // The face loads go through the shared nodeHelpArray(:, 1:3), as in the
    // reference (its columns 1..3 are zeroed first and left holding them).
    void forces3(double *out) {
        Level &g = lv[0];
        for (int k = 0; k < 3; ++k) std::fill(nh[k].begin(), nh[k].end(), 0.0);
        const double pinf = 1. / (c.gamma * c.MachNumber * c.MachNumber);
        for (int b = 0; b < g.B; ++b) {
            const int i1 = g.b1[b], i2 = g.b2[b], ind = g.bind[b];
            if (!(ind == 1 || ind == 9)) continue;
            if (!((g.cz[i1] > (c.groundplane + 0.01)) || (g.cz[i2] > (c.groundplane + 0.01)))) continue;
            const double p1 = g.p[i1] - pinf, p2 = g.p[i2] - pinf;
            const double w[3] = {g.bwx[b], g.bwy[b], g.bwz[b]};
            for (int k = 0; k < 3; ++k) nh[k][i1] = nh[k][i1] + 4.0 * w[k] * p1;
            for (int k = 0; k < 3; ++k) nh[k][i2] = nh[k][i2] + 4.0 * w[k] * p2;
            if (c.ReynoldsNumber > 0.0 && ind == 1) {
                const double area = std::sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]);
                for (int k = 0; k < 3; ++k) nh[k][i1] = nh[k][i1] + 4.0 * g.wallStress[k][i1] * area;
                for (int k = 0; k < 3; ++k) nh[k][i2] = nh[k][i2] + 4.0 * g.wallStress[k][i2] * area;
            }
        }
        const double PI = 4.0 * std::atan(1.0);
        double aR = c.alpha * PI / 180., bR = c.beta * PI / 180.;
        double ft[3] = {std::cos(aR) * std::cos(bR), std::sin(bR), std::sin(aR)};
        double fn1[3] = {-ft[2], 0.0, ft[0]}, fn2[3] = {-ft[1], ft[0], 0.0};
        double lift = 0, drag = 0, latF = 0, latM = 0, longMl = 0, longMd = 0, rollM = 0;
        for_range(g, -20, -19, [&](int ip) {
            double xd = g.cx[ip] - c.datum[0], yd = g.cy[ip] - c.datum[1], zd = g.cz[ip] - c.datum[2];
            auto hd = [&](const double *a) { return (nh[0][ip] * a[0] + nh[1][ip] * a[1]) + nh[2][ip] * a[2]; };
            lift = lift + hd(fn1);
            drag = drag + hd(ft);
            latF = latF + hd(fn2);
            latM = latM - xd * hd(fn2);
            latM = latM + yd * hd(ft);
            rollM = rollM - yd * hd(fn1);
            rollM = rollM + zd * hd(fn2);
            longMl = longMl - xd * hd(fn1);
            longMd = longMd + zd * hd(ft);
        });
        const double A = c.referenceArea;
        out[0] = 2.0 * lift / A; out[1] = 2.0 * drag / A; out[2] = 2.0 * latF / A; out[3] = 2.0 * latM / A;
        out[4] = 2.0 * longMl / A; out[5] = 2.0 * longMd / A; out[6] = 2.0 * rollM / A;
    }
};

int check_controls(const flite_controls &c) {
    // flowType 1: dual time on a static mesh; 2: on a moving mesh
    if (c.flowType != 0 && !(c.physicalTimeStep > 0)) return FLITE_EUNSUPPORTED;
    if (c.flowType == 2 && c.reconstruction != FLITE_RECON_NONE) return FLITE_EUNSUPPORTED;
    // SAS (SST only) and patchInitialization (communicateSeq's start-up only)
    // have no effect on this path
    if ((c.flowType != 0 && c.flowType != 1 && c.flowType != 2) || c.GUSTMODEL || c.movingwall ||
        c.nspan != 0 || c.residualSmoothingFactor > 0 ||
        c.prolongationSmoothingFactor > 0)
        return FLITE_EUNSUPPORTED;
    // Spalart-Allmaras (1) is on the path and needs a viscous run; k-omega
    // and SST (2, 3) are not
    if (c.turbulenceModel != 0 && c.turbulenceModel != 1) return FLITE_EUNSUPPORTED;
    if (c.forceCalcType != 1 && c.forceCalcType != 3) return FLITE_EUNSUPPORTED;
    if (c.turbulenceModel == 1 && !(c.ReynoldsNumber > 0)) return FLITE_EUNSUPPORTED;
    if (c.ReynoldsNumber > 0 && c.viscosityScheme != 1 && c.viscosityScheme != 2) return FLITE_EUNSUPPORTED;
    if (c.fluxType < 1 || c.fluxType > 4) return FLITE_EUNSUPPORTED;
    // least-squares gradients divide by |dx|^2 of coarse-level coordinates
    // the reference never fills (0*inf = NaN): single-grid runs only
    if (c.fluxType == 4 && c.HLLCFluxOrder > 1 && c.GradientMethod != 1 && c.numberOfGridsToUse != 1)
        return FLITE_EUNSUPPORTED;
    // scheme 1 on coarse levels reads coordinates through seed-node indices
    // of the finer level (def_par:10874-10878) beyond the coarse arrays
    if (c.coarseGridDissipationScheme == 1) return FLITE_EUNSUPPORTED;
    if (c.prolongationMappingScheme != 1) return FLITE_EUNSUPPORTED;
    // the upwind extension (no reference counterpart)
    if (c.rungeKuttaStages != 3 && c.rungeKuttaStages != 5) return FLITE_EUNSUPPORTED;
    if (c.reconstruction != FLITE_RECON_NONE && c.reconstruction != FLITE_RECON_VAN_ALBADA) return FLITE_EUNSUPPORTED;
    if (c.reconstruction == FLITE_RECON_VAN_ALBADA && c.fluxType != 3) return FLITE_EUNSUPPORTED;
    return FLITE_OK;
}


// ---- tangent of the edge residual (central flux + boundary fluxes) -------
// forward-mode dual numbers; the CPU reference for the GPU adjoint product
struct Dl {
    double v, d;
    Dl(double a = 0, double b = 0) : v(a), d(b) {}
};
inline Dl operator+(Dl a, Dl b) { return {a.v + b.v, a.d + b.d}; }
inline Dl operator-(Dl a, Dl b) { return {a.v - b.v, a.d - b.d}; }
inline Dl operator-(Dl a) { return {-a.v, -a.d}; }
inline Dl operator*(Dl a, Dl b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dl operator/(Dl a, Dl b) { double q = a.v / b.v; return {q, (a.d - q * b.d) / b.v}; }
inline Dl dsqrt(Dl a) { double s = std::sqrt(a.v); return {s, s > 0 ? 0.5 * a.d / s : 0.0}; }
inline Dl dabs(Dl a) { return a.v < 0 ? -a : a; }

Dl tan_pressure(const flite_controls &c, const Dl *u) {
    Dl p = Dl(c.gamma - 1.0) * (u[4] - Dl(0.5) * ((u[1] * u[1] + u[2] * u[2]) + u[3] * u[3]) / u[0]);
    return p.v < 0.1 ? Dl(0.1) : p;
}
// one-sided flux G(u; w) = F(u).w
void tan_G(const Dl *u, Dl p, const double *w, Dl *G) {
    Dl mw = (u[1] * w[0] + u[2] * w[1]) + u[3] * w[2];
    G[0] = mw;
    for (int c = 0; c < 3; ++c) G[1 + c] = u[1 + c] * mw / u[0] + p * w[c];
    G[4] = (u[4] + p) * mw / u[0];
}
void tan_farfield(const flite_controls &c, const Dl *q, Dl pr, const double *n, const double *inf, Dl *F) {
    const double gam1 = c.gamma - 1.0;
    double ro = inf[0], ro1 = 1. / ro, uo = inf[1], vo = inf[2], wo = inf[3], eo = inf[4], po = inf[5];
    Dl rhol = q[0], rinvl = Dl(1.0) / rhol, rhl = q[4] + pr;
    Dl ul = q[1] * rinvl, vl = q[2] * rinvl, wl = q[3] * rinvl, epsl = q[4], hl = rhl * rinvl;
    Dl nvl = (ul * n[0] + vl * n[1]) + wl * n[2];
    Dl fl[5] = {rhol * nvl, pr * n[0] + rhol * ul * nvl, pr * n[1] + rhol * vl * nvl,
                pr * n[2] + rhol * wl * nvl, rhl * nvl};
    double rhor = ro, epsr = eo * ro, hr = eo + po * ro1;
    double unr = (uo * n[0] + vo * n[1]) + wo * n[2];
    double fr[5] = {rhor * unr, n[0] * po + rhor * uo * unr, n[1] * po + rhor * vo * unr,
                    n[2] * po + rhor * wo * unr, (epsr + po) * unr};
    Dl di = dsqrt(Dl(rhor) / rhol), d1 = Dl(1.0) / (di + Dl(1.0));
    Dl ui = (di * uo + ul) * d1, vi = (di * vo + vl) * d1, wi = (di * wo + wl) * d1, hi = (di * hr + hl) * d1;
    Dl ci2 = Dl(gam1) * (hi - Dl(0.5) * ((ui * ui + vi * vi) + wi * wi));
    if (ci2.v < 1.0e-5) ci2 = Dl(1.0e-5);
    Dl ci = dsqrt(ci2), af = Dl(0.5) * ((ui * ui + vi * vi) + wi * wi);
    Dl ucp = (ui * n[0] + vi * n[1]) + wi * n[2];
    Dl du[5] = {Dl(rhor) - rhol, Dl(rhor * uo) - rhol * ul, Dl(rhor * vo) - rhol * vl, Dl(rhor * wo) - rhol * wl,
                Dl(epsr) - epsl};
    Dl l1 = dabs(ucp + ci), l2 = dabs(ucp - ci), l3 = dabs(ucp);
    Dl s1 = Dl(0.5) * (l1 + l2), s2 = Dl(0.5) * (l1 - l2);
    Dl al1x = Dl(gam1) * ((((af * du[0] - ui * du[1]) - vi * du[2]) - wi * du[3]) + du[4]);
    Dl al2x = ((-ucp * du[0] + du[1] * n[0]) + du[2] * n[1]) + du[3] * n[2];
    Dl cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci), cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
    Dl ex[5] = {cc1, cc1 * ui + cc2 * n[0], cc1 * vi + cc2 * n[1], cc1 * wi + cc2 * n[2], cc1 * hi + cc2 * ucp};
    for (int k = 0; k < 5; ++k) F[k] = Dl(0.5) * (Dl(fr[k]) + fl[k]) - Dl(0.5) * (l3 * du[k] + ex[k]);
}

// ---- tangent of one smoother iteration on level 1 ------------------------
// singleIteration with calcDiss (def_par:1002-1181) for the central flux
// (fluxType 1), scalar JST dissipation (def_par:11484-11993) and an inviscid
// run, restated with dual numbers whose derivative part carries one
// direction in the state u and in the level-1 geometry (side_w, bnd_w,
// volume; the node normals and wall areas follow from bnd_w as in
// makeBoundaryNormals def_par:15394-15521 and makeSurfaceArea :15523-15634).
// The value parts repeat the double routines' operations in their order, so
// they equal one doTimeIterations step of this restatement bit for bit.
inline Dl dmaxl(Dl a, Dl b) { return a.v < b.v ? b : a; }        // std::max
inline Dl dminl(Dl a, Dl b) { return b.v < a.v ? b : a; }        // std::min
inline Dl dmaxc(Dl a, double c) { return a.v < c ? Dl(c) : a; }  // std::max(a, c)
// |vn| of the time step with the derivative 0 where vn = w.m/rho is rounding
// noise (|w.m| <= 1e-12 |w||m|: the momentum of a slip-wall or symmetry node
// projected onto the plane), the mean of the one-sided derivatives there
inline Dl kink_abs(Dl vn, Dl wm, Dl al, const Dl *m) {
    double mm = std::sqrt((m[0].v * m[0].v + m[1].v * m[1].v) + m[2].v * m[2].v);
    if (std::fabs(wm.v) <= 1.0e-12 * std::sqrt(al.v) * mm) return Dl(std::fabs(vn.v), 0.0);
    return dabs(vn);
}

// far-field Roe flux (def_par:2258-2419) with the normal as a dual number
void tan_farfield_n(const flite_controls &c, const Dl *q, Dl prl, const Dl *n, const double *inf, Dl *F) {
    const double gam1 = c.gamma - 1.0;
    double ro = inf[0], ro1 = 1. / ro, uo = inf[1], vo = inf[2], wo = inf[3], eo = inf[4], po = inf[5];
    Dl rhol = q[0], rinvl = Dl(1.) / rhol;
    Dl rul = q[1], rvl = q[2], rwl = q[3], rhl = q[4] + prl;
    Dl ul = rul * rinvl, vl = rvl * rinvl, wl = rwl * rinvl;
    Dl epsl = q[4], hl = rhl * rinvl;
    Dl nvl = (ul * n[0] + vl * n[1]) + wl * n[2];
    Dl fl1 = rhol * nvl, fl2 = prl * n[0] + rhol * ul * nvl, fl3 = prl * n[1] + rhol * vl * nvl;
    Dl fl4 = prl * n[2] + rhol * wl * nvl, fl5 = rhl * nvl;
    double rhor = ro, uxr = uo, vyr = vo, wzr = wo, epsr = eo * ro, presr = po, hr = eo + po * ro1;
    Dl unr = (Dl(uxr) * n[0] + Dl(vyr) * n[1]) + Dl(wzr) * n[2];
    Dl fr1 = Dl(rhor) * unr, fr2 = n[0] * presr + Dl(rhor * uxr) * unr, fr3 = n[1] * presr + Dl(rhor * vyr) * unr;
    Dl fr4 = n[2] * presr + Dl(rhor * wzr) * unr, fr5 = Dl(epsr + presr) * unr;
    Dl di = dsqrt(Dl(rhor) / rhol), d1 = Dl(1.0) / (di + Dl(1.0));
    Dl ui = (di * uxr + ul) * d1, vi = (di * vyr + vl) * d1, wi = (di * wzr + wl) * d1;
    Dl hi = (di * hr + hl) * d1;
    Dl ci2 = Dl(gam1) * (hi - Dl(0.5) * ((ui * ui + vi * vi) + wi * wi));
    ci2 = dmaxc(ci2, 1.0e-5);
    Dl ci = dsqrt(ci2);
    Dl af = Dl(0.5) * ((ui * ui + vi * vi) + wi * wi);
    Dl ucp = (ui * n[0] + vi * n[1]) + wi * n[2];
    Dl du1 = Dl(rhor) - rhol, du2 = Dl(rhor * uxr) - rhol * ul, du3 = Dl(rhor * vyr) - rhol * vl;
    Dl du4 = Dl(rhor * wzr) - rhol * wl, du5 = Dl(epsr) - epsl;
    Dl l1 = dabs(ucp + ci), l2 = dabs(ucp - ci), l3 = dabs(ucp);
    Dl s1 = Dl(0.5) * (l1 + l2), s2 = Dl(0.5) * (l1 - l2);
    Dl al1x = Dl(gam1) * ((((af * du1 - ui * du2) - vi * du3) - wi * du4) + du5);
    Dl al2x = ((-ucp * du1 + du2 * n[0]) + du3 * n[1]) + du4 * n[2];
    Dl cc1 = ((s1 - l3) * al1x / ci2) + (s2 * al2x / ci);
    Dl cc2 = (s2 * al1x / ci) + (s1 - l3) * al2x;
    F[0] = Dl(0.5) * (fr1 + fl1) - Dl(0.5) * (l3 * du1 + cc1);
    F[1] = Dl(0.5) * (fr2 + fl2) - Dl(0.5) * ((l3 * du2 + cc1 * ui) + cc2 * n[0]);
    F[2] = Dl(0.5) * (fr3 + fl3) - Dl(0.5) * ((l3 * du3 + cc1 * vi) + cc2 * n[1]);
    F[3] = Dl(0.5) * (fr4 + fl4) - Dl(0.5) * ((l3 * du4 + cc1 * wi) + cc2 * n[2]);
    F[4] = Dl(0.5) * (fr5 + fl5) - Dl(0.5) * ((l3 * du5 + cc1 * hi) + cc2 * ucp);
}

struct TanIteration {
    const Oracle &o;
    const Level &g;
    const flite_controls &c;
    int N, E, B;
    std::vector<Dl> wx, wy, wz, bwx, bwy, bwz, V, nx, ny, nz, area;

    TanIteration(const Oracle &o_, const double *dsw, const double *dbw, const double *dvol)
        : o(o_), g(o_.lv[0]), c(o_.c), N(g.N), E(g.E), B(g.B) {
        wx.resize(E); wy.resize(E); wz.resize(E);
        for (int e = 0; e < E; ++e) {
            wx[e] = Dl(g.wx[e], dsw ? dsw[e] : 0.0);
            wy[e] = Dl(g.wy[e], dsw ? dsw[(size_t)E + e] : 0.0);
            wz[e] = Dl(g.wz[e], dsw ? dsw[2 * (size_t)E + e] : 0.0);
        }
        bwx.resize(B); bwy.resize(B); bwz.resize(B);
        for (int b = 0; b < B; ++b) {
            bwx[b] = Dl(g.bwx[b], dbw ? dbw[b] : 0.0);
            bwy[b] = Dl(g.bwy[b], dbw ? dbw[(size_t)B + b] : 0.0);
            bwz[b] = Dl(g.bwz[b], dbw ? dbw[2 * (size_t)B + b] : 0.0);
        }
        V.resize(N);
        for (int i = 0; i < N; ++i) V[i] = Dl(g.V[i], dvol ? dvol[i] : 0.0);
        // makeBoundaryNormals and makeSurfaceArea (the setup_level forms)
        nx.assign(N, Dl()); ny.assign(N, Dl()); nz.assign(N, Dl()); area.assign(N, Dl());
        for (int b = 0; b < B; ++b) {
            int a = g.b1[b], d = g.b2[b];
            nx[a] = nx[a] - bwx[b]; ny[a] = ny[a] - bwy[b]; nz[a] = nz[a] - bwz[b];
            nx[d] = nx[d] - bwx[b]; ny[d] = ny[d] - bwy[b]; nz[d] = nz[d] - bwz[b];
        }
        for (int i = 0; i < g.Nb; ++i) {
            Dl nrm = dsqrt((nx[i] * nx[i] + ny[i] * ny[i]) + nz[i] * nz[i]);
            if (nrm.v > 1.0e-10) { nx[i] = nx[i] / nrm; ny[i] = ny[i] / nrm; nz[i] = nz[i] / nrm; }
            else { nx[i] = Dl(); ny[i] = Dl(); nz[i] = Dl(); }
        }
        for (int b = 0; b < B; ++b) {
            Dl ai = dsqrt((bwx[b] * bwx[b] + bwy[b] * bwy[b]) + bwz[b] * bwz[b]);
            area[g.b1[b]] = area[g.b1[b]] + Dl(4.0) * ai;
            area[g.b2[b]] = area[g.b2[b]] + Dl(4.0) * ai;
        }
    }

    template <class Fn>
    void for_range(int a, int b, Fn fn) const {
        for (int ib = g.R(a); ib <= g.R(b); ++ib) fn(g.node_ind[ib - 1]);
    }
    Dl pressure(const std::vector<Dl> *u, int i) const {
        Dl pp = Dl(c.gamma - 1.0) * (u[4][i] - Dl(0.5) * ((u[1][i] * u[1][i] + u[2][i] * u[2][i]) + u[3][i] * u[3][i]) / u[0][i]);
        return dmaxc(pp, 0.1);
    }
    void remove_normal(std::vector<Dl> *x, int ip, double scale) const {
        Dl n[3] = {nx[ip], ny[ip], nz[ip]};
        Dl nv = (x[1][ip] * n[0] + x[2][ip] * n[1]) + x[3][ip] * n[2];
        for (int k = 0; k < 3; ++k) x[1 + k][ip] = x[1 + k][ip] - Dl(scale) * nv * n[k];
    }
    // makeTimeSteps, inviscid (def_par:13335-13610)
    void timesteps(const std::vector<Dl> *u, const std::vector<Dl> &p, const std::vector<Dl> *mu,
                   std::vector<Dl> &dt) const {
        const double c1 = c.gamma;
        dt.assign(N, Dl());
        std::vector<Dl> h1(N, Dl());
        const bool visc = c.ReynoldsNumber > 0.0;
        const double am = visc ? 1.0 / c.ReynoldsNumber : 0.0;
        auto vis = [&](int i) { return am < (*mu)[i].v ? (*mu)[i] : Dl(am); };  // std::max(am, mu)
        for (int e = 0; e < E; ++e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            Dl al = (wx[e] * wx[e] + wy[e] * wy[e]) + wz[e] * wz[e];
            Dl ro1 = Dl(1.) / u[0][i1], ro2 = Dl(1.) / u[0][i2];
            Dl cc1 = dmaxc(Dl(c1) * p[i1] * ro1, 0.001), cc2 = dmaxc(Dl(c1) * p[i2] * ro2, 0.001);
            Dl wm1 = (wx[e] * u[1][i1] + wy[e] * u[2][i1]) + wz[e] * u[3][i1];
            Dl wm2 = (wx[e] * u[1][i2] + wy[e] * u[2][i2]) + wz[e] * u[3][i2];
            Dl vn1 = wm1 * ro1, vn2 = wm2 * ro2;
            const Dl m1[3] = {u[1][i1], u[2][i1], u[3][i1]}, m2[3] = {u[1][i2], u[2][i2], u[3][i2]};
            dt[i1] = (dt[i1] + kink_abs(vn1, wm1, al, m1)) + dsqrt(cc1 * al);
            dt[i2] = (dt[i2] + kink_abs(vn2, wm2, al, m2)) + dsqrt(cc2 * al);
            if (visc) {
                Dl dv1 = Dl(2.0) * vis(i1) * al / u[0][i1], dv2 = Dl(2.0) * vis(i2) * al / u[0][i2];
                h1[i1] = h1[i1] + dv2;
                h1[i2] = h1[i2] + dv1;
            }
        }
        for (int b = 0; b < B; ++b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            Dl al = (bwx[b] * bwx[b] + bwy[b] * bwy[b]) + bwz[b] * bwz[b];
            Dl ro1 = Dl(1.) / u[0][i1], ro2 = Dl(1.) / u[0][i2];
            Dl cc1 = dmaxc(Dl(c1) * p[i1] * ro1, 0.001), cc2 = dmaxc(Dl(c1) * p[i2] * ro2, 0.001);
            Dl wm1 = (bwx[b] * u[1][i1] + bwy[b] * u[2][i1]) + bwz[b] * u[3][i1];
            Dl wm2 = (bwx[b] * u[1][i2] + bwy[b] * u[2][i2]) + bwz[b] * u[3][i2];
            Dl vn1 = wm1 * ro1, vn2 = wm2 * ro2;
            const Dl m1[3] = {u[1][i1], u[2][i1], u[3][i1]}, m2[3] = {u[1][i2], u[2][i2], u[3][i2]};
            vn1 = kink_abs(vn1, wm1, al, m1); vn2 = kink_abs(vn2, wm2, al, m2);
            Dl vnm = vn1 + vn2;
            cc1 = dsqrt(cc1 * al); cc2 = dsqrt(cc2 * al);
            Dl ccm = cc1 + cc2;
            dt[i1] = (((dt[i1] + vn1) + vnm) + cc1) + ccm;
            dt[i2] = (((dt[i2] + vn2) + vnm) + cc2) + ccm;
            if (visc) {
                Dl dv1 = Dl(2.0) * vis(i1) * al / u[0][i1], dv2 = Dl(2.0) * vis(i2) * al / u[0][i2];
                Dl dvm = dv1 + dv2;
                h1[i1] = (h1[i1] + dv1) + dvm;
                h1[i2] = (h1[i2] + dv2) + dvm;
            }
        }
        for (int i = 0; i < N; ++i) dt[i] = Dl(0.5) / (dt[i] / V[i] + h1[i] / (V[i] * V[i]));
    }
    // makeViscosityTerm, wide stencil (def_par:5198-5893), laminar: subtracts the
    // viscous fluxes from diss, returns the laminar viscosity mu of each node and,
    // on level 1, the wall stress of the boundary nodes (ws [3][N], may be null)
    void viscous(const std::vector<Dl> *u, const std::vector<Dl> &p, std::vector<Dl> *diss, std::vector<Dl> &mu,
                 std::vector<Dl> *ws) const {
        const double gOg = c.gamma / (c.gamma - 1.0);
        const double tempConv = (c.gamma - 1.0) * c.MachNumber * c.MachNumber;
        const double Tin = c.inflowTemperature;
        std::vector<Dl> q[4], G[12], t[9], f[4];
        for (auto &v : q) v.resize(N);
        for (auto &v : G) v.assign(N, Dl());
        for (auto &v : t) v.assign(N, Dl());
        for (auto &v : f) v.assign(N, Dl());
        for (int i = 0; i < N; ++i) {
            Dl r = u[0][i];
            q[0][i] = u[1][i] / r; q[1][i] = u[2][i] / r; q[2][i] = u[3][i] / r;
            q[3][i] = Dl(gOg) * p[i] / r;
        }
        for (int e = 0; e < E; ++e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            const Dl w[3] = {wx[e], wy[e], wz[e]};
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    Dl d = (q[k][i1] + q[k][i2]) * w[a];
                    G[a * 4 + k][i1] = G[a * 4 + k][i1] + d;
                    G[a * 4 + k][i2] = G[a * 4 + k][i2] - d;
                }
        }
        for (int b = 0; b < B; ++b) {
            int i1 = g.b1[b], i2 = g.b2[b];
            const Dl w[3] = {bwx[b], bwy[b], bwz[b]};
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    Dl sm = q[k][i1] + q[k][i2];
                    G[a * 4 + k][i1] = G[a * 4 + k][i1] + (Dl(2.) * q[k][i1] + sm) * w[a];
                }
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 4; ++k) {
                    Dl sm = q[k][i1] + q[k][i2];
                    G[a * 4 + k][i2] = G[a * 4 + k][i2] + (Dl(2.) * q[k][i2] + sm) * w[a];
                }
        }
        const double twoThirds = 2. / 3., fourThirds = 4. / 3.;
        const double oRe = 1. / c.ReynoldsNumber, oPr = 1. / c.PrandtlNumber;
        mu.assign(N, Dl());
        for (int i = 0; i < N; ++i) {
            Dl vt = Dl(1.) / V[i];
            Dl dudx = G[0][i] * vt, dvdx = G[1][i] * vt, dwdx = G[2][i] * vt, dTdx = G[3][i] * vt;
            Dl dudy = G[4][i] * vt, dvdy = G[5][i] * vt, dwdy = G[6][i] * vt, dTdy = G[7][i] * vt;
            Dl dudz = G[8][i] * vt, dvdz = G[9][i] * vt, dwdz = G[10][i] * vt, dTdz = G[11][i] * vt;
            Dl T = Dl(gOg) * p[i] / u[0][i];
            if (T.v <= 0.001) T = Dl(0.001);
            Dl a = Dl(tempConv) * T;
            Dl m = Dl(oRe) * ((a * dsqrt(a)) * (Dl(Tin + 198.6) / (Dl(tempConv * Tin) * T + Dl(198.6))));
            Dl k = Dl(oPr) * m;
            mu[i] = m;
            t[0][i] = m * (Dl(fourThirds) * dudx - Dl(twoThirds) * (dvdy + dwdz));
            t[1][i] = m * (dudy + dvdx);
            t[2][i] = m * (dudz + dwdx);
            t[3][i] = m * (Dl(fourThirds) * dvdy - Dl(twoThirds) * (dudx + dwdz));
            t[4][i] = m * (dvdz + dwdy);
            t[5][i] = m * (Dl(fourThirds) * dwdz - Dl(twoThirds) * (dudx + dvdy));
            t[6][i] = k * dTdx;
            t[7][i] = k * dTdy;
            t[8][i] = k * dTdz;
        }
        if (g.grid == 1) {
            for_range(-20, -19, [&](int ip) {
                Dl n[3] = {nx[ip], ny[ip], nz[ip]};
                Dl dT[3] = {t[6][ip], t[7][ip], t[8][ip]};
                Dl nt = (dT[0] * n[0] + dT[1] * n[1]) + dT[2] * n[2];
                for (int kk = 0; kk < 3; ++kk) t[6 + kk][ip] = dT[kk] - nt * n[kk];
            });
            if (ws)
                for (int ib = 0; ib < std::min(g.Nb, g.nnorm); ++ib) {
                    int ip = g.node_ind[ib];
                    Dl n[3] = {nx[ip], ny[ip], nz[ip]};
                    ws[0][ip] = (t[0][ip] * n[0] + t[1][ip] * n[1]) + t[2][ip] * n[2];
                    ws[1][ip] = (t[1][ip] * n[0] + t[3][ip] * n[1]) + t[4][ip] * n[2];
                    ws[2][ip] = (t[2][ip] * n[0] + t[4][ip] * n[1]) + t[5][ip] * n[2];
                }
        }
        auto loadt = [&](int i, Dl *tt, Dl *uu) {
            for (int kk = 0; kk < 9; ++kk) tt[kk] = t[kk][i];
            uu[0] = u[1][i] / u[0][i]; uu[1] = u[2][i] / u[0][i]; uu[2] = u[3][i] / u[0][i];
        };
        for (int e = 0; e < E; ++e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            Dl wx_ = wx[e], wy_ = wy[e], wz_ = wz[e];
            Dl a[9], b[9], ua[3], ub[3];
            loadt(i1, a, ua); loadt(i2, b, ub);
            Dl dt[9];
            for (int kk = 0; kk < 9; ++kk) dt[kk] = a[kk] + b[kk];
            Dl dut1 = ((((ua[0] * a[0] + ub[0] * b[0]) + ua[1] * a[1]) + ub[1] * b[1]) + ua[2] * a[2]) + ub[2] * b[2];
            Dl dut2 = ((((ua[0] * a[1] + ub[0] * b[1]) + ua[1] * a[3]) + ub[1] * b[3]) + ua[2] * a[4]) + ub[2] * b[4];
            Dl dut3 = ((((ua[0] * a[2] + ub[0] * b[2]) + ua[1] * a[4]) + ub[1] * b[4]) + ua[2] * a[5]) + ub[2] * b[5];
            Dl ff[4] = {(wx_ * dt[0] + wy_ * dt[1]) + wz_ * dt[2], (wx_ * dt[1] + wy_ * dt[3]) + wz_ * dt[4],
                        (wx_ * dt[2] + wy_ * dt[4]) + wz_ * dt[5],
                        (wx_ * (dt[6] + dut1) + wy_ * (dt[7] + dut2)) + wz_ * (dt[8] + dut3)};
            for (int kk = 0; kk < 4; ++kk) {
                f[kk][i1] = f[kk][i1] + ff[kk];
                f[kk][i2] = f[kk][i2] - ff[kk];
            }
        }
        for (int bb = 0; bb < B; ++bb) {
            int ind = g.bind[bb];
            if (ind == 2 || ind == 9) continue;
            int i1 = g.b1[bb], i2 = g.b2[bb];
            Dl wx_ = bwx[bb], wy_ = bwy[bb], wz_ = bwz[bb];
            Dl a[9], b[9], ua[3], ub[3];
            loadt(i1, a, ua); loadt(i2, b, ub);
            Dl dt[9];
            for (int kk = 0; kk < 9; ++kk) dt[kk] = a[kk] + b[kk];
            Dl d11 = (ua[0] * a[0] + ua[1] * a[1]) + ua[2] * a[2];
            Dl d12 = (ub[0] * b[0] + ub[1] * b[1]) + ub[2] * b[2];
            Dl d21 = (ua[0] * a[1] + ua[1] * a[3]) + ua[2] * a[4];
            Dl d22 = (ub[0] * b[1] + ub[1] * b[3]) + ub[2] * b[4];
            Dl d31 = (ua[0] * a[2] + ua[1] * a[4]) + ua[2] * a[5];
            Dl d32 = (ub[0] * b[2] + ub[1] * b[4]) + ub[2] * b[5];
            Dl dut1 = d11 + d12, dut2 = d21 + d22, dut3 = d31 + d32;
            Dl f2 = (wx_ * dt[0] + wy_ * dt[1]) + wz_ * dt[2];
            Dl f3 = (wx_ * dt[1] + wy_ * dt[3]) + wz_ * dt[4];
            Dl f4 = (wx_ * dt[2] + wy_ * dt[4]) + wz_ * dt[5];
            Dl f5 = (wx_ * (dt[6] + dut1) + wy_ * (dt[7] + dut2)) + wz_ * (dt[8] + dut3);
            f[0][i1] = (f[0][i1] + f2) + Dl(2.0) * ((wx_ * a[0] + wy_ * a[1]) + wz_ * a[2]);
            f[1][i1] = (f[1][i1] + f3) + Dl(2.0) * ((wx_ * a[1] + wy_ * a[3]) + wz_ * a[4]);
            f[2][i1] = (f[2][i1] + f4) + Dl(2.0) * ((wx_ * a[2] + wy_ * a[4]) + wz_ * a[5]);
            f[3][i1] = (f[3][i1] + f5) + Dl(2.0) * ((wx_ * (a[6] + d11) + wy_ * (a[7] + d21)) + wz_ * (a[8] + d31));
            f[0][i2] = (f[0][i2] + f2) + Dl(2.0) * ((wx_ * b[0] + wy_ * b[1]) + wz_ * b[2]);
            f[1][i2] = (f[1][i2] + f3) + Dl(2.0) * ((wx_ * b[1] + wy_ * b[3]) + wz_ * b[4]);
            f[2][i2] = (f[2][i2] + f4) + Dl(2.0) * ((wx_ * b[2] + wy_ * b[4]) + wz_ * b[5]);
            f[3][i2] = (f[3][i2] + f5) + Dl(2.0) * ((wx_ * (b[6] + d12) + wy_ * (b[7] + d22)) + wz_ * (b[8] + d32));
        }
        for (int i = 0; i < N; ++i)
            for (int kk = 0; kk < 4; ++kk) diss[1 + kk][i] = diss[1 + kk][i] - f[kk][i];
    }
    // makeArtificialDissipation2 on level 1, unweighted (def_par:11484-11993)
    void jst(const std::vector<Dl> *u, const std::vector<Dl> &p, const std::vector<Dl> &dt,
             std::vector<Dl> *diss) const {
        for (int k = 0; k < 5; ++k) diss[k].assign(N, Dl());
        if (c.fourthOrderDissipationFactor == 0 && c.secondOrderDissipationFactor == 0) return;
        std::vector<Dl> nh[9];
        for (auto &v : nh) v.assign(N, Dl());
        for (int e = 0; e < E; ++e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            Dl d[5];
            for (int k = 0; k < 4; ++k) d[k] = u[k][i1] - u[k][i2];
            d[4] = ((u[4][i1] - u[4][i2]) + p[i1]) - p[i2];
            for (int k = 0; k < 5; ++k) {
                nh[k][i1] = nh[k][i1] - d[k] * Dl(1.0);
                nh[k][i2] = nh[k][i2] + d[k] * Dl(1.0);
            }
        }
        for (int e = 0; e < E; ++e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            Dl dp = p[i1] - p[i2], sp = p[i1] + p[i2];
            nh[6][i1] = nh[6][i1] - dp;
            nh[7][i1] = nh[7][i1] + sp;
            nh[6][i2] = nh[6][i2] + dp;
            nh[7][i2] = nh[7][i2] + sp;
        }
        for (int i = 0; i < N; ++i) {
            double fact = 1. / g.conn[i];
            nh[8][i] = Dl(12.) * dabs(nh[6][i] / nh[7][i]);
            for (int k = 0; k < 5; ++k) nh[k][i] = Dl(fact) * nh[k][i];
        }
        const double k2 = c.secondOrderDissipationFactor, k4 = c.fourthOrderDissipationFactor;
        for (int e = 0; e < E; ++e) {
            int i1 = g.s1[e], i2 = g.s2[e];
            Dl d4v[5], d2v[5];
            for (int k = 0; k < 5; ++k) d4v[k] = nh[k][i1] - nh[k][i2];
            for (int k = 0; k < 5; ++k) d2v[k] = u[k][i1] - u[k][i2];
            Dl d0 = dminl(V[i1] / dt[i1], V[i2] / dt[i2]) / Dl(g.conn[i1] + g.conn[i2]);
            Dl d2 = d0 * Dl(k2) * dmaxl(nh[8][i1], nh[8][i2]);
            Dl d4 = d0 * Dl(k4);
            d4 = d4.v > d2.v ? d4 - d2 : Dl(0.0);
            for (int k = 0; k < 5; ++k) {
                diss[k][i1] = (diss[k][i1] - d4v[k] * d4) + d2v[k] * d2;
                diss[k][i2] = (diss[k][i2] + d4v[k] * d4) - d2v[k] * d2;
            }
        }
    }
    void wall_flux(const std::vector<Dl> *u, const std::vector<Dl> &p, int i, const Dl *rn, Dl *F) const {
        Dl pr = p[i], rho = u[0][i], rinv = Dl(1.) / rho;
        Dl ru = u[1][i], rv = u[2][i], rw = u[3][i], rh = u[4][i] + pr;
        Dl uu = ru * rinv, vv = rv * rinv, ww = rw * rinv;
        Dl nv = (uu * rn[0] + vv * rn[1]) + ww * rn[2];
        F[0] = rho * nv;
        F[1] = pr * rn[0] + rho * uu * nv;
        F[2] = pr * rn[1] + rho * vv * nv;
        F[3] = pr * rn[2] + rho * ww * nv;
        F[4] = rh * nv;
    }
    // makeRHS for the central flux with the boundary faces (def_par:1525-2512)
    void rhs(const std::vector<Dl> *u, const std::vector<Dl> &p, std::vector<Dl> *r) const {
        for (int k = 0; k < 5; ++k) r[k].assign(N, Dl());
        for (int e = 0; e < E; ++e) {
            const int i1 = g.s1[e], i2 = g.s2[e];
            Dl pr1 = p[i1], rinv1 = Dl(1.) / u[0][i1];
            Dl ru1 = u[1][i1], rv1 = u[2][i1], rw1 = u[3][i1];
            Dl u1 = rinv1 * ru1, v1 = rinv1 * rv1, w1 = rinv1 * rw1;
            Dl rh1 = u[4][i1] + pr1;
            Dl pr2 = p[i2], rinv2 = Dl(1.) / u[0][i2];
            Dl ru2 = u[1][i2], rv2 = u[2][i2], rw2 = u[3][i2];
            Dl u2 = rinv2 * ru2, v2 = rinv2 * rv2, w2 = rinv2 * rw2;
            Dl rh2 = u[4][i2] + pr2;
            const Dl wx_ = wx[e], wy_ = wy[e], wz_ = wz[e];
            Dl f[5];
            f[0] = (wx_ * (ru1 + ru2) + wy_ * (rv1 + rv2)) + wz_ * (rw1 + rw2);
            f[1] = (wx_ * (((ru1 * u1 + pr1) + ru2 * u2) + pr2) + wy_ * (ru1 * v1 + ru2 * v2)) + wz_ * (ru1 * w1 + ru2 * w2);
            f[2] = (wx_ * (rv1 * u1 + rv2 * u2) + wy_ * (((rv1 * v1 + pr1) + rv2 * v2) + pr2)) + wz_ * (rv1 * w1 + rv2 * w2);
            f[3] = (wx_ * (rw1 * u1 + rw2 * u2) + wy_ * (rw1 * v1 + rw2 * v2)) + wz_ * (((rw1 * w1 + pr1) + rw2 * w2) + pr2);
            f[4] = (wx_ * (rh1 * u1 + rh2 * u2) + wy_ * (rh1 * v1 + rh2 * v2)) + wz_ * (rh1 * w1 + rh2 * w2);
            for (int k = 0; k < 5; ++k) {
                r[k][i1] = r[k][i1] + f[k];
                r[k][i2] = r[k][i2] - f[k];
            }
        }
        const bool fe = c.boundaryTerm == 1;
        for (int b = 0; b < B; ++b) {
            const int i1 = g.b1[b], i2 = g.b2[b], ind = g.bind[b];
            Dl g1[5], g2[5];
            Dl rnorm = dsqrt((bwx[b] * bwx[b] + bwy[b] * bwy[b]) + bwz[b] * bwz[b]);
            if ((ind <= 4 || ind == 9) && rnorm.v > 1.0e-10) {
                Dl rn[3] = {bwx[b] / rnorm, bwy[b] / rnorm, bwz[b] / rnorm};
                Dl F1[5], F2[5];
                if (ind <= 2 || ind == 9) {
                    wall_flux(u, p, i1, rn, F1);
                    wall_flux(u, p, i2, rn, F2);
                } else {
                    const double *inf = &c.inflowField[(ind - 3) * 6];
                    Dl q1[5], q2[5];
                    for (int k = 0; k < 5; ++k) { q1[k] = u[k][i1]; q2[k] = u[k][i2]; }
                    tan_farfield_n(c, q1, p[i1], rn, inf, F1);
                    tan_farfield_n(c, q2, p[i2], rn, inf, F2);
                }
                for (int k = 0; k < 5; ++k) {
                    if (fe) { g1[k] = rnorm * (Dl(3.) * F1[k] + F2[k]); g2[k] = rnorm * (F1[k] + Dl(3.) * F2[k]); }
                    else { g1[k] = rnorm * Dl(4.) * F1[k]; g2[k] = rnorm * Dl(4.) * F2[k]; }
                }
            } else {
                for (int k = 0; k < 5; ++k) { g1[k] = Dl(); g2[k] = Dl(); }
            }
            for (int k = 0; k < 5; ++k) r[k][i1] = r[k][i1] + g1[k];
            for (int k = 0; k < 5; ++k) r[k][i2] = r[k][i2] + g2[k];
        }
    }
    // one doTimeIterations step on level 1: u <- G(u)
    // mu: the laminar viscosity the time step reads (viscous runs), replaced
    // by the one makeViscosityTerm computes from u
    void iterate(std::vector<Dl> *u, std::vector<Dl> *mu) const {
        std::vector<Dl> up[5], p(N), dt, diss[5], r[5];
        for (int k = 0; k < 5; ++k) up[k] = u[k];
        for (int i = 0; i < N; ++i) p[i] = dabs(pressure(u, i));
        const bool visc = c.ReynoldsNumber > 0.0;
        timesteps(u, p, mu, dt);
        jst(u, p, dt, diss);
        if (visc) {
            std::vector<Dl> mu_new;
            viscous(u, p, diss, mu_new, nullptr);
            *mu = mu_new;
        }
        const double relax = o.relaxation_param(g);
        for (int st = 1; st <= 3; ++st) {
            for (int i = 0; i < N; ++i) p[i] = pressure(u, i);
            rhs(u, p, r);
            for (int k = 0; k < 5; ++k)
                for (int i = 0; i < N; ++i) r[k][i] = r[k][i] + diss[k][i];
            for (int i = 0; i < N; ++i)
                for (int k = 0; k < 5; ++k) r[k][i] = dt[i] * r[k][i] / V[i];
            if (visc)
                for_range(-20, -19, [&](int ip) {
                    r[1][ip] = Dl(); r[2][ip] = Dl(); r[3][ip] = Dl();
                    if (!c.wallsAreIsentropic) r[4][ip] = Dl();
                });
            else
                for_range(-20, -19, [&](int ip) { remove_normal(r, ip, 1.0); });
            for_range(-4, -3, [&](int ip) { remove_normal(r, ip, 1.0); });
            for_range(-18, -17, [&](int ip) { remove_normal(r, ip, 1.0); });
            const double dtJ = c.CFLNumber * o.RK[st - 1];
            for (int k = 0; k < 5; ++k)
                for (int i = 0; i < N; ++i) r[k][i] = Dl(dtJ) * r[k][i];
            for (int i = 0; i < N; ++i) {
                Dl inc = r[0][i];
                if (std::fabs(inc.v / up[0][i].v) < c.maxIncrementFactor) {
                    u[0][i] = up[0][i] - inc;
                } else {
                    double sign = inc.v / std::fabs(inc.v);
                    u[0][i] = up[0][i] - Dl(sign * c.maxIncrementFactor) * up[0][i];
                }
                for (int k = 1; k < 5; ++k) u[k][i] = up[k][i] - r[k][i];
                if (u[0][i].v < c.minimumDensity) u[0][i] = Dl(c.minimumDensity);
            }
            if (visc)
                for_range(-20, -19, [&](int ip) {
                    const double cm[3] = {g.cmx[ip], g.cmy[ip], g.cmz[ip]};
                    for (int k = 0; k < 3; ++k) u[1 + k][ip] = u[0][ip] * Dl(cm[k]) / Dl(c.physicalTimeStep);
                    if (!c.wallsAreIsentropic) u[4][ip] = u[0][ip] * Dl(c.inflowTemperature) / Dl(c.gamma);
                });
            else
                for_range(-20, -19, [&](int ip) { remove_normal(u, ip, 1.0); });
            for_range(-4, -3, [&](int ip) {
                remove_normal(u, ip, relax);
                if (!c.wallsAreIsentropic) {
                    Dl ke = (u[1][ip] * u[1][ip] + u[2][ip] * u[2][ip]) + u[3][ip] * u[3][ip];
                    u[4][ip] = u[0][ip] * Dl(c.inflowTemperature) / Dl(c.gamma) + Dl(0.5) * ke / u[0][ip];
                }
            });
            for_range(-18, -17, [&](int ip) { remove_normal(u, ip, 1.0); });
            for (int i = 0; i < N; ++i) u[0][i] = dmaxc(u[0][i], c.minimumDensity);
            const double gm1 = c.gamma - 1.0;
            for (int side = 0; side < 2; ++side) {
                const double *inf = &c.inflowField[side * 6];
                double iR = inf[0], iU1 = inf[1], iU2 = inf[2], iU3 = inf[3], iE = inf[4], iP = inf[5];
                for_range(side == 0 ? -16 : -14, side == 0 ? -15 : -13, [&](int ip) {
                    Dl rho = u[0][ip], U1 = u[1][ip], U2 = u[2][ip], U3 = u[3][ip];
                    double nvel = (iU1 * nx[ip].v + iU2 * ny[ip].v) + iU3 * nz[ip].v;
                    if (nvel > 0.00) {
                        u[0][ip] = Dl(iR); u[1][ip] = Dl(iU1 * iR); u[2][ip] = Dl(iU2 * iR); u[3][ip] = Dl(iU3 * iR);
                        if (c.MachNumber > 1.0) u[4][ip] = Dl(iE * iR);
                        else u[4][ip] = p[ip] / Dl(gm1) + Dl(0.5 * ((iU1 * iU1 + iU2 * iU2) + iU3 * iU3) * iR);
                    } else {
                        if (c.MachNumber < 1.0)
                            u[4][ip] = Dl(iP / gm1) + Dl(0.5) * ((U1 * U1 + U2 * U2) + U3 * U3) / rho;
                    }
                });
            }
        }
    }
    // lift (which 0) or drag (which 1) coefficient of calculateLiftAndDrag
    // (def_par:14710-14870), inviscid, with the pressure of the state u
    Dl objective(const std::vector<Dl> *u, int which) const {
        const double PI = 4.0 * std::atan(1.0);
        double aR = c.alpha * PI / 180., bR = c.beta * PI / 180.;
        double ft[3] = {std::cos(aR) * std::cos(bR), std::sin(bR), std::sin(aR)};
        double fn1[3] = {-ft[2], 0.0, ft[0]};
        const double *dir = which == 0 ? fn1 : ft;
        const double pinf = 1. / (c.gamma * c.MachNumber * c.MachNumber);
        const bool visc = c.ReynoldsNumber > 0.0;
        std::vector<Dl> ws[3];
        if (visc) {  // the wall stress of makeViscosityTerm at the state u
            std::vector<Dl> p(N), mu, d[5];
            for (int i = 0; i < N; ++i) p[i] = dabs(pressure(u, i));
            for (auto &x : d) x.assign(N, Dl());
            for (auto &x : ws) x.assign(N, Dl());
            viscous(u, p, d, mu, ws);
        }
        Dl acc;
        for_range(-20, -19, [&](int ip) {
            if (!(g.cz[ip] > (c.groundplane + 0.01))) return;
            Dl dn = (nx[ip] * dir[0] + ny[ip] * dir[1]) + nz[ip] * dir[2];
            Dl dp = pressure(u, ip) - Dl(pinf);
            acc = acc - area[ip] * dp * dn;
            if (visc) {
                Dl sd = (ws[0][ip] * dir[0] + ws[1][ip] * dir[1]) + ws[2][ip] * dir[2];
                acc = acc + area[ip] * sd;
            }
        });
        return Dl(2.0) * acc / Dl(c.referenceArea);
    }
};

}  // namespace

struct oracle_ctx {
    Oracle o;
};

// The geometry of a level from its descriptor (readGridComputationData,
// def_par:13812-14074): coefficients, side lengths, volumes, wall distances,
// coordinates and their movement, restriction weights, the normals, wall
// area and connectivity derived from them; for a moving mesh the GCL
// weights, combined as 1.5 GCL - 0.5 GCLprev on level 1 with timeScheme 2
// (def_par:816-818, 13858-13860), and the previous volumes.
static int load_geometry(Oracle &o, Level &g, int l, const flite_level_desc &d) {
    const size_t E = g.E, B = g.B, N = g.N;
    g.wx.resize(E); g.wy.resize(E); g.wz.resize(E); g.slen.assign(E, 0.0);
    for (size_t e = 0; e < E; ++e) {
        g.wx[e] = d.side_w[e]; g.wy[e] = d.side_w[E + e]; g.wz[e] = d.side_w[2 * E + e];
        if (d.side_len) g.slen[e] = d.side_len[e];
    }
    g.bwx.resize(B); g.bwy.resize(B); g.bwz.resize(B);
    for (size_t b = 0; b < B; ++b) {
        g.bwx[b] = d.bnd_w[b]; g.bwy[b] = d.bnd_w[B + b]; g.bwz[b] = d.bnd_w[2 * B + b];
    }
    g.V.assign(d.volume, d.volume + N);
    g.wdist.assign(N, 0.0);
    if (d.wall_dist) g.wdist.assign(d.wall_dist, d.wall_dist + N);
    g.cx.assign(N, 0.0); g.cy.assign(N, 0.0); g.cz.assign(N, 0.0);
    if (l == 0 && d.coords)
        for (size_t i = 0; i < N; ++i) {
            g.cx[i] = d.coords[i]; g.cy[i] = d.coords[N + i]; g.cz[i] = d.coords[2 * N + i];
        }
    g.cmx.assign(N, 0.0); g.cmy.assign(N, 0.0); g.cmz.assign(N, 0.0);
    if (l == 0 && d.coord_move)
        for (size_t i = 0; i < N; ++i) {
            g.cmx[i] = d.coord_move[i]; g.cmy[i] = d.coord_move[N + i]; g.cmz[i] = d.coord_move[2 * N + i];
        }
    if (l > 0) {
        if (!d.rweight) return FLITE_EINVAL;
        g.rweight.assign(d.rweight, d.rweight + o.lv[l - 1].N);
    }
    if (o.c.flowType == 2) {
        if (!d.side_gcl || !d.bnd_gcl || (l == 0 && (!d.volume_prev || !d.volume_prev2))) return FLITE_EINVAL;
        const bool comb = l == 0 && o.c.timeScheme == 2;
        auto w = [&](double x, double xp) { return comb ? 1.5 * x - 0.5 * xp : x; };
        g.gcl.resize(E); g.bgcl1.resize(B); g.bgcl2.resize(B);
        for (size_t e = 0; e < E; ++e) g.gcl[e] = w(d.side_gcl[e], d.side_gcl[E + e]);
        for (size_t b = 0; b < B; ++b) {
            g.bgcl1[b] = w(d.bnd_gcl[b], d.bnd_gcl[2 * B + b]);
            g.bgcl2[b] = w(d.bnd_gcl[B + b], d.bnd_gcl[3 * B + b]);
        }
        if (l == 0) {
            g.Vp.assign(d.volume_prev, d.volume_prev + N);
            g.Vp2.assign(d.volume_prev2, d.volume_prev2 + N);
        }
    }
    o.setup_level(g);
    return FLITE_OK;
}

extern "C" {

int oracle_create(const flite_controls *c, int nlevels, const flite_level_desc *lv, oracle_ctx **out) {
    if (!c || !lv || !out || nlevels < 1) return FLITE_EINVAL;
    int st = check_controls(*c);
    if (st) return st;
    auto ctx = std::make_unique<oracle_ctx>();
    Oracle &o = ctx->o;
    o.c = *c;
    o.set_stages(c->rungeKuttaStages);
    o.pts_global = c->physicalTimeStep;
    o.nvar = c->turbulenceModel == 1 ? 6 : 5;
    int G = nlevels;
    if (c->numberOfGridsToUse > 0) G = std::min(G, c->numberOfGridsToUse);
    o.lv.resize(G);
    for (int l = 0; l < G; ++l) {
        const flite_level_desc &d = lv[l];
        Level &g = o.lv[l];
        g.grid = l + 1;
        g.N = d.n_nodes; g.E = d.n_sides; g.B = d.n_bsides; g.Nb = d.n_bnodes; g.nnorm = d.n_normals;
        g.s1.resize(g.E); g.s2.resize(g.E);
        for (int e = 0; e < g.E; ++e) {
            g.s1[e] = d.side_idx[e] - 1; g.s2[e] = d.side_idx[(size_t)g.E + e] - 1;
        }
        g.b1.resize(g.B); g.b2.resize(g.B); g.bind.resize(g.B);
        for (int b = 0; b < g.B; ++b) {
            g.b1[b] = d.bnd_idx[b] - 1; g.b2[b] = d.bnd_idx[(size_t)g.B + b] - 1;
            g.bind[b] = d.bnd_idx[2 * (size_t)g.B + b];
            if (g.bind[b] >= 5 && g.bind[b] <= 8) o.engines = true;
        }
        std::memcpy(g.reg, d.node_reg, sizeof g.reg);
        for (int r = -12; r <= -5; r += 2)
            if (g.R(r + 1) >= g.R(r)) o.engines = true;  // engine nodes
        const int ne = d.n_engine_sides;
        if (ne < 0 || (ne > 0 && (!d.engine_idx || !d.engine_w))) return FLITE_EINVAL;
        g.e1.resize(ne); g.e2.resize(ne); g.ein.resize(ne);
        g.ewx.resize(ne); g.ewy.resize(ne); g.ewz.resize(ne);
        for (int s = 0; s < ne; ++s) {
            g.e1[s] = d.engine_idx[s] - 1; g.e2[s] = d.engine_idx[(size_t)ne + s] - 1;
            g.ein[s] = d.engine_idx[2 * (size_t)ne + s] - 1;
            if (g.e1[s] < 0 || g.e1[s] >= g.N || g.e2[s] < 0 || g.e2[s] >= g.N || g.ein[s] < 0 || g.ein[s] > 1)
                return FLITE_EINVAL;
            g.ewx[s] = d.engine_w[s]; g.ewy[s] = d.engine_w[(size_t)ne + s]; g.ewz[s] = d.engine_w[2 * (size_t)ne + s];
        }
        if (ne > 0) o.engines = true;
        // engine conditions on a moving mesh would need the engine sides of
        // every step
        if (o.engines && c->flowType == 2) return FLITE_EUNSUPPORTED;
        g.node_ind.resize(g.nnorm);
        for (int i = 0; i < g.nnorm; ++i) g.node_ind[i] = d.node_ind[i] - 1;
        if (l > 0) {
            int nf = o.lv[l - 1].N;
            if (!d.parent || !d.rweight) return FLITE_EINVAL;
            g.parent.resize(nf);
            for (int i = 0; i < nf; ++i) g.parent[i] = d.parent[i] - 1;
        }
        if (int rc = load_geometry(o, g, l, d)) return rc;
        for (int k = 0; k < 6; ++k) {
            g.u[k].assign(g.N, 0.0); g.uprev[k].assign(g.N, 0.0); g.rhs[k].assign(g.N, 0.0);
            g.src[k].assign(g.N, 0.0);
        }
        for (int k = 0; k < 5; ++k) g.diss[k].assign(g.N, 0.0);
        for (int k = 0; k < 6; ++k) { g.uold[k].assign(g.N, 0.0); g.uold2[k].assign(g.N, 0.0); }
        g.p.assign(g.N, 0.0); g.dt.assign(g.N, 0.0); g.mu.assign(g.N, 0.0);
        g.turbDiff.assign(g.N, 0.0); g.dtT.assign(g.N, 0.0); g.vort.assign(g.N, 0.0); g.divg.assign(g.N, 0.0);
        for (int k = 0; k < 3; ++k) g.wallStress[k].assign(g.N, 0.0);
        g.cycleNumber = l == 0 ? 1 : 0;
    }
    o.nh.assign(25, vec(o.lv[0].N, 0.0));
    *out = ctx.release();
    return FLITE_OK;
}

int oracle_destroy(oracle_ctx *o) { delete o; return FLITE_OK; }

static Level *lvl(oracle_ctx *o, int level) {
    if (!o || level < 1 || level > (int)o->o.lv.size()) return nullptr;
    return &o->o.lv[level - 1];
}

int oracle_set_state(oracle_ctx *o, int level, const double *u) {
    Level *g = lvl(o, level);
    if (!g || !u) return FLITE_EINVAL;
    for (int k = 0; k < o->o.nvar; ++k) std::memcpy(g->u[k].data(), u + (size_t)k * g->N, 8 * (size_t)g->N);
    return FLITE_OK;
}

int oracle_get_state(oracle_ctx *o, int level, double *u) {
    Level *g = lvl(o, level);
    if (!g || !u) return FLITE_EINVAL;
    for (int k = 0; k < o->o.nvar; ++k) std::memcpy(u + (size_t)k * g->N, g->u[k].data(), 8 * (size_t)g->N);
    return FLITE_OK;
}

int oracle_get_pressure(oracle_ctx *o, int level, double *p) {
    Level *g = lvl(o, level);
    if (!g || !p) return FLITE_EINVAL;
    std::memcpy(p, g->p.data(), 8 * (size_t)g->N);
    return FLITE_OK;
}

int oracle_get_array(oracle_ctx *o, int level, const char *name, double *out) {
    Level *g = lvl(o, level);
    if (!g || !name || !out) return FLITE_EINVAL;
    const size_t N = g->N;
    std::string n(name);
    auto cols = [&](const vec *a, int nc) { for (int k = 0; k < nc; ++k) std::memcpy(out + k * N, a[k].data(), 8 * N); };
    if (n == "dt") std::memcpy(out, g->dt.data(), 8 * N);
    else if (n == "diss") cols(g->diss, 5);
    else if (n == "rhs") cols(g->rhs, 5);
    else if (n == "uprev") cols(g->uprev, 5);
    else if (n == "src") cols(g->src, 5);
    else if (n == "mu") std::memcpy(out, g->mu.data(), 8 * N);
    else if (n == "conn") std::memcpy(out, g->conn.data(), 8 * N);
    else if (n == "turbDiff") std::memcpy(out, g->turbDiff.data(), 8 * N);
    else if (n == "dtT") std::memcpy(out, g->dtT.data(), 8 * N);
    else if (n == "vort") std::memcpy(out, g->vort.data(), 8 * N);
    else if (n == "div") std::memcpy(out, g->divg.data(), 8 * N);
    else if (n == "wallArea") std::memcpy(out, g->wallArea.data(), 8 * N);
    else if (n == "wallStress") cols(g->wallStress, 3);
    else if (n == "normal") {
        std::memcpy(out, g->nx.data(), 8 * N); std::memcpy(out + N, g->ny.data(), 8 * N);
        std::memcpy(out + 2 * N, g->nz.data(), 8 * N);
    } else if (n == "grad") {
        for (int k = 0; k < 15; ++k) std::memcpy(out + k * N, o->o.nh[k].data(), 8 * N);
    } else return FLITE_EINVAL;
    return FLITE_OK;
}

int oracle_init_freestream(oracle_ctx *o) {
    if (!o) return FLITE_EINVAL;
    Level &g = o->o.lv[0];
    for (int i = 0; i < g.N; ++i)
        for (int k = 0; k < 5; ++k) g.u[k][i] = o->o.c.inflowField[k];
    // setUpInitialField2's freestream branch (def_par:3953-3963)
    if (o->o.c.ReynoldsNumber > 0.0) std::fill(g.mu.begin(), g.mu.end(), 1. / o->o.c.ReynoldsNumber);
    if (o->o.sa()) std::fill(g.u[5].begin(), g.u[5].end(), 0.1);
    return FLITE_OK;
}

static void physical_step_head(Oracle &O);

int oracle_start(oracle_ctx *o) {
    if (!o) return FLITE_EINVAL;
    Oracle &O = o->o;
    Level &g = O.lv[0];
    O.makePressureField(g, g.u);
    g.cycleNumber = 1;
    O.setBCsOnSolutionField(g, g.u);
    if (O.c.flowType != 0)  // uold = uold2 = u (def_par:3594-3596)
        for (int k = 0; k < O.nvar; ++k) { g.uold[k] = g.u[k]; g.uold2[k] = g.u[k]; }
    physical_step_head(O);
    return FLITE_OK;
}

// the head of a physical time step (mg_par:586-602): laminar viscosity on
// every level, u and (unsteady) uold restricted to every coarse level
static void physical_step_head(Oracle &O) {
    const double mu = O.c.ReynoldsNumber > 0.0 ? 1. / O.c.ReynoldsNumber : 0.0;
    for (size_t l = 0; l < O.lv.size(); ++l) {
        std::fill(O.lv[l].mu.begin(), O.lv[l].mu.end(), mu);
        if (l > 0) {
            O.mapFineToCoarse(O.lv[l - 1], O.lv[l], O.lv[l - 1].u, O.lv[l].u, O.nvar);
            if (O.c.flowType != 0) O.mapFineToCoarse(O.lv[l - 1], O.lv[l], O.lv[l - 1].uold, O.lv[l].uold, O.nvar);
        }
    }
}

int oracle_explicit_time_step(oracle_ctx *o, double *dt) {
    if (!o || !dt) return FLITE_EINVAL;
    *dt = o->o.pts_global;
    return FLITE_OK;
}

int oracle_next_physical_step(oracle_ctx *o) {
    if (!o || o->o.c.flowType == 0) return FLITE_EINVAL;
    Oracle &O = o->o;
    Level &g = O.lv[0];
    for (int k = 0; k < O.nvar; ++k) { g.uold2[k] = g.uold[k]; g.uold[k] = g.u[k]; }  // mg_par:889-890
    physical_step_head(O);
    return FLITE_OK;
}

int oracle_update_geometry(oracle_ctx *o, int nlevels, const flite_level_desc *lv) {
    if (!o || !lv || o->o.c.flowType != 2 || nlevels < (int)o->o.lv.size()) return FLITE_EINVAL;
    Oracle &O = o->o;
    for (size_t l = 0; l < O.lv.size(); ++l) {
        Level &g = O.lv[l];
        const flite_level_desc &d = lv[l];
        if (d.n_nodes != g.N || d.n_sides != g.E || d.n_bsides != g.B) return FLITE_EINVAL;
        if (int rc = load_geometry(O, g, (int)l, d)) return rc;
    }
    physical_step_head(O);  // again, with the new restriction weights
    return FLITE_OK;
}

int oracle_do_time_iterations(oracle_ctx *o, int level, int nsteps, int calc_diss, int calc_turb,
                              int cycle_no) {
    if (!lvl(o, level)) return FLITE_EINVAL;
    o->o.calcTurbOfCycle = calc_turb != 0;
    o->o.doTimeIterations(level - 1, nsteps, calc_diss != 0, cycle_no);
    return FLITE_OK;
}

int oracle_restrict(oracle_ctx *o, int fine_level, int calc_turb) {
    if (!lvl(o, fine_level) || !lvl(o, fine_level + 1)) return FLITE_EINVAL;
    o->o.restrictGrid(fine_level - 1, calc_turb != 0);
    return FLITE_OK;
}

int oracle_prolong(oracle_ctx *o, int coarse_level) {
    if (coarse_level < 2 || !lvl(o, coarse_level)) return FLITE_EINVAL;
    o->o.prolongateGrid(coarse_level - 1);
    return FLITE_OK;
}

int oracle_map_fine_to_coarse(oracle_ctx *o, int fine_level) {
    if (!lvl(o, fine_level) || !lvl(o, fine_level + 1)) return FLITE_EINVAL;
    Oracle &O = o->o;
    O.mapFineToCoarse(O.lv[fine_level - 1], O.lv[fine_level], O.lv[fine_level - 1].u, O.lv[fine_level].u, 5);
    return FLITE_OK;
}

int oracle_cycle(oracle_ctx *o, int cycle_no) {
    if (!o) return FLITE_EINVAL;
    try {
        o->o.oneCycle(cycle_no);
    } catch (const std::exception &) {
        return FLITE_EUNSUPPORTED;
    }
    return FLITE_OK;
}

int oracle_residuals(oracle_ctx *o, double res[7], double maxres[7], int maxind[7]) {
    if (!o) return FLITE_EINVAL;
    Oracle &O = o->o;
    Level &g = O.c.multigridScheme > 0 ? O.lv[0] : O.lv.back();
    const int nres = O.nvar;  // writeResiduals: 6 with SA (mg_par:1292-1293)
    for (int k = 0; k < 7; ++k) { res[k] = 0.0; maxres[k] = 0.0; maxind[k] = 1; }
    for (int k = 0; k < nres; ++k) {
        double s = 0.0;
        for (int i = 0; i < g.N; ++i) {
            double d = g.u[k][i] - g.uprev[k][i];
            s = s + d * d;
        }
        res[k] = std::sqrt(s);
    }
    for (int i = 0; i < g.N; ++i)
        for (int k = 0; k < nres; ++k) {
            double cr = std::fabs(g.u[k][i] - g.uprev[k][i]);
            if (cr > maxres[k]) { maxres[k] = cr; maxind[k] = i + 1; }
        }
    for (int k = 0; k < nres; ++k)
        if (!std::isfinite(res[k])) return FLITE_ENAN;
    return FLITE_OK;
}

int oracle_forces(oracle_ctx *o, double out[9]) {
    if (!o || !out) return FLITE_EINVAL;
    o->o.forces(out);
    return FLITE_OK;
}

// the pinned exp (which = 0) and log (which = 1) of the SA source term,
// exported for their accuracy test
int oracle_pinned_math(int which, const double *x, double *y, int n) {
    if (!x || !y || n < 0) return FLITE_EINVAL;
    for (int i = 0; i < n; ++i) y[i] = which == 0 ? flite_pm::pm_exp(x[i]) : flite_pm::pm_log(x[i]);
    return FLITE_OK;
}

int oracle_set_threads(int n) {
    if (n < 1) return FLITE_EINVAL;
    g_threads = n;
    return FLITE_OK;
}

int oracle_residual_fwd(oracle_ctx *o, int level, const double *u, double *r) {
    Level *g = lvl(o, level);
    if (!g || !u || !r) return FLITE_EINVAL;
    for (int k = 0; k < 5; ++k) std::memcpy(g->u[k].data(), u + (size_t)k * g->N, 8 * (size_t)g->N);
    o->o.makePressureField(*g, g->u);
    for (int k = 0; k < 5; ++k) std::fill(g->rhs[k].begin(), g->rhs[k].end(), 0.0);
    o->o.makeRHS(*g);
    for (int k = 0; k < 5; ++k) std::memcpy(r + (size_t)k * g->N, g->rhs[k].data(), 8 * (size_t)g->N);
    return FLITE_OK;
}

// makeViscosityTerm (def_par:5198-5893) alone at the state u of a level:
// pressure, |p|, then the term subtracted from a zeroed dissipation array;
// diss [5][N] out (column 1 stays 0), with the laminar viscosity mu [N] and,
// on level 1, the wall stress [3][N] it leaves behind
int oracle_viscous_term(oracle_ctx *o, int level, const double *u, double *diss, double *mu,
                        double *wall_stress) {
    Level *g = lvl(o, level);
    if (!g || !u || !diss || !mu || !wall_stress) return FLITE_EINVAL;
    for (int k = 0; k < 5; ++k) std::memcpy(g->u[k].data(), u + (size_t)k * g->N, 8 * (size_t)g->N);
    o->o.makePressureField(*g, g->u);
    for (int i = 0; i < g->N; ++i) g->p[i] = std::fabs(g->p[i]);
    for (int k = 0; k < 5; ++k) std::fill(g->diss[k].begin(), g->diss[k].end(), 0.0);
    o->o.viscousTerm(*g);
    for (int k = 0; k < 5; ++k) std::memcpy(diss + (size_t)k * g->N, g->diss[k].data(), 8 * (size_t)g->N);
    std::memcpy(mu, g->mu.data(), 8 * (size_t)g->N);
    for (int k = 0; k < 3; ++k)
        if (!g->wallStress[k].empty())
            std::memcpy(wall_stress + (size_t)k * g->N, g->wallStress[k].data(), 8 * (size_t)g->N);
    return FLITE_OK;
}

// one column of the shared help array (nodeHelpArray(:, col + 1)) after the
// last evaluation, for tests of the dissipation schemes' intermediate sums
int oracle_help_column(oracle_ctx *o, int col, double *out) {
    if (!o || !out || col < 0 || col >= (int)o->o.nh.size() || o->o.lv.empty()) return FLITE_EINVAL;
    std::memcpy(out, o->o.nh[col].data(), 8 * (size_t)o->o.lv[0].N);
    return FLITE_OK;
}

// the artificial dissipation of singleIteration (def_par:1022-1036) at the
// state u of a level: pressure, |p|, local time steps, then the run's
// dissipation scheme; diss [5][N] out
int oracle_dissipation(oracle_ctx *o, int level, const double *u, double *diss) {
    Level *g = lvl(o, level);
    if (!g || !u || !diss) return FLITE_EINVAL;
    for (int k = 0; k < 5; ++k) std::memcpy(g->u[k].data(), u + (size_t)k * g->N, 8 * (size_t)g->N);
    o->o.makePressureField(*g, g->u);
    for (int i = 0; i < g->N; ++i) g->p[i] = std::fabs(g->p[i]);
    o->o.makeTimeSteps(*g);
    o->o.dissipation_for(*g, false);
    for (int k = 0; k < 5; ++k) std::memcpy(diss + (size_t)k * g->N, g->diss[k].data(), 8 * (size_t)g->N);
    return FLITE_OK;
}


// tangent J du of the residual of oracle_residual_fwd (central flux, wall,
// symmetry and far-field boundary fluxes)
int oracle_residual_jvp(oracle_ctx *o, int level, const double *u, const double *du, double *jv) {
    Level *g = lvl(o, level);
    if (!g || !u || !du || !jv) return FLITE_EINVAL;
    const flite_controls &c = o->o.c;
    if (c.fluxType != 1 || o->o.engines) return FLITE_EUNSUPPORTED;  // tangents of the engine-free path
    const size_t N = g->N;
    std::vector<Dl> acc(5 * N);
    auto state = [&](int i, Dl *q) { for (int k = 0; k < 5; ++k) q[k] = Dl(u[k * N + i], du[k * N + i]); };
    for (int e = 0; e < g->E; ++e) {
        int i1 = g->s1[e], i2 = g->s2[e];
        double w[3] = {g->wx[e], g->wy[e], g->wz[e]};
        Dl q1[5], q2[5], G1[5], G2[5];
        state(i1, q1); state(i2, q2);
        tan_G(q1, tan_pressure(c, q1), w, G1);
        tan_G(q2, tan_pressure(c, q2), w, G2);
        for (int k = 0; k < 5; ++k) {
            Dl f = G1[k] + G2[k];
            acc[k * N + i1] = acc[k * N + i1] + f;
            acc[k * N + i2] = acc[k * N + i2] - f;
        }
    }
    const bool fe = c.boundaryTerm == 1;
    for (int b = 0; b < g->B; ++b) {
        int i1 = g->b1[b], i2 = g->b2[b], ind = g->bind[b];
        double w[3] = {g->bwx[b], g->bwy[b], g->bwz[b]};
        double rn = std::sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]);
        if (!(rn > 1.0e-10)) continue;
        Dl q1[5], q2[5], F1[5], F2[5];
        state(i1, q1); state(i2, q2);
        if (ind <= 2 || ind == 9) {
            tan_G(q1, tan_pressure(c, q1), w, F1);
            tan_G(q2, tan_pressure(c, q2), w, F2);
            for (int k = 0; k < 5; ++k) { F1[k] = F1[k] / Dl(rn); F2[k] = F2[k] / Dl(rn); }
        } else if (ind <= 4) {
            double n[3] = {w[0] / rn, w[1] / rn, w[2] / rn};
            const double *inf = &c.inflowField[(ind - 3) * 6];
            tan_farfield(c, q1, tan_pressure(c, q1), n, inf, F1);
            tan_farfield(c, q2, tan_pressure(c, q2), n, inf, F2);
        } else {
            continue;
        }
        for (int k = 0; k < 5; ++k) {
            Dl g1 = fe ? Dl(rn) * (Dl(3.) * F1[k] + F2[k]) : Dl(rn) * Dl(4.) * F1[k];
            Dl g2 = fe ? Dl(rn) * (F1[k] + Dl(3.) * F2[k]) : Dl(rn) * Dl(4.) * F2[k];
            acc[k * N + i1] = acc[k * N + i1] + g1;
            acc[k * N + i2] = acc[k * N + i2] + g2;
        }
    }
    for (size_t k = 0; k < 5 * N; ++k) jv[k] = acc[k].d;
    return FLITE_OK;
}

// tangent of one smoother iteration on level 1 (central flux, scalar JST,
// inviscid): v = G(u), dv = G_u du + G_g dg for the geometry direction dg =
// (dsw [3][E], dbw [3][B], dvol [N]); any of the geometry directions may be
// NULL (zero)
int oracle_iteration_jvp(oracle_ctx *o, const double *u, const double *du, const double *dsw, const double *dbw,
                         const double *dvol, double *v, double *dv, const double *mu, const double *dmu,
                         double *mu_out, double *dmu_out) {
    if (!o || !u || !du || !v || !dv) return FLITE_EINVAL;
    const flite_controls &c = o->o.c;
    if (c.fluxType != 1 || c.turbulenceModel != 0 || c.dissipationScheme == 1 || c.dissipationScheme == 3 ||
        c.useDissipationWeighting || (c.ReynoldsNumber > 0 && c.viscosityScheme != 1) ||
        c.useMatrixDissipation || c.flowType != 0 || c.rungeKuttaStages != 3 || o->o.engines)
        return FLITE_EUNSUPPORTED;
    const bool visc = c.ReynoldsNumber > 0;
    if (visc && (!mu || !mu_out || !dmu_out)) return FLITE_EINVAL;
    TanIteration T(o->o, dsw, dbw, dvol);
    const size_t N = T.N;
    std::vector<Dl> x[5], m(N);
    for (int k = 0; k < 5; ++k) {
        x[k].resize(N);
        for (size_t i = 0; i < N; ++i) x[k][i] = Dl(u[k * N + i], du[k * N + i]);
    }
    if (visc)
        for (size_t i = 0; i < N; ++i) m[i] = Dl(mu[i], dmu ? dmu[i] : 0.0);
    T.iterate(x, &m);
    for (int k = 0; k < 5; ++k)
        for (size_t i = 0; i < N; ++i) { v[k * N + i] = x[k][i].v; dv[k * N + i] = x[k][i].d; }
    if (visc)
        for (size_t i = 0; i < N; ++i) { mu_out[i] = m[i].v; dmu_out[i] = m[i].d; }
    return FLITE_OK;
}

// lift (which 0) or drag (which 1) coefficient of the level-1 state u with
// its tangent along (du, dsw, dbw, dvol); the geometry directions may be NULL
int oracle_objective_jvp(oracle_ctx *o, int which, const double *u, const double *du, const double *dsw,
                         const double *dbw, const double *dvol, double *J, double *dJ) {
    if (!o || !u || !du || !J || !dJ || which < 0 || which > 1) return FLITE_EINVAL;
    if (o->o.c.turbulenceModel != 0 || o->o.engines) return FLITE_EUNSUPPORTED;
    if (o->o.c.ReynoldsNumber > 0 && o->o.c.viscosityScheme != 1) return FLITE_EUNSUPPORTED;
    TanIteration T(o->o, dsw, dbw, dvol);
    const size_t N = T.N;
    std::vector<Dl> x[5];
    for (int k = 0; k < 5; ++k) {
        x[k].resize(N);
        for (size_t i = 0; i < N; ++i) x[k][i] = Dl(u[k * N + i], du[k * N + i]);
    }
    Dl j = T.objective(x, which);
    *J = j.v;
    *dJ = j.d;
    return FLITE_OK;
}

}  // extern "C"

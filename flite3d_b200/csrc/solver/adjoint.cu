// Discrete adjoint of the edge residual: the transpose Jacobian-vector
// product ubar = (dR/du)^T rbar of makeRHS (def_par:1525-2512) for the
// central interior flux and the wall/symmetry/far-field boundary fluxes.
//
// The central flux of an edge and the wall flux of a boundary edge are sums of
// one-sided fluxes G(u; w) = F(u).w, linear in the coefficients w:
//   interior  f = G(u1; w) + G(u2; w), rhs(i1) += f, rhs(i2) -= f
//   wall      g1 = 3G(u1; w) + G(u2; w), g2 = G(u1; w) + 3G(u2; w)
// so for node i,  ubar_i = sum_d A_d(u_i)^T b_d  with  b_d = sum over its
// edges of w_d times the adjoint weights (rbar(i1)-rbar(i2) for interior
// edges, 3 rbar_own + rbar_other for wall edges); A_d = dF_d/du with the
// pressure p(u) (zero derivative where the 0.1 floor holds).  One node
// gather builds b_d and one 3x(5x5) transpose product per node finishes it:
// no edge buffer, and nothing stored beyond the state.
// The far-field Roe flux against the freestream (def_par:2258-2446) is
// nonlinear in the normal; its 5x5 Jacobians are formed with forward-mode
// dual numbers per far-field edge.
#include <cuda_runtime.h>

#include "adjoint.cuh"
#include "context.h"
#include "flux.cuh"

namespace flite {

// far-field contributions per boundary edge: J(u_b1)^T |w|(3 rbar1 + rbar2)
// and J(u_b2)^T |w|(rbar1 + 3 rbar2) (FV weighting: 4 rbar_own)
__global__ void k_vjp_farfield(Params P, LevelView L, const double *x, const double *rbar, double *bvjp) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= L.B) return;
    double *o = bvjp + (size_t)b * 10;
    for (int k = 0; k < 10; ++k) o[k] = 0.0;
    const int ind = L.bind[b];
    if (ind != 3 && ind != 4) return;
    const double wx = L.bwx[b], wy = L.bwy[b], wz = L.bwz[b];
    const double rnorm = sqrt((wx * wx + wy * wy) + wz * wz);
    if (!(rnorm > 1.0e-10)) return;
    const double rnx = wx / rnorm, rny = wy / rnorm, rnz = wz / rnorm;
    const double *inf = &P.inf[(ind - 3) * 6];
    const int2 nd = L.bedge[b];
    const int N = L.N;
    const bool fe = P.boundaryTerm == 1;
    for (int side = 0; side < 2; ++side) {
        const int n = side == 0 ? nd.x : nd.y;
        double a[5];
        for (int k = 0; k < 5; ++k) {
            double r1 = rbar[(size_t)k * N + nd.x], r2 = rbar[(size_t)k * N + nd.y];
            a[k] = fe ? rnorm * (side == 0 ? 3. * r1 + r2 : r1 + 3. * r2) : rnorm * 4. * (side == 0 ? r1 : r2);
        }
        double u[5], p, dp[5];
        for (int k = 0; k < 5; ++k) u[k] = x[(size_t)k * N + n];
        pressure_grad(P, u, &p, dp);
        for (int j = 0; j < 5; ++j) {  // column j of the Jacobian
            Dual q[5];
            for (int k = 0; k < 5; ++k) q[k] = Dual(u[k], k == j ? 1.0 : 0.0);
            Dual F[5];
            farfield_dual(P, q, Dual(p, dp[j]), rnx, rny, rnz, inf, F);
            double s = 0.0;
            for (int k = 0; k < 5; ++k) s += F[k].d * a[k];
            o[side * 5 + j] = s;
        }
    }
}

// ubar = (dR/dx)^T rbar at the state x, plus pbar (dp/dx) when pbar is given
// (a pressure read by the caller's own use of the state); add = 1 adds the
// product to ubar instead of storing it
__global__ void k_vjp_node(Params P, LevelView L, const double *x, const double *rbar, const double *bvjp,
                           const double *pbar, double *ubar, int add) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.N) return;
    const int N = L.N;
    double b[3][5];
    for (int d = 0; d < 3; ++d)
        for (int k = 0; k < 5; ++k) b[d][k] = 0.0;
    double ri[5];
    for (int k = 0; k < 5; ++k) ri[k] = rbar[(size_t)k * N + i];
    for (int q = L.inc_ptr[i]; q < L.inc_ptr[i + 1]; ++q) {
        int2 t = L.inc[q];
        int e = t.x >= 0 ? t.x : ~t.x, j = t.y;
        const double w[3] = {L.wx[e], L.wy[e], L.wz[e]};
        double a[5];
        for (int k = 0; k < 5; ++k) {
            double rj = rbar[(size_t)k * N + j];
            a[k] = t.x >= 0 ? ri[k] - rj : rj - ri[k];  // rbar(i1) - rbar(i2)
        }
        for (int d = 0; d < 3; ++d)
            for (int k = 0; k < 5; ++k) b[d][k] += w[d] * a[k];
    }
    double extra[5] = {0, 0, 0, 0, 0};
    const bool fe = P.boundaryTerm == 1;
    for (int q = L.binc_ptr[i]; q < L.binc_ptr[i + 1]; ++q) {
        int bb = L.binc[q] >> 1, side = L.binc[q] & 1;
        int ind = L.bind[bb];
        if (ind == 3 || ind == 4) {
            for (int k = 0; k < 5; ++k) extra[k] += bvjp[(size_t)bb * 10 + side * 5 + k];
            continue;
        }
        if (!(ind <= 2 || ind == 9)) continue;
        const double w[3] = {L.bwx[bb], L.bwy[bb], L.bwz[bb]};
        if (!(sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]) > 1.0e-10)) continue;
        const int2 nd = L.bedge[bb];
        double a[5];
        for (int k = 0; k < 5; ++k) {
            double r1 = rbar[(size_t)k * N + nd.x], r2 = rbar[(size_t)k * N + nd.y];
            a[k] = fe ? (side == 0 ? 3. * r1 + r2 : r1 + 3. * r2) : 4. * (side == 0 ? r1 : r2);
        }
        for (int d = 0; d < 3; ++d)
            for (int k = 0; k < 5; ++k) b[d][k] += w[d] * a[k];
    }
    double u[5], ub[5];
    for (int k = 0; k < 5; ++k) u[k] = x[(size_t)k * N + i];
    apply_flux_jacobian_t(P, u, b, ub);
    if (pbar) {
        double p, dp[5];
        pressure_grad(P, u, &p, dp);
        const double pb = pbar[i];
        for (int k = 0; k < 5; ++k) extra[k] += pb * dp[k];
    }
    for (int k = 0; k < 5; ++k) {
        const double v = ub[k] + extra[k];
        ubar[(size_t)k * N + i] = add ? ubar[(size_t)k * N + i] + v : v;
    }
}

}  // namespace flite

extern "C" int flite_residual_vjp(flite_ctx *ctx, int level, const double *u, const double *rbar, double *ubar) {
    if (!ctx || level < 1 || level > (int)ctx->lv.size() || !u || !rbar || !ubar) return FLITE_EINVAL;
    // the transpose of the static-mesh residual (no GCL terms)
    if (ctx->c.fluxType != 1 || ctx->c.precision != FLITE_FP64 || ctx->c.flowType == 2 || ctx->P.engines)
        return FLITE_EUNSUPPORTED;  // the products of the engine-free residual
    try {
        flite_ctx &X = *ctx;
        LevelView &L = X.V(level - 1);
        const size_t n5 = 5 * (size_t)L.N;
        // the adjoint input and output reuse the level's residual and
        // dissipation-sized state buffers are not touched: dedicated buffers
        if (!X.adj_rbar || X.adj_n < n5) {
            if (X.adj_rbar) { cudaFree(X.adj_rbar); cudaFree(X.adj_ubar); cudaFree(X.adj_b); }
            CK(cudaMalloc(&X.adj_rbar, n5 * sizeof(double)));
            CK(cudaMalloc(&X.adj_ubar, n5 * sizeof(double)));
            size_t maxB = 1;
            for (auto &D : X.lv) maxB = std::max(maxB, (size_t)D.B);
            CK(cudaMalloc(&X.adj_b, 10 * maxB * sizeof(double)));
            X.adj_n = n5;
        }
        X.put_nodes(level - 1, L.u, u, 5);
        X.put_nodes(level - 1, X.adj_rbar, rbar, 5);
        X.vjp_kernels(level - 1);
        X.get_nodes(level - 1, ubar, X.adj_ubar, 5);
        CK(cudaStreamSynchronize(X.s));
        return FLITE_OK;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return FLITE_ECUDA;
    }
}

void flite_ctx::vjp_kernels(int l) {
    LevelView &L = V(l);
    if (L.B > 0) k_vjp_farfield<<<eblk(L.B), eb, 0, s>>>(P, L, L.u, adj_rbar, adj_b);
    k_vjp_node<<<nblk(L.N), nb, 0, s>>>(P, L, L.u, adj_rbar, adj_b, nullptr, adj_ubar, 0);
}

extern "C" int flite_profile_adjoint(flite_ctx *ctx, int level, int reps, double *fwd_ms, double *vjp_ms) {
    if (!ctx || level < 1 || level > (int)ctx->lv.size() || reps < 1 || !fwd_ms || !vjp_ms) return FLITE_EINVAL;
    if (ctx->c.fluxType != 1 || ctx->c.precision != FLITE_FP64) return FLITE_EUNSUPPORTED;
    try {
        flite_ctx &X = *ctx;
        const int l = level - 1;
        LevelView &L = X.V(l);
        const size_t n5 = 5 * (size_t)L.N;
        if (!X.adj_rbar || X.adj_n < n5) {
            std::vector<double> zero(n5, 1.0);
            std::vector<double> u(n5);
            X.get_nodes(l, u.data(), L.u, 5);
            CK(cudaStreamSynchronize(X.s));
            std::vector<double> out(n5);
            int rc = flite_residual_vjp(ctx, level, u.data(), zero.data(), out.data());
            if (rc != FLITE_OK) return rc;
        }
        cudaEvent_t e[4];
        for (auto &x : e) CK(cudaEventCreate(&x));
        double tf = 0, tv = 0;
        for (int r = 0; r < reps; ++r) {
            // forward residual: pressure, edge fluxes, boundary fluxes, gather
            CK(cudaEventRecord(e[0], X.s));
            X.pressure(l);
            X.rhs_terms(l);
            X.launch_node_update(l, MODE_RESID, 0, true);
            CK(cudaEventRecord(e[1], X.s));
            CK(cudaEventRecord(e[2], X.s));
            X.vjp_kernels(l);
            CK(cudaEventRecord(e[3], X.s));
            CK(cudaEventSynchronize(e[3]));
            float a = 0, b = 0;
            CK(cudaEventElapsedTime(&a, e[0], e[1]));
            CK(cudaEventElapsedTime(&b, e[2], e[3]));
            tf += a; tv += b;
        }
        for (auto &x : e) cudaEventDestroy(x);
        *fwd_ms = tf / reps;
        *vjp_ms = tv / reps;
        return FLITE_OK;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return FLITE_ECUDA;
    }
}

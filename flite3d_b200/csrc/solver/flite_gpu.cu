// Host side of the C ABI (include/flite_gpu.h): context, device layout and
// the orchestration of the reference's solver calls as kernel sequences.
//
// The call structure mirrors SolverSource/mgnsg3d_def_par.F90 and
// mgnsg3d_mg_par.F90 routine for routine (cited at each function); only the
// inner loops moved into the kernels of kernels.cu.  One oneCycle is a fixed
// kernel sequence for given controls, so it is captured once into a CUDA
// graph and replayed; the cycle number reaches the kernels through device
// memory so the same graph serves every cycle.
#include <cuda_runtime.h>

#include <functional>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "context.h"
#include "renumber.h"

namespace {

// Message of the calling thread's last failed flite_create/flite_batch_create,
// which leave no context to hold it; flite_last_error(NULL, ...) returns it.
thread_local std::string t_create_err;

int fail(flite_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

template <class F>
int guarded(flite_ctx *ctx, F &&f) {
    if (!ctx) return FLITE_EINVAL;
    try {
        return f();
    } catch (const cuda_error &e) {
        return fail(ctx, FLITE_ECUDA, e.what());
    } catch (const std::bad_alloc &) {
        return fail(ctx, FLITE_ENOMEM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(ctx, FLITE_EINVAL, e.what());
    }
}

// The staging data of the tiled gathers of one level (TileView).
struct TileHost {
    int ntiles = 0, stage_max = 0;
    std::vector<int> halo_ptr, halo, row;
    std::vector<unsigned> meta, nmeta;
    std::vector<double> wx, wy, wz;
};

void build_tiles(int N, const std::vector<int> &ip, const std::vector<int2> &inc, const std::vector<double> &wx,
                 const std::vector<double> &wy, const std::vector<double> &wz, TileHost &T) {
    if (N <= 0 || N >= (int)kTileIndexMask) return;
    T.ntiles = (N + kTile - 1) / kTile;
    T.halo_ptr.assign(T.ntiles + 1, 0);
    T.row.assign(T.ntiles + 1, 0);
    for (int t = 0; t < T.ntiles; ++t) {
        const int n0 = t * kTile, n1 = std::min(N, n0 + kTile);
        int kmax = 0;
        for (int i = n0; i < n1; ++i) kmax = std::max(kmax, ip[i + 1] - ip[i]);
        T.row[t + 1] = T.row[t] + kmax;
    }
    const size_t cells = (size_t)T.row[T.ntiles] * kTile;
    T.meta.assign(std::max<size_t>(cells, 1), 0u);
    T.nmeta.assign(std::max<size_t>(cells, 1), 0u);
    T.wx.assign(std::max<size_t>(cells, 1), 0.0);
    T.wy.assign(std::max<size_t>(cells, 1), 0.0);
    T.wz.assign(std::max<size_t>(cells, 1), 0.0);
    T.stage_max = kTile;
    std::vector<int> h;
    for (int t = 0; t < T.ntiles; ++t) {
        const int n0 = t * kTile, n1 = std::min(N, n0 + kTile);
        h.clear();
        for (int i = n0; i < n1; ++i)
            for (int k = ip[i]; k < ip[i + 1]; ++k) {
                const int j = inc[k].y;
                if (j < n0 || j >= n1) h.push_back(j);
            }
        std::sort(h.begin(), h.end());
        h.erase(std::unique(h.begin(), h.end()), h.end());
        T.halo_ptr[t + 1] = T.halo_ptr[t] + (int)h.size();
        T.halo.insert(T.halo.end(), h.begin(), h.end());
        const int staged = std::min((int)h.size(), kTileStageMax - kTile);
        T.stage_max = std::max(T.stage_max, kTile + staged);
        for (int i = n0; i < n1; ++i)
            for (int k = ip[i]; k < ip[i + 1]; ++k) {
                const int es = inc[k].x, j = inc[k].y, e = es >= 0 ? es : ~es;
                unsigned m;
                if (j >= n0 && j < n1) {
                    m = (unsigned)(j - n0);
                } else {
                    const int pos = (int)(std::lower_bound(h.begin(), h.end(), j) - h.begin());
                    m = pos < staged ? (unsigned)(kTile + pos) : (kTileGlobal | (unsigned)j);
                }
                const unsigned second = es < 0 ? kTileSecond : 0u;
                const size_t x = ((size_t)T.row[t] + (k - ip[i])) * kTile + (i - n0);
                T.meta[x] = m | second;
                T.nmeta[x] = kTileGlobal | (unsigned)j | second;
                T.wx[x] = wx[e]; T.wy[x] = wy[e]; T.wz[x] = wz[e];
            }
    }
    if (T.halo.empty()) T.halo.push_back(0);
}

const char *unsupported_reason(const flite_controls &c) {
    if (c.flowType != 0 && c.flowType != 1 && c.flowType != 2)
        return "flowType must be 0 (steady), 1 (unsteady, static mesh) or 2 (unsteady, moving mesh)";
    if (c.flowType != 0 && !(c.physicalTimeStep > 0)) return "unsteady runs need physicalTimeStep > 0";
    if (c.flowType == 2 && c.precision != FLITE_FP64) return "moving meshes (flowType 2) run in FP64";
    if (c.flowType == 2 && c.reconstruction != FLITE_RECON_NONE)
        return "moving meshes (flowType 2) take the reference's fluxes (no reconstruction extension)";
    if (c.forceCalcType != 1 && c.forceCalcType != 3)
        return "forceCalcType must be 1 or 3 (2 is the spanwise load of gust runs)";
    // SAS acts only on the SST model (turbulenceModel 3, def_par:1053-1056, 9002)
    // and patchInitialization only in the interactive start-up of
    // communicateSeq (setUpInitialField, def_par:3620-3675; mg_par:1579): both
    // are read and have no effect on this path, as in the reference's solver
    if (c.GUSTMODEL || c.movingwall || c.nspan != 0)
        return "gust, moving-wall and spanwise loads are not supported";
    if (c.residualSmoothingFactor > 0 || c.prolongationSmoothingFactor > 0)
        return "residual and prolongation smoothing are not supported";
    if (c.turbulenceModel != 0 && c.turbulenceModel != 1)
        return "turbulenceModel 2 and 3 (k-omega, SST) are not supported";
    if (c.turbulenceModel == 1 && !(c.ReynoldsNumber > 0)) return "the Spalart-Allmaras model needs ReynoldsNumber > 0";
    if (c.turbulenceModel == 1 && c.precision != FLITE_FP64) return "the Spalart-Allmaras model runs in FP64";
    if (c.ReynoldsNumber > 0 && c.viscosityScheme != 1 && c.viscosityScheme != 2)
        return "viscosityScheme must be 1 or 2";
    if (c.fluxType < 1 || c.fluxType > 4) return "fluxType must be 1..4";
    if (c.fluxType == 4 && c.HLLCFluxOrder > 1 && c.GradientMethod != 1 && c.numberOfGridsToUse != 1)
        return "least-squares gradients need numberOfGridsToUse = 1: the reference's LS gradient divides "
               "by |dx|^2 of coarse-level coordinates it never fills";
    if (c.coarseGridDissipationScheme == 1)
        return "coarseGridDissipationScheme 1 is not supported: the reference's scheme 1 on a coarse level reads "
               "coordinates through finer-level seed indices beyond the coarse arrays";
    if (c.prolongationMappingScheme != 1) return "prolongationMappingScheme must be 1";
    if (c.precision != FLITE_FP64 && c.precision != FLITE_MIXED) return "precision must be FLITE_FP64 or FLITE_MIXED";
    if (c.precision == FLITE_MIXED && c.fluxType != 1) return "FLITE_MIXED supports the central flux (fluxType 1)";
    if (c.rungeKuttaStages != 3 && c.rungeKuttaStages != 5) return "rungeKuttaStages must be 3 or 5";
    if (c.reconstruction != FLITE_RECON_NONE && c.reconstruction != FLITE_RECON_VAN_ALBADA)
        return "reconstruction must be FLITE_RECON_NONE or FLITE_RECON_VAN_ALBADA";
    if (c.reconstruction == FLITE_RECON_VAN_ALBADA && c.fluxType != 3)
        return "the Van Albada reconstruction acts on the Roe flux (fluxType 3)";
    int s = c.multigridScheme;
    if (!(s <= 0 || (s >= 1 && s <= 5) || s == 7)) return "multigridScheme not implemented";
    return nullptr;
}

}  // namespace

// The geometry arrays of level l (readGridComputationData and the set-up
// it performs): coefficients, side lengths, volumes, wall distances, normals
// (makeBoundaryNormals def_par:15394-15521), wall area (makeSurfaceArea
// :15523-15634, level 1), coordinates and their movement, restriction
// weights; on a moving mesh the GCL weights over physicalTimeStep (wgcl of
// makeRHS, combined as 1.5 GCL - 0.5 GCLprev on level 1 with timeScheme 2,
// def_par:816-818, 13858-13860) and the previous volumes.  Allocated and
// uploaded at creation (create), copied over the existing arrays otherwise.
void flite::put_geometry(flite_ctx &X, int l, const flite_level_desc &d, bool create) {
    LevelView &L = X.lv[l].v;
    const int N = L.N, E = L.E, B = L.B;
    auto put = [&](auto &field, const auto &h) {
        using T = typename std::decay_t<decltype(h)>::value_type;
        if (create) field = X.upload(h);
        else if (!h.empty())
            CK(cudaMemcpy(const_cast<T *>(field), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    };
    std::vector<double> wx(E), wy(E), wz(E), slen(E, 0.0);
    std::vector<EdgeW> ew(std::max(E, 1));
    for (int e = 0; e < E; ++e) {
        wx[e] = d.side_w[e]; wy[e] = d.side_w[(size_t)E + e]; wz[e] = d.side_w[2 * (size_t)E + e];
        if (d.side_len) slen[e] = d.side_len[e];
        ew[e] = EdgeW{wx[e], wy[e], wz[e], 0.0};
    }
    std::vector<int2> bedge(B);
    std::vector<double> bwx(B), bwy(B), bwz(B);
    for (int b = 0; b < B; ++b) {
        const int a = d.bnd_idx[b] - 1, q = d.bnd_idx[(size_t)B + b] - 1;
        if (a < 0 || a >= N || q < 0 || q >= N) throw std::runtime_error("boundary edge index out of range");
        bedge[b] = make_int2(a, q);
        bwx[b] = d.bnd_w[b]; bwy[b] = d.bnd_w[(size_t)B + b]; bwz[b] = d.bnd_w[2 * (size_t)B + b];
    }
    std::vector<double> nx(N, 0.0), ny(N, 0.0), nz(N, 0.0), wa(N, 0.0);
    for (int b = 0; b < B; ++b) {
        const int a = bedge[b].x, q = bedge[b].y;
        nx[a] = nx[a] - bwx[b]; ny[a] = ny[a] - bwy[b]; nz[a] = nz[a] - bwz[b];
        nx[q] = nx[q] - bwx[b]; ny[q] = ny[q] - bwy[b]; nz[q] = nz[q] - bwz[b];
    }
    for (int i = 0; i < L.Nb; ++i) {
        const double nrm = std::sqrt((nx[i] * nx[i] + ny[i] * ny[i]) + nz[i] * nz[i]);
        if (nrm > 1.0e-10) { nx[i] = nx[i] / nrm; ny[i] = ny[i] / nrm; nz[i] = nz[i] / nrm; }
        else { nx[i] = 0.0; ny[i] = 0.0; nz[i] = 0.0; }
    }
    if (l == 0)
        for (int b = 0; b < B; ++b) {
            const double ai = std::sqrt((bwx[b] * bwx[b] + bwy[b] * bwy[b]) + bwz[b] * bwz[b]);
            wa[bedge[b].x] = wa[bedge[b].x] + 4.0 * ai;
            wa[bedge[b].y] = wa[bedge[b].y] + 4.0 * ai;
        }
    std::vector<double> coords(3 * (size_t)N, 0.0), cm(3 * (size_t)N, 0.0);
    if (l == 0 && d.coords) std::memcpy(coords.data(), d.coords, 3 * (size_t)N * sizeof(double));
    if (l == 0 && d.coord_move) std::memcpy(cm.data(), d.coord_move, 3 * (size_t)N * sizeof(double));
    put(L.wx, wx); put(L.wy, wy); put(L.wz, wz); put(L.slen, slen); put(L.ew, ew);
    put(L.bwx, bwx); put(L.bwy, bwy); put(L.bwz, bwz);
    put(L.V, std::vector<double>(d.volume, d.volume + N));
    put(L.wdist, d.wall_dist ? std::vector<double>(d.wall_dist, d.wall_dist + N) : std::vector<double>(N, 0.0));
    put(L.nx, nx); put(L.ny, ny); put(L.nz, nz); put(L.wallArea, wa);
    put(L.cx, coords);
    L.cy = L.cx + N; L.cz = L.cx + 2 * (size_t)N;
    put(L.cmx, cm);
    L.cmy = L.cmx + N; L.cmz = L.cmx + 2 * (size_t)N;
    if (l > 0) {
        if (!d.rweight) throw std::runtime_error("coarse level without transfer operators");
        put(L.rweight, std::vector<double>(d.rweight, d.rweight + X.lv[l - 1].N));
    }
    if (X.c.flowType == 2) {
        if (!d.side_gcl || !d.bnd_gcl || (l == 0 && (!d.volume_prev || !d.volume_prev2)))
            throw std::invalid_argument("a moving mesh (flowType 2) needs side_gcl, bnd_gcl and, on level 1, "
                                        "volume_prev and volume_prev2");
        const bool comb = l == 0 && X.c.timeScheme == 2;
        const double dtp = X.c.physicalTimeStep;
        auto w = [&](double x, double xp) { return comb ? 1.5 * x - 0.5 * xp : x; };
        std::vector<double> gw(std::max(E, 1)), bgw(2 * (size_t)std::max(B, 1));
        for (int e = 0; e < E; ++e) gw[e] = w(d.side_gcl[e], d.side_gcl[(size_t)E + e]) / dtp;
        for (int b = 0; b < B; ++b) {
            const double g1 = w(d.bnd_gcl[b], d.bnd_gcl[2 * (size_t)B + b]);
            const double g2 = w(d.bnd_gcl[(size_t)B + b], d.bnd_gcl[3 * (size_t)B + b]);
            bgw[b] = X.c.boundaryTerm == 1 ? g1 / dtp : 4.0 * g1 / dtp;
            bgw[(size_t)B + b] = X.c.boundaryTerm == 1 ? g2 / dtp : 4.0 * g2 / dtp;
        }
        put(L.gclw, gw);
        put(L.bgclw, bgw);
        if (l == 0) {
            put(L.Vp, std::vector<double>(d.volume_prev, d.volume_prev + N));
            put(L.Vp2, std::vector<double>(d.volume_prev2, d.volume_prev2 + N));
        }
    }
}

extern "C" {

int flite_last_error(const flite_ctx *ctx, char *buf, size_t len) {
    if (!buf || !len) return FLITE_EINVAL;
    std::snprintf(buf, len, "%s", ctx ? ctx->err.c_str() : t_create_err.c_str());
    return FLITE_OK;
}

}  // extern "C"

// Create one solve's context.  With a donor context on the same mesh, the
// device copy of the mesh (edges, coefficients, incidence lists, transfer
// operators, geometry) is shared and only the solution state is allocated.
int flite::create_context(const flite_controls *c, int nlevels, const flite_level_desc *levels,
                          const flite_ctx *donor, flite_ctx **out) {
    t_create_err.clear();
    if (!c || !levels || !out || nlevels < 1) {
        t_create_err = "null argument or nlevels < 1";
        return FLITE_EINVAL;
    }
    *out = nullptr;
    if (const char *why = unsupported_reason(*c)) {
        t_create_err = why;
        return FLITE_EUNSUPPORTED;
    }
    auto ctx = std::make_unique<flite_ctx>();
    int rc = guarded(ctx.get(), [&]() -> int {
        flite_ctx &X = *ctx;
        X.c = *c;
        Params &P = X.P;
        P.gamma = c->gamma; P.gm1 = c->gamma - 1.0; P.hllcBeta0 = std::sqrt(P.gm1 / (2 * P.gamma));
        P.CFL = c->CFLNumber; P.maxInc = c->maxIncrementFactor;
        P.minRho = c->minimumDensity; P.Re = c->ReynoldsNumber; P.am = c->ReynoldsNumber > 0 ? 1.0 / c->ReynoldsNumber : 0.0;
        P.k2 = c->secondOrderDissipationFactor; P.k4 = c->fourthOrderDissipationFactor;
        P.cgdf = c->coarseGridDissipationFactor; P.pts = c->physicalTimeStep; P.Tinf = c->inflowTemperature;
        P.mach = c->MachNumber; P.mgBCRelax = c->multigridBCRelaxation; P.prolRelax = c->prolongationRelaxation;
        P.clip = c->HLLCClipping; P.Pr = c->PrandtlNumber;
        for (int i = 0; i < 12; ++i) P.inf[i] = c->inflowField[i];
        if (c->rungeKuttaStages == 5) {  // extension: no reference counterpart
            P.RK[0] = 0.25; P.RK[1] = 1. / 6.; P.RK[2] = 0.375; P.RK[3] = 0.5; P.RK[4] = 1.0;
        } else {
            P.RK[0] = 0.6; P.RK[1] = 0.6; P.RK[2] = 1.0;  // def_par:14240-14244
            P.RK[3] = P.RK[4] = 0.0;
        }
        P.nstage = c->rungeKuttaStages;
        P.matrixDiss = c->useMatrixDissipation != 0;
        P.harten = c->HartensCorrectionFactor;
        P.recon = c->reconstruction;
        P.fluxType = c->fluxType; P.hllcOrder = c->HLLCFluxOrder; P.autoClip = c->Automaticlipping;
        P.nsig = c->ReynoldsNumber < 1 ? 4 : 2;       // def_par:1592-1596
        P.isentropic = c->wallsAreIsentropic; P.viscous = c->ReynoldsNumber > 0.0;
        P.boundaryTerm = c->boundaryTerm; P.useDissW = c->useDissipationWeighting; P.ncfl = c->numberOfCFLIncrements;
        P.unsteady = c->flowType != 0; P.bdf2 = c->timeScheme == 2; P.dtp = c->physicalTimeStep;
        P.explicit_ = c->explicit_ != 0;
        P.addts = P.unsteady && !P.explicit_;
        P.sa = c->turbulenceModel == 1; P.nTurbGrids = c->numberOfTurbulenceGrids;
        P.turbCFL = c->turbulentCFLNumber; P.turbK = c->turbK; P.maxTurb = c->maxTurbulenceValue;
        P.turbProlRelax = c->turbProlongationRelaxation;
        P.oPrt = c->turbulentPrandtlNumber > 0 ? 1. / c->turbulentPrandtlNumber : 0.0;
        P.engines = 0;  // set from level 1 below
        P.eftype = c->engineFlowType; P.eoSteps = c->numberOfEORelaxationSteps;
        P.engRelax = c->engineBCRelaxation;
        for (int k = 0; k < 2; ++k) P.front[k] = c->enginesFrontMassFlow[k];
        for (int k = 0; k < 14; ++k) P.rear[k] = c->enginesRearParameters[k];

        int G = nlevels;
        if (c->numberOfGridsToUse > 0) G = std::min(G, c->numberOfGridsToUse);  // mg_par:1212-1214
        // the device numbering of the nodes (renumber.h); a context sharing
        // a donor's mesh shares its numbering
        Renumbered R;
        X.shares_mesh = donor != nullptr;
        if (donor) {
            X.renumbered = donor->renumbered;
            X.perm = donor->perm; X.iperm = donor->iperm;
            X.d_perm = donor->d_perm; X.d_iperm = donor->d_iperm;
        } else {
            renumber_levels(G, levels, default_node_order(), R);
            levels = R.desc.data();
            X.renumbered = !R.identity;
            X.perm = std::move(R.perm);
            X.iperm = std::move(R.iperm);
            if (X.renumbered)
                for (int l = 0; l < G; ++l) {
                    X.d_perm.push_back(X.upload(X.perm[l]));
                    X.d_iperm.push_back(X.upload(X.iperm[l]));
                }
        }
        CK(cudaStreamCreateWithFlags(&X.s, cudaStreamNonBlocking));
        // shared memory of the staged incidence-row gathers (above the
        // default 48 KB for the wider node fields)
        for (bool ahead : {true, false}) {
            CK(cudaFuncSetAttribute(ahead ? k_jst_flux_tiled<true, true> : k_jst_flux_tiled<true, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 13 * 8 * kTileStageMax));
            CK(cudaFuncSetAttribute(ahead ? k_visc_flux_tiled<true, true> : k_visc_flux_tiled<true, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 12 * 8 * kTileStageMax));
            CK(cudaFuncSetAttribute(ahead ? k_jst_lap_tiled<true, true> : k_jst_lap_tiled<true, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 6 * 8 * kTileStageMax));
        }
        CK(cudaMallocHost(&X.h_cycle, sizeof(int)));
        X.d_cycle = X.alloc<int>(1);
        X.d_cyc = X.alloc<int>(G);
        {
            std::vector<int> cyc0(G, 0);
            cyc0[0] = 1;  // setUpInitialField2 sets grid 1 (def_par:3992)
            CK(cudaMemcpy(X.d_cyc, cyc0.data(), G * sizeof(int), cudaMemcpyHostToDevice));
        }
        X.d_part = X.alloc<double>(kResidBlocks * 18);
        X.d_out = X.alloc<double>(32);
        // ivd%physicalTimeStep, which explicit time stepping overwrites
        X.d_ptsg = X.alloc<double>(1);
        CK(cudaMemcpy(X.d_ptsg, &c->physicalTimeStep, sizeof(double), cudaMemcpyHostToDevice));
        X.lv.resize(G);
        for (int l = 0; l < G; ++l) {
            const flite_level_desc &d = levels[l];
            DevLevel &D = X.lv[l];
            const int N = d.n_nodes, E = d.n_sides, B = d.n_bsides, Nb = d.n_bnodes;
            if (N <= 0 || E < 0 || B < 0 || Nb < 0 || Nb > N || d.n_normals < 0)
                throw std::runtime_error("bad level sizes");
            if (!d.side_idx || !d.side_w || !d.bnd_idx || !d.bnd_w || !d.node_reg || !d.volume ||
                (d.n_normals > 0 && !d.node_ind))
                throw std::runtime_error("missing level array");
            D.N = N; D.E = E; D.B = B; D.Nb = Nb;
            LevelView &L = D.v;
            L.N = N; L.E = E; L.B = B; L.Nb = Nb; L.grid = l + 1;
            if (donor) {
                if ((int)donor->lv.size() <= l || donor->lv[l].N != N || donor->lv[l].E != E || donor->lv[l].B != B)
                    throw std::runtime_error("mesh donor differs from the levels given");
                L = donor->lv[l].v;  // mesh arrays shared; state set below
                D.wall = donor->lv[l].wall;
                D.d_wall = donor->lv[l].d_wall;
                if (l == 0) P.engines = donor->P.engines;
            } else {
            // edges
            std::vector<int2> edge(E);
            for (int e = 0; e < E; ++e) {
                int a = d.side_idx[e] - 1, b = d.side_idx[(size_t)E + e] - 1;
                if (a < 0 || a >= N || b < 0 || b >= N || a == b) throw std::runtime_error("edge index out of range");
                edge[e] = make_int2(a, b);
            }
            std::vector<int2> bedge(B);
            std::vector<int> bind(B);
            for (int b = 0; b < B; ++b) {
                int a = d.bnd_idx[b] - 1, q = d.bnd_idx[(size_t)B + b] - 1;
                if (a < 0 || a >= N || q < 0 || q >= N) throw std::runtime_error("boundary edge index out of range");
                bedge[b] = make_int2(a, q);
                bind[b] = d.bnd_idx[2 * (size_t)B + b];
                if (l == 0 && bind[b] >= 5 && bind[b] <= 8) P.engines = 1;  // engine faces
            }
            // node -> incident edges in edge order
            std::vector<int> ip(N + 1, 0);
            for (int e = 0; e < E; ++e) { ip[edge[e].x + 1]++; ip[edge[e].y + 1]++; }
            for (int i = 0; i < N; ++i) ip[i + 1] += ip[i];
            std::vector<int2> inc(2 * (size_t)E);
            {
                std::vector<int> fill(ip.begin(), ip.end() - 1);
                for (int e = 0; e < E; ++e) {
                    inc[fill[edge[e].x]++] = make_int2(e, edge[e].y);
                    inc[fill[edge[e].y]++] = make_int2(~e, edge[e].x);
                }
            }
            std::vector<int> bp(N + 1, 0);
            for (int b = 0; b < B; ++b) { bp[bedge[b].x + 1]++; bp[bedge[b].y + 1]++; }
            for (int i = 0; i < N; ++i) bp[i + 1] += bp[i];
            std::vector<int> binc(2 * (size_t)B);
            {
                std::vector<int> fill(bp.begin(), bp.end() - 1);
                for (int b = 0; b < B; ++b) {
                    binc[fill[bedge[b].x]++] = 2 * b;
                    binc[fill[bedge[b].y]++] = 2 * b + 1;
                }
            }
            // connectivity (def_par:14262-14275)
            std::vector<double> conn(N, 0.0);
            for (int e = 0; e < E; ++e) { conn[edge[e].x] += 1.0; conn[edge[e].y] += 1.0; }
            // boundary classes from the indicator register
            std::vector<unsigned char> bc(N, BC_NONE);
            auto R = [&](int i) { return d.node_reg[i + 20]; };
            const int cls_of[10] = {0, BC_WALL, BC_SYM, BC_FAR3, BC_FAR4, 5, 6, 7, 8, BC_IWALL};
            for (int k = 1; k <= 9; ++k) {
                int st = R(-20 + 2 * (k - 1)), en = R(-19 + 2 * (k - 1));
                for (int ib = st; ib <= en; ++ib) {
                    if (ib < 1 || ib > d.n_normals) throw std::runtime_error("indicator register out of range");
                    int n = d.node_ind[ib - 1] - 1;
                    if (n < 0 || n >= N) throw std::runtime_error("indicator node out of range");
                    bc[n] = (unsigned char)cls_of[k];
                    if (l == 0 && k == 1) D.wall.push_back(n);
                }
            }
            // upload
            L.edge = X.upload(edge);
            L.bedge = X.upload(bedge); L.bind = X.upload(bind);
            L.inc_ptr = X.upload(ip); L.inc = X.upload(inc);
            L.binc_ptr = X.upload(bp); L.binc = X.upload(binc);
            L.conn = X.upload(conn);
            L.bc = X.upload(bc);
            L.eng = EngineView{};
            if (l == 0) {
                // engine inlet sides and engine nodes (level 1)
                const int ns = d.n_engine_sides;
                if (ns < 0 || (ns > 0 && (!d.engine_idx || !d.engine_w)))
                    throw std::runtime_error("bad engine inlet sides");
                std::vector<int2> es(ns);
                std::vector<int> ein(ns);
                for (int s = 0; s < ns; ++s) {
                    const int a = d.engine_idx[s] - 1, q = d.engine_idx[(size_t)ns + s] - 1;
                    const int in = d.engine_idx[2 * (size_t)ns + s];
                    if (a < 0 || a >= N || q < 0 || q >= N || in < 1 || in > 2)
                        throw std::runtime_error("engine inlet side out of range");
                    es[s] = make_int2(a, q);
                    ein[s] = in - 1;
                }
                std::vector<int> en;
                for (int i = 0; i < N; ++i)
                    if (bc[i] >= BC_EIN1 && bc[i] <= BC_EOUT2) en.push_back(i);
                if (ns > 0 || !en.empty()) P.engines = 1;
                if (P.engines) {
                    EngineView &G = L.eng;
                    G.nside = ns;
                    G.nnode = (int)en.size();
                    G.side = X.upload(es);
                    G.inlet = X.upload(ein);
                    G.wx = X.upload(std::vector<double>(d.engine_w, d.engine_w + ns));
                    G.wy = X.upload(std::vector<double>(d.engine_w + ns, d.engine_w + 2 * (size_t)ns));
                    G.wz = X.upload(std::vector<double>(d.engine_w + 2 * (size_t)ns, d.engine_w + 3 * (size_t)ns));
                    G.node = X.upload(en);
                }
            }
            put_geometry(X, l, d, true);
            L.inc32 = nullptr;
            L.tile = TileView{};
            if (X.fused()) {
                // staging of node blocks for the fused central gather
                std::vector<double> wx(d.side_w, d.side_w + E), wy(d.side_w + E, d.side_w + 2 * (size_t)E),
                    wz(d.side_w + 2 * (size_t)E, d.side_w + 3 * (size_t)E);
                TileHost T;
                build_tiles(N, ip, inc, wx, wy, wz, T);
                if (T.ntiles > 0) {
                    L.tile.ntiles = T.ntiles;
                    L.tile.stage_max = T.stage_max;
                    L.tile.halo_ptr = X.upload(T.halo_ptr);
                    L.tile.halo = X.upload(T.halo);
                    L.tile.row = X.upload(T.row);
                    L.tile.meta = X.upload(T.meta);
                    L.tile.nmeta = X.upload(T.nmeta);
                    L.tile.wx = X.upload(T.wx); L.tile.wy = X.upload(T.wy); L.tile.wz = X.upload(T.wz);
                }
            }
            if (l > 0) {
                const int nf = X.lv[l - 1].N;
                if (!d.parent || !d.rweight) throw std::runtime_error("coarse level without transfer operators");
                std::vector<int> par(nf);
                std::vector<int> cp(N + 1, 0);
                for (int f = 0; f < nf; ++f) {
                    par[f] = d.parent[f] - 1;
                    if (par[f] >= N) throw std::runtime_error("parent out of range");
                    if (par[f] >= 0) cp[par[f] + 1]++;
                }
                for (int i = 0; i < N; ++i) cp[i + 1] += cp[i];
                // children in the order of the caller's fine numbering, the
                // order of mapFineToCoarse's loop (def_par:12572-12679)
                std::vector<int> ch(std::max(cp[N], 1));
                std::vector<int> fill(cp.begin(), cp.end() - 1);
                for (int fo = 0; fo < nf; ++fo) {
                    const int f = X.iperm[l - 1][fo];
                    if (par[f] >= 0) ch[fill[par[f]]++] = f;
                }
                L.parent = X.upload(par);
                L.child_ptr = X.upload(cp); L.child = X.upload(ch);
            }
            if (!D.wall.empty()) D.d_wall = X.upload(D.wall);
            L.perm = X.renumbered ? X.d_perm[l] : nullptr;
            }  // mesh upload
            L.ptsg = X.d_ptsg;
            if (l > 0) L.eng = EngineView{};
            if (l == 0 && P.engines) {
                if (c->flowType == 2) {
                    X.err = "engine conditions on a moving mesh (flowType 2) are not supported";
                    return FLITE_EUNSUPPORTED;
                }
                // the engine pass's scratch belongs to this context
                L.eng.pbc = X.alloc<double>(N);
                CK(cudaMemset(L.eng.pbc, 0, (size_t)N * sizeof(double)));
                L.eng.f = X.alloc<EngineFactors>(1);
                CK(cudaMemset(L.eng.f, 0, sizeof(EngineFactors)));
            }
            // state
            const size_t nv = (size_t)X.nvar();
            L.u = X.alloc<double>(nv * N); L.uprev = X.alloc<double>(nv * N);
            L.rhs = X.alloc<double>(nv * N); L.src = X.alloc<double>(nv * N);
            L.diss = X.alloc<double>(5 * (size_t)N);
            L.p = X.alloc<double>(N); L.dt = X.alloc<double>(N); L.mu = X.alloc<double>(N);
            L.hvis = X.alloc<double>(N);
            for (double *a : {L.u, L.uprev, L.rhs, L.src})
                CK(cudaMemset(a, 0, nv * N * sizeof(double)));
            CK(cudaMemset(L.diss, 0, 5 * (size_t)N * sizeof(double)));
            if (c->turbulenceModel == 1) {
                L.turbDiff = X.alloc<double>(N); L.dtT = X.alloc<double>(N);
                L.vort = X.alloc<double>(N); L.divg = X.alloc<double>(N);
                L.sag = X.alloc<double>(3 * (size_t)N); L.sanh = X.alloc<double>(N);
                for (double *a : {L.turbDiff, L.dtT, L.vort, L.divg, L.sanh})
                    CK(cudaMemset(a, 0, (size_t)N * sizeof(double)));
            } else {
                L.turbDiff = L.dtT = L.vort = L.divg = L.sag = L.sanh = nullptr;
            }
            for (double *a : {L.p, L.dt, L.mu, L.hvis}) CK(cudaMemset(a, 0, (size_t)N * sizeof(double)));
            const bool hllc2 = c->fluxType == 4 && c->HLLCFluxOrder > 1 && l == 0;
            const bool muscl = c->reconstruction == FLITE_RECON_VAN_ALBADA && l == 0;
            const bool visc = c->ReynoldsNumber > 0.0;
            L.q = X.alloc<NodeRec>(N);
            CK(cudaMemset(L.q, 0, (size_t)N * sizeof(NodeRec)));
            // stress and heat flux (scheme 1), or the scaled gradients with mu
            // and k (scheme 2)
            L.tau = visc ? X.alloc<double>((c->viscosityScheme == 2 ? 14 : 9) * (size_t)N) : nullptr;
            L.prim = visc ? X.alloc<double>(4 * (size_t)N) : nullptr;
            L.lap = X.alloc<double>(5 * (size_t)N);
            L.sens = X.alloc<double>(N);
            L.lpw = c->dissipationScheme == 1 && l == 0 ? X.alloc<double>(N) : nullptr;
            L.vdt = X.alloc<double>(N);
            L.wstress = X.alloc<double>(3 * (size_t)N);
            CK(cudaMemset(L.wstress, 0, 3 * (size_t)N * sizeof(double)));
            L.grad = hllc2 ? X.alloc<double>(15 * (size_t)N) : nullptr;
            L.bnd = hllc2 ? X.alloc<double>(10 * (size_t)N) : nullptr;
            L.qp = muscl ? X.alloc<PrimRec>(N) : nullptr;
            L.gq = muscl ? X.alloc<GradRec>(N) : nullptr;
            // the edge buffer carries the upwind fluxes; the central flux is
            // computed inside the node gather
            L.flux = !X.fused() ? X.alloc<double>(5 * (size_t)std::max(E, 1)) : nullptr;
            if (c->precision == FLITE_MIXED) {
                L.ua = X.alloc<double>(5 * (size_t)N);
                L.ra = X.alloc<double>(5 * (size_t)N);
                L.pa = X.alloc<double>(N);
                L.a32 = X.alloc<float>(5 * (size_t)N);
                L.dq = X.alloc<DeltaRec>(N);
                // a zero anchor makes the increments the full FP32 fluxes
                // until the first FP64 evaluation
                for (double *a : {L.ua, L.ra}) CK(cudaMemset(a, 0, 5 * (size_t)N * sizeof(double)));
                CK(cudaMemset(L.pa, 0, (size_t)N * sizeof(double)));
                CK(cudaMemset(L.a32, 0, 5 * (size_t)N * sizeof(float)));
                if (!L.inc32) {
                    IncRec32 *d32 = X.alloc<IncRec32>(2 * (size_t)std::max(E, 1));
                    if (E > 0) k_make_inc32<<<(unsigned)((2 * (size_t)E + 255) / 256), 256>>>(L.inc, L.ew, 2 * E, d32);
                    CK(cudaGetLastError());
                    L.inc32 = d32;
                }
            } else {
                L.ua = L.ra = L.pa = nullptr;
                L.a32 = nullptr;
                L.dq = nullptr;
            }
            L.bflux = X.alloc<double>(10 * (size_t)std::max(B, 1));
            L.bgterm = c->flowType == 2 ? X.alloc<double>(10 * (size_t)std::max(B, 1)) : nullptr;
            L.uold = c->flowType != 0 ? X.alloc<double>(nv * N) : nullptr;
            L.uold2 = c->flowType != 0 && l == 0 ? X.alloc<double>(nv * N) : nullptr;
            L.cyc = X.d_cyc + l;
            L.nvar = X.nvar();
        }
        CK(cudaDeviceSynchronize());
        return FLITE_OK;
    });
    if (rc != FLITE_OK) {
        t_create_err = ctx->err;
        return rc;
    }
    *out = ctx.release();
    return FLITE_OK;
}

extern "C" {

int flite_create(const flite_controls *c, int nlevels, const flite_level_desc *levels, flite_ctx **out) {
    return flite::create_context(c, nlevels, levels, nullptr, out);
}

int flite_destroy(flite_ctx *ctx) {
    if (!ctx) return FLITE_EINVAL;
    cudaStreamSynchronize(ctx->s);
    delete ctx;
    return FLITE_OK;
}

static bool bad_level(flite_ctx *ctx, int level) { return !ctx || level < 1 || level > (int)ctx->lv.size(); }

int flite_set_state(flite_ctx *ctx, int level, const double *u) {
    if (bad_level(ctx, level) || !u) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->put_nodes(level - 1, ctx->V(level - 1).u, u, ctx->nvar());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_get_state(flite_ctx *ctx, int level, double *u) {
    if (bad_level(ctx, level) || !u) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->get_nodes(level - 1, u, ctx->V(level - 1).u, ctx->nvar());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_get_pressure(flite_ctx *ctx, int level, double *p) {
    if (bad_level(ctx, level) || !p) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->get_nodes(level - 1, p, ctx->V(level - 1).p, 1);
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_init_freestream(flite_ctx *ctx) {
    if (!ctx) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        LevelView &L = ctx->V(0);
        for (int k = 0; k < 5; ++k)
            k_fill<<<flite_ctx::blocks(L.N), kBlock, 0, ctx->s>>>(L.u + (size_t)k * L.N, L.N, ctx->c.inflowField[k]);
        // setUpInitialField2's freestream branch (def_par:3953-3963)
        if (ctx->c.ReynoldsNumber > 0.0)
            k_fill<<<flite_ctx::blocks(L.N), kBlock, 0, ctx->s>>>(L.mu, L.N, 1. / ctx->c.ReynoldsNumber);
        if (ctx->P.sa) k_fill<<<flite_ctx::blocks(L.N), kBlock, 0, ctx->s>>>(L.u + 5 * (size_t)L.N, L.N, 0.1);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_start(flite_ctx *ctx) {
    if (!ctx) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        // makePressureField + setBCsOnSolutionField on level 1 with
        // cycleNumber = 1 (def_par:3990-3994)
        X.pressure(0);
        X.set_cycle(1);
        k_set_int<<<1, 1, 0, X.s>>>(X.V(0).cyc, X.d_cycle);
        k_bc_solution<<<flite_ctx::blocks(X.V(0).N), kBlock, 0, X.s>>>(X.P, X.V(0));
        X.engine_pass(0, MODE_START);
        // an unsteady run starts with uold = uold2 = u (def_par:3594-3596)
        if (X.P.unsteady) {
            const size_t n5 = X.nvar() * (size_t)X.V(0).N;
            CK(cudaMemcpyAsync(X.V(0).uold, X.V(0).u, n5 * sizeof(double), cudaMemcpyDeviceToDevice, X.s));
            CK(cudaMemcpyAsync(X.V(0).uold2, X.V(0).u, n5 * sizeof(double), cudaMemcpyDeviceToDevice, X.s));
        }
        X.physical_step_start();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(X.s));
        return FLITE_OK;
    });
}

int flite_explicit_time_step(flite_ctx *ctx, double *dt) {
    if (!ctx || !dt) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        CK(cudaStreamSynchronize(ctx->s));
        CK(cudaMemcpy(dt, ctx->d_ptsg, sizeof(double), cudaMemcpyDeviceToHost));
        return FLITE_OK;
    });
}

int flite_next_physical_step(flite_ctx *ctx) {
    if (!ctx) return FLITE_EINVAL;
    if (!ctx->P.unsteady) return fail(ctx, FLITE_EINVAL, "not an unsteady run (flowType 0)");
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        // end of the step (mg_par:889-890): uold2 = uold, uold = u on level 1
        const size_t n5 = X.nvar() * (size_t)X.V(0).N;
        CK(cudaMemcpyAsync(X.V(0).uold2, X.V(0).uold, n5 * sizeof(double), cudaMemcpyDeviceToDevice, X.s));
        CK(cudaMemcpyAsync(X.V(0).uold, X.V(0).u, n5 * sizeof(double), cudaMemcpyDeviceToDevice, X.s));
        // head of the next one
        X.physical_step_start();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(X.s));
        return FLITE_OK;
    });
}

int flite_update_geometry(flite_ctx *ctx, int nlevels, const flite_level_desc *levels) {
    if (!ctx || !levels || nlevels < (int)ctx->lv.size()) return FLITE_EINVAL;
    if (ctx->c.flowType != 2) return fail(ctx, FLITE_EINVAL, "not a moving-mesh run (flowType 2)");
    if (ctx->shares_mesh) return fail(ctx, FLITE_EUNSUPPORTED, "the mesh is shared with other cases of a batch");
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        const int G = (int)X.lv.size();
        for (int l = 0; l < G; ++l)
            if (levels[l].n_nodes != X.lv[l].N || levels[l].n_sides != X.lv[l].E || levels[l].n_bsides != X.lv[l].B ||
                !levels[l].side_w || !levels[l].bnd_w || !levels[l].bnd_idx || !levels[l].volume)
                throw std::invalid_argument("the levels differ from those the context was created with");
        // the device numbering of flite_create
        Renumbered R;
        renumber_as(G, levels, X.perm, X.iperm, !X.renumbered, R);
        CK(cudaStreamSynchronize(X.s));
        for (int l = 0; l < G; ++l) put_geometry(X, l, R.desc[l], false);
        // the captured cycle holds no geometry value (only pointers), but the
        // head of the step runs again with the new restriction weights
        X.physical_step_start();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(X.s));
        return FLITE_OK;
    });
}

int flite_do_time_iterations(flite_ctx *ctx, int level, int nsteps, int calc_diss, int calc_turb, int cycle_no) {
    if (bad_level(ctx, level) || nsteps < 0) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->calcTurb = calc_turb != 0;
        ctx->set_cycle(cycle_no);
        ctx->doTimeIterations(level - 1, nsteps, calc_diss != 0);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_restrict(flite_ctx *ctx, int fine_level, int calc_turb) {
    if (bad_level(ctx, fine_level) || bad_level(ctx, fine_level + 1)) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->calcTurb = calc_turb != 0;
        ctx->restrictGrid(fine_level - 1);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_prolong(flite_ctx *ctx, int coarse_level) {
    if (bad_level(ctx, coarse_level) || coarse_level < 2) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->prolongateGrid(coarse_level - 1);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_map_fine_to_coarse(flite_ctx *ctx, int fine_level) {
    if (bad_level(ctx, fine_level) || bad_level(ctx, fine_level + 1)) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->mapFineToCoarse(fine_level - 1);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_cycle(flite_ctx *ctx, int cycle_no) {
    if (!ctx) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->select_cycle(cycle_no);
        ctx->ensure_graph();
        ctx->set_cycle(cycle_no);
        CK(cudaGraphLaunch(ctx->graph, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        return FLITE_OK;
    });
}

int flite_residuals(flite_ctx *ctx, double res[7], double maxres[7], int32_t maxind[7]) {
    if (!ctx || !res || !maxres || !maxind) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        const LevelView &L = X.c.multigridScheme > 0 ? X.V(0) : X.V((int)X.lv.size() - 1);
        k_resid_partial<<<kResidBlocks, 256, 0, X.s>>>(L, X.d_part, kResidBlocks);
        k_resid_final<<<1, 192, 0, X.s>>>(X.d_part, kResidBlocks, X.d_out);
        double h[18];
        CK(cudaMemcpyAsync(h, X.d_out, sizeof h, cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
        for (int k = 0; k < 7; ++k) { res[k] = 0.0; maxres[k] = 0.0; maxind[k] = 1; }
        bool finite = true;
        for (int k = 0; k < X.nvar(); ++k) {  // nres = 6 with SA (mg_par:1292-1293)
            res[k] = h[k];
            maxres[k] = h[6 + k];
            maxind[k] = (int32_t)h[12 + k] + 1;
            if (!std::isfinite(res[k])) finite = false;
        }
        if (!finite) return fail(ctx, FLITE_ENAN, "NaN in residual");
        return FLITE_OK;
    });
}

int flite_forces(flite_ctx *ctx, double out[9]) {
    if (!ctx || !out) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        DevLevel &D = X.lv[0];
        const double PI = 4.0 * std::atan(1.0);
        for (int k = 0; k < 9; ++k) out[k] = 0.0;
        if (D.wall.empty()) return FLITE_OK;
        const double aR = X.c.alpha * PI / 180., bR = X.c.beta * PI / 180.;
        const bool calc3 = X.c.forceCalcType == 3;
        // partials: calculateLiftAndDrag's 6 sums per block, then (type 3)
        // calculateLiftAndDrag3's 7 sums per block
        double *part1 = X.d_part, *part3 = X.d_part + 6 * kForceBlocks;
        k_forces<<<kForceBlocks, 256, 0, X.s>>>(X.P, D.v, D.d_wall, (int)D.wall.size(), aR, bR, X.c.groundplane,
                                               X.c.datum[0], X.c.datum[1], X.c.datum[2], part1);
        k_forces_final<<<1, 32, 0, X.s>>>(part1, kForceBlocks, 6, X.d_out);
        if (calc3) {
            k_forces3<<<kForceBlocks, 256, 0, X.s>>>(X.P, D.v, D.d_wall, (int)D.wall.size(), aR, bR,
                                                    X.c.groundplane, X.c.datum[0], X.c.datum[1], X.c.datum[2],
                                                    part3);
            k_forces_final<<<1, 32, 0, X.s>>>(part3, kForceBlocks, 7, X.d_out + 8);
        }
        double h[15];
        CK(cudaMemcpyAsync(h, X.d_out, sizeof h, cudaMemcpyDeviceToHost, X.s));
        CK(cudaStreamSynchronize(X.s));
        const double A = X.c.referenceArea;
        // lift, drag, latF, frictionDrag as coefficients; latM, longM as sums
        for (int k = 0; k < 6; ++k) out[k] = k < 4 ? 2.0 * h[k] / A : h[k];
        if (calc3) {
            // writeResiduals (mg_par:1364-1366): type 3 replaces lift, drag,
            // latF and latM and adds longMl, longMd and rollM; frictionDrag
            // and longM stay calculateLiftAndDrag's
            const double *g = h + 8;
            out[0] = 2.0 * g[0] / A;
            out[1] = 2.0 * g[1] / A;
            out[2] = 2.0 * g[2] / A;
            out[4] = 2.0 * g[3] / A;
            out[6] = 2.0 * g[4] / A;
            out[7] = 2.0 * g[5] / A;
            out[8] = 2.0 * g[6] / A;
        }
        return FLITE_OK;
    });
}

int flite_residual_fwd(flite_ctx *ctx, int level, const double *u, double *r) {
    if (bad_level(ctx, level) || !u || !r) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        const int l = level - 1;
        LevelView &L = X.V(l);
        if (X.mixed()) {
            // anchor at the level's current state, then the increments to u
            X.pressure(l);
            X.rhs_terms(l, true);
            X.node_update(l, MODE_RESID, 0, true);
        }
        X.put_nodes(l, L.u, u, 5);
        X.pressure(l);
        X.rhs_terms(l, false);
        X.node_update(l, MODE_RESID, 0, false);
        X.get_nodes(l, r, L.rhs, 5);
        CK(cudaStreamSynchronize(X.s));
        return FLITE_OK;
    });
}

int flite_time_cycles(flite_ctx *ctx, int cycle_no, int ncycles, double *ms) {
    if (!ctx || ncycles < 1 || !ms) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        X.select_cycle(cycle_no);
        X.ensure_graph();
        X.set_cycle(cycle_no);
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        CK(cudaEventRecord(a, X.s));
        for (int i = 0; i < ncycles; ++i) CK(cudaGraphLaunch(X.graph, X.s));
        CK(cudaEventRecord(b, X.s));
        CK(cudaEventSynchronize(b));
        float t = 0;
        CK(cudaEventElapsedTime(&t, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        *ms = t;
        return FLITE_OK;
    });
}

int flite_cycle_launches(flite_ctx *ctx, int64_t *n) {
    if (!ctx || !n) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        ctx->ensure_graph();
        *n = ctx->launches;
        return FLITE_OK;
    });
}

int flite_profile_level(flite_ctx *ctx, int level, int reps, double *edge_ms, double *node_ms) {
    if (bad_level(ctx, level) || reps < 1 || !edge_ms || !node_ms) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        const int l = level - 1;
        LevelView &L = X.V(l);
        cudaEvent_t ev[4];
        for (auto &e : ev) CK(cudaEventCreate(&e));
        double te = 0, tn = 0;
        for (int r = 0; r < reps; ++r) {
            X.pressure(l);
            CK(cudaEventRecord(ev[0], X.s));
            // the edge pass before the gather: the upwind-flux edge kernel,
            // the increment records of FLITE_MIXED, or nothing for the FP64
            // central flux (computed in the gather)
            if (X.mixed()) k_delta_state<<<X.nblk(L.N), X.nb, 0, X.s>>>(L);
            else if (!X.fused()) X.edge_flux_launch(L);
            CK(cudaEventRecord(ev[1], X.s));
            if (L.B > 0) k_bnd_flux<<<X.eblk(L.B), X.eb, 0, X.s>>>(X.P, L);
            CK(cudaEventRecord(ev[2], X.s));
            // the node kernel with the whole read set of an RK stage
            // (restrictGrid's fine increment: the result goes to rhs)
            X.launch_node_update(l, MODE_RFINE, 0, false);
            CK(cudaEventRecord(ev[3], X.s));
            CK(cudaEventSynchronize(ev[3]));
            float a = 0, b = 0;
            CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
            CK(cudaEventElapsedTime(&b, ev[2], ev[3]));
            te += a; tn += b;
        }
        for (auto &e : ev) cudaEventDestroy(e);
        *edge_ms = te / reps;
        *node_ms = tn / reps;
        return FLITE_OK;
    });
}

int flite_set_kernel_options(flite_ctx *ctx, int32_t edge_block, int32_t node_block, int32_t gather_unroll) {
    if (!ctx || edge_block < 32 || edge_block > 256 || node_block < 32 || node_block > 256 || edge_block % 32 ||
        node_block % 32 || (gather_unroll != 1 && gather_unroll != 2))
        return FLITE_EINVAL;
    ctx->drop_graph();
    ctx->eb = edge_block;
    ctx->nb = node_block;
    ctx->unroll = gather_unroll;
    return FLITE_OK;
}

int flite_set_tiled_gather(flite_ctx *ctx, int32_t level, int32_t on) {
    if (bad_level(ctx, level) || on < 0 || on > 4 || level > kMaxLevels) return FLITE_EINVAL;
    ctx->tiled_mode[level - 1] = on == 0 ? -1 : on;
    ctx->drop_graph();
    return FLITE_OK;
}

int flite_set_gather_fusion(flite_ctx *ctx, int32_t level, int32_t on) {
    if (bad_level(ctx, level) || (on != 0 && on != 1) || level > kMaxLevels) return FLITE_EINVAL;
    ctx->fuse_mode[level - 1] = on ? 1 : -1;
    ctx->drop_graph();
    return FLITE_OK;
}

int flite_set_gather_lanes(flite_ctx *ctx, int32_t level, int32_t lanes) {
    if (bad_level(ctx, level) || level > kMaxLevels) return FLITE_EINVAL;
    if (!(lanes == 0 || lanes == 1 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32)) return FLITE_EINVAL;
    ctx->drop_graph();
    ctx->lanes[level - 1] = lanes;
    return FLITE_OK;
}

int flite_profile_kernels(flite_ctx *ctx, int level, int reps, double *ms, int32_t nmax, int32_t *n) {
    if (bad_level(ctx, level) || reps < 1 || !ms || !n || nmax < 1) return FLITE_EINVAL;
    return guarded(ctx, [&] {
        flite_ctx &X = *ctx;
        const int l = level - 1;
        LevelView &L = X.V(l);
        // the kernels of one relaxation step of this level, in cycle order
        // (with shared walks the time step and Laplacian are timed as
        // ts_lap, the JST flux and viscous gradients as jflux_vgrad, and
        // their separate groups hold what is left of them)
        const int fz = X.step_fusion(l);
        const bool visc = X.c.ReynoldsNumber > 0;
        // each group launches its kernels and tells whether it had any (a
        // group without kernels reports 0 ms)
        std::vector<std::function<bool()>> k;
        k.push_back([&] { X.pressure(l); return true; });
        k.push_back([&] { if (!fz) X.timesteps(l); return !fz; });
        k.push_back([&] {
            if (!fz) X.dissipation(l);
            else if (fz == 1) X.jst_flux(l);
            return fz != 2;
        });
        k.push_back([&] { if (visc) k_visc_prim<<<X.nblk(L.N), X.nb, 0, X.s>>>(X.P, L); return visc; });
        k.push_back([&] { if (visc && fz != 2) X.visc_grad(l); return visc && fz != 2; });
        k.push_back([&] { if (visc) X.visc_flux(l); return visc; });
        k.push_back([&] { X.rhs_terms(l, true); return true; });
        k.push_back([&] { X.launch_node_update(l, MODE_RFINE, 0, true); return true; });
        k.push_back([&] { if (fz) k_ts_lap<<<X.nblk(L.N), X.nb, 0, X.s>>>(X.P, L); return fz != 0; });
        k.push_back([&] { if (fz == 2) k_jflux_vgrad<<<X.nblk(L.N), X.nb, 0, X.s>>>(X.P, L); return fz == 2; });
        const int m = std::min<int>((int)k.size(), nmax);
        std::vector<cudaEvent_t> ev(m + 1);
        for (auto &e : ev) CK(cudaEventCreate(&e));
        std::vector<double> acc(m, 0.0);
        std::vector<char> ran(m, 0);
        for (int r = 0; r < reps; ++r) {
            CK(cudaEventRecord(ev[0], X.s));
            for (int q = 0; q < m; ++q) {
                ran[q] = k[q]() ? 1 : 0;
                CK(cudaEventRecord(ev[q + 1], X.s));
            }
            CK(cudaEventSynchronize(ev[m]));
            for (int q = 0; q < m; ++q) {
                float t = 0;
                CK(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
                acc[q] += t;
            }
        }
        for (auto &e : ev) cudaEventDestroy(e);
        for (int q = 0; q < m; ++q) ms[q] = ran[q] ? acc[q] / reps : 0.0;
        *n = m;
        return FLITE_OK;
    });
}

}  // extern "C"

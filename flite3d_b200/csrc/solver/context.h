// Device context of one solve: the per-level device layout and the host
// orchestration that mirrors the reference's solver routines.  Shared by the
// single-solve ABI (flite_gpu.cu) and the batched one (batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "flite_gpu.h"
#include "kernels.h"

using namespace flite;

namespace flite {
// buffers of the steady adjoint (steady_adjoint.cu), made on its first call
struct SteadyAdjoint;
void destroy_steady_adjoint(SteadyAdjoint *a);
}  // namespace flite

namespace flite_detail {

struct cuda_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            throw cuda_error(std::string(#call) + ": " + cudaGetErrorString(_e));             \
    } while (0)

constexpr int kBlock = 256;
constexpr int kResidBlocks = 296;  // 2 x 148 SMs

struct DevLevel {
    int N = 0, E = 0, B = 0, Nb = 0;
    LevelView v{};
    std::vector<int> wall;  // level-1 wall nodes in register order (forces)
    int *d_wall = nullptr;
};

}  // namespace flite_detail

using namespace flite_detail;

#define FLITE_UNPAREN(...) __VA_ARGS__
// a launch of kernel template `kern` (its other template arguments `targs`,
// parenthesised with a trailing comma, or ()) for this context, or in group
// form for every case of its group: the same grid for each case, the case
// in blockIdx.y
#define FLITE_LAUNCH(kern, targs, grid, block, smem, ...)                                                     \
    do {                                                                                                       \
        if (group) launch_group(kern<FLITE_UNPAREN targs true>, dim3((grid), group), (block), (smem), __VA_ARGS__); \
        else kern<FLITE_UNPAREN targs false><<<(grid), (block), (smem), s>>>(__VA_ARGS__);                     \
    } while (0)

// a gather kernel template launched with the lanes per node of level l
#define FLITE_GATHER(kern, l, ...)                                                       \
    do {                                                                                 \
        switch (lanes_of(l)) {                                                           \
            case 4: FLITE_LAUNCH(kern, (4,), gblk(l, 4), nb, 0, __VA_ARGS__); break;     \
            case 8: FLITE_LAUNCH(kern, (8,), gblk(l, 8), nb, 0, __VA_ARGS__); break;     \
            case 16: FLITE_LAUNCH(kern, (16,), gblk(l, 16), nb, 0, __VA_ARGS__); break;  \
            case 32: FLITE_LAUNCH(kern, (32,), gblk(l, 32), nb, 0, __VA_ARGS__); break;  \
            default: FLITE_LAUNCH(kern, (1,), gblk(l, 1), nb, 0, __VA_ARGS__);           \
        }                                                                                \
    } while (0)

// a row-gather kernel template (STAGE, AHEAD) launched for mode m (1: staged,
// one ahead; 2: staged; 3: one ahead; 4: neither) over the level's blocks g,
// staging K fields per node
#define FLITE_ROWS(kern, K)                                                                    \
    do {                                                                                       \
        switch (m) {                                                                           \
            case 1: kern<true, true><<<g, kTile, tile_smem(l, m, K), s>>>(P, V(l)); break;      \
            case 2: kern<true, false><<<g, kTile, tile_smem(l, m, K), s>>>(P, V(l)); break;     \
            case 3: kern<false, true><<<g, kTile, 0, s>>>(P, V(l)); break;                      \
            default: kern<false, false><<<g, kTile, 0, s>>>(P, V(l));                           \
        }                                                                                      \
    } while (0)

struct flite_ctx {
    flite_controls c{};
    Params P{};
    std::vector<DevLevel> lv;
    std::vector<void *> allocs;
    cudaStream_t s = nullptr;
    int *d_cycle = nullptr;
    int *d_cyc = nullptr;  // per-level cycle numbers
    double *d_part = nullptr, *d_out = nullptr;
    double *d_ptsg = nullptr;  // ivd%physicalTimeStep (explicit time stepping)
    int *h_cycle = nullptr;  // pinned
    cudaGraphExec_t graph = nullptr;
    int64_t launches = 0;
    bool counting = false;
    // a case group (batch cases on one mesh, advanced together): while
    // `group` > 0 the cycle's launches run in group form for that many
    // cases, with every case's parameters and level views (gP, gV) in the
    // kernel's parameter bank.  Paths without a group form refuse it.
    int group = 0;
    CaseTab<Params> gP{};
    std::vector<CaseTab<LevelView>> gV;
    const CaseTab<Params> &to_group(const Params &) const { return gP; }
    const CaseTab<LevelView> &to_group(const LevelView &v) const {
        for (size_t l = 0; l < lv.size(); ++l)
            if (&lv[l].v == &v) return gV[l];
        throw std::runtime_error("a group launch argument is not one of the context's level views");
    }
    template <class T>
    const T &to_group(const T &x) const { return x; }
    template <class... KP, class... A>
    void launch_group(void (*k)(KP...), dim3 g, unsigned b, size_t sm, const A &...a) {
        k<<<g, b, sm, s>>>(to_group(a)...);
    }
    struct no_group_error : std::runtime_error {
        using std::runtime_error::runtime_error;
    };
    void no_group(const char *what) const {
        if (group) throw no_group_error(std::string(what) + " has no case-group form");
    }
    // threads per block of the edge kernels and of the node kernels (the
    // batch autotuner may change them; kernels with launch bounds take <= 256)
    int eb = kBlock, nb = kBlock;
    // incidences per load batch of the fused central gather (1 or 2)
    int unroll = 1;
    // calculateTurbulence of the cycle being run or captured (Spalart-
    // Allmaras: cycleNo <= numberOfTurbulenceSteps, mg_par:922-926), and the
    // value the instantiated graph was captured with
    bool calcTurb = true, graphTurb = true;
    int nvar() const { return c.turbulenceModel == 1 ? 6 : 5; }
    bool sa() const { return c.turbulenceModel == 1; }
    bool turb() const { return sa() && calcTurb; }
    // set calcTurb for cycle `cyc`, dropping a graph captured with the other value
    void select_cycle(int cyc) {
        const bool t = !sa() || cyc <= c.numberOfTurbulenceSteps;
        if (graph && graphTurb != t) drop_graph();
        calcTurb = t;
    }
    // adjoint buffers (allocated on the first flite_residual_vjp)
    double *adj_rbar = nullptr, *adj_ubar = nullptr, *adj_b = nullptr;
    size_t adj_n = 0;
    void vjp_kernels(int l);
    flite::SteadyAdjoint *sadj = nullptr;
    // node numbering of the device (renumber.h): perm[l][new] = the caller's
    // number, iperm[l] its inverse; d_perm/d_iperm on the device (shared with
    // contexts that share this mesh); a scratch array for the permutations
    bool renumbered = false;
    // the mesh arrays are another context's (a batch case on a shared mesh)
    bool shares_mesh = false;
    std::vector<std::vector<int>> perm, iperm;
    std::vector<int *> d_perm, d_iperm;
    double *d_io = nullptr;
    size_t io_n = 0;
    double *io_buffer(size_t n) {
        if (io_n < n) {
            if (d_io) CK(cudaFree(d_io));
            d_io = nullptr;
            io_n = 0;
            CK(cudaMalloc(&d_io, n * sizeof(double)));
            io_n = n;
        }
        return d_io;
    }
    // host [ncomp][N] in the caller's numbering -> device array in the
    // device's numbering (stream-ordered on s)
    void put_nodes(int l, double *dst, const double *host, int ncomp) {
        const size_t n = (size_t)lv[l].v.N * ncomp;
        if (!renumbered) {
            CK(cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, s));
            return;
        }
        double *t = io_buffer(n);
        CK(cudaMemcpyAsync(t, host, n * sizeof(double), cudaMemcpyHostToDevice, s));
        k_permute_nodes<<<blocks(n), kBlock, 0, s>>>(dst, t, d_perm[l], lv[l].v.N, ncomp);
        CK(cudaGetLastError());
    }
    // device array -> host [ncomp][N] in the caller's numbering (the copy is
    // stream-ordered on s: the caller synchronises before reading host)
    void get_nodes(int l, double *host, const double *src, int ncomp) {
        const size_t n = (size_t)lv[l].v.N * ncomp;
        if (!renumbered) {
            CK(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, s));
            return;
        }
        double *t = io_buffer(n);
        k_permute_nodes<<<blocks(n), kBlock, 0, s>>>(t, src, d_iperm[l], lv[l].v.N, ncomp);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(host, t, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    int adj_method = 1, adj_restart = 50;  // flite_set_adjoint_method (GMRES(50))
    std::string err;

    template <class T>
    T *alloc(size_t n) {
        void *p = nullptr;
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) throw cuda_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs.push_back(p);
        return (T *)p;
    }
    template <class T>
    T *upload(const std::vector<T> &h) {
        T *d = alloc<T>(h.size());
        if (!h.empty()) CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
        return d;
    }
    ~flite_ctx() {
        if (graph) cudaGraphExecDestroy(graph);
        if (adj_rbar) { cudaFree(adj_rbar); cudaFree(adj_ubar); cudaFree(adj_b); }
        if (sadj) flite::destroy_steady_adjoint(sadj);
        if (d_io) cudaFree(d_io);
        for (void *p : allocs) cudaFree(p);
        if (h_cycle) cudaFreeHost(h_cycle);
        if (s) cudaStreamDestroy(s);
    }

    static unsigned blocks(size_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }
    unsigned nblk(size_t n) const { return (unsigned)((n + nb - 1) / nb); }
    unsigned eblk(size_t n) const { return (unsigned)((n + eb - 1) / eb); }
    void counted() {
        if (counting) ++launches;
    }

    // ---- single-grid building blocks ------------------------------------
    LevelView &V(int l) { return lv[l].v; }
    // small levels gather with a warp per node (the lanes load and evaluate
    // the incidences in parallel, the sums keep their order): there a
    // thread per node leaves most SMs idle and each thread waits on a long
    // chain of dependent loads
    // lanes per node of each level's gathers (1, 4, 8, 16 or 32)
    int lanes[kMaxLevels] = {0};
    int lanes_of(int l) const {
        if (l < kMaxLevels && lanes[l] > 0) return lanes[l];
        return lv[l].v.N < kSmallLevelNodes ? 32 : 1;
    }
    unsigned gblk(int l, int g) const { return (unsigned)((g * (size_t)lv[l].v.N + nb - 1) / nb); }
    // levels whose gathers that walk the same incidence list share one walk
    // (k_ts_lap, k_jflux_vgrad) where a thread serves a node
    // (flite_set_gather_fusion: 1 on, the default; 0 off, held as -1)
    int fuse_mode[kMaxLevels] = {0};
    bool fuse_walks(int l) const {
        if (lanes_of(l) != 1 || tiled_other(l)) return false;
        return !(l < kMaxLevels && fuse_mode[l] < 0);
    }

    void pressure(int l) {
        counted();
        FLITE_LAUNCH(k_pressure, (), nblk(V(l).N), nb, 0, P, V(l));
    }
    // makeTimeSteps's ivd%physicalTimeStep under explicit time stepping
    // (unsteady runs read it; steady ones never do)
    void explicit_step(int l) {
        if (!(P.explicit_ && P.unsteady)) return;
        no_group("explicit time stepping");
        counted();
        k_min_dt_init<<<1, 1, 0, s>>>(V(l));
        counted();
        k_min_dt<<<(unsigned)std::min<size_t>((V(l).N + 255) / 256, kResidBlocks), 256, 0, s>>>(V(l));
    }
    void timesteps(int l) {
        timestep_kernels(l);
        explicit_step(l);
    }
    void timestep_kernels(int l) {
        counted();
        if (const int m = tiled_other(l)) {
            const int K = !P.viscous ? 0 : (P.sa ? 3 : 2);
            const unsigned g = V(l).tile.ntiles;
            const size_t sm = tile_smem(l, m, K);
#define FLITE_TS(KK)                                                                                      \
    switch (m) {                                                                                           \
        case 1: k_timestep_tiled<KK, true, true><<<g, kTile, sm, s>>>(P, V(l)); break;                     \
        case 2: k_timestep_tiled<KK, true, false><<<g, kTile, sm, s>>>(P, V(l)); break;                    \
        case 3: k_timestep_tiled<KK, false, true><<<g, kTile, 0, s>>>(P, V(l)); break;                     \
        default: k_timestep_tiled<KK, false, false><<<g, kTile, 0, s>>>(P, V(l));                          \
    }
            if (K == 0) { FLITE_TS(0) }
            else if (K == 2) { FLITE_TS(2) }
            else { FLITE_TS(3) }
#undef FLITE_TS
            return;
        }
        FLITE_GATHER(k_timestep, l, P, V(l));
    }
    // the incidence-row form of a level's other gathers (the mode of
    // flite_set_tiled_gather: 1, 2 staged, 3, 4 not), where a thread serves
    // a node and the rows exist; 0 otherwise
    int tiled_other(int l) const {
        if (group || lv[l].v.tile.ntiles <= 0 || lanes_of(l) != 1) return 0;
        const int m = l < kMaxLevels ? tiled_mode[l] : 0;
        return m < 0 ? 0 : m;
    }
    size_t tile_smem(int l, int m, int K) const {
        return m <= 2 ? (size_t)lv[l].v.tile.stage_max * K * sizeof(double) : 0;
    }
    void zero_diss(int l) {
        counted();
        FLITE_LAUNCH(k_case_zero, (), nblk(5 * (size_t)V(l).N), nb, 0, V(l), 0, 5 * (size_t)V(l).N);
    }
    // makeArtificialDissipation2 (def_par:11484-11993), scalar form
    void jst(int l) {
        if (!jst_gathers(l)) {
            zero_diss(l);
            return;
        }
        jst_lap(l);
        jst_flux(l);
    }
    // the JST kernels run (not the zero dissipation of jst)
    bool jst_gathers(int l) {
        return !((c.fluxType == 4 && V(l).grid == 1) ||
                 (c.fourthOrderDissipationFactor == 0 && c.secondOrderDissipationFactor == 0));
    }
    void jst_lap(int l) {
        const LevelView &L = V(l);
        const int m = tiled_other(l);
        const unsigned g = L.tile.ntiles;
        counted();
        if (m && !P.useDissW) {
            FLITE_ROWS(k_jst_lap_tiled, 6);
        } else {
            FLITE_GATHER(k_jst_lap, l, P, L);
        }
    }
    void jst_flux(int l) {
        const LevelView &L = V(l);
        const int m = tiled_other(l);
        const unsigned g = L.tile.ntiles;
        counted();
        if (P.matrixDiss) {
            no_group("the matrix dissipation");
            k_jst_flux_matrix<<<nblk(L.N), nb, 0, s>>>(P, L);
        }
        else if (m) {
            FLITE_ROWS(k_jst_flux_tiled, 13);
        } else {
            FLITE_GATHER(k_jst_flux, l, P, L);
        }
    }
    // the time step (ts), the JST dissipation (or its zero) and the viscous
    // terms of a level, in the order of singleIteration and restrictGrid.
    // Where a thread serves a node, the time step and the Laplacian share one
    // walk of the incidence lists (k_ts_lap), and so do the JST flux and the
    // viscous gradients (k_jflux_vgrad); the viscous primitives, which only
    // these gradients read, go before the JST flux.
    // the walks singleIteration's relaxation step shares on level l: 0 none;
    // 1 k_ts_lap; 2 k_ts_lap and k_jflux_vgrad
    int step_fusion(int l) {
        if ((c.dissipationScheme == 1 && V(l).grid == 1) || c.dissipationScheme == 3) return 0;
        if (!fuse_walks(l) || !jst_gathers(l)) return 0;
        return (c.ReynoldsNumber > 0.0 && !P.matrixDiss && c.viscosityScheme == 1) ? 2 : 1;
    }
    void ts_jst_viscous(int l, bool ts) {
        const bool visc = c.ReynoldsNumber > 0.0;
        if (!fuse_walks(l) || !jst_gathers(l)) {
            if (ts) timesteps(l);
            jst(l);
            viscous(l);
            return;
        }
        if (ts) {
            counted();
            FLITE_LAUNCH(k_ts_lap, (), nblk(V(l).N), nb, 0, P, V(l));
            explicit_step(l);
        } else {
            jst_lap(l);
        }
        if (visc) {
            counted();
            FLITE_LAUNCH(k_visc_prim, (), nblk(V(l).N), nb, 0, P, V(l));
        }
        if (visc && !P.matrixDiss && c.viscosityScheme == 1) {
            counted();
            FLITE_LAUNCH(k_jflux_vgrad, (), nblk(V(l).N), nb, 0, P, V(l));
        } else {
            jst_flux(l);
            if (visc) {
                counted();
                visc_grad(l);
            }
        }
        if (visc) {
            counted();
            visc_flux(l);
        }
    }
    void first_order_diss(int l) {
        no_group("dissipation scheme 3");
        counted();
        k_first_order_diss<1><<<nblk(V(l).N), nb, 0, s>>>(P, V(l));
    }
    // dissipation choice of singleIteration (def_par:1030-1036)
    void dissipation(int l) {
        if (c.dissipationScheme == 1 && V(l).grid == 1) lp_diss(l);
        else if (c.dissipationScheme == 3) first_order_diss(l);
        else jst(l);
    }
    // makeArtificialDissipation1 (def_par:10706-11482), level 1 only
    void lp_diss(int l) {
        no_group("dissipation scheme 1");
        counted();
        k_lp_sums<<<nblk(V(l).N), nb, 0, s>>>(P, V(l));
        counted();
        k_lp_flux<<<nblk(V(l).N), nb, 0, s>>>(P, V(l));
    }
    // makeViscosityTerm (def_par:5198-5893), subtracted from the dissipation
    void viscous(int l) {
        if (!(c.ReynoldsNumber > 0.0)) return;
        counted();
        FLITE_LAUNCH(k_visc_prim, (), nblk(V(l).N), nb, 0, P, V(l));
        counted();
        visc_grad(l);
        counted();
        visc_flux(l);
    }
    void visc_grad(int l) {
        if (c.viscosityScheme == 2) {  // makeViscosityTerm2 (def_par:5896-6807)
            FLITE_GATHER(k_visc2_grad, l, P, V(l));
            return;
        }
        if (const int m = tiled_other(l)) {
            const unsigned g = V(l).tile.ntiles;
            FLITE_ROWS(k_visc_grad_tiled, 4);
            return;
        }
        FLITE_GATHER(k_visc_grad, l, P, V(l));
    }
    void visc_flux(int l) {
        if (c.viscosityScheme == 2) {
            FLITE_GATHER(k_visc2_flux, l, P, V(l));
            return;
        }
        if (const int m = tiled_other(l)) {
            const unsigned g = V(l).tile.ntiles;
            FLITE_ROWS(k_visc_flux_tiled, 12);
            return;
        }
        FLITE_GATHER(k_visc_flux, l, P, V(l));
    }
    // ---- Spalart-Allmaras ----------------------------------------------
    void sa_timesteps(int l) {
        no_group("the Spalart-Allmaras model");
        counted();
        k_sa_timestep<<<nblk(V(l).N), nb, 0, s>>>(P, V(l));
    }
    void sa_diffusion(int l) {
        no_group("the Spalart-Allmaras model");
        counted();
        k_sa_grad<<<nblk(V(l).N), nb, 0, s>>>(P, V(l));
        counted();
        k_sa_diff<<<nblk(V(l).N), nb, 0, s>>>(P, V(l));
    }
    // the nu~ part of a stage or one-step update; before the mean-flow node
    // update, which overwrites the density the source term reads
    void sa_stage(int l, int mode, int stage) {
        if (!sa()) return;
        no_group("the Spalart-Allmaras model");
        if (turb()) {
            counted();
            k_sa_conv<<<nblk(V(l).N), nb, 0, s>>>(P, V(l), P.addts && mode == MODE_STAGE ? 1 : 0);
        }
        counted();
        k_sa_stage<<<nblk(V(l).N), nb, 0, s>>>(P, V(l), mode, stage, turb() ? 1 : 0);
    }
    // makeRHS up to the node gather (def_par:1587-1607 and the edge loops);
    // with FLITE_MIXED, `anchor` selects the FP64 evaluation that refreshes
    // the anchor state, otherwise the FP32 increments over it
    void rhs_terms(int l, bool anchor = true) {
        const LevelView &L = V(l);
        if (c.reconstruction == FLITE_RECON_VAN_ALBADA && L.grid == 1) {
            // the extension reconstructs from the Galerkin gradients, through
            // the primitive and gradient records
            no_group("the reconstruction extension");
            counted();
            k_prim_rec<<<nblk(L.N), nb, 0, s>>>(L);
            counted();
            k_gradient_rec<<<nblk(L.N), nb, 0, s>>>(L);
        } else if (c.fluxType == 4 && c.HLLCFluxOrder > 1 && L.grid == 1) {
            no_group("the HLLC order-2 gradients");
            counted();
            if (c.GradientMethod == 1) k_gradient<<<nblk(L.N), nb, 0, s>>>(P, L);
            else k_ls_gradient<<<nblk(L.N), nb, 0, s>>>(P, L);
            if (c.Automaticlipping == 1) {
                counted();
                k_minmax<<<nblk(L.N), nb, 0, s>>>(P, L);
            }
        }
        if (L.E > 0) {
            if (mixed() && !anchor) {
                // FP32 records of the increments over the anchor
                counted();
                FLITE_LAUNCH(k_delta_state, (), nblk(L.N), nb, 0, L);
            } else if (!fused()) {
                no_group("the upwind fluxes");
                counted();
                edge_flux_launch(L);
            }
        }
        if (L.B > 0) {
            counted();
            FLITE_LAUNCH(k_bnd_flux, (), eblk(L.B), eb, 0, P, L);
        }
    }
    bool mixed() const { return c.precision == FLITE_MIXED; }
    // the central flux (and FLITE_MIXED, which only takes it) is computed
    // inside the node gather; the upwind fluxes, and every flux of a moving
    // mesh (with its GCL term), go through the edge buffer
    bool fused() const { return c.fluxType == 1 && c.flowType != 2; }
    // the flux kernel instance of this run's fluxType (and HLLC order; the
    // reconstruction only acts on level 1, where coordinates exist)
    void edge_flux_launch(const LevelView &L) {
        const unsigned ng = eblk(L.E);
        switch (c.fluxType) {
            case 2: k_edge_flux<2, false><<<ng, eb, 0, s>>>(P, L); break;
            case 3:
                // the extension: MUSCL on level 1, upwind first order below
                if (P.recon == FLITE_RECON_VAN_ALBADA && L.grid == 1)  // 256 threads: its store staging
                    k_edge_flux_muscl<<<(unsigned)((L.E + 255) / 256), 256, 0, s>>>(P, L);
                else if (P.recon == FLITE_RECON_VAN_ALBADA) k_edge_flux<3, true><<<ng, eb, 0, s>>>(P, L);
                else k_edge_flux<3, false><<<ng, eb, 0, s>>>(P, L);
                break;
            case 4:
                if (c.HLLCFluxOrder > 1) k_edge_flux<4, true><<<ng, eb, 0, s>>>(P, L);
                else k_edge_flux<4, false><<<ng, eb, 0, s>>>(P, L);
                break;
            default: k_edge_flux<1, false><<<ng, eb, 0, s>>>(P, L);
        }
    }
    void node_update(int l, int mode, int stage, bool anchor = true) {
        counted();
        launch_node_update(l, mode, stage, anchor);
    }
    // the level-1 engine inlet terms after a node pass of `mode` (engine.cu)
    void engine_pass(int l, int mode) {
        const LevelView &L = V(l);
        if (l != 0 || !L.eng.f) return;
        no_group("the engine conditions");
        counted();
        k_engine_sums<<<1, kEngineLanes, 0, s>>>(P, L, mode);
        const bool all = P.eftype == 2;
        const int n = all ? L.N : L.eng.nnode;
        if (n > 0) {
            counted();
            k_engine_finish<<<nblk(n), nb, 0, s>>>(P, L, mode, all ? 1 : 0);
        }
    }
    void launch_node_update(int l, int mode, int stage, bool anchor) {
        switch (lanes_of(l)) {
            case 4: launch_node_update_u<4>(l, mode, stage, anchor); break;
            case 8: launch_node_update_u<8>(l, mode, stage, anchor); break;
            case 16: launch_node_update_u<16>(l, mode, stage, anchor); break;
            case 32: launch_node_update_u<32>(l, mode, stage, anchor); break;
            default: launch_node_update_u<1>(l, mode, stage, anchor);
        }
    }
    // levels whose gathers read the incidences through the rows of node
    // blocks (flite_set_tiled_gather: 0 off; 1, 2 staged in shared memory
    // with two or three blocks of 256 threads per SM; 3, 4 the same rows
    // without staging; tiled_mode holds -1 for 0 and 0 for the default, off)
    int tiled_mode[kMaxLevels] = {0};
    int tiled(int l) const {
        if (group || !(fused() && !mixed() && lv[l].v.tile.ntiles > 0)) return 0;
        const int m = l < kMaxLevels ? tiled_mode[l] : 0;
        return m < 0 ? 0 : m;
    }
    template <int U>
    void launch_node_update_u(int l, int mode, int stage, bool anchor) {
        const unsigned g = gblk(l, U);
        if (U == 1 && tiled(l)) {
            const TileView &T = V(l).tile;
            const size_t sm = (size_t)T.stage_max * sizeof(NodeRec);
            switch (tiled(l)) {
                case 2: k_node_update_tiled<true, false><<<T.ntiles, kTile, sm, s>>>(P, V(l), mode, stage); break;
                case 3: k_node_update_tiled<false, true><<<T.ntiles, kTile, 0, s>>>(P, V(l), mode, stage); break;
                case 4: k_node_update_tiled<false, false><<<T.ntiles, kTile, 0, s>>>(P, V(l), mode, stage); break;
                default: k_node_update_tiled<true, true><<<T.ntiles, kTile, sm, s>>>(P, V(l), mode, stage);
            }
            return;
        }
        if (mixed()) {
            if (anchor) FLITE_LAUNCH(k_node_update, (GATHER_ANCHOR, U,), g, nb, 0, P, V(l), mode, stage);
            else FLITE_LAUNCH(k_node_update, (GATHER_DELTA, U,), g, nb, 0, P, V(l), mode, stage);
        } else if (fused()) {
            if (unroll == 2 && U == 1) FLITE_LAUNCH(k_node_update, (GATHER_CENTRAL2, 1,), g, nb, 0, P, V(l), mode, stage);
            else if (U == 1 && !P.engines && !(P.unsteady && P.explicit_))
                FLITE_LAUNCH(k_node_update, (GATHER_LEAN, 1,), g, nb, 0, P, V(l), mode, stage);
            else FLITE_LAUNCH(k_node_update, (GATHER_CENTRAL, U,), g, nb, 0, P, V(l), mode, stage);
        } else {
            FLITE_LAUNCH(k_node_update, (GATHER_BUFFER, U,), g, nb, 0, P, V(l), mode, stage);
        }
    }

    // ---- singleIteration (def_par:1002-1181) -----------------------------
    void singleIteration(int l, bool calcDiss) {
        if (calcDiss) {
            pressure(l);  // p = |p| is the identity after the 0.1 floor
            if ((c.dissipationScheme == 1 && V(l).grid == 1) || c.dissipationScheme == 3) {
                timesteps(l);
                dissipation(l);
                viscous(l);
            } else {
                ts_jst_viscous(l, true);
            }
            if (turb()) {
                sa_timesteps(l);
                sa_diffusion(l);
            }
        }
        for (int st = 1; st <= P.nstage; ++st) {
            // u == uprev at stage 1: the FP64 evaluation there is the anchor
            // of the mixed-precision increments of the later stages.  The
            // pressure and flux records of stage 1 are those of the step's
            // own pressure pass when it ran (nothing has changed u since)
            if (st > 1 || !calcDiss) pressure(l);
            rhs_terms(l, st == 1);
            sa_stage(l, MODE_STAGE, st);
            node_update(l, MODE_STAGE, st, st == 1);
            engine_pass(l, MODE_STAGE);
        }
    }
    // ---- doTimeIterations (def_par:966-1000) -----------------------------
    void doTimeIterations(int l, int nsteps, bool calcDiss) {
        counted();
        FLITE_LAUNCH(k_case_cycle, (), 1, 1, 0, V(l), d_cycle);
        for (int i = 0; i < nsteps; ++i) {
            counted();
            FLITE_LAUNCH(k_case_save_u, (), nblk(nvar() * (size_t)V(l).N), nb, 0, V(l), nvar() * (size_t)V(l).N);
            singleIteration(l, calcDiss);
        }
    }
    // ---- restrictGrid (def_par:12141-12430) ------------------------------
    void restrictGrid(int fl) {
        const int cl = fl + 1;
        counted();
        FLITE_LAUNCH(k_restrict_state, (), nblk(V(cl).N), nb, 0, P, V(cl), V(fl));
        if (c.coarseGridDissipationScheme == 2) {
            ts_jst_viscous(cl, true);
        } else {
            timesteps(cl);
            if (c.coarseGridDissipationScheme == 3) first_order_diss(cl);
            viscous(cl);
        }
        rhs_terms(cl);
        if (turb()) {
            sa_timesteps(cl);
            sa_diffusion(cl);
        }
        sa_stage(cl, MODE_RCOARSE, 0);
        node_update(cl, MODE_RCOARSE, 0);
        pressure(fl);
        // the fine part uses scheme 1 on level 1 under dissipationScheme 1,
        // scheme 2 otherwise (def_par:12269-12273)
        if (c.dissipationScheme == 1 && V(fl).grid == 1) {
            lp_diss(fl);
            viscous(fl);
        } else {
            ts_jst_viscous(fl, false);
        }
        rhs_terms(fl, false);
        if (turb()) sa_diffusion(fl);  // the fine level keeps its turbulent time steps
        sa_stage(fl, MODE_RFINE, 0);
        node_update(fl, MODE_RFINE, 0, false);
        engine_pass(fl, MODE_RFINE);
        counted();
        FLITE_LAUNCH(k_restrict_incr, (), nblk(V(cl).N), nb, 0, P, V(cl), V(fl));
    }
    // ---- prolongateGrid (def_par:12432-12570) ----------------------------
    void prolongateGrid(int cl) {
        const int fl = cl - 1;
        counted();
        FLITE_LAUNCH(k_prolong_coarse, (), nblk(V(cl).N), nb, 0, P, V(cl), V(fl));
        counted();
        FLITE_LAUNCH(k_prolong_fine, (), nblk(V(fl).N), nb, 0, P, V(cl), V(fl));
        engine_pass(fl, MODE_PROLONG);
    }
    // the head of a physical time step (mg_par:586-602): laminar viscosity
    // 1/Re on every level, u (and in unsteady runs uold) restricted to every
    // coarse level
    void physical_step_start() {
        const double mu = c.ReynoldsNumber > 0.0 ? 1. / c.ReynoldsNumber : 0.0;
        for (size_t l = 0; l < lv.size(); ++l) {
            k_fill<<<blocks(V(l).N), kBlock, 0, s>>>(V(l).mu, V(l).N, mu);
            if (l > 0) {
                mapFineToCoarse((int)l - 1);
                if (P.unsteady)
                    k_restrict_arr<<<nblk(V(l).N), nb, 0, s>>>(V(l), V(l - 1), V(l - 1).uold, V(l).uold, nvar());
            }
        }
    }
    void mapFineToCoarse(int fl) {
        counted();
        FLITE_LAUNCH(k_restrict_u, (), nblk(V(fl + 1).N), nb, 0, V(fl + 1), V(fl));
    }
    // ---- oneCycle (mg_par:907-1196) --------------------------------------
    void oneCycle() {
        const int G = (int)lv.size();
        const int nr = c.numberOfRelaxationSteps;
        auto relax = [&](int j1, int steps, bool calc) { doTimeIterations(j1 - 1, steps, calc); };
        const int sch = c.multigridScheme;
        if (sch <= 0) {
            for (int i = 1; i <= G - 1; ++i) {
                counted();
                FLITE_LAUNCH(k_case_save_u, (), nblk(nvar() * (size_t)V(i - 1).N), nb, 0, V(i - 1),
                             nvar() * (size_t)V(i - 1).N);
                mapFineToCoarse(i - 1);
            }
            counted();
            FLITE_LAUNCH(k_case_zero, (), nblk(nvar() * (size_t)V(G - 1).N), nb, 0, V(G - 1), 1,
                         nvar() * (size_t)V(G - 1).N);
            relax(G, nr, true);
            for (int i = G; i >= 2; --i) {
                counted();
                FLITE_LAUNCH(k_inject_u, (), nblk(V(i - 2).N), nb, 0, V(i - 1), V(i - 2));
            }
        } else if (sch == 1) {
            for (int i = 1; i <= G - 1; ++i) {
                relax(i, nr, i == 1);
                restrictGrid(i - 1);
                mapFineToCoarse(i - 1);
            }
            relax(G, nr, G == 1);
            for (int i = G; i >= 2; --i) {
                prolongateGrid(i - 1);
                relax(i - 1, nr, (i - 1) == 1);
            }
        } else if (sch == 2 || sch == 5) {
            int nsw = G <= 2 ? 1 : 2 * G - 4;
            int fsl = 1;
            for (int i = 1; i <= nsw; ++i) {
                for (int j = fsl; j <= G - 1; ++j) {
                    relax(j, sch == 5 ? j : nr, j == fsl);
                    restrictGrid(j - 1);
                }
                relax(G, sch == 5 ? G : nr, G == 1);
                if (fsl == 1) fsl = G > 2 ? G - 1 : G;
                else if (i <= nsw / 2) fsl = fsl - 1;
                else fsl = fsl + 1;
                for (int j = G; j >= fsl + 1; --j) {
                    prolongateGrid(j - 1);
                    relax(j - 1, nr, (j - 1) == 1);
                }
            }
            for (int j = G; j >= 2; --j) {
                prolongateGrid(j - 1);
                relax(j - 1, nr, (j - 1) == 1);
            }
        } else if (sch == 3 || sch == 7) {
            int nsw = G == 1 ? 1 : G - 1;
            int fsl = 1;
            for (int i = 1; i <= nsw; ++i) {
                for (int j = fsl; j <= G - 1; ++j) {
                    relax(j, nr, j == fsl);
                    restrictGrid(j - 1);
                }
                relax(G, nr, G == 1);
                if (fsl == 1) fsl = G >= 2 ? G - 1 : G;
                else fsl = fsl - 1;
                for (int j = G; j >= fsl + 1; --j) {
                    prolongateGrid(j - 1);
                    if (sch == 7) relax(j - 1, nr, (j - 1) == 1);
                }
            }
        } else if (sch == 4) {
            int nsw = G == 1 ? 1 : G - 1;
            int fsl = 1;
            for (int i = 1; i <= nsw; ++i) {
                for (int j = fsl; j <= G - 1; ++j) {
                    relax(j, nr, j == fsl);
                    restrictGrid(j - 1);
                }
                relax(G, nr, G == 1);
                fsl = fsl + 1;
                for (int j = G; j >= fsl + 1; --j) {
                    prolongateGrid(j - 1);
                    relax(j - 1, nr, (j - 1) == 1);
                }
            }
            for (int j = G; j >= 2; --j) {
                prolongateGrid(j - 1);
                relax(j - 1, nr, (j - 1) == 1);
            }
        }
    }

    void set_cycle(int cyc) {
        *h_cycle = cyc;
        CK(cudaMemcpyAsync(d_cycle, h_cycle, sizeof(int), cudaMemcpyHostToDevice, s));
    }

    // capture one oneCycle into a graph (not instantiated)
    void capture_cycle(cudaGraph_t *g) {
        *g = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        launches = 0;
        counting = true;
        try {
            oneCycle();
        } catch (...) {
            counting = false;
            cudaStreamEndCapture(s, g);
            if (*g) cudaGraphDestroy(*g);
            *g = nullptr;
            throw;
        }
        counting = false;
        CK(cudaStreamEndCapture(s, g));
    }
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }

    void ensure_graph() {
        if (graph) return;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        launches = 0;
        counting = true;
        try {
            oneCycle();
        } catch (...) {
            counting = false;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        counting = false;
        CK(cudaStreamEndCapture(s, &g));
        graphTurb = calcTurb;
        cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }
};

namespace flite {
int create_context(const flite_controls *c, int nlevels, const flite_level_desc *levels, const flite_ctx *donor,
                   flite_ctx **out);
// the geometry arrays of level l from its descriptor (allocated when create)
void put_geometry(flite_ctx &X, int l, const flite_level_desc &d, bool create);
}  // namespace flite

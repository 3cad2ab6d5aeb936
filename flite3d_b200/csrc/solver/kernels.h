// Kernel declarations shared by the host orchestration.
#pragma once
#include "device.cuh"

namespace flite {

// node passes: an RK stage, restrictGrid's coarse and fine one-step updates,
// makeRHS alone; MODE_PROLONG and MODE_START name prolongateGrid's fine part
// and the start-up conditions for the engine pass that follows them
enum { MODE_STAGE = 0, MODE_RCOARSE = 1, MODE_RFINE = 2, MODE_RESID = 3, MODE_PROLONG = 4, MODE_START = 5 };

template <bool B = false>
__global__ void k_pressure(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_timestep(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_jst_lap(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_jst_flux(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U>
__global__ void k_first_order_diss(Params P, LevelView L);
template <bool B = false>
__global__ void k_visc_prim(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_visc_grad(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_visc_flux(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <bool B = false>
__global__ void k_ts_lap(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <bool B = false>
__global__ void k_jflux_vgrad(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_visc2_grad(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
template <int U, bool B = false>
__global__ void k_visc2_flux(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
__global__ void k_fill(double *a, size_t n, double v);
__global__ void k_gradient(Params P, LevelView L);
__global__ void k_jst_flux_matrix(Params P, LevelView L);
__global__ void k_lp_sums(Params P, LevelView L);
__global__ void k_lp_flux(Params P, LevelView L);
__global__ void k_prim_rec(LevelView L);
__global__ void k_gradient_rec(LevelView L);
__global__ void k_edge_flux_muscl(Params P, LevelView L);
__global__ void k_ls_gradient(Params P, LevelView L);
__global__ void k_minmax(Params P, LevelView L);
template <int FT, bool O2>
__global__ void k_edge_flux(Params P, LevelView L);
template <bool B = false>
__global__ void k_bnd_flux(CaseArg<B, Params> P, CaseArg<B, LevelView> L);
// GATHER_LEAN: GATHER_CENTRAL for runs without engine conditions and
// without explicit time stepping, whose node tail leaves those branches out
// (they cost the thread-per-node form its last free registers)
enum { GATHER_BUFFER = 0, GATHER_CENTRAL = 1, GATHER_ANCHOR = 2, GATHER_DELTA = 3, GATHER_CENTRAL2 = 4, GATHER_LEAN = 5 };
template <int PREC, int U, bool B = false>
__global__ void k_node_update(CaseArg<B, Params> P, CaseArg<B, LevelView> L, int mode, int stage);
// gathers: U lanes per node (1 = a thread per node); by default levels
// below kSmallLevelNodes nodes use a warp per node
constexpr int kSmallLevelNodes = 8192;
constexpr int kMaxLevels = 16;
template <bool B = false>
__global__ void k_delta_state(CaseArg<B, LevelView> L);
__global__ void k_sa_timestep(Params P, LevelView L);
__global__ void k_sa_grad(Params P, LevelView L);
__global__ void k_sa_diff(Params P, LevelView L);
__global__ void k_sa_conv(Params P, LevelView L, int td);
__global__ void k_sa_stage(Params P, LevelView L, int mode, int stage, int turb);
__global__ void k_make_inc32(const int2 *inc, const EdgeW *ew, int n, IncRec32 *o);
__global__ void k_copy(const double *a, double *b, size_t n);
template <bool B = false>
__global__ void k_restrict_u(CaseArg<B, LevelView> C, CaseArg<B, LevelView> F);
__global__ void k_restrict_arr(LevelView C, LevelView F, const double *fsrc, double *cdst, int ncomp);
template <bool B = false>
__global__ void k_restrict_state(CaseArg<B, Params> P, CaseArg<B, LevelView> C, CaseArg<B, LevelView> F);
template <bool B = false>
__global__ void k_restrict_incr(CaseArg<B, Params> P, CaseArg<B, LevelView> C, CaseArg<B, LevelView> F);
template <bool B = false>
__global__ void k_prolong_coarse(CaseArg<B, Params> P, CaseArg<B, LevelView> C, CaseArg<B, LevelView> F);
template <bool B = false>
__global__ void k_prolong_fine(CaseArg<B, Params> P, CaseArg<B, LevelView> C, CaseArg<B, LevelView> F);
template <bool B = false>
__global__ void k_inject_u(CaseArg<B, LevelView> C, CaseArg<B, LevelView> F);
__global__ void k_bc_solution(Params P, LevelView L);
// level-1 engine inlet terms after a node pass (engine.cu)
constexpr int kEngineLanes = 256;
__global__ void __launch_bounds__(kEngineLanes) k_engine_sums(Params P, LevelView L, int mode);
__global__ void k_engine_finish(Params P, LevelView L, int mode, int all);
__global__ void k_set_int(int *dst, const int *src);
// the explicit time step: the level's smallest local time step (256 threads a block)
__global__ void k_min_dt_init(LevelView L);
__global__ void k_min_dt(LevelView L);
// steps of the cycle on a level view (group form: every case of a group)
template <bool B = false>
__global__ void k_case_cycle(CaseArg<B, LevelView> L, const int *src);
template <bool B = false>
__global__ void k_case_save_u(CaseArg<B, LevelView> L, size_t n);
template <bool B = false>
__global__ void k_case_zero(CaseArg<B, LevelView> L, int which, size_t n);
__global__ void k_resid_partial(LevelView L, double *part, int nblk);
__global__ void k_resid_final(const double *part, int nblk, double *out);
__global__ void k_forces(Params P, LevelView L, const int *wall, int nwall, double alphaR, double betaR,
                         double ground, double d0, double d1, double d2, double *part);
template <bool STAGE, bool AHEAD>
__global__ void k_node_update_tiled(Params P, LevelView L, int mode, int stage);
template <int K, bool STAGE, bool AHEAD>
__global__ void k_timestep_tiled(Params P, LevelView L);
template <bool STAGE, bool AHEAD>
__global__ void k_jst_lap_tiled(Params P, LevelView L);
template <bool STAGE, bool AHEAD>
__global__ void k_jst_flux_tiled(Params P, LevelView L);
template <bool STAGE, bool AHEAD>
__global__ void k_visc_grad_tiled(Params P, LevelView L);
template <bool STAGE, bool AHEAD>
__global__ void k_visc_flux_tiled(Params P, LevelView L);
// dst[c*N + i] = src[c*N + map[i]] for c < ncomp (node arrays between the
// caller's numbering and the device's)
__global__ void k_permute_nodes(double *dst, const double *src, const int *map, int N, int ncomp);
__global__ void k_forces3(Params P, LevelView L, const int *wall, int nwall, double alphaR, double betaR,
                          double ground, double d0, double d1, double d2, double *part);
__global__ void k_forces_final(const double *part, int nblk, int nval, double *out);
constexpr int kForceBlocks = 64;
// transposed residual Jacobian at the state x (adjoint.cu)
__global__ void k_vjp_farfield(Params P, LevelView L, const double *x, const double *rbar, double *bvjp);
__global__ void k_vjp_node(Params P, LevelView L, const double *x, const double *rbar, const double *bvjp,
                           const double *pbar, double *ubar, int add);

}  // namespace flite

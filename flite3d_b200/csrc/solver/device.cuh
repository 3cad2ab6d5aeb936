// Device-side views of one grid level and the per-edge / per-node physics
// shared by the kernels.  Every function restates the reference expression
// it cites in the same operation order (the FP64 kernels are compiled with
// --fmad=false), so that the GPU result equals the CPU restatement bit for
// bit.
#pragma once
#include <cstdint>

namespace flite {

// Node boundary classes, from the indicator ranges of nodeIndicatorRegister
// (def_par:4033-4042): 1 wall, 2 symmetry, 3/4 far field, 5/6 engine inlets
// 1 and 2, 7/8 engine exhausts 1 and 2, 9 inviscid wall.
enum : unsigned char {
    BC_NONE = 0, BC_WALL = 1, BC_SYM = 2, BC_FAR3 = 3, BC_FAR4 = 4,
    BC_EIN1 = 5, BC_EIN2 = 6, BC_EOUT1 = 7, BC_EOUT2 = 8, BC_IWALL = 9
};
__device__ __forceinline__ bool is_engine(unsigned char c) { return c >= BC_EIN1 && c <= BC_EOUT2; }
__device__ __forceinline__ bool is_inlet(unsigned char c) { return c == BC_EIN1 || c == BC_EIN2; }
__device__ __forceinline__ bool is_exhaust(unsigned char c) { return c == BC_EOUT1 || c == BC_EOUT2; }

struct Params {
    double gamma, gm1, CFL, maxInc, minRho, Re, am, k2, k4, cgdf, pts, Tinf, mach;
    double mgBCRelax, prolRelax, clip, Pr;
    // the HLLC wave-speed factor sqrt((gamma-1)/(2 gamma)) (def_par:1826, 1953),
    // correctly rounded on the host like the per-edge expression it replaces
    double hllcBeta0;
    double inf[12];
    // stage coefficients: the reference's three (def_par:14240-14244) or the
    // five of the extension; recon selects the MUSCL reconstruction of the
    // Roe flux (an extension, level 1 only)
    double RK[5];
    int nstage, recon;
    // the matrix variant of the JST dissipation and Harten's correction
    int matrixDiss;
    double harten;
    int fluxType, hllcOrder, autoClip, nsig, isentropic, viscous, boundaryTerm, useDissW, ncfl;
    // unsteady dual time (flowType 1): the physical time step and the
    // second-order backward difference on level 1 (timeScheme 2); addts
    // whether the time differences are added (addTimeStep: unsteady and not
    // explicit, def_par:386-394); explicit time stepping, whose solve takes
    // one step for every node (LevelView::ptsg)
    int unsteady, bdf2, addts, explicit_;
    double dtp;
    // Spalart-Allmaras (turbulenceModel 1)
    int sa, nTurbGrids;
    double turbCFL, turbK, maxTurb, turbProlRelax, oPrt;
    // engine boundary conditions (def_par:4488-4918, 5084-5125): engines
    // set when the mesh has engine faces or nodes; the inlet mass flow kind
    // (engineFlowType), the cycles of the exhaust ramp, the increment
    // relaxation of the inlets, the mass flow targets and the exhaust states
    // (enginesRearParameters(7,2), column-major)
    int engines, eftype, eoSteps;
    double engRelax;
    double front[2];
    double rear[14];
};

// The level-1 engine inlet terms: the sides with their nodes, inlet (0|1)
// and coefficients; the engine nodes; the exhaust pressure each node pass
// leaves in pbc; and the factors and the go-ahead of the inlet scaling
// (scale = 0 where engineFlowType 2 jumps past it, def_par:4784-4801).
struct EngineFactors {
    double fac[2];
    int scale;
};
struct EngineView {
    int nside, nnode;
    const int2 *side;            // [nside]
    const int *inlet;            // [nside]
    const double *wx, *wy, *wz;  // [nside]
    const int *node;             // [nnode] the level's engine nodes
    double *pbc;                 // [N]
    EngineFactors *f;
};

// Records gathered by node kernels from a node's incident edges and from its
// neighbours.  Each is a multiple of 16 bytes and read with 16-byte loads,
// so that a neighbour costs one or two 32-byte sectors instead of one sector
// per component of an SoA array.
struct __align__(16) EdgeW {  // coefficients of an edge (32 B)
    double wx, wy, wz, pad;
};
struct __align__(16) IncRec32 {  // the same in FP32 (16 B); j is ~j when this
    float wx, wy, wz;            // node is the edge's second node
    int j;
};
struct __align__(16) NodeRec {  // what the central flux reads of a node (48 B)
    double ru, rv, rw, rinv, p, rh;  // momentum, 1/rho, pressure, E + p
};
struct __align__(16) DeltaRec {  // FP32 anchor primitives and increments (48 B)
    float ra, vax, vay, vaz, ha;  // anchor rho, velocity, E + p
    float dr, dmx, dmy, dmz, dE, dp, pad;  // u - ua and p - pa
};

// Level-1 records of the upwind extension (no reference counterpart): the
// primitives of the Galerkin gradient with the node's coordinates (64 B, two
// sectors), and that gradient, component-major (g[3c + a] = d q_c / d x_a,
// 128 B), so that an edge end costs six sectors instead of twenty-four SoA
// ones and no divisions.
struct __align__(16) PrimRec {
    double r, u, v, w, E, x, y, z;  // rho, (rho u)/rho, ..., rho E, coordinates
};
struct __align__(16) GradRec {
    double g[16];  // 15 used
};

// A level's mesh and state on the device.  Node-indexed arrays are SoA
// ([component][node]), like the reference's column-major u(N,nvar).
// Shared-memory staging of node blocks for the gathers with a thread per
// node: block t of kTile consecutive nodes and its halo (the other nodes its
// edges reach).  The incidences of the block are stored row by row: row k
// holds incidence k (in edge order) of each of the block's nodes, with the
// edge coefficients and the other node's staged slot (or, beyond the stage's
// capacity, its node number with kTileGlobal set); kTileSecond marks the
// node as the edge's second node.
constexpr int kTile = 256;
constexpr int kTileStageMax = 1024;  // records staged per block: 48 KB
constexpr unsigned kTileSecond = 0x80000000u, kTileGlobal = 0x40000000u, kTileIndexMask = 0x3fffffffu;
struct TileView {
    int ntiles;                   // 0: no staging data for this level
    int stage_max;                // staged records of the largest block (<= kTileStageMax)
    const int *halo_ptr, *halo;   // [ntiles+1], halo nodes of each block in increasing order
    const int *row;               // [ntiles+1] first incidence row of each block
    const unsigned *meta;         // [rows*kTile]
    const unsigned *nmeta;        // [rows*kTile] the same with every other node as a node number
    const double *wx, *wy, *wz;   // [rows*kTile]
};

struct LevelView {
    int N, E, B, Nb, grid;
    int nvar;                    // 5, or 6 with the Spalart-Allmaras nu~
    const int2 *edge;            // [E] (i1, i2), 0-based
    const double *wx, *wy, *wz;  // [E] edge coefficients
    const double *slen;          // [E]
    const int2 *bedge;           // [B]
    const int *bind;             // [B] face indicator
    const double *bwx, *bwy, *bwz;
    // node -> incident edges in edge order: (signed edge, other node); a
    // negative entry ~e marks the node as the second node of edge e
    const int *inc_ptr;
    const int2 *inc;
    const EdgeW *ew;             // [E] the edge coefficients as one record
    // node -> incident boundary edges in boundary-edge order: 2*b + side
    const int *binc_ptr;
    const int *binc;
    const double *V, *conn, *nx, *ny, *nz, *wallArea;
    const double *wdist;             // wall distance (zero where the mesh has none)
    const double *cx, *cy, *cz;      // level 1; zero on coarse levels
    const double *cmx, *cmy, *cmz;   // coordinateMovement (level 1)
    const unsigned char *bc;         // [N] boundary class
    // coarse levels: fine -> coarse parent map and the inverse (children in
    // increasing fine order)
    const int *parent;               // [N_fine]
    const double *rweight;           // [N_fine]
    const int *child_ptr;            // [N+1]
    const int *child;                // [N_fine]
    // state
    double *u, *uprev, *rhs, *src, *diss;  // [5][N]
    double *p, *dt, *mu;                   // [N]
    double *hvis;                          // [N]  viscous time-step term
    double *lap;                           // [5][N] undivided Laplacian
    double *sens;                          // [N]  pressure sensor
    double *lpw;                           // [N]  edge-factor sums of dissipation scheme 1 (level 1)
    double *tau;                           // [9][N] stress tensor + heat flux
    double *prim;                          // [4][N] u, v, w, T of the viscous term
    NodeRec *q;                            // [N] written with p by k_pressure (48 B: the level-1
                                           // records of the bench mesh fit the 126 MB L2)
    // Spalart-Allmaras: nu~ is component 6 of u, uprev, rhs, src ([6][N])
    double *turbDiff, *dtT, *vort, *divg;  // [N] diffusion, turbulent dt, |curl u|, div u
    double *sag;                           // [3][N] Galerkin gradient of nu~
    double *sanh;                          // [N] the cb2 term of the diffusion
    double *vdt;                           // [N]  V/dt of the dissipation
    double *wstress;                       // [3][N] wall stress (level 1)
    double *grad;                          // [15][N] (level 1, HLLC order 2)
    PrimRec *qp;                           // [N] (level 1, upwind extension)
    GradRec *gq;                           // [N] (level 1, upwind extension)
    double *bnd;                           // [10][N]
    double *flux;                          // [E][5] edge flux buffer
    // mixed precision (FLITE_MIXED): interior central fluxes as FP32
    // increments over an FP64 anchor state
    double *ua, *ra, *pa;                  // anchor u [5][N], its interior-edge residual [5][N], p [N]
    float *a32;                            // [5][N] anchor rho, u, v, w, E+p
    DeltaRec *dq;                          // [N] anchor primitives and increments
    const IncRec32 *inc32;                 // [2E] incidences in FP32
    double *bflux;                         // [B][10] boundary-edge contributions
    // moving meshes (flowType 2; NULL on a static mesh): per edge the GCL
    // weight over physicalTimeStep (wgcl of makeRHS), per boundary edge its
    // two nodes' (times 4 with boundaryTerm 2), the boundary edges' GCL
    // terms, and the volumes of the two previous steps (level 1)
    const double *gclw;                    // [E]
    const double *bgclw;                   // [2][B]
    double *bgterm;                        // [B][10]
    const double *Vp, *Vp2;                // [N]
    // unsteady dual time: the solution of the previous physical time steps
    // (uold2 on level 1 only)
    double *uold, *uold2;                  // [nvar][N]
    int *cyc;                              // cycle number of this level
    // the caller's number of each node (renumber.h); NULL when the device
    // numbering is the caller's
    const int *perm;                       // [N]
    TileView tile;                         // staging of node blocks (fluxType 1)
    EngineView eng;                        // level 1 of a mesh with engines; zero otherwise
    // ivd%physicalTimeStep under explicit time stepping: the smallest local
    // time step of the last makeTimeSteps on any level (one per context)
    double *ptsg;
};

// The view and parameters a kernel works on: its own arguments, or in the
// group form (B) those of case blockIdx.y of its group, whose every case has
// the same mesh and so the same grid.  The group form takes every case's
// arguments in its parameter bank (CaseTab; kernel parameters of up to
// 32,764 bytes: kGroupMax cases of a kernel with two level views), read
// with the case's index like the single form's own.  The kernels name their
// arguments P_ and L_ (C_, F_) and take P and L (C, F) from these.
constexpr int kGroupMax = 14;
template <class T>
struct CaseTab {
    T v[kGroupMax];
};
template <bool B, class T>
struct CaseArgT {
    using type = T;
};
template <class T>
struct CaseArgT<true, T> {
    using type = CaseTab<T>;
};
template <bool B, class T>
using CaseArg = typename CaseArgT<B, T>::type;
template <bool B, class T>
__device__ __forceinline__ const T &case_of(const CaseArg<B, T> &a) {
    if constexpr (B) return a.v[blockIdx.y];
    else return a;
}
#define FLITE_CASE_P(B, P, V) const Params &P = case_of<B, Params>(P##_)
#define FLITE_CASE_L(B, V) const LevelView &V = case_of<B, LevelView>(V##_)

__device__ __forceinline__ EdgeW load_edgew(const EdgeW *w, int e) {
    const double2 *p = reinterpret_cast<const double2 *>(w + e);
    const double2 a = __ldg(p), b = __ldg(p + 1);
    EdgeW o;
    o.wx = a.x; o.wy = a.y; o.wz = b.x; o.pad = b.y;
    return o;
}
__device__ __forceinline__ IncRec32 load_inc32(const IncRec32 *r, int k) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(r + k));
    IncRec32 o;
    o.wx = a.x; o.wy = a.y; o.wz = a.z; o.j = __float_as_int(a.w);
    return o;
}

// 16-byte loads (read-only path) and stores of the node records
template <class R, int K>
__device__ __forceinline__ R load_rec(const R *base, int j) {
    static_assert(sizeof(R) == 16 * K, "record size");
    const double2 *p = reinterpret_cast<const double2 *>(base + j);
    R o;
    double2 *d = reinterpret_cast<double2 *>(&o);
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = __ldg(p + k);
    return o;
}
template <class R, int K>
__device__ __forceinline__ void store_rec(R *base, int j, const R &o) {
    static_assert(sizeof(R) == 16 * K, "record size");
    double2 *p = reinterpret_cast<double2 *>(base + j);
    const double2 *d = reinterpret_cast<const double2 *>(&o);
#pragma unroll
    for (int k = 0; k < K; ++k) p[k] = d[k];
}
__device__ __forceinline__ NodeRec load_node(const NodeRec *q, int j) { return load_rec<NodeRec, 3>(q, j); }
__device__ __forceinline__ PrimRec load_prim(const PrimRec *q, int j) { return load_rec<PrimRec, 4>(q, j); }
// 1/rho and E + p are the operations the central flux performs per edge
// end, done once per node
__device__ __forceinline__ void store_node(NodeRec *q, int j, double r, double ru, double rv, double rw, double E,
                                           double p) {
    NodeRec o;
    o.ru = ru; o.rv = rv; o.rw = rw; o.rinv = 1. / r; o.p = p; o.rh = E + p;
    store_rec<NodeRec, 3>(q, j, o);
}

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

// makePressureField (def_par:13624-13627)
__device__ __forceinline__ double pressure(const Params &P, double r, double m1, double m2, double m3, double E) {
    double pp = P.gm1 * (E - 0.5 * ((m1 * m1 + m2 * m2) + m3 * m3) / r);
    return dmax(pp, 0.1);
}

// addTimeDifferences (def_par:1184-1241) of component c at node i: the
// second-order backward difference on level 1 with timeScheme 2 (with the
// previous volumes of a moving mesh; a static mesh's are the volumes), first
// order elsewhere
__device__ __forceinline__ double time_difference(const Params &P, const LevelView &L, int i, int c) {
    const size_t k = (size_t)c * L.N + i;
    const double Vi = L.V[i];
    if (L.grid == 1 && P.bdf2) {
        const double Vp = L.Vp ? L.Vp[i] : Vi, Vp2 = L.Vp2 ? L.Vp2[i] : Vi;
        return (((1.5 * Vi) * L.u[k] - (2.0 * Vp) * L.uold[k]) + (0.5 * Vp2) * L.uold2[k]) / P.dtp;
    }
    return Vi * (L.u[k] - L.uold[k]) / P.dtp;
}

// tangential projection used by every slip condition (def_par:4448-4451,
// 4480-4484, 4494-4499 and the increment forms :5028-5031, 5061-5066)
__device__ __forceinline__ void remove_normal(double *x, double n0, double n1, double n2, double scale) {
    double nv = (x[1] * n0 + x[2] * n1) + x[3] * n2;
    double s = scale * nv;
    x[1] = x[1] - s * n0;
    x[2] = x[2] - s * n1;
    x[3] = x[3] - s * n2;
}

// setBCsOnIncrementField (def_par:4978-5140); ENG = false leaves out the
// engine classes (for a level without engine nodes)
template <bool ENG = true>
__device__ __forceinline__ void bc_increment(const Params &P, unsigned char cls, double n0, double n1, double n2,
                                             double *r) {
    if (cls == BC_WALL) {
        if (P.viscous) {
            r[1] = 0.0; r[2] = 0.0; r[3] = 0.0;
            if (!P.isentropic) r[4] = 0.0;
        } else {
            remove_normal(r, n0, n1, n2, 1.0);
        }
    } else if (cls == BC_IWALL || cls == BC_SYM) {
        remove_normal(r, n0, n1, n2, 1.0);
    } else if (ENG && is_inlet(cls)) {  // engine inlets relaxed (def_par:5084-5099)
        for (int c = 0; c < 5; ++c) r[c] = P.engRelax * r[c];
    } else if (ENG && is_exhaust(cls)) {  // engine exhausts held (def_par:5100-5125)
        for (int c = 0; c < 5; ++c) r[c] = 0.0;
    }
}

// setBCsOnSolutionField for static walls (def_par:4364-4500)
__device__ __forceinline__ void bc_solution(const Params &P, unsigned char cls, double n0, double n1, double n2,
                                            double cm0, double cm1, double cm2, double relax, double *u) {
    if (cls == BC_WALL) {
        if (P.viscous) {
            u[1] = u[0] * cm0 / P.pts;
            u[2] = u[0] * cm1 / P.pts;
            u[3] = u[0] * cm2 / P.pts;
            if (!P.isentropic) u[4] = u[0] * P.Tinf / P.gamma;
        } else {
            remove_normal(u, n0, n1, n2, 1.0);
        }
    } else if (cls == BC_IWALL) {
        remove_normal(u, n0, n1, n2, relax);
        if (!P.isentropic) {
            double ke = (u[1] * u[1] + u[2] * u[2]) + u[3] * u[3];
            u[4] = u[0] * P.Tinf / P.gamma + 0.5 * ke / u[0];
        }
    } else if (cls == BC_SYM) {
        remove_normal(u, n0, n1, n2, 1.0);
    }
}

// setOuterBoundaryConditions (def_par:4018-4251)
__device__ __forceinline__ void bc_outer(const Params &P, unsigned char cls, double n0, double n1, double n2,
                                         double p, double *u) {
    if (cls != BC_FAR3 && cls != BC_FAR4) return;
    const double *inf = &P.inf[cls == BC_FAR3 ? 0 : 6];
    double iR = inf[0], iU1 = inf[1], iU2 = inf[2], iU3 = inf[3], iE = inf[4], iP = inf[5];
    double rho = u[0], U1 = u[1], U2 = u[2], U3 = u[3];
    double nvel = (iU1 * n0 + iU2 * n1) + iU3 * n2;
    if (nvel > 0.00) {
        u[0] = iR; u[1] = iU1 * iR; u[2] = iU2 * iR; u[3] = iU3 * iR;
        if (P.mach > 1.0) u[4] = iE * iR;
        else u[4] = p / P.gm1 + 0.5 * ((iU1 * iU1 + iU2 * iU2) + iU3 * iU3) * iR;
    } else {
        if (P.mach < 1.0) u[4] = iP / P.gm1 + 0.5 * ((U1 * U1 + U2 * U2) + U3 * U3) / rho;
    }
}

// relaxation parameter of the slip conditions (def_par:4389-4394)
__device__ __forceinline__ double relax_param(const Params &P, int cycle) {
    if (P.ncfl > 0) {
        double r = (double)(cycle - 1) / (double)P.ncfl;
        return dmin(r, 1.0);
    }
    return 1.0;
}

// ramp of the engine exhaust state (def_par:4490-4495)
__device__ __forceinline__ double eo_relax(const Params &P, int cycle) {
    if (P.eoSteps > 0) {
        double r = (double)(cycle - 1) / (double)P.eoSteps;
        return dmin(r, 1.0);
    }
    return 1.0;
}

// the state of an engine exhaust node (def_par:4497-4540); returns the
// exhaust pressure, which the reference stores into grp%p
__device__ __forceinline__ double bc_exhaust(const Params &P, unsigned char cls, double rp, double *u) {
    // the exhaust's column selected per component: constant offsets into
    // the parameters, which keeps them out of local memory
    const bool one = cls == BC_EOUT1;
#pragma unroll
    for (int c = 0; c < 5; ++c) u[c] = (1.0 - rp) * P.inf[c] + rp * (one ? P.rear[c] : P.rear[7 + c]);
    return (1.0 - rp) * P.inf[5] + rp * (one ? P.rear[5] : P.rear[12]);
}
// the exhaust nu~ (def_par:4507-4509, 4528-4530)
__device__ __forceinline__ double sa_exhaust(const Params &P, unsigned char cls, double rp) {
    return rp * (cls == BC_EOUT1 ? P.rear[6] : P.rear[13]);
}

// density update with the increment clip (def_par:1343-1366)
__device__ __forceinline__ void clipped_update(const Params &P, const double *up, const double *d, double *u) {
    double inc = d[0];
    if (fabs(inc / up[0]) < P.maxInc) {
        u[0] = up[0] - inc;
    } else {
        double sign = inc / fabs(inc);
        u[0] = up[0] - sign * P.maxInc * up[0];
    }
    u[1] = up[1] - d[1];
    u[2] = up[2] - d[2];
    u[3] = up[3] - d[3];
    u[4] = up[4] - d[4];
}

}  // namespace flite

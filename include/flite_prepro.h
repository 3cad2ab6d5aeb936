/*
 * flite_prepro.h -- C ABI of the host-side preprocessor and file formats.
 *
 * The reference builds its solver input with the separate gen3d executable
 * (PreProSource/*.f90) and reads/writes Fortran sequential-unformatted files.
 * This library restates gen3d's tetrahedral path (median-dual edge and
 * boundary coefficients, boundary-first numbering, node indicators, greedy
 * agglomeration) for synthetic meshes and reads/writes the reference's
 * formats: .sol (multi-level solver input), .rst (restart), .res (result),
 * .unk (merged result), plotreg.reg and .plt.  It also parses the NAMELIST
 * subset of the run deck (&InputVariables ivd%... = ...).
 */
#ifndef FLITE_PREPRO_H
#define FLITE_PREPRO_H

#include <stddef.h>
#include <stdint.h>
#include "flite_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fp_mesh fp_mesh;

/* Bump channel [0,3]x[0,1]x[0,1]: nx*ny*nz hexes, each split into 6 tets
 * (Kuhn split), lower wall lifted by bump_h*sin^2(pi(x-1)) on x in [1,2].
 * Surfaces: z=0 wall (indicator 1), z=1/y=0/y=1 symmetry (2), x=0/x=3 far
 * field (3).  nlevels agglomerated levels are built.                       */
int fp_bump_channel(int nx, int ny, int nz, double bump_h, int nlevels,
                    fp_mesh **out);
/* General tetrahedral input (the .plt content): coordinates [3][n] column
 * major, tets [4][ntet] 1-based, boundary triangles [3][ntri] 1-based and a
 * per-triangle boundary indicator (1..9).                                  */
int fp_from_tets(int32_t nnodes, const double *xyz, int32_t ntet,
                 const int32_t *tets, int32_t ntri, const int32_t *tris,
                 const int32_t *tri_ind, int nlevels, fp_mesh **out);
/* The same from hybrid elements (gen3d's element types): tetrahedra
 * [4][ntet], pyramids [5][npyr] (base 1-2-3-4, apex 5), prisms [6][npri]
 * (triangles 1-2-3 and 4-5-6, edge 1-4), hexahedra [8][nhex] (faces 1-2-3-4
 * and 5-6-7-8, edge 1-5), boundary triangles [3][ntri] and quadrilaterals
 * [4][nquad] with their indicators; any count may be 0 (the pointer then
 * NULL).  Median-dual coefficients and volumes per element type as
 * makeCalcDataForHex / Pri / Pyr / Tet (gen3d_grid.f90:902-2332, in that
 * order) and makeCalcDataForBoundary (gen3d_boundary.f90:511-766); the face
 * diagonals of hexahedra and prisms follow the lower boundary-first node
 * number.  Elements must be positively oriented (FLITE_EINVAL otherwise);
 * boundary faces are oriented here.                                          */
int fp_from_elements(int32_t nnodes, const double *xyz, int32_t ntet, const int32_t *tets, int32_t npyr,
                     const int32_t *pyrs, int32_t npri, const int32_t *pris, int32_t nhex, const int32_t *hexes,
                     int32_t ntri, const int32_t *tris, const int32_t *tri_ind, int32_t nquad, const int32_t *quads,
                     const int32_t *quad_ind, int nlevels, fp_mesh **out);
/* Extruded NACA0012 O-grid: ni points around the section, nj cells from the
 * wall (nlayer cells from first_cell growing by `growth`, then stretched to a
 * circular far field of radius `farfield` chords), nk cells over `span`.
 * Wall 1, span ends 2 (symmetry), far field 3.                              */
int fp_naca0012(int ni, int nj, int nk, double first_cell, double growth, int nlayer, double farfield,
                double span, int nlevels, fp_mesh **out);
int fp_free(fp_mesh *m);

int fp_num_levels(const fp_mesh *m);
/* Fill a level descriptor whose pointers stay valid while m lives.        */
int fp_level_desc(const fp_mesh *m, int level, flite_level_desc *out);
/* Coordinates of level 1 in original (generator) numbering are permuted to
 * boundary-first numbering; perm[new-1] = old (1-based), length N.         */
int fp_node_perm(const fp_mesh *m, int32_t *perm);
/* Max closure error |sum_j +-w_ij + 2 sum_b w_b| over nodes, relative to
 * max |w| (def_par:14430-14568), and total volume.                         */
int fp_check(const fp_mesh *m, int level, double *closure, double *volume);
/* Level-1 geometry of the mesh's own tetrahedra and boundary triangles at
 * node coordinates xyz [3][N] (boundary-first numbering; NULL = the mesh's
 * own): side_w [3][E], bnd_w [3][B] and volume [N] in the mesh's side and
 * boundary-side order (makeCalcDataForTet gen3d_grid.f90:2092-2332,
 * makeCalcDataForBoundary gen3d_boundary.f90:511-620).  The mesh's own
 * coordinates give its level-1 arrays back.  Meshes read from a .sol hold
 * no elements: FLITE_EINVAL.                                                */
int fp_geometry(const fp_mesh *m, const double *xyz, double *side_w, double *bnd_w, double *volume);
/* Transpose of the derivative of fp_geometry at xyz: xyz_bar [3][N] =
 * (d(side_w, bnd_w, volume)/d xyz)^T (side_w_bar, bnd_w_bar, volume_bar).   */
int fp_geometry_vjp(const fp_mesh *m, const double *xyz, const double *side_w_bar, const double *bnd_w_bar,
                    const double *volume_bar, double *xyz_bar);
/* Moving meshes (flowType 2): the arrays gen3d writes into a physical step's
 * .sol, from the node coordinates of the step, xyz, and of the two steps
 * before, xyz_prev and xyz_prev2 ([3][N], boundary-first numbering).  Level
 * 1 takes the coefficients, volumes at the three steps and GCL weights of the
 * mesh's own elements (makeCalcDataForTet / registerSideGCL gen3d_grid.f90:
 * 786-855, 2092-2332; makeCalcDataForBoundary / registerBoundarySideGCL
 * gen3d_boundary.f90:289-372, 511-766): per side the swept volume of its
 * dual faces between the step and the one before (GCL) and between the two
 * before (GCLprev), per boundary side those of each of its nodes; the side
 * lengths and coordinates of the step and the coordinate movement of the
 * solver's reader for time_scheme 1 or 2 (def_par:13896-13900).  Coarse
 * levels sum them through the agglomeration (restriction weights from the
 * new volumes).  The level descriptors then carry side_gcl, bnd_gcl,
 * volume_prev, volume_prev2 and coord_move.  Three equal coordinate sets give
 * the static arrays back bit for bit with zero GCL weights.  A mesh with
 * engine inlet sides returns FLITE_EUNSUPPORTED (the solver takes no engine
 * conditions on a moving mesh).                                            */
int fp_set_moving_geometry(fp_mesh *m, const double *xyz, const double *xyz_prev, const double *xyz_prev2,
                           int32_t time_scheme);
/* The level-1 coordinate movement of the solver's reader from the
 * coordinates of the step and of the two before (a mesh read from a moving
 * .sol holds all three).                                                    */
int fp_coordinate_movement(fp_mesh *m, int32_t time_scheme);
/* The discrete geometric conservation law of a moving level, as the solver
 * checks it (def_par:14590-14703): per node the sum over its sides of
 * +-2 GCL and over its boundary sides of 4 GCL (with time_scheme 2 the
 * weights 1.5 GCL - 0.5 GCLprev) against V - Vprev (time_scheme 1) or
 * 1.5 V - 2 Vprev + 0.5 Vprev2; *err is the largest difference, *scale the
 * largest volume change.                                                    */
int fp_gcl_check(const fp_mesh *m, int level, int32_t time_scheme, double *err, double *scale);

/* The canonical form of a mesh (a new mesh in *out): level-1 nodes keep
 * their numbers; the sides of every level run from the smaller to the larger
 * node (a reversed side's coefficients and GCL weights change sign) in
 * node-pair order, the boundary sides likewise (a reversed one's nodes swap
 * their GCL weights); coarse nodes are numbered boundary nodes first, each
 * class in the order of its smallest child; seeds become the smallest
 * level-1 descendant, wall-node numbers are dropped.  Values are moved, not
 * recomputed: two orderings of one mesh have equal canonical forms.         */
int fp_canonical(const fp_mesh *m, fp_mesh **out);

/* ---- multi-domain files (parallel runs of the reference) ----------------- */
/* gen3d's greedy partition of level 1 (greedyMeshPartition,
 * gen3d_struct.f90:890-1055): color [N] in 1..*ndomains_out (the front may
 * produce a different number of domains than asked for).                    */
int fp_partition(const fp_mesh *m, int32_t ndomains, int32_t *color, int32_t *ndomains_out);
/* The files of a parallel run: prefix.sol_1 .. prefix.sol_n, one per domain,
 * with every level's local numbering, ghost nodes, domain-crossing sides and
 * boundary sides, send/receive lists and the coarse levels' cross-domain
 * transfer lists, and plotreg (the owned nodes' global numbers), as
 * writeParallelComputationFiles writes them (gen3d_grid.f90:4082-5231).
 * color [N] gives level 1's domains (1-based; NULL: fp_partition's for
 * ndomains); coarse nodes go to the domain of most of their children
 * (mergeNodes :2843-2864).                                                   */
int fp_write_sol_domains(const fp_mesh *m, const char *prefix, const char *plotreg, int32_t ndomains,
                         const int32_t *color);
/* The mesh of a parallel run's files, merged into one: ghosts resolved
 * through the matching send and receive lists (level 1's global numbers from
 * plotreg, makeplot mgnsg3d_mg_par.F90:1599-1707), each side and node taken
 * once, in the canonical form of fp_canonical.                              */
int fp_read_sol_domains(const char *prefix, const char *plotreg, fp_mesh **out);

/* ---- files (Fortran sequential unformatted, 4-byte record markers) ---- */
int fp_write_sol(const fp_mesh *m, const char *path);
int fp_read_sol(const char *path, fp_mesh **out);
/* .rst: N; then rho, u, v, w, E/rho [, nu] column-major (def_par:3740-3873) */
int fp_write_rst(const char *path, int32_t n, int nvar, const double *prim);
int fp_read_rst(const char *path, int32_t n, int nvar, double *prim);
/* .res: N; rho, (u_j/rho) j=2..nvar from conserved u (def_par:15315-15346) */
int fp_write_res(const char *path, int32_t n, int nvar, const double *u);
/* .unk: N_global; u(N,nvar) as stored (mg_par:1698-1700)                   */
int fp_write_unk(const char *path, int32_t n, int nvar, const double *u);
int fp_read_unk(const char *path, int32_t n, int nvar, double *u);
/* plotreg.reg for one domain: (N,1); N; N x (local, global)              */
int fp_write_plotreg(const fp_mesh *m, const char *path);
/* makeplot (mg_par:1599-1707): merge the result files <res_prefix>1 ..
 * <res_prefix>nDomains (N_d, then nvar columns) through plotreg.reg's
 * (local, global) pairs into one .unk (N, then nvar columns).               */
int fp_makeplot(const char *plotreg, const char *res_prefix, int nvar, const char *unk);
/* .plt (tet form, gen3d_generator.f90:377-389): (nEl,N,nBF); iel(4,nEl);
 * x(3,N); iface(5,nBF) with column 5 the surface (indicator) number.       */
int fp_write_plt(const fp_mesh *m, const char *path);

/* ---- residual history (writeResiduals, mg_par:1449-1516) ------------- */
/* One .rsd line (format 504): iteration, log10(res1/initial_res) (-100/ln10
 * below 1e-15), lift, drag (E14.5), then F13.6 columns: latF, frictionDrag,
 * latM and longM with log10 res(2..nres), or with forceCalcType 3 longMl,
 * longMd, rollM.  forces as flite_forces fills them; res[nres].            */
int fp_rsd_line(char *buf, size_t len, int32_t iteration, double res1, double initial_res,
                const double forces[9], const double *res, int32_t nres, int32_t force_calc_type);
/* The same line written to path: a new file when first != 0, else appended
 * (the reference reopens the file for every cycle, mg_par:1481-1488).       */
int fp_append_rsd(const char *path, int32_t first, int32_t iteration, double res1, double initial_res,
                  const double forces[9], const double *res, int32_t nres, int32_t force_calc_type);
/* The screen line of a cycle (format 501): iteration, then res_k * scale
 * with (max |u - uprev|) for k = 1..5, then lift and drag; the reference's
 * scale is 1/(numberOfProcesses * N) (def_par:14258).                      */
int fp_cycle_line(char *buf, size_t len, int32_t iteration, const double res[5], const double maxres[5],
                  double scale, double lift, double drag);

/* ---- controls (the defaults and derivation of flite_gpu.h, host only) -- */
int fp_controls_default(flite_controls *c);
int fp_controls_derive(flite_controls *c);

/* ---- controls deck -------------------------------------------------- */
/* Parse "&InputVariables ivd%key = value, ... /" onto c (which should hold
 * defaults).  Unknown keys are listed (comma separated) in unknown.         */
int fp_read_inp(const char *path, flite_controls *c, char *unknown,
                size_t unknown_len);
int fp_parse_inp_text(const char *text, flite_controls *c, char *unknown,
                      size_t unknown_len);

#ifdef __cplusplus
}
#endif
#endif

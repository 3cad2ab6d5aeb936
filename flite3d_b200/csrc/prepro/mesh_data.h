// The preprocessor's mesh: one LevelData per multigrid level as the .sol
// records hold it, plus the level-1 elements (shared by the files of the
// preprocessor library; not part of the C ABI).
#pragma once
#include <cstdint>
#include <vector>

namespace fp_internal {

struct LevelData {
    int32_t N = 0, E = 0, B = 0, Nb = 0;
    std::vector<int32_t> side;   // [2][E] column-major, 1-based
    std::vector<double> sw;      // [3][E]
    std::vector<double> slen;    // [E]
    std::vector<int32_t> bside;  // [3][B] (i1, i2, indicator)
    std::vector<double> bw;      // [3][B]
    int32_t reg[21] = {0};       // nodeIndicatorRegister(-20:0)
    std::vector<int32_t> node_ind;
    std::vector<double> bnormal;  // [3][n_normals]
    std::vector<int32_t> bnd_indicator;  // [Nb] indicator per boundary node
    std::vector<double> vol, wdist;
    std::vector<int32_t> wnode;
    std::vector<double> xyz;      // [3][N] (level 1 only)
    std::vector<int32_t> seed;    // [N] (coarse levels)
    std::vector<int32_t> parent;  // [N_finer] (coarse levels)
    std::vector<double> rweight;  // [N_finer]
    // moving meshes (fp_set_moving_geometry): the GCL weights of the step and
    // of the step before, the volumes at the two previous steps and the
    // coordinate movement (level 1)
    std::vector<double> gcl;         // [2][E]
    std::vector<double> bgcl;        // [4][B] (GCL(1), GCL(2), GCLP(1), GCLP(2))
    std::vector<double> volp, volp2;  // [N]
    std::vector<double> cmove;       // [3][N]
    std::vector<double> xyzp, xyzp2;  // [3][N] coordinates at the two previous steps
    // coarse levels: the coarse side of each finer side (1-based, negative
    // where the finer side runs the other way, 0 inside an aggregate) and
    // the coarse boundary side of each finer one (negative where its two
    // nodes swap)
    std::vector<int32_t> side_of, bside_of;
    // engine inlet sides (makeEngineInflowData, gen3d_boundary.f90:768-920;
    // coarse levels agglomerateBoundary :1061-1099): (i1 <= i2, inlet 1|2)
    // and the coefficient vector of each, [3][n] column-major, 1-based
    std::vector<int32_t> eside;
    std::vector<double> ew;
    int32_t nes() const { return (int32_t)(eside.size() / 3); }
};

}  // namespace fp_internal

struct fp_mesh {
    std::vector<fp_internal::LevelData> lv;
    std::vector<int32_t> perm;    // new -> old, 1-based
    std::vector<int32_t> tets;    // [4][ntet] new numbering
    std::vector<int32_t> tris;    // [3][ntri]
    std::vector<int32_t> tri_ind;
    // the other elements and the quadrilateral boundary faces
    std::vector<int32_t> hexes;     // [8][nhex]
    std::vector<int32_t> prisms;    // [6][npri]
    std::vector<int32_t> pyramids;  // [5][npyr]
    std::vector<int32_t> quads;     // [4][nquad]
    std::vector<int32_t> quad_ind;
    bool hybrid() const { return !hexes.empty() || !prisms.empty() || !pyramids.empty() || !quads.empty(); }
};


namespace fp_internal {
// the indicator register, the node list per indicator and the boundary
// normals of a level from its boundary-node indicators and coefficients
void build_register(LevelData &L);
// the canonical form of fp_canonical, in place
void canonicalize(fp_mesh &M);
}  // namespace fp_internal

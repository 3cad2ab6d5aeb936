// Host-side preprocessor: synthetic tetrahedral meshes, a restatement of
// gen3d's tetrahedral path, greedy agglomeration, and the reference's
// Fortran-record file formats.  C ABI in include/flite_prepro.h.
//
// What follows the reference step by step (file:line in PreProSource/):
//   * median-dual edge coefficients and nodal volumes of a tetrahedron:
//     makeCalcDataForTet gen3d_grid.f90:2092-2332 with registerSideGCL
//     :786-855 (a static mesh's GCL terms vanish and are written as 0);
//   * edge registration with i1<i2 orientation and coefficient summation:
//     registerSideData gen3d_struct.f90:366-464;
//   * boundary-edge coefficients of a triangle: makeCalcDataForBoundary
//     gen3d_boundary.f90:511-620 with registerBoundarySideGCL :289-372;
//   * node-indicator priority (inviscid < symmetry < wall < far field <
//     engine): setBoundIndForViscousMesh gen3d_boundary.f90:1587-1640;
//   * the indicator register and the node list written per indicator:
//     writeParallelComputationFiles gen3d_grid.f90:4548-4580;
//   * coarse edges as sums of fine edges between different parents:
//     createSides gen3d_grid.f90:3558-3611; coarse boundary edges including
//     self-edges of one coarse node: agglomerateBoundary gen3d_boundary.f90:
//     922-1023; coarse node indicators by the same priority :1101-1121;
//   * coarse volumes as sums of fine volumes (mergeNodes gen3d_grid.f90:
//     2822-2829) and restriction weights V_f/V_c; coarse wall distances as
//     the children's volume-weighted mean (makeDistanceFieldsForCoarseMesh
//     :5823-5846);
//   * moving meshes: makeCalcDataForTet / registerSideGCL with three
//     coordinate levels and makeCalcDataForBoundary / registerBoundarySideGCL
//     (GCL weights of the step and of the step before), coarse levels by
//     summation (fp_set_moving_geometry).
// The seed selection of the agglomeration is this project's own greedy
// scheme (largest available connectivity first, boundary nodes before
// interior nodes, all free neighbours merged, single-node aggregates merged
// into their strongest neighbour); gen3d's mergeNodes (:2358-2902) follows
// the same priority idea with a different list-update order.
#include <algorithm>
#include <chrono>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "flite_prepro.h"
#include "fortran_io.hpp"

#include "mesh_data.h"

using fp_internal::LevelData;

namespace {

thread_local std::string g_err;

// optional section timing on stderr (FP_TIMING=1)
struct SectionTimer {
    const char *name;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    explicit SectionTimer(const char *n) : name(n) {}
    ~SectionTimer() {
        static const bool on = std::getenv("FP_TIMING") != nullptr;
        if (on)
            std::fprintf(stderr, "[prepro] %s %.3f s\n", name,
                         std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
};

// ---- open-addressing map from an ordered node pair to a slot -------------
class PairMap {
  public:
    explicit PairMap(size_t expect) {
        size_t cap = 16;
        while (cap < expect * 2 + 16) cap <<= 1;
        keys_.assign(cap, ~0ull);
        vals_.assign(cap, -1);
        mask_ = cap - 1;
    }
    // returns existing value or inserts `val` and returns -1
    int64_t find_or_insert(uint64_t key, int64_t val) {
        size_t h = hash(key) & mask_;
        while (true) {
            if (keys_[h] == key) return vals_[h];
            if (keys_[h] == ~0ull) {
                keys_[h] = key; vals_[h] = val;
                if (++count_ * 2 > keys_.size()) grow();
                return -1;
            }
            h = (h + 1) & mask_;
        }
    }
    int64_t find(uint64_t key) const {
        size_t h = hash(key) & mask_;
        while (true) {
            if (keys_[h] == key) return vals_[h];
            if (keys_[h] == ~0ull) return -1;
            h = (h + 1) & mask_;
        }
    }

  private:
    static size_t hash(uint64_t k) {
        k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33;
        k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
        return (size_t)k;
    }
    void grow() {
        std::vector<uint64_t> ok; std::vector<int64_t> ov;
        ok.swap(keys_); ov.swap(vals_);
        keys_.assign(ok.size() * 2, ~0ull); vals_.assign(ok.size() * 2, -1);
        mask_ = keys_.size() - 1; count_ = 0;
        for (size_t i = 0; i < ok.size(); ++i)
            if (ok[i] != ~0ull) find_or_insert(ok[i], ov[i]);
    }
    std::vector<uint64_t> keys_;
    std::vector<int64_t> vals_;
    size_t mask_ = 0, count_ = 0;
};

inline uint64_t pkey(int64_t a, int64_t b) { return ((uint64_t)a << 32) | (uint64_t)(uint32_t)b; }

// 3-vectors of a scalar type S: double, or the forward-mode numbers of the
// geometry derivative below
template <class S>
struct V3T { S x, y, z; };
using V3 = V3T<double>;
template <class S> inline V3T<S> operator+(V3T<S> a, V3T<S> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> inline V3T<S> operator-(V3T<S> a, V3T<S> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> inline V3T<S> scl(double s, V3T<S> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class S> inline V3T<S> div3(V3T<S> a) { return {a.x / 3., a.y / 3., a.z / 3.}; }

// Cxx(1,:) = 0.5*(r1(2)*r2(3)-r1(3)*r2(2)) ... (gen3d_grid.f90:799-804)
template <class S>
inline V3T<S> halfcross(V3T<S> r1, V3T<S> r2) {
    return {0.5 * (r1.y * r2.z - r1.z * r2.y), 0.5 * (r1.z * r2.x - r1.x * r2.z),
            0.5 * (r1.x * r2.y - r1.y * r2.x)};
}

// Forward-mode number with K derivative slots (the geometry derivative with
// respect to the K vertex coordinates of one element)
template <int K>
struct DN {
    double v = 0, d[K] = {};
};
template <int K> inline DN<K> operator+(const DN<K> &a, const DN<K> &b) {
    DN<K> o; o.v = a.v + b.v;
    for (int k = 0; k < K; ++k) o.d[k] = a.d[k] + b.d[k];
    return o;
}
template <int K> inline DN<K> operator-(const DN<K> &a, const DN<K> &b) {
    DN<K> o; o.v = a.v - b.v;
    for (int k = 0; k < K; ++k) o.d[k] = a.d[k] - b.d[k];
    return o;
}
template <int K> inline DN<K> operator*(const DN<K> &a, const DN<K> &b) {
    DN<K> o; o.v = a.v * b.v;
    for (int k = 0; k < K; ++k) o.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return o;
}
template <int K> inline DN<K> operator*(double s, const DN<K> &a) {
    DN<K> o; o.v = s * a.v;
    for (int k = 0; k < K; ++k) o.d[k] = s * a.d[k];
    return o;
}
template <int K> inline DN<K> operator/(const DN<K> &a, double s) {
    DN<K> o; o.v = a.v / s;
    for (int k = 0; k < K; ++k) o.d[k] = a.d[k] / s;
    return o;
}

// The six sides of a tetrahedron with positively oriented vertices x[0..3],
// in the order of makeCalcDataForTet (gen3d_grid.f90:2092-2332): the local
// vertex pair, half the side coefficient Cxx of its two dual-face triangles
// (registerSideGCL :786-855) and the nodal-volume share rv.Cxx/3 that both
// vertices receive.
template <class S>
struct TetSide { int a, b; V3T<S> coef; S nv; };
template <class S>
void tet_sides(const V3T<S> *x, TetSide<S> *out) {
    int n = 0;
    auto side = [&](int a, int b, V3T<S> r1, V3T<S> r2, V3T<S> r3, V3T<S> r4, V3T<S> rv) {
        V3T<S> c1 = halfcross(r1, r2), c2 = halfcross(r3, r4);
        V3T<S> cxx = c1 + c2;
        out[n].a = a; out[n].b = b;
        out[n].nv = (rv.x * cxx.x + rv.y * cxx.y + rv.z * cxx.z) / 3.;
        out[n].coef = scl(0.5, cxx);
        ++n;
    };
    const V3T<S> x1 = x[0], x2 = x[1], x3 = x[2], x4 = x[3];
    V3T<S> xmm = scl(0.25, x1 + x2 + x3 + x4);
    {   // node 1
        V3T<S> xm1 = scl(0.5, x1 + x2), xm2 = scl(0.5, x1 + x3), xm3 = scl(0.5, x1 + x4);
        V3T<S> xb1 = div3(x1 + x2 + x3), xb2 = div3(x1 + x2 + x4), xb3 = div3(x1 + x3 + x4);
        side(0, 1, xmm - xm1, xb2 - xm1, xb1 - xm1, xmm - xm1, xm1 - x1);
        side(0, 2, xmm - xm2, xb1 - xm2, xb3 - xm2, xmm - xm2, xm2 - x1);
        side(0, 3, xmm - xm3, xb3 - xm3, xb2 - xm3, xmm - xm3, xm3 - x1);
    }
    {   // node 2
        V3T<S> xm1 = scl(0.5, x2 + x3), xm2 = scl(0.5, x2 + x4);
        V3T<S> xb1 = div3(x1 + x2 + x3), xb2 = div3(x2 + x3 + x4), xb3 = div3(x1 + x2 + x4);
        side(1, 2, xmm - xm1, xb2 - xm1, xb1 - xm1, xmm - xm1, xm1 - x2);
        side(1, 3, xmm - xm2, xb3 - xm2, xb2 - xm2, xmm - xm2, xm2 - x2);
    }
    {   // node 3
        V3T<S> xm1 = scl(0.5, x3 + x4);
        V3T<S> xb1 = div3(x1 + x3 + x4), xb2 = div3(x2 + x3 + x4);
        side(2, 3, xmm - xm1, xb2 - xm1, xb1 - xm1, xmm - xm1, xm1 - x3);
    }
}

// The three sides of a boundary triangle oriented into the domain, in the
// order of makeCalcDataForBoundary (gen3d_boundary.f90:511-620): the local
// vertex pair and the quarter of Cxx that registerBoundarySideGCL (:289-372)
// adds to the boundary side.
template <class S>
struct TriSide { int a, b; V3T<S> coef; };
template <class S>
void tri_sides(const V3T<S> *x, TriSide<S> *out) {
    const V3T<S> x1 = x[0], x2 = x[1], x3 = x[2];
    V3T<S> xm = div3(x1 + x2 + x3);
    V3T<S> xb1 = scl(0.5, x1 + x2), xb2 = scl(0.5, x2 + x3), xb3 = scl(0.5, x3 + x1);
    out[0] = {0, 1, scl(0.25, halfcross(xm - x1, xb1 - x1))};
    out[1] = {0, 2, scl(0.25, halfcross(xb3 - x1, xm - x1))};
    out[2] = {1, 2, scl(0.25, halfcross(xm - x2, xb2 - x2))};
}

// ---- moving meshes: three time levels (t = 0 the step, 1 and 2 the two
// before), as makeCalcDataForTet and makeCalcDataForBoundary receive them
// from crp, crpPrev and crpPrev2 ---------------------------------------------
inline double dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
// the quarter cross product of the mixed time levels (Cyy of
// registerSideGCL, gen3d_grid.f90:806-818)
inline V3 qcross(V3 a, V3 b) {
    return {0.25 * (a.y * b.z - a.z * b.y), 0.25 * (a.z * b.x - a.x * b.z), 0.25 * (a.x * b.y - a.y * b.x)};
}
// the displacement of a dual-face triangle's centroid between levels k and
// k+1: ((p - p') + (q - q') + (r - r')) / 3 in the reference's order
inline V3 sweep(const V3 *p, const V3 *q, const V3 *r, int k) {
    return div3((((((p[k] - p[k + 1]) + q[k]) - q[k + 1]) + r[k]) - r[k + 1]));
}

// A tetrahedron side at three time levels (registerSideGCL, gen3d_grid.f90:
// 786-855): half the side coefficient at t = 0, the nodal-volume share at
// each level, and GCL(1) (levels 0-1) and GCL(2) (levels 1-2), the volumes
// its two dual-face triangles sweep
struct TetSideMoving { int a, b; V3 coef; double nv[3], gcl[2]; };
// side a-b of an element with the centroid xmm and the dual-face points xm
// (edge midpoint), P1 and P2 (face points) at the three levels: r1 = xmm -
// xm, r2 = P1 - xm, r3 = P2 - xm, r4 = xmm - xm, rv = xm - x_a
// (registerSideGCL gen3d_grid.f90:786-855 with the vectors every element
// routine builds)
void dual_side(int a, int b, const V3 *xa, const V3 *xmm, const V3 *xm, const V3 *P1, const V3 *P2,
               TetSideMoving &o) {
    V3 r1[3], r2[3], r3[3], r4[3], rv[3], c1[3], c2[3];
    for (int t = 0; t < 3; ++t) {
        r1[t] = xmm[t] - xm[t]; r2[t] = P1[t] - xm[t]; r3[t] = P2[t] - xm[t]; r4[t] = xmm[t] - xm[t];
        rv[t] = xm[t] - xa[t];
        c1[t] = halfcross(r1[t], r2[t]);
        c2[t] = halfcross(r3[t], r4[t]);
    }
    o.a = a; o.b = b;
    for (int t = 0; t < 3; ++t) {
        const V3 cxx = c1[t] + c2[t];
        o.nv[t] = (rv[t].x * cxx.x + rv[t].y * cxx.y + rv[t].z * cxx.z) / 3.;
        if (t == 0) o.coef = scl(0.5, cxx);
    }
    for (int k = 0; k < 2; ++k) {
        const V3 vr1 = sweep(xm, xmm, P1, k), vr2 = sweep(xm, P2, xmm, k);
        const V3 y1 = qcross(r1[k], r2[k + 1]) + qcross(r1[k + 1], r2[k]);
        const V3 y2 = qcross(r3[k], r4[k + 1]) + qcross(r3[k + 1], r4[k]);
        o.gcl[k] = (dot3((c1[k] + y1) + c1[k + 1], vr1) + dot3((c2[k] + y2) + c2[k + 1], vr2)) / 3.;
    }
}

// the element's points at the three levels: edge midpoints 0.5 (x_i + x_j),
// face centroids (x_i + x_j + x_k) / 3, and the quarter sum 0.5 of four
template <int NV>
struct ElemPts {
    const V3 (*x)[NV];
    void H(int i, int j, V3 *o) const { for (int t = 0; t < 3; ++t) o[t] = scl(0.5, x[t][i] + x[t][j]); }
    void T(int i, int j, int k, V3 *o) const {
        for (int t = 0; t < 3; ++t) o[t] = div3(x[t][i] + x[t][j] + x[t][k]);
    }
    void Q(int i, int j, int k, int l, V3 *o) const {
        for (int t = 0; t < 3; ++t) o[t] = scl(0.25, x[t][i] + x[t][j] + x[t][k] + x[t][l]);
    }
    // 0.5 (x_i + x_j) when q_c < q_d, else 0.5 (x_k + x_l): the diagonal of
    // a quadrilateral face through its lower-numbered corner of c, d
    void D(const int32_t *q, int c, int d, int i, int j, int k, int l, V3 *o) const {
        if (q[c] < q[d]) H(i, j, o);
        else H(k, l, o);
    }
    void vertex(int i, V3 *o) const { for (int t = 0; t < 3; ++t) o[t] = x[t][i]; }
};

void tet_sides_moving(const V3 (*x)[4], TetSideMoving *out) {
    V3 xmm[3];
    for (int t = 0; t < 3; ++t) xmm[t] = scl(0.25, x[t][0] + x[t][1] + x[t][2] + x[t][3]);
    int n = 0;
    auto side = [&](int a, int b, const V3 *xm, const V3 *P1, const V3 *P2) {
        V3 xa[3];
        for (int t = 0; t < 3; ++t) xa[t] = x[t][a];
        dual_side(a, b, xa, xmm, xm, P1, P2, out[n++]);
    };
    V3 xm1[3], xm2[3], xm3[3], xb1[3], xb2[3], xb3[3];
    const ElemPts<4> e{x};
    // node 1
    e.H(0, 1, xm1); e.H(0, 2, xm2); e.H(0, 3, xm3);
    e.T(0, 1, 2, xb1); e.T(0, 1, 3, xb2); e.T(0, 2, 3, xb3);
    side(0, 1, xm1, xb2, xb1);
    side(0, 2, xm2, xb1, xb3);
    side(0, 3, xm3, xb3, xb2);
    // node 2
    e.H(1, 2, xm1); e.H(1, 3, xm2);
    e.T(0, 1, 2, xb1); e.T(1, 2, 3, xb2); e.T(0, 1, 3, xb3);
    side(1, 2, xm1, xb2, xb1);
    side(1, 3, xm2, xb3, xb2);
    // node 3
    e.H(2, 3, xm1);
    e.T(0, 2, 3, xb1); e.T(1, 2, 3, xb2);
    side(2, 3, xm1, xb2, xb1);
}

// The twelve sides of a hexahedron (vertices 1-4 one face, 5-8 the
// opposite one, 1-5 an edge) from its four corners 1, 6, 3 and 8
// (makeCalcDataForHex gen3d_grid.f90:902-1379): the centroid of the inner
// tetrahedron 1-3-5-7 and, on each face, the diagonal through the corner
// of the lower node number q.
void hex_sides(const V3 (*x)[8], const int32_t *q, TetSideMoving *out) {
    const ElemPts<8> e{x};
    V3 xmm[3], xm1[3], xm2[3], xm3[3], xb1[3], xb2[3], xb3[3];
    e.Q(0, 2, 4, 6, xmm);
    int n = 0;
    auto corner = [&](int c, int n1, int n2, int n3) {
        V3 xa[3];
        e.vertex(c, xa);
        dual_side(c, n1, xa, xmm, xm1, xb2, xb1, out[n++]);
        dual_side(c, n2, xa, xmm, xm2, xb1, xb3, out[n++]);
        dual_side(c, n3, xa, xmm, xm3, xb3, xb2, out[n++]);
    };
    e.H(0, 1, xm1); e.H(0, 3, xm2); e.H(0, 4, xm3); e.H(0, 2, xb1);
    e.D(q, 4, 5, 1, 4, 0, 5, xb2); e.D(q, 4, 7, 3, 4, 0, 7, xb3);
    corner(0, 1, 3, 4);
    e.H(5, 4, xm1); e.H(5, 6, xm2); e.H(5, 1, xm3); e.H(4, 6, xb1);
    e.D(q, 4, 5, 1, 4, 0, 5, xb2); e.D(q, 5, 6, 5, 2, 1, 6, xb3);
    corner(5, 4, 6, 1);
    e.H(2, 3, xm1); e.H(1, 2, xm2); e.H(2, 6, xm3); e.H(0, 2, xb1);
    e.D(q, 6, 7, 6, 3, 2, 7, xb2); e.D(q, 5, 6, 5, 2, 1, 6, xb3);
    corner(2, 3, 1, 6);
    e.H(7, 6, xm1); e.H(7, 4, xm2); e.H(7, 3, xm3); e.H(4, 6, xb1);
    e.D(q, 6, 7, 6, 3, 2, 7, xb2); e.D(q, 4, 7, 4, 3, 0, 7, xb3);
    corner(7, 6, 4, 3);
}

// The nine sides of a prism (triangles 1-2-3 and 4-5-6, 1-4 an edge)
// (makeCalcDataForPri gen3d_grid.f90:1381-1777): the centroid of the three
// quadrilateral faces' diagonal midpoints, each diagonal through the corner
// of the lower node number q.
void pri_sides(const V3 (*x)[6], const int32_t *q, TetSideMoving *out) {
    const ElemPts<6> e{x};
    V3 xmm[3], xm1[3], xm2[3], xm3[3], xb1[3], xb2[3], xb3[3], xa[3];
    e.D(q, 3, 4, 3, 1, 0, 4, xb1); e.D(q, 3, 5, 3, 2, 0, 5, xb2); e.D(q, 4, 5, 4, 2, 1, 5, xb3);
    for (int t = 0; t < 3; ++t) xmm[t] = div3(xb1[t] + xb2[t] + xb3[t]);
    int n = 0;
    // node 1
    e.H(0, 1, xm1); e.H(0, 2, xm2); e.H(0, 3, xm3); e.T(0, 1, 2, xb1);
    e.D(q, 3, 4, 3, 1, 0, 4, xb2); e.D(q, 3, 5, 3, 2, 0, 5, xb3);
    e.vertex(0, xa);
    dual_side(0, 1, xa, xmm, xm1, xb2, xb1, out[n++]);
    dual_side(0, 2, xa, xmm, xm2, xb1, xb3, out[n++]);
    dual_side(0, 3, xa, xmm, xm3, xb3, xb2, out[n++]);
    // node 6
    e.H(5, 4, xm1); e.H(5, 3, xm2); e.H(5, 2, xm3); e.T(3, 4, 5, xb1);
    e.D(q, 4, 5, 4, 2, 1, 5, xb2); e.D(q, 3, 5, 3, 2, 0, 5, xb3);
    e.vertex(5, xa);
    dual_side(5, 4, xa, xmm, xm1, xb2, xb1, out[n++]);
    dual_side(5, 3, xa, xmm, xm2, xb1, xb3, out[n++]);
    dual_side(5, 2, xa, xmm, xm3, xb3, xb2, out[n++]);
    // node 2
    e.H(1, 4, xm1); e.H(1, 2, xm2); e.T(0, 1, 2, xb3);
    e.D(q, 4, 5, 4, 2, 1, 5, xb1); e.D(q, 3, 4, 3, 1, 0, 4, xb2);
    e.vertex(1, xa);
    dual_side(1, 2, xa, xmm, xm2, xb1, xb3, out[n++]);
    dual_side(1, 4, xa, xmm, xm1, xb2, xb1, out[n++]);
    // node 4
    e.H(3, 4, xm1); e.T(3, 4, 5, xb1);
    e.D(q, 3, 4, 3, 1, 0, 4, xb2);
    e.vertex(3, xa);
    dual_side(3, 4, xa, xmm, xm1, xb1, xb2, out[n++]);
}

// The eight sides of a pyramid (base 1-2-3-4, apex 5) (makeCalcDataForPyr
// gen3d_grid.f90:1779-2090): the point (2 (x1 + x3) + x5) / 5 and the base
// diagonal 1-3.
void pyr_sides(const V3 (*x)[5], TetSideMoving *out) {
    const ElemPts<5> e{x};
    V3 xmm[3], xm1[3], xm2[3], xm3[3], xb1[3], xb2[3], xb3[3], xa[3];
    for (int t = 0; t < 3; ++t) {
        const V3 s = x[t][0] + x[t][2];
        const V3 u = {2.0 * s.x + x[t][4].x, 2.0 * s.y + x[t][4].y, 2.0 * s.z + x[t][4].z};
        xmm[t] = {u.x / 5., u.y / 5., u.z / 5.};
    }
    int n = 0;
    // node 1
    e.H(0, 1, xm1); e.H(0, 3, xm2); e.H(0, 4, xm3); e.H(0, 2, xb1); e.T(0, 1, 4, xb2); e.T(0, 3, 4, xb3);
    e.vertex(0, xa);
    dual_side(0, 1, xa, xmm, xm1, xb2, xb1, out[n++]);
    dual_side(0, 3, xa, xmm, xm2, xb1, xb3, out[n++]);
    dual_side(0, 4, xa, xmm, xm3, xb3, xb2, out[n++]);
    // node 3
    e.H(1, 2, xm1); e.H(2, 3, xm2); e.H(2, 4, xm3); e.H(0, 2, xb1); e.T(1, 2, 4, xb2); e.T(2, 3, 4, xb3);
    e.vertex(2, xa);
    dual_side(2, 1, xa, xmm, xm1, xb1, xb2, out[n++]);
    dual_side(2, 3, xa, xmm, xm2, xb3, xb1, out[n++]);
    dual_side(2, 4, xa, xmm, xm3, xb2, xb3, out[n++]);
    // node 2
    e.H(1, 4, xm3); e.T(1, 2, 4, xb2); e.T(0, 1, 4, xb3);
    e.vertex(1, xa);
    dual_side(1, 4, xa, xmm, xm3, xb3, xb2, out[n++]);
    // node 4
    e.H(3, 4, xm3); e.T(0, 3, 4, xb2); e.T(2, 3, 4, xb3);
    e.vertex(3, xa);
    dual_side(3, 4, xa, xmm, xm3, xb3, xb2, out[n++]);
}

// A boundary triangle side at three time levels (registerBoundarySideGCL,
// gen3d_boundary.f90:289-372, from makeCalcDataForBoundary :511-620): the
// quarter coefficient at t = 0 and, for its first and second vertex,
// GCL(1 or 2, 1) (levels 0-1) and GCL(1 or 2, 2) (levels 1-2)
struct TriSideMoving { int a, b; V3 coef; double gcl[2][2]; };
// boundary side a-b of a face with the centre ctr (sweeps) through the edge
// midpoint mid: r1 = A - x_a, r2 = B - x_a
void bnd_side(int a, int b, const V3 *xa, const V3 *xb, const V3 *A, const V3 *B, const V3 *mid, const V3 *ctr,
              TriSideMoving &o) {
    V3 r1[3], r2[3], cxx[3];
    for (int t = 0; t < 3; ++t) {
        r1[t] = A[t] - xa[t]; r2[t] = B[t] - xa[t];
        cxx[t] = halfcross(r1[t], r2[t]);
    }
    o.a = a; o.b = b;
    o.coef = scl(0.25, cxx[0]);
    for (int k = 0; k < 2; ++k) {
        const V3 vr1 = sweep(xa, ctr, mid, k), vr2 = sweep(xb, ctr, mid, k);
        const V3 y = qcross(r1[k], r2[k + 1]) + qcross(r1[k + 1], r2[k]);
        const V3 s = (cxx[k] + y) + cxx[k + 1];
        o.gcl[0][k] = dot3(s, vr1) / 3.;
        o.gcl[1][k] = dot3(s, vr2) / 3.;
    }
}

void tri_sides_moving(const V3 (*x)[3], TriSideMoving *out) {
    V3 xm[3], xb[3][3], v[3][3];
    for (int t = 0; t < 3; ++t) {
        xm[t] = div3(x[t][0] + x[t][1] + x[t][2]);
        xb[0][t] = scl(0.5, x[t][0] + x[t][1]);
        xb[1][t] = scl(0.5, x[t][1] + x[t][2]);
        xb[2][t] = scl(0.5, x[t][2] + x[t][0]);
        for (int k = 0; k < 3; ++k) v[k][t] = x[t][k];
    }
    bnd_side(0, 1, v[0], v[1], xm, xb[0], xb[0], xm, out[0]);
    bnd_side(0, 2, v[0], v[2], xb[2], xm, xb[2], xm, out[1]);
    bnd_side(1, 2, v[1], v[2], xm, xb[1], xb[1], xm, out[2]);
}

// The four sides of a quadrilateral boundary face (makeCalcDataForBoundary
// gen3d_boundary.f90:627-766): the centre is the midpoint of the diagonal
// 1-3
void quad_sides_moving(const V3 (*x)[4], TriSideMoving *out) {
    V3 xm[3], xb[4][3], v[4][3];
    for (int t = 0; t < 3; ++t) {
        xm[t] = scl(0.5, x[t][0] + x[t][2]);
        xb[0][t] = scl(0.5, x[t][0] + x[t][1]);
        xb[1][t] = scl(0.5, x[t][1] + x[t][2]);
        xb[2][t] = scl(0.5, x[t][2] + x[t][3]);
        xb[3][t] = scl(0.5, x[t][0] + x[t][3]);
        for (int k = 0; k < 4; ++k) v[k][t] = x[t][k];
    }
    bnd_side(0, 1, v[0], v[1], xm, xb[0], xb[0], xm, out[0]);
    bnd_side(0, 3, v[0], v[3], xb[3], xm, xb[3], xm, out[1]);
    bnd_side(2, 1, v[2], v[1], xb[1], xm, xb[1], xm, out[2]);
    bnd_side(2, 3, v[2], v[3], xm, xb[2], xb[2], xm, out[3]);
}

// Indicator priority of setBoundIndForViscousMesh (gen3d_boundary.f90:
// 1607-1620) and agglomerateBoundary (:1101-1121).
inline int merge_indicator(int cur, int nw) {
    if (nw == cur) return cur;
    if (cur > 0) {
        if (cur == 9) return nw;
        if (cur == 2 && nw != 9) return nw;
        if (cur == 1 && nw > 2) return nw;
        if (cur <= 4 && nw > 4) return nw;
        return cur;
    }
    return nw;
}

// Register and node list from per-boundary-node indicators (gen3d_grid.f90:
// 4548-4580): counts at -21+2k, then running (start, end) pairs.


// k-d tree over a point subset for nearest-point queries
class KdTree {
  public:
    template <class Get>
    KdTree(const std::vector<int32_t> &ids, Get get) : id_(ids) {
        pt_.resize(id_.size());
        for (size_t i = 0; i < id_.size(); ++i) pt_[i] = get(id_[i]);
        build(0, id_.size(), 0);
    }
    int32_t nearest(V3 q, double *d2) const {
        best_ = 1e300; bid_ = 0;
        search(0, id_.size(), 0, q);
        *d2 = best_;
        return bid_;
    }

  private:
    static double comp(V3 p, int a) { return a == 0 ? p.x : (a == 1 ? p.y : p.z); }
    void build(size_t lo, size_t hi, int depth) {
        if (hi - lo <= 8) return;
        size_t mid = (lo + hi) / 2;
        int a = depth % 3;
        std::vector<size_t> idx(hi - lo);
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = lo + i;
        std::nth_element(idx.begin(), idx.begin() + (mid - lo), idx.end(),
                         [&](size_t x, size_t y) { return comp(pt_[x], a) < comp(pt_[y], a); });
        std::vector<V3> p2(idx.size()); std::vector<int32_t> i2(idx.size());
        for (size_t i = 0; i < idx.size(); ++i) { p2[i] = pt_[idx[i]]; i2[i] = id_[idx[i]]; }
        for (size_t i = 0; i < idx.size(); ++i) { pt_[lo + i] = p2[i]; id_[lo + i] = i2[i]; }
        build(lo, mid, depth + 1);
        build(mid + 1, hi, depth + 1);
    }
    void visit(size_t i, V3 q) const {
        V3 d = pt_[i] - q;
        double dd = d.x * d.x + d.y * d.y + d.z * d.z;
        if (dd < best_ || (dd == best_ && id_[i] < bid_)) { best_ = dd; bid_ = id_[i]; }
    }
    void search(size_t lo, size_t hi, int depth, V3 q) const {
        if (hi - lo <= 8) { for (size_t i = lo; i < hi; ++i) visit(i, q); return; }
        size_t mid = (lo + hi) / 2;
        int a = depth % 3;
        visit(mid, q);
        double diff = comp(q, a) - comp(pt_[mid], a);
        if (diff < 0) {
            search(lo, mid, depth + 1, q);
            if (diff * diff <= best_) search(mid + 1, hi, depth + 1, q);
        } else {
            search(mid + 1, hi, depth + 1, q);
            if (diff * diff <= best_) search(lo, mid, depth + 1, q);
        }
    }
    std::vector<int32_t> id_;
    std::vector<V3> pt_;
    mutable double best_ = 0;
    mutable int32_t bid_ = 0;
};

// ---- level 1 from tetrahedra --------------------------------------------
// the elements other than tetrahedra and the quadrilateral boundary faces,
// [k][n] column-major, 1-based
struct Hybrid {
    std::vector<int32_t> hex, pri, pyr, quad, quad_ind;
};

// The engine inlet sides of a level under construction: a side is found by
// its node pair and its coefficients are summed; a new one is appended with
// its inlet number (registerEngineInletSide, gen3d_boundary.f90:431-485, and
// its coarse-level form in agglomerateBoundary :1061-1099).
struct EngineSideSet {
    std::map<std::pair<int32_t, int32_t>, int32_t> at;
    std::vector<int32_t> a, b, inlet;
    std::vector<V3> w;
    void add(int32_t p1, int32_t p2, V3 c, int32_t in) {
        const std::pair<int32_t, int32_t> key{std::min(p1, p2), std::max(p1, p2)};
        auto it = at.find(key);
        if (it != at.end()) { w[it->second] = w[it->second] + c; return; }
        at.emplace(key, (int32_t)a.size());
        a.push_back(key.first); b.push_back(key.second); inlet.push_back(in); w.push_back(c);
    }
    void store(LevelData &L) const {
        const size_t n = a.size();
        L.eside.resize(3 * n); L.ew.resize(3 * n);
        for (size_t s = 0; s < n; ++s) {
            L.eside[s] = a[s]; L.eside[n + s] = b[s]; L.eside[2 * n + s] = inlet[s];
            L.ew[s] = w[s].x; L.ew[n + s] = w[s].y; L.ew[2 * n + s] = w[s].z;
        }
    }
};

// The engine inlet sides of one boundary face of indicator 5 (inlet 1) or 6
// (inlet 2), from the face's median-dual pieces (makeEngineInflowData,
// triangles gen3d_boundary.f90:790-843, quadrilaterals :846-916).  The faces
// are taken in the orientation the preprocessor gives them (right-hand normal
// into the domain), so the coefficients point out of the domain and the mass
// flow into an engine is positive.
void engine_tri_sides(const int32_t p[3], const V3 x[3], int32_t inlet, EngineSideSet &es) {
    const V3 xm = div3((x[0] + x[1]) + x[2]);
    const V3 xb1 = scl(0.5, x[0] + x[1]), xb2 = scl(0.5, x[1] + x[2]), xb3 = scl(0.5, x[2] + x[0]);
    es.add(p[0], p[1], halfcross(xm - x[0], xb1 - x[0]), inlet);
    es.add(p[0], p[2], halfcross(xb3 - x[0], xm - x[0]), inlet);
    es.add(p[1], p[2], halfcross(xm - x[1], xb2 - x[1]), inlet);
}
void engine_quad_sides(const int32_t p[4], const V3 x[4], int32_t inlet, EngineSideSet &es) {
    const V3 xm = scl(0.25, ((x[0] + x[1]) + x[2]) + x[3]);
    const V3 xb1 = scl(0.5, x[0] + x[1]), xb2 = scl(0.5, x[1] + x[2]), xb3 = scl(0.5, x[2] + x[3]),
             xb4 = scl(0.5, x[0] + x[3]);
    es.add(p[0], p[1], halfcross(xm - x[0], xb1 - x[0]), inlet);
    es.add(p[0], p[3], halfcross(xb4 - x[0], xm - x[0]), inlet);
    es.add(p[2], p[1], halfcross(xb2 - x[2], xm - x[2]), inlet);
    es.add(p[2], p[3], halfcross(xm - x[2], xb3 - x[2]), inlet);
}

void build_fine(fp_mesh &M, int32_t N, const std::vector<double> &xyz_old,
                std::vector<int32_t> tets_old, std::vector<int32_t> tris_old,
                const std::vector<int32_t> &tri_ind, Hybrid hy = Hybrid{}) {
    const int32_t NT = (int32_t)(tets_old.size() / 4);
    const int32_t NF = (int32_t)(tris_old.size() / 3);
    const int32_t NH = (int32_t)(hy.hex.size() / 8), NP = (int32_t)(hy.pri.size() / 6);
    const int32_t NY = (int32_t)(hy.pyr.size() / 5), NQ = (int32_t)(hy.quad.size() / 4);
    // boundary-first numbering (gen3d_grid.f90:127-383): boundary nodes keep
    // their relative order and take 1..Nb, interior nodes follow
    std::vector<char> isb(N, 0);
    for (int32_t f = 0; f < NF; ++f)
        for (int k = 0; k < 3; ++k) isb[tris_old[(size_t)k * NF + f] - 1] = 1;
    for (int32_t f = 0; f < NQ; ++f)
        for (int k = 0; k < 4; ++k) isb[hy.quad[(size_t)k * NQ + f] - 1] = 1;
    std::vector<int32_t> o2n(N), n2o(N);
    int32_t nb = 0;
    for (int32_t i = 0; i < N; ++i) if (isb[i]) { o2n[i] = nb; n2o[nb] = i; ++nb; }
    int32_t ni = nb;
    for (int32_t i = 0; i < N; ++i) if (!isb[i]) { o2n[i] = ni; n2o[ni] = i; ++ni; }
    M.perm.resize(N);
    for (int32_t i = 0; i < N; ++i) M.perm[i] = n2o[i] + 1;

    LevelData L;
    L.N = N; L.Nb = nb;
    L.xyz.resize(3 * (size_t)N);
    for (int32_t i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) L.xyz[(size_t)k * N + i] = xyz_old[(size_t)k * N + n2o[i]];
    auto X = [&](int32_t p) -> V3 {  // 1-based new index
        return {L.xyz[p - 1], L.xyz[(size_t)N + p - 1], L.xyz[2 * (size_t)N + p - 1]};
    };
    for (auto &t : tets_old) t = o2n[t - 1] + 1;
    for (auto &t : tris_old) t = o2n[t - 1] + 1;
    for (std::vector<int32_t> *v : {&hy.hex, &hy.pri, &hy.pyr, &hy.quad})
        for (auto &t : *v) t = o2n[t - 1] + 1;

    // edges of every tetrahedron (makeCalcDataForTet, gen3d_grid.f90:2092-2332)
    auto *tm_edges = new SectionTimer("tet edges");
    // side lookup: a few slots per first node (edges are keyed by their
    // smaller node, and tets arrive roughly in node order, so this stays in
    // cache); nodes with more sides spill into a hash map
    constexpr int kSlots = 12;
    std::vector<int32_t> slot_i2((size_t)N * kSlots, 0), slot_id((size_t)N * kSlots, -1);
    PairMap smap(1024);
    std::vector<int32_t> s1, s2;
    std::vector<V3> sc;
    std::vector<double> sl;
    s1.reserve(NT * 7 / 6 + 16); s2.reserve(NT * 7 / 6 + 16);
    sc.reserve(NT * 7 / 6 + 16); sl.reserve(NT * 7 / 6 + 16);
    L.vol.assign(N, 0.0);
    int64_t nneg = 0;
    auto register_side = [&](int32_t p1, int32_t p2, const TetSide<double> &ts) -> double {
        const double nv = ts.nv;
        L.vol[p1 - 1] += nv;
        L.vol[p2 - 1] += nv;
        V3 coef = ts.coef;  // half the side coefficient
        V3 d = X(p2) - X(p1);
        double len = std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
        int32_t i1 = std::min(p1, p2), i2 = p1 + p2 - i1;
        if (i1 != p1) coef = scl(-1.0, coef);
        int64_t slot = -1;
        {
            const size_t base = (size_t)(i1 - 1) * kSlots;
            int q = 0;
            for (; q < kSlots; ++q) {
                if (slot_id[base + q] < 0) break;
                if (slot_i2[base + q] == i2) { slot = slot_id[base + q]; break; }
            }
            if (slot < 0) {
                if (q < kSlots) {
                    slot_i2[base + q] = i2; slot_id[base + q] = (int32_t)s1.size();
                } else {
                    slot = smap.find_or_insert(pkey(i1, i2), (int64_t)s1.size());
                }
            }
        }
        if (slot < 0) {
            s1.push_back(i1); s2.push_back(i2); sc.push_back(coef); sl.push_back(len);
        } else {
            sc[slot] = sc[slot] + coef;
        }
        return nv;
    };
    // hexahedra, prisms and pyramids (makeCalculationData gen3d_grid.f90:
    // 699-785 takes them in this order before the tetrahedra); a negative
    // element volume is an error (gen3d warns)
    auto hybrid = [&](const std::vector<int32_t> &el, int nv, int ns, auto &&sides_of) {
        const int32_t ne = (int32_t)(el.size() / nv);
        for (int32_t t = 0; t < ne; ++t) {
            int32_t p[8];
            V3 xv[3][8];
            for (int k = 0; k < nv; ++k) {
                p[k] = el[(size_t)k * ne + t];
                xv[0][k] = xv[1][k] = xv[2][k] = X(p[k]);
            }
            TetSideMoving ts[12];
            sides_of(xv, p, ts);
            double ev = 0;
            for (int k = 0; k < ns; ++k) {
                TetSide<double> s1{ts[k].a, ts[k].b, ts[k].coef, ts[k].nv[0]};
                ev += 2. * register_side(p[ts[k].a], p[ts[k].b], s1);
            }
            if (ev <= 0) ++nneg;
        }
    };
    hybrid(hy.hex, 8, 12, [](const V3 (*x)[8], const int32_t *q, TetSideMoving *o) { hex_sides(x, q, o); });
    hybrid(hy.pri, 6, 9, [](const V3 (*x)[8], const int32_t *q, TetSideMoving *o) {
        V3 y[3][6];
        for (int t = 0; t < 3; ++t) for (int k = 0; k < 6; ++k) y[t][k] = x[t][k];
        pri_sides(y, q, o);
    });
    hybrid(hy.pyr, 5, 8, [](const V3 (*x)[8], const int32_t *, TetSideMoving *o) {
        V3 y[3][5];
        for (int t = 0; t < 3; ++t) for (int k = 0; k < 5; ++k) y[t][k] = x[t][k];
        pyr_sides(y, o);
    });
    for (int32_t t = 0; t < NT; ++t) {
        int32_t p[4] = {tets_old[t], tets_old[(size_t)NT + t], tets_old[2 * (size_t)NT + t],
                        tets_old[3 * (size_t)NT + t]};
        // orientation: the element volume of gen3d must be positive; a tet
        // given with the opposite orientation is flipped (swap nodes 3, 4)
        {
            V3 a = X(p[1]) - X(p[0]), b = X(p[2]) - X(p[0]), c = X(p[3]) - X(p[0]);
            double det = a.x * (b.y * c.z - b.z * c.y) - a.y * (b.x * c.z - b.z * c.x) +
                         a.z * (b.x * c.y - b.y * c.x);
            if (det < 0) std::swap(p[2], p[3]);
        }
        tets_old[t] = p[0]; tets_old[(size_t)NT + t] = p[1];
        tets_old[2 * (size_t)NT + t] = p[2]; tets_old[3 * (size_t)NT + t] = p[3];
        const V3 xv[4] = {X(p[0]), X(p[1]), X(p[2]), X(p[3])};
        TetSide<double> ts[6];
        tet_sides(xv, ts);
        double ev = 0;
        for (int k = 0; k < 6; ++k) ev += 2. * register_side(p[ts[k].a], p[ts[k].b], ts[k]);
        if (ev <= 0) ++nneg;
    }
    delete tm_edges;
    { std::vector<int32_t>().swap(slot_i2); std::vector<int32_t>().swap(slot_id); }
    if (nneg) throw std::runtime_error("negative element volumes: " + std::to_string(nneg));
    L.E = (int32_t)s1.size();
    L.side.resize(2 * (size_t)L.E); L.sw.resize(3 * (size_t)L.E); L.slen = sl;
    for (int32_t e = 0; e < L.E; ++e) {
        L.side[e] = s1[e]; L.side[(size_t)L.E + e] = s2[e];
        L.sw[e] = sc[e].x; L.sw[(size_t)L.E + e] = sc[e].y; L.sw[2 * (size_t)L.E + e] = sc[e].z;
    }
    { std::vector<V3>().swap(sc); }

    // boundary triangles: orient each so that its right-hand normal points
    // into the domain (towards the tet that owns it), which makes the
    // boundary coefficients outward like the edge coefficients
    SectionTimer tm_faces("boundary faces");
    PairMap fmap((size_t)NF + 16);
    auto fkey = [&](int32_t a, int32_t b, int32_t c) {
        int32_t s[3] = {a, b, c};
        std::sort(s, s + 3);
        // 21 bits per index would overflow for big meshes; combine two keys
        return std::make_pair(pkey(s[0], s[1]), (uint64_t)s[2]);
    };
    // face -> a point inside its element (a tetrahedron's opposite vertex,
    // another element's vertex mean): a map keyed by (min,mid) with a
    // per-face list; faces sharing (min,mid) are few, resolved linearly
    std::vector<int32_t> fopp(NF, 0);
    std::vector<V3> fint(NF);
    std::vector<char> fhas(NF, 0);
    auto centroid = [&](const int32_t *p, int nv) {
        V3 c = {0, 0, 0};
        for (int k = 0; k < nv; ++k) c = c + X(p[k]);
        return scl(1.0 / nv, c);
    };
    {
        std::vector<std::vector<std::pair<int32_t, int32_t>>> buckets;  // (max, face)
        buckets.reserve(NF);
        for (int32_t f = 0; f < NF; ++f) {
            auto k = fkey(tris_old[f], tris_old[(size_t)NF + f], tris_old[2 * (size_t)NF + f]);
            int64_t slot = fmap.find_or_insert(k.first, (int64_t)buckets.size());
            if (slot < 0) { buckets.emplace_back(); slot = (int64_t)buckets.size() - 1; }
            buckets[slot].push_back({(int32_t)k.second, f});
        }
        for (int32_t t = 0; t < NT; ++t) {
            int32_t p[4] = {tets_old[t], tets_old[(size_t)NT + t], tets_old[2 * (size_t)NT + t],
                            tets_old[3 * (size_t)NT + t]};
            int nbn = (p[0] <= nb) + (p[1] <= nb) + (p[2] <= nb) + (p[3] <= nb);
            if (nbn < 3) continue;  // a boundary face has three boundary nodes
            for (int o = 0; o < 4; ++o) {
                int32_t a = p[(o + 1) % 4], b = p[(o + 2) % 4], c = p[(o + 3) % 4];
                auto k = fkey(a, b, c);
                int64_t slot = fmap.find(k.first);
                if (slot < 0) continue;
                for (auto &pr : buckets[slot])
                    if (pr.first == (int32_t)k.second) { fopp[pr.second] = p[o]; fint[pr.second] = X(p[o]); fhas[pr.second] = 1; }
            }
        }
        // triangular faces of prisms (the two caps) and pyramids (the sides)
        auto tri_faces = [&](const std::vector<int32_t> &el, int nv, const int (*fc)[3], int nf) {
            const int32_t ne = (int32_t)(el.size() / nv);
            for (int32_t t = 0; t < ne; ++t) {
                int32_t p[8];
                for (int k = 0; k < nv; ++k) p[k] = el[(size_t)k * ne + t];
                for (int o = 0; o < nf; ++o) {
                    auto k = fkey(p[fc[o][0]], p[fc[o][1]], p[fc[o][2]]);
                    int64_t slot = fmap.find(k.first);
                    if (slot < 0) continue;
                    for (auto &pr : buckets[slot])
                        if (pr.first == (int32_t)k.second) { fint[pr.second] = centroid(p, nv); fhas[pr.second] = 1; }
                }
            }
        };
        const int pri_tri[2][3] = {{0, 1, 2}, {3, 4, 5}};
        const int pyr_tri[4][3] = {{0, 1, 4}, {1, 2, 4}, {2, 3, 4}, {3, 0, 4}};
        tri_faces(hy.pri, 6, pri_tri, 2);
        tri_faces(hy.pyr, 5, pyr_tri, 4);
    }
    // quadrilateral faces -> the vertex mean of their element (hexahedra,
    // prism sides, pyramid bases)
    std::vector<V3> qint(NQ);
    std::vector<char> qhas(NQ, 0);
    {
        auto qkey = [&](int32_t a, int32_t b, int32_t c, int32_t d) {
            int32_t q4[4] = {a, b, c, d};
            std::sort(q4, q4 + 4);
            return std::make_pair(pkey(q4[0], q4[1]), pkey(q4[2], q4[3]));
        };
        std::map<std::pair<uint64_t, uint64_t>, int32_t> qmap;
        for (int32_t f = 0; f < NQ; ++f)
            qmap[qkey(hy.quad[f], hy.quad[(size_t)NQ + f], hy.quad[2 * (size_t)NQ + f], hy.quad[3 * (size_t)NQ + f])] = f;
        auto quad_faces = [&](const std::vector<int32_t> &el, int nv, const int (*fc)[4], int nf) {
            const int32_t ne = (int32_t)(el.size() / nv);
            for (int32_t t = 0; t < ne; ++t) {
                int32_t p[8];
                for (int k = 0; k < nv; ++k) p[k] = el[(size_t)k * ne + t];
                for (int o = 0; o < nf; ++o) {
                    auto it = qmap.find(qkey(p[fc[o][0]], p[fc[o][1]], p[fc[o][2]], p[fc[o][3]]));
                    if (it != qmap.end()) { qint[it->second] = centroid(p, nv); qhas[it->second] = 1; }
                }
            }
        };
        const int hex_q[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
        const int pri_q[3][4] = {{0, 1, 4, 3}, {1, 2, 5, 4}, {2, 0, 3, 5}};
        const int pyr_q[1][4] = {{0, 1, 2, 3}};
        quad_faces(hy.hex, 8, hex_q, 6);
        quad_faces(hy.pri, 6, pri_q, 3);
        quad_faces(hy.pyr, 5, pyr_q, 1);
    }
    PairMap bmap((size_t)NF * 2 + 16);
    std::vector<int32_t> b1, b2, bi;
    std::vector<V3> bc;
    auto register_bside = [&](int32_t p1, int32_t p2, V3 coef, int ind) {
        int32_t i1 = std::min(p1, p2), i2 = std::max(p1, p2);
        int64_t slot = bmap.find_or_insert(pkey(i1, i2), (int64_t)b1.size());
        if (slot >= 0) {
            bc[slot] = bc[slot] + coef;
        } else {
            b1.push_back(i1); b2.push_back(i2); bi.push_back(ind); bc.push_back(coef);
        }
    };
    EngineSideSet esides;
    std::vector<int32_t> tris_new(3 * (size_t)NF);
    for (int32_t f = 0; f < NF; ++f) {
        int32_t p1 = tris_old[f], p2 = tris_old[(size_t)NF + f], p3 = tris_old[2 * (size_t)NF + f];
        if (!fhas[f]) throw std::runtime_error("boundary triangle without an element");
        V3 a = X(p2) - X(p1), b = X(p3) - X(p1), d = fint[f] - X(p1);
        V3 n = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
        if (n.x * d.x + n.y * d.y + n.z * d.z < 0) std::swap(p2, p3);
        tris_new[f] = p1; tris_new[(size_t)NF + f] = p2; tris_new[2 * (size_t)NF + f] = p3;
        int ind = tri_ind[f];
        const int32_t pv[3] = {p1, p2, p3};
        const V3 xv[3] = {X(p1), X(p2), X(p3)};
        TriSide<double> ts[3];
        tri_sides(xv, ts);
        for (int k = 0; k < 3; ++k) register_bside(pv[ts[k].a], pv[ts[k].b], ts[k].coef, ind);
        if (ind == 5 || ind == 6) engine_tri_sides(pv, xv, ind - 4, esides);
    }
    // quadrilateral faces after the triangles (makeCalcDataForBoundary
    // gen3d_boundary.f90:627-766), oriented like them
    std::vector<int32_t> quads_new(4 * (size_t)NQ);
    for (int32_t f = 0; f < NQ; ++f) {
        int32_t p[4] = {hy.quad[f], hy.quad[(size_t)NQ + f], hy.quad[2 * (size_t)NQ + f], hy.quad[3 * (size_t)NQ + f]};
        if (!qhas[f]) throw std::runtime_error("boundary quadrilateral without an element");
        V3 a = X(p[2]) - X(p[0]), b = X(p[3]) - X(p[1]), d = qint[f] - X(p[0]);
        V3 n = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
        if (n.x * d.x + n.y * d.y + n.z * d.z < 0) std::swap(p[1], p[3]);
        V3 xv[3][4];
        for (int k = 0; k < 4; ++k) {
            quads_new[(size_t)k * NQ + f] = p[k];
            xv[0][k] = xv[1][k] = xv[2][k] = X(p[k]);
        }
        TriSideMoving ts[4];
        quad_sides_moving(xv, ts);
        for (int k = 0; k < 4; ++k) register_bside(p[ts[k].a], p[ts[k].b], ts[k].coef, hy.quad_ind[f]);
        if (hy.quad_ind[f] == 5 || hy.quad_ind[f] == 6) engine_quad_sides(p, xv[0], hy.quad_ind[f] - 4, esides);
    }
    esides.store(L);
    L.B = (int32_t)b1.size();
    L.bside.resize(3 * (size_t)L.B); L.bw.resize(3 * (size_t)L.B);
    for (int32_t b = 0; b < L.B; ++b) {
        L.bside[b] = b1[b]; L.bside[(size_t)L.B + b] = b2[b]; L.bside[2 * (size_t)L.B + b] = bi[b];
        L.bw[b] = bc[b].x; L.bw[(size_t)L.B + b] = bc[b].y; L.bw[2 * (size_t)L.B + b] = bc[b].z;
    }
    // node indicators by priority over the faces in order
    L.bnd_indicator.assign(nb, 0);
    for (int32_t f = 0; f < NF; ++f)
        for (int k = 0; k < 3; ++k) {
            int32_t n = tris_new[(size_t)k * NF + f] - 1;
            L.bnd_indicator[n] = merge_indicator(L.bnd_indicator[n], tri_ind[f]);
        }
    for (int32_t f = 0; f < NQ; ++f)
        for (int k = 0; k < 4; ++k) {
            int32_t n = quads_new[(size_t)k * NQ + f] - 1;
            L.bnd_indicator[n] = merge_indicator(L.bnd_indicator[n], hy.quad_ind[f]);
        }
    build_register(L);

    // wall distance: Euclidean distance to the nearest wall (indicator 1)
    // node and that node's number, by a k-d tree over the wall nodes
    L.wdist.assign(N, 1.0e6);
    L.wnode.assign(N, 0);
    std::vector<int32_t> wall;
    for (int32_t j = 0; j < nb; ++j) if (L.bnd_indicator[j] == 1) wall.push_back(j + 1);
    SectionTimer tm_wall("wall distance");
    if (!wall.empty()) {
        KdTree kd(wall, [&](int32_t p) { return X(p); });
        unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                KdTree local = kd;  // queries keep per-tree scratch state
                for (int32_t i = (int32_t)t; i < N; i += (int32_t)nt) {
                    double d2; int32_t w = local.nearest(X(i + 1), &d2);
                    L.wdist[i] = std::sqrt(d2);
                    L.wnode[i] = w;
                }
            });
        for (auto &x : th) x.join();
    }
    M.tets = std::move(tets_old);
    M.tris = std::move(tris_new);
    M.tri_ind = tri_ind;
    M.hexes = std::move(hy.hex); M.prisms = std::move(hy.pri); M.pyramids = std::move(hy.pyr);
    M.quads = std::move(quads_new); M.quad_ind = std::move(hy.quad_ind);
    M.lv.clear();
    M.lv.push_back(std::move(L));
}

// ---- agglomeration --------------------------------------------------------
void agglomerate(const LevelData &F, LevelData &C) {
    const int32_t N = F.N, E = F.E;
    // node -> incident edges in edge order
    std::vector<int32_t> rp(N + 1, 0), adj(2 * (size_t)E);
    for (int32_t e = 0; e < E; ++e) { rp[F.side[e]]++; rp[F.side[(size_t)E + e]]++; }
    for (int32_t i = 0; i < N; ++i) rp[i + 1] += rp[i];
    {
        std::vector<int32_t> fill(rp.begin(), rp.end() - 1);
        for (int32_t e = 0; e < E; ++e) {
            adj[fill[F.side[e] - 1]++] = e;
            adj[fill[F.side[(size_t)E + e] - 1]++] = e;
        }
    }
    auto other = [&](int32_t e, int32_t i) {  // 0-based node
        int32_t a = F.side[e] - 1, b = F.side[(size_t)E + e] - 1;
        return a == i ? b : a;
    };
    auto wnorm = [&](int32_t e) {
        double x = F.sw[e], y = F.sw[(size_t)E + e], z = F.sw[2 * (size_t)E + e];
        return std::sqrt(x * x + y * y + z * z);
    };
    std::vector<int32_t> avail(N), agg(N, -1);
    int32_t maxdeg = 0;
    for (int32_t i = 0; i < N; ++i) { avail[i] = rp[i + 1] - rp[i]; maxdeg = std::max(maxdeg, avail[i]); }
    std::vector<int32_t> seed_of;  // aggregate -> fine seed (0-based)
    for (int grp = 0; grp < 2; ++grp) {
        int32_t lo = grp == 0 ? 0 : F.Nb, hi = grp == 0 ? F.Nb : N;
        std::vector<std::deque<int32_t>> bucket(maxdeg + 1);
        for (int32_t i = lo; i < hi; ++i) bucket[avail[i]].push_back(i);
        int cur = maxdeg;
        while (true) {
            while (cur >= 0 && bucket[cur].empty()) --cur;
            if (cur < 0) break;
            int32_t s = bucket[cur].front(); bucket[cur].pop_front();
            if (agg[s] >= 0 || avail[s] != cur) continue;  // stale entry
            int32_t a = (int32_t)seed_of.size();
            seed_of.push_back(s);
            agg[s] = a; avail[s] = 0;
            std::vector<int32_t> merged;
            for (int32_t k = rp[s]; k < rp[s + 1]; ++k) {
                int32_t n = other(adj[k], s);
                if (agg[n] < 0) { agg[n] = a; avail[n] = 0; merged.push_back(n); }
            }
            for (int32_t n : merged)
                for (int32_t k = rp[n]; k < rp[n + 1]; ++k) {
                    int32_t m = other(adj[k], n);
                    if (agg[m] < 0) {
                        avail[m] -= 1;
                        if (m >= lo && m < hi) bucket[avail[m]].push_back(m);
                    }
                }
        }
    }
    // single-node aggregates join the neighbour aggregate of the strongest edge
    int32_t na = (int32_t)seed_of.size();
    std::vector<int32_t> size(na, 0);
    for (int32_t i = 0; i < N; ++i) size[agg[i]]++;
    std::vector<int32_t> remap(na);
    for (int32_t a = 0; a < na; ++a) remap[a] = a;
    for (int32_t a = 0; a < na; ++a) {
        if (size[a] != 1) continue;
        int32_t s = seed_of[a];
        double best = -1; int32_t to = -1;
        for (int32_t k = rp[s]; k < rp[s + 1]; ++k) {
            int32_t n = other(adj[k], s);
            int32_t an = remap[agg[n]];
            if (an == a) continue;
            double w = wnorm(adj[k]);
            if (w > best) { best = w; to = an; }
        }
        if (to >= 0) { remap[a] = to; size[to] += 1; size[a] = 0; }
    }
    for (int32_t i = 0; i < N; ++i) agg[i] = remap[agg[i]];
    // number boundary aggregates first (those holding a fine boundary node)
    std::vector<char> live(na, 0), bnd(na, 0);
    for (int32_t i = 0; i < N; ++i) { live[agg[i]] = 1; if (i < F.Nb) bnd[agg[i]] = 1; }
    std::vector<int32_t> newid(na, -1);
    int32_t nc = 0;
    for (int32_t a = 0; a < na; ++a) if (live[a] && bnd[a]) newid[a] = nc++;
    int32_t ncb = nc;
    for (int32_t a = 0; a < na; ++a) if (live[a] && !bnd[a]) newid[a] = nc++;

    C = LevelData();
    C.N = nc; C.Nb = ncb;
    C.parent.resize(N);
    for (int32_t i = 0; i < N; ++i) C.parent[i] = newid[agg[i]] + 1;
    C.vol.assign(nc, 0.0);
    for (int32_t i = 0; i < N; ++i) C.vol[C.parent[i] - 1] += F.vol[i];
    C.rweight.resize(N);
    for (int32_t i = 0; i < N; ++i) C.rweight[i] = F.vol[i] / C.vol[C.parent[i] - 1];
    C.seed.assign(nc, 0); C.wdist.assign(nc, 0.0); C.wnode.assign(nc, 0);
    for (int32_t a = 0; a < na; ++a) {
        if (!live[a] || seed_of[a] < 0) continue;
        int32_t c = newid[a], s = seed_of[a];
        int32_t lvl1 = F.seed.empty() ? s + 1 : F.seed[s];
        C.seed[c] = lvl1;
    }
    // wall distance: the children's volume-weighted mean, and the wall node:
    // the parent of the first child's (makeDistanceFieldsForCoarseMesh
    // gen3d_grid.f90:5823-5846)
    for (int32_t i = 0; i < N; ++i) {
        const int32_t c = C.parent[i] - 1;
        C.wdist[c] = C.wdist[c] + F.vol[i] * F.wdist[i] / C.vol[c];
        if (C.wnode[c] == 0 && F.wnode[i] >= 1) C.wnode[c] = C.parent[F.wnode[i] - 1];
    }
    // a merged single-node aggregate has no own coarse node: nothing to fix
    // coarse edges (createSides)
    PairMap smap((size_t)E / 4 + 16);
    std::vector<int32_t> s1, s2; std::vector<V3> sc; std::vector<double> sl;
    C.side_of.assign(E, 0);
    for (int32_t e = 0; e < E; ++e) {
        int32_t c1 = C.parent[F.side[e] - 1], c2 = C.parent[F.side[(size_t)E + e] - 1];
        if (c1 == c2) continue;
        V3 w = {F.sw[e], F.sw[(size_t)E + e], F.sw[2 * (size_t)E + e]};
        int32_t i1 = std::min(c1, c2), i2 = c1 + c2 - i1;
        if (i1 != c1) w = scl(-1.0, w);
        int64_t slot = smap.find_or_insert(pkey(i1, i2), (int64_t)s1.size());
        const int32_t id = slot < 0 ? (int32_t)s1.size() : (int32_t)slot;
        C.side_of[e] = i1 != c1 ? -(id + 1) : id + 1;
        if (slot < 0) { s1.push_back(i1); s2.push_back(i2); sc.push_back(w); sl.push_back(F.slen[e]); }
        else sc[slot] = sc[slot] + w;
    }
    C.E = (int32_t)s1.size();
    C.side.resize(2 * (size_t)C.E); C.sw.resize(3 * (size_t)C.E); C.slen = sl;
    for (int32_t e = 0; e < C.E; ++e) {
        C.side[e] = s1[e]; C.side[(size_t)C.E + e] = s2[e];
        C.sw[e] = sc[e].x; C.sw[(size_t)C.E + e] = sc[e].y; C.sw[2 * (size_t)C.E + e] = sc[e].z;
    }
    // coarse boundary edges (agglomerateBoundary): self-edges are kept
    PairMap bmap((size_t)F.B + 16);
    std::vector<int32_t> b1, b2, bi; std::vector<V3> bc;
    C.bside_of.assign(F.B, 0);
    for (int32_t b = 0; b < F.B; ++b) {
        int32_t c1 = C.parent[F.bside[b] - 1], c2 = C.parent[F.bside[(size_t)F.B + b] - 1];
        int32_t i1 = std::min(c1, c2), i2 = std::max(c1, c2);
        V3 w = {F.bw[b], F.bw[(size_t)F.B + b], F.bw[2 * (size_t)F.B + b]};
        int64_t slot = bmap.find_or_insert(pkey(i1, i2), (int64_t)b1.size());
        const int32_t id = slot < 0 ? (int32_t)b1.size() : (int32_t)slot;
        C.bside_of[b] = c1 > c2 ? -(id + 1) : id + 1;
        if (slot < 0) { b1.push_back(i1); b2.push_back(i2); bi.push_back(F.bside[2 * (size_t)F.B + b]); bc.push_back(w); }
        else bc[slot] = bc[slot] + w;
    }
    C.B = (int32_t)b1.size();
    C.bside.resize(3 * (size_t)C.B); C.bw.resize(3 * (size_t)C.B);
    for (int32_t b = 0; b < C.B; ++b) {
        C.bside[b] = b1[b]; C.bside[(size_t)C.B + b] = b2[b]; C.bside[2 * (size_t)C.B + b] = bi[b];
        C.bw[b] = bc[b].x; C.bw[(size_t)C.B + b] = bc[b].y; C.bw[2 * (size_t)C.B + b] = bc[b].z;
    }
    // coarse engine inlet sides: a side whose two nodes fall in one aggregate
    // is kept (agglomerateBoundary, gen3d_boundary.f90:1061-1099)
    {
        EngineSideSet es;
        const int32_t n = F.nes();
        for (int32_t s = 0; s < n; ++s) {
            const int32_t c1 = C.parent[F.eside[s] - 1], c2 = C.parent[F.eside[(size_t)n + s] - 1];
            es.add(c1, c2, {F.ew[s], F.ew[(size_t)n + s], F.ew[2 * (size_t)n + s]}, F.eside[2 * (size_t)n + s]);
        }
        es.store(C);
    }
    C.bnd_indicator.assign(ncb, 0);
    for (int32_t i = 0; i < F.Nb; ++i) {
        int32_t c = C.parent[i] - 1;
        C.bnd_indicator[c] = merge_indicator(C.bnd_indicator[c], F.bnd_indicator[i]);
    }
    build_register(C);
}

void build_levels(fp_mesh &M, int nlevels) {
    for (int l = 1; l < nlevels; ++l) {
        LevelData C;
        SectionTimer tm("agglomeration");
        agglomerate(M.lv.back(), C);
        if (C.N >= M.lv.back().N || C.N < 2) break;
        M.lv.push_back(std::move(C));
    }
}

// level-1 side numbers by node pair: for the smaller (1-based) node of a
// pair, the larger nodes of its sides and the sides' 0-based numbers
struct PairIndex {
    std::vector<int32_t> ptr, other, id;
    PairIndex(int32_t N, int32_t n, const int32_t *first, const int32_t *second) : ptr(N + 2, 0) {
        for (int32_t e = 0; e < n; ++e) ++ptr[std::min(first[e], second[e]) + 1];
        for (int32_t i = 0; i <= N; ++i) ptr[i + 1] += ptr[i];
        other.resize(n); id.resize(n);
        std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1);
        for (int32_t e = 0; e < n; ++e) {
            int32_t a = std::min(first[e], second[e]), b = std::max(first[e], second[e]);
            other[pos[a]] = b; id[pos[a]++] = e;
        }
    }
    int32_t find(int32_t a, int32_t b) const {
        for (int32_t q = ptr[a]; q < ptr[a + 1]; ++q)
            if (other[q] == b) return id[q];
        throw std::runtime_error("element side not in the mesh's side list");
    }
};

// The level-1 geometry of the mesh's own (oriented) tetrahedra and boundary
// triangles at the coordinates xyz, accumulated in the element order of
// build_fine so that the mesh's own coordinates give its arrays back bit for
// bit; with DN numbers, the derivative with respect to each element's vertex
// coordinates.
struct Geometry {
    const fp_mesh &M;
    const LevelData &L;
    PairIndex sides, bsides;
    int32_t NT, NF;
    explicit Geometry(const fp_mesh &m)
        : M(m), L(m.lv.at(0)),
          sides(L.N, L.E, L.side.data(), L.side.data() + L.E),
          bsides(L.N, L.B, L.bside.data(), L.bside.data() + L.B),
          NT((int32_t)(m.tets.size() / 4)), NF((int32_t)(m.tris.size() / 3)) {}
    V3 X(const double *xyz, int32_t p) const {
        return {xyz[p - 1], xyz[(size_t)L.N + p - 1], xyz[2 * (size_t)L.N + p - 1]};
    }
    void tet(int32_t t, int32_t *p) const {
        for (int k = 0; k < 4; ++k) p[k] = M.tets[(size_t)k * NT + t];
    }
    void tri(int32_t f, int32_t *p) const {
        for (int k = 0; k < 3; ++k) p[k] = M.tris[(size_t)k * NF + f];
    }
    // the sides of the hexahedra, prisms and pyramids (in this order) at the
    // three coordinate levels x[0..2], each passed to f(p1, p2, side)
    template <class F>
    void hybrid_sides(const double *const x[3], F &&f) const {
        auto run = [&](const std::vector<int32_t> &el, int nv, int ns, auto &&sides_of) {
            const int32_t ne = (int32_t)(el.size() / nv);
            for (int32_t t = 0; t < ne; ++t) {
                int32_t p[8];
                V3 xv[3][8];
                for (int k = 0; k < nv; ++k) {
                    p[k] = el[(size_t)k * ne + t];
                    for (int q = 0; q < 3; ++q) xv[q][k] = X(x[q], p[k]);
                }
                TetSideMoving ts[12];
                sides_of(xv, p, ts);
                for (int k = 0; k < ns; ++k) f(p[ts[k].a], p[ts[k].b], ts[k]);
            }
        };
        run(M.hexes, 8, 12, [](const V3 (*xv)[8], const int32_t *q, TetSideMoving *o) { hex_sides(xv, q, o); });
        run(M.prisms, 6, 9, [](const V3 (*xv)[8], const int32_t *q, TetSideMoving *o) {
            V3 y[3][6];
            for (int t = 0; t < 3; ++t) for (int k = 0; k < 6; ++k) y[t][k] = xv[t][k];
            pri_sides(y, q, o);
        });
        run(M.pyramids, 5, 8, [](const V3 (*xv)[8], const int32_t *, TetSideMoving *o) {
            V3 y[3][5];
            for (int t = 0; t < 3; ++t) for (int k = 0; k < 5; ++k) y[t][k] = xv[t][k];
            pyr_sides(y, o);
        });
    }
    // the quadrilateral boundary faces' sides, each passed to f(pa, pb, side)
    template <class F>
    void quad_sides(const double *const x[3], F &&f) const {
        const int32_t NQ = (int32_t)(M.quads.size() / 4);
        for (int32_t q4 = 0; q4 < NQ; ++q4) {
            int32_t p[4];
            V3 xv[3][4];
            for (int k = 0; k < 4; ++k) {
                p[k] = M.quads[(size_t)k * NQ + q4];
                for (int q = 0; q < 3; ++q) xv[q][k] = X(x[q], p[k]);
            }
            TriSideMoving ts[4];
            quad_sides_moving(xv, ts);
            for (int k = 0; k < 4; ++k) f(p[ts[k].a], p[ts[k].b], ts[k]);
        }
    }
    void eval(const double *xyz, double *sw, double *bw, double *vol) const {
        const size_t E = L.E, B = L.B;
        std::fill(sw, sw + 3 * E, 0.0);
        std::fill(bw, bw + 3 * B, 0.0);
        std::fill(vol, vol + L.N, 0.0);
        const double *x3[3] = {xyz, xyz, xyz};
        hybrid_sides(x3, [&](int32_t p1, int32_t p2, const TetSideMoving &ts) {
            vol[p1 - 1] += ts.nv[0];
            vol[p2 - 1] += ts.nv[0];
            V3 coef = ts.coef;
            int32_t i1 = std::min(p1, p2), i2 = p1 + p2 - i1;
            if (i1 != p1) coef = scl(-1.0, coef);
            const int32_t e = sides.find(i1, i2);
            sw[e] = sw[e] + coef.x; sw[E + e] = sw[E + e] + coef.y; sw[2 * E + e] = sw[2 * E + e] + coef.z;
        });
        for (int32_t t = 0; t < NT; ++t) {
            int32_t p[4];
            tet(t, p);
            const V3 xv[4] = {X(xyz, p[0]), X(xyz, p[1]), X(xyz, p[2]), X(xyz, p[3])};
            TetSide<double> ts[6];
            tet_sides(xv, ts);
            for (int k = 0; k < 6; ++k) {
                int32_t p1 = p[ts[k].a], p2 = p[ts[k].b];
                vol[p1 - 1] += ts[k].nv;
                vol[p2 - 1] += ts[k].nv;
                V3 coef = ts[k].coef;
                int32_t i1 = std::min(p1, p2), i2 = p1 + p2 - i1;
                if (i1 != p1) coef = scl(-1.0, coef);
                const int32_t e = sides.find(i1, i2);
                sw[e] = sw[e] + coef.x; sw[E + e] = sw[E + e] + coef.y; sw[2 * E + e] = sw[2 * E + e] + coef.z;
            }
        }
        for (int32_t f = 0; f < NF; ++f) {
            int32_t p[3];
            tri(f, p);
            const V3 xv[3] = {X(xyz, p[0]), X(xyz, p[1]), X(xyz, p[2])};
            TriSide<double> ts[3];
            tri_sides(xv, ts);
            for (int k = 0; k < 3; ++k) {
                const int32_t b = bsides.find(std::min(p[ts[k].a], p[ts[k].b]), std::max(p[ts[k].a], p[ts[k].b]));
                const V3 c = ts[k].coef;
                bw[b] = bw[b] + c.x; bw[B + b] = bw[B + b] + c.y; bw[2 * B + b] = bw[2 * B + b] + c.z;
            }
        }
        quad_sides(x3, [&](int32_t pa, int32_t pb, const TriSideMoving &ts) {
            const int32_t b = bsides.find(std::min(pa, pb), std::max(pa, pb));
            const V3 c = ts.coef;
            bw[b] = bw[b] + c.x; bw[B + b] = bw[B + b] + c.y; bw[2 * B + b] = bw[2 * B + b] + c.z;
        });
    }
    // The level-1 arrays of a moving mesh from the coordinates of the step
    // and of the two before, x[0..2]: the coefficients at the step, the
    // volumes at each level and the GCL weights of the step and of the one
    // before, accumulated in the element order of eval with registerSideData's
    // orientation rule (gen3d_struct.f90:381-396) and registerBoundarySideGCL's
    // (gen3d_boundary.f90:316-362)
    void eval_moving(const double *const x[3], double *sw, double *bw, double *vol, double *volp, double *volp2,
                     double *gcl, double *bgcl) const {
        const size_t E = L.E, B = L.B;
        std::fill(sw, sw + 3 * E, 0.0);
        std::fill(bw, bw + 3 * B, 0.0);
        std::fill(gcl, gcl + 2 * E, 0.0);
        std::fill(bgcl, bgcl + 4 * B, 0.0);
        for (double *v : {vol, volp, volp2}) std::fill(v, v + L.N, 0.0);
        auto add_side = [&](int32_t p1, int32_t p2, const TetSideMoving &ts) {
            vol[p1 - 1] += ts.nv[0]; vol[p2 - 1] += ts.nv[0];
            volp[p1 - 1] += ts.nv[1]; volp[p2 - 1] += ts.nv[1];
            volp2[p1 - 1] += ts.nv[2]; volp2[p2 - 1] += ts.nv[2];
            V3 coef = ts.coef;
            double g0 = 0.5 * ts.gcl[0], g1 = 0.5 * ts.gcl[1];
            int32_t i1 = std::min(p1, p2), i2 = p1 + p2 - i1;
            if (i1 != p1) { coef = scl(-1.0, coef); g0 = -g0; g1 = -g1; }
            const int32_t e = sides.find(i1, i2);
            sw[e] = sw[e] + coef.x; sw[E + e] = sw[E + e] + coef.y; sw[2 * E + e] = sw[2 * E + e] + coef.z;
            gcl[e] = gcl[e] + g0; gcl[E + e] = gcl[E + e] + g1;
        };
        hybrid_sides(x, add_side);
        for (int32_t t = 0; t < NT; ++t) {
            int32_t p[4];
            tet(t, p);
            V3 xv[3][4];
            for (int q = 0; q < 3; ++q)
                for (int k = 0; k < 4; ++k) xv[q][k] = X(x[q], p[k]);
            TetSideMoving ts[6];
            tet_sides_moving(xv, ts);
            for (int k = 0; k < 6; ++k) add_side(p[ts[k].a], p[ts[k].b], ts[k]);
        }
        auto add_bside = [&](int32_t pa, int32_t pb, const TriSideMoving &ts) {
            const int32_t b = bsides.find(std::min(pa, pb), std::max(pa, pb));
            const V3 c = ts.coef;
            bw[b] = bw[b] + c.x; bw[B + b] = bw[B + b] + c.y; bw[2 * B + b] = bw[2 * B + b] + c.z;
            // the smaller node's weights first
            const int s1 = pa < pb ? 0 : 1, s2 = 1 - s1;
            bgcl[b] = bgcl[b] + 0.25 * ts.gcl[s1][0];
            bgcl[B + b] = bgcl[B + b] + 0.25 * ts.gcl[s2][0];
            bgcl[2 * B + b] = bgcl[2 * B + b] + 0.25 * ts.gcl[s1][1];
            bgcl[3 * B + b] = bgcl[3 * B + b] + 0.25 * ts.gcl[s2][1];
        };
        for (int32_t f = 0; f < NF; ++f) {
            int32_t p[3];
            tri(f, p);
            V3 xv[3][3];
            for (int q = 0; q < 3; ++q)
                for (int k = 0; k < 3; ++k) xv[q][k] = X(x[q], p[k]);
            TriSideMoving ts[3];
            tri_sides_moving(xv, ts);
            for (int k = 0; k < 3; ++k) add_bside(p[ts[k].a], p[ts[k].b], ts[k]);
        }
        quad_sides(x, add_bside);
    }
    // xyz_bar = (d(sw, bw, vol)/d xyz)^T (sw_bar, bw_bar, vol_bar)
    void vjp(const double *xyz, const double *swb, const double *bwb, const double *volb, double *xb) const {
        if (M.hybrid()) throw std::invalid_argument("the geometry derivative covers tetrahedral meshes");
        const size_t E = L.E, B = L.B, N = L.N;
        std::fill(xb, xb + 3 * N, 0.0);
        for (int32_t t = 0; t < NT; ++t) {
            int32_t p[4];
            tet(t, p);
            V3T<DN<12>> xv[4];
            for (int k = 0; k < 4; ++k) {
                const V3 x = X(xyz, p[k]);
                xv[k].x.v = x.x; xv[k].y.v = x.y; xv[k].z.v = x.z;
                xv[k].x.d[3 * k] = 1.0; xv[k].y.d[3 * k + 1] = 1.0; xv[k].z.d[3 * k + 2] = 1.0;
            }
            TetSide<DN<12>> ts[6];
            tet_sides(xv, ts);
            double g[12] = {};
            for (int k = 0; k < 6; ++k) {
                int32_t p1 = p[ts[k].a], p2 = p[ts[k].b];
                int32_t i1 = std::min(p1, p2), i2 = p1 + p2 - i1;
                const double sg = i1 != p1 ? -1.0 : 1.0;
                const int32_t e = sides.find(i1, i2);
                const double cb[3] = {sg * swb[e], sg * swb[E + e], sg * swb[2 * E + e]};
                const double vb = volb[p1 - 1] + volb[p2 - 1];
                for (int j = 0; j < 12; ++j)
                    g[j] += ((cb[0] * ts[k].coef.x.d[j] + cb[1] * ts[k].coef.y.d[j]) + cb[2] * ts[k].coef.z.d[j]) +
                            vb * ts[k].nv.d[j];
            }
            for (int k = 0; k < 4; ++k)
                for (int c = 0; c < 3; ++c) xb[(size_t)c * N + p[k] - 1] += g[3 * k + c];
        }
        for (int32_t f = 0; f < NF; ++f) {
            int32_t p[3];
            tri(f, p);
            V3T<DN<9>> xv[3];
            for (int k = 0; k < 3; ++k) {
                const V3 x = X(xyz, p[k]);
                xv[k].x.v = x.x; xv[k].y.v = x.y; xv[k].z.v = x.z;
                xv[k].x.d[3 * k] = 1.0; xv[k].y.d[3 * k + 1] = 1.0; xv[k].z.d[3 * k + 2] = 1.0;
            }
            TriSide<DN<9>> ts[3];
            tri_sides(xv, ts);
            double g[9] = {};
            for (int k = 0; k < 3; ++k) {
                const int32_t b = bsides.find(std::min(p[ts[k].a], p[ts[k].b]), std::max(p[ts[k].a], p[ts[k].b]));
                for (int j = 0; j < 9; ++j)
                    g[j] += (bwb[b] * ts[k].coef.x.d[j] + bwb[B + b] * ts[k].coef.y.d[j]) + bwb[2 * B + b] * ts[k].coef.z.d[j];
            }
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c) xb[(size_t)c * N + p[k] - 1] += g[3 * k + c];
        }
    }
};

template <class F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const fio::io_error &e) {
        g_err = e.what();
        return FLITE_EIO;
    } catch (const std::exception &e) {
        g_err = e.what();
        return FLITE_EINVAL;
    }
}

}  // namespace

// the indicator register (the layout of writeParallelComputationFiles
// gen3d_grid.f90:4548-4580), the node list per indicator and the normals
void fp_internal::build_register(LevelData &L) {
    int32_t r[21] = {0};
    auto R = [&](int i) -> int32_t & { return r[i + 20]; };
    for (int j = 0; j < L.Nb; ++j) {
        int ind = L.bnd_indicator[j];
        if (ind > 0) R(-21 + ind * 2) += 1;
    }
    R(-20) = 1;
    for (int j = -18; j <= -2; j += 2) {
        R(j + 1) = R(j + 1) + R(j - 1);
        R(j) = R(j - 1) + 1;
    }
    std::memcpy(L.reg, r, sizeof r);
    L.node_ind.clear();
    std::vector<double> nrm;
    for (int k = 1; k <= 9; ++k)
        for (int j = 0; j < L.Nb; ++j)
            if (L.bnd_indicator[j] == k) L.node_ind.push_back(j + 1);
    // normals written beside each node (not read by the solver): -sum w_b
    std::vector<double> acc(3 * (size_t)L.Nb, 0.0);
    for (int b = 0; b < L.B; ++b) {
        for (int s = 0; s < 2; ++s) {
            int n = L.bside[(size_t)s * L.B + b] - 1;
            for (int k = 0; k < 3; ++k) acc[3 * (size_t)n + k] -= L.bw[(size_t)k * L.B + b];
        }
    }
    size_t nn = L.node_ind.size();
    L.bnormal.assign(3 * nn, 0.0);
    for (size_t i = 0; i < nn; ++i) {
        int n = L.node_ind[i] - 1;
        double a = acc[3 * n], b = acc[3 * n + 1], c = acc[3 * n + 2];
        double s = std::sqrt(a * a + b * b + c * c);
        if (s > 1e-20) { a /= s; b /= s; c /= s; } else { a = b = c = 0; }
        L.bnormal[0 * nn + i] = a; L.bnormal[1 * nn + i] = b; L.bnormal[2 * nn + i] = c;
    }
}

// The canonical form of a mesh: level-1 nodes keep their numbers; every
// level's sides run from the smaller to the larger node (a reversed side's
// coefficients and GCL weights change sign) in node-pair order, and so do
// the boundary sides (a reversed one's two nodes swap their GCL weights);
// coarse nodes are numbered boundary nodes first, each class in the order
// of their first (smallest) child; seeds become the smallest level-1
// descendant and the wall-node numbers are dropped (the solver reads only
// the distances).  Values are moved, never recomputed, so the canonical
// forms of two orderings of one mesh are equal bit for bit.
void fp_internal::canonicalize(fp_mesh &M) {
    const size_t G = M.lv.size();
    for (size_t l = 0; l < G; ++l) {
        LevelData &L = M.lv[l];
        const int32_t N = L.N, E = L.E, B = L.B;
        std::vector<int32_t> newid(N);
        for (int32_t j = 0; j < N; ++j) newid[j] = j;
        if (l > 0) {
            std::vector<int32_t> first(N, INT32_MAX);
            const LevelData &F = M.lv[l - 1];
            for (int32_t f = 0; f < F.N; ++f) {
                const int32_t c = L.parent[f] - 1;
                first[c] = std::min(first[c], f);
            }
            std::vector<int32_t> order(N);
            for (int32_t j = 0; j < N; ++j) order[j] = j;
            std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
                const int ca = a >= L.Nb, cb = b >= L.Nb;
                return ca != cb ? ca < cb : first[a] < first[b];
            });
            for (int32_t k = 0; k < N; ++k) newid[order[k]] = k;
            auto perm_d = [&](std::vector<double> &v, int ncomp) {
                if (v.empty()) return;
                std::vector<double> o(v.size());
                for (int c = 0; c < ncomp; ++c)
                    for (int32_t j = 0; j < N; ++j) o[(size_t)c * N + newid[j]] = v[(size_t)c * N + j];
                v.swap(o);
            };
            perm_d(L.vol, 1); perm_d(L.wdist, 1); perm_d(L.volp, 1); perm_d(L.volp2, 1);
            std::vector<int32_t> bi(L.bnd_indicator.size());
            for (int32_t j = 0; j < L.Nb; ++j) bi[newid[j]] = L.bnd_indicator[j];
            L.bnd_indicator.swap(bi);
            for (auto &p : L.parent) p = newid[p - 1] + 1;
            // seeds: the smallest level-1 descendant
            L.seed.assign(N, INT32_MAX);
            for (int32_t f = 0; f < F.N; ++f) {
                const int32_t c = L.parent[f] - 1;
                const int32_t s1 = l == 1 ? f + 1 : F.seed[f];
                L.seed[c] = std::min(L.seed[c], s1);
            }
        }
        if (!L.wnode.empty()) std::fill(L.wnode.begin(), L.wnode.end(), 0);
        // the next level's arrays indexed by this level's nodes follow
        if (l + 1 < G && l > 0) {
            LevelData &C = M.lv[l + 1];
            std::vector<int32_t> par(C.parent.size());
            std::vector<double> rw(C.rweight.size());
            for (int32_t f = 0; f < N; ++f) { par[newid[f]] = C.parent[f]; rw[newid[f]] = C.rweight[f]; }
            C.parent.swap(par);
            C.rweight.swap(rw);
        }
        // sides
        {
            std::vector<int32_t> a(E), b(E), ord(E);
            std::vector<double> sg(E, 1.0);
            for (int32_t e = 0; e < E; ++e) {
                int32_t x = newid[L.side[e] - 1] + 1, y = newid[L.side[(size_t)E + e] - 1] + 1;
                if (x > y) { std::swap(x, y); sg[e] = -1.0; }
                a[e] = x; b[e] = y; ord[e] = e;
            }
            std::stable_sort(ord.begin(), ord.end(), [&](int32_t p, int32_t q) {
                return a[p] != a[q] ? a[p] < a[q] : b[p] < b[q];
            });
            std::vector<int32_t> side(2 * (size_t)E);
            std::vector<double> sw(3 * (size_t)E), slen(E), gcl(L.gcl.empty() ? 0 : 2 * (size_t)E);
            for (int32_t k = 0; k < E; ++k) {
                const int32_t e = ord[k];
                side[k] = a[e]; side[(size_t)E + k] = b[e];
                for (int c = 0; c < 3; ++c) sw[(size_t)c * E + k] = sg[e] * L.sw[(size_t)c * E + e];
                slen[k] = L.slen[e];
                if (!gcl.empty())
                    for (int c = 0; c < 2; ++c) gcl[(size_t)c * E + k] = sg[e] * L.gcl[(size_t)c * E + e];
            }
            L.side.swap(side); L.sw.swap(sw); L.slen.swap(slen); L.gcl.swap(gcl);
        }
        // boundary sides
        {
            std::vector<int32_t> a(B), b(B), ord(B);
            std::vector<char> sw(B, 0);
            for (int32_t q = 0; q < B; ++q) {
                int32_t x = newid[L.bside[q] - 1] + 1, y = newid[L.bside[(size_t)B + q] - 1] + 1;
                if (x > y) { std::swap(x, y); sw[q] = 1; }
                a[q] = x; b[q] = y; ord[q] = q;
            }
            std::stable_sort(ord.begin(), ord.end(), [&](int32_t p, int32_t q) {
                return a[p] != a[q] ? a[p] < a[q] : b[p] < b[q];
            });
            std::vector<int32_t> bside(3 * (size_t)B);
            std::vector<double> bw(3 * (size_t)B), bgcl(L.bgcl.empty() ? 0 : 4 * (size_t)B);
            for (int32_t k = 0; k < B; ++k) {
                const int32_t q = ord[k];
                bside[k] = a[q]; bside[(size_t)B + k] = b[q]; bside[2 * (size_t)B + k] = L.bside[2 * (size_t)B + q];
                for (int c = 0; c < 3; ++c) bw[(size_t)c * B + k] = L.bw[(size_t)c * B + q];
                if (!bgcl.empty()) {
                    const int from[4] = {sw[q] ? 1 : 0, sw[q] ? 0 : 1, sw[q] ? 3 : 2, sw[q] ? 2 : 3};
                    for (int c = 0; c < 4; ++c) bgcl[(size_t)c * B + k] = L.bgcl[(size_t)from[c] * B + q];
                }
            }
            L.bside.swap(bside); L.bw.swap(bw); L.bgcl.swap(bgcl);
        }
        // engine inlet sides, in node-pair order
        {
            const int32_t n = L.nes();
            std::vector<int32_t> a(n), b(n), ord(n);
            for (int32_t s = 0; s < n; ++s) {
                int32_t x = newid[L.eside[s] - 1] + 1, y = newid[L.eside[(size_t)n + s] - 1] + 1;
                a[s] = std::min(x, y); b[s] = std::max(x, y); ord[s] = s;
            }
            std::stable_sort(ord.begin(), ord.end(), [&](int32_t p, int32_t q) {
                return a[p] != a[q] ? a[p] < a[q] : b[p] < b[q];
            });
            std::vector<int32_t> es(3 * (size_t)n);
            std::vector<double> ew(3 * (size_t)n);
            for (int32_t k = 0; k < n; ++k) {
                const int32_t s = ord[k];
                es[k] = a[s]; es[(size_t)n + k] = b[s]; es[2 * (size_t)n + k] = L.eside[2 * (size_t)n + s];
                for (int c = 0; c < 3; ++c) ew[(size_t)c * n + k] = L.ew[(size_t)c * n + s];
            }
            L.eside.swap(es); L.ew.swap(ew);
        }
        build_register(L);
    }
    // the maps from finer to coarse sides of the canonical levels
    for (size_t l = 1; l < G; ++l) {
        const LevelData &F = M.lv[l - 1];
        LevelData &C = M.lv[l];
        std::map<std::pair<int32_t, int32_t>, int32_t> sid, bid;
        for (int32_t e = 0; e < C.E; ++e) sid[{C.side[e], C.side[(size_t)C.E + e]}] = e;
        for (int32_t q = 0; q < C.B; ++q) bid[{C.bside[q], C.bside[(size_t)C.B + q]}] = q;
        C.side_of.assign(F.E, 0);
        for (int32_t e = 0; e < F.E; ++e) {
            const int32_t c1 = C.parent[F.side[e] - 1], c2 = C.parent[F.side[(size_t)F.E + e] - 1];
            if (c1 == c2) continue;
            auto it = sid.find({std::min(c1, c2), std::max(c1, c2)});
            if (it == sid.end()) throw std::runtime_error("a side between two aggregates has no coarse side");
            C.side_of[e] = c1 < c2 ? it->second + 1 : -(it->second + 1);
        }
        C.bside_of.assign(F.B, 0);
        for (int32_t q = 0; q < F.B; ++q) {
            const int32_t c1 = C.parent[F.bside[q] - 1], c2 = C.parent[F.bside[(size_t)F.B + q] - 1];
            auto it = bid.find({std::min(c1, c2), std::max(c1, c2)});
            if (it == bid.end()) throw std::runtime_error("a boundary side has no coarse boundary side");
            C.bside_of[q] = c1 > c2 ? -(it->second + 1) : it->second + 1;
        }
    }
}


// ===========================================================================
extern "C" {

int fp_from_tets(int32_t nnodes, const double *xyz, int32_t ntet, const int32_t *tets,
                 int32_t ntri, const int32_t *tris, const int32_t *tri_ind, int nlevels,
                 fp_mesh **out) {
    return guarded([&] {
        if (!out || nnodes <= 0 || ntet <= 0 || ntri <= 0 || nlevels < 1) return FLITE_EINVAL;
        auto M = std::make_unique<fp_mesh>();
        std::vector<double> x(xyz, xyz + 3 * (size_t)nnodes);
        std::vector<int32_t> t(tets, tets + 4 * (size_t)ntet), f(tris, tris + 3 * (size_t)ntri),
            fi(tri_ind, tri_ind + ntri);
        for (auto v : t) if (v < 1 || v > nnodes) throw std::runtime_error("tet index out of range");
        for (auto v : f) if (v < 1 || v > nnodes) throw std::runtime_error("face index out of range");
        for (auto v : fi) if (v < 1 || v > 9) throw std::runtime_error("boundary indicator out of range");
        build_fine(*M, nnodes, x, std::move(t), std::move(f), fi);
        build_levels(*M, nlevels);
        *out = M.release();
        return FLITE_OK;
    });
}

int fp_from_elements(int32_t nnodes, const double *xyz, int32_t ntet, const int32_t *tets, int32_t npyr,
                     const int32_t *pyrs, int32_t npri, const int32_t *pris, int32_t nhex, const int32_t *hexes,
                     int32_t ntri, const int32_t *tris, const int32_t *tri_ind, int32_t nquad, const int32_t *quads,
                     const int32_t *quad_ind, int nlevels, fp_mesh **out) {
    return guarded([&] {
        if (!out || !xyz || nnodes <= 0 || nlevels < 1 || ntet < 0 || npyr < 0 || npri < 0 || nhex < 0 || ntri < 0 ||
            nquad < 0 || ntet + npyr + npri + nhex == 0 || ntri + nquad == 0)
            return FLITE_EINVAL;
        auto take = [&](const int32_t *a, int32_t n, int nv, const char *what) {
            if (n > 0 && !a) throw std::invalid_argument(std::string("missing ") + what);
            std::vector<int32_t> v(a ? a : nullptr, a ? a + (size_t)nv * n : nullptr);
            for (auto x : v)
                if (x < 1 || x > nnodes) throw std::runtime_error(std::string(what) + " index out of range");
            return v;
        };
        auto inds = [&](const int32_t *a, int32_t n) {
            if (n > 0 && !a) throw std::invalid_argument("missing boundary indicators");
            std::vector<int32_t> v(a ? a : nullptr, a ? a + n : nullptr);
            for (auto x : v)
                if (x < 1 || x > 9) throw std::runtime_error("boundary indicator out of range");
            return v;
        };
        auto M = std::make_unique<fp_mesh>();
        std::vector<double> x(xyz, xyz + 3 * (size_t)nnodes);
        Hybrid hy;
        hy.hex = take(hexes, nhex, 8, "hexahedron");
        hy.pri = take(pris, npri, 6, "prism");
        hy.pyr = take(pyrs, npyr, 5, "pyramid");
        hy.quad = take(quads, nquad, 4, "quadrilateral");
        hy.quad_ind = inds(quad_ind, nquad);
        build_fine(*M, nnodes, x, take(tets, ntet, 4, "tetrahedron"), take(tris, ntri, 3, "triangle"),
                   inds(tri_ind, ntri), std::move(hy));
        build_levels(*M, nlevels);
        *out = M.release();
        return FLITE_OK;
    });
}

int fp_bump_channel(int nx, int ny, int nz, double bump_h, int nlevels, fp_mesh **out) {
    return guarded([&] {
        if (nx < 1 || ny < 1 || nz < 1) return FLITE_EINVAL;
        const int32_t NX = nx + 1, NY = ny + 1, NZ = nz + 1;
        const int64_t N = (int64_t)NX * NY * NZ;
        if (N > 2000000000LL) return FLITE_EINVAL;
        auto id = [&](int i, int j, int k) { return (int32_t)(i + NX * (j + (int64_t)NY * k)) + 1; };
        std::vector<double> xyz(3 * (size_t)N);
        const double PI = 4.0 * std::atan(1.0);
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j)
                for (int i = 0; i < NX; ++i) {
                    double x = 3.0 * i / nx, y = (double)j / ny, s = (double)k / nz;
                    double hb = 0.0;
                    if (x >= 1.0 && x <= 2.0) { double sn = std::sin(PI * (x - 1.0)); hb = bump_h * sn * sn; }
                    double z = hb * (1.0 - s) + s;
                    size_t n = (size_t)id(i, j, k) - 1;
                    xyz[n] = x; xyz[(size_t)N + n] = y; xyz[2 * (size_t)N + n] = z;
                }
        // Kuhn split: 6 tets per hex along the main diagonal
        const int64_t NT = 6LL * nx * ny * nz;
        std::vector<int32_t> tets(4 * (size_t)NT);
        static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        size_t t = 0;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    for (int p = 0; p < 6; ++p) {
                        int c[3] = {i, j, k};
                        int32_t v[4];
                        v[0] = id(c[0], c[1], c[2]);
                        for (int s = 0; s < 3; ++s) { c[perm[p][s]] += 1; v[s + 1] = id(c[0], c[1], c[2]); }
                        for (int q = 0; q < 4; ++q) tets[(size_t)q * NT + t] = v[q];
                        ++t;
                    }
        // boundary triangles on the six faces, split along the diagonal of
        // the Kuhn tets that touch them
        std::vector<int32_t> tri, ind;
        auto quad = [&](int a, int lo, int i, int j, int k, int indicator) {
            // face normal to axis a at the low (lo=1) or high side of hex (i,j,k)
            int b = (a + 1) % 3, c = (a + 2) % 3;
            int base[3] = {i, j, k};
            if (!lo) base[a] += 1;
            int p0[3] = {base[0], base[1], base[2]};
            int pb[3] = {base[0], base[1], base[2]}; pb[b] += 1;
            int pc[3] = {base[0], base[1], base[2]}; pc[c] += 1;
            int pbc[3] = {base[0], base[1], base[2]}; pbc[b] += 1; pbc[c] += 1;
            int32_t v0 = id(p0[0], p0[1], p0[2]), vb = id(pb[0], pb[1], pb[2]);
            int32_t vc = id(pc[0], pc[1], pc[2]), vbc = id(pbc[0], pbc[1], pbc[2]);
            tri.push_back(v0); tri.push_back(vb); tri.push_back(vbc); ind.push_back(indicator);
            tri.push_back(v0); tri.push_back(vc); tri.push_back(vbc); ind.push_back(indicator);
        };
        for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) {
            quad(0, 1, 0, j, k, 3); quad(0, 0, nx - 1, j, k, 3);
        }
        for (int k = 0; k < nz; ++k) for (int i = 0; i < nx; ++i) {
            quad(1, 1, i, 0, k, 2); quad(1, 0, i, ny - 1, k, 2);
        }
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
            quad(2, 1, i, j, 0, 1); quad(2, 0, i, j, nz - 1, 2);
        }
        const size_t NF = ind.size();
        std::vector<int32_t> tris(3 * NF);
        for (size_t f = 0; f < NF; ++f)
            for (int q = 0; q < 3; ++q) tris[q * NF + f] = tri[3 * f + q];
        auto M = std::make_unique<fp_mesh>();
        build_fine(*M, (int32_t)N, xyz, std::move(tets), std::move(tris), ind);
        build_levels(*M, nlevels);
        *out = M.release();
        return FLITE_OK;
    });
}

// Extruded NACA0012 O-grid (the RANS configuration's geometry): ni points
// around the section (cosine-clustered at the leading and trailing edges, the
// standard 4-digit thickness law with its open trailing edge), nj cells from
// the wall to a circular far field of radius `farfield` chords about x = 0.5
// (nlayer layers from first_cell with ratio `growth`, then a geometric
// stretching whose ratio makes the lines end on the circle), nk cells over
// the span.  Hexes are split into 6 tets as in the bump channel (periodic
// around the section).  Indicators: wall 1, span ends 2 (symmetry), far
// field 3.
int fp_naca0012(int ni, int nj, int nk, double first_cell, double growth, int nlayer, double farfield, double span,
                int nlevels, fp_mesh **out) {
    return guarded([&] {
        if (ni < 8 || nj < 2 || nk < 1 || !(first_cell > 0) || !(growth >= 1) || nlayer < 0 || nlayer >= nj ||
            !(farfield > 1) || !(span > 0))
            return FLITE_EINVAL;
        const int32_t NJ = nj + 1, NK = nk + 1;
        const int64_t N = (int64_t)ni * NJ * NK;
        if (N > 2000000000LL) return FLITE_EINVAL;
        auto id = [&](int i, int j, int k) { return (int32_t)((i % ni) + ni * (j + (int64_t)NJ * k)) + 1; };
        const double PI = 4.0 * std::atan(1.0);
        // radial distances along each line, as a fraction of its length:
        // fixed cells near the wall, then a ratio q found by bisection
        auto yt = [](double x) {
            return 0.6 * ((((0.2969 * std::sqrt(x) - 0.1260 * x) - 0.3516 * x * x) + 0.2843 * x * x * x) -
                          0.1015 * x * x * x * x);
        };
        std::vector<double> sx(ni), sy(ni), cx(ni), cy(ni), len(ni);
        for (int i = 0; i < ni; ++i) {
            const double th = 2.0 * PI * i / ni;
            const double x = 0.5 * (1.0 + std::cos(th));
            sx[i] = x;
            sy[i] = (th <= PI ? 1.0 : -1.0) * yt(x);
            cx[i] = 0.5 + farfield * std::cos(th);
            cy[i] = farfield * std::sin(th);
            len[i] = std::hypot(cx[i] - sx[i], cy[i] - sy[i]);
        }
        double Lmin = len[0];
        for (double v : len) Lmin = std::min(Lmin, v);
        std::vector<double> d(NJ, 0.0);  // distances for the shortest line
        for (int j = 1; j <= nlayer; ++j) d[j] = d[j - 1] + first_cell * std::pow(growth, j - 1);
        const double rest = Lmin - d[nlayer];
        const double h0 = first_cell * std::pow(growth, nlayer);
        const int m = nj - nlayer;
        if (!(rest > h0 * m * 0.5)) throw std::runtime_error("far field too close for the wall layers");
        double lo = 1.0, hi = 2.0;
        auto total = [&](double q) { return q == 1.0 ? h0 * m : h0 * (std::pow(q, m) - 1.0) / (q - 1.0); };
        while (total(hi) < rest) hi *= 2.0;
        for (int it = 0; it < 200; ++it) {
            const double q = 0.5 * (lo + hi);
            (total(q) < rest ? lo : hi) = q;
        }
        const double q = 0.5 * (lo + hi);
        for (int j = nlayer + 1; j <= nj; ++j) d[j] = d[j - 1] + h0 * std::pow(q, j - nlayer - 1);
        std::vector<double> xyz(3 * (size_t)N);
        for (int k = 0; k < NK; ++k)
            for (int j = 0; j < NJ; ++j)
                for (int i = 0; i < ni; ++i) {
                    const double f = d[j] / d[nj];  // the same fraction on every line
                    const size_t n = (size_t)id(i, j, k) - 1;
                    xyz[n] = sx[i] + f * (cx[i] - sx[i]);
                    xyz[(size_t)N + n] = sy[i] + f * (cy[i] - sy[i]);
                    xyz[2 * (size_t)N + n] = span * k / nk;
                }
        const int64_t NT = 6LL * ni * nj * nk;
        std::vector<int32_t> tets(4 * (size_t)NT);
        static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        size_t t = 0;
        for (int k = 0; k < nk; ++k)
            for (int j = 0; j < nj; ++j)
                for (int i = 0; i < ni; ++i)
                    for (int p = 0; p < 6; ++p) {
                        int c[3] = {i, j, k};
                        int32_t v[4];
                        v[0] = id(c[0], c[1], c[2]);
                        for (int r = 0; r < 3; ++r) { c[perm[p][r]] += 1; v[r + 1] = id(c[0], c[1], c[2]); }
                        for (int qq = 0; qq < 4; ++qq) tets[(size_t)qq * NT + t] = v[qq];
                        ++t;
                    }
        std::vector<int32_t> tri, ind;
        auto quad = [&](int a, int lo_side, int i, int j, int k, int indicator) {
            int b = (a + 1) % 3, c = (a + 2) % 3;
            int base[3] = {i, j, k};
            if (!lo_side) base[a] += 1;
            int pb[3] = {base[0], base[1], base[2]}; pb[b] += 1;
            int pc[3] = {base[0], base[1], base[2]}; pc[c] += 1;
            int pbc[3] = {base[0], base[1], base[2]}; pbc[b] += 1; pbc[c] += 1;
            int32_t v0 = id(base[0], base[1], base[2]), vb = id(pb[0], pb[1], pb[2]);
            int32_t vc = id(pc[0], pc[1], pc[2]), vbc = id(pbc[0], pbc[1], pbc[2]);
            tri.push_back(v0); tri.push_back(vb); tri.push_back(vbc); ind.push_back(indicator);
            tri.push_back(v0); tri.push_back(vc); tri.push_back(vbc); ind.push_back(indicator);
        };
        for (int k = 0; k < nk; ++k)
            for (int i = 0; i < ni; ++i) {
                quad(1, 1, i, 0, k, 1);       // wall
                quad(1, 0, i, nj - 1, k, 3);  // far field
            }
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                quad(2, 1, i, j, 0, 2);
                quad(2, 0, i, j, nk - 1, 2);
            }
        const size_t NF = ind.size();
        std::vector<int32_t> tris(3 * NF);
        for (size_t f = 0; f < NF; ++f)
            for (int qq = 0; qq < 3; ++qq) tris[qq * NF + f] = tri[3 * f + qq];
        auto M = std::make_unique<fp_mesh>();
        build_fine(*M, (int32_t)N, xyz, std::move(tets), std::move(tris), ind);
        build_levels(*M, nlevels);
        *out = M.release();
        return FLITE_OK;
    });
}

int fp_free(fp_mesh *m) { delete m; return FLITE_OK; }

int fp_num_levels(const fp_mesh *m) { return m ? (int)m->lv.size() : 0; }

int fp_level_desc(const fp_mesh *m, int level, flite_level_desc *o) {
    if (!m || !o || level < 1 || level > (int)m->lv.size()) return FLITE_EINVAL;
    const LevelData &L = m->lv[level - 1];
    std::memset(o, 0, sizeof *o);
    o->n_nodes = L.N; o->n_sides = L.E; o->n_bsides = L.B; o->n_bnodes = L.Nb;
    o->n_normals = (int32_t)L.node_ind.size();
    o->side_idx = L.side.data(); o->side_w = L.sw.data(); o->side_len = L.slen.data();
    o->bnd_idx = L.bside.data(); o->bnd_w = L.bw.data();
    o->node_reg = L.reg; o->node_ind = L.node_ind.data();
    o->volume = L.vol.data(); o->wall_dist = L.wdist.data();
    o->coords = L.xyz.empty() ? nullptr : L.xyz.data();
    o->coord_move = L.cmove.empty() ? nullptr : L.cmove.data();
    o->side_gcl = L.gcl.empty() ? nullptr : L.gcl.data();
    o->bnd_gcl = L.bgcl.empty() ? nullptr : L.bgcl.data();
    o->volume_prev = L.volp.empty() || level > 1 ? nullptr : L.volp.data();
    o->volume_prev2 = L.volp2.empty() || level > 1 ? nullptr : L.volp2.data();
    o->parent = L.parent.empty() ? nullptr : L.parent.data();
    o->rweight = L.rweight.empty() ? nullptr : L.rweight.data();
    o->n_engine_sides = L.nes();
    o->engine_idx = L.eside.empty() ? nullptr : L.eside.data();
    o->engine_w = L.ew.empty() ? nullptr : L.ew.data();
    return FLITE_OK;
}

int fp_node_perm(const fp_mesh *m, int32_t *perm) {
    if (!m || !perm || m->perm.empty()) return FLITE_EINVAL;
    std::memcpy(perm, m->perm.data(), m->perm.size() * 4);
    return FLITE_OK;
}

int fp_geometry(const fp_mesh *m, const double *xyz, double *side_w, double *bnd_w, double *volume) {
    if (!m || m->lv.empty() || (m->tets.empty() && !m->hybrid()) || !side_w || !bnd_w || !volume) return FLITE_EINVAL;
    return guarded([&] {
        Geometry G(*m);
        G.eval(xyz ? xyz : m->lv[0].xyz.data(), side_w, bnd_w, volume);
        return FLITE_OK;
    });
}

int fp_geometry_vjp(const fp_mesh *m, const double *xyz, const double *side_w_bar, const double *bnd_w_bar,
                    const double *volume_bar, double *xyz_bar) {
    if (!m || m->lv.empty() || m->tets.empty() || !side_w_bar || !bnd_w_bar || !volume_bar || !xyz_bar)
        return FLITE_EINVAL;
    return guarded([&] {
        Geometry G(*m);
        G.vjp(xyz ? xyz : m->lv[0].xyz.data(), side_w_bar, bnd_w_bar, volume_bar, xyz_bar);
        return FLITE_OK;
    });
}

int fp_coordinate_movement(fp_mesh *m, int32_t time_scheme) {
    if (!m || m->lv.empty() || (time_scheme != 1 && time_scheme != 2)) return FLITE_EINVAL;
    LevelData &L = m->lv[0];
    if (L.xyz.empty() || L.xyzp.size() != L.xyz.size() || L.xyzp2.size() != L.xyz.size()) return FLITE_EINVAL;
    // readGridComputationData (def_par:13896-13900)
    L.cmove.resize(L.xyz.size());
    for (size_t k = 0; k < L.xyz.size(); ++k)
        L.cmove[k] = time_scheme == 1 ? L.xyz[k] - L.xyzp[k]
                                      : (1.5 * L.xyz[k] - 2.0 * L.xyzp[k]) + 0.5 * L.xyzp2[k];
    return FLITE_OK;
}

int fp_set_moving_geometry(fp_mesh *m, const double *xyz, const double *xyz_prev, const double *xyz_prev2,
                           int32_t time_scheme) {
    if (!m || m->lv.empty() || (m->tets.empty() && !m->hybrid()) || !xyz || !xyz_prev || !xyz_prev2 ||
        (time_scheme != 1 && time_scheme != 2))
        return FLITE_EINVAL;
    // the engine inlet sides would need the step's coordinates too; the
    // solver takes no engine conditions on a moving mesh
    if (m->lv[0].nes() > 0) return FLITE_EUNSUPPORTED;
    return guarded([&] {
        LevelData &L = m->lv[0];
        const size_t N = L.N, E = L.E, B = L.B;
        std::vector<double> sw(3 * E), bw(3 * B), vol(N), volp(N), volp2(N), gcl(2 * E), bgcl(4 * B);
        {
            Geometry G(*m);
            const double *x[3] = {xyz, xyz_prev, xyz_prev2};
            G.eval_moving(x, sw.data(), bw.data(), vol.data(), volp.data(), volp2.data(), gcl.data(), bgcl.data());
        }
        L.sw = std::move(sw); L.bw = std::move(bw); L.vol = std::move(vol);
        L.volp = std::move(volp); L.volp2 = std::move(volp2); L.gcl = std::move(gcl); L.bgcl = std::move(bgcl);
        L.xyz.assign(xyz, xyz + 3 * N);
        L.xyzp.assign(xyz_prev, xyz_prev + 3 * N);
        L.xyzp2.assign(xyz_prev2, xyz_prev2 + 3 * N);
        // side lengths at the step's coordinates (registerSideGCL's
        // sideLength; |x2 - x1| does not depend on the side's direction)
        for (size_t e = 0; e < E; ++e) {
            const int32_t a = L.side[e] - 1, b = L.side[E + e] - 1;
            const double dx = L.xyz[b] - L.xyz[a], dy = L.xyz[N + b] - L.xyz[N + a];
            const double dz = L.xyz[2 * N + b] - L.xyz[2 * N + a];
            L.slen[e] = std::sqrt(dx * dx + dy * dy + dz * dz);
        }
        int rc = fp_coordinate_movement(m, time_scheme);
        if (rc != FLITE_OK) return rc;
        // coarse levels: the finer level's arrays summed through the
        // agglomeration, in the order agglomerate sums the static ones
        for (size_t l = 1; l < m->lv.size(); ++l) {
            const LevelData &F = m->lv[l - 1];
            LevelData &C = m->lv[l];
            const size_t Nf = F.N, Ef = F.E, Bf = F.B, Nc = C.N, Ec = C.E, Bc = C.B;
            C.vol.assign(Nc, 0.0); C.volp.assign(Nc, 0.0); C.volp2.assign(Nc, 0.0);
            for (size_t i = 0; i < Nf; ++i) {
                const int32_t c = C.parent[i] - 1;
                C.vol[c] += F.vol[i]; C.volp[c] += F.volp[i]; C.volp2[c] += F.volp2[i];
            }
            for (size_t i = 0; i < Nf; ++i) C.rweight[i] = F.vol[i] / C.vol[C.parent[i] - 1];
            C.sw.assign(3 * Ec, 0.0); C.gcl.assign(2 * Ec, 0.0);
            std::vector<char> seen(Ec, 0);
            for (size_t e = 0; e < Ef; ++e) {
                const int32_t so = C.side_of[e];
                if (so == 0) continue;
                const size_t id = (size_t)std::abs(so) - 1;
                const double sg = so < 0 ? -1.0 : 1.0;
                for (int k = 0; k < 3; ++k) C.sw[k * Ec + id] = C.sw[k * Ec + id] + sg * F.sw[k * Ef + e];
                for (int k = 0; k < 2; ++k) C.gcl[k * Ec + id] = C.gcl[k * Ec + id] + sg * F.gcl[k * Ef + e];
                if (!seen[id]) { seen[id] = 1; C.slen[id] = F.slen[e]; }
            }
            C.bw.assign(3 * Bc, 0.0); C.bgcl.assign(4 * Bc, 0.0);
            for (size_t b = 0; b < Bf; ++b) {
                const int32_t so = C.bside_of[b];
                const size_t id = (size_t)std::abs(so) - 1;
                for (int k = 0; k < 3; ++k) C.bw[k * Bc + id] = C.bw[k * Bc + id] + F.bw[k * Bf + b];
                // the weights stay with their nodes when the coarse side's
                // nodes come in the other order
                const int sw1 = so < 0 ? 1 : 0;
                const int from[4] = {sw1, 1 - sw1, 2 + sw1, 3 - sw1};
                for (int k = 0; k < 4; ++k)
                    C.bgcl[k * Bc + id] = C.bgcl[k * Bc + id] + F.bgcl[from[k] * Bf + b];
            }
        }
        return FLITE_OK;
    });
}

int fp_gcl_check(const fp_mesh *m, int level, int32_t time_scheme, double *err, double *scale) {
    if (!m || level < 1 || level > (int)m->lv.size() || (time_scheme != 1 && time_scheme != 2) || !err || !scale)
        return FLITE_EINVAL;
    const LevelData &L = m->lv[level - 1];
    if (L.gcl.empty() || L.volp.empty()) return FLITE_EINVAL;
    const size_t N = L.N, E = L.E, B = L.B;
    // the GCL weights as the solver's reader takes them (def_par:816-818,
    // 13858-13860) and the sums of def_par:14590-14610
    auto comb = [&](double g, double gp) { return time_scheme == 2 ? 1.5 * g - 0.5 * gp : g; };
    std::vector<double> d(N, 0.0);
    for (size_t e = 0; e < E; ++e) {
        const double ww = comb(L.gcl[e], L.gcl[E + e]);
        d[L.side[e] - 1] = d[L.side[e] - 1] + 2.0 * ww;
        d[L.side[E + e] - 1] = d[L.side[E + e] - 1] - 2.0 * ww;
    }
    for (size_t b = 0; b < B; ++b) {
        d[L.bside[b] - 1] = d[L.bside[b] - 1] + 4.0 * comb(L.bgcl[b], L.bgcl[2 * B + b]);
        d[L.bside[B + b] - 1] = d[L.bside[B + b] - 1] + 4.0 * comb(L.bgcl[B + b], L.bgcl[3 * B + b]);
    }
    double e_max = 0, s_max = 0;
    for (size_t i = 0; i < N; ++i) {
        const double dv = time_scheme == 1 ? L.vol[i] - L.volp[i]
                                           : (1.5 * L.vol[i] - 2.0 * L.volp[i]) + 0.5 * L.volp2[i];
        e_max = std::max(e_max, std::fabs(d[i] - dv));
        s_max = std::max(s_max, std::fabs(dv));
    }
    *err = e_max;
    *scale = s_max;
    return FLITE_OK;
}

int fp_canonical(const fp_mesh *m, fp_mesh **out) {
    if (!m || !out) return FLITE_EINVAL;
    *out = nullptr;
    return guarded([&] {
        auto c = std::make_unique<fp_mesh>(*m);
        fp_internal::canonicalize(*c);
        *out = c.release();
        return FLITE_OK;
    });
}

int fp_check(const fp_mesh *m, int level, double *closure, double *volume) {
    if (!m || level < 1 || level > (int)m->lv.size()) return FLITE_EINVAL;
    const LevelData &L = m->lv[level - 1];
    // closure of def_par:14430-14568: sum_j +-w + 2 sum_b w_b per node
    std::vector<double> chk(3 * (size_t)L.N, 0.0);
    double wmax = 0;
    for (int32_t e = 0; e < L.E; ++e) {
        int32_t a = L.side[e] - 1, b = L.side[(size_t)L.E + e] - 1;
        for (int k = 0; k < 3; ++k) {
            double w = L.sw[(size_t)k * L.E + e];
            chk[3 * (size_t)a + k] += w; chk[3 * (size_t)b + k] -= w;
            wmax = std::max(wmax, std::fabs(w));
        }
    }
    for (int32_t e = 0; e < L.B; ++e) {
        int32_t a = L.bside[e] - 1, b = L.bside[(size_t)L.B + e] - 1;
        for (int k = 0; k < 3; ++k) {
            double w = L.bw[(size_t)k * L.B + e];
            chk[3 * (size_t)a + k] += 2 * w; chk[3 * (size_t)b + k] += 2 * w;
        }
    }
    double mx = 0;
    for (double v : chk) mx = std::max(mx, std::fabs(v));
    if (closure) *closure = wmax > 0 ? mx / wmax : mx;
    double vs = 0;
    for (double v : L.vol) vs += v;
    if (volume) *volume = vs;
    return FLITE_OK;
}

// ---- .sol: the record sequence read by readComputationData (mg_par:
// 1210-1266) and readGridComputationData (def_par:13837-14074) ------------
int fp_write_sol(const fp_mesh *m, const char *path) {
    if (!m || !path) return FLITE_EINVAL;
    return guarded([&] {
        fio::Writer w(path);
        w.i4((int32_t)m->lv.size()).end();
        w.i4(1).i4(1).end();  // domain, numberOfGridDomains
        for (size_t l = 0; l < m->lv.size(); ++l) {
            const LevelData &L = m->lv[l];
            const bool fine = l == 0;
            // readBoundarySolverData (def_par:803-864)
            w.i4(L.B).end();
            for (int32_t b = 0; b < L.B; ++b) {
                w.i4(L.bside[b]).i4(L.bside[(size_t)L.B + b]).i4(L.bside[2 * (size_t)L.B + b]);
                w.r8(L.bw[b]).r8(L.bw[(size_t)L.B + b]).r8(L.bw[2 * (size_t)L.B + b]);
                if (L.bgcl.empty()) {
                    w.r8(0).r8(0).r8(0).r8(0).end();  // GCL(2), GCLprev(2): static mesh
                } else {
                    for (int k = 0; k < 4; ++k) w.r8(L.bgcl[(size_t)k * L.B + b]);
                    w.end();
                }
            }
            const int32_t nn = (int32_t)L.node_ind.size();
            w.i4(L.Nb).i4(nn).end();
            for (int j = 0; j < 21; ++j) w.i4(L.reg[j]).end();
            for (int32_t i = 0; i < nn; ++i)
                w.i4(L.node_ind[i]).r8(L.bnormal[i]).r8(L.bnormal[(size_t)nn + i])
                    .r8(L.bnormal[2 * (size_t)nn + i]).end();
            // engine inlet sides (def_par:852-864)
            const int32_t ne = L.nes();
            w.i4(ne).end();
            for (int32_t s = 0; s < ne; ++s)
                w.i4(L.eside[s]).i4(L.eside[(size_t)ne + s]).i4(L.eside[2 * (size_t)ne + s])
                    .r8(L.ew[s]).r8(L.ew[(size_t)ne + s]).r8(L.ew[2 * (size_t)ne + s]).end();
            // sides
            w.i4(L.E).end();
            for (int32_t e = 0; e < L.E; ++e) {
                w.i4(L.side[e]).i4(L.side[(size_t)L.E + e]);
                w.r8(L.sw[e]).r8(L.sw[(size_t)L.E + e]).r8(L.sw[2 * (size_t)L.E + e]);
                if (L.gcl.empty()) w.r8(0).r8(0);
                else w.r8(L.gcl[e]).r8(L.gcl[(size_t)L.E + e]);
                w.r8(L.slen[e]).end();
            }
            // nodes
            w.i4(L.N).end();
            if (fine) {
                for (int32_t i = 0; i < L.N; ++i) {
                    // a static mesh's previous volumes and coordinates are its own
                    const bool mv = !L.volp.empty() && !L.xyzp.empty();
                    const std::vector<double> &xp = mv ? L.xyzp : L.xyz, &xp2 = mv ? L.xyzp2 : L.xyz;
                    w.i4(i + 1).r8(L.vol[i]).r8(mv ? L.volp[i] : L.vol[i]).r8(mv ? L.volp2[i] : L.vol[i]);
                    w.r8(L.wdist[i]).i4(L.wnode[i]);
                    for (const std::vector<double> *x : {&L.xyz, &xp, &xp2})
                        w.r8((*x)[i]).r8((*x)[(size_t)L.N + i]).r8((*x)[2 * (size_t)L.N + i]);
                    w.end();
                }
                w.i4(0).end();  // trip nodes
                w.i4(0).end();  // trip field nodes
            } else {
                for (int32_t i = 0; i < L.N; ++i)
                    w.i4(i + 1).r8(L.vol[i]).r8(L.wdist[i]).i4(L.wnode[i]).i4(L.seed[i]).end();
            }
            // parallel data, one process (def_par:667-683)
            w.i4(0).i4(0).end();
            w.i4(0).end();
            w.i4(0).end();
            if (!fine) {
                const int32_t nf = (int32_t)L.parent.size();
                // prolongation (def_par:455-482)
                w.i4(nf).end();
                w.i4(L.N).end();
                for (int32_t i = 0; i < nf; ++i) w.i4(i + 1).i4(L.parent[i]).end();
                w.i4(0).end();
                // restriction (def_par:517-540)
                w.i4(nf).end();
                w.i4(L.N).end();
                for (int32_t i = 0; i < nf; ++i) w.i4(i + 1).r8(L.rweight[i]).end();
                w.i4(0).end();
                // com-parallel (def_par:703-737)
                w.i4(0).end();
                w.i4(0).end();
                w.i4(0).end();
                w.i4(0).end();
            }
        }
        w.close();
        return FLITE_OK;
    });
}

int fp_read_sol(const char *path, fp_mesh **out) {
    if (!path || !out) return FLITE_EINVAL;
    return guarded([&] {
        fio::Reader r(path);
        auto M = std::make_unique<fp_mesh>();
        r.next(); int32_t ng = r.i4();
        r.next(); int32_t dom = r.i4(), ndom = r.i4();
        (void)dom;
        if (ndom != 1) throw std::runtime_error("multi-domain .sol is not supported (one GPU, one domain)");
        if (ng < 1 || ng > 32) throw fio::io_error("bad number of grids");
        for (int32_t l = 0; l < ng; ++l) {
            LevelData L;
            const bool fine = l == 0;
            r.next(); L.B = r.i4();
            if (L.B < 0) throw fio::io_error("negative count");
            L.bside.resize(3 * (size_t)L.B); L.bw.resize(3 * (size_t)L.B); L.bgcl.assign(4 * (size_t)L.B, 0.0);
            for (int32_t b = 0; b < L.B; ++b) {
                r.next();
                for (int k = 0; k < 3; ++k) L.bside[(size_t)k * L.B + b] = r.i4();
                for (int k = 0; k < 3; ++k) L.bw[(size_t)k * L.B + b] = r.r8();
                if (r.remaining() >= 32)
                    for (int k = 0; k < 4; ++k) L.bgcl[(size_t)k * L.B + b] = r.r8();
            }
            r.next(); L.Nb = r.i4(); int32_t nn = r.i4();
            for (int j = 0; j < 21; ++j) { r.next(); L.reg[j] = r.i4(); }
            L.node_ind.resize(nn); L.bnormal.assign(3 * (size_t)nn, 0.0);
            for (int32_t i = 0; i < nn; ++i) {
                r.next(); L.node_ind[i] = r.i4();
                if (r.remaining() >= 24)
                    for (int k = 0; k < 3; ++k) L.bnormal[(size_t)k * nn + i] = r.r8();
            }
            r.next(); const int32_t neis = r.i4();
            if (neis < 0) throw std::runtime_error("negative engine inlet side count");
            L.eside.resize(3 * (size_t)neis); L.ew.resize(3 * (size_t)neis);
            for (int32_t s = 0; s < neis; ++s) {
                r.next();
                for (int k = 0; k < 3; ++k) L.eside[(size_t)k * neis + s] = r.i4();
                for (int k = 0; k < 3; ++k) L.ew[(size_t)k * neis + s] = r.r8();
            }
            r.next(); L.E = r.i4();
            L.side.resize(2 * (size_t)L.E); L.sw.resize(3 * (size_t)L.E); L.slen.resize(L.E);
            L.gcl.resize(2 * (size_t)L.E);
            for (int32_t e = 0; e < L.E; ++e) {
                r.next();
                L.side[e] = r.i4(); L.side[(size_t)L.E + e] = r.i4();
                for (int k = 0; k < 3; ++k) L.sw[(size_t)k * L.E + e] = r.r8();
                L.gcl[e] = r.r8(); L.gcl[(size_t)L.E + e] = r.r8();
                L.slen[e] = r.r8();
            }
            r.next(); L.N = r.i4();
            for (int32_t s = 0; s < neis; ++s) {
                const int32_t a = L.eside[s], b = L.eside[(size_t)neis + s], in = L.eside[2 * (size_t)neis + s];
                if (a < 1 || a > L.N || b < 1 || b > L.N || in < 1 || in > 2)
                    throw fio::io_error("bad engine inlet side record");
            }
            L.vol.resize(L.N); L.wdist.resize(L.N); L.wnode.resize(L.N);
            if (fine) {
                L.xyz.resize(3 * (size_t)L.N); L.xyzp.resize(3 * (size_t)L.N); L.xyzp2.resize(3 * (size_t)L.N);
                L.volp.resize(L.N); L.volp2.resize(L.N);
                for (int32_t i = 0; i < L.N; ++i) {
                    r.next();
                    int32_t id = r.i4();
                    if (id < 1 || id > L.N) throw fio::io_error("node id out of range");
                    --id;
                    L.vol[id] = r.r8(); L.volp[id] = r.r8(); L.volp2[id] = r.r8();
                    L.wdist[id] = r.r8(); L.wnode[id] = r.i4();
                    for (std::vector<double> *x : {&L.xyz, &L.xyzp, &L.xyzp2})
                        for (int k = 0; k < 3; ++k) (*x)[(size_t)k * L.N + id] = r.r8();
                }
                r.next(); int32_t ntrip = r.i4();
                for (int32_t i = 0; i < ntrip; ++i) r.next();
                r.next(); int32_t ntf = r.i4();
                for (int32_t i = 0; i < ntf; ++i) r.next();
            } else {
                L.seed.resize(L.N);
                for (int32_t i = 0; i < L.N; ++i) {
                    r.next();
                    int32_t id = r.i4();
                    if (id < 1 || id > L.N) throw fio::io_error("node id out of range");
                    --id;
                    L.vol[id] = r.r8(); L.wdist[id] = r.r8(); L.wnode[id] = r.i4();
                    L.seed[i] = r.i4();
                }
            }
            r.next(); r.i4(); r.i4();
            r.next(); r.i4();
            r.next(); r.i4();
            if (!fine) {
                const int32_t nfine = M->lv.back().N;
                L.parent.assign(nfine, 0); L.rweight.assign(nfine, 0.0);
                r.next(); int32_t nif = r.i4();
                r.next(); r.i4();
                for (int32_t i = 0; i < nif; ++i) {
                    r.next(); int32_t f = r.i4(); int32_t p = r.i4();
                    if (f < 1 || f > nfine || p < 1 || p > L.N) throw fio::io_error("bad prolongation record");
                    L.parent[f - 1] = p;
                }
                r.next(); int32_t ncom = r.i4();
                for (int32_t i = 0; i < ncom; ++i) r.next();
                r.next(); nif = r.i4();
                r.next(); r.i4();
                for (int32_t i = 0; i < nif; ++i) {
                    r.next(); int32_t f = r.i4(); double wv = r.r8();
                    if (f < 1 || f > nfine) throw fio::io_error("bad restriction record");
                    L.rweight[f - 1] = wv;
                }
                r.next(); ncom = r.i4();
                for (int32_t i = 0; i < ncom; ++i) r.next();
                for (int s = 0; s < 2; ++s) {
                    r.next(); r.i4();  // numberOfComS/RNodes
                    r.next(); int32_t cnt = r.i4();
                    for (int32_t i = 0; i < cnt; ++i) r.next();
                }
            }
            // indicators per boundary node from the register
            L.bnd_indicator.assign(L.Nb, 0);
            for (int k = 1; k <= 9; ++k) {
                int32_t st = L.reg[(-20 + 2 * (k - 1)) + 20], en = L.reg[(-19 + 2 * (k - 1)) + 20];
                for (int32_t ib = st; ib <= en; ++ib)
                    if (ib >= 1 && ib <= nn) {
                        int32_t n = L.node_ind[ib - 1];
                        if (n >= 1 && n <= L.Nb) L.bnd_indicator[n - 1] = k;
                    }
            }
            M->lv.push_back(std::move(L));
        }
        M->perm.resize(M->lv[0].N);
        for (int32_t i = 0; i < M->lv[0].N; ++i) M->perm[i] = i + 1;
        *out = M.release();
        return FLITE_OK;
    });
}

int fp_write_rst(const char *path, int32_t n, int nvar, const double *prim) {
    if (!path || n <= 0 || nvar < 5 || !prim) return FLITE_EINVAL;
    return guarded([&] {
        fio::Writer w(path);
        w.i4(n).end();
        w.r8s(prim, (size_t)n * nvar).end();
        w.close();
        return FLITE_OK;
    });
}

int fp_read_rst(const char *path, int32_t n, int nvar, double *prim) {
    if (!path || n <= 0 || nvar < 5 || !prim) return FLITE_EINVAL;
    return guarded([&] {
        fio::Reader r(path);
        r.next();
        int32_t num = r.i4();
        if (num != n) throw fio::io_error("Startup file is not compatible");  // def_par:3748
        r.next();
        if (r.remaining() < (size_t)n * nvar * 8) throw fio::io_error("restart record too short");
        r.r8s(prim, (size_t)n * nvar);
        return FLITE_OK;
    });
}

int fp_write_res(const char *path, int32_t n, int nvar, const double *u) {
    if (!path || n <= 0 || nvar < 5 || !u) return FLITE_EINVAL;
    return guarded([&] {
        fio::Writer w(path);
        w.i4(n).end();
        std::vector<double> col((size_t)n * nvar);
        for (int32_t i = 0; i < n; ++i) col[i] = u[i];
        for (int j = 1; j < nvar; ++j)
            for (int32_t i = 0; i < n; ++i) col[(size_t)j * n + i] = u[(size_t)j * n + i] / u[i];
        w.r8s(col.data(), col.size()).end();
        w.close();
        return FLITE_OK;
    });
}

int fp_write_unk(const char *path, int32_t n, int nvar, const double *u) {
    if (!path || n <= 0 || nvar < 1 || !u) return FLITE_EINVAL;
    return guarded([&] {
        fio::Writer w(path);
        w.i4(n).end();
        w.r8s(u, (size_t)n * nvar).end();
        w.close();
        return FLITE_OK;
    });
}

int fp_read_unk(const char *path, int32_t n, int nvar, double *u) {
    if (!path || n <= 0 || nvar < 1 || !u) return FLITE_EINVAL;
    return guarded([&] {
        fio::Reader r(path);
        r.next();
        if (r.i4() != n) throw fio::io_error("node count differs");
        r.next();
        if (r.remaining() < (size_t)n * nvar * 8) throw fio::io_error("unk record too short");
        r.r8s(u, (size_t)n * nvar);
        return FLITE_OK;
    });
}

int fp_write_plotreg(const fp_mesh *m, const char *path) {
    if (!m || !path) return FLITE_EINVAL;
    return guarded([&] {
        fio::Writer w(path);
        const int32_t N = m->lv[0].N;
        w.i4(N).i4(1).end();
        w.i4(N).end();
        for (int32_t i = 0; i < N; ++i) w.i4(i + 1).i4(m->perm[i]).end();
        w.close();
        return FLITE_OK;
    });
}

// makeplot (mg_par:1599-1707): plotreg.reg = (N, nDomains), per domain
// nLocal and nLocal records (local, global); the result file of domain d is
// res_prefix followed by d; u(global, :) = unk_d(local, :); the .unk holds N
// and the merged columns
int fp_makeplot(const char *plotreg, const char *res_prefix, int nvar, const char *unk) {
    if (!plotreg || !res_prefix || !unk || nvar < 1 || nvar > 7) return FLITE_EINVAL;
    return guarded([&] {
        fio::Reader r(plotreg);
        r.next();
        const int32_t N = r.i4(), nd = r.i4();
        if (N < 1 || nd < 1) throw fio::io_error("bad plotreg header");
        std::vector<double> u((size_t)N * nvar, 0.0);
        for (int32_t d = 1; d <= nd; ++d) {
            r.next();
            const int32_t nl = r.i4();
            if (nl < 0) throw fio::io_error("bad plotreg domain size");
            std::vector<int32_t> loc(nl), glob(nl);
            for (int32_t j = 0; j < nl; ++j) {
                r.next();
                loc[j] = r.i4();
                glob[j] = r.i4();
            }
            const std::string rpath = std::string(res_prefix) + std::to_string(d);
            fio::Reader rd(rpath.c_str());
            rd.next();
            const int32_t nto = rd.i4();
            rd.next();
            if (rd.remaining() < (size_t)nto * nvar * 8) throw fio::io_error("result record too short");
            std::vector<double> x((size_t)nto * nvar);
            rd.r8s(x.data(), x.size());
            for (int32_t j = 0; j < nl; ++j) {
                if (loc[j] < 1 || loc[j] > nto || glob[j] < 1 || glob[j] > N)
                    throw fio::io_error("plotreg node out of range");
                for (int k = 0; k < nvar; ++k)
                    u[(size_t)k * N + glob[j] - 1] = x[(size_t)k * nto + loc[j] - 1];
            }
        }
        fio::Writer w(unk);
        w.i4(N).end();
        w.r8s(u.data(), u.size()).end();
        w.close();
        return FLITE_OK;
    });
}

int fp_write_plt(const fp_mesh *m, const char *path) {
    if (!m || !path || m->tets.empty()) return FLITE_EINVAL;
    return guarded([&] {
        fio::Writer w(path);
        const LevelData &L = m->lv[0];
        const int32_t NT = (int32_t)(m->tets.size() / 4), NF = (int32_t)m->tri_ind.size();
        w.i4(NT).i4(L.N).i4(NF).end();
        w.i4s(m->tets.data(), m->tets.size()).end();
        w.r8s(L.xyz.data(), L.xyz.size()).end();
        std::vector<int32_t> f(5 * (size_t)NF);
        for (int32_t i = 0; i < NF; ++i) {
            for (int k = 0; k < 3; ++k) f[(size_t)k * NF + i] = m->tris[(size_t)k * NF + i];
            f[3 * (size_t)NF + i] = 0;
            f[4 * (size_t)NF + i] = m->tri_ind[i];
        }
        w.i4s(f.data(), f.size()).end();
        w.close();
        return FLITE_OK;
    });
}

}  // extern "C"

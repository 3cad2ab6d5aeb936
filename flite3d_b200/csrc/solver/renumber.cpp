// Node renumbering for locality: see renumber.h.
#include "renumber.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <stdexcept>

namespace flite {
namespace {

std::atomic<int> g_default_order{0};

// 21 bits of each coordinate interleaved into a 63-bit Morton key
uint64_t spread3(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

// order the nodes [lo, hi) by key, ties by their old number
void sort_range(std::vector<int> &perm, const std::vector<uint64_t> &key, int lo, int hi) {
    std::stable_sort(perm.begin() + lo, perm.begin() + hi, [&](int a, int b) { return key[a] < key[b]; });
}

int32_t remap(int32_t v, const std::vector<int> &iperm) {
    const int n = (int)iperm.size();
    return (v >= 1 && v <= n) ? iperm[v - 1] + 1 : v;  // invalid indices are left for create to refuse
}

}  // namespace

int default_node_order() { return g_default_order.load(); }

void renumber_levels(int nlevels, const flite_level_desc *lv, int mode, Renumbered &out) {
    out = Renumbered{};
    out.perm.resize(nlevels);
    out.iperm.resize(nlevels);
    out.desc.assign(lv, lv + nlevels);
    out.identity = mode == 0;
    for (int l = 0; l < nlevels; ++l) {
        const flite_level_desc &d = lv[l];
        const int N = d.n_nodes, Nb = d.n_bnodes;
        if (N <= 0 || Nb < 0 || Nb > N) throw std::runtime_error("bad level sizes");
        std::vector<int> &perm = out.perm[l];
        perm.resize(N);
        std::iota(perm.begin(), perm.end(), 0);
        if (mode != 0) {
            std::vector<uint64_t> key(N, 0);
            if (l == 0) {
                if (d.coords) {
                    double lo[3], hi[3];
                    for (int a = 0; a < 3; ++a) {
                        const double *x = d.coords + (size_t)a * N;
                        lo[a] = *std::min_element(x, x + N);
                        hi[a] = *std::max_element(x, x + N);
                    }
                    double span = 0.0;
                    for (int a = 0; a < 3; ++a) span = std::max(span, hi[a] - lo[a]);
                    const double scale = span > 0 ? 2097151.0 / span : 0.0;  // one scale: the curve stays isotropic
                    for (int i = 0; i < N; ++i) {
                        uint64_t k = 0;
                        for (int a = 0; a < 3; ++a) {
                            double q = (d.coords[(size_t)a * N + i] - lo[a]) * scale;
                            q = std::min(std::max(q, 0.0), 2097151.0);
                            k |= spread3((uint64_t)q) << a;
                        }
                        key[i] = k;
                    }
                } else {
                    for (int i = 0; i < N; ++i) key[i] = (uint64_t)i;
                }
            } else {
                // the smallest new number among a coarse node's children
                const int nf = lv[l - 1].n_nodes;
                std::fill(key.begin(), key.end(), ~uint64_t(0));
                if (d.parent)
                    for (int f = 0; f < nf; ++f) {
                        const int c = d.parent[f] - 1;
                        if (c >= 0 && c < N) key[c] = std::min<uint64_t>(key[c], (uint64_t)out.iperm[l - 1][f]);
                    }
            }
            sort_range(perm, key, 0, Nb);
            sort_range(perm, key, Nb, N);
        }
        std::vector<int> &iperm = out.iperm[l];
        iperm.resize(N);
        for (int i = 0; i < N; ++i) iperm[perm[i]] = i;
    }
    permute_levels(nlevels, lv, out);
}

void renumber_as(int nlevels, const flite_level_desc *lv, const std::vector<std::vector<int>> &perm,
                 const std::vector<std::vector<int>> &iperm, bool identity, Renumbered &out) {
    out = Renumbered{};
    out.desc.assign(lv, lv + nlevels);
    out.perm = perm;
    out.iperm = iperm;
    out.identity = identity;
    for (int l = 0; l < nlevels; ++l)
        if ((int)perm.size() <= l || (int)perm[l].size() != lv[l].n_nodes) throw std::runtime_error("bad level sizes");
    permute_levels(nlevels, lv, out);
}

void permute_levels(int nlevels, const flite_level_desc *lv, Renumbered &out) {
    if (out.identity) return;
    const size_t L = (size_t)nlevels;
    out.side_idx.resize(L); out.bnd_idx.resize(L); out.node_ind.resize(L); out.parent.resize(L);
    out.engine_idx.resize(L);
    out.volume.resize(L); out.wall_dist.resize(L); out.coords.resize(L); out.coord_move.resize(L);
    out.rweight.resize(L); out.volume_prev.resize(L); out.volume_prev2.resize(L);
    for (int l = 0; l < nlevels; ++l) {
        const flite_level_desc &d = lv[l];
        flite_level_desc &o = out.desc[l];
        const int N = d.n_nodes, E = d.n_sides, B = d.n_bsides;
        const std::vector<int> &perm = out.perm[l], &iperm = out.iperm[l];
        if (d.side_idx && E > 0) {
            auto &v = out.side_idx[l];
            v.resize(2 * (size_t)E);
            for (size_t k = 0; k < v.size(); ++k) v[k] = remap(d.side_idx[k], iperm);
            o.side_idx = v.data();
        }
        if (d.bnd_idx && B > 0) {
            auto &v = out.bnd_idx[l];
            v.assign(d.bnd_idx, d.bnd_idx + 3 * (size_t)B);
            for (size_t k = 0; k < 2 * (size_t)B; ++k) v[k] = remap(d.bnd_idx[k], iperm);
            o.bnd_idx = v.data();
        }
        if (d.engine_idx && d.n_engine_sides > 0) {
            const size_t ns = (size_t)d.n_engine_sides;
            auto &v = out.engine_idx[l];
            v.assign(d.engine_idx, d.engine_idx + 3 * ns);
            for (size_t k = 0; k < 2 * ns; ++k) v[k] = remap(d.engine_idx[k], iperm);
            o.engine_idx = v.data();
        }
        if (d.node_ind && d.n_normals > 0) {
            auto &v = out.node_ind[l];
            v.resize(d.n_normals);
            for (int k = 0; k < d.n_normals; ++k) v[k] = remap(d.node_ind[k], iperm);
            o.node_ind = v.data();
        }
        auto permute = [&](const double *src, int ncomp, std::vector<double> &dst) -> const double * {
            if (!src) return nullptr;
            dst.resize((size_t)ncomp * N);
            for (int a = 0; a < ncomp; ++a)
                for (int i = 0; i < N; ++i) dst[(size_t)a * N + i] = src[(size_t)a * N + perm[i]];
            return dst.data();
        };
        o.volume = permute(d.volume, 1, out.volume[l]);
        o.wall_dist = permute(d.wall_dist, 1, out.wall_dist[l]);
        o.coords = permute(d.coords, 3, out.coords[l]);
        o.coord_move = permute(d.coord_move, 3, out.coord_move[l]);
        o.volume_prev = permute(d.volume_prev, 1, out.volume_prev[l]);
        o.volume_prev2 = permute(d.volume_prev2, 1, out.volume_prev2[l]);
        if (l > 0) {
            // fine-indexed transfer arrays of this level: fine node in the
            // finer level's new numbering, parent in this level's
            const int nf = lv[l - 1].n_nodes;
            const std::vector<int> &pf = out.perm[l - 1];
            if (d.parent) {
                auto &v = out.parent[l];
                v.resize(nf);
                for (int f = 0; f < nf; ++f) v[f] = remap(d.parent[pf[f]], iperm);
                o.parent = v.data();
            }
            if (d.rweight) {
                auto &v = out.rweight[l];
                v.resize(nf);
                for (int f = 0; f < nf; ++f) v[f] = d.rweight[pf[f]];
                o.rweight = v.data();
            }
        }
    }
}

}  // namespace flite

extern "C" int flite_set_node_order(int32_t order) {
    if (order != 0 && order != 1) return FLITE_EINVAL;
    flite::g_default_order.store(order);
    return FLITE_OK;
}

// Multi-domain .sol files: gen3d's greedy partition, the per-domain writer
// and the ingest that merges the domains of a parallel run into one mesh (a
// GPU solves the whole mesh).  C ABI in include/flite_prepro.h.
//
// What follows the reference step by step (file:line in PreProSource/):
//   * the partition: greedyMeshPartition gen3d_struct.f90:890-1055 (a
//     frontal colouring with a priority list; the reference's colours end
//     0-based, the writer numbers domains from 1, so 1-based colours are
//     kept);
//   * the colour of a coarse node: the domain holding most of its children,
//     the first such domain on ties (mergeNodes gen3d_grid.f90:2843-2864),
//     and the fine nodes whose coarse parent lies in another domain
//     (:2866-2898);
//   * the records of each domain's file, level by level: the local
//     numbering (owned boundary nodes, boundary ghosts, owned interior nodes,
//     interior ghosts), the boundary sides (domain-crossing ones first, each
//     in the lower domain), the indicator register and node list, the sides
//     (crossing ones first, each in the lower domain), the node records, the
//     send and receive lists, and on coarse levels the prolongation and
//     restriction maps with their lists of fine nodes across domains:
//     writeParallelComputationFiles gen3d_grid.f90:4082-5231;
//   * plotreg.reg, the owned nodes of each domain with their global numbers
//     (:4805-4812), read back as makeplot does (mgnsg3d_mg_par.F90:1599-1707).
// The ingest resolves every ghost through the matching send and receive
// lists, takes each side and node once, and returns the mesh in the
// canonical form of fp_canonical (level-1 nodes keep their global numbers;
// sides in node-pair order; coarse nodes ordered by their first child), so
// that the files of any partition give one and the same mesh.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "flite_prepro.h"
#include "fortran_io.hpp"
#include "mesh_data.h"

using fp_internal::LevelData;

namespace {

template <class F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const fio::io_error &) {
        return FLITE_EIO;
    } catch (const std::exception &) {
        return FLITE_EINVAL;
    }
}

// ---- greedyMeshPartition (gen3d_struct.f90:890-1055) ------------------------
std::vector<int32_t> greedy_partition(int npart, const LevelData &L) {
    const int32_t npoin = L.N, nside = L.E;
    auto side = [&](int32_t is, int k) { return L.side[(size_t)(k - 1) * nside + (is - 1)]; };  // 1-based
    std::vector<int32_t> lph(npoin + 1, 0), lcp(npoin + 1, 0), lct(npoin + 1, 0), list(npoin + 1, 0),
        lbf(npoin + 1, 0), lpw(npoin + 1, 0), icone(2 * (size_t)nside + 1, 0);
    const int32_t nsm = (nside + npart) / npart;
    int32_t ncl = 1, nsc = 0;
    for (int32_t is = 1; is <= nside; ++is) { lph[side(is, 1)]++; lph[side(is, 2)]++; }
    lpw[1] = 1;
    int32_t iss = 1;
    for (int32_t i = 2; i <= npoin; ++i) {
        if (lph[i] < lph[iss]) iss = i;
        lpw[i] = lpw[i - 1] + lph[i - 1];
    }
    std::fill(lph.begin(), lph.end(), 0);
    for (int32_t is = 1; is <= nside; ++is) {
        const int32_t i1 = side(is, 1);
        lph[i1]++;
        icone[lpw[i1] + lph[i1] - 1] = is;
        const int32_t i2 = side(is, 2);
        lph[i2]++;
        icone[lpw[i2] + lph[i2] - 1] = is;
    }
    const int64_t guard = 8 * ((int64_t)npoin + nside) + 64;  // the walks below are bounded
    int64_t steps = 0;
    int32_t ist = iss;
    while (true) {
        lcp[ist] = ncl;
        for (int32_t ij = lpw[ist]; ij <= lpw[ist] + lph[ist] - 1; ++ij) {
            const int32_t is = icone[ij];
            int32_t i2 = side(is, 2) + side(is, 1) - ist;
            if (lcp[ist] == lcp[i2]) continue;  // (the reference counts these in nei)
            lct[i2]++;
            if (lcp[i2] != 0) continue;
            nsc++;
            if (lbf[i2] != 0) list[lbf[i2]] = 0;
            // insert i2 into the front list after ist, in the order of
            // lph - 2 lct
            int32_t isp = ist;
            while (true) {
                if (++steps > guard * 64) throw std::runtime_error("the partition's front list does not end");
                const int32_t in = list[isp];
                if (in == 0) {
                    list[isp] = i2;
                    lbf[i2] = isp;
                    break;
                }
                if ((lph[i2] - 2 * lct[i2]) < (lph[in] - 2 * lct[in])) {
                    list[isp] = i2;
                    lbf[i2] = isp;
                    isp = i2;
                    i2 = in;
                } else {
                    isp = in;
                }
            }
        }
        ist = list[ist];
        if (nsc >= nsm || ist == 0) {
            ncl++;
            nsc = 0;
            std::fill(lct.begin(), lct.end(), 0);
        }
        if (ist == 0) break;
        if (++steps > guard * 64) throw std::runtime_error("the partition does not end");
    }
    std::vector<int32_t> color(npoin);
    for (int32_t ip = 1; ip <= npoin; ++ip) {
        if (lcp[ip] == 0) throw std::runtime_error("the greedy partition left a node without a domain");
        color[ip - 1] = lcp[ip];
    }
    return color;
}

// the colours of a coarse level from its finer level's (mergeNodes
// gen3d_grid.f90:2843-2864)
std::vector<int32_t> coarse_colors(const LevelData &C, const std::vector<int32_t> &fine, int nd) {
    std::vector<int32_t> best(C.N, 0), col(C.N, 0), cnt(C.N, 0);
    for (int d = 1; d <= nd; ++d) {
        std::fill(cnt.begin(), cnt.end(), 0);
        for (size_t j = 0; j < fine.size(); ++j)
            if (fine[j] == d) cnt[C.parent[j] - 1]++;
        for (int32_t j = 0; j < C.N; ++j)
            if (cnt[j] > best[j]) { best[j] = cnt[j]; col[j] = d; }
    }
    return col;
}

// The local numbering of one domain of one level (writeParallelComputationFiles
// gen3d_grid.f90:4296-4455): o2n[j] = local number of global node j (0 = not
// in the domain), with the counts the records need.
struct Local {
    std::vector<int32_t> o2n;
    int32_t owned = 0, owned_b = 0, ghosts_b = 0, nlocal = 0, normals = 0;
};

Local local_numbering(const LevelData &L, const std::vector<int32_t> &col, int d) {
    Local o;
    const int32_t N = L.N, E = L.E, Nb = L.Nb;
    o.o2n.assign(N, 0);
    for (int32_t j = 0; j < N; ++j)
        if (col[j] == d) {
            o.owned++;
            if (j < Nb) {
                o.owned_b++;
                if (L.bnd_indicator[j] > 0) o.normals++;
            }
            o.o2n[j] = o.owned;
        }
    // the side's ghost end in domain d (the lower of the two domains)
    auto ghost_of = [&](int32_t e) -> int32_t {
        const int32_t a = L.side[e] - 1, b = L.side[(size_t)E + e] - 1;
        const int32_t da = col[a], db = col[b];
        if (da < db && da == d) return b;
        if (da > db && db == d) return a;
        return -1;
    };
    std::vector<char> flag(N, 0);
    for (int32_t e = 0; e < E; ++e) {
        const int32_t g = ghost_of(e);
        if (g >= 0 && g < Nb && !flag[g]) { flag[g] = 1; o.ghosts_b++; }
    }
    for (int32_t j = 0; j < N; ++j)
        if (o.o2n[j] > o.owned_b) o.o2n[j] += o.ghosts_b;
    int32_t count = 0;
    o.nlocal = o.ghosts_b + o.owned;
    for (int32_t e = 0; e < E; ++e) {
        const int32_t g = ghost_of(e);
        if (g < 0 || o.o2n[g] != 0) continue;
        if (g < Nb) {
            if (L.bnd_indicator[g] > 0) o.normals++;
            o.o2n[g] = o.owned_b + (++count);
        } else {
            o.o2n[g] = ++o.nlocal;
        }
    }
    return o;
}

std::string domain_path(const char *prefix, int d) { return std::string(prefix) + ".sol_" + std::to_string(d); }

// ---- one domain's records of one level (gen3d_grid.f90:4358-5200) ---------
void write_domain_level(fio::Writer &w, const LevelData &L, const std::vector<int32_t> &col, int nd, int d,
                        const Local &lo, bool fine, const LevelData *F, const std::vector<int32_t> *fcol,
                        const std::vector<int32_t> *ffull, const std::vector<int32_t> &l1full,
                        fio::Writer *reg) {
    const int32_t N = L.N, E = L.E, B = L.B, Nb = L.Nb;
    const std::vector<int32_t> &o2n = lo.o2n;
    auto lower = [&](int32_t a, int32_t b) { return std::min(col[a], col[b]); };
    // boundary sides: the domain-crossing ones of this (lower) domain, then
    // the domain's own
    int32_t nbs = 0, nbcs = 0;
    for (int32_t b = 0; b < B; ++b) {
        const int32_t a = L.bside[b] - 1, q = L.bside[(size_t)B + b] - 1;
        if (lower(a, q) == d) nbs++;
    }
    w.i4(nbs).end();
    auto bside_rec = [&](int32_t b) {
        const int32_t a = L.bside[b] - 1, q = L.bside[(size_t)B + b] - 1;
        w.i4(o2n[a]).i4(o2n[q]).i4(L.bside[2 * (size_t)B + b]);
        for (int k = 0; k < 3; ++k) w.r8(L.bw[(size_t)k * B + b]);
        for (int k = 0; k < 4; ++k) w.r8(L.bgcl.empty() ? 0.0 : L.bgcl[(size_t)k * B + b]);
        w.end();
    };
    for (int32_t b = 0; b < B; ++b) {
        const int32_t a = L.bside[b] - 1, q = L.bside[(size_t)B + b] - 1;
        if (col[a] != col[q] && lower(a, q) == d) { bside_rec(b); nbcs++; }
    }
    for (int32_t b = 0; b < B; ++b) {
        const int32_t a = L.bside[b] - 1, q = L.bside[(size_t)B + b] - 1;
        if (col[a] == d && col[q] == d) bside_rec(b);
    }
    // indicator register and node list over the domain's boundary nodes
    int32_t r[21] = {0};
    auto R = [&](int i) -> int32_t & { return r[i + 20]; };
    for (int32_t j = 0; j < Nb; ++j)
        if (o2n[j] > 0 && L.bnd_indicator[j] > 0) R(-21 + L.bnd_indicator[j] * 2) += 1;
    R(-20) = 1;
    for (int j = -18; j <= -2; j += 2) {
        R(j + 1) = R(j + 1) + R(j - 1);
        R(j) = R(j - 1) + 1;
    }
    w.i4(lo.owned_b + lo.ghosts_b).i4(lo.normals).end();
    for (int j = 0; j < 21; ++j) w.i4(r[j]).end();
    std::vector<double> nrm(3 * (size_t)Nb, 0.0);
    {
        const size_t nn = L.node_ind.size();
        for (size_t i = 0; i < nn; ++i)
            for (int k = 0; k < 3; ++k) nrm[3 * (size_t)(L.node_ind[i] - 1) + k] = L.bnormal[k * nn + i];
    }
    for (int ind = 1; ind <= 9; ++ind)
        for (int32_t j = 0; j < Nb; ++j)
            if (o2n[j] > 0 && L.bnd_indicator[j] == ind)
                w.i4(o2n[j]).r8(nrm[3 * (size_t)j]).r8(nrm[3 * (size_t)j + 1]).r8(nrm[3 * (size_t)j + 2]).end();
    // engine inlet sides, each in the lower domain of its two nodes
    // (gen3d_grid.f90:4599-4630)
    {
        const int32_t n = L.nes();
        int32_t cnt = 0;
        for (int32_t s = 0; s < n; ++s)
            if (lower(L.eside[s] - 1, L.eside[(size_t)n + s] - 1) == d) cnt++;
        w.i4(cnt).end();
        for (int32_t s = 0; s < n; ++s) {
            const int32_t a = L.eside[s] - 1, b = L.eside[(size_t)n + s] - 1;
            if (lower(a, b) != d) continue;
            w.i4(o2n[a]).i4(o2n[b]).i4(L.eside[2 * (size_t)n + s]);
            w.r8(L.ew[s]).r8(L.ew[(size_t)n + s]).r8(L.ew[2 * (size_t)n + s]).end();
        }
    }
    // sides
    int32_t ns = 0, ncs = 0;
    for (int32_t e = 0; e < E; ++e)
        if (lower(L.side[e] - 1, L.side[(size_t)E + e] - 1) == d) ns++;
    w.i4(ns).end();
    auto side_rec = [&](int32_t e) {
        const int32_t a = L.side[e] - 1, b = L.side[(size_t)E + e] - 1;
        w.i4(o2n[a]).i4(o2n[b]);
        for (int k = 0; k < 3; ++k) w.r8(L.sw[(size_t)k * E + e]);
        w.r8(L.gcl.empty() ? 0.0 : L.gcl[e]).r8(L.gcl.empty() ? 0.0 : L.gcl[(size_t)E + e]);
        w.r8(L.slen[e]).end();
    };
    for (int32_t e = 0; e < E; ++e) {
        const int32_t a = L.side[e] - 1, b = L.side[(size_t)E + e] - 1;
        if (col[a] != col[b] && lower(a, b) == d) { side_rec(e); ncs++; }
    }
    for (int32_t e = 0; e < E; ++e) {
        const int32_t a = L.side[e] - 1, b = L.side[(size_t)E + e] - 1;
        if (col[a] == d && col[b] == d) side_rec(e);
    }
    // node records (the wall node's number is the domain's own, 0 when the
    // wall node lies elsewhere; a coarse node's seed is its level-1 seed's
    // number in the seed's domain)
    w.i4(lo.nlocal).end();
    auto local_of = [&](int32_t g1) { return g1 >= 1 && g1 <= N ? o2n[g1 - 1] : 0; };
    for (int32_t j = 0; j < N; ++j) {
        if (o2n[j] == 0) continue;
        const int32_t wn = L.wnode.empty() ? 0 : local_of(L.wnode[j]);
        if (fine) {
            const bool mv = !L.volp.empty() && !L.xyzp.empty();
            w.i4(o2n[j]).r8(L.vol[j]).r8(mv ? L.volp[j] : L.vol[j]).r8(mv ? L.volp2[j] : L.vol[j]);
            w.r8(L.wdist[j]).i4(wn);
            for (const std::vector<double> *x : {&L.xyz, mv ? &L.xyzp : &L.xyz, mv ? &L.xyzp2 : &L.xyz})
                w.r8((*x)[j]).r8((*x)[(size_t)N + j]).r8((*x)[2 * (size_t)N + j]);
            w.end();
        } else {
            const int32_t s = L.seed.empty() ? 0 : L.seed[j];
            w.i4(o2n[j]).r8(L.vol[j]).r8(L.wdist[j]).i4(wn).i4(s >= 1 ? l1full[s - 1] : 0).end();
        }
    }
    if (fine) {
        w.i4(0).end();  // trip nodes
        w.i4(0).end();  // trip field nodes
        if (reg) {
            reg->i4(lo.owned).end();
            for (int32_t j = 0; j < N; ++j)
                if (col[j] == d) reg->i4(o2n[j]).i4(j + 1).end();
        }
    }
    // send and receive lists over the domain-crossing sides in side order
    std::vector<char> flag(lo.nlocal + 1, 0);
    auto lists = [&](bool send, int other, std::vector<int32_t> *out) {
        std::fill(flag.begin(), flag.end(), 0);
        for (int32_t e = 0; e < E; ++e) {
            const int32_t a = L.side[e] - 1, b = L.side[(size_t)E + e] - 1;
            const int32_t da = col[a], db = col[b];
            if (da == db) continue;
            const int32_t lo_d = std::min(da, db), hi_d = std::max(da, db);
            const int32_t hi_node = da < db ? b : a;  // the node in the higher domain
            const bool take = send ? (lo_d == d && hi_d == other) : (lo_d == other && hi_d == d);
            if (!take) continue;
            const int32_t loc = o2n[hi_node];
            if (!flag[loc]) { flag[loc] = 1; out->push_back(loc); }
        }
    };
    w.i4(ncs).i4(nbcs).end();
    std::vector<std::vector<int32_t>> snd(nd + 1), rcv(nd + 1);
    for (int j = 1; j <= nd; ++j) lists(true, j, &snd[j]);
    for (int j = 1; j <= nd; ++j) w.i4((int32_t)snd[j].size()).end();
    for (int j = 1; j <= nd; ++j)
        for (int32_t v : snd[j]) w.i4(v).end();
    for (int j = 1; j <= nd; ++j) lists(false, j, &rcv[j]);
    for (int j = 1; j <= nd; ++j) w.i4((int32_t)rcv[j].size()).end();
    for (int j = 1; j <= nd; ++j)
        for (int32_t v : rcv[j]) w.i4(v).end();
    if (fine) return;
    // prolongation and restriction maps of the finer level's nodes of this
    // domain; fine nodes whose parent lies in another domain go through the
    // com lists (gen3d_grid.f90:5018-5180)
    const int32_t nf = F->N;
    const std::vector<int32_t> &fc = *fcol, &full = *ffull;
    std::vector<int32_t> com;  // fineComNodes, in fine order
    for (int32_t j = 0; j < nf; ++j)
        if (fc[j] != col[L.parent[j] - 1]) com.push_back(j);
    std::vector<char> is_com(nf, 0);
    for (int32_t j : com) is_com[j] = 1;
    std::vector<int32_t> local_com(com.size(), 0);
    int32_t ncom_local = 0, n_noncom = 0;
    for (size_t k = 0; k < com.size(); ++k)
        if (fc[com[k]] == d) local_com[k] = ++ncom_local;
    for (int32_t j = 0; j < nf; ++j)
        if (fc[j] == d && !is_com[j]) n_noncom++;
    w.i4(n_noncom).end();
    w.i4(lo.owned).end();
    for (int32_t j = 0; j < nf; ++j)
        if (fc[j] == d && !is_com[j]) w.i4(full[j]).i4(o2n[L.parent[j] - 1]).end();
    w.i4(ncom_local).end();
    for (size_t k = 0; k < com.size(); ++k)
        if (fc[com[k]] == d) w.i4(full[com[k]]).end();
    w.i4(n_noncom).end();
    w.i4(lo.owned).end();
    for (int32_t j = 0; j < nf; ++j)
        if (fc[j] == d && col[L.parent[j] - 1] == d) w.i4(full[j]).r8(F->vol[j] / L.vol[L.parent[j] - 1]).end();
    w.i4(ncom_local).end();
    for (size_t k = 0; k < com.size(); ++k)
        if (fc[com[k]] == d) w.r8(F->vol[com[k]] / L.vol[L.parent[com[k]] - 1]).end();
    // com send lists: this domain's com nodes by the parent's domain; com
    // receive lists: the parents here of other domains' com nodes
    auto com_count = [&](int from, int to) {
        int32_t c = 0;
        for (size_t k = 0; k < com.size(); ++k)
            if (col[L.parent[com[k]] - 1] == to && fc[com[k]] == from) c++;
        return c;
    };
    int32_t mx = 0;
    for (int j = 1; j <= nd; ++j)
        if (j != d) mx = std::max(mx, com_count(d, j));
    w.i4(mx).end();
    for (int j = 1; j <= nd; ++j) {
        w.i4(j != d ? com_count(d, j) : 0).end();
        if (j == d) continue;
        for (size_t k = 0; k < com.size(); ++k)
            if (col[L.parent[com[k]] - 1] == j && fc[com[k]] == d) w.i4(local_com[k]).end();
    }
    mx = 0;
    for (int j = 1; j <= nd; ++j)
        if (j != d) mx = std::max(mx, com_count(j, d));
    w.i4(mx).end();
    for (int j = 1; j <= nd; ++j) {
        w.i4(j != d ? com_count(j, d) : 0).end();
        if (j == d) continue;
        for (size_t k = 0; k < com.size(); ++k)
            if (col[L.parent[com[k]] - 1] == d && fc[com[k]] == j) w.i4(o2n[L.parent[com[k]] - 1]).end();
    }
}

// ---- the ingest ---------------------------------------------------------------
// one domain's records of one level
struct DomLevel {
    int32_t N = 0, nbnd = 0;
    int32_t reg[21] = {0};
    std::vector<int32_t> bs1, bs2, bind, s1, s2, node_ind;  // local, 1-based
    std::vector<int32_t> es1, es2, ein;                     // engine inlet sides, local
    std::vector<double> ew;                                 // [n][3]
    std::vector<double> bw, bgcl, sw, gcl, slen;           // [B][3], [B][4], [E][3], [E][2], [E]
    std::vector<double> vol, volp, volp2, wdist, xyz, xyzp, xyzp2;  // by local node (0-based)
    std::vector<int32_t> wnode, seed;
    std::vector<std::vector<int32_t>> snd, rcv;  // per other domain (1-based index)
    // coarse levels
    std::vector<int32_t> pf, pc, comf;             // non-com (fine full, coarse local); com fine full
    std::vector<double> rw, rwc;                   // restriction weights (non-com, com)
    std::vector<std::vector<int32_t>> csnd, crcv;  // com lists per other domain
};

DomLevel read_domain_level(fio::Reader &r, bool fine, int nd) {
    DomLevel D;
    r.next(); const int32_t B = r.i4();
    if (B < 0) throw fio::io_error("negative count");
    for (int32_t b = 0; b < B; ++b) {
        r.next();
        D.bs1.push_back(r.i4()); D.bs2.push_back(r.i4()); D.bind.push_back(r.i4());
        for (int k = 0; k < 3; ++k) D.bw.push_back(r.r8());
        for (int k = 0; k < 4; ++k) D.bgcl.push_back(r.remaining() >= 8 ? r.r8() : 0.0);
    }
    r.next(); D.nbnd = r.i4(); const int32_t nn = r.i4();
    for (int j = 0; j < 21; ++j) { r.next(); D.reg[j] = r.i4(); }
    for (int32_t i = 0; i < nn; ++i) { r.next(); D.node_ind.push_back(r.i4()); }
    r.next(); const int32_t neis = r.i4();
    if (neis < 0) throw fio::io_error("negative count");
    for (int32_t s = 0; s < neis; ++s) {
        r.next();
        D.es1.push_back(r.i4()); D.es2.push_back(r.i4()); D.ein.push_back(r.i4());
        for (int k = 0; k < 3; ++k) D.ew.push_back(r.r8());
    }
    r.next(); const int32_t E = r.i4();
    if (E < 0) throw fio::io_error("negative count");
    for (int32_t e = 0; e < E; ++e) {
        r.next();
        D.s1.push_back(r.i4()); D.s2.push_back(r.i4());
        for (int k = 0; k < 3; ++k) D.sw.push_back(r.r8());
        D.gcl.push_back(r.r8()); D.gcl.push_back(r.r8());
        D.slen.push_back(r.r8());
    }
    r.next(); D.N = r.i4();
    if (D.N < 1) throw fio::io_error("bad node count");
    const size_t N = D.N;
    D.vol.assign(N, 0.0); D.wdist.assign(N, 0.0); D.wnode.assign(N, 0);
    if (fine) {
        D.volp.assign(N, 0.0); D.volp2.assign(N, 0.0);
        D.xyz.assign(3 * N, 0.0); D.xyzp.assign(3 * N, 0.0); D.xyzp2.assign(3 * N, 0.0);
    } else {
        D.seed.assign(N, 0);
    }
    for (size_t i = 0; i < N; ++i) {
        r.next();
        const int32_t id = r.i4();
        if (id < 1 || id > D.N) throw fio::io_error("node id out of range");
        const size_t j = id - 1;
        D.vol[j] = r.r8();
        if (fine) { D.volp[j] = r.r8(); D.volp2[j] = r.r8(); }
        D.wdist[j] = r.r8(); D.wnode[j] = r.i4();
        if (fine) {
            for (std::vector<double> *x : {&D.xyz, &D.xyzp, &D.xyzp2})
                for (int k = 0; k < 3; ++k) (*x)[3 * j + k] = r.r8();
        } else {
            D.seed[j] = r.i4();
        }
    }
    if (fine) {
        r.next(); const int32_t nt = r.i4();
        for (int32_t i = 0; i < nt; ++i) r.next();
        r.next(); const int32_t ntf = r.i4();
        for (int32_t i = 0; i < ntf; ++i) r.next();
    }
    r.next(); r.i4(); r.i4();  // communication sides (the first ones of each list)
    std::vector<int32_t> cnt(nd + 1);
    D.snd.assign(nd + 1, {}); D.rcv.assign(nd + 1, {});
    for (int j = 1; j <= nd; ++j) { r.next(); cnt[j] = r.i4(); }
    for (int j = 1; j <= nd; ++j)
        for (int32_t k = 0; k < cnt[j]; ++k) { r.next(); D.snd[j].push_back(r.i4()); }
    for (int j = 1; j <= nd; ++j) { r.next(); cnt[j] = r.i4(); }
    for (int j = 1; j <= nd; ++j)
        for (int32_t k = 0; k < cnt[j]; ++k) { r.next(); D.rcv[j].push_back(r.i4()); }
    if (fine) return D;
    r.next(); const int32_t nnc = r.i4();
    r.next(); r.i4();
    for (int32_t k = 0; k < nnc; ++k) { r.next(); D.pf.push_back(r.i4()); D.pc.push_back(r.i4()); }
    r.next(); const int32_t nc = r.i4();
    for (int32_t k = 0; k < nc; ++k) { r.next(); D.comf.push_back(r.i4()); }
    r.next(); const int32_t nnc2 = r.i4();
    r.next(); r.i4();
    if (nnc2 != nnc) throw fio::io_error("restriction and prolongation maps differ in size");
    for (int32_t k = 0; k < nnc; ++k) {
        r.next();
        if (r.i4() != D.pf[k]) throw fio::io_error("restriction and prolongation maps differ");
        D.rw.push_back(r.r8());
    }
    r.next(); if (r.i4() != nc) throw fio::io_error("com weights and com nodes differ in number");
    for (int32_t k = 0; k < nc; ++k) { r.next(); D.rwc.push_back(r.r8()); }
    D.csnd.assign(nd + 1, {}); D.crcv.assign(nd + 1, {});
    for (int pass = 0; pass < 2; ++pass) {
        r.next(); r.i4();  // the largest list
        for (int j = 1; j <= nd; ++j) {
            r.next(); const int32_t n = r.i4();
            for (int32_t k = 0; k < n; ++k) { r.next(); (pass == 0 ? D.csnd : D.crcv)[j].push_back(r.i4()); }
        }
    }
    return D;
}

}  // namespace

extern "C" {

int fp_partition(const fp_mesh *m, int32_t ndomains, int32_t *color, int32_t *ndomains_out) {
    if (!m || m->lv.empty() || ndomains < 1 || !color || !ndomains_out) return FLITE_EINVAL;
    return guarded([&] {
        std::vector<int32_t> c = greedy_partition(ndomains, m->lv[0]);
        std::memcpy(color, c.data(), c.size() * 4);
        *ndomains_out = *std::max_element(c.begin(), c.end());
        return FLITE_OK;
    });
}

int fp_write_sol_domains(const fp_mesh *m, const char *prefix, const char *plotreg, int32_t ndomains,
                         const int32_t *color) {
    if (!m || m->lv.empty() || !prefix || !plotreg || ndomains < 1) return FLITE_EINVAL;
    return guarded([&] {
        const size_t G = m->lv.size();
        std::vector<std::vector<int32_t>> col(G);
        col[0] = color ? std::vector<int32_t>(color, color + m->lv[0].N) : greedy_partition(ndomains, m->lv[0]);
        int nd = 0;
        for (int32_t c : col[0]) {
            if (c < 1) throw std::invalid_argument("domain colours are 1-based");
            nd = std::max(nd, (int)c);
        }
        for (size_t l = 1; l < G; ++l) col[l] = coarse_colors(m->lv[l], col[l - 1], nd);
        // the local numbering of every domain on every level and each node's
        // number in its own domain
        std::vector<std::vector<Local>> lo(G, std::vector<Local>(nd + 1));
        std::vector<std::vector<int32_t>> full(G);
        for (size_t l = 0; l < G; ++l) {
            full[l].assign(m->lv[l].N, 0);
            for (int d = 1; d <= nd; ++d) {
                lo[l][d] = local_numbering(m->lv[l], col[l], d);
                for (int32_t j = 0; j < m->lv[l].N; ++j)
                    if (col[l][j] == d) full[l][j] = lo[l][d].o2n[j];
            }
        }
        fio::Writer reg(plotreg);
        reg.i4(m->lv[0].N).i4(nd).end();
        for (int d = 1; d <= nd; ++d) {
            fio::Writer w(domain_path(prefix, d).c_str());
            w.i4((int32_t)G).end();
            w.i4(d).i4(nd).end();
            for (size_t l = 0; l < G; ++l)
                write_domain_level(w, m->lv[l], col[l], nd, d, lo[l][d], l == 0, l ? &m->lv[l - 1] : nullptr,
                                   l ? &col[l - 1] : nullptr, l ? &full[l - 1] : nullptr, full[0],
                                   l == 0 ? &reg : nullptr);
            w.close();
        }
        reg.close();
        return FLITE_OK;
    });
}

int fp_read_sol_domains(const char *prefix, const char *plotreg, fp_mesh **out) {
    if (!prefix || !plotreg || !out) return FLITE_EINVAL;
    *out = nullptr;
    return guarded([&] {
        // plotreg.reg: the global number of every domain's owned nodes
        fio::Reader pr(plotreg);
        pr.next(); const int32_t Ng = pr.i4(); const int32_t nd = pr.i4();
        if (Ng < 1 || nd < 1 || nd > 100000) throw fio::io_error("bad plot register header");
        std::vector<std::vector<std::pair<int32_t, int32_t>>> owned1(nd + 1);
        for (int d = 1; d <= nd; ++d) {
            pr.next(); const int32_t n = pr.i4();
            for (int32_t k = 0; k < n; ++k) { pr.next(); const int32_t a = pr.i4(); owned1[d].push_back({a, pr.i4()}); }
        }
        // every domain's records
        std::vector<std::vector<DomLevel>> dom(nd + 1);
        int32_t G = -1;
        for (int d = 1; d <= nd; ++d) {
            fio::Reader r(domain_path(prefix, d).c_str());
            r.next(); const int32_t g = r.i4();
            r.next(); const int32_t dd = r.i4(), ndd = r.i4();
            if (dd != d || ndd != nd || g < 1 || g > 32 || (G >= 0 && g != G))
                throw fio::io_error("domain file header does not match the plot register");
            G = g;
            for (int32_t l = 0; l < G; ++l) dom[d].push_back(read_domain_level(r, l == 0, nd));
        }
        auto M = std::make_unique<fp_mesh>();
        // global numbers of every domain's local nodes, level by level
        std::vector<std::vector<int32_t>> prev_glob;  // finer level: [d][local-1] -> global (0-based)
        std::vector<std::vector<char>> prev_owned;
        for (int32_t l = 0; l < G; ++l) {
            std::vector<std::vector<int32_t>> glob(nd + 1);
            std::vector<std::vector<char>> owned(nd + 1);
            for (int d = 1; d <= nd; ++d) {
                glob[d].assign(dom[d][l].N, -1);
                owned[d].assign(dom[d][l].N, 1);
                // the ghosts: this domain's send lists
                for (int j = 1; j <= nd; ++j)
                    for (int32_t v : dom[d][l].snd[j]) {
                        if (v < 1 || v > dom[d][l].N) throw fio::io_error("send list entry out of range");
                        owned[d][v - 1] = 0;
                    }
            }
            int32_t Nl = 0, Nbl = 0;
            if (l == 0) {
                for (int d = 1; d <= nd; ++d)
                    for (auto &p : owned1[d]) {
                        if (p.first < 1 || p.first > dom[d][0].N || p.second < 1 || p.second > Ng)
                            throw fio::io_error("plot register entry out of range");
                        glob[d][p.first - 1] = p.second - 1;
                    }
                Nl = Ng;
            } else {
                // owned boundary nodes of every domain first, then the owned
                // interior nodes (fp_canonical orders them afterwards)
                for (int pass = 0; pass < 2; ++pass)
                    for (int d = 1; d <= nd; ++d)
                        for (int32_t k = 0; k < dom[d][l].N; ++k) {
                            const bool bnd = k < dom[d][l].nbnd;
                            if (owned[d][k] && bnd == (pass == 0)) glob[d][k] = Nl++;
                        }
            }
            // the ghosts through the matching receive lists of their owners
            for (int d = 1; d <= nd; ++d)
                for (int j = 1; j <= nd; ++j) {
                    const auto &s = dom[d][l].snd[j], &rv = dom[j][l].rcv[d];
                    if (s.size() != rv.size()) throw fio::io_error("send and receive lists differ in length");
                    for (size_t k = 0; k < s.size(); ++k) {
                        if (rv[k] < 1 || rv[k] > dom[j][l].N) throw fio::io_error("receive list entry out of range");
                        glob[d][s[k] - 1] = glob[j][rv[k] - 1];
                    }
                }
            for (int d = 1; d <= nd; ++d)
                for (int32_t k = 0; k < dom[d][l].N; ++k)
                    if (glob[d][k] < 0) throw fio::io_error("a node of a domain has no global number");
            LevelData L;
            L.N = Nl;
            // boundary nodes: those a domain lists among its boundary nodes
            std::vector<int32_t> ind(Nl, -1);
            for (int d = 1; d <= nd; ++d) {
                const DomLevel &D = dom[d][l];
                for (int k = 1; k <= 9; ++k) {
                    const int32_t st = D.reg[2 * (k - 1)], en = D.reg[2 * (k - 1) + 1];
                    for (int32_t ib = st; ib <= en; ++ib) {
                        if (ib < 1 || ib > (int32_t)D.node_ind.size()) throw fio::io_error("indicator register out of range");
                        ind[glob[d][D.node_ind[ib - 1] - 1]] = k;
                    }
                }
                for (int32_t k = 0; k < D.nbnd; ++k)
                    if (ind[glob[d][k]] < 0) ind[glob[d][k]] = 0;
            }
            for (int32_t j = 0; j < Nl; ++j)
                if (ind[j] >= 0) L.Nb = std::max(L.Nb, j + 1);
            for (int32_t j = 0; j < L.Nb; ++j)
                if (ind[j] < 0) throw fio::io_error("the boundary nodes do not come first");
            L.bnd_indicator.assign(ind.begin(), ind.begin() + L.Nb);
            // node records from the owning domain
            L.vol.assign(Nl, 0.0); L.wdist.assign(Nl, 0.0); L.wnode.assign(Nl, 0);
            const bool fine = l == 0;
            if (fine) {
                L.volp.assign(Nl, 0.0); L.volp2.assign(Nl, 0.0);
                L.xyz.assign(3 * (size_t)Nl, 0.0); L.xyzp.assign(3 * (size_t)Nl, 0.0); L.xyzp2.assign(3 * (size_t)Nl, 0.0);
            }
            for (int d = 1; d <= nd; ++d) {
                const DomLevel &D = dom[d][l];
                for (int32_t k = 0; k < D.N; ++k) {
                    if (!owned[d][k]) continue;
                    const int32_t g = glob[d][k];
                    L.vol[g] = D.vol[k]; L.wdist[g] = D.wdist[k];
                    L.wnode[g] = fine && D.wnode[k] >= 1 && D.wnode[k] <= D.N ? glob[d][D.wnode[k] - 1] + 1 : 0;
                    if (fine) {
                        L.volp[g] = D.volp[k]; L.volp2[g] = D.volp2[k];
                        for (int c = 0; c < 3; ++c) {
                            L.xyz[(size_t)c * Nl + g] = D.xyz[3 * (size_t)k + c];
                            L.xyzp[(size_t)c * Nl + g] = D.xyzp[3 * (size_t)k + c];
                            L.xyzp2[(size_t)c * Nl + g] = D.xyzp2[3 * (size_t)k + c];
                        }
                    }
                }
            }
            // sides and boundary sides, each once (in its lower domain)
            for (int d = 1; d <= nd; ++d) {
                const DomLevel &D = dom[d][l];
                auto gid = [&](int32_t loc) {  // global 1-based number of a local node
                    if (loc < 1 || loc > D.N) throw fio::io_error("side record node out of range");
                    return glob[d][loc - 1] + 1;
                };
                for (size_t e = 0; e < D.s1.size(); ++e) {
                    L.side.push_back(gid(D.s1[e]));
                    L.side.push_back(gid(D.s2[e]));
                    for (int k = 0; k < 3; ++k) L.sw.push_back(D.sw[3 * e + k]);
                    L.gcl.push_back(D.gcl[2 * e]); L.gcl.push_back(D.gcl[2 * e + 1]);
                    L.slen.push_back(D.slen[e]);
                }
                for (size_t s = 0; s < D.es1.size(); ++s) {
                    if (D.ein[s] < 1 || D.ein[s] > 2) throw fio::io_error("bad engine inlet number");
                    L.eside.push_back(gid(D.es1[s]));
                    L.eside.push_back(gid(D.es2[s]));
                    L.eside.push_back(D.ein[s]);
                    for (int k = 0; k < 3; ++k) L.ew.push_back(D.ew[3 * s + k]);
                }
                for (size_t b = 0; b < D.bs1.size(); ++b) {
                    L.bside.push_back(gid(D.bs1[b]));
                    L.bside.push_back(gid(D.bs2[b]));
                    L.bside.push_back(D.bind[b]);
                    for (int k = 0; k < 3; ++k) L.bw.push_back(D.bw[3 * b + k]);
                    for (int k = 0; k < 4; ++k) L.bgcl.push_back(D.bgcl[4 * b + k]);
                }
            }
            // interleaved -> column-major
            auto transpose = [](std::vector<double> &v, size_t n, int k) {
                std::vector<double> o(v.size());
                for (size_t i = 0; i < n; ++i)
                    for (int c = 0; c < k; ++c) o[c * n + i] = v[(size_t)k * i + c];
                v.swap(o);
            };
            auto transpose_i = [](std::vector<int32_t> &v, size_t n, int k) {
                std::vector<int32_t> o(v.size());
                for (size_t i = 0; i < n; ++i)
                    for (int c = 0; c < k; ++c) o[c * n + i] = v[(size_t)k * i + c];
                v.swap(o);
            };
            L.E = (int32_t)L.slen.size();
            L.B = (int32_t)(L.bw.size() / 3);
            transpose_i(L.side, L.E, 2); transpose(L.sw, L.E, 3); transpose(L.gcl, L.E, 2);
            transpose_i(L.bside, L.B, 3); transpose(L.bw, L.B, 3); transpose(L.bgcl, L.B, 4);
            transpose_i(L.eside, L.ew.size() / 3, 3); transpose(L.ew, L.ew.size() / 3, 3);
            // coarse levels: parents and restriction weights of the finer
            // level's nodes
            if (l > 0) {
                const int32_t nf = M->lv[l - 1].N;
                L.parent.assign(nf, 0);
                L.rweight.assign(nf, 0.0);
                L.seed.assign(Nl, 0);
                for (int d = 1; d <= nd; ++d) {
                    const DomLevel &D = dom[d][l];
                    auto fine_glob = [&](int32_t loc) {
                        if (loc < 1 || loc > dom[d][l - 1].N || !prev_owned[d][loc - 1])
                            throw fio::io_error("a mapped fine node is not owned by its domain");
                        return prev_glob[d][loc - 1];
                    };
                    for (size_t k = 0; k < D.pf.size(); ++k) {
                        const int32_t f = fine_glob(D.pf[k]);
                        if (D.pc[k] < 1 || D.pc[k] > D.N) throw fio::io_error("coarse map entry out of range");
                        L.parent[f] = glob[d][D.pc[k] - 1] + 1;
                        L.rweight[f] = D.rw[k];
                    }
                    for (size_t k = 0; k < D.comf.size(); ++k) L.rweight[fine_glob(D.comf[k])] = D.rwc[k];
                    // com nodes: this domain's send list to j matches j's
                    // receive list from this domain
                    for (int j = 1; j <= nd; ++j) {
                        const auto &s = D.csnd[j], &rv = dom[j][l].crcv[d];
                        if (s.size() != rv.size()) throw fio::io_error("com lists differ in length");
                        for (size_t k = 0; k < s.size(); ++k) {
                            if (s[k] < 1 || s[k] > (int32_t)D.comf.size() || rv[k] < 1 || rv[k] > dom[j][l].N)
                                throw fio::io_error("com list entry out of range");
                            L.parent[fine_glob(D.comf[s[k] - 1])] = glob[j][rv[k] - 1] + 1;
                        }
                    }
                }
                for (int32_t f = 0; f < nf; ++f)
                    if (L.parent[f] < 1) throw fio::io_error("a fine node has no parent");
            }
            M->lv.push_back(std::move(L));
            prev_glob = std::move(glob);
            prev_owned = std::move(owned);
        }
        fp_internal::canonicalize(*M);
        *out = M.release();
        return FLITE_OK;
    });
}

}  // extern "C"

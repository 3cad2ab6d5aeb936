// Batched solves: many flow conditions on several meshes advanced together.
//
// A batch holds one context per case (mesh x flow condition).  Cases on the
// same mesh share that mesh's device copy (edges, coefficients, incidence
// lists, transfer operators, geometry); each case has its own solution state
// and controls.  One batch cycle is ONE launch of a CUDA graph.  The cases on
// one mesh form case groups: every kernel of the cycle runs once for a whole
// group, its grid's y index naming the case (the kernels' group form, which
// takes every case's level view and parameters as its arguments), so a group
// of G cases costs the launches of one case, and the coarse levels of all G
// fill the GPU together.  The groups (and cases whose controls take a path
// without a group form, each as its own cycle graph) are independent
// branches of the batch graph and run concurrently.  All cases read the
// cycle number from one device word.
//
// The autotuner times batch cycles for a set of edge-kernel and node-kernel
// block sizes and keeps the fastest pair (the caller stores the choice).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "context.h"

struct flite_batch {
    std::vector<flite_ctx *> cases;
    std::vector<int> donor;  // index of the case owning the mesh copy
    std::vector<char> active;  // cases the batch graph advances
    std::vector<char> turb;    // calculateTurbulence each case's part of the graph was captured with
    double *h_res = nullptr;   // pinned: res1 of every case
    cudaStream_t s = nullptr;
    int *d_cycle = nullptr;
    int *h_cycle = nullptr;
    cudaGraphExec_t graph = nullptr;
    int64_t launches = 0;
    std::string err;
    bool grouping = true;          // cases on one mesh advance as a case group
    int ngroups = 0;               // case groups in the graph

    ~flite_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        // cases that borrow a mesh go first, mesh owners last
        for (size_t i = cases.size(); i-- > 0;)
            if (donor[i] != (int)i && cases[i]) { flite_destroy(cases[i]); cases[i] = nullptr; }
        for (size_t i = cases.size(); i-- > 0;)
            if (cases[i]) { flite_destroy(cases[i]); cases[i] = nullptr; }
        if (d_cycle) cudaFree(d_cycle);
        if (h_cycle) cudaFreeHost(h_cycle);
        if (h_res) cudaFreeHost(h_res);
        if (s) cudaStreamDestroy(s);
    }

    // calculateTurbulence of every case for cycle `cyc` (SA cases); a change
    // drops the batch graph
    void select_cycle(int cyc) {
        for (size_t i = 0; i < cases.size(); ++i) {
            cases[i]->select_cycle(cyc);
            if (graph && turb[i] != (char)cases[i]->calcTurb) drop_graph();
        }
    }
    // cases whose cycles take the same launches (the controls that choose
    // kernels and grids agree; the freestream, CFL numbers and the other
    // values the kernels read may differ) and whose path has a group form
    static bool same_path(const flite_ctx &a, const flite_ctx &b) {
        const flite_controls &x = a.c, &y = b.c;
        return x.fluxType == y.fluxType && x.precision == y.precision &&
               (x.ReynoldsNumber > 0) == (y.ReynoldsNumber > 0) && x.viscosityScheme == y.viscosityScheme &&
               x.dissipationScheme == y.dissipationScheme &&
               x.coarseGridDissipationScheme == y.coarseGridDissipationScheme &&
               x.useMatrixDissipation == y.useMatrixDissipation &&
               x.useDissipationWeighting == y.useDissipationWeighting &&
               (x.secondOrderDissipationFactor == 0 && x.fourthOrderDissipationFactor == 0) ==
                   (y.secondOrderDissipationFactor == 0 && y.fourthOrderDissipationFactor == 0) &&
               x.multigridScheme == y.multigridScheme && x.numberOfRelaxationSteps == y.numberOfRelaxationSteps &&
               x.rungeKuttaStages == y.rungeKuttaStages && x.turbulenceModel == y.turbulenceModel &&
               x.flowType == y.flowType && x.reconstruction == y.reconstruction &&
               x.HLLCFluxOrder == y.HLLCFluxOrder && x.GradientMethod == y.GradientMethod &&
               x.Automaticlipping == y.Automaticlipping && a.lv.size() == b.lv.size() &&
               a.P.engines == b.P.engines && x.explicit_ == y.explicit_;
    }
    // the cycle graph of a case group led by its first case, or nullptr
    // when the group's path has no group form
    cudaGraph_t capture_group(const std::vector<int> &m) {
        flite_ctx *lead = cases[m[0]];
        for (int k : m)
            if (!same_path(*lead, *cases[k])) return nullptr;
        const size_t G = m.size(), nl = lead->lv.size();
        lead->gV.assign(nl, CaseTab<LevelView>{});
        for (size_t k = 0; k < G; ++k) {
            lead->gP.v[k] = cases[m[k]]->P;
            for (size_t l = 0; l < nl; ++l) lead->gV[l].v[k] = cases[m[k]]->lv[l].v;
        }
        lead->group = (int)G;
        cudaGraph_t g = nullptr;
        try {
            lead->capture_cycle(&g);
        } catch (const flite_ctx::no_group_error &) {  // a path without a group form
            g = nullptr;
        }
        lead->group = 0;
        return g;
    }
    void build_graph() {
        if (graph) return;
        turb.resize(cases.size());
        for (size_t i = 0; i < cases.size(); ++i) turb[i] = (char)cases[i]->calcTurb;
        cudaGraph_t parent = nullptr;
        CK(cudaGraphCreate(&parent, 0));
        launches = 0;
        ngroups = 0;
        auto add = [&](cudaGraph_t g) {
            cudaGraphNode_t node;
            cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, g);
            cudaGraphDestroy(g);
            CK(e);
        };
        try {
            std::vector<char> done(cases.size(), 0);
            for (size_t i = 0; i < cases.size(); ++i) {
                if (!active[i] || done[i]) continue;
                // the active cases on case i's mesh
                std::vector<int> m;
                for (size_t j = i; j < cases.size(); ++j)
                    if (active[j] && !done[j] && donor[j] == donor[i]) m.push_back((int)j);
                // at most kGroupMax cases a group (the parameter bank), in
                // groups of even size
                const size_t nchunk = (m.size() + kGroupMax - 1) / kGroupMax;
                m.resize((m.size() + nchunk - 1) / nchunk);
                cudaGraph_t g = grouping && m.size() > 1 ? capture_group(m) : nullptr;
                if (g) {
                    launches += cases[m[0]]->launches;
                    ++ngroups;
                    add(g);
                    for (int k : m) done[k] = 1;
                    continue;
                }
                flite_ctx *c = cases[i];
                c->capture_cycle(&g);
                launches += c->launches;
                add(g);
                done[i] = 1;
            }
            CK(cudaGraphInstantiate(&graph, parent, 0));
        } catch (...) {
            cudaGraphDestroy(parent);
            throw;
        }
        cudaGraphDestroy(parent);
    }
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (flite_ctx *c : cases) c->drop_graph();
    }
    void set_cycle(int cyc) {
        *h_cycle = cyc;
        CK(cudaMemcpyAsync(d_cycle, h_cycle, sizeof(int), cudaMemcpyHostToDevice, s));
    }
    // res1 of every active case (writeResiduals' density norm), one
    // synchronisation for all of them
    void residuals() {
        for (size_t i = 0; i < cases.size(); ++i) {
            if (!active[i]) continue;
            flite_ctx *c = cases[i];
            const LevelView &L = c->c.multigridScheme > 0 ? c->V(0) : c->V((int)c->lv.size() - 1);
            k_resid_partial<<<kResidBlocks, 256, 0, s>>>(L, c->d_part, kResidBlocks);
            k_resid_final<<<1, 192, 0, s>>>(c->d_part, kResidBlocks, c->d_out);
            CK(cudaMemcpyAsync(h_res + i, c->d_out, sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
    }
    // the cases' own graphs launched one after another on the batch stream
    void launch_sequential() {
        for (flite_ctx *c : cases) {
            c->ensure_graph();
            CK(cudaGraphLaunch(c->graph, s));
        }
    }
};

namespace {
template <class F>
int bguard(flite_batch *b, F &&f) {
    if (!b) return FLITE_EINVAL;
    try {
        return f();
    } catch (const std::exception &e) {
        b->err = e.what();
        return FLITE_ECUDA;
    }
}
}  // namespace

extern "C" {

int flite_batch_create(int ncases, const flite_controls *controls, const int32_t *mesh_of_case, int nmeshes,
                       const int32_t *nlevels, const flite_level_desc *const *levels, flite_batch **out) {
    if (ncases < 1 || !controls || !mesh_of_case || nmeshes < 1 || !nlevels || !levels || !out)
        return FLITE_EINVAL;
    *out = nullptr;
    auto B = std::make_unique<flite_batch>();
    B->cases.assign(ncases, nullptr);
    B->donor.assign(ncases, -1);
    B->active.assign(ncases, 1);
    std::vector<int> owner(nmeshes, -1);
    for (int i = 0; i < ncases; ++i) {
        const int m = mesh_of_case[i];
        if (m < 0 || m >= nmeshes || !levels[m] || nlevels[m] < 1) return FLITE_EINVAL;
        if (controls[i].flowType == 2) return FLITE_EUNSUPPORTED;  // moving meshes are not batched
        const flite_ctx *donor = owner[m] >= 0 ? B->cases[owner[m]] : nullptr;
        int rc = flite::create_context(&controls[i], nlevels[m], levels[m], donor, &B->cases[i]);
        if (rc != FLITE_OK) return rc;
        if (owner[m] < 0) owner[m] = i;
        B->donor[i] = owner[m];
    }
    int rc = bguard(B.get(), [&] {
        CK(cudaStreamCreateWithFlags(&B->s, cudaStreamNonBlocking));
        CK(cudaMalloc(&B->d_cycle, sizeof(int)));
        CK(cudaMallocHost(&B->h_cycle, sizeof(int)));
        CK(cudaMallocHost(&B->h_res, (size_t)ncases * sizeof(double)));
        // every case reads the batch's cycle number
        for (flite_ctx *c : B->cases) c->d_cycle = B->d_cycle;
        return FLITE_OK;
    });
    if (rc != FLITE_OK) return rc;
    *out = B.release();
    return FLITE_OK;
}

int flite_batch_destroy(flite_batch *b) {
    if (!b) return FLITE_EINVAL;
    if (b->s) cudaStreamSynchronize(b->s);
    delete b;
    return FLITE_OK;
}

int flite_batch_context(flite_batch *b, int case_index, flite_ctx **ctx) {
    if (!b || !ctx || case_index < 0 || case_index >= (int)b->cases.size()) return FLITE_EINVAL;
    *ctx = b->cases[case_index];
    return FLITE_OK;
}

int flite_batch_cycle(flite_batch *b, int cycle_no) {
    return bguard(b, [&] {
        b->select_cycle(cycle_no);
        b->build_graph();
        b->set_cycle(cycle_no);
        CK(cudaGraphLaunch(b->graph, b->s));
        CK(cudaStreamSynchronize(b->s));
        return FLITE_OK;
    });
}

int flite_batch_run(flite_batch *b, int first_cycle, int max_cycles, double orders, int check_every,
                    int32_t *cycles, double *log10_reduction) {
    if (!b || max_cycles < 1 || check_every < 1 || !cycles || !log10_reduction || !(orders > 0))
        return FLITE_EINVAL;
    return bguard(b, [&] {
        const size_t n = b->cases.size();
        std::vector<double> r0(n, 0.0), last(n, 0.0);
        for (size_t i = 0; i < n; ++i) { cycles[i] = 0; log10_reduction[i] = 0.0; }
        b->drop_graph();
        std::fill(b->active.begin(), b->active.end(), 1);
        const double target = std::pow(10.0, -orders);
        size_t left = n;
        for (int k = 0; k < max_cycles && left > 0; ++k) {
            b->select_cycle(first_cycle + k);
            b->build_graph();
            b->set_cycle(first_cycle + k);
            CK(cudaGraphLaunch(b->graph, b->s));
            for (size_t i = 0; i < n; ++i)
                if (b->active[i]) cycles[i] = k + 1;
            if (k > 0 && (k + 1) % check_every != 0 && k + 1 != max_cycles) continue;
            b->residuals();
            bool changed = false;
            for (size_t i = 0; i < n; ++i) {
                if (!b->active[i]) continue;
                const double r = b->h_res[i];
                if (!std::isfinite(r)) {
                    b->err = "NaN in the residual of case " + std::to_string(i);
                    return FLITE_ENAN;
                }
                if (k == 0) r0[i] = r;
                last[i] = r;
                if (r0[i] > 0 && r <= target * r0[i]) {
                    b->active[i] = 0;
                    --left;
                    changed = true;
                }
            }
            if (changed) {
                // converged cases leave the batch graph (and their groups)
                if (b->graph) cudaGraphExecDestroy(b->graph);
                b->graph = nullptr;
            }
        }
        for (size_t i = 0; i < n; ++i)
            log10_reduction[i] = (r0[i] > 0 && last[i] > 0) ? std::log10(last[i] / r0[i]) : 0.0;
        std::fill(b->active.begin(), b->active.end(), 1);
        b->drop_graph();
        return FLITE_OK;
    });
}

int flite_batch_time_cycles(flite_batch *b, int cycle_no, int ncycles, int sequential, double *ms,
                            int64_t *launches_per_cycle) {
    if (ncycles < 1 || !ms) return FLITE_EINVAL;
    return bguard(b, [&] {
        b->select_cycle(cycle_no);
        if (sequential) {
            for (flite_ctx *c : b->cases) c->ensure_graph();
        } else {
            b->build_graph();
        }
        b->set_cycle(cycle_no);
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, b->s));
        for (int k = 0; k < ncycles; ++k) {
            if (sequential) b->launch_sequential();
            else CK(cudaGraphLaunch(b->graph, b->s));
        }
        CK(cudaEventRecord(e1, b->s));
        CK(cudaEventSynchronize(e1));
        float t = 0;
        CK(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = t;
        if (launches_per_cycle) {
            int64_t n = 0;
            if (sequential)
                for (flite_ctx *c : b->cases) n += c->launches;
            else
                n = b->launches;
            *launches_per_cycle = n;
        }
        return FLITE_OK;
    });
}

int flite_batch_autotune(flite_batch *b, int cycle_no, int reps, int32_t *edge_block, int32_t *node_block,
                         double *best_ms) {
    if (!edge_block || !node_block || reps < 1) return FLITE_EINVAL;
    return bguard(b, [&] {
        static const int cand[3] = {64, 128, 256};
        double best = 1e300;
        int be = 256, bn = 256;
        for (int e : cand)
            for (int n : cand) {
                b->drop_graph();
                for (flite_ctx *c : b->cases) { c->eb = e; c->nb = n; }
                b->build_graph();
                b->set_cycle(cycle_no);
                CK(cudaGraphLaunch(b->graph, b->s));  // warm
                cudaEvent_t e0, e1;
                CK(cudaEventCreate(&e0));
                CK(cudaEventCreate(&e1));
                CK(cudaEventRecord(e0, b->s));
                for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(b->graph, b->s));
                CK(cudaEventRecord(e1, b->s));
                CK(cudaEventSynchronize(e1));
                float t = 0;
                CK(cudaEventElapsedTime(&t, e0, e1));
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                if (t / reps < best) { best = t / reps; be = e; bn = n; }
            }
        b->drop_graph();
        for (flite_ctx *c : b->cases) { c->eb = be; c->nb = bn; }
        // case groups on or off, whichever runs the batch cycle faster (the
        // groups save launches; separate case graphs overlap more freely)
        double tg[2] = {0, 0};
        for (int g = 0; g < 2; ++g) {
            b->drop_graph();
            b->grouping = g == 1;
            b->build_graph();
            b->set_cycle(cycle_no);
            CK(cudaGraphLaunch(b->graph, b->s));  // warm
            cudaEvent_t e0, e1;
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            CK(cudaEventRecord(e0, b->s));
            for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(b->graph, b->s));
            CK(cudaEventRecord(e1, b->s));
            CK(cudaEventSynchronize(e1));
            float t = 0;
            CK(cudaEventElapsedTime(&t, e0, e1));
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            tg[g] = t / reps;
        }
        b->drop_graph();
        b->grouping = tg[1] <= tg[0];
        best = std::min(best, std::min(tg[0], tg[1]));
        *edge_block = be;
        *node_block = bn;
        if (best_ms) *best_ms = best;
        return FLITE_OK;
    });
}

// The lanes per node of each level's gathers (the gather tile: a thread, or
// 4..32 lanes of a warp per node), chosen level by level, coarsest first,
// by timing batch cycles; the other levels keep their choice meanwhile.
// lanes[l] receives level l+1's choice for l < nlevels (0 past the deepest
// level of any case).
int flite_batch_autotune_lanes(flite_batch *b, int cycle_no, int reps, int32_t nlevels, int32_t *lanes,
                               double *best_ms) {
    if (!b || reps < 1 || nlevels < 1 || !lanes) return FLITE_EINVAL;
    return bguard(b, [&] {
        static const int cand[5] = {1, 4, 8, 16, 32};
        int deep = 0;
        for (flite_ctx *c : b->cases) deep = std::max(deep, (int)c->lv.size());
        deep = std::min(deep, std::min((int)nlevels, kMaxLevels));
        auto time = [&]() {
            b->drop_graph();
            b->build_graph();
            b->set_cycle(cycle_no);
            CK(cudaGraphLaunch(b->graph, b->s));  // warm
            cudaEvent_t e0, e1;
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            CK(cudaEventRecord(e0, b->s));
            for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(b->graph, b->s));
            CK(cudaEventRecord(e1, b->s));
            CK(cudaEventSynchronize(e1));
            float t = 0;
            CK(cudaEventElapsedTime(&t, e0, e1));
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return (double)t / reps;
        };
        double best = 1e300;
        for (int l = deep - 1; l >= 0; --l) {
            int keep = 1;
            double bl = 1e300;
            for (int u : cand) {
                for (flite_ctx *c : b->cases)
                    if (l < (int)c->lv.size()) c->lanes[l] = u;
                const double t = time();
                if (t < bl) { bl = t; keep = u; }
            }
            for (flite_ctx *c : b->cases)
                if (l < (int)c->lv.size()) c->lanes[l] = keep;
            best = bl;
        }
        b->drop_graph();
        for (int l = 0; l < nlevels; ++l) {
            int v = 0;
            for (flite_ctx *c : b->cases)
                if (l < (int)c->lv.size() && l < kMaxLevels) v = c->lanes[l];
            lanes[l] = v;
        }
        if (best_ms) *best_ms = best;
        return FLITE_OK;
    });
}

int flite_batch_set_grouping(flite_batch *b, int on) {
    if (!b) return FLITE_EINVAL;
    b->drop_graph();
    b->grouping = on != 0;
    return FLITE_OK;
}

int flite_batch_groups(const flite_batch *b, int32_t *ngroups) {
    if (!b || !ngroups) return FLITE_EINVAL;
    *ngroups = b->grouping ? b->ngroups : 0;
    return FLITE_OK;
}

int flite_batch_grouping(const flite_batch *b, int32_t *on) {
    if (!b || !on) return FLITE_EINVAL;
    *on = b->grouping ? 1 : 0;
    return FLITE_OK;
}

int flite_batch_set_blocks(flite_batch *b, int32_t edge_block, int32_t node_block) {
    if (!b || edge_block < 32 || edge_block > 256 || node_block < 32 || node_block > 256 ||
        edge_block % 32 || node_block % 32)
        return FLITE_EINVAL;
    b->drop_graph();
    for (flite_ctx *c : b->cases) { c->eb = edge_block; c->nb = node_block; }
    return FLITE_OK;
}

}  // extern "C"

// Residual evaluation that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host whose device memory is owned by
// another allocator (a framework's caching pool, CUDA Fortran arrays managed
// by the host program, a process that must not grow its footprint between
// checkpoints) or code running where allocation is forbidden.  For them
// flite_residual_noalloc computes the same interior + boundary residual as
// flite_residual_fwd (central flux, fluxType 1, def_par:1664-1669 and the
// boundary faces def_par:2182-2446) from caller-owned device arrays in the
// reference layout, using as scratch one file-scope device array of a fixed
// size instead of allocations.
//
// The scratch array below is part of the library image: every GPU that loads
// the library holds kScratchBytes of it until the process exits.  Its device
// address is looked up once per device with cudaGetSymbolAddress, on the
// first call made while that device is current.  A call copies its status
// into host memory and synchronises the stream it is given, so no call may be
// made while any stream is being captured into a CUDA graph.  All calls share
// the one array and it keeps the last call's contents; each call
// re-initialises what must start at zero.  Calls that overlap on the GPU
// (different streams, or different host threads on the same device) race on
// the scratch and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "flite_gpu.h"
#include "flux.cuh"

namespace flite {
namespace {

constexpr int64_t kMaxNodes = 65536;
constexpr int64_t kMaxEdges = 262144;
constexpr int64_t kMaxBEdges = 65536;

// scratch layout (bytes, each region 256-aligned)
constexpr int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }
constexpr int64_t kOffP = 0;                                               // double p[N]
constexpr int64_t kOffFlux = kOffP + align256(8 * kMaxNodes);               // double flux[E][5]
constexpr int64_t kOffBflux = kOffFlux + align256(40 * kMaxEdges);          // double bflux[B][10]
constexpr int64_t kOffIncPtr = kOffBflux + align256(80 * kMaxBEdges);       // int inc_ptr[N+1]
constexpr int64_t kOffInc = kOffIncPtr + align256(4 * (kMaxNodes + 1));     // int2 inc[2E]
constexpr int64_t kOffBPtr = kOffInc + align256(16 * kMaxEdges);            // int binc_ptr[N+1]
constexpr int64_t kOffBinc = kOffBPtr + align256(4 * (kMaxNodes + 1));      // int binc[2B]
constexpr int64_t kOffEdge = kOffBinc + align256(8 * kMaxBEdges);           // int2 edge[E]
constexpr int64_t kOffBEdge = kOffEdge + align256(8 * kMaxEdges);           // int2 bedge[B]
constexpr int64_t kOffBind = kOffBEdge + align256(8 * kMaxBEdges);          // int bind[B]
constexpr int64_t kOffFlag = kOffBind + align256(4 * kMaxBEdges);          // int error flag
constexpr int64_t kScratchBytes = kOffFlag + 256;

// the scratch: static device storage, no allocation at run time
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};

__global__ void na_clear_flag(int *flag) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *flag = 0;
}

// The error flag: an index outside 1..N or a boundary code outside 1..9
// (FLITE_EINVAL).
constexpr int kFlagInvalid = 1;

// 0-based copies of the caller's 1-based index arrays; an edge that raises
// the error flag is dropped from every pass
__global__ void na_prepare(int N, int E, int B, const int32_t *side_idx, const int32_t *bnd_idx,
                           int2 *edge, int2 *bedge, int *bind, int *inc_ptr, int *binc_ptr, int *flag) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < E) {
        int a = side_idx[t] - 1, b = side_idx[E + t] - 1;
        if (a < 0 || a >= N || b < 0 || b >= N || a == b) { atomicOr(flag, kFlagInvalid); a = -1; b = -1; }
        edge[t] = make_int2(a, b);
    }
    if (t < B) {
        int a = bnd_idx[t] - 1, b = bnd_idx[B + t] - 1;
        const int code = bnd_idx[2 * B + t];
        if (a < 0 || a >= N || b < 0 || b >= N || code < 1 || code > 9) {
            atomicOr(flag, kFlagInvalid); a = -1; b = -1;
        }
        bedge[t] = make_int2(a, b);
        bind[t] = code;
    }
    if (t <= N) { inc_ptr[t] = 0; binc_ptr[t] = 0; }
}

// incidence counts; integer atomics only, whose results do not depend on order
__global__ void na_count(int E, int B, const int2 *edge, const int2 *bedge, int *inc_ptr, int *binc_ptr) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < E && edge[t].x >= 0) {
        atomicAdd(&inc_ptr[edge[t].x + 1], 1);
        atomicAdd(&inc_ptr[edge[t].y + 1], 1);
    }
    if (t < B && bedge[t].x >= 0) {
        atomicAdd(&binc_ptr[bedge[t].x + 1], 1);
        atomicAdd(&binc_ptr[bedge[t].y + 1], 1);
    }
}

// exclusive prefix sums of the counts (one block; sizes are bounded)
__global__ void na_scan(int N, int *inc_ptr, int *binc_ptr) {
    __shared__ int carry[2];
    if (threadIdx.x == 0) { carry[0] = 0; carry[1] = 0; }
    __syncthreads();
    for (int base = 1; base <= N; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v0 = i <= N ? inc_ptr[i] : 0, v1 = i <= N ? binc_ptr[i] : 0;
        // block-wide inclusive scan by warp shuffles + shared partials
        __shared__ int ws0[32], ws1[32];
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            int a = __shfl_up_sync(0xffffffffu, v0, o), b = __shfl_up_sync(0xffffffffu, v1, o);
            if (lane >= o) { v0 += a; v1 += b; }
        }
        if (lane == 31) { ws0[wid] = v0; ws1[wid] = v1; }
        __syncthreads();
        if (wid == 0) {
            int nw = blockDim.x / 32;
            int a = lane < nw ? ws0[lane] : 0, b = lane < nw ? ws1[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int x = __shfl_up_sync(0xffffffffu, a, o), y = __shfl_up_sync(0xffffffffu, b, o);
                if (lane >= o) { a += x; b += y; }
            }
            if (lane < nw) { ws0[lane] = a; ws1[lane] = b; }
        }
        __syncthreads();
        if (wid > 0) { v0 += ws0[wid - 1]; v1 += ws1[wid - 1]; }
        if (i <= N) { inc_ptr[i] = v0 + carry[0]; binc_ptr[i] = v1 + carry[1]; }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) { carry[0] += v0; carry[1] += v1; }
        __syncthreads();
    }
}

// one thread per node: gather the node's incident edges in increasing edge
// order by scanning candidate edges through the edge array is too slow, so
// positions are claimed with integer atomics and each node's short segment is
// then insertion-sorted by edge number
__global__ void na_place(int E, int B, const int2 *edge, const int2 *bedge, const int *inc_ptr,
                         const int *binc_ptr, int *cursor, int *bcursor, int2 *inc, int *binc) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < E && edge[t].x >= 0) {
        int a = edge[t].x, b = edge[t].y;
        int pa = inc_ptr[a] + atomicAdd(&cursor[a], 1);
        inc[pa] = make_int2(t, b);
        int pb = inc_ptr[b] + atomicAdd(&cursor[b], 1);
        inc[pb] = make_int2(~t, a);
    }
    if (t < B && bedge[t].x >= 0) {
        int a = bedge[t].x, b = bedge[t].y;
        int pa = binc_ptr[a] + atomicAdd(&bcursor[a], 1);
        binc[pa] = 2 * t;
        int pb = binc_ptr[b] + atomicAdd(&bcursor[b], 1);
        binc[pb] = 2 * t + 1;
    }
}

__device__ __forceinline__ int edge_of(int2 v) { return v.x >= 0 ? v.x : ~v.x; }

__global__ void na_sort(int N, const int *inc_ptr, const int *binc_ptr, int2 *inc, int *binc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int k = inc_ptr[i] + 1; k < inc_ptr[i + 1]; ++k) {
        int2 v = inc[k];
        int q = k - 1;
        while (q >= inc_ptr[i] && edge_of(inc[q]) > edge_of(v)) { inc[q + 1] = inc[q]; --q; }
        inc[q + 1] = v;
    }
    // boundary entries: 2b+side sorts by boundary edge, side 0 before side 1
    for (int k = binc_ptr[i] + 1; k < binc_ptr[i + 1]; ++k) {
        int v = binc[k];
        int q = k - 1;
        while (q >= binc_ptr[i] && binc[q] > v) { binc[q + 1] = binc[q]; --q; }
        binc[q + 1] = v;
    }
}

__global__ void na_zero(int *a, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = 0;
}

__global__ void na_pressure(Params P, LevelView L) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.N) return;
    const int N = L.N;
    L.p[i] = pressure(P, L.u[i], L.u[N + i], L.u[2 * N + i], L.u[3 * N + i], L.u[4 * N + i]);
}

__global__ void na_edge(Params P, LevelView L) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L.E) return;
    int2 nd = L.edge[e];
    if (nd.x < 0) return;  // dropped by the index check
    double f[5];
    edge_flux<1, false>(P, L, e, nd.x, nd.y, f);
    double *o = L.flux + (size_t)e * 5;
    for (int k = 0; k < 5; ++k) o[k] = f[k];
}

__global__ void na_bnd(Params P, LevelView L) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= L.B) return;
    if (L.bedge[b].x < 0) return;  // dropped by the index check
    double g1[5], g2[5];
    boundary_flux(P, L, b, g1, g2);
    double *o = L.bflux + (size_t)b * 10;
    for (int k = 0; k < 5; ++k) { o[k] = g1[k]; o[5 + k] = g2[k]; }
}

__global__ void na_gather(LevelView L, double *rhs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.N) return;
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = L.inc_ptr[i]; k < L.inc_ptr[i + 1]; ++k) {
        int s = L.inc[k].x;
        const double *f = L.flux + (size_t)(s >= 0 ? s : ~s) * 5;
        if (s >= 0) for (int c = 0; c < 5; ++c) r[c] = r[c] + f[c];
        else for (int c = 0; c < 5; ++c) r[c] = r[c] - f[c];
    }
    for (int k = L.binc_ptr[i]; k < L.binc_ptr[i + 1]; ++k) {
        int v = L.binc[k];
        const double *g = L.bflux + (size_t)(v >> 1) * 10 + (v & 1) * 5;
        for (int c = 0; c < 5; ++c) r[c] = r[c] + g[c];
    }
    for (int c = 0; c < 5; ++c) rhs[(size_t)c * L.N + i] = r[c];
}

// the device address of the scratch for the current device, looked up once
int scratch_for_current_device(unsigned char **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FLITE_ECUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return FLITE_ECUDA;
        g_scratch_ptr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_ptr[dev];
    return FLITE_OK;
}

}  // namespace
}  // namespace flite

using namespace flite;

extern "C" int flite_residual_noalloc(const flite_controls *c, int32_t n_nodes, int32_t n_sides,
                                      int32_t n_bsides, const int32_t *d_side_idx, const double *d_side_w,
                                      const int32_t *d_bnd_idx, const double *d_bnd_w, const double *d_u,
                                      double *d_rhs, void *stream) {
    if (!c || !d_side_idx || !d_side_w || !d_u || !d_rhs || (n_bsides > 0 && (!d_bnd_idx || !d_bnd_w)))
        return FLITE_EINVAL;
    if (n_nodes <= 0 || n_sides < 0 || n_bsides < 0) return FLITE_EINVAL;
    // sizes beyond the static scratch are rejected
    if (n_nodes > kMaxNodes || n_sides > kMaxEdges || n_bsides > kMaxBEdges) return FLITE_EINVAL;
    if (c->fluxType != 1) return FLITE_EUNSUPPORTED;
    unsigned char *base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc != FLITE_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;

    Params P{};
    P.gamma = c->gamma; P.gm1 = c->gamma - 1.0; P.boundaryTerm = c->boundaryTerm;
    for (int i = 0; i < 12; ++i) P.inf[i] = c->inflowField[i];
    const int N = n_nodes, E = n_sides, B = n_bsides;
    LevelView L{};
    L.N = N; L.E = E; L.B = B; L.grid = 1;
    L.wx = d_side_w; L.wy = d_side_w + E; L.wz = d_side_w + 2 * (size_t)E;
    L.bwx = d_bnd_w; L.bwy = d_bnd_w + B; L.bwz = d_bnd_w + 2 * (size_t)B;
    L.u = const_cast<double *>(d_u);
    L.p = (double *)(base + kOffP);
    L.flux = (double *)(base + kOffFlux);
    L.bflux = (double *)(base + kOffBflux);
    int *inc_ptr = (int *)(base + kOffIncPtr), *binc_ptr = (int *)(base + kOffBPtr);
    int2 *inc = (int2 *)(base + kOffInc), *edge = (int2 *)(base + kOffEdge), *bedge = (int2 *)(base + kOffBEdge);
    int *binc = (int *)(base + kOffBinc), *bind = (int *)(base + kOffBind);
    L.inc_ptr = inc_ptr; L.inc = inc; L.binc_ptr = binc_ptr; L.binc = binc;
    L.edge = edge; L.bedge = bedge; L.bind = bind;
    // cursors for the placement reuse the flux region, which is rewritten
    // after the incidence lists are complete
    int *cursor = (int *)(base + kOffFlux), *bcursor = cursor + (N + 1);
    int *flag = (int *)(base + kOffFlag);

    const int T = 256;
    const int nmax = (int)std::max<int64_t>(std::max<int64_t>(E, B), N + 1);
    const int ne = std::max(E, B);
    // an error left pending by earlier, unrelated work is not this call's
    (void)cudaGetLastError();
    na_clear_flag<<<1, 1, 0, s>>>(flag);
    na_prepare<<<(nmax + T - 1) / T, T, 0, s>>>(N, E, B, d_side_idx, d_bnd_idx, edge, bedge, bind, inc_ptr,
                                               binc_ptr, flag);
    na_zero<<<(2 * (N + 1) + T - 1) / T, T, 0, s>>>(cursor, 2 * (N + 1));
    if (ne > 0) na_count<<<(ne + T - 1) / T, T, 0, s>>>(E, B, edge, bedge, inc_ptr, binc_ptr);
    na_scan<<<1, 1024, 0, s>>>(N, inc_ptr, binc_ptr);
    if (ne > 0)
        na_place<<<(ne + T - 1) / T, T, 0, s>>>(E, B, edge, bedge, inc_ptr, binc_ptr, cursor, bcursor, inc, binc);
    na_sort<<<(N + T - 1) / T, T, 0, s>>>(N, inc_ptr, binc_ptr, inc, binc);
    na_pressure<<<(N + T - 1) / T, T, 0, s>>>(P, L);
    if (E > 0) na_edge<<<(E + T - 1) / T, T, 0, s>>>(P, L);
    if (B > 0) na_bnd<<<(B + T - 1) / T, T, 0, s>>>(P, L);
    na_gather<<<(N + T - 1) / T, T, 0, s>>>(L, d_rhs);
    if (cudaGetLastError() != cudaSuccess) return FLITE_ECUDA;
    // the checks' verdict (a 4-byte copy into host memory; no allocation);
    // this synchronises the caller's stream
    int hflag = 0;
    if (cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return FLITE_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FLITE_ECUDA;
    if (hflag & kFlagInvalid) return FLITE_EINVAL;
    return FLITE_OK;
}

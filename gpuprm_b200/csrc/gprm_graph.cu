/*
 * gprm_graph.cu - roadmap graph operations on the device (gprm_graph_* of
 * include/gprm_b200.h).
 *
 * The reference keeps its roadmaps as host adjacency lists and, once start
 * and goal are connected, runs Dijkstra on each (do_dijkstra,
 * prm/src/lib/prm/prmsolver.cpp:2805-2846; edge insertion and connection
 * flags: 2099-2186, calc_conn 2763-2787).  Here the roadmap stays an edge
 * list in device memory (u[e], v[e], an optional mask of usable edges,
 * float weights) and every operation is a handful of kernels:
 *
 *   components  lock-free union-find: each usable edge hooks the larger of
 *               its two roots under the smaller (atomicCAS), finds halve
 *               paths; the label of a vertex is the smallest vertex of its
 *               component (deterministic);
 *   forest      breadth-first forest from every component's label vertex,
 *               level-synchronous over the edge list; a vertex's parent is
 *               the smallest vertex of the previous level adjacent to it
 *               (deterministic); depth = level;
 *   paths       the forest path between two vertices of one component,
 *               counted, then written (one thread per query);
 *   sssp        single-source shortest paths under float path sums
 *               accumulated from the source (Bellman-Ford relaxation until
 *               no distance drops; float addition is monotone, so these
 *               are the distances Dijkstra computes with the same
 *               arithmetic); parent = smallest neighbour u with
 *               dist[u] + w == dist[v].
 *
 * All calls are asynchronous on the given stream except where a loop over
 * levels / rounds needs the device's "changed" flag (forest, sssp), which
 * is read back every few levels.
 */
#include <cuda_runtime.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "../../include/gprm_b200.h"

namespace {

constexpr int UNSEEN = INT_MAX;

__device__ __forceinline__ int find_root(volatile int* parent, int x)
{
    /* parent[x] <= x always (roots hook under smaller roots), so any
       ancestor is a valid parent: path halving with plain stores */
    while (true) {
        const int p = parent[x];
        if (p == x) return x;
        const int g = parent[p];
        if (g == p) return p;
        parent[x] = g;
        x = g;
    }
}

__global__ void k_uf_init(int V, int* parent)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) parent[i] = i;
}

__global__ void k_uf_union(int V, int E, const int* __restrict__ eu, const int* __restrict__ ev,
                           const unsigned char* __restrict__ mask, int* parent)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        if (mask && !mask[e]) continue;
        int a = eu[e], b = ev[e];
        if ((unsigned)a >= (unsigned)V || (unsigned)b >= (unsigned)V) continue;   /* bad edge: skipped */
        while (true) {
            a = find_root(parent, a);
            b = find_root(parent, b);
            if (a == b) break;
            if (a < b) { int t = a; a = b; b = t; }
            const int old = atomicCAS(&parent[a], a, b);
            if (old == a) break;
            a = old;
        }
    }
}

__global__ void k_uf_flatten(int V, int* parent, int* label)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
        label[i] = find_root(parent, i);
}

/* ---------------------------------------------------------------- forest */

__global__ void k_forest_init(int V, const int* __restrict__ label, int* depth, int* parent, int* cand)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        const bool root = label[i] == i;
        depth[i] = root ? 0 : UNSEEN;
        parent[i] = -1;
        cand[i] = UNSEEN;
    }
}

__global__ void k_forest_expand(int V, int E, const int* __restrict__ eu, const int* __restrict__ ev,
                                const unsigned char* __restrict__ mask, const int* __restrict__ depth, int level,
                                int* cand)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        if (mask && !mask[e]) continue;
        const int a = eu[e], b = ev[e];
        if ((unsigned)a >= (unsigned)V || (unsigned)b >= (unsigned)V) continue;
        const int da = depth[a], db = depth[b];
        if (da == level && db == UNSEEN) atomicMin(&cand[b], a);
        if (db == level && da == UNSEEN) atomicMin(&cand[a], b);
    }
}

__global__ void k_forest_settle(int V, int level, int* depth, int* parent, int* cand, int* changed)
{
    int any = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        const int c = cand[i];
        if (c != UNSEEN) {
            depth[i] = level + 1;
            parent[i] = c;
            cand[i] = UNSEEN;
            any = 1;
        }
    }
    if (any) atomicOr(changed, 1);
}

/* ---------------------------------------------------------------- paths */

__device__ __forceinline__ int forest_lca(const int* parent, const int* depth, int a, int b)
{
    while (depth[a] > depth[b]) a = parent[a];
    while (depth[b] > depth[a]) b = parent[b];
    while (a != b) { a = parent[a]; b = parent[b]; }
    return a;
}

__global__ void k_path_len(int V, int Q, const int* __restrict__ qs, const int* __restrict__ qt,
                           const int* __restrict__ label, const int* __restrict__ parent,
                           const int* __restrict__ depth, int* len)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < Q; t += gridDim.x * blockDim.x) {
        const int s = qs[t], g = qt[t];
        if ((unsigned)s >= (unsigned)V || (unsigned)g >= (unsigned)V || label[s] != label[g] || depth[s] == UNSEEN || depth[g] == UNSEEN) {
            len[t] = 0;
            continue;
        }
        const int c = forest_lca(parent, depth, s, g);
        len[t] = depth[s] - depth[c] + depth[g] - depth[c] + 1;
    }
}

__global__ void k_path_write(int Q, const int* __restrict__ qs, const int* __restrict__ qt,
                             const int* __restrict__ parent, const int* __restrict__ depth,
                             const long long* __restrict__ off, const int* __restrict__ len, int* out)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < Q; t += gridDim.x * blockDim.x) {
        const int L = len[t];
        if (L == 0) continue;
        const int s = qs[t], g = qt[t];
        const int c = forest_lca(parent, depth, s, g);
        int* o = out + off[t];
        int k = 0;
        for (int x = s; x != c; x = parent[x]) o[k++] = x;      /* s .. just below c */
        o[k] = c;
        int m = depth[g] - depth[c];                            /* g's side, reversed */
        for (int x = g; x != c; x = parent[x]) o[k + m--] = x;
    }
}

/* ---------------------------------------------------------------- sssp */

__global__ void k_sssp_init(int V, int src, float* dist, int* parent)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        dist[i] = i == src ? 0.0f : INFINITY;
        parent[i] = i == src ? src : -1;
    }
}

/* non-negative floats order like their bit patterns */
__device__ __forceinline__ bool relax(float* dist, int v, float nd)
{
    const int old = atomicMin(reinterpret_cast<int*>(dist) + v, __float_as_int(nd));
    return nd < __int_as_float(old);
}

__global__ void k_sssp_relax(int V, int E, const int* __restrict__ eu, const int* __restrict__ ev,
                             const unsigned char* __restrict__ mask, const float* __restrict__ w, float* dist,
                             int* changed)
{
    int any = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        if (mask && !mask[e]) continue;
        const int a = eu[e], b = ev[e];
        if ((unsigned)a >= (unsigned)V || (unsigned)b >= (unsigned)V) continue;
        const float we = w[e];
        const float da = ((volatile float*)dist)[a], db = ((volatile float*)dist)[b];
        if (da + we < db && relax(dist, b, da + we)) any = 1;
        if (db + we < da && relax(dist, a, db + we)) any = 1;
    }
    if (any) atomicOr(changed, 1);
}

__global__ void k_sssp_parent(int V, int E, const int* __restrict__ eu, const int* __restrict__ ev,
                              const unsigned char* __restrict__ mask, const float* __restrict__ w,
                              const float* __restrict__ dist, int src, int* parent)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        if (mask && !mask[e]) continue;
        const int a = eu[e], b = ev[e];
        if ((unsigned)a >= (unsigned)V || (unsigned)b >= (unsigned)V) continue;
        const float we = w[e];
        if (b != src && isfinite(dist[a]) && dist[a] + we == dist[b]) atomicMin((unsigned*)&parent[b], (unsigned)a);
        if (a != src && isfinite(dist[b]) && dist[b] + we == dist[a]) atomicMin((unsigned*)&parent[a], (unsigned)b);
    }
}

}  // namespace

struct gprm_graph {
    int device = 0;
    int sms = 0;
    int* changed = nullptr;     /* device flag */
    int* host_changed = nullptr;/* pinned */
    int* cand = nullptr;
    int* uf = nullptr;
    size_t cap_v = 0;
    std::string err = "no error";
};

namespace {

thread_local std::string g_graph_create_error = "no error";

int gfail(gprm_graph* h, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    else g_graph_create_error = buf;
    return code;
}

#define GRAPH_TRY(h, call)                                                                  \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return gfail((h), e_ == cudaErrorMemoryAllocation ? GPRM_ERR_NOMEM : GPRM_ERR_CUDA, \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

int ensure_v(gprm_graph* h, int V)
{
    if ((size_t)V <= h->cap_v && h->cand) return GPRM_OK;
    cudaFree(h->cand);
    cudaFree(h->uf);
    h->cand = h->uf = nullptr;
    const size_t c = (size_t)V + V / 4 + 64;
    GRAPH_TRY(h, cudaMalloc((void**)&h->cand, c * sizeof(int)));
    GRAPH_TRY(h, cudaMalloc((void**)&h->uf, c * sizeof(int)));
    h->cap_v = c;
    return GPRM_OK;
}

int grid_for(const gprm_graph* h, long long n)
{
    long long b = (n + 255) / 256;
    const long long cap = (long long)h->sms * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

/* Runs `step(level)` until the device flag stays clear, reading it back
 * every `every` levels; at most max_levels levels. */
template <class F>
int until_stable(gprm_graph* h, cudaStream_t st, int max_levels, int every, F step, int* levels_out)
{
    int level = 0;
    while (level < max_levels) {
        GRAPH_TRY(h, cudaMemsetAsync(h->changed, 0, sizeof(int), st));
        const int upto = level + every < max_levels ? level + every : max_levels;
        for (; level < upto; ++level) {
            int rc = step(level);
            if (rc) return rc;
        }
        GRAPH_TRY(h, cudaMemcpyAsync(h->host_changed, h->changed, sizeof(int), cudaMemcpyDeviceToHost, st));
        GRAPH_TRY(h, cudaStreamSynchronize(st));
        if (!*h->host_changed) break;
    }
    if (levels_out) *levels_out = level;
    return GPRM_OK;
}

}  // namespace

extern "C" {

int gprm_graph_create(gprm_graph** out)
{
    if (!out) return gfail(nullptr, GPRM_ERR_ARG, "null output");
    *out = nullptr;
    gprm_graph* h = new gprm_graph();
    if (cudaGetDevice(&h->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess ||
        cudaMalloc((void**)&h->changed, sizeof(int)) != cudaSuccess ||
        cudaHostAlloc((void**)&h->host_changed, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
        cudaFree(h->changed);
        delete h;
        return gfail(nullptr, GPRM_ERR_CUDA, "no CUDA device or allocation failed");
    }
    *out = h;
    return GPRM_OK;
}

void gprm_graph_destroy(gprm_graph* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    cudaFree(h->changed);
    cudaFreeHost(h->host_changed);
    cudaFree(h->cand);
    cudaFree(h->uf);
    delete h;
}

const char* gprm_graph_last_error(const gprm_graph* h) { return h ? h->err.c_str() : g_graph_create_error.c_str(); }

int gprm_graph_components(gprm_graph* h, int V, int E, const int* eu, const int* ev, const unsigned char* mask,
                          int* label, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (V < 0 || E < 0 || (V > 0 && !label) || (E > 0 && (!eu || !ev))) return gfail(h, GPRM_ERR_ARG, "bad sizes or pointers");
    if (V == 0) return GPRM_OK;
    GRAPH_TRY(h, cudaSetDevice(h->device));
    int rc = ensure_v(h, V);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    k_uf_init<<<grid_for(h, V), 256, 0, st>>>(V, h->uf);
    if (E > 0) k_uf_union<<<grid_for(h, E), 256, 0, st>>>(V, E, eu, ev, mask, h->uf);
    k_uf_flatten<<<grid_for(h, V), 256, 0, st>>>(V, h->uf, label);
    GRAPH_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

int gprm_graph_forest(gprm_graph* h, int V, int E, const int* eu, const int* ev, const unsigned char* mask,
                      const int* label, int* parent, int* depth, int* levels, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (V < 0 || E < 0 || (V > 0 && (!label || !parent || !depth)) || (E > 0 && (!eu || !ev)))
        return gfail(h, GPRM_ERR_ARG, "bad sizes or pointers");
    if (V == 0) return GPRM_OK;
    GRAPH_TRY(h, cudaSetDevice(h->device));
    int rc = ensure_v(h, V);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    k_forest_init<<<grid_for(h, V), 256, 0, st>>>(V, label, depth, parent, h->cand);
    GRAPH_TRY(h, cudaGetLastError());
    if (E == 0) {
        if (levels) *levels = 0;
        return GPRM_OK;
    }
    auto step = [&](int level) -> int {
        k_forest_expand<<<grid_for(h, E), 256, 0, st>>>(V, E, eu, ev, mask, depth, level, h->cand);
        k_forest_settle<<<grid_for(h, V), 256, 0, st>>>(V, level, depth, parent, h->cand, h->changed);
        GRAPH_TRY(h, cudaGetLastError());
        return GPRM_OK;
    };
    return until_stable(h, st, V, 16, step, levels);
}

int gprm_graph_path_lengths(gprm_graph* h, int V, int Q, const int* qs, const int* qt, const int* label,
                            const int* parent, const int* depth, int* len, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (Q < 0 || (Q > 0 && (!qs || !qt || !label || !parent || !depth || !len)))
        return gfail(h, GPRM_ERR_ARG, "bad sizes or pointers");
    if (Q == 0) return GPRM_OK;
    GRAPH_TRY(h, cudaSetDevice(h->device));
    k_path_len<<<grid_for(h, Q), 256, 0, (cudaStream_t)stream>>>(V, Q, qs, qt, label, parent, depth, len);
    GRAPH_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

int gprm_graph_path_write(gprm_graph* h, int Q, const int* qs, const int* qt, const int* parent, const int* depth,
                          const int* len, const long long* offsets, int* out, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (Q < 0 || (Q > 0 && (!qs || !qt || !parent || !depth || !len || !offsets || !out)))
        return gfail(h, GPRM_ERR_ARG, "bad sizes or pointers");
    if (Q == 0) return GPRM_OK;
    GRAPH_TRY(h, cudaSetDevice(h->device));
    k_path_write<<<grid_for(h, Q), 256, 0, (cudaStream_t)stream>>>(Q, qs, qt, parent, depth, offsets, len, out);
    GRAPH_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

int gprm_graph_sssp(gprm_graph* h, int V, int E, const int* eu, const int* ev, const unsigned char* mask,
                    const float* w, int src, float* dist, int* parent, int* rounds, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (V < 1 || E < 0 || src < 0 || src >= V || !dist || !parent || (E > 0 && (!eu || !ev || !w)))
        return gfail(h, GPRM_ERR_ARG, "bad sizes, source or pointers");
    GRAPH_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    k_sssp_init<<<grid_for(h, V), 256, 0, st>>>(V, src, dist, parent);
    GRAPH_TRY(h, cudaGetLastError());
    if (E == 0) {
        if (rounds) *rounds = 0;
        return GPRM_OK;
    }
    auto step = [&](int) -> int {
        k_sssp_relax<<<grid_for(h, E), 256, 0, st>>>(V, E, eu, ev, mask, w, dist, h->changed);
        GRAPH_TRY(h, cudaGetLastError());
        return GPRM_OK;
    };
    int rc = until_stable(h, st, V + 1, 8, step, rounds);
    if (rc) return rc;
    /* parents from the converged distances (parent[] still -1 except src) */
    k_sssp_parent<<<grid_for(h, E), 256, 0, st>>>(V, E, eu, ev, mask, w, dist, src, parent);
    GRAPH_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

}  /* extern "C" */

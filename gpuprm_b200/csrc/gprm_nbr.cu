/*
 * gprm_nbr.cu - neighbour search on the device (gprm_nbr_* of
 * include/gprm_b200.h).
 *
 * The reference planner finds the roadmap nodes within distance D of a new
 * node by scanning the key blocks of its host map (get_near_vertices,
 * prm/src/lib/prm/prmsolver.cpp:2533-2574): squared distance accumulated
 * over the joints in order in float, kept when normsq < D*D, written until
 * the caller's buffer is full.  Here the nodes stay on the device:
 *
 *   radius   one warp per query walks the nodes in index order, 32 at a
 *            time; a ballot compacts the hits, so a query's neighbours come
 *            out in ascending index order and the first `cap` are kept
 *            (the reference's "terminate if buffer full");
 *   knn      the k nearest nodes under the same distance, ties broken by
 *            the lower index.  Nodes are bucketed into a uniform grid over
 *            all joints (counting sort by cell); a query scans the
 *            3^ndof cells around its own and keeps a sorted top-k
 *            (a thread per query for the nodes themselves, a warp per query
 *            for outside queries); a
 *            result is accepted only when its k-th distance is below the
 *            distance to the scanned block's boundary (with slack for float
 *            rounding), otherwise the query is redone over the 5^ndof block
 *            by a block of threads, and if that block's test fails too, by a
 *            block that scans every node.  The result is therefore the exact
 *            top-k.
 *
 * Distances use the reference's arithmetic: d = x_j - q_j, s = s + d*d
 * (no FMA; the library is compiled with -fmad=false), dist = sqrt(s).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../../include/gprm_b200.h"

namespace {

constexpr int NBR_MAX_GRID = GPRM_MAX_DOF;
constexpr int NBR_MAX_K = 32;
constexpr int NBR_MAX_CELLS = 1 << 21;

struct GridView {
    int ndof, G, n;
    float lo[NBR_MAX_GRID];
    float inv_cell;   /* 1 / cell */
    float cell;
    float slack;      /* rounding allowance of the exactness test */
    int nc[NBR_MAX_GRID];
    const float* xs;      /* nodes sorted by cell, SoA [ndof][n] */
    const int* id;        /* original index of each sorted node */
    const int* start;     /* cell start offsets [ncells + 1] */
};

__device__ __forceinline__ float dist2(const float* __restrict__ x, long long xstride, long long i,
                                       const float* qv, int ndof)
{
    float s = 0.0f;
    for (int j = 0; j < ndof; ++j) {
        const float d = x[i + xstride * j] - qv[j];
        s = s + d * d;
    }
    return s;
}

__device__ __forceinline__ int cell_coord(float v, float lo, float inv_cell, int nc)
{
    float c = floorf((v - lo) * inv_cell);
    int ci = isfinite(c) ? (int)fminf(fmaxf(c, 0.0f), (float)(nc - 1)) : 0;
    return ci;
}

/* dist2 of four consecutive nodes p..p+3: the same arithmetic per node,
 * the four nodes' loads issued together. */
__device__ __forceinline__ void dist2_4(const float* __restrict__ x, long long xstride, long long p, const float* qv,
                                        int ndof, float* s)
{
    s[0] = s[1] = s[2] = s[3] = 0.0f;
    for (int j = 0; j < ndof; ++j) {
        const float* xj = x + p + xstride * j;
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = xj[u];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float d = v[u] - qv[j];
            s[u] = s[u] + d * d;
        }
    }
}

/* (s, id) lexicographic order */
__device__ __forceinline__ bool less_pair(float s, int i, float t, int j)
{
    return s < t || (s == t && i < j);
}

__global__ void k_minmax(const float* __restrict__ x, int n, long long stride, int ndof, float* out)
{
    /* out[2j] = min, out[2j+1] = max of joint j; out pre-set to +inf/-inf */
    for (int j = 0; j < ndof; ++j) {
        float lo = INFINITY, hi = -INFINITY;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const float v = x[i + stride * j];
            if (isfinite(v)) { lo = fminf(lo, v); hi = fmaxf(hi, v); }
        }
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if ((threadIdx.x & 31) == 0) {
            /* float min/max through the ordered-int trick (values are finite) */
            int* o2 = reinterpret_cast<int*>(out);
            if (lo <= hi) {
                if (lo >= 0) atomicMin(&o2[2 * j], __float_as_int(lo));
                else atomicMax((unsigned*)&o2[2 * j], __float_as_uint(lo));
                if (hi >= 0) atomicMax(&o2[2 * j + 1], __float_as_int(hi));
                else atomicMin((unsigned*)&o2[2 * j + 1], __float_as_uint(hi));
            }
        }
    }
}

__global__ void k_cell_keys(const float* __restrict__ x, int n, long long stride, GridView g, int* key, int* count)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int k = 0;
        for (int d = g.G - 1; d >= 0; --d) k = k * g.nc[d] + cell_coord(x[i + stride * d], g.lo[d], g.inv_cell, g.nc[d]);
        key[i] = k;
        atomicAdd(&count[k], 1);
    }
}

/* exclusive scan of count[0..nc) into start[0..nc], one block */
__global__ void k_scan(const int* __restrict__ count, int nc, int* start)
{
    __shared__ int part[1024];
    const int t = threadIdx.x, T = blockDim.x;
    const int per = (nc + T - 1) / T;
    const int b = t * per, e = min(nc, b + per);
    int s = 0;
    for (int i = b; i < e; ++i) s += count[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {
        int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = t > 0 ? part[t - 1] : 0;
    for (int i = b; i < e; ++i) {
        start[i] = run;
        run += count[i];
    }
    if (t == T - 1) start[nc] = part[T - 1];
}

__global__ void k_scatter(const float* __restrict__ x, int n, long long stride, int ndof, const int* __restrict__ key,
                          const int* __restrict__ start, int* cursor, float* xs, int* id)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int k = key[i];
        const int p = start[k] + atomicAdd(&cursor[k], 1);
        for (int j = 0; j < ndof; ++j) xs[p + (long long)n * j] = x[i + stride * j];
        id[p] = i;
    }
}

/* ---------------------------------------------------------------- radius */

__global__ void k_radius(const float* __restrict__ x, int n, long long xstride, const float* __restrict__ q, int m,
                         long long qstride, int ndof, float D2, int cap, int* counts, int* idx, float* dist)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (long long w = (long long)blockIdx.x * wpb + (threadIdx.x >> 5); w < m; w += (long long)gridDim.x * wpb) {
        float qv[GPRM_MAX_DOF];
        for (int j = 0; j < ndof; ++j) qv[j] = q[w + qstride * j];
        int found = 0;
        for (int base = 0; base < n && found < cap; base += 32) {
            const int i = base + lane;
            float s = 0.0f;
            bool hit = false;
            if (i < n) {
                s = dist2(x, xstride, i, qv, ndof);
                hit = s < D2;
            }
            const unsigned hm = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                const int slot = found + __popc(hm & ((1u << lane) - 1u));
                if (slot < cap) {
                    idx[w * (long long)cap + slot] = i;
                    dist[w * (long long)cap + slot] = sqrtf(s);
                }
            }
            found += __popc(hm);
        }
        if (lane == 0) counts[w] = found < cap ? found : cap;
    }
}

/* ---------------------------------------------------------------- knn */

/* The list's current k-th entry, kept in registers so that most
 * candidates are rejected by one comparison, before their index is even
 * loaded: (INFINITY, INT_MAX) until the list is full. */
struct TopkBound {
    float s;
    int i;
};

__device__ __forceinline__ void topk_bound(const float* ts, const int* ti, int len, int k, TopkBound& b)
{
    if (len == k) { b.s = ts[k - 1]; b.i = ti[k - 1]; }
}

/* Inserts (s, i) into the sorted top list (len entries used, capacity k). */
__device__ __forceinline__ void topk_insert(float* ts, int* ti, int& len, int k, float s, int i)
{
    if (len == k && !less_pair(s, i, ts[k - 1], ti[k - 1])) return;
    int p = len < k ? len : k - 1;
    while (p > 0 && less_pair(s, i, ts[p - 1], ti[p - 1])) {
        ts[p] = ts[p - 1];
        ti[p] = ti[p - 1];
        --p;
    }
    ts[p] = s;
    ti[p] = i;
    if (len < k) ++len;
}

/* The block of cells a query scans: cells c-radius..c+radius in each
 * gridded joint (clipped to the grid); guard = the distance from q to the block's faces
 * that have cells beyond them (infinite when none).  Returns false when a
 * gridded coordinate is not finite. */
__device__ __forceinline__ bool query_block(const GridView& g, const float* qv, int* lo, int* hi, float* guard,
                                            int radius = 1)
{
    bool finite = true;
    float gd = INFINITY;
    for (int d = 0; d < g.G; ++d) {
        finite &= isfinite(qv[d]);
        const int c = cell_coord(qv[d], g.lo[d], g.inv_cell, g.nc[d]);
        lo[d] = max(c - radius, 0);
        hi[d] = min(c + radius, g.nc[d] - 1);
        if (lo[d] > 0) gd = fminf(gd, qv[d] - (g.lo[d] + (float)lo[d] * g.cell));
        if (hi[d] < g.nc[d] - 1) gd = fminf(gd, (g.lo[d] + (float)(hi[d] + 1) * g.cell) - qv[d]);
    }
    for (int j = g.G; j < g.ndof; ++j) finite &= isfinite(qv[j]);
    *guard = gd;
    return finite;
}

/* Number of rows of the block (cells varying in joints 1..G-1) and the
 * sorted-node range of row r (joint 0 runs lo[0]..hi[0], contiguous). */
__device__ __forceinline__ int block_rows(const GridView& g, const int* lo, const int* hi)
{
    int r = 1;
    for (int d = 1; d < g.G; ++d) r *= hi[d] - lo[d] + 1;
    return r;
}

__device__ __forceinline__ void block_row_range(const GridView& g, const int* lo, const int* hi, int r, int* b, int* e)
{
    int cell = 0;
    int rest = r;
    int coord[NBR_MAX_GRID];
    for (int d = 1; d < g.G; ++d) {
        const int span = hi[d] - lo[d] + 1;
        coord[d] = lo[d] + rest % span;
        rest /= span;
    }
    for (int d = g.G - 1; d >= 1; --d) cell = cell * g.nc[d] + coord[d];
    const int row = cell * g.nc[0];
    *b = g.start[row + lo[0]];
    *e = g.start[row + hi[0] + 1];
}

/* The exactness test: k results strictly inside the guard ball, with slack
 * for the rounding of the cell assignment and of s. */
__device__ __forceinline__ bool knn_exact(const GridView& g, bool finite, int len, int k, float kth, float guard)
{
    const float gs = guard - g.slack;
    return finite && len == k && (!isfinite(gs) || (gs > 0.0f && kth < gs * gs * 0.99999f));
}

/* Thread per query: the node at sorted position t (queries are the nodes;
 * neighbouring threads hold neighbouring nodes). */
__global__ void k_knn_grid(GridView g, int m, int k, int* out_idx, float* out_dist, int* redo, int* nredo)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        float qv[GPRM_MAX_DOF];
        const int qid = g.id[t];
        for (int j = 0; j < g.ndof; ++j) qv[j] = g.xs[t + (long long)g.n * j];
        float ts[NBR_MAX_K];
        int ti[NBR_MAX_K];
        int len = 0;
        TopkBound bound{INFINITY, 0x7fffffff};
        int lo[NBR_MAX_GRID], hi[NBR_MAX_GRID];
        float guard;
        const bool finite = query_block(g, qv, lo, hi, &guard);
        const int rows = block_rows(g, lo, hi);
        for (int r = 0; r < rows; ++r) {
            int b, e;
            block_row_range(g, lo, hi, r, &b, &e);
            int p = b;
            for (; p + 4 <= e; p += 4) {
                float s4[4];
                dist2_4(g.xs, g.n, p, qv, g.ndof, s4);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    float sd = s4[u];
                    if (p + u == t) continue;      /* the query itself */
                    if (sd != sd) sd = INFINITY;   /* NaN sorts last */
                    if (sd > bound.s) continue;    /* cannot enter the list */
                    const int nid = g.id[p + u];
                    if (!less_pair(sd, nid, bound.s, bound.i)) continue;
                    topk_insert(ts, ti, len, k, sd, nid);
                    topk_bound(ts, ti, len, k, bound);
                }
            }
            for (; p < e; ++p) {
                if (p == t) continue;
                float sd = dist2(g.xs, g.n, p, qv, g.ndof);
                if (sd != sd) sd = INFINITY;
                if (sd > bound.s) continue;
                const int nid = g.id[p];
                if (!less_pair(sd, nid, bound.s, bound.i)) continue;
                topk_insert(ts, ti, len, k, sd, nid);
                topk_bound(ts, ti, len, k, bound);
            }
        }
        if (knn_exact(g, finite, len, k, len ? ts[len - 1] : INFINITY, guard)) {
            for (int r = 0; r < k; ++r) {
                out_idx[(long long)qid * k + r] = ti[r];
                out_dist[(long long)qid * k + r] = sqrtf(ts[r]);
            }
        } else {
            redo[atomicAdd(nredo, 1)] = qid;
        }
    }
}

/* Merges the lanes' sorted top lists into the warp's k smallest (k rounds
 * of a warp argmin); every lane gets round r's winner in (ws, wi) when
 * r == its lane. */
__device__ __forceinline__ void warp_topk_merge(const float* ts, const int* ti, int len, int k, float* my_s, int* my_i,
                                                float* kth, int* found)
{
    const int lane = threadIdx.x & 31;
    int head = 0, cnt = 0;
    float last = INFINITY;
    *my_s = INFINITY;
    *my_i = -1;
    for (int r = 0; r < k; ++r) {
        float bs = head < len ? ts[head] : INFINITY;
        int bi = head < len ? ti[head] : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            const float os = __shfl_xor_sync(0xffffffffu, bs, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (less_pair(os, oi, bs, bi)) { bs = os; bi = oi; }
        }
        if (head < len && ti[head] == bi && ts[head] == bs) ++head;
        if (bi != 0x7fffffff) { ++cnt; last = bs; }
        if (lane == r) { *my_s = bs; *my_i = bi != 0x7fffffff ? bi : -1; }
    }
    *kth = last;
    *found = cnt;
}

/* Warp per query (outside queries q): lanes split the block's nodes. */
__global__ void k_knn_grid_warp(GridView g, const float* __restrict__ q, int m, long long qstride, int k,
                                int* out_idx, float* out_dist, int* redo, int* nredo)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int t = blockIdx.x * wpb + (threadIdx.x >> 5); t < m; t += gridDim.x * wpb) {
        float qv[GPRM_MAX_DOF];
        for (int j = 0; j < g.ndof; ++j) qv[j] = q[t + qstride * j];
        float ts[NBR_MAX_K];
        int ti[NBR_MAX_K];
        int len = 0;
        TopkBound bound{INFINITY, 0x7fffffff};
        int lo[NBR_MAX_GRID], hi[NBR_MAX_GRID];
        float guard;
        const bool finite = query_block(g, qv, lo, hi, &guard);
        const int rows = block_rows(g, lo, hi);
        /* many short rows (every joint gridded): the lanes split the rows;
           few long rows: the lanes split each row's nodes */
        const bool by_row = rows >= 32;
        for (int r = by_row ? lane : 0; r < rows; r += by_row ? 32 : 1) {
            int b, e;
            block_row_range(g, lo, hi, r, &b, &e);
            for (int p = b + (by_row ? 0 : lane); p < e; p += by_row ? 1 : 32) {
                float sd = dist2(g.xs, g.n, p, qv, g.ndof);
                if (sd != sd) sd = INFINITY;
                if (sd > bound.s) continue;
                const int nid = g.id[p];
                if (!less_pair(sd, nid, bound.s, bound.i)) continue;
                topk_insert(ts, ti, len, k, sd, nid);
                topk_bound(ts, ti, len, k, bound);
            }
        }
        float my_s, kth;
        int my_i, found;
        warp_topk_merge(ts, ti, len, k, &my_s, &my_i, &kth, &found);
        if (knn_exact(g, finite, found, k, kth, guard)) {
            if (lane < k) {
                out_idx[(long long)t * k + lane] = my_i;
                out_dist[(long long)t * k + lane] = sqrtf(my_s);
            }
        } else if (lane == 0) {
            redo[atomicAdd(nredo, 1)] = t;
        }
    }
}

/* Second try for the queries the 3^ndof block could not settle: one block
 * of threads per query scans the 5^ndof block around it (its rows split
 * over the threads, each keeping its own top-k, merged as in k_knn_full)
 * and applies the same exactness test with that block's guard; a query it
 * cannot settle either goes to the full scan (redo2). */
__global__ void __launch_bounds__(256) k_knn_wide(GridView g, const float* __restrict__ q, long long qstride, int k,
                                                  int exclude_self, const int* __restrict__ redo,
                                                  const int* __restrict__ nredo, int* redo2, int* nredo2,
                                                  int* out_idx, float* out_dist)
{
    __shared__ float ms[8 * NBR_MAX_K];
    __shared__ int mi[8 * NBR_MAX_K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cnt = *nredo;
    for (int w = blockIdx.x; w < cnt; w += gridDim.x) {
        const int qid = redo[w];
        float qv[GPRM_MAX_DOF];
        for (int j = 0; j < g.ndof; ++j) qv[j] = q[qid + qstride * j];
        float ts[NBR_MAX_K];
        int ti[NBR_MAX_K];
        int len = 0;
        TopkBound bound{INFINITY, 0x7fffffff};
        int lo[NBR_MAX_GRID], hi[NBR_MAX_GRID];
        float guard;
        const bool finite = query_block(g, qv, lo, hi, &guard, 2);
        const int rows = block_rows(g, lo, hi);
        for (int r = threadIdx.x; r < rows; r += blockDim.x) {
            int b, e;
            block_row_range(g, lo, hi, r, &b, &e);
            for (int p = b; p < e; ++p) {
                const int nid = g.id[p];
                if (exclude_self && nid == qid) continue;
                float sd = dist2(g.xs, g.n, p, qv, g.ndof);
                if (sd != sd) sd = INFINITY;
                if (!less_pair(sd, nid, bound.s, bound.i)) continue;
                topk_insert(ts, ti, len, k, sd, nid);
                topk_bound(ts, ti, len, k, bound);
            }
        }
        float my_s, kth;
        int my_i, found;
        warp_topk_merge(ts, ti, len, k, &my_s, &my_i, &kth, &found);
        if (lane < k) {
            ms[warp * k + lane] = my_s;
            mi[warp * k + lane] = my_i < 0 ? 0x7fffffff : my_i;
        }
        __syncthreads();
        if (warp == 0) {
            len = 0;
            bound = TopkBound{INFINITY, 0x7fffffff};
            for (int e = lane; e < 8 * k; e += 32) {
                if (mi[e] == 0x7fffffff) continue;
                if (!less_pair(ms[e], mi[e], bound.s, bound.i)) continue;
                topk_insert(ts, ti, len, k, ms[e], mi[e]);
                topk_bound(ts, ti, len, k, bound);
            }
            warp_topk_merge(ts, ti, len, k, &my_s, &my_i, &kth, &found);
            if (knn_exact(g, finite, found, k, kth, guard)) {
                if (lane < k) {
                    out_idx[(long long)qid * k + lane] = my_i;
                    out_dist[(long long)qid * k + lane] = sqrtf(my_s);
                }
            } else if (lane == 0) {
                redo2[atomicAdd(nredo2, 1)] = qid;
            }
        }
        __syncthreads();
    }
}

/* Redo of the queries the grid could not settle: one block per query scans
 * every node (each thread four consecutive nodes at a time, keeping its own
 * top-k); each warp merges its lanes' lists by k rounds of a warp argmin,
 * then warp 0 merges the eight warp lists the same way. */
__global__ void __launch_bounds__(256) k_knn_full(const float* __restrict__ x, int n, long long xstride,
                                                  const float* __restrict__ q, long long qstride, int ndof, int k,
                                                  int exclude_self, const int* __restrict__ redo,
                                                  const int* __restrict__ nredo, int* out_idx, float* out_dist)
{
    __shared__ float ms[8 * NBR_MAX_K];
    __shared__ int mi[8 * NBR_MAX_K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cnt = *nredo;
    for (int w = blockIdx.x; w < cnt; w += gridDim.x) {
        const int qid = redo[w];
        float qv[GPRM_MAX_DOF];
        for (int j = 0; j < ndof; ++j) qv[j] = q[qid + qstride * j];
        float ts[NBR_MAX_K];
        int ti[NBR_MAX_K];
        int len = 0;
        TopkBound bound{INFINITY, 0x7fffffff};
        /* thread t takes nodes 4t.. 4t+3, 4(t+256).. : four loads in flight */
        for (int i0 = 4 * threadIdx.x; i0 < n; i0 += 4 * 256) {
            float s4[4];
            if (i0 + 4 <= n) {
                dist2_4(x, xstride, i0, qv, ndof, s4);
            } else {
                for (int u = 0; u < 4; ++u) s4[u] = i0 + u < n ? dist2(x, xstride, i0 + u, qv, ndof) : INFINITY;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = i0 + u;
                if (i >= n || (exclude_self && i == qid)) continue;
                float s = s4[u];
                if (s != s) s = INFINITY;   /* NaN sorts last */
                if (!less_pair(s, i, bound.s, bound.i)) continue;
                topk_insert(ts, ti, len, k, s, i);
                topk_bound(ts, ti, len, k, bound);
            }
        }
        /* per warp: the k smallest of its lanes; then warp 0 merges the 8 lists */
        float my_s, kth;
        int my_i, found;
        warp_topk_merge(ts, ti, len, k, &my_s, &my_i, &kth, &found);
        if (lane < k) {
            ms[warp * k + lane] = my_s;
            mi[warp * k + lane] = my_i < 0 ? 0x7fffffff : my_i;
        }
        __syncthreads();
        if (warp == 0) {
            len = 0;
            bound = TopkBound{INFINITY, 0x7fffffff};
            for (int e = lane; e < 8 * k; e += 32) {
                if (mi[e] == 0x7fffffff) continue;
                if (!less_pair(ms[e], mi[e], bound.s, bound.i)) continue;
                topk_insert(ts, ti, len, k, ms[e], mi[e]);
                topk_bound(ts, ti, len, k, bound);
            }
            warp_topk_merge(ts, ti, len, k, &my_s, &my_i, &kth, &found);
            if (lane < k) {
                const bool have = my_i >= 0;
                out_idx[(long long)qid * k + lane] = have ? my_i : -1;
                out_dist[(long long)qid * k + lane] = have ? sqrtf(my_s) : INFINITY;
            }
        }
        __syncthreads();
    }
}

}  // namespace

struct gprm_nbr {
    int ndof = 0;
    int device = 0;
    int sms = 0;
    int n = 0;
    GridView g{};
    const float* x = nullptr;     /* caller's nodes (kept for radius and the redo path) */
    long long xstride = 0;
    float* xs = nullptr;
    int* id = nullptr;
    int* start = nullptr;
    int* key = nullptr;
    int* count = nullptr;
    int* cursor = nullptr;
    float* mm = nullptr;
    int* redo = nullptr;
    int* nredo = nullptr;          /* [0]: queries the 3^ndof block left, [1]: the 5^ndof block */
    int* redo2 = nullptr;
    size_t cap_xs = 0, cap_id = 0, cap_key = 0, cap_start = 0, cap_count = 0, cap_cursor = 0, cap_redo = 0,
           cap_redo2 = 0;
    std::string err = "no error";
};

namespace {

thread_local std::string g_nbr_create_error = "no error";

int nfail(gprm_nbr* h, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    else g_nbr_create_error = buf;
    return code;
}

#define NBR_TRY(h, call)                                                                    \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return nfail((h), e_ == cudaErrorMemoryAllocation ? GPRM_ERR_NOMEM : GPRM_ERR_CUDA, \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

template <class T>
int grow(gprm_nbr* h, T** p, size_t& cap, size_t need)
{
    if (need <= cap && *p) return GPRM_OK;
    cudaFree(*p);
    *p = nullptr;
    size_t c = need + need / 4 + 16;
    NBR_TRY(h, cudaMalloc((void**)p, c * sizeof(T)));
    cap = c;
    return GPRM_OK;
}

}  // namespace

extern "C" {

int gprm_nbr_create(int ndof, gprm_nbr** out)
{
    if (!out) return nfail(nullptr, GPRM_ERR_ARG, "null output");
    *out = nullptr;
    if (ndof < 1 || ndof > GPRM_MAX_DOF) return nfail(nullptr, GPRM_ERR_ARG, "ndof %d outside 1..%d", ndof, GPRM_MAX_DOF);
    gprm_nbr* h = new gprm_nbr();
    h->ndof = ndof;
    if (cudaGetDevice(&h->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess) {
        delete h;
        return nfail(nullptr, GPRM_ERR_CUDA, "no CUDA device");
    }
    *out = h;
    return GPRM_OK;
}

void gprm_nbr_destroy(gprm_nbr* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    cudaFree(h->xs);
    cudaFree(h->id);
    cudaFree(h->start);
    cudaFree(h->key);
    cudaFree(h->count);
    cudaFree(h->cursor);
    cudaFree(h->mm);
    cudaFree(h->redo);
    cudaFree(h->redo2);
    cudaFree(h->nredo);
    delete h;
}

const char* gprm_nbr_last_error(const gprm_nbr* h) { return h ? h->err.c_str() : g_nbr_create_error.c_str(); }

int gprm_nbr_build(gprm_nbr* h, const float* x, int n, int stride, float cell, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (n < 0 || (n > 0 && !x) || stride < n) return nfail(h, GPRM_ERR_ARG, "bad x/n/stride");
    if (!(cell >= 0.0f) || !isfinite(cell)) return nfail(h, GPRM_ERR_ARG, "cell must be finite and >= 0");
    NBR_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    /* every joint is gridded: a query's block of 3^ndof cells then holds
       about 3^ndof x (nodes per cell) candidates, far fewer than a grid over
       some joints whose block spans the others' whole range */
    const int nd = h->ndof, G = nd < NBR_MAX_GRID ? nd : NBR_MAX_GRID;
    h->n = n;
    h->x = x;
    h->xstride = stride;
    GridView& g = h->g;
    g = GridView{};
    g.ndof = nd;
    g.G = G;
    g.n = n;
    int rc;
    if (!h->mm) NBR_TRY(h, cudaMalloc((void**)&h->mm, 2 * GPRM_MAX_DOF * sizeof(float)));
    if (!h->nredo) NBR_TRY(h, cudaMalloc((void**)&h->nredo, 2 * sizeof(int)));
    std::vector<float> mm(2 * nd);
    for (int j = 0; j < nd; ++j) { mm[2 * j] = INFINITY; mm[2 * j + 1] = -INFINITY; }
    NBR_TRY(h, cudaMemcpyAsync(h->mm, mm.data(), 2 * nd * sizeof(float), cudaMemcpyHostToDevice, st));
    if (n > 0) k_minmax<<<h->sms * 4, 256, 0, st>>>(x, n, stride, nd, h->mm);
    NBR_TRY(h, cudaGetLastError());
    NBR_TRY(h, cudaMemcpyAsync(mm.data(), h->mm, 2 * nd * sizeof(float), cudaMemcpyDeviceToHost, st));
    NBR_TRY(h, cudaStreamSynchronize(st));
    /* cell size: given, or about the distance of the 16th neighbour of
       uniformly spread nodes (full-dimensional estimate) */
    double vol = 1.0;
    for (int j = 0; j < nd; ++j) {
        double e = (n > 0 && mm[2 * j + 1] > mm[2 * j]) ? (double)mm[2 * j + 1] - mm[2 * j] : 1e-3;
        vol *= e;
    }
    double c = cell;
    if (!(c > 0.0)) {
        const double unit = pow(M_PI, nd / 2.0) / tgamma(nd / 2.0 + 1.0);
        c = 1.1 * pow(16.0 * vol / ((n > 0 ? n : 1) * unit), 1.0 / nd);
    }
    long long ncells = 1;
    for (int d = 0; d < G; ++d) {
        const double e = (n > 0 && mm[2 * d + 1] > mm[2 * d]) ? (double)mm[2 * d + 1] - mm[2 * d] : 0.0;
        long long k = (long long)ceil(e / c);
        if (k < 1) k = 1;
        if (k > 1024) k = 1024;
        g.nc[d] = (int)k;
        g.lo[d] = n > 0 ? mm[2 * d] : 0.0f;
        ncells *= k;
    }
    while (ncells > NBR_MAX_CELLS) {   /* coarsen until the grid fits */
        c *= 1.25;
        ncells = 1;
        for (int d = 0; d < G; ++d) {
            const double e = (double)mm[2 * d + 1] - mm[2 * d];
            long long k = (long long)ceil(e / c);
            g.nc[d] = (int)(k < 1 ? 1 : k);
            ncells *= g.nc[d];
        }
    }
    g.cell = (float)c;
    g.inv_cell = (float)(1.0 / c);
    /* slack of the exactness test: rounding of the cell assignment and of
       the block faces, relative to the coordinates' magnitude */
    double mag = 0.0;
    for (int d = 0; d < G; ++d) mag = fmax(mag, fabs((double)g.lo[d]) + g.nc[d] * c);
    g.slack = (float)(1e-5 * c + 1e-6 * mag);
    /* buffers only grow, so rebuilding an index allocates nothing */
    if ((rc = grow(h, &h->xs, h->cap_xs, (size_t)n * nd + 1)) != GPRM_OK) return rc;
    if ((rc = grow(h, &h->id, h->cap_id, (size_t)n + 1)) != GPRM_OK) return rc;
    if ((rc = grow(h, &h->key, h->cap_key, (size_t)n + 1)) != GPRM_OK) return rc;
    if ((rc = grow(h, &h->start, h->cap_start, (size_t)ncells + 1)) != GPRM_OK) return rc;
    if ((rc = grow(h, &h->count, h->cap_count, (size_t)ncells)) != GPRM_OK) return rc;
    if ((rc = grow(h, &h->cursor, h->cap_cursor, (size_t)ncells)) != GPRM_OK) return rc;
    NBR_TRY(h, cudaMemsetAsync(h->count, 0, (size_t)ncells * sizeof(int), st));
    NBR_TRY(h, cudaMemsetAsync(h->cursor, 0, (size_t)ncells * sizeof(int), st));
    if (n > 0) k_cell_keys<<<h->sms * 8, 256, 0, st>>>(x, n, stride, g, h->key, h->count);
    k_scan<<<1, 1024, 0, st>>>(h->count, (int)ncells, h->start);
    if (n > 0) k_scatter<<<h->sms * 8, 256, 0, st>>>(x, n, stride, nd, h->key, h->start, h->cursor, h->xs, h->id);
    NBR_TRY(h, cudaGetLastError());
    g.xs = h->xs;
    g.id = h->id;
    g.start = h->start;
    return GPRM_OK;
}

int gprm_nbr_radius(gprm_nbr* h, const float* q, int m, int qstride, float D, int cap, int* counts, int* idx,
                    float* dist, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (m < 0 || (m > 0 && (!q || !counts || !idx || !dist)) || qstride < m || cap < 1)
        return nfail(h, GPRM_ERR_ARG, "bad q/m/qstride/cap/outputs");
    if (!(D >= 0.0f) || !isfinite(D)) return nfail(h, GPRM_ERR_ARG, "D must be finite and >= 0");
    if (m == 0) return GPRM_OK;
    NBR_TRY(h, cudaSetDevice(h->device));
    const float D2 = D * D;   /* D2 = D*D in float, prmsolver.cpp:71 */
    k_radius<<<h->sms * 8, 256, 0, (cudaStream_t)stream>>>(h->x, h->n, h->xstride, q, m, qstride, h->ndof, D2, cap,
                                                           counts, idx, dist);
    NBR_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

int gprm_nbr_knn(gprm_nbr* h, const float* q, int m, int qstride, int k, int queries_are_nodes, int* idx,
                 float* dist, void* stream)
{
    if (!h) return GPRM_ERR_ARG;
    if (k < 1 || k > NBR_MAX_K) return nfail(h, GPRM_ERR_ARG, "k=%d outside 1..%d", k, NBR_MAX_K);
    if (queries_are_nodes) {
        q = h->x;
        m = h->n;
        qstride = (int)h->xstride;
    }
    if (m < 0 || (m > 0 && (!q || !idx || !dist)) || qstride < m) return nfail(h, GPRM_ERR_ARG, "bad q/m/qstride/outputs");
    if (m == 0) return GPRM_OK;
    NBR_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    int rc = grow(h, &h->redo, h->cap_redo, (size_t)m);
    if (rc) return rc;
    if ((rc = grow(h, &h->redo2, h->cap_redo2, (size_t)m))) return rc;
    NBR_TRY(h, cudaMemsetAsync(h->nredo, 0, 2 * sizeof(int), st));
    if (queries_are_nodes) {
        const int threads = 128;
        const int blocks = (int)((m + threads - 1) / threads);
        k_knn_grid<<<blocks, threads, 0, st>>>(h->g, m, k, idx, dist, h->redo, h->nredo);
    } else {
        const int wpb = 8;
        const long long wblocks = ((long long)m + wpb - 1) / wpb;
        const int blocks = (int)(wblocks < (long long)h->sms * 16 ? wblocks : (long long)h->sms * 16);
        k_knn_grid_warp<<<blocks, 32 * wpb, 0, st>>>(h->g, q, m, qstride, k, idx, dist, h->redo, h->nredo);
    }
    NBR_TRY(h, cudaGetLastError());
    k_knn_wide<<<h->sms * 8, 256, 0, st>>>(h->g, q, qstride, k, queries_are_nodes ? 1 : 0, h->redo, h->nredo,
                                           h->redo2, h->nredo + 1, idx, dist);
    NBR_TRY(h, cudaGetLastError());
    k_knn_full<<<h->sms * 8, 256, 0, st>>>(h->x, h->n, h->xstride, q, qstride, h->ndof, k, queries_are_nodes ? 1 : 0,
                                           h->redo2, h->nredo + 1, idx, dist);
    NBR_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

int gprm_nbr_redo_count(gprm_nbr* h, int* out)
{
    if (!h || !out) return GPRM_ERR_ARG;
    NBR_TRY(h, cudaSetDevice(h->device));
    NBR_TRY(h, cudaMemcpy(out, h->nredo, sizeof(int), cudaMemcpyDeviceToHost));
    return GPRM_OK;
}

}  /* extern "C" */

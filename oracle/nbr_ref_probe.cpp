/*
 * nbr_ref_probe.cpp - C ABI over the reference planner's own radius search,
 * PRMSolver<ndof>::get_near_vertices (prm/src/lib/prm/prmsolver.cpp:
 * 2533-2574), compiled from the reference sources.
 *
 * TEST INFRASTRUCTURE ONLY: pins oracle/nbr_oracle.py.  The nodes are
 * inserted into the solver's left graph with its own insert()
 * (prmsolver.cpp:2408-2469, key blocks of width H over joint 0); a query
 * returns the neighbours within D in the solver's block order, mapped back
 * to the caller's node indices.  The members are private in the reference
 * header, so this translation unit opens them.
 *
 * ref_random_nodes runs the planner's node sampler get_random_nodes
 * (prmsolver.cpp:2585-2624) on such a graph (pins oracle/sampler_oracle.py
 * and the batched sampler distributionally).
 */
#include <mpi.h>

/* standard headers first, so that only the planner's classes are opened */
#include <assert.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <fstream>
#include <iostream>
#include <map>
#include <queue>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "prm/prmsolver.cpp"
#undef private
#undef protected

template class PRMSolver<6>;

template <int ndof>
static int near_impl(const float* x, int n, const float* q, int m, float D, float H, int nbuf, int* counts,
                     int* idx, float* dist)
{
    PRMSolver<ndof>* s = new PRMSolver<ndof>(nullptr, H, D, n + 256 * 64, 256);
    std::vector<int> node_of(n + 1024 * 256, -1);
    for (int i = 0; i < n; ++i) {
        float v[ndof];
        for (int j = 0; j < ndof; ++j) v[j] = x[(size_t)i * ndof + j];
        int pos = s->insert(v, 1, s->graphl);
        if (pos < 0 || pos >= (int)node_of.size()) { delete s; return -1; }
        node_of[pos] = i;
    }
    std::vector<float> qlist((size_t)ndof * nbuf);
    std::vector<int> posq(nbuf);
    std::vector<float> dl(nbuf);
    for (int t = 0; t < m; ++t) {
        int w = s->get_near_vertices(&q[(size_t)t * ndof], 1, qlist.data(), posq.data(), dl.data(), nbuf, nbuf,
                                     s->graphl);
        counts[t] = w;
        for (int r = 0; r < w; ++r) {
            idx[(size_t)t * nbuf + r] = node_of[posq[r]];
            dist[(size_t)t * nbuf + r] = dl[r];
        }
    }
    delete s;
    return 0;
}

/* x: (n, ndof) and q: (m, ndof) row-major; outputs (m, nbuf). */
extern "C" int ref_near_vertices(int ndof, const float* x, int n, const float* q, int m, float D, float H, int nbuf,
                                 int* counts, int* idx, float* dist)
{
    if (ndof == 4) return near_impl<4>(x, n, q, m, D, H, nbuf, counts, idx, dist);
    if (ndof == 6) return near_impl<6>(x, n, q, m, D, H, nbuf, counts, idx, dist);
    return -2;
}

/* do_dijkstra (prmsolver.cpp:2805-2846) on a graph of n nodes x (n, ndof)
 * and m undirected edges (eu[e], ev[e], weight w[e]), entered the way
 * processing_step_part3a stores them (prmsolver.cpp:2111-2126: both
 * directions, in edge order).  Writes the path (node indices, goal first, as
 * the reference builds it) and returns its length, 0 when there is none,
 * <0 on error; *dist_to gets the goal's distance. */
template <int ndof>
static int dijkstra_impl(const float* x, int n, const int* eu, const int* ev, const float* w, int m, int from,
                         int to, int* path, int path_cap, float* dist_to)
{
    PRMSolver<ndof>* s = new PRMSolver<ndof>(nullptr, 1.0f, 1.0f, n + 256 * 64, 256);
    auto& g = s->graphl;   /* its type is private to the class: name it through the member */
    g.edgelists.resize(n + 256 * 1024);
    g.edgeweights.resize(n + 256 * 1024);
    std::vector<int> pos_of(n), node_of(n + 256 * 1024, -1);
    for (int i = 0; i < n; ++i) {
        float v[ndof];
        for (int j = 0; j < ndof; ++j) v[j] = x[(size_t)i * ndof + j];
        int p = s->insert(v, 1, g);
        if (p < 0 || p >= (int)node_of.size()) { delete s; return -1; }
        pos_of[i] = p;
        node_of[p] = i;
    }
    for (int e = 0; e < m; ++e) {
        const int a = pos_of[eu[e]], b = pos_of[ev[e]];
        g.edgelists[a].push_back(b);
        g.edgeweights[a].push_back(w[e]);
        g.edgelists[b].push_back(a);
        g.edgeweights[b].push_back(w[e]);
    }
    decltype(s->dijkstral) d;
    const int found = s->do_dijkstra(g, d, pos_of[from], pos_of[to]);
    int len = 0;
    if (found) {
        len = (int)d.path.size();
        if (len > path_cap) { delete s; return -2; }
        for (int k = 0; k < len; ++k) path[k] = node_of[d.path[k]];
        *dist_to = d.dist[pos_of[to]];
    }
    delete s;
    return len;
}

extern "C" int ref_dijkstra(int ndof, const float* x, int n, const int* eu, const int* ev, const float* w, int m,
                            int from, int to, int* path, int path_cap, float* dist_to)
{
    if (ndof == 4) return dijkstra_impl<4>(x, n, eu, ev, w, m, from, to, path, path_cap, dist_to);
    if (ndof == 6) return dijkstra_impl<6>(x, n, eu, ev, w, m, from, to, path, path_cap, dist_to);
    return -3;
}

/* A Configspace<ndof> whose indicator(q) reports a collision exactly when
 * q[0] > wall: the sampler's only call into the space. */
template <int ndof>
class WallSpace : public Configspace<ndof>
{
public:
    explicit WallSpace(float wall) : wall_(wall) {}
    int init(const int, const int) override { return 0; }
    int indicator(const float* q, int* res, const int N, const int offset) override
    {
        for (int i = 0; i < N; ++i) res[i] = q[i] > wall_ ? 1 : 0;
        (void)offset;
        return 0;
    }
    int indicator(const float* q) override { return q[0] > wall_ ? 1 : 0; }
    int indicator2(const float*, const float*, int*, const int, const int) override { return -1; }
    int indicator2_async(const float*, const float*, int*, const int, const int, int&) override { return -1; }
    int indicator2_async_wait(int) override { return -1; }
    int indicator2(const float*, const int, const float*, int*, const int*, const int*, const int) override
    {
        return -1;
    }
    int check_boundaries(const float*, int*, const int, const int) override { return -1; }
    int check_boundaries(const float*) override { return -1; }
    float min(int) override { return -1e30f; }
    float max(int) override { return 1e30f; }
    float deltaq() override { return 0.01f; }
    int dim() override { return ndof; }

private:
    float wall_;
};

template <int ndof>
static int random_impl(const float* x, int n, const int* surrnum, float H, float D, float wall, int seed, int num,
                       float* q_out, int* slot_of, int* block_pos, int* block_num, int* nblocks,
                       long long* counters)
{
    PRMSolver<ndof>* s = new PRMSolver<ndof>(nullptr, H, D, n + 256 * 64, 256);
    auto& g = s->graphl;
    for (int i = 0; i < n; ++i) {
        float v[ndof];
        for (int j = 0; j < ndof; ++j) v[j] = x[(size_t)i * ndof + j];
        int p = s->insert(v, 1, g);
        if (p < 0) { delete s; return -1; }
        slot_of[i] = p;
        g.surrnum[p] = surrnum[i];
    }
    *nblocks = g.blocknum;
    for (int b = 0; b < g.blocknum; ++b) {
        block_pos[b] = g.blocks[b].pos;
        block_num[b] = g.blocks[b].num;
    }
    WallSpace<ndof> space(wall);
    PRMSolver<ndof>::rand_nodes_all = 0;
    PRMSolver<ndof>::rand_nodes_dismissed_prob = 0;
    PRMSolver<ndof>::rand_nodes_accepted = 0;
    PRMSolver<ndof>::rand_block_numbers = 0;
    srand(seed);
    s->get_random_nodes(g, 0, num, q_out, D, &space);
    counters[0] = PRMSolver<ndof>::rand_nodes_all;
    counters[1] = PRMSolver<ndof>::rand_nodes_dismissed_prob;
    counters[2] = PRMSolver<ndof>::rand_nodes_accepted;
    counters[3] = PRMSolver<ndof>::rand_block_numbers;
    delete s;
    return 0;
}

/* x: (n, ndof) nodes inserted in order (keys of width H over joint 0) with
 * surrnum[i]; draws num free nodes (free: q[0] <= wall) into q_out (num,
 * ndof) after srand(seed).  slot_of[i]: node i's storage slot; the graph's
 * blocks (pos, num) go to block_pos/block_num (capacity n + 64), their count
 * to *nblocks; counters: rand_nodes_all, rand_nodes_dismissed_prob,
 * rand_nodes_accepted, rand_block_numbers. */
extern "C" int ref_random_nodes(int ndof, const float* x, int n, const int* surrnum, float H, float D, float wall,
                                int seed, int num, float* q_out, int* slot_of, int* block_pos, int* block_num,
                                int* nblocks, long long* counters)
{
    if (ndof == 4)
        return random_impl<4>(x, n, surrnum, H, D, wall, seed, num, q_out, slot_of, block_pos, block_num, nblocks,
                              counters);
    if (ndof == 6)
        return random_impl<6>(x, n, surrnum, H, D, wall, seed, num, q_out, slot_of, block_pos, block_num, nblocks,
                              counters);
    return -3;
}

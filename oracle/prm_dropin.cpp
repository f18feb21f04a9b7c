/*
 * prm_dropin.cpp - runs GPUPRM's own planner, PRMSolver<4>::process_mpi5
 * (prm/src/lib/prm/prmsolver.cpp:1765), compiled from the reference's
 * unmodified sources, with either collision checker behind its
 * Configspace<4> interface (prm/src/lib/prm/configspace.hpp:10-50):
 *
 *   --checker ref   RobotConfigspace<4>, the reference's CPU checker
 *                   (robotconfigspace.cpp, built without GPU_VERSION)
 *   --checker b200  B200RobotConfigspace<4> (include/gprm_configspace.hpp)
 *                   over libgprm_b200.so
 *
 * TEST INFRASTRUCTURE ONLY: it demonstrates the drop-in boundary and lets
 * a test compare the two runs.  The flow follows the reference's
 * prm/src/main.cpp:30-190 (seeding, start (0,0,0,0), goal (3,3,3,3),
 * process_mpi5, store_results); MPI is the single-rank stand-in of
 * oracle/mpi_single/mpi.h.  The planner's console output goes to
 * /dev/null; one JSON line with the timing and counters goes to stdout.
 *
 * prmsolver.cpp is compiled in its own translation unit at -O0 with
 * -fno-unreachable-traps (oracle/Makefile): its get_random_nodes{,2} are
 * declared to return int but end without a return statement
 * (prmsolver.cpp:2585-2698), undefined behaviour that current g++ turns
 * into a loop running past its bound at -O1 and above, and into a trap at
 * -O0 unless unreachable traps are off.
 *
 * --dump DIR writes the planner's final roadmaps as raw arrays (blocks,
 * node storage, adjacency with float weights, start/end positions, the
 * Dijkstra path) so that a test can feed them to another store_results
 * writer and compare its files with the planner's own.
 *
 * --start / --goal a,b,c,d replace main.cpp's start (0,0,0,0) and goal
 * (3,3,3,3) (for scenes where those are not free).
 *
 * --mode fp32 (default) runs the B200 checker in FP32 mode, whose verdicts
 * equal the reference's, so both runs draw the same random numbers and
 * build the same roadmap; --mode band enables the FP64 near-contact recheck.
 */
#include <mpi.h>

/* standard headers first: the planner's members are opened for --dump only */
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
#include "prm/prmsolver.h"
#undef private
#undef protected
#include "robotspace/robotconfigspace.cpp"
#include "gprm_configspace.hpp"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

/* Forwards every call to another Configspace<4> and, when a trace file is
 * given, records each verdict the planner asked for: 'V' records (q[4],
 * code) for indicator(q), 'E' records (N, then per edge qs[4], qe[4], res)
 * for each indicator2 request once its results are known.  Two traces of
 * the same planner run agree record by record up to the first verdict in
 * which the checkers differ. */
class TracingSpace : public Configspace<4>
{
public:
    TracingSpace(Configspace<4>* inner, FILE* f) : in_(inner), f_(f) {}
    int init(const int r = 0, const int s = 1) { return in_->init(r, s); }
    int indicator(const float* q, int* res, const int N, const int offset) { return in_->indicator(q, res, N, offset); }
    int indicator(const float* q)
    {
        int code = in_->indicator(q);
        if (f_) { fputc('V', f_); fwrite(q, sizeof(float), 4, f_); fwrite(&code, sizeof(int), 1, f_); }
        return code;
    }
    int indicator2(const float* qs, const float* qe, int* res, const int N, const int offset)
    {
        int rc = in_->indicator2(qs, qe, res, N, offset);
        log_edges(qs, qe, res, N, offset);
        return rc;
    }
    int indicator2_async(const float* qs, const float* qe, int* res, const int N, const int offset, int& request)
    {
        int rc = in_->indicator2_async(qs, qe, res, N, offset, request);
        pending_[request] = Pending{qs, qe, res, N, offset};
        return rc;
    }
    int indicator2_async_wait(int request)
    {
        int rc = in_->indicator2_async_wait(request);
        auto it = pending_.find(request);
        if (it != pending_.end()) {
            log_edges(it->second.qs, it->second.qe, it->second.res, it->second.n, it->second.offset);
            pending_.erase(it);
        }
        return rc;
    }
    int indicator2(const float* qs, const int M, const float* qe, int* res, const int* posqe, const int* numqe,
                   const int offset)
    {
        return in_->indicator2(qs, M, qe, res, posqe, numqe, offset);
    }
    int check_boundaries(const float* q, int* res, const int N, const int offset)
    {
        return in_->check_boundaries(q, res, N, offset);
    }
    int check_boundaries(const float* q) { return in_->check_boundaries(q); }
    float min(int i) { return in_->min(i); }
    float max(int i) { return in_->max(i); }
    float deltaq() { return in_->deltaq(); }
    int dim() { return in_->dim(); }

private:
    struct Pending { const float* qs; const float* qe; int* res; int n; int offset; };
    void log_edges(const float* qs, const float* qe, const int* res, int n, int offset)
    {
        if (!f_) return;
        fputc('E', f_);
        fwrite(&n, sizeof(int), 1, f_);
        for (int k = 0; k < n; ++k) {
            float a[4], b[4];
            for (int j = 0; j < 4; ++j) { a[j] = qs[k + offset * j]; b[j] = qe[k + offset * j]; }
            fwrite(a, sizeof(float), 4, f_);
            fwrite(b, sizeof(float), 4, f_);
            fwrite(&res[k], sizeof(int), 1, f_);
        }
    }
    Configspace<4>* in_;
    FILE* f_;
    std::map<int, Pending> pending_;
};

template <class T>
static void dump_array(const std::string& path, const T* p, size_t n)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return;
    if (n) fwrite(p, sizeof(T), n, f);
    fclose(f);
}

/* One roadmap as raw arrays: meta = [ndof, blocknum, newblockpos, start,
 * end, path length]; blocks = (pos, num) per block; qstorage; surrnum;
 * adjacency in CSR over positions with float weights; path positions. */
template <class G, class D>
static void dump_graph(const std::string& dir, const G& g, const D& d, int start, int end, bool with_path)
{
    const int n = g.newblockpos;
    std::vector<int> meta = {4, g.blocknum, n, start, end, with_path ? (int)d.path.size() : 0};
    dump_array(dir + "/meta.bin", meta.data(), meta.size());
    std::vector<int> blocks;
    for (int l = 0; l < g.blocknum; ++l) { blocks.push_back(g.blocks[l].pos); blocks.push_back(g.blocks[l].num); }
    dump_array(dir + "/blocks.bin", blocks.data(), blocks.size());
    dump_array(dir + "/qstorage.bin", g.qstorage.data(), (size_t)4 * n);
    dump_array(dir + "/surrnum.bin", g.surrnum.data(), (size_t)n);
    std::vector<int> off(1, 0), dest;
    std::vector<float> w;
    for (int p = 0; p < n; ++p) {
        for (size_t i = 0; i < g.edgelists[p].size(); ++i) { dest.push_back(g.edgelists[p][i]); w.push_back(g.edgeweights[p][i]); }
        off.push_back((int)dest.size());
    }
    dump_array(dir + "/adj_off.bin", off.data(), off.size());
    dump_array(dir + "/adj_dest.bin", dest.data(), dest.size());
    dump_array(dir + "/adj_w.bin", w.data(), w.size());
    if (with_path) dump_array(dir + "/path.bin", d.path.data(), d.path.size());
}

int main(int argc, char** argv)
{
    std::string checker = "ref", config, out, mode = "fp32", trace, dump;
    int num = 32, nbuf = 2048, seed = 0, blocksize = 256, workerversion = 1, maxsteps = 10000;
    int maxstorage = 1024 * 1024;
    float dq = 0.01f, distD = 1.0f, distH = 1.0f;
    float qstart[4] = {0, 0, 0, 0}, qend[4] = {3, 3, 3, 3};
    auto parse4 = [](const std::string& v, float* q) {
        return sscanf(v.c_str(), "%f,%f,%f,%f", &q[0], &q[1], &q[2], &q[3]) == 4;
    };
    for (int i = 1; i + 1 < argc; i += 2) {
        std::string k = argv[i], v = argv[i + 1];
        if (k == "--checker") checker = v;
        else if (k == "--config") config = v;
        else if (k == "--out") out = v;
        else if (k == "--num") num = atoi(v.c_str());
        else if (k == "--nbuf") nbuf = atoi(v.c_str());
        else if (k == "--seed") seed = atoi(v.c_str());
        else if (k == "--dq") dq = (float)atof(v.c_str());
        else if (k == "--distD") distD = (float)atof(v.c_str());
        else if (k == "--distH") distH = (float)atof(v.c_str());
        else if (k == "--maxsteps") maxsteps = atoi(v.c_str());
        else if (k == "--workerversion") workerversion = atoi(v.c_str());
        else if (k == "--blocksize") blocksize = atoi(v.c_str());
        else if (k == "--mode") mode = v;
        else if (k == "--trace") trace = v;
        else if (k == "--dump") dump = v;
        else if (k == "--start") { if (!parse4(v, qstart)) { fprintf(stderr, "bad --start\n"); return 2; } }
        else if (k == "--goal") { if (!parse4(v, qend)) { fprintf(stderr, "bad --goal\n"); return 2; } }
        else { fprintf(stderr, "unknown argument %s\n", k.c_str()); return 2; }
    }
    if (config.empty() || out.empty() || (checker != "ref" && checker != "b200")) {
        fprintf(stderr, "usage: prm_dropin --checker ref|b200 --config DIR --out DIR [...]\n");
        return 2;
    }
    /* the planner prints to stdout; keep fd 1 for the result line */
    fflush(stdout);
    const int saved = dup(1);
    const int nul = open("/dev/null", O_WRONLY);
    dup2(nul, 1);
    close(nul);

    MPI_Init(&argc, &argv);
    const int confignbuf = 2 * nbuf;
    srand(seed);   /* main.cpp:112 with rank 0 */
    const int firstrand = rand();
    (void)firstrand;

    Configspace<4>* space = nullptr;
    RobotConfigspace<4>* ref = nullptr;
    B200RobotConfigspace<4>* b200 = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    try {
        if (checker == "ref") {
            ref = new RobotConfigspace<4>(config, dq, confignbuf);
            ref->init(0, 1);
            space = ref;
        } else {
            b200 = new B200RobotConfigspace<4>(config, dq, confignbuf);
            b200->init(0, 1);
            if (gprm_set_mode(b200->handle(), mode == "band" ? GPRM_MODE_FP64_BAND : GPRM_MODE_FP32) != GPRM_OK)
                throw std::runtime_error("gprm_set_mode failed");
            space = b200;
        }
    } catch (const std::exception& e) {
        dup2(saved, 1);
        fprintf(stderr, "checker init failed: %s\n", e.what());
        return 3;
    }
    auto t1 = std::chrono::steady_clock::now();

    FILE* tf = trace.empty() ? nullptr : fopen(trace.c_str(), "wb");
    TracingSpace traced(space, tf);
    space = &traced;
    PRMSolver<4> prm(space, distH, distD, maxstorage, blocksize);
    const int start_free = space->indicator(qstart) == 0, end_free = space->indicator(qend) == 0;
    prm.init(qstart, qend);
    auto t2 = std::chrono::steady_clock::now();
    const int found = prm.process_mpi5(num, nbuf, maxsteps, seed, workerversion);
    auto t3 = std::chrono::steady_clock::now();
    prm.store_results(out);
    if (!dump.empty()) {
        /* the arguments store_results gives store_graph (prmsolver.cpp:2965-2976) */
        mkdir(dump.c_str(), 0755);
        mkdir((dump + "/graphl").c_str(), 0755);
        mkdir((dump + "/graphr").c_str(), 0755);
        dump_graph(dump + "/graphl", prm.graphl, prm.dijkstral, prm.i0l, prm.connection.index_left,
                   prm.connection_found);
        dump_graph(dump + "/graphr", prm.graphr, prm.dijkstrar, prm.connection.index_right, prm.i0r,
                   prm.connection_found);
        int cf = prm.connection_found ? 1 : 0;
        dump_array(dump + "/connection.bin", &cf, 1);
    }
    MPI_Finalize();
    if (tf) fclose(tf);

    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    const double init_s = std::chrono::duration<double>(t1 - t0).count();
    const double plan_s = std::chrono::duration<double>(t3 - t2).count();
    long long steps = 0;
    if (ref) {
        steps = ref->get_numthreads_all();
    } else {
        gprm_stats st;
        if (gprm_get_stats(b200->handle(), &st) == GPRM_OK) steps = (long long)st.edge_steps_nominal;
    }
    printf("{\"checker\": \"%s\", \"init_seconds\": %.6f, \"plan_seconds\": %.6f, \"process_result\": %d, "
           "\"connection_found\": %d, "
           "\"start_free\": %d, \"end_free\": %d, \"num_nodes\": %d, \"rand_nodes_all\": %d, "
           "\"rand_nodes_accepted\": %d, \"edge_step_checks\": %lld}\n",
           checker.c_str(), init_s, plan_s, found, prm.connection_found ? 1 : 0, start_free, end_free,
           PRMSolver<4>::num_nodes,
           PRMSolver<4>::rand_nodes_all, PRMSolver<4>::rand_nodes_accepted, steps);
    delete ref;
    delete b200;
    return 0;
}

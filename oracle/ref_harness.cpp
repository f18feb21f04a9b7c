/*
 * ref_harness.cpp - builds GPUPRM's own CPU collision checker from its
 * unmodified sources and gives it a C ABI.
 *
 * TEST INFRASTRUCTURE ONLY (pins the oracle restatement and times the CPU
 * baseline).  The translation unit includes the reference's
 * prm/src/lib/robotspace/robotconfigspace.cpp as it lies in the reference
 * tree (include path -I <reference>/prm/src/lib, see oracle/Makefile) and
 * adds explicit instantiations for 5-7 DOF next to the file's own
 * RobotConfigspace<4> (robotconfigspace.cpp:809).  Built without GPU_VERSION,
 * so indicator2 runs kernel_indicator2 on the host
 * (robotconfigspace.cpp:389-399, 694-705).
 */
#include "robotspace/robotconfigspace.cpp"

#include <atomic>
#include <mutex>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>
#include <thread>
#include <vector>

template class RobotConfigspace<5>;
template class RobotConfigspace<6>;
template class RobotConfigspace<7>;

namespace {

/* The reference prints sumn and summ while it initialises
 * (robotconfigspace.cpp:281-282); file descriptor 1 points at /dev/null for
 * the duration, under a lock so that concurrent opens do not interleave. */
static std::mutex g_stdout_lock;

struct QuietStdout {
    int saved;
    QuietStdout() : saved(-1) {
        g_stdout_lock.lock();
        std::cout.flush();
        fflush(stdout);
        int nul = open("/dev/null", O_WRONLY);
        if (nul >= 0) { saved = dup(1); dup2(nul, 1); close(nul); }
    }
    ~QuietStdout() {
        std::cout.flush();
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
        g_stdout_lock.unlock();
    }
};

struct Handle {
    int ndof;
    int nbuf;
    void* space;
};

template <int D>
static void* open_space(const char* dir, float dq, int nbuf)
{
    QuietStdout quiet;
    RobotConfigspace<D>* s = new RobotConfigspace<D>(std::string(dir), dq, nbuf);
    s->init(0, 1);
    return s;
}

template <int D>
static int indicator1(void* s, const float* q) { return ((RobotConfigspace<D>*)s)->indicator(q); }

template <int D>
static int indicator2(void* s, const float* qs, const float* qe, int* res, int n, int offset)
{
    return ((RobotConfigspace<D>*)s)->indicator2(qs, qe, res, n, offset);
}

template <int D>
static void close_space(void* s) { delete (RobotConfigspace<D>*)s; }

#define DISPATCH(nd, expr4, expr5, expr6, expr7) \
    switch (nd) { case 4: expr4; break; case 5: expr5; break; case 6: expr6; break; case 7: expr7; break; default: break; }

} /* namespace */

extern "C" {

void* ref_open(const char* dir, int ndof, float dq, int nbuf)
{
    if (ndof < 4 || ndof > 7 || nbuf < 1) return NULL;
    void* s = NULL;
    DISPATCH(ndof, s = open_space<4>(dir, dq, nbuf), s = open_space<5>(dir, dq, nbuf),
             s = open_space<6>(dir, dq, nbuf), s = open_space<7>(dir, dq, nbuf));
    Handle* h = new Handle{ndof, nbuf, s};
    return h;
}

void ref_close(void* hv)
{
    Handle* h = (Handle*)hv;
    if (!h) return;
    DISPATCH(h->ndof, close_space<4>(h->space), close_space<5>(h->space),
             close_space<6>(h->space), close_space<7>(h->space));
    delete h;
}

/* indicator(q) for one configuration q[ndof] */
int ref_indicator(void* hv, const float* q)
{
    Handle* h = (Handle*)hv;
    int r = 0;
    DISPATCH(h->ndof, r = indicator1<4>(h->space, q), r = indicator1<5>(h->space, q),
             r = indicator1<6>(h->space, q), r = indicator1<7>(h->space, q));
    return r;
}

/* indicator(q) over n configurations stored q[i + offset*j] */
int ref_check_configs(void* hv, const float* q, int n, int offset, int* code)
{
    Handle* h = (Handle*)hv;
    float qi[8];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < h->ndof; ++j) qi[j] = q[i + (size_t)offset * j];
        code[i] = ref_indicator(hv, qi);
    }
    return 0;
}

/* indicator2 over n edges, in chunks of at most nbuf edges (the reference
 * asserts N <= nbuf, robotconfigspace.cpp:618-619) */
int ref_check_edges(void* hv, const float* qs, const float* qe, int n, int offset, int* res)
{
    Handle* h = (Handle*)hv;
    for (int s = 0; s < n; s += h->nbuf) {
        int c = n - s < h->nbuf ? n - s : h->nbuf;
        DISPATCH(h->ndof,
                 indicator2<4>(h->space, qs + s, qe + s, res + s, c, offset),
                 indicator2<5>(h->space, qs + s, qe + s, res + s, c, offset),
                 indicator2<6>(h->space, qs + s, qe + s, res + s, c, offset),
                 indicator2<7>(h->space, qs + s, qe + s, res + s, c, offset));
    }
    return 0;
}

/* Multi-threaded drivers: each thread opens its own RobotConfigspace (the
 * class is not thread-safe, robotconfigspace.h:116,166) and takes chunks of
 * `chunk` items from a shared counter. */
int ref_check_edges_mt(const char* dir, int ndof, float dq, int nbuf, const float* qs,
                       const float* qe, int n, int offset, int* res, int nthreads, int chunk)
{
    if (nthreads < 1) nthreads = 1;
    if (chunk < 1) chunk = 64;
    std::atomic<int> next(0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&]() {
            void* hv = ref_open(dir, ndof, dq, nbuf);
            if (!hv) return;
            for (;;) {
                int s = next.fetch_add(chunk);
                if (s >= n) break;
                int c = n - s < chunk ? n - s : chunk;
                ref_check_edges(hv, qs + s, qe + s, c, offset, res + s);
            }
            ref_close(hv);
        });
    for (auto& x : th) x.join();
    return 0;
}

int ref_check_configs_mt(const char* dir, int ndof, const float* q, int n, int offset,
                         int* code, int nthreads, int chunk)
{
    if (nthreads < 1) nthreads = 1;
    if (chunk < 1) chunk = 256;
    std::atomic<int> next(0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&]() {
            void* hv = ref_open(dir, ndof, 0.01f, 1);
            if (!hv) return;
            for (;;) {
                int s = next.fetch_add(chunk);
                if (s >= n) break;
                int c = n - s < chunk ? n - s : chunk;
                ref_check_configs(hv, q + s, c, offset, code + s);
            }
            ref_close(hv);
        });
    for (auto& x : th) x.join();
    return 0;
}

} /* extern "C" */

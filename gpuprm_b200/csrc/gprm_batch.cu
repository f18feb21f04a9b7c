/*
 * gprm_batch.cu - many independent problems per launch (gprm_batch_* of
 * include/gprm_b200.h).
 *
 * The reference holds one scene per RobotConfigspace and launches once per
 * request (robotconfigspace.cpp:687-693).  A batch groups initialised
 * handles of one device - different robots, DOF, obstacle sets and dq -
 * and checks the configurations or edges of all of them in one persistent
 * launch: warps grab work items from one counter, look up the item's
 * problem and switch their cached scene descriptor when it changes
 * (k_check_configs_multi / k_check_edges_multi in gprm_kernels.cu).  The
 * per-call sequence (control reset, check kernel, FP64 recheck, edge
 * finalisation, counter accumulation) allocates nothing and never
 * synchronises, so it can be captured once into a CUDA graph and replayed
 * as one graph launch (gprm_batch_capture / gprm_batch_replay).  The launch
 * shape is chosen by timing the candidates on the caller's input
 * (gprm_batch_autotune).
 */
#include <cuda_runtime.h>
#include <limits.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/gprm_b200.h"
#include "gprm_host.h"
#include "gprm_internal.h"

using namespace gprm;

namespace {

/* Item layout and work buffers of one kind (configurations or edges). */
struct Layout {
    bool set = false;
    std::vector<long long> offs;     /* host copy, count+1 */
    long long total = 0;
    long long nchunks = 0;           /* vertex chunks of the shared launch */
    long long* d_offs = nullptr;
    int4* d_chunks = nullptr;
    /* problems checked by their own launches (at least solo_min items) and
       the edge ranges of the shared launch (BatchView) */
    std::vector<int> solo;
    long long nwork_e = 0;
    int K = 0;
    long long* d_woffs = nullptr;
    long long* d_wbase = nullptr;
    int* d_wprob = nullptr;
    int graph_launches = 0;          /* kernels in the captured graph */
    unsigned* d_key = nullptr;       /* edges: per-edge decision key */
    uint2* d_queue = nullptr;
    unsigned* d_qpair = nullptr;     /* pair range of each queue item's recheck (BandQueue) */
    size_t qcap = 0;
    bool qpair_ok = false;           /* every problem's pair indices fit 16 bits */
    unsigned* d_ovf = nullptr;       /* overflow record of the queue (BandQueue), 2 words per item */
    cudaGraphExec_t graph = nullptr; /* captured call sequence */
};

void free_layout(Layout& L)
{
    cudaFree(L.d_offs);
    cudaFree(L.d_chunks);
    cudaFree(L.d_woffs);
    cudaFree(L.d_wbase);
    cudaFree(L.d_wprob);
    cudaFree(L.d_key);
    cudaFree(L.d_queue);
    cudaFree(L.d_qpair);
    cudaFree(L.d_ovf);
    if (L.graph) cudaGraphExecDestroy(L.graph);
    L = Layout();
}

}  // namespace

struct gprm_batch {
    std::vector<gprm_space*> spaces;
    int device = 0;
    int sms = 0;
    int mode = GPRM_MODE_FP64_BAND;
    int policy = GPRM_EDGES_EARLY_EXIT;
    float band = 1e-5f;
    int lane_floats[2] = {0, 0};    /* [0] edge kernels, [1] vertex kernels */
    DevScene* d_scenes = nullptr;
    Control* ctl = nullptr;          /* per-call control block */
    Control* d_total = nullptr;      /* counters of all calls */
    Control* d_scratch_total = nullptr; /* counters of autotuning runs (discarded) */
    cudaStream_t stream = nullptr;   /* autotuning and capture */
    Layout lay[2];                   /* [0] edges, [1] configurations */
    LaunchCfg cfg[2];
    int64_t vertex_checks = 0;
    int64_t launches = 0;
    /* the last autotune's candidates per kind: threads, blocks per SM (0 =
       as many as fit), resident blocks per SM, ms per run */
    struct TuneRow { int threads, cap, per_sm; long long solo_min; float ms; };
    std::vector<TuneRow> tune[2];
    /* problems with at least this many items run in their own launches
       (the single-problem kernels, the scene in the constant bank); -1: none */
    long long solo_min[2] = {-1, -1};
    std::string err = "no error";
};

namespace {

thread_local std::string g_batch_create_error = "no error";

int bfail(gprm_batch* b, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    else g_batch_create_error = buf;
    return code;
}

#define BATCH_TRY(b, call)                                                                  \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? GPRM_ERR_NOMEM : GPRM_ERR_CUDA, \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

BatchView view_of(const gprm_batch* b, int vertex_kernel)
{
    const Layout& L = b->lay[vertex_kernel];
    BatchView v;
    v.scenes = b->d_scenes;
    v.offs = L.d_offs;
    v.chunks = L.d_chunks;
    v.nwork = vertex_kernel ? L.nchunks : L.nwork_e;
    v.woffs = L.d_woffs;
    v.wbase = L.d_wbase;
    v.wprob = L.d_wprob;
    v.K = L.K;
    v.S = (int)b->spaces.size();
    v.lane_floats = b->lane_floats[vertex_kernel ? 1 : 0];
    v.fast = (b->mode & GPRM_MODE_FAST) != 0;
    return v;
}

/* The call sequence of one batched check on stream `st`: every solo
 * problem through the single-problem kernels (its own scene and launch
 * shape), then the other problems in one shared launch, each part with its
 * FP64 recheck and overflow pass.  Allocates nothing and never
 * synchronises (capturable). */
int enqueue_batch(gprm_batch* b, int vertex_kernel, const float* qa, const float* qb, int* res, long long stride,
                  const LaunchCfg& cfg, Control* total, cudaStream_t st)
{
    Layout& L = b->lay[vertex_kernel];
    const BatchView v = view_of(b, vertex_kernel);
    const int band_on = (b->mode & GPRM_MODE_FP64_BAND) != 0;
    const int recheck_blocks = b->sms * 4;
    if (!vertex_kernel)
        BATCH_TRY(b, cudaMemsetAsync(L.d_key, b->policy == GPRM_EDGES_EARLY_EXIT ? 0xff : 0x00,
                                     (size_t)L.total * sizeof(unsigned), st));
    for (int p : L.solo) {
        const gprm_space* s = b->spaces[p];
        const long long off = L.offs[p], n = L.offs[p + 1] - off;
        BandQueue bq;
        bq.items = L.d_queue;
        bq.cap = (unsigned)L.qcap;
        bq.pair_range = L.qpair_ok ? L.d_qpair : nullptr;
        bq.ovf = band_on ? L.d_ovf + 2 * off : nullptr;
        bq.n = n;
        BATCH_TRY(b, cudaMemsetAsync(b->ctl, 0, sizeof(Control), st));
        if (bq.ovf) BATCH_TRY(b, cudaMemsetAsync(bq.ovf + n, 0, (size_t)((n + 31) / 32) * sizeof(unsigned), st));
        if (vertex_kernel) {
            BATCH_TRY(b, launch_check_configs(s->dsc, s->cfg_v, qa + off, n, stride, res + off, band_on, b->band, bq,
                                              b->ctl, st));
            if (band_on) {
                BATCH_TRY(b, launch_recheck(s->dsc, recheck_blocks, 0, qa + off, nullptr, nullptr, stride, s->dsc.dq,
                                            b->policy, res + off, nullptr, bq, b->ctl, st));
                BATCH_TRY(b, launch_overflow(s->dsc, recheck_blocks, 0, qa + off, nullptr, nullptr, stride,
                                             s->dsc.dq, b->policy, b->band, res + off, nullptr, bq, b->ctl, st));
            }
        } else {
            unsigned* key = L.d_key + off;
            BATCH_TRY(b, launch_check_edges(s->dsc, s->cfg_e, qa + off, qb + off, n, stride, s->dsc.dq, b->policy,
                                            key, band_on, b->band, bq, b->ctl, st));
            if (band_on) {
                BATCH_TRY(b, launch_recheck(s->dsc, recheck_blocks, 1, nullptr, qa + off, qb + off, stride,
                                            s->dsc.dq, b->policy, nullptr, key, bq, b->ctl, st));
                BATCH_TRY(b, launch_overflow(s->dsc, recheck_blocks, 1, nullptr, qa + off, qb + off, stride,
                                             s->dsc.dq, b->policy, b->band, nullptr, key, bq, b->ctl, st));
            }
        }
        BATCH_TRY(b, launch_accumulate(b->ctl, total, st));
    }
    if (v.nwork > 0) {
        BandQueue bq;
        bq.items = L.d_queue;
        bq.cap = (unsigned)L.qcap;
        bq.pair_range = L.qpair_ok ? L.d_qpair : nullptr;
        bq.ovf = band_on ? L.d_ovf : nullptr;
        bq.n = L.total;
        BATCH_TRY(b, cudaMemsetAsync(b->ctl, 0, sizeof(Control), st));
        if (bq.ovf)
            BATCH_TRY(b, cudaMemsetAsync(bq.ovf + L.total, 0, (size_t)((L.total + 31) / 32) * sizeof(unsigned), st));
        if (vertex_kernel) {
            BATCH_TRY(b, launch_check_configs_multi(v, cfg, qa, stride, res, band_on, b->band, bq, b->ctl, st));
            if (band_on) {
                BATCH_TRY(b, launch_recheck_multi(v, recheck_blocks, 0, qa, nullptr, nullptr, stride, b->policy, res,
                                                  nullptr, bq, b->ctl, st));
                BATCH_TRY(b, launch_overflow_multi(v, recheck_blocks, 0, qa, nullptr, nullptr, stride, b->policy,
                                                   b->band, res, nullptr, bq, b->ctl, st));
            }
        } else {
            BATCH_TRY(b, launch_check_edges_multi(v, cfg, qa, qb, stride, b->policy, L.d_key, band_on, b->band,
                                                  bq, b->ctl, st));
            if (band_on) {
                BATCH_TRY(b, launch_recheck_multi(v, recheck_blocks, 1, nullptr, qa, qb, stride, b->policy, nullptr,
                                                  L.d_key, bq, b->ctl, st));
                BATCH_TRY(b, launch_overflow_multi(v, recheck_blocks, 1, nullptr, qa, qb, stride, b->policy,
                                                   b->band, nullptr, L.d_key, bq, b->ctl, st));
            }
        }
        BATCH_TRY(b, launch_accumulate(b->ctl, total, st));
    }
    if (!vertex_kernel) BATCH_TRY(b, launch_finalize_edges(L.total, b->policy, L.d_key, res, st));
    return GPRM_OK;
}

/* Kernels one call launches: check (+ recheck and overflow pass) and the
 * counter accumulation per part, and the edge decode. */
int launches_per_call(const gprm_batch* b, int vertex_kernel)
{
    const Layout& L = b->lay[vertex_kernel];
    const int band_on = (b->mode & GPRM_MODE_FP64_BAND) != 0;
    const int per_part = 2 + 2 * band_on;
    const long long shared = vertex_kernel ? L.nchunks : L.nwork_e;
    return per_part * ((int)L.solo.size() + (shared > 0 ? 1 : 0)) + (vertex_kernel ? 0 : 1);
}

/* The solo problems and the shared launch's work of layout L under the
 * threshold solo_min (-1: no solo problems): vertex chunks of at most 32
 * configurations, edge ranges. */
int build_work(gprm_batch* b, int vertex_kernel, long long solo_min)
{
    Layout& L = b->lay[vertex_kernel];
    const int S = (int)b->spaces.size();
    cudaFree(L.d_chunks);
    cudaFree(L.d_woffs);
    cudaFree(L.d_wbase);
    cudaFree(L.d_wprob);
    L.d_chunks = nullptr;
    L.d_woffs = L.d_wbase = nullptr;
    L.d_wprob = nullptr;
    L.nchunks = L.nwork_e = 0;
    L.K = 0;
    L.solo.clear();
    std::vector<char> own(S, 0);
    for (int p = 0; p < S; ++p) {
        const long long n = L.offs[p + 1] - L.offs[p];
        if (solo_min >= 0 && n > 0 && n >= solo_min) {
            own[p] = 1;
            L.solo.push_back(p);
        }
    }
    if (vertex_kernel) {
        std::vector<int4> ch;
        for (int p = 0; p < S; ++p) {
            if (own[p]) continue;
            for (long long s = L.offs[p]; s < L.offs[p + 1]; s += 32) {
                const long long c = L.offs[p + 1] - s;
                ch.push_back(make_int4(p, (int)s, (int)(c < 32 ? c : 32), 0));
            }
        }
        L.nchunks = (long long)ch.size();
        if (!ch.empty()) {
            BATCH_TRY(b, dev_malloc((void**)&L.d_chunks, sizeof(int4) * ch.size()));
            BATCH_TRY(b, cudaMemcpy(L.d_chunks, ch.data(), sizeof(int4) * ch.size(), cudaMemcpyHostToDevice));
        }
    } else {
        std::vector<long long> woffs(1, 0), wbase;
        std::vector<int> wprob;
        for (int p = 0; p < S; ++p) {
            const long long n = L.offs[p + 1] - L.offs[p];
            if (own[p] || n == 0) continue;
            wbase.push_back(L.offs[p]);
            wprob.push_back(p);
            woffs.push_back(woffs.back() + n);
        }
        L.K = (int)wprob.size();
        L.nwork_e = woffs.back();
        BATCH_TRY(b, dev_malloc((void**)&L.d_woffs, sizeof(long long) * woffs.size()));
        BATCH_TRY(b, cudaMemcpy(L.d_woffs, woffs.data(), sizeof(long long) * woffs.size(), cudaMemcpyHostToDevice));
        if (L.K > 0) {
            BATCH_TRY(b, dev_malloc((void**)&L.d_wbase, sizeof(long long) * L.K));
            BATCH_TRY(b, dev_malloc((void**)&L.d_wprob, sizeof(int) * L.K));
            BATCH_TRY(b, cudaMemcpy(L.d_wbase, wbase.data(), sizeof(long long) * L.K, cudaMemcpyHostToDevice));
            BATCH_TRY(b, cudaMemcpy(L.d_wprob, wprob.data(), sizeof(int) * L.K, cudaMemcpyHostToDevice));
        }
    }
    return GPRM_OK;
}

int check_call(gprm_batch* b, int vertex_kernel, const float* qa, const float* qb, const int* res, long long stride)
{
    if (!b) return GPRM_ERR_ARG;
    const Layout& L = b->lay[vertex_kernel];
    if (!L.set) return bfail(b, GPRM_ERR_STATE, "no %s layout set", vertex_kernel ? "configuration" : "edge");
    if (stride < L.total) return bfail(b, GPRM_ERR_ARG, "stride %lld < %lld items", stride, L.total);
    if (L.total > 0 && (!qa || !res || (!vertex_kernel && !qb))) return bfail(b, GPRM_ERR_ARG, "null input or result");
    BATCH_TRY(b, cudaSetDevice(b->device));
    return GPRM_OK;
}

}  // namespace

extern "C" {

int gprm_batch_create(gprm_space* const* spaces, int count, gprm_batch** out)
{
    if (!out) return bfail(nullptr, GPRM_ERR_ARG, "null output");
    *out = nullptr;
    if (!spaces || count < 1) return bfail(nullptr, GPRM_ERR_ARG, "need at least one space");
    for (int i = 0; i < count; ++i) {
        if (!spaces[i]) return bfail(nullptr, GPRM_ERR_ARG, "space %d is null", i);
        if (!spaces[i]->inited) return bfail(nullptr, GPRM_ERR_STATE, "space %d is not initialised", i);
        if (spaces[i]->device != spaces[0]->device)
            return bfail(nullptr, GPRM_ERR_ARG, "space %d is on device %d, space 0 on %d", i, spaces[i]->device,
                         spaces[0]->device);
        if (spaces[i]->mode != spaces[0]->mode || spaces[i]->band != spaces[0]->band)
            return bfail(nullptr, GPRM_ERR_ARG, "space %d differs from space 0 in mode or FP64 band", i);
    }
    gprm_batch* b = new gprm_batch();
    b->spaces.assign(spaces, spaces + count);
    b->device = spaces[0]->device;
    b->sms = spaces[0]->sms;
    b->mode = spaces[0]->mode;
    b->policy = spaces[0]->policy;
    b->band = spaces[0]->band;
    std::vector<DevScene> sc(count);
    for (int i = 0; i < count; ++i) {
        sc[i] = spaces[i]->dsc;
        for (int k = 0; k < 2; ++k) {
            const int lf = (int)lane_floats(sc[i], k == 1);
            if (lf > b->lane_floats[k]) b->lane_floats[k] = lf;
        }
    }
    auto bad = [&](int rc) {
        g_batch_create_error = b->err;
        gprm_batch_destroy(b);
        return rc;
    };
    int rc;
    if ((rc = [&]() -> int {
            BATCH_TRY(b, cudaSetDevice(b->device));
            BATCH_TRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
            BATCH_TRY(b, dev_malloc((void**)&b->d_scenes, sizeof(DevScene) * count));
            BATCH_TRY(b, cudaMemcpy(b->d_scenes, sc.data(), sizeof(DevScene) * count, cudaMemcpyHostToDevice));
            BATCH_TRY(b, dev_malloc((void**)&b->ctl, sizeof(Control)));
            BATCH_TRY(b, dev_malloc((void**)&b->d_total, sizeof(Control)));
            BATCH_TRY(b, dev_malloc((void**)&b->d_scratch_total, sizeof(Control)));
            BATCH_TRY(b, cudaMemset(b->d_total, 0, sizeof(Control)));
            BatchView v = view_of(b, 1);
            BATCH_TRY(b, configure_batch_launch(v, 1, 128, &b->cfg[1]));
            BATCH_TRY(b, configure_batch_launch(v, 0, 128, &b->cfg[0]));
            return GPRM_OK;
        }()))
        return bad(rc);
    *out = b;
    return GPRM_OK;
}

void gprm_batch_destroy(gprm_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaDeviceSynchronize();
    free_layout(b->lay[0]);
    free_layout(b->lay[1]);
    cudaFree(b->d_scenes);
    cudaFree(b->ctl);
    cudaFree(b->d_total);
    cudaFree(b->d_scratch_total);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* gprm_batch_last_error(const gprm_batch* b)
{
    return b ? b->err.c_str() : g_batch_create_error.c_str();
}

int gprm_batch_set_layout(gprm_batch* b, int vertex_kernel, const long long* offsets, long long queue_capacity)
{
    if (!b) return GPRM_ERR_ARG;
    vertex_kernel = vertex_kernel ? 1 : 0;
    const int S = (int)b->spaces.size();
    if (!offsets || offsets[0] != 0) return bfail(b, GPRM_ERR_ARG, "offsets must start at 0");
    for (int p = 0; p < S; ++p)
        if (offsets[p + 1] < offsets[p]) return bfail(b, GPRM_ERR_ARG, "offsets decrease at problem %d", p);
    const long long total = offsets[S];
    if (total > (long long)INT_MAX) return bfail(b, GPRM_ERR_ARG, "%lld items exceed %d", total, INT_MAX);
    if (queue_capacity < 0 || queue_capacity > (long long)UINT_MAX)
        return bfail(b, GPRM_ERR_ARG, "queue capacity %lld out of range", queue_capacity);
    BATCH_TRY(b, cudaSetDevice(b->device));
    BATCH_TRY(b, cudaDeviceSynchronize());
    Layout& L = b->lay[vertex_kernel];
    free_layout(L);
    L.offs.assign(offsets, offsets + S + 1);
    L.total = total;
    if (queue_capacity > 0) L.qcap = (size_t)queue_capacity;
    else L.qcap = vertex_kernel ? (size_t)total : (size_t)total * 4 + 65536;   /* one entry per configuration */
    if (L.qcap < 1) L.qcap = 1;
    BATCH_TRY(b, dev_malloc((void**)&L.d_offs, sizeof(long long) * (S + 1)));
    BATCH_TRY(b, cudaMemcpy(L.d_offs, offsets, sizeof(long long) * (S + 1), cudaMemcpyHostToDevice));
    BATCH_TRY(b, dev_malloc((void**)&L.d_queue, sizeof(uint2) * L.qcap));
    BATCH_TRY(b, dev_malloc((void**)&L.d_qpair, sizeof(unsigned) * L.qcap));
    L.qpair_ok = true;
    for (int p = 0; p < S; ++p)
        if (b->spaces[p]->dsc.npairs > 65535) L.qpair_ok = false;
    BATCH_TRY(b, dev_malloc((void**)&L.d_ovf, sizeof(unsigned) * (2 * (size_t)total + 64)));
    if (!vertex_kernel && total > 0) BATCH_TRY(b, dev_malloc((void**)&L.d_key, sizeof(unsigned) * total));
    const int rc = build_work(b, vertex_kernel, b->solo_min[vertex_kernel]);
    if (rc) return rc;
    L.set = true;
    return GPRM_OK;
}

int gprm_batch_set_solo_threshold(gprm_batch* b, int vertex_kernel, long long min_items)
{
    if (!b) return GPRM_ERR_ARG;
    vertex_kernel = vertex_kernel ? 1 : 0;
    if (min_items < -1) return bfail(b, GPRM_ERR_ARG, "min_items must be -1 (none) or >= 0");
    BATCH_TRY(b, cudaSetDevice(b->device));
    b->solo_min[vertex_kernel] = min_items;
    Layout& L = b->lay[vertex_kernel];
    if (!L.set) return GPRM_OK;
    /* the work arrays change: earlier calls must be done, and a captured
       graph (which holds the old arrays) is dropped */
    BATCH_TRY(b, cudaDeviceSynchronize());
    if (L.graph) {
        cudaGraphExecDestroy(L.graph);
        L.graph = nullptr;
    }
    return build_work(b, vertex_kernel, min_items);
}

int gprm_batch_get_solo_threshold(const gprm_batch* b, int vertex_kernel, long long* min_items, int* solo_problems)
{
    if (!b || !min_items || !solo_problems) return GPRM_ERR_ARG;
    vertex_kernel = vertex_kernel ? 1 : 0;
    *min_items = b->solo_min[vertex_kernel];
    *solo_problems = (int)b->lay[vertex_kernel].solo.size();
    return GPRM_OK;
}

int gprm_batch_indicator_device(gprm_batch* b, const float* q, int* res, long long stride, void* stream)
{
    int rc = check_call(b, 1, q, nullptr, res, stride);
    if (rc) return rc;
    if (b->lay[1].total == 0) return GPRM_OK;
    rc = enqueue_batch(b, 1, q, nullptr, res, stride, b->cfg[1], b->d_total, (cudaStream_t)stream);
    if (rc) return rc;
    b->vertex_checks += b->lay[1].total;
    b->launches += launches_per_call(b, 1);
    return GPRM_OK;
}

int gprm_batch_indicator2_device(gprm_batch* b, const float* qs, const float* qe, int* res, long long stride,
                                 void* stream)
{
    int rc = check_call(b, 0, qs, qe, res, stride);
    if (rc) return rc;
    if (b->lay[0].total == 0) return GPRM_OK;
    rc = enqueue_batch(b, 0, qs, qe, res, stride, b->cfg[0], b->d_total, (cudaStream_t)stream);
    if (rc) return rc;
    b->launches += launches_per_call(b, 0);
    return GPRM_OK;
}

int gprm_batch_capture(gprm_batch* b, int vertex_kernel, const float* qa, const float* qb, int* res, long long stride)
{
    vertex_kernel = vertex_kernel ? 1 : 0;
    int rc = check_call(b, vertex_kernel, qa, qb, res, stride);
    if (rc) return rc;
    Layout& L = b->lay[vertex_kernel];
    if (L.graph) {
        cudaGraphExecDestroy(L.graph);
        L.graph = nullptr;
    }
    /* earlier calls on any stream may still use the batch's buffers */
    BATCH_TRY(b, cudaDeviceSynchronize());
    BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_batch(b, vertex_kernel, qa, qb, res, stride, b->cfg[vertex_kernel], b->d_total, b->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return bfail(b, GPRM_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&L.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        L.graph = nullptr;
        return bfail(b, GPRM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    L.graph_launches = launches_per_call(b, vertex_kernel);
    return GPRM_OK;
}

int gprm_batch_replay(gprm_batch* b, int vertex_kernel, void* stream)
{
    if (!b) return GPRM_ERR_ARG;
    vertex_kernel = vertex_kernel ? 1 : 0;
    Layout& L = b->lay[vertex_kernel];
    if (!L.graph) return bfail(b, GPRM_ERR_STATE, "nothing captured for this kind");
    BATCH_TRY(b, cudaSetDevice(b->device));
    BATCH_TRY(b, cudaGraphLaunch(L.graph, (cudaStream_t)stream));
    if (vertex_kernel) b->vertex_checks += L.total;
    b->launches += L.graph_launches;
    return GPRM_OK;
}

int gprm_batch_set_launch_shape(gprm_batch* b, int vertex_kernel, int threads, int blocks_per_sm)
{
    if (!b) return GPRM_ERR_ARG;
    vertex_kernel = vertex_kernel ? 1 : 0;
    if (threads < 32 || threads > 512 || threads % 32)
        return bfail(b, GPRM_ERR_ARG, "threads must be 32..512, a multiple of 32");
    if (blocks_per_sm < 0 || blocks_per_sm > 64) return bfail(b, GPRM_ERR_ARG, "blocks_per_sm must be 0..64");
    BATCH_TRY(b, cudaSetDevice(b->device));
    LaunchCfg c{};
    cudaError_t e = configure_batch_launch(view_of(b, vertex_kernel), vertex_kernel, threads, &c, blocks_per_sm);
    if (e != cudaSuccess) {
        cudaGetLastError();
        LaunchCfg& cur = b->cfg[vertex_kernel];
        configure_batch_launch(view_of(b, vertex_kernel), vertex_kernel, cur.threads, &cur,
                               cur.carveout >= 0 ? cur.blocks_per_sm : 0);
        return bfail(b, GPRM_ERR_UNSUPPORTED, "launch shape of %d threads does not fit: %s", threads,
                     cudaGetErrorString(e));
    }
    b->cfg[vertex_kernel] = c;
    /* a captured graph keeps the shape it was captured with */
    return GPRM_OK;
}

int gprm_batch_set_launch(gprm_batch* b, int vertex_kernel, int threads)
{
    return gprm_batch_set_launch_shape(b, vertex_kernel, threads, 0);
}

int gprm_batch_get_launch(const gprm_batch* b, int vertex_kernel, int* threads, int* warps_per_sm)
{
    if (!b || !threads || !warps_per_sm) return GPRM_ERR_ARG;
    const LaunchCfg& c = b->cfg[vertex_kernel ? 1 : 0];
    *threads = c.threads;
    *warps_per_sm = c.warps_per_sm;
    return GPRM_OK;
}

int gprm_batch_get_launch_shape(const gprm_batch* b, int vertex_kernel, int* threads, int* blocks_per_sm,
                                int* warps_per_sm)
{
    if (!b || !threads || !blocks_per_sm || !warps_per_sm) return GPRM_ERR_ARG;
    const LaunchCfg& c = b->cfg[vertex_kernel ? 1 : 0];
    *threads = c.threads;
    *blocks_per_sm = c.blocks_per_sm;
    *warps_per_sm = c.warps_per_sm;
    return GPRM_OK;
}

int gprm_batch_autotune(gprm_batch* b, int vertex_kernel, const float* qa, const float* qb, int* res,
                        long long stride, int reps, int* best_threads, float* best_ms)
{
    vertex_kernel = vertex_kernel ? 1 : 0;
    int rc = check_call(b, vertex_kernel, qa, qb, res, stride);
    if (rc) return rc;
    if (reps < 1 || reps > 1000) return bfail(b, GPRM_ERR_ARG, "reps must be 1..1000");
    /* the runs use the batch's buffers on its own stream: let earlier calls finish */
    BATCH_TRY(b, cudaDeviceSynchronize());
    Layout& L = b->lay[vertex_kernel];
    if (L.graph) {   /* the work arrays may change below */
        cudaGraphExecDestroy(L.graph);
        L.graph = nullptr;
    }
    cudaEvent_t e0, e1;
    BATCH_TRY(b, cudaEventCreate(&e0));
    BATCH_TRY(b, cudaEventCreate(&e1));
    b->tune[vertex_kernel].clear();
    /* one untimed run, then `reps` timed ones; counters go to a scratch total */
    auto time_runs = [&](const LaunchCfg& c, float* ms) -> int {
        for (int r = 0; r <= reps; ++r) {
            if (r == 1) cudaEventRecord(e0, b->stream);
            const int rr = enqueue_batch(b, vertex_kernel, qa, qb, res, stride, c, b->d_scratch_total, b->stream);
            if (rr) return rr;
        }
        cudaEventRecord(e1, b->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return bfail(b, GPRM_ERR_CUDA, "autotune run: %s", cudaGetErrorString(e));
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= (float)reps;
        return GPRM_OK;
    };
    /* 1. the shared launch's shape, under the current solo threshold:
       threads per block x resident blocks per SM (every block size with as
       many blocks as fit, and with 3/4 and 1/2 of them: the L1 that the
       smaller carveout leaves caches more of the scenes' tables) */
    std::vector<std::pair<int, int>> cand;
    for (int threads : {64, 128, 256, 512}) {
        LaunchCfg full{};
        if (configure_batch_launch(view_of(b, vertex_kernel), vertex_kernel, threads, &full) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        cand.push_back({threads, 0});
        const int per_sm = full.blocks_per_sm;
        const int caps[2] = {(3 * per_sm) / 4, per_sm / 2};
        for (int k = 0; k < 2; ++k)
            if (caps[k] >= 1 && caps[k] < per_sm && (k == 0 || caps[1] != caps[0])) cand.push_back({threads, caps[k]});
    }
    float best = -1.0f;
    LaunchCfg best_cfg = b->cfg[vertex_kernel];
    int best_cap = 0;
    const long long solo0 = b->solo_min[vertex_kernel];
    const bool shared = (vertex_kernel ? L.nchunks : L.nwork_e) > 0;
    for (const auto& tc : cand) {
        LaunchCfg c{};
        if (configure_batch_launch(view_of(b, vertex_kernel), vertex_kernel, tc.first, &c, tc.second) !=
            cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        float ms = 0;
        if ((rc = time_runs(c, &ms))) break;
        b->tune[vertex_kernel].push_back({tc.first, tc.second, c.blocks_per_sm, solo0, ms});
        if (best < 0 || ms < best) {
            best = ms;
            best_cfg = c;
            best_cap = tc.second;
        }
        if (!shared) break;   /* every problem runs solo: the shape is not used */
    }
    if (!rc && best < 0) rc = bfail(b, GPRM_ERR_UNSUPPORTED, "no launch shape fits");
    /* re-apply the winner (each candidate set the kernel's shared-memory attribute) */
    if (!rc) {
        cudaError_t e = configure_batch_launch(view_of(b, vertex_kernel), vertex_kernel, best_cfg.threads,
                                               &b->cfg[vertex_kernel], best_cap);
        if (e != cudaSuccess) rc = bfail(b, GPRM_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
    }
    /* 2. which problems get their own launches: none, those of at least
       2^18, 2^16 or 2^14 items, or all */
    long long best_solo = solo0;
    if (!rc) {
        for (long long sm : {-1ll, 1ll << 18, 1ll << 16, 1ll << 14, 0ll}) {
            if (sm == solo0) continue;
            if ((rc = build_work(b, vertex_kernel, sm))) break;
            BatchView v = view_of(b, vertex_kernel);
            LaunchCfg c{};
            if (configure_batch_launch(v, vertex_kernel, best_cfg.threads, &c, best_cap) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            float ms = 0;
            if ((rc = time_runs(c, &ms))) break;
            b->tune[vertex_kernel].push_back({best_cfg.threads, best_cap, c.blocks_per_sm, sm, ms});
            if (ms < best) {
                best = ms;
                best_solo = sm;
            }
        }
        const int rr = build_work(b, vertex_kernel, best_solo);
        if (!rc) rc = rr;
        b->solo_min[vertex_kernel] = best_solo;
        cudaError_t e = configure_batch_launch(view_of(b, vertex_kernel), vertex_kernel, best_cfg.threads,
                                               &b->cfg[vertex_kernel], best_cap);
        if (!rc && e != cudaSuccess) rc = bfail(b, GPRM_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (best_threads) *best_threads = best_cfg.threads;
    if (best_ms) *best_ms = best;
    return GPRM_OK;
}

int gprm_batch_get_tune_table(const gprm_batch* b, int vertex_kernel, int cap, int* threads, int* blocks_per_sm,
                              long long* solo_min, float* ms, int* count)
{
    if (!b || !count || cap < 0 || (cap > 0 && (!threads || !blocks_per_sm || !solo_min || !ms)))
        return GPRM_ERR_ARG;
    const auto& t = b->tune[vertex_kernel ? 1 : 0];
    *count = (int)t.size();
    for (int i = 0; i < cap && i < (int)t.size(); ++i) {
        threads[i] = t[i].threads;
        blocks_per_sm[i] = t[i].per_sm;
        solo_min[i] = t[i].solo_min;
        ms[i] = t[i].ms;
    }
    return GPRM_OK;
}

int gprm_batch_get_stats(const gprm_batch* bc, gprm_stats* out)
{
    gprm_batch* b = const_cast<gprm_batch*>(bc);
    if (!b || !out) return GPRM_ERR_ARG;
    memset(out, 0, sizeof(*out));
    out->vertex_checks = b->vertex_checks;
    out->launches = b->launches;
    BATCH_TRY(b, cudaSetDevice(b->device));
    BATCH_TRY(b, cudaDeviceSynchronize());
    Control tot;
    BATCH_TRY(b, cudaMemcpy(&tot, b->d_total, sizeof(Control), cudaMemcpyDeviceToHost));
    out->edge_steps_nominal = (int64_t)tot.steps_nominal;
    out->edge_steps_executed = (int64_t)tot.steps_exec;
    out->band_rechecks = (int64_t)tot.band_checks;
    out->band_flips = (int64_t)tot.band_flips;
    out->pairs_certified = (int64_t)(tot.cert_far + tot.cert_dir);
    out->pairs_tested = (int64_t)tot.full_tests;
    out->band_overflow_items = (int64_t)tot.ovf_count;
    if (tot.flags & GPRM_DEVFLAG_BAD_EDGE)
        return bfail(b, GPRM_ERR_DEVICE, "a call held a non-finite or oversized edge");
    return GPRM_OK;
}

}  /* extern "C" */

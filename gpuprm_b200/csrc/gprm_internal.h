/*
 * gprm_internal.h - interface between the C ABI (gprm_api.cu) and the
 * kernels (gprm_kernels.cu).  Not installed; not part of the public ABI.
 */
#ifndef GPRM_INTERNAL_H
#define GPRM_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>
#include "gprm_device.cuh"

namespace gprm {

/* Per-request control block in device memory, zeroed before each request. */
struct Control {
    unsigned long long next;          /* work counter (items handed out) */
    unsigned int qcount;              /* FP64 queue entries appended (may exceed capacity) */
    unsigned int flags;               /* GPRM_DEVFLAG_* */
    unsigned long long steps_nominal; /* sum of testnum of the request's edges */
    unsigned long long steps_exec;    /* steps evaluated in FP32 */
    unsigned long long band_checks;   /* checks recomputed in FP64 */
    unsigned long long band_flips;    /* FP64 verdict differs from FP32 verdict */
    unsigned long long configs_exec;  /* vertex checks that ran the pair loop */
    unsigned long long cert_far;      /* pair tests settled by the distance certificate */
    unsigned long long cert_dir;      /* ... by the first-direction certificate */
    unsigned long long full_tests;    /* pair tests that ran the Chung-Wang iteration */
    unsigned long long ovf_count;     /* items recorded in the overflow list (BandQueue) */
};

#define GPRM_DEVFLAG_BAD_EDGE    1u   /* non-finite or oversized edge length */
#define GPRM_DEVFLAG_QUEUE_FULL  2u   /* FP64 queue overflowed (the overflow pass completed the results) */

/* The FP64 recheck queue of one request.  A check that does not fit
 * records its item (configuration or edge) in the overflow list instead,
 * once per item (bitmap), and the overflow pass recomputes every listed
 * item in full, so a request's results are complete whatever the
 * capacity.  ovf: n list words, then (n + 31) / 32 bitmap words, which the
 * request zeroes; null where the capacity covers every check (one entry
 * per configuration). */
struct BandQueue {
    uint2* items;
    unsigned cap;
    unsigned* ovf;
    long long n;
    /* per item (null: not recorded): the pairs the FP64 recheck has to
       test, [lo, hi) packed as lo | hi << 16.  lo: the first pair that the
       FP32 check decided within the band (every pair before it was decided
       outside it); hi: one past the last such pair for a check the FP32
       pass found free (every later pair was decided outside the band), the
       pair count for one it found colliding (the pairs after the deciding
       one were not tested) */
    unsigned* pair_range = nullptr;
};

/* How a launch reads its scene. */
struct LaunchCfg {
    int blocks;          /* persistent grid size */
    int threads;         /* threads per block (multiple of 32) */
    size_t smem_bytes;   /* dynamic shared memory: per-lane frames (+ scene copy) */
    int scene_in_smem;   /* the scene table is copied into shared memory */
    int warps_per_sm;    /* resident warps per SM at this configuration */
    int blocks_per_sm;   /* resident blocks per SM of the persistent grid */
    int carveout;        /* shared-memory carveout (percent) set before each launch; -1: default */
};

enum EdgePolicy { EDGE_EARLY_EXIT = 0, EDGE_ALL_STEPS = 1 };

/* Adds the counters of request control block c to `total` (one thread). */
cudaError_t launch_accumulate(const Control* c, Control* total, cudaStream_t st);

/* Many independent problems in one launch.  Items (configurations or
 * edges) of problem p are offs[p] .. offs[p+1]-1 of the input arrays, which
 * hold GPRM_MAX_DOF rows (rows >= the problem's ndof are ignored).  Vertex
 * work is handed out in chunks of at most 32 configurations of one problem
 * (problem, first item, count). */
struct BatchView {
    const DevScene* scenes;   /* [S], device */
    const long long* offs;    /* [S+1], device */
    const int4* chunks;       /* vertex chunks, device */
    long long nwork;          /* chunks (vertex) or edges (edge) of the shared launch */
    /* edges of the shared launch: K ranges, range k = work items
       woffs[k] .. woffs[k+1]-1 = edges wbase[k] .. of problem wprob[k]
       (problems with their own launches are left out) */
    const long long* woffs;   /* [K+1], device */
    const long long* wbase;   /* [K], device */
    const int* wprob;         /* [K], device */
    int K;
    int S;
    int lane_floats;          /* per-lane shared floats: max over the problems */
    int fast;                 /* GPRM_MODE_FAST arithmetic (the problems share the mode) */
};

/* Launch shape of the batched kernels. */
/* blocks_cap > 0: at most that many resident blocks per SM, with a
 * shared-memory carveout just large enough for them (the rest of the SM's
 * L1/shared storage left to L1), applied as a launch attribute. */
cudaError_t configure_batch_launch(const BatchView& B, int vertex_kernel, int threads, LaunchCfg* cfg,
                                   int blocks_cap = 0);
cudaError_t launch_check_configs_multi(const BatchView& B, const LaunchCfg& cfg, const float* q, long long offset,
                                       int* res, int band_on, float band, BandQueue bq, Control* ctl,
                                       cudaStream_t st);
cudaError_t launch_check_edges_multi(const BatchView& B, const LaunchCfg& cfg, const float* qs, const float* qe,
                                     long long offset, int policy, unsigned* key, int band_on, float band,
                                     BandQueue bq, Control* ctl, cudaStream_t st);
cudaError_t launch_recheck_multi(const BatchView& B, int blocks, int kind, const float* q, const float* qs,
                                 const float* qe, long long offset, int policy, int* res, unsigned* key,
                                 BandQueue bq, Control* ctl, cudaStream_t st);

/* Per-lane shared floats of a warp's block: frames 1..ndof (12 floats
 * each), the world ball centres of the slots (3 floats each), the world
 * vertex 0 of the slots' polytopes (3 floats each), lane-interleaved; then,
 * in the vertex kernels only, DEFER_LANE_FLOATS per lane, together the
 * warp's queue of deferred exact pair tests (64 items) and one batch's
 * results (32 codes, 32 margins); then SWEEP_LANE_FLOATS per lane,
 * together the warp's per-slot sweep balls (GPRM_MAX_SLOTS float4). */
#define SWEEP_LANE_FLOATS 2
static_assert(SWEEP_LANE_FLOATS * 32 >= GPRM_MAX_SLOTS * 4, "sweep area too small");
#define DEFER_LANE_FLOATS 4
__host__ __device__ __forceinline__ size_t lane_floats(const DevScene& sc, bool vertex_kernel)
{
    return (size_t)sc.ndof * 12 + (size_t)sc.nslots * 6 + (vertex_kernel ? DEFER_LANE_FLOATS : 0) +
           SWEEP_LANE_FLOATS;
}

/* Scene bytes when staged in shared memory; per-lane frame bytes of a block. */
size_t scene_smem_bytes(const DevScene& sc);
size_t frame_smem_bytes(const DevScene& sc, int threads, bool vertex_kernel);

/* Sets up one launch variant (threads per block, scene in shared memory or
 * read through L1, at most blocks_cap resident blocks per SM, 0 = as many
 * as fit) and its persistent grid; fails if it does not fit. */
cudaError_t configure_launch(const DevScene& sc, int vertex_kernel, int threads, int scene_in_smem,
                             LaunchCfg* cfg, int blocks_cap = 0);

/* Vertex checks: res[i] = code of configuration q[i + offset*j]. */
cudaError_t launch_check_configs(const DevScene& sc, const LaunchCfg& cfg, const float* q,
                                 long long n, long long offset, int* res, int band_on, float band,
                                 BandQueue bq, Control* ctl, cudaStream_t st);

/* Edge checks, FP32 pass: key[e] is set per the edge policy (see kernels).
 * seg_off (edge_seg_words(n) words of scratch) or null: with it, n <=
 * EDGE_SPLIT_MAX and every edge longer than seg_rounds rounds of 32 steps
 * is split into segments that different warps check (batches of long
 * edges, where one warp per edge would leave the GPU idle or wait on its
 * longest edges).  Up to EDGE_SPLIT_ONE_BLOCK edges the segment offsets
 * are scanned by one block; above, by a three-pass scan over
 * EDGE_SEG_BLOCKS blocks whose sums follow the n + 1 offsets. */
constexpr long long EDGE_SPLIT_MAX = 1ll << 22;
constexpr long long EDGE_SPLIT_ONE_BLOCK = 16384;
constexpr int EDGE_SEG_BLOCKS = 1024;
inline size_t edge_seg_words(long long n) { return (size_t)n + 1 + EDGE_SEG_BLOCKS; }
cudaError_t launch_check_edges(const DevScene& sc, const LaunchCfg& cfg, const float* qs,
                               const float* qe, long long n, long long offset, float dq, int policy,
                               unsigned* key, int band_on, float band, BandQueue bq,
                               Control* ctl, cudaStream_t st, unsigned* seg_off = nullptr, int seg_rounds = 0);

/* FP64 recheck of queued vertex (kind 0) or edge-step (kind 1) items. */
cudaError_t launch_recheck(const DevScene& sc, int blocks, int kind, const float* q, const float* qs,
                           const float* qe, long long offset, float dq, int policy, int* res,
                           unsigned* key, BandQueue bq, Control* ctl,
                           cudaStream_t st);

/* The overflow pass after the recheck (band mode): recomputes every item
 * the queue could not hold (kind 0 configurations -> res, kind 1 edges ->
 * key).  Nothing to do when bq.ovf is null. */
cudaError_t launch_overflow(const DevScene& sc, int blocks, int kind, const float* q, const float* qs,
                            const float* qe, long long offset, float dq, int policy, float band, int* res,
                            unsigned* key, BandQueue bq, Control* ctl, cudaStream_t st);
cudaError_t launch_overflow_multi(const BatchView& B, int blocks, int kind, const float* q, const float* qs,
                                  const float* qe, long long offset, int policy, float band, int* res, unsigned* key,
                                  BandQueue bq, Control* ctl, cudaStream_t st);

/* res[e] = code decoded from key[e] */
cudaError_t launch_finalize_edges(long long n, int policy, const unsigned* key, int* res,
                                  cudaStream_t st);

/* Occupancy-derived persistent grid for the FP32 kernels. */
cudaError_t plan_launch(const DevScene& sc, int vertex_kernel, int threads, LaunchCfg* cfg);

/* FMA throughput probe: every thread runs `iters` rounds of
 * GPRM_FMA_PROBE_CHAINS independent FMAs. */
#define GPRM_FMA_PROBE_CHAINS 16
cudaError_t launch_fma_probe(int blocks, int threads, int iters, float* out, cudaStream_t st);

/* The FP32 per-configuration FK used by tests: out[(ndof+1)*12]. */
cudaError_t launch_fk_probe(const DevScene& sc, const float* q, float* out, cudaStream_t st);

}  // namespace gprm

#endif

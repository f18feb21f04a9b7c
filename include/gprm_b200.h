/*
 * gprm_b200.h - C ABI of the B200 configuration-space collision checker.
 *
 * This library replaces the collision-checking half of GPUPRM's
 * RobotConfigspace<ndof> (prm/src/lib/robotspace/robotconfigspace.{h,cpp})
 * behind the planner-facing interface Configspace<ndof>
 * (prm/src/lib/prm/configspace.hpp:10-50).  Every entry point takes plain
 * pointers and sizes, returns an int status (GPRM_OK == 0, negative on
 * error, never aborts) and leaves a message for gprm_last_error().
 *
 * Verdict codes are the reference's (collision4.h:226-332,
 * robotconfigspace.cpp:313-346): 0 = free, > 0 = the Chung-Wang iteration
 * that found "no separating half plane", -1 = iteration cap reached,
 * 1 = outside the joint bounds (vertex checks only).  Any nonzero code means
 * "not free".
 *
 * Layouts follow the reference:
 *   configurations  q[i + offset*j]  (component j of configuration i; SoA
 *                   with row stride `offset`, as in indicator(q,res,N,offset)
 *                   and indicator2, configspace.hpp:262,268)
 *   single config   q[j]             (indicator(q), configspace.hpp:264)
 *
 * Threading: one host thread per handle, like the reference
 * (robotconfigspace.h:116,166); different handles may be used concurrently.
 */
#ifndef GPRM_B200_H
#define GPRM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define GPRM_OK               0
#define GPRM_ERR_ARG         -1   /* bad argument (null pointer, size, ...) */
#define GPRM_ERR_SCENE       -2   /* scene failed validation */
#define GPRM_ERR_IO          -3   /* config directory unreadable */
#define GPRM_ERR_CUDA        -4   /* CUDA runtime error */
#define GPRM_ERR_NOMEM       -5   /* device or host allocation failed */
#define GPRM_ERR_STATE       -6   /* call out of order (e.g. not initialised) */
#define GPRM_ERR_REQUEST     -7   /* unknown async request id */
#define GPRM_ERR_DEVICE      -8   /* device-side watchdog or bounds flag */
#define GPRM_ERR_UNSUPPORTED -9

/* ---- limits (the reference asserts n <= 100, robotconfigspace.cpp:50) -- */
#define GPRM_MAX_VERTICES 100
#define GPRM_MAX_DOF      7

/* ---- check modes (gprm_set_mode) ------------------------------------- */
/* FP32 only: verdicts bit-identical to the reference CPU path. */
#define GPRM_MODE_FP32        0
/* FP32, then every check whose separation margin is inside the band is
 * recomputed in FP64 and the FP64 verdict is returned for it. */
#define GPRM_MODE_FP64_BAND   1
/* Flag, or-ed with either mode: the FP32 pass runs the same algorithm in
 * contracted arithmetic (fused multiply-add, hardware reciprocal square
 * roots, sincosf) and finds support vertices among per-direction-bin
 * candidate lists instead of by hill climbing.  Codes may differ from the reference's by rounding
 * (iteration counts, and verdicts of checks within rounding of contact);
 * with GPRM_MODE_FP64_BAND the free/not-free verdicts equal the
 * reference's for every check whose margin lies outside the band, and the
 * checks inside it get their FP64 verdict.  No counterpart in the
 * reference (its kernels and CPU path share the FP32 arithmetic of
 * collision4.h:226-332). */
#define GPRM_MODE_FAST        2

/* Edge evaluation (gprm_set_edge_policy). */
/* Stop an edge at its first colliding step; res[e] is that step's code
 * (0: free).  "First" is the kernel's order, fixed for given inputs: the
 * steps go in rounds of 32 (round r holds steps lane*R + r, R = rounds of
 * the edge), each round pair by pair in the reference's pair order; the
 * first round in which a step collides outside the FP64 band decides, at
 * the lowest lane among the steps that collide at the earliest such pair,
 * unless a lower lane of that round, or any step of an earlier round, was
 * left in the band and collides in the FP64 check (then the lowest such
 * round and lane).  The verdict (res != 0) is that of every other policy. */
#define GPRM_EDGES_EARLY_EXIT 0
/* res[e] is the code of the last colliding step, exactly what the
 * reference CPU path writes (robotconfigspace.cpp:458,694-705).  The steps
 * go from the qs end in rounds of 32 consecutive steps; a round with a
 * collision outside the FP64 band finishes its steps nearer qs and ends the
 * edge, since the steps after it cannot hold the last colliding one.  The
 * default: besides giving the reference's codes, its rounds of neighbouring
 * steps let the warp-wide sweep certificates settle more pairs, and it ran
 * faster than the early-exit order on every workload measured (headline
 * edges 198 vs 218 ms, 7-DOF wall edges 1.64 vs 1.91 s). */
#define GPRM_EDGES_ALL_STEPS  1

/* ---- scene description --------------------------------------------- */
/* The arrays of a config directory (robotconfigspace.cpp:101-208) and of
 * RobotConfigspace's array constructor (robotconfigspace.cpp:75-82, with
 * Robot<ndof> from robot.h:10-22 and polytope from polytope.h:5-16).
 * Polytopes must be sorted by sys and pairs by `pair_from`, as
 * polytope4data::build requires (polytope4data.h:224-291). */
typedef struct gprm_scene_desc {
    int ndof;                 /* 1..GPRM_MAX_DOF */
    const float* dh_a;        /* [ndof] modified-DH a */
    const float* dh_alpha;    /* [ndof] modified-DH alpha */
    const float* dh_q;        /* [ndof] theta of prismatic joints */
    const float* dh_d;        /* [ndof] d of revolute joints */
    const int*   dh_types;    /* [ndof] 0 revolute, 1 prismatic */
    const float* mins;        /* [ndof] joint lower bounds */
    const float* maxs;        /* [ndof] joint upper bounds */
    int num_polytopes;        /* N */
    const int*   poly_n;      /* [N] vertices per polytope */
    const int*   poly_m;      /* [N] CRS entries per polytope */
    const float* vertices;    /* [3*sum(n)] xyz, body frame, concatenated */
    const int*   dsp;         /* [sum(n)] CRS offsets, local to the polytope */
    const int*   cnt;         /* [sum(n)] neighbour counts, all > 0 */
    const int*   dest;        /* [sum(m)] neighbour indices, local */
    const int*   sys;         /* [N] frame index 0..ndof (0 = world) */
    int num_pairs;            /* M */
    const int*   pair_from;   /* [M] sorted ascending */
    const int*   pair_to;     /* [M] */
} gprm_scene_desc;

typedef struct gprm_space gprm_space;   /* one scene on one device */

/* Counters since creation (numthreads_all, robotconfigspace.h:169, plus
 * the FP64 band statistics). */
typedef struct gprm_stats {
    int64_t vertex_checks;        /* configurations checked */
    int64_t edge_steps_nominal;   /* sum of testnum over checked edges */
    int64_t edge_steps_executed;  /* steps actually evaluated */
    int64_t band_rechecks;        /* checks recomputed in FP64 */
    int64_t band_flips;           /* of those, verdict changed free<->not free */
    int64_t launches;             /* kernels launched */
    int64_t pairs_certified;      /* FP32 pair tests settled by a separation certificate */
    int64_t pairs_tested;         /* FP32 pair tests that ran the full iteration */
    int64_t band_overflow_items;  /* configurations or edges the FP64 queue could not hold,
                                     recomputed in full by the overflow pass */
} gprm_stats;

/* ---- lifetime --------------------------------------------------------- */

/* RobotConfigspace(robot, polys, sys, N, from, to, M, mins, maxs, dq, nbuf)
 * (robotconfigspace.cpp:75-82).  `nbuf` bounds N of every edge request like
 * the reference's nbuf (robotconfigspace.cpp:618-619); 0 means unbounded. */
int gprm_create(const gprm_scene_desc* desc, float dq, int nbuf, gprm_space** out);

/* RobotConfigspace(path, dq, nbuf) (robotconfigspace.cpp:84-98): reads the
 * reference's config directory; `ndof` must match ndof.bin. */
int gprm_create_from_dir(const char* path, int ndof, float dq, int nbuf, gprm_space** out);

/* init(rank, size) (configspace.hpp:13, robotconfigspace.cpp:213-287):
 * selects device rank*devcount/size, uploads the scene, creates a stream. */
int gprm_init(gprm_space* h, int rank, int size);

/* Frees device and host state (the reference's clear() is a stub,
 * robotconfigspace.cpp:289-295). Safe on NULL. */
void gprm_destroy(gprm_space* h);

/* Message of the last failed call on `h` (or of the last failed create
 * when h == NULL).  Never NULL. */
const char* gprm_last_error(const gprm_space* h);

int gprm_set_mode(gprm_space* h, int mode);
int gprm_set_edge_policy(gprm_space* h, int policy);
/* Edge batches of at most max_edges edges (0..4194304, default 16384)
 * check each edge longer than seg_rounds x 32 steps (default 2) with
 * several warps, one per segment of about seg_rounds x 32 steps, so that a
 * small batch of long edges (lazy planning rounds, query attachment, path
 * verification) keeps the GPU busy; larger batches give each edge one
 * warp.  The codes do not depend on it.  No reference counterpart (the
 * reference runs one CUDA thread per edge step, robotconfigspace.cpp:362-595). */
int gprm_set_edge_split(gprm_space* h, int max_edges, int seg_rounds);
/* FP64 band half-width in metres (default 1e-5). */
int gprm_set_band(gprm_space* h, float band_m);
int gprm_get_stats(const gprm_space* h, gprm_stats* out);

/* ---- queries (host buffers) ------------------------------------------ */

/* indicator(q) (configspace.hpp:264, robotconfigspace.cpp:313-346):
 * bounds check (code 1), then the pair loop; *code gets the first nonzero
 * pair result or 0. */
int gprm_indicator(gprm_space* h, const float* q, int* code);

/* indicator(q, res, N, offset) (configspace.hpp:262): batched vertex check,
 * q[i + offset*j]; res[i] gets the code of configuration i.  The reference
 * leaves this unimplemented (robotconfigspace.cpp:304-309). */
int gprm_indicator_batch(gprm_space* h, const float* q, int* res, int n, int offset);

/* indicator2(qs, qe, res, N, offset) (configspace.hpp:268,
 * robotconfigspace.cpp:745-752): edge i runs from qs[i+offset*j] to
 * qe[i+offset*j] in testnum = (int)(|qe-qs|/dq)+1 steps; res[i] = 0 if every
 * step is free, else nonzero (see the edge policies above). */
int gprm_indicator2(gprm_space* h, const float* qs, const float* qe, int* res, int n, int offset);

/* The compressed edge check indicator2(qs, M, qe, res, posqe, numqe,
 * offset) (configspace.hpp:29-32), which the reference's robot space
 * declares and leaves unimplemented (robotconfigspace.cpp:764-772), with
 * the meaning its 2-D array space gives it (arrayconfigspace.cpp:88-120):
 * for k = 0..M-1 and l = posqe[k] .. posqe[k]+numqe[k]-1, res[l] = the
 * code of the edge from qs[k + M*j] to qe[l + offset*j] (as
 * gprm_indicator2, under the edge policy); a later k overwrites an earlier
 * one's res[l]; entries of res that no range covers are left as they are.
 * Star-shaped batches (one start, many ends) are what a planner's
 * neighbour search produces.  Needs 0 <= posqe[k], numqe[k] >= 0 and
 * posqe[k] + numqe[k] <= offset.  Host buffers; synchronous. */
int gprm_indicator2_compressed(gprm_space* h, const float* qs, int M, const float* qe, int* res, const int* posqe,
                               const int* numqe, int offset);

/* indicator2_async / indicator2_async_wait (configspace.hpp:269-270,
 * robotconfigspace.cpp:617-742).  `qs`, `qe` are read before the call
 * returns; `res` must stay valid until gprm_indicator2_wait returns, which
 * synchronises the request's stream. */
int gprm_indicator2_async(gprm_space* h, const float* qs, const float* qe, int* res,
                          int n, int offset, int* request);
int gprm_indicator2_wait(gprm_space* h, int request);

/* check_boundaries(q, res, N, offset) and check_boundaries(q)
 * (configspace.hpp:277-279, robotconfigspace.cpp:780-802): 1 outside. */
int gprm_check_boundaries(gprm_space* h, const float* q, int* res, int n, int offset);
int gprm_check_boundaries1(gprm_space* h, const float* q, int* inside_violation);

/* min(i), max(i), deltaq(), dim() (configspace.hpp:282-289). */
float gprm_min(const gprm_space* h, int i);
float gprm_max(const gprm_space* h, int i);
float gprm_deltaq(const gprm_space* h);
int   gprm_dim(const gprm_space* h);

/* ---- queries (device buffers, caller's stream; no host sync) ----------
 * Pointers are device pointers; `stream` is the cudaStream_t to launch on
 * (NULL is the legacy default stream).  These never synchronise; after one
 * call with a given n they allocate nothing for calls with n no larger, so
 * they can be captured in a CUDA graph.  Calls on one handle share its
 * device scratch: do not overlap two of them on different streams. */
int gprm_indicator_batch_device(gprm_space* h, const float* q, int* res, int n,
                                int offset, void* stream);
int gprm_indicator2_device(gprm_space* h, const float* qs, const float* qe, int* res,
                           int n, int offset, void* stream);

/* ---- learned collision predictor (no counterpart in the reference) -------
 * An MLP (sin/cos of the joints -> 256 -> 256 -> 256 -> 256 -> 1, GELU,
 * sigmoid) estimating P(collision) of a configuration, trained on the exact
 * checker's verdicts; BF16 operands with FP32 accumulation on the tensor
 * cores, FP32 master weights, Adam.  The planner uses it to order lazy
 * edge checks and to prune samples; the exact checker still decides. */
typedef struct gprm_mlp gprm_mlp;
int  gprm_mlp_create(int ndof, unsigned long long seed, gprm_mlp** out);
void gprm_mlp_destroy(gprm_mlp* h);
const char* gprm_mlp_last_error(const gprm_mlp* h);
/* parameter count; parameters as one FP32 vector
 * [W1 (256x16, inputs padded) b1 W2 b2 W3 b3 W4 b4 w5 (1x256) b5] */
long long gprm_mlp_num_params(const gprm_mlp* h);
int gprm_mlp_get_params(gprm_mlp* h, float* out);
int gprm_mlp_set_params(gprm_mlp* h, const float* in);
/* p[i] = P(collision) of device configurations q[i + offset*j], launched on
 * `stream` (NULL: the legacy default stream) */
int gprm_mlp_predict(gprm_mlp* h, const float* q, int n, int offset, float* p, void* stream);
/* Inference path of gprm_mlp_predict: the fused tcgen05 kernel (default;
 * every layer of a 128-row tile on one SM, BF16 tensor-core MMAs into TMEM,
 * activations kept in shared memory), the tcgen05 layers (one persistent
 * kernel per layer, activations through device memory) or the training
 * GEMMs.  All compute the same function (BF16 operands and activations,
 * FP32 accumulation) up to FP32 summation order; the two tcgen05 paths
 * produce the same hidden activations bit for bit. */
#define GPRM_MLP_INFER_TCGEN05        0
#define GPRM_MLP_INFER_TRAINING_GEMM  1
#define GPRM_MLP_INFER_TCGEN05_LAYERS 2
int gprm_mlp_set_inference(gprm_mlp* h, int path);
/* GEMMs of training (gprm_mlp_train, gprm_mlp_gradients, and the
 * GPRM_MLP_INFER_TRAINING_GEMM inference path): tcgen05 tensor-core GEMMs
 * with TMA-loaded operands (default) or warp-level mma.sync GEMMs.  Both
 * compute the same gradients up to FP32 summation order. */
#define GPRM_MLP_TRAIN_TCGEN05        0
#define GPRM_MLP_TRAIN_MMA_SYNC       1
int gprm_mlp_set_training(gprm_mlp* h, int path);
/* Synchronises the device; *flags != 0 (and GPRM_ERR_DEVICE) when a
 * tensor-core kernel gave up waiting for its MMAs or copies. */
int gprm_mlp_device_status(gprm_mlp* h, unsigned* flags);
/* one forward/backward on n device configurations with labels y (device):
 * mean BCE loss and its gradient (host arrays) */
int gprm_mlp_gradients(gprm_mlp* h, const float* q, const float* y, int n, int offset, float* grads,
                       float* loss);
/* one Adam step (beta 0.9/0.999, eps 1e-8) with the last gradients */
int gprm_mlp_adam_step(gprm_mlp* h, float lr);
/* training: perm (device) holds `epochs` permutations of 0..n-1 */
int gprm_mlp_train(gprm_mlp* h, const float* q, const float* y, int n, int offset, const int* perm,
                   int epochs, int batch, float lr, float* losses);
/* Test hook: the clock budget (SM cycles) of every pipeline wait of the
 * tensor-core kernels (fused inference, training GEMMs); 0 restores the
 * default (about one second).  A budget too small for the copies and MMAs
 * makes the waits expire: the kernel stops, drains its own copies and MMAs
 * under the default budget, frees its tensor memory and returns, and
 * gprm_mlp_device_status reports it.  Setting the budget also clears that
 * status.  No counterpart in the reference. */
int gprm_mlp_set_wait_budget(gprm_mlp* h, long long cycles);

/* ---- vertex checks without allocation (no counterpart in the reference) --
 * For callers that must not allocate device memory while they run: a
 * planner inside a real-time control loop (cudaMalloc and cudaFree can
 * block and synchronise the whole device), or a host whose device memory is
 * owned by another allocator and cannot hand out raw allocations.  Same
 * result as gprm_indicator_batch_device, but the work buffers (a control
 * block and the FP64 recheck queue) live in a fixed device array inside the
 * library, sized for GPRM_NOALLOC_MAX_CONFIGS configurations
 * (about 0.5 MB, held by every GPU that loads the library until the process
 * exits).  Larger n is rejected with GPRM_ERR_ARG.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  The address is kept for the
 * life of the process: do not use this entry point after cudaDeviceReset
 * (or any other teardown of the device's primary context), which may move
 * the array.  All calls share the array:
 * calls that overlap on the GPU (other streams, other handles, other host
 * threads) race and must be serialised by the caller.  q and res are
 * device pointers as in gprm_indicator_batch_device; `stream` NULL is the
 * legacy default stream.  Nothing is allocated by this call. */
#define GPRM_NOALLOC_MAX_CONFIGS 65536
int gprm_indicator_batch_device_noalloc(gprm_space* h, const float* q, int* res, int n, int offset,
                                        void* stream);

/* ---- many problems per launch (no counterpart in the reference) --------
 * The reference holds one scene per RobotConfigspace and launches once per
 * request (robotconfigspace.cpp:687-693).  A batch groups `count`
 * initialised handles on one device - different robots, DOF, obstacle
 * sets, dq - and checks the configurations or edges of all of them in one
 * persistent launch.  Mode, edge policy and FP64 band are taken from
 * spaces[0] at creation; every space must share its mode and band.  The
 * batch reads the spaces' device tables: set their mode, policy and band
 * before creating it, and destroy it before them.
 *
 * Item layout: problem p owns items offsets[p] .. offsets[p+1]-1 (host
 * array of count+1 entries, offsets[0] = 0, non-decreasing, total at most
 * INT_MAX).  Inputs are device arrays with one row per joint and row
 * stride `stride` >= total: joint j of item i at q[i + stride*j]; problem
 * p reads rows 0 .. ndof_p-1.  res[i] is the code gprm_indicator_batch /
 * gprm_indicator2 would give item i on its own handle.  set_layout
 * allocates (and synchronises); the check calls allocate nothing and never
 * synchronise.  queue_capacity: FP64 recheck queue entries, 0 = total for
 * configurations, 4*total + 65536 for edges; any capacity gives complete
 * results (the checks it cannot hold are recomputed by the overflow pass
 * on the stream, counted in gprm_batch_get_stats' band_overflow_items).
 * Calls on one batch share
 * its control block: do not overlap them on different streams. */
typedef struct gprm_batch gprm_batch;
int  gprm_batch_create(gprm_space* const* spaces, int count, gprm_batch** out);
void gprm_batch_destroy(gprm_batch* b);
const char* gprm_batch_last_error(const gprm_batch* b);
int  gprm_batch_set_layout(gprm_batch* b, int vertex_kernel, const long long* offsets,
                           long long queue_capacity);
int  gprm_batch_indicator_device(gprm_batch* b, const float* q, int* res, long long stride,
                                 void* stream);
int  gprm_batch_indicator2_device(gprm_batch* b, const float* qs, const float* qe, int* res,
                                  long long stride, void* stream);
/* Captures one check call (those pointers, the current launch shape) into
 * a CUDA graph held by the batch; replay launches it on `stream` as one
 * graph launch.  Re-capture after changing the layout or launch shape. */
int  gprm_batch_capture(gprm_batch* b, int vertex_kernel, const float* qa, const float* qb,
                        int* res, long long stride);
int  gprm_batch_replay(gprm_batch* b, int vertex_kernel, void* stream);
/* Launch shape: threads per block (32..512); blocks fill every SM. */
int  gprm_batch_set_launch(gprm_batch* b, int vertex_kernel, int threads);
int  gprm_batch_get_launch(const gprm_batch* b, int vertex_kernel, int* threads, int* warps_per_sm);
/* Launch shape with a cap on the resident blocks per SM (0: as many as
 * fit); a cap sets a shared-memory carveout just large enough for those
 * blocks, so that the rest of the SM's storage serves as L1 for the
 * scenes' tables.  gprm_batch_set_launch(b, k, t) = ..._shape(b, k, t, 0). */
int  gprm_batch_set_launch_shape(gprm_batch* b, int vertex_kernel, int threads, int blocks_per_sm);
int  gprm_batch_get_launch_shape(const gprm_batch* b, int vertex_kernel, int* threads, int* blocks_per_sm,
                                 int* warps_per_sm);
/* Problems with at least min_items items (of the kind) are checked by the
 * single-problem kernels in launches of their own, inside the same call
 * (and captured graph): their scene sits in the kernel's constant bank and
 * they keep their own launch shape, while the rest share one persistent
 * launch that reads each warp's scene from shared memory.  -1 (the
 * default): no problem runs alone; 0: every non-empty problem does.
 * Changing it drops the kind's captured graph (capture again). */
int  gprm_batch_set_solo_threshold(gprm_batch* b, int vertex_kernel, long long min_items);
int  gprm_batch_get_solo_threshold(const gprm_batch* b, int vertex_kernel, long long* min_items,
                                   int* solo_problems);
/* Times the candidates on this input, `reps` runs each after one untimed
 * run, and keeps the fastest: first the shared launch's shape (64, 128,
 * 256 and 512 threads per block, each with as many resident blocks per SM
 * as fit and with 3/4 and 1/2 of them), then with that shape the solo
 * threshold (none, 2^18, 2^16, 2^14 items, every problem).  best_threads
 * gets the winner's block size (gprm_batch_get_launch_shape and
 * gprm_batch_get_solo_threshold give the rest).  Synchronous; drops the
 * kind's captured graph; the runs' counters are discarded. */
int  gprm_batch_autotune(gprm_batch* b, int vertex_kernel, const float* qa, const float* qb,
                         int* res, long long stride, int reps, int* best_threads, float* best_ms);
/* The last autotune's candidates for a kind: up to cap rows of (threads per
 * block, resident blocks per SM, solo threshold, ms per run); *count gets
 * the number of candidates timed. */
int  gprm_batch_get_tune_table(const gprm_batch* b, int vertex_kernel, int cap, int* threads,
                               int* blocks_per_sm, long long* solo_min, float* ms, int* count);
int  gprm_batch_get_stats(const gprm_batch* b, gprm_stats* out);

/* ---- neighbour search on the device -------------------------------------
 * get_near_vertices (prmsolver.cpp:2533-2574) keeps the nodes whose squared
 * distance, accumulated over the joints in order in float, is below D*D.
 * A gprm_nbr indexes n device nodes x[i + stride*j] (the array must stay
 * valid and unchanged until the next build); queries are device arrays
 * q[t + qstride*j].  build synchronises its stream (it reads the nodes'
 * extent); radius and knn never synchronise.
 *   radius: counts[t] <= cap neighbours of query t in ascending node index,
 *           idx/dist[t*cap + r] (the first cap in index order, like the
 *           reference's full buffer);
 *   knn:    the k <= 32 nearest nodes by the same distance, ties by lower
 *           index, idx/dist[t*k + r] in ascending order (-1 / inf where
 *           fewer exist); queries_are_nodes = 1 queries every node against
 *           the others (q, m, qstride ignored).
 * `cell` is the grid cell edge used by knn (0: chosen from the extent so
 * that a cell holds about the 16-neighbour radius). */
typedef struct gprm_nbr gprm_nbr;
int  gprm_nbr_create(int ndof, gprm_nbr** out);
void gprm_nbr_destroy(gprm_nbr* h);
const char* gprm_nbr_last_error(const gprm_nbr* h);
int  gprm_nbr_build(gprm_nbr* h, const float* x, int n, int stride, float cell, void* stream);
int  gprm_nbr_radius(gprm_nbr* h, const float* q, int m, int qstride, float D, int cap, int* counts,
                     int* idx, float* dist, void* stream);
int  gprm_nbr_knn(gprm_nbr* h, const float* q, int m, int qstride, int k, int queries_are_nodes,
                  int* idx, float* dist, void* stream);
/* queries of the last knn call that the grid could not settle and a full
 * scan answered (synchronises) */
int  gprm_nbr_redo_count(gprm_nbr* h, int* out);

/* ---- roadmap graphs on the device ----------------------------------------
 * The reference keeps roadmaps as host adjacency lists and runs Dijkstra
 * once start and goal connect (do_dijkstra, prmsolver.cpp:2805-2846).  Here a
 * roadmap is an undirected edge list in device memory: eu[e], ev[e] in
 * 0..V-1, an optional mask (nonzero = usable edge, NULL = all) and, for
 * shortest paths, float weights w[e] >= 0.  All pointers are device
 * pointers; calls run on `stream`.
 *   components: label[i] = smallest vertex of i's component (asynchronous);
 *   forest:     breadth-first forest from each component's label vertex:
 *               parent[i] (-1 at roots and unreached), depth[i] (INT_MAX when
 *               unreached); the parent is the smallest vertex of the
 *               previous level adjacent to i.  Synchronises every 16 levels;
 *               *levels (may be NULL) gets the number of levels run;
 *   path_lengths / path_write: the forest path from qs[t] to qt[t]
 *               (vertex ids, both ends included) when they share a
 *               component, else length 0; write it at out[offsets[t]..]
 *               with offsets the caller's exclusive prefix sum of len
 *               (path_write only follows queries path_lengths measured);
 * Edges or query vertices outside 0..V-1 are skipped (length 0).
 *   sssp:       distances from src under float path sums accumulated from
 *               the source (those of Dijkstra with the same arithmetic),
 *               dist = inf where unreachable; parent[v] = the smallest u with
 *               dist[u] + w == dist[v] (parent[src] = src, -1 unreached).
 *               Synchronises every 8 relaxation rounds. */
typedef struct gprm_graph gprm_graph;
int  gprm_graph_create(gprm_graph** out);
void gprm_graph_destroy(gprm_graph* h);
const char* gprm_graph_last_error(const gprm_graph* h);
int  gprm_graph_components(gprm_graph* h, int V, int E, const int* eu, const int* ev,
                           const unsigned char* mask, int* label, void* stream);
int  gprm_graph_forest(gprm_graph* h, int V, int E, const int* eu, const int* ev,
                       const unsigned char* mask, const int* label, int* parent, int* depth,
                       int* levels, void* stream);
int  gprm_graph_path_lengths(gprm_graph* h, int V, int Q, const int* qs, const int* qt, const int* label,
                             const int* parent, const int* depth, int* len, void* stream);
int  gprm_graph_path_write(gprm_graph* h, int Q, const int* qs, const int* qt, const int* parent,
                           const int* depth, const int* len, const long long* offsets, int* out,
                           void* stream);
int  gprm_graph_sssp(gprm_graph* h, int V, int E, const int* eu, const int* ev,
                     const unsigned char* mask, const float* w, int src, float* dist, int* parent,
                     int* rounds, void* stream);

/* ---- sampling near roadmap nodes ----------------------------------------
 * get_random_nodes (prmsolver.cpp:2585-2624; get_random_nodes2 :2635-2698
 * with power 2) as a batch: candidate t (t = t0 .. t0+B-1) picks node m
 * uniformly among n device nodes[m + stride*j], is accepted when its 31-bit
 * random value r <= (2^31-1) / (1+surrnum[m])^power (the reference's integer
 * test) and becomes q = (nodes[m] - D) + (2*D) * ((float)r' / 2^31) per
 * joint.  Writes q_out[t - t0 + out_stride*j] and parent_out[t - t0] = m, or
 * -1 when the candidate is dismissed.  Random numbers: Philox4x32-10 with key
 * = seed and counters (t, 0..2), so (seed, t) fixes a candidate.  The caller
 * vertex-checks the accepted candidates (gprm_indicator_batch_device).
 * Device pointers; asynchronous on `stream`. */
int gprm_sample_near(int ndof, const float* nodes, int n, int stride, const int* surrnum, int power,
                     float D, unsigned long long seed, long long t0, int B, float* q_out, int out_stride,
                     int* parent_out, void* stream);

/* The same over the reference's block storage of a roadmap (graph::blocks,
 * prmsolver.h:29-59; the node choice of prmsolver.cpp:2589-2597): nodes
 * are the n storage slots, block b holds slots block_pos[b] ..
 * block_pos[b] + block_num[b] - 1.  Candidate t picks block
 * r0 % nblocks, then slot block_pos[b] + r9 % block_num[b] (r9 from the
 * counter-2 block's second word), so every node weighs
 * 1 / (nblocks * block_num[its block]) as in the reference when the blocks
 * passed are its non-empty ones; a block with block_num <= 0, or a slot
 * outside 0..n-1, dismisses the candidate.  Device pointers; asynchronous. */
int gprm_sample_near_blocks(int ndof, const float* nodes, int n, int stride, const int* block_pos,
                            const int* block_num, int nblocks, const int* surrnum, int power, float D,
                            unsigned long long seed, long long t0, int B, float* q_out, int out_stride,
                            int* parent_out, void* stream);

/* ---- diagnostics (no counterpart in the reference) -------------------- */

/* The FP32 frames the kernels compute for one configuration q[ndof]:
 * out[(ndof+1)*12], frame f column c row r at out[f*12 + c*3 + r], in the
 * column layout of trafo4 (geo4.h:24). */
int gprm_debug_fk(gprm_space* h, const float* q, float* out);

/* Test hook, process-wide: the nth device allocation of the library from
 * now on (checker handles and batches) fails as if the device were out of
 * memory (0 = none).  The call that makes it returns GPRM_ERR_NOMEM and
 * leaves its handle usable: a later call allocates again.  No counterpart
 * in the reference (it aborts on any CUDA error, util.hpp:45). */
void gprm_debug_fail_device_alloc(long long nth);

/* Test hook: caps the FP64 recheck queue of every later request at
 * `capacity` entries (0 = no cap), so that tests can make it overflow.
 * Results do not depend on it: checks the queue cannot hold are recorded
 * per configuration or edge and recomputed in full on the stream after the
 * recheck (counted in gprm_stats.band_overflow_items); only the code of an
 * early-exit edge may change, to that of its first colliding step in step
 * order.  No counterpart in the reference. */
int gprm_debug_set_queue_capacity(gprm_space* h, unsigned capacity);

/* Support candidates of the fast path (GPRM_MODE_FAST) for polytope
 * `polytope` and direction bin `bin` (0..53: cube face 0..5 = +x,-x,+y,-y,
 * +z,-z, then the 3 x 3 cell of the other two components, each compared
 * with a third of the face component): writes up to cap vertex indices
 * (ascending) and returns their count, or a negative status.  Host data,
 * available after gprm_create; no counterpart in the reference. */
int gprm_debug_support_candidates(const gprm_space* h, int polytope, int bin, int* idx, int cap);

/* Streaming multiprocessors of the handle's device (0 before init). */
int gprm_device_sm_count(const gprm_space* h);

/* Launch shape of the FP32 kernels (vertex_kernel = 1: vertex checks,
 * 0: edge checks): threads per block (a multiple of 32, <= 512) and
 * whether the scene table is copied into shared memory (1) or read through
 * L1 (0).  Fails without changing anything if the shape does not fit.
 * gprm_init picks the shape with the most resident warps. */
int gprm_set_launch(gprm_space* h, int vertex_kernel, int threads, int scene_in_smem);
/* The same with at most blocks_per_sm resident blocks per SM (0 = as many
 * as fit): the kernel's shared-memory carveout is then set, before each
 * launch with this shape, to what those blocks need, and the rest of the
 * SM's combined L1/shared memory caches the scene table and the pair
 * records.  Fewer resident warps, more L1.  No counterpart in the
 * reference (one CUDA thread per edge step, robotconfigspace.cpp:676-693). */
int gprm_set_launch_shape(gprm_space* h, int vertex_kernel, int threads, int scene_in_smem, int blocks_per_sm);
int gprm_get_launch(const gprm_space* h, int vertex_kernel, int* threads, int* scene_in_smem,
                    int* warps_per_sm);

/* Kernel timing: while enabled, every request records CUDA events around
 * its FP32 check kernel and its FP64 recheck kernel on the stream they run
 * on; gprm_profile_read synchronises the device and returns the summed
 * durations (ms) and the number of timed FP32 launches since enabling. */
int gprm_profile_enable(gprm_space* h, int on);
int gprm_profile_read(gprm_space* h, double* fp32_ms, double* fp64_ms, int64_t* fp32_launches);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (2 flops
 * per FMA), from a register-resident FMA loop on every SM. */
int gprm_measure_fp32_peak(double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* GPRM_B200_H */

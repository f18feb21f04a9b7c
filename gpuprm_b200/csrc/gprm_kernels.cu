/*
 * gprm_kernels.cu - sm_100a kernels of the collision checker.
 *
 * Replaces kernel_indicator2 / kernel_indicator2_1 and set_kernel
 * (prm/src/lib/robotspace/robotconfigspace.cpp:362-595) and the host loop
 * over indicator(q) (robotconfigspace.cpp:313-346, prmsolver.cpp:2611).
 *
 * Work mapping (persistent grid, warps take work from a device counter):
 *   vertex checks  a warp takes 32 configurations, one per lane; every lane
 *                  runs FK and then the reference's pair loop with its own
 *                  early exit, lanes stepping through the pairs together.
 *   edge checks    a warp takes one edge; its lanes hold 32 steps of that
 *                  edge (coarse-to-fine: round r, lane i -> step i*R + r with
 *                  R = ceil(testnum/32); or descending steps when every step's
 *                  code is wanted) and step through the pairs together.  Nearby
 *                  steps take nearly the same path through the algorithm, so
 *                  the lanes stay converged, and one warp vote after each pair
 *                  ends the edge at its first colliding step.
 * The scene (vertices with packed adjacency, neighbour bytes, pair table)
 * is copied into shared memory per block when it fits.
 *
 * FP64 band: a check whose FP32 result is decided within the band (or by
 * the iteration cap) is appended to a queue; k_recheck recomputes it in
 * FP64, thread per item, and its verdict replaces the FP32 one.
 */
#include "gprm_internal.h"

#include <math.h>
#include <mutex>
#include <unordered_map>

namespace gprm {

#define FULL_MASK 0xffffffffu

/* minimum resident blocks of 128 threads the FP32 kernels are compiled for
 * (caps registers per thread; 0 = no cap) */
#ifndef GPRM_MIN_BLOCKS
#define GPRM_MIN_BLOCKS 0
#endif
#if GPRM_MIN_BLOCKS > 0
#define GPRM_BOUNDS __launch_bounds__(128, GPRM_MIN_BLOCKS)
#else
#define GPRM_BOUNDS __launch_bounds__(512)
#endif

size_t scene_smem_bytes(const DevScene& sc)
{
    /* tab | pairs | pairs_b | far | scan_c | scan_b, padded to 16 bytes */
    return ((size_t)sc.ntab * 16 + (size_t)sc.npairs * 80 + 15) & ~(size_t)15;
}

size_t frame_smem_bytes(const DevScene& sc, int threads, bool vertex_kernel)
{
    return (size_t)(threads / 32) * lane_floats(sc, vertex_kernel) * 32 * sizeof(float);
}

struct SceneView {
    const float4* tab;
    const int4* pairs;
    const float4* pairs_b;
    const float4* far;
    const int4* scan_c;
    const float4* scan_b;
    float* frames;   /* this lane's frames (lane-interleaved, stride 32) */
    float* cen;      /* this lane's slot ball centres, then the slots' world vertex 0 */
    float4* sweep;   /* the warp's per-slot sweep balls (GPRM_MAX_SLOTS) */
    unsigned* defer; /* the warp's deferred-test queue (64) and batch results (32 + 32) */
};

/* The warp's sweep area: the last SWEEP_LANE_FLOATS entries of its block. */
template <bool VERTEX>
__device__ __forceinline__ float4* sweep_area(const DevScene& sc, float* lane_frames)
{
    const int lane = threadIdx.x & 31;
    return reinterpret_cast<float4*>(lane_frames - lane + (lane_floats(sc, VERTEX) - SWEEP_LANE_FLOATS) * 32);
}

/* The warp's deferred-test area (vertex kernels): the DEFER_LANE_FLOATS
 * entries before the sweep area; null in the edge kernels. */
template <bool VERTEX>
__device__ __forceinline__ unsigned* defer_area(const DevScene& sc, float* lane_frames)
{
    if constexpr (!VERTEX) return nullptr;
    const int lane = threadIdx.x & 31;
    return reinterpret_cast<unsigned*>(lane_frames - lane +
                                       (lane_floats(sc, true) - SWEEP_LANE_FLOATS - DEFER_LANE_FLOATS) * 32);
}

/* Copies the scene into shared memory (SMEM) and returns the pointers the
 * warp uses, including its lane's slice of the frame array (laid out for
 * the vertex or the edge kernels, VERTEX). */
template <bool SMEM, bool VERTEX>
__device__ __forceinline__ SceneView stage_scene(const DevScene& sc, unsigned char* smem)
{
    SceneView s;
    size_t off = 0;
    if (SMEM) {
        const size_t np = (size_t)sc.npairs;
        float4* t = reinterpret_cast<float4*>(smem);
        int4* p = reinterpret_cast<int4*>(smem + (size_t)sc.ntab * 16);
        float4* pb = reinterpret_cast<float4*>(smem + (size_t)sc.ntab * 16 + np * 16);
        float4* fr = reinterpret_cast<float4*>(smem + (size_t)sc.ntab * 16 + np * 32);
        int4* scc = reinterpret_cast<int4*>(smem + (size_t)sc.ntab * 16 + np * 48);
        float4* scb = reinterpret_cast<float4*>(smem + (size_t)sc.ntab * 16 + np * 64);
        for (int i = threadIdx.x; i < sc.ntab; i += blockDim.x) t[i] = sc.tab[i];
        for (int i = threadIdx.x; i < sc.npairs; i += blockDim.x) {
            p[i] = sc.pairs[i];
            pb[i] = sc.pairs_b[i];
            fr[i] = sc.far[i];
            scc[i] = sc.scan_c[i];
            scb[i] = sc.scan_b[i];
        }
        s.tab = t;
        s.pairs = p;
        s.pairs_b = pb;
        s.far = fr;
        s.scan_c = scc;
        s.scan_b = scb;
        off = ((size_t)sc.ntab * 16 + np * 80 + 15) & ~(size_t)15;   /* frames stay 16-byte aligned */
    } else {
        s.tab = sc.tab;
        s.pairs = sc.pairs;
        s.pairs_b = sc.pairs_b;
        s.far = sc.far;
        s.scan_c = sc.scan_c;
        s.scan_b = sc.scan_b;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    s.frames = reinterpret_cast<float*>(smem + off) + (size_t)warp * lane_floats(sc, VERTEX) * 32 + lane;
    s.cen = s.frames + (size_t)sc.ndof * 12 * 32;
    s.sweep = sweep_area<VERTEX>(sc, s.frames);
    s.defer = defer_area<VERTEX>(sc, s.frames);
    __syncthreads();
    return s;
}

/* Per slot, a ball holding that slot's ball centre in every lane of `mask`
 * (lanes whose frames are current): centre m = the midpoint of the lanes'
 * bounding box, radius rho >= max |c_lane - m| (the box half-diagonal from
 * m, rounded up).  Lanes with a non-finite centre make rho infinite, which
 * disables the sweep tests for the slot.  Lanes 0.. nslots-1 bound the
 * slots' ball centres (sweep[slot]); with at most SWEEP_V0_SLOTS slots,
 * lanes 16.. bound the slots' vertex 0 the same way (sweep[SWEEP_V0_SLOTS
 * + slot]), for the swept direction test of cert_scan. */
constexpr int SWEEP_V0_SLOTS = GPRM_MAX_SLOTS / 2;
__device__ __forceinline__ void sweep_bounds(const DevScene& sc, const SceneView& S, unsigned mask)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();   /* the lanes' centres are written */
    const bool v0 = lane >= 16 && lane - 16 < sc.nslots && sc.nslots <= SWEEP_V0_SLOTS;
    if (lane < sc.nslots || v0) {
        const int sl = v0 ? lane - 16 : lane;
        /* lane 0's points of slot sl; lane i at +i */
        const float* c0 = S.cen - lane + (v0 ? sc.nslots * 3 * 32 : 0) + sl * 3 * 32;
        float lo[3], hi[3];
        bool bad = false;
        for (int c = 0; c < 3; ++c) { lo[c] = PF32::inf(); hi[c] = -PF32::inf(); }
        for (unsigned m = mask; m; m &= m - 1u) {
            const int i = __ffs(m) - 1;
            for (int c = 0; c < 3; ++c) {
                const float v = c0[c * 32 + i];
                bad |= !isfinite(v);
                lo[c] = fminf(lo[c], v);
                hi[c] = fmaxf(hi[c], v);
            }
        }
        float mc[3], e2 = 0.0f;
        for (int c = 0; c < 3; ++c) {
            mc[c] = 0.5f * (lo[c] + hi[c]);
            const float e = fmaxf(hi[c] - mc[c], mc[c] - lo[c]);
            e2 = __fmaf_rn(e, e, e2);
        }
        float rho = __fsqrt_ru(e2) * (1.0f + 4e-6f) + 1e-30f;
        if (bad || !mask || !isfinite(rho)) rho = PF32::inf();
        S.sweep[v0 ? SWEEP_V0_SLOTS + sl : sl] = make_float4(mc[0], mc[1], mc[2], rho);
    }
    __syncwarp();
}

/* Per-lane counts of how pair tests were settled. */
struct PairCounts {
    unsigned long long far, dir, full;
};

/* The ball-distance test of pair_certified for a usable pair (scan_c.w)
 * and this lane: true when it certifies; *d2o and *Do get |D|^2 and D =
 * c_Q - c_P (the moving ball centres from the slots, a static one from
 * far). */
__device__ __forceinline__ bool cert_dist(const SceneView& S, int4 c, float4 f, float* d2o, float3* Do)
{
    const float* cen = S.cen;
    float px = f.x, py = f.y, pz = f.z, qx = f.x, qy = f.y, qz = f.z;
    if (c.x >= 0) { px = cen[(c.x * 3) * 32]; py = cen[(c.x * 3 + 1) * 32]; pz = cen[(c.x * 3 + 2) * 32]; }
    if (c.y >= 0) { qx = cen[(c.y * 3) * 32]; qy = cen[(c.y * 3 + 1) * 32]; qz = cen[(c.y * 3 + 2) * 32]; }
    const float dx = qx - px, dy = qy - py, dz = qz - pz;
    const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
    *d2o = d2;
    *Do = make_float3(dx, dy, dz);
    return d2 > f.w;
}

/* The direction test of pair_certified for a usable pair whose distance
 * test failed (D, d2 from cert_dist), the world vertex 0 of a moving
 * polytope from its slot (the FK pass wrote it with the FMA chain T*v0)
 * and that of a static one from scan_b; branch-free, so that two pairs can
 * be evaluated side by side. */
__device__ __forceinline__ bool cert_dir(const DevScene& sc, const SceneView& S, int4 c, float4 b, float d2,
                                         float3 D)
{
    const float* v0w = S.cen + sc.nslots * 3 * 32;
    float ax = b.x, ay = b.y, az = b.z, bx = b.x, by = b.y, bz = b.z;
    if (c.x >= 0) { ax = v0w[(c.x * 3) * 32]; ay = v0w[(c.x * 3 + 1) * 32]; az = v0w[(c.x * 3 + 2) * 32]; }
    if (c.y >= 0) { bx = v0w[(c.y * 3) * 32]; by = v0w[(c.y * 3 + 1) * 32]; bz = v0w[(c.y * 3 + 2) * 32]; }
    const float dx = D.x, dy = D.y, dz = D.z;
    const float sx = bx - ax, sy = by - ay, sz = bz - az;
    const float n2 = __fmaf_rn(sx, sx, __fmaf_rn(sy, sy, sz * sz));
    const float inv = rsqrtf(n2);
    const float G = __fmaf_rn(sx, dx, __fmaf_rn(sy, dy, sz * dz)) * inv - b.w;
    /* |D| from above: d2 * rsqrt(d2) is within 3 ulp of |D| (rsqrtf <= 2
       ulp), the factor covers it; d2 = 0 gives NaN, which fails the test */
    const float dn = d2 * rsqrtf(d2) * (1.0f + 2e-6f);
    /* direction error <= eps_dir*inv (+ rsqrt and rounding, 1e-6) */
    const float err = (dn + b.w) * __fmaf_rn(sc.eps_dir, inv, 1e-6f);
    return n2 > 1e-6f && G - err > sc.thr_dir;
}

/* The direction test of pair_certified_dir for every lane of the warp at
 * once, for a pair with one moving polytope (slot balls bc: its ball
 * centre, bv: its vertex 0, over the lanes; f: the static partner's ball
 * centre; b: its vertex 0 and R).  With s = b_Q - a_P (vertex 0 of Q minus
 * that of P) = sbar - alpha, |alpha| <= rho_v, and D = c_Q - c_P = Dbar -
 * gamma, |gamma| <= rho_c, every lane has
 *     <s, D> >= <sbar, Dbar> - |sbar| rho_c - rho_v |Dbar| - rho_v rho_c = N
 *     |s| in [|sbar| - rho_v, |sbar| + rho_v],  |D| <= |Dbar| + rho_c,
 * so when N > 0, its G - err of the per-lane test is at least
 *     N / (|sbar| + rho_v) - R - (|Dbar| + rho_c + R)(eps_dir / (|sbar| - rho_v) + 1e-6),
 * which must exceed thr_dir (with 1e-5 relative allowances for the
 * rounding of this bound).  True when every lane's test would certify. */
__device__ __forceinline__ bool swept_direction(const DevScene& sc, bool moving_p, float4 bc, float4 bv, float4 f,
                                                float4 b)
{
    float sx, sy, sz, dx, dy, dz;
    if (moving_p) {
        sx = b.x - bv.x; sy = b.y - bv.y; sz = b.z - bv.z;
        dx = f.x - bc.x; dy = f.y - bc.y; dz = f.z - bc.z;
    } else {
        sx = bv.x - b.x; sy = bv.y - b.y; sz = bv.z - b.z;
        dx = bc.x - f.x; dy = bc.y - f.y; dz = bc.z - f.z;
    }
    const float sn = sqrtf(__fmaf_rn(sx, sx, __fmaf_rn(sy, sy, sz * sz)));
    const float dn = sqrtf(__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz)));
    const float rv = bv.w, rc = bc.w;
    const float N = __fmaf_rn(sx, dx, __fmaf_rn(sy, dy, sz * dz)) * (1.0f - 1e-5f) -
                    (sn * rc + rv * dn + rv * rc) * (1.0f + 1e-5f);
    const float slo = (sn - rv) * (1.0f - 1e-5f), sup = (sn + rv) * (1.0f + 1e-5f);
    if (!(N > 0.0f) || !(slo > 1e-3f)) return false;
    const float err = (dn + rc + b.w) * (sc.eps_dir / slo + 1e-6f) * (1.0f + 1e-5f);
    return (N / sup) * (1.0f - 1e-5f) - b.w * (1.0f + 1e-5f) - err > sc.thr_dir;
}

/* Certificates of pairs j0 .. j0+jn-1 (jn <= 32) for this lane, all
 * order-free (a certified pair is free with its margin above the band, so
 * it changes neither a code nor a band decision), in three stages:
 *   sweep     (SWEPT, lanes holding nearby configurations) lane k tests pair
 *             j0+k against the sweep ball of its moving slot: a pair whose
 *             static partner lies farther than rho + sqrt(T2) from the sweep
 *             centre is settled for every lane at once (each lane's exact
 *             distance then exceeds sqrt(T2)); else the direction test is
 *             bounded over every lane at once (swept_direction) from the
 *             balls of the slot's centre and vertex 0;
 *   per lane  the other pairs, two at a time: the ball-distance and
 *             direction tests (cert_dist_dir), then for the few pairs both
 *             miss the box test of pair_certified_dir; pairs the scan cannot
 *             use go through pair_certified.
 * Returns the pairs that need the exact test (bit k: pair j0+k); 0 for an
 * inactive lane.  Every lane of the warp must call it (the sweep stage
 * votes). */
template <bool SWEPT>
__device__ __forceinline__ unsigned cert_scan(const DevScene& sc, const SceneView& S, int j0, int jn, bool active,
                                              PairCounts& pc)
{
    const int lane = threadIdx.x & 31;
    const unsigned all = jn >= 32 ? FULL_MASK : ((1u << jn) - 1u);
    unsigned cand = all, swept_dir = 0u;
    if constexpr (SWEPT) {
        bool maybe = false, by_dir = false;
        if (lane < jn) {
            maybe = true;
            const int4 c = S.scan_c[j0 + lane];
            if (c.w && ((c.x < 0) != (c.y < 0))) {
                const int ms = c.x >= 0 ? c.x : c.y;
                const float4 f = S.far[j0 + lane];
                const float4 b = S.sweep[ms];
                const float dx = f.x - b.x, dy = f.y - b.y, dz = f.z - b.z;
                const float dd2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
                const float A = (__int_as_float(c.z) + b.w) * (1.0f + 1e-6f);
                /* |m - c|^2 >= dd2 (1 - 1e-6) > A^2 >= (rho + sqrt(T2))^2 */
                if (dd2 * (1.0f - 1e-6f) > A * A) maybe = false;
                else if (sc.nslots <= SWEEP_V0_SLOTS &&
                         swept_direction(sc, c.x >= 0, b, S.sweep[SWEEP_V0_SLOTS + ms], f, S.scan_b[j0 + lane]))
                    maybe = false, by_dir = true;
            }
        }
        cand = __ballot_sync(FULL_MASK, maybe);
        swept_dir = __ballot_sync(FULL_MASK, by_dir);
    }
    if (!active) return 0u;
    pc.far += (unsigned)__popc(all & ~cand & ~swept_dir);
    pc.dir += (unsigned)__popc(swept_dir);
    unsigned need = 0;
#pragma unroll 1
    while (cand) {
        const int k0 = __ffs(cand) - 1;
        cand &= cand - 1u;
        int k1 = k0;
        const bool two = cand != 0;
        if (two) {
            k1 = __ffs(cand) - 1;
            cand &= cand - 1u;
        }
        const int ja = j0 + k0, jb = j0 + k1;
        const int4 ca = S.scan_c[ja], cb = S.scan_c[jb];
        const float4 fa = S.far[ja], fb = S.far[jb];
        const float4 ba = S.scan_b[ja], bb = S.scan_b[jb];
        float d2a = 0.0f, d2b = 0.0f;
        float3 Da = make_float3(0.0f, 0.0f, 0.0f), Db = Da;
        /* 1: distance, 2: direction, 0: neither, -1: not usable by the scan */
        int ra = ca.w ? (cert_dist(S, ca, fa, &d2a, &Da) ? 1 : 0) : -1;
        int rb = (two && cb.w) ? (cert_dist(S, cb, fb, &d2b, &Db) ? 1 : 0) : -1;
        if (ra == 0 && rb == 0) {
            /* both need the direction test: side by side */
            const bool oa = cert_dir(sc, S, ca, ba, d2a, Da), ob = cert_dir(sc, S, cb, bb, d2b, Db);
            ra = oa ? 2 : 0;
            rb = ob ? 2 : 0;
        } else {
            if (ra == 0 && cert_dir(sc, S, ca, ba, d2a, Da)) ra = 2;
            if (rb == 0 && cert_dir(sc, S, cb, bb, d2b, Db)) rb = 2;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 1 && !two) break;
            const int r = h ? rb : ra;
            const int j = h ? jb : ja;
            const int k = h ? k1 : k0;
            if (r == 1) { ++pc.far; continue; }
            if (r == 2) { ++pc.dir; continue; }
            bool ok;
            if (r == 0) {
                /* the box test (pair_certified_dir's last stage) */
                const float3 D = h ? Db : Da;
                ok = pair_certified_dir(sc, S.tab, S.pairs[j], S.pairs_b[j], S.cen, S.frames, j, D.x, D.y, D.z,
                                        h ? d2b : d2a, true);
                if (ok) ++pc.dir;
            } else {
                bool used_dir;
                ok = pair_certified(sc, S.tab, S.pairs[j], S.pairs_b[j], S.cen, S.frames, &used_dir, j);
                if (ok) { if (used_dir) ++pc.dir; else ++pc.far; }
            }
            if (!ok) need |= 1u << k;
        }
    }
    return need;
}

/* The exact test of pair j for this lane (its certificates failed in
 * cert_scan): the pair's code, and its margin in *margin. */
template <bool FAST>
__device__ __forceinline__ int eval_pair(const DevScene& sc, const SceneView& S, int j, float* margin,
                                         PairCounts& pc);

/* The frames of a pair, from the lane's frame array (frame 0 is unused). */
__device__ __forceinline__ void pair_frames(const float* fr, int4 pr, Frame<float>& tp, Frame<float>& tq)
{
    if (pr.z) load_frame(fr, pr.z, tp);
    if (pr.w) load_frame(fr, pr.w, tq);
}

template <bool FAST>
__device__ __forceinline__ int eval_pair(const DevScene& sc, const SceneView& S, int j, float* margin,
                                         PairCounts& pc)
{
    const int4 pr = S.pairs[j];
    ++pc.full;
    Frame<float> tp, tq;
    pair_frames(S.frames, pr, tp, tq);
    if constexpr (FAST) return pair_test_fast(sc, S.tab, pr, sc.ppoly[j], tp, tq, margin);
    else return pair_test<PF32>(sc, S.tab, pr, tp, tq, margin);
}

/* Forward kinematics of a lane into its shared-memory frames, in the
 * arithmetic of the kernel variant. */
template <bool FAST>
__device__ __forceinline__ void lane_fk(const DevScene& sc, const SceneView& S, const float* q)
{
    if constexpr (FAST) forward_kinematics_smem_fast(sc, S.tab, q, S.frames, S.cen);
    else forward_kinematics_smem(sc, S.tab, q, S.frames, S.cen);
}

__device__ __forceinline__ void flush_counts(PairCounts pc, Control* ctl)
{
    for (int o = 16; o > 0; o >>= 1) {
        pc.far += __shfl_xor_sync(0xffffffffu, pc.far, o);
        pc.dir += __shfl_xor_sync(0xffffffffu, pc.dir, o);
        pc.full += __shfl_xor_sync(0xffffffffu, pc.full, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (pc.far) atomicAdd(&ctl->cert_far, pc.far);
        if (pc.dir) atomicAdd(&ctl->cert_dir, pc.dir);
        if (pc.full) atomicAdd(&ctl->full_tests, pc.full);
    }
}

/* ------------------------------------------------------------------ */
/* deferred exact pair tests                                            */
/* ------------------------------------------------------------------ */
/*
 * Within a chunk of 32 pairs, the pairs a lane must test exactly are not run
 * where they are found (where most of the warp would idle) but queued as
 * items (owner lane, pair - j0) in the warp's shared area; every 32 items
 * the whole warp runs one each on its owner's frames.  Items reach the
 * queue in pair order, so each owner applies its results in pair order:
 * the first colliding pair decides its code (later items are ignored) and
 * the free ones before it feed its minimum margin, exactly as the
 * sequential loop.  first_k records the chunk index of that first
 * collision (DEFER_NONE: none in this chunk).
 *
 * Vertex checks use it: their lanes hold unrelated configurations, so the
 * pairs left to test differ from lane to lane (measured on hull6 with 2^20
 * samples: 11.0 -> 8.6 ms).  The lanes of an edge check hold neighbouring
 * steps of one edge, which mostly need the same pairs; there the queue
 * costs more than it saves (357 -> 436 ms) and the sequential loop stays.
 */
constexpr int DEFER_NONE = 32;

struct LaneState {
    int code;
    float mdec, mmin;
    bool active;
    int first_k;
    int jrec, jlast;   /* first and last pair decided within the band (collision or margin < band) */
};

__device__ __forceinline__ void defer_push(unsigned* q, int& n, bool want, int k)
{
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(FULL_MASK, want);
    if (want) q[n + __popc(m & ((1u << lane) - 1u))] = (unsigned)lane | ((unsigned)k << 5);
    n += __popc(m);
}

/* Runs the first cnt (<= 32) queued items, one per lane, and lets every
 * owner apply its results; the remaining items move to the front. */
template <bool FAST>
__device__ __forceinline__ void defer_run(const DevScene& sc, const SceneView& S, int j0, int& n, int cnt,
                                          LaneState& st, PairCounts& pc, float band)
{
    const int lane = threadIdx.x & 31;
    unsigned* q = S.defer;
    int* rcode = reinterpret_cast<int*>(q + 64);
    float* rm = reinterpret_cast<float*>(q + 96);
    __syncwarp();
    int c = 0;
    float m = 0.0f;
    if (lane < cnt) {
        const unsigned it = q[lane];
        const int owner = (int)(it & 31u);
        const int jj = j0 + (int)(it >> 5);
        const int4 pr = S.pairs[jj];
        Frame<float> tp, tq;
        pair_frames(S.frames - lane + owner, pr, tp, tq);
        if constexpr (FAST) c = pair_test_fast(sc, S.tab, pr, sc.ppoly[jj], tp, tq, &m);
        else c = pair_test<PF32>(sc, S.tab, pr, tp, tq, &m);
        ++pc.full;
    }
    rcode[lane] = c;
    rm[lane] = m;
    __syncwarp();
#pragma unroll 1
    for (int t = 0; t < cnt; ++t) {
        const unsigned it = q[t];
        if ((int)(it & 31u) == lane && st.first_k == DEFER_NONE) {
            const int ct = rcode[t];
            const int jj = j0 + (int)(it >> 5);
            if (ct != 0) {
                st.code = ct;
                st.mdec = rm[t];
                st.first_k = (int)(it >> 5);
                st.active = false;
                st.jrec = min(st.jrec, jj);
            } else {
                st.mmin = min_nan(st.mmin, rm[t]);
                if (!(rm[t] >= band)) {
                    st.jrec = min(st.jrec, jj);
                    st.jlast = max(st.jlast, jj);
                }
            }
        }
    }
    const int rest = n - cnt;
    __syncwarp();
    const unsigned mv = lane < rest ? q[cnt + lane] : 0u;
    __syncwarp();
    if (lane < rest) q[lane] = mv;
    n = rest;
    __syncwarp();
}

/* One chunk's ordered pass with deferral: the pairs whose certificates
 * failed (need, from cert_scan) are queued in pair order. */
template <bool FAST>
__device__ __forceinline__ void defer_chunk(const DevScene& sc, const SceneView& S, int j0, unsigned need,
                                            unsigned todo, LaneState& st, PairCounts& pc, float band)
{
    int n = 0;
    st.first_k = DEFER_NONE;
    while (todo) {
        const int k = __ffs(todo) - 1;
        todo &= todo - 1u;
        const bool full = st.active && ((need >> k) & 1u);
        defer_push(S.defer, n, full, k);
        if (n >= 32) defer_run<FAST>(sc, S, j0, n, 32, st, pc, band);
    }
    while (n > 0) defer_run<FAST>(sc, S, j0, n, n < 32 ? n : 32, st, pc, band);
}

/* Appends the items of the lanes with `want` set, one atomic per warp;
 * range: the pairs the item's FP64 recheck tests (BandQueue::pair_range). */
__device__ __forceinline__ unsigned recheck_range(int code, int jfirst, int jlast, int npairs)
{
    if (jfirst >= npairs) return (unsigned)npairs << 16;          /* not recorded: every pair */
    const int hi = code != 0 ? npairs : (jlast < npairs ? jlast + 1 : npairs);
    return (unsigned)jfirst | ((unsigned)hi << 16);
}

__device__ __forceinline__ void warp_append(bool want, uint2 item, unsigned range, BandQueue bq,
                                            Control* ctl)
{
    unsigned m = __ballot_sync(FULL_MASK, want);
    if (!m) return;
    int lane = threadIdx.x & 31;
    unsigned base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(&ctl->qcount, (unsigned)__popc(m));
    base = __shfl_sync(FULL_MASK, base, __ffs(m) - 1);
    if (want) {
        unsigned slot = base + __popc(m & ((1u << lane) - 1));
        if (slot < bq.cap) {
            bq.items[slot] = item;
            if (bq.pair_range) bq.pair_range[slot] = range;
        } else {
            atomicOr(&ctl->flags, GPRM_DEVFLAG_QUEUE_FULL);
            const unsigned x = item.x;
            if (bq.ovf && (long long)x < bq.n) {
                const unsigned bit = 1u << (x & 31u);
                if (!(atomicOr(&bq.ovf[bq.n + (x >> 5)], bit) & bit))
                    bq.ovf[atomicAdd(&ctl->ovf_count, 1ull)] = x;
            }
        }
    }
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x)
{
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
    return x;
}

/* ------------------------------------------------------------------ */
/* vertex checks                                                        */
/* ------------------------------------------------------------------ */

/* Configurations i0 .. i0+count-1 (count <= 32), one per lane. */
template <bool FAST>
__device__ __forceinline__ void check_config_chunk(const DevScene& sc, const SceneView& S, const float* __restrict__ q,
                                                   long long offset, long long i0, int count, int* __restrict__ res,
                                                   int band_on, float band, BandQueue bq,
                                                   Control* ctl, PairCounts& pc, unsigned long long& exec)
{
    const int lane = threadIdx.x & 31;
    const long long i = i0 + lane;
    const bool valid = lane < count;
    float qi[GPRM_MAX_FRAMES];
    int code = 0;
    bool active = valid;
    if (valid) {
        for (int j = 0; j < sc.ndof; ++j) qi[j] = q[i + offset * j];
        /* check_boundaries(q) (robotconfigspace.cpp:795-802) */
        for (int j = 0; j < sc.ndof; ++j)
            if (qi[j] < sc.mins[j] || qi[j] > sc.maxs[j]) { code = 1; active = false; break; }
    }
    if (active) lane_fk<FAST>(sc, S, qi);
    LaneState st{code, 0.0f, PF32::inf(), active, DEFER_NONE, 0x7fffffff, -1};
    /* pairs in chunks of 32: the order-free certificate scan, then the
       pairs left for the exact test in the reference's order, their exact
       tests deferred and run by the whole warp */
#pragma unroll 1
    for (int j0 = 0; j0 < sc.npairs; j0 += 32) {
        if (!__any_sync(FULL_MASK, st.active)) break;
        const int jn = min(32, sc.npairs - j0);
        const unsigned need = cert_scan<false>(sc, S, j0, jn, st.active, pc);
        const unsigned todo = __reduce_or_sync(FULL_MASK, need);
        defer_chunk<FAST>(sc, S, j0, need, todo, st, pc, band);
    }
    code = st.code;
    const float mmin = st.mmin, mdec = st.mdec;
    if (valid) {
        exec += (code != 1);
        res[i] = code;
    }
    bool want = valid && band_on && code != 1 && in_band(code, code == 0 ? mmin : mdec, band);
    warp_append(want, make_uint2((unsigned)i, (unsigned)(code + 1) << 27),
                recheck_range(code, st.jrec, st.jlast, sc.npairs), bq, ctl);
}

template <bool SMEM, bool FAST>
__global__ void GPRM_BOUNDS k_check_configs(DevScene sc, const float* __restrict__ q,
                                            long long n, long long offset,
                                            int* __restrict__ res, int band_on, float band,
                                            BandQueue bq,
                                            Control* ctl)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SceneView S = stage_scene<SMEM, true>(sc, smem);
    const int lane = threadIdx.x & 31;
    unsigned long long exec = 0;
    PairCounts pc = {0, 0, 0};
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&ctl->next, 32ull);
        base = __shfl_sync(FULL_MASK, base, 0);
        if (base >= (unsigned long long)n) break;
        const long long left = n - (long long)base;
        check_config_chunk<FAST>(sc, S, q, offset, (long long)base, left < 32 ? (int)left : 32, res, band_on,
                                 band, bq, ctl, pc, exec);
    }
    exec = warp_sum(exec);
    if (lane == 0 && exec) atomicAdd(&ctl->configs_exec, exec);
    flush_counts(pc, ctl);
}

/* ------------------------------------------------------------------ */
/* edge checks                                                          */
/* ------------------------------------------------------------------ */

/* Edge keys (one uint32 per edge, decoded by k_finalize_edges):
 *   early exit  min over colliding steps of (order << 4 | (code+1)),
 *               0xffffffff = free
 *   all steps   max over colliding steps of ((t+1) << 4 | (code+1)),
 *               0 = free                                                   */
__device__ __forceinline__ unsigned early_key(unsigned order, int code) { return (order << 4) | (unsigned)(code + 1); }
__device__ __forceinline__ unsigned all_key(int t, int code) { return ((unsigned)(t + 1) << 4) | (unsigned)(code + 1); }

/* Segments of an edge of R rounds when a batch splits its edges into
 * pieces of about seg_rounds rounds (at most EDGE_MAX_SEGS per edge). */
constexpr int EDGE_MAX_SEGS = 64;
__device__ __forceinline__ int edge_seg_count(int R, int seg_rounds)
{
    const int s = (R + seg_rounds - 1) / seg_rounds;
    return s < EDGE_MAX_SEGS ? s : EDGE_MAX_SEGS;
}

/* One edge e (testnum steps, rounds of 32 steps over the lanes), or with
 * seg_rounds > 0 its segment `seg`: a contiguous range of rounds, so that
 * several warps share a long edge.  The rounds keep their step order, a
 * segment's decision is merged into key[e] atomically (min for early exit,
 * max for all steps, the same merge as the FP64 recheck) and a segment
 * stops once key[e] holds a decision that none of its remaining rounds can
 * improve on. */
template <int POLICY, bool SPLIT, bool FAST>
__device__ __forceinline__ void check_edge(const DevScene& sc, const SceneView& S, const float* __restrict__ qs,
                                           const float* __restrict__ qe, long long e, long long offset, float dq,
                                           unsigned* __restrict__ key, int band_on, float band,
                                           BandQueue bq, Control* ctl, PairCounts& pc,
                                           unsigned long long& exec, unsigned long long& nominal,
                                           int seg = 0, int seg_rounds = 0)
{
    const int lane = threadIdx.x & 31;
    const int tn = edge_testnum(qs, qe, e, offset, sc.ndof, dq);
    if (tn < 0) {
        if (lane == 0 && seg == 0) atomicOr(&ctl->flags, GPRM_DEVFLAG_BAD_EDGE);
        return;
    }
    if (lane == 0 && seg == 0) nominal += tn;
    const int R = (tn + 31) >> 5;
    int r_begin = 0, r_end = R;
    if constexpr (SPLIT) {
        const int ns = edge_seg_count(R, seg_rounds);
        const int rs = (R + ns - 1) / ns;
        r_begin = seg * rs;
        r_end = min(R, r_begin + rs);
    }
    bool decided = false;
#pragma unroll 1
    for (int r = r_begin; r < r_end && !decided; ++r) {
        if constexpr (SPLIT) {
            const unsigned kv = *(volatile const unsigned*)&key[e];
            const bool beaten = (POLICY == EDGE_EARLY_EXIT)
                ? (kv != 0xffffffffu && (kv >> 4) < (unsigned)(r * 32))
                : (kv != 0u && (int)(kv >> 4) - 1 > tn - 1 - r * 32);
            if (__any_sync(FULL_MASK, beaten)) break;
        }
        int t;
        unsigned order;
        bool valid;
        if (POLICY == EDGE_EARLY_EXIT) {
            t = lane * R + r;
            valid = t < tn;
            order = (unsigned)(r * 32 + lane);
        } else {
            int idx = r * 32 + lane;
            t = tn - 1 - idx;
            valid = idx < tn;
            order = 0;
        }
        float qi[GPRM_MAX_FRAMES];
        if (valid) {
            edge_step_config(qs, qe, e, offset, sc.ndof, t, tn, qi);
            lane_fk<FAST>(sc, S, qi);
        }
        const unsigned valid_mask = __ballot_sync(FULL_MASK, valid);
        if (lane == 0) exec += __popc(valid_mask);
        sweep_bounds(sc, S, valid_mask);
        bool active = valid;
        int code = 0;
        float mmin = PF32::inf(), mdec = 0.0f;
        int cut = 32;   /* lanes above the highest-priority colliding lane no longer matter */
        int jend = 0;   /* pairs processed by the warp */
        int jrec = 0x7fffffff, jlast = -1;   /* first and last pair decided within the band */
        bool stop = false;
        /* pairs in chunks of 32: the order-free certificate scan, then the
           pairs left for the exact test in the reference's order; a code can
           only change at such a pair, so the vote runs only there */
#pragma unroll 1
        for (int j0 = 0; j0 < sc.npairs && !stop; j0 += 32) {
            if (!__any_sync(FULL_MASK, active)) break;
            const int jn = min(32, sc.npairs - j0);
            const unsigned need = cert_scan<true>(sc, S, j0, jn, active, pc);
            unsigned todo = __reduce_or_sync(FULL_MASK, need);
            while (todo) {
                const int k = __ffs(todo) - 1;
                todo &= todo - 1u;
                if (active && ((need >> k) & 1u)) {
                    float m;
                    const int rr = eval_pair<FAST>(sc, S, j0 + k, &m, pc);
                    if (rr != 0) { code = rr; mdec = m; active = false; jrec = min(jrec, j0 + k); }
                    else {
                        mmin = min_nan(mmin, m);
                        if (!(m >= band)) { jrec = min(jrec, j0 + k); jlast = j0 + k; }
                    }
                }
                jend = j0 + k + 1;
                bool oobj = code != 0 && !(band_on && in_band(code, mdec, band));
                unsigned hits = __ballot_sync(FULL_MASK, oobj);
                if (hits) {
                    int Lj = __ffs(hits) - 1;
                    if (Lj < cut) cut = Lj;
                    if (POLICY == EDGE_EARLY_EXIT) { stop = true; break; }
                    if (lane > cut) active = false;
                }
            }
            if (!stop) jend = j0 + jn;
        }
        /* settle the round */
        const bool oob = code != 0 && !(band_on && in_band(code, mdec, band));
        const unsigned hits = __ballot_sync(FULL_MASK, oob && lane <= cut);
        const int L = hits ? __ffs(hits) - 1 : 32;
        const bool free_done = valid && code == 0 && active && jend == sc.npairs;
        const bool inb = band_on && ((code != 0 && !oob) || (free_done && in_band(0, mmin, band)));
        /* in-band steps earlier in order (early exit) or higher t (all steps)
           than the deciding step go to the FP64 queue */
        const bool want = inb && lane < L;
        warp_append(want, make_uint2((unsigned)e, (unsigned)t | ((unsigned)(code + 1) << 27)),
                    recheck_range(code, jrec, jlast, sc.npairs), bq, ctl);
        if (hits) {
            if (lane == L) {
                const unsigned kv = (POLICY == EDGE_EARLY_EXIT) ? early_key(order, code) : all_key(t, code);
                if constexpr (!SPLIT) key[e] = kv;
                else if (POLICY == EDGE_EARLY_EXIT) atomicMin(&key[e], kv);
                else atomicMax(&key[e], kv);
            }
            decided = true;
        }
    }
}

__device__ __forceinline__ void flush_edge_counts(unsigned long long exec, unsigned long long nominal, PairCounts pc,
                                                  Control* ctl)
{
    exec = warp_sum(exec);
    nominal = warp_sum(nominal);
    if ((threadIdx.x & 31) == 0) {
        if (exec) atomicAdd(&ctl->steps_exec, exec);
        if (nominal) atomicAdd(&ctl->steps_nominal, nominal);
    }
    flush_counts(pc, ctl);
}

/* SPLIT: the work items are the segments of the edges, edge e owning
 * items [seg_off[e], seg_off[e+1]) (seg_off from k_edge_segments);
 * otherwise one item per edge and seg_off is unused. */
template <bool SMEM, int POLICY, bool SPLIT, bool FAST>
__global__ void GPRM_BOUNDS k_check_edges(DevScene sc, const float* __restrict__ qs,
                                          const float* __restrict__ qe, long long n,
                                          long long offset, float dq, unsigned* __restrict__ key,
                                          int band_on, float band, BandQueue bq, Control* ctl,
                                          const unsigned* __restrict__ seg_off,
                                          int seg_rounds)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SceneView S = stage_scene<SMEM, false>(sc, smem);
    const int lane = threadIdx.x & 31;
    unsigned long long exec = 0, nominal = 0;
    PairCounts pc = {0, 0, 0};
    if constexpr (!SPLIT) {
        for (;;) {
            unsigned long long eu = 0;
            if (lane == 0) eu = atomicAdd(&ctl->next, 1ull);
            eu = __shfl_sync(FULL_MASK, eu, 0);
            if (eu >= (unsigned long long)n) break;
            check_edge<POLICY, false, FAST>(sc, S, qs, qe, (long long)eu, offset, dq, key, band_on, band, bq, ctl,
                                            pc, exec, nominal);
        }
        flush_edge_counts(exec, nominal, pc, ctl);
        return;
    }
    const unsigned long long items = (unsigned long long)seg_off[n];
    for (;;) {
        unsigned long long eu = 0;
        long long e = 0;
        int seg = 0;
        if (lane == 0) {
            eu = atomicAdd(&ctl->next, 1ull);
            if (eu < items) {
                long long lo = 0, hi = n;       /* seg_off[lo] <= eu < seg_off[hi] */
                while (hi - lo > 1) {
                    const long long mid = (lo + hi) >> 1;
                    if ((unsigned long long)seg_off[mid] <= eu) lo = mid;
                    else hi = mid;
                }
                e = lo;
                seg = (int)(eu - seg_off[lo]);
            }
        }
        eu = __shfl_sync(FULL_MASK, eu, 0);
        if (eu >= items) break;
        e = __shfl_sync(FULL_MASK, e, 0);
        seg = __shfl_sync(FULL_MASK, seg, 0);
        check_edge<POLICY, true, FAST>(sc, S, qs, qe, e, offset, dq, key, band_on, band, bq, ctl, pc,
                                       exec, nominal, seg, seg_rounds);
    }
    flush_edge_counts(exec, nominal, pc, ctl);
}

/* Segment offsets of n edges (one block): seg_off[e] = sum over e' < e of
 * the segment count of edge e', seg_off[n] = the total.  Edges the check
 * rejects (non-finite or oversized) count one segment. */
__global__ void __launch_bounds__(1024) k_edge_segments(const float* __restrict__ qs, const float* __restrict__ qe,
                                                        long long n, long long offset, int ndof, float dq,
                                                        int seg_rounds, unsigned* __restrict__ seg_off)
{
    __shared__ unsigned wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long per = (n + blockDim.x - 1) / blockDim.x;
    const long long b0 = min(n, (long long)tid * per), b1 = min(n, b0 + per);
    auto segs = [&](long long e) -> unsigned {
        const int tn = edge_testnum(qs, qe, e, offset, ndof, dq);
        return tn < 0 ? 1u : (unsigned)edge_seg_count((tn + 31) >> 5, seg_rounds);
    };
    unsigned s = 0;
    for (long long e = b0; e < b1; ++e) s += segs(e);
    unsigned x = s;                                    /* inclusive scan in the warp */
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned y = __shfl_up_sync(FULL_MASK, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        unsigned w = lane < nw ? wsum[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned y = __shfl_up_sync(FULL_MASK, w, d);
            if (lane >= d) w += y;
        }
        if (lane < nw) wsum[lane] = w;                 /* inclusive warp totals */
    }
    __syncthreads();
    unsigned base = x - s + (warp > 0 ? wsum[warp - 1] : 0u);
    for (long long e = b0; e < b1; ++e) {
        seg_off[e] = base;
        base += segs(e);
    }
    if (tid == (int)blockDim.x - 1) seg_off[n] = base;
}

/* Segment count of edge e for the split kernels (a rejected edge counts
 * one segment). */
__device__ __forceinline__ unsigned edge_segs(const float* __restrict__ qs, const float* __restrict__ qe, long long e,
                                              long long offset, int ndof, float dq, int seg_rounds)
{
    const int tn = edge_testnum(qs, qe, e, offset, ndof, dq);
    return tn < 0 ? 1u : (unsigned)edge_seg_count((tn + 31) >> 5, seg_rounds);
}

/* Exclusive scan of x over the block (blockDim.x <= 1024, a multiple of
 * 32); *total gets the block's sum.  wsum: 32 words of shared memory. */
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned x, unsigned* wsum, unsigned* total)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    unsigned v = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned y = __shfl_up_sync(FULL_MASK, v, d);
        if (lane >= d) v += y;
    }
    if (lane == 31) wsum[warp] = v;
    __syncthreads();
    if (warp == 0) {
        unsigned w = lane < nw ? wsum[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned y = __shfl_up_sync(FULL_MASK, w, d);
            if (lane >= d) w += y;
        }
        if (lane < nw) wsum[lane] = w;                 /* inclusive warp totals */
    }
    __syncthreads();
    const unsigned ex = v - x + (warp > 0 ? wsum[warp - 1] : 0u);
    *total = wsum[nw - 1];
    __syncthreads();
    return ex;
}

/* Segment offsets of more than EDGE_SPLIT_ONE_BLOCK edges, in three
 * passes: block b (of EDGE_SEG_BLOCKS) takes the edges [b c, (b+1) c),
 * c = ceil(n / blocks), each thread a contiguous run of them.  Pass 0
 * writes the block's segment count to bsum[b]; k_seg_scan_blocks turns
 * bsum into exclusive offsets (and seg_off[n] into the total); pass 1
 * writes seg_off[e] for the block's edges. */
template <int PASS>
__global__ void __launch_bounds__(256) k_seg_pass(const float* __restrict__ qs, const float* __restrict__ qe,
                                                  long long n, long long offset, int ndof, float dq, int seg_rounds,
                                                  unsigned* __restrict__ seg_off, unsigned* __restrict__ bsum)
{
    __shared__ unsigned wsum[32];
    const long long chunk = (n + gridDim.x - 1) / gridDim.x;
    const long long c0 = min(n, (long long)blockIdx.x * chunk), c1 = min(n, c0 + chunk);
    const long long per = (c1 - c0 + blockDim.x - 1) / blockDim.x;
    const long long b0 = min(c1, c0 + (long long)threadIdx.x * per), b1 = min(c1, b0 + per);
    unsigned s = 0;
    for (long long e = b0; e < b1; ++e) s += edge_segs(qs, qe, e, offset, ndof, dq, seg_rounds);
    unsigned total = 0;
    unsigned base = block_exclusive_scan(s, wsum, &total);
    if (PASS == 0) {
        if (threadIdx.x == 0) bsum[blockIdx.x] = total;
        return;
    }
    base += bsum[blockIdx.x];
    for (long long e = b0; e < b1; ++e) {
        seg_off[e] = base;
        base += edge_segs(qs, qe, e, offset, ndof, dq, seg_rounds);
    }
}

/* bsum[0..nb) -> exclusive offsets, *total_out = their sum (one block of
 * 1024 threads, nb <= 1024). */
__global__ void __launch_bounds__(1024) k_seg_scan_blocks(unsigned* __restrict__ bsum, int nb,
                                                          unsigned* __restrict__ total_out)
{
    __shared__ unsigned wsum[32];
    const int t = threadIdx.x;
    const unsigned x = t < nb ? bsum[t] : 0u;
    unsigned total = 0;
    const unsigned ex = block_exclusive_scan(x, wsum, &total);
    if (t < nb) bsum[t] = ex;
    if (t == 0) *total_out = total;
}

/* ------------------------------------------------------------------ */
/* FP64 recheck and finalisation                                        */
/* ------------------------------------------------------------------ */

/* The FP64 check of one configuration (in bounds): the reference's pair
 * loop in double with the FP64 certificates, over pairs [j_start, j_end)
 * (the pairs outside that range were decided separated outside the band by
 * the FP32 check, so in FP64 they are separated too, and the first
 * colliding pair, hence the code, is the same as over every pair). */
__device__ __forceinline__ int check_config64(const DevScene& sc, const float* qi, int j_start = 0, int j_end = -1)
{
    if (j_end < 0 || j_end > sc.npairs) j_end = sc.npairs;
    Frame<double> F[GPRM_MAX_FRAMES];
    forward_kinematics<PF64>(sc, qi, F);
    /* slot ball centres in FP64, once per check (the same transform the
       certificate would apply per pair) */
    double cen[GPRM_MAX_SLOTS * 3];
    for (int sl = 0; sl < sc.nslots; ++sl) {
        const float4 b = sc.tab[sc.slot_block[sl]];
        const V3<double> c = xform<double>(F[sc.slot_sys[sl]], (double)b.x, (double)b.y, (double)b.z);
        cen[3 * sl] = c.x; cen[3 * sl + 1] = c.y; cen[3 * sl + 2] = c.z;
    }
#pragma unroll 1
    for (int j = j_start; j < j_end; ++j) {
        const int4 pr = sc.pairs[j];
        if (pair_certified64(sc, sc.tab, pr, sc.pairs_b[j], F, cen, j)) continue;
        double m;
        const int r = pair_test<PF64>(sc, sc.tab, pr, F[pr.z], F[pr.w], &m);
        if (r != 0) return r;
    }
    return 0;
}

/* The item's configuration (vertex kind 0 or edge step kind 1); for an
 * edge step also its step t and the edge's step count tn. */
__device__ __forceinline__ void recheck_config(const DevScene& sc, int kind, uint2 it, const float* __restrict__ q,
                                               const float* __restrict__ qs, const float* __restrict__ qe,
                                               long long offset, float dq, float* qi, int& t, int& tn)
{
    t = 0;
    tn = 0;
    if (kind == 0) {
        for (int j = 0; j < sc.ndof; ++j) qi[j] = q[(long long)it.x + offset * j];
    } else {
        t = (int)(it.y & ((1u << 27) - 1));
        tn = edge_testnum(qs, qe, (long long)it.x, offset, sc.ndof, dq);
        edge_step_config(qs, qe, (long long)it.x, offset, sc.ndof, t, tn, qi);
    }
}

/* Writes an FP64 recheck's code: a configuration's result, or an edge
 * step's key merge (the order of the check kernel for early exit). */
__device__ __forceinline__ void recheck_store(int kind, uint2 it, int code, int t, int tn, int policy,
                                              int* __restrict__ res, unsigned* __restrict__ key)
{
    if (kind == 0) {
        res[it.x] = code;
    } else if (code != 0) {
        if (policy == EDGE_EARLY_EXIT) {
            const int R = (tn + 31) >> 5;
            const unsigned order = (unsigned)((t % R) * 32 + t / R);
            atomicMin(&key[it.x], early_key(order, code));
        } else {
            atomicMax(&key[it.x], all_key(t, code));
        }
    }
}

/* The FP32 check of one configuration (in bounds) in one thread, in the
 * arithmetic of the kernel variant (FAST), frames in registers: every
 * pair's exact test in the reference's order (the certificates only ever
 * skip pairs whose test gives 0 with a margin above the band, so the code
 * and the band decision are those of the warp kernels).  *margin: the
 * deciding pair's margin, or the minimum over the pairs of a free check;
 * *jdec (when given): the deciding pair's index, npairs for a free check. */
template <bool FAST>
__device__ __forceinline__ int check_config32(const DevScene& sc, const float* qi, float* margin,
                                              int* jdec = nullptr)
{
    Frame<float> F[GPRM_MAX_FRAMES];
    if constexpr (FAST) forward_kinematics_fast(sc, qi, F);
    else forward_kinematics<PF32>(sc, qi, F);
    float mmin = PF32::inf();
#pragma unroll 1
    for (int j = 0; j < sc.npairs; ++j) {
        const int4 pr = sc.pairs[j];
        float m;
        int r;
        if constexpr (FAST) r = pair_test_fast(sc, sc.tab, pr, sc.ppoly[j], F[pr.z], F[pr.w], &m);
        else r = pair_test<PF32>(sc, sc.tab, pr, F[pr.z], F[pr.w], &m);
        if (r != 0) {
            *margin = m;
            if (jdec) *jdec = j;
            return r;
        }
        mmin = min_nan(mmin, m);
    }
    *margin = mmin;
    if (jdec) *jdec = sc.npairs;
    return 0;
}

/* One item of the overflow list, recomputed in full by one thread: a
 * configuration (kind 0: bounds, FP32, FP64 inside the band -> res), or an
 * edge (kind 1), whose key is rebuilt from scratch as the check and recheck
 * kernels build it when nothing overflows:
 *   all steps   the max over every step (FP32, FP64 inside the band);
 *   early exit  the check kernel's rounds (round r: steps t = lane*R + r,
 *               order r*32 + lane) until the first round with a collision
 *               outside the band.  The kernel runs a round pair by pair in
 *               the reference's pair order and stops at the first pair
 *               index j* at which some step collides outside the band; its
 *               lowest such lane L decides.  Steps of lower lanes whose
 *               loop had ended by then in the band (a collision at a pair
 *               <= j*, or a free check when nothing decided) go to the FP64
 *               check, and a collision there takes the lower order. */
template <bool FAST>
__device__ __forceinline__ void overflow_item(const DevScene& sc, int kind, unsigned x, const float* __restrict__ q,
                                              const float* __restrict__ qs, const float* __restrict__ qe,
                                              long long offset, float dq, int policy, float band,
                                              int* __restrict__ res, unsigned* __restrict__ key,
                                              unsigned long long& checks, unsigned long long& flips)
{
    float qi[GPRM_MAX_FRAMES];
    if (kind == 0) {
        for (int j = 0; j < sc.ndof; ++j) qi[j] = q[(long long)x + offset * j];
        int code = 0;
        for (int j = 0; j < sc.ndof; ++j)
            if (qi[j] < sc.mins[j] || qi[j] > sc.maxs[j]) { code = 1; break; }
        if (code == 0) {
            float m;
            code = check_config32<FAST>(sc, qi, &m);
            if (in_band(code, m, band)) {
                const int c64 = check_config64(sc, qi);
                ++checks;
                flips += ((c64 != 0) != (code != 0));
                code = c64;
            }
        }
        res[x] = code;
        return;
    }
    const int tn = edge_testnum(qs, qe, (long long)x, offset, sc.ndof, dq);
    if (tn < 0) return;   /* flagged by the check kernel */
    const int R = (tn + 31) >> 5;
    if (policy != EDGE_EARLY_EXIT) {
        unsigned k = 0u;
#pragma unroll 1
        for (int t = 0; t < tn; ++t) {
            edge_step_config(qs, qe, (long long)x, offset, sc.ndof, t, tn, qi);
            float m;
            int code = check_config32<FAST>(sc, qi, &m);
            if (in_band(code, m, band)) {
                const int c64 = check_config64(sc, qi);
                ++checks;
                flips += ((c64 != 0) != (code != 0));
                code = c64;
            }
            if (code != 0) {
                const unsigned kv = all_key(t, code);
                if (kv > k) k = kv;
            }
        }
        key[x] = k;
        return;
    }
    unsigned k = 0xffffffffu;
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
        /* the round's deciding pair index j* and lane L */
        int jstar = 0x7fffffff, L = 32, codeL = 0;
#pragma unroll 1
        for (int lane = 0; lane < 32; ++lane) {
            const int t = lane * R + r;
            if (t >= tn) break;
            edge_step_config(qs, qe, (long long)x, offset, sc.ndof, t, tn, qi);
            float m;
            int j;
            const int code = check_config32<FAST>(sc, qi, &m, &j);
            if (code != 0 && !in_band(code, m, band) && j < jstar) { jstar = j; L = lane; codeL = code; }
        }
        /* the in-band steps below L that the kernel queues */
#pragma unroll 1
        for (int lane = 0; lane < L; ++lane) {
            const int t = lane * R + r;
            if (t >= tn) break;
            edge_step_config(qs, qe, (long long)x, offset, sc.ndof, t, tn, qi);
            float m;
            int j;
            const int code = check_config32<FAST>(sc, qi, &m, &j);
            const bool queued = code != 0 ? (in_band(code, m, band) && j <= jstar)
                                          : (L == 32 && in_band(0, m, band));
            if (!queued) continue;
            const int c64 = check_config64(sc, qi);
            ++checks;
            flips += ((c64 != 0) != (code != 0));
            if (c64 != 0) {
                const unsigned kv = early_key((unsigned)(r * 32 + lane), c64);
                if (kv < k) k = kv;
            }
        }
        if (L < 32) {
            const unsigned kv = early_key((unsigned)(r * 32 + L), codeL);
            if (kv < k) k = kv;
            break;
        }
    }
    key[x] = k;
}

/* The FP64 recheck of the queued items, one thread per item.  (A warp per
 * item, the pairs spread over the lanes, ran 1.4x slower on the hull6
 * edge workload: the items' own parallelism hides the FP64 latency better.) */
constexpr int RECHECK_THREADS = 128;

__device__ __forceinline__ void recheck_item(const DevScene& sc, int kind, uint2 it, const float* __restrict__ q,
                                             const float* __restrict__ qs, const float* __restrict__ qe,
                                             long long offset, float dq, int policy, int* __restrict__ res,
                                             unsigned* __restrict__ key, unsigned long long& checks,
                                             unsigned long long& flips, unsigned range)
{
    float qi[GPRM_MAX_FRAMES];
    int t, tn;
    recheck_config(sc, kind, it, q, qs, qe, offset, dq, qi, t, tn);
    const int code = check_config64(sc, qi, (int)(range & 0xffffu), (int)(range >> 16));
    ++checks;
    flips += ((code != 0) != ((int)(it.y >> 27) - 1 != 0));
    recheck_store(kind, it, code, t, tn, policy, res, key);
}

__global__ void __launch_bounds__(RECHECK_THREADS) k_recheck(DevScene sc, int kind, const float* __restrict__ q,
                                                             const float* __restrict__ qs,
                                                             const float* __restrict__ qe, long long offset,
                                                             float dq, int policy, int* __restrict__ res,
                                                             unsigned* __restrict__ key, const BandQueue bq,
                                                             Control* ctl)
{
    unsigned cnt = ctl->qcount;
    if (cnt > bq.cap) cnt = bq.cap;
    unsigned long long checks = 0, flips = 0;
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += gridDim.x * blockDim.x)
        recheck_item(sc, kind, bq.items[idx], q, qs, qe, offset, dq, policy, res, key, checks, flips,
                     bq.pair_range ? bq.pair_range[idx] : 0xffff0000u);
    if (checks) atomicAdd(&ctl->band_checks, checks);
    if (flips) atomicAdd(&ctl->band_flips, flips);
}

/* The overflow pass of a request: every item in the overflow list,
 * recomputed by one thread (overflow_item).  Exits at once when nothing
 * overflowed. */
template <bool FAST>
__global__ void __launch_bounds__(128) k_overflow(DevScene sc, int kind, const float* __restrict__ q,
                                                  const float* __restrict__ qs, const float* __restrict__ qe,
                                                  long long offset, float dq, int policy, float band,
                                                  int* __restrict__ res, unsigned* __restrict__ key, BandQueue bq,
                                                  Control* ctl)
{
    const unsigned long long cnt = ctl->ovf_count;
    if (cnt == 0 || !bq.ovf) return;
    unsigned long long checks = 0, flips = 0;
    for (unsigned long long idx = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; idx < cnt;
         idx += (unsigned long long)gridDim.x * blockDim.x)
        overflow_item<FAST>(sc, kind, bq.ovf[idx], q, qs, qe, offset, dq, policy, band, res, key, checks, flips);
    if (checks) atomicAdd(&ctl->band_checks, checks);
    if (flips) atomicAdd(&ctl->band_flips, flips);
}

__global__ void k_finalize_edges(long long n, int policy, const unsigned* __restrict__ key,
                                 int* __restrict__ res)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        unsigned k = key[e];
        bool none = (policy == EDGE_EARLY_EXIT) ? (k == 0xffffffffu) : (k == 0u);
        res[e] = none ? 0 : (int)(k & 15u) - 1;
    }
}

__global__ void k_fk_probe(DevScene sc, const float* q, float* out)
{
    Frame<float> F[GPRM_MAX_FRAMES];
    float qi[GPRM_MAX_FRAMES];
    for (int j = 0; j < sc.ndof; ++j) qi[j] = q[j];
    forward_kinematics<PF32>(sc, qi, F);
    for (int f = 0; f <= sc.ndof; ++f)
        for (int c = 0; c < 12; ++c) out[f * 12 + c] = F[f].m[c];
}

/* ------------------------------------------------------------------ */
/* launchers                                                            */
/* ------------------------------------------------------------------ */

/* The dynamic shared-memory cap is an attribute of the kernel, shared by
 * every handle in the process: it is opened to the device's opt-in limit
 * (less the kernel's static shared memory), so that configuring one handle
 * never shrinks what another handle launches with.  Fails when `need`
 * bytes do not fit. */
static cudaError_t open_smem_cap(const void* fn, int optin, size_t need)
{
    cudaFuncAttributes fa;
    cudaError_t err = cudaFuncGetAttributes(&fa, fn);
    if (err != cudaSuccess) return err;
    const int cap = optin - (int)fa.sharedSizeBytes;
    if (cap < 0 || need > (size_t)cap) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

/* Occupancy of one FP32 kernel variant, in resident warps per SM. */
static cudaError_t variant_warps(const void* fn, int threads, size_t smem, int* warps_per_sm)
{
    int per_sm = 0;
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    *warps_per_sm = per_sm * (threads / 32);
    return err;
}

template <bool FAST>
static const void* kernel_fn_t(int vertex_kernel, bool smem, int policy, bool split)
{
    if (vertex_kernel) return smem ? (const void*)k_check_configs<true, FAST> : (const void*)k_check_configs<false, FAST>;
    if (split) {
        if (policy == EDGE_EARLY_EXIT)
            return smem ? (const void*)k_check_edges<true, EDGE_EARLY_EXIT, true, FAST>
                        : (const void*)k_check_edges<false, EDGE_EARLY_EXIT, true, FAST>;
        return smem ? (const void*)k_check_edges<true, EDGE_ALL_STEPS, true, FAST>
                    : (const void*)k_check_edges<false, EDGE_ALL_STEPS, true, FAST>;
    }
    if (policy == EDGE_EARLY_EXIT)
        return smem ? (const void*)k_check_edges<true, EDGE_EARLY_EXIT, false, FAST>
                    : (const void*)k_check_edges<false, EDGE_EARLY_EXIT, false, FAST>;
    return smem ? (const void*)k_check_edges<true, EDGE_ALL_STEPS, false, FAST>
                : (const void*)k_check_edges<false, EDGE_ALL_STEPS, false, FAST>;
}

static const void* kernel_fn(int vertex_kernel, bool smem, int policy, bool split = false, bool fast = false)
{
    return fast ? kernel_fn_t<true>(vertex_kernel, smem, policy, split)
                : kernel_fn_t<false>(vertex_kernel, smem, policy, split);
}

/* Sets a kernel's preferred shared-memory carveout (percent of the SM's
 * maximum; -1 restores the default) when it differs from the value last
 * set for it, so that every launch runs with its own handle's split of the
 * SM's L1 and shared memory. */
static cudaError_t apply_carveout(const void* fn, int pct)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> last;
    std::lock_guard<std::mutex> lock(mu);
    auto it = last.find(fn);
    const int cur = it == last.end() ? -1 : it->second;
    if (cur == pct) return cudaSuccess;
    cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (err == cudaSuccess) last[fn] = pct;
    return err;
}

cudaError_t configure_launch(const DevScene& sc, int vertex_kernel, int threads, int scene_in_smem,
                             LaunchCfg* cfg, int blocks_cap)
{
    int dev = 0, sms = 0, optin = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t smem = frame_smem_bytes(sc, threads, vertex_kernel != 0) + (scene_in_smem ? scene_smem_bytes(sc) : 0);
    for (int pol = 0; pol < (vertex_kernel ? 1 : 2); ++pol)
        for (int split = 0; split < (vertex_kernel ? 1 : 2); ++split)
            for (int fast = 0; fast < 2; ++fast) {
                err = open_smem_cap(kernel_fn(vertex_kernel, scene_in_smem != 0, pol, split != 0, fast != 0), optin,
                                    smem);
                if (err != cudaSuccess) return err;
            }
    /* occupancy of the slower-to-fit of the two arithmetic variants, with
       the default carveout */
    for (int pol = 0; pol < (vertex_kernel ? 1 : 2); ++pol)
        for (int split = 0; split < (vertex_kernel ? 1 : 2); ++split)
            for (int fast = 0; fast < 2; ++fast) {
                err = apply_carveout(kernel_fn(vertex_kernel, scene_in_smem != 0, pol, split != 0, fast != 0), -1);
                if (err != cudaSuccess) return err;
            }
    int warps = 0, warps_fast = 0;
    err = variant_warps(kernel_fn(vertex_kernel, scene_in_smem != 0, 0), threads, smem, &warps);
    if (err != cudaSuccess) return err;
    err = variant_warps(kernel_fn(vertex_kernel, scene_in_smem != 0, 0, false, true), threads, smem, &warps_fast);
    if (err != cudaSuccess) return err;
    if (warps_fast < warps) warps = warps_fast;
    if (warps < 1) return cudaErrorInvalidConfiguration;
    int per_sm = warps / (threads / 32);
    int carveout = -1;
    if (blocks_cap > 0 && blocks_cap < per_sm) {
        /* fewer resident blocks: a carveout just large enough for them (each
           block also reserves 1 KB), the rest of the SM's combined L1 and
           shared memory left to L1 */
        int smem_sm = 0;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        per_sm = blocks_cap;
        const double need = (double)per_sm * (double)(smem + 1024);
        carveout = smem_sm > 0 ? (int)ceil(100.0 * need / smem_sm) : -1;
        if (carveout > 100) carveout = 100;
    }
    cfg->threads = threads;
    cfg->smem_bytes = smem;
    cfg->scene_in_smem = scene_in_smem;
    cfg->blocks = sms * per_sm;
    cfg->blocks_per_sm = per_sm;
    cfg->warps_per_sm = per_sm * (threads / 32);
    cfg->carveout = carveout;
    return cudaSuccess;
}

cudaError_t plan_launch(const DevScene& sc, int vertex_kernel, int threads, LaunchCfg* cfg)
{
    /* default: the variant with the most resident warps, the scene in shared
       memory on ties (the autotuner times the candidates instead) */
    LaunchCfg best{};
    int best_w = -1;
    const int cand_threads[4] = {threads, 256, 384, 512};
    for (int ci = 0; ci < 4; ++ci)
        for (int sm = 1; sm >= 0; --sm) {
            LaunchCfg c{};
            if (configure_launch(sc, vertex_kernel, cand_threads[ci], sm, &c) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            if (c.warps_per_sm > best_w) { best = c; best_w = c.warps_per_sm; }
        }
    if (best_w < 0) return cudaErrorInvalidConfiguration;
    /* re-apply the chosen variant's shared-memory attribute */
    cudaError_t err = configure_launch(sc, vertex_kernel, best.threads, best.scene_in_smem, cfg);
    return err;
}

cudaError_t launch_check_configs(const DevScene& sc, const LaunchCfg& cfg, const float* q, long long n,
                                 long long offset, int* res, int band_on, float band, BandQueue bq, Control* ctl,
                                 cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    {
        cudaError_t err = apply_carveout(kernel_fn(1, cfg.scene_in_smem != 0, 0, false, sc.fast != 0), cfg.carveout);
        if (err != cudaSuccess) return err;
    }
#define GPRM_CFG_LAUNCH(SM_, FAST_)                                                                            \
    k_check_configs<SM_, FAST_><<<cfg.blocks, cfg.threads, cfg.smem_bytes, st>>>(sc, q, n, offset, res, band_on, \
                                                                                band, bq, ctl)
    if (cfg.scene_in_smem) { if (sc.fast) GPRM_CFG_LAUNCH(true, true); else GPRM_CFG_LAUNCH(true, false); }
    else { if (sc.fast) GPRM_CFG_LAUNCH(false, true); else GPRM_CFG_LAUNCH(false, false); }
#undef GPRM_CFG_LAUNCH
    return cudaGetLastError();
}

cudaError_t launch_check_edges(const DevScene& sc, const LaunchCfg& cfg, const float* qs, const float* qe,
                               long long n, long long offset, float dq, int policy, unsigned* key,
                               int band_on, float band, BandQueue bq, Control* ctl,
                               cudaStream_t st, unsigned* seg_off, int seg_rounds)
{
    if (n <= 0) return cudaSuccess;
    if (seg_off && (seg_rounds < 1 || n > EDGE_SPLIT_MAX)) return cudaErrorInvalidValue;
    if (seg_off) {
        if (n <= EDGE_SPLIT_ONE_BLOCK) {
            k_edge_segments<<<1, 1024, 0, st>>>(qs, qe, n, offset, sc.ndof, dq, seg_rounds, seg_off);
        } else {
            static_assert(EDGE_SEG_BLOCKS <= 1024, "one block scans the block sums");
            unsigned* bsum = seg_off + n + 1;   /* EDGE_SEG_BLOCKS words after the offsets */
            k_seg_pass<0><<<EDGE_SEG_BLOCKS, 256, 0, st>>>(qs, qe, n, offset, sc.ndof, dq, seg_rounds, seg_off, bsum);
            k_seg_scan_blocks<<<1, 1024, 0, st>>>(bsum, EDGE_SEG_BLOCKS, seg_off + n);
            k_seg_pass<1><<<EDGE_SEG_BLOCKS, 256, 0, st>>>(qs, qe, n, offset, sc.ndof, dq, seg_rounds, seg_off, bsum);
        }
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    size_t sm = cfg.smem_bytes;
    {
        cudaError_t err = apply_carveout(kernel_fn(0, cfg.scene_in_smem != 0, policy, seg_off != nullptr, sc.fast != 0),
                                         cfg.carveout);
        if (err != cudaSuccess) return err;
    }
#define GPRM_EDGE_LAUNCH2(SM_, POL_, SPLIT_, FAST_)                                                           \
    k_check_edges<SM_, POL_, SPLIT_, FAST_><<<cfg.blocks, cfg.threads, sm, st>>>(                                 \
        sc, qs, qe, n, offset, dq, key, band_on, band, bq, ctl, seg_off, seg_rounds)
#define GPRM_EDGE_LAUNCH(SM_, POL_, SPLIT_)                                                                   \
    do { if (sc.fast) GPRM_EDGE_LAUNCH2(SM_, POL_, SPLIT_, true); else GPRM_EDGE_LAUNCH2(SM_, POL_, SPLIT_, false); } \
    while (0)
    const bool split = seg_off != nullptr;
    if (policy == EDGE_EARLY_EXIT) {
        if (cfg.scene_in_smem) { if (split) GPRM_EDGE_LAUNCH(true, EDGE_EARLY_EXIT, true); else GPRM_EDGE_LAUNCH(true, EDGE_EARLY_EXIT, false); }
        else { if (split) GPRM_EDGE_LAUNCH(false, EDGE_EARLY_EXIT, true); else GPRM_EDGE_LAUNCH(false, EDGE_EARLY_EXIT, false); }
    } else {
        if (cfg.scene_in_smem) { if (split) GPRM_EDGE_LAUNCH(true, EDGE_ALL_STEPS, true); else GPRM_EDGE_LAUNCH(true, EDGE_ALL_STEPS, false); }
        else { if (split) GPRM_EDGE_LAUNCH(false, EDGE_ALL_STEPS, true); else GPRM_EDGE_LAUNCH(false, EDGE_ALL_STEPS, false); }
    }
#undef GPRM_EDGE_LAUNCH
#undef GPRM_EDGE_LAUNCH2
    return cudaGetLastError();
}

cudaError_t launch_recheck(const DevScene& sc, int blocks, int kind, const float* q, const float* qs,
                           const float* qe, long long offset, float dq, int policy, int* res, unsigned* key,
                           BandQueue bq, Control* ctl, cudaStream_t st)
{
    k_recheck<<<blocks, RECHECK_THREADS, 0, st>>>(sc, kind, q, qs, qe, offset, dq, policy, res, key, bq, ctl);
    return cudaGetLastError();
}

cudaError_t launch_overflow(const DevScene& sc, int blocks, int kind, const float* q, const float* qs,
                            const float* qe, long long offset, float dq, int policy, float band, int* res,
                            unsigned* key, BandQueue bq, Control* ctl, cudaStream_t st)
{
    if (!bq.ovf) return cudaSuccess;
    if (sc.fast)
        k_overflow<true><<<blocks, 128, 0, st>>>(sc, kind, q, qs, qe, offset, dq, policy, band, res, key, bq, ctl);
    else
        k_overflow<false><<<blocks, 128, 0, st>>>(sc, kind, q, qs, qe, offset, dq, policy, band, res, key, bq, ctl);
    return cudaGetLastError();
}

cudaError_t launch_finalize_edges(long long n, int policy, const unsigned* key, int* res, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    long long b = (n + 255) / 256;
    if (b > 4096) b = 4096;
    k_finalize_edges<<<(int)b, 256, 0, st>>>(n, policy, key, res);
    return cudaGetLastError();
}


/* ------------------------------------------------------------------ */
/* many problems in one launch                                          */
/* ------------------------------------------------------------------ */

/* shared bytes of one warp's cached scene descriptor */
constexpr int SCENE_CACHE_BYTES = (int)((sizeof(DevScene) + 15) / 16 * 16);

/* Problem of item `it`: the p with offs[p] <= it < offs[p+1]. */
__device__ __forceinline__ int problem_of(const BatchView& B, long long it)
{
    int lo = 0, hi = B.S;   /* offs[lo] <= it < offs[hi] */
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (B.offs[mid] <= it) lo = mid;
        else hi = mid;
    }
    return lo;
}

/* Range of work item w of the shared edge launch: the k with
 * woffs[k] <= w < woffs[k+1]. */
__device__ __forceinline__ int range_of(const BatchView& B, long long w)
{
    int lo = 0, hi = B.K;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (B.woffs[mid] <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

/* Makes problem p's descriptor the warp's current scene (warp-uniform p). */
template <bool VERTEX>
__device__ __forceinline__ void switch_scene(const BatchView& B, int p, DevScene* wsc, float* frames, SceneView& S)
{
    __syncwarp();
    const unsigned* src = reinterpret_cast<const unsigned*>(B.scenes + p);
    unsigned* dst = reinterpret_cast<unsigned*>(wsc);
    for (int k = threadIdx.x & 31; k < (int)(sizeof(DevScene) / 4); k += 32) dst[k] = src[k];
    __syncwarp();
    S.tab = wsc->tab;
    S.pairs = wsc->pairs;
    S.pairs_b = wsc->pairs_b;
    S.far = wsc->far;
    S.scan_c = wsc->scan_c;
    S.scan_b = wsc->scan_b;
    S.frames = frames;
    S.cen = frames + (size_t)wsc->ndof * 12 * 32;
    S.sweep = sweep_area<VERTEX>(*wsc, frames);
    S.defer = defer_area<VERTEX>(*wsc, frames);
}

template <bool FAST>
__global__ void GPRM_BOUNDS k_check_configs_multi(BatchView B, const float* __restrict__ q, long long offset,
                                                  int* __restrict__ res, int band_on, float band,
                                                  BandQueue bq, Control* ctl)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    DevScene* wsc = reinterpret_cast<DevScene*>(smem + warp * SCENE_CACHE_BYTES);
    float* frames = reinterpret_cast<float*>(smem + nw * SCENE_CACHE_BYTES) + (size_t)warp * B.lane_floats * 32 + lane;
    SceneView S;
    int cur = -1;
    unsigned long long exec = 0;
    PairCounts pc = {0, 0, 0};
    for (;;) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(&ctl->next, 1ull);
        c = __shfl_sync(FULL_MASK, c, 0);
        if (c >= (unsigned long long)B.nwork) break;
        const int4 ch = B.chunks[c];
        if (ch.x != cur) { switch_scene<true>(B, ch.x, wsc, frames, S); cur = ch.x; }
        check_config_chunk<FAST>(*wsc, S, q, offset, (long long)ch.y, ch.z, res, band_on, band, bq, ctl, pc,
                                 exec);
    }
    exec = warp_sum(exec);
    if (lane == 0 && exec) atomicAdd(&ctl->configs_exec, exec);
    flush_counts(pc, ctl);
}

template <int POLICY, bool FAST>
__global__ void GPRM_BOUNDS k_check_edges_multi(BatchView B, const float* __restrict__ qs, const float* __restrict__ qe,
                                                long long offset, unsigned* __restrict__ key, int band_on, float band,
                                                BandQueue bq, Control* ctl)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    DevScene* wsc = reinterpret_cast<DevScene*>(smem + warp * SCENE_CACHE_BYTES);
    float* frames = reinterpret_cast<float*>(smem + nw * SCENE_CACHE_BYTES) + (size_t)warp * B.lane_floats * 32 + lane;
    SceneView S;
    int cur = -1;
    unsigned long long exec = 0, nominal = 0;
    PairCounts pc = {0, 0, 0};
    for (;;) {
        unsigned long long eu = 0;
        if (lane == 0) eu = atomicAdd(&ctl->next, 1ull);
        eu = __shfl_sync(FULL_MASK, eu, 0);
        if (eu >= (unsigned long long)B.nwork) break;
        const int k = range_of(B, (long long)eu);
        const int p = B.wprob[k];
        const long long e = B.wbase[k] + ((long long)eu - B.woffs[k]);
        if (p != cur) { switch_scene<false>(B, p, wsc, frames, S); cur = p; }
        check_edge<POLICY, false, FAST>(*wsc, S, qs, qe, e, offset, wsc->dq, key, band_on, band, bq, ctl,
                                        pc, exec, nominal);
    }
    flush_edge_counts(exec, nominal, pc, ctl);
}

__global__ void __launch_bounds__(RECHECK_THREADS) k_recheck_multi(BatchView B, int kind,
                                                                   const float* __restrict__ q,
                                                                   const float* __restrict__ qs,
                                                                   const float* __restrict__ qe, long long offset,
                                                                   int policy, int* __restrict__ res,
                                                                   unsigned* __restrict__ key, BandQueue bq,
                                                                   Control* ctl)
{
    unsigned cnt = ctl->qcount;
    if (cnt > bq.cap) cnt = bq.cap;
    unsigned long long checks = 0, flips = 0;
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += gridDim.x * blockDim.x) {
        const uint2 it = bq.items[idx];
        const DevScene& sc = B.scenes[problem_of(B, (long long)it.x)];
        recheck_item(sc, kind, it, q, qs, qe, offset, sc.dq, policy, res, key, checks, flips,
                     bq.pair_range ? bq.pair_range[idx] : 0xffff0000u);
    }
    if (checks) atomicAdd(&ctl->band_checks, checks);
    if (flips) atomicAdd(&ctl->band_flips, flips);
}

/* The overflow pass over many problems: each item's problem by binary
 * search over the layout's offsets. */
template <bool FAST>
__global__ void __launch_bounds__(128) k_overflow_multi(BatchView B, int kind, const float* __restrict__ q,
                                                        const float* __restrict__ qs, const float* __restrict__ qe,
                                                        long long offset, int policy, float band,
                                                        int* __restrict__ res, unsigned* __restrict__ key,
                                                        BandQueue bq, Control* ctl)
{
    const unsigned long long cnt = ctl->ovf_count;
    if (cnt == 0 || !bq.ovf) return;
    unsigned long long checks = 0, flips = 0;
    for (unsigned long long idx = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; idx < cnt;
         idx += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned x = bq.ovf[idx];
        const DevScene& sc = B.scenes[problem_of(B, (long long)x)];
        overflow_item<FAST>(sc, kind, x, q, qs, qe, offset, sc.dq, policy, band, res, key, checks, flips);
    }
    if (checks) atomicAdd(&ctl->band_checks, checks);
    if (flips) atomicAdd(&ctl->band_flips, flips);
}

cudaError_t launch_overflow_multi(const BatchView& B, int blocks, int kind, const float* q, const float* qs,
                                  const float* qe, long long offset, int policy, float band, int* res, unsigned* key,
                                  BandQueue bq, Control* ctl, cudaStream_t st)
{
    if (!bq.ovf) return cudaSuccess;
    if (B.fast)
        k_overflow_multi<true><<<blocks, 128, 0, st>>>(B, kind, q, qs, qe, offset, policy, band, res, key, bq, ctl);
    else
        k_overflow_multi<false><<<blocks, 128, 0, st>>>(B, kind, q, qs, qe, offset, policy, band, res, key, bq, ctl);
    return cudaGetLastError();
}

static const void* batch_kernel_fn(int vertex_kernel, int policy, bool fast)
{
    if (vertex_kernel) return fast ? (const void*)k_check_configs_multi<true> : (const void*)k_check_configs_multi<false>;
    if (fast)
        return policy == EDGE_EARLY_EXIT ? (const void*)k_check_edges_multi<EDGE_EARLY_EXIT, true>
                                         : (const void*)k_check_edges_multi<EDGE_ALL_STEPS, true>;
    return policy == EDGE_EARLY_EXIT ? (const void*)k_check_edges_multi<EDGE_EARLY_EXIT, false>
                                     : (const void*)k_check_edges_multi<EDGE_ALL_STEPS, false>;
}

cudaError_t configure_batch_launch(const BatchView& B, int vertex_kernel, int threads, LaunchCfg* cfg,
                                   int blocks_cap)
{
    int dev = 0, sms = 0, optin = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int nw = threads / 32;
    size_t smem = (size_t)nw * SCENE_CACHE_BYTES + (size_t)nw * B.lane_floats * 32 * sizeof(float);
    for (int pol = 0; pol < (vertex_kernel ? 1 : 2); ++pol) {
        err = open_smem_cap(batch_kernel_fn(vertex_kernel, pol, B.fast != 0), optin, smem);
        if (err != cudaSuccess) return err;
    }
    int warps = 0;
    err = variant_warps(batch_kernel_fn(vertex_kernel, 0, B.fast != 0), threads, smem, &warps);
    if (err != cudaSuccess) return err;
    if (warps < 1) return cudaErrorInvalidConfiguration;
    int per_sm = warps / nw;
    int carveout = -1;
    if (blocks_cap > 0 && blocks_cap < per_sm) {
        int smem_sm = 0;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        per_sm = blocks_cap;
        const double need = (double)per_sm * (double)(smem + 1024);
        carveout = smem_sm > 0 ? (int)ceil(100.0 * need / smem_sm) : -1;
        if (carveout > 100) carveout = 100;
    }
    cfg->threads = threads;
    cfg->smem_bytes = smem;
    cfg->scene_in_smem = 0;
    cfg->blocks = sms * per_sm;
    cfg->warps_per_sm = per_sm * nw;
    cfg->blocks_per_sm = per_sm;
    cfg->carveout = carveout;
    return cudaSuccess;
}

/* Launches a persistent batch kernel with the configuration's grid and,
 * when it caps the resident blocks, its carveout as a launch attribute
 * (kept by a captured graph's kernel node). */
template <typename... KArgs, typename... Args>
static cudaError_t launch_multi(void (*kernel)(KArgs...), const LaunchCfg& cfg, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)cfg.blocks);
    lc.blockDim = dim3((unsigned)cfg.threads);
    lc.dynamicSmemBytes = cfg.smem_bytes;
    lc.stream = st;
    cudaLaunchAttribute at[1];
    if (cfg.carveout >= 0) {
        at[0].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
        at[0].val.sharedMemCarveout = (unsigned)cfg.carveout;
        lc.attrs = at;
        lc.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&lc, kernel, args...);
}

cudaError_t launch_check_configs_multi(const BatchView& B, const LaunchCfg& cfg, const float* q, long long offset,
                                       int* res, int band_on, float band, BandQueue bq, Control* ctl,
                                       cudaStream_t st)
{
    if (B.nwork <= 0) return cudaSuccess;
    if (B.fast) return launch_multi(k_check_configs_multi<true>, cfg, st, B, q, offset, res, band_on, band, bq, ctl);
    return launch_multi(k_check_configs_multi<false>, cfg, st, B, q, offset, res, band_on, band, bq, ctl);
}

cudaError_t launch_check_edges_multi(const BatchView& B, const LaunchCfg& cfg, const float* qs, const float* qe,
                                     long long offset, int policy, unsigned* key, int band_on, float band,
                                     BandQueue bq, Control* ctl, cudaStream_t st)
{
    if (B.nwork <= 0) return cudaSuccess;
    if (policy == EDGE_EARLY_EXIT)
        return B.fast ? launch_multi(k_check_edges_multi<EDGE_EARLY_EXIT, true>, cfg, st, B, qs, qe, offset, key,
                                     band_on, band, bq, ctl)
                      : launch_multi(k_check_edges_multi<EDGE_EARLY_EXIT, false>, cfg, st, B, qs, qe, offset, key,
                                     band_on, band, bq, ctl);
    return B.fast ? launch_multi(k_check_edges_multi<EDGE_ALL_STEPS, true>, cfg, st, B, qs, qe, offset, key, band_on,
                                 band, bq, ctl)
                  : launch_multi(k_check_edges_multi<EDGE_ALL_STEPS, false>, cfg, st, B, qs, qe, offset, key, band_on,
                                 band, bq, ctl);
}

cudaError_t launch_recheck_multi(const BatchView& B, int blocks, int kind, const float* q, const float* qs,
                                 const float* qe, long long offset, int policy, int* res, unsigned* key,
                                 BandQueue bq, Control* ctl, cudaStream_t st)
{
    k_recheck_multi<<<blocks, RECHECK_THREADS, 0, st>>>(B, kind, q, qs, qe, offset, policy, res, key, bq, ctl);
    return cudaGetLastError();
}

/* Adds a request's counters to the handle's running totals. */
__global__ void k_accumulate(const Control* c, Control* total)
{
    /* atomics: requests on different streams accumulate concurrently */
    atomicAdd(&total->steps_nominal, c->steps_nominal);
    atomicAdd(&total->steps_exec, c->steps_exec);
    atomicAdd(&total->band_checks, c->band_checks);
    atomicAdd(&total->band_flips, c->band_flips);
    atomicAdd(&total->configs_exec, c->configs_exec);
    atomicAdd(&total->cert_far, c->cert_far);
    atomicAdd(&total->cert_dir, c->cert_dir);
    atomicAdd(&total->full_tests, c->full_tests);
    atomicAdd(&total->ovf_count, c->ovf_count);
    atomicOr(&total->flags, c->flags);
    atomicAdd(&total->next, 1ull);  /* requests completed */
}

cudaError_t launch_accumulate(const Control* c, Control* total, cudaStream_t st)
{
    k_accumulate<<<1, 1, 0, st>>>(c, total);
    return cudaGetLastError();
}

__global__ void k_fma_probe(int iters, float* out)
{
    float x[GPRM_FMA_PROBE_CHAINS];
    const float a = 1.0000001f, b = -0.9999999f;
#pragma unroll
    for (int c = 0; c < GPRM_FMA_PROBE_CHAINS; ++c) x[c] = (float)(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < GPRM_FMA_PROBE_CHAINS; ++c) x[c] = __fmaf_rn(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < GPRM_FMA_PROBE_CHAINS; ++c) s += x[c];
    out[(blockIdx.x * blockDim.x + threadIdx.x) & (1024 * 1024 - 1)] = s;
}

cudaError_t launch_fma_probe(int blocks, int threads, int iters, float* out, cudaStream_t st)
{
    k_fma_probe<<<blocks, threads, 0, st>>>(iters, out);
    return cudaGetLastError();
}

cudaError_t launch_fk_probe(const DevScene& sc, const float* q, float* out, cudaStream_t st)
{
    k_fk_probe<<<1, 1, 0, st>>>(sc, q, out);
    return cudaGetLastError();
}

}  // namespace gprm

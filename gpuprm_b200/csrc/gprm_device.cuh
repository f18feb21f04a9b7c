/*
 * gprm_device.cuh - device-side geometry of the collision checker.
 *
 * The arithmetic restates GPUPRM's collision4/geo4/kinematics headers
 * (prm/src/lib/collision4/geo4.h, collision4.h, robotspace/kinematics.h)
 * operation for operation, so that with FMA contraction off (this library
 * is compiled with -fmad=false) and IEEE division and square root, every
 * FP32 result is bit-identical to the reference CPU build, except that the
 * sine and cosine of joint angles are the correctly rounded values (from
 * gprm_sincos64) where the reference calls glibc's sincosf.  The FP64
 * policy runs the same steps in double for the near-contact recheck.
 *
 * Scene layout in memory (global, or copied to shared memory per block):
 *   float4 tab[2N + sum(m)] one block per polytope: entry 0 is its bounding
 *                           ball (centre xyz in the body frame, radius),
 *                           entry 1 is vertex 0, then the polytope's CRS
 *                           adjacency in order, each entry holding the
 *                           NEIGHBOUR's body-frame xyz and, in w (int
 *                           bits), the neighbour's index | its degree << 7 |
 *                           its CRS offset << 15.  A support climb reads one
 *                           16-byte entry per candidate, no indirection.
 *   int4   pairs[M]         (blockA, blockB, sysA, sysB) in the reference's
 *                           pair order (CRS by `from`)
 *   float4 pairs_b[M]       (R = rA + rB, T2, slotA, slotB) for the
 *                           separation certificates (see pair_certified)
 * A polytope in frame 0 (the world) is used untransformed: the reference
 * multiplies it by trafos[0], whose entries are exactly 1 and +-0, which
 * changes at most the sign of a zero coordinate; no comparison or nonzero
 * result depends on that sign.
 */
#ifndef GPRM_DEVICE_CUH
#define GPRM_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include "gprm_sincos64.h"

#define GPRM_MAX_FRAMES 8   /* ndof + 1 */
#define GPRM_MAX_SLOTS 16   /* moving polytopes whose ball centre is tracked per lane */
/* neighbours evaluated together by the support climb (1 or 4) */
#ifndef GPRM_CLIMB_CHUNK
#define GPRM_CLIMB_CHUNK 1
#endif
#define GPRM_MAX_ITERS 10   /* max_for_loop, max_for_loop_whole (collision4.h:17-18) */

namespace gprm {

/* Scene constants and pointers passed to every kernel by value. */
struct DevScene {
    int ndof, npoly, npairs, sumn, summ;
    float a[GPRM_MAX_FRAMES], ca[GPRM_MAX_FRAMES], sa[GPRM_MAX_FRAMES];
    double ca64[GPRM_MAX_FRAMES], sa64[GPRM_MAX_FRAMES];
    float q0[GPRM_MAX_FRAMES], d0[GPRM_MAX_FRAMES];
    int types[GPRM_MAX_FRAMES];
    float mins[GPRM_MAX_FRAMES], maxs[GPRM_MAX_FRAMES];
    /* (double)dp >= -1e-6  <=>  dp >= sep_thr ; (double)n < 1e-6 <=> n < tiny_thr */
    float sep_thr, tiny_thr;
    int ntab;               /* entries of tab */
    const float4* tab;
    const int4* pairs;
    const float4* pairs_b;
    /* certificate scan per pair: far = (static partner's ball centre, T2);
       scan_c = (slot of P, slot of Q (-1: in frame 0), sqrt(T2) rounded up
       (float bits), usable by the scan); scan_b = (static partner's vertex
       0, R) */
    const float4* far;
    const int4* scan_c;
    const float4* scan_b;
    /* certificates: a pair whose guaranteed separation along the first
       search direction exceeds thr_dir is reported free without the test;
       eps_dir bounds the direction error of the approximate first direction
       times its distance (see pair_certified) */
    float thr_dir, eps_dir;
    /* box certificate: per polytope 3 records (unit axis in its frame, half
       extent about the ball centre, inflated); per pair the two polytopes */
    const float4* box;
    const int2* ppoly;
    float dq;                            /* edge resolution (batched problems) */
    int nslots;                          /* moving polytopes with a ball slot */
    int slot_sys[GPRM_MAX_SLOTS];        /* frame of each slot */
    int slot_block[GPRM_MAX_SLOTS];      /* its table block (entry 0 = ball) */
    /* fast arithmetic (GPRM_MODE_FAST): the kernels run pair_test_fast */
    int fast;
    /* every polytope's vertices as table entries (xyz, packed w), and per
       polytope (first entry, vertex count, near-tie tolerance of its support
       values (float bits), 0): the fast path's support search */
    const float4* vtab;
    const int4* vinfo;
    /* per polytope and direction bin: its support candidates as vertex
       entries (vtab's), ascending vertex index, in cslots slots (slots past
       the count repeat the last candidate), and the count */
    const float4* ctab;
    const unsigned char* ccnt;
    int cslots;
};

/* fields of a table entry's w word */
__device__ __forceinline__ int ent_idx(float4 e) { return __float_as_int(e.w) & 127; }
__device__ __forceinline__ int ent_cnt(float4 e) { return (__float_as_int(e.w) >> 7) & 255; }
__device__ __forceinline__ int ent_dsp(float4 e) { return (int)((unsigned)__float_as_int(e.w) >> 15); }

/* ---------------------------------------------------------------- */
/* precision policies                                                 */
/* ---------------------------------------------------------------- */

struct PF32 {
    typedef float R;
    static __device__ __forceinline__ float sqrt_(float x) { return __fsqrt_rn(x); }
    static __device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
    static __device__ __forceinline__ float rsqrt2(float s) { return __frcp_rn(__fsqrt_rn(s)); }
    static __device__ __forceinline__ bool separated(const DevScene& sc, float dp) { return dp >= sc.sep_thr; }
    static __device__ __forceinline__ bool tiny(const DevScene& sc, float n) { return n < sc.tiny_thr; }
    static __device__ __forceinline__ void trig(float x, float& c, float& s) {
        double sd, cd;
        gprm_sincos64((double)x, &sd, &cd);
        c = __double2float_rn(cd);
        s = __double2float_rn(sd);
    }
    static __device__ __forceinline__ void trig_alpha(const DevScene& sc, int i, float& c, float& s) {
        c = sc.ca[i];
        s = sc.sa[i];
    }
    static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
};

struct PF64 {
    typedef double R;
    static __device__ __forceinline__ double sqrt_(double x) { return __dsqrt_rn(x); }
    static __device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }
    static __device__ __forceinline__ double rsqrt2(double s) { return __drcp_rn(__dsqrt_rn(s)); }
    static __device__ __forceinline__ bool separated(const DevScene&, double dp) { return dp >= -0.000001; }
    static __device__ __forceinline__ bool tiny(const DevScene&, double n) { return n < 0.000001; }
    static __device__ __forceinline__ void trig(float x, double& c, double& s) {
        gprm_sincos64((double)x, &s, &c);
    }
    static __device__ __forceinline__ void trig_alpha(const DevScene& sc, int i, double& c, double& s) {
        c = sc.ca64[i];
        s = sc.sa64[i];
    }
    static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000LL); }
};

template <class R> struct V3 { R x, y, z; };

template <class R>
__device__ __forceinline__ R dot3(R ax, R ay, R az, R bx, R by, R bz)
{
    return ax * bx + ay * by + az * bz;
}

/* Frame storage: f[c*3 + r] = column c, row r of trafo4 (geo4.h:24). */
template <class R> struct Frame { R m[12]; };

/* trafo4::set (geo4.h:194-203) */
template <class P>
__device__ __forceinline__ void dh_frame(Frame<typename P::R>& T, typename P::R cq, typename P::R sq,
                                         typename P::R ca, typename P::R sa, typename P::R a,
                                         typename P::R d)
{
    typedef typename P::R R;
    T.m[0] = cq;      T.m[1] = sq * ca;  T.m[2] = sq * sa;
    T.m[3] = -sq;     T.m[4] = cq * ca;  T.m[5] = cq * sa;
    T.m[6] = R(0.0f); T.m[7] = -sa;      T.m[8] = ca;
    T.m[9] = a;       T.m[10] = -sa * d; T.m[11] = ca * d;
}

/* Kinematics::calculate (kinematics.h:28-37): F[0] = set(0,0,0,0),
 * F[i+1] = F[i] * set(a_i, alpha_i, theta_i, d_i) (lapply, geo4.h:272-279). */
template <class P>
__device__ __forceinline__ void forward_kinematics(const DevScene& sc, const float* q,
                                                   Frame<typename P::R>* F)
{
    typedef typename P::R R;
    {
        R c0, s0;
        P::trig(0.0f, c0, s0);
        dh_frame<P>(F[0], c0, s0, c0, s0, R(0.0f), R(0.0f));
    }
#pragma unroll 1
    for (int i = 0; i < sc.ndof; ++i) {
        float th = sc.q0[i], d = sc.d0[i];
        if (sc.types[i] == 0) th = q[i];
        else d = q[i];
        R cq, sq, ca, sa;
        P::trig(th, cq, sq);
        P::trig_alpha(sc, i, ca, sa);
        Frame<R> L;
        dh_frame<P>(L, cq, sq, ca, sa, (R)sc.a[i], (R)d);
        const Frame<R>& T = F[i];
        Frame<R>& O = F[i + 1];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            R ux = L.m[3 * c], uy = L.m[3 * c + 1], uz = L.m[3 * c + 2];
            R ox = T.m[0] * ux + T.m[3] * uy + T.m[6] * uz;
            R oy = T.m[1] * ux + T.m[4] * uy + T.m[7] * uz;
            R oz = T.m[2] * ux + T.m[5] * uy + T.m[8] * uz;
            if (c == 3) { ox = ox + T.m[9]; oy = oy + T.m[10]; oz = oz + T.m[11]; }
            O.m[3 * c] = ox; O.m[3 * c + 1] = oy; O.m[3 * c + 2] = oz;
        }
    }
}

/* The same chain for the FP32 kernels, storing frames 1..ndof to a
 * lane-interleaved shared-memory array: entry e of frame f at
 * out[((f-1)*12 + e) * 32] (out already offset by the lane).  The world
 * centre of every slot's bounding ball follows at
 * cen[(slot*3 + c) * 32], then the world position of the slot polytope's
 * vertex 0 at cen[((nslots + slot)*3 + c) * 32] (both with FMA: they only
 * feed the certificates, whose slack covers their rounding). */
__device__ __forceinline__ void slot_points(const DevScene& sc, const float4* __restrict__ tab, const Frame<float>& O,
                                            int slot, float* cen)
{
    const float4 b = tab[sc.slot_block[slot]];
    cen[(slot * 3 + 0) * 32] = __fmaf_rn(O.m[0], b.x, __fmaf_rn(O.m[3], b.y, __fmaf_rn(O.m[6], b.z, O.m[9])));
    cen[(slot * 3 + 1) * 32] = __fmaf_rn(O.m[1], b.x, __fmaf_rn(O.m[4], b.y, __fmaf_rn(O.m[7], b.z, O.m[10])));
    cen[(slot * 3 + 2) * 32] = __fmaf_rn(O.m[2], b.x, __fmaf_rn(O.m[5], b.y, __fmaf_rn(O.m[8], b.z, O.m[11])));
    const float4 v = tab[sc.slot_block[slot] + 1];
    float* w = cen + sc.nslots * 3 * 32;
    w[(slot * 3 + 0) * 32] = __fmaf_rn(O.m[0], v.x, __fmaf_rn(O.m[3], v.y, __fmaf_rn(O.m[6], v.z, O.m[9])));
    w[(slot * 3 + 1) * 32] = __fmaf_rn(O.m[1], v.x, __fmaf_rn(O.m[4], v.y, __fmaf_rn(O.m[7], v.z, O.m[10])));
    w[(slot * 3 + 2) * 32] = __fmaf_rn(O.m[2], v.x, __fmaf_rn(O.m[5], v.y, __fmaf_rn(O.m[8], v.z, O.m[11])));
}

__device__ __forceinline__ void forward_kinematics_smem(const DevScene& sc, const float4* __restrict__ tab,
                                                        const float* q, float* out, float* cen)
{
    Frame<float> T;
    {
        float c0, s0;
        PF32::trig(0.0f, c0, s0);
        dh_frame<PF32>(T, c0, s0, c0, s0, 0.0f, 0.0f);
    }
    int slot = 0;
#pragma unroll 1
    for (int i = 0; i < sc.ndof; ++i) {
        float th = sc.q0[i], d = sc.d0[i];
        if (sc.types[i] == 0) th = q[i];
        else d = q[i];
        float cq, sq, ca, sa;
        PF32::trig(th, cq, sq);
        PF32::trig_alpha(sc, i, ca, sa);
        Frame<float> L;
        dh_frame<PF32>(L, cq, sq, ca, sa, sc.a[i], d);
        Frame<float> O;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float ux = L.m[3 * c], uy = L.m[3 * c + 1], uz = L.m[3 * c + 2];
            float ox = T.m[0] * ux + T.m[3] * uy + T.m[6] * uz;
            float oy = T.m[1] * ux + T.m[4] * uy + T.m[7] * uz;
            float oz = T.m[2] * ux + T.m[5] * uy + T.m[8] * uz;
            if (c == 3) { ox = ox + T.m[9]; oy = oy + T.m[10]; oz = oz + T.m[11]; }
            O.m[3 * c] = ox; O.m[3 * c + 1] = oy; O.m[3 * c + 2] = oz;
        }
#pragma unroll
        for (int e = 0; e < 12; ++e) out[(i * 12 + e) * 32] = O.m[e];
        for (; slot < sc.nslots && sc.slot_sys[slot] == i + 1; ++slot) slot_points(sc, tab, O, slot, cen);
        T = O;
    }
}

/* Loads frame f (1..ndof) of the lane from the array written above. */
__device__ __forceinline__ void load_frame(const float* fr, int f, Frame<float>& T)
{
#pragma unroll
    for (int e = 0; e < 12; ++e) T.m[e] = fr[((f - 1) * 12 + e) * 32];
}

/* T*v (geo4.h:215-221) */
template <class R>
__device__ __forceinline__ V3<R> xform(const Frame<R>& T, R x, R y, R z)
{
    V3<R> o;
    o.x = T.m[0] * x + T.m[3] * y + T.m[6] * z + T.m[9];
    o.y = T.m[1] * x + T.m[4] * y + T.m[7] * z + T.m[10];
    o.z = T.m[2] * x + T.m[5] * y + T.m[8] * z + T.m[11];
    return o;
}

/* R'*v (geo4.h:249-255) */
template <class R>
__device__ __forceinline__ V3<R> rot_t(const Frame<R>& T, R x, R y, R z)
{
    V3<R> o;
    o.x = T.m[0] * x + T.m[1] * y + T.m[2] * z;
    o.y = T.m[3] * x + T.m[4] * y + T.m[5] * z;
    o.z = T.m[6] * x + T.m[7] * y + T.m[8] * z;
    return o;
}

/* geo4::normalize(float4&) (geo4.h:165-171) */
template <class P>
__device__ __forceinline__ typename P::R normalize3(V3<typename P::R>& u)
{
    typedef typename P::R R;
    R norm = P::sqrt_(u.x * u.x + u.y * u.y + u.z * u.z);
    R f = P::recip(norm);
    if (f == P::inf()) f = R(0.0f);
    u.x = u.x * f; u.y = u.y * f; u.z = u.z * f;
    return norm;
}

/* support_vertex_searcher::search_support_vertex (collision4.h:66-103):
 * first-improvement climb over the vertex adjacency, starting at `cur`
 * (an entry of the polytope's block B).  The neighbours of the current
 * vertex are evaluated four at a time (independent loads and dot
 * products); the move goes to the first of them, in CRS order, whose dot
 * product exceeds the current maximum, which is the vertex the reference's
 * one-at-a-time scan moves to.  The maximum rises strictly, so there are at
 * most n-1 moves; the loop bound only guards corrupt data. */
template <class P>
__device__ __forceinline__ float4 climb(const float4* __restrict__ B, float4 cur, typename P::R dx,
                                        typename P::R dy, typename P::R dz)
{
    typedef typename P::R R;
    R best = dot3<R>((R)cur.x, (R)cur.y, (R)cur.z, dx, dy, dz);
#pragma unroll 1
    for (int guard = 0; guard < 128; ++guard) {
        const float4* e = B + 2 + ent_dsp(cur);
        const int c = ent_cnt(cur);
        bool moved = false;
#if GPRM_CLIMB_CHUNK == 4
#pragma unroll 1
        for (int i = 0; i < c && !moved; i += 4) {
            const int left = c - i;
            float4 u0 = e[i], u1 = u0, u2 = u0, u3 = u0;
            if (left > 1) u1 = e[i + 1];
            if (left > 2) u2 = e[i + 2];
            if (left > 3) u3 = e[i + 3];
            R d0 = dot3<R>((R)u0.x, (R)u0.y, (R)u0.z, dx, dy, dz);
            R d1 = dot3<R>((R)u1.x, (R)u1.y, (R)u1.z, dx, dy, dz);
            R d2 = dot3<R>((R)u2.x, (R)u2.y, (R)u2.z, dx, dy, dz);
            R d3 = dot3<R>((R)u3.x, (R)u3.y, (R)u3.z, dx, dy, dz);
            if (d0 > best) { best = d0; cur = u0; moved = true; }
            else if (left > 1 && d1 > best) { best = d1; cur = u1; moved = true; }
            else if (left > 2 && d2 > best) { best = d2; cur = u2; moved = true; }
            else if (left > 3 && d3 > best) { best = d3; cur = u3; moved = true; }
        }
#else
#pragma unroll 1
        for (int i = 0; i < c; ++i) {
            float4 u = e[i];
            R d = dot3<R>((R)u.x, (R)u.y, (R)u.z, dx, dy, dz);
            if (d > best) { best = d; cur = u; moved = true; break; }
        }
#endif
        if (!moved) break;
    }
    return cur;
}

template <class R> struct V2 { R x, y; };

template <class P>
__device__ __forceinline__ void normalize2(V2<typename P::R>& u)
{
    typename P::R f = P::rsqrt2(u.x * u.x + u.y * u.y);
    u.x = u.x * f; u.y = u.y * f;
}

template <class R>
__device__ __forceinline__ R cross2(const V2<R>& v, const V2<R>& w) { return v.x * w.y - v.y * w.x; }

/* find_half_plane (collision4.h:136-223) with orthtrafo23 (:111-134).
 * hist holds R[0..k-1] (x,y,z per entry). */
template <class P>
__device__ __forceinline__ bool half_plane(const V3<typename P::R>* hist, int k, V3<typename P::R>& w,
                                           const V3<typename P::R>& rk)
{
    typedef typename P::R R;
    if (dot3<R>(w.x, w.y, w.z, rk.x, rk.y, rk.z) > R(0.0f)) return true;
    R x = rk.x, y = rk.y, z = rk.z;
    R d = P::sqrt_(x * x + y * y);
    R m0 = x * z / d, m1 = y * z / d, m2 = -d;
    R m3 = -y / d, m4 = x / d, m5 = R(0.0f);
    V2<R> ra, rb, t;
    ra.x = m0 * hist[0].x + m1 * hist[0].y + m2 * hist[0].z;
    ra.y = m3 * hist[0].x + m4 * hist[0].y + m5 * hist[0].z;
    rb.x = m0 * hist[1].x + m1 * hist[1].y + m2 * hist[1].z;
    rb.y = m3 * hist[1].x + m4 * hist[1].y + m5 * hist[1].z;
    if (cross2<R>(ra, rb) < R(0.0f)) { V2<R> tmp = ra; ra = rb; rb = tmp; }
#pragma unroll 1
    for (int i = 2; i < k; ++i) {
        t.x = m0 * hist[i].x + m1 * hist[i].y + m2 * hist[i].z;
        t.y = m3 * hist[i].x + m4 * hist[i].y + m5 * hist[i].z;
        R cb = cross2<R>(rb, t);
        if (cross2<R>(ra, t) > R(0.0f)) {
            if (cb > R(0.0f)) rb = t;
        } else {
            if (cb < R(0.0f)) ra = t;
            else return false;
        }
    }
    normalize2<P>(ra);
    normalize2<P>(rb);
    t.x = ra.x + rb.x;
    t.y = ra.y + rb.y;
    normalize2<P>(t);
    w.x = m0 * t.x + m3 * t.y;
    w.y = m1 * t.x + m4 * t.y;
    w.z = m2 * t.x + m5 * t.y;
    return true;
}

/* seperating_vector_algorithm (collision4.h:226-332) for pair `pr`, with
 * frames tp, tq (ignored for a polytope in frame 0).
 * Returns 0 (separated), l+1 (no separating half plane) or -1 (cap).
 * *margin: h = dp*|q0-p0| at the deciding iteration if separated, else the
 * largest h seen. */
template <class P>
__device__ __forceinline__ int pair_test(const DevScene& sc, const float4* __restrict__ tab, int4 pr,
                                         const Frame<typename P::R>& tp, const Frame<typename P::R>& tq,
                                         typename P::R* margin)
{
    typedef typename P::R R;
    const float4* BP = tab + pr.x;
    const float4* BQ = tab + pr.y;
    const bool idP = pr.z == 0, idQ = pr.w == 0;
    float4 ep = BP[1], eq = BQ[1];
    V3<R> Sa, Sb;
    if (idQ) { Sa.x = (R)eq.x; Sa.y = (R)eq.y; Sa.z = (R)eq.z; }
    else Sa = xform<R>(tq, (R)eq.x, (R)eq.y, (R)eq.z);
    if (idP) { Sb.x = (R)ep.x; Sb.y = (R)ep.y; Sb.z = (R)ep.z; }
    else Sb = xform<R>(tp, (R)ep.x, (R)ep.y, (R)ep.z);
    V3<R> S;
    S.x = Sa.x - Sb.x; S.y = Sa.y - Sb.y; S.z = Sa.z - Sb.z;
    R norm = normalize3<P>(S);
    if (P::tiny(sc, norm)) S.x = R(1.0f);
    V3<R> w; w.x = w.y = w.z = R(0.0f);
    V3<R> hist[GPRM_MAX_ITERS];
    int combs[GPRM_MAX_ITERS];
    R best = R(0.0f);
    int k = 0, l = 0;
#pragma unroll 1
    for (; k < GPRM_MAX_ITERS && l < GPRM_MAX_ITERS; ++l) {
        V3<R> Sp, Sq;
        if (idP) Sp = S;
        else Sp = rot_t<R>(tp, S.x, S.y, S.z);
        if (idQ) { Sq.x = -S.x; Sq.y = -S.y; Sq.z = -S.z; }
        else Sq = rot_t<R>(tq, -S.x, -S.y, -S.z);
        ep = climb<P>(BP, ep, Sp.x, Sp.y, Sp.z);
        eq = climb<P>(BQ, eq, Sq.x, Sq.y, Sq.z);
        V3<R> p0, q0;
        if (idP) { p0.x = (R)ep.x; p0.y = (R)ep.y; p0.z = (R)ep.z; }
        else p0 = xform<R>(tp, (R)ep.x, (R)ep.y, (R)ep.z);
        if (idQ) { q0.x = (R)eq.x; q0.y = (R)eq.y; q0.z = (R)eq.z; }
        else q0 = xform<R>(tq, (R)eq.x, (R)eq.y, (R)eq.z);
        V3<R> r;
        r.x = q0.x - p0.x; r.y = q0.y - p0.y; r.z = q0.z - p0.z;
        R rn = normalize3<P>(r);
        R dp = dot3<R>(S.x, S.y, S.z, r.x, r.y, r.z);
        R h = dp * rn;
        if (l == 0 || h > best) best = h;
        if (P::separated(sc, dp)) {
            *margin = h;
            return 0;
        }
        hist[k] = r;
        int comb = ent_idx(ep) | (ent_idx(eq) << 8);
        combs[k] = comb;
        bool rep = false;
#pragma unroll 1
        for (int j = 0; j < k; ++j)
            if (combs[j] == comb) { rep = true; break; }
        if (rep) {
            S = w;
        } else {
            if (k == 1) {
                w.x = hist[0].x + r.x; w.y = hist[0].y + r.y; w.z = hist[0].z + r.z;
                normalize3<P>(w);
            }
            if (k >= 2 && !half_plane<P>(hist, k, w, r)) {
                *margin = best;
                return l + 1;
            }
            R b = R(-2.0f) * dp;
            S.x = S.x + b * r.x; S.y = S.y + b * r.y; S.z = S.z + b * r.z;
            ++k;
        }
    }
    *margin = best;
    return -1;
}

/* Separation certificate for pair `pr` (FP32 kernels).
 *
 * Balls: every world vertex the reference computes for polytope X lies in
 * the ball (c_X, r_X) (radii are inflated on the host by the rounding of
 * the reference's transforms and of the centre computed here).  For ANY
 * vertices p*, q* the first Chung-Wang iteration may reach,
 *     <S0, q0 - p0> >= G := <S0, c_Q - c_P> - (r_P + r_Q)
 * with S0 the algorithm's unit first direction.  If G > band + slack, the
 * reference's first iteration has dp > 0 >= -1e-6 (returns 0) and its
 * margin h = dp*|q0-p0| exceeds the band, so the pair contributes code 0
 * and no band-relevant margin: it can be skipped with identical output.
 *   far test   without S0: S0 = (D + e)/|D + e| with |e| <= R (e = the
 *              vertex-0 offsets from the centres) gives
 *              <S0, D> >= (|D|^2 - R|D|)/(|D| + R); pairs_b.y holds the
 *              squared distance T2 beyond which that bound passes.
 *   direction  S0 from vertex 0 of each polytope (FMA, rsqrt); its error
 *              against the reference's S0 is at most eps_dir/|s| (s the
 *              vertex-0 offset), charged against G with |D| + R.
 * NaN never passes (every test is a '>' comparison). */
/* Support of polytope box B (3 records) along u, u in world coordinates;
 * frame f (0: world) rotates the box: its local direction is R^T u. */
__device__ __forceinline__ float box_support(const float4* __restrict__ B, const float* frames, int f, float ux,
                                             float uy, float uz)
{
    float lx = ux, ly = uy, lz = uz;
    if (f) {
        const float* fr = frames + (f - 1) * 12 * 32;
        const float m0 = fr[0], m1 = fr[32], m2 = fr[64], m3 = fr[96], m4 = fr[128], m5 = fr[160];
        const float m6 = fr[192], m7 = fr[224], m8 = fr[256];
        lx = __fmaf_rn(m0, ux, __fmaf_rn(m1, uy, m2 * uz));
        ly = __fmaf_rn(m3, ux, __fmaf_rn(m4, uy, m5 * uz));
        lz = __fmaf_rn(m6, ux, __fmaf_rn(m7, uy, m8 * uz));
    }
    float h = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float4 b = B[a];
        h = __fmaf_rn(b.w, fabsf(__fmaf_rn(b.x, lx, __fmaf_rn(b.y, ly, b.z * lz))), h);
    }
    return h;
}

/* The direction and box tests of pair_certified, for a pair whose distance
 * test failed: D = c_Q - c_P and d2 = |D|^2 as that test computed them.
 * The world vertex 0 of a moving polytope comes from its slot (written by
 * the FK pass with the FMA chain T*v0; cen points at the slot ball
 * centres, the vertex-0 points follow them), that of a static polytope is
 * its body-frame vertex 0.  A moving polytope without a slot has R = T2 =
 * infinity: nothing can be certified. */
__device__ __forceinline__ bool pair_certified_dir(const DevScene& sc, const float4* __restrict__ tab, int4 pr,
                                                   float4 pb, const float* cen, const float* frames, int j,
                                                   float dx, float dy, float dz, float d2, bool box_only = false)
{
    if (!(pb.x < PF32::inf())) return false;
    const int sa = __float_as_int(pb.z), sb = __float_as_int(pb.w);
    const float* v0w = cen + sc.nslots * 3 * 32;
    float ax, ay, az, bx, by, bz;
    if (sa >= 0) { ax = v0w[(sa * 3) * 32]; ay = v0w[(sa * 3 + 1) * 32]; az = v0w[(sa * 3 + 2) * 32]; }
    else { const float4 v = tab[pr.x + 1]; ax = v.x; ay = v.y; az = v.z; }
    if (sb >= 0) { bx = v0w[(sb * 3) * 32]; by = v0w[(sb * 3 + 1) * 32]; bz = v0w[(sb * 3 + 2) * 32]; }
    else { const float4 v = tab[pr.y + 1]; bx = v.x; by = v.y; bz = v.z; }
    const float sx = bx - ax, sy = by - ay, sz = bz - az;
    const float n2 = __fmaf_rn(sx, sx, __fmaf_rn(sy, sy, sz * sz));
    if (!(n2 > 1e-6f)) return false;           /* |s| < 1e-3: leave it to the test */
    const float inv = rsqrtf(n2);
    const float G = __fmaf_rn(sx, dx, __fmaf_rn(sy, dy, sz * dz)) * inv - pb.x;
    /* |D| from above (d2 * rsqrt(d2) is within 3 ulp of it) */
    const float dn = d2 * rsqrtf(d2) * (1.0f + 2e-6f);
    /* direction error <= eps_dir*inv (+ rsqrt and rounding, 1e-6) */
    const float err = (dn + pb.x) * __fmaf_rn(sc.eps_dir, inv, 1e-6f);
    if (!box_only && G - err > sc.thr_dir) return true;
    /* box test: the same bound with each polytope's support along S taken
       from its bounding box instead of its ball (every vertex v of X has
       <S, v - c_X> <= sum_a e_a |<a_a, R_X^T S>|), tighter for elongated
       links and flat obstacles */
    if (!sc.box || !(pb.x < PF32::inf())) return false;
    const int2 pp = sc.ppoly[j];
    const float ux = sx * inv, uy = sy * inv, uz = sz * inv;
    const float hp = box_support(sc.box + 3 * pp.x, frames, pr.z, ux, uy, uz);
    const float hq = box_support(sc.box + 3 * pp.y, frames, pr.w, ux, uy, uz);
    const float Gb = __fmaf_rn(ux, dx, __fmaf_rn(uy, dy, uz * dz)) - (hp + hq) * (1.0f + 1e-5f);
    return Gb - err > sc.thr_dir;
}

__device__ __forceinline__ bool pair_certified(const DevScene& sc, const float4* __restrict__ tab,
                                               int4 pr, float4 pb, const float* cen,
                                               const float* frames, bool* used_dir, int j)
{
    *used_dir = false;
    const int sa = __float_as_int(pb.z), sb = __float_as_int(pb.w);
    float px, py, pz, qx, qy, qz;
    if (sa >= 0) { px = cen[(sa * 3) * 32]; py = cen[(sa * 3 + 1) * 32]; pz = cen[(sa * 3 + 2) * 32]; }
    else { float4 b = tab[pr.x]; px = b.x; py = b.y; pz = b.z; }
    if (sb >= 0) { qx = cen[(sb * 3) * 32]; qy = cen[(sb * 3 + 1) * 32]; qz = cen[(sb * 3 + 2) * 32]; }
    else { float4 b = tab[pr.y]; qx = b.x; qy = b.y; qz = b.z; }
    const float dx = qx - px, dy = qy - py, dz = qz - pz;
    const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, dz * dz));
    if (d2 > pb.y) return true;
    /* direction test: approximate first direction from vertex 0 of each */
    *used_dir = true;
    return pair_certified_dir(sc, tab, pr, pb, cen, frames, j, dx, dy, dz, d2);
}

/* The same certificate for the FP64 recheck, in double from the FP64
 * frames: the balls bound the FP64 world vertices as well (their inflation
 * covers float rounding, which exceeds double rounding), and the first
 * direction is computed in double, so its error term only needs the
 * 1e-6 relative allowance. */
/* box_support with the FP64 frames of check_config64 */
__device__ __forceinline__ double box_support64(const float4* __restrict__ B, const Frame<double>* F, int f, double ux,
                                                double uy, double uz)
{
    double lx = ux, ly = uy, lz = uz;
    if (f) {
        const Frame<double>& T = F[f];
        lx = T.m[0] * ux + T.m[1] * uy + T.m[2] * uz;
        ly = T.m[3] * ux + T.m[4] * uy + T.m[5] * uz;
        lz = T.m[6] * ux + T.m[7] * uy + T.m[8] * uz;
    }
    double h = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float4 b = B[a];
        h += (double)b.w * fabs((double)b.x * lx + (double)b.y * ly + (double)b.z * lz);
    }
    return h;
}

__device__ __forceinline__ bool pair_certified64(const DevScene& sc, const float4* __restrict__ tab, int4 pr,
                                                 float4 pb, const Frame<double>* F, const double* cen, int j)
{
    /* ball centres: a moving polytope's from its slot (the FP64 transform of
       its ball centre, computed once per check), a static one's from the
       table.  A moving polytope without a slot has T2 = R = infinity, so
       neither test can pass for its pairs whatever centre is used. */
    const int sa = __float_as_int(pb.z), sb = __float_as_int(pb.w);
    double px, py, pz, qx, qy, qz;
    if (sa >= 0) { px = cen[3 * sa]; py = cen[3 * sa + 1]; pz = cen[3 * sa + 2]; }
    else { const float4 bp = tab[pr.x]; px = bp.x; py = bp.y; pz = bp.z; }
    if (sb >= 0) { qx = cen[3 * sb]; qy = cen[3 * sb + 1]; qz = cen[3 * sb + 2]; }
    else { const float4 bq = tab[pr.y]; qx = bq.x; qy = bq.y; qz = bq.z; }
    const double dx = qx - px, dy = qy - py, dz = qz - pz;
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > (double)pb.y) return true;
    const float4 vp = tab[pr.x + 1], vq = tab[pr.y + 1];
    V3<double> a, b;
    if (pr.z) a = xform<double>(F[pr.z], (double)vp.x, (double)vp.y, (double)vp.z);
    else { a.x = vp.x; a.y = vp.y; a.z = vp.z; }
    if (pr.w) b = xform<double>(F[pr.w], (double)vq.x, (double)vq.y, (double)vq.z);
    else { b.x = vq.x; b.y = vq.y; b.z = vq.z; }
    const double sx = b.x - a.x, sy = b.y - a.y, sz = b.z - a.z;
    const double n2 = sx * sx + sy * sy + sz * sz;
    if (!(n2 > 1e-6)) return false;
    const double inv = 1.0 / sqrt(n2);
    const double G = (sx * dx + sy * dy + sz * dz) * inv - (double)pb.x;
    const double err = (sqrt(d2) + (double)pb.x) * 1e-6;
    if (G - err > (double)sc.thr_dir) return true;
    /* the box test of pair_certified_dir: each polytope's support along the
       first direction bounded by its box about the ball centre (the box
       records are inflated for float rounding, which covers FP64 vertices
       too); a moving polytope without a slot has no usable centre */
    if (!sc.box || !((double)pb.x < 1e300)) return false;
    const int2 pp = sc.ppoly[j];
    const double ux = sx * inv, uy = sy * inv, uz = sz * inv;
    const double hp = box_support64(sc.box + 3 * pp.x, F, pr.z, ux, uy, uz);
    const double hq = box_support64(sc.box + 3 * pp.y, F, pr.w, ux, uy, uz);
    const double Gb = (ux * dx + uy * dy + uz * dz) - (hp + hq) * (1.0 + 1e-5);
    return Gb - err > (double)sc.thr_dir;
}

/* ---------------------------------------------------------------- */
/* fast FP32 arithmetic (GPRM_MODE_FAST)                             */
/* ---------------------------------------------------------------- */
/*
 * The separating-vector algorithm of collision4.h:226-332 with the same
 * steps, decisions and thresholds as pair_test, in contracted arithmetic:
 *   - dot products and transforms as fused multiply-add chains;
 *   - normalisation by the reciprocal square root of the MUFU unit
 *     (rsqrtf, <= 2 ulp) instead of IEEE sqrt and division, and the
 *     half-plane basis (orthtrafo23) by one reciprocal square root instead
 *     of four divisions;
 *   - support vertices by a maximum over the few candidates of the
 *     direction's bin (fsupport_cand2) instead of the first-improvement
 *     climb from the previous support; the climb ends at a maximiser of the
 *     dot product too (on a convex polytope every vertex without an
 *     improving neighbour is one), so the two agree unless several vertices
 *     tie within rounding.
 * Results differ from the reference's FP32 arithmetic by rounding: codes
 * (iteration counts) may differ, free/not-free verdicts agree wherever the
 * separation margin lies outside the FP64 band, which is what the band
 * exists for.  The exact policy (PF32) stays the drop-in default.
 */
#ifndef GPRM_BIN_CELLS
#define GPRM_BIN_CELLS 3     /* cells per axis of a cube face */
#endif
#define GPRM_START_BINS (6 * GPRM_BIN_CELLS * GPRM_BIN_CELLS)   /* direction bins: 6 faces x cells */

/* Cube-map bin of a direction: the face of the largest |component| (with
 * its sign), then each of the other two components against the cell
 * borders m (-1 + 2k / GPRM_BIN_CELLS), m the largest |component|.
 * Any input, NaN included, gives a bin in [0, GPRM_START_BINS). */
__host__ __device__ __forceinline__ int dir_bin(float x, float y, float z)
{
    const float ax = fabsf(x), ay = fabsf(y), az = fabsf(z);
    int face;
    float m, u, v;
    if (ax >= ay && ax >= az) { face = x < 0.0f ? 1 : 0; m = ax; u = y; v = z; }
    else if (ay >= az) { face = y < 0.0f ? 3 : 2; m = ay; u = z; v = x; }
    else { face = z < 0.0f ? 5 : 4; m = az; u = x; v = y; }
    int iu = 0, iv = 0;
#pragma unroll
    for (int k = 1; k < GPRM_BIN_CELLS; ++k) {
        const float t = m * (-1.0f + 2.0f * (float)k / (float)GPRM_BIN_CELLS);
        iu += u > t;
        iv += v > t;
    }
    return (face * GPRM_BIN_CELLS + iu) * GPRM_BIN_CELLS + iv;
}

__device__ __forceinline__ float fdot3(float ax, float ay, float az, float bx, float by, float bz)
{
    return __fmaf_rn(ax, bx, __fmaf_rn(ay, by, az * bz));
}

__device__ __forceinline__ V3<float> fxform(const Frame<float>& T, float x, float y, float z)
{
    V3<float> o;
    o.x = __fmaf_rn(T.m[0], x, __fmaf_rn(T.m[3], y, __fmaf_rn(T.m[6], z, T.m[9])));
    o.y = __fmaf_rn(T.m[1], x, __fmaf_rn(T.m[4], y, __fmaf_rn(T.m[7], z, T.m[10])));
    o.z = __fmaf_rn(T.m[2], x, __fmaf_rn(T.m[5], y, __fmaf_rn(T.m[8], z, T.m[11])));
    return o;
}

__device__ __forceinline__ V3<float> frot_t(const Frame<float>& T, float x, float y, float z)
{
    V3<float> o;
    o.x = fdot3(T.m[0], T.m[1], T.m[2], x, y, z);
    o.y = fdot3(T.m[3], T.m[4], T.m[5], x, y, z);
    o.z = fdot3(T.m[6], T.m[7], T.m[8], x, y, z);
    return o;
}

/* normalize (geo4.h:165-171): a zero vector stays zero; returns the norm */
__device__ __forceinline__ float fnormalize3(V3<float>& u)
{
    const float n2 = fdot3(u.x, u.y, u.z, u.x, u.y, u.z);
    const float f = n2 > 0.0f ? rsqrtf(n2) : 0.0f;
    u.x *= f; u.y *= f; u.z *= f;
    return n2 * f;
}

/* Support vertices of polytopes kP (along p) and kQ (along q) from the
 * candidate lists of the directions' bins: every vertex whose normal cone
 * (the directions for which it is a maximiser) meets the bin, found on the
 * host for bins slightly larger than dir_bin's, so the maximum over the
 * list is the maximum over the whole polytope, up to ties within rounding.
 * A few candidates instead of every vertex; P and Q side by side.
 * Returns true when the runner-up of either list comes within tieP / tieQ
 * of its maximum: the reference's climb, in its own rounding, may then end
 * at a different vertex. */
__device__ __forceinline__ bool fsupport_cand2(const DevScene& sc, int kP, int4 vP, float4& cp, float px, float py,
                                               float pz, int kQ, int4 vQ, float4& cq, float qx, float qy, float qz)
{
    const float tieP = __int_as_float(vP.z), tieQ = __int_as_float(vQ.z);
    /* the bin's slots and count are found from the bin alone: the count
       and the first candidate load side by side */
    const int bP = kP * GPRM_START_BINS + dir_bin(px, py, pz);
    const int bQ = kQ * GPRM_START_BINS + dir_bin(qx, qy, qz);
    const float4* CP = sc.ctab + (size_t)bP * sc.cslots;
    const float4* CQ = sc.ctab + (size_t)bQ * sc.cslots;
    const int nP = sc.ccnt[bP], nQ = sc.ccnt[bQ];
    int ip = 0, iq = 0;
    float4 u = CP[0], v = CQ[0];
    float bp = fdot3(u.x, u.y, u.z, px, py, pz), bq = fdot3(v.x, v.y, v.z, qx, qy, qz);
    const float ninf = __int_as_float(0xff800000);
    float sp = ninf, sq = ninf;   /* runners-up */
    const int n = nP > nQ ? nP : nQ;
    /* branch-free top two; past its count a list's slots repeat its last
       candidate, counted as -infinity */
#pragma unroll 1
    for (int c = 1; c < n; ++c) {
        u = CP[c];
        v = CQ[c];
        float du = fdot3(u.x, u.y, u.z, px, py, pz), dv = fdot3(v.x, v.y, v.z, qx, qy, qz);
        du = c < nP ? du : ninf;
        dv = c < nQ ? dv : ninf;
        ip = du > bp ? c : ip;
        iq = dv > bq ? c : iq;
        sp = fmaxf(sp, fminf(bp, du));
        sq = fmaxf(sq, fminf(bq, dv));
        bp = fmaxf(bp, du);
        bq = fmaxf(bq, dv);
    }
    cp = CP[ip];
    cq = CQ[iq];
    return !(bp - sp > tieP) || !(bq - sq > tieQ);
}

/* find_half_plane with orthtrafo23 (collision4.h:111-223), contracted */
__device__ __forceinline__ bool fhalf_plane(const V3<float>* hist, int k, V3<float>& w, const V3<float>& rk)
{
    if (fdot3(w.x, w.y, w.z, rk.x, rk.y, rk.z) > 0.0f) return true;
    const float x = rk.x, y = rk.y, z = rk.z;
    const float inv = rsqrtf(__fmaf_rn(x, x, y * y));   /* 1/d, d = |(x, y)| */
    const float m0 = x * z * inv, m1 = y * z * inv, m2 = -__fmaf_rn(x, x, y * y) * inv;
    const float m3 = -y * inv, m4 = x * inv;
    V2<float> ra, rb, t;
    ra.x = fdot3(m0, m1, m2, hist[0].x, hist[0].y, hist[0].z);
    ra.y = __fmaf_rn(m3, hist[0].x, m4 * hist[0].y);
    rb.x = fdot3(m0, m1, m2, hist[1].x, hist[1].y, hist[1].z);
    rb.y = __fmaf_rn(m3, hist[1].x, m4 * hist[1].y);
    if (__fmaf_rn(ra.x, rb.y, -ra.y * rb.x) < 0.0f) { V2<float> tmp = ra; ra = rb; rb = tmp; }
#pragma unroll 1
    for (int i = 2; i < k; ++i) {
        t.x = fdot3(m0, m1, m2, hist[i].x, hist[i].y, hist[i].z);
        t.y = __fmaf_rn(m3, hist[i].x, m4 * hist[i].y);
        const float cb = __fmaf_rn(rb.x, t.y, -rb.y * t.x);
        if (__fmaf_rn(ra.x, t.y, -ra.y * t.x) > 0.0f) {
            if (cb > 0.0f) rb = t;
        } else {
            if (cb < 0.0f) ra = t;
            else return false;
        }
    }
    float f = rsqrtf(__fmaf_rn(ra.x, ra.x, ra.y * ra.y));
    ra.x *= f; ra.y *= f;
    f = rsqrtf(__fmaf_rn(rb.x, rb.x, rb.y * rb.y));
    rb.x *= f; rb.y *= f;
    t.x = ra.x + rb.x;
    t.y = ra.y + rb.y;
    f = rsqrtf(__fmaf_rn(t.x, t.x, t.y * t.y));
    t.x *= f; t.y *= f;
    w.x = __fmaf_rn(m0, t.x, m3 * t.y);
    w.y = __fmaf_rn(m1, t.x, m4 * t.y);
    w.z = m2 * t.x;
    return true;
}

/* pair_test in fast arithmetic.  pp: the pair's two polytope indices (for
 * the vertex lists and start tables).  Same returns and margin as
 * pair_test, and the same first search direction (the line between the
 * two vertices 0): the iteration cap (code -1, always inside the band)
 * depends on the path from it, so a different start would change which
 * checks the band recomputes. */
__device__ __forceinline__ int pair_test_fast(const DevScene& sc, const float4* __restrict__ tab, int4 pr, int2 pp,
                                              const Frame<float>& tp, const Frame<float>& tq, float* margin)
{
    const float4* BP = tab + pr.x;
    const float4* BQ = tab + pr.y;
    const bool idP = pr.z == 0, idQ = pr.w == 0;
    float4 ep = BP[1], eq = BQ[1];
    V3<float> Sa, Sb;
    if (idQ) { Sa.x = eq.x; Sa.y = eq.y; Sa.z = eq.z; }
    else Sa = fxform(tq, eq.x, eq.y, eq.z);
    if (idP) { Sb.x = ep.x; Sb.y = ep.y; Sb.z = ep.z; }
    else Sb = fxform(tp, ep.x, ep.y, ep.z);
    V3<float> S;
    S.x = Sa.x - Sb.x; S.y = Sa.y - Sb.y; S.z = Sa.z - Sb.z;
    const float norm = fnormalize3(S);
    if (norm < sc.tiny_thr) S.x = 1.0f;
    V3<float> w; w.x = w.y = w.z = 0.0f;
    V3<float> hist[GPRM_MAX_ITERS];
    int combs[GPRM_MAX_ITERS];
    float best = 0.0f;
    int k = 0, l = 0;
    /* vertex lists, candidate lists and near-tie tolerances of the two */
    const int4 vP = sc.vinfo[pp.x], vQ = sc.vinfo[pp.y];
    bool tie = false;
#pragma unroll 1
    for (; k < GPRM_MAX_ITERS && l < GPRM_MAX_ITERS; ++l) {
        V3<float> Sp, Sq;
        if (idP) Sp = S;
        else Sp = frot_t(tp, S.x, S.y, S.z);
        if (idQ) { Sq.x = -S.x; Sq.y = -S.y; Sq.z = -S.z; }
        else Sq = frot_t(tq, -S.x, -S.y, -S.z);
        tie |= fsupport_cand2(sc, pp.x, vP, ep, Sp.x, Sp.y, Sp.z, pp.y, vQ, eq, Sq.x, Sq.y, Sq.z);
        V3<float> p0, q0;
        if (idP) { p0.x = ep.x; p0.y = ep.y; p0.z = ep.z; }
        else p0 = fxform(tp, ep.x, ep.y, ep.z);
        if (idQ) { q0.x = eq.x; q0.y = eq.y; q0.z = eq.z; }
        else q0 = fxform(tq, eq.x, eq.y, eq.z);
        V3<float> r;
        r.x = q0.x - p0.x; r.y = q0.y - p0.y; r.z = q0.z - p0.z;
        const float rn = fnormalize3(r);
        const float dp = fdot3(S.x, S.y, S.z, r.x, r.y, r.z);
        const float h = dp * rn;
        if (l == 0 || h > best) best = h;
        if (dp >= sc.sep_thr) {
            *margin = tie ? 0.0f : h;
            return 0;
        }
        hist[k] = r;
        const int comb = ent_idx(ep) | (ent_idx(eq) << 8);
        combs[k] = comb;
        bool rep = false;
#pragma unroll 1
        for (int j = 0; j < k; ++j)
            if (combs[j] == comb) { rep = true; break; }
        if (rep) {
            S = w;
        } else {
            if (k == 1) {
                w.x = hist[0].x + r.x; w.y = hist[0].y + r.y; w.z = hist[0].z + r.z;
                fnormalize3(w);
            }
            if (k >= 2 && !fhalf_plane(hist, k, w, r)) {
                *margin = tie ? 0.0f : best;
                return l + 1;
            }
            const float b = -2.0f * dp;
            S.x = __fmaf_rn(b, r.x, S.x); S.y = __fmaf_rn(b, r.y, S.y); S.z = __fmaf_rn(b, r.z, S.z);
            ++k;
        }
    }
    *margin = best;
    return -1;
}

/* Frame i+1 of the fast path from frame i (T): sincosf of the joint angle
 * and FMA products.  Shared by the shared-memory and register versions so
 * that both give the same bits. */
__device__ __forceinline__ Frame<float> fast_link(const DevScene& sc, const Frame<float>& T, const float* q, int i)
{
    float th = sc.q0[i], d = sc.d0[i];
    if (sc.types[i] == 0) th = q[i];
    else d = q[i];
    float cq, sq;
    sincosf(th, &sq, &cq);
    const float ca = sc.ca[i], sa = sc.sa[i];
    Frame<float> L;
    dh_frame<PF32>(L, cq, sq, ca, sa, sc.a[i], d);
    Frame<float> O;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float ux = L.m[3 * c], uy = L.m[3 * c + 1], uz = L.m[3 * c + 2];
        O.m[3 * c] = __fmaf_rn(T.m[0], ux, __fmaf_rn(T.m[3], uy, __fmaf_rn(T.m[6], uz, c == 3 ? T.m[9] : 0.0f)));
        O.m[3 * c + 1] = __fmaf_rn(T.m[1], ux, __fmaf_rn(T.m[4], uy, __fmaf_rn(T.m[7], uz, c == 3 ? T.m[10] : 0.0f)));
        O.m[3 * c + 2] = __fmaf_rn(T.m[2], ux, __fmaf_rn(T.m[5], uy, __fmaf_rn(T.m[8], uz, c == 3 ? T.m[11] : 0.0f)));
    }
    return O;
}

__device__ __forceinline__ void identity_frame(Frame<float>& T)
{
#pragma unroll
    for (int e = 0; e < 12; ++e) T.m[e] = 0.0f;
    T.m[0] = T.m[4] = T.m[8] = 1.0f;
}

/* The fast path's frames 0..ndof in registers (the overflow pass). */
__device__ __forceinline__ void forward_kinematics_fast(const DevScene& sc, const float* q, Frame<float>* F)
{
    identity_frame(F[0]);
#pragma unroll 1
    for (int i = 0; i < sc.ndof; ++i) F[i + 1] = fast_link(sc, F[i], q, i);
}

/* Forward kinematics of the fast path into the lane's shared-memory frames
 * (same layout as forward_kinematics_smem). */
__device__ __forceinline__ void forward_kinematics_smem_fast(const DevScene& sc, const float4* __restrict__ tab,
                                                             const float* q, float* out, float* cen)
{
    Frame<float> T;
    identity_frame(T);
    int slot = 0;
#pragma unroll 1
    for (int i = 0; i < sc.ndof; ++i) {
        const Frame<float> O = fast_link(sc, T, q, i);
#pragma unroll
        for (int e = 0; e < 12; ++e) out[(i * 12 + e) * 32] = O.m[e];
        for (; slot < sc.nslots && sc.slot_sys[slot] == i + 1; ++slot) slot_points(sc, tab, O, slot, cen);
        T = O;
    }
}

/* FP32 check band test: the check's result is decided within `band` of
 * contact (free with minimum margin below band, colliding with the deciding
 * pair's best margin above -band) or by the iteration cap. */
__device__ __forceinline__ bool in_band(int code, float margin, float band)
{
    if (code == -1) return true;
    if (code == 0) return !(margin >= band);
    return !(margin <= -band);
}

/* NaN-propagating minimum used for the free-check margin: NaN sticks. */
__device__ __forceinline__ float min_nan(float acc, float m)
{
    return (m < acc || m != m) ? m : acc;
}

/* Step configuration of an edge (robotconfigspace.cpp:409-420). */
__device__ __forceinline__ void edge_step_config(const float* __restrict__ qs, const float* __restrict__ qe,
                                                 long long e, long long offset, int ndof, int t, int tn,
                                                 float* q)
{
    float c1 = (float)t / (float)(tn - 1);
    float c2 = 1.0f - c1;
    for (int j = 0; j < ndof; ++j)
        q[j] = c1 * qs[e + offset * j] + c2 * qe[e + offset * j];
}

/* testnum = (int)(|qe-qs|/dq)+1 (robotconfigspace.cpp:665-671).  Returns
 * -1 for a non-finite or oversized edge. */
__device__ __forceinline__ int edge_testnum(const float* __restrict__ qs, const float* __restrict__ qe,
                                            long long e, long long offset, int ndof, float dq)
{
    float norm = 0.0f;
    for (int i = 0; i < ndof; ++i) {
        float diff = qe[e + offset * i] - qs[e + offset * i];
        norm = norm + diff * diff;
    }
    norm = __fsqrt_rn(norm);
    float x = norm / dq;
    if (!(x < 1.0e8f)) return -1;
    return (int)x + 1;
}

} /* namespace gprm */

#endif /* GPRM_DEVICE_CUH */

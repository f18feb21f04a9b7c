/*
 * gprm_oracle.cpp - CPU restatement of GPUPRM's collision checker.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
 * CUDA library: only tests, the smoke check and the bench's CPU-baseline
 * leg load it, and only to check or to time against.  No product code path
 * links, loads or calls it.
 *
 * What it restates (reference paths are relative to the GPUPRM tree):
 *   - modified-DH forward kinematics  prm/src/lib/robotspace/kinematics.h:27-37
 *     with trafo4::set/lapply/apply   prm/src/lib/collision4/geo4.h:183-288
 *   - normalize (zero norm -> zero)   geo4.h:165-171, float2 version geo4.h:80-83
 *   - first-improvement support-vertex hill climb
 *                                     prm/src/lib/collision4/collision4.h:66-103
 *   - orthtrafo23 + find_half_plane   collision4.h:111-223
 *   - Chung-Wang separating vector    collision4.h:226-332
 *   - indicator(q): bounds, FK, first nonzero pair result
 *                                     prm/src/lib/robotspace/robotconfigspace.cpp:313-346
 *   - edge steps: testnum/testpos, lerp, last nonzero step code
 *                                     robotconfigspace.cpp:378-465, 659-705
 *
 * Precision policies:
 *   F32   the reference CPU build's arithmetic: float storage and float
 *         + - * /, libm sincosf/sqrtf (cuda_head.h:20-29 resolve to the
 *         float overloads), the double literals of geo4.h:81,167 and
 *         collision4.h:20,321 kept as double.  Compiled without FMA
 *         contraction, so it equals the reference bit for bit.
 *   F32D  F32 with correctly rounded sin/cos of the joint angles: the
 *         arithmetic of the CUDA FP32 kernels, bit for bit.
 *   F64   the same algorithm with every value in double (the FP64 band
 *         recheck; no counterpart in the reference).  sin/cos come from
 *         gprm_sincos64.h so that the GPU recheck matches it bit for bit.
 *   FCNT  F32 with every floating-point operation counted (the algorithmic
 *         FLOP figure used for the roofline).
 *
 * The separation margin (a metric, in metres) is defined here and in the
 * kernels identically: at each Chung-Wang iteration h = dp * |q0 - p0|
 * (dp = <S, r/|r|>, so h is the gap along the unit direction S).  A
 * separated pair's margin is h at the deciding iteration; a colliding or
 * capped pair's margin is the largest h seen.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <algorithm>
#include <vector>

#include "../include/gprm_b200.h"
#include "../gpuprm_b200/csrc/gprm_sincos64.h"

namespace {

/* ------------------------------------------------------------------ */
/* precision policies                                                   */
/* ------------------------------------------------------------------ */

/* The reference's CPU build calls the float overloads that <math.h> brings
 * into C++ (cuda_head.h:23-28 name sin/cos/sqrt on float arguments): the
 * object code calls sincosf and sqrtf.  `float factor = 1.0/x` divides in
 * double and rounds to float, which equals the correctly rounded float
 * quotient (53 >= 2*24+2 bits, so the double rounding is innocuous). */
struct F32 {
    typedef float R;
    static R sqrt_(R x) { return sqrtf(x); }
    /* float factor = 1.0/norm (geo4.h:167) */
    static R recip(R n) { return (float)(1.0 / (double)n); }
    /* float factor = 1.0/sqrt_(x) (geo4.h:81) */
    static R rsqrt2(R s) { return (float)(1.0 / (double)sqrtf(s)); }
    static bool separated(R dp) { return (double)dp >= -0.000001; }
    static bool tiny(R n) { return (double)n < 0.000001; }
    static void trig(float x, R& c, R& s) { sincosf(x, &s, &c); }
    static void trig_alpha(float x, R& c, R& s) { sincosf(x, &s, &c); }
    static R from_f(float x) { return x; }
    static float to_f(R x) { return x; }
    /* b = -2.0*dp (collision4.h:321): exact in float */
    static R minus2(R dp) { return (float)(-2.0 * (double)dp); }
};

/* F32 with correctly rounded sin/cos of the joint angle (the double
 * sincos64 rounded to float), the trigonometry the CUDA kernels use; the
 * constant alpha terms keep libm's values (the library computes them on the
 * host with sincosf); everything else is F32. */
struct F32D : F32 {
    static void trig(float x, R& c, R& s) {
        double sd, cd;
        gprm_sincos64((double)x, &sd, &cd);
        c = (float)cd;
        s = (float)sd;
    }
};

struct F64 {
    typedef double R;
    static R sqrt_(R x) { return sqrt(x); }
    static R recip(R n) { return 1.0 / n; }
    static R rsqrt2(R s) { return 1.0 / sqrt(s); }
    static bool separated(R dp) { return dp >= -0.000001; }
    static bool tiny(R n) { return n < 0.000001; }
    static void trig(float x, R& c, R& s) { gprm_sincos64((double)x, &s, &c); }
    static void trig_alpha(float x, R& c, R& s) { gprm_sincos64((double)x, &s, &c); }
    static R from_f(float x) { return (double)x; }
    static float to_f(R x) { return (float)x; }
    static R minus2(R dp) { return -2.0 * dp; }
};

/* operation counters for FCNT */
struct Counters {
    double add, mul, div, sqrt, trig, cmp;
    double pairs, iters, climb_dots, checks;
};
static thread_local Counters g_cnt;

struct CF {
    float v;
    CF() : v(0) {}
    CF(float x) : v(x) {}
};
static inline CF operator+(CF a, CF b) { g_cnt.add++; return CF(a.v + b.v); }
static inline CF operator-(CF a, CF b) { g_cnt.add++; return CF(a.v - b.v); }
static inline CF operator*(CF a, CF b) { g_cnt.mul++; return CF(a.v * b.v); }
static inline CF operator/(CF a, CF b) { g_cnt.div++; return CF(a.v / b.v); }
static inline CF operator-(CF a) { return CF(-a.v); }
static inline bool operator>(CF a, CF b) { g_cnt.cmp++; return a.v > b.v; }
static inline bool operator<(CF a, CF b) { g_cnt.cmp++; return a.v < b.v; }
static inline bool operator==(CF a, CF b) { g_cnt.cmp++; return a.v == b.v; }

struct FCNT {
    typedef CF R;
    static R sqrt_(R x) { g_cnt.sqrt++; return CF(sqrtf(x.v)); }
    static R recip(R n) { g_cnt.div++; return CF((float)(1.0 / (double)n.v)); }
    static R rsqrt2(R s) { g_cnt.sqrt++; g_cnt.div++; return CF((float)(1.0 / (double)sqrtf(s.v))); }
    static bool separated(R dp) { g_cnt.cmp++; return (double)dp.v >= -0.000001; }
    static bool tiny(R n) { g_cnt.cmp++; return (double)n.v < 0.000001; }
    static void trig(float x, R& c, R& s) { g_cnt.trig += 2; float sf, cf; sincosf(x, &sf, &cf); c = CF(cf); s = CF(sf); }
    static void trig_alpha(float x, R& c, R& s) { float sf, cf; sincosf(x, &sf, &cf); c = CF(cf); s = CF(sf); }
    static R from_f(float x) { return CF(x); }
    static float to_f(R x) { return x.v; }
    static R minus2(R dp) { g_cnt.mul++; return CF((float)(-2.0 * (double)dp.v)); }
};

/* ------------------------------------------------------------------ */
/* scene                                                                */
/* ------------------------------------------------------------------ */

struct Scene {
    int ndof;
    float a[GPRM_MAX_DOF], alpha[GPRM_MAX_DOF], q0[GPRM_MAX_DOF], d0[GPRM_MAX_DOF];
    int types[GPRM_MAX_DOF];
    float mins[GPRM_MAX_DOF], maxs[GPRM_MAX_DOF];
    int N, M;
    std::vector<int> voff, n, moff, sys;
    std::vector<float> vx, vy, vz;
    std::vector<int> dsp, cnt, dest;
    std::vector<int> pfrom, pto;
};

template <class R> struct V3 { R x, y, z; };

/* affine frame, column form like trafo4::col[4] (geo4.h:24) */
template <class R> struct Frame { V3<R> c[4]; };

template <class P>
static inline typename P::R dot3(const V3<typename P::R>& u, const V3<typename P::R>& v)
{
    return u.x * v.x + u.y * v.y + u.z * v.z;
}

/* trafo4::set (geo4.h:194-203) */
template <class P>
static void dh_frame(Frame<typename P::R>& T, float a, float alpha, float theta, float d)
{
    typedef typename P::R R;
    R cq, sq, ca, sa;
    P::trig(theta, cq, sq);
    P::trig_alpha(alpha, ca, sa);
    R A = P::from_f(a), D = P::from_f(d);
    T.c[0].x = cq;       T.c[1].x = -sq;      T.c[2].x = R(0.0f); T.c[3].x = A;
    T.c[0].y = sq * ca;  T.c[1].y = cq * ca;  T.c[2].y = -sa;     T.c[3].y = -sa * D;
    T.c[0].z = sq * sa;  T.c[1].z = cq * sa;  T.c[2].z = ca;      T.c[3].z = ca * D;
}

/* R*u */
template <class P>
static inline V3<typename P::R> rot(const Frame<typename P::R>& T, const V3<typename P::R>& u)
{
    V3<typename P::R> o;
    o.x = T.c[0].x * u.x + T.c[1].x * u.y + T.c[2].x * u.z;
    o.y = T.c[0].y * u.x + T.c[1].y * u.y + T.c[2].y * u.z;
    o.z = T.c[0].z * u.x + T.c[1].z * u.y + T.c[2].z * u.z;
    return o;
}

/* T*u (geo4.h:215-221) */
template <class P>
static inline V3<typename P::R> xform(const Frame<typename P::R>& T, const V3<typename P::R>& u)
{
    V3<typename P::R> o;
    o.x = T.c[0].x * u.x + T.c[1].x * u.y + T.c[2].x * u.z + T.c[3].x;
    o.y = T.c[0].y * u.x + T.c[1].y * u.y + T.c[2].y * u.z + T.c[3].y;
    o.z = T.c[0].z * u.x + T.c[1].z * u.y + T.c[2].z * u.z + T.c[3].z;
    return o;
}

/* R'*u (geo4.h:249-255) */
template <class P>
static inline V3<typename P::R> rot_t(const Frame<typename P::R>& T, const V3<typename P::R>& u)
{
    V3<typename P::R> o;
    o.x = T.c[0].x * u.x + T.c[0].y * u.y + T.c[0].z * u.z;
    o.y = T.c[1].x * u.x + T.c[1].y * u.y + T.c[1].z * u.z;
    o.z = T.c[2].x * u.x + T.c[2].y * u.y + T.c[2].z * u.z;
    return o;
}

/* Kinematics::calculate (kinematics.h:28-37): F[0] = set(0,0,0,0),
 * F[i+1] = F[i] * set(a_i, alpha_i, theta_i, d_i). */
template <class P>
static void forward_kinematics(const Scene& s, const float* q, Frame<typename P::R>* F)
{
    typedef typename P::R R;
    dh_frame<P>(F[0], 0.0f, 0.0f, 0.0f, 0.0f);
    for (int i = 0; i < s.ndof; ++i) {
        float th = s.q0[i], d = s.d0[i];
        if (s.types[i] == 0) th = q[i];
        else d = q[i];
        Frame<R> L;
        dh_frame<P>(L, s.a[i], s.alpha[i], th, d);
        for (int c = 0; c < 3; ++c) F[i + 1].c[c] = rot<P>(F[i], L.c[c]);
        F[i + 1].c[3] = xform<P>(F[i], L.c[3]);
    }
}

/* geo4::normalize(float4&) (geo4.h:165-171): returns the norm; a zero norm
 * (infinite reciprocal) leaves a zero vector. */
template <class P>
static inline typename P::R normalize3(V3<typename P::R>& u)
{
    typedef typename P::R R;
    R norm = P::sqrt_(u.x * u.x + u.y * u.y + u.z * u.z);
    R f = P::recip(norm);
    if (f == R(INFINITY)) f = R(0.0f);
    u.x = u.x * f; u.y = u.y * f; u.z = u.z * f;
    return norm;
}

template <class R> struct V2 { R x, y; };

/* geo4::normalize(float2&) (geo4.h:80-83): no zero guard */
template <class P>
static inline void normalize2(V2<typename P::R>& u)
{
    typename P::R f = P::rsqrt2(u.x * u.x + u.y * u.y);
    u.x = u.x * f; u.y = u.y * f;
}

template <class P>
static inline typename P::R cross2(const V2<typename P::R>& v, const V2<typename P::R>& w)
{
    return v.x * w.y - v.y * w.x;
}

struct PolyRef { int voff, n, moff; };

template <class P>
static inline V3<typename P::R> vert(const Scene& s, const PolyRef& pr, int i)
{
    V3<typename P::R> v;
    v.x = P::from_f(s.vx[pr.voff + i]);
    v.y = P::from_f(s.vy[pr.voff + i]);
    v.z = P::from_f(s.vz[pr.voff + i]);
    return v;
}

/* support_vertex_searcher::search_support_vertex (collision4.h:66-103):
 * move to the first neighbour (in CRS order) with a strictly larger dot
 * product until none exists. */
template <class P>
static int climb(const Scene& s, const PolyRef& pr, int p, const V3<typename P::R>& dir)
{
    typedef typename P::R R;
    R best = dot3<P>(vert<P>(s, pr, p), dir);
    g_cnt.climb_dots++;
    for (;;) {
        bool moved = false;
        int b = s.dsp[pr.voff + p], e = b + s.cnt[pr.voff + p];
        for (int i = b; i < e; ++i) {
            int v = s.dest[pr.moff + i];
            R d = dot3<P>(vert<P>(s, pr, v), dir);
            g_cnt.climb_dots++;
            if (d > best) { best = d; p = v; moved = true; break; }
        }
        if (!moved) return p;
    }
}

/* find_half_plane (collision4.h:136-223) with orthtrafo23 (:111-134) */
template <class P>
static bool half_plane(const V3<typename P::R>* hist, int k, V3<typename P::R>& w,
                       const V3<typename P::R>& rk)
{
    typedef typename P::R R;
    if (dot3<P>(w, rk) > R(0.0f)) return true;
    R x = rk.x, y = rk.y, z = rk.z;
    R d = P::sqrt_(x * x + y * y);
    R m0 = x * z / d, m1 = y * z / d, m2 = -d;
    R m3 = -y / d, m4 = x / d, m5 = R(0.0f);
    V2<R> ra, rb, t;
    ra.x = m0 * hist[0].x + m1 * hist[0].y + m2 * hist[0].z;
    ra.y = m3 * hist[0].x + m4 * hist[0].y + m5 * hist[0].z;
    rb.x = m0 * hist[1].x + m1 * hist[1].y + m2 * hist[1].z;
    rb.y = m3 * hist[1].x + m4 * hist[1].y + m5 * hist[1].z;
    if (cross2<P>(ra, rb) < R(0.0f)) std::swap(ra, rb);
    for (int i = 2; i < k; ++i) {
        t.x = m0 * hist[i].x + m1 * hist[i].y + m2 * hist[i].z;
        t.y = m3 * hist[i].x + m4 * hist[i].y + m5 * hist[i].z;
        R cb = cross2<P>(rb, t);
        if (cross2<P>(ra, t) > R(0.0f)) {
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

#define MAX_ITERS 10  /* max_for_loop, max_for_loop_whole (collision4.h:17-18) */

/* seperating_vector_algorithm (collision4.h:226-332).  Returns 0 (separated),
 * l+1 (no separating half plane) or -1 (iteration cap). */
template <class P>
static int pair_test(const Scene& s, const PolyRef& P_, const PolyRef& Q_,
                     const Frame<typename P::R>& tp, const Frame<typename P::R>& tq,
                     typename P::R* margin)
{
    typedef typename P::R R;
    g_cnt.pairs++;
    int p = 0, q = 0;
    V3<R> Sa = xform<P>(tq, vert<P>(s, Q_, 0));
    V3<R> Sb = xform<P>(tp, vert<P>(s, P_, 0));
    V3<R> S;
    S.x = Sa.x - Sb.x; S.y = Sa.y - Sb.y; S.z = Sa.z - Sb.z;
    R norm = normalize3<P>(S);
    if (P::tiny(norm)) S.x = R(1.0f);
    V3<R> w; w.x = w.y = w.z = R(0.0f);
    V3<R> hist[MAX_ITERS];
    int combs[MAX_ITERS];
    R best = R(-INFINITY);
    bool have_best = false;
    int k = 0, l = 0;
    for (; k < MAX_ITERS && l < MAX_ITERS; ++l) {
        g_cnt.iters++;
        V3<R> nS; nS.x = -S.x; nS.y = -S.y; nS.z = -S.z;
        V3<R> Sp = rot_t<P>(tp, S);
        V3<R> Sq = rot_t<P>(tq, nS);
        p = climb<P>(s, P_, p, Sp);
        q = climb<P>(s, Q_, q, Sq);
        V3<R> p0 = xform<P>(tp, vert<P>(s, P_, p));
        V3<R> q0 = xform<P>(tq, vert<P>(s, Q_, q));
        V3<R>& r = hist[k];
        r.x = q0.x - p0.x; r.y = q0.y - p0.y; r.z = q0.z - p0.z;
        R rn = normalize3<P>(r);
        R dp = dot3<P>(S, r);
        R h = dp * rn;
        if (!have_best || h > best) { best = h; have_best = true; }
        if (P::separated(dp)) {
            if (margin) *margin = h;
            return 0;
        }
        int comb = p | (q << 8);
        combs[k] = comb;
        bool rep = false;
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
                if (margin) *margin = best;
                return l + 1;
            }
            R b = P::minus2(dp);
            S.x = S.x + b * r.x; S.y = S.y + b * r.y; S.z = S.z + b * r.z;
            ++k;
        }
    }
    if (margin) *margin = best;
    return -1;
}

/* The pair loop of indicator(q) / kernel_indicator2: first nonzero result
 * in pair order.  *pair_margin gets the deciding pair's margin (colliding)
 * or the minimum margin over all pairs (free). */
template <class P>
static int check_config(const Scene& s, const float* q, float* check_margin)
{
    typedef typename P::R R;
    g_cnt.checks++;
    Frame<R> F[GPRM_MAX_DOF + 1];
    forward_kinematics<P>(s, q, F);
    float mmin = INFINITY;
    for (int j = 0; j < s.M; ++j) {
        int a = s.pfrom[j], b = s.pto[j];
        PolyRef pa = {s.voff[a], s.n[a], s.moff[a]};
        PolyRef pb = {s.voff[b], s.n[b], s.moff[b]};
        R m = R(0.0f);
        int res = pair_test<P>(s, pa, pb, F[s.sys[a]], F[s.sys[b]], &m);
        float mf = P::to_f(m);
        if (res != 0) {
            if (check_margin) *check_margin = mf;
            return res;
        }
        if (mf < mmin || mf != mf) mmin = mf;
    }
    if (check_margin) *check_margin = mmin;
    return 0;
}

/* The same pair loop over pairs [j0, j1) only (first nonzero result in
 * pair order). */
template <class P>
static int check_config_range(const Scene& s, const float* q, int j0, int j1)
{
    typedef typename P::R R;
    Frame<R> F[GPRM_MAX_DOF + 1];
    forward_kinematics<P>(s, q, F);
    for (int j = j0; j < j1 && j < s.M; ++j) {
        int a = s.pfrom[j], b = s.pto[j];
        PolyRef pa = {s.voff[a], s.n[a], s.moff[a]};
        PolyRef pb = {s.voff[b], s.n[b], s.moff[b]};
        R m = R(0.0f);
        const int res = pair_test<P>(s, pa, pb, F[s.sys[a]], F[s.sys[b]], &m);
        if (res != 0) return res;
    }
    return 0;
}

/* The pairs an FP64 recheck has to test, from the FP32 pair loop: lo = the
 * first pair decided within the band (a collision, or a separation with
 * margin below band); hi = one past the last such pair when the check is
 * free, the pair count when it collides (the pairs after the deciding one
 * are not tested in FP32).  Returns the FP32 code. */
template <class P>
static int band_pair_range(const Scene& s, const float* q, float band, int* lo, int* hi)
{
    typedef typename P::R R;
    Frame<R> F[GPRM_MAX_DOF + 1];
    forward_kinematics<P>(s, q, F);
    *lo = s.M;
    int last = -1;
    for (int j = 0; j < s.M; ++j) {
        int a = s.pfrom[j], b = s.pto[j];
        PolyRef pa = {s.voff[a], s.n[a], s.moff[a]};
        PolyRef pb = {s.voff[b], s.n[b], s.moff[b]};
        R m = R(0.0f);
        const int res = pair_test<P>(s, pa, pb, F[s.sys[a]], F[s.sys[b]], &m);
        const float mf = P::to_f(m);
        if (res != 0) {
            if (j < *lo) *lo = j;
            *hi = s.M;
            return res;
        }
        if (!(mf >= band)) {
            if (j < *lo) *lo = j;
            last = j;
        }
    }
    *hi = last + 1;
    return 0;
}

/* check_boundaries(q) (robotconfigspace.cpp:795-802) */
static int out_of_bounds(const Scene& s, const float* q)
{
    for (int i = 0; i < s.ndof; ++i)
        if (q[i] < s.mins[i] || q[i] > s.maxs[i]) return 1;
    return 0;
}

/* A check is inside the FP64 band when its FP32 result is decided by a pair
 * whose margin lies within `band` of contact: free with minimum margin
 * below band, colliding with the deciding pair's best margin above -band,
 * or stopped by the iteration cap (code -1, margin undefined). */
static inline bool in_band(int code, float margin, float band)
{
    if (code == -1) return true;
    if (code == 0) return !(margin >= band);
    return !(margin <= -band);
}

/* FP32 check with the reference's libm trigonometry (device_trig == 0) or
 * the kernels' correctly rounded trigonometry (device_trig != 0). */
static inline int check32(const Scene& s, const float* q, float* m, int device_trig)
{
    return device_trig ? check_config<F32D>(s, q, m) : check_config<F32>(s, q, m);
}

} /* namespace */

/* ====================================================================== */
/* C ABI of the oracle (loaded by tests through ctypes)                    */
/* ====================================================================== */
extern "C" {

void* orc_create(const gprm_scene_desc* d)
{
    if (!d || d->ndof < 1 || d->ndof > GPRM_MAX_DOF || d->num_polytopes < 1 || d->num_pairs < 0)
        return NULL;
    Scene* s = new Scene();
    s->ndof = d->ndof;
    for (int i = 0; i < d->ndof; ++i) {
        s->a[i] = d->dh_a[i]; s->alpha[i] = d->dh_alpha[i];
        s->q0[i] = d->dh_q[i]; s->d0[i] = d->dh_d[i]; s->types[i] = d->dh_types[i];
        s->mins[i] = d->mins[i]; s->maxs[i] = d->maxs[i];
    }
    s->N = d->num_polytopes;
    s->M = d->num_pairs;
    int vo = 0, mo = 0;
    for (int k = 0; k < s->N; ++k) {
        s->voff.push_back(vo); s->n.push_back(d->poly_n[k]);
        s->moff.push_back(mo); s->sys.push_back(d->sys[k]);
        vo += d->poly_n[k]; mo += d->poly_m[k];
    }
    for (int i = 0; i < vo; ++i) {
        s->vx.push_back(d->vertices[3 * i]);
        s->vy.push_back(d->vertices[3 * i + 1]);
        s->vz.push_back(d->vertices[3 * i + 2]);
        s->dsp.push_back(d->dsp[i]);
        s->cnt.push_back(d->cnt[i]);
    }
    for (int i = 0; i < mo; ++i) s->dest.push_back(d->dest[i]);
    for (int j = 0; j < s->M; ++j) { s->pfrom.push_back(d->pair_from[j]); s->pto.push_back(d->pair_to[j]); }
    return s;
}

void orc_destroy(void* h) { delete (Scene*)h; }

/* mode & 3: 0 = FP32, 1 = FP64 only, 2 = FP32 with FP64 band recheck;
 * mode & 4: FP32 with the kernels' trigonometry (F32D) instead of libm's.
 * Vertex semantics of indicator(q) including the bounds check (code 1).
 * margin/inband may be NULL. */
int orc_check_configs(void* h, const float* q, int n, int offset, int mode, float band,
                      int* code, float* margin, unsigned char* inband)
{
    const Scene& s = *(const Scene*)h;
    float qi[GPRM_MAX_DOF];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < s.ndof; ++j) qi[j] = q[i + (size_t)offset * j];
        if (out_of_bounds(s, qi)) {
            code[i] = 1;
            if (margin) margin[i] = 0.0f;
            if (inband) inband[i] = 0;
            continue;
        }
        float m = 0.0f;
        int c;
        int prec = mode & 3, dt = mode & 4;
        if (prec == 1) {
            c = check_config<F64>(s, qi, &m);
            if (inband) inband[i] = 0;
        } else {
            c = check32(s, qi, &m, dt);
            bool ib = in_band(c, m, band);
            if (inband) inband[i] = ib;
            if (prec == 2 && ib) c = check_config<F64>(s, qi, NULL);
        }
        code[i] = c;
        if (margin) margin[i] = m;
    }
    return 0;
}

/* Pair ranges of an FP64 recheck (band_pair_range, FP32 with the
 * kernels' trigonometry when mode & 4) and the FP64 check over a range:
 * code[i] of configuration i over pairs [lo[i], hi[i]).  Configurations
 * out of bounds get lo = hi = 0 and code 1. */
int orc_band_pair_range(void* h, const float* q, int n, int offset, int mode, float band, int* lo, int* hi,
                        int* code32)
{
    const Scene& s = *(const Scene*)h;
    float qi[GPRM_MAX_DOF];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < s.ndof; ++j) qi[j] = q[i + (size_t)offset * j];
        if (out_of_bounds(s, qi)) { lo[i] = hi[i] = 0; code32[i] = 1; continue; }
        code32[i] = (mode & 4) ? band_pair_range<F32D>(s, qi, band, &lo[i], &hi[i])
                               : band_pair_range<F32>(s, qi, band, &lo[i], &hi[i]);
    }
    return 0;
}

int orc_check_configs64_range(void* h, const float* q, int n, int offset, const int* lo, const int* hi, int* code)
{
    const Scene& s = *(const Scene*)h;
    float qi[GPRM_MAX_DOF];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < s.ndof; ++j) qi[j] = q[i + (size_t)offset * j];
        code[i] = out_of_bounds(s, qi) ? 1 : check_config_range<F64>(s, qi, lo[i], hi[i]);
    }
    return 0;
}

/* testnum[l] = (int)(|qe-qs|/dq)+1 with float accumulation
 * (robotconfigspace.cpp:660-673). */
int orc_edge_testnum(const float* qs, const float* qe, int n, int offset, int ndof, float dq,
                     int* testnum)
{
    for (int l = 0; l < n; ++l) {
        float norm = 0.0f;
        for (int i = 0; i < ndof; ++i) {
            float diff = qe[l + (size_t)offset * i] - qs[l + (size_t)offset * i];
            norm += diff * diff;
        }
        norm = (float)sqrt((double)norm);
        testnum[l] = (int)(norm / dq) + 1;
    }
    return 0;
}

/* Configuration of step t of edge l (robotconfigspace.cpp:409-420):
 * c1 = t/(testnum-1), q = c1*qs + (1-c1)*qe. */
static void edge_step_config(const float* qs, const float* qe, int l, int offset, int ndof,
                             int t, int tn, float* q)
{
    float c1 = (float)t / (float)(tn - 1);
    float c2 = (float)(1.0 - (double)c1);
    for (int j = 0; j < ndof; ++j)
        q[j] = c1 * qs[l + (size_t)offset * j] + c2 * qe[l + (size_t)offset * j];
}

/* Edge checks.  mode as in orc_check_configs.  res[l] = code of the last
 * colliding step (0 if none), the value the reference's CPU path leaves
 * (robotconfigspace.cpp:458, 694-705).  No bounds check on edge steps, as
 * in kernel_indicator2.  *steps gets sum(testnum). */
int orc_check_edges(void* h, const float* qs, const float* qe, int n, int offset, float dq,
                    int mode, float band, int* res, int64_t* steps)
{
    const Scene& s = *(const Scene*)h;
    std::vector<int> tn(n > 0 ? n : 1);
    orc_edge_testnum(qs, qe, n, offset, s.ndof, dq, tn.data());
    int64_t total = 0;
    float q[GPRM_MAX_DOF];
    for (int l = 0; l < n; ++l) {
        int last = 0;
        for (int t = 0; t < tn[l]; ++t) {
            edge_step_config(qs, qe, l, offset, s.ndof, t, tn[l], q);
            int c;
            int prec = mode & 3, dt = mode & 4;
            if (prec == 1) {
                c = check_config<F64>(s, q, NULL);
            } else {
                float m = 0.0f;
                c = check32(s, q, &m, dt);
                if (prec == 2 && in_band(c, m, band)) c = check_config<F64>(s, q, NULL);
            }
            if (c != 0) last = c;
        }
        res[l] = last;
        total += tn[l];
    }
    if (steps) *steps = total;
    return 0;
}

/* Per-step FP32 results of edges: codes[step], margins[step], in the
 * global step order (edge-major, t ascending); mode & 4 selects F32D. */
int orc_edge_steps(void* h, const float* qs, const float* qe, int n, int offset, float dq,
                   int mode, int* codes, float* margins)
{
    const Scene& s = *(const Scene*)h;
    std::vector<int> tn(n > 0 ? n : 1);
    orc_edge_testnum(qs, qe, n, offset, s.ndof, dq, tn.data());
    float q[GPRM_MAX_DOF];
    int64_t pos = 0;
    for (int l = 0; l < n; ++l)
        for (int t = 0; t < tn[l]; ++t, ++pos) {
            edge_step_config(qs, qe, l, offset, s.ndof, t, tn[l], q);
            float m = 0.0f;
            codes[pos] = check32(s, q, &m, mode & 4);
            if (margins) margins[pos] = m;
        }
    return 0;
}

/* Verdict classes of edges, for comparing any FP32 checker's free/not-free
 * verdicts with the reference's at scale.  From the FP32 results of every
 * step (mode & 4: F32D trigonometry, else libm's):
 *   cls[l] = 1  a step collides outside the band (code > 0 with margin
 *               <= -band): the edge is "not free" whatever the rounding
 *            0  every step is free outside the band (margin >= band): "free"
 *            2  neither: the verdict is decided inside the band
 *   band_res[l]     the FP32 + FP64-band result (code of the last colliding
 *                   step, in-band steps recomputed in FP64), the value the
 *                   GPU's band mode must reproduce
 *   inband_steps[l] the number of in-band steps
 * (band_res and inband_steps may be NULL.)  Edge semantics as in
 * orc_check_edges (robotconfigspace.cpp:378-465, 694-705). */
int orc_edge_classify(void* h, const float* qs, const float* qe, int n, int offset, float dq, int mode,
                      float band, unsigned char* cls, int* band_res, int* inband_steps)
{
    const Scene& s = *(const Scene*)h;
    std::vector<int> tn(n > 0 ? n : 1);
    orc_edge_testnum(qs, qe, n, offset, s.ndof, dq, tn.data());
    float q[GPRM_MAX_DOF];
    for (int l = 0; l < n; ++l) {
        bool coll_out = false, any_in = false;
        int last = 0, nin = 0;
        for (int t = 0; t < tn[l]; ++t) {
            edge_step_config(qs, qe, l, offset, s.ndof, t, tn[l], q);
            float m = 0.0f;
            int c = check32(s, q, &m, mode & 4);
            const bool ib = in_band(c, m, band);
            if (ib) {
                any_in = true;
                ++nin;
                c = check_config<F64>(s, q, NULL);
            } else if (c != 0) {
                coll_out = true;
            }
            if (c != 0) last = c;
        }
        cls[l] = coll_out ? 1 : (any_in ? 2 : 0);
        if (band_res) band_res[l] = last;
        if (inband_steps) inband_steps[l] = nin;
    }
    return 0;
}

/* The same classes for vertex checks (indicator(q) semantics: out of
 * bounds is code 1, decided outside the band); band_code gets the FP32 +
 * FP64-band code. */
int orc_config_classify(void* h, const float* q, int n, int offset, int mode, float band, unsigned char* cls,
                        int* band_code)
{
    std::vector<int> code(n > 0 ? n : 1);
    std::vector<float> margin(n > 0 ? n : 1);
    std::vector<unsigned char> ib(n > 0 ? n : 1);
    orc_check_configs(h, q, n, offset, 2 | (mode & 4), band, code.data(), margin.data(), ib.data());
    for (int i = 0; i < n; ++i) {
        cls[i] = ib[i] ? 2 : (code[i] != 0 ? 1 : 0);
        if (band_code) band_code[i] = code[i];
    }
    return 0;
}

/* Counted FP32 work of vertex checks (no bounds short cut is taken for
 * in-bounds configurations; out-of-bounds ones count nothing).
 * out[0..9] = adds, muls, divs, sqrts, trig, compares, pairs, iterations,
 * climb dot products, checks. */
int orc_count_ops_configs(void* h, const float* q, int n, int offset, double* out)
{
    const Scene& s = *(const Scene*)h;
    memset(&g_cnt, 0, sizeof(g_cnt));
    float qi[GPRM_MAX_DOF];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < s.ndof; ++j) qi[j] = q[i + (size_t)offset * j];
        if (out_of_bounds(s, qi)) continue;
        check_config<FCNT>(s, qi, NULL);
    }
    double* c = (double*)&g_cnt;
    for (int i = 0; i < 10; ++i) out[i] = c[i];
    return 0;
}

/* The same for edge steps. */
int orc_count_ops_edges(void* h, const float* qs, const float* qe, int n, int offset, float dq,
                        double* out)
{
    const Scene& s = *(const Scene*)h;
    memset(&g_cnt, 0, sizeof(g_cnt));
    std::vector<int> tn(n > 0 ? n : 1);
    orc_edge_testnum(qs, qe, n, offset, s.ndof, dq, tn.data());
    float q[GPRM_MAX_DOF];
    for (int l = 0; l < n; ++l)
        for (int t = 0; t < tn[l]; ++t) {
            edge_step_config(qs, qe, l, offset, s.ndof, t, tn[l], q);
            check_config<FCNT>(s, q, NULL);
        }
    double* c = (double*)&g_cnt;
    for (int i = 0; i < 10; ++i) out[i] = c[i];
    return 0;
}

/* FP32 frames of a configuration: out[(ndof+1)*12], frame f column c row r
 * at out[f*12 + c*3 + r]; mode & 4 selects the kernels' trigonometry. */
int orc_forward_kinematics(void* h, const float* q, int mode, float* out)
{
    const Scene& s = *(const Scene*)h;
    Frame<float> F[GPRM_MAX_DOF + 1];
    if (mode & 4) forward_kinematics<F32D>(s, q, F);
    else forward_kinematics<F32>(s, q, F);
    for (int f = 0; f <= s.ndof; ++f)
        for (int c = 0; c < 4; ++c) {
            out[f * 12 + c * 3 + 0] = F[f].c[c].x;
            out[f * 12 + c * 3 + 1] = F[f].c[c].y;
            out[f * 12 + c * 3 + 2] = F[f].c[c].z;
        }
    return 0;
}

void orc_sincos64(const double* x, int n, double* s, double* c)
{
    for (int i = 0; i < n; ++i) gprm_sincos64(x[i], &s[i], &c[i]);
}

} /* extern "C" */

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
 *   float4 verts[sumn]   xyz in the body frame; w holds the adjacency of
 *                        the vertex as int bits: (dsp_local << 8) | cnt
 *   uint8  dest[summ]    neighbour indices, local to the polytope
 *   int4   pairs[M]      (voffA, moffA | sysA << 28, voffB, moffB | sysB << 28)
 *                        in the reference's pair order (CRS by `from`)
 */
#ifndef GPRM_DEVICE_CUH
#define GPRM_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include "gprm_sincos64.h"

#define GPRM_MAX_FRAMES 8   /* ndof + 1 */
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
    const float4* verts;
    const uint8_t* dest;
    const int4* pairs;
};

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
 * first-improvement climb over the vertex adjacency.  The maximum rises
 * strictly, so there are at most n-1 moves; the loop bound is never hit on
 * validated scenes and only guards corrupt data. */
template <class P>
__device__ __forceinline__ int climb(const float4* __restrict__ V, const uint8_t* __restrict__ D,
                                     int p, typename P::R dx, typename P::R dy, typename P::R dz)
{
    typedef typename P::R R;
    float4 v = V[p];
    R best = dot3<R>((R)v.x, (R)v.y, (R)v.z, dx, dy, dz);
#pragma unroll 1
    for (int guard = 0; guard < 128; ++guard) {
        int adj = __float_as_int(v.w);
        int b = adj >> 8, c = adj & 255;
        bool moved = false;
#pragma unroll 1
        for (int i = 0; i < c; ++i) {
            int u = D[b + i];
            float4 vu = V[u];
            R d = dot3<R>((R)vu.x, (R)vu.y, (R)vu.z, dx, dy, dz);
            if (d > best) { best = d; p = u; v = vu; moved = true; break; }
        }
        if (!moved) break;
    }
    return p;
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

/* seperating_vector_algorithm (collision4.h:226-332) for pair `pr`.
 * Returns 0 (separated), l+1 (no separating half plane) or -1 (cap).
 * *margin: h = dp*|q0-p0| at the deciding iteration if separated, else the
 * largest h seen. */
template <class P>
__device__ __forceinline__ int pair_test(const DevScene& sc, const float4* __restrict__ verts,
                                         const uint8_t* __restrict__ dest, int4 pr,
                                         const Frame<typename P::R>* F, typename P::R* margin)
{
    typedef typename P::R R;
    const float4* VP = verts + pr.x;
    const uint8_t* DP = dest + (pr.y & 0x0fffffff);
    const float4* VQ = verts + pr.z;
    const uint8_t* DQ = dest + (pr.w & 0x0fffffff);
    const Frame<R>& tp = F[(unsigned)pr.y >> 28];
    const Frame<R>& tq = F[(unsigned)pr.w >> 28];

    float4 vq0 = VQ[0], vp0 = VP[0];
    V3<R> Sa = xform<R>(tq, (R)vq0.x, (R)vq0.y, (R)vq0.z);
    V3<R> Sb = xform<R>(tp, (R)vp0.x, (R)vp0.y, (R)vp0.z);
    V3<R> S;
    S.x = Sa.x - Sb.x; S.y = Sa.y - Sb.y; S.z = Sa.z - Sb.z;
    R norm = normalize3<P>(S);
    if (P::tiny(sc, norm)) S.x = R(1.0f);
    V3<R> w; w.x = w.y = w.z = R(0.0f);
    V3<R> hist[GPRM_MAX_ITERS];
    int combs[GPRM_MAX_ITERS];
    R best = R(0.0f);
    int p = 0, q = 0, k = 0, l = 0;
#pragma unroll 1
    for (; k < GPRM_MAX_ITERS && l < GPRM_MAX_ITERS; ++l) {
        V3<R> Sp = rot_t<R>(tp, S.x, S.y, S.z);
        V3<R> Sq = rot_t<R>(tq, -S.x, -S.y, -S.z);
        p = climb<P>(VP, DP, p, Sp.x, Sp.y, Sp.z);
        q = climb<P>(VQ, DQ, q, Sq.x, Sq.y, Sq.z);
        float4 vp = VP[p], vq = VQ[q];
        V3<R> p0 = xform<R>(tp, (R)vp.x, (R)vp.y, (R)vp.z);
        V3<R> q0 = xform<R>(tq, (R)vq.x, (R)vq.y, (R)vq.z);
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
        int comb = p | (q << 8);
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

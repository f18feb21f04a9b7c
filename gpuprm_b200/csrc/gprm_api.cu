/*
 * gprm_api.cu - the C ABI of include/gprm_b200.h.
 *
 * Host side of RobotConfigspace<ndof> (prm/src/lib/robotspace/
 * robotconfigspace.{h,cpp}) rebuilt for one B200:
 *   - scene ingest and validation (load_config/construct,
 *     robotconfigspace.cpp:20-208) into a device layout built for the
 *     kernels (gprm_device.cuh), with every CRS index checked on the host
 *     so that no kernel can read out of bounds;
 *   - a request pool like the reference's buffer/stream pool
 *     (robotconfigspace.cpp:627-650, 726-742): each in-flight request owns a
 *     stream, pinned staging buffers and device buffers; wait() synchronises
 *     the request's stream before copying results out (the reference relied
 *     on pageable-memory copies being synchronous);
 *   - every failure returns a status code and leaves a message instead of
 *     asserting (util.hpp:44-46).
 */
#include <algorithm>
#include <limits.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <fstream>
#include <map>
#include <string>
#include <vector>

#include <atomic>

#include "../../include/gprm_b200.h"
#include "gprm_host.h"
#include "gprm_internal.h"

using namespace gprm;

namespace {

thread_local std::string g_create_error = "no error";

/* allocation-failure test hook: the n-th device allocation from the time
   it is set fails (0 = none) */
std::atomic<long long> g_fail_alloc{0};

}  // namespace

namespace gprm {

cudaError_t dev_malloc(void** p, size_t bytes)
{
    long long k = g_fail_alloc.load();
    while (k > 0) {
        if (g_fail_alloc.compare_exchange_weak(k, k - 1)) {
            if (k == 1) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

}  // namespace gprm

namespace {

int fail(gprm_space* h, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    else g_create_error = buf;
    return code;
}

#define CUDA_TRY(h, call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((h), e_ == cudaErrorMemoryAllocation ? GPRM_ERR_NOMEM : GPRM_ERR_CUDA, \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

/* smallest float f with (double)f >= x */
float float_ceil(double x)
{
    float f = (float)x;
    if ((double)f < x) f = nextafterf(f, INFINITY);
    while ((double)nextafterf(f, -INFINITY) >= x) f = nextafterf(f, -INFINITY);
    return f;
}

/* Certificate thresholds (see pair_certified in gprm_device.cuh).
 * eps_pos bounds, per coordinate, both the rounding of the reference's
 * world vertices (float transforms) and of the kernel's FMA ball centres;
 * radii are inflated by 2*eps_pos and by 1e-5 relative for the deviation
 * of the float rotation from orthogonality.  The slack added to the band
 * covers the rounding of the reference's dp and h (a few ulps of metres). */
/* Eigenvectors of a symmetric 3x3 matrix A (cyclic Jacobi rotations);
 * V's columns are the eigenvectors. */
void jacobi3(double A[3][3], double V[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) V[i][k] = i == k ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 50; ++sweep) {
        const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        if (off < 1e-300) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (A[p][q] == 0.0) continue;
                const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < 3; ++k) {   /* A <- A J */
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - sn * akq;
                    A[k][q] = sn * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {   /* A <- J^T A */
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - sn * aqk;
                    A[q][k] = sn * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {   /* V <- V J */
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - sn * vkq;
                    V[k][q] = sn * vkp + c * vkq;
                }
            }
    }
}

/* Clips the convex polygon `poly` (points (u, v)) by a*u + b*v + c >= 0. */
void clip_halfplane(std::vector<double>& poly, double a, double b, double c)
{
    std::vector<double> out;
    const size_t n = poly.size() / 2;
    for (size_t i = 0; i < n; ++i) {
        const double pu = poly[2 * i], pv = poly[2 * i + 1];
        const double qu = poly[2 * ((i + 1) % n)], qv = poly[2 * ((i + 1) % n) + 1];
        const double fp = a * pu + b * pv + c, fq = a * qu + b * qv + c;
        if (fp >= 0) { out.push_back(pu); out.push_back(pv); }
        if ((fp >= 0) != (fq >= 0)) {
            const double t = fp / (fp - fq);
            out.push_back(pu + t * (qu - pu));
            out.push_back(pv + t * (qv - pv));
        }
    }
    poly.swap(out);
}

/* Support candidates of every polytope for every direction bin of dir_bin:
 * vertex i is a candidate of a bin when some direction d of the bin has
 * <d, x_i - x_j> >= 0 for every CRS neighbour j of i (its normal cone,
 * enlarged when the adjacency misses an edge, so the set can only grow).
 * A bin's directions are d = s e_a + u e_b + v e_c on its cube face, with
 * (u, v) in the bin's cell of [-1, 1]^2 widened by 1e-2 on every side to
 * cover the float evaluation of dir_bin near cell and face borders.  Lists
 * hold ascending vertex indices; an empty list (rounding) falls back to
 * every vertex. */
void compute_support_candidates(gprm_space* h, const gprm_scene_desc* d, const std::vector<int>& voff,
                                const std::vector<int>& moff)
{
    h->cbin.assign((size_t)GPRM_START_BINS * h->npoly, 0u);
    h->cidx.clear();
    constexpr int C = GPRM_BIN_CELLS;
    const double eps = 1e-2;
    double lo[C], hi[C];
    for (int i = 0; i < C; ++i) {
        lo[i] = -1.0 + 2.0 * i / C - eps;
        hi[i] = -1.0 + 2.0 * (i + 1) / C + eps;
    }
    std::vector<double> poly;
    std::vector<unsigned char> list;
    for (int k = 0; k < h->npoly; ++k) {
        const int n = d->poly_n[k];
        for (int b = 0; b < GPRM_START_BINS; ++b) {
            const int face = b / (C * C), iu = (b % (C * C)) / C, iv = b % C;
            const double s = (face & 1) ? -1.0 : 1.0;
            const int ax = face / 2, bu = (ax + 1) % 3, bv = (ax + 2) % 3;   /* x:(y,z) y:(z,x) z:(x,y) */
            list.clear();
            for (int i = 0; i < n; ++i) {
                poly = {lo[iu], lo[iv], hi[iu], lo[iv], hi[iu], hi[iv], lo[iu], hi[iv]};
                const float* xi = d->vertices + 3 * (size_t)(voff[k] + i);
                const int g = voff[k] + i;
                for (int e = 0; e < d->cnt[g] && !poly.empty(); ++e) {
                    const int j = d->dest[moff[k] + d->dsp[g] + e];
                    const float* xj = d->vertices + 3 * (size_t)(voff[k] + j);
                    const double D[3] = {(double)xi[0] - xj[0], (double)xi[1] - xj[1], (double)xi[2] - xj[2]};
                    const double norm = sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
                    clip_halfplane(poly, D[bu], D[bv], s * D[ax] + 1e-9 * norm);
                }
                if (poly.size() >= 2) list.push_back((unsigned char)i);
            }
            if (list.empty())
                for (int i = 0; i < n; ++i) list.push_back((unsigned char)i);
            h->cbin[(size_t)GPRM_START_BINS * k + b] = ((unsigned)h->cidx.size() << 8) | (unsigned)list.size();
            h->cidx.insert(h->cidx.end(), list.begin(), list.end());
        }
    }
}

void compute_certificates(gprm_space* h, const int* from, const int* to)
{
    const double eps_pos = 1e-6 * h->extent;
    const double slack = 1e-4 + 1e-5 * h->extent;
    const double thr = (double)h->band + slack;
    (void)from;
    (void)to;
    h->pairs_b.resize(h->npairs);
    h->far.resize(h->npairs);
    h->scan_c.resize(h->npairs);
    h->scan_b.resize(h->npairs);
    for (int j = 0; j < h->npairs; ++j) {
        int a = h->pair_poly[2 * j], b = h->pair_poly[2 * j + 1];
        bool ok = (h->pair_sys[2 * j] == 0 || h->slot[a] >= 0) && (h->pair_sys[2 * j + 1] == 0 || h->slot[b] >= 0);
        double R = h->rad[a] * (1 + 1e-5) + h->rad[b] * (1 + 1e-5) + 4 * eps_pos;
        double x = 0.5 * ((2 * R + thr) + sqrt((2 * R + thr) * (2 * R + thr) + 4 * R * (R + thr)));
        float Rf = nextafterf((float)R, INFINITY);
        float T2 = nextafterf((float)(x * x * (1 + 1e-5)), INFINITY);
        if (!ok) { Rf = INFINITY; T2 = INFINITY; }
        int sa = h->pair_sys[2 * j] == 0 ? -1 : h->slot[a];
        int sb = h->pair_sys[2 * j + 1] == 0 ? -1 : h->slot[b];
        float fa, fb;
        memcpy(&fa, &sa, 4);
        memcpy(&fb, &sb, 4);
        h->pairs_b[j] = make_float4(Rf, T2, fa, fb);
        /* certificate-scan records: the static partner's ball centre and
         * vertex 0 inline (a polytope in frame 0 is used untransformed), the
         * slots of the moving ones, T2 and sqrt(T2) rounded up (for the
         * sweep test), R.  A pair without a slot for each moving polytope,
         * or with two static polytopes, is not usable by the scan (its
         * certificates go through pair_certified). */
        float4 fr = make_float4(0.0f, 0.0f, 0.0f, INFINITY);
        float4 sbv = make_float4(0.0f, 0.0f, 0.0f, Rf);
        int usable = 0;
        if (T2 < INFINITY && (sa >= 0 || sb >= 0)) {
            usable = 1;
            if (sa < 0 || sb < 0) {
                const int blk = sa < 0 ? h->pairs[j].x : h->pairs[j].y;
                const float4 c = h->tab[blk], v = h->tab[blk + 1];
                fr = make_float4(c.x, c.y, c.z, T2);
                sbv = make_float4(v.x, v.y, v.z, Rf);
            } else {
                fr.w = T2;
            }
        }
        float sq = nextafterf((float)sqrt((double)T2), INFINITY);
        int sqb;
        memcpy(&sqb, &sq, 4);
        h->far[j] = fr;
        h->scan_c[j] = make_int4(sa, sb, sqb, usable);
        h->scan_b[j] = sbv;
    }
    h->thr_dir = (float)thr;
    h->eps_dir = (float)(7.0 * eps_pos);
    /* box records: half extents inflated like the ball radii (the
       reference's and this code's transform rounding, 2 eps_pos per
       polytope) and by 2e-6 r for the FP32 axes' departure from an exact
       orthonormal basis; rounded up */
    h->box.resize((size_t)3 * h->npoly);
    for (int k = 0; k < h->npoly; ++k)
        for (int a = 0; a < 3; ++a) {
            const double e = h->box_e[3 * k + a] * (1 + 1e-5) + 2 * eps_pos + 2e-6 * h->rad[k];
            h->box[3 * k + a] = make_float4((float)h->box_ax[9 * k + 3 * a], (float)h->box_ax[9 * k + 3 * a + 1],
                                            (float)h->box_ax[9 * k + 3 * a + 2], nextafterf((float)e, INFINITY));
        }
}

int build_space(const gprm_scene_desc* d, float dq, int nbuf, gprm_space** out)
{
    if (!d || !out) return fail(nullptr, GPRM_ERR_ARG, "null argument");
    *out = nullptr;
    if (d->ndof < 1 || d->ndof > GPRM_MAX_DOF)
        return fail(nullptr, GPRM_ERR_SCENE, "ndof %d outside 1..%d", d->ndof, GPRM_MAX_DOF);
    if (d->num_polytopes < 1) return fail(nullptr, GPRM_ERR_SCENE, "N<=0");
    if (d->num_pairs < 0) return fail(nullptr, GPRM_ERR_SCENE, "M<0");
    if (!d->dh_a || !d->dh_alpha || !d->dh_q || !d->dh_d || !d->dh_types || !d->mins || !d->maxs ||
        !d->poly_n || !d->poly_m || !d->vertices || !d->dsp || !d->cnt || !d->dest || !d->sys ||
        (d->num_pairs > 0 && (!d->pair_from || !d->pair_to)))
        return fail(nullptr, GPRM_ERR_ARG, "null array in scene description");
    if (!(dq > 0.0f) || !isfinite(dq)) return fail(nullptr, GPRM_ERR_ARG, "dq must be positive");
    if (nbuf < 0) return fail(nullptr, GPRM_ERR_ARG, "nbuf < 0");

    gprm_space* h = new gprm_space();
    h->ndof = d->ndof;
    h->dq = dq;
    h->nbuf = nbuf;
    for (int i = 0; i < d->ndof; ++i) {
        h->a[i] = d->dh_a[i]; h->alpha[i] = d->dh_alpha[i];
        h->q0[i] = d->dh_q[i]; h->d0[i] = d->dh_d[i];
        h->types[i] = d->dh_types[i];
        h->mins[i] = d->mins[i]; h->maxs[i] = d->maxs[i];
        if (h->types[i] != 0 && h->types[i] != 1) {
            delete h;
            return fail(nullptr, GPRM_ERR_SCENE, "joint %d: type %d is neither 0 nor 1", i, d->dh_types[i]);
        }
    }
    h->npoly = d->num_polytopes;
    std::vector<int> voff(h->npoly), moff(h->npoly);
    long long sn = 0, sm = 0;
    for (int k = 0; k < h->npoly; ++k) {
        int n = d->poly_n[k], m = d->poly_m[k];
        /* robotconfigspace.cpp:44-51 asserts cnt>0 and n<=100 */
        if (n < 1 || n > GPRM_MAX_VERTICES || m < 0) {
            delete h;
            return fail(nullptr, GPRM_ERR_SCENE, "polytope %d: n=%d (1..%d) m=%d", k, n, GPRM_MAX_VERTICES, m);
        }
        if (d->sys[k] < 0 || d->sys[k] > d->ndof) {
            delete h;
            return fail(nullptr, GPRM_ERR_SCENE, "polytope %d: sys %d outside 0..%d", k, d->sys[k], d->ndof);
        }
        voff[k] = (int)sn; moff[k] = (int)sm;
        sn += n; sm += m;
    }
    if (sm >= (1LL << 17) * 64 || sn >= (1LL << 30)) {
        delete h;
        return fail(nullptr, GPRM_ERR_SCENE, "scene too large (sum n=%lld, sum m=%lld)", sn, sm);
    }
    h->sumn = (int)sn;
    h->summ = (int)sm;
    /* validate the CRS, then lay out one table block per polytope:
       [vertex 0][entries of dest in CRS order], each entry the neighbour's
       coordinates with (index | degree << 7 | offset << 15) in w */
    std::vector<int> boff(h->npoly);
    size_t ntab = 0;
    for (int k = 0; k < h->npoly; ++k) { boff[k] = (int)ntab; ntab += 2 + (size_t)d->poly_m[k]; }
    h->tab.resize(ntab);
    h->rad.assign(h->npoly, 0.0);
    h->box_ax.assign((size_t)9 * h->npoly, 0.0);
    h->box_e.assign((size_t)3 * h->npoly, 0.0);
    h->slot.assign(h->npoly, -1);
    for (int k = 0; k < h->npoly; ++k) {
        int n = d->poly_n[k], m = d->poly_m[k];
        if (m >= (1 << 17)) {
            delete h;
            return fail(nullptr, GPRM_ERR_SCENE, "polytope %d: m=%d >= 131072", k, m);
        }
        auto entry = [&](int v) {
            int g = voff[k] + v;
            int packed = v | (d->cnt[g] << 7) | (d->dsp[g] << 15);
            float w;
            memcpy(&w, &packed, 4);
            return make_float4(d->vertices[3 * (size_t)g], d->vertices[3 * (size_t)g + 1],
                               d->vertices[3 * (size_t)g + 2], w);
        };
        for (int i = 0; i < n; ++i) {
            int g = voff[k] + i;
            int ds = d->dsp[g], c = d->cnt[g];
            if (c < 1 || c > 255 || ds < 0 || ds + c > m) {
                delete h;
                return fail(nullptr, GPRM_ERR_SCENE,
                            "polytope %d vertex %d: dsp=%d cnt=%d (need cnt in 1..255, dsp+cnt<=m=%d)", k, i, ds, c, m);
            }
            float x = d->vertices[3 * (size_t)g], y = d->vertices[3 * (size_t)g + 1], z = d->vertices[3 * (size_t)g + 2];
            if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
                delete h;
                return fail(nullptr, GPRM_ERR_SCENE, "polytope %d vertex %d is not finite", k, i);
            }
        }
        for (int j = 0; j < m; ++j) {
            int v = d->dest[moff[k] + j];
            if (v < 0 || v >= n) {
                delete h;
                return fail(nullptr, GPRM_ERR_SCENE, "polytope %d: dest[%d]=%d outside 0..%d", k, j, v, n - 1);
            }
            h->tab[boff[k] + 2 + j] = entry(v);
        }
        h->tab[boff[k] + 1] = entry(0);
        {
            /* near-tie tolerance of the fast path's support values: 1e-5 of
               the largest vertex norm (body frame), about three times the
               largest difference between its dot products and the
               reference's (their rounding, the frames' and the search
               directions' accumulated rounding) */
            double vmax = 0;
            for (int i = 0; i < n; ++i) {
                const float* x = d->vertices + 3 * (size_t)(voff[k] + i);
                vmax = fmax(vmax, sqrt((double)x[0] * x[0] + (double)x[1] * x[1] + (double)x[2] * x[2]));
            }
            const float tie = (float)(1e-5 * vmax);
            int tb;
            memcpy(&tb, &tie, 4);
            h->vinfo.push_back(make_int4((int)h->vtab.size(), n, tb, 0));
        }
        for (int i = 0; i < n; ++i) h->vtab.push_back(entry(i));
        /* bounding ball: centre of the bounding box, radius to the farthest
           vertex (inflated in compute_certificates) */
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) {
                double x = d->vertices[3 * (size_t)(voff[k] + i) + c];
                lo[c] = x < lo[c] ? x : lo[c];
                hi[c] = x > hi[c] ? x : hi[c];
            }
        double cc[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
        float cf[3] = {(float)cc[0], (float)cc[1], (float)cc[2]};
        double r = 0;
        for (int i = 0; i < n; ++i) {
            double dd = 0;
            for (int c = 0; c < 3; ++c) {
                double x = d->vertices[3 * (size_t)(voff[k] + i) + c] - (double)cf[c];
                dd += x * x;
            }
            r = dd > r ? dd : r;
        }
        h->rad[k] = sqrt(r);
        h->tab[boff[k]] = make_float4(cf[0], cf[1], cf[2], (float)h->rad[k]);
        /* bounding box about the same centre: principal axes of the
           vertices, rounded to FP32, half extents measured along those */
        {
            double mean[3] = {0, 0, 0}, C[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, V[3][3];
            for (int i = 0; i < n; ++i)
                for (int c = 0; c < 3; ++c) mean[c] += d->vertices[3 * (size_t)(voff[k] + i) + c] / n;
            for (int i = 0; i < n; ++i) {
                double v[3];
                for (int c = 0; c < 3; ++c) v[c] = d->vertices[3 * (size_t)(voff[k] + i) + c] - mean[c];
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) C[a][b] += v[a] * v[b];
            }
            jacobi3(C, V);
            for (int a = 0; a < 3; ++a) {
                double nn = sqrt(V[0][a] * V[0][a] + V[1][a] * V[1][a] + V[2][a] * V[2][a]);
                if (!(nn > 0)) nn = 1;
                double ax[3];
                for (int c = 0; c < 3; ++c) ax[c] = (double)(float)(V[c][a] / nn);
                double e = 0;
                for (int i = 0; i < n; ++i) {
                    double t = 0;
                    for (int c = 0; c < 3; ++c) t += (d->vertices[3 * (size_t)(voff[k] + i) + c] - (double)cf[c]) * ax[c];
                    e = fabs(t) > e ? fabs(t) : e;
                }
                for (int c = 0; c < 3; ++c) h->box_ax[9 * k + 3 * a + c] = ax[c];
                h->box_e[3 * k + a] = e;
            }
        }
    }
    if ((size_t)sn * GPRM_START_BINS >= (1u << 24)) {
        delete h;
        return fail(nullptr, GPRM_ERR_SCENE, "scene too large for the support candidate lists");
    }
    compute_support_candidates(h, d, voff, moff);
    /* slots: moving polytopes in frame order */
    for (int f = 1; f <= h->ndof; ++f)
        for (int k = 0; k < h->npoly; ++k)
            if (d->sys[k] == f && (int)h->slot_sys.size() < GPRM_MAX_SLOTS) {
                h->slot[k] = (int)h->slot_sys.size();
                h->slot_sys.push_back(f);
                h->slot_block.push_back(boff[k]);
            }
    /* length scale: farthest static ball, plus the arm's reach */
    {
        double reach = 0, world = 0, link = 0;
        for (int i = 0; i < h->ndof; ++i) {
            double dm = fabs((double)h->d0[i]);
            if (h->types[i] == 1) dm = fmax(fabs((double)h->mins[i]), fabs((double)h->maxs[i]));
            reach += fabs((double)h->a[i]) + dm;
        }
        for (int k = 0; k < h->npoly; ++k) {
            float4 b = h->tab[boff[k]];
            double c = sqrt((double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z) + h->rad[k];
            if (d->sys[k] == 0) world = fmax(world, c);
            else link = fmax(link, c);
        }
        h->extent = fmax(1.0, fmax(world, reach + link));
    }
    h->npairs = d->num_pairs;
    h->pairs.resize(h->npairs);
    for (int j = 0; j < h->npairs; ++j) {
        int f = d->pair_from[j], t = d->pair_to[j];
        if (f < 0 || f >= h->npoly || t < 0 || t >= h->npoly) {
            delete h;
            return fail(nullptr, GPRM_ERR_SCENE, "pair %d: (%d,%d) outside 0..%d", j, f, t, h->npoly - 1);
        }
        /* polytope4data::build orders pairs in CRS by `from` (polytope4data.h:268-288) */
        if (j > 0 && f < d->pair_from[j - 1]) {
            delete h;
            return fail(nullptr, GPRM_ERR_SCENE, "pairs must be sorted by from (pair %d)", j);
        }
        h->pairs[j] = make_int4(boff[f], boff[t], d->sys[f], d->sys[t]);
        h->pair_poly.push_back(f); h->pair_poly.push_back(t);
        h->pair_sys.push_back(d->sys[f]); h->pair_sys.push_back(d->sys[t]);
    }
    compute_certificates(h, d->pair_from, d->pair_to);
    *out = h;
    return GPRM_OK;
}

template <class T>
bool read_bin(const std::string& path, T* dst, size_t n)
{
    std::ifstream f(path.c_str(), std::ios::in | std::ios::binary);
    if (!f) return false;
    f.read((char*)dst, (std::streamsize)(n * sizeof(T)));
    return (size_t)f.gcount() == n * sizeof(T);
}

void release_request(Request& r)
{
    if (r.st) cudaStreamDestroy(r.st);
    cudaFree(r.ctl);
    cudaFree(r.d_a);
    cudaFree(r.d_b);
    cudaFree(r.d_res);
    cudaFree(r.d_key);
    cudaFree(r.d_seg);
    cudaFree(r.d_queue);
    cudaFree(r.d_qpair);
    cudaFree(r.d_ovf);
    cudaFreeHost(r.ctl_host);
    cudaFreeHost(r.h_qwant);
    if (r.ev_q) cudaEventDestroy(r.ev_q);
    cudaFreeHost(r.h_a);
    cudaFreeHost(r.h_b);
    cudaFreeHost(r.h_res);
    r = Request();
}

/* Records the FP64 queue demand of one edge call (or part of one): `items`
 * queued (or wanted past the queue's end) for m edges. */
void note_queue_demand(gprm_space* h, unsigned items, long long m)
{
    const double d = (double)items / (double)m;
    if (d > h->qdens_edges) h->qdens_edges = d;
}

/* Grows the buffers of `r` to hold `n` items of `kind`; the stream and
 * the control block are created on first use.  with_host: pinned staging. */
int ensure_request(gprm_space* h, Request& r, int kind, size_t n, bool with_host, bool own_stream)
{
    if (own_stream && !r.st) CUDA_TRY(h, cudaStreamCreateWithFlags(&r.st, cudaStreamNonBlocking));
    if (!r.ctl) {
        CUDA_TRY(h, dev_malloc((void**)&r.ctl, HOST_PARTS * sizeof(Control)));
        CUDA_TRY(h, cudaHostAlloc((void**)&r.ctl_host, HOST_PARTS * sizeof(Control), cudaHostAllocDefault));
    }
    /* segment offsets for the batches that split their edges */
    if (kind == 1 && h->split_rounds > 0 && h->split_max > 0) {
        const size_t want = (size_t)std::min<long long>((long long)n, (long long)h->split_max);
        if (want > r.cap_seg || !r.d_seg) {
            cudaFree(r.d_seg);
            r.d_seg = nullptr;
            r.cap_seg = 0;
            const size_t cap = std::max<size_t>(want + want / 4, (size_t)EDGE_SPLIT_ONE_BLOCK);
            CUDA_TRY(h, dev_malloc((void**)&r.d_seg, edge_seg_words((long long)cap) * sizeof(unsigned)));
            r.cap_seg = cap;
        }
    }
    /* the demand of the last device-pointer edge call, once it has finished */
    if (r.q_pending) {
        const cudaError_t e = cudaEventQuery(r.ev_q);
        if (e != cudaErrorNotReady) r.q_pending = false;
        if (e == cudaSuccess && r.q_n > 0) note_queue_demand(h, *r.h_qwant, r.q_n);
        cudaGetLastError();   /* a query that is not ready is no error of this call */
    }
    /* a configuration queues at most one item; an edge as many as the
       busiest scene so far needed per edge (the overflow pass completes any
       call whose queue still runs over) */
    size_t need_q = (kind == 0) ? n : 4 * n + 65536;
    if (kind == 1 && h->qdens_edges > 0.0) {
        const double want = h->qdens_edges * (double)n * 1.25 + 65536.0;
        if (want > (double)need_q) need_q = want < 4e9 ? (size_t)want : (size_t)4e9;
    }
    if (n > r.cap_items || need_q > r.cap_queue || (with_host && !r.h_res && n > 0)) {
        size_t cap = n > r.cap_items ? n + n / 4 + 64 : r.cap_items;
        size_t qcap = (need_q > r.cap_queue) ? need_q + need_q / 4 : r.cap_queue;
        if (qcap < cap * 4 + 65536) qcap = cap * 4 + 65536;
        cudaFree(r.d_a); cudaFree(r.d_b); cudaFree(r.d_res); cudaFree(r.d_key); cudaFree(r.d_queue);
        cudaFree(r.d_qpair); cudaFree(r.d_ovf);
        r.d_a = r.d_b = nullptr; r.d_res = nullptr; r.d_key = nullptr; r.d_queue = nullptr; r.d_ovf = nullptr;
        r.d_qpair = nullptr;
        /* the capacities describe the buffers only once every one exists */
        r.cap_items = 0;
        r.cap_queue = 0;
        size_t nd = (size_t)h->ndof;
        CUDA_TRY(h, dev_malloc((void**)&r.d_res, cap * sizeof(int)));
        CUDA_TRY(h, dev_malloc((void**)&r.d_key, cap * sizeof(unsigned)));
        CUDA_TRY(h, dev_malloc((void**)&r.d_queue, qcap * sizeof(uint2)));
        CUDA_TRY(h, dev_malloc((void**)&r.d_qpair, qcap * sizeof(unsigned)));
        CUDA_TRY(h, dev_malloc((void**)&r.d_ovf, (2 * cap + 2 * HOST_PARTS + 64) * sizeof(unsigned)));
        if (with_host) {
            CUDA_TRY(h, dev_malloc((void**)&r.d_a, cap * nd * sizeof(float)));
            CUDA_TRY(h, dev_malloc((void**)&r.d_b, cap * nd * sizeof(float)));
            cudaFreeHost(r.h_a); cudaFreeHost(r.h_b); cudaFreeHost(r.h_res);
            r.h_a = r.h_b = nullptr; r.h_res = nullptr;
            CUDA_TRY(h, cudaHostAlloc((void**)&r.h_a, cap * nd * sizeof(float), cudaHostAllocDefault));
            CUDA_TRY(h, cudaHostAlloc((void**)&r.h_b, cap * nd * sizeof(float), cudaHostAllocDefault));
            CUDA_TRY(h, cudaHostAlloc((void**)&r.h_res, cap * sizeof(int), cudaHostAllocDefault));
        }
        r.cap_items = cap;
        r.cap_queue = qcap;
    }
    return GPRM_OK;
}

/* Returns a start/stop event pair from the handle's pool (grown on demand). */
int event_pair(gprm_space* h, std::vector<cudaEvent_t>& pool, size_t& used, cudaEvent_t* a, cudaEvent_t* b)
{
    while (pool.size() < used + 2) {
        cudaEvent_t e;
        CUDA_TRY(h, cudaEventCreate(&e));
        pool.push_back(e);
    }
    *a = pool[used];
    *b = pool[used + 1];
    used += 2;
    return GPRM_OK;
}

/* Enqueues one request on stream `st` with device inputs/outputs.
 * kind 0: q -> res.  kind 1: (qs, qe) -> res. */
int enqueue_part(gprm_space* h, Request& r, int kind, const float* a, const float* b, int* res, long long n,
                 long long offset, cudaStream_t st, Control* ctl, unsigned* key);

int enqueue(gprm_space* h, Request& r, int kind, const float* a, const float* b, int* res, long long n,
            long long offset, cudaStream_t st)
{
    int rc = enqueue_part(h, r, kind, a, b, res, n, offset, st, r.ctl, r.d_key);
    if (rc || kind != 1 || !(h->mode & GPRM_MODE_FP64_BAND) || r.q_pending) return rc;
    /* read the queue demand back for the next call's sizing, unless the
       stream is being captured (a graph replays without this host) */
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(h, cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone) return GPRM_OK;
    if (!r.h_qwant) CUDA_TRY(h, cudaHostAlloc((void**)&r.h_qwant, sizeof(unsigned), cudaHostAllocDefault));
    if (!r.ev_q) CUDA_TRY(h, cudaEventCreateWithFlags(&r.ev_q, cudaEventDisableTiming));
    CUDA_TRY(h, cudaMemcpyAsync(r.h_qwant, &r.ctl->qcount, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaEventRecord(r.ev_q, st));
    r.q_pending = true;
    r.q_n = n;
    return GPRM_OK;
}

/* One check request on stream st: items a[i + offset*j] (b: edge ends),
 * codes to res[0..n), with the control block ctl and the edge keys key. */
int enqueue_part(gprm_space* h, Request& r, int kind, const float* a, const float* b, int* res, long long n,
                 long long offset, cudaStream_t st, Control* ctl, unsigned* key)
{
    const int band_on = (h->mode & GPRM_MODE_FP64_BAND) != 0;
    CUDA_TRY(h, cudaMemsetAsync(ctl, 0, sizeof(Control), st));
    int recheck_blocks = h->sms * 4;
    /* the FP64 queue and, after the items' own region of the request
       (2 words per item from the part's first item), its overflow record */
    BandQueue bq;
    bq.items = r.d_queue;
    bq.cap = (unsigned)(r.cap_queue < 0xffffffffull ? r.cap_queue : 0xffffffffull);
    if (h->debug_qcap && h->debug_qcap < bq.cap) bq.cap = h->debug_qcap;
    bq.n = n;
    bq.ovf = nullptr;
    /* pair indices fit 16 bits on every scene the library builds; a larger
       pair list rechecks every pair */
    bq.pair_range = h->dsc.npairs <= 65535 ? r.d_qpair : nullptr;
    if (band_on && r.d_ovf) {
        /* every part's keys start at its first item (key = d_key + c0) */
        bq.ovf = r.d_ovf + 2 * (size_t)(key - r.d_key);
        CUDA_TRY(h, cudaMemsetAsync(bq.ovf + n, 0, (size_t)((n + 31) / 32) * sizeof(unsigned), st));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
    if (h->profiling) {
        int rc = event_pair(h, h->ev32, h->ev32_used, &e0, &e1);
        if (rc) return rc;
        if (band_on && (rc = event_pair(h, h->ev64, h->ev64_used, &e2, &e3))) return rc;
    }
    if (kind == 1)
        CUDA_TRY(h, cudaMemsetAsync(key, h->policy == GPRM_EDGES_EARLY_EXIT ? 0xff : 0x00,
                                    (size_t)n * sizeof(unsigned), st));
    if (e0) CUDA_TRY(h, cudaEventRecord(e0, st));
    if (kind == 0)
        CUDA_TRY(h, launch_check_configs(h->dsc, h->cfg_v, a, n, offset, res, band_on, h->band, bq, ctl, st));
    else {
        /* small batches split their long edges over several warps */
        const bool split = r.d_seg && h->split_rounds > 0 && n <= (long long)h->split_max &&
                           (size_t)n <= r.cap_seg;
        CUDA_TRY(h, launch_check_edges(h->dsc, h->cfg_e, a, b, n, offset, h->dq, h->policy, key, band_on,
                                       h->band, bq, ctl, st, split ? r.d_seg : nullptr, split ? h->split_rounds : 0));
        if (split) h->host_stats.launches += n <= EDGE_SPLIT_ONE_BLOCK ? 1 : 3;
    }
    if (e1) CUDA_TRY(h, cudaEventRecord(e1, st));
    if (band_on) {
        if (e2) CUDA_TRY(h, cudaEventRecord(e2, st));
        if (kind == 0)
            CUDA_TRY(h, launch_recheck(h->dsc, recheck_blocks, 0, a, nullptr, nullptr, offset, h->dq, h->policy,
                                       res, nullptr, bq, ctl, st));
        else
            CUDA_TRY(h, launch_recheck(h->dsc, recheck_blocks, 1, nullptr, a, b, offset, h->dq, h->policy,
                                       nullptr, key, bq, ctl, st));
        /* items the queue could not hold, recomputed in full */
        CUDA_TRY(h, launch_overflow(h->dsc, recheck_blocks, kind, kind == 0 ? a : nullptr, kind == 1 ? a : nullptr,
                                    b, offset, h->dq, h->policy, h->band, res, key, bq, ctl, st));
        if (e3) CUDA_TRY(h, cudaEventRecord(e3, st));
    }
    if (kind == 1) CUDA_TRY(h, launch_finalize_edges(n, h->policy, key, res, st));
    /* check + accumulate, plus recheck, overflow pass and finalize where they run */
    h->host_stats.launches += 2 + (band_on ? 2 : 0) + (kind == 1 ? 1 : 0);
    CUDA_TRY(h, launch_accumulate(ctl, h->d_total, st));
    return GPRM_OK;
}

int check_ready(gprm_space* h)
{
    if (!h) return GPRM_ERR_ARG;
    if (!h->inited) return fail(h, GPRM_ERR_STATE, "gprm_init has not been called");
    CUDA_TRY(h, cudaSetDevice(h->device));
    return GPRM_OK;
}

/* Host-buffer request: gather into pinned staging, copy, enqueue. */
int submit_host(gprm_space* h, int kind, const float* a, const float* b, int* res, int n, int offset, int* slot_out)
{
    int slot = -1;
    for (size_t i = 0; i < h->reqs.size(); ++i)
        if (!h->reqs[i].busy) { slot = (int)i; break; }
    if (slot < 0) {
        h->reqs.emplace_back();
        slot = (int)h->reqs.size() - 1;
    }
    Request& r = h->reqs[slot];
    int rc = ensure_request(h, r, kind, (size_t)(n > 0 ? n : 1), true, true);
    if (rc) return rc;
    const int nd = h->ndof;
    /* parts: the host copies part p into pinned staging while the device
       transfers and checks part p-1 (same stream, so the parts' checks run
       in order and share the FP64 queue) */
    const int parts = n >= (1 << 16) ? HOST_PARTS : 1;
    r.parts = parts;
    /* part boundaries (in 16ths): a small first part, whose staging is the
       only one not hidden, then three equal parts */
    static const int edge16[HOST_PARTS + 1] = {0, 1, 6, 11, 16};
    for (int p = 0; p < parts && n > 0; ++p) {
        const size_t c0 = parts == 1 ? 0 : (size_t)n * edge16[p] / 16;
        const size_t c1 = parts == 1 ? (size_t)n : (size_t)n * edge16[p + 1] / 16, m = c1 - c0;
        for (int j = 0; j < nd; ++j) {
            memcpy(r.h_a + (size_t)j * n + c0, a + (size_t)offset * j + c0, m * sizeof(float));
            if (kind == 1) memcpy(r.h_b + (size_t)j * n + c0, b + (size_t)offset * j + c0, m * sizeof(float));
        }
        const size_t pitch = (size_t)n * sizeof(float);
        CUDA_TRY(h, cudaMemcpy2DAsync(r.d_a + c0, pitch, r.h_a + c0, pitch, m * sizeof(float), nd,
                                      cudaMemcpyHostToDevice, r.st));
        if (kind == 1)
            CUDA_TRY(h, cudaMemcpy2DAsync(r.d_b + c0, pitch, r.h_b + c0, pitch, m * sizeof(float), nd,
                                          cudaMemcpyHostToDevice, r.st));
        rc = enqueue_part(h, r, kind, r.d_a + c0, kind == 1 ? r.d_b + c0 : nullptr, r.d_res + c0, (long long)m, n,
                          r.st, r.ctl + p, r.d_key + c0);
        if (rc) return rc;
        CUDA_TRY(h, cudaMemcpyAsync(r.h_res + c0, r.d_res + c0, m * sizeof(int), cudaMemcpyDeviceToHost, r.st));
    }
    if (n > 0)
        CUDA_TRY(h, cudaMemcpyAsync(r.ctl_host, r.ctl, parts * sizeof(Control), cudaMemcpyDeviceToHost, r.st));
    r.busy = true;
    r.kind = kind;
    r.user_res = res;
    r.n = n;
    r.user_a = a;
    r.user_b = b;
    r.user_offset = offset;
    *slot_out = slot;
    return GPRM_OK;
}

int complete_host(gprm_space* h, int slot)
{
    Request& r = h->reqs[slot];
    r.busy = false;
    if (r.n == 0) return GPRM_OK;
    CUDA_TRY(h, cudaStreamSynchronize(r.st));
    Control c = r.ctl_host[0];
    for (int p = 1; p < r.parts; ++p) {
        c.flags |= r.ctl_host[p].flags;
        c.steps_nominal += r.ctl_host[p].steps_nominal;
    }
    if (c.flags & GPRM_DEVFLAG_BAD_EDGE)
        return fail(h, GPRM_ERR_ARG, "an edge has a non-finite or oversized length (|qe-qs|/dq >= 1e8)");
    if (r.kind == 1) {
        static const int edge16[HOST_PARTS + 1] = {0, 1, 6, 11, 16};
        for (int p = 0; p < r.parts; ++p) {
            const long long m = r.parts == 1 ? r.n
                                              : (long long)r.n * edge16[p + 1] / 16 - (long long)r.n * edge16[p] / 16;
            if (m > 0) note_queue_demand(h, r.ctl_host[p].qcount, m);
        }
    }
    /* GPRM_DEVFLAG_QUEUE_FULL: the overflow pass has completed the results */
    memcpy(r.user_res, r.h_res, (size_t)r.n * sizeof(int));
    /* edge-step and band counters accumulate on the device (d_total) */
    if (r.kind == 0) h->host_stats.vertex_checks += r.n;
    return GPRM_OK;
}

}  // namespace

/* ====================================================================== */

extern "C" {

int gprm_create(const gprm_scene_desc* desc, float dq, int nbuf, gprm_space** out)
{
    return build_space(desc, dq, nbuf, out);
}

int gprm_create_from_dir(const char* path, int ndof, float dq, int nbuf, gprm_space** out)
{
    if (!path || !out) return fail(nullptr, GPRM_ERR_ARG, "null argument");
    std::string p(path);
    int nd = 0;
    if (!read_bin(p + "/ndof.bin", &nd, 1)) return fail(nullptr, GPRM_ERR_IO, "cannot read %s/ndof.bin", path);
    if (nd != ndof) return fail(nullptr, GPRM_ERR_SCENE, "wrong ndof: file has %d, caller asked for %d", nd, ndof);
    if (nd < 1 || nd > GPRM_MAX_DOF) return fail(nullptr, GPRM_ERR_SCENE, "ndof %d unsupported", nd);
    std::vector<float> a(nd), alpha(nd), q(nd), d(nd), mins(nd), maxs(nd);
    std::vector<int> types(nd);
    bool ok = read_bin(p + "/dh/a.bin", a.data(), nd) && read_bin(p + "/dh/alpha.bin", alpha.data(), nd) &&
              read_bin(p + "/dh/q.bin", q.data(), nd) && read_bin(p + "/dh/d.bin", d.data(), nd) &&
              read_bin(p + "/dh/types.bin", types.data(), nd) && read_bin(p + "/mins.bin", mins.data(), nd) &&
              read_bin(p + "/maxs.bin", maxs.data(), nd);
    if (!ok) return fail(nullptr, GPRM_ERR_IO, "cannot read the DH or bound files under %s", path);
    int N = 0, M = 0;
    if (!read_bin(p + "/polys/N.bin", &N, 1) || N <= 0) return fail(nullptr, GPRM_ERR_IO, "bad polys/N.bin");
    if (!read_bin(p + "/pairs/M.bin", &M, 1) || M < 0) return fail(nullptr, GPRM_ERR_IO, "bad pairs/M.bin");
    std::vector<int> sys(N), from(M > 0 ? M : 1), to(M > 0 ? M : 1), pn(N), pm(N);
    if (!read_bin(p + "/polys/sys.bin", sys.data(), N) ||
        (M > 0 && (!read_bin(p + "/pairs/from.bin", from.data(), M) || !read_bin(p + "/pairs/to.bin", to.data(), M))))
        return fail(nullptr, GPRM_ERR_IO, "cannot read sys/from/to");
    std::vector<float> verts;
    std::vector<int> dsp, cnt, dest;
    for (int i = 0; i < N; ++i) {
        std::string pp = p + "/polys/poly" + std::to_string(i);
        int size[2];
        if (!read_bin(pp + "/size.bin", size, 2)) return fail(nullptr, GPRM_ERR_IO, "cannot read %s/size.bin", pp.c_str());
        int n = size[0], m = size[1];
        if (n < 1 || n > GPRM_MAX_VERTICES || m < 0)
            return fail(nullptr, GPRM_ERR_SCENE, "polytope %d: n=%d m=%d", i, n, m);
        pn[i] = n; pm[i] = m;
        size_t v0 = verts.size(), c0 = dsp.size(), e0 = dest.size();
        verts.resize(v0 + 3 * (size_t)n);
        dsp.resize(c0 + n); cnt.resize(c0 + n); dest.resize(e0 + m);
        if (!read_bin(pp + "/vertices.bin", verts.data() + v0, 3 * (size_t)n) ||
            !read_bin(pp + "/dsp.bin", dsp.data() + c0, n) || !read_bin(pp + "/cnt.bin", cnt.data() + c0, n) ||
            (m > 0 && !read_bin(pp + "/dest.bin", dest.data() + e0, m)))
            return fail(nullptr, GPRM_ERR_IO, "cannot read polytope files under %s", pp.c_str());
    }
    gprm_scene_desc desc;
    desc.ndof = nd;
    desc.dh_a = a.data(); desc.dh_alpha = alpha.data(); desc.dh_q = q.data(); desc.dh_d = d.data();
    desc.dh_types = types.data(); desc.mins = mins.data(); desc.maxs = maxs.data();
    desc.num_polytopes = N; desc.poly_n = pn.data(); desc.poly_m = pm.data();
    desc.vertices = verts.data(); desc.dsp = dsp.data(); desc.cnt = cnt.data();
    desc.dest = dest.empty() ? pn.data() : dest.data();
    desc.sys = sys.data(); desc.num_pairs = M; desc.pair_from = from.data(); desc.pair_to = to.data();
    return build_space(&desc, dq, nbuf, out);
}

int gprm_init(gprm_space* h, int rank, int size)
{
    if (!h) return fail(nullptr, GPRM_ERR_ARG, "null handle");
    if (h->inited) return GPRM_OK;
    if (size < 1 || rank < 0 || rank >= size) return fail(h, GPRM_ERR_ARG, "rank %d / size %d", rank, size);
    int devcount = 0;
    CUDA_TRY(h, cudaGetDeviceCount(&devcount));
    if (devcount < 1) return fail(h, GPRM_ERR_CUDA, "no CUDA device");
    /* device = rank*devcount/size (robotconfigspace.cpp:229) */
    h->device = (int)(((long long)rank * devcount) / size);
    CUDA_TRY(h, cudaSetDevice(h->device));
    CUDA_TRY(h, cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device));
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));

    /* the candidate lists in fixed slots per (polytope, bin): cslots = the
       longest list, shorter ones padded with their last entry */
    h->cslots = 1;
    for (unsigned hb : h->cbin) h->cslots = std::max(h->cslots, (int)(hb & 255u));
    h->ccnt.assign(h->cbin.size(), 0);
    h->ctab.assign(h->cbin.size() * (size_t)h->cslots, make_float4(0.f, 0.f, 0.f, 0.f));
    for (size_t kb = 0; kb < h->cbin.size(); ++kb) {
        const int k = (int)(kb / GPRM_START_BINS), n = (int)(h->cbin[kb] & 255u);
        const size_t off = h->cbin[kb] >> 8;
        h->ccnt[kb] = (unsigned char)n;
        for (int s = 0; s < h->cslots; ++s) {
            const int idx = n > 0 ? h->cidx[off + (s < n ? s : n - 1)] : 0;
            h->ctab[kb * h->cslots + s] = h->vtab[(size_t)h->vinfo[k].x + idx];
        }
    }

    /* d_scene: tab | pairs | pairs_b | far | scan_c | scan_b | ppoly | box | vtab | vinfo | ctab | ccnt */
    size_t tb = h->tab.size() * sizeof(float4), pb = (size_t)h->npairs * sizeof(int4);
    size_t fsb = (size_t)h->npairs * sizeof(int2);
    size_t bxo = tb + 5 * pb + fsb, bxb = h->box.size() * sizeof(float4);
    bxo = (bxo + 15) & ~(size_t)15;
    const size_t vto = (bxo + bxb + 15) & ~(size_t)15, vtb = h->vtab.size() * sizeof(float4);
    const size_t vio = vto + vtb, vib = h->vinfo.size() * sizeof(int4);
    const size_t cbo = (vio + vib + 15) & ~(size_t)15, cbb = h->ctab.size() * sizeof(float4);
    const size_t cio = cbo + cbb, cib = h->ccnt.size();
    CUDA_TRY(h, dev_malloc((void**)&h->d_scene, cio + cib + 64));
    char* base = (char*)h->d_scene;
    CUDA_TRY(h, cudaMemcpy(base, h->tab.data(), tb, cudaMemcpyHostToDevice));
    if (pb) CUDA_TRY(h, cudaMemcpy(base + tb, h->pairs.data(), pb, cudaMemcpyHostToDevice));
    if (pb) CUDA_TRY(h, cudaMemcpy(base + tb + pb, h->pairs_b.data(), pb, cudaMemcpyHostToDevice));
    if (pb) CUDA_TRY(h, cudaMemcpy(base + tb + 2 * pb, h->far.data(), pb, cudaMemcpyHostToDevice));
    if (pb) CUDA_TRY(h, cudaMemcpy(base + tb + 3 * pb, h->scan_c.data(), pb, cudaMemcpyHostToDevice));
    if (pb) CUDA_TRY(h, cudaMemcpy(base + tb + 4 * pb, h->scan_b.data(), pb, cudaMemcpyHostToDevice));
    if (pb) CUDA_TRY(h, cudaMemcpy(base + tb + 5 * pb, h->pair_poly.data(), fsb, cudaMemcpyHostToDevice));
    if (bxb) CUDA_TRY(h, cudaMemcpy(base + bxo, h->box.data(), bxb, cudaMemcpyHostToDevice));
    if (vtb) CUDA_TRY(h, cudaMemcpy(base + vto, h->vtab.data(), vtb, cudaMemcpyHostToDevice));
    if (vib) CUDA_TRY(h, cudaMemcpy(base + vio, h->vinfo.data(), vib, cudaMemcpyHostToDevice));
    if (cbb) CUDA_TRY(h, cudaMemcpy(base + cbo, h->ctab.data(), cbb, cudaMemcpyHostToDevice));
    if (cib) CUDA_TRY(h, cudaMemcpy(base + cio, h->ccnt.data(), cib, cudaMemcpyHostToDevice));

    DevScene& s = h->dsc;
    memset(&s, 0, sizeof(s));
    s.ndof = h->ndof; s.dq = h->dq; s.npoly = h->npoly; s.npairs = h->npairs; s.sumn = h->sumn; s.summ = h->summ;
    for (int i = 0; i < h->ndof; ++i) {
        s.a[i] = h->a[i]; s.q0[i] = h->q0[i]; s.d0[i] = h->d0[i]; s.types[i] = h->types[i];
        s.mins[i] = h->mins[i]; s.maxs[i] = h->maxs[i];
        /* cos_/sin_(alpha) as the reference CPU build evaluates them (sincosf) */
        float sa, ca;
        sincosf(h->alpha[i], &sa, &ca);
        s.ca[i] = ca; s.sa[i] = sa;
        gprm_sincos64((double)h->alpha[i], &s.sa64[i], &s.ca64[i]);
    }
    s.sep_thr = float_ceil(-0.000001);
    s.tiny_thr = float_ceil(0.000001);
    s.ntab = (int)h->tab.size();
    s.tab = (const float4*)base;
    s.pairs = (const int4*)(base + tb);
    s.pairs_b = (const float4*)(base + tb + pb);
    s.far = (const float4*)(base + tb + 2 * pb);
    s.scan_c = (const int4*)(base + tb + 3 * pb);
    s.scan_b = (const float4*)(base + tb + 4 * pb);
    s.ppoly = (const int2*)(base + tb + 5 * pb);
    s.box = bxb ? (const float4*)(base + bxo) : nullptr;
    s.vtab = (const float4*)(base + vto);
    s.vinfo = (const int4*)(base + vio);
    s.ctab = cbb ? (const float4*)(base + cbo) : nullptr;
    s.ccnt = (const unsigned char*)(base + cio);
    s.cslots = h->cslots;
    s.fast = (h->mode & GPRM_MODE_FAST) != 0;
    s.thr_dir = h->thr_dir;
    s.eps_dir = h->eps_dir;
    s.nslots = (int)h->slot_sys.size();
    for (int i = 0; i < s.nslots; ++i) { s.slot_sys[i] = h->slot_sys[i]; s.slot_block[i] = h->slot_block[i]; }

    CUDA_TRY(h, plan_launch(s, 1, 128, &h->cfg_v));
    CUDA_TRY(h, plan_launch(s, 0, 128, &h->cfg_e));
    CUDA_TRY(h, dev_malloc((void**)&h->d_total, sizeof(Control)));
    CUDA_TRY(h, cudaMemset(h->d_total, 0, sizeof(Control)));
    memset(&h->host_stats, 0, sizeof(h->host_stats));
    h->inited = true;
    return GPRM_OK;
}

void gprm_destroy(gprm_space* h)
{
    if (!h) return;
    if (h->inited) {
        cudaSetDevice(h->device);
        for (auto& r : h->reqs) {
            if (r.st) cudaStreamSynchronize(r.st);
            release_request(r);
        }
        if (h->stream) cudaStreamSynchronize(h->stream);
        release_request(h->dev);
        cudaFree(h->d_total);
        cudaFree(h->d_scene);
        if (h->stream) cudaStreamDestroy(h->stream);
    }
    delete h;
}

const char* gprm_last_error(const gprm_space* h)
{
    return h ? h->err.c_str() : g_create_error.c_str();
}

int gprm_set_mode(gprm_space* h, int mode)
{
    if (!h) return GPRM_ERR_ARG;
    if (mode & ~(GPRM_MODE_FP64_BAND | GPRM_MODE_FAST)) return fail(h, GPRM_ERR_ARG, "unknown mode %d", mode);
    h->mode = mode;
    h->dsc.fast = (mode & GPRM_MODE_FAST) != 0;
    return GPRM_OK;
}

int gprm_set_edge_policy(gprm_space* h, int policy)
{
    if (!h) return GPRM_ERR_ARG;
    if (policy != GPRM_EDGES_EARLY_EXIT && policy != GPRM_EDGES_ALL_STEPS)
        return fail(h, GPRM_ERR_ARG, "unknown edge policy %d", policy);
    h->policy = policy;
    return GPRM_OK;
}

int gprm_set_edge_split(gprm_space* h, int max_edges, int seg_rounds)
{
    if (!h) return GPRM_ERR_ARG;
    if (max_edges < 0 || max_edges > (int)EDGE_SPLIT_MAX || seg_rounds < 1)
        return fail(h, GPRM_ERR_ARG, "edge split: max_edges must be in [0, %d] and seg_rounds >= 1",
                    (int)EDGE_SPLIT_MAX);
    h->split_max = max_edges;
    h->split_rounds = seg_rounds;
    return GPRM_OK;
}

int gprm_set_band(gprm_space* h, float band_m)
{
    if (!h) return GPRM_ERR_ARG;
    if (!(band_m >= 0.0f) || !isfinite(band_m)) return fail(h, GPRM_ERR_ARG, "band must be finite and >= 0");
    h->band = band_m;
    compute_certificates(h, nullptr, nullptr);
    if (h->inited) {
        CUDA_TRY(h, cudaSetDevice(h->device));
        CUDA_TRY(h, cudaDeviceSynchronize());
        size_t tb = h->tab.size() * sizeof(float4), pb = (size_t)h->npairs * sizeof(int4);
        if (pb) CUDA_TRY(h, cudaMemcpy((char*)h->d_scene + tb + pb, h->pairs_b.data(), pb, cudaMemcpyHostToDevice));
        if (pb) CUDA_TRY(h, cudaMemcpy((char*)h->d_scene + tb + 2 * pb, h->far.data(), pb, cudaMemcpyHostToDevice));
        if (pb) CUDA_TRY(h, cudaMemcpy((char*)h->d_scene + tb + 3 * pb, h->scan_c.data(), pb, cudaMemcpyHostToDevice));
        if (pb) CUDA_TRY(h, cudaMemcpy((char*)h->d_scene + tb + 4 * pb, h->scan_b.data(), pb, cudaMemcpyHostToDevice));
        h->dsc.thr_dir = h->thr_dir;
        h->dsc.eps_dir = h->eps_dir;
    }
    return GPRM_OK;
}

int gprm_get_stats(const gprm_space* hc, gprm_stats* out)
{
    gprm_space* h = const_cast<gprm_space*>(hc);
    if (!h || !out) return GPRM_ERR_ARG;
    *out = h->host_stats;
    if (!h->inited) return GPRM_OK;
    int rc = check_ready(h);
    if (rc) return rc;
    /* the edge-step and band counters of every request accumulate on the device */
    Control tot;
    CUDA_TRY(h, cudaDeviceSynchronize());
    CUDA_TRY(h, cudaMemcpy(&tot, h->d_total, sizeof(Control), cudaMemcpyDeviceToHost));
    out->edge_steps_nominal = (int64_t)tot.steps_nominal;
    out->edge_steps_executed = (int64_t)tot.steps_exec;
    out->band_rechecks = (int64_t)tot.band_checks;
    out->band_flips = (int64_t)tot.band_flips;
    out->pairs_certified = (int64_t)(tot.cert_far + tot.cert_dir);
    out->pairs_tested = (int64_t)tot.full_tests;
    out->band_overflow_items = (int64_t)tot.ovf_count;
    if (tot.flags & GPRM_DEVFLAG_BAD_EDGE)
        return fail(h, GPRM_ERR_DEVICE, "a device-pointer request held a non-finite or oversized edge");
    return GPRM_OK;
}

int gprm_indicator_batch(gprm_space* h, const float* q, int* res, int n, int offset)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!q || !res)) || offset < n) return fail(h, GPRM_ERR_ARG, "bad q/res/n/offset (offset must be >= n)");
    int slot;
    rc = submit_host(h, 0, q, nullptr, res, n, offset, &slot);
    if (rc) return rc;
    return complete_host(h, slot);
}

int gprm_indicator(gprm_space* h, const float* q, int* code)
{
    if (!q || !code) return fail(h, GPRM_ERR_ARG, "null argument");
    return gprm_indicator_batch(h, q, code, 1, 1);
}

int gprm_indicator2_async(gprm_space* h, const float* qs, const float* qe, int* res, int n, int offset, int* request)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!request || n < 0 || (n > 0 && (!qs || !qe || !res)) || offset < n)
        return fail(h, GPRM_ERR_ARG, "bad qs/qe/res/n/offset/request (offset must be >= n)");
    /* N <= nbuf (robotconfigspace.cpp:618-619) */
    if (h->nbuf > 0 && n > h->nbuf) return fail(h, GPRM_ERR_ARG, "N=%d exceeds nbuf=%d", n, h->nbuf);
    int slot;
    rc = submit_host(h, 1, qs, qe, res, n, offset, &slot);
    if (rc) return rc;
    int id = ++h->next_id;
    h->live[id] = slot;
    *request = id;
    return GPRM_OK;
}

int gprm_indicator2_wait(gprm_space* h, int request)
{
    int rc = check_ready(h);
    if (rc) return rc;
    auto it = h->live.find(request);
    if (it == h->live.end()) return fail(h, GPRM_ERR_REQUEST, "unknown request %d", request);
    int slot = it->second;
    h->live.erase(it);
    return complete_host(h, slot);
}

int gprm_indicator2(gprm_space* h, const float* qs, const float* qe, int* res, int n, int offset)
{
    int req;
    int rc = gprm_indicator2_async(h, qs, qe, res, n, offset, &req);
    if (rc) return rc;
    return gprm_indicator2_wait(h, req);
}

int gprm_indicator2_compressed(gprm_space* h, const float* qs, int M, const float* qe, int* res, const int* posqe,
                               const int* numqe, int offset)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (M < 0 || offset < 0 || (M > 0 && (!qs || !qe || !res || !posqe || !numqe)))
        return fail(h, GPRM_ERR_ARG, "bad qs/qe/res/posqe/numqe/M/offset");
    long long n = 0;
    for (int k = 0; k < M; ++k) {
        if (posqe[k] < 0 || numqe[k] < 0 || (long long)posqe[k] + numqe[k] > (long long)offset)
            return fail(h, GPRM_ERR_ARG, "range %d: posqe %d, numqe %d outside the %d end configurations", k,
                        posqe[k], numqe[k], offset);
        n += numqe[k];
    }
    if (n == 0) return GPRM_OK;
    if (n > (long long)INT_MAX) return fail(h, GPRM_ERR_ARG, "%lld edges exceed %d", n, INT_MAX);
    /* the pairs as a plain edge batch (SoA, offset n), in (k, l) order */
    const int nd = h->ndof;
    std::vector<float> a((size_t)n * nd), b((size_t)n * nd);
    std::vector<int> out((size_t)n), dst((size_t)n);
    size_t e = 0;
    for (int k = 0; k < M; ++k)
        for (int l = posqe[k]; l < posqe[k] + numqe[k]; ++l, ++e) {
            for (int j = 0; j < nd; ++j) {
                a[e + (size_t)n * j] = qs[k + (size_t)M * j];
                b[e + (size_t)n * j] = qe[l + (size_t)offset * j];
            }
            dst[e] = l;
        }
    rc = gprm_indicator2(h, a.data(), b.data(), out.data(), (int)n, (int)n);
    if (rc) return rc;
    for (size_t i = 0; i < (size_t)n; ++i) res[dst[i]] = out[i];   /* later ranges overwrite earlier ones */
    return GPRM_OK;
}

int gprm_check_boundaries(gprm_space* h, const float* q, int* res, int n, int offset)
{
    if (!h || (n > 0 && (!q || !res)) || n < 0 || offset < n) return fail(h, GPRM_ERR_ARG, "bad arguments");
    for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int j = 0; j < h->ndof; ++j) {
            float qi = q[i + (size_t)offset * j];
            if (qi < h->mins[j] || qi > h->maxs[j]) { r = 1; break; }
        }
        res[i] = r;
    }
    return GPRM_OK;
}

int gprm_check_boundaries1(gprm_space* h, const float* q, int* out)
{
    if (!h || !q || !out) return fail(h, GPRM_ERR_ARG, "null argument");
    return gprm_check_boundaries(h, q, out, 1, 1);
}

float gprm_min(const gprm_space* h, int i) { return (h && i >= 0 && i < h->ndof) ? h->mins[i] : NAN; }
float gprm_max(const gprm_space* h, int i) { return (h && i >= 0 && i < h->ndof) ? h->maxs[i] : NAN; }
float gprm_deltaq(const gprm_space* h) { return h ? h->dq : NAN; }
int gprm_dim(const gprm_space* h) { return h ? h->ndof : GPRM_ERR_ARG; }

int gprm_indicator_batch_device(gprm_space* h, const float* q, int* res, int n, int offset, void* stream)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!q || !res)) || offset < n) return fail(h, GPRM_ERR_ARG, "bad q/res/n/offset");
    if (n == 0) return GPRM_OK;
    rc = ensure_request(h, h->dev, 0, (size_t)n, false, false);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    h->host_stats.vertex_checks += n;
    return enqueue(h, h->dev, 0, q, nullptr, res, n, offset, st);
}

int gprm_indicator2_device(gprm_space* h, const float* qs, const float* qe, int* res, int n, int offset, void* stream)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!qs || !qe || !res)) || offset < n) return fail(h, GPRM_ERR_ARG, "bad qs/qe/res/n/offset");
    if (n == 0) return GPRM_OK;
    rc = ensure_request(h, h->dev, 1, (size_t)n, false, false);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    return enqueue(h, h->dev, 1, qs, qe, res, n, offset, st);
}

/* ---- diagnostics ------------------------------------------------------ */

int gprm_debug_fk(gprm_space* h, const float* q, float* out)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!q || !out) return fail(h, GPRM_ERR_ARG, "null argument");
    float* d = nullptr;
    size_t nf = (size_t)(h->ndof + 1) * 12;
    CUDA_TRY(h, dev_malloc((void**)&d, (nf + 8) * sizeof(float)));
    cudaMemcpy(d + nf, q, h->ndof * sizeof(float), cudaMemcpyHostToDevice);
    cudaError_t e = launch_fk_probe(h->dsc, d + nf, d, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, nf * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(h, GPRM_ERR_CUDA, "fk probe: %s", cudaGetErrorString(e));
    return GPRM_OK;
}

int gprm_device_sm_count(const gprm_space* h) { return h ? h->sms : 0; }

void gprm_debug_fail_device_alloc(long long nth)
{
    g_fail_alloc.store(nth > 0 ? nth : 0);
}

int gprm_debug_set_queue_capacity(gprm_space* h, unsigned capacity)
{
    if (!h) return GPRM_ERR_ARG;
    h->debug_qcap = capacity;
    return GPRM_OK;
}

int gprm_debug_support_candidates(const gprm_space* h, int polytope, int bin, int* idx, int cap)
{
    if (!h || polytope < 0 || polytope >= h->npoly || bin < 0 || bin >= GPRM_START_BINS || (cap > 0 && !idx))
        return GPRM_ERR_ARG;
    const unsigned hb = h->cbin[(size_t)GPRM_START_BINS * polytope + bin];
    const int n = (int)(hb & 255u);
    for (int i = 0; i < n && i < cap; ++i) idx[i] = h->cidx[(hb >> 8) + i];
    return n;
}

int gprm_set_launch(gprm_space* h, int vertex_kernel, int threads, int scene_in_smem)
{
    return gprm_set_launch_shape(h, vertex_kernel, threads, scene_in_smem, 0);
}

int gprm_set_launch_shape(gprm_space* h, int vertex_kernel, int threads, int scene_in_smem, int blocks_per_sm)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (threads < 32 || threads > 512 || threads % 32) return fail(h, GPRM_ERR_ARG, "threads must be 32..512, a multiple of 32");
    if (blocks_per_sm < 0 || blocks_per_sm > 64) return fail(h, GPRM_ERR_ARG, "blocks_per_sm must be 0..64");
    LaunchCfg c{};
    cudaError_t e = configure_launch(h->dsc, vertex_kernel ? 1 : 0, threads, scene_in_smem ? 1 : 0, &c, blocks_per_sm);
    if (e != cudaSuccess) {
        cudaGetLastError();
        /* restore the attribute of the current shape */
        LaunchCfg& cur = vertex_kernel ? h->cfg_v : h->cfg_e;
        configure_launch(h->dsc, vertex_kernel ? 1 : 0, cur.threads, cur.scene_in_smem, &cur,
                         cur.carveout < 0 ? 0 : cur.blocks_per_sm);
        return fail(h, GPRM_ERR_UNSUPPORTED, "launch shape %d threads / scene_in_smem=%d does not fit: %s",
                    threads, scene_in_smem, cudaGetErrorString(e));
    }
    (vertex_kernel ? h->cfg_v : h->cfg_e) = c;
    return GPRM_OK;
}

int gprm_get_launch(const gprm_space* h, int vertex_kernel, int* threads, int* scene_in_smem, int* warps_per_sm)
{
    if (!h || !threads || !scene_in_smem || !warps_per_sm) return GPRM_ERR_ARG;
    if (!h->inited) return GPRM_ERR_STATE;
    const LaunchCfg& c = vertex_kernel ? h->cfg_v : h->cfg_e;
    *threads = c.threads;
    *scene_in_smem = c.scene_in_smem;
    *warps_per_sm = c.warps_per_sm;
    return GPRM_OK;
}

int gprm_profile_enable(gprm_space* h, int on)
{
    int rc = check_ready(h);
    if (rc) return rc;
    CUDA_TRY(h, cudaDeviceSynchronize());
    h->profiling = on != 0;
    h->ev32_used = h->ev64_used = 0;
    return GPRM_OK;
}

int gprm_profile_read(gprm_space* h, double* fp32_ms, double* fp64_ms, int64_t* fp32_launches)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!fp32_ms || !fp64_ms || !fp32_launches) return fail(h, GPRM_ERR_ARG, "null argument");
    CUDA_TRY(h, cudaDeviceSynchronize());
    double t32 = 0, t64 = 0;
    for (size_t i = 0; i + 1 < h->ev32_used; i += 2) {
        float ms = 0;
        CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev32[i], h->ev32[i + 1]));
        t32 += ms;
    }
    for (size_t i = 0; i + 1 < h->ev64_used; i += 2) {
        float ms = 0;
        CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev64[i], h->ev64[i + 1]));
        t64 += ms;
    }
    *fp32_ms = t32;
    *fp64_ms = t64;
    *fp32_launches = (int64_t)(h->ev32_used / 2);
    return GPRM_OK;
}

int gprm_measure_fp32_peak(double* tflops)
{
    if (!tflops) return GPRM_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GPRM_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* out = nullptr;
    if (dev_malloc((void**)&out, sizeof(float) * 1024 * 1024) != cudaSuccess) return GPRM_ERR_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    gprm::launch_fma_probe(blocks, threads, iters, out, 0);   /* warm-up */
    cudaEventRecord(a, 0);
    gprm::launch_fma_probe(blocks, threads, iters, out, 0);
    cudaEventRecord(b, 0);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0) return GPRM_ERR_CUDA;
    double flops = 2.0 * (double)blocks * threads * iters * GPRM_FMA_PROBE_CHAINS;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return GPRM_OK;
}

}  /* extern "C" */

/* ====================================================================== */
/* vertex checks without allocation                                        */
/* ====================================================================== */

namespace {

/* Work buffers of gprm_indicator_batch_device_noalloc: the control block
 * (zeroed by every call) at offset 0, the FP64 queue (at most one entry per
 * configuration, so it cannot overflow) at NOALLOC_QUEUE_OFFSET.  The name is
 * a host-side stand-in; kernels get the device address looked up below. */
constexpr size_t NOALLOC_QUEUE_OFFSET = 256;
static_assert(sizeof(Control) <= NOALLOC_QUEUE_OFFSET, "control block outgrew its slot");
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_QUEUE_OFFSET +
                                                                 (size_t)GPRM_NOALLOC_MAX_CONFIGS * sizeof(uint2)];

/* Device address of the scratch array in the current context, looked up
 * on every call (a lookup, no allocation once the module is loaded), so that
 * a context made again after a device reset gets the array's new address. */
int noalloc_scratch(gprm_space* h, unsigned char** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(h, GPRM_ERR_CUDA, "cudaGetSymbolAddress(no-allocation scratch): %s", cudaGetErrorString(e));
    *out = (unsigned char*)p;
    return GPRM_OK;
}

}  // namespace

extern "C" int gprm_indicator_batch_device_noalloc(gprm_space* h, const float* q, int* res, int n, int offset,
                                                   void* stream)
{
    int rc = check_ready(h);   /* makes the handle's device current */
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!q || !res)) || offset < n) return fail(h, GPRM_ERR_ARG, "bad q/res/n/offset");
    if (n > GPRM_NOALLOC_MAX_CONFIGS)
        return fail(h, GPRM_ERR_ARG, "n=%d exceeds the no-allocation limit of %d configurations per call",
                    n, GPRM_NOALLOC_MAX_CONFIGS);
    if (n == 0) return GPRM_OK;
    unsigned char* base = nullptr;
    rc = noalloc_scratch(h, &base);
    if (rc) return rc;
    Control* ctl = (Control*)base;
    /* one queue entry per configuration: the queue cannot overflow */
    BandQueue bq;
    bq.items = (uint2*)(base + NOALLOC_QUEUE_OFFSET);
    bq.cap = (unsigned)GPRM_NOALLOC_MAX_CONFIGS;
    bq.ovf = nullptr;
    bq.n = n;
    cudaStream_t st = (cudaStream_t)stream;
    const int band_on = (h->mode & GPRM_MODE_FP64_BAND) != 0;
    CUDA_TRY(h, cudaMemsetAsync(ctl, 0, sizeof(Control), st));
    CUDA_TRY(h, launch_check_configs(h->dsc, h->cfg_v, q, n, offset, res, band_on, h->band, bq, ctl, st));
    if (band_on)
        CUDA_TRY(h, launch_recheck(h->dsc, h->sms * 4, 0, q, nullptr, nullptr, offset, h->dq, h->policy, res,
                                   nullptr, bq, ctl, st));
    CUDA_TRY(h, launch_accumulate(ctl, h->d_total, st));
    h->host_stats.vertex_checks += n;
    h->host_stats.launches += 2 + (band_on ? 1 : 0);
    return GPRM_OK;
}

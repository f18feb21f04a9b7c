/*
 * gprm_mlp.cu - the learned collision-probability predictor.
 *
 * No counterpart in GPUPRM.  A multilayer perceptron
 *     x (sin/cos of the joints, padded to 16) -> 256 -> 256 -> 256 -> 256 -> 1
 * with GELU (tanh form) on the hidden
 * layers and a sigmoid output, trained
 * with binary cross-entropy and Adam.  Weights are kept in FP32 (master)
 * and BF16 (the GEMM operands); activations are stored in BF16; every GEMM
 * accumulates in FP32 on the tensor cores (warp-level BF16 MMA, m16n8k16).
 *
 * Layout (row-major): W_l is [out x in] like a Linear layer; activations
 * are [batch x features].  Forward:  Z_l = H_{l-1} W_l^T + b_l,
 * H_l = gelu(Z_l).  Backward:  dZ_l = dH_l * gelu'(Z_l),
 * dW_l = dZ_l^T H_{l-1},  db_l = colsum(dZ_l),  dH_{l-1} = dZ_l W_l.
 */
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/gprm_b200.h"

namespace {

constexpr int IN_PAD = 16;     /* input features padded to one MMA k-step */
constexpr int HID = 256;
constexpr int NLAYER = 4;      /* hidden layers */

/* ------------------------------------------------------------------ */
/* GEMM: C[M x N] = sum_k A(m,k) B(k,n), BF16 in, FP32 accumulate        */
/*   A(m,k) = TA ? A[k*lda + m] : A[m*lda + k]                            */
/*   B(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n]                            */
/* 64x64 block tile, 32-deep k tile, 4 warps of 32x32, mma m16n8k16.     */
/* ------------------------------------------------------------------ */

constexpr int BM = 64, BN = 64, BK = 32, KPAD = 8;

enum Epi {
    EPI_FWD_HIDDEN = 0,   /* Z = acc + bias (fp32 out), H = gelu(Z) (bf16 out) */
    EPI_BWD_DH = 1,       /* dZ = acc * gelu'(Z) (bf16 out) */
    EPI_GRAD_W = 2        /* dW = acc (fp32 out) */
};

struct EpiArgs {
    const float* bias;        /* [N] (FWD) */
    float* zout;              /* [M x N] fp32 (FWD) */
    __nv_bfloat16* hout;      /* [M x N] bf16 (FWD: H, BWD: dZ) */
    const float* zin;         /* [M x N] fp32 pre-activation (BWD) */
    float* gout;              /* [M x N] fp32 (GRAD) */
    int ldc;
};

/* GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear
 * Units", 2016, sec. 2):
 *     GELU(z) = z/2 (1 + tanh(u)),   u = k (z + c z^3),  k = sqrt(2/pi), c = 0.044715,
 * evaluated as u = z (k + kc z^2), GELU = hz + hz t with hz = z/2, t = tanh(u).
 * The one special-function instruction is tanh.approx.f32 (relative error
 * about 2^-11, below the BF16 rounding of the activations it feeds); the
 * network is trained and evaluated with this same function, and the FP64
 * oracle states it with an exact tanh.  Derivative:
 *     GELU'(z) = (1 + t)/2 + hz (1 - t^2) k (1 + 3 c z^2). */
constexpr float GELU_K = 0.7978845608028654f;              /* sqrt(2/pi) */
constexpr float GELU_KC = 0.035677408136300125f;           /* sqrt(2/pi) * 0.044715 */
constexpr float GELU_3KC = 0.10703222440890038f;           /* 3 sqrt(2/pi) * 0.044715 */

__device__ __forceinline__ float tanh_approx(float x)
{
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float gelu_f(float z)
{
    const float u = __fmul_rn(z, __fmaf_rn(__fmul_rn(z, z), GELU_KC, GELU_K));
    const float t = tanh_approx(u);
    const float hz = __fmul_rn(z, 0.5f);
    return __fmaf_rn(hz, t, hz);
}

/* Two lanes of FP32 in one 64-bit register for the packed FP32 x2
 * instructions of sm_100 (each half rounded exactly like the scalar
 * instruction, so results equal gelu_f's bit for bit). */
__device__ __forceinline__ unsigned long long f2_pack(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b, unsigned long long c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

/* gelu_f of (2 y0, 2 y1) from (y0, y1) = z/2, which k_mlp_fused's MMAs
 * produce (weights and bias halved, exactly): u = y (2k + 8kc y^2) and
 * GELU = y + y t.  Scaling by powers of two commutes with rounding, so each
 * step equals gelu_f's on z = 2y bit for bit, with one multiply fewer. */
__device__ __forceinline__ void gelu_half_f2(unsigned long long y, float& g0, float& g1)
{
    const unsigned long long w = f2_fma(f2_mul(y, y), f2_pack(8.0f * GELU_KC, 8.0f * GELU_KC),
                                        f2_pack(2.0f * GELU_K, 2.0f * GELU_K));
    float u0, u1;
    f2_unpack(f2_mul(y, w), u0, u1);
    const unsigned long long t = f2_pack(tanh_approx(u0), tanh_approx(u1));
    f2_unpack(f2_fma(y, t, y), g0, g1);
}

__device__ __forceinline__ float gelu_grad(float z)
{
    const float z2 = __fmul_rn(z, z);
    const float t = tanh_approx(__fmul_rn(z, __fmaf_rn(z2, GELU_KC, GELU_K)));
    const float du = __fmaf_rn(z2, GELU_3KC, GELU_K);                 /* k (1 + 3 c z^2) */
    const float hz = __fmul_rn(z, 0.5f);
    const float s = __fmaf_rn(-t, t, 1.0f);                           /* 1 - t^2 */
    return __fmaf_rn(__fmul_rn(hz, s), du, __fmaf_rn(0.5f, t, 0.5f));
}

/* two floats -> a packed BF16 pair (a in the low half), round to nearest
 * even like __float2bfloat16; kept in registers (no local arrays) */
__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    uint32_t u;
    memcpy(&u, &h, sizeof(u));
    return u;
}
__device__ __forceinline__ float bf16_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                              const __nv_bfloat16* __restrict__ B, int ldb, EpiArgs ep)
{
    __shared__ __align__(16) __nv_bfloat16 As[BM][BK + KPAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + KPAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, t = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    for (int k0 = 0; k0 < K; k0 += BK) {
        /* stage the tiles, k contiguous in shared memory */
        for (int idx = tid; idx < BM * BK; idx += 128) {
            int mm, kk;
            if (TA) { mm = idx % BM; kk = idx / BM; }   /* global m contiguous */
            else { kk = idx % BK; mm = idx / BK; }       /* global k contiguous */
            int gm = m0 + mm, gk = k0 + kk;
            __nv_bfloat16 v = zero;
            if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[mm][kk] = v;
        }
        for (int idx = tid; idx < BN * BK; idx += 128) {
            int nn, kk;
            if (TB) { kk = idx % BK; nn = idx / BK; }   /* global k contiguous */
            else { nn = idx % BN; kk = idx / BN; }       /* global n contiguous */
            int gn = n0 + nn, gk = k0 + kk;
            __nv_bfloat16 v = zero;
            if (gn < N && gk < K) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            Bs[nn][kk] = v;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t af[2][4], bfr[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + g;
                af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * t]);
                af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * t]);
                af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * t + 8]);
                af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * t + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn + j * 8 + g;
                bfr[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * t]);
                bfr[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * t + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
        }
        __syncthreads();
    }
    /* epilogue: accumulator element (row g / g+8, cols 2t, 2t+1) */
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int gm = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
                const int gn = n0 + wn + j * 8 + 2 * t + (r & 1);
                if (gm >= M || gn >= N) continue;
                const size_t o = (size_t)gm * ep.ldc + gn;
                const float a = acc[i][j][r];
                if (EPI == EPI_FWD_HIDDEN) {
                    const float z = a + ep.bias[gn];
                    ep.zout[o] = z;
                    ep.hout[o] = __float2bfloat16(gelu_f(z));
                } else if (EPI == EPI_BWD_DH) {
                    ep.hout[o] = __float2bfloat16(a * gelu_grad(ep.zin[o]));
                } else {
                    ep.gout[o] = a;
                }
            }
}

/* ------------------------------------------------------------------ */
/* small kernels                                                        */
/* ------------------------------------------------------------------ */

/* features: (sin q_j, cos q_j) for j < ndof, zero padded to IN_PAD;
 * q is SoA q[i + offset*j]; rows are optionally gathered through idx */
__global__ void k_features(const float* __restrict__ q, long long offset, int ndof, int n,
                           const int* __restrict__ idx, const long long* __restrict__ idx_off,
                           __nv_bfloat16* __restrict__ X)
{
    const long long io = idx_off ? *idx_off : 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const long long src = idx ? idx[io + i] : i;
        __nv_bfloat16* row = X + (size_t)i * IN_PAD;
        for (int j = 0; j < IN_PAD / 2; ++j) {
            float s = 0.0f, c = 0.0f;
            if (j < ndof) sincosf(q[src + offset * j], &s, &c);
            row[2 * j] = __float2bfloat16(j < ndof ? s : 0.0f);
            row[2 * j + 1] = __float2bfloat16(j < ndof ? c : 0.0f);
        }
    }
}

/* output layer (256 -> 1) and the loss: one warp per row.
 * p = sigmoid(H4 . w5 + b5); with labels: loss += BCE, dlogit = (p - y)/B */
__global__ void k_out(int n, const __nv_bfloat16* __restrict__ H, const __nv_bfloat16* __restrict__ w5,
                      const float* __restrict__ b5, float* __restrict__ p, const float* __restrict__ y,
                      const int* __restrict__ yidx, const long long* __restrict__ idx_off, float* __restrict__ dlogit,
                      float* __restrict__ loss, float inv_b)
{
    const long long io = idx_off ? *idx_off : 0;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < n; r += nw) {
        float s = 0.0f;
        for (int k = lane; k < HID; k += 32)
            s += __bfloat162float(H[(size_t)r * HID + k]) * __bfloat162float(w5[k]);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const float logit = s + b5[0];
            const float pr = 1.0f / (1.0f + expf(-logit));
            if (p) p[r] = pr;
            if (y) {
                const float yy = y[yidx ? yidx[io + r] : r];
                /* BCE with logits, stable form */
                const float l = fmaxf(logit, 0.0f) - logit * yy + log1pf(expf(-fabsf(logit)));
                atomicAdd(loss, l * inv_b);
                dlogit[r] = (pr - yy) * inv_b;
            }
        }
    }
}

/* output-layer backward: dZ4 = (dlogit w5) * gelu'(Z4), and per block the
 * partial sums of dw5 = H4^T dlogit (part[b][0..HID)) and db5 = sum dlogit
 * (part[b][HID]) over the rows r = b (mod gridDim.x); the partials are
 * added in block order afterwards, so the gradients do not depend on
 * scheduling. */
__global__ void k_out_back(int n, const __nv_bfloat16* __restrict__ H, const float* __restrict__ Z,
                           const __nv_bfloat16* __restrict__ w5, const float* __restrict__ dlogit,
                           float* __restrict__ part, __nv_bfloat16* __restrict__ dZ)
{
    /* column k = threadIdx.x (HID threads) */
    const int k = threadIdx.x;
    float acc = 0.0f, accb = 0.0f;
    for (int r = blockIdx.x; r < n; r += gridDim.x) {
        const float d = dlogit[r];
        acc += d * __bfloat162float(H[(size_t)r * HID + k]);
        accb += d;
        dZ[(size_t)r * HID + k] = __float2bfloat16(d * __bfloat162float(w5[k]) * gelu_grad(Z[(size_t)r * HID + k]));
    }
    part[(size_t)blockIdx.x * (HID + 1) + k] = acc;
    if (k == 0) part[(size_t)blockIdx.x * (HID + 1) + HID] = accb;
}

/* per-block partial column sums: part[b][c] = sum over rows r = b (mod
 * gridDim.x) of dZ[r][c] */
__global__ void k_colsum(int n, int cols, const __nv_bfloat16* __restrict__ dZ, float* __restrict__ part)
{
    const int c = threadIdx.x;
    if (c >= cols) return;
    float acc = 0.0f;
    for (int r = blockIdx.x; r < n; r += gridDim.x) acc += __bfloat162float(dZ[(size_t)r * cols + c]);
    part[(size_t)blockIdx.x * cols + c] = acc;
}

/* out[c] = sum over b < parts of part[b][c], in b order */
__global__ void k_reduce_parts(int parts, int cols, const float* __restrict__ part, float* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float acc = 0.0f;
    for (int b = 0; b < parts; ++b) acc += part[(size_t)b * cols + c];
    out[c] = acc;
}

/* Adam on the FP32 master parameters, refreshing their BF16 copies.
 * bf_map[i] = index into the bf16 array or -1. */
__global__ void k_adam(long long n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, const int* __restrict__ bf_map, __nv_bfloat16* __restrict__ wbf,
                       float lr, float b1, float b2, float eps, const long long* __restrict__ t_base, long long t_step)
{
    /* step t = (*t_base) + t_step: read on the device so that one captured
       training epoch serves every epoch */
    const double t = (double)((t_base ? *t_base : 0) + t_step);
    const float c1 = (float)(1.0 - pow(0.9, t)), c2 = (float)(1.0 - pow(0.999, t));
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        const int b = bf_map[i];
        if (b >= 0) wbf[b] = __float2bfloat16(wi);
    }
}

__global__ void k_to_bf16(long long n, const float* __restrict__ w, const int* __restrict__ bf_map,
                          __nv_bfloat16* __restrict__ wbf)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = bf_map[i];
        if (b >= 0) wbf[b] = __float2bfloat16(w[i]);
    }
}


/* ------------------------------------------------------------------ */
/* inference layers on the 5th-generation tensor cores (tcgen05)         */
/* ------------------------------------------------------------------ */
/*
 * One persistent CTA per SM (256 threads) holds a layer's weights W
 * [256 x K] in shared memory and runs 128-row tiles through it:
 *   1. all threads stage the tile's inputs A [128 x K] in shared memory
 *      (for the first layer: sin/cos features computed on the fly);
 *   2. one thread issues K/16 tcgen05.mma (M=128, N=256, K=16, BF16 in,
 *      FP32 accumulate) into a 256-column TMEM accumulator and commits
 *      them to an mbarrier;
 *   3. the eight warps read the accumulator back (tcgen05.ld, warp w owns
 *      TMEM lanes 32*(w%4).. and columns 128*(w/4)..), add the bias,
 *      apply GELU and store BF16 activations - or, for the last hidden
 *      layer, reduce them against the output weights to P(collision).
 * Operands use the no-swizzle K-major layout of 8-row x 16-byte core
 * matrices: byte offset of (row r, k) = (r/8)*SBO + (k/8)*128 + (r%8)*16 +
 * (k%8)*2 with SBO = 16*K, LBO = 128.  Waits on the mbarrier are bounded;
 * on expiry the kernel sets *err, stops, and frees its TMEM.
 */
constexpr int TC_ROWS = 128;
constexpr int TC_COLS = HID;                 /* 256 accumulator columns */
constexpr long long TC_WAIT_LIMIT = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

/* shared-memory matrix descriptor: no swizzle, K-major (version 1) */
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

/* shared-memory matrix descriptor: 128-byte swizzle, K-major (version 1):
 * 8-row x 128-byte atoms (64 BF16 of K), 1024 bytes apart along M/N
 * (SBO); the leading offset is unused for swizzled K-major operands and
 * set to 16 bytes. */
__device__ __forceinline__ uint64_t tc_sdesc_sw128(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

/* instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, M=128, N=256 */
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_COLS >> 3) << 17) |
                              ((uint32_t)(TC_ROWS >> 4) << 24);

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase)
{
    for (long long i = 0; i < TC_WAIT_LIMIT; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(done) : "r"(mbar), "r"(phase) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                   "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                   "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

/* A 16-column TMEM load in two halves, so that a load can be in flight
 * while the previous columns are processed: the issue, then the wait, which
 * names the destination registers so that no use of them moves above it. */
__device__ __forceinline__ void tc_ld16_issue(uint32_t taddr, uint32_t* r)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_ld16_wait(uint32_t* r)
{
    asm volatile("tcgen05.wait::ld.sync.aligned;\n"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                   "+r"(r[14]), "+r"(r[15])
                 :: "memory");
}

/* Stores 16 FP32 columns of this warp's 32 TMEM lanes, all lanes the same
 * 16 values (a bias row), and waits for the stores. */
__device__ __forceinline__ void tc_st16_bias(uint32_t taddr, const float* b)
{
    const float4 b0 = reinterpret_cast<const float4*>(b)[0], b1 = reinterpret_cast<const float4*>(b)[1];
    const float4 b2 = reinterpret_cast<const float4*>(b)[2], b3 = reinterpret_cast<const float4*>(b)[3];
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
                 "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n"
                 :: "r"(taddr), "f"(b0.x), "f"(b0.y), "f"(b0.z), "f"(b0.w), "f"(b1.x), "f"(b1.y), "f"(b1.z), "f"(b1.w),
                    "f"(b2.x), "f"(b2.y), "f"(b2.z), "f"(b2.w), "f"(b3.x), "f"(b3.y), "f"(b3.z), "f"(b3.w)
                 : "memory");
}
__device__ __forceinline__ void tc_st_wait()
{
    asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
}

/* shared memory of k_mlp_tc<K>: W | A | mbarrier | TMEM address | row partials */
template <int K>
struct TcSmem {
    static constexpr size_t W = (size_t)HID * K * 2;
    static constexpr size_t A = (size_t)TC_ROWS * K * 2;
    static constexpr size_t MBAR = W + A;
    static constexpr size_t TADDR = MBAR + 8;
    static constexpr size_t RED = TADDR + 8;                       /* 4 x 128 floats */
    static constexpr size_t BYTES = RED + 4 * TC_ROWS * 4;
    /* at least half of the SM's shared memory: one CTA per SM, so that the
       256 TMEM columns this CTA allocates are always available */
    static constexpr size_t LAUNCH = BYTES > 120 * 1024 ? BYTES : 120 * 1024;
};

template <int K, bool FEAT, bool LAST>
__global__ void __launch_bounds__(256, 1)
k_mlp_tc(int n, const float* __restrict__ q, long long qoff, int ndof, const __nv_bfloat16* __restrict__ Hin,
         const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias, __nv_bfloat16* __restrict__ Hout,
         const __nv_bfloat16* __restrict__ w5, const float* __restrict__ b5, float* __restrict__ p,
         unsigned* err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    using L = TcSmem<K>;
    constexpr uint32_t SBO = 16u * K, LBO = 128u;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* Ws = sm;
    unsigned char* As = sm + L::W;
    const uint32_t mbar = smem_u32(sm + L::MBAR);
    uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(sm + L::TADDR);
    float* red = reinterpret_cast<float*>(sm + L::RED);

    /* weights -> shared memory, core-matrix layout */
    for (int idx = tid; idx < HID * (K / 8); idx += blockDim.x) {
        const int nrow = idx % HID, c = idx / HID;
        const uint4 v = *reinterpret_cast<const uint4*>(W + (size_t)nrow * K + c * 8);
        *reinterpret_cast<uint4*>(Ws + (nrow / 8) * SBO + c * LBO + (nrow % 8) * 16) = v;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(smem_u32(taddr_slot)), "r"(TC_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *taddr_slot;
    const int ntiles = (n + TC_ROWS - 1) / TC_ROWS;
    uint32_t phase = 0;
    bool failed = false;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int row0 = tile * TC_ROWS;
        /* 1. inputs of the tile -> shared memory */
        if (FEAT) {
            if (tid < TC_ROWS) {
                const int r = row0 + tid;
                uint32_t x[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float sv = 0.0f, cv = 0.0f;
                    if (j < ndof && r < n) sincosf(q[r + qoff * j], &sv, &cv);
                    x[j] = pack_bf16(j < ndof ? sv : 0.0f, j < ndof ? cv : 0.0f);
                }
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    *reinterpret_cast<uint4*>(As + (tid / 8) * SBO + c * LBO + (tid % 8) * 16) =
                        make_uint4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
            }
        } else {
            for (int idx = tid; idx < TC_ROWS * (K / 8); idx += blockDim.x) {
                const int r = idx % TC_ROWS, c = idx / TC_ROWS;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (row0 + r < n) v = *reinterpret_cast<const uint4*>(Hin + (size_t)(row0 + r) * K + c * 8);
                *reinterpret_cast<uint4*>(As + (r / 8) * SBO + c * LBO + (r % 8) * 16) = v;
            }
        }
        /* the accumulator starts at the bias: warp w writes its 32 lanes,
           columns 128 (w / 4) .. +127 */
#pragma unroll 1
        for (int c = 0; c < 8; ++c)
            tc_st16_bias(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 * (warp >> 2) + 16 * c),
                         bias + 128 * (warp >> 2) + 16 * c);
        tc_st_wait();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        /* 2. the MMAs, accumulating onto the bias */
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t a0 = smem_u32(As), b0 = smem_u32(Ws);
#pragma unroll
            for (int s = 0; s < K / 16; ++s) {
                const uint64_t ad = tc_sdesc(a0 + s * 2 * LBO, LBO, SBO);
                const uint64_t bd = tc_sdesc(b0 + s * 2 * LBO, LBO, SBO);
                const uint32_t acc = 1u;
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                             :: "r"(tmem), "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc),
                                "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         :: "r"(mbar) : "memory");
        }
        /* 3. accumulator (bias included) -> GELU -> out */
        const bool ok = tc_wait(mbar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(err, 1u);
            failed = true;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int rl = 32 * (warp & 3) + lane;          /* this thread's row in the tile */
        const int r = row0 + rl;
        /* warp half h owns columns 64r + 32h .. 64r + 32h + 31 (r = 0..3);
           the output head sums columns 64r + 16q .. 64r + 16q + 15 over r
           into partial q and adds the partials as ((0 + 1) + (2 + 3)), the
           same split and order as the fused kernel */
        const int h = warp >> 2;
        float part[2] = {0.0f, 0.0f};
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            const int col = 64 * cc + 32 * h;
            float v[32];
            tc_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col, v);
            uint32_t hp[16];
#pragma unroll
            for (int j = 0; j < 16; ++j)
                hp[j] = pack_bf16(gelu_f(v[2 * j]), gelu_f(v[2 * j + 1]));
            if (LAST) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    part[j >> 3] = __fmaf_rn(bf16_lo(hp[j]), __bfloat162float(w5[col + 2 * j]), part[j >> 3]);
                    part[j >> 3] = __fmaf_rn(bf16_hi(hp[j]), __bfloat162float(w5[col + 2 * j + 1]), part[j >> 3]);
                }
            } else if (r < n) {
#pragma unroll
                for (int c4 = 0; c4 < 4; ++c4)
                    *reinterpret_cast<uint4*>(Hout + (size_t)r * HID + col + 8 * c4) =
                        make_uint4(hp[4 * c4], hp[4 * c4 + 1], hp[4 * c4 + 2], hp[4 * c4 + 3]);
            }
        }
        if (LAST) {
            red[(2 * h) * TC_ROWS + rl] = part[0];
            red[(2 * h + 1) * TC_ROWS + rl] = part[1];
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        if (LAST && tid < TC_ROWS && row0 + tid < n) {
            const float logit = ((red[tid] + red[TC_ROWS + tid]) + (red[2 * TC_ROWS + tid] + red[3 * TC_ROWS + tid])) + b5[0];
            p[row0 + tid] = 1.0f / (1.0f + expf(-logit));
        }
    }
    if (failed) {
        /* let an outstanding commit land before the accumulator is freed */
        tc_wait(mbar, phase ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(TC_COLS) : "memory");
}


/* ------------------------------------------------------------------ */
/* the whole network in one kernel (tcgen05, warp-specialised)          */
/* ------------------------------------------------------------------ */
/*
 * k_mlp_fused runs all layers of a 128-row tile on one SM; the hidden
 * activations never leave shared memory.  One persistent CTA per SM with
 * 22 warps in four roles:
 *   warps 0-15  epilogue: TMEM -> GELU -> BF16 activations (the
 *               next layer's A operand, written in place) or, after the
 *               last hidden layer, the output head.  Warp w reads TMEM
 *               lanes 32*(w%4).. (its rows) and, in round r = 0..3, the
 *               columns 64r + 16q .. 64r + 16q + 15, q = w/4;
 *   warp 16     loads the weights of hidden layers 2-4 in chunks of K = 64
 *               (256 x 64 BF16 = 32 KB, pre-arranged by k_mlp_relayout)
 *               with bulk copies into a 4-stage ring: a whole layer can be
 *               in flight, so the next layer's weights arrive while the
 *               epilogue works;
 *   warp 17     issues the MMAs (one thread);
 *   warps 18-21 compute the input features of the next tile.
 * The hidden layers' operands (activations and weight chunks) use the
 * 128-byte-swizzled K-major layout: 8-row x 64-element atoms of 1 KB in
 * which the 16-byte group g of row r sits at group g ^ (r % 8), so the
 * tensor core and the epilogue's row-per-thread stores read and write
 * shared memory without bank conflicts.  Layer l accumulates into TMEM
 * columns 256*(l%2)..: MMA chunk c of layer l+1 (K columns 64c..64c+63)
 * is issued as soon as the epilogue's round c of layer l has written them, so the MMAs of a layer run under the
 * epilogue of the previous one, and the first layer of the next tile runs
 * under the last layer's epilogue.  Each accumulator starts at the bias of
 * the layer that uses it (written by the epilogue warps with tcgen05.st
 * when they have read the previous layer out), so the epilogue adds no
 * bias.  Weights and biases are halved (exact in binary), so the
 * accumulators hold z/2 and the GELU needs no multiply by 1/2; every step
 * rounds like the per-layer kernels' GELU of z.  The MMAs start from the
 * bias and run in the same K order as
 * k_mlp_tc and the output head uses the same split and order, so both
 * kernels give the same bits.  Every wait is bounded by a clock budget: an
 * expired wait sets *err and an abort flag that ends the other roles'
 * waits; the CTA then waits (bounded) for its own MMAs and copies before
 * it frees TMEM and returns.
 */
constexpr unsigned FULL_MASK_MLP = 0xffffffffu;
constexpr int FU_EPI_WARPS = 16;
constexpr int FU_PRODUCER_WARP = FU_EPI_WARPS, FU_MMA_WARP = FU_EPI_WARPS + 1, FU_FEAT_WARP0 = FU_EPI_WARPS + 2;
constexpr int FU_THREADS = (FU_EPI_WARPS + 6) * 32;        /* 704 */
constexpr int FU_NS = 4;                                   /* weight ring stages */
constexpr int FU_CK = 64;                                  /* K columns per weight chunk: one swizzle atom */
constexpr int FU_CHUNK_BYTES = HID * FU_CK * 2;            /* 32 KB */
constexpr int FU_CHUNKS = HID / FU_CK;                     /* 4 chunks per hidden layer */
constexpr long long FU_WAIT_CYCLES = 1ll << 31;            /* ~1 s at the boost clock */
constexpr size_t FU_RELAYOUT_BYTES = (size_t)(NLAYER - 1) * FU_CHUNKS * FU_CHUNK_BYTES + (size_t)HID * IN_PAD * 2;

struct FuSmem {
    static constexpr size_t BUF = 0;                                   /* 64 KB activations */
    static constexpr size_t RING = BUF + (size_t)TC_ROWS * HID * 2;
    static constexpr size_t W1 = RING + (size_t)FU_NS * FU_CHUNK_BYTES;  /* 8 KB */
    static constexpr size_t FEAT = W1 + (size_t)HID * IN_PAD * 2;        /* 4 KB */
    static constexpr size_t BIAS = FEAT + (size_t)TC_ROWS * IN_PAD * 2;  /* 4 x 256 floats */
    static constexpr size_t W5 = BIAS + (size_t)NLAYER * HID * 4;        /* 256 floats */
    static constexpr size_t RED = W5 + (size_t)HID * 4;                  /* 4 x 128 floats */
    static constexpr size_t BARS = RED + 4 * (size_t)TC_ROWS * 4;
    static constexpr int NBARS = 3 * FU_NS + 9;
    static constexpr size_t TADDR = BARS + NBARS * 8;
    static constexpr size_t ABORT = TADDR + 4;
    static constexpr size_t B5 = ABORT + 4;
    static constexpr size_t BYTES = B5 + 16;
};
static_assert(FuSmem::BYTES <= 227 * 1024, "fused MLP shared memory");
static_assert(FuSmem::BARS % 8 == 0, "mbarrier alignment");
static_assert(FU_CHUNKS == FU_NS, "one hready barrier per chunk; the ring holds a layer");
static_assert(FuSmem::BUF % 1024 == 0 && FuSmem::RING % 1024 == 0, "swizzle atoms are 1024-byte aligned");

/* mbarrier indices */
enum {
    FB_WFULL = 0, FB_WEMPTY = FB_WFULL + FU_NS, FB_HREADY = FB_WEMPTY + FU_NS, FB_ACCFULL = FB_HREADY + FU_CHUNKS,
    FB_ACCEMPTY = FB_ACCFULL + 2, FB_FEATREADY = FB_ACCEMPTY + 2, FB_FEATEMPTY, FB_HEADFULL, FB_HEADEMPTY, FB_DRAIN,
    FB_COUNT
};
static_assert(FB_COUNT == FuSmem::NBARS, "barrier count");

struct FuParams {
    const float* q;
    long long qoff;
    int ndof, n;
    const unsigned char* wtc;       /* k_mlp_relayout output */
    const float* bias[NLAYER];
    const __nv_bfloat16* w5;
    const float* b5;
    float* p;
    unsigned* err;
    long long wait_cycles;          /* budget of each pipeline wait (the drains keep FU_WAIT_CYCLES) */
};

__device__ __forceinline__ void fu_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" :: "r"(bar) : "memory");
}

__device__ __forceinline__ bool fu_try(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}\n"
                 : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    return done != 0;
}

/* Waits for the phase of `parity`; false when the clock budget (cycles)
 * runs out (sets the abort flag and *err) or another role has aborted.  Roles off
 * the critical path pass a sleep between polls, so that their polling does
 * not take issue slots from the epilogue warps on the same SM sub-partition. */
__device__ __forceinline__ bool fu_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, unsigned* err,
                                        long long budget, unsigned sleep_ns = 0)
{
    const long long t0 = clock64();
    if (budget <= 0) budget = FU_WAIT_CYCLES;
    while (!fu_try(bar, parity)) {
        if (sleep_ns) __nanosleep(sleep_ns);
        if (*abort_flag) return false;
        if (clock64() - t0 > budget) {
            *abort_flag = 1;
            atomicOr(err, 1u);
            return false;
        }
    }
    return true;
}

/* The same wait without the abort flag: used while draining. */
__device__ __forceinline__ void fu_wait_drain(uint32_t bar, uint32_t parity, unsigned* err)
{
    const long long t0 = clock64();
    while (!fu_try(bar, parity)) {
        if (clock64() - t0 > FU_WAIT_CYCLES) {
            atomicOr(err, 2u);
            return;
        }
    }
}

__device__ __forceinline__ void fu_mma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 :: "r"(tmem), "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void fu_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" :: "r"(bar)
                 : "memory");
}

/* Weights of hidden layers 2-4, halved (k_mlp_fused accumulates z/2), in chunk order (layer, K chunk), each chunk
 * [256 rows x 64 K] in the 128-byte-swizzled K-major layout (row n, k at
 * (n/8)*1024 + (n%8)*128 + ((k/8) ^ (n%8))*16 + (k%8)*2), then W1
 * [256 x 16] in the no-swizzle core-matrix order (SBO 256 B, LBO 128 B). */
/* the 8 BF16 values of v times 1/2 (exact for normal values) */
__device__ __forceinline__ uint4 half_bf16x8(uint4 v)
{
    const __nv_bfloat162 h = __float2bfloat162_rn(0.5f);
    uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        __nv_bfloat162 x;
        memcpy(&x, &w[i], 4);
        x = __hmul2(x, h);
        memcpy(&w[i], &x, 4);
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

__global__ void k_mlp_relayout(const __nv_bfloat16* __restrict__ wbf, long long o0, long long o1, long long o2,
                               long long o3, unsigned char* __restrict__ out)
{
    const int per_layer = HID * (HID / 8);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (NLAYER - 1) * per_layer) {
        const int l = t / per_layer, r = t % per_layer;
        const int nrow = r % HID, kg = r / HID;   /* kg: 8-element group of K, 0..31 */
        const long long off = l == 0 ? o1 : (l == 1 ? o2 : o3);
        const uint4 v = half_bf16x8(*reinterpret_cast<const uint4*>(wbf + off + (long long)nrow * HID + kg * 8));
        unsigned char* dst = out + (size_t)(l * FU_CHUNKS + kg / 8) * FU_CHUNK_BYTES + (nrow / 8) * 1024 +
                             (nrow % 8) * 128 + (((kg % 8) ^ (nrow % 8)) * 16);
        *reinterpret_cast<uint4*>(dst) = v;
    } else if (t < (NLAYER - 1) * per_layer + HID * (IN_PAD / 8)) {
        const int r = t - (NLAYER - 1) * per_layer;
        const int nrow = r % HID, kg = r / HID;
        const uint4 v = half_bf16x8(*reinterpret_cast<const uint4*>(wbf + o0 + (long long)nrow * IN_PAD + kg * 8));
        unsigned char* dst = out + (size_t)(NLAYER - 1) * FU_CHUNKS * FU_CHUNK_BYTES + (nrow / 8) * (IN_PAD * 16) +
                             kg * 128 + (nrow % 8) * 16;
        *reinterpret_cast<uint4*>(dst) = v;
    }
}

__global__ void __launch_bounds__(FU_THREADS, 1) k_mlp_fused(FuParams P)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    using L = FuSmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bars = smem_u32(sm + L::BARS);
    auto bar = [&](int i) { return bars + 8u * (uint32_t)i; };
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::ABORT);
    uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(sm + L::TADDR);
    float* bias_s = reinterpret_cast<float*>(sm + L::BIAS);
    float* w5_s = reinterpret_cast<float*>(sm + L::W5);
    float* red = reinterpret_cast<float*>(sm + L::RED);
    const float* b5_s = reinterpret_cast<const float*>(sm + L::B5);
    const unsigned char* wtc = P.wtc;
    if (smem_u32(sm) & 1023u) {     /* the swizzle atoms need 1024-byte alignment */
        if (tid == 0) atomicOr(P.err, 4u);
        return;
    }

    /* resident parameters: W1 (pre-arranged), biases, head */
    {
        const unsigned char* w1g = wtc + (size_t)(NLAYER - 1) * FU_CHUNKS * FU_CHUNK_BYTES;
        for (int i = tid; i < HID * IN_PAD * 2 / 16; i += FU_THREADS)
            reinterpret_cast<uint4*>(sm + L::W1)[i] = reinterpret_cast<const uint4*>(w1g)[i];
#pragma unroll
        for (int l = 0; l < NLAYER; ++l)   /* constant indices keep P.bias out of local memory */
            for (int i = tid; i < HID; i += FU_THREADS) bias_s[l * HID + i] = 0.5f * P.bias[l][i];
        for (int i = tid; i < HID; i += FU_THREADS) w5_s[i] = __bfloat162float(P.w5[i]);
        if (tid == 0) {
            *reinterpret_cast<float*>(sm + L::B5) = P.b5[0];
            *abort_flag = 0;
            for (int i = 0; i < FB_COUNT; ++i) {
                int cnt = 1;                                                      /* one arrive / one commit */
                if (i >= FB_HREADY && i < FB_HREADY + FU_CHUNKS) cnt = FU_EPI_WARPS;   /* every epilogue warp */
                if (i == FB_ACCEMPTY || i == FB_ACCEMPTY + 1) cnt = FU_EPI_WARPS;
                if (i == FB_FEATREADY) cnt = TC_ROWS;                             /* the feature threads */
                if (i == FB_HEADFULL) cnt = FU_EPI_WARPS - 4;                     /* partials 1-3 */
                if (i == FB_HEADEMPTY) cnt = 4;                                   /* partial 0 */
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(bar(i)), "r"(cnt) : "memory");
            }
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(smem_u32(taddr_slot)), "r"(2 * TC_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *taddr_slot;
    const int ntiles = (P.n + TC_ROWS - 1) / TC_ROWS;
    const uint32_t buf0 = smem_u32(sm + L::BUF), ring0 = smem_u32(sm + L::RING);

    if (warp < FU_EPI_WARPS) {
        /* ---------------- epilogue ---------------- */
        const int g = warp & 3, q = warp >> 2;
        const int rl = 32 * g + lane;
        uint32_t af_ph = 0u, hf_ph = 0u, he_ph = 0u;   /* phase bits (af: bit a = accumulator a) */
        bool ok = true;
        /* this thread's row in the activation buffer: atom column kc at kc * 16 KB */
        unsigned char* hb_row = sm + L::BUF + (rl / 8) * 1024 + (rl % 8) * 128;
        /* accumulator a starts at the bias of the layer that uses it next
           (layers 0 and 1 first): this warp's lanes, columns 64r + 16q */
        const uint32_t tlanes = tmem + ((uint32_t)(32 * g) << 16);
#pragma unroll 1
        for (int a = 0; a < 2; ++a)
#pragma unroll 1
            for (int r = 0; r < FU_CHUNKS; ++r)
                tc_st16_bias(tlanes + (uint32_t)(a * TC_COLS + 64 * r + 16 * q), bias_s + a * HID + 64 * r + 16 * q);
        tc_st_wait();
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) {
            fu_arrive(bar(FB_ACCEMPTY));
            fu_arrive(bar(FB_ACCEMPTY + 1));
        }
        for (int tile = blockIdx.x, it = 0; tile < ntiles && ok; tile += gridDim.x, ++it) {
            for (int l = 0; l < NLAYER; ++l) {
                const int a = l & 1;
                ok = __all_sync(FULL_MASK_MLP, fu_wait(bar(FB_ACCFULL + a), (af_ph >> a) & 1u, abort_flag, P.err, P.wait_cycles));
                if (!ok) break;
                af_ph ^= 1u << a;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                float part = 0.0f;
                /* round r: columns 64r + 16q .. +15, so that round r completes
                   K chunk r of the next layer's A operand; the TMEM load of
                   round r + 1 is in flight while round r is processed */
                const uint32_t tbase = tmem + ((uint32_t)(32 * g) << 16) + (uint32_t)(a * TC_COLS + 16 * q);
                uint32_t acc[FU_CHUNKS][16];
                tc_ld16_issue(tbase, acc[0]);
                tc_ld16_wait(acc[0]);
#pragma unroll
                for (int r = 0; r < FU_CHUNKS; ++r) {
                    const int col = 64 * r + 16 * q;
                    if (r + 1 < FU_CHUNKS) tc_ld16_issue(tbase + (uint32_t)(64 * (r + 1)), acc[r + 1]);
                    uint32_t hp[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        float g0, g1;
                        gelu_half_f2(f2_pack(__uint_as_float(acc[r][2 * j]), __uint_as_float(acc[r][2 * j + 1])), g0, g1);
                        hp[j] = pack_bf16(g0, g1);
                    }
                    if (l < NLAYER - 1) {
                        /* over the previous layer's activations (whose MMAs have all
                           completed): atom column r, 16-byte groups 2q, 2q+1 */
#pragma unroll
                        for (int c4 = 0; c4 < 2; ++c4)
                            *reinterpret_cast<uint4*>(hb_row + r * (TC_ROWS * 128) + (((2 * q + c4) ^ (rl % 8)) * 16)) =
                                make_uint4(hp[4 * c4], hp[4 * c4 + 1], hp[4 * c4 + 2], hp[4 * c4 + 3]);
                        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                        __syncwarp();
                        if (lane == 0) fu_arrive(bar(FB_HREADY + r));
                    } else {
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            part = __fmaf_rn(bf16_lo(hp[j]), w5_s[col + 2 * j], part);
                            part = __fmaf_rn(bf16_hi(hp[j]), w5_s[col + 2 * j + 1], part);
                        }
                    }
                    if (r + 1 < FU_CHUNKS) tc_ld16_wait(acc[r + 1]);
                }
                /* the accumulator's next user is layer (l + 2) mod 4 (of the
                   next tile for l >= 2): its bias goes in now */
#pragma unroll 1
                for (int r = 0; r < FU_CHUNKS; ++r)
                    tc_st16_bias(tlanes + (uint32_t)(a * TC_COLS + 64 * r + 16 * q),
                                 bias_s + ((l + 2) % NLAYER) * HID + 64 * r + 16 * q);
                tc_st_wait();
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncwarp();
                if (lane == 0) fu_arrive(bar(FB_ACCEMPTY + a));
                if (l == NLAYER - 1) {
                    /* output head: partials 1-3 are handed to the warps of partial 0 */
                    if (q > 0) {
                        if (it > 0) {
                            ok = __all_sync(FULL_MASK_MLP, fu_wait(bar(FB_HEADEMPTY), he_ph, abort_flag, P.err, P.wait_cycles));
                            if (!ok) break;
                            he_ph ^= 1u;
                        }
                        red[q * TC_ROWS + rl] = part;
                        __syncwarp();
                        if (lane == 0) fu_arrive(bar(FB_HEADFULL));
                    } else {
                        ok = __all_sync(FULL_MASK_MLP, fu_wait(bar(FB_HEADFULL), hf_ph, abort_flag, P.err, P.wait_cycles));
                        if (!ok) break;
                        hf_ph ^= 1u;
                        const float logit = ((part + red[TC_ROWS + rl]) + (red[2 * TC_ROWS + rl] + red[3 * TC_ROWS + rl])) +
                                            b5_s[0];
                        const int row = tile * TC_ROWS + rl;
                        if (row < P.n) P.p[row] = 1.0f / (1.0f + expf(-logit));
                        __syncwarp();
                        if (lane == 0) fu_arrive(bar(FB_HEADEMPTY));
                    }
                }
            }
        }
    } else if (warp == FU_PRODUCER_WARP) {
        /* ---------------- weight loads ---------------- */
        if (lane == 0) {
            uint32_t issued = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                for (int ch = 0; ch < (NLAYER - 1) * FU_CHUNKS; ++ch, ++issued) {
                    const uint32_t st = issued % FU_NS, k = issued / FU_NS;
                    if (k > 0 && !(ok = fu_wait(bar(FB_WEMPTY + st), (k - 1) & 1u, abort_flag, P.err, P.wait_cycles, 32u))) break;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                                 :: "r"(bar(FB_WFULL + st)), "r"(FU_CHUNK_BYTES) : "memory");
                    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                                 :: "r"(ring0 + st * FU_CHUNK_BYTES), "l"(wtc + (size_t)ch * FU_CHUNK_BYTES),
                                    "r"(FU_CHUNK_BYTES), "r"(bar(FB_WFULL + st))
                                 : "memory");
                }
            }
            /* the copies still in flight land before the CTA leaves */
            for (uint32_t j = issued > FU_NS ? issued - FU_NS : 0u; j < issued; ++j)
                fu_wait_drain(bar(FB_WFULL + j % FU_NS), (j / FU_NS) & 1u, P.err);
        }
    } else if (warp == FU_MMA_WARP) {
        /* ---------------- MMA issue ---------------- */
        if (lane == 0) {
            uint32_t consumed = 0, fr_ph = 0u, ae_ph = 0u, hr_ph = 0u;   /* ae_ph bit a: accumulator a */
            bool ok = true;
            const uint64_t w1d = tc_sdesc(smem_u32(sm + L::W1), 128u, IN_PAD * 16u);
            const uint64_t fd = tc_sdesc(smem_u32(sm + L::FEAT), 128u, IN_PAD * 16u);
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                for (int l = 0; l < NLAYER && ok; ++l) {
                    const int a = l & 1;
                    /* the accumulator's previous layer has been read out and the
                       bias of this layer written in (the first time: the bias only) */
                    if (!(ok = fu_wait(bar(FB_ACCEMPTY + a), (ae_ph >> a) & 1u, abort_flag, P.err, P.wait_cycles))) break;
                    ae_ph ^= 1u << a;
                    const uint32_t acc = tmem + (uint32_t)(a * TC_COLS);
                    if (l == 0) {
                        if (!(ok = fu_wait(bar(FB_FEATREADY), fr_ph, abort_flag, P.err, P.wait_cycles))) break;
                        fr_ph ^= 1u;
                        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                        fu_mma(acc, fd, w1d, 1u);
                        fu_commit(bar(FB_FEATEMPTY));
                    } else {
                        for (int c = 0; c < FU_CHUNKS; ++c, ++consumed) {
                            /* K columns 64c.. of the previous layer's activations (hready
                               phases advance once per hidden layer, in order) */
                            if (!(ok = fu_wait(bar(FB_HREADY + c), hr_ph, abort_flag, P.err, P.wait_cycles))) break;
                            const uint32_t st = consumed % FU_NS;
                            if (!(ok = fu_wait(bar(FB_WFULL + st), (consumed / FU_NS) & 1u, abort_flag, P.err, P.wait_cycles))) break;
                            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
                            for (int s2 = 0; s2 < FU_CK / 16; ++s2) {
                                /* K step 4c + s2: 32 bytes into the swizzle atoms of column c */
                                const uint64_t ad = tc_sdesc_sw128(buf0 + (uint32_t)c * (TC_ROWS * 128) + (uint32_t)s2 * 32u);
                                const uint64_t bd = tc_sdesc_sw128(ring0 + st * FU_CHUNK_BYTES + (uint32_t)s2 * 32u);
                                fu_mma(acc, ad, bd, 1u);
                            }
                            fu_commit(bar(FB_WEMPTY + st));
                        }
                        if (!ok) break;
                        hr_ph ^= 1u;
                    }
                    fu_commit(bar(FB_ACCFULL + a));
                }
            }
            /* every MMA issued so far completes before TMEM is freed */
            fu_commit(bar(FB_DRAIN));
            fu_wait_drain(bar(FB_DRAIN), 0u, P.err);
        }
    } else {
        /* ---------------- input features ---------------- */
        const int t = tid - FU_FEAT_WARP0 * 32;
        uint32_t fe_ph = 0u;
        bool ok = true;
        for (int tile = blockIdx.x, it = 0; tile < ntiles; tile += gridDim.x, ++it) {
            if (it > 0) {
                ok = __all_sync(FULL_MASK_MLP, fu_wait(bar(FB_FEATEMPTY), fe_ph, abort_flag, P.err, P.wait_cycles, 256u));
                if (!ok) break;
                fe_ph ^= 1u;
            }
            const int r = tile * TC_ROWS + t;
            uint32_t x[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float sv = 0.0f, cv = 0.0f;
                if (j < P.ndof && r < P.n) sincosf(P.q[r + P.qoff * j], &sv, &cv);
                x[j] = pack_bf16(j < P.ndof ? sv : 0.0f, j < P.ndof ? cv : 0.0f);
            }
#pragma unroll
            for (int c = 0; c < 2; ++c)
                *reinterpret_cast<uint4*>(sm + L::FEAT + (t / 8) * (IN_PAD * 16) + c * 128 + (t % 8) * 16) =
                    make_uint4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            fu_arrive(bar(FB_FEATREADY));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    __syncwarp();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(2 * TC_COLS)
                     : "memory");
}


/* ------------------------------------------------------------------ */
/* training GEMMs on the tensor cores (tcgen05, operands loaded by TMA)  */
/* ------------------------------------------------------------------ */
/*
 * k_tc_gemm computes one 128 x BN tile of C = A B^T over a range of K,
 * with A [M x K] and B [N x K] row-major BF16 in global memory, both read
 * by 2-D TMA loads (box 64 K x rows, 128-byte swizzle, zero fill outside
 * the tensor) into a 4-stage ring; one thread issues M=128 N=BN K=16
 * tcgen05.mma into a BN-column TMEM accumulator; four epilogue warps read
 * it back and apply one of:
 *   TG_FWD    z = acc + bias[n]: Z (FP32) and H = GELU(z) (BF16), row-major;
 *   TG_DH     dZ = acc * GELU'(Zin) (BF16), row-major (backward through a layer);
 *   TG_WPART  the FP32 partial sum of this K split, row-major into the
 *             split's slice of a workspace (weight gradients, reduced by
 *             k_reduce_w in a fixed order).
 * Warps: 0 loads, 1 issues the MMAs (and owns TMEM), 2-5 run the epilogue
 * (warp w reads TMEM lanes 32 (w % 4) ..).  Waits are bounded like those of
 * k_mlp_fused.
 */
enum { TG_FWD = 0, TG_DH = 1, TG_WPART = 2 };
constexpr int TG_STAGES = 4;
constexpr int TG_MAX_SPLITS = 32;
/* column tile of the layer GEMMs (forward, backward through a layer): 64
   columns, 4 x more CTAs than one 256-column tile, so that the epilogue
   (GELU, GELU', row stores) spreads over more SMs */
constexpr int TG_BN_LAYER = 64;
constexpr int TG_THREADS = 192;

template <int BN>
struct TgSmem {
    static constexpr size_t A_BYTES = (size_t)TC_ROWS * 128;       /* 128 rows x 64 BF16 */
    static constexpr size_t B_BYTES = (size_t)BN * 128;
    static constexpr size_t STAGE = A_BYTES + B_BYTES;
    static constexpr size_t BARS = TG_STAGES * STAGE;
    static constexpr size_t TADDR = BARS + (2 * TG_STAGES + 2) * 8;
    static constexpr size_t ABORT = TADDR + 4;
    static constexpr size_t BYTES = ABORT + 4 + 1024;               /* + alignment slack */
};

struct TgArgs {
    int M, N, K, kps;          /* rows, columns, depth, K per split (multiple of 64) */
    const float* bias;         /* TG_FWD */
    float* zout;               /* TG_FWD: Z [M x ldc] */
    __nv_bfloat16* hout;       /* TG_FWD: H, TG_DH: dZ [M x ldc] */
    const float* zin;          /* TG_DH: Z of the layer below [M x ldc] */
    float* ws;                 /* TG_WPART: [splits][M x ldc] */
    int ldc;
    unsigned* err;
    long long wait_cycles;     /* budget of each pipeline wait (the drains keep FU_WAIT_CYCLES) */
};

__device__ __forceinline__ void tg_tma_load(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                 :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}

template <int EPI, int BN>
__global__ void __launch_bounds__(TG_THREADS, 1)
k_tc_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TgArgs g)
{
    extern __shared__ __align__(1024) unsigned char sm_raw[];
    using L = TgSmem<BN>;
    /* the swizzle atoms need 1024-byte alignment */
    unsigned char* sm = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bars = smem_u32(sm + L::BARS);
    auto bar = [&](int i) { return bars + 8u * (uint32_t)i; };   /* full 0..3, empty 4..7, accfull 8 */
    volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::ABORT);
    uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(sm + L::TADDR);
    const int m0 = blockIdx.y * TC_ROWS, n0 = blockIdx.x * BN;
    const int kb = blockIdx.z * g.kps;
    const int ke = min(g.K, kb + g.kps);
    const int nchunks = ke > kb ? (ke - kb + 63) / 64 : 0;
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(TC_ROWS >> 4) << 24);
    if (tid == 0) {
        *abort_flag = 0;
        for (int i = 0; i < 2 * TG_STAGES + 1; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(bar(i)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(smem_u32(taddr_slot)), "r"(BN < 32 ? 32 : BN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *taddr_slot;
    const uint32_t st0 = smem_u32(sm);

    if (warp == 0) {
        if (lane == 0) {
            bool ok = true;
            int c = 0;
            for (; c < nchunks && ok; ++c) {
                const int s = c % TG_STAGES, k = c / TG_STAGES;
                if (k > 0 && !(ok = fu_wait(bar(TG_STAGES + s), (k - 1) & 1u, abort_flag, g.err, g.wait_cycles))) break;
                const uint32_t a_dst = st0 + (uint32_t)(s * L::STAGE);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                             :: "r"(bar(s)), "r"((uint32_t)L::STAGE) : "memory");
                tg_tma_load(a_dst, &mapA, kb + 64 * c, m0, bar(s));
                tg_tma_load(a_dst + (uint32_t)L::A_BYTES, &mapB, kb + 64 * c, n0, bar(s));
            }
            /* the loads still in flight land before the CTA leaves */
            for (int j = c > TG_STAGES ? c - TG_STAGES : 0; j < c; ++j)
                fu_wait_drain(bar(j % TG_STAGES), (j / TG_STAGES) & 1u, g.err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            bool ok = true;
            for (int c = 0; c < nchunks && ok; ++c) {
                const int s = c % TG_STAGES;
                if (!(ok = fu_wait(bar(s), (c / TG_STAGES) & 1u, abort_flag, g.err, g.wait_cycles))) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t a = st0 + (uint32_t)(s * L::STAGE), b = a + (uint32_t)L::A_BYTES;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint64_t ad = tc_sdesc_sw128(a + 32u * j), bd = tc_sdesc_sw128(b + 32u * j);
                    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                                 :: "r"(tmem), "l"(ad), "l"(bd), "r"(IDESC), "r"((c | j) != 0 ? 1u : 0u),
                                    "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                }
                fu_commit(bar(TG_STAGES + s));
            }
            /* accfull: every MMA issued has completed; on the abort path the
               epilogue stops waiting for it, so this thread waits (under the
               drain budget) before the CTA frees its tensor memory */
            fu_commit(bar(2 * TG_STAGES));
            fu_wait_drain(bar(2 * TG_STAGES), 0u, g.err);
        }
    } else {
        const int q = warp & 3;                      /* TMEM lane quarter */
        const int rl = 32 * q + lane, m = m0 + rl;
        const bool ok = __all_sync(FULL_MASK_MLP, fu_wait(bar(2 * TG_STAGES), 0u, abort_flag, g.err, g.wait_cycles));
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (ok) {
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                float v[32];
                __syncwarp();
                tc_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                if (nchunks == 0) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = 0.0f;
                }
                const int n = n0 + c0;
                const size_t o = (size_t)m * g.ldc + n;
                if (m >= g.M || n >= g.N) {
                    /* row or columns outside C: nothing to store */
                } else if (EPI == TG_FWD) {
#pragma unroll
                    for (int j = 0; j < 32; j += 4) {
                        const float4 b4 = *reinterpret_cast<const float4*>(g.bias + n + j);
                        const float4 z4 = make_float4(v[j] + b4.x, v[j + 1] + b4.y, v[j + 2] + b4.z, v[j + 3] + b4.w);
                        *reinterpret_cast<float4*>(g.zout + o + j) = z4;
                        v[j] = z4.x; v[j + 1] = z4.y; v[j + 2] = z4.z; v[j + 3] = z4.w;
                    }
#pragma unroll
                    for (int c4 = 0; c4 < 4; ++c4)
                        *reinterpret_cast<uint4*>(g.hout + o + 8 * c4) = make_uint4(
                            pack_bf16(gelu_f(v[8 * c4]), gelu_f(v[8 * c4 + 1])),
                            pack_bf16(gelu_f(v[8 * c4 + 2]), gelu_f(v[8 * c4 + 3])),
                            pack_bf16(gelu_f(v[8 * c4 + 4]), gelu_f(v[8 * c4 + 5])),
                            pack_bf16(gelu_f(v[8 * c4 + 6]), gelu_f(v[8 * c4 + 7])));
                } else if (EPI == TG_DH) {
                    float zz[32];
#pragma unroll
                    for (int j = 0; j < 32; j += 4) {
                        const float4 z4 = *reinterpret_cast<const float4*>(g.zin + o + j);
                        zz[j] = z4.x; zz[j + 1] = z4.y; zz[j + 2] = z4.z; zz[j + 3] = z4.w;
                    }
#pragma unroll
                    for (int c4 = 0; c4 < 4; ++c4)
                        *reinterpret_cast<uint4*>(g.hout + o + 8 * c4) = make_uint4(
                            pack_bf16(v[8 * c4] * gelu_grad(zz[8 * c4]), v[8 * c4 + 1] * gelu_grad(zz[8 * c4 + 1])),
                            pack_bf16(v[8 * c4 + 2] * gelu_grad(zz[8 * c4 + 2]), v[8 * c4 + 3] * gelu_grad(zz[8 * c4 + 3])),
                            pack_bf16(v[8 * c4 + 4] * gelu_grad(zz[8 * c4 + 4]), v[8 * c4 + 5] * gelu_grad(zz[8 * c4 + 5])),
                            pack_bf16(v[8 * c4 + 6] * gelu_grad(zz[8 * c4 + 6]), v[8 * c4 + 7] * gelu_grad(zz[8 * c4 + 7])));
                } else {
                    float* w = g.ws + (size_t)blockIdx.z * ((size_t)g.M * g.ldc) + o;
#pragma unroll
                    for (int j = 0; j < 32; j += 4)
                        *reinterpret_cast<float4*>(w + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 1) {
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(BN < 32 ? 32 : BN)
                     : "memory");
    }
}

/* g_w[o][i] (i < kin) = sum over the splits of ws[s][o][i] (ld ldw), in split order. */
/* Threads [0, rows*kin): gw = the split partials of ws added in split
 * order.  Then, with cpart, rows x 32 threads: gb[o] = sum over
 * b < cparts of cpart[b][o]; then, with opart, (HID + 1) x 32 threads:
 * go[c] = sum over b < oparts of opart[b][c] (the output layer's k_out_back
 * partials); both a warp per column in a fixed order.  rows * kin is a
 * multiple of 32, so every warp lies in one segment. */
__global__ void k_reduce_w(int splits, int rows, int ldw, int kin, const float* __restrict__ ws, float* __restrict__ gw,
                           int cparts, const float* __restrict__ cpart, float* __restrict__ gb,
                           int oparts, const float* __restrict__ opart, float* __restrict__ go)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < rows * kin) {
        const int o = t / kin, i = t % kin;
        float acc = 0.0f;
#pragma unroll 8
        for (int s = 0; s < splits; ++s) acc += ws[(size_t)s * rows * ldw + (size_t)o * ldw + i];
        gw[t] = acc;
        return;
    }
    t -= rows * kin;
    if (cpart) {
        /* biases: one warp per column, lane l sums the partials l, l + 32,
           ... in order, then a fixed shuffle tree adds the lanes */
        if (t < rows * 32) {
            const int c = t >> 5, lane = t & 31;
            float acc = 0.0f;
#pragma unroll 4
            for (int b = lane; b < cparts; b += 32) acc += cpart[(size_t)b * rows + c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) gb[c] = acc;
            return;
        }
        t -= rows * 32;
    }
    /* output layer: one warp per column c (the segment starts at a multiple
       of 32 threads, so its warps are whole): lane l sums the partials
       l, l + 32, ... in order, then a fixed shuffle tree adds the lanes */
    if (opart && t < (HID + 1) * 32) {
        const int c = t >> 5, lane = t & 31;
        float acc = 0.0f;
#pragma unroll 4
        for (int b = lane; b < oparts; b += 32) acc += opart[(size_t)b * (HID + 1) + c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) go[c] = acc;
    }
}

/* Two transposes in one launch, 32x32 tiles: blocks x < xa write
 * ta[c][r] = a[r][c] (cols_a columns) and colsum[blockIdx.y][c] = the sum
 * of the tile's 32 rows of column c (rows past the end count zero: fixed
 * order, deterministic column sums); the others tb[c][r] = b[r][c]
 * (cols_b columns).  ldd: the leading dimension of ta and tb. */
__global__ void k_transpose2_bf16(int rows, int xa, int cols_a, const __nv_bfloat16* __restrict__ a, int lda,
                                  __nv_bfloat16* __restrict__ ta, float* __restrict__ colsum, int cols_b,
                                  const __nv_bfloat16* __restrict__ b, int ldb, __nv_bfloat16* __restrict__ tb,
                                  int ldd)
{
    __shared__ __nv_bfloat16 t[32][33];
    const bool first = (int)blockIdx.x < xa;
    const int cols = first ? cols_a : cols_b, lds = first ? lda : ldb;
    const __nv_bfloat16* src = first ? a : b;
    __nv_bfloat16* dst = first ? ta : tb;
    const int r0 = blockIdx.y * 32, c0 = (first ? blockIdx.x : blockIdx.x - xa) * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        t[k][threadIdx.x] = (r < rows && c < cols) ? src[(size_t)r * lds + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    if (first && colsum && threadIdx.y == 0 && c0 + threadIdx.x < cols) {
        float acc = 0.0f;
        for (int k = 0; k < 32; ++k) acc += __bfloat162float(t[k][threadIdx.x]);
        colsum[(size_t)blockIdx.y * cols + c0 + threadIdx.x] = acc;
    }
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) dst[(size_t)c * ldd + r] = t[threadIdx.x][k];
    }
}

/* The tensor-core training copies of the weights: W1 padded to 64 inputs
 * (zeros) and W_l^T for the hidden layers 2..4 (the B operand of the
 * backward GEMMs through them). */
__global__ void k_tc_weights(const __nv_bfloat16* __restrict__ wbf, long long o0, long long o1, long long o2,
                             long long o3, __nv_bfloat16* __restrict__ w1p, __nv_bfloat16* __restrict__ wt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < HID * 64) {
        const int o = t / 64, i = t % 64;
        w1p[t] = i < IN_PAD ? wbf[o0 + (long long)o * IN_PAD + i] : __float2bfloat16(0.0f);
    } else if (t < HID * 64 + 3 * HID * HID) {
        const int u = t - HID * 64, l = u / (HID * HID), r = u % (HID * HID);
        const int i = r / HID, o = r % HID;                 /* wt_l[i][o] = W_l[o][i] */
        const long long off = l == 0 ? o1 : (l == 1 ? o2 : o3);
        wt[u] = wbf[off + (long long)o * HID + i];
    }
}

/* Features padded to 64 columns (the tensor-core K step): row i of X64 =
 * sin/cos of configuration idx[i] (or i), zeros beyond 2 ndof. */
__global__ void k_features64(const float* __restrict__ q, long long offset, int ndof, int n,
                             const int* __restrict__ idx, const long long* __restrict__ idx_off,
                             __nv_bfloat16* __restrict__ X)
{
    const long long io = idx_off ? *idx_off : 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const long long src = idx ? idx[io + i] : i;
        uint32_t x[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = 0u;
#pragma unroll
        for (int j = 0; j < IN_PAD / 2; ++j) {
            float sv = 0.0f, cv = 0.0f;
            if (j < ndof) sincosf(q[src + offset * j], &sv, &cv);
            x[j] = pack_bf16(j < ndof ? sv : 0.0f, j < ndof ? cv : 0.0f);
        }
        uint4* row = reinterpret_cast<uint4*>(X + (size_t)i * 64);
#pragma unroll
        for (int c = 0; c < 8; ++c) row[c] = make_uint4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
    }
}

}  // namespace

/* ====================================================================== */
/* host side                                                              */
/* ====================================================================== */

struct gprm_mlp {
    int ndof = 6;
    int max_batch = 0;
    /* parameter vector (fp32 master): W1[HID x IN_PAD] b1 W2 b2 W3 b3 W4 b4 w5[HID] b5[1] */
    long long nparam = 0;
    long long offW[NLAYER + 1], offB[NLAYER + 1];
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    int* bf_map = nullptr;
    __nv_bfloat16* wbf = nullptr;       /* bf16 copies of W1..W4, w5 */
    long long offWbf[NLAYER + 1];
    long long nbf = 0;
    /* activations for max_batch rows */
    __nv_bfloat16* X = nullptr;
    __nv_bfloat16* H[NLAYER] = {nullptr};
    float* Z[NLAYER] = {nullptr};
    __nv_bfloat16* dZ[NLAYER] = {nullptr};
    float *p = nullptr, *dlogit = nullptr, *loss = nullptr, *ybatch = nullptr;
    int* idx = nullptr;
    long long adam_t = 0;
    cudaStream_t st = nullptr;
    /* inference on the tensor-core layers (k_mlp_tc) */
    int infer_path = GPRM_MLP_INFER_TCGEN05;
    __nv_bfloat16 *Ha = nullptr, *Hb = nullptr;
    int infer_rows = 0;
    unsigned char* wtc = nullptr;       /* weights in the fused kernel's chunk order */
    /* training on the tensor cores (k_tc_gemm) */
    int train_path = GPRM_MLP_TRAIN_TCGEN05;
    __nv_bfloat16* X64 = nullptr;       /* features padded to 64 columns [rows x 64] */
    /* the weight-gradient chain of each layer (transposes, split-K GEMM,
       ordered reduction) has its own buffers, so that the chains of
       different layers can run side by side on st_w */
    __nv_bfloat16 *Ta = nullptr, *Tb = nullptr;   /* transposes [NLAYER][256 x ldT] */
    int ldT = 0;
    __nv_bfloat16* w1p = nullptr;       /* W1 padded [256 x 64] */
    __nv_bfloat16* wt = nullptr;        /* W_l^T, layers 2..4 [3 x 256 x 256] */
    float* ws = nullptr;                /* split-K partials [NLAYER][TG_MAX_SPLITS x 256 x 256] */
    float* cpart = nullptr;             /* bias-gradient partials [NLAYER][cparts x 256] */
    size_t cparts = 0;
    cudaStream_t st_w = nullptr;        /* weight-gradient chains */
    cudaEvent_t ev_dz[NLAYER] = {};     /* dZ_l written (on st) */
    cudaEvent_t ev_w = nullptr;         /* every chain done (on st_w) */
    float* opart = nullptr;             /* output-layer gradient partials [1024 x 257] */
    int tc_n = -1;                      /* batch the tensor maps were made for */
    int tc_attr = 0;
    long long* d_ctl = nullptr;         /* training epoch: [row offset into perm, Adam step before it] */
    const long long* idx_off = nullptr; /* set while a training epoch is captured */
    CUtensorMap m_x64, m_h[NLAYER - 1], m_dz[NLAYER], m_w1p, m_w[NLAYER - 1], m_wt[NLAYER - 1], m_ta[NLAYER],
        m_tb256[NLAYER], m_tb64;
    unsigned* dev_err = nullptr;
    long long wait_cycles = 0;          /* pipeline wait budget of the tensor-core kernels, 0 = default */
    int sms = 0;
    std::string err = "no error";
};

namespace {

/* The pipeline wait budget the tensor-core kernels get (0: their default). */
long long wait_budget(const gprm_mlp* h) { return h->wait_cycles; }

int mfail(gprm_mlp* h, int code, const char* msg, cudaError_t e = cudaSuccess)
{
    if (h) h->err = std::string(msg) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return code;
}

#define MLP_TRY(h, call)                                                         \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return mfail((h), GPRM_ERR_CUDA, #call, e_);      \
    } while (0)

int alloc_batch(gprm_mlp* h, int rows)
{
    if (rows <= h->max_batch) return GPRM_OK;
    cudaFree(h->X);
    for (int l = 0; l < NLAYER; ++l) { cudaFree(h->H[l]); cudaFree(h->Z[l]); cudaFree(h->dZ[l]); }
    cudaFree(h->p); cudaFree(h->dlogit); cudaFree(h->ybatch); cudaFree(h->idx);
    size_t R = (size_t)rows;
    MLP_TRY(h, cudaMalloc((void**)&h->X, R * IN_PAD * sizeof(__nv_bfloat16)));
    for (int l = 0; l < NLAYER; ++l) {
        MLP_TRY(h, cudaMalloc((void**)&h->H[l], R * HID * sizeof(__nv_bfloat16)));
        MLP_TRY(h, cudaMalloc((void**)&h->Z[l], R * HID * sizeof(float)));
        MLP_TRY(h, cudaMalloc((void**)&h->dZ[l], R * HID * sizeof(__nv_bfloat16)));
    }
    MLP_TRY(h, cudaMalloc((void**)&h->p, R * sizeof(float)));
    MLP_TRY(h, cudaMalloc((void**)&h->dlogit, R * sizeof(float)));
    MLP_TRY(h, cudaMalloc((void**)&h->ybatch, R * sizeof(float)));
    MLP_TRY(h, cudaMalloc((void**)&h->idx, R * sizeof(int)));
    cudaFree(h->X64); cudaFree(h->Ta); cudaFree(h->Tb); cudaFree(h->cpart);
    h->cpart = nullptr;
    const size_t cparts = std::max<size_t>(1024, (R + 31) / 32);
    h->cparts = cparts;
    MLP_TRY(h, cudaMalloc((void**)&h->cpart, (size_t)NLAYER * cparts * HID * sizeof(float)));
    if (!h->opart) MLP_TRY(h, cudaMalloc((void**)&h->opart, (size_t)1024 * (HID + 1) * sizeof(float)));
    h->ldT = (rows + 63) / 64 * 64;
    MLP_TRY(h, cudaMalloc((void**)&h->X64, R * 64 * sizeof(__nv_bfloat16)));
    MLP_TRY(h, cudaMalloc((void**)&h->Ta, (size_t)NLAYER * HID * h->ldT * sizeof(__nv_bfloat16)));
    MLP_TRY(h, cudaMalloc((void**)&h->Tb, (size_t)NLAYER * HID * h->ldT * sizeof(__nv_bfloat16)));
    if (!h->w1p) {
        MLP_TRY(h, cudaMalloc((void**)&h->w1p, (size_t)HID * 64 * sizeof(__nv_bfloat16)));
        MLP_TRY(h, cudaMalloc((void**)&h->wt, (size_t)(NLAYER - 1) * HID * HID * sizeof(__nv_bfloat16)));
        MLP_TRY(h, cudaMalloc((void**)&h->ws, (size_t)NLAYER * TG_MAX_SPLITS * HID * HID * sizeof(float)));
    }
    if (!h->st_w) {
        MLP_TRY(h, cudaStreamCreateWithFlags(&h->st_w, cudaStreamNonBlocking));
        for (int l = 0; l < NLAYER; ++l) MLP_TRY(h, cudaEventCreateWithFlags(&h->ev_dz[l], cudaEventDisableTiming));
        MLP_TRY(h, cudaEventCreateWithFlags(&h->ev_w, cudaEventDisableTiming));
    }
    h->tc_n = -1;
    h->max_batch = rows;
    return GPRM_OK;
}

dim3 ggrid(int M, int N) { return dim3((N + BN - 1) / BN, (M + BM - 1) / BM); }


/* ---- training on the tensor cores: tensor maps, forward, backward ---- */

int tc_setup(gprm_mlp* h);

PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;

int tc_map(gprm_mlp* h, CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
           uint32_t box_outer)
{
    if (!g_encode_tiled) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return mfail(h, GPRM_ERR_CUDA, "cuTensorMapEncodeTiled is not available", e);
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {64u, box_outer};
    const cuuint32_t es[2] = {1u, 1u};
    const CUresult r = g_encode_tiled(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                                      box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mfail(h, GPRM_ERR_CUDA, "encoding a tensor map");
    return GPRM_OK;
}

/* Tensor maps of the training buffers for a batch of n rows (made again
 * when n or the buffers change). */
int tc_maps(gprm_mlp* h, int n)
{
    if (h->tc_n == n) return GPRM_OK;
    int rc;
    const uint64_t N = (uint64_t)n;
    if ((rc = tc_map(h, &h->m_x64, h->X64, 64, N, 64 * 2, TC_ROWS))) return rc;
    for (int l = 0; l < NLAYER - 1; ++l)
        if ((rc = tc_map(h, &h->m_h[l], h->H[l], HID, N, HID * 2, TC_ROWS))) return rc;
    for (int l = 0; l < NLAYER; ++l)
        if ((rc = tc_map(h, &h->m_dz[l], h->dZ[l], HID, N, HID * 2, TC_ROWS))) return rc;
    if ((rc = tc_map(h, &h->m_w1p, h->w1p, 64, HID, 64 * 2, TG_BN_LAYER))) return rc;
    for (int l = 1; l < NLAYER; ++l) {
        if ((rc = tc_map(h, &h->m_w[l - 1], h->wbf + h->offWbf[l], HID, HID, HID * 2, TG_BN_LAYER))) return rc;
        if ((rc = tc_map(h, &h->m_wt[l - 1], h->wt + (size_t)(l - 1) * HID * HID, HID, HID, HID * 2, TG_BN_LAYER)))
            return rc;
    }
    for (int l = 0; l < NLAYER; ++l) {
        const size_t o = (size_t)l * HID * h->ldT;
        if ((rc = tc_map(h, &h->m_ta[l], h->Ta + o, N, HID, (uint64_t)h->ldT * 2, TC_ROWS))) return rc;
        if ((rc = tc_map(h, &h->m_tb256[l], h->Tb + o, N, HID, (uint64_t)h->ldT * 2, HID))) return rc;
    }
    if ((rc = tc_map(h, &h->m_tb64, h->Tb, N, 64, (uint64_t)h->ldT * 2, 64))) return rc;
    if (!h->tc_attr) {
        MLP_TRY(h, cudaFuncSetAttribute(k_tc_gemm<TG_FWD, TG_BN_LAYER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)TgSmem<TG_BN_LAYER>::BYTES));
        MLP_TRY(h, cudaFuncSetAttribute(k_tc_gemm<TG_DH, TG_BN_LAYER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)TgSmem<TG_BN_LAYER>::BYTES));
        MLP_TRY(h, cudaFuncSetAttribute(k_tc_gemm<TG_WPART, HID>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)TgSmem<HID>::BYTES));
        MLP_TRY(h, cudaFuncSetAttribute(k_tc_gemm<TG_WPART, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)TgSmem<64>::BYTES));
        h->tc_attr = 1;
    }
    h->tc_n = n;
    return GPRM_OK;
}

/* Forward through the tensor-core GEMMs on rows featurised in h->X64. */
int forward_tc(gprm_mlp* h, int n, float* p, const float* y, const int* yidx, float inv_b, cudaStream_t st)
{
    int rc = tc_setup(h);
    if (rc || (rc = tc_maps(h, n))) return rc;
    const int items = HID * 64 + (NLAYER - 1) * HID * HID;
    k_tc_weights<<<(items + 255) / 256, 256, 0, st>>>(h->wbf, h->offWbf[0], h->offWbf[1], h->offWbf[2],
                                                      h->offWbf[3], h->w1p, h->wt);
    const dim3 grid(HID / TG_BN_LAYER, (n + TC_ROWS - 1) / TC_ROWS, 1);
    for (int l = 0; l < NLAYER; ++l) {
        TgArgs a{};
        a.M = n; a.N = HID; a.K = l == 0 ? 64 : HID; a.kps = a.K;
        a.bias = h->w + h->offB[l]; a.zout = h->Z[l]; a.hout = h->H[l]; a.ldc = HID; a.err = h->dev_err; a.wait_cycles = wait_budget(h);
        k_tc_gemm<TG_FWD, TG_BN_LAYER><<<grid, TG_THREADS, TgSmem<TG_BN_LAYER>::BYTES, st>>>(
            l == 0 ? h->m_x64 : h->m_h[l - 1],
                                                                          l == 0 ? h->m_w1p : h->m_w[l - 1], a);
    }
    int blocks = (n * 32 + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_out<<<blocks, 256, 0, st>>>(n, h->H[NLAYER - 1], h->wbf + h->offWbf[NLAYER], h->w + h->offB[NLAYER], p, y,
                                  yidx, h->idx_off, h->dlogit, h->loss, inv_b);
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

/* Backward through the tensor-core GEMMs (after forward_tc on the same rows). */
int backward_tc(gprm_mlp* h, int n, cudaStream_t st)
{
    /* every gradient entry is written below (weights and biases by the
       ordered reductions of k_reduce_w), so h->g needs no clearing */
    int blocks = n < 1024 ? n : 1024;
    k_out_back<<<blocks, HID, 0, st>>>(n, h->H[NLAYER - 1], h->Z[NLAYER - 1], h->wbf + h->offWbf[NLAYER], h->dlogit,
                                       h->opart, h->dZ[NLAYER - 1]);
    /* weight gradients: K = n split over CTAs, partials reduced in split
       order (128 rows per split: 512-row splits made the step 1.4x slower,
       the GEMM's longer K loop costing more than the partials it saves) */
    int splits = (n + 127) / 128;
    if (splits > TG_MAX_SPLITS) splits = TG_MAX_SPLITS;
    const int kps = ((n + splits - 1) / splits + 63) / 64 * 64;
    splits = (n + kps - 1) / kps;
    const dim3 tblock(32, 8);
    /* layer l's weight gradients (transposes, split-K GEMM, ordered
       reduction) depend only on dZ_l and the forward activations: they run
       on st_w, in their own buffers, while st carries the chain of backward
       GEMMs dZ_l -> dZ_{l-1}; st waits for all of them at the end (a fork
       and join that a captured graph keeps as dependencies) */
    MLP_TRY(h, cudaEventRecord(h->ev_dz[NLAYER - 1], st));
    for (int l = NLAYER - 1; l >= 0; --l) {
        const int kin = l == 0 ? IN_PAD : HID, kin_p = l == 0 ? 64 : HID;
        __nv_bfloat16* Ta = h->Ta + (size_t)l * HID * h->ldT;
        __nv_bfloat16* Tb = h->Tb + (size_t)l * HID * h->ldT;
        float* ws = h->ws + (size_t)l * TG_MAX_SPLITS * HID * HID;
        float* cpart = h->cpart + (size_t)l * h->cparts * HID;
        MLP_TRY(h, cudaStreamWaitEvent(h->st_w, h->ev_dz[l], 0));
        /* dW_l = dZ_l^T H_{l-1}: A = dZ_l^T [256 x n], B = H_{l-1}^T [kin_p x n] */
        k_transpose2_bf16<<<dim3(HID / 32 + kin_p / 32, (n + 31) / 32), tblock, 0, h->st_w>>>(
            n, HID / 32, HID, h->dZ[l], HID, Ta, cpart, kin_p, l == 0 ? h->X64 : h->H[l - 1], kin_p, Tb, h->ldT);
        TgArgs a{};
        a.M = HID; a.N = kin_p; a.K = n; a.kps = kps; a.ws = ws; a.ldc = kin_p; a.err = h->dev_err; a.wait_cycles = wait_budget(h);
        if (l == 0)
            k_tc_gemm<TG_WPART, 64><<<dim3(1, HID / TC_ROWS, splits), TG_THREADS, TgSmem<64>::BYTES, h->st_w>>>(
                h->m_ta[0], h->m_tb64, a);
        else
            k_tc_gemm<TG_WPART, HID><<<dim3(1, HID / TC_ROWS, splits), TG_THREADS, TgSmem<HID>::BYTES, h->st_w>>>(
                h->m_ta[l], h->m_tb256[l], a);
        /* weights, this layer's biases (column sums of dZ_l from the transpose)
           and, with the last layer, the output layer's partials */
        const bool out_l = l == NLAYER - 1;
        const int red_threads = HID * kin + HID * 32 + (out_l ? (HID + 1) * 32 : 0);   /* segments of whole warps */
        k_reduce_w<<<(red_threads + 255) / 256, 256, 0, h->st_w>>>(splits, HID, kin_p, kin, ws, h->g + h->offW[l],
                                                                   (n + 31) / 32, cpart, h->g + h->offB[l],
                                                                   out_l ? blocks : 0, out_l ? h->opart : nullptr,
                                                                   h->g + h->offW[NLAYER]);
        if (l > 0) {
            /* dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1}): A = dZ_l [n x 256], B = W_l^T [256 x 256] */
            TgArgs d{};
            d.M = n; d.N = HID; d.K = HID; d.kps = HID; d.zin = h->Z[l - 1]; d.hout = h->dZ[l - 1]; d.ldc = HID;
            d.err = h->dev_err;
            d.wait_cycles = wait_budget(h);
            k_tc_gemm<TG_DH, TG_BN_LAYER><<<dim3(HID / TG_BN_LAYER, (n + TC_ROWS - 1) / TC_ROWS, 1), TG_THREADS,
                                            TgSmem<TG_BN_LAYER>::BYTES, st>>>(
                h->m_dz[l], h->m_wt[l - 1], d);
            MLP_TRY(h, cudaEventRecord(h->ev_dz[l - 1], st));
        }
    }
    MLP_TRY(h, cudaEventRecord(h->ev_w, h->st_w));
    MLP_TRY(h, cudaStreamWaitEvent(st, h->ev_w, 0));
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

/* Features of n rows (idx: row gather or null) for the current training path. */
void features(gprm_mlp* h, const float* q, int offset, int n, const int* idx, cudaStream_t st)
{
    if (h->train_path == GPRM_MLP_TRAIN_TCGEN05)
        k_features64<<<(n + 255) / 256, 256, 0, st>>>(q, offset, h->ndof, n, idx, h->idx_off, h->X64);
    else
        k_features<<<(n + 255) / 256, 256, 0, st>>>(q, offset, h->ndof, n, idx, h->idx_off, h->X);
}

/* Forward on rows already featurised in h->X; p written to `p`. */
int forward(gprm_mlp* h, int n, float* p, const float* y, const int* yidx, float inv_b, cudaStream_t st)
{
    if (h->train_path == GPRM_MLP_TRAIN_TCGEN05) return forward_tc(h, n, p, y, yidx, inv_b, st);
    const __nv_bfloat16* in = h->X;
    int kin = IN_PAD;
    for (int l = 0; l < NLAYER; ++l) {
        EpiArgs ep{};
        ep.bias = h->w + h->offB[l];
        ep.zout = h->Z[l];
        ep.hout = h->H[l];
        ep.ldc = HID;
        k_gemm<false, true, EPI_FWD_HIDDEN><<<ggrid(n, HID), 128, 0, st>>>(n, HID, kin, in, kin,
                                                                           h->wbf + h->offWbf[l], kin, ep);
        in = h->H[l];
        kin = HID;
    }
    int blocks = (n * 32 + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_out<<<blocks, 256, 0, st>>>(n, h->H[NLAYER - 1], h->wbf + h->offWbf[NLAYER], h->w + h->offB[NLAYER], p, y,
                                  yidx, h->idx_off, h->dlogit, h->loss, inv_b);
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

/* Backward for a batch of n rows whose forward pass just ran; gradients
 * accumulate into h->g (zeroed here). */
int backward(gprm_mlp* h, int n, cudaStream_t st)
{
    if (h->train_path == GPRM_MLP_TRAIN_TCGEN05) return backward_tc(h, n, st);
    MLP_TRY(h, cudaMemsetAsync(h->g, 0, (size_t)h->nparam * sizeof(float), st));
    int blocks = n < 1024 ? n : 1024;
    k_out_back<<<blocks, HID, 0, st>>>(n, h->H[NLAYER - 1], h->Z[NLAYER - 1], h->wbf + h->offWbf[NLAYER], h->dlogit,
                                       h->opart, h->dZ[NLAYER - 1]);
    k_reduce_parts<<<(HID + 1 + 255) / 256, 256, 0, st>>>(blocks, HID + 1, h->opart, h->g + h->offW[NLAYER]);
    for (int l = NLAYER - 1; l >= 0; --l) {
        const int kin = l == 0 ? IN_PAD : HID;
        const __nv_bfloat16* hin = l == 0 ? h->X : h->H[l - 1];
        /* dW_l = dZ_l^T H_{l-1}: M = HID, N = kin, K = n */
        EpiArgs eg{};
        eg.gout = h->g + h->offW[l];
        eg.ldc = kin;
        k_gemm<true, false, EPI_GRAD_W><<<ggrid(HID, kin), 128, 0, st>>>(HID, kin, n, h->dZ[l], HID, hin, kin, eg);
        k_colsum<<<blocks, HID, 0, st>>>(n, HID, h->dZ[l], h->cpart);
        k_reduce_parts<<<1, HID, 0, st>>>(blocks, HID, h->cpart, h->g + h->offB[l]);
        if (l > 0) {
            /* dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1}): M = n, N = HID, K = HID */
            EpiArgs ed{};
            ed.hout = h->dZ[l - 1];
            ed.zin = h->Z[l - 1];
            ed.ldc = HID;
            k_gemm<false, false, EPI_BWD_DH><<<ggrid(n, HID), 128, 0, st>>>(n, HID, HID, h->dZ[l], HID,
                                                                            h->wbf + h->offWbf[l], HID, ed);
        }
    }
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

/* One Adam step: step number (*t_base) + t_step (t_base null: t_step). */
int adam_at(gprm_mlp* h, float lr, const long long* t_base, long long t_step, cudaStream_t st)
{
    k_adam<<<1024, 256, 0, st>>>(h->nparam, h->w, h->g, h->m, h->v, h->bf_map, h->wbf, lr, 0.9f, 0.999f, 1e-8f,
                                 t_base, t_step);
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

int adam(gprm_mlp* h, float lr, cudaStream_t st)
{
    h->adam_t += 1;
    return adam_at(h, lr, nullptr, h->adam_t, st);
}

/* deterministic uniform init in [-1/sqrt(in), 1/sqrt(in)] (Linear's default
 * range) from a 64-bit LCG */
double lcg_uniform(uint64_t& s)
{
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

namespace {

/* Error flag and SM count for the tensor-core kernels (first use). */
int tc_setup(gprm_mlp* h)
{
    if (h->dev_err) return GPRM_OK;
    MLP_TRY(h, cudaMalloc((void**)&h->dev_err, sizeof(unsigned)));
    MLP_TRY(h, cudaMemset(h->dev_err, 0, sizeof(unsigned)));
    int dev = 0;
    MLP_TRY(h, cudaGetDevice(&dev));
    MLP_TRY(h, cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, dev));
    MLP_TRY(h, cudaFuncSetAttribute(k_mlp_tc<IN_PAD, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TcSmem<IN_PAD>::LAUNCH));
    MLP_TRY(h, cudaFuncSetAttribute(k_mlp_tc<HID, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TcSmem<HID>::LAUNCH));
    MLP_TRY(h, cudaFuncSetAttribute(k_mlp_tc<HID, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)TcSmem<HID>::LAUNCH));
    MLP_TRY(h, cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FuSmem::BYTES));
    return GPRM_OK;
}

/* Predictions of n rows (q[i + offset*j]) by the fused kernel: the weights
 * are put in chunk order, then one persistent launch runs every layer. */
int predict_fused(gprm_mlp* h, const float* q, int n, int offset, float* p, cudaStream_t st)
{
    int rc = tc_setup(h);
    if (rc) return rc;
    if (!h->wtc) MLP_TRY(h, cudaMalloc((void**)&h->wtc, FU_RELAYOUT_BYTES));
    const int items = (NLAYER - 1) * HID * (HID / 8) + HID * (IN_PAD / 8);
    k_mlp_relayout<<<(items + 255) / 256, 256, 0, st>>>(h->wbf, h->offWbf[0], h->offWbf[1], h->offWbf[2],
                                                        h->offWbf[3], h->wtc);
    FuParams P;
    P.q = q;
    P.qoff = offset;
    P.ndof = h->ndof;
    P.n = n;
    P.wtc = h->wtc;
    for (int l = 0; l < NLAYER; ++l) P.bias[l] = h->w + h->offB[l];
    P.w5 = h->wbf + h->offWbf[NLAYER];
    P.b5 = h->w + h->offB[NLAYER];
    P.p = p;
    P.err = h->dev_err;
    P.wait_cycles = wait_budget(h);
    const int tiles = (n + TC_ROWS - 1) / TC_ROWS;
    const int grid = tiles < h->sms ? tiles : h->sms;
    k_mlp_fused<<<grid, FU_THREADS, FuSmem::BYTES, st>>>(P);
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

/* Predictions of n rows (q[i + offset*j]) through the tensor-core layers,
 * one kernel per layer. */
int predict_tc(gprm_mlp* h, const float* q, int n, int offset, float* p, cudaStream_t st)
{
    const int chunk = 1 << 18;
    const int rows = n < chunk ? n : chunk;
    if (rows > h->infer_rows) {
        cudaFree(h->Ha);
        cudaFree(h->Hb);
        h->Ha = h->Hb = nullptr;
        h->infer_rows = 0;
        MLP_TRY(h, cudaMalloc((void**)&h->Ha, (size_t)rows * HID * sizeof(__nv_bfloat16)));
        MLP_TRY(h, cudaMalloc((void**)&h->Hb, (size_t)rows * HID * sizeof(__nv_bfloat16)));
        h->infer_rows = rows;
    }
    int rc = tc_setup(h);
    if (rc) return rc;
    const __nv_bfloat16* wb = h->wbf;
    const float* w = h->w;
    for (int s = 0; s < n; s += chunk) {
        const int c = n - s < chunk ? n - s : chunk;
        const int tiles = (c + TC_ROWS - 1) / TC_ROWS;
        const int grid = tiles < h->sms ? tiles : h->sms;
        k_mlp_tc<IN_PAD, true, false><<<grid, 256, TcSmem<IN_PAD>::LAUNCH, st>>>(
            c, q + s, offset, h->ndof, nullptr, wb + h->offWbf[0], w + h->offB[0], h->Ha, nullptr, nullptr, nullptr,
            h->dev_err);
        k_mlp_tc<HID, false, false><<<grid, 256, TcSmem<HID>::LAUNCH, st>>>(
            c, nullptr, 0, 0, h->Ha, wb + h->offWbf[1], w + h->offB[1], h->Hb, nullptr, nullptr, nullptr, h->dev_err);
        k_mlp_tc<HID, false, false><<<grid, 256, TcSmem<HID>::LAUNCH, st>>>(
            c, nullptr, 0, 0, h->Hb, wb + h->offWbf[2], w + h->offB[2], h->Ha, nullptr, nullptr, nullptr, h->dev_err);
        k_mlp_tc<HID, false, true><<<grid, 256, TcSmem<HID>::LAUNCH, st>>>(
            c, nullptr, 0, 0, h->Ha, wb + h->offWbf[3], w + h->offB[3], nullptr, wb + h->offWbf[NLAYER],
            w + h->offB[NLAYER], p + s, h->dev_err);
        MLP_TRY(h, cudaGetLastError());
    }
    return GPRM_OK;
}

}  // namespace

extern "C" {

int gprm_mlp_create(int ndof, unsigned long long seed, gprm_mlp** out)
{
    if (!out || ndof < 1 || ndof > IN_PAD / 2) return GPRM_ERR_ARG;
    gprm_mlp* h = new gprm_mlp();
    h->ndof = ndof;
    long long off = 0, offbf = 0;
    for (int l = 0; l <= NLAYER; ++l) {
        const int nin = l == 0 ? IN_PAD : HID, nout = l == NLAYER ? 1 : HID;
        h->offW[l] = off; off += (long long)nout * nin;
        h->offB[l] = off; off += nout;
        h->offWbf[l] = offbf; offbf += (long long)nout * nin;
    }
    /* the inference kernels read the hidden layers' biases as float4 */
    for (int l = 0; l < NLAYER; ++l)
        if (h->offB[l] % 4 != 0) {
            delete h;
            return GPRM_ERR_ARG;
        }
    h->nparam = off;
    h->nbf = offbf;
    std::vector<float> w(off, 0.0f);
    std::vector<int> map(off, -1);
    uint64_t s = seed * 0x9E3779B97F4A7C15ULL + 12345;
    for (int l = 0; l <= NLAYER; ++l) {
        const int nin = l == 0 ? IN_PAD : HID, nout = l == NLAYER ? 1 : HID;
        const int fan_in = l == 0 ? 2 * ndof : nin;
        const double bound = 1.0 / sqrt((double)fan_in);
        for (int o = 0; o < nout; ++o) {
            for (int i = 0; i < nin; ++i) {
                long long k = h->offW[l] + (long long)o * nin + i;
                bool pad = (l == 0 && i >= 2 * ndof);
                w[k] = pad ? 0.0f : (float)((2.0 * lcg_uniform(s) - 1.0) * bound);
                map[k] = (int)(h->offWbf[l] + (long long)o * nin + i);
            }
            w[h->offB[l] + o] = (float)((2.0 * lcg_uniform(s) - 1.0) * bound);
        }
    }
    cudaError_t e;
    if ((e = cudaMalloc((void**)&h->w, off * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->g, off * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->m, off * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->v, off * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->bf_map, off * sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->wbf, offbf * sizeof(__nv_bfloat16))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->loss, sizeof(float))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)) != cudaSuccess) {
        gprm_mlp_destroy(h);
        return e == cudaErrorMemoryAllocation ? GPRM_ERR_NOMEM : GPRM_ERR_CUDA;
    }
    cudaMemcpy(h->w, w.data(), off * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(h->bf_map, map.data(), off * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemset(h->m, 0, off * sizeof(float));
    cudaMemset(h->v, 0, off * sizeof(float));
    k_to_bf16<<<256, 256>>>(off, h->w, h->bf_map, h->wbf);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
        gprm_mlp_destroy(h);
        return GPRM_ERR_CUDA;
    }
    *out = h;
    return GPRM_OK;
}

void gprm_mlp_destroy(gprm_mlp* h)
{
    if (!h) return;
    if (h->st) cudaStreamSynchronize(h->st);
    cudaFree(h->w); cudaFree(h->g); cudaFree(h->m); cudaFree(h->v); cudaFree(h->bf_map); cudaFree(h->wbf);
    cudaFree(h->loss); cudaFree(h->X);
    for (int l = 0; l < NLAYER; ++l) { cudaFree(h->H[l]); cudaFree(h->Z[l]); cudaFree(h->dZ[l]); }
    cudaFree(h->p); cudaFree(h->dlogit); cudaFree(h->ybatch); cudaFree(h->idx);
    cudaFree(h->Ha); cudaFree(h->Hb); cudaFree(h->dev_err); cudaFree(h->wtc);
    cudaFree(h->X64); cudaFree(h->Ta); cudaFree(h->Tb); cudaFree(h->w1p); cudaFree(h->wt); cudaFree(h->ws);
    cudaFree(h->cpart); cudaFree(h->opart);
    cudaFree(h->d_ctl);
    if (h->st_w) {
        cudaStreamSynchronize(h->st_w);
        cudaStreamDestroy(h->st_w);
    }
    for (int l = 0; l < NLAYER; ++l)
        if (h->ev_dz[l]) cudaEventDestroy(h->ev_dz[l]);
    if (h->ev_w) cudaEventDestroy(h->ev_w);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

const char* gprm_mlp_last_error(const gprm_mlp* h) { return h ? h->err.c_str() : "null handle"; }

long long gprm_mlp_num_params(const gprm_mlp* h) { return h ? h->nparam : 0; }

int gprm_mlp_get_params(gprm_mlp* h, float* out)
{
    if (!h || !out) return GPRM_ERR_ARG;
    MLP_TRY(h, cudaStreamSynchronize(h->st));
    MLP_TRY(h, cudaMemcpy(out, h->w, h->nparam * sizeof(float), cudaMemcpyDeviceToHost));
    return GPRM_OK;
}

int gprm_mlp_set_params(gprm_mlp* h, const float* in)
{
    if (!h || !in) return GPRM_ERR_ARG;
    MLP_TRY(h, cudaStreamSynchronize(h->st));
    MLP_TRY(h, cudaMemcpy(h->w, in, h->nparam * sizeof(float), cudaMemcpyHostToDevice));
    k_to_bf16<<<256, 256, 0, h->st>>>(h->nparam, h->w, h->bf_map, h->wbf);
    MLP_TRY(h, cudaStreamSynchronize(h->st));
    return GPRM_OK;
}

/* p[i] = P(collision) for configurations q (device SoA, q[i + offset*j]). */
int gprm_mlp_predict(gprm_mlp* h, const float* q, int n, int offset, float* p, void* stream)
{
    if (!h || n < 0 || (n > 0 && (!q || !p)) || offset < n) return mfail(h, GPRM_ERR_ARG, "bad arguments");
    if (n == 0) return GPRM_OK;
    cudaStream_t st = (cudaStream_t)stream;   /* NULL: the legacy default stream */
    if (h->infer_path == GPRM_MLP_INFER_TCGEN05) return predict_fused(h, q, n, offset, p, st);
    if (h->infer_path == GPRM_MLP_INFER_TCGEN05_LAYERS) return predict_tc(h, q, n, offset, p, st);
    const int chunk = 1 << 16;
    int rc = alloc_batch(h, n < chunk ? n : chunk);
    if (rc) return rc;
    for (int s = 0; s < n; s += chunk) {
        int c = n - s < chunk ? n - s : chunk;
        features(h, q + s, offset, c, nullptr, st);
        rc = forward(h, c, p + s, nullptr, nullptr, 0.0f, st);
        if (rc) return rc;
    }
    MLP_TRY(h, cudaGetLastError());
    return GPRM_OK;
}

/* Gradients of the mean BCE over the n labelled configurations (one
 * forward/backward, no update): grads[nparam] and *loss on the host. */
int gprm_mlp_gradients(gprm_mlp* h, const float* q, const float* y, int n, int offset, float* grads, float* loss)
{
    if (!h || n < 1 || !q || !y || !grads || !loss || offset < n) return mfail(h, GPRM_ERR_ARG, "bad arguments");
    int rc = alloc_batch(h, n);
    if (rc) return rc;
    MLP_TRY(h, cudaMemsetAsync(h->loss, 0, sizeof(float), h->st));
    features(h, q, offset, n, nullptr, h->st);
    if ((rc = forward(h, n, h->p, y, nullptr, 1.0f / n, h->st))) return rc;
    if ((rc = backward(h, n, h->st))) return rc;
    MLP_TRY(h, cudaStreamSynchronize(h->st));
    MLP_TRY(h, cudaMemcpy(grads, h->g, h->nparam * sizeof(float), cudaMemcpyDeviceToHost));
    MLP_TRY(h, cudaMemcpy(loss, h->loss, sizeof(float), cudaMemcpyDeviceToHost));
    return GPRM_OK;
}

/* One Adam step (lr, beta 0.9/0.999, eps 1e-8) with the current gradients. */
int gprm_mlp_adam_step(gprm_mlp* h, float lr)
{
    if (!h) return GPRM_ERR_ARG;
    int rc = adam(h, lr, h->st);
    if (rc) return rc;
    MLP_TRY(h, cudaStreamSynchronize(h->st));
    return GPRM_OK;
}

/* Trains on n labelled configurations (device SoA q, labels y in {0,1}):
 * `epochs` passes in shuffled order (perm: device array of epochs*n
 * indices, each epoch a permutation), batches of `batch`, Adam at `lr`.
 * Every step runs features, forward, loss, backward and Adam on the
 * device; each epoch's launches are captured into one CUDA graph.
 * losses[epoch] gets the mean batch loss of each epoch (host array). */
int gprm_mlp_train(gprm_mlp* h, const float* q, const float* y, int n, int offset, const int* perm, int epochs,
                   int batch, float lr, float* losses)
{
    if (!h || !q || !y || !perm || n < batch || batch < 1 || epochs < 1 || offset < n)
        return mfail(h, GPRM_ERR_ARG, "bad arguments");
    int rc = alloc_batch(h, batch);
    if (rc) return rc;
    /* set-up that must not run inside the stream capture below */
    if (h->train_path == GPRM_MLP_TRAIN_TCGEN05 && ((rc = tc_setup(h)) || (rc = tc_maps(h, batch)))) return rc;
    const int steps = n / batch;
    std::vector<float> ep_loss(epochs, 0.0f);
    if (!h->d_ctl) MLP_TRY(h, cudaMalloc((void**)&h->d_ctl, 2 * sizeof(long long)));
    /* one epoch's launches are captured once into a graph; each epoch sets
       its offset into perm and its first Adam step in device memory */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    MLP_TRY(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int crc = GPRM_OK;
    h->idx_off = h->d_ctl;
    cudaMemsetAsync(h->loss, 0, sizeof(float), h->st);
    for (int s = 0; s < steps && !crc; ++s) {
        const int* idx = perm + (size_t)s * batch;
        features(h, q, offset, batch, idx, h->st);
        if (!crc) crc = forward(h, batch, h->p, y, idx, 1.0f / batch, h->st);
        if (!crc) crc = backward(h, batch, h->st);
        if (!crc) crc = adam_at(h, lr, h->d_ctl + 1, s + 1, h->st);
    }
    h->idx_off = nullptr;
    cudaError_t ce = cudaStreamEndCapture(h->st, &graph);
    if (crc) { if (graph) cudaGraphDestroy(graph); return crc; }
    if (ce != cudaSuccess) return mfail(h, GPRM_ERR_CUDA, "capturing the training epoch", ce);
    ce = cudaGraphInstantiate(&exec, graph, 0);
    for (int e = 0; e < epochs && ce == cudaSuccess; ++e) {
        const long long ctl[2] = {(long long)e * n, h->adam_t};
        ce = cudaMemcpyAsync(h->d_ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, h->st);
        if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, h->st);
        float l = 0;
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(&l, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
        ep_loss[e] = l / steps;
        h->adam_t += steps;
    }
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return mfail(h, GPRM_ERR_CUDA, "running the training epochs", ce);
    if (losses) memcpy(losses, ep_loss.data(), epochs * sizeof(float));
    if (h->dev_err) {
        unsigned f = 0;
        MLP_TRY(h, cudaMemcpy(&f, h->dev_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (f) return mfail(h, GPRM_ERR_DEVICE, "a tensor-core kernel timed out waiting for its MMAs or copies");
    }
    return GPRM_OK;
}

int gprm_mlp_set_inference(gprm_mlp* h, int path)
{
    if (!h) return GPRM_ERR_ARG;
    if (path != GPRM_MLP_INFER_TCGEN05 && path != GPRM_MLP_INFER_TRAINING_GEMM &&
        path != GPRM_MLP_INFER_TCGEN05_LAYERS)
        return mfail(h, GPRM_ERR_ARG, "unknown inference path");
    h->infer_path = path;
    return GPRM_OK;
}

int gprm_mlp_set_training(gprm_mlp* h, int path)
{
    if (!h) return GPRM_ERR_ARG;
    if (path != GPRM_MLP_TRAIN_TCGEN05 && path != GPRM_MLP_TRAIN_MMA_SYNC)
        return mfail(h, GPRM_ERR_ARG, "unknown training path");
    h->train_path = path;
    return GPRM_OK;
}

int gprm_mlp_set_wait_budget(gprm_mlp* h, long long cycles)
{
    if (!h || cycles < 0) return GPRM_ERR_ARG;
    MLP_TRY(h, cudaDeviceSynchronize());
    h->wait_cycles = cycles;
    if (h->dev_err) MLP_TRY(h, cudaMemset(h->dev_err, 0, sizeof(unsigned)));
    return GPRM_OK;
}

int gprm_mlp_device_status(gprm_mlp* h, unsigned* flags)
{
    if (!h || !flags) return GPRM_ERR_ARG;
    *flags = 0;
    MLP_TRY(h, cudaDeviceSynchronize());
    if (h->dev_err) MLP_TRY(h, cudaMemcpy(flags, h->dev_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (*flags) return mfail(h, GPRM_ERR_DEVICE, "a tensor-core kernel timed out waiting for its MMAs or copies");
    return GPRM_OK;
}

}  /* extern "C" */

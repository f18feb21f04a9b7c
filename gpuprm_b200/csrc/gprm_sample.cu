/*
 * gprm_sample.cu - batched sampling near roadmap nodes (gprm_sample_near of
 * include/gprm_b200.h).
 *
 * The reference grows its roadmaps with get_random_nodes
 * (prm/src/lib/prm/prmsolver.cpp:2585-2624): pick a stored node m, keep it
 * with probability about 1/(1+surrnum[m])^3 (the integer test
 * rand() <= RAND_MAX / x^3, x = 1 + surrnum[m]; get_random_nodes2, :2635-2698,
 * uses x^2), move it uniformly within +-D in every joint
 * (q = qstorage - D + 2*D*((float)rand()/RAND_MAX)) and keep the result when
 * indicator(q) == 0, one host call per candidate.  Here a batch of candidates
 * is drawn in one kernel and checked in one batched vertex check.
 *
 * Candidate t draws its random numbers from Philox4x32-10 (Salmon, Moraes,
 * Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011) with
 * key = seed and counters (t, block): the stream is fixed by (seed, t), so a
 * CPU restatement reproduces every candidate, and the "first num accepted
 * and free candidates in t order" is the same set whatever the batch size.
 * A 31-bit value r = x >> 1 stands in for rand() (RAND_MAX = 2^31 - 1).
 *
 * The reference picks the node in two draws over its block storage
 * (prmsolver.cpp:2589-2597): a block uniformly among the used ones, again
 * while it is empty, then a node uniformly among the block's num nodes, so
 * a node's weight is 1 / (non-empty blocks * its block's num).
 * gprm_sample_near_blocks takes that storage (block pos/num arrays over the
 * node slots) and draws the same way: block b = r0 % nblocks among the
 * blocks passed (the caller passes the non-empty ones; a block with num <= 0
 * dismisses its candidates), node pos[b] + r9 % num[b].  gprm_sample_near
 * draws the node uniformly (r0 % n), the same distribution when every node
 * is its own block.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gprm_b200.h"

namespace {

constexpr uint32_t PH_M0 = 0xD2511F53u, PH_M1 = 0xCD9E8D57u;
constexpr uint32_t PH_W0 = 0x9E3779B9u, PH_W1 = 0xBB67AE85u;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = PH_M0 * c.x, hi0 = __umulhi(PH_M0, c.x);
        const uint32_t lo1 = PH_M1 * c.z, hi1 = __umulhi(PH_M1, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += PH_W0;
        k.y += PH_W1;
    }
    return c;
}

__global__ void k_sample_near(int ndof, const float* __restrict__ nodes, int n, long long stride,
                              const int* __restrict__ block_pos, const int* __restrict__ block_num, int nblocks,
                              const int* __restrict__ surrnum, int power, float D, uint2 key, long long t0, int B,
                              float* __restrict__ q_out, long long out_stride, int* __restrict__ parent_out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
        const unsigned long long t = (unsigned long long)(t0 + i);
        const uint32_t tl = (uint32_t)t, th = (uint32_t)(t >> 32);
        const uint4 a = philox4x32_10(make_uint4(tl, th, 0u, 0u), key);
        const uint4 b = philox4x32_10(make_uint4(tl, th, 1u, 0u), key);
        const uint4 c = philox4x32_10(make_uint4(tl, th, 2u, 0u), key);
        const uint32_t r[10] = {a.x >> 1, a.y >> 1, a.z >> 1, a.w >> 1, b.x >> 1, b.y >> 1,
                                b.z >> 1, b.w >> 1, c.x >> 1, c.y >> 1};
        int m;
        if (block_pos) {
            const int blk = (int)(r[0] % (uint32_t)nblocks);
            const int cnt = block_num[blk];
            if (cnt <= 0) {                                  /* an empty block: dismissed */
                for (int j = 0; j < ndof; ++j) q_out[i + out_stride * j] = 0.0f;
                parent_out[i] = -1;
                continue;
            }
            m = block_pos[blk] + (int)(r[9] % (uint32_t)cnt);
            if (m < 0 || m >= n) {                           /* a block outside the node slots */
                for (int j = 0; j < ndof; ++j) q_out[i + out_stride * j] = 0.0f;
                parent_out[i] = -1;
                continue;
            }
        } else {
            m = (int)(r[0] % (uint32_t)n);
        }
        /* prob = RAND_MAX / x^p in integers; rand() > prob dismisses */
        const long long x = 1 + (long long)max(surrnum[m], 0);
        long long xp = 1;
        for (int e = 0; e < power; ++e) xp = xp > (1ll << 40) ? xp : xp * x;
        const long long prob = 2147483647ll / xp;
        const bool accept = (long long)r[1] <= prob;
        const float twoD = 2.0f * D;
        for (int j = 0; j < ndof; ++j) {
            const float u = (float)r[2 + j] / 2147483648.0f;   /* (float)rand() / RAND_MAX, RAND_MAX as float */
            q_out[i + out_stride * j] = (nodes[m + stride * j] - D) + twoD * u;
        }
        parent_out[i] = accept ? m : -1;
    }
}

}  // namespace

static int launch_sample(int ndof, const float* nodes, int n, int stride, const int* block_pos,
                         const int* block_num, int nblocks, const int* surrnum, int power, float D,
                         unsigned long long seed, long long t0, int B, float* q_out, int out_stride, int* parent_out,
                         void* stream)
{
    if (ndof < 1 || ndof > GPRM_MAX_DOF || n < 1 || stride < n || !nodes || !surrnum || power < 0 || power > 8 ||
        B < 0 || (B > 0 && (!q_out || !parent_out)) || out_stride < B || t0 < 0 || !(D >= 0.0f))
        return GPRM_ERR_ARG;
    if (B == 0) return GPRM_OK;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GPRM_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256;
    long long blocks = ((long long)B + threads - 1) / threads;
    if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    k_sample_near<<<(int)blocks, threads, 0, (cudaStream_t)stream>>>(ndof, nodes, n, stride, block_pos, block_num,
                                                                     nblocks, surrnum, power, D, key, t0, B, q_out,
                                                                     out_stride, parent_out);
    return cudaGetLastError() == cudaSuccess ? GPRM_OK : GPRM_ERR_CUDA;
}

extern "C" int gprm_sample_near(int ndof, const float* nodes, int n, int stride, const int* surrnum, int power,
                                float D, unsigned long long seed, long long t0, int B, float* q_out, int out_stride,
                                int* parent_out, void* stream)
{
    return launch_sample(ndof, nodes, n, stride, nullptr, nullptr, 0, surrnum, power, D, seed, t0, B, q_out,
                         out_stride, parent_out, stream);
}

extern "C" int gprm_sample_near_blocks(int ndof, const float* nodes, int n, int stride, const int* block_pos,
                                       const int* block_num, int nblocks, const int* surrnum, int power, float D,
                                       unsigned long long seed, long long t0, int B, float* q_out, int out_stride,
                                       int* parent_out, void* stream)
{
    if (!block_pos || !block_num || nblocks < 1) return GPRM_ERR_ARG;
    return launch_sample(ndof, nodes, n, stride, block_pos, block_num, nblocks, surrnum, power, D, seed, t0, B, q_out,
                         out_stride, parent_out, stream);
}

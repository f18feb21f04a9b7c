/*
 * gprm_host.h - host-side state of a gprm_space handle, shared by the
 * library's host sources (gprm_api.cu, gprm_batch.cu).  Not installed.
 */
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/gprm_b200.h"
#include "gprm_internal.h"

namespace gprm {

/* cudaMalloc through the library's allocation-failure test hook
 * (gprm_debug_fail_device_alloc): every device allocation of the checker
 * and the batches goes through it. */
cudaError_t dev_malloc(void** p, size_t bytes);

/* One request of the pool: stream, control block, device buffers and
 * pinned staging. */
/* host-buffer requests are split into up to this many parts, so that the
 * staging copy and the transfer of one part overlap the checks of the
 * previous one */
constexpr int HOST_PARTS = 4;

struct Request {
    cudaStream_t st = nullptr;
    Control* ctl = nullptr;       /* device, HOST_PARTS blocks (one per part) */
    Control* ctl_host = nullptr;  /* pinned copies read after the request */
    int parts = 1;                /* parts of the request in flight */
    float* d_a = nullptr;         /* q or qs (contiguous SoA, offset = n) */
    float* d_b = nullptr;         /* qe */
    int* d_res = nullptr;
    unsigned* d_key = nullptr;
    unsigned* d_seg = nullptr;    /* edge segment offsets (edge_seg_words of cap_seg edges) */
    size_t cap_seg = 0;           /* edges d_seg serves */
    uint2* d_queue = nullptr;
    unsigned* d_qpair = nullptr;  /* pair range of each queue item's recheck (BandQueue) */
    unsigned* d_ovf = nullptr;    /* overflow record of the FP64 queue: 2 words per item (BandQueue) */
    float* h_a = nullptr;         /* pinned staging */
    float* h_b = nullptr;
    int* h_res = nullptr;
    size_t cap_items = 0;         /* edges or configurations */
    size_t cap_queue = 0;
    /* FP64 queue demand of the last device-pointer edge call, read back
       without a synchronisation: the items it wanted (h_qwant, pinned),
       ready once ev_q has completed, for q_n edges */
    unsigned* h_qwant = nullptr;
    cudaEvent_t ev_q = nullptr;
    bool q_pending = false;
    long long q_n = 0;
    bool busy = false;
    /* the request in flight */
    int kind = 0;                 /* 0 vertices, 1 edges */
    int* user_res = nullptr;
    int n = 0;
    const float* user_a = nullptr;
    const float* user_b = nullptr;
    int user_offset = 0;
};

}  // namespace gprm

struct gprm_space {
    int ndof = 0;
    float dq = 0.01f;
    int nbuf = 0;
    float a[GPRM_MAX_DOF], alpha[GPRM_MAX_DOF], q0[GPRM_MAX_DOF], d0[GPRM_MAX_DOF];
    float mins[GPRM_MAX_DOF], maxs[GPRM_MAX_DOF];
    int types[GPRM_MAX_DOF];
    int npoly = 0, npairs = 0, sumn = 0, summ = 0;
    std::vector<float4> tab;       /* per-polytope blocks, see gprm_device.cuh */
    std::vector<int4> pairs;
    std::vector<float4> pairs_b;   /* certificate data per pair */
    std::vector<float4> far;       /* distance test: static ball centre, T2 */
    std::vector<int4> scan_c;      /* certificate scan: slots of P and Q (-1 static), sqrt(T2) up, usable */
    std::vector<float4> scan_b;    /* certificate scan: static polytope's vertex 0, R */
    std::vector<double> rad;       /* inflated ball radius per polytope */
    /* bounding box per polytope about its ball centre: PCA axes (FP32
       values), half extents (exact), and the device records (axis, inflated
       half extent) x 3 */
    std::vector<double> box_ax, box_e;
    std::vector<float4> box;
    std::vector<int> slot;         /* ball-centre slot of moving polytopes, -1 otherwise */
    std::vector<int> slot_sys, slot_block;
    std::vector<int> pair_poly, pair_sys;  /* polytopes and frames of each pair */
    /* every polytope's vertices as table entries, and (first, count) per polytope */
    std::vector<float4> vtab;
    std::vector<int4> vinfo;
    /* support candidates per polytope and direction bin (see fsupport_cand2) */
    std::vector<unsigned> cbin;
    std::vector<unsigned char> cidx;
    /* the lists as the device reads them: per (polytope, bin) cslots
       vertex entries (the list, then copies of its last entry) and the count */
    std::vector<float4> ctab;
    std::vector<unsigned char> ccnt;
    int cslots = 1;
    double extent = 1.0;           /* length scale of the scene (m) */
    float thr_dir = 0, eps_dir = 0;

    bool inited = false;
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    void* d_scene = nullptr;
    gprm::DevScene dsc;
    gprm::LaunchCfg cfg_v, cfg_e;

    int mode = GPRM_MODE_FP64_BAND;
    int policy = GPRM_EDGES_ALL_STEPS;
    int split_max = 16384;        /* edge batches up to this size split long edges */
    int split_rounds = 2;         /* rounds of 32 steps per segment */
    float band = 1e-5f;
    unsigned debug_qcap = 0;      /* test hook: FP64 queue capacity cap (0 = none) */
    double qdens_edges = 0.0;     /* most FP64 queue items per edge seen in a call (sizes later queues) */

    std::vector<gprm::Request> reqs;
    std::map<int, int> live;       /* request id -> slot */
    int next_id = 0;
    gprm::Request dev;             /* scratch of the device-pointer entry points */
    gprm::Control* d_total = nullptr;  /* cumulative counters of all requests */
    gprm_stats host_stats;         /* host-side counters */

    bool profiling = false;
    std::vector<cudaEvent_t> ev32, ev64;   /* start/stop pairs */
    size_t ev32_used = 0, ev64_used = 0;

    std::string err = "no error";
};

// vll_split.h -- the split-precision pipeline (FP64 geometry, FP32 window
// statistics, exact FP64 re-evaluation inside the FP32 error band).
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>
#include <cuda_runtime.h>

namespace vll {

struct DevLevel;

// Raises a kernel's dynamic shared-memory limit in the current context to at
// least `bytes`, never lowering it (thread-safe; see vll_split.cu).
cudaError_t ensure_smem_limit(const void *func, size_t bytes);

// Device scratch of the split pipeline, grown on demand and owned by a context.
struct SplitBuffers {
    void *node_k = nullptr;        // int32  [N+1] slots per active node (0 = inactive)
    void *slot_off = nullptr;      // int64  [N+1] prefix sum of node_k (the slot total)
    void *rho = nullptr;           // float  [pend_cap] FP32 slot values of queued nodes, then
                                   // the window kernel's per-warp slot scratch, then the
                                   // voxel slots listed for an exact INCC (int64 [fix_cap])
    void *gsum = nullptr;          // double [N] GNCC sums (FP64)
    void *gcnt = nullptr;          // double [N]
    void *scan_tmp = nullptr;      // cub temporary storage
    void *ctl = nullptr;           // uint64 [8] queue heads, counts, cursor
    void *pending = nullptr;       // int64  [N]  nodes queued for the exact pass
    void *pend_off = nullptr;      // int64  [N]  their offsets in rho (-1: none)
    void *base = nullptr;          // int64  [levels+1] first global node of each level
    void *acc_level = nullptr;     // uint64 [levels+1] Accessable_grid of each level
    size_t cap_nodes = 0, cap_slots = 0, cap_scan = 0, cap_levels = 0;
    int64_t pend_cap = 0;          // slots of rho in use
    int64_t fix_cap = 0;           // int64 entries of the voxel slot-fix list after them
    std::vector<int64_t> h_base;   // host copy of the level table
    bool capturing = false;        // enqueueing into a stream capture
};

// Launch parameters of the window kernel that the autotuner chooses.
struct SplitTuning {
    int blocks_per_sm = 0;      // CTAs per SM (0: the occupancy maximum)
    int grab = 8;               // nodes taken per queue access (at most 32)
    float box_margin = 1.1f;    // footprint budget over the swept-box estimate
};

// A level set's pipeline captured as a CUDA graph, with its own buffers.
struct SplitPlan {
    SplitBuffers bufs;
    cudaGraphExec_t exec = nullptr;
    int64_t n_slots = 0, launches = 0;
};

void split_release(SplitBuffers &b);

// Whether the split pipeline implements this level (stereo, no frame sensor,
// no relative-adjustment mode, H within the compiled window sizes; levels
// with combined-level INCC are evaluated in FP64 inside it); other levels run
// the plain FP64 kernel.
bool split_supported(const DevLevel &P);

// Encodes the level's TMA tiles (tensor maps of the reference and target
// planes, tile sized from the footprint sweep times `margin`) into P, or
// leaves them off (P.tma_w[0] = 0) where they do not apply.  Call on the host
// copy with its device image pointers, before it is copied to the device.
void split_prepare_tma(DevLevel &P, float margin);

// Runs the split pipeline for a level whose DevLevel block is at dP (device)
// and mirrored in P (host).  counters: [0] accessable, [1] evals,
// [2] FP64 re-checks, [3] error flag.
// Per-call timing / launch bookkeeping of the split pipeline.
struct SplitTiming {
    bool enabled = false;
    cudaEvent_t ev[9] = {};
    int64_t slots = 0;
    int64_t launches = 0;
};

cudaError_t run_split(SplitBuffers &b, const DevLevel &P, const DevLevel *dP,
                      unsigned long long *counters, cudaStream_t s, std::string *err,
                      SplitTiming *timing, const SplitTuning &tuning);

// The same pipeline over a set of levels (tiles and / or pyramid levels)
// whose blocks are hl (host copies) and dl (device array): one prep pass, one
// persistent window launch draining all levels' nodes (FindPeakNcc in the
// same warp), and one exact pass over the nodes it queued.  Per-level
// Accessable_grid counts are left in b.acc_level[0..n_levels).
cudaError_t run_split_set(SplitBuffers &b, const DevLevel *hl, const DevLevel *dl, int n_levels,
                          unsigned long long *counters, cudaStream_t s, std::string *err,
                          SplitTiming *timing, const SplitTuning &tuning);

// Sizes the plan's buffers with one pass of the front phase, then captures
// the whole pipeline of the level set into pl.exec (replayed with
// cudaGraphLaunch).  counters and dl must stay valid while the plan is used.
// `pre` (optional) enqueues work that belongs in front of the pipeline (the
// orthoimage rasters) both in the sizing pass and in the captured graph.
cudaError_t split_plan(SplitPlan &pl, SplitBuffers &b, const DevLevel *hl, const DevLevel *dl,
                       int n_levels, unsigned long long *counters, cudaStream_t s,
                       std::string *err, const SplitTuning &tuning,
                       const std::function<cudaError_t(cudaStream_t)> &pre);

}  // namespace vll

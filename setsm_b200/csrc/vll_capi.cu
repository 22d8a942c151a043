// vll_capi.cu -- the plain-C entry points of include/setsm_vll.h.
//
// A vll_context owns one CUDA stream and grow-only device buffers.  The
// host-buffer entry points upload a call's inputs, run the selected kernel and
// download the outputs; the *_device variants take device pointers and leave
// data resident (used by the serving loop and the benchmark).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "setsm_vll.h"
#include "vll_device.cuh"
#include "vll_internal.h"
#include "vll_split.h"

namespace {

struct Buf {
    void *p = nullptr;
    size_t cap = 0;
    // the host bytes the buffer holds a copy of (resident planes)
    const void *src = nullptr;
    size_t src_bytes = 0;
    uint64_t src_fp = 0;
};

cudaError_t ensure(Buf &b, size_t n) {
    if (n == 0) n = 1;
    if (n <= b.cap) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    b.src = nullptr;
    cudaError_t e = cudaMalloc(&b.p, n);
    if (e == cudaSuccess) b.cap = n;
    return e;
}

void release(Buf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    b.src = nullptr;
}

// Fingerprint of a host buffer: FNV-1a over 64 blocks of 64 bytes spread
// evenly over it (the whole buffer when it is smaller than 8 KB), the last
// 64 bytes and the size.
uint64_t sample_fingerprint(const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    uint64_t h = 1469598103934665603ull ^ (uint64_t)n;
    auto mix = [&](size_t off, size_t len) {
        for (size_t i = 0; i < len; ++i) h = (h ^ b[off + i]) * 1099511628211ull;
    };
    if (n <= 8192) {
        mix(0, n);
        return h;
    }
    const size_t step = (n - 64) / 63;
    for (int k = 0; k < 64; ++k) mix((size_t)k * step, 64);
    mix(n - 64, 64);
    return h;
}

thread_local std::string g_last_error;

// NVTX range around each public call (visible in Nsight Systems / Compute
// timelines; header-only, no cost when no tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

}  // namespace

struct vll_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    std::string err;
    Buf level, counters;
    Buf img[VLL_MAX_IMAGES][6];
    Buf wgs, pts, gp3, ncc, vox, voxoff, gsum, gcnt;
    Buf ocd[VLL_MAX_IMAGES], ocdn[VLL_MAX_IMAGES], ocdptr;
    Buf pre_tmp, pre_wt, pre_img, pre_mag, pre_ori;
    Buf sumcost;                       // SGM aggregation (float per voxel slot)
    Buf sgm_lr;                        // SGM: the 8 directions' costs per slot
    Buf tin_pts, tin_tris, tin_scratch;  // Ortho_blunder: points, triangles, work arrays
    vll::TinWork tin_work;             // TINCreate_list: work arrays
    int residency = 0;                 // VLL_RESIDENT_* flags
    Buf rvox, rvox_off;                // resident voxel packing and its offsets
    int64_t rvox_total = -1;           // its length (-1: none)
    int64_t rvox_nodes = 0;
    vll::SplitBuffers split;
    vll::SplitTuning tuning;
    void *set = nullptr;               // SetResources of batch calls (vll_capi.cu)
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEvent_t stage_ev[9] = {};
    int64_t launches_total = 0;
    int64_t tin_reruns = 0;   // blunder_detection_TIN calls that re-ran the point pass
    vll::DevLevel *hlevel = nullptr;   // pinned host staging of the level block
};

namespace {

int fail(vll_context *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    g_last_error = msg;
    return code;
}

int cuda_fail(vll_context *ctx, cudaError_t e, const char *where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(ctx, VLL_ERR_CUDA, m);
}

#define VLL_CUDA(ctx, call)                                     \
    do {                                                        \
        cudaError_t e__ = (call);                               \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, #call); \
    } while (0)

// SetNCC_alpha, setsm_code.cpp:6014-6047
double ncc_alpha(int L, int it, int is_ra) {
    double a;
    if (L >= 4) {
        a = 1.0 - ((4 - L) * 0.2 + (it - 1) * 0.05);
        if (a < 0.8) a = 0.8;
    } else if (L >= 3) {
        a = 1.0 - ((4 - L) * 0.2 + (it - 1) * 0.05);
        if (a < 0.6) a = 0.6;
    } else if (L == 2) {
        a = 1.0 - (0.4 + (it - 1) * 0.05);
        if (a < 0.4) a = 0.4;
    } else
        a = 1.0 - ((4 - L) * 0.2 + (it - 1) * 0.05);
    if (a < 0.1) a = 0.1;
    if (is_ra) a = 1.0;
    return a;
}

}  // namespace

namespace vll {

// Derives the per-call constants of VerticalLineLocus (setsm_code.cpp:6050-6137)
// from the descriptor.  Image / grid pointers are copied as given.
int derive_level(const vll_level_desc *d, DevLevel *P, std::string *err, bool vll_window) {
    memset(P, 0, sizeof(*P));
    if (!d) {
        *err = "null level descriptor";
        return VLL_ERR_INVALID;
    }
    if (d->sensor_type != 0) {
        *err = "only RPC (SB) sensors are supported";
        return VLL_ERR_UNSUPPORTED;
    }
    if (d->num_images < 2 || d->num_images > VLL_MAX_IMAGES) {
        *err = "num_images must be in [2, VLL_MAX_IMAGES]";
        return VLL_ERR_INVALID;
    }
    if (d->reference_id < 0 || d->reference_id >= d->num_images) {
        *err = "reference_id out of range";
        return VLL_ERR_INVALID;
    }
    if (d->grid_width <= 0 || d->grid_height <= 0 || !(d->height_step > 0) ||
        d->pyramid_step < 0 || d->pyramid_step > 12 || d->template_size < 1 ||
        d->template_size > 255) {
        *err = "invalid grid size, height step, pyramid step or template size";
        return VLL_ERR_INVALID;
    }
    const int L = d->pyramid_step;
    int template_size = d->template_size;
    if (L >= 1) {
        const double area = 5.0;
        const int t = (int)((area / (d->resolution * (1 << L))) / 2.0) * 2 + 1;
        if (d->template_size < t) template_size = t;
    }
    int H = template_size / 2;
    if (L == 3)
        H = H - 1;
    else if (L < 3)
        H = H - 2;
    if (vll_window && (H < 1 || H > kMaxHalf)) {
        *err = "window half-size out of the supported range [1, 8]";
        return VLL_ERR_UNSUPPORTED;
    }
    P->num_images = d->num_images;
    P->ref = d->reference_id;
    P->L = L;
    P->H = H;
    P->iteration = d->iteration;
    P->cmr = d->check_matching_rate != 0;
    P->is_ra = d->is_ra != 0;
    P->check_matchtag = d->check_matchtag != 0;
    P->pre_dem_tif = d->pre_dem_tif != 0;
    P->sgm_py = d->sgm_py;
    P->blunder_level = d->images[0].image_b ? d->blunder_level : L;
    P->combined = !P->is_ra && (L > d->py_combined_level);
    P->combined_incc = P->combined && (L >= 1 && d->iteration % 2 == 0);
    P->im_res_next = d->resolution;
    if (P->combined) P->im_res_next = d->resolution * (1 << (L - 1));
    P->im_res = d->resolution * (1 << L);
    int co = !((L == 4 && d->iteration == 1) || P->is_ra);
    if (d->pre_dem_tif && !(L == 4 && d->iteration == 1)) co = 1;
    if (d->check_matchtag) co = 1;
    if (L <= d->sgm_py) co = 0;
    P->check_ortho = co;
    P->alpha = ncc_alpha(L, d->iteration, P->is_ra);
    P->beta = 1.0 - P->alpha;
    P->ortho_th = 0.7 - (4 - L) * 0.10;
    P->th_height = d->dem_resolution <= 4 ? 500 : 1000;
    P->height_step = d->height_step;
    P->grid_res = d->grid_resolution;
    P->bin_angle = d->bin_angle;
    P->dem_res = d->dem_resolution;
    for (int i = 0; i < 4; ++i) P->boundary[i] = d->boundary[i];
    P->minmax[0] = d->minmax_height[0];
    P->minmax[1] = d->minmax_height[1];
    P->grid_w = d->grid_width;
    P->grid_h = d->grid_height;
    P->n_nodes = d->grid_width * d->grid_height;
    P->grid_wgs = d->grid_wgs;
    P->grid_pts = d->grid_pts;
    P->param = d->param;
    if (co) {
        P->ow = (int64_t)((d->boundary[2] - d->boundary[0]) / P->im_res) + 1;
        P->oh = (int64_t)((d->boundary[3] - d->boundary[1]) / P->im_res) + 1;
        if (P->combined) {
            P->own = (int64_t)((d->boundary[2] - d->boundary[0]) / P->im_res_next) + 1;
            P->ohn = (int64_t)((d->boundary[3] - d->boundary[1]) / P->im_res_next) + 1;
        }
    }
    // rotation table: rot_theta = (double)(diff_theta * bin_angle * PI / 180.0)
    for (int i = 0; i < kRotTable; ++i) {
        const double dtheta = (double)(i - kRotOffset) / 2.0;
        const double rot = (double)(dtheta * d->bin_angle * 3.141592653589793 / 180.0);
        P->rot_cos[i] = cos(-rot);
        P->rot_sin[i] = sin(-rot);
    }
    for (int ti = 0; ti < d->num_images; ++ti) {
        const vll_image_desc &s = d->images[ti];
        DevImage &m = P->im[ti];
        m.img = s.image;
        m.mag = s.mag;
        m.ori = s.ori;
        m.img_n = s.image_next;
        m.mag_n = s.mag_next;
        m.ori_n = s.ori_next;
        m.w = s.width;
        m.h = s.height;
        m.wn = s.width_next;
        m.hn = s.height_next;
        m.sx = s.startpos[0];
        m.sy = s.startpos[1];
        m.sxn = s.startpos_next[0];
        m.syn = s.startpos_next[1];
        memcpy(m.rpc, s.rpc, sizeof(m.rpc));
        m.adj[0] = s.image_adjust[0];
        m.adj[1] = s.image_adjust[1];
        m.selected = s.selected != 0;
        if (s.image_b) {
            m.img_b = s.image_b;
            m.mag_b = s.mag_b;
            m.wb = s.width_b;
            m.hb = s.height_b;
            m.sxb = s.startpos_b[0];
            m.syb = s.startpos_b[1];
        } else {
            m.img_b = s.image;
            m.mag_b = s.mag;
            m.wb = s.width;
            m.hb = s.height;
            m.sxb = s.startpos[0];
            m.syb = s.startpos[1];
        }
        if (m.selected && (s.width < 2 || s.height < 2)) {
            *err = "selected image with size < 2";
            return VLL_ERR_INVALID;
        }
    }
    if (!P->im[P->ref].selected) {
        *err = "the reference image must be selected";
        return VLL_ERR_INVALID;
    }
    return VLL_OK;
}

bool needs_next(const DevLevel &P) { return P.combined_incc || (P.combined && P.check_ortho); }

}  // namespace vll

using vll::DevLevel;

namespace {

// Allocates and fills the orthoimage coordinate rasters (SetOrthoImageCoord).
int run_ortho(vll_context *ctx, DevLevel *P, const DevLevel *dP_unused) {
    (void)dP_unused;
    if (!P->check_ortho) return VLL_OK;
    const size_t total = (size_t)(P->ow * P->oh);
    const size_t totaln = P->combined ? (size_t)(P->own * P->ohn) : 0;
    for (int ti = 0; ti < P->num_images; ++ti) {
        if (!P->im[ti].selected) continue;
        VLL_CUDA(ctx, ensure(ctx->ocd[ti], total * sizeof(double2)));
        VLL_CUDA(ctx, cudaMemsetAsync(ctx->ocd[ti].p, 0, total * sizeof(double2), ctx->stream));
        P->ocd[ti] = (const double2 *)ctx->ocd[ti].p;
        if (P->combined) {
            VLL_CUDA(ctx, ensure(ctx->ocdn[ti], totaln * sizeof(double2)));
            VLL_CUDA(ctx, cudaMemsetAsync(ctx->ocdn[ti].p, 0, totaln * sizeof(double2), ctx->stream));
            P->ocd_n[ti] = (const double2 *)ctx->ocdn[ti].p;
        }
    }
    return VLL_OK;
}

int upload_level_block(vll_context *ctx, const DevLevel &P) {
    VLL_CUDA(ctx, ensure(ctx->level, sizeof(DevLevel)));
    if (!ctx->hlevel) VLL_CUDA(ctx, cudaMallocHost((void **)&ctx->hlevel, sizeof(DevLevel)));
    // the pinned staging block may still be in flight from a previous call
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(ctx->hlevel, &P, sizeof(DevLevel));
    VLL_CUDA(ctx, cudaMemcpyAsync(ctx->level.p, ctx->hlevel, sizeof(DevLevel),
                                  cudaMemcpyHostToDevice, ctx->stream));
    return VLL_OK;
}

// Runs the matching kernels on a level whose pointers are all device pointers.
int run_device(vll_context *ctx, DevLevel &P, int kernel, vll_stats *stats) {
    int rc = run_ortho(ctx, &P, nullptr);
    if (rc) return rc;
    VLL_CUDA(ctx, ensure(ctx->counters, 8 * sizeof(unsigned long long)));
    VLL_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, 8 * sizeof(unsigned long long), ctx->stream));
    if (kernel != VLL_KERNEL_FP64_PLAIN && vll::split_supported(P))
        vll::split_prepare_tma(P, ctx->tuning.box_margin);
    rc = upload_level_block(ctx, P);
    if (rc) return rc;
    const DevLevel *dP = (const DevLevel *)ctx->level.p;
    if (!ctx->e0) {
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e0));
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e1));
    }
    VLL_CUDA(ctx, cudaEventRecord(ctx->e0, ctx->stream));
    if (P.check_ortho) {
        // device array of the per-image raster pointers
        double2 *ptrs[2 * VLL_MAX_IMAGES] = {};
        for (int ti = 0; ti < P.num_images; ++ti) {
            ptrs[ti] = (double2 *)P.ocd[ti];
            ptrs[VLL_MAX_IMAGES + ti] = (double2 *)P.ocd_n[ti];
        }
        VLL_CUDA(ctx, ensure(ctx->ocdptr, sizeof(ptrs)));
        VLL_CUDA(ctx, cudaMemcpyAsync(ctx->ocdptr.p, ptrs, sizeof(ptrs), cudaMemcpyHostToDevice,
                                      ctx->stream));
        double2 *const *dptr = (double2 *const *)ctx->ocdptr.p;
        VLL_CUDA(ctx, vll::launch_ortho(dP, P.ow * P.oh, dptr, dptr + VLL_MAX_IMAGES, ctx->stream));
    }
    unsigned long long *counters = (unsigned long long *)ctx->counters.p;
    vll::SplitTiming tm;
    tm.enabled = stats != nullptr;
    int64_t launches = P.check_ortho ? 1 : 0;
    bool split_ran = false;
    if (tm.enabled && !ctx->stage_ev[0])
        for (auto &ev : ctx->stage_ev) VLL_CUDA(ctx, cudaEventCreate(&ev));
    for (int i = 0; i < 9; ++i) tm.ev[i] = ctx->stage_ev[i];
    if (kernel == VLL_KERNEL_FP64_PLAIN || !vll::split_supported(P)) {
        if (kernel != VLL_KERNEL_FP64_PLAIN && kernel != VLL_KERNEL_SPLIT)
            return fail(ctx, VLL_ERR_INVALID, "unknown kernel id");
        VLL_CUDA(ctx, vll::launch_plain(dP, P.n_nodes, counters, nullptr, nullptr, ctx->stream));
        launches += 1;
    } else {
        std::string err;
        cudaError_t e = vll::run_split(ctx->split, P, dP, counters, ctx->stream, &err, &tm,
                                       ctx->tuning);
        if (e != cudaSuccess) return cuda_fail(ctx, e, err.c_str());
        launches += tm.launches;
        split_ran = true;
    }
    VLL_CUDA(ctx, cudaEventRecord(ctx->e1, ctx->stream));
    ctx->launches_total += launches;
    if (stats) {
        unsigned long long h[8];
        VLL_CUDA(ctx, cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        unsigned long long ctlh[4] = {0, 0, 0, 0};
        if (split_ran && ctx->split.ctl)
            VLL_CUDA(ctx, cudaMemcpyAsync(ctlh, ctx->split.ctl, sizeof(ctlh), cudaMemcpyDeviceToHost,
                                          ctx->stream));
        VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        VLL_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->e0, ctx->e1));
        memset(stats, 0, sizeof(*stats));
        stats->accessable_grid = (int64_t)h[0];
        stats->evals = (int64_t)h[1];
        stats->fp64_rechecks = (int64_t)h[2];
        stats->kernel_ms = ms;
        stats->launches = launches;
        stats->window_ms = ms;
        if (split_ran) {
            for (int i = 0; i < 8; ++i) {
                float t = 0;
                cudaEventElapsedTime(&t, tm.ev[i], tm.ev[i + 1]);
                stats->stage_ms[i] = t;
            }
            stats->window_ms = stats->stage_ms[4];
            stats->slots = tm.slots;
            stats->exact_nodes = (int64_t)ctlh[2];
            stats->fp64_nodes = (int64_t)h[5];
            stats->scan_rounds = (int64_t)h[6];
        }
        if (h[3] != 0) return fail(ctx, VLL_ERR_TIMEOUT, "persistent kernel reported an error flag");
    }
    return VLL_OK;
}

// Device resources of a level set: the level blocks, the orthoimage rasters
// of the levels that use GNCC, counters and the split pipeline's scratch.
struct SetResources {
    std::vector<DevLevel> hl;           // host copies of the level blocks
    Buf dl;                             // device array of the level blocks
    DevLevel *staging = nullptr;        // pinned staging of the upload
    size_t staging_cap = 0;
    std::vector<Buf> ocd;               // [level][image][level, next level]
    Buf ocdptr;                         // [level][2 * VLL_MAX_IMAGES] raster pointers
    Buf counters;
    vll::SplitBuffers split;
    std::vector<int64_t> ortho_total;   // per level: raster pixels (0 = no GNCC)
};

void release_set(SetResources &r) {
    release(r.dl);
    if (r.staging) cudaFreeHost(r.staging);
    r.staging = nullptr;
    r.staging_cap = 0;
    for (auto &b : r.ocd) release(b);
    r.ocd.clear();
    release(r.ocdptr);
    release(r.counters);
    vll::split_release(r.split);
}

SetResources *ctx_set(vll_context *ctx) {
    if (!ctx->set) ctx->set = new SetResources();
    return (SetResources *)ctx->set;
}

// Derives, checks and uploads the level blocks of a batch; allocates the
// orthoimage rasters (filled by enqueue_set_ortho).
int prepare_set(vll_context *ctx, SetResources &r, const vll_level_io *levels, int n) {
    if (!levels || n < 1) return fail(ctx, VLL_ERR_INVALID, "empty level list");
    r.hl.assign((size_t)n, DevLevel());
    r.ortho_total.assign((size_t)n, 0);
    for (int l = 0; l < n; ++l) {
        const vll_level_io &io = levels[l];
        if (!io.desc || !io.d_gridpt3 || !io.d_nccresult)
            return fail(ctx, VLL_ERR_INVALID, "level " + std::to_string(l) + ": null pointer");
        DevLevel &P = r.hl[l];
        std::string err;
        const int rc = vll::derive_level(io.desc, &P, &err);
        if (rc) return fail(ctx, rc, "level " + std::to_string(l) + ": " + err);
        if (!vll::split_supported(P))
            return fail(ctx, VLL_ERR_UNSUPPORTED,
                        "level " + std::to_string(l) +
                            ": not a level the batched split pipeline implements (stereo, "
                            "window half-size 2..7)");
        if (!P.cmr && !P.is_ra && (!io.d_voxels || !io.d_voxel_offsets))
            return fail(ctx, VLL_ERR_INVALID,
                        "level " + std::to_string(l) + ": voxel route needs voxel rows and offsets");
        P.gp3 = io.d_gridpt3;
        P.ncc = io.d_nccresult;
        P.vox = io.d_voxels;
        P.vox_off = io.d_voxel_offsets;
    }
    // orthoimage rasters, one set per GNCC level
    r.ocd.resize((size_t)n * VLL_MAX_IMAGES * 2);
    VLL_CUDA(ctx, ensure(r.ocdptr, (size_t)n * 2 * VLL_MAX_IMAGES * sizeof(void *)));
    std::vector<const void *> ptrs((size_t)n * 2 * VLL_MAX_IMAGES, nullptr);
    for (int l = 0; l < n; ++l) {
        DevLevel &P = r.hl[l];
        if (!P.check_ortho) continue;
        r.ortho_total[l] = P.ow * P.oh;
        for (int ti = 0; ti < P.num_images; ++ti) {
            if (!P.im[ti].selected) continue;
            Buf &a = r.ocd[((size_t)l * VLL_MAX_IMAGES + ti) * 2];
            VLL_CUDA(ctx, ensure(a, (size_t)(P.ow * P.oh) * sizeof(double2)));
            P.ocd[ti] = (const double2 *)a.p;
            ptrs[(size_t)l * 2 * VLL_MAX_IMAGES + ti] = a.p;
            if (P.combined) {
                Buf &b = r.ocd[((size_t)l * VLL_MAX_IMAGES + ti) * 2 + 1];
                VLL_CUDA(ctx, ensure(b, (size_t)(P.own * P.ohn) * sizeof(double2)));
                P.ocd_n[ti] = (const double2 *)b.p;
                ptrs[(size_t)l * 2 * VLL_MAX_IMAGES + VLL_MAX_IMAGES + ti] = b.p;
            }
        }
    }
    for (int l = 0; l < n; ++l) vll::split_prepare_tma(r.hl[l], ctx->tuning.box_margin);
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // staging may be in flight
    if (r.staging_cap < (size_t)n) {
        if (r.staging) cudaFreeHost(r.staging);
        r.staging = nullptr;
        r.staging_cap = 0;
        VLL_CUDA(ctx, cudaMallocHost((void **)&r.staging, (size_t)n * sizeof(DevLevel)));
        r.staging_cap = (size_t)n;
    }
    memcpy(r.staging, r.hl.data(), (size_t)n * sizeof(DevLevel));
    VLL_CUDA(ctx, ensure(r.dl, (size_t)n * sizeof(DevLevel)));
    VLL_CUDA(ctx, cudaMemcpyAsync(r.dl.p, r.staging, (size_t)n * sizeof(DevLevel),
                                  cudaMemcpyHostToDevice, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(r.ocdptr.p, ptrs.data(), ptrs.size() * sizeof(void *),
                                  cudaMemcpyHostToDevice, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // ptrs is pageable and local
    VLL_CUDA(ctx, ensure(r.counters, 8 * sizeof(unsigned long long)));
    return VLL_OK;
}

// SetOrthoImageCoord of every GNCC level of the set (clear + fill).
cudaError_t enqueue_set_ortho(SetResources &r, cudaStream_t s) {
    const int n = (int)r.hl.size();
    for (int l = 0; l < n; ++l) {
        if (!r.ortho_total[l]) continue;
        const DevLevel &P = r.hl[l];
        for (int ti = 0; ti < P.num_images; ++ti) {
            if (!P.im[ti].selected) continue;
            Buf &a = r.ocd[((size_t)l * VLL_MAX_IMAGES + ti) * 2];
            cudaError_t e = cudaMemsetAsync(a.p, 0, a.cap, s);
            if (e != cudaSuccess) return e;
            if (P.combined) {
                Buf &b = r.ocd[((size_t)l * VLL_MAX_IMAGES + ti) * 2 + 1];
                e = cudaMemsetAsync(b.p, 0, b.cap, s);
                if (e != cudaSuccess) return e;
            }
        }
        double2 *const *dptr = (double2 *const *)r.ocdptr.p + (size_t)l * 2 * VLL_MAX_IMAGES;
        cudaError_t e = vll::launch_ortho((const DevLevel *)r.dl.p + l, r.ortho_total[l], dptr,
                                          dptr + VLL_MAX_IMAGES, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Copies per-level Accessable_grid and the totals after a pass (waits).
int finish_set(vll_context *ctx, SetResources &r, const vll::SplitBuffers &b, int n,
               int64_t *accessable, vll_stats *stats, float ms, int64_t launches) {
    unsigned long long h[8] = {};
    std::vector<unsigned long long> acc((size_t)n, 0);
    VLL_CUDA(ctx, cudaMemcpyAsync(h, r.counters.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(acc.data(), b.acc_level, (size_t)n * 8, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    unsigned long long ctl[8] = {};
    VLL_CUDA(ctx, cudaMemcpyAsync(ctl, b.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (accessable)
        for (int l = 0; l < n; ++l) accessable[l] = (int64_t)acc[l];
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->accessable_grid = (int64_t)h[0];
        stats->evals = (int64_t)h[1];
        stats->fp64_rechecks = (int64_t)h[2];
        stats->kernel_ms = ms;
        stats->window_ms = ms;
        stats->launches = launches;
        stats->fp64_nodes = (int64_t)h[5];
        stats->scan_rounds = (int64_t)h[6];
        stats->exact_nodes = (int64_t)ctl[2];
    }
    if (h[3] != 0) return fail(ctx, VLL_ERR_TIMEOUT, "persistent kernel reported an error flag");
    return VLL_OK;
}

// Scratch of the all-directions SGM, or nullptr (one launch per direction)
// when it exceeds the budget or cannot be allocated.
float *sgm_scratch(vll_context *ctx, int64_t n_slots) {
    // SETSM_VLL_SGM_SEQUENTIAL=1 selects the per-direction form (same results)
    const char *seq = getenv("SETSM_VLL_SGM_SEQUENTIAL");
    if (seq && seq[0] == '1') return nullptr;
    const size_t b = vll::sgm_scratch_bytes(n_slots);
    if (!b) return nullptr;
    if (ensure(ctx->sgm_lr, b) != cudaSuccess) {
        cudaGetLastError();   // an allocation failure leaves no sticky error
        return nullptr;
    }
    return (float *)ctx->sgm_lr.p;
}

int upload(vll_context *ctx, Buf &b, const void *src, size_t n) {
    VLL_CUDA(ctx, ensure(b, n));
    b.src = nullptr;
    if (n) VLL_CUDA(ctx, cudaMemcpyAsync(b.p, src, n, cudaMemcpyHostToDevice, ctx->stream));
    return VLL_OK;
}

// An image plane or grid array: with VLL_RESIDENT_PLANES, sent only when
// the buffer does not hold these host bytes already (pointer, size and
// sampled fingerprint).
int upload_plane(vll_context *ctx, Buf &b, const void *src, size_t n) {
    if (!(ctx->residency & VLL_RESIDENT_PLANES)) return upload(ctx, b, src, n);
    const uint64_t fp = sample_fingerprint(src, n);
    if (b.p && b.src == src && b.src_bytes == n && b.src_fp == fp) return VLL_OK;
    int rc = upload(ctx, b, src, n);
    if (rc) return rc;
    b.src = src;
    b.src_bytes = n;
    b.src_fp = fp;
    return VLL_OK;
}

// Template half-size of VerticalLineLocus_seeddem (setsm_code.cpp:7722-7729):
// the 5 m template area at the matched level, at every level.
int seeddem_half(const vll_level_desc *d) {
    int T = d->template_size;
    const int t = (int)((5.0 / (d->resolution * (double)(1 << d->pyramid_step))) / 2.0) * 2 + 1;
    if (T < t) T = t;
    return (int)(T / 2.0);
}

// Template half-size of VerticalLineLocus_blunder (setsm_code.cpp:7884-7910):
// the template is a uint8 there, enlarged for the blunder level's GSD.
int blunder_half(const vll_level_desc *d, int iteration, bool bblunder, int blevel) {
    uint8_t T = (uint8_t)d->template_size;
    const int t = (int)((5.0 / (d->resolution * (double)(1 << blevel))) / 2.0) * 2 + 1;
    if (T < t) T = (uint8_t)t;
    int H = (int)(T / 2.0);
    if (bblunder) {
        const uint8_t it = (uint8_t)iteration;
        if (d->pyramid_step == 4) {
            H = T - it * 2;
            if (H < (int)(T / 2.0)) H = (int)(T / 2.0);
        } else if (d->pyramid_step == 3) {
            H = T - 2 - it * 2;
            if (H < (int)(T / 2.0)) H = (int)(T / 2.0);
        }
    }
    return H;
}

// Uploads the selected images' intensity and magnitude planes the variant
// samples (the matched level's, or the blunder level's when use_b).
int upload_ortho_images(vll_context *ctx, const vll_level_desc *desc, DevLevel &P, bool use_b) {
    int rc;
    for (int ti = 0; ti < P.num_images; ++ti) {
        const vll_image_desc &s = desc->images[ti];
        if (!s.selected) continue;
        vll::DevImage &m = P.im[ti];
        const uint16_t *img = use_b ? m.img_b : m.img, *mag = use_b ? m.mag_b : m.mag;
        const size_t n = use_b ? (size_t)m.wb * m.hb : (size_t)m.w * m.h;
        if (!img || !mag) return fail(ctx, VLL_ERR_INVALID, "null image plane");
        if ((rc = upload(ctx, ctx->img[ti][0], img, n * 2))) return rc;
        if ((rc = upload(ctx, ctx->img[ti][1], mag, n * 2))) return rc;
        if (use_b) {
            m.img_b = (const uint16_t *)ctx->img[ti][0].p;
            m.mag_b = (const uint16_t *)ctx->img[ti][1].p;
        } else {
            m.img = (const uint16_t *)ctx->img[ti][0].p;
            m.mag = (const uint16_t *)ctx->img[ti][1].p;
        }
    }
    return VLL_OK;
}

// The orthoimage variants on device data: rasterise the orthoimage
// coordinates (SetOrthoImageCoord, OR or BD pyramid) and run the per-node
// pass; d_ncc selects the blunder pass.  gp3 is updated in place.
int run_ortho_variant(vll_context *ctx, DevLevel &P, vll_ugrid *d_gp3, int H, double im_res,
                      bool use_b, float *d_ncc, vll_stats *stats) {
    if (use_b && P.blunder_level < 0) return fail(ctx, VLL_ERR_INVALID, "negative blunder level");
    if (use_b && P.blunder_level > 12) return fail(ctx, VLL_ERR_INVALID, "blunder level above 12");
    for (int ti = 0; ti < P.num_images; ++ti) {
        const vll::DevImage &m = P.im[ti];
        if (m.selected && use_b && (m.wb < 2 || m.hb < 2))
            return fail(ctx, VLL_ERR_INVALID, "selected blunder-level image with size < 2");
    }
    const int64_t ow = (int64_t)((P.boundary[2] - P.boundary[0]) / im_res) + 1;
    const int64_t oh = (int64_t)((P.boundary[3] - P.boundary[1]) / im_res) + 1;
    if (ow <= 0 || oh <= 0) return fail(ctx, VLL_ERR_INVALID, "empty orthoimage boundary");
    const size_t total = (size_t)(ow * oh);
    double2 *ptrs[2 * VLL_MAX_IMAGES] = {};
    for (int ti = 0; ti < P.num_images; ++ti) {
        if (!P.im[ti].selected) continue;
        VLL_CUDA(ctx, ensure(ctx->ocd[ti], total * sizeof(double2)));
        VLL_CUDA(ctx, cudaMemsetAsync(ctx->ocd[ti].p, 0, total * sizeof(double2), ctx->stream));
        ptrs[ti] = (double2 *)ctx->ocd[ti].p;
    }
    P.gp3 = d_gp3;
    int rc = upload_level_block(ctx, P);
    if (rc) return rc;
    VLL_CUDA(ctx, ensure(ctx->ocdptr, sizeof(ptrs)));
    VLL_CUDA(ctx, cudaMemcpyAsync(ctx->ocdptr.p, ptrs, sizeof(ptrs), cudaMemcpyHostToDevice,
                                  ctx->stream));
    const DevLevel *dP = (const DevLevel *)ctx->level.p;
    double2 *const *dptr = (double2 *const *)ctx->ocdptr.p;
    if (!ctx->e0) {
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e0));
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e1));
    }
    VLL_CUDA(ctx, cudaEventRecord(ctx->e0, ctx->stream));
    VLL_CUDA(ctx, vll::launch_ortho_raster(dP, dptr, ow, oh, im_res, use_b ? 1 : 0, ctx->stream));
    if (d_ncc)
        VLL_CUDA(ctx, vll::launch_blunder(dP, P.n_nodes, dptr, ow, oh, im_res, H, d_gp3, d_ncc,
                                          ctx->stream));
    else
        VLL_CUDA(ctx, vll::launch_seeddem(dP, P.n_nodes, dptr, ow, oh, im_res, H, use_b ? 1 : 0,
                                          d_gp3, ctx->stream));
    VLL_CUDA(ctx, cudaEventRecord(ctx->e1, ctx->stream));
    ctx->launches_total += 2;
    if (stats) {
        VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->e0, ctx->e1);
        memset(stats, 0, sizeof(*stats));
        stats->kernel_ms = ms;
    }
    return VLL_OK;
}

// Shared front of the four variant entry points: descriptor checks and the
// window / raster constants.  blunder: H from blunder_half, raster at the
// blunder level; seeddem: H from seeddem_half, raster at the matched level
// (sampling the blunder level's images with check_Matchtag).
int prepare_variant(vll_context *ctx, const vll_level_desc *desc, bool blunder, int iteration,
                    int bblunder, DevLevel &P, int &H, double &im_res, bool &use_b) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc) return fail(ctx, VLL_ERR_INVALID, "null descriptor");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    if (!blunder && desc->pyramid_step > 12)
        return fail(ctx, VLL_ERR_INVALID, "pyramid step above 12");
    if (blunder) {
        use_b = true;
        H = blunder_half(desc, iteration, bblunder != 0, P.blunder_level);
        im_res = desc->resolution * (double)(1 << P.blunder_level);
    } else {
        use_b = P.check_matchtag;
        H = seeddem_half(desc);
        im_res = desc->resolution * (double)(1 << P.L);
    }
    return VLL_OK;
}

}  // namespace

extern "C" {

int vll_abi_version(void) { return VLL_ABI_VERSION; }

const char *vll_last_error(const vll_context *ctx) {
    if (ctx) return ctx->err.c_str();
    return g_last_error.c_str();
}

int vll_create(int device, vll_context **out) {
    if (!out) return fail(nullptr, VLL_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(nullptr, VLL_ERR_INVALID, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    vll_context *ctx = new vll_context();
    ctx->device = device;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(nullptr, e, "cudaStreamCreate");
    }
    *out = ctx;
    return VLL_OK;
}

void vll_destroy(vll_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    release(ctx->level);
    release(ctx->counters);
    for (auto &a : ctx->img)
        for (auto &b : a) release(b);
    release(ctx->wgs);
    release(ctx->pts);
    release(ctx->gp3);
    release(ctx->ncc);
    release(ctx->vox);
    release(ctx->voxoff);
    release(ctx->gsum);
    release(ctx->gcnt);
    for (auto &b : ctx->ocd) release(b);
    for (auto &b : ctx->ocdn) release(b);
    release(ctx->ocdptr);
    release(ctx->pre_tmp);
    release(ctx->pre_wt);
    release(ctx->pre_img);
    release(ctx->pre_mag);
    release(ctx->pre_ori);
    release(ctx->sumcost);
    release(ctx->sgm_lr);
    release(ctx->rvox);
    release(ctx->rvox_off);
    release(ctx->tin_pts);
    release(ctx->tin_tris);
    release(ctx->tin_scratch);
    vll::tin_release(ctx->tin_work);
    vll::split_release(ctx->split);
    if (ctx->set) {
        release_set(*(SetResources *)ctx->set);
        delete (SetResources *)ctx->set;
    }
    if (ctx->hlevel) cudaFreeHost(ctx->hlevel);
    if (ctx->e0) cudaEventDestroy(ctx->e0);
    if (ctx->e1) cudaEventDestroy(ctx->e1);
    for (auto &ev : ctx->stage_ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream && ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int vll_set_stream(vll_context *ctx, void *stream) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (ctx->stream && ctx->own_stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamCreate");
        ctx->own_stream = true;
    }
    return VLL_OK;
}

void *vll_get_stream(vll_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int64_t vll_launch_count(const vll_context *ctx) { return ctx ? ctx->launches_total : 0; }

int64_t vll_tin_rerun_count(const vll_context *ctx) { return ctx ? ctx->tin_reruns : 0; }

int vll_debug_tin_threshold(int pyramid_step, int iteration, int is_ra, double grid_resolution,
                            double hinterval, double sd, double sd2, int64_t m_terms,
                            int64_t dh_count, const uint32_t *hbin, uint32_t hdiffcount,
                            int exact, double *lo, double *hi) {
    if (!lo || !hi || (hdiffcount > 0 && !hbin) || pyramid_step < 0 || pyramid_step > 12 ||
        m_terms < 0 || dh_count < 0)
        return VLL_ERR_INVALID;
    vll::TinArgs a;
    memset(&a, 0, sizeof(a));
    a.L = pyramid_step;
    a.iteration = iteration;
    a.is_ra = is_ra != 0;
    a.gs = grid_resolution;
    a.hinterval = hinterval;
    vll::tin_threshold_band(a, sd, sd2, m_terms, (long)dh_count, hbin, hdiffcount, exact != 0, lo,
                            hi);
    return VLL_OK;
}

int64_t vll_voxel_count(const vll_nccresult *ncc, int64_t n) {
    if (!ncc || n <= 0) return 0;
    int64_t s = 0;
    for (int64_t i = 0; i < n; ++i) s += ncc[i].NumOfHeight;
    return s;
}

int vll_vertical_line_locus(vll_context *ctx, const vll_level_desc *desc, const vll_ugrid *gridpt3,
                            vll_nccresult *nccresult, vll_voxel *voxels, int64_t voxel_capacity,
                            int kernel, vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !gridpt3 || !nccresult)
        return fail(ctx, VLL_ERR_INVALID, "null descriptor, gridpt3 or nccresult");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err);
    if (rc) return fail(ctx, rc, err);
    if (!desc->grid_wgs || !desc->grid_pts) return fail(ctx, VLL_ERR_INVALID, "null grid arrays");
    const int64_t N = P.n_nodes;
    const bool voxel_route = !P.cmr && !P.is_ra;
    std::vector<int64_t> off;
    bool resident_vox = false;
    if (voxel_route) {
        off.resize((size_t)N + 1);
        off[0] = 0;
        for (int64_t i = 0; i < N; ++i) off[i + 1] = off[i] + nccresult[i].NumOfHeight;
        resident_vox = !voxels && (ctx->residency & VLL_RESIDENT_VOXELS);
        if (resident_vox) {
            if (ctx->rvox_total != off[N] || ctx->rvox_nodes != N)
                return fail(ctx, VLL_ERR_INVALID,
                            "no resident voxel packing matching sum(NumOfHeight)");
        } else if (off[N] > 0 && (!voxels || voxel_capacity < off[N])) {
            return fail(ctx, VLL_ERR_CAPACITY, "voxel buffer smaller than sum(NumOfHeight)");
        }
    }
    // images (only what the level reads)
    const bool next = vll::needs_next(P);
    for (int ti = 0; ti < P.num_images; ++ti) {
        const vll_image_desc &s = desc->images[ti];
        if (!s.selected) continue;
        if (!s.image || !s.mag || !s.ori) return fail(ctx, VLL_ERR_INVALID, "null image plane");
        const size_t n = (size_t)s.width * s.height;
        if ((rc = upload_plane(ctx, ctx->img[ti][0], s.image, n * 2))) return rc;
        if ((rc = upload_plane(ctx, ctx->img[ti][1], s.mag, n * 2))) return rc;
        if ((rc = upload_plane(ctx, ctx->img[ti][2], s.ori, n))) return rc;
        P.im[ti].img = (const uint16_t *)ctx->img[ti][0].p;
        P.im[ti].mag = (const uint16_t *)ctx->img[ti][1].p;
        P.im[ti].ori = (const uint8_t *)ctx->img[ti][2].p;
        if (next) {
            if (!s.image_next || !s.mag_next || !s.ori_next || s.width_next < 2 || s.height_next < 2)
                return fail(ctx, VLL_ERR_INVALID, "combined level needs the next pyramid level");
            const size_t nn = (size_t)s.width_next * s.height_next;
            if ((rc = upload_plane(ctx, ctx->img[ti][3], s.image_next, nn * 2))) return rc;
            if ((rc = upload_plane(ctx, ctx->img[ti][4], s.mag_next, nn * 2))) return rc;
            if ((rc = upload_plane(ctx, ctx->img[ti][5], s.ori_next, nn))) return rc;
            P.im[ti].img_n = (const uint16_t *)ctx->img[ti][3].p;
            P.im[ti].mag_n = (const uint16_t *)ctx->img[ti][4].p;
            P.im[ti].ori_n = (const uint8_t *)ctx->img[ti][5].p;
        }
    }
    if ((rc = upload_plane(ctx, ctx->wgs, desc->grid_wgs, (size_t)N * 16))) return rc;
    if ((rc = upload_plane(ctx, ctx->pts, desc->grid_pts, (size_t)N * 16))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->ncc, nccresult, (size_t)N * sizeof(vll_nccresult)))) return rc;
    P.grid_wgs = (const double *)ctx->wgs.p;
    P.grid_pts = (const double *)ctx->pts.p;
    P.gp3 = (const vll_ugrid *)ctx->gp3.p;
    P.ncc = (vll_nccresult *)ctx->ncc.p;
    if (voxel_route && resident_vox) {
        P.vox = (vll_voxel *)ctx->rvox.p;
        P.vox_off = (const int64_t *)ctx->rvox_off.p;
    } else if (voxel_route) {
        if ((rc = upload(ctx, ctx->voxoff, off.data(), off.size() * sizeof(int64_t)))) return rc;
        if ((rc = upload(ctx, ctx->vox, voxels, (size_t)off[N] * sizeof(vll_voxel)))) return rc;
        P.vox = (vll_voxel *)ctx->vox.p;
        P.vox_off = (const int64_t *)ctx->voxoff.p;
    }
    vll_stats local;
    rc = run_device(ctx, P, kernel, stats ? stats : &local);
    if (rc) return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(nccresult, ctx->ncc.p, (size_t)N * sizeof(vll_nccresult),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    if (voxel_route && !resident_vox && off[N] > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(voxels, ctx->vox.p, (size_t)off[N] * sizeof(vll_voxel),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_vertical_line_locus_device(vll_context *ctx, const vll_level_desc *desc,
                                   const vll_ugrid *d_gridpt3, vll_nccresult *d_nccresult,
                                   vll_voxel *d_voxels, const int64_t *d_voxel_offsets, int kernel,
                                   vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus_device");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !d_gridpt3 || !d_nccresult)
        return fail(ctx, VLL_ERR_INVALID, "null descriptor, gridpt3 or nccresult");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err);
    if (rc) return fail(ctx, rc, err);
    if (!P.cmr && !P.is_ra && (!d_voxels || !d_voxel_offsets))
        return fail(ctx, VLL_ERR_INVALID, "voxel route needs voxel rows and offsets");
    P.gp3 = d_gridpt3;
    P.ncc = d_nccresult;
    P.vox = d_voxels;
    P.vox_off = d_voxel_offsets;
    return run_device(ctx, P, kernel, stats);
}

int vll_debug_slot_rho(vll_context *ctx, const vll_level_desc *desc, const vll_ugrid *gridpt3,
                       vll_nccresult *nccresult, int kernel, double *rho_out, int64_t capacity,
                       uint64_t *diag_out) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !gridpt3 || !nccresult || !rho_out) return fail(ctx, VLL_ERR_INVALID, "null argument");
    if (!desc->check_matching_rate)
        return fail(ctx, VLL_ERR_UNSUPPORTED, "slot diagnostics cover the memory-tight route");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err);
    if (rc) return fail(ctx, rc, err);
    const int64_t N = P.n_nodes;
    std::vector<int64_t> off((size_t)N + 1);
    off[0] = 0;
    for (int64_t i = 0; i < N; ++i) {
        const int nh = (uint16_t)(int)((gridpt3[i].maxHeight - gridpt3[i].minHeight) / desc->height_step);
        off[i + 1] = off[i] + nh;
    }
    if (capacity < off[N]) return fail(ctx, VLL_ERR_CAPACITY, "rho buffer too small");
    for (int ti = 0; ti < P.num_images; ++ti) {
        const vll_image_desc &s = desc->images[ti];
        if (!s.selected) continue;
        const size_t n = (size_t)s.width * s.height;
        if ((rc = upload(ctx, ctx->img[ti][0], s.image, n * 2))) return rc;
        if ((rc = upload(ctx, ctx->img[ti][1], s.mag, n * 2))) return rc;
        if ((rc = upload(ctx, ctx->img[ti][2], s.ori, n))) return rc;
        P.im[ti].img = (const uint16_t *)ctx->img[ti][0].p;
        P.im[ti].mag = (const uint16_t *)ctx->img[ti][1].p;
        P.im[ti].ori = (const uint8_t *)ctx->img[ti][2].p;
    }
    if ((rc = upload(ctx, ctx->wgs, desc->grid_wgs, (size_t)N * 16))) return rc;
    if ((rc = upload(ctx, ctx->pts, desc->grid_pts, (size_t)N * 16))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->ncc, nccresult, (size_t)N * sizeof(vll_nccresult)))) return rc;
    P.grid_wgs = (const double *)ctx->wgs.p;
    P.grid_pts = (const double *)ctx->pts.p;
    P.gp3 = (const vll_ugrid *)ctx->gp3.p;
    P.ncc = (vll_nccresult *)ctx->ncc.p;
    Buf dbg, dbgoff;
    VLL_CUDA(ctx, ensure(dbg, (size_t)off[N] * sizeof(double)));
    VLL_CUDA(ctx, cudaMemsetAsync(dbg.p, 0xff, (size_t)off[N] * sizeof(double), ctx->stream));
    rc = upload(ctx, dbgoff, off.data(), off.size() * sizeof(int64_t));
    if (rc) return rc;
    Buf diag;
    if (kernel == VLL_KERNEL_SPLIT) {
        P.dbg_rho = (double *)dbg.p;
        P.dbg_off = (const int64_t *)dbgoff.p;
        if (diag_out) {
            VLL_CUDA(ctx, ensure(diag, 16 * sizeof(unsigned long long)));
            VLL_CUDA(ctx, cudaMemsetAsync(diag.p, 0, 16 * sizeof(unsigned long long), ctx->stream));
            P.diag = (unsigned long long *)diag.p;
        }
        rc = run_device(ctx, P, kernel, nullptr);
        if (!rc && diag_out) {
            VLL_CUDA(ctx, cudaMemcpyAsync(diag_out, diag.p, 16 * sizeof(unsigned long long),
                                          cudaMemcpyDeviceToHost, ctx->stream));
        }
    } else {
        VLL_CUDA(ctx, ensure(ctx->counters, 8 * sizeof(unsigned long long)));
        VLL_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, 8 * sizeof(unsigned long long), ctx->stream));
        rc = upload_level_block(ctx, P);
        if (!rc)
            VLL_CUDA(ctx, vll::launch_plain((const DevLevel *)ctx->level.p, N,
                                            (unsigned long long *)ctx->counters.p, (double *)dbg.p,
                                            (const int64_t *)dbgoff.p, ctx->stream));
    }
    if (!rc) {
        VLL_CUDA(ctx, cudaMemcpyAsync(rho_out, dbg.p, (size_t)off[N] * sizeof(double),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        VLL_CUDA(ctx, cudaMemcpyAsync(nccresult, ctx->ncc.p, (size_t)N * sizeof(vll_nccresult),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    release(dbg);
    release(dbgoff);
    release(diag);
    return rc;
}

int vll_awncc_peaks(vll_context *ctx, const vll_level_desc *desc, const vll_ugrid *gridpt3,
                    vll_nccresult *nccresult, const vll_voxel *voxels, int64_t voxel_capacity,
                    vll_stats *stats) {
    NvtxRange nvtx_range("vll_awncc_peaks");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !gridpt3 || !nccresult) return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err);
    if (rc) return fail(ctx, rc, err);
    const bool sgm = P.L <= desc->sgm_py;   // AWNCC's check_SGM (setsm_code.cpp:7013-7015)
    const int64_t N = P.n_nodes;
    std::vector<int64_t> off((size_t)N + 1);
    off[0] = 0;
    int max_h = 0;
    for (int64_t i = 0; i < N; ++i) {
        off[i + 1] = off[i] + nccresult[i].NumOfHeight;
        if (nccresult[i].NumOfHeight > max_h) max_h = nccresult[i].NumOfHeight;
    }
    const bool resident_vox = !voxels && (ctx->residency & VLL_RESIDENT_VOXELS);
    if (resident_vox) {
        if (ctx->rvox_total != off[N] || ctx->rvox_nodes != N)
            return fail(ctx, VLL_ERR_INVALID, "no resident voxel packing matching sum(NumOfHeight)");
    } else if (off[N] > 0 && (!voxels || voxel_capacity < off[N])) {
        return fail(ctx, VLL_ERR_CAPACITY, "voxel buffer smaller than sum(NumOfHeight)");
    }
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->ncc, nccresult, (size_t)N * sizeof(vll_nccresult)))) return rc;
    P.gp3 = (const vll_ugrid *)ctx->gp3.p;
    P.ncc = (vll_nccresult *)ctx->ncc.p;
    if (resident_vox) {
        P.vox = (vll_voxel *)ctx->rvox.p;
        P.vox_off = (const int64_t *)ctx->rvox_off.p;
    } else {
        if ((rc = upload(ctx, ctx->voxoff, off.data(), off.size() * sizeof(int64_t)))) return rc;
        if ((rc = upload(ctx, ctx->vox, voxels, (size_t)off[N] * sizeof(vll_voxel)))) return rc;
        P.vox = (vll_voxel *)ctx->vox.p;
        P.vox_off = (const int64_t *)ctx->voxoff.p;
    }
    if ((rc = upload_level_block(ctx, P))) return rc;
    if (!ctx->e0) {
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e0));
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e1));
    }
    VLL_CUDA(ctx, cudaEventRecord(ctx->e0, ctx->stream));
    const float *sumcost = nullptr;
    if (sgm) {
        VLL_CUDA(ctx, ensure(ctx->sumcost, (size_t)(off[N] > 0 ? off[N] : 1) * sizeof(float)));
        VLL_CUDA(ctx, vll::launch_sgm((const DevLevel *)ctx->level.p, P.grid_w, P.grid_h, max_h,
                                      (float *)ctx->sumcost.p, off[N], ctx->stream,
                                      sgm_scratch(ctx, off[N])));
        sumcost = (const float *)ctx->sumcost.p;
    }
    VLL_CUDA(ctx, vll::launch_awncc((const DevLevel *)ctx->level.p, N, sumcost, ctx->stream));
    VLL_CUDA(ctx, cudaEventRecord(ctx->e1, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(nccresult, ctx->ncc.p, (size_t)N * sizeof(vll_nccresult),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->e0, ctx->e1);
        memset(stats, 0, sizeof(*stats));
        stats->kernel_ms = ms;
    }
    return VLL_OK;
}

int vll_vertical_line_locus_seeddem_device(vll_context *ctx, const vll_level_desc *desc,
                                           vll_ugrid *d_gridpt3, vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus_seeddem_device");
    DevLevel P;
    int H;
    double im_res;
    bool use_b;
    int rc = prepare_variant(ctx, desc, false, 0, 0, P, H, im_res, use_b);
    if (rc) return rc;
    if (!d_gridpt3) return fail(ctx, VLL_ERR_INVALID, "null gridpt3");
    return run_ortho_variant(ctx, P, d_gridpt3, H, im_res, use_b, nullptr, stats);
}

int vll_vertical_line_locus_seeddem(vll_context *ctx, const vll_level_desc *desc,
                                    vll_ugrid *gridpt3, vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus_seeddem");
    DevLevel P;
    int H;
    double im_res;
    bool use_b;
    int rc = prepare_variant(ctx, desc, false, 0, 0, P, H, im_res, use_b);
    if (rc) return rc;
    if (!gridpt3 || !desc->grid_pts) return fail(ctx, VLL_ERR_INVALID, "null gridpt3 or grid_pts");
    const int64_t N = P.n_nodes;
    if ((rc = upload_ortho_images(ctx, desc, P, use_b))) return rc;
    if ((rc = upload(ctx, ctx->pts, desc->grid_pts, (size_t)N * 16))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    P.grid_pts = (const double *)ctx->pts.p;
    if ((rc = run_ortho_variant(ctx, P, (vll_ugrid *)ctx->gp3.p, H, im_res, use_b, nullptr,
                                stats)))
        return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_vertical_line_locus_blunder_device(vll_context *ctx, const vll_level_desc *desc,
                                           vll_ugrid *d_gridpt3, int iteration, int bblunder,
                                           float *d_nccresult, vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus_blunder_device");
    DevLevel P;
    int H;
    double im_res;
    bool use_b;
    int rc = prepare_variant(ctx, desc, true, iteration, bblunder, P, H, im_res, use_b);
    if (rc) return rc;
    if (!d_gridpt3 || !d_nccresult) return fail(ctx, VLL_ERR_INVALID, "null gridpt3 or nccresult");
    return run_ortho_variant(ctx, P, d_gridpt3, H, im_res, true, d_nccresult, stats);
}

int vll_vertical_line_locus_blunder(vll_context *ctx, const vll_level_desc *desc,
                                    vll_ugrid *gridpt3, int iteration, int bblunder,
                                    float *nccresult, vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus_blunder");
    DevLevel P;
    int H;
    double im_res;
    bool use_b;
    int rc = prepare_variant(ctx, desc, true, iteration, bblunder, P, H, im_res, use_b);
    if (rc) return rc;
    if (!gridpt3 || !nccresult || !desc->grid_pts)
        return fail(ctx, VLL_ERR_INVALID, "null gridpt3, nccresult or grid_pts");
    const int64_t N = P.n_nodes;
    if ((rc = upload_ortho_images(ctx, desc, P, true))) return rc;
    if ((rc = upload(ctx, ctx->pts, desc->grid_pts, (size_t)N * 16))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    VLL_CUDA(ctx, ensure(ctx->gsum, (size_t)N * sizeof(float)));
    P.grid_pts = (const double *)ctx->pts.p;
    if ((rc = run_ortho_variant(ctx, P, (vll_ugrid *)ctx->gp3.p, H, im_res, true,
                                (float *)ctx->gsum.p, stats)))
        return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(nccresult, ctx->gsum.p, (size_t)N * sizeof(float),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_vertical_line_locus_ortho(vll_context *ctx, const vll_level_desc *desc, double mpp,
                                  const vll_point3 *ref1, const vll_point3 *ref2,
                                  const vll_point3 *target, const vll_ugrid *gridpt3,
                                  int64_t target_index, double *f_height, double *f_sncc,
                                  int *selected_count) {
    NvtxRange nvtx_range("vll_vertical_line_locus_ortho");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !ref1 || !ref2 || !target || !gridpt3 || !f_height || !f_sncc || !selected_count)
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    if (target_index < 0 || target_index >= P.n_nodes)
        return fail(ctx, VLL_ERR_INVALID, "target_index outside the grid");
    const int64_t N = P.n_nodes;
    if ((rc = upload_ortho_images(ctx, desc, P, false))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    P.gp3 = (const vll_ugrid *)ctx->gp3.p;
    const vll_point3 three[3] = {*ref1, *ref2, *target};
    if ((rc = upload(ctx, ctx->tin_pts, three, sizeof(three)))) return rc;
    VLL_CUDA(ctx, ensure(ctx->tin_scratch, 4 * sizeof(double)));
    if ((rc = upload_level_block(ctx, P))) return rc;
    VLL_CUDA(ctx, vll::launch_ortho_search((const DevLevel *)ctx->level.p, mpp,
                                           (const vll_point3 *)ctx->tin_pts.p, target_index,
                                           (double *)ctx->tin_scratch.p, ctx->stream));
    double out[3];
    VLL_CUDA(ctx, cudaMemcpyAsync(out, ctx->tin_scratch.p, sizeof(out), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->launches_total += 1;
    *f_height = out[0];
    if (out[0] != -9999.0) *f_sncc = out[1];
    *selected_count = (int)out[2];
    return VLL_OK;
}

// Ortho_blunder on device data: P's pointers (images, gp3) are device pointers.
static int ortho_blunder_run(vll_context *ctx, DevLevel &P, double mpp, vll_point3 *d_pts,
                             int64_t n_pts, const vll_tri *d_tris, int64_t n_tris,
                             vll_ugrid *d_gp3, int *rounds) {
    if (n_pts < 0 || n_tris < 0 || n_pts > 0x7fffffff || n_tris > 0x7fffffff)
        return fail(ctx, VLL_ERR_INVALID, "point or triangle count out of range");
    if (rounds) *rounds = 0;
    if (n_tris == 0) return VLL_OK;
    P.gp3 = d_gp3;
    int rc = upload_level_block(ctx, P);
    if (rc) return rc;
    const size_t bytes = vll::ortho_blunder_scratch(n_pts, n_tris, P.n_nodes);
    VLL_CUDA(ctx, ensure(ctx->tin_scratch, bytes));
    int it = 0, bad = 0;
    VLL_CUDA(ctx, vll::run_ortho_blunder((const DevLevel *)ctx->level.p, P, mpp, d_pts, n_pts,
                                         d_tris, n_tris, d_gp3, ctx->tin_scratch.p, bytes, &it,
                                         &bad, ctx->stream));
    if (bad) return fail(ctx, VLL_ERR_INVALID, "a triangle vertex lies outside the grid");
    // own kernels: the node and lon/lat passes, then search / records / apply / anchor per
    // round (the radix sort between them is CUB's)
    ctx->launches_total += 2 + 4 * (int64_t)it;
    if (rounds) *rounds = it;
    return VLL_OK;
}

int vll_ortho_blunder(vll_context *ctx, const vll_level_desc *desc, double mpp, vll_point3 *pts,
                      int64_t n_pts, const vll_tri *tris, int64_t n_tris, vll_ugrid *gridpt3,
                      int *rounds) {
    NvtxRange nvtx_range("vll_ortho_blunder");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !gridpt3 || (n_pts > 0 && !pts) || (n_tris > 0 && !tris))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    const int64_t N = P.n_nodes;
    if ((rc = upload_ortho_images(ctx, desc, P, false))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->tin_pts, pts, (size_t)n_pts * sizeof(vll_point3)))) return rc;
    if ((rc = upload(ctx, ctx->tin_tris, tris, (size_t)n_tris * sizeof(vll_tri)))) return rc;
    rc = ortho_blunder_run(ctx, P, mpp, (vll_point3 *)ctx->tin_pts.p, n_pts,
                           (const vll_tri *)ctx->tin_tris.p, n_tris, (vll_ugrid *)ctx->gp3.p,
                           rounds);
    if (rc) return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    if (n_pts > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(pts, ctx->tin_pts.p, (size_t)n_pts * sizeof(vll_point3),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_ortho_blunder_device(vll_context *ctx, const vll_level_desc *desc, double mpp,
                             vll_point3 *d_pts, int64_t n_pts, const vll_tri *d_tris,
                             int64_t n_tris, vll_ugrid *d_gridpt3, int *rounds) {
    NvtxRange nvtx_range("vll_ortho_blunder_device");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !d_gridpt3 || (n_pts > 0 && !d_pts) || (n_tris > 0 && !d_tris))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    return ortho_blunder_run(ctx, P, mpp, d_pts, n_pts, d_tris, n_tris, d_gridpt3, rounds);
}

// InitializeVoxel on device pointers; d_off (N + 1) receives the offsets.
static int init_voxel_run(vll_context *ctx, const vll_level_desc *desc, vll_ugrid *d_gp3,
                          vll_nccresult *d_ncc, const vll_voxel *d_vin, vll_voxel *d_vout,
                          int64_t capacity, int64_t *d_off, int64_t *n_out, bool grid_on_device,
                          int64_t *old_total) {
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    if (!(desc->height_step > 0)) return fail(ctx, VLL_ERR_INVALID, "height_step must be > 0");
    const int64_t N = P.n_nodes;
    if (N > 0x7fffffff) return fail(ctx, VLL_ERR_INVALID, "grid too large");
    if (!grid_on_device) {
        if ((rc = upload_plane(ctx, ctx->wgs, desc->grid_wgs, (size_t)N * 16))) return rc;
        P.grid_wgs = (const double *)ctx->wgs.p;
    }
    P.gp3 = d_gp3;
    if ((rc = upload_level_block(ctx, P))) return rc;
    const size_t bytes = vll::init_voxel_scratch(N);
    VLL_CUDA(ctx, ensure(ctx->tin_scratch, bytes));
    int64_t total = 0, old_tot = 0;
    VLL_CUDA(ctx, vll::run_init_voxel((const DevLevel *)ctx->level.p, N, d_gp3, d_ncc,
                                      ctx->tin_scratch.p, d_off, &total, &old_tot, ctx->stream));
    ctx->launches_total += 1;
    *n_out = total;
    if (old_total) *old_total = old_tot;
    if (total > capacity) return VLL_ERR_CAPACITY;
    VLL_CUDA(ctx, vll::run_commit_voxel(N, ctx->tin_scratch.p, d_gp3, d_ncc, ctx->stream));
    if (total > 0) {
        VLL_CUDA(ctx, vll::run_pack_voxel(N, d_off, ctx->tin_scratch.p, d_vin, d_vout,
                                          ctx->stream));
        ctx->launches_total += 1;
    }
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

// InitializeVoxel with the voxel packing kept in the context: the input rows
// are the caller's (the first call of a session) or the previous packing
// (when its length matches the old NumOfHeight sum); the output replaces it.
// Records go both ways, voxels stay on the device.
static int init_voxel_resident(vll_context *ctx, const vll_level_desc *desc, vll_ugrid *gridpt3,
                               vll_nccresult *nccresult, const vll_voxel *voxels_in,
                               int64_t old_total, int64_t *n_out) {
    const int64_t N = desc->grid_width * desc->grid_height;
    int rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->ncc, nccresult, (size_t)N * sizeof(vll_nccresult)))) return rc;
    const vll_voxel *d_vin = nullptr;
    if (voxels_in && old_total > 0) {
        if ((rc = upload(ctx, ctx->rvox, voxels_in, (size_t)old_total * sizeof(vll_voxel))))
            return rc;
        d_vin = (const vll_voxel *)ctx->rvox.p;
    } else if (ctx->rvox_total == old_total && ctx->rvox_nodes == N && old_total > 0) {
        d_vin = (const vll_voxel *)ctx->rvox.p;
    }
    // the output packing goes to ctx->vox (then swapped in), sized from the
    // ranges and grown once if that estimate falls short
    int64_t cap = 1;
    for (int64_t i = 0; i < N; ++i) {
        const int64_t span = (int64_t)gridpt3[i].maxHeight - gridpt3[i].minHeight +
                             (int64_t)nccresult[i].maxHeight - nccresult[i].minHeight;
        cap += (int64_t)((span < 0 ? -span : span) / desc->height_step) + 8 +
               nccresult[i].NumOfHeight;
    }
    VLL_CUDA(ctx, ensure(ctx->voxoff, (size_t)(N + 1) * sizeof(int64_t)));
    int64_t total = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        VLL_CUDA(ctx, ensure(ctx->vox, (size_t)cap * sizeof(vll_voxel)));
        ctx->vox.src = nullptr;
        rc = init_voxel_run(ctx, desc, (vll_ugrid *)ctx->gp3.p, (vll_nccresult *)ctx->ncc.p, d_vin,
                            (vll_voxel *)ctx->vox.p, cap, (int64_t *)ctx->voxoff.p, &total, false,
                            nullptr);
        if (rc != VLL_ERR_CAPACITY) break;
        cap = total;
    }
    *n_out = total;
    if (rc) return rc == VLL_ERR_CAPACITY ? fail(ctx, rc, "voxel packing estimate") : rc;
    std::swap(ctx->vox, ctx->rvox);
    std::swap(ctx->voxoff, ctx->rvox_off);
    ctx->rvox_total = total;
    ctx->rvox_nodes = N;
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(nccresult, ctx->ncc.p, (size_t)N * sizeof(vll_nccresult),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_initialize_voxel(vll_context *ctx, const vll_level_desc *desc, vll_ugrid *gridpt3,
                         vll_nccresult *nccresult, const vll_voxel *voxels_in,
                         vll_voxel *voxels_out, int64_t capacity, int64_t *n_out) {
    NvtxRange nvtx_range("vll_initialize_voxel");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    const bool resident = !voxels_out && (ctx->residency & VLL_RESIDENT_VOXELS);
    if (!desc || !gridpt3 || !nccresult || !n_out || !desc->grid_wgs || capacity < 0 ||
        (capacity > 0 && !voxels_out && !resident))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    const int64_t N = desc->grid_width * desc->grid_height;
    if (N <= 0) return fail(ctx, VLL_ERR_INVALID, "empty grid");
    int64_t old_total = 0;
    for (int64_t i = 0; i < N; ++i) old_total += nccresult[i].NumOfHeight;
    int rc;
    if (resident)
        return init_voxel_resident(ctx, desc, gridpt3, nccresult, voxels_in, old_total, n_out);
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->ncc, nccresult, (size_t)N * sizeof(vll_nccresult)))) return rc;
    const vll_voxel *d_vin = nullptr;
    if (voxels_in && old_total > 0) {
        if ((rc = upload(ctx, ctx->vox, voxels_in, (size_t)old_total * sizeof(vll_voxel))))
            return rc;
        d_vin = (const vll_voxel *)ctx->vox.p;
    }
    VLL_CUDA(ctx, ensure(ctx->voxoff, (size_t)(N + 1) * sizeof(int64_t)));
    // the output rows go to a second buffer (the input rows are read while
    // they are written)
    VLL_CUDA(ctx, ensure(ctx->gsum, (size_t)(capacity > 0 ? capacity : 1) * sizeof(vll_voxel)));
    int64_t total = 0;
    rc = init_voxel_run(ctx, desc, (vll_ugrid *)ctx->gp3.p, (vll_nccresult *)ctx->ncc.p, d_vin,
                        (vll_voxel *)ctx->gsum.p, capacity, (int64_t *)ctx->voxoff.p, &total,
                        false, nullptr);
    *n_out = total;
    if (rc == VLL_ERR_CAPACITY)
        return fail(ctx, VLL_ERR_CAPACITY, "more voxels than the output buffer holds");
    if (rc) return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(nccresult, ctx->ncc.p, (size_t)N * sizeof(vll_nccresult),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    if (total > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(voxels_out, ctx->gsum.p, (size_t)total * sizeof(vll_voxel),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_initialize_voxel_device(vll_context *ctx, const vll_level_desc *desc,
                                vll_ugrid *d_gridpt3, vll_nccresult *d_nccresult,
                                const vll_voxel *d_voxels_in, vll_voxel *d_voxels_out,
                                int64_t capacity, int64_t *d_voxel_offsets, int64_t *n_out) {
    NvtxRange nvtx_range("vll_initialize_voxel_device");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !d_gridpt3 || !d_nccresult || !d_voxel_offsets || !n_out || !desc->grid_wgs ||
        capacity < 0 || (capacity > 0 && !d_voxels_out))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    const int rc = init_voxel_run(ctx, desc, d_gridpt3, d_nccresult, d_voxels_in, d_voxels_out,
                                  capacity, d_voxel_offsets, n_out, true, nullptr);
    if (rc == VLL_ERR_CAPACITY)
        return fail(ctx, VLL_ERR_CAPACITY, "more voxels than the output buffer holds");
    return rc;
}

// SelectMPs on device data; out: d_points (capacity entries).
static int select_mps_run(vll_context *ctx, const vll_level_desc *desc, const vll_nccresult *d_ncc,
                          vll_ugrid *d_gp3, const double *d_grid_pts, double th_roh,
                          double th_roh_min, double th_roh_start, double th_roh_next,
                          int iteration, double mpp, int final_level_iteration,
                          double mpp_stereo_angle, vll_point3 *d_points, int64_t capacity,
                          int64_t *count) {
    const int L = desc->pyramid_step;
    const bool is_ra = desc->is_ra != 0;
    // the level's quota of the histogram; unset in the reference above level 4
    double min_roh_th = 0;
    bool quota = true;
    if (L == 4)
        min_roh_th = 0.05 + (iteration - 1) * 0.01;
    else if (L == 3)
        min_roh_th = 0.15 + (iteration - 1) * 0.01;
    else if (L == 2)
        min_roh_th = 0.60;
    else if (L == 1)
        min_roh_th = 0.80;
    else
        quota = false;
    if (L <= desc->sgm_py) {
        min_roh_th = 0.95 - L * 0.1;
        if (min_roh_th < 0.5) min_roh_th = 0.5;
        quota = true;
    }
    if (!is_ra && L > 0 && !quota)
        return fail(ctx, VLL_ERR_UNSUPPORTED, "SelectMPs threshold undefined above level 4");
    const int64_t N = desc->grid_width * desc->grid_height;
    const size_t bytes = vll::select_mps_scratch(N);
    VLL_CUDA(ctx, ensure(ctx->tin_scratch, bytes));
    double minimum_th = 0.2;
    if (!is_ra && L > 0) {
        int hist[100];
        int64_t total = 0;
        VLL_CUDA(ctx, vll::run_roh_hist(d_ncc, N, ctx->tin_scratch.p, hist, &total, ctx->stream));
        ctx->launches_total += 1;
        if (total > 0) {
            int roh_iter = 99;
            int sum = 0;
            while (roh_iter > 0) {
                sum += hist[roh_iter];
                if (sum / (double)total > min_roh_th) {
                    minimum_th = (double)roh_iter / (double)100;
                    break;
                }
                --roh_iter;
            }
            if (minimum_th > 0.95) minimum_th = 0.95;
        }
    }
    vll::SelectArgs a;
    a.pyramid_step = L;
    a.iteration = iteration;
    a.final_level_iteration = final_level_iteration;
    if (L <= 3 || is_ra)
        a.check_iter_end = th_roh - 0.10 < th_roh_min;
    else
        a.check_iter_end = th_roh - 0.06 < th_roh_min;
    a.minimum_th = minimum_th;
    a.th_roh = th_roh;
    a.th_roh_start = th_roh_start;
    a.th_roh_next = th_roh_next;
    a.mpp = mpp;
    a.mpp_stereo_angle = mpp_stereo_angle;
    int64_t n_sel = 0;
    VLL_CUDA(ctx, vll::run_select_mps(d_ncc, d_gp3, d_grid_pts, N, a, ctx->tin_scratch.p,
                                      d_points, capacity, &n_sel, ctx->stream));
    ctx->launches_total += 2;
    *count = n_sel;
    if (n_sel > capacity)
        return fail(ctx, VLL_ERR_CAPACITY, "more selected points than the points buffer holds");
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

static int select_mps_check(vll_context *ctx, const vll_level_desc *desc, const void *ncc,
                            const void *gp3, const int64_t *count, const void *points,
                            int64_t capacity) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !ncc || !gp3 || !count || !desc->grid_pts || (capacity > 0 && !points) ||
        capacity < 0)
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    if (desc->grid_width <= 0 || desc->grid_height <= 0 ||
        desc->grid_width * desc->grid_height > 0x7fffffff)
        return fail(ctx, VLL_ERR_INVALID, "invalid grid size");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    return VLL_OK;
}

int vll_select_mps(vll_context *ctx, const vll_level_desc *desc, const vll_nccresult *nccresult,
                   vll_ugrid *gridpt3, double th_roh, double th_roh_min, double th_roh_start,
                   double th_roh_next, int iteration, double mpp, int final_level_iteration,
                   double mpp_stereo_angle, vll_point3 *points, int64_t capacity,
                   int64_t *count) {
    NvtxRange nvtx_range("vll_select_mps");
    int rc = select_mps_check(ctx, desc, nccresult, gridpt3, count, points, capacity);
    if (rc) return rc;
    const int64_t N = desc->grid_width * desc->grid_height;
    if ((rc = upload(ctx, ctx->ncc, nccresult, (size_t)N * sizeof(vll_nccresult)))) return rc;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    VLL_CUDA(ctx, ensure(ctx->tin_pts, (size_t)(capacity > 0 ? capacity : 1) * sizeof(vll_point3)));
    // the grid coordinates stay on the host: the points come back with their
    // node in x and take the coordinates here
    rc = select_mps_run(ctx, desc, (const vll_nccresult *)ctx->ncc.p, (vll_ugrid *)ctx->gp3.p,
                        nullptr, th_roh, th_roh_min, th_roh_start, th_roh_next, iteration, mpp,
                        final_level_iteration, mpp_stereo_angle, (vll_point3 *)ctx->tin_pts.p,
                        capacity, count);
    if (rc) return rc;   // host buffers untouched
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    if (*count > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(points, ctx->tin_pts.p, (size_t)*count * sizeof(vll_point3),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t j = 0; j < *count; ++j) {
        const int64_t node = (int64_t)points[j].x;
        points[j].x = desc->grid_pts[2 * node];
        points[j].y = desc->grid_pts[2 * node + 1];
    }
    return VLL_OK;
}

int vll_select_mps_device(vll_context *ctx, const vll_level_desc *desc,
                          const vll_nccresult *d_nccresult, vll_ugrid *d_gridpt3, double th_roh,
                          double th_roh_min, double th_roh_start, double th_roh_next,
                          int iteration, double mpp, int final_level_iteration,
                          double mpp_stereo_angle, vll_point3 *d_points, int64_t capacity,
                          int64_t *count) {
    NvtxRange nvtx_range("vll_select_mps_device");
    int rc = select_mps_check(ctx, desc, d_nccresult, d_gridpt3, count, d_points, capacity);
    if (rc) return rc;
    return select_mps_run(ctx, desc, d_nccresult, d_gridpt3, desc->grid_pts, th_roh, th_roh_min,
                          th_roh_start, th_roh_next, iteration, mpp, final_level_iteration,
                          mpp_stereo_angle, d_points, capacity, count);
}

// SetHeightRange's BufferOfHeight and th_HG (setsm_code.cpp:9863-9922).
static void height_range_constants(const vll_level_desc *d, int iteration, double mpp, bool lcmr,
                                   double seed_sigma, double *buffer, double *th_hg) {
    const int L = d->pyramid_step;
    double b = mpp * 4.0 * (double)(1 << L);
    if (L == 1) {
        b = iteration >= 2 ? mpp * 2 : mpp * 3;
    } else if (L == 0) {
        b = iteration == 1 ? mpp * 2 : mpp;
        if (b < 0.5) b = 0.5;
    }
    if (d->pre_dem_tif && b > seed_sigma) b = seed_sigma;
    b = ceil(b);
    if (b > 100) b = 100;
    double th = 100000;
    if (d->dem_resolution >= 4) {
        if (L <= 1) th = 1000;
    } else {
        if (!lcmr) {
            if (L == 2 && iteration >= 5)
                th = 1000;
            else if (L == 1)
                th = 500;
            else if (L == 0)
                th = 100;
        } else if (L <= 2) {
            th = 100;
        }
        if (L == 0 && d->dem_resolution < 2 && iteration > 1) th = 50;
    }
    *buffer = b;
    *th_hg = th;
}

// blunder_detection_TIN's argument checks; 1 = nothing to do (level 0,
// iteration 3, which the reference skips).
static int tin_blunder_check(vll_context *ctx, const vll_level_desc *desc, int iteration,
                             const void *ortho_ncc, double hinterval, const void *pts,
                             const void *detected, int64_t n_pts, const void *tris,
                             int64_t n_tris, const void *gridpt3, const void *blunder_count,
                             const void *minz_mp, const void *maxz_mp) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !ortho_ncc || !gridpt3 || !blunder_count || !minz_mp || !maxz_mp ||
        (n_pts > 0 && (!pts || !detected)) || (n_tris > 0 && !tris))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    if (n_pts < 0 || n_tris < 0 || n_pts > 0x7fffffff || 3 * n_tris > 0x7fffffff)
        return fail(ctx, VLL_ERR_INVALID, "point or triangle count out of range");
    if (desc->grid_width <= 0 || desc->grid_height <= 0 || !(desc->grid_resolution > 0) ||
        desc->pyramid_step < 0 || desc->pyramid_step > 12)
        return fail(ctx, VLL_ERR_INVALID, "invalid grid or level");
    if (desc->pyramid_step == 0 && iteration == 3) return 1;   // the reference skips it
    if (!(hinterval >= 0) || hinterval > 1e8)
        return fail(ctx, VLL_ERR_INVALID, "Hinterval out of range");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    return VLL_OK;
}

// blunder_detection_TIN on device data; counts and extent accumulate into
// the host outputs as the reference's do.
static int tin_blunder_run(vll_context *ctx, const vll_level_desc *desc, int iteration,
                           const float *d_oncc, int flag_blunder, int count_bl, double hinterval,
                           vll_point3 *d_pts, uint8_t *d_det, int64_t n_pts, const vll_tri *d_tris,
                           int64_t n_tris, vll_ugrid *d_gp3, int64_t *blunder_count,
                           double *minz_mp, double *maxz_mp, vll_ugrid *host_gp3 = nullptr) {
    const uint32_t hdiffcount = (uint32_t)hinterval;
    vll::TinArgs a;
    a.b0 = desc->boundary[0];
    a.b1 = desc->boundary[1];
    a.gs = desc->grid_resolution;
    a.width = desc->grid_width;
    a.n_nodes = desc->grid_width * desc->grid_height;
    a.n_pts = n_pts;
    a.n_tris = n_tris;
    a.L = desc->pyramid_step;
    a.iteration = iteration;
    a.is_ra = desc->is_ra != 0;
    a.flag_blunder = flag_blunder != 0;
    a.count_bl = count_bl;
    a.height_th = a.ortho_ncc_th = a.th_ref_ncc = 0;
    a.hinterval = hinterval;
    a.height_th_hi = 0;
    // SETSM_VLL_TIN_SUMS=exact: the sequential sums always (no band);
    // =wideband: the band widened by 1 m (the exact re-run on nearly every
    // input)
    int mode = vll::kTinSumsBand;
    if (const char *m = getenv("SETSM_VLL_TIN_SUMS")) {
        if (!strcmp(m, "exact")) mode = vll::kTinSumsExact;
        else if (!strcmp(m, "wideband")) mode = vll::kTinSumsWideBand;
    }
    const size_t bytes = vll::tin_blunder_scratch(n_pts, n_tris, hdiffcount);
    VLL_CUDA(ctx, ensure(ctx->tin_scratch, bytes));
    vll::TinOutput out;
    memset(&out, 0, sizeof(out));
    VLL_CUDA(ctx, vll::run_tin_blunder(a, d_pts, d_tris, d_oncc, d_gp3, d_det, hdiffcount, mode,
                                       host_gp3 != nullptr, ctx->tin_scratch.p, bytes, &out,
                                       ctx->stream));
    if (out.bad_input) return fail(ctx, VLL_ERR_INVALID, "a point's grid node lies outside the grid");
    if (host_gp3 && n_pts > 0) {
        // the pass's anchor_flag writes, applied to the caller's grid in point
        // order (the grid itself never crosses the bus)
        std::vector<int64_t> node((size_t)n_pts);
        std::vector<uint8_t> val((size_t)n_pts);
        VLL_CUDA(ctx, cudaMemcpyAsync(node.data(), out.anchor_node, (size_t)n_pts * 8,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        VLL_CUDA(ctx, cudaMemcpyAsync(val.data(), out.anchor_val, (size_t)n_pts,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        for (int64_t i = 0; i < n_pts; ++i)
            if (node[i] >= 0) host_gp3[node[i]].anchor_flag = val[i];
    }
    // terms, sums, scan (2), fill, thresholds, snapshot, point pass, close; a
    // re-run adds the undo, the sequential sums, the thresholds, the point
    // pass and close
    ctx->launches_total += (n_tris > 0 ? 9 : 6) + (out.rerun ? (n_tris > 0 ? 5 : 4) : 0);
    ctx->tin_reruns += out.rerun;
    blunder_count[0] += out.count[0];
    blunder_count[1] += out.count[1];
    if (out.has_z) {
        if (*minz_mp > out.z[0]) *minz_mp = out.z[0];
        if (*maxz_mp < out.z[1]) *maxz_mp = out.z[1];
    }
    return VLL_OK;
}

int vll_blunder_detection_tin(vll_context *ctx, const vll_level_desc *desc, int iteration,
                              const float *ortho_ncc, int flag_blunder, int count_bl,
                              double hinterval, vll_point3 *pts, uint8_t *detected_blunders,
                              int64_t n_pts, const vll_tri *tris, int64_t n_tris,
                              vll_ugrid *gridpt3, int64_t *blunder_count, double *minz_mp,
                              double *maxz_mp) {
    NvtxRange nvtx_range("vll_blunder_detection_tin");
    int rc = tin_blunder_check(ctx, desc, iteration, ortho_ncc, hinterval, pts, detected_blunders,
                               n_pts, tris, n_tris, gridpt3, blunder_count, minz_mp, maxz_mp);
    if (rc) return rc > 0 ? VLL_OK : rc;
    const int64_t N = desc->grid_width * desc->grid_height;
    // the pass reads no UGRID field and writes only anchor_flag at the
    // points' nodes: the grid stays on the host and takes the listed writes
    if ((rc = upload(ctx, ctx->tin_pts, pts, (size_t)n_pts * sizeof(vll_point3)))) return rc;
    if ((rc = upload(ctx, ctx->tin_tris, tris, (size_t)n_tris * sizeof(vll_tri)))) return rc;
    if ((rc = upload(ctx, ctx->gsum, ortho_ncc, (size_t)N * sizeof(float)))) return rc;
    if ((rc = upload(ctx, ctx->gcnt, detected_blunders, (size_t)(n_pts > 0 ? n_pts : 1))))
        return rc;
    if ((rc = tin_blunder_run(ctx, desc, iteration, (const float *)ctx->gsum.p, flag_blunder,
                              count_bl, hinterval, (vll_point3 *)ctx->tin_pts.p,
                              (uint8_t *)ctx->gcnt.p, n_pts, (const vll_tri *)ctx->tin_tris.p,
                              n_tris, nullptr, blunder_count, minz_mp, maxz_mp, gridpt3)))
        return rc;
    if (n_pts > 0) {
        VLL_CUDA(ctx, cudaMemcpyAsync(pts, ctx->tin_pts.p, (size_t)n_pts * sizeof(vll_point3),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        VLL_CUDA(ctx, cudaMemcpyAsync(detected_blunders, ctx->gcnt.p, (size_t)n_pts,
                                      cudaMemcpyDeviceToHost, ctx->stream));
    }
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_blunder_detection_tin_device(vll_context *ctx, const vll_level_desc *desc, int iteration,
                                     const float *d_ortho_ncc, int flag_blunder, int count_bl,
                                     double hinterval, vll_point3 *d_pts,
                                     uint8_t *d_detected_blunders, int64_t n_pts,
                                     const vll_tri *d_tris, int64_t n_tris, vll_ugrid *d_gridpt3,
                                     int64_t *blunder_count, double *minz_mp, double *maxz_mp) {
    NvtxRange nvtx_range("vll_blunder_detection_tin_device");
    int rc = tin_blunder_check(ctx, desc, iteration, d_ortho_ncc, hinterval, d_pts,
                               d_detected_blunders, n_pts, d_tris, n_tris, d_gridpt3,
                               blunder_count, minz_mp, maxz_mp);
    if (rc) return rc > 0 ? VLL_OK : rc;
    return tin_blunder_run(ctx, desc, iteration, d_ortho_ncc, flag_blunder, count_bl, hinterval,
                           d_pts, d_detected_blunders, n_pts, d_tris, n_tris, d_gridpt3,
                           blunder_count, minz_mp, maxz_mp);
}

static int height_range_check(vll_context *ctx, const vll_level_desc *desc, const void *pts,
                              int64_t n_pts, const void *tris, int64_t n_tris, const void *gp3,
                              const void *result, const double *min_h, const double *max_h) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !gp3 || !result || !min_h || !max_h || (n_pts > 0 && !pts) ||
        (n_tris > 0 && !tris))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    if (n_pts < 0 || n_tris < 0 || n_pts > 0x7fffffff || n_tris > 0x7fffffff)
        return fail(ctx, VLL_ERR_INVALID, "point or triangle count out of range");
    if (desc->grid_width <= 0 || desc->grid_height <= 0 || desc->pyramid_step < 0 ||
        desc->pyramid_step > 12 || !(desc->grid_resolution > 0) || desc->num_images < 1 ||
        desc->num_images > VLL_MAX_IMAGES)
        return fail(ctx, VLL_ERR_INVALID, "invalid grid, level or image count");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    return VLL_OK;
}

// SetHeightRange on device data.
static int height_range_run(vll_context *ctx, const vll_level_desc *desc, const vll_point3 *d_pts,
                            int64_t n_pts, const vll_tri *d_tris, int64_t n_tris,
                            vll_ugrid *d_gp3, vll_ugrid *d_result, int iteration, double mpp,
                            int lcmr, double seed_dem_sigma, double *min_h, double *max_h) {
    // only the grid geometry, the level and the image selection are read
    DevLevel P;
    memset(&P, 0, sizeof(P));
    P.num_images = desc->num_images;
    P.ref = desc->reference_id;
    P.L = desc->pyramid_step;
    P.grid_res = desc->grid_resolution;
    P.im_res = desc->resolution * (double)(1 << P.L);
    for (int i = 0; i < 4; ++i) P.boundary[i] = desc->boundary[i];
    P.grid_w = desc->grid_width;
    P.grid_h = desc->grid_height;
    P.n_nodes = P.grid_w * P.grid_h;
    for (int ti = 0; ti < P.num_images; ++ti) P.im[ti].selected = desc->images[ti].selected != 0;
    P.gp3 = d_gp3;
    int rc = upload_level_block(ctx, P);
    if (rc) return rc;
    const size_t bytes = vll::height_range_scratch(P.n_nodes);
    VLL_CUDA(ctx, ensure(ctx->tin_scratch, bytes));
    double buffer, th_hg;
    height_range_constants(desc, iteration, mpp, lcmr != 0, seed_dem_sigma, &buffer, &th_hg);
    // triangles with a vertex index >= n_pts are skipped, as the reference does;
    // bounding boxes are clamped to the grid, so every node index is in range
    VLL_CUDA(ctx, vll::run_height_range((const DevLevel *)ctx->level.p, P, d_pts, n_pts, d_tris,
                                        n_tris, d_gp3, d_result, buffer, th_hg, iteration,
                                        ctx->tin_scratch.p, bytes, min_h, max_h, ctx->stream));
    ctx->launches_total += (n_tris > 0 ? 6 : 5);
    return VLL_OK;
}

int vll_set_height_range(vll_context *ctx, const vll_level_desc *desc, const vll_point3 *pts,
                         int64_t n_pts, const vll_tri *tris, int64_t n_tris, vll_ugrid *gridpt3,
                         vll_ugrid *result, int iteration, double mpp,
                         int level_check_matching_rate, double seed_dem_sigma,
                         double *min_h_grid, double *max_h_grid) {
    NvtxRange nvtx_range("vll_set_height_range");
    int rc = height_range_check(ctx, desc, pts, n_pts, tris, n_tris, gridpt3, result, min_h_grid,
                                max_h_grid);
    if (rc) return rc;
    const int64_t N = desc->grid_width * desc->grid_height;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    if ((rc = upload(ctx, ctx->tin_pts, pts, (size_t)n_pts * sizeof(vll_point3)))) return rc;
    if ((rc = upload(ctx, ctx->tin_tris, tris, (size_t)n_tris * sizeof(vll_tri)))) return rc;
    VLL_CUDA(ctx, ensure(ctx->ncc, (size_t)N * sizeof(vll_ugrid)));
    if ((rc = height_range_run(ctx, desc, (const vll_point3 *)ctx->tin_pts.p, n_pts,
                               (const vll_tri *)ctx->tin_tris.p, n_tris, (vll_ugrid *)ctx->gp3.p,
                               (vll_ugrid *)ctx->ncc.p, iteration, mpp, level_check_matching_rate,
                               seed_dem_sigma, min_h_grid, max_h_grid)))
        return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(gridpt3, ctx->gp3.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(result, ctx->ncc.p, (size_t)N * sizeof(vll_ugrid),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_set_height_range_device(vll_context *ctx, const vll_level_desc *desc,
                                const vll_point3 *d_pts, int64_t n_pts, const vll_tri *d_tris,
                                int64_t n_tris, vll_ugrid *d_gridpt3, vll_ugrid *d_result,
                                int iteration, double mpp, int level_check_matching_rate,
                                double seed_dem_sigma, double *min_h_grid, double *max_h_grid) {
    NvtxRange nvtx_range("vll_set_height_range_device");
    int rc = height_range_check(ctx, desc, d_pts, n_pts, d_tris, n_tris, d_gridpt3, d_result,
                                min_h_grid, max_h_grid);
    if (rc) return rc;
    return height_range_run(ctx, desc, d_pts, n_pts, d_tris, n_tris, d_gridpt3, d_result,
                            iteration, mpp, level_check_matching_rate, seed_dem_sigma,
                            min_h_grid, max_h_grid);
}

int vll_debug_ortho_raster(vll_context *ctx, const vll_level_desc *desc, const vll_ugrid *gridpt3,
                           int use_b, double im_res, int ti, double *out, int64_t capacity,
                           int64_t *width, int64_t *height) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !gridpt3 || !out || !width || !height || !desc->grid_pts)
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    if (ti < 0 || ti >= P.num_images || !P.im[ti].selected)
        return fail(ctx, VLL_ERR_INVALID, "image index out of range or not selected");
    if (!(im_res > 0)) return fail(ctx, VLL_ERR_INVALID, "non-positive resolution");
    const int64_t ow = (int64_t)((P.boundary[2] - P.boundary[0]) / im_res) + 1;
    const int64_t oh = (int64_t)((P.boundary[3] - P.boundary[1]) / im_res) + 1;
    *width = ow;
    *height = oh;
    if (ow <= 0 || oh <= 0) return fail(ctx, VLL_ERR_INVALID, "empty orthoimage boundary");
    if (capacity < ow * oh) return fail(ctx, VLL_ERR_CAPACITY, "raster larger than the buffer");
    const int64_t N = P.n_nodes;
    if ((rc = upload(ctx, ctx->gp3, gridpt3, (size_t)N * sizeof(vll_ugrid)))) return rc;
    P.gp3 = (const vll_ugrid *)ctx->gp3.p;
    const size_t total = (size_t)(ow * oh);
    double2 *ptrs[2 * VLL_MAX_IMAGES] = {};
    for (int i = 0; i < P.num_images; ++i) {
        if (!P.im[i].selected) continue;
        VLL_CUDA(ctx, ensure(ctx->ocd[i], total * sizeof(double2)));
        VLL_CUDA(ctx, cudaMemsetAsync(ctx->ocd[i].p, 0, total * sizeof(double2), ctx->stream));
        ptrs[i] = (double2 *)ctx->ocd[i].p;
    }
    if ((rc = upload_level_block(ctx, P))) return rc;
    VLL_CUDA(ctx, ensure(ctx->ocdptr, sizeof(ptrs)));
    VLL_CUDA(ctx, cudaMemcpyAsync(ctx->ocdptr.p, ptrs, sizeof(ptrs), cudaMemcpyHostToDevice,
                                  ctx->stream));
    VLL_CUDA(ctx, vll::launch_ortho_raster((const DevLevel *)ctx->level.p,
                                           (double2 *const *)ctx->ocdptr.p, ow, oh, im_res,
                                           use_b ? 1 : 0, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(out, ctx->ocd[ti].p, total * sizeof(double2),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_awncc_peaks_device(vll_context *ctx, const vll_level_desc *desc,
                           const vll_ugrid *d_gridpt3, vll_nccresult *d_nccresult,
                           const vll_voxel *d_voxels, const int64_t *d_voxel_offsets,
                           vll_stats *stats) {
    NvtxRange nvtx_range("vll_awncc_peaks_device");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!desc || !d_gridpt3 || !d_nccresult || !d_voxel_offsets)
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    DevLevel P;
    std::string err;
    int rc = vll::derive_level(desc, &P, &err, false);
    if (rc) return fail(ctx, rc, err);
    const bool sgm = P.L <= desc->sgm_py;
    const int64_t N = P.n_nodes;
    P.gp3 = d_gridpt3;
    P.ncc = d_nccresult;
    P.vox = const_cast<vll_voxel *>(d_voxels);
    P.vox_off = d_voxel_offsets;
    int max_h = 0;
    int64_t total = 0;
    VLL_CUDA(ctx, ensure(ctx->counters, 8 * sizeof(unsigned long long)));
    VLL_CUDA(ctx, vll::row_extent(d_nccresult, N, d_voxel_offsets, (int *)ctx->counters.p,
                                  &max_h, &total, ctx->stream));
    if (total > 0 && !d_voxels) return fail(ctx, VLL_ERR_INVALID, "null voxel rows");
    if ((rc = upload_level_block(ctx, P))) return rc;
    if (!ctx->e0) {
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e0));
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e1));
    }
    VLL_CUDA(ctx, cudaEventRecord(ctx->e0, ctx->stream));
    const float *sumcost = nullptr;
    if (sgm) {
        VLL_CUDA(ctx, ensure(ctx->sumcost, (size_t)(total > 0 ? total : 1) * sizeof(float)));
        VLL_CUDA(ctx, vll::launch_sgm((const DevLevel *)ctx->level.p, P.grid_w, P.grid_h, max_h,
                                      (float *)ctx->sumcost.p, total, ctx->stream,
                                      sgm_scratch(ctx, total)));
        sumcost = (const float *)ctx->sumcost.p;
        ctx->launches_total += 8;
    }
    VLL_CUDA(ctx, vll::launch_awncc((const DevLevel *)ctx->level.p, N, sumcost, ctx->stream));
    VLL_CUDA(ctx, cudaEventRecord(ctx->e1, ctx->stream));
    ctx->launches_total += 2;
    if (stats) {
        VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->e0, ctx->e1);
        memset(stats, 0, sizeof(*stats));
        stats->kernel_ms = ms;
    }
    return VLL_OK;
}

int vll_preprocess_level_device(vll_context *ctx, const uint16_t *d_image, uint32_t width,
                                uint32_t height, int template_size, uint16_t *d_mag,
                                uint8_t *d_ori) {
    NvtxRange nvtx_range("vll_preprocess_level_device");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!d_image || !d_mag || !d_ori || width < 1 || height < 1)
        return fail(ctx, VLL_ERR_INVALID, "invalid preprocessing arguments");
    // Orientation's column extents (numcols, SubFunctions.cpp:8) are sized for
    // the 15-pixel template SetPyramidImages uses (SubFunctions.cpp:3399).
    if (template_size != 15)
        return fail(ctx, VLL_ERR_UNSUPPORTED, "orientation template size must be 15");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = (size_t)width * height;
    VLL_CUDA(ctx, ensure(ctx->pre_tmp, n));
    // Gaussian weights exp(-(r^2+c^2)/4.5) of Orientation, SubFunctions.cpp:2489-2497
    const int half = template_size / 2;
    const int sz = 2 * half - 1;
    std::vector<double> wt((size_t)sz * sz);
    for (int r = -half + 1; r <= half - 1; ++r)
        for (int c = -half + 1; c <= half - 1; ++c)
            wt[(size_t)(half - 1 + r) * sz + (half - 1 + c)] = exp(-(double)(r * r + c * c) / 4.5);
    VLL_CUDA(ctx, ensure(ctx->pre_wt, wt.size() * sizeof(double)));
    VLL_CUDA(ctx, cudaMemcpyAsync(ctx->pre_wt.p, wt.data(), wt.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    VLL_CUDA(ctx, vll::launch_sobel(d_image, width, height, d_mag, (uint8_t *)ctx->pre_tmp.p,
                                    ctx->stream));
    VLL_CUDA(ctx, vll::launch_orientation(d_mag, (const uint8_t *)ctx->pre_tmp.p, width, height,
                                          half, (const double *)ctx->pre_wt.p, d_ori, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_preprocess_level(vll_context *ctx, const uint16_t *image, uint32_t width, uint32_t height,
                         int template_size, uint16_t *mag_out, uint8_t *ori_out) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!image || !mag_out || !ori_out) return fail(ctx, VLL_ERR_INVALID, "null buffer");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = (size_t)width * height;
    int rc;
    if ((rc = upload(ctx, ctx->pre_img, image, n * 2))) return rc;
    VLL_CUDA(ctx, ensure(ctx->pre_mag, n * 2));
    VLL_CUDA(ctx, ensure(ctx->pre_ori, n));
    rc = vll_preprocess_level_device(ctx, (const uint16_t *)ctx->pre_img.p, width, height,
                                     template_size, (uint16_t *)ctx->pre_mag.p,
                                     (uint8_t *)ctx->pre_ori.p);
    if (rc) return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(mag_out, ctx->pre_mag.p, n * 2, cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaMemcpyAsync(ori_out, ctx->pre_ori.p, n, cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_pyramid_down_device(vll_context *ctx, const uint16_t *d_image, uint32_t width,
                            uint32_t height, uint16_t *d_out) {
    NvtxRange nvtx_range("vll_pyramid_down_device");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!d_image || !d_out || width < 2 || height < 2)
        return fail(ctx, VLL_ERR_INVALID, "invalid pyramid arguments");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    // CreateGaussianFilter(9, 1.5), Template.hpp:45-80
    double f[81];
    double sum = 0;
    const double sigma = 1.5;
    const double tmp = -1 / (2 * sigma * sigma);
    const double scale = 1 / (sqrt(2 * 3.141592653589793) * sigma);
    for (int i = -4; i <= 4; ++i)
        for (int j = -4; j <= 4; ++j) {
            const double val = exp((i * i + j * j) * tmp) * scale;
            f[(i + 4) * 9 + (j + 4)] = val;
            sum += val;
        }
    for (double &v : f) v /= sum;
    VLL_CUDA(ctx, ensure(ctx->pre_wt, sizeof(f)));
    VLL_CUDA(ctx, cudaMemcpyAsync(ctx->pre_wt.p, f, sizeof(f), cudaMemcpyHostToDevice, ctx->stream));
    VLL_CUDA(ctx, vll::launch_pyramid(d_image, width, height, (const double *)ctx->pre_wt.p, d_out,
                                      ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

int vll_pyramid_down(vll_context *ctx, const uint16_t *image, uint32_t width, uint32_t height,
                     uint16_t *out) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!image || !out) return fail(ctx, VLL_ERR_INVALID, "null buffer");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = (size_t)width * height;
    const size_t no = (size_t)(width / 2) * (height / 2);
    int rc;
    if ((rc = upload(ctx, ctx->pre_img, image, n * 2))) return rc;
    VLL_CUDA(ctx, ensure(ctx->pre_mag, no * 2));
    rc = vll_pyramid_down_device(ctx, (const uint16_t *)ctx->pre_img.p, width, height,
                                 (uint16_t *)ctx->pre_mag.p);
    if (rc) return rc;
    VLL_CUDA(ctx, cudaMemcpyAsync(out, ctx->pre_mag.p, no * 2, cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

// ---- batches, plans, tuning ------------------------------------------------
struct vll_plan {
    vll_context *ctx = nullptr;
    SetResources res;
    vll::SplitPlan plan;
    int n_levels = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

int vll_vertical_line_locus_batch(vll_context *ctx, const vll_level_io *levels, int n_levels,
                                  int64_t *accessable, vll_stats *stats) {
    NvtxRange nvtx_range("vll_vertical_line_locus_batch");
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    SetResources &r = *ctx_set(ctx);
    int rc = prepare_set(ctx, r, levels, n_levels);
    if (rc) return rc;
    VLL_CUDA(ctx, cudaMemsetAsync(r.counters.p, 0, 8 * sizeof(unsigned long long), ctx->stream));
    if (!ctx->e0) {
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e0));
        VLL_CUDA(ctx, cudaEventCreate(&ctx->e1));
    }
    VLL_CUDA(ctx, cudaEventRecord(ctx->e0, ctx->stream));
    VLL_CUDA(ctx, enqueue_set_ortho(r, ctx->stream));
    std::string err;
    vll::SplitTiming tm;
    cudaError_t e = vll::run_split_set(r.split, r.hl.data(), (const DevLevel *)r.dl.p, n_levels,
                                       (unsigned long long *)r.counters.p, ctx->stream, &err, &tm,
                                       ctx->tuning);
    if (e != cudaSuccess) return cuda_fail(ctx, e, err.c_str());
    VLL_CUDA(ctx, cudaEventRecord(ctx->e1, ctx->stream));
    VLL_CUDA(ctx, cudaEventSynchronize(ctx->e1));
    float ms = 0;
    VLL_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->e0, ctx->e1));
    ctx->launches_total += tm.launches;
    rc = finish_set(ctx, r, r.split, n_levels, accessable, stats, ms, tm.launches);
    if (!rc && stats) stats->slots = tm.slots;
    return rc;
}

int vll_plan_create(vll_context *ctx, const vll_level_io *levels, int n_levels, vll_plan **out) {
    NvtxRange nvtx_range("vll_plan_create");
    if (!ctx || !out) return fail(ctx, VLL_ERR_INVALID, "null context or output pointer");
    *out = nullptr;
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    vll_plan *pl = new vll_plan();
    pl->ctx = ctx;
    pl->n_levels = n_levels;
    int rc = prepare_set(ctx, pl->res, levels, n_levels);
    if (rc) {
        release_set(pl->res);
        delete pl;
        return rc;
    }
    std::string err;
    SetResources *rp = &pl->res;
    VLL_CUDA(ctx, cudaMemsetAsync(pl->res.counters.p, 0, 8 * sizeof(unsigned long long),
                                  ctx->stream));
    // the graph clears the counters itself at the start of every replay
    auto pre = [rp](cudaStream_t s) -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(rp->counters.p, 0, 8 * sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        return enqueue_set_ortho(*rp, s);
    };
    cudaError_t e = vll::split_plan(pl->plan, pl->plan.bufs, pl->res.hl.data(),
                                    (const DevLevel *)pl->res.dl.p, n_levels,
                                    (unsigned long long *)pl->res.counters.p, ctx->stream, &err,
                                    ctx->tuning, pre);
    if (e != cudaSuccess) {
        rc = cuda_fail(ctx, e, err.c_str());
        vll_plan_destroy(pl);
        return rc;
    }
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *out = pl;
    return VLL_OK;
}

int vll_plan_run(vll_plan *pl, int64_t *accessable, vll_stats *stats) {
    NvtxRange nvtx_range("vll_plan_run");
    if (!pl || !pl->ctx) return fail(nullptr, VLL_ERR_INVALID, "null plan");
    vll_context *ctx = pl->ctx;
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    const bool wait = accessable || stats;
    if (wait && !pl->e0) {
        VLL_CUDA(ctx, cudaEventCreate(&pl->e0));
        VLL_CUDA(ctx, cudaEventCreate(&pl->e1));
    }
    if (wait) VLL_CUDA(ctx, cudaEventRecord(pl->e0, ctx->stream));
    VLL_CUDA(ctx, cudaGraphLaunch(pl->plan.exec, ctx->stream));
    ctx->launches_total += pl->plan.launches;
    if (!wait) return VLL_OK;
    VLL_CUDA(ctx, cudaEventRecord(pl->e1, ctx->stream));
    VLL_CUDA(ctx, cudaEventSynchronize(pl->e1));
    float ms = 0;
    VLL_CUDA(ctx, cudaEventElapsedTime(&ms, pl->e0, pl->e1));
    const int rc = finish_set(ctx, pl->res, pl->plan.bufs, pl->n_levels, accessable, stats, ms,
                              pl->plan.launches);
    if (!rc && stats) stats->slots = pl->plan.n_slots;
    return rc;
}

void vll_plan_destroy(vll_plan *pl) {
    if (!pl) return;
    if (pl->ctx) {
        cudaSetDevice(pl->ctx->device);
        cudaStreamSynchronize(pl->ctx->stream);
    }
    if (pl->plan.exec) cudaGraphExecDestroy(pl->plan.exec);
    vll::split_release(pl->plan.bufs);
    release_set(pl->res);
    if (pl->e0) cudaEventDestroy(pl->e0);
    if (pl->e1) cudaEventDestroy(pl->e1);
    delete pl;
}

int vll_set_tuning(vll_context *ctx, const vll_tuning *t) {
    if (!ctx || !t) return fail(ctx, VLL_ERR_INVALID, "null context or tuning");
    if (t->blocks_per_sm < 0 || t->grab < 0 || t->grab > 64 || t->box_margin < 0.f ||
        (t->box_margin > 0.f && t->box_margin < 1.0f) || t->box_margin > 4.0f)
        return fail(ctx, VLL_ERR_INVALID, "tuning out of range");
    ctx->tuning.blocks_per_sm = t->blocks_per_sm;
    ctx->tuning.grab = t->grab > 0 ? t->grab : vll::SplitTuning().grab;
    ctx->tuning.box_margin = t->box_margin > 0.f ? t->box_margin : vll::SplitTuning().box_margin;
    return VLL_OK;
}

int vll_get_tuning(const vll_context *ctx, vll_tuning *t) {
    if (!ctx || !t) return VLL_ERR_INVALID;
    memset(t, 0, sizeof(*t));
    t->blocks_per_sm = ctx->tuning.blocks_per_sm;
    t->grab = ctx->tuning.grab;
    t->box_margin = ctx->tuning.box_margin;
    return VLL_OK;
}

// ---- TINCreate_list (SubFunctions.cpp:2768-2846) ------------------------------
static int tin_create_check(vll_context *ctx, const void *pts, int64_t n_pts,
                            const double *min_max, double resolution, const void *tris,
                            int64_t capacity, int64_t *count) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (!min_max || !count || (n_pts > 0 && !pts) || (capacity > 0 && !tris))
        return fail(ctx, VLL_ERR_INVALID, "null argument");
    if (n_pts < 0 || capacity < 0) return fail(ctx, VLL_ERR_INVALID, "negative count");
    if (!(resolution > 0) || !(min_max[2] >= min_max[0]) || !(min_max[3] >= min_max[1]))
        return fail(ctx, VLL_ERR_INVALID, "invalid resolution or extent");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    return VLL_OK;
}

int vll_tin_create_device(vll_context *ctx, const vll_point3 *d_pts, int64_t n_pts,
                          const double min_max[4], double resolution, vll_tri *d_tris,
                          int64_t capacity, int64_t *count) {
    NvtxRange nvtx_range("vll_tin_create_device");
    int rc = tin_create_check(ctx, d_pts, n_pts, min_max, resolution, d_tris, capacity, count);
    if (rc) return rc;
    std::string err;
    rc = vll::run_tin_create(ctx->tin_work, d_pts, n_pts, min_max, resolution, d_tris, capacity,
                             count, ctx->stream, &err);
    if (rc) return fail(ctx, rc, err);
    ctx->launches_total += 1;
    return VLL_OK;
}

int vll_tin_create(vll_context *ctx, const vll_point3 *pts, int64_t n_pts, const double min_max[4],
                   double resolution, vll_tri *tris, int64_t capacity, int64_t *count) {
    NvtxRange nvtx_range("vll_tin_create");
    int rc = tin_create_check(ctx, pts, n_pts, min_max, resolution, tris, capacity, count);
    if (rc) return rc;
    VLL_CUDA(ctx, ensure(ctx->tin_pts, (size_t)std::max<int64_t>(n_pts, 1) * sizeof(vll_point3)));
    VLL_CUDA(ctx, ensure(ctx->tin_tris, (size_t)std::max<int64_t>(capacity, 1) * sizeof(vll_tri)));
    if (n_pts > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(ctx->tin_pts.p, pts, (size_t)n_pts * sizeof(vll_point3),
                                      cudaMemcpyHostToDevice, ctx->stream));
    std::string err;
    rc = vll::run_tin_create(ctx->tin_work, (const vll_point3 *)ctx->tin_pts.p, n_pts, min_max,
                             resolution, (vll_tri *)ctx->tin_tris.p, capacity, count, ctx->stream,
                             &err);
    if (rc) return fail(ctx, rc, err);
    if (*count > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(tris, ctx->tin_tris.p, (size_t)*count * sizeof(vll_tri),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

// ---- residency of the host-buffer calls ------------------------------------
int vll_set_residency(vll_context *ctx, int flags) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    if (flags & ~(VLL_RESIDENT_PLANES | VLL_RESIDENT_VOXELS))
        return fail(ctx, VLL_ERR_INVALID, "unknown residency flag");
    ctx->residency = flags;
    if (!(flags & VLL_RESIDENT_VOXELS)) ctx->rvox_total = -1;
    return VLL_OK;
}

int vll_get_residency(const vll_context *ctx) { return ctx ? ctx->residency : 0; }

int vll_resident_reset(vll_context *ctx) {
    if (!ctx) return fail(nullptr, VLL_ERR_INVALID, "null context");
    ctx->rvox_total = -1;
    ctx->rvox_nodes = 0;
    return VLL_OK;
}

int vll_resident_voxels(vll_context *ctx, vll_voxel *voxels, int64_t capacity, int64_t *total) {
    if (!ctx || !total) return fail(ctx, VLL_ERR_INVALID, "null argument");
    if (ctx->rvox_total < 0) return fail(ctx, VLL_ERR_INVALID, "no resident voxel packing");
    *total = ctx->rvox_total;
    if (ctx->rvox_total > capacity || (ctx->rvox_total > 0 && !voxels))
        return fail(ctx, VLL_ERR_CAPACITY, "resident packing longer than the buffer");
    VLL_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->rvox_total > 0)
        VLL_CUDA(ctx, cudaMemcpyAsync(voxels, ctx->rvox.p,
                                      (size_t)ctx->rvox_total * sizeof(vll_voxel),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    VLL_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return VLL_OK;
}

}  // extern "C"

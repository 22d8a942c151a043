// vll_split.cu -- split-precision VerticalLineLocus (setsm_code.cpp:6049-6548).
//
// Pipeline for one level (all on one stream, no host round trips):
//   gncc    FP64 GNCC per node (height independent), when the level uses it
//   prep    per node: image-boundary and blunder tests, the nccresult fields
//           VerticalLineLocus sets before its height loop, slot count K
//   scan    exclusive prefix sums -> slot offsets and (node, 32-slot) items
//   ncc     persistent kernel draining the item queue: one warp per item,
//           one lane per height slot.  FP64 RPC projection; the warp's
//           window footprints in both images are staged in shared memory as
//           FP32 (intensity, magnitude) texel pairs; bilinear sampling and
//           shifted (mean-centred) window sums in FP32; per-slot rho.
//   peaks   ordered FindPeakNcc scan per node over the FP32 rho; any decision
//           whose FP32 inputs lie inside the error band (direction ties,
//           rounding / truncation boundaries, variance threshold) queues the
//           slots involved for exact re-evaluation
//   recheck FP64 re-evaluation of the queued slots (the plain kernel's code)
//   rescan  the scan again with the exact values; a node whose outcome still
//           depends on an unverified FP32 value is recomputed entirely in FP64
// The result is identical to the FP64 kernel's; FP32 only decides when it is
// provably far enough from every boundary.
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <cub/device/device_scan.cuh>

#include "vll_exact.cuh"
#include "vll_internal.h"
#include "vll_split.h"

namespace vll {

// Half-width of the FP32 error band in rho units.  The measured FP32-vs-FP64
// error of rho is below 2e-6; decisions closer than this to a boundary are
// settled in FP64.
constexpr float kBand = 2e-5f;
constexpr int kMaxRecheck = 32;         // per node, beyond which the node is redone in FP64
constexpr int kFullRedo = 255;

// Per-slot markers in the rho buffer (.x):
constexpr float kNotEvaluated = INFINITY;    // slot skipped (range / image bounds)
constexpr float kRejected = -INFINITY;       // orientation check failed

// ---------------------------------------------------------------------------
// prep: per-node setup (setsm_code.cpp:6158-6328)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) prep_kernel(const DevLevel *__restrict__ Pp,
                                                   const double *__restrict__ gsum,
                                                   const double *__restrict__ gcnt,
                                                   int32_t *__restrict__ node_k,
                                                   int32_t *__restrict__ item_cnt,
                                                   unsigned long long *__restrict__ counters) {
    const DevLevel &P = *Pp;
    unsigned long long acc = 0;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        int K = 0;
        const vll_ugrid g = P.gp3[pt];
        const int start_H = g.minHeight, end_H = g.maxHeight;
        const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
        if (check_image_boundary(P, lon, lat, (double)start_H, (double)end_H, P.H) &&
            !blunder_cell(P, g)) {
            acc++;
            vll_nccresult &R = P.ncc[pt];
            const int ti = 1;
            if (P.check_ortho && dq_result(ugrid_ortho_ncc(P.gp3, P.n_nodes, pt, ti)) > P.ortho_th)
                R.GNCC = gcnt[pt] > 0 ? q_result(__ddiv_rn(gsum[pt], gcnt[pt])) : q_result(-1.0);
            else
                R.GNCC = q_result(-1.0);
            const int num_heights = (int)__ddiv_rn((double)(end_H - start_H), P.height_step);
            if (P.is_ra || P.cmr) {
                R.check_height_change = 1;
                R.NumOfHeight = (uint16_t)num_heights;
            }
            if (P.is_ra || P.cmr || R.check_height_change || (P.L == 0 && P.dem_res < 2)) {
                R.result0 = q_result(-1.0);
                R.result2 = -1000;
                R.result1 = q_result(-1.0);
                R.result3 = -1000;
                R.result4 = 0;
                K = R.NumOfHeight;
                if (K == 0 && R.check_height_change) R.max_WNCC = q_result(-100.0);
            }
        }
        node_k[pt] = K;
        item_cnt[pt] = (K + 31) / 32;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&counters[0], acc);
}

__global__ void __launch_bounds__(256) items_kernel(int64_t n, const int32_t *__restrict__ item_cnt,
                                                    const int64_t *__restrict__ item_off,
                                                    int64_t *__restrict__ items) {
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < n;
         pt += (int64_t)gridDim.x * blockDim.x) {
        const int c = item_cnt[pt];
        const int64_t o = item_off[pt];
        for (int i = 0; i < c; ++i) items[o + i] = (pt << 16) | (int64_t)(32 * i);
    }
}

// ---------------------------------------------------------------------------
// ncc: the FP32 window kernel
// ---------------------------------------------------------------------------
// Ring of a window offset: 2 = innermost sub-window, 1 = middle, 0 = outer.
__host__ __device__ constexpr int ring_of(int H, int row, int col) {
    const int r2 = row * row + col * col;
    const int s1 = H / 2;
    const int s2 = s1 + (int)((s1 / 2.0) + 0.5);
    const bool w1 = r2 <= (H - s1 + 1) * (H - s1 + 1) && row >= -H + s1 && row <= H - s1 &&
                    col >= -H + s1 && col <= H - s1;
    const bool w2 = r2 <= (H - s2 + 1) * (H - s2 + 1) && row >= -H + s2 && row <= H - s2 &&
                    col >= -H + s2 && col <= H - s2;
    return w2 ? 2 : (w1 ? 1 : 0);
}

__host__ __device__ constexpr int ring_count(int H, int ring) {
    int n = 0;
    for (int row = -H; row <= H; ++row)
        for (int col = -H; col <= H; ++col)
            if (row * row + col * col <= (H + 1) * (H + 1) && ring_of(H, row, col) == ring) ++n;
    return n;
}

// floor and fraction of a small float with full-rate ALU ops only:
// round-to-nearest of (x - 0.5) through the 1.5*2^23 magic constant.
__device__ __forceinline__ int floor_frac(float x, float &frac) {
    const float t = __fadd_rn(__fadd_rn(x, -0.5f), 12582912.0f);
    const float r = __fadd_rn(t, -12582912.0f);
    frac = x - r;
    return __float_as_int(t) - 0x4B400000;
}

struct Acc {
    float sl, sr, sll, srr, slr;
};

// Pearson rho from shifted sums; returns -99 when a variance is below the
// reference's 1e-8 threshold and flags results whose variance is too small
// for FP32 to decide that threshold safely.
__device__ __forceinline__ float corr_from(const Acc &a, float n, bool &unsure) {
    const float inv = 1.0f / n;
    const float vl = a.sll - a.sl * a.sl * inv;
    const float vr = a.srr - a.sr * a.sr * inv;
    const float cv = a.slr - a.sl * a.sr * inv;
    // FP32 relative error of vl is ~n * 6e-8 * (sll / vl); treat anything
    // within a factor of the threshold, or heavily cancelled, as uncertain.
    if (vl < 1e-3f * a.sll + 1e-4f || vr < 1e-3f * a.srr + 1e-4f) unsure = true;
    if (!(vl > 1e-8f && vr > 1e-8f)) return -99.0f;
    return cv * rsqrtf(vl * vr);
}

template <int H>
__device__ __forceinline__ void window_fp32(const float4 *__restrict__ qr, int rbw, float rfx,
                                            float rfy, const float4 *__restrict__ qt, int tbw,
                                            float tfx, float tfy, float c, float s, float &incc_avg,
                                            bool &unsure) {
    Acc acc[3][2];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int p = 0; p < 2; ++p) acc[r][p] = Acc{0.f, 0.f, 0.f, 0.f, 0.f};
    const float w00 = (1.f - rfx) * (1.f - rfy), w10 = rfx * (1.f - rfy);
    const float w01 = (1.f - rfx) * rfy, w11 = rfx * rfy;
#pragma unroll
    for (int row = -H; row <= H; ++row) {
        const float4 *q0 = qr + (row + H) * rbw;
        const float4 *q1 = q0 + rbw;
        const float bx = fmaf(-s, (float)row, tfx);
        const float by = fmaf(c, (float)row, tfy);
#pragma unroll
        for (int col = -H; col <= H; ++col) {
            if (row * row + col * col > (H + 1) * (H + 1)) continue;
            const int ring = ring_of(H, row, col);
            const float4 a = q0[col + H];
            const float4 b = q1[col + H];
            const float lI = fmaf(w11, b.z, fmaf(w01, b.x, fmaf(w10, a.z, w00 * a.x)));
            const float lM = fmaf(w11, b.w, fmaf(w01, b.y, fmaf(w10, a.w, w00 * a.y)));
            const float fx = fmaf(c, (float)col, bx);
            const float fy = fmaf(s, (float)col, by);
            float frx, fry;
            const int ix = floor_frac(fx, frx);
            const int iy = floor_frac(fy, fry);
            const float4 *t = qt + iy * tbw + ix;
            const float4 ta = t[0];
            const float4 tb = t[tbw];
            const float topI = fmaf(frx, ta.z - ta.x, ta.x);
            const float botI = fmaf(frx, tb.z - tb.x, tb.x);
            const float rI = fmaf(fry, botI - topI, topI);
            const float topM = fmaf(frx, ta.w - ta.y, ta.y);
            const float botM = fmaf(frx, tb.w - tb.y, tb.y);
            const float rM = fmaf(fry, botM - topM, topM);
            Acc &x = acc[ring][0];
            x.sl += lI;
            x.sr += rI;
            x.sll = fmaf(lI, lI, x.sll);
            x.srr = fmaf(rI, rI, x.srr);
            x.slr = fmaf(lI, rI, x.slr);
            Acc &y = acc[ring][1];
            y.sl += lM;
            y.sr += rM;
            y.sll = fmaf(lM, lM, y.sll);
            y.srr = fmaf(rM, rM, y.srr);
            y.slr = fmaf(lM, rM, y.slr);
        }
    }
    // nested windows: 2 = ring 2; 1 = rings 1+2; 0 = all rings
    constexpr int n2 = ring_count(H, 2);
    constexpr int n1 = n2 + ring_count(H, 1);
    constexpr int n0 = n1 + ring_count(H, 0);
    float tot = 0.f;
    int nv = 0;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        Acc w = acc[2][p];
        const float r2 = corr_from(w, (float)n2, unsure);
        w.sl += acc[1][p].sl;
        w.sr += acc[1][p].sr;
        w.sll += acc[1][p].sll;
        w.srr += acc[1][p].srr;
        w.slr += acc[1][p].slr;
        const float r1 = corr_from(w, (float)n1, unsure);
        w.sl += acc[0][p].sl;
        w.sr += acc[0][p].sr;
        w.sll += acc[0][p].sll;
        w.srr += acc[0][p].srr;
        w.slr += acc[0][p].slr;
        const float r0 = corr_from(w, (float)n0, unsure);
        if (r0 != -99.0f) { tot += r0; ++nv; }
        if (r1 != -99.0f) { tot += r1; ++nv; }
        if (r2 != -99.0f) { tot += r2; ++nv; }
    }
    // count_incc is 1 when any of the six correlations is defined
    incc_avg = nv > 0 ? tot / (float)nv : -1.0f;
    if (nv == 0) incc_avg = -2.0f;   // no valid correlation: count_incc stays 0
}

struct ItemCtx {
    int64_t node;
    int k0;
    int K;
};

// Stages the texel pairs of box [x0, x0+bw) x [y0, y0+bh) of one image into
// shared memory as float4 {I(x)-sI, M(x)-sM, I(x+1)-sI, M(x+1)-sM}; returns
// true (warp-uniform) when some intensity texel in the box is zero.
__device__ __forceinline__ bool stage_box(float4 *__restrict__ dst, const uint16_t *__restrict__ I,
                                          const uint16_t *__restrict__ M, uint32_t W, int x0, int y0,
                                          int bw, int bh, float sI, float sM, int lane) {
    bool zero = false;
    const int n = bw * bh;
    for (int i = lane; i < n; i += 32) {
        const int by = i / bw;
        const int bx = i - by * bw;
        const int64_t p = (int64_t)(y0 + by) * W + (x0 + bx);
        const uint16_t a = __ldg(I + p), b = __ldg(I + p + 1);
        const uint16_t cm = __ldg(M + p), d = __ldg(M + p + 1);
        zero |= (a == 0) | (b == 0);
        dst[i] = make_float4((float)a - sI, (float)cm - sM, (float)b - sI, (float)d - sM);
    }
    return __any_sync(0xffffffffu, zero);
}

template <int H>
__global__ void __launch_bounds__(128) ncc_kernel(const DevLevel *__restrict__ Pp,
                                                  const int64_t *__restrict__ items, int64_t n_items,
                                                  const int64_t *__restrict__ slot_off,
                                                  const double *__restrict__ gsum,
                                                  const double *__restrict__ gcnt,
                                                  float2 *__restrict__ rho,
                                                  unsigned long long *__restrict__ counters,
                                                  unsigned long long *__restrict__ queue,
                                                  int warp_quads) {
    extern __shared__ float4 smem[];
    const DevLevel &P = *Pp;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float4 *sw = smem + (size_t)warp * warp_quads;
    const DevImage &ri = P.im[P.ref];
    const DevImage &tI = P.im[1];
    PatchSrc S, Sn;
    make_src(P, 1, S, Sn);
    unsigned long long evals = 0;
    constexpr int kGrab = 4;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(queue, (unsigned long long)kGrab);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)n_items) break;
        for (int g = 0; g < kGrab; ++g) {
            const int64_t it = (int64_t)base + g;
            if (it >= n_items) break;
            const int64_t code = items[it];
            const int64_t pt = code >> 16;
            const int k0 = (int)(code & 0xFFFF);
            const int64_t so = slot_off[pt];
            const int K = (int)(slot_off[pt + 1] - so);
            const int k = k0 + lane;
            const vll_ugrid gg = P.gp3[pt];
            const int start_H = gg.minHeight, end_H = gg.maxHeight;
            const int ncc_min = P.ncc[pt].minHeight;
            const double cnt_g = gcnt ? gcnt[pt] : 0.0, sum_g = gsum ? gsum[pt] : 0.0;
            // ---- per-lane geometry (FP64) ----
            int status = 0;   // 0 idle/skip, 1 orientation reject, 2 evaluate
            double2 rp = make_double2(0, 0), tp = make_double2(0, 0);
            int rot = kRotOffset;
            float hgt = 0.f;
            if (k < K) {
                hgt = slot_height(P, start_H, ncc_min, k);
                if (hgt >= (float)start_H && hgt <= (float)end_H) {
                    const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
                    rp = to_pyramid(rpc_project(ri.rpc, ri.adj, lon, lat, (double)hgt), ri.sx, ri.sy, P.L);
                    tp = to_pyramid(rpc_project(tI.rpc, tI.adj, lon, lat, (double)hgt), tI.sx, tI.sy, P.L);
                    if (in_image(rp, ri.w, ri.h) && in_image(tp, tI.w, tI.h)) {
                        const int od = (int)ri.ori[(int64_t)(int)rp.y * ri.w + (int)rp.x] -
                                       (int)tI.ori[(int64_t)(int)tp.y * tI.w + (int)tp.x];
                        bool ok = true;
                        if (!P.is_ra && P.L >= 3) {
                            const double a = __dmul_rn((double)od, P.bin_angle);
                            ok = a < 90 && a > -90;
                        }
                        status = ok ? 2 : 1;
                        rot = 2 * od + kRotOffset;
                    }
                }
            }
            // ---- footprint of the evaluating lanes ----
            const float cf = (float)P.rot_cos[rot], sf = (float)P.rot_sin[rot];
            const int rix = (int)floor(rp.x), riy = (int)floor(rp.y);
            const int tix = (int)floor(tp.x), tiy = (int)floor(tp.y);
            const int R = (int)ceilf((fabsf(cf) + fabsf(sf)) * (float)H) + 1;
            bool inside = status == 2 && rix - H >= 0 && riy - H >= 0 &&
                          rix + H + 2 < (int)ri.w && riy + H + 2 < (int)ri.h && tix - R >= 0 &&
                          tiy - R >= 0 && tix + R + 2 < (int)tI.w && tiy + R + 2 < (int)tI.h;
            int rx0 = inside ? rix - H : INT_MAX, ry0 = inside ? riy - H : INT_MAX;
            int rx1 = inside ? rix + H + 1 : INT_MIN, ry1 = inside ? riy + H + 1 : INT_MIN;
            int tx0 = inside ? tix - R : INT_MAX, ty0 = inside ? tiy - R : INT_MAX;
            int tx1 = inside ? tix + R + 1 : INT_MIN, ty1 = inside ? tiy + R + 1 : INT_MIN;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                rx0 = min(rx0, __shfl_xor_sync(0xffffffffu, rx0, o));
                ry0 = min(ry0, __shfl_xor_sync(0xffffffffu, ry0, o));
                rx1 = max(rx1, __shfl_xor_sync(0xffffffffu, rx1, o));
                ry1 = max(ry1, __shfl_xor_sync(0xffffffffu, ry1, o));
                tx0 = min(tx0, __shfl_xor_sync(0xffffffffu, tx0, o));
                ty0 = min(ty0, __shfl_xor_sync(0xffffffffu, ty0, o));
                tx1 = max(tx1, __shfl_xor_sync(0xffffffffu, tx1, o));
                ty1 = max(ty1, __shfl_xor_sync(0xffffffffu, ty1, o));
            }
            const bool any_inside = __any_sync(0xffffffffu, inside);
            bool staged = false;
            int rbw = 0, tbw = 0;
            if (any_inside) {
                rbw = rx1 - rx0 + 1;
                const int rbh = ry1 - ry0 + 1;
                tbw = tx1 - tx0 + 1;
                const int tbh = ty1 - ty0 + 1;
                if (rbw * rbh + tbw * tbh <= warp_quads) {
                    // shift: texel at the centre of the reference box
                    float sI = 0.f, sM = 0.f, tsI = 0.f, tsM = 0.f;
                    if (lane == 0) {
                        const int64_t pc = (int64_t)(ry0 + rbh / 2) * ri.w + (rx0 + rbw / 2);
                        sI = (float)__ldg(ri.img + pc);
                        sM = (float)__ldg(ri.mag + pc);
                        const int64_t pt2 = (int64_t)(ty0 + tbh / 2) * tI.w + (tx0 + tbw / 2);
                        tsI = (float)__ldg(tI.img + pt2);
                        tsM = (float)__ldg(tI.mag + pt2);
                    }
                    sI = __shfl_sync(0xffffffffu, sI, 0);
                    sM = __shfl_sync(0xffffffffu, sM, 0);
                    tsI = __shfl_sync(0xffffffffu, tsI, 0);
                    tsM = __shfl_sync(0xffffffffu, tsM, 0);
                    __syncwarp();
                    const bool z1 = stage_box(sw, ri.img, ri.mag, ri.w, rx0, ry0, rbw, rbh, sI, sM, lane);
                    const bool z2 = stage_box(sw + rbw * rbh, tI.img, tI.mag, tI.w, tx0, ty0, tbw, tbh,
                                              tsI, tsM, lane);
                    __syncwarp();
                    staged = !(z1 || z2);
                }
            }
            float rho_v = kNotEvaluated, incc_v = 0.f;
            bool all_pos = false;
            if (status == 1) {
                rho_v = kRejected;
            } else if (status == 2) {
                if (staged && inside) {
                    float incc;
                    bool unsure = false;
                    window_fp32<H>(sw + (riy - H - ry0) * rbw + (rix - H - rx0), rbw,
                                   (float)(rp.x - (double)rix), (float)(rp.y - (double)riy),
                                   sw + rbw * (ry1 - ry0 + 1) + (tiy - ty0) * tbw + (tix - tx0), tbw,
                                   (float)(tp.x - (double)tix), (float)(tp.y - (double)tiy), cf, sf,
                                   incc, unsure);
                    double rho_d;
                    const double incc_d = incc == -2.0f ? -1.0 : (double)incc;
                    const bool has = incc != -2.0f;
                    if (P.check_ortho && cnt_g > 0)
                        rho_d = has ? incc_d * P.alpha + __ddiv_rn(sum_g, cnt_g) * P.beta
                                    : __ddiv_rn(0.0, 0.0);
                    else
                        rho_d = incc_d;
                    rho_v = (float)rho_d;
                    incc_v = unsure ? __int_as_float(0x7fc00000) : (float)incc_d;
                    all_pos = true;   // window inside the image, no zero texels
                } else {
                    const SlotOut o = eval_slot(P, pt, 1, S, Sn, hgt, cnt_g, sum_g);
                    all_pos = o.all_pos;
                    rho_v = (float)o.rho;
                    incc_v = (float)(o.count_incc > 0 ? __ddiv_rn(o.sum_incc, o.count_incc) : -1.0);
                }
                evals++;
            }
            if (k < K) rho[so + k] = make_float2(rho_v, incc_v);
            if (k < K && P.vox && !P.cmr && !P.is_ra) {
                vll_voxel *v = P.vox + P.vox_off[pt] + k;
                if (status == 1) v->flag_cal = 0;
                if (status == 2) {
                    if (all_pos) v->flag_cal = 1;
                    v->INCC = q_voxel((double)incc_v);
                }
            }
            __syncwarp();
        }
    }
    for (int o = 16; o; o >>= 1) evals += __shfl_down_sync(0xffffffffu, evals, o);
    if (lane == 0 && evals) atomicAdd(&counters[1], evals);
}

// ---------------------------------------------------------------------------
// peaks / rescan
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool near_round(double v) {
    const double x = v * 1000.0;
    return fabs(x - floor(x) - 0.5) < (double)kBand * 1000.0;
}
__device__ __forceinline__ bool near_trunc(double v) {
    const double x = v * 1000.0;
    return fabs(x - rint(x)) < (double)kBand * 1000.0;
}

struct Overrides {
    int n;
    int k[kMaxRecheck];
    double rho[kMaxRecheck];
    double incc[kMaxRecheck];
};

struct NeedList {
    int n = 0;
    bool overflow = false;
    int k[kMaxRecheck];
    __device__ void add(int kk) {
        for (int i = 0; i < n; ++i)
            if (k[i] == kk) return;
        if (n < kMaxRecheck)
            k[n++] = kk;
        else
            overflow = true;
    }
};

__device__ __forceinline__ bool lookup(const Overrides &ov, int k, int &oi, double &v, double &incc) {
    while (oi < ov.n && ov.k[oi] < k) ++oi;
    if (oi < ov.n && ov.k[oi] == k) {
        v = ov.rho[oi];
        incc = ov.incc[oi];
        return true;
    }
    return false;
}

// One node's FindPeakNcc scan (setsm_code.cpp:6672-6752) and max_WNCC over
// the slot values (FP32 from the window kernel, or exact FP64 for slots in
// `ov`).  Every decision whose FP32 inputs lie within kBand of a boundary --
// the sign tests and the difference of the direction rule, the rounding of a
// peak value or of the maximum, the truncation of a voxel -- adds the FP32
// slot(s) to `need`.  The outcome is exact when `need` stays empty.
__device__ void scan_node(const DevLevel &P, int64_t pt, const float2 *__restrict__ rv, int K,
                          const Overrides &ov, NeedList &need, vll_nccresult &R) {
    R = P.ncc[pt];
    const bool voxels = !P.cmr && !P.is_ra;
    const int start_H = P.gp3[pt].minHeight;
    int check_rho = 0, direction = 0, pre_k = -1;
    double pre_rho = -1.0;
    float pre_height = 0.0f;
    bool pre_exact = true;
    double max_w = -100;
    int oi = 0;
    for (int k = 0; k < K; ++k) {
        const float2 v2 = rv[k];
        if (v2.x == kNotEvaluated || v2.x == kRejected) continue;
        double v = (double)v2.x, incc = (double)v2.y;
        const bool exact = lookup(ov, k, oi, v, incc);
        if (!exact && (isnan(v2.y) || (voxels && near_trunc(incc)))) need.add(k);
        if (P.cmr) {
            if (check_rho && !(exact && pre_exact) &&
                (fabs(v - pre_rho) < kBand || fabs(v) < kBand || fabs(pre_rho) < kBand)) {
                if (!exact) need.add(k);
                if (!pre_exact) need.add(pre_k);
            }
            double diff;
            if (v >= 0 && pre_rho >= 0)
                diff = v - pre_rho;
            else if (v < 0 && pre_rho < 0)
                diff = -(fabs(v) - fabs(pre_rho));
            else if (v >= 0 && pre_rho < 0)
                diff = 1;
            else
                diff = -1;
            int td = diff > 0 ? 1 : (diff < 0 ? -1 : 0);
            if (!check_rho) {
                check_rho = 1;
                td = -1;
            } else if (pre_rho != -1) {
                if (direction > 0 && td < 0) {
                    if (!pre_exact && near_round(pre_rho)) need.add(pre_k);
                    if (R.result4 < 10) R.result4 += 1;
                    const int16_t qpre = q_result(pre_rho);
                    if (R.result0 < qpre) {
                        const double t1 = dq_result(R.result0);
                        R.result0 = qpre;
                        const float t2 = R.result2;
                        R.result2 = pre_height;
                        const int16_t q1 = q_result(t1);
                        if (R.result1 < q1) {
                            R.result1 = q1;
                            R.result3 = t2;
                        }
                    } else if (R.result1 < qpre) {
                        R.result1 = qpre;
                        R.result3 = pre_height;
                    }
                }
            }
            pre_rho = v;
            pre_height = slot_height(P, start_H, R.minHeight, k);
            direction = td;
            pre_k = k;
            pre_exact = exact;
        }
        if (max_w < v) max_w = v;
    }
    if (R.check_height_change) {
        // the rounded maximum: any FP32 value within the band of the maximum
        // that sits near a rounding boundary must be exact
        oi = 0;
        for (int k = 0; k < K; ++k) {
            const float2 v2 = rv[k];
            if (v2.x == kNotEvaluated || v2.x == kRejected) continue;
            double v = (double)v2.x, incc = (double)v2.y;
            if (lookup(ov, k, oi, v, incc)) continue;
            if (v >= max_w - kBand && near_round(v)) need.add(k);
        }
        R.max_WNCC = q_result(max_w);
    }
}

__global__ void __launch_bounds__(128) peaks_kernel(const DevLevel *__restrict__ Pp,
                                                    const int64_t *__restrict__ slot_off,
                                                    const float2 *__restrict__ rho,
                                                    int64_t *__restrict__ re_items, int64_t cap_re,
                                                    int64_t *__restrict__ node_re,
                                                    int64_t *__restrict__ pending,
                                                    unsigned long long *__restrict__ ctl,
                                                    unsigned long long *__restrict__ counters) {
    const DevLevel &P = *Pp;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        const int64_t so = slot_off[pt];
        const int K = (int)(slot_off[pt + 1] - so);
        if (K == 0) continue;
        Overrides none;
        none.n = 0;
        NeedList need;
        vll_nccresult R;
        scan_node(P, pt, rho + so, K, none, need, R);
        if (need.n == 0 && !need.overflow) {
            P.ncc[pt] = R;
            continue;
        }
        int64_t code = kFullRedo;
        if (!need.overflow) {
            // ascending slot order for the re-scan's merge
            for (int i = 1; i < need.n; ++i) {
                const int x = need.k[i];
                int j = i - 1;
                while (j >= 0 && need.k[j] > x) {
                    need.k[j + 1] = need.k[j];
                    --j;
                }
                need.k[j + 1] = x;
            }
            const unsigned long long start = atomicAdd(&ctl[1], (unsigned long long)need.n);
            if ((int64_t)(start + need.n) <= cap_re) {
                for (int i = 0; i < need.n; ++i) re_items[start + i] = (pt << 16) | need.k[i];
                code = ((int64_t)start << 8) | need.n;
                atomicAdd(&counters[2], (unsigned long long)need.n);
            }
        }
        if (code == kFullRedo) atomicAdd(&counters[2], (unsigned long long)K);
        node_re[pt] = code;
        const unsigned long long slot = atomicAdd(&ctl[2], 1ull);
        pending[slot] = pt;
    }
}

__global__ void __launch_bounds__(64) rescan_kernel(const DevLevel *__restrict__ Pp,
                                                    const int64_t *__restrict__ slot_off,
                                                    const float2 *__restrict__ rho,
                                                    const int64_t *__restrict__ node_re,
                                                    const int64_t *__restrict__ pending,
                                                    const int64_t *__restrict__ re_items,
                                                    const double *__restrict__ re_out,
                                                    const unsigned long long *__restrict__ ctl) {
    const DevLevel &P = *Pp;
    const unsigned long long n = ctl[2];
    const bool voxels = P.vox && !P.cmr && !P.is_ra;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const int64_t pt = pending[i];
        const int64_t code = node_re[pt];
        bool redo = code == kFullRedo;
        if (!redo) {
            const int64_t start = code >> 8;
            Overrides ov;
            ov.n = (int)(code & 0xFF);
            for (int j = 0; j < ov.n; ++j) {
                ov.k[j] = (int)(re_items[start + j] & 0xFFFF);
                ov.rho[j] = re_out[2 * (start + j)];
                ov.incc[j] = re_out[2 * (start + j) + 1];
            }
            const int64_t so = slot_off[pt];
            const int K = (int)(slot_off[pt + 1] - so);
            NeedList need;
            vll_nccresult R;
            scan_node(P, pt, rho + so, K, ov, need, R);
            if (need.n == 0 && !need.overflow) {
                P.ncc[pt] = R;
                if (voxels) {
                    vll_voxel *row = P.vox + P.vox_off[pt];
                    for (int j = 0; j < ov.n; ++j) row[ov.k[j]].INCC = q_voxel(ov.incc[j]);
                }
            } else {
                redo = true;
            }
        }
        if (redo) {
            // outcome still depends on FP32 values near a boundary: recompute
            // the node exactly (resets its results like VerticalLineLocus)
            unsigned long long a = 0, e = 0;
            plain_node(P, pt, a, e, nullptr, nullptr);
        }
    }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
namespace {

cudaError_t grow(void *&p, size_t &cap, size_t need) {
    if (need == 0) need = 1;
    if (need <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, need);
    if (e == cudaSuccess) cap = need;
    return e;
}

unsigned grid_1d(int64_t n, int threads, int64_t cap_blocks) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap_blocks) b = cap_blocks;
    return (unsigned)b;
}

template <int H>
cudaError_t launch_ncc(const DevLevel *dP, const int64_t *items, int64_t n_items,
                       const int64_t *slot_off, const double *gsum, const double *gcnt, float2 *rho,
                       unsigned long long *counters, unsigned long long *queue, cudaStream_t s) {
    // per-warp shared footprint: both images' boxes, float4 texel pairs
    const int warp_quads = 1024;
    const int threads = 128;
    const size_t smem = (size_t)(threads / 32) * warp_quads * sizeof(float4);
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(ncc_kernel<H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ncc_kernel<H>, threads, smem);
    if (per_sm < 1) per_sm = 1;
    ncc_kernel<H><<<sms * per_sm, threads, smem, s>>>(dP, items, n_items, slot_off, gsum, gcnt, rho,
                                                      counters, queue, warp_quads);
    return cudaGetLastError();
}

}  // namespace

bool split_supported(const DevLevel &P) {
    return P.num_images == 2 && P.ref == 0 && P.im[1].selected && !P.is_ra && !P.combined_incc &&
           (P.H == 2 || P.H == 3 || P.H == 4 || P.H == 5 || P.H == 6 || P.H == 7);
}

void split_release(SplitBuffers &b) {
    void **all[] = {&b.node_k, &b.slot_off, &b.item_cnt, &b.item_off, &b.items, &b.rho, &b.gsum,
                    &b.gcnt, &b.re_items, &b.re_out, &b.node_re, &b.scan_tmp, &b.ctl, &b.pending};
    for (void **p : all) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    b.cap_nodes = b.cap_slots = b.cap_items = b.cap_re = b.cap_scan = 0;
}

#define SPLIT_CUDA(call)                       \
    do {                                       \
        cudaError_t e__ = (call);              \
        if (e__ != cudaSuccess) {              \
            *err = #call;                      \
            return e__;                        \
        }                                      \
    } while (0)

cudaError_t run_split(SplitBuffers &b, const DevLevel &P, const DevLevel *dP,
                      unsigned long long *counters, cudaStream_t s, std::string *err,
                      SplitTiming *tm) {
    const int64_t N = P.n_nodes;
    auto mark = [&](int i) {
        if (tm && tm->enabled) cudaEventRecord(tm->ev[i], s);
    };
    int64_t launches = 0;
    size_t cap;
    // node-sized buffers
    if ((size_t)(N + 1) > b.cap_nodes) {
        size_t c8 = 0;
        void **nb[] = {&b.node_k, &b.item_cnt};
        for (void **p : nb) {
            if (*p) cudaFree(*p);
            *p = nullptr;
            SPLIT_CUDA(cudaMalloc(p, (size_t)(N + 1) * sizeof(int32_t)));
        }
        void **nb8[] = {&b.slot_off, &b.item_off, &b.gsum, &b.gcnt, &b.node_re, &b.pending};
        for (void **p : nb8) {
            if (*p) cudaFree(*p);
            *p = nullptr;
            SPLIT_CUDA(cudaMalloc(p, (size_t)(N + 1) * 8));
        }
        (void)c8;
        b.cap_nodes = (size_t)(N + 1);
    }
    if (!b.ctl) SPLIT_CUDA(cudaMalloc(&b.ctl, 8 * sizeof(unsigned long long)));
    SPLIT_CUDA(cudaMemsetAsync(b.ctl, 0, 8 * sizeof(unsigned long long), s));
    SPLIT_CUDA(cudaMemsetAsync(b.node_k, 0, (size_t)(N + 1) * sizeof(int32_t), s));
    SPLIT_CUDA(cudaMemsetAsync(b.item_cnt, 0, (size_t)(N + 1) * sizeof(int32_t), s));
    double *gsum = nullptr, *gcnt = nullptr;
    mark(0);
    if (P.check_ortho) {
        gsum = (double *)b.gsum;
        gcnt = (double *)b.gcnt;
        SPLIT_CUDA(launch_gncc(dP, N, gsum, gcnt, s));
        ++launches;
    }
    mark(1);
    prep_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(dP, gsum, gcnt, (int32_t *)b.node_k,
                                                          (int32_t *)b.item_cnt, counters);
    SPLIT_CUDA(cudaGetLastError());
    ++launches;
    mark(2);
    // prefix sums (int32 counts -> int64 offsets)
    size_t tmp1 = 0, tmp2 = 0;
    SPLIT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp1, (const int32_t *)b.node_k,
                                             (int64_t *)b.slot_off, (int)(N + 1), s));
    SPLIT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, (const int32_t *)b.item_cnt,
                                             (int64_t *)b.item_off, (int)(N + 1), s));
    cap = tmp1 > tmp2 ? tmp1 : tmp2;
    SPLIT_CUDA(grow(b.scan_tmp, b.cap_scan, cap));
    tmp1 = b.cap_scan;
    SPLIT_CUDA(cub::DeviceScan::ExclusiveSum(b.scan_tmp, tmp1, (const int32_t *)b.node_k,
                                             (int64_t *)b.slot_off, (int)(N + 1), s));
    tmp2 = b.cap_scan;
    SPLIT_CUDA(cub::DeviceScan::ExclusiveSum(b.scan_tmp, tmp2, (const int32_t *)b.item_cnt,
                                             (int64_t *)b.item_off, (int)(N + 1), s));
    launches += 4;   // two scans of two kernels each
    mark(3);
    int64_t totals[2];
    SPLIT_CUDA(cudaMemcpyAsync(&totals[0], (int64_t *)b.slot_off + N, 8, cudaMemcpyDeviceToHost, s));
    SPLIT_CUDA(cudaMemcpyAsync(&totals[1], (int64_t *)b.item_off + N, 8, cudaMemcpyDeviceToHost, s));
    SPLIT_CUDA(cudaStreamSynchronize(s));
    const int64_t n_slots = totals[0], n_items = totals[1];
    size_t c = b.cap_slots;
    SPLIT_CUDA(grow(b.rho, c, (size_t)n_slots * sizeof(float2)));
    b.cap_slots = c;
    c = b.cap_items;
    SPLIT_CUDA(grow(b.items, c, (size_t)n_items * sizeof(int64_t)));
    b.cap_items = c;
    const int64_t max_re = N * 4 + 1024;
    if ((size_t)max_re > b.cap_re) {
        if (b.re_items) cudaFree(b.re_items);
        if (b.re_out) cudaFree(b.re_out);
        b.re_items = b.re_out = nullptr;
        SPLIT_CUDA(cudaMalloc(&b.re_items, (size_t)max_re * sizeof(int64_t)));
        SPLIT_CUDA(cudaMalloc(&b.re_out, (size_t)max_re * 2 * sizeof(double)));
        b.cap_re = (size_t)max_re;
    }
    if (n_items > 0) {
        items_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(N, (const int32_t *)b.item_cnt,
                                                               (const int64_t *)b.item_off,
                                                               (int64_t *)b.items);
        SPLIT_CUDA(cudaGetLastError());
        ++launches;
        mark(4);
        unsigned long long *queue = (unsigned long long *)b.ctl;
        cudaError_t e = cudaSuccess;
        switch (P.H) {
            case 2: e = launch_ncc<2>(dP, (const int64_t *)b.items, n_items, (const int64_t *)b.slot_off, gsum, gcnt, (float2 *)b.rho, counters, queue, s); break;
            case 3: e = launch_ncc<3>(dP, (const int64_t *)b.items, n_items, (const int64_t *)b.slot_off, gsum, gcnt, (float2 *)b.rho, counters, queue, s); break;
            case 4: e = launch_ncc<4>(dP, (const int64_t *)b.items, n_items, (const int64_t *)b.slot_off, gsum, gcnt, (float2 *)b.rho, counters, queue, s); break;
            case 5: e = launch_ncc<5>(dP, (const int64_t *)b.items, n_items, (const int64_t *)b.slot_off, gsum, gcnt, (float2 *)b.rho, counters, queue, s); break;
            case 6: e = launch_ncc<6>(dP, (const int64_t *)b.items, n_items, (const int64_t *)b.slot_off, gsum, gcnt, (float2 *)b.rho, counters, queue, s); break;
            case 7: e = launch_ncc<7>(dP, (const int64_t *)b.items, n_items, (const int64_t *)b.slot_off, gsum, gcnt, (float2 *)b.rho, counters, queue, s); break;
            default: e = cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) {
            *err = "ncc_kernel launch";
            return e;
        }
        ++launches;
        mark(5);
        unsigned long long *ctl = (unsigned long long *)b.ctl;
        peaks_kernel<<<grid_1d(N, 128, 148 * 64), 128, 0, s>>>(
            dP, (const int64_t *)b.slot_off, (const float2 *)b.rho, (int64_t *)b.re_items,
            (int64_t)b.cap_re, (int64_t *)b.node_re, (int64_t *)b.pending, ctl, counters);
        SPLIT_CUDA(cudaGetLastError());
        mark(6);
        SPLIT_CUDA(launch_recheck(dP, (const int64_t *)b.re_items, ctl + 1, (int64_t)b.cap_re, gsum,
                                  gcnt, (double *)b.re_out, s));
        mark(7);
        rescan_kernel<<<148 * 8, 64, 0, s>>>(dP, (const int64_t *)b.slot_off, (const float2 *)b.rho,
                                             (const int64_t *)b.node_re, (const int64_t *)b.pending,
                                             (const int64_t *)b.re_items, (const double *)b.re_out,
                                             ctl);
        SPLIT_CUDA(cudaGetLastError());
        launches += 3;
    } else {
        mark(4);
        mark(5);
        mark(6);
        mark(7);
    }
    mark(8);
    if (tm) {
        tm->slots = n_slots;
        tm->launches = launches;
    }
    return cudaSuccess;
}

}  // namespace vll

// ---------------------------------------------------------------------------
// Allocation-free variant of the split pipeline.
//
// Some callers cannot allocate device memory at call time: code running under
// a memory pool that owns the whole device, inside another framework's
// allocator, or in a real-time loop where cudaMalloc's implicit device
// synchronisation is not acceptable.  vll_vertical_line_locus_noalloc runs the
// same split pipeline with every scratch buffer carved out of the file-scope
// array below, so it calls no cudaMalloc / cudaFree / allocating library
// routine.  The array is kNoAllocScratchBytes (64 MiB) and every GPU that
// loads this library holds it until the process exits.
// ---------------------------------------------------------------------------
namespace vll {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[256] = {};

// Device address of the scratch array for the current device, looked up once
// per device (host code cannot use the symbol's address directly).
cudaError_t noalloc_scratch(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

// Slot count per node without touching any output (same tests as prep_kernel
// on the memory-tight route), so that capacity is checked before writing.
__global__ void __launch_bounds__(256) noalloc_count_kernel(const DevLevel *__restrict__ Pp,
                                                            int32_t *__restrict__ node_k,
                                                            int32_t *__restrict__ item_cnt) {
    const DevLevel &P = *Pp;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        int K = 0;
        const vll_ugrid g = P.gp3[pt];
        const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
        if (check_image_boundary(P, lon, lat, (double)g.minHeight, (double)g.maxHeight, P.H) &&
            !blunder_cell(P, g))
            K = (uint16_t)(int)__ddiv_rn((double)(g.maxHeight - g.minHeight), P.height_step);
        node_k[pt] = K;
        item_cnt[pt] = (K + 31) / 32;
    }
}

struct Carver {
    unsigned char *base;
    size_t used, cap;
    void *take(size_t n) {
        const size_t a = (used + 255) & ~(size_t)255;
        if (a + n > cap) return nullptr;
        used = a + n;
        return base + a;
    }
};

thread_local DevLevel g_noalloc_level_host;

}  // namespace

int derive_level(const vll_level_desc *d, DevLevel *P, std::string *err);

}  // namespace vll

extern "C" int vll_vertical_line_locus_noalloc(const vll_level_desc *desc,
                                               const vll_ugrid *d_gridpt3,
                                               vll_nccresult *d_nccresult, void *stream,
                                               int64_t *accessable_grid, char *err_buf,
                                               int err_len) {
    using namespace vll;
    auto fail = [&](int code, const char *msg) {
        if (err_buf && err_len > 0) {
            strncpy(err_buf, msg, (size_t)err_len - 1);
            err_buf[err_len - 1] = 0;
        }
        return code;
    };
    if (!desc || !d_gridpt3 || !d_nccresult) return fail(VLL_ERR_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    DevLevel &P = g_noalloc_level_host;
    std::string err;
    int rc = derive_level(desc, &P, &err);
    if (rc) return fail(rc, err.c_str());
    if (!P.cmr || P.check_ortho || !split_supported(P))
        return fail(VLL_ERR_UNSUPPORTED,
                    "the allocation-free call covers the memory-tight route of stereo levels "
                    "without orthoimage GNCC");
    P.gp3 = d_gridpt3;
    P.ncc = d_nccresult;
    P.vox = nullptr;
    P.vox_off = nullptr;
    void *base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess)
        return fail(VLL_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    const int64_t N = P.n_nodes;
    Carver cv{(unsigned char *)base, 0, kNoAllocScratchBytes};
    DevLevel *dP = (DevLevel *)cv.take(sizeof(DevLevel));
    unsigned long long *ctl = (unsigned long long *)cv.take(8 * sizeof(unsigned long long));
    unsigned long long *counters = (unsigned long long *)cv.take(4 * sizeof(unsigned long long));
    int32_t *node_k = (int32_t *)cv.take((size_t)(N + 1) * 4);
    int32_t *item_cnt = (int32_t *)cv.take((size_t)(N + 1) * 4);
    int64_t *slot_off = (int64_t *)cv.take((size_t)(N + 1) * 8);
    int64_t *item_off = (int64_t *)cv.take((size_t)(N + 1) * 8);
    int64_t *node_re = (int64_t *)cv.take((size_t)(N + 1) * 8);
    int64_t *pending = (int64_t *)cv.take((size_t)(N + 1) * 8);
    size_t scan_bytes = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const int32_t *)node_k, slot_off,
                                      (int)(N + 1), s) != cudaSuccess)
        return fail(VLL_ERR_CUDA, "scan size query failed");
    void *scan_tmp = cv.take(scan_bytes);
    if (!dP || !ctl || !counters || !node_k || !item_cnt || !slot_off || !item_off || !node_re ||
        !pending || !scan_tmp) {
        char m[160];
        snprintf(m, sizeof m, "grid of %lld nodes exceeds the %zu MiB scratch array",
                 (long long)N, kNoAllocScratchBytes >> 20);
        return fail(VLL_ERR_CAPACITY, m);
    }
#define NA_CUDA(call)                                                     \
    do {                                                                  \
        if ((call) != cudaSuccess) return fail(VLL_ERR_CUDA, #call);      \
    } while (0)
    NA_CUDA(cudaMemcpyAsync(dP, &P, sizeof(DevLevel), cudaMemcpyHostToDevice, s));
    // the array keeps the previous call's contents: clear what must start at zero
    NA_CUDA(cudaMemsetAsync(ctl, 0, 8 * sizeof(unsigned long long), s));
    NA_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), s));
    NA_CUDA(cudaMemsetAsync(node_k, 0, (size_t)(N + 1) * 4, s));
    NA_CUDA(cudaMemsetAsync(item_cnt, 0, (size_t)(N + 1) * 4, s));
    // capacity: count slots and items first, without writing any output
    noalloc_count_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(dP, node_k, item_cnt);
    NA_CUDA(cudaGetLastError());
    size_t t1 = scan_bytes;
    NA_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, t1, (const int32_t *)node_k, slot_off,
                                          (int)(N + 1), s));
    t1 = scan_bytes;
    NA_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, t1, (const int32_t *)item_cnt, item_off,
                                          (int)(N + 1), s));
    int64_t totals[2] = {0, 0};
    NA_CUDA(cudaMemcpyAsync(&totals[0], slot_off + N, 8, cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaMemcpyAsync(&totals[1], item_off + N, 8, cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
    const int64_t n_slots = totals[0], n_items = totals[1];
    const int64_t max_re = N * 4 + 1024;
    int64_t *items = (int64_t *)cv.take((size_t)(n_items > 0 ? n_items : 1) * 8);
    float2 *rho = (float2 *)cv.take((size_t)(n_slots > 0 ? n_slots : 1) * sizeof(float2));
    int64_t *re_items = (int64_t *)cv.take((size_t)max_re * 8);
    double *re_out = (double *)cv.take((size_t)max_re * 2 * sizeof(double));
    if (!items || !rho || !re_items || !re_out) {
        char m[200];
        snprintf(m, sizeof m,
                 "%lld nodes with %lld height slots exceed the %zu MiB scratch array",
                 (long long)N, (long long)n_slots, kNoAllocScratchBytes >> 20);
        return fail(VLL_ERR_CAPACITY, m);
    }
    // the pipeline proper (same kernels and order as run_split)
    NA_CUDA(cudaMemsetAsync(node_k, 0, (size_t)(N + 1) * 4, s));
    NA_CUDA(cudaMemsetAsync(item_cnt, 0, (size_t)(N + 1) * 4, s));
    prep_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(dP, nullptr, nullptr, node_k, item_cnt,
                                                          counters);
    NA_CUDA(cudaGetLastError());
    t1 = scan_bytes;
    NA_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, t1, (const int32_t *)node_k, slot_off,
                                          (int)(N + 1), s));
    t1 = scan_bytes;
    NA_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, t1, (const int32_t *)item_cnt, item_off,
                                          (int)(N + 1), s));
    if (n_items > 0) {
        items_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(N, item_cnt, item_off, items);
        NA_CUDA(cudaGetLastError());
        cudaError_t e = cudaSuccess;
        switch (P.H) {
            case 2: e = launch_ncc<2>(dP, items, n_items, slot_off, nullptr, nullptr, rho, counters, ctl, s); break;
            case 3: e = launch_ncc<3>(dP, items, n_items, slot_off, nullptr, nullptr, rho, counters, ctl, s); break;
            case 4: e = launch_ncc<4>(dP, items, n_items, slot_off, nullptr, nullptr, rho, counters, ctl, s); break;
            case 5: e = launch_ncc<5>(dP, items, n_items, slot_off, nullptr, nullptr, rho, counters, ctl, s); break;
            case 6: e = launch_ncc<6>(dP, items, n_items, slot_off, nullptr, nullptr, rho, counters, ctl, s); break;
            case 7: e = launch_ncc<7>(dP, items, n_items, slot_off, nullptr, nullptr, rho, counters, ctl, s); break;
            default: e = cudaErrorInvalidValue;
        }
        NA_CUDA(e);
        peaks_kernel<<<grid_1d(N, 128, 148 * 64), 128, 0, s>>>(dP, slot_off, rho, re_items, max_re,
                                                              node_re, pending, ctl, counters);
        NA_CUDA(cudaGetLastError());
        NA_CUDA(launch_recheck(dP, re_items, ctl + 1, max_re, nullptr, nullptr, re_out, s));
        rescan_kernel<<<148 * 8, 64, 0, s>>>(dP, slot_off, rho, node_re, pending, re_items, re_out,
                                             ctl);
        NA_CUDA(cudaGetLastError());
    }
    unsigned long long acc = 0;
    NA_CUDA(cudaMemcpyAsync(&acc, counters, sizeof(acc), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
#undef NA_CUDA
    if (accessable_grid) *accessable_grid = (int64_t)acc;
    return VLL_OK;
}

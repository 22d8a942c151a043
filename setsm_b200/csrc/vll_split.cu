// vll_split.cu -- split-precision VerticalLineLocus (setsm_code.cpp:6049-6548
// with FindPeakNcc, :6672-6752).
//
// Pipeline for one level, all on one stream:
//   gncc    FP64 GNCC per node (height independent), when the level uses it
//   prep    per node: image-boundary and blunder tests, the nccresult fields
//           VerticalLineLocus sets before its height loop, slot count K
//   scan    exclusive prefix sums -> slot offsets and (node, 32-slot) items
//   window  persistent kernel draining the item queue: one warp per item,
//           one lane per height slot.  The RPC numerators / denominators are
//           cubics in the normalised height per node (FP64, Horner), with the
//           reference-order RPC wherever a coordinate lies within 1e-7 px of
//           an integer or a clamp, so every integer decision (orientation
//           pixel, image bounds) equals the reference's.  The warp's window
//           footprints in both images are staged in shared memory as FP32
//           texel pairs; bilinear sampling and window sums in FP32, each sum
//           centred on its window's centre sample -> per-slot rho (float2:
//           rho, INCC average or NaN when FP32 cannot decide a variance test).
//   peaks   one warp per node: the FindPeakNcc scan, warp-parallel (a slot's
//           direction and whether its predecessor is a peak depend only on
//           neighbouring evaluated values); every decision whose FP32 inputs
//           lie within kBand of a boundary (direction ties, sign tests,
//           rounding of a top-two peak or of the maximum, truncation of a
//           voxel) marks the slots involved, which the warp re-evaluates in
//           exact FP64 (the reference's operation order) before repeating the
//           scan; then the ordered top-two fold and the nccresult write.
// The outputs are identical to the FP64 kernel's.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>
#include <cub/device/device_scan.cuh>
#include <cuda.h>

#include "vll_exact.cuh"
#include "vll_internal.h"
#include "vll_split.h"
#include "vll_window.cuh"

namespace vll {

// Exclusive prefix sum of per-node int32 counts into int64 offsets, with an
// int64 accumulator: the totals of a large level set exceed 2^31 (a 4096^2
// grid already carries ~2 G height slots), and cub's ExclusiveSum would
// accumulate in the input's 32-bit type.
inline cudaError_t scan64(void *tmp, size_t &bytes, const int32_t *in, int64_t *out, int n,
                          cudaStream_t s) {
    return cub::DeviceScan::ExclusiveScan(tmp, bytes, in, out, cub::Sum(), (int64_t)0, n, s);
}


// Half-width of the FP32 error band of rho: decisions whose FP32 inputs lie
// closer than this to their boundary are settled in FP64.  The FP32-vs-FP64
// error of rho measured over 4.2 M slots of 7x7 and 11x11 windows stays below
// 6.8e-7 (tests/test_gpu_accuracy.py asserts < kBand / 2), a margin of ~3x.
constexpr float kBand = 4e-6f;
constexpr double kEdge = 1e-7;          // coordinate distance to an integer / clamp
constexpr int kSlotCap = 512;           // slots per node the peak kernel holds in shared memory
constexpr int kWarpPerSlotMax = 8;      // re-checks per round done a warp per slot (more: a lane each)
constexpr int kMaxRounds = 3;           // scan / re-check rounds before a full FP64 pass

// Per-slot markers in the rho buffer (.x):
constexpr float kNotEvaluated = INFINITY;    // slot skipped (range / image bounds)
constexpr float kRejected = -INFINITY;       // orientation check failed

// ---------------------------------------------------------------------------
// Level set: the levels matched by one pass of the pipeline (one level for a
// VerticalLineLocus call; many tiles and pyramid levels for a batch).  Their
// nodes are numbered consecutively: global node g belongs to the level l with
// base[l] <= g < base[l + 1] and is that level's node g - base[l].  Per-node
// and per-slot work arrays are indexed by g.
// ---------------------------------------------------------------------------
struct LevelSet {
    const DevLevel *lv;       // [n] level blocks (device)
    const int64_t *base;      // [n + 1] first global node of each level (device)
    int n;
    int64_t total;            // base[n]
};

__device__ __forceinline__ int level_of(const LevelSet &S, int64_t g) {
    int lo = 0, hi = S.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(S.base + mid) <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// prep: per-node setup (setsm_code.cpp:6158-6328)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) prep_kernel(const LevelSet S,
                                                   const double *__restrict__ gsum,
                                                   const double *__restrict__ gcnt,
                                                   int32_t *__restrict__ node_k,
                                                   unsigned long long *__restrict__ counters,
                                                   unsigned long long *__restrict__ acc_level) {
    unsigned long long acc = 0, acc_l = 0;
    int cur = -1;
    for (int64_t gn = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gn < S.total;
         gn += (int64_t)gridDim.x * blockDim.x) {
        const int l = level_of(S, gn);
        if (l != cur) {
            if (acc_l) atomicAdd(&acc_level[cur], acc_l);
            acc_l = 0;
            cur = l;
        }
        const DevLevel &P = S.lv[l];
        const int64_t pt = gn - __ldg(S.base + l);
        int K = 0;
        const vll_ugrid g = P.gp3[pt];
        const int start_H = g.minHeight, end_H = g.maxHeight;
        const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
        if (check_image_boundary(P, lon, lat, (double)start_H, (double)end_H, P.H) &&
            !blunder_cell(P, g)) {
            acc++;
            acc_l++;
            vll_nccresult &R = P.ncc[pt];
            const int ti = 1;
            if (P.check_ortho && dq_result(ugrid_ortho_ncc(P.gp3, P.n_nodes, pt, ti)) > P.ortho_th)
                R.GNCC = gcnt[gn] > 0 ? q_result(__ddiv_rn(gsum[gn], gcnt[gn])) : q_result(-1.0);
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
        node_k[gn] = K;
    }
    if (acc_l) atomicAdd(&acc_level[cur], acc_l);
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&counters[0], acc);
}

// ---------------------------------------------------------------------------
// geometry helpers of the window kernel
// ---------------------------------------------------------------------------
// Per-node RPC: normalised L, P (with the reference's +-360 wrap) and the
// four cubics in the normalised height.  RPC00B terms grouped by power of H:
//   a0: 1 L P LP LL PP LLL LPP LLP PPP   a1: H LH PH PLH LLH PPH
//   a2: HH LHH PHH                        a3: HHH
// Coefficients a0..a3 of one of the four RPC cubics (j: LINE_NUM, LINE_DEN,
// SAMP_NUM, SAMP_DEN) as a polynomial in the normalised height, for fixed
// normalised L, P (with the reference's +-360 wrap).
__device__ __forceinline__ void node_horner_poly(const double *rpc, double lon, double lat, int j,
                                                 double *a) {
    double L = (lon - rpc[2]) / rpc[7];
    double P = (lat - rpc[3]) / rpc[8];
    if (L < -10.0 || L > 10.0) {
        const double X = lon > 0 ? lon - 360 : lon + 360;
        L = (X - rpc[2]) / rpc[7];
    }
    if (P < -10.0 || P > 10.0) {
        const double Y = lat > 0 ? lat - 360 : lat + 360;
        P = (Y - rpc[3]) / rpc[8];
    }
    const double *c = rpc + 10 + 20 * j;
    a[0] = c[0] + c[1] * L + c[2] * P + c[4] * L * P + c[7] * L * L + c[8] * P * P +
           c[11] * L * L * L + c[12] * L * P * P + c[14] * L * L * P + c[15] * P * P * P;
    a[1] = c[3] + c[5] * L + c[6] * P + c[10] * P * L + c[17] * L * L + c[18] * P * P;
    a[2] = c[9] + c[13] * L + c[16] * P;
    a[3] = c[19];
}

// Reciprocal for the fast geometry path: FP32 seed refined by two Newton
// steps (relative error ~1e-16).  A seed that is not a finite non-zero float
// sends the slot to the exact projection.
__device__ __forceinline__ double fast_rcp(double v, bool &edge) {
    const float f = __frcp_rn((float)v);
    if (!(fabsf(f) > 0.f && fabsf(f) < 3.0e38f)) edge = true;
    double r = (double)f;
    r = fma(r, fma(-v, r, 1.0), r);
    r = fma(r, fma(-v, r, 1.0), r);
    return r;
}

// Image coordinate (pyramid level) of one slot from the per-node cubics.
// Sets `edge` when a coordinate is too close to an integer, or to a clamp,
// for the Horner rounding to be trusted with the reference's integer tests.
__device__ __forceinline__ double2 fast_coord(const double (*a)[4], const double *hn,
                                              const DevImage &im, double hgt, double inv_s,
                                              bool &edge) {
    const double H = (hgt - hn[0]) * hn[1];   // hn[1]: reciprocal of the height scale
    double v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = fma(fma(fma(a[j][3], H, a[j][2]), H, a[j][1]), H, a[j][0]);
    double y = im.adj[0] + ((v[0] * fast_rcp(v[1], edge)) * im.rpc[5] + im.rpc[0]);
    double x = im.adj[1] + ((v[2] * fast_rcp(v[3], edge)) * im.rpc[6] + im.rpc[1]);
    const double ymax = im.rpc[0] + im.rpc[5] * 1.2, xmax = im.rpc[1] + im.rpc[6] * 1.2;
    if (fabs(y) < kEdge || fabs(y - ymax) < kEdge || fabs(x) < kEdge || fabs(x - xmax) < kEdge)
        edge = true;
    y = y < 0 ? 0 : (y > ymax ? ymax : y);
    x = x < 0 ? 0 : (x > xmax ? xmax : x);
    const double px = x * inv_s - im.sx, py = y * inv_s - im.sy;   // inv_s = 2^-L (exact)
    const double fx = px - floor(px), fy = py - floor(py);
    if (fx < kEdge || fx > 1.0 - kEdge || fy < kEdge || fy > 1.0 - kEdge) edge = true;
    return make_double2(px, py);
}

__device__ __forceinline__ bool near_round(double v) {
    const double x = v * 1000.0;
    return fabs(x - floor(x) - 0.5) < (double)kBand * 1000.0;
}
__device__ __forceinline__ bool near_trunc(double v) {
    const double x = v * 1000.0;
    return fabs(x - rint(x)) < (double)kBand * 1000.0;
}



// ---------------------------------------------------------------------------
// FindPeakNcc decisions over the slots of one node, lane-parallel (shared by
// the window kernel's FP32 pass and the exact pass)
// ---------------------------------------------------------------------------
// FindPeakNcc's sign rule for the direction from b to a (setsm_code.cpp:6676-6692)
__device__ __forceinline__ int dir_sign(double a, double b) {
    double d;
    if (a >= 0 && b >= 0)
        d = a - b;
    else if (a < 0 && b < 0)
        d = -(fabs(a) - fabs(b));
    else if (a >= 0 && b < 0)
        d = 1;
    else
        d = -1;
    return d > 0 ? 1 : (d < 0 ? -1 : 0);
}

__device__ __forceinline__ bool bit(const uint32_t *m, int k) { return (m[k >> 5] >> (k & 31)) & 1u; }
__device__ __forceinline__ void set_bit(uint32_t *m, int k) { atomicOr(&m[k >> 5], 1u << (k & 31)); }

// Index of the last evaluated slot before k (or -1); `carry` is the last
// evaluated slot of earlier 32-slot groups.
__device__ __forceinline__ int prev_eval(uint32_t mask, int lane, int carry) {
    const uint32_t below = mask & ((1u << lane) - 1u);
    return below ? (31 - __clz(below)) : carry;
}

// Bit masks over the slots of one node (kSlotCap at most), in shared memory.
struct SlotMasks {
    uint32_t evaluated[kSlotCap / 32];   // slot evaluated (not skipped / rejected)
    uint32_t need[kSlotCap / 32];        // slot needs an exact FP64 value
    uint32_t peak[kSlotCap / 32];        // slot is a FindPeakNcc peak
};

// One pass of FindPeakNcc's decisions over a node's K slot values, every lane
// taking one slot of each 32-slot group:
//  (a) the direction of each slot and whether its predecessor is a peak (a
//      slot's direction depends only on it and the previous evaluated
//      slot); near ties, and values near zero, mark both slots `need`;
//  (a2) peaks whose rounding to rho*1000 could enter or reorder the top two
//      (a peak more than 0.002 + 2 bands below the second best rounds
//      strictly below it) and round ambiguously;
//  (b) the maximum (max_WNCC), and slots near it that round ambiguously.
// `val(k, ex)` gives slot k's value and whether it is exact (exact values
// never need re-evaluation).  Returns the maximum.
template <class Val>
__device__ double scan_pass(const DevLevel &P, bool check_height_change, int K, SlotMasks &M,
                            Val val, int lane) {
    int carry = -1;
    for (int k0 = 0; k0 < K; k0 += 32) {
        const int k = k0 + lane;
        const uint32_t em = M.evaluated[k0 >> 5];
        const bool ev = k < K && ((em >> lane) & 1u);
        const int p_in = prev_eval(em, lane, -1);
        const int p = p_in >= 0 ? k0 + p_in : carry;
        bool need_me = false, need_p = false;
        if (ev && P.cmr && p >= 0) {
            int pp = -1;
            const int pg = p >> 5, pl = p & 31;
            const uint32_t pm = M.evaluated[pg] & ((1u << pl) - 1u);
            if (pm) {
                pp = (pg << 5) + 31 - __clz(pm);
            } else {
                for (int gi = pg - 1; gi >= 0 && pp < 0; --gi)
                    if (M.evaluated[gi]) pp = (gi << 5) + 31 - __clz(M.evaluated[gi]);
            }
            bool ex_k, ex_p;
            const double v = val(k, ex_k);
            const double pv = val(p, ex_p);
            if (!(ex_k && ex_p) && (fabs(v - pv) < kBand || fabs(v) < kBand || fabs(pv) < kBand)) {
                need_me = !ex_k;
                need_p = !ex_p;
            }
            // direction of k (td) and of p (dp): a peak at p needs dp > 0 and
            // td < 0 (the first evaluated slot's direction is -1)
            const int td = dir_sign(v, pv);
            int dp = -1;
            if (pp >= 0) {
                bool ex_pp;
                dp = dir_sign(pv, val(pp, ex_pp));
            }
            if (pv != -1 && dp > 0 && td < 0) set_bit(M.peak, p);
        }
        if (need_me) set_bit(M.need, k);
        if (need_p) set_bit(M.need, p);
        const uint32_t any = em & ((k0 + 32 <= K) ? 0xffffffffu : ((1u << (K - k0)) - 1u));
        if (any) carry = k0 + 31 - __clz(any);
    }
    __syncwarp();
    if (P.cmr) {
        double b1 = -1e30, b2 = -1e30;
        for (int k = lane; k < K; k += 32) {
            if (!bit(M.peak, k)) continue;
            bool ex;
            const double v = val(k, ex);
            if (v > b1) {
                b2 = b1;
                b1 = v;
            } else if (v > b2) {
                b2 = v;
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double o1 = __shfl_xor_sync(0xffffffffu, b1, o);
            const double o2 = __shfl_xor_sync(0xffffffffu, b2, o);
            const double n1 = fmax(b1, o1);
            const double n2 = fmax(fmin(b1, o1), fmax(b2, o2));
            b1 = n1;
            b2 = n2;
        }
        const double thr = (b2 > -1e29 ? b2 : b1) - 0.002 - 2.0 * (double)kBand;
        for (int k = lane; k < K; k += 32) {
            if (!bit(M.peak, k)) continue;
            bool ex;
            const double v = val(k, ex);
            if (!ex && v >= thr && near_round(v)) set_bit(M.need, k);
        }
    }
    __syncwarp();
    double m = -100;
    for (int k = lane; k < K; k += 32) {
        if (!bit(M.evaluated, k)) continue;
        bool ex;
        const double v = val(k, ex);
        if (m < v) m = v;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (check_height_change) {
        for (int k = lane; k < K; k += 32) {
            if (!bit(M.evaluated, k)) continue;
            bool ex;
            const double v = val(k, ex);
            if (!ex && v >= m - kBand && near_round(v)) set_bit(M.need, k);
        }
    }
    __syncwarp();
    return m;
}

// FindPeakNcc's ordered top-two fold over the marked peaks (one lane).
template <class Val>
__device__ void fold_peaks(const DevLevel &P, vll_nccresult &R, int K, int start_H,
                           const uint32_t *peak, Val val) {
    for (int i = 0; i < (K + 31) / 32; ++i) {
        uint32_t pm = peak[i];
        while (pm) {
            const int b = __ffs(pm) - 1;
            pm &= pm - 1;
            const int p = (i << 5) + b;
            bool ex;
            const double pv = val(p, ex);
            const float ph = slot_height(P, start_H, R.minHeight, p);
            if (R.result4 < 10) R.result4 += 1;
            const int16_t qpre = q_result(pv);
            if (R.result0 < qpre) {
                const double t1 = dq_result(R.result0);
                R.result0 = qpre;
                const float t2 = R.result2;
                R.result2 = ph;
                const int16_t q1 = q_result(t1);
                if (R.result1 < q1) {
                    R.result1 = q1;
                    R.result3 = t2;
                }
            } else if (R.result1 < qpre) {
                R.result1 = qpre;
                R.result3 = ph;
            }
        }
    }
}

// A node settled entirely in exact FP64 (eval_slot: the reference's
// operation order), the warp's lanes evaluating 32 slots at a time; lane 0
// folds each chunk into FindPeakNcc and the maximum in slot order, so no
// per-slot buffer is needed.  Voxel rows get the exact flags and INCC.
// `first` = this is the node's first evaluation (counted as evaluations and
// written to the debug slot values), otherwise a re-evaluation.
__device__ void node_exact_chunked(const DevLevel &P, int64_t pt, int K, const PatchSrc &S,
                                   const PatchSrc &Sn, double cnt_g, double sum_g,
                                   vll_nccresult R, vll_voxel *vrow, double *chunk, int lane,
                                   bool first, unsigned long long &count) {
    const vll_ugrid g = P.gp3[pt];
    const int start_H = g.minHeight, end_H = g.maxHeight;
    PeakState st;
    peak_init(st);
    double max_w = -100;
    for (int k0 = 0; k0 < K; k0 += 32) {
        const int k = k0 + lane;
        double out = (double)kNotEvaluated;
        if (k < K) {
            const float hgt = slot_height(P, start_H, R.minHeight, k);
            if (hgt >= (float)start_H && hgt <= (float)end_H) {
                const SlotOut o = eval_slot(P, pt, 1, S, Sn, hgt, cnt_g, sum_g);
                if (o.evaluated) {
                    out = o.rho;
                    if (vrow) {
                        if (o.all_pos) vrow[k].flag_cal = 1;
                        vrow[k].INCC = o.count_incc > 0
                                           ? q_voxel(__ddiv_rn(o.sum_incc, o.count_incc))
                                           : q_voxel(-1.0);
                    }
                    // debug values: every slot on a first evaluation, else only
                    // slots that have no FP32 value (NaN)
                    if (P.dbg_rho && (first || isnan(P.dbg_rho[P.dbg_off[pt] + k])))
                        P.dbg_rho[P.dbg_off[pt] + k] = o.rho;
                    count++;
                } else if (o.orient_reject) {
                    out = (double)kRejected;
                    if (vrow) vrow[k].flag_cal = 0;
                }
            }
        }
        chunk[lane] = out;
        __syncwarp();
        if (lane == 0) {
            const int n = min(32, K - k0);
            for (int i = 0; i < n; ++i) {
                const double v = chunk[i];
                if (isinf(v)) continue;
                if (P.cmr) find_peak(st, v, slot_height(P, start_H, R.minHeight, k0 + i), R);
                if (max_w < v) max_w = v;
            }
        }
        __syncwarp();
    }
    if (lane == 0) {
        if (R.check_height_change) R.max_WNCC = q_result(max_w);
        P.ncc[pt] = R;
    }
    __syncwarp();
}


// ---------------------------------------------------------------------------
// window kernel
// ---------------------------------------------------------------------------
// Warps per window block and the minimum resident blocks per SM (the latter
// sets the register budget: 65536 / (warps * 32 * blocks)).
#ifndef VLL_WIN_WARPS
#define VLL_WIN_WARPS 4
#endif
#ifndef VLL_WIN_MINB
#define VLL_WIN_MINB 3
#endif
constexpr int kWinWarps = VLL_WIN_WARPS;
constexpr int kWinMaxBlocksPerSm = 2048 / (kWinWarps * 32);
constexpr int kZeroCap = 32;          // zero intensity texels listed per staged group

// Node flags of the window kernel
constexpr uint32_t kNfCmr = 1u;       // memory-tight route (FindPeakNcc on the values)
constexpr uint32_t kNfOri = 2u;       // orientation-difference test (level >= 3)
constexpr uint32_t kNfVox = 4u;       // voxel rows written
constexpr uint32_t kNfChc = 8u;       // check_height_change (max_WNCC written)
constexpr uint32_t kNfGncc = 16u;     // rho blends the INCC with the node's GNCC
constexpr uint32_t kNfVec = 32u;      // image rows 16-byte aligned (vector staging)
constexpr uint32_t kNfTma = 64u;      // the level has tensor maps for its footprints
constexpr uint32_t kNfDbg = 128u;     // per-slot debug values written

// Optional instrumentation of the window kernel's phases (compiled with
// -DVLL_PHASE_CYCLES: `python -m setsm_b200.build --phase-cycles` builds
// lib/libsetsm_vll_phases.so).  Each warp sums clock64 deltas per phase
// (0 tile wait, 1 box conversion, 2 node set-up, 3 geometry and tile copies,
// 4 window statistics, 5 FindPeakNcc scan and writes, 6 node end) and counts
// groups and nodes; vll_window_phase_cycles reads the totals.  The kernel's
// work is the same with and without it.
#ifdef VLL_PHASE_CYCLES
__device__ unsigned long long g_phase_cycles[16];
#define PHASE_DECL                                 \
    unsigned long long ph_[8] = {}, ph_n_[2] = {}; \
    long long ph_t_ = clock64()
#define PHASE(i)                                             \
    do {                                                     \
        const long long t_ = clock64();                      \
        ph_[i] += (unsigned long long)(t_ - ph_t_);          \
        ph_t_ = t_;                                          \
    } while (0)
#define PHASE_COUNT(i) (++ph_n_[i])
#define PHASE_FLUSH()                                                      \
    do {                                                                   \
        if (lane == 0) {                                                   \
            for (int i_ = 0; i_ < 8; ++i_) atomicAdd(&g_phase_cycles[i_], ph_[i_]); \
            atomicAdd(&g_phase_cycles[8], ph_n_[0]);                       \
            atomicAdd(&g_phase_cycles[9], ph_n_[1]);                       \
        }                                                                  \
    } while (0)
#else
#define PHASE_DECL (void)0
#define PHASE(i) (void)0
#define PHASE_COUNT(i) (void)0
#define PHASE_FLUSH() (void)0
#endif

// Per-node state of the window kernel in shared memory: the RPC cubics, the
// level constants the slot loop reads (here rather than from the level block
// in global memory), the record folded by lane 0 and the streamed scan's
// carry.  A warp holds two: the node of the group being evaluated and the
// node of the group being fetched.
struct NodeCtx {
    double horner[2][4][4];           // [image][num/den poly][a0..a3]
    double hnorm[2][2];               // [image] {h_off, 1 / h_scale}
    double geo[2][8];                 // [image] adj0, adj1, rpc0, rpc1, rpc5, rpc6, sx, sy
    double inv_s, hbase, hstep, bin_angle, alpha, gterm;
    const uint16_t *img[2], *mag[2];
    const uint8_t *ori[2];
    const DevLevel *P;
    vll_voxel *vrow;
    int64_t gn, pt;
    uint32_t w[2], h[2];
    int tma_w[2], tma_h[2];
    int K, H, start_H, end_H;
    uint32_t flags;
    vll_nccresult R;
    float pre_v;                      // streamed scan: the last evaluated slot's value,
    int pre_dir, pre_k, have;         // direction and index, and whether there is one
};

// The constants of the launch's first level, loaded once per block: node
// set-ups on that level (every node of a single-level call) read them from
// shared memory and fetch only the node's own records from global memory.
struct LevelConst {
    double rpc[2][90];                // [image] RPC00B block (offsets, scales, 4 x 20 terms)
    double geo[2][8];                 // as NodeCtx::geo
    double inv_s, hstep, bin_angle, alpha, beta;
    const uint16_t *img[2], *mag[2];
    const uint8_t *ori[2];
    uint32_t w[2], h[2];
    int tma_w[2], tma_h[2];
    int H, is_ra, cmr, check_ortho, voxels;
    uint32_t flags;                   // kNfOri | kNfVec | kNfTma | kNfDbg
};

// Per-warp shared state of the window kernel.
struct WinShared {
    NodeCtx node[2];
    uint32_t zl[kZeroCap];            // zero intensity texels of the staged boxes
    int zn;                           // their count (more than kZeroCap: not listed)
    uint64_t mbar;                    // completion of the group's tile copies
    const DevLevel *tmap_level;       // level whose tensor maps lane 0 has acquired
};

__host__ __device__ constexpr size_t win_level_offset() {
    return (sizeof(WinShared) * kWinWarps + 15) & ~(size_t)15;
}

__host__ __device__ constexpr size_t win_boxes_offset() {
    return (win_level_offset() + sizeof(LevelConst) + 15) & ~(size_t)15;
}

// Fills the block's LevelConst from level P (every thread of the block takes
// part; the caller synchronises the block afterwards).
__device__ void level_const_load(LevelConst &C, const DevLevel &P) {
    const int t = threadIdx.x, nt = blockDim.x;
    for (int i = t; i < 180; i += nt) {
        const int im = i / 90;
        C.rpc[im][i - im * 90] = P.im[im == 0 ? P.ref : 1].rpc[i - im * 90];
    }
    if (t < 2) {
        const DevImage &I = P.im[t == 0 ? P.ref : 1];
        double *g = C.geo[t];
        g[0] = I.adj[0];
        g[1] = I.adj[1];
        g[2] = I.rpc[0];
        g[3] = I.rpc[1];
        g[4] = I.rpc[5];
        g[5] = I.rpc[6];
        g[6] = I.sx;
        g[7] = I.sy;
        C.img[t] = I.img;
        C.mag[t] = I.mag;
        C.ori[t] = I.ori;
        C.w[t] = I.w;
        C.h[t] = I.h;
        C.tma_w[t] = P.tma_w[t];
        C.tma_h[t] = P.tma_h[t];
    } else if (t == 2) {
        const DevImage &ri = P.im[P.ref], &tI = P.im[1];
        C.inv_s = 1.0 / (double)(1 << P.L);
        C.hstep = P.height_step;
        C.bin_angle = P.bin_angle;
        C.alpha = P.alpha;
        C.beta = P.beta;
        C.H = P.H;
        C.is_ra = P.is_ra;
        C.cmr = P.cmr;
        C.check_ortho = P.check_ortho;
        C.voxels = P.vox && !P.cmr && !P.is_ra;
        const bool vec_ok = (ri.w % 8 == 0) && (tI.w % 8 == 0) &&
                            ((reinterpret_cast<uintptr_t>(ri.img) | reinterpret_cast<uintptr_t>(ri.mag) |
                              reinterpret_cast<uintptr_t>(tI.img) |
                              reinterpret_cast<uintptr_t>(tI.mag)) & 15) == 0;
        C.flags = ((!P.is_ra && P.L >= 3) ? kNfOri : 0u) | (vec_ok ? kNfVec : 0u) |
                  (P.tma_w[0] > 0 ? kNfTma : 0u) | (P.dbg_rho ? kNfDbg : 0u);
    }
}

// the TMA tiles follow the boxes, 128-byte aligned (warp_raw is a multiple of 128)
__host__ __device__ constexpr size_t win_raw_offset(int warp_quads) {
    return (win_boxes_offset() + (size_t)kWinWarps * warp_quads * 16 + 127) & ~(size_t)127;
}

// FP32 window statistics of one slot for the level's window half-size
// (the window code is unrolled per half-size; a batch may mix them).
__device__ __forceinline__ void window_any(int H, const float4 *qr, int rbw, float rfx, float rfy,
                                           const TgtBox &tb, float tfx, float tfy, float c,
                                           float s, float &incc, bool &unsure) {
    switch (H) {
        case 2: window_fp32<2>(qr, rbw, rfx, rfy, tb, tfx, tfy, c, s, incc, unsure); break;
        case 3: window_fp32<3>(qr, rbw, rfx, rfy, tb, tfx, tfy, c, s, incc, unsure); break;
        case 4: window_fp32<4>(qr, rbw, rfx, rfy, tb, tfx, tfy, c, s, incc, unsure); break;
        case 5: window_fp32<5>(qr, rbw, rfx, rfy, tb, tfx, tfy, c, s, incc, unsure); break;
        case 6: window_fp32<6>(qr, rbw, rfx, rfy, tb, tfx, tfy, c, s, incc, unsure); break;
        default: window_fp32<7>(qr, rbw, rfx, rfy, tb, tfx, tfy, c, s, incc, unsure); break;
    }
}

// Fills the warp's node context for global node gn (level lvl, K slots);
// every lane takes part, the context is complete after the final __syncwarp.
__device__ __noinline__ void node_setup(NodeCtx &N, const LevelSet &LS, int lvl, int64_t gn, int K,
                                        const double *__restrict__ gsum,
                                        const double *__restrict__ gcnt,
                                        const LevelConst *lc, int lane) {
    const DevLevel &P = LS.lv[lvl];
    const int64_t pt = gn - __ldg(LS.base + lvl);
    if (lc) {
        // the level's constants from the block's copy; the node's own
        // records from global memory, one load per lane
        if (lane < 8) {
            const int im = lane >> 2, j = lane & 3;
            const double *rpc = lc->rpc[im];
            node_horner_poly(rpc, P.grid_wgs[2 * pt], P.grid_wgs[2 * pt + 1], j, N.horner[im][j]);
            if (j == 0) {
                N.hnorm[im][0] = rpc[4];
                N.hnorm[im][1] = 1.0 / rpc[9];
            }
        } else if (lane < 26) {
            const int i = lane - 8;   // 16 geo values, then 2 lanes of pointers
            if (i < 16) {
                N.geo[i >> 3][i & 7] = lc->geo[i >> 3][i & 7];
            } else {
                const int im = i - 16;
                N.img[im] = lc->img[im];
                N.mag[im] = lc->mag[im];
                N.ori[im] = lc->ori[im];
                N.w[im] = lc->w[im];
                N.h[im] = lc->h[im];
                N.tma_w[im] = lc->tma_w[im];
                N.tma_h[im] = lc->tma_h[im];
            }
        } else if (lane == 26) {
            const vll_ugrid g = P.gp3[pt];
            const vll_nccresult R = P.ncc[pt];
            const double cnt_g = gcnt ? gcnt[gn] : 0.0;
            const double sum_g = gcnt ? gsum[gn] : 0.0;
            N.P = &P;
            N.gn = gn;
            N.pt = pt;
            N.K = K;
            N.H = lc->H;
            N.start_H = g.minHeight;
            N.end_H = g.maxHeight;
            N.R = R;
            N.hbase = (double)((lc->is_ra || lc->cmr) ? g.minHeight : R.minHeight);
            N.hstep = lc->hstep;
            N.inv_s = lc->inv_s;
            N.bin_angle = lc->bin_angle;
            N.alpha = lc->alpha;
            const bool gncc = lc->check_ortho && cnt_g > 0;
            N.gterm = gncc ? (sum_g / cnt_g) * lc->beta : 0.0;
            N.vrow = lc->voxels ? P.vox + P.vox_off[pt] : nullptr;
            N.flags = lc->flags | (lc->cmr ? kNfCmr : 0u) | (lc->voxels ? kNfVox : 0u) |
                      (R.check_height_change ? kNfChc : 0u) | (gncc ? kNfGncc : 0u);
            N.pre_v = -1.0f;
            N.pre_dir = 0;
            N.pre_k = -1;
            N.have = 0;
        }
        __syncwarp();
        return;
    }
    if (lane < 8) {
        // per-node RPC cubics: lanes 0..7 = (image, polynomial)
        const int im = lane >> 2, j = lane & 3;
        const double *rpc = P.im[im == 0 ? P.ref : 1].rpc;
        node_horner_poly(rpc, P.grid_wgs[2 * pt], P.grid_wgs[2 * pt + 1], j, N.horner[im][j]);
        if (j == 0) {
            N.hnorm[im][0] = rpc[4];
            N.hnorm[im][1] = 1.0 / rpc[9];
        }
    } else if (lane < 10) {
        const int im = lane - 8;
        const DevImage &I = P.im[im == 0 ? P.ref : 1];
        double *g = N.geo[im];
        g[0] = I.adj[0];
        g[1] = I.adj[1];
        g[2] = I.rpc[0];
        g[3] = I.rpc[1];
        g[4] = I.rpc[5];
        g[5] = I.rpc[6];
        g[6] = I.sx;
        g[7] = I.sy;
        N.img[im] = I.img;
        N.mag[im] = I.mag;
        N.ori[im] = I.ori;
        N.w[im] = I.w;
        N.h[im] = I.h;
        N.tma_w[im] = P.tma_w[im];
        N.tma_h[im] = P.tma_h[im];
    } else if (lane == 10) {
        const vll_ugrid g = P.gp3[pt];
        const vll_nccresult R = P.ncc[pt];
        const DevImage &ri = P.im[P.ref], &tI = P.im[1];
        N.P = &P;
        N.gn = gn;
        N.pt = pt;
        N.K = K;
        N.H = P.H;
        N.start_H = g.minHeight;
        N.end_H = g.maxHeight;
        N.R = R;
        N.hbase = (double)((P.is_ra || P.cmr) ? g.minHeight : R.minHeight);
        N.hstep = P.height_step;
        N.inv_s = 1.0 / (double)(1 << P.L);
        N.bin_angle = P.bin_angle;
        N.alpha = P.alpha;
        const double cnt_g = gcnt ? gcnt[gn] : 0.0;
        const bool gncc = P.check_ortho && cnt_g > 0;
        N.gterm = gncc ? (gsum[gn] / cnt_g) * P.beta : 0.0;
        const bool voxels = P.vox && !P.cmr && !P.is_ra;
        N.vrow = voxels ? P.vox + P.vox_off[pt] : nullptr;
        const bool vec_ok = (ri.w % 8 == 0) && (tI.w % 8 == 0) &&
                            ((reinterpret_cast<uintptr_t>(ri.img) | reinterpret_cast<uintptr_t>(ri.mag) |
                              reinterpret_cast<uintptr_t>(tI.img) |
                              reinterpret_cast<uintptr_t>(tI.mag)) & 15) == 0;
        N.flags = (P.cmr ? kNfCmr : 0u) | ((!P.is_ra && P.L >= 3) ? kNfOri : 0u) |
                  (voxels ? kNfVox : 0u) | (R.check_height_change ? kNfChc : 0u) |
                  (gncc ? kNfGncc : 0u) | (vec_ok ? kNfVec : 0u) | (P.tma_w[0] > 0 ? kNfTma : 0u) |
                  (P.dbg_rho ? kNfDbg : 0u);
        N.pre_v = -1.0f;
        N.pre_dir = 0;
        N.pre_k = -1;
        N.have = 0;
    }
    __syncwarp();
}

// Image coordinate (pyramid level) of one slot of node N in image im from
// the node's cubics (fast_coord's arithmetic on the node context).
__device__ __forceinline__ double2 node_coord(const NodeCtx &N, int im, double hgt, bool &edge) {
    const double H = (hgt - N.hnorm[im][0]) * N.hnorm[im][1];
    double v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double *a = N.horner[im][j];
        v[j] = fma(fma(fma(a[3], H, a[2]), H, a[1]), H, a[0]);
    }
    const double *g = N.geo[im];
    double y = g[0] + ((v[0] * fast_rcp(v[1], edge)) * g[4] + g[2]);
    double x = g[1] + ((v[2] * fast_rcp(v[3], edge)) * g[5] + g[3]);
    const double ymax = g[2] + g[4] * 1.2, xmax = g[3] + g[5] * 1.2;
    if (fabs(y) < kEdge || fabs(y - ymax) < kEdge || fabs(x) < kEdge || fabs(x - xmax) < kEdge)
        edge = true;
    y = y < 0 ? 0 : (y > ymax ? ymax : y);
    x = x < 0 ? 0 : (x > xmax ? xmax : x);
    const double px = x * N.inv_s - g[6], py = y * N.inv_s - g[7];   // inv_s = 2^-L (exact)
    const double fx = px - floor(px), fy = py - floor(py);
    if (fx < kEdge || fx > 1.0 - kEdge || fy < kEdge || fy > 1.0 - kEdge) edge = true;
    return make_double2(px, py);
}

// Both images' coordinates of a slot by the reference's own RPC order (the
// slots whose fast coordinates lie too close to an integer or a clamp).
__device__ __noinline__ void slot_coords_exact(const NodeCtx &N, double hgt, double2 &rp,
                                               double2 &tp) {
    const DevLevel &P = *N.P;
    const double lon = P.grid_wgs[2 * N.pt], lat = P.grid_wgs[2 * N.pt + 1];
#pragma unroll 1
    for (int im = 0; im < 2; ++im) {
        const DevImage &I = P.im[im == 0 ? P.ref : 1];
        const double2 q = to_pyramid(rpc_project(I.rpc, I.adj, lon, lat, hgt), I.sx, I.sy, P.L);
        if (im == 0)
            rp = q;
        else
            tp = q;
    }
}

// One persistent launch over the nodes of every level of the set, a warp per
// node, nodes taken from a global queue in level order; each node's slots in
// groups of 32 (a lane per slot).  The groups form one stream per warp that
// is software-pipelined: while the window statistics of a group are
// computed, the footprints of the next group (of this node or the next one)
// are already being copied into shared memory by the TMA engine.  Per group:
//   fetch     FP64 geometry of the 32 slots (RPC cubics of the node, the
//             reference's RPC order near integers and clamps), the loads of
//             the orientation bytes, the boxes covering the footprints, four
//             tile copies;
//   stage     (a group later) conversion of the tiles to FP32 box texels,
//             two per lane step, listing zero intensity texels;
//   evaluate  the orientation test and rotation from the bytes loaded a
//             group earlier, FP32 window statistics of every slot whose
//             footprint holds no zero texel, then FindPeakNcc / max_WNCC
//             streamed over the group (the top-two fold in registers).
// A node whose every decision lies outside the error band is written here;
// any other node is queued for the exact pass with its FP32 values (NaN
// marking the slots that need an exact value) in the pending buffer, or with
// offset -1 (evaluated wholly in FP64 there) when the buffer is full.  Nodes
// of combined-level INCC, or with more slots than kSlotCap, are queued with
// offset -2 (evaluated wholly in FP64 by the exact pass).
__global__ void __launch_bounds__(kWinWarps * 32, VLL_WIN_MINB) window_kernel(
    const LevelSet LS, const int32_t *__restrict__ node_k, const double *__restrict__ gsum,
    const double *__restrict__ gcnt, float *__restrict__ pend_vals, int64_t pend_cap,
    int64_t *__restrict__ pend_node, int64_t *__restrict__ pend_off,
    float *__restrict__ warp_vals, int64_t *__restrict__ fix_list, int64_t fix_cap,
    unsigned long long *__restrict__ counters, unsigned long long *__restrict__ ctl,
    int warp_quads, int warp_raw, int grab) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    WinShared &W = reinterpret_cast<WinShared *>(smem_raw)[warp];
    const uint32_t box_off = (uint32_t)(win_boxes_offset() + (size_t)warp * warp_quads * 16);
    float4 *boxes = reinterpret_cast<float4 *>(smem_raw + box_off);
    unsigned char *raw = smem_raw + win_raw_offset(warp_quads) + (size_t)warp * warp_raw;
    // the FP32 values of the warp's current node (read back only by the lane
    // that wrote them, when the node is queued for the exact pass)
    float *wv = warp_vals + ((size_t)blockIdx.x * kWinWarps + warp) * kSlotCap;
    LevelConst &LC = *reinterpret_cast<LevelConst *>(smem_raw + win_level_offset());
    level_const_load(LC, LS.lv[0]);
    if (lane == 0) {
        mbar_init(&W.mbar);
        W.tmap_level = nullptr;
    }
    __syncthreads();
    uint32_t phase = 0;   // parity of the mbarrier phase the next copies complete
    unsigned long long evals = 0;
    // node queue: batches of `grab` nodes
    unsigned long long qbase = 0;
    int qi = grab, qk = 0;
    bool qdone = false;
    // the last fetched group: its node's context, first slot and the node's slot count
    int pb = 1, pk0 = 0, pK = 0;
    // the fetched group, per lane: status | inside << 2 | target radius << 8,
    // reference window and target centre offsets in the boxes (row << 16 |
    // column), fractions, and the two orientation bytes (loaded when the
    // group is fetched, read when it is evaluated: the loads' latency passes
    // under the evaluation of the group before)
    int nst = 0;
    uint32_t nro = 0, nto = 0, nor0 = 0, nor1 = 0;
    float nrfx = 0.f, nrfy = 0.f, ntfx = 0.f, ntfy = 0.f;
    // ... and its boxes (warp-uniform): mode 0 none / 1 tiles / 2 loads
    int nmode = 0, nrx0 = 0, nry0 = 0, nrw = 0, nrbh = 0, ntx0 = 0, nty0 = 0, ntw = 0, ntbh = 0;
    // the group being evaluated
    bool have_cur = false;
    int cb = 0, ck0 = 0;
    // per-lane running values of the streamed scan over the current node
    float vmax = -100.0f, amb = -INFINITY, amb_peak = -INFINITY;
    float b1 = -INFINITY, b2 = -INFINITY;
    bool need = false;
    PHASE_DECL;
    for (;;) {
        const int st = nst;
        const uint32_t ro = nro, to = nto, or0 = nor0, or1 = nor1;
        const float rfx = nrfx, rfy = nrfy, tfx = ntfx, tfy = ntfy;
        const int rbw = nrw | 1, rbh = nrbh, tbw = ntw | 1, tbh = ntbh;
        bool staged = false;
        // ---- stage the current group's boxes ----
        if (have_cur && nmode != 0) {
            const NodeCtx &C = W.node[cb];
            if (lane == 0) W.zn = 0;
            __syncwarp();
            float4 *tbox = boxes + rbw * rbh;
            if (nmode == 1) {
                if (!__all_sync(0xffffffffu, mbar_wait(&W.mbar, phase, 2000000000ll))) {
                    // the copies did not complete within ~1 s: report, wait
                    // once more (bounded) for them, and stop this warp
                    if (lane == 0) atomicExch(&counters[3], 1ull);
                    mbar_wait(&W.mbar, phase, 2000000000ll);
                    return;
                }
                phase ^= 1u;
                PHASE(0);
                const int tw0 = C.tma_w[0], tw1 = C.tma_w[1];
                const int rtile = (tw0 * C.tma_h[0] * 2 + 127) & ~127;   // bytes per plane tile
                const int ttile = (tw1 * C.tma_h[1] * 2 + 127) & ~127;
                const unsigned char *rI = raw, *rM = raw + rtile;
                const unsigned char *tIr = raw + 2 * rtile, *tMr = tIr + ttile;
                const int rxa = nrx0 & ~7, txa = ntx0 & ~7;
                const int rnb = 2 * tw0, tnb = 2 * tw1;   // tile row bytes
                // box shifts: the centre texels
                const int rc = (rbh / 2) * rnb + 2 * (nrx0 + nrw / 2 - rxa);
                const int tc = (tbh / 2) * tnb + 2 * (ntx0 + ntw / 2 - txa);
                const float sI = (float)*reinterpret_cast<const uint16_t *>(rI + rc);
                const float sM = (float)*reinterpret_cast<const uint16_t *>(rM + rc);
                const float tsI = (float)*reinterpret_cast<const uint16_t *>(tIr + tc);
                const float tsM = (float)*reinterpret_cast<const uint16_t *>(tMr + tc);
                // reference box (pairs), then target box (value + difference)
#pragma unroll 1
                for (int im = 0; im < 2; ++im) {
                    if (im == 0)
                        convert_tile(boxes, rbw, rI, rM, rnb, rxa, nrx0, nrw, rbh, sI, sM, 0.f,
                                     W.zl, &W.zn, kZeroCap, 0u, lane);
                    else
                        convert_tile(tbox, tbw, tIr, tMr, tnb, txa, ntx0, ntw, tbh, tsI, tsM, -1.f,
                                     W.zl, &W.zn, kZeroCap, 0x80000000u, lane);
                }
                // the tiles are rewritten by the next group's copies: every
                // value read from them has been stored into the boxes, so the
                // reads are complete once the warp has synchronised
                __syncwarp();
            } else {
                float sI = 0.f, sM = 0.f, tsI = 0.f, tsM = 0.f;
                if (lane == 0) {
                    const int64_t pc = (int64_t)(nry0 + rbh / 2) * C.w[0] + (nrx0 + rbw / 2);
                    sI = (float)__ldg(C.img[0] + pc);
                    sM = (float)__ldg(C.mag[0] + pc);
                    const int64_t p2 = (int64_t)(nty0 + tbh / 2) * C.w[1] + (ntx0 + tbw / 2);
                    tsI = (float)__ldg(C.img[1] + p2);
                    tsM = (float)__ldg(C.mag[1] + p2);
                }
                sI = __shfl_sync(0xffffffffu, sI, 0);
                sM = __shfl_sync(0xffffffffu, sM, 0);
                tsI = __shfl_sync(0xffffffffu, tsI, 0);
                tsM = __shfl_sync(0xffffffffu, tsM, 0);
                bool z;
                if (C.flags & kNfVec) {
                    z = stage_box_vec<false>(boxes, rbw, C.img[0], C.mag[0], C.w[0], nrx0, nry0,
                                             nrw, rbh, sI, sM, lane);
                    z |= stage_box_vec<true>(tbox, tbw, C.img[1], C.mag[1], C.w[1], ntx0, nty0,
                                             ntw, tbh, tsI, tsM, lane);
                } else {
                    z = stage_box_strided<false>(boxes, rbw, C.img[0], C.mag[0], C.w[0], nrx0,
                                                 nry0, nrw, rbh, sI, sM, lane);
                    z |= stage_box_strided<true>(tbox, tbw, C.img[1], C.mag[1], C.w[1], ntx0,
                                                 nty0, ntw, tbh, tsI, tsM, lane);
                }
                // a zero texel in these boxes sends every slot to the exact pass
                if (z && lane == 0) W.zn = kZeroCap + 1;
                __syncwarp();
            }
            staged = true;
        }
        PHASE(1);

        // ---- fetch the next group: node, geometry, boxes, tile copies ----
        bool have_next = false;
        if (pK > 0 && pk0 + 32 < pK) {
            pk0 += 32;
            have_next = true;
        } else {
            pK = 0;
            while (!qdone) {
                if (qi >= grab) {
                    // a batch of `grab` nodes and their slot counts (lane i: node i)
                    unsigned long long b = 0;
                    if (lane == 0) b = atomicAdd(&ctl[0], (unsigned long long)grab);
                    qbase = __shfl_sync(0xffffffffu, b, 0);
                    qk = (lane < grab && (int64_t)qbase + lane < LS.total)
                             ? node_k[(int64_t)qbase + lane] : 0;
                    qi = 0;
                }
                const int64_t gn = (int64_t)qbase + qi;
                const int K = __shfl_sync(0xffffffffu, qk, qi);
                ++qi;
                if (gn >= LS.total) {
                    qdone = true;
                    break;
                }
                if (K == 0) continue;
                const int lvl = level_of(LS, gn);
                if (LS.lv[lvl].combined_incc || K > kSlotCap) {
                    // combined-level INCC (setsm_code.cpp:6378-6464: the windows at
                    // this level and the next finer one, the averaged orientation
                    // and both bounds tests), or a range longer than the slot
                    // scratch: the node is evaluated wholly in FP64 by the exact
                    // pass (offset -2: not evaluated yet)
                    if (lane == 0) {
                        const unsigned long long idx = atomicAdd(&ctl[2], 1ull);
                        pend_node[idx] = gn;
                        pend_off[idx] = -2;
                    }
                    continue;
                }
                pb ^= 1;
                node_setup(W.node[pb], LS, lvl, gn, K, gsum, gcnt, lvl == 0 ? &LC : nullptr, lane);
                pk0 = 0;
                pK = K;
                have_next = true;
                break;
            }
        }
        PHASE(2);
        nmode = 0;
        if (have_next) {
            const NodeCtx &N = W.node[pb];
            const int k = pk0 + lane;
            const int H = N.H;
            int status = 0;   // 0 idle/skip, 2 inside both images
            double2 rp = make_double2(0, 0), tp = make_double2(0, 0);
            uint32_t o0 = 0, o1 = 0;
            if (k < N.K) {
                const float hgt = (float)__dadd_rn(N.hbase, __dmul_rn((double)k, N.hstep));
                if (hgt >= (float)N.start_H && hgt <= (float)N.end_H) {
                    bool edge = false;
#pragma unroll 1
                    for (int im = 0; im < 2; ++im) {
                        const double2 q = node_coord(N, im, (double)hgt, edge);
                        if (im == 0)
                            rp = q;
                        else
                            tp = q;
                    }
                    if (edge) slot_coords_exact(N, (double)hgt, rp, tp);
                    if (in_image(rp, N.w[0], N.h[0]) && in_image(tp, N.w[1], N.h[1])) {
                        o0 = N.ori[0][(int64_t)(int)rp.y * N.w[0] + (int)rp.x];
                        o1 = N.ori[1][(int64_t)(int)tp.y * N.w[1] + (int)tp.x];
                        status = 2;
                    }
                }
            }
            const int rix = (int)floor(rp.x), riy = (int)floor(rp.y);
            const int tix = (int)floor(tp.x), tiy = (int)floor(tp.y);
            // target footprint radius: the window is the square |col|, |row| <= H
            // cut by the disc of radius H + 1, so a rotation moves its samples
            // at most H + 1 from the centre (+1 for the bilinear neighbour and
            // FP32 rounding); the bound holds for every rotation, so the boxes
            // are placed before the orientation bytes arrive
            const int R = H + 2;
            const bool inside = status == 2 && rix - H >= 0 && riy - H >= 0 &&
                                rix + H + 2 < (int)N.w[0] && riy + H + 2 < (int)N.h[0] &&
                                tix - R >= 0 && tiy - R >= 0 && tix + R + 2 < (int)N.w[1] &&
                                tiy + R + 2 < (int)N.h[1];
            const int rx0 = __reduce_min_sync(0xffffffffu, inside ? rix - H : INT_MAX);
            const int ry0 = __reduce_min_sync(0xffffffffu, inside ? riy - H : INT_MAX);
            const int rx1 = __reduce_max_sync(0xffffffffu, inside ? rix + H + 1 : INT_MIN);
            const int ry1 = __reduce_max_sync(0xffffffffu, inside ? riy + H + 1 : INT_MIN);
            const int tx0 = __reduce_min_sync(0xffffffffu, inside ? tix - R : INT_MAX);
            const int ty0 = __reduce_min_sync(0xffffffffu, inside ? tiy - R : INT_MAX);
            const int tx1 = __reduce_max_sync(0xffffffffu, inside ? tix + R + 1 : INT_MIN);
            const int ty1 = __reduce_max_sync(0xffffffffu, inside ? tiy + R + 1 : INT_MIN);
            nst = status | (inside ? 4 : 0) | (R << 8);
            nro = inside ? ((uint32_t)(riy - H - ry0) << 16) | (uint32_t)(rix - H - rx0) : 0u;
            nto = inside ? ((uint32_t)(tiy - ty0) << 16) | (uint32_t)(tix - tx0) : 0u;
            nrfx = (float)(rp.x - (double)rix);
            nrfy = (float)(rp.y - (double)riy);
            ntfx = (float)(tp.x - (double)tix);
            ntfy = (float)(tp.y - (double)tiy);
            nor0 = o0;
            nor1 = o1;
            if (rx0 != INT_MAX) {
                // pairs [x0, x1] of rows [y0, y1]; odd row strides spread
                // consecutive rows over the shared-memory bank groups
                nrx0 = rx0;
                nry0 = ry0;
                nrw = rx1 - rx0 + 1;
                nrbh = ry1 - ry0 + 1;
                ntx0 = tx0;
                nty0 = ty0;
                ntw = tx1 - tx0 + 1;
                ntbh = ty1 - ty0 + 1;
                const bool fits = (nrw | 1) * nrbh + (ntw | 1) * ntbh <= warp_quads;
                // the level's TMA tiles: texels [xa, xa + tma_w) x rows [y0, y0 +
                // tma_h) of each plane, xa = x0 rounded down to 8 (16 bytes)
                const int rxa = rx0 & ~7, txa = tx0 & ~7;
                const int tw0 = N.tma_w[0], th0 = N.tma_h[0];
                const int tw1 = N.tma_w[1], th1 = N.tma_h[1];
                const int rtile = (tw0 * th0 * 2 + 127) & ~127;   // bytes per plane tile
                const int ttile = (tw1 * th1 * 2 + 127) & ~127;
                const bool tma = (N.flags & kNfTma) && rx1 + 2 - rxa <= tw0 && nrbh <= th0 &&
                                 tx1 + 2 - txa <= tw1 && ntbh <= th1 &&
                                 2 * (rtile + ttile) <= warp_raw;
                if (fits && tma) {
                    nmode = 1;
                    if (lane == 0) {
                        const DevLevel &P = *N.P;
                        if (&P != W.tmap_level) {
                            // the level's tensor maps were written by the host
                            // (the level block is reused between calls): make
                            // them visible to this thread's copies
                            tmap_acquire(P.tmap[0][0]);
                            tmap_acquire(P.tmap[0][1]);
                            tmap_acquire(P.tmap[1][0]);
                            tmap_acquire(P.tmap[1][1]);
                            W.tmap_level = &P;
                        }
                        unsigned char *rI = raw, *rM = raw + rtile;
                        unsigned char *tIr = raw + 2 * rtile, *tMr = tIr + ttile;
                        mbar_arrive_expect(&W.mbar, (uint32_t)(2 * (tw0 * th0 + tw1 * th1) * 2));
                        tma_tile_2d(rI, P.tmap[0][0], rxa, ry0, &W.mbar);
                        tma_tile_2d(rM, P.tmap[0][1], rxa, ry0, &W.mbar);
                        tma_tile_2d(tIr, P.tmap[1][0], txa, ty0, &W.mbar);
                        tma_tile_2d(tMr, P.tmap[1][1], txa, ty0, &W.mbar);
                    }
                } else if (fits) {
                    nmode = 2;
                }
            }
        }

        PHASE(3);
        // ---- evaluate the current group ----
        if (have_cur) {
            NodeCtx &C = W.node[cb];
            const int K = C.K;
            const int k = ck0 + lane;
            const bool inside = (st & 4) != 0;
            const uint32_t flags = C.flags;
            // the orientation difference (setsm_code.cpp:6395-6427): the
            // angle test and the target window's rotation
            int status = st & 3;
            float cf = 1.f, sf = 0.f;
            if (status == 2) {
                const int od = (int)or0 - (int)or1;
                if (flags & kNfOri) {
                    const double a = __dmul_rn((double)od, C.bin_angle);
                    if (!(a < 90 && a > -90)) status = 1;
                }
                const int rot = 2 * od + kRotOffset;
                cf = (float)C.P->rot_cos[rot];
                sf = (float)C.P->rot_sin[rot];
            }
            // a zero intensity texel within the slot's footprints: the
            // reference drops the samples whose interpolated intensity is not
            // positive, which FP32 on shifted texels cannot decide
            bool zero_hit = false;
            if (staged && status == 2 && inside) {
                const int zn = W.zn;
                if (zn > kZeroCap) {
                    zero_hit = true;
                } else if (zn > 0) {
                    const int H = C.H, R = st >> 8;
                    const int rxo = (int)(ro & 0xFFFFu), ryo = (int)(ro >> 16);
                    const int txo = (int)(to & 0xFFFFu), tyo = (int)(to >> 16);
                    for (int i = 0; i < zn; ++i) {
                        const uint32_t e = W.zl[i];
                        const int ex = (int)(e & 0xFFFFu), ey = (int)((e >> 16) & 0x7FFFu);
                        if (e & 0x80000000u)
                            zero_hit |= ex >= txo - R && ex <= txo + R + 1 && ey >= tyo - R &&
                                        ey <= tyo + R + 1;
                        else
                            zero_hit |= ex >= rxo && ex <= rxo + 2 * H + 1 && ey >= ryo &&
                                        ey <= ryo + 2 * H + 1;
                    }
                }
            }
            float rho_v = kNotEvaluated, incc_v = 0.f;
            bool all_pos = false, deferred = false;
            if (status == 1) {
                rho_v = kRejected;
            } else if (status == 2) {
                if (staged && inside && !zero_hit) {
                    float incc;
                    bool unsure = false;
                    const float4 *qr = boxes + (int)(ro >> 16) * rbw + (int)(ro & 0xFFFFu);
                    const uint32_t tcen =
                        box_off + (uint32_t)(rbw * rbh + (int)(to >> 16) * tbw + (int)(to & 0xFFFFu)) * 16u;
                    window_any(C.H, qr, rbw, rfx, rfy, tgt_box(smem_raw, tcen, (uint32_t)tbw * 16u),
                               tfx, tfy, cf, sf, incc, unsure);
                    const bool has = incc != -2.0f;
                    const double incc_d = has ? (double)incc : -1.0;
                    double rho_d;
                    if (flags & kNfGncc)
                        rho_d = has ? incc_d * C.alpha + C.gterm : __ddiv_rn(0.0, 0.0);
                    else
                        rho_d = incc_d;
                    rho_v = (float)rho_d;
                    incc_v = unsure ? __int_as_float(0x7fc00000) : (float)incc_d;
                    all_pos = true;   // window inside the image, no zero texels
                } else {
                    // window not staged (near an image edge, a zero texel in
                    // its footprint, or boxes beyond the budget): the exact pass
                    // evaluates the slot in FP64
                    rho_v = 0.f;
                    incc_v = __int_as_float(0x7fc00000);
                    deferred = true;
                }
                evals++;
            }

            PHASE(4);
            // ---- FindPeakNcc streamed over this group of 32 slots ----
            // (setsm_code.cpp:6672-6752 on the FP32 values; every decision
            // within the error band, and every value the FP32 pass could not
            // take -- deferred windows, unsure variances, voxel truncations
            // near an integer, NaN --, sends the node to the exact pass)
            const bool voxels = (flags & kNfVox) != 0;
            const bool ev = k < K && status == 2;
            // a voxel INCC whose truncation FP32 cannot decide needs only its
            // own exact value: the slot is listed for slot_fix_kernel (or,
            // the list full, taken as unusable)
            bool unusable = ev && (isnan(incc_v) || isnan(rho_v));
            if (ev && !unusable && voxels && near_trunc((double)incc_v)) {
                const unsigned long long q = atomicAdd(&ctl[5], 1ull);
                if ((int64_t)q < fix_cap)
                    fix_list[q] = C.gn * kSlotCap + k;
                else
                    unusable = true;
            }
            if (k < K) wv[k] = unusable ? __int_as_float(0x7fc00000) : rho_v;
            bool band = unusable;
            const uint32_t em = __ballot_sync(0xffffffffu, ev);
            if (em) {
                const int p_in = prev_eval(em, lane, -1);
                const float pv_in = __shfl_sync(0xffffffffu, rho_v, p_in < 0 ? 0 : p_in);
                const bool has_p = p_in >= 0 || C.have;
                const float pv = p_in >= 0 ? pv_in : C.pre_v;
                // direction of this slot: the sign of the change (the
                // reference's sign rule reduces to it); -1 on the first one
                const int td = has_p ? (rho_v > pv) - (rho_v < pv) : -1;
                const int td_in = __shfl_sync(0xffffffffu, td, p_in < 0 ? 0 : p_in);
                const int dp = p_in >= 0 ? td_in : C.pre_dir;
                bool is_peak = false;
                if (ev && !unusable) {
                    const float fv = rho_v;
                    if (fv > vmax) vmax = fv;
                    if (near_round((double)fv) && fv > amb) amb = fv;
                    if ((flags & kNfCmr) && has_p) {
                        if (fabsf(fv - pv) < kBand || fabsf(fv) < kBand || fabsf(pv) < kBand)
                            band = true;
                        is_peak = pv != -1.0f && dp > 0 && td < 0;
                    }
                }
                // each peak's rounded value and height (its lane), then the
                // ordered top-two fold of this group's peaks (lane 0)
                int q_l = 0;
                float ph_l = 0.f;
                if (is_peak) {
                    if (near_round((double)pv) && pv > amb_peak) amb_peak = pv;
                    if (pv > b1) {
                        b2 = b1;
                        b1 = pv;
                    } else if (pv > b2) {
                        b2 = pv;
                    }
                    const int p_slot = p_in >= 0 ? ck0 + p_in : C.pre_k;
                    q_l = q_result((double)pv);
                    ph_l = (float)__dadd_rn(C.hbase, __dmul_rn((double)p_slot, C.hstep));
                }
                uint32_t pm = __ballot_sync(0xffffffffu, is_peak);
                if (pm) {
                    // the fold in registers on every lane (the same values);
                    // the replaced maximum re-quantised, q_result(dq_result(x)),
                    // is x for every int16 x (|x / 1000 * 1000 - x| < 1e-11)
                    vll_nccresult &R = C.R;
                    int16_t r0 = R.result0, r1 = R.result1;
                    float r2 = R.result2, r3 = R.result3;
                    int r4 = R.result4;
                    do {
                        const int b = __ffs(pm) - 1;
                        pm &= pm - 1;
                        const int16_t qpre = (int16_t)__shfl_sync(0xffffffffu, q_l, b);
                        const float ph = __shfl_sync(0xffffffffu, ph_l, b);
                        if (r4 < 10) ++r4;
                        if (r0 < qpre) {
                            if (r1 < r0) {
                                r1 = r0;
                                r3 = r2;
                            }
                            r0 = qpre;
                            r2 = ph;
                        } else if (r1 < qpre) {
                            r1 = qpre;
                            r3 = ph;
                        }
                    } while (pm);
                    __syncwarp();
                    if (lane == 0) {
                        R.result0 = r0;
                        R.result1 = r1;
                        R.result2 = r2;
                        R.result3 = r3;
                        R.result4 = (decltype(R.result4))r4;
                    }
                }
                // carry the last evaluated slot into the next group
                const int last = 31 - __clz(em);
                const float lv = __shfl_sync(0xffffffffu, rho_v, last);
                const int ld = __shfl_sync(0xffffffffu, td, last);
                __syncwarp();
                if (lane == 0) {
                    C.pre_v = lv;
                    C.pre_dir = ld;
                    C.pre_k = ck0 + last;
                    C.have = 1;
                }
            }
            if (__any_sync(0xffffffffu, band)) need = true;
            if (status == 2 && (flags & kNfDbg))
                C.P->dbg_rho[C.P->dbg_off[C.pt] + k] =
                    deferred ? __longlong_as_double(0x7ff8000000000000ll) : (double)rho_v;
            if (k < K && voxels) {
                vll_voxel *v = C.vrow + k;
                if (status == 1) v->flag_cal = 0;
                if (status == 2) {
                    if (all_pos) v->flag_cal = 1;
                    v->INCC = q_voxel(isnan(incc_v) ? 0.0 : (double)incc_v);
                }
            }
            __syncwarp();
            PHASE(5);
            PHASE_COUNT(0);
            if (ck0 + 32 >= K) {
                PHASE_COUNT(1);
                // ---- the node's last group: write it, or queue it ----
                // the maximum, and roundings that could change the maximum or
                // the top two (a peak more than 0.002 + 2 bands below the
                // second best rounds strictly below it)
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
                    amb = fmaxf(amb, __shfl_xor_sync(0xffffffffu, amb, o));
                    amb_peak = fmaxf(amb_peak, __shfl_xor_sync(0xffffffffu, amb_peak, o));
                    const float o1 = __shfl_xor_sync(0xffffffffu, b1, o);
                    const float o2 = __shfl_xor_sync(0xffffffffu, b2, o);
                    const float n1 = fmaxf(b1, o1);
                    const float n2 = fmaxf(fminf(b1, o1), fmaxf(b2, o2));
                    b1 = n1;
                    b2 = n2;
                }
                if ((flags & kNfChc) && (double)amb >= (double)vmax - (double)kBand) need = true;
                if ((flags & kNfCmr) && amb_peak > -1e29f) {
                    const double thr =
                        (double)(b2 > -1e29f ? b2 : b1) - 0.002 - 2.0 * (double)kBand;
                    if ((double)amb_peak >= thr) need = true;
                }
                if (!need) {
                    if (lane == 0) {
                        vll_nccresult R = C.R;
                        if (R.check_height_change) R.max_WNCC = q_result((double)vmax);
                        C.P->ncc[C.pt] = R;
                    }
                } else {
                    long long off = -1;
                    if (lane == 0) {
                        off = (long long)atomicAdd(&ctl[4], (unsigned long long)K);
                        if (off + K > pend_cap) off = -1;
                        const unsigned long long idx = atomicAdd(&ctl[2], 1ull);
                        pend_node[idx] = C.gn;
                        pend_off[idx] = off;
                    }
                    off = __shfl_sync(0xffffffffu, off, 0);
                    if (off >= 0)
                        for (int kk = lane; kk < K; kk += 32) pend_vals[off + kk] = wv[kk];
                }
                vmax = -100.0f;
                amb = amb_peak = b1 = b2 = -INFINITY;
                need = false;
                __syncwarp();
            }
        }
        PHASE(6);
        if (!have_next) break;
        have_cur = true;
        cb = pb;
        ck0 = pk0;
    }
    PHASE_FLUSH();
    for (int o = 16; o; o >>= 1) evals += __shfl_down_sync(0xffffffffu, evals, o);
    if (lane == 0 && evals) atomicAdd(&counters[1], evals);
}

// ---------------------------------------------------------------------------
// slot fix: exact voxel INCC of the listed slots
// ---------------------------------------------------------------------------
// One lane per slot listed by the window kernel (node * kSlotCap + slot):
// the slot is evaluated in exact FP64 (eval_slot, the reference's operation
// order) and its voxel's INCC rewritten; the node's other outputs did not
// depend on the truncation.
__global__ void __launch_bounds__(128) slot_fix_kernel(const LevelSet LS,
                                                       const int64_t *__restrict__ fix_list,
                                                       int64_t fix_cap,
                                                       const double *__restrict__ gsum,
                                                       const double *__restrict__ gcnt,
                                                       const unsigned long long *__restrict__ ctl) {
    const int64_t n = min((int64_t)ctl[5], fix_cap);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = fix_list[i];
        const int64_t gn = e / kSlotCap;
        const int k = (int)(e - gn * kSlotCap);
        const int lvl = level_of(LS, gn);
        const DevLevel &P = LS.lv[lvl];
        const int64_t pt = gn - __ldg(LS.base + lvl);
        PatchSrc S, Sn;
        make_src(P, 1, S, Sn);
        const int start_H = P.gp3[pt].minHeight;
        const float hgt = slot_height(P, start_H, P.ncc[pt].minHeight, k);
        const double cnt_g = gcnt ? gcnt[gn] : 0.0, sum_g = gsum ? gsum[gn] : 0.0;
        const SlotOut o = eval_slot(P, pt, 1, S, Sn, hgt, cnt_g, sum_g);
        if (o.evaluated)
            P.vox[P.vox_off[pt] + k].INCC =
                o.count_incc > 0 ? q_voxel(__ddiv_rn(o.sum_incc, o.count_incc)) : q_voxel(-1.0);
    }
}

// ---------------------------------------------------------------------------
// peak kernel: the exact pass, one warp per queued node
// ---------------------------------------------------------------------------
constexpr int kPeakWarps = 4;

struct WarpShared {
    float rho[kSlotCap];
    double xrho[kSlotCap];           // exact value of each re-checked slot
    int todo[kSlotCap];              // this round's slots to re-check
    SlotMasks m;
    uint32_t exact[kSlotCap / 32];
    double chunk[32];
};

// value of slot k for the scan: exact if re-checked, else the FP32 one
__device__ __forceinline__ double slot_value(const WarpShared &w, int k, bool &ex) {
    ex = bit(w.exact, k);
    return ex ? w.xrho[k] : (double)w.rho[k];
}

// Exact FP64 evaluation of one slot by the whole warp, bit-identical with
// eval_slot (the reference's operation order): lanes 0/1 project into the two
// images; every lane bilinear-samples its share of the window offsets (each
// sample is computed independently, so this is exact); lanes 0..5 then run
// the six two-pass Pearson sums (3 sub-windows x {intensity, magnitude}) over
// the samples in the reference's scan order; lane 0 combines them in
// ComputeMultiNCC's order.  `scratch` holds (2H+1)^2 x 4 doubles + flags.
template <int H>
__device__ __noinline__ SlotOut eval_slot_warp(const DevLevel &P, int64_t pt, const PatchSrc &S, float hgt,
                                  double cnt_g, double sum_g, double *scratch, int lane) {
    constexpr int D = 2 * H + 1;
    SlotOut o;
    o.evaluated = false;
    o.orient_reject = false;
    o.all_pos = false;
    o.rho = -1.0;
    o.count_incc = 0;
    o.sum_incc = 0;
    const DevImage &ri = P.im[P.ref];
    const DevImage &tI = P.im[1];
    const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
    double2 c = make_double2(0, 0);
    if (lane < 2) {
        const DevImage &im = lane == 0 ? ri : tI;
        c = rpc_project(im.rpc, im.adj, lon, lat, (double)hgt);
    }
    const double2 rc = make_double2(__shfl_sync(0xffffffffu, c.x, 0), __shfl_sync(0xffffffffu, c.y, 0));
    const double2 tc = make_double2(__shfl_sync(0xffffffffu, c.x, 1), __shfl_sync(0xffffffffu, c.y, 1));
    const double2 rp = to_pyramid(rc, ri.sx, ri.sy, P.L);
    const double2 tp = to_pyramid(tc, tI.sx, tI.sy, P.L);
    if (!(in_image(rp, ri.w, ri.h) && in_image(tp, tI.w, tI.h))) return o;
    const int od = (int)ri.ori[(int64_t)(int)rp.y * ri.w + (int)rp.x] -
                   (int)tI.ori[(int64_t)(int)tp.y * tI.w + (int)tp.x];
    if (!P.is_ra && P.L >= 3) {
        const double a = __dmul_rn((double)od, P.bin_angle);
        if (!(a < 90 && a > -90)) {
            o.orient_reject = true;
            return o;
        }
    }
    o.evaluated = true;
    const double c0 = P.rot_cos[2 * od + kRotOffset], s0 = P.rot_sin[2 * od + kRotOffset];
    unsigned char *flag = reinterpret_cast<unsigned char *>(scratch + 4 * D * D);
    for (int idx = lane; idx < D * D; idx += 32) {
        const int row = idx / D - H, col = idx % D - H;
        const int r2 = row * row + col * col;
        unsigned char f = 0;
        if (r2 <= (H + 1) * (H + 1)) {
            const double ox = __dadd_rn(__dmul_rn(c0, (double)col), -__dmul_rn(s0, (double)row));
            const double oy = __dadd_rn(__dmul_rn(s0, (double)col), __dmul_rn(c0, (double)row));
            const double2 pl = make_double2(__dadd_rn(rp.x, (double)col), __dadd_rn(rp.y, (double)row));
            const double2 pr = make_double2(__dadd_rn(tp.x, ox), __dadd_rn(tp.y, oy));
            double v[4];
            if (sample4(S, pl, pr, v)) {
                f = (unsigned char)(1 + window_depth(H, row, col, r2));   // 1 + depth
#pragma unroll
                for (int ch = 0; ch < 4; ++ch) scratch[4 * idx + ch] = v[ch];
            }
        }
        flag[idx] = f;
    }
    __syncwarp();
    // lanes 0..5: Correlate for (window w, channel pair p), SubFunctions.cpp:974-1018
    double r = -99.0;
    int n = 0;
    if (lane < 6) {
        const int w = lane >> 1, p = lane & 1;
        double Ls = 0, Rs = 0;
        for (int idx = 0; idx < D * D; ++idx) {
            const int f = flag[idx];
            if (f == 0 || f - 1 < w) continue;
            Ls = __dadd_rn(Ls, scratch[4 * idx + p]);
            Rs = __dadd_rn(Rs, scratch[4 * idx + p + 2]);
            ++n;
        }
        if (n > 0) {
            const double Lm = __ddiv_rn(Ls, (double)n), Rm = __ddiv_rn(Rs, (double)n);
            double slr = 0, sl2 = 0, sr2 = 0;
            for (int idx = 0; idx < D * D; ++idx) {
                const int f = flag[idx];
                if (f == 0 || f - 1 < w) continue;
                const double dl = __dadd_rn(scratch[4 * idx + p], -Lm);
                const double dr = __dadd_rn(scratch[4 * idx + p + 2], -Rm);
                slr = __dadd_rn(slr, __dmul_rn(dl, dr));
                sl2 = __dadd_rn(sl2, __dmul_rn(dl, dl));
                sr2 = __dadd_rn(sr2, __dmul_rn(dr, dr));
            }
            if (sl2 > 1e-8 && sr2 > 1e-8) r = __ddiv_rn(slr, sqrt(__dmul_rn(sl2, sr2)));
        }
    }
    double rv[6];
    int nv[3];
#pragma unroll
    for (int j = 0; j < 6; ++j) rv[j] = __shfl_sync(0xffffffffu, r, j);
#pragma unroll
    for (int w = 0; w < 3; ++w) nv[w] = __shfl_sync(0xffffffffu, n, 2 * w);
    __syncwarp();
    o.all_pos = nv[0] > 0 && nv[1] > 0 && nv[2] > 0;
    double count = 0, sum = 0;
    if (o.all_pos) {
        double tot = 0, cntv = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            if (rv[j] != -99.0) {
                cntv = __dadd_rn(cntv, 1.0);
                tot = __dadd_rn(tot, rv[j]);
            }
        }
        if (cntv > 0) {
            sum = __ddiv_rn(tot, cntv);
            count = 1.0;
        }
    }
    o.count_incc = count;
    o.sum_incc = sum;
    if (P.check_ortho && cnt_g > 0)
        o.rho = __dadd_rn(__dmul_rn(__ddiv_rn(sum, count), P.alpha),
                          __dmul_rn(__ddiv_rn(sum_g, cnt_g), P.beta));
    else
        o.rho = count > 0 ? __ddiv_rn(sum, count) : -1.0;
    return o;
}


// bytes of eval_slot_warp scratch for window half-size H
__host__ __device__ constexpr size_t exact_scratch_bytes(int H) {
    return (size_t)(2 * H + 1) * (2 * H + 1) * 33 + 16;
}

// Exact FP64 evaluation of one slot by the warp for the level's half-size.
__device__ __forceinline__ SlotOut eval_slot_warp_any(const DevLevel &P, int64_t pt,
                                                      const PatchSrc &S, float hgt, double cnt_g,
                                                      double sum_g, double *scratch, int lane) {
    switch (P.H) {
        case 2: return eval_slot_warp<2>(P, pt, S, hgt, cnt_g, sum_g, scratch, lane);
        case 3: return eval_slot_warp<3>(P, pt, S, hgt, cnt_g, sum_g, scratch, lane);
        case 4: return eval_slot_warp<4>(P, pt, S, hgt, cnt_g, sum_g, scratch, lane);
        case 5: return eval_slot_warp<5>(P, pt, S, hgt, cnt_g, sum_g, scratch, lane);
        case 6: return eval_slot_warp<6>(P, pt, S, hgt, cnt_g, sum_g, scratch, lane);
        default: return eval_slot_warp<7>(P, pt, S, hgt, cnt_g, sum_g, scratch, lane);
    }
}

// The exact pass for the nodes the window kernel could not settle in FP32:
// the decisions within the error band are re-taken on exact FP64 values of
// the slots involved (rounds of scan and re-evaluation: a few slots a warp
// each, more a lane each); a node still unsettled after kMaxRounds, or
// queued without its FP32 values, is evaluated wholly in FP64.
// `max_h`: the largest window half-size of the level set (scratch layout).
#ifndef VLL_PEAK_MINB
#define VLL_PEAK_MINB 3
#endif
__global__ void __launch_bounds__(kPeakWarps * 32, VLL_PEAK_MINB) peaks_kernel(
    const LevelSet LS, int max_h, const int32_t *__restrict__ node_k,
    const float *__restrict__ pend_vals, const int64_t *__restrict__ pend_node,
    const int64_t *__restrict__ pend_off, const double *__restrict__ gsum,
    const double *__restrict__ gcnt, unsigned long long *__restrict__ counters,
    unsigned long long *__restrict__ ctl) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    WarpShared &W = reinterpret_cast<WarpShared *>(smem_raw)[warp];
    constexpr size_t ws = (sizeof(WarpShared) + 15) & ~(size_t)15;
    const size_t xs = (exact_scratch_bytes(max_h) + 15) & ~(size_t)15;
    double *boxes = reinterpret_cast<double *>(smem_raw + ws * kPeakWarps + xs * warp);
    unsigned long long rechecks = 0, evals = 0;
    const unsigned long long n_pend = ctl[2];
    for (;;) {
        unsigned long long idx = 0;
        if (lane == 0) idx = atomicAdd(&ctl[1], 1ull);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= n_pend) break;
        const int64_t gn = pend_node[idx];
        const int64_t off = pend_off[idx];
        const int K = node_k[gn];
        if (K == 0) continue;
        const int lvl = level_of(LS, gn);
        const DevLevel &P = LS.lv[lvl];
        const int64_t pt = gn - __ldg(LS.base + lvl);
        PatchSrc S, Sn;
        make_src(P, 1, S, Sn);
        const bool voxels = P.vox && !P.cmr && !P.is_ra;
        vll_nccresult R = P.ncc[pt];
        const int start_H = P.gp3[pt].minHeight;
        const double cnt_g = gcnt ? gcnt[gn] : 0.0, sum_g = gsum ? gsum[gn] : 0.0;
        vll_voxel *vrow = voxels ? P.vox + P.vox_off[pt] : nullptr;
        if (off < 0 || K > kSlotCap || P.combined_incc) {
            // queued without FP32 values: not evaluated yet (-2: combined-level
            // INCC or more slots than kSlotCap), or the pending buffer was full
            const bool first = off == -2;
            if (lane == 0) atomicAdd(&counters[5], 1ull);
            node_exact_chunked(P, pt, K, S, Sn, cnt_g, sum_g, R, vrow, W.chunk, lane, first,
                               first ? evals : rechecks);
            continue;
        }
        if (lane < kSlotCap / 32) {
            W.m.evaluated[lane] = 0;
            W.m.need[lane] = 0;
            W.m.peak[lane] = 0;
            W.exact[lane] = 0;
        }
        __syncwarp();
        for (int k0 = 0; k0 < K; k0 += 32) {
            const int k = k0 + lane;
            float v = kNotEvaluated;
            if (k < K) v = pend_vals[off + k];
            const bool ev = k < K && !isinf(v);
            const bool nd = ev && isnan(v);
            const uint32_t em = __ballot_sync(0xffffffffu, ev);
            const uint32_t nm = __ballot_sync(0xffffffffu, nd);
            if (k < K) W.rho[k] = nd ? 0.f : v;
            if (lane == 0) {
                W.m.evaluated[k0 >> 5] = em;
                W.m.need[k0 >> 5] = nm;
            }
        }
        __syncwarp();
        auto xval = [&](int kk, bool &ex) { return slot_value(W, kk, ex); };
        // ---- scan, re-check, repeat ----
        double max_w = -100;
        bool redone = false;
        for (int round = 0;; ++round) {
            max_w = scan_pass(P, R.check_height_change != 0, K, W.m, xval, lane);
            // slots still needing an exact value
            int n_need = 0;
            for (int i = 0; i < (K + 31) / 32; ++i) n_need += __popc(W.m.need[i] & ~W.exact[i]);
            if (n_need == 0) break;
            const bool overflow = round + 1 >= kMaxRounds;
            if (lane == 0) atomicAdd(&counters[6], 1ull);
            if (overflow) {
                if (lane == 0) atomicAdd(&counters[5], 1ull);
                // give up on the FP32 values: the whole node exactly
                node_exact_chunked(P, pt, K, S, Sn, cnt_g, sum_g, R, vrow, W.chunk, lane, false,
                                   rechecks);
                redone = true;   // results already written
                break;
            }
            // compact the list of slots to re-check
            int n_todo = 0;
            for (int i = 0; i < (K + 31) / 32; ++i) {
                const uint32_t todo = W.m.need[i] & ~W.exact[i];
                if ((todo >> lane) & 1u) W.todo[n_todo + __popc(todo & ((1u << lane) - 1u))] = (i << 5) + lane;
                n_todo += __popc(todo);
            }
            __syncwarp();
            if (n_todo <= kWarpPerSlotMax) {
                // a few slots: the whole warp per slot
                for (int j = 0; j < n_todo; ++j) {
                    const int k = W.todo[j];
                    const float hh = slot_height(P, start_H, R.minHeight, k);
                    const SlotOut o = eval_slot_warp_any(P, pt, S, hh, cnt_g, sum_g,
                                                        reinterpret_cast<double *>(boxes), lane);
                    if (lane == 0) {
                        if (P.dbg_rho && o.evaluated && isnan(P.dbg_rho[P.dbg_off[pt] + k]))
                            P.dbg_rho[P.dbg_off[pt] + k] = o.rho;
                        W.xrho[k] = o.rho;
                        if (vrow) {
                            if (o.all_pos) vrow[k].flag_cal = 1;
                            vrow[k].INCC = q_voxel(o.count_incc > 0
                                                       ? __ddiv_rn(o.sum_incc, o.count_incc)
                                                       : -1.0);
                        }
                        rechecks++;
                    }
                    __syncwarp();
                }
            } else {
                // many (windows the FP32 pass could not stage): a lane per slot
                for (int j = lane; j < n_todo; j += 32) {
                    const int k = W.todo[j];
                    const float hh = slot_height(P, start_H, R.minHeight, k);
                    const SlotOut o = eval_slot(P, pt, 1, S, Sn, hh, cnt_g, sum_g);
                    if (P.dbg_rho && o.evaluated && isnan(P.dbg_rho[P.dbg_off[pt] + k]))
                        P.dbg_rho[P.dbg_off[pt] + k] = o.rho;
                    W.xrho[k] = o.rho;
                    if (vrow) {
                        if (o.all_pos) vrow[k].flag_cal = 1;
                        vrow[k].INCC = q_voxel(o.count_incc > 0 ? __ddiv_rn(o.sum_incc, o.count_incc)
                                                                : -1.0);
                    }
                    rechecks++;
                }
            }
            __syncwarp();
            for (int j = lane; j < n_todo; j += 32) set_bit(W.exact, W.todo[j]);
            if (lane < kSlotCap / 32) W.m.peak[lane] = 0;
            __syncwarp();
        }
        if (redone) continue;   // the node went through the FP64 path
        if (lane == 0) {
            if (P.cmr) fold_peaks(P, R, K, start_H, W.m.peak, xval);
            if (R.check_height_change) R.max_WNCC = q_result(max_w);
            P.ncc[pt] = R;
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) {
        rechecks += __shfl_down_sync(0xffffffffu, rechecks, o);
        evals += __shfl_down_sync(0xffffffffu, evals, o);
    }
    if (lane == 0 && rechecks) atomicAdd(&counters[2], rechecks);
    if (lane == 0 && evals) atomicAdd(&counters[1], evals);
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

// Host-side RPC line/sample (no clamp) for footprint estimates.
void host_rpc(const double *rpc, double lon, double lat, double h, double &x, double &y) {
    const double L = (lon - rpc[2]) / rpc[7], Pn = (lat - rpc[3]) / rpc[8], Hn = (h - rpc[4]) / rpc[9];
    const double t[20] = {1, L, Pn, Hn, L * Pn, L * Hn, Pn * Hn, L * L, Pn * Pn, Hn * Hn,
                          Pn * L * Hn, L * L * L, L * Pn * Pn, L * Hn * Hn, L * L * Pn,
                          Pn * Pn * Pn, Pn * Hn * Hn, L * L * Hn, Pn * Pn * Hn, Hn * Hn * Hn};
    double c[4] = {0, 0, 0, 0};
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 20; ++i) c[j] += rpc[10 + 20 * j + i] * t[i];
    y = c[0] / c[1] * rpc[5] + rpc[0];
    x = c[2] / c[3] * rpc[6] + rpc[1];
}

// The boxes covering 32 consecutive height slots of one node in both images
// -- the reference window and the target window (rotated; its samples lie
// within H + 1 of the centre) swept along their epipolar lines -- in texel
// pairs (w x h), per image [0] reference, [1] target.  The sweep per slot,
// along x and y, is measured from the RPCs over the image footprint; the
// boxes are the worst case times `margin` (an item with a larger footprint
// falls back to slower staging or to FP64).
struct WindowBoxes {
    int w[2], h[2];
};

WindowBoxes window_boxes(const DevLevel &P, float margin) {
    const int H = P.H;
    double rx[2] = {0, 0}, ry[2] = {0, 0};
    for (int ti = 0; ti < 2; ++ti) {
        const double *r = P.im[ti == 0 ? P.ref : 1].rpc;
        for (int a = -1; a <= 1; ++a)
            for (int b = -1; b <= 1; ++b) {
                const double lon = r[2] + 0.8 * a * r[7], lat = r[3] + 0.8 * b * r[8];
                double x0, y0, x1, y1;
                host_rpc(r, lon, lat, r[4] - 50.0, x0, y0);
                host_rpc(r, lon, lat, r[4] + 50.0, x1, y1);
                rx[ti] = std::max(rx[ti], fabs(x1 - x0) / 100.0 / (1 << P.L));
                ry[ti] = std::max(ry[ti], fabs(y1 - y0) / 100.0 / (1 << P.L));
            }
    }
    // one slot's box (texel pairs, rows: the reference window 2H + 2, the
    // target's rotated footprint 2(H + 2) + 2), plus the sweep of 31 height
    // steps with the margin, plus one texel of rounding
    const double m = margin > 0 ? margin : 1.1;
    const int side[2] = {2 * H + 2, 2 * (H + 2) + 2};
    WindowBoxes B;
    for (int ti = 0; ti < 2; ++ti) {
        B.w[ti] = side[ti] + (int)std::ceil(31.0 * P.height_step * rx[ti] * m) + 1;
        B.h[ti] = side[ti] + (int)std::ceil(31.0 * P.height_step * ry[ti] * m) + 1;
    }
    return B;
}

// Shared-memory budget per warp: the boxes as texel pairs (odd row strides)
// and, where the level has TMA tiles, the four tiles.
struct WarpBudget {
    int quads;   // float4 texel pairs
    int raw;     // bytes of TMA tiles (multiple of 128)
};

WarpBudget window_warp_budget(const DevLevel &P, float margin) {
    const WindowBoxes B = window_boxes(P, margin);
    WarpBudget wb;
    // boxes up to the budget's sides, rows of odd stride
    wb.quads = (B.w[0] | 1) * B.h[0] + (B.w[1] | 1) * B.h[1];
    wb.raw = 128;
    if (P.tma_w[0] > 0)
        wb.raw = 2 * (((P.tma_w[0] * P.tma_h[0] * 2 + 127) & ~127) +
                      ((P.tma_w[1] * P.tma_h[1] * 2 + 127) & ~127));
    // at most ~200 KB for the block: beyond, the tiles go (staging by loads)
    // and then the boxes shrink
    const size_t per_warp = (200 * 1024 - win_boxes_offset()) / kWinWarps - 128;
    if ((size_t)wb.quads * sizeof(float4) + wb.raw > per_warp) wb.raw = 128;
    if ((size_t)wb.quads * sizeof(float4) + wb.raw > per_warp)
        wb.quads = (int)((per_warp - wb.raw) / sizeof(float4));
    return wb;
}

// Budget of a level set: the largest of its levels' budgets.
WarpBudget set_warp_budget(const DevLevel *hl, int n, float margin) {
    WarpBudget q{1, 128};
    for (int l = 0; l < n; ++l)
        if (hl[l].n_nodes > 0) {
            const WarpBudget b = window_warp_budget(hl[l], margin);
            q.quads = std::max(q.quads, b.quads);
            q.raw = std::max(q.raw, b.raw);
        }
    return q;
}

int set_max_h(const DevLevel *hl, int n) {
    int h = 2;
    for (int l = 0; l < n; ++l)
        if (hl[l].n_nodes > 0) h = std::max(h, hl[l].H);
    return h;
}

int window_max_blocks_per_sm();
int64_t window_scratch_floats();
unsigned long long current_context_id();


cudaError_t launch_window(const DevLevel *hl, int n, const LevelSet &LS, const int32_t *node_k,
                          const double *gsum, const double *gcnt, float *pend_vals,
                          int64_t pend_cap, int64_t *pend_node, int64_t *pend_off,
                          int64_t *fix_list, int64_t fix_cap,
                          unsigned long long *counters, unsigned long long *ctl,
                          const SplitTuning &tu, cudaStream_t s) {
    const WarpBudget wb = set_warp_budget(hl, n, tu.box_margin);
    const size_t smem = win_raw_offset(wb.quads) + (size_t)kWinWarps * wb.raw;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaError_t e = ensure_smem_limit((const void *)window_kernel, smem);
    if (e != cudaSuccess) return e;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, window_kernel, kWinWarps * 32, smem);
    if (tu.blocks_per_sm > 0 && tu.blocks_per_sm < per_sm) per_sm = tu.blocks_per_sm;
    per_sm = std::max(1, std::min(per_sm, window_max_blocks_per_sm()));
    // nodes per queue access (their slot counts are read one per lane)
    const int grab = tu.grab > 0 ? std::min(tu.grab, 32) : 1;
    // the warps' slot scratch follows the pending buffer's pend_cap values
    // (window_scratch_floats sizes it for the largest grid)
    float *warp_vals = pend_vals + pend_cap;
    window_kernel<<<sms * per_sm, kWinWarps * 32, smem, s>>>(LS, node_k, gsum, gcnt, pend_vals,
                                                             pend_cap, pend_node, pend_off,
                                                             warp_vals, fix_list, fix_cap,
                                                             counters, ctl, wb.quads, wb.raw,
                                                             grab);
    return cudaGetLastError();
}

cudaError_t launch_peaks(const LevelSet &LS, int max_h, const int32_t *node_k,
                         const float *pend_vals, const int64_t *pend_node, const int64_t *pend_off,
                         const double *gsum, const double *gcnt, unsigned long long *counters,
                         unsigned long long *ctl, cudaStream_t s) {
    const size_t ws = (sizeof(WarpShared) + 15) & ~(size_t)15;
    const size_t xs = (exact_scratch_bytes(max_h) + 15) & ~(size_t)15;
    const size_t smem = (ws + xs) * kPeakWarps;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaError_t e = ensure_smem_limit((const void *)peaks_kernel, smem);
    if (e != cudaSuccess) return e;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, peaks_kernel, kPeakWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    peaks_kernel<<<sms * per_sm, kPeakWarps * 32, smem, s>>>(LS, max_h, node_k, pend_vals,
                                                             pend_node, pend_off, gsum, gcnt,
                                                             counters, ctl);
    return cudaGetLastError();
}

// the window and exact stages of the pipeline on given buffers (ctl cleared
// by the caller: [0] node queue, [1] exact-pass queue, [2] queued nodes,
// [4] pending-buffer cursor)
cudaError_t window_and_peaks(const DevLevel *hl, int n, const LevelSet &LS, const int32_t *node_k,
                             const double *gsum, const double *gcnt, float *pend_vals,
                             int64_t pend_cap, int64_t *pend_node, int64_t *pend_off,
                             int64_t fix_cap, unsigned long long *counters,
                             unsigned long long *ctl, const SplitTuning &tu, cudaStream_t s,
                             SplitTiming *tm) {
    // the voxel slots listed for an exact INCC follow the warps' scratch
    int64_t *fix_list = reinterpret_cast<int64_t *>(
        pend_vals + ((pend_cap + window_scratch_floats() + 1) & ~(int64_t)1));
    cudaError_t e = launch_window(hl, n, LS, node_k, gsum, gcnt, pend_vals, pend_cap, pend_node,
                                  pend_off, fix_list, fix_cap, counters, ctl, tu, s);
    if (e != cudaSuccess) return e;
    if (fix_cap > 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        slot_fix_kernel<<<sms * 8, 128, 0, s>>>(LS, fix_list, fix_cap, gsum, gcnt, ctl);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (tm && tm->enabled) {
        cudaEventRecord(tm->ev[5], s);
        cudaEventRecord(tm->ev[6], s);
    }
    return launch_peaks(LS, set_max_h(hl, n), node_k, pend_vals, pend_node, pend_off, gsum, gcnt,
                        counters, ctl, s);
}

// Most window-kernel CTAs an SM can hold whatever the footprint budget (its
// registers bound it; the launch never exceeds it).
int window_max_blocks_per_sm() {
    // computed once (thread-safe initialisation of a function-local static)
    static const int cached = [] {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, window_kernel, kWinWarps * 32,
                                                          win_boxes_offset()) != cudaSuccess ||
            b < 1)
            b = kWinMaxBlocksPerSm;
        return std::min(b, kWinMaxBlocksPerSm);
    }();
    return cached;
}

// Floats of per-warp slot scratch the window kernel needs after the pending
// buffer's values: kSlotCap per warp of the largest grid on this device.
int64_t window_scratch_floats() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int64_t)sms * window_max_blocks_per_sm() * kWinWarps * kSlotCap;
}

// Slots of FP32 values the pending buffer holds for a pass of n_slots slots:
// an eighth of them (a few percent of nodes are queued for the exact pass),
// at least 4 M; SETSM_VLL_PENDING_SLOTS overrides it (a node that finds the
// buffer full is evaluated wholly in FP64 instead).
int64_t pending_capacity(int64_t n_slots) {
    const char *env = getenv("SETSM_VLL_PENDING_SLOTS");
    if (env && *env) return std::max<int64_t>(0, atoll(env));
    return std::min<int64_t>(n_slots, std::max<int64_t>(n_slots / 8, (int64_t)1 << 22));
}

}  // namespace

// Raises `func`'s dynamic shared-memory limit to at least `bytes` in the
// calling thread's context and never lowers it.  The limit belongs to the
// function in the whole context, and contexts used from several threads
// launch the same kernel with different footprints: setting each launch's
// own size could lower the limit under another thread's larger launch
// (which then fails as an invalid argument).  Without a context id the
// limit is set for every launch, as a single thread needs.
cudaError_t ensure_smem_limit(const void *func, size_t bytes) {
    static std::mutex mu;
    struct Seen {
        const void *func;
        unsigned long long ctx;
        size_t bytes;
    };
    static std::vector<Seen> seen;
    const unsigned long long ctx = current_context_id();
    if (ctx == 0)
        return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    std::lock_guard<std::mutex> lk(mu);
    for (Seen &t : seen)
        if (t.func == func && t.ctx == ctx) {
            if (bytes <= t.bytes) return cudaSuccess;
            const cudaError_t e =
                cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e == cudaSuccess) t.bytes = bytes;
            return e;
        }
    const cudaError_t e =
        cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) seen.push_back(Seen{func, ctx, bytes});
    return e;
}

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

}  // namespace

void split_prepare_tma(DevLevel &P, float margin) {
    P.tma_w[0] = P.tma_w[1] = P.tma_h[0] = P.tma_h[1] = 0;
    EncodeTiledFn enc = encode_tiled();
    if (!enc || !split_supported(P) || P.combined_incc) return;
    const WindowBoxes B = window_boxes(P, margin);
    int tw[2], th[2];
    for (int ti = 0; ti < 2; ++ti) {
        const DevImage &im = P.im[ti == 0 ? P.ref : 1];
        // tiles need 16-byte aligned rows; the tile width covers the box's
        // pairs, their right texels and the rounding of x down to 8
        if (im.w % 8 || !im.img || !im.mag || (reinterpret_cast<uintptr_t>(im.img) & 15) ||
            (reinterpret_cast<uintptr_t>(im.mag) & 15))
            return;
        tw[ti] = (B.w[ti] + 1 + 7 + 7) & ~7;
        th[ti] = B.h[ti];
        if (tw[ti] > 256 || th[ti] > 256) return;
        for (int pl = 0; pl < 2; ++pl) {
            const cuuint64_t dims[2] = {im.w, im.h};
            const cuuint64_t strides[1] = {(cuuint64_t)im.w * 2};
            const cuuint32_t box[2] = {(cuuint32_t)tw[ti], (cuuint32_t)th[ti]};
            const cuuint32_t estr[2] = {1, 1};
            void *base = const_cast<uint16_t *>(pl == 0 ? im.img : im.mag);
            if (enc(reinterpret_cast<CUtensorMap *>(P.tmap[ti][pl]), CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                    base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return;
        }
    }
    for (int ti = 0; ti < 2; ++ti) {
        P.tma_w[ti] = tw[ti];
        P.tma_h[ti] = th[ti];
    }
}

bool split_supported(const DevLevel &P) {
    return P.num_images == 2 && P.ref == 0 && P.im[1].selected && !P.is_ra && P.H >= 2 &&
           P.H <= 7;
}

void split_release(SplitBuffers &b) {
    void **all[] = {&b.node_k, &b.slot_off, &b.rho, &b.gsum, &b.gcnt, &b.scan_tmp, &b.ctl,
                    &b.pending, &b.pend_off, &b.base, &b.acc_level};
    for (void **p : all) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    b.cap_nodes = b.cap_slots = b.cap_scan = b.cap_levels = 0;
    b.pend_cap = 0;
    b.fix_cap = 0;
}

#define SPLIT_CUDA(call)                       \
    do {                                       \
        cudaError_t e__ = (call);              \
        if (e__ != cudaSuccess) {              \
            *err = #call;                      \
            return e__;                        \
        }                                      \
    } while (0)

// Phase 1 of a pass over a level set: node-sized buffers, the level table,
// GNCC, prep and the prefix sum of the slot counts (all enqueued on s, no
// host wait).
cudaError_t split_front(SplitBuffers &b, const DevLevel *hl, const DevLevel *dl, int n_levels,
                        unsigned long long *counters, cudaStream_t s, std::string *err,
                        SplitTiming *tm, LevelSet *LS_out, double **gsum_out, double **gcnt_out,
                        int64_t *launches) {
    auto mark = [&](int i) {
        if (tm && tm->enabled) cudaEventRecord(tm->ev[i], s);
    };
    std::vector<int64_t> &base = b.h_base;
    base.assign((size_t)n_levels + 1, 0);
    bool any_ortho = false;
    for (int l = 0; l < n_levels; ++l) {
        base[l + 1] = base[l] + hl[l].n_nodes;
        any_ortho = any_ortho || hl[l].check_ortho;
    }
    const int64_t N = base[n_levels];
    if ((size_t)(N + 1) > b.cap_nodes) {
        if (b.node_k) cudaFree(b.node_k);
        b.node_k = nullptr;
        SPLIT_CUDA(cudaMalloc(&b.node_k, (size_t)(N + 1) * sizeof(int32_t)));
        void **nb8[] = {&b.slot_off, &b.gsum, &b.gcnt, &b.pending, &b.pend_off};
        for (void **p : nb8) {
            if (*p) cudaFree(*p);
            *p = nullptr;
            SPLIT_CUDA(cudaMalloc(p, (size_t)(N + 1) * 8));
        }
        b.cap_nodes = (size_t)(N + 1);
    }
    if ((size_t)n_levels + 1 > b.cap_levels) {
        if (b.base) cudaFree(b.base);
        if (b.acc_level) cudaFree(b.acc_level);
        b.base = b.acc_level = nullptr;
        SPLIT_CUDA(cudaMalloc(&b.base, ((size_t)n_levels + 1) * 8));
        SPLIT_CUDA(cudaMalloc(&b.acc_level, ((size_t)n_levels + 1) * 8));
        b.cap_levels = (size_t)n_levels + 1;
    }
    if (!b.ctl) SPLIT_CUDA(cudaMalloc(&b.ctl, 8 * sizeof(unsigned long long)));
    size_t tmp1 = 0;
    SPLIT_CUDA(scan64(nullptr, tmp1, (const int32_t *)b.node_k, (int64_t *)b.slot_off,
                      (int)(N + 1), s));
    SPLIT_CUDA(grow(b.scan_tmp, b.cap_scan, tmp1));
    // the level table is uploaded outside any capture (plan time) by the caller
    // of split_front when capturing; here it is copied on the stream
    if (!b.capturing)
        SPLIT_CUDA(cudaMemcpyAsync(b.base, base.data(), base.size() * 8, cudaMemcpyHostToDevice, s));
    SPLIT_CUDA(cudaMemsetAsync(b.acc_level, 0, ((size_t)n_levels + 1) * 8, s));
    *LS_out = LevelSet{dl, (const int64_t *)b.base, n_levels, N};
    SPLIT_CUDA(cudaMemsetAsync(b.ctl, 0, 8 * sizeof(unsigned long long), s));
    SPLIT_CUDA(cudaMemsetAsync(b.node_k, 0, (size_t)(N + 1) * sizeof(int32_t), s));
    double *gsum = nullptr, *gcnt = nullptr;
    mark(0);
    if (any_ortho) {
        gsum = (double *)b.gsum;
        gcnt = (double *)b.gcnt;
        for (int l = 0; l < n_levels; ++l) {
            if (!hl[l].check_ortho || hl[l].n_nodes == 0) continue;
            SPLIT_CUDA(launch_gncc(dl + l, hl[l].n_nodes, gsum + base[l], gcnt + base[l], s));
            ++*launches;
        }
    }
    mark(1);
    prep_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(*LS_out, gsum, gcnt, (int32_t *)b.node_k,
                                                          counters,
                                                          (unsigned long long *)b.acc_level);
    SPLIT_CUDA(cudaGetLastError());
    ++*launches;
    mark(2);
    tmp1 = b.cap_scan;
    SPLIT_CUDA(scan64(b.scan_tmp, tmp1, (const int32_t *)b.node_k, (int64_t *)b.slot_off,
                      (int)(N + 1), s));
    *launches += 2;   // one scan of two kernels
    mark(3);
    *gsum_out = gsum;
    *gcnt_out = gcnt;
    return cudaSuccess;
}

// Phase 2: the persistent window launch and the exact pass.
cudaError_t split_back(SplitBuffers &b, const DevLevel *hl, int n_levels, const LevelSet &LS,
                       const double *gsum, const double *gcnt, unsigned long long *counters,
                       const SplitTuning &tu, cudaStream_t s, std::string *err, SplitTiming *tm,
                       int64_t *launches) {
    auto mark = [&](int i) {
        if (tm && tm->enabled) cudaEventRecord(tm->ev[i], s);
    };
    mark(4);
    cudaError_t e = window_and_peaks(hl, n_levels, LS, (const int32_t *)b.node_k, gsum, gcnt,
                                     (float *)b.rho, b.pend_cap, (int64_t *)b.pending,
                                     (int64_t *)b.pend_off, b.fix_cap, counters,
                                     (unsigned long long *)b.ctl, tu, s, tm);
    if (e != cudaSuccess) {
        *err = "window / exact kernel launch";
        return e;
    }
    *launches += 2 + (b.fix_cap > 0 ? 1 : 0);
    mark(7);
    mark(8);
    return cudaSuccess;
}

// Whether a level of the set writes voxel rows (the voxel route).
bool voxel_route(const DevLevel *hl, int n) {
    for (int l = 0; l < n; ++l)
        if (hl[l].vox && !hl[l].cmr && !hl[l].is_ra) return true;
    return false;
}

// Sizes the pending buffer from the slot total of a completed front phase
// (one host wait).
cudaError_t split_size(SplitBuffers &b, int64_t N, cudaStream_t s, std::string *err,
                       int64_t *n_slots, bool voxel_route) {
    int64_t total = 0;
    SPLIT_CUDA(cudaMemcpyAsync(&total, (int64_t *)b.slot_off + N, 8, cudaMemcpyDeviceToHost, s));
    SPLIT_CUDA(cudaStreamSynchronize(s));
    *n_slots = total;
    if (total < 0) {
        *err = "slot total overflow";
        return cudaErrorInvalidValue;
    }
    const int64_t cap = pending_capacity(total);
    // voxel-route levels list the slots whose INCC truncation needs an exact
    // value (about 1 %; a slot that finds the list full goes to the exact pass)
    const int64_t fix = voxel_route ? std::min<int64_t>(total, std::max<int64_t>(total / 32, 1 << 20))
                                    : 0;
    size_t c = b.cap_slots;
    SPLIT_CUDA(grow(b.rho, c,
                    (size_t)(((cap + window_scratch_floats() + 1) & ~(int64_t)1) + 2 * fix) *
                        sizeof(float)));
    b.cap_slots = c;
    b.pend_cap = cap;
    b.fix_cap = fix;
    return cudaSuccess;
}

cudaError_t run_split_set(SplitBuffers &b, const DevLevel *hl, const DevLevel *dl, int n_levels,
                          unsigned long long *counters, cudaStream_t s, std::string *err,
                          SplitTiming *tm, const SplitTuning &tu) {
    int64_t launches = 0;
    LevelSet LS;
    double *gsum = nullptr, *gcnt = nullptr;
    b.capturing = false;
    cudaError_t e = split_front(b, hl, dl, n_levels, counters, s, err, tm, &LS, &gsum, &gcnt,
                                &launches);
    if (e != cudaSuccess) return e;
    int64_t n_slots = 0;
    e = split_size(b, LS.total, s, err, &n_slots, voxel_route(hl, n_levels));
    if (e != cudaSuccess) return e;
    e = split_back(b, hl, n_levels, LS, gsum, gcnt, counters, tu, s, err, tm, &launches);
    if (e != cudaSuccess) return e;
    if (tm) {
        tm->slots = n_slots;
        tm->launches = launches;
    }
    return cudaSuccess;
}

// Planned pass: sizes the buffers with one uncaptured front phase, then
// captures front + back into a CUDA graph that later replays with no host
// wait.  The buffers depend on the node count only (the pending buffer's
// size steers performance, not correctness), so replays stay valid when the
// levels' height ranges change.
cudaError_t split_plan(SplitPlan &pl, SplitBuffers &b, const DevLevel *hl, const DevLevel *dl,
                       int n_levels, unsigned long long *counters, cudaStream_t s,
                       std::string *err, const SplitTuning &tu,
                       const std::function<cudaError_t(cudaStream_t)> &pre) {
    int64_t launches = 0;
    LevelSet LS;
    double *gsum = nullptr, *gcnt = nullptr;
    b.capturing = false;
    cudaError_t e = pre ? pre(s) : cudaSuccess;
    if (e != cudaSuccess) {
        *err = "orthoimage rasters";
        return e;
    }
    e = split_front(b, hl, dl, n_levels, counters, s, err, nullptr, &LS, &gsum, &gcnt,
                                &launches);
    if (e != cudaSuccess) return e;
    e = split_size(b, LS.total, s, err, &pl.n_slots, voxel_route(hl, n_levels));
    if (e != cudaSuccess) return e;
    if (pl.exec) {
        cudaGraphExecDestroy(pl.exec);
        pl.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    b.capturing = true;
    SPLIT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    launches = 0;
    e = pre ? pre(s) : cudaSuccess;
    if (e == cudaSuccess)
        e = split_front(b, hl, dl, n_levels, counters, s, err, nullptr, &LS, &gsum, &gcnt,
                        &launches);
    if (e == cudaSuccess)
        e = split_back(b, hl, n_levels, LS, gsum, gcnt, counters, tu, s, err, nullptr, &launches);
    cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    b.capturing = false;
    if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return e;
    }
    if (e2 != cudaSuccess) {
        *err = "cudaStreamEndCapture";
        return e2;
    }
    e = cudaGraphInstantiate(&pl.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        *err = "cudaGraphInstantiate";
        return e;
    }
    pl.launches = launches;
    return cudaSuccess;
}

cudaError_t run_split(SplitBuffers &b, const DevLevel &P, const DevLevel *dP,
                      unsigned long long *counters, cudaStream_t s, std::string *err,
                      SplitTiming *tm, const SplitTuning &tu) {
    return run_split_set(b, &P, dP, 1, counters, s, err, tm, tu);
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
unsigned long long g_noalloc_ctx[256] = {};

// Unique id of the calling thread's current context (0 when unknown),
// through the driver entry points (no link against the driver library).
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    struct Fns {
        GetCurrent get_current = nullptr;
        GetId get_id = nullptr;
    };
    // looked up once; the initialisation of a function-local static is
    // thread-safe (callers run on several host threads)
    static const Fns fns = [] {
        Fns f;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f.get_current = (GetCurrent)p;
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f.get_id = (GetId)p;
        return f;
    }();
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (fns.get_current && fns.get_id && fns.get_current(&c) == CUDA_SUCCESS && c)
        fns.get_id(c, &id);
    return id;
}

// Device address of the scratch array for the current device: looked up
// (cudaGetSymbolAddress, host code cannot use the symbol's address) on the
// first call on a device, and again when the device's context changed.
cudaError_t noalloc_scratch(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    // 0 when this thread has no current context yet (the lookup makes the
    // device's primary context current)
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
        g_noalloc_ctx[dev] = current_context_id();
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
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
    if (const cudaError_t se = noalloc_scratch(&base); se != cudaSuccess) {
        char m[200];
        snprintf(m, sizeof m, "device address of the %zu MiB scratch array: %s",
                 kNoAllocScratchBytes >> 20, cudaGetErrorString(se));
        return fail(VLL_ERR_CUDA, m);
    }
    const int64_t N = P.n_nodes;
    Carver cv{(unsigned char *)base, 0, kNoAllocScratchBytes};
    DevLevel *dP = (DevLevel *)cv.take(sizeof(DevLevel));
    unsigned long long *ctl = (unsigned long long *)cv.take(8 * sizeof(unsigned long long));
    unsigned long long *counters = (unsigned long long *)cv.take(8 * sizeof(unsigned long long));
    int32_t *node_k = (int32_t *)cv.take((size_t)(N + 1) * 4);
    int64_t *pending = (int64_t *)cv.take((size_t)(N + 1) * 8);
    int64_t *pend_off = (int64_t *)cv.take((size_t)(N + 1) * 8);
    int64_t *lbase = (int64_t *)cv.take(2 * 8);
    unsigned long long *acc_level = (unsigned long long *)cv.take(2 * 8);
    if (!dP || !ctl || !counters || !node_k || !pending || !pend_off || !lbase || !acc_level) {
        char m[160];
        snprintf(m, sizeof m, "grid of %lld nodes exceeds the %zu MiB scratch array",
                 (long long)N, kNoAllocScratchBytes >> 20);
        return fail(VLL_ERR_CAPACITY, m);
    }
    // the rest of the array holds the FP32 slot values of the nodes queued
    // for the exact pass; a node that finds it full is evaluated wholly in
    // FP64 there, so its size affects speed only
    const size_t used = (cv.used + 255) & ~(size_t)255;
    float *pend_vals = (float *)((unsigned char *)base + used);
    // ... after the window kernel's per-warp slot scratch is set aside
    const int64_t pend_cap = (int64_t)((kNoAllocScratchBytes - used) / sizeof(float)) -
                             window_scratch_floats();
    if (pend_cap < 0) {
        char m[160];
        snprintf(m, sizeof m, "grid of %lld nodes exceeds the %zu MiB scratch array",
                 (long long)N, kNoAllocScratchBytes >> 20);
        return fail(VLL_ERR_CAPACITY, m);
    }
#define NA_CUDA(call)                                                     \
    do {                                                                  \
        if ((call) != cudaSuccess) return fail(VLL_ERR_CUDA, #call);      \
    } while (0)
    split_prepare_tma(P, SplitTuning().box_margin);
    NA_CUDA(cudaMemcpyAsync(dP, &P, sizeof(DevLevel), cudaMemcpyHostToDevice, s));
    // the array keeps the previous call's contents: clear what must start at zero
    NA_CUDA(cudaMemsetAsync(ctl, 0, 8 * sizeof(unsigned long long), s));
    NA_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), s));
    NA_CUDA(cudaMemsetAsync(acc_level, 0, 2 * 8, s));
    static thread_local int64_t lbase_host[2];
    lbase_host[0] = 0;
    lbase_host[1] = N;
    NA_CUDA(cudaMemcpyAsync(lbase, lbase_host, sizeof(lbase_host), cudaMemcpyHostToDevice, s));
    const LevelSet LS{dP, lbase, 1, N};
    NA_CUDA(cudaMemsetAsync(node_k, 0, (size_t)(N + 1) * 4, s));
    // the pipeline proper (same kernels and order as run_split)
    prep_kernel<<<grid_1d(N, 256, 148 * 32), 256, 0, s>>>(LS, nullptr, nullptr, node_k, counters,
                                                          acc_level);
    NA_CUDA(cudaGetLastError());
    NA_CUDA(window_and_peaks(&P, 1, LS, node_k, nullptr, nullptr, pend_vals, pend_cap, pending,
                             pend_off, 0, counters, ctl, SplitTuning(), s, nullptr));
    unsigned long long acc = 0;
    NA_CUDA(cudaMemcpyAsync(&acc, counters, sizeof(acc), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
#undef NA_CUDA
    if (accessable_grid) *accessable_grid = (int64_t)acc;
    return VLL_OK;
}

#ifdef VLL_PHASE_CYCLES
// The window kernel's phase totals of the instrumented build (see
// VLL_PHASE_CYCLES): out[0..6] warp cycles per phase, out[8] groups,
// out[9] nodes, summed over the launches since the last reset.
extern "C" int vll_window_phase_cycles(unsigned long long *out, int reset) {
    if (out && cudaMemcpyFromSymbol(out, vll::g_phase_cycles, 16 * sizeof(unsigned long long)) !=
                   cudaSuccess)
        return -1;
    if (reset) {
        static const unsigned long long zero[16] = {};
        if (cudaMemcpyToSymbol(vll::g_phase_cycles, zero, sizeof zero) != cudaSuccess) return -1;
    }
    return 0;
}
#endif

// vll_tinblunder.cu -- blunder_detection_TIN (setsm_code.cpp:9158-9787): the
// matched points whose TIN neighbourhood is inconsistent in height are marked
// as blunders.
//
// The reference runs three passes: statistics over the triangles in order
// (per point its first 30 triangles; FP64 sums of the vertices' ortho NCC and
// of the edges' height differences; a histogram of the differences), the
// thresholds from them, and a parallel pass over the points in which a point
// may mark itself (flag 1) or a neighbour (flag 3).  Its marks race only on
// which of 1 / 3 lands first on a point that was 0 (set_blunder, :9121); the
// closing pass turns 3 into 1, so the outputs do not depend on the race.
//
// GPU: the per-triangle terms in parallel (height differences, histogram,
// per-point triangle counts), the two FP64 sums in parallel with a proven
// bound on their distance from the reference's sequential sums (the height
// threshold is then known to lie in a band; a point pass in which some
// comparison falls inside the band is undone and run again with the sums in
// the reference's order), the per-point triangle lists by counting and a
// fill, the point pass one warp per point (lane k takes the point's k-th
// triangle in triangle order, after a warp sort) with the same
// compare-and-swap marking, and the closing pass with warp-aggregated atomics
// (order-free counts, min / max).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "vll_ddmath.cuh"
#include "vll_device.cuh"
#include "vll_internal.h"

namespace vll {

namespace {

constexpr int kMaxNodes = 30;   // max_nodes (:9168)

__device__ __forceinline__ int64_t grid_index(const TinArgs &a, double x, double y) {
    const int64_t c = (int64_t)__dadd_rn(__ddiv_rn(__dadd_rn(x, -a.b0), a.gs), 0.5);
    const int64_t r = (int64_t)__dadd_rn(__ddiv_rn(__dadd_rn(y, -a.b1), a.gs), 0.5);
    return a.width * r + c;
}

// Per triangle: its three edge height differences (+0 for a triangle with a
// vertex past the points, which adds nothing to the sums of non-negative
// terms: s + 0 == s for every s those sums take), the count of valid
// triangles and the histogram of the differences (order-free), and the check
// that every vertex's grid node lies in the grid.  The vertices' ortho NCC
// statistics of the reference (:9200-9252) feed only an ortho-NCC threshold
// that it overwrites with the level's constant (:9304-9313), so they are not
// formed.
constexpr int kSmemBins = 2048;   // histogram bins kept in shared memory

__global__ void __launch_bounds__(256)
    tri_terms_kernel(TinArgs a, const vll_point3 *pts, const vll_tri *tris, double *dhv,
                     uint32_t *hbin, uint32_t hdiffcount, unsigned long long *n_valid,
                     unsigned int *count, unsigned int *bad) {
    __shared__ uint32_t sh[kSmemBins];
    const bool use_sh = hdiffcount <= (uint32_t)kSmemBins;
    if (use_sh)
        for (uint32_t i = threadIdx.x; i < hdiffcount; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    unsigned int nv = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < a.n_tris;
         t += (int64_t)gridDim.x * blockDim.x) {
        const vll_tri tr = tris[t];
        const uint32_t v[3] = {tr.a, tr.b, tr.c};
        bool valid = true;
        double z[3];
        for (int k = 0; k < 3; ++k) {
            if (v[k] < (uint64_t)a.n_pts) {
                atomicAdd(count + v[k], 1u);
                const vll_point3 p = pts[v[k]];
                z[k] = p.z;
                // int t_col / t_row and an int index, as the reference
                const int tc = (int)__dadd_rn(__ddiv_rn(__dadd_rn(p.x, -a.b0), a.gs), 0.5);
                const int trw = (int)__dadd_rn(__ddiv_rn(__dadd_rn(p.y, -a.b1), a.gs), 0.5);
                const int idx = (int)((unsigned)a.width * (unsigned)trw + (unsigned)tc);
                if (idx < 0 || (int64_t)idx >= a.n_nodes) atomicExch(bad, 1u);
            } else {
                valid = false;
            }
        }
        double dh[3] = {0.0, 0.0, 0.0};
        if (valid) {
            dh[0] = fabs(__dadd_rn(z[0], -z[1]));
            dh[1] = fabs(__dadd_rn(z[0], -z[2]));
            dh[2] = fabs(__dadd_rn(z[1], -z[2]));
            for (int k = 0; k < 3; ++k) {
                const double f = (double)(uint32_t)dh[k];
                if (f < (double)hdiffcount) {
                    if (use_sh)
                        atomicAdd(sh + (uint32_t)f, 1u);
                    else
                        atomicAdd(hbin + (uint32_t)f, 1u);
                }
            }
            ++nv;
        }
        for (int k = 0; k < 3; ++k) dhv[3 * t + k] = dh[k];
    }
    nv = __reduce_add_sync(0xffffffffu, nv);
    if ((threadIdx.x & 31) == 0 && nv) atomicAdd(n_valid, (unsigned long long)nv);
    if (use_sh) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < hdiffcount; i += blockDim.x)
            if (sh[i]) atomicAdd(hbin + i, sh[i]);
    }
}

// The sums of the differences and of their squares in any order (sums[0],
// sums[1], zeroed before): a grid-stride pass, warp and block reduction, one
// atomic add per block.  Any summation order of m non-negative terms lies
// within (m-1) u (1 + O(u)) of the exact sum, as does the reference's
// sequential order; the thresholds take the band that follows.
__global__ void dh_psum_kernel(int64_t n_vals, const double *__restrict__ dhv, double *sums) {
    double s = 0, s2 = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_vals;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v = dhv[i];
        s = __dadd_rn(s, v);
        s2 = __dadd_rn(s2, __dmul_rn(v, v));
    }
    for (int o = 16; o > 0; o >>= 1) {
        s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
        s2 = __dadd_rn(s2, __shfl_down_sync(0xffffffffu, s2, o));
    }
    __shared__ double part[2][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        part[0][w] = s;
        part[1][w] = s2;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        s = lane < nw ? part[0][lane] : 0.0;
        s2 = lane < nw ? part[1][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
            s2 = __dadd_rn(s2, __shfl_down_sync(0xffffffffu, s2, o));
        }
        if (lane == 0) {
            atomicAdd(sums, s);
            atomicAdd(sums + 1, s2);
        }
    }
}

// The reference's sums in its order (triangle by triangle, three edges each,
// :9257-9273) into sums[0], sums[1]: the block stages 2048 terms and their
// squares in shared memory, one thread adds them in sequence, so the running
// sums round as the reference's do.  A dependent FP64 add takes about 4 ns
// here, so this is the slow path (the band's re-run).
constexpr int kSerialChunk = 2048;
__global__ void __launch_bounds__(512) dh_serial_sum_kernel(int64_t n_vals,
                                                            const double *__restrict__ dhv,
                                                            double *sums) {
    __shared__ double val[kSerialChunk], sq[kSerialChunk];
    double sd = 0, sd2 = 0;
    for (int64_t base = 0; base < n_vals; base += kSerialChunk) {
        for (int i = threadIdx.x; i < kSerialChunk; i += blockDim.x) {
            const double v = base + i < n_vals ? dhv[base + i] : 0.0;
            val[i] = v;
            sq[i] = __dmul_rn(v, v);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll 16
            for (int i = 0; i < kSerialChunk; ++i) {
                sd = __dadd_rn(sd, val[i]);
                sd2 = __dadd_rn(sd2, sq[i]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[0] = sd;
        sums[1] = sd2;
    }
}

// The per-point triangle lists (the reference's savenode, :9190-9241): each
// point's slots [start, start + count) take its triangles in arbitrary order
// (the point pass orders them); a triangle listing a point twice is kept
// twice, as there.
__global__ void fill_kernel(TinArgs a, const vll_tri *tris, const int64_t *start,
                            unsigned int *cursor, int32_t *list) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < a.n_tris;
         t += (int64_t)gridDim.x * blockDim.x) {
        const vll_tri tr = tris[t];
        const uint32_t v[3] = {tr.a, tr.b, tr.c};
        for (int k = 0; k < 3; ++k)
            if (v[k] < (uint64_t)a.n_pts) list[start[v[k]] + atomicAdd(cursor + v[k], 1u)] = (int32_t)t;
    }
}

// Ascending bitonic sort of one value per lane across the warp.
__device__ __forceinline__ uint32_t warp_sort32(uint32_t v, int lane) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
            v = keep_min ? min(v, o) : max(v, o);
        }
    }
    return v;
}

// Lane k's triangle: the k-th smallest of the point's e list entries (with
// multiplicity), for k < n_take <= 30; 0xffffffff on the other lanes.
__device__ uint32_t lane_triangle(const int32_t *list, int64_t st, unsigned int e, int n_take,
                                  int lane) {
    uint32_t mine = 0xffffffffu;
    if (e <= 32) {
        mine = warp_sort32(lane < (int)e ? (uint32_t)list[st + lane] : 0xffffffffu, lane);
    } else {
        // a point of more than 32 triangles: select the smallest n_take by
        // (triangle, slot) keys, one per round
        unsigned long long last = 0;
        for (int k = 0; k < n_take; ++k) {
            unsigned long long best = ~0ull;
            for (unsigned int j = lane; j < e; j += 32) {
                const unsigned long long key =
                    ((unsigned long long)(uint32_t)list[st + j] << 32) | j;
                if ((k == 0 || key > last) && key < best) best = key;
            }
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
                if (x < best) best = x;
            }
            if (lane == k) mine = (uint32_t)(best >> 32);
            last = best;
        }
    }
    return lane < n_take ? mine : 0xffffffffu;
}

// set_blunder (:9121-9156): a point that is still 0 takes `val`; the call
// that changed it from 0 records the new blunder.
__device__ void set_blunder(vll_point3 *pts, int64_t i, uint8_t val, uint8_t *detected) {
    unsigned int *word = reinterpret_cast<unsigned int *>(
        reinterpret_cast<unsigned char *>(pts + i) + 24);   // flag's 4-byte word
    unsigned int old = *reinterpret_cast<volatile unsigned int *>(word);
    for (;;) {
        if ((old & 0xffu) != 0) return;
        const unsigned int nw = (old & ~0xffu) | val;
        const unsigned int got = atomicCAS(word, old, nw);
        if (got == old) break;
        old = got;
    }
    detected[i] = 1;
}

__device__ double normal_angle(const vll_point3 &p0, const vll_point3 &p1, const vll_point3 &p2) {
    const double ux = __dadd_rn(p1.x, -p0.x), uy = __dadd_rn(p1.y, -p0.y), uz = __dadd_rn(p1.z, -p0.z);
    const double vx = __dadd_rn(p2.x, -p0.x), vy = __dadd_rn(p2.y, -p0.y), vz = __dadd_rn(p2.z, -p0.z);
    const double nx = __dadd_rn(__dmul_rn(uy, vz), -__dmul_rn(vy, uz));
    const double ny = -__dadd_rn(__dmul_rn(ux, vz), -__dmul_rn(vx, uz));
    const double nz = __dadd_rn(__dmul_rn(ux, vy), -__dmul_rn(vx, uy));
    const double norm =
        sqrt(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)), __dmul_rn(nz, nz)));
    // a vertical-free triangle of a TIN has norm > 0; the reference leaves the
    // angle unset otherwise
    double angle = 0;
    if (norm != 0)
        angle = __ddiv_rn(__dmul_rn(ddm::acos_cr(__ddiv_rn(fabs(nz), norm)), 180.0), kPi);
    if (angle <= 0 && angle >= -90)
        angle = fabs(angle);
    else if (angle <= -270 && angle >= -360)
        angle = __dadd_rn(360.0, angle);
    else if (angle >= 270 && angle <= 360)
        angle = __dadd_rn(360.0, -angle);
    return angle;
}

// normal_angle(p0, p1, p2) > 30, the only use the point pass makes of the
// angle: CUDA's acos (within a few ulp, the CUDA Math API's bound) decides it
// unless the angle lies within 1e-9 degrees of 30 (an ulp of 30 is 3.6e-15),
// where the correctly rounded angle does.
__device__ bool angle_above_30(const vll_point3 &p0, const vll_point3 &p1, const vll_point3 &p2) {
    const double ux = __dadd_rn(p1.x, -p0.x), uy = __dadd_rn(p1.y, -p0.y), uz = __dadd_rn(p1.z, -p0.z);
    const double vx = __dadd_rn(p2.x, -p0.x), vy = __dadd_rn(p2.y, -p0.y), vz = __dadd_rn(p2.z, -p0.z);
    const double nx = __dadd_rn(__dmul_rn(uy, vz), -__dmul_rn(vy, uz));
    const double ny = -__dadd_rn(__dmul_rn(ux, vz), -__dmul_rn(vx, uz));
    const double nz = __dadd_rn(__dmul_rn(ux, vy), -__dmul_rn(vx, uy));
    const double norm =
        sqrt(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)), __dmul_rn(nz, nz)));
    if (norm == 0) return false;   // the angle normal_angle gives, 0
    const double fast = __ddiv_rn(__dmul_rn(acos(__ddiv_rn(fabs(nz), norm)), 180.0), kPi);
    if (!(fabs(__dadd_rn(fast, -30.0)) <= 1e-9)) return fast > 30;   // NaN: false either way
    return normal_angle(p0, p1, p2) > 30;
}

// x > the reference's height threshold, which lies in [height_th,
// height_th_hi]: when the two ends disagree the answer is not known and the
// pass is marked for an exact re-run.
__device__ __forceinline__ bool above_th(double x, const TinArgs &a, unsigned int *rerun) {
    const bool hi = x > a.height_th_hi;
    if (hi != (x > a.height_th)) *rerun = 1u;
    return hi;
}

// The point pass (:9426-9756), one warp per point: lane k evaluates the
// point's k-th triangle (the reference's loop iterations are independent but
// for the counts, which the warp adds up, and the marks, which are
// compare-and-swaps either way).
__global__ void __launch_bounds__(256)
    point_kernel(TinArgs a, vll_point3 *pts, const vll_tri *tris, const float *ortho_ncc,
                 const int32_t *list, const int64_t *start, const unsigned int *count,
                 vll_ugrid *gp3, uint8_t *detected, const uint8_t *flag0, unsigned int *bad,
                 unsigned int *rerun, int64_t *anchor_node, uint8_t *anchor_val,
                 const double *th) {
    if (*bad) return;   // a triangle's vertex outside the grid: the call fails
    a.height_th = th[0];
    a.height_th_hi = th[1];
    a.ortho_ncc_th = th[2];
    a.th_ref_ncc = th[3];
    const int lane = threadIdx.x & 31;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t index = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; index < a.n_pts;
         index += n_warps) {
        if (anchor_node && lane == 0) anchor_node[index] = -1;
        if (flag0[index] == 1) continue;
        bool pt_is_blunder = false;
        const unsigned int e = count[index];
        const int max_iter = e < (unsigned)kMaxNodes ? (int)e : kMaxNodes;
        const vll_point3 rp = pts[index];
        const int64_t ref_index = grid_index(a, rp.x, rp.y);
        if (ref_index < 0 || ref_index >= a.n_nodes) {
            if (lane == 0) atomicExch(bad, 1u);
            continue;
        }
        const float ref_oncc = ortho_ncc[ref_index];
        if (!a.is_ra && ref_oncc < a.th_ref_ncc && a.L >= 2) pt_is_blunder = true;
        const uint8_t anchor =
            (a.L >= 3 && a.iteration >= 4 && ref_oncc >= 0.95 && a.flag_blunder) ? 1 : 0;
        if (lane == 0) {
            if (anchor_node) {
                anchor_node[index] = ref_index;
                anchor_val[index] = anchor;
            } else {
                gp3[ref_index].anchor_flag = anchor;
            }
        }
        const uint32_t tcu = lane_triangle(list, start[index], e, max_iter, lane);
        bool counted = false, pos = false, neg = false, neigh = false;
        // triangle 0 is never used here, as in the reference (savenode > 0)
        if (lane < max_iter && tcu < (uint64_t)a.n_tris && tcu > 0) {
            const int64_t tc = tcu;
            const vll_tri tr = tris[tc];
            const uint32_t tt[3] = {tr.a, tr.b, tr.c};
            int64_t reference_index = 0, t0 = 0, t1 = 0;
            bool check_index = false;
            for (int kk = 0; kk < 3; ++kk) {
                if (tt[kk] == (uint64_t)index)
                    reference_index = index;
                else if (!check_index) {
                    t0 = tt[kk];
                    check_index = true;
                } else {
                    t1 = tt[kk];
                }
            }
            if (reference_index < a.n_pts && t0 < a.n_pts && t1 < a.n_pts) {
                counted = true;
                const vll_point3 p0 = pts[reference_index], p1 = pts[t0], p2 = pts[t1];
                const double dh1 = __dadd_rn(p0.z, -p1.z), dh2 = __dadd_rn(p0.z, -p2.z),
                             dh3 = __dadd_rn(p1.z, -p2.z);
                // the angle only counts when both differences have one sign
                if ((dh1 >= 0 && dh2 >= 0) || (dh1 < 0 && dh2 < 0)) {
                    const bool steep = angle_above_30(p0, p1, p2);
                    pos = dh1 >= 0 && dh2 >= 0 && steep;
                    neg = dh1 < 0 && dh2 < 0 && steep;
                }
                bool check_match = false;
                if (a.L > 1)
                    check_match = true;
                else if (a.L == 1)
                    check_match = a.iteration == 1 && a.count_bl <= 5;
                else if (a.L == 0) {
                    if (a.iteration == 1 && a.count_bl <= 5)
                        check_match = true;
                    else if (a.iteration == 2 && a.count_bl <= 5)
                        check_match = false;
                }
                if (check_match) {
                    const double d1 = __dadd_rn(fabs(dh1), -fabs(dh2));
                    const double d2 = __dadd_rn(fabs(dh1), -fabs(dh3));
                    const double d3 = __dadd_rn(fabs(dh2), -fabs(dh3));
                    if (above_th(fabs(d1), a, rerun) || above_th(fabs(d2), a, rerun) ||
                        above_th(fabs(d3), a, rerun)) {
                        const int64_t order[3] = {reference_index, t0, t1};
                        const double h[3] = {p0.z, p1.z, p2.z};
                        const int64_t Index[3] = {grid_index(a, p0.x, p0.y), grid_index(a, p1.x, p1.y),
                                                  grid_index(a, p2.x, p2.y)};
                        neigh = true;
                        int mx, mn, md;
                        if (h[0] > h[1]) {
                            if (h[0] > h[2]) {
                                mx = 0;
                                if (h[1] > h[2]) {
                                    mn = 2;
                                    md = 1;
                                } else {
                                    mn = 1;
                                    md = 2;
                                }
                            } else {
                                mx = 2;
                                mn = 1;
                                md = 0;
                            }
                        } else {
                            if (h[1] > h[2]) {
                                mx = 1;
                                if (h[0] > h[2]) {
                                    mn = 2;
                                    md = 0;
                                } else {
                                    mn = 0;
                                    md = 2;
                                }
                            } else {
                                mx = 2;
                                md = 1;
                                mn = 0;
                            }
                        }
                        const double h1 = __dadd_rn(h[md], -h[mn]);
                        const double h2 = __dadd_rn(h[mx], -h[md]);
                        const double dh = __dadd_rn(h1, -h2);
                        int64_t bn = -1;
                        int pick = -1;
                        if (dh > 0 && above_th(dh, a, rerun))
                            pick = mn;
                        else if (dh < 0 && above_th(fabs(dh), a, rerun))
                            pick = mx;
                        if (pick >= 0) {
                            if (a.is_ra) {
                                bn = order[pick];
                            } else {
                                const int64_t gi = Index[pick];
                                if (gi < 0 || gi >= a.n_nodes) {
                                    atomicExch(bad, 1u);
                                } else {
                                    const double th = a.flag_blunder ? a.ortho_ncc_th : 100.0;
                                    if (ortho_ncc[gi] < th) bn = order[pick];
                                }
                            }
                        }
                        if (bn >= 0) set_blunder(pts, bn, 3, detected);
                    }
                }
            }
        }
        const int cnt = __popc(__ballot_sync(0xffffffffu, counted));
        const int count_pos = __popc(__ballot_sync(0xffffffffu, pos));
        const int count_neg = __popc(__ballot_sync(0xffffffffu, neg));
        const bool check_neigh = __ballot_sync(0xffffffffu, neigh) != 0;
        if (a.is_ra) {
            if (check_neigh && !a.flag_blunder) pt_is_blunder = true;
            if ((count_pos >= (int)__dadd_rn(__dmul_rn((double)cnt, 0.7), 0.5) ||
                 count_neg >= (int)__dadd_rn(__dmul_rn((double)cnt, 0.7), 0.5)) &&
                cnt > 1)
                pt_is_blunder = true;
        } else {
            if (check_neigh && !a.flag_blunder) {
                if (ref_oncc < 100.0) pt_is_blunder = true;
            }
            double cth = __dmul_rn((double)cnt, 0.5);
            if (a.L >= 2)
                cth = __dmul_rn((double)cnt, 0.5);
            else if (a.L == 1)
                cth = (double)(int)__dadd_rn(__dmul_rn((double)cnt, 0.6), 0.5);
            else
                cth = (double)(int)__dadd_rn(__dmul_rn((double)cnt, 0.7), 0.5);
            if ((count_pos >= cth || count_neg >= cth) && cnt > 1) {
                if (a.flag_blunder) {
                    double tmp = __dadd_rn(0.6, -__dmul_rn((double)(4 - a.L), 0.1));
                    if (a.L == 1) tmp = 0.6;
                    if (a.L >= 1) {
                        if (ref_oncc < tmp) pt_is_blunder = true;
                    } else {
                        if (a.iteration <= 1) {
                            if (ref_oncc < 0.9) pt_is_blunder = true;
                        } else if (a.iteration == 2) {
                            pt_is_blunder = true;
                        } else if (ref_oncc < a.ortho_ncc_th) {
                            pt_is_blunder = true;
                        }
                    }
                } else if (ref_oncc < 100.0) {
                    pt_is_blunder = true;
                }
            }
        }
        if (pt_is_blunder && lane == 0) set_blunder(pts, index, 1, detected);
    }
}

__device__ __forceinline__ unsigned long long dkey(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// The closing pass (:9765-9781): blunder counts, 3 -> 1, the height extent
// of the remaining points.
__global__ void close_kernel(int64_t n_pts, vll_point3 *pts, unsigned long long *cnt,
                             unsigned long long *zkey, const unsigned int *rerun,
                             const unsigned int *bad) {
    if (*rerun || *bad) return;   // the point pass runs again first, or the call fails
    unsigned long long kept = 0, blunders = 0, zmin = ~0ull, zmax = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pts;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t f = pts[i].flag;
        if (f == 1) {
            ++blunders;
        } else if (f == 3) {
            ++blunders;
            pts[i].flag = 1;
        } else {
            ++kept;
            const unsigned long long k = dkey(pts[i].z);
            zmin = k < zmin ? k : zmin;
            zmax = k > zmax ? k : zmax;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        kept += __shfl_xor_sync(0xffffffffu, kept, o);
        blunders += __shfl_xor_sync(0xffffffffu, blunders, o);
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, zmin, o);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, zmax, o);
        zmin = a < zmin ? a : zmin;
        zmax = b > zmax ? b : zmax;
    }
    if ((threadIdx.x & 31) == 0) {
        if (blunders) atomicAdd(cnt + 1, blunders);
        if (kept) {
            atomicAdd(cnt, kept);
            atomicMax(zkey, ~zmin);   // the minimum as the maximum complement: 0 starts both
            atomicMax(zkey + 1, zmax);
        }
    }
}

// Snapshot of the point flags and the new-blunder marks before the point
// pass, and its undoing before a re-run (the pass's UGRID writes do not
// depend on the height threshold and are simply repeated).
__global__ void copy_flags_kernel(int64_t n, const vll_point3 *pts, uint8_t *flag0,
                                  const uint8_t *det, uint8_t *det0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        flag0[i] = pts[i].flag;
        det0[i] = det[i];
    }
}

__global__ void restore_flags_kernel(int64_t n, vll_point3 *pts, const uint8_t *flag0,
                                     uint8_t *det, const uint8_t *det0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        pts[i].flag = flag0[i];
        det[i] = det0[i];
    }
}

unsigned blocks_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

size_t scan_tmp_bytes(int64_t n) {
    size_t u = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, u, (const unsigned int *)nullptr, (int64_t *)nullptr,
                                  (int)n);
    return u;
}

}  // namespace

namespace {

// The reference's height threshold as a function of up_3sigma (:9362-9418):
// clamp(up, H/2, H) from level 3 on, min(up, th80, 50) below; a NaN up
// compares false, as +inf would.  Non-decreasing in up.
__host__ __device__ double height_th_of(bool ge3, double H, uint32_t th80, double up) {
    if (ge3) {
        double h = H;
        if (up < h) h = up < h / 2.0 ? h / 2.0 : up;
        return h;
    }
    double h = up < th80 ? up : (double)th80;
    if (h > 50) h = 50;
    return h;
}

// The thresholds of the level from the sums' bounds (sd, sd2: [lo, hi]),
// their count and th80, the 99th-percentile bin of the height differences
// (used below level 3); host and device share it.
__host__ __device__ void thresholds_of(const TinArgs &a, const double sd[2], const double sd2[2],
                                       long dh_count, uint32_t th80, TinThresholds *th) {
    const int L = a.L, it = a.iteration;
    // the ortho-NCC threshold of the level (:9304-9313; the statistics-based
    // value computed before it is overwritten there)
    double ortho_ncc_th;
    if (L == 4)
        ortho_ncc_th = 0.6 - (it - 1) * 0.01;
    else if (L >= 3)
        ortho_ncc_th = 0.5 - (it - 1) * 0.01;
    else if (L == 2)
        ortho_ncc_th = 0.4 - (it - 1) * 0.01;
    else if (L == 1)
        ortho_ncc_th = 0.3;
    else
        ortho_ncc_th = 0.2;
    double th_ref_ncc = 0.1 + (it - 1) * 0.05;
    if (th_ref_ncc > ortho_ncc_th) th_ref_ncc = ortho_ncc_th;
    bool check_dh = false;
    if (L <= 4 && L >= 3)
        check_dh = true;
    else if (L == 2)
        check_dh = it <= 4;
    else if (L <= 1)
        check_dh = it <= 2;
    const bool ge3 = L >= 3;
    double H = 0;
    if (ge3) {
        double gsd = a.gs;
        if (gsd < (double)(1 << (L - 1))) gsd = (double)(1 << (L - 1));
        double th2 = gsd * 10;
        if (a.is_ra == 1) th2 = gsd * 30;
        H = a.hinterval < th2 ? a.hinterval : th2;
    }
    double lo, hi;
    if (ge3 && !check_dh) {
        lo = hi = height_th_of(true, H, th80, H);
    } else {
        // up = mean + 3 std, evaluated as the reference does; each operation
        // is non-decreasing in its operand (or non-increasing, for the
        // subtrahend) over sums >= 0, and rounding to nearest is
        // monotone, so the corners of the sums' box bound the reference's
        // rounded value
        const double n = (double)dh_count;
        const double mean_lo = sd[0] / n, mean_hi = sd[1] / n;
        const double vn_lo = sd2[0] - sd[1] * sd[1] / n, vn_hi = sd2[1] - sd[0] * sd[0] / n;
        const double not_a_number = nan("");
        if (vn_hi < 0) {
            lo = hi = height_th_of(ge3, H, th80, not_a_number);   // sqrt of a negative: NaN
        } else if (vn_lo < 0) {
            // std >= 0, or NaN (which compares as +inf)
            lo = height_th_of(ge3, H, th80, mean_lo);
            hi = height_th_of(ge3, H, th80, not_a_number);
        } else {
            lo = height_th_of(ge3, H, th80, mean_lo + 3 * sqrt(vn_lo / n));
            hi = height_th_of(ge3, H, th80, mean_hi + 3 * sqrt(vn_hi / n));
        }
        if (hi < lo) hi = lo;
    }
    th->height_th = lo;
    th->height_th_hi = hi;
    th->ortho_ncc_th = ortho_ncc_th;
    th->th_ref_ncc = th_ref_ncc;
}

// The sums' bound (lo, hi) around the reference's sequential sums, given the
// sums s in another order of m terms >= 0: |seq - s| <= 2 (m-1) u (1 + O(u))
// * exact, and exact <= s (1 + (m-1) u (1 + O(u))); 3 m u covers both.
__host__ __device__ void sum_band(double s, int64_t m, double out[2]) {
    const double e = s * (3.0 * (double)m * 0x1p-53) * (1.0 + 0x1p-40);
    out[0] = nextafter(s - e, -(double)INFINITY);
    if (out[0] < 0) out[0] = 0;
    out[1] = nextafter(s + e, (double)INFINITY);
}

// Slots of the per-call counters (unsigned long long): [0..1] counts, [2]
// complement of the minimum z key, [3] maximum z key, [4] bad input, [5]
// valid triangles, [6] re-run due, [8..9] the two sums (doubles), [10..13]
// the thresholds (doubles: band low, band high, ortho NCC, reference NCC);
// the histogram follows at [16].
constexpr int kMiscSums = 8, kMiscTh = 10, kMiscHist = 16;

// The level's thresholds on the device, after the sums: th80 by a warp's
// prefix sums over the histogram (32-bit, wrapping as the reference's
// counter), then the band from the sums (mode: kTinSums*; `exact`: the sums
// are the reference's own).
__global__ void threshold_kernel(TinArgs a, unsigned long long *misc, uint32_t hdiffcount,
                                 int64_t m_terms, int mode, int exact) {
    const int lane = threadIdx.x & 31;
    const uint32_t *hbin = reinterpret_cast<const uint32_t *>(misc + kMiscHist);
    const long dh_count = (long)(3 * misc[5]);
    uint32_t th80 = 1000;
    if (a.L < 3) {
        uint32_t carry = 0;
        bool found = false;
        for (uint32_t base = 0; base < hdiffcount && !found; base += 32) {
            const uint32_t t = base + lane;
            uint32_t v = t < hdiffcount ? hbin[t] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += x;
            }
            const uint32_t cum = carry + v;
            const double per = __dmul_rn(__ddiv_rn((double)cum, (double)dh_count), 100.0);
            const unsigned hit = __ballot_sync(0xffffffffu, t < hdiffcount && per > 99);
            if (hit) {
                th80 = base + (uint32_t)(__ffs(hit) - 1);
                found = true;
            }
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (!found) th80 = hdiffcount - 1u;   // the reference's t - 1 after the loop
    }
    if (lane != 0) return;
    double *md = reinterpret_cast<double *>(misc);
    const double s = md[kMiscSums], s2 = md[kMiscSums + 1];
    double sd[2] = {s, s}, sd2[2] = {s2, s2};
    const bool finite = isfinite(s) && isfinite(s2);
    if (!exact && finite) {
        sum_band(s, m_terms, sd);
        sum_band(s2, m_terms, sd2);
    }
    TinThresholds th;
    thresholds_of(a, sd, sd2, dh_count, th80, &th);
    if (!exact && !finite) {
        // a sum that is not finite: every compared value falls inside the
        // band, so a pass that compares anything re-runs on the ordered sums
        th.height_th = -INFINITY;
        th.height_th_hi = INFINITY;
    } else if (!exact && mode == kTinSumsWideBand) {
        th.height_th -= 1.0;
        th.height_th_hi += 1.0;
    }
    md[kMiscTh] = th.height_th;
    md[kMiscTh + 1] = th.height_th_hi;
    md[kMiscTh + 2] = th.ortho_ncc_th;
    md[kMiscTh + 3] = th.th_ref_ncc;
}

}  // namespace

void tin_thresholds(const TinArgs &a, const double sd[2], const double sd2[2], long dh_count,
                    const uint32_t *hbin, uint32_t hdiffcount, TinThresholds *th) {
    // levels 0-2: the 99th percentile of the integer height differences
    uint32_t th80 = 1000;
    if (a.L < 3) {
        uint32_t total_dh = 0;
        long t = 0;
        bool found = false;
        while (t < (long)hdiffcount && !found) {
            total_dh += hbin[t];
            const double per = (double)total_dh / (double)dh_count * 100.0;
            if (per > 99) {
                th80 = (uint32_t)t;
                found = true;
            }
            ++t;
        }
        if (!found) th80 = (uint32_t)(t - 1);
    }
    thresholds_of(a, sd, sd2, dh_count, th80, th);
}

size_t tin_blunder_scratch(int64_t n_pts, int64_t n_tris, uint32_t hdiffcount) {
    const int64_t np = 3 * n_tris;
    return al(scan_tmp_bytes(n_pts + 1)) + al(3 * n_tris * sizeof(double)) +
           al(128 + (hdiffcount + 1) * 4) + al((np > 0 ? np : 1) * 4) +
           al(2 * (n_pts + 1) * 4) + al((n_pts + 1) * 8) + 2 * al(n_pts) + al(n_pts * 8) +
           al(n_pts);
}

void tin_threshold_band(const TinArgs &a, double sd, double sd2, int64_t m_terms, long dh_count,
                        const uint32_t *hbin, uint32_t hdiffcount, bool exact, double *lo,
                        double *hi) {
    double b1[2] = {sd, sd}, b2[2] = {sd2, sd2};
    if (!exact) {
        sum_band(sd, m_terms, b1);
        sum_band(sd2, m_terms, b2);
    }
    TinThresholds th;
    tin_thresholds(a, b1, b2, dh_count, hbin, hdiffcount, &th);
    *lo = th.height_th;
    *hi = th.height_th_hi;
}


cudaError_t run_tin_blunder(TinArgs a, vll_point3 *pts, const vll_tri *tris,
                            const float *ortho_ncc, vll_ugrid *gp3, uint8_t *detected,
                            uint32_t hdiffcount, int sums_mode, bool anchor_list,
                            void *scratch, size_t bytes, TinOutput *out, cudaStream_t s) {
    const int64_t np = 3 * a.n_tris;
    size_t tmp_b = scan_tmp_bytes(a.n_pts + 1);
    char *p = (char *)scratch;
    auto take = [&](size_t b) {
        void *r = p;
        p += al(b);
        return r;
    };
    void *tmp = take(tmp_b);
    double *dhv = (double *)take(3 * a.n_tris * sizeof(double));
    const size_t misc_b = 8 * kMiscHist + (hdiffcount + 1) * 4;
    unsigned long long *misc = (unsigned long long *)take(misc_b);
    double *sums = reinterpret_cast<double *>(misc + kMiscSums);
    const double *th = reinterpret_cast<const double *>(misc + kMiscTh);
    uint32_t *hbin = reinterpret_cast<uint32_t *>(misc + kMiscHist);
    int32_t *list = (int32_t *)take((np > 0 ? np : 1) * 4);
    unsigned int *count = (unsigned int *)take(2 * (a.n_pts + 1) * 4);
    unsigned int *cursor = count + a.n_pts + 1;
    int64_t *start = (int64_t *)take((a.n_pts + 1) * 8);
    uint8_t *flag0 = (uint8_t *)take(a.n_pts);
    uint8_t *det0 = (uint8_t *)take(a.n_pts);
    int64_t *anchor_node = (int64_t *)take(a.n_pts * 8);
    uint8_t *anchor_val = (uint8_t *)take(a.n_pts);
    if (!anchor_list) anchor_node = nullptr, anchor_val = nullptr;
    if ((size_t)(p - (char *)scratch) > bytes) return cudaErrorInvalidValue;
    unsigned int *bad = reinterpret_cast<unsigned int *>(misc + 4);
    unsigned int *rerun = reinterpret_cast<unsigned int *>(misc + 6);
    const bool exact = sums_mode == kTinSumsExact;
    cudaError_t e;
    if ((e = cudaMemsetAsync(misc, 0, misc_b, s))) return e;
    if ((e = cudaMemsetAsync(count, 0, 2 * (a.n_pts + 1) * 4, s))) return e;
    if (a.n_tris > 0) {
        int64_t tb = (a.n_tris + 255) / 256;
        if (tb > 148 * 4) tb = 148 * 4;   // bounds the per-block histogram flushes
        tri_terms_kernel<<<(unsigned)tb, 256, 0, s>>>(a, pts, tris, dhv, hbin, hdiffcount,
                                                      misc + 5, count, bad);
        if (exact)
            dh_serial_sum_kernel<<<1, 512, 0, s>>>(np, dhv, sums);
        else
            dh_psum_kernel<<<blocks_for(np, 256), 256, 0, s>>>(np, dhv, sums);
        if ((e = cudaGetLastError())) return e;
    }
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, tmp_b, count, start, (int)(a.n_pts + 1), s)))
        return e;
    if (a.n_tris > 0) fill_kernel<<<blocks_for(a.n_tris, 256), 256, 0, s>>>(a, tris, start, cursor, list);
    // the thresholds on the device: the point pass follows without a host wait
    threshold_kernel<<<1, 32, 0, s>>>(a, misc, hdiffcount, np, sums_mode, exact ? 1 : 0);
    copy_flags_kernel<<<blocks_for(a.n_pts, 256), 256, 0, s>>>(a.n_pts, pts, flag0, detected,
                                                               det0);
    const unsigned pblocks = blocks_for(a.n_pts * 32, 256);
    auto point_pass = [&]() -> cudaError_t {
        point_kernel<<<pblocks, 256, 0, s>>>(a, pts, tris, ortho_ncc, list, start, count, gp3,
                                             detected, flag0, bad, rerun, anchor_node,
                                             anchor_val, th);
        close_kernel<<<blocks_for(a.n_pts, 256), 256, 0, s>>>(a.n_pts, pts, misc, misc + 2,
                                                             rerun, bad);
        return cudaGetLastError();
    };
    if ((e = point_pass())) return e;
    unsigned long long m[kMiscHist];
    if ((e = cudaMemcpyAsync(m, misc, sizeof(m), cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    out->rerun = 0;
    if (m[6] && !m[4]) {
        // a comparison fell inside the band: undo the pass and run it again
        // with the threshold from the sums in the reference's order
        out->rerun = 1;
        restore_flags_kernel<<<blocks_for(a.n_pts, 256), 256, 0, s>>>(a.n_pts, pts, flag0,
                                                                      detected, det0);
        if (a.n_tris > 0) dh_serial_sum_kernel<<<1, 512, 0, s>>>(np, dhv, sums);
        else if ((e = cudaMemsetAsync(sums, 0, 16, s))) return e;
        threshold_kernel<<<1, 32, 0, s>>>(a, misc, hdiffcount, np, sums_mode, 1);
        // counts, z keys and the re-run flag start again ([4] bad and [5] the
        // valid count stay)
        if ((e = cudaMemsetAsync(misc, 0, 32, s))) return e;
        if ((e = cudaMemsetAsync(misc + 6, 0, 8, s))) return e;
        if ((e = point_pass())) return e;
        if ((e = cudaMemcpyAsync(m, misc, sizeof(m), cudaMemcpyDeviceToHost, s))) return e;
        if ((e = cudaStreamSynchronize(s))) return e;
    }
    out->bad_input = m[4] != 0;
    out->count[0] = (int64_t)m[0];
    out->count[1] = (int64_t)m[1];
    out->has_z = m[0] > 0;
    for (int k = 0; k < 2; ++k) {
        const unsigned long long b = k == 0 ? ~m[2] : m[3];
        const unsigned long long bits = (b >> 63) ? (b & 0x7fffffffffffffffull) : ~b;
        double v;
        memcpy(&v, &bits, 8);
        out->z[k] = v;
    }
    double th_lo;
    memcpy(&th_lo, &m[kMiscTh], 8);
    out->height_th = th_lo;
    out->anchor_node = anchor_node;
    out->anchor_val = anchor_val;
    return cudaSuccess;
}

}  // namespace vll

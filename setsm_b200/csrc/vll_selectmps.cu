// vll_selectmps.cu -- SelectMPs (setsm_code.cpp:8535-8895): the matched
// points of an iteration from the per-node peaks, and the UGRID updates that
// go with them.
//
// The reference makes a histogram of the first-peak correlations (levels > 0)
// to set its minimum threshold, then walks the grid nodes in order: each
// node's decision reads only that node's NCCresult and UGRID, updates its
// UGRID, and appends its point to the list.  On the GPU: one histogram pass
// (atomics), the threshold from the 100 bins, one pass that decides every
// node, and an order-preserving compaction (exclusive scan of the decisions)
// that writes the points in the reference's list order.
#include <cstdint>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "vll_device.cuh"
#include "vll_internal.h"

namespace vll {

namespace {

constexpr int kRohBins = 100;   // rohconvert

// Histogram of ceil(result0 * 100) over nodes with more than two heights.
__global__ void roh_hist_kernel(const vll_nccresult *__restrict__ ncc, int64_t n, int *hist,
                                unsigned long long *total) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (ncc[i].NumOfHeight > 2) {
            int r = (int)ceil(__dmul_rn(dq_result(ncc[i].result0), (double)kRohBins));
            if (r > kRohBins - 1) r = kRohBins - 1;
            if (r >= 0) atomicAdd(hist + r, 1);
            atomicAdd(total, 1ull);
        }
    }
}

__device__ __forceinline__ double dq_grid(int16_t v) { return __ddiv_rn((double)v, 1000.0); }

// The per-node decision (setsm_code.cpp:8658-8891).  Writes the node's
// UGRID and, for a selected node, keep[i] = 1 and its point (without
// grid_pts, the point's x holds the node index, exact in a double).
__global__ void select_kernel(const vll_nccresult *__restrict__ ncc, vll_ugrid *gp3,
                              const double *__restrict__ grid_pts, int64_t n, SelectArgs a,
                              int *keep, vll_point3 *cand) {
    const double roh_th = 0.05;
    const int L = a.pyramid_step;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        keep[i] = 0;
        const vll_nccresult r = ncc[i];
        if (!(r.NumOfHeight > 2)) continue;
        vll_ugrid g = gp3[i];
        if (L == 4 && a.iteration == 1) g.Height = -1000.0f;
        const double r0 = dq_result(r.result0), r1 = dq_result(r.result1);
        double ror;
        if ((a.iteration <= 2 && L >= 3) || (a.iteration <= 1 && L == 2))
            ror = 1.0;
        else
            ror = fabs(r0) > 0 ? __ddiv_rn(__dadd_rn(r0, -r1), r0) : 0;
        const double ror_th0 = __dadd_rn(0.1, -__dmul_rn(0.03, (double)(3 - L)));
        bool index = false, index_1 = false, index_2 = false, index_3 = false, roh_index = false;
        if (L == 0) {
            if (ror >= ror_th0 && r0 > a.minimum_th) index_2 = true;
        } else {
            if (ror >= 0.1 && r0 > a.minimum_th) index_2 = true;
        }
        if (r0 > __dadd_rn(dq_grid(g.roh), -roh_th)) index_3 = true;
        if (r.result4 > 0) index = true;
        if (a.mpp_stereo_angle > 5) {
            if (L >= 2) {
                roh_index = index & index_2 & index_3;
            } else if (L >= 1) {
                if (index_3 && r0 > a.minimum_th) index_1 = true;
                roh_index = (index_3 & index_2) | index_1;
            } else if (L == 0 && a.final_level_iteration < 3) {
                roh_index = index & index_2 & index_3;
            } else {
                if (index_3) index_1 = true;
                roh_index = index_2 & index_1;
            }
        } else {
            if (L >= 1) {
                roh_index = index & index_2 & index_3;
            } else if (L == 0 && a.final_level_iteration < 3) {
                roh_index = index & index_2 & index_3;
            } else {
                if (index_3) index_1 = true;
                roh_index = index_2 & index_1;
            }
        }
        if (g.Matched_flag != 0) {
            index = false;
            index_1 = false;
            index_2 = false;
            const double gr = __dadd_rn(dq_grid(g.roh), -roh_th);
            if (L <= 0) {
                if (ror < ror_th0 && r1 > gr) index = true;
            } else {
                if (ror < 0.1 && r1 > gr) index = true;
            }
            if (r.result2 > r.result3) index_1 = true;
            index_2 = !index_1;
            index_1 = index & index_1;
            index_2 = index & index_2;
            if (index_1) {
                g.minHeight = to_short(floor(__dadd_rn((double)r.result3, -0.5)));
                g.maxHeight = to_short(ceil(__dadd_rn((double)r.result2, 0.5)));
                g.Matched_flag = 4;
            }
            if (index_2) {
                g.minHeight = to_short(floor(__dadd_rn((double)r.result2, -0.5)));
                g.maxHeight = to_short(ceil(__dadd_rn((double)r.result3, 0.5)));
                g.Matched_flag = 4;
            }
        }
        const int16_t q_min_th = q_result(a.minimum_th);
        const int16_t q_th_roh = q_result(a.th_roh);
        bool sel = false;
        const double z = (double)r.result2;
        if (roh_index) {
            if (L < 2) {
                const double pre_h = (double)g.Height;
                const double pre_range = (double)(g.maxHeight - g.minHeight);
                const uint8_t pre_match = g.Matched_flag;
                const bool i1 = pre_match == 0, i2 = pre_match == 2,
                           i3 = pre_match == 1 || pre_match == 4;
                const double s2 = __dmul_rn(__dmul_rn(a.mpp, 2.0), (double)(1 << L));
                const double s3 = __dmul_rn(__dmul_rn(a.mpp, 3.0), (double)(1 << L));
                const bool i4 = fabs(__dadd_rn(pre_h, -z)) <= s2;
                const bool i5 = fabs(__dadd_rn(pre_h, -z)) <= __ddiv_rn(pre_range, 2.0);
                const bool i41 = fabs(__dadd_rn(z, -(double)g.minHeight)) <= s3;
                const bool i42 = fabs(__dadd_rn(z, -(double)g.maxHeight)) <= s3;
                const bool i6 = (i4 | i5 | i41 | i42) & i3;
                const bool i7 = i2 & i4;
                if ((i1 | i7 | i6) && z > -100 && z < 10000) {
                    sel = true;
                    g.roh = r.result0;
                    if (g.roh < q_min_th) g.roh = q_min_th;
                } else {
                    g.roh = q_th_roh;
                    if (a.check_iter_end && a.th_roh_start == dq_grid(g.roh))
                        g.roh = q_result(a.th_roh_next);
                }
            } else {
                if (z > -100 && z < 10000) sel = true;
                g.roh = r.result0;
                if (g.roh < q_min_th) g.roh = q_min_th;
            }
        } else {
            g.roh = q_th_roh;
            if (a.check_iter_end && a.th_roh_start == dq_grid(g.roh))
                g.roh = q_result(a.th_roh_next);
        }
        gp3[i] = g;
        if (sel) {
            keep[i] = 1;
            vll_point3 p;
            memset(&p, 0, sizeof(p));
            if (grid_pts) {
                p.x = grid_pts[2 * i];
                p.y = grid_pts[2 * i + 1];
            } else {
                p.x = (double)i;   // the node: the caller fills the coordinates
            }
            p.z = z;
            p.flag = 0;
            cand[i] = p;
        }
    }
}

__global__ void compact_kernel(const int *keep, const int64_t *pos, const vll_point3 *cand,
                               int64_t n, vll_point3 *out, int64_t cap) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (keep[i] && pos[i] < cap) out[pos[i]] = cand[i];
}

unsigned blocks_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

}  // namespace

size_t select_mps_scratch(int64_t n) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int *)nullptr, (int64_t *)nullptr, (int)n);
    return al(tmp) + al(kRohBins * 4) + al(8) + al(n * 4) + al(n * 8) + al(n * sizeof(vll_point3));
}

cudaError_t run_roh_hist(const vll_nccresult *ncc, int64_t n, void *scratch, int *hist_out,
                         int64_t *total_out, cudaStream_t s) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int *)nullptr, (int64_t *)nullptr, (int)n);
    char *p = (char *)scratch + al(tmp);
    int *hist = (int *)p;
    unsigned long long *total = (unsigned long long *)(p + al(kRohBins * 4));
    cudaError_t e;
    if ((e = cudaMemsetAsync(hist, 0, kRohBins * 4, s))) return e;
    if ((e = cudaMemsetAsync(total, 0, 8, s))) return e;
    roh_hist_kernel<<<blocks_for(n, 256), 256, 0, s>>>(ncc, n, hist, total);
    if ((e = cudaGetLastError())) return e;
    unsigned long long t = 0;
    if ((e = cudaMemcpyAsync(hist_out, hist, kRohBins * 4, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(&t, total, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    *total_out = (int64_t)t;
    return cudaSuccess;
}

cudaError_t run_select_mps(const vll_nccresult *ncc, vll_ugrid *gp3, const double *grid_pts,
                           int64_t n, const SelectArgs &a, void *scratch,
                           vll_point3 *out, int64_t cap, int64_t *count, cudaStream_t s) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int *)nullptr, (int64_t *)nullptr, (int)n);
    char *p = (char *)scratch;
    void *tmp_p = p;
    p += al(tmp) + al(kRohBins * 4) + al(8);
    int *keep = (int *)p;
    p += al(n * 4);
    int64_t *pos = (int64_t *)p;
    p += al(n * 8);
    vll_point3 *cand = (vll_point3 *)p;
    cudaError_t e;
    select_kernel<<<blocks_for(n, 128), 128, 0, s>>>(ncc, gp3, grid_pts, n, a, keep, cand);
    if ((e = cudaGetLastError())) return e;
    if ((e = cub::DeviceScan::ExclusiveSum(tmp_p, tmp, keep, pos, (int)n, s))) return e;
    int64_t last_pos = 0;
    int last_keep = 0;
    if ((e = cudaMemcpyAsync(&last_pos, pos + n - 1, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(&last_keep, keep + n - 1, 4, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    *count = last_pos + last_keep;
    if (*count <= cap) {
        compact_kernel<<<blocks_for(n, 256), 256, 0, s>>>(keep, pos, cand, n, out, cap);
        if ((e = cudaGetLastError())) return e;
    }
    return cudaSuccess;
}

}  // namespace vll

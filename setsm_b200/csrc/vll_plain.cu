// vll_plain.cu -- the plain FP64 drop-in: one grid node per thread, FP64
// everywhere, the reference's operation order (VerticalLineLocus,
// setsm_code.cpp:6049-6548).  It is both a product kernel (exact mode) and
// the baseline the split-precision kernel is measured against.  Compiled with
// -fmad=false; the shared helpers use explicit _rn intrinsics in any case.
#include "vll_exact.cuh"
#include "vll_geo.cuh"
#include "vll_internal.h"

namespace vll {

__global__ void __launch_bounds__(128) plain_kernel(const DevLevel *__restrict__ Pp,
                                                    unsigned long long *__restrict__ counters,
                                                    double *rho_out, const int64_t *rho_off) {
    const DevLevel &P = *Pp;
    unsigned long long acc = 0, evals = 0;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x)
        plain_node(P, pt, acc, evals, rho_out, rho_off);
    if (acc) atomicAdd(&counters[0], acc);
    if (evals) atomicAdd(&counters[1], evals);
}

// Re-evaluate a list of (node, slot) pairs exactly (FP64).  Used by the split
// pipeline for the evaluations whose FP32 value sits inside the error band of
// a quantisation boundary or of a neighbour comparison.
__global__ void __launch_bounds__(128) recheck_kernel(const DevLevel *__restrict__ Pp,
                                                      const int64_t *__restrict__ items,
                                                      const unsigned long long *__restrict__ n_items,
                                                      int64_t max_items,
                                                      const double *__restrict__ gncc_sum,
                                                      const double *__restrict__ gncc_cnt,
                                                      double *__restrict__ out) {
    const DevLevel &P = *Pp;
    unsigned long long n = *n_items;
    if (n > (unsigned long long)max_items) n = (unsigned long long)max_items;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const int64_t code = items[i];
        const int64_t pt = code >> 16;
        const int k = (int)(code & 0xFFFF);
        const int ti = P.num_images - 1;
        PatchSrc S, Sn;
        make_src(P, ti, S, Sn);
        const vll_ugrid g = P.gp3[pt];
        const float hgt = slot_height(P, g.minHeight, P.ncc[pt].minHeight, k);
        const SlotOut o = eval_slot(P, pt, ti, S, Sn, hgt, gncc_cnt ? gncc_cnt[pt] : 0.0,
                                    gncc_sum ? gncc_sum[pt] : 0.0);
        out[2 * i] = o.rho;
        out[2 * i + 1] = o.count_incc > 0 ? __ddiv_rn(o.sum_incc, o.count_incc) : -1.0;
    }
}

// GNCC only (per node), for the split pipeline: exact FP64.
__global__ void __launch_bounds__(128) gncc_kernel(const DevLevel *__restrict__ Pp,
                                                   double *__restrict__ gsum,
                                                   double *__restrict__ gcnt) {
    const DevLevel &P = *Pp;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        const int ti = P.num_images - 1;
        double c = 0, s = 0;
        if (P.check_ortho && dq_result(ugrid_ortho_ncc(P.gp3, P.n_nodes, pt, ti)) > P.ortho_th) {
            const vll_ugrid g = P.gp3[pt];
            const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
            if (check_image_boundary(P, lon, lat, (double)g.minHeight, (double)g.maxHeight, P.H) &&
                !blunder_cell(P, g)) {
                PatchSrc S, Sn;
                make_src(P, ti, S, Sn);
                node_gncc(P, pt, ti, S, Sn, c, s);
            }
        }
        gsum[pt] = s;
        gcnt[pt] = c;
    }
}

// SetOrthoImageCoord, setsm_code.cpp:6550-6670 (OR pyramid): image coordinates
// of every ortho pixel of the tile at its grid node's height, per image.
__global__ void __launch_bounds__(256) ortho_kernel(const DevLevel *__restrict__ Pp,
                                                    double2 *const *__restrict__ cd,
                                                    double2 *const *__restrict__ cdn) {
    const DevLevel &P = *Pp;
    const double *B = P.boundary;
    const int64_t total = P.ow * P.oh;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < total;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = it / P.ow;
        const int64_t col = it % P.ow;
        const double tX = __dadd_rn(B[0], __dmul_rn((double)col, P.im_res));
        const double tY = __dadd_rn(B[1], __dmul_rn((double)row, P.im_res));
        const int64_t t_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.grid_res);
        const int64_t t_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.grid_res);
        const int64_t pt = t_row * P.grid_w + t_col;
        int64_t tcn = 0, trn = 0, pimn = 0;
        if (P.combined) {
            tcn = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.im_res_next);
            trn = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.im_res_next);
            pimn = trn * P.own + tcn;
        }
        if (!(pt < P.n_nodes && t_col < P.grid_w && t_row < P.grid_h)) continue;
        const float Hh = P.gp3[pt].Height;
        if (Hh == -1000) continue;
        const double2 w = ps2wgs_dev(P.param, tX, tY);
        for (int ti = 0; ti < P.num_images; ++ti) {
            const DevImage &im = P.im[ti];
            if (!im.selected) continue;
            const double2 ic = rpc_project(im.rpc, im.adj, w.x, w.y, (double)Hh);
            cd[ti][it] = to_pyramid(ic, im.sx, im.sy, P.L);
            if (P.combined && pimn < P.own * P.ohn && tcn < P.own && trn < P.ohn)
                cdn[ti][pimn] = to_pyramid(ic, im.sxn, im.syn, P.L - 1);
        }
    }
}

// AWNCC peak loop without SGM, setsm_code.cpp:7511-7702: one node per thread
// over the quantised voxel row.
__global__ void __launch_bounds__(256) awncc_kernel(const DevLevel *__restrict__ Pp,
                                                    const float *__restrict__ sumcost) {
    const DevLevel &P = *Pp;
    // with SGM (Pyramid_step <= SGM_py) the scan runs on the aggregated
    // SumCost, keeping the window NCC of the chosen peak (max_roh)
    const bool sgm = sumcost != nullptr;
    const int L = P.L, it = P.iteration;
    int check_ortho = !(L == 4 && it == 1);
    if (P.pre_dem_tif && !(L == 4 && it == 1)) check_ortho = 1;
    const bool max_mode = (it <= 3 && L == 4) || (it <= 2 && L == 3) || (it <= 1 && L == 2);
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        vll_nccresult R = P.ncc[pt];
        const vll_ugrid g = P.gp3[pt];
        double pre_rho = -1.0;
        float pre_height = 0.0f;
        int direction = 0, check_rho = 0;
        double best = -100.0, second = -100.0;
        double max_roh = 0, pre_wncc = -1.0;
        R.result0 = q_result(-1.0);
        R.result2 = -1000;
        R.result1 = q_result(-1.0);
        R.result3 = -1000;
        R.result4 = 0;
        const vll_voxel *row = P.vox + P.vox_off[pt];
        const float *srow = sgm ? sumcost + P.vox_off[pt] : nullptr;
        const double gncc = dq_result(R.GNCC);
        for (int64_t k = 0; k < R.NumOfHeight; ++k) {
            const float hgt = (float)__dadd_rn((double)R.minHeight, __dmul_rn((double)k, P.height_step));
            if (!(hgt >= (float)g.minHeight && hgt <= (float)g.maxHeight)) continue;
            const double incc = dq_voxel(row[k].INCC);
            double wncc;
            if (check_ortho && gncc > -1.0)
                wncc = __dadd_rn(__dmul_rn(incc, P.alpha), __dmul_rn(gncc, P.beta));
            else
                wncc = incc;
            const double rho = sgm ? (double)srow[k] : wncc;
            double diff;
            if (rho >= 0 && pre_rho >= 0)
                diff = __dadd_rn(rho, -pre_rho);
            else if (rho < 0 && pre_rho < 0)
                diff = -(__dadd_rn(fabs(rho), -fabs(pre_rho)));
            else if (rho >= 0 && pre_rho < 0)
                diff = 1;
            else
                diff = -1;
            int td = diff > 0 ? 1 : (diff < 0 ? -1 : 0);
            if (!check_rho) {
                check_rho = 1;
                td = -1;
            } else if (pre_rho != -1) {
                const bool is_peak = direction > 0 && td < 0;
                if (max_mode) {
                    if (best < rho) {
                        if (R.result4 < 10) R.result4 += 1;
                        best = rho;
                        R.result2 = hgt;
                        second = -1.0;
                        R.result3 = -9999;
                        max_roh = wncc;
                    }
                } else if (is_peak) {
                    if (R.result4 < 10) R.result4 += 1;
                    if (best < pre_rho) {
                        const double t1 = best;
                        best = pre_rho;
                        const float t2 = R.result2;
                        R.result2 = pre_height;
                        max_roh = pre_wncc;
                        if (second < t1) {
                            second = t1;
                            R.result3 = t2;
                        }
                    } else if (second < pre_rho) {
                        second = pre_rho;
                        R.result3 = pre_height;
                    }
                }
            }
            pre_rho = rho;
            pre_wncc = wncc;
            pre_height = hgt;
            direction = td;
        }
        if (sgm && P.L == 0 && it >= 2) {
            // the final iteration at level 0 keeps the window NCC of the peak
            // (setsm_code.cpp:7683-7688)
            R.result0 = q_result(max_roh);
            R.result1 = q_result(-1.0);
            R.result3 = -9999;
        } else {
            R.result0 = q_result(best);
            R.result1 = q_result(second);
        }
        P.ncc[pt] = R;
    }
}

// ---- launchers -----------------------------------------------------------------
cudaError_t launch_plain(const DevLevel *dP, int64_t n_nodes, unsigned long long *counters,
                         double *rho_out, const int64_t *rho_off, cudaStream_t s) {
    const int threads = 128;
    int64_t blocks = (n_nodes + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > (1 << 30)) blocks = 1 << 30;
    plain_kernel<<<(unsigned)blocks, threads, 0, s>>>(dP, counters, rho_out, rho_off);
    return cudaGetLastError();
}

namespace {
__global__ void row_max_kernel(const vll_nccresult *ncc, int64_t n, int *out) {
    int m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, (int)ncc[i].NumOfHeight);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}
}  // namespace

cudaError_t row_extent(const vll_nccresult *ncc, int64_t n, const int64_t *off, int *d_max,
                       int *max_h, int64_t *total, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(d_max, 0, sizeof(int), s))) return e;
    int64_t blocks = (n + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 16) blocks = 148 * 16;
    row_max_kernel<<<(unsigned)blocks, 256, 0, s>>>(ncc, n, d_max);
    if ((e = cudaGetLastError())) return e;
    if ((e = cudaMemcpyAsync(max_h, d_max, sizeof(int), cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(total, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s)))
        return e;
    return cudaStreamSynchronize(s);
}

cudaError_t launch_ortho(const DevLevel *dP, int64_t total, double2 *const *cd, double2 *const *cdn,
                         cudaStream_t s) {
    const int threads = 256;
    int64_t blocks = (total + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 64) blocks = 148 * 64;
    ortho_kernel<<<(unsigned)blocks, threads, 0, s>>>(dP, cd, cdn);
    return cudaGetLastError();
}

cudaError_t launch_awncc(const DevLevel *dP, int64_t n_nodes, const float *sumcost,
                         cudaStream_t s) {
    const int threads = 256;
    int64_t blocks = (n_nodes + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 64) blocks = 148 * 64;
    awncc_kernel<<<(unsigned)blocks, threads, 0, s>>>(dP, sumcost);
    return cudaGetLastError();
}

cudaError_t launch_gncc(const DevLevel *dP, int64_t n_nodes, double *gsum, double *gcnt,
                        cudaStream_t s) {
    const int threads = 128;
    int64_t blocks = (n_nodes + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 64) blocks = 148 * 64;
    gncc_kernel<<<(unsigned)blocks, threads, 0, s>>>(dP, gsum, gcnt);
    return cudaGetLastError();
}

cudaError_t launch_recheck(const DevLevel *dP, const int64_t *items, const unsigned long long *n_items,
                           int64_t max_items, const double *gsum, const double *gcnt, double *out,
                           cudaStream_t s) {
    const int threads = 128;
    int64_t blocks = (max_items + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 16) blocks = 148 * 16;
    recheck_kernel<<<(unsigned)blocks, threads, 0, s>>>(dP, items, n_items, max_items, gsum, gcnt, out);
    return cudaGetLastError();
}

}  // namespace vll

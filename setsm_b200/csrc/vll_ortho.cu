// vll_ortho.cu -- the orthoimage-window variants of VerticalLineLocus:
// VerticalLineLocus_seeddem (setsm_code.cpp:7720-7880) and
// VerticalLineLocus_blunder (:7882-8026).  Both project every ortho pixel of
// the tile through the RPCs at its grid node's height (SetOrthoImageCoord,
// :6550-6670, at the matched level or at the blunder-selected level) and run
// the multi-window NCC of each grid node over the ortho pixels around it; the
// seed-DEM pass widens or voids the node's height range where that NCC is
// low, the blunder pass records it (ortho_ncc, Mean_ortho_ncc, one float per
// node).  FP64 in the reference's operation order (compiled -fmad=false).
#include <cstdint>
#include <cuda_runtime.h>

#include "vll_exact.cuh"
#include "vll_geo.cuh"
#include "vll_internal.h"

namespace vll {

namespace {

// SetOrthoImageCoord for a raster of ow x oh pixels at im_res; `use_b`
// selects the blunder level's pyramid (py_BStartpos, blunder_selected_level).
__global__ void __launch_bounds__(256) ortho_raster_kernel(const DevLevel *__restrict__ Pp,
                                                           double2 *const *__restrict__ cd,
                                                           int64_t ow, int64_t oh, double im_res,
                                                           int use_b) {
    const DevLevel &P = *Pp;
    const double *B = P.boundary;
    const int64_t total = ow * oh;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < total;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = it / ow;
        const int64_t col = it % ow;
        const double tX = __dadd_rn(B[0], __dmul_rn((double)col, im_res));
        const double tY = __dadd_rn(B[1], __dmul_rn((double)row, im_res));
        const int64_t t_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.grid_res);
        const int64_t t_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.grid_res);
        const int64_t pt = t_row * P.grid_w + t_col;
        if (!(pt < P.n_nodes && t_col < P.grid_w && t_row < P.grid_h)) continue;
        const float Hh = P.gp3[pt].Height;
        if (Hh == -1000) continue;
        const double2 w = ps2wgs_dev(P.param, tX, tY);
        for (int ti = 0; ti < P.num_images; ++ti) {
            const DevImage &im = P.im[ti];
            if (!im.selected) continue;
            const double2 ic = rpc_project(im.rpc, im.adj, w.x, w.y, (double)Hh);
            cd[ti][it] = use_b ? to_pyramid(ic, im.sxb, im.syb, P.blunder_level)
                               : to_pyramid(ic, im.sx, im.sy, P.L);
        }
    }
}

// UGRID.ortho_ncc[ti] = v with the reference's indexing: the array has two
// entries, so ti = 2..4 land on the record's following fields (Mean_ortho_ncc,
// the flags, padding).  ti >= 5 would reach the next node's record, a write
// that races with that node's own update in the reference; it is not made.
__device__ __forceinline__ void set_ortho_ncc(vll_ugrid &g, int ti, int16_t v) {
    const int byte = 10 + 2 * ti;
    if (byte + 2 <= (int)sizeof(vll_ugrid))
        *reinterpret_cast<int16_t *>(reinterpret_cast<unsigned char *>(&g) + byte) = v;
}

struct OrthoArgs {
    double2 *const *cd;     // [num_images] rasters
    int64_t ow, oh;
    double im_res;
    int H;
    int r2max;              // window offsets kept: row^2 + col^2 <= r2max
    int use_b;              // sample the blunder level's images
};

// Multi-window NCC of node pt against image ti over the ortho pixels of its
// window (the window loops of setsm_code.cpp:7772-7805 / :7958-7996).
__device__ void ortho_node_ncc(const DevLevel &P, const OrthoArgs &A, int64_t pt, int ti,
                               double &ncc, int &cnt0) {
    const DevImage &ri = P.im[P.ref], &tI = P.im[ti];
    PatchSrc S;
    if (A.use_b) {
        S = PatchSrc{ri.img_b, ri.mag_b, tI.img_b, tI.mag_b, ri.wb, ri.hb, tI.wb, tI.hb};
    } else {
        S = PatchSrc{ri.img, ri.mag, tI.img, tI.mag, ri.w, ri.h, tI.w, tI.h};
    }
    const double gx = P.grid_pts[2 * pt], gy = P.grid_pts[2 * pt + 1];
    const double *B = P.boundary;
    const double2 *cr = A.cd[P.ref], *ct = A.cd[ti];
    double count = 0, sum = 0;
    cnt0 = 0;
    multi_ncc(S, A.H,
              [&](int row, int col, double2 &pl, double2 &pr) -> bool {
                  if (row * row + col * col > A.r2max) return false;
                  const double tX = __dadd_rn(gx, __dmul_rn((double)col, A.im_res));
                  const double tY = __dadd_rn(gy, __dmul_rn((double)row, A.im_res));
                  const int64_t t_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), A.im_res);
                  const int64_t t_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), A.im_res);
                  const int64_t pit = t_row * A.ow + t_col;
                  const int64_t tt_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.grid_res);
                  const int64_t tt_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.grid_res);
                  const int64_t pdem = tt_row * P.grid_w + tt_col;
                  if (!(pit >= 0 && pit < A.ow * A.oh && t_col >= 0 && t_col < A.ow &&
                        t_row >= 0 && t_row < A.oh && pdem >= 0 && pdem < P.n_nodes &&
                        tt_col >= 0 && tt_col < P.grid_w && tt_row >= 0 && tt_row < P.grid_h &&
                        cr != nullptr && ct != nullptr))
                      return false;
                  if (P.gp3[pdem].Height == -1000) return false;
                  pl = cr[pit];
                  pr = ct[pit];
                  return true;
              },
              count, sum, &cnt0);
    ncc = sum;   // ComputeMultiNCC adds to a sum that starts at 0
}

// VerticalLineLocus_seeddem's per-node update (setsm_code.cpp:7806-7853).
__global__ void __launch_bounds__(128) seeddem_kernel(const DevLevel *__restrict__ Pp,
                                                      const OrthoArgs A,
                                                      vll_ugrid *__restrict__ gout) {
    const DevLevel &P = *Pp;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        vll_ugrid g = P.gp3[pt];
        for (int ti = 1; ti < P.num_images; ++ti) {
            if (!P.im[ti].selected) continue;
            double ncc;
            int cnt0;
            ortho_node_ncc(P, A, pt, ti, ncc, cnt0);
            if (cnt0 == 0) ncc = -10;
            if (ncc < 0.3 && !P.check_matchtag) {
                g.minHeight = (int16_t)(g.minHeight - 100);
                if (g.minHeight < P.minmax[0]) g.minHeight = (int16_t)floor(P.minmax[0]);
                g.maxHeight = (int16_t)(g.maxHeight + 100);
                if (g.maxHeight > P.minmax[1]) g.maxHeight = (int16_t)ceil(P.minmax[1]);
                if (ncc < 0.1) {
                    g.minHeight = -9999;
                    g.maxHeight = -9999;
                }
            }
            set_ortho_ncc(g, ti, q_result(ncc));
            if (P.check_matchtag) g.roh = q_result(ncc >= 0.2 ? ncc : -0.2);
        }
        gout[pt] = g;
    }
}

// VerticalLineLocus_blunder's per-node result (setsm_code.cpp:7940-8012).
__global__ void __launch_bounds__(128) blunder_kernel(const DevLevel *__restrict__ Pp,
                                                      const OrthoArgs A,
                                                      vll_ugrid *__restrict__ gout,
                                                      float *__restrict__ ncc_out) {
    const DevLevel &P = *Pp;
    for (int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; pt < P.n_nodes;
         pt += (int64_t)gridDim.x * blockDim.x) {
        vll_ugrid g = P.gp3[pt];
        double max_ncc = -100;
        for (int ti = 1; ti < P.num_images; ++ti) {
            if (!P.im[ti].selected) continue;
            double ncc;
            int cnt0;
            ortho_node_ncc(P, A, pt, ti, ncc, cnt0);
            if (max_ncc < ncc) max_ncc = ncc;
            set_ortho_ncc(g, ti, q_result(ncc));
        }
        g.Mean_ortho_ncc = q_result(max_ncc);
        gout[pt] = g;
        ncc_out[pt] = (float)max_ncc;
    }
}

unsigned blocks_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return (unsigned)b;
}

}  // namespace

cudaError_t launch_ortho_raster(const DevLevel *dP, double2 *const *cd, int64_t ow, int64_t oh,
                                double im_res, int use_b, cudaStream_t s) {
    ortho_raster_kernel<<<blocks_for(ow * oh, 256), 256, 0, s>>>(dP, cd, ow, oh, im_res, use_b);
    return cudaGetLastError();
}

cudaError_t launch_seeddem(const DevLevel *dP, int64_t n_nodes, double2 *const *cd, int64_t ow,
                           int64_t oh, double im_res, int H, int use_b, vll_ugrid *gout,
                           cudaStream_t s) {
    const OrthoArgs A{cd, ow, oh, im_res, H, (H + 1) * (H + 1), use_b};
    seeddem_kernel<<<blocks_for(n_nodes, 128), 128, 0, s>>>(dP, A, gout);
    return cudaGetLastError();
}

cudaError_t launch_blunder(const DevLevel *dP, int64_t n_nodes, double2 *const *cd, int64_t ow,
                           int64_t oh, double im_res, int H, vll_ugrid *gout, float *ncc_out,
                           cudaStream_t s) {
    const OrthoArgs A{cd, ow, oh, im_res, H, (H - 1) * (H - 1), 1};
    blunder_kernel<<<blocks_for(n_nodes, 128), 128, 0, s>>>(dP, A, gout, ncc_out);
    return cudaGetLastError();
}

}  // namespace vll

// vll_internal.h -- launchers shared between the CUDA translation units and
// the C-ABI layer.  Not part of the public interface.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "setsm_vll.h"

namespace vll {

struct DevLevel;

// vll_plain.cu
cudaError_t launch_plain(const DevLevel *dP, int64_t n_nodes, unsigned long long *counters,
                         double *rho_out, const int64_t *rho_off, cudaStream_t s);
cudaError_t launch_ortho(const DevLevel *dP, int64_t total, double2 *const *cd,
                         double2 *const *cdn, cudaStream_t s);
cudaError_t launch_awncc(const DevLevel *dP, int64_t n_nodes, const float *sumcost,
                         cudaStream_t s);

// vll_plain.cu: the largest row length and the total (off[n]) of a packing.
cudaError_t row_extent(const vll_nccresult *ncc, int64_t n, const int64_t *off, int *d_max,
                       int *max_h, int64_t *total, cudaStream_t s);
// vll_sgm.cu: the 8-direction aggregation of AWNCC into sumcost (packed like
// the voxel rows); max_h is the level's largest NumOfHeight.  lr: scratch of
// sgm_scratch_bytes(n_slots) for the all-directions form, or nullptr (one
// launch per direction); sgm_scratch_bytes is 0 above its memory budget.
size_t sgm_scratch_bytes(int64_t n_slots);
cudaError_t launch_sgm(const DevLevel *dP, int64_t grid_w, int64_t grid_h, int max_h,
                       float *sumcost, int64_t n_slots, cudaStream_t s, float *lr);
cudaError_t launch_gncc(const DevLevel *dP, int64_t n_nodes, double *gsum, double *gcnt,
                        cudaStream_t s);
cudaError_t launch_recheck(const DevLevel *dP, const int64_t *items,
                           const unsigned long long *n_items, int64_t max_items,
                           const double *gsum, const double *gcnt, double *out, cudaStream_t s);

// vll_capi.cu: the per-call constants of a level from its descriptor;
// vll_window = false skips the VerticalLineLocus window-size check (the
// orthoimage variants choose their own window).
int derive_level(const vll_level_desc *d, DevLevel *P, std::string *err, bool vll_window = true);

// vll_ortho.cu: SetOrthoImageCoord at a chosen resolution / pyramid, and the
// seed-DEM and blunder ortho-NCC passes (gout may alias the level's gp3).
cudaError_t launch_ortho_raster(const DevLevel *dP, double2 *const *cd, int64_t ow, int64_t oh,
                                double im_res, int use_b, cudaStream_t s);
cudaError_t launch_seeddem(const DevLevel *dP, int64_t n_nodes, double2 *const *cd, int64_t ow,
                           int64_t oh, double im_res, int H, int use_b, vll_ugrid *gout,
                           cudaStream_t s);
cudaError_t launch_blunder(const DevLevel *dP, int64_t n_nodes, double2 *const *cd, int64_t ow,
                           int64_t oh, double im_res, int H, vll_ugrid *gout, float *ncc_out,
                           cudaStream_t s);

// vll_tinblunder.cu: blunder_detection_TIN.  TinArgs: the grid geometry,
// sizes, switches and (filled by run_tin_blunder) the thresholds.
struct TinArgs {
    double b0, b1, gs;
    int64_t width, n_nodes, n_pts, n_tris;
    int L, iteration, is_ra, flag_blunder, count_bl;
    // the height threshold lies in [height_th, height_th_hi] (equal when it
    // is known exactly)
    double height_th, height_th_hi, ortho_ncc_th, th_ref_ncc, hinterval;
};
// How the height-difference sums are formed: kTinSumsBand (default) in
// parallel, with a bound on their distance from the reference's sequential
// sums and an exact re-run when a comparison falls inside the resulting
// threshold band; kTinSumsExact sequentially on one SM; kTinSumsWideBand as
// kTinSumsBand with the band widened by 1 m on each side (re-runs on nearly
// every input: exercises the re-run).
enum { kTinSumsBand = 0, kTinSumsExact = 1, kTinSumsWideBand = 2 };
struct TinThresholds {
    double height_th, height_th_hi, ortho_ncc_th, th_ref_ncc;
};
struct TinOutput {
    int bad_input;        // a vertex's grid node outside the grid
    int64_t count[2];     // blunder_count additions: [0] kept, [1] blunders
    int has_z;            // z: height extent of the kept points
    double z[2];
    double height_th;
    int rerun;            // the point pass ran again with the exact threshold
    // anchor_list: per point the grid node whose anchor_flag the pass set (-1:
    // none) and the value (device pointers into the scratch)
    const int64_t *anchor_node;
    const uint8_t *anchor_val;
};
// The thresholds from the triangle statistics as the reference derives them
// (setsm_code.cpp:9289-9418): sd, sd2 = the sums of the height differences and
// of their squares, each known to lie in [lo, hi]; dh_count their number;
// hbin the histogram of the integer parts.  th->height_th / height_th_hi
// bound the reference's height threshold (equal when lo == hi).
void tin_thresholds(const TinArgs &a, const double sd[2], const double sd2[2], long dh_count,
                    const uint32_t *hbin, uint32_t hdiffcount, TinThresholds *th);
// The height-threshold band from sums in any order of m_terms terms (exact:
// the sums are the reference's own).
void tin_threshold_band(const TinArgs &a, double sd, double sd2, int64_t m_terms, long dh_count,
                        const uint32_t *hbin, uint32_t hdiffcount, bool exact, double *lo,
                        double *hi);
// anchor_list: the pass leaves gp3 alone and lists its anchor_flag writes
// (TinOutput::anchor_node / anchor_val) for the caller to apply.
size_t tin_blunder_scratch(int64_t n_pts, int64_t n_tris, uint32_t hdiffcount);
cudaError_t run_tin_blunder(TinArgs a, vll_point3 *pts, const vll_tri *tris,
                            const float *ortho_ncc, vll_ugrid *gp3, uint8_t *detected,
                            uint32_t hdiffcount, int sums_mode, bool anchor_list,
                            void *scratch, size_t bytes, TinOutput *out, cudaStream_t s);

// vll_initvoxel.cu: InitializeVoxel.  run_init_voxel decides every node
// (into scratch) and fills new_off[0..n] with the new packing, *total the new
// voxel count, *old_total the count of the incoming packing; run_commit_voxel
// writes the decided records to gp3 / ncc and run_pack_voxel the rows.
size_t init_voxel_scratch(int64_t n_nodes);
cudaError_t run_init_voxel(const DevLevel *dP, int64_t n, vll_ugrid *gp3, vll_nccresult *ncc,
                           void *scratch, int64_t *new_off, int64_t *total, int64_t *old_total,
                           cudaStream_t s);
cudaError_t run_commit_voxel(int64_t n, void *scratch, vll_ugrid *gp3, vll_nccresult *ncc,
                             cudaStream_t s);
cudaError_t run_pack_voxel(int64_t n, const int64_t *new_off, void *scratch, const vll_voxel *vin,
                           vll_voxel *vout, cudaStream_t s);

// vll_selectmps.cu: SelectMPs.  run_roh_hist fills the 100-bin histogram of
// the first-peak correlations (and the node count behind it); run_select_mps
// decides every node, updates gp3 and writes the selected points in node
// order to out (when *count <= cap).  Both wait.
struct SelectArgs {
    int pyramid_step, iteration, final_level_iteration, check_iter_end;
    double minimum_th, th_roh, th_roh_start, th_roh_next, mpp, mpp_stereo_angle;
};
size_t select_mps_scratch(int64_t n_nodes);
cudaError_t run_roh_hist(const vll_nccresult *ncc, int64_t n, void *scratch, int *hist_out,
                         int64_t *total_out, cudaStream_t s);
cudaError_t run_select_mps(const vll_nccresult *ncc, vll_ugrid *gp3, const double *grid_pts,
                           int64_t n, const SelectArgs &a, void *scratch, vll_point3 *out,
                           int64_t cap, int64_t *count, cudaStream_t s);

// vll_heightrange.cu: SetHeightRange on device data (gp3 updated in place,
// out = the returned grid); waits and returns the grid's height extent.
size_t height_range_scratch(int64_t n_nodes);
cudaError_t run_height_range(const DevLevel *dP, const DevLevel &hP, const vll_point3 *pts,
                             int64_t n_pts, const vll_tri *tris, int64_t n_tris, vll_ugrid *gp3,
                             vll_ugrid *out, double buffer, double th_hg, int iteration,
                             void *scratch, size_t scratch_bytes, double *min_h, double *max_h,
                             cudaStream_t s);

// vll_orthotin.cu: VerticalLineLocus_Ortho (one triangle; d_out = {F_Height,
// F_sncc, selected count}) and Ortho_blunder on device data.
cudaError_t launch_ortho_search(const DevLevel *dP, double mpp, const vll_point3 *d_pts3,
                                int64_t target_index, double *d_out, cudaStream_t s);
size_t ortho_blunder_scratch(int64_t n_pts, int64_t n_tris, int64_t n_nodes);
cudaError_t run_ortho_blunder(const DevLevel *dP, const DevLevel &hP, double mpp, vll_point3 *pts,
                              int64_t n_pts, const vll_tri *tris, int64_t n_tris,
                              vll_ugrid *gp3, void *scratch, size_t scratch_bytes,
                              int *iterations, int *bad_input, cudaStream_t s);

// vll_preprocess.cu
cudaError_t launch_sobel(const uint16_t *src, uint32_t w, uint32_t h, uint16_t *mag, uint8_t *bin,
                         cudaStream_t s);
cudaError_t launch_orientation(const uint16_t *mag, const uint8_t *bin, uint32_t w, uint32_t h,
                               int half, const double *wt, uint8_t *ori, cudaStream_t s);
cudaError_t launch_pyramid(const uint16_t *src, uint32_t w, uint32_t h, const double *f,
                           uint16_t *out, cudaStream_t s);

// vll_tin.cu: TINCreate_list.  TinWork holds the device work arrays between
// calls (grown on demand); run_tin_create writes the ordered triangle list of
// the n points (device) into d_tris (capacity entries; *count = the list's
// length), returning a VLL_* status and a message in *err.
struct TinWork {
    std::vector<std::pair<void *, size_t>> bufs;
};
void tin_release(TinWork &w);
int run_tin_create(TinWork &w, const vll_point3 *d_pts, int64_t n, const double min_max[4],
                   double resolution, vll_tri *d_tris, int64_t capacity, int64_t *count,
                   cudaStream_t s, std::string *err);

}  // namespace vll

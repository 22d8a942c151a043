/*
 * vll_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of SETSM's vertical-line-locus hot path, used as the
 * CPU checker for the CUDA kernels (and as the "port" CPU baseline).  It is
 * pinned bit-for-bit against the reference implementation compiled from its
 * own sources (oracle/_ref).  The product never links it.
 */
#ifndef SETSM_VLL_ORACLE_H
#define SETSM_VLL_ORACLE_H

#include <stdint.h>
#include "setsm_vll.h"

#ifdef __cplusplus
extern "C" {
#endif

void vo_set_threads(int threads);
int vo_max_threads(void);

/* MakeSobelMagnitudeImage, SubFunctions.cpp:2418-2471 */
void vo_sobel(uint32_t w, uint32_t h, const uint16_t *src, uint16_t *mag, int16_t *dir);
/* Orientation, SubFunctions.cpp:2473-2560 */
void vo_orientation(uint32_t w, uint32_t h, const uint16_t *mag, const int16_t *dir,
                    int template_size, uint8_t *ori);
/* CreateImagePyramid<uint16>(.., 9, 1.5), Template.hpp:45-131 */
void vo_pyramid_down(uint32_t w, uint32_t h, const uint16_t *src, uint16_t *out);

/* GetObjectToImageRPC_single, CoordConversion.hpp:26-86; xy = {sample, line} */
void vo_rpc_project(const vll_image_desc *im, long n, const double *lon, const double *lat,
                    const double *hgt, double *xy);
/* ps2wgs_single, CoordConversion.cpp:396-490; lonlat = {lon, lat} */
void vo_ps2wgs(const vll_transparam *p, long n, const double *xy, double *lonlat);

/* InitializeVoxel, setsm_code.cpp:5759-6012 on packed voxel rows. */
long vo_initialize_voxel(const vll_level_desc *d, vll_ugrid *gridpt3, vll_nccresult *ncc,
                         const vll_voxel *voxels_in, vll_voxel *voxels_out, long cap);

/* VerticalLineLocus, setsm_code.cpp:6049-6548.  Returns Accessable_grid.
 * Optional per-evaluation output: rho_out[rho_offsets[i] + k] receives the
 * FP64 temp_rho of node i at height index k (NaN where not evaluated);
 * evals_out receives the number of window evaluations. */
long vo_vertical_line_locus(const vll_level_desc *d, const vll_ugrid *gridpt3,
                            vll_nccresult *ncc, vll_voxel *voxels, long cap,
                            const int64_t *rho_offsets, double *rho_out, int64_t *evals_out);

/* AWNCC peak loop without SGM, setsm_code.cpp:7511-7702. */
void vo_awncc_peaks(const vll_level_desc *d, const vll_ugrid *gridpt3, vll_nccresult *ncc,
                    const vll_voxel *voxels, long cap);

/* Known-answer hooks on the building blocks of the window evaluation. */
/* Correlate, SubFunctions.cpp:974-1018 */
double vo_correlate(const double *L, const double *R, int N);
/* _result / _voxel quantisers, Template.hpp:964-993 */
int16_t vo_quantize_result(double v);
int16_t vo_quantize_voxel(double v);
/* Sub-window sample counts of the circular window of half-size `half` when
 * every sample is valid: SetVecKernelValue (SubFunctions.cpp:3249-3315)
 * driven by VerticalLineLocus's window loop (setsm_code.cpp:6429-6453). */
void vo_window_counts(int half, int counts[3]);

#ifdef __cplusplus
}
#endif
#endif

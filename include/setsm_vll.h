/*
 * setsm_vll.h -- C ABI of the B200 vertical-line-locus matcher.
 *
 * This is the drop-in boundary for SETSM's matching hot path:
 *   int VerticalLineLocus(VOXEL **grid_voxel, const ProInfo *proinfo,
 *                         NCCresult *nccresult, LevelInfo &plevelinfo,
 *                         const UGRID *GridPT3, const uint8 iteration,
 *                         const double *minmaxHeight);
 * declared at setsm_code.hpp:81 and defined at setsm_code.cpp:6049-6548 of the
 * reference.  That symbol is C++ (it takes a reference), so the library ships
 * a C++ shim with the same mangled signature (setsm_vll_compat.hpp) on top of
 * the plain-C entry points below.  Everything here takes plain pointers and
 * sizes; all status codes are negative on failure and the library never
 * exits the process (the reference calls exit(1) on allocation failure,
 * setsm_code.cpp:6571-6584).
 *
 * Record layouts (vll_nccresult, vll_ugrid, vll_voxel, vll_transparam) are
 * byte-identical to the reference's NCCresult, UGRID, VOXEL and TransParam
 * (Typedefine.hpp:248-293, Typedefine.hpp:214-230) so host arrays produced by
 * the reference's callers are passed through without repacking.
 */
#ifndef SETSM_VLL_H
#define SETSM_VLL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VLL_ABI_VERSION 3
#define VLL_MAX_IMAGES 8

/* ---- status codes ------------------------------------------------------ */
enum vll_status {
    VLL_OK = 0,
    VLL_ERR_INVALID = -1,      /* bad argument or inconsistent descriptor   */
    VLL_ERR_UNSUPPORTED = -2,  /* e.g. frame (AB) sensor, too many images   */
    VLL_ERR_CUDA = -3,         /* CUDA runtime error; see vll_last_error()  */
    VLL_ERR_NOMEM = -4,        /* device or pinned-host allocation failed   */
    VLL_ERR_TIMEOUT = -5,      /* persistent kernel hit its bounded wait    */
    VLL_ERR_CAPACITY = -6      /* caller buffer too small                   */
};

/* ---- kernels ----------------------------------------------------------- */
enum vll_kernel {
    /* One grid node per thread, FP64 everywhere, operation order of the
     * reference; bit-exact with VerticalLineLocus on the same inputs. */
    VLL_KERNEL_FP64_PLAIN = 0,
    /* FP64 RPC, FP32 tile-relative sampling and mean-centred NCC sums,
     * persistent (node, height-chunk) work queue, in-kernel FP64 re-check of
     * evaluations whose quantised or compared value sits within the FP32
     * error band. */
    VLL_KERNEL_SPLIT = 1
};

/* ---- record layouts identical to the reference ------------------------- */
/* NCCresult, Typedefine.hpp:248-268 (24 bytes). */
typedef struct vll_nccresult {
    float result2;            /* first peak height  */
    float result3;            /* second peak height */
    int16_t minHeight;
    int16_t maxHeight;
    int16_t result0;          /* first peak rho x 1000 (rounded)  */
    int16_t result1;          /* second peak rho x 1000 (rounded) */
    int16_t max_WNCC;
    int16_t GNCC;
    uint16_t NumOfHeight;
    uint8_t result4;          /* peak count, capped at 10 */
    uint8_t check_height_change;
} vll_nccresult;

/* D3DPOINT, Typedefine.hpp:139-194 (32 bytes): a matched point, projected
 * metres and height, and its flag. */
typedef struct vll_point3 {
    double x, y, z;
    uint8_t flag;
    uint8_t _pad[7];
} vll_point3;

/* UI3DPOINT, Typedefine.hpp:74-97: a TIN triangle's vertex indices. */
typedef struct vll_tri {
    uint32_t a, b, c;
} vll_tri;

/* UGRID, Typedefine.hpp:270-283 (20 bytes). */
typedef struct vll_ugrid {
    float Height;
    int16_t minHeight;
    int16_t maxHeight;
    int16_t roh;
    int16_t ortho_ncc[2];
    int16_t Mean_ortho_ncc;
    uint8_t Matched_flag;
    uint8_t anchor_flag;
} vll_ugrid;

/* VOXEL, Typedefine.hpp:285-291 (4 bytes). */
typedef struct vll_voxel {
    uint8_t flag_cal;
    int16_t INCC;             /* rho x 1000, truncated toward zero */
} vll_voxel;

/* TransParam, Typedefine.hpp:214-230 (polar-stereographic / UTM constants). */
typedef struct vll_transparam {
    double t_c, m_c;
    double sa, sb, e2, e2cuadrada, c;
    double a, e;
    double phi_c, lambda_0;
    int32_t pm;
    int32_t projection;       /* 1 = polar stereographic, otherwise UTM */
    int32_t utm_zone;
    char direction[2];
    int32_t bHemisphere;
} vll_transparam;

/* ---- level descriptor (what LevelInfo + ProInfo carry for this path) --- */
/* One image of the stereo set at the matched pyramid level (and at the next
 * finer level when the level is matched in combined mode,
 * setsm_code.cpp:6084-6088). */
typedef struct vll_image_desc {
    const uint16_t *image;       /* py_Images[ti], row-major width*height  */
    const uint16_t *mag;         /* py_MagImages[ti]                       */
    const uint8_t *ori;          /* py_OriImages[ti]                       */
    uint32_t width, height;      /* py_Sizes[ti][Pyramid_step]             */
    double startpos[2];          /* py_Startpos[ti] {x, y}                 */
    const uint16_t *image_next;  /* py_Images_next[ti]; NULL unless combined */
    const uint16_t *mag_next;
    const uint8_t *ori_next;
    uint32_t width_next, height_next;
    double startpos_next[2];
    /* RPC in the reference's row layout (SubFunctions.cpp:1494-1582):
     * [0..4]  line_off, samp_off, lon_off, lat_off, h_off
     * [5..9]  the matching scales
     * [10..29] LINE_NUM, [30..49] LINE_DEN, [50..69] SAMP_NUM,
     * [70..89] SAMP_DEN, RPC00B term order. */
    double rpc[90];
    double image_adjust[2];      /* ImageAdjust[ti] {deltaLine, deltaSamp} */
    int32_t selected;            /* proinfo->check_selected_image[ti]      */
    int32_t _pad;
    /* The blunder-selected pyramid level (LevelInfo.blunder_selected_level,
     * setsm_code.cpp:3560-3565), read by VerticalLineLocus_blunder and by
     * VerticalLineLocus_seeddem with check_Matchtag; NULL = the matched level. */
    const uint16_t *image_b;     /* py_BImages[ti]                         */
    const uint16_t *mag_b;       /* py_BMagImages[ti]                      */
    uint32_t width_b, height_b;  /* py_Sizes[ti][blunder_selected_level]   */
    double startpos_b[2];        /* py_BStartpos[ti]                       */
} vll_image_desc;

typedef struct vll_level_desc {
    int32_t num_images;          /* proinfo->number_of_images (<= VLL_MAX_IMAGES) */
    int32_t reference_id;        /* plevelinfo.reference_id (0 in SETSM)  */
    int32_t pyramid_step;        /* *plevelinfo.Pyramid_step              */
    int32_t template_size;       /* *plevelinfo.Template_size             */
    int32_t py_combined_level;   /* *plevelinfo.Py_combined_level         */
    int32_t iteration;           /* VerticalLineLocus's `iteration`       */
    int32_t check_matching_rate; /* 1: memory-tight route, peaks streamed  */
    int32_t is_ra;               /* proinfo->IsRA                          */
    int32_t pre_dem_tif;         /* proinfo->pre_DEMtif                    */
    int32_t check_matchtag;      /* proinfo->check_Matchtag                */
    int32_t sgm_py;              /* proinfo->SGM_py                        */
    int32_t sensor_type;         /* 0 = SB (RPC); frame cameras unsupported */
    double resolution;           /* proinfo->resolution (image GSD, m)     */
    double dem_resolution;       /* proinfo->DEM_resolution                */
    double height_step;          /* *plevelinfo.height_step                */
    double grid_resolution;      /* *plevelinfo.grid_resolution            */
    double bin_angle;            /* *plevelinfo.bin_angle (degrees)        */
    double boundary[4];          /* plevelinfo.Boundary                    */
    double minmax_height[2];     /* minmaxHeight                           */
    int64_t grid_width;          /* Size_Grid2D->width                     */
    int64_t grid_height;         /* Size_Grid2D->height                    */
    const double *grid_pts;      /* GridPts  [N][2] projected metres       */
    const double *grid_wgs;      /* Grid_wgs [N][2] lon, lat degrees       */
    vll_transparam param;        /* *plevelinfo.param                      */
    vll_image_desc images[VLL_MAX_IMAGES];
    int32_t blunder_level;       /* *plevelinfo.blunder_selected_level (used
                                    when images[].image_b is set)           */
    int32_t _pad2;
} vll_level_desc;

/* Per-call statistics (filled when a vll_stats pointer is passed; the call
 * then waits for the GPU). */
typedef struct vll_stats {
    int64_t accessable_grid;     /* VerticalLineLocus's return value        */
    int64_t evals;               /* (node, height) NCC evaluations computed */
    int64_t fp64_rechecks;       /* split kernel: evaluations redone in FP64 */
    double kernel_ms;            /* device time of all matching kernels     */
    double window_ms;            /* device time of the window (NCC) kernel  */
    int64_t slots;               /* height slots scheduled                  */
    int64_t launches;            /* kernels launched by the call            */
    double stage_ms[8];          /* split pipeline: gncc, prep, prefix sums,
                                    items, window, scan, exact path, tail   */
    int64_t exact_nodes;         /* split: nodes sent to the exact path     */
    int64_t fp64_nodes;          /* split: nodes recomputed wholly in FP64  */
    int64_t scan_rounds;         /* split: scan rounds on the exact path    */
} vll_stats;

typedef struct vll_context vll_context;

/* ---- context ------------------------------------------------------------ */
int vll_create(int device, vll_context **out);
void vll_destroy(vll_context *ctx);
/* Last error message of this context (or of the process when ctx is NULL). */
const char *vll_last_error(const vll_context *ctx);
int vll_abi_version(void);

/* Size of the packed voxel array for a level: sum of nccresult[i].NumOfHeight
 * over all grid nodes.  The packed layout concatenates grid_voxel[i][0..n) in
 * node order, which is how the shim marshals the reference's VOXEL** rows. */
int64_t vll_voxel_count(const vll_nccresult *nccresult, int64_t n_nodes);

/*
 * One VerticalLineLocus call on HOST buffers (setsm_code.cpp:6049-6548).
 *   gridpt3    [N] in   (UGRID)
 *   nccresult  [N] in/out (NCCresult; range fields set by InitializeVoxel in
 *                   the voxel route, peaks written in the memory-tight route)
 *   voxels     packed in/out voxel rows (voxel route); may be NULL when
 *                   desc->check_matching_rate is set
 *   stats      optional
 * Uploads inputs, runs `kernel`, downloads results.  Returns VLL_OK or a
 * negative status.
 */
int vll_vertical_line_locus(vll_context *ctx, const vll_level_desc *desc,
                            const vll_ugrid *gridpt3, vll_nccresult *nccresult,
                            vll_voxel *voxels, int64_t voxel_capacity,
                            int kernel, vll_stats *stats);

/*
 * Same call with every pointer on the DEVICE: the image planes and grid
 * arrays inside `desc`, gridpt3, nccresult, the packed voxel rows and their
 * row offsets (int64 [N+1], exclusive prefix sum of NumOfHeight; voxel route
 * only).  Inputs stay resident; nothing is copied to or from the host.  Work
 * is queued on the context's stream; the call waits for it only when `stats`
 * is non-NULL.
 */
int vll_vertical_line_locus_device(vll_context *ctx, const vll_level_desc *desc,
                                   const vll_ugrid *d_gridpt3, vll_nccresult *d_nccresult,
                                   vll_voxel *d_voxels, const int64_t *d_voxel_offsets,
                                   int kernel, vll_stats *stats);

/* Diagnostics (memory-tight route): runs `kernel` on host inputs and returns
 * the per-slot rho it computed, at offset prefix(K)[node] + slot where
 * K = (int)((maxHeight - minHeight) / height_step) of each node's UGRID;
 * slots that were not evaluated are NaN.  For VLL_KERNEL_SPLIT these are the
 * FP32 values before any FP64 re-check; for VLL_KERNEL_FP64_PLAIN the exact
 * FP64 temp_rho. */
int vll_debug_slot_rho(vll_context *ctx, const vll_level_desc *desc, const vll_ugrid *gridpt3,
                       vll_nccresult *nccresult, int kernel, double *rho_out, int64_t capacity,
                       uint64_t *diag_out);
/* diag_out (optional, 16 entries, split kernel): cycles summed over warps in
 * node setup, coordinates, staging, window, scan, re-check and fold, then
 * counts of nodes, 32-slot passes, FP64 slow-path lanes, un-staged passes,
 * whole-node FP64 fallbacks, scan rounds and re-checked slots. */

/*
 * Residency of the host-buffer calls.  Matching_SETSM calls VerticalLineLocus
 * once per iteration on the same level images (setsm_code.cpp:3774-3844) and
 * passes its voxel rows through InitializeVoxel, VerticalLineLocus and AWNCC
 * only.  With VLL_RESIDENT_PLANES, the image planes (intensity, magnitude,
 * orientation, next level) and the grid's coordinate arrays of
 * vll_vertical_line_locus stay on the device between calls and are sent
 * again only when their host pointer, size or a sampled fingerprint of
 * their bytes (64 spread 64-byte blocks) changes; a caller that rewrites a
 * plane in place between calls without any of these changing must clear the
 * flag.  With VLL_RESIDENT_VOXELS, vll_initialize_voxel called with a NULL
 * output pointer keeps its output packing in the context (the input rows
 * are `voxels_in` when given, else the context's packing when its length
 * equals the old NumOfHeight sum, else none), and vll_vertical_line_locus /
 * vll_awncc_peaks called with a NULL voxel pointer use that packing in place
 * (its length must equal the sum of NumOfHeight); vll_resident_voxels copies
 * it out.  Both flags are off by default.
 */
enum {
    VLL_RESIDENT_PLANES = 1,
    VLL_RESIDENT_VOXELS = 2
};
int vll_set_residency(vll_context *ctx, int flags);
int vll_get_residency(const vll_context *ctx);
/* Forgets the resident voxel packing (a new grid or level). */
int vll_resident_reset(vll_context *ctx);
/* Copies the resident voxel packing to `voxels` (capacity entries); `total`
 * receives its length (VLL_ERR_CAPACITY when it does not fit). */
int vll_resident_voxels(vll_context *ctx, vll_voxel *voxels, int64_t capacity, int64_t *total);

/* Use `stream` (a cudaStream_t) for this context's work; NULL restores a
 * private stream.  vll_get_stream returns the stream in use. */
int vll_set_stream(vll_context *ctx, void *stream);
void *vll_get_stream(vll_context *ctx);
/* Number of kernels this context has launched for matching calls so far. */
int64_t vll_launch_count(const vll_context *ctx);

/*
 * Allocation-free VerticalLineLocus.  This entry point has no counterpart in
 * the reference; it exists for callers that cannot allocate device memory at
 * call time (a pool allocator that owns the whole GPU, another framework's
 * memory manager, a latency-critical loop that cannot absorb cudaMalloc's
 * implicit synchronisation).  It runs the split-precision pipeline with every
 * scratch buffer taken from one file-scope device array of 64 MiB that each
 * GPU loading this library holds until process exit, and calls no
 * cudaMalloc, cudaFree or allocating library routine; no vll_context is used.
 *   - All pointers are DEVICE pointers (as for
 *     vll_vertical_line_locus_device); `stream` is a cudaStream_t (NULL =
 *     legacy default stream).  The call waits on the host for its work to
 *     finish before it returns.
 *   - Memory-tight route only (check_matching_rate = 1), stereo, levels
 *     without orthoimage GNCC; anything else returns VLL_ERR_UNSUPPORTED.
 *   - Grids whose per-node scratch (20 bytes a node) does not fit the 64 MiB
 *     array beside the window kernel's per-warp slot scratch (2 KiB a warp,
 *     about 3.5 MiB on a B200), about 3.1 M nodes, return VLL_ERR_CAPACITY
 *     before any output is written; `err_buf` receives a message.  The rest of the array holds
 *     the FP32 values of the few nodes queued for the exact FP64 pass; a node
 *     that finds it full is evaluated wholly in FP64, so results never depend
 *     on its size (only the time does).
 *   - The array is committed on a device when this library's module is
 *     loaded there; under CUDA's lazy module loading that is this call's
 *     first use on the device, so make a first call before a memory pool
 *     reserves the device's memory.  That call also looks up the array's
 *     device address (cudaGetSymbolAddress) with the device current; make it
 *     before any stream capture.  The address is looked up again when the
 *     device's context changed (after cudaDeviceReset).
 *   - Every call shares the one array, which keeps the previous call's
 *     contents; calls that overlap on the GPU (different streams or threads
 *     at the same time) race on it and must be serialised by the caller.
 */
int vll_vertical_line_locus_noalloc(const vll_level_desc *desc, const vll_ugrid *d_gridpt3,
                                    vll_nccresult *d_nccresult, void *stream,
                                    int64_t *accessable_grid, char *err_buf, int err_len);

/*
 * TINCreate_list (SubFunctions.cpp:2768-2846): the Delaunay triangulation of
 * the matched points, each snapped to the level's grid (column and row =
 * 0.5 + the offset from min_max[0] / min_max[1] in `resolution` cells,
 * truncated), as the reference's ordered list of vertex-index triples: the
 * triangles of its divide and conquer (grid_triangulation.cpp, co-circular
 * ties decided as there), listed point by point in grid order.  The points'
 * grid cells must be distinct (else VLL_ERR_INVALID); grids wider or taller
 * than 32767 cells return VLL_ERR_INVALID (the reference exits).  `count`
 * receives the list's length; a list longer than `capacity` returns
 * VLL_ERR_CAPACITY with `count` set and `tris` unwritten.  Fewer than 3 points
 * give an empty list.  The reference also returns its triangulation object
 * (for TINUpdate_list); this call returns the list only.
 */
int vll_tin_create(vll_context *ctx, const vll_point3 *pts, int64_t n_pts, const double min_max[4],
                   double resolution, vll_tri *tris, int64_t capacity, int64_t *count);
/* The same on DEVICE points and triangle arrays (min_max stays on the host). */
int vll_tin_create_device(vll_context *ctx, const vll_point3 *d_pts, int64_t n_pts,
                          const double min_max[4], double resolution, vll_tri *d_tris,
                          int64_t capacity, int64_t *count);

/* ---- batches: many tiles / pyramid levels in one pass ------------------- */
/* One level of a batch: a descriptor whose every pointer is on the DEVICE (as
 * for vll_vertical_line_locus_device) and the level's device arrays. */
typedef struct vll_level_io {
    const vll_level_desc *desc;
    const vll_ugrid *d_gridpt3;
    vll_nccresult *d_nccresult;
    vll_voxel *d_voxels;              /* voxel route only, else NULL */
    const int64_t *d_voxel_offsets;   /* int64 [N+1], voxel route only */
} vll_level_io;

/*
 * VerticalLineLocus (setsm_code.cpp:6049-6548) on n_levels independent
 * levels -- tiles of one or several scenes, pyramid levels, window sizes --
 * in ONE pass of the split pipeline: one prep pass over all their nodes, ONE
 * persistent window launch draining every level's (node, 32-slot) work items,
 * one peak scan and one exact FP64 pass.  Each level's outputs are exactly
 * those of vll_vertical_line_locus_device on that level alone.  Every level
 * must be one the split kernel implements (stereo, window half-size 2..7);
 * otherwise VLL_ERR_UNSUPPORTED.  Levels matched in combined mode (the
 * next finer level's window added to the INCC, setsm_code.cpp:6378-6464) are
 * evaluated in exact FP64 inside the same launch.  accessable (optional, host, n_levels)
 * receives each level's Accessable_grid.  Waits for the GPU.
 */
int vll_vertical_line_locus_batch(vll_context *ctx, const vll_level_io *levels, int n_levels,
                                  int64_t *accessable, vll_stats *stats);

/*
 * The same batch as a CUDA graph.  vll_plan_create sizes every buffer (one
 * uncaptured pass of the pipeline's front half, which initialises the
 * outputs' per-node fields) and captures the whole
 * pipeline; vll_plan_run replays it on the context's stream with no host
 * synchronisation inside (it waits only when `accessable` or `stats` is
 * given).  The plan owns its scratch; the level arrays and images must stay
 * valid and unmoved while it is used.  It holds while each level's height
 * ranges keep the plan's total of height slots: a replay after ranges change
 * that total does no matching and returns VLL_ERR_INVALID (create a new plan).
 */
typedef struct vll_plan vll_plan;
int vll_plan_create(vll_context *ctx, const vll_level_io *levels, int n_levels, vll_plan **out);
int vll_plan_run(vll_plan *plan, int64_t *accessable, vll_stats *stats);
void vll_plan_destroy(vll_plan *plan);

/* ---- launch tuning (chosen by setsm_b200/autotune.py) -------------------- */
typedef struct vll_tuning {
    int32_t blocks_per_sm;   /* window kernel CTAs per SM; 0 = occupancy maximum   */
    int32_t grab;            /* nodes a warp takes per queue access (1..64; 0:
                                default 8; at most 32 are used)                  */
    float box_margin;        /* shared-memory footprint budget over the estimate  */
    int32_t _pad;
} vll_tuning;
int vll_set_tuning(vll_context *ctx, const vll_tuning *t);
int vll_get_tuning(const vll_context *ctx, vll_tuning *t);

/*
 * AWNCC (setsm_code.cpp:7001-7702) over the packed voxel rows, on HOST
 * buffers: on levels with Pyramid_step <= SGM_py the 8-direction semi-global
 * aggregation of the voxel INCC (SGM_start_pos / SGM_con_pos, :6755-6999)
 * followed by the peak loop on the aggregated cost; on other levels the peak
 * loop on the voxels and the node's GNCC.  First / second peaks per node are
 * selected exactly as the reference does.
 */
int vll_awncc_peaks(vll_context *ctx, const vll_level_desc *desc,
                    const vll_ugrid *gridpt3, vll_nccresult *nccresult,
                    const vll_voxel *voxels, int64_t voxel_capacity,
                    vll_stats *stats);
/* The same on device data: the packed voxel rows and their N + 1 int64
 * offsets (as vll_initialize_voxel_device writes them).  Asynchronous on the
 * context's stream unless `stats` is given. */
int vll_awncc_peaks_device(vll_context *ctx, const vll_level_desc *desc,
                           const vll_ugrid *d_gridpt3, vll_nccresult *d_nccresult,
                           const vll_voxel *d_voxels, const int64_t *d_voxel_offsets,
                           vll_stats *stats);

/* ---- orthoimage-window variants (setsm_code.cpp:7720-8026) ------------- */
/*
 * VerticalLineLocus_seeddem (setsm_code.cpp:7720-7880): the orthoimage NCC of
 * every grid node against each selected image at the node's height; where it
 * is below 0.3 the node's height range is widened by 100 m (clamped to
 * desc->minmax_height) and voided (-9999) below 0.1; ortho_ncc[ti] (and roh
 * with check_Matchtag, which samples the blunder level's images) are set.
 * Template size and window follow the reference (5 m template area, radius
 * Half+1).  gridpt3 is updated in place; bit-exact with the reference.
 * The _device forms take device pointers in the descriptor and gridpt3 and
 * are asynchronous on the context's stream (they wait only when `stats` is
 * given); the host forms copy in and out and wait.
 */
int vll_vertical_line_locus_seeddem(vll_context *ctx, const vll_level_desc *desc,
                                    vll_ugrid *gridpt3, vll_stats *stats);
int vll_vertical_line_locus_seeddem_device(vll_context *ctx, const vll_level_desc *desc,
                                           vll_ugrid *d_gridpt3, vll_stats *stats);
/*
 * VerticalLineLocus_blunder (setsm_code.cpp:7882-8026): the same orthoimage
 * NCC at the blunder-selected level (images[].image_b, desc->blunder_level;
 * radius Half-1, Half from iteration and bblunder as the reference), written
 * to ortho_ncc[ti], Mean_ortho_ncc (the maximum over images) and
 * nccresult[node] (float).  Returns VLL_OK where the reference returns true.
 * The UGRID fields are bit-exact; the float NCC equals the reference's but
 * for rare last-bit differences of the map projection's libm calls (about
 * one node in a thousand, by ~1e-10).
 */
int vll_vertical_line_locus_blunder(vll_context *ctx, const vll_level_desc *desc,
                                    vll_ugrid *gridpt3, int iteration, int bblunder,
                                    float *nccresult, vll_stats *stats);
int vll_vertical_line_locus_blunder_device(vll_context *ctx, const vll_level_desc *desc,
                                           vll_ugrid *d_gridpt3, int iteration, int bblunder,
                                           float *d_nccresult, vll_stats *stats);

/*
 * VerticalLineLocus_Ortho (setsm_code.cpp:8234-8533): the height search of a
 * TIN triangle's target vertex.  Its height is swept over the UGRID range of
 * grid node `target_index` in steps of resolution * 2^Pyramid_step * MPP (MPP
 * clamped to [1, 3]); at each height the triangle's plane is sampled on the
 * grid cells inside it, both images are read at the level (images[].image,
 * mag), and the mean Pearson correlation of intensities and magnitudes over
 * the target images picks the height.  Outputs as the reference: *f_height
 * (-9999 when none qualifies), *f_sncc (written when a height was found) and
 * the selected sample count (the reference's return value).  Host buffers.
 */
int vll_vertical_line_locus_ortho(vll_context *ctx, const vll_level_desc *desc, double mpp,
                                  const vll_point3 *ref1, const vll_point3 *ref2,
                                  const vll_point3 *target, const vll_ugrid *gridpt3,
                                  int64_t target_index, double *f_height, double *f_sncc,
                                  int *selected_count);
/*
 * Ortho_blunder (setsm_code.cpp:8028-8232): up to 200 rounds of the height
 * search over every TIN triangle with exactly two anchored vertices
 * (UGRID.anchor_flag 1 or 3), each round applying the best height per target
 * point in triangle order (point height, flag, node anchor_flag = 3) until a
 * round finds none.  pts, tris and gridpt3 are updated in place exactly as the
 * reference does; *rounds (optional) receives the number of rounds.  The
 * _device form takes device pointers (descriptor planes included) and waits.
 */
int vll_ortho_blunder(vll_context *ctx, const vll_level_desc *desc, double mpp, vll_point3 *pts,
                      int64_t n_pts, const vll_tri *tris, int64_t n_tris, vll_ugrid *gridpt3,
                      int *rounds);
int vll_ortho_blunder_device(vll_context *ctx, const vll_level_desc *desc, double mpp,
                             vll_point3 *d_pts, int64_t n_pts, const vll_tri *d_tris,
                             int64_t n_tris, vll_ugrid *d_gridpt3, int *rounds);

/*
 * InitializeVoxel (setsm_code.cpp:5759-6012): every node's search range for
 * the voxel route (image-boundary test at the UGRID range, blunder-cell rules,
 * range carried over or extended from the previous NCCresult) and its voxel
 * row.  gridpt3 and nccresult are updated in place; voxels_in holds the rows
 * packed by the incoming NumOfHeight (NULL on the first iteration),
 * voxels_out receives them packed by the new NumOfHeight: rows whose range
 * changed initialised (flag_cal 1, INCC -1000), the others carried over.
 * *n_out receives the new voxel count; with *n_out > capacity the call
 * returns VLL_ERR_CAPACITY and leaves every buffer untouched.  Host buffers
 * (desc->grid_wgs, images' sizes / RPCs / startpos).  Bit-exact.
 */
int vll_initialize_voxel(vll_context *ctx, const vll_level_desc *desc, vll_ugrid *gridpt3,
                         vll_nccresult *nccresult, const vll_voxel *voxels_in,
                         vll_voxel *voxels_out, int64_t capacity, int64_t *n_out);
/*
 * The same on device data (desc->grid_wgs a device pointer; no image plane
 * is read): d_voxel_offsets (N + 1 int64) receives the new row offsets, the
 * form vll_vertical_line_locus_device takes, so the voxel route runs on the
 * device end to end.  d_voxels_out must not overlap d_voxels_in.  On
 * VLL_ERR_CAPACITY only *n_out and d_voxel_offsets are written.  Waits.
 */
int vll_initialize_voxel_device(vll_context *ctx, const vll_level_desc *desc,
                                vll_ugrid *d_gridpt3, vll_nccresult *d_nccresult,
                                const vll_voxel *d_voxels_in, vll_voxel *d_voxels_out,
                                int64_t capacity, int64_t *d_voxel_offsets, int64_t *n_out);

/*
 * SelectMPs (setsm_code.cpp:8535-8895): the matched points of an iteration.
 * At levels > 0 the first-peak correlations of the nodes with more than two
 * heights set the minimum threshold (a 100-bin histogram against the level's
 * quota); every node's peaks (nccresult) and UGRID then decide whether it
 * yields a point, update its roh, and at matched nodes with ambiguous peaks
 * widen its range (Matched_flag 4).  The points (x, y of grid_pts, z = first
 * peak height, flag 0) go to points[] in node order, *count receives their
 * number; with *count > capacity the call returns VLL_ERR_CAPACITY and leaves
 * gridpt3 and points untouched.  The other arguments are the reference's.
 * Host buffers; bit-exact with the reference.
 */
int vll_select_mps(vll_context *ctx, const vll_level_desc *desc, const vll_nccresult *nccresult,
                   vll_ugrid *gridpt3, double th_roh, double th_roh_min, double th_roh_start,
                   double th_roh_next, int iteration, double mpp, int final_level_iteration,
                   double mpp_stereo_angle, vll_point3 *points, int64_t capacity,
                   int64_t *count);
/* The same on device data (desc->grid_pts, the NCCresult, UGRID and points
 * buffers are device pointers); on VLL_ERR_CAPACITY d_gridpt3 has been
 * updated and no point written.  Waits. */
int vll_select_mps_device(vll_context *ctx, const vll_level_desc *desc,
                          const vll_nccresult *d_nccresult, vll_ugrid *d_gridpt3, double th_roh,
                          double th_roh_min, double th_roh_start, double th_roh_next,
                          int iteration, double mpp, int final_level_iteration,
                          double mpp_stereo_angle, vll_point3 *d_points, int64_t capacity,
                          int64_t *count);

/*
 * blunder_detection_TIN (setsm_code.cpp:9158-9787): marks the matched points
 * whose TIN neighbourhood is inconsistent in height.  Statistics over the
 * triangles (the vertices' ortho_ncc, the edges' height differences against
 * hinterval = *LevelInfo.Hinterval) set the thresholds; each point not already
 * flagged 1 then tests its first 30 triangles and may flag itself or a
 * neighbour as a blunder (pts[].flag 1, detected_blunders[] set for points that
 * were 0), resets / sets its node's anchor_flag; blunder_count[0..1] are
 * incremented by the kept / blunder points and *minz_mp / *maxz_mp take the
 * kept points' height extent.  Does nothing at level 0, iteration 3, as the
 * reference.  Host buffers; bit-exact with the reference.
 */
int vll_blunder_detection_tin(vll_context *ctx, const vll_level_desc *desc, int iteration,
                              const float *ortho_ncc, int flag_blunder, int count_bl,
                              double hinterval, vll_point3 *pts, uint8_t *detected_blunders,
                              int64_t n_pts, const vll_tri *tris, int64_t n_tris,
                              vll_ugrid *gridpt3, int64_t *blunder_count, double *minz_mp,
                              double *maxz_mp);
/* The same on device data (ortho_ncc, pts, detected_blunders, tris and
 * gridpt3 are device pointers; blunder_count, minz_mp and maxz_mp are host
 * pointers).  Waits.  A point whose grid node lies outside the grid is found
 * during the point pass: the call then returns VLL_ERR_INVALID with the
 * device buffers pts[].flag, detected_blunders and gridpt3[].anchor_flag
 * partly written (undefined); the host outputs are unchanged.  (The host
 * entry leaves every caller buffer as it was.) */
int vll_blunder_detection_tin_device(vll_context *ctx, const vll_level_desc *desc, int iteration,
                                     const float *d_ortho_ncc, int flag_blunder, int count_bl,
                                     double hinterval, vll_point3 *d_pts,
                                     uint8_t *d_detected_blunders, int64_t n_pts,
                                     const vll_tri *d_tris, int64_t n_tris, vll_ugrid *d_gridpt3,
                                     int64_t *blunder_count, double *minz_mp, double *maxz_mp);
/* blunder_detection_TIN forms its height-difference sums in parallel and
 * bounds their distance from the reference's sequential sums; a point pass in
 * which some comparison falls inside the resulting threshold band is undone
 * and run again with the sequential sums.  The number of such calls on this
 * context. */
int64_t vll_tin_rerun_count(const vll_context *ctx);

/*
 * SetHeightRange (setsm_code.cpp:9851-10255): the next iteration's height
 * ranges from the TIN of matched points.  Every grid node inside a triangle
 * takes the plane's height (the vertex height on a vertex at levels 0-1) and
 * a range from the triangle's height extent plus a buffer set by the level,
 * `iteration`, `mpp`, the triangle's slope and the node's Mean_ortho_ncc
 * (a node is set by the first triangle, in order, that contains it); nodes in
 * no triangle take their matched neighbours' range union.  gridpt3 is updated
 * in place as the reference updates GridPT3 before freeing it; `result` (N
 * records) receives the returned grid, *min_h_grid / *max_h_grid the range
 * extent.  seed_dem_sigma is proinfo->seedDEMsigma (read with pre_DEMtif).
 * Bit-exact with the reference for up to five images.
 */
int vll_set_height_range(vll_context *ctx, const vll_level_desc *desc, const vll_point3 *pts,
                         int64_t n_pts, const vll_tri *tris, int64_t n_tris, vll_ugrid *gridpt3,
                         vll_ugrid *result, int iteration, double mpp,
                         int level_check_matching_rate, double seed_dem_sigma,
                         double *min_h_grid, double *max_h_grid);
/* The same on device data (points, triangles, UGRID and result). Waits. */
int vll_set_height_range_device(vll_context *ctx, const vll_level_desc *desc,
                                const vll_point3 *d_pts, int64_t n_pts, const vll_tri *d_tris,
                                int64_t n_tris, vll_ugrid *d_gridpt3, vll_ugrid *d_result,
                                int iteration, double mpp, int level_check_matching_rate,
                                double seed_dem_sigma, double *min_h_grid, double *max_h_grid);

/* Diagnostics: the orthoimage coordinate raster of image `ti`
 * (SetOrthoImageCoord, setsm_code.cpp:6550-6670) at resolution im_res, on
 * the matched level's pyramid (use_b = 0) or the blunder level's (1), as
 * {x, y} doubles row-major into out[2 * capacity]; *width / *height receive
 * the raster size. */
int vll_debug_ortho_raster(vll_context *ctx, const vll_level_desc *desc, const vll_ugrid *gridpt3,
                           int use_b, double im_res, int ti, double *out, int64_t capacity,
                           int64_t *width, int64_t *height);

/* Diagnostics (host only, no GPU): blunder_detection_TIN's height threshold
 * (setsm_code.cpp:9320-9418) bounded from sums formed in any order.
 * sd / sd2: the sums of the m_terms height differences and of their squares
 * in some order; dh_count, hbin[hdiffcount]: the count and the histogram of
 * their integer parts.  exact != 0 takes sd / sd2 as the reference's own
 * sequential sums.  [*lo, *hi] receives the band that holds the reference's
 * threshold (lo == hi when it is known exactly). */
int vll_debug_tin_threshold(int pyramid_step, int iteration, int is_ra, double grid_resolution,
                            double hinterval, double sd, double sd2, int64_t m_terms,
                            int64_t dh_count, const uint32_t *hbin, uint32_t hdiffcount,
                            int exact, double *lo, double *hi);

/* ---- image preprocessing (SubFunctions.cpp:2418-2560, Template.hpp:82) -- */
/* Sobel magnitude (uint16) and 20-degree direction bin per pixel, on host
 * buffers; bit-exact with MakeSobelMagnitudeImage + Orientation. */
int vll_preprocess_level(vll_context *ctx, const uint16_t *image,
                         uint32_t width, uint32_t height, int template_size,
                         uint16_t *mag_out, uint8_t *ori_out);
/* 9x9 sigma=1.5 Gaussian 2x downsample, bit-exact with CreateImagePyramid. */
int vll_pyramid_down(vll_context *ctx, const uint16_t *image, uint32_t width,
                     uint32_t height, uint16_t *out);
/* Device-pointer variants of the two preprocessing calls. */
int vll_preprocess_level_device(vll_context *ctx, const uint16_t *d_image,
                                uint32_t width, uint32_t height, int template_size,
                                uint16_t *d_mag, uint8_t *d_ori);
int vll_pyramid_down_device(vll_context *ctx, const uint16_t *d_image, uint32_t width,
                            uint32_t height, uint16_t *d_out);

#ifdef __cplusplus
}
#endif
#endif /* SETSM_VLL_H */

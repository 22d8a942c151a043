/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C entry points that run the reference SETSM implementation (compiled
 * from its own sources by oracle/Makefile into oracle/_ref/libsetsm_ref.so)
 * on a vll_level_desc.  It is used to pin the C restatement in
 * oracle/vll_oracle.c, to generate golden fixtures and as the timed CPU
 * baseline.  Nothing in the product links or loads it.
 *
 * Every function below only marshals arguments into the reference's own
 * structures (ProInfo, LevelInfo, VOXEL**, RPC row arrays) and calls:
 *   InitializeVoxel      setsm_code.cpp:5759
 *   VerticalLineLocus    setsm_code.cpp:6049
 *   AWNCC                setsm_code.cpp:7001
 *   MakeSobelMagnitudeImage / Orientation   SubFunctions.cpp:2418 / :2473
 *   CreateImagePyramid   Template.hpp:82
 *   GetObjectToImageRPC_single  CoordConversion.hpp:26
 *   ps2wgs_single / wgs2ps_single  CoordConversion.cpp:396 / :103
 */
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>

#include "setsm_code.hpp"
#include "CoordConversion.hpp"
#include "SubFunctions.hpp"
#include "Template.hpp"

#include "setsm_vll.h"

namespace {

struct RefLevel {
    ProInfo *proinfo = nullptr;
    LevelInfo li;
    const uint16 *imgs[VLL_MAX_IMAGES];
    const uint16 *mags[VLL_MAX_IMAGES];
    const uint8 *oris[VLL_MAX_IMAGES];
    const uint16 *imgs_next[VLL_MAX_IMAGES];
    const uint16 *mags_next[VLL_MAX_IMAGES];
    const uint8 *oris_next[VLL_MAX_IMAGES];
    const uint16 *imgs_b[VLL_MAX_IMAGES];
    const uint16 *mags_b[VLL_MAX_IMAGES];
    D2DPOINT startpos_b[VLL_MAX_IMAGES];
    D2DPOINT startpos[VLL_MAX_IMAGES];
    D2DPOINT startpos_next[VLL_MAX_IMAGES];
    CSize sizes_store[VLL_MAX_IMAGES][16];
    const CSize *sizes[VLL_MAX_IMAGES];
    const double *rpc_rows[VLL_MAX_IMAGES][7];
    const double *const *rpcs[VLL_MAX_IMAGES];
    double errbias[2] = {0.0, 0.0};
    const double *adjust[VLL_MAX_IMAGES];
    TransParam param;
    int pyramid_step;
    int blunder_level;
    unsigned char template_size;
    unsigned char num_ia = 2;
    unsigned char iteration;
    double bin_angle, height_step, grid_resolution, hinterval = 0.0;
    int py_combined_level;
    CSize grid_size;
    long grid_length;
    bool check_matching_rate;

    explicit RefLevel(const vll_level_desc *d) {
        proinfo = (ProInfo *)calloc(1, sizeof(ProInfo));
        proinfo->resolution = d->resolution;
        proinfo->DEM_resolution = d->dem_resolution;
        proinfo->number_of_images = d->num_images;
        proinfo->sensor_type = SB;
        proinfo->IsRA = d->is_ra != 0;
        proinfo->pre_DEMtif = d->pre_dem_tif != 0;
        proinfo->check_Matchtag = d->check_matchtag != 0;
        proinfo->SGM_py = d->sgm_py;
        for (int ti = 0; ti < d->num_images; ++ti)
            proinfo->check_selected_image[ti] = d->images[ti].selected != 0;

        pyramid_step = d->pyramid_step;
        blunder_level = d->images[0].image_b ? d->blunder_level : d->pyramid_step;
        template_size = (unsigned char)d->template_size;
        iteration = (unsigned char)d->iteration;
        bin_angle = d->bin_angle;
        height_step = d->height_step;
        grid_resolution = d->grid_resolution;
        py_combined_level = d->py_combined_level;
        grid_size.width = (unsigned)d->grid_width;
        grid_size.height = (unsigned)d->grid_height;
        grid_length = (long)d->grid_width * (long)d->grid_height;
        check_matching_rate = d->check_matching_rate != 0;

        memset(&param, 0, sizeof(param));
        param.t_c = d->param.t_c; param.m_c = d->param.m_c;
        param.sa = d->param.sa; param.sb = d->param.sb; param.e2 = d->param.e2;
        param.e2cuadrada = d->param.e2cuadrada; param.c = d->param.c;
        param.a = d->param.a; param.e = d->param.e;
        param.phi_c = d->param.phi_c; param.lambda_0 = d->param.lambda_0;
        param.pm = d->param.pm; param.projection = d->param.projection;
        param.utm_zone = d->param.utm_zone;
        param.direction[0] = d->param.direction[0];
        param.direction[1] = d->param.direction[1];
        param.bHemisphere = d->param.bHemisphere;

        for (int ti = 0; ti < d->num_images; ++ti) {
            const vll_image_desc &im = d->images[ti];
            imgs[ti] = im.image; mags[ti] = im.mag; oris[ti] = im.ori;
            imgs_next[ti] = im.image_next; mags_next[ti] = im.mag_next; oris_next[ti] = im.ori_next;
            startpos[ti] = D2DPOINT(im.startpos[0], im.startpos[1]);
            startpos_next[ti] = D2DPOINT(im.startpos_next[0], im.startpos_next[1]);
            for (int l = 0; l < 16; ++l) sizes_store[ti][l] = CSize(0, 0);
            sizes_store[ti][pyramid_step] = CSize((int)im.width, (int)im.height);
            if (pyramid_step >= 1)
                sizes_store[ti][pyramid_step - 1] = CSize((int)im.width_next, (int)im.height_next);
            if (im.image_b) {
                imgs_b[ti] = im.image_b;
                mags_b[ti] = im.mag_b;
                startpos_b[ti] = D2DPOINT(im.startpos_b[0], im.startpos_b[1]);
                sizes_store[ti][blunder_level] = CSize((int)im.width_b, (int)im.height_b);
            } else {
                imgs_b[ti] = im.image;
                mags_b[ti] = im.mag;
                startpos_b[ti] = startpos[ti];
            }
            sizes[ti] = sizes_store[ti];
            rpc_rows[ti][0] = im.rpc + 0;
            rpc_rows[ti][1] = im.rpc + 5;
            rpc_rows[ti][2] = im.rpc + 10;
            rpc_rows[ti][3] = im.rpc + 30;
            rpc_rows[ti][4] = im.rpc + 50;
            rpc_rows[ti][5] = im.rpc + 70;
            rpc_rows[ti][6] = errbias;
            rpcs[ti] = rpc_rows[ti];
            adjust[ti] = im.image_adjust;
        }

        memset(&li, 0, sizeof(li));
        li.py_Images = imgs;
        li.py_OriImages = oris;
        li.py_MagImages = mags;
        li.py_BImages = imgs_b;
        li.py_BMagImages = mags_b;
        li.py_Images_next = imgs_next;
        li.py_OriImages_next = oris_next;
        li.py_MagImages_next = mags_next;
        li.py_Startpos = startpos;
        li.py_BStartpos = startpos_b;
        li.py_Startpos_next = startpos_next;
        li.RPCs = rpcs;
        li.Boundary = d->boundary;
        li.Pyramid_step = &pyramid_step;
        li.py_Sizes = sizes;
        li.Template_size = &template_size;
        li.ImageAdjust = adjust;
        li.param = &param;
        li.NumOfIAparam = &num_ia;
        li.bin_angle = &bin_angle;
        li.blunder_selected_level = &blunder_level;
        li.Size_Grid2D = &grid_size;
        li.Grid_length = &grid_length;
        li.GridPts = reinterpret_cast<const D2DPOINT *>(d->grid_pts);
        li.Grid_wgs = reinterpret_cast<const D2DPOINT *>(d->grid_wgs);
        li.reference_id = d->reference_id;
        li.height_step = &height_step;
        li.grid_resolution = &grid_resolution;
        li.Hinterval = &hinterval;
        li.Py_combined_level = &py_combined_level;
        li.iteration = &iteration;
        li.check_matching_rate = &check_matching_rate;
    }
    ~RefLevel() { free(proinfo); }
};

/* Build VOXEL** rows from the packed array (NumOfHeight entries per node). */
VOXEL **unpack_voxels(const vll_nccresult *ncc, long n, const vll_voxel *packed) {
    VOXEL **rows = (VOXEL **)calloc((size_t)n, sizeof(VOXEL *));
    long off = 0;
    for (long i = 0; i < n; ++i) {
        const int k = ncc[i].NumOfHeight;
        if (k > 0) {
            rows[i] = (VOXEL *)malloc(sizeof(VOXEL) * (size_t)k);
            for (int h = 0; h < k; ++h) {
                rows[i][h].flag_cal = packed ? packed[off + h].flag_cal != 0 : false;
                rows[i][h].INCC = packed ? packed[off + h].INCC : 0;
            }
            off += k;
        }
    }
    return rows;
}

/* Pack rows back by the (possibly updated) NumOfHeight, then free them. */
long pack_and_free_voxels(const vll_nccresult *ncc, long n, VOXEL **rows,
                          vll_voxel *packed, long cap) {
    long off = 0;
    for (long i = 0; i < n; ++i) {
        const int k = ncc[i].NumOfHeight;
        if (k > 0 && rows[i]) {
            for (int h = 0; h < k; ++h) {
                if (packed && off + h < cap) {
                    packed[off + h].flag_cal = rows[i][h].flag_cal ? 1 : 0;
                    packed[off + h].INCC = rows[i][h].INCC;
                }
            }
            off += k;
            free(rows[i]);
        }
        /* rows of nodes whose NumOfHeight is now 0 were already released by
         * InitializeVoxel (which frees without clearing the pointer). */
    }
    free(rows);
    return off;
}

}  // namespace

extern "C" {

int ref_sizeof_nccresult(void) { return (int)sizeof(NCCresult); }
int ref_sizeof_ugrid(void) { return (int)sizeof(UGRID); }
int ref_sizeof_voxel(void) { return (int)sizeof(VOXEL); }
int ref_sizeof_transparam(void) { return (int)sizeof(TransParam); }

void ref_set_threads(int threads) {
    if (threads > 0) omp_set_num_threads(threads);
}
int ref_max_threads(void) { return omp_get_max_threads(); }

/* InitializeVoxel on the packed voxel rows: `voxels_in` holds the rows of the
 * previous iteration (by the incoming NumOfHeight), `voxels_out` receives the
 * rows by the updated NumOfHeight.  Returns the packed count written. */
typedef void (*init_voxel_signature)(const ProInfo *, VOXEL **, LevelInfo &, UGRID *,
                                     NCCresult *, const int, const double *);
typedef void (*awncc_signature)(ProInfo *, VOXEL **, CSize, UGRID *, NCCresult *, double, uint8,
                                uint8, int);

/* InitializeVoxel, or the function at `fn` with its signature
 * (setsm_code.hpp:75); voxels in/out in packed form. */
long ref_call_initialize_voxel(void *fn, const vll_level_desc *d, vll_ugrid *gridpt3,
                               vll_nccresult *ncc, const vll_voxel *voxels_in,
                               vll_voxel *voxels_out, long cap) {
    RefLevel L(d);
    const long n = L.grid_length;
    VOXEL **rows = unpack_voxels(ncc, n, voxels_in);
    init_voxel_signature f = fn ? reinterpret_cast<init_voxel_signature>(fn) : &InitializeVoxel;
    f(L.proinfo, rows, L.li, reinterpret_cast<UGRID *>(gridpt3),
      reinterpret_cast<NCCresult *>(ncc), d->iteration, d->minmax_height);
    return pack_and_free_voxels(ncc, n, rows, voxels_out, cap);
}

long ref_initialize_voxel(const vll_level_desc *d, vll_ugrid *gridpt3, vll_nccresult *ncc,
                          const vll_voxel *voxels_in, vll_voxel *voxels_out, long cap) {
    return ref_call_initialize_voxel(nullptr, d, gridpt3, ncc, voxels_in, voxels_out, cap);
}

/* AWNCC through the function at `fn` with its signature (setsm_code.hpp:91). */
void ref_call_awncc(void *fn, const vll_level_desc *d, vll_ugrid *gridpt3, vll_nccresult *ncc,
                    vll_voxel *voxels, long cap) {
    RefLevel L(d);
    const long n = L.grid_length;
    VOXEL **rows = unpack_voxels(ncc, n, voxels);
    const int max_voxel = (int)((d->minmax_height[1] - d->minmax_height[0]) / d->height_step);
    reinterpret_cast<awncc_signature>(fn)(L.proinfo, rows, L.grid_size,
                                          reinterpret_cast<UGRID *>(gridpt3),
                                          reinterpret_cast<NCCresult *>(ncc), d->height_step,
                                          (uint8)d->pyramid_step, (uint8)d->iteration, max_voxel);
    pack_and_free_voxels(ncc, n, rows, voxels, cap);
}

/* VerticalLineLocus; voxels are in/out in packed form (ignored on the
 * memory-tight route).  Returns Accessable_grid. */
long ref_vertical_line_locus(const vll_level_desc *d, const vll_ugrid *gridpt3,
                             vll_nccresult *ncc, vll_voxel *voxels, long cap) {
    RefLevel L(d);
    const long n = L.grid_length;
    VOXEL **rows = nullptr;
    if (!L.check_matching_rate) rows = unpack_voxels(ncc, n, voxels);
    const int acc = VerticalLineLocus(rows, L.proinfo, reinterpret_cast<NCCresult *>(ncc), L.li,
                                      reinterpret_cast<const UGRID *>(gridpt3),
                                      (uint8)d->iteration, d->minmax_height);
    if (rows) pack_and_free_voxels(ncc, n, rows, voxels, cap);
    return acc;
}

/* AWNCC (peak loop; SGM too when pyramid_step <= sgm_py). */
void ref_awncc(const vll_level_desc *d, vll_ugrid *gridpt3, vll_nccresult *ncc,
               vll_voxel *voxels, long cap) {
    RefLevel L(d);
    const long n = L.grid_length;
    VOXEL **rows = unpack_voxels(ncc, n, voxels);
    const int max_voxel = (int)((d->minmax_height[1] - d->minmax_height[0]) / d->height_step);
    AWNCC(L.proinfo, rows, L.grid_size, reinterpret_cast<UGRID *>(gridpt3),
          reinterpret_cast<NCCresult *>(ncc), d->height_step, (uint8)d->pyramid_step,
          (uint8)d->iteration, max_voxel);
    pack_and_free_voxels(ncc, n, rows, voxels, cap);
}

void ref_sobel(uint32_t w, uint32_t h, const uint16_t *src, uint16_t *mag, int16_t *dir) {
    MakeSobelMagnitudeImage(CSize((int)w, (int)h), src, mag, dir);
}

void ref_orientation(uint32_t w, uint32_t h, const uint16_t *mag, const int16_t *dir,
                     int template_size, uint8_t *ori) {
    Orientation(CSize((int)w, (int)h), mag, dir, (uint8)template_size, ori);
}

/* CreateImagePyramid<uint16>(src, size, 9, 1.5) into `out` ((w/2)*(h/2)). */
void ref_pyramid_down(uint32_t w, uint32_t h, const uint16_t *src, uint16_t *out) {
    uint16 *r = CreateImagePyramid((uint16 *)src, CSize((int)w, (int)h), 9, 1.5);
    memcpy(out, r, sizeof(uint16) * (size_t)(w / 2) * (size_t)(h / 2));
    free(r);
}

/* GetObjectToImageRPC_single for n points; xy_out[2i] = sample, [2i+1] = line. */
void ref_rpc_project(const vll_image_desc *im, long n, const double *lon, const double *lat,
                     const double *hgt, double *xy_out) {
    const double *rows[7] = {im->rpc + 0, im->rpc + 5, im->rpc + 10, im->rpc + 30,
                             im->rpc + 50, im->rpc + 70, im->rpc + 0};
    for (long i = 0; i < n; ++i) {
        D3DPOINT gp(lon[i], lat[i], hgt[i]);
        D2DPOINT ip = GetObjectToImageRPC_single(rows, 2, im->image_adjust, gp);
        xy_out[2 * i] = ip.m_X;
        xy_out[2 * i + 1] = ip.m_Y;
    }
}

void ref_ps2wgs(const vll_transparam *p, long n, const double *xy, double *lonlat) {
    TransParam tp;
    memset(&tp, 0, sizeof(tp));
    memcpy(&tp, p, sizeof(TransParam) < sizeof(*p) ? sizeof(TransParam) : sizeof(*p));
    for (long i = 0; i < n; ++i) {
        D2DPOINT o = ps2wgs_single(tp, D2DPOINT(xy[2 * i], xy[2 * i + 1]));
        lonlat[2 * i] = o.m_X;
        lonlat[2 * i + 1] = o.m_Y;
    }
}

void ref_wgs2ps(const vll_transparam *p, long n, const double *lonlat, double *xy) {
    TransParam tp;
    memset(&tp, 0, sizeof(tp));
    memcpy(&tp, p, sizeof(TransParam) < sizeof(*p) ? sizeof(TransParam) : sizeof(*p));
    for (long i = 0; i < n; ++i) {
        D2DPOINT o = wgs2ps_single(tp, D2DPOINT(lonlat[2 * i], lonlat[2 * i + 1]));
        xy[2 * i] = o.m_X;
        xy[2 * i + 1] = o.m_Y;
    }
}

/* SetTransParam_param (SubFunctions.cpp:1186) for the given hemisphere. */
void ref_set_transparam(int north, int projection, vll_transparam *out) {
    TransParam tp;
    memset(&tp, 0, sizeof(tp));
    tp.projection = projection;
    SetTransParam_param(&tp, north != 0);
    tp.bHemisphere = north ? 1 : 0;
    memset(out, 0, sizeof(*out));
    memcpy(out, &tp, sizeof(TransParam) < sizeof(*out) ? sizeof(TransParam) : sizeof(*out));
}

double ref_get_height_step(int pyramid_step, double im_resolution) {
    return GetHeightStep(pyramid_step, im_resolution);
}

/* VerticalLineLocus_seeddem (setsm_code.cpp:7720-7880): GridPT3 in/out. */
void ref_vll_seeddem(const vll_level_desc *d, vll_ugrid *gridpt3) {
    RefLevel L(d);
    VerticalLineLocus_seeddem(L.proinfo, L.li, reinterpret_cast<UGRID *>(gridpt3),
                              d->minmax_height);
}

/* VerticalLineLocus_blunder (setsm_code.cpp:7882-8026): GridPT3 in/out, the
 * per-node ortho NCC into ncc_out. */
void ref_vll_blunder(const vll_level_desc *d, vll_ugrid *gridpt3, int iteration, int bblunder,
                     float *ncc_out) {
    RefLevel L(d);
    VerticalLineLocus_blunder(L.proinfo, L.li, ncc_out, reinterpret_cast<UGRID *>(gridpt3),
                              (uint8)iteration, bblunder != 0);
}

/* Known-answer hooks: the reference's own building blocks.
 * Correlate, SubFunctions.cpp:974-1018. */
double ref_correlate(const double *L, const double *R, int N) { return Correlate(L, R, N); }

/* Sub-window counts from SetVecKernelValue (SubFunctions.cpp:3249-3315) over
 * the window loop of VerticalLineLocus (setsm_code.cpp:6429-6453), on a
 * constant image so every sample is valid. */
void ref_window_counts(int half, int counts[3]) {
    const int n = 4 * half + 8;
    std::vector<uint16> img((size_t)n * n, 100);
    SetKernel k(0, 1, half);
    KernelPatchArg patch{k, CSize(n, n), CSize(n, n), img.data(), img.data(), img.data(), img.data()};
    int cnt[3] = {0, 0, 0};
    const double c = 0.5 * n + 0.25;
    for (int row = -half; row <= half; row++)
        for (int col = -half; col <= half; col++) {
            const int r2 = row * row + col * col;
            if (r2 <= (half + 1) * (half + 1)) {
                D2DPOINT p(c + col, c + row);
                SetVecKernelValue(patch, row, col, p, p, r2, cnt);
            }
        }
    for (int w = 0; w < 3; ++w) counts[w] = cnt[w];
}

/* Calls a VerticalLineLocus with the reference's exact C++ signature
 * (setsm_code.hpp:81) -- e.g. the drop-in exported by libsetsm_vll.so -- on
 * structures built by the reference's own headers, the way Matching_SETSM
 * calls it (setsm_code.cpp:3829).  Voxels are packed in/out as in
 * ref_vertical_line_locus. */
typedef int (*vll_signature)(VOXEL **, const ProInfo *, NCCresult *, LevelInfo &, const UGRID *,
                             const uint8, const double *);
long ref_call_vertical_line_locus(void *fn, const vll_level_desc *d, const vll_ugrid *gridpt3,
                                  vll_nccresult *ncc, vll_voxel *voxels, long cap) {
    RefLevel L(d);
    const long n = L.grid_length;
    VOXEL **rows = nullptr;
    if (!L.check_matching_rate) rows = unpack_voxels(ncc, n, voxels);
    const int acc = reinterpret_cast<vll_signature>(fn)(
        rows, L.proinfo, reinterpret_cast<NCCresult *>(ncc), L.li,
        reinterpret_cast<const UGRID *>(gridpt3), (uint8)d->iteration, d->minmax_height);
    if (rows) pack_and_free_voxels(ncc, n, rows, voxels, cap);
    return acc;
}

/* Matching_SETSM's voxel-route inner loop (setsm_code.cpp:3743-3844) over
 * `n_iter` iterations on ONE VOXEL** array: InitializeVoxel, VerticalLineLocus
 * and AWNCC per iteration (iteration numbers in iters[]), through the
 * functions at fn_init / fn_vll / fn_awncc (nullptr: the reference's own),
 * rows freed at the end as the caller does (:4581-4585).  gridpt3 and ncc
 * in/out; acc[i] receives each iteration's Accessable_grid. */
void ref_call_voxel_iterations(void *fn_init, void *fn_vll, void *fn_awncc, const vll_level_desc *d,
                               vll_ugrid *gridpt3, vll_nccresult *ncc, int n_iter,
                               const int *iters, long *acc) {
    RefLevel L(d);
    const long n = L.grid_length;
    VOXEL **rows = (VOXEL **)calloc((size_t)n, sizeof(VOXEL *));
    init_voxel_signature fi = fn_init ? reinterpret_cast<init_voxel_signature>(fn_init)
                                      : &InitializeVoxel;
    vll_signature fv = fn_vll ? reinterpret_cast<vll_signature>(fn_vll) : &VerticalLineLocus;
    awncc_signature fa = fn_awncc ? reinterpret_cast<awncc_signature>(fn_awncc) : &AWNCC;
    const int max_voxel = (int)((d->minmax_height[1] - d->minmax_height[0]) / d->height_step);
    for (int k = 0; k < n_iter; ++k) {
        L.iteration = (unsigned char)iters[k];
        fi(L.proinfo, rows, L.li, reinterpret_cast<UGRID *>(gridpt3),
           reinterpret_cast<NCCresult *>(ncc), iters[k], d->minmax_height);
        acc[k] = fv(rows, L.proinfo, reinterpret_cast<NCCresult *>(ncc), L.li,
                    reinterpret_cast<const UGRID *>(gridpt3), (uint8)iters[k], d->minmax_height);
        fa(L.proinfo, rows, L.grid_size, reinterpret_cast<UGRID *>(gridpt3),
           reinterpret_cast<NCCresult *>(ncc), d->height_step, (uint8)d->pyramid_step,
           (uint8)iters[k], max_voxel);
    }
    // InitializeVoxel frees a row without clearing its pointer when the row
    // drops to zero heights; the rows still owned are the NumOfHeight > 0 ones
    // (the release at setsm_code.cpp:4576-4585)
    for (long i = 0; i < n; ++i)
        if (ncc[i].NumOfHeight > 0 && rows[i]) free(rows[i]);
    free(rows);
}

/* VerticalLineLocus_Ortho (setsm_code.cpp:8234-8533) for the triangle
 * three[0..2] = ref1, ref2, target; out = {F_Height, F_sncc} (F_sncc keeps
 * the value passed in out[1] when no height is found); returns its value. */
static D3DPOINT d3(const vll_point3 &p) { return D3DPOINT(p.x, p.y, p.z, p.flag); }
int ref_vll_ortho(const vll_level_desc *d, double mpp, const vll_point3 *three, vll_ugrid *gridpt3,
                  int target_index, double *out) {
    RefLevel L(d);
    double fh = 0, fs = out[1];
    const int r = VerticalLineLocus_Ortho(L.proinfo, L.li, mpp, &fh, d3(three[0]), d3(three[1]),
                                          d3(three[2]), reinterpret_cast<UGRID *>(gridpt3),
                                          target_index, &fs);
    out[0] = fh;
    out[1] = fs;
    return r;
}

/* Ortho_blunder (setsm_code.cpp:8028-8232): pts, tris and GridPT3 in/out. */
int ref_ortho_blunder(const vll_level_desc *d, double mpp, vll_point3 *pts, int n_pts,
                      vll_tri *tris, int n_tris, vll_ugrid *gridpt3) {
    static_assert(sizeof(vll_point3) == sizeof(D3DPOINT), "D3DPOINT layout");
    static_assert(sizeof(vll_tri) == sizeof(UI3DPOINT), "UI3DPOINT layout");
    RefLevel L(d);
    return Ortho_blunder(L.proinfo, L.li, mpp, reinterpret_cast<D3DPOINT *>(pts), n_pts,
                         reinterpret_cast<UI3DPOINT *>(tris), n_tris,
                         reinterpret_cast<UGRID *>(gridpt3));
}

/* The same, through functions with the reference's signatures at `fn` (the
 * library's C++ drop-ins, setsm_code.hpp:97, :118). */
typedef int (*vll_ortho_signature)(ProInfo *, LevelInfo &, double, double *, D3DPOINT, D3DPOINT,
                                   D3DPOINT, UGRID *, int, double *);
typedef int (*ortho_blunder_signature)(ProInfo *, LevelInfo &, double, D3DPOINT *, int,
                                       UI3DPOINT *, int, UGRID *);
int ref_call_vll_ortho(void *fn, const vll_level_desc *d, double mpp, const vll_point3 *three,
                       vll_ugrid *gridpt3, int target_index, double *out) {
    RefLevel L(d);
    double fh = 0, fs = out[1];
    const int r = reinterpret_cast<vll_ortho_signature>(fn)(
        L.proinfo, L.li, mpp, &fh, d3(three[0]), d3(three[1]), d3(three[2]),
        reinterpret_cast<UGRID *>(gridpt3), target_index, &fs);
    out[0] = fh;
    out[1] = fs;
    return r;
}
int ref_call_ortho_blunder(void *fn, const vll_level_desc *d, double mpp, vll_point3 *pts,
                           int n_pts, vll_tri *tris, int n_tris, vll_ugrid *gridpt3) {
    RefLevel L(d);
    return reinterpret_cast<ortho_blunder_signature>(fn)(
        L.proinfo, L.li, mpp, reinterpret_cast<D3DPOINT *>(pts), n_pts,
        reinterpret_cast<UI3DPOINT *>(tris), n_tris, reinterpret_cast<UGRID *>(gridpt3));
}

/* SelectMPs (setsm_code.cpp:8535-8895), or the function at `fn` with its
 * signature; gridpt3 in/out, up to cap points out; returns its value. */
typedef long (*select_mps_signature)(const ProInfo *, LevelInfo &, const NCCresult *, UGRID *,
                                     const double, const double, const double, const double,
                                     const int, const double, const int, const double,
                                     vector<D3DPOINT> *);
long ref_select_mps(void *fn, const vll_level_desc *d, const vll_nccresult *ncc,
                    vll_ugrid *gridpt3, const double *params, const int *iparams,
                    vll_point3 *out, long cap, long *n_out) {
    RefLevel L(d);
    vector<D3DPOINT> v;
    select_mps_signature f = fn ? reinterpret_cast<select_mps_signature>(fn) : &SelectMPs;
    const long r = f(L.proinfo, L.li, reinterpret_cast<const NCCresult *>(ncc),
                     reinterpret_cast<UGRID *>(gridpt3), params[0], params[1], params[2],
                     params[3], iparams[0], params[4], iparams[1], params[5], &v);
    *n_out = (long)v.size();
    for (size_t i = 0; i < v.size() && (long)i < cap; ++i) {
        memset(&out[i], 0, sizeof(vll_point3));
        out[i].x = v[i].m_X;
        out[i].y = v[i].m_Y;
        out[i].z = v[i].m_Z;
        out[i].flag = v[i].flag;
    }
    return r;
}

/* blunder_detection_TIN (setsm_code.cpp:9158-9787), or the function at `fn`
 * with its signature (setsm_code.hpp:116); everything in / out in place,
 * counts[2] and zext[2] (min, max) accumulated as the reference does. */
typedef bool (*tin_blunder_signature)(const ProInfo *, LevelInfo &, const int, float *, bool,
                                      uint16, D3DPOINT *, bool *, long, UI3DPOINT *, long,
                                      UGRID *, long *, double *, double *);
int ref_blunder_detection_tin(void *fn, const vll_level_desc *d, int iteration, float *ortho_ncc,
                              int flag_blunder, int count_bl, double hinterval, vll_point3 *pts,
                              uint8_t *detected, long n_pts, vll_tri *tris, long n_tris,
                              vll_ugrid *gridpt3, long *counts, double *zext) {
    RefLevel L(d);
    L.li.Hinterval = &hinterval;
    tin_blunder_signature f = fn ? reinterpret_cast<tin_blunder_signature>(fn)
                                 : &blunder_detection_TIN;
    static_assert(sizeof(bool) == 1, "bool layout");
    return f(L.proinfo, L.li, iteration, ortho_ncc, flag_blunder != 0, (uint16)count_bl,
             reinterpret_cast<D3DPOINT *>(pts), reinterpret_cast<bool *>(detected), n_pts,
             reinterpret_cast<UI3DPOINT *>(tris), n_tris, reinterpret_cast<UGRID *>(gridpt3),
             counts, &zext[0], &zext[1])
               ? 1
               : 0;
}

/* SetHeightRange (setsm_code.cpp:9851-10255) on a copy of gridpt3 (the
 * reference frees its GridPT3); result and the extent {min, max} out. */
typedef UGRID *(*set_height_range_signature)(ProInfo *, LevelInfo &, NCCresult *, const int,
                                             const int, UGRID *, const int, double *, double *,
                                             D3DPOINT *, const UI3DPOINT *, const double,
                                             const bool);
int ref_set_height_range(void *fn, const vll_level_desc *d, vll_point3 *pts, int n_pts,
                         const vll_tri *tris, int n_tris, const vll_ugrid *gridpt3,
                         vll_ugrid *result, int iteration, double mpp, int lcmr,
                         double seed_sigma, double *extent) {
    RefLevel L(d);
    L.proinfo->seedDEMsigma = seed_sigma;
    const long n = L.grid_length;
    UGRID *g = (UGRID *)malloc(sizeof(UGRID) * (size_t)n);
    memcpy(g, gridpt3, sizeof(UGRID) * (size_t)n);
    set_height_range_signature f = fn ? reinterpret_cast<set_height_range_signature>(fn)
                                      : &SetHeightRange;
    UGRID *r = f(L.proinfo, L.li, nullptr, n_pts, n_tris, g, iteration, &extent[0], &extent[1],
                 reinterpret_cast<D3DPOINT *>(pts), reinterpret_cast<const UI3DPOINT *>(tris),
                 mpp, lcmr != 0);
    memcpy(result, r, sizeof(UGRID) * (size_t)n);
    free(r);
    return 0;
}

/* SetOrthoImageCoord (setsm_code.cpp:6550-6670): the orthoimage coordinate
 * raster of image ti at im_res, OR (use_b = 0) or BD pyramid. */
long ref_ortho_raster(const vll_level_desc *d, const vll_ugrid *gridpt3, int use_b, double im_res,
                      int ti, double *out, long cap) {
    RefLevel L(d);
    D2DPOINT **cd = (D2DPOINT **)calloc((size_t)d->num_images, sizeof(D2DPOINT *));
    long w = 0, h = 0, wn = 0, hn = 0;
    SetOrthoImageCoord(L.proinfo, L.li, reinterpret_cast<const UGRID *>(gridpt3), false,
                       use_b ? BD : OR, im_res, 0, w, h, wn, hn, cd, nullptr);
    const long n = w * h;
    if (n <= cap && cd[ti]) memcpy(out, cd[ti], (size_t)n * sizeof(D2DPOINT));
    for (int i = 0; i < d->num_images; ++i) free(cd[i]);
    free(cd);
    return n <= cap ? n : -n;
}

/* The same structures handed to a function with the signature of
 * VerticalLineLocus_seeddem (setsm_code.hpp:93) / VerticalLineLocus_blunder
 * (:95) at `fn` (the library's C++ drop-ins). */
typedef void (*seeddem_signature)(const ProInfo *, LevelInfo &, UGRID *, const double *);
typedef bool (*blunder_signature)(const ProInfo *, LevelInfo &, float *, UGRID *, uint8, bool);
void ref_call_vll_seeddem(void *fn, const vll_level_desc *d, vll_ugrid *gridpt3) {
    RefLevel L(d);
    reinterpret_cast<seeddem_signature>(fn)(L.proinfo, L.li, reinterpret_cast<UGRID *>(gridpt3),
                                            d->minmax_height);
}
int ref_call_vll_blunder(void *fn, const vll_level_desc *d, vll_ugrid *gridpt3, int iteration,
                         int bblunder, float *ncc_out) {
    RefLevel L(d);
    return reinterpret_cast<blunder_signature>(fn)(L.proinfo, L.li, ncc_out,
                                                   reinterpret_cast<UGRID *>(gridpt3),
                                                   (uint8)iteration, bblunder != 0)
               ? 1
               : 0;
}

/* Byte offsets of the fields the drop-in reads, in the order of the
 * library's vll_compat_layout(), taken from the reference's own headers. */
int ref_layout(int64_t *out, int cap) {
    const int64_t v[] = {
        (int64_t)sizeof(ProInfo),
        (int64_t)offsetof(ProInfo, resolution),
        (int64_t)offsetof(ProInfo, DEM_resolution),
        (int64_t)offsetof(ProInfo, number_of_images),
        (int64_t)offsetof(ProInfo, sensor_type),
        (int64_t)offsetof(ProInfo, IsRA),
        (int64_t)offsetof(ProInfo, pre_DEMtif),
        (int64_t)offsetof(ProInfo, check_Matchtag),
        (int64_t)offsetof(ProInfo, check_selected_image),
        (int64_t)offsetof(ProInfo, SGM_py),
        (int64_t)sizeof(LevelInfo),
        (int64_t)offsetof(LevelInfo, py_Images),
        (int64_t)offsetof(LevelInfo, py_OriImages),
        (int64_t)offsetof(LevelInfo, py_MagImages),
        (int64_t)offsetof(LevelInfo, py_Images_next),
        (int64_t)offsetof(LevelInfo, py_OriImages_next),
        (int64_t)offsetof(LevelInfo, py_MagImages_next),
        (int64_t)offsetof(LevelInfo, py_Startpos),
        (int64_t)offsetof(LevelInfo, py_Startpos_next),
        (int64_t)offsetof(LevelInfo, RPCs),
        (int64_t)offsetof(LevelInfo, Boundary),
        (int64_t)offsetof(LevelInfo, Pyramid_step),
        (int64_t)offsetof(LevelInfo, py_Sizes),
        (int64_t)offsetof(LevelInfo, Template_size),
        (int64_t)offsetof(LevelInfo, ImageAdjust),
        (int64_t)offsetof(LevelInfo, param),
        (int64_t)offsetof(LevelInfo, bin_angle),
        (int64_t)offsetof(LevelInfo, Size_Grid2D),
        (int64_t)offsetof(LevelInfo, GridPts),
        (int64_t)offsetof(LevelInfo, Grid_wgs),
        (int64_t)offsetof(LevelInfo, reference_id),
        (int64_t)offsetof(LevelInfo, height_step),
        (int64_t)offsetof(LevelInfo, grid_resolution),
        (int64_t)offsetof(LevelInfo, Py_combined_level),
        (int64_t)offsetof(LevelInfo, check_matching_rate),
        (int64_t)offsetof(LevelInfo, py_BImages),
        (int64_t)offsetof(LevelInfo, py_BMagImages),
        (int64_t)offsetof(LevelInfo, py_BStartpos),
        (int64_t)offsetof(LevelInfo, blunder_selected_level),
        (int64_t)offsetof(LevelInfo, iteration),
        (int64_t)sizeof(NCCresult),
        (int64_t)sizeof(UGRID),
        (int64_t)offsetof(UGRID, ortho_ncc),
        (int64_t)offsetof(UGRID, Matched_flag),
        (int64_t)sizeof(VOXEL),
        (int64_t)offsetof(VOXEL, INCC),
        (int64_t)sizeof(TransParam),
        (int64_t)offsetof(TransParam, bHemisphere),
        (int64_t)sizeof(D2DPOINT),
        (int64_t)sizeof(CSize),
    };
    const int nv = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < nv && i < cap; ++i) out[i] = v[i];
    return nv;
}

/* TINCreate_list (SubFunctions.cpp:2768-2846): the ordered triangle list of
 * the points (vertex indices); the triangulation object is deleted.  Returns
 * the list's length (the first `cap` triangles are copied out). */
long ref_tin_create(const vll_point3 *pts, long n, const double *min_max, double resolution,
                    vll_tri *out, long cap) {
    D3DPOINT *p = new D3DPOINT[n > 0 ? n : 1];
    for (long i = 0; i < n; ++i) {
        p[i].m_X = pts[i].x;
        p[i].m_Y = pts[i].y;
        p[i].m_Z = pts[i].z;
        p[i].flag = pts[i].flag;
    }
    vector<UI3DPOINT> tris;
    double mm[4] = {min_max[0], min_max[1], min_max[2], min_max[3]};
    int count_tri = 0;
    FullTriangulation *t = TINCreate_list(p, (int)n, &tris, mm, &count_tri, resolution);
    delete t;
    delete[] p;
    for (size_t i = 0; i < tris.size() && (long)i < cap; ++i) {
        out[i].a = tris[i].m_X;
        out[i].b = tris[i].m_Y;
        out[i].c = tris[i].m_Z;
    }
    return (long)tris.size();
}

}  // extern "C"

// vll_shim.cu -- the C++ drop-ins for VerticalLineLocus (setsm_code.hpp:81)
// and its orthoimage variants (:93, :95) on top of the C ABI.  Marshals the caller's ProInfo / LevelInfo into a
// vll_level_desc, packs the VOXEL** rows (voxel route), runs the GPU, unpacks.
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "setsm_vll_compat.hpp"

namespace {

struct ShimState {
    vll_context *ctx = nullptr;
    int kernel = VLL_KERNEL_SPLIT;
    std::vector<vll_voxel> packed;
    bool resident_voxels = false;   // SETSM_VLL_RESIDENT (read per call)
    // The VOXEL** array whose rows the context holds on the device, and the
    // drop-in that last wrote them there.  A session continues only along
    // InitializeVoxel -> VerticalLineLocus -> AWNCC -> InitializeVoxel ... on
    // the same array; any other order (a reference function in between, a
    // new array) falls back to the host rows.
    tagVoxelinfo **session = nullptr;
    int64_t session_nodes = 0;
    enum { kNone, kInit, kVll, kAwncc } last = kNone;
};

ShimState &state() {
    thread_local ShimState s;
    return s;
}

[[noreturn]] void die(const char *what, const char *detail) {
    fprintf(stderr, "setsm_vll: VerticalLineLocus: %s%s%s\n", what, detail ? ": " : "",
            detail ? detail : "");
    fflush(stderr);
    abort();
}

vll_context *shim_context() {
    ShimState &s = state();
    if (!s.ctx) {
        const char *dev = getenv("SETSM_VLL_DEVICE");
        const char *ker = getenv("SETSM_VLL_KERNEL");
        if (ker && strcmp(ker, "plain") == 0) s.kernel = VLL_KERNEL_FP64_PLAIN;
        if (vll_create(dev ? atoi(dev) : 0, &s.ctx) != VLL_OK)
            die("cannot create the GPU context", vll_last_error(nullptr));
    }
    // SETSM_VLL_RESIDENT: unset = image planes and grid arrays stay on the
    // device between calls (re-sent when pointer, size or fingerprint
    // change); "1" = voxel rows also stay there between the InitializeVoxel,
    // VerticalLineLocus and AWNCC drop-ins (when all three replace the
    // reference's, called as Matching_SETSM calls them); "0" = nothing stays
    const char *res = getenv("SETSM_VLL_RESIDENT");
    int flags = VLL_RESIDENT_PLANES;
    if (res && strcmp(res, "0") == 0) flags = 0;
    if (res && strcmp(res, "1") == 0) flags = VLL_RESIDENT_PLANES | VLL_RESIDENT_VOXELS;
    s.resident_voxels = (flags & VLL_RESIDENT_VOXELS) != 0;
    if (vll_get_residency(s.ctx) != flags && vll_set_residency(s.ctx, flags) != VLL_OK)
        die("cannot set residency", vll_last_error(s.ctx));
    return s.ctx;
}

// Fills a level descriptor from the caller's ProInfo / LevelInfo (the fields
// VerticalLineLocus and its orthoimage variants read).
void fill_desc(const ProjectInfo *proinfo, const taglevelinfo &pl, int iteration,
               const double *minmaxHeight, vll_level_desc &d) {
    memset(&d, 0, sizeof(d));
    const int L = *pl.Pyramid_step;
    d.num_images = proinfo->number_of_images;
    d.reference_id = pl.reference_id;
    d.pyramid_step = L;
    d.template_size = *pl.Template_size;
    d.py_combined_level = pl.Py_combined_level ? *pl.Py_combined_level : 0;
    d.iteration = iteration;
    d.check_matching_rate = pl.check_matching_rate && *pl.check_matching_rate ? 1 : 0;
    d.is_ra = proinfo->IsRA;
    d.pre_dem_tif = proinfo->pre_DEMtif;
    d.check_matchtag = proinfo->check_Matchtag;
    d.sgm_py = proinfo->SGM_py;
    d.sensor_type = 0;
    d.resolution = proinfo->resolution;
    d.dem_resolution = proinfo->DEM_resolution;
    d.height_step = pl.height_step ? *pl.height_step : 1.0;
    d.grid_resolution = *pl.grid_resolution;
    d.bin_angle = pl.bin_angle ? *pl.bin_angle : 0.0;
    for (int i = 0; i < 4; ++i) d.boundary[i] = pl.Boundary[i];
    if (minmaxHeight) {
        d.minmax_height[0] = minmaxHeight[0];
        d.minmax_height[1] = minmaxHeight[1];
    }
    d.grid_width = pl.Size_Grid2D->width;
    d.grid_height = pl.Size_Grid2D->height;
    d.grid_pts = reinterpret_cast<const double *>(pl.GridPts);
    d.grid_wgs = reinterpret_cast<const double *>(pl.Grid_wgs);
    memcpy(&d.param, pl.param, sizeof(d.param));
    const bool combined = !proinfo->IsRA && L > d.py_combined_level;
    const int BL = pl.blunder_selected_level ? *pl.blunder_selected_level : L;
    d.blunder_level = BL;
    for (int ti = 0; ti < d.num_images; ++ti) {
        vll_image_desc &im = d.images[ti];
        im.selected = proinfo->check_selected_image[ti] ? 1 : 0;
        if (!im.selected) continue;
        im.image = pl.py_Images ? pl.py_Images[ti] : nullptr;
        im.mag = pl.py_MagImages ? pl.py_MagImages[ti] : nullptr;
        im.ori = pl.py_OriImages ? pl.py_OriImages[ti] : nullptr;
        im.width = pl.py_Sizes[ti][L].width;
        im.height = pl.py_Sizes[ti][L].height;
        if (pl.py_Startpos) {
            im.startpos[0] = pl.py_Startpos[ti].m_X;
            im.startpos[1] = pl.py_Startpos[ti].m_Y;
        }
        if (combined && L >= 1 && pl.py_Images_next) {
            im.image_next = pl.py_Images_next[ti];
            im.mag_next = pl.py_MagImages_next[ti];
            im.ori_next = pl.py_OriImages_next[ti];
            im.width_next = pl.py_Sizes[ti][L - 1].width;
            im.height_next = pl.py_Sizes[ti][L - 1].height;
            if (pl.py_Startpos_next) {
                im.startpos_next[0] = pl.py_Startpos_next[ti].m_X;
                im.startpos_next[1] = pl.py_Startpos_next[ti].m_Y;
            }
        }
        if (pl.py_BImages && pl.py_BMagImages && pl.blunder_selected_level) {
            im.image_b = pl.py_BImages[ti];
            im.mag_b = pl.py_BMagImages[ti];
            im.width_b = pl.py_Sizes[ti][BL].width;
            im.height_b = pl.py_Sizes[ti][BL].height;
            if (pl.py_BStartpos) {
                im.startpos_b[0] = pl.py_BStartpos[ti].m_X;
                im.startpos_b[1] = pl.py_BStartpos[ti].m_Y;
            }
        }
        // RPC rows: offsets[5], scales[5], 4 x 20 coefficients
        const double *const *rpc = pl.RPCs[ti];
        memcpy(im.rpc + 0, rpc[0], 5 * sizeof(double));
        memcpy(im.rpc + 5, rpc[1], 5 * sizeof(double));
        for (int j = 0; j < 4; ++j) memcpy(im.rpc + 10 + 20 * j, rpc[2 + j], 20 * sizeof(double));
        im.image_adjust[0] = pl.ImageAdjust[ti][0];
        im.image_adjust[1] = pl.ImageAdjust[ti][1];
    }
}

void check_sensor(const ProjectInfo *proinfo) {
    if (proinfo->sensor_type != kSensorSB) die("frame (AB) sensors are not supported", nullptr);
    if (proinfo->number_of_images > VLL_MAX_IMAGES) die("too many images", nullptr);
}

}  // namespace

int VerticalLineLocus(tagVoxelinfo **grid_voxel, const ProjectInfo *proinfo,
                      tagNCCresult *nccresult, taglevelinfo &pl, const UpdateGrid *GridPT3,
                      const unsigned char iteration, const double *minmaxHeight) {
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    ShimState &st = state();
    vll_level_desc d;
    fill_desc(proinfo, pl, iteration, minmaxHeight, d);

    const int64_t n = d.grid_width * d.grid_height;
    const bool voxel_route = !d.check_matching_rate && !d.is_ra;
    // within an InitializeVoxel session the rows are on the device already
    const bool in_session = voxel_route && st.resident_voxels && grid_voxel &&
                            grid_voxel == st.session && n == st.session_nodes &&
                            st.last == ShimState::kInit;
    st.last = in_session ? ShimState::kVll : ShimState::kNone;
    vll_voxel *vox = nullptr;
    int64_t nvox = 0;
    if (voxel_route && grid_voxel && !in_session) {
        for (int64_t i = 0; i < n; ++i) nvox += nccresult[i].NumOfHeight;
        st.packed.resize((size_t)(nvox > 0 ? nvox : 1));
        vox = st.packed.data();
        int64_t o = 0;
        for (int64_t i = 0; i < n; ++i) {
            const int k = nccresult[i].NumOfHeight;
            if (k > 0) {
                memcpy(vox + o, grid_voxel[i], (size_t)k * sizeof(vll_voxel));
                o += k;
            }
        }
    }
    vll_stats stats;
    const int rc = vll_vertical_line_locus(ctx, &d, reinterpret_cast<const vll_ugrid *>(GridPT3),
                                           reinterpret_cast<vll_nccresult *>(nccresult), vox, nvox,
                                           st.kernel, &stats);
    if (rc != VLL_OK) die("GPU call failed", vll_last_error(ctx));
    if (vox) {
        int64_t o = 0;
        for (int64_t i = 0; i < n; ++i) {
            const int k = nccresult[i].NumOfHeight;
            if (k > 0) {
                memcpy(grid_voxel[i], vox + o, (size_t)k * sizeof(vll_voxel));
                o += k;
            }
        }
    }
    return (int)stats.accessable_grid;
}

void VerticalLineLocus_seeddem(const ProjectInfo *proinfo, taglevelinfo &pl, UpdateGrid *GridPT3,
                               const double *minmaxHeight) {
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    vll_level_desc d;
    fill_desc(proinfo, pl, pl.iteration ? *pl.iteration : 1, minmaxHeight, d);
    if (vll_vertical_line_locus_seeddem(ctx, &d, reinterpret_cast<vll_ugrid *>(GridPT3), nullptr) !=
        VLL_OK)
        die("VerticalLineLocus_seeddem: GPU call failed", vll_last_error(ctx));
}

bool VerticalLineLocus_blunder(const ProjectInfo *proinfo, taglevelinfo &pl, float *nccresult,
                               UpdateGrid *GridPT3, unsigned char iteration, bool bblunder) {
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    vll_level_desc d;
    fill_desc(proinfo, pl, iteration, nullptr, d);
    if (vll_vertical_line_locus_blunder(ctx, &d, reinterpret_cast<vll_ugrid *>(GridPT3), iteration,
                                        bblunder ? 1 : 0, nccresult, nullptr) != VLL_OK)
        die("VerticalLineLocus_blunder: GPU call failed", vll_last_error(ctx));
    return true;
}

static vll_point3 point_of(const tagD3DPoint &p) {
    vll_point3 q;
    memset(&q, 0, sizeof(q));
    q.x = p.m_X;
    q.y = p.m_Y;
    q.z = p.m_Z;
    q.flag = p.flag;
    return q;
}

int VerticalLineLocus_Ortho(ProjectInfo *proinfo, taglevelinfo &pl, double MPP, double *F_Height,
                            tagD3DPoint ref1_pt, tagD3DPoint ref2_pt, tagD3DPoint target_pt,
                            UpdateGrid *GridPT3, int target_index, double *F_sncc) {
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    vll_level_desc d;
    fill_desc(proinfo, pl, pl.iteration ? *pl.iteration : 1, nullptr, d);
    const vll_point3 r1 = point_of(ref1_pt), r2 = point_of(ref2_pt), tg = point_of(target_pt);
    int selected = 0;
    if (vll_vertical_line_locus_ortho(ctx, &d, MPP, &r1, &r2, &tg,
                                      reinterpret_cast<const vll_ugrid *>(GridPT3), target_index,
                                      F_Height, F_sncc, &selected) != VLL_OK)
        die("VerticalLineLocus_Ortho: GPU call failed", vll_last_error(ctx));
    return selected;
}

int Ortho_blunder(ProjectInfo *proinfo, taglevelinfo &pl, double MPP, tagD3DPoint *pts,
                  int numOfPts, tagUI3DPoint *tris, int numOfTri, UpdateGrid *GridPT3) {
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    vll_level_desc d;
    fill_desc(proinfo, pl, pl.iteration ? *pl.iteration : 1, nullptr, d);
    if (vll_ortho_blunder(ctx, &d, MPP, reinterpret_cast<vll_point3 *>(pts), numOfPts,
                          reinterpret_cast<const vll_tri *>(tris), numOfTri,
                          reinterpret_cast<vll_ugrid *>(GridPT3), nullptr) != VLL_OK)
        die("Ortho_blunder: GPU call failed", vll_last_error(ctx));
    return numOfPts;
}

void InitializeVoxel(const ProjectInfo *proinfo, tagVoxelinfo **grid_voxel, taglevelinfo &pl,
                     UpdateGrid *GridPT3, tagNCCresult *nccresult, const int iteration,
                     const double *minmaxHeight) {
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    ShimState &st = state();
    vll_level_desc d;
    fill_desc(proinfo, pl, iteration, minmaxHeight, d);
    const int64_t n = d.grid_width * d.grid_height;
    std::vector<uint16_t> old_n((size_t)n);
    int64_t cap = 1;
    for (int64_t i = 0; i < n; ++i) {
        old_n[(size_t)i] = nccresult[i].NumOfHeight;
        const int64_t span = (int64_t)GridPT3[i].maxHeight - GridPT3[i].minHeight +
                             (int64_t)nccresult[i].maxHeight - nccresult[i].minHeight;
        cap += (int64_t)((span < 0 ? -span : span) / d.height_step) + 8 + old_n[(size_t)i];
    }
    int64_t total = 0;
    if (st.resident_voxels) {
        // a new VOXEL** array starts a new session; rows it already holds
        // (carried over by the reference) start the device packing
        const vll_voxel *vin = nullptr;
        if (grid_voxel != st.session || n != st.session_nodes || st.last != ShimState::kAwncc) {
            vll_resident_reset(ctx);
            st.session = grid_voxel;
            st.session_nodes = n;
            int64_t old_total = 0;
            for (int64_t i = 0; i < n; ++i) old_total += old_n[(size_t)i];
            if (old_total > 0) {
                st.packed.resize((size_t)old_total);
                int64_t o = 0;
                for (int64_t i = 0; i < n; ++i) {
                    const int k = old_n[(size_t)i];
                    if (k <= 0) continue;
                    if (grid_voxel[i])
                        memcpy(st.packed.data() + o, grid_voxel[i], (size_t)k * sizeof(vll_voxel));
                    else
                        memset(st.packed.data() + o, 0, (size_t)k * sizeof(vll_voxel));
                    o += k;
                }
                vin = st.packed.data();
            }
        }
        if (vll_initialize_voxel(ctx, &d, reinterpret_cast<vll_ugrid *>(GridPT3),
                                 reinterpret_cast<vll_nccresult *>(nccresult), vin, nullptr, 0,
                                 &total) != VLL_OK)
            die("InitializeVoxel: GPU call failed", vll_last_error(ctx));
        st.last = ShimState::kInit;
    }
    // the rows are rebuilt here from the new NumOfHeight, so no old rows go up
    for (int attempt = 0; attempt < 2 && !st.resident_voxels; ++attempt) {
        st.packed.resize((size_t)cap);
        const int rc = vll_initialize_voxel(ctx, &d, reinterpret_cast<vll_ugrid *>(GridPT3),
                                            reinterpret_cast<vll_nccresult *>(nccresult), nullptr,
                                            st.packed.data(), cap, &total);
        if (rc == VLL_OK) break;
        if (rc != VLL_ERR_CAPACITY || attempt == 1)
            die("InitializeVoxel: GPU call failed", vll_last_error(ctx));
        cap = total;
    }
    // the reference's row management: a row whose range changed is freed and
    // reallocated with (flag_cal, INCC -1000) voxels, a row that drops to zero
    // heights is freed, the others are kept as they are
    for (int64_t i = 0; i < n; ++i) {
        const int k = nccresult[i].NumOfHeight;
        const int k0 = old_n[(size_t)i];
        if (k > 0 && nccresult[i].check_height_change) {
            if (k0 > 0 && grid_voxel[i]) free(grid_voxel[i]);
            grid_voxel[i] = (tagVoxelinfo *)calloc((size_t)k, sizeof(tagVoxelinfo));
            if (!grid_voxel[i]) die("InitializeVoxel: out of memory", nullptr);
            for (int h = 0; h < k; ++h) {
                grid_voxel[i][h].flag_cal = true;
                grid_voxel[i][h].INCC = -1000;
            }
        } else if (k == 0 && k0 > 0 && grid_voxel[i]) {
            free(grid_voxel[i]);
        }
    }
}

void AWNCC(ProjectInfo *proinfo, tagVoxelinfo **grid_voxel, tagCSize Size_Grid2D,
           UpdateGrid *GridPT3, tagNCCresult *nccresult, double step_height,
           unsigned char Pyramid_step, unsigned char iteration, int MaxNumberofHeightVoxel) {
    (void)MaxNumberofHeightVoxel;   // sizes the reference's own buffers only
    check_sensor(proinfo);
    vll_context *ctx = shim_context();
    ShimState &st = state();
    // AWNCC reads no image: the descriptor carries the level, the iteration,
    // the switches and the grid; selected images get placeholder sizes
    vll_level_desc d;
    memset(&d, 0, sizeof(d));
    d.num_images = proinfo->number_of_images;
    d.pyramid_step = Pyramid_step;
    d.template_size = 11;
    d.iteration = iteration;
    d.is_ra = proinfo->IsRA;
    d.check_matchtag = proinfo->check_Matchtag;
    d.sgm_py = proinfo->SGM_py;
    d.resolution = proinfo->resolution;
    d.dem_resolution = proinfo->DEM_resolution;
    d.height_step = step_height;
    d.grid_width = Size_Grid2D.width;
    d.grid_height = Size_Grid2D.height;
    for (int ti = 0; ti < d.num_images && ti < VLL_MAX_IMAGES; ++ti) {
        d.images[ti].selected = proinfo->check_selected_image[ti] ? 1 : 0;
        d.images[ti].width = d.images[ti].height = 2;
    }
    const int64_t n = d.grid_width * d.grid_height;
    const bool in_session = st.resident_voxels && grid_voxel && grid_voxel == st.session &&
                            n == st.session_nodes && st.last == ShimState::kVll;
    st.last = in_session ? ShimState::kAwncc : ShimState::kNone;
    int64_t nvox = 0;
    if (!in_session) {
        for (int64_t i = 0; i < n; ++i) nvox += nccresult[i].NumOfHeight;
        st.packed.resize((size_t)(nvox > 0 ? nvox : 1));
        int64_t o = 0;
        for (int64_t i = 0; i < n; ++i) {
            const int k = nccresult[i].NumOfHeight;
            if (k > 0) {
                memcpy(st.packed.data() + o, grid_voxel[i], (size_t)k * sizeof(vll_voxel));
                o += k;
            }
        }
    }
    if (vll_awncc_peaks(ctx, &d, reinterpret_cast<const vll_ugrid *>(GridPT3),
                        reinterpret_cast<vll_nccresult *>(nccresult),
                        in_session ? nullptr : st.packed.data(), nvox, nullptr) != VLL_OK)
        die("AWNCC: GPU call failed", vll_last_error(ctx));
}

bool blunder_detection_TIN(const ProjectInfo *proinfo, taglevelinfo &pl, const int iteration,
                           float *ortho_ncc, bool flag_blunder, unsigned short count_bl,
                           tagD3DPoint *pts, bool *detectedBlunders, long num_points,
                           tagUI3DPoint *tris, long num_triangles, UpdateGrid *Gridpts,
                           long *blunder_count, double *minz_mp, double *maxz_mp) {
    vll_context *ctx = shim_context();
    vll_level_desc d;
    memset(&d, 0, sizeof(d));
    d.pyramid_step = *pl.Pyramid_step;
    d.is_ra = proinfo->IsRA;
    d.grid_resolution = *pl.grid_resolution;
    for (int i = 0; i < 4; ++i) d.boundary[i] = pl.Boundary[i];
    d.grid_width = pl.Size_Grid2D->width;
    d.grid_height = pl.Size_Grid2D->height;
    int64_t counts[2] = {blunder_count[0], blunder_count[1]};
    static_assert(sizeof(bool) == sizeof(uint8_t), "bool layout");
    if (vll_blunder_detection_tin(ctx, &d, iteration, ortho_ncc, flag_blunder ? 1 : 0, count_bl,
                                  pl.Hinterval ? *pl.Hinterval : 0.0,
                                  reinterpret_cast<vll_point3 *>(pts),
                                  reinterpret_cast<uint8_t *>(detectedBlunders), num_points,
                                  reinterpret_cast<const vll_tri *>(tris), num_triangles,
                                  reinterpret_cast<vll_ugrid *>(Gridpts), counts, minz_mp,
                                  maxz_mp) != VLL_OK)
        die("blunder_detection_TIN: GPU call failed", vll_last_error(ctx));
    blunder_count[0] = (long)counts[0];
    blunder_count[1] = (long)counts[1];
    return true;
}

long SelectMPs(const ProjectInfo *proinfo, taglevelinfo &pl, const tagNCCresult *roh_height,
               UpdateGrid *GridPT3, const double Th_roh, const double Th_roh_min,
               const double Th_roh_start, const double Th_roh_next, const int iteration,
               const double MPP, const int final_level_iteration, const double MPP_stereo_angle,
               std::vector<tagD3DPoint> *linkedlist) {
    vll_context *ctx = shim_context();
    vll_level_desc d;
    memset(&d, 0, sizeof(d));
    d.num_images = proinfo->number_of_images;
    d.pyramid_step = *pl.Pyramid_step;
    d.is_ra = proinfo->IsRA;
    d.sgm_py = proinfo->SGM_py;
    d.grid_width = pl.Size_Grid2D->width;
    d.grid_height = pl.Size_Grid2D->height;
    d.grid_pts = reinterpret_cast<const double *>(pl.GridPts);
    const int64_t n = d.grid_width * d.grid_height;
    std::vector<vll_point3> pts((size_t)(n > 0 ? n : 1));
    int64_t count = 0;
    if (vll_select_mps(ctx, &d, reinterpret_cast<const vll_nccresult *>(roh_height),
                       reinterpret_cast<vll_ugrid *>(GridPT3), Th_roh, Th_roh_min, Th_roh_start,
                       Th_roh_next, iteration, MPP, final_level_iteration, MPP_stereo_angle,
                       pts.data(), n, &count) != VLL_OK)
        die("SelectMPs: GPU call failed", vll_last_error(ctx));
    for (int64_t i = 0; i < count; ++i) {
        tagD3DPoint p;
        p.m_X = pts[(size_t)i].x;
        p.m_Y = pts[(size_t)i].y;
        p.m_Z = pts[(size_t)i].z;
        p.flag = pts[(size_t)i].flag;
        linkedlist->push_back(p);
    }
    return (long)count;
}

UpdateGrid *SetHeightRange(ProjectInfo *proinfo, taglevelinfo &pl, tagNCCresult *nccresult,
                           const int numOfPts, const int num_triangles, UpdateGrid *GridPT3,
                           const int iteration, double *minH_grid, double *maxH_grid,
                           tagD3DPoint *pts, const tagUI3DPoint *tris, const double MPP,
                           const bool level_check_matching_rate) {
    (void)nccresult;   // not read by the reference either
    vll_context *ctx = shim_context();
    vll_level_desc d;
    memset(&d, 0, sizeof(d));
    d.num_images = proinfo->number_of_images;
    d.reference_id = pl.reference_id;
    d.pyramid_step = *pl.Pyramid_step;
    d.pre_dem_tif = proinfo->pre_DEMtif;
    d.resolution = proinfo->resolution;
    d.dem_resolution = proinfo->DEM_resolution;
    d.grid_resolution = *pl.grid_resolution;
    for (int i = 0; i < 4; ++i) d.boundary[i] = pl.Boundary[i];
    d.grid_width = pl.Size_Grid2D->width;
    d.grid_height = pl.Size_Grid2D->height;
    for (int ti = 0; ti < d.num_images && ti < VLL_MAX_IMAGES; ++ti)
        d.images[ti].selected = proinfo->check_selected_image[ti] ? 1 : 0;
    const int64_t n = d.grid_width * d.grid_height;
    UpdateGrid *result = (UpdateGrid *)calloc((size_t)n, sizeof(UpdateGrid));
    if (!result) die("SetHeightRange: out of memory", nullptr);
    if (vll_set_height_range(ctx, &d, reinterpret_cast<const vll_point3 *>(pts), numOfPts,
                             reinterpret_cast<const vll_tri *>(tris), num_triangles,
                             reinterpret_cast<vll_ugrid *>(GridPT3),
                             reinterpret_cast<vll_ugrid *>(result), iteration, MPP,
                             level_check_matching_rate ? 1 : 0, proinfo->seedDEMsigma, minH_grid,
                             maxH_grid) != VLL_OK)
        die("SetHeightRange: GPU call failed", vll_last_error(ctx));
    free(GridPT3);
    return result;
}

extern "C" int vll_compat_layout(int64_t *out, int cap) {
    const int64_t v[] = {
        (int64_t)sizeof(ProjectInfo),
        (int64_t)offsetof(ProjectInfo, resolution),
        (int64_t)offsetof(ProjectInfo, DEM_resolution),
        (int64_t)offsetof(ProjectInfo, number_of_images),
        (int64_t)offsetof(ProjectInfo, sensor_type),
        (int64_t)offsetof(ProjectInfo, IsRA),
        (int64_t)offsetof(ProjectInfo, pre_DEMtif),
        (int64_t)offsetof(ProjectInfo, check_Matchtag),
        (int64_t)offsetof(ProjectInfo, check_selected_image),
        (int64_t)offsetof(ProjectInfo, SGM_py),
        (int64_t)sizeof(taglevelinfo),
        (int64_t)offsetof(taglevelinfo, py_Images),
        (int64_t)offsetof(taglevelinfo, py_OriImages),
        (int64_t)offsetof(taglevelinfo, py_MagImages),
        (int64_t)offsetof(taglevelinfo, py_Images_next),
        (int64_t)offsetof(taglevelinfo, py_OriImages_next),
        (int64_t)offsetof(taglevelinfo, py_MagImages_next),
        (int64_t)offsetof(taglevelinfo, py_Startpos),
        (int64_t)offsetof(taglevelinfo, py_Startpos_next),
        (int64_t)offsetof(taglevelinfo, RPCs),
        (int64_t)offsetof(taglevelinfo, Boundary),
        (int64_t)offsetof(taglevelinfo, Pyramid_step),
        (int64_t)offsetof(taglevelinfo, py_Sizes),
        (int64_t)offsetof(taglevelinfo, Template_size),
        (int64_t)offsetof(taglevelinfo, ImageAdjust),
        (int64_t)offsetof(taglevelinfo, param),
        (int64_t)offsetof(taglevelinfo, bin_angle),
        (int64_t)offsetof(taglevelinfo, Size_Grid2D),
        (int64_t)offsetof(taglevelinfo, GridPts),
        (int64_t)offsetof(taglevelinfo, Grid_wgs),
        (int64_t)offsetof(taglevelinfo, reference_id),
        (int64_t)offsetof(taglevelinfo, height_step),
        (int64_t)offsetof(taglevelinfo, grid_resolution),
        (int64_t)offsetof(taglevelinfo, Py_combined_level),
        (int64_t)offsetof(taglevelinfo, check_matching_rate),
        (int64_t)offsetof(taglevelinfo, py_BImages),
        (int64_t)offsetof(taglevelinfo, py_BMagImages),
        (int64_t)offsetof(taglevelinfo, py_BStartpos),
        (int64_t)offsetof(taglevelinfo, blunder_selected_level),
        (int64_t)offsetof(taglevelinfo, iteration),
        (int64_t)sizeof(tagNCCresult),
        (int64_t)sizeof(UpdateGrid),
        (int64_t)offsetof(UpdateGrid, ortho_ncc),
        (int64_t)offsetof(UpdateGrid, Matched_flag),
        (int64_t)sizeof(tagVoxelinfo),
        (int64_t)offsetof(tagVoxelinfo, INCC),
        (int64_t)sizeof(tagTransParam),
        (int64_t)offsetof(tagTransParam, bHemisphere),
        (int64_t)sizeof(tagD2DPoint),
        (int64_t)sizeof(tagCSize),
    };
    const int nv = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < nv && i < cap; ++i) out[i] = v[i];
    return nv;
}

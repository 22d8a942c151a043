// setsm_vll_compat.hpp -- the C++ drop-in for SETSM's VerticalLineLocus.
//
// SETSM calls
//   int VerticalLineLocus(VOXEL **grid_voxel, const ProInfo *proinfo,
//                         NCCresult *nccresult, LevelInfo &plevelinfo,
//                         const UGRID *GridPT3, const uint8 iteration,
//                         const double *minmaxHeight);
// (setsm_code.hpp:81, setsm_code.cpp:6049).  libsetsm_vll.so exports a
// function with exactly that C++ signature and mangled name, implemented on
// the C ABI of setsm_vll.h.  To produce the same mangled name and read the
// caller's structures, this header declares the reference's record types
// under their own tag names with the same member types and order
// (Typedefine.hpp:93-293, :311-419, :604-643).  Only the layout matters;
// tests/test_abi_layout.py checks every offset against the reference headers.
#ifndef SETSM_VLL_COMPAT_HPP
#define SETSM_VLL_COMPAT_HPP

#include <cstdint>
#include <vector>

#include "setsm_vll.h"

namespace setsm_compat {
constexpr int kMaxImages = 100;   // MaxImages, Typedefine.hpp:29
constexpr int kMaxNcc = 2;        // MaxNCC, Typedefine.hpp:30
}  // namespace setsm_compat

struct tagD2DPoint {
    double m_X;
    double m_Y;
};

// With a user-written copy constructor, as the reference's (a CSize passed
// by value -- AWNCC's Size_Grid2D -- travels by hidden reference).
struct tagCSize {
    unsigned int width;
    unsigned int height;
    tagCSize() : width(0), height(0) {}
    tagCSize(const tagCSize &s) : width(s.width), height(s.height) {}
};

struct tagTransParam {
    double t_c, m_c;
    double sa, sb, e2, e2cuadrada, c;
    double a, e;
    double phi_c, lambda_0;
    int pm;
    int projection;
    int utm_zone;
    char direction[2];
    int bHemisphere;
};

struct tagNCCresult {
    float result2;
    float result3;
    short minHeight;
    short maxHeight;
    short result0;
    short result1;
    short max_WNCC;
    short GNCC;
    unsigned short NumOfHeight;
    unsigned char result4;
    bool check_height_change;
};

struct UpdateGrid {
    float Height;
    short minHeight;
    short maxHeight;
    short roh;
    short ortho_ncc[setsm_compat::kMaxNcc];
    short Mean_ortho_ncc;
    unsigned char Matched_flag;
    unsigned char anchor_flag;
};

struct tagVoxelinfo {
    bool flag_cal;
    short INCC;
};

struct tagCameraInfo {
    double m_focalLength;
    tagCSize m_ImageSize;
    double m_CCDSize;
    double m_ppx;
    double m_ppy;
};

struct tagRotationMatrix {
    double m11, m12, m13, m21, m22, m23, m31, m32, m33;
};

struct tagEO {
    int strip_ID;
    int photo_ID;
    char path[500];
    double m_Xl, m_Yl, m_Zl, m_Wl, m_Pl, m_Kl;
    tagRotationMatrix m_Rm;
};

struct tagFrameInfo {
    tagCameraInfo m_Camera;
    int NumberofStip;
    int NumberofPhotos;
    int start_stripID;
    int end_stripID;
    tagEO *Photoinfo;
};

enum SetsmSensorType { kSensorSB = 0, kSensorAB = 1 };   // enum SensorType {SB, AB}

struct ProjectInfo {
    double resolution;
    double DEM_resolution;
    double preDEM_space;
    double cal_boundary[4];
    double RA_param[setsm_compat::kMaxImages][2];
    double seedDEMsigma;
    double LBoundary[4];
    double RBoundary[4];
    double GCP_spacing;
    double minHeight;
    double maxHeight;
    double System_memory;
    int start_row;
    int end_row;
    int start_col;
    int end_col;
    int threads_num;
    int number_of_images;
    SetsmSensorType sensor_type;
    unsigned char pyramid_level;
    unsigned char end_level;
    unsigned char SDM_SS;
    double SDM_AS;
    double SDM_days;
    unsigned char image_bits;
    char Imagefilename[setsm_compat::kMaxImages][500];
    char RPCfilename[setsm_compat::kMaxImages][500];
    char save_filepath[500];
    char Outputpath_name[500];
    char tmpdir[500];
    char tile_info[500];
    char priori_DEM_tif[500];
    char metafilename[500];
    bool check_minH, check_maxH, check_tiles_SR, check_tiles_ER, check_tiles_SC, check_tiles_EC;
    bool check_gridonly, check_boundary, check_checktiff, check_ortho;
    bool IsRA, IsSP, IsRR, IsSaveStep, Overall_DEM, Affine_RA, pre_DEMtif, check_tile_array;
    bool check_Matchtag;
    bool check_selected_image[setsm_compat::kMaxImages];
    bool check_full_cal;
    bool check_tif_rounding;
    bool check_SNCC, check_updateheight, check_blunderdetection, check_NCCpeak, check_minTH;
    bool check_adaptive_P2, check_orthoblunder, check_8d;
    int SGM_py;
    tagFrameInfo frameinfo;
    unsigned char SPnumber[2], NumOfTile_row, NumOfTile_col;
};

struct taglevelinfo {
    const uint16_t *const *py_Images;
    const uint8_t *const *py_OriImages;
    const uint16_t *const *py_MagImages;
    const uint16_t *const *py_BImages;
    const uint16_t *const *py_BMagImages;
    const uint16_t *const *py_Images_next;
    const uint8_t *const *py_OriImages_next;
    const uint16_t *const *py_MagImages_next;
    const tagD2DPoint *py_Startpos;
    const tagD2DPoint *py_BStartpos;
    const tagD2DPoint *py_Startpos_next;
    const double *const *const *RPCs;
    const double *Boundary;
    const int *Pyramid_step;
    const tagCSize *const *py_Sizes;
    const unsigned char *Template_size;
    const double *const *ImageAdjust;
    const tagTransParam *param;
    const unsigned char *NumOfIAparam;
    const double *bin_angle;
    const int *blunder_selected_level;
    const tagCSize *Size_Grid2D;
    const long *Grid_length;
    const tagD2DPoint *GridPts;
    const tagD2DPoint *Grid_wgs;
    int reference_id;
    const double *height_step;
    const double *grid_resolution;
    const double *Hinterval;
    const int *Py_combined_level;
    const unsigned char *iteration;
    bool *check_matching_rate;
};

static_assert(sizeof(tagNCCresult) == sizeof(vll_nccresult), "NCCresult layout");
static_assert(sizeof(UpdateGrid) == sizeof(vll_ugrid), "UGRID layout");
static_assert(sizeof(tagVoxelinfo) == sizeof(vll_voxel), "VOXEL layout");
static_assert(sizeof(tagTransParam) == sizeof(vll_transparam), "TransParam layout");

// The drop-in (setsm_code.hpp:81).  Runs on the GPU selected by
// SETSM_VLL_DEVICE (default 0) with the kernel selected by SETSM_VLL_KERNEL
// ("split", the default, or "plain").  Unsupported inputs (frame sensors)
// and CUDA failures terminate with a message on stderr, like the reference's
// own error handling; there is no CPU path.
int VerticalLineLocus(tagVoxelinfo **grid_voxel, const ProjectInfo *proinfo,
                      tagNCCresult *nccresult, taglevelinfo &plevelinfo, const UpdateGrid *GridPT3,
                      const unsigned char iteration, const double *minmaxHeight);

// D3DPOINT and UI3DPOINT (Typedefine.hpp:74-97, :139-194).  D3DPOINT has a
// user-written copy constructor in the reference, so a D3DPOINT passed by
// value travels by hidden reference; this one must have one too.
struct tagD3DPoint {
    double m_X, m_Y, m_Z;
    unsigned char flag;
    tagD3DPoint() : m_X(0), m_Y(0), m_Z(0), flag(0) {}
    tagD3DPoint(const tagD3DPoint &p) : m_X(p.m_X), m_Y(p.m_Y), m_Z(p.m_Z), flag(p.flag) {}
};
struct tagUI3DPoint {
    uint32_t m_X, m_Y, m_Z;
    tagUI3DPoint() : m_X(0), m_Y(0), m_Z(0) {}
    tagUI3DPoint(const tagUI3DPoint &p) : m_X(p.m_X), m_Y(p.m_Y), m_Z(p.m_Z) {}
};
static_assert(sizeof(tagD3DPoint) == sizeof(vll_point3), "D3DPOINT layout");
static_assert(sizeof(tagUI3DPoint) == sizeof(vll_tri), "UI3DPOINT layout");

// The TIN-triangle height search and its driver (setsm_code.hpp:97, :118),
// same behaviour: VerticalLineLocus_Ortho returns the selected sample count
// and writes *F_Height (-9999 when none) and *F_sncc (when found);
// Ortho_blunder updates pts, GridPT3 in place and returns numOfPts.
int VerticalLineLocus_Ortho(ProjectInfo *proinfo, taglevelinfo &plevelinfo, double MPP,
                            double *F_Height, tagD3DPoint ref1_pt, tagD3DPoint ref2_pt,
                            tagD3DPoint target_pt, UpdateGrid *GridPT3, int target_index,
                            double *F_sncc);
int Ortho_blunder(ProjectInfo *proinfo, taglevelinfo &plevelinfo, double MPP, tagD3DPoint *pts,
                  int numOfPts, tagUI3DPoint *tris, int numOfTri, UpdateGrid *GridPT3);
// InitializeVoxel (setsm_code.hpp:75) and AWNCC (:91), same behaviour:
// InitializeVoxel frees and (re)allocates grid_voxel rows as the reference
// does; AWNCC reads the rows and writes the peaks.
void InitializeVoxel(const ProjectInfo *proinfo, tagVoxelinfo **grid_voxel,
                     taglevelinfo &plevelinfo, UpdateGrid *GridPT3, tagNCCresult *nccresult,
                     const int iteration, const double *minmaxHeight);
void AWNCC(ProjectInfo *proinfo, tagVoxelinfo **grid_voxel, tagCSize Size_Grid2D,
           UpdateGrid *GridPT3, tagNCCresult *nccresult, double step_height,
           unsigned char Pyramid_step, unsigned char iteration, int MaxNumberofHeightVoxel);
// blunder_detection_TIN (setsm_code.hpp:116), same behaviour; returns true.
bool blunder_detection_TIN(const ProjectInfo *proinfo, taglevelinfo &plevelinfo,
                           const int iteration, float *ortho_ncc, bool flag_blunder,
                           unsigned short count_bl, tagD3DPoint *pts, bool *detectedBlunders,
                           long num_points, tagUI3DPoint *tris, long num_triangles,
                           UpdateGrid *Gridpts, long *blunder_count, double *minz_mp,
                           double *maxz_mp);
// SelectMPs (setsm_code.hpp:99), same behaviour: appends the matched points
// to *linkedlist, updates GridPT3, returns their number.
long SelectMPs(const ProjectInfo *proinfo, taglevelinfo &plevelinfo,
               const tagNCCresult *roh_height, UpdateGrid *GridPT3, const double Th_roh,
               const double Th_roh_min, const double Th_roh_start, const double Th_roh_next,
               const int iteration, const double MPP, const int final_level_iteration,
               const double MPP_stereo_angle, std::vector<tagD3DPoint> *linkedlist);
// SetHeightRange (setsm_code.hpp:122), same behaviour: returns a new grid
// (calloc) and frees GridPT3, which must come from malloc / calloc.
UpdateGrid *SetHeightRange(ProjectInfo *proinfo, taglevelinfo &plevelinfo,
                           tagNCCresult *nccresult, const int numOfPts, const int num_triangles,
                           UpdateGrid *GridPT3, const int iteration, double *minH_grid,
                           double *maxH_grid, tagD3DPoint *pts, const tagUI3DPoint *tris,
                           const double MPP, const bool level_check_matching_rate);

// The orthoimage-window variants (setsm_code.hpp:93, :95), same behaviour:
// VerticalLineLocus_seeddem updates GridPT3; VerticalLineLocus_blunder
// writes GridPT3's ortho NCC and nccresult[node], and returns true.
void VerticalLineLocus_seeddem(const ProjectInfo *proinfo, taglevelinfo &plevelinfo,
                               UpdateGrid *GridPT3, const double *minmaxHeight);
bool VerticalLineLocus_blunder(const ProjectInfo *proinfo, taglevelinfo &plevelinfo,
                               float *nccresult, UpdateGrid *GridPT3, unsigned char iteration,
                               bool bblunder);

extern "C" {
// Byte offsets of the fields the drop-in reads, in a fixed order (used by the
// layout test); returns the number of entries written.
int vll_compat_layout(int64_t *out, int cap);
}

#endif

// vll_device.cuh -- device-side building blocks shared by every kernel of the
// vertical-line-locus path (sm_100a).
//
// Exactness: every FP64 operation that the reference performs on the path
// (RPC, pyramid shift, bilinear sampling, Pearson sums) is written with
// explicit round-to-nearest intrinsics (__dmul_rn, __dadd_rn, ...), which the
// compiler never fuses into FMAs.  Together with IEEE division and square root
// that reproduces the x86-64 reference bit for bit, whatever -fmad setting the
// including translation unit uses.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "setsm_vll.h"

namespace vll {

constexpr double kPi = 3.141592653589793;
constexpr int kMaxHalf = 8;          // largest window half-size supported (17x17)
// cos/sin of the window rotation for every possible orientation difference:
// diff_theta = (i - kRotOffset) / 2 covers uint8 differences and their halves.
constexpr int kRotOffset = 510;
constexpr int kRotTable = 2 * kRotOffset + 1;

// One image at the matched level (+ the next finer level in combined mode).
struct DevImage {
    const uint16_t *img, *mag;
    const uint8_t *ori;
    const uint16_t *img_n, *mag_n;
    const uint8_t *ori_n;
    uint32_t w, h, wn, hn;
    double sx, sy, sxn, syn;        // py_Startpos, py_Startpos_next
    double rpc[90];
    double adj[2];
    int selected;
    int pad_;
    // the blunder-selected pyramid level (VerticalLineLocus_blunder / _seeddem)
    const uint16_t *img_b, *mag_b;
    uint32_t wb, hb;
    double sxb, syb;
};

// Everything one VerticalLineLocus call needs on the device.  Lives in device
// global memory (too large for kernel parameters with 8 images).
struct DevLevel {
    int num_images, ref, L, H;
    int iteration, cmr, is_ra, check_matchtag;
    int combined, combined_incc, check_ortho, sgm_py;
    int pre_dem_tif, blunder_level;
    double alpha, beta, ortho_th, th_height;
    double height_step, grid_res, bin_angle, dem_res;
    double im_res, im_res_next;
    double boundary[4];
    double minmax[2];
    int64_t grid_w, grid_h, n_nodes;
    const double *grid_wgs;         // [N][2] lon, lat
    const double *grid_pts;         // [N][2] projected metres
    const vll_ugrid *gp3;           // [N]
    vll_nccresult *ncc;             // [N] in/out
    vll_voxel *vox;                 // packed rows (voxel route) or nullptr
    const int64_t *vox_off;         // [N+1] row offsets by NumOfHeight (voxel route)
    // orthoimage coordinates (SetOrthoImageCoord), per image, or nullptr
    const double2 *ocd[VLL_MAX_IMAGES];
    const double2 *ocd_n[VLL_MAX_IMAGES];
    int64_t ow, oh, own, ohn;
    // diagnostics: per-slot rho as computed by the kernel (FP32 values before
    // any FP64 re-check in the split kernel), at dbg_off[node] + slot
    double *dbg_rho;
    const int64_t *dbg_off;
    // diagnostics: per-phase cycle totals and event counts of the split
    // kernel (see fused::Diag), or nullptr
    unsigned long long *diag;
    vll_transparam param;
    double rot_cos[kRotTable];      // cos(-theta) for diff_theta = (i-kRotOffset)/2
    double rot_sin[kRotTable];
    DevImage im[VLL_MAX_IMAGES];
    // Footprint tiles of the split kernel's window staging: tensor maps (TMA)
    // of the reference [0] and target [1] images' intensity [.][0] and
    // magnitude [.][1] planes with the level's tile of tma_w x tma_h texels
    // (tma_w a multiple of 8), or tma_w[0] == 0 (staging by loads).
    alignas(64) unsigned char tmap[2][2][128];
    int tma_w[2], tma_h[2];
};

// ---- quantisers (Template.hpp:964-993) ------------------------------------
// The reference converts double -> short through a 32-bit integer (x86-64
// cvttsd2si): out of range / NaN -> 0x80000000, then the low 16 bits.
__device__ __forceinline__ int16_t to_short(double v) {
    if (!(v > -2147483649.0 && v < 2147483648.0)) return 0;
    return (int16_t)(int32_t)v;
}
__device__ __forceinline__ int16_t q_result(double v) { return to_short(round(__dmul_rn(v, 1000.0))); }
__device__ __forceinline__ double dq_result(int16_t v) { return __ddiv_rn((double)v, 1000.0); }
__device__ __forceinline__ int16_t q_voxel(double v) { return to_short(__dmul_rn(v, 1000.0)); }
__device__ __forceinline__ double dq_voxel(int16_t v) { return __ddiv_rn((double)v, 1000.0); }

// ---- geometry ----------------------------------------------------------------
// GetObjectToImageRPC_single, CoordConversion.hpp:26-86.  The cubic is summed
// in RPC00B term order, each monomial associated as the reference writes it.
__device__ __forceinline__ double2 rpc_project(const double *__restrict__ rpc,
                                               const double *__restrict__ adj, double X,
                                               double Y, double Z) {
    double L = __ddiv_rn(__dadd_rn(X, -rpc[2]), rpc[7]);
    double P = __ddiv_rn(__dadd_rn(Y, -rpc[3]), rpc[8]);
    const double H = __ddiv_rn(__dadd_rn(Z, -rpc[4]), rpc[9]);
    if (L < -10.0 || L > 10.0) {
        X = X > 0 ? __dadd_rn(X, -360.0) : __dadd_rn(X, 360.0);
        L = __ddiv_rn(__dadd_rn(X, -rpc[2]), rpc[7]);
    }
    if (P < -10.0 || P > 10.0) {
        Y = Y > 0 ? __dadd_rn(Y, -360.0) : __dadd_rn(Y, 360.0);
        P = __ddiv_rn(__dadd_rn(Y, -rpc[3]), rpc[8]);
    }
    const double PL = __dmul_rn(P, L), LL = __dmul_rn(L, L), LP = __dmul_rn(L, P),
                 LH = __dmul_rn(L, H), PP = __dmul_rn(P, P), PH = __dmul_rn(P, H),
                 HH = __dmul_rn(H, H);
    double cf[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double *c = rpc + 10 + 20 * j;
        double s = c[0];
        s = __dadd_rn(s, __dmul_rn(c[1], L));
        s = __dadd_rn(s, __dmul_rn(c[2], P));
        s = __dadd_rn(s, __dmul_rn(c[3], H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[4], L), P));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[5], L), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[6], P), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[7], L), L));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[8], P), P));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[9], H), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[10], PL), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[11], LL), L));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[12], LP), P));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[13], LH), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[14], LL), P));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[15], PP), P));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[16], PH), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[17], LL), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[18], PP), H));
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(c[19], HH), H));
        cf[j] = s;
    }
    const double line = __dadd_rn(__dmul_rn(__ddiv_rn(cf[0], cf[1]), rpc[5]), rpc[0]);
    const double samp = __dadd_rn(__dmul_rn(__ddiv_rn(cf[2], cf[3]), rpc[6]), rpc[1]);
    double y = __dadd_rn(adj[0], line);
    double x = __dadd_rn(adj[1], samp);
    const double ymax = __dadd_rn(rpc[0], __dmul_rn(rpc[5], 1.2));
    const double xmax = __dadd_rn(rpc[1], __dmul_rn(rpc[6], 1.2));
    if (y < 0) y = 0;
    if (y > ymax) y = ymax;
    if (x < 0) x = 0;
    if (x > xmax) x = xmax;
    return make_double2(x, y);
}

// OriginalToPyramid_single, CoordConversion.hpp:96-106
__device__ __forceinline__ double2 to_pyramid(double2 p, double sx, double sy, int level) {
    const double s = (double)(1 << level);
    return make_double2(__dadd_rn(__ddiv_rn(p.x, s), -sx), __dadd_rn(__ddiv_rn(p.y, s), -sy));
}

// check_image_boundary, setsm_code.cpp:11002-11083 (RPC sensor).  The
// right-hand limits are computed in unsigned int like the reference.
__device__ __forceinline__ bool check_image_boundary(const DevLevel &P, double lon, double lat,
                                                     double minH, double maxH, int H) {
    int selected = 0;
    bool check_reference = true;
    const int buff = 1;
    for (int ti = 0; ti < P.num_images; ++ti) {
        const DevImage &im = P.im[ti];
        if (!im.selected) continue;
        const double lim_w = (double)(unsigned)(im.w - (unsigned)H - (unsigned)buff);
        const double lim_h = (double)(unsigned)(im.h - (unsigned)H - (unsigned)buff);
        double2 t = to_pyramid(rpc_project(im.rpc, im.adj, lon, lat, minH), im.sx, im.sy, P.L);
        const bool s_ok = t.x > H + buff && t.x < lim_w && t.y > H + buff && t.y < lim_h;
        t = to_pyramid(rpc_project(im.rpc, im.adj, lon, lat, maxH), im.sx, im.sy, P.L);
        const bool e_ok = t.x > H + buff && t.x < lim_w && t.y > H + buff && t.y < lim_h;
        if (s_ok && e_ok)
            selected++;
        else if (ti == 0)
            check_reference = false;
    }
    if (!check_reference) return false;
    return selected >= 2;
}

// Blunder-cell filter of VerticalLineLocus, setsm_code.cpp:6162-6204.
__device__ __forceinline__ bool blunder_cell(const DevLevel &P, const vll_ugrid &g) {
    bool b;
    const int span = abs((int)g.maxHeight - (int)g.minHeight);
    if (P.L >= 2)
        b = false;
    else if (g.Matched_flag == 0)
        b = true;
    else
        b = !(span < P.th_height);
    if (P.L <= 1 && (g.maxHeight > P.minmax[1] || g.minHeight < P.minmax[0])) b = true;
    if (P.check_matchtag && P.iteration <= 2) {
        b = false;
        if (g.maxHeight > P.minmax[1] || g.minHeight < P.minmax[0])
            b = true;
        else if (span > P.th_height)
            b = true;
    }
    return b;
}

// UGRID.ortho_ncc[ti] with the reference's indexing (the array has two
// entries; larger ti read the record's following fields).
__device__ __forceinline__ int16_t ugrid_ortho_ncc(const vll_ugrid *G, int64_t n, int64_t pt,
                                                   int ti) {
    const int64_t byte = 10 + 2 * (int64_t)ti;
    const int64_t rec = pt + byte / (int64_t)sizeof(vll_ugrid);
    if (rec >= n) return 0;
    const unsigned char *p = (const unsigned char *)G + pt * (int64_t)sizeof(vll_ugrid) + byte;
    return (int16_t)((uint16_t)p[0] | ((uint16_t)p[1] << 8));
}

// ---- FindPeakNcc, setsm_code.cpp:6672-6752 ---------------------------------
struct PeakState {
    int check_rho;
    int direction;
    double pre_rho;
    float pre_height;
};

__device__ __forceinline__ void peak_init(PeakState &s) {
    s.check_rho = 0;
    s.direction = 0;
    s.pre_rho = -1.0;
    s.pre_height = 0.0f;
}

__device__ __forceinline__ void find_peak(PeakState &st, double rho, float height,
                                          vll_nccresult &r) {
    double diff;
    if (rho >= 0 && st.pre_rho >= 0)
        diff = __dadd_rn(rho, -st.pre_rho);
    else if (rho < 0 && st.pre_rho < 0)
        diff = -(__dadd_rn(fabs(rho), -fabs(st.pre_rho)));
    else if (rho >= 0 && st.pre_rho < 0)
        diff = 1;
    else
        diff = -1;
    int td = diff > 0 ? 1 : (diff < 0 ? -1 : 0);
    if (!st.check_rho) {
        st.check_rho = 1;
        td = -1;
    } else if (st.pre_rho != -1) {
        if (st.direction > 0 && td < 0) {
            if (r.result4 < 10) r.result4 += 1;
            const int16_t qpre = q_result(st.pre_rho);
            if (r.result0 < qpre) {
                const double t1 = dq_result(r.result0);
                r.result0 = qpre;
                const float t2 = r.result2;
                r.result2 = st.pre_height;
                const int16_t q1 = q_result(t1);
                if (r.result1 < q1) {
                    r.result1 = q1;
                    r.result3 = t2;
                }
            } else if (r.result1 < qpre) {
                r.result1 = qpre;
                r.result3 = st.pre_height;
            }
        }
    }
    st.pre_rho = rho;
    st.pre_height = height;
    st.direction = td;
}

// Height of slot k (setsm_code.cpp:6331-6336), computed in double and stored
// as float like the reference's `float iter_height`.
__device__ __forceinline__ float slot_height(const DevLevel &P, int start_H, int ncc_min, int k) {
    const int base = (P.is_ra || P.cmr) ? start_H : ncc_min;
    return (float)__dadd_rn((double)base, __dmul_rn((double)k, P.height_step));
}

}  // namespace vll

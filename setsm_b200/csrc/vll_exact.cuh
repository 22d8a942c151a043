// vll_exact.cuh -- exact FP64 evaluation of VerticalLineLocus on the device
// (setsm_code.cpp:6049-6548 with SubFunctions.cpp:974-1018, :3249-3360):
// shared by the plain FP64 kernel and by the split pipeline's FP64 re-checks.
#pragma once

#include "vll_device.cuh"

namespace vll {

struct PatchSrc {
    const uint16_t *li, *lm, *ri, *rm;
    uint32_t lw, lh, rw, rh;
};

// InterpolatePatch, SubFunctions.cpp:3317-3326
__device__ __forceinline__ double interp(const uint16_t *__restrict__ I, int64_t pos, uint32_t w,
                                         double dx, double dy) {
    const double omx = __dadd_rn(1.0, -dx), omy = __dadd_rn(1.0, -dy);
    const double t0 = __dmul_rn(__dmul_rn((double)I[pos], omx), omy);
    const double t1 = __dmul_rn(__dmul_rn((double)I[pos + 1], dx), omy);
    const double t2 = __dmul_rn(__dmul_rn((double)I[pos + w], omx), dy);
    const double t3 = __dmul_rn(__dmul_rn((double)I[pos + 1 + w], dx), dy);
    return __dadd_rn(__dadd_rn(__dadd_rn(t0, t1), t2), t3);
}

// SetVecKernelValue's sampling step, SubFunctions.cpp:3252-3274: bounds check,
// four bilinear samples, and the `left > 0 && right > 0` filter.
__device__ __forceinline__ bool sample4(const PatchSrc &S, double2 pl, double2 pr, double v[4]) {
    if (!(pr.y >= 0 && __dadd_rn(pr.y, 1.0) < (double)S.rh && pr.x >= 0 &&
          __dadd_rn(pr.x, 1.0) < (double)S.rw && pl.y >= 0 && __dadd_rn(pl.y, 1.0) < (double)S.lh &&
          pl.x >= 0 && __dadd_rn(pl.x, 1.0) < (double)S.lw))
        return false;
    const int64_t pos = (int64_t)pl.x + (int64_t)pl.y * (int64_t)S.lw;
    const int64_t posr = (int64_t)pr.x + (int64_t)pr.y * (int64_t)S.rw;
    const double dx = __dadd_rn(pl.x, -floor(pl.x)), dy = __dadd_rn(pl.y, -floor(pl.y));
    const double dxr = __dadd_rn(pr.x, -floor(pr.x)), dyr = __dadd_rn(pr.y, -floor(pr.y));
    v[0] = interp(S.li, pos, S.lw, dx, dy);
    v[1] = interp(S.lm, pos, S.lw, dx, dy);
    v[2] = interp(S.ri, posr, S.rw, dxr, dyr);
    v[3] = interp(S.rm, posr, S.rw, dxr, dyr);
    return v[0] > 0 && v[2] > 0;
}

// Sub-window membership of a window offset (SubFunctions.cpp:3281-3313);
// window 0 holds every sample, windows 1 and 2 are nested inner windows.
__device__ __forceinline__ int window_depth(int H, int row, int col, int r2) {
    const int s1 = H / 2;
    const int s2 = s1 + (int)((s1 / 2.0) + 0.5);
    int d = 0;
    if (r2 <= (H - s1 + 1) * (H - s1 + 1) && row >= -H + s1 && row <= H - s1 && col >= -H + s1 &&
        col <= H - s1)
        d = 1;
    if (r2 <= (H - s2 + 1) * (H - s2 + 1) && row >= -H + s2 && row <= H - s2 && col >= -H + s2 &&
        col <= H - s2)
        d = 2;
    return d;
}

// ComputeMultiNCC over one circular window (SubFunctions.cpp:3328-3360 with
// Correlate, :974-1018).  Correlate is two-pass; instead of keeping the sample
// vectors, pass 1 accumulates the sums for the means and pass 2 re-samples the
// identical positions for the centred products, in the same order, so every
// partial sum equals the reference's.  `pos(row, col, r2, pl, pr)` supplies the
// sample positions (and may veto a window offset).  Returns true when all
// three sub-windows received samples.
template <class PosFn>
__device__ bool multi_ncc(const PatchSrc &S, int H, PosFn pos, double &count_ncc, double &sum_ncc,
                          int *cnt0_out = nullptr) {
    double s[3][4];
    int cnt[3] = {0, 0, 0};
#pragma unroll
    for (int w = 0; w < 3; ++w)
#pragma unroll
        for (int c = 0; c < 4; ++c) s[w][c] = 0.0;
    for (int row = -H; row <= H; ++row)
        for (int col = -H; col <= H; ++col) {
            const int r2 = row * row + col * col;
            if (r2 > (H + 1) * (H + 1)) continue;
            double2 pl, pr;
            if (!pos(row, col, pl, pr)) continue;
            double v[4];
            if (!sample4(S, pl, pr, v)) continue;
            const int dep = window_depth(H, row, col, r2);
            for (int w = 0; w <= dep; ++w) {
                cnt[w]++;
#pragma unroll
                for (int c = 0; c < 4; ++c) s[w][c] = __dadd_rn(s[w][c], v[c]);
            }
        }
    if (cnt0_out) *cnt0_out = cnt[0];
    const bool all_pos = cnt[0] > 0 && cnt[1] > 0 && cnt[2] > 0;
    if (!all_pos) return false;
    double m[3][4];
#pragma unroll
    for (int w = 0; w < 3; ++w)
#pragma unroll
        for (int c = 0; c < 4; ++c) m[w][c] = __ddiv_rn(s[w][c], (double)cnt[w]);
    double acc[3][2][3];   // [window][intensity|magnitude][LR, L2, R2]
#pragma unroll
    for (int w = 0; w < 3; ++w)
#pragma unroll
        for (int p = 0; p < 2; ++p) acc[w][p][0] = acc[w][p][1] = acc[w][p][2] = 0.0;
    for (int row = -H; row <= H; ++row)
        for (int col = -H; col <= H; ++col) {
            const int r2 = row * row + col * col;
            if (r2 > (H + 1) * (H + 1)) continue;
            double2 pl, pr;
            if (!pos(row, col, pl, pr)) continue;
            double v[4];
            if (!sample4(S, pl, pr, v)) continue;
            const int dep = window_depth(H, row, col, r2);
            for (int w = 0; w <= dep; ++w) {
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const double dl = __dadd_rn(v[p], -m[w][p]);
                    const double dr = __dadd_rn(v[p + 2], -m[w][p + 2]);
                    acc[w][p][0] = __dadd_rn(acc[w][p][0], __dmul_rn(dl, dr));
                    acc[w][p][1] = __dadd_rn(acc[w][p][1], __dmul_rn(dl, dl));
                    acc[w][p][2] = __dadd_rn(acc[w][p][2], __dmul_rn(dr, dr));
                }
            }
        }
    double tot = 0, n = 0;
#pragma unroll
    for (int w = 0; w < 3; ++w)
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            if (acc[w][p][1] > 1e-8 && acc[w][p][2] > 1e-8) {
                const double r = __ddiv_rn(acc[w][p][0], sqrt(__dmul_rn(acc[w][p][1], acc[w][p][2])));
                if (r != -99) {
                    n = __dadd_rn(n, 1.0);
                    tot = __dadd_rn(tot, r);
                }
            }
        }
    if (n > 0) {
        sum_ncc = __dadd_rn(sum_ncc, __ddiv_rn(tot, n));
        count_ncc = __dadd_rn(count_ncc, 1.0);
    }
    return true;
}

// GNCC of one node (setsm_code.cpp:6241-6305): the same multi-window NCC over
// the ortho-projected coordinates of the node's neighbourhood.
static __device__ __noinline__ void node_gncc(const DevLevel &P, int64_t pt, int ti, const PatchSrc &S,
                          const PatchSrc &Sn, double &count_g, double &sum_g) {
    const int H = P.H;
    const double gx = P.grid_pts[2 * pt], gy = P.grid_pts[2 * pt + 1];
    const double *B = P.boundary;
    const double2 *cr = P.ocd[P.ref], *ct = P.ocd[ti];
    auto inside = [&](int row, int col, double &tX, double &tY, int64_t &pit) -> bool {
        tX = __dadd_rn(gx, __dmul_rn((double)col, P.im_res));
        tY = __dadd_rn(gy, __dmul_rn((double)row, P.im_res));
        const int64_t t_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.im_res);
        const int64_t t_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.im_res);
        pit = t_row * P.ow + t_col;
        const int64_t tt_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.grid_res);
        const int64_t tt_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.grid_res);
        const int64_t pdem = tt_row * P.grid_w + tt_col;
        if (!(pit >= 0 && pit < P.ow * P.oh && t_col >= 0 && t_col < P.ow && t_row >= 0 &&
              t_row < P.oh && pdem >= 0 && pdem < P.n_nodes && tt_col >= 0 && tt_col < P.grid_w &&
              tt_row >= 0 && tt_row < P.grid_h && cr != nullptr && ct != nullptr))
            return false;
        return P.gp3[pdem].Height != -1000;
    };
    multi_ncc(S, H,
              [&](int row, int col, double2 &pl, double2 &pr) -> bool {
                  double tX, tY;
                  int64_t pit;
                  if (!inside(row, col, tX, tY, pit)) return false;
                  pl = cr[pit];
                  pr = ct[pit];
                  return true;
              },
              count_g, sum_g);
    if (P.combined) {
        const double2 *crn = P.ocd_n[P.ref], *ctn = P.ocd_n[ti];
        multi_ncc(Sn, H,
                  [&](int row, int col, double2 &pl, double2 &pr) -> bool {
                      double tX, tY;
                      int64_t pit;
                      if (!inside(row, col, tX, tY, pit)) return false;
                      const int64_t t_col = (int64_t)__ddiv_rn(__dadd_rn(tX, -B[0]), P.im_res_next);
                      const int64_t t_row = (int64_t)__ddiv_rn(__dadd_rn(tY, -B[1]), P.im_res_next);
                      const int64_t pn = t_row * P.own + t_col;
                      if (!(pn >= 0 && pn < P.own * P.ohn && t_col < P.own && t_row < P.ohn))
                          return false;
                      pl = crn[pn];
                      pr = ctn[pn];
                      return true;
                  },
                  count_g, sum_g);
    }
}

__device__ __forceinline__ bool in_image(double2 p, uint32_t w, uint32_t h) {
    return (int)p.y >= 0 && (unsigned)((int)p.y + 1) < h && (int)p.x >= 0 &&
           (unsigned)((int)p.x + 1) < w;
}

// One (node, height slot) evaluation: projection, orientation, window NCC.
// Returns false when the slot is skipped (out of range / outside images /
// orientation check); otherwise sets rho (temp_rho) and the voxel values.
struct SlotOut {
    double rho;
    double count_incc, sum_incc;
    bool all_pos;
    bool evaluated;
    bool orient_reject;   // orientation check failed: the voxel flag is cleared
};

static __device__ __noinline__ SlotOut eval_slot(const DevLevel &P, int64_t pt, int ti, const PatchSrc &S,
                             const PatchSrc &Sn, float hgt, double count_g, double sum_g) {
    SlotOut o;
    o.evaluated = false;
    o.orient_reject = false;
    o.all_pos = false;
    o.rho = -1.0;
    o.count_incc = 0;
    o.sum_incc = 0;
    const DevImage &ri = P.im[P.ref];
    const DevImage &tI = P.im[ti];
    const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
    const double2 rc = rpc_project(ri.rpc, ri.adj, lon, lat, (double)hgt);
    const double2 tc = rpc_project(tI.rpc, tI.adj, lon, lat, (double)hgt);
    const double2 rp = to_pyramid(rc, ri.sx, ri.sy, P.L);
    const double2 tp = to_pyramid(tc, tI.sx, tI.sy, P.L);
    if (!(in_image(rp, ri.w, ri.h) && in_image(tp, tI.w, tI.h))) return o;
    double2 rpn = make_double2(0, 0), tpn = make_double2(0, 0);
    if (P.combined_incc) {
        rpn = to_pyramid(rc, ri.sxn, ri.syn, P.L - 1);
        tpn = to_pyramid(tc, tI.sxn, tI.syn, P.L - 1);
        if (!(in_image(rpn, ri.wn, ri.hn) && in_image(tpn, tI.wn, tI.hn))) return o;
    }
    const int od = (int)ri.ori[(int64_t)(int)rp.y * ri.w + (int)rp.x] -
                   (int)tI.ori[(int64_t)(int)tp.y * tI.w + (int)tp.x];
    int odn = 0;
    if (P.combined_incc)
        odn = (int)ri.ori_n[(int64_t)(int)rpn.y * ri.wn + (int)rpn.x] -
              (int)tI.ori_n[(int64_t)(int)tpn.y * tI.wn + (int)tpn.x];
    // diff_theta is an integer, or a half-integer in combined mode
    const int twice = P.combined_incc ? (od + odn) : 2 * od;
    const double dtheta = P.combined_incc ? __ddiv_rn((double)(od + odn), 2.0) : (double)od;
    bool check_orient;
    if (!P.is_ra) {
        const double a = __dmul_rn(dtheta, P.bin_angle);
        check_orient = (P.L >= 3 && a < 90 && a > -90) || (P.L <= 2);
    } else
        check_orient = true;
    if (!check_orient) {
        o.orient_reject = true;
        return o;
    }
    o.evaluated = true;
    const int ti_rot = twice + kRotOffset;
    const double c0 = P.rot_cos[ti_rot], s0 = P.rot_sin[ti_rot];
    double count = 0, sum = 0;
    o.all_pos = multi_ncc(S, P.H,
                          [&](int row, int col, double2 &pl, double2 &pr) -> bool {
                              const double ox = __dadd_rn(__dmul_rn(c0, (double)col), -__dmul_rn(s0, (double)row));
                              const double oy = __dadd_rn(__dmul_rn(s0, (double)col), __dmul_rn(c0, (double)row));
                              pl = make_double2(__dadd_rn(rp.x, (double)col), __dadd_rn(rp.y, (double)row));
                              pr = make_double2(__dadd_rn(tp.x, ox), __dadd_rn(tp.y, oy));
                              return true;
                          },
                          count, sum);
    if (P.combined_incc)
        multi_ncc(Sn, P.H,
                  [&](int row, int col, double2 &pl, double2 &pr) -> bool {
                      const double ox = __dadd_rn(__dmul_rn(c0, (double)col), -__dmul_rn(s0, (double)row));
                      const double oy = __dadd_rn(__dmul_rn(s0, (double)col), __dmul_rn(c0, (double)row));
                      pl = make_double2(__dadd_rn(rpn.x, (double)col), __dadd_rn(rpn.y, (double)row));
                      pr = make_double2(__dadd_rn(tpn.x, ox), __dadd_rn(tpn.y, oy));
                      return true;
                  },
                  count, sum);
    o.count_incc = count;
    o.sum_incc = sum;
    if (P.check_ortho && count_g > 0)
        o.rho = __dadd_rn(__dmul_rn(__ddiv_rn(sum, count), P.alpha),
                          __dmul_rn(__ddiv_rn(sum_g, count_g), P.beta));
    else
        o.rho = count > 0 ? __ddiv_rn(sum, count) : -1.0;
    return o;
}

__device__ __forceinline__ void make_src(const DevLevel &P, int ti, PatchSrc &S, PatchSrc &Sn) {
    const DevImage &ri = P.im[P.ref];
    const DevImage &tI = P.im[ti];
    S = {ri.img, ri.mag, tI.img, tI.mag, ri.w, ri.h, tI.w, tI.h};
    Sn = {ri.img_n, ri.mag_n, tI.img_n, tI.mag_n, ri.wn, ri.hn, tI.wn, tI.hn};
}

// One node of VerticalLineLocus.  `rho_out` (optional) receives temp_rho of
// each evaluated slot; NaN elsewhere is left to the caller's initialisation.
static __device__ __noinline__ void plain_node(const DevLevel &P, int64_t pt, unsigned long long &acc,
                           unsigned long long &evals, double *rho_out, const int64_t *rho_off) {
    const vll_ugrid g = P.gp3[pt];
    const int start_H = g.minHeight, end_H = g.maxHeight;
    const double lon = P.grid_wgs[2 * pt], lat = P.grid_wgs[2 * pt + 1];
    if (!check_image_boundary(P, lon, lat, (double)start_H, (double)end_H, P.H)) return;
    if (blunder_cell(P, g)) return;
    vll_nccresult &R = P.ncc[pt];
    for (int ti = 1; ti < P.num_images; ++ti) {
        if (!P.im[ti].selected) continue;
        acc++;
        PatchSrc S, Sn;
        make_src(P, ti, S, Sn);
        double count_g = 0, sum_g = 0;
        if (P.check_ortho && dq_result(ugrid_ortho_ncc(P.gp3, P.n_nodes, pt, ti)) > P.ortho_th) {
            node_gncc(P, pt, ti, S, Sn, count_g, sum_g);
            R.GNCC = count_g > 0 ? q_result(__ddiv_rn(sum_g, count_g)) : q_result(-1.0);
        } else {
            R.GNCC = q_result(-1.0);
        }
        const int num_heights = (int)__ddiv_rn((double)(end_H - start_H), P.height_step);
        if (P.is_ra || P.cmr) {
            R.check_height_change = 1;
            R.NumOfHeight = (uint16_t)num_heights;
        }
        if (!(P.is_ra || P.cmr || R.check_height_change || (P.L == 0 && P.dem_res < 2))) continue;
        PeakState st;
        peak_init(st);
        double max_wncc = -100;
        R.result0 = q_result(-1.0);
        R.result2 = -1000;
        R.result1 = q_result(-1.0);
        R.result3 = -1000;
        R.result4 = 0;
        const int nh = R.NumOfHeight;
        vll_voxel *vrow = (P.vox && !P.cmr && !P.is_ra) ? P.vox + P.vox_off[pt] : nullptr;
        for (int k = 0; k < nh; ++k) {
            const float hgt = slot_height(P, start_H, R.minHeight, k);
            if (!(hgt >= (float)start_H && hgt <= (float)end_H)) continue;
            const SlotOut o = eval_slot(P, pt, ti, S, Sn, hgt, count_g, sum_g);
            if (!o.evaluated) {
                if (o.orient_reject && vrow) vrow[k].flag_cal = 0;
                continue;
            }
            evals++;
            if (vrow) {
                if (o.all_pos) vrow[k].flag_cal = 1;
                vrow[k].INCC = o.count_incc > 0 ? q_voxel(__ddiv_rn(o.sum_incc, o.count_incc))
                                                 : q_voxel(-1.0);
            }
            if (rho_out) rho_out[rho_off[pt] + k] = o.rho;
            if (max_wncc < o.rho) max_wncc = o.rho;
            if (P.cmr) find_peak(st, o.rho, hgt, R);
        }
        if (R.check_height_change) R.max_WNCC = q_result(max_wncc);
    }
}

}  // namespace vll

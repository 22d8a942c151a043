// vll_orthotin.cu -- the TIN-triangle orthoimage height search of SETSM's
// blunder removal: VerticalLineLocus_Ortho (setsm_code.cpp:8234-8533) and the
// loop that drives it, Ortho_blunder (:8028-8232).
//
// For a triangle of matched points with two anchored vertices, the third
// (target) vertex's height is swept over its UGRID range; at each height the
// triangle's plane is rasterised over the grid cells of its bounding box, every
// cell inside the triangle is projected through the RPCs of the reference and
// each target image, and the Pearson correlation of the sampled intensities
// and magnitudes (Correlate, SubFunctions.cpp:974-1018) picks the height.
//
// GPU layout: one warp per triangle.  The triangle's box and its inside cells
// do not depend on the swept height, so the inside cells are listed once;
// each height projects only those, 32 at a time, and stages their samples in
// shared memory for both of Correlate's passes.  Every sum is accumulated in
// the reference's cell order (each lane reads the staged samples in
// sequence), so the FP64 results are the reference's bit for bit.  A
// triangle with more than 256 inside cells tests its box per height and
// recomputes the samples in the second pass.  The sequential "apply" pass of
// Ortho_blunder is restated in parallel with the same result: triangles that
// found a height are grouped by target point (stable radix sort), each
// point's triangles are walked in triangle order to find the record-breakers
// of the running maximum (the reference's com_count test), and the anchor
// counts of the second half of the pass use, per grid node, the first
// triangle index that anchored it.
#include <cstdint>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "vll_exact.cuh"
#include "vll_geo.cuh"
#include "vll_internal.h"

namespace vll {

namespace {

struct P3 {
    double x, y, z;
};

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

// One cell's samples (InterpolatePatch of both planes of both images at the
// plane height) are cell_sample's, for a cell that cell_inside accepts;
// setsm_code.cpp:8331-8451.
// Whether the cell lies in the triangle: the three edge tests (D3DPOINT
// differences; z unused, so the answer is the same at every height).
__device__ bool cell_inside(const DevLevel &P, const P3 &T1, const P3 &T2, const P3 &T3,
                            int64_t row, int64_t col) {
    const double gs = P.grid_res;
    const double cx = __dadd_rn(__dmul_rn((double)col, gs), P.boundary[0]);
    const double cy = __dadd_rn(__dmul_rn((double)row, gs), P.boundary[1]);
    int sum = 3;
    if (__dadd_rn(__dmul_rn(__dadd_rn(T2.x, -T1.x), __dadd_rn(cy, -T1.y)),
                  -__dmul_rn(__dadd_rn(T2.y, -T1.y), __dadd_rn(cx, -T1.x))) <= 0)
        --sum;
    if (__dadd_rn(__dmul_rn(__dadd_rn(T3.x, -T2.x), __dadd_rn(cy, -T2.y)),
                  -__dmul_rn(__dadd_rn(T3.y, -T2.y), __dadd_rn(cx, -T2.x))) <= 0)
        --sum;
    if (__dadd_rn(__dmul_rn(__dadd_rn(T1.x, -T3.x), __dadd_rn(cy, -T3.y)),
                  -__dmul_rn(__dadd_rn(T1.y, -T3.y), __dadd_rn(cx, -T3.x))) <= 0)
        --sum;
    return sum == 0 || sum == 3;
}

// The samples of a cell inside the triangle at the plane's height, or false
// when the plane is degenerate or a window corner leaves an image.
__device__ bool cell_sample(const DevLevel &P, const double2 *__restrict__ lonlat, int ti,
                            bool plane_ok, double A, double B, double C, double D, int64_t row,
                            int64_t col, double v[4]) {
    if (!plane_ok) return false;
    const double gs = P.grid_res;
    const double cx = __dadd_rn(__dmul_rn((double)col, gs), P.boundary[0]);
    const double cy = __dadd_rn(__dmul_rn((double)row, gs), P.boundary[1]);
    // Z = -1.0 * ((A x) + (B y) + D) / C
    const double z = __ddiv_rn(-__dadd_rn(__dadd_rn(__dmul_rn(A, cx), __dmul_rn(B, cy)), D), C);
    // the cell's longitude / latitude: from the grid-wide table when given
    // (the same function of the same coordinates), else computed here
    const double2 w = lonlat ? lonlat[row * P.grid_w + col] : ps2wgs_dev(P.param, cx, cy);
    const DevImage &ri = P.im[P.ref], &tI = P.im[ti];
    // the target image is projected with the reference image's adjustment,
    // as the reference does (temp_LIA, setsm_code.cpp:8392)
    const double2 rp = to_pyramid(rpc_project(ri.rpc, ri.adj, w.x, w.y, z), ri.sx, ri.sy, P.L);
    const double2 tp = to_pyramid(rpc_project(tI.rpc, ri.adj, w.x, w.y, z), tI.sx, tI.sy, P.L);
    if (!(tp.y >= 0 && __dadd_rn(tp.y, 1.0) < (double)tI.h && tp.x >= 0 &&
          __dadd_rn(tp.x, 1.0) < (double)tI.w && rp.y >= 0 && __dadd_rn(rp.y, 1.0) < (double)ri.h &&
          rp.x >= 0 && __dadd_rn(rp.x, 1.0) < (double)ri.w))
        return false;
    const double dx = __dadd_rn(rp.x, -(double)(int)rp.x), dy = __dadd_rn(rp.y, -(double)(int)rp.y);
    const int64_t pos = (int64_t)rp.x + (int64_t)rp.y * (int64_t)ri.w;
    const double dxr = __dadd_rn(tp.x, -(double)(int)tp.x), dyr = __dadd_rn(tp.y, -(double)(int)tp.y);
    const int64_t posr = (int64_t)tp.x + (int64_t)tp.y * (int64_t)tI.w;
    v[0] = interp(ri.img, pos, ri.w, dx, dy);
    v[1] = interp(tI.img, posr, tI.w, dxr, dyr);
    v[2] = interp(ri.mag, pos, ri.w, dx, dy);
    v[3] = interp(tI.mag, posr, tI.w, dxr, dyr);
    return true;
}

// Correlate's final step (SubFunctions.cpp:1000-1010).
__device__ __forceinline__ double corr_of(double slr, double sl2, double sr2) {
    if (sl2 > 1e-8 && sr2 > 1e-8) return __ddiv_rn(slr, sqrt(__dmul_rn(sl2, sr2)));
    return -99.0;
}

struct SearchOut {
    double f_height, f_sncc;
    int selected;
};

// Per-warp shared staging.  The triangle's bounding box and which of its
// cells lie inside do not depend on the swept height, so the inside cells are
// listed once per triangle; when at most kCellCap are inside, each height
// projects only those, 32 per step, and keeps their samples for both of
// Correlate's passes.  Otherwise every box cell is tested per height and the
// second pass recomputes its samples.  Either way the sums read the samples
// back in cell order.
constexpr int kCellCap = 256;
struct CellStage {
    double2 v[2 * kCellCap];        // item i: {img ref, img tgt}, {mag ref, mag tgt}
    unsigned int valid[kCellCap / 32];
    int32_t cell[kCellCap];         // the box's cells inside the triangle, in cell order
};

// VerticalLineLocus_Ortho for one triangle, by one warp (all lanes return
// the same result); st: the warp's staging.
__device__ SearchOut ortho_search(const DevLevel &P, const double2 *__restrict__ lonlat,
                                  double mpp, P3 r1, P3 r2, P3 tg, int64_t target_index,
                                  CellStage &st) {
    const int lane = threadIdx.x & 31;
    SearchOut o{-9999.0, 0.0, 0};
    double f_ncc = -1.0;
    double selected_count = 0;
    if (mpp > 3) mpp = 3;
    if (mpp < 1) mpp = 1;
    const double hstep = __dmul_rn(P.im_res, mpp);
    const int start_h = P.gp3[target_index].minHeight;
    const int end_h = P.gp3[target_index].maxHeight;
    const int n_heights = (int)__ddiv_rn((double)(end_h - start_h), hstep) + 1;
    const int th_count = 10;
    const int min_th_count = P.L < 4 ? 0 : 2;
    const double min_th_sncc = P.L < 4 ? 0.5 : 0.2;
    const double gs = P.grid_res;
    const int gw = (int)P.grid_w, gh = (int)P.grid_h;
    // the bounding box of the cells (the reference recomputes it per height
    // from the same x, y)
    const double mn0 = dmin(dmin(r1.x, r2.x), tg.x), mn1 = dmin(dmin(r1.y, r2.y), tg.y);
    const double mx0 = dmax(dmax(r1.x, r2.x), tg.x), mx1 = dmax(dmax(r1.y, r2.y), tg.y);
    int pmin0 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mn0, -P.boundary[0]), gs), 0.5);
    int pmin1 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mn1, -P.boundary[1]), gs), 0.5);
    int pmax0 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mx0, -P.boundary[0]), gs), 0.5);
    int pmax1 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mx1, -P.boundary[1]), gs), 0.5);
    pmin0 -= 1;
    pmin1 -= 1;
    pmax0 += 1;
    pmax1 += 1;
    if (pmax0 >= gw) pmax0 = gw - 1;
    if (pmax1 >= gh) pmax1 = gh - 1;
    if (pmin0 < 0) pmin0 = 0;
    if (pmin1 < 0) pmin1 = 0;
    if (!(pmax1 - pmin1 > 0 && pmax0 - pmin0 > 0)) return o;   // every height skips
    const int64_t ncol = pmax0 - pmin0 + 1;
    const int64_t ncell = (int64_t)(pmax1 - pmin1 + 1) * ncol;
    // the inside cells, in cell order
    int64_t n_in = 0;
    for (int64_t base = 0; base < ncell; base += 32) {
        const int64_t i = base + lane;
        const bool in = i < ncell && cell_inside(P, r1, r2, tg, pmin1 + i / ncol, pmin0 + i % ncol);
        const unsigned m = __ballot_sync(0xffffffffu, in);
        const int64_t at = n_in + __popc(m & ((1u << lane) - 1u));
        if (in && at < kCellCap) st.cell[at] = (int32_t)i;
        n_in += __popc(m);
    }
    __syncwarp();
    const bool listed = n_in <= kCellCap;
    const int64_t n_items = listed ? n_in : ncell;
    for (int64_t kh = 0; kh < n_heights; ++kh) {
        const float iter_height = (float)__dadd_rn((double)start_h, __dmul_rn((double)kh, hstep));
        const P3 T1 = r1, T2 = r2, T3 = {tg.x, tg.y, (double)iter_height};
        // the triangle's plane (the same for every cell of this height)
        const double v12x = __dadd_rn(T2.x, -T1.x), v12y = __dadd_rn(T2.y, -T1.y),
                     v12z = __dadd_rn(T2.z, -T1.z);
        const double v13x = __dadd_rn(T3.x, -T1.x), v13y = __dadd_rn(T3.y, -T1.y),
                     v13z = __dadd_rn(T3.z, -T1.z);
        double nx = __dadd_rn(__dmul_rn(v12y, v13z), -__dmul_rn(v12z, v13y));
        double ny = __dadd_rn(__dmul_rn(v12z, v13x), -__dmul_rn(v12x, v13z));
        double nz = __dadd_rn(__dmul_rn(v12x, v13y), -__dmul_rn(v12y, v13x));
        const double len =
            sqrt(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)), __dmul_rn(nz, nz)));
        bool plane_ok = len > 0;
        double A = 0, B = 0, C = 0, D = 0;
        if (plane_ok) {
            nx = __ddiv_rn(nx, len);
            ny = __ddiv_rn(ny, len);
            nz = __ddiv_rn(nz, len);
            A = nx;
            B = ny;
            C = nz;
            D = -__dadd_rn(__dadd_rn(__dmul_rn(A, T1.x), __dmul_rn(B, T1.y)), __dmul_rn(C, T1.z));
            plane_ok = C != 0;
        }
        double sum_ncc = 0;
        int count_ncc = 0;
        int sum_count_n = 0;
        const bool cached = listed;
        for (int ti = 1; ti < P.num_images; ++ti) {
            if (!P.im[ti].selected) continue;
            // pass 0: sums for the means; pass 1: centred products
            double s[6] = {0, 0, 0, 0, 0, 0};
            double m[4] = {0, 0, 0, 0};
            int count_n = 0;
            for (int pass = 0; pass < 2; ++pass) {
                for (int64_t base = 0; base < n_items; base += 32) {
                    const int64_t i = base + lane;
                    // staged item of this chunk's first lane: the chunk's own
                    // slots when the items are cached, else slots 0..31
                    const int64_t first = cached ? base : 0;
                    unsigned valid;
                    if (pass == 0 || !cached) {
                        double v[4] = {0, 0, 0, 0};
                        bool ok = false;
                        if (i < n_items) {
                            const int64_t c = listed ? (int64_t)st.cell[i] : i;
                            const int64_t row = pmin1 + c / ncol, col = pmin0 + c % ncol;
                            ok = (listed || cell_inside(P, T1, T2, T3, row, col)) &&
                                 cell_sample(P, lonlat, ti, plane_ok, A, B, C, D, row, col, v);
                        }
                        valid = __ballot_sync(0xffffffffu, ok);
                        st.v[2 * (first + lane)] = make_double2(v[0], v[1]);
                        st.v[2 * (first + lane) + 1] = make_double2(v[2], v[3]);
                        if (cached && lane == 0) st.valid[base >> 5] = valid;
                    } else {
                        valid = st.valid[base >> 5];
                    }
                    __syncwarp();
                    for (int j = 0; j < 32; ++j) {
                        if (!((valid >> j) & 1u)) continue;
                        const double2 a = st.v[2 * (first + j)], b = st.v[2 * (first + j) + 1];
                        const double u[4] = {a.x, a.y, b.x, b.y};
                        if (pass == 0) {
#pragma unroll
                            for (int c = 0; c < 4; ++c) s[c] = __dadd_rn(s[c], u[c]);
                            ++count_n;
                        } else {
                            const double dl = __dadd_rn(u[0], -m[0]), dr = __dadd_rn(u[1], -m[1]);
                            const double el = __dadd_rn(u[2], -m[2]), er = __dadd_rn(u[3], -m[3]);
                            s[0] = __dadd_rn(s[0], __dmul_rn(dl, dr));
                            s[1] = __dadd_rn(s[1], __dmul_rn(dl, dl));
                            s[2] = __dadd_rn(s[2], __dmul_rn(dr, dr));
                            s[3] = __dadd_rn(s[3], __dmul_rn(el, er));
                            s[4] = __dadd_rn(s[4], __dmul_rn(el, el));
                            s[5] = __dadd_rn(s[5], __dmul_rn(er, er));
                        }
                    }
                    __syncwarp();   // the slots are rewritten by the next chunk
                }
                if (pass == 0) {
                    if (count_n < 1) break;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        m[c] = __ddiv_rn(s[c], (double)count_n);
                        s[c] = 0;
                    }
                }
            }
            if (count_n >= 1) {
                double temp_roh = 0, count_roh = 0;
                const double ncc1 = corr_of(s[0], s[1], s[2]);
                if (ncc1 != -99) {
                    count_roh = __dadd_rn(count_roh, 1.0);
                    temp_roh = __dadd_rn(temp_roh, ncc1);
                }
                const double ncc2 = corr_of(s[3], s[4], s[5]);
                if (ncc2 != -99) {
                    count_roh = __dadd_rn(count_roh, 1.0);
                    temp_roh = __dadd_rn(temp_roh, ncc2);
                }
                const double ncc = count_roh > 0 ? __ddiv_rn(temp_roh, count_roh) : -1.0;
                sum_count_n += count_n;
                sum_ncc = __dadd_rn(sum_ncc, ncc);
                ++count_ncc;
            }
        }
        if (count_ncc > 0) {
            const double sncc = __ddiv_rn(sum_ncc, (double)count_ncc);
            const double cnt = __ddiv_rn((double)sum_count_n, (double)count_ncc);
            if (sum_count_n / count_ncc >= th_count) {
                if (sncc > min_th_sncc && f_ncc < sncc) {
                    f_ncc = sncc;
                    o.f_height = (double)iter_height;
                    selected_count = cnt;
                    o.f_sncc = f_ncc;
                }
            } else if (sum_count_n / count_ncc > min_th_count) {
                if (sncc > __dadd_rn(min_th_sncc, 0.2) && f_ncc < sncc) {
                    f_ncc = sncc;
                    o.f_height = __ddiv_rn(__dadd_rn(r1.z, r2.z), 2.0);
                    selected_count = cnt;
                    o.f_sncc = f_ncc;
                }
            }
        }
    }
    o.selected = (int)selected_count;
    return o;
}

// Grid node of a matched point (setsm_code.cpp:8073-8075).
__device__ __forceinline__ int64_t node_of(const DevLevel &P, const vll_point3 &p) {
    const int64_t r = (int64_t)__dadd_rn(__ddiv_rn(__dadd_rn(p.y, -P.boundary[1]), P.grid_res), 0.5);
    const int64_t c = (int64_t)__dadd_rn(__ddiv_rn(__dadd_rn(p.x, -P.boundary[0]), P.grid_res), 0.5);
    return r * P.grid_w + c;
}

__device__ __forceinline__ bool anchored(uint8_t f) { return f == 1 || f == 3; }

// Single search (the VerticalLineLocus_Ortho entry point): one warp.
__global__ void __launch_bounds__(32) ortho_search_kernel(const DevLevel *__restrict__ Pp,
                                                          double mpp, const vll_point3 *pts3,
                                                          int64_t target_index, double *out) {
    const DevLevel &P = *Pp;
    __shared__ CellStage st;
    const SearchOut o = ortho_search(P, nullptr, mpp, P3{pts3[0].x, pts3[0].y, pts3[0].z},
                                     P3{pts3[1].x, pts3[1].y, pts3[1].z},
                                     P3{pts3[2].x, pts3[2].y, pts3[2].z}, target_index, st);
    if (threadIdx.x == 0) {
        out[0] = o.f_height;
        out[1] = o.f_sncc;
        out[2] = (double)o.selected;
    }
}

// Ortho_blunder, first (parallel) loop over the triangles (setsm_code.cpp:
// 8060-8146): one warp per triangle.
__global__ void __launch_bounds__(128, 3) tri_search_kernel(const DevLevel *__restrict__ Pp,
                                                         double mpp, const vll_point3 *pts,
                                                         int64_t n_pts, const vll_tri *tris,
                                                         int64_t n_tris, const int64_t *tri_nodes,
                                                         uint8_t *tris_check, uint8_t *upd,
                                                         double *hgt, int32_t *cnt,
                                                         uint32_t *sort_key,
                                                         const double2 *__restrict__ lonlat) {
    const DevLevel &P = *Pp;
    __shared__ CellStage stage[4];   // one per warp of the 128-thread block
    CellStage &st = stage[threadIdx.x >> 5];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t none = (uint32_t)n_pts;
    for (int64_t t = warp; t < n_tris; t += n_warps) {
        const int lane = threadIdx.x & 31;
        uint32_t key = none;
        uint8_t u = 0;
        if (tris_check[t] == 0) {
            const vll_tri tr = tris[t];
            if (tr.a < n_pts && tr.b < n_pts && tr.c < n_pts) {
                const int64_t n1 = tri_nodes[3 * t], n2 = tri_nodes[3 * t + 1],
                              n3 = tri_nodes[3 * t + 2];
                const uint8_t f1 = P.gp3[n1].anchor_flag, f2 = P.gp3[n2].anchor_flag,
                              f3 = P.gp3[n3].anchor_flag;
                const int nf = (int)anchored(f1) + (int)anchored(f2) + (int)anchored(f3);
                if (nf == 3) {
                    if (lane == 0) tris_check[t] = 1;
                } else if (nf == 2) {
                    const vll_point3 &p0 = pts[tr.a], &p1 = pts[tr.b], &p2 = pts[tr.c];
                    P3 r1, r2, tg;
                    int64_t tnode;
                    uint32_t tpt;
                    if (f1 == 2) {
                        r1 = {p1.x, p1.y, p1.z};
                        r2 = {p2.x, p2.y, p2.z};
                        tg = {p0.x, p0.y, p0.z};
                        tnode = n1;
                        tpt = tr.a;
                    } else if (f2 == 2) {
                        r1 = {p0.x, p0.y, p0.z};
                        r2 = {p2.x, p2.y, p2.z};
                        tg = {p1.x, p1.y, p1.z};
                        tnode = n2;
                        tpt = tr.b;
                    } else {
                        r1 = {p0.x, p0.y, p0.z};
                        r2 = {p1.x, p1.y, p1.z};
                        tg = {p2.x, p2.y, p2.z};
                        tnode = n3;
                        tpt = tr.c;
                    }
                    const SearchOut o = ortho_search(P, lonlat, mpp, r1, r2, tg, tnode, st);
                    if (o.f_height != -9999.0) {
                        u = 1;
                        key = tpt;
                        if (lane == 0) {
                            hgt[t] = o.f_height;
                            cnt[t] = o.selected;
                        }
                    }
                }
            }
        }
        if (lane == 0) {
            upd[t] = u;
            sort_key[t] = key;
        }
    }
}

// Record-breakers of the running maximum per target point: triangles sorted
// by point (stable, so in triangle order within a point).  The last record
// sets the point's height; each record anchors the point's grid node, and
// the node remembers the first triangle that anchored it.
__global__ void records_kernel(const uint32_t *skey, const int32_t *sval, int64_t n, uint32_t none,
                               const int32_t *cnt, const double *hgt, const int64_t *tnode_of_pt,
                               vll_point3 *pts, uint8_t *rec, unsigned long long *first_anchor,
                               int *any_record) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = skey[i];
        if (k == none || (i > 0 && skey[i - 1] == k)) continue;
        int32_t best = 0;
        int32_t last = -1, first = -1;
        for (int64_t j = i; j < n && skey[j] == k; ++j) {
            const int32_t t = sval[j];
            if (best < cnt[t]) {   // com_count[target] < selected_count[tcnt]
                best = cnt[t];
                rec[t] = 1;
                last = t;
                if (first < 0) first = t;
            }
        }
        if (last >= 0) {
            pts[k].z = hgt[last];
            pts[k].flag = 0;
            atomicMin(first_anchor + tnode_of_pt[k], (unsigned long long)first);
            *any_record = 1;
        }
    }
}

// Second half of the apply pass (setsm_code.cpp:8164-8212) for every
// triangle still unchecked: records are checked, and a triangle whose three
// nodes are anchored (before this pass, or by a record of a triangle at or
// before it) is checked; anchored vertices lose their flag.
__global__ void apply_kernel(const DevLevel *__restrict__ Pp, vll_point3 *pts, int64_t n_pts,
                             const vll_tri *tris, int64_t n_tris, const int64_t *tri_nodes,
                             uint8_t *tris_check, const uint8_t *rec,
                             const unsigned long long *first_anchor) {
    const DevLevel &P = *Pp;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_tris;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (tris_check[t] != 0) continue;
        const vll_tri tr = tris[t];
        if (!(tr.a < n_pts && tr.b < n_pts && tr.c < n_pts)) continue;
        bool done = rec[t] != 0;
        const uint32_t v[3] = {tr.a, tr.b, tr.c};
        int nf = 0;
        for (int k = 0; k < 3; ++k) {
            const int64_t nd = tri_nodes[3 * t + k];
            if (anchored(P.gp3[nd].anchor_flag) || first_anchor[nd] <= (unsigned long long)t) {
                ++nf;
                pts[v[k]].flag = 0;
            }
        }
        if (nf == 3) done = true;
        if (done) tris_check[t] = 1;
    }
}

// Anchors the record nodes (anchor_flag = 3) and clears the per-node and
// per-triangle marks for the next iteration.
__global__ void anchor_kernel(vll_ugrid *gp3, int64_t n_nodes, unsigned long long *first_anchor,
                              uint8_t *rec, int64_t n_tris) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_nodes; i += stride) {
        if (first_anchor[i] != ~0ull) {
            gp3[i].anchor_flag = 3;
            first_anchor[i] = ~0ull;
        }
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_tris; i += stride)
        rec[i] = 0;
}

// Longitude / latitude of every grid cell position (col * gs + B0,
// row * gs + B1), the map projection VerticalLineLocus_Ortho applies to every
// cell it samples: computed once per call instead of per height and image.
__global__ void lonlat_kernel(const DevLevel *__restrict__ Pp, double2 *lonlat) {
    const DevLevel &P = *Pp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P.n_nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = i / P.grid_w, col = i % P.grid_w;
        const double cx = __dadd_rn(__dmul_rn((double)col, P.grid_res), P.boundary[0]);
        const double cy = __dadd_rn(__dmul_rn((double)row, P.grid_res), P.boundary[1]);
        lonlat[i] = ps2wgs_dev(P.param, cx, cy);
    }
}

// Grid nodes of every triangle vertex and of every point; flags vertices
// whose node lies outside the grid.
__global__ void nodes_kernel(const DevLevel *__restrict__ Pp, const vll_point3 *pts, int64_t n_pts,
                             const vll_tri *tris, int64_t n_tris, int64_t *tri_nodes,
                             int64_t *pt_nodes, int *bad) {
    const DevLevel &P = *Pp;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pts; i += stride) {
        const int64_t nd = node_of(P, pts[i]);
        pt_nodes[i] = nd;
    }
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_tris; t += stride) {
        const vll_tri tr = tris[t];
        const uint32_t v[3] = {tr.a, tr.b, tr.c};
        for (int k = 0; k < 3; ++k) {
            int64_t nd = 0;
            if (v[k] < n_pts) {
                nd = node_of(P, pts[v[k]]);
                if (nd < 0 || nd >= P.n_nodes) {
                    atomicExch(bad, 1);
                    nd = 0;
                }
            }
            tri_nodes[3 * t + k] = nd;
        }
    }
}

unsigned blocks_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

}  // namespace

cudaError_t launch_ortho_search(const DevLevel *dP, double mpp, const vll_point3 *d_pts3,
                                int64_t target_index, double *d_out, cudaStream_t s) {
    ortho_search_kernel<<<1, 32, 0, s>>>(dP, mpp, d_pts3, target_index, d_out);
    return cudaGetLastError();
}

size_t ortho_blunder_scratch(int64_t n_pts, int64_t n_tris, int64_t n_nodes) {
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int)n_tris);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(tmp) + al(n_tris * 24) + al(n_pts * 8) + al(n_tris) * 3 + al(n_tris * 8) +
           al(n_tris * 4) * 5 + al(n_nodes * 8) + al(16) + al(n_nodes * 16);
}

// Ortho_blunder on device data (scratch of ortho_blunder_scratch bytes).
// Returns the number of iterations in *iterations, or an error.
cudaError_t run_ortho_blunder(const DevLevel *dP, const DevLevel &hP, double mpp, vll_point3 *pts,
                              int64_t n_pts, const vll_tri *tris, int64_t n_tris,
                              vll_ugrid *gp3, void *scratch, size_t scratch_bytes,
                              int *iterations, int *bad_input, cudaStream_t s) {
    *iterations = 0;
    *bad_input = 0;
    char *p = (char *)scratch;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    auto take = [&](size_t b) {
        void *r = p;
        p += al(b);
        return r;
    };
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (const uint32_t *)nullptr,
                                    (uint32_t *)nullptr, (const int32_t *)nullptr,
                                    (int32_t *)nullptr, (int)n_tris);
    void *tmp = take(tmp_bytes);
    int64_t *tri_nodes = (int64_t *)take(n_tris * 24);
    int64_t *pt_nodes = (int64_t *)take(n_pts * 8);
    uint8_t *tris_check = (uint8_t *)take(n_tris);
    uint8_t *upd = (uint8_t *)take(n_tris);
    uint8_t *rec = (uint8_t *)take(n_tris);
    double *hgt = (double *)take(n_tris * 8);
    int32_t *cnt = (int32_t *)take(n_tris * 4);
    uint32_t *key = (uint32_t *)take(n_tris * 4);
    uint32_t *skey = (uint32_t *)take(n_tris * 4);
    int32_t *val = (int32_t *)take(n_tris * 4);
    int32_t *sval = (int32_t *)take(n_tris * 4);
    unsigned long long *first_anchor = (unsigned long long *)take(hP.n_nodes * 8);
    int *flags = (int *)take(16);   // [0] any record, [1] bad input
    double2 *lonlat = (double2 *)take(hP.n_nodes * 16);
    if ((size_t)(p - (char *)scratch) > scratch_bytes) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemsetAsync(tris_check, 0, n_tris, s))) return e;
    if ((e = cudaMemsetAsync(rec, 0, n_tris, s))) return e;
    if ((e = cudaMemsetAsync(first_anchor, 0xff, hP.n_nodes * 8, s))) return e;
    if ((e = cudaMemsetAsync(flags, 0, 16, s))) return e;
    nodes_kernel<<<blocks_for(n_pts > n_tris ? n_pts : n_tris, 256), 256, 0, s>>>(
        dP, pts, n_pts, tris, n_tris, tri_nodes, pt_nodes, flags + 1);
    lonlat_kernel<<<blocks_for(hP.n_nodes, 128), 128, 0, s>>>(dP, lonlat);
    // triangle index as the sort value
    {
        std::vector<int32_t> iota((size_t)n_tris);
        for (int64_t i = 0; i < n_tris; ++i) iota[(size_t)i] = (int32_t)i;
        if ((e = cudaMemcpyAsync(val, iota.data(), n_tris * 4, cudaMemcpyHostToDevice, s)))
            return e;
        if ((e = cudaStreamSynchronize(s))) return e;
    }
    int hflags[2] = {0, 0};
    if ((e = cudaMemcpyAsync(hflags, flags, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    if (hflags[1]) {
        *bad_input = 1;
        return cudaSuccess;
    }
    int end_bit = 1;
    while (end_bit < 32 && ((uint64_t)1 << end_bit) <= (uint64_t)n_pts) ++end_bit;
    const unsigned warps_blocks = blocks_for(n_tris * 32, 128);
    for (int it = 0; it < 200; ++it) {
        *iterations = it + 1;
        if ((e = cudaMemsetAsync(flags, 0, 4, s))) return e;
        tri_search_kernel<<<warps_blocks, 128, 0, s>>>(dP, mpp, pts, n_pts, tris, n_tris,
                                                       tri_nodes, tris_check, upd, hgt, cnt, key,
                                                       lonlat);
        if ((e = cudaGetLastError())) return e;
        if ((e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, skey, val, sval, (int)n_tris,
                                                 0, end_bit, s)))
            return e;
        records_kernel<<<blocks_for(n_tris, 256), 256, 0, s>>>(
            skey, sval, n_tris, (uint32_t)n_pts, cnt, hgt, pt_nodes, pts, rec, first_anchor, flags);
        apply_kernel<<<blocks_for(n_tris, 256), 256, 0, s>>>(dP, pts, n_pts, tris, n_tris,
                                                             tri_nodes, tris_check, rec,
                                                             first_anchor);
        anchor_kernel<<<blocks_for(hP.n_nodes > n_tris ? hP.n_nodes : n_tris, 256), 256, 0, s>>>(
            gp3, hP.n_nodes, first_anchor, rec, n_tris);
        if ((e = cudaGetLastError())) return e;
        if ((e = cudaMemcpyAsync(hflags, flags, 4, cudaMemcpyDeviceToHost, s))) return e;
        if ((e = cudaStreamSynchronize(s))) return e;
        if (!hflags[0]) break;   // no record: check_ortho_cal false, the loop stops
    }
    return cudaSuccess;
}

}  // namespace vll

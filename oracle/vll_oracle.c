/*
 * vll_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C restatement of SETSM's vertical-line-locus matching path.  Each
 * function cites the reference lines it follows.  The arithmetic is written
 * in the reference's evaluation order and compiled without FP contraction
 * (-ffp-contract=off), so on x86-64 it reproduces the reference bit for bit;
 * tests/test_oracle_vs_ref.py checks that against the reference compiled from
 * its own sources (oracle/_ref/libsetsm_ref.so) and tests/golden/ holds the
 * fixtures that pin it when the reference is absent.
 */
#include "vll_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VO_PI 3.141592653589793
#define VO_MAX_HALF 16

void vo_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int vo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- quantisers, Template.hpp:964-993 ------------------------------------
 * The reference converts double -> short through a 32-bit integer
 * (cvttsd2si on x86-64): an out-of-range or NaN input yields 0x80000000 and
 * the short keeps the low 16 bits.  AWNCC's "no peak" sentinel -100.0 thus
 * quantises to (short)(-100000) = 31072. */
static int16_t to_short(double v) {
    if (!(v > -2147483649.0 && v < 2147483648.0)) return 0;
    return (int16_t)(int32_t)v;
}
static int16_t q_result(double v) { return to_short(round(v * 1000.0)); }
static double dq_result(int16_t v) { return (double)v / 1000.0; }
static int16_t q_voxel(double v) { return to_short(v * 1000.0); }
static double dq_voxel(int16_t v) { return (double)v / 1000.0; }

/* ---- geometry -------------------------------------------------------------- */
typedef struct { double x, y; } pt2;

/* GetObjectToImageRPC_single, CoordConversion.hpp:26-86.  rpc is the 90-double
 * row layout; the cubic is summed in the reference's term order and each
 * monomial is multiplied in the reference's association order. */
static pt2 rpc_project(const double *rpc, const double *adj, double X, double Y, double Z) {
    double L = (X - rpc[2]) / rpc[7];
    double P = (Y - rpc[3]) / rpc[8];
    const double H = (Z - rpc[4]) / rpc[9];
    if (L < -10.0 || L > 10.0) {
        X = X > 0 ? X - 360 : X + 360;
        L = (X - rpc[2]) / rpc[7];
    }
    if (P < -10.0 || P > 10.0) {
        Y = Y > 0 ? Y - 360 : Y + 360;
        P = (Y - rpc[3]) / rpc[8];
    }
    const double PL = P * L, LL = L * L, LP = L * P, LH = L * H, PP = P * P, PH = P * H,
                 HH = H * H;
    double coef[4];
    for (int j = 0; j < 4; ++j) {
        const double *c = rpc + 10 + 20 * j;
        double s = c[0] * 1.0;
        s = s + c[1] * L;
        s = s + c[2] * P;
        s = s + c[3] * H;
        s = s + c[4] * L * P;
        s = s + c[5] * L * H;
        s = s + c[6] * P * H;
        s = s + c[7] * L * L;
        s = s + c[8] * P * P;
        s = s + c[9] * H * H;
        s = s + c[10] * PL * H;
        s = s + c[11] * LL * L;
        s = s + c[12] * LP * P;
        s = s + c[13] * LH * H;
        s = s + c[14] * LL * P;
        s = s + c[15] * PP * P;
        s = s + c[16] * PH * H;
        s = s + c[17] * LL * H;
        s = s + c[18] * PP * H;
        s = s + c[19] * HH * H;
        coef[j] = s;
    }
    const double line = (coef[0] / coef[1]) * rpc[5] + rpc[0];
    const double samp = (coef[2] / coef[3]) * rpc[6] + rpc[1];
    pt2 ip;
    ip.y = adj[0] + line;
    ip.x = adj[1] + samp;
    if (ip.y < 0) ip.y = 0;
    if (ip.y > rpc[0] + rpc[5] * 1.2) ip.y = rpc[0] + rpc[5] * 1.2;
    if (ip.x < 0) ip.x = 0;
    if (ip.x > rpc[1] + rpc[6] * 1.2) ip.x = rpc[1] + rpc[6] * 1.2;
    return ip;
}

/* OriginalToPyramid_single, CoordConversion.hpp:96-106 */
static pt2 to_pyramid(pt2 p, const double *startpos, int level) {
    pt2 o;
    o.x = (p.x / (double)(1 << level)) - startpos[0];
    o.y = (p.y / (double)(1 << level)) - startpos[1];
    return o;
}

/* ps2wgs_single, CoordConversion.cpp:396-490 */
static pt2 ps2wgs(const vll_transparam *p, double X, double Y) {
    pt2 w;
    if (p->projection == 1) {
        const double a = p->a, e = p->e, lambda_0 = p->lambda_0, t_c = p->t_c, m_c = p->m_c;
        const int pm = p->pm;
        const double e2 = e * e, e4 = e2 * e2, e6 = e2 * e4, e8 = e4 * e4;
        const double x = X * pm, y = Y * pm;
        const double rho = sqrt(pow(x, 2) + pow(y, 2));
        const double t = rho * t_c / (a * m_c);
        const double chi = VO_PI / 2 - 2 * atan(t);
        double phi = chi + (e2 / 2 + 5 * e4 / 24 + e6 / 12 + 13 * e8 / 360) * sin(2 * chi) +
                     (7 * e4 / 48 + 29 * e6 / 240 + 811 * e8 / 11520) * sin(4 * chi) +
                     (7 * e6 / 120 + 81 * e8 / 1120) * sin(6 * chi) +
                     (4279 * e8 / 161280) * sin(8 * chi);
        double lambda = lambda_0 + atan2(x, -y);
        phi = pm * phi;
        lambda = pm * lambda;
        if (lambda > VO_PI)
            lambda = lambda - 2 * VO_PI;
        else if (lambda < -VO_PI)
            lambda = lambda + 2 * VO_PI;
        w.y = 180 / VO_PI * phi;
        w.x = 180 / VO_PI * lambda;
        return w;
    }
    const int hemis = p->pm;
    const double e2c = p->e2cuadrada, c = p->c;
    const double X0 = X - 500000;
    double Yv = Y;
    if (hemis < 0) Yv = Yv - 10000000;
    const int S = ((p->utm_zone * 6) - 183);
    const double lat = Yv / (6366197.724 * 0.9996);
    const double v = (c / (sqrt(1.0 + (e2c * (cos(lat) * cos(lat)))))) * 0.9996;
    const double a = X0 / v;
    const double a1 = sin(2 * lat);
    const double a2 = a1 * (cos(lat) * cos(lat));
    const double j2 = lat + (a1 / 2.0);
    const double j4 = ((3 * j2) + a2) / 4.0;
    const double j6 = ((5 * j4) + (a2 * (cos(lat) * cos(lat)))) / 3;
    const double alfa = (3 / 4.0) * e2c;
    const double beta = (5 / 3.0) * alfa * alfa;
    const double gama = (35 / 27.0) * alfa * alfa * alfa;
    const double Bm = 0.9996 * c * (lat - alfa * j2 + beta * j4 - gama * j6);
    const double b = (Yv - Bm) / v;
    const double Epsi = ((e2c * a * a) / 2.0) * (cos(lat) * cos(lat));
    const double Eps = a * (1 - (Epsi / 3.0));
    const double nab = (b * (1 - Epsi)) + lat;
    const double senoheps = (exp(Eps) - exp(-Eps)) / 2;
    const double Delt = atan(senoheps / (cos(nab)));
    const double TaO = atan(cos(Delt) * tan(nab));
    w.x = (Delt * (180 / VO_PI)) + S;
    w.y = (lat + (1 + e2c * (cos(lat) * cos(lat)) -
                  (3 / 2.0) * e2c * sin(lat) * cos(lat) * (TaO - lat)) *
                     (TaO - lat)) *
          (180 / VO_PI);
    return w;
}

void vo_rpc_project(const vll_image_desc *im, long n, const double *lon, const double *lat,
                    const double *hgt, double *xy) {
    for (long i = 0; i < n; ++i) {
        pt2 p = rpc_project(im->rpc, im->image_adjust, lon[i], lat[i], hgt[i]);
        xy[2 * i] = p.x;
        xy[2 * i + 1] = p.y;
    }
}

void vo_ps2wgs(const vll_transparam *p, long n, const double *xy, double *lonlat) {
    for (long i = 0; i < n; ++i) {
        pt2 w = ps2wgs(p, xy[2 * i], xy[2 * i + 1]);
        lonlat[2 * i] = w.x;
        lonlat[2 * i + 1] = w.y;
    }
}

/* check_image_boundary, setsm_code.cpp:11002-11083 (RPC sensor). The
 * reference compares against `width - H - 1` computed in unsigned int. */
static int check_image_boundary(const vll_level_desc *d, const double *wgs, double minH,
                                double maxH, int H) {
    int selected = 0, check_reference = 1;
    const int buff = 1;
    for (int ti = 0; ti < d->num_images; ++ti) {
        const vll_image_desc *im = &d->images[ti];
        if (!im->selected) continue;
        const double lim_w = (double)(unsigned)(im->width - (unsigned)H - (unsigned)buff);
        const double lim_h = (double)(unsigned)(im->height - (unsigned)H - (unsigned)buff);
        pt2 t = to_pyramid(rpc_project(im->rpc, im->image_adjust, wgs[0], wgs[1], minH),
                           im->startpos, d->pyramid_step);
        const int s_ok = t.x > H + buff && t.x < lim_w && t.y > H + buff && t.y < lim_h;
        t = to_pyramid(rpc_project(im->rpc, im->image_adjust, wgs[0], wgs[1], maxH),
                       im->startpos, d->pyramid_step);
        const int e_ok = t.x > H + buff && t.x < lim_w && t.y > H + buff && t.y < lim_h;
        if (s_ok && e_ok)
            selected++;
        else if (ti == 0)
            check_reference = 0;
    }
    if (!check_reference) return 0;
    return selected >= 2;
}

/* ---- NCC helpers ----------------------------------------------------------- */
typedef struct {
    int half;
    int cap;
    double *v[4][3];   /* [left, left_mag, right, right_mag][window] */
} kernel_buf;

static void kbuf_init(kernel_buf *k, int half) {
    k->half = half;
    k->cap = (2 * half + 1) * (2 * half + 1);
    for (int c = 0; c < 4; ++c)
        for (int w = 0; w < 3; ++w) k->v[c][w] = (double *)malloc(sizeof(double) * k->cap);
}
static void kbuf_free(kernel_buf *k) {
    for (int c = 0; c < 4; ++c)
        for (int w = 0; w < 3; ++w) free(k->v[c][w]);
}

typedef struct {
    const uint16_t *li, *lm, *ri, *rm;
    uint32_t lw, lh, rw, rh;
} patch_src;

/* InterpolatePatch, SubFunctions.cpp:3317-3326 */
static double interp(const uint16_t *I, long pos, uint32_t width, double dx, double dy) {
    return (double)(I[pos]) * (1 - dx) * (1 - dy) + (double)(I[pos + 1]) * dx * (1 - dy) +
           (double)(I[pos + width]) * (1 - dx) * dy + (double)(I[pos + 1 + width]) * dx * dy;
}

/* SetVecKernelValue, SubFunctions.cpp:3249-3315 */
static void set_vec(kernel_buf *k, const patch_src *s, int row, int col, pt2 pl, pt2 pr,
                    int radius2, int *cnt) {
    if (!(pr.y >= 0 && pr.y + 1 < s->rh && pr.x >= 0 && pr.x + 1 < s->rw && pl.y >= 0 &&
          pl.y + 1 < s->lh && pl.x >= 0 && pl.x + 1 < s->lw))
        return;
    const long pos = (long)pl.x + (long)pl.y * (long)s->lw;
    const long pos_r = (long)pr.x + (long)pr.y * (long)s->rw;
    const double dx = pl.x - floor(pl.x), dy = pl.y - floor(pl.y);
    const double dxr = pr.x - floor(pr.x), dyr = pr.y - floor(pr.y);
    const double lp = interp(s->li, pos, s->lw, dx, dy);
    const double lmp = interp(s->lm, pos, s->lw, dx, dy);
    const double rp = interp(s->ri, pos_r, s->rw, dxr, dyr);
    const double rmp = interp(s->rm, pos_r, s->rw, dxr, dyr);
    if (!(lp > 0 && rp > 0)) return;
    const int H = k->half;
    const double vals[4] = {lp, lmp, rp, rmp};
    for (int c = 0; c < 4; ++c) k->v[c][0][cnt[0]] = vals[c];
    cnt[0]++;
    const int size_1 = (int)(H / 2);
    if (radius2 <= (H - size_1 + 1) * (H - size_1 + 1) && row >= -H + size_1 &&
        row <= H - size_1 && col >= -H + size_1 && col <= H - size_1) {
        for (int c = 0; c < 4; ++c) k->v[c][1][cnt[1]] = vals[c];
        cnt[1]++;
    }
    const int size_2 = size_1 + (int)((size_1 / 2.0) + 0.5);
    if (radius2 <= (H - size_2 + 1) * (H - size_2 + 1) && row >= -H + size_2 &&
        row <= H - size_2 && col >= -H + size_2 && col <= H - size_2) {
        for (int c = 0; c < 4; ++c) k->v[c][2][cnt[2]] = vals[c];
        cnt[2]++;
    }
}

/* Correlate, SubFunctions.cpp:974-1018 (two-pass Pearson, -99 when undefined) */
static double correlate(const double *L, const double *R, int N) {
    if (N <= 0) return -99.0;
    double Lm = 0, Rm = 0;
    for (int i = 0; i < N; ++i) {
        Lm += L[i];
        Rm += R[i];
    }
    Lm = Lm / N;
    Rm = Rm / N;
    double SLR = 0, SL2 = 0, SR2 = 0;
    for (int i = 0; i < N; ++i) {
        SLR += (L[i] - Lm) * (R[i] - Rm);
        SL2 += (L[i] - Lm) * (L[i] - Lm);
        SR2 += (R[i] - Rm) * (R[i] - Rm);
    }
    if (SL2 > 1e-8 && SR2 > 1e-8) return SLR / (sqrt(SL2 * SR2));
    return -99.0;
}

/* ComputeMultiNCC, SubFunctions.cpp:3328-3360 (threshold TH_N = 0) */
static void multi_ncc(const kernel_buf *k, const int *cnt, double *count_ncc, double *sum_ncc) {
    if (!(cnt[0] > 0 && cnt[1] > 0 && cnt[2] > 0)) return;
    double s = 0, n = 0;
    for (int w = 0; w < 3; ++w) {
        const double a = correlate(k->v[0][w], k->v[2][w], cnt[w]);
        if (a != -99) {
            n++;
            s += a;
        }
        const double b = correlate(k->v[1][w], k->v[3][w], cnt[w]);
        if (b != -99) {
            n++;
            s += b;
        }
    }
    if (n > 0) {
        *sum_ncc += s / n;
        *count_ncc += 1;
    }
}

/* SetNCC_alpha, setsm_code.cpp:6014-6047 */
static double ncc_alpha_of(int L, int it, int is_ra) {
    double a;
    if (L >= 4) {
        a = 1.0 - ((4 - L) * 0.2 + (it - 1) * 0.05);
        if (a < 0.8) a = 0.8;
    } else if (L >= 3) {
        a = 1.0 - ((4 - L) * 0.2 + (it - 1) * 0.05);
        if (a < 0.6) a = 0.6;
    } else if (L == 2) {
        a = 1.0 - (0.4 + (it - 1) * 0.05);
        if (a < 0.4) a = 0.4;
    } else
        a = 1.0 - ((4 - L) * 0.2 + (it - 1) * 0.05);
    if (a < 0.1) a = 0.1;
    if (is_ra) a = 1.0;
    return a;
}

/* FindPeakNcc, setsm_code.cpp:6672-6752 (all three branches test the same
 * condition, direction > 0 && t_direction < 0). */
typedef struct {
    int check_rho;
    double pre_rho;
    float pre_height;
    int direction;
} peak_state;

static void find_peak(peak_state *st, double rho, float height, vll_nccresult *r) {
    double diff;
    int td;
    if (rho >= 0 && st->pre_rho >= 0)
        diff = rho - st->pre_rho;
    else if (rho < 0 && st->pre_rho < 0)
        diff = -(fabs(rho) - fabs(st->pre_rho));
    else if (rho >= 0 && st->pre_rho < 0)
        diff = 1;
    else
        diff = -1;
    td = diff > 0 ? 1 : (diff < 0 ? -1 : 0);
    if (!st->check_rho) {
        st->check_rho = 1;
        td = -1;
    } else if (st->pre_rho != -1) {
        if (st->direction > 0 && td < 0) {
            if (r->result4 < 10) r->result4 += 1;
            if (r->result0 < q_result(st->pre_rho)) {
                const double t1 = dq_result(r->result0);
                r->result0 = q_result(st->pre_rho);
                const float t2 = r->result2;
                r->result2 = st->pre_height;
                if (r->result1 < q_result(t1)) {
                    r->result1 = q_result(t1);
                    r->result3 = t2;
                }
            } else if (r->result1 < q_result(st->pre_rho)) {
                r->result1 = q_result(st->pre_rho);
                r->result3 = st->pre_height;
            }
        }
    }
    st->pre_rho = rho;
    st->pre_height = height;
    st->direction = td;
}

/* ---- SetOrthoImageCoord, setsm_code.cpp:6550-6670 (OR pyramid) ------------- */
typedef struct {
    long w, h, w_next, h_next;
    pt2 *cd[VLL_MAX_IMAGES];
    pt2 *cd_next[VLL_MAX_IMAGES];
} ortho_coords;

static void ortho_coords_build(const vll_level_desc *d, const vll_ugrid *g, int combined,
                               double im_res, double im_res_next, ortho_coords *oc) {
    memset(oc, 0, sizeof(*oc));
    const double *B = d->boundary;
    oc->w = (long)((B[2] - B[0]) / im_res) + 1;
    oc->h = (long)((B[3] - B[1]) / im_res) + 1;
    if (combined) {
        oc->w_next = (long)((B[2] - B[0]) / im_res_next) + 1;
        oc->h_next = (long)((B[3] - B[1]) / im_res_next) + 1;
    }
    const long total = oc->w * oc->h;
    for (int ti = 0; ti < d->num_images; ++ti) {
        if (!d->images[ti].selected) continue;
        oc->cd[ti] = (pt2 *)calloc((size_t)total, sizeof(pt2));
        if (combined) oc->cd_next[ti] = (pt2 *)calloc((size_t)(oc->w_next * oc->h_next), sizeof(pt2));
    }
    const long grid_len = d->grid_width * d->grid_height;
#pragma omp parallel for schedule(guided)
    for (long it = 0; it < total; ++it) {
        const long row = (long)floor(it / oc->w);
        const long col = it % oc->w;
        const double tX = B[0] + col * im_res;
        const double tY = B[1] + row * im_res;
        const long t_col = (long)((tX - B[0]) / d->grid_resolution);
        const long t_row = (long)((tY - B[1]) / d->grid_resolution);
        const long pt = t_row * (long)d->grid_width + t_col;
        const long pim = row * oc->w + col;
        long tcn = 0, trn = 0, pimn = 0;
        if (combined) {
            tcn = (long)((tX - B[0]) / im_res_next);
            trn = (long)((tY - B[1]) / im_res_next);
            pimn = trn * oc->w_next + tcn;
        }
        if (pt < grid_len && t_col < d->grid_width && t_row < d->grid_height &&
            g[pt].Height != -1000) {
            const pt2 w = ps2wgs(&d->param, tX, tY);
            const double Z = (double)g[pt].Height;
            for (int ti = 0; ti < d->num_images; ++ti) {
                const vll_image_desc *im = &d->images[ti];
                if (!im->selected) continue;
                const pt2 ic = rpc_project(im->rpc, im->image_adjust, w.x, w.y, Z);
                oc->cd[ti][pim] = to_pyramid(ic, im->startpos, d->pyramid_step);
                if (combined && pimn < oc->w_next * oc->h_next && tcn < oc->w_next &&
                    trn < oc->h_next)
                    oc->cd_next[ti][pimn] = to_pyramid(ic, im->startpos_next, d->pyramid_step - 1);
            }
        }
    }
}

static void ortho_coords_free(ortho_coords *oc) {
    for (int ti = 0; ti < VLL_MAX_IMAGES; ++ti) {
        free(oc->cd[ti]);
        free(oc->cd_next[ti]);
    }
}

/* UGRID.ortho_ncc[ti] (Typedefine.hpp:270-283).  The array has MaxNCC = 2
 * entries; the reference indexes it by image id, so for ti >= 2 it reads the
 * following fields of the record.  Reads past the last record yield 0. */
static int16_t ugrid_ortho_ncc(const vll_ugrid *G, long n, long pt, int ti) {
    const long byte = 10 + 2 * (long)ti;
    const long rec = pt + byte / (long)sizeof(vll_ugrid);
    if (rec >= n) return 0;
    int16_t v;
    memcpy(&v, (const char *)G + pt * (long)sizeof(vll_ugrid) + byte, sizeof(v));
    return v;
}

/* ---- VerticalLineLocus, setsm_code.cpp:6049-6548 --------------------------- */
long vo_vertical_line_locus(const vll_level_desc *d, const vll_ugrid *G, vll_nccresult *R,
                            vll_voxel *voxels, long cap, const int64_t *rho_offsets,
                            double *rho_out, int64_t *evals_out) {
    const int L = d->pyramid_step;
    const int is_ra = d->is_ra != 0;
    const int cmr = d->check_matching_rate != 0;
    int template_size = d->template_size;
    if (L >= 1) {
        const double area = 5.0;
        const int t = (int)((area / (d->resolution * (1 << L))) / 2.0) * 2 + 1;
        if (d->template_size < t) template_size = t;
    }
    int H = template_size / 2;
    if (L == 3)
        H = H - 1;
    else if (L < 3)
        H = H - 2;
    if (H < 1 || H > VO_MAX_HALF) return -1;

    const long N = d->grid_width * d->grid_height;
    const int combined = !is_ra && (L > d->py_combined_level);
    const int combined_incc = combined && (L >= 1 && d->iteration % 2 == 0);
    double im_res_next = d->resolution;
    if (combined) im_res_next = d->resolution * (1 << (L - 1));
    const double im_res = d->resolution * (1 << L);

    int check_ortho = !((L == 4 && d->iteration == 1) || is_ra);
    if (d->pre_dem_tif && !(L == 4 && d->iteration == 1)) check_ortho = 1;
    if (d->check_matchtag) check_ortho = 1;
    if (L <= d->sgm_py) check_ortho = 0;

    ortho_coords oc;
    memset(&oc, 0, sizeof(oc));
    if (check_ortho) ortho_coords_build(d, G, combined, im_res, im_res_next, &oc);

    const double alpha = ncc_alpha_of(L, d->iteration, is_ra);
    const double beta = 1.0 - alpha;
    const int ref = d->reference_id;
    const double ortho_th = 0.7 - (4 - L) * 0.10;
    const double *B = d->boundary;

    /* voxel row offsets by the incoming NumOfHeight */
    int64_t *voff = NULL;
    if (!cmr && !is_ra && voxels) {
        voff = (int64_t *)malloc(sizeof(int64_t) * (size_t)(N + 1));
        voff[0] = 0;
        for (long i = 0; i < N; ++i) voff[i + 1] = voff[i] + R[i].NumOfHeight;
        if (voff[N] > cap) {
            free(voff);
            ortho_coords_free(&oc);
            return -2;
        }
    }

    long accessable = 0;
    int64_t evals = 0;
#pragma omp parallel reduction(+ : accessable, evals)
    {
        kernel_buf kb, kbn;
        kbuf_init(&kb, H);
        kbuf_init(&kbn, H);
#pragma omp for schedule(dynamic, 16)
        for (long pt = 0; pt < N; ++pt) {
            const int start_H = G[pt].minHeight;
            const int end_H = G[pt].maxHeight;
            const double *wgs = d->grid_wgs + 2 * pt;
            if (!check_image_boundary(d, wgs, start_H, end_H, H)) continue;
            double th_height = 1000;
            if (d->dem_resolution <= 4) th_height = 500;
            int blunder = 0;
            if (L >= 2)
                blunder = 0;
            else if (G[pt].Matched_flag == 0)
                blunder = 1;
            else
                blunder = !(abs(G[pt].maxHeight - G[pt].minHeight) < th_height);
            if (L <= 1 && (G[pt].maxHeight > d->minmax_height[1] ||
                           G[pt].minHeight < d->minmax_height[0]))
                blunder = 1;
            if (d->check_matchtag && d->iteration <= 2) {
                blunder = 0;
                if (G[pt].maxHeight > d->minmax_height[1] || G[pt].minHeight < d->minmax_height[0])
                    blunder = 1;
                else if (abs(G[pt].maxHeight - G[pt].minHeight) > th_height)
                    blunder = 1;
            }
            if (blunder) continue;

            for (int ti = 1; ti < d->num_images; ++ti) {
                if (!d->images[ti].selected) continue;
                accessable++;
                const vll_image_desc *ri = &d->images[ref];
                const vll_image_desc *tI = &d->images[ti];
                const patch_src ps = {ri->image, ri->mag, tI->image, tI->mag,
                                      ri->width, ri->height, tI->width, tI->height};
                const patch_src psn = {ri->image_next, ri->mag_next, tI->image_next, tI->mag_next,
                                       ri->width_next, ri->height_next, tI->width_next,
                                       tI->height_next};
                double sum_gncc = 0, count_gncc = 0;

                /* GNCC, setsm_code.cpp:6241-6305 */
                if (check_ortho && dq_result(ugrid_ortho_ncc(G, N, pt, ti)) > ortho_th) {
                    int cnt[3] = {0, 0, 0}, cntn[3] = {0, 0, 0};
                    const double gx = d->grid_pts[2 * pt], gy = d->grid_pts[2 * pt + 1];
                    for (int row = -H; row <= H; ++row) {
                        for (int col = -H; col <= H; ++col) {
                            const int r2 = row * row + col * col;
                            if (r2 > (H + 1) * (H + 1)) continue;
                            const double tX = gx + col * im_res;
                            const double tY = gy + row * im_res;
                            long t_col = (long)((tX - B[0]) / im_res);
                            long t_row = (long)((tY - B[1]) / im_res);
                            long pit = t_row * oc.w + t_col;
                            const long tt_col = (long)((tX - B[0]) / d->grid_resolution);
                            const long tt_row = (long)((tY - B[1]) / d->grid_resolution);
                            const long pdem = tt_row * (long)d->grid_width + tt_col;
                            if (pit >= 0 && pit < oc.w * oc.h && t_col >= 0 && t_col < oc.w &&
                                t_row >= 0 && t_row < oc.h && pdem >= 0 && pdem < N &&
                                tt_col >= 0 && tt_col < d->grid_width && tt_row >= 0 &&
                                tt_row < d->grid_height && oc.cd[ref] && oc.cd[ti]) {
                                if (G[pdem].Height != -1000) {
                                    set_vec(&kb, &ps, row, col, oc.cd[ref][pit], oc.cd[ti][pit],
                                            r2, cnt);
                                    if (combined) {
                                        t_col = (long)((tX - B[0]) / im_res_next);
                                        t_row = (long)((tY - B[1]) / im_res_next);
                                        pit = t_row * oc.w_next + t_col;
                                        if (pit >= 0 && pit < oc.w_next * oc.h_next &&
                                            t_col < oc.w_next && t_row < oc.h_next)
                                            set_vec(&kbn, &psn, row, col, oc.cd_next[ref][pit],
                                                    oc.cd_next[ti][pit], r2, cntn);
                                    }
                                }
                            }
                        }
                    }
                    multi_ncc(&kb, cnt, &count_gncc, &sum_gncc);
                    if (combined) multi_ncc(&kbn, cntn, &count_gncc, &sum_gncc);
                    R[pt].GNCC = count_gncc > 0 ? q_result(sum_gncc / count_gncc) : q_result(-1.0);
                } else {
                    R[pt].GNCC = q_result(-1.0);
                }

                /* INCC, setsm_code.cpp:6307-6514 */
                const int num_heights = (int)((end_H - start_H) / d->height_step);
                if (is_ra || cmr) {
                    R[pt].check_height_change = 1;
                    R[pt].NumOfHeight = (uint16_t)num_heights;
                }
                if (!(is_ra || cmr || R[pt].check_height_change ||
                      (L == 0 && d->dem_resolution < 2)))
                    continue;
                peak_state st = {0, -1.0, 0.0f, 0};
                double max_wncc = -100;
                R[pt].result0 = q_result(-1.0);
                R[pt].result2 = -1000;
                R[pt].result1 = q_result(-1.0);
                R[pt].result3 = -1000;
                R[pt].result4 = 0;
                const int nh = R[pt].NumOfHeight;
                for (int k = 0; k < nh; ++k) {
                    float hgt;
                    if (is_ra || cmr)
                        hgt = (float)(start_H + k * d->height_step);
                    else
                        hgt = (float)(R[pt].minHeight + k * d->height_step);
                    if (!(hgt >= start_H && hgt <= end_H)) continue;
                    const pt2 rc = rpc_project(ri->rpc, ri->image_adjust, wgs[0], wgs[1], (double)hgt);
                    const pt2 tc = rpc_project(tI->rpc, tI->image_adjust, wgs[0], wgs[1], (double)hgt);
                    const pt2 rp = to_pyramid(rc, ri->startpos, L);
                    const pt2 tp = to_pyramid(tc, tI->startpos, L);
                    const int ok = (int)rp.y >= 0 && (unsigned)((int)rp.y + 1) < ri->height &&
                                   (int)rp.x >= 0 && (unsigned)((int)rp.x + 1) < ri->width &&
                                   (int)tp.y >= 0 && (unsigned)((int)tp.y + 1) < tI->height &&
                                   (int)tp.x >= 0 && (unsigned)((int)tp.x + 1) < tI->width;
                    pt2 rpn = {0, 0}, tpn = {0, 0};
                    int okn = 1;
                    if (combined_incc) {
                        rpn = to_pyramid(rc, ri->startpos_next, L - 1);
                        tpn = to_pyramid(tc, tI->startpos_next, L - 1);
                        okn = (int)rpn.y >= 0 && (unsigned)((int)rpn.y + 1) < ri->height_next &&
                              (int)rpn.x >= 0 && (unsigned)((int)rpn.x + 1) < ri->width_next &&
                              (int)tpn.y >= 0 && (unsigned)((int)tpn.y + 1) < tI->height_next &&
                              (int)tpn.x >= 0 && (unsigned)((int)tpn.x + 1) < tI->width_next;
                    }
                    if (!(ok && okn)) continue;
                    const int od = (int)ri->ori[(long)(int)rp.y * ri->width + (int)rp.x] -
                                   (int)tI->ori[(long)(int)tp.y * tI->width + (int)tp.x];
                    int odn = 0;
                    if (combined_incc)
                        odn = (int)ri->ori_next[(long)(int)rpn.y * ri->width_next + (int)rpn.x] -
                              (int)tI->ori_next[(long)(int)tpn.y * tI->width_next + (int)tpn.x];
                    double dtheta = (double)od;
                    if (combined_incc) dtheta = (dtheta + (double)odn) / 2.0;
                    int check_orient = 0;
                    if (!is_ra) {
                        if (L >= 3 && dtheta * d->bin_angle < 90 && dtheta * d->bin_angle > -90)
                            check_orient = 1;
                        else if (L <= 2)
                            check_orient = 1;
                    } else
                        check_orient = 1;
                    vll_voxel *vx = voff ? &voxels[voff[pt] + k] : NULL;
                    if (!check_orient) {
                        if (vx) vx->flag_cal = 0;
                        continue;
                    }
                    double sum_incc = 0, count_incc = 0;
                    int cnt[3] = {0, 0, 0}, cntn[3] = {0, 0, 0};
                    const double rot = (double)(dtheta * d->bin_angle * VO_PI / 180.0);
                    const double c0 = cos(-rot), s0 = sin(-rot);
                    for (int row = -H; row <= H; ++row) {
                        for (int col = -H; col <= H; ++col) {
                            const int r2 = row * row + col * col;
                            if (r2 > (H + 1) * (H + 1)) continue;
                            const pt2 pl = {rp.x + col, rp.y + row};
                            const pt2 off = {c0 * col - s0 * row, s0 * col + c0 * row};
                            const pt2 pr = {tp.x + off.x, tp.y + off.y};
                            set_vec(&kb, &ps, row, col, pl, pr, r2, cnt);
                            if (combined_incc) {
                                const pt2 pln = {rpn.x + col, rpn.y + row};
                                const pt2 prn = {tpn.x + off.x, tpn.y + off.y};
                                set_vec(&kbn, &psn, row, col, pln, prn, r2, cntn);
                            }
                        }
                    }
                    evals++;
                    multi_ncc(&kb, cnt, &count_incc, &sum_incc);
                    if (cnt[0] > 0 && cnt[1] > 0 && cnt[2] > 0 && vx) vx->flag_cal = 1;
                    if (combined_incc) multi_ncc(&kbn, cntn, &count_incc, &sum_incc);
                    if (vx)
                        vx->INCC = count_incc > 0 ? q_voxel(sum_incc / count_incc) : q_voxel(-1.0);
                    double rho;
                    if (check_ortho && count_gncc > 0)
                        rho = sum_incc / count_incc * alpha + sum_gncc / count_gncc * beta;
                    else
                        rho = count_incc > 0 ? sum_incc / count_incc : -1.0;
                    if (rho_out) rho_out[rho_offsets[pt] + k] = rho;
                    if (max_wncc < rho) max_wncc = rho;
                    if (cmr) {
                        find_peak(&st, rho, hgt, &R[pt]);
                        if (max_wncc < rho) max_wncc = rho;
                    }
                }
                if (R[pt].check_height_change) R[pt].max_WNCC = q_result(max_wncc);
            }
        }
        kbuf_free(&kb);
        kbuf_free(&kbn);
    }
    free(voff);
    ortho_coords_free(&oc);
    if (evals_out) *evals_out = evals;
    return accessable;
}

/* ---- AWNCC peak loop without SGM, setsm_code.cpp:7511-7702 ------------------ */
void vo_awncc_peaks(const vll_level_desc *d, const vll_ugrid *G, vll_nccresult *R,
                    const vll_voxel *voxels, long cap) {
    const int L = d->pyramid_step, it = d->iteration;
    int check_ortho = !(L == 4 && it == 1);
    if (d->pre_dem_tif && !(L == 4 && it == 1)) check_ortho = 1;
    const double alpha = ncc_alpha_of(L, it, d->is_ra);
    const double beta = 1.0 - alpha;
    const int max_mode = (it <= 3 && L == 4) || (it <= 2 && L == 3) || (it <= 1 && L == 2);
    const long N = d->grid_width * d->grid_height;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * (size_t)(N + 1));
    off[0] = 0;
    for (long i = 0; i < N; ++i) off[i + 1] = off[i] + R[i].NumOfHeight;
    if (off[N] > cap) {
        free(off);
        return;
    }
#pragma omp parallel for schedule(guided)
    for (long pt = 0; pt < N; ++pt) {
        double pre_rho = -1.0;
        float pre_height = 0.0f;
        int direction = 0, check_rho = 0;
        double best = -100.0, second = -100.0;
        R[pt].result0 = q_result(-1.0);
        R[pt].result2 = -1000;
        R[pt].result1 = q_result(-1.0);
        R[pt].result3 = -1000;
        R[pt].result4 = 0;
        for (long k = 0; k < R[pt].NumOfHeight; ++k) {
            const float hgt = (float)(R[pt].minHeight + k * d->height_step);
            if (!(hgt >= G[pt].minHeight && hgt <= G[pt].maxHeight)) continue;
            const vll_voxel v = voxels[off[pt] + k];
            double rho;
            if (check_ortho && dq_result(R[pt].GNCC) > -1.0)
                rho = dq_voxel(v.INCC) * alpha + dq_result(R[pt].GNCC) * beta;
            else
                rho = dq_voxel(v.INCC);
            double diff;
            int td;
            if (rho >= 0 && pre_rho >= 0)
                diff = rho - pre_rho;
            else if (rho < 0 && pre_rho < 0)
                diff = -(fabs(rho) - fabs(pre_rho));
            else if (rho >= 0 && pre_rho < 0)
                diff = 1;
            else
                diff = -1;
            td = diff > 0 ? 1 : (diff < 0 ? -1 : 0);
            if (!check_rho) {
                check_rho = 1;
                td = -1;
            } else if (pre_rho != -1) {
                const int is_peak = direction > 0 && td < 0;
                if (max_mode) {
                    if (best < rho) {
                        if (R[pt].result4 < 10) R[pt].result4 += 1;
                        best = rho;
                        R[pt].result2 = hgt;
                        second = -1.0;
                        R[pt].result3 = -9999;
                    }
                } else if (is_peak) {
                    if (R[pt].result4 < 10) R[pt].result4 += 1;
                    if (best < pre_rho) {
                        const double t1 = best;
                        best = pre_rho;
                        const float t2 = R[pt].result2;
                        R[pt].result2 = pre_height;
                        if (second < t1) {
                            second = t1;
                            R[pt].result3 = t2;
                        }
                    } else if (second < pre_rho) {
                        second = pre_rho;
                        R[pt].result3 = pre_height;
                    }
                }
            }
            pre_rho = rho;
            pre_height = hgt;
            direction = td;
        }
        R[pt].result0 = q_result(best);
        R[pt].result1 = q_result(second);
    }
    free(off);
}

/* ---- InitializeVoxel, setsm_code.cpp:5759-6012 ----------------------------- */
long vo_initialize_voxel(const vll_level_desc *d, vll_ugrid *G, vll_nccresult *R,
                         const vll_voxel *vin, vll_voxel *vout, long cap) {
    const double hs = d->height_step;
    const int L = d->pyramid_step, it = d->iteration;
    const long N = d->grid_width * d->grid_height;
    /* nodes whose voxel row is (re)initialised; others keep their previous row */
    uint8_t *fresh = (uint8_t *)calloc((size_t)N, 1);
    int64_t *old_off = (int64_t *)malloc(sizeof(int64_t) * (size_t)(N + 1));
    uint16_t *old_n = (uint16_t *)malloc(sizeof(uint16_t) * (size_t)N);
    old_off[0] = 0;
    for (long i = 0; i < N; ++i) {
        old_n[i] = R[i].NumOfHeight;
        old_off[i + 1] = old_off[i] + R[i].NumOfHeight;
    }
#pragma omp parallel for schedule(guided)
    for (long t = 0; t < N; ++t) {
        vll_ugrid *g = &G[t];
        vll_nccresult *r = &R[t];
        if (check_image_boundary(d, d->grid_wgs + 2 * t, g->minHeight, g->maxHeight, 7)) {
            int csmin = 0, csmax = 0;
            int blunder = 1;
            double th_height = 1000;
            if (d->dem_resolution <= 4) th_height = 500;
            if (d->check_matchtag || it == 1) {
                r->minHeight = g->minHeight;
                r->maxHeight = g->maxHeight;
                r->GNCC = q_result(-1.0);
                r->check_height_change = 1;
                blunder = 0;
            } else {
                if (L >= 2)
                    blunder = 0;
                else if (g->Matched_flag != 0) {
                    if (g->maxHeight - g->minHeight > 0) {
                        if (L <= 1) {
                            if (it > 1)
                                blunder = !(g->maxHeight <= d->minmax_height[1] &&
                                            g->minHeight >= d->minmax_height[0] &&
                                            r->maxHeight <= d->minmax_height[1] &&
                                            r->minHeight >= d->minmax_height[0]);
                            else
                                blunder = !(g->maxHeight <= d->minmax_height[1] &&
                                            g->minHeight >= d->minmax_height[0]);
                        }
                        if (L == 1) blunder = !(abs(g->maxHeight - g->minHeight) < 1000);
                        if (L == 0) {
                            if (it > 1)
                                blunder = !((abs(r->maxHeight - r->minHeight) < th_height) &&
                                            (abs(g->maxHeight - g->minHeight) < th_height));
                            else if (abs(g->maxHeight - g->minHeight) < th_height)
                                blunder = 0;
                            else
                                r->NumOfHeight = 0;
                        }
                    } else {
                        r->NumOfHeight = 0;
                        blunder = 1;
                    }
                } else {
                    r->NumOfHeight = 0;
                    blunder = 1;
                }
            }
            if (!blunder) {
                if (it == 1 || (L == 0 && d->dem_resolution < 2)) {
                    r->minHeight = g->minHeight;
                    r->maxHeight = g->maxHeight;
                    r->GNCC = q_result(-1.0);
                    r->check_height_change = 1;
                    if (L == 1) {
                        if (abs((int)g->maxHeight - (int)g->minHeight) > 1000) {
                            g->maxHeight = -100;
                            g->minHeight = -100;
                            r->check_height_change = 0;
                        }
                    } else if (L == 0) {
                        if (abs((int)g->maxHeight - (int)g->minHeight) > th_height) {
                            g->maxHeight = -100;
                            g->minHeight = -100;
                            r->check_height_change = 0;
                        }
                    }
                } else {
                    const int nv = (int)((g->maxHeight - g->minHeight) / hs);
                    if (r->NumOfHeight == 0 && nv > 0) {
                        csmin = 0;
                        csmax = 0;
                        r->check_height_change = 1;
                    } else if (r->minHeight > g->minHeight || r->maxHeight < g->maxHeight) {
                        if (r->minHeight > g->minHeight)
                            csmin = (int)((r->minHeight - g->minHeight) / hs + 0.5);
                        if (r->maxHeight < g->maxHeight)
                            csmax = (int)((g->maxHeight - r->maxHeight) / hs + 0.5);
                        r->minHeight = (int16_t)floor(r->minHeight - csmin * hs);
                        r->maxHeight = (int16_t)ceil(r->maxHeight + csmax * hs);
                        r->check_height_change = 1;
                        if (L == 0 && abs(r->maxHeight - r->minHeight) > th_height)
                            r->check_height_change = 0;
                    } else {
                        r->check_height_change = 0;
                    }
                }
                if (r->check_height_change) {
                    r->minHeight = (int16_t)floor(r->minHeight - csmin * hs);
                    r->maxHeight = (int16_t)ceil(r->maxHeight + csmax * hs);
                    const int nv = (int)((float)(r->maxHeight - r->minHeight) / hs);
                    if (nv > 0) {
                        r->NumOfHeight = (uint16_t)nv;
                        fresh[t] = 1;
                    } else {
                        r->NumOfHeight = 0;
                        r->check_height_change = 0;
                    }
                }
            } else {
                r->NumOfHeight = 0;
                r->check_height_change = 0;
            }
        } else {
            r->NumOfHeight = 0;
            r->check_height_change = 0;
        }
        if (r->minHeight == 0 || r->maxHeight == 0) {
            r->NumOfHeight = 0;
            r->check_height_change = 0;
        }
        if (L == 0 && r->NumOfHeight > 1000) {
            r->NumOfHeight = 0;
            r->check_height_change = 0;
        }
    }
    /* pack: fresh rows are (flag_cal = 1, INCC = -1000); kept rows carry over */
    long o = 0;
    for (long t = 0; t < N; ++t) {
        const int n = R[t].NumOfHeight;
        for (int h = 0; h < n; ++h) {
            if (o + h >= cap) break;
            if (fresh[t] || !vin || h >= old_n[t]) {
                vout[o + h].flag_cal = 1;
                vout[o + h].INCC = q_voxel(-1);
            } else {
                vout[o + h] = vin[old_off[t] + h];
            }
        }
        o += n;
    }
    free(fresh);
    free(old_off);
    free(old_n);
    return o;
}

/* ---- image preprocessing --------------------------------------------------- */
/* MakeSobelMagnitudeImage, SubFunctions.cpp:2418-2471 */
void vo_sobel(uint32_t w, uint32_t h, const uint16_t *s, uint16_t *mag, int16_t *dir) {
#pragma omp parallel for
    for (long i = 0; i < (long)h; ++i) {
        for (long j = 0; j < (long)w; ++j) {
            const long p = i * w + j;
            if (j == 0 || j == (long)w - 1 || i == 0 || i == (long)h - 1) {
                mag[p] = 0;
                dir[p] = 0;
                continue;
            }
            const int a = s[p - w - 1], b = s[p - w], c = s[p - w + 1];
            const int dd = s[p - 1], f = s[p + 1];
            const int g = s[p + w - 1], hh = s[p + w], k = s[p + w + 1];
            const double gx = (double)(-a + c - 2 * dd + 2 * f - g + k);
            const double gy = (double)(a + 2 * b + c - g - 2 * hh - k);
            const double m = sqrt(gx * gx + gy * gy);
            dir[p] = (int16_t)(floor(atan2(gy, gx) * 180 / VO_PI));
            mag[p] = (uint16_t)(m + 0.5);
        }
    }
}

/* Orientation, SubFunctions.cpp:2473-2560.  The window walks rows
 * -half+1..half-1 and, per row, columns from max(-mask_row, -numcols[|row|])
 * (the reference bounds the column start by the ROW index) to
 * min(numcols[|row|], w-mask_col-1); pixels it addresses before the first
 * image row contribute nothing here (the reference reads whatever precedes
 * the buffer).  The final bin search scans [(int)(sub*4.6), (int)(sub*4.6+4.6)). */
void vo_orientation(uint32_t w, uint32_t h, const uint16_t *mag, const int16_t *dir,
                    int template_size, uint8_t *ori) {
    static const int numcols[7] = {6, 5, 5, 5, 4, 3, 0};
    const int half = template_size / 2;
    const int sz = 2 * half - 1;
    double *wt = (double *)malloc(sizeof(double) * (size_t)(sz * sz));
    for (int r = -half + 1; r <= half - 1; ++r)
        for (int c = -half + 1; c <= half - 1; ++c)
            wt[(half - 1 + r) * sz + (half - 1 + c)] = exp(-(double)(r * r + c * c) / 4.5);
    const long W = w, Hh = h;
#pragma omp parallel for
    for (long mr = 0; mr < Hh; ++mr) {
        for (long mc = 0; mc < W; ++mc) {
            double bin[18] = {0};
            double sub[4] = {0};
            const long r_lo = (-mr > -half + 1) ? -mr : -half + 1;
            const long r_hi = (Hh - mr - 1 < half - 1) ? Hh - mr - 1 : half - 1;
            for (long r = r_lo; r <= r_hi; ++r) {
                const int dcol = numcols[r < 0 ? -r : r];
                const long c_lo = (-mr > -dcol) ? -mr : -dcol;
                const long c_hi = (dcol < W - mc - 1) ? dcol : W - mc - 1;
                for (long c = c_lo; c <= c_hi; ++c) {
                    const double gw = wt[(half - 1 + r) * sz + (half - 1 + c)];
                    const long idx = (mr + r) * W + (mc + c);
                    if (idx < 0) continue;
                    const double m = mag[idx];
                    double theta = (double)dir[idx];
                    if (theta < 0)
                        theta += 360;
                    else if (theta > 360)
                        theta -= 360;
                    const long bi = (long)(theta / 20.0);
                    if (bi >= 0 && bi < 18) {
                        bin[bi] += m * gw;
                        sub[(int)(bi / 4.6)] += m * gw;
                    }
                }
            }
            double mx = -100;
            int sub_th = 0, th = 0;
            for (int i = 0; i < 4; ++i)
                if (sub[i] > mx) {
                    mx = sub[i];
                    sub_th = i;
                }
            mx = -100;
            for (int i = (int)(sub_th * 4.6); i < (int)(sub_th * 4.6 + 4.6); ++i) {
                if (bin[i] > mx) {
                    mx = bin[i];
                    th = i;
                }
            }
            ori[mr * W + mc] = (uint8_t)th;
        }
    }
    free(wt);
}

/* CreateImagePyramid<uint16>(.., 9, 1.5), Template.hpp:45-131: 9x9 Gaussian
 * normalised to unit sum, applied at every even pixel; border outputs copy
 * the source pixel. */
void vo_pyramid_down(uint32_t w, uint32_t h, const uint16_t *src, uint16_t *out) {
    const int fs = 9, hf = 4;
    const double sigma = 1.5;
    double f[81];
    double sum = 0;
    const double tmp = -1 / (2 * sigma * sigma);
    const double scale = 1 / (sqrt(2 * VO_PI) * sigma);
    for (int i = -hf; i <= hf; ++i)
        for (int j = -hf; j <= hf; ++j) {
            const double val = exp((i * i + j * j) * tmp) * scale;
            f[(i + hf) * fs + (j + hf)] = val;
            sum += val;
        }
    for (int i = 0; i < 81; ++i) f[i] /= sum;
    const long ow = w / 2, oh = h / 2;
#pragma omp parallel for
    for (long r = 0; r < oh; ++r) {
        for (long c = 0; c < ow; ++c) {
            double v = 0;
            int count = 0;
            for (int l = -hf; l <= hf; ++l)
                for (int k = -hf; k <= hf; ++k) {
                    if ((2 * r + l) >= 0 && (2 * c + k) >= 0 && (2 * r + l) < (long)h &&
                        (2 * c + k) < (long)w) {
                        v += f[(l + hf) * fs + (k + hf)] * src[(2 * r + l) * (long)w + (2 * c + k)];
                        count++;
                    }
                }
            out[r * ow + c] = (count == fs * fs) ? (uint16_t)v : src[(2 * r) * (long)w + (2 * c)];
        }
    }
}

/* ---- known-answer hooks ---------------------------------------------------- */
double vo_correlate(const double *L, const double *R, int N) { return correlate(L, R, N); }
int16_t vo_quantize_result(double v) { return q_result(v); }
int16_t vo_quantize_voxel(double v) { return q_voxel(v); }

/* Drives set_vec over the window loop of VerticalLineLocus (setsm_code.cpp:
 * 6429-6453) on a constant image, so every sample passes the positivity test
 * and the counts are those of the window geometry alone. */
void vo_window_counts(int half, int counts[3]) {
    const uint32_t n = (uint32_t)(4 * half + 8);
    uint16_t *img = (uint16_t *)malloc(sizeof(uint16_t) * n * n);
    for (uint32_t i = 0; i < n * n; ++i) img[i] = 100;
    patch_src s = {img, img, img, img, n, n, n, n};
    kernel_buf k;
    kbuf_init(&k, half);
    int cnt[3] = {0, 0, 0};
    const double c = 0.5 * n + 0.25;
    for (int row = -half; row <= half; row++)
        for (int col = -half; col <= half; col++) {
            const int r2 = row * row + col * col;
            if (r2 <= (half + 1) * (half + 1)) {
                pt2 p = {c + col, c + row};
                set_vec(&k, &s, row, col, p, p, r2, cnt);
            }
        }
    for (int w = 0; w < 3; ++w) counts[w] = cnt[w];
    kbuf_free(&k);
    free(img);
}

// vll_window.cuh -- FP32 window statistics of the split-precision path:
// shared-memory staging of texel pairs and the multi-window Pearson sums
// (ComputeMultiNCC + Correlate, SubFunctions.cpp:974-1018, :3328-3360, in
// FP32 with shifted sums).
#pragma once

#include "vll_device.cuh"

namespace vll {

// Ring of a window offset: 2 = innermost sub-window, 1 = middle, 0 = outer.
__host__ __device__ constexpr int ring_of(int H, int row, int col) {
    const int r2 = row * row + col * col;
    const int s1 = H / 2;
    const int s2 = s1 + (int)((s1 / 2.0) + 0.5);
    const bool w1 = r2 <= (H - s1 + 1) * (H - s1 + 1) && row >= -H + s1 && row <= H - s1 &&
                    col >= -H + s1 && col <= H - s1;
    const bool w2 = r2 <= (H - s2 + 1) * (H - s2 + 1) && row >= -H + s2 && row <= H - s2 &&
                    col >= -H + s2 && col <= H - s2;
    return w2 ? 2 : (w1 ? 1 : 0);
}

__host__ __device__ constexpr int ring_count(int H, int ring) {
    int n = 0;
    for (int row = -H; row <= H; ++row)
        for (int col = -H; col <= H; ++col)
            if (row * row + col * col <= (H + 1) * (H + 1) && ring_of(H, row, col) == ring) ++n;
    return n;
}

// floor and fraction of a small float with full-rate ALU ops only:
// round-to-nearest of (x - 0.5) through the 1.5*2^23 magic constant.
__device__ __forceinline__ int floor_frac(float x, float &frac) {
    const float t = __fadd_rn(__fadd_rn(x, -0.5f), 12582912.0f);
    const float r = __fadd_rn(t, -12582912.0f);
    frac = x - r;
    return __float_as_int(t) - 0x4B400000;
}

struct Acc {
    float sl, sr, sll, srr, slr;
};

// Pearson rho from shifted sums; returns -99 when a variance is below the
// reference's 1e-8 threshold and flags results whose variance is too small
// for FP32 to decide that threshold safely.
__device__ __forceinline__ float corr_from(const Acc &a, float n, bool &unsure) {
    const float inv = 1.0f / n;
    const float vl = a.sll - a.sl * a.sl * inv;
    const float vr = a.srr - a.sr * a.sr * inv;
    const float cv = a.slr - a.sl * a.sr * inv;
    // FP32 relative error of vl is ~n * 6e-8 * (sll / vl); treat anything
    // within a factor of the threshold, or heavily cancelled, as uncertain.
    if (vl < 1e-3f * a.sll + 1e-4f || vr < 1e-3f * a.srr + 1e-4f) unsure = true;
    if (!(vl > 1e-8f && vr > 1e-8f)) return -99.0f;
    return cv * rsqrtf(vl * vr);
}

struct WinCtx {
    float w00, w10, w01, w11;    // reference bilinear weights (same for all samples)
    float c, s;                  // target rotation cos(-theta), sin(-theta)
    float cI, cM, tcI, tcM;      // centring samples (window centre)
    int rbw, tbw;                // staged box widths (texel pairs)
};

// One window row of sub-window pattern |row| = AR at signed offset `row`:
// columns unrolled, each accumulating into its compile-time ring.
template <int H, int AR>
__device__ __forceinline__ void win_row(const WinCtx &x, int row, const float4 *__restrict__ qr,
                                        const float4 *__restrict__ qt, float tfx, float tfy,
                                        Acc (&acc)[3][2]) {
    const float4 *q0 = qr + (row + H) * x.rbw;
    const float4 *q1 = q0 + x.rbw;
    const float bx = fmaf(-x.s, (float)row, tfx);
    const float by = fmaf(x.c, (float)row, tfy);
#pragma unroll
    for (int col = -H; col <= H; ++col) {
        if (AR * AR + col * col > (H + 1) * (H + 1)) continue;
        const int ring = ring_of(H, AR, col);
        const float4 a = q0[col + H];
        const float4 b = q1[col + H];
        const float lI = fmaf(x.w11, b.z, fmaf(x.w01, b.x, fmaf(x.w10, a.z, x.w00 * a.x))) - x.cI;
        const float lM = fmaf(x.w11, b.w, fmaf(x.w01, b.y, fmaf(x.w10, a.w, x.w00 * a.y))) - x.cM;
        const float fx = fmaf(x.c, (float)col, bx);
        const float fy = fmaf(x.s, (float)col, by);
        float frx, fry;
        const int ix = floor_frac(fx, frx);
        const int iy = floor_frac(fy, fry);
        const float4 *t = qt + iy * x.tbw + ix;
        const float4 ta = t[0];
        const float4 tb = t[x.tbw];
        const float topI = fmaf(frx, ta.z - ta.x, ta.x);
        const float botI = fmaf(frx, tb.z - tb.x, tb.x);
        const float rI = fmaf(fry, botI - topI, topI) - x.tcI;
        const float topM = fmaf(frx, ta.w - ta.y, ta.y);
        const float botM = fmaf(frx, tb.w - tb.y, tb.y);
        const float rM = fmaf(fry, botM - topM, topM) - x.tcM;
        Acc &u = acc[ring][0];
        u.sl += lI;
        u.sr += rI;
        u.sll = fmaf(lI, lI, u.sll);
        u.srr = fmaf(rI, rI, u.srr);
        u.slr = fmaf(lI, rI, u.slr);
        Acc &v = acc[ring][1];
        v.sl += lM;
        v.sr += rM;
        v.sll = fmaf(lM, lM, v.sll);
        v.srr = fmaf(rM, rM, v.srr);
        v.slr = fmaf(lM, rM, v.slr);
    }
}

// Rows +AR and -AR share the pattern of |row| = AR (the sub-windows are
// symmetric), so each pattern's unrolled code serves two rows.
template <int H, int AR>
__device__ __forceinline__ void win_rows(const WinCtx &x, const float4 *__restrict__ qr,
                                         const float4 *__restrict__ qt, float tfx, float tfy,
                                         Acc (&acc)[3][2]) {
    if constexpr (AR <= H) {
#pragma unroll 1
        for (int sgn = (AR == 0 ? 1 : -1); sgn <= 1; sgn += 2)
            win_row<H, AR>(x, sgn * AR, qr, qt, tfx, tfy, acc);
        win_rows<H, AR + 1>(x, qr, qt, tfx, tfy, acc);
    }
}

// FP32 multi-window NCC of one slot (ComputeMultiNCC over the three nested
// sub-windows, intensity and magnitude, SubFunctions.cpp:3328-3360) from the
// staged texel pairs.  qr: top-left texel pair of the reference window;
// qt: target texel pair at the window centre; (rfx, rfy), (tfx, tfy): the
// fractional positions.  Sums are shifted by each window's centre sample.
template <int H>
__device__ __forceinline__ void window_fp32(const float4 *__restrict__ qr, int rbw, float rfx,
                                            float rfy, const float4 *__restrict__ qt, int tbw,
                                            float tfx, float tfy, float c, float s,
                                            float &incc_avg, bool &unsure) {
    Acc acc[3][2];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int p = 0; p < 2; ++p) acc[r][p] = Acc{0.f, 0.f, 0.f, 0.f, 0.f};
    WinCtx x;
    x.w00 = (1.f - rfx) * (1.f - rfy);
    x.w10 = rfx * (1.f - rfy);
    x.w01 = (1.f - rfx) * rfy;
    x.w11 = rfx * rfy;
    x.c = c;
    x.s = s;
    x.rbw = rbw;
    x.tbw = tbw;
    {
        const float4 a = qr[H * rbw + H];
        const float4 b = qr[(H + 1) * rbw + H];
        x.cI = fmaf(x.w11, b.z, fmaf(x.w01, b.x, fmaf(x.w10, a.z, x.w00 * a.x)));
        x.cM = fmaf(x.w11, b.w, fmaf(x.w01, b.y, fmaf(x.w10, a.w, x.w00 * a.y)));
        float frx, fry;
        const int ix = floor_frac(tfx, frx);
        const int iy = floor_frac(tfy, fry);
        const float4 *t = qt + iy * tbw + ix;
        const float4 ta = t[0];
        const float4 tb = t[tbw];
        const float topI = fmaf(frx, ta.z - ta.x, ta.x);
        const float botI = fmaf(frx, tb.z - tb.x, tb.x);
        x.tcI = fmaf(fry, botI - topI, topI);
        const float topM = fmaf(frx, ta.w - ta.y, ta.y);
        const float botM = fmaf(frx, tb.w - tb.y, tb.y);
        x.tcM = fmaf(fry, botM - topM, topM);
    }
    win_rows<H, 0>(x, qr, qt, tfx, tfy, acc);
    // nested windows: 2 = ring 2; 1 = rings 1+2; 0 = all rings
    constexpr int n2 = ring_count(H, 2);
    constexpr int n1 = n2 + ring_count(H, 1);
    constexpr int n0 = n1 + ring_count(H, 0);
    float tot = 0.f;
    int nv = 0;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        Acc w = acc[2][p];
        const float r2 = corr_from(w, (float)n2, unsure);
        w.sl += acc[1][p].sl;
        w.sr += acc[1][p].sr;
        w.sll += acc[1][p].sll;
        w.srr += acc[1][p].srr;
        w.slr += acc[1][p].slr;
        const float r1 = corr_from(w, (float)n1, unsure);
        w.sl += acc[0][p].sl;
        w.sr += acc[0][p].sr;
        w.sll += acc[0][p].sll;
        w.srr += acc[0][p].srr;
        w.slr += acc[0][p].slr;
        const float r0 = corr_from(w, (float)n0, unsure);
        if (r0 != -99.0f) { tot += r0; ++nv; }
        if (r1 != -99.0f) { tot += r1; ++nv; }
        if (r2 != -99.0f) { tot += r2; ++nv; }
    }
    // count_incc is 1 when any of the six correlations is defined
    incc_avg = nv > 0 ? tot / (float)nv : -1.0f;
    if (nv == 0) incc_avg = -2.0f;   // no valid correlation: count_incc stays 0
}

// Vectorised staging of the same box: each lane converts one 8-texel,
// 16-byte-aligned chunk of a box row per plane (two 128-bit loads) into up to
// eight texel pairs.  Requires the image rows to start on 16-byte boundaries
// (width multiple of 8 and 16-byte aligned planes); `dst` rows have stride
// `ds` pairs.  Returns (warp-uniform) whether an intensity texel is zero.
__device__ __forceinline__ bool stage_box_vec(float4 *__restrict__ dst, int ds,
                                              const uint16_t *__restrict__ I,
                                              const uint16_t *__restrict__ M, uint32_t W, int x0,
                                              int y0, int bw, int bh, float sI, float sM, int lane) {
    bool zero = false;
    const int xa = x0 & ~7;
    const int x1 = x0 + bw - 1;                 // last pair's left texel
    const int nch = ((x1 + 1) - xa) / 8 + 1;    // chunks covering [xa, x1 + 1]
    const int n = nch * bh;
    for (int i = lane; i < n; i += 32) {
        const int by = i / nch;
        const int c = i - by * nch;
        const int xc = xa + 8 * c;
        const int64_t row = (int64_t)(y0 + by) * W;
        const uint4 vi = __ldg(reinterpret_cast<const uint4 *>(I + row + xc));
        const uint4 vm = __ldg(reinterpret_cast<const uint4 *>(M + row + xc));
        const bool need9 = xc + 7 <= x1;        // the 8th pair needs texel xc + 8
        const uint16_t i8 = need9 ? __ldg(I + row + xc + 8) : (uint16_t)0;
        const uint16_t m8 = need9 ? __ldg(M + row + xc + 8) : (uint16_t)0;
        float fi[9], fm[9];
        const uint32_t wi[4] = {vi.x, vi.y, vi.z, vi.w};
        const uint32_t wm[4] = {vm.x, vm.y, vm.z, vm.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            fi[2 * q] = (float)(wi[q] & 0xFFFFu) - sI;
            fi[2 * q + 1] = (float)(wi[q] >> 16) - sI;
            fm[2 * q] = (float)(wm[q] & 0xFFFFu) - sM;
            fm[2 * q + 1] = (float)(wm[q] >> 16) - sM;
            zero |= (xc + 2 * q >= x0 && xc + 2 * q <= x1 + 1 && (wi[q] & 0xFFFFu) == 0);
            zero |= (xc + 2 * q + 1 >= x0 && xc + 2 * q + 1 <= x1 + 1 && (wi[q] >> 16) == 0);
        }
        fi[8] = (float)i8 - sI;
        fm[8] = (float)m8 - sM;
        zero |= need9 && i8 == 0;
        float4 *drow = dst + by * ds;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int x = xc + t;
            if (x >= x0 && x <= x1) drow[x - x0] = make_float4(fi[t], fm[t], fi[t + 1], fm[t + 1]);
        }
    }
    return __any_sync(0xffffffffu, zero);
}

// Scalar staging of a box whose destination rows have stride `ds` pairs
// (used when image rows are not 16-byte aligned).
__device__ __forceinline__ bool stage_box_strided(float4 *__restrict__ dst, int ds,
                                                  const uint16_t *__restrict__ I,
                                                  const uint16_t *__restrict__ M, uint32_t W, int x0,
                                                  int y0, int bw, int bh, float sI, float sM, int lane) {
    bool zero = false;
    const int n = bw * bh;
    for (int i = lane; i < n; i += 32) {
        const int by = i / bw;
        const int bx = i - by * bw;
        const int64_t p = (int64_t)(y0 + by) * W + (x0 + bx);
        const uint16_t a = __ldg(I + p), b = __ldg(I + p + 1);
        const uint16_t cm = __ldg(M + p), d = __ldg(M + p + 1);
        zero |= (a == 0) | (b == 0);
        dst[by * ds + bx] = make_float4((float)a - sI, (float)cm - sM, (float)b - sI, (float)d - sM);
    }
    return __any_sync(0xffffffffu, zero);
}

// Stages the texel pairs of box [x0, x0+bw) x [y0, y0+bh) of one image into
// shared memory as float4 {I(x)-sI, M(x)-sM, I(x+1)-sI, M(x+1)-sM}; returns
// true (warp-uniform) when some intensity texel in the box is zero.
__device__ __forceinline__ bool stage_box(float4 *__restrict__ dst, const uint16_t *__restrict__ I,
                                          const uint16_t *__restrict__ M, uint32_t W, int x0, int y0,
                                          int bw, int bh, float sI, float sM, int lane) {
    bool zero = false;
    const int n = bw * bh;
    // four texel pairs per lane in flight before any is converted, so the
    // global-load latency is paid once per batch instead of once per pair
    constexpr int U = 4;
    for (int base = lane; base < n; base += 32 * U) {
        uint16_t a[U], b[U], cm[U], d[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + 32 * u;
            if (i < n) {
                const int by = i / bw;
                const int bx = i - by * bw;
                const int64_t p = (int64_t)(y0 + by) * W + (x0 + bx);
                a[u] = __ldg(I + p);
                b[u] = __ldg(I + p + 1);
                cm[u] = __ldg(M + p);
                d[u] = __ldg(M + p + 1);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + 32 * u;
            if (i < n) {
                zero |= (a[u] == 0) | (b[u] == 0);
                dst[i] = make_float4((float)a[u] - sI, (float)cm[u] - sM, (float)b[u] - sI,
                                     (float)d[u] - sM);
            }
        }
    }
    return __any_sync(0xffffffffu, zero);
}

}  // namespace vll

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

// Packed (intensity, magnitude) arithmetic: sm_100 issues one FFMA2/FADD2
// for both planes of a sample.
__device__ __forceinline__ float2 lo2(const float4 &v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4 &v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
// b - a with a single rounding (fma with a -1 multiplier)
__device__ __forceinline__ float2 sub2(float2 b, float2 a) {
    return __ffma2_rn(a, make_float2(-1.f, -1.f), b);
}

constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23

// Window sums of one ring for both planes: .x intensity, .y magnitude.
struct Acc2 {
    float2 sl, sr, sll, srr, slr;
};

// The target box lives in the block's shared memory at byte offsets from
// `base`; `tq` is the offset of the window centre's texel, biased so that
// the fixed-point bits of the round-to-nearest constant index it directly:
// offset of texel (cx + dx, cy + dy) = tq + bits(M + dy) * row + bits(M + dx) * 16
// (mod 2^32), M = 1.5 * 2^23.
struct TgtBox {
    const unsigned char *base;   // shared-memory window of the block
    uint32_t tq;                 // biased offset (see above)
    uint32_t row;                // row stride in bytes
};

__device__ __forceinline__ TgtBox tgt_box(const unsigned char *base, uint32_t centre_off,
                                          uint32_t row) {
    return TgtBox{base, centre_off - 0x4B400000u * (row + 16u), row};
}

struct WinCtx {
    float2 w00, w10, w01, w11;   // reference bilinear weights (same for all samples), broadcast
    float2 ncl;                  // -(reference centre sample) per plane
    float2 ntc;                  // -(target centre sample) per plane
    float2 cs;                   // target rotation (cos(-theta), sin(-theta))
    float2 nsc;                  // (-sin(-theta), cos(-theta))
    int rbw;                     // reference box row stride (texel pairs)
    TgtBox tb;
};

// Reference-window sample from the staged pairs of rows y (a) and y+1 (b),
// plus `init` (the negated centre, or zero).
__device__ __forceinline__ float2 ref_sample(const WinCtx &x, const float4 &a, const float4 &b,
                                             float2 init) {
    float2 l = __ffma2_rn(x.w00, lo2(a), init);
    l = __ffma2_rn(x.w10, hi2(a), l);
    l = __ffma2_rn(x.w01, lo2(b), l);
    return __ffma2_rn(x.w11, hi2(b), l);
}

// Target sample at centre-relative position f (x, y): floor and fraction
// through the 1.5*2^23 round-to-nearest constant, then bilinear on both
// planes.  Target texels are staged as {I(x), M(x), I(x+1) - I(x),
// M(x+1) - M(x)} (the differences of integers are exact, so each row's
// interpolation rounds once, as I(x) + fx * (I(x+1) - I(x))).
__device__ __forceinline__ float2 tgt_sample(const TgtBox &tb, float2 f, float2 init) {
    const float2 t = __fadd2_rn(__fadd2_rn(f, make_float2(-0.5f, -0.5f)), bc2(kMagic));
    const float2 fr = __fadd2_rn(f, __ffma2_rn(t, make_float2(-1.f, -1.f), bc2(kMagic)));
    const uint32_t a = (uint32_t)__float_as_int(t.y) * tb.row +
                       ((uint32_t)__float_as_int(t.x) << 4) + tb.tq;
    const float4 ta = *reinterpret_cast<const float4 *>(tb.base + a);
    const float4 tv = *reinterpret_cast<const float4 *>(tb.base + a + tb.row);
    const float2 fx = bc2(fr.x), fy = bc2(fr.y);
    const float2 top = __ffma2_rn(fx, hi2(ta), lo2(ta));
    const float2 bot = __ffma2_rn(fx, hi2(tv), lo2(tv));
    return __fadd2_rn(__ffma2_rn(fy, sub2(bot, top), top), init);
}

// First window column of rows with |row| = AR (the circle r^2 <= (H+1)^2).
__host__ __device__ constexpr int row_cmin(int H, int AR) {
    int c = -H;
    while (AR * AR + c * c > (H + 1) * (H + 1)) ++c;
    return c;
}

// One window row of sub-window pattern |row| = AR at signed offset `row`:
// columns unrolled, each accumulating into its compile-time ring.
template <int H, int AR>
__device__ __forceinline__ void win_row(const WinCtx &x, int row, const float4 *__restrict__ qr,
                                        float2 tf, Acc2 (&acc)[3]) {
    const float4 *q0 = qr + (row + H) * x.rbw;
    const float4 *q1 = q0 + x.rbw;
    const float2 b = __ffma2_rn(x.nsc, bc2((float)row), tf);
    // Reference texel pairs {I(c), M(c), I(c+1), M(c+1)} are read only at even
    // offsets from the row's first column: a sample at an odd offset takes
    // its left texel from the previous pair's high half and its right texel
    // from the next pair's low half, so each pair feeds two samples.
    constexpr int c0 = row_cmin(H, AR);
    float4 a0 = q0[c0 + H], b0 = q1[c0 + H];   // pair at the last even offset
    float4 a1 = a0, b1 = b0;                   // pair at the next even offset
#pragma unroll
    for (int col = -H; col <= H; ++col) {
        if (AR * AR + col * col > (H + 1) * (H + 1)) continue;
        const int ring = ring_of(H, AR, col);
        float2 l;
        if (((col - c0) & 1) == 0) {
            if (col != c0) {
                a0 = a1;
                b0 = b1;
            }
            l = ref_sample(x, a0, b0, x.ncl);
        } else {
            a1 = q0[col + 1 + H];
            b1 = q1[col + 1 + H];
            l = ref_sample(x, make_float4(a0.z, a0.w, a1.x, a1.y),
                           make_float4(b0.z, b0.w, b1.x, b1.y), x.ncl);
        }
        const float2 r = tgt_sample(x.tb, __ffma2_rn(x.cs, bc2((float)col), b), x.ntc);
        Acc2 &u = acc[ring];
        u.sl = __fadd2_rn(u.sl, l);
        u.sr = __fadd2_rn(u.sr, r);
        u.sll = __ffma2_rn(l, l, u.sll);
        u.srr = __ffma2_rn(r, r, u.srr);
        u.slr = __ffma2_rn(l, r, u.slr);
    }
}

// Rows +AR and -AR share the pattern of |row| = AR (the sub-windows are
// symmetric), so each pattern's unrolled code serves two rows.
template <int H, int AR>
__device__ __forceinline__ void win_rows(const WinCtx &x, const float4 *__restrict__ qr,
                                         float2 tf, Acc2 (&acc)[3]) {
    if constexpr (AR <= H) {
#pragma unroll 1
        for (int sgn = (AR == 0 ? 1 : -1); sgn <= 1; sgn += 2)
            win_row<H, AR>(x, sgn * AR, qr, tf, acc);
        win_rows<H, AR + 1>(x, qr, tf, acc);
    }
}

__device__ __forceinline__ Acc plane(const Acc2 &a, int p) {
    return p == 0 ? Acc{a.sl.x, a.sr.x, a.sll.x, a.srr.x, a.slr.x}
                  : Acc{a.sl.y, a.sr.y, a.sll.y, a.srr.y, a.slr.y};
}

__device__ __forceinline__ void add_to(Acc2 &w, const Acc2 &a) {
    w.sl = __fadd2_rn(w.sl, a.sl);
    w.sr = __fadd2_rn(w.sr, a.sr);
    w.sll = __fadd2_rn(w.sll, a.sll);
    w.srr = __fadd2_rn(w.srr, a.srr);
    w.slr = __fadd2_rn(w.slr, a.slr);
}

// FP32 multi-window NCC of one slot (ComputeMultiNCC over the three nested
// sub-windows, intensity and magnitude, SubFunctions.cpp:3328-3360) from the
// staged texels.  qr: top-left texel pair of the reference window; tb: the
// target box addressed from the window centre's texel; (rfx, rfy), (tfx,
// tfy): the fractional positions.  Sums are shifted by each window's centre
// sample.
template <int H>
__device__ __forceinline__ void window_fp32(const float4 *__restrict__ qr, int rbw, float rfx,
                                            float rfy, const TgtBox &tb, float tfx, float tfy,
                                            float c, float s, float &incc_avg, bool &unsure) {
    Acc2 acc[3];
    const float2 z = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < 3; ++r) acc[r] = Acc2{z, z, z, z, z};
    WinCtx x;
    x.w00 = bc2((1.f - rfx) * (1.f - rfy));
    x.w10 = bc2(rfx * (1.f - rfy));
    x.w01 = bc2((1.f - rfx) * rfy);
    x.w11 = bc2(rfx * rfy);
    x.cs = make_float2(c, s);
    x.nsc = make_float2(-s, c);
    x.rbw = rbw;
    x.tb = tb;
    const float2 tf = make_float2(tfx, tfy);
    {
        const float2 cl = ref_sample(x, qr[H * rbw + H], qr[(H + 1) * rbw + H], z);
        const float2 ct = tgt_sample(tb, tf, z);
        x.ncl = make_float2(-cl.x, -cl.y);
        x.ntc = make_float2(-ct.x, -ct.y);
    }
    win_rows<H, 0>(x, qr, tf, acc);
    // nested windows: 2 = ring 2; 1 = rings 1+2; 0 = all rings
    constexpr int n2 = ring_count(H, 2);
    constexpr int n1 = n2 + ring_count(H, 1);
    constexpr int n0 = n1 + ring_count(H, 0);
    Acc2 w1 = acc[2];
    add_to(w1, acc[1]);
    Acc2 w0 = w1;
    add_to(w0, acc[0]);
    float tot = 0.f;
    int nv = 0;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const float r2 = corr_from(plane(acc[2], p), (float)n2, unsure);
        const float r1 = corr_from(plane(w1, p), (float)n1, unsure);
        const float r0 = corr_from(plane(w0, p), (float)n0, unsure);
        if (r0 != -99.0f) { tot += r0; ++nv; }
        if (r1 != -99.0f) { tot += r1; ++nv; }
        if (r2 != -99.0f) { tot += r2; ++nv; }
    }
    // count_incc is 1 when any of the six correlations is defined
    incc_avg = nv > 0 ? tot / (float)nv : -1.0f;
    if (nv == 0) incc_avg = -2.0f;   // no valid correlation: count_incc stays 0
}

// u16 texel pair (intensity word, magnitude word; low or high halves by
// `sel`) as floats minus the box shift: the texel is placed in the mantissa
// of 2^23 (exact), and `nshift` = -(2^23 + shift) removes both at once.
__device__ __forceinline__ float2 texel_pair(uint32_t wi, uint32_t wm, uint32_t sel, float2 nshift) {
    const float a = __int_as_float(__byte_perm(wi, 0x4B000000u, sel));
    const float b = __int_as_float(__byte_perm(wm, 0x4B000000u, sel));
    return __fadd2_rn(make_float2(a, b), nshift);
}

// Non-zero when some 16-bit half of w is zero.
__device__ __forceinline__ uint32_t zero_half(uint32_t w) { return (w - 0x00010001u) & ~w; }

// Staged texel of the box at x from the converted texels f[t] (x) and f[t+1]
// (x + 1): reference boxes hold pairs {I(x), M(x), I(x+1), M(x+1)}, target
// boxes (kDiff) {I(x), M(x), I(x+1) - I(x), M(x+1) - M(x)}.
template <bool kDiff>
__device__ __forceinline__ float4 box_texel(float2 a, float2 b) {
    if constexpr (kDiff) {
        const float2 d = sub2(b, a);
        return make_float4(a.x, a.y, d.x, d.y);
    } else {
        return make_float4(a.x, a.y, b.x, b.y);
    }
}

// Converts the nine texels of one 8-texel chunk (words vi/vm, ninth texel
// i8/m8) and stores the box texels of [xc, xc + 8) that lie in [x0, x1].
template <bool kDiff>
__device__ __forceinline__ void store_chunk(float4 *__restrict__ drow, const uint4 &vi,
                                            const uint4 &vm, uint32_t i8, uint32_t m8, int xc,
                                            int x0, int x1, float2 ns) {
    float2 f[9];
    f[0] = texel_pair(vi.x, vm.x, 0x7610, ns);
    f[1] = texel_pair(vi.x, vm.x, 0x7632, ns);
    f[2] = texel_pair(vi.y, vm.y, 0x7610, ns);
    f[3] = texel_pair(vi.y, vm.y, 0x7632, ns);
    f[4] = texel_pair(vi.z, vm.z, 0x7610, ns);
    f[5] = texel_pair(vi.z, vm.z, 0x7632, ns);
    f[6] = texel_pair(vi.w, vm.w, 0x7610, ns);
    f[7] = texel_pair(vi.w, vm.w, 0x7632, ns);
    f[8] = texel_pair(i8, m8, 0x7610, ns);
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int x = xc + t;
        if (x >= x0 && x <= x1) drow[x - x0] = box_texel<kDiff>(f[t], f[t + 1]);
    }
}

// Vectorised staging of the box by loads: each lane converts one 8-texel,
// 16-byte-aligned chunk of a box row per plane (two 128-bit loads) into up to
// eight box texels.  Requires the image rows to start on 16-byte boundaries
// (width multiple of 8 and 16-byte aligned planes); `dst` rows have stride
// `ds` texels.  Returns (warp-uniform) whether an intensity texel of the
// loaded chunks is zero (a superset of the box: the caller then takes the
// exact path).
template <bool kDiff>
__device__ __forceinline__ bool stage_box_vec(float4 *__restrict__ dst, int ds,
                                              const uint16_t *__restrict__ I,
                                              const uint16_t *__restrict__ M, uint32_t W, int x0,
                                              int y0, int bw, int bh, float sI, float sM, int lane) {
    uint32_t zacc = 0;
    bool z8 = false;
    const float2 ns = make_float2(-(8388608.0f + sI), -(8388608.0f + sM));
    const int xa = x0 & ~7;
    const int x1 = x0 + bw - 1;                 // last texel's left texel
    const int nch = ((x1 + 1) - xa) / 8 + 1;    // chunks covering [xa, x1 + 1]
    const int n = nch * bh;
    for (int i = lane; i < n; i += 32) {
        const int by = i / nch;
        const int c = i - by * nch;
        const int xc = xa + 8 * c;
        const int64_t row = (int64_t)(y0 + by) * W;
        const uint4 vi = __ldg(reinterpret_cast<const uint4 *>(I + row + xc));
        const uint4 vm = __ldg(reinterpret_cast<const uint4 *>(M + row + xc));
        const bool need9 = xc + 7 <= x1;        // the 8th texel needs texel xc + 8
        const uint32_t i8 = need9 ? __ldg(I + row + xc + 8) : 1u;
        const uint32_t m8 = need9 ? __ldg(M + row + xc + 8) : 0u;
        zacc |= zero_half(vi.x) | zero_half(vi.y) | zero_half(vi.z) | zero_half(vi.w);
        z8 |= i8 == 0;
        store_chunk<kDiff>(dst + by * ds, vi, vm, i8, m8, xc, x0, x1, ns);
    }
    return __any_sync(0xffffffffu, (zacc & 0x80008000u) != 0 || z8);
}

// Scalar staging of a box whose destination rows have stride `ds` texels
// (used when image rows are not 16-byte aligned).
template <bool kDiff>
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
        dst[by * ds + bx] = box_texel<kDiff>(make_float2((float)a - sI, (float)cm - sM),
                                             make_float2((float)b - sI, (float)d - sM));
    }
    return __any_sync(0xffffffffu, zero);
}

// ---- footprint staging by the tensor-memory-access (TMA) engine --------------
// Each group's footprints are copied raw (uint16) from global to shared
// memory as four 2-D tiles (intensity and magnitude of both images) that
// complete on the warp's mbarrier; the warp then converts them to box texels
// with 128-bit shared loads (convert_tile).

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also expects `bytes` of asynchronous copies.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

// Waits for phase `parity` of `bar` to complete, for at most ~`limit`
// cycles; returns false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// Orders this thread's earlier generic shared-memory accesses before later
// asynchronous-proxy (TMA) writes to the same memory.
__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 2-D tile of a tensor map (TMA, no multicast) into this CTA's shared memory
// at `dst` (128-byte aligned): x (innermost, a multiple of 16 bytes) and y
// are the tile's first texel; completes the tile's bytes on `bar`.
__device__ __forceinline__ void tma_tile_2d(void *dst, const void *tmap, int x, int y,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Makes a tensor map written to global memory by the host visible to the
// TMA unit before its first use by this thread.
__device__ __forceinline__ void tmap_acquire(const void *tmap) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
}

// Box texels of [x0, x0 + bw) x rows [0, bh) from the raw tiles in shared
// memory: rawI / rawM hold, per box row (stride `nb` bytes), the uint16
// texels from xa = x0 rounded down to 8 on.  Two adjacent box texels per
// lane and step (three loads per plane give both): each box texel's two
// texels of each plane become {v(x), v(x+1) + dm * v(x)}
// (dm = 0: reference pairs; dm = -1: target value and difference, exact for
// integers), each value placed in the mantissa of 2^23 and shifted by
// -(2^23 + shift) in one exact addition.  Zero intensity texels among the
// texels the box reads ([x0, x0 + bw] of each row) are listed in `zl` as
// tag | row << 16 | (x - x0), counted in *zn (entries beyond `cap` are
// counted, not stored).
__device__ __forceinline__ void convert_tile(float4 *__restrict__ dst, int ds,
                                             const unsigned char *__restrict__ rawI,
                                             const unsigned char *__restrict__ rawM, int nb,
                                             int xa, int x0, int bw, int bh, float sI, float sM,
                                             float dm, uint32_t *zl, int *zn, int cap,
                                             uint32_t tag, int lane) {
    const float2 ns = make_float2(-(8388608.0f + sI), -(8388608.0f + sM));
    const float2 dm2 = bc2(dm);
    const unsigned char *rI = rawI + 2 * (x0 - xa);
    const unsigned char *rM = rawM + 2 * (x0 - xa);
    // box texels (row by, columns bx = 2 bq and bx + 1): the lane's first
    // pair, then steps of 32 pairs
    const int bp = (bw + 1) >> 1;            // texel pairs per row
    const int n2 = bp * bh;
    // lane / bp and 32 / bp without an integer division: (n + 0.5) / bp lies
    // at least 0.5 / bp from an integer, far beyond the quotient's FP32 error
    const float rbp = __fdividef(1.f, (float)bp);
    int by = (int)(((float)lane + 0.5f) * rbp), bq = lane - by * bp;
    const int dby = (int)(32.5f * rbp), dbq = 32 - dby * bp;
    for (int q = lane; q < n2; q += 32) {
        const int bx = 2 * bq;
        const bool two = bx + 1 < bw;
        const int ro = by * nb + 2 * bx;
        const uint32_t i0 = *reinterpret_cast<const uint16_t *>(rI + ro);
        const uint32_t i1 = *reinterpret_cast<const uint16_t *>(rI + ro + 2);
        const uint32_t m0 = *reinterpret_cast<const uint16_t *>(rM + ro);
        const uint32_t m1 = *reinterpret_cast<const uint16_t *>(rM + ro + 2);
        const uint32_t i2 = two ? *reinterpret_cast<const uint16_t *>(rI + ro + 4) : 1u;
        const uint32_t m2 = two ? *reinterpret_cast<const uint16_t *>(rM + ro + 4) : 0u;
        // zero texels among those the box reads ([0, bw] of the row): this
        // lane lists texels bx and bx + 1, and texel bx + 2 when it ends the
        // row (otherwise the next pair lists it)
        const bool end2 = two && bx + 2 == bw;
        if (i0 == 0 || i1 == 0 || (end2 && i2 == 0)) {
            const uint32_t t3[3] = {i0, i1, i2};
#pragma unroll
            for (int t = 0; t < 3; ++t)
                if (t3[t] == 0 && (t < 2 || end2)) {
                    const int k = atomicAdd(zn, 1);
                    if (k < cap) zl[k] = tag | ((uint32_t)by << 16) | (uint32_t)(bx + t);
                }
        }
        const float2 a = __fadd2_rn(make_float2(__int_as_float(i0 | 0x4B000000u),
                                                __int_as_float(m0 | 0x4B000000u)), ns);
        const float2 b = __fadd2_rn(make_float2(__int_as_float(i1 | 0x4B000000u),
                                                __int_as_float(m1 | 0x4B000000u)), ns);
        float4 *d = dst + by * ds + bx;
        const float2 h0 = __ffma2_rn(dm2, a, b);
        d[0] = make_float4(a.x, a.y, h0.x, h0.y);
        if (two) {
            const float2 c = __fadd2_rn(make_float2(__int_as_float(i2 | 0x4B000000u),
                                                    __int_as_float(m2 | 0x4B000000u)), ns);
            const float2 h1 = __ffma2_rn(dm2, b, c);
            d[1] = make_float4(b.x, b.y, h1.x, h1.y);
        }
        bq += dbq;
        by += dby;
        if (bq >= bp) {
            bq -= bp;
            ++by;
        }
    }
}

}  // namespace vll

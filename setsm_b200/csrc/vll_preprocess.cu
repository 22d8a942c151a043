// vll_preprocess.cu -- image preprocessing on the device, bit-exact with
// SETSM's L2 functions (SubFunctions.cpp:2418-2560, Template.hpp:45-131):
// Sobel magnitude, 18-bin gradient orientation, 9x9 Gaussian 2x pyramid.
// These are stencils bound by HBM bandwidth; one thread per output pixel.
// Compiled with -fmad=false; FP64 accumulations keep the reference's order.
#include <cstdint>
#include <cuda_runtime.h>

#include "vll_internal.h"

namespace vll {

constexpr double kPiPre = 3.141592653589793;

// MakeSobelMagnitudeImage, SubFunctions.cpp:2418-2471.  Instead of the int16
// degree image the kernel stores what Orientation consumes from it: the
// 20-degree bin of floor(atan2(gy, gx) * 180 / PI) after the [0, 360) wrap.
__global__ void __launch_bounds__(256) sobel_kernel(const uint16_t *__restrict__ s, uint32_t w,
                                                    uint32_t h, uint16_t *__restrict__ mag,
                                                    uint8_t *__restrict__ bin) {
    const int64_t n = (int64_t)w * h;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = p / w, j = p % w;
        if (j == 0 || j == (int64_t)w - 1 || i == 0 || i == (int64_t)h - 1) {
            mag[p] = 0;
            bin[p] = 0;   // dir 0 -> theta 0 -> bin 0
            continue;
        }
        const int a = s[p - w - 1], b = s[p - w], c = s[p - w + 1];
        const int d = s[p - 1], f = s[p + 1];
        const int g = s[p + w - 1], hh = s[p + w], k = s[p + w + 1];
        const double gx = (double)(-a + c - 2 * d + 2 * f - g + k);
        const double gy = (double)(a + 2 * b + c - g - 2 * hh - k);
        const double m = sqrt(__dadd_rn(__dmul_rn(gx, gx), __dmul_rn(gy, gy)));
        const int16_t dir = (int16_t)floor(__ddiv_rn(__dmul_rn(atan2(gy, gx), 180.0), kPiPre));
        double theta = (double)dir;
        if (theta < 0)
            theta += 360;
        else if (theta > 360)
            theta -= 360;
        const long idx = (long)__ddiv_rn(theta, 20.0);
        bin[p] = (idx >= 0 && idx < 18) ? (uint8_t)idx : (uint8_t)255;
        mag[p] = (uint16_t)__dadd_rn(m, 0.5);
    }
}

// Orientation, SubFunctions.cpp:2473-2560: Gaussian-weighted 18-bin histogram
// of gradient magnitude over a 13x13 disc-like window, coarse 4-way sub-bin
// vote, then the best bin inside the winning sub-bin.  The window bounds
// reproduce the reference exactly, including its column lower bound
// max(-mask_row, -numcols[|row|]); addresses before the first pixel add 0.
__global__ void __launch_bounds__(128) orientation_kernel(const uint16_t *__restrict__ mag,
                                                          const uint8_t *__restrict__ bin_img,
                                                          uint32_t w, uint32_t h, int half,
                                                          const double *__restrict__ wt,
                                                          uint8_t *__restrict__ ori) {
    const int numcols[7] = {6, 5, 5, 5, 4, 3, 0};
    const int64_t W = w, Hh = h;
    const int sz = 2 * half - 1;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < W * Hh;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mr = p / W, mc = p % W;
        double bins[18];
#pragma unroll
        for (int i = 0; i < 18; ++i) bins[i] = 0.0;
        double sub[4] = {0.0, 0.0, 0.0, 0.0};
        const int64_t r_lo = (-mr > -half + 1) ? -mr : -half + 1;
        const int64_t r_hi = (Hh - mr - 1 < half - 1) ? Hh - mr - 1 : half - 1;
        for (int64_t r = r_lo; r <= r_hi; ++r) {
            const int ar = (int)(r < 0 ? -r : r);
            const int dcol = ar < 7 ? numcols[ar] : 0;
            const int64_t c_lo = (-mr > -dcol) ? -mr : -dcol;
            const int64_t c_hi = (dcol < W - mc - 1) ? dcol : W - mc - 1;
            for (int64_t c = c_lo; c <= c_hi; ++c) {
                const int64_t idx = (mr + r) * W + (mc + c);
                if (idx < 0) continue;
                const uint8_t bi = bin_img[idx];
                if (bi >= 18) continue;
                const double gw = wt[(half - 1 + r) * sz + (half - 1 + c)];
                const double v = __dmul_rn((double)mag[idx], gw);
                bins[bi] = __dadd_rn(bins[bi], v);
                const int sb = (int)__ddiv_rn((double)bi, 4.6);
                sub[sb] = __dadd_rn(sub[sb], v);
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
        const int lo = (int)__dmul_rn((double)sub_th, 4.6);
        const int hi = (int)__dadd_rn(__dmul_rn((double)sub_th, 4.6), 4.6);
        for (int i = lo; i < hi; ++i)
            if (bins[i] > mx) {
                mx = bins[i];
                th = i;
            }
        ori[p] = (uint8_t)th;
    }
}

// CreateImagePyramid<uint16>(.., 9, 1.5), Template.hpp:82-131.
__global__ void __launch_bounds__(256) pyramid_kernel(const uint16_t *__restrict__ src, uint32_t w,
                                                      uint32_t h, const double *__restrict__ f,
                                                      uint16_t *__restrict__ out) {
    const int64_t ow = w / 2, oh = h / 2;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < ow * oh;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = p / ow, c = p % ow;
        double v = 0;
        int count = 0;
        for (int l = -4; l <= 4; ++l)
            for (int k = -4; k <= 4; ++k) {
                const int64_t y = 2 * r + l, x = 2 * c + k;
                if (y >= 0 && x >= 0 && y < (int64_t)h && x < (int64_t)w) {
                    v = __dadd_rn(v, __dmul_rn(f[(l + 4) * 9 + (k + 4)], (double)src[y * w + x]));
                    count++;
                }
            }
        out[p] = (count == 81) ? (uint16_t)v : src[(2 * r) * (int64_t)w + 2 * c];
    }
}

static unsigned grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

cudaError_t launch_sobel(const uint16_t *src, uint32_t w, uint32_t h, uint16_t *mag, uint8_t *bin,
                         cudaStream_t s) {
    sobel_kernel<<<grid_for((int64_t)w * h, 256), 256, 0, s>>>(src, w, h, mag, bin);
    return cudaGetLastError();
}

cudaError_t launch_orientation(const uint16_t *mag, const uint8_t *bin, uint32_t w, uint32_t h,
                               int half, const double *wt, uint8_t *ori, cudaStream_t s) {
    orientation_kernel<<<grid_for((int64_t)w * h, 128), 128, 0, s>>>(mag, bin, w, h, half, wt, ori);
    return cudaGetLastError();
}

cudaError_t launch_pyramid(const uint16_t *src, uint32_t w, uint32_t h, const double *f,
                           uint16_t *out, cudaStream_t s) {
    pyramid_kernel<<<grid_for((int64_t)(w / 2) * (h / 2), 256), 256, 0, s>>>(src, w, h, f, out);
    return cudaGetLastError();
}

}  // namespace vll

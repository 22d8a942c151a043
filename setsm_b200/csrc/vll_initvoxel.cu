// vll_initvoxel.cu -- InitializeVoxel (setsm_code.cpp:5759-6012) on the GPU:
// each node's search range for the voxel route and its voxel row.
//
// Per node, independently: the image-boundary test at the UGRID range, the
// blunder-cell rules of the level and iteration, the range carried over or
// extended from the previous iteration's NCCresult (check_height_change), and
// the number of height voxels.  Rows whose range changed are (re)initialised
// (flag_cal = 1, INCC = -1000 quantised); the others keep their previous
// iteration's voxels.  The voxel rows are packed in node order by
// NumOfHeight, the layout of vll_vertical_line_locus[_device]: two exclusive
// scans (the old and the new row lengths) place every row, and one pass
// writes or carries them over.
#include <cstdint>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "vll_device.cuh"
#include "vll_internal.h"

namespace vll {

namespace {

__global__ void init_voxel_kernel(const DevLevel *__restrict__ Pp, const vll_ugrid *gp3,
                                  const vll_nccresult *ncc, vll_ugrid *gout, vll_nccresult *nout,
                                  int64_t *new_n, int64_t *old_n, uint8_t *fresh) {
    const DevLevel &P = *Pp;
    const int L = P.L, it = P.iteration;
    const double hs = P.height_step;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < P.n_nodes;
         t += (int64_t)gridDim.x * blockDim.x) {
        vll_ugrid g = gp3[t];
        vll_nccresult r = ncc[t];
        old_n[t] = r.NumOfHeight;
        uint8_t f = 0;
        const double lon = P.grid_wgs[2 * t], lat = P.grid_wgs[2 * t + 1];
        if (check_image_boundary(P, lon, lat, (double)g.minHeight, (double)g.maxHeight, 7)) {
            int csmin = 0, csmax = 0;
            bool blunder = true;
            const double th_height = P.dem_res <= 4 ? 500 : 1000;
            if (P.check_matchtag || it == 1) {
                r.minHeight = g.minHeight;
                r.maxHeight = g.maxHeight;
                r.GNCC = q_result(-1.0);
                r.check_height_change = 1;
                blunder = false;
            } else if (L >= 2) {
                blunder = false;
            } else if (g.Matched_flag != 0) {
                if (g.maxHeight - g.minHeight > 0) {
                    if (L <= 1) {
                        if (it > 1)
                            blunder = !(g.maxHeight <= P.minmax[1] && g.minHeight >= P.minmax[0] &&
                                        r.maxHeight <= P.minmax[1] && r.minHeight >= P.minmax[0]);
                        else
                            blunder = !(g.maxHeight <= P.minmax[1] && g.minHeight >= P.minmax[0]);
                    }
                    if (L == 1) blunder = !(abs(g.maxHeight - g.minHeight) < 1000);
                    if (L == 0) {
                        if (it > 1)
                            blunder = !((abs(r.maxHeight - r.minHeight) < th_height) &&
                                        (abs(g.maxHeight - g.minHeight) < th_height));
                        else if (abs(g.maxHeight - g.minHeight) < th_height)
                            blunder = false;
                        else
                            r.NumOfHeight = 0;
                    }
                } else {
                    r.NumOfHeight = 0;
                    blunder = true;
                }
            } else {
                r.NumOfHeight = 0;
                blunder = true;
            }
            if (!blunder) {
                if (it == 1 || (L == 0 && P.dem_res < 2)) {
                    r.minHeight = g.minHeight;
                    r.maxHeight = g.maxHeight;
                    r.GNCC = q_result(-1.0);
                    r.check_height_change = 1;
                    if (L == 1) {
                        if (abs((int)g.maxHeight - (int)g.minHeight) > 1000) {
                            g.maxHeight = -100;
                            g.minHeight = -100;
                            r.check_height_change = 0;
                        }
                    } else if (L == 0) {
                        if (abs((int)g.maxHeight - (int)g.minHeight) > th_height) {
                            g.maxHeight = -100;
                            g.minHeight = -100;
                            r.check_height_change = 0;
                        }
                    }
                } else {
                    const int nv = (int)__ddiv_rn((double)(g.maxHeight - g.minHeight), hs);
                    if (r.NumOfHeight == 0 && nv > 0) {
                        csmin = 0;
                        csmax = 0;
                        r.check_height_change = 1;
                    } else if (r.minHeight > g.minHeight || r.maxHeight < g.maxHeight) {
                        if (r.minHeight > g.minHeight)
                            csmin = (int)__dadd_rn(__ddiv_rn((double)(r.minHeight - g.minHeight), hs),
                                                   0.5);
                        if (r.maxHeight < g.maxHeight)
                            csmax = (int)__dadd_rn(__ddiv_rn((double)(g.maxHeight - r.maxHeight), hs),
                                                   0.5);
                        r.minHeight = to_short(
                            floor(__dadd_rn((double)r.minHeight, -__dmul_rn((double)csmin, hs))));
                        r.maxHeight = to_short(
                            ceil(__dadd_rn((double)r.maxHeight, __dmul_rn((double)csmax, hs))));
                        r.check_height_change = 1;
                        if (L == 0 && abs(r.maxHeight - r.minHeight) > th_height)
                            r.check_height_change = 0;
                    } else {
                        r.check_height_change = 0;
                    }
                }
                if (r.check_height_change) {
                    r.minHeight = to_short(
                        floor(__dadd_rn((double)r.minHeight, -__dmul_rn((double)csmin, hs))));
                    r.maxHeight = to_short(
                        ceil(__dadd_rn((double)r.maxHeight, __dmul_rn((double)csmax, hs))));
                    const int nv =
                        (int)__ddiv_rn((double)(float)(r.maxHeight - r.minHeight), hs);
                    if (nv > 0) {
                        r.NumOfHeight = (uint16_t)nv;
                        f = 1;
                    } else {
                        r.NumOfHeight = 0;
                        r.check_height_change = 0;
                    }
                }
            } else {
                r.NumOfHeight = 0;
                r.check_height_change = 0;
            }
        } else {
            r.NumOfHeight = 0;
            r.check_height_change = 0;
        }
        if (r.minHeight == 0 || r.maxHeight == 0) {
            r.NumOfHeight = 0;
            r.check_height_change = 0;
        }
        if (L == 0 && r.NumOfHeight > 1000) {
            r.NumOfHeight = 0;
            r.check_height_change = 0;
        }
        gout[t] = g;
        nout[t] = r;
        new_n[t] = r.NumOfHeight;
        fresh[t] = f;
    }
}

// Writes the new packed rows: fresh rows initialised, kept rows copied from
// the previous packing (one warp per node, lanes over its heights).
__global__ void pack_voxel_kernel(int64_t n_nodes, const int64_t *new_n, const int64_t *new_off,
                                  const int64_t *old_n, const int64_t *old_off,
                                  const uint8_t *fresh, const vll_voxel *vin, vll_voxel *vout) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    vll_voxel init;
    init.flag_cal = 1;
    init.INCC = q_voxel(-1.0);
    for (int64_t t = warp; t < n_nodes; t += n_warps) {
        const int64_t n = new_n[t], o = new_off[t];
        const bool reinit = fresh[t] || vin == nullptr;
        for (int64_t h = lane; h < n; h += 32) {
            if (reinit || h >= old_n[t])
                vout[o + h] = init;
            else
                vout[o + h] = vin[old_off[t] + h];
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

size_t init_voxel_scratch(int64_t n) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int64_t *)nullptr, (int64_t *)nullptr,
                                  (int)n);
    return al(tmp) + 3 * al(n * 8) + al((n + 1) * 8) + al(n) + al(n * sizeof(vll_ugrid)) +
           al(n * sizeof(vll_nccresult));
}

// Phase 1: the per-node decisions (into scratch copies of the UGRID and
// NCCresult records) and the offsets.  new_off (n + 1 entries, device)
// receives the new packing; *total the new voxel count and *old_total the
// count the old packing holds.  gp3 / ncc are not written (run_commit_voxel).
cudaError_t run_init_voxel(const DevLevel *dP, int64_t n, vll_ugrid *gp3, vll_nccresult *ncc,
                           void *scratch, int64_t *new_off, int64_t *total, int64_t *old_total,
                           cudaStream_t s) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int64_t *)nullptr, (int64_t *)nullptr,
                                  (int)n);
    char *p = (char *)scratch;
    void *tmp_p = p;
    p += al(tmp);
    int64_t *new_n = (int64_t *)p;
    p += al(n * 8);
    int64_t *old_n = (int64_t *)p;
    p += al(n * 8);
    int64_t *old_off = (int64_t *)p;
    p += al(n * 8);
    p += al((n + 1) * 8);   // spare
    uint8_t *fresh = (uint8_t *)p;
    p += al(n);
    vll_ugrid *gout = (vll_ugrid *)p;
    p += al(n * sizeof(vll_ugrid));
    vll_nccresult *nout = (vll_nccresult *)p;
    cudaError_t e;
    init_voxel_kernel<<<blocks_for(n, 128), 128, 0, s>>>(dP, gp3, ncc, gout, nout, new_n, old_n,
                                                         fresh);
    if ((e = cudaGetLastError())) return e;
    if ((e = cub::DeviceScan::ExclusiveSum(tmp_p, tmp, new_n, new_off, (int)n, s))) return e;
    if ((e = cub::DeviceScan::ExclusiveSum(tmp_p, tmp, old_n, old_off, (int)n, s))) return e;
    int64_t h[4];
    if ((e = cudaMemcpyAsync(h, new_off + n - 1, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(h + 1, new_n + n - 1, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(h + 2, old_off + n - 1, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(h + 3, old_n + n - 1, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    *total = h[0] + h[1];
    *old_total = h[2] + h[3];
    return cudaMemcpyAsync(new_off + n, total, 8, cudaMemcpyHostToDevice, s);
}

// Phase 2a: the decided records back into gp3 / ncc.
cudaError_t run_commit_voxel(int64_t n, void *scratch, vll_ugrid *gp3, vll_nccresult *ncc,
                             cudaStream_t s) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int64_t *)nullptr, (int64_t *)nullptr,
                                  (int)n);
    const char *p = (const char *)scratch + al(tmp) + 3 * al(n * 8) + al((n + 1) * 8) + al(n);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(gp3, p, n * sizeof(vll_ugrid), cudaMemcpyDeviceToDevice, s)))
        return e;
    p += al(n * sizeof(vll_ugrid));
    return cudaMemcpyAsync(ncc, p, n * sizeof(vll_nccresult), cudaMemcpyDeviceToDevice, s);
}

// Phase 2b: the packed rows (vin packed by the old lengths, or nullptr).
cudaError_t run_pack_voxel(int64_t n, const int64_t *new_off, void *scratch, const vll_voxel *vin,
                           vll_voxel *vout, cudaStream_t s) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const int64_t *)nullptr, (int64_t *)nullptr,
                                  (int)n);
    char *p = (char *)scratch + al(tmp);
    const int64_t *new_n = (const int64_t *)p;
    p += al(n * 8);
    const int64_t *old_n = (const int64_t *)p;
    p += al(n * 8);
    const int64_t *old_off = (const int64_t *)p;
    p += al(n * 8);
    p += al((n + 1) * 8);
    const uint8_t *fresh = (const uint8_t *)p;
    pack_voxel_kernel<<<blocks_for(n * 32, 256), 256, 0, s>>>(n, new_n, new_off, old_n, old_off,
                                                              fresh, vin, vout);
    return cudaGetLastError();
}

}  // namespace vll

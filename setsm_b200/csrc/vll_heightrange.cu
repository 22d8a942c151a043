// vll_heightrange.cu -- SetHeightRange (setsm_code.cpp:9851-10255): the
// next iteration's per-node height ranges from the TIN of matched points.
//
// Every grid node inside a triangle takes its height from the triangle's
// plane (IsTinInside, SubFunctions.cpp:2946-2995; at levels 0-1 the vertex
// height where the node coincides with a vertex) and a range from the
// triangle's height extent widened by a buffer that depends on the level,
// the iteration, the triangle's slope (SetNormalAngle, :2997-3012) and the
// node's orthoimage NCC; nodes in no triangle take the union of their matched
// neighbours' ranges.  The reference walks the triangles in order and a node
// is set by the first triangle that contains it; here one warp per triangle
// marks, per node, the smallest containing triangle index (atomicMin), and a
// pass over the nodes then applies that triangle's update -- the same result.
#include <cstdint>
#include <cuda_runtime.h>

#include "vll_ddmath.cuh"
#include "vll_device.cuh"
#include "vll_internal.h"

namespace vll {

namespace {

struct Tri3 {
    double x[3], y[3], z[3];
};

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

// Order-preserving 64-bit key of a double (for atomic min / max).
__device__ __forceinline__ unsigned long long dkey(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ Tri3 tri_of(const vll_point3 *pts, const vll_tri &t) {
    Tri3 r;
    const uint32_t v[3] = {t.a, t.b, t.c};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r.x[k] = pts[v[k]].x;
        r.y[k] = pts[v[k]].y;
        r.z[k] = pts[v[k]].z;
    }
    return r;
}

// IsTinInside (SubFunctions.cpp:2946-2995): the edge tests and the plane
// height (float) at (cx, cy).
__device__ bool tin_inside(const Tri3 &T, double cx, double cy, float &z) {
    int sum = 3;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int n = (k + 1) % 3;
        const double ex = __dadd_rn(T.x[n], -T.x[k]), ey = __dadd_rn(T.y[n], -T.y[k]);
        const double px = __dadd_rn(cx, -T.x[k]), py = __dadd_rn(cy, -T.y[k]);
        if (__dadd_rn(__dmul_rn(ex, py), -__dmul_rn(ey, px)) <= 0) --sum;
    }
    if (!(sum == 0 || sum == 3)) return false;
    const double v12x = __dadd_rn(T.x[1], -T.x[0]), v12y = __dadd_rn(T.y[1], -T.y[0]),
                 v12z = __dadd_rn(T.z[1], -T.z[0]);
    const double v13x = __dadd_rn(T.x[2], -T.x[0]), v13y = __dadd_rn(T.y[2], -T.y[0]),
                 v13z = __dadd_rn(T.z[2], -T.z[0]);
    double nx = __dadd_rn(__dmul_rn(v12y, v13z), -__dmul_rn(v12z, v13y));
    double ny = __dadd_rn(__dmul_rn(v12z, v13x), -__dmul_rn(v12x, v13z));
    double nz = __dadd_rn(__dmul_rn(v12x, v13y), -__dmul_rn(v12y, v13x));
    const double len =
        sqrt(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)), __dmul_rn(nz, nz)));
    if (!(len > 0)) return false;
    nx = __ddiv_rn(nx, len);
    ny = __ddiv_rn(ny, len);
    nz = __ddiv_rn(nz, len);
    const double d = -__dadd_rn(__dadd_rn(__dmul_rn(nx, T.x[0]), __dmul_rn(ny, T.y[0])),
                                __dmul_rn(nz, T.z[0]));
    if (nz == 0) return false;
    z = (float)__ddiv_rn(-__dadd_rn(__dadd_rn(__dmul_rn(nx, cx), __dmul_rn(ny, cy)), d), nz);
    return true;
}

// SetNormalAngle + SetAngle (SubFunctions.cpp:2997-3022), in degrees.
__device__ double normal_angle(const Tri3 &T) {
    const double ux = __dadd_rn(T.x[1], -T.x[0]), uy = __dadd_rn(T.y[1], -T.y[0]),
                 uz = __dadd_rn(T.z[1], -T.z[0]);
    const double vx = __dadd_rn(T.x[2], -T.x[0]), vy = __dadd_rn(T.y[2], -T.y[0]),
                 vz = __dadd_rn(T.z[2], -T.z[0]);
    const double nx = __dadd_rn(__dmul_rn(uy, vz), -__dmul_rn(vy, uz));
    const double ny = -__dadd_rn(__dmul_rn(ux, vz), -__dmul_rn(vx, uz));
    const double nz = __dadd_rn(__dmul_rn(ux, vy), -__dmul_rn(vx, uy));
    const double norm =
        sqrt(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)), __dmul_rn(nz, nz)));
    // norm == 0 leaves the reference's angle unset; such a triangle contains
    // no node (its plane has no normal), so the value is never used
    double angle = 0;
    if (norm != 0)
        angle = __ddiv_rn(__dmul_rn(ddm::acos_cr(__ddiv_rn(fabs(nz), norm)), 180.0), kPi);
    if (angle <= 0 && angle >= -90)
        angle = fabs(angle);
    else if (angle <= -270 && angle >= -360)
        angle = __dadd_rn(360.0, angle);
    else if (angle >= 270 && angle <= 360)
        angle = __dadd_rn(360.0, -angle);
    return angle;
}

struct BBox {
    int x0, y0, x1, y1;
};

// SetTinBoundary's pixel box (SubFunctions.cpp:2915-2944).
__device__ BBox tin_box(const DevLevel &P, const Tri3 &T) {
    const double gs = P.grid_res;
    const double mnx = dmin(dmin(T.x[0], T.x[1]), T.x[2]), mny = dmin(dmin(T.y[0], T.y[1]), T.y[2]);
    const double mxx = dmax(dmax(T.x[0], T.x[1]), T.x[2]), mxy = dmax(dmax(T.y[0], T.y[1]), T.y[2]);
    BBox b;
    b.x0 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mnx, -P.boundary[0]), gs), 0.5) - 1;
    b.y0 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mny, -P.boundary[1]), gs), 0.5) - 1;
    b.x1 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mxx, -P.boundary[0]), gs), 0.5) + 1;
    b.y1 = (int)__dadd_rn(__ddiv_rn(__dadd_rn(mxy, -P.boundary[1]), gs), 0.5) + 1;
    if (b.x1 >= (int)P.grid_w) b.x1 = (int)P.grid_w - 1;
    if (b.y1 >= (int)P.grid_h) b.y1 = (int)P.grid_h - 1;
    if (b.x0 < 0) b.x0 = 0;
    if (b.y0 < 0) b.y0 = 0;
    return b;
}

__device__ __forceinline__ double node_x(const DevLevel &P, int64_t col) {
    return __dadd_rn(__dmul_rn((double)col, P.grid_res), P.boundary[0]);
}
__device__ __forceinline__ double node_y(const DevLevel &P, int64_t row) {
    return __dadd_rn(__dmul_rn((double)row, P.grid_res), P.boundary[1]);
}

// Per triangle (one warp): the running extent of the vertex heights and,
// per node of its box inside it, the smallest containing triangle index.
__global__ void __launch_bounds__(128) cover_kernel(const DevLevel *__restrict__ Pp,
                                                    const vll_point3 *pts, int64_t n_pts,
                                                    const vll_tri *tris, int64_t n_tris,
                                                    unsigned int *winner,
                                                    unsigned long long *zext) {
    const DevLevel &P = *Pp;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = warp; t < n_tris; t += n_warps) {
        const vll_tri tr = tris[t];
        if (!(tr.a < n_pts && tr.b < n_pts && tr.c < n_pts)) continue;
        const Tri3 T = tri_of(pts, tr);
        if (lane == 0) {
            atomicMin(zext, dkey(dmin(dmin(T.z[0], T.z[1]), T.z[2])));
            atomicMax(zext + 1, dkey(dmax(dmax(T.z[0], T.z[1]), T.z[2])));
        }
        const BBox b = tin_box(P, T);
        if (b.x1 < b.x0 || b.y1 < b.y0) continue;
        const int64_t ncol = b.x1 - b.x0 + 1;
        const int64_t ncell = ncol * (b.y1 - b.y0 + 1);
        for (int64_t i = lane; i < ncell; i += 32) {
            const int64_t row = b.y0 + i / ncol, col = b.x0 + i % ncol;
            float z;
            if (tin_inside(T, node_x(P, col), node_y(P, row), z))
                atomicMin(winner + row * P.grid_w + col, (unsigned int)t);
        }
    }
}

struct RangeArgs {
    double buffer;      // BufferOfHeight
    double th_hg;
    int iteration;
};

// The first containing triangle's update of each node (setsm_code.cpp:
// 9968-10076).  newh: the node's new Height (-1000 when none), mb: m_bHeight.
__global__ void node_update_kernel(const DevLevel *__restrict__ Pp, const vll_point3 *pts,
                                   const vll_tri *tris, const unsigned int *winner, vll_ugrid *gp3,
                                   float *newh, uint8_t *mb, RangeArgs a) {
    const DevLevel &P = *Pp;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < P.n_nodes;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const unsigned int w = winner[idx];
        if (w == 0xffffffffu) {
            newh[idx] = -1000.0f;
            mb[idx] = 0;
            continue;
        }
        const Tri3 T = tri_of(pts, tris[w]);
        const int64_t row = idx / P.grid_w, col = idx % P.grid_w;
        const double cx = node_x(P, col), cy = node_y(P, row);
        float z = -1000.0f;
        tin_inside(T, cx, cy, z);
        const double tmin = dmin(dmin(T.z[0], T.z[1]), T.z[2]);
        const double tmax = dmax(dmax(T.z[0], T.z[1]), T.z[2]);
        double bf;
        if (P.L >= 3) {
            const double angle = normal_angle(T);
            const double weight = angle <= 30 ? __dadd_rn(1.0, __ddiv_rn(__dmul_rn(0.05, angle), 5.0))
                                              : 1.3;
            bf = ceil(__dmul_rn(a.buffer, weight));
        } else {
            bf = ceil(a.buffer);
        }
        vll_ugrid g = gp3[idx];
        if (P.L < 2) {
            // a node on a vertex takes the vertex's height (IDW branch)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double dx = __dadd_rn(cx, -T.x[k]), dy = __dadd_rn(cy, -T.y[k]);
                if (sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))) == 0) {
                    z = (float)T.z[k];
                    g.Matched_flag = 2;
                    break;
                }
            }
        }
        mb[idx] = 1;
        g.Height = z;
        newh[idx] = g.Height;
        double th;
        if (P.L == 4)
            th = 0.7;
        else if (P.L == 3)
            th = __dadd_rn(0.6, -__dmul_rn((double)(a.iteration - 1), 0.02));
        else if (P.L == 2)
            th = __dadd_rn(0.5, -__dmul_rn((double)(a.iteration - 1), 0.02));
        else if (P.L == 1)
            th = 0.4;
        else
            th = 0.3;
        if (th < 0.3) th = 0.3;
        const double zd = (double)z;
        const double t1 = dmin(tmin, zd);
        if (g.Matched_flag == 4) {
            if (__dadd_rn(t1, -bf) <= g.minHeight) g.minHeight = to_short(floor(__dadd_rn(t1, -bf)));
        } else {
            g.minHeight = to_short(floor(__dadd_rn(t1, -bf)));
        }
        const double t2 = dmax(tmax, zd);
        if (g.Matched_flag == 4) {
            if (__dadd_rn(t2, bf) >= g.maxHeight) g.maxHeight = to_short(ceil(__dadd_rn(t2, bf)));
        } else {
            g.maxHeight = to_short(ceil(__dadd_rn(t2, bf)));
        }
        if (g.minHeight > g.maxHeight) {
            const int16_t tmp = g.minHeight;
            g.minHeight = g.maxHeight;
            g.maxHeight = tmp;
        }
        if (g.Matched_flag == 2) {
            // through an int, as the reference's mintemp / maxtemp
            g.minHeight = to_short(floor(__dadd_rn(zd, -bf)));
            g.maxHeight = to_short(ceil(__dadd_rn(zd, bf)));
        } else {
            g.Matched_flag = 1;
            if (g.Mean_ortho_ncc > q_result(th)) {
                g.minHeight = to_short(floor(__dadd_rn(zd, -bf)));
                g.maxHeight = to_short(ceil(__dadd_rn(zd, bf)));
            } else if (P.L >= 2) {
                g.minHeight = to_short(floor(__dadd_rn(t1, -bf)));
                g.maxHeight = to_short(ceil(__dadd_rn(t2, bf)));
            }
        }
        const int gap = (int)g.maxHeight - (int)g.minHeight;
        if (gap > a.th_hg) {
            g.minHeight = -100;
            g.maxHeight = -100;
        }
        gp3[idx] = g;
    }
}

// Heights of the pass written back, and the snapshot the neighbour pass reads.
__global__ void snapshot_kernel(vll_ugrid *gp3, const float *newh, vll_ugrid *snap, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        gp3[i].Height = newh[i];
        snap[i] = gp3[i];
    }
}

// Nodes in no triangle (setsm_code.cpp:10096-10167): the union of the
// matched neighbours' ranges, or the scene extent at levels 0-1; the min /
// max of the ranges over the grid.
__global__ void neighbour_kernel(const DevLevel *__restrict__ Pp, vll_ugrid *gp3,
                                 const vll_ugrid *snap, uint8_t *mb,
                                 const unsigned long long *zext_key, const double *zext,
                                 RangeArgs a, int *hext) {
    const DevLevel &P = *Pp;
    const int64_t W = P.grid_w, H = P.grid_h;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < P.n_nodes;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = idx / W, col = idx % W;
        vll_ugrid g = gp3[idx];
        if (g.Matched_flag == 0) {
            int min_h = 10000, max_h = -10000;
            bool any = false;
            for (int64_t dr = -1; dr <= 1; ++dr)
                for (int64_t dc = -1; dc <= 1; ++dc) {
                    if (col + dc >= 0 && col + dc < W && row + dr >= 0 && row + dr < H) {
                        const vll_ugrid &n = snap[(col + dc) + (row + dr) * W];
                        if (n.Matched_flag != 0) {
                            any = true;
                            if (min_h > n.minHeight) min_h = n.minHeight;
                            if (max_h < n.maxHeight) max_h = n.maxHeight;
                        }
                    }
                }
            if (any) {
                g.minHeight = (int16_t)min_h;
                g.maxHeight = (int16_t)max_h;
                mb[idx] = 2;
            } else if (P.L <= 1) {
                const double tmin = zext[0], tmax = zext[1];
                const double diff = __ddiv_rn(fabs(__dadd_rn(tmax, -tmin)), 3.0);
                double bf = a.buffer > diff ? diff : a.buffer;
                // pwrtwo(Pyramid_step) * resolution
                if (bf < P.im_res) bf = P.im_res;
                if (g.minHeight < __dadd_rn(tmin, -bf)) g.minHeight = to_short(floor(__dadd_rn(tmin, -bf)));
                if (g.maxHeight > __dadd_rn(tmax, bf)) g.maxHeight = to_short(ceil(__dadd_rn(tmax, bf)));
            }
        } else if (mb[idx] == 0) {
            g.Matched_flag = 0;
        }
        atomicMin(hext, (int)g.minHeight);
        atomicMax(hext + 1, (int)g.maxHeight);
        const int gap = (int)g.maxHeight - (int)g.minHeight;
        if (gap > a.th_hg) {
            g.minHeight = -100;
            g.maxHeight = -100;
        }
        gp3[idx] = g;
    }
}

// The returned grid (setsm_code.cpp:10180-10237); `out` starts zeroed.
__global__ void result_kernel(const DevLevel *__restrict__ Pp, vll_ugrid *gp3, const uint8_t *mb,
                              vll_ugrid *out) {
    const DevLevel &P = *Pp;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < P.n_nodes;
         idx += (int64_t)gridDim.x * blockDim.x) {
        vll_ugrid g = gp3[idx];
        if (g.minHeight > g.maxHeight) {
            const int16_t tmp = g.maxHeight;
            g.maxHeight = g.minHeight;
            g.minHeight = tmp;
            gp3[idx] = g;
        }
        vll_ugrid r;
        memset(&r, 0, sizeof(r));
        r.Height = -1000;
        r.Matched_flag = g.Matched_flag;
        if (mb[idx] == 2 && g.Matched_flag == 0) r.Matched_flag = 1;
        r.roh = g.roh;
        r.Height = g.Height;
        r.anchor_flag = 0;
        // ortho_ncc[ti] with the reference's indexing (entries past the two
        // of the array are the record's following bytes; within the record only)
        const unsigned char *src = reinterpret_cast<const unsigned char *>(&g);
        unsigned char *dst = reinterpret_cast<unsigned char *>(&r);
        for (int ti = 1; ti < P.num_images; ++ti) {
            if (!P.im[ti].selected) continue;
            const int byte = 10 + 2 * ti;
            if (byte + 2 > (int)sizeof(vll_ugrid)) break;
            dst[byte] = src[byte];
            dst[byte + 1] = src[byte + 1];
        }
        r.Mean_ortho_ncc = g.Mean_ortho_ncc;
        r.minHeight = g.minHeight;
        if (r.minHeight < -100) r.minHeight = -100;
        r.maxHeight = g.maxHeight;
        if (mb[idx] == 0) r.Height = -1000.0f;
        if (r.minHeight == 0) r.minHeight = -1;
        if (r.maxHeight == 0) r.maxHeight = 1;
        out[idx] = r;
    }
}

__global__ void zext_kernel(const unsigned long long *key, double *zext) {
    // back from keys to doubles; the reference starts from +-100000
    double v[2];
    for (int k = 0; k < 2; ++k) {
        const unsigned long long b = key[k];
        v[k] = __longlong_as_double((long long)((b >> 63) ? (b & 0x7fffffffffffffffull) : ~b));
    }
    zext[0] = key[0] == ~0ull ? 100000.0 : dmin(100000.0, v[0]);
    zext[1] = key[1] == 0ull ? -100000.0 : dmax(-100000.0, v[1]);
}

unsigned blocks_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

}  // namespace

size_t height_range_scratch(int64_t n_nodes) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(n_nodes * 4) + al(n_nodes * 4) + al(n_nodes) + al(n_nodes * sizeof(vll_ugrid)) +
           al(16) + al(16) + al(8);
}

cudaError_t run_height_range(const DevLevel *dP, const DevLevel &hP, const vll_point3 *pts,
                             int64_t n_pts, const vll_tri *tris, int64_t n_tris, vll_ugrid *gp3,
                             vll_ugrid *out, double buffer, double th_hg, int iteration,
                             void *scratch, size_t scratch_bytes, double *min_h, double *max_h,
                             cudaStream_t s) {
    char *p = (char *)scratch;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    auto take = [&](size_t b) {
        void *r = p;
        p += al(b);
        return r;
    };
    const int64_t N = hP.n_nodes;
    unsigned int *winner = (unsigned int *)take(N * 4);
    float *newh = (float *)take(N * 4);
    uint8_t *mb = (uint8_t *)take(N);
    vll_ugrid *snap = (vll_ugrid *)take(N * sizeof(vll_ugrid));
    unsigned long long *zkey = (unsigned long long *)take(16);
    double *zext = (double *)take(16);
    int *hext = (int *)take(8);
    if ((size_t)(p - (char *)scratch) > scratch_bytes) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemsetAsync(winner, 0xff, N * 4, s))) return e;
    const unsigned long long zinit[2] = {~0ull, 0ull};
    const int hinit[2] = {2147483647, -2147483647 - 1};
    if ((e = cudaMemcpyAsync(zkey, zinit, 16, cudaMemcpyHostToDevice, s))) return e;
    if ((e = cudaMemcpyAsync(hext, hinit, 8, cudaMemcpyHostToDevice, s))) return e;
    if ((e = cudaMemsetAsync(out, 0, N * sizeof(vll_ugrid), s))) return e;
    const RangeArgs a{buffer, th_hg, iteration};
    if (n_tris > 0)
        cover_kernel<<<blocks_for(n_tris * 32, 128), 128, 0, s>>>(dP, pts, n_pts, tris, n_tris,
                                                                 winner, zkey);
    zext_kernel<<<1, 1, 0, s>>>(zkey, zext);
    node_update_kernel<<<blocks_for(N, 128), 128, 0, s>>>(dP, pts, tris, winner, gp3, newh, mb, a);
    snapshot_kernel<<<blocks_for(N, 256), 256, 0, s>>>(gp3, newh, snap, N);
    neighbour_kernel<<<blocks_for(N, 256), 256, 0, s>>>(dP, gp3, snap, mb, zkey, zext, a, hext);
    result_kernel<<<blocks_for(N, 256), 256, 0, s>>>(dP, gp3, mb, out);
    if ((e = cudaGetLastError())) return e;
    int h[2];
    if ((e = cudaMemcpyAsync(h, hext, 8, cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    // the reference starts its extent at +-100000
    *min_h = N > 0 && h[0] < 100000 ? (double)h[0] : 100000.0;
    *max_h = N > 0 && h[1] > -100000 ? (double)h[1] : -100000.0;
    return cudaSuccess;
}

}  // namespace vll

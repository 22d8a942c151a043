// vll_sgm.cu -- semi-global aggregation of AWNCC (setsm_code.cpp:7017-7509,
// SGM_start_pos / SGM_con_pos :6755-6999) on the GPU.
//
// SumCost[node][slot] accumulates, over 8 path directions, a cost that runs
// along every grid row, column and diagonal: at a path's first node the
// node's INCC, at each following node its INCC plus the best of the previous
// node's costs at the same height (and +-1 slot with penalty P1) or its
// maximum (penalty P2), minus that maximum.  The reference's arithmetic is
// reproduced exactly: costs are stored as float and combined in double, and
// SumCost is a float accumulated direction by direction in the reference's
// order (0: left->right, 1: right->left, 2: top->bottom, 3: bottom->top,
// 4..7: the diagonals).
//
// GPU mapping: one warp per path, lanes over the height slots of the current
// node.  All 8 directions run in one launch, each storing its path costs per
// slot, and a second pass adds the 8 in the reference's order (the float sums
// come out the same); when the 8 stores do not fit the scratch budget, one
// launch per direction accumulates in order instead.  In both, the previous
// node's costs and the current ones live in two shared-memory rows of the
// warp, and the path's voxel rows are copied into a four-row shared-memory
// ring two nodes ahead of their step (cp.async).  A diagonal direction's paths start from two
// walls (a column of rows and a row of columns); the path that starts at their
// common corner is walked by both of the reference's loops, so its nodes get
// the same contribution twice -- here one warp walks it and adds it twice.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include "vll_device.cuh"
#include "vll_internal.h"
#include "vll_split.h"

namespace vll {

namespace {

constexpr double kP1 = 0.3;   // AWNCC's P1 (setsm_code.cpp:7004)
constexpr double kP2 = 0.6;   // AWNCC's P2 (setsm_code.cpp:7005)
constexpr int kPHS = 1;       // P_HS_step (:7007)

// Start node and step of path `line` of direction `dir` (rows/columns of the
// reference's loops at setsm_code.cpp:7037-7499).  Returns false if `line` is
// beyond the direction's paths.  `twice` marks the corner path of a diagonal.
__device__ __forceinline__ bool path_of(int dir, int64_t line, int64_t W, int64_t H, int64_t &r0,
                                        int64_t &c0, int &dr, int &dc, bool &twice) {
    twice = false;
    switch (dir) {
        case 0: if (line >= H) return false; r0 = line; c0 = 0;     dr = 0;  dc = 1;  return true;
        case 1: if (line >= H) return false; r0 = line; c0 = W - 1; dr = 0;  dc = -1; return true;
        case 2: if (line >= W) return false; r0 = 0;     c0 = line; dr = 1;  dc = 0;  return true;
        case 3: if (line >= W) return false; r0 = H - 1; c0 = line; dr = -1; dc = 0;  return true;
        default: break;
    }
    // diagonals: lines [0, H) start on the side wall (rows), lines [H, H + W)
    // on the top / bottom wall (columns); the corner path is the first of both
    // loops and is walked once here, twice-counted
    const bool top_down = dir == 4 || dir == 5;   // rows advance +1
    const bool rightwards = dir == 4 || dir == 6; // columns advance +1
    dr = top_down ? 1 : -1;
    dc = rightwards ? 1 : -1;
    const int64_t wall_row = top_down ? 0 : H - 1;     // start row of column paths
    const int64_t wall_col = rightwards ? 0 : W - 1;   // start column of row paths
    if (line < H) {
        // side wall: the reference iterates its rows from start_row; the
        // corner row is the one equal to wall_row
        r0 = top_down ? line : H - 1 - line;
        c0 = wall_col;
        if (r0 == wall_row) twice = true;
        return true;
    }
    const int64_t k = line - H;
    if (k >= W) return false;
    c0 = rightwards ? k : W - 1 - k;
    r0 = wall_row;
    if (c0 == wall_col) return false;   // the corner path, walked by the side-wall line
    return true;
}

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// Lines of direction `dir`.
__host__ __device__ __forceinline__ int64_t lines_of(int dir, int64_t W, int64_t H) {
    return dir < 2 ? H : (dir < 4 ? W : H + W);
}

// The records of one path node the recurrence reads (warp-uniform).
struct NodeRec {
    int64_t off;             // the node's first voxel in the packed rows
    int n;                   // NumOfHeight
    int16_t min_h, max_w;    // NCCresult minHeight, max_WNCC
    int16_t g_min, g_max;    // UGRID minHeight, maxHeight
};

__device__ __forceinline__ NodeRec load_rec(const DevLevel &P, int64_t q) {
    const vll_nccresult R = P.ncc[q];
    const vll_ugrid g = P.gp3[q];
    NodeRec x;
    x.off = P.vox_off[q];
    x.n = R.NumOfHeight;
    x.min_h = R.minHeight;
    x.max_w = R.max_WNCC;
    x.g_min = g.minHeight;
    x.g_max = g.maxHeight;
    return x;
}

// Voxel rows in flight per warp: node j's row is read at step j, node j-1's
// (its flags) too, and node j+2's is being copied, so four slots.
constexpr int kRing = 4;
constexpr int kRowsPerWarp = 2 + kRing;   // two cost rows, kRing voxel rows

// Asynchronous copy of a node's voxel row (4-byte words) into a ring slot;
// one commit group per call, empty when the node is past the path's end.
__device__ __forceinline__ void issue_row(uint32_t *dst, const vll_voxel *src, int n, bool live,
                                          int lane) {
    if (live)
        for (int h = lane; h < n; h += 32) __pipeline_memcpy_async(dst + h, src + h, 4);
    __pipeline_commit();
}

__device__ __forceinline__ uint8_t vox_flag(uint32_t w) { return (uint8_t)(w & 0xffu); }
__device__ __forceinline__ int16_t vox_incc(uint32_t w) { return (int16_t)(w >> 16); }

// One direction's path costs.  Accumulating form (lr == nullptr): the costs
// are added into sumcost (one launch per direction, in order).  Storing form:
// blockIdx.y is the direction and every slot's cost goes to lr[dir][slot]
// (0 where the reference adds nothing), for sgm_sum_kernel.
//
// A path is a chain of steps, each waiting for its node's voxel row, so the
// rows are copied into shared memory two nodes ahead (cp.async) and the
// nodes' records loaded four ahead; a step then waits only for a row issued
// two steps earlier.
__global__ void __launch_bounds__(128) sgm_dir_kernel(const DevLevel *__restrict__ Pp, int dir,
                                                      int64_t n_lines, float *__restrict__ sumcost,
                                                      int max_h, float *__restrict__ lr,
                                                      int64_t n_slots) {
    extern __shared__ float sm_lh[];
    const DevLevel &P = *Pp;
    if (lr) {
        dir = blockIdx.y;
        n_lines = lines_of(dir, P.grid_w, P.grid_h);
        lr += (int64_t)dir * n_slots;
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *buf0 = sm_lh + (size_t)warp * kRowsPerWarp * max_h;
    float *buf1 = buf0 + max_h;
    uint32_t *ring = reinterpret_cast<uint32_t *>(buf1 + max_h);
    const int64_t W = P.grid_w, Hh = P.grid_h;
    const double step = P.height_step;
    // a power-of-two step divides exactly as a multiplication by its
    // reciprocal (also a power of two): the same bits as the division
    int step_exp = 0;
    const bool step_pow2 = step > 0 && frexp(step, &step_exp) == 0.5;
    const double inv_step = step_pow2 ? ldexp(1.0, 1 - step_exp) : 0.0;
    const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t line = blockIdx.x * (int64_t)(blockDim.x >> 5) + warp; line < n_lines;
         line += warps_total) {
        int64_t r, c;
        int dr, dc;
        bool twice;
        if (!path_of(dir, line, W, Hh, r, c, dr, dc, twice)) continue;
        const int64_t len_r = dr > 0 ? Hh - r : (dr < 0 ? r + 1 : INT64_MAX);
        const int64_t len_c = dc > 0 ? W - c : (dc < 0 ? c + 1 : INT64_MAX);
        const int64_t len = len_r < len_c ? len_r : len_c;   // nodes on the path
        auto node = [&](int64_t j) { return (r + j * dr) * W + (c + j * dc); };
        // records of nodes j .. j+4
        NodeRec q0, q1, q2, q3, q4;
        q0 = load_rec(P, node(0));
        q1 = len > 1 ? load_rec(P, node(1)) : q0;
        q2 = len > 2 ? load_rec(P, node(2)) : q0;
        q3 = len > 3 ? load_rec(P, node(3)) : q0;
        q4 = len > 4 ? load_rec(P, node(4)) : q0;
        issue_row(ring, P.vox + q0.off, q0.n, true, lane);
        issue_row(ring + max_h, P.vox + q1.off, q1.n, len > 1, lane);
        float *pre = buf0, *cur = buf1;
        NodeRec T = q0;   // previous node
        for (int64_t j = 0; j < len; ++j) {
            issue_row(ring + ((j + 2) & (kRing - 1)) * max_h, P.vox + q2.off, q2.n, j + 2 < len,
                      lane);
            __pipeline_wait_prior(2);   // node j's row (the two newest may still fly)
            __syncwarp();
            const uint32_t *vrow = ring + (j & (kRing - 1)) * max_h;
            const uint32_t *trow = ring + ((j - 1) & (kRing - 1)) * max_h;
            const NodeRec R = q0;
            float *sc = sumcost + R.off;
            if (j == 0) {
                // ---- first node: SGM_start_pos (:6755-6767) ----
                for (int h = lane; h < R.n; h += 32) {
                    const float hgt = (float)__dadd_rn((double)R.min_h, __dmul_rn((double)h, step));
                    float v = 0.f;
                    if (hgt >= (float)R.g_min && hgt <= (float)R.g_max) {
                        v = (float)dq_voxel(vox_incc(vrow[h]));
                        if (!lr) {
                            float s = sc[h] + v;
                            if (twice) s = s + v;
                            sc[h] = s;
                        }
                    }
                    if (lr) lr[R.off + h] = v;
                    pre[h] = v;
                }
            } else {
                // ---- following nodes: SGM_con_pos (:6769-6999) ----
                const float max_w = (float)dq_result(T.max_w);
                const int tn = T.n;
                for (int h = lane; h < R.n; h += 32) {
                    const float hgt = (float)__dadd_rn((double)R.min_h, __dmul_rn((double)h, step));
                    float out = 0.f;
                    if (hgt >= (float)R.g_min && hgt <= (float)R.g_max) {
                        const double wncc = dq_voxel(vox_incc(vrow[h]));
                        // (float iter_height - short minHeight) is a float subtraction in
                        // the reference, then divided by the double step
                        const double dh = (double)__fsub_rn(hgt, (float)T.min_h);
                        const int i0 = (int)(step_pow2 ? __dmul_rn(dh, inv_step) : __ddiv_rn(dh, step));
                        const int i1 = i0 - kPHS, i2 = i0 + kPHS;
                        double V1 = 0, V2 = 0, V3 = 0;
                        const double V4 = __dadd_rn((double)max_w, -kP2);
                        double m;
                        if (i0 == 0 && i2 >= 0 && i2 < tn) {
                            const bool f = vox_flag(trow[i0]), f2 = vox_flag(trow[i2]);
                            if (f && f2) {
                                V2 = __dadd_rn((double)pre[i2], -kP1);
                                V3 = (double)pre[i0];
                                m = dmax(dmax(V2, V3), V4);
                            } else if (f) {
                                V3 = (double)pre[i0];
                                m = dmax(V3, V4);
                            } else if (f2) {
                                V2 = __dadd_rn((double)pre[i2], -kP1);
                                m = dmax(V2, V4);
                            } else {
                                m = V4;
                            }
                        } else if (i0 == tn - 1 && i1 >= 0 && i1 < tn) {
                            const bool f = vox_flag(trow[i0]), f1 = vox_flag(trow[i1]);
                            if (f && f1) {
                                V1 = __dadd_rn((double)pre[i1], -kP1);
                                V3 = (double)pre[i0];
                                m = dmax(dmax(V1, V3), V4);
                            } else if (f) {
                                V3 = (double)pre[i0];
                                m = dmax(V3, V4);
                            } else if (f1) {
                                V1 = __dadd_rn((double)pre[i1], -kP1);
                                m = dmax(V1, V4);
                            } else {
                                m = V4;
                            }
                        } else if (i0 > 0 && i0 < tn - 1 && i1 >= 0 && i1 < tn && i2 >= 0 && i2 < tn) {
                            const bool f = vox_flag(trow[i0]), f1 = vox_flag(trow[i1]),
                                       f2 = vox_flag(trow[i2]);
                            if (f && f1 && f2) {
                                V1 = __dadd_rn((double)pre[i1], -kP1);
                                V2 = __dadd_rn((double)pre[i2], -kP1);
                                V3 = (double)pre[i0];
                                m = dmax(dmax(dmax(V1, V2), V3), V4);
                            } else if (f && f1) {
                                V1 = __dadd_rn((double)pre[i1], -kP1);
                                V3 = (double)pre[i0];
                                m = dmax(dmax(V1, V3), V4);
                            } else if (f1 && f2) {
                                // V3 keeps its initial 0 and takes part (setsm_code.cpp:6917-6925)
                                V1 = __dadd_rn((double)pre[i1], -kP1);
                                V2 = __dadd_rn((double)pre[i2], -kP1);
                                m = dmax(dmax(dmax(V1, V2), V3), V4);
                            } else if (f && f2) {
                                V2 = __dadd_rn((double)pre[i2], -kP1);
                                V3 = (double)pre[i0];
                                m = dmax(dmax(V2, V3), V4);
                            } else if (f) {
                                V3 = (double)pre[i0];
                                m = dmax(V3, V4);
                            } else if (f1) {
                                V1 = __dadd_rn((double)pre[i1], -kP1);
                                m = dmax(V1, V4);
                            } else if (f2) {
                                V2 = __dadd_rn((double)pre[i2], -kP1);
                                m = dmax(V2, V4);
                            } else {
                                m = V4;
                            }
                        } else {
                            m = V4;
                        }
                        const double t = __dadd_rn(m, -(double)max_w);
                        out = (float)__dadd_rn(wncc, t);
                        if (!lr) {
                            float s = sc[h] + out;
                            if (twice) s = s + out;
                            sc[h] = s;
                        }
                    }
                    if (lr) lr[R.off + h] = out;
                    cur[h] = out;
                }
                float *tmp = pre;
                pre = cur;
                cur = tmp;
            }
            __syncwarp();   // node j-1's row slot is refilled at the next step
            T = q0;
            q0 = q1;
            q1 = q2;
            q2 = q3;
            q3 = q4;
            if (j + 5 < len) q4 = load_rec(P, node(j + 5));
        }
        __pipeline_wait_prior(0);
        __syncwarp();
    }
}

// SumCost of every slot from the 8 stored direction costs, added in the
// reference's direction order, a diagonal's corner path twice (the nodes
// (k, k) of direction 4, (k, W-1-k) of 5, (H-1-k, k) of 6, (H-1-k, W-1-k) of 7).
__global__ void sgm_sum_kernel(const DevLevel *__restrict__ Pp, const float *__restrict__ lr,
                               int64_t n_slots, float *__restrict__ sumcost) {
    const DevLevel &P = *Pp;
    const int64_t W = P.grid_w, H = P.grid_h;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t pt = warp; pt < P.n_nodes; pt += n_warps) {
        const int64_t r = pt / W, c = pt % W;
        const bool twice[8] = {false, false, false, false, r == c, r == W - 1 - c,
                               H - 1 - r == c, H - 1 - r == W - 1 - c};
        const int64_t o = P.vox_off[pt];
        const int n = P.ncc[pt].NumOfHeight;
        for (int h = lane; h < n; h += 32) {
            float sc = 0.f;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const float v = lr[(int64_t)d * n_slots + o + h];
                sc = sc + v;
                if (twice[d]) sc = sc + v;
            }
            sumcost[o + h] = sc;
        }
    }
}

}  // namespace

// The stored-direction form needs 8 floats per slot of scratch; it runs when
// that fits this budget, else the directions run one launch after another.
constexpr double kSgmConcurrentBytes = 24e9;

size_t sgm_scratch_bytes(int64_t n_slots) {
    const double b = 8.0 * 4.0 * (double)(n_slots > 0 ? n_slots : 1);
    return b <= kSgmConcurrentBytes ? (size_t)b : 0;
}

// All 8 directions of the aggregation into sumcost (float, the packed voxel
// layout).  With `lr` (sgm_scratch_bytes(n_slots) bytes) the 8 directions run
// in one launch and sgm_sum_kernel forms the sums; without, one launch per
// direction in the reference's order accumulates them.  max_h: the largest
// NumOfHeight of the level.
cudaError_t launch_sgm(const DevLevel *dP, int64_t grid_w, int64_t grid_h, int max_h,
                       float *sumcost, int64_t n_slots, cudaStream_t s, float *lr) {
    cudaError_t e;
    if (!lr) {
        e = cudaMemsetAsync(sumcost, 0, (size_t)(n_slots > 0 ? n_slots : 1) * 4, s);
        if (e != cudaSuccess) return e;
    }
    if (max_h < 1) max_h = 1;
    const size_t per_warp = (size_t)kRowsPerWarp * max_h * sizeof(float);
    if (per_warp > 200 * 1024) return cudaErrorInvalidValue;
    int warps = (int)std::min<size_t>(4, (200 * 1024) / per_warp);
    if (warps < 1) warps = 1;
    const size_t smem = per_warp * warps;
    e = ensure_smem_limit((const void *)sgm_dir_kernel, smem);
    if (e != cudaSuccess) return e;
    if (lr) {
        // every direction at once (blockIdx.y); blocks beyond a direction's
        // lines find no path and return
        const int64_t most = grid_h + grid_w;
        int64_t blocks = (most + warps - 1) / warps;
        if (blocks > 148 * 64) blocks = 148 * 64;
        if (blocks < 1) blocks = 1;
        sgm_dir_kernel<<<dim3((unsigned)blocks, 8), warps * 32, smem, s>>>(dP, 0, 0, sumcost, max_h,
                                                                          lr, n_slots);
        if ((e = cudaGetLastError())) return e;
        int64_t sb = (grid_w * grid_h + 7) / 8;
        if (sb > 148 * 32) sb = 148 * 32;
        if (sb < 1) sb = 1;
        sgm_sum_kernel<<<(unsigned)sb, 256, 0, s>>>(dP, lr, n_slots, sumcost);
        return cudaGetLastError();
    }
    for (int dir = 0; dir < 8; ++dir) {
        const int64_t n_lines = lines_of(dir, grid_w, grid_h);
        int64_t blocks = (n_lines + warps - 1) / warps;
        if (blocks > 148 * 64) blocks = 148 * 64;
        if (blocks < 1) blocks = 1;
        sgm_dir_kernel<<<(unsigned)blocks, warps * 32, smem, s>>>(dP, dir, n_lines, sumcost, max_h,
                                                                 nullptr, n_slots);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace vll

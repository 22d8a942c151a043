// vll_tin.cu -- TINCreate_list (SubFunctions.cpp:2768-2846) on the GPU: the
// Delaunay triangulation of the matched points snapped to the level's grid,
// returned as the reference's ordered list of vertex-index triples.
//
// The reference triangulates with an alternating-cut divide and conquer
// (grid_triangulation.cpp, after Guibas-Stolfi and Wu et al.): a node sorts
// its points by (col, row) -- or by (row, -col) one level down --, splits them
// at the median, triangulates both halves and zips them together from the
// lower (or right) common tangent, preferring the left candidate on
// co-circular ties.  On an integer grid co-circular points are common, so
// the triangles depend on that exact order of decisions, and the list's
// order on where each half-edge lives in memory (the edge allocator's stack,
// split and merged with the recursion; a point's triangles are listed from
// the edge of it stored last).  This file replays the same recursion level
// by level: every node of a depth sorts its range at once (segmented radix
// sort), then, deepest first, every node of a depth triangulates its base
// case or merges its children in one thread, each on its own slice of the
// shared half-edge pool and allocator stack.  Then one thread per point walks
// its triangles in the reference's order.  Integer predicates are 64-bit with
// the reference's wrap-around arithmetic.
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include "vll_internal.h"
#include "vll_tin_core.cuh"

namespace vll {
namespace {

using namespace tin;

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// Grid coordinates of the points (SubFunctions.cpp:2793-2798: 0.5 plus the
// offset in grid cells, truncated to int) and their grid index.
__global__ void tin_coords_kernel(const vll_point3 *__restrict__ pts, int n, double minx,
                                  double miny, double res, int width, int *__restrict__ row,
                                  int *__restrict__ col, unsigned long long *__restrict__ gkey,
                                  int *__restrict__ ids) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = (int)(0.5 + __ddiv_rn(__dadd_rn(pts[i].x, -minx), res));
        const int r = (int)(0.5 + __ddiv_rn(__dadd_rn(pts[i].y, -miny), res));
        col[i] = c;
        row[i] = r;
        // grid index row * width + col, biased so that any int pair sorts
        gkey[i] = (unsigned long long)((long long)r * width + c + (1ll << 62));
        ids[i] = i;
    }
}

// Flags a grid cell holding two points (the triangulation needs distinct points).
__global__ void tin_dup_kernel(const unsigned long long *__restrict__ sorted, int n,
                               unsigned int *__restrict__ err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += gridDim.x * blockDim.x)
        if (sorted[i] == sorted[i - 1]) atomicExch(err + 1, 1u);
}

// Sort keys of the positions inside this depth's ranges: (col, row) or
// (row, -col), both non-negative in the biased 32-bit halves.
__global__ void tin_keys_kernel(const int *__restrict__ perm, int n, int horiz,
                                const int *__restrict__ row, const int *__restrict__ col,
                                unsigned long long *__restrict__ keys) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = perm[i];
        const unsigned int r = (unsigned int)row[p] ^ 0x80000000u;
        const unsigned int c = (unsigned int)col[p] ^ 0x80000000u;
        keys[i] = horiz ? (((unsigned long long)c << 32) | r)
                        : (((unsigned long long)r << 32) | (0xFFFFFFFFu - c));
    }
}

__global__ void tin_iota_kernel(int *__restrict__ a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = (int)i;
}

// One thread per subtree of fewer than 100 points, over its post-order list
// (order[start[i] .. start[i + 1])).
__global__ void tin_serial_kernel(TinGraph G, TinNode *nodes, const int *__restrict__ order,
                                  const int *__restrict__ start, int m, const int *__restrict__ perm,
                                  long long bound) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        serial_subtree(G, nodes, order + start[i], start[i + 1] - start[i], perm, bound);
}

// EdgeList::MergeEdgeLists (edge_list.cpp:96-106): the right (top) child's
// free stack moves down onto the left (bottom) child's.  One warp per node;
// the destination precedes the source, so copying 32 entries at a time in
// increasing order (each group read before written) is safe.
__global__ void tin_concat_kernel(TinGraph G, const TinNode *nodes, const int *__restrict__ list,
                                  int m) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < m; w += warps) {
        const TinNode &N = nodes[list[w]];
        const TinNode &L = nodes[N.left];
        const TinNode &R = nodes[N.right];
        const int src = 6 * R.lo, dst = 6 * N.lo + L.idx;
        for (int k0 = 0; k0 < R.idx; k0 += 32) {
            const int k = k0 + lane;
            int v = 0;
            if (k < R.idx) v = G.unused[src + k];
            __syncwarp();
            if (k < R.idx) G.unused[dst + k] = v;
            __syncwarp();
        }
    }
}

__global__ void tin_merge_kernel(TinGraph G, TinNode *nodes, const int *__restrict__ list, int m,
                                 long long bound) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        threaded_merge(G, nodes, list[i], bound);
}

// EdgeList::SetGrid (basic_topology_types.hpp:157-202): a point keeps the
// in-use edge out of it that is last in the pool.
__global__ void tin_invalid_kernel(const int *__restrict__ unused, int n_free,
                                   unsigned char *__restrict__ invalid) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_free; i += gridDim.x * blockDim.x)
        invalid[unused[i]] = 1;
}

__global__ void tin_store_kernel(const int *__restrict__ orig, const unsigned char *__restrict__ invalid,
                                 long long n_edges, int *__restrict__ stored) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n_edges;
         t += (long long)gridDim.x * blockDim.x)
        if (!invalid[t]) atomicMax(stored + orig[t], (int)t);
}

// Grid::GetAllTris (grid.cpp:16-51): the points in grid order, each listing
// the triangles around it (AdjTriIter, counter-clockwise from its stored
// edge) of which it is the (col, row)-smallest vertex.  Pass 0 counts, pass 1
// writes the vertices' input indices at the exclusive prefix `off`.
template <bool WRITE>
__global__ void tin_tris_kernel(TinGraph G, const int *__restrict__ order, int n,
                                const int *__restrict__ stored, long long *__restrict__ cnt,
                                const long long *__restrict__ off, vll_tri *__restrict__ out,
                                long long cap, long long bound) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = order[i];
        long long c = 0;
        long long o = WRITE ? off[i] : 0;
        point_tris(G, stored[p], bound, [&](int q0, int q1, int q2) {
            if (WRITE && o < cap) out[o] = vll_tri{(uint32_t)q0, (uint32_t)q1, (uint32_t)q2};
            ++o;
            ++c;
        });
        if (!WRITE) cnt[i] = c;
    }
}

// THREADED_CUTOFF (basic_topology_types.hpp:15): nodes below it recurse
// serially on one edge list.
constexpr int kThreadedCutoff = 100;

inline int grid1(long long n, int threads, int cap = 148 * 32) {
    const long long b = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(b, cap));
}

}  // namespace

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
void tin_release(TinWork &w) {
    for (auto &b : w.bufs)
        if (b.first) cudaFree(b.first);
    w.bufs.clear();
}

namespace {

// A device array of the work area, grown on demand (kept between calls).
template <class T>
cudaError_t tin_buf(TinWork &w, size_t slot, size_t count, T **out) {
    if (w.bufs.size() <= slot) w.bufs.resize(slot + 1, {nullptr, 0});
    auto &b = w.bufs[slot];
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (b.second < bytes) {
        if (b.first) cudaFree(b.first);
        b.first = nullptr;
        b.second = 0;
        const cudaError_t e = cudaMalloc(&b.first, bytes);
        if (e != cudaSuccess) return e;
        b.second = bytes;
    }
    *out = (T *)b.first;
    return cudaSuccess;
}

}  // namespace

int run_tin_create(TinWork &w, const vll_point3 *d_pts, int64_t n64, const double min_max[4],
                   double resolution, vll_tri *d_tris, int64_t capacity, int64_t *count,
                   cudaStream_t s, std::string *err) {
#define TIN_CUDA(call)                                              \
    do {                                                            \
        const cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) {                                   \
            *err = std::string(#call) + ": " + cudaGetErrorString(e__); \
            return VLL_ERR_CUDA;                                    \
        }                                                           \
    } while (0)
    *count = 0;
    if (n64 <= 2) return VLL_OK;   // TINCreate_list: no triangulation below 3 points
    if (n64 > (1 << 26)) {
        *err = "more points than the triangulation's 32-bit edge indices allow";
        return VLL_ERR_CAPACITY;
    }
    const int n = (int)n64;
    const int width = (int)(1 + (min_max[2] - min_max[0]) / resolution);
    const int height = (int)(1 + (min_max[3] - min_max[1]) / resolution);
    if (width > 32767 || height > 32767) {
        char m[160];
        snprintf(m, sizeof m, "grid of %d x %d cells exceeds the triangulation's 16-bit limit",
                 width, height);
        *err = m;
        return VLL_ERR_INVALID;
    }
    // ---- the recursion tree (it depends on n only) ----
    std::vector<TinNode> nodes;
    std::vector<int> depth;
    nodes.reserve((size_t)n);
    {
        struct Item {
            int lo, cnt, horiz, depth, parent, side;
        };
        std::vector<Item> stack{{0, n, 1, 0, -1, 0}};
        while (!stack.empty()) {
            const Item it = stack.back();
            stack.pop_back();
            const int id = (int)nodes.size();
            TinNode N{};
            N.lo = it.lo;
            N.cnt = it.cnt;
            N.left = N.right = -1;
            N.horiz = it.horiz;
            nodes.push_back(N);
            depth.push_back(it.depth);
            if (it.parent >= 0) (it.side ? nodes[it.parent].right : nodes[it.parent].left) = id;
            if (it.cnt >= 4) {
                const int mid = it.cnt / 2;
                stack.push_back({it.lo + mid, it.cnt - mid, !it.horiz, it.depth + 1, id, 1});
                stack.push_back({it.lo, mid, !it.horiz, it.depth + 1, id, 0});
            }
        }
    }
    const int n_nodes = (int)nodes.size();
    const int max_depth = *std::max_element(depth.begin(), depth.end());
    // per depth: the ranges sorted there (every internal node) and the
    // merges of nodes of 100 points or more; and the post-order lists of the
    // subtrees below 100 points, each triangulated by one thread
    std::vector<std::vector<int>> inner(max_depth + 1), threaded(max_depth + 1);
    std::vector<int> parent((size_t)n_nodes, -1);
    for (int i = 0; i < n_nodes; ++i) {
        if (nodes[i].left < 0) continue;
        inner[depth[i]].push_back(i);
        if (nodes[i].cnt >= kThreadedCutoff) threaded[depth[i]].push_back(i);
        parent[nodes[i].left] = parent[nodes[i].right] = i;
    }
    std::vector<int> lists, serial_start{0};
    std::vector<size_t> threaded_at(max_depth + 1);
    for (int d = 0; d <= max_depth; ++d) {
        threaded_at[d] = lists.size();
        lists.insert(lists.end(), threaded[d].begin(), threaded[d].end());
    }
    const size_t serial_at = lists.size();
    {
        std::vector<std::pair<int, int>> stk;
        for (int r = 0; r < n_nodes; ++r) {
            if (nodes[r].cnt >= kThreadedCutoff) continue;
            if (parent[r] >= 0 && nodes[parent[r]].cnt < kThreadedCutoff) continue;
            stk.assign(1, {r, 0});
            while (!stk.empty()) {
                auto &t = stk.back();
                const int v = t.first;
                if (nodes[v].left < 0 || t.second == 2) {
                    lists.push_back(v);
                    stk.pop_back();
                    continue;
                }
                const int c = t.second++ == 0 ? nodes[v].left : nodes[v].right;
                stk.push_back({c, 0});
            }
            serial_start.push_back((int)(lists.size() - serial_at));
        }
    }
    const int n_serial = (int)serial_start.size() - 1;
    // begin / end of every depth's sorted ranges, uploaded once
    std::vector<int> seg_begin, seg_end;
    std::vector<size_t> seg_at(max_depth + 1);
    for (int d = 0; d <= max_depth; ++d) {
        seg_at[d] = seg_begin.size();
        for (int id : inner[d]) {
            seg_begin.push_back(nodes[id].lo);
            seg_end.push_back(nodes[id].lo + nodes[id].cnt);
        }
    }
    // ---- device buffers ----
    const long long n_edges = 6ll * n;
    int *row, *col, *ids, *ids_sorted, *perm, *perm2, *unused, *stored, *dlist, *sb, *se, *dstart;
    int *dnext, *oprev, *twin, *orig;
    unsigned long long *gkey, *gkey_sorted, *keys, *keys2;
    unsigned int *flags;
    unsigned char *invalid;
    long long *tcnt, *toff;
    TinNode *dnodes;
    size_t slot = 0;
    TIN_CUDA(tin_buf(w, slot++, n, &row));
    TIN_CUDA(tin_buf(w, slot++, n, &col));
    TIN_CUDA(tin_buf(w, slot++, n, &ids));
    TIN_CUDA(tin_buf(w, slot++, n, &ids_sorted));
    TIN_CUDA(tin_buf(w, slot++, n, &perm));
    TIN_CUDA(tin_buf(w, slot++, n, &perm2));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_edges, &unused));
    TIN_CUDA(tin_buf(w, slot++, n, &stored));
    TIN_CUDA(tin_buf(w, slot++, lists.size(), &dlist));
    TIN_CUDA(tin_buf(w, slot++, serial_start.size(), &dstart));
    TIN_CUDA(tin_buf(w, slot++, seg_begin.size(), &sb));
    TIN_CUDA(tin_buf(w, slot++, seg_end.size(), &se));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_edges, &dnext));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_edges, &oprev));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_edges, &twin));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_edges, &orig));
    TIN_CUDA(tin_buf(w, slot++, n, &gkey));
    TIN_CUDA(tin_buf(w, slot++, n, &gkey_sorted));
    TIN_CUDA(tin_buf(w, slot++, n, &keys));
    TIN_CUDA(tin_buf(w, slot++, n, &keys2));
    TIN_CUDA(tin_buf(w, slot++, 4, &flags));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_edges, &invalid));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n + 1, &tcnt));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n + 1, &toff));
    TIN_CUDA(tin_buf(w, slot++, (size_t)n_nodes, &dnodes));
    // temporary storage of the library sorts and scans
    size_t tmp_bytes = 0, t1 = 0;
    TIN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, gkey, gkey_sorted, ids, ids_sorted, n, 0,
                                             64, s));
    tmp_bytes = std::max(tmp_bytes, t1);
    TIN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t1, tcnt, toff, n + 1, s));
    tmp_bytes = std::max(tmp_bytes, t1);
    int max_segs = 1;
    for (int d = 0; d <= max_depth; ++d) max_segs = std::max(max_segs, (int)inner[d].size());
    TIN_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, t1, keys, keys2, perm, perm2, n, max_segs,
                                                 sb, se, s));
    tmp_bytes = std::max(tmp_bytes, t1);
    void *tmp;
    TIN_CUDA(tin_buf(w, slot++, tmp_bytes, (unsigned char **)&tmp));

    TIN_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(unsigned int), s));
    TIN_CUDA(cudaMemcpyAsync(dnodes, nodes.data(), nodes.size() * sizeof(TinNode),
                             cudaMemcpyHostToDevice, s));
    TIN_CUDA(cudaMemcpyAsync(dlist, lists.data(), lists.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    TIN_CUDA(cudaMemcpyAsync(dstart, serial_start.data(), serial_start.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    if (!seg_begin.empty()) {
        TIN_CUDA(cudaMemcpyAsync(sb, seg_begin.data(), seg_begin.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
        TIN_CUDA(cudaMemcpyAsync(se, seg_end.data(), seg_end.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
    }
    tin_coords_kernel<<<grid1(n, 256), 256, 0, s>>>(d_pts, n, min_max[0], min_max[1], resolution,
                                                    width, row, col, gkey, ids);
    TIN_CUDA(cudaGetLastError());
    // grid order of the points (GetAllTris walks it) and the distinctness check
    t1 = tmp_bytes;
    TIN_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t1, gkey, gkey_sorted, ids, ids_sorted, n, 0, 64,
                                             s));
    tin_dup_kernel<<<grid1(n, 256), 256, 0, s>>>(gkey_sorted, n, flags);
    TIN_CUDA(cudaGetLastError());
    // ---- ranges sorted top-down, depth by depth ----
    tin_iota_kernel<<<grid1(n, 256), 256, 0, s>>>(perm, n);
    TIN_CUDA(cudaGetLastError());
    for (int d = 0; d <= max_depth; ++d) {
        if (inner[d].empty()) continue;
        // positions outside this depth's ranges keep their place
        TIN_CUDA(cudaMemcpyAsync(perm2, perm, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, s));
        tin_keys_kernel<<<grid1(n, 256), 256, 0, s>>>(perm, n, nodes[inner[d][0]].horiz, row, col,
                                                      keys);
        TIN_CUDA(cudaGetLastError());
        t1 = tmp_bytes;
        TIN_CUDA(cub::DeviceSegmentedSort::SortPairs(tmp, t1, keys, keys2, perm, perm2, n,
                                                     (int)inner[d].size(), sb + seg_at[d],
                                                     se + seg_at[d], s));
        std::swap(perm, perm2);
    }
    // ---- triangulation bottom-up ----
    TinGraph G{dnext, oprev, twin, orig, row, col, unused, flags};
    tin_iota_kernel<<<grid1(n_edges, 256), 256, 0, s>>>(unused, n_edges);
    TIN_CUDA(cudaGetLastError());
    const long long bound = 64ll * n + 1024;
    tin_serial_kernel<<<grid1(n_serial, 32), 32, 0, s>>>(G, dnodes, dlist + serial_at, dstart,
                                                         n_serial, perm, bound);
    TIN_CUDA(cudaGetLastError());
    for (int d = max_depth; d >= 0; --d) {
        const int ni = (int)threaded[d].size();
        if (!ni) continue;
        tin_concat_kernel<<<grid1(32ll * ni, 128), 128, 0, s>>>(G, dnodes, dlist + threaded_at[d], ni);
        TIN_CUDA(cudaGetLastError());
        tin_merge_kernel<<<grid1(ni, 32), 32, 0, s>>>(G, dnodes, dlist + threaded_at[d], ni, bound);
        TIN_CUDA(cudaGetLastError());
    }
    // ---- stored edge per point, then the triangle list ----
    TinNode root;
    TIN_CUDA(cudaMemcpyAsync(&root, dnodes, sizeof(TinNode), cudaMemcpyDeviceToHost, s));
    TIN_CUDA(cudaStreamSynchronize(s));
    TIN_CUDA(cudaMemsetAsync(invalid, 0, (size_t)n_edges, s));
    TIN_CUDA(cudaMemsetAsync(stored, 0xff, (size_t)n * sizeof(int), s));
    if (root.idx > 0) {
        tin_invalid_kernel<<<grid1(root.idx, 256), 256, 0, s>>>(unused, root.idx, invalid);
        TIN_CUDA(cudaGetLastError());
    }
    tin_store_kernel<<<grid1(n_edges, 256), 256, 0, s>>>(orig, invalid, n_edges, stored);
    TIN_CUDA(cudaGetLastError());
    tin_tris_kernel<false><<<grid1(n, 128), 128, 0, s>>>(G, ids_sorted, n, stored, tcnt, nullptr,
                                                         nullptr, 0, bound);
    TIN_CUDA(cudaGetLastError());
    TIN_CUDA(cudaMemsetAsync(tcnt + n, 0, sizeof(long long), s));
    t1 = tmp_bytes;
    TIN_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t1, tcnt, toff, n + 1, s));
    long long total = 0;
    unsigned int hflags[4];
    TIN_CUDA(cudaMemcpyAsync(&total, toff + n, sizeof(total), cudaMemcpyDeviceToHost, s));
    TIN_CUDA(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
    TIN_CUDA(cudaStreamSynchronize(s));
    if (hflags[1]) {
        *err = "two points fall into one grid cell (the triangulation needs distinct points)";
        return VLL_ERR_INVALID;
    }
    if (hflags[0]) {
        *err = "triangulation walk exceeded its bound (malformed input)";
        return VLL_ERR_INVALID;
    }
    *count = total;
    if (total > capacity) {
        *err = "triangle list longer than the output capacity";
        return VLL_ERR_CAPACITY;
    }
    tin_tris_kernel<true><<<grid1(n, 128), 128, 0, s>>>(G, ids_sorted, n, stored, nullptr, toff,
                                                        d_tris, capacity, bound);
    TIN_CUDA(cudaGetLastError());
    TIN_CUDA(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
    TIN_CUDA(cudaStreamSynchronize(s));
    if (hflags[0]) {
        *err = "triangulation walk exceeded its bound (malformed input)";
        return VLL_ERR_INVALID;
    }
#undef TIN_CUDA
    return VLL_OK;
}

}  // namespace vll

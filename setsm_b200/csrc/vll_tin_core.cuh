// vll_tin_core.cuh -- the triangulation steps of TINCreate_list
// (grid_triangulation.cpp): half-edge pool, the reference's edge allocator,
// integer predicates, base cases and the merge of two halves.  Compiled for
// the device by vll_tin.cu; the functions are host-callable too, so the same
// steps can run serially on the CPU.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define VLL_TIN_HD __host__ __device__
#else
#define VLL_TIN_HD
#endif

namespace vll {
namespace tin {

// Half-edges (struct Edge, basic_topology_types.hpp:73-79) as arrays of
// indices into the pool; orig is a point id (the points are distinct, so a
// point's id stands for its grid coordinates).
struct TinGraph {
    int *dnext;    // next edge out of the destination, counter-clockwise
    int *oprev;    // previous edge into the origin, counter-clockwise
    int *twin;
    int *orig;
    const int *row, *col;   // grid coordinates by point id
    int *unused;            // the allocator's stack of free edges
    unsigned int *err;      // [0] set when a walk exceeds its bound
};

// A node of the recursion: points [lo, lo + cnt) of the permutation.
struct TinNode {
    int lo, cnt;
    int left, right;   // children (-1 for a base case of 2 or 3 points)
    int horiz;         // sorted by (col, row) and cut into left / right halves
    int idx;           // height of the node's free-edge stack (base 6 lo)
    int ex[4];         // hull extremes: left ccw, right cw, bottom ccw, top cw
};
enum { EX_L = 0, EX_R = 1, EX_B = 2, EX_T = 3 };

VLL_TIN_HD inline bool less_xy(const TinGraph &G, int a, int b) {
    const int ac = G.col[a], bc = G.col[b];
    return ac < bc || (ac == bc && G.row[a] < G.row[b]);
}
VLL_TIN_HD inline bool less_yx(const TinGraph &G, int a, int b) {
    const int ar = G.row[a], br = G.row[b];
    return ar < br || (ar == br && G.col[a] > G.col[b]);
}

// Orientation / InCircle (grid_triangulation.cpp:29-61) in 64-bit integers;
// the products wrap like the reference's (its 128-bit type is an alias of
// int64_t), computed unsigned to keep the wrap-around defined.
VLL_TIN_HD inline long long orient(const TinGraph &G, int a, int b, int c) {
    const unsigned long long d11 = (unsigned long long)(long long)(G.col[a] - G.col[c]);
    const unsigned long long d21 = (unsigned long long)(long long)(G.col[b] - G.col[c]);
    const unsigned long long d12 = (unsigned long long)(long long)(G.row[a] - G.row[c]);
    const unsigned long long d22 = (unsigned long long)(long long)(G.row[b] - G.row[c]);
    return (long long)(d11 * d22 - d12 * d21);
}

VLL_TIN_HD inline long long incircle(const TinGraph &G, int a, int b, int c, int d) {
    const long long d11 = (long long)(G.col[a] - G.col[d]), d12 = (long long)(G.row[a] - G.row[d]);
    const long long d21 = (long long)(G.col[b] - G.col[d]), d22 = (long long)(G.row[b] - G.row[d]);
    const long long d31 = (long long)(G.col[c] - G.col[d]), d32 = (long long)(G.row[c] - G.row[d]);
    typedef unsigned long long U;
    const U d13 = (U)d11 * (U)d11 + (U)d12 * (U)d12;
    const U d23 = (U)d21 * (U)d21 + (U)d22 * (U)d22;
    const U d33 = (U)d31 * (U)d31 + (U)d32 * (U)d32;
    const U bc = (U)d21 * (U)d32 - (U)d31 * (U)d22;
    const U ac = (U)d11 * (U)d32 - (U)d31 * (U)d12;
    const U ab = (U)d11 * (U)d22 - (U)d21 * (U)d12;
    return (long long)(d13 * bc - d23 * ac + d33 * ab);
}

// The node's slice of the allocator (EdgeList::GetNewEdge / RemoveEdge,
// edge_list.cpp:62-83): a stack of free edge indices at unused[base ...).
struct Alloc {
    int base, idx;
};

VLL_TIN_HD inline int new_edge(const TinGraph &G, Alloc &a) {
    a.idx--;
    return G.unused[a.base + a.idx];
}
VLL_TIN_HD inline void free_edge(const TinGraph &G, Alloc &a, int e) {
    G.unused[a.base + a.idx] = e;
    a.idx++;
}

// AddEdgeAndTwin, RemoveEdgeAndTwin, Weld, Bridge (grid_triangulation.cpp:
// 95-177), in the reference's statement order.
VLL_TIN_HD inline int add_edge_twin(const TinGraph &G, Alloc &a, int o, int d) {
    const int e = new_edge(G, a);
    const int et = new_edge(G, a);
    G.dnext[e] = et;
    G.oprev[e] = et;
    G.twin[e] = et;
    G.dnext[et] = e;
    G.oprev[et] = e;
    G.twin[et] = e;
    G.orig[e] = o;
    G.orig[et] = d;
    return e;
}

VLL_TIN_HD inline void remove_edge_twin(const TinGraph &G, Alloc &a, int e) {
    const int et = G.twin[e];
    G.dnext[G.oprev[e]] = G.dnext[et];
    G.oprev[G.dnext[e]] = G.oprev[et];
    G.dnext[G.oprev[et]] = G.dnext[e];
    G.oprev[G.dnext[et]] = G.oprev[e];
    free_edge(G, a, e);
    free_edge(G, a, et);
}

VLL_TIN_HD inline void weld(const TinGraph &G, int in, int out) {
    const int prev = G.oprev[out];
    G.oprev[out] = in;
    G.dnext[in] = out;
    G.oprev[G.twin[in]] = prev;
    G.dnext[prev] = G.twin[in];
}

VLL_TIN_HD inline int bridge(const TinGraph &G, Alloc &a, int start, int end) {
    const int o = G.orig[G.twin[start]];
    const int d = G.orig[end];
    const int e = add_edge_twin(G, a, o, d);
    const int et = G.twin[e];
    weld(G, et, G.dnext[start]);
    weld(G, e, end);
    return e;
}

// Walks in this file stop after this many steps (a well-formed structure
// never needs that many) and raise the error flag.
VLL_TIN_HD inline bool step_ok(const TinGraph &G, long long &steps, long long bound) {
    if (++steps <= bound) return true;
#ifdef __CUDA_ARCH__
    atomicExch(G.err, 1u);
#else
    *G.err = 1u;
#endif
    return false;
}

// NextCrossEdge (grid_triangulation.cpp:1287-1335): the next bridge of the
// merge zipper above `base`, or -1 at the upper common tangent.
VLL_TIN_HD inline int next_cross_edge(const TinGraph &G, Alloc &a, int base, long long &steps,
                               long long bound) {
    int l_cand = G.dnext[base];
    const bool valid_l = orient(G, G.orig[base], G.orig[l_cand], G.orig[G.twin[l_cand]]) < 0;
    if (valid_l) {
        int next_cand = G.dnext[G.twin[l_cand]];
        while (incircle(G, G.orig[l_cand], G.orig[base], G.orig[G.twin[l_cand]],
                        G.orig[G.twin[next_cand]]) > 0) {
            if (!step_ok(G, steps, bound)) return -1;
            remove_edge_twin(G, a, l_cand);
            l_cand = next_cand;
            next_cand = G.dnext[G.twin[l_cand]];
        }
    }
    int r_cand = G.twin[G.oprev[base]];
    const bool valid_r = orient(G, G.orig[G.twin[base]], G.orig[base], G.orig[G.twin[r_cand]]) > 0;
    if (valid_r) {
        int next_cand = G.twin[G.oprev[r_cand]];
        while (incircle(G, G.orig[G.twin[base]], G.orig[base], G.orig[G.twin[r_cand]],
                        G.orig[G.twin[next_cand]]) > 0) {
            if (!step_ok(G, steps, bound)) return -1;
            remove_edge_twin(G, a, r_cand);
            r_cand = next_cand;
            next_cand = G.twin[G.oprev[r_cand]];
        }
    }
    if (!valid_l && !valid_r) return -1;
    if (!valid_l || (valid_r && incircle(G, G.orig[G.twin[l_cand]], G.orig[l_cand],
                                         G.orig[r_cand], G.orig[G.twin[r_cand]]) > 0))
        return G.twin[bridge(G, a, base, G.twin[r_cand])];
    return G.twin[bridge(G, a, l_cand, base)];
}

// Triangulate2 / Triangulate3 (grid_triangulation.cpp:580-699) on the node's
// points in the order its parent sorted them.
VLL_TIN_HD inline void base_case(const TinGraph &G, TinNode &N, const int *perm, Alloc &a) {
    if (N.cnt == 2) {
        const int pa = perm[N.lo], pb = perm[N.lo + 1];
        const int e = add_edge_twin(G, a, pa, pb);
        if (less_xy(G, pa, pb)) {
            N.ex[EX_L] = e;
            N.ex[EX_R] = G.twin[e];
        } else {
            N.ex[EX_L] = G.twin[e];
            N.ex[EX_R] = e;
        }
        if (less_yx(G, pa, pb)) {
            N.ex[EX_B] = e;
            N.ex[EX_T] = G.twin[e];
        } else {
            N.ex[EX_B] = G.twin[e];
            N.ex[EX_T] = e;
        }
        return;
    }
    int p[3] = {perm[N.lo], perm[N.lo + 1], perm[N.lo + 2]};
    // sort the three by (col, row)
    for (int i = 1; i < 3; ++i)
        for (int j = i; j > 0 && less_xy(G, p[j], p[j - 1]); --j) {
            const int t = p[j];
            p[j] = p[j - 1];
            p[j - 1] = t;
        }
    int A = p[0], B = p[1], C = p[2];
    int e1 = add_edge_twin(G, a, A, B);
    int e2 = add_edge_twin(G, a, B, C);
    weld(G, e1, e2);
    int e3;
    long long s = orient(G, A, B, C);
    if (s > 0) {
        e3 = bridge(G, a, e2, e1);
        N.ex[EX_L] = e1;
        N.ex[EX_R] = G.twin[e2];
    } else if (s < 0) {
        e3 = bridge(G, a, e2, e1);
        N.ex[EX_L] = G.twin[e3];
        N.ex[EX_R] = e3;
    } else {
        N.ex[EX_L] = e1;
        N.ex[EX_R] = G.twin[e2];
    }
    // the same three by (row, -col)
    for (int i = 1; i < 3; ++i)
        for (int j = i; j > 0 && less_yx(G, p[j], p[j - 1]); --j) {
            const int t = p[j];
            p[j] = p[j - 1];
            p[j - 1] = t;
        }
    A = p[0];
    B = p[1];
    C = p[2];
    const int e = (G.orig[e1] == A) ? e1 : (G.orig[e2] == A ? e2 : G.twin[e2]);
    e1 = (G.orig[G.twin[e]] == B) ? e : G.dnext[G.twin[e]];
    e2 = G.dnext[e1];
    e3 = G.dnext[e2];
    s = orient(G, A, B, C);
    if (s >= 0) {
        N.ex[EX_B] = e1;
        N.ex[EX_T] = G.twin[e2];
    } else {
        N.ex[EX_B] = G.twin[e3];
        N.ex[EX_T] = e3;
    }
}

// The merge of a node's two triangulated halves
// (TriangulateHorizontalSerial / TriangulateVerticalSerial,
// grid_triangulation.cpp:417-578): common tangent, zipper, new extremes.
VLL_TIN_HD inline void merge_node(const TinGraph &G, TinNode *nodes, int ni, Alloc &a,
                                  long long bound) {
    TinNode &N = nodes[ni];
    TinNode &L = nodes[N.left];
    TinNode &R = nodes[N.right];
    long long steps = 0;
    if (N.horiz) {
        int le = L.ex[EX_R], re = R.ex[EX_L];
        for (;;) {
            if (!step_ok(G, steps, bound)) return;
            if (orient(G, G.orig[le], G.orig[G.twin[le]], G.orig[re]) > 0)
                le = G.twin[G.oprev[G.twin[le]]];
            else if (orient(G, G.orig[re], G.orig[G.twin[re]], G.orig[le]) < 0)
                re = G.dnext[re];
            else
                break;
        }
        const int lct = bridge(G, a, G.oprev[re], G.dnext[G.twin[le]]);
        if (G.orig[le] == G.orig[L.ex[EX_L]]) L.ex[EX_L] = G.twin[lct];
        if (G.orig[re] == G.orig[R.ex[EX_R]]) R.ex[EX_R] = lct;
        int nb = lct, uct = -1;
        while (nb != -1) {
            if (!step_ok(G, steps, bound)) return;
            uct = nb;
            nb = next_cross_edge(G, a, uct, steps, bound);
        }
        N.ex[EX_L] = L.ex[EX_L];
        N.ex[EX_R] = R.ex[EX_R];
        int t = G.twin[lct];
        while (less_yx(G, G.orig[t], G.orig[G.twin[t]]) && step_ok(G, steps, bound)) t = G.oprev[t];
        t = G.dnext[t];
        while (less_yx(G, G.orig[G.twin[t]], G.orig[t]) && step_ok(G, steps, bound)) t = G.dnext[t];
        N.ex[EX_B] = t;
        t = G.twin[uct];
        while (less_yx(G, G.orig[G.twin[t]], G.orig[t]) && step_ok(G, steps, bound))
            t = G.twin[G.dnext[G.twin[t]]];
        t = G.twin[G.oprev[G.twin[t]]];
        while (less_yx(G, G.orig[t], G.orig[G.twin[t]]) && step_ok(G, steps, bound))
            t = G.twin[G.oprev[G.twin[t]]];
        N.ex[EX_T] = t;
    } else {
        int be = L.ex[EX_T], te = R.ex[EX_B];
        for (;;) {
            if (!step_ok(G, steps, bound)) return;
            if (orient(G, G.orig[be], G.orig[G.twin[be]], G.orig[te]) > 0)
                be = G.twin[G.oprev[G.twin[be]]];
            else if (orient(G, G.orig[te], G.orig[G.twin[te]], G.orig[be]) < 0)
                te = G.dnext[te];
            else
                break;
        }
        const int rct = bridge(G, a, G.oprev[te], G.dnext[G.twin[be]]);
        if (G.orig[be] == G.orig[L.ex[EX_B]]) L.ex[EX_B] = G.twin[rct];
        if (G.orig[te] == G.orig[R.ex[EX_T]]) R.ex[EX_T] = rct;
        int nb = rct, lct = -1;
        while (nb != -1) {
            if (!step_ok(G, steps, bound)) return;
            lct = nb;
            nb = next_cross_edge(G, a, lct, steps, bound);
        }
        N.ex[EX_B] = L.ex[EX_B];
        N.ex[EX_T] = R.ex[EX_T];
        int t = rct;
        while (less_xy(G, G.orig[G.twin[t]], G.orig[t]) && step_ok(G, steps, bound))
            t = G.twin[G.dnext[G.twin[t]]];
        t = G.twin[G.oprev[G.twin[t]]];
        while (less_xy(G, G.orig[t], G.orig[G.twin[t]]) && step_ok(G, steps, bound))
            t = G.twin[G.oprev[G.twin[t]]];
        N.ex[EX_R] = t;
        t = lct;
        while (less_xy(G, G.orig[t], G.orig[G.twin[t]]) && step_ok(G, steps, bound)) t = G.oprev[t];
        t = G.dnext[t];
        while (less_xy(G, G.orig[G.twin[t]], G.orig[t]) && step_ok(G, steps, bound)) t = G.dnext[t];
        N.ex[EX_L] = t;
    }
}

// A subtree of fewer than 100 points (TriangulateHorizontalSerial /
// TriangulateVerticalSerial): the reference recurses without splitting its
// edge list, so the whole subtree draws from one allocator stack, children
// before parents, left before right.  `order` lists the subtree's nodes in
// that post-order; the stack is the subtree root's slice, fresh.
VLL_TIN_HD inline void serial_subtree(const TinGraph &G, TinNode *nodes, const int *order, int m,
                                      const int *perm, long long bound) {
    TinNode &root = nodes[order[m - 1]];
    Alloc a{6 * root.lo, 6 * root.cnt};
    for (int i = 0; i < m; ++i) {
        TinNode &N = nodes[order[i]];
        if (N.left < 0)
            base_case(G, N, perm, a);
        else
            merge_node(G, nodes, order[i], a, bound);
    }
    root.idx = a.idx;
}

// A node of 100 points or more (TriangulateHorizontalThreaded /
// TriangulateVerticalThreaded): its halves drew from split slices of its
// stack, which are concatenated (EdgeList::MergeEdgeLists) before the merge.
VLL_TIN_HD inline void threaded_merge(const TinGraph &G, TinNode *nodes, int ni, long long bound) {
    TinNode &N = nodes[ni];
    Alloc a{6 * N.lo, nodes[N.left].idx + nodes[N.right].idx};
    merge_node(G, nodes, ni, a, bound);
    N.idx = a.idx;
}

// The triangles around point p (Grid::GetAllTris, grid.cpp:16-51, and
// AdjTriIter, grid_iterators.hpp:63-110): counter-clockwise from the first
// face that is a triangle at or after its stored edge `e`, those of which p
// is the (col, row)-smallest vertex, passed to emit(q0, q1, q2).  Points of
// degree <= 2 whose edges are collinear have none.
template <class Emit>
VLL_TIN_HD inline void point_tris(const TinGraph &G, int e, long long bound, Emit emit) {
    if (e < 0) return;
    const int f = G.dnext[G.twin[G.dnext[G.twin[e]]]];
    const int p1 = G.orig[e], p2 = G.orig[G.twin[e]], p3 = G.orig[G.twin[G.dnext[G.twin[e]]]];
    const bool collinear = (G.col[p1] - G.col[p2]) * (G.row[p1] - G.row[p3]) ==
                           (G.row[p1] - G.row[p2]) * (G.col[p1] - G.col[p3]);
    if (f == e && collinear) return;
    long long steps = 0;
    int start = e;
    while (G.dnext[G.dnext[G.dnext[start]]] != start && step_ok(G, steps, bound))
        start = G.dnext[G.twin[start]];
    int cur = start;
    do {
        const int q0 = G.orig[cur], q1 = G.orig[G.dnext[cur]], q2 = G.orig[G.dnext[G.dnext[cur]]];
        if (less_xy(G, q0, q1) && less_xy(G, q0, q2)) emit(q0, q1, q2);
        cur = G.dnext[G.twin[cur]];
        while (G.dnext[G.dnext[G.dnext[cur]]] != cur && step_ok(G, steps, bound))
            cur = G.dnext[G.twin[cur]];
    } while (cur != start && step_ok(G, steps, bound));
}

}  // namespace tin
}  // namespace vll

// In-place sort of kd-tree split candidates with the exact permutation of
// the reference's std::sort, for host and device.
//
// kdTree_t::minimalCost (kdtree.cc:311-406) sorts its boundEdge array with
// std::sort, ordered by (position, end) only (boundEdge::operator<,
// kdtree.h:71-75).  Edges of different triangles often compare equal
// (shared vertices), and std::sort is not stable, so the order of equal
// edges — and with it the order of the triangles in the child lists and
// in every leaf below — is the one the reference's standard library
// produces.  That library (libstdc++ of the GCC that builds the
// reference) implements std::sort as Musser's introsort: median-of-three
// quicksort on ranges above 16 elements with a depth limit of
// 2*floor(log2 n), after which heapsort takes the range, then one
// insertion sort pass over the whole array.  This file restates that
// published algorithm step by step so a GPU build produces the same arrays
// as the host build, and the host build uses it too (its trees are pinned
// node for node against the reference's).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define YR_HD __host__ __device__ __forceinline__
#else
#define YR_HD inline
#endif

namespace yr {

struct KdEdge {
    float pos;
    int prim;
    int end;  // 0 lower, 1 both (flat), 2 upper (kdtree.cc:10-12)
};

YR_HD bool kd_edge_less(const KdEdge &a, const KdEdge &b) {
    if (a.pos == b.pos) return a.end < b.end;
    return a.pos < b.pos;
}

YR_HD void kd_swap(KdEdge &a, KdEdge &b) {
    KdEdge t = a;
    a = b;
    b = t;
}

// Sift `v` down from `hole` in the max-heap e[0, len), then back up towards
// the starting index (the two-phase heap adjustment of the SGI heap
// algorithms).
YR_HD void kd_heap_adjust(KdEdge *e, int hole, int len, KdEdge v) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (kd_edge_less(e[child], e[child - 1])) child--;
        e[hole] = e[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        e[hole] = e[child - 1];
        hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && kd_edge_less(e[parent], v)) {
        e[hole] = e[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    e[hole] = v;
}

// Heapsort of e[0, n): build the heap bottom-up, then move the maximum to
// the back one element at a time.
YR_HD void kd_heapsort(KdEdge *e, int n) {
    if (n < 2) return;
    for (int parent = (n - 2) / 2;; parent--) {
        kd_heap_adjust(e, parent, n, e[parent]);
        if (parent == 0) break;
    }
    for (int last = n - 1; last > 0; last--) {
        const KdEdge v = e[last];
        e[last] = e[0];
        kd_heap_adjust(e, 0, last, v);
    }
}

// Move the median of e[a], e[b], e[c] into e[r].
YR_HD void kd_median_to(KdEdge *e, int r, int a, int b, int c) {
    if (kd_edge_less(e[a], e[b])) {
        if (kd_edge_less(e[b], e[c])) kd_swap(e[r], e[b]);
        else if (kd_edge_less(e[a], e[c])) kd_swap(e[r], e[c]);
        else kd_swap(e[r], e[a]);
    } else if (kd_edge_less(e[a], e[c])) {
        kd_swap(e[r], e[a]);
    } else if (kd_edge_less(e[b], e[c])) {
        kd_swap(e[r], e[c]);
    } else {
        kd_swap(e[r], e[b]);
    }
}

// Hoare partition of e[lo, hi) around the pivot at e[p] (p < lo), without
// bounds checks: the median-of-three guarantees both scans stop.
YR_HD int kd_partition(KdEdge *e, int lo, int hi, int p) {
    for (;;) {
        while (kd_edge_less(e[lo], e[p])) ++lo;
        --hi;
        while (kd_edge_less(e[p], e[hi])) --hi;
        if (!(lo < hi)) return lo;
        kd_swap(e[lo], e[hi]);
        ++lo;
    }
}

// Insert e[i] into the sorted run to its left, knowing a smaller-or-equal
// element stops the scan.
YR_HD void kd_insert_unguarded(KdEdge *e, int i) {
    const KdEdge v = e[i];
    int j = i - 1;
    while (kd_edge_less(v, e[j])) {
        e[i] = e[j];
        i = j;
        --j;
    }
    e[i] = v;
}

YR_HD void kd_insertion_sort(KdEdge *e, int lo, int hi) {
    if (lo == hi) return;
    for (int i = lo + 1; i != hi; ++i) {
        if (kd_edge_less(e[i], e[lo])) {
            const KdEdge v = e[i];
            for (int j = i; j > lo; --j) e[j] = e[j - 1];
            e[lo] = v;
        } else {
            kd_insert_unguarded(e, i);
        }
    }
}

constexpr int kKdSortThreshold = 16;

// The quicksort phase on e[lo, hi): the right part of each partition is
// sorted before the left one, whose bounds wait on an explicit stack (the
// depth limit 2*log2 n keeps it below 64 entries for every 32-bit size).
// The parts are disjoint, so the order only matters for readability.
YR_HD void kd_introsort_loop(KdEdge *e, int lo, int hi, int depth) {
    int st_lo[64], st_hi[64], st_depth[64];
    int sp = 0;
    for (;;) {
        while (hi - lo > kKdSortThreshold) {
            if (depth == 0) {
                kd_heapsort(e + lo, hi - lo);
                break;
            }
            --depth;
            const int mid = lo + (hi - lo) / 2;
            kd_median_to(e, lo, lo + 1, mid, hi - 1);
            const int cut = kd_partition(e, lo + 1, hi, lo);
            st_lo[sp] = lo;
            st_hi[sp] = cut;
            st_depth[sp] = depth;
            ++sp;
            lo = cut;
        }
        if (sp == 0) return;
        --sp;
        lo = st_lo[sp];
        hi = st_hi[sp];
        depth = st_depth[sp];
    }
}

YR_HD int kd_floor_log2(int n) {
    int k = 0;
    while (n > 1) {
        n >>= 1;
        ++k;
    }
    return k;
}

YR_HD void kd_sort(KdEdge *e, int n) {
    if (n <= 0) return;
    kd_introsort_loop(e, 0, n, 2 * kd_floor_log2(n));
    if (n > kKdSortThreshold) {
        kd_insertion_sort(e, 0, kKdSortThreshold);
        for (int i = kKdSortThreshold; i < n; ++i) kd_insert_unguarded(e, i);
    } else {
        kd_insertion_sort(e, 0, n);
    }
}

}  // namespace yr

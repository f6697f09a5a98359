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

// The same edge in 8 bytes: triangle index << 2 | end.
struct KdEdge8 {
    float pos;
    uint32_t pe;
};

YR_HD bool kd_edge_less(const KdEdge &a, const KdEdge &b) {
    if (a.pos == b.pos) return a.end < b.end;
    return a.pos < b.pos;
}

YR_HD bool kd_edge_less(const KdEdge8 &a, const KdEdge8 &b) {
    if (a.pos == b.pos) return (a.pe & 3u) < (b.pe & 3u);
    return a.pos < b.pos;
}

// An array whose elements lie `s` apart (one thread's column of an
// interleaved shared-memory block).
template <class T>
struct KdStrided {
    T *p;
    int s;
    YR_HD T &operator[](int i) const { return p[(size_t)i * s]; }
    YR_HD KdStrided operator+(int k) const { return KdStrided{p + (size_t)k * s, s}; }
};

// The functions below take any array-like `E` (a pointer or KdStrided).
template <class E>
YR_HD void kd_swap_at(E e, int i, int j) {
    auto t = e[i];
    e[i] = e[j];
    e[j] = t;
}

// Sift `v` down from `hole` in the max-heap e[0, len), then back up towards
// the starting index (the two-phase heap adjustment of the SGI heap
// algorithms).
template <class E, class T>
YR_HD void kd_heap_adjust(E e, int hole, int len, T v) {
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
template <class E>
YR_HD void kd_heapsort(E e, int n) {
    if (n < 2) return;
    for (int parent = (n - 2) / 2;; parent--) {
        auto v = e[parent];
        kd_heap_adjust(e, parent, n, v);
        if (parent == 0) break;
    }
    for (int last = n - 1; last > 0; last--) {
        auto v = e[last];
        e[last] = e[0];
        kd_heap_adjust(e, 0, last, v);
    }
}

// Move the median of e[a], e[b], e[c] into e[r].
template <class E>
YR_HD void kd_median_to(E e, int r, int a, int b, int c) {
    if (kd_edge_less(e[a], e[b])) {
        if (kd_edge_less(e[b], e[c])) kd_swap_at(e, r, b);
        else if (kd_edge_less(e[a], e[c])) kd_swap_at(e, r, c);
        else kd_swap_at(e, r, a);
    } else if (kd_edge_less(e[a], e[c])) {
        kd_swap_at(e, r, a);
    } else if (kd_edge_less(e[b], e[c])) {
        kd_swap_at(e, r, c);
    } else {
        kd_swap_at(e, r, b);
    }
}

// Hoare partition of e[lo, hi) around the pivot at e[p] (p < lo), without
// bounds checks: the median-of-three guarantees both scans stop.
template <class E>
YR_HD int kd_partition(E e, int lo, int hi, int p) {
    for (;;) {
        while (kd_edge_less(e[lo], e[p])) ++lo;
        --hi;
        while (kd_edge_less(e[p], e[hi])) --hi;
        if (!(lo < hi)) return lo;
        kd_swap_at(e, lo, hi);
        ++lo;
    }
}

// Insert e[i] into the sorted run to its left, knowing a smaller-or-equal
// element stops the scan.
template <class E>
YR_HD void kd_insert_unguarded(E e, int i) {
    const auto v = e[i];
    int j = i - 1;
    while (kd_edge_less(v, e[j])) {
        e[i] = e[j];
        i = j;
        --j;
    }
    e[i] = v;
}

template <class E>
YR_HD void kd_insertion_sort(E e, int lo, int hi) {
    if (lo == hi) return;
    for (int i = lo + 1; i != hi; ++i) {
        if (kd_edge_less(e[i], e[lo])) {
            const auto v = e[i];
            for (int j = i; j > lo; --j) e[j] = e[j - 1];
            e[lo] = v;
        } else {
            kd_insert_unguarded(e, i);
        }
    }
}

constexpr int kKdSortThreshold = 16;

// The quicksort phase on e[lo, hi): the right part of each partition is
// sorted before the left one, whose bounds wait on an explicit stack.  Each
// entry uses up one level of the depth limit 2*floor(log2 n), so kCap
// entries serve every n below 2^(kCap/2 + 1) (16 entries: n <= 511).
// The parts are disjoint, so the order only matters for readability.
template <int kCap, class E>
YR_HD void kd_introsort_loop(E e, int lo, int hi, int depth) {
    int st_lo[kCap], st_hi[kCap], st_depth[kCap];
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

template <int kCap = 64, class E>
YR_HD void kd_sort(E e, int n) {
    if (n <= 0) return;
    kd_introsort_loop<kCap>(e, 0, n, 2 * kd_floor_log2(n));
    if (n > kKdSortThreshold) {
        kd_insertion_sort(e, 0, kKdSortThreshold);
        for (int i = kKdSortThreshold; i < n; ++i) kd_insert_unguarded(e, i);
    } else {
        kd_insertion_sort(e, 0, n);
    }
}

}  // namespace yr

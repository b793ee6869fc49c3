// The unstable sort of the reference's dissection (src/sparse.rs:108,
// `set.sort_unstable_by(coordinate)`): Rust's `slice::sort_unstable_by`, which since
// Rust 1.81 is ipnsort (core::slice::sort::unstable). Equal coordinates are common in
// meshes (whole planes of nodes), and the order this sort leaves them in is the node
// order inside the fronts, so the product restates that algorithm step for step for
// the element type the reference sorts (usize: 8 bytes, Copy, so the small sorts are
// the sorting-network variant):
//
//  * n <= 20: insertion sort;
//  * a whole-slice run (non-descending, or strictly descending and then reversed)
//    is left as it is;
//  * else quicksort with an imbalance budget of 2·⌊log2(n | 1)⌋ partitions (heapsort
//    once it is spent): pivot = median of three (recursive pseudo-median of nine
//    from 64 elements) at offsets 0, 4·⌊n/8⌋, 7·⌊n/8⌋; a pivot not greater than the
//    previous pivot of the slice splits off the elements equal to it instead;
//    partition = cyclic branchless Lomuto; slices of at most 32 elements go to the
//    small sort: the optimal 9- or 13-input network plus insertion sort, on two
//    halves merged (stably) from 18 elements.
//
// The quicksort's two sides are independent once partitioned, so `fork` may sort the
// left side on another thread: the result is the same element for element.
#pragma once

#include <algorithm>
#include <cstdint>
#include <future>
#include <utility>

namespace rfg {
namespace unstable_sort {

constexpr int64_t ALWAYS_INSERTION = 20;
constexpr int64_t SMALL = 32;
constexpr int64_t NO_MERGE = 18;
constexpr int64_t PSEUDO_MEDIAN = 64;

// compare-exchange pairs of the optimal 9-input (25) and 13-input (45) networks, in order
constexpr uint8_t kNet9[25][2] = {{0, 3}, {1, 7}, {2, 5}, {4, 8}, {0, 7}, {2, 4}, {3, 8}, {5, 6}, {0, 2},
                                  {1, 3}, {4, 5}, {7, 8}, {1, 4}, {3, 6}, {5, 7}, {0, 1}, {2, 4}, {3, 5},
                                  {6, 8}, {2, 3}, {4, 5}, {6, 7}, {1, 2}, {3, 4}, {5, 6}};
constexpr uint8_t kNet13[45][2] = {
    {0, 12}, {1, 10}, {2, 9},  {3, 7},   {5, 11}, {6, 8},  {1, 6},  {2, 3},  {4, 11}, {7, 9},  {8, 10}, {0, 4},
    {1, 2},  {3, 6},  {7, 8},  {9, 10},  {11, 12}, {4, 6},  {5, 9},  {8, 11}, {10, 12}, {0, 5}, {3, 8},  {4, 7},
    {6, 11}, {9, 10}, {0, 1},  {2, 5},   {6, 9},  {7, 8},  {10, 11}, {1, 3},  {2, 4},  {5, 6},  {9, 10}, {1, 2},
    {3, 4},  {5, 7},  {6, 8},  {2, 3},   {4, 5},  {6, 7},  {8, 9},  {3, 4},  {5, 6}};

template <class T, class Less>
inline void insertion(T* v, int64_t n, int64_t sorted, const Less& lt) {
    for (int64_t i = std::max<int64_t>(sorted, 1); i < n; i++) {
        if (!lt(v[i], v[i - 1])) continue;
        const T x = v[i];
        int64_t j = i - 1;
        v[i] = v[j];
        while (j > 0 && lt(x, v[j - 1])) {
            v[j] = v[j - 1];
            j--;
        }
        v[j] = x;
    }
}

template <class T, class Less, int N>
inline void network(T* v, const uint8_t (&net)[N][2], const Less& lt) {
    for (int e = 0; e < N; e++) {
        const T a = v[net[e][0]], b = v[net[e][1]];
        const bool sw = lt(b, a);
        v[net[e][0]] = sw ? b : a;
        v[net[e][1]] = sw ? a : b;
    }
}

template <class T, class Less>
inline void small_region(T* v, int64_t n, const Less& lt) {
    if (n >= 13) {
        network(v, kNet13, lt);
        insertion(v, n, 13, lt);
    } else if (n >= 9) {
        network(v, kNet9, lt);
        insertion(v, n, 9, lt);
    } else {
        insertion(v, n, 1, lt);
    }
}

template <class T, class Less>
inline void small_sort(T* v, int64_t n, const Less& lt) {
    if (n < 2) return;
    if (n < NO_MERGE) {
        small_region(v, n, lt);
        return;
    }
    const int64_t h = n / 2;
    small_region(v, h, lt);
    small_region(v + h, n - h, lt);
    // the bidirectional merge fills the output from both ends, the front taking the left
    // element on ties and the back the right one: together the stable merge
    T m[SMALL];
    int64_t i = 0, j = h, k = 0;
    while (i < h && j < n) {
        const bool right = lt(v[j], v[i]);
        m[k++] = right ? v[j] : v[i];
        j += right;
        i += !right;
    }
    while (i < h) m[k++] = v[i++];
    while (j < n) m[k++] = v[j++];
    std::copy(m, m + n, v);
}

template <class T, class Less>
inline void heap_sort(T* v, int64_t n, const Less& lt) {
    auto sift_down = [&](int64_t node, int64_t len) {
        for (int64_t c = 2 * node + 1; c < len; c = 2 * node + 1) {
            if (c + 1 < len) c += lt(v[c], v[c + 1]);
            if (!lt(v[node], v[c])) break;
            std::swap(v[node], v[c]);
            node = c;
        }
    };
    for (int64_t i = n + n / 2 - 1; i >= 0; i--) {
        if (i >= n) {
            sift_down(i - n, n);
        } else {
            std::swap(v[0], v[i]);
            sift_down(0, i);
        }
    }
}

template <class T, class Less>
inline const T* median3(const T* a, const T* b, const T* c, const Less& lt) {
    const bool x = lt(*a, *b);
    if (x != lt(*a, *c)) return a;
    return (lt(*b, *c) ^ x) ? c : b;
}

template <class T, class Less>
inline const T* median3_rec(const T* a, const T* b, const T* c, int64_t m, const Less& lt) {
    if (m * 8 >= PSEUDO_MEDIAN) {
        const int64_t m8 = m / 8;
        a = median3_rec(a, a + 4 * m8, a + 7 * m8, m8, lt);
        b = median3_rec(b, b + 4 * m8, b + 7 * m8, m8, lt);
        c = median3_rec(c, c + 4 * m8, c + 7 * m8, m8, lt);
    }
    return median3(a, b, c, lt);
}

template <class T, class Less>
inline int64_t pivot_index(const T* v, int64_t n, const Less& lt) {
    const int64_t n8 = n / 8;
    const T* p = n < PSEUDO_MEDIAN ? median3(v, v + 4 * n8, v + 7 * n8, lt) : median3_rec(v, v + 4 * n8, v + 7 * n8, n8, lt);
    return p - v;
}

// Pivot to v[0]; then each element of v[1..n) in turn, v[1] last, is written at the end of
// the block of elements that pass, and the element it displaces moves into the slot the
// previous one left; the pivot goes between the blocks. Returns the size of the block.
template <class T, class Pass>
inline int64_t partition(T* v, int64_t n, int64_t p, const Pass& pass) {
    std::swap(v[0], v[p]);
    const T piv = v[0];
    T* w = v + 1;
    const int64_t m = n - 1;
    int64_t k = 0;
    if (m > 0) {
        const T held = w[0];
        T* hole = w;
        for (int64_t r = 1; r < m; r++) {
            const T x = w[r];
            const bool ok = pass(x, piv);
            *hole = w[k];
            w[k] = x;
            hole = w + r;
            k += ok;
        }
        const bool ok = pass(held, piv);
        *hole = w[k];
        w[k] = held;
        k += ok;
    }
    std::swap(v[0], v[k]);
    return k;
}

// Fork policy: take(n) true = sort a side of n elements on another thread, then give()
struct NoFork {
    bool take(int64_t) { return false; }
    void give() {}
};

template <class T, class Less, class Fork>
void quicksort(T* v, int64_t n, const T* anc, uint32_t limit, const Less& lt, Fork& fork) {
    std::future<void> left;
    for (;;) {
        if (n <= SMALL) {
            small_sort(v, n, lt);
            break;
        }
        if (limit == 0) {
            heap_sort(v, n, lt);
            break;
        }
        limit--;
        const int64_t p = pivot_index(v, n, lt);
        if (anc && !lt(*anc, v[p])) {
            const int64_t k = partition(v, n, p, [&](const T& a, const T& b) { return !lt(b, a); });
            v += k + 1;
            n -= k + 1;
            anc = nullptr;
            continue;
        }
        const int64_t k = partition(v, n, p, lt);
        if (!left.valid() && fork.take(k)) {
            left = std::async(std::launch::async, [=, &lt, &fork] { quicksort(v, k, anc, limit, lt, fork); });
        } else {
            quicksort(v, k, anc, limit, lt, fork);
        }
        anc = v + k;
        v += k + 1;
        n -= k + 1;
    }
    if (left.valid()) {
        left.get();
        fork.give();
    }
}

// v.sort_unstable_by(lt) on v[0..n); limit >= 0 replaces the imbalance budget
template <class T, class Less, class Fork = NoFork>
void sort(T* v, int64_t n, const Less& lt, Fork&& fork = Fork(), int64_t limit = -1) {
    if (n < 2) return;
    if (n <= ALWAYS_INSERTION) {
        insertion(v, n, 1, lt);
        return;
    }
    const bool desc = lt(v[1], v[0]);
    int64_t run = 2;
    if (desc)
        while (run < n && lt(v[run], v[run - 1])) run++;
    else
        while (run < n && !lt(v[run], v[run - 1])) run++;
    if (run == n) {
        if (desc) std::reverse(v, v + n);
        return;
    }
    uint32_t lg = 0;
    for (uint64_t t = (uint64_t)n | 1; t > 1; t >>= 1) lg++;
    quicksort(v, n, (const T*)nullptr, limit >= 0 ? (uint32_t)limit : 2 * lg, lt, fork);
}

}  // namespace unstable_sort
}  // namespace rfg

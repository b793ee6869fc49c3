// ============================================================================
// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of RustyFEM's multifrontal sparse LDLᵀ (the reference's
// src/sparse.rs, src/sparse/indef.rs, src/solver/indefinite.rs and the C
// interface ffi/src/lib.rs), used as the checker for the GPU library and as
// the timed CPU baseline. Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline / reference arm load it. The product library never links it.
//
// Each function cites the reference file:line it follows. Arithmetic order is
// kept where it decides rounding: `dot` keeps its 8 partial sums, the dense
// kernels use fused multiply-add exactly where the reference calls mul_add
// (chosen at run time from the CPU's AVX2+FMA support, src/sparse.rs:387-442),
// and everything else is compiled with -ffp-contract=off so that no other
// operation is fused.
//
// Parity status of this restatement:
//  * pinned against the reference's own known answers: the 40-DOF chain test
//    (ffi/src/lib.rs:429-478), the 4×4 indefinite test
//    (src/steps/nlgeom_solver.rs:145-175) and the Laplacian inertia check
//    (examples/solver_bench.rs:87-157), all under tests/;
//  * tree shape (front membership, k, u, children, work) is independent of
//    sort ties and is checked against front statistics computed from an
//    independent restatement of src/sparse.rs:78-232;
//  * the order of nodes INSIDE a front follows the tie order of Rust's
//    `slice::sort_unstable_by` (src/sparse.rs:108), restated below (rsort) for
//    the standard library's ipnsort (Rust 1.81 and later) and checked on
//    hand-traced tie cases; with no rustc and no dump of the reference's
//    permutation here, that part of the permutation is "parity unpinned".
// ============================================================================

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <condition_variable>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace oref {

using std::size_t;
using std::vector;

static const size_t NONE = std::numeric_limits<size_t>::max();
static int g_threads = 0;  // 0 = hardware concurrency (src/par.rs:3-5)

static size_t threads() {
    if (g_threads > 0) return (size_t)g_threads;
    unsigned t = std::thread::hardware_concurrency();
    return t ? t : 1;
}

// ---------------------------------------------------------------------------
// src/par.rs:44-77 — contiguous row blocks of about equal cost, one scoped
// thread per block.
// ---------------------------------------------------------------------------
static void blocks_mut(size_t nrows, size_t nthreads, const std::function<double(size_t)>& cost,
                       const std::function<void(size_t, size_t)>& f /* (first row, number of rows) */) {
    size_t t = std::max<size_t>(std::min(nthreads, nrows), 1);
    if (t == 1) {
        f(0, nrows);
        return;
    }
    double total = 0.0;
    for (size_t r = 0; r < nrows; r++) total += cost(r);
    vector<size_t> bounds{0};
    double acc = 0.0;
    for (size_t r = 0; r < nrows; r++) {
        acc += cost(r);
        if (acc >= total * (double)bounds.size() / (double)t && bounds.size() < t) bounds.push_back(r + 1);
    }
    bounds.push_back(nrows);
    bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
    vector<std::thread> th;
    for (size_t i = 0; i + 1 < bounds.size(); i++) {
        size_t r0 = bounds[i], nr = bounds[i + 1] - bounds[i];
        th.emplace_back([&f, r0, nr] { f(r0, nr); });
    }
    for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------
// Symbolic analysis — src/sparse.rs:18-36, 78-275
// ---------------------------------------------------------------------------
struct TNode {
    vector<size_t> nodes, children;
    size_t start = 0, k = 0;
    vector<size_t> rows;
    double work = 0.0;
};

struct Symbolic {
    vector<TNode> tree;
    vector<size_t> roots;
    vector<size_t> first_dof;
    size_t n = 0;
};

typedef vector<vector<size_t>> Adj;

// ---------------------------------------------------------------------------
// src/sparse.rs:108 sorts with Rust's `slice::sort_unstable_by`: the standard
// library's unstable sort since Rust 1.81 (core::slice::sort::unstable, "ipnsort"),
// here for the element the reference sorts (usize: 8 bytes, Copy), whose small
// sorts are the sorting-network variant. Restated from the algorithm's published
// description; what matters is where it leaves equal keys.
namespace rsort {

template <class T, class L>
static void insert_from(T* v, size_t n, size_t start, L& lt) {  // insertion_sort_shift_left
    for (size_t i = std::max<size_t>(start, 1); i < n; i++) {
        T x = v[i];
        size_t j = i;
        while (j > 0 && lt(x, v[j - 1])) {
            v[j] = v[j - 1];
            j--;
        }
        v[j] = x;
    }
}

// optimal 9- and 13-input networks; (a, b) exchanges when v[b] < v[a]
static const uint8_t NET9[25][2] = {{0, 3}, {1, 7}, {2, 5}, {4, 8}, {0, 7}, {2, 4}, {3, 8}, {5, 6}, {0, 2},
                                    {1, 3}, {4, 5}, {7, 8}, {1, 4}, {3, 6}, {5, 7}, {0, 1}, {2, 4}, {3, 5},
                                    {6, 8}, {2, 3}, {4, 5}, {6, 7}, {1, 2}, {3, 4}, {5, 6}};
static const uint8_t NET13[45][2] = {{0, 12}, {1, 10}, {2, 9},  {3, 7},  {5, 11}, {6, 8},  {1, 6},  {2, 3},  {4, 11},
                                     {7, 9},  {8, 10}, {0, 4},  {1, 2},  {3, 6},  {7, 8},  {9, 10}, {11, 12}, {4, 6},
                                     {5, 9},  {8, 11}, {10, 12}, {0, 5}, {3, 8},  {4, 7},  {6, 11}, {9, 10}, {0, 1},
                                     {2, 5},  {6, 9},  {7, 8},  {10, 11}, {1, 3}, {2, 4},  {5, 6},  {9, 10}, {1, 2},
                                     {3, 4},  {5, 7},  {6, 8},  {2, 3},  {4, 5},  {6, 7},  {8, 9},  {3, 4},  {5, 6}};

template <class T, class L>
static void region(T* v, size_t n, L& lt) {
    size_t pre = 1;
    if (n >= 13) {
        for (auto& e : NET13)
            if (lt(v[e[1]], v[e[0]])) std::swap(v[e[0]], v[e[1]]);
        pre = 13;
    } else if (n >= 9) {
        for (auto& e : NET9)
            if (lt(v[e[1]], v[e[0]])) std::swap(v[e[0]], v[e[1]]);
        pre = 9;
    }
    insert_from(v, n, pre, lt);
}

template <class T, class L>
static void small_sort(T* v, size_t n, L& lt) {  // small_sort_network, n <= 32
    if (n < 2) return;
    if (n < 18) {
        region(v, n, lt);
        return;
    }
    const size_t h = n / 2;
    region(v, h, lt);
    region(v + h, n - h, lt);
    T out[32];  // the two ends of the bidirectional merge meet in the stable merge
    size_t i = 0, j = h, k = 0;
    while (i < h && j < n) out[k++] = lt(v[j], v[i]) ? v[j++] : v[i++];
    while (i < h) out[k++] = v[i++];
    while (j < n) out[k++] = v[j++];
    std::copy(out, out + n, v);
}

template <class T, class L>
static void heapsort(T* v, size_t n, L& lt) {
    auto sift = [&](size_t node, size_t end) {
        for (;;) {
            size_t c = 2 * node + 1;
            if (c >= end) return;
            if (c + 1 < end && lt(v[c], v[c + 1])) c++;
            if (!lt(v[node], v[c])) return;
            std::swap(v[node], v[c]);
            node = c;
        }
    };
    for (size_t i = n + n / 2; i-- > 0;) {
        if (i >= n) {
            sift(i - n, n);
        } else {
            std::swap(v[0], v[i]);
            sift(0, i);
        }
    }
}

template <class T, class L>
static size_t median3(const T* v, size_t a, size_t b, size_t c, L& lt) {
    const bool x = lt(v[a], v[b]), y = lt(v[a], v[c]);
    if (x != y) return a;
    return (lt(v[b], v[c]) != x) ? c : b;
}

template <class T, class L>
static size_t median3_rec(const T* v, size_t a, size_t b, size_t c, size_t m, L& lt) {
    if (m * 8 >= 64) {
        const size_t m8 = m / 8;
        a = median3_rec(v, a, a + 4 * m8, a + 7 * m8, m8, lt);
        b = median3_rec(v, b, b + 4 * m8, b + 7 * m8, m8, lt);
        c = median3_rec(v, c, c + 4 * m8, c + 7 * m8, m8, lt);
    }
    return median3(v, a, b, c, lt);
}

// pivot to v[0]; cyclic Lomuto over v[1..n): every element in turn is written at the end
// of the block of elements that pass `pass`, the element it displaces goes to the hole
// it left, v[1] last; then the pivot goes between the blocks. Returns the passing count.
template <class T, class P>
static size_t partition(T* v, size_t n, size_t p, P pass) {
    std::swap(v[0], v[p]);
    const T piv = v[0];
    T* w = v + 1;
    const size_t m = n - 1;
    size_t cnt = 0;
    if (m > 0) {
        const T first = w[0];
        size_t hole = 0;
        for (size_t r = 1; r <= m; r++) {
            const T x = r == m ? first : w[r];
            const bool ok = pass(x, piv);
            w[hole] = w[cnt];
            w[cnt] = x;
            hole = r;
            cnt += ok;
        }
    }
    std::swap(v[0], v[cnt]);
    return cnt;
}

template <class T, class L>
static void quicksort(T* v, size_t n, const T* anc, uint32_t limit, L& lt) {
    for (;;) {
        if (n <= 32) {
            small_sort(v, n, lt);
            return;
        }
        if (limit == 0) {
            heapsort(v, n, lt);
            return;
        }
        limit--;
        const size_t n8 = n / 8;
        const size_t p = n < 64 ? median3(v, 0, 4 * n8, 7 * n8, lt) : median3_rec(v, 0, 4 * n8, 7 * n8, n8, lt);
        if (anc && !lt(*anc, v[p])) {
            const size_t nle = partition(v, n, p, [&](const T& a, const T& b) { return !lt(b, a); });
            v += nle + 1;
            n -= nle + 1;
            anc = nullptr;
            continue;
        }
        const size_t nlt = partition(v, n, p, lt);
        quicksort(v, nlt, anc, limit, lt);
        anc = v + nlt;
        v += nlt + 1;
        n -= nlt + 1;
    }
}

// slice::sort_unstable_by; limit >= 0 replaces the imbalance budget 2·⌊log2(n | 1)⌋
template <class T, class L>
static void sort_unstable(T* v, size_t n, L lt, long limit = -1) {
    if (n < 2) return;
    if (n <= 20) {
        insert_from(v, n, 1, lt);
        return;
    }
    const bool desc = lt(v[1], v[0]);
    size_t run = 2;
    while (run < n && (desc ? lt(v[run], v[run - 1]) : !lt(v[run], v[run - 1]))) run++;
    if (run == n) {
        if (desc) std::reverse(v, v + n);
        return;
    }
    uint32_t lg = 0;
    for (size_t t = n | 1; t > 1; t >>= 1) lg++;
    quicksort(v, n, (const T*)nullptr, limit >= 0 ? (uint32_t)limit : 2 * lg, lt);
}

}  // namespace rsort

// src/sparse.rs:78-157
static long dissect(vector<size_t> set, const double* coords, const Adj& adj, vector<uint8_t>& side, vector<TNode>& tree,
                    size_t leaf_max) {
    if (set.empty()) return -1;
    if (set.size() <= leaf_max) {
        TNode t;
        t.nodes = std::move(set);
        tree.push_back(std::move(t));
        return (long)tree.size() - 1;
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t v : set)
        for (int a = 0; a < 3; a++) {
            lo[a] = std::fmin(lo[a], coords[3 * v + a]);
            hi[a] = std::fmax(hi[a], coords[3 * v + a]);
        }
    // :100-101 stable sort of the axes by decreasing extent (the longest first, ties keep 0,1,2)
    int axes[3] = {0, 1, 2};
    std::stable_sort(axes, axes + 3, [&](int a, int b) { return (hi[a] - lo[a]) > (hi[b] - lo[b]); });
    size_t n = set.size();
    bool have = false;
    double bscore = 0.0, bt = 0.0;
    int bax = 0;
    bool bleft = true;
    for (int ax : axes) {
        if (!(hi[ax] > lo[ax])) continue;
        // :108 set.sort_unstable_by(coordinate ax)
        rsort::sort_unstable(set.data(), set.size(),
                             [&](size_t a, size_t b) { return coords[3 * a + ax] < coords[3 * b + ax]; });
        const size_t qs[3] = {n / 2, 2 * n / 5, 3 * n / 5};
        for (size_t q : qs) {
            double t = coords[3 * set[q] + ax];
            // :112 partition_point
            size_t nl = (size_t)(std::lower_bound(set.begin(), set.end(), t,
                                                  [&](size_t v, double tv) { return coords[3 * v + ax] < tv; }) -
                                 set.begin());
            if (nl == 0 || nl == n) continue;
            for (size_t i = 0; i < n; i++) side[set[i]] = (uint8_t)(i >= nl);
            size_t sep_l = 0, sep_r = 0;
            for (size_t i = 0; i < nl; i++) {
                size_t v = set[i];
                for (size_t w : adj[v])
                    if (side[w] == 1) {
                        sep_l++;
                        break;
                    }
            }
            for (size_t i = nl; i < n; i++) {
                size_t v = set[i];
                for (size_t w : adj[v])
                    if (side[w] == 0) {
                        sep_r++;
                        break;
                    }
            }
            size_t s;
            bool in_left;
            if (sep_r < sep_l) {
                s = sep_r;
                in_left = false;
            } else {
                s = sep_l;
                in_left = true;
            }
            double score = (double)s / ((double)std::min(nl, n - nl) / (double)n);
            if (!have || score < bscore) {
                have = true;
                bscore = score;
                bax = ax;
                bt = t;
                bleft = in_left;
            }
        }
    }
    vector<size_t> left, right;
    if (have) {
        for (size_t v : set) (coords[3 * v + bax] < bt ? left : right).push_back(v);
    } else {
        left.assign(set.begin(), set.begin() + n / 2);
        right.assign(set.begin() + n / 2, set.end());
    }
    bool in_left = have ? bleft : true;
    for (size_t v : left) side[v] = 0;
    for (size_t v : right) side[v] = 1;
    vector<size_t> sep, a, b;
    auto touches = [&](size_t v, uint8_t other) {
        for (size_t w : adj[v])
            if (side[w] == other) return true;
        return false;
    };
    if (in_left) {
        for (size_t v : left) (touches(v, 1) ? sep : a).push_back(v);
        b = right;
    } else {
        for (size_t v : right) (touches(v, 0) ? sep : b).push_back(v);
        a = left;
    }
    for (size_t v : left) side[v] = 2;
    for (size_t v : right) side[v] = 2;
    left.clear();
    left.shrink_to_fit();
    right.clear();
    right.shrink_to_fit();
    vector<size_t> children;
    long ca = dissect(std::move(a), coords, adj, side, tree, leaf_max);
    long cb = dissect(std::move(b), coords, adj, side, tree, leaf_max);
    if (ca >= 0) children.push_back((size_t)ca);
    if (cb >= 0) children.push_back((size_t)cb);
    TNode t;
    t.nodes = std::move(sep);
    t.children = std::move(children);
    tree.push_back(std::move(t));
    return (long)tree.size() - 1;
}

// src/sparse.rs:167-232
static Symbolic* analyse_with_leaf(size_t nn, const double* coords, const Adj& adj, const size_t* ndof, size_t leaf_max) {
    leaf_max = std::max<size_t>(leaf_max, 1);
    Symbolic* s = new Symbolic();
    vector<uint8_t> side(nn, 2);
    vector<size_t> all(nn);
    for (size_t i = 0; i < nn; i++) all[i] = i;
    long r = dissect(std::move(all), coords, adj, side, s->tree, leaf_max);
    if (r >= 0) s->roots.push_back((size_t)r);
    auto& tree = s->tree;
    // postorder via an explicit stack (:176-187)
    vector<size_t> post;
    post.reserve(tree.size());
    vector<std::pair<size_t, bool>> stack;
    for (size_t rt : s->roots) stack.push_back({rt, false});
    while (!stack.empty()) {
        auto [t, done] = stack.back();
        stack.pop_back();
        if (done) {
            post.push_back(t);
        } else {
            stack.push_back({t, true});
            for (size_t i = tree[t].children.size(); i-- > 0;) stack.push_back({tree[t].children[i], false});
        }
    }
    s->first_dof.assign(nn, 0);
    size_t next = 0;
    for (size_t t : post) {
        tree[t].start = next;
        for (size_t v : tree[t].nodes) {
            s->first_dof[v] = next;
            next += ndof[v];
        }
        tree[t].k = next - tree[t].start;
    }
    // front pattern (:201-230)
    vector<vector<size_t>> unodes(tree.size());
    vector<size_t> stamp(nn, NONE);
    for (size_t t : post) {
        size_t end = tree[t].start + tree[t].k;
        vector<size_t> list;
        auto take = [&](size_t w) {
            if (s->first_dof[w] >= end && stamp[w] != t) {
                stamp[w] = t;
                list.push_back(w);
            }
        };
        for (size_t v : tree[t].nodes)
            for (size_t w : adj[v]) take(w);
        for (size_t c : tree[t].children)
            for (size_t w : unodes[c]) take(w);
        std::sort(list.begin(), list.end(), [&](size_t a, size_t b) { return s->first_dof[a] < s->first_dof[b]; });
        tree[t].rows.clear();
        for (size_t w : list)
            for (size_t q = s->first_dof[w]; q < s->first_dof[w] + ndof[w]; q++) tree[t].rows.push_back(q);
        double k = (double)tree[t].k, u = (double)tree[t].rows.size();
        double own = k * k * k / 3.0 + u * k * k + u * u * k;
        double cw = 0.0;
        for (size_t c : tree[t].children) cw += tree[c].work;
        tree[t].work = own + cw;
        unodes[t] = std::move(list);
    }
    s->n = next;
    return s;
}

// src/sparse.rs:236-238
static double sym_work(const Symbolic* s) {
    double w = 0.0;
    for (size_t r : s->roots) w += s->tree[r].work;
    return w;
}
// :241-243
static size_t sym_factor_size(const Symbolic* s) {
    size_t z = 0;
    for (auto& t : s->tree) z += t.k * (t.k ? t.k - 1 : 0) / 2 + t.k * t.rows.size();
    return z;
}

// ---------------------------------------------------------------------------
// src/sparse.rs:39-56, 256-275 — lower triangle in column format
// ---------------------------------------------------------------------------
struct Lower {
    vector<size_t> colptr, rowidx;
    vector<double> val;
    void add(size_t r, size_t c, double v) {
        size_t lo = colptr[c], hi = colptr[c + 1];
        auto it = std::lower_bound(rowidx.begin() + lo, rowidx.begin() + hi, r);
        if (it == rowidx.begin() + hi || *it != r) {
            fprintf(stderr, "oracle: entry (%zu, %zu) missing in the pattern\n", r, c);
            abort();
        }
        val[(size_t)(it - rowidx.begin())] += v;
    }
    double diag(size_t c) const { return val[colptr[c]]; }
};

static Lower* sym_pattern(const Symbolic* s, const Adj& adj, const size_t* ndof) {
    Lower* L = new Lower();
    L->colptr.assign(s->n + 1, 0);
    size_t nn = adj.size();
    vector<size_t> order(nn);
    for (size_t i = 0; i < nn; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return s->first_dof[a] < s->first_dof[b]; });
    for (size_t v : order) {
        vector<size_t> nb(adj[v]);
        nb.push_back(v);
        std::sort(nb.begin(), nb.end(), [&](size_t a, size_t b) { return s->first_dof[a] < s->first_dof[b]; });
        size_t f = s->first_dof[v];
        for (size_t c = f; c < f + ndof[v]; c++) {
            for (size_t w : nb) {
                size_t fw = s->first_dof[w];
                for (size_t r = fw; r < fw + ndof[w]; r++)
                    if (r >= c) L->rowidx.push_back(r);
            }
            L->colptr[c + 1] = L->rowidx.size();
        }
    }
    L->val.assign(L->rowidx.size(), 0.0);
    return L;
}

// ---------------------------------------------------------------------------
// src/sparse.rs:58-76 — dot with 8 partial sums
// ---------------------------------------------------------------------------
static double dot(const double* a, const double* b, size_t n) {
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t n8 = n / 8 * 8;
    for (size_t i = 0; i < n8; i += 8)
        for (int l = 0; l < 8; l++) s[l] += a[i + l] * b[i + l];
    double t = (s[0] + s[4]) + (s[1] + s[5]) + ((s[2] + s[6]) + (s[3] + s[7]));
    for (size_t i = n8; i < n; i++) t += a[i] * b[i];
    return t;
}

// ---------------------------------------------------------------------------
// Dense kernels — src/sparse.rs:279-443
// ---------------------------------------------------------------------------
namespace kern {

template <bool FMA>
static inline double fmaop(double a, double b, double c) {
    return FMA ? std::fma(a, b, c) : c + a * b;
}

// :291-303
template <bool FMA>
static inline void forward_impl(double* w, const double* lt, size_t n) {
    for (size_t p = 0; p < n; p++) {
        double wp = -w[p];
        if (wp == 0.0) continue;
        const double* col = lt + p * n;
        for (size_t q = p + 1; q < n; q++) w[q] = fmaop<FMA>(wp, col[q], w[q]);
    }
}

// :309-369 (the 4×8 register block; each C entry is one sequential multiply-add
// chain over p starting at 0, then subtracted)
template <bool FMA>
static inline void gemm_impl(double* c, size_t ldc, size_t nrows, size_t ncols, const double* a, size_t lda, const double* b,
                             size_t ldb, size_t kk) {
    const size_t YB = 512;
    size_t j0 = 0;
    while (j0 < ncols) {
        size_t j1 = std::min(j0 + YB, ncols);
        size_t i = 0;
        while (i + 4 <= nrows) {
            size_t j = j0;
            while (j + 8 <= j1) {
                double acc[4][8] = {};
                for (size_t p = 0; p < kk; p++) {
                    const double* bp = b + p * ldb + j;
                    for (int r = 0; r < 4; r++) {
                        double ar = a[(i + r) * lda + p];
                        for (int l = 0; l < 8; l++) acc[r][l] = fmaop<FMA>(ar, bp[l], acc[r][l]);
                    }
                }
                for (int r = 0; r < 4; r++) {
                    double* cr = c + (i + r) * ldc + j;
                    for (int l = 0; l < 8; l++) cr[l] -= acc[r][l];
                }
                j += 8;
            }
            for (int r = 0; r < 4; r++)
                for (size_t jj = j; jj < j1; jj++) {
                    double s = 0.0;
                    for (size_t p = 0; p < kk; p++) s = fmaop<FMA>(a[(i + r) * lda + p], b[p * ldb + jj], s);
                    c[(i + r) * ldc + jj] -= s;
                }
            i += 4;
        }
        while (i < nrows) {
            for (size_t jj = j0; jj < j1; jj++) {
                double s = 0.0;
                for (size_t p = 0; p < kk; p++) s = fmaop<FMA>(a[i * lda + p], b[p * ldb + jj], s);
                c[i * ldc + jj] -= s;
            }
            i += 1;
        }
        j0 = j1;
    }
}

#if defined(__x86_64__)
// The AVX2/FMA instantiation: the 4×8 block in eight 256-bit accumulators, the
// same multiply-add chain per entry as gemm_impl<true>.
__attribute__((target("avx2,fma"))) static void gemm_avx(double* c, size_t ldc, size_t nrows, size_t ncols,
                                                          const double* a, size_t lda, const double* b, size_t ldb,
                                                          size_t kk) {
    const size_t YB = 512;
    size_t j0 = 0;
    while (j0 < ncols) {
        size_t j1 = std::min(j0 + YB, ncols);
        size_t i = 0;
        while (i + 4 <= nrows) {
            size_t j = j0;
            while (j + 8 <= j1) {
                __m256d acc[4][2];
                for (int r = 0; r < 4; r++) acc[r][0] = acc[r][1] = _mm256_setzero_pd();
                for (size_t p = 0; p < kk; p++) {
                    const double* bp = b + p * ldb + j;
                    __m256d b0 = _mm256_loadu_pd(bp), b1 = _mm256_loadu_pd(bp + 4);
                    for (int r = 0; r < 4; r++) {
                        __m256d ar = _mm256_broadcast_sd(a + (i + r) * lda + p);
                        acc[r][0] = _mm256_fmadd_pd(ar, b0, acc[r][0]);
                        acc[r][1] = _mm256_fmadd_pd(ar, b1, acc[r][1]);
                    }
                }
                for (int r = 0; r < 4; r++) {
                    double* cr = c + (i + r) * ldc + j;
                    _mm256_storeu_pd(cr, _mm256_sub_pd(_mm256_loadu_pd(cr), acc[r][0]));
                    _mm256_storeu_pd(cr + 4, _mm256_sub_pd(_mm256_loadu_pd(cr + 4), acc[r][1]));
                }
                j += 8;
            }
            for (int r = 0; r < 4; r++)
                for (size_t jj = j; jj < j1; jj++) {
                    double s = 0.0;
                    for (size_t p = 0; p < kk; p++) s = std::fma(a[(i + r) * lda + p], b[p * ldb + jj], s);
                    c[(i + r) * ldc + jj] -= s;
                }
            i += 4;
        }
        while (i < nrows) {
            for (size_t jj = j0; jj < j1; jj++) {
                double s = 0.0;
                for (size_t p = 0; p < kk; p++) s = std::fma(a[i * lda + p], b[p * ldb + jj], s);
                c[i * ldc + jj] -= s;
            }
            i += 1;
        }
        j0 = j1;
    }
}

__attribute__((target("avx2,fma"))) static void forward_avx(double* w, const double* lt, size_t n) {
    forward_impl<true>(w, lt, n);
}

// :387-391
static bool avx() {
    static int f = -1;
    if (f < 0) f = (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) ? 1 : 0;
    return f == 1;
}
#else
static bool avx() { return false; }
#endif

static void forward(double* w, const double* lt, size_t n) {
#if defined(__x86_64__)
    if (avx()) return forward_avx(w, lt, n);
#endif
    forward_impl<false>(w, lt, n);
}

static void gemm(double* c, size_t ldc, size_t nrows, size_t ncols, const double* a, size_t lda, const double* b,
                 size_t ldb, size_t kk) {
#if defined(__x86_64__)
    if (avx()) return gemm_avx(c, ldc, nrows, ncols, a, lda, b, ldb, kk);
#endif
    gemm_impl<false>(c, ldc, nrows, ncols, a, lda, b, ldb, kk);
}

// :375-385 — rows r0..r0+nr (relative to the chunk start) of the trailing block;
// `chunk` points at row r0.
static void syrk(double* chunk, size_t ldc, size_t r0, size_t nr, size_t coloff, size_t rows, size_t kk, const double* w,
                 const double* lt) {
    const size_t YB = 512;
    size_t xend = r0 + nr;
    size_t yb0 = 0;
    while (yb0 < xend) {
        size_t yb1 = std::min(yb0 + YB, xend);
        size_t rs = std::max(r0, yb0);
        gemm(chunk + (rs - r0) * ldc + coloff + yb0, ldc, xend - rs, yb1 - yb0, w + rs * kk, kk, lt + yb0, rows, kk);
        yb0 = yb1;
    }
}

}  // namespace kern

// ---------------------------------------------------------------------------
// Positive definite numeric factorization — src/sparse.rs:445-602
// ---------------------------------------------------------------------------
static const double PAR_FLOPS = 4e6;  // :16
static const size_t KB = 96;          // :461

struct Front {
    size_t start, k;
    vector<size_t> rows;
    vector<double> l11, d, l21;
};

struct Factor {
    vector<Front> fronts;
};

struct NodeResult {
    long err = -1;  // internal equation of the failing pivot, or -1
    vector<double> upd;
    vector<Front> fronts;
};

static size_t front_local(const TNode& node, size_t dof) {
    if (dof >= node.start && dof < node.start + node.k) return dof - node.start;
    auto it = std::lower_bound(node.rows.begin(), node.rows.end(), dof);
    return node.k + (size_t)(it - node.rows.begin());
}

// Results of subtrees finished by an earlier part of a staged factorization
// (oref_staged_*): done[t] marks front t's subtree as factored, res[t] holds its
// fronts and update matrix until the parent takes them. Not part of the
// reference; the plain factorization passes none.
struct Stash {
    vector<char> done;
    vector<NodeResult> res;
};

// :463-592
static NodeResult factor_node(const Symbolic* sym, const Lower* a, size_t t, size_t nthreads, Stash* stash = nullptr) {
    const TNode& node = sym->tree[t];
    const auto& ch = node.children;
    vector<NodeResult> child_res(ch.size());
    auto child = [&](size_t i, size_t nt) {
        if (stash && stash->done[ch[i]])
            child_res[i] = std::move(stash->res[ch[i]]);
        else
            child_res[i] = factor_node(sym, a, ch[i], nt, stash);
    };
    if (ch.size() == 2 && nthreads > 1 && std::min(sym->tree[ch[0]].work, sym->tree[ch[1]].work) > 2e7) {
        size_t half = nthreads / 2;
        std::thread h([&] { child(0, half); });
        child(1, nthreads - half);
        h.join();
    } else {
        for (size_t i = 0; i < ch.size(); i++) child(i, nthreads);
    }
    NodeResult out;
    size_t start = node.start, k = node.k, u = node.rows.size();
    size_t m = k + u;
    vector<double> f(m * m, 0.0);
    for (size_t c = 0; c < k; c++) {
        size_t col = start + c;
        for (size_t p = a->colptr[col]; p < a->colptr[col + 1]; p++) f[front_local(node, a->rowidx[p]) * m + c] += a->val[p];
    }
    for (size_t i = 0; i < ch.size(); i++) {
        NodeResult& res = child_res[i];
        if (res.err >= 0) {
            out.err = res.err;
            return out;
        }
        for (auto& fr : res.fronts) out.fronts.push_back(std::move(fr));
        const auto& crows = sym->tree[ch[i]].rows;
        size_t uc = crows.size();
        vector<size_t> map(uc);
        for (size_t x = 0; x < uc; x++) map[x] = front_local(node, crows[x]);
        for (size_t x = 0; x < uc; x++) {
            size_t fx = map[x] * m;
            const double* ux = res.upd.data() + x * uc;
            for (size_t y = 0; y <= x; y++) f[fx + map[y]] += ux[y];
        }
        res.upd.clear();
        res.upd.shrink_to_fit();
    }
    vector<double> d(k, 0.0);
    size_t j0 = 0;
    while (j0 < k) {
        size_t j1 = std::min(j0 + KB, k);
        size_t jb = j1 - j0;
        // 1. diagonal block, row-wise (:516-538)
        vector<double> lb(jb * jb, 0.0), w(jb, 0.0);
        for (size_t i = 0; i < jb; i++) {
            size_t row = (j0 + i) * m + j0;
            for (size_t j = 0; j < i; j++) w[j] = f[row + j] - dot(w.data(), lb.data() + j * jb, j);
            double di = f[row + i];
            for (size_t p = 0; p < i; p++) di -= w[p] * w[p] / d[j0 + p];
            double orig = a->diag(start + j0 + i);
            if (!(orig > 0.0) || !(di > 1e-12 * orig)) {
                out.err = (long)(start + j0 + i);
                return out;
            }
            d[j0 + i] = di;
            for (size_t p = 0; p < i; p++) {
                double l = w[p] / d[j0 + p];
                lb[i * jb + p] = l;
                f[row + p] = l;
            }
        }
        if (j1 < m) {
            size_t rows = m - j1;
            vector<double> lbt(jb * jb, 0.0);
            for (size_t i = 0; i < jb; i++)
                for (size_t p = 0; p < i; p++) lbt[p * jb + i] = lb[i * jb + p];
            // 2. panel (:547-558)
            size_t tp = ((double)(rows * jb * jb) > PAR_FLOPS) ? nthreads : 1;
            const double* dj = d.data() + j0;
            blocks_mut(rows, tp, [](size_t) { return 1.0; }, [&](size_t r0, size_t nr) {
                for (size_t r = r0; r < r0 + nr; r++) {
                    double* wr = f.data() + (j1 + r) * m + j0;
                    kern::forward(wr, lbt.data(), jb);
                    for (size_t p = 0; p < jb; p++) wr[p] /= dj[p];
                }
            });
            // 3. update (:559-573)
            vector<double> wt(rows * jb), lt(jb * rows);
            for (size_t r = 0; r < rows; r++) {
                const double* fr = f.data() + (j1 + r) * m + j0;
                for (size_t p = 0; p < jb; p++) {
                    wt[r * jb + p] = fr[p] * d[j0 + p];
                    lt[p * rows + r] = fr[p];
                }
            }
            tp = ((double)(rows * rows * jb) / 2.0 > PAR_FLOPS) ? nthreads : 1;
            blocks_mut(rows, tp, [](size_t r) { return (double)(r + 1); }, [&](size_t r0, size_t nr) {
                kern::syrk(f.data() + (j1 + r0) * m, m, r0, nr, j1, rows, jb, wt.data(), lt.data());
            });
        }
        j0 = j1;
    }
    // pack (:578-591)
    Front fr;
    fr.start = start;
    fr.k = k;
    fr.rows = node.rows;
    fr.l11.reserve(k * (k ? k - 1 : 0) / 2);
    for (size_t i = 0; i < k; i++) fr.l11.insert(fr.l11.end(), f.begin() + i * m, f.begin() + i * m + i);
    fr.l21.assign(u * k, 0.0);
    out.upd.assign(u * u, 0.0);
    for (size_t r = 0; r < u; r++) {
        const double* frow = f.data() + (k + r) * m;
        std::copy(frow, frow + k, fr.l21.begin() + r * k);
        std::copy(frow + k, frow + k + r + 1, out.upd.begin() + r * u);
    }
    fr.d = std::move(d);
    out.fronts.push_back(std::move(fr));
    return out;
}

// :595-602
static Factor* factor(const Symbolic* sym, const Lower* a, long* err) {
    Factor* F = new Factor();
    *err = -1;
    for (size_t r : sym->roots) {
        NodeResult res = factor_node(sym, a, r, threads());
        if (res.err >= 0) {
            *err = res.err;
            delete F;
            return nullptr;
        }
        for (auto& fr : res.fronts) F->fronts.push_back(std::move(fr));
    }
    return F;
}

// :606-612
static void pivots(const Factor* F, double* d) {
    for (auto& fr : F->fronts) std::copy(fr.d.begin(), fr.d.end(), d + fr.start);
}

// :615-652
static void solve(const Factor* F, double* x) {
    for (auto& fr : F->fronts) {
        size_t k = fr.k;
        double* xp = x + fr.start;
        for (size_t i = 0; i < k; i++) {
            size_t r = i * (i ? i - 1 : 0) / 2;
            xp[i] -= dot(fr.l11.data() + r, xp, i);
        }
        vector<double> xc(xp, xp + k);
        for (size_t r = 0; r < fr.rows.size(); r++) x[fr.rows[r]] -= dot(fr.l21.data() + r * k, xc.data(), k);
    }
    for (auto& fr : F->fronts)
        for (size_t i = 0; i < fr.k; i++) x[fr.start + i] /= fr.d[i];
    for (size_t fi = F->fronts.size(); fi-- > 0;) {
        const Front& fr = F->fronts[fi];
        size_t k = fr.k;
        vector<double> xp(x + fr.start, x + fr.start + k);
        for (size_t r = 0; r < fr.rows.size(); r++) {
            double xr = x[fr.rows[r]];
            const double* l = fr.l21.data() + r * k;
            for (size_t p = 0; p < k; p++) xp[p] -= l[p] * xr;
        }
        for (size_t i = k; i-- > 0;) {
            double xi = xp[i];
            size_t r = i * (i ? i - 1 : 0) / 2;
            for (size_t q = 0; q < i; q++) xp[q] -= fr.l11[r + q] * xi;
        }
        std::copy(xp.begin(), xp.end(), x + fr.start);
    }
}

// ---------------------------------------------------------------------------
// Indefinite LDLᵀ — src/sparse/indef.rs
// ---------------------------------------------------------------------------
namespace indef {

static const double THRESHOLD = 0.01;           // :27
static const double ZERO_TOL = 1e-12;           // :29
static const double ALPHA = 0.6403882032022079; // :31
static const size_t IKB = 64;                   // :33

struct Inertia {
    size_t neg = 0, zero = 0, pos = 0;
};

struct IFront {  // :44-59
    vector<size_t> piv;
    vector<double> l11, d, e;
    vector<uint8_t> kind;
    vector<size_t> rows;
    vector<double> l21;
};

struct IndefFactor {  // :62-68
    vector<IFront> fronts;
    Inertia inertia;
    size_t delayed = 0, two_by_two = 0;
};

struct Ctx {  // :83-88
    const Symbolic* sym;
    const Lower* a;
    vector<double> scale;
    double thr;
};

struct NodeOut {  // :90-95
    long err = -1;
    vector<double> upd;
    vector<size_t> idx;
    vector<IFront> fronts;
    size_t delayed = 0;
};

// :98-108
static vector<double> column_scale(const Lower* a, size_t n) {
    vector<double> s(n, 0.0);
    for (size_t c = 0; c < n; c++)
        for (size_t p = a->colptr[c]; p < a->colptr[c + 1]; p++) {
            size_t r = a->rowidx[p];
            double v = std::fabs(a->val[p]);
            s[c] = std::fmax(s[c], v);
            s[r] = std::fmax(s[r], v);
        }
    return s;
}

// :262-273
static void swap(double* f, size_t m, size_t kf, vector<size_t>& fs, size_t p, size_t q) {
    if (p == q) return;
    for (size_t c = 0; c < kf; c++) std::swap(f[p * m + c], f[q * m + c]);
    for (size_t i = 0; i < m; i++) std::swap(f[i * m + p], f[i * m + q]);
    std::swap(fs[p], fs[q]);
}

// :277-285
static double colmax(const double* f, size_t m, size_t p, size_t j, size_t x) {
    double g = 0.0;
    for (size_t i = p; i < m; i++)
        if (i != j && i != x) g = std::fmax(g, std::fabs(f[i * m + j]));
    return g;
}

enum PivKind { NO_PIVOT = 0, ONE = 1, TWO = 2 };
struct Pivot {
    PivKind kind;
    size_t j, r;
};

// :288-323
static Pivot choose(const double* f, size_t m, size_t p, size_t end, const vector<size_t>& fs, const Ctx& ctx) {
    double thr = ctx.thr;
    for (size_t j = p; j < end; j++) {
        double ajj = f[j * m + j];
        double sj = ctx.scale[fs[j]];
        double gj = colmax(f, m, p, j, NONE);
        if (std::fabs(ajj) > ZERO_TOL * sj && std::fabs(ajj) >= thr * gj) return {ONE, j, 0};
        size_t r = NONE;
        double best = 0.0;
        for (size_t i = p; i < end; i++)
            if (i != j && std::fabs(f[i * m + j]) > best) {
                best = std::fabs(f[i * m + j]);
                r = i;
            }
        if (r == NONE) continue;
        double a = ajj, b = f[r * m + j], c = f[r * m + r];
        double det = a * c - b * b;
        double sr = ctx.scale[fs[r]];
        if (!(std::fabs(det) > ZERO_TOL * sj * sr)) continue;
        double gj2 = colmax(f, m, p, j, r);
        double gr2 = colmax(f, m, p, r, j);
        double ad = std::fabs(det);
        if ((std::fabs(c) * gj2 + std::fabs(b) * gr2) / ad <= 1.0 / thr &&
            (std::fabs(b) * gj2 + std::fabs(a) * gr2) / ad <= 1.0 / thr)
            return {TWO, j, r};
    }
    return {NO_PIVOT, 0, 0};
}

// :326-372 — returns kind NO_PIVOT with j = the singular equation on failure
static Pivot choose_forced(const double* f, size_t m, size_t p, size_t kf, const vector<size_t>& fs, const Ctx& ctx,
                           long* err) {
    size_t bi = p, bj = p;
    double big = -1.0;
    for (size_t j = p; j < kf; j++)
        for (size_t i = j; i < kf; i++) {
            double v = std::fabs(f[i * m + j]);
            if (v > big) {
                big = v;
                bi = i;
                bj = j;
            }
        }
    auto one = [&](size_t j) -> Pivot {
        if (std::fabs(f[j * m + j]) > ZERO_TOL * ctx.scale[fs[j]]) return {ONE, j, 0};
        *err = (long)fs[j];
        return {NO_PIVOT, 0, 0};
    };
    if (!(big > ZERO_TOL * std::fmax(ctx.scale[fs[bj]], ctx.scale[fs[bi]]))) {
        *err = (long)fs[bj];
        return {NO_PIVOT, 0, 0};
    }
    if (bi == bj) return one(bj);
    size_t j = bj, r = bi;
    double lam = big;
    double ajj = std::fabs(f[j * m + j]);
    if (ajj >= ALPHA * lam) return one(j);
    double sig = 0.0;
    for (size_t i = p; i < kf; i++) {
        if (i == r) continue;
        double v = std::fabs(i >= r ? f[i * m + r] : f[r * m + i]);
        sig = std::fmax(sig, v);
    }
    if (ajj * sig >= ALPHA * lam * lam) return one(j);
    if (std::fabs(f[r * m + r]) >= ALPHA * sig) return one(r);
    double a = f[j * m + j], b = f[r * m + j], c = f[r * m + r];
    double det = a * c - b * b;
    if (!(std::fabs(det) > ZERO_TOL * ctx.scale[fs[j]] * ctx.scale[fs[r]])) {
        *err = (long)fs[j];
        return {NO_PIVOT, 0, 0};
    }
    return {TWO, j, r};
}

// :375-389
static double elim1(double* f, size_t m, size_t p, size_t bend) {
    double dp = f[p * m + p];
    vector<double> w;
    for (size_t c = p + 1; c < bend; c++) w.push_back(f[c * m + p]);
    for (size_t i = p + 1; i < m; i++) {
        double li = f[i * m + p] / dp;
        if (li != 0.0) {
            double* row = f + i * m + p + 1;
            for (size_t x = 0; x < w.size(); x++) row[x] -= li * w[x];
        }
        f[i * m + p] = li;
    }
    return dp;
}

// :392-411
static void elim2(double* f, size_t m, size_t p, size_t bend, double* a_out, double* b_out, double* c_out) {
    double a = f[p * m + p], b = f[(p + 1) * m + p], c = f[(p + 1) * m + p + 1];
    double det = a * c - b * b;
    vector<double> w0, w1;
    for (size_t q = p + 2; q < bend; q++) {
        w0.push_back(f[q * m + p]);
        w1.push_back(f[q * m + p + 1]);
    }
    for (size_t i = p + 2; i < m; i++) {
        double x0 = f[i * m + p], x1 = f[i * m + p + 1];
        double l0 = (x0 * c - x1 * b) / det;
        double l1 = (x1 * a - x0 * b) / det;
        if (l0 != 0.0 || l1 != 0.0) {
            double* row = f + i * m + p + 2;
            for (size_t x = 0; x < w0.size(); x++) row[x] -= l0 * w0[x] + l1 * w1[x];
        }
        f[i * m + p] = l0;
        f[i * m + p + 1] = l1;
    }
    *a_out = a;
    *b_out = b;
    *c_out = c;
}

// :504-532
static void trailing_update(double* f, size_t m, size_t p0, size_t npb, size_t b1, const double* d, const double* e,
                            const uint8_t* kind, size_t nthreads) {
    size_t rows = m - b1;
    vector<double> w(rows * npb, 0.0), lt(npb * rows, 0.0);
    for (size_t r = 0; r < rows; r++) {
        const double* fr = f + (b1 + r) * m + p0;
        double* wr = w.data() + r * npb;
        size_t q = 0;
        while (q < npb) {
            if (kind[q] == 2) {
                double l0 = fr[q], l1 = fr[q + 1];
                wr[q] = l0 * d[q] + l1 * e[q];
                wr[q + 1] = l0 * e[q] + l1 * d[q + 1];
                q += 2;
            } else {
                wr[q] = fr[q] * d[q];
                q += 1;
            }
        }
        for (q = 0; q < npb; q++) lt[q * rows + r] = fr[q];
    }
    size_t tp = ((double)(rows * rows * npb) / 2.0 > PAR_FLOPS) ? nthreads : 1;
    blocks_mut(rows, tp, [](size_t r) { return (double)(r + 1); }, [&](size_t r0, size_t nr) {
        kern::syrk(f + (b1 + r0) * m, m, r0, nr, b1, rows, npb, w.data(), lt.data());
    });
}

// :416-500 — returns the number of eliminated pivots, or -1 with *err set
static long eliminate(double* f, size_t m, size_t kf, vector<size_t>& fs, const Ctx& ctx, bool root, size_t nthreads,
                      vector<double>& d, vector<double>& e, vector<uint8_t>& kind, long* err) {
    size_t p = 0, width = IKB;
    while (p < kf) {
        size_t p0 = p;
        size_t b1 = std::min(p + width, kf);
        while (p < b1) {
            Pivot pv = choose(f, m, p, b1, fs, ctx);
            if (pv.kind == ONE) {
                swap(f, m, kf, fs, p, pv.j);
                d.push_back(elim1(f, m, p, b1));
                e.push_back(0.0);
                kind.push_back(1);
                p += 1;
            } else if (pv.kind == TWO) {
                size_t r = (pv.r == p) ? pv.j : pv.r;
                swap(f, m, kf, fs, p, pv.j);
                swap(f, m, kf, fs, p + 1, r);
                double a, b, c;
                elim2(f, m, p, b1, &a, &b, &c);
                d.push_back(a);
                d.push_back(c);
                e.push_back(b);
                e.push_back(0.0);
                kind.push_back(2);
                kind.push_back(0);
                p += 2;
            } else {
                break;
            }
        }
        size_t npb = p - p0;
        if (npb > 0 && b1 < m) {
            trailing_update(f, m, p0, npb, b1, d.data() + p0, e.data() + p0, kind.data() + p0, nthreads);
            for (size_t i = b1; i < kf; i++)
                for (size_t j = p; j < i; j++) f[j * m + i] = f[i * m + j];
        }
        if (npb == 0) {
            if (b1 == kf) break;
            width *= 2;
        } else {
            width = IKB;
        }
    }
    if (p < kf && root) {
        while (p < kf) {
            Pivot pv = choose_forced(f, m, p, kf, fs, ctx, err);
            if (pv.kind == NO_PIVOT) return -1;
            if (pv.kind == ONE) {
                swap(f, m, kf, fs, p, pv.j);
                d.push_back(elim1(f, m, p, kf));
                e.push_back(0.0);
                kind.push_back(1);
                p += 1;
            } else {
                size_t r = (pv.r == p) ? pv.j : pv.r;
                swap(f, m, kf, fs, p, pv.j);
                swap(f, m, kf, fs, p + 1, r);
                double a, b, c;
                elim2(f, m, p, kf, &a, &b, &c);
                d.push_back(a);
                d.push_back(c);
                e.push_back(b);
                e.push_back(0.0);
                kind.push_back(2);
                kind.push_back(0);
                p += 2;
            }
        }
    }
    return (long)p;
}

// :158-254
static NodeOut factor_node(const Ctx& ctx, size_t t, size_t nthreads, bool root) {
    const Symbolic* sym = ctx.sym;
    const TNode& node = sym->tree[t];
    const auto& ch = node.children;
    vector<NodeOut> child_res(ch.size());
    if (ch.size() == 2 && nthreads > 1 && std::min(sym->tree[ch[0]].work, sym->tree[ch[1]].work) > 2e7) {
        size_t half = nthreads / 2;
        std::thread h([&] { child_res[0] = factor_node(ctx, ch[0], half, false); });
        child_res[1] = factor_node(ctx, ch[1], nthreads - half, false);
        h.join();
    } else {
        for (size_t i = 0; i < ch.size(); i++) child_res[i] = factor_node(ctx, ch[i], nthreads, false);
    }
    NodeOut out;
    size_t start = node.start, k = node.k, u = node.rows.size();
    vector<size_t> fs;
    for (size_t g = start; g < start + k; g++) fs.push_back(g);
    size_t delayed = 0;
    for (auto& o : child_res) {
        if (o.err >= 0) {
            out.err = o.err;
            return out;
        }
        for (auto& fr : o.fronts) out.fronts.push_back(std::move(fr));
        delayed += o.delayed;
        for (size_t g : o.idx)
            if (g < start) fs.push_back(g);
    }
    size_t kf = fs.size();
    delayed += kf - k;
    size_t m = kf + u;
    vector<std::pair<size_t, size_t>> dmap;
    for (size_t i = k; i < kf; i++) dmap.push_back({fs[i], i});
    std::sort(dmap.begin(), dmap.end());
    auto local = [&](size_t g) -> size_t {
        if (g >= start && g < start + k) return g - start;
        if (g < start) {
            auto it = std::lower_bound(dmap.begin(), dmap.end(), std::make_pair(g, (size_t)0));
            return it->second;
        }
        auto it = std::lower_bound(node.rows.begin(), node.rows.end(), g);
        return kf + (size_t)(it - node.rows.begin());
    };
    vector<double> f(m * m, 0.0);
    const Lower* a = ctx.a;
    for (size_t c = 0; c < k; c++) {
        size_t col = start + c;
        for (size_t p = a->colptr[col]; p < a->colptr[col + 1]; p++) f[local(a->rowidx[p]) * m + c] += a->val[p];
    }
    for (auto& o : child_res) {
        size_t s = o.idx.size();
        vector<size_t> map(s);
        for (size_t x = 0; x < s; x++) map[x] = local(o.idx[x]);
        for (size_t x = 0; x < s; x++)
            for (size_t y = 0; y <= x; y++) {
                size_t i = map[x], j = map[y];
                if (i < j) std::swap(i, j);
                f[i * m + j] += o.upd[x * s + y];
            }
        o.upd.clear();
        o.upd.shrink_to_fit();
    }
    for (size_t i = 0; i < kf; i++)
        for (size_t j = 0; j < i; j++) f[j * m + i] = f[i * m + j];
    vector<double> d, e;
    vector<uint8_t> kind;
    long err = -1;
    long np = eliminate(f.data(), m, kf, fs, ctx, root, nthreads, d, e, kind, &err);
    if (np < 0) {
        out.err = err;
        return out;
    }
    size_t npiv = (size_t)np;
    IFront fr;
    fr.l11.reserve(npiv * (npiv ? npiv - 1 : 0) / 2);
    for (size_t i = 0; i < npiv; i++) {
        size_t sl = fr.l11.size();
        fr.l11.insert(fr.l11.end(), f.begin() + i * m, f.begin() + i * m + i);
        if (kind[i] == 0) fr.l11[sl + i - 1] = 0.0;
    }
    vector<size_t> rows(fs.begin() + npiv, fs.begin() + kf);
    rows.insert(rows.end(), node.rows.begin(), node.rows.end());
    size_t nr = rows.size();
    fr.l21.assign(nr * npiv, 0.0);
    out.upd.assign(nr * nr, 0.0);
    for (size_t r = 0; r < nr; r++) {
        const double* frow = f.data() + (npiv + r) * m;
        std::copy(frow, frow + npiv, fr.l21.begin() + r * npiv);
        std::copy(frow + npiv, frow + npiv + r + 1, out.upd.begin() + r * nr);
    }
    fr.piv.assign(fs.begin(), fs.begin() + npiv);
    fr.d = std::move(d);
    fr.e = std::move(e);
    fr.kind = std::move(kind);
    fr.rows = rows;
    out.fronts.push_back(std::move(fr));
    out.idx = std::move(rows);
    out.delayed = delayed;
    return out;
}

// :116-156
static IndefFactor* factor_with(const Symbolic* sym, const Lower* a, double threshold, long* err) {
    Ctx ctx{sym, a, column_scale(a, sym->n), std::min(std::max(threshold, 1e-8), 0.5)};
    IndefFactor* F = new IndefFactor();
    *err = -1;
    for (size_t r : sym->roots) {
        NodeOut o = factor_node(ctx, r, threads(), true);
        if (o.err >= 0) {
            *err = o.err;
            delete F;
            return nullptr;
        }
        for (auto& fr : o.fronts) F->fronts.push_back(std::move(fr));
        F->delayed += o.delayed;
    }
    size_t two = 0;
    for (auto& fr : F->fronts) {
        size_t i = 0;
        while (i < fr.d.size()) {
            if (fr.kind[i] == 2) {
                two++;
                double a_ = fr.d[i], b = fr.e[i], c = fr.d[i + 1];
                double det = a_ * c - b * b;
                if (det < 0.0) {
                    F->inertia.neg++;
                    F->inertia.pos++;
                } else if (a_ + c < 0.0) {
                    F->inertia.neg += 2;
                } else {
                    F->inertia.pos += 2;
                }
                i += 2;
            } else {
                if (fr.d[i] < 0.0)
                    F->inertia.neg++;
                else if (fr.d[i] > 0.0)
                    F->inertia.pos++;
                else
                    F->inertia.zero++;
                i += 1;
            }
        }
    }
    F->two_by_two = two;
    return F;
}

// :536-591
static void solve(const IndefFactor* F, double* x) {
    for (auto& fr : F->fronts) {
        size_t k = fr.piv.size();
        vector<double> xp(k);
        for (size_t i = 0; i < k; i++) xp[i] = x[fr.piv[i]];
        for (size_t i = 0; i < k; i++) {
            size_t r = i * (i ? i - 1 : 0) / 2;
            xp[i] -= dot(fr.l11.data() + r, xp.data(), i);
        }
        for (size_t r = 0; r < fr.rows.size(); r++) x[fr.rows[r]] -= dot(fr.l21.data() + r * k, xp.data(), k);
        for (size_t i = 0; i < k; i++) x[fr.piv[i]] = xp[i];
    }
    for (auto& fr : F->fronts) {
        size_t i = 0;
        while (i < fr.piv.size()) {
            if (fr.kind[i] == 2) {
                double a = fr.d[i], b = fr.e[i], c = fr.d[i + 1];
                double det = a * c - b * b;
                size_t g0 = fr.piv[i], g1 = fr.piv[i + 1];
                double y0 = x[g0], y1 = x[g1];
                x[g0] = (c * y0 - b * y1) / det;
                x[g1] = (a * y1 - b * y0) / det;
                i += 2;
            } else {
                x[fr.piv[i]] /= fr.d[i];
                i += 1;
            }
        }
    }
    for (size_t fi = F->fronts.size(); fi-- > 0;) {
        const IFront& fr = F->fronts[fi];
        size_t k = fr.piv.size();
        vector<double> xp(k);
        for (size_t i = 0; i < k; i++) xp[i] = x[fr.piv[i]];
        for (size_t r = 0; r < fr.rows.size(); r++) {
            double xr = x[fr.rows[r]];
            if (xr != 0.0) {
                const double* l = fr.l21.data() + r * k;
                for (size_t p = 0; p < k; p++) xp[p] -= l[p] * xr;
            }
        }
        for (size_t i = k; i-- > 0;) {
            double xi = xp[i];
            size_t r = i * (i ? i - 1 : 0) / 2;
            for (size_t q = 0; q < i; q++) xp[q] -= fr.l11[r + q] * xi;
        }
        for (size_t i = 0; i < k; i++) x[fr.piv[i]] = xp[i];
    }
}

static size_t factor_size(const IndefFactor* F) {
    size_t z = 0;
    for (auto& f : F->fronts) z += f.l11.size() + f.l21.size();
    return z;
}

}  // namespace indef

// ---------------------------------------------------------------------------
// Unsymmetric multifrontal LU — src/sparse/lu.rs:1-409 (same tree as LDLᵀ,
// full fronts, diagonal threshold pivoting with delays, partial pivoting at
// the root)
// ---------------------------------------------------------------------------
namespace lu {

static const double THRESHOLD = 0.01;  // :22
static const size_t KB = 64;           // :23

// :27-92 — lower triangle in `lower`, the strictly upper triangle transposed in `upper_t`
struct Full {
    Lower lower, upper_t;
    void add(size_t r, size_t c, double v) {
        if (r >= c)
            lower.add(r, c, v);
        else
            upper_t.add(c, r, v);
    }
    void matvec(const double* x, double* y, size_t n) const {
        for (size_t i = 0; i < n; i++) y[i] = 0.0;
        for (size_t c = 0; c + 1 < lower.colptr.size(); c++)
            for (size_t p = lower.colptr[c]; p < lower.colptr[c + 1]; p++) {
                size_t r = lower.rowidx[p];
                y[r] += lower.val[p] * x[c];
                if (r != c) y[c] += upper_t.val[p] * x[r];
            }
    }
    vector<double> scale(size_t n) const {
        vector<double> s(n, 0.0);
        for (int t = 0; t < 2; t++) {
            const Lower& mm = t ? upper_t : lower;
            for (size_t c = 0; c < n; c++)
                for (size_t p = mm.colptr[c]; p < mm.colptr[c + 1]; p++) {
                    size_t r = mm.rowidx[p];
                    if (t && r == c) continue;
                    double v = std::fabs(mm.val[p]);
                    s[c] = std::fmax(s[c], v);
                    s[r] = std::fmax(s[r], v);
                }
        }
        return s;
    }
};

struct LuFront {  // :94-105
    vector<size_t> piv, rperm;
    vector<double> lu11;  // k×k: L11 strictly below the diagonal (unit), U11 on and above it
    vector<size_t> rows;
    vector<double> l21, u12;  // rows×k and k×rows
};

struct LuFactor {
    vector<LuFront> fronts;
    size_t delayed = 0;
};

struct Ctx {
    const Symbolic* sym;
    const Full* a;
    vector<double> scale;
    double thr;
};

struct NodeOut {
    vector<double> upd;
    vector<size_t> idx;
    vector<LuFront> fronts;
    size_t delayed = 0;
    long err = -1;
};

// :272-283 — symmetric swap of p and q: rows, then columns, then the variables
static void swap(double* f, size_t m, vector<size_t>& fs, size_t p, size_t q) {
    if (p == q) return;
    for (size_t c = 0; c < m; c++) std::swap(f[p * m + c], f[q * m + c]);
    for (size_t i = 0; i < m; i++) std::swap(f[i * m + p], f[i * m + q]);
    std::swap(fs[p], fs[q]);
}

// :285-361
static size_t eliminate(double* f, size_t m, size_t kf, vector<size_t>& fs, const Ctx& ctx, size_t nthreads) {
    size_t p = 0, width = KB;
    vector<double> urow;
    while (p < kf) {
        size_t p0 = p;
        size_t b1 = std::min(p + width, kf);
        while (p < b1) {
            // the first candidate that passes the threshold test
            long pick = -1;
            for (size_t j = p; j < b1; j++) {
                double ajj = std::fabs(f[j * m + j]);
                if (!(ajj > indef::ZERO_TOL * ctx.scale[fs[j]])) continue;
                double g = 0.0;
                for (size_t i = p; i < m; i++)
                    if (i != j) g = std::fmax(g, std::fabs(f[i * m + j]));
                if (ajj >= ctx.thr * g) {
                    pick = (long)j;
                    break;
                }
            }
            if (pick < 0) break;
            swap(f, m, fs, p, (size_t)pick);
            double dp = f[p * m + p];
            urow.assign(f + p * m + p + 1, f + p * m + m);
            for (size_t i = p + 1; i < m; i++) {
                double li = f[i * m + p] / dp;
                f[i * m + p] = li;
                if (li == 0.0) continue;
                // the block's columns for all rows, the whole row for rows in the block
                size_t end = i < b1 ? m : b1;
                double* row = f + i * m + p + 1;
                for (size_t x = 0; x + p + 1 < end; x++) row[x] -= li * urow[x];
            }
            p++;
        }
        size_t npb = p - p0;
        if (npb > 0 && b1 < m) {
            // F[b1.., b1..] −= L[b1.., p0..p]·U[p0..p, b1..]
            size_t rows = m - b1;
            vector<double> a(rows * npb), b(npb * rows);
            for (size_t r = 0; r < rows; r++)
                std::copy(f + (b1 + r) * m + p0, f + (b1 + r) * m + p, a.begin() + r * npb);
            for (size_t q = 0; q < npb; q++)
                std::copy(f + (p0 + q) * m + b1, f + (p0 + q) * m + m, b.begin() + q * rows);
            size_t tp = ((double)(rows * rows * npb) > PAR_FLOPS) ? nthreads : 1;
            blocks_mut(rows, tp, [](size_t) { return 1.0; }, [&](size_t r0, size_t nr) {
                kern::gemm(f + (b1 + r0) * m + b1, m, nr, rows, a.data() + r0 * npb, npb, b.data(), rows, npb);
            });
        }
        if (npb == 0) {
            if (b1 == kf) break;
            width *= 2;
        } else {
            width = KB;
        }
    }
    return p;
}

// :244-270 — dense LU with partial pivoting in place; the row permutation, or err
static bool dense_lu(double* s, size_t r, const vector<size_t>& vars, const vector<double>& scale,
                     vector<size_t>& perm, long* err) {
    perm.resize(r);
    for (size_t i = 0; i < r; i++) perm[i] = i;
    for (size_t p = 0; p < r; p++) {
        size_t bi = p;
        double big = 0.0;
        for (size_t i = p; i < r; i++)
            if (std::fabs(s[i * r + p]) > big) {
                big = std::fabs(s[i * r + p]);
                bi = i;
            }
        if (!(big > indef::ZERO_TOL * scale[vars[p]])) {
            *err = (long)vars[p];
            return false;
        }
        if (bi != p) {
            for (size_t c = 0; c < r; c++) std::swap(s[p * r + c], s[bi * r + c]);
            std::swap(perm[p], perm[bi]);
        }
        double dp = s[p * r + p];
        for (size_t i = p + 1; i < r; i++) {
            double l = s[i * r + p] / dp;
            s[i * r + p] = l;
            if (l != 0.0)
                for (size_t c = p + 1; c < r; c++) s[i * r + c] -= l * s[p * r + c];
        }
    }
    return true;
}

// :139-242
static NodeOut factor_node(const Ctx& ctx, size_t t, size_t nthreads, bool root) {
    const Symbolic* sym = ctx.sym;
    const TNode& node = sym->tree[t];
    const auto& ch = node.children;
    vector<NodeOut> child_res(ch.size());
    if (ch.size() == 2 && nthreads > 1 && std::min(sym->tree[ch[0]].work, sym->tree[ch[1]].work) > 2e7) {
        size_t half = nthreads / 2;
        std::thread h([&] { child_res[0] = factor_node(ctx, ch[0], half, false); });
        child_res[1] = factor_node(ctx, ch[1], nthreads - half, false);
        h.join();
    } else {
        for (size_t i = 0; i < ch.size(); i++) child_res[i] = factor_node(ctx, ch[i], nthreads, false);
    }
    NodeOut out;
    size_t start = node.start, k = node.k, u = node.rows.size();
    vector<size_t> fs;
    for (size_t g = start; g < start + k; g++) fs.push_back(g);
    size_t delayed = 0;
    for (auto& o : child_res) {
        if (o.err >= 0) {
            out.err = o.err;
            return out;
        }
        for (auto& fr : o.fronts) out.fronts.push_back(std::move(fr));
        delayed += o.delayed;
        for (size_t g : o.idx)
            if (g < start) fs.push_back(g);
    }
    size_t kf = fs.size();
    delayed += kf - k;
    size_t m = kf + u;
    vector<std::pair<size_t, size_t>> dmap;
    for (size_t i = k; i < kf; i++) dmap.push_back({fs[i], i});
    std::sort(dmap.begin(), dmap.end());
    auto local = [&](size_t g) -> size_t {
        if (g >= start && g < start + k) return g - start;
        if (g < start) return std::lower_bound(dmap.begin(), dmap.end(), std::make_pair(g, (size_t)0))->second;
        return kf + (size_t)(std::lower_bound(node.rows.begin(), node.rows.end(), g) - node.rows.begin());
    };
    vector<double> f(m * m, 0.0);
    const Lower& lo = ctx.a->lower;
    const Lower& ut = ctx.a->upper_t;
    for (size_t c = 0; c < k; c++) {
        size_t col = start + c;
        for (size_t p = lo.colptr[col]; p < lo.colptr[col + 1]; p++) {
            size_t lr = local(lo.rowidx[p]);
            f[lr * m + c] += lo.val[p];
            if (lr != c) f[c * m + lr] += ut.val[p];
        }
    }
    for (auto& o : child_res) {
        size_t s = o.idx.size();
        vector<size_t> map(s);
        for (size_t x = 0; x < s; x++) map[x] = local(o.idx[x]);
        for (size_t x = 0; x < s; x++)
            for (size_t y = 0; y < s; y++) f[map[x] * m + map[y]] += o.upd[x * s + y];
        o.upd.clear();
        o.upd.shrink_to_fit();
    }
    size_t npiv = eliminate(f.data(), m, kf, fs, ctx, nthreads);
    vector<size_t> rows(fs.begin() + npiv, fs.begin() + kf);
    rows.insert(rows.end(), node.rows.begin(), node.rows.end());
    size_t nr = rows.size();
    {
        LuFront fr;
        size_t kk = npiv;
        fr.piv.assign(fs.begin(), fs.begin() + npiv);
        fr.lu11.resize(kk * kk);
        for (size_t i = 0; i < kk; i++) std::copy(f.begin() + i * m, f.begin() + i * m + kk, fr.lu11.begin() + i * kk);
        fr.l21.resize(nr * kk);
        fr.u12.resize(kk * nr);
        for (size_t r = 0; r < nr; r++)
            std::copy(f.begin() + (kk + r) * m, f.begin() + (kk + r) * m + kk, fr.l21.begin() + r * kk);
        for (size_t i = 0; i < kk; i++)
            std::copy(f.begin() + i * m + kk, f.begin() + i * m + kk + nr, fr.u12.begin() + i * nr);
        fr.rows = rows;
        out.fronts.push_back(std::move(fr));
    }
    if (root && npiv < kf) {
        // root: partial pivoting with row swaps on the rest (no later rows)
        size_t r = kf - npiv;
        vector<double> sq(r * r);
        for (size_t i = 0; i < r; i++)
            std::copy(f.begin() + (npiv + i) * m + npiv, f.begin() + (npiv + i) * m + npiv + r, sq.begin() + i * r);
        vector<size_t> vars(fs.begin() + npiv, fs.begin() + kf);
        LuFront fr;
        long err = -1;
        if (!dense_lu(sq.data(), r, vars, ctx.scale, fr.rperm, &err)) {
            out.err = err;
            return out;
        }
        fr.piv = vars;
        fr.lu11 = std::move(sq);
        out.fronts.push_back(std::move(fr));
        out.delayed = delayed;
        return out;
    }
    out.upd.resize(nr * nr);
    for (size_t x = 0; x < nr; x++)
        std::copy(f.begin() + (npiv + x) * m + npiv, f.begin() + (npiv + x) * m + npiv + nr, out.upd.begin() + x * nr);
    out.idx = std::move(rows);
    out.delayed = delayed;
    return out;
}

// :121-137
static LuFactor* factor_with(const Symbolic* sym, const Full* a, double threshold, long* err) {
    Ctx ctx{sym, a, a->scale(sym->n), std::min(std::max(threshold, 1e-8), 1.0)};
    LuFactor* F = new LuFactor();
    *err = -1;
    for (size_t r : sym->roots) {
        NodeOut o = factor_node(ctx, r, threads(), true);
        if (o.err >= 0) {
            *err = o.err;
            delete F;
            return nullptr;
        }
        for (auto& fr : o.fronts) F->fronts.push_back(std::move(fr));
        F->delayed += o.delayed;
    }
    return F;
}

// :364-402 — A x = b in place (internal numbering)
static void solve(const LuFactor* F, double* x) {
    vector<double> xp, xr;
    for (const LuFront& fr : F->fronts) {
        size_t k = fr.piv.size();
        xp.resize(k);
        for (size_t i = 0; i < k; i++) xp[i] = fr.rperm.empty() ? x[fr.piv[i]] : x[fr.piv[fr.rperm[i]]];
        for (size_t i = 0; i < k; i++) xp[i] -= dot(fr.lu11.data() + i * k, xp.data(), i);
        for (size_t r = 0; r < fr.rows.size(); r++) x[fr.rows[r]] -= dot(fr.l21.data() + r * k, xp.data(), k);
        for (size_t i = 0; i < k; i++) x[fr.piv[i]] = xp[i];
    }
    for (size_t fi = F->fronts.size(); fi-- > 0;) {
        const LuFront& fr = F->fronts[fi];
        size_t k = fr.piv.size(), nr = fr.rows.size();
        xr.resize(nr);
        for (size_t r = 0; r < nr; r++) xr[r] = x[fr.rows[r]];
        xp.resize(k);
        for (size_t i = 0; i < k; i++) xp[i] = x[fr.piv[i]];
        for (size_t i = 0; i < k; i++) xp[i] -= dot(fr.u12.data() + i * nr, xr.data(), nr);
        for (size_t i = k; i-- > 0;) {
            double s = dot(fr.lu11.data() + i * k + i + 1, xp.data() + i + 1, k - i - 1);
            xp[i] = (xp[i] - s) / fr.lu11[i * k + i];
        }
        for (size_t i = 0; i < k; i++) x[fr.piv[i]] = xp[i];
    }
}

static size_t factor_size(const LuFactor* F) {  // :404-406
    size_t s = 0;
    for (auto& fr : F->fronts) s += fr.lu11.size() + fr.l21.size() + fr.u12.size();
    return s;
}

}  // namespace lu

// src/sparse/indef.rs:600-611
static void sym_matvec(const Lower* a, const double* x, double* y, size_t n) {
    for (size_t i = 0; i < n; i++) y[i] = 0.0;
    for (size_t c = 0; c + 1 < a->colptr.size(); c++)
        for (size_t p = a->colptr[c]; p < a->colptr[c + 1]; p++) {
            size_t r = a->rowidx[p];
            double v = a->val[p];
            y[r] += v * x[c];
            if (r != c) y[c] += v * x[r];
        }
}

// src/solver/indefinite.rs:47-64 — up to two refinement steps
static double norm2(const double* v, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += v[i] * v[i];
    return std::sqrt(s);
}

static void refine(const double* b, double* x, size_t n, const std::function<void(const double*, double*)>& matvec,
                   const std::function<void(double*)>& solve_fn) {
    double bn = norm2(b, n);
    if (bn == 0.0) return;
    vector<double> ax(n), r(n);
    for (int it = 0; it < 2; it++) {
        matvec(x, ax.data());
        for (size_t i = 0; i < n; i++) r[i] = b[i] - ax[i];
        if (norm2(r.data(), n) <= 1e-13 * bn) return;
        solve_fn(r.data());
        for (size_t i = 0; i < n; i++) x[i] += r[i];
    }
}

// ---------------------------------------------------------------------------
// The C interface — ffi/src/lib.rs:17-407
// ---------------------------------------------------------------------------
static const size_t FFI_LEAF = 16;  // :17

enum Mode { PD, INDEF, LU };

struct Handle {  // :44-55
    Mode mode;
    Factor* pd = nullptr;
    indef::IndefFactor* idf = nullptr;
    lu::LuFactor* luf = nullptr;
    vector<size_t> eq;
    vector<std::pair<size_t, double>> iso;
    size_t n_sym = 0;
    double work = 0.0;
    size_t factor_size = 0;
    int64_t inertia[3] = {0, 0, 0};
    // kept for diagnostics: the symbolic data of the handle
    Symbolic* sym = nullptr;
    ~Handle() {
        delete pd;
        delete idf;
        delete luf;
        delete sym;
    }
};

static bool g_dump_fronts() { return getenv("RUSTYFEM_FRONTS") != nullptr; }

// A positive definite build stopped before the numeric factorization (used by the
// staged factorization of oref_staged_*): the handle with its analysis, the
// assembled lower matrix in the internal numbering and the internal→caller map.
struct PdStage {
    Handle* h = nullptr;
    Lower* K = nullptr;
    vector<size_t> owner;
};

// :100-229 — returns the handle, or nullptr with *err (the caller's DOF, or -1).
// With `stage` (PD only) it stops after assembling K and hands the pieces over.
static Handle* build(size_t n, size_t nn, const int64_t* loc_in, const double* coords, const int64_t* indptr,
                     const int64_t* indices, const double* data, Mode mode, vector<double>* d_out, int64_t* err,
                     PdStage* stage = nullptr) {
    *err = -1;
    vector<size_t> loc(n);
    for (size_t i = 0; i < n; i++) loc[i] = (size_t)loc_in[i];
    size_t nnz = (size_t)indptr[n];
    for (size_t i = 0; i < n; i++)
        if (loc_in[i] < 0 || loc[i] >= nn) return nullptr;
    for (size_t p = 0; p < nnz; p++)
        if (indices[p] < 0 || (size_t)indices[p] >= n) return nullptr;
    vector<bool> coupled(n, false);
    vector<double> diag(n, 0.0);
    for (size_t c = 0; c < n; c++)
        for (size_t p = (size_t)indptr[c]; p < (size_t)indptr[c + 1]; p++) {
            size_t r = (size_t)indices[p];
            if (r == c)
                diag[c] += data[p];
            else if (data[p] != 0.0) {
                coupled[c] = true;
                coupled[r] = true;
            }
        }
    Handle* h = new Handle();
    h->mode = mode;
    for (size_t i = 0; i < n; i++) {
        if (coupled[i]) continue;
        bool ok = (mode == PD) ? (diag[i] > 0.0) : (diag[i] != 0.0 && std::isfinite(diag[i]));
        if (!ok) {
            *err = (int64_t)i;
            delete h;
            return nullptr;
        }
        h->iso.push_back({i, diag[i]});
    }
    vector<size_t> nid(nn, NONE);
    vector<double> xyz;
    for (size_t i = 0; i < n; i++) {
        if (!coupled[i]) continue;
        size_t v = loc[i];
        if (nid[v] == NONE) {
            nid[v] = xyz.size() / 3;
            xyz.push_back(coords[3 * v]);
            xyz.push_back(coords[3 * v + 1]);
            xyz.push_back(coords[3 * v + 2]);
        }
    }
    size_t nc = xyz.size() / 3;
    vector<size_t> ndof(nc, 0), local(n, 0);
    for (size_t i = 0; i < n; i++) {
        if (!coupled[i]) continue;
        size_t v = nid[loc[i]];
        local[i] = ndof[v];
        ndof[v]++;
    }
    Adj adj(nc);
    for (size_t c = 0; c < n; c++) {
        if (!coupled[c]) continue;
        for (size_t p = (size_t)indptr[c]; p < (size_t)indptr[c + 1]; p++) {
            size_t r = (size_t)indices[p];
            if (coupled[r] && nid[loc[r]] != nid[loc[c]]) {
                adj[nid[loc[c]]].push_back(nid[loc[r]]);
                adj[nid[loc[r]]].push_back(nid[loc[c]]);
            }
        }
    }
    for (auto& a : adj) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    Symbolic* sym = analyse_with_leaf(nc, xyz.data(), adj, ndof.data(), FFI_LEAF);
    h->sym = sym;
    if (g_dump_fronts())
        for (auto& t : sym->tree) fprintf(stderr, "front %zu %zu %zu %zu\n", t.start, t.k, t.rows.size(), t.children.size());
    h->eq.assign(n, NONE);
    for (size_t i = 0; i < n; i++)
        if (coupled[i]) h->eq[i] = sym->first_dof[nid[loc[i]]] + local[i];
    vector<size_t> owner(sym->n, 0);
    for (size_t i = 0; i < n; i++)
        if (h->eq[i] != NONE) owner[h->eq[i]] = i;
    Lower* K = sym_pattern(sym, adj, ndof.data());
    h->n_sym = sym->n;
    h->work = sym_work(sym);
    if (mode == LU) {
        // :76-91 — all entries (both triangles), into the full matrix of the same pattern
        lu::Full full;
        full.lower = *K;
        full.upper_t.colptr = K->colptr;
        full.upper_t.rowidx = K->rowidx;
        full.upper_t.val.assign(K->val.size(), 0.0);
        delete K;
        for (size_t c = 0; c < n; c++) {
            if (!coupled[c]) continue;
            size_t qc = h->eq[c];
            for (size_t p = (size_t)indptr[c]; p < (size_t)indptr[c + 1]; p++) {
                size_t qr = h->eq[(size_t)indices[p]];
                if (qr != NONE) full.add(qr, qc, data[p]);
            }
        }
        long e = -1;
        lu::LuFactor* F = lu::factor_with(sym, &full, lu::THRESHOLD, &e);
        if (!F) {
            *err = (int64_t)owner[(size_t)e];
            delete h;
            return nullptr;
        }
        h->luf = F;
        h->factor_size = lu::factor_size(F);
        h->inertia[0] = h->inertia[1] = h->inertia[2] = -1;
        return h;
    }
    if (mode == INDEF) {
        for (size_t c = 0; c < n; c++) {
            if (!coupled[c]) continue;
            size_t qc = h->eq[c];
            for (size_t p = (size_t)indptr[c]; p < (size_t)indptr[c + 1]; p++) {
                size_t r = (size_t)indices[p];
                size_t qr = h->eq[r];
                if (qr != NONE && r >= c) K->add(std::max(qr, qc), std::min(qr, qc), data[p]);
            }
        }
        long e = -1;
        indef::IndefFactor* F = indef::factor_with(sym, K, indef::THRESHOLD, &e);
        delete K;
        if (!F) {
            *err = (int64_t)owner[(size_t)e];
            delete h;
            return nullptr;
        }
        indef::Inertia ine = F->inertia;
        for (auto& pr : h->iso) {
            if (pr.second < 0.0)
                ine.neg++;
            else
                ine.pos++;
        }
        h->idf = F;
        h->factor_size = indef::factor_size(F);
        h->inertia[0] = (int64_t)ine.neg;
        h->inertia[1] = (int64_t)ine.zero;
        h->inertia[2] = (int64_t)ine.pos;
        return h;
    }
    for (size_t c = 0; c < n; c++) {
        if (!coupled[c]) continue;
        size_t qc = h->eq[c];
        for (size_t p = (size_t)indptr[c]; p < (size_t)indptr[c + 1]; p++) {
            size_t qr = h->eq[(size_t)indices[p]];
            if (qr != NONE && qr >= qc) K->add(qr, qc, data[p]);
        }
    }
    if (stage) {
        h->factor_size = sym_factor_size(sym);
        h->inertia[0] = 0;
        h->inertia[1] = 0;
        h->inertia[2] = (int64_t)n;
        stage->h = h;
        stage->K = K;
        stage->owner = std::move(owner);
        return h;
    }
    long e = -1;
    Factor* F = factor(sym, K, &e);
    delete K;
    if (!F) {
        *err = (int64_t)owner[(size_t)e];
        delete h;
        return nullptr;
    }
    if (d_out) {
        vector<double> dq(sym->n, 0.0);
        pivots(F, dq.data());
        d_out->assign(n, 0.0);
        for (size_t i = 0; i < n; i++) (*d_out)[i] = coupled[i] ? dq[h->eq[i]] : diag[i];
    }
    h->pd = F;
    h->factor_size = sym_factor_size(sym);
    h->inertia[0] = 0;
    h->inertia[1] = 0;
    h->inertia[2] = (int64_t)n;
    return h;
}

}  // namespace oref

using namespace oref;

// ---------------------------------------------------------------------------
// Exported C functions. oref_factor … oref_free have the signatures of the
// reference's rustyfem_factor … rustyfem_free (ffi/src/lib.rs:64-407).
// ---------------------------------------------------------------------------
extern "C" {

void oref_set_threads(int t) { g_threads = t; }
int oref_threads(void) { return (int)threads(); }
int oref_uses_fma(void) { return kern::avx() ? 1 : 0; }

// ffi/src/lib.rs:64-97
void* oref_factor(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                  const int64_t* indices, const double* data, double* d_out, int64_t* err_dof) {
    vector<double> d;
    Handle* h = build(n, nn, loc, coords, indptr, indices, data, PD, d_out ? &d : nullptr, err_dof);
    if (h && d_out) std::copy(d.begin(), d.end(), d_out);
    return h;
}

// ffi/src/lib.rs:273-290
void* oref_factor_indef(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                        const int64_t* indices, const double* data, int64_t* inertia_out, int64_t* err_dof) {
    Handle* h = build(n, nn, loc, coords, indptr, indices, data, INDEF, nullptr, err_dof);
    if (h && inertia_out) std::copy(h->inertia, h->inertia + 3, inertia_out);
    return h;
}

// ffi/src/lib.rs:320-329
int32_t oref_inertia(const void* hp, int64_t* out) {
    const Handle* h = (const Handle*)hp;
    if (h->luf) return -1;  // no inertia for an LU handle (:320-329)
    std::copy(h->inertia, h->inertia + 3, out);
    return 0;
}

// ffi/src/lib.rs:300-311 — multifrontal LU of an unsymmetric matrix (CSC with both triangles)
void* oref_factor_unsym(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                        const int64_t* indices, const double* data, int64_t* err_dof) {
    return build(n, nn, loc, coords, indptr, indices, data, LU, nullptr, err_dof);
}

// Delayed pivots of an LU handle (the reference's LuFactor::delayed), -1 for other handles.
int64_t oref_lu_delayed(const void* hp) {
    const Handle* h = (const Handle*)hp;
    return h->luf ? (int64_t)h->luf->delayed : -1;
}

// ffi/src/lib.rs:337-371 (right-hand sides solved in parallel)
int32_t oref_solve(const void* hp, size_t nrhs, double* b) {
    const Handle* h = (const Handle*)hp;
    size_t n = h->eq.size();
    if (n == 0 || nrhs == 0) return 0;
    auto one = [&](double* col) {
        vector<double> x(h->n_sym, 0.0);
        for (size_t i = 0; i < n; i++)
            if (h->eq[i] != NONE) x[h->eq[i]] = col[i];
        if (h->pd)
            solve(h->pd, x.data());
        else if (h->luf)
            lu::solve(h->luf, x.data());
        else
            indef::solve(h->idf, x.data());
        for (size_t i = 0; i < n; i++)
            if (h->eq[i] != NONE) col[i] = x[h->eq[i]];
        for (auto& pr : h->iso) col[pr.first] /= pr.second;
    };
    size_t t = std::min(threads(), nrhs);
    if (t <= 1) {
        for (size_t j = 0; j < nrhs; j++) one(b + j * n);
    } else {
        size_t per = (nrhs + t - 1) / t;
        vector<std::thread> th;
        for (size_t j0 = 0; j0 < nrhs; j0 += per) {
            size_t j1 = std::min(j0 + per, nrhs);
            th.emplace_back([&, j0, j1] {
                for (size_t j = j0; j < j1; j++) one(b + j * n);
            });
        }
        for (auto& x : th) x.join();
    }
    return 0;
}

// ffi/src/lib.rs:378-383
void oref_info(const void* hp, double* out) {
    const Handle* h = (const Handle*)hp;
    out[0] = h->work;
    out[1] = (double)h->factor_size;
}

// ffi/src/lib.rs:391-398
void oref_order(const void* hp, int64_t* out) {
    const Handle* h = (const Handle*)hp;
    size_t next = h->n_sym;
    for (size_t i = 0; i < h->eq.size(); i++) {
        if (h->eq[i] == NONE) {
            next++;
            out[i] = (int64_t)(next - 1);
        } else {
            out[i] = (int64_t)h->eq[i];
        }
    }
}

// ffi/src/lib.rs:403-407
void oref_free(void* hp) { delete (Handle*)hp; }

// ---------------------------------------------------------------------------
// Staged positive definite factorization (no counterpart in the reference): one
// rustyfem_factor call cut into consecutive parts, so that a benchmark can time a
// whole factorization in slices of bounded length. oref_staged_begin does the
// analysis (everything rustyfem_factor does before the numeric phase); the parts
// then go up the elimination tree by depth: part 0 factors every subtree whose
// root lies at depth D = nparts - 1 (root depth 0), part p ≥ 1 the fronts at
// depth D - p, whose children the parts before finished; oref_staged_finish
// returns the handle. Every front runs the same factor_node code on the same
// inputs as in oref_factor, so the factor is bit for bit the same. Each front (or
// subtree) of a part gets the threads the plain recursion gives it (halved at each
// parallel split of :466-475) and the fronts of a part run concurrently while their
// threads fit in the total, which is the plain recursion's schedule with a join at
// the end of each depth.
// ---------------------------------------------------------------------------
struct Staged {
    PdStage st;
    Stash stash;
    vector<size_t> parent, nt, depth;
    vector<double> part_work;
    size_t dmax = 0;
    Factor* F = nullptr;
    long err = -1;
    size_t next = 0;
    ~Staged() {
        delete st.h;
        delete st.K;
        delete F;
    }
};

void* oref_staged_begin(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                        const int64_t* indices, const double* data, size_t nparts, int64_t* err_dof) {
    Staged* S = new Staged();
    if (!build(n, nn, loc, coords, indptr, indices, data, PD, nullptr, err_dof, &S->st)) {
        delete S;
        return nullptr;
    }
    const Symbolic* sym = S->st.h->sym;
    size_t nf = sym->tree.size();
    nparts = std::max<size_t>(nparts, 1);
    S->dmax = nparts - 1;
    S->parent.assign(nf, NONE);
    for (size_t t = 0; t < nf; t++)
        for (size_t c : sym->tree[t].children) S->parent[c] = t;
    // depth and the threads of each subtree in the plain recursion (children have
    // lower indices than their parent, so one pass from the top sets both)
    S->nt.assign(nf, 0);
    S->depth.assign(nf, 0);
    for (size_t r : sym->roots) S->nt[r] = threads();
    for (size_t t = nf; t-- > 0;) {
        const auto& ch = sym->tree[t].children;
        size_t T = S->nt[t];
        bool split = ch.size() == 2 && T > 1 && std::min(sym->tree[ch[0]].work, sym->tree[ch[1]].work) > 2e7;
        for (size_t i = 0; i < ch.size(); i++) {
            S->nt[ch[i]] = split ? (i == 0 ? T / 2 : T - T / 2) : T;
            S->depth[ch[i]] = S->depth[t] + 1;
        }
    }
    S->part_work.assign(nparts, 0.0);
    for (size_t t = 0; t < nf; t++) {
        double cw = 0.0;
        for (size_t c : sym->tree[t].children) cw += sym->tree[c].work;
        size_t d = S->depth[t];
        S->part_work[d >= S->dmax ? 0 : S->dmax - d] += sym->tree[t].work - cw;
    }
    S->stash.done.assign(nf, 0);
    S->stash.res.resize(nf);
    S->F = new Factor();
    return S;
}

size_t oref_staged_nparts(const void* sp) { return ((const Staged*)sp)->part_work.size(); }
double oref_staged_part_work(const void* sp, size_t p) { return ((const Staged*)sp)->part_work[p]; }

// Runs part p (parts in order). 0, or -1 when a pivot failed (here or earlier).
int32_t oref_staged_part(void* sp, size_t p) {
    Staged* S = (Staged*)sp;
    if (p != S->next || p >= S->part_work.size()) return -1;
    S->next++;
    if (S->err >= 0) return -1;
    const Symbolic* sym = S->st.h->sym;
    const size_t d = S->dmax - p;
    vector<size_t> top;  // the part's fronts (subtrees for part 0), in tree order
    for (size_t t = 0; t < sym->tree.size(); t++)
        if (S->depth[t] == d) top.push_back(t);
    vector<NodeResult> res(top.size());
    const size_t T = threads();
    std::mutex mu;
    std::condition_variable cv;
    size_t used = 0;
    vector<std::thread> running;
    for (size_t i = 0; i < top.size(); i++) {
        size_t want = std::max<size_t>(1, std::min(S->nt[top[i]], T));
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return used == 0 || used + want <= T; });
            used += want;
        }
        running.emplace_back([&, i, want] {
            res[i] = factor_node(sym, S->st.K, top[i], want, &S->stash);
            std::lock_guard<std::mutex> lk(mu);
            used -= want;
            cv.notify_all();
        });
    }
    for (auto& th : running) th.join();
    for (size_t i = 0; i < top.size(); i++) {
        size_t t = top[i];
        if (res[i].err >= 0) {
            if (S->err < 0) S->err = res[i].err;
            continue;
        }
        if (S->parent[t] == NONE) {
            for (auto& fr : res[i].fronts) S->F->fronts.push_back(std::move(fr));
        } else {
            S->stash.res[t] = std::move(res[i]);
            S->stash.done[t] = 1;
        }
    }
    return S->err >= 0 ? -1 : 0;
}

// After the last part: the factor handle (as oref_factor returns it), or nullptr
// with *err_dof = the caller's DOF of the failing pivot. Frees the stage.
void* oref_staged_finish(void* sp, int64_t* err_dof) {
    Staged* S = (Staged*)sp;
    *err_dof = -1;
    Handle* h = nullptr;
    if (S->err >= 0) {
        *err_dof = (int64_t)S->st.owner[(size_t)S->err];
    } else if (S->next == S->part_work.size()) {
        h = S->st.h;
        h->pd = S->F;
        S->st.h = nullptr;
        S->F = nullptr;
    }
    delete S;
    return h;
}

// Diagnostics of a handle: number of fronts and the (start, k, u, children)
// list of the handle's symbolic analysis (the RUSTYFEM_FRONTS dump).
size_t oref_handle_nfronts(const void* hp) { return ((const Handle*)hp)->sym->tree.size(); }
void oref_handle_fronts(const void* hp, int64_t* out4) {
    const Handle* h = (const Handle*)hp;
    size_t i = 0;
    for (auto& t : h->sym->tree) {
        out4[4 * i] = (int64_t)t.start;
        out4[4 * i + 1] = (int64_t)t.k;
        out4[4 * i + 2] = (int64_t)t.rows.size();
        out4[4 * i + 3] = (int64_t)t.children.size();
        i++;
    }
}

// --- engine-level API (src/sparse.rs analyse / pattern / factor / solve) ---

static Adj make_adj(size_t nn, const int64_t* adj_ptr, const int64_t* adj_idx) {
    Adj adj(nn);
    for (size_t v = 0; v < nn; v++)
        for (int64_t p = adj_ptr[v]; p < adj_ptr[v + 1]; p++) adj[v].push_back((size_t)adj_idx[p]);
    return adj;
}

struct SymBundle {
    Symbolic* sym;
    Adj adj;
    vector<size_t> ndof;
    ~SymBundle() { delete sym; }
};

void* oref_analyse(size_t nn, const double* coords, const int64_t* adj_ptr, const int64_t* adj_idx,
                   const int64_t* ndof, size_t leaf) {
    SymBundle* b = new SymBundle();
    b->adj = make_adj(nn, adj_ptr, adj_idx);
    b->ndof.resize(nn);
    for (size_t i = 0; i < nn; i++) b->ndof[i] = (size_t)ndof[i];
    b->sym = analyse_with_leaf(nn, coords, b->adj, b->ndof.data(), leaf);
    return b;
}
void oref_sym_free(void* p) { delete (SymBundle*)p; }
size_t oref_sym_n(const void* p) { return ((const SymBundle*)p)->sym->n; }
size_t oref_sym_nfronts(const void* p) { return ((const SymBundle*)p)->sym->tree.size(); }
double oref_sym_work(const void* p) { return sym_work(((const SymBundle*)p)->sym); }
size_t oref_sym_factor_size(const void* p) { return sym_factor_size(((const SymBundle*)p)->sym); }
size_t oref_sym_total_rows(const void* p) {
    size_t z = 0;
    for (auto& t : ((const SymBundle*)p)->sym->tree) z += t.rows.size();
    return z;
}
// per front: start, k, u, nchildren (4 entries each)
void oref_sym_fronts(const void* p, int64_t* out4) {
    size_t i = 0;
    for (auto& t : ((const SymBundle*)p)->sym->tree) {
        out4[4 * i] = (int64_t)t.start;
        out4[4 * i + 1] = (int64_t)t.k;
        out4[4 * i + 2] = (int64_t)t.rows.size();
        out4[4 * i + 3] = (int64_t)t.children.size();
        i++;
    }
}
void oref_sym_first_dof(const void* p, int64_t* out) {
    auto& fd = ((const SymBundle*)p)->sym->first_dof;
    for (size_t i = 0; i < fd.size(); i++) out[i] = (int64_t)fd[i];
}
void oref_sym_rows(const void* p, int64_t* out) {
    size_t z = 0;
    for (auto& t : ((const SymBundle*)p)->sym->tree)
        for (size_t r : t.rows) out[z++] = (int64_t)r;
}
// children indices (into the front list), concatenated
void oref_sym_children(const void* p, int64_t* out) {
    size_t z = 0;
    for (auto& t : ((const SymBundle*)p)->sym->tree)
        for (size_t c : t.children) out[z++] = (int64_t)c;
}
size_t oref_sym_nnz(const void* p) {
    const SymBundle* b = (const SymBundle*)p;
    Lower* L = sym_pattern(b->sym, b->adj, b->ndof.data());
    size_t z = L->rowidx.size();
    delete L;
    return z;
}
// The CSC lower pattern (colptr n+1, rowidx nnz) in the internal numbering.
void oref_sym_pattern(const void* p, int64_t* colptr, int64_t* rowidx) {
    const SymBundle* b = (const SymBundle*)p;
    Lower* L = sym_pattern(b->sym, b->adj, b->ndof.data());
    for (size_t i = 0; i < L->colptr.size(); i++) colptr[i] = (int64_t)L->colptr[i];
    for (size_t i = 0; i < L->rowidx.size(); i++) rowidx[i] = (int64_t)L->rowidx[i];
    delete L;
}

static Lower* lower_from(size_t n, const int64_t* colptr, const int64_t* rowidx, const double* val) {
    Lower* L = new Lower();
    L->colptr.resize(n + 1);
    for (size_t i = 0; i <= n; i++) L->colptr[i] = (size_t)colptr[i];
    size_t nnz = L->colptr[n];
    L->rowidx.resize(nnz);
    L->val.resize(nnz);
    for (size_t i = 0; i < nnz; i++) {
        L->rowidx[i] = (size_t)rowidx[i];
        L->val[i] = val[i];
    }
    return L;
}

struct PdBundle {
    Factor* F;
    ~PdBundle() { delete F; }
};

// src/sparse.rs:595-602 on a lower CSC in the internal numbering; *err = internal equation or -1
void* oref_pd_factor(const void* symp, const int64_t* colptr, const int64_t* rowidx, const double* val, int64_t* err) {
    const SymBundle* b = (const SymBundle*)symp;
    Lower* L = lower_from(b->sym->n, colptr, rowidx, val);
    long e = -1;
    Factor* F = factor(b->sym, L, &e);
    delete L;
    *err = e;
    if (!F) return nullptr;
    PdBundle* pb = new PdBundle{F};
    return pb;
}
void oref_pd_solve(const void* p, double* x) { solve(((const PdBundle*)p)->F, x); }
void oref_pd_pivots(const void* p, double* d) { pivots(((const PdBundle*)p)->F, d); }
void oref_pd_free(void* p) { delete (PdBundle*)p; }

struct IdBundle {
    indef::IndefFactor* F;
    ~IdBundle() { delete F; }
};

// src/sparse/indef.rs:116-156
void* oref_indef_factor(const void* symp, const int64_t* colptr, const int64_t* rowidx, const double* val,
                        double threshold, int64_t* err) {
    const SymBundle* b = (const SymBundle*)symp;
    Lower* L = lower_from(b->sym->n, colptr, rowidx, val);
    long e = -1;
    indef::IndefFactor* F = indef::factor_with(b->sym, L, threshold, &e);
    delete L;
    *err = e;
    if (!F) return nullptr;
    return new IdBundle{F};
}
void oref_indef_solve(const void* p, double* x) { indef::solve(((const IdBundle*)p)->F, x); }
// neg, zero, pos, delayed, two_by_two, factor_size
void oref_indef_stats(const void* p, int64_t* out6) {
    const indef::IndefFactor* F = ((const IdBundle*)p)->F;
    out6[0] = (int64_t)F->inertia.neg;
    out6[1] = (int64_t)F->inertia.zero;
    out6[2] = (int64_t)F->inertia.pos;
    out6[3] = (int64_t)F->delayed;
    out6[4] = (int64_t)F->two_by_two;
    out6[5] = (int64_t)indef::factor_size(F);
}
void oref_indef_free(void* p) { delete (IdBundle*)p; }

// src/sparse/indef.rs:600-611
void oref_sym_matvec(size_t n, const int64_t* colptr, const int64_t* rowidx, const double* val, const double* x,
                     double* y) {
    Lower* L = lower_from(n, colptr, rowidx, val);
    sym_matvec(L, x, y, n);
    delete L;
}

// src/solver/indefinite.rs:47-64 + 264-269: indefinite solve followed by up to
// two refinement steps against the lower CSC.
void oref_indef_solve_refined(const void* p, size_t n, const int64_t* colptr, const int64_t* rowidx, const double* val,
                              double* b) {
    const indef::IndefFactor* F = ((const IdBundle*)p)->F;
    Lower* L = lower_from(n, colptr, rowidx, val);
    vector<double> rhs(b, b + n);
    indef::solve(F, b);
    refine(rhs.data(), b, n, [&](const double* x, double* y) { sym_matvec(L, x, y, n); },
           [&](double* r) { indef::solve(F, r); });
    delete L;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Assembly of K — src/fem/assembly.rs:315-420 (the element loop of `internal`,
// symmetric system matrix, no constraints), with the C3D8 linear-elastic
// element matrix of src/elements/continuum3d.rs:39-131 (2×2×2 Gauss points,
// volumetric B-bar: src/elements/common.rs:142-218), the tangent of
// src/elements/common.rs:308-380 (add_btdb per integration point, :264-289)
// and isotropic elasticity (src/materials/elastic.rs:47-72). Every product and
// sum is rounded separately, in the reference's order (this file is built
// with -ffp-contract=off).
// ---------------------------------------------------------------------------
namespace assembly {

const double G2 = 0.5773502691896258;  // 1/√3 (src/elements/continuum3d.rs)
const double HEX8_NAT[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                               {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// src/elements/common.rs:48-70
static double inv3(const double m[3][3], double inv[3][3]) {
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    double id = 1.0 / det;
    inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
    return det;
}

// K_e of one C3D8 (x: 8 nodes × 3, row-major ke 24 × 24). False if an integration
// point has det J <= 0 (src/elements/continuum3d.rs:55-57, a distorted element).
static bool ke_hex8(const double* x, double E, double nu, double* ke) {
    const int nd = 24, ns = 6;
    double B[8][ns * nd];
    double w[8];
    int q = 0;
    const double gp[2] = {-G2, G2};
    for (double zeta : gp)  // src/elements/continuum3d.rs:73-84: ξ fastest, then η, then ζ
        for (double eta : gp)
            for (double xi : gp) {
                const double p[3] = {xi, eta, zeta};
                double dn[3][8];
                for (int i = 0; i < 8; i++) {  // :39-49
                    const double* nat = HEX8_NAT[i];
                    const double f0 = 1.0 + p[0] * nat[0], f1 = 1.0 + p[1] * nat[1], f2 = 1.0 + p[2] * nat[2];
                    dn[0][i] = 0.125 * nat[0] * f1 * f2;
                    dn[1][i] = 0.125 * nat[1] * f0 * f2;
                    dn[2][i] = 0.125 * nat[2] * f0 * f1;
                }
                double J[3][3];
                for (int r = 0; r < 3; r++)  // :50-55
                    for (int c = 0; c < 3; c++) {
                        double s = 0.0;
                        for (int i = 0; i < 8; i++) s += dn[r][i] * x[i * 3 + c];
                        J[r][c] = s;
                    }
                double ji[3][3];
                const double det = inv3(J, ji);
                if (det <= 0.0) return false;
                double* b = B[q];
                for (int k = 0; k < ns * nd; k++) b[k] = 0.0;
                for (int i = 0; i < 8; i++) {  // :59-68, then the B matrix (common.rs:142-171)
                    double d[3];
                    for (int c = 0; c < 3; c++) {
                        double s = 0.0;
                        for (int r = 0; r < 3; r++) s += ji[c][r] * dn[r][i];
                        d[c] = s;
                    }
                    const int c = 3 * i;
                    b[c] = d[0];
                    b[nd + c + 1] = d[1];
                    b[2 * nd + c + 2] = d[2];
                    b[3 * nd + c] = d[1];
                    b[3 * nd + c + 1] = d[0];
                    b[4 * nd + c] = d[2];
                    b[4 * nd + c + 2] = d[0];
                    b[5 * nd + c + 1] = d[2];
                    b[5 * nd + c + 2] = d[1];
                }
                w[q] = det * 1.0;
                q++;
            }
    // volumetric B-bar (src/elements/common.rs:174-200)
    auto vol = [&](const double* b, int c) { return b[c] + b[nd + c] + b[2 * nd + c]; };
    double wsum = 0.0;
    for (int k = 0; k < 8; k++) wsum += w[k];
    double avg[nd];
    for (int c = 0; c < nd; c++) {
        double s = 0.0;
        for (int k = 0; k < 8; k++) s += w[k] * vol(B[k], c);
        avg[c] = s / wsum;
    }
    for (int k = 0; k < 8; k++)
        for (int c = 0; c < nd; c++) {
            const double corr = (avg[c] - vol(B[k], c)) / 3.0;
            for (int r = 0; r < 3; r++) B[k][r * nd + c] += corr;
        }
    // isotropic elasticity (src/materials/elastic.rs:57-70)
    double D[ns * ns] = {};
    const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) D[i * ns + j] = lam;
        D[i * ns + i] = lam + 2.0 * mu;
    }
    for (int i = 3; i < ns; i++) D[i * ns + i] = mu;
    // K = Σ_q Bᵀ D B w (src/elements/common.rs:264-289)
    for (int k = 0; k < nd * nd; k++) ke[k] = 0.0;
    double db[ns * nd];
    for (int k = 0; k < 8; k++) {
        const double* b = B[k];
        for (int i = 0; i < ns * nd; i++) db[i] = 0.0;
        for (int r = 0; r < ns; r++)
            for (int m = 0; m < ns; m++) {
                const double drm = D[r * ns + m];
                if (drm != 0.0)
                    for (int c = 0; c < nd; c++) db[r * nd + c] += drm * b[m * nd + c];
            }
        for (int r = 0; r < ns; r++)
            for (int i = 0; i < nd; i++) {
                const double bri = b[r * nd + i] * w[k];
                if (bri != 0.0)
                    for (int j = 0; j < nd; j++) ke[i * nd + j] += bri * db[r * nd + j];
            }
    }
    return true;
}

// Lower::add (src/sparse.rs:47-51): false when (r, c) is not in the pattern
static bool lower_add(const int64_t* colptr, const int64_t* rowidx, double* val, int64_t r, int64_t c, double v) {
    const int64_t* b = rowidx + colptr[c];
    const int64_t* e = rowidx + colptr[c + 1];
    const int64_t* it = std::lower_bound(b, e, r);
    if (it == e || *it != r) return false;
    val[it - rowidx] += v;
    return true;
}

// the symmetric branch of src/fem/assembly.rs:388-412 for element e
static int64_t add_element(const int64_t* colptr, const int64_t* rowidx, double* val, int64_t nd, const int64_t* map,
                           const double* ke, int64_t* bad) {
    for (int64_t a = 0; a < nd; a++) {
        const int64_t ia = map[a];
        if (ia < 0) continue;
        for (int64_t b = 0; b < nd; b++) {
            const int64_t ib = map[b];
            if (ib < 0) continue;
            if (ia >= ib) {
                const double v = 0.5 * (ke[a * nd + b] + ke[b * nd + a]);
                if (v != 0.0 && !lower_add(colptr, rowidx, val, ia, ib, v)) {
                    bad[0] = ia;
                    bad[1] = ib;
                    return -1;
                }
            }
        }
    }
    return 0;
}

}  // namespace assembly

extern "C" {

// The element matrix of one C3D8 (x: 8×3 node coordinates). 0, or -1 for a distorted element.
int32_t oref_ke_hex8(const double* x, double E, double nu, double* ke) {
    return assembly::ke_hex8(x, E, nu, ke) ? 0 : -1;
}

// K (values of the lower CSC colptr/rowidx, internal numbering) = zero, then the
// element matrices ke (nelem × nd × nd) added in element order through their
// equation maps edof (nelem × nd, -1 = no equation). 0, or -1 with bad = the
// (row, column) missing in the pattern.
int32_t oref_assemble(size_t n, const int64_t* colptr, const int64_t* rowidx, size_t nelem, size_t nd,
                      const int64_t* edof, const double* ke, double* val, int64_t* bad) {
    for (int64_t p = 0; p < colptr[n]; p++) val[p] = 0.0;  // SystemMatrix::zero
    for (size_t e = 0; e < nelem; e++)
        if (assembly::add_element(colptr, rowidx, val, (int64_t)nd, edof + e * nd, ke + e * nd * nd, bad) != 0)
            return -1;
    return 0;
}

// The whole of `internal`'s tangent assembly for a C3D8 mesh (conn: nelem × 8 node ids,
// xyz: 3 per node, emod: E per element): the element matrices in blocks of 8192
// elements, each block's elements in parallel (src/par.rs:8-29), then added in
// element order. 0, -1 (pattern) or -2 (distorted element, bad[0] = element).
int32_t oref_assemble_hex8(size_t n, const int64_t* colptr, const int64_t* rowidx, size_t nelem, const int64_t* conn,
                           const double* xyz, const double* emod, double nu, const int64_t* edof, double* val,
                           int64_t* bad) {
    for (int64_t p = 0; p < colptr[n]; p++) val[p] = 0.0;
    const size_t BLOCK = 8192, nd = 24;
    vector<double> ke(BLOCK * nd * nd);
    vector<char> ok(BLOCK);
    for (size_t b0 = 0; b0 < nelem; b0 += BLOCK) {
        const size_t nb = std::min(BLOCK, nelem - b0);
        const size_t t = std::max<size_t>(std::min(threads(), nb), 1);
        vector<std::thread> th;
        for (size_t w = 0; w < t; w++)
            th.emplace_back([&, w] {
                for (size_t i = nb * w / t; i < nb * (w + 1) / t; i++) {
                    double x[24];
                    for (int a = 0; a < 8; a++)
                        for (int c = 0; c < 3; c++) x[a * 3 + c] = xyz[conn[(b0 + i) * 8 + a] * 3 + c];
                    ok[i] = assembly::ke_hex8(x, emod[b0 + i], nu, ke.data() + i * nd * nd);
                }
            });
        for (auto& x : th) x.join();
        for (size_t i = 0; i < nb; i++) {
            if (!ok[i]) {
                bad[0] = (int64_t)(b0 + i);
                return -2;
            }
            if (assembly::add_element(colptr, rowidx, val, (int64_t)nd, edof + (b0 + i) * nd, ke.data() + i * nd * nd,
                                      bad) != 0)
                return -1;
        }
    }
    return 0;
}

// The restated slice::sort_unstable_by on the indices 0..n by key (limit < 0: the
// default imbalance budget): perm receives the sorted indices.
void oref_sort_unstable_keys(const int64_t* keys, size_t n, long limit, int64_t* perm) {
    vector<int64_t> v(n);
    for (size_t i = 0; i < n; i++) v[i] = (int64_t)i;
    rsort::sort_unstable(v.data(), n, [&](int64_t a, int64_t b) { return keys[a] < keys[b]; }, limit);
    std::copy(v.begin(), v.end(), perm);
}

}  // extern "C"

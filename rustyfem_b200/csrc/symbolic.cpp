// Host symbolic stage (see symbolic.h).
//
// The nested dissection works in place on one permutation array: every call
// owns a contiguous range of it, sorts and stably partitions that range, and
// hands disjoint sub-ranges to its two children, which may run on separate
// threads. Node-to-side marks carry the id of the set that wrote them, so a
// neighbour outside the current set never reads as being on one of its sides
// (the reference keeps side = 2 for such nodes, src/sparse.rs:116-152). The
// resulting tree, its push order and the node order inside every front are
// those of the recursive formulation in src/sparse.rs:78-157, with the
// coordinate sort's ties where Rust's sort_unstable_by leaves them.

#include "symbolic.h"

#include "par.h"
#include "sort_unstable.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <thread>

namespace rfg {

namespace {

struct TN {
    int64_t lo, hi;                 // the front's nodes: perm[lo..hi)
    std::vector<int64_t> children;  // indices into the same subtree list
};

struct Dissector {
    static constexpr int64_t PAR_SLAB = 4096;  // slab nodes from which a cut is counted on the pool
    const Graph& g;
    int64_t leaf;
    HostVec<int64_t> perm;
    HostVec<std::atomic<uint64_t>> mark;  // (set id << 1) | side
    std::atomic<uint64_t> next_id{1};
    std::atomic<int> spare_threads{0};

    double reach[3] = {0.0, 0.0, 0.0};  // largest |x(w) − x(v)| over the edges, per axis (with margin)
    double cmax[3] = {0.0, 0.0, 0.0};   // largest |x(v)| per axis

    Dissector(const Graph& gr, int64_t leaf_max) : g(gr), leaf(leaf_max), perm(gr.nn), mark(gr.nn) {
        for (int64_t i = 0; i < gr.nn; i++) {
            perm[i] = i;
            mark[i].store(0, std::memory_order_relaxed);
        }
        unsigned hw = std::thread::hardware_concurrency();
        spare_threads = (int)std::max(1u, hw) - 1;
        {
            std::mutex mu;
            parallel_chunks(gr.nn, 16384, [&](int64_t v0, int64_t v1) {
                double r[3] = {0.0, 0.0, 0.0}, c[3] = {0.0, 0.0, 0.0};
                for (int64_t v = v0; v < v1; v++) {
                    for (int a = 0; a < 3; a++) c[a] = std::fmax(c[a], std::fabs(x(v, a)));
                    for (int64_t p = gr.adj_ptr[v]; p < gr.adj_ptr[v + 1]; p++)
                        for (int a = 0; a < 3; a++) r[a] = std::fmax(r[a], std::fabs(x(gr.adj_idx[p], a) - x(v, a)));
                }
                std::lock_guard<std::mutex> lock(mu);
                for (int a = 0; a < 3; a++) {
                    reach[a] = std::fmax(reach[a], r[a]);
                    cmax[a] = std::fmax(cmax[a], c[a]);
                }
            });
        }
        // a node farther than this from a cut plane has no neighbour on the other side: a
        // left node v with a right neighbour w has x(v) >= t − (x(w) − x(v)). The margin covers
        // the rounding of the edge differences and of t ± reach (a few units in the last
        // place of the largest coordinate), so the slab test stays exact
        for (int a = 0; a < 3; a++)
            reach[a] = std::isfinite(reach[a]) && std::isfinite(cmax[a])
                           ? reach[a] + 64.0 * std::numeric_limits<double>::epsilon() * (cmax[a] + reach[a]) + 1e-300
                           : INFINITY;
        build_ranks();
    }

    double x(int64_t v, int a) const { return g.coords[3 * v + a]; }

    // s[0..n).sort_unstable_by(coordinate a), src/sparse.rs:108 (sort_unstable.h). The
    // keys are the nodes' dense ranks of that coordinate over the whole graph (equal
    // coordinates, equal rank; computed once), packed above the node index, so the sort
    // moves and compares plain 8-byte words.
    HostVec<uint32_t> rank[3];

    void build_ranks() {
        auto one = [&](int a) {
            // (coordinate, node) pairs sorted in place: the comparisons read contiguous memory;
            // the order among equal coordinates does not matter, they get the same rank
            HostVec<std::pair<double, int64_t>> ord(g.nn);
            for (int64_t i = 0; i < g.nn; i++) ord[i] = {x(i, a), i};
            std::sort(ord.begin(), ord.end(),
                      [](const std::pair<double, int64_t>& p, const std::pair<double, int64_t>& q) { return p.first < q.first; });
            rank[a].assign(g.nn, 0);
            uint32_t r = 0;
            for (int64_t i = 0; i < g.nn; i++) {
                if (i > 0 && ord[i - 1].first < ord[i].first) r++;
                rank[a][ord[i].second] = r;
            }
        };
        if (g.nn >= 65536) {
            auto f1 = std::async(std::launch::async, one, 1);
            auto f2 = std::async(std::launch::async, one, 2);
            one(0);
            f1.get();
            f2.get();
        } else {
            for (int a = 0; a < 3; a++) one(a);
        }
    }

    // the quicksort's left sides of 32k elements and more go to spare threads
    struct SortFork {
        std::atomic<int>& spare;
        bool take(int64_t n) {
            if (n < 32768) return false;
            if (spare.fetch_sub(1) > 0) return true;
            spare.fetch_add(1);
            return false;
        }
        void give() { spare.fetch_add(1); }
    };

    void sort_axis(int64_t* s, int64_t n, int a) {
        const uint32_t* rk = rank[a].data();
        if (g.nn <= (int64_t)UINT32_MAX + 1) {
            thread_local std::vector<uint64_t> kv;
            kv.resize(n);
            for (int64_t i = 0; i < n; i++) kv[i] = ((uint64_t)rk[s[i]] << 32) | (uint64_t)s[i];
            unstable_sort::sort(kv.data(), n, [](uint64_t p, uint64_t q) { return (p >> 32) < (q >> 32); },
                                SortFork{spare_threads});
            for (int64_t i = 0; i < n; i++) s[i] = (int64_t)(kv[i] & 0xffffffffu);
        } else {
            unstable_sort::sort(s, n, [rk](int64_t p, int64_t q) { return rk[p] < rk[q]; }, SortFork{spare_threads});
        }
    }

    bool touches(int64_t v, uint64_t want) const {
        for (int64_t p = g.adj_ptr[v]; p < g.adj_ptr[v + 1]; p++)
            if (mark[g.adj_idx[p]].load(std::memory_order_relaxed) == want) return true;
        return false;
    }

    // Returns the subtree of perm[lo..hi) in push order (children before parents).
    std::vector<TN> run(int64_t lo, int64_t hi) {
        std::vector<TN> out;
        int64_t n = hi - lo;
        if (n == 0) return out;
        if (n <= leaf) {
            out.push_back(TN{lo, hi, {}});
            return out;
        }
        int64_t* s = perm.data() + lo;
        double blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < n; i++)
            for (int a = 0; a < 3; a++) {
                blo[a] = std::fmin(blo[a], x(s[i], a));
                bhi[a] = std::fmax(bhi[a], x(s[i], a));
            }
        int axes[3] = {0, 1, 2};
        std::stable_sort(axes, axes + 3, [&](int a, int b) { return (bhi[a] - blo[a]) > (bhi[b] - blo[b]); });
        uint64_t id = next_id.fetch_add(1);
        const uint64_t L = id << 1, R = (id << 1) | 1;
        bool have = false, bleft = true;
        double bscore = 0.0, bt = 0.0;
        int bax = 0;
        for (int ax : axes) {
            if (!(bhi[ax] > blo[ax])) continue;
            sort_axis(s, n, ax);
            auto first_at = [&](double tv) {
                return (int64_t)(std::lower_bound(s, s + n, tv, [&](int64_t v, double c) { return x(v, ax) < c; }) - s);
            };
            const int64_t qs[3] = {n / 2, 2 * n / 5, 3 * n / 5};
            for (int64_t q : qs) {
                double t = x(s[q], ax);
                int64_t nl = first_at(t);
                if (nl == 0 || nl == n) continue;
                // only nodes within reach of the plane can have a neighbour across it, and
                // those neighbours are within reach too: marks (with an id of this cut, so
                // older marks never match) are needed on that slab only
                const int64_t i0 = std::min(nl, first_at(t - reach[ax]));
                const int64_t i1 = std::max(nl, first_at(t + reach[ax]));
                const uint64_t cid = next_id.fetch_add(1);
                const uint64_t cL = cid << 1, cR = (cid << 1) | 1;
                int64_t sep_l = 0, sep_r = 0;
                if (i1 - i0 >= PAR_SLAB) {
                    // large slabs (the top of the tree): marks, then counts, over the pool
                    // (counts of a set: the same sums in any order)
                    pool_chunks_or_serial(i1 - i0, PAR_SLAB / 4, [&](int64_t a, int64_t b) {
                        for (int64_t i = i0 + a; i < i0 + b; i++)
                            mark[s[i]].store(i >= nl ? cR : cL, std::memory_order_relaxed);
                    });
                    std::atomic<int64_t> al{0}, ar{0};
                    pool_chunks_or_serial(i1 - i0, PAR_SLAB / 4, [&](int64_t a, int64_t b) {
                        int64_t l = 0, r = 0;
                        for (int64_t i = i0 + a; i < i0 + b; i++) {
                            if (i < nl)
                                l += touches(s[i], cR);
                            else
                                r += touches(s[i], cL);
                        }
                        al.fetch_add(l, std::memory_order_relaxed);
                        ar.fetch_add(r, std::memory_order_relaxed);
                    });
                    sep_l = al.load();
                    sep_r = ar.load();
                } else {
                    for (int64_t i = i0; i < i1; i++) mark[s[i]].store(i >= nl ? cR : cL, std::memory_order_relaxed);
                    for (int64_t i = i0; i < nl; i++) sep_l += touches(s[i], cR);
                    for (int64_t i = nl; i < i1; i++) sep_r += touches(s[i], cL);
                }
                int64_t sz;
                bool in_left;
                if (sep_r < sep_l) {
                    sz = sep_r;
                    in_left = false;
                } else {
                    sz = sep_l;
                    in_left = true;
                }
                double score = (double)sz / ((double)std::min(nl, n - nl) / (double)n);
                if (!have || score < bscore) {
                    have = true;
                    bscore = score;
                    bax = ax;
                    bt = t;
                    bleft = in_left;
                }
            }
        }
        int64_t nl;
        if (have) {
            nl = (int64_t)(std::stable_partition(s, s + n, [&](int64_t v) { return x(v, bax) < bt; }) - s);
        } else {
            nl = n / 2;
        }
        bool in_left = have ? bleft : true;
        for (int64_t i = 0; i < n; i++) mark[s[i]].store(i >= nl ? R : L, std::memory_order_relaxed);
        int64_t sep_lo, sep_hi, a_lo, a_hi, b_lo, b_hi;
        if (in_left) {
            const double lim = have ? bt - reach[bax] : -INFINITY;
            int64_t ns = (int64_t)(std::stable_partition(s, s + nl, [&](int64_t v) {
                             return !(x(v, bax) < lim) && touches(v, R);
                         }) - s);
            sep_lo = lo;
            sep_hi = lo + ns;
            a_lo = lo + ns;
            a_hi = lo + nl;
            b_lo = lo + nl;
            b_hi = hi;
        } else {
            const double lim = have ? bt + reach[bax] : INFINITY;
            int64_t ns = (int64_t)(std::stable_partition(s + nl, s + n, [&](int64_t v) {
                             return x(v, bax) < lim && touches(v, L);
                         }) - (s + nl));
            sep_lo = lo + nl;
            sep_hi = lo + nl + ns;
            a_lo = lo;
            a_hi = lo + nl;
            b_lo = lo + nl + ns;
            b_hi = hi;
        }
        std::vector<TN> ta, tb;
        bool par = false;
        if ((a_hi - a_lo) > 4000 && (b_hi - b_lo) > 4000) {
            if (spare_threads.fetch_sub(1) > 0)
                par = true;
            else
                spare_threads.fetch_add(1);
        }
        if (par) {
            auto fa = std::async(std::launch::async, [&] { return run(a_lo, a_hi); });
            tb = run(b_lo, b_hi);
            ta = fa.get();
            spare_threads.fetch_add(1);
        } else {
            ta = run(a_lo, a_hi);
            tb = run(b_lo, b_hi);
        }
        out.reserve(ta.size() + tb.size() + 1);
        TN parent{sep_lo, sep_hi, {}};
        for (auto& t : ta) out.push_back(std::move(t));
        if (!ta.empty()) parent.children.push_back((int64_t)out.size() - 1);
        int64_t off = (int64_t)out.size();
        for (auto& t : tb) {
            for (auto& c : t.children) c += off;
            out.push_back(std::move(t));
        }
        if (!tb.empty()) parent.children.push_back((int64_t)out.size() - 1);
        out.push_back(std::move(parent));
        return out;
    }
};

}  // namespace

double Symbolic::work() const {
    double w = 0.0;
    for (int64_t r : roots) w += fronts[r].work;
    return w;
}

int64_t Symbolic::factor_size() const {
    int64_t z = 0;
    for (auto& f : fronts) z += f.k * (f.k > 0 ? f.k - 1 : 0) / 2 + f.k * f.u;
    return z;
}

void Symbolic::largest_front(int64_t* k, int64_t* u) const {
    // Iterator::max_by_key keeps the last of equal maxima
    *k = 0;
    *u = 0;
    int64_t best = -1;
    for (auto& f : fronts)
        if (f.k + f.u >= best) {
            best = f.k + f.u;
            *k = f.k;
            *u = f.u;
        }
}

Symbolic analyse(const Graph& g, int64_t leaf_max) {
    leaf_max = std::max<int64_t>(leaf_max, 1);
    HostTimer timer("analyse");
    Symbolic S;
    Dissector D(g, leaf_max);
    std::vector<TN> tree = D.run(0, g.nn);
    timer.lap("dissect");
    int64_t nt = (int64_t)tree.size();
    // postorder by an explicit depth-first walk from the root (src/sparse.rs:176-187)
    std::vector<int64_t> post;
    post.reserve(nt);
    if (nt > 0) {
        std::vector<std::pair<int64_t, bool>> st{{nt - 1, false}};
        S.roots.push_back(0);  // renumbered below
        while (!st.empty()) {
            auto [t, done] = st.back();
            st.pop_back();
            if (done) {
                post.push_back(t);
            } else {
                st.push_back({t, true});
                for (size_t i = tree[t].children.size(); i-- > 0;) st.push_back({tree[t].children[i], false});
            }
        }
    }
    std::vector<int64_t> newid(nt);
    for (int64_t i = 0; i < nt; i++) newid[post[i]] = i;
    if (nt > 0) S.roots[0] = newid[nt - 1];
    S.fronts.resize(nt);
    S.first_dof.assign(g.nn, 0);
    S.front_nodes_off.assign(nt + 1, 0);
    S.front_nodes.reserve(g.nn);
    int64_t next = 0;
    for (int64_t i = 0; i < nt; i++) {
        const TN& t = tree[post[i]];
        SymFront& f = S.fronts[i];
        f.start = next;
        for (int64_t p = t.lo; p < t.hi; p++) {
            int64_t v = D.perm[p];
            S.first_dof[v] = next;
            next += g.ndof[v];
            S.front_nodes.push_back(v);
        }
        S.front_nodes_off[i + 1] = (int64_t)S.front_nodes.size();
        f.k = next - f.start;
        f.child_off = (int64_t)S.children.size();
        f.nchild = (int64_t)t.children.size();
        for (int64_t c : t.children) {
            S.children.push_back(newid[c]);
            S.fronts[newid[c]].parent = i;
        }
    }
    S.n = next;
    timer.lap("postorder");
    // front patterns (src/sparse.rs:201-230). A front needs only its children's
    // node lists, so the fronts of one height (leaves 0, a parent one above its highest
    // child) are independent and run in parallel; rows are concatenated in postorder
    // afterwards.
    std::vector<int64_t> height(nt, 0);
    int64_t hmax = 0;
    for (int64_t t = 0; t < nt; t++) {
        const SymFront& f = S.fronts[t];
        for (int64_t c = 0; c < f.nchild; c++) height[t] = std::max(height[t], height[S.children[f.child_off + c]] + 1);
        hmax = std::max(hmax, height[t]);
    }
    std::vector<std::vector<int64_t>> by_h(nt > 0 ? hmax + 1 : 0);
    for (int64_t t = 0; t < nt; t++) by_h[height[t]].push_back(t);
    std::vector<std::vector<int64_t>> unodes(nt), rows_t(nt);
    static std::atomic<int64_t> call_counter{0};
    const int64_t call_id = ++call_counter;
    const int64_t nthreads = std::max(1u, std::thread::hardware_concurrency());
    for (auto& level : by_h) {
        // chunks of up to 16 fronts, fewer near the top so that a height of a few large fronts
        // still runs on several threads
        const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(16, (int64_t)level.size() / (4 * nthreads)));
        parallel_chunks((int64_t)level.size(), chunk, [&](int64_t a0, int64_t a1) {
            // per-thread marks: the mark of node w is (call, front) of the front that took it
            thread_local std::vector<std::pair<int64_t, int64_t>> stamp;
            if ((int64_t)stamp.size() < g.nn) stamp.assign(g.nn, {0, -1});
            for (int64_t li = a0; li < a1; li++) {
                int64_t t = level[li];
                SymFront& f = S.fronts[t];
                int64_t end = f.start + f.k;
                std::vector<int64_t> list;
                auto take = [&](int64_t w) {
                    if (S.first_dof[w] >= end && !(stamp[w].first == call_id && stamp[w].second == t)) {
                        stamp[w] = {call_id, t};
                        list.push_back(w);
                    }
                };
                for (int64_t p = S.front_nodes_off[t]; p < S.front_nodes_off[t + 1]; p++) {
                    int64_t v = S.front_nodes[p];
                    for (int64_t q = g.adj_ptr[v]; q < g.adj_ptr[v + 1]; q++) take(g.adj_idx[q]);
                }
                for (int64_t c = 0; c < f.nchild; c++)
                    for (int64_t w : unodes[S.children[f.child_off + c]]) take(w);
                std::sort(list.begin(), list.end(),
                          [&](int64_t x0, int64_t x1) { return S.first_dof[x0] < S.first_dof[x1]; });
                std::vector<int64_t>& rt = rows_t[t];
                for (int64_t w : list)
                    for (int64_t q = S.first_dof[w]; q < S.first_dof[w] + g.ndof[w]; q++) rt.push_back(q);
                const int64_t u = (int64_t)rt.size();
                f.u = u;
                double k = (double)f.k, ud = (double)u;
                double own = k * k * k / 3.0 + ud * k * k + ud * ud * k;
                double cw = 0.0;
                for (int64_t c = 0; c < f.nchild; c++) cw += S.fronts[S.children[f.child_off + c]].work;
                f.work = own + cw;
                unodes[t] = std::move(list);
            }
        });
        // the children's lists are no longer needed once their parents have theirs
        for (int64_t t : level) {
            const SymFront& f = S.fronts[t];
            for (int64_t c = 0; c < f.nchild; c++) {
                auto& v = unodes[S.children[f.child_off + c]];
                v.clear();
                v.shrink_to_fit();
            }
        }
    }
    // rows in postorder: the DOFs of each later-row node, node after node
    int64_t total = 0;
    for (int64_t t = 0; t < nt; t++) {
        S.fronts[t].rows_off = total;
        total += S.fronts[t].u;
    }
    S.rows.resize(total);
    parallel_chunks(nt, 64, [&](int64_t a0, int64_t a1) {
        for (int64_t t = a0; t < a1; t++) {
            std::copy(rows_t[t].begin(), rows_t[t].end(), S.rows.begin() + S.fronts[t].rows_off);
            std::vector<int64_t>().swap(rows_t[t]);
        }
    });
    timer.lap("front patterns");
    return S;
}

void lower_pattern(const Symbolic& s, const Graph& g, std::vector<int64_t>& colptr, std::vector<int64_t>& rowidx) {
    colptr.assign(s.n + 1, 0);
    rowidx.clear();
    // columns of node v are contiguous and nodes appear in first_dof order within fronts
    std::vector<int64_t> order(g.nn);
    for (int64_t i = 0; i < g.nn; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return s.first_dof[a] < s.first_dof[b]; });
    std::vector<int64_t> nb;
    for (int64_t v : order) {
        nb.assign(g.adj_idx.begin() + g.adj_ptr[v], g.adj_idx.begin() + g.adj_ptr[v + 1]);
        nb.push_back(v);
        std::sort(nb.begin(), nb.end(), [&](int64_t a, int64_t b) { return s.first_dof[a] < s.first_dof[b]; });
        int64_t f = s.first_dof[v];
        for (int64_t c = f; c < f + g.ndof[v]; c++) {
            for (int64_t w : nb) {
                int64_t fw = s.first_dof[w];
                for (int64_t r = std::max(fw, c); r < fw + g.ndof[w]; r++) rowidx.push_back(r);
            }
            colptr[c + 1] = (int64_t)rowidx.size();
        }
    }
}

}  // namespace rfg

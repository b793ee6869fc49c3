"""Generates the golden fixtures of tests/golden/ (run from the repository root:
``python tests/golden/make_golden.py``).

1. known_answers.json — the reference's own known answers for this path:
   * the 40-DOF chain of ffi/src/lib.rs:429-478: tridiag(-1, 2-σ, -1) with σ = 1.3,
     whose inertia is the analytic count of 2 - 2cos(kπ/41) < σ; the positive
     definite factorization must refuse it; a chain whose DOF 7 is zero is singular
     with err_dof = 7;
   * the unsymmetric 40-DOF convection–diffusion chain of ffi/src/lib.rs:458-469:
     A(i, i) = 2, A(i, i−1) = −1.3, A(i, i+1) = −0.7, solved by the LU handle to a
     residual below 1e-10 per row; rustyfem_inertia returns −1 for it;
   * the 4×4 indefinite system of src/steps/nlgeom_solver.rs:145-175
     (2 negative eigenvalues, x = [1, -2, 0.5, 3]);
   * the shifted 7-point Laplacian of examples/solver_bench.rs:89-157 for small
     grids: σ and the analytic number of eigenvalues below σ;
   * front statistics of the 20³ C3D8 cube (n = 26,460): 287 fronts with leaf 48,
     614 with leaf 16, the flop estimate and nnz(L).
2. symbolic_<mesh>_leaf<L>.json — front lists (start, k, u, children), the
   equation of the first DOF of every node and the rows of every front, from
   the pure-Python restatement of src/sparse.rs:78-232 below. It is written
   from the reference's source independently of the C++ oracle and the C++
   product code; the coordinate sort (src/sparse.rs:108) is the restatement of
   Rust's slice::sort_unstable_by below, so equal coordinates end where the
   reference's sort leaves them.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


# ---------------------------------------------------------------------------
# Rust's `slice::sort_unstable_by` (core::slice::sort::unstable, "ipnsort", the
# standard library's unstable sort since Rust 1.81) for the element type the
# reference sorts at src/sparse.rs:108 (usize: 8 bytes, Copy), whose small sorts
# are the sorting-network variant. Restated from the algorithm's published
# description; the order it leaves equal keys in is the point. `lt(a, b)` is the
# caller's is_less on elements.

def _insert_from(v, lo, hi, start, lt):
    """insertion_sort_shift_left(v[lo:hi], start - lo): stable."""
    for i in range(max(start, lo + 1), hi):
        x = v[i]
        if not lt(x, v[i - 1]):
            continue
        j = i
        while j > lo and lt(x, v[j - 1]):
            v[j] = v[j - 1]
            j -= 1
        v[j] = x


# Optimal networks of 9 and 13 inputs (25 and 45 compare-exchanges), applied in
# this order; a pair (a, b) exchanges when v[b] < v[a].
NET9 = [(0, 3), (1, 7), (2, 5), (4, 8), (0, 7), (2, 4), (3, 8), (5, 6), (0, 2), (1, 3), (4, 5), (7, 8),
        (1, 4), (3, 6), (5, 7), (0, 1), (2, 4), (3, 5), (6, 8), (2, 3), (4, 5), (6, 7), (1, 2), (3, 4), (5, 6)]
NET13 = [(0, 12), (1, 10), (2, 9), (3, 7), (5, 11), (6, 8), (1, 6), (2, 3), (4, 11), (7, 9), (8, 10),
         (0, 4), (1, 2), (3, 6), (7, 8), (9, 10), (11, 12), (4, 6), (5, 9), (8, 11), (10, 12),
         (0, 5), (3, 8), (4, 7), (6, 11), (9, 10), (0, 1), (2, 5), (6, 9), (7, 8), (10, 11),
         (1, 3), (2, 4), (5, 6), (9, 10), (1, 2), (3, 4), (5, 7), (6, 8), (2, 3), (4, 5), (6, 7), (8, 9),
         (3, 4), (5, 6)]


def _network_region(v, lo, hi, lt):
    n = hi - lo
    net = NET13 if n >= 13 else NET9 if n >= 9 else []
    for a, b in net:
        if lt(v[lo + b], v[lo + a]):
            v[lo + a], v[lo + b] = v[lo + b], v[lo + a]
    _insert_from(v, lo, hi, lo + (13 if n >= 13 else 9 if n >= 9 else 1), lt)


def _small_sort(v, lo, hi, lt):
    """small_sort_network (at most 32 elements): below 18 one region, else the two
    halves sorted apart and merged (the bidirectional merge is the stable merge)."""
    n = hi - lo
    if n < 2:
        return
    if n < 18:
        _network_region(v, lo, hi, lt)
        return
    mid = lo + n // 2
    _network_region(v, lo, mid, lt)
    _network_region(v, mid, hi, lt)
    a, b = v[lo:mid], v[mid:hi]
    i = j = 0
    out = []
    while i < len(a) and j < len(b):
        if lt(b[j], a[i]):
            out.append(b[j])
            j += 1
        else:
            out.append(a[i])
            i += 1
    v[lo:hi] = out + a[i:] + b[j:]


def _heapsort(v, lo, hi, lt):
    n = hi - lo

    def sift(node, end):
        while True:
            c = 2 * node + 1
            if c >= end:
                return
            if c + 1 < end and lt(v[lo + c], v[lo + c + 1]):
                c += 1
            if not lt(v[lo + node], v[lo + c]):
                return
            v[lo + node], v[lo + c] = v[lo + c], v[lo + node]
            node = c

    for i in range(n + n // 2 - 1, -1, -1):
        if i >= n:
            sift(i - n, n)
        else:
            v[lo], v[lo + i] = v[lo + i], v[lo]
            sift(0, i)


def _median3(v, a, b, c, lt):
    x, y = lt(v[a], v[b]), lt(v[a], v[c])
    if x == y:
        return c if lt(v[b], v[c]) != x else b
    return a


def _median3_rec(v, a, b, c, m, lt):
    if m * 8 >= 64:
        m8 = m // 8
        a = _median3_rec(v, a, a + 4 * m8, a + 7 * m8, m8, lt)
        b = _median3_rec(v, b, b + 4 * m8, b + 7 * m8, m8, lt)
        c = _median3_rec(v, c, c + 4 * m8, c + 7 * m8, m8, lt)
    return _median3(v, a, b, c, lt)


def _choose_pivot(v, lo, hi, lt):
    n8 = (hi - lo) // 8
    a, b, c = lo, lo + 4 * n8, lo + 7 * n8
    return _median3(v, a, b, c, lt) if hi - lo < 64 else _median3_rec(v, a, b, c, n8, lt)


def _partition(v, lo, hi, p, lt):
    """Pivot to the front, cyclic branchless Lomuto over the rest (each element in
    turn goes to the end of the `lt` block, the element it displaces into the hole
    it left, the first element last), pivot between the blocks."""
    v[lo], v[p] = v[p], v[lo]
    piv = v[lo]
    w0 = lo + 1
    m = hi - w0
    if m == 0:
        return 0
    saved = v[w0]
    hole = w0
    nlt = 0
    for r in range(w0 + 1, hi + 1):
        x = saved if r == hi else v[r]
        is_lt = lt(x, piv)
        v[hole] = v[w0 + nlt]
        v[w0 + nlt] = x
        hole = r
        nlt += is_lt
    v[lo], v[lo + nlt] = v[lo + nlt], v[lo]
    return nlt


def _quicksort(v, lo, hi, anc, limit, lt):
    while True:
        if hi - lo <= 32:
            _small_sort(v, lo, hi, lt)
            return
        if limit == 0:
            _heapsort(v, lo, hi, lt)
            return
        limit -= 1
        p = _choose_pivot(v, lo, hi, lt)
        if anc is not None and not lt(anc, v[p]):
            nle = _partition(v, lo, hi, p, lambda a, b: not lt(b, a))
            lo += nle + 1
            anc = None
            continue
        nlt = _partition(v, lo, hi, p, lt)
        _quicksort(v, lo, lo + nlt, anc, limit, lt)
        anc = v[lo + nlt]
        lo += nlt + 1


def sort_unstable(v, lt, limit=None):
    """In place, as `v.sort_unstable_by(..)` with is_less = lt. `limit` overrides the
    quicksort's imbalance budget 2·⌊log2(n | 1)⌋ (0 sends a slice of more than 32
    elements straight to the heapsort)."""
    n = len(v)
    if n < 2:
        return
    if n <= 20:
        _insert_from(v, 0, n, 1, lt)
        return
    desc = lt(v[1], v[0])
    run = 2
    while run < n and (lt(v[run], v[run - 1]) if desc else not lt(v[run], v[run - 1])):
        run += 1
    if run == n:
        if desc:
            v.reverse()
        return
    _quicksort(v, 0, n, None, 2 * ((n | 1).bit_length() - 1) if limit is None else limit, lt)


def dissect(nodes, coords, adj, side, tree, leaf_max):
    """src/sparse.rs:78-157."""
    if not nodes:
        return None
    if len(nodes) <= leaf_max:
        tree.append({"nodes": list(nodes), "children": []})
        return len(tree) - 1
    lo = [min(coords[v][a] for v in nodes) for a in range(3)]
    hi = [max(coords[v][a] for v in nodes) for a in range(3)]
    axes = sorted(range(3), key=lambda a: -(hi[a] - lo[a]))  # stable: ties keep 0, 1, 2
    n = len(nodes)
    s = list(nodes)
    best = None
    for ax in axes:
        if not hi[ax] > lo[ax]:
            continue
        sort_unstable(s, lambda p, q, ax=ax: coords[p][ax] < coords[q][ax])  # :108
        for q in (n // 2, 2 * n // 5, 3 * n // 5):
            t = coords[s[q]][ax]
            nl = sum(1 for v in s if coords[v][ax] < t)
            if nl == 0 or nl == n:
                continue
            for i, v in enumerate(s):
                side[v] = 1 if i >= nl else 0
            sep_l = sum(1 for v in s[:nl] if any(side[w] == 1 for w in adj[v]))
            sep_r = sum(1 for v in s[nl:] if any(side[w] == 0 for w in adj[v]))
            sz, in_left = (sep_r, False) if sep_r < sep_l else (sep_l, True)
            score = sz / (min(nl, n - nl) / n)
            if best is None or score < best[0]:
                best = (score, ax, t, in_left)
    if best is not None:
        _, ax, t, in_left = best
        left = [v for v in s if coords[v][ax] < t]
        right = [v for v in s if not coords[v][ax] < t]
    else:
        in_left = True
        left, right = s[: n // 2], s[n // 2:]
    for v in left:
        side[v] = 0
    for v in right:
        side[v] = 1
    if in_left:
        sep = [v for v in left if any(side[w] == 1 for w in adj[v])]
        a = [v for v in left if not any(side[w] == 1 for w in adj[v])]
        b = right
    else:
        sep = [v for v in right if any(side[w] == 0 for w in adj[v])]
        a = left
        b = [v for v in right if not any(side[w] == 0 for w in adj[v])]
    for v in left + right:
        side[v] = 2
    children = [c for c in (dissect(a, coords, adj, side, tree, leaf_max), dissect(b, coords, adj, side, tree, leaf_max))
                if c is not None]
    tree.append({"nodes": sep, "children": children})
    return len(tree) - 1


def analyse(coords, adj, ndof, leaf_max):
    """src/sparse.rs:167-232."""
    sys.setrecursionlimit(10000)
    nn = len(coords)
    tree = []
    side = [2] * nn
    root = dissect(list(range(nn)), coords, adj, side, tree, max(leaf_max, 1))
    post = []
    stack = [(root, False)] if root is not None else []
    while stack:
        t, done = stack.pop()
        if done:
            post.append(t)
        else:
            stack.append((t, True))
            for c in reversed(tree[t]["children"]):
                stack.append((c, False))
    first = [0] * nn
    nxt = 0
    for t in post:
        tree[t]["start"] = nxt
        for v in tree[t]["nodes"]:
            first[v] = nxt
            nxt += ndof[v]
        tree[t]["k"] = nxt - tree[t]["start"]
    unodes = {}
    for t in post:
        end = tree[t]["start"] + tree[t]["k"]
        seen = set()
        lst = []
        for v in tree[t]["nodes"]:
            for w in adj[v]:
                if first[w] >= end and w not in seen:
                    seen.add(w)
                    lst.append(w)
        for c in tree[t]["children"]:
            for w in unodes[c]:
                if first[w] >= end and w not in seen:
                    seen.add(w)
                    lst.append(w)
        lst.sort(key=lambda w: first[w])
        tree[t]["rows"] = [q for w in lst for q in range(first[w], first[w] + ndof[w])]
        k, u = float(tree[t]["k"]), float(len(tree[t]["rows"]))
        tree[t]["work"] = k * k * k / 3.0 + u * k * k + u * u * k + sum(tree[c]["work"] for c in tree[t]["children"])
        unodes[t] = lst
    return tree, first, nxt


def graph_lists(graph):
    coords = [tuple(map(float, c)) for c in graph.coords]
    adj = [list(map(int, graph.adj_idx[graph.adj_ptr[i]:graph.adj_ptr[i + 1]])) for i in range(len(graph.ndof))]
    return coords, adj, [int(x) for x in graph.ndof]


def symbolic_fixture(name, graph, leaf):
    coords, adj, ndof = graph_lists(graph)
    tree, first, n = analyse(coords, adj, ndof, leaf)
    fronts = [[t["start"], t["k"], len(t["rows"]), len(t["children"])] for t in tree]
    work = tree[-1]["work"] if tree else 0.0  # the root is pushed last
    return {
        "mesh": name, "leaf": leaf, "n": n, "fronts": fronts, "first_dof": first,
        "rows": [q for t in tree for q in t["rows"]],
        "children": [c for t in tree for c in t["children"]],
        "work": work,
        "factor_size": sum(t["k"] * max(t["k"] - 1, 0) // 2 + t["k"] * len(t["rows"]) for t in tree),
    }


def known_answers():
    n, sigma = 40, 1.3
    below = sum(1 for k in range(1, n + 1) if 2.0 - 2.0 * math.cos(k * math.pi / (n + 1)) < sigma)
    from rustyfem_b200 import workloads as W

    lap = []
    for g in (6, 8, 10):
        s = W.laplace_sigma(g)
        _, cnt = W.laplace3d(g, s)
        lap.append({"g": g, "sigma": s, "below": cnt})
    return {
        "chain": {"n": n, "sigma": sigma, "inertia": [below, 0, n - below], "pd_refuses": True,
                  "singular_dof": 7, "residual_tol": 1e-10},
        "lu_chain": {"n": n, "diag": 2.0, "sub": -1.3, "sup": -0.7, "residual_tol": 1e-10, "inertia_rc": -1},
        "dual4": {"a": [[2.0, 1.0, 0.0, 0.0], [1.0, -3.0, 1.0, 0.0], [0.0, 1.0, 1.0, 2.0], [0.0, 0.0, 2.0, 1.0]],
                  "x": [1.0, -2.0, 0.5, 3.0], "negative": 2, "tol": 1e-12},
        "laplace": lap,
        "cube20": {"n": 26460, "fronts_leaf48": 287, "fronts_leaf16": 614, "work_leaf48": 1.302e10,
                   "factor_size_leaf48": 1.52e7, "largest_front": [660, 1260]},
        "cube60": {"n": 669780, "fronts_leaf48": 6245, "work_leaf48": 8.729e12, "factor_size_leaf48": 1.31e9,
                   "largest_front": [5580, 10980]},
    }


def main():
    from rustyfem_b200 import workloads as W

    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known_answers(), f, indent=1)
    meshes = [("hex8_6", W.hex8_cube(6).graph), ("plate_40x4", W.plate(40, 4).graph),
              ("hex20_2", W.hex20_cube(2).graph)]
    for name, g in meshes:
        for leaf in (48, 16):
            fx = symbolic_fixture(name, g, leaf)
            with open(os.path.join(HERE, f"symbolic_{name}_leaf{leaf}.json"), "w") as f:
                json.dump(fx, f)
    print("written to", HERE)


if __name__ == "__main__":
    main()

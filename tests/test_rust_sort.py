"""The coordinate sort of the dissection (src/sparse.rs:108, `set.sort_unstable_by`).

Rust's `slice::sort_unstable_by` is ipnsort (core::slice::sort::unstable, Rust 1.81
and later); where it leaves equal coordinates is the node order inside the fronts.
Three restatements of it are checked here: the golden generator's (Python), the
oracle's and the product's (C++, through rfg_selftest_sort_unstable).

* Hand-traced tie cases, one per branch of the algorithm: insertion sort (n <= 20),
  the 9- and 13-input networks of the small sort with its stable merge of two halves,
  a cyclic Lomuto partition, the heapsort.
* The networks sort every 0/1 input (0-1 principle).
* The three agree element for element on seeded inputs with many ties, presorted and
  reversed runs, and forced heapsorts.
"""
import os
import sys

import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_golden as G  # noqa: E402


def py_sort(keys, limit=None):
    v = [(int(k), i) for i, k in enumerate(keys)]
    G.sort_unstable(v, lambda a, b: a[0] < b[0], limit)
    return [i for _, i in v]


def all_three(keys, limit=-1):
    a = py_sort(keys, None if limit < 0 else limit)
    b = refcpu.sort_unstable_keys(keys, limit).tolist()
    c = ffi.sort_unstable_keys(keys, limit).tolist()
    return a, b, c


def _ones(n, zeros):
    k = [1] * n
    for z in zeros:
        k[z] = 0
    return k


# (keys, order the sort leaves them in), traced by hand from the algorithm:
HAND = [
    # n <= 20: insertion sort, stable
    ([1, 0, 1, 0, 0], [1, 3, 4, 0, 2]),
    # n = 21: no whole run (key 0 at 3), quicksort of <= 32 elements = small sort: halves of
    # 10 and 11; the 9-network's first exchange (0, 3) moves key 0 to the front and id 0 to
    # slot 3, no later exchange fires; the stable merge keeps the rest in place
    (_ones(21, [3]), [3, 1, 2, 0] + list(range(4, 21))),
    # n = 30: halves of 15; the 13-network's first exchange (0, 12) swaps ids 0 and 12
    (_ones(30, [12]), [12] + list(range(1, 12)) + [0] + list(range(13, 30))),
    # n = 33: pivot = median of ids 0, 16, 28 = id 16 (key 1), swapped to the front (id 0 to
    # slot 16); the cyclic Lomuto over slots 1..32 (zeros at ids 3, 10, 28) leaves
    # [3, 10, 28, 1, 5..9, 2, 11..15, 0, 17..27, 4, 29..32], the pivot swaps with the last
    # lesser element (id 28); both sides are all-equal small sorts and stay put
    (_ones(33, [3, 10, 28]),
     [28, 3, 10, 16, 1, 5, 6, 7, 8, 9, 2, 11, 12, 13, 14, 15, 0] + list(range(17, 28)) + [4, 29, 30, 31, 32]),
    # strictly descending whole run: reversed
    (list(range(24, -1, -1)), list(range(24, -1, -1))),
    # non-descending whole run with ties: untouched
    ([0] * 10 + [1] * 15, list(range(25))),
]


@pytest.mark.parametrize("case", range(len(HAND)))
def test_hand_traced_tie_cases(case):
    keys, want = HAND[case]
    a, b, c = all_three(keys)
    assert a == want and b == want and c == want, (a, b, c)


def test_hand_traced_heapsort():
    # heapsort of keys [1, 1, 0, 1]: build (no exchange), then 0↔3, 0↔2 and a sift of id 2
    # over id 1, then 0↔1: [2, 1, 3, 0] (a stable sort gives [2, 0, 1, 3])
    v = [(1, 0), (1, 1), (0, 2), (1, 3)]
    G._heapsort(v, 0, 4, lambda a, b: a[0] < b[0])
    assert [i for _, i in v] == [2, 1, 3, 0]
    # through the sort with the imbalance budget at 0 (more than 32 elements: heapsort)
    keys = [(7 * i) % 5 for i in range(40)]
    a, b, c = all_three(keys, limit=0)
    v = [(k, i) for i, k in enumerate(keys)]
    G._heapsort(v, 0, 40, lambda p, q: p[0] < q[0])
    assert a == b == c == [i for _, i in v]


@pytest.mark.parametrize("net,n", [(G.NET9, 9), (G.NET13, 13)])
def test_networks_sort_every_01_input(net, n):
    for bits in range(1 << n):
        v = [(bits >> i) & 1 for i in range(n)]
        for a, b in net:
            if v[b] < v[a]:
                v[a], v[b] = v[b], v[a]
        assert v == sorted(v), (n, bits)


def test_three_restatements_agree():
    rng = np.random.default_rng(108)
    for t in range(600):
        n = int(rng.integers(0, 700))
        kind = t % 6
        if kind == 0:
            keys = rng.integers(0, 3, n)
        elif kind == 1:
            keys = rng.integers(0, 1 << 31, n)
        elif kind == 2:
            keys = np.sort(rng.integers(0, 8, n))  # a run broken in three places
            if n:
                keys[rng.integers(0, n, 3)] = 0
        elif kind == 3:
            keys = np.sort(rng.integers(0, 8, n))[::-1].copy()
        elif kind == 4:
            keys = np.repeat(rng.integers(0, 50, max(n // 7, 1)), 7)[:n]
        else:
            keys = rng.integers(0, 20, n)
        limit = [-1, -1, 0, 1, 3][t % 5]
        a, b, c = all_three(keys, limit)
        assert a == b == c, (t, n, kind, limit)
        assert np.all(np.diff(np.asarray(keys)[a]) >= 0)


def test_oracle_and_product_agree_on_large_inputs():
    rng = np.random.default_rng(7)
    for n, m in ((100_000, 64), (300_000, 3), (200_000, 1 << 30)):
        keys = rng.integers(0, m, n)
        b = refcpu.sort_unstable_keys(keys)
        c = ffi.sort_unstable_keys(keys)
        assert np.array_equal(b, c), (n, m)
        assert np.all(np.diff(keys[c]) >= 0)

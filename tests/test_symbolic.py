"""The product's host symbolic stage (librustyfem_gpu.so, rfg_sym_*) against the
oracle and the golden fixtures: the front list, equation numbering, front rows,
children, flop estimate, factor size and lower pattern must be identical."""
import json
import os

import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def same(p, o):
    assert p.n == o.n
    assert np.array_equal(p.fronts(), o.fronts())
    assert np.array_equal(p.first_dof(), o.first_dof())
    assert np.array_equal(p.rows(), o.rows())
    assert np.array_equal(p.children(), o.children())
    assert p.work() == o.work()
    assert p.factor_size() == o.factor_size()
    pc, pr = p.pattern()
    oc, orr = o.pattern()
    assert np.array_equal(pc, oc) and np.array_equal(pr, orr)


MESHES = {
    "hex8_5": lambda: W.hex8_cube(5),
    "hex8_20": lambda: W.hex8_cube(20),
    "hex8_18_emod": lambda: W.hex8_cube(18, emod=W.log_uniform_moduli(18)),
    "plate_200x20": lambda: W.plate(200, 20),
    "plate_23x2": lambda: W.plate(23, 2),
    "hex20_4": lambda: W.hex20_cube(4),
}


@pytest.mark.parametrize("mesh", list(MESHES))
@pytest.mark.parametrize("leaf", [48, 16, 1])
def test_product_symbolic_equals_oracle(mesh, leaf):
    m = MESHES[mesh]()
    same(ffi.Symbolic(m.graph, leaf), refcpu.Symbolic(m.graph, leaf))


def test_product_symbolic_60cube():
    """The 60³ C3D8 cube (n = 669,780) of the large benchmark configurations; the
    parallel dissection must give the same tree as the serial oracle."""
    m = W.hex8_cube(60)
    k = json.load(open(os.path.join(GOLD, "known_answers.json")))["cube60"]
    p = ffi.Symbolic(m.graph, 48)
    o = refcpu.Symbolic(m.graph, 48)
    assert p.n == k["n"] and p.nfronts == k["fronts_leaf48"]
    assert abs(p.work() / k["work_leaf48"] - 1) < 1e-3
    assert np.array_equal(p.fronts(), o.fronts())
    assert np.array_equal(p.first_dof(), o.first_dof())
    assert np.array_equal(p.rows(), o.rows())


@pytest.mark.parametrize("name", ["hex8_6", "plate_40x4", "hex20_2"])
@pytest.mark.parametrize("leaf", [48, 16])
def test_product_symbolic_matches_golden(name, leaf):
    with open(os.path.join(GOLD, f"symbolic_{name}_leaf{leaf}.json")) as f:
        g = json.load(f)
    mesh = {"hex8_6": lambda: W.hex8_cube(6), "plate_40x4": lambda: W.plate(40, 4),
            "hex20_2": lambda: W.hex20_cube(2)}[name]()
    s = ffi.Symbolic(mesh.graph, leaf)
    assert s.fronts().tolist() == g["fronts"]
    assert s.first_dof().tolist() == g["first_dof"]
    assert s.rows().tolist() == g["rows"]
    assert s.children().tolist() == g["children"]
    assert s.work() == g["work"]


def test_plan_is_consistent():
    """Plan figures: every level has fronts, the update arena reuses memory."""
    m = W.hex8_cube(20)
    s = ffi.Symbolic(m.graph, 48)
    st = s.plan_stats()
    f = s.fronts()
    assert st["levels"] >= 1 and st["steps"] >= st["levels"]
    no_reuse = int(np.sum(f[:, 2] * ((f[:, 2] + 7) // 8 * 8)))
    assert 0 < st["update_elems"] <= no_reuse


def test_disconnected_graph():
    """Two separate plates in one graph: an empty separator gives a front with k = 0."""
    a = W.plate(10, 2).graph
    nb = len(a.ndof)
    coords = np.vstack([a.coords, a.coords + np.array([1.0, 0.0, 0.0])])
    adj_ptr = np.concatenate([a.adj_ptr, a.adj_ptr[1:] + a.adj_ptr[-1]])
    adj_idx = np.concatenate([a.adj_idx, a.adj_idx + nb])
    g = W.Graph(coords, adj_ptr, adj_idx, np.concatenate([a.ndof, a.ndof]))
    for leaf in (48, 4):
        same(ffi.Symbolic(g, leaf), refcpu.Symbolic(g, leaf))


def test_host_block_cache_reuse():
    """Large host scratch arrays come from a cache of freed blocks that are handed out again
    without being cleared: analyses of other meshes in between, and a release of the cache,
    leave the result of a repeated analysis unchanged."""
    a = MESHES["hex8_20"]()
    first = ffi.Symbolic(a.graph, 16)
    for step in range(3):
        ffi.Symbolic(MESHES["plate_200x20"]().graph, 16 if step else 1)
        if step == 1:
            ffi.lib().rfg_release_cached_memory()
        again = ffi.Symbolic(a.graph, 16)
        same(again, first)

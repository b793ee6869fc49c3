"""The oracle's restatement of the tangent assembly (src/fem/assembly.rs:315-420) and of the
C3D8 element matrix (src/elements/continuum3d.rs:39-131) on the CPU: against the workload
generator's independent restatement (unit stiffness scaled by E), rigid-body modes, and a
plain-Python replay of the element loop."""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import workloads as W


def rigid_modes(x):
    """Six rigid-body displacement fields of the 8 nodes (24-vectors)."""
    modes = []
    for d in range(3):
        u = np.zeros((8, 3))
        u[:, d] = 1.0
        modes.append(u.ravel())
    for a, b in ((0, 1), (0, 2), (1, 2)):
        u = np.zeros((8, 3))
        u[:, a] = -x[:, b]
        u[:, b] = x[:, a]
        modes.append(u.ravel())
    return np.array(modes)


def test_ke_hex8_symmetric_and_rigid_modes():
    x = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    x = x * [0.3, 0.5, 0.7] + [[0.01 * i, -0.02 * i, 0.015 * i] for i in range(8)]  # a distorted brick
    ke = refcpu.ke_hex8(x, 210e9, 0.3)
    s = np.max(np.abs(ke))
    assert np.max(np.abs(ke - ke.T)) <= 1e-14 * s
    assert np.max(np.abs(ke @ rigid_modes(x).T)) <= 1e-12 * s
    w = np.linalg.eigvalsh(0.5 * (ke + ke.T))
    assert np.sum(w > 1e-10 * s) == 18  # 24 DOFs − 6 rigid modes


def test_ke_hex8_distorted_element_is_refused():
    x = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    with pytest.raises(ValueError):
        refcpu.ke_hex8(x[[1, 0, 2, 3, 4, 5, 6, 7]], 1.0, 0.3)  # two corners swapped: det J < 0


@pytest.mark.parametrize("emod", [None, "log"])
def test_assembly_matches_the_generator(emod):
    """The oracle's element loop (E inside D) against the generator's K (unit matrix × E): the
    same operator to rounding."""
    n = 5
    E = W.log_uniform_moduli(n, seed=3) if emod else None
    m = W.hex8_cube(n, emod=E)
    me = W.hex8_mesh(n, emod=E)
    assert np.array_equal(m.coords.reshape(-1, 3), me.xyz)
    sym = refcpu.Symbolic(m.graph, 48)
    colptr, rowidx, val, eq = refcpu.to_internal(m, sym)
    v = refcpu.assemble_hex8(colptr, rowidx, me.conn, me.xyz, me.emod, me.nu, me.edof(sym.first_dof()))
    scale = np.abs(val).max()
    # (entries that cancel to rounding level, ~1e-17 of the scale, may differ in sign or vanish)
    assert np.max(np.abs(v - val)) <= 2e-15 * scale


def _replay(colptr, rowidx, edof, ke):
    """src/fem/assembly.rs:388-412 in plain Python: zero, then element by element."""
    val = np.zeros(int(colptr[-1]))
    nelem, nd = edof.shape
    for e in range(nelem):
        for a in range(nd):
            ia = edof[e, a]
            if ia < 0:
                continue
            for b in range(nd):
                ib = edof[e, b]
                if ib < 0 or ia < ib:
                    continue
                v = 0.5 * (ke[e, a, b] + ke[e, b, a])
                if v != 0.0:
                    lo, hi = colptr[ib], colptr[ib + 1]
                    p = lo + int(np.searchsorted(rowidx[lo:hi], ia))
                    assert rowidx[p] == ia
                    val[p] += v
    return val


def test_assemble_generic_matches_a_replay_bit_for_bit():
    """Unsymmetric element matrices (the symmetric part goes in), zeros and constrained DOFs."""
    n = 3
    m = W.hex8_cube(n)
    me = W.hex8_mesh(n)
    sym = refcpu.Symbolic(m.graph, 48)
    colptr, rowidx = sym.pattern()
    edof = me.edof(sym.first_dof())
    rng = np.random.default_rng(7)
    ke = rng.standard_normal((len(edof), 24, 24))
    ke[:, 3, 5] = 0.0
    ke[:, 5, 3] = 0.0
    val = refcpu.assemble(colptr, rowidx, edof, ke)
    assert np.array_equal(val, _replay(colptr, rowidx, edof, ke))


def test_assemble_reports_a_missing_entry():
    n = 2
    m = W.hex8_cube(n)
    me = W.hex8_mesh(n)
    sym = refcpu.Symbolic(m.graph, 48)
    colptr, rowidx = sym.pattern()
    edof = me.edof(sym.first_dof()).copy()
    # element 0 (at the origin) coupled to a DOF of the far corner node: not in the pattern
    far = sym.first_dof()[me.block[len(me.xyz) - 1]]
    edof[0, np.argmax(edof[0] >= 0)] = far
    with pytest.raises(KeyError):
        refcpu.assemble(colptr, rowidx, edof, np.ones((len(edof), 24, 24)))

"""Assembly of K on the GPU (rfg_assembly_*, the element loop of src/fem/assembly.rs:315-420)
against the oracle's restatement: the values bit for bit (element matrices computed on the
device, or given from the host or the device), then factor and solve from the device values."""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import solver, workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def setup(n, emod=None, precision="direct-gpu"):
    m = W.hex8_cube(n, emod=emod)
    me = W.hex8_mesh(n, emod=emod)
    sm = solver.select(precision).prepare(m.graph)
    sym = refcpu.Symbolic(m.graph, 48)
    assert np.array_equal(sm.first_dof(), sym.first_dof())
    colptr, rowidx = sym.pattern()
    return m, me, sm, sym, colptr, rowidx, me.edof(sm.first_dof())


@pytest.mark.parametrize("n,emod", [(6, None), (14, None), (12, "log")])
def test_hex8_elements_on_the_device_match_the_oracle_bit_for_bit(gpu, n, emod):
    E = W.log_uniform_moduli(n, seed=1) if emod else None
    m, me, sm, sym, colptr, rowidx, edof = setup(n, E)
    asm = sm.assembly(edof)
    asm.hex8(me.xyz, me.conn, me.emod, me.nu)
    v = sm.values()
    vo = refcpu.assemble_hex8(colptr, rowidx, me.conn, me.xyz, me.emod, me.nu, edof)
    assert np.array_equal(v, vo)
    t_el, t_ga = asm.times()
    assert t_el > 0 and t_ga > 0


def test_element_matrices_from_host_and_device(gpu):
    """Unsymmetric element matrices with zeros (the symmetric part is assembled, zero terms
    skipped), and a clamped face (-1 equations): bit for bit against the oracle."""
    import torch
    m, me, sm, sym, colptr, rowidx, edof = setup(5)
    rng = np.random.default_rng(11)
    ke = rng.standard_normal((len(edof), 24, 24))
    ke[:, 0, 7] = 0.0
    ke[:, 7, 0] = 0.0
    vo = refcpu.assemble(colptr, rowidx, edof, ke)
    asm = sm.assembly(edof)
    asm.set(ke)
    assert np.array_equal(sm.values(), vo)
    sm.zero()
    assert not sm.values().any()
    dke = torch.from_numpy(ke).cuda()
    asm.set_device(dke.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(sm.values(), vo)
    assert asm.contributions() == int(np.sum((edof[:, :, None] >= 0) & (edof[:, None, :] >= 0) &
                                             (edof[:, :, None] >= edof[:, None, :])))


@pytest.mark.parametrize("precision", ["direct-gpu", "direct-gpu-mixed"])
def test_factor_and_solve_from_device_values(gpu, precision):
    """zero → assemble on the device → factor → solve equals the same matrix added from the host,
    and the FP64 solution matches the oracle's."""
    n = 10
    m, me, sm, sym, colptr, rowidx, edof = setup(n, precision=precision)
    asm = sm.assembly(edof)
    asm.hex8(me.xyz, me.conn, me.emod, me.nu)
    vals = sm.values()
    sm.factor()
    b = np.zeros(sm.n())
    _, _, _, eq = refcpu.to_internal(m, sym)
    b[eq] = m.rhs
    x = b.copy()
    sm.solve(x)
    sm2 = solver.select(precision).prepare(m.graph)
    cols = np.repeat(np.arange(sm2.n()), np.diff(colptr))
    sm2.add_many(rowidx, cols, vals)
    sm2.factor()
    x2 = b.copy()
    sm2.solve(x2)
    assert np.array_equal(x, x2)
    F, e = sym.pd_factor(colptr, rowidx, vals)
    assert e == -1
    assert rel(x, F.solve(b)) <= (1e-10 if precision == "direct-gpu" else 1e-9)


def test_host_adds_after_a_device_assembly(gpu):
    """SystemMatrix::add after the device assembly adds to the assembled values (they are
    copied down first); zero clears them."""
    m, me, sm, sym, colptr, rowidx, edof = setup(4)
    asm = sm.assembly(edof)
    asm.hex8(me.xyz, me.conn, me.emod, me.nu)
    v = sm.values()
    sm.add(int(rowidx[colptr[3]]), 3, 2.5)
    v2 = sm.values()
    assert v2[colptr[3]] == v[colptr[3]] + 2.5
    assert np.array_equal(np.delete(v2, colptr[3]), np.delete(v, colptr[3]))


def test_missing_pattern_entry_and_distorted_element(gpu):
    m, me, sm, sym, colptr, rowidx, edof = setup(3)
    # element 0 (at the origin) coupled to a DOF of the far corner node: not in the pattern
    bad = edof.copy()
    far = sm.first_dof()[me.block[len(me.xyz) - 1]]
    bad[0, np.argmax(bad[0] >= 0)] = far
    with pytest.raises(KeyError, match="missing in the pattern"):
        sm.assembly(bad)
    asm = sm.assembly(edof)
    conn = me.conn.copy()
    conn[4, [0, 1]] = conn[4, [1, 0]]  # two corners swapped: det J < 0
    with pytest.raises(ValueError, match="element 4"):
        asm.hex8(me.xyz, conn, me.emod, me.nu)


def test_empty_element_set(gpu):
    m, me, sm, sym, colptr, rowidx, edof = setup(2)
    asm = sm.assembly(edof[:0])
    asm.set(np.zeros((0, 24, 24)))
    assert asm.contributions() == 0
    assert not sm.values().any()

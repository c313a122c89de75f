"""Harmonic-balance assembly on the GPU against the oracle restatement (which is itself
pinned to the reference gateway on linear materials, tests/test_oracle.py)."""
import numpy as np
import pytest
import torch
from conftest import bits_equal

from magpackage_b200 import material, quadrature, synth
from magpackage_b200.hbfem import AFT, assemble_hbfem
from magpackage_b200.plan import AssemblyPlan
from oracle.oracle import mex_inputs

pytestmark = pytest.mark.gpu


def _case(port, harmonics, n=(5, 4, 3), seed=12, scale=1.0, imag=True):
    mesh = synth.kuhn_box(*n, seed=seed)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = port.generate_edges(mesh.T)
    E = edges.shape[0]
    m = mex_inputs(mesh.P, mesh.T, t2e, sign, tags)
    pk = material.pack_material_data(synth.standard_materials())
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    plan.set_materials(pk)
    rng = np.random.default_rng(seed)
    K = len(harmonics)
    # a spread of magnitudes drives the iron through the spline's interior, knee and extrapolation
    amp = scale * np.exp(rng.uniform(-4, 1, (E, K)))
    sol = amp * rng.normal(0, 1, (E, K)) + (1j * amp * rng.normal(0, 1, (E, K)) if imag else 0.0)
    return plan, m, pk, sol, E


@pytest.mark.parametrize("harmonics,imag", [((0, 1, 3), True), ((1, 3, 5, 7), True), ((0, 1), False), ((1,), True),
                                            ((1, 3, 5, 7, 9), True)])
def test_hbfem_matches_oracle(oracle_port, harmonics, imag):
    plan, m, pk, sol, E = _case(oracle_port, harmonics, imag=imag)
    aft = AFT(harmonics)
    qw, val, curl = quadrature.reference_data(2)
    K = len(harmonics)
    I, J, V, Rr, Rc, Rre, Rim = oracle_port.hbfem(m, sol, aft.D, aft.P, qw, curl, pk, True)
    R, vals = assemble_hbfem(plan, sol, aft, True)
    R = R.cpu().numpy()
    # residual: sparse(R_rows, R_cols, R_val, Ndof, K), summed in order of appearance
    lin = Rr + (Rc - 1) * E
    ref_re = oracle_port.sparse_vec(lin, Rre, E * K).reshape(K, E)
    ref_im = oracle_port.sparse_vec(lin, Rim, E * K).reshape(K, E)
    assert bits_equal(np.real(R), ref_re)
    assert bits_equal(np.imag(R), ref_im)
    assert np.abs(ref_re).max() > 0 and np.abs(ref_im).max() > 0
    # Jacobian: the first harmonic's block (scaling 1) on the structural pattern
    first = I <= E
    rp, ci, rv = oracle_port.sparse_csr(I[first], J[first], V[first], E, drop_zeros=False)
    assert np.array_equal(plan.row_ptr.cpu().numpy(), rp)
    assert np.array_equal(plan.col_idx.cpu().numpy(), ci)
    assert bits_equal(vals.cpu().numpy(), rv)


def test_hbfem_residual_only_and_errors(oracle_port):
    plan, m, pk, sol, E = _case(oracle_port, (1, 3))
    aft = AFT((1, 3))
    R1, v1 = assemble_hbfem(plan, sol, aft, True)
    R0, v0 = assemble_hbfem(plan, sol, aft, False)
    assert v0 is None and torch.equal(R0, R1)
    from magpackage_b200 import _lib
    with pytest.raises(_lib.MagError):
        assemble_hbfem(plan, np.zeros((E, 17)), AFT(list(range(17))), False)  # more than 16 harmonics


def test_hbfem_device_resident_field_gives_the_same_bits(oracle_port):
    """A complex CUDA tensor or a (re, im) pair already in [K, Ndof] layout is used without
    a host round trip and gives the host array's result."""
    plan, m, pk, sol, E = _case(oracle_port, (0, 1, 3))
    aft = AFT((0, 1, 3))
    R0, v0 = assemble_hbfem(plan, sol, aft, True)
    R1, v1 = assemble_hbfem(plan, torch.as_tensor(sol, device="cuda"), aft, True)
    pair = (torch.as_tensor(np.ascontiguousarray(sol.real.T), device="cuda"),
            torch.as_tensor(np.ascontiguousarray(sol.imag.T), device="cuda"))
    R2, v2 = assemble_hbfem(plan, pair, aft, True)
    for R, v in ((R1, v1), (R2, v2)):
        assert torch.equal(R, R0) and torch.equal(v, v0)
    with pytest.raises(ValueError):
        assemble_hbfem(plan, pair[0][:2], aft, False)
